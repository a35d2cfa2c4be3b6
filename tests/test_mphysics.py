"""The reference-named MPhysicsAPI exports (MPhysics/MPhysics.h:14-104) served
by libhfgrid.so: JSON scene loading, stepping and the Euler-particle / fluid
SDF copies, driven through ctypes the way the reference's host binds its DLL.

The CPU tests cover the loader's error paths (they fail before any device
work); the GPU tests check a loaded dam-break scene against the oracle stepped
from the same boundaries, fluid domain and seeded particles.
"""
import ctypes as C
import json

import numpy as np
import pytest

import hfgrid
import oracle

PF = C.POINTER(C.c_float)
RF = C.POINTER(C.c_float)


def mp():
    L = hfgrid.lib()
    L.mphysics_last_error.restype = C.c_char_p
    L.mphysics_grid_solver.restype = C.c_void_p
    L.mphysics_grid_solver.argtypes = [C.c_char_p]
    L.loadScene.argtypes = [C.c_char_p]
    L.update.argtypes = [C.c_float]
    L.getEulerParticleSize.restype = C.c_uint
    L.getEulerParticleSize.argtypes = [C.c_char_p]
    L.getParticleSize.restype = C.c_uint
    L.getParticleSize.argtypes = [C.c_char_p]
    for f in ("copyEulerParticlesPosToCPU", "copyEulerParticlesVelToCPU", "copyFluidSDFToCPU", "copyPositionToCPU"):
        getattr(L, f).argtypes = [C.c_char_p, PF]
    L.copyFluidSDFGradientToCPU.argtypes = [C.c_char_p, PF, PF, PF]
    L.getEulerGridInfo.argtypes = [C.c_char_p] + [RF] * 6
    return L


def err(L):
    return L.mphysics_last_error().decode()


def scene_json(name="Water", res=(14, 12, 10), kind="MixPICAndFLIP", seed=3):
    """A dam break in the reference's scene format (SceneManager.cpp:6-47,
    GridFluidSolver.cpp:43-159)."""
    return json.dumps({"HybridSimulator": [{
        "Name": name,
        "GridSolver": {
            "GridResolution": {"x": res[0], "y": res[1], "z": res[2]},
            "SimulationDomain": {"Start": {"x": 0, "y": 0, "z": 0}, "End": {"x": 1.4, "y": 1.2, "z": 1.0}},
            "DeltaT": 0.02,
            "Solids": [{"Type": "Walls"}],
            "EulerFluidDomain": [{"Range": {"Start": {"x": 0.05, "y": 0.05, "z": 0.05},
                                            "End": {"x": 0.6, "y": 0.7, "z": 0.95}}}],
            "PressureSolver": {"Preconditioner": "jacobi", "ToleranceMode": "relative", "Tolerance": 1e-6,
                               "MaxIterations": 400},
            "AdvectionSolver": {"Type": kind, "NumOfParticlesPerCell": 8, "CFLNumber": 1.0,
                                "MixingCoefficient": 0.1, "PGTransferAlg": "LINEAR"},
            "Seed": seed,
        }}]})


def test_loader_errors_without_device():
    L = mp()
    L.loadScene(b"{ not json")
    assert "json" in err(L).lower() or "expected" in err(L).lower()
    L.loadScene(b'{"Nothing": []}')
    assert "HybridSimulator" in err(L)
    out = np.zeros(3, np.float32)
    L.copyEulerParticlesPosToCPU(b"missing", out.ctypes.data_as(PF))
    assert "does not exist" in err(L)
    assert L.getParticleSize(b"missing") == 0
    L.copyPositionToCPU(b"missing", out.ctypes.data_as(PF))
    assert "not supported" in err(L)


@pytest.mark.gpu
def test_loaded_scene_matches_oracle(cuda):
    L = mp()
    L.initMPhysics()
    assert err(L) == ""
    try:
        L.loadScene(scene_json().encode())
        assert err(L) == "", err(L)
        o3 = [C.c_float() for _ in range(6)]
        L.getEulerGridInfo(b"Water", *[C.byref(v) for v in o3])
        origin = tuple(v.value for v in o3[:3])
        spacing = tuple(v.value for v in o3[3:])
        res = (16, 14, 12)  # the scene's resolution plus one padding cell per side
        np.testing.assert_allclose(spacing, (0.1, 0.1, 0.1), rtol=1e-6)
        np.testing.assert_allclose(origin, (-0.1, -0.1, -0.1), rtol=1e-6)
        g = hfgrid.Solver.attach(L.mphysics_grid_solver(b"Water"), 0.02, res, origin, spacing)

        n = L.getEulerParticleSize(b"Water")
        assert n == g.num_particles and n > 0
        pos0 = np.empty((n, 3), np.float32)
        L.copyEulerParticlesPosToCPU(b"Water", pos0.ctypes.data_as(PF))
        dom = oracle.fluid_domain_from_bbox(res, origin, spacing, (0.05, 0.05, 0.05), (0.6, 0.7, 0.95))
        solid = g.solid_sdf()
        assert np.array_equal(pos0, oracle.seed_particles(res, origin, spacing, dom, solid, 8, 3))

        o = oracle.Solver(0.02, res, origin, spacing, dbl=1)
        o.add_solid_boundary(solid, (0, 0, 0))
        o.set_fluid_domain_field(dom)
        o.set_advection(hfgrid.ADV_MIX_PIC_FLIP, 2, 2, 1.0, 0.1, 1, 1)
        o.set_particles(pos0, np.zeros_like(pos0))
        o.set_pcg(1, 1, 1e-6, 400)
        for _ in range(2):
            L.update(0.5)  # the argument is ignored, like the reference's
            assert err(L) == "", err(L)
            o.update()
        pos = np.empty((n, 3), np.float32)
        vel = np.empty((n, 3), np.float32)
        L.copyEulerParticlesPosToCPU(b"Water", pos.ctypes.data_as(PF))
        L.copyEulerParticlesVelToCPU(b"Water", vel.ctypes.data_as(PF))
        op, ov = o.particles()
        assert np.abs(pos - op).max() < 2e-4
        assert np.linalg.norm(vel - ov) / np.linalg.norm(ov) < 1e-3

        sdf = np.empty(res[::-1], np.float32)
        L.copyFluidSDFToCPU(b"Water", sdf.ctypes.data_as(PF))
        assert np.array_equal(sdf, oracle.build_fluid_sdf(res, g.fluid_domain_field()))
        gx, gy, gz = (np.empty(res[::-1], np.float32) for _ in range(3))
        L.copyFluidSDFGradientToCPU(b"Water", *[a.ctypes.data_as(PF) for a in (gx, gy, gz)])
        ref = np.gradient(np.pad(sdf.astype(np.float64), 1, mode="edge"), *spacing[::-1])
        for a, gr in zip((gz, gy, gx), ref):
            np.testing.assert_allclose(a, gr[1:-1, 1:-1, 1:-1], rtol=1e-5, atol=1e-3)

        # generateCurFluidDensity on the same current domain and total solid
        assert np.array_equal(g.fluid_density(), oracle.build_fluid_density(res, g.fluid_domain_field(), solid))

        # loading a name that exists stops the load and keeps the old simulator
        L.loadScene(scene_json(seed=9).encode())
        assert L.getEulerParticleSize(b"Water") == n
        g.close()
    finally:
        L.freeMPhysics()
    assert L.mphysics_grid_solver(b"Water") is None
