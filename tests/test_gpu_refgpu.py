"""Parity against the reference's own CUDA implementation of the step.

`oracle/refgpu/build.sh` compiles the reference's CGridFluidSolver and every
kernel it calls, unmodified, for sm_100a (oracle/_ref/refgpu); `refgpu`
drives it.  Each case builds the same scene in both, gives the reference the
particles libhfgrid seeded (the count of the reference's own seeding rule,
EulerParticles.cpp:140-179, once its boundaries are assembled), steps both
and compares:

* cell markers (PressureSolver markers, EulerSolverTool.cu:30-56) bit-exact
  after the first step, when both have advected the same particles through a
  field at rest;
* particle positions: within 1e-5 per step in units of the domain;
* face velocities: relative L2 within 1e-4 after one step, 1e-3 after three;
* CG iterations of the reference's own stop rule (identity preconditioner,
  sqrt(r.r) < 1e-3, PressureSolver.cpp:80-82 and CuMatrixFreePCG.cpp:22-65)
  within 2 % of libhfgrid's in its reference mode on the small grid, and
  within 15 % on the 64^3 grid.

The reference's FP64 build (its own DOUBLE_REAL switch) pins the FP64 oracle
the other tests measure error against: both run the whole step in FP64 from
the same particles and agree to 1e-9.

The two FP32 solvers differ only in rounding: FMA contraction in both, and the dot
products of the CG (cuBLAS Sdot in FP32 in the reference, FP64 block
partials here).  On the 64^3 grid the absolute stop rule is reached on a
slow tail of the residual, so those differences move the iteration count
that reaches it by up to ~10 %; the velocities agree all the same.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import refgpu  # noqa: E402

import hfgrid  # noqa: E402
import scenes  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refgpu.available(),
                                 reason="the reference's CUDA build (oracle/refgpu/build.sh) is not present")]


U = np.finfo(np.float32).max


def rel_l2(a, b):
    """Relative L2 difference of two face fields over the faces both know;
    the faces left UNKNOWN (the type's max: FLT_MAX, or DBL_MAX in the FP64
    builds) must be the same in both."""
    a = np.concatenate([x.ravel() for x in a])
    b = np.concatenate([x.ravel() for x in b])
    assert np.array_equal(a >= U, b >= U)
    k = a < U
    a, b = a[k].astype(np.float64), b[k].astype(np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def twins(sc, cap=-1):
    """libhfgrid in the reference's pressure mode, and the reference itself,
    on the same scene and particles (solids with their velocities)."""
    g = scenes.gpu_solver(sc, precond=hfgrid.PRECOND_IDENTITY, tol_mode=hfgrid.TOL_REFERENCE, tol=1e-3,
                          max_iter=cap, advect_scalars=True)
    r = refgpu.RefSolver(sc.dt, sc.res, sc.origin, sc.spacing)
    for sdf, vel in scenes.boundaries(sc):
        r.add_solid_boundary(sdf, vel)
    r.generate_fluid_domain_from_bbox(*scenes.fluid_bbox(sc))
    r.update_boundaries()
    pos, _ = g.particles()
    assert r.set_mix_pic_flip(sc.per_cell, sc.cfl, sc.mixing, pos) == g.num_particles
    if cap > 0:
        r.set_cg_iteration_cap(cap)
    r.take_ax_calls()
    return g, r


def step_both(g, r):
    g.update()
    r.update()
    r.synchronize()
    calls = r.take_ax_calls()
    return g.stats()["cg_iterations"], max(calls - 1, 0)


def small_scene(n=(20, 18, 16)):
    return scenes.Scene(res=n, solids=[scenes.Solid("sphere", (0.55, 0.2, 0.5), (0.15, 0, 0))], seed=7)


def test_reference_seeding_rule(cuda):
    """The reference seeds per_cell particles in every cell inside the fluid
    domain and outside the total solid SDF (EulerParticlesTool.cu:5-25,
    EulerParticles.cpp:140-179).  Built before any update, as its own setup
    does (HybridSimulator.cpp:111-115), the total SDF is still all zeros and
    the solids exclude nothing; with the boundaries assembled first it seeds
    exactly the cells libhfgrid seeds."""
    sc = small_scene()
    g = scenes.gpu_solver(sc)
    domain_cells = int((g.fluid_domain_field() < 0).sum())

    def ref(assemble):
        r = refgpu.RefSolver(sc.dt, sc.res, sc.origin, sc.spacing)
        for sdf, _ in scenes.boundaries(sc):
            r.add_solid_boundary(sdf)
        r.generate_fluid_domain_from_bbox(*scenes.fluid_bbox(sc))
        if assemble:
            r.update_boundaries()
        return r, r.set_mix_pic_flip(sc.per_cell, sc.cfl, sc.mixing)

    _, n_stock = ref(False)
    assert n_stock == sc.per_cell * domain_cells
    r, n = ref(True)
    assert n == g.num_particles < n_stock
    pos, vel = r.particles()
    gp, _ = g.particles()

    def cells(p):
        c = np.floor((p - np.array(sc.origin)) / np.array(sc.spacing)).astype(np.int64)
        return np.sort(c[:, 0] + sc.res[0] * (c[:, 1] + sc.res[1] * c[:, 2]))

    assert np.array_equal(cells(pos), cells(gp))
    assert not vel.any()


@pytest.mark.parametrize("steps", [1, 3])
def test_step_vs_reference_gpu(cuda, steps):
    sc = small_scene()
    g, r = twins(sc)
    for k in range(steps):
        it_g, it_r = step_both(g, r)
        assert abs(it_g - it_r) <= max(1, 0.02 * it_r), (k, it_g, it_r)
        if k == 0:
            assert np.array_equal(g.markers().astype(np.float32), r.markers())
    gp, _ = g.particles()
    rp, _ = r.particles()
    assert np.abs(gp - rp).max() < 1e-5 * steps
    assert (g.markers().astype(np.float32) != r.markers()).mean() < 2e-3
    assert rel_l2(g.velocity_field(), r.velocity_field()) < (1e-4 if steps == 1 else 1e-3)


def test_c1_dam_break_vs_reference_gpu(cuda):
    """The 64^3 dam break with the static sphere (0.48 M particles), three
    steps, each compared with the reference's own CUDA step."""
    sc = scenes.dam_break_64(seed=0)
    g, r = twins(sc)
    rows = []
    for k in range(3):
        it_g, it_r = step_both(g, r)
        gp, _ = g.particles()
        rp, _ = r.particles()
        err = rel_l2(g.velocity_field(), r.velocity_field())
        mk = float((g.markers().astype(np.float32) == r.markers()).mean())
        rows.append((k + 1, it_g, it_r, err, float(np.abs(gp - rp).max()), mk))
    print("\nstep  CG its (ours, reference)  vel rel L2  max |dx|  markers equal")
    for row in rows:
        print("%4d  %10d %12d  %10.3e  %8.2e  %13.5f" % row)
    for k, it_g, it_r, err, dx, mk in rows:
        assert abs(it_g - it_r) <= 0.15 * it_r
        assert dx < 1e-5 * k
        assert mk >= (1.0 if k == 1 else 0.998)
        assert err < (1e-4 if k == 1 else 1e-3)


def test_moving_solid_vs_reference_gpu(cuda):
    """A sphere moving at a constant velocity through the fluid (the
    reference's CBoundarys motion: translation -dt v per step and the SDF
    resampled, Boundary.cpp:115-136), three steps against the reference's own
    CUDA step: markers bit-exact after the first step, then >= 99.8 %, velocity
    within 1e-4 / 1e-3, particles within 1e-5 per step."""
    sc = scenes.Scene(res=(24, 20, 18), solids=[scenes.Solid("sphere", (0.45, 0.25, 0.5), (0.15, 0, 0),
                                                            (0.6, 0.0, -0.3))], seed=11)
    g, r = twins(sc)
    for k in range(3):
        it_g, it_r = step_both(g, r)
        assert abs(it_g - it_r) <= max(2, 0.05 * it_r), (k, it_g, it_r)
        mk = float((g.markers().astype(np.float32) == r.markers()).mean())
        assert mk >= (1.0 if k == 0 else 0.998)
        gp, _ = g.particles()
        rp, _ = r.particles()
        assert np.abs(gp - rp).max() < 1e-5 * (k + 1)
        assert rel_l2(g.velocity_field(), r.velocity_field()) < (1e-4 if k == 0 else 1e-3)


def fp64_pair(sc, pos):
    """The reference's FP64 build and the FP64 oracle, same scene and
    particles, both in the reference's own pressure mode."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    r = refgpu.RefSolver(sc.dt, sc.res, sc.origin, sc.spacing, fp64=True)
    o = oracle.Solver(sc.dt, sc.res, sc.origin, sc.spacing, dbl=1)
    for sdf, v in scenes.boundaries(sc):
        r.add_solid_boundary(sdf)
        o.add_solid_boundary(sdf, v)
    r.generate_fluid_domain_from_bbox(*scenes.fluid_bbox(sc))
    r.update_boundaries()
    assert r.set_mix_pic_flip(sc.per_cell, sc.cfl, sc.mixing, pos) == len(pos)
    o.set_fluid_domain_field(oracle.fluid_domain_from_bbox(sc.res, sc.origin, sc.spacing, *scenes.fluid_bbox(sc)))
    o.set_advection(hfgrid.ADV_MIX_PIC_FLIP, 2, 2, sc.cfl, sc.mixing, 1, 1)
    o.set_particles(pos)
    o.set_pcg(0, 0, 1e-3, -1)
    r.take_ax_calls()
    return r, o


@pytest.mark.skipif(not refgpu.available(fp64=True), reason="the reference's FP64 build is not present")
@pytest.mark.parametrize("which", ["small", "c1"])
def test_fp64_oracle_matches_the_reference_fp64_step(cuda, which):
    """Three steps of the FP64 oracle (oracle/hfg_oracle.cpp, the CPU
    restatement the other tests measure error against) beside the
    reference's own step built in FP64, from the same particles: equal CG
    iteration counts (within one), markers equal, velocities within 1e-9
    relative L2 and particles within 1e-9."""
    sc = small_scene() if which == "small" else scenes.dam_break_64(seed=0)
    pos, _ = scenes.gpu_solver(sc).particles()
    r, o = fp64_pair(sc, pos)
    rows = []
    for k in range(3):
        r.update()
        o.update()
        r.synchronize()
        it_r = max(r.take_ax_calls() - 1, 0)
        it_o = o.stats()["cg_iterations"]
        rp, _ = r.particles()
        op, _ = o.particles_f64()
        vr = r.velocity_field()
        vo = o.velocity_field_f64()
        err = rel_l2(vo, vr)
        rows.append((k + 1, it_o, it_r, err, float(np.abs(rp - op).max()),
                     float((o.markers().astype(np.float64) == r.markers()).mean())))
    print("\nstep  CG its (oracle, reference FP64)  vel rel L2  max |dx|  markers equal")
    for row in rows:
        print("%4d  %10d %12d  %10.3e  %8.2e  %13.5f" % row)
    for k, it_o, it_r, err, dx, mk in rows:
        assert abs(it_o - it_r) <= 1
        assert mk == 1.0
        assert err < 1e-9
        assert dx < 1e-9
