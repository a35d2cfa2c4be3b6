"""The scene server (hfg_server_*): admission arithmetic on the CPU, and on
the GPU continuous batching whose results match each request run alone.

The reference has no server: its simulators step one after another
(MPhysics.cpp:19-25).  What must hold is that a scene's result does not depend
on what else shares the GPU, and that admission respects slots and the byte
budget.
"""
import numpy as np
import pytest

import hfgrid
import scenes


def test_scene_bytes_arithmetic():
    b64 = hfgrid.scene_bytes((64, 64, 64), 0)
    b64p = hfgrid.scene_bytes((64, 64, 64), 100000)
    b128 = hfgrid.scene_bytes((128, 128, 128), 0)
    assert b64p - b64 == 100000 * 52
    assert 7 < (b128 - (64 << 20)) / (b64 - (64 << 20)) < 9      # grid bytes scale with the cell count
    assert hfgrid.scene_bytes((64, 64, 64), 0, 2) - b64 == 64 ** 3 * 4  # one SDF per extra boundary
    assert hfgrid.scene_bytes((64, 64, 64), 0, 1, hfgrid.PRECOND_MG) > b64


def test_particles_bound_and_validation():
    import ctypes as C
    d = hfgrid.scene_desc((20, 10, 8), fluid_max=(0.5, 0.5, 1.0), per_cell=8)
    n = C.c_longlong()
    assert hfgrid.lib().hfg_scene_particles_bound(C.byref(d), C.byref(n)) == 0
    assert n.value == 10 * 5 * 8 * 8
    d.res[0] = 2
    assert hfgrid.lib().hfg_scene_particles_bound(C.byref(d), C.byref(n)) == -1
    assert "res" in hfgrid.lib().hfg_last_error().decode()


def test_server_needs_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("needs a host without a CUDA device")
    with pytest.raises(hfgrid.HfgError):
        hfgrid.Server(slots=2, budget_bytes=1 << 30)


def _requests():
    sizes = [(32, 32, 32), (40, 36, 32), (48, 40, 40), (36, 44, 32), (32, 48, 40), (44, 32, 36)]
    out = []
    for i, res in enumerate(sizes):
        spheres = [(0.5, 0.15, 0.5, 0.12)] if i % 2 else [(0.7, 0.2, 0.3, 0.1), (0.3, 0.5, 0.7, 0.08)]
        out.append(hfgrid.scene_desc(res, steps=4, spheres=spheres, seed=11 + i, keep_particles=True,
                                     precond=hfgrid.PRECOND_JACOBI, tol_mode=hfgrid.TOL_RELATIVE, tol=1e-6,
                                     max_iter=200))
    return out


@pytest.mark.gpu
def test_mixed_results_match_each_request_alone(cuda):
    reqs = _requests()
    alone = []
    srv = hfgrid.Server(slots=1, budget_bytes=8 << 30)
    for d in reqs:
        rid = srv.submit(d)
        inf = srv.wait(rid)
        assert inf["status"] == 2, inf
        alone.append((inf, srv.particles(rid, inf["particles"])))
    srv.close()

    srv = hfgrid.Server(slots=4, budget_bytes=8 << 30)
    ids = [srv.submit(d) for d in reqs]
    srv.drain()
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["peak_running"] >= 2  # the scenes really overlapped
    for rid, (inf0, pos0) in zip(ids, alone):
        inf = srv.wait(rid)
        assert inf["status"] == 2 and inf["particles"] == inf0["particles"] and inf["steps_done"] == 4
        pos = srv.particles(rid, inf["particles"])
        # P2G sums with atomics in scheduling order: FP32 rounding only
        assert np.abs(pos - pos0).max() < 1e-4
        assert inf["last"]["substeps"] == inf0["last"]["substeps"]
        assert len(srv.step_times(rid)) == 4
    srv.close()


@pytest.mark.gpu
def test_admission_respects_budget_and_rejects_oversized(cuda):
    reqs = _requests()
    import ctypes as C
    fps = []
    for d in reqs:
        n = C.c_longlong()
        assert hfgrid.lib().hfg_scene_particles_bound(C.byref(d), C.byref(n)) == 0
        fps.append(hfgrid.scene_bytes(tuple(d.res), n.value, 1 + d.n_spheres, hfgrid.PRECOND_JACOBI))
    budget = max(fps) + min(fps) + min(fps) // 2  # never room for three scenes
    srv = hfgrid.Server(slots=6, budget_bytes=budget)
    ids = [srv.submit(d) for d in reqs]
    big = srv.submit(hfgrid.scene_desc((512, 512, 512), steps=1))
    srv.drain()
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["rejected"] == 1
    assert st["peak_bytes"] <= budget
    assert 1 <= st["peak_running"] <= 2
    assert srv.wait(big)["status"] == -3
    assert all(srv.wait(i)["status"] == 2 for i in ids)
    srv.close()


@pytest.mark.gpu
def test_analytic_solids_match_host_sdfs(cuda):
    sc = scenes.dam_break_256(n=40)
    s = hfgrid.Solver(sc.dt, sc.res, sc.origin, sc.spacing)
    s.add_analytic_solid(hfgrid.SOLID_WALLS)
    for b in sc.solids:
        s.add_analytic_solid(hfgrid.SOLID_BOX, tuple(b.center) + tuple(b.size))
    s.add_analytic_solid(hfgrid.SOLID_SPHERE, (0.5, 0.15, 0.5, 0.15))
    s.update()
    t = scenes.Scene(res=sc.res, solids=sc.solids + [scenes.Solid("sphere", (0.5, 0.15, 0.5), (0.15, 0, 0))])
    ref = scenes.total_solid(t)
    got = s.solid_sdf()
    # spacing enters as FP32 on the device and FP64 on the host: cell classes
    # agree except where a centre lies on a solid surface
    assert (got != ref).mean() < 1e-3


@pytest.mark.gpu
def test_batch_matches_each_scene_alone(cuda):
    """hfg_batch_*: the CFL substeps of all scenes in one launch per substep
    (each scene with its own CFL state), the rest on the scenes' streams.
    Every scene ends where it ends alone: the same substep counts, particle
    positions within 1e-4 (P2G float atomics add in scheduling order)."""
    reqs = _requests()
    alone = []
    srv = hfgrid.Server(slots=1, budget_bytes=8 << 30)
    for d in reqs:
        rid = srv.submit(d)
        inf = srv.wait(rid)
        assert inf["status"] == 2, inf
        alone.append((inf, srv.particles(rid, inf["particles"])))
    srv.close()
    b = hfgrid.Batch(reqs, threads=3)
    ms = b.step(4)
    assert len(ms) == 4 and all(m > 0 for m in ms)
    for i, (inf0, pos0) in enumerate(alone):
        st = b.stats(i)
        assert st["num_particles"] == inf0["particles"]
        assert st["substeps"] == inf0["last"]["substeps"]
        assert abs(st["cg_iterations"] - inf0["last"]["cg_iterations"]) <= 1
        pos = b.particles(i, st["num_particles"])
        assert np.abs(pos - pos0).max() < 1e-4
    b.close()
