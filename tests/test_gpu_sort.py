"""The particle sort (hfg_sort.cu; option sort_interval, hfg_solver_sort_particles).

No reference counterpart: the reference keeps its seeding order.  The sort
must be a stable permutation by cell (the binning of transPos2Index,
EulerMathTool.cu:29-40), restated here with numpy's stable argsort, and
stepping with it must give the results of stepping without it, up to the
order of the FP32 P2G atomics.  Under the reference's clamp (the boundary
fix reaches the first min(N, P) particles only) each of the two ranges is
sorted within itself.
"""
import numpy as np
import pytest

import scenes

pytestmark = pytest.mark.gpu

U = np.finfo(np.float32).max


def cell_keys(pos, res, origin, spacing):
    """binCell: truncation of (p - o) / h toward zero in FP32, then clamp."""
    p = pos.astype(np.float32)
    k = []
    for a in range(3):
        r = (p[:, a] - np.float32(origin[a])) / np.float32(spacing[a])
        i = np.clip(np.trunc(r).astype(np.int64), 0, res[a] - 1)
        k.append(i)
    return (k[2] * res[1] + k[1]) * res[0] + k[0]


def scene():
    return scenes.Scene(res=(32, 28, 24), solids=[scenes.Solid("sphere", (0.55, 0.2, 0.5), (0.15, 0, 0))], seed=5)


def test_sort_is_the_stable_permutation_by_cell(cuda):
    sc = scene()
    g = scenes.gpu_solver(sc, precond=1, tol_mode=1, tol=1e-6, max_iter=400, advect_scalars=True, clamp_mode=0)
    for _ in range(4):
        g.update()
    pos, vel = g.particles()
    keys = cell_keys(pos, sc.res, sc.origin, sc.spacing)
    perm = np.argsort(keys, kind="stable")
    assert not np.array_equal(perm, np.arange(len(perm))), "four steps should have mixed the order"
    g.sort_particles()
    pos2, vel2 = g.particles()
    assert np.array_equal(pos2, pos[perm])
    assert np.array_equal(vel2, vel[perm])
    assert np.all(np.diff(cell_keys(pos2, sc.res, sc.origin, sc.spacing)) >= 0)
    g.sort_particles()  # sorted input: the identity
    pos3, _ = g.particles()
    assert np.array_equal(pos3, pos2)


@pytest.mark.parametrize("interval,clamp", [(1, 0), (2, 0), (2, 1)])
def test_steps_with_sorting_match_steps_without(cuda, interval, clamp):
    """Same scene stepped with and without the sort: equal substep counts,
    the velocity field within 1e-5 relative L2 and the particle sets within
    1e-5 (the P2G atomics add in another order), markers >= 99.9 % equal."""
    sc = scene()
    a = scenes.gpu_solver(sc, precond=1, tol_mode=1, tol=1e-6, max_iter=400, advect_scalars=True, clamp_mode=clamp)
    b = scenes.gpu_solver(sc, precond=1, tol_mode=1, tol=1e-6, max_iter=400, advect_scalars=True, clamp_mode=clamp,
                          sort_interval=interval)
    for _ in range(5):
        a.update()
        b.update()
        assert a.stats()["substeps"] == b.stats()["substeps"]
    va = np.concatenate([x.ravel() for x in a.velocity_field()])
    vb = np.concatenate([x.ravel() for x in b.velocity_field()])
    assert np.array_equal(va == U, vb == U)
    k = va != U
    d = va[k].astype(np.float64) - vb[k]
    assert np.linalg.norm(d) / np.linalg.norm(va[k].astype(np.float64)) < 1e-5
    assert (a.markers() == b.markers()).mean() >= 0.999
    pa, _ = a.particles()
    pb, _ = b.particles()
    # the same particles, in another order: nearest neighbours pair them one to one
    from scipy.spatial import cKDTree
    dist, idx = cKDTree(pa.astype(np.float64)).query(pb.astype(np.float64))
    assert dist.max() < 1e-5
    assert len(np.unique(idx)) == len(idx)


def test_sort_keeps_the_particles_the_reference_clamp_reaches(cuda):
    """Under clamp_mode 1 the boundary fix reaches the first min(N, P)
    particles only (EulerParticlesTool.cu:880).  With P > N the sort orders
    the first N and the rest each within its own range, so the fix reaches
    the same particles: the permutation is the stable argsort by cell of each
    range."""
    sc = scene()
    g = scenes.gpu_solver(sc, precond=1, tol_mode=1, tol=1e-6, max_iter=400, clamp_mode=1)
    n = sc.n_cells
    assert g.num_particles > n
    for _ in range(4):
        g.update()
    pos, vel = g.particles()
    keys = cell_keys(pos, sc.res, sc.origin, sc.spacing)
    perm = np.concatenate([np.argsort(keys[:n], kind="stable"), n + np.argsort(keys[n:], kind="stable")])
    g.sort_particles()
    pos2, vel2 = g.particles()
    assert np.array_equal(pos2, pos[perm])
    assert np.array_equal(vel2, vel[perm])
