"""Parity of each CUDA stage of the grid step against the CPU oracle.

Every test drives libhfgrid.so through its C ABI (hfg_op_*) on seeded inputs
and compares with the oracle restatement of the same reference stage.
Integer and index work (markers, bin counts, layers, seeding) must be
bit-exact; floating-point results are held to the tolerances written in each
test (FP32 kernels vs the FP32 operation-by-operation oracle, or vs FP64).
"""
import numpy as np
import pytest
import torch

import hfgrid
import oracle

pytestmark = pytest.mark.gpu

RES = (13, 11, 9)           # ragged on purpose
ORIGIN = (0.25, -0.5, 1.0)
SPACING = (0.1, 0.12, 0.09)


def dev(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def face_arrays(res, rng, scale=1.0):
    return [(rng.standard_normal(s) * scale).astype(np.float32) for s in oracle.face_shapes(res)]


def random_particles(rng, n, res=RES, origin=ORIGIN, spacing=SPACING, margin=0.5):
    lo = np.array(origin) - margin * np.array(spacing)
    hi = np.array(origin) + (np.array(res) + margin) * np.array(spacing)
    return (lo + rng.random((n, 3)) * (hi - lo)).astype(np.float32)


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


def test_markers_and_bins_bit_exact(cuda):
    rng = np.random.default_rng(1)
    solid = rng.standard_normal(RES[::-1]).astype(np.float32)
    pos = random_particles(rng, 5000)
    # particles exactly on cell faces and outside the grid exercise truncation/clamping
    pos[:50, 0] = (ORIGIN[0] + SPACING[0] * rng.integers(-2, RES[0] + 2, 50)).astype(np.float32)
    mk_ref, cnt_ref = oracle.markers_from_particles(RES, ORIGIN, SPACING, solid, pos)
    mk = torch.empty(RES[::-1], dtype=torch.uint8, device=cuda)
    cnt = torch.empty(RES[::-1], dtype=torch.int32, device=cuda)
    hfgrid.op_markers_from_particles(RES, ORIGIN, SPACING, dev(solid), dev(pos), mk)
    hfgrid.op_bin_counts(RES, ORIGIN, SPACING, dev(pos), cnt)
    assert np.array_equal(host(mk), mk_ref)
    assert np.array_equal(host(cnt).astype(np.uint32), cnt_ref)
    # empty particle set: solid cells only
    hfgrid.op_markers_from_particles(RES, ORIGIN, SPACING, dev(solid), dev(pos[:0]), mk)
    assert np.array_equal(host(mk), np.where(solid < 0, 2, 0).astype(np.uint8))


def test_markers_from_sdf(cuda):
    rng = np.random.default_rng(2)
    solid = rng.standard_normal(RES[::-1]).astype(np.float32)
    fluid = rng.standard_normal(RES[::-1]).astype(np.float32)
    mk = torch.empty(RES[::-1], dtype=torch.uint8, device=cuda)
    hfgrid.op_markers_from_sdf(RES, dev(solid), dev(fluid), mk)
    assert np.array_equal(host(mk), oracle.markers_from_sdf(RES, solid, fluid))


def random_markers(rng, res=RES, p=(0.3, 0.5, 0.2)):
    return rng.choice(np.array([0, 1, 2], np.uint8), size=res[::-1], p=p)


def test_matrix_a_exact(cuda):
    rng = np.random.default_rng(3)
    mk = random_markers(rng)
    A = torch.empty(4 * np.prod(RES), dtype=torch.float32, device=cuda)
    hfgrid.op_build_matrix_a(RES, SPACING, 0.05, dev(mk), A)
    assert np.array_equal(host(A), oracle.build_matrix_a(RES, SPACING, 0.05, mk))


def test_apply_a(cuda):
    rng = np.random.default_rng(4)
    mk = random_markers(rng)
    x = rng.standard_normal(RES[::-1]).astype(np.float32)
    y = torch.empty(RES[::-1], dtype=torch.float32, device=cuda)
    hfgrid.op_apply_a(RES, SPACING, 0.05, dev(mk), dev(x), y)
    ref = oracle.apply_a(RES, SPACING, 0.05, mk, x)
    # products in FP32, sum in FP64 on both sides: identical up to the last bit
    np.testing.assert_allclose(host(y), ref, rtol=1e-6, atol=1e-6 * np.abs(ref).max())


def test_rhs(cuda):
    rng = np.random.default_rng(5)
    mk = random_markers(rng)
    v = face_arrays(RES, rng)
    sv = face_arrays(RES, rng, 0.3)
    b = torch.empty(RES[::-1], dtype=torch.float32, device=cuda)
    hfgrid.op_build_rhs(RES, SPACING, [dev(a) for a in v], [dev(a) for a in sv], dev(mk), b)
    ref = oracle.build_rhs(RES, SPACING, v, sv, mk)
    np.testing.assert_allclose(host(b), ref, rtol=1e-5, atol=1e-5 * np.abs(ref).max())


def blob_markers(res, rng):
    """Fluid blob with solid walls and some air, like a dam break."""
    nz, ny, nx = res[::-1]
    mk = np.zeros((nz, ny, nx), np.uint8)
    mk[:, : ny // 2 + 1, : nx // 2 + 2] = 1
    mk[0, :, :] = mk[-1, :, :] = 2
    mk[:, 0, :] = mk[:, -1, :] = 2
    mk[:, :, 0] = mk[:, :, -1] = 2
    mk[rng.random(mk.shape) < 0.03] = 2
    return mk


@pytest.mark.parametrize("precond,tol_mode,tol", [(0, 0, 1e-3), (1, 1, 1e-7)])
def test_project(cuda, precond, tol_mode, tol):
    rng = np.random.default_rng(6)
    res = (20, 18, 16)
    h = (1 / 20, 1 / 18, 1 / 16)
    dt = 1 / 60
    mk = blob_markers(res, rng)
    v = face_arrays(res, rng, 0.5)
    sv = face_arrays(res, rng, 0.1)
    vd = [dev(a) for a in v]
    p = torch.empty(res[::-1], dtype=torch.float32, device=cuda)
    st = hfgrid.op_project(res, h, dt, dev(mk), vd, [dev(a) for a in sv], precond=precond, tol_mode=tol_mode,
                           tol=tol, max_iter=-1, p_out=p)
    v64, p64, st64 = oracle.project(res, h, dt, mk, v, sv, precond=precond, tol_mode=tol_mode, tol=1e-10 if
                                    tol_mode == 1 else tol, max_iter=-1, dbl=1)
    assert st["converged"]
    # the CG stops on its own residual rule: pressure within 1e-4 relative of
    # the FP64 solve, velocities (known faces) likewise
    assert rel_err(host(p), p64) < 1e-4
    for a in range(3):
        g, r = host(vd[a]), v64[a]
        known = r != np.finfo(np.float32).max
        assert np.array_equal(g == np.finfo(np.float32).max, ~known)
        assert rel_err(g[known], r[known]) < 1e-4


def test_extrapolation_bit_exact(cuda):
    rng = np.random.default_rng(7)
    res = (17, 12, 10)
    U = np.finfo(np.float32).max
    v = face_arrays(res, rng)
    for a in range(3):
        unknown = rng.random(v[a].shape) < 0.9
        unknown[..., :3] = True
        v[a][unknown] = U
    # one fully unknown component: nothing to extrapolate from
    v[2][:] = U
    ref = oracle.extrapolate_fc(res, v, 1000)
    vd = [dev(a) for a in v]
    hfgrid.op_extrapolate_fc(res, vd, 1000)
    for a in range(3):
        assert np.array_equal(host(vd[a]), ref[a])
    # a depth cap: only the first few layers are filled
    vd = [dev(a) for a in v]
    hfgrid.op_extrapolate_fc(res, vd, 3)
    ref3 = oracle.extrapolate_fc(res, v, 3)
    for a in range(3):
        assert np.array_equal(host(vd[a]), ref3[a])


def test_extrapolation_large_layers_bit_exact(cuda):
    """Layers far larger than the one-block path takes (kExtrapSmallLayer =
    4096 entries): a 96^3 face grid known only in a small blob, so the layer
    at distance d holds ~d^2 faces (up to ~11,900) and the grid-strided path
    with the bounded grid barrier between layers runs for most of the ~160
    layers.  Values and
    the UNKNOWN entries left must equal the oracle's bit for bit."""
    rng = np.random.default_rng(17)
    res = (96, 96, 96)
    U = np.finfo(np.float32).max
    v = face_arrays(res, rng)
    for a in range(3):
        keep = np.zeros(v[a].shape, bool)
        keep[40:48, 44:52, 20:30] = rng.random((8, 8, 10)) < 0.7
        v[a][~keep] = U
    ref = oracle.extrapolate_fc(res, v, 1000)
    for a in range(3):
        _, mk = oracle.extrapolate(v[a].shape[::-1], v[a], 1000, with_markers=True)
        widths = np.bincount(mk[mk != U].astype(np.int64))
        assert (widths > 4096).sum() >= 50 and widths.max() > 11000  # the large-layer path runs
    vd = [dev(a) for a in v]
    hfgrid.op_extrapolate_fc(res, vd, 1000)
    for a in range(3):
        assert np.array_equal(host(vd[a]), ref[a])


def test_extrapolation_cc_layers(cuda):
    rng = np.random.default_rng(8)
    res = (31, 7, 5)
    U = np.finfo(np.float32).max
    f = rng.standard_normal(res[::-1]).astype(np.float32)
    f[rng.random(f.shape) < 0.97] = U
    f.flat[0] = 1.0
    ref = oracle.extrapolate(res, f, 1000)
    fd = dev(f)
    hfgrid.op_extrapolate_cc(res, fd, 1000)
    assert np.array_equal(host(fd), ref)


def test_sampling(cuda):
    rng = np.random.default_rng(9)
    v = face_arrays(RES, rng)
    pos = random_particles(rng, 3000, margin=2.0)
    out = torch.empty((3000, 3), dtype=torch.float32, device=cuda)
    hfgrid.op_sample_fc(RES, ORIGIN, SPACING, [dev(a) for a in v], dev(pos), out)
    ref = oracle.sample_fc(RES, ORIGIN, SPACING, v, pos)
    np.testing.assert_allclose(host(out), ref, rtol=2e-5, atol=2e-5)
    f = rng.standard_normal(RES[::-1]).astype(np.float32)
    o1 = torch.empty(3000, dtype=torch.float32, device=cuda)
    hfgrid.op_sample_cc(RES, ORIGIN, SPACING, dev(f), dev(pos), o1)
    np.testing.assert_allclose(host(o1), oracle.sample_cc(RES, ORIGIN, SPACING, f, pos), rtol=2e-5, atol=2e-5)


@pytest.mark.parametrize("alg", [hfgrid.LINEAR, hfgrid.QUADRATIC, hfgrid.CUBIC, hfgrid.G2PNEAREST])
def test_g2p(cuda, alg):
    rng = np.random.default_rng(10 + alg)
    v = face_arrays(RES, rng)
    pos = random_particles(rng, 2000)
    out = torch.empty((2000, 3), dtype=torch.float32, device=cuda)
    hfgrid.op_g2p_fc(RES, ORIGIN, SPACING, [dev(a) for a in v], dev(pos), alg, out)
    np.testing.assert_allclose(host(out), oracle.g2p_fc(RES, ORIGIN, SPACING, v, pos, alg), rtol=1e-5, atol=1e-5)
    f = rng.standard_normal(RES[::-1]).astype(np.float32)
    o1 = torch.empty(2000, dtype=torch.float32, device=cuda)
    hfgrid.op_g2p_cc(RES, ORIGIN, SPACING, dev(f), dev(pos), alg, o1)
    np.testing.assert_allclose(host(o1), oracle.g2p_cc(RES, ORIGIN, SPACING, f, pos, alg), rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("alg", [hfgrid.LINEAR, hfgrid.QUADRATIC, hfgrid.CUBIC, hfgrid.P2GSUM])
def test_p2g(cuda, alg):
    rng = np.random.default_rng(20 + alg)
    pos = random_particles(rng, 4000)
    vel = rng.standard_normal((4000, 3)).astype(np.float32)
    outs = [torch.empty(s, dtype=torch.float32, device=cuda) for s in oracle.face_shapes(RES)]
    ws = [torch.empty(s, dtype=torch.float32, device=cuda) for s in oracle.face_shapes(RES)]
    hfgrid.op_p2g_fc(RES, ORIGIN, SPACING, dev(pos), dev(vel), alg, outs, ws)
    ref, wref = oracle.p2g_fc(RES, ORIGIN, SPACING, pos, vel, alg, dbl=1)
    for a in range(3):
        # unordered FP32 atomics vs an ordered FP64 sum
        np.testing.assert_allclose(host(outs[a]), ref[a], rtol=1e-4, atol=1e-4)
        np.testing.assert_allclose(host(ws[a]), wref[a], rtol=1e-5, atol=1e-4)
    val = rng.standard_normal(4000).astype(np.float32)
    f = torch.empty(RES[::-1], dtype=torch.float32, device=cuda)
    w = torch.empty(RES[::-1], dtype=torch.float32, device=cuda)
    hfgrid.op_p2g_cc(RES, ORIGIN, SPACING, dev(pos), dev(val), alg, f, w)
    fr, wr = oracle.p2g_cc(RES, ORIGIN, SPACING, pos, val, alg)
    np.testing.assert_allclose(host(f), fr, rtol=1e-4, atol=1e-4)
    np.testing.assert_allclose(host(w), wr, rtol=1e-4, atol=1e-4)


def test_p2g_linear_grouped_particles(cuda):
    """LINEAR face P2G with particles in seeding order (eight per cell, next
    to each other), the layout where lanes of a warp share corners and sum by
    shuffles first.  Cells near every wall (the clamped-corner cases), cells
    with fewer than eight particles and a ragged tail cover full octets,
    quads, pairs and single lanes; the result must match the FP64 oracle as
    for unordered particles."""
    rng = np.random.default_rng(77)
    nx, ny, nz = RES
    cells = [(x, y, z) for z in range(nz) for y in range(ny) for x in range(nx)]
    pos = []
    for i, (x, y, z) in enumerate(cells):
        k = 8 if i % 5 else (i % 8)  # every fifth cell holds fewer than eight
        for _ in range(k):
            jitter = rng.random(3)
            pos.append([ORIGIN[0] + (x + jitter[0]) * SPACING[0], ORIGIN[1] + (y + jitter[1]) * SPACING[1],
                        ORIGIN[2] + (z + jitter[2]) * SPACING[2]])
    pos = np.array(pos[: len(pos) - 3], np.float32)  # ragged tail
    vel = rng.standard_normal((len(pos), 3)).astype(np.float32)
    outs = [torch.empty(sh, dtype=torch.float32, device=cuda) for sh in oracle.face_shapes(RES)]
    ws = [torch.empty(sh, dtype=torch.float32, device=cuda) for sh in oracle.face_shapes(RES)]
    hfgrid.op_p2g_fc(RES, ORIGIN, SPACING, dev(pos), dev(vel), hfgrid.LINEAR, outs, ws)
    ref, wref = oracle.p2g_fc(RES, ORIGIN, SPACING, pos, vel, hfgrid.LINEAR, dbl=1)
    for a in range(3):
        np.testing.assert_allclose(host(outs[a]), ref[a], rtol=1e-4, atol=1e-4)
        np.testing.assert_allclose(host(ws[a]), wref[a], rtol=1e-5, atol=1e-4)


@pytest.mark.parametrize("acc", [0, 1, 2])
def test_advect_particles(cuda, acc):
    rng = np.random.default_rng(30 + acc)
    v = face_arrays(RES, rng, 0.3)
    pos = random_particles(rng, 3000, margin=0.0)
    pd = dev(pos)
    n = hfgrid.op_advect_particles(RES, ORIGIN, SPACING, [dev(a) for a in v], pd, 0.05, 1.0, acc, 1)
    ref, nref = oracle.advect_particles(RES, ORIGIN, SPACING, v, pos, 0.05, 1.0, acc, 1, dbl=1)
    assert n == nref
    np.testing.assert_allclose(host(pd), ref, rtol=1e-5, atol=2e-5)


@pytest.mark.parametrize("acc", [0, 1, 2])
def test_semi_lagrangian(cuda, acc):
    rng = np.random.default_rng(40 + acc)
    v = face_arrays(RES, rng, 0.2)
    f = face_arrays(RES, rng)
    out = [torch.empty(s, dtype=torch.float32, device=cuda) for s in oracle.face_shapes(RES)]
    hfgrid.op_sl_advect_fc(RES, ORIGIN, SPACING, [dev(a) for a in f], [dev(a) for a in v], 0.05, acc, out)
    ref = oracle.sl_advect_fc(RES, ORIGIN, SPACING, f, v, 0.05, acc, dbl=1)
    for a in range(3):
        np.testing.assert_allclose(host(out[a]), ref[a], rtol=1e-4, atol=1e-4)
    c = rng.standard_normal(RES[::-1]).astype(np.float32)
    o1 = torch.empty(RES[::-1], dtype=torch.float32, device=cuda)
    hfgrid.op_sl_advect_cc(RES, ORIGIN, SPACING, dev(c), [dev(a) for a in v], 0.05, acc, o1)
    np.testing.assert_allclose(host(o1), oracle.sl_advect_cc(RES, ORIGIN, SPACING, c, v, 0.05, acc), rtol=1e-4,
                               atol=1e-4)


@pytest.mark.parametrize("samp", [1, 2, 3, 4])
def test_cubic_sampling(cuda, samp):
    """Catmull-Rom, monotonic Catmull-Rom, Bridson and clamped Bridson
    sampling of a cell-centred grid and of the face grids against the FP32
    oracle, points inside and outside the grid (clamp-to-edge)."""
    rng = np.random.default_rng(80 + samp)
    f = rng.standard_normal(RES[::-1]).astype(np.float32)
    pos = random_particles(rng, 4000, margin=2.0)
    out = torch.empty(4000, dtype=torch.float32, device=cuda)
    hfgrid.op_sample_cc_ex(RES, ORIGIN, SPACING, dev(f), dev(pos), samp, out)
    ref = oracle.sample_cc(RES, ORIGIN, SPACING, f, pos, alg=samp)
    np.testing.assert_allclose(host(out), ref, rtol=1e-5, atol=1e-5)
    v = face_arrays(RES, rng)
    o3 = torch.empty((4000, 3), dtype=torch.float32, device=cuda)
    hfgrid.op_sample_fc_ex(RES, ORIGIN, SPACING, [dev(a) for a in v], dev(pos), samp, o3)
    np.testing.assert_allclose(host(o3), oracle.sample_fc_alg(RES, ORIGIN, SPACING, v, pos, samp), rtol=1e-5,
                               atol=1e-5)


def test_cubic_sampling_reference_cases(cuda):
    """The reference's own cubic-sampling known answers
    (UnitTest-CellCenteredScalarField.cu) through the GPU entry point."""
    import json
    import os
    import test_oracle_golden as gold
    cases = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "sampling_golden.json")))["cases"]
    for case in cases:
        res, dres = case["res"], case.get("res2", case["res"])
        src = gold._grid_eval(case["src"], res)
        pos = np.stack([gold._grid_eval(case["pos"][a], dres) for a in "XYZ"], axis=-1).reshape(-1, 3)
        out = torch.empty(pos.shape[0], dtype=torch.float32, device=cuda)
        hfgrid.op_sample_cc_ex(res, case["origin"], case["spacing"], dev(src), dev(pos),
                               gold.SAMPLING_ALG[case["alg"]], out)
        got = host(out)
        for e in case["expect"]:
            assert abs(got[e["index"]] - e["value"]) < 1e-4, (case["line"], e)
        if "expect_formula" in case:
            assert np.abs(got - gold._grid_eval(case["expect_formula"], dres).reshape(-1)).max() < 1e-4


@pytest.mark.parametrize("samp", [1, 2, 3, 4])
def test_semi_lagrangian_cubic(cuda, samp):
    """Semi-Lagrangian RK3 advection with a cubic sampler for every back-trace
    and final sample, against the FP32 oracle with the same sampler."""
    rng = np.random.default_rng(90 + samp)
    v = face_arrays(RES, rng, 0.2)
    f = face_arrays(RES, rng)
    out = [torch.empty(s, dtype=torch.float32, device=cuda) for s in oracle.face_shapes(RES)]
    hfgrid.op_sl_advect_fc(RES, ORIGIN, SPACING, [dev(a) for a in f], [dev(a) for a in v], 0.05, 2, out,
                           sampling=samp)
    ref = oracle.sl_advect_fc(RES, ORIGIN, SPACING, f, v, 0.05, 2, sampling=samp)
    for a in range(3):
        np.testing.assert_allclose(host(out[a]), ref[a], rtol=1e-4, atol=1e-4)
    c = rng.standard_normal(RES[::-1]).astype(np.float32)
    o1 = torch.empty(RES[::-1], dtype=torch.float32, device=cuda)
    hfgrid.op_sl_advect_cc(RES, ORIGIN, SPACING, dev(c), [dev(a) for a in v], 0.05, 2, o1, sampling=samp)
    np.testing.assert_allclose(host(o1), oracle.sl_advect_cc(RES, ORIGIN, SPACING, c, v, 0.05, 2, sampling=samp),
                               rtol=1e-4, atol=1e-4)


def test_fluid_domain_and_seeding_bit_exact(cuda):
    res = (24, 20, 16)
    h = tuple(1.0 / r for r in res)
    o = (0.0, 0.0, 0.0)
    out = torch.empty(res[::-1], dtype=torch.float32, device=cuda)
    hfgrid.op_fluid_domain_from_bbox(res, o, h, (0, 0, 0), (0.4, 0.6, 1.0), out)
    ref = oracle.fluid_domain_from_bbox(res, o, h, (0, 0, 0), (0.4, 0.6, 1.0))
    dom = host(out)
    assert np.array_equal(dom, ref)
    rng = np.random.default_rng(50)
    solid = np.where(rng.random(res[::-1]) < 0.1, -1.0, 1.0).astype(np.float32)
    n = hfgrid.op_seed_particles(res, o, h, out, dev(solid), 8, 1234)
    pos = torch.empty((n, 3), dtype=torch.float32, device=cuda)
    hfgrid.op_seed_particles(res, o, h, out, dev(solid), 8, 1234, pos, n)
    pref = oracle.seed_particles(res, o, h, dom, solid, 8, 1234)
    assert pref.shape[0] == n
    assert np.array_equal(host(pos), pref)


def test_fluid_sdf_bit_exact(cuda):
    """generateCurFluidSDF / buildFluidSDF (EulerSolverTool.cu:324-406): the
    frontier BFS gives the reference's layered values exactly."""
    rng = np.random.default_rng(60)
    res = (23, 17, 13)
    dom = np.where(rng.random(res[::-1]) < 0.3, -500.0, 500.0).astype(np.float32)
    dom[:, :8, :10] = -500.0
    for layers in (1000, 4):
        out = torch.empty(res[::-1], dtype=torch.float32, device=cuda)
        hfgrid.op_build_fluid_sdf(res, dev(dom), out, layers)
        assert np.array_equal(host(out), oracle.build_fluid_sdf(res, dom, layers))


def test_fluid_density_bit_exact(cuda):
    """buildFluidDensity (EulerSolverTool.cu:408-448): 1 / 0.2 / 0 exactly."""
    rng = np.random.default_rng(61)
    res = (19, 15, 11)
    dom = np.where(rng.random(res[::-1]) < 0.5, -500.0, 500.0).astype(np.float32)
    dom[:, :6, :8] = -500.0
    solid = np.where(rng.random(res[::-1]) < 0.1, -1.0, np.finfo(np.float32).max).astype(np.float32)
    out = torch.empty(res[::-1], dtype=torch.float32, device=cuda)
    hfgrid.op_build_fluid_density(res, dev(dom), dev(solid), out)
    ref = oracle.build_fluid_density(res, dom, solid)
    assert np.array_equal(host(out), ref)
    assert set(np.unique(ref)) <= {0.0, np.float32(0.2), 1.0}


def _density_case(seed, res):
    """A fluid density of the reference's buildFluidDensity (oracle) over a
    blocky fluid domain with scattered solid cells."""
    rng = np.random.default_rng(seed)
    dom = np.where(rng.random(res[::-1]) < 0.15, -500.0, 500.0).astype(np.float32)
    dom[:, : res[1] // 2, : res[0] * 2 // 3] = -500.0
    solid = np.where(rng.random(res[::-1]) < 0.05, -1.0, np.finfo(np.float32).max).astype(np.float32)
    solid[0], solid[-1] = -1.0, -1.0
    return oracle.build_fluid_density(res, dom, solid), solid


@pytest.mark.parametrize("outside", [False, True])
def test_fluid_side_sdf_bit_exact(cuda, outside):
    """buildFluidInsideSDF / buildFluidOutsideSDF of the hybrid coupler
    (HybridSimulatorBuildSDF.cu:4-146,177-238): the frontier BFS gives the
    reference's swept shells exactly, with the invokers' 1000 sweeps, a short
    sweep count that leaves cells UNKNOWN, and 0 sweeps (clamp only)."""
    res = (29, 21, 17)
    density, solid = _density_case(70 + outside, res)
    op = hfgrid.op_build_fluid_outside_sdf if outside else hfgrid.op_build_fluid_inside_sdf
    for distance in (1000, 3):
        out = torch.empty(res[::-1], dtype=torch.float32, device=cuda)
        op(res, dev(density), dev(solid), out, distance)
        ref = oracle.build_fluid_side_sdf(res, density, solid, outside, distance)
        assert np.array_equal(host(out), ref)
        if distance == 3:
            assert (ref == np.finfo(np.float32).max).any(), "3 sweeps should leave far cells UNKNOWN"
        else:
            assert ref.max() > 3
    start = np.random.default_rng(72).standard_normal(res[::-1]).astype(np.float32)
    out = dev(start)
    op(res, dev(density), dev(solid), out, 0)
    assert np.array_equal(host(out), oracle.build_fluid_side_sdf(res, density, solid, outside, 0, out=start))


def _shell_index(v, seed, passable, seeds):
    """Shell k of every value k + seed (formed in double, rounded to float as
    the reference does); seeds 0, unreached or other cells -1."""
    k = np.full(v.shape, -1, np.int32)
    near = np.rint(v.astype(np.float64) - seed)
    ok = passable & (v != np.finfo(np.float32).max) & (near >= 1)
    ok &= v == (near + seed).astype(np.float32)
    k[ok] = near[ok].astype(np.int32)
    k[seeds] = 0
    return k


def _neighbour_extremes(k):
    """Min and max of the six clamp-to-edge neighbours' shells, over the
    neighbours that hold one (k >= 0)."""
    big = np.int32(1 << 30)
    lo = np.where(k >= 0, k, big)
    hi = k.copy()
    p_lo, p_hi = np.pad(lo, 1, mode="edge"), np.pad(hi, 1, mode="edge")
    mn = np.full(k.shape, big, np.int32)
    mx = np.full(k.shape, -1, np.int32)
    for axis in range(3):
        for d in (-1, 1):
            sl = [slice(1, -1)] * 3
            sl[axis] = slice(1 + d, p_lo.shape[axis] - 1 + d)
            mn = np.minimum(mn, p_lo[tuple(sl)])
            mx = np.maximum(mx, p_hi[tuple(sl)])
    return mn, mx


@pytest.mark.parametrize("outside", [False, True])
def test_fluid_side_sdf_properties_256(cuda, outside):
    """The inside / outside distance fields at the benchmark's size (the
    256^3 dam break's fluid density, solids included), by the properties
    that define a breadth-first distance: every reached cell has a
    neighbour exactly one shell nearer the surface and none nearer than
    that, and no unreached cell touches a shell short of the sweep limit."""
    import scenes
    sc = scenes.dam_break_256()
    res = sc.res
    dom = oracle.fluid_domain_from_bbox(res, sc.origin, sc.spacing, *scenes.fluid_bbox(sc))
    solid = scenes.total_solid(sc)
    rho = torch.empty(res[::-1], dtype=torch.float32, device=cuda)
    hfgrid.op_build_fluid_density(res, dev(dom), dev(solid), rho)
    out = torch.empty_like(rho)
    op = hfgrid.op_build_fluid_outside_sdf if outside else hfgrid.op_build_fluid_inside_sdf
    distance = 1000
    op(res, rho, dev(solid), out, distance)
    density, v = host(rho), host(out)
    open_ = solid >= 0
    seeds = open_ & (density == np.float32(0.2))
    # the sweeps grow into the air (outside) or the fluid's interior (inside)
    passable = open_ & (density == (np.float32(0.0) if outside else np.float32(1.0)))
    U = np.finfo(np.float32).max
    # cells that are neither seeds nor passable hold 0; seeds hold max(seed, 0)
    seed = 0.5 - 0.2 if outside else 0.2 - 0.5
    assert (v[~(seeds | passable)] == 0).all()
    assert (v[seeds] == np.float32(max(seed, 0.0))).all() and seeds.any()
    k = _shell_index(v, seed, passable, seeds)
    reached = passable & (v != U)
    assert (k[reached] >= 1).all(), "a reached cell holds a value that is no shell"
    mn, mx = _neighbour_extremes(k)
    assert (mn[reached] == k[reached] - 1).all()
    unreached = passable & (v == U)
    assert not (mn[unreached] < distance - 1).any()
    assert k.max() > 10  # the shells reach well into the domain

    """buildMixedFluidOutsideSDF (HybridSimulatorBuildSDF.cu:139-175): 0.5 -
    mixed density at surface cells (negative -> 0), the grid's outside SDF
    elsewhere."""
    res = (23, 19, 13)
    density, solid = _density_case(73, res)
    grid_out = oracle.build_fluid_side_sdf(res, density, solid, True, 1000)
    mixed = (density + np.random.default_rng(74).random(res[::-1]).astype(np.float32)).astype(np.float32)
    out = torch.empty(res[::-1], dtype=torch.float32, device=cuda)
    hfgrid.op_build_mixed_fluid_outside_sdf(res, dev(density), dev(mixed), dev(grid_out), out)
    ref = oracle.build_mixed_fluid_outside_sdf(res, density, mixed, grid_out)
    assert np.array_equal(host(out), ref)
    surf = density == np.float32(0.2)
    assert surf.any() and (ref[surf] == 0).any() and (ref[surf] > 0).any()


def test_mix_field_with_density(cuda):
    """mixFieldWithDensity (HybridSimulatorMixFieldWithDensity.cu): cell and
    face grids, zero total weight leaves B unchanged."""
    rng = np.random.default_rng(62)
    n = int(np.prod(RES))
    wa = rng.random(RES[::-1]).astype(np.float32)
    wb = rng.random(RES[::-1]).astype(np.float32)
    wa[0, 0, :4] = 0.0
    wb[0, 0, :4] = 0.0
    a = rng.standard_normal(RES[::-1]).astype(np.float32)
    b = rng.standard_normal(RES[::-1]).astype(np.float32)
    bd = dev(b)
    hfgrid.op_mix_field_with_density_cc(dev(a), bd, dev(wa), dev(wb))
    np.testing.assert_allclose(host(bd), oracle.mix_field_with_density_cc(a, b, wa, wb).reshape(RES[::-1]),
                               rtol=1e-6, atol=1e-7)
    A = face_arrays(RES, rng)
    B = face_arrays(RES, rng)
    Bd = [dev(x) for x in B]
    hfgrid.op_mix_field_with_density_fc(RES, [dev(x) for x in A], Bd, dev(wa), dev(wb))
    ref = oracle.mix_field_with_density_fc(RES, A, B, wa, wb)
    for k in range(3):
        np.testing.assert_allclose(host(Bd[k]), ref[k], rtol=1e-6, atol=1e-7)
    assert n > 0


def test_mix_particle_vel_pic_flip(cuda):
    """mixParitcleVelWithPICAndFLIP: every distance band (PIC, PIC->predicted,
    FLIP, FLIP->predicted, predicted)."""
    rng = np.random.default_rng(63)
    n = 5000
    pic, flip, pred = (rng.standard_normal((n, 3)).astype(np.float32) for _ in range(3))
    dist = (rng.random(n) * 6.0 - 0.5).astype(np.float32)
    args = (0.1, 1.0, 2.0, 3.5, 5.0)
    pd = dev(pred)
    hfgrid.op_mix_particle_vel_pic_flip(dev(pic), dev(flip), dev(dist), *args, pd)
    ref = oracle.mix_particle_vel(pic, flip, dist, *args, pred)
    np.testing.assert_allclose(host(pd), ref, rtol=1e-6, atol=1e-6)
