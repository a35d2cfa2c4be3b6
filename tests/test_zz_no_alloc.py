"""hfg_op_p2g_fc_static, the allocation-free P2G onto the face grids, against
hfg_op_p2g_fc on the same inputs.

Collected last (file name) so it also runs after every other GPU test has used
the device; it passes alone in a fresh process too.  Two calls in a row with
different particles show that each call starts from zeroed accumulators.
"""
import ctypes

import numpy as np
import pytest
import torch

import hfgrid
import oracle

RES = (21, 17, 13)
ORIGIN = (0.1, -0.3, 0.2)
SPACING = (0.05, 0.06, 0.07)


def _particles(rng, n):
    lo = np.array(ORIGIN) - 0.5 * np.array(SPACING)
    hi = np.array(ORIGIN) + (np.array(RES) + 0.5) * np.array(SPACING)
    pos = (lo + rng.random((n, 3)) * (hi - lo)).astype(np.float32)
    vel = rng.standard_normal((n, 3)).astype(np.float32)
    return pos, vel


# (nx+1) ny nz + nx (ny+1) nz + nx ny (nz+1) faces: exactly the limit, and one over
AT_LIMIT = (33, 46, 226)     # 1,048,576 faces
ONE_OVER = (17, 85, 236)     # 1,048,577 faces


def _faces(res):
    return sum(int(np.prod(s)) for s in oracle.face_shapes(res))


@pytest.mark.parametrize("res", [ONE_OVER, (101, 100, 100)])
def test_static_p2g_rejects_oversized_grids(res):
    """The size check comes before any device work, so it runs without a GPU."""
    assert _faces(ONE_OVER) == (1 << 20) + 1 and _faces(AT_LIMIT) == 1 << 20
    lib = hfgrid.lib()
    out = ctypes.c_void_p(16)  # never dereferenced: the call is rejected first
    rc = lib.hfg_op_p2g_fc_static(hfgrid._i3(res), hfgrid._f3(ORIGIN), hfgrid._f3(SPACING), None, None,
                                  0, 2, out, out, out, None, None, None, None)
    assert rc == -1  # HFG_ERR_INVALID
    msg = lib.hfg_last_error().decode()
    assert "1048576" in msg and "hfg_op_p2g_fc" in msg


@pytest.mark.gpu
@pytest.mark.parametrize("alg", [hfgrid.LINEAR, hfgrid.QUADRATIC, hfgrid.CUBIC, hfgrid.P2GSUM])
def test_static_p2g_matches_allocating_entry_point(cuda, alg):
    rng = np.random.default_rng(70 + alg)
    shapes = oracle.face_shapes(RES)
    for n in (40000, 9000):  # two calls in a row, different particle sets
        pos, vel = _particles(rng, n)
        pd, vd = torch.from_numpy(pos).to(cuda), torch.from_numpy(vel).to(cuda)
        ref = [torch.empty(s, dtype=torch.float32, device=cuda) for s in shapes]
        ref_w = [torch.empty(s, dtype=torch.float32, device=cuda) for s in shapes]
        got = [torch.full(s, np.nan, dtype=torch.float32, device=cuda) for s in shapes]
        got_w = [torch.full(s, np.nan, dtype=torch.float32, device=cuda) for s in shapes]
        hfgrid.op_p2g_fc(RES, ORIGIN, SPACING, pd, vd, alg, ref, ref_w)
        hfgrid.op_p2g_fc_static(RES, ORIGIN, SPACING, pd, vd, alg, got, got_w)
        torch.cuda.synchronize()
        for a in range(3):
            # atomics add in a different order on each call: FP32 rounding only
            r, g = ref[a].cpu().numpy(), got[a].cpu().numpy()
            rw, gw = ref_w[a].cpu().numpy(), got_w[a].cpu().numpy()
            np.testing.assert_allclose(gw, rw, rtol=1e-5, atol=1e-5 * max(1.0, float(np.abs(rw).max())))
            np.testing.assert_allclose(g, r, rtol=1e-4, atol=1e-5 * max(1.0, float(np.abs(r).max())))
    # a grid of exactly 2^20 faces: the z faces end on the array's last entry
    res = AT_LIMIT
    assert _faces(res) == 1 << 20
    rng = np.random.default_rng(79)
    pos = (rng.random((300000, 3)) * np.array(res)).astype(np.float32)
    vel = rng.standard_normal((300000, 3)).astype(np.float32)
    pd, vd = torch.from_numpy(pos).to(cuda), torch.from_numpy(vel).to(cuda)
    ref = [torch.empty(s, dtype=torch.float32, device=cuda) for s in oracle.face_shapes(res)]
    got = [torch.empty(s, dtype=torch.float32, device=cuda) for s in oracle.face_shapes(res)]
    hfgrid.op_p2g_fc(res, (0, 0, 0), (1, 1, 1), pd, vd, alg, ref)
    hfgrid.op_p2g_fc_static(res, (0, 0, 0), (1, 1, 1), pd, vd, alg, got)
    for a in range(3):
        r, g = ref[a].cpu().numpy(), got[a].cpu().numpy()
        np.testing.assert_allclose(g, r, rtol=1e-4, atol=1e-5 * max(1.0, float(np.abs(r).max())))
