"""Failure paths of the library, none of which faults or hangs a GPU.

* Every wait of the TMA-fed CG kernels (an mbarrier per stage) and of the
  cooperative extrapolation (a grid barrier between layers) is bounded: the
  self-test runs the same wait helpers against conditions nothing satisfies
  and checks that both give up, report it and leave the context usable.
* A device allocation failure, injected on the host, surfaces as
  HFG_ERR_NOMEM from the call that allocates, frees what the call had
  allocated, and leaves later calls working.
* A solve stopped by its iteration cap reports it (not converged, the
  iteration count) and the step still completes.
"""
import numpy as np
import pytest
import torch

import hfgrid
import scenes

pytestmark = pytest.mark.gpu

HFG_ERR_NOMEM = -3


def _small_step():
    sc = scenes.Scene(res=(16, 14, 12), seed=3)
    g = scenes.gpu_solver(sc, precond=1, tol_mode=1, tol=1e-6, max_iter=400)
    g.update()
    return g


def test_bounded_waits_give_up_and_context_survives(cuda):
    mb, gb = hfgrid.selftest_bounded_waits(20)
    assert (mb, gb) == (1, 1)
    g = _small_step()  # the context still runs kernels
    assert g.stats()["cg_converged"] == 1


@pytest.mark.parametrize("after", [1, 7, 25])
def test_injected_allocation_failure(cuda, after):
    sc = scenes.Scene(res=(24, 20, 16), seed=3)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    hfgrid.inject_alloc_failure(after)
    with pytest.raises(hfgrid.HfgError) as e:
        scenes.gpu_solver(sc)
    hfgrid.inject_alloc_failure(0)
    assert e.value.code == HFG_ERR_NOMEM
    assert "injected" in str(e.value)
    torch.cuda.synchronize()
    # what the failed constructor had allocated went back (the stream-ordered
    # pool may keep a little cached)
    assert torch.cuda.mem_get_info()[0] > free0 - (64 << 20)
    g = _small_step()
    assert g.stats()["cg_iterations"] > 0


def test_iteration_cap_reports_not_converged(cuda):
    sc = scenes.Scene(res=(20, 18, 16), seed=3)
    g = scenes.gpu_solver(sc, precond=1, tol_mode=1, tol=1e-6, max_iter=1)
    g.update()
    g.update()
    st = g.stats()
    assert st["cg_iterations"] == 1 and st["cg_converged"] == 0
    assert st["cg_residual"] > 1e-6 * st["cg_rhs_norm"]
    vel = g.velocity_field()
    assert all(np.isfinite(v[v != np.finfo(np.float32).max]).all() for v in vel)
