"""Host-side multi-GPU plumbing for independent scenes.

One scene never spans GPUs (its grid step has no exchange step on one GPU's
worth of cells), so N GPUs run N independent workloads: replicas of one scene
for the benchmark (weak scaling), or a set of scenes split across ranks by
their device-memory footprint.  No collective touches the data path; the only
collectives are the barrier / max reduction of the timing and the scene
assignment agreement.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple


def scene_bytes(res: Sequence[int], particles: int, boundaries: int = 1, precond: int = 1) -> int:
    """Device bytes of one scene: the library's own accounting
    (hfg_scene_bytes), the footprint the scene server admits by."""
    import hfgrid
    return hfgrid.scene_bytes(tuple(int(v) for v in res), int(particles), boundaries, precond)


def assign_scenes(footprints: Sequence[int], n_ranks: int, budget: int) -> Tuple[List[List[int]], List[int]]:
    """Greedy largest-first placement of scenes on ranks under a per-rank
    byte budget.  Returns (scene indices per rank, rejected scene indices).
    Deterministic: every rank computes the same answer from the same input."""
    order = sorted(range(len(footprints)), key=lambda i: (-footprints[i], i))
    load = [0] * n_ranks
    placed: List[List[int]] = [[] for _ in range(n_ranks)]
    rejected: List[int] = []
    for i in order:
        r = min(range(n_ranks), key=lambda k: (load[k], k))
        if load[r] + footprints[i] > budget:
            rejected.append(i)
            continue
        load[r] += footprints[i]
        placed[r].append(i)
    for p in placed:
        p.sort()
    return placed, sorted(rejected)


def max_over_ranks(value: float, device=None) -> float:
    """Max of `value` over all ranks of the default process group (identity
    without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def agree(values: Sequence[int], device=None) -> bool:
    """True when every rank passed the same integer list (checked by a max
    and a min reduction of each entry)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return True
    t = torch.tensor(list(values), dtype=torch.int64, device=device or "cpu")
    hi, lo = t.clone(), t.clone()
    dist.all_reduce(hi, op=dist.ReduceOp.MAX)
    dist.all_reduce(lo, op=dist.ReduceOp.MIN)
    return bool(torch.equal(hi, lo))
