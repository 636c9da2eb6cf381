"""Several GPUs: per-rank workloads and the cross-rank reductions of a timed step.

Conformers are independent and the optimizer has no exchange step, so N GPUs
run N independent launches, one process per GPU, with torch.distributed as the
plumbing:

* weak scaling: every rank optimises its own seeded copy of a workload
  (``rank_seed``);
* strong scaling: the molecules of one workload are split across ranks by
  estimated cost, each molecule's conformers kept on one rank because they
  share its tables (``partition_molecules``).

The only collectives are the host-side reductions of a timed step: the step
time is the maximum over ranks and the converged counts are summed
(``reduce_step``).  No optimizer data crosses GPUs.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np


def rank_seed(base_seed: int, rank: int) -> int:
    """Seed of a rank's own copy of a workload (weak scaling)."""
    return int(base_seed) + int(rank)


def molecule_cost(n_atoms: Sequence[int], conf_counts: Sequence[int]) -> np.ndarray:
    """Relative optimisation cost of each molecule: conformers x atoms squared.

    The inverse-Hessian pass and the non-bonded pairs both grow with N^2 per
    iteration, and they dominate an iteration.
    """
    n = np.asarray(n_atoms, dtype=np.float64)
    return np.asarray(conf_counts, dtype=np.float64) * n * n


def partition_molecules(costs: Sequence[float], world: int) -> list[np.ndarray]:
    """Split molecule indices over ``world`` ranks, largest cost first onto the least-loaded rank.

    Deterministic (ties go to the lower rank and to the lower molecule index);
    every molecule lands on exactly one rank; each rank's indices are returned
    in ascending order.
    """
    if world < 1:
        raise ValueError("world must be >= 1")
    costs = np.asarray(costs, dtype=np.float64)
    order = np.lexsort((np.arange(len(costs)), -costs))
    load = np.zeros(world)
    parts: list[list[int]] = [[] for _ in range(world)]
    for m in order:
        r = int(np.argmin(load))
        parts[r].append(int(m))
        load[r] += costs[m]
    return [np.array(sorted(p), dtype=np.int64) for p in parts]


def reduce_step(dist, ms: float, converged: float, device="cpu") -> tuple[float, float]:
    """Whole-job figures of a timed step: (max step time over ranks, summed converged count).

    ``dist`` is ``torch.distributed`` with an initialised process group, or None
    for a single process.  ``device`` is where the reduction tensors live (the
    rank's GPU under NCCL, the CPU under gloo).
    """
    if dist is None:
        return float(ms), float(converged)
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    c = torch.tensor([float(converged)], dtype=torch.float64, device=device)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t.item()), float(c.item())
