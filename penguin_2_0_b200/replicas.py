"""Multi-GPU use of the hydro step: independent replicas, one per rank.

The path has no exchange step at the workload sizes (one disk fits one GPU),
so N GPUs advance N independent disks (ensemble members / served runs); the
only collective is a max over ranks of the timed region, which is how the
whole-job throughput is reported.  No halo exchange is built (the
reference's radial slab split, main.cu:145-188 / ppm.cu:326-355, is a
single-run decomposition for disks larger than one GPU's memory).
"""
from __future__ import annotations


def rank_params(p, rank: int):
    """The disk a rank advances: same workload, its own noise seed."""
    import copy
    q = copy.copy(p)
    q.seed = int(p.seed) + rank
    return q


def max_over_ranks(x: float, dist=None, device: str = "cpu") -> float:
    """Max of a per-rank scalar (elapsed time) over the process group."""
    if dist is None or not dist.is_initialized():
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(cells_per_rank: int, steps: int, world: int, t_max_s: float) -> float:
    """Whole-job zone-updates/s: all ranks' cells x steps over the slowest rank."""
    return cells_per_rank * steps * world / t_max_s
