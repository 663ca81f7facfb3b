"""Multi-GPU scaling by replicas: every anneal is a pure function of (seed, trial id, couplings, tables), so ranks run
disjoint trial-id ranges with no exchange during the run; only the per-rank timings and success counts are reduced
at the end (max of the device times, sum of the counts), over torch.distributed (NCCL on GPUs, gloo on CPU)."""
from __future__ import annotations

TRIALS_PER_RANK = 1 << 20


def trial_base(rank: int) -> int:
    """First trial id of a rank's range [rank * 2^20, (rank + 1) * 2^20)."""
    return rank * TRIALS_PER_RANK


def _dist():
    import torch.distributed as dist
    return dist if dist.is_available() and dist.is_initialized() else None


def _device():
    import torch
    dist = _dist()
    if dist is not None and dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def reduce_max(x: float) -> float:
    """Max over ranks (the identity without a process group)."""
    dist = _dist()
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(values):
    """Element-wise sum over ranks of a list of integers."""
    dist = _dist()
    if dist is None:
        return [int(v) for v in values]
    import torch
    t = torch.tensor([int(v) for v in values], dtype=torch.int64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return [int(v) for v in t.tolist()]
