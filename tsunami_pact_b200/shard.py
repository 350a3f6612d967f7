"""Data-parallel sharding of a batch over ranks (one process per GPU).

Pairs are independent, so N GPUs align N shards with no collective on the
data path (weak scaling: rank r aligns its own n pairs, pair indices
[r*n, (r+1)*n) of the seeded workload).  Collectives only line the ranks up
around the timed region and combine what they measured: the step time is the
maximum over ranks, work (cells, pairs) the sum, so the whole-job throughput
is the summed work over the slowest rank's time.
"""
from __future__ import annotations

from typing import Optional, Sequence, Tuple


def shard(rank: int, world: int, n_per_rank: int) -> Tuple[int, int]:
    """(first pair index, pair count) of a rank's shard."""
    if not 0 <= rank < world or n_per_rank < 0:
        raise ValueError(f"rank {rank} of {world}, {n_per_rank} pairs per rank")
    return rank * n_per_rank, n_per_rank


def combine(values: Sequence[float], ops: Sequence[str], dist=None, device=None) -> list:
    """Reduce per-rank figures over all ranks: each value with its op
    ("max" or "sum").  Without a process group the values come back as they
    are.  device: where the reduction tensor lives (CUDA for NCCL, CPU for
    gloo)."""
    if len(values) != len(ops) or any(o not in ("max", "sum") for o in ops):
        raise ValueError("one op, max or sum, per value")
    if dist is None:
        return [float(v) for v in values]
    import torch

    out = [0.0] * len(values)
    for op_name, op in (("max", dist.ReduceOp.MAX), ("sum", dist.ReduceOp.SUM)):
        idx = [i for i, o in enumerate(ops) if o == op_name]
        if not idx:
            continue
        t = torch.tensor([float(values[i]) for i in idx], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=op)
        for j, i in enumerate(idx):
            out[i] = float(t[j].item())
    return out


def throughput(work: float, ms_max: float) -> float:
    """Whole-job rate: summed work per second of the slowest rank."""
    return work / (ms_max / 1e3) if ms_max > 0 else 0.0


def barrier(dist=None, device: Optional[object] = None) -> None:
    """Synchronise the device (if CUDA) and the ranks."""
    if device is not None and str(device).startswith("cuda"):
        import torch

        torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
