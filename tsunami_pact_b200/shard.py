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


# ---- one batch over several GPUs (strong scaling) ---------------------------
# A job that holds ONE batch splits it by predicted work rather than by pair
# count: the lengths of a mixed batch span two orders of magnitude and a
# pair's work grows with the square of its score, so equal pair counts leave
# the GPUs unevenly loaded.  Every rank computes the same plan
# (tsu_shard_plan is deterministic), aligns its own pairs with no
# communication, and the results meet in pair order on the host.


def plan_by_work(pbuf, poff, plen, tbuf, toff, tlen, world: int, penalties=(4, 6, 2), max_error_hint: float = 0.0):
    """Shard of every pair and predicted work per shard, from the native
    planner tsu_shard_plan (largest pair first onto the least-loaded shard;
    max_error_hint 0 estimates each pair's edit rate from shared k-mers)."""
    import ctypes

    import numpy as np

    from ._lib import TSU_OK, AlignError, Batch, Penalties, _ptr, lib

    plen = np.ascontiguousarray(plen, dtype=np.int32)
    tlen = np.ascontiguousarray(tlen, dtype=np.int32)
    poff = np.ascontiguousarray(poff, dtype=np.int64)
    toff = np.ascontiguousarray(toff, dtype=np.int64)
    n = len(plen)
    if len(tlen) != n or len(poff) != n or len(toff) != n:
        raise ValueError("offset and length arrays differ in size")
    of = np.zeros(max(n, 1), dtype=np.int32)
    work = np.zeros(max(world, 1), dtype=np.float64)
    b = Batch(n, _ptr(pbuf), _ptr(poff), _ptr(plen), _ptr(tbuf), _ptr(toff), _ptr(tlen))
    L = lib()
    rc = L.tsu_shard_plan(ctypes.byref(Penalties(*penalties)), ctypes.byref(b), int(world), float(max_error_hint),
                          _ptr(of), _ptr(work))
    if rc != TSU_OK:
        raise AlignError(rc, L.tsu_status_str(rc).decode())
    return of[:n], work[:world]


def _gather_seqs(buf, off, ln, idx, block: int = 1 << 16):
    """Sequences idx of (buf, off, ln) copied into one new buffer."""
    import numpy as np

    lens = ln[idx].astype(np.int64)
    new_off = np.zeros(len(idx), dtype=np.int64)
    if len(idx) > 1:
        np.cumsum(lens[:-1], out=new_off[1:])
    total = int(lens.sum())
    out = np.zeros(total + 1, dtype=np.uint8)
    for a in range(0, len(idx), block):  # bounded index arrays per block
        i, l, d = idx[a:a + block], lens[a:a + block], new_off[a:a + block]
        cnt = int(l.sum())
        if cnt == 0:
            continue
        start = int(d[0])
        src = np.repeat(off[i] - (d - start), l) + np.arange(cnt, dtype=np.int64)
        out[start:start + cnt] = buf[src]
    return out, new_off, ln[idx].astype(np.int32)


def take(shard_of_pair, rank: int, pbuf, poff, plen, tbuf, toff, tlen):
    """(pair indices, compact batch) of one rank's shard: the indices in
    increasing order and the six batch arrays with the shard's sequences
    packed contiguously, ready for Aligner.align_arrays."""
    import numpy as np

    idx = np.flatnonzero(np.asarray(shard_of_pair) == rank)
    pb, po, pl = _gather_seqs(pbuf, poff, plen, idx)
    tb, to, tl = _gather_seqs(tbuf, toff, tlen, idx)
    return idx, (pb, po, pl, tb, to, tl)


def gather_results(idx, scores, cigars, n_total: int, dist=None):
    """Every rank's (pair indices, scores, per-pair CIGARs) put back in pair
    order, on every rank (one all_gather of host objects; without a process
    group the rank's own results are placed as they are).  cigars: a list
    with one entry per pair of the shard (operation strings or run arrays),
    or None for scores only."""
    import numpy as np

    parts = [(np.asarray(idx), np.asarray(scores), cigars)]
    if dist is not None:
        parts = [None] * dist.get_world_size()
        dist.all_gather_object(parts, (np.asarray(idx), np.asarray(scores), cigars))
    out_scores = np.zeros(n_total, dtype=np.int32)
    out_cigars = [None] * n_total if any(c is not None for _, _, c in parts) else None
    seen = np.zeros(n_total, dtype=bool)
    for i, s, c in parts:
        if seen[i].any():
            raise ValueError("a pair appears in two shards")
        seen[i] = True
        out_scores[i] = s
        if out_cigars is not None and c is not None:
            for j, p in enumerate(i):
                out_cigars[int(p)] = c[j]
    if not seen.all():
        raise ValueError("pairs missing from every shard")
    return out_scores, out_cigars
