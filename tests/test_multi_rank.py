"""The N > 1 path of the benchmark on the CPU: two ranks over gloo.

Each rank takes its shard of a seeded workload (tsunami_pact_b200/shard.py),
aligns it -- with the oracle standing in for the GPU, which this path does
not need to be tested -- times it, and the ranks combine their figures the
way bench.py does (step time: max over ranks; cells and pairs: sum).  The
test checks that the shards are disjoint and together are the first 2n pairs
of the workload, that the concatenated per-rank results equal a single
process's over those 2n pairs, and the combined figures."""
import json
import os
import socket

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
N_PER_RANK = 300


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import sys
    import time

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist

    from oracle import oracle as O
    from tsunami_pact_b200 import datasets
    from tsunami_pact_b200.shard import barrier, combine, shard, throughput

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        first, n = shard(rank, world, N_PER_RANK)
        pb, po, pl, tb, to, tl = datasets.generate("c1", n, first=first)
        barrier(dist)
        t0 = time.perf_counter()
        scores, ops = O.align_batch_arrays(pb, po, pl, tb, to, tl, 4, 6, 2, cigar=True, threads=2)
        ms = (time.perf_counter() - t0) * 1e3 + 50.0 * rank  # rank 1 reports the slower step
        barrier(dist)
        cells = float(np.sum(pl.astype(np.float64) * tl))
        ms_max, cells_all, pairs_all = combine([ms, cells, float(n)], ["max", "sum", "sum"], dist)
        pats = [bytes(pb[po[i]:po[i] + pl[i]]).decode() for i in range(n)]
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"first": first, "n": n, "scores": [int(x) for x in scores], "ops": ops, "pats": pats,
                       "ms": ms, "ms_max": ms_max, "cells": cells, "cells_all": cells_all, "pairs_all": pairs_all,
                       "value": throughput(cells_all, ms_max)}, f)
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo(tmp_path):
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp

    from oracle import oracle as O
    from tsunami_pact_b200 import datasets
    from tsunami_pact_b200.shard import shard

    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    r = [json.load(open(tmp_path / f"rank{k}.json")) for k in range(world)]
    # disjoint shards covering [0, 2n)
    assert [x["first"] for x in r] == [0, N_PER_RANK] and all(x["n"] == N_PER_RANK for x in r)
    assert shard(1, 2, N_PER_RANK) == (N_PER_RANK, N_PER_RANK)
    with pytest.raises(ValueError):
        shard(2, 2, N_PER_RANK)
    # per-rank results concatenated = one process over the union
    pb, po, pl, tb, to, tl = datasets.generate("c1", world * N_PER_RANK)
    scores, ops = O.align_batch_arrays(pb, po, pl, tb, to, tl, 4, 6, 2, cigar=True, threads=2)
    pats = [bytes(pb[po[i]:po[i] + pl[i]]).decode() for i in range(len(pl))]
    assert r[0]["pats"] + r[1]["pats"] == pats
    assert r[0]["scores"] + r[1]["scores"] == [int(x) for x in scores]
    assert r[0]["ops"] + r[1]["ops"] == ops
    # combined figures: max time, summed work, identical on every rank
    for x in r:
        assert x["ms_max"] == pytest.approx(max(y["ms"] for y in r))
        assert x["cells_all"] == pytest.approx(sum(y["cells"] for y in r))
        assert x["pairs_all"] == world * N_PER_RANK
        assert x["value"] == pytest.approx(x["cells_all"] / (x["ms_max"] / 1e3))
