"""One batch over several GPUs: the work-balanced shard plan
(tsu_shard_plan through tsunami_pact_b200/shard.py) and the gather of the
ranks' results back into pair order.

The plan is host code; the two-rank test runs it as gloo ranks on the CPU,
with the oracle standing in for each rank's GPU, and checks that the
gathered scores and operation strings equal one process's over the whole
batch."""
import json
import os
import socket

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _uneven(n, seed=11, lo=100, hi=2000):
    """Pairs with log-uniform lengths and 1-15 % edits (the mixed workload's
    shape at sizes the oracle finishes in seconds)."""
    from tsunami_pact_b200 import gen_batch

    rng = np.random.default_rng(seed)
    lengths = np.exp(rng.uniform(np.log(lo), np.log(hi), n)).astype(np.int32)
    rates = rng.uniform(0.01, 0.15, n)
    return gen_batch(0x5453554E414D49 + seed, lengths, rates)


def _pair_work(batch, hint=0.0):
    """Predicted work of every pair: a plan with one shard per pair puts
    each pair on its own shard."""
    from tsunami_pact_b200.shard import plan_by_work

    n = len(batch[2])
    of, w = plan_by_work(*batch, n, max_error_hint=hint)
    assert sorted(of.tolist()) == list(range(n))
    work = np.zeros(n)
    work[np.arange(n)] = w[of]
    return work


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_plan_is_balanced_and_deterministic(world):
    from tsunami_pact_b200.shard import plan_by_work

    batch = _uneven(600)
    of, w = plan_by_work(*batch, world)
    of2, w2 = plan_by_work(*batch, world)
    assert np.array_equal(of, of2) and np.array_equal(w, w2)
    assert of.min() >= 0 and of.max() < world
    work = _pair_work(batch)
    loads = np.array([work[of == r].sum() for r in range(world)])
    assert np.allclose(loads, w)
    # largest-first placement: no shard exceeds the mean by more than one pair
    assert w.max() <= w.sum() / world + work.max() + 1e-6


def test_plan_beats_equal_counts_on_uneven_pairs():
    """The estimate-based plan, scored by the pairs' true shapes
    ((length x edit rate)^2), loads 4 shards more evenly than contiguous
    equal-count slices."""
    from tsunami_pact_b200 import datasets
    from tsunami_pact_b200.shard import plan_by_work

    n, world = 4000, 4
    batch = datasets.generate("c4", n)
    lengths, rates, _ = datasets.shape("c4", n)
    true = (lengths * rates) ** 2 + lengths / 16.0
    of, _ = plan_by_work(*batch, world)
    plan = max(true[of == r].sum() for r in range(world)) / (true.sum() / world)
    slices = max(true[r * n // world:(r + 1) * n // world].sum() for r in range(world)) / (true.sum() / world)
    assert plan < slices and plan < 1.02, (plan, slices)


def test_plan_with_a_fixed_hint_needs_no_sequences():
    from tsunami_pact_b200.shard import plan_by_work

    plen = np.array([100, 5000, 300, 20000, 0, 7], dtype=np.int32)
    tlen = np.array([100, 5100, 290, 19000, 4, 0], dtype=np.int32)
    off = np.zeros(6, dtype=np.int64)
    of, w = plan_by_work(None, off, plen, None, off, tlen, 2, max_error_hint=0.1)
    # the longest pair alone on one shard
    assert (of == of[3]).sum() == 1
    with pytest.raises(Exception):  # estimating needs the sequence bytes
        plan_by_work(None, off, plen, None, off, tlen, 2)


def test_plan_rejects_bad_arguments():
    from tsunami_pact_b200 import AlignError
    from tsunami_pact_b200.shard import plan_by_work

    batch = _uneven(10)
    for kw in ({"world": 0}, {"world": 2, "penalties": (0, 6, 2)}, {"world": 2, "max_error_hint": -0.5},
               {"world": 2, "max_error_hint": 3.0}):
        world = kw.pop("world")
        with pytest.raises(AlignError):
            plan_by_work(*batch, world, **kw)
    bad = list(batch)
    bad[2] = batch[2].copy()
    bad[2][4] = -1
    with pytest.raises(AlignError):
        plan_by_work(*bad, 2)
    empty = (np.zeros(1, np.uint8), np.zeros(0, np.int64), np.zeros(0, np.int32)) * 2
    of, w = plan_by_work(*empty, 3)
    assert len(of) == 0 and list(w) == [0.0, 0.0, 0.0]


def test_take_packs_the_shard(oracle):
    from tsunami_pact_b200.shard import gather_results, plan_by_work, take

    batch = _uneven(200, seed=5, hi=600)
    pb, po, pl, tb, to, tl = batch
    of, _ = plan_by_work(*batch, 3)
    got_s, got_o = [], []
    idxs = []
    for r in range(3):
        idx, (a, b, c, d, e, f) = take(of, r, *batch)
        idxs.append(idx)
        assert np.all(np.diff(idx) > 0)
        for j, i in enumerate(idx):
            assert bytes(a[b[j]:b[j] + c[j]]) == bytes(pb[po[i]:po[i] + pl[i]])
            assert bytes(d[e[j]:e[j] + f[j]]) == bytes(tb[to[i]:to[i] + tl[i]])
        s, o = oracle.align_batch_arrays(a, b, c, d, e, f, 4, 6, 2, cigar=True, threads=2)
        got_s.append(s)
        got_o.append(o)
    assert sorted(np.concatenate(idxs).tolist()) == list(range(200))
    # gathering by hand (no process group): each shard's results placed
    scores = np.zeros(200, dtype=np.int32)
    ops = [None] * 200
    for idx, s, o in zip(idxs, got_s, got_o):
        part_s, part_o = gather_results(np.arange(len(idx)), s, o, len(idx))
        scores[idx] = part_s
        for j, i in enumerate(idx):
            ops[i] = part_o[j]
    ref_s, ref_o = oracle.align_batch_arrays(*batch, 4, 6, 2, cigar=True, threads=2)
    assert scores.tolist() == [int(x) for x in ref_s] and ops == ref_o
    with pytest.raises(ValueError):
        gather_results(np.array([0, 0]), np.array([1, 2]), None, 2)
    with pytest.raises(ValueError):
        gather_results(np.array([0]), np.array([1]), None, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime
    import sys

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    from oracle import oracle as O
    from tsunami_pact_b200.shard import gather_results, plan_by_work, take

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        batch = _uneven(240, seed=7, hi=800)
        of, work = plan_by_work(*batch, world)
        idx, shard_batch = take(of, rank, *batch)
        s, o = O.align_batch_arrays(*shard_batch, 4, 6, 2, cigar=True, threads=2)
        scores, ops = gather_results(idx, s, o, len(batch[2]), dist)
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"idx": idx.tolist(), "scores": scores.tolist(), "ops": ops, "of": of.tolist()}, f)
    finally:
        dist.destroy_process_group()


def test_two_ranks_plan_align_gather(tmp_path, oracle):
    pytest.importorskip("torch")
    import torch.multiprocessing as mp

    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    r = [json.load(open(tmp_path / f"rank{k}.json")) for k in range(world)]
    assert r[0]["of"] == r[1]["of"]  # the same plan on every rank
    assert set(r[0]["idx"]).isdisjoint(r[1]["idx"]) and len(r[0]["idx"]) + len(r[1]["idx"]) == 240
    batch = _uneven(240, seed=7, hi=800)
    ref_s, ref_o = oracle.align_batch_arrays(*batch, 4, 6, 2, cigar=True, threads=2)
    for x in r:  # every rank holds the whole batch's results in pair order
        assert x["scores"] == [int(v) for v in ref_s]
        assert x["ops"] == ref_o
