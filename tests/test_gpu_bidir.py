"""Bidirectional mode (TSU_BIDIRECTIONAL) on the GPU.  Scores: the
breakpoint kernel (tsu_bidir.cuh) over whole pairs; its crossing totals must
equal the oracle's optimal scores (the forward engine's too) on random pairs
of every size class, unequal and empty pairs and pairs with bytes outside
ACGT.  CIGARs: the recursion on crossings with base-case segments
(tsu_segment.cuh); every pair's operations must equal the oracle's
bidirectional alignment (ora_bialign_ring) with the same base score, byte
for byte, and cost the optimal score.  Argument checks; device memory of a
50 kbp pair against the forward pass."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _batch(T, seed, lengths, rates):
    return T.gen_batch(seed, np.asarray(lengths, np.int32), np.asarray(rates))


@pytest.mark.parametrize("pen", [(4, 6, 2), (3, 5, 1), (5, 11, 3)])
def test_bidirectional_scores_equal_the_oracle(aligner_factory, oracle, pen):
    import tsunami_pact_b200 as T

    rng = np.random.default_rng(sum(pen))
    lengths = np.concatenate([rng.integers(0, 400, 600), rng.integers(400, 3000, 60), [0, 1, 5000]])
    rates = np.concatenate([rng.uniform(0, 0.2, 660), [0.0, 1.0, 0.1]])
    pb, po, pl, tb, to, tl = _batch(T, 11 + pen[0], lengths, rates)
    al = aligner_factory(pen)
    got, _, _ = al.align_arrays(pb, po, pl, tb, to, tl, cigar=False, bidirectional=True)
    want, _ = oracle.align_batch_arrays(pb, po, pl, tb, to, tl, *pen, cigar=False)
    assert np.array_equal(got, want), np.nonzero(got != want)[0][:10]
    fwd, _, _ = al.align_arrays(pb, po, pl, tb, to, tl, cigar=False)
    assert np.array_equal(got, fwd)


def test_bidirectional_unequal_and_non_acgt(aligner_factory, oracle):
    rng = np.random.default_rng(3)
    pats, txts = [], []
    for i in range(300):
        alpha = list("ACGTN") if i % 5 == 0 else list("ACGT")
        p = "".join(rng.choice(alpha, rng.integers(0, 300)))
        t = "".join(rng.choice(alpha, rng.integers(0, 300))) if i % 7 == 0 else p[: max(0, len(p) - 17)] + "ACG"
        pats.append(p)
        txts.append(t)
    al = aligner_factory((4, 6, 2))
    import tsunami_pact_b200 as T
    from tsunami_pact_b200._lib import _concat

    pb, po, pl = _concat(pats)
    tb, to, tl = _concat(txts)
    got, _, _ = al.align_arrays(pb, po, pl, tb, to, tl, cigar=False, bidirectional=True)
    want, _ = oracle.align_batch(pats, txts, 4, 6, 2, cigar=False)
    assert np.array_equal(got, want)
    assert T.TSU_BIDIRECTIONAL == 4


def test_bidirectional_long_pairs(aligner_factory, oracle):
    import tsunami_pact_b200 as T

    pb, po, pl, tb, to, tl = _batch(T, 21, [10_000] * 6 + [20_000] * 2, [0.15] * 6 + [0.05] * 2)
    al = aligner_factory((4, 6, 2))
    got, _, _ = al.align_arrays(pb, po, pl, tb, to, tl, cigar=False, bidirectional=True)
    want, _ = oracle.align_batch_arrays(pb, po, pl, tb, to, tl, 4, 6, 2, cigar=False)
    assert np.array_equal(got, want)


def test_bidirectional_argument_checks(oracle):
    import tsunami_pact_b200 as T

    pb, po, pl, tb, to, tl = _batch(T, 5, [100] * 4, [0.05] * 4)
    with T.Aligner(4, 6, 2, gap_opening2=24, gap_extension2=1) as al:
        with pytest.raises(T.AlignError):  # one gap piece only
            al.align_arrays(pb, po, pl, tb, to, tl, cigar=False, bidirectional=True)
    with T.Aligner(4, 6, 2) as al:
        al.set_ends_free(10, 10, 10, 10)
        with pytest.raises(T.AlignError):  # end to end only
            al.align_arrays(pb, po, pl, tb, to, tl, cigar=False, bidirectional=True)
        with pytest.raises(T.AlignError):  # CIGARs too
            al.align_arrays(pb, po, pl, tb, to, tl, cigar=True, bidirectional=True)


def base_score(pen):
    """The base score of the recursion in penalty units: segments whose
    crossing total is at most max(2 max(x, o + e), 256) score units are
    aligned whole."""
    g = math.gcd(*pen)
    x, go = pen[0] // g, (pen[1] + pen[2]) // g
    return max(2 * max(x, go), 256) * g


def _check_cigars(T, oracle, al, pen, pb, po, pl, tb, to, tl):
    got, coff, runs = al.align_arrays(pb, po, pl, tb, to, tl, cigar=True, bidirectional=True)
    want, _ = oracle.align_batch_arrays(pb, po, pl, tb, to, tl, *pen, cigar=False)
    assert np.array_equal(got, want), np.nonzero(got != want)[0][:10]
    base = base_score(pen)
    for i in range(len(pl)):
        p = bytes(pb[po[i]:po[i] + pl[i]])
        t = bytes(tb[to[i]:to[i] + tl[i]])
        ops = T.runs_to_ops(runs[coff[i]:coff[i + 1]])
        ref = oracle.bialign(p, t, *pen, base_score=base, ring=True)
        assert ops == ref, (i, len(p), len(t))
        assert oracle.cigar_cost(ops, p, t, *pen) == want[i]


@pytest.mark.parametrize("pen", [(4, 6, 2), (3, 5, 1), (5, 11, 3), (20, 1, 1)])
def test_bidirectional_cigars_equal_the_oracle(aligner_factory, oracle, pen):
    import tsunami_pact_b200 as T

    rng = np.random.default_rng(7 + sum(pen))
    lengths = np.concatenate([rng.integers(0, 300, 300), rng.integers(300, 2500, 40), [0, 1, 2, 4000]])
    rates = np.concatenate([rng.uniform(0, 0.25, 340), [0.0, 1.0, 0.5, 0.12]])
    pb, po, pl, tb, to, tl = _batch(T, 31 + pen[1], lengths, rates)
    _check_cigars(T, oracle, aligner_factory(pen), pen, pb, po, pl, tb, to, tl)


def test_bidirectional_cigars_unequal_and_non_acgt(aligner_factory, oracle):
    import tsunami_pact_b200 as T
    from tsunami_pact_b200._lib import _concat

    rng = np.random.default_rng(13)
    pats, txts = [], []
    for i in range(200):
        alpha = list("ACGTN") if i % 5 == 0 else list("ACGT")
        p = "".join(rng.choice(alpha, rng.integers(0, 400)))
        if i % 7 == 0:
            t = "".join(rng.choice(alpha, rng.integers(0, 400)))
        elif i % 7 == 1:
            t = ""
        else:
            t = p[: max(0, len(p) - 23)] + "ACGTTG" + p[len(p) // 2:]
        pats.append(p)
        txts.append(t)
    pb, po, pl = _concat(pats)
    tb, to, tl = _concat(txts)
    _check_cigars(T, oracle, aligner_factory((4, 6, 2)), (4, 6, 2), pb, po, pl, tb, to, tl)


def test_bidirectional_cigars_long_pairs(aligner_factory, oracle):
    import tsunami_pact_b200 as T

    pb, po, pl, tb, to, tl = _batch(T, 41, [10_000, 10_000, 20_000], [0.15, 0.02, 0.05])
    _check_cigars(T, oracle, aligner_factory((4, 6, 2)), (4, 6, 2), pb, po, pl, tb, to, tl)


def test_bidirectional_cigars_device_entry(aligner_factory, oracle):
    """The device-resident entry point gives the same runs as the host one."""
    import torch

    import tsunami_pact_b200 as T

    pb, po, pl, tb, to, tl = _batch(T, 51, [150] * 200 + [1000] * 20, [0.05] * 220)
    al = aligner_factory((4, 6, 2))
    s0, c0, r0 = al.align_arrays(pb, po, pl, tb, to, tl, cigar=True, bidirectional=True)

    def d(a):
        return torch.from_numpy(np.ascontiguousarray(a)).cuda()

    n = len(pl)
    sc = torch.zeros(n, dtype=torch.int32, device="cuda")
    off = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    runs = torch.zeros(int(c0[-1]) + 16, dtype=torch.int32, device="cuda")
    st = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    used = al.align_device(d(pb), d(po), d(pl), d(tb), d(to), d(tl), sc, runs, off, st, bidirectional=True)
    assert used == int(c0[-1])
    assert np.array_equal(sc.cpu().numpy(), s0)
    assert np.array_equal(off.cpu().numpy(), c0)
    assert np.array_equal(runs.cpu().numpy()[:used].view(np.uint32), r0)
    assert (st.cpu().numpy() == 0).all()


def test_bidirectional_memory_50kbp(oracle):
    """One 50 kbp pair at 20 % edits: the bidirectional CIGAR holds a small
    fraction of the device memory of the forward pass's history (fresh
    contexts, so no workspace is carried over), with the same score and a
    CIGAR of that cost."""
    import tsunami_pact_b200 as T

    pb, po, pl, tb, to, tl = _batch(T, 61, [50_000], [0.2])
    with T.Aligner(4, 6, 2) as al:
        s0, c0, r0 = al.align_arrays(pb, po, pl, tb, to, tl, cigar=True)
        fwd_bytes = al.timing()["device_bytes"]
    with T.Aligner(4, 6, 2) as al:
        s1, c1, r1 = al.align_arrays(pb, po, pl, tb, to, tl, cigar=True, bidirectional=True)
        bi_bytes = al.timing()["device_bytes"]
    assert s1[0] == s0[0]
    p, t = bytes(pb[: pl[0]]), bytes(tb[: tl[0]])
    assert oracle.cigar_cost(T.runs_to_ops(r1), p, t, 4, 6, 2) == s0[0]
    print(f"50 kbp @ 20 %: score {s0[0]}, device bytes forward {fwd_bytes / 1e6:.1f} MB, "
          f"bidirectional {bi_bytes / 1e6:.1f} MB")
    assert 0 < bi_bytes < fwd_bytes / 4


def test_bidirectional_chunked_host_pipeline(aligner_factory, oracle):
    """300,000 pairs from host buffers run as a pipeline of chunks (one
    recursion per chunk): the same scores and runs as the same pairs in
    calls of 60,000 (one chunk each), and the scores of the forward pass."""
    import tsunami_pact_b200 as T

    rng = np.random.default_rng(71)
    n = 300_000
    pb, po, pl, tb, to, tl = _batch(T, 71, rng.integers(20, 120, n), rng.uniform(0.0, 0.3, n))
    al = aligner_factory((4, 6, 2))
    s, c, r = al.align_arrays(pb, po, pl, tb, to, tl, cigar=True, bidirectional=True)
    fwd, _, _ = al.align_arrays(pb, po, pl, tb, to, tl, cigar=False)
    assert np.array_equal(s, fwd)
    step = 60_000
    for a in range(0, n, step):
        sl = slice(a, a + step)
        s1, c1, r1 = al.align_arrays(pb, po[sl], pl[sl], tb, to[sl], tl[sl], cigar=True, bidirectional=True)
        assert np.array_equal(s1, s[sl])
        assert np.array_equal(c1, c[a:a + step + 1] - c[a])
        assert np.array_equal(r1, r[c[a]:c[min(a + step, n)]])
    for i in range(0, n, 9973):  # a sample against the oracle's recursion
        p, t = bytes(pb[po[i]:po[i] + pl[i]]), bytes(tb[to[i]:to[i] + tl[i]])
        assert T.runs_to_ops(r[c[i]:c[i + 1]]) == oracle.bialign(p, t, 4, 6, 2, base_score=base_score((4, 6, 2)),
                                                                 ring=True)


def test_bidirectional_tight_budget(aligner_factory):
    """Under a 64 MB device budget the breakpoint groups, the leaf warps and
    the run arena shrink to fit, and the results stay those of the default
    budget."""
    import tsunami_pact_b200 as T

    rng = np.random.default_rng(81)
    lengths = np.concatenate([rng.integers(100, 1500, 1500), [10_000, 10_000, 6_000]])
    rates = np.concatenate([rng.uniform(0.0, 0.2, 1500), [0.15, 0.05, 0.3]])
    pb, po, pl, tb, to, tl = _batch(T, 81, lengths, rates)
    s0, c0, r0 = aligner_factory((4, 6, 2)).align_arrays(pb, po, pl, tb, to, tl, cigar=True, bidirectional=True)
    with T.Aligner(4, 6, 2, mem_budget=64 << 20) as al:
        s1, c1, r1 = al.align_arrays(pb, po, pl, tb, to, tl, cigar=True, bidirectional=True)
        assert al.timing()["device_bytes"] <= 64 << 20
    assert np.array_equal(s0, s1)
    assert np.array_equal(c0, c1)
    assert np.array_equal(r0, r1)


@pytest.mark.parametrize("metric,xe", [("edit", (1, 1)), ("indel", (3, 1)), ("gap_linear", (2, 1))])
def test_bidirectional_gap_linear_metrics(oracle, metric, xe):
    """Edit, indel and gap-linear contexts run the bidirectional mode as
    gap-affine with a zero gap opening: scores equal the linear oracle's (and
    the forward kernels'), CIGARs equal the oracle's recursion at o = 0 and
    cost the score."""
    import tsunami_pact_b200 as T

    x, e = xe
    rng = np.random.default_rng(91 + x)
    lengths = np.concatenate([rng.integers(0, 400, 250), rng.integers(400, 3000, 20), [0, 1, 6000]])
    rates = np.concatenate([rng.uniform(0, 0.25, 270), [0.0, 1.0, 0.2]])
    pb, po, pl, tb, to, tl = _batch(T, 91 + x, lengths, rates)
    kw = {"metric": metric}
    args = (x, 0, e) if metric == "gap_linear" else ()
    with T.Aligner(*args, **kw) as al:
        s, c, r = al.align_arrays(pb, po, pl, tb, to, tl, cigar=True, bidirectional=True)
        fwd, _, _ = al.align_arrays(pb, po, pl, tb, to, tl, cigar=False)
    want, _ = oracle.align_batch_linear_arrays(pb, po, pl, tb, to, tl, x, e, cigar=False)
    assert np.array_equal(s, want)
    assert np.array_equal(s, fwd)
    base = base_score((x, 0, e))
    for i in range(len(pl)):
        p, t = bytes(pb[po[i]:po[i] + pl[i]]), bytes(tb[to[i]:to[i] + tl[i]])
        ops = T.runs_to_ops(r[c[i]:c[i + 1]])
        assert ops == oracle.bialign(p, t, x, 0, e, base_score=base, ring=True), i
        assert oracle.cigar_cost(ops, p, t, x, 0, e) == want[i]
