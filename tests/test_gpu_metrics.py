"""GPU parity of the gap-linear kernels (align_kernel<..., kModelLinear>)
behind tsu_create_metric: edit, indel and gap-linear distance against the
gap-linear oracle.  Bar: bit-exact scores and byte-identical operation
strings for every pair."""
import random

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (metric, (mismatch, gap_opening, gap_extension) of the Aligner, oracle x, oracle e);
# edit and indel take no penalties, gap_linear takes mismatch and gap_extension
METRICS = [("edit", (4, 6, 2), 1, 1), ("indel", (4, 6, 2), 3, 1), ("gap_linear", (2, 0, 3), 2, 3),
           ("gap_linear", (4, 0, 2), 4, 2)]


def _pairs(seed, n, lo, hi, rate):
    rng = random.Random(seed)
    pats, txts = [], []
    for _ in range(n):
        p = "".join(rng.choice("ACGT") for _ in range(rng.randint(lo, hi)))
        t = list(p)
        for _ in range(int(len(p) * rate * rng.random() * 2)):
            pos = rng.randint(0, max(0, len(t) - 1))
            r = rng.random()
            if r < 0.33 and t:
                t[pos] = rng.choice("ACGT")
            elif r < 0.66:
                t.insert(pos, rng.choice("ACGT"))
            elif t:
                del t[pos]
        pats.append(p)
        txts.append("".join(t))
    return pats, txts


def _check(al, oracle, pats, txts, x, e):
    scores, ops = al.align(pats, txts)
    osc, oops = oracle.align_batch_linear(pats, txts, x, e)
    bad = [i for i in range(len(pats)) if scores[i] != osc[i] or ops[i] != oops[i]]
    assert not bad, [(i, len(pats[i]), len(txts[i]), scores[i], osc[i]) for i in bad[:3]]
    return scores, ops


def _aligner(aligner_factory, metric, pen):
    return aligner_factory(pen, metric=metric)


@pytest.mark.parametrize("metric,pen,x,e", METRICS)
def test_metric_random_short(aligner_factory, oracle, metric, pen, x, e):
    pats, txts = _pairs(x * 7 + e, 400, 0, 200, 0.1)
    pats += ["", "", "ACGT", "ACGTNNNNACGT", "kitten"]
    txts += ["", "ACGTACGTAC", "", "ACGTACGT", "sitting"]
    scores, ops = _check(_aligner(aligner_factory, metric, pen), oracle, pats, txts, x, e)
    if metric == "indel":
        assert not any("X" in o for o in ops)


@pytest.mark.parametrize("metric,pen,x,e", METRICS[:2])
def test_metric_kbp_and_long(aligner_factory, oracle, metric, pen, x, e):
    al = _aligner(aligner_factory, metric, pen)
    _check(al, oracle, *_pairs(21, 3000, 900, 1100, 0.05), x, e)
    _check(al, oracle, *_pairs(22, 8, 10000, 30000, 0.1), x, e)


def test_metric_score_only(aligner_factory, oracle):
    pats, txts = _pairs(23, 600, 100, 3000, 0.08)
    scores, ops = _aligner(aligner_factory, "edit", (4, 6, 2)).align(pats, txts, cigar=False)
    assert ops is None
    assert list(scores) == list(oracle.align_batch_linear(pats, txts, 1, 1, cigar=False)[0])


def test_metric_every_starting_rung(oracle):
    import ctypes

    import tsunami_pact_b200 as T

    pats, txts = _pairs(24, 90, 100, 5000, 0.12)
    osc, oops = oracle.align_batch_linear(pats, txts, 1, 1)
    L = T.lib()
    L.tsu_set_band_start.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    with T.Aligner(metric="edit") as al:
        for mode, gw in [(0, 1), (0, 2), (0, 4), (0, 8), (0, 16), (0, 32), (1, 1), (1, 8), (1, 16), (1, 32)]:
            for band in range(6):
                assert L.tsu_set_band_start(al._h, band, mode, gw) == 0
            scores, ops = al.align(pats, txts)
            assert list(scores) == list(osc), (mode, gw)
            assert ops == oops, (mode, gw)


def test_metric_matches_affine_scores(aligner_factory):
    """Gap-linear scores equal gap-affine scores with a zero gap opening (the
    two models are the same score function)."""
    pats, txts = _pairs(25, 500, 50, 1500, 0.1)
    s_lin, _ = _aligner(aligner_factory, "gap_linear", (4, 0, 2)).align(pats, txts)
    s_aff, _ = aligner_factory((4, 0, 2)).align(pats, txts)
    assert np.array_equal(s_lin, s_aff)


def test_metric_server(oracle):
    import tsunami_pact_b200 as T

    pats, txts = _pairs(26, 300, 100, 2000, 0.08)
    with T.Server(workers=4, metric="edit") as srv:
        ids = [srv.submit(pats[i:i + 50], txts[i:i + 50]) for i in range(0, 300, 50)]
        got_s, got_o = [], []
        for rid in ids:
            s, co, runs, _info = srv.wait(rid, 60000)
            got_s += list(s)
            got_o += [T.runs_to_ops(runs[co[i]:co[i + 1]]) for i in range(len(s))]
    osc, oops = oracle.align_batch_linear(pats, txts, 1, 1)
    assert got_s == list(osc) and got_o == oops
