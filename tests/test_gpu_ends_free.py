"""GPU parity of ends-free gap-affine alignment (tsu_set_ends_free) against
the ends-free oracle.  Bar: bit-exact scores and byte-identical operation
strings for every pair."""
import random

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FREES = [(30, 30, 30, 30), (0, 0, 200, 200), (200, 200, 0, 0), (5, 0, 0, 12), (2000, 2000, 2000, 2000)]


def _flanked(seed, n, lo, hi, flank=30, subs=0.05):
    rng = random.Random(seed)
    pats, txts = [], []
    for _ in range(n):
        core = "".join(rng.choice("ACGT") for _ in range(rng.randint(lo, hi)))
        t = list(core)
        for _ in range(int(len(core) * subs)):
            pos = rng.randint(0, max(0, len(t) - 1))
            r = rng.random()
            if r < 0.5 and t:
                t[pos] = rng.choice("ACGT")
            elif r < 0.75:
                t.insert(pos, rng.choice("ACGT"))
            elif t:
                del t[pos]
        fl = lambda: "".join(rng.choice("ACGT") for _ in range(rng.randint(0, flank)))
        pats.append(fl() + core + fl())
        txts.append(fl() + "".join(t) + fl())
    return pats, txts


def _check(al, oracle, pats, txts, free):
    al.set_ends_free(*free)
    scores, ops = al.align(pats, txts)
    osc, oops = oracle.align_batch_ends_free(pats, txts, free)
    bad = [i for i in range(len(pats)) if scores[i] != osc[i] or ops[i] != oops[i]]
    assert not bad, [(i, len(pats[i]), len(txts[i]), scores[i], osc[i]) for i in bad[:3]]
    return scores, ops


@pytest.mark.parametrize("free", FREES)
def test_ends_free_random(oracle, free):
    import tsunami_pact_b200 as T

    pats, txts = _flanked(sum(free), 500, 0, 300)
    pats += ["", "", "ACGT", "ACGTNNNNACGT", "GGGGACGT"]
    txts += ["", "ACGTACGTAC", "", "ACGTACGT", "ACGTCCCC"]
    with T.Aligner(4, 6, 2) as al:
        _check(al, oracle, pats, txts, free)


def test_ends_free_kbp_and_long(oracle):
    import tsunami_pact_b200 as T

    with T.Aligner(4, 6, 2) as al:
        _check(al, oracle, *_flanked(41, 2000, 900, 1100, flank=100), (100, 100, 100, 100))
        _check(al, oracle, *_flanked(42, 8, 8000, 20000, flank=500, subs=0.1), (500, 500, 500, 500))
        # back to end-to-end: the same results as a fresh context
        pats, txts = _flanked(43, 200, 100, 500)
        al.set_ends_free(0, 0, 0, 0)
        s, ops = al.align(pats, txts)
        osc, oops = oracle.align_batch(pats, txts, 4, 6, 2)
        assert list(s) == list(osc) and ops == oops


def test_ends_free_every_starting_rung(oracle):
    import ctypes

    import tsunami_pact_b200 as T

    pats, txts = _flanked(44, 90, 100, 4000, flank=200, subs=0.1)
    free = (150, 150, 150, 150)
    osc, oops = oracle.align_batch_ends_free(pats, txts, free)
    L = T.lib()
    L.tsu_set_band_start.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    with T.Aligner(4, 6, 2) as al:
        al.set_ends_free(*free)
        for mode, gw in [(0, 1), (0, 2), (0, 4), (0, 8), (0, 16), (0, 32), (1, 1), (1, 8), (1, 16), (1, 32)]:
            for band in range(6):
                assert L.tsu_set_band_start(al._h, band, mode, gw) == 0
            scores, ops = al.align(pats, txts)
            assert list(scores) == list(osc), (mode, gw)
            assert ops == oops, (mode, gw)


def test_ends_free_score_only_and_checks(oracle):
    import tsunami_pact_b200 as T

    pats, txts = _flanked(45, 400, 100, 2000)
    free = (30, 30, 30, 30)
    with T.Aligner(4, 6, 2) as al:
        al.set_ends_free(*free)
        scores, ops = al.align(pats, txts, cigar=False)
        assert list(scores) == list(oracle.align_batch_ends_free(pats, txts, free, cigar=False)[0])
        with pytest.raises(T.AlignError):
            al.set_ends_free(-1, 0, 0, 0)



@pytest.mark.parametrize("free", [(30, 30, 30, 30), (0, 0, 300, 300)])
def test_ends_free_edit_and_dual(oracle, free):
    """Semi-global edit distance and dual gap-affine with free ends."""
    import tsunami_pact_b200 as T

    pats, txts = _flanked(50 + free[2], 400, 0, 1200, flank=200)
    with T.Aligner(metric="edit") as al:
        al.set_ends_free(*free)
        s, ops = al.align(pats, txts)
        osc, oops = oracle.align_batch_linear_ends_free(pats, txts, free, 1, 1)
        assert list(s) == list(osc) and ops == oops
    with T.Aligner(4, 6, 2, gap_opening2=24, gap_extension2=1) as al:
        al.set_ends_free(*free)
        s, ops = al.align(pats, txts)
        osc, oops = oracle.align_batch2_ends_free(pats, txts, free)
        assert list(s) == list(osc) and ops == oops
