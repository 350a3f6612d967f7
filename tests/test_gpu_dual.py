"""GPU parity of the dual gap-affine mode (tsu_create_dual, the
align_kernel<..., kDual> instantiations) against the dual oracle.

Bar: bit-exact scores and byte-identical operation strings for every pair."""
import ctypes
import random

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DUAL = (4, 6, 2, 24, 1)


def _dual(aligner_factory, pen=DUAL):
    return aligner_factory(pen[:3], gap_opening2=pen[3], gap_extension2=pen[4])


def _long_indel_pairs(seed, n, lo, hi, n_indels=4, max_indel=40, subs=0.02):
    rng = random.Random(seed)
    pats, txts = [], []
    for _ in range(n):
        p = "".join(rng.choice("ACGT") for _ in range(rng.randint(lo, hi)))
        t = list(p)
        for _ in range(rng.randint(0, n_indels)):
            pos = rng.randint(0, len(t))
            L = rng.randint(1, max_indel)
            if rng.random() < 0.5:
                t[pos:pos] = [rng.choice("ACGT") for _ in range(L)]
            else:
                del t[pos:pos + L]
        for _ in range(int(len(t) * subs)):
            if t:
                t[rng.randrange(len(t))] = rng.choice("ACGT")
        pats.append(p)
        txts.append("".join(t))
    return pats, txts


def _check(al, oracle, pats, txts, pen=DUAL):
    scores, ops = al.align(pats, txts)
    osc, oops = oracle.align_batch2(pats, txts, *pen)
    bad = [i for i in range(len(pats)) if scores[i] != osc[i] or ops[i] != oops[i]]
    assert not bad, [(i, len(pats[i]), len(txts[i]), scores[i], osc[i]) for i in bad[:3]]
    return scores, ops


@pytest.mark.parametrize("pen", [DUAL, (3, 5, 3, 20, 1), (6, 2, 3, 10, 1), (1, 1, 1, 1, 1), (8, 4, 4, 12, 2),
                                 (4, 0, 3, 9, 1)])
def test_dual_random_short(aligner_factory, oracle, pen):
    rng = random.Random(sum(pen) * 17)
    pats, txts = _long_indel_pairs(sum(pen), 300, 0, 200)
    for _ in range(60):  # unrelated pairs, small alphabets, empties
        alpha = rng.choice(["ACGT", "AC"])
        pats.append("".join(rng.choice(alpha) for _ in range(rng.randint(0, 60))))
        txts.append("".join(rng.choice(alpha) for _ in range(rng.randint(0, 60))))
    pats += ["", "", "ACGT", "ACGTNNNNACGT"]
    txts += ["", "ACGTACGTAC", "", "ACGTACGT"]
    _check(_dual(aligner_factory, pen), oracle, pats, txts, pen)


def test_dual_kbp_pairs(aligner_factory, oracle):
    """1 kbp pairs with long indels (the second piece wins) and substitutions."""
    pats, txts = _long_indel_pairs(5, 3000, 900, 1100, n_indels=3, max_indel=60, subs=0.03)
    scores, ops = _check(_dual(aligner_factory), oracle, pats, txts)
    one_piece = oracle.align_batch(pats, txts, 4, 6, 2, cigar=False)[0]
    assert (scores < one_piece).sum() > 1000  # the long gaps take the cheaper piece


def test_dual_long_reads(aligner_factory, oracle):
    pats, txts = _long_indel_pairs(6, 12, 8000, 20000, n_indels=8, max_indel=300, subs=0.04)
    _check(_dual(aligner_factory), oracle, pats, txts)


def test_dual_score_only(aligner_factory, oracle):
    pats, txts = _long_indel_pairs(7, 500, 100, 2000)
    scores, ops = _dual(aligner_factory).align(pats, txts, cigar=False)
    assert ops is None
    assert list(scores) == list(oracle.align_batch2(pats, txts, *DUAL, cigar=False)[0])


def test_dual_every_starting_rung(oracle):
    """Every dual kernel instantiation (shared ring with 1-32 warps, global
    ring with 1-32) as the starting rung: same results."""
    import tsunami_pact_b200 as T

    pats, txts = _long_indel_pairs(8, 90, 100, 5000, n_indels=5, max_indel=100, subs=0.05)
    osc, oops = oracle.align_batch2(pats, txts, *DUAL)
    L = T.lib()
    L.tsu_set_band_start.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    with T.Aligner(4, 6, 2, gap_opening2=24, gap_extension2=1) as al:
        for mode, gw in [(0, 1), (0, 2), (0, 4), (0, 8), (0, 16), (0, 32), (1, 1), (1, 2), (1, 4), (1, 8), (1, 16),
                         (1, 32)]:
            for band in range(6):
                assert L.tsu_set_band_start(al._h, band, mode, gw) == 0
            scores, ops = al.align(pats, txts)
            assert list(scores) == list(osc), (mode, gw)
            assert ops == oops, (mode, gw)


def test_dual_argument_checks():
    import tsunami_pact_b200 as T

    with pytest.raises(T.AlignError):
        T.Aligner(4, 6, 2, gap_opening2=-1, gap_extension2=1)
    with pytest.raises(T.AlignError):
        T.Aligner(4, 6, 2, gap_opening2=24, gap_extension2=0)
    with T.Aligner(4, 6, 2, gap_opening2=24, gap_extension2=1) as al:
        big = b"A" * ((1 << 24) - 1)  # beyond the dual offset range
        with pytest.raises(T.AlignError):
            al.align([big], [b"A"])
        s, ops = al.align([b"ACGT"], [b"ACGT"])
        assert int(s[0]) == 0 and ops[0] == "MMMM"


def test_dual_server(oracle):
    import tsunami_pact_b200 as T

    pats, txts = _long_indel_pairs(9, 400, 100, 3000)
    with T.Server(4, 6, 2, workers=4, gap_opening2=24, gap_extension2=1) as srv:
        ids = [srv.submit(pats[i:i + 50], txts[i:i + 50]) for i in range(0, 400, 50)]
        got_s, got_o = [], []
        for rid in ids:
            s, co, runs, _info = srv.wait(rid, 60000)
            got_s += list(s)
            got_o += [T.runs_to_ops(runs[co[i]:co[i + 1]]) for i in range(len(s))]
    osc, oops = oracle.align_batch2(pats, txts, *DUAL)
    assert got_s == list(osc) and got_o == oops
