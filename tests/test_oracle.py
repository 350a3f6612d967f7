"""CPU tests of the oracle: pinned against the hand-derived known answers and
against an independent Gotoh DP (the optimal score is unique)."""
import random

import numpy as np
import pytest


def test_kat(oracle, kat_cases):
    for c in kat_cases:
        s, ops = oracle.align(c["p"], c["t"], *c["pen"])
        assert s == c["score"], c
        assert ops == c["ops"], c


def test_regression_fixture(oracle, regress_cases):
    for c in regress_cases:
        s, ops = oracle.align(c["p"], c["t"], *c["pen"])
        assert (s, ops) == (c["score"], c["ops"])


@pytest.mark.parametrize("pen", [(4, 6, 2), (1, 0, 1), (3, 5, 1), (7, 2, 3), (20, 1, 1), (2, 10, 1), (6, 4, 2)])
def test_random_vs_gotoh(oracle, pen):
    rng = random.Random(hash(pen) & 0xFFFF)
    for it in range(300):
        alpha = "ACGT" if it % 3 else "AC"
        m, n = rng.randint(0, 45), rng.randint(0, 45)
        p = "".join(rng.choice(alpha) for _ in range(m))
        t = "".join(rng.choice(alpha) for _ in range(n))
        s, ops = oracle.align(p, t, *pen)
        assert s == oracle.gotoh(p, t, *pen)
        assert oracle.cigar_cost(ops, p, t, *pen) == s


def test_batch_matches_single(oracle):
    rng = random.Random(7)
    pats = ["".join(rng.choice("ACGT") for _ in range(rng.randint(0, 200))) for _ in range(64)]
    txts = ["".join(rng.choice("ACGT") for _ in range(rng.randint(0, 200))) for _ in range(64)]
    sc, cg = oracle.align_batch(pats, txts, threads=4)
    for i in range(64):
        assert (sc[i], cg[i]) == oracle.align(pats[i], txts[i])


def test_rle_roundtrip(oracle):
    runs = oracle.ops_to_rle("MMMXIIDDDM")
    assert list(runs) == [(3 << 4) | 0, (1 << 4) | 8, (2 << 4) | 1, (3 << 4) | 2, (1 << 4) | 0]


def test_checker_plugin_symbol(oracle):
    """The CPU-check plugin the wfa_gpu CLI loads (TSU_CHECK_LIB) gives oracle scores."""
    import ctypes

    L = oracle.lib()
    fn = L.tsu_check_align_scores
    fn.restype = ctypes.c_int
    pats = [b"ACGT", b"ACGGT", b""]
    txts = [b"AGGT", b"ACGT", b"AC"]
    pl = np.array([len(p) for p in pats], np.int32)
    tl = np.array([len(t) for t in txts], np.int32)
    po = np.array([0, 4, 9], np.int64)
    to = np.array([0, 4, 8], np.int64)
    pb = np.frombuffer(b"".join(pats) + b"\0", np.uint8)
    tb = np.frombuffer(b"".join(txts) + b"\0", np.uint8)
    out = np.zeros(3, np.int32)
    rc = fn(ctypes.c_int64(3), ctypes.c_void_p(pb.ctypes.data), ctypes.c_void_p(po.ctypes.data),
            ctypes.c_void_p(pl.ctypes.data), ctypes.c_void_p(tb.ctypes.data), ctypes.c_void_p(to.ctypes.data),
            ctypes.c_void_p(tl.ctypes.data), 4, 6, 2, ctypes.c_void_p(out.ctypes.data), 2)
    assert rc == 0
    assert list(out) == [4, 8, 10]


# --- dual gap-affine (two-piece) oracle --------------------------------------

DUAL_PENS = [(4, 6, 2, 24, 1), (4, 4, 2, 12, 1), (3, 5, 3, 20, 1), (6, 2, 3, 10, 1), (2, 0, 2, 5, 1),
             (1, 1, 1, 1, 1), (5, 3, 3, 3, 1)]


def test_dual_known_answers(oracle):
    """Hand-derived: a lone gap of length L costs min(o1 + e1*L, o2 + e2*L)."""
    pen = (4, 6, 2, 24, 1)
    assert oracle.align2("", "AAAAA", *pen) == (16, "IIIII")      # 6+2*5 < 24+5
    assert oracle.align2("A" * 20, "", *pen) == (44, "D" * 20)    # 24+20 < 6+2*20
    assert oracle.align2("ACGT", "ACGT", *pen) == (0, "MMMM")
    assert oracle.align2("ACGT", "AGGT", *pen) == (4, "MXMM")
    # an 18-base insertion is where the pieces cross (6+36 == 24+18)
    p = "ACGTTGCA" * 4
    t = p[:16] + "G" * 18 + p[16:]
    s, ops = oracle.align2(p, t, *pen)
    assert s == 42 and oracle.cigar_cost2(ops, p, t, *pen) == 42


@pytest.mark.parametrize("pen", DUAL_PENS)
def test_dual_random_vs_dp(oracle, pen):
    """The dual oracle's score is the five-matrix DP optimum and its
    operation string costs exactly that score."""
    rng = random.Random(hash(pen) & 0xFFFF)
    for it in range(250):
        alpha = "ACGT" if it % 3 else "AC"
        m = rng.randint(0, 60)
        p = "".join(rng.choice(alpha) for _ in range(m))
        if it % 2:
            t = "".join(rng.choice(alpha) for _ in range(rng.randint(0, 60)))
        else:  # a long indel, where the second piece is the cheaper one
            i = rng.randint(0, m)
            L = rng.randint(1, 40)
            t = p[:i] + "".join(rng.choice(alpha) for _ in range(L)) + p[i:] if it % 4 else p[:i] + p[i + L:]
        s, ops = oracle.align2(p, t, *pen)
        assert s == oracle.gotoh2(p, t, *pen)
        assert oracle.cigar_cost2(ops, p, t, *pen) == s


def test_dual_reduces_to_one_piece(oracle):
    """With a second piece that never wins, the two-piece result (score and
    operation string) is the one-piece result."""
    rng = random.Random(11)
    for _ in range(200):
        p = "".join(rng.choice("ACGT") for _ in range(rng.randint(0, 80)))
        t = "".join(c for c in p if rng.random() > 0.1) + "".join(rng.choice("ACGT") for _ in range(3))
        assert oracle.align2(p, t, 4, 6, 2, 1000, 5) == oracle.align(p, t, 4, 6, 2)


def test_dual_batch_matches_single(oracle):
    rng = random.Random(5)
    pats = ["".join(rng.choice("ACGT") for _ in range(rng.randint(0, 150))) for _ in range(48)]
    txts = [p[: len(p) // 2] + "T" * rng.randint(0, 40) + p[len(p) // 2:] for p in pats]
    sc, cg = oracle.align_batch2(pats, txts, threads=4)
    for i in range(48):
        assert (sc[i], cg[i]) == oracle.align2(pats[i], txts[i])


# --- gap-linear oracle (edit, indel) ----------------------------------------

def _levenshtein(a, b):
    prev = list(range(len(b) + 1))
    for i, ca in enumerate(a, 1):
        cur = [i]
        for j, cb in enumerate(b, 1):
            cur.append(min(prev[j] + 1, cur[j - 1] + 1, prev[j - 1] + (ca != cb)))
        prev = cur
    return prev[-1]


def _lcs(a, b):
    prev = [0] * (len(b) + 1)
    for ca in a:
        cur = [0]
        for j, cb in enumerate(b, 1):
            cur.append(prev[j - 1] + 1 if ca == cb else max(prev[j], cur[j - 1]))
        prev = cur
    return prev[-1]


def test_linear_known_answers(oracle):
    assert oracle.align_linear("kitten", "sitting") == (3, "XMMMXMI")
    assert oracle.align_linear("", "ACG") == (3, "III")
    assert oracle.align_linear("ACG", "", 2, 3) == (9, "DDD")
    assert oracle.align_linear("ACGT", "ACGT", 3, 1) == (0, "MMMM")
    # indel distance: a substitution becomes a deletion and an insertion
    s, ops = oracle.align_linear("ACGT", "AGGT", 3, 1)
    assert s == 2 and "X" not in ops


@pytest.mark.parametrize("pen", [(1, 1), (3, 1), (2, 3), (4, 2), (5, 1), (1, 4)])
def test_linear_random_vs_dp(oracle, pen):
    """Scores equal the Needleman-Wunsch optimum (edit distance: also a plain
    Levenshtein; indel distance: m + n - 2 LCS), and the operation string
    costs exactly the score."""
    rng = random.Random(hash(pen) & 0xFFFF)
    for it in range(250):
        alpha = "ACGT" if it % 3 else "AC"
        p = "".join(rng.choice(alpha) for _ in range(rng.randint(0, 50)))
        t = "".join(rng.choice(alpha) for _ in range(rng.randint(0, 50)))
        s, ops = oracle.align_linear(p, t, *pen)
        assert s == oracle.linear_dp(p, t, *pen)
        if pen == (1, 1):
            assert s == _levenshtein(p, t)
        if pen == (3, 1):
            assert s == len(p) + len(t) - 2 * _lcs(p, t)
        # cost of the string under linear gaps = affine with open 0
        assert oracle.cigar_cost(ops, p, t, pen[0], 0, pen[1]) == s


def test_linear_batch_matches_single(oracle):
    rng = random.Random(13)
    pats = ["".join(rng.choice("ACGT") for _ in range(rng.randint(0, 150))) for _ in range(40)]
    txts = ["".join(rng.choice("ACGT") for _ in range(rng.randint(0, 150))) for _ in range(40)]
    sc, cg = oracle.align_batch_linear(pats, txts, 2, 1, threads=4)
    for i in range(40):
        assert (sc[i], cg[i]) == oracle.align_linear(pats[i], txts[i], 2, 1)


# --- ends-free gap-affine ----------------------------------------------------

FREES = [(0, 0, 0, 0), (5, 5, 5, 5), (100, 100, 0, 0), (0, 0, 100, 100), (3, 0, 0, 7), (0, 9, 2, 0),
         (1000, 1000, 1000, 1000)]


def test_ends_free_known_answers(oracle):
    pen = (4, 6, 2)
    # the pattern inside the text: the text's flanks are free insertions
    assert oracle.align_ends_free("ACGTTGCA", "GGGACGTTGCATT", (0, 0, 3, 2), *pen) == (0, "IIIMMMMMMMMII")
    # flanks longer than allowed cost the excess as one gap: 2 free + gap(1)
    s, ops = oracle.align_ends_free("ACGTTGCA", "GGGACGTTGCA", (0, 0, 2, 0), *pen)
    assert s == 8 and ops == "IIIMMMMMMMM"
    # the text inside the pattern: free deletions
    assert oracle.align_ends_free("TTACGTAA", "ACGT", (2, 2, 0, 0), *pen) == (0, "DDMMMMDD")
    # overlap (suffix of the pattern = prefix of the text)
    assert oracle.align_ends_free("GGGGACGT", "ACGTCCCC", (4, 0, 0, 4), *pen) == (0, "DDDDMMMMIIII")
    # all zero: end-to-end
    assert oracle.align_ends_free("ACGT", "AGGT", (0, 0, 0, 0), *pen) == oracle.align("ACGT", "AGGT", *pen)


@pytest.mark.parametrize("free", FREES)
def test_ends_free_random_vs_dp(oracle, free):
    rng = random.Random(hash(free) & 0xFFFF)
    pen = (4, 6, 2)
    for it in range(200):
        alpha = "ACGT" if it % 3 else "AC"
        core = "".join(rng.choice(alpha) for _ in range(rng.randint(0, 40)))
        p = "".join(rng.choice(alpha) for _ in range(rng.randint(0, 8))) + core + \
            "".join(rng.choice(alpha) for _ in range(rng.randint(0, 8)))
        t = "".join(rng.choice(alpha) for _ in range(rng.randint(0, 8))) + core + \
            "".join(rng.choice(alpha) for _ in range(rng.randint(0, 8)))
        if it % 4 == 0:
            t = "".join(rng.choice(alpha) for _ in range(rng.randint(0, 40)))
        s, ops = oracle.align_ends_free(p, t, free, *pen)
        assert s == oracle.gotoh_ends_free(p, t, free, *pen), (p, t, free)
        assert oracle.cigar_cost_ends_free(ops, p, t, free, *pen) == s, (p, t, free, ops)
        if free == (0, 0, 0, 0):
            assert (s, ops) == oracle.align(p, t, *pen)


def test_ends_free_batch_matches_single(oracle):
    rng = random.Random(17)
    pats = ["".join(rng.choice("ACGT") for _ in range(rng.randint(0, 120))) for _ in range(40)]
    txts = [p[rng.randint(0, 10):] + "".join(rng.choice("ACGT") for _ in range(rng.randint(0, 10))) for p in pats]
    free = (10, 10, 10, 10)
    sc, cg = oracle.align_batch_ends_free(pats, txts, free, threads=4)
    for i in range(40):
        assert (sc[i], cg[i]) == oracle.align_ends_free(pats[i], txts[i], free)


def _cost_free(ops, p, t, free, x, gap):
    """Cost of an operation string with free ends under a gap cost function
    (test-side restatement, independent of the oracle's C code)."""
    v = h = 0
    cost = 0
    runs = []
    i = 0
    while i < len(ops):
        j = i
        while j < len(ops) and ops[j] == ops[i]:
            j += 1
        runs.append((ops[i], j - i))
        i = j
    for r, (c, L) in enumerate(runs):
        if c in "MX":
            for _ in range(L):
                assert (c == "M") == (p[v] == t[h])
                cost += x if c == "X" else 0
                v += 1
                h += 1
            continue
        free_len = 0
        if r == 0:
            free_len += free[2] if c == "I" else free[0]
        if r == len(runs) - 1:
            free_len += free[3] if c == "I" else free[1]
        if c == "I":
            h += L
        else:
            v += L
        if L > free_len:
            cost += gap(L - free_len)
    assert v == len(p) and h == len(t)
    return cost


@pytest.mark.parametrize("free", FREES)
def test_linear_and_dual_ends_free_vs_dp(oracle, free):
    """Gap-linear (scores = gap-affine with opening 0) and dual gap-affine
    with free ends, against the ends-free DPs; operation strings cost the
    score; all-zero free ends reproduce the end-to-end oracles."""
    rng = random.Random(hash(free) & 0xFFF)
    for it in range(120):
        alpha = "ACGT" if it % 3 else "AC"
        core = "".join(rng.choice(alpha) for _ in range(rng.randint(0, 40)))
        fl = lambda: "".join(rng.choice(alpha) for _ in range(rng.randint(0, 10)))
        p, t = fl() + core + fl(), fl() + core + fl()
        for x, e in [(1, 1), (3, 1), (2, 3)]:
            s, ops = oracle.align_linear_ends_free(p, t, free, x, e)
            assert s == oracle.gotoh_ends_free(p, t, free, x, 0, e), (p, t, free, x, e)
            assert _cost_free(ops, p, t, free, x, lambda L: e * L) == s
            if free == (0, 0, 0, 0):
                assert (s, ops) == oracle.align_linear(p, t, x, e)
        pen = (4, 6, 2, 24, 1)
        s, ops = oracle.align2_ends_free(p, t, free, *pen)
        assert s == oracle.gotoh2_ends_free(p, t, free, *pen), (p, t, free)
        assert _cost_free(ops, p, t, free, 4, lambda L: min(6 + 2 * L, 24 + L)) == s
        if free == (0, 0, 0, 0):
            assert (s, ops) == oracle.align2(p, t, *pen)


def test_linear_dual_ends_free_batches(oracle):
    rng = random.Random(23)
    pats = ["".join(rng.choice("ACGT") for _ in range(rng.randint(0, 100))) for _ in range(30)]
    txts = [p[rng.randint(0, 8):] + "".join(rng.choice("ACGT") for _ in range(rng.randint(0, 8))) for p in pats]
    free = (8, 8, 8, 8)
    sc, cg = oracle.align_batch_linear_ends_free(pats, txts, free, 1, 1, threads=4)
    sc2, cg2 = oracle.align_batch2_ends_free(pats, txts, free, threads=4)
    for i in range(30):
        assert (sc[i], cg[i]) == oracle.align_linear_ends_free(pats[i], txts[i], free, 1, 1)
        assert (sc2[i], cg2[i]) == oracle.align2_ends_free(pats[i], txts[i], free)
