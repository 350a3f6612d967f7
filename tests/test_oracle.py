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
