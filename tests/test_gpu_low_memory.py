"""GPU parity of the low-memory mode (tsu_set_low_memory: checkpointed
wavefront rings, history recomputed segment by segment): the same scores and
CIGARs as the oracle, and less predicted device memory for long pairs."""
import random

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pairs(seed, n, lo, hi, rate):
    rng = random.Random(seed)
    pats, txts = [], []
    for _ in range(n):
        p = "".join(rng.choice("ACGT") for _ in range(rng.randint(lo, hi)))
        t = list(p)
        for _ in range(int(len(p) * rate)):
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


@pytest.mark.parametrize("K", [1, 7, 64, -1])
def test_low_memory_affine(oracle, K):
    import tsunami_pact_b200 as T

    pats, txts = _pairs(80 + K, 400, 0, 1500, 0.1)
    pats += ["", "ACGT", "ACGTNNNNACGT"]
    txts += ["ACGTAC", "", "ACGTACGT"]
    with T.Aligner(4, 6, 2) as al:
        al.set_low_memory(K)
        s, ops = al.align(pats, txts)
    osc, oops = oracle.align_batch(pats, txts, 4, 6, 2)
    assert list(s) == list(osc) and ops == oops


def test_low_memory_long_reads_and_models(oracle):
    import tsunami_pact_b200 as T

    pats, txts = _pairs(90, 10, 8000, 25000, 0.15)
    with T.Aligner(4, 6, 2) as al:
        al.set_low_memory(-1)
        s, ops = al.align(pats, txts)
    osc, oops = oracle.align_batch(pats, txts, 4, 6, 2)
    assert list(s) == list(osc) and ops == oops
    pats, txts = _pairs(91, 200, 100, 3000, 0.1)
    with T.Aligner(4, 6, 2, gap_opening2=24, gap_extension2=1) as al:
        al.set_low_memory(-1)
        s, ops = al.align(pats, txts)
    osc, oops = oracle.align_batch2(pats, txts)
    assert list(s) == list(osc) and ops == oops
    with T.Aligner(metric="edit") as al:
        al.set_low_memory(-1)
        al.set_ends_free(50, 50, 50, 50)
        s, ops = al.align(pats, txts)
    osc, oops = oracle.align_batch_linear_ends_free(pats, txts, (50, 50, 50, 50), 1, 1)
    assert list(s) == list(osc) and ops == oops


def test_low_memory_needs_less_memory():
    """The predicted device memory of a batch of long divergent pairs is much
    smaller with checkpoints."""
    import tsunami_pact_b200 as T

    plen = np.full(64, 50000, np.int32)
    with T.Aligner(4, 6, 2, max_error_hint=0.2) as al:
        full_hi, min_hi = al.predict_bytes(plen, plen)
        al.set_low_memory(-1)
        full_lo, min_lo = al.predict_bytes(plen, plen)
    assert min_lo * 4 < min_hi, (min_lo, min_hi)
    assert full_lo < full_hi


def test_low_memory_every_starting_rung(oracle):
    """Every low-memory kernel (shared ring with 1-32 warps, global ring with
    1-32) as the starting rung: the oracle's results."""
    import ctypes

    import tsunami_pact_b200 as T

    pats, txts = _pairs(95, 60, 100, 4000, 0.12)
    osc, oops = oracle.align_batch(pats, txts, 4, 6, 2)
    L = T.lib()
    L.tsu_set_band_start.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    with T.Aligner(4, 6, 2) as al:
        al.set_low_memory(5)
        for mode, gw in [(0, 1), (0, 2), (0, 4), (0, 8), (0, 16), (0, 32), (1, 1), (1, 8), (1, 16), (1, 32)]:
            for band in range(6):
                assert L.tsu_set_band_start(al._h, band, mode, gw) == 0
            scores, ops = al.align(pats, txts)
            assert list(scores) == list(osc), (mode, gw)
            assert ops == oops, (mode, gw)


def test_server_runs_oversized_cigar_in_low_memory(oracle):
    """A request whose smallest CIGAR footprint exceeds the server's budget
    runs in low-memory mode instead of failing; its score-only form has no
    such mode and is rejected."""
    import tsunami_pact_b200 as T

    pats, txts = _pairs(97, 1, 30000, 30000, 0.2)
    plen = np.array([len(pats[0])], np.int32)
    tlen = np.array([len(txts[0])], np.int32)
    with T.Aligner(4, 6, 2) as al:
        _, min_hi = al.predict_bytes(plen, tlen)
        al.set_low_memory(-1)
        _, min_lo = al.predict_bytes(plen, tlen)
        _, min_score = al.predict_bytes(plen, tlen, cigar=False)
    assert min_lo < min_hi
    budget = (min_lo + min_hi) // 2
    # the server sizes the pair by the same hint as the predictions above
    with T.Server(4, 6, 2, workers=2, mem_budget=budget, estimate_hint=False) as srv:
        rid = srv.submit(pats, txts)
        s, co, runs, _info = srv.wait(rid, 300000)
        ops = T.runs_to_ops(runs[co[0]:co[1]])
        if min_score > budget:
            with pytest.raises(T.AlignError):
                srv.submit(pats, txts, cigar=False)
    osc, oops = oracle.align_batch(pats, txts, 4, 6, 2)
    assert int(s[0]) == int(osc[0]) and ops == oops[0]
