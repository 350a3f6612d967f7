"""GPU: the request server (tsu_server_* through the C ABI).

Each request's scores and CIGARs must be the same alone (one request per job,
one at a time) and in the mix (submitted at once, merged into shared jobs,
jobs overlapping on the device), equal to the batch path's on the same pairs,
and equal to the oracle's for the pairs the oracle finishes quickly."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _requests(n_req, max_pairs, index=0, cap_len=None):
    """Requests of the serving mixture: a list of (pbuf, poff, plen, tbuf, toff, tlen)."""
    import tsunami_pact_b200 as T
    from tsunami_pact_b200 import datasets as D

    _, sizes = D.c5_stream(n_req, 100.0, index=index, max_pairs=max_pairs)
    total = int(sizes.sum())
    lengths, rates, seed = D.shape("c5", total)
    if cap_len:
        lengths = np.minimum(lengths, cap_len).astype(np.int32)
    pbuf, poff, plen, tbuf, toff, tlen = T.gen_batch(seed, lengths, rates)
    out, k = [], 0
    for s in sizes:
        s = int(s)
        sl = slice(k, k + s)
        out.append((pbuf, poff[sl].copy(), plen[sl].copy(), tbuf, toff[sl].copy(), tlen[sl].copy()))
        k += s
    return out


def _collect(srv, ids):
    res = []
    for rid in ids:
        r = srv.wait(rid, 600_000)
        assert r is not None, "request timed out"
        res.append(r)
    return res


def _same(a, b):
    sa, ca, ra, _ = a
    sb, cb, rb, _ = b
    assert np.array_equal(sa, sb)
    if ca is None:
        assert cb is None
        return
    assert np.array_equal(ca, cb)
    assert np.array_equal(ra, rb)


def test_alone_equals_mix(aligner_factory, oracle):
    import tsunami_pact_b200 as T

    reqs = _requests(24, 64, index=0)
    with T.Server(4, 6, 2, workers=8, mem_budget=48 << 30) as srv:
        # alone: one request per job, nothing else on the device
        alone = []
        for r in reqs:
            rid = srv.submit_arrays(*r)
            out = srv.wait(rid, 600_000)
            assert out is not None and out[3]["job_requests"] == 1
            alone.append(out)
        srv.reset_stats()
        # in the mix: everything at once
        ids = [srv.submit_arrays(*r) for r in reqs]
        mix = _collect(srv, ids)
        st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["mean_requests_per_job"] > 1.0  # requests queued behind running jobs were merged
    assert st["peak_granted_bytes"] <= 48 << 30
    for a, m in zip(alone, mix):
        _same(a, m)
    # the batch path on the same pairs
    al = aligner_factory()
    for r, a in zip(reqs, alone):
        s, co, runs = al.align_arrays(*r)
        assert np.array_equal(s, a[0])
        assert np.array_equal(co, a[1])
        assert np.array_equal(runs, a[2])
    # the oracle on the pairs up to 5 kbp
    pats, txts, got_s, got_ops = [], [], [], []
    for (pbuf, poff, plen, tbuf, toff, tlen), (s, co, runs, _) in zip(reqs, alone):
        for i in range(len(plen)):
            if max(plen[i], tlen[i]) > 5000:
                continue
            pats.append(bytes(pbuf[poff[i]:poff[i] + plen[i]]))
            txts.append(bytes(tbuf[toff[i]:toff[i] + tlen[i]]))
            got_s.append(int(s[i]))
            got_ops.append(T.runs_to_ops(runs[co[i]:co[i + 1]]))
    osc, oops = oracle.align_batch(pats, txts, 4, 6, 2)
    assert list(osc) == got_s
    assert oops == got_ops


def test_tight_budget_admission(aligner_factory):
    """A budget that holds one long-read job at a time: every request still
    completes, the grants never exceed the budget, results equal the batch."""
    import tsunami_pact_b200 as T

    reqs = _requests(12, 32, index=1, cap_len=20000)
    budget = 3 << 30
    with T.Server(4, 6, 2, workers=4, mem_budget=budget, max_error_hint=0.2) as srv:
        ids = [srv.submit_arrays(*r) for r in reqs]
        outs = _collect(srv, ids)
        st = srv.stats()
    assert st["completed"] == len(reqs)
    assert st["peak_granted_bytes"] <= budget
    al = aligner_factory()
    for r, o in zip(reqs, outs):
        s, co, runs = al.align_arrays(*r)
        assert np.array_equal(s, o[0]) and np.array_equal(co, o[1]) and np.array_equal(runs, o[2])


def test_reject_cancel_score_only(aligner_factory):
    import tsunami_pact_b200 as T

    big = T.gen_batch(7, np.array([50000], np.int32), np.array([0.2]))
    small = _requests(6, 16, index=2, cap_len=2000)
    with T.Server(4, 6, 2, workers=1, mem_budget=256 << 20) as srv:
        with pytest.raises(T.AlignError) as ei:
            srv.submit_arrays(*big)  # cannot fit even alone
        assert ei.value.code == 2
        ids = [srv.submit_arrays(*r, cigar=(k % 2 == 0)) for k, r in enumerate(small)]
        assert srv.cancel(ids[-1]) == 0  # queued, running or done: dropped
        outs = _collect(srv, ids[:-1])
        assert srv.cancel(ids[-1]) == 7  # TSU_ENOTFOUND
        st = srv.stats()
    assert st["rejected"] == 1
    al = aligner_factory()
    for k, (r, o) in enumerate(zip(small[:-1], outs)):
        s = al.align_arrays(*r, cigar=False)[0]
        assert np.array_equal(s, o[0])
        assert (o[1] is None) == (k % 2 == 1)


def test_predict_is_enough():
    """A context whose budget is tsu_predict_bytes' full figure runs the batch
    (pairs that need no retry pass: up to 2 kbp at the mixture's rates)."""
    import ctypes

    import tsunami_pact_b200 as T
    from tsunami_pact_b200 import _lib as Lb

    reqs = _requests(4, 128, index=3, cap_len=2000)
    with T.Aligner(4, 6, 2) as al:
        L = T.lib()
        for pbuf, poff, plen, tbuf, toff, tlen in reqs:
            b = Lb.Batch(len(plen), pbuf.ctypes.data, poff.ctypes.data, plen.ctypes.data, tbuf.ctypes.data,
                         toff.ctypes.data, tlen.ctypes.data)
            full, mn = ctypes.c_size_t(), ctypes.c_size_t()
            assert L.tsu_predict_bytes(al._h, ctypes.byref(b), 0, ctypes.byref(full), ctypes.byref(mn)) == 0
            assert 0 < mn.value <= full.value
            # a fresh context with exactly the prediction as its budget runs the batch
            with T.Aligner(4, 6, 2, mem_budget=full.value) as tight:
                s1 = tight.align_arrays(pbuf, poff, plen, tbuf, toff, tlen)[0]
            s0 = al.align_arrays(pbuf, poff, plen, tbuf, toff, tlen)[0]
            assert np.array_equal(s0, s1)


def test_bidirectional_requests(aligner_factory):
    """Requests with TSU_BIDIRECTIONAL, mixed with plain ones: every
    bidirectional result equals the batch path's bidirectional one on the
    same pairs, every plain result the plain one (requests of different
    flags never share a job); a dual gap-affine server fails them with
    TSU_EINVAL."""
    import tsunami_pact_b200 as T

    reqs = _requests(12, 48, index=3, cap_len=12_000)
    al = aligner_factory((4, 6, 2))
    with T.Server(4, 6, 2, workers=4, mem_budget=32 << 30) as srv:
        ids = [srv.submit_arrays(*r, cigar=(k % 3 != 2), bidirectional=(k % 2 == 0)) for k, r in enumerate(reqs)]
        got = _collect(srv, ids)
    for k, (r, g) in enumerate(zip(reqs, got)):
        cig, bi = k % 3 != 2, k % 2 == 0
        s, c, runs = al.align_arrays(*r, cigar=cig, bidirectional=bi)
        assert np.array_equal(g[0][: len(s)], s), k
        if cig:
            assert np.array_equal(g[1], c), k
            assert np.array_equal(g[2][: int(c[-1])], runs), k
    with T.Server(4, 6, 2, gap_opening2=24, gap_extension2=1, workers=1) as srv:
        rid = srv.submit_arrays(*reqs[0], bidirectional=True)
        with pytest.raises(T.AlignError):
            srv.wait(rid, 600_000)
