"""tsu_align_scores_noalloc: scores without any device allocation.

Callers that cannot call cudaMalloc (plug-ins under a host framework that
owns all device memory, services that must not block in the allocator
mid-request) use this entry point; its scratch is a fixed array compiled into
the library.  The test calls it through the C ABI twice in a row and checks
each result against the context-based entry point (tsu_align_batch_device)
and against the CPU oracle; scores are integers, so the tolerance is exact
equality.  It also checks that oversized batches are refused before any score
is written and that the second call takes no device memory.

This file is named to be collected last, so a run that stops at the first
failure has already run every other test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TSU_OK, TSU_EINVAL, TSU_EOVERFLOW = 0, 1, 5


def _noalloc_fn():
    import tsunami_pact_b200 as T
    from tsunami_pact_b200._lib import Batch, Penalties

    L = T.lib()
    fn = L.tsu_align_scores_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.POINTER(Penalties), ctypes.POINTER(Batch), ctypes.c_void_p, ctypes.c_void_p]
    return fn, Batch, Penalties


def _device_batch(torch, seed, lengths, rates):
    import tsunami_pact_b200 as T

    pbuf, poff, plen, tbuf, toff, tlen = T.gen_batch(seed, np.asarray(lengths, np.int32), np.asarray(rates))
    dev = "cuda:0"
    return [torch.from_numpy(x).to(dev) for x in (pbuf, poff, plen, tbuf, toff, tlen)]


def _call_noalloc(fn, Batch, Penalties, t, pen=(4, 6, 2), out=None, free_mem=None):
    """Call the entry point; with free_mem=[], record the device's free memory
    right before and right after the C call itself."""
    import torch

    p, po, pl, tx, to, tl = t
    n = int(pl.numel())
    if out is None:
        out = torch.full((n,), -7, dtype=torch.int32, device="cuda:0")
    b = Batch(n, p.data_ptr(), po.data_ptr(), pl.data_ptr(), tx.data_ptr(), to.data_ptr(), tl.data_ptr())
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    if free_mem is not None:
        free_mem.append(torch.cuda.mem_get_info(0)[0])
    rc = fn(ctypes.byref(Penalties(*pen)), ctypes.byref(b), ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
    torch.cuda.synchronize()
    if free_mem is not None:
        free_mem.append(torch.cuda.mem_get_info(0)[0])
    return rc, out


def _reference_scores(t, pen=(4, 6, 2)):
    import torch

    import tsunami_pact_b200 as T

    p, po, pl, tx, to, tl = t
    n = int(pl.numel())
    out = torch.zeros(n, dtype=torch.int32, device="cuda:0")
    with T.Aligner(*pen) as al:
        al.align_device(p, po, pl, tx, to, tl, out)
    return out.cpu().numpy()


def test_noalloc_matches_context_path_twice():
    torch = pytest.importorskip("torch")
    fn, Batch, Penalties = _noalloc_fn()
    rng = np.random.default_rng(11)
    # two different batches in a row: mixed lengths (some pairs exceed the
    # shared-memory ring and take the global pass), unequal and empty pairs
    lens1 = np.concatenate([np.full(3000, 150), np.full(500, 1000), rng.integers(0, 400, 400), [0, 1, 2500, 4000]])
    rates1 = np.concatenate([np.full(3000, 0.02), np.full(500, 0.05), rng.uniform(0, 0.3, 400), [0, 1.0, 0.15, 0.12]])
    lens2 = rng.integers(50, 2000, 1500)
    rates2 = rng.uniform(0.01, 0.15, 1500)
    for seed, lens, rates in [(101, lens1, rates1), (202, lens2, rates2)]:
        t = _device_batch(torch, seed, lens, rates)
        rc, out = _call_noalloc(fn, Batch, Penalties, t)
        assert rc == TSU_OK
        got = out.cpu().numpy()
        ref = _reference_scores(t)
        assert np.array_equal(got, ref), np.nonzero(got != ref)[0][:10]
        # and against the oracle directly: the long pairs (2500, 4000 bp)
        # take the score-only global-ring pass, which keeps no history
        from oracle import oracle as O

        h = [x.cpu().numpy() for x in t]
        osc, _ = O.align_batch_arrays(h[0], h[1], h[2], h[3], h[4], h[5], 4, 6, 2, cigar=False)
        assert np.array_equal(got, osc), np.nonzero(got != osc)[0][:10]


def test_noalloc_takes_no_device_memory_and_refuses_oversized():
    torch = pytest.importorskip("torch")
    fn, Batch, Penalties = _noalloc_fn()
    t = _device_batch(torch, 303, np.full(2000, 1000), np.full(2000, 0.05))
    out = torch.full((2000,), -7, dtype=torch.int32, device="cuda:0")
    rc, _ = _call_noalloc(fn, Batch, Penalties, t, out=out)  # first call on the device: set-up
    assert rc == TSU_OK
    free_mem = []
    rc, out = _call_noalloc(fn, Batch, Penalties, t, out=out, free_mem=free_mem)
    assert rc == TSU_OK
    assert free_mem[1] == free_mem[0]
    assert np.array_equal(out.cpu().numpy(), _reference_scores(t))
    # 80,000 pairs of 1 kbp need more packed-sequence scratch than 32 MiB
    big = _device_batch(torch, 404, np.full(80000, 1000), np.full(80000, 0.05))
    rc, out = _call_noalloc(fn, Batch, Penalties, big)
    assert rc == TSU_EOVERFLOW
    assert int((out == -7).sum()) == 80000  # outputs untouched
    # invalid penalties are refused
    rc, _ = _call_noalloc(fn, Batch, Penalties, t, pen=(0, 6, 2))
    assert rc == TSU_EINVAL


def test_noalloc_deep_rings_refused_up_front_or_aligned_in_hbm():
    """A deep ring (mismatch 1000, opening 0, extension 1: 1,005 ring slots)
    does not fit one warp's shared memory, so every pair takes the HBM ring.
    For 5 kbp pairs that ring is 1,005 x 10,003 x 4 B = 40 MB, more than the
    32 MiB array: refused up front, no score written.  For 4 kbp pairs it is
    32.2 MB, which fits: the scores equal the context path's and the
    oracle's."""
    torch = pytest.importorskip("torch")
    fn, Batch, Penalties = _noalloc_fn()
    pen = (1000, 0, 1)
    t = _device_batch(torch, 505, np.full(4, 5000), np.full(4, 0.05))
    rc, out = _call_noalloc(fn, Batch, Penalties, t, pen=pen)
    assert rc == TSU_EOVERFLOW
    assert int((out == -7).sum()) == 4
    t = _device_batch(torch, 506, np.full(4, 4000), np.full(4, 0.05))
    rc, out = _call_noalloc(fn, Batch, Penalties, t, pen=pen)
    assert rc == TSU_OK
    got = out.cpu().numpy()
    assert np.array_equal(got, _reference_scores(t, pen))
    from oracle import oracle as O

    h = [x.cpu().numpy() for x in t]
    osc, _ = O.align_batch_arrays(h[0], h[1], h[2], h[3], h[4], h[5], *pen, cigar=False)
    assert np.array_equal(got, osc)
