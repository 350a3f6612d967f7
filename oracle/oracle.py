"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
as the checker and by ``bench.py``'s CPU-baseline / reference leg.  The
product (``tsunami_pact_b200``) never imports this module.

The oracle restates the gap-affine end-to-end WFA of the reference kernel
(wfa_gpu.cu:191-722) and of the WFA2-lib call it checks against
(wfa_gpu.cu:150-166); see ``wfa_oracle.h`` for the parity status.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import List, Optional, Sequence, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


class OraStats(ctypes.Structure):
    _fields_ = [
        ("steps", ctypes.c_int64),
        ("cells", ctypes.c_int64),
        ("ext_chars", ctypes.c_int64),
        ("ext_calls", ctypes.c_int64),
        ("final_score", ctypes.c_int64),
    ]


class OraEnds(ctypes.Structure):
    """Free ends: pattern_begin_free, pattern_end_free, text_begin_free, text_end_free."""
    _fields_ = [("pattern_begin_free", ctypes.c_int32), ("pattern_end_free", ctypes.c_int32),
                ("text_begin_free", ctypes.c_int32), ("text_end_free", ctypes.c_int32)]


def build() -> str:
    """Compile liboracle.so with the Makefile beside this file."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        c_char_p = ctypes.c_char_p
        i32, i64 = ctypes.c_int32, ctypes.c_int64
        P = ctypes.POINTER
        L.ora_align.restype = ctypes.c_int
        L.ora_align.argtypes = [c_char_p, ctypes.c_int, c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                ctypes.c_int, ctypes.c_void_p, ctypes.c_int, P(ctypes.c_int), P(OraStats)]
        L.ora_bialign.restype = ctypes.c_int
        L.ora_align_segment.restype = ctypes.c_int
        L.ora_align_segment.argtypes = [c_char_p, ctypes.c_int, c_char_p, ctypes.c_int] + [ctypes.c_int] * 3 + [
            ctypes.c_char, ctypes.c_char, ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.ora_crossing_split.restype = ctypes.c_int
        L.ora_crossing_split.argtypes = [c_char_p, ctypes.c_int, c_char_p, ctypes.c_int] + [ctypes.c_int] * 3 + [
            ctypes.c_char, ctypes.c_char, P(ctypes.c_int), ctypes.c_char_p, P(ctypes.c_int), P(ctypes.c_int)]
        L.ora_bialign_ring.restype = ctypes.c_int
        L.ora_bialign_ring.argtypes = [c_char_p, ctypes.c_int, c_char_p, ctypes.c_int] + [ctypes.c_int] * 4 + [
            ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.ora_bialign.argtypes = [c_char_p, ctypes.c_int, c_char_p, ctypes.c_int] + [ctypes.c_int] * 4 + [
            ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.ora_gotoh_score.restype = ctypes.c_int
        L.ora_gotoh_score.argtypes = [c_char_p, ctypes.c_int, c_char_p, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_int]
        L.ora_cigar_cost.restype = i64
        L.ora_cigar_cost.argtypes = [c_char_p, ctypes.c_int, c_char_p, ctypes.c_int, c_char_p, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.ora_align_batch.restype = ctypes.c_int
        L.ora_align_batch.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, P(OraStats)]
        L.ora_ops_to_rle.restype = ctypes.c_int
        L.ora_ops_to_rle.argtypes = [c_char_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
        L.ora_max_threads.restype = ctypes.c_int
        L.ora_align2.restype = ctypes.c_int
        L.ora_align2.argtypes = [c_char_p, ctypes.c_int, c_char_p, ctypes.c_int] + [ctypes.c_int] * 5 + [
            ctypes.c_void_p, ctypes.c_int, P(ctypes.c_int), P(OraStats)]
        L.ora_gotoh2_score.restype = ctypes.c_int
        L.ora_gotoh2_score.argtypes = [c_char_p, ctypes.c_int, c_char_p, ctypes.c_int] + [ctypes.c_int] * 5
        L.ora_cigar_cost2.restype = i64
        L.ora_cigar_cost2.argtypes = [c_char_p, ctypes.c_int, c_char_p, ctypes.c_int, c_char_p,
                                      ctypes.c_int] + [ctypes.c_int] * 5
        L.ora_align_linear.restype = ctypes.c_int
        L.ora_align_linear.argtypes = [c_char_p, ctypes.c_int, c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_void_p, ctypes.c_int, P(ctypes.c_int), P(OraStats)]
        L.ora_linear_dp_score.restype = ctypes.c_int
        L.ora_linear_dp_score.argtypes = [c_char_p, ctypes.c_int, c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.ora_align_batch_linear.restype = ctypes.c_int
        L.ora_align_batch_linear.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 6 + [ctypes.c_int] * 2 + [
            ctypes.c_void_p] * 4 + [ctypes.c_int]
        L.ora_align_ends_free.restype = ctypes.c_int
        L.ora_align_ends_free.argtypes = [c_char_p, ctypes.c_int, c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, P(OraEnds), ctypes.c_void_p, ctypes.c_int, P(ctypes.c_int),
                                          P(OraStats)]
        L.ora_align_batch_ends_free.restype = ctypes.c_int
        L.ora_align_batch_ends_free.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 6 + [ctypes.c_int] * 3 + [
            P(OraEnds)] + [ctypes.c_void_p] * 4 + [ctypes.c_int]
        L.ora_gotoh_ends_free_score.restype = ctypes.c_int
        L.ora_gotoh_ends_free_score.argtypes = [c_char_p, ctypes.c_int, c_char_p, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_int, ctypes.c_int, P(OraEnds)]
        L.ora_cigar_cost_ends_free.restype = i64
        L.ora_cigar_cost_ends_free.argtypes = [c_char_p, ctypes.c_int, c_char_p, ctypes.c_int, c_char_p,
                                               ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, P(OraEnds)]
        L.ora_align_linear_ends_free.restype = ctypes.c_int
        L.ora_align_linear_ends_free.argtypes = [c_char_p, ctypes.c_int, c_char_p, ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_int, P(OraEnds), ctypes.c_void_p, ctypes.c_int,
                                                 P(ctypes.c_int), P(OraStats)]
        L.ora_align_batch_linear_ends_free.restype = ctypes.c_int
        L.ora_align_batch_linear_ends_free.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 6 + [ctypes.c_int] * 2 + [
            P(OraEnds)] + [ctypes.c_void_p] * 4 + [ctypes.c_int]
        L.ora_align2_ends_free.restype = ctypes.c_int
        L.ora_align2_ends_free.argtypes = [c_char_p, ctypes.c_int, c_char_p, ctypes.c_int] + [ctypes.c_int] * 5 + [
            P(OraEnds), ctypes.c_void_p, ctypes.c_int, P(ctypes.c_int), P(OraStats)]
        L.ora_align_batch2_ends_free.restype = ctypes.c_int
        L.ora_align_batch2_ends_free.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 6 + [ctypes.c_int] * 5 + [
            P(OraEnds)] + [ctypes.c_void_p] * 4 + [ctypes.c_int]
        L.ora_gotoh2_ends_free_score.restype = ctypes.c_int
        L.ora_gotoh2_ends_free_score.argtypes = [c_char_p, ctypes.c_int, c_char_p, ctypes.c_int] + [
            ctypes.c_int] * 5 + [P(OraEnds)]
        L.ora_align_batch2.restype = ctypes.c_int
        L.ora_align_batch2.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 6 + [ctypes.c_int] * 5 + [
            ctypes.c_void_p] * 4 + [ctypes.c_int]
        L.ora_gen_batch.argtypes = [ctypes.c_uint64, ctypes.c_int64, ctypes.c_int64] + [ctypes.c_void_p] * 8
        L.ora_refk_batch.argtypes = [ctypes.c_void_p] * 2 + [ctypes.c_int64] * 3 + [ctypes.c_int] * 6 + [
            ctypes.c_void_p] * 4
        _lib = L
    return _lib


def _b(s) -> bytes:
    return s if isinstance(s, (bytes, bytearray)) else s.encode()


def align(pattern, text, x=4, o=6, e=2, cigar=True) -> Tuple[int, Optional[str]]:
    """Align one pair; returns (score, WFA2-style operation string or None)."""
    p, t = _b(pattern), _b(text)
    cap = len(p) + len(t) + 1
    buf = ctypes.create_string_buffer(cap) if cigar else None
    n_ops = ctypes.c_int(0)
    r = lib().ora_align(p, len(p), t, len(t), x, o, e, buf, cap, ctypes.byref(n_ops), None)
    if r < 0:
        raise RuntimeError(f"oracle error {r}")
    return r, (buf.raw[: n_ops.value].decode() if cigar else None)


def gotoh(pattern, text, x=4, o=6, e=2) -> int:
    p, t = _b(pattern), _b(text)
    return lib().ora_gotoh_score(p, len(p), t, len(t), x, o, e)


def cigar_cost(ops: str, pattern, text, x=4, o=6, e=2) -> int:
    p, t, c = _b(pattern), _b(text), _b(ops)
    return lib().ora_cigar_cost(c, len(c), p, len(p), t, len(t), x, o, e)


def ops_to_rle(ops: str) -> np.ndarray:
    c = _b(ops)
    out = np.zeros(max(1, len(c)), dtype=np.uint32)
    n = lib().ora_ops_to_rle(c, len(c), out.ctypes.data, out.size)
    return out[:n]


def align_batch(patterns: Sequence, texts: Sequence, x=4, o=6, e=2, cigar=True, threads=0,
                stats: bool = False):
    """OpenMP batch alignment.  Returns (scores int32[N], list of op strings or None[, OraStats])."""
    pats = [_b(p) for p in patterns]
    txts = [_b(t) for t in texts]
    n = len(pats)
    plen = np.array([len(p) for p in pats], dtype=np.int32)
    tlen = np.array([len(t) for t in txts], dtype=np.int32)
    poff = np.zeros(n + 1, dtype=np.int64)
    toff = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(plen, out=poff[1:])
    np.cumsum(tlen, out=toff[1:])
    pbuf = np.frombuffer(b"".join(pats) + b"\0", dtype=np.uint8)
    tbuf = np.frombuffer(b"".join(txts) + b"\0", dtype=np.uint8)
    return align_batch_arrays(pbuf, poff, plen, tbuf, toff, tlen, x, o, e, cigar, threads, stats)


def align_batch_arrays(pbuf, poff, plen, tbuf, toff, tlen, x=4, o=6, e=2, cigar=True, threads=0,
                       stats: bool = False):
    n = len(plen)
    scores = np.zeros(n, dtype=np.int32)
    ops = ops_off = ops_len = None
    if cigar:
        caps = plen.astype(np.int64) + tlen.astype(np.int64) + 1
        ops_off = np.zeros(n + 1, dtype=np.int64)
        np.cumsum(caps, out=ops_off[1:])
        ops = np.zeros(int(ops_off[-1]) + 1, dtype=np.uint8)
        ops_len = np.zeros(n, dtype=np.int32)
    st = OraStats()
    r = lib().ora_align_batch(
        n, pbuf.ctypes.data, poff.ctypes.data, plen.ctypes.data, tbuf.ctypes.data, toff.ctypes.data,
        tlen.ctypes.data, x, o, e, scores.ctypes.data,
        ops.ctypes.data if cigar else None, ops_off.ctypes.data if cigar else None,
        ops_len.ctypes.data if cigar else None, threads, ctypes.byref(st))
    if r < 0:
        raise RuntimeError(f"oracle batch error {r}")
    cig: Optional[List[str]] = None
    if cigar:
        raw = ops.tobytes()
        cig = [raw[ops_off[i]: ops_off[i] + ops_len[i]].decode() for i in range(n)]
    if stats:
        return scores, cig, st
    return scores, cig


def max_threads() -> int:
    return lib().ora_max_threads()


# --- dual gap-affine (two-piece) mode: a gap of length L costs
# min(o1 + e1*L, o2 + e2*L) --------------------------------------------------

def align2(pattern, text, x=4, o1=6, e1=2, o2=24, e2=1, cigar=True) -> Tuple[int, Optional[str]]:
    """Align one pair under the two-piece model; returns (score, ops or None)."""
    p, t = _b(pattern), _b(text)
    cap = len(p) + len(t) + 1
    buf = ctypes.create_string_buffer(cap) if cigar else None
    n_ops = ctypes.c_int(0)
    r = lib().ora_align2(p, len(p), t, len(t), x, o1, e1, o2, e2, buf, cap, ctypes.byref(n_ops), None)
    if r < 0:
        raise RuntimeError(f"oracle error {r}")
    return r, (buf.raw[: n_ops.value].decode() if cigar else None)


def gotoh2(pattern, text, x=4, o1=6, e1=2, o2=24, e2=1) -> int:
    p, t = _b(pattern), _b(text)
    return lib().ora_gotoh2_score(p, len(p), t, len(t), x, o1, e1, o2, e2)


def cigar_cost2(ops: str, pattern, text, x=4, o1=6, e1=2, o2=24, e2=1) -> int:
    p, t, c = _b(pattern), _b(text), _b(ops)
    return lib().ora_cigar_cost2(c, len(c), p, len(p), t, len(t), x, o1, e1, o2, e2)


def align_batch2(patterns: Sequence, texts: Sequence, x=4, o1=6, e1=2, o2=24, e2=1, cigar=True, threads=0):
    """OpenMP batch under the two-piece model.  Returns (scores int32[N], op strings or None)."""
    pats = [_b(p) for p in patterns]
    txts = [_b(t) for t in texts]
    n = len(pats)
    plen = np.array([len(p) for p in pats], dtype=np.int32)
    tlen = np.array([len(t) for t in txts], dtype=np.int32)
    poff = np.zeros(n + 1, dtype=np.int64)
    toff = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(plen, out=poff[1:])
    np.cumsum(tlen, out=toff[1:])
    pbuf = np.frombuffer(b"".join(pats) + b"\0", dtype=np.uint8)
    tbuf = np.frombuffer(b"".join(txts) + b"\0", dtype=np.uint8)
    return align_batch2_arrays(pbuf, poff, plen, tbuf, toff, tlen, x, o1, e1, o2, e2, cigar, threads)


def align_batch2_arrays(pbuf, poff, plen, tbuf, toff, tlen, x=4, o1=6, e1=2, o2=24, e2=1, cigar=True, threads=0):
    n = len(plen)
    scores = np.zeros(n, dtype=np.int32)
    ops = ops_off = ops_len = None
    if cigar:
        caps = plen.astype(np.int64) + tlen.astype(np.int64) + 1
        ops_off = np.zeros(n + 1, dtype=np.int64)
        np.cumsum(caps, out=ops_off[1:])
        ops = np.zeros(int(ops_off[-1]) + 1, dtype=np.uint8)
        ops_len = np.zeros(n, dtype=np.int32)
    r = lib().ora_align_batch2(
        n, pbuf.ctypes.data, poff.ctypes.data, plen.ctypes.data, tbuf.ctypes.data, toff.ctypes.data,
        tlen.ctypes.data, x, o1, e1, o2, e2, scores.ctypes.data,
        ops.ctypes.data if cigar else None, ops_off.ctypes.data if cigar else None,
        ops_len.ctypes.data if cigar else None, threads)
    if r < 0:
        raise RuntimeError(f"oracle batch error {r}")
    cig: Optional[List[str]] = None
    if cigar:
        raw = ops.tobytes()
        cig = [raw[ops_off[i]: ops_off[i] + ops_len[i]].decode() for i in range(n)]
    return scores, cig


# --- gap-linear mode (edit distance: x = e = 1; indel: x = 3, e = 1) ---------

def align_linear(pattern, text, x=1, e=1, cigar=True) -> Tuple[int, Optional[str]]:
    """Align one pair with gap cost e*L; returns (score, ops or None)."""
    p, t = _b(pattern), _b(text)
    cap = len(p) + len(t) + 1
    buf = ctypes.create_string_buffer(cap) if cigar else None
    n_ops = ctypes.c_int(0)
    r = lib().ora_align_linear(p, len(p), t, len(t), x, e, buf, cap, ctypes.byref(n_ops), None)
    if r < 0:
        raise RuntimeError(f"oracle error {r}")
    return r, (buf.raw[: n_ops.value].decode() if cigar else None)


def linear_dp(pattern, text, x=1, e=1) -> int:
    p, t = _b(pattern), _b(text)
    return lib().ora_linear_dp_score(p, len(p), t, len(t), x, e)


def align_batch_linear(patterns: Sequence, texts: Sequence, x=1, e=1, cigar=True, threads=0):
    """OpenMP batch with gap cost e*L.  Returns (scores int32[N], op strings or None)."""
    pats = [_b(p) for p in patterns]
    txts = [_b(t) for t in texts]
    n = len(pats)
    plen = np.array([len(p) for p in pats], dtype=np.int32)
    tlen = np.array([len(t) for t in txts], dtype=np.int32)
    poff = np.zeros(n + 1, dtype=np.int64)
    toff = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(plen, out=poff[1:])
    np.cumsum(tlen, out=toff[1:])
    pbuf = np.frombuffer(b"".join(pats) + b"\0", dtype=np.uint8)
    tbuf = np.frombuffer(b"".join(txts) + b"\0", dtype=np.uint8)
    return align_batch_linear_arrays(pbuf, poff, plen, tbuf, toff, tlen, x, e, cigar, threads)


def align_batch_linear_arrays(pbuf, poff, plen, tbuf, toff, tlen, x=1, e=1, cigar=True, threads=0):
    n = len(plen)
    scores = np.zeros(n, dtype=np.int32)
    ops = ops_off = ops_len = None
    if cigar:
        caps = plen.astype(np.int64) + tlen.astype(np.int64) + 1
        ops_off = np.zeros(n + 1, dtype=np.int64)
        np.cumsum(caps, out=ops_off[1:])
        ops = np.zeros(int(ops_off[-1]) + 1, dtype=np.uint8)
        ops_len = np.zeros(n, dtype=np.int32)
    r = lib().ora_align_batch_linear(
        n, pbuf.ctypes.data, poff.ctypes.data, plen.ctypes.data, tbuf.ctypes.data, toff.ctypes.data,
        tlen.ctypes.data, x, e, scores.ctypes.data,
        ops.ctypes.data if cigar else None, ops_off.ctypes.data if cigar else None,
        ops_len.ctypes.data if cigar else None, threads)
    if r < 0:
        raise RuntimeError(f"oracle batch error {r}")
    cig: Optional[List[str]] = None
    if cigar:
        raw = ops.tobytes()
        cig = [raw[ops_off[i]: ops_off[i] + ops_len[i]].decode() for i in range(n)]
    return scores, cig


# --- ends-free gap-affine (free = (pattern_begin, pattern_end, text_begin, text_end)) --

def align_ends_free(pattern, text, free, x=4, o=6, e=2, cigar=True) -> Tuple[int, Optional[str]]:
    p, t = _b(pattern), _b(text)
    cap = len(p) + len(t) + 1
    buf = ctypes.create_string_buffer(cap) if cigar else None
    n_ops = ctypes.c_int(0)
    r = lib().ora_align_ends_free(p, len(p), t, len(t), x, o, e, ctypes.byref(OraEnds(*free)), buf, cap,
                                  ctypes.byref(n_ops), None)
    if r < 0:
        raise RuntimeError(f"oracle error {r}")
    return r, (buf.raw[: n_ops.value].decode() if cigar else None)


def gotoh_ends_free(pattern, text, free, x=4, o=6, e=2) -> int:
    p, t = _b(pattern), _b(text)
    return lib().ora_gotoh_ends_free_score(p, len(p), t, len(t), x, o, e, ctypes.byref(OraEnds(*free)))


def cigar_cost_ends_free(ops: str, pattern, text, free, x=4, o=6, e=2) -> int:
    p, t, c = _b(pattern), _b(text), _b(ops)
    return lib().ora_cigar_cost_ends_free(c, len(c), p, len(p), t, len(t), x, o, e, ctypes.byref(OraEnds(*free)))


def align_batch_ends_free(patterns: Sequence, texts: Sequence, free, x=4, o=6, e=2, cigar=True, threads=0):
    """OpenMP batch with free ends.  Returns (scores int32[N], op strings or None)."""
    pats = [_b(p) for p in patterns]
    txts = [_b(t) for t in texts]
    n = len(pats)
    plen = np.array([len(p) for p in pats], dtype=np.int32)
    tlen = np.array([len(t) for t in txts], dtype=np.int32)
    poff = np.zeros(n + 1, dtype=np.int64)
    toff = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(plen, out=poff[1:])
    np.cumsum(tlen, out=toff[1:])
    pbuf = np.frombuffer(b"".join(pats) + b"\0", dtype=np.uint8)
    tbuf = np.frombuffer(b"".join(txts) + b"\0", dtype=np.uint8)
    return align_batch_ends_free_arrays(pbuf, poff, plen, tbuf, toff, tlen, free, x, o, e, cigar, threads)


def align_batch_ends_free_arrays(pbuf, poff, plen, tbuf, toff, tlen, free, x=4, o=6, e=2, cigar=True, threads=0):
    n = len(plen)
    scores = np.zeros(n, dtype=np.int32)
    ops = ops_off = ops_len = None
    if cigar:
        caps = plen.astype(np.int64) + tlen.astype(np.int64) + 1
        ops_off = np.zeros(n + 1, dtype=np.int64)
        np.cumsum(caps, out=ops_off[1:])
        ops = np.zeros(int(ops_off[-1]) + 1, dtype=np.uint8)
        ops_len = np.zeros(n, dtype=np.int32)
    r = lib().ora_align_batch_ends_free(
        n, pbuf.ctypes.data, poff.ctypes.data, plen.ctypes.data, tbuf.ctypes.data, toff.ctypes.data,
        tlen.ctypes.data, x, o, e, ctypes.byref(OraEnds(*free)), scores.ctypes.data,
        ops.ctypes.data if cigar else None, ops_off.ctypes.data if cigar else None,
        ops_len.ctypes.data if cigar else None, threads)
    if r < 0:
        raise RuntimeError(f"oracle batch error {r}")
    cig: Optional[List[str]] = None
    if cigar:
        raw = ops.tobytes()
        cig = [raw[ops_off[i]: ops_off[i] + ops_len[i]].decode() for i in range(n)]
    return scores, cig


# --- free ends for the gap-linear and dual gap-affine oracles ------------------

def align_linear_ends_free(pattern, text, free, x=1, e=1, cigar=True):
    p, t = _b(pattern), _b(text)
    cap = len(p) + len(t) + 1
    buf = ctypes.create_string_buffer(cap) if cigar else None
    n_ops = ctypes.c_int(0)
    r = lib().ora_align_linear_ends_free(p, len(p), t, len(t), x, e, ctypes.byref(OraEnds(*free)), buf, cap,
                                         ctypes.byref(n_ops), None)
    if r < 0:
        raise RuntimeError(f"oracle error {r}")
    return r, (buf.raw[: n_ops.value].decode() if cigar else None)


def align2_ends_free(pattern, text, free, x=4, o1=6, e1=2, o2=24, e2=1, cigar=True):
    p, t = _b(pattern), _b(text)
    cap = len(p) + len(t) + 1
    buf = ctypes.create_string_buffer(cap) if cigar else None
    n_ops = ctypes.c_int(0)
    r = lib().ora_align2_ends_free(p, len(p), t, len(t), x, o1, e1, o2, e2, ctypes.byref(OraEnds(*free)), buf, cap,
                                   ctypes.byref(n_ops), None)
    if r < 0:
        raise RuntimeError(f"oracle error {r}")
    return r, (buf.raw[: n_ops.value].decode() if cigar else None)


def gotoh2_ends_free(pattern, text, free, x=4, o1=6, e1=2, o2=24, e2=1) -> int:
    p, t = _b(pattern), _b(text)
    return lib().ora_gotoh2_ends_free_score(p, len(p), t, len(t), x, o1, e1, o2, e2, ctypes.byref(OraEnds(*free)))


def _batch_free(fn, patterns, texts, pen, free, cigar, threads):
    pats = [_b(p) for p in patterns]
    txts = [_b(t) for t in texts]
    n = len(pats)
    plen = np.array([len(p) for p in pats], dtype=np.int32)
    tlen = np.array([len(t) for t in txts], dtype=np.int32)
    poff = np.zeros(n + 1, dtype=np.int64)
    toff = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(plen, out=poff[1:])
    np.cumsum(tlen, out=toff[1:])
    pbuf = np.frombuffer(b"".join(pats) + b"\0", dtype=np.uint8)
    tbuf = np.frombuffer(b"".join(txts) + b"\0", dtype=np.uint8)
    scores = np.zeros(n, dtype=np.int32)
    ops = ops_off = ops_len = None
    if cigar:
        caps = plen.astype(np.int64) + tlen.astype(np.int64) + 1
        ops_off = np.zeros(n + 1, dtype=np.int64)
        np.cumsum(caps, out=ops_off[1:])
        ops = np.zeros(int(ops_off[-1]) + 1, dtype=np.uint8)
        ops_len = np.zeros(n, dtype=np.int32)
    r = fn(n, pbuf.ctypes.data, poff.ctypes.data, plen.ctypes.data, tbuf.ctypes.data, toff.ctypes.data,
           tlen.ctypes.data, *pen, ctypes.byref(OraEnds(*free)), scores.ctypes.data,
           ops.ctypes.data if cigar else None, ops_off.ctypes.data if cigar else None,
           ops_len.ctypes.data if cigar else None, threads)
    if r < 0:
        raise RuntimeError(f"oracle batch error {r}")
    cig: Optional[List[str]] = None
    if cigar:
        raw = ops.tobytes()
        cig = [raw[ops_off[i]: ops_off[i] + ops_len[i]].decode() for i in range(n)]
    return scores, cig


def align_batch_linear_ends_free(patterns, texts, free, x=1, e=1, cigar=True, threads=0):
    return _batch_free(lib().ora_align_batch_linear_ends_free, patterns, texts, (x, e), free, cigar, threads)


def align_batch2_ends_free(patterns, texts, free, x=4, o1=6, e1=2, o2=24, e2=1, cigar=True, threads=0):
    return _batch_free(lib().ora_align_batch2_ends_free, patterns, texts, (x, o1, e1, o2, e2), free, cigar, threads)


def bialign(pattern, text, x=4, o=6, e=2, base_score=0, ring=False) -> str:
    """Operations of the bidirectional alignment (ora_bialign: breakpoint
    recursion, the C form of bidir_rule.bialign; ring=True: cut by the
    two-ring crossing search, ora_bialign_ring)."""
    p, t = _b(pattern), _b(text)
    cap = len(p) + len(t) + 1
    buf = ctypes.create_string_buffer(cap)
    n = ctypes.c_int(0)
    fn = lib().ora_bialign_ring if ring else lib().ora_bialign
    rc = fn(p, len(p), t, len(t), x, o, e, base_score, buf, cap, ctypes.byref(n))
    if rc != 0:
        raise RuntimeError(f"ora_bialign failed: {rc}")
    return buf.raw[: n.value].decode()


def align_segment(pattern, text, x=4, o=6, e=2, begin="M", end="M"):
    """(cost, operations) of one segment with gap components
    (ora_align_segment, the C form of bidir_rule.wfa_segment)."""
    p, t = _b(pattern), _b(text)
    cap = len(p) + len(t) + 1
    buf = ctypes.create_string_buffer(cap)
    n = ctypes.c_int(0)
    rc = lib().ora_align_segment(p, len(p), t, len(t), x, o, e, begin.encode(), end.encode(), buf, cap,
                                 ctypes.byref(n))
    if rc < 0:
        raise RuntimeError(f"ora_align_segment failed: {rc}")
    return rc, buf.raw[: n.value].decode()


def gen_batch(seed: int, lengths: np.ndarray, rates: np.ndarray, first: int = 0):
    """Seeded synthetic pairs (ora_gen_batch, wfa_gen.c): the same bytes as
    the engine's tsu_gen_batch for the same arguments, without loading the
    engine library.  Returns (pbuf, poff, plen, tbuf, toff, tlen)."""
    lengths = np.ascontiguousarray(lengths, dtype=np.int32)
    rates = np.ascontiguousarray(rates, dtype=np.float64)
    n = lengths.size
    off = np.zeros(n, dtype=np.int64)
    if n > 1:
        np.cumsum(lengths[:-1], out=off[1:])
    total = int(lengths.sum())
    pbuf = np.zeros(total + 16, dtype=np.uint8)
    tbuf = np.zeros(total + 16, dtype=np.uint8)
    plen = np.zeros(n, dtype=np.int32)
    tlen = np.zeros(n, dtype=np.int32)
    rc = lib().ora_gen_batch(seed, first, n, lengths.ctypes.data, rates.ctypes.data, pbuf.ctypes.data,
                             off.ctypes.data, plen.ctypes.data, tbuf.ctypes.data, off.ctypes.data, tlen.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"ora_gen_batch error {rc}")
    return pbuf, off, plen, tbuf, off.copy(), tlen


def refk_batch(seed: int, first: int, num: int, length: int, rate: float, x=4, o=6, e=2, wf_length: int = 0,
               step_cap: int = 32000):
    """The CPU model of the reference's GPU kernel (ref_kernel_model.c) on the
    pairs oracle/_ref/ref_harness generates for the same arguments, laid out
    as the harness lays them out (pairs of `length` bytes back to back,
    2 * length + 256 pad bytes before and after, 0x01 in the pattern buffer
    and 0x02 in the text buffer).  Returns (scores int16, codes, steps,
    max |k|) per pair; codes are 0 or ORA_REFK_* (-10 ring, -11 sequence
    read, -12 step cap)."""
    lengths = np.full(num, length, np.int32)
    pb, po, pl, tb, to, tl = gen_batch(seed, lengths, np.full(num, rate), first=first)
    if not (np.all(pl == length) and np.all(tl == length)):
        raise ValueError("the reference kernel needs pairs of equal length")
    pad = 2 * length + 256
    P = np.full(pad + num * length + pad, 1, np.uint8)
    T = np.full(pad + num * length + pad, 2, np.uint8)
    P[pad:pad + num * length] = pb[:num * length]
    T[pad:pad + num * length] = tb[:num * length]
    wf = wf_length or 2 * (length + 3) + 2
    sc = np.zeros(num, np.int16)
    codes = np.zeros(num, np.int32)
    steps = np.zeros(num, np.int32)
    maxk = np.zeros(num, np.int32)
    rc = lib().ora_refk_batch(P.ctypes.data + pad, T.ctypes.data + pad, pad, pad, num, length, x, o, e, wf, step_cap,
                              sc.ctypes.data, codes.ctypes.data, steps.ctypes.data, maxk.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"ora_refk_batch error {rc}")
    return sc, codes, steps, maxk


def crossing_split(pattern, text, x=4, o=6, e=2, begin="M", end="M"):
    """The two-ring breakpoint search on one segment (ora_crossing_split):
    (total, component, forward diagonal, cut offset), or None when nothing
    crosses."""
    p, t = _b(pattern), _b(text)
    T, k, h = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
    comp = ctypes.create_string_buffer(1)
    rc = lib().ora_crossing_split(p, len(p), t, len(t), x, o, e, begin.encode(), end.encode(), ctypes.byref(T),
                                  comp, ctypes.byref(k), ctypes.byref(h))
    if rc < 0:
        raise RuntimeError(f"ora_crossing_split failed: {rc}")
    if rc == 0:
        return None
    return T.value, comp.raw[:1].decode(), k.value, h.value
