"""ctypes binding of libtsunami_b200.so (include/tsunami_b200.h)."""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import List, Optional, Sequence, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "libtsunami_b200.so")
_lib = None

TSU_OK = 0
TSU_ENOMEM = 2
TSU_ETIMEOUT = 4
TSU_EOVERFLOW = 5
TSU_EBUSY = 6
TSU_ENOTFOUND = 7
TSU_EPENDING = 10
TSU_SCORE_ONLY = 0x1
TSU_ONE_WARP = 0x2
TSU_BIDIRECTIONAL = 0x4

P = ctypes.POINTER
c_i32, c_i64, c_u32, c_vp = ctypes.c_int32, ctypes.c_int64, ctypes.c_uint32, ctypes.c_void_p


class Penalties(ctypes.Structure):
    _fields_ = [("mismatch", c_i32), ("gap_opening", c_i32), ("gap_extension", c_i32)]


class Penalties2(ctypes.Structure):
    """Dual gap-affine penalties: a gap of length L costs
    min(gap_opening + gap_extension*L, gap_opening2 + gap_extension2*L)."""
    _fields_ = [("mismatch", c_i32), ("gap_opening", c_i32), ("gap_extension", c_i32), ("gap_opening2", c_i32),
                ("gap_extension2", c_i32)]


class Config(ctypes.Structure):
    _fields_ = [("device", c_i32), ("reserved0", c_i32), ("mem_budget", ctypes.c_size_t),
                ("max_error_hint", ctypes.c_double)]


class Batch(ctypes.Structure):
    _fields_ = [("num_pairs", c_i64), ("pattern", c_vp), ("pattern_off", c_vp), ("pattern_len", c_vp),
                ("text", c_vp), ("text_off", c_vp), ("text_len", c_vp)]


class Result(ctypes.Structure):
    _fields_ = [("score", c_vp), ("cigar", c_vp), ("cigar_capacity", c_i64), ("cigar_offset", c_vp),
                ("cigar_needed", c_i64), ("pair_status", c_vp)]


class Timing(ctypes.Structure):
    _fields_ = [("h2d_ms", ctypes.c_double), ("pack_ms", ctypes.c_double), ("align_ms", ctypes.c_double),
                ("compact_ms", ctypes.c_double), ("d2h_ms", ctypes.c_double), ("total_ms", ctypes.c_double),
                ("kernel_launches", c_i64), ("retried_pairs", c_i64), ("h2d_bytes", c_i64),
                ("d2h_bytes", c_i64), ("cells", c_i64), ("steps", c_i64), ("ext_bases", c_i64),
                ("device_bytes", c_i64)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("device", c_i32), ("workers", c_i32), ("mem_budget", ctypes.c_size_t),
                ("max_error_hint", ctypes.c_double), ("max_queue", c_i64), ("max_job_pairs", c_i64),
                ("max_job_requests", c_i32), ("heavy_len", c_i32), ("heavy_workers", c_i32), ("estimate_hint", c_i32),
                ("watchdog_ms", ctypes.c_double), ("resident_bytes", ctypes.c_size_t)]


class RequestInfo(ctypes.Structure):
    _fields_ = [("num_pairs", c_i64), ("queue_ms", ctypes.c_double), ("latency_ms", ctypes.c_double),
                ("job_requests", c_i32), ("attempts", c_i32), ("job_seq", c_i64)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", c_i64), ("completed", c_i64), ("failed", c_i64), ("rejected", c_i64),
                ("cancelled", c_i64), ("timed_out", c_i64), ("queued", c_i64), ("running", c_i64),
                ("jobs", c_i64), ("pairs_completed", c_i64), ("mean_requests_per_job", ctypes.c_double),
                ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double), ("p999_ms", ctypes.c_double),
                ("mean_ms", ctypes.c_double), ("max_ms", ctypes.c_double), ("elapsed_s", ctypes.c_double),
                ("budget_bytes", ctypes.c_uint64), ("granted_bytes", ctypes.c_uint64),
                ("peak_granted_bytes", ctypes.c_uint64), ("workers", c_i32), ("reserved0", c_i32),
                ("heavy_jobs", c_i64), ("busy_s", ctypes.c_double), ("heavy_busy_s", ctypes.c_double)]


class AlignError(RuntimeError):
    def __init__(self, code: int, msg: str, needed: int = 0):
        super().__init__(f"tsunami_b200 error {code}: {msg}")
        self.code = code
        self.needed = needed  # CIGAR runs needed, for TSU_EOVERFLOW


def lib_path() -> str:
    return _LIB


def build() -> None:
    """Compile the engine in-tree (nvcc, sm_100a)."""
    subprocess.run(["make", "-s", "-C", os.path.join(_HERE, "csrc")], check=True)


def lib():
    """Load libtsunami_b200.so; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB):
        raise RuntimeError(f"{_LIB} is missing: build the CUDA engine first (tsunami_pact_b200.build())")
    L = ctypes.CDLL(_LIB)
    L.tsu_create.argtypes = [P(Penalties), P(Config), P(c_vp)]
    L.tsu_create_dual.argtypes = [P(Penalties2), P(Config), P(c_vp)]
    L.tsu_create_metric.argtypes = [ctypes.c_int, c_vp, ctypes.c_int, P(Config), P(c_vp)]
    L.tsu_server_create_metric.argtypes = [ctypes.c_int, c_vp, ctypes.c_int, c_vp, P(c_vp)]
    L.tsu_destroy.argtypes = [c_vp]
    L.tsu_status_str.restype = ctypes.c_char_p
    L.tsu_status_str.argtypes = [ctypes.c_int]
    L.tsu_last_error.restype = ctypes.c_char_p
    L.tsu_last_error.argtypes = [c_vp]
    L.tsu_get_timing.argtypes = [c_vp, P(Timing)]
    L.tsu_align_batch.argtypes = [c_vp, P(Batch), P(Result), c_u32]
    L.tsu_align_batch_device.argtypes = [c_vp, P(Batch), P(Result), c_u32]
    L.tsu_align_fixed.argtypes = [c_vp, c_vp, c_vp, c_i64, c_i32, c_i32, c_vp, c_u32]
    L.tsu_cigar_to_ops.restype = c_i64
    L.tsu_cigar_to_ops.argtypes = [c_vp, c_i64, c_vp, c_i64]
    L.tsu_cigar_to_string.restype = c_i64
    L.tsu_cigar_to_string.argtypes = [c_vp, c_i64, c_vp, c_i64]
    L.tsu_file_read.argtypes = [ctypes.c_char_p, P(c_vp)]
    L.tsu_file_read_pairs.argtypes = [ctypes.c_char_p, ctypes.c_char_p, P(c_vp)]
    L.tsu_file_batch.argtypes = [c_vp, P(Batch)]
    L.tsu_file_header.argtypes = [c_vp, P(c_i64), P(c_i32), P(c_i32)]
    L.tsu_file_free.argtypes = [c_vp]
    L.tsu_file_free.restype = None
    L.tsu_file_write.argtypes = [ctypes.c_char_p, c_i64, c_i32, c_i32, P(Batch)]
    L.tsu_gen_pair.argtypes = [ctypes.c_uint64, c_i64, c_i32, ctypes.c_double, c_vp, P(c_i32), c_vp, P(c_i32)]
    L.tsu_gen_batch.argtypes = [ctypes.c_uint64, c_i64, c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp,
                                ctypes.c_int]
    L.tsu_predict_bytes.argtypes = [c_vp, P(Batch), c_u32, P(ctypes.c_size_t), P(ctypes.c_size_t)]
    L.tsu_shard_plan.argtypes = [P(Penalties), P(Batch), c_i32, ctypes.c_double, c_vp, c_vp]
    L.tsu_server_create.argtypes = [P(Penalties), P(ServerConfig), P(c_vp)]
    L.tsu_server_create_dual.argtypes = [P(Penalties2), P(ServerConfig), P(c_vp)]
    L.tsu_server_destroy.argtypes = [c_vp]
    L.tsu_submit.argtypes = [c_vp, P(Batch), c_u32, P(ctypes.c_uint64)]
    L.tsu_poll.argtypes = [c_vp, ctypes.c_uint64, P(Result), P(RequestInfo)]
    L.tsu_wait.argtypes = [c_vp, ctypes.c_uint64, ctypes.c_double, P(Result), P(RequestInfo)]
    L.tsu_cancel.argtypes = [c_vp, ctypes.c_uint64]
    L.tsu_server_get_stats.argtypes = [c_vp, P(ServerStats)]
    L.tsu_server_reset_stats.argtypes = [c_vp]
    L.tsu_server_last_error.restype = ctypes.c_char_p
    L.tsu_server_last_error.argtypes = [c_vp]
    _lib = L
    return L


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data


def _concat(seqs: Sequence) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    bs = [s if isinstance(s, (bytes, bytearray)) else s.encode() for s in seqs]
    lens = np.fromiter((len(b) for b in bs), dtype=np.int32, count=len(bs))
    off = np.zeros(len(bs), dtype=np.int64)
    if len(bs) > 1:
        np.cumsum(lens[:-1], out=off[1:])
    buf = np.frombuffer(b"".join(bs) + b"\0", dtype=np.uint8)
    return buf, off, lens


def runs_to_ops(runs: np.ndarray) -> str:
    """Run-length CIGAR -> WFA2 operation string ('M','X','I','D' per op)."""
    runs = np.ascontiguousarray(runs, dtype=np.uint32)
    total = int((runs >> 4).sum()) if runs.size else 0
    out = ctypes.create_string_buffer(total + 1)
    w = lib().tsu_cigar_to_ops(_ptr(runs), runs.size, out, total + 1)
    return out.raw[:w].decode()


def runs_to_string(runs: np.ndarray) -> str:
    runs = np.ascontiguousarray(runs, dtype=np.uint32)
    cap = 12 * runs.size + 1
    out = ctypes.create_string_buffer(cap)
    w = lib().tsu_cigar_to_string(_ptr(runs), runs.size, out, cap)
    return out.raw[:w].decode()


# TSU_METRIC_* (include/tsunami_b200.h): WFA2-lib's distance metrics
METRICS = {"indel": 0, "edit": 1, "gap_linear": 2, "gap_affine": 3, "gap_affine_2p": 4}


def metric_penalties(metric: Optional[str], mismatch, gap_opening, gap_extension, gap_opening2, gap_extension2):
    """(TSU_METRIC_* code, penalties tuple) of the constructor arguments:
    metric None means gap_affine, or gap_affine_2p when a second gap piece is
    given."""
    if metric is None:
        metric = "gap_affine" if gap_opening2 is None and gap_extension2 is None else "gap_affine_2p"
    if metric not in METRICS:
        raise ValueError(f"unknown metric {metric!r} (one of {', '.join(METRICS)})")
    pens = {"indel": (), "edit": (), "gap_linear": (mismatch, gap_extension),
            "gap_affine": (mismatch, gap_opening, gap_extension),
            "gap_affine_2p": (mismatch, gap_opening, gap_extension,
                              -1 if gap_opening2 is None else gap_opening2,
                              0 if gap_extension2 is None else gap_extension2)}[metric]
    return METRICS[metric], tuple(int(v) for v in pens)


class Aligner:
    """One device context with fixed penalties (reference argv 1-3,
    wfa_gpu.cu:59-61).  With ``gap_opening2`` and ``gap_extension2`` the
    context aligns under dual gap-affine penalties; ``metric`` selects any of
    WFA2-lib's distance metrics ("indel", "edit", "gap_linear" with mismatch
    and gap_extension, "gap_affine", "gap_affine_2p"), tsu_create_metric."""

    def __init__(self, mismatch: int = 4, gap_opening: int = 6, gap_extension: int = 2, device: int = 0,
                 mem_budget: int = 0, max_error_hint: float = 0.0, gap_opening2: Optional[int] = None,
                 gap_extension2: Optional[int] = None, metric: Optional[str] = None):
        L = lib()
        cfg = Config(device, 0, mem_budget, max_error_hint)
        h = c_vp()
        code, pens = metric_penalties(metric, mismatch, gap_opening, gap_extension, gap_opening2, gap_extension2)
        self.metric = [k for k, v in METRICS.items() if v == code][0]
        self.penalties = pens
        arr = (ctypes.c_int32 * max(1, len(pens)))(*pens)
        rc = L.tsu_create_metric(code, ctypes.cast(arr, c_vp) if pens else None, len(pens), ctypes.byref(cfg),
                                 ctypes.byref(h))
        if rc != TSU_OK:
            raise AlignError(rc, L.tsu_status_str(rc).decode())
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().tsu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc: int):
        if rc != TSU_OK:
            L = lib()
            raise AlignError(rc, f"{L.tsu_status_str(rc).decode()}: {L.tsu_last_error(self._h).decode()}")

    def timing(self) -> dict:
        t = Timing()
        lib().tsu_get_timing(self._h, ctypes.byref(t))
        return {f: getattr(t, f) for f, _ in Timing._fields_}

    def set_ends_free(self, pattern_begin_free: int = 0, pattern_end_free: int = 0, text_begin_free: int = 0,
                      text_end_free: int = 0) -> None:
        """Ends-free alignment for the later calls (tsu_set_ends_free; WFA2-lib's
        wavefront_aligner_set_alignment_free_ends).  All 0: end-to-end."""
        L = lib()
        L.tsu_set_ends_free.argtypes = [c_vp, c_i32, c_i32, c_i32, c_i32]
        self._check(L.tsu_set_ends_free(self._h, pattern_begin_free, pattern_end_free, text_begin_free,
                                        text_end_free))

    def set_low_memory(self, checkpoint_interval: int = -1) -> None:
        """Low-memory CIGARs (tsu_set_low_memory): checkpoint the wavefront
        ring every checkpoint_interval scores (< 0: chosen per pass; 0: off)
        and recompute the history segment by segment for the backtrace."""
        L = lib()
        L.tsu_set_low_memory.argtypes = [c_vp, c_i32]
        self._check(L.tsu_set_low_memory(self._h, checkpoint_interval))

    def predict_bytes(self, plen, tlen, cigar: bool = True):
        """(full, min) device bytes tsu_align_batch would hold for pairs of
        these lengths (tsu_predict_bytes)."""
        L = lib()
        plen = np.ascontiguousarray(plen, dtype=np.int32)
        tlen = np.ascontiguousarray(tlen, dtype=np.int32)
        n = len(plen)
        poff = np.zeros(n, dtype=np.int64)
        toff = np.zeros(n, dtype=np.int64)
        if n:
            np.cumsum(plen[:-1], out=poff[1:])
            np.cumsum(tlen[:-1], out=toff[1:])
        dummy = np.zeros(1, dtype=np.uint8)  # sequences are not read, only lengths and offsets
        b = Batch(n, dummy.ctypes.data, poff.ctypes.data, plen.ctypes.data, dummy.ctypes.data, toff.ctypes.data,
                  tlen.ctypes.data)
        full, mn = ctypes.c_size_t(), ctypes.c_size_t()
        self._check(L.tsu_predict_bytes(self._h, ctypes.byref(b), 0 if cigar else TSU_SCORE_ONLY, ctypes.byref(full),
                                        ctypes.byref(mn)))
        return full.value, mn.value

    def pass_log(self) -> str:
        """Align passes of the last call: mode+warps per pair x groups : pairs @ time."""
        L = lib()
        L.tsu_pass_log.restype = ctypes.c_char_p
        L.tsu_pass_log.argtypes = [c_vp]
        return L.tsu_pass_log(self._h).decode()

    # -- host buffers ------------------------------------------------------
    def align_arrays(self, pbuf: np.ndarray, poff: np.ndarray, plen: np.ndarray, tbuf: np.ndarray,
                     toff: np.ndarray, tlen: np.ndarray, cigar: bool = True, status: bool = False,
                     cigar_capacity: Optional[int] = None, out=None, bidirectional: bool = False):
        """Align pairs given as concatenated byte buffers + offsets/lengths.

        Returns ``(scores, cigar_offsets, runs)``; the CIGAR parts are None
        with ``cigar=False``.  ``status=True`` appends per-pair statuses.
        ``out=(scores, offsets, runs)`` supplies preallocated (e.g. pinned)
        output arrays; ``runs.size`` is then the CIGAR capacity.
        ``bidirectional=True``: TSU_BIDIRECTIONAL -- scores by the
        bidirectional breakpoint search and CIGARs by its recursion, in
        memory linear in the score per pair."""
        n = len(plen)
        poff = np.ascontiguousarray(poff, dtype=np.int64)
        toff = np.ascontiguousarray(toff, dtype=np.int64)
        plen = np.ascontiguousarray(plen, dtype=np.int32)
        tlen = np.ascontiguousarray(tlen, dtype=np.int32)
        b = Batch(n, _ptr(pbuf), _ptr(poff), _ptr(plen), _ptr(tbuf), _ptr(toff), _ptr(tlen))
        scores = out[0] if out is not None else np.zeros(n, dtype=np.int32)
        st = np.zeros(n, dtype=np.int32)
        L = lib()
        if not cigar:
            r = Result(_ptr(scores), None, 0, None, 0, _ptr(st))
            flags = TSU_SCORE_ONLY | (TSU_BIDIRECTIONAL if bidirectional else 0)
            self._check(L.tsu_align_batch(self._h, ctypes.byref(b), ctypes.byref(r), flags))
            return (scores, None, None, st) if status else (scores, None, None)
        if out is not None:
            coff, runs = out[1], out[2]
            cigar_capacity = runs.size
        else:
            coff = np.zeros(n + 1, dtype=np.int64)
        cap = int(cigar_capacity) if cigar_capacity is not None else 0
        if out is None:
            runs = np.zeros(max(cap, 1), dtype=np.uint32)
        r = Result(_ptr(scores), _ptr(runs), cap, _ptr(coff), 0, _ptr(st))
        flags = TSU_BIDIRECTIONAL if bidirectional else 0
        rc = L.tsu_align_batch(self._h, ctypes.byref(b), ctypes.byref(r), flags)
        if rc == TSU_EOVERFLOW and cigar_capacity is None:
            need = int(r.cigar_needed)
            runs = np.zeros(max(need, 1), dtype=np.uint32)
            r = Result(_ptr(scores), _ptr(runs), need, _ptr(coff), 0, _ptr(st))
            rc = L.tsu_align_batch(self._h, ctypes.byref(b), ctypes.byref(r), flags)
        self._check(rc)
        runs = runs[: int(coff[-1])]
        return (scores, coff, runs, st) if status else (scores, coff, runs)

    def align(self, patterns: Sequence, texts: Sequence, cigar: bool = True):
        """Align lists of str/bytes.  Returns (scores, list of op strings or None)."""
        if len(patterns) != len(texts):
            raise ValueError("patterns and texts differ in length")
        pb, po, pl = _concat(patterns)
        tb, to, tl = _concat(texts)
        scores, coff, runs = self.align_arrays(pb, po, pl, tb, to, tl, cigar=cigar)
        if not cigar:
            return scores, None
        ops = [runs_to_ops(runs[coff[i]:coff[i + 1]]) for i in range(len(pl))]
        return scores, ops

    def align_fixed(self, pattern: bytes, text: bytes, num: int, plen: int, tlen: int) -> np.ndarray:
        """Reference host layout (wfa_gpu.cu:75-81): fixed stride, scores only."""
        scores = np.zeros(num, dtype=np.int32)
        pa = np.frombuffer(pattern, dtype=np.uint8)
        ta = np.frombuffer(text, dtype=np.uint8)
        self._check(lib().tsu_align_fixed(self._h, _ptr(pa), _ptr(ta), num, plen, tlen, _ptr(scores), 0))
        return scores

    # -- device buffers (torch CUDA tensors) --------------------------------
    def align_device(self, pat, poff, plen, txt, toff, tlen, scores, cigar_runs=None, cigar_off=None,
                     pair_status=None, one_warp: bool = False, bidirectional: bool = False) -> int:
        """All arguments are CUDA tensors (uint8 / int64 / int32).  Returns the
        number of CIGAR runs written (0 with cigar_runs=None).
        ``bidirectional=True``: TSU_BIDIRECTIONAL."""
        n = int(plen.numel())
        b = Batch(n, pat.data_ptr(), poff.data_ptr(), plen.data_ptr(), txt.data_ptr(), toff.data_ptr(),
                  tlen.data_ptr())
        flags = ((0 if cigar_runs is not None else TSU_SCORE_ONLY) | (TSU_ONE_WARP if one_warp else 0) |
                 (TSU_BIDIRECTIONAL if bidirectional else 0))
        r = Result(scores.data_ptr(), cigar_runs.data_ptr() if cigar_runs is not None else None,
                   int(cigar_runs.numel()) if cigar_runs is not None else 0,
                   cigar_off.data_ptr() if cigar_off is not None else None, 0,
                   pair_status.data_ptr() if pair_status is not None else None)
        rc = lib().tsu_align_batch_device(self._h, ctypes.byref(b), ctypes.byref(r), flags)
        if rc == TSU_EOVERFLOW:
            raise AlignError(rc, f"cigar buffer too small: need {r.cigar_needed} runs", int(r.cigar_needed))
        self._check(rc)
        return int(r.cigar_needed)


class Server:
    """Request server (tsu_server_*): continuous batching of alignment
    requests on one device with memory admission.  ``submit`` returns a
    request id at once; ``wait``/``poll`` return its results."""

    def __init__(self, mismatch: int = 4, gap_opening: int = 6, gap_extension: int = 2, device: int = 0,
                 workers: int = 0, mem_budget: int = 0, max_error_hint: float = 0.0, max_queue: int = 0,
                 max_job_pairs: int = 0, max_job_requests: int = 0, heavy_len: int = 0, heavy_workers: int = 0,
                 estimate_hint: bool = True, watchdog_ms: float = 0.0, resident_bytes: int = 0,
                 gap_opening2: Optional[int] = None, gap_extension2: Optional[int] = None,
                 metric: Optional[str] = None):
        L = lib()
        cfg = ServerConfig(device, workers, mem_budget, max_error_hint, max_queue, max_job_pairs,
                           max_job_requests, heavy_len, heavy_workers, 0 if estimate_hint else -1, watchdog_ms,
                           resident_bytes)
        h = c_vp()
        code, pens = metric_penalties(metric, mismatch, gap_opening, gap_extension, gap_opening2, gap_extension2)
        arr = (ctypes.c_int32 * max(1, len(pens)))(*pens)
        rc = L.tsu_server_create_metric(code, ctypes.cast(arr, c_vp) if pens else None, len(pens),
                                        ctypes.byref(cfg), ctypes.byref(h))
        if rc != TSU_OK:
            raise AlignError(rc, L.tsu_status_str(rc).decode())
        self._h = h
        self._cigar = {}  # id -> (wants CIGAR, pairs, run capacity)

    def close(self):
        if getattr(self, "_h", None):
            lib().tsu_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _err(self, rc: int) -> AlignError:
        L = lib()
        return AlignError(rc, f"{L.tsu_status_str(rc).decode()}: {L.tsu_server_last_error(self._h).decode()}")

    def submit_arrays(self, pbuf, poff, plen, tbuf, toff, tlen, cigar: bool = True,
                      bidirectional: bool = False) -> int:
        """Submit one request (tsu_submit); ``bidirectional=True``:
        TSU_BIDIRECTIONAL (gap-affine and gap-linear servers)."""
        n = len(plen)
        poff = np.ascontiguousarray(poff, dtype=np.int64)
        toff = np.ascontiguousarray(toff, dtype=np.int64)
        plen = np.ascontiguousarray(plen, dtype=np.int32)
        tlen = np.ascontiguousarray(tlen, dtype=np.int32)
        b = Batch(n, _ptr(pbuf), _ptr(poff), _ptr(plen), _ptr(tbuf), _ptr(toff), _ptr(tlen))
        rid = ctypes.c_uint64()
        flags = (0 if cigar else TSU_SCORE_ONLY) | (TSU_BIDIRECTIONAL if bidirectional else 0)
        rc = lib().tsu_submit(self._h, ctypes.byref(b), flags, ctypes.byref(rid))
        if rc != TSU_OK:
            raise self._err(rc)
        cap = int(plen.astype(np.int64).sum() + tlen.astype(np.int64).sum()) + 1
        self._cigar[rid.value] = (cigar, n, cap)
        return rid.value

    def submit(self, patterns: Sequence, texts: Sequence, cigar: bool = True, bidirectional: bool = False) -> int:
        if len(patterns) != len(texts):
            raise ValueError("patterns and texts differ in length")
        pb, po, pl = _concat(patterns)
        tb, to, tl = _concat(texts)
        return self.submit_arrays(pb, po, pl, tb, to, tl, cigar=cigar, bidirectional=bidirectional)

    def _take(self, rid: int, timeout_ms: Optional[float]):
        cig, n, cap = self._cigar[rid]
        scores = np.zeros(max(n, 1), dtype=np.int32)
        st = np.zeros(max(n, 1), dtype=np.int32)
        coff = np.zeros(n + 1, dtype=np.int64) if cig else None
        runs = np.zeros(cap, dtype=np.uint32) if cig else None
        r = Result(_ptr(scores), _ptr(runs), cap if cig else 0, _ptr(coff), 0, _ptr(st))
        info = RequestInfo()
        L = lib()
        if timeout_ms is None:
            rc = L.tsu_poll(self._h, rid, ctypes.byref(r), ctypes.byref(info))
        else:
            rc = L.tsu_wait(self._h, rid, timeout_ms, ctypes.byref(r), ctypes.byref(info))
        if rc in (TSU_EPENDING, TSU_ETIMEOUT):
            return None
        self._cigar.pop(rid, None)
        if rc != TSU_OK:
            raise self._err(rc)
        inf = {f: getattr(info, f) for f, _ in RequestInfo._fields_}
        if not cig:
            return scores[:n], None, None, inf
        return scores[:n], coff, runs[: int(coff[-1])], inf

    def poll(self, rid: int):
        """(scores, cigar_offsets, runs, info) if done, else None."""
        return self._take(rid, None)

    def wait(self, rid: int, timeout_ms: float = -1.0):
        """Block until done (timeout_ms < 0: no limit); None on timeout."""
        return self._take(rid, timeout_ms)

    def cancel(self, rid: int) -> int:
        self._cigar.pop(rid, None)
        return lib().tsu_cancel(self._h, rid)

    def stats(self) -> dict:
        s = ServerStats()
        lib().tsu_server_get_stats(self._h, ctypes.byref(s))
        return {f: getattr(s, f) for f, _ in ServerStats._fields_}

    def reset_stats(self) -> None:
        lib().tsu_server_reset_stats(self._h)


def read_sequences(path: str):
    """Parse sequences.txt (wfa_gpu.cu:71-81).  Returns (header, patterns, texts)
    with header = (num, seq_len, error_rate) and sequences as bytes."""
    L = lib()
    h = c_vp()
    rc = L.tsu_file_read(path.encode(), ctypes.byref(h))
    if rc != TSU_OK:
        raise AlignError(rc, f"cannot read {path}")
    return _file_contents(L, h)


def read_pairs(pattern_path: str, text_path: str):
    """Pairs from two FASTA/FASTQ files (record i of each file is pair i).
    Returns (header, patterns, texts) like read_sequences."""
    L = lib()
    h = c_vp()
    rc = L.tsu_file_read_pairs(pattern_path.encode(), text_path.encode(), ctypes.byref(h))
    if rc != TSU_OK:
        raise AlignError(rc, f"cannot read {pattern_path} / {text_path}")
    return _file_contents(L, h)


def _file_contents(L, h):
    try:
        b = Batch()
        L.tsu_file_batch(h, ctypes.byref(b))
        num, sl, er = c_i64(), c_i32(), c_i32()
        L.tsu_file_header(h, ctypes.byref(num), ctypes.byref(sl), ctypes.byref(er))
        n = b.num_pairs
        po = np.ctypeslib.as_array(ctypes.cast(b.pattern_off, P(c_i64)), (n,)) if n else np.zeros(0, np.int64)
        pl = np.ctypeslib.as_array(ctypes.cast(b.pattern_len, P(c_i32)), (n,)) if n else np.zeros(0, np.int32)
        to = np.ctypeslib.as_array(ctypes.cast(b.text_off, P(c_i64)), (n,)) if n else np.zeros(0, np.int64)
        tl = np.ctypeslib.as_array(ctypes.cast(b.text_len, P(c_i32)), (n,)) if n else np.zeros(0, np.int32)
        pats = [ctypes.string_at(b.pattern + int(po[i]), int(pl[i])) for i in range(n)]
        txts = [ctypes.string_at(b.text + int(to[i]), int(tl[i])) for i in range(n)]
        return (num.value, sl.value, er.value), pats, txts
    finally:
        L.tsu_file_free(h)


def write_sequences(path: str, patterns: Sequence, texts: Sequence, seq_len: int, error_rate: int) -> None:
    pb, po, pl = _concat(patterns)
    tb, to, tl = _concat(texts)
    b = Batch(len(pl), _ptr(pb), _ptr(po), _ptr(pl), _ptr(tb), _ptr(to), _ptr(tl))
    rc = lib().tsu_file_write(path.encode(), len(pl), seq_len, error_rate, ctypes.byref(b))
    if rc != TSU_OK:
        raise AlignError(rc, f"cannot write {path}")


def gen_batch(seed: int, lengths: np.ndarray, rates: np.ndarray, first: int = 0, threads: int = 0):
    """Seeded synthetic pairs (tsu_gen_batch).  Returns concatenated buffers
    (pbuf, poff, plen, tbuf, toff, tlen); text i has the length of pattern i."""
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
    rc = lib().tsu_gen_batch(seed, first, n, _ptr(lengths), _ptr(rates), _ptr(pbuf), _ptr(off), _ptr(plen),
                             _ptr(tbuf), _ptr(off), _ptr(tlen), threads)
    if rc != TSU_OK:
        raise AlignError(rc, "tsu_gen_batch failed")
    return pbuf, off, plen, tbuf, off.copy(), tlen
