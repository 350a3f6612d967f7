"""Autotuner of the pass plan: the starting rung of each length band.

The batch engine splits a batch into length bands (max(m, n) < 1 k, 2 k,
4 k, 8 k, 16 k, >= 16 k) and starts each band at the rung of a table.  The
tuner takes the pairs of each band out of the workloads it is given (by
default the uniform 1 kbp configuration, c2: 1 kbp at 5 %, the uneven
batched one, c4: lengths log-uniform 100-20,000, edit rates 1-15 %, and the
long-read one, c3: 10 kbp at 15 %; seeded, see datasets.py; penalties
4/6/2), aligns them from every candidate rung
(wavefront ring in shared memory with 1, 2, 4, 8, 16 or 32 warps per pair,
or in device memory with 8, 16 or 32), checks that every rung gives the same scores and
CIGARs, and keeps the rung with the shortest device time of the align passes
summed over the workloads (each the minimum over --reps runs after one
warm-up).  Bands are measured at the sizes they have in the workloads,
because a rung's cost includes the retry passes of the pairs that outgrow
it, whose weight depends on how many pairs share the band.

It writes the table as a C header (tsunami_pact_b200/csrc/tsu_tuning.h by
default; rebuild the library afterwards) and every measurement as JSON.
With five --penalties (mismatch, open, extend, open2, extend2) it tunes the
dual gap-affine kernels instead and writes their table, TSU_BAND_START_DUAL,
to tsu_tuning_dual.h: their wavefront ring is deeper (M back to s - o2 - e2)
and, with a small e2, wider, so they start at other rungs.

usage: python -m tsunami_pact_b200.tune [--out-header PATH] [--out-json PATH]
                                         [--workloads c2:200000,c4:100000,c3:5000]
                                         [--reps N] [--device D] [--penalties 4,6,2]
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BAND_NAMES = ["< 1024", "< 2048", "< 4096", "< 8192", "< 16384", ">= 16384"]
BAND_LIMITS = [1024, 2048, 4096, 8192, 16384]  # tsu::length_band
N_BANDS = 6
CANDIDATES = [(0, 1), (0, 2), (0, 4), (0, 8), (0, 16), (0, 32), (1, 8), (1, 16), (1, 32)]
SHARED_MAX_LEN = 32000  # the int16 shared ring's limit
DEFAULT_WORKLOADS = "c2:200000,c4:100000,c3:5000"


def rung_name(r) -> str:
    return ("s" if r[0] == 0 else "g") + str(r[1])


def length_band(L: np.ndarray) -> np.ndarray:
    """The engine's length band of max(m, n) (tsu::length_band)."""
    return np.searchsorted(np.asarray(BAND_LIMITS), L, side="right")


def band_batches(workloads: str):
    """{band: [(workload, batch)]}: each workload's pairs split by band, as
    (pbuf, poff, plen, tbuf, toff, tlen) views into the workload's buffers."""
    from . import datasets

    out = {b: [] for b in range(N_BANDS)}
    for item in workloads.split(","):
        name, _, n = item.partition(":")
        pbuf, poff, plen, tbuf, toff, tlen = datasets.generate(name, int(n) if n else 0)
        bands = length_band(np.maximum(plen, tlen))
        for b in range(N_BANDS):
            sel = np.nonzero(bands == b)[0]
            if sel.size:
                out[b].append((name, (pbuf, poff[sel].copy(), plen[sel].copy(), tbuf, toff[sel].copy(),
                                      tlen[sel].copy())))
    return out


def header_macro(dual: bool) -> str:
    return "TSU_BAND_START_DUAL" if dual else "TSU_BAND_START"


def render_header(table, source: str, times=None, dual: bool = False) -> str:
    """tsu_tuning.h (tsu_tuning_dual.h) for a table [(mode, warps)] * 6;
    times[band][rung] in ms become a comment."""
    lines = [
        "// %s -- starting rung of the pass ladder per length band%s." % (
            "tsu_tuning_dual.h" if dual else "tsu_tuning.h", " (dual gap-affine kernels)" if dual else ""),
        "// Written by tsunami_pact_b200/tune.py (the autotuner); rebuild the library after changing it.",
        "// band: max(m, n) < 1024, < 2048, < 4096, < 8192, < 16384, >= 16384",
        "// rung: {ring mode (0 shared, 1 global), warps per pair}",
    ]
    if times:
        lines.append("// align time in ms per starting rung (" + " ".join(rung_name(r) for r in CANDIDATES) + "):")
        for b, row in enumerate(times):
            cells = " ".join("%.1f" % row[rung_name(r)] if rung_name(r) in row else "-" for r in CANDIDATES)
            lines.append("//   band %d (%s): %s" % (b, BAND_NAMES[b], cells))
    lines += [
        "#pragma once",
        '#define %s "%s"' % ("TSU_TUNING_DUAL_SOURCE" if dual else "TSU_TUNING_SOURCE", source),
        "#define %s {" % header_macro(dual) + ", ".join("{%d, %d}" % (m, w) for m, w in table) + "}",
        "",
    ]
    return "\n".join(lines)


def parse_header(text: str, dual: bool = False):
    """The table of a tsu_tuning.h (tsu_tuning_dual.h): [(mode, warps)] * 6."""
    import re

    m = re.search(r"#define %s \{(.*)\}" % header_macro(dual), text)
    if not m:
        raise ValueError("no " + header_macro(dual))
    pairs = re.findall(r"\{\s*(\d+)\s*,\s*(\d+)\s*\}", m.group(1))
    return [(int(a), int(b)) for a, b in pairs]


def gpu_name(device: int) -> str:
    try:
        out = subprocess.run(["nvidia-smi", f"--id={device}", "--query-gpu=name", "--format=csv,noheader"],
                             capture_output=True, text=True, timeout=30).stdout.strip()
        return out or "unknown GPU"
    except (OSError, subprocess.TimeoutExpired):
        return "unknown GPU"


def tune(workloads: str = DEFAULT_WORKLOADS, reps: int = 2, device: int = 0, log=print, penalties=(4, 6, 2)):
    """Returns (table, times per band {rung: ms}, one record per measurement)."""
    import ctypes

    from . import Aligner, lib

    L = lib()
    L.tsu_set_band_start.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.tsu_get_band_start.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_int)]
    per_band = band_batches(workloads)
    table, times, record = [], [], []
    dual_kw = {"gap_opening2": penalties[3], "gap_extension2": penalties[4]} if len(penalties) == 5 else {}
    with Aligner(*penalties[:3], device=device, **dual_kw) as al:
        for band in range(N_BANDS):
            if not per_band[band]:  # no pairs of this band: keep the compiled rung
                m, w = ctypes.c_int(), ctypes.c_int()
                L.tsu_get_band_start(al._h, band, ctypes.byref(m), ctypes.byref(w))
                table.append((m.value, w.value))
                times.append({})
                continue
            longest = max(int(np.maximum(d[2], d[5]).max()) for _, d in per_band[band])
            row, refs, best = {}, {}, None
            for r in CANDIDATES:
                if r[0] == 0 and longest > SHARED_MAX_LEN:
                    continue
                rc = L.tsu_set_band_start(al._h, band, r[0], r[1])
                if rc != 0:
                    raise RuntimeError(f"tsu_set_band_start({band}, {r}) = {rc}")
                total = 0.0
                for name, data in per_band[band]:
                    cap = int(data[2].astype(np.int64).sum() + data[5].astype(np.int64).sum()) + 1
                    ms = []
                    for k in range(reps + 1):
                        s, co, runs = al.align_arrays(*data, cigar_capacity=cap)
                        if k:
                            ms.append(al.timing()["align_ms"])
                    got = (s.copy(), co.copy(), runs.copy())
                    if name not in refs:
                        refs[name] = got
                    elif not all(np.array_equal(a, b) for a, b in zip(refs[name], got)):
                        raise RuntimeError(f"band {band}: rung {rung_name(r)} changed the results of {name}")
                    total += min(ms)
                    record.append({"band": band, "workload": name, "pairs": int(len(data[2])), "rung": rung_name(r),
                                   "align_ms": ms, "passes": al.pass_log()})
                    log("band %d %-3s %-6s %6d pairs %9.2f ms  %s" % (band, name, rung_name(r), len(data[2]), min(ms),
                                                                   al.pass_log()))
                row[rung_name(r)] = total
            # the fastest rung; of rungs within 1.5 % of it, the last (widest)
            # one, whose first pass does the work the narrower ones hand on
            fastest = min(row.values())
            best = [r for r in CANDIDATES if rung_name(r) in row and row[rung_name(r)] <= 1.015 * fastest][-1]
            table.append(best)
            times.append(row)
            L.tsu_set_band_start(al._h, band, best[0], best[1])
    return table, times, record


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out-header", default="", help="default: csrc/tsu_tuning.h (csrc/tsu_tuning_dual.h)")
    ap.add_argument("--out-json", default="")
    ap.add_argument("--workloads", default=DEFAULT_WORKLOADS, help="name:pairs,... (tsunami_pact_b200/datasets.py)")
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--penalties", default="4,6,2", help="mismatch,open,extend[,open2,extend2]")
    args = ap.parse_args(argv)
    pen = tuple(int(v) for v in args.penalties.split(","))
    if len(pen) not in (3, 5):
        raise SystemExit("--penalties takes 3 or 5 values")
    dual = len(pen) == 5
    out_header = args.out_header or os.path.join(HERE, "csrc", "tsu_tuning_dual.h" if dual else "tsu_tuning.h")
    table, times, record = tune(args.workloads, args.reps, args.device, penalties=pen)
    stamp = datetime.datetime.now(datetime.timezone.utc).strftime("%Y-%m-%d")
    source = "tune.py on %s, %s, workloads %s, penalties %s" % (gpu_name(args.device), stamp, args.workloads,
                                                               "/".join(map(str, pen)))
    with open(out_header, "w") as f:
        f.write(render_header(table, source, times, dual))
    if args.out_json:
        with open(args.out_json, "w") as f:
            json.dump({"source": source, "workloads": args.workloads, "table": table, "times_ms": times,
                       "runs": record}, f, indent=1)
    print("table:", " ".join(rung_name(r) for r in table), file=sys.stderr)


if __name__ == "__main__":
    main()
