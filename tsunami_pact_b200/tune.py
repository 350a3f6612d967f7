"""Autotuner of the pass plan: the starting rung of each length band.

For each length band (max(m, n) < 1 k, 2 k, 4 k, 8 k, 16 k, >= 16 k) it aligns
a seeded workload of that band -- lengths log-uniform over the band, edit
rates uniform 1-15 %, penalties 4/6/2, the uneven batched configuration --
from every candidate rung (wavefront ring in shared memory with 1, 2, 4, 8 or
16 warps per pair, or in device memory with 8 or 16), checks that every rung
gives the same scores and CIGARs, and keeps the rung with the shortest device
time of the align passes (the minimum over --reps runs after one warm-up).

It writes the table as a C header (tsunami_pact_b200/csrc/tsu_tuning.h by
default; rebuild the library afterwards) and every measurement as JSON.

usage: python -m tsunami_pact_b200.tune [--out-header PATH] [--out-json PATH]
                                         [--reps N] [--scale F] [--device D]
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
# (shortest, longest + 1, pairs) per band
BANDS = [(100, 1024, 40000), (1024, 2048, 16000), (2048, 4096, 6000), (4096, 8192, 2400), (8192, 16384, 800),
         (16384, 32001, 300)]
CANDIDATES = [(0, 1), (0, 2), (0, 4), (0, 8), (0, 16), (1, 8), (1, 16)]
SEED = 0x54554E45


def rung_name(r) -> str:
    return ("s" if r[0] == 0 else "g") + str(r[1])


def band_workload(band: int, scale: float = 1.0):
    """Seeded pairs of one band: (pbuf, poff, plen, tbuf, toff, tlen)."""
    from . import gen_batch

    lo, hi, n = BANDS[band]
    n = max(16, int(n * scale))
    rng = np.random.Generator(np.random.PCG64(SEED + band))
    lengths = np.exp(rng.uniform(np.log(lo), np.log(hi - 1), n)).astype(np.int32)
    rates = rng.uniform(0.01, 0.15, n)
    return gen_batch(SEED + band, lengths, rates)


def render_header(table, source: str, times=None) -> str:
    """tsu_tuning.h for a table [(mode, warps)] * 6; times[band][rung] in ms
    become a comment."""
    lines = [
        "// tsu_tuning.h -- starting rung of the pass ladder per length band.",
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
        '#define TSU_TUNING_SOURCE "%s"' % source,
        "#define TSU_BAND_START {" + ", ".join("{%d, %d}" % (m, w) for m, w in table) + "}",
        "",
    ]
    return "\n".join(lines)


def parse_header(text: str):
    """The table of a tsu_tuning.h: [(mode, warps)] * 6."""
    import re

    m = re.search(r"#define TSU_BAND_START \{(.*)\}", text)
    if not m:
        raise ValueError("no TSU_BAND_START")
    pairs = re.findall(r"\{\s*(\d+)\s*,\s*(\d+)\s*\}", m.group(1))
    return [(int(a), int(b)) for a, b in pairs]


def gpu_name(device: int) -> str:
    try:
        out = subprocess.run(["nvidia-smi", f"--id={device}", "--query-gpu=name", "--format=csv,noheader"],
                             capture_output=True, text=True, timeout=30).stdout.strip()
        return out or "unknown GPU"
    except (OSError, subprocess.TimeoutExpired):
        return "unknown GPU"


def tune(reps: int = 2, scale: float = 1.0, device: int = 0, log=print):
    import ctypes

    from . import Aligner, lib

    L = lib()
    L.tsu_set_band_start.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    table, times, record = [], [], []
    with Aligner(4, 6, 2, device=device) as al:
        for band in range(len(BANDS)):
            data = band_workload(band, scale)
            cap = int(data[2].astype(np.int64).sum() + data[5].astype(np.int64).sum()) + 1
            row, ref, best = {}, None, None
            for r in CANDIDATES:
                if r[0] == 0 and BANDS[band][1] - 1 > 32000:
                    continue
                rc = L.tsu_set_band_start(al._h, band, r[0], r[1])
                if rc != 0:
                    raise RuntimeError(f"tsu_set_band_start({band}, {r}) = {rc}")
                ms = []
                for k in range(reps + 1):
                    s, co, runs = al.align_arrays(*data, cigar_capacity=cap)
                    t = al.timing()
                    if k:
                        ms.append(t["align_ms"])
                got = (s.copy(), co.copy(), runs.copy())
                if ref is None:
                    ref = got
                elif not all(np.array_equal(a, b) for a, b in zip(ref, got)):
                    raise RuntimeError(f"band {band}: rung {rung_name(r)} changed the results")
                row[rung_name(r)] = min(ms)
                record.append({"band": band, "rung": rung_name(r), "align_ms": ms, "pairs": int(len(data[2])),
                               "passes": al.pass_log()})
                log("band %d %-6s %8.2f ms  %s" % (band, rung_name(r), min(ms), al.pass_log()))
                if best is None or min(ms) < row[rung_name(best)]:
                    best = r
            table.append(best)
            times.append(row)
            L.tsu_set_band_start(al._h, band, best[0], best[1])
    return table, times, record


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out-header", default=os.path.join(HERE, "csrc", "tsu_tuning.h"))
    ap.add_argument("--out-json", default="")
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--scale", type=float, default=1.0, help="pairs per band x this")
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)
    table, times, record = tune(args.reps, args.scale, args.device)
    stamp = datetime.datetime.now(datetime.timezone.utc).strftime("%Y-%m-%d")
    source = "tune.py on %s, %s" % (gpu_name(args.device), stamp)
    with open(args.out_header, "w") as f:
        f.write(render_header(table, source, times))
    if args.out_json:
        with open(args.out_json, "w") as f:
            json.dump({"source": source, "table": table, "times_ms": times, "runs": record,
                       "bands": [{"lengths": [lo, hi - 1], "pairs": n, "rates": [0.01, 0.15]} for lo, hi, n in BANDS]},
                      f, indent=1)
    print("table:", " ".join(rung_name(r) for r in table), file=sys.stderr)


if __name__ == "__main__":
    main()
