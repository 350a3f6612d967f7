#!/usr/bin/env python
"""Benchmark of the B200 gap-affine WFA engine (one JSON line on rank 0).

A step is one pass of the path over one batch: pack -> align (scores and
WFA2-style CIGARs) -> CIGAR compaction, for the whole batch.

  value  GCUPS (reference formula sum(m*n)/t/1e9, wfa_gpu.cu:130-133) with the
         batch resident in HBM, time from CUDA events on the engine's stream
  e2e    the same through tsu_align_batch with pinned HOST buffers: H2D of
         the sequences, the device work and D2H of scores + CIGARs per step

Default workload (c4): 200,000 pairs of uneven length (log-uniform
100-20,000 bp) and edit rate (uniform 1-15 % per pair, equal
sub/ins/del), penalties 4/6/2, seeded synthetic data, aligned by the batched
form (length bands, persistent launches over a device work queue, one CUDA
graph per call) and, beside it, by the plain form (one launch per
floor(log2 L) bucket, one warp per pair).  A full c2 record (1,000,000 x
1 kbp at 5 %, the plain one-launch shape) is nested under "secondary".
`--impl reference` times the CPU path (the oracle's WFA, the stand-in for
the reference's WFA2-lib check, wfa_gpu.cu:150-166) on all host cores over
a bounded sample of the same workload, with pairs from the oracle's copy of
the generator.  Under torchrun each rank aligns its own batch (weak
scaling, no collective on the data path); the step time is the max over
ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SEED = 0x5453554E414D49
METRIC = "GCUPS & pairs/s on 1 B200 vs plain launch; serving p50/p99 latency; bit-exact"
WORKLOADS = {
    # name: [pairs per GPU, description]  (shapes: tsunami_pact_b200/datasets.py)
    "c1": [10_000, "150 bp, 2% edits"],
    "c2": [1_000_000, "1,000 bp, 5% edits"],
    "c3": [20_000, "10,000 bp, 15% edits"],
    "c4": [200_000, "lengths log-uniform 100-20,000 bp, edits uniform 1-15% per pair"],
}
PEN = (4, 6, 2)  # --penalties; five values (open2, extend2 last): dual gap-affine
METRIC_NAME = None  # --metric edit | indel | gap_linear (PEN then (mismatch, gap_extension))
ENDS_FREE = (0, 0, 0, 0)  # --ends-free pattern_begin,pattern_end,text_begin,text_end (gap-affine)
LOW_MEM = 0  # --low-memory checkpoint interval (0 off, < 0 chosen per pass)
BIDIR = False  # --bidirectional: TSU_BIDIRECTIONAL (breakpoint search; CIGARs by its recursion)
LINEAR_XE = {"edit": (1, 1), "indel": (3, 1)}  # the gap-linear penalties of these metrics


def linear_xe():
    return LINEAR_XE.get(METRIC_NAME, PEN[:2])


def pen_str() -> str:
    ef = ", free ends %d/%d/%d/%d" % ENDS_FREE if any(ENDS_FREE) else ""
    if LOW_MEM:
        ef += ", low-memory (checkpoint interval %s)" % ("auto" if LOW_MEM < 0 else LOW_MEM)
    if BIDIR:
        ef += ", bidirectional"
    if METRIC_NAME in LINEAR_XE:
        return METRIC_NAME + " distance" + ef
    if METRIC_NAME == "gap_linear":
        return "gap-linear %d/%d" % PEN[:2] + ef
    return "/".join(str(v) for v in PEN) + (" (dual gap-affine)" if len(PEN) == 5 else "") + ef


def make_aligner(T, **kw):
    """An engine context over the bench's penalties or metric (and free ends)."""
    if METRIC_NAME in LINEAR_XE:
        al = T.Aligner(metric=METRIC_NAME, **kw)
    elif METRIC_NAME == "gap_linear":
        al = T.Aligner(PEN[0], 0, PEN[1], metric="gap_linear", **kw)
    else:
        dual_kw = {"gap_opening2": PEN[3], "gap_extension2": PEN[4]} if len(PEN) == 5 else {}
        al = T.Aligner(*PEN[:3], **dual_kw, **kw)
    if any(ENDS_FREE):
        al.set_ends_free(*ENDS_FREE)
    if LOW_MEM:
        al.set_low_memory(LOW_MEM)
    return al


def oracle_batch(O, pbuf, poff, plen, tbuf, toff, tlen, threads):
    """The oracle over the bench's penalties (one or two gap pieces, or a
    gap-linear metric; free ends when set)."""
    if any(ENDS_FREE):
        if METRIC_NAME is None and len(PEN) == 3:
            return O.align_batch_ends_free_arrays(pbuf, poff, plen, tbuf, toff, tlen, ENDS_FREE, *PEN, cigar=True,
                                                  threads=threads)
        pats = [bytes(pbuf[poff[i]:poff[i] + plen[i]]) for i in range(len(plen))]
        txts = [bytes(tbuf[toff[i]:toff[i] + tlen[i]]) for i in range(len(tlen))]
        if METRIC_NAME is not None:
            return O.align_batch_linear_ends_free(pats, txts, ENDS_FREE, *linear_xe(), threads=threads)
        return O.align_batch2_ends_free(pats, txts, ENDS_FREE, *PEN, threads=threads)
    if METRIC_NAME is not None:
        return O.align_batch_linear_arrays(pbuf, poff, plen, tbuf, toff, tlen, *linear_xe(), cigar=True,
                                           threads=threads)
    if len(PEN) == 5:
        return O.align_batch2_arrays(pbuf, poff, plen, tbuf, toff, tlen, *PEN, cigar=True, threads=threads)
    return O.align_batch_arrays(pbuf, poff, plen, tbuf, toff, tlen, *PEN, cigar=True, threads=threads)


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def make_batch(workload: str, rank: int, world: int):
    from tsunami_pact_b200 import datasets
    from tsunami_pact_b200.shard import shard

    first, n = shard(rank, world, WORKLOADS[workload][0])  # this rank's own pairs
    return datasets.generate(workload, n, first=first)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def load_traffic(kernel_key: str):
    """ncu figures of the dominant kernel from the committed summary
    (profiles/traffic.json): DRAM bytes of one captured launch and the pairs
    it processed (traffic grows in proportion to pairs), issue and ALU pipe
    utilisation; or None."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            return json.load(f).get(kernel_key)
    except (OSError, ValueError):
        return None


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, ValueError, KeyError):
        return 6650.0, "fallback"


def cpu_baseline(pbuf, poff, plen, tbuf, toff, tlen, target_s=15.0):
    from oracle import oracle as O

    cores = os.cpu_count() or 1
    n = len(plen)
    probe = min(n, max(256, cores * 64))
    t0 = time.perf_counter()
    oracle_batch(O, pbuf, poff[:probe], plen[:probe], tbuf, toff[:probe], tlen[:probe], cores)
    dt = time.perf_counter() - t0
    rate = probe / max(dt, 1e-6)
    sample = int(min(n, max(probe, rate * target_s)))
    t0 = time.perf_counter()
    oracle_batch(O, pbuf, poff[:sample], plen[:sample], tbuf, toff[:sample], tlen[:sample], cores)
    dt = time.perf_counter() - t0
    cells = float(np.sum(plen[:sample].astype(np.float64) * tlen[:sample]))
    return {"value": cells / dt / 1e9, "unit": "GCUPS", "cores": cores, "kind": "port",
            "pairs_per_s": sample / dt,
            "sample": f"first {sample} pairs of the workload, scores + CIGARs, {cores} threads, {dt:.1f} s"}


def run_serving(args):
    """c5: the request server under Poisson arrivals.  For each offered rate,
    `--requests` requests of uniform 1..256 pairs from the serving mixture
    (70 % 150 bp @ 1-3 %, 25 % 1-5 kbp @ 5-10 %, 5 % 10-50 kbp @ 10-20 %) are
    submitted from host buffers at their arrival times by one
    client thread while another waits for the results; one JSON line per
    rate: pairs/s completed, GCUPS, latency percentiles (submit -> result
    visible, measured by the server), requests merged per job."""
    import queue

    import tsunami_pact_b200 as T
    from tsunami_pact_b200 import datasets as D

    rates = [float(x) for x in args.rates.split(",") if x]
    budget = int(args.budget_gb * (1 << 30))
    if METRIC_NAME:
        pen_args, pen_kw = ((PEN[0], 0, PEN[1]) if METRIC_NAME == "gap_linear" else ()), {"metric": METRIC_NAME}
    else:
        pen_args = PEN[:3]
        pen_kw = {"gap_opening2": PEN[3], "gap_extension2": PEN[4]} if len(PEN) == 5 else {}
    srv = T.Server(*pen_args, workers=args.workers, mem_budget=budget, max_error_hint=args.hint or 0.2,
                   estimate_hint=not args.no_estimate, **pen_kw)

    def stream(index, n_req, rate):
        arrivals, sizes = D.c5_stream(n_req, rate if rate > 0 else 1.0, index=index)
        if rate <= 0:  # all at once: the server's capacity
            arrivals = np.zeros_like(arrivals)
        lengths, rates_, seed = D.shape("c5", int(sizes.sum()) + 1000 * index)
        first = 1000 * index
        lengths, rates_ = lengths[first:], rates_[first:]
        pbuf, poff, plen, tbuf, toff, tlen = T.gen_batch(seed, lengths, rates_, first=first)
        reqs, k = [], 0
        for sz in sizes:
            sl = slice(k, k + int(sz))
            reqs.append((pbuf, poff[sl].copy(), plen[sl].copy(), tbuf, toff[sl].copy(), tlen[sl].copy()))
            k += int(sz)
        cells = float(np.sum(plen.astype(np.float64) * tlen))
        return arrivals, sizes, reqs, cells

    # warm-up: a few requests through every worker
    _, _, wreqs, _ = stream(99, 4 * max(args.workers, 1), 1000.0)
    for rid in [srv.submit_arrays(*r) for r in wreqs]:
        srv.wait(rid)
    for k, rate in enumerate(rates):
        arrivals, sizes, reqs, cells = stream(k, args.requests, rate)
        srv.reset_stats()
        ids: "queue.Queue" = queue.Queue()
        errors = []

        def submitter():
            t0 = time.perf_counter()
            for a, r in zip(arrivals, reqs):
                dt = t0 + a - time.perf_counter()
                if dt > 0:
                    time.sleep(dt)
                try:
                    ids.put(srv.submit_arrays(*r))
                except T.AlignError as e:
                    errors.append(str(e))
                    ids.put(None)

        clocks = ClockSampler(0)
        clocks.start()
        t0 = time.perf_counter()
        th = threading.Thread(target=submitter)
        th.start()
        for _ in reqs:
            rid = ids.get()
            if rid is not None:
                srv.wait(rid)
        t1 = time.perf_counter()
        th.join()
        clk = clocks.stop()
        st = srv.stats()
        wall = t1 - t0
        out = {
            "metric": "pairs/s (serving)", "value": st["pairs_completed"] / wall, "unit": "pairs/s",
            "n_gpus": 1, "higher_is_better": True, "dtype": "int32", "data": "synthetic",
            "config": {"workload": "c5 serving: Poisson arrivals, requests of U{1..256} pairs, mixture 70% 150 bp "
                                   "@1-3%, 25% 1-5 kbp @5-10%, 5% 10-50 kbp @10-20%, penalties " + pen_str(),
                       "offered_rate_rps": rate, "requests": len(reqs), "pairs": int(sizes.sum()),
                       "workers": args.workers, "budget_gb": st["budget_bytes"] / 2**30,
                       "long_pair_memory": "max_error_hint" if args.no_estimate else "k-mer estimate"},
            "offered_pairs_s": float(sizes.sum()) / float(arrivals[-1]) if arrivals[-1] > 0 else None,
            "gcups": cells / wall / 1e9,
            "latency_ms": {"p50": st["p50_ms"], "p99": st["p99_ms"], "p999": st["p999_ms"], "mean": st["mean_ms"],
                           "max": st["max_ms"]},
            "completed": st["completed"], "failed": st["failed"], "rejected": st["rejected"] + len(errors),
            "jobs": st["jobs"], "mean_requests_per_job": st["mean_requests_per_job"],
            "peak_granted_gb": st["peak_granted_bytes"] / 2**30, "wall_s": wall, "clocks": clk,
            "heavy_jobs": st["heavy_jobs"], "mean_jobs_running": st["busy_s"] / wall,
            "mean_heavy_job_ms": 1e3 * st["heavy_busy_s"] / max(st["heavy_jobs"], 1),
            "mean_light_job_ms": 1e3 * (st["busy_s"] - st["heavy_busy_s"]) / max(st["jobs"] - st["heavy_jobs"], 1),
        }
        print(json.dumps(out), flush=True)
    srv.close()


def run_reference(args, workload):
    """CPU path on the host cores, rank 0 only (other ranks exit 0).  The
    pairs come from the oracle's copy of the seeded generator, so this arm
    never loads the engine library (checked at the end)."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle import oracle as O

    from tsunami_pact_b200.datasets import shape

    n_all, desc = WORKLOADS[workload]
    cores = os.cpu_count() or 1

    def generate(n):
        lengths, rates, seed = shape(workload, n)
        return O.gen_batch(seed, lengths, rates)

    # a bounded sample of the same workload: sized so each step is ~5-10 s
    probe = max(256, cores * 64)
    pb, po, pl, tb, to, tl = generate(probe)
    t0 = time.perf_counter()
    oracle_batch(O, pb, po, pl, tb, to, tl, cores)
    r = probe / max(time.perf_counter() - t0, 1e-6)
    sample = int(min(n_all, max(probe, r * 6.0)))
    pb, po, pl, tb, to, tl = generate(sample)
    cells = float(np.sum(pl.astype(np.float64) * tl))
    for _ in range(args.warmup):
        k = min(sample, probe)
        oracle_batch(O, pb, po[:k], pl[:k], tb, to[:k], tl[:k], cores)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle_batch(O, pb, po, pl, tb, to, tl, cores)
        times.append(time.perf_counter() - t0)
    t = float(np.mean(times))
    gcups = cells / t / 1e9
    try:
        with open("/proc/self/maps") as f:
            if "libtsunami_b200" in f.read():
                raise SystemExit("reference arm: the engine library was loaded")
    except OSError:
        pass
    out = {
        "metric": METRIC, "value": gcups, "unit": "GCUPS", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded, uniform ACGT, equal sub/ins/del edits)",
        "impl": "reference",
        "config": {"workload": f"{workload}: {n_all} pairs, {desc}, penalties {pen_str()}", "sample_pairs": sample},
        "pairs_per_s": sample / t,
        "cpu_baseline": {"value": gcups, "unit": "GCUPS", "cores": cores, "kind": "port",
                         "sample": f"first {sample} pairs of the workload per step, scores + CIGARs, "
                                   f"{cores} threads (WFA2-lib absent: the oracle's CPU WFA)"},
        "e2e": {"value": gcups, "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="tsunami", choices=["tsunami", "reference"])
    ap.add_argument("--workload", default="c4", choices=sorted(WORKLOADS) + ["c5"])
    ap.add_argument("--no-secondary", action="store_true", help="c4: skip the nested c2 record")
    ap.add_argument("--e2e-steps", type=int, default=0,
                    help="timed steps of the host-buffer leg (0: --steps; c4: at most 3)")
    ap.add_argument("--score-only", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--pairs", type=int, default=0, help="override the pair count (small profiling cases)")
    ap.add_argument("--hint", type=float, default=0.0, help="max_error_hint of the engine context")
    ap.add_argument("--plain", action="store_true", help="also time the plain one-warp-per-pair bucketed form")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain form (c4)")
    ap.add_argument("--plain-steps", type=int, default=1, help="timed repetitions of the plain form")
    ap.add_argument("--rates", default="5,10,20,0", help="c5: offered request rates (requests/s; 0: all at once)")
    ap.add_argument("--requests", type=int, default=200, help="c5: requests per rate")
    ap.add_argument("--workers", type=int, default=32, help="c5: server workers")
    ap.add_argument("--no-estimate", action="store_true", help="c5: size long pairs by --hint, not by estimate")
    ap.add_argument("--budget-gb", type=float, default=0.0,
                    help="device memory budget of the engine context (0: 80%% of free)")
    ap.add_argument("--penalties", default="4,6,2",
                    help="mismatch,open,extend[,open2,extend2]: five values align with dual gap-affine penalties")
    ap.add_argument("--metric", default=None, choices=["edit", "indel", "gap_linear"],
                    help="a gap-linear metric instead of gap-affine (gap_linear: --penalties mismatch,extend)")
    ap.add_argument("--ends-free", default="0,0,0,0",
                    help="pattern_begin,pattern_end,text_begin,text_end free lengths (gap-affine)")
    ap.add_argument("--low-memory", type=int, default=0,
                    help="checkpointed-history CIGARs: checkpoint interval (-1: chosen per pass)")
    ap.add_argument("--bidirectional", action="store_true",
                    help="bidirectional WFA (TSU_BIDIRECTIONAL): breakpoint search, CIGARs by its recursion")
    args = ap.parse_args()
    global PEN, METRIC_NAME, ENDS_FREE, LOW_MEM, BIDIR
    LOW_MEM = args.low_memory
    BIDIR = args.bidirectional
    ENDS_FREE = tuple(int(v) for v in args.ends_free.split(","))
    if len(ENDS_FREE) != 4:
        raise SystemExit("--ends-free takes 4 values")
    PEN = tuple(int(v) for v in args.penalties.split(","))
    METRIC_NAME = args.metric
    if METRIC_NAME == "gap_linear" and args.penalties == "4,6,2":
        PEN = (4, 2)
    if METRIC_NAME == "gap_linear" and len(PEN) != 2:
        raise SystemExit("--metric gap_linear takes --penalties mismatch,extend")
    if METRIC_NAME is None and len(PEN) not in (3, 5):
        raise SystemExit("--penalties takes 3 or 5 values")
    if args.workload == "c5":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "no serving path in the reference"}))
        else:
            run_serving(args)
        return
    if args.pairs:
        WORKLOADS[args.workload][0] = args.pairs
    workload = args.workload
    if args.impl == "reference":
        run_reference(args, workload)
        return
    if workload == "c4" and args.e2e_steps <= 0:
        args.e2e_steps = min(args.steps, 3)  # one c4 step is seconds long

    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    head = measure(args, workload, rank, world, local, dist,
                   with_plain=(workload == "c4" or args.plain) and not args.no_plain and not BIDIR,
                   with_cpu=world == 1 and not args.no_cpu_baseline, e2e_steps=args.e2e_steps)
    # the default run (c4) nests a full c2 record: the plain one-launch GPU
    # shape at scale (1,000,000 x 1 kbp), measured the same way
    if workload == "c4" and not args.no_secondary and not args.pairs:
        sec = measure(args, "c2", rank, world, local, dist, with_plain=False, with_cpu=False, e2e_steps=args.steps)
        if head is not None:
            head["secondary"] = {"c2": {k: sec[k] for k in ("value", "unit", "ms_per_step", "pairs_per_s", "steps",
                                                           "warmup", "gpu_launches", "e2e", "roofline", "clocks",
                                                           "config")}}
    if rank == 0 and head is not None:
        print(json.dumps(head), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def measure(args, workload, rank, world, local, dist, with_plain, with_cpu, e2e_steps):
    """One workload on this rank's GPU: the device-resident leg (value), the
    plain form (with_plain), the host-buffer leg (e2e) and the roofline of the
    align passes; the JSON record on rank 0 (None elsewhere)."""
    import torch

    import tsunami_pact_b200 as T
    from tsunami_pact_b200.shard import barrier as shard_barrier
    from tsunami_pact_b200.shard import combine, throughput

    def barrier():
        shard_barrier(dist, f"cuda:{local}")

    def max_over_ranks(x: float) -> float:
        return combine([x], ["max"], dist, f"cuda:{local}")[0]

    n_pairs, desc = WORKLOADS[workload]
    pbuf, poff, plen, tbuf, toff, tlen = make_batch(workload, rank, world)
    cells = float(np.sum(plen.astype(np.float64) * tlen))
    want_cigar = not args.score_only
    al = make_aligner(T, device=local, max_error_hint=args.hint, mem_budget=int(args.budget_gb * (1 << 30)))

    # ---- value: batch resident in HBM ----------------------------------
    dev = torch.device("cuda", local)
    d_p = torch.from_numpy(pbuf).to(dev)
    d_t = torch.from_numpy(tbuf).to(dev)
    d_po, d_pl, d_to, d_tl = (torch.from_numpy(x).to(dev) for x in (poff, plen, toff, tlen))
    d_sc = torch.zeros(n_pairs, dtype=torch.int32, device=dev)
    d_off = torch.zeros(n_pairs + 1, dtype=torch.int64, device=dev)
    cap = n_pairs * 64 + 1024
    d_runs = torch.zeros(cap, dtype=torch.int32, device=dev) if want_cigar else None

    def dev_step():
        nonlocal d_runs, cap
        try:
            return al.align_device(d_p, d_po, d_pl, d_t, d_to, d_tl, d_sc, d_runs, d_off if want_cigar else None,
                                   bidirectional=BIDIR)
        except T.AlignError as e:
            if e.code != 5:
                raise
            cap = int(e.needed) + 1024
            d_runs = torch.zeros(cap, dtype=torch.int32, device=dev)
            return al.align_device(d_p, d_po, d_pl, d_t, d_to, d_tl, d_sc, d_runs, d_off, bidirectional=BIDIR)

    for _ in range(max(args.warmup, 1)):
        nruns = dev_step()
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    step_ms, align_ms, launches, work_cells, work_steps, ext_bases = [], [], 0, 0, 0, 0
    t_wall = time.perf_counter()
    for _ in range(args.steps):
        nruns = dev_step()
        tm = al.timing()
        step_ms.append(tm["total_ms"])
        align_ms.append(tm["align_ms"])
        launches += int(tm["kernel_launches"])
        work_cells, work_steps, ext_bases = tm["cells"], tm["steps"], tm["ext_bases"]
        pass_log = al.pass_log()
    barrier()
    wall_ms = (time.perf_counter() - t_wall) * 1e3 / args.steps
    clk = clocks.stop()
    # slowest rank's step time; work summed over ranks
    ms, cells_all, pairs_all = combine([float(np.mean(step_ms)), cells, float(n_pairs)], ["max", "sum", "sum"], dist,
                                       f"cuda:{local}")
    value = throughput(cells_all, ms) / 1e9
    pairs_s = throughput(pairs_all, ms)

    # ---- plain form: one call per log2-length bucket, one warp per pair
    plain = None
    if with_plain:
        from tsunami_pact_b200 import datasets

        buckets = datasets.length_buckets(plen)
        ref_scores = d_sc.cpu().numpy()
        sub = []
        for b in np.unique(buckets):
            idx = np.nonzero(buckets == b)[0]
            sub.append((int(b), len(idx), [torch.from_numpy(x[idx]).to(dev) for x in (poff, plen, toff, tlen)]))
        p_ms, p_launch = [], 0
        # the first repetition warms up; each timed one is a whole uneven
        # batch in one-warp launches, so the plain form has its own
        # repetition count
        for rep in range(max(args.plain_steps, 1) + 1):
            tot = 0.0
            for b, nb, (bo, bl, to_, tl_) in sub:
                sc = torch.zeros(nb, dtype=torch.int32, device=dev)
                off = torch.zeros(nb + 1, dtype=torch.int64, device=dev)
                runs = torch.zeros(max(int(nb * 64), 1024), dtype=torch.int32, device=dev) if want_cigar else None
                try:
                    al.align_device(d_p, bo, bl, d_t, to_, tl_, sc, runs, off if want_cigar else None, one_warp=True)
                except T.AlignError as e:
                    if e.code != 5:
                        raise
                    runs = torch.zeros(int(e.needed) + 1024, dtype=torch.int32, device=dev)
                    al.align_device(d_p, bo, bl, d_t, to_, tl_, sc, runs, off, one_warp=True)
                tm = al.timing()
                tot += tm["total_ms"]
                if rep:
                    p_launch += int(tm["kernel_launches"])
                if rep == 0:  # same scores as the batched form
                    idx = np.nonzero(buckets == b)[0]
                    if not np.array_equal(sc.cpu().numpy(), ref_scores[idx]):
                        raise SystemExit(f"plain form differs from the batched form in bucket {b}")
            if rep:
                p_ms.append(tot)
        pm = max_over_ranks(float(np.mean(p_ms)))
        plain = {"form": "one call per floor(log2 L) bucket, one warp per pair (TSU_ONE_WARP), in turn",
                 "buckets": len(sub), "ms_per_step": pm, "value": throughput(cells_all, pm) / 1e9,
                 "unit": "GCUPS", "pairs_per_s": throughput(pairs_all, pm),
                 "batched_over_plain_pairs_per_s": pm / ms, "gpu_launches": p_launch,
                 "steps": max(args.plain_steps, 1), "warmup": 1}

    # ---- e2e: host buffers (pinned) through tsu_align_batch ---------------
    e2e = None
    if not args.no_e2e:
        e_steps = max(1, e2e_steps if e2e_steps > 0 else args.steps)

        def pinned(a):
            t = torch.empty(a.shape, dtype={np.uint8: torch.uint8, np.int64: torch.int64,
                                            np.int32: torch.int32}[a.dtype.type], pin_memory=True)
            t.numpy()[...] = a
            return t

        hp = [pinned(x) for x in (pbuf, poff, plen, tbuf, toff, tlen)]
        h_sc = torch.empty(n_pairs, dtype=torch.int32, pin_memory=True)
        h_off = torch.empty(n_pairs + 1, dtype=torch.int64, pin_memory=True)
        h_runs = torch.empty(max(nruns, 1) + 4096, dtype=torch.int32, pin_memory=True)
        outs = (h_sc.numpy(), h_off.numpy(), h_runs.numpy().view(np.uint32)) if want_cigar else None

        def e2e_step():
            return al.align_arrays(*(t.numpy() for t in hp), cigar=want_cigar, out=outs, bidirectional=BIDIR)

        for _ in range(max(1, min(args.warmup, 2))):
            e2e_step()
        barrier()
        e_ms, hb, db = [], 0, 0
        for _ in range(e_steps):
            e2e_step()
            tm = al.timing()
            e_ms.append(tm["total_ms"])
            hb, db = tm["h2d_bytes"], tm["d2h_bytes"]
        barrier()
        ems = max_over_ranks(float(np.mean(e_ms)))
        e2e = {"value": throughput(cells_all, ems) / 1e9, "unit": "GCUPS", "h2d_bytes_per_step": int(hb),
               "d2h_bytes_per_step": int(db), "ms_per_step": ems, "pairs_per_s": throughput(pairs_all, ems),
               "steps": e_steps}
        # correctness of the e2e output against the device leg
        if want_cigar and not np.array_equal(outs[0], d_sc.cpu().numpy()):
            raise SystemExit("e2e scores differ from the device-resident leg")

    # ---- roofline of the align passes ---------------------------------------
    a_ms = float(np.mean(align_ms))
    roof = roofline(workload, n_pairs, plen, tlen, nruns if want_cigar else 0, work_cells, work_steps, ext_bases,
                    a_ms, clk, want_cigar, pass_log)

    cpu = cpu_baseline(pbuf, poff, plen, tbuf, toff, tlen) if (with_cpu and rank == 0) else None
    out = None
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "GCUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded, uniform ACGT, equal sub/ins/del edits)",
            "config": {"workload": f"{workload}: {n_pairs} pairs per GPU, {desc}, penalties {pen_str()}",
                       "output": "scores + CIGARs" if want_cigar else "scores only",
                       "l2": f"inputs larger than L2 ({(pbuf.nbytes + tbuf.nbytes) / 1e9:.1f} GB ASCII per GPU)",
                       "parallelism": f"data-parallel over pairs, {world} GPU(s)"},
            "pairs_per_s": pairs_s,
            "wall_ms_per_step": wall_ms,
            "gpu_launches": launches,
            "plain": plain,
            "e2e": e2e,
            "roofline": roof,
            "cpu_baseline": cpu,
            "clocks": clk,
        }
        try:  # device memory the engine plans for this batch (tsu_predict_bytes, forward passes)
            if not BIDIR:
                full_b, min_b = al.predict_bytes(plen, tlen, cigar=want_cigar)
                out["predicted_device_bytes"] = {"full": int(full_b), "min": int(min_b)}
        except T.AlignError:
            pass
    al.close()
    del d_p, d_t, d_po, d_pl, d_to, d_tl, d_sc, d_off, d_runs
    torch.cuda.empty_cache()
    return out


# Integer-issue model of the align kernel (see the kernel roofline section of
# the design notes): the fewest thread instructions the algorithm as written
# needs per (score, diagonal) cell (five ring loads, the I/D/M maxima and
# source bits, the bounds test, one 16-base extend window, the end test, the
# trimming bounds, three ring stores with their int16 clamps, the history
# word, the loop), per further 16-base extend window, and the warp
# instructions of one score step of a pair (source limits, envelope, seven
# warp reductions, limit stores, step table) and of one CIGAR run of the
# backtrace walk (one lane).
C_CELL, C_EXT, C_STEP, C_RUN = 76, 16, 70, 24


def roofline(workload, n_pairs, plen, tlen, nruns, work_cells, work_steps, ext_bases, a_ms, clk, want_cigar,
             pass_log):
    """Roofline of the align passes (the dominant kernels: 95-99.9 % of
    device time).  Binding resource: integer instruction issue --
    algorithmic warp instructions (the model above times the counted cells,
    extension bases, steps and runs) per second against 148 SMs x 4
    schedulers x the sampled SM clock.  Secondary: HBM, algorithmic bytes
    (packed input, scores, CIGAR runs, one 4-byte backtrace word per
    wavefront cell) per second against the measured copy bandwidth, with the
    DRAM traffic of an ncu capture of the same kernel scaled by pairs."""
    import torch

    if BIDIR:
        # the issue model above is the forward kernel's; the bidirectional
        # kernels report their wavefront cells and steps only
        return {"bound": "int_issue", "achieved": None, "peak": None, "unit": "Gwarp-inst/s", "frac": None,
                "traffic": None, "kernel": "bidir_kernel" + (" + segment_kernel" if want_cigar else ""),
                "kernel_ms": a_ms, "cells": work_cells, "score_steps": work_steps,
                "cells_per_s": work_cells / (a_ms / 1e3), "passes": pass_log,
                "note": "no calibrated issue model for the bidirectional kernels"}
    peak, peak_kind = measured_peaks()
    words = float(np.sum((plen.astype(np.int64) + 31) // 32 + 1) + np.sum((tlen.astype(np.int64) + 31) // 32 + 1))
    packed_in = words * 8
    out_bytes = n_pairs * 4 + 4 * nruns
    hist_bytes = 4 * work_cells if want_cigar else 0
    algo = packed_in + out_bytes + hist_bytes
    achieved = algo / (a_ms / 1e3) / 1e9
    model = "_" + METRIC_NAME if METRIC_NAME else ("_dual" if len(PEN) == 5 else "")
    prof = load_traffic(f"align_{workload}{model}") if want_cigar else None
    traffic = prof["dram_bytes"] * n_pairs / prof["pairs"] if prof else None
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    mhz = clk.get("sm_mhz") or clk.get("sm_max_mhz") or 1965.0
    warp_inst = (C_CELL * work_cells + C_EXT * ext_bases / 16.0) / 32.0 + C_STEP * work_steps + C_RUN * nruns
    issue_peak = sms * 4 * mhz * 1e6  # warp instructions per second
    inst_rate = warp_inst / (a_ms / 1e3)
    roof = {"bound": "int_issue", "achieved": inst_rate / 1e9, "peak": issue_peak / 1e9, "unit": "Gwarp-inst/s",
            "frac": inst_rate / issue_peak, "traffic": traffic, "peak_kind": f"{sms} SMs x 4 schedulers x {mhz:.0f} MHz "
            "(sampled SM clock under load)", "kernel": "align_kernel<cigar>" if want_cigar else "align_kernel<score>",
            "kernel_ms": a_ms, "algorithmic_warp_instructions": warp_inst,
            "model": {"c_cell": C_CELL, "c_ext_per_16_bases": C_EXT, "c_step": C_STEP, "c_run": C_RUN},
            "cells": work_cells, "score_steps": work_steps, "extension_bases": ext_bases, "cigar_runs": nruns,
            "cells_per_s": work_cells / (a_ms / 1e3), "passes": pass_log,
            "hbm": {"achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "peak_kind": peak_kind, "algorithmic_bytes_per_launch": algo, "traffic": traffic}}
    if prof:
        roof["ncu_issue_active_frac"] = prof.get("issue_active_frac")
        roof["ncu_alu_pipe_frac"] = prof.get("alu_pipe_frac")
        roof["traffic_source"] = prof.get("source")
    return roof


if __name__ == "__main__":
    main()
