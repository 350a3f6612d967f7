"""Reference-run score fixtures: tests/golden/ref_scores.json.

Runs the reference's own GPU kernel (wfa_dispatcher, wfa_gpu.cu:191-752,
built unchanged by oracle/ref_build.sh into oracle/_ref/ref_harness) on seeded
pair sets and stores its int16 scores.  Needs a GPU; the harness certifies
every set with the CPU model of the kernel (oracle/ref_kernel_model.c) before
it launches anything, and records whether the GPU scores equal the model's.

    python tests/golden/make_ref_scores.py --out tests/golden/ref_scores.json
    python tests/golden/make_ref_scores.py --from-dir gpurun_out --out ...  # assemble earlier harness runs

Sets (penalties 4/6/2, text = pattern with round(L * rate) edits, equal
insertion and deletion counts, so every pair is L x L as the kernel needs):
  c1   10,000 x 150 bp at 2 %   (the CPU-runnable configuration, in full)
  c2r   3,000 x 1,000 bp at 5 % (the first pairs of the 1 kbp configuration)
  c2t  20,000 x 1,000 bp at 5 % (the same stream; also timed)
"""
import argparse
import base64
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
SEED = 0x5453554E414D49
SETS = [
    {"name": "c1", "seed": SEED + 0, "first": 0, "num": 10_000, "len": 150, "rate": 0.02, "reps": 3},
    {"name": "c2r", "seed": SEED + 1, "first": 0, "num": 3_000, "len": 1000, "rate": 0.05, "reps": 1},
    {"name": "c2t", "seed": SEED + 1, "first": 0, "num": 20_000, "len": 1000, "rate": 0.05, "reps": 2},
]
PEN = (4, 6, 2)
STEP_CAP = 32000


def parse(txt_path, summary_path):
    gpu, model = [], []
    with open(txt_path) as f:
        for ln in f:
            i, g, m = ln.split()
            gpu.append(int(g))
            model.append(int(m))
    with open(summary_path) as f:
        summary = json.loads(f.read().strip().splitlines()[-1])
    return np.array(gpu, np.int16), np.array(model, np.int16), summary


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden", "ref_scores.json"))
    ap.add_argument("--harness", default=os.path.join(ROOT, "oracle", "_ref", "ref_harness"))
    ap.add_argument("--from-dir", default=None, help="use ref_<set>.txt / ref_<set>.json written by earlier runs")
    ap.add_argument("--work", default=os.path.join(ROOT, "gpurun_out"))
    args = ap.parse_args()
    os.makedirs(args.work, exist_ok=True)
    out = {"what": "scores of the reference's own GPU kernel (wfa_dispatcher, wfa_gpu.cu:191-752), built unchanged "
                   "for sm_100a by oracle/ref_build.sh and run by oracle/ref_harness on one B200",
           "made_by": "tests/golden/make_ref_scores.py", "penalties": list(PEN),
           "generator": "ora_gen_batch (oracle/wfa_gen.c) = tsu_gen_batch", "step_cap": STEP_CAP, "sets": []}
    for s in SETS:
        name = s["name"]
        base = args.from_dir or args.work
        txt, js = os.path.join(base, f"ref_{name}.txt"), os.path.join(base, f"ref_{name}.json")
        if not args.from_dir:
            cmd = [args.harness, *map(str, PEN), str(s["seed"]), str(s["first"]), str(s["num"]), str(s["len"]),
                   str(s["rate"]), "0", str(STEP_CAP), txt, str(s["reps"])]
            with open(js, "w") as f:
                subprocess.run(cmd, stdout=f, check=True, timeout=900)
        gpu, model, summary = parse(txt, js)
        if len(gpu) != s["num"]:
            sys.exit(f"{name}: {len(gpu)} scores, expected {s['num']}")
        rec = {k: s[k] for k in ("name", "seed", "first", "num", "len", "rate")}
        rec.update({"wf_length": summary["wf_length"], "max_abs_k": summary["max_abs_k"],
                    "kernel_ms": summary["kernel_ms"], "gcups": summary["gcups"], "launches": summary["reps"],
                    "gpu_equals_model": bool(np.array_equal(gpu, model)),
                    "scores_int16_b64": base64.b64encode(gpu.astype("<i2").tobytes()).decode()})
        out["sets"].append(rec)
        print(f"{name}: {s['num']} pairs, kernel {summary['kernel_ms']:.2f} ms, {summary['gcups']:.1f} GCUPS, "
              f"GPU == model: {rec['gpu_equals_model']}")
    with open(args.out, "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
