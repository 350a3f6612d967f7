"""The CUDA kernels' own source, run on the CPU through the warp emulator
(tests/emu/warp_emu.h) under AddressSanitizer/UBSan, against the oracle.

This checks the kernels' index arithmetic and outputs without a GPU: any
shared- or global-memory access outside its buffer aborts the run, and every
score and operation string must equal the oracle's."""
import os
import random
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EMU_DIR = os.path.join(ROOT, "tests", "emu")
EXE = os.path.join(EMU_DIR, "_build", "emu_driver")
SRCS = [os.path.join(EMU_DIR, f) for f in ("emu_driver.cpp", "emu_model.cpp", "warp_emu.h")] + [
    os.path.join(ROOT, "tsunami_pact_b200", "csrc", f)
    for f in os.listdir(os.path.join(ROOT, "tsunami_pact_b200", "csrc"))
    if f.endswith((".cuh", ".h"))
]


@pytest.fixture(scope="module")
def emu():
    os.makedirs(os.path.dirname(EXE), exist_ok=True)
    newest = max(os.path.getmtime(s) for s in SRCS)
    if not os.path.exists(EXE) or os.path.getmtime(EXE) < newest:
        # the driver and one object per penalty model, compiled in parallel
        flags = ["-std=c++20", "-O1", "-g", "-fsanitize=address,undefined", "-fno-omit-frame-pointer",
                 "-fno-sanitize-recover=undefined"]
        # objects and the executable are built under a per-process name and
        # renamed into place, so parallel pytest workers never run a
        # half-written binary
        build = os.path.join(os.path.dirname(EXE), f"tmp{os.getpid()}")
        os.makedirs(build, exist_ok=True)
        jobs = [(os.path.join(build, "driver.o"), [os.path.join(EMU_DIR, "emu_driver.cpp")])]
        for model, fn in ((0, "run_pass_affine"), (1, "run_pass_dual"), (2, "run_pass_linear")):
            jobs.append((os.path.join(build, f"model{model}.o"),
                         [f"-DEMU_MODEL={model}", f"-DEMU_RUN_FN={fn}", os.path.join(EMU_DIR, "emu_model.cpp")]))
        procs = [subprocess.Popen(["g++", *flags, "-c", "-o", obj, *args]) for obj, args in jobs]
        assert all(p.wait() == 0 for p in procs), "emulator build failed"
        tmp_exe = os.path.join(build, "emu_driver")
        subprocess.run(["g++", *flags, "-o", tmp_exe, *(obj for obj, _ in jobs), "-lpthread"], check=True)
        os.replace(tmp_exe, EXE)
        shutil.rmtree(build, ignore_errors=True)
    return EXE


def run_emu(exe, pairs, pen=(4, 6, 2), cigar=True, hint=0.2, shared_first=True, gw=1, free=(0, 0, 0, 0), lowmem=0):
    o2, e2 = (pen[3], pen[4]) if len(pen) == 5 else (-1, 0)
    hdr = (f"{pen[0]} {pen[1]} {pen[2]} {o2} {e2} {free[0]} {free[1]} {free[2]} {free[3]} {lowmem} {int(cigar)} "
           f"{hint} {int(shared_first)} {gw} {len(pairs)}\n")
    body = b"".join(f"{len(p)} {len(t)}\n".encode() + p + b"\n" + t + b"\n" for p, t in pairs)
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=0:abort_on_error=1", UBSAN_OPTIONS="halt_on_error=1")
    r = subprocess.run([exe], input=hdr.encode() + body, capture_output=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr.decode()[-3000:]
    lines = r.stdout.decode().split("\n")
    out = []
    for ln in lines[: len(pairs)]:
        s, ops = ln.split("\t")
        out.append((int(s), ops))
    tail = lines[len(pairs)].split()
    return out, int(tail[1]), int(tail[3]), tail[5]


def _b(s):
    return s if isinstance(s, bytes) else s.encode()


def _edited(rng, L, rate):
    """A random pattern and a text with about L*rate substitutions/indels."""
    p = "".join(rng.choice("ACGT") for _ in range(L))
    t = list(p)
    for _ in range(int(L * rate)):
        pos = rng.randint(0, max(0, len(t) - 1))
        r = rng.random()
        if r < 0.33 and t:
            t[pos] = rng.choice("ACGT")
        elif r < 0.66:
            t.insert(pos, rng.choice("ACGT"))
        elif t:
            del t[pos]
    return p, "".join(t)


def check(exe, oracle, pairs, pen=(4, 6, 2), **kw):
    pairs = [(_b(p), _b(t)) for p, t in pairs]
    got, passes, retried, gws = run_emu(exe, pairs, pen, **kw)
    for (p, t), (s, ops) in zip(pairs, got):
        es, eops = oracle.align(p, t, *pen)
        assert (s, ops) == (es, eops), (p, t, pen, s, es, ops, eops)
    return passes, retried, gws


def test_kat_each_alone(emu, oracle, kat_cases):
    """One pair per batch: single-pair launches, tiny rings."""
    for c in kat_cases:
        check(emu, oracle, [(c["p"], c["t"])], tuple(c["pen"]))


def test_kat_as_batch(emu, oracle, kat_cases):
    by = {}
    for c in kat_cases:
        by.setdefault(tuple(c["pen"]), []).append((c["p"], c["t"]))
    for pen, pairs in by.items():
        check(emu, oracle, pairs, pen)


def test_regression_fixture(emu, oracle, regress_cases):
    """The regression set up to 600 bp (the longer pairs run in the GPU suite)."""
    by = {}
    for c in regress_cases:
        if max(len(c["p"]), len(c["t"])) <= 600:
            by.setdefault(tuple(c["pen"]), []).append((c["p"], c["t"]))
    for pen, pairs in by.items():
        check(emu, oracle, pairs, pen)


@pytest.mark.parametrize("pen", [(4, 6, 2), (20, 1, 1), (3, 5, 1), (5, 11, 3)])
def test_random_mixed(emu, oracle, pen):
    rng = random.Random(sum(pen))
    pairs = []
    for i in range(60):
        alpha = "ACGT" if i % 5 else "ACGTN"
        p = "".join(rng.choice(alpha) for _ in range(rng.randint(0, 120)))
        t = list(p)
        for _ in range(rng.randint(0, 12)):
            pos = rng.randint(0, max(0, len(t) - 1))
            r = rng.random()
            if r < 0.33 and t:
                t[pos] = rng.choice(alpha)
            elif r < 0.66:
                t.insert(pos, rng.choice(alpha))
            elif t:
                del t[pos]
        pairs.append((p, "".join(t)))
    check(emu, oracle, pairs, pen)


def test_global_mode_and_retries(emu, oracle):
    """A tiny hint forces scratch overflow and several global-mode passes."""
    rng = random.Random(3)
    pairs = []
    for _ in range(3):
        p = "".join(rng.choice("ACGT") for _ in range(rng.randint(40, 120)))
        t = "".join(rng.choice("ACGT") for _ in range(rng.randint(40, 120)))
        pairs.append((p, t))
    passes, retried, gws = check(emu, oracle, pairs, hint=0.0001)
    assert passes > 1 and retried > 0
    check(emu, oracle, pairs, shared_first=False)


def test_wide_pairs_leave_shared_ring(emu, oracle):
    """Wavefronts wider than the shared ring (384 diagonals) are re-run in
    global mode; a batch mixing both kinds."""
    rng = random.Random(9)
    pairs = [_edited(rng, 330, 0.25)]
    pairs += [("ACGT" * 10, "ACGA" * 10), ("", "A" * 400)]
    passes, retried, gws = check(emu, oracle, pairs)
    assert retried >= 1 and gws.split(",")[1] != "s1", gws


def test_score_only(emu, oracle):
    rng = random.Random(4)
    pairs = [("".join(rng.choice("ACGT") for _ in range(rng.randint(0, 90))),
              "".join(rng.choice("ACGT") for _ in range(rng.randint(0, 90)))) for _ in range(30)]
    got, _, _, _ = run_emu(emu, [(_b(p), _b(t)) for p, t in pairs], cigar=False)
    for (p, t), (s, ops) in zip(pairs, got):
        assert s == oracle.align(p, t)[0] and ops == ""


@pytest.mark.parametrize("gw,shared", [(2, True), (4, True), (8, True), (16, True), (2, False), (8, False),
                                       (16, False), (32, True), (32, False)])
def test_warp_groups(emu, oracle, gw, shared):
    """Several warps per pair (named barriers, partial reductions combined
    across warps), in both ring modes, with CIGARs."""
    rng = random.Random(gw * 7 + shared)
    pairs = []
    for i in range(6):
        L = rng.randint(100, 700)
        p = "".join(rng.choice("ACGT") for _ in range(L))
        t = list(p)
        for _ in range(rng.randint(0, L // 8)):
            pos = rng.randint(0, max(0, len(t) - 1))
            r = rng.random()
            if r < 0.33 and t:
                t[pos] = rng.choice("ACGT")
            elif r < 0.66:
                t.insert(pos, rng.choice("ACGT"))
            elif t:
                del t[pos]
        pairs.append((p, "".join(t)))
    pairs += [("", "ACGTACGTAC"), ("ACGTNNACGT", "ACGTACGT"), ("A" * 64, "A" * 64)]
    passes, retried, gws = check(emu, oracle, pairs, shared_first=shared, gw=gw)
    assert gws.split(",")[0] == ("s" if shared else "g") + str(gw) or not shared


@pytest.mark.parametrize("gw,shared", [(1, True), (1, False), (2, True), (4, True), (4, False)])
def test_end_diagonal_positions(emu, oracle, gw, shared):
    """The end-to-end end test reads M on diagonal n - m back from the ring
    in the thread that computed it: end diagonals at every offset around the
    warp and group boundaries (n - m from -70 to 100, including 0, +-1,
    +-31, +-32, +-33, 63-65), pairs that end at score 0 and empty sides,
    with and without CIGARs, on both rings; gap-affine, dual gap-affine and
    gap-linear kernels."""
    rng = random.Random(90 + gw * 2 + shared)
    pairs = []
    for d in [-70, -65, -64, -63, -33, -32, -31, -1, 0, 1, 31, 32, 33, 63, 64, 65, 100]:
        p, t = _edited(rng, rng.randint(80, 160), 0.04)
        if d > 0:
            t = t + "".join(rng.choice("ACGT") for _ in range(d))
        elif d < 0:
            p = p + "".join(rng.choice("ACGT") for _ in range(-d))
        pairs.append((p, t))
    pairs += [("ACGT" * 20, "ACGT" * 20), ("", "ACG"), ("ACG", ""), ("", "")]
    check(emu, oracle, pairs, shared_first=shared, gw=gw)
    bp = [(_b(p), _b(t)) for p, t in pairs]
    got, _, _, _ = run_emu(emu, bp, cigar=False, shared_first=shared, gw=gw)
    for (p, t), (sc, ops) in zip(bp, got):
        assert sc == oracle.align(p, t)[0] and ops == "", (p, t)
    # the dual gap-affine and gap-linear kernels take the same end test
    got, _, _, _ = run_emu(emu, bp, (4, 6, 2, 24, 1), shared_first=shared, gw=gw)
    for (p, t), (sc, ops) in zip(bp, got):
        assert (sc, ops) == oracle.align2(p, t), (p, t)
    got, _, _, _ = run_emu(emu, bp, (1, -1, 1), shared_first=shared, gw=gw)
    for (p, t), (sc, ops) in zip(bp, got):
        assert (sc, ops) == oracle.align_linear(p, t, 1, 1), (p, t)


def test_ladder_to_groups(emu, oracle):
    """Pairs whose wavefronts outgrow one warp's shared ring (384 diagonals)
    climb the ladder to a group with a wider shared ring."""
    rng = random.Random(21)
    pairs = [_edited(rng, 420, 0.22) for _ in range(2)]
    pairs += [("ACGT" * 30, "ACGA" * 30)]
    passes, retried, gws = check(emu, oracle, pairs)
    steps = gws.split(",")
    assert steps[0] == "s1" and steps[1].startswith("s") and int(steps[1][1:]) > 1, gws


# --- dual gap-affine kernels (align_kernel<..., kDual = true>) ---------------

def check_dual(exe, oracle, pairs, pen, **kw):
    pairs = [(_b(p), _b(t)) for p, t in pairs]
    got, passes, retried, gws = run_emu(exe, pairs, pen, **kw)
    for (p, t), (s, ops) in zip(pairs, got):
        es, eops = oracle.align2(p, t, *pen)
        if kw.get("cigar", True):
            assert (s, ops) == (es, eops), (p, t, pen, s, es, ops, eops)
        else:
            assert s == es and ops == "", (p, t, pen, s, es)
    return passes, retried, gws


def _long_indels(rng, n, lo=0, hi=160):
    """Pairs with substitutions and long insertions / deletions (where the
    second gap piece is the cheaper one)."""
    pairs = []
    for _ in range(n):
        p = "".join(rng.choice("ACGT") for _ in range(rng.randint(lo, hi)))
        t = list(p)
        for _ in range(rng.randint(0, 4)):
            pos = rng.randint(0, len(t))
            L = rng.randint(1, 30)
            if rng.random() < 0.5:
                t[pos:pos] = [rng.choice("ACGT") for _ in range(L)]
            else:
                del t[pos:pos + L]
        for _ in range(rng.randint(0, 6)):
            if t:
                t[rng.randrange(len(t))] = rng.choice("ACGT")
        pairs.append((p, "".join(t)))
    return pairs


@pytest.mark.parametrize("pen", [(4, 6, 2, 24, 1), (3, 5, 3, 20, 1), (6, 2, 3, 10, 1), (1, 1, 1, 1, 1),
                                 (8, 4, 4, 12, 2)])
def test_dual_random(emu, oracle, pen):
    """One warp per pair, shared ring first, ladder as the engine."""
    rng = random.Random(sum(pen))
    pairs = _long_indels(rng, 24) + [("", ""), ("", "ACGTACGT"), ("ACGTAC", ""), ("ACGTNNACGT", "ACGTACGT")]
    check_dual(emu, oracle, pairs, pen)


def test_dual_score_only(emu, oracle):
    rng = random.Random(3)
    check_dual(emu, oracle, _long_indels(rng, 20), (4, 6, 2, 24, 1), cigar=False)


@pytest.mark.parametrize("gw,shared", [(4, True), (16, True), (2, False), (8, False), (32, False)])
def test_dual_warp_groups(emu, oracle, gw, shared):
    """Several warps per pair: the 11 partials combined across warps."""
    rng = random.Random(gw * 5 + shared)
    pairs = _long_indels(rng, 3, 150, 360)
    check_dual(emu, oracle, pairs, (4, 6, 2, 24, 1), shared_first=shared, gw=gw)


def test_dual_ladder(emu, oracle):
    """Wide dual wavefronts leave one warp's shared ring and climb the ladder."""
    rng = random.Random(9)
    pairs = [_edited(rng, 400, 0.22)] + _long_indels(rng, 1, 200, 300)
    passes, retried, gws = check_dual(emu, oracle, pairs, (4, 6, 2, 24, 1))
    assert passes > 1, gws


# --- gap-linear kernels (align_kernel<..., kModelLinear>; edit, indel) -------

def check_linear(exe, oracle, pairs, x, e, **kw):
    pairs = [(_b(p), _b(t)) for p, t in pairs]
    got, passes, retried, gws = run_emu(exe, pairs, (x, -1, e), **kw)
    for (p, t), (s, ops) in zip(pairs, got):
        es, eops = oracle.align_linear(p, t, x, e)
        if kw.get("cigar", True):
            assert (s, ops) == (es, eops), (p, t, x, e, s, es, ops, eops)
        else:
            assert s == es and ops == "", (p, t, x, e, s, es)
    return passes, retried, gws


@pytest.mark.parametrize("xe", [(1, 1), (3, 1), (2, 3), (4, 2)])
def test_linear_random(emu, oracle, xe):
    rng = random.Random(xe[0] * 10 + xe[1])
    pairs = [_edited(rng, rng.randint(0, 160), 0.1) for _ in range(24)]
    pairs += [("", ""), ("", "ACGT"), ("ACG", ""), ("ACGTNNACGT", "ACGTACGT"), ("kitten", "sitting")]
    check_linear(emu, oracle, pairs, *xe)


def test_linear_score_only_and_groups(emu, oracle):
    rng = random.Random(4)
    pairs = [_edited(rng, rng.randint(100, 400), 0.12) for _ in range(4)]
    check_linear(emu, oracle, pairs, 1, 1, cigar=False)
    for gw, shared in [(4, True), (8, False)]:
        check_linear(emu, oracle, pairs, 1, 1, shared_first=shared, gw=gw)


def test_linear_ladder(emu, oracle):
    rng = random.Random(12)
    # two unrelated 420 bp sequences: edit distance > 192, so more than one
    # warp's 384 diagonals
    pairs = [("".join(rng.choice("ACGT") for _ in range(420)), "".join(rng.choice("ACGT") for _ in range(420)))]
    passes, retried, gws = check_linear(emu, oracle, pairs, 1, 1)
    assert passes > 1, gws


# --- free ends (gap-affine) --------------------------------------------------

def check_ends_free(exe, oracle, pairs, free, pen=(4, 6, 2), **kw):
    pairs = [(_b(p), _b(t)) for p, t in pairs]
    got, passes, retried, gws = run_emu(exe, pairs, pen, free=free, **kw)
    for (p, t), (s, ops) in zip(pairs, got):
        es, eops = oracle.align_ends_free(p, t, free, *pen)
        if kw.get("cigar", True):
            assert (s, ops) == (es, eops), (p, t, free, s, es, ops, eops)
        else:
            assert s == es and ops == "", (p, t, free, s, es)
    return passes, retried, gws


def _flanked(rng, n, lo, hi):
    """A core sequence with random flanks on the pattern and on the text."""
    out = []
    for _ in range(n):
        core = "".join(rng.choice("ACGT") for _ in range(rng.randint(lo, hi)))
        t = list(core)
        for _ in range(len(core) // 20):
            t[rng.randrange(len(t))] = rng.choice("ACGT")
        fl = lambda: "".join(rng.choice("ACGT") for _ in range(rng.randint(0, 30)))
        out.append((fl() + core + fl(), fl() + "".join(t) + fl()))
    return out


@pytest.mark.parametrize("free", [(0, 0, 0, 0), (30, 30, 30, 30), (0, 0, 40, 40), (40, 40, 0, 0), (5, 0, 0, 12),
                                  (1000, 1000, 1000, 1000)])
def test_ends_free_random(emu, oracle, free):
    rng = random.Random(sum(free) + 1)
    pairs = _flanked(rng, 16, 0, 150) + [("", ""), ("", "ACGT"), ("ACG", ""), ("ACGTNNACGT", "ACGTACGT")]
    check_ends_free(emu, oracle, pairs, free)


def test_ends_free_groups_and_score_only(emu, oracle):
    rng = random.Random(31)
    pairs = _flanked(rng, 4, 200, 400)
    check_ends_free(emu, oracle, pairs, (50, 50, 50, 50), cigar=False)
    for gw, shared in [(4, True), (8, False)]:
        check_ends_free(emu, oracle, pairs, (50, 50, 50, 50), shared_first=shared, gw=gw)



def test_ends_free_linear_and_dual(emu, oracle):
    """Free ends with the gap-linear and the dual gap-affine kernels."""
    rng = random.Random(41)
    pairs = _flanked(rng, 10, 0, 120) + [("", "ACGT"), ("ACG", "")]
    bpairs = [(_b(p), _b(t)) for p, t in pairs]
    for free in [(20, 20, 20, 20), (0, 0, 30, 30)]:
        got, _, _, _ = run_emu(emu, bpairs, (1, -1, 1), free=free)
        for (p, t), (s, ops) in zip(bpairs, got):
            assert (s, ops) == oracle.align_linear_ends_free(p, t, free, 1, 1), (p, t, free)
        got, _, _, _ = run_emu(emu, bpairs, (4, 6, 2, 24, 1), free=free)
        for (p, t), (s, ops) in zip(bpairs, got):
            assert (s, ops) == oracle.align2_ends_free(p, t, free), (p, t, free)



# --- low-memory mode (checkpointed history) ----------------------------------

@pytest.mark.parametrize("K", [1, 3, 10, -1])
def test_low_memory_same_cigars(emu, oracle, K):
    """Checkpoint every K scores and recompute the history segment by
    segment: the same scores and CIGARs as the oracle (gap-affine; K = 1
    makes every segment one score, -1 lets the planner choose)."""
    rng = random.Random(60 + K)
    pairs = [_edited(rng, rng.randint(0, 250), 0.15) for _ in range(10)]
    pairs += [("", ""), ("", "ACGT"), ("ACG", ""), ("ACGTNNACGT", "ACGTACGT"), ("A" * 64, "A" * 64)]
    bp = [(_b(p), _b(t)) for p, t in pairs]
    for shared in (True, False):
        got, passes, retried, gws = run_emu(emu, bp, lowmem=K, shared_first=shared)
        for (p, t), (s, ops) in zip(bp, got):
            assert (s, ops) == oracle.align(p, t), (p, t, K, shared)


def test_low_memory_models_groups_free_ends(emu, oracle):
    """Low-memory mode with the dual and gap-linear kernels, warp groups and
    free ends."""
    rng = random.Random(70)
    pairs = [_edited(rng, rng.randint(50, 300), 0.12) for _ in range(5)]
    bp = [(_b(p), _b(t)) for p, t in pairs]
    got, _, _, _ = run_emu(emu, bp, (4, 6, 2, 24, 1), lowmem=4)
    for (p, t), (s, ops) in zip(bp, got):
        assert (s, ops) == oracle.align2(p, t), (p, t)
    got, _, _, _ = run_emu(emu, bp, (1, -1, 1), lowmem=5, gw=4, shared_first=False)
    for (p, t), (s, ops) in zip(bp, got):
        assert (s, ops) == oracle.align_linear(p, t, 1, 1), (p, t)
    free = (20, 20, 20, 20)
    got, _, _, _ = run_emu(emu, bp, lowmem=7, gw=2, shared_first=False, free=free)
    for (p, t), (s, ops) in zip(bp, got):
        assert (s, ops) == oracle.align_ends_free(p, t, free), (p, t)
