"""The GPU BiWFA kernels, run on the CPU through the warp emulator under
AddressSanitizer/UBSan, against the CPU oracle.  The breakpoint kernel
(tsu_bidir.cuh) against the oracle's two-ring breakpoint search
(ora_crossing_split, the C form of oracle/bidir_rule.py crossing_split): the
same lowest crossing total, component, forward diagonal and cut offset for
every segment -- begin and end components M, I and D, empty and unequal
segments, sub-ranges of longer pairs, one warp and warp groups, and a
zero gap opening (the gap-linear metrics run this way).  The
base-case kernel (tsu_segment.cuh) against the oracle's segment alignment
(ora_align_segment): the same operations."""
import math
import os
import random
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EMU_DIR = os.path.join(ROOT, "tests", "emu")
EXE = os.path.join(EMU_DIR, "_build", "emu_bidir")
SRCS = [os.path.join(EMU_DIR, f) for f in ("emu_bidir.cpp", "warp_emu.h")] + [
    os.path.join(ROOT, "tsunami_pact_b200", "csrc", f)
    for f in ("tsu_bidir.cuh", "tsu_segment.cuh", "tsu_common.cuh", "tsu_extend.cuh", "tsu_pack.cuh",
              "tsu_kernels.cuh")
]


@pytest.fixture(scope="module")
def emu_bidir():
    os.makedirs(os.path.dirname(EXE), exist_ok=True)
    newest = max(os.path.getmtime(s) for s in SRCS)
    if not os.path.exists(EXE) or os.path.getmtime(EXE) < newest:
        tmp = EXE + f".tmp{os.getpid()}"
        subprocess.run(["g++", "-std=c++20", "-O1", "-g", "-fsanitize=address,undefined", "-fno-omit-frame-pointer",
                        "-fno-sanitize-recover=undefined", "-o", tmp, os.path.join(EMU_DIR, "emu_bidir.cpp"),
                        "-lpthread"], check=True)
        os.replace(tmp, EXE)
    return EXE


def _input(recs, hdr):
    body = []
    for p, t, b, e, sub in recs:
        extra = f" S {sub[0]} {sub[1]} {sub[2]} {sub[3]}" if sub else ""
        body.append(f"{len(p)} {len(t)} {b} {e}{extra}\n".encode() + p + b"\n" + t + b"\n")
    return hdr.encode() + b"".join(body)


def _run(exe, data):
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=0:abort_on_error=1", UBSAN_OPTIONS="halt_on_error=1")
    r = subprocess.run([exe], input=data, capture_output=True, env=env, timeout=900)
    assert r.returncode == 0, r.stderr.decode()[-3000:]
    return r.stdout.decode().split("\n")


def run(exe, recs, pen, gw):
    out = []
    lines = _run(exe, _input(recs, f"{pen[0]} {pen[1]} {pen[2]} {gw} {len(recs)}\n"))
    for ln in lines[: len(recs)]:
        T, c, k, h = ln.split()
        out.append(None if int(T) < 0 else (int(T), c, int(k), int(h)))
    return out


def _edited(rng, L, rate, alpha="ACGT"):
    p = "".join(rng.choice(alpha) for _ in range(L))
    t = list(p)
    for _ in range(int(L * rate) + rng.randint(0, 2)):
        pos = rng.randint(0, max(0, len(t) - 1))
        r = rng.random()
        if r < 0.33 and t:
            t[pos] = rng.choice(alpha)
        elif r < 0.66:
            t.insert(pos, rng.choice(alpha))
        elif t:
            del t[pos]
    return p.encode(), "".join(t).encode()


def _check(exe, oracle, recs, pen, gw):
    got = run(exe, recs, pen, gw)
    for (p, t, b, e, sub), g in zip(recs, got):
        if sub:
            v0, h0, sm, sn = sub
            p, t = p[v0:v0 + sm], t[h0:h0 + sn]
        want = oracle.crossing_split(p, t, *pen, begin=b, end=e)
        assert g == want, (p, t, b, e, pen, g, want)


@pytest.mark.parametrize("pen,gw", [((4, 6, 2), 1), ((3, 5, 1), 1), ((5, 11, 3), 1), ((20, 1, 1), 1),
                                    ((4, 6, 2), 4), ((1, 0, 1), 1), ((3, 0, 1), 4)])
def test_segments_match_oracle(emu_bidir, oracle, pen, gw):
    rng = random.Random(hash((pen, gw)) & 0xFFFF)
    recs = []
    for i in range(30 if gw == 1 else 16):
        L = rng.choice([0, 1, 2, 5, 17, 40, 90, 150])
        p, t = _edited(rng, L, rng.choice([0.0, 0.02, 0.1, 0.3]))
        recs.append((p, t, rng.choice("MID"), rng.choice("MID"), None))
    _check(emu_bidir, oracle, recs, pen, gw)


@pytest.mark.parametrize("gw", [1, 4])
def test_sub_ranges_and_non_acgt(emu_bidir, oracle, gw):
    """Segments inside longer pairs (the recursion's halves), and pairs with
    bytes outside ACGT (compared byte by byte)."""
    rng = random.Random(5 + gw)
    recs = []
    for i in range(40 if gw == 1 else 16):
        alpha = "ACGTN" if i % 4 == 0 else "ACGT"
        p, t = _edited(rng, rng.randint(20, 300), 0.08, alpha)
        v0, h0 = rng.randint(0, len(p) // 2), rng.randint(0, len(t) // 2)
        sm, sn = rng.randint(0, len(p) - v0), rng.randint(0, len(t) - h0)
        recs.append((p, t, rng.choice("MID"), rng.choice("MID"), (v0, h0, sm, sn)))
    _check(emu_bidir, oracle, recs, (4, 6, 2), gw)


def test_long_segments_warp_group(emu_bidir, oracle):
    rng = random.Random(9)
    recs = [(*_edited(rng, 1000, 0.05), "M", "M", None), (*_edited(rng, 500, 0.15), "I", "D", None)]
    _check(emu_bidir, oracle, recs, (4, 6, 2), 16)


def _seg_ops(exe, recs, pen, step_cap, retries=None, h32=False):
    out = []
    lines = _run(exe, _input(recs, f"{pen[0]} {pen[1]} {pen[2]} {-1 if h32 else 0} {len(recs)} {step_cap}\n"))
    for ln in lines[: len(recs)]:
        st, ops = ln.split()
        out.append((int(st), "" if ops == "-" else ops))
    if retries is not None:
        retries.append(int(lines[len(recs)].split()[1]))
    return out


@pytest.mark.parametrize("pen,h32", [((4, 6, 2), False), ((3, 5, 1), False), ((20, 1, 1), False),
                                     ((4, 6, 2), True), ((1, 0, 1), False)])
def test_base_case_segments_match_oracle(emu_bidir, oracle, pen, h32):
    """The base-case kernel (tsu_segment.cuh): every segment's operations
    equal the oracle's segment alignment (ora_align_segment) for every begin
    and end component, whole pairs, sub-ranges and bytes outside ACGT; a
    step cap below what a segment needs gives status 1 (more scratch); a
    run arena too small gives status 2 and the segment's second run, with
    room, the same operations.  History as int16 and as int32."""
    rng = random.Random(hash(pen) & 0xFFFF)
    recs = []
    for i in range(36):
        alpha = "ACGTN" if i % 6 == 0 else "ACGT"
        p, t = _edited(rng, rng.choice([1, 3, 12, 40, 90]), rng.choice([0.0, 0.05, 0.15]), alpha)
        sub = None
        if i % 3 == 0 and len(p) > 4 and len(t) > 4:
            v0, h0 = rng.randint(0, len(p) // 2), rng.randint(0, len(t) // 2)
            sub = (v0, h0, rng.randint(1, len(p) - v0), rng.randint(1, len(t) - h0))
        recs.append((p, t, rng.choice("MID"), rng.choice("MID"), sub))
    g = math.gcd(*pen)
    step_cap = 400
    retries = []
    got = _seg_ops(emu_bidir, recs, pen, step_cap, retries, h32)
    assert retries[0] > 0  # the arena of 24 runs cannot hold them all
    compared = 0
    for (p, t, b, e, sub), (st, ops) in zip(recs, got):
        if sub:
            v0, h0, sm, sn = sub
            p, t = p[v0:v0 + sm], t[h0:h0 + sn]
        cost, want = oracle.align_segment(p, t, *pen, begin=b, end=e)
        if cost // g + pen[1] // g + pen[2] // g + 2 < step_cap:
            assert st == 0, (p, t, b, e, st)
            assert ops == want, (p, t, b, e, ops, want)
            compared += 1
    assert compared >= 30
    # a cap too small for the longer segments
    small = _seg_ops(emu_bidir, recs, pen, 3, None, h32)
    assert any(st == 1 for st, _ in small)
    for (st, ops), (st0, ops0) in zip(small, got):
        assert st in (0, 1)
        if st == 0:
            assert ops == ops0
