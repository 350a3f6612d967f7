"""Generate tests/golden/kat.json and tests/golden/regress.json.

kat.json: hand-derived known-answer cases.  Each expected score and operation
string below was worked out by hand from the gap-affine WFA recurrences
(reference wfa_gpu.cu:616-629) and the backtrace tie order of the piggyback
codes in the reference's common.h:67-77 (mismatch > D_ext > D_open > I_ext >
I_open); the derivation of the non-obvious ones is written next to them.  The
script refuses to write the file unless the independent Gotoh DP agrees with
every expected score and every expected operation string re-costs to it.

regress.json: seeded random pairs (Python's own PRNG, independent of the
engine's generator) with the oracle's score and operation string, each score
checked against the Gotoh DP.  These pin the oracle's outputs so that a change
to the oracle shows up as a diff here.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import random
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402

P462 = (4, 6, 2)

KAT = [
    # identical sequences: all matches at score 0
    dict(p="ACGT", t="ACGT", pen=P462, score=0, ops="MMMM"),
    dict(p="ACGTACGT", t="ACGTACGT", pen=P462, score=0, ops="MMMMMMMM"),
    # one substitution: x=4 beats any gap pair (2*(o+e)=16)
    dict(p="ACGT", t="AGGT", pen=P462, score=4, ops="MXMM"),
    dict(p="GATTACA", t="GATCACA", pen=P462, score=4, ops="MMMXMMM"),
    dict(p="A", t="C", pen=P462, score=4, ops="X"),
    # one inserted G in a GG run.  s=0 extends M[0][0] to 3 (ACG);
    # s=8: I[8][1] = M[0][0]+1 = 4, extends T=T to 5 = n on k = n-m = 1.
    # Backtrace: candidates of M[8][1] are only I_open (4): 1 match, then I,
    # then M[0][0]=3 gives 3 matches -> the insertion lands after ACG.
    dict(p="ACGT", t="ACGGT", pen=P462, score=8, ops="MMMIM"),
    # the mirror case: D_open from M[0][2]... same reasoning on k = -1
    dict(p="ACGGT", t="ACGT", pen=P462, score=8, ops="MMMDM"),
    # empty sequences: one gap of the other's length, or nothing
    dict(p="", t="", pen=P462, score=0, ops=""),
    dict(p="", t="ACG", pen=P462, score=12, ops="III"),
    dict(p="ACG", t="", pen=P462, score=12, ops="DDD"),
    # one 3-base gap after 4 matches: 6 + 3*2 = 12; M[0][0] extends to 4,
    # then I_open at s=8, I_ext at s=10, 12 (ext beats nothing else).
    dict(p="AAAA", t="AAAAAAA", pen=P462, score=12, ops="MMMMIII"),
    # x=20 > 2(o+e)=4: a mismatch is cheaper as I + D.  At s=4 (gcd 1),
    # M[4][0] has two candidates with offset 1: I_open from M[2][-1] (=0, +1)
    # and D_open from M[2][1] (=1).  D wins the tie (code 5 > 1): the last
    # operation is D, then v=0 leaves one leading I -> "ID".
    dict(p="A", t="C", pen=(20, 1, 1), score=4, ops="ID"),
    # bytes outside ACGT are compared exactly (case-sensitive): 4 mismatches
    # (16) beat deleting and inserting all four (2*(6+8)=28).
    dict(p="acgt", t="ACGT", pen=P462, score=16, ops="XXXX"),
    dict(p="ANNA", t="ANNA", pen=P462, score=0, ops="MMMM"),
]


def _mutate(rng: random.Random, s: str, n_edits: int, alpha: str) -> str:
    t = list(s)
    for _ in range(n_edits):
        r = rng.random()
        pos = rng.randint(0, max(0, len(t) - 1))
        if r < 1 / 3 and t:
            t[pos] = rng.choice([c for c in alpha if c != t[pos]] or alpha)
        elif r < 2 / 3:
            t.insert(pos, rng.choice(alpha))
        elif t:
            del t[pos]
    return "".join(t)


def regress_cases():
    rng = random.Random(0x5453554E)
    cases = []
    pens = [(4, 6, 2), (1, 0, 1), (3, 5, 1), (7, 2, 3), (20, 1, 1), (2, 10, 1), (5, 11, 3), (4, 6, 2)]
    # short random pairs, mixed penalties
    for i in range(120):
        alpha = "ACGT" if i % 5 else "AC"
        m = rng.randint(0, 60)
        p = "".join(rng.choice(alpha) for _ in range(m))
        t = _mutate(rng, p, rng.randint(0, 8), alpha) if i % 7 else "".join(
            rng.choice(alpha) for _ in range(rng.randint(0, 60)))
        cases.append((p, t, pens[i % len(pens)]))
    # C1 shape (150 bp, 2%) and reduced C2/C3 shapes, 4/6/2
    for L, rate, cnt in [(150, 0.02, 40), (1000, 0.05, 12), (3000, 0.15, 3)]:
        for _ in range(cnt):
            p = "".join(rng.choice("ACGT") for _ in range(L))
            cases.append((p, _mutate(rng, p, int(round(L * rate)), "ACGT"), P462))
    out = []
    for p, t, pen in cases:
        s, ops = O.align(p, t, *pen)
        g = O.gotoh(p, t, *pen)
        assert s == g, (p, t, pen, s, g)
        assert O.cigar_cost(ops, p, t, *pen) == s
        out.append(dict(p=p, t=t, pen=list(pen), score=s, ops=ops))
    return out


def main():
    kat = []
    for c in KAT:
        p, t, pen = c["p"], c["t"], c["pen"]
        g = O.gotoh(p, t, *pen)
        assert g == c["score"], f"Gotoh disagrees with the hand-derived score: {c} -> {g}"
        assert O.cigar_cost(c["ops"], p, t, *pen) == c["score"], f"expected ops do not re-cost: {c}"
        kat.append(dict(p=p, t=t, pen=list(pen), score=c["score"], ops=c["ops"]))
    with open(os.path.join(HERE, "kat.json"), "w") as f:
        json.dump(kat, f, indent=1)
    with open(os.path.join(HERE, "regress.json"), "w") as f:
        json.dump(regress_cases(), f)
    print(f"wrote {len(kat)} known-answer cases and the regression set")


if __name__ == "__main__":
    main()
