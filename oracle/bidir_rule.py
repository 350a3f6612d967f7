"""Breakpoint rule of a bidirectional (BiWFA-style) gap-affine alignment --
TEST INFRASTRUCTURE ONLY: a small pure-Python model, pinned by
tests/test_bidir_rule.py against the Gotoh DP, that a future ultralow-memory
mode (two-ring forward/reverse wavefronts, recursion on the breakpoints)
rests on.  Nothing in the product imports it.

Forward WFA on (pattern, text) and reverse WFA on the reversed strings keep,
per score and diagonal, M (after extension), M's pre-extension offset, I and
D.  For growing totals T the first overlap is:
  * M-M at scores (sf, sr), sf + sr = T, on diagonal k (reverse diagonal
    n - m - k): the forward extension run [pre_f, off_f] and the reverse one,
    mapped forward, [n - off_r, n - pre_r], intersect.  A cut inside both
    runs splits the pair into two halves of cost <= sf and <= sr;
  * I-I or D-D at scores sf + sr = T + o (the gap is opened on both sides):
    forward and reverse gap cells meet exactly (off_f + off_r == n); the left
    half ends in the gap, the right half continues it without an opening.
Soundness (the halves cost at most T) holds by construction; that the first
such T is the optimal score is what the test checks.
"""
from __future__ import annotations

NULL = -(10 ** 9)


def wavefronts(p: str, t: str, x: int, o: int, e: int, smax: int):
    """All forward wavefronts to smax: (M, M_pre, I, D), each {s: {k: offset}}."""
    m, n = len(p), len(t)

    def ext(k: int, off: int) -> int:
        v = off - k
        while v < m and off < n and p[v] == t[off]:
            v += 1
            off += 1
        return off

    def inb(off: int, k: int) -> bool:
        return 0 <= off <= n and 0 <= off - k <= m

    M, Mp, I, D = {0: {0: ext(0, 0)}}, {0: {0: 0}}, {0: {}}, {0: {}}
    for s in range(1, smax + 1):
        ks = set()
        for src in (M.get(s - x, {}), M.get(s - o - e, {}), I.get(s - e, {}), D.get(s - e, {})):
            for k in src:
                ks.update((k - 1, k, k + 1))
        Ms, Mps, Is, Ds = {}, {}, {}, {}
        for k in ks:
            ins = max(M.get(s - o - e, {}).get(k - 1, NULL), I.get(s - e, {}).get(k - 1, NULL)) + 1
            dele = max(M.get(s - o - e, {}).get(k + 1, NULL), D.get(s - e, {}).get(k + 1, NULL))
            mis = M.get(s - x, {}).get(k, NULL) + 1
            if inb(ins, k):
                Is[k] = ins
            if inb(dele, k):
                Ds[k] = dele
            pv = max(mis, ins, dele)
            if inb(pv, k):
                Mps[k] = pv
                Ms[k] = ext(k, pv)
        M[s], Mp[s], I[s], D[s] = Ms, Mps, Is, Ds
    return M, Mp, I, D


def first_breakpoint(p: str, t: str, x: int, o: int, e: int, smax: int):
    """(T, (component, sf, sr, k)) of the first overlap, or (None, None)."""
    m, n = len(p), len(t)
    FM, FMp, FI, FD = wavefronts(p, t, x, o, e, smax)
    RM, RMp, RI, RD = wavefronts(p[::-1], t[::-1], x, o, e, smax)
    for T in range(0, 2 * smax + 1):
        for sf in range(0, min(T, smax) + 1):
            sr = T - sf
            if sr > smax:
                continue
            for k, hf in FM[sf].items():
                kr = (n - m) - k
                if kr in RM[sr]:
                    lo = max(FMp[sf][k], n - RM[sr][kr])
                    hi = min(hf, n - RMp[sr][kr])
                    if lo <= hi:
                        return T, ("M", sf, sr, k)
        for sf in range(0, min(T + o, smax) + 1):
            sr = T + o - sf
            if sr > smax or sr < 0:
                continue
            for comp, Fw, Rw in (("I", FI, RI), ("D", FD, RD)):
                for k, hf in Fw[sf].items():
                    kr = (n - m) - k
                    if kr in Rw[sr] and hf + Rw[sr][kr] == n:
                        return T, (comp, sf, sr, k)
    return None, None
