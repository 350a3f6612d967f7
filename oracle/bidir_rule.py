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

A recursion on breakpoints hands out segments that continue a gap from the
left half (begin I/D: the forward pass starts in that gap, a leading run
costs e per base) or must end in the gap the right half continues (end
I/D: the reverse pass is forced to begin with it).  gotoh_components is
the O(mn) DP of exactly those costs, which pins the rule for all nine
begin/end pairs, and split() cuts a segment into two halves whose optimal
costs add up to the segment's.
"""
from __future__ import annotations

NULL = -(10 ** 9)


def wavefronts(p: str, t: str, x: int, o: int, e: int, smax: int, start: str = "M", forced: str = "M"):
    """All forward wavefronts to smax: (M, M_pre, I, D), each {s: {k: offset}}.

    start "I" / "D": the segment continues a gap opened before it, so a
    leading run of that gap costs e per base (I or D holds offset 0 at score
    0).  forced "I" / "D": the alignment must begin with that operation at
    its ordinary cost o + e (the reverse pass of a segment that must end in
    a gap).  "M": neither."""
    m, n = len(p), len(t)

    def ext(k: int, off: int) -> int:
        v = off - k
        while v < m and off < n and p[v] == t[off]:
            v += 1
            off += 1
        return off

    def inb(off: int, k: int) -> bool:
        return 0 <= off <= n and 0 <= off - k <= m

    # cells fixed before the recurrences: {score: {k: offset}} per gap component
    seed_i, seed_d = {}, {}
    if forced == "I" and inb(1, 1):
        seed_i[o + e] = {1: 1}
    if forced == "D" and inb(0, -1):
        seed_d[o + e] = {-1: 0}
    if forced == "M":
        M, Mp = {0: {0: ext(0, 0)}}, {0: {0: 0}}
        I, D = {0: {0: 0} if start == "I" else {}}, {0: {0: 0} if start == "D" else {}}
    else:
        M, Mp, I, D = {0: {}}, {0: {}}, {0: {}}, {0: {}}
    for s in range(1, smax + 1):
        ks = set(seed_i.get(s, {})) | set(seed_d.get(s, {}))
        for src in (M.get(s - x, {}), M.get(s - o - e, {}), I.get(s - e, {}), D.get(s - e, {})):
            for k in src:
                ks.update((k - 1, k, k + 1))
        Ms, Mps, Is, Ds = {}, {}, {}, {}
        for k in ks:
            ins = max(M.get(s - o - e, {}).get(k - 1, NULL), I.get(s - e, {}).get(k - 1, NULL)) + 1
            ins = max(ins, seed_i.get(s, {}).get(k, NULL))
            dele = max(M.get(s - o - e, {}).get(k + 1, NULL), D.get(s - e, {}).get(k + 1, NULL))
            dele = max(dele, seed_d.get(s, {}).get(k, NULL))
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


def first_breakpoint(p: str, t: str, x: int, o: int, e: int, smax: int, begin: str = "M", end: str = "M"):
    """(T, (component, sf, sr, k, h)) of the first overlap, or (None, None):
    the cut is at text offset h on diagonal k (the lowest offset inside both
    M runs, or where the gap cells meet).

    begin / end: the segment's components.  begin "I"/"D" continues a gap
    from the left (forward pass started in that gap); end "I"/"D" means the
    segment must end in that gap (reverse pass forced to begin with it).
    Where the gaps meet, the two halves paid one opening each and the total
    counts one."""
    m, n = len(p), len(t)
    FM, FMp, FI, FD = wavefronts(p, t, x, o, e, smax, start=begin)
    RM, RMp, RI, RD = wavefronts(p[::-1], t[::-1], x, o, e, smax, forced=end)
    for T in range(0, 2 * smax + 1):
        # forward and reverse advance in turns: at each total the overlap
        # closest to the middle in score (sf ~ sr, the lower sf first) wins,
        # so both halves of a cut carry about half the score
        for sf in sorted(range(0, min(T, smax) + 1), key=lambda a: (abs(2 * a - T), a)):
            sr = T - sf
            if sr > smax:
                continue
            for k, hf in FM[sf].items():
                kr = (n - m) - k
                if kr in RM[sr]:
                    lo = max(FMp[sf][k], n - RM[sr][kr])
                    hi = min(hf, n - RMp[sr][kr])
                    if lo <= hi:
                        return T, ("M", sf, sr, k, lo)
        for sf in sorted(range(0, min(T + o, smax) + 1), key=lambda a: (abs(2 * a - T - o), a)):
            sr = T + o - sf
            if sr > smax or sr < 0:
                continue
            for comp, Fw, Rw in (("I", FI, RI), ("D", FD, RD)):
                for k, hf in Fw[sf].items():
                    kr = (n - m) - k
                    if kr in Rw[sr] and hf + Rw[sr][kr] == n:
                        return T, (comp, sf, sr, k, hf)
    return None, None


INF = 10 ** 9


def gotoh_components(p: str, t: str, x: int, o: int, e: int, begin: str = "M", end: str = "M") -> int:
    """Optimal cost of a segment with components (O(mn) Gotoh DP, the pin of
    the rule above): begin "I"/"D" makes a leading run of that gap cost e per
    base; end "I"/"D" requires the last operation to be that gap; "M" leaves
    either side free.  INF when no alignment qualifies."""
    m, n = len(p), len(t)
    H = [[INF] * (n + 1) for _ in range(m + 1)]
    I = [[INF] * (n + 1) for _ in range(m + 1)]
    D = [[INF] * (n + 1) for _ in range(m + 1)]
    H[0][0] = 0
    if begin == "I":
        I[0][0] = 0
    if begin == "D":
        D[0][0] = 0
    for i in range(m + 1):
        for j in range(n + 1):
            if i == 0 and j == 0:
                continue
            if j:
                I[i][j] = min(H[i][j - 1] + o + e, I[i][j - 1] + e)
            if i:
                D[i][j] = min(H[i - 1][j] + o + e, D[i - 1][j] + e)
            diag = H[i - 1][j - 1] + (0 if p[i - 1] == t[j - 1] else x) if i and j else INF
            H[i][j] = min(diag, I[i][j], D[i][j])
    return {"M": H, "I": I, "D": D}[end][m][n]


def split(p: str, t: str, x: int, o: int, e: int, begin: str = "M", end: str = "M"):
    """The segment cut at its first breakpoint: (T, left, right), each half
    (pattern, text, begin, end).  An M cut leaves both halves free at the
    cut; a gap cut makes the left half end in the gap and the right half
    continue it (its opening paid on the left)."""
    smax = max(len(p), len(t)) * max(x, o + e) + o + e + 2
    T, where = first_breakpoint(p, t, x, o, e, smax, begin, end)
    if T is None:
        return None, None, None
    comp, _, _, k, h = where
    v = h - k
    return T, (p[:v], t[:h], begin, comp), (p[v:], t[h:], comp, end)
