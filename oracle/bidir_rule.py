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

bialign() is the whole bidirectional alignment: split until a segment's
score is small, then wfa_segment(), the plain WFA of the segment with its
components and the C oracle's backtrace (byte-identical to it for free
ends).  A segment that must end in a gap is aligned on the reversed
sequences, because greedy extension towards a constrained end can pass the
cell the closing gap has to leave from.  Its CIGARs are optimal; where the
optimum is tied they may differ from the one-direction backtrace, so a GPU
bidirectional mode is checked against this recursion, not against the
plain oracle.
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
            for k, hf in sorted(FM[sf].items()):  # diagonals in ascending order
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
                for k, hf in sorted(Fw[sf].items()):
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


# piggyback codes of the backtrace's tie order (oracle/wfa_oracle.c, after
# the reference's bt_type_t, common.h:67-77): M > D_ext > D_open > I_ext > I_open
_BT_M, _BT_DX, _BT_DO, _BT_IX, _BT_IO = 9, 6, 5, 2, 1


def _wfa_forward(p: str, t: str, x: int, o: int, e: int, start: str, forced: str, free_end: str):
    """(score, operations) by the plain WFA with greedy extension: wavefronts
    from `start` / `forced` (as in wavefronts()), ended in M at (m, n), or
    -- free_end "I"/"D" -- in that gap at a discount of o (a trailing run
    that continues a gap opened after the segment), the lower cost winning
    (M on ties); then the backtrace of oracle/wfa_oracle.c (wf_backtrace:
    the highest piggyback value among the sources, M runs emitted from the
    pre-extension offset, the border reached with v or h at 0 finished by
    D and I runs)."""
    m, n = len(p), len(t)
    k_end = n - m
    smax = (m + n) * max(x, o + e) + 2 * (o + e)
    M, Mp, I, D = wavefronts(p, t, x, o, e, smax, start=start, forced=forced)
    best = None  # (cost, score, component)
    for s in range(smax + 1):
        if best is not None and s - (o if free_end != "M" else 0) > best[0]:
            break
        if M.get(s, {}).get(k_end, NULL) >= n and (best is None or s < best[0]):
            best = (s, s, "M")
        if free_end in ("I", "D"):
            g = (I if free_end == "I" else D).get(s, {})
            if g.get(k_end, NULL) == n and (best is None or s - o < best[0]):
                best = (s - o, s, free_end)
    if best is None:
        return None, None
    cost, s_end, state = best
    comp = {"M": M, "I": I, "D": D}[state]

    def src(w, s, k, delta, code):
        if s < 0 or k not in w.get(s, {}):
            return NULL
        return (w[s][k] + delta) * 16 + code

    ops = []
    s, k = s_end, k_end
    off = comp[s_end][k_end]
    v, h = off - k, off
    while v > 0 and h > 0 and s > 0:
        io = src(M, s - o - e, k - 1, 1, _BT_IO)
        ix = src(I, s - e, k - 1, 1, _BT_IX)
        dop = src(M, s - o - e, k + 1, 0, _BT_DO)
        dx = src(D, s - e, k + 1, 0, _BT_DX)
        # a forced first gap opens from the empty origin
        if forced == "I" and s == o + e and k == 1:
            io = max(io, 1 * 16 + _BT_IO)
        if forced == "D" and s == o + e and k == -1:
            dop = max(dop, 0 * 16 + _BT_DO)
        if state == "M":
            best_src = max(src(M, s - x, k, 1, _BT_M), io, ix, dop, dx)
        elif state == "I":
            best_src = max(io, ix)
        else:
            best_src = max(dop, dx)
        if best_src < 0:
            raise AssertionError("backtrace found no source")
        if state == "M":
            moff = best_src // 16
            ops.extend("M" * (off - moff))
            off = moff
            v, h = off - k, off
            if v <= 0 or h <= 0:
                break
        code = best_src % 16
        if code == _BT_M:
            s, state = s - x, "M"
            ops.append("X")
            off -= 1
        elif code in (_BT_IO, _BT_IX):
            s, state = (s - o - e, "M") if code == _BT_IO else (s - e, "I")
            ops.append("I")
            k -= 1
            off -= 1
        else:
            s, state = (s - o - e, "M") if code == _BT_DO else (s - e, "D")
            ops.append("D")
            k += 1
        v, h = off - k, off
    if v > 0 and h > 0:
        nm = min(v, h)
        ops.extend("M" * nm)
        v, h = v - nm, h - nm
    ops.extend("D" * max(v, 0))
    ops.extend("I" * max(h, 0))
    return cost, "".join(reversed(ops))


def wfa_segment(p: str, t: str, x: int, o: int, e: int, begin: str = "M", end: str = "M"):
    """(score, operations) of one segment with components by the plain WFA.
    A segment free at its end runs forward from `begin`.  One that must end
    in a gap runs on the reversed sequences instead, forced to begin with
    that gap (greedy extension forward could run an M run past the cell the
    closing gap has to leave from; a constraint at the start of the greedy
    direction costs nothing), a gap it continues becoming a free trailing
    run; its operations are then read backwards."""
    if not p and not t:
        return 0, ""
    if end == "M":
        return _wfa_forward(p, t, x, o, e, begin, "M", "M")
    cost, ops = _wfa_forward(p[::-1], t[::-1], x, o, e, "M", end, begin)
    return cost, None if ops is None else ops[::-1]


def bialign(p: str, t: str, x: int, o: int, e: int, begin: str = "M", end: str = "M", base_score: int = 0,
            ring: bool = False) -> str:
    """Operations of a bidirectional alignment: split at the breakpoint
    until a segment's score is at most base_score (default two of the
    dearest single edits) or a cut makes no progress, then the plain WFA of
    the segment (wfa_segment), the pieces concatenated in order.  ring:
    cut by the two-ring crossing search (crossing_split) instead of the
    full intersection search (split)."""
    if not p and not t:
        return ""
    base = base_score or 2 * max(x, o + e)
    total, left, right = (crossing_split if ring else split)(p, t, x, o, e, begin, end)
    if total is None:
        raise AssertionError("no breakpoint")
    whole = len(p) + len(t)
    if total <= base or len(left[0]) + len(left[1]) in (0, whole) or len(right[0]) + len(right[1]) in (0, whole):
        return wfa_segment(p, t, x, o, e, begin, end)[1]
    return (bialign(left[0], left[1], x, o, e, left[2], left[3], base, ring)
            + bialign(right[0], right[1], x, o, e, right[2], right[3], base, ring))


def ops_cost(ops: str, p: str, t: str, x: int, o: int, e: int, begin: str = "M", end: str = "M"):
    """Cost of an operation string for a segment with components, or None
    if it does not turn p into t or breaks the end component."""
    i = j = 0
    cost = 0
    prev = begin  # a leading run of the begin gap continues it
    for c in ops:
        if c in "MX":
            if i >= len(p) or j >= len(t) or (p[i] == t[j]) != (c == "M"):
                return None
            cost += 0 if c == "M" else x
            i, j = i + 1, j + 1
        elif c == "I":
            if j >= len(t):
                return None
            cost += e if prev == "I" else o + e
            j += 1
        elif c == "D":
            if i >= len(p):
                return None
            cost += e if prev == "D" else o + e
            i += 1
        else:
            return None
        prev = c if c in "ID" else "M"
    if i != len(p) or j != len(t):
        return None
    if end in "ID" and (not ops or ops[-1] != end) and not (not ops and begin == end):
        return None
    return cost


def _crossing_search(p: str, t: str, x: int, o: int, e: int, begin: str, end: str):
    """(total, component, k, h) of the ring-window crossing search (see
    crossing_total), or None."""
    m, n = len(p), len(t)
    mx = max(x, o + e)
    smax = (m + n) * mx + 2 * (o + e) + 2
    FM, FMp, FI, FD = wavefronts(p, t, x, o, e, smax, start=begin)
    RM, _, RI, RD = wavefronts(p[::-1], t[::-1], x, o, e, smax, forced=end)

    def check(sf, sr):
        found = None
        for comp, Fw, Rw, cut in (("M", FM, RM, 0), ("I", FI, RI, o), ("D", FD, RD, o)):
            for k in sorted(Fw.get(sf, {})):
                hf = Fw[sf][k]
                hr = Rw.get(sr, {}).get((n - m) - k)
                if hr is not None and hf + hr >= n:
                    h = max(FMp[sf][k], n - hr) if comp == "M" else hf
                    if found is None or sf + sr - cut < found[0]:
                        found = (sf + sr - cut, comp, k, h)
        return found

    sf = sr = 0
    best = check(0, 0)
    while sf <= smax:
        if best is not None and sf + sr - 2 * mx - o > best[0]:
            break
        if sf <= sr:
            sf += 1
            pairs = [(sf, s2) for s2 in range(max(0, sr - mx), sr + 1)]
        else:
            sr += 1
            pairs = [(s1, sr) for s1 in range(max(0, sf - mx), sf + 1)]
        for a, b in pairs:
            c = check(a, b)
            if c is not None and (best is None or c[0] < best[0]):
                best = c
    return best


def crossing_total(p: str, t: str, x: int, o: int, e: int, begin: str = "M", end: str = "M"):
    """Lowest total found the way a two-ring kernel could search: forward and
    reverse advance in turns (the lower score first, forward on ties), and
    each new wavefront is checked only against the other direction's last
    max(x, o + e) + 1 scores.  Overlap is offsets crossing on a diagonal
    (forward + reverse >= n; in I or D the total counts one opening); the
    lowest total wins (the first found on ties: M before I before D,
    diagonals ascending).  The search stops once no unchecked pair can beat
    the best total.  It finds the optimum of segments free at their end and
    of every segment the recursion produces (pinned by the tests).  For an
    arbitrary segment forced to end in a gap it can miss it: the forward
    greedy run passes the cell the closing gap leaves from, and only an
    outer split, outside the window, meets."""
    found = _crossing_search(p, t, x, o, e, begin, end)
    return None if found is None else found[0]


def crossing_split(p: str, t: str, x: int, o: int, e: int, begin: str = "M", end: str = "M"):
    """split() driven by the ring-window crossing search: (T, left, right).
    An M crossing is cut at max(forward pre-extension offset, n - reverse
    offset) -- inside the forward run, where the reverse side has already
    reached -- and a gap crossing where the forward gap cell is."""
    found = _crossing_search(p, t, x, o, e, begin, end)
    if found is None:
        return None, None, None
    T, comp, k, h = found
    v = h - k
    return T, (p[:v], t[:h], begin, comp), (p[v:], t[h:], comp, end)
