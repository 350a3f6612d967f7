"""The bidirectional breakpoint rule (oracle/bidir_rule.py) finds the optimal
gap-affine score: the first total at which forward and reverse wavefronts
overlap -- M extension runs intersecting, or gap cells meeting exactly with
the opening counted once -- equals the Gotoh DP score."""
import random

from oracle import bidir_rule


def test_first_breakpoint_is_the_optimal_score(oracle):
    rng = random.Random(1)
    for it in range(1500):
        p = "".join(rng.choice("AC" if it % 2 else "ACGT") for _ in range(rng.randint(0, 40)))
        t = list(p)
        for _ in range(rng.randint(0, 10)):
            pos = rng.randint(0, max(0, len(t) - 1))
            r = rng.random()
            if r < 0.33 and t:
                t[pos] = rng.choice("ACGT")
            elif r < 0.66:
                t.insert(pos, rng.choice("ACGT"))
            elif t:
                del t[pos]
        t = "".join(t)
        pen = rng.choice([(4, 6, 2), (2, 3, 1), (3, 5, 2), (1, 1, 1), (5, 2, 3)])
        best = oracle.gotoh(p, t, *pen)
        total, where = bidir_rule.first_breakpoint(p, t, *pen, best + 2)
        assert total == best, (p, t, pen, best, total, where)


def _case(rng, it, maxlen=14, maxedits=5):
    p = "".join(rng.choice("AC" if it % 2 else "ACGT") for _ in range(rng.randint(0, maxlen)))
    t = list(p)
    for _ in range(rng.randint(0, maxedits)):
        pos = rng.randint(0, max(0, len(t) - 1))
        r = rng.random()
        if r < 0.33 and t:
            t[pos] = rng.choice("ACGT")
        elif r < 0.66:
            t.insert(pos, rng.choice("ACGT"))
        elif t:
            del t[pos]
    return p, "".join(t), rng.choice([(4, 6, 2), (2, 3, 1), (3, 5, 2), (1, 1, 1), (5, 2, 3)])


def test_segments_with_gap_components():
    """Segments that continue a gap from the left (begin I/D) or must end in
    one (end I/D), as a recursion on breakpoints produces them: the first
    overlap total equals the component-constrained Gotoh DP, for all nine
    begin/end pairs."""
    rng = random.Random(5)
    checked = 0
    for it in range(500):
        p, t, pen = _case(rng, it)
        if not p and not t:
            continue
        for a in "MID":
            for b in "MID":
                best = bidir_rule.gotoh_components(p, t, *pen, a, b)
                if best >= bidir_rule.INF:
                    continue
                total, where = bidir_rule.first_breakpoint(p, t, *pen, best + pen[1] + pen[2] + 2, a, b)
                assert total == best, (p, t, pen, a, b, best, total, where)
                checked += 1
    assert checked > 3000


def test_split_halves_are_optimal():
    """Cutting a segment at its breakpoint: the halves' optimal costs add up
    to the segment's, and where the score is positive both halves are
    usually cheaper (the cut sits near the middle in score).  The search
    must still try every split of a total: forward and reverse greedy
    passes can follow different optimal paths (a gap placed in different
    rows) that meet only at an outer split."""
    rng = random.Random(9)
    positive = cheaper = 0
    for it in range(300):
        p, t, pen = _case(rng, it)
        if not p and not t:
            continue
        for a in "MID":
            for b in "MID":
                best = bidir_rule.gotoh_components(p, t, *pen, a, b)
                if best >= bidir_rule.INF:
                    continue
                total, left, right = bidir_rule.split(p, t, *pen, a, b)
                assert total == best
                assert left[0] + right[0] == p and left[1] + right[1] == t
                assert left[2] == a and right[3] == b and left[3] == right[2]
                cl = bidir_rule.gotoh_components(left[0], left[1], *pen, left[2], left[3])
                cr = bidir_rule.gotoh_components(right[0], right[1], *pen, right[2], right[3])
                assert cl + cr == best, (p, t, pen, a, b, left, right, cl, cr)
                if best > 0:
                    positive += 1
                    cheaper += max(cl, cr) < best
    assert cheaper > positive // 2


def test_segment_wfa_with_components(oracle):
    """The base case of the recursion: the plain WFA of a segment with
    components reaches the component-constrained optimum with operations
    that cost exactly that, and for free ends (M, M) it is the C oracle
    byte for byte (same backtrace, same ties)."""
    rng = random.Random(4)
    for it in range(120):
        p, t, pen = _case(rng, it)
        if not p and not t:
            continue
        for a in "MID":
            for b in "MID":
                best = bidir_rule.gotoh_components(p, t, *pen, a, b)
                if best >= bidir_rule.INF:
                    continue
                score, ops = bidir_rule.wfa_segment(p, t, *pen, a, b)
                assert score == best and bidir_rule.ops_cost(ops, p, t, *pen, a, b) == best, (p, t, pen, a, b)
        assert bidir_rule.wfa_segment(p, t, *pen) == oracle.align(p, t, *pen)


def test_bidirectional_alignment_is_optimal(oracle):
    """Recursion on breakpoints down to segment WFAs: every operation string
    turns the pattern into the text at the Gotoh optimum (ties at a cut may
    resolve differently from the plain backtrace)."""
    rng = random.Random(12)
    identical = 0
    for it in range(40):
        L = rng.randint(0, 80)
        p = "".join(rng.choice("ACGT") for _ in range(L))
        t = list(p)
        for _ in range(int(L * rng.uniform(0, 0.2))):
            pos = rng.randint(0, max(0, len(t) - 1))
            r = rng.random()
            if r < 0.33 and t:
                t[pos] = rng.choice("ACGT")
            elif r < 0.66:
                t.insert(pos, rng.choice("ACGT"))
            elif t:
                del t[pos]
        t = "".join(t)
        pen = rng.choice([(4, 6, 2), (2, 3, 1), (3, 5, 2), (1, 1, 1), (5, 2, 3)])
        ops = bidir_rule.bialign(p, t, *pen)
        assert bidir_rule.ops_cost(ops, p, t, *pen) == oracle.gotoh(p, t, *pen), (p, t, pen, ops)
        assert oracle.cigar_cost(ops, p, t, *pen) == oracle.gotoh(p, t, *pen)
        identical += ops == oracle.align(p, t, *pen)[1]
    assert identical >= 20


def test_c_bialign_equals_the_model(oracle):
    """ora_bialign (oracle/wfa_oracle_bidir.c) is the Python recursion byte
    for byte, zero gap-open penalties included."""
    rng = random.Random(21)
    for it in range(60):
        L = rng.randint(0, 70)
        p = "".join(rng.choice("AC" if it % 4 == 0 else "ACGT") for _ in range(L))
        t = list(p)
        for _ in range(int(L * rng.uniform(0, 0.25))):
            pos = rng.randint(0, max(0, len(t) - 1))
            r = rng.random()
            if r < 0.33 and t:
                t[pos] = rng.choice("ACGT")
            elif r < 0.66:
                t.insert(pos, rng.choice("ACGT"))
            elif t:
                del t[pos]
        t = "".join(t)
        pen = rng.choice([(4, 6, 2), (2, 3, 1), (3, 5, 2), (1, 1, 1), (5, 2, 3), (4, 0, 2), (1, 10, 1), (9, 1, 1)])
        assert oracle.bialign(p, t, *pen) == bidir_rule.bialign(p, t, *pen), (p, t, pen)


def test_c_bialign_optimal_at_1kbp(oracle):
    """At the 1 kbp, 5 % shape every bidirectional CIGAR costs the optimum
    (about half of them differ from the one-direction backtrace)."""
    import numpy as np

    from tsunami_pact_b200 import gen_batch

    pb, po, pl, tb, to, tl = gen_batch(77, np.full(16, 1000, np.int32), np.full(16, 0.05))
    for i in range(16):
        p, t = bytes(pb[po[i]:po[i] + pl[i]]), bytes(tb[to[i]:to[i] + tl[i]])
        ops = oracle.bialign(p, t, 4, 6, 2)
        assert oracle.cigar_cost(ops, p, t, 4, 6, 2) == oracle.align(p, t, 4, 6, 2)[0]


def test_outer_split_needed():
    """'GC' against 'GTGAGC' at 5/2/3: the forward pass puts the gap after
    the first base, the reverse pass before it, so the first overlap is at
    an outer split (one side at score 0), not near the middle."""
    total, where = bidir_rule.first_breakpoint("GC", "GTGAGC", 5, 2, 3, 30)
    assert total == 14 == bidir_rule.gotoh_components("GC", "GTGAGC", 5, 2, 3)
    assert 0 in (where[1], where[2])


def test_ring_window_crossing_finds_free_end_optimum():
    """The overlap search a two-ring kernel could run (turns, a window of the
    last max(x, o+e) + 1 scores, offsets crossing) reaches the optimum of
    segments free at their end; for 'AG' against 'AG' forced to end in an
    insertion it does not (the outer split it needs lies outside the
    window)."""
    rng = random.Random(1)
    checked = 0
    for it in range(600):
        p, t, pen = _case(rng, it)
        if not p and not t:
            continue
        for a in "MID":
            best = bidir_rule.gotoh_components(p, t, *pen, a, "M")
            assert bidir_rule.crossing_total(p, t, *pen, a, "M") == best, (p, t, pen, a)
            checked += 1
    assert checked > 1500
    assert bidir_rule.crossing_total("AG", "AG", 1, 1, 1, "M", "I") != bidir_rule.gotoh_components(
        "AG", "AG", 1, 1, 1, "M", "I")


def test_ring_window_crossing_on_recursion_segments():
    """The segments a recursion on breakpoints actually produces -- a
    gap-ended left half comes from a gap meet, where the forward pass itself
    reached the corner in that gap -- all get their optimum from the
    ring-window crossing search."""
    rng = random.Random(7)
    count = 0

    def walk(p, t, pen, a, b):
        nonlocal count
        if not p and not t:
            return
        assert bidir_rule.crossing_total(p, t, *pen, a, b) == bidir_rule.gotoh_components(p, t, *pen, a, b)
        count += 1
        total, left, right = bidir_rule.split(p, t, *pen, a, b)
        whole = len(p) + len(t)
        if total <= 0 or len(left[0]) + len(left[1]) in (0, whole) or len(right[0]) + len(right[1]) in (0, whole):
            return
        walk(*left[:2], pen, *left[2:])
        walk(*right[:2], pen, *right[2:])

    for it in range(100):
        p, t, pen = _case(rng, it, maxlen=40, maxedits=10)
        walk(p, t, pen, "M", "M")
    assert count > 250


def test_crossing_split_recursion_is_optimal():
    """A recursion driven only by the ring-window crossing search: every cut
    yields halves whose optimal costs add up to the segment's optimum."""
    rng = random.Random(3)
    count = 0

    def walk(p, t, pen, a, b):
        nonlocal count
        if not p and not t:
            return
        best = bidir_rule.gotoh_components(p, t, *pen, a, b)
        total, left, right = bidir_rule.crossing_split(p, t, *pen, a, b)
        assert total == best
        assert left[0] + right[0] == p and left[1] + right[1] == t
        cl = bidir_rule.gotoh_components(left[0], left[1], *pen, left[2], left[3])
        cr = bidir_rule.gotoh_components(right[0], right[1], *pen, right[2], right[3])
        assert cl + cr == best, (p, t, pen, a, b, left, right, cl, cr)
        count += 1
        whole = len(p) + len(t)
        if total <= 0 or len(left[0]) + len(left[1]) in (0, whole) or len(right[0]) + len(right[1]) in (0, whole):
            return
        walk(*left[:2], pen, *left[2:])
        walk(*right[:2], pen, *right[2:])

    for it in range(120):
        p, t, pen = _case(rng, it, maxlen=40, maxedits=10)
        walk(p, t, pen, "M", "M")
    assert count > 300


def test_c_ring_bialign_equals_the_model_and_is_optimal(oracle):
    """ora_bialign_ring (the recursion a two-ring GPU kernel computes) is
    bidir_rule.bialign(ring=True) byte for byte, and optimal at the 1 kbp,
    5 % shape and on a 5 kbp, 15 % pair."""
    import numpy as np

    from tsunami_pact_b200 import gen_batch

    rng = random.Random(22)
    for it in range(50):
        p, t, pen = _case(rng, it, maxlen=60, maxedits=12)
        assert oracle.bialign(p, t, *pen, ring=True) == bidir_rule.bialign(p, t, *pen, ring=True), (p, t, pen)
    lengths = np.array([1000] * 12 + [5000], np.int32)
    pb, po, pl, tb, to, tl = gen_batch(79, lengths, np.array([0.05] * 12 + [0.15]))
    for i in range(len(lengths)):
        p, t = bytes(pb[po[i]:po[i] + pl[i]]), bytes(tb[to[i]:to[i] + tl[i]])
        ops = oracle.bialign(p, t, 4, 6, 2, ring=True)
        assert oracle.cigar_cost(ops, p, t, 4, 6, 2) == oracle.gotoh(p, t, 4, 6, 2)


def test_c_segment_equals_the_model(oracle):
    """ora_align_segment, the checker for segment components in a GPU CIGAR
    kernel, is bidir_rule.wfa_segment (cost and operations) for all nine
    begin/end pairs."""
    rng = random.Random(8)
    checked = 0
    for it in range(120):
        p, t, pen = _case(rng, it, maxlen=16, maxedits=6)
        for a in "MID":
            for b in "MID":
                if (p or t) and bidir_rule.gotoh_components(p, t, *pen, a, b) >= bidir_rule.INF:
                    continue
                assert oracle.align_segment(p, t, *pen, a, b) == bidir_rule.wfa_segment(p, t, *pen, a, b)
                checked += 1
    assert checked > 800
