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
