"""GPU parity across combinations of the engine's options: penalty model
(gap-affine, dual gap-affine, edit, indel), free ends, low-memory mode and the
starting rung, each combination on a small seeded batch against the matching
oracle.  Bar: bit-exact scores and byte-identical operation strings."""
import ctypes
import itertools
import random

import pytest

pytestmark = pytest.mark.gpu

MODELS = ["affine", "dual", "edit", "indel"]
FREES = [(0, 0, 0, 0), (25, 25, 25, 25)]
LOWMEM = [0, 6]
RUNGS = [(0, 1), (0, 8), (1, 4)]


def _batch(seed):
    rng = random.Random(seed)
    pats, txts = [], []
    for _ in range(40):
        core = "".join(rng.choice("ACGT") for _ in range(rng.randint(0, 900)))
        t = list(core)
        for _ in range(int(len(core) * rng.uniform(0, 0.15))):
            pos = rng.randint(0, max(0, len(t) - 1))
            r = rng.random()
            if r < 0.33 and t:
                t[pos] = rng.choice("ACGT")
            elif r < 0.66:
                t.insert(pos, rng.choice("ACGT"))
            elif t:
                del t[pos]
        fl = lambda: "".join(rng.choice("ACGT") for _ in range(rng.randint(0, 30)))
        pats.append(fl() + core + fl())
        txts.append(fl() + "".join(t) + fl())
    return pats, txts


def _aligner(T, model):
    if model == "affine":
        return T.Aligner(4, 6, 2)
    if model == "dual":
        return T.Aligner(4, 6, 2, gap_opening2=24, gap_extension2=1)
    return T.Aligner(metric=model)


def _expected(oracle, model, pats, txts, free):
    if model == "affine":
        return oracle.align_batch_ends_free(pats, txts, free)
    if model == "dual":
        return oracle.align_batch2_ends_free(pats, txts, free)
    x, e = (1, 1) if model == "edit" else (3, 1)
    return oracle.align_batch_linear_ends_free(pats, txts, free, x, e)


@pytest.mark.parametrize("model", MODELS)
def test_feature_matrix(oracle, model):
    import tsunami_pact_b200 as T

    L = T.lib()
    L.tsu_set_band_start.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    pats, txts = _batch(hash(model) & 0xFFFF)
    with _aligner(T, model) as al:
        for free, lowmem, rung in itertools.product(FREES, LOWMEM, RUNGS):
            al.set_ends_free(*free)
            al.set_low_memory(lowmem)
            for band in range(6):
                assert L.tsu_set_band_start(al._h, band, *rung) == 0
            s, ops = al.align(pats, txts)
            es, eops = _expected(oracle, model, pats, txts, free)
            assert list(s) == list(es), (model, free, lowmem, rung)
            assert ops == eops, (model, free, lowmem, rung)
