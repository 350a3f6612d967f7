"""The autotuner's table format (tsunami_pact_b200/tune.py): the committed
tsu_tuning.h parses to one valid rung per length band, and rendering then
parsing a table gives it back.  The tuning run itself needs a GPU
(python -m tsunami_pact_b200.tune)."""
import os

from tsunami_pact_b200 import tune

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "tsunami_pact_b200", "csrc", "tsu_tuning.h")


def test_committed_table_is_valid():
    with open(HEADER) as f:
        text = f.read()
    table = tune.parse_header(text)
    assert len(table) == len(tune.BANDS) == 6
    for mode, warps in table:
        assert mode in (0, 1) and warps in (1, 2, 4, 8, 16)
    assert "TSU_TUNING_SOURCE" in text


def test_render_parse_round_trip():
    table = [(0, 1), (0, 2), (0, 4), (0, 16), (1, 8), (1, 16)]
    times = [{"s1": 1.0, "g8": 2.5}] * 6
    text = tune.render_header(table, "test", times)
    assert tune.parse_header(text) == table
    assert '#define TSU_TUNING_SOURCE "test"' in text


def test_band_workloads_stay_in_band():
    import numpy as np

    from tsunami_pact_b200 import datasets  # noqa: F401  (package import only)

    for b, (lo, hi, _) in enumerate(tune.BANDS):
        rng = np.random.Generator(np.random.PCG64(tune.SEED + b))
        L = np.exp(rng.uniform(np.log(lo), np.log(hi - 1), 1000)).astype(np.int32)
        assert L.min() >= lo - 1 and L.max() < hi
