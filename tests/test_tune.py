"""The autotuner's table format (tsunami_pact_b200/tune.py): the committed
tsu_tuning.h parses to one valid rung per length band, and rendering then
parsing a table gives it back.  The tuning run itself needs a GPU
(python -m tsunami_pact_b200.tune)."""
import os

from tsunami_pact_b200 import tune

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "tsunami_pact_b200", "csrc", "tsu_tuning.h")
HEADER_DUAL = os.path.join(ROOT, "tsunami_pact_b200", "csrc", "tsu_tuning_dual.h")


def test_committed_table_is_valid():
    with open(HEADER) as f:
        text = f.read()
    table = tune.parse_header(text)
    assert len(table) == tune.N_BANDS == 6
    for mode, warps in table:
        assert mode in (0, 1) and warps in (1, 2, 4, 8, 16, 32)
    assert "TSU_TUNING_SOURCE" in text


def test_render_parse_round_trip():
    table = [(0, 1), (0, 2), (0, 4), (0, 16), (1, 8), (1, 16)]
    times = [{"s1": 1.0, "g8": 2.5}] * 6
    text = tune.render_header(table, "test", times)
    assert tune.parse_header(text) == table
    assert '#define TSU_TUNING_SOURCE "test"' in text


def test_length_band_matches_engine():
    import numpy as np

    L = np.array([0, 1023, 1024, 2047, 2048, 4095, 4096, 8191, 8192, 16383, 16384, 50000])
    assert list(tune.length_band(L)) == [0, 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5]


def test_committed_dual_table_is_valid():
    with open(HEADER_DUAL) as f:
        text = f.read()
    table = tune.parse_header(text, dual=True)
    assert len(table) == tune.N_BANDS
    for mode, warps in table:
        assert mode in (0, 1) and warps in (1, 2, 4, 8, 16, 32)
    assert "TSU_TUNING_DUAL_SOURCE" in text
    table2 = [(0, 8), (0, 16), (0, 16), (1, 16), (1, 32), (1, 32)]
    text2 = tune.render_header(table2, "t", None, dual=True)
    assert tune.parse_header(text2, dual=True) == table2 and "TSU_BAND_START_DUAL" in text2
