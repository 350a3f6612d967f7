"""CPU tests of the host side: the C-ABI library loads and exports every
symbol include/*.h declares, the sequences.txt format, the seeded generator,
CIGAR rendering and the drop-in command lines' argument handling.  No compute
call reaches a GPU here."""
import glob
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(tsu_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    import ctypes

    import tsunami_pact_b200 as T

    names = _declared_functions()
    assert len(names) >= 15, names
    L = ctypes.CDLL(T.lib_path())
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_status_strings():
    T = pytest.importorskip("tsunami_pact_b200")
    L = T.lib()
    assert L.tsu_status_str(0) == b"ok"
    assert L.tsu_status_str(5) == b"output buffer too small"


def test_render_runs():
    import tsunami_pact_b200 as T

    runs = np.array([(3 << 4) | 0, (1 << 4) | 8, (2 << 4) | 1, (3 << 4) | 2], np.uint32)
    assert T.runs_to_ops(runs) == "MMMXIIDDD"
    assert T.runs_to_string(runs) == "3M1X2I3D"


def test_generator_deterministic_and_edit_counts():
    import tsunami_pact_b200 as T

    lengths = np.array([150, 1000, 0, 1, 999], np.int32)
    rates = np.array([0.02, 0.05, 0.1, 1.0, 0.15])
    a = T.gen_batch(12345, lengths, rates)
    b = T.gen_batch(12345, lengths, rates, threads=1)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    pbuf, poff, plen, tbuf, toff, tlen = a
    assert np.array_equal(plen, lengths) and np.array_equal(tlen, lengths)
    for i in range(len(lengths)):
        p = bytes(pbuf[poff[i]:poff[i] + plen[i]])
        assert set(p) <= set(b"ACGT")
    # pair i depends only on (seed, index): generating from index 1 matches
    c = T.gen_batch(12345, lengths[1:], rates[1:], first=1)
    assert bytes(c[0][:1000]) == bytes(pbuf[150:1150])


def test_generator_edits_are_exact(oracle):
    """E = round(L*rate) edits with equal insertion/deletion counts: the
    optimal score never exceeds the cost of those edits."""
    import tsunami_pact_b200 as T

    L, rate = 300, 0.05
    pbuf, poff, plen, tbuf, toff, tlen = T.gen_batch(7, np.full(20, L, np.int32), np.full(20, rate))
    E = round(L * rate)
    ni = E // 3
    ns = E - 2 * ni
    for i in range(20):
        p = bytes(pbuf[poff[i]:poff[i] + L])
        t = bytes(tbuf[toff[i]:toff[i] + L])
        s = oracle.gotoh(p, t)
        assert 0 < s <= ns * 4 + 2 * ni * 8


def test_sequences_file_roundtrip(tmp_path):
    import tsunami_pact_b200 as T

    pats = [b"ACGT", b"AAAAAAA", b"ANNA"]
    txts = [b"AGGT", b"AAAA", b"acgt"]
    path = str(tmp_path / "sequences.txt")
    T.write_sequences(path, pats, txts, 7, 2)
    text = open(path).read()
    assert text.startswith("3\n7\n2\nACGT\nAGGT\n")
    hdr, p2, t2 = T.read_sequences(path)
    assert hdr == (3, 7, 2)
    assert p2 == pats and t2 == txts


def test_reads_reference_style_file(tmp_path):
    """The reader takes whitespace-separated tokens like fscanf("%s")
    (wfa_gpu.cu:71-81), including a file without a trailing newline."""
    import tsunami_pact_b200 as T

    path = tmp_path / "s.txt"
    path.write_text("2 4 1\nACGT   AGGT\n\nTTTT\nTTTA")
    hdr, p, t = T.read_sequences(str(path))
    assert hdr == (2, 4, 1) and p == [b"ACGT", b"TTTT"] and t == [b"AGGT", b"TTTA"]


def test_cli_usage_and_missing_file():
    exe = os.path.join(ROOT, "tsunami_pact_b200", "bin", "wfa_gpu")
    r = subprocess.run([exe, "4", "6"], capture_output=True, text=True)
    assert r.returncode == 0  # wfa_gpu.cu:45-48 returns 0 on bad argc
    assert r.stdout.startswith("ERROR! Please specify in order: mismatch, gap_opening, gap_extension")
    r = subprocess.run([exe, "4", "6", "2", "/nonexistent/seq.txt", "21", "0"], capture_output=True, text=True)
    assert r.returncode == 1 and r.stdout == "ERROR: Cannot open file.\n"


def test_generate_dataset_cli(tmp_path):
    exe = os.path.join(ROOT, "tsunami_pact_b200", "bin", "generate_dataset")
    r = subprocess.run([exe, "2"], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 1 and "Required arguments" in r.stdout
    r = subprocess.run([exe, "5", "128", "2"], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 0
    lines = (tmp_path / "sequences.txt").read_text().split("\n")
    assert lines[:3] == ["5", "128", "2"]
    assert all(len(x) == 128 for x in lines[3:13])
    first = (tmp_path / "sequences.txt").read_text()
    subprocess.run([exe, "5", "128", "2"], check=True, cwd=tmp_path)
    assert (tmp_path / "sequences.txt").read_text() == first  # seeded: reproducible
    r = subprocess.run([exe, "3", "100", "5", "7", "sub"], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 0
    ls = (tmp_path / "sequences.txt").read_text().split("\n")
    for i in range(3):
        p, t = ls[3 + 2 * i], ls[4 + 2 * i]
        assert len(p) == len(t) == 100 and 0 < sum(a != b for a, b in zip(p, t)) <= 5


def test_no_gpu_fails_loudly():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import tsunami_pact_b200 as T

    with pytest.raises(T.AlignError):
        T.Aligner(4, 6, 2)


def test_dual_create_rejects_bad_penalties():
    """tsu_create_dual / tsu_server_create_dual check the second gap piece
    before touching a device."""
    import ctypes

    import tsunami_pact_b200 as T
    from tsunami_pact_b200._lib import Penalties2

    L = T.lib()
    h = ctypes.c_void_p()
    for pen in [(4, 6, 2, -1, 1), (4, 6, 2, 24, 0), (0, 6, 2, 24, 1), (4, 6, 2, 24, 1 << 21)]:
        p2 = Penalties2(*pen)
        assert L.tsu_create_dual(ctypes.byref(p2), None, ctypes.byref(h)) == 1, pen  # TSU_EINVAL
        assert L.tsu_server_create_dual(ctypes.byref(p2), None, ctypes.byref(h)) == 1, pen


def test_metric_create_rejects_bad_arguments():
    """tsu_create_metric / tsu_server_create_metric check the metric and its
    penalties before touching a device."""
    import ctypes

    import tsunami_pact_b200 as T

    L = T.lib()
    h = ctypes.c_void_p()
    bad = [(7, []), (-1, []), (1, [1]), (0, [1, 1]), (2, [0, 1]), (2, [1, 0]), (2, [1]), (3, [4, 6]),
           (3, [4, -1, 2]), (4, [4, 6, 2, 24]), (4, [4, 6, 2, -1, 1]), (3, [1 << 21, 6, 2])]
    for metric, pens in bad:
        arr = (ctypes.c_int32 * max(1, len(pens)))(*pens)
        ptr = ctypes.cast(arr, ctypes.c_void_p) if pens else None
        assert L.tsu_create_metric(metric, ptr, len(pens), None, ctypes.byref(h)) == 1, (metric, pens)
        assert L.tsu_server_create_metric(metric, ptr, len(pens), None, ctypes.byref(h)) == 1, (metric, pens)
    with pytest.raises(ValueError):
        T.Aligner(metric="levenshtein")
