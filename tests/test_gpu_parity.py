"""GPU parity: the CUDA engine (through its C ABI) against the CPU oracle.

Bar: bit-exact scores and byte-identical WFA2-style operation strings for
every pair, on the golden fixtures, on seeded random pairs with many penalty
sets, and on reduced versions of the benchmark shapes."""
import os
import random
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _check_same(aligner, oracle, pats, txts, pen=(4, 6, 2), threads=0):
    scores, ops = aligner.align(pats, txts)
    osc, oops = oracle.align_batch(pats, txts, *pen, threads=threads)
    bad = [i for i in range(len(pats)) if scores[i] != osc[i] or ops[i] != oops[i]]
    assert not bad, [(i, pats[i], txts[i], scores[i], osc[i], ops[i], oops[i]) for i in bad[:3]]
    return scores, ops


def _gen(seed, lengths, rates):
    import tsunami_pact_b200 as T

    pbuf, poff, plen, tbuf, toff, tlen = T.gen_batch(seed, np.asarray(lengths, np.int32), np.asarray(rates))
    pats = [bytes(pbuf[poff[i]:poff[i] + plen[i]]) for i in range(len(plen))]
    txts = [bytes(tbuf[toff[i]:toff[i] + tlen[i]]) for i in range(len(tlen))]
    return pats, txts


def test_kat(aligner_factory, kat_cases):
    for c in kat_cases:
        al = aligner_factory(tuple(c["pen"]))
        s, ops = al.align([c["p"]], [c["t"]])
        assert int(s[0]) == c["score"] and ops[0] == c["ops"], c


def test_regression_fixture(aligner_factory, regress_cases):
    by_pen = {}
    for c in regress_cases:
        by_pen.setdefault(tuple(c["pen"]), []).append(c)
    for pen, cases in by_pen.items():
        al = aligner_factory(pen)
        s, ops = al.align([c["p"] for c in cases], [c["t"] for c in cases])
        for i, c in enumerate(cases):
            assert int(s[i]) == c["score"] and ops[i] == c["ops"], (pen, c)


@pytest.mark.parametrize("pen", [(4, 6, 2), (1, 0, 1), (3, 5, 1), (7, 2, 3), (20, 1, 1), (2, 10, 1), (6, 4, 2),
                                 (5, 11, 3)])
def test_random_short(aligner_factory, oracle, pen):
    rng = random.Random(sum(pen) * 131)
    pats, txts = [], []
    for it in range(400):
        alpha = "ACGT" if it % 4 else "AC"
        m = rng.randint(0, 80)
        p = "".join(rng.choice(alpha) for _ in range(m))
        if it % 3:
            t = list(p)
            for _ in range(rng.randint(0, 10)):
                pos = rng.randint(0, max(0, len(t) - 1))
                r = rng.random()
                if r < 0.33 and t:
                    t[pos] = rng.choice(alpha)
                elif r < 0.66:
                    t.insert(pos, rng.choice(alpha))
                elif t:
                    del t[pos]
            t = "".join(t)
        else:
            t = "".join(rng.choice(alpha) for _ in range(rng.randint(0, 80)))
        pats.append(p)
        txts.append(t)
    _check_same(aligner_factory(pen), oracle, pats, txts, pen)


def test_c1_full(aligner_factory, oracle):
    """10,000 pairs of 150 bp at 2% (the CPU-runnable configuration), full size."""
    pats, txts = _gen(0x5453554E414D49 + 0, [150] * 10000, [0.02] * 10000)
    _check_same(aligner_factory(), oracle, pats, txts)


def test_c2_reduced(aligner_factory, oracle):
    pats, txts = _gen(0x5453554E414D49 + 1, [1000] * 3000, [0.05] * 3000)
    _check_same(aligner_factory(), oracle, pats, txts)


def test_c3_reduced(aligner_factory, oracle):
    pats, txts = _gen(0x5453554E414D49 + 2, [10000] * 6, [0.15] * 6)
    _check_same(aligner_factory(), oracle, pats, txts)


def test_c4_reduced_uneven(aligner_factory, oracle):
    rng = np.random.default_rng(4)
    n = 400
    lengths = np.exp(rng.uniform(np.log(100), np.log(4000), n)).astype(np.int32)
    rates = rng.uniform(0.01, 0.15, n)
    pats, txts = _gen(0x5453554E414D49 + 3, lengths, rates)
    _check_same(aligner_factory(), oracle, pats, txts)


def test_wide_wavefronts_global_ring(aligner_factory, oracle):
    """Pairs of 16-20 kbp whose wavefronts (up to ~40,000 diagonals) outgrow
    every shared ring (16,368 diagonals at most): 32-warp passes on the
    global ring, with bytes outside ACGT in one pair and one pair whose end
    diagonal lies ~16,000 from 0; scores and CIGARs equal the oracle's, with
    and without CIGARs."""
    rng = np.random.default_rng(16)
    lengths = rng.integers(16500, 20000, 4).astype(np.int32)
    pats, txts = _gen(0x5453554E414D49 + 16, lengths, [0.25, 0.2, 0.15, 0.3])
    p0 = bytearray(pats[0])
    for i in range(0, len(p0), 997):
        p0[i] = ord("N")
    pats[0] = bytes(p0)
    pats.append(pats[1][:3000])
    txts.append(txts[1])  # n - m > 13,000: the end diagonal far from 0
    al = aligner_factory()
    _check_same(al, oracle, pats, txts)
    assert "g32" in al.pass_log(), al.pass_log()
    scores, _ = oracle.align_batch(pats, txts, 4, 6, 2, cigar=False)
    got, _ = al.align(pats, txts, cigar=False)
    assert list(got) == list(scores)


def test_unequal_lengths_and_empty(aligner_factory, oracle):
    rng = random.Random(11)
    pats = ["", "", "A", "ACGT" * 50, "T" * 300, "ACGT" * 10]
    txts = ["", "ACGTACGT", "", "", "T" * 7, "ACGT" * 60]
    for _ in range(200):
        pats.append("".join(rng.choice("ACGT") for _ in range(rng.randint(0, 300))))
        txts.append("".join(rng.choice("ACGT") for _ in range(rng.randint(0, 300))))
    _check_same(aligner_factory(), oracle, pats, txts)


def test_byte_mode_mixed_batch(aligner_factory, oracle):
    """Pairs with bytes outside ACGT take the byte path; others stay packed."""
    rng = random.Random(5)
    pats, txts = [], []
    for i in range(300):
        alpha = "ACGTN" if i % 3 == 0 else ("acgtACGT" if i % 3 == 1 else "ACGT")
        p = "".join(rng.choice(alpha) for _ in range(rng.randint(0, 200)))
        t = list(p)
        for _ in range(rng.randint(0, 8)):
            if t:
                t[rng.randint(0, len(t) - 1)] = rng.choice(alpha)
        pats.append(p)
        txts.append("".join(t))
    _check_same(aligner_factory(), oracle, pats, txts)


def test_score_only_matches(aligner_factory):
    pats, txts = _gen(99, [700] * 500, [0.08] * 500)
    al = aligner_factory()
    s1, _ = al.align(pats, txts, cigar=True)
    s2, _ = al.align(pats, txts, cigar=False)
    assert np.array_equal(s1, s2)


def test_fixed_stride_api(aligner_factory, oracle):
    """Reference host layout (wfa_gpu.cu:75-81): fixed stride, equal lengths."""
    pats, txts = _gen(123, [512] * 800, [0.05] * 800)
    al = aligner_factory()
    s = al.align_fixed(b"".join(pats), b"".join(txts), len(pats), 512, 512)
    osc, _ = oracle.align_batch(pats, txts, cigar=False)
    assert np.array_equal(s, osc)


def test_retry_with_small_scratch(aligner_factory, oracle):
    """A tiny error hint forces every pair to outgrow the first pass's scratch;
    the retry passes must give identical results."""
    pats, txts = _gen(321, [2000] * 40 + [300] * 40, [0.12] * 80)
    al = aligner_factory(max_error_hint=0.0005)
    _check_same(al, oracle, pats, txts)
    assert al.timing()["retried_pairs"] > 0


def test_device_api(aligner_factory, oracle):
    torch = pytest.importorskip("torch")
    import tsunami_pact_b200 as T

    pbuf, poff, plen, tbuf, toff, tlen = T.gen_batch(77, np.full(600, 400, np.int32), np.full(600, 0.06))
    dev = "cuda:0"
    tp = torch.from_numpy(pbuf).to(dev)
    tt = torch.from_numpy(tbuf).to(dev)
    a = [torch.from_numpy(x).to(dev) for x in (poff, plen, toff, tlen)]
    scores = torch.zeros(600, dtype=torch.int32, device=dev)
    runs = torch.zeros(600 * 200, dtype=torch.int32, device=dev)
    coff = torch.zeros(601, dtype=torch.int64, device=dev)
    al = aligner_factory()
    nr = al.align_device(tp, a[0], a[1], tt, a[2], a[3], scores, runs, coff)
    pats = [bytes(pbuf[poff[i]:poff[i] + plen[i]]) for i in range(600)]
    txts = [bytes(tbuf[toff[i]:toff[i] + tlen[i]]) for i in range(600)]
    osc, oops = oracle.align_batch(pats, txts)
    assert np.array_equal(scores.cpu().numpy(), osc)
    r = runs[:nr].cpu().numpy().view(np.uint32)
    c = coff.cpu().numpy()
    for i in range(600):
        assert T.runs_to_ops(r[c[i]:c[i + 1]]) == oops[i]


def test_chunked_host_pipeline(aligner_factory, oracle):
    """A batch large enough for the multi-chunk host pipeline (several chunks
    uploaded, aligned and downloaded on three streams) gives the same scores
    and CIGARs as the single-launch device path, and the oracle's on a sample."""
    torch = pytest.importorskip("torch")
    import tsunami_pact_b200 as T

    n = 300_000
    rng = np.random.default_rng(8)
    lengths = rng.integers(60, 160, n).astype(np.int32)
    rates = rng.uniform(0.0, 0.06, n)
    pbuf, poff, plen, tbuf, toff, tlen = T.gen_batch(555, lengths, rates)
    al = aligner_factory()
    scores, coff, runs = al.align_arrays(pbuf, poff, plen, tbuf, toff, tlen)
    dev = "cuda:0"
    d = [torch.from_numpy(x).to(dev) for x in (pbuf, poff, plen, tbuf, toff, tlen)]
    dsc = torch.zeros(n, dtype=torch.int32, device=dev)
    druns = torch.zeros(int(coff[-1]) + 16, dtype=torch.int32, device=dev)
    doff = torch.zeros(n + 1, dtype=torch.int64, device=dev)
    nr = al.align_device(d[0], d[1], d[2], d[3], d[4], d[5], dsc, druns, doff)
    assert np.array_equal(scores, dsc.cpu().numpy())
    assert nr == int(coff[-1]) and np.array_equal(coff, doff.cpu().numpy())
    assert np.array_equal(runs, druns[:nr].cpu().numpy().view(np.uint32))
    idx = rng.choice(n, 2000, replace=False)
    pats = [bytes(pbuf[poff[i]:poff[i] + plen[i]]) for i in idx]
    txts = [bytes(tbuf[toff[i]:toff[i] + tlen[i]]) for i in idx]
    osc, oops = oracle.align_batch(pats, txts)
    for j, i in enumerate(idx):
        assert scores[i] == osc[j] and T.runs_to_ops(runs[coff[i]:coff[i + 1]]) == oops[j]


def test_one_warp_flag_same_results(aligner_factory):
    """TSU_ONE_WARP (the plain baseline: one warp per pair in every pass, no
    warp groups, no longest-first order) gives the same scores and CIGARs as
    the default scheduling on a mixed batch with long pairs."""
    torch = pytest.importorskip("torch")
    import tsunami_pact_b200 as T

    lengths = np.array([150] * 300 + [1000] * 100 + [3000] * 8 + [6000] * 2, np.int32)
    rates = np.array([0.02] * 300 + [0.08] * 100 + [0.15] * 8 + [0.12] * 2)
    pbuf, poff, plen, tbuf, toff, tlen = T.gen_batch(31, lengths, rates)
    dev = "cuda:0"
    d = [torch.from_numpy(x).to(dev) for x in (pbuf, poff, plen, tbuf, toff, tlen)]
    al = aligner_factory()
    outs = []
    for one in (False, True):
        sc = torch.zeros(len(plen), dtype=torch.int32, device=dev)
        runs = torch.zeros(2_000_000, dtype=torch.int32, device=dev)
        off = torch.zeros(len(plen) + 1, dtype=torch.int64, device=dev)
        nr = al.align_device(d[0], d[1], d[2], d[3], d[4], d[5], sc, runs, off, one_warp=one)
        outs.append((sc.cpu().numpy(), off.cpu().numpy(), runs[:nr].cpu().numpy()))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1]) and np.array_equal(outs[0][2], outs[1][2])


def test_empty_batch(aligner_factory):
    al = aligner_factory()
    s, ops = al.align([], [])
    assert len(s) == 0 and ops == []


def test_cli_check(tmp_path):
    """generate_dataset + wfa_gpu with check=1: the reference's artifact flow
    (run_h100-a100.sh) with the oracle plugged in as the CPU checker."""
    bindir = os.path.join(ROOT, "tsunami_pact_b200", "bin")
    subprocess.run([os.path.join(bindir, "generate_dataset"), "3000", "512", "2"], check=True, cwd=tmp_path)
    env = dict(os.environ, TSU_CHECK_LIB=os.path.join(ROOT, "oracle", "liboracle.so"),
               TSU_CIGAR_OUT=str(tmp_path / "cig.tsv"))
    r = subprocess.run([os.path.join(bindir, "wfa_gpu"), "4", "6", "2", "sequences.txt", "42", "1"],
                       capture_output=True, text=True, cwd=tmp_path, env=env)
    assert r.returncode == 0, r.stderr
    assert "GPU Time: " in r.stdout and "Estimated GCUPS GPU: : " in r.stdout
    assert "CPU Time: " in r.stdout and "Estimated GCUPS SW: " in r.stdout
    assert "|ALIGNEMENT FINISHED CORRECTLY|" in r.stdout, r.stdout
    rows = (tmp_path / "cig.tsv").read_text().strip().split("\n")
    assert len(rows) == 3000


def test_every_starting_rung_same_results(aligner_factory, oracle):
    """tsu_set_band_start: whatever rung a band starts at (shared ring with
    1-32 warps per pair, global ring with 1-32), pairs that outgrow it are
    retried and the results are the oracle's."""
    import ctypes

    import tsunami_pact_b200 as T

    rng = np.random.default_rng(21)
    n = 120
    lengths = np.exp(rng.uniform(np.log(100), np.log(6000), n)).astype(np.int32)
    rates = rng.uniform(0.01, 0.15, n)
    pats, txts = _gen(0x5453554E414D49 + 9, lengths, rates)
    osc, oops = oracle.align_batch(pats, txts, 4, 6, 2)
    L = T.lib()
    L.tsu_set_band_start.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    with T.Aligner(4, 6, 2) as al:
        assert L.tsu_set_band_start(al._h, 6, 0, 1) != 0  # no band 6
        assert L.tsu_set_band_start(al._h, 0, 0, 3) != 0  # no 3-warp groups
        assert L.tsu_set_band_start(al._h, 0, 0, 64) != 0  # no 64-warp groups
        for mode, gw in [(0, 1), (0, 2), (0, 4), (0, 8), (0, 16), (0, 32), (1, 1), (1, 8), (1, 16), (1, 32)]:
            for band in range(6):
                assert L.tsu_set_band_start(al._h, band, mode, gw) == 0
            scores, ops = al.align(pats, txts)
            assert list(scores) == list(osc), (mode, gw)
            assert ops == oops, (mode, gw)
