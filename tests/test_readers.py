"""Input readers on the CPU: sequences.txt (parallel preads and chunked
tokenization, checked on files large enough to be split) and FASTA/FASTQ
pair files (wrapped FASTA, FASTQ, mixed, malformed)."""
import os
import random

import numpy as np
import pytest

import tsunami_pact_b200 as T


def _rand_pairs(rng, n, lo, hi):
    pats, txts = [], []
    for _ in range(n):
        L = rng.randint(lo, hi)
        p = "".join(rng.choice("ACGT") for _ in range(L))
        t = list(p)
        for _ in range(rng.randint(0, max(1, L // 20))):
            if t:
                t[rng.randrange(len(t))] = rng.choice("ACGTN")
        pats.append(p.encode())
        txts.append("".join(t).encode())
    return pats, txts


def test_large_sequences_file_roundtrip(tmp_path):
    """A 20+ MB file (split into parallel chunks at arbitrary byte offsets)
    reads back pair for pair."""
    lengths = np.random.default_rng(1).integers(200, 1200, 30000).astype(np.int32)
    pb, po, pl, tb, to, tl = T.gen_batch(99, lengths, np.full(lengths.size, 0.05))
    pats = [bytes(pb[po[i]:po[i] + pl[i]]) for i in range(lengths.size)]
    txts = [bytes(tb[to[i]:to[i] + tl[i]]) for i in range(lengths.size)]
    path = str(tmp_path / "big.txt")
    T.write_sequences(path, pats, txts, 1200, 5)
    assert os.path.getsize(path) > 8 << 20
    hdr, p2, t2 = T.read_sequences(path)
    assert hdr == (lengths.size, 1200, 5)
    assert p2 == pats and t2 == txts


def test_whitespace_variants_and_truncation(tmp_path):
    rng = random.Random(3)
    pats, txts = _rand_pairs(rng, 50, 0, 40)
    pats = [p or b"A" for p in pats]
    txts = [t or b"C" for t in txts]
    body = "".join(f"{p.decode()}\r\n  {t.decode()}\t\n" for p, t in zip(pats, txts))
    path = tmp_path / "ws.txt"
    path.write_text(f"  {len(pats)}\r\n40\n3\n{body}extra tokens are ignored\n")
    hdr, p2, t2 = T.read_sequences(str(path))
    assert hdr == (50, 40, 3) and p2 == pats and t2 == txts
    path.write_text(f"{len(pats) + 1}\n40\n3\n{body}")  # one pair short
    with pytest.raises(T.AlignError):
        T.read_sequences(str(path))
    path.write_text("x\n1\n1\nA\nC\n")  # bad header
    with pytest.raises(T.AlignError):
        T.read_sequences(str(path))


def _fasta(seqs, wrap=60):
    out = []
    for i, s in enumerate(seqs):
        out.append(f">seq{i} description\n")
        s = s.decode()
        for k in range(0, len(s), wrap):
            out.append(s[k:k + wrap] + "\n")
        if not s:
            out.append("\n")
    return "".join(out)


def _fastq(seqs):
    return "".join(f"@r{i}\n{s.decode()}\n+\n{'I' * len(s)}\n" for i, s in enumerate(seqs))


def test_fasta_fastq_pairs(tmp_path):
    rng = random.Random(5)
    pats, txts = _rand_pairs(rng, 200, 1, 500)
    fa, fq = tmp_path / "p.fa", tmp_path / "t.fq"
    fa.write_text(_fasta(pats, wrap=rng.choice([50, 60, 80])))
    fq.write_text(_fastq(txts))
    hdr, p2, t2 = T.read_pairs(str(fa), str(fq))
    assert p2 == pats and t2 == txts
    assert hdr[0] == 200 and hdr[1] == max(max(map(len, pats)), max(map(len, txts)))
    # both FASTA, CRLF line ends
    fb = tmp_path / "t.fa"
    fb.write_text(_fasta(txts, wrap=70).replace("\n", "\r\n"))
    _, p3, t3 = T.read_pairs(str(fa), str(fb))
    assert p3 == pats and t3 == txts


def test_large_fasta_pairs(tmp_path):
    """Files past the parallel threshold (record starts found in chunks)."""
    lengths = np.random.default_rng(2).integers(500, 3000, 6000).astype(np.int32)
    pb, po, pl, tb, to, tl = T.gen_batch(7, lengths, np.full(lengths.size, 0.1))
    pats = [bytes(pb[po[i]:po[i] + pl[i]]) for i in range(lengths.size)]
    txts = [bytes(tb[to[i]:to[i] + tl[i]]) for i in range(lengths.size)]
    fa, fb = tmp_path / "p.fa", tmp_path / "t.fa"
    fa.write_text(_fasta(pats))
    fb.write_text(_fasta(txts))
    assert os.path.getsize(fa) > 8 << 20
    _, p2, t2 = T.read_pairs(str(fa), str(fb))
    assert p2 == pats and t2 == txts


def test_pair_files_rejected(tmp_path):
    a, b = tmp_path / "a.fa", tmp_path / "b.fa"
    a.write_text(">x\nACGT\n>y\nAC\n")
    b.write_text(">x\nACGT\n")
    with pytest.raises(T.AlignError):  # record counts differ
        T.read_pairs(str(a), str(b))
    b.write_text("ACGT\n")  # no header
    with pytest.raises(T.AlignError):
        T.read_pairs(str(a), str(b))
    b.write_text("@x\nACGT\nIIII\n@y\nAC\n+\nII\n")  # FASTQ without '+'
    with pytest.raises(T.AlignError):
        T.read_pairs(str(a), str(b))
    with pytest.raises(T.AlignError):
        T.read_pairs(str(a), str(tmp_path / "missing.fa"))


@pytest.mark.parametrize("workload,seed_first", [("c1", 0), ("c2", 5), ("c3", 0), ("c4", 123), ("c5", 40)])
def test_oracle_generator_matches_engine(oracle, workload, seed_first):
    """bench.py's CPU reference arm generates its pairs with the oracle's
    ora_gen_batch so that it never loads the engine library: the bytes must
    equal tsu_gen_batch's for the same seed, first index and shapes."""
    from tsunami_pact_b200 import datasets

    lengths, rates, seed = datasets.shape(workload, 300 if workload != "c3" else 20)
    a = T.gen_batch(seed, lengths, rates, first=seed_first)
    b = oracle.gen_batch(seed, lengths, rates, first=seed_first)
    for x, y in zip(a, b):
        assert x.dtype == y.dtype and np.array_equal(x, y)
