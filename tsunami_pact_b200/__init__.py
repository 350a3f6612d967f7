"""B200-native gap-affine WaveFront Alignment (WFA) engine.

Python mirror of the reference's interface for this path (the ``wfa_gpu``
host driver, wfa_gpu.cu:43-188): penalties ``mismatch / gap_opening /
gap_extension``, a batch of pattern/text pairs (``sequences.txt`` format,
generate_dataset.cpp:39-41,68-69) in, one score per pair out -- plus the
WFA2-lib-style CIGAR the reference's check computes (wfa_gpu.cu:164).

Everything goes through the C ABI of ``libtsunami_b200.so`` (built in-tree
for sm_100a, see ``include/tsunami_b200.h``).  There is no CPU fallback: if
the library is missing or CUDA is unavailable the calls raise.
"""
from ._lib import (  # noqa: F401
    Aligner,
    AlignError,
    Server,
    TSU_BIDIRECTIONAL,
    TSU_SCORE_ONLY,
    build,
    gen_batch,
    lib,
    lib_path,
    read_pairs,
    read_sequences,
    runs_to_ops,
    runs_to_string,
    write_sequences,
)

__all__ = [
    "Aligner",
    "AlignError",
    "Server",
    "TSU_BIDIRECTIONAL",
    "TSU_SCORE_ONLY",
    "build",
    "gen_batch",
    "lib",
    "lib_path",
    "read_pairs",
    "read_sequences",
    "runs_to_ops",
    "runs_to_string",
    "write_sequences",
]
