import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: longer CPU test")


@pytest.fixture(scope="session")
def kat_cases():
    with open(os.path.join(GOLDEN, "kat.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def regress_cases():
    with open(os.path.join(GOLDEN, "regress.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O

    O.lib()
    return O


@pytest.fixture(scope="session")
def aligner_factory():
    """Contexts per penalty set, created on first use (GPU tests only)."""
    import tsunami_pact_b200 as T

    cache = {}

    def get(pen=(4, 6, 2), **kw):
        key = (tuple(pen), tuple(sorted(kw.items())))
        if key not in cache:
            cache[key] = T.Aligner(*pen, **kw)
        return cache[key]

    yield get
    for a in cache.values():
        a.close()
