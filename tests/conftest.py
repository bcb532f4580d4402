import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: larger CPU cases")


def golden_cases():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def manifest():
    return golden_cases()


def case_paths(name, meta):
    d = os.path.join(GOLDEN, "cases", name)
    return dict(dir=d, fq=os.path.join(d, "reads.fq.gz"), sai=os.path.join(d, "expected.sai"),
                per_read=os.path.join(d, "per_read.npz"),
                prefix=os.path.join(GOLDEN, meta["ref"], "ref"))
