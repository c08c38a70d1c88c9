"""Shared fixtures.  Tests marked `gpu` need a CUDA device (run with -m gpu); everything else
runs on the CPU: the oracle against the golden fixtures, host topology logic, the C ABI surface."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: full-size workload on the CPU")


@pytest.fixture(scope="session")
def golden_summary():
    p = GOLDEN / "reference_summary.json"
    if not p.exists():
        pytest.skip("reference fixtures not generated yet (tests/golden/make_golden.py)")
    return json.loads(p.read_text())


def golden_npz(name: str):
    p = GOLDEN / f"{name}.npz"
    if not p.exists():
        pytest.skip(f"reference fixture {p.name} not generated yet")
    return np.load(p)


@pytest.fixture(scope="session")
def built_cache():
    """Workloads built once per session by the product's host topology builder."""
    from cirrus_b200 import workloads as W

    cache = {}

    def get(name: str, seed: int = 0):
        key = (name, seed)
        if key not in cache:
            cache[key] = W.build(W.make(name, seed))
        return cache[key]
    return get
