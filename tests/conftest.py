import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from netflix_prize_b200.data import Dataset  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_fixtures.json")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU")


def load_golden():
    with open(GOLDEN) as f:
        return json.load(f)


def tiny_sets():
    """make_tiny_train / make_tiny_probe (reference tests/helpers.rs:37-95)."""
    g = load_golden()
    tr = np.array(g["tiny_train"])
    pr = np.array(g["tiny_probe"])
    T = Dataset.from_ratings(tr[:, 0], tr[:, 1], tr[:, 2], tr[:, 3], g["n_users"], g["n_items"], "tiny_train")
    P = Dataset.from_ratings(pr[:, 0], pr[:, 1], pr[:, 2], pr[:, 3], g["n_users"], g["n_items"], "tiny_probe")
    return T, P


@pytest.fixture(scope="session")
def golden():
    return load_golden()


@pytest.fixture(scope="session")
def tiny():
    return tiny_sets()


_SMALL = {}


def small_sets(n_users=600, n_items=300, n_train=30000, seed=7):
    key = (n_users, n_items, n_train, seed)
    if key not in _SMALL:
        from netflix_prize_b200 import synth
        spec = synth.scaled(synth.spec_c1(seed), n_users, n_items, n_train, f"small{seed}")
        _SMALL[key] = synth.generate(spec)
    return _SMALL[key]


@pytest.fixture(scope="session")
def small():
    return small_sets()
