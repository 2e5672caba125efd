"""Shared pytest set-up: the `gpu` marker and helpers to load golden fixtures."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built extension")


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def min_abs_tilt_index(tilts):
    """Index of the tilt MainCode.cu:46-49 reprojects at: the first of the
    smallest |angle| among the negated angles."""
    neg = -np.asarray(tilts, np.float32)
    om, idx = neg[0], 0
    for i, t in enumerate(neg):
        if abs(om) > abs(t):
            om, idx = t, i
    return idx


def cfg2_fp64(z):
    """The FP64 oracle's result stored in tests/golden/cfg2.npz (as its
    int16-quantised difference from the reference's), in float64."""
    return z["ref_m"].astype(np.float64) + z["fp64_minus_ref_q"].astype(np.float64) * float(z["fp64_minus_ref_step"])


@pytest.fixture(scope="session")
def golden():
    return {n: load_golden(n) for n in ("a", "b", "c", "cli")}
