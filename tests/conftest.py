"""Shared helpers for the test suite.

Tests marked ``gpu`` need a CUDA device; everything else runs on CPU.  The
oracle (oracle/) is the checker: GPU results must equal its results bit for
bit, and both must agree with the reference's golden vectors within the
tolerances of the benchmark statement (counts exact; eigenvalues within
10*n*eps*||T||; scaled residual and orthogonality <= 10).
"""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

EPS = np.finfo(np.float64).eps
GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def load_golden():
    with open(os.path.join(GOLDEN_DIR, "golden.json")) as f:
        man = json.load(f)
    arr = np.load(os.path.join(GOLDEN_DIR, "golden.npz"))
    return man["cases"], arr


def tnorm(D, E):
    n = len(D)
    return max(np.abs(D).max(), np.abs(E[: n - 1]).max() if n > 1 else 0.0)


def assert_same(a: dict, b: dict, what: str = ""):
    """Bitwise equality of two solver results (dicts from mrrr wrappers)."""
    assert a["info"] == b["info"], f"{what}: info {a['info']} != {b['info']}"
    assert a["m"] == b["m"], f"{what}: m {a['m']} != {b['m']}"
    for k in ("W", "D", "E", "Z", "Zsupp"):
        if k in a or k in b:
            x, y = np.asarray(a[k]), np.asarray(b[k])
            assert x.shape == y.shape, f"{what}: {k} shape {x.shape} != {y.shape}"
            if not np.array_equal(x, y):
                d = np.nonzero(x != y)
                first = tuple(int(v[0]) for v in d)
                raise AssertionError(f"{what}: {k} differs at {len(d[0])} entries, first {first}: "
                                     f"{x[first]!r} vs {y[first]!r}")
    for k in ("vl", "vu"):
        assert a[k] == b[k] or (np.isnan(a[k]) and np.isnan(b[k])), f"{what}: {k} {a[k]} != {b[k]}"
    for k in ("il", "iu", "tryrac"):
        assert a[k] == b[k], f"{what}: {k} {a[k]} != {b[k]}"
