"""The large single-problem configurations: 30 glued Wilkinson W+ blocks of
667 rows (n = 20010, the lower half of the spectrum, range I) and a 40000-row
matrix that is half uniform random, half glued W+ blocks (range A).  The
oracle would take minutes here; the checks are the size-independent ones:
count, ordering, supports, scaled residual and orthogonality (<= 10, the
bar the reference's own examples use), and identical results on a repeat."""
import time

import numpy as np
import pytest

import mr3smp_b200 as M
from mr3smp_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _check(D, E, r, m_expect, label):
    assert r["info"] == 0, label
    assert r["m"] == m_expect, label
    W = r["W"]
    assert np.all(np.diff(W) >= 0.0), label
    Zs = r["Zsupp"].reshape(-1, 2)
    assert np.all(Zs[:, 0] >= 1) and np.all(Zs[:, 1] <= len(D)) and np.all(Zs[:, 0] <= Zs[:, 1])
    res, orth = wl.residual_orth_torch(D, E, W, r["Z"])
    print(f"{label}: m={r['m']} resid={res:.3g} orth={orth:.3g}")
    assert res <= 10.0 and orth <= 10.0, (label, res, orth)


def test_glued_wilkinson_20010_range_i():
    D, E = wl.glued_wilkinson(30, 667, 1e-12)
    n = len(D)
    t0 = time.perf_counter()
    r = M.mrrr("V", "I", D, E, il=1, iu=n // 2)
    print(f"n={n} range I: {time.perf_counter() - t0:.2f} s (host arrays)")
    _check(D, E, r, n // 2, "glued W+ 20010")
    r2 = M.mrrr("V", "I", D, E, il=1, iu=n // 2)
    assert np.array_equal(r["W"], r2["W"]) and np.array_equal(r["Z"], r2["Z"])


def test_large_mixed_40000_range_a():
    D, E = wl.large_mixed(40000)
    t0 = time.perf_counter()
    r = M.mrrr("V", "A", D, E)
    print(f"n=40000 range A: {time.perf_counter() - t0:.2f} s (host arrays)")
    _check(D, E, r, 40000, "half random, half glued W+ 40000")
