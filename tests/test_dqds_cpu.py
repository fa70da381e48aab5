"""dqds (LAPACK 3.2.2 dlasq2-dlasq6, SRC/LAPACK/odsq2.f-odsq6.f) in the
oracle, and the route of the reference's eigenvalue stage that uses it
(SRC/mrrr_val.c:279-285, 409-412, 459-506): the reference takes it for a
block when its thread count is low (nthreads <= ceil(12 m / n)) and more
than half of the block's eigenvalues are wanted.  MR3_NTHREADS sets that
thread count for the oracle (and the library).

Pins: the oracle's dlasq2 against LAPACK's own (scipy's bundled OpenBLAS, a
newer LAPACK whose shift strategy differs in details, so within 4 n eps
relative, not bitwise) and against numpy; the oracle's dqds route against
the reference's own mrrr() run with 8 threads (which takes dqds for n >=
500): counts exact, eigenvalues within 10 n eps ||T||, residual and
orthogonality <= 10."""
import ctypes as C
import glob
import os

import numpy as np
import pytest

import oracle
from conftest import EPS, tnorm
from mr3smp_b200 import workloads as wl

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def _lapack():
    import scipy
    so = glob.glob(os.path.join(os.path.dirname(scipy.__file__), "..", "scipy.libs",
                                "libscipy_openblas-*.so"))
    if not so:
        pytest.skip("scipy's bundled LAPACK not found")
    return C.CDLL(so[0])


def _qd(rng, n, kind):
    d = rng.uniform(0.1, 2.0, n)
    l = rng.uniform(-1.0, 1.0, n)
    if kind == 1:
        d = 10.0 ** rng.uniform(-10, 0, n)
    elif kind == 2:
        l *= 1e-6
    z = np.zeros(4 * n + 8)
    z[0:2 * n:2] = d
    z[1:2 * n - 1:2] = l[: n - 1] ** 2 * d[: n - 1]
    return z, d, l


def test_oracle_dlasq2_against_lapack_and_numpy():
    L = oracle.lib()
    L.or_dlasq2.restype = None
    L.or_dlasq2.argtypes = [C.c_int, _dp, C.POINTER(C.c_int)]
    LP = _lapack()
    rng = np.random.default_rng(1)
    for trial in range(240):
        n = int(rng.integers(1, 300))
        z, d, l = _qd(rng, n, trial % 3)
        z2 = z.copy()
        info, info2 = C.c_int(), C.c_int()
        L.or_dlasq2(n, z, C.byref(info))
        LP.scipy_dlasq2_(C.byref(C.c_int(n)), z2.ctypes.data_as(C.POINTER(C.c_double)),
                         C.byref(info2))
        assert info.value == 0 and info2.value == 0
        a, b = z[:n], z2[:n]
        assert np.all(np.diff(a) <= 0.0)
        assert np.all(np.abs(a - b) <= 4 * n * EPS * np.abs(b)), trial
        if trial % 3 != 1 and n <= 150:
            dd = d.copy()
            dd[1:] += l[: n - 1] ** 2 * d[: n - 1]
            ee = l[: n - 1] * d[: n - 1]
            T = np.diag(dd) + np.diag(ee, 1) + np.diag(ee, -1)
            w = np.sort(np.linalg.eigvalsh(T))[::-1]
            assert np.abs(w - a).max() <= 100 * n * EPS * np.abs(w).max()


def _cases():
    out = []
    for n in (600, 1500):
        D, E = wl.uniform(n, seed=n)
        out.append((f"uniform{n}_V_A", D, E, "V", "A", {}))
    D, E = wl.one_two_one(800)
    out.append(("121_800_V_A", D, E, "V", "A", {}))
    D, E = wl.glued_wilkinson(4, 201, 1e-12)
    out.append(("glued4x201_V_A", D, E, "V", "A", {}))
    D, E = wl.uniform(1000, seed=3)
    out.append(("uniform1000_V_I", D, E, "V", "I", dict(il=1, iu=700)))
    out.append(("uniform1000_N_A", D, E, "N", "A", {}))
    return out


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_oracle_dqds_route_matches_reference(case, monkeypatch):
    if oracle.ref_lib() is None:
        pytest.skip("the reference library (oracle/_ref) is not built")
    name, D, E, jz, rg, kw = case
    monkeypatch.setenv("MR3_NTHREADS", "8")
    o = oracle.mrrr(jz, rg, D, E, **kw)
    r = oracle.ref_mrrr(jz, rg, D, E, threads=8, **kw)
    n = len(D)
    assert o["info"] == 0 and r["info"] == 0
    assert o["m"] == r["m"]
    assert np.abs(o["W"] - r["W"]).max() <= 10 * n * EPS * tnorm(D, E)
    if jz == "V":
        res, orth = wl.residual_orth(D, E, o["W"], o["Z"])
        assert res <= 10 and orth <= 10, (res, orth)
