"""CPU tests of the oracle: pinned against the reference's golden vectors,
against LAPACK's own kernels (bitwise) and against closed forms."""
import ctypes as C
import glob
import math
import os

import numpy as np
import pytest

import oracle
from conftest import EPS, load_golden, tnorm
from mr3smp_b200 import workloads as wl
from zoo import small_zoo

CASES, GOLD = load_golden()


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_matches_reference_golden(case):
    name = case["name"]
    D, E, Wref = GOLD[name + "/D"], GOLD[name + "/E"], GOLD[name + "/W"]
    r = oracle.mrrr(case["jobz"], case["range"], D, E, **case["kw"])
    assert r["info"] == 0
    assert r["m"] == case["m"], "eigenvalue count must be exact"
    n = len(D)
    tn = tnorm(D, E)
    assert np.abs(r["W"] - Wref).max() <= 10 * n * EPS * tn
    if n >= 500:   # below 500 the reference hands over to dstemr, which leaves il/iu alone
        assert (r["il"], r["iu"]) == (case["il"], case["iu"])
    if case["jobz"] == "V":
        res, orth = wl.residual_orth(D, E, r["W"], r["Z"])
        bound = max(10.0, case["ref_orth"]) if name.startswith("w21") else 10.0
        assert res <= 10.0 and orth <= bound, (res, orth)
        # eigenvector columns of isolated eigenvalues agree with the reference's
        cols = GOLD[name + "/zcols"]
        Zr = GOLD[name + "/Z"]
        full = np.linalg.eigvalsh(np.diag(D) + np.diag(E[:-1], 1) + np.diag(E[:-1], -1))
        for k, j in enumerate(cols):
            lam = Wref[j]
            others = np.delete(full, np.argmin(np.abs(full - lam)))
            gap = np.abs(others - lam).min() if len(others) else np.inf
            if gap < 1e-6 * tn:
                continue
            c = abs(float(r["Z"][:, j] @ Zr[:, k]))
            assert abs(c - 1.0) <= 1e3 * n * EPS * tn / gap, (j, c)


def test_count_only_matches_reference():
    for c in CASES:
        if c["count_m"] is not None:
            D, E = GOLD[c["name"] + "/D"], GOLD[c["name"] + "/E"]
            r = oracle.mrrr("C", c["range"], D, E, **c["kw"])
            assert r["info"] == 0 and r["m"] == c["count_m"]


@pytest.mark.parametrize("n", [50, 600, 2048])
def test_oracle_121_closed_form(n):
    D, E = wl.one_two_one(n)
    r = oracle.mrrr("V", "A", D, E)
    assert r["m"] == n
    assert np.abs(r["W"] - wl.one_two_one_eigs(n)).max() <= 10 * n * EPS * 2.0
    if n <= 600:
        res, orth = wl.residual_orth(D, E, r["W"], r["Z"])
        assert res <= 10 and orth <= 10


@pytest.mark.parametrize("case", small_zoo(), ids=lambda c: c[0])
def test_oracle_zoo_accuracy(case):
    name, D, E, jz, rg, kw = case
    r = oracle.mrrr(jz, rg, D, E, **kw)
    assert r["info"] == 0, name
    T = np.diag(D) + np.diag(E[:-1], 1) + np.diag(E[:-1], -1)
    ev = np.linalg.eigvalsh(T)
    n = len(D)
    tn = max(tnorm(D, E), np.finfo(float).tiny)
    if jz == "C":
        return
    if rg == "A":
        assert r["m"] == n
        assert np.abs(np.sort(r["W"]) - ev).max() <= 10 * n * EPS * tn
    if jz == "V" and r["m"] and not name.startswith("w21"):
        res, orth = wl.residual_orth(D, E, r["W"], r["Z"])
        assert res <= 10 and orth <= 10, (res, orth)


def test_oracle_bad_arguments():
    D, E = wl.uniform(10, seed=0)
    assert oracle.mrrr("X", "A", D, E)["info"] == 1
    assert oracle.mrrr("V", "Q", D, E)["info"] == 1
    assert oracle.mrrr("V", "V", D, E, vl=1.0, vu=0.5)["info"] == 1
    assert oracle.mrrr("V", "I", D, E, il=0, iu=3)["info"] == 1
    assert oracle.mrrr("V", "I", D, E, il=4, iu=3)["info"] == 1
    assert oracle.mrrr("V", "I", D, E, il=1, iu=11)["info"] == 1
    assert oracle.mrrr("C", "A", D, E)["m"] == 10
    assert oracle.mrrr("C", "I", D, E, il=2, iu=5)["m"] == 4


def test_or_log_accuracy():
    L = oracle.lib()
    xs = np.exp(np.random.default_rng(0).uniform(-700, 700, 5000))
    for x in xs:
        if x == 1.0:
            continue
        ref = math.log(x)
        assert abs(L.or_log(float(x)) - ref) <= 2 * abs(ref) * EPS
    assert L.or_log(1.0) == 0.0


# ---- bitwise pins of the restated kernels against LAPACK's own routines ----
def _lapack():
    import scipy
    so = glob.glob(os.path.join(os.path.dirname(scipy.__file__), "..", "scipy.libs",
                                "libscipy_openblas-*.so"))
    if not so:
        pytest.skip("scipy's bundled LAPACK not found")
    return C.CDLL(so[0])


_pd = C.POINTER(C.c_double)
_pi = C.POINTER(C.c_int)


def _dp(a):
    return a.ctypes.data_as(_pd)


def _ip(a):
    return a.ctypes.data_as(_pi)


def _I(v):
    return C.byref(C.c_int(v))


def _D(v):
    return C.byref(C.c_double(v))


def _ldl(rng, n):
    D = rng.uniform(-1, 1, n)
    E = rng.uniform(-1, 1, n - 1)
    T = np.diag(D) + np.diag(E, 1) + np.diag(E, -1)
    ev = np.linalg.eigvalsh(T)
    sig = ev[0] - 0.01
    d = np.zeros(n)
    l = np.zeros(n)
    d[0] = D[0] - sig
    for i in range(n - 1):
        l[i] = E[i] / d[i]
        d[i + 1] = D[i + 1] - sig - l[i] * E[i]
    return d, l, ev - sig


def test_dlaneg_bitwise_vs_lapack():
    LP, L = _lapack(), oracle.lib()
    LP.scipy_dlaneg_.restype = C.c_int
    rng = np.random.default_rng(0)
    for _ in range(300):
        n = int(rng.integers(2, 400))
        d = rng.uniform(-2, 2, n)
        lld = rng.uniform(0, 1, n)
        sig = rng.uniform(-3, 3)
        r = int(rng.integers(1, n + 1))
        assert L.or_dlaneg(n, d, lld, sig, 1e-300, r) == \
            LP.scipy_dlaneg_(_I(n), _dp(d), _dp(lld), _D(sig), _D(1e-300), _I(r))


def test_dlarnv_bitwise_vs_lapack():
    LP, L = _lapack(), oracle.lib()
    s1 = np.array([1, 1, 1, 1], dtype=np.int32)
    s2 = s1.copy()
    x1, x2 = np.zeros(1000), np.zeros(1000)
    L.or_dlarnv2(s1, 1000, x1)
    LP.scipy_dlarnv_(_I(2), _ip(s2), _I(1000), _dp(x2))
    assert np.array_equal(x1, x2) and np.array_equal(s1, s2)


def test_dlarrb_dlar1v_bitwise_vs_lapack():
    LP, L = _lapack(), oracle.lib()
    rng = np.random.default_rng(1)
    for _ in range(40):
        n = int(rng.integers(5, 300))
        d, l, ev = _ldl(rng, n)
        ld = d * l
        lld = ld * l
        ld[-1] = lld[-1] = 0.0
        i1 = int(rng.integers(1, n))
        i2 = int(rng.integers(i1, n + 1))
        m = i2 - i1 + 1
        w0 = ev[i1 - 1:i2] * (1 + rng.uniform(-1e-6, 1e-6, m))
        e0 = np.abs(ev[i1 - 1:i2]) * 2e-6 + 1e-12
        g0 = np.maximum(0, np.r_[ev[i1:i2] - ev[i1 - 1:i2 - 1], 0.1])
        outs = []
        for f in (0, 1):
            w, we, wg = w0.copy(), e0.copy(), g0.copy()
            work, iwork, info = np.zeros(2 * n), np.zeros(2 * n, dtype=np.int32), C.c_int(0)
            if f == 0:
                L.or_dlarrb(n, d, lld, i1, i2, 1e-8, 4 * EPS, i1 - 1, w, wg, we, work, iwork,
                            1e-300, 4.0, n, C.byref(info))
            else:
                LP.scipy_dlarrb_(_I(n), _dp(d), _dp(lld), _I(i1), _I(i2), _D(1e-8), _D(4 * EPS),
                                 _I(i1 - 1), _dp(w), _dp(wg), _dp(we), _dp(work), _ip(iwork),
                                 _D(1e-300), _D(4.0), _I(n), C.byref(info))
            outs.append((w, we, wg))
        for a, b in zip(*outs):
            assert np.array_equal(a, b)
        k = int(rng.integers(0, n))
        lam = ev[k] * (1 + 1e-14)
        res = []
        for f in (0, 1):
            z, work, isz = np.zeros(n), np.zeros(4 * n), np.zeros(2, dtype=np.int32)
            neg, ztz, mg, r, nr, rs, rq = (C.c_int(), C.c_double(), C.c_double(), C.c_int(0),
                                           C.c_double(), C.c_double(), C.c_double())
            if f == 0:
                L.or_dlar1v(n, 1, n, lam, d, l, ld, lld, 1e-300, 1e-17, z, 1, C.byref(neg),
                            C.byref(ztz), C.byref(mg), C.byref(r), isz, C.byref(nr), C.byref(rs),
                            C.byref(rq), work)
            else:
                LP.scipy_dlar1v_(_I(n), _I(1), _I(n), _D(lam), _dp(d), _dp(l), _dp(ld), _dp(lld),
                                 _D(1e-300), _D(1e-17), _dp(z), C.byref(C.c_int(1)), C.byref(neg),
                                 C.byref(ztz), C.byref(mg), C.byref(r), _ip(isz), C.byref(nr),
                                 C.byref(rs), C.byref(rq), _dp(work))
            res.append((z, isz, neg.value, ztz.value, mg.value, r.value, nr.value, rs.value, rq.value))
        assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])
        assert res[0][2:] == res[1][2:]


def test_sturm_count_bitwise_vs_lapack_dlaebz():
    LP, L = _lapack(), oracle.lib()
    rng = np.random.default_rng(2)
    for _ in range(200):
        n = int(rng.integers(2, 300))
        D, E = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
        E2 = E * E
        x = rng.uniform(-2, 2)
        ab = np.array([x, x])
        nab = np.zeros(2, dtype=np.int32)
        c, work = np.zeros(1), np.zeros(1)
        iwork, nval = np.zeros(1, dtype=np.int32), np.zeros(1, dtype=np.int32)
        mout, info = C.c_int(), C.c_int()
        LP.scipy_dlaebz_(_I(1), _I(0), _I(n), _I(1), _I(1), _I(0), _D(0.0), _D(0.0), _D(1e-300),
                         _dp(D), _dp(E), _dp(E2), _ip(nval), _dp(ab), _dp(c), C.byref(mout),
                         _ip(nab), _dp(work), _ip(iwork), C.byref(info))
        assert L.or_count_ijob1(n, D, E2, 1e-300, x) == nab[0]


def test_dlarrr_vs_lapack():
    LP, L = _lapack(), oracle.lib()
    rng = np.random.default_rng(3)
    for _ in range(100):
        n = int(rng.integers(2, 50))
        scale = rng.choice([1e-3, 1.0, 10.0])
        D = rng.uniform(0.5, 2, n) * rng.choice([-1, 1], n)
        E = rng.uniform(-1, 1, n) * scale
        info = C.c_int()
        LP.scipy_dlarrr_(_I(n), _dp(D), _dp(E), C.byref(info))
        assert L.or_dlarrr(n, D, E) == info.value
