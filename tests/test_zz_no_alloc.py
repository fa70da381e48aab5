"""The allocation-free eigenvector entry point (mr3_cuda_eigvec_noalloc).

Callers that cannot call cudaMalloc -- code inside a device-memory budget
owned by another allocator, or latency-critical loops that cannot afford its
implicit synchronisation -- get eigenvectors of a representation from this
entry point, whose scratch is a static device array of the library.  This
test feeds it the root representation and the eigenvalues that mrrr() (the
existing entry point) returns for matrices whose eigenvalues are all
singletons of the root, and checks, on two calls in a row, that its vectors
agree with mrrr()'s within the tolerance the parity tests use; it also checks
n = 1 and, against the oracle's dlar1v bit for bit, a shift that makes a
pivot exactly zero (the NaN-safe sweeps) with the pivot threshold the entry
point derives from the representation.  It lives in its own file, collected
last, and passes alone or after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

import mr3smp_b200 as M
import oracle
from conftest import EPS, tnorm
from mr3smp_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _matrices():
    D, E = wl.one_two_one(40)
    yield "121_40", D, E
    n = 500
    D = np.linspace(1.0, 2.0, n)
    E = np.full(n, 1e-3)
    E[-1] = 0.0
    yield "graded_500", D, E


def _call(L, n, Dd, Ld, m, lam, gaptol, Z, ldz, Zs, stream):
    return L.mr3_cuda_eigvec_noalloc(n, C.c_void_p(Dd.data_ptr()), C.c_void_p(Ld.data_ptr()), m,
                                     C.c_void_p(lam.data_ptr()), C.c_double(gaptol),
                                     C.c_void_p(Z.data_ptr()), ldz, C.c_void_p(Zs.data_ptr()),
                                     C.c_void_p(stream))


@pytest.mark.parametrize("name,D,E", list(_matrices()), ids=[x[0] for x in _matrices()])
def test_noalloc_eigvecs_match_mrrr_two_calls(name, D, E):
    import torch
    L = M.lib()
    L.mr3_cuda_eigvec_noalloc.restype = C.c_int
    L.mr3_cuda_eigvec_noalloc.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                          C.c_double, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    n = len(D)
    r = M.mrrr("V", "A", D, E)
    assert r["info"] == 0 and r["m"] == n
    W = r["W"]
    # the overwritten D/E hold the root representation and its shift
    sigma = r["E"][n - 1]
    gaps = np.minimum(np.r_[np.inf, np.diff(W)], np.r_[np.diff(W), np.inf])
    # every eigenvalue must be a singleton of the root: relative gap (w.r.t.
    # the shifted eigenvalue) above MRRR's 1e-3 threshold, with margin
    assert np.all(gaps >= 1.5e-3 * np.abs(W - sigma)), "test matrix must have only singletons"
    dev = torch.device("cuda")
    Dd = torch.from_numpy(r["D"]).to(dev)
    Ld = torch.from_numpy(r["E"]).to(dev)
    lam = torch.from_numpy(W - sigma).to(dev)
    tn = tnorm(D, E)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        Z = torch.full((n * n,), np.nan, dtype=torch.float64, device=dev)
        Zs = torch.zeros(2 * n, dtype=torch.int32, device=dev)
        rc = _call(L, n, Dd, Ld, n, lam, 0.0, Z, n, Zs, stream)
        assert rc == 0
        torch.cuda.synchronize()
        Zn = Z.cpu().numpy().reshape(n, n).T
        assert np.all(np.isfinite(Zn)), f"call {call}: unwritten entries"
        res, orth = wl.residual_orth(D, E, W, Zn)
        assert res <= 10.0 and orth <= 10.0, (call, res, orth)
        c = np.abs(np.sum(Zn * r["Z"], axis=0))
        assert np.all(np.abs(1.0 - c) <= 1e3 * n * EPS * tn / gaps), (call, np.abs(1 - c).max())


def test_noalloc_rejects_sizes_beyond_the_limit():
    import torch
    L = M.lib()
    L.mr3_cuda_eigvec_noalloc.restype = C.c_int
    L.mr3_cuda_eigvec_noalloc.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                          C.c_double, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    n = 2049
    t = torch.zeros(4, dtype=torch.float64, device="cuda")
    rc = L.mr3_cuda_eigvec_noalloc(n, C.c_void_p(t.data_ptr()), C.c_void_p(t.data_ptr()), 1,
                                   C.c_void_p(t.data_ptr()), C.c_double(0.0),
                                   C.c_void_p(t.data_ptr()), n, C.c_void_p(t.data_ptr()), None)
    assert rc == 1


def _setup(L):
    L.mr3_cuda_eigvec_noalloc.restype = C.c_int
    L.mr3_cuda_eigvec_noalloc.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                          C.c_double, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]


def test_noalloc_n1_unit_vectors():
    import torch
    L = M.lib()
    _setup(L)
    dev = torch.device("cuda")
    D = torch.tensor([0.7], dtype=torch.float64, device=dev)
    lam = torch.tensor([0.7, 0.7], dtype=torch.float64, device=dev)
    Z = torch.full((6,), np.nan, dtype=torch.float64, device=dev)
    Zs = torch.zeros(4, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    rc = _call(L, 1, D, D, 2, lam, 0.0, Z, 3, Zs, stream)
    torch.cuda.synchronize()
    assert rc == 0
    assert Z.cpu().numpy()[0] == 1.0 and Z.cpu().numpy()[3] == 1.0
    assert Zs.cpu().numpy().tolist() == [1, 1, 1, 1]


def test_noalloc_zero_pivot_matches_oracle_dlar1v():
    """lambda = D(1) makes the first stationary pivot exactly zero, so the
    sweeps rerun with the NaN-safe formulas; the vector, its support and the
    twist must be the oracle's dlar1v with the same pivot threshold."""
    import torch
    L = M.lib()
    _setup(L)
    OL = oracle.lib()
    n = 60
    rng = np.random.default_rng(4)
    d = rng.uniform(0.5, 2.0, n)
    l = rng.uniform(-0.9, 0.9, n)
    l[-1] = 0.0
    ld = d * l
    lld = ld * l
    pivmin = 2.2250738585072014e-308 * max(1.0, float(np.max(np.abs(ld[: n - 1])) ** 2))
    lams = np.array([d[0], 0.5 * (d[3] + d[4])])
    dev = torch.device("cuda")
    Dd = torch.from_numpy(d).to(dev)
    Ld = torch.from_numpy(l).to(dev)
    lam = torch.from_numpy(lams).to(dev)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        Z = torch.full((n * 2,), np.nan, dtype=torch.float64, device=dev)
        Zs = torch.zeros(4, dtype=torch.int32, device=dev)
        assert _call(L, n, Dd, Ld, 2, lam, 0.0, Z, n, Zs, stream) == 0
        torch.cuda.synchronize()
        Zn = Z.cpu().numpy().reshape(2, n)
        Zsn = Zs.cpu().numpy()
        for j, lm in enumerate(lams):
            z = np.zeros(n)
            isz = np.zeros(2, dtype=np.int32)
            work = np.zeros(4 * n)
            neg, r = C.c_int(), C.c_int(0)
            ztz, mg, nr, rs, rq = (C.c_double() for _ in range(5))
            OL.or_dlar1v(n, 1, n, float(lm), d, l, ld, lld, pivmin, 0.0, z, 0, C.byref(neg),
                         C.byref(ztz), C.byref(mg), C.byref(r), isz, C.byref(nr), C.byref(rs),
                         C.byref(rq), work)
            want = np.zeros(n)
            a, b = isz[0] - 1, isz[1]
            want[a:b] = z[a:b] * nr.value
            assert Zsn[2 * j] == isz[0] and Zsn[2 * j + 1] == isz[1], (call, j)
            assert np.array_equal(Zn[j], want), (call, j, np.abs(Zn[j] - want).max())
