"""The allocation-free eigenvector entry point (mr3_cuda_eigvec_noalloc).

Callers that cannot call cudaMalloc -- code inside a device-memory budget
owned by another allocator, or latency-critical loops that cannot afford its
implicit synchronisation -- get eigenvectors of a representation from this
entry point, whose scratch is a static device array of the library.  This
test feeds it the root representation and the eigenvalues that mrrr() (the
existing entry point) returns for matrices whose eigenvalues are all
singletons of the root, and checks, on two calls in a row, that its vectors
agree with mrrr()'s within the tolerance the parity tests use.  It lives in
its own file, collected last, and passes alone or after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

import mr3smp_b200 as M
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
