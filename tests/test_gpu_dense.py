"""The device dense driver dsyeig (SRC/dense.c:151-232) on the GPU.

The reduction (dsytrd) and back-transformation (dormtr) are a different
LAPACK's here (cuSOLVER) than the reference's, so the results match in
exact arithmetic only: eigenvalues are compared with numpy's and, where the
reference library is built, with the reference's own dsyeig, within
10*n*eps*||A||; vectors by scaled residual and orthogonality <= 10.
"""
import numpy as np
import pytest

from conftest import EPS, gpu_available

import oracle

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]


def _sym(n, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    B = rng.uniform(-1.0, 1.0, (n, n))
    return (B + B.T) * (0.5 * scale)


def _have_ref():
    L = oracle.ref_lib()
    return L is not None and hasattr(L, "dsyeig")


def _check(A, r, w_all, idx):
    n = A.shape[0]
    nrm = max(np.abs(w_all).max(), np.finfo(float).tiny)
    assert r["info"] == 0, r["info"]
    assert r["m"] == len(idx), (r["m"], len(idx))
    W = r["W"]
    assert np.abs(W - w_all[idx]).max() <= 10 * n * EPS * nrm
    if "Z" in r and r["m"] > 0:
        Z = r["Z"]
        resid = np.abs(A @ Z - Z * W).max() / (n * EPS * nrm)
        orth = np.abs(Z.T @ Z - np.eye(r["m"])).max() / (n * EPS)
        assert resid <= 10 and orth <= 10, (resid, orth)


@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("n", [1, 2, 37, 300])
def test_dsyeig_all(n, uplo):
    import mr3smp_b200 as M
    A = _sym(n, 20 + n)
    w = np.linalg.eigvalsh(A)
    r = M.dsyeig("V", "A", uplo, A)
    _check(A, r, w, np.arange(n))
    if _have_ref():
        ref = oracle.ref_dsyeig("V", "A", uplo, A)
        assert ref["m"] == r["m"]
        assert np.abs(ref["W"] - r["W"]).max() <= 10 * n * EPS * np.abs(w).max()


def test_dsyeig_ranges_and_jobs():
    import mr3smp_b200 as M
    n = 200
    A = _sym(n, 5)
    w = np.linalg.eigvalsh(A)
    _check(A, M.dsyeig("V", "I", "L", A, il=11, iu=90), w, np.arange(10, 90))
    vl, vu = -1.5, 0.25
    sel = np.nonzero((w > vl) & (w <= vu))[0]
    _check(A, M.dsyeig("V", "V", "U", A, vl=vl, vu=vu), w, sel)
    _check(A, M.dsyeig("N", "A", "L", A), w, np.arange(n))
    r = M.dsyeig("C", "V", "L", A, vl=vl, vu=vu)
    assert r["info"] == 0 and r["m"] == len(sel)
    # padded leading dimensions on both sides
    r = M.dsyeig("V", "A", "L", A, lda=n + 3, ldz=n + 5)
    _check(A, r, w, np.arange(n))


@pytest.mark.parametrize("scale", [1e-160, 1e100])
def test_dsyeig_scaled(scale):
    """The scaling path of dscale_matrix (SRC/dense.c:477-527)."""
    import mr3smp_b200 as M
    n = 80
    A = _sym(n, 9, scale)
    w = np.linalg.eigvalsh(A)
    _check(A, M.dsyeig("V", "A", "L", A), w, np.arange(n))
    vl, vu = -0.5 * scale, 0.5 * scale
    sel = np.nonzero((w > vl) & (w <= vu))[0]
    _check(A, M.dsyeig("V", "V", "L", A, vl=vl, vu=vu), w, sel)


def test_dsyeig_clustered():
    """A matrix with a tight cluster (Q diag(1, 1+1e-13, ...) Q^T): the
    tridiagonal stage's cluster path behind the reduction."""
    import mr3smp_b200 as M
    n = 120
    rng = np.random.default_rng(4)
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    lam = np.sort(np.concatenate([1.0 + 1e-13 * np.arange(20), rng.uniform(-2, 2, n - 20)]))
    A = (Q * lam) @ Q.T
    A = 0.5 * (A + A.T)
    w = np.linalg.eigvalsh(A)
    _check(A, M.dsyeig("V", "A", "L", A), w, np.arange(n))


# ---- packed and generalized drivers (SRC/dense.c:236-470) -----------------

@pytest.mark.parametrize("uplo", ["L", "U"])
def test_dspeig(uplo):
    import mr3smp_b200 as M
    n = 150
    A = _sym(n, 31)
    w = np.linalg.eigvalsh(A)
    AP = M.pack(A, uplo)
    _check(A, M.dspeig("V", "A", uplo, AP, n), w, np.arange(n))
    _check(A, M.dspeig("V", "I", uplo, AP, n, il=20, iu=70, ldz=n + 2), w, np.arange(19, 70))
    _check(A, M.dspeig("N", "A", uplo, AP, n), w, np.arange(n))
    if _have_ref():
        ref = oracle.ref_dspeig("V", "A", uplo, AP, n)
        assert np.abs(ref["W"] - w).max() <= 10 * n * EPS * np.abs(w).max()


@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("itype", [1, 2, 3])
def test_dsygeig(itype, uplo):
    import scipy.linalg as sl
    import mr3smp_b200 as M
    from test_dense_cpu import _spd, check_generalized
    n = 120
    A, B = _sym(n, 70 + itype), _spd(n, 80 + itype)
    w = sl.eigh(A, B, type=itype, eigvals_only=True)
    r = M.dsygeig(itype, "V", "A", uplo, A, B)
    check_generalized(itype, A, B, r, w, np.arange(n))
    # B comes back as its Cholesky factor (uplo triangle)
    Lc = np.linalg.cholesky(B)
    F = np.tril(r["B"]) if uplo == "L" else np.triu(r["B"])
    G = Lc if uplo == "L" else Lc.T
    assert np.abs(F - G).max() <= 100 * n * EPS * np.abs(B).max()
    check_generalized(itype, A, B, M.dsygeig(itype, "V", "I", uplo, A, B, il=5, iu=40), w,
                      np.arange(4, 40))
    vl, vu = float(0.5 * (w[10] + w[11])), float(0.5 * (w[60] + w[61]))
    check_generalized(itype, A, B, M.dsygeig(itype, "N", "V", uplo, A, B, vl=vl, vu=vu), w,
                      np.arange(11, 61))
    if _have_ref():
        ref = oracle.ref_dsygeig(itype, "V", "A", uplo, A, B)
        assert np.abs(ref["W"] - r["W"]).max() <= 50 * n * EPS * max(np.abs(w).max(), 1.0)


@pytest.mark.parametrize("itype", [1, 2, 3])
def test_dspgeig(itype):
    import scipy.linalg as sl
    import mr3smp_b200 as M
    from test_dense_cpu import _spd, check_generalized
    n = 90
    A, B = _sym(n, 90 + itype), _spd(n, 95 + itype)
    w = sl.eigh(A, B, type=itype, eigvals_only=True)
    for uplo in "LU":
        r = M.dspgeig(itype, "V", "A", uplo, M.pack(A, uplo), M.pack(B, uplo), n)
        check_generalized(itype, A, B, r, w, np.arange(n))
        Lc = np.linalg.cholesky(B)
        assert np.abs(r["BP"] - M.pack(Lc if uplo == "L" else Lc.T, uplo)).max() <= \
            100 * n * EPS * np.abs(B).max()
    # n = 1 is allowed for the packed generalized driver
    r = M.dspgeig(itype, "V", "A", "L", np.array([3.0]), np.array([4.0]), 1)
    expect = {1: 0.75, 2: 12.0, 3: 12.0}[itype]
    assert r["info"] == 0 and r["m"] == 1 and abs(r["W"][0] - expect) <= 4 * EPS * expect


def test_dsygeig_not_definite():
    """B that is not positive definite: return 2 (the reference asserts)."""
    import mr3smp_b200 as M
    n = 20
    A, B = _sym(n, 1), -np.eye(n)
    assert M.dsygeig(1, "V", "A", "L", A, B)["info"] == 2
