"""The dense symmetric driver dsyeig on the CPU.

* The reference's own dsyeig (SRC/dense.c:151-232, built from its sources
  into oracle/_ref against scipy's LAPACK) is pinned against numpy's
  symmetric eigensolver: it is the checker of the device driver's tests.
* The device driver's argument checks (mr3smp_b200 dsyeig) run before any
  CUDA call and are tested here without a GPU.
"""
import numpy as np
import pytest

from conftest import EPS

import oracle


def _sym(n, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    B = rng.uniform(-1.0, 1.0, (n, n))
    return (B + B.T) * (0.5 * scale)


def _check(A, r, w_all, idx):
    """Eigenvalues within 10*n*eps*||A|| of numpy's; scaled residual and
    orthogonality of the vectors <= 10 (units n*eps*||A||, n*eps)."""
    n = A.shape[0]
    nrm = max(np.abs(w_all).max(), np.finfo(float).tiny)
    W = r["W"]
    assert r["info"] == 0 and r["m"] == len(idx)
    assert np.abs(W - w_all[idx]).max() <= 10 * n * EPS * nrm
    if "Z" in r and r["m"] > 0:
        Z = r["Z"]
        resid = np.abs(A @ Z - Z * W).max() / (n * EPS * nrm)
        orth = np.abs(Z.conj().T @ Z - np.eye(r["m"])).max() / (n * EPS)
        assert resid <= 10 and orth <= 10, (resid, orth)


needs_ref = pytest.mark.skipif(oracle.ref_lib() is None or not hasattr(oracle.ref_lib(), "dsyeig"),
                               reason="reference library (oracle/_ref) not built")


@needs_ref
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("n", [1, 2, 37, 120])
def test_reference_dsyeig_all(n, uplo):
    A = _sym(n, 10 + n)
    w = np.linalg.eigvalsh(A)
    r = oracle.ref_dsyeig("V", "A", uplo, A)
    _check(A, r, w, np.arange(n))


@needs_ref
def test_reference_dsyeig_ranges():
    n = 90
    A = _sym(n, 7)
    w = np.linalg.eigvalsh(A)
    r = oracle.ref_dsyeig("V", "I", "L", A, il=5, iu=40)
    _check(A, r, w, np.arange(4, 40))
    vl, vu = -0.8, 0.3
    r = oracle.ref_dsyeig("V", "V", "U", A, vl=vl, vu=vu)
    _check(A, r, w, np.nonzero((w > vl) & (w <= vu))[0])
    r = oracle.ref_dsyeig("N", "A", "L", A)
    assert r["info"] == 0 and np.abs(r["W"] - w).max() <= 10 * n * EPS * np.abs(w).max()


@needs_ref
@pytest.mark.parametrize("scale", [1e-160, 1e100])
def test_reference_dsyeig_scaled(scale):
    """max|a_ij| outside [sqrt(DBL_MIN/eps), ~8e76] takes dscale_matrix's
    scaling path (SRC/dense.c:477-527)."""
    n = 50
    A = _sym(n, 3, scale)
    w = np.linalg.eigvalsh(A)
    r = oracle.ref_dsyeig("V", "A", "L", A)
    _check(A, r, w, np.arange(n))


def test_dsyeig_argument_checks():
    """Return 1 for bad arguments without touching the device (the checks of
    SRC/dense.c:177-186, plus lda, ldz and uplo)."""
    import mr3smp_b200 as M
    A = _sym(6, 1)
    assert M.dsyeig("X", "A", "L", A)["info"] == 1
    assert M.dsyeig("V", "X", "L", A)["info"] == 1
    assert M.dsyeig("V", "A", "X", A)["info"] == 1
    assert M.dsyeig("V", "V", "L", A, vl=1.0, vu=1.0)["info"] == 1
    assert M.dsyeig("V", "I", "L", A, il=0, iu=3)["info"] == 1
    assert M.dsyeig("V", "I", "L", A, il=4, iu=3)["info"] == 1
    assert M.dsyeig("V", "I", "L", A, il=1, iu=7)["info"] == 1
    assert M.dsyeig("V", "A", "L", A, lda=5)["info"] == 1
    assert M.dsyeig("V", "A", "L", A, ldz=5)["info"] == 1
    assert M.dsyeig("V", "A", "L", np.zeros((0, 0)))["info"] == 1
    # counting with range A or I needs no device work
    r = M.dsyeig("C", "I", "U", A, il=2, iu=5)
    assert r["info"] == 0 and r["m"] == 4
    r = M.dsyeig("C", "A", "L", A)
    assert r["info"] == 0 and r["m"] == 6


# ---- packed and generalized drivers (SRC/dense.c:236-470) -----------------

def _spd(n, seed):
    rng = np.random.default_rng(seed)
    Y = rng.standard_normal((n, n))
    return np.eye(n) + 0.1 * (Y @ Y.T) / n


def check_generalized(itype, A, B, r, w_all, idx, tol=50.0):
    """Eigenvalues of the pencil (scipy) within tol*n*eps*max|lambda|; the
    residual of the generalized equation and the B-orthogonality of the
    vectors (X^T B X = I for itypes 1 and 2, X^T inv(B) X = I for itype 3)
    within tol, in units of n*eps times the norms involved."""
    n = A.shape[0]
    assert r["info"] == 0 and r["m"] == len(idx), (r["info"], r["m"], len(idx))
    W = r["W"]
    lam = max(np.abs(w_all).max(), 1.0)
    assert np.abs(W - w_all[idx]).max() <= tol * n * EPS * lam
    if "Z" not in r or r["m"] == 0:
        return
    X = r["Z"]
    nA, nB = np.abs(A).max() * n, np.abs(B).max() * n
    if itype == 1:
        R = A @ X - (B @ X) * W
        scale = (nA + lam * nB) * np.abs(X).max()
        G = X.conj().T @ B @ X
    elif itype == 2:
        R = A @ (B @ X) - X * W
        scale = (nA * nB + lam) * np.abs(X).max()
        G = X.conj().T @ B @ X
    else:
        R = B @ (A @ X) - X * W
        scale = (nA * nB + lam) * np.abs(X).max()
        G = X.conj().T @ np.linalg.solve(B, X)
    assert np.abs(R).max() / (n * EPS * scale) <= tol
    assert np.abs(G - np.eye(r["m"])).max() / (n * EPS * np.linalg.cond(B)) <= tol


@needs_ref
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("itype", [1, 2, 3])
def test_reference_dsygeig(itype, uplo):
    import scipy.linalg as sl
    n = 70
    A, B = _sym(n, 40 + itype), _spd(n, 50 + itype)
    w = sl.eigh(A, B, type=itype, eigvals_only=True)
    check_generalized(itype, A, B, oracle.ref_dsygeig(itype, "V", "A", uplo, A, B), w,
                      np.arange(n))
    check_generalized(itype, A, B, oracle.ref_dsygeig(itype, "V", "I", uplo, A, B, il=4, iu=30),
                      w, np.arange(3, 30))


@needs_ref
@pytest.mark.parametrize("uplo", ["L", "U"])
def test_reference_packed(uplo):
    import scipy.linalg as sl
    import mr3smp_b200 as M
    n = 64
    A, B = _sym(n, 61), _spd(n, 62)
    w = np.linalg.eigvalsh(A)
    _check(A, oracle.ref_dspeig("V", "A", uplo, M.pack(A, uplo), n), w, np.arange(n))
    for itype in (1, 2, 3):
        wg = sl.eigh(A, B, type=itype, eigvals_only=True)
        r = oracle.ref_dspgeig(itype, "V", "A", uplo, M.pack(A, uplo), M.pack(B, uplo), n)
        check_generalized(itype, A, B, r, wg, np.arange(n))


def test_pack_layout():
    """pack() follows LAPACK's packed storage: column j of the lower triangle
    starts at j*n - j*(j-1)/2, of the upper triangle at j*(j+1)/2."""
    import mr3smp_b200 as M
    n = 5
    A = np.arange(n * n, dtype=float).reshape(n, n)
    L, U = M.pack(A, "L"), M.pack(A, "U")
    for j in range(n):
        for i in range(n):
            if i >= j:
                assert L[i + j * (2 * n - j - 1) // 2] == A[i, j]
            if i <= j:
                assert U[i + j * (j + 1) // 2] == A[i, j]


def test_packed_generalized_argument_checks():
    """The checks of SRC/dense.c:257-262, 340-347, 420-425 (and ldz, uplo,
    range bounds) return 1 without touching the device."""
    import mr3smp_b200 as M
    n = 6
    A, B = _sym(n, 1), _spd(n, 2)
    AP, BP = M.pack(A, "L"), M.pack(B, "L")
    assert M.dsygeig(0, "V", "A", "L", A, B)["info"] == 1
    assert M.dsygeig(4, "V", "A", "L", A, B)["info"] == 1
    assert M.dsygeig(1, "V", "A", "X", A, B)["info"] == 1
    assert M.dsygeig(1, "X", "A", "L", A, B)["info"] == 1
    assert M.dsygeig(1, "V", "I", "L", A, B, il=3, iu=2)["info"] == 1
    assert M.dsygeig(1, "V", "A", "L", A[:1, :1], B[:1, :1])["info"] == 1   # n <= 1
    assert M.dspeig("V", "X", "L", AP, n)["info"] == 1
    assert M.dspeig("V", "A", "X", AP, n)["info"] == 1
    assert M.dspeig("V", "A", "L", AP, n, ldz=n - 1)["info"] == 1
    assert M.dspeig("V", "V", "L", AP, n, vl=2.0, vu=1.0)["info"] == 1
    r = M.dspeig("C", "I", "L", AP, n, il=2, iu=4)
    assert r["info"] == 0 and r["m"] == 3
    assert M.dspgeig(0, "V", "A", "L", AP, BP, n)["info"] == 1
    assert M.dspgeig(1, "V", "A", "L", AP, BP, 0)["info"] == 1
    assert M.dspgeig(1, "V", "A", "L", AP, BP, n, ldz=n - 1)["info"] == 1


# ---- complex Hermitian drivers (SRC/dense.c:568-936, COMPLEX_SUPPORTED) ----

def _herm(n, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    X = rng.uniform(-1, 1, (n, n)) + 1j * rng.uniform(-1, 1, (n, n))
    return (X + X.conj().T) * (0.5 * scale)


def _hpd(n, seed):
    rng = np.random.default_rng(seed)
    Y = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    return np.eye(n) + 0.1 * (Y @ Y.conj().T) / n


def _cpack(A, uplo):
    n = A.shape[0]
    cols = [A[j:, j] for j in range(n)] if uplo == "L" else [A[: j + 1, j] for j in range(n)]
    return np.concatenate(cols)


needs_cref = pytest.mark.skipif(oracle.ref_lib() is None or not hasattr(oracle.ref_lib(), "zheeig"),
                                reason="reference library (oracle/_ref) without complex drivers")


@needs_cref
@pytest.mark.parametrize("uplo", ["L", "U"])
def test_reference_zheeig(uplo):
    n = 64
    A = _herm(n, 71)
    w = np.linalg.eigvalsh(A)
    _check(A, oracle.ref_zheeig("V", "A", uplo, A), w, np.arange(n))
    _check(A, oracle.ref_zheeig("V", "I", uplo, A, il=3, iu=30), w, np.arange(2, 30))
    _check(A, oracle.ref_zhpeig("V", "A", uplo, _cpack(A, uplo), n), w, np.arange(n))
    _check(A * 1e-160, oracle.ref_zheeig("V", "A", uplo, A * 1e-160), w * 1e-160, np.arange(n))


@needs_cref
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("itype", [1, 2, 3])
def test_reference_zhegeig(itype, uplo):
    import scipy.linalg as sl
    n = 56
    A, B = _herm(n, 80 + itype), _hpd(n, 90 + itype)
    w = sl.eigh(A, B, type=itype, eigvals_only=True)
    check_generalized(itype, A, B, oracle.ref_zhegeig(itype, "V", "A", uplo, A, B), w,
                      np.arange(n))
    r = oracle.ref_zhpgeig(itype, "V", "A", uplo, _cpack(A, uplo), _cpack(B, uplo), n)
    check_generalized(itype, A, B, r, w, np.arange(n))


def test_complex_argument_checks():
    """The complex drivers' argument checks (SRC/dense.c:596-602, 697-701,
    788-796, 888-892, plus lda, ldb, ldz, uplo) return 1 without touching the
    device."""
    import mr3smp_b200 as M
    n = 5
    A, B = _herm(n, 1), _hpd(n, 2)
    AP, BP = _cpack(A, "L"), _cpack(B, "L")
    assert M.zheeig("X", "A", "L", A)["info"] == 1
    assert M.zheeig("V", "A", "X", A)["info"] == 1
    assert M.zheeig("V", "I", "L", A, il=2, iu=9)["info"] == 1
    assert M.zheeig("V", "A", "L", A, lda=4)["info"] == 1
    assert M.zheeig("V", "A", "L", A, ldz=4)["info"] == 1
    r = M.zheeig("C", "I", "U", A, il=2, iu=4)
    assert r["info"] == 0 and r["m"] == 3
    assert M.zhpeig("V", "V", "L", AP, n, vl=1.0, vu=0.0)["info"] == 1
    assert M.zhpeig("V", "A", "L", AP, n, ldz=4)["info"] == 1
    r = M.zhpeig("C", "A", "L", AP, n)
    assert r["info"] == 0 and r["m"] == n
    assert M.zhegeig(0, "V", "A", "L", A, B)["info"] == 1
    assert M.zhegeig(1, "V", "A", "L", A[:1, :1], B[:1, :1])["info"] == 1
    assert M.zhegeig(1, "V", "X", "L", A, B)["info"] == 1
    assert M.zhpgeig(4, "V", "A", "L", AP, BP, n)["info"] == 1
    assert M.zhpgeig(1, "V", "A", "L", AP[:1], BP[:1], 1)["info"] == 1
    assert M.zhpgeig(1, "V", "A", "L", AP, BP, n, ldz=4)["info"] == 1
