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
        orth = np.abs(Z.T @ Z - np.eye(r["m"])).max() / (n * EPS)
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
