"""The complex Hermitian dense drivers (zheeig, zhpeig, zhegeig, zhpgeig;
SRC/dense.c:568-936) on the GPU.

As for the real drivers, the reduction and back-transformation are
cuSOLVER's/cuBLAS's, so the results match the reference's within
tolerances: eigenvalues against numpy/scipy and the reference's own complex
drivers (oracle/_ref) within 10*n*eps*||A|| (50 for the generalized
problems), vectors by residual and (B-)orthogonality.
"""
import numpy as np
import pytest

from conftest import EPS, gpu_available

import oracle

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]


def _have_ref():
    L = oracle.ref_lib()
    return L is not None and hasattr(L, "zheeig")


@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("n", [1, 2, 40, 200])
def test_zheeig(n, uplo):
    import mr3smp_b200 as M
    from test_dense_cpu import _check, _cpack, _herm
    A = _herm(n, 200 + n)
    w = np.linalg.eigvalsh(A)
    _check(A, M.zheeig("V", "A", uplo, A), w, np.arange(n))
    if n > 2:
        _check(A, M.zheeig("V", "I", uplo, A, il=2, iu=n // 2, lda=n + 1, ldz=n + 3), w,
               np.arange(1, n // 2))
        _check(A, M.zhpeig("V", "A", uplo, _cpack(A, uplo), n), w, np.arange(n))
        _check(A, M.zheeig("N", "A", uplo, A), w, np.arange(n))
    if _have_ref():
        ref = oracle.ref_zheeig("V", "A", uplo, A)
        assert np.abs(ref["W"] - w).max() <= 10 * n * EPS * max(np.abs(w).max(), 1e-300)


@pytest.mark.parametrize("scale", [1e-160, 1e100])
def test_zheeig_scaled(scale):
    import mr3smp_b200 as M
    from test_dense_cpu import _check, _herm
    n = 60
    A = _herm(n, 7, scale)
    w = np.linalg.eigvalsh(A)
    _check(A, M.zheeig("V", "A", "L", A), w, np.arange(n))


@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("itype", [1, 2, 3])
def test_zhegeig(itype, uplo):
    import scipy.linalg as sl
    import mr3smp_b200 as M
    from test_dense_cpu import _cpack, _herm, _hpd, check_generalized
    n = 80
    A, B = _herm(n, 300 + itype), _hpd(n, 310 + itype)
    w = sl.eigh(A, B, type=itype, eigvals_only=True)
    r = M.zhegeig(itype, "V", "A", uplo, A, B)
    check_generalized(itype, A, B, r, w, np.arange(n))
    Lc = np.linalg.cholesky(B)
    F = np.tril(r["B"]) if uplo == "L" else np.triu(r["B"])
    G = Lc if uplo == "L" else Lc.conj().T
    assert np.abs(F - G).max() <= 100 * n * EPS * np.abs(B).max()
    check_generalized(itype, A, B, M.zhegeig(itype, "V", "I", uplo, A, B, il=3, iu=30), w,
                      np.arange(2, 30))
    rp = M.zhpgeig(itype, "V", "A", uplo, _cpack(A, uplo), _cpack(B, uplo), n)
    check_generalized(itype, A, B, rp, w, np.arange(n))
    if _have_ref():
        ref = oracle.ref_zhegeig(itype, "V", "A", uplo, A, B)
        assert np.abs(ref["W"] - r["W"]).max() <= 50 * n * EPS * max(np.abs(w).max(), 1.0)
