"""B200-native MRRR tridiagonal eigensolver (drop-in for MR3-SMP's ``mrrr``).

Python mirror of the reference's entry point ``mrrr(jobz, range, n, D, E, vl,
vu, il, iu, tryrac, m, W, Z, ldz, Zsupp)`` (INCLUDE/mrrr.h:62-65), backed by
the in-tree shared library ``lib/libmr3b200.so`` (C host library + sm_100a
kernels).  There is no CPU fallback: if the library cannot be loaded, every
call raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

__all__ = ["mrrr", "mrrr_batched", "mrrr_batched_device", "lib", "last_launches", "MR3Error"]

LIB_PATH = _build.LIB
_pd = C.POINTER(C.c_double)
_pi = C.POINTER(C.c_int)


class MR3Error(RuntimeError):
    """Raised when the native library is missing or a call fails."""


class HostProb(C.Structure):
    """Mirror of ``mr3_host_prob`` in include/mr3_b200.h."""
    _fields_ = [("jobz", C.c_char), ("range", C.c_char), ("n", C.c_int), ("il", C.c_int),
                ("iu", C.c_int), ("tryrac", C.c_int), ("ldz", C.c_int), ("vl", C.c_double),
                ("vu", C.c_double), ("D", _pd), ("E", _pd), ("W", _pd), ("Z", _pd),
                ("Zsupp", _pi), ("m", C.c_int), ("info", C.c_int), ("vl_out", C.c_double),
                ("vu_out", C.c_double), ("il_out", C.c_int), ("iu_out", C.c_int),
                ("tryrac_out", C.c_int)]


class CudaProb(C.Structure):
    """Mirror of ``mr3_cuda_prob`` in include/mr3_cuda.h (device pointers)."""
    _fields_ = [("n", C.c_int), ("jobz", C.c_int), ("range", C.c_int), ("il", C.c_int),
                ("iu", C.c_int), ("tryrac", C.c_int), ("ldz", C.c_int), ("vl", C.c_double),
                ("vu", C.c_double), ("D", C.c_void_p), ("E", C.c_void_p), ("W", C.c_void_p),
                ("Z", C.c_void_p), ("Zsupp", C.c_void_p), ("m", C.c_int), ("info", C.c_int),
                ("il_out", C.c_int), ("iu_out", C.c_int), ("tryrac_out", C.c_int),
                ("vl_out", C.c_double), ("vu_out", C.c_double)]


_lib: C.CDLL | None = None


def lib() -> C.CDLL:
    """The loaded native library (raises MR3Error if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise MR3Error(f"native library missing: {LIB_PATH} (run python -m mr3smp_b200.build)")
        L = C.CDLL(LIB_PATH)
        L.mrrr.restype = C.c_int
        L.mrrr.argtypes = [C.c_char_p, C.c_char_p, _pi, _pd, _pd, _pd, _pd, _pi, _pi, _pi, _pi,
                           _pd, _pd, _pi, _pi]
        L.mr3_batched.restype = C.c_int
        L.mr3_batched.argtypes = [C.c_int, C.POINTER(HostProb)]
        L.mr3_batched_device.restype = C.c_int
        L.mr3_batched_device.argtypes = [C.c_int, C.POINTER(CudaProb), C.c_void_p]
        L.dsyeig.restype = C.c_int
        L.dsyeig.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, _pi, _pd, _pi, _pd, _pd, _pi,
                             _pi, _pi, _pd, _pd, _pi]
        L.dspeig.restype = C.c_int
        L.dspeig.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, _pi, _pd, _pd, _pd, _pi, _pi,
                             _pi, _pd, _pd, _pi]
        L.dsygeig.restype = C.c_int
        L.dsygeig.argtypes = [_pi, C.c_char_p, C.c_char_p, C.c_char_p, _pi, _pd, _pi, _pd, _pi,
                              _pd, _pd, _pi, _pi, _pi, _pd]
        L.dspgeig.restype = C.c_int
        L.dspgeig.argtypes = [_pi, C.c_char_p, C.c_char_p, C.c_char_p, _pi, _pd, _pd, _pd, _pd,
                              _pi, _pi, _pi, _pd, _pd, _pi]
        # complex drivers: complex arrays as interleaved (re, im) doubles
        L.zheeig.restype = C.c_int
        L.zheeig.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, _pi, _pd, _pi, _pd, _pd, _pi,
                             _pi, _pi, _pd, _pd, _pi]
        L.zhpeig.restype = C.c_int
        L.zhpeig.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, _pi, _pd, _pd, _pd, _pi, _pi,
                             _pi, _pd, _pd, _pi]
        L.zhegeig.restype = C.c_int
        L.zhegeig.argtypes = [_pi, C.c_char_p, C.c_char_p, C.c_char_p, _pi, _pd, _pi, _pd, _pi,
                              _pd, _pd, _pi, _pi, _pi, _pd]
        L.zhpgeig.restype = C.c_int
        L.zhpgeig.argtypes = [_pi, C.c_char_p, C.c_char_p, C.c_char_p, _pi, _pd, _pd, _pd, _pd,
                              _pi, _pi, _pi, _pd, _pd, _pi]
        L.mr3_last_launches.restype = C.c_longlong
        L.mr3_last_error.restype = C.c_char_p
        _lib = L
    return _lib


def last_launches() -> int:
    """Kernels launched by this thread's last solve."""
    return int(lib().mr3_last_launches())


def last_error() -> str:
    return lib().mr3_last_error().decode()


def _ncols(jobz: str, rng: str, n: int, il: int, iu: int) -> int:
    if jobz[0] not in "Vv":
        return 1
    if rng[0] in "Ii":
        return max(iu - il + 1, 1)
    return max(n, 1)


def mrrr(jobz: str, rng: str, D, E, vl: float = 0.0, vu: float = 0.0, il: int = 1,
         iu: int = 1, tryrac: int = 0, ldz: int | None = None) -> dict:
    """Solve one tridiagonal problem through the C ABI ``mrrr()``.

    Arguments mean what they mean for the reference.  Returns a dict with
    ``info`` (return code), ``m``, ``W`` (m,), ``Z`` (n, m), ``Zsupp`` (2m,),
    the overwritten ``D``/``E`` and the refined ``vl, vu, il, iu, tryrac``.
    """
    L = lib()
    D = np.array(D, dtype=np.float64, copy=True)
    E = np.array(E, dtype=np.float64, copy=True)
    n = int(D.shape[0])
    if E.shape[0] < n:
        E = np.concatenate([E, np.zeros(n - E.shape[0])])
    ldz = n if ldz is None else int(ldz)
    want_z = jobz[0] in "Vv"
    W = np.zeros(max(n, 1))
    Z = np.zeros(_ncols(jobz, rng, n, il, iu) * (ldz if want_z else 1))
    Zs = np.zeros(2 * max(n, 1), dtype=np.int32)
    n_, vl_, vu_ = C.c_int(n), C.c_double(vl), C.c_double(vu)
    il_, iu_, tr_, m_, ldz_ = C.c_int(il), C.c_int(iu), C.c_int(tryrac), C.c_int(0), C.c_int(ldz)
    info = L.mrrr(jobz.encode(), rng.encode(), C.byref(n_), D.ctypes.data_as(_pd),
                  E.ctypes.data_as(_pd), C.byref(vl_), C.byref(vu_), C.byref(il_), C.byref(iu_),
                  C.byref(tr_), C.byref(m_), W.ctypes.data_as(_pd), Z.ctypes.data_as(_pd),
                  C.byref(ldz_), Zs.ctypes.data_as(_pi))
    m = m_.value if info == 0 else 0
    out = dict(info=info, m=m, W=W[:m].copy(), D=D, E=E, vl=vl_.value, vu=vu_.value,
               il=il_.value, iu=iu_.value, tryrac=tr_.value)
    if want_z:
        out["Z"] = Z[: ldz * m].reshape(m, ldz).T[:n].copy() if m > 0 else np.zeros((n, 0))
        out["Zsupp"] = Zs[: 2 * m].copy()
    return out


def dsyeig(jobz: str, rng: str, uplo: str, A, vl: float = 0.0, vu: float = 0.0, il: int = 1,
           iu: int = 1, lda: int | None = None, ldz: int | None = None) -> dict:
    """Eigenpairs of a dense symmetric matrix through the C ABI ``dsyeig()``.

    ``A`` is an (n, n) array of which the ``uplo`` triangle is read.  Returns
    a dict with ``info``, ``m``, ``W`` (m,), ``Z`` (n, m) for jobz "V", and the
    refined ``vl, vu, il, iu``.
    """
    L = lib()
    A = np.asarray(A, dtype=np.float64)
    n = int(A.shape[0])
    lda = n if lda is None else int(lda)
    Ah = np.zeros(lda * max(n, 1))
    if n > 0 and lda > 0:
        r = min(n, lda)   # (lda < n is an argument error the library reports)
        Ah.reshape(n, lda)[:, :r] = A.T[:, :r]   # column-major, leading dimension lda
    ldz = n if ldz is None else int(ldz)
    want_z = jobz[0] in "Vv"
    W = np.zeros(max(n, 1))
    Z = np.zeros(_ncols(jobz, rng, n, il, iu) * (ldz if want_z else 1))
    n_, lda_, ldz_ = C.c_int(n), C.c_int(lda), C.c_int(ldz)
    vl_, vu_, il_, iu_, m_ = C.c_double(vl), C.c_double(vu), C.c_int(il), C.c_int(iu), C.c_int(0)
    info = L.dsyeig(jobz.encode(), rng.encode(), uplo.encode(), C.byref(n_),
                    Ah.ctypes.data_as(_pd), C.byref(lda_), C.byref(vl_), C.byref(vu_),
                    C.byref(il_), C.byref(iu_), C.byref(m_), W.ctypes.data_as(_pd),
                    Z.ctypes.data_as(_pd), C.byref(ldz_))
    m = m_.value if info == 0 else 0
    out = dict(info=info, m=m, W=W[:m].copy(), vl=vl_.value, vu=vu_.value, il=il_.value,
               iu=iu_.value)
    if want_z:
        out["Z"] = Z[: ldz * m].reshape(m, ldz).T[:n].copy() if m > 0 else np.zeros((n, 0))
    return out


def pack(A, uplo: str):
    """The uplo triangle of a square array in LAPACK packed storage."""
    A = np.asarray(A, dtype=np.float64)
    n = A.shape[0]
    if uplo[0] in "Ll":
        return np.concatenate([A[j:, j] for j in range(n)]) if n else np.zeros(0)
    return np.concatenate([A[: j + 1, j] for j in range(n)]) if n else np.zeros(0)


def dspeig(jobz: str, rng: str, uplo: str, AP, n: int, vl: float = 0.0, vu: float = 0.0,
           il: int = 1, iu: int = 1, ldz: int | None = None) -> dict:
    """``dspeig()``: dsyeig with A in packed storage (``AP``, see :func:`pack`)."""
    L = lib()
    AP = np.array(AP, dtype=np.float64, copy=True)
    ldz = n if ldz is None else int(ldz)
    want_z = jobz[0] in "Vv"
    W = np.zeros(max(n, 1))
    Z = np.zeros(_ncols(jobz, rng, n, il, iu) * (ldz if want_z else 1))
    n_, ldz_ = C.c_int(n), C.c_int(ldz)
    vl_, vu_, il_, iu_, m_ = C.c_double(vl), C.c_double(vu), C.c_int(il), C.c_int(iu), C.c_int(0)
    info = L.dspeig(jobz.encode(), rng.encode(), uplo.encode(), C.byref(n_),
                    AP.ctypes.data_as(_pd), C.byref(vl_), C.byref(vu_), C.byref(il_),
                    C.byref(iu_), C.byref(m_), W.ctypes.data_as(_pd), Z.ctypes.data_as(_pd),
                    C.byref(ldz_))
    m = m_.value if info == 0 else 0
    out = dict(info=info, m=m, W=W[:m].copy(), vl=vl_.value, vu=vu_.value, il=il_.value,
               iu=iu_.value)
    if want_z:
        out["Z"] = Z[: ldz * m].reshape(m, ldz).T[:n].copy() if m > 0 else np.zeros((n, 0))
    return out


def dsygeig(itype: int, jobz: str, rng: str, uplo: str, A, B, vl: float = 0.0, vu: float = 0.0,
            il: int = 1, iu: int = 1) -> dict:
    """``dsygeig()``: the generalized problem (itype 1 A x = l B x, 2 A B x = l x,
    3 B A x = l x).  Returns ``info, m, W``, the eigenvectors ``Z`` (n, m) for
    jobz "V" (the library returns them in A) and ``B`` (its Cholesky factor)."""
    L = lib()
    A = np.asarray(A, dtype=np.float64)
    n = int(A.shape[0])
    Af = np.array(A.T, dtype=np.float64, copy=True).reshape(-1)
    Bf = np.array(np.asarray(B, dtype=np.float64).T, copy=True).reshape(-1)
    W = np.zeros(max(n, 1))
    it_, n_, lda_, ldb_ = C.c_int(itype), C.c_int(n), C.c_int(n), C.c_int(n)
    vl_, vu_, il_, iu_, m_ = C.c_double(vl), C.c_double(vu), C.c_int(il), C.c_int(iu), C.c_int(0)
    info = L.dsygeig(C.byref(it_), jobz.encode(), rng.encode(), uplo.encode(), C.byref(n_),
                     Af.ctypes.data_as(_pd), C.byref(lda_), Bf.ctypes.data_as(_pd),
                     C.byref(ldb_), C.byref(vl_), C.byref(vu_), C.byref(il_), C.byref(iu_),
                     C.byref(m_), W.ctypes.data_as(_pd))
    m = m_.value if info == 0 else 0
    out = dict(info=info, m=m, W=W[:m].copy(), vl=vl_.value, vu=vu_.value, il=il_.value,
               iu=iu_.value, B=Bf.reshape(max(n, 1), n).T.copy() if n else Bf)
    if jobz[0] in "Vv":
        out["Z"] = Af[: n * m].reshape(m, n).T.copy() if m > 0 else np.zeros((n, 0))
    return out


def dspgeig(itype: int, jobz: str, rng: str, uplo: str, AP, BP, n: int, vl: float = 0.0,
            vu: float = 0.0, il: int = 1, iu: int = 1, ldz: int | None = None) -> dict:
    """``dspgeig()``: dsygeig with A and B in packed storage; ``BP`` returns the
    packed Cholesky factor."""
    L = lib()
    AP = np.array(AP, dtype=np.float64, copy=True)
    BP = np.array(BP, dtype=np.float64, copy=True)
    ldz = n if ldz is None else int(ldz)
    want_z = jobz[0] in "Vv"
    W = np.zeros(max(n, 1))
    Z = np.zeros(_ncols(jobz, rng, n, il, iu) * (ldz if want_z else 1))
    it_, n_, ldz_ = C.c_int(itype), C.c_int(n), C.c_int(ldz)
    vl_, vu_, il_, iu_, m_ = C.c_double(vl), C.c_double(vu), C.c_int(il), C.c_int(iu), C.c_int(0)
    info = L.dspgeig(C.byref(it_), jobz.encode(), rng.encode(), uplo.encode(), C.byref(n_),
                     AP.ctypes.data_as(_pd), BP.ctypes.data_as(_pd), C.byref(vl_), C.byref(vu_),
                     C.byref(il_), C.byref(iu_), C.byref(m_), W.ctypes.data_as(_pd),
                     Z.ctypes.data_as(_pd), C.byref(ldz_))
    m = m_.value if info == 0 else 0
    out = dict(info=info, m=m, W=W[:m].copy(), vl=vl_.value, vu=vu_.value, il=il_.value,
               iu=iu_.value, BP=BP)
    if want_z:
        out["Z"] = Z[: ldz * m].reshape(m, ldz).T[:n].copy() if m > 0 else np.zeros((n, 0))
    return out


def _zcols(jobz, rng, n, il, iu, ldz):
    return np.zeros(_ncols(jobz, rng, n, il, iu) * (ldz if jobz[0] in "Vv" else 1),
                    dtype=np.complex128)


def _zout(info, m_, W, vl_, vu_, il_, iu_):
    m = m_.value if info == 0 else 0
    return m, dict(info=info, m=m, W=W[:m].copy(), vl=vl_.value, vu=vu_.value, il=il_.value,
                   iu=iu_.value)


def zheeig(jobz: str, rng: str, uplo: str, A, vl: float = 0.0, vu: float = 0.0, il: int = 1,
           iu: int = 1, lda: int | None = None, ldz: int | None = None) -> dict:
    """``zheeig()``: eigenpairs of a dense Hermitian matrix (``A`` complex
    (n, n), the ``uplo`` triangle read); ``Z`` (n, m) complex for jobz "V"."""
    L = lib()
    A = np.asarray(A, dtype=np.complex128)
    n = int(A.shape[0])
    lda = n if lda is None else int(lda)
    Ah = np.zeros(lda * max(n, 1), dtype=np.complex128)
    if n > 0 and lda > 0:
        r = min(n, lda)
        Ah.reshape(n, lda)[:, :r] = A.T[:, :r]
    ldz = n if ldz is None else int(ldz)
    W, Z = np.zeros(max(n, 1)), _zcols(jobz, rng, n, il, iu, ldz)
    n_, lda_, ldz_ = C.c_int(n), C.c_int(lda), C.c_int(ldz)
    vl_, vu_, il_, iu_, m_ = C.c_double(vl), C.c_double(vu), C.c_int(il), C.c_int(iu), C.c_int(0)
    info = L.zheeig(jobz.encode(), rng.encode(), uplo.encode(), C.byref(n_),
                    Ah.ctypes.data_as(_pd), C.byref(lda_), C.byref(vl_), C.byref(vu_),
                    C.byref(il_), C.byref(iu_), C.byref(m_), W.ctypes.data_as(_pd),
                    Z.ctypes.data_as(_pd), C.byref(ldz_))
    m, out = _zout(info, m_, W, vl_, vu_, il_, iu_)
    if jobz[0] in "Vv":
        out["Z"] = Z[: ldz * m].reshape(m, ldz).T[:n].copy() if m > 0 else np.zeros((n, 0), complex)
    return out


def zhpeig(jobz: str, rng: str, uplo: str, AP, n: int, vl: float = 0.0, vu: float = 0.0,
           il: int = 1, iu: int = 1, ldz: int | None = None) -> dict:
    """``zhpeig()``: zheeig with A in packed storage (see :func:`pack`)."""
    L = lib()
    AP = np.array(AP, dtype=np.complex128, copy=True)
    ldz = n if ldz is None else int(ldz)
    W, Z = np.zeros(max(n, 1)), _zcols(jobz, rng, n, il, iu, ldz)
    n_, ldz_ = C.c_int(n), C.c_int(ldz)
    vl_, vu_, il_, iu_, m_ = C.c_double(vl), C.c_double(vu), C.c_int(il), C.c_int(iu), C.c_int(0)
    info = L.zhpeig(jobz.encode(), rng.encode(), uplo.encode(), C.byref(n_),
                    AP.ctypes.data_as(_pd), C.byref(vl_), C.byref(vu_), C.byref(il_),
                    C.byref(iu_), C.byref(m_), W.ctypes.data_as(_pd), Z.ctypes.data_as(_pd),
                    C.byref(ldz_))
    m, out = _zout(info, m_, W, vl_, vu_, il_, iu_)
    if jobz[0] in "Vv":
        out["Z"] = Z[: ldz * m].reshape(m, ldz).T[:n].copy() if m > 0 else np.zeros((n, 0), complex)
    return out


def zhegeig(itype: int, jobz: str, rng: str, uplo: str, A, B, vl: float = 0.0, vu: float = 0.0,
            il: int = 1, iu: int = 1) -> dict:
    """``zhegeig()``: the generalized Hermitian-definite problem; eigenvectors
    ``Z`` (returned in A by the library) and ``B`` (its Cholesky factor)."""
    L = lib()
    A = np.asarray(A, dtype=np.complex128)
    n = int(A.shape[0])
    Af = np.array(A.T, dtype=np.complex128, copy=True).reshape(-1)
    Bf = np.array(np.asarray(B, dtype=np.complex128).T, copy=True).reshape(-1)
    W = np.zeros(max(n, 1))
    it_, n_, lda_, ldb_ = C.c_int(itype), C.c_int(n), C.c_int(n), C.c_int(n)
    vl_, vu_, il_, iu_, m_ = C.c_double(vl), C.c_double(vu), C.c_int(il), C.c_int(iu), C.c_int(0)
    info = L.zhegeig(C.byref(it_), jobz.encode(), rng.encode(), uplo.encode(), C.byref(n_),
                     Af.ctypes.data_as(_pd), C.byref(lda_), Bf.ctypes.data_as(_pd),
                     C.byref(ldb_), C.byref(vl_), C.byref(vu_), C.byref(il_), C.byref(iu_),
                     C.byref(m_), W.ctypes.data_as(_pd))
    m, out = _zout(info, m_, W, vl_, vu_, il_, iu_)
    out["B"] = Bf.reshape(max(n, 1), n).T.copy() if n else Bf
    if jobz[0] in "Vv":
        out["Z"] = Af[: n * m].reshape(m, n).T.copy() if m > 0 else np.zeros((n, 0), complex)
    return out


def zhpgeig(itype: int, jobz: str, rng: str, uplo: str, AP, BP, n: int, vl: float = 0.0,
            vu: float = 0.0, il: int = 1, iu: int = 1, ldz: int | None = None) -> dict:
    """``zhpgeig()``: zhegeig with A and B packed; ``BP`` returns the packed
    Cholesky factor."""
    L = lib()
    AP = np.array(AP, dtype=np.complex128, copy=True)
    BP = np.array(BP, dtype=np.complex128, copy=True)
    ldz = n if ldz is None else int(ldz)
    W, Z = np.zeros(max(n, 1)), _zcols(jobz, rng, n, il, iu, ldz)
    it_, n_, ldz_ = C.c_int(itype), C.c_int(n), C.c_int(ldz)
    vl_, vu_, il_, iu_, m_ = C.c_double(vl), C.c_double(vu), C.c_int(il), C.c_int(iu), C.c_int(0)
    info = L.zhpgeig(C.byref(it_), jobz.encode(), rng.encode(), uplo.encode(), C.byref(n_),
                     AP.ctypes.data_as(_pd), BP.ctypes.data_as(_pd), C.byref(vl_), C.byref(vu_),
                     C.byref(il_), C.byref(iu_), C.byref(m_), W.ctypes.data_as(_pd),
                     Z.ctypes.data_as(_pd), C.byref(ldz_))
    m, out = _zout(info, m_, W, vl_, vu_, il_, iu_)
    out["BP"] = BP
    if jobz[0] in "Vv":
        out["Z"] = Z[: ldz * m].reshape(m, ldz).T[:n].copy() if m > 0 else np.zeros((n, 0), complex)
    return out


def mrrr_batched(problems: list[dict]) -> list[dict]:
    """Solve a list of problems in one batched device pass (host arrays).

    Each problem is a dict with keys ``jobz, range, D, E`` and optionally
    ``vl, vu, il, iu, tryrac``.  Returns one result dict per problem, as
    :func:`mrrr` does.
    """
    L = lib()
    P = len(problems)
    arr = (HostProb * P)()
    keep = []
    for k, pb in enumerate(problems):
        D = np.array(pb["D"], dtype=np.float64, copy=True)
        n = int(D.shape[0])
        E = np.array(pb["E"], dtype=np.float64, copy=True)
        if E.shape[0] < n:
            E = np.concatenate([E, np.zeros(n - E.shape[0])])
        jz, rg = pb["jobz"], pb["range"]
        il, iu = int(pb.get("il", 1)), int(pb.get("iu", 1))
        want_z = jz[0] in "Vv"
        W = np.zeros(max(n, 1))
        Z = np.zeros(_ncols(jz, rg, n, il, iu) * (n if want_z else 1))
        Zs = np.zeros(2 * max(n, 1), dtype=np.int32)
        keep.append((D, E, W, Z, Zs, n, jz))
        h = arr[k]
        h.jobz, h.range, h.n, h.il, h.iu = jz[0].encode(), rg[0].encode(), n, il, iu
        h.tryrac, h.ldz = int(pb.get("tryrac", 0)), n
        h.vl, h.vu = float(pb.get("vl", 0.0)), float(pb.get("vu", 0.0))
        h.D, h.E, h.W = D.ctypes.data_as(_pd), E.ctypes.data_as(_pd), W.ctypes.data_as(_pd)
        h.Z, h.Zsupp = Z.ctypes.data_as(_pd), Zs.ctypes.data_as(_pi)
    L.mr3_batched(P, arr)
    res = []
    for k in range(P):
        h = arr[k]
        D, E, W, Z, Zs, n, jz = keep[k]
        m = h.m if h.info == 0 else 0
        out = dict(info=h.info, m=m, W=W[:m].copy(), D=D, E=E, vl=h.vl_out, vu=h.vu_out,
                   il=h.il_out, iu=h.iu_out, tryrac=h.tryrac_out)
        if jz[0] in "Vv":
            out["Z"] = Z[: n * m].reshape(m, n).T.copy() if m > 0 else np.zeros((n, 0))
            out["Zsupp"] = Zs[: 2 * m].copy()
        res.append(out)
    return res


_JOB = {"N": 0, "V": 1, "C": 2}
_RANGE = {"A": 1, "V": 2, "I": 3}


def mrrr_batched_device(problems: list[dict], stream: int | None = None) -> tuple[int, list]:
    """Batched solve on device-resident torch tensors (float64 / int32).

    Each problem dict holds ``jobz, range`` and CUDA tensors ``D, E, W`` (n),
    ``Z`` (m_max*n, column-major, ldz = n) and ``Zsupp`` (2*m_max) for jobz V.
    Returns (rc, list of CudaProb results).
    """
    L = lib()
    P = len(problems)
    arr = (CudaProb * P)()
    for k, pb in enumerate(problems):
        arr[k] = device_request(pb)
    rc = L.mr3_batched_device(P, arr, C.c_void_p(stream) if stream else None)
    return rc, [arr[k] for k in range(P)]


class Solver:
    """A solver context on one device (wraps ``mr3_cuda_ctx``).

    ``solve(probs, stream)`` runs one batched pass over ``CudaProb`` records
    whose arrays live on the device; ``profile(True)`` turns on per-kernel
    CUDA-event timing and the device work counters, read back with
    ``profile_read()``.
    """

    KERNEL_GROUPS = ("bisect", "refine_root", "newrrr", "refine_cl", "singletons", "other")

    def __init__(self, device: int = 0):
        L = lib()
        L.mr3_cuda_ctx_create.restype = C.c_int
        L.mr3_cuda_ctx_create.argtypes = [C.c_int, C.POINTER(C.c_void_p)]
        L.mr3_cuda_ctx_destroy.argtypes = [C.c_void_p]
        L.mr3_cuda_solve.restype = C.c_int
        L.mr3_cuda_solve.argtypes = [C.c_void_p, C.c_int, C.POINTER(CudaProb), C.c_void_p]
        L.mr3_cuda_profile.argtypes = [C.c_void_p, C.c_int]
        L.mr3_cuda_profile_read.restype = C.c_int
        L.mr3_cuda_profile_read.argtypes = [C.c_void_p, C.c_int, C.c_char_p,
                                            C.POINTER(C.c_double), C.POINTER(C.c_longlong),
                                            C.POINTER(C.c_ulonglong)]
        L.mr3_cuda_last_launches.restype = C.c_longlong
        L.mr3_cuda_last_launches.argtypes = [C.c_void_p]
        L.mr3_cuda_last_error.restype = C.c_char_p
        L.mr3_cuda_last_error.argtypes = [C.c_void_p]
        self._L = L
        self._ctx = C.c_void_p()
        if L.mr3_cuda_ctx_create(int(device), C.byref(self._ctx)) != 0:
            raise MR3Error("could not create a solver context on device %d" % device)

    def close(self):
        if self._ctx:
            self._L.mr3_cuda_ctx_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve(self, probs, stream: int | None = None) -> int:
        """probs: a ctypes array of CudaProb (device pointers)."""
        rc = self._L.mr3_cuda_solve(self._ctx, len(probs), probs,
                                    C.c_void_p(stream) if stream else None)
        if rc != 0:
            raise MR3Error("mr3_cuda_solve failed: " + self._L.mr3_cuda_last_error(self._ctx).decode())
        return rc

    def last_launches(self) -> int:
        return int(self._L.mr3_cuda_last_launches(self._ctx))

    def profile(self, on: int | bool):
        """0/False off; 1/True per-kernel events and work counters; 2 the
        same with the streams serialised (each kernel's time its own)."""
        self._L.mr3_cuda_profile(self._ctx, int(on))

    def profile_read(self):
        """-> (dict kernel -> (ms_total, launches), counters[6][4])."""
        mx = 64
        names = C.create_string_buffer(32 * mx)
        ms = (C.c_double * mx)()
        cnt = (C.c_longlong * mx)()
        ctr = (C.c_ulonglong * 24)()
        k = self._L.mr3_cuda_profile_read(self._ctx, mx, names, ms, cnt, ctr)
        raw = names.raw
        kern = {}
        for i in range(k):
            nm = raw[32 * i: 32 * i + 32].split(b"\0", 1)[0].decode()
            kern[nm] = (float(ms[i]), int(cnt[i]))
        counters = [[int(ctr[4 * g + j]) for j in range(4)] for g in range(6)]
        return kern, counters


def _host_request(pb: dict, pinned: bool = False, arrays=None):
    """Build an HostProb for one problem dict; returns (struct, arrays kept
    alive).  ``arrays`` (D, E, W, Z, Zsupp of a finished request of the same
    shape, see Server.poll(raw=True)) are reused instead of new buffers."""
    def alloc(n, dtype):
        if arrays is not None:
            return alloc.pool.pop(0)
        if pinned:
            import torch
            t = torch.empty(max(n, 1), dtype=torch.float64 if dtype == np.float64 else torch.int32,
                            pin_memory=True)
            return t.numpy()
        return np.zeros(max(n, 1), dtype=dtype)
    if arrays is not None:
        alloc.pool = list(arrays[:5])
    n = int(len(pb["D"]))
    D = alloc(n, np.float64)
    D[:n] = pb["D"]
    E = alloc(n, np.float64)
    E[:] = 0.0
    E[: min(n, len(pb["E"]))] = np.asarray(pb["E"], dtype=np.float64)[:n]
    jz, rg = pb["jobz"], pb["range"]
    il, iu = int(pb.get("il", 1)), int(pb.get("iu", 1))
    want_z = jz[0] in "Vv"
    W = alloc(n, np.float64)
    Z = alloc(_ncols(jz, rg, n, il, iu) * n if want_z else 1, np.float64)
    Zs = alloc(2 * n, np.int32)
    h = HostProb()
    h.jobz, h.range, h.n, h.il, h.iu = jz[0].encode(), rg[0].encode(), n, il, iu
    h.tryrac, h.ldz = int(pb.get("tryrac", 0)), n
    h.vl, h.vu = float(pb.get("vl", 0.0)), float(pb.get("vu", 0.0))
    h.D, h.E, h.W = D.ctypes.data_as(_pd), E.ctypes.data_as(_pd), W.ctypes.data_as(_pd)
    h.Z, h.Zsupp = Z.ctypes.data_as(_pd), Zs.ctypes.data_as(_pi)
    return h, (D, E, W, Z, Zs, n, jz)


def _host_result(h, keep) -> dict:
    D, E, W, Z, Zs, n, jz = keep
    m = h.m if h.info == 0 else 0
    out = dict(info=h.info, m=m, W=W[:m].copy(), D=D[:n].copy(), E=E[:n].copy(), vl=h.vl_out,
               vu=h.vu_out, il=h.il_out, iu=h.iu_out, tryrac=h.tryrac_out)
    if jz[0] in "Vv":
        out["Z"] = Z[: n * m].reshape(m, n).T.copy() if m > 0 else np.zeros((n, 0))
        out["Zsupp"] = Zs[: 2 * m].copy()
    return out


def device_request(pb: dict):
    """A ``CudaProb`` for one problem dict whose ``D, E, W`` (and for jobz V
    ``Z``, ``Zsupp``) are CUDA tensors (float64 / int32, Z column-major with
    ldz = n); the tensors must outlive the request."""
    q = CudaProb()
    q.n = int(pb["D"].numel())
    q.jobz = _JOB[pb["jobz"][0].upper()]
    q.range = _RANGE[pb["range"][0].upper()]
    q.il, q.iu, q.tryrac = int(pb.get("il", 1)), int(pb.get("iu", 1)), int(pb.get("tryrac", 0))
    q.vl, q.vu = float(pb.get("vl", 0.0)), float(pb.get("vu", 0.0))
    q.ldz = q.n
    q.D, q.E, q.W = pb["D"].data_ptr(), pb["E"].data_ptr(), pb["W"].data_ptr()
    q.Z = pb["Z"].data_ptr() if pb.get("Z") is not None else None
    q.Zsupp = pb["Zsupp"].data_ptr() if pb.get("Zsupp") is not None else None
    return q


class Server:
    """Serving handle (mr3_server_*): requests solved with continuous batching.

    ``submit(problem)`` takes a problem dict as :func:`mrrr_batched` does
    (host arrays) and returns a ticket; ``submit_device(problem)`` takes one
    whose arrays are CUDA tensors (results stay resident on the device);
    ``poll(ticket, wait)`` returns ``(result, latency_ms)`` once the request
    is done (``(None, None)`` while pending).  Results are those of a call
    alone.
    """

    def __init__(self, device: int = 0, budget_bytes: int = 0, pinned: bool = False):
        L = lib()
        L.mr3_server_create.restype = C.c_int
        L.mr3_server_create.argtypes = [C.c_int, C.c_size_t, C.POINTER(C.c_void_p)]
        L.mr3_server_submit.restype = C.c_longlong
        L.mr3_server_submit.argtypes = [C.c_void_p, C.POINTER(HostProb)]
        L.mr3_server_submit_device.restype = C.c_longlong
        L.mr3_server_submit_device.argtypes = [C.c_void_p, C.POINTER(CudaProb)]
        L.mr3_server_poll.restype = C.c_int
        L.mr3_server_poll.argtypes = [C.c_void_p, C.c_longlong, C.c_int, C.POINTER(C.c_double)]
        L.mr3_server_timing.restype = C.c_int
        L.mr3_server_timing.argtypes = [C.c_void_p, C.c_longlong, C.POINTER(C.c_double),
                                        C.POINTER(C.c_double)]
        L.mr3_server_stats.restype = C.c_int
        L.mr3_server_stats.argtypes = [C.c_void_p, C.POINTER(C.c_longlong),
                                       C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
        L.mr3_server_stats2.restype = C.c_int
        L.mr3_server_stats2.argtypes = [C.c_void_p, C.POINTER(C.c_longlong), C.POINTER(C.c_int),
                                        C.POINTER(C.c_size_t)]
        L.mr3_server_destroy.argtypes = [C.c_void_p]
        self._L = L
        self._pinned = pinned
        self._h = C.c_void_p()
        rc = L.mr3_server_create(device, budget_bytes, C.byref(self._h))
        if rc != 0:
            raise MR3Error(f"mr3_server_create failed ({rc})")
        self._live = {}

    def submit(self, problem: dict, arrays=None) -> int:
        h, keep = _host_request(problem, self._pinned, arrays)
        t = self._L.mr3_server_submit(self._h, C.byref(h))
        if t < 1:
            raise MR3Error(f"mr3_server_submit refused the request ({t})")
        self._live[t] = (h, keep)
        return t

    def submit_device(self, problem: dict, req: CudaProb | None = None) -> int:
        """A device request: ``problem`` as for :func:`device_request` (or a
        prepared ``req``); the tensors must stay alive until polled."""
        q = req if req is not None else device_request(problem)
        t = self._L.mr3_server_submit_device(self._h, C.byref(q))
        if t < 1:
            raise MR3Error(f"mr3_server_submit_device refused the request ({t})")
        self._live[t] = (q, None)
        return t

    def poll(self, ticket: int, wait: bool = True, raw: bool = False):
        """(result dict, latency ms), or with raw=True ((info, m, arrays),
        latency ms) where arrays can be passed to submit() again.  For a
        device request the result is ``{"info", "m", ...}`` (the arrays are
        the caller's tensors)."""
        lat = C.c_double(0.0)
        rc = self._L.mr3_server_poll(self._h, ticket, 1 if wait else 0, C.byref(lat))
        if rc < 0:
            raise MR3Error(f"unknown ticket {ticket}")
        if rc == 0:
            return None, None
        h, keep = self._live.pop(ticket)
        if keep is None:   # device request
            r = dict(info=h.info, m=h.m, vl=h.vl_out, vu=h.vu_out, il=h.il_out, iu=h.iu_out,
                     tryrac=h.tryrac_out)
            return ((h.info, h.m, None) if raw else r), lat.value
        if raw:
            return (h.info, h.m, keep[:5]), lat.value
        return _host_result(h, keep), lat.value

    def timing(self, ticket: int):
        """(queued ms, solve ms) of a done request."""
        a, b = C.c_double(0.0), C.c_double(0.0)
        if self._L.mr3_server_timing(self._h, ticket, C.byref(a), C.byref(b)) != 1:
            return None
        return a.value, b.value

    def stats(self):
        a, b, c = C.c_longlong(), C.c_longlong(), C.c_longlong()
        self._L.mr3_server_stats(self._h, C.byref(a), C.byref(b), C.byref(c))
        o, ln, bud = C.c_longlong(), C.c_int(), C.c_size_t()
        self._L.mr3_server_stats2(self._h, C.byref(o), C.byref(ln), C.byref(bud))
        return {"submitted": a.value, "solved": b.value, "batches": c.value,
                "batches_overlapping_others": o.value, "lanes": ln.value,
                "budget_bytes": bud.value}

    def close(self):
        if self._h:
            self._L.mr3_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def device_batch(host_problems, device: str = "cuda", with_z: bool = True):
    """Lay out a list of (D, E) numpy pairs on the device for batched solves.

    Returns (records, tensors) where ``records`` is a ctypes CudaProb array for
    jobz V (or N when ``with_z`` is False), range A, and ``tensors`` holds the
    torch buffers: D0/E0 (pristine inputs), D/E (work copies, overwritten by
    the solve), W, Z (sum of n^2 doubles, column-major per problem), Zsupp.
    """
    import torch
    ns = [len(D) for D, E in host_problems]
    offs = np.concatenate([[0], np.cumsum(ns)]).astype(np.int64)
    N = int(offs[-1])
    zoffs = np.concatenate([[0], np.cumsum([n * n for n in ns])]).astype(np.int64)
    D0 = torch.from_numpy(np.concatenate([np.asarray(D, np.float64) for D, E in host_problems])).to(device)
    E0 = torch.from_numpy(np.concatenate([np.asarray(E, np.float64) for D, E in host_problems])).to(device)
    D = D0.clone()
    E = E0.clone()
    W = torch.zeros(N, dtype=torch.float64, device=device)
    Z = torch.empty(int(zoffs[-1]) if with_z else 1, dtype=torch.float64, device=device)
    Zs = torch.zeros(2 * N, dtype=torch.int32, device=device)
    recs = (CudaProb * len(ns))()
    for k, n in enumerate(ns):
        q = recs[k]
        q.n, q.jobz, q.range = n, (1 if with_z else 0), 1
        q.il = q.iu = 1
        q.ldz = n
        q.D = D.data_ptr() + 8 * int(offs[k])
        q.E = E.data_ptr() + 8 * int(offs[k])
        q.W = W.data_ptr() + 8 * int(offs[k])
        q.Z = (Z.data_ptr() + 8 * int(zoffs[k])) if with_z else None
        q.Zsupp = (Zs.data_ptr() + 8 * int(offs[k])) if with_z else None
    tens = dict(D0=D0, E0=E0, D=D, E=E, W=W, Z=Z, Zsupp=Zs, offs=offs, zoffs=zoffs, ns=ns)
    return recs, tens
