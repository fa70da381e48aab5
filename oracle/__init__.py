"""CPU oracle for the MRRR path (TEST INFRASTRUCTURE ONLY).

Loads two shared libraries built by ``oracle/Makefile``:

* ``_build/libmr3_oracle.so`` -- the C restatement in ``mr3_oracle.c`` of the
  reference's ``mrrr()`` (SRC/mrrr.c:87-296) and of the LAPACK kernels it calls;
* ``_ref/libmrrr_ref.so`` -- the reference's own C sources linked against
  scipy's bundled LAPACK (present only where the reference was built).

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline legs of
``bench.py`` import this package, and only as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libmr3_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmrrr_ref.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_pi = C.POINTER(C.c_int)
_pd = C.POINTER(C.c_double)

_libs: dict[str, C.CDLL] = {}


def build(force: bool = False) -> None:
    """Compile the oracle (and, where the reference sources exist, the reference)."""
    if force or not os.path.exists(ORACLE_SO):
        subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def _mrrr_sig(fn):
    fn.restype = C.c_int
    fn.argtypes = [C.c_char_p, C.c_char_p, _pi, _pd, _pd, _pd, _pd, _pi, _pi, _pi,
                   _pi, _pd, _pd, _pi, _pi]
    return fn


def lib() -> C.CDLL:
    """The oracle library (restatement)."""
    if "oracle" not in _libs:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        _mrrr_sig(L.or_mrrr)
        L.or_dlaneg.restype = C.c_int
        L.or_dlaneg.argtypes = [C.c_int, _dp, _dp, C.c_double, C.c_double, C.c_int]
        L.or_log.restype = C.c_double
        L.or_log.argtypes = [C.c_double]
        L.or_count_bisect.restype = C.c_int
        L.or_count_bisect.argtypes = [C.c_int, _dp, _dp, C.c_double, C.c_double]
        L.or_count_ijob1.restype = C.c_int
        L.or_count_ijob1.argtypes = [C.c_int, _dp, _dp, C.c_double, C.c_double]
        L.or_dlarrb.restype = None
        L.or_dlarrb.argtypes = [C.c_int, _dp, _dp, C.c_int, C.c_int, C.c_double, C.c_double,
                                C.c_int, _dp, _dp, _dp, _dp, _ip, C.c_double, C.c_double,
                                C.c_int, _pi]
        L.or_dlar1v.restype = None
        L.or_dlar1v.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, _dp, _dp, _dp, _dp,
                                C.c_double, C.c_double, _dp, C.c_int, _pi, _pd, _pd, _pi,
                                _ip, _pd, _pd, _pd, _dp]
        L.or_dlarrf.restype = None
        L.or_dlarrf.argtypes = [C.c_int, _dp, _dp, _dp, C.c_int, C.c_int, _dp, _dp, _dp,
                                C.c_double, C.c_double, C.c_double, C.c_double, _pd, _dp,
                                _dp, _dp, _pi]
        L.or_dlarnv2.restype = None
        L.or_dlarnv2.argtypes = [_ip, C.c_int, _dp]
        L.or_dlarrr.restype = C.c_int
        L.or_dlarrr.argtypes = [C.c_int, _dp, _dp]
        _libs["oracle"] = L
    return _libs["oracle"]


def ref_lib() -> C.CDLL | None:
    """The reference library built from the reference's own sources, if built."""
    if "ref" not in _libs:
        if not os.path.exists(REF_SO):
            return None
        os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
        L = C.CDLL(REF_SO)
        _mrrr_sig(L.mrrr)
        if hasattr(L, "dsyeig"):
            L.dsyeig.restype = C.c_int
            L.dsyeig.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, _pi, _pd, _pi, _pd, _pd,
                                 _pi, _pi, _pi, _pd, _pd, _pi]
            L.dspeig.restype = C.c_int
            L.dspeig.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, _pi, _pd, _pd, _pd, _pi,
                                 _pi, _pi, _pd, _pd, _pi]
            L.dsygeig.restype = C.c_int
            L.dsygeig.argtypes = [_pi, C.c_char_p, C.c_char_p, C.c_char_p, _pi, _pd, _pi, _pd,
                                  _pi, _pd, _pd, _pi, _pi, _pi, _pd]
            L.dspgeig.restype = C.c_int
            L.dspgeig.argtypes = [_pi, C.c_char_p, C.c_char_p, C.c_char_p, _pi, _pd, _pd, _pd,
                                  _pd, _pi, _pi, _pi, _pd, _pd, _pi]
        if hasattr(L, "zheeig"):
            # complex arrays are passed as interleaved (re, im) doubles
            L.zheeig.restype = C.c_int
            L.zheeig.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, _pi, _pd, _pi, _pd, _pd,
                                 _pi, _pi, _pi, _pd, _pd, _pi]
            L.zhpeig.restype = C.c_int
            L.zhpeig.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, _pi, _pd, _pd, _pd, _pi,
                                 _pi, _pi, _pd, _pd, _pi]
            L.zhegeig.restype = C.c_int
            L.zhegeig.argtypes = [_pi, C.c_char_p, C.c_char_p, C.c_char_p, _pi, _pd, _pi, _pd,
                                  _pi, _pd, _pd, _pi, _pi, _pi, _pd]
            L.zhpgeig.restype = C.c_int
            L.zhpgeig.argtypes = [_pi, C.c_char_p, C.c_char_p, C.c_char_p, _pi, _pd, _pd, _pd,
                                  _pd, _pi, _pi, _pi, _pd, _pd, _pi]
        _libs["ref"] = L
    return _libs["ref"]


def _call(fn, jobz, rng, D, E, vl=0.0, vu=0.0, il=1, iu=1, tryrac=0, ldz=None):
    D = np.array(D, dtype=np.float64, copy=True)
    E = np.array(E, dtype=np.float64, copy=True)
    n = D.shape[0]
    if E.shape[0] < n:
        E = np.concatenate([E, np.zeros(n - E.shape[0])])
    ldz = n if ldz is None else ldz
    want_z = jobz[0] in "Vv"
    W = np.zeros(max(n, 1))
    nz = max(n, 1)
    if want_z and rng[0] in "Ii":
        nz = iu - il + 1
    Z = np.zeros((nz if want_z else 1) * (ldz if want_z else 1))
    Zs = np.zeros(2 * max(n, 1), dtype=np.int32)
    n_ = C.c_int(n)
    vl_ = C.c_double(vl)
    vu_ = C.c_double(vu)
    il_ = C.c_int(il)
    iu_ = C.c_int(iu)
    tr_ = C.c_int(tryrac)
    m_ = C.c_int(0)
    ldz_ = C.c_int(ldz)
    info = fn(jobz.encode(), rng.encode(), C.byref(n_), D.ctypes.data_as(_pd),
              E.ctypes.data_as(_pd), C.byref(vl_), C.byref(vu_), C.byref(il_), C.byref(iu_),
              C.byref(tr_), C.byref(m_), W.ctypes.data_as(_pd), Z.ctypes.data_as(_pd),
              C.byref(ldz_), Zs.ctypes.data_as(_pi))
    m = m_.value
    out = dict(info=info, m=m, W=W[:m].copy(), D=D, E=E, vl=vl_.value, vu=vu_.value,
               il=il_.value, iu=iu_.value, tryrac=tr_.value)
    if want_z:
        out["Z"] = Z[: ldz * m].reshape(m, ldz).T[:n].copy() if m > 0 else np.zeros((n, 0))
        out["Zsupp"] = Zs[: 2 * m].copy()
    return out


def mrrr(jobz, rng, D, E, vl=0.0, vu=0.0, il=1, iu=1, tryrac=0, ldz=None):
    """Oracle solve with the reference's argument contract; returns a dict."""
    return _call(lib().or_mrrr, jobz, rng, D, E, vl, vu, il, iu, tryrac, ldz)


def ref_mrrr(jobz, rng, D, E, vl=0.0, vu=0.0, il=1, iu=1, tryrac=0, ldz=None,
             threads: int = 2):
    """The reference's own mrrr() (needs the _ref build)."""
    L = ref_lib()
    if L is None:
        raise RuntimeError("reference library not built (oracle/_ref)")
    os.environ["PMR_NUM_THREADS"] = str(threads)
    return _call(L.mrrr, jobz, rng, D, E, vl, vu, il, iu, tryrac, ldz)


def ref_dsyeig(jobz, rng, uplo, A, vl=0.0, vu=0.0, il=1, iu=1, threads: int = 2):
    """The reference's own dense driver dsyeig() (SRC/dense.c:151-232; needs
    the _ref build): scipy's LAPACK dsytrd/dormtr around the reference's
    mrrr().  A is an (n, n) array; returns info, m, W, Z, vl, vu, il, iu."""
    L = ref_lib()
    if L is None:
        raise RuntimeError("reference library not built (oracle/_ref)")
    os.environ["PMR_NUM_THREADS"] = str(threads)
    A = np.asarray(A, dtype=np.float64)
    n = A.shape[0]
    Af = np.array(A.T, dtype=np.float64, copy=True).reshape(-1)   # column-major
    want_z = jobz[0] in "Vv"
    W = np.zeros(max(n, 1))
    # the reference back-transforms Z (dormtr) for every jobz, so Z must hold
    # n x m doubles even when no eigenvectors are wanted
    Z = np.zeros(max(n, 1) * max(n, 1))
    n_, lda_, ldz_ = C.c_int(n), C.c_int(n), C.c_int(n)
    vl_, vu_, il_, iu_, m_ = C.c_double(vl), C.c_double(vu), C.c_int(il), C.c_int(iu), C.c_int(0)
    info = L.dsyeig(jobz.encode(), rng.encode(), uplo.encode(), C.byref(n_),
                    Af.ctypes.data_as(_pd), C.byref(lda_), C.byref(vl_), C.byref(vu_),
                    C.byref(il_), C.byref(iu_), C.byref(m_), W.ctypes.data_as(_pd),
                    Z.ctypes.data_as(_pd), C.byref(ldz_))
    m = m_.value
    out = dict(info=info, m=m, W=W[:m].copy(), vl=vl_.value, vu=vu_.value, il=il_.value,
               iu=iu_.value)
    if want_z:
        out["Z"] = Z[: n * m].reshape(m, n).T.copy() if m > 0 else np.zeros((n, 0))
    return out


def _ref(threads):
    L = ref_lib()
    if L is None:
        raise RuntimeError("reference library not built (oracle/_ref)")
    os.environ["PMR_NUM_THREADS"] = str(threads)
    return L


def ref_dspeig(jobz, rng, uplo, AP, n, vl=0.0, vu=0.0, il=1, iu=1, threads: int = 2):
    """The reference's dspeig() (SRC/dense.c:319-398), A packed in AP."""
    L = _ref(threads)
    AP = np.array(AP, dtype=np.float64, copy=True)
    W = np.zeros(max(n, 1))
    Z = np.zeros(max(n, 1) * max(n, 1))   # back-transformed for every jobz
    n_, ldz_ = C.c_int(n), C.c_int(n)
    vl_, vu_, il_, iu_, m_ = C.c_double(vl), C.c_double(vu), C.c_int(il), C.c_int(iu), C.c_int(0)
    info = L.dspeig(jobz.encode(), rng.encode(), uplo.encode(), C.byref(n_),
                    AP.ctypes.data_as(_pd), C.byref(vl_), C.byref(vu_), C.byref(il_),
                    C.byref(iu_), C.byref(m_), W.ctypes.data_as(_pd), Z.ctypes.data_as(_pd),
                    C.byref(ldz_))
    m = m_.value
    out = dict(info=info, m=m, W=W[:m].copy())
    if jobz[0] in "Vv":
        out["Z"] = Z[: n * m].reshape(m, n).T.copy() if m > 0 else np.zeros((n, 0))
    return out


def ref_dsygeig(itype, jobz, rng, uplo, A, B, vl=0.0, vu=0.0, il=1, iu=1, threads: int = 2):
    """The reference's dsygeig() (SRC/dense.c:236-313): eigenvectors in A."""
    L = _ref(threads)
    A = np.asarray(A, dtype=np.float64)
    n = A.shape[0]
    Af = np.array(A.T, dtype=np.float64, copy=True).reshape(-1)
    Bf = np.array(np.asarray(B, dtype=np.float64).T, copy=True).reshape(-1)
    W = np.zeros(max(n, 1))
    it_, n_, lda_, ldb_ = C.c_int(itype), C.c_int(n), C.c_int(n), C.c_int(n)
    vl_, vu_, il_, iu_, m_ = C.c_double(vl), C.c_double(vu), C.c_int(il), C.c_int(iu), C.c_int(0)
    info = L.dsygeig(C.byref(it_), jobz.encode(), rng.encode(), uplo.encode(), C.byref(n_),
                     Af.ctypes.data_as(_pd), C.byref(lda_), Bf.ctypes.data_as(_pd),
                     C.byref(ldb_), C.byref(vl_), C.byref(vu_), C.byref(il_), C.byref(iu_),
                     C.byref(m_), W.ctypes.data_as(_pd))
    m = m_.value
    out = dict(info=info, m=m, W=W[:m].copy())
    if jobz[0] in "Vv":
        out["Z"] = Af[: n * m].reshape(m, n).T.copy() if m > 0 else np.zeros((n, 0))
    return out


def ref_dspgeig(itype, jobz, rng, uplo, AP, BP, n, vl=0.0, vu=0.0, il=1, iu=1,
                threads: int = 2):
    """The reference's dspgeig() (SRC/dense.c:403-470)."""
    L = _ref(threads)
    AP = np.array(AP, dtype=np.float64, copy=True)
    BP = np.array(BP, dtype=np.float64, copy=True)
    W = np.zeros(max(n, 1))
    Z = np.zeros(max(n, 1) * max(n, 1))
    it_, n_, ldz_ = C.c_int(itype), C.c_int(n), C.c_int(n)
    vl_, vu_, il_, iu_, m_ = C.c_double(vl), C.c_double(vu), C.c_int(il), C.c_int(iu), C.c_int(0)
    info = L.dspgeig(C.byref(it_), jobz.encode(), rng.encode(), uplo.encode(), C.byref(n_),
                     AP.ctypes.data_as(_pd), BP.ctypes.data_as(_pd), C.byref(vl_), C.byref(vu_),
                     C.byref(il_), C.byref(iu_), C.byref(m_), W.ctypes.data_as(_pd),
                     Z.ctypes.data_as(_pd), C.byref(ldz_))
    m = m_.value
    out = dict(info=info, m=m, W=W[:m].copy())
    if jobz[0] in "Vv":
        out["Z"] = Z[: n * m].reshape(m, n).T.copy() if m > 0 else np.zeros((n, 0))
    return out


def _cpd(a):
    """A complex128 array's data as a double pointer (interleaved re, im)."""
    return a.ctypes.data_as(_pd)


def ref_zheeig(jobz, rng, uplo, A, vl=0.0, vu=0.0, il=1, iu=1, threads: int = 2):
    """The reference's zheeig() (SRC/dense.c:568-671; built with its
    COMPLEX_SUPPORTED switch): A is an (n, n) Hermitian array."""
    L = _ref(threads)
    A = np.asarray(A, dtype=np.complex128)
    n = A.shape[0]
    Af = np.array(A.T, dtype=np.complex128, copy=True).reshape(-1)
    W = np.zeros(max(n, 1))
    Z = np.zeros(max(n, 1) * max(n, 1), dtype=np.complex128)
    n_, lda_, ldz_ = C.c_int(n), C.c_int(n), C.c_int(n)
    vl_, vu_, il_, iu_, m_ = C.c_double(vl), C.c_double(vu), C.c_int(il), C.c_int(iu), C.c_int(0)
    info = L.zheeig(jobz.encode(), rng.encode(), uplo.encode(), C.byref(n_), _cpd(Af),
                    C.byref(lda_), C.byref(vl_), C.byref(vu_), C.byref(il_), C.byref(iu_),
                    C.byref(m_), W.ctypes.data_as(_pd), _cpd(Z), C.byref(ldz_))
    m = m_.value
    out = dict(info=info, m=m, W=W[:m].copy())
    if jobz[0] in "Vv":
        out["Z"] = Z[: n * m].reshape(m, n).T.copy() if m > 0 else np.zeros((n, 0), complex)
    return out


def ref_zhpeig(jobz, rng, uplo, AP, n, vl=0.0, vu=0.0, il=1, iu=1, threads: int = 2):
    """The reference's zhpeig() (packed Hermitian, SRC/dense.c:760-862)."""
    L = _ref(threads)
    AP = np.array(AP, dtype=np.complex128, copy=True)
    W = np.zeros(max(n, 1))
    Z = np.zeros(max(n, 1) * max(n, 1), dtype=np.complex128)
    n_, ldz_ = C.c_int(n), C.c_int(n)
    vl_, vu_, il_, iu_, m_ = C.c_double(vl), C.c_double(vu), C.c_int(il), C.c_int(iu), C.c_int(0)
    info = L.zhpeig(jobz.encode(), rng.encode(), uplo.encode(), C.byref(n_), _cpd(AP),
                    C.byref(vl_), C.byref(vu_), C.byref(il_), C.byref(iu_), C.byref(m_),
                    W.ctypes.data_as(_pd), _cpd(Z), C.byref(ldz_))
    m = m_.value
    out = dict(info=info, m=m, W=W[:m].copy())
    if jobz[0] in "Vv":
        out["Z"] = Z[: n * m].reshape(m, n).T.copy() if m > 0 else np.zeros((n, 0), complex)
    return out


def ref_zhegeig(itype, jobz, rng, uplo, A, B, vl=0.0, vu=0.0, il=1, iu=1, threads: int = 2):
    """The reference's zhegeig() (SRC/dense.c:676-754): eigenvectors in A."""
    L = _ref(threads)
    A = np.asarray(A, dtype=np.complex128)
    n = A.shape[0]
    Af = np.array(A.T, dtype=np.complex128, copy=True).reshape(-1)
    Bf = np.array(np.asarray(B, dtype=np.complex128).T, copy=True).reshape(-1)
    W = np.zeros(max(n, 1))
    it_, n_, lda_, ldb_ = C.c_int(itype), C.c_int(n), C.c_int(n), C.c_int(n)
    vl_, vu_, il_, iu_, m_ = C.c_double(vl), C.c_double(vu), C.c_int(il), C.c_int(iu), C.c_int(0)
    info = L.zhegeig(C.byref(it_), jobz.encode(), rng.encode(), uplo.encode(), C.byref(n_),
                     _cpd(Af), C.byref(lda_), _cpd(Bf), C.byref(ldb_), C.byref(vl_),
                     C.byref(vu_), C.byref(il_), C.byref(iu_), C.byref(m_),
                     W.ctypes.data_as(_pd))
    m = m_.value
    out = dict(info=info, m=m, W=W[:m].copy())
    if jobz[0] in "Vv":
        out["Z"] = Af[: n * m].reshape(m, n).T.copy() if m > 0 else np.zeros((n, 0), complex)
    return out


def ref_zhpgeig(itype, jobz, rng, uplo, AP, BP, n, vl=0.0, vu=0.0, il=1, iu=1,
                threads: int = 2):
    """The reference's zhpgeig() (packed generalized Hermitian, SRC/dense.c:869-936)."""
    L = _ref(threads)
    AP = np.array(AP, dtype=np.complex128, copy=True)
    BP = np.array(BP, dtype=np.complex128, copy=True)
    W = np.zeros(max(n, 1))
    Z = np.zeros(max(n, 1) * max(n, 1), dtype=np.complex128)
    it_, n_, ldz_ = C.c_int(itype), C.c_int(n), C.c_int(n)
    vl_, vu_, il_, iu_, m_ = C.c_double(vl), C.c_double(vu), C.c_int(il), C.c_int(iu), C.c_int(0)
    info = L.zhpgeig(C.byref(it_), jobz.encode(), rng.encode(), uplo.encode(), C.byref(n_),
                     _cpd(AP), _cpd(BP), C.byref(vl_), C.byref(vu_), C.byref(il_),
                     C.byref(iu_), C.byref(m_), W.ctypes.data_as(_pd), _cpd(Z), C.byref(ldz_))
    m = m_.value
    out = dict(info=info, m=m, W=W[:m].copy())
    if jobz[0] in "Vv":
        out["Z"] = Z[: n * m].reshape(m, n).T.copy() if m > 0 else np.zeros((n, 0), complex)
    return out
