/*
 * dense.cu -- the dense drivers of SRC/dense.c: dsyeig (:151-232), dspeig
 * (packed storage, :319-398), dsygeig (generalized, :236-313) and dspgeig
 * (generalized, packed, :403-470).
 *
 * The reference scales A (dscale_matrix, SRC/dense.c:477-527), reduces it to
 * tridiagonal form with LAPACK's dsytrd, solves the tridiagonal problem with
 * mrrr(), back-transforms Z = Q Z with LAPACK's dormtr and unscales W.  Here
 * every step runs on the device that runs the tridiagonal solve, so A, the
 * Householder vectors, D, E and Z stay in HBM between the steps: the max-norm
 * and the scaling are two kernels of this file, the tridiagonal solve is the
 * batched solver (mr3_batched_device), and dsytrd/dormtr -- external LAPACK
 * calls in the reference as well -- are cuSOLVER's, loaded at first use so
 * that the rest of the library does not depend on it.  Packed matrices are
 * unpacked into a full device copy (HBM holds n^2 doubles easily), so the
 * packed drivers share the full drivers' path.  The generalized drivers add
 * the Cholesky factorisation of B (cuSOLVER's dpotrf), the reduction to a
 * standard problem (dsygst: two triangular solves or products with the
 * factor, cuBLAS's dtrsm/dtrmm on the full symmetric A) and the
 * back-transformation of Z with the factor (dtrsm/dtrmm).
 */
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>
#include <dlfcn.h>
#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#include "mr3_b200.h"

namespace {

// ---- cuSOLVER entry points (dlopen'ed once) ------------------------------
struct Cusolver {
  decltype(&cusolverDnCreate) create;
  decltype(&cusolverDnDestroy) destroy;
  decltype(&cusolverDnDsytrd_bufferSize) sytrd_ws;
  decltype(&cusolverDnDsytrd) sytrd;
  decltype(&cusolverDnDormtr_bufferSize) ormtr_ws;
  decltype(&cusolverDnDormtr) ormtr;
  decltype(&cusolverDnDpotrf_bufferSize) potrf_ws;
  decltype(&cusolverDnDpotrf) potrf;
  decltype(&cublasCreate_v2) bcreate;
  decltype(&cublasDestroy_v2) bdestroy;
  decltype(&cublasDtrsm_v2) trsm;
  decltype(&cublasDtrmm_v2) trmm;
  bool ok, blas_ok;
};
Cusolver g_cs;
pthread_once_t g_cs_once = PTHREAD_ONCE_INIT;

void load_cusolver() {
  const char *names[] = {"libcusolver.so.11", "libcusolver.so",
                         "/usr/local/cuda/lib64/libcusolver.so.11"};
  void *h = nullptr;
  for (const char *nm : names)
    if ((h = dlopen(nm, RTLD_NOW | RTLD_GLOBAL)) != nullptr) break;
  if (!h) return;
  g_cs.create = (decltype(g_cs.create))dlsym(h, "cusolverDnCreate");
  g_cs.destroy = (decltype(g_cs.destroy))dlsym(h, "cusolverDnDestroy");
  g_cs.sytrd_ws = (decltype(g_cs.sytrd_ws))dlsym(h, "cusolverDnDsytrd_bufferSize");
  g_cs.sytrd = (decltype(g_cs.sytrd))dlsym(h, "cusolverDnDsytrd");
  g_cs.ormtr_ws = (decltype(g_cs.ormtr_ws))dlsym(h, "cusolverDnDormtr_bufferSize");
  g_cs.ormtr = (decltype(g_cs.ormtr))dlsym(h, "cusolverDnDormtr");
  g_cs.potrf_ws = (decltype(g_cs.potrf_ws))dlsym(h, "cusolverDnDpotrf_bufferSize");
  g_cs.potrf = (decltype(g_cs.potrf))dlsym(h, "cusolverDnDpotrf");
  g_cs.ok = g_cs.create && g_cs.destroy && g_cs.sytrd_ws && g_cs.sytrd && g_cs.ormtr_ws &&
            g_cs.ormtr && g_cs.potrf_ws && g_cs.potrf;
  const char *bnames[] = {"libcublas.so.12", "libcublas.so", "/usr/local/cuda/lib64/libcublas.so.12"};
  void *hb = nullptr;
  for (const char *nm : bnames)
    if ((hb = dlopen(nm, RTLD_NOW | RTLD_GLOBAL)) != nullptr) break;
  if (!hb) return;
  g_cs.bcreate = (decltype(g_cs.bcreate))dlsym(hb, "cublasCreate_v2");
  g_cs.bdestroy = (decltype(g_cs.bdestroy))dlsym(hb, "cublasDestroy_v2");
  g_cs.trsm = (decltype(g_cs.trsm))dlsym(hb, "cublasDtrsm_v2");
  g_cs.trmm = (decltype(g_cs.trmm))dlsym(hb, "cublasDtrmm_v2");
  g_cs.blas_ok = g_cs.bcreate && g_cs.bdestroy && g_cs.trsm && g_cs.trmm;
}

// ---- max-norm and scaling of the stored triangle (dlansy 'M', dscal) -----
// Element (i, j) of the n x n device copy (leading dimension n) is in the
// stored triangle when i >= j (lower) or i <= j (upper).

// max |a_ij| over the triangle; NaN if any element is NaN (dlansy 'M' keeps
// a NaN once seen).  One block-wide reduction per CTA, combined with an
// atomic max on the bit pattern (non-negative doubles order like their bits;
// a NaN is flagged separately).
__global__ void k_tri_absmax(int n, const double *A, int lower, unsigned long long *maxbits,
                             int *nan) {
  __shared__ double red[32];
  __shared__ int rnan;
  if (threadIdx.x == 0) rnan = 0;
  __syncthreads();
  double v = 0.0;
  bool sawnan = false;
  const long long total = (long long)n * n;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
       k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % n), j = (int)(k / n);
    if (lower ? i < j : i > j) continue;
    const double a = fabs(A[k]);
    if (isnan(a)) sawnan = true;
    else v = fmax(v, a);
  }
  if (sawnan) rnan = 1;
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (threadIdx.x == 0) {
      atomicMax(maxbits, (unsigned long long)__double_as_longlong(v));
      if (rnan) atomicExch(nan, 1);
    }
  }
}

__global__ void k_tri_scale(int n, double *A, int lower, double sigma) {
  const long long total = (long long)n * n;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
       k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % n), j = (int)(k / n);
    if (lower ? i >= j : i <= j) A[k] = A[k] * sigma;
  }
}

// Packed triangle (LAPACK 'L'/'U' packed, column by column) to the same
// triangle of a full n x n matrix, or back (to_packed).
__global__ void k_packed(int n, double *ap, double *A, int lower, int to_packed) {
  const long long total = (long long)n * n;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
       k += (long long)gridDim.x * blockDim.x) {
    const long long i = k % n, j = k / n;
    if (lower ? i < j : i > j) continue;
    const long long p = lower ? i + j * (2LL * n - j - 1) / 2 : i + j * (j + 1) / 2;
    if (to_packed) ap[p] = A[k];
    else A[k] = ap[p];
  }
}

// The other triangle of a symmetric matrix from the stored one.
__global__ void k_symmetrize(int n, double *A, int lower) {
  const long long total = (long long)n * n;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
       k += (long long)gridDim.x * blockDim.x) {
    const long long i = k % n, j = k / n;
    if (lower ? i < j : i > j) A[k] = A[j + i * n];
  }
}

int device_id() {
  const char *s = getenv("MR3_DEVICE");
  return s ? atoi(s) : 0;
}

int job_code(char c) {
  if (c == 'N' || c == 'n') return MR3_JOB_N;
  if (c == 'V' || c == 'v') return MR3_JOB_V;
  if (c == 'C' || c == 'c') return MR3_JOB_C;
  return -1;
}

int range_code(char c) {
  if (c == 'A' || c == 'a') return MR3_RANGE_A;
  if (c == 'V' || c == 'v') return MR3_RANGE_V;
  if (c == 'I' || c == 'i') return MR3_RANGE_I;
  return -1;
}

// Device buffers of one call, released on every exit path.
struct DenseBufs {
  double *A = nullptr, *B = nullptr, *AP = nullptr, *D = nullptr, *E = nullptr, *tau = nullptr,
         *W = nullptr, *Z = nullptr, *work = nullptr;
  int *Zsupp = nullptr, *info = nullptr, *nan = nullptr;
  unsigned long long *maxbits = nullptr;
  cusolverDnHandle_t h = nullptr;
  cublasHandle_t hb = nullptr;
  ~DenseBufs() {
    void *p[] = {A, B, AP, D, E, tau, W, Z, work, Zsupp, info, nan, maxbits};
    for (void *q : p)
      if (q) cudaFree(q);
    if (h) g_cs.destroy(h);
    if (hb) g_cs.bdestroy(hb);
  }
};

#define DCK(x)                          \
  do {                                  \
    if ((x) != cudaSuccess) return 2;   \
  } while (0)
#define SCK(x)                                            \
  do {                                                    \
    if ((x) != CUSOLVER_STATUS_SUCCESS) return 2;         \
  } while (0)
#define BCK(x)                                            \
  do {                                                    \
    if ((x) != CUBLAS_STATUS_SUCCESS) return 2;           \
  } while (0)

const int kGrid = 148 * 8;

// Argument checks shared by the drivers (SRC/dense.c:177-186).
int check_common(int jz, int rg, int n, const double *vl, const double *vu, const int *il,
                 const int *iu) {
  if (jz < 0 || rg < 0 || n <= 0) return 1;
  if (rg == MR3_RANGE_V) {
    if (*vu <= *vl) return 1;
  } else if (rg == MR3_RANGE_I) {
    if (*il < 1 || *il > n || *iu < *il || *iu > n) return 1;
  }
  return 0;
}

int start(DenseBufs &b, int n, int jz, int ncols) {
  pthread_once(&g_cs_once, load_cusolver);
  if (!g_cs.ok) return 2;
  DCK(cudaSetDevice(device_id()));
  const size_t nn = (size_t)n * n;
  DCK(cudaMalloc((void **)&b.A, nn * sizeof(double)));
  DCK(cudaMalloc((void **)&b.D, n * sizeof(double)));
  DCK(cudaMalloc((void **)&b.E, n * sizeof(double)));
  DCK(cudaMalloc((void **)&b.tau, n * sizeof(double)));
  DCK(cudaMalloc((void **)&b.W, n * sizeof(double)));
  DCK(cudaMalloc((void **)&b.Zsupp, 2 * (size_t)n * sizeof(int)));
  DCK(cudaMalloc((void **)&b.info, sizeof(int)));
  DCK(cudaMalloc((void **)&b.nan, sizeof(int)));
  DCK(cudaMalloc((void **)&b.maxbits, sizeof(unsigned long long)));
  if (jz == MR3_JOB_V) DCK(cudaMalloc((void **)&b.Z, (size_t)n * ncols * sizeof(double)));
  DCK(cudaMemset(b.E, 0, n * sizeof(double)));
  DCK(cudaMemset(b.nan, 0, sizeof(int)));
  DCK(cudaMemset(b.maxbits, 0, sizeof(unsigned long long)));
  SCK(g_cs.create(&b.h));
  return 0;
}

// The symmetric eigenproblem of the device matrix b.A (n x n, leading
// dimension n, the `lower` triangle referenced): dsyeig's steps after the
// copy-in (SRC/dense.c:198-221).  W (host, m entries) is unscaled; Z stays
// on the device in b.Z (leading dimension n).
int dense_core(DenseBufs &b, int jz, int rg, bool lower, int n, int ncols, double *vlp,
               double *vup, int *ilp, int *iup, int *mp, double *W) {
  // scaling (dscale_matrix): into [rmin, rmax] when the max-norm is outside
  const double smlnum = DBL_MIN / DBL_EPSILON, bignum = 1.0 / smlnum;
  const double rmin = sqrt(smlnum), rmax = fmin(sqrt(bignum), 1.0 / sqrt(sqrt(DBL_MIN)));
  k_tri_absmax<<<kGrid, 256>>>(n, b.A, lower, b.maxbits, b.nan);
  DCK(cudaGetLastError());
  unsigned long long bits = 0;
  int sawnan = 0;
  DCK(cudaMemcpy(&bits, b.maxbits, sizeof(bits), cudaMemcpyDeviceToHost));
  DCK(cudaMemcpy(&sawnan, b.nan, sizeof(int), cudaMemcpyDeviceToHost));
  double norm;
  memcpy(&norm, &bits, sizeof(norm));
  if (sawnan) norm = NAN;
  double sigma = 1.0;
  bool scaled = false;
  if (norm > 0.0 && norm < rmin) {
    scaled = true;
    sigma = rmin / norm;
  } else if (norm > rmax) {
    scaled = true;
    sigma = rmax / norm;
  }
  if (scaled) {
    k_tri_scale<<<kGrid, 256>>>(n, b.A, lower, sigma);
    DCK(cudaGetLastError());
    if (rg == MR3_RANGE_V) {
      *vlp *= sigma;
      *vup *= sigma;
    }
  }

  // reduction to tridiagonal form (dsytrd): D, E, tau; Q in A
  const cublasFillMode_t fill = lower ? CUBLAS_FILL_MODE_LOWER : CUBLAS_FILL_MODE_UPPER;
  int lw1 = 0, lw2 = 0;
  if (n > 1) SCK(g_cs.sytrd_ws(b.h, fill, n, b.A, n, b.D, b.E, b.tau, &lw1));
  if (n > 1 && jz == MR3_JOB_V)
    SCK(g_cs.ormtr_ws(b.h, CUBLAS_SIDE_LEFT, fill, CUBLAS_OP_N, n, ncols, b.A, n, b.tau, b.Z, n,
                      &lw2));
  if (b.work) cudaFree(b.work);
  b.work = nullptr;
  DCK(cudaMalloc((void **)&b.work, (size_t)(lw1 > lw2 ? lw1 : lw2) * sizeof(double) + 8));
  int hinfo = 0;
  if (n > 1) {
    SCK(g_cs.sytrd(b.h, fill, n, b.A, n, b.D, b.E, b.tau, b.work, lw1, b.info));
    DCK(cudaMemcpy(&hinfo, b.info, sizeof(int), cudaMemcpyDeviceToHost));
    if (hinfo != 0) return 2;
  } else {
    DCK(cudaMemcpy(b.D, b.A, sizeof(double), cudaMemcpyDeviceToDevice));   // Q = 1
  }

  // the tridiagonal problem (mrrr with tryrac = 1, SRC/dense.c:205-207)
  mr3_cuda_prob q;
  memset(&q, 0, sizeof(q));
  q.n = n; q.jobz = jz; q.range = rg; q.il = *ilp; q.iu = *iup; q.tryrac = 1; q.ldz = n;
  q.vl = *vlp; q.vu = *vup;
  q.D = b.D; q.E = b.E; q.W = b.W; q.Z = b.Z; q.Zsupp = b.Zsupp;
  DCK(cudaDeviceSynchronize());
  const int rc = mr3_batched_device(1, &q, nullptr);
  if (rc != MR3_OK) return rc;
  const int m = q.m;

  // back-transformation Z = Q Z (dormtr)
  if (jz == MR3_JOB_V && m > 0 && n > 1) {
    DCK(cudaDeviceSynchronize());
    SCK(g_cs.ormtr(b.h, CUBLAS_SIDE_LEFT, fill, CUBLAS_OP_N, n, m, b.A, n, b.tau, b.Z, n, b.work,
                   lw2, b.info));
    DCK(cudaMemcpy(&hinfo, b.info, sizeof(int), cudaMemcpyDeviceToHost));
    if (hinfo != 0) return 2;
  }
  if (jz != MR3_JOB_C && m > 0) DCK(cudaMemcpy(W, b.W, m * sizeof(double), cudaMemcpyDeviceToHost));

  // outputs as mrrr() leaves them, then the unscaling of SRC/dense.c:215-221
  *mp = m;
  if (n > 1) {
    *vlp = q.vl_out; *vup = q.vu_out;
    *ilp = q.il_out; *iup = q.iu_out;
  }
  if (scaled) {
    const double invscale = 1.0 / sigma;
    *vlp *= invscale;
    *vup *= invscale;
    if (jz != MR3_JOB_C)
      for (int i = 0; i < m; i++) W[i] = W[i] * invscale;
  }
  return 0;
}

// Cholesky factor of b.B (dpotrf) and the reduction of b.A to the standard
// problem (dsygst, SRC/dense.c:268-274): with B = L L^T (uplo L) or U^T U
// (uplo U), A becomes inv(L) A inv(L)^T or inv(U)^T A inv(U) for itype 1 and
// L^T A L or U A U^T for itypes 2 and 3, each as two triangular solves or
// products on the full symmetric A.
int reduce_generalized(DenseBufs &b, int itype, bool lower, int n) {
  if (!g_cs.blas_ok) return 2;
  const cublasFillMode_t fill = lower ? CUBLAS_FILL_MODE_LOWER : CUBLAS_FILL_MODE_UPPER;
  int lw = 0, hinfo = 0;
  SCK(g_cs.potrf_ws(b.h, fill, n, b.B, n, &lw));
  DCK(cudaMalloc((void **)&b.work, (size_t)lw * sizeof(double) + 8));
  SCK(g_cs.potrf(b.h, fill, n, b.B, n, b.work, lw, b.info));
  DCK(cudaMemcpy(&hinfo, b.info, sizeof(int), cudaMemcpyDeviceToHost));
  if (hinfo != 0) return 2;   // B is not positive definite
  k_symmetrize<<<kGrid, 256>>>(n, b.A, lower);
  DCK(cudaGetLastError());
  BCK(g_cs.bcreate(&b.hb));
  const double one = 1.0;
  const cublasDiagType_t nu = CUBLAS_DIAG_NON_UNIT;
  if (itype == 1) {
    // lower: L^-1 A, then (.) L^-T;  upper: U^-T A, then (.) U^-1
    BCK(g_cs.trsm(b.hb, CUBLAS_SIDE_LEFT, fill, lower ? CUBLAS_OP_N : CUBLAS_OP_T, nu, n, n, &one,
                  b.B, n, b.A, n));
    BCK(g_cs.trsm(b.hb, CUBLAS_SIDE_RIGHT, fill, lower ? CUBLAS_OP_T : CUBLAS_OP_N, nu, n, n,
                  &one, b.B, n, b.A, n));
  } else {
    // lower: L^T A, then (.) L;  upper: U A, then (.) U^T
    BCK(g_cs.trmm(b.hb, CUBLAS_SIDE_LEFT, fill, lower ? CUBLAS_OP_T : CUBLAS_OP_N, nu, n, n, &one,
                  b.B, n, b.A, n, b.A, n));
    BCK(g_cs.trmm(b.hb, CUBLAS_SIDE_RIGHT, fill, lower ? CUBLAS_OP_N : CUBLAS_OP_T, nu, n, n,
                  &one, b.B, n, b.A, n, b.A, n));
  }
  DCK(cudaDeviceSynchronize());
  return 0;
}

// Eigenvectors of the standard problem back to the generalized one
// (SRC/dense.c:280-300): x = inv(L)^T y or inv(U) y (itypes 1, 2),
// x = L y or U^T y (itype 3).
int backtransform_generalized(DenseBufs &b, int itype, bool lower, int n, int m) {
  const cublasFillMode_t fill = lower ? CUBLAS_FILL_MODE_LOWER : CUBLAS_FILL_MODE_UPPER;
  const double one = 1.0;
  const cublasDiagType_t nu = CUBLAS_DIAG_NON_UNIT;
  if (m <= 0) return 0;
  if (itype == 1 || itype == 2)
    BCK(g_cs.trsm(b.hb, CUBLAS_SIDE_LEFT, fill, lower ? CUBLAS_OP_T : CUBLAS_OP_N, nu, n, m, &one,
                  b.B, n, b.Z, n));
  else
    BCK(g_cs.trmm(b.hb, CUBLAS_SIDE_LEFT, fill, lower ? CUBLAS_OP_N : CUBLAS_OP_T, nu, n, m, &one,
                  b.B, n, b.Z, n, b.Z, n));
  DCK(cudaDeviceSynchronize());
  return 0;
}

}  // namespace

extern "C" int dsyeig(char *jobz, char *range, char *uplo, int *np, double *A, int *ldap,
                      double *vlp, double *vup, int *ilp, int *iup, int *mp, double *W,
                      double *Z, int *ldzp) {
  const int n = *np, jz = job_code(jobz[0]), rg = range_code(range[0]);
  const bool lower = uplo[0] == 'L' || uplo[0] == 'l';
  // argument checks of SRC/dense.c:177-186, plus the array extents that the
  // reference leaves to LAPACK (lda, ldz) and the triangle selector
  if (check_common(jz, rg, n, vlp, vup, ilp, iup)) return 1;
  if (!(lower || uplo[0] == 'U' || uplo[0] == 'u') || *ldap < n) return 1;
  if (jz == MR3_JOB_V && *ldzp < n) return 1;
  // counting with range A or I needs no work (mrrr(), SRC/mrrr.c:130-138)
  if (jz == MR3_JOB_C && rg != MR3_RANGE_V) {
    *mp = rg == MR3_RANGE_A ? n : *iup - *ilp + 1;
    return 0;
  }
  DenseBufs b;
  const int ncols = rg == MR3_RANGE_I ? *iup - *ilp + 1 : n;
  int rc = start(b, n, jz, ncols);
  if (rc) return rc;
  DCK(cudaMemcpy2D(b.A, n * sizeof(double), A, (size_t)*ldap * sizeof(double), n * sizeof(double),
                   n, cudaMemcpyHostToDevice));
  if ((rc = dense_core(b, jz, rg, lower, n, ncols, vlp, vup, ilp, iup, mp, W))) return rc;
  if (jz == MR3_JOB_V && *mp > 0)
    DCK(cudaMemcpy2D(Z, (size_t)*ldzp * sizeof(double), b.Z, n * sizeof(double),
                     n * sizeof(double), *mp, cudaMemcpyDeviceToHost));
  return 0;
}

extern "C" int dspeig(char *jobz, char *range, char *uplo, int *np, double *AP, double *vlp,
                      double *vup, int *ilp, int *iup, int *mp, double *W, double *Z, int *ldzp) {
  const int n = *np, jz = job_code(jobz[0]), rg = range_code(range[0]);
  const bool lower = uplo[0] == 'L' || uplo[0] == 'l';
  // SRC/dense.c:340-347, plus ldz and uplo
  if (check_common(jz, rg, n, vlp, vup, ilp, iup)) return 1;
  if (!(lower || uplo[0] == 'U' || uplo[0] == 'u')) return 1;
  if (jz == MR3_JOB_V && *ldzp < n) return 1;
  if (jz == MR3_JOB_C && rg != MR3_RANGE_V) {
    *mp = rg == MR3_RANGE_A ? n : *iup - *ilp + 1;
    return 0;
  }
  DenseBufs b;
  const int ncols = rg == MR3_RANGE_I ? *iup - *ilp + 1 : n;
  int rc = start(b, n, jz, ncols);
  if (rc) return rc;
  const size_t np_ = (size_t)n * (n + 1) / 2;
  DCK(cudaMalloc((void **)&b.AP, np_ * sizeof(double)));
  DCK(cudaMemcpy(b.AP, AP, np_ * sizeof(double), cudaMemcpyHostToDevice));
  k_packed<<<kGrid, 256>>>(n, b.AP, b.A, lower, 0);
  DCK(cudaGetLastError());
  if ((rc = dense_core(b, jz, rg, lower, n, ncols, vlp, vup, ilp, iup, mp, W))) return rc;
  if (jz == MR3_JOB_V && *mp > 0)
    DCK(cudaMemcpy2D(Z, (size_t)*ldzp * sizeof(double), b.Z, n * sizeof(double),
                     n * sizeof(double), *mp, cudaMemcpyDeviceToHost));
  return 0;
}

extern "C" int dsygeig(int *itype, char *jobz, char *range, char *uplo, int *np, double *A,
                       int *ldap, double *B, int *ldbp, double *vlp, double *vup, int *ilp,
                       int *iup, int *mp, double *W) {
  const int n = *np, jz = job_code(jobz[0]), rg = range_code(range[0]);
  const bool lower = uplo[0] == 'L' || uplo[0] == 'l';
  // SRC/dense.c:257-262 (n <= 1 is refused there), plus lda, ldb and the
  // range bounds that its dsyeig call checks
  if (n <= 1 || *itype < 1 || *itype > 3) return 1;
  if (!(lower || uplo[0] == 'U' || uplo[0] == 'u')) return 1;
  if (check_common(jz, rg, n, vlp, vup, ilp, iup)) return 1;
  if (*ldap < n || *ldbp < n) return 1;
  DenseBufs b;
  const int ncols = rg == MR3_RANGE_I ? *iup - *ilp + 1 : n;
  int rc = start(b, n, jz, ncols);
  if (rc) return rc;
  DCK(cudaMalloc((void **)&b.B, (size_t)n * n * sizeof(double)));
  DCK(cudaMemcpy2D(b.A, n * sizeof(double), A, (size_t)*ldap * sizeof(double), n * sizeof(double),
                   n, cudaMemcpyHostToDevice));
  DCK(cudaMemcpy2D(b.B, n * sizeof(double), B, (size_t)*ldbp * sizeof(double), n * sizeof(double),
                   n, cudaMemcpyHostToDevice));
  if ((rc = reduce_generalized(b, *itype, lower, n))) return rc;
  if (jz == MR3_JOB_C && rg != MR3_RANGE_V) {
    *mp = rg == MR3_RANGE_A ? n : *iup - *ilp + 1;
  } else {
    if ((rc = dense_core(b, jz, rg, lower, n, ncols, vlp, vup, ilp, iup, mp, W))) return rc;
    if (jz == MR3_JOB_V && (rc = backtransform_generalized(b, *itype, lower, n, *mp))) return rc;
  }
  // B holds its Cholesky factor, A the eigenvectors (SRC/dense.c:302-305)
  DCK(cudaMemcpy2D(B, (size_t)*ldbp * sizeof(double), b.B, n * sizeof(double), n * sizeof(double),
                   n, cudaMemcpyDeviceToHost));
  if (jz == MR3_JOB_V && *mp > 0)
    DCK(cudaMemcpy2D(A, (size_t)*ldap * sizeof(double), b.Z, n * sizeof(double),
                     n * sizeof(double), *mp, cudaMemcpyDeviceToHost));
  return 0;
}

extern "C" int dspgeig(int *itype, char *jobz, char *range, char *uplo, int *np, double *AP,
                       double *BP, double *vlp, double *vup, int *ilp, int *iup, int *mp,
                       double *W, double *Z, int *ldzp) {
  const int n = *np, jz = job_code(jobz[0]), rg = range_code(range[0]);
  const bool lower = uplo[0] == 'L' || uplo[0] == 'l';
  // SRC/dense.c:420-425, plus ldz and the range bounds of its dspeig call
  if (n < 1 || *itype < 1 || *itype > 3) return 1;
  if (!(lower || uplo[0] == 'U' || uplo[0] == 'u')) return 1;
  if (check_common(jz, rg, n, vlp, vup, ilp, iup)) return 1;
  if (jz == MR3_JOB_V && *ldzp < n) return 1;
  DenseBufs b;
  const int ncols = rg == MR3_RANGE_I ? *iup - *ilp + 1 : n;
  int rc = start(b, n, jz, ncols);
  if (rc) return rc;
  const size_t np_ = (size_t)n * (n + 1) / 2;
  DCK(cudaMalloc((void **)&b.B, (size_t)n * n * sizeof(double)));
  DCK(cudaMalloc((void **)&b.AP, np_ * sizeof(double)));
  DCK(cudaMemset(b.B, 0, (size_t)n * n * sizeof(double)));
  DCK(cudaMemcpy(b.AP, AP, np_ * sizeof(double), cudaMemcpyHostToDevice));
  k_packed<<<kGrid, 256>>>(n, b.AP, b.A, lower, 0);
  DCK(cudaGetLastError());
  DCK(cudaMemcpy(b.AP, BP, np_ * sizeof(double), cudaMemcpyHostToDevice));
  k_packed<<<kGrid, 256>>>(n, b.AP, b.B, lower, 0);
  DCK(cudaGetLastError());
  if ((rc = reduce_generalized(b, *itype, lower, n))) return rc;
  if (jz == MR3_JOB_C && rg != MR3_RANGE_V) {
    *mp = rg == MR3_RANGE_A ? n : *iup - *ilp + 1;
  } else {
    if ((rc = dense_core(b, jz, rg, lower, n, ncols, vlp, vup, ilp, iup, mp, W))) return rc;
    if (jz == MR3_JOB_V && (rc = backtransform_generalized(b, *itype, lower, n, *mp))) return rc;
  }
  // BP holds the packed Cholesky factor (dpptrf's output)
  k_packed<<<kGrid, 256>>>(n, b.AP, b.B, lower, 1);
  DCK(cudaGetLastError());
  DCK(cudaMemcpy(BP, b.AP, np_ * sizeof(double), cudaMemcpyDeviceToHost));
  if (jz == MR3_JOB_V && *mp > 0)
    DCK(cudaMemcpy2D(Z, (size_t)*ldzp * sizeof(double), b.Z, n * sizeof(double),
                     n * sizeof(double), *mp, cudaMemcpyDeviceToHost));
  return 0;
}

extern "C" void dsyeig_(char *jobz, char *range, char *uplo, int *n, double *A, int *lda,
                        double *vl, double *vu, int *il, int *iu, int *m, double *W, double *Z,
                        int *ldz, int *info) {
  *info = dsyeig(jobz, range, uplo, n, A, lda, vl, vu, il, iu, m, W, Z, ldz);
}

extern "C" void dspeig_(char *jobz, char *range, char *uplo, int *n, double *AP, double *vl,
                        double *vu, int *il, int *iu, int *m, double *W, double *Z, int *ldz,
                        int *info) {
  *info = dspeig(jobz, range, uplo, n, AP, vl, vu, il, iu, m, W, Z, ldz);
}

extern "C" void dsygeig_(int *itype, char *jobz, char *range, char *uplo, int *n, double *A,
                         int *lda, double *B, int *ldb, double *vl, double *vu, int *il, int *iu,
                         int *m, double *W, int *info) {
  *info = dsygeig(itype, jobz, range, uplo, n, A, lda, B, ldb, vl, vu, il, iu, m, W);
}

extern "C" void dspgeig_(int *itype, char *jobz, char *range, char *uplo, int *n, double *AP,
                         double *BP, double *vl, double *vu, int *il, int *iu, int *m, double *W,
                         double *Z, int *ldz, int *info) {
  *info = dspgeig(itype, jobz, range, uplo, n, AP, BP, vl, vu, il, iu, m, W, Z, ldz);
}
