/*
 * zdense.cu -- the complex Hermitian dense drivers of SRC/dense.c, which the
 * reference compiles only with its COMPLEX_SUPPORTED switch: zheeig
 * (:568-671), zhegeig (:676-754), zhpeig (:760-862) and zhpgeig (:869-936).
 *
 * zhetrd reduces a Hermitian A to a real symmetric tridiagonal T = Q^H A Q,
 * so the tridiagonal problem is the real solver's (mr3_batched_device); its
 * real eigenvectors are widened to complex columns on the device and
 * back-transformed with Q (zunmtr).  The packed and generalized variants
 * follow the real drivers (dense.cu) with conjugate transposes: packed
 * storage is unpacked into a full device copy, B = L L^H (or U^H U) comes
 * from zpotrf, the reduction to a standard problem and the back-
 * transformation are cuBLAS triangular solves or products.  cuSOLVER
 * (zhetrd, zunmtr, zpotrf) and cuBLAS (ztrsm, ztrmm) are loaded at the first
 * call.  Complex arrays are column-major with interleaved (re, im) doubles,
 * the layout of C99 double complex.
 */
#include <cublas_v2.h>
#include <cuComplex.h>
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

struct ZLib {
  decltype(&cusolverDnCreate) create;
  decltype(&cusolverDnDestroy) destroy;
  decltype(&cusolverDnZhetrd_bufferSize) hetrd_ws;
  decltype(&cusolverDnZhetrd) hetrd;
  decltype(&cusolverDnZunmtr_bufferSize) unmtr_ws;
  decltype(&cusolverDnZunmtr) unmtr;
  decltype(&cusolverDnZpotrf_bufferSize) potrf_ws;
  decltype(&cusolverDnZpotrf) potrf;
  decltype(&cublasCreate_v2) bcreate;
  decltype(&cublasDestroy_v2) bdestroy;
  decltype(&cublasZtrsm_v2) trsm;
  decltype(&cublasZtrmm_v2) trmm;
  bool ok, blas_ok;
};
ZLib g_z;
pthread_once_t g_z_once = PTHREAD_ONCE_INIT;

void *open_first(const char *const *names, int count) {
  for (int i = 0; i < count; i++)
    if (void *h = dlopen(names[i], RTLD_NOW | RTLD_GLOBAL)) return h;
  return nullptr;
}

void load_libs() {
  const char *sn[] = {"libcusolver.so.11", "libcusolver.so", "/usr/local/cuda/lib64/libcusolver.so.11"};
  void *h = open_first(sn, 3);
  if (!h) return;
  g_z.create = (decltype(g_z.create))dlsym(h, "cusolverDnCreate");
  g_z.destroy = (decltype(g_z.destroy))dlsym(h, "cusolverDnDestroy");
  g_z.hetrd_ws = (decltype(g_z.hetrd_ws))dlsym(h, "cusolverDnZhetrd_bufferSize");
  g_z.hetrd = (decltype(g_z.hetrd))dlsym(h, "cusolverDnZhetrd");
  g_z.unmtr_ws = (decltype(g_z.unmtr_ws))dlsym(h, "cusolverDnZunmtr_bufferSize");
  g_z.unmtr = (decltype(g_z.unmtr))dlsym(h, "cusolverDnZunmtr");
  g_z.potrf_ws = (decltype(g_z.potrf_ws))dlsym(h, "cusolverDnZpotrf_bufferSize");
  g_z.potrf = (decltype(g_z.potrf))dlsym(h, "cusolverDnZpotrf");
  g_z.ok = g_z.create && g_z.destroy && g_z.hetrd_ws && g_z.hetrd && g_z.unmtr_ws && g_z.unmtr &&
           g_z.potrf_ws && g_z.potrf;
  const char *bn[] = {"libcublas.so.12", "libcublas.so", "/usr/local/cuda/lib64/libcublas.so.12"};
  void *hb = open_first(bn, 3);
  if (!hb) return;
  g_z.bcreate = (decltype(g_z.bcreate))dlsym(hb, "cublasCreate_v2");
  g_z.bdestroy = (decltype(g_z.bdestroy))dlsym(hb, "cublasDestroy_v2");
  g_z.trsm = (decltype(g_z.trsm))dlsym(hb, "cublasZtrsm_v2");
  g_z.trmm = (decltype(g_z.trmm))dlsym(hb, "cublasZtrmm_v2");
  g_z.blas_ok = g_z.bcreate && g_z.bdestroy && g_z.trsm && g_z.trmm;
}

// ---- element-wise kernels on the n x n device copy (leading dimension n) --
// Element (i, j) is in the stored triangle when i >= j (lower) or i <= j.

// zlanhe 'M': max over the triangle of |a_ij| off the diagonal and |Re a_jj|
// on it (the imaginary part of a Hermitian diagonal is not referenced); a
// NaN is flagged.  Non-negative doubles order like their bit patterns.
__global__ void k_herm_absmax(int n, const cuDoubleComplex *A, int lower,
                              unsigned long long *maxbits, int *nan) {
  __shared__ double red[32];
  __shared__ int rnan;
  if (threadIdx.x == 0) rnan = 0;
  __syncthreads();
  double v = 0.0;
  bool sawnan = false;
  const long long total = (long long)n * n;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
       k += (long long)gridDim.x * blockDim.x) {
    const long long i = k % n, j = k / n;
    if (lower ? i < j : i > j) continue;
    const cuDoubleComplex a = A[k];
    const double x = (i == j) ? fabs(cuCreal(a)) : hypot(cuCreal(a), cuCimag(a));
    if (isnan(x)) sawnan = true;
    else v = fmax(v, x);
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

// zdscal of the stored triangle by the real sigma.
__global__ void k_herm_scale(int n, cuDoubleComplex *A, int lower, double sigma) {
  const long long total = (long long)n * n;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
       k += (long long)gridDim.x * blockDim.x) {
    const long long i = k % n, j = k / n;
    if (lower ? i >= j : i <= j) A[k] = make_cuDoubleComplex(cuCreal(A[k]) * sigma,
                                                             cuCimag(A[k]) * sigma);
  }
}

// Packed triangle (column by column) to the full matrix's triangle, or back.
__global__ void k_herm_packed(int n, cuDoubleComplex *ap, cuDoubleComplex *A, int lower,
                              int to_packed) {
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

// The full Hermitian matrix from its stored triangle: the other triangle
// conjugated, the diagonal real.
__global__ void k_herm_fill(int n, cuDoubleComplex *A, int lower) {
  const long long total = (long long)n * n;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
       k += (long long)gridDim.x * blockDim.x) {
    const long long i = k % n, j = k / n;
    if (i == j) A[k] = make_cuDoubleComplex(cuCreal(A[k]), 0.0);
    else if (lower ? i < j : i > j) A[k] = cuConj(A[j + i * n]);
  }
}

// The diagonal made real (zhetrd's assumption for a Hermitian matrix).
__global__ void k_herm_realdiag(int n, cuDoubleComplex *A) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    A[(long long)j * n + j] = make_cuDoubleComplex(cuCreal(A[(long long)j * n + j]), 0.0);
}

// Real n x m eigenvectors (leading dimension n) as complex columns.
__global__ void k_widen(long long count, const double *Zr, cuDoubleComplex *Z) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < count;
       k += (long long)gridDim.x * blockDim.x)
    Z[k] = make_cuDoubleComplex(Zr[k], 0.0);
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

bool is_uplo(char c) { return c == 'L' || c == 'l' || c == 'U' || c == 'u'; }

struct ZBufs {
  cuDoubleComplex *A = nullptr, *B = nullptr, *AP = nullptr, *tau = nullptr, *Z = nullptr,
                  *work = nullptr;
  double *D = nullptr, *E = nullptr, *W = nullptr, *Zr = nullptr;
  int *Zsupp = nullptr, *info = nullptr, *nan = nullptr;
  unsigned long long *maxbits = nullptr;
  cusolverDnHandle_t h = nullptr;
  cublasHandle_t hb = nullptr;
  ~ZBufs() {
    void *p[] = {A, B, AP, tau, Z, work, D, E, W, Zr, Zsupp, info, nan, maxbits};
    for (void *q : p)
      if (q) cudaFree(q);
    if (h) g_z.destroy(h);
    if (hb) g_z.bdestroy(hb);
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
const size_t kC = sizeof(cuDoubleComplex);

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

int zstart(ZBufs &b, int n, int jz, int ncols) {
  pthread_once(&g_z_once, load_libs);
  if (!g_z.ok) return 2;
  DCK(cudaSetDevice(device_id()));
  DCK(cudaMalloc((void **)&b.A, (size_t)n * n * kC));
  DCK(cudaMalloc((void **)&b.tau, (size_t)n * kC));
  DCK(cudaMalloc((void **)&b.D, n * sizeof(double)));
  DCK(cudaMalloc((void **)&b.E, n * sizeof(double)));
  DCK(cudaMalloc((void **)&b.W, n * sizeof(double)));
  DCK(cudaMalloc((void **)&b.Zsupp, 2 * (size_t)n * sizeof(int)));
  DCK(cudaMalloc((void **)&b.info, sizeof(int)));
  DCK(cudaMalloc((void **)&b.nan, sizeof(int)));
  DCK(cudaMalloc((void **)&b.maxbits, sizeof(unsigned long long)));
  if (jz == MR3_JOB_V) {
    DCK(cudaMalloc((void **)&b.Zr, (size_t)n * ncols * sizeof(double)));
    DCK(cudaMalloc((void **)&b.Z, (size_t)n * ncols * kC));
  }
  DCK(cudaMemset(b.E, 0, n * sizeof(double)));
  DCK(cudaMemset(b.nan, 0, sizeof(int)));
  DCK(cudaMemset(b.maxbits, 0, sizeof(unsigned long long)));
  SCK(g_z.create(&b.h));
  return 0;
}

// zheeig's steps after the copy-in (SRC/dense.c:620-662) on the device
// matrix b.A: scaling (zscale_matrix), zhetrd, the real tridiagonal solve,
// widening and zunmtr.  W (host) is unscaled; Z stays in b.Z.
int zcore(ZBufs &b, int jz, int rg, bool lower, int n, int ncols, double *vlp, double *vup,
          int *ilp, int *iup, int *mp, double *W) {
  const double smlnum = DBL_MIN / DBL_EPSILON, bignum = 1.0 / smlnum;
  const double rmin = sqrt(smlnum), rmax = fmin(sqrt(bignum), 1.0 / sqrt(sqrt(DBL_MIN)));
  k_herm_absmax<<<kGrid, 256>>>(n, b.A, lower, b.maxbits, b.nan);
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
    k_herm_scale<<<kGrid, 256>>>(n, b.A, lower, sigma);
    DCK(cudaGetLastError());
    if (rg == MR3_RANGE_V) {
      *vlp *= sigma;
      *vup *= sigma;
    }
  }

  // zhetrd: real D, E; complex tau; Q in A
  k_herm_realdiag<<<(n + 255) / 256, 256>>>(n, b.A);
  DCK(cudaGetLastError());
  const cublasFillMode_t fill = lower ? CUBLAS_FILL_MODE_LOWER : CUBLAS_FILL_MODE_UPPER;
  int lw1 = 0, lw2 = 0, hinfo = 0;
  if (n > 1) SCK(g_z.hetrd_ws(b.h, fill, n, b.A, n, b.D, b.E, b.tau, &lw1));
  if (n > 1 && jz == MR3_JOB_V)
    SCK(g_z.unmtr_ws(b.h, CUBLAS_SIDE_LEFT, fill, CUBLAS_OP_N, n, ncols, b.A, n, b.tau, b.Z, n,
                     &lw2));
  if (b.work) cudaFree(b.work);
  b.work = nullptr;
  DCK(cudaMalloc((void **)&b.work, (size_t)(lw1 > lw2 ? lw1 : lw2) * kC + 16));
  if (n > 1) {
    SCK(g_z.hetrd(b.h, fill, n, b.A, n, b.D, b.E, b.tau, b.work, lw1, b.info));
    DCK(cudaMemcpy(&hinfo, b.info, sizeof(int), cudaMemcpyDeviceToHost));
    if (hinfo != 0) return 2;
  } else {
    // a 1 x 1 Hermitian matrix is its real diagonal entry; Q = 1
    DCK(cudaMemcpy(b.D, b.A, sizeof(double), cudaMemcpyDeviceToDevice));
  }

  mr3_cuda_prob q;
  memset(&q, 0, sizeof(q));
  q.n = n; q.jobz = jz; q.range = rg; q.il = *ilp; q.iu = *iup; q.tryrac = 1; q.ldz = n;
  q.vl = *vlp; q.vu = *vup;
  q.D = b.D; q.E = b.E; q.W = b.W; q.Z = b.Zr; q.Zsupp = b.Zsupp;
  DCK(cudaDeviceSynchronize());
  const int rc = mr3_batched_device(1, &q, nullptr);
  if (rc != MR3_OK) return rc;
  const int m = q.m;

  if (jz == MR3_JOB_V && m > 0) {
    DCK(cudaDeviceSynchronize());
    k_widen<<<kGrid, 256>>>((long long)n * m, b.Zr, b.Z);
    DCK(cudaGetLastError());
    if (n > 1) {
      SCK(g_z.unmtr(b.h, CUBLAS_SIDE_LEFT, fill, CUBLAS_OP_N, n, m, b.A, n, b.tau, b.Z, n, b.work,
                    lw2, b.info));
      DCK(cudaMemcpy(&hinfo, b.info, sizeof(int), cudaMemcpyDeviceToHost));
      if (hinfo != 0) return 2;
    }
  }
  if (jz != MR3_JOB_C && m > 0) DCK(cudaMemcpy(W, b.W, m * sizeof(double), cudaMemcpyDeviceToHost));

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

// zpotrf of b.B and the reduction of b.A (zhegst): inv(L) A inv(L)^H or
// inv(U)^H A inv(U) for itype 1, L^H A L or U A U^H for itypes 2 and 3.
int zreduce(ZBufs &b, int itype, bool lower, int n) {
  if (!g_z.blas_ok) return 2;
  const cublasFillMode_t fill = lower ? CUBLAS_FILL_MODE_LOWER : CUBLAS_FILL_MODE_UPPER;
  int lw = 0, hinfo = 0;
  SCK(g_z.potrf_ws(b.h, fill, n, b.B, n, &lw));
  DCK(cudaMalloc((void **)&b.work, (size_t)lw * kC + 16));
  SCK(g_z.potrf(b.h, fill, n, b.B, n, b.work, lw, b.info));
  DCK(cudaMemcpy(&hinfo, b.info, sizeof(int), cudaMemcpyDeviceToHost));
  if (hinfo != 0) return 2;   // B is not positive definite
  k_herm_fill<<<kGrid, 256>>>(n, b.A, lower);
  DCK(cudaGetLastError());
  BCK(g_z.bcreate(&b.hb));
  const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0);
  const cublasDiagType_t nu = CUBLAS_DIAG_NON_UNIT;
  if (itype == 1) {
    BCK(g_z.trsm(b.hb, CUBLAS_SIDE_LEFT, fill, lower ? CUBLAS_OP_N : CUBLAS_OP_C, nu, n, n, &one,
                 b.B, n, b.A, n));
    BCK(g_z.trsm(b.hb, CUBLAS_SIDE_RIGHT, fill, lower ? CUBLAS_OP_C : CUBLAS_OP_N, nu, n, n, &one,
                 b.B, n, b.A, n));
  } else {
    BCK(g_z.trmm(b.hb, CUBLAS_SIDE_LEFT, fill, lower ? CUBLAS_OP_C : CUBLAS_OP_N, nu, n, n, &one,
                 b.B, n, b.A, n, b.A, n));
    BCK(g_z.trmm(b.hb, CUBLAS_SIDE_RIGHT, fill, lower ? CUBLAS_OP_N : CUBLAS_OP_C, nu, n, n, &one,
                 b.B, n, b.A, n, b.A, n));
  }
  DCK(cudaDeviceSynchronize());
  return 0;
}

// x = inv(L)^H y or inv(U) y (itypes 1, 2), x = L y or U^H y (itype 3)
// (SRC/dense.c:721-745).
int zbacktransform(ZBufs &b, int itype, bool lower, int n, int m) {
  const cublasFillMode_t fill = lower ? CUBLAS_FILL_MODE_LOWER : CUBLAS_FILL_MODE_UPPER;
  const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0);
  const cublasDiagType_t nu = CUBLAS_DIAG_NON_UNIT;
  if (m <= 0) return 0;
  if (itype == 1 || itype == 2)
    BCK(g_z.trsm(b.hb, CUBLAS_SIDE_LEFT, fill, lower ? CUBLAS_OP_C : CUBLAS_OP_N, nu, n, m, &one,
                 b.B, n, b.Z, n));
  else
    BCK(g_z.trmm(b.hb, CUBLAS_SIDE_LEFT, fill, lower ? CUBLAS_OP_N : CUBLAS_OP_C, nu, n, m, &one,
                 b.B, n, b.Z, n, b.Z, n));
  DCK(cudaDeviceSynchronize());
  return 0;
}

int copy_z_out(const ZBufs &b, int n, int m, void *Z, int ldz) {
  if (m > 0)
    DCK(cudaMemcpy2D(Z, (size_t)ldz * kC, b.Z, n * kC, n * kC, m, cudaMemcpyDeviceToHost));
  return 0;
}

}  // namespace

extern "C" int zheeig(char *jobz, char *range, char *uplo, int *np, void *A, int *ldap,
                      double *vlp, double *vup, int *ilp, int *iup, int *mp, double *W, void *Z,
                      int *ldzp) {
  const int n = *np, jz = job_code(jobz[0]), rg = range_code(range[0]);
  const bool lower = uplo[0] == 'L' || uplo[0] == 'l';
  // SRC/dense.c:596-602, plus lda, ldz and uplo
  if (check_common(jz, rg, n, vlp, vup, ilp, iup)) return 1;
  if (!is_uplo(uplo[0]) || *ldap < n) return 1;
  if (jz == MR3_JOB_V && *ldzp < n) return 1;
  if (jz == MR3_JOB_C && rg != MR3_RANGE_V) {
    *mp = rg == MR3_RANGE_A ? n : *iup - *ilp + 1;
    return 0;
  }
  ZBufs b;
  const int ncols = rg == MR3_RANGE_I ? *iup - *ilp + 1 : n;
  int rc = zstart(b, n, jz, ncols);
  if (rc) return rc;
  DCK(cudaMemcpy2D(b.A, n * kC, A, (size_t)*ldap * kC, n * kC, n, cudaMemcpyHostToDevice));
  if ((rc = zcore(b, jz, rg, lower, n, ncols, vlp, vup, ilp, iup, mp, W))) return rc;
  return jz == MR3_JOB_V ? copy_z_out(b, n, *mp, Z, *ldzp) : 0;
}

extern "C" int zhpeig(char *jobz, char *range, char *uplo, int *np, void *AP, double *vlp,
                      double *vup, int *ilp, int *iup, int *mp, double *W, void *Z, int *ldzp) {
  const int n = *np, jz = job_code(jobz[0]), rg = range_code(range[0]);
  const bool lower = uplo[0] == 'L' || uplo[0] == 'l';
  // SRC/dense.c:788-796, plus ldz and uplo
  if (check_common(jz, rg, n, vlp, vup, ilp, iup)) return 1;
  if (!is_uplo(uplo[0])) return 1;
  if (jz == MR3_JOB_V && *ldzp < n) return 1;
  if (jz == MR3_JOB_C && rg != MR3_RANGE_V) {
    *mp = rg == MR3_RANGE_A ? n : *iup - *ilp + 1;
    return 0;
  }
  ZBufs b;
  const int ncols = rg == MR3_RANGE_I ? *iup - *ilp + 1 : n;
  int rc = zstart(b, n, jz, ncols);
  if (rc) return rc;
  const size_t np_ = (size_t)n * (n + 1) / 2;
  DCK(cudaMalloc((void **)&b.AP, np_ * kC));
  DCK(cudaMemcpy(b.AP, AP, np_ * kC, cudaMemcpyHostToDevice));
  k_herm_packed<<<kGrid, 256>>>(n, b.AP, b.A, lower, 0);
  DCK(cudaGetLastError());
  if ((rc = zcore(b, jz, rg, lower, n, ncols, vlp, vup, ilp, iup, mp, W))) return rc;
  return jz == MR3_JOB_V ? copy_z_out(b, n, *mp, Z, *ldzp) : 0;
}

extern "C" int zhegeig(int *itype, char *jobz, char *range, char *uplo, int *np, void *A,
                       int *ldap, void *B, int *ldbp, double *vlp, double *vup, int *ilp,
                       int *iup, int *mp, double *W) {
  const int n = *np, jz = job_code(jobz[0]), rg = range_code(range[0]);
  const bool lower = uplo[0] == 'L' || uplo[0] == 'l';
  // SRC/dense.c:697-701 (n <= 1 refused), plus lda, ldb and the range bounds
  if (n <= 1 || *itype < 1 || *itype > 3 || !is_uplo(uplo[0])) return 1;
  if (check_common(jz, rg, n, vlp, vup, ilp, iup)) return 1;
  if (*ldap < n || *ldbp < n) return 1;
  ZBufs b;
  const int ncols = rg == MR3_RANGE_I ? *iup - *ilp + 1 : n;
  int rc = zstart(b, n, jz, ncols);
  if (rc) return rc;
  DCK(cudaMalloc((void **)&b.B, (size_t)n * n * kC));
  DCK(cudaMemcpy2D(b.A, n * kC, A, (size_t)*ldap * kC, n * kC, n, cudaMemcpyHostToDevice));
  DCK(cudaMemcpy2D(b.B, n * kC, B, (size_t)*ldbp * kC, n * kC, n, cudaMemcpyHostToDevice));
  if ((rc = zreduce(b, *itype, lower, n))) return rc;
  if (jz == MR3_JOB_C && rg != MR3_RANGE_V) {
    *mp = rg == MR3_RANGE_A ? n : *iup - *ilp + 1;
  } else {
    if ((rc = zcore(b, jz, rg, lower, n, ncols, vlp, vup, ilp, iup, mp, W))) return rc;
    if (jz == MR3_JOB_V && (rc = zbacktransform(b, *itype, lower, n, *mp))) return rc;
  }
  // B holds its Cholesky factor, A the eigenvectors (SRC/dense.c:747-750)
  DCK(cudaMemcpy2D(B, (size_t)*ldbp * kC, b.B, n * kC, n * kC, n, cudaMemcpyDeviceToHost));
  return jz == MR3_JOB_V ? copy_z_out(b, n, *mp, A, *ldap) : 0;
}

extern "C" int zhpgeig(int *itype, char *jobz, char *range, char *uplo, int *np, void *AP,
                       void *BP, double *vlp, double *vup, int *ilp, int *iup, int *mp,
                       double *W, void *Z, int *ldzp) {
  const int n = *np, jz = job_code(jobz[0]), rg = range_code(range[0]);
  const bool lower = uplo[0] == 'L' || uplo[0] == 'l';
  // SRC/dense.c:888-892 (n <= 1 refused), plus ldz and the range bounds
  if (n <= 1 || *itype < 1 || *itype > 3 || !is_uplo(uplo[0])) return 1;
  if (check_common(jz, rg, n, vlp, vup, ilp, iup)) return 1;
  if (jz == MR3_JOB_V && *ldzp < n) return 1;
  ZBufs b;
  const int ncols = rg == MR3_RANGE_I ? *iup - *ilp + 1 : n;
  int rc = zstart(b, n, jz, ncols);
  if (rc) return rc;
  const size_t np_ = (size_t)n * (n + 1) / 2;
  DCK(cudaMalloc((void **)&b.B, (size_t)n * n * kC));
  DCK(cudaMalloc((void **)&b.AP, np_ * kC));
  DCK(cudaMemset(b.B, 0, (size_t)n * n * kC));
  DCK(cudaMemcpy(b.AP, AP, np_ * kC, cudaMemcpyHostToDevice));
  k_herm_packed<<<kGrid, 256>>>(n, b.AP, b.A, lower, 0);
  DCK(cudaGetLastError());
  DCK(cudaMemcpy(b.AP, BP, np_ * kC, cudaMemcpyHostToDevice));
  k_herm_packed<<<kGrid, 256>>>(n, b.AP, b.B, lower, 0);
  DCK(cudaGetLastError());
  if ((rc = zreduce(b, *itype, lower, n))) return rc;
  if (jz == MR3_JOB_C && rg != MR3_RANGE_V) {
    *mp = rg == MR3_RANGE_A ? n : *iup - *ilp + 1;
  } else {
    if ((rc = zcore(b, jz, rg, lower, n, ncols, vlp, vup, ilp, iup, mp, W))) return rc;
    if (jz == MR3_JOB_V && (rc = zbacktransform(b, *itype, lower, n, *mp))) return rc;
  }
  // BP holds the packed Cholesky factor (zpptrf's output)
  k_herm_packed<<<kGrid, 256>>>(n, b.AP, b.B, lower, 1);
  DCK(cudaGetLastError());
  DCK(cudaMemcpy(BP, b.AP, np_ * kC, cudaMemcpyDeviceToHost));
  return jz == MR3_JOB_V ? copy_z_out(b, n, *mp, Z, *ldzp) : 0;
}

extern "C" void zheeig_(char *jobz, char *range, char *uplo, int *n, void *A, int *lda,
                        double *vl, double *vu, int *il, int *iu, int *m, double *W, void *Z,
                        int *ldz, int *info) {
  *info = zheeig(jobz, range, uplo, n, A, lda, vl, vu, il, iu, m, W, Z, ldz);
}

extern "C" void zhpeig_(char *jobz, char *range, char *uplo, int *n, void *AP, double *vl,
                        double *vu, int *il, int *iu, int *m, double *W, void *Z, int *ldz,
                        int *info) {
  *info = zhpeig(jobz, range, uplo, n, AP, vl, vu, il, iu, m, W, Z, ldz);
}

extern "C" void zhegeig_(int *itype, char *jobz, char *range, char *uplo, int *n, void *A,
                         int *lda, void *B, int *ldb, double *vl, double *vu, int *il, int *iu,
                         int *m, double *W, int *info) {
  *info = zhegeig(itype, jobz, range, uplo, n, A, lda, B, ldb, vl, vu, il, iu, m, W);
}

extern "C" void zhpgeig_(int *itype, char *jobz, char *range, char *uplo, int *n, void *AP,
                         void *BP, double *vl, double *vu, int *il, int *iu, int *m, double *W,
                         void *Z, int *ldz, int *info) {
  *info = zhpgeig(itype, jobz, range, uplo, n, AP, BP, vl, vu, il, iu, m, W, Z, ldz);
}
