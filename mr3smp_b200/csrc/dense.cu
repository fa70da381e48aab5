/*
 * dense.cu -- the dense symmetric driver dsyeig (SRC/dense.c:151-232).
 *
 * The reference scales A (dscale_matrix, SRC/dense.c:477-527), reduces it to
 * tridiagonal form with LAPACK's dsytrd, solves the tridiagonal problem with
 * mrrr(), back-transforms Z = Q Z with LAPACK's dormtr and unscales W.  Here
 * every step runs on the device that runs the tridiagonal solve, so A, the
 * Householder vectors, D, E and Z stay in HBM between the steps: the max-norm
 * and the scaling are two kernels of this file, the tridiagonal solve is the
 * batched solver (mr3_batched_device), and dsytrd/dormtr -- external LAPACK
 * calls in the reference as well -- are cuSOLVER's, loaded at first use so
 * that the rest of the library does not depend on it.
 */
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
  bool ok;
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
  g_cs.ok = g_cs.create && g_cs.destroy && g_cs.sytrd_ws && g_cs.sytrd && g_cs.ormtr_ws &&
            g_cs.ormtr;
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
  double *A = nullptr, *D = nullptr, *E = nullptr, *tau = nullptr, *W = nullptr, *Z = nullptr,
         *work = nullptr;
  int *Zsupp = nullptr, *info = nullptr, *nan = nullptr;
  unsigned long long *maxbits = nullptr;
  cusolverDnHandle_t h = nullptr;
  ~DenseBufs() {
    void *p[] = {A, D, E, tau, W, Z, work, Zsupp, info, nan, maxbits};
    for (void *q : p)
      if (q) cudaFree(q);
    if (h) g_cs.destroy(h);
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

}  // namespace

extern "C" int dsyeig(char *jobz, char *range, char *uplo, int *np, double *A, int *ldap,
                      double *vlp, double *vup, int *ilp, int *iup, int *mp, double *W,
                      double *Z, int *ldzp) {
  const int n = *np, jz = job_code(jobz[0]), rg = range_code(range[0]);
  const bool lower = uplo[0] == 'L' || uplo[0] == 'l';
  // argument checks of SRC/dense.c:177-186, plus the array extents that the
  // reference leaves to LAPACK (lda, ldz) and the triangle selector
  if (jz < 0 || rg < 0 || n <= 0) return 1;
  if (rg == MR3_RANGE_V) {
    if (*vup <= *vlp) return 1;
  } else if (rg == MR3_RANGE_I) {
    if (*ilp < 1 || *ilp > n || *iup < *ilp || *iup > n) return 1;
  }
  if (!(lower || uplo[0] == 'U' || uplo[0] == 'u') || *ldap < n) return 1;
  if (jz == MR3_JOB_V && *ldzp < n) return 1;
  // counting with range A or I needs no work (mrrr(), SRC/mrrr.c:130-138)
  if (jz == MR3_JOB_C && rg != MR3_RANGE_V) {
    *mp = rg == MR3_RANGE_A ? n : *iup - *ilp + 1;
    return 0;
  }
  pthread_once(&g_cs_once, load_cusolver);
  if (!g_cs.ok) return 2;
  DCK(cudaSetDevice(device_id()));

  DenseBufs b;
  const size_t nn = (size_t)n * n;
  const int ncols = rg == MR3_RANGE_I ? *iup - *ilp + 1 : n;
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
  DCK(cudaMemcpy2D(b.A, n * sizeof(double), A, (size_t)*ldap * sizeof(double), n * sizeof(double),
                   n, cudaMemcpyHostToDevice));
  DCK(cudaMemset(b.E, 0, n * sizeof(double)));
  DCK(cudaMemset(b.nan, 0, sizeof(int)));
  DCK(cudaMemset(b.maxbits, 0, sizeof(unsigned long long)));

  // scaling (dscale_matrix): into [rmin, rmax] when the max-norm is outside
  const double smlnum = DBL_MIN / DBL_EPSILON, bignum = 1.0 / smlnum;
  const double rmin = sqrt(smlnum), rmax = fmin(sqrt(bignum), 1.0 / sqrt(sqrt(DBL_MIN)));
  const int grid = 148 * 8;
  k_tri_absmax<<<grid, 256>>>(n, b.A, lower, b.maxbits, b.nan);
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
    k_tri_scale<<<grid, 256>>>(n, b.A, lower, sigma);
    DCK(cudaGetLastError());
    if (rg == MR3_RANGE_V) {
      *vlp *= sigma;
      *vup *= sigma;
    }
  }

  // reduction to tridiagonal form (dsytrd): D, E, tau; Q in A
  const cublasFillMode_t fill = lower ? CUBLAS_FILL_MODE_LOWER : CUBLAS_FILL_MODE_UPPER;
  SCK(g_cs.create(&b.h));
  int lw1 = 0, lw2 = 0;
  if (n > 1) SCK(g_cs.sytrd_ws(b.h, fill, n, b.A, n, b.D, b.E, b.tau, &lw1));
  if (n > 1 && jz == MR3_JOB_V)
    SCK(g_cs.ormtr_ws(b.h, CUBLAS_SIDE_LEFT, fill, CUBLAS_OP_N, n, ncols, b.A, n, b.tau, b.Z, n,
                      &lw2));
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
  if (jz == MR3_JOB_V && m > 0) {
    DCK(cudaDeviceSynchronize());
    if (n > 1) {
      SCK(g_cs.ormtr(b.h, CUBLAS_SIDE_LEFT, fill, CUBLAS_OP_N, n, m, b.A, n, b.tau, b.Z, n, b.work,
                     lw2, b.info));
      DCK(cudaMemcpy(&hinfo, b.info, sizeof(int), cudaMemcpyDeviceToHost));
      if (hinfo != 0) return 2;
    }
    DCK(cudaMemcpy2D(Z, (size_t)*ldzp * sizeof(double), b.Z, n * sizeof(double),
                     n * sizeof(double), m, cudaMemcpyDeviceToHost));
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

extern "C" void dsyeig_(char *jobz, char *range, char *uplo, int *n, double *A, int *lda,
                        double *vl, double *vu, int *il, int *iu, int *m, double *W, double *Z,
                        int *ldz, int *info) {
  *info = dsyeig(jobz, range, uplo, n, A, lda, vl, vu, il, iu, m, W, Z, ldz);
}
