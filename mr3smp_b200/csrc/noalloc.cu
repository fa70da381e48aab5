// noalloc.cu -- eigenvectors of an L D L^T representation with no allocation.
//
// Some callers cannot call cudaMalloc: code running inside a device-memory
// budget that another allocator owns (a framework's caching allocator that
// has reserved the device), or latency-critical loops where cudaMalloc's
// implicit device synchronisation is not acceptable.  For them this file
// offers mr3_cuda_eigvec_noalloc(): the twisted-factorisation eigenvector
// kernel of the solver (the singleton step, one dlar1v per eigenvalue),
// with its scratch in a file-scope device array instead of a context
// workspace.  The caller passes the representation, the eigenvalues and the
// output arrays; the call allocates nothing.
//
// Scratch: packed representation rows (4 * NMAX doubles), the pivot
// threshold, and, for each of NA_WARPS warps, two per-lane arrays of NMAX
// rows x 32 lanes: 16.8 MB that every GPU which loads the library holds
// until the process exits.  All calls share it and it keeps the last call's
// contents; every call rewrites what it reads before reading it, so nothing
// has to start at zero.  Calls that overlap on the GPU (different streams
// or host threads at the same time) race on it.
//
// The pivot threshold is the solver's, pivmin = DBL_MIN * max(1, max e_i^2)
// (SRC/mrrr_val.c:226-233), with the off-diagonal e_i of the represented
// matrix taken as D(i) L(i); for a root representation L D L^T = T - sigma I
// that is T's off-diagonal up to rounding.  Each warp runs on an SM of its
// own (one-warp blocks).
#include <cuda_runtime.h>
#include <float.h>

#include <mutex>

#include "mr3_cuda.h"
#include "mr3_device.cuh"

#define NA_NMAX 2048   // largest n accepted (MR3_NOALLOC_NMAX in mr3_cuda.h)
#define NA_WARPS 16    // warps that share the scratch
#define NA_ROWS_OFF 0
#define NA_PIV_OFF (4 * NA_NMAX)
#define NA_LANES_OFF (4 * NA_NMAX + 32)
#define NA_TOTAL (4 * NA_NMAX + 32 + NA_WARPS * 2 * NA_NMAX * 32)

static_assert(NA_NMAX == MR3_NOALLOC_NMAX, "limit must match the header");

static __device__ __align__(256) double g_noalloc_scratch[NA_TOTAL];

// Device address of g_noalloc_scratch, looked up once per device.
static double *g_na_ptr[128];
static std::mutex g_na_mu;

namespace {

// Rows of the representation: P[i] = (D(i), D(i)L(i)^2), Q[i] = (L(i), D(i)L(i)),
// and the pivot threshold (one block).
__global__ void __launch_bounds__(1024) k_na_pack(int n, const double *D, const double *L,
                                                  double *scratch) {
  __shared__ double red[32];
  double2 *P = reinterpret_cast<double2 *>(scratch + NA_ROWS_OFF);
  double2 *Q = P + NA_NMAX;
  double emax = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double dv = D[i];
    if (i < n - 1) {
      double lv = L[i];
      double ld = dv * lv;
      P[i] = make_double2(dv, ld * lv);
      Q[i] = make_double2(lv, ld);
      emax = fmax(emax, fabs(ld));
    } else {
      P[i] = make_double2(dv, 0.0);
      Q[i] = make_double2(0.0, 0.0);
    }
  }
  for (int o = 16; o > 0; o >>= 1) emax = fmax(emax, __shfl_xor_sync(0xffffffffu, emax, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = emax;
  __syncthreads();
  if (threadIdx.x == 0) {
    double e = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) e = fmax(e, red[w]);
    scratch[NA_PIV_OFF] = MR3_SAFMIN * fmax(1.0, e * e);
  }
}

// n = 1: every eigenvector is (1), support {1}.
__global__ void k_na_unit(int m, double *Z, int ldz, int *Zsupp) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < m; v += gridDim.x * blockDim.x) {
    Z[(size_t)v * ldz] = 1.0;
    Zsupp[2 * v] = 1;
    Zsupp[2 * v + 1] = 1;
  }
}

// One lane per eigenvalue: dlar1v with the twist index searched over 1..n,
// then the normalised vector (zero outside its support) into Z.
__global__ void __launch_bounds__(32)
k_na_vec(int n, int m, const double *lambda, double gaptol, double *Z, int ldz, int *Zsupp,
         double *scratch) {
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const double2 *P = reinterpret_cast<const double2 *>(scratch + NA_ROWS_OFF);
  const double2 *Q = P + NA_NMAX;
  const double pivmin = scratch[NA_PIV_OFF];
  double *X = scratch + NA_LANES_OFF + (size_t)gw * 2 * NA_NMAX * 32 + lane;
  double *Y = X + (size_t)NA_NMAX * 32;
  for (int v0 = gw * 32; v0 < m; v0 += NA_WARPS * 32) {
    const int v = v0 + lane;
    const bool active = v < m;
    r1v_state st;
    st.r = 0; st.mingma = 0.0; st.sawnan = false;
    int negc = 0;
    dv_r1v_factor(active, n, active ? lambda[v] : 0.0, P, Q, 1, pivmin, false, 0, X, Y, &negc,
                  &st);
    dlar1v_out o;
    o.isupp1 = 1; o.isupp2 = n; o.nrminv = 0.0; o.r = 0;
    dv_r1v_solve(active, n, Q, 1, gaptol, X, Y, st, &o);
    if (active) {
      double *zc = Z + (size_t)v * ldz;
      for (int k = 1; k <= n; k++) {
        double val = 0.0;
        if (k >= o.isupp1 && k <= o.isupp2) val = dv_zget(X, Y, o.r, k) * o.nrminv;
        zc[k - 1] = val;
      }
      Zsupp[2 * v] = o.isupp1;
      Zsupp[2 * v + 1] = o.isupp2;
    }
    __syncwarp();
  }
}

}  // namespace

extern "C" int mr3_cuda_eigvec_noalloc(int n, const double *D, const double *L, int m,
                                       const double *lambda, double gaptol, double *Z, int ldz,
                                       int *Zsupp, void *stream) {
  if (n < 1 || n > NA_NMAX || m < 0 || ldz < n) return MR3_EARG;
  if (m == 0) return MR3_OK;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128) return MR3_EMISC;
  double *scratch;
  {
    std::lock_guard<std::mutex> g(g_na_mu);
    if (!g_na_ptr[dev]) {
      double *p = nullptr;
      if (cudaGetSymbolAddress((void **)&p, g_noalloc_scratch) != cudaSuccess || !p)
        return MR3_EMISC;
      g_na_ptr[dev] = p;
    }
    scratch = g_na_ptr[dev];
  }
  cudaStream_t st = (cudaStream_t)stream;
  if (n == 1) {
    k_na_unit<<<(m + 255) / 256, 256, 0, st>>>(m, Z, ldz, Zsupp);
    return cudaGetLastError() == cudaSuccess ? MR3_OK : MR3_EMISC;
  }
  k_na_pack<<<1, 1024, 0, st>>>(n, D, L, scratch);
  k_na_vec<<<NA_WARPS, 32, 0, st>>>(n, m, lambda, gaptol, Z, ldz, Zsupp, scratch);
  return cudaGetLastError() == cudaSuccess ? MR3_OK : MR3_EMISC;
}
