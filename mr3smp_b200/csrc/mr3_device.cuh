// mr3_device.cuh -- thread-level FP64 numerics of the MRRR path for sm_100a.
//
// Each function follows one LAPACK 3.2.x routine vendored by the reference
// (SRC/LAPACK/od*.f) operation for operation, so that a thread computes the
// same bits as a sequential CPU run of that routine.  The translation unit is
// compiled with -fmad=false: no multiply-add contraction, IEEE division and
// square root, exactly the arithmetic of the Fortran.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#define MR3_EPS    2.220446049250313080847e-16   // dlamch('P') = DBL_EPSILON
#define MR3_SAFMIN 2.225073858507201383090e-308  // dlamch('S') = DBL_MIN
#define MR3_MAX_GROWTH   64.0                    // INCLUDE/mrrr.h MAX_GROWTH
#define MR3_MIN_RELGAP   1e-3                    // INCLUDE/mrrr.h MIN_RELGAP
#define MR3_MAX_TRY_ROOT 6                       // INCLUDE/mrrr.h MAX_TRY_ROOT
#define MR3_MAXITER      10                      // SRC/process_singleton.c:57
#define MR3_EXPAND_CAP   4096                    // bound on interval widening
#define MR3_LCG_A        33952834046453ULL       // dlaruv multiplier (SRC/LAPACK/odruv.f)

// An L D L^T representation is stored as two packed row arrays:
//   P[i] = (D(i), D(i)L(i)^2)   read by every Sturm count (dlaneg)
//   Q[i] = (L(i), D(i)L(i))     read in addition by the twisted factorization

static __device__ __forceinline__ int d_imin(int a, int b) { return a < b ? a : b; }
static __device__ __forceinline__ int d_imax(int a, int b) { return a > b ? a : b; }

// Deterministic natural log: log(x) = e*ln2 + 2*atanh((m-1)/(m+1)) with the
// atanh Taylor series to s^25 and the fdlibm hi/lo split of ln2.  Same
// operations as the CPU copy used by the oracle, hence the same bits.
static __device__ __noinline__ double dv_log(double x) {
  const double ln2_hi = 6.93147180369123816490e-01;
  const double ln2_lo = 1.90821492927058770002e-10;
  if (isnan(x) || x < 0.0) return __longlong_as_double(0x7ff8000000000000LL);
  if (x == 0.0) return -__longlong_as_double(0x7ff0000000000000LL);
  if (isinf(x)) return x;
  int e;
  double m = frexp(x, &e);
  if (m < 0.70710678118654752440) { m = m * 2.0; e = e - 1; }
  double s = (m - 1.0) / (m + 1.0);
  double s2 = s * s;
  double p = 1.0 / 25.0;
  p = 1.0 / 23.0 + s2 * p;
  p = 1.0 / 21.0 + s2 * p;
  p = 1.0 / 19.0 + s2 * p;
  p = 1.0 / 17.0 + s2 * p;
  p = 1.0 / 15.0 + s2 * p;
  p = 1.0 / 13.0 + s2 * p;
  p = 1.0 / 11.0 + s2 * p;
  p = 1.0 / 9.0 + s2 * p;
  p = 1.0 / 7.0 + s2 * p;
  p = 1.0 / 5.0 + s2 * p;
  p = 1.0 / 3.0 + s2 * p;
  double r = s + (s * s2) * p;
  return (double)e * ln2_hi + (2.0 * r + (double)e * ln2_lo);
}

// INT((LOG(a)-LOG(b))/LOG(2)) + 2: iteration cap of dlarrb/dlarrd/dlarrj.
static __device__ __forceinline__ int dv_itmax(double a, double b) {
  return (int)((dv_log(a) - dv_log(b)) / dv_log(2.0)) + 2;
}

#ifndef MR3_U
#define MR3_U 4     // rows per chunk of the software-pipelined sweeps
#endif

// Sturm count of T - x, IJOB=1 rule of dlaebz (SRC/LAPACK/odebz.f:255-270).
// tp[j] = (d[j], e2[j-1]); tp[0].y unused.  The threads of a warp count the
// same matrix, so every load is a broadcast that L1 serves; the plain loop
// is faster here than the chunked sweeps used for per-lane data.
static __device__ __noinline__ int dv_count_ijob1(int n, const double2 *__restrict__ tp,
                                           double pivmin, double x) {
  double2 v = tp[0];
  double tmp = v.x - x;
  if (fabs(tmp) < pivmin) tmp = -pivmin;
  int cnt = (tmp <= 0.0);
  for (int j = 1; j < n; j++) {
    v = tp[j];
    tmp = v.x - v.y / tmp - x;
    if (fabs(tmp) < pivmin) tmp = -pivmin;
    cnt += (tmp <= 0.0);
  }
  return cnt;
}

// Sturm count, IJOB=2/3 rule of dlaebz's serial loop (odebz.f loop 90).
static __device__ __forceinline__ int dv_count_bisect(int n, const double2 *__restrict__ tp,
                                               double pivmin, double c) {
  double2 v = tp[0];
  double tmp2 = v.x - c;
  int cnt = 0;
  if (tmp2 <= pivmin) { cnt = 1; tmp2 = fmin(tmp2, -pivmin); }
  for (int j = 1; j < n; j++) {
    v = tp[j];
    tmp2 = v.x - v.y / tmp2 - c;
    if (tmp2 <= pivmin) { cnt++; tmp2 = fmin(tmp2, -pivmin); }
  }
  return cnt;
}

// One interval of dlaebz IJOB=3 from the user-supplied point c.
static __device__ __noinline__ void dv_ijob3(int n, const double2 *__restrict__ tp, double pivmin,
                                      double abstol, double reltol, int nitmax, int nval,
                                      double c, double *a, double *b, int *na, int *nb) {
  for (int it = 1; it <= nitmax; it++) {
    int cnt = dv_count_bisect(n, tp, pivmin, c);
    if (cnt <= nval) { *a = c; *na = cnt; }
    if (cnt >= nval) { *b = c; *nb = cnt; }
    double w = fabs(*b - *a);
    double t = fmax(fabs(*b), fabs(*a));
    if (w < fmax(fmax(abstol, pivmin), reltol * t) || *na >= *nb) break;
    c = 0.5 * (*a + *b);
  }
}

// dv_ijob3 by a group of L lanes (L = 2..32, a power of two; every lane of
// the group passes the same arguments and gets the same results).  The
// first count is at the given point c, as in the loop; after it the points
// are midpoints, and the midpoints of the next log2(L) steps form a binary
// tree that follows from the current interval: lane t of the group counts
// at node max(t,1) (heap numbering; its interval computed along the node's
// path with the loop's operations), then the group walks the tree applying
// the loop's updates and tests after each step.  A count equal to nval
// closes the interval (a = b = c), which the width test then stops.  The
// same points, counts and results as dv_ijob3; log2(L) steps per count.
static __device__ __noinline__ void dv_ijob3_tree(int L, int n, const double2 *__restrict__ tp,
                                           double pivmin, double abstol, double reltol,
                                           int nitmax, int nval, double c, double *a_,
                                           double *b_, int *na_, int *nb_) {
  const int lane = threadIdx.x & 31;
  const int t = lane & (L - 1), g0 = lane - t, depth = 31 - __clz(L);
  const unsigned gm = ((L == 32) ? 0xffffffffu : ((1u << L) - 1u)) << g0;
  const int node_t = t == 0 ? 1 : t;
  const double tol0 = fmax(abstol, pivmin);
  double a = *a_, b = *b_;
  int na = *na_, nb = *nb_, it = 0;
  bool done = nitmax < 1;
  if (!done) {   // the first step, at the given point
    const int cnt = dv_count_bisect(n, tp, pivmin, c);
    if (cnt <= nval) { a = c; na = cnt; }
    if (cnt >= nval) { b = c; nb = cnt; }
    it = 1;
    const double w = fabs(b - a), tt = fmax(fabs(b), fabs(a));
    if (w < fmax(tol0, reltol * tt) || na >= nb || it >= nitmax) done = true;
  }
  while (!done) {
    double l = a, r = b;
    for (int k = 30 - __clz(node_t); k >= 0; k--) {
      const double m = 0.5 * (l + r);
      if ((node_t >> k) & 1) l = m; else r = m;
    }
    const int raw = dv_count_bisect(n, tp, pivmin, 0.5 * (l + r));
    int node = 1;
    for (int d = 0; d < depth; d++) {
      const int cv = __shfl_sync(gm, raw, g0 + node);
      if (!done) {
        const double cm = 0.5 * (a + b);
        if (cv <= nval) { a = cm; na = cv; }
        if (cv >= nval) { b = cm; nb = cv; }
        node = (cv < nval) ? 2 * node + 1 : 2 * node;
        it++;
        const double w = fabs(b - a), tt = fmax(fabs(b), fabs(a));
        if (w < fmax(tol0, reltol * tt) || na >= nb || it >= nitmax) done = true;
      }
    }
  }
  *a_ = a;
  *b_ = b;
  *na_ = na;
  *nb_ = nb;
}

// The interval of eigenvalue j under dlaebz IJOB=2 started from [a,b] with
// counts (na,nb): midpoint bisection of that one interval (odebz.f 90-120).
// it0 > 0 continues a bisection whose first it0 steps ended in [a,b].
static __device__ __noinline__ int dv_bisect_one(int n, const double2 *__restrict__ tp, double pivmin,
                                          double abstol, double reltol, int itmax, int j,
                                          double *a, double *b, int na, int nb, int *iters,
                                          int it0 = 0) {
  double c = 0.5 * (*a + *b);
  for (int it = it0 + 1; it <= itmax; it++) {
    int cnt = dv_count_bisect(n, tp, pivmin, c);
    cnt = d_imin(nb, d_imax(na, cnt));
    if (j <= cnt) { *b = c; nb = cnt; } else { *a = c; na = cnt; }
    double w = fabs(*b - *a);
    double t = fmax(fabs(*b), fabs(*a));
    *iters = it;
    if (w < fmax(fmax(abstol, pivmin), reltol * t) || na >= nb) return 1;
    c = 0.5 * (*a + *b);
  }
  return 0;
}

// dv_bisect_one by a group of L lanes (L = 4..32; groups independent): the
// midpoints of the next log2(L) steps form a binary tree that follows from
// the current interval; lane t of the group counts at node max(t,1) (its
// interval computed along the node's path with the loop's operations), then
// the group walks the tree, clamping each count to the walk's (na, nb) and
// applying the loop's convergence test after each step, as the sequential
// loop does.  The same sequence of intervals; log2(L) steps per count.
static __device__ __noinline__ int dv_bisect_tree(int L, int n, const double2 *__restrict__ tp,
                                           double pivmin, double abstol, double reltol, int itmax,
                                           int j, double *a_, double *b_, int na, int nb,
                                           int *iters) {
  const int lane = threadIdx.x & 31;
  const int t = lane & (L - 1), g0 = lane - t, depth = 31 - __clz(L);
  const unsigned gm = ((L == 32) ? 0xffffffffu : ((1u << L) - 1u)) << g0;
  const int node_t = t == 0 ? 1 : t;
  double a = *a_, b = *b_;
  int it = 0, done = itmax < 1, conv = 0;
  while (!done) {
    double l = a, r = b;
    for (int k = 30 - __clz(node_t); k >= 0; k--) {
      const double m = 0.5 * (l + r);
      if ((node_t >> k) & 1) l = m; else r = m;
    }
    const int raw = dv_count_bisect(n, tp, pivmin, 0.5 * (l + r));
    int node = 1;
    for (int d = 0; d < depth; d++) {
      const int cv = __shfl_sync(gm, raw, g0 + node);
      if (!done) {
        const double c = 0.5 * (a + b);
        const int cnt = d_imin(nb, d_imax(na, cv));
        if (j <= cnt) { b = c; nb = cnt; node = 2 * node; } else { a = c; na = cnt; node = 2 * node + 1; }
        it++;
        const double w = fabs(b - a), tt = fmax(fabs(b), fabs(a));
        if (w < fmax(fmax(abstol, pivmin), reltol * tt) || na >= nb) { done = 1; conv = 1; }
        else if (it >= itmax) done = 1;
      }
    }
  }
  *a_ = a;
  *b_ = b;
  *iters = it;
  return conv;
}

// dlaneg (SRC/LAPACK/odneg.f:98-163) on packed rows P[(i)*ps]; r is 1-based.
// U > 1: rows are read in chunks of U with the next chunk's loads issued
// ahead of the current chunk's arithmetic (see the dlar1v sweeps below),
// for representations that the threads of a warp do not share (cluster
// groups in the level arenas); the NaN re-run of a 128-row block reads its
// rows again.  U == 1: the plain row loop, best when a warp's threads all
// read the same rows (a block's root representation), which L1 serves.
template <int U>
static __device__ __noinline__ int dv_dlaneg(int n, const double2 *__restrict__ P, int ps, double sigma,
                                      int r) {
  static_assert(128 % U == 0, "chunks must not straddle the 128-row blocks");
  const int blklen = 128;
  int negcnt = 0;
  double t = -sigma;
  if constexpr (U == 1) {
    for (int bj = 1; bj <= r - 1; bj += blklen) {
      int jend = d_imin(bj + blklen - 1, r - 1);
      int neg1 = 0;
      double bsav = t;
      for (int j = bj; j <= jend; j++) {
        const double2 v = P[(size_t)(j - 1) * ps];
        double dplus = v.x + t;
        neg1 += (dplus < 0.0);
        double tmp = t / dplus;
        t = tmp * v.y - sigma;
      }
      if (isnan(t)) {
        neg1 = 0;
        t = bsav;
        for (int j = bj; j <= jend; j++) {
          const double2 v = P[(size_t)(j - 1) * ps];
          double dplus = v.x + t;
          neg1 += (dplus < 0.0);
          double tmp = t / dplus;
          if (isnan(tmp)) tmp = 1.0;
          t = tmp * v.y - sigma;
        }
      }
      negcnt += neg1;
    }
    double p = P[(size_t)(n - 1) * ps].x - sigma;
    for (int bj = n - 1; bj >= r; bj -= blklen) {
      int jend = d_imax(bj - blklen + 1, r);
      int neg2 = 0;
      double bsav = p;
      for (int j = bj; j >= jend; j--) {
        const double2 v = P[(size_t)(j - 1) * ps];
        double dminus = v.y + p;
        neg2 += (dminus < 0.0);
        double tmp = p / dminus;
        p = tmp * v.x - sigma;
      }
      if (isnan(p)) {
        neg2 = 0;
        p = bsav;
        for (int j = bj; j >= jend; j--) {
          const double2 v = P[(size_t)(j - 1) * ps];
          double dminus = v.y + p;
          neg2 += (dminus < 0.0);
          double tmp = p / dminus;
          if (isnan(tmp)) tmp = 1.0;
          p = tmp * v.x - sigma;
        }
      }
      negcnt += neg2;
    }
    double gamma = (t + sigma) + p;
    if (gamma < 0.0) negcnt++;
    return negcnt;
  }
  if (r - 1 >= 1) {
    const int last = r - 1;
    double2 c[U], nx[U];
#pragma unroll
    for (int u = 0; u < U; u++) c[u] = P[(size_t)(d_imin(1 + u, last) - 1) * ps];
    for (int bj = 1; bj <= last; bj += blklen) {
      const int jend = d_imin(bj + blklen - 1, last);
      int neg1 = 0;
      const double bsav = t;
      for (int j0 = bj; j0 <= jend; j0 += U) {
#pragma unroll
        for (int u = 0; u < U; u++) nx[u] = P[(size_t)(d_imin(j0 + U + u, last) - 1) * ps];
#pragma unroll
        for (int u = 0; u < U; u++) {
          if (j0 + u <= jend) {
            double dplus = c[u].x + t;
            neg1 += (dplus < 0.0);
            double tmp = t / dplus;
            t = tmp * c[u].y - sigma;
          }
        }
#pragma unroll
        for (int u = 0; u < U; u++) c[u] = nx[u];
      }
      if (isnan(t)) {
        neg1 = 0;
        t = bsav;
        for (int j = bj; j <= jend; j++) {
          const double2 v = P[(size_t)(j - 1) * ps];
          double dplus = v.x + t;
          neg1 += (dplus < 0.0);
          double tmp = t / dplus;
          if (isnan(tmp)) tmp = 1.0;
          t = tmp * v.y - sigma;
        }
      }
      negcnt += neg1;
    }
  }
  double p = P[(size_t)(n - 1) * ps].x - sigma;
  if (n - 1 >= r) {
    double2 c[U], nx[U];
#pragma unroll
    for (int u = 0; u < U; u++) c[u] = P[(size_t)(d_imax(n - 1 - u, r) - 1) * ps];
    for (int bj = n - 1; bj >= r; bj -= blklen) {
      const int jend = d_imax(bj - blklen + 1, r);
      int neg2 = 0;
      const double bsav = p;
      for (int j0 = bj; j0 >= jend; j0 -= U) {
#pragma unroll
        for (int u = 0; u < U; u++) nx[u] = P[(size_t)(d_imax(j0 - U - u, r) - 1) * ps];
#pragma unroll
        for (int u = 0; u < U; u++) {
          if (j0 - u >= jend) {
            double dminus = c[u].y + p;
            neg2 += (dminus < 0.0);
            double tmp = p / dminus;
            p = tmp * c[u].x - sigma;
          }
        }
#pragma unroll
        for (int u = 0; u < U; u++) c[u] = nx[u];
      }
      if (isnan(p)) {
        neg2 = 0;
        p = bsav;
        for (int j = bj; j >= jend; j--) {
          const double2 v = P[(size_t)(j - 1) * ps];
          double dminus = v.y + p;
          neg2 += (dminus < 0.0);
          double tmp = p / dminus;
          if (isnan(tmp)) tmp = 1.0;
          p = tmp * v.x - sigma;
        }
      }
      negcnt += neg2;
    }
  }
  double gamma = (t + sigma) + p;
  if (gamma < 0.0) negcnt++;
  return negcnt;
}

// One interval of dlarrb (SRC/LAPACK/odrrb.f:136-293).  Intervals of one
// dlarrb call never read each other's state: the convergence test reads the
// gaps of the input WGAP, which dlarrb rewrites only after every interval has
// converged.  So one thread per interval yields the sequential result.
//   i      : 1-based eigenvalue index of this interval (IFIRST..ILAST)
//   first  : i == IFIRST (initial-phase left gap is then the own right gap)
//   has_left: II > 1 (main-loop left gap is WGAP(II-1))
//   w, werr: in/out; updated only if the interval went through the main loop
// Returns the number of counts spent, or -1 if a widening loop hit its cap.
template <int U>
static __device__ __noinline__ int dv_dlarrb_one(int n, const double2 *__restrict__ R, int ps, int i,
                                          int first,
                                          int has_left, double rgap_own, double lgap_in,
                                          double rtol1, double rtol2, double pivmin,
                                          int maxitr, int r, double *w, double *werr,
                                          int *ncount) {
  double mnwdth = 2.0 * pivmin;
  double left = *w - *werr, right = *w + *werr;
  double gap = fmin(first ? rgap_own : lgap_in, rgap_own);
  double back = *werr;
  int negcnt, cap, status = 0;
  int nc = 0;
  for (cap = 0; cap < MR3_EXPAND_CAP; cap++) {
    negcnt = dv_dlaneg<U>(n, R, ps, left, r);
    nc++;
    if (negcnt > i - 1) { left = left - back; back = 2.0 * back; } else break;
  }
  if (cap == MR3_EXPAND_CAP) status = -1;
  back = *werr;
  for (cap = 0; cap < MR3_EXPAND_CAP; cap++) {
    negcnt = dv_dlaneg<U>(n, R, ps, right, r);
    nc++;
    if (negcnt < i) { right = right + back; back = 2.0 * back; } else break;
  }
  if (cap == MR3_EXPAND_CAP) status = -1;
  *ncount += nc;
  double width = 0.5 * fabs(left - right);
  double tmp = fmax(fabs(left), fabs(right));
  double cvrgd = fmax(rtol1 * gap, rtol2 * tmp);
  if (width <= cvrgd || width <= mnwdth) return status;   // converged early: W, WERR kept
  gap = fmin(has_left ? lgap_in : rgap_own, rgap_own);
  for (int iter = 0; iter <= maxitr; iter++) {
    double mid = 0.5 * (left + right);
    width = right - mid;
    tmp = fmax(fabs(left), fabs(right));
    cvrgd = fmax(rtol1 * gap, rtol2 * tmp);
    if (width <= cvrgd || width <= mnwdth || iter == maxitr) break;
    negcnt = dv_dlaneg<U>(n, R, ps, mid, r);
    *ncount += 1;
    if (negcnt <= i - 1) left = mid; else right = mid;
  }
  *w = 0.5 * (left + right);
  *werr = right - *w;
  return status;
}

// dv_dlarrb_one for one interval per group of L lanes (L = 4, 8, 16 or 32,
// the same for the whole warp; every lane of a group calls it with the same
// arguments and gets the same results; groups are independent, a group may
// skip the call).  The bisection
// midpoints of the next log2(L) steps form a binary tree whose nodes follow
// from the current interval alone: lane t of the group evaluates the count
// at node max(t,1) (heap numbering, computed along the node's path with the
// same operations the sequential loop uses), then the group walks the tree
// with the counts, applying the sequential loop's convergence test before
// each step.  The widening loops are evaluated the same way, L/2 candidate
// ends per side in one sweep.  The sequence of intervals is exactly the
// sequential one.
static __device__ __noinline__ int dv_dlarrb_tree(int L, int n, const double2 *__restrict__ R, int ps,
                                           int i, int first, int has_left, double rgap_own,
                                           double lgap_in, double rtol1, double rtol2,
                                           double pivmin, int maxitr, int r, double *w,
                                           double *werr, int *ncount) {
  const int lane = threadIdx.x & 31;
  const int t = lane & (L - 1), g0 = lane - t, half = L >> 1;
  const int depth = 31 - __clz(L);
  const unsigned gbits = (L == 32) ? 0xffffffffu : ((1u << L) - 1u);
  const unsigned full = gbits << g0;   // the group's lanes: groups run independently
  const double mnwdth = 2.0 * pivmin;
  double left = *w - *werr, right = *w + *werr;
  double gap = fmin(first ? rgap_own : lgap_in, rgap_own);
  int status = 0;
  // widening: the first L/2 lanes hold the left end after 0..L/2-1 widening
  // steps, the others the right end; the first candidate that passes is the
  // end the sequential loop stops at
  {
    const int side = t >= half, k = t & (half - 1);
    double xs0 = left, xs1 = right, bs0 = *werr, bs1 = *werr;
    bool need0 = true, need1 = true;
    int steps0 = 0, steps1 = 0;
    while (__any_sync(full, need0 || need1)) {
      double x = side ? xs1 : xs0, back = side ? bs1 : bs0;
      for (int j = 0; j < k; j++) { x = side ? x + back : x - back; back = 2.0 * back; }
      const bool mine = side ? need1 : need0;
      int cnt = 0;
      if (mine) cnt = dv_dlaneg<MR3_U>(n, R, ps, x, r);
      const bool ok = mine && (side ? (cnt >= i) : (cnt <= i - 1));
      const unsigned gb = (__ballot_sync(full, ok) >> g0) & gbits;
      for (int sd = 0; sd < 2; sd++) {
        const unsigned pass = (gb >> (half * sd)) & ((1u << half) - 1u);
        const int k0 = pass ? __ffs(pass) - 1 : half - 1;
        const double xsrc = __shfl_sync(full, x, g0 + half * sd + k0);
        const double bsrc = __shfl_sync(full, back, g0 + half * sd + k0);
        bool &need = sd ? need1 : need0;
        double &xs = sd ? xs1 : xs0, &bs = sd ? bs1 : bs0;
        int &steps = sd ? steps1 : steps0;
        if (!need) continue;
        if (pass) {
          *ncount += k0 + 1;
          xs = xsrc;
          need = false;
        } else {
          *ncount += half;
          xs = sd ? xsrc + bsrc : xsrc - bsrc;
          bs = 2.0 * bsrc;
          steps += half;
          if (steps >= MR3_EXPAND_CAP) { status = -1; need = false; }
        }
      }
    }
    left = xs0;
    right = xs1;
  }
  double width = 0.5 * fabs(left - right);
  double tmp = fmax(fabs(left), fabs(right));
  double cvrgd = fmax(rtol1 * gap, rtol2 * tmp);
  const bool early = (width <= cvrgd || width <= mnwdth);   // W, WERR kept
  bool done = early;
  gap = fmin(has_left ? lgap_in : rgap_own, rgap_own);
  int iter = 0;
  const int node_t = t == 0 ? 1 : t;
  while (__any_sync(full, !done)) {
    double l = left, rr = right;
    for (int b = 30 - __clz(node_t); b >= 0; b--) {
      const double m = 0.5 * (l + rr);
      if ((node_t >> b) & 1) l = m; else rr = m;
    }
    int cnt = 0;
    if (!done) cnt = dv_dlaneg<MR3_U>(n, R, ps, 0.5 * (l + rr), r);
    int node = 1;
    for (int d = 0; d < depth; d++) {
      const int c = __shfl_sync(full, cnt, g0 + node);
      if (!done) {
        const double mid = 0.5 * (left + right);
        width = right - mid;
        tmp = fmax(fabs(left), fabs(right));
        cvrgd = fmax(rtol1 * gap, rtol2 * tmp);
        if (width <= cvrgd || width <= mnwdth || iter == maxitr) {
          done = true;
        } else {
          *ncount += 1;
          if (c <= i - 1) { left = mid; node = 2 * node + 1; } else { right = mid; node = 2 * node; }
          iter++;
        }
      }
    }
  }
  if (!early) {
    *w = 0.5 * (left + right);
    *werr = right - *w;
  }
  return status;
}

/* ------------------------------------------------------------------------
 * dqds on one thread: all eigenvalues of a positive definite L D L^T to
 * high relative accuracy (LAPACK 3.2.2 dlasq2-dlasq6, SRC/LAPACK/odsq2.f -
 * odsq6.f; the reference calls it at SRC/mrrr_val.c:464-477), operation for
 * operation as written there.  Z is the qd
 * array in Fortran's 1-based numbering, Zq(i) = z[i-1].  IEEE arithmetic is
 * assumed (odsq2.f's IEEE flag from ilaenv 10/11 is true on this hardware);
 * MIN and MAX propagate a NaN so that dlasq3's NaN test sees it.
 * ------------------------------------------------------------------------ */
#define Zq(i) z[(i) - 1]

static __device__ __forceinline__ double dv_fmin2(double a, double b) { return (a != a || b != b) ? NAN : (a < b ? a : b); }
static __device__ __forceinline__ double dv_fmax2(double a, double b) { return (a != a || b != b) ? NAN : (a > b ? a : b); }

/* odsq5.f: one dqds transform with shift tau (IEEE form). */
static __device__ void dv_dlasq5(int i0, int n0, double *z, int pp, double tau, double *dmin,
                      double *dmin1, double *dmin2, double *dn, double *dnm1, double *dnm2)
{
  int j4, j4p2;
  double d, emin, temp;
  if (n0 - i0 - 1 <= 0) return;
  j4 = 4 * i0 + pp - 3;
  emin = Zq(j4 + 4);
  d = Zq(j4) - tau;
  *dmin = d;
  *dmin1 = -Zq(j4);
  if (pp == 0) {
    for (j4 = 4 * i0; j4 <= 4 * (n0 - 3); j4 += 4) {
      Zq(j4 - 2) = d + Zq(j4 - 1);
      temp = Zq(j4 + 1) / Zq(j4 - 2);
      d = d * temp - tau;
      *dmin = dv_fmin2(*dmin, d);
      Zq(j4) = Zq(j4 - 1) * temp;
      emin = dv_fmin2(Zq(j4), emin);
    }
  } else {
    for (j4 = 4 * i0; j4 <= 4 * (n0 - 3); j4 += 4) {
      Zq(j4 - 3) = d + Zq(j4);
      temp = Zq(j4 + 2) / Zq(j4 - 3);
      d = d * temp - tau;
      *dmin = dv_fmin2(*dmin, d);
      Zq(j4 - 1) = Zq(j4) * temp;
      emin = dv_fmin2(Zq(j4 - 1), emin);
    }
  }
  *dnm2 = d;
  *dmin2 = *dmin;
  j4 = 4 * (n0 - 2) - pp;
  j4p2 = j4 + 2 * pp - 1;
  Zq(j4 - 2) = *dnm2 + Zq(j4p2);
  Zq(j4) = Zq(j4p2 + 2) * (Zq(j4p2) / Zq(j4 - 2));
  *dnm1 = Zq(j4p2 + 2) * (*dnm2 / Zq(j4 - 2)) - tau;
  *dmin = dv_fmin2(*dmin, *dnm1);
  *dmin1 = *dmin;
  j4 = j4 + 4;
  j4p2 = j4 + 2 * pp - 1;
  Zq(j4 - 2) = *dnm1 + Zq(j4p2);
  Zq(j4) = Zq(j4p2 + 2) * (Zq(j4p2) / Zq(j4 - 2));
  *dn = Zq(j4p2 + 2) * (*dnm1 / Zq(j4 - 2)) - tau;
  *dmin = dv_fmin2(*dmin, *dn);
  Zq(j4 + 2) = *dn;
  Zq(4 * n0 - pp) = emin;
}

/* odsq6.f: one dqd transform (no shift), guarded against underflow. */
static __device__ void dv_dlasq6(int i0, int n0, double *z, int pp, double *dmin, double *dmin1,
                      double *dmin2, double *dn, double *dnm1, double *dnm2)
{
  int j4, j4p2;
  double d, emin, temp;
  const double safmin = MR3_SAFMIN;
  if (n0 - i0 - 1 <= 0) return;
  j4 = 4 * i0 + pp - 3;
  emin = Zq(j4 + 4);
  d = Zq(j4);
  *dmin = d;
  if (pp == 0) {
    for (j4 = 4 * i0; j4 <= 4 * (n0 - 3); j4 += 4) {
      Zq(j4 - 2) = d + Zq(j4 - 1);
      if (Zq(j4 - 2) == 0.0) {
        Zq(j4) = 0.0;
        d = Zq(j4 + 1);
        *dmin = d;
        emin = 0.0;
      } else if (safmin * Zq(j4 + 1) < Zq(j4 - 2) && safmin * Zq(j4 - 2) < Zq(j4 + 1)) {
        temp = Zq(j4 + 1) / Zq(j4 - 2);
        Zq(j4) = Zq(j4 - 1) * temp;
        d = d * temp;
      } else {
        Zq(j4) = Zq(j4 + 1) * (Zq(j4 - 1) / Zq(j4 - 2));
        d = Zq(j4 + 1) * (d / Zq(j4 - 2));
      }
      *dmin = dv_fmin2(*dmin, d);
      emin = dv_fmin2(emin, Zq(j4));
    }
  } else {
    for (j4 = 4 * i0; j4 <= 4 * (n0 - 3); j4 += 4) {
      Zq(j4 - 3) = d + Zq(j4);
      if (Zq(j4 - 3) == 0.0) {
        Zq(j4 - 1) = 0.0;
        d = Zq(j4 + 2);
        *dmin = d;
        emin = 0.0;
      } else if (safmin * Zq(j4 + 2) < Zq(j4 - 3) && safmin * Zq(j4 - 3) < Zq(j4 + 2)) {
        temp = Zq(j4 + 2) / Zq(j4 - 3);
        Zq(j4 - 1) = Zq(j4) * temp;
        d = d * temp;
      } else {
        Zq(j4 - 1) = Zq(j4 + 2) * (Zq(j4) / Zq(j4 - 3));
        d = Zq(j4 + 2) * (d / Zq(j4 - 3));
      }
      *dmin = dv_fmin2(*dmin, d);
      emin = dv_fmin2(emin, Zq(j4 - 1));
    }
  }
  *dnm2 = d;
  *dmin2 = *dmin;
  j4 = 4 * (n0 - 2) - pp;
  j4p2 = j4 + 2 * pp - 1;
  Zq(j4 - 2) = *dnm2 + Zq(j4p2);
  if (Zq(j4 - 2) == 0.0) {
    Zq(j4) = 0.0;
    *dnm1 = Zq(j4p2 + 2);
    *dmin = *dnm1;
    emin = 0.0;
  } else if (safmin * Zq(j4p2 + 2) < Zq(j4 - 2) && safmin * Zq(j4 - 2) < Zq(j4p2 + 2)) {
    temp = Zq(j4p2 + 2) / Zq(j4 - 2);
    Zq(j4) = Zq(j4p2) * temp;
    *dnm1 = *dnm2 * temp;
  } else {
    Zq(j4) = Zq(j4p2 + 2) * (Zq(j4p2) / Zq(j4 - 2));
    *dnm1 = Zq(j4p2 + 2) * (*dnm2 / Zq(j4 - 2));
  }
  *dmin = dv_fmin2(*dmin, *dnm1);
  *dmin1 = *dmin;
  j4 = j4 + 4;
  j4p2 = j4 + 2 * pp - 1;
  Zq(j4 - 2) = *dnm1 + Zq(j4p2);
  if (Zq(j4 - 2) == 0.0) {
    Zq(j4) = 0.0;
    *dn = Zq(j4p2 + 2);
    *dmin = *dn;
    emin = 0.0;
  } else if (safmin * Zq(j4p2 + 2) < Zq(j4 - 2) && safmin * Zq(j4 - 2) < Zq(j4p2 + 2)) {
    temp = Zq(j4p2 + 2) / Zq(j4 - 2);
    Zq(j4) = Zq(j4p2) * temp;
    *dn = *dnm1 * temp;
  } else {
    Zq(j4) = Zq(j4p2 + 2) * (Zq(j4p2) / Zq(j4 - 2));
    *dn = Zq(j4p2 + 2) * (*dnm1 / Zq(j4 - 2));
  }
  *dmin = dv_fmin2(*dmin, *dn);
  Zq(j4 + 2) = *dn;
  Zq(4 * n0 - pp) = emin;
}

/* dqds shift state carried between calls of dlasq3 (odsq2.f's locals). */
typedef struct {
  int ttype;
  double dmin1, dmin2, dn, dn1, dn2, g, tau;
} dv_sq_t;

/* odsq4.f: the shift. */
static __device__ void dv_dlasq4(int i0, int n0, const double *z, int pp, int n0in, double dmin,
                      dv_sq_t *q)
{
  const double cnst1 = 0.5630, cnst2 = 1.010, cnst3 = 1.050;
  const double qurtr = 0.250, third = 0.3330, half = 0.50, hundrd = 100.0;
  int i4, nn, np;
  double a2, b1, b2, gam, gap1, gap2, s = 0.0;
  const double dmin1 = q->dmin1, dmin2 = q->dmin2, dn = q->dn, dn1 = q->dn1, dn2 = q->dn2;
  if (dmin <= 0.0) {
    q->tau = -dmin;
    q->ttype = -1;
    return;
  }
  nn = 4 * n0 + pp;
  if (n0in == n0) {
    if (dmin == dn || dmin == dn1) {
      b1 = sqrt(Zq(nn - 3)) * sqrt(Zq(nn - 5));
      b2 = sqrt(Zq(nn - 7)) * sqrt(Zq(nn - 9));
      a2 = Zq(nn - 7) + Zq(nn - 5);
      if (dmin == dn && dmin1 == dn1) {
        gap2 = dmin2 - a2 - dmin2 * qurtr;
        if (gap2 > 0.0 && gap2 > b2) gap1 = a2 - dn - (b2 / gap2) * b2;
        else gap1 = a2 - dn - (b1 + b2);
        if (gap1 > 0.0 && gap1 > b1) {
          s = dv_fmax2(dn - (b1 / gap1) * b1, half * dmin);
          q->ttype = -2;
        } else {
          s = 0.0;
          if (dn > b1) s = dn - b1;
          if (a2 > (b1 + b2)) s = dv_fmin2(s, a2 - (b1 + b2));
          s = dv_fmax2(s, third * dmin);
          q->ttype = -3;
        }
      } else {
        q->ttype = -4;
        s = qurtr * dmin;
        if (dmin == dn) {
          gam = dn;
          a2 = 0.0;
          if (Zq(nn - 5) > Zq(nn - 7)) return;   /* tau unchanged, as odsq4.f returns */
          b2 = Zq(nn - 5) / Zq(nn - 7);
          np = nn - 9;
        } else {
          np = nn - 2 * pp;
          b2 = Zq(np - 2);
          gam = dn1;
          if (Zq(np - 4) > Zq(np - 2)) return;   /* tau unchanged, as odsq4.f returns */
          a2 = Zq(np - 4) / Zq(np - 2);
          if (Zq(nn - 9) > Zq(nn - 11)) return;   /* tau unchanged, as odsq4.f returns */
          b2 = Zq(nn - 9) / Zq(nn - 11);
          np = nn - 13;
        }
        a2 = a2 + b2;
        for (i4 = np; i4 >= 4 * i0 - 1 + pp; i4 -= 4) {
          if (b2 == 0.0) break;
          b1 = b2;
          if (Zq(i4) > Zq(i4 - 2)) return;   /* tau unchanged, as odsq4.f returns */
          b2 = b2 * (Zq(i4) / Zq(i4 - 2));
          a2 = a2 + b2;
          if (hundrd * dv_fmax2(b2, b1) < a2 || cnst1 < a2) break;
        }
        a2 = cnst3 * a2;
        if (a2 < cnst1) s = gam * (1.0 - sqrt(a2)) / (1.0 + a2);
      }
    } else if (dmin == dn2) {
      q->ttype = -5;
      s = qurtr * dmin;
      np = nn - 2 * pp;
      b1 = Zq(np - 2);
      b2 = Zq(np - 6);
      gam = dn2;
      if (Zq(np - 8) > b2 || Zq(np - 4) > b1) return;   /* tau unchanged, as odsq4.f returns */
      a2 = (Zq(np - 8) / b2) * (1.0 + Zq(np - 4) / b1);
      if (n0 - i0 > 2) {
        b2 = Zq(nn - 13) / Zq(nn - 15);
        a2 = a2 + b2;
        for (i4 = nn - 17; i4 >= 4 * i0 - 1 + pp; i4 -= 4) {
          if (b2 == 0.0) break;
          b1 = b2;
          if (Zq(i4) > Zq(i4 - 2)) return;   /* tau unchanged, as odsq4.f returns */
          b2 = b2 * (Zq(i4) / Zq(i4 - 2));
          a2 = a2 + b2;
          if (hundrd * dv_fmax2(b2, b1) < a2 || cnst1 < a2) break;
        }
        a2 = cnst3 * a2;
      }
      if (a2 < cnst1) s = gam * (1.0 - sqrt(a2)) / (1.0 + a2);
    } else {
      if (q->ttype == -6) q->g = q->g + third * (1.0 - q->g);
      else if (q->ttype == -18) q->g = qurtr * third;
      else q->g = qurtr;
      s = q->g * dmin;
      q->ttype = -6;
    }
  } else if (n0in == n0 + 1) {
    if (dmin1 == dn1 && dmin2 == dn2) {
      q->ttype = -7;
      s = third * dmin1;
      if (Zq(nn - 5) > Zq(nn - 7)) return;   /* tau unchanged, as odsq4.f returns */
      b1 = Zq(nn - 5) / Zq(nn - 7);
      b2 = b1;
      if (b2 != 0.0) {
        for (i4 = 4 * n0 - 9 + pp; i4 >= 4 * i0 - 1 + pp; i4 -= 4) {
          a2 = b1;
          if (Zq(i4) > Zq(i4 - 2)) return;   /* tau unchanged, as odsq4.f returns */
          b1 = b1 * (Zq(i4) / Zq(i4 - 2));
          b2 = b2 + b1;
          if (hundrd * dv_fmax2(b1, a2) < b2) break;
        }
      }
      b2 = sqrt(cnst3 * b2);
      a2 = dmin1 / (1.0 + b2 * b2);
      gap2 = half * dmin2 - a2;
      if (gap2 > 0.0 && gap2 > b2 * a2) {
        s = dv_fmax2(s, a2 * (1.0 - cnst2 * a2 * (b2 / gap2) * b2));
      } else {
        s = dv_fmax2(s, a2 * (1.0 - cnst2 * b2));
        q->ttype = -8;
      }
    } else {
      s = qurtr * dmin1;
      if (dmin1 == dn1) s = half * dmin1;
      q->ttype = -9;
    }
  } else if (n0in == n0 + 2) {
    if (dmin2 == dn2 && 2.0 * Zq(nn - 5) < Zq(nn - 7)) {
      q->ttype = -10;
      s = third * dmin2;
      if (Zq(nn - 5) > Zq(nn - 7)) return;   /* tau unchanged, as odsq4.f returns */
      b1 = Zq(nn - 5) / Zq(nn - 7);
      b2 = b1;
      if (b2 != 0.0) {
        for (i4 = 4 * n0 - 9 + pp; i4 >= 4 * i0 - 1 + pp; i4 -= 4) {
          if (Zq(i4) > Zq(i4 - 2)) return;   /* tau unchanged, as odsq4.f returns */
          b1 = b1 * (Zq(i4) / Zq(i4 - 2));
          b2 = b2 + b1;
          if (hundrd * b1 < b2) break;
        }
      }
      b2 = sqrt(cnst3 * b2);
      a2 = dmin2 / (1.0 + b2 * b2);
      gap2 = Zq(nn - 7) + Zq(nn - 9) - sqrt(Zq(nn - 11)) * sqrt(Zq(nn - 9)) - a2;
      if (gap2 > 0.0 && gap2 > b2 * a2) s = dv_fmax2(s, a2 * (1.0 - cnst2 * a2 * (b2 / gap2) * b2));
      else s = dv_fmax2(s, a2 * (1.0 - cnst2 * b2));
    } else {
      s = qurtr * dmin2;
      q->ttype = -11;
    }
  } else if (n0in > n0 + 2) {
    s = 0.0;
    q->ttype = -12;
  }
  q->tau = s;
}

/* odsq3.f: deflation, the shift and one dqds step (with retries). */
static __device__ void dv_dlasq3(int i0, int *n0p, double *z, int *ppp, double *dminp, double *sigmap,
                      double *desigp, double *qmaxp, int *nfail, int *iter, int *ndiv,
                      dv_sq_t *q)
{
  const double cbias = 1.50, qurtr = 0.250, half = 0.5, hundrd = 100.0;
  const double eps = MR3_EPS, tol = eps * hundrd, tol2 = tol * tol;
  int n0 = *n0p, pp = *ppp, ipn4, j4, nn;
  const int n0in = n0;
  double dmin = *dminp, sigma = *sigmap, desig = *desigp, qmax = *qmaxp, s, t, temp;
  for (;;) {   /* label 10: deflation */
    if (n0 < i0) goto out;
    if (n0 == i0) goto l20;
    nn = 4 * n0 + pp;
    if (n0 == i0 + 1) goto l40;
    if (Zq(nn - 5) > tol2 * (sigma + Zq(nn - 3)) && Zq(nn - 2 * pp - 4) > tol2 * Zq(nn - 7))
      goto l30;
  l20:
    Zq(4 * n0 - 3) = Zq(4 * n0 + pp - 3) + sigma;
    n0 = n0 - 1;
    continue;
  l30:
    if (Zq(nn - 9) > tol2 * sigma && Zq(nn - 2 * pp - 8) > tol2 * Zq(nn - 11)) break;
  l40:
    if (Zq(nn - 3) > Zq(nn - 7)) {
      s = Zq(nn - 3);
      Zq(nn - 3) = Zq(nn - 7);
      Zq(nn - 7) = s;
    }
    if (Zq(nn - 5) > Zq(nn - 3) * tol2) {
      t = half * ((Zq(nn - 7) - Zq(nn - 3)) + Zq(nn - 5));
      s = Zq(nn - 3) * (Zq(nn - 5) / t);
      if (s <= t) s = Zq(nn - 3) * (Zq(nn - 5) / (t * (1.0 + sqrt(1.0 + s / t))));
      else s = Zq(nn - 3) * (Zq(nn - 5) / (t + sqrt(t) * sqrt(t + s)));
      t = Zq(nn - 7) + (s + Zq(nn - 5));
      Zq(nn - 3) = Zq(nn - 3) * (Zq(nn - 7) / t);
      Zq(nn - 7) = t;
    }
    Zq(4 * n0 - 7) = Zq(nn - 7) + sigma;
    Zq(4 * n0 - 3) = Zq(nn - 3) + sigma;
    n0 = n0 - 2;
  }
  /* label 50 */
  if (pp == 2) pp = 0;
  if (dmin <= 0.0 || n0 < n0in) {
    if (cbias * Zq(4 * i0 + pp - 3) < Zq(4 * n0 + pp - 3)) {
      ipn4 = 4 * (i0 + n0);
      for (j4 = 4 * i0; j4 <= 2 * (i0 + n0 - 1); j4 += 4) {
        temp = Zq(j4 - 3); Zq(j4 - 3) = Zq(ipn4 - j4 - 3); Zq(ipn4 - j4 - 3) = temp;
        temp = Zq(j4 - 2); Zq(j4 - 2) = Zq(ipn4 - j4 - 2); Zq(ipn4 - j4 - 2) = temp;
        temp = Zq(j4 - 1); Zq(j4 - 1) = Zq(ipn4 - j4 - 5); Zq(ipn4 - j4 - 5) = temp;
        temp = Zq(j4); Zq(j4) = Zq(ipn4 - j4 - 4); Zq(ipn4 - j4 - 4) = temp;
      }
      if (n0 - i0 <= 4) {
        Zq(4 * n0 + pp - 1) = Zq(4 * i0 + pp - 1);
        Zq(4 * n0 - pp) = Zq(4 * i0 - pp);
      }
      q->dmin2 = dv_fmin2(q->dmin2, Zq(4 * n0 + pp - 1));
      Zq(4 * n0 + pp - 1) =
          dv_fmin2(dv_fmin2(Zq(4 * n0 + pp - 1), Zq(4 * i0 + pp - 1)), Zq(4 * i0 + pp + 3));
      Zq(4 * n0 - pp) = dv_fmin2(dv_fmin2(Zq(4 * n0 - pp), Zq(4 * i0 - pp)), Zq(4 * i0 - pp + 4));
      qmax = dv_fmax2(dv_fmax2(qmax, Zq(4 * i0 + pp - 3)), Zq(4 * i0 + pp + 1));
      dmin = -0.0;
    }
  }
  dv_dlasq4(i0, n0, z, pp, n0in, dmin, q);
  for (;;) {   /* label 70 */
    dv_dlasq5(i0, n0, z, pp, q->tau, &dmin, &q->dmin1, &q->dmin2, &q->dn, &q->dn1, &q->dn2);
    *ndiv = *ndiv + (n0 - i0 + 2);
    *iter = *iter + 1;
    if (dmin >= 0.0 && q->dmin1 > 0.0) {
      goto l90;
    } else if (dmin < 0.0 && q->dmin1 > 0.0 && Zq(4 * (n0 - 1) - pp) < tol * (sigma + q->dn1) &&
               fabs(q->dn) < tol * sigma) {
      Zq(4 * (n0 - 1) - pp + 2) = 0.0;
      dmin = 0.0;
      goto l90;
    } else if (dmin < 0.0) {
      *nfail = *nfail + 1;
      if (q->ttype < -22) {
        q->tau = 0.0;
      } else if (q->dmin1 > 0.0) {
        q->tau = (q->tau + dmin) * (1.0 - 2.0 * eps);
        q->ttype = q->ttype - 11;
      } else {
        q->tau = qurtr * q->tau;
        q->ttype = q->ttype - 12;
      }
      continue;
    } else if (dmin != dmin) {
      if (q->tau == 0.0) break;
      q->tau = 0.0;
      continue;
    } else {
      break;
    }
  }
  /* label 80 */
  dv_dlasq6(i0, n0, z, pp, &dmin, &q->dmin1, &q->dmin2, &q->dn, &q->dn1, &q->dn2);
  *ndiv = *ndiv + (n0 - i0 + 2);
  *iter = *iter + 1;
  q->tau = 0.0;
l90:
  if (q->tau < sigma) {
    desig = desig + q->tau;
    t = sigma + desig;
    desig = desig - (t - sigma);
  } else {
    t = sigma + q->tau;
    desig = sigma - (t - q->tau) + desig;
  }
  sigma = t;
out:
  *n0p = n0;
  *ppp = pp;
  *dminp = dmin;
  *sigmap = sigma;
  *desigp = desig;
  *qmaxp = qmax;
}

/* Sort of x[0..n-1] in decreasing order (dlasrt('D'), SRC/LAPACK/odsrt.f;
 * the order of equal values is immaterial): a heap sort, O(n log n) on
 * one thread. */
static __device__ void dv_sort_desc(double *x, int n)
{
  // min-heap of the values, repeatedly moving the smallest to the end
  for (int k = n / 2 - 1; k >= 0; k--)
    for (int r = k;;) {
      int c = 2 * r + 1;
      if (c >= n) break;
      if (c + 1 < n && x[c + 1] < x[c]) c++;
      if (x[r] <= x[c]) break;
      const double t = x[r]; x[r] = x[c]; x[c] = t;
      r = c;
    }
  for (int end = n - 1; end > 0; end--) {
    const double t = x[0]; x[0] = x[end]; x[end] = t;
    for (int r = 0;;) {
      int c = 2 * r + 1;
      if (c >= end) break;
      if (c + 1 < end && x[c + 1] < x[c]) c++;
      if (x[r] <= x[c]) break;
      const double u = x[r]; x[r] = x[c]; x[c] = u;
      r = c;
    }
  }
}

/* odsq2.f: the eigenvalues of the qd array z (z[2k-2] = q_k, z[2k-1] = e_k,
 * 4n doubles of room) in z[0..n-1], decreasing; info as LAPACK's. */
static __device__ __noinline__ void dv_dlasq2(int n, double *z, int *info)
{
  const double cbias = 1.50, half = 0.5, four = 4.0, hundrd = 100.0;
  const double eps = MR3_EPS, safmin = MR3_SAFMIN, tol = eps * hundrd, tol2 = tol * tol;
  int i0, i4, ipn4, iter, iwhila, iwhilb, k, kmin, n0, n1, i1, nbig, ndiv, nfail, pp, splt;
  double d, dee, deemin, desig, dmin, e, emax, emin, oldemn, qmax, qmin, s, sigma, t, temp,
      trace, zmax, tempe, tempq;
  dv_sq_t q;
  *info = 0;
  if (n < 0) { *info = -1; return; }
  if (n == 0) return;
  if (n == 1) {
    if (Zq(1) < 0.0) *info = -201;
    return;
  }
  if (n == 2) {
    if (Zq(2) < 0.0 || Zq(3) < 0.0) { *info = -2; return; }
    if (Zq(3) > Zq(1)) { d = Zq(3); Zq(3) = Zq(1); Zq(1) = d; }
    Zq(5) = Zq(1) + Zq(2) + Zq(3);
    if (Zq(2) > Zq(3) * tol2) {
      t = half * ((Zq(1) - Zq(3)) + Zq(2));
      s = Zq(3) * (Zq(2) / t);
      if (s <= t) s = Zq(3) * (Zq(2) / (t * (1.0 + sqrt(1.0 + s / t))));
      else s = Zq(3) * (Zq(2) / (t + sqrt(t) * sqrt(t + s)));
      t = Zq(1) + (s + Zq(2));
      Zq(3) = Zq(3) * (Zq(1) / t);
      Zq(1) = t;
    }
    Zq(2) = Zq(3);
    Zq(6) = Zq(2) + Zq(1);
    return;
  }
  Zq(2 * n) = 0.0;
  emin = Zq(2);
  qmax = 0.0;
  zmax = 0.0;
  d = 0.0;
  e = 0.0;
  for (k = 1; k <= 2 * (n - 1); k += 2) {
    if (Zq(k) < 0.0) { *info = -(200 + k); return; }
    if (Zq(k + 1) < 0.0) { *info = -(200 + k + 1); return; }
    d = d + Zq(k);
    e = e + Zq(k + 1);
    qmax = dv_fmax2(qmax, Zq(k));
    emin = dv_fmin2(emin, Zq(k + 1));
    zmax = dv_fmax2(dv_fmax2(qmax, zmax), Zq(k + 1));
  }
  if (Zq(2 * n - 1) < 0.0) { *info = -(200 + 2 * n - 1); return; }
  d = d + Zq(2 * n - 1);
  qmax = dv_fmax2(qmax, Zq(2 * n - 1));
  zmax = dv_fmax2(qmax, zmax);
  if (e == 0.0) {
    for (k = 2; k <= n; k++) Zq(k) = Zq(2 * k - 1);
    dv_sort_desc(z, n);
    Zq(2 * n - 1) = d;
    return;
  }
  trace = d + e;
  if (trace == 0.0) { Zq(2 * n - 1) = 0.0; return; }
  for (k = 2 * n; k >= 2; k -= 2) {
    Zq(2 * k) = 0.0;
    Zq(2 * k - 1) = Zq(k);
    Zq(2 * k - 2) = 0.0;
    Zq(2 * k - 3) = Zq(k - 1);
  }
  i0 = 1;
  n0 = n;
  if (cbias * Zq(4 * i0 - 3) < Zq(4 * n0 - 3)) {
    ipn4 = 4 * (i0 + n0);
    for (i4 = 4 * i0; i4 <= 2 * (i0 + n0 - 1); i4 += 4) {
      temp = Zq(i4 - 3); Zq(i4 - 3) = Zq(ipn4 - i4 - 3); Zq(ipn4 - i4 - 3) = temp;
      temp = Zq(i4 - 1); Zq(i4 - 1) = Zq(ipn4 - i4 - 5); Zq(ipn4 - i4 - 5) = temp;
    }
  }
  pp = 0;
  for (k = 1; k <= 2; k++) {
    d = Zq(4 * n0 + pp - 3);
    for (i4 = 4 * (n0 - 1) + pp; i4 >= 4 * i0 + pp; i4 -= 4) {
      if (Zq(i4 - 1) <= tol2 * d) {
        Zq(i4 - 1) = -0.0;
        d = Zq(i4 - 3);
      } else {
        d = Zq(i4 - 3) * (d / (d + Zq(i4 - 1)));
      }
    }
    emin = Zq(4 * i0 + pp + 1);
    d = Zq(4 * i0 + pp - 3);
    for (i4 = 4 * i0 + pp; i4 <= 4 * (n0 - 1) + pp; i4 += 4) {
      Zq(i4 - 2 * pp - 2) = d + Zq(i4 - 1);
      if (Zq(i4 - 1) <= tol2 * d) {
        Zq(i4 - 1) = -0.0;
        Zq(i4 - 2 * pp - 2) = d;
        Zq(i4 - 2 * pp) = 0.0;
        d = Zq(i4 + 1);
      } else if (safmin * Zq(i4 + 1) < Zq(i4 - 2 * pp - 2) &&
                 safmin * Zq(i4 - 2 * pp - 2) < Zq(i4 + 1)) {
        temp = Zq(i4 + 1) / Zq(i4 - 2 * pp - 2);
        Zq(i4 - 2 * pp) = Zq(i4 - 1) * temp;
        d = d * temp;
      } else {
        Zq(i4 - 2 * pp) = Zq(i4 + 1) * (Zq(i4 - 1) / Zq(i4 - 2 * pp - 2));
        d = Zq(i4 + 1) * (d / Zq(i4 - 2 * pp - 2));
      }
      emin = dv_fmin2(emin, Zq(i4 - 2 * pp));
    }
    Zq(4 * n0 - pp - 2) = d;
    qmax = Zq(4 * i0 - pp - 2);
    for (i4 = 4 * i0 - pp + 2; i4 <= 4 * n0 - pp - 2; i4 += 4) qmax = dv_fmax2(qmax, Zq(i4));
    pp = 1 - pp;
  }
  q.ttype = 0;
  q.dmin1 = 0.0; q.dmin2 = 0.0; q.dn = 0.0; q.dn1 = 0.0; q.dn2 = 0.0; q.g = 0.0; q.tau = 0.0;
  iter = 2;
  nfail = 0;
  ndiv = 2 * (n0 - i0);
  for (iwhila = 1; iwhila <= n + 1; iwhila++) {
    if (n0 < 1) goto l170;
    desig = 0.0;
    if (n0 == n) sigma = 0.0;
    else sigma = -Zq(4 * n0 - 1);
    if (sigma < 0.0) { *info = 1; return; }
    emax = 0.0;
    if (n0 > i0) emin = fabs(Zq(4 * n0 - 5));
    else emin = 0.0;
    qmin = Zq(4 * n0 - 3);
    qmax = qmin;
    for (i4 = 4 * n0; i4 >= 8; i4 -= 4) {
      if (Zq(i4 - 5) <= 0.0) goto l100;
      if (qmin >= four * emax) {
        qmin = dv_fmin2(qmin, Zq(i4 - 3));
        emax = dv_fmax2(emax, Zq(i4 - 5));
      }
      qmax = dv_fmax2(qmax, Zq(i4 - 7) + Zq(i4 - 5));
      emin = dv_fmin2(emin, Zq(i4 - 5));
    }
    i4 = 4;
  l100:
    i0 = i4 / 4;
    pp = 0;
    if (n0 - i0 > 1) {
      dee = Zq(4 * i0 - 3);
      deemin = dee;
      kmin = i0;
      for (i4 = 4 * i0 + 1; i4 <= 4 * n0 - 3; i4 += 4) {
        dee = Zq(i4) * (dee / (dee + Zq(i4 - 2)));
        if (dee <= deemin) {
          deemin = dee;
          kmin = (i4 + 3) / 4;
        }
      }
      if ((kmin - i0) * 2 < n0 - kmin && deemin <= half * Zq(4 * n0 - 3)) {
        ipn4 = 4 * (i0 + n0);
        pp = 2;
        for (i4 = 4 * i0; i4 <= 2 * (i0 + n0 - 1); i4 += 4) {
          temp = Zq(i4 - 3); Zq(i4 - 3) = Zq(ipn4 - i4 - 3); Zq(ipn4 - i4 - 3) = temp;
          temp = Zq(i4 - 2); Zq(i4 - 2) = Zq(ipn4 - i4 - 2); Zq(ipn4 - i4 - 2) = temp;
          temp = Zq(i4 - 1); Zq(i4 - 1) = Zq(ipn4 - i4 - 5); Zq(ipn4 - i4 - 5) = temp;
          temp = Zq(i4); Zq(i4) = Zq(ipn4 - i4 - 4); Zq(ipn4 - i4 - 4) = temp;
        }
      }
    }
    dmin = -dv_fmax2(0.0, qmin - 2.0 * sqrt(qmin) * sqrt(emax));
    nbig = 100 * (n0 - i0 + 1);
    for (iwhilb = 1; iwhilb <= nbig; iwhilb++) {
      if (i0 > n0) goto l150;
      dv_dlasq3(i0, &n0, z, &pp, &dmin, &sigma, &desig, &qmax, &nfail, &iter, &ndiv, &q);
      pp = 1 - pp;
      if (pp == 0 && n0 - i0 >= 3) {
        if (Zq(4 * n0) <= tol2 * qmax || Zq(4 * n0 - 1) <= tol2 * sigma) {
          splt = i0 - 1;
          qmax = Zq(4 * i0 - 3);
          emin = Zq(4 * i0 - 1);
          oldemn = Zq(4 * i0);
          for (i4 = 4 * i0; i4 <= 4 * (n0 - 3); i4 += 4) {
            if (Zq(i4) <= tol2 * Zq(i4 - 3) || Zq(i4 - 1) <= tol2 * sigma) {
              Zq(i4 - 1) = -sigma;
              splt = i4 / 4;
              qmax = 0.0;
              emin = Zq(i4 + 3);
              oldemn = Zq(i4 + 4);
            } else {
              qmax = dv_fmax2(qmax, Zq(i4 + 1));
              emin = dv_fmin2(emin, Zq(i4 - 1));
              oldemn = dv_fmin2(oldemn, Zq(i4));
            }
          }
          Zq(4 * n0 - 1) = emin;
          Zq(4 * n0) = oldemn;
          i0 = splt + 1;
        }
      }
    }
    /* maximum number of iterations exceeded: restore the shift and return
     * the unconverged block in z (info 2) */
    *info = 2;
    i1 = i0;
    n1 = n0;
  l145:
    tempq = Zq(4 * i0 - 3);
    Zq(4 * i0 - 3) = Zq(4 * i0 - 3) + sigma;
    for (k = i0 + 1; k <= n0; k++) {
      tempe = Zq(4 * k - 5);
      Zq(4 * k - 5) = Zq(4 * k - 5) * (tempq / Zq(4 * k - 7));
      tempq = Zq(4 * k - 3);
      Zq(4 * k - 3) = Zq(4 * k - 3) + sigma + tempe - Zq(4 * k - 5);
    }
    if (i1 > 1) {
      n1 = i1 - 1;
      while (i1 >= 2 && Zq(4 * i1 - 5) >= 0.0) i1 = i1 - 1;
      sigma = -Zq(4 * n1 - 1);
      goto l145;
    }
    for (k = 1; k <= n; k++) {
      Zq(2 * k - 1) = Zq(4 * k - 3);
      if (k < n0) Zq(2 * k) = Zq(4 * k - 1);
      else Zq(2 * k) = 0;
    }
    return;
  l150:;
  }
  *info = 3;
  return;
l170:
  for (k = 2; k <= n; k++) Zq(k) = Zq(4 * k - 3);
  dv_sort_desc(z, n);
  e = 0.0;
  for (k = n; k >= 1; k--) e = e + Zq(k);
  Zq(2 * n + 1) = trace;
  Zq(2 * n + 2) = e;
  Zq(2 * n + 3) = (double)iter;
  Zq(2 * n + 4) = (double)ndiv / (double)((long long)n * n);
  Zq(2 * n + 5) = hundrd * nfail / (double)iter;
  (void)zmax; (void)n1; (void)oldemn; (void)emin;
}
#undef Zq

// dlarrk (SRC/LAPACK/odrrk.f:120-161): the iw-th eigenvalue of T by
// bisection on [gl, gu]; T packed as tp[k] = (d[k], e2[k-1]).
static __device__ __noinline__ void dv_dlarrk(int n, int iw, double gl, double gu,
                                              const double2 *__restrict__ tp, double pivmin,
                                              double reltol, double *w, double *werr) {
  const double eps = MR3_EPS, fudge = 2.0;
  const double tnorm = fmax(fabs(gl), fabs(gu)), atoli = fudge * 2.0 * pivmin;
  const int itmax = (int)((dv_log(tnorm + pivmin) - dv_log(pivmin)) / dv_log(2.0)) + 2;
  double left = gl - fudge * tnorm * eps * n - fudge * 2.0 * pivmin;
  double right = gu + fudge * tnorm * eps * n + fudge * 2.0 * pivmin;
  int it = 0;
  for (;;) {
    double tmp1 = fabs(right - left);
    const double tmp2 = fmax(fabs(right), fabs(left));
    if (tmp1 < fmax(fmax(atoli, pivmin), reltol * tmp2)) break;
    if (it > itmax) break;
    it++;
    const double mid = 0.5 * (left + right);
    int negcnt = 0;
    tmp1 = tp[0].x - mid;
    if (fabs(tmp1) < pivmin) tmp1 = -pivmin;
    if (tmp1 <= 0.0) negcnt++;
    for (int k = 1; k < n; k++) {
      tmp1 = tp[k].x - tp[k].y / tmp1 - mid;
      if (fabs(tmp1) < pivmin) tmp1 = -pivmin;
      if (tmp1 <= 0.0) negcnt++;
    }
    if (negcnt >= iw) right = mid;
    else left = mid;
  }
  *w = 0.5 * (left + right);
  *werr = 0.5 * fabs(right - left);
}

// x_k = 2*(s*a^k mod 2^48)/2^48 - 1: the k-th (1-based) number of dlarnv(2)
// from the 48-bit seed s (SRC/LAPACK/odrnv.f, odruv.f).
static __device__ __forceinline__ double dv_lcg_uniform(uint64_t seed, uint64_t k) {
  const uint64_t mask = (1ULL << 48) - 1ULL;
  uint64_t acc = 1, base = MR3_LCG_A;
  while (k) {
    if (k & 1ULL) acc = (acc * base) & mask;
    base = (base * base) & mask;
    k >>= 1;
  }
  uint64_t s = (seed * acc) & mask;
  return 2.0 * ((double)s * 3.5527136788005009e-15) - 1.0;   // 2^-48
}

// Prefetch the L1 line holding *p (PTX prefetch.global.L1).  Only issued for
// addresses inside the arrays being read.
static __device__ __forceinline__ void pf_l1(const void *p) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

#ifndef MR3_PF
#define MR3_PF 16   // L1 prefetch distance in rows (0: none)
#endif

// dlar1v (SRC/LAPACK/odr1v.f:158-362) with B1 = 1, BN = n.  Each lane of a
// warp runs its own eigenvector; the three sweeps (stationary transform,
// progressive transform, back-substitution) run over the rows in lock-step
// so every per-lane scratch access is one coalesced 256-byte row.
// Scratch per lane: X[i*R1V_LD], Y[i*R1V_LD], i < n (lane-interleaved rows).
//   stationary  : X[i] = LPLUS(i), Y[i] = S(i)
//   progressive : Y[i] = UMINUS(i) once S(i) has been used; the twist search
//                 runs inside this sweep from the top index down with a strict
//                 '<', which selects the same index as the Fortran's upward
//                 scan with '<='
//   solve       : z(k) for k < r in X[k], z(r) = 1, z(k) for k > r in Y[k-1]
// r_in = 0 means "search the twist index over 1..n".
//
// The sweeps are latency chains (one division per row) whose inputs come
// from memory that is mostly not in L1: the rows are read in chunks of MR3_U
// rows, and the loads of the next chunk are issued before the current chunk
// is computed, so a load's latency overlaps MR3_U rows of arithmetic.  The
// arithmetic of every row is exactly that of the row-by-row recurrence.
#define R1V_LD 32

struct dlar1v_out {
  int negcnt, r, isupp1, isupp2;
  double ztz, mingma, nrminv, resid, rqcorr;
  bool sawnan;
};

static __device__ __forceinline__ double dv_zget(const double *X, const double *Y, int r, int k) {
  return k < r ? X[(size_t)k * R1V_LD] : (k == r ? 1.0 : Y[(size_t)(k - 1) * R1V_LD]);
}

static __device__ __noinline__ bool dv_r1v_passA(int n, double lambda, const double2 *__restrict__ P,
                                          const double2 *__restrict__ Q, int ps, double pivmin, int r1,
                                          int r2, double *__restrict__ X, double *__restrict__ Y,
                                          int *neg1o) {
  constexpr int U = MR3_U;
  int neg1 = 0;
  double s = 0.0 - lambda;
  Y[0] = 0.0;
  bool sawnan = false;
  const int last = r2 - 1;   // rows 1..last
  if (last >= 1) {
    double cd[U], cl[U], cld[U], nd[U], nl[U], nld[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int i = d_imin(1 + u, last);
      cd[u] = P[(size_t)(i - 1) * ps].x;
      const double2 q = Q[(size_t)(i - 1) * ps];
      cl[u] = q.x; cld[u] = q.y;
    }
    for (int i0 = 1; i0 <= last; i0 += U) {
#pragma unroll
      for (int u = 0; u < U; u++) {   // next chunk (clamped to the last row)
        const int i = d_imin(i0 + U + u, last);
        nd[u] = P[(size_t)(i - 1) * ps].x;
        const double2 q = Q[(size_t)(i - 1) * ps];
        nl[u] = q.x; nld[u] = q.y;
        if (MR3_PF && i0 + u + MR3_PF <= last) {
          pf_l1(&P[(size_t)(i0 + u + MR3_PF - 1) * ps]);
          pf_l1(&Q[(size_t)(i0 + u + MR3_PF - 1) * ps]);
        }
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int i = i0 + u;
        if (i <= last) {
          double dplus = cd[u] + s;
          double lp = cld[u] / dplus;
          X[(size_t)i * R1V_LD] = lp;
          if (i <= r1 - 1) neg1 += (dplus < 0.0);
          double si = s * lp * cl[u];
          Y[(size_t)i * R1V_LD] = si;
          s = si - lambda;
          // rows past R1-1 computed after a NaN are redone by the slow sweep
          if (i == r1 - 1 && isnan(s)) sawnan = true;
        }
      }
      if (sawnan) break;
#pragma unroll
      for (int u = 0; u < U; u++) { cd[u] = nd[u]; cl[u] = nl[u]; cld[u] = nld[u]; }
    }
  }
  if (!sawnan) sawnan = isnan(s);
  if (sawnan) {
    neg1 = 0;
    s = 0.0 - lambda;
    for (int i = 1; i <= r2 - 1; i++) {
      const double2 pp = P[(size_t)(i - 1) * ps];
      const double2 q = Q[(size_t)(i - 1) * ps];
      double dplus = pp.x + s;
      if (fabs(dplus) < pivmin) dplus = -pivmin;
      double lp = q.y / dplus;
      X[(size_t)i * R1V_LD] = lp;
      if (i <= r1 - 1) neg1 += (dplus < 0.0);
      double si = s * lp * q.x;
      if (lp == 0.0) si = pp.y;
      Y[(size_t)i * R1V_LD] = si;
      s = si - lambda;
    }
  }
  *neg1o = neg1;
  return sawnan;
}

// Progressive transform with the fused twist search, for the whole warp:
// the lanes sweep the rows by absolute index from the largest N-1 of the
// active lanes down to the smallest R1, each lane working on its own rows
// (R1..N-1), so the per-lane scratch rows stay aligned across lanes when
// the lanes' matrices differ in size.  Returns P(R1-1) of this lane.
static __device__ __noinline__ double dv_r1v_passB(bool active, int n, double lambda,
                                            const double2 *__restrict__ P,
                                            const double2 *__restrict__ Q, int ps, double pivmin, int r1,
                                            int r2, bool slow, double *__restrict__ Y, int *neg2o,
                                            int *rbest, double *best, bool *have) {
  constexpr int U = MR3_U;
  const double eps = MR3_EPS;
  int neg2 = 0;
  double p = 0.0;
  *have = false;
  const int top = n - 1;   // this lane's rows top..r1, descending
  if (active) {
    p = P[(size_t)(n - 1) * ps].x - lambda;   // P(n-1)
    if (r2 == n && n > r1) {          // candidate r = n
      double s = Y[(size_t)(n - 1) * R1V_LD];
      double c = s + p;
      if (c == 0.0) c = eps * s;
      *best = c; *rbest = n; *have = true;
    }
  }
  const bool work = active && top >= r1;
  const int topw = __reduce_max_sync(0xffffffffu, work ? top : 0);
  const int r1w = __reduce_min_sync(0xffffffffu, work ? r1 : 0x7fffffff);
  if (topw >= 1) {
    double cpx[U], cpy[U], cqx[U], csp[U], npx[U], npy[U], nqx[U], nsp[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      if (work) {
        const int i = d_imax(d_imin(topw - u, top), r1);
        const double2 pp = P[(size_t)(i - 1) * ps];
        cpx[u] = pp.x; cpy[u] = pp.y;
        cqx[u] = Q[(size_t)(i - 1) * ps].x;
        csp[u] = Y[(size_t)(i - 1) * R1V_LD];
      }
    }
    for (int i0 = topw; i0 >= r1w; i0 -= U) {
      // next chunk: rows i0-U .. i0-2U+1, none of which this chunk writes
#pragma unroll
      for (int u = 0; u < U; u++) {
        if (work) {
          const int i = d_imax(d_imin(i0 - U - u, top), r1);
          const double2 pp = P[(size_t)(i - 1) * ps];
          npx[u] = pp.x; npy[u] = pp.y;
          nqx[u] = Q[(size_t)(i - 1) * ps].x;
          nsp[u] = Y[(size_t)(i - 1) * R1V_LD];
          const int f = i0 - u - MR3_PF;
          if (MR3_PF && f >= r1 && f <= top) {
            pf_l1(&P[(size_t)(f - 1) * ps]);
            pf_l1(&Q[(size_t)(f - 1) * ps]);
            pf_l1(&Y[(size_t)(f - 1) * R1V_LD]);
          }
        }
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int i = i0 - u;
        if (work && i >= r1 && i <= top) {
          double dminus = cpy[u] + p;
          if (slow && fabs(dminus) < pivmin) dminus = -pivmin;
          double tmp = cpx[u] / dminus;
          neg2 += (dminus < 0.0);
          double um = cqx[u] * tmp;
          double pn = p * tmp - lambda;
          if (slow && tmp == 0.0) pn = cpx[u] - lambda;
          Y[(size_t)i * R1V_LD] = um;
          p = pn;
          if (i > r1 && i <= r2) {        // candidate r = i: S(i-1) + P(i-1)
            const double sprev = csp[u];
            double c = sprev + p;
            if (c == 0.0) c = eps * sprev;
            if (!*have || fabs(c) < fabs(*best)) { *best = c; *rbest = i; *have = true; }
          }
        }
      }
#pragma unroll
      for (int u = 0; u < U; u++) { cpx[u] = npx[u]; cpy[u] = npy[u]; cqx[u] = nqx[u]; csp[u] = nsp[u]; }
    }
  }
  *neg2o = neg2;
  return p;
}

// The two factorisation sweeps and the twist choice of dlar1v, for the
// whole warp (every lane calls it; `active` lanes have a factorisation to
// do).  Leaves the lane's state for dv_r1v_solve.
struct r1v_state {
  int r;
  double mingma;
  bool sawnan;
};

static __device__ __noinline__ void dv_r1v_factor(bool active, int n, double lambda,
                                           const double2 *__restrict__ P,
                                           const double2 *__restrict__ Q, int ps, double pivmin,
                                           bool wantnc, int r_in, double *X, double *Y,
                                           int *negcnt, r1v_state *st) {
  const double eps = MR3_EPS;
  int r1 = 1, r2 = n, neg1 = 0, neg2 = 0, rbest = 0;
  if (r_in != 0) { r1 = r_in; r2 = r_in; }
  bool sawnan1 = false;
  if (active) sawnan1 = dv_r1v_passA(n, lambda, P, Q, ps, pivmin, r1, r2, X, Y, &neg1);
  double best = 0.0;
  bool have = false;
  double pr1 = dv_r1v_passB(active, n, lambda, P, Q, ps, pivmin, r1, r2, false, Y, &neg2, &rbest,
                            &best, &have);
  bool sawnan2 = active && isnan(pr1);
  if (__any_sync(0xffffffffu, sawnan2)) {
    // S was overwritten by UMINUS; recompute the stationary sweep (same bits)
    // and run the slow progressive sweep
    if (sawnan2) dv_r1v_passA(n, lambda, P, Q, ps, pivmin, r1, r2, X, Y, &neg1);
    int n2b = 0, rbb = 0;
    double bb = 0.0;
    bool hb = false;
    double pb = dv_r1v_passB(sawnan2, n, lambda, P, Q, ps, pivmin, r1, r2, true, Y, &n2b, &rbb,
                             &bb, &hb);
    if (sawnan2) { pr1 = pb; neg2 = n2b; rbest = rbb; best = bb; have = hb; }
  }
  if (!active) return;
  double sr1 = Y[(size_t)(r1 - 1) * R1V_LD];
  double mg = sr1 + pr1;
  if (mg < 0.0) neg1++;
  *negcnt = wantnc ? neg1 + neg2 : -1;
  if (fabs(mg) == 0.0) mg = eps * sr1;
  int r = r1;
  if (have && fabs(best) <= fabs(mg)) { mg = best; r = rbest; }
  st->mingma = mg;
  st->r = r;
  st->sawnan = sawnan1 || sawnan2;
}

// Back-substitution N^T z = e_r of dlar1v (odr1v.f:285-355) for a whole warp
// in lock-step: rows are visited from the largest twist index down (upward
// solve) and then from the smallest up to the largest N-1 (downward solve);
// a lane works on its own rows.  `active` says whether this lane has a
// solve to do.  Writes z over X/Y as described above and returns the
// outputs.  Rows are read in chunks as in the factorisation sweeps; a row's
// LPLUS/UMINUS is read before the row is overwritten with z.
static __device__ __noinline__ void dv_r1v_solve(bool active, int n, const double2 *__restrict__ Q, int ps,
                                          double gaptol, double *X, double *Y,
                                          const r1v_state &st, dlar1v_out *o) {
  constexpr int U = MR3_U;
  const int r = active ? st.r : 0;
  const int rmax = __reduce_max_sync(0xffffffffu, active ? r : 0);
  int rmin = __reduce_min_sync(0xffffffffu, active ? r : 0x7fffffff);
  const int nw = __reduce_max_sync(0xffffffffu, active ? n : 0);
  int is1 = 1, is2 = n;
  double ztz = 1.0;
  const bool slow = active && st.sawnan;
  // upward solve: i = r-1 .. 1
  bool go = active;
  double zp = 1.0;
  if (rmax - 1 >= 1) {
    double cx[U], cq[U], nx[U], nq[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      if (active) {
        const int i = d_imax(d_imin(rmax - 1 - u, n - 1), 1);
        cx[u] = X[(size_t)i * R1V_LD];
        cq[u] = Q[(size_t)(i - 1) * ps].y;
      }
    }
    for (int i0 = rmax - 1; i0 >= 1; i0 -= U) {
      if (!__any_sync(0xffffffffu, go)) break;
#pragma unroll
      for (int u = 0; u < U; u++) {
        if (active) {
          const int i = d_imax(d_imin(i0 - U - u, n - 1), 1);
          nx[u] = X[(size_t)i * R1V_LD];
          nq[u] = Q[(size_t)(i - 1) * ps].y;
          const int f = i0 - u - MR3_PF;
          if (MR3_PF && f >= 1 && f < r) pf_l1(&X[(size_t)f * R1V_LD]);
        }
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int i = i0 - u;
        if (i >= 1 && go && i < r) {
          double zi;
          if (!slow) {
            zi = -(cx[u] * zp);
          } else {
            double zi1 = dv_zget(X, Y, r, i + 1);
            if (zi1 == 0.0) zi = -(Q[(size_t)i * ps].y / cq[u]) * dv_zget(X, Y, r, i + 2);
            else zi = -(cx[u] * zi1);
            zp = zi1;
          }
          if ((fabs(zi) + fabs(zp)) * fabs(cq[u]) < gaptol) {
            X[(size_t)i * R1V_LD] = 0.0;
            is1 = i + 1;
            go = false;
          } else {
            ztz = ztz + zi * zi;
            X[(size_t)i * R1V_LD] = zi;
            zp = zi;
          }
        }
      }
#pragma unroll
      for (int u = 0; u < U; u++) { cx[u] = nx[u]; cq[u] = nq[u]; }
    }
  }
  // downward solve: i = r .. n-1
  go = active;
  double zc = 1.0;
  if (rmin == 0x7fffffff) rmin = nw;
  if (rmin <= nw - 1) {
    double cy[U], cq[U], ny[U], nq[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      if (active) {
        const int i = d_imax(d_imin(rmin + u, n - 1), 1);
        cy[u] = Y[(size_t)i * R1V_LD];
        cq[u] = Q[(size_t)(i - 1) * ps].y;
      }
    }
    for (int i0 = rmin; i0 <= nw - 1; i0 += U) {
      if (!__any_sync(0xffffffffu, go)) break;
#pragma unroll
      for (int u = 0; u < U; u++) {
        if (active) {
          const int i = d_imax(d_imin(i0 + U + u, n - 1), 1);
          ny[u] = Y[(size_t)i * R1V_LD];
          nq[u] = Q[(size_t)(i - 1) * ps].y;
          const int f = i0 + u + MR3_PF;
          if (MR3_PF && f >= r && f <= n - 1) pf_l1(&Y[(size_t)f * R1V_LD]);
        }
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int i = i0 + u;
        if (i <= n - 1 && go && i >= r) {
          double zn;
          if (!slow) {
            zn = -(cy[u] * zc);
          } else {
            double zci = dv_zget(X, Y, r, i);
            if (zci == 0.0) zn = -(Q[(size_t)(i - 2) * ps].y / cq[u]) * dv_zget(X, Y, r, i - 1);
            else zn = -(cy[u] * zci);
            zc = zci;
          }
          if ((fabs(zc) + fabs(zn)) * fabs(cq[u]) < gaptol) {
            Y[(size_t)i * R1V_LD] = 0.0;
            is2 = i;
            go = false;
          } else {
            ztz = ztz + zn * zn;
            Y[(size_t)i * R1V_LD] = zn;
            zc = zn;
          }
        }
      }
#pragma unroll
      for (int u = 0; u < U; u++) { cy[u] = ny[u]; cq[u] = nq[u]; }
    }
  }
  if (active) {
    o->r = r;
    o->mingma = st.mingma;
    o->isupp1 = is1;
    o->isupp2 = is2;
    o->ztz = ztz;
    double tmp = 1.0 / ztz;
    o->nrminv = sqrt(tmp);
    o->resid = fabs(o->mingma) * o->nrminv;
    o->rqcorr = o->mingma * tmp;
    o->sawnan = st.sawnan;
  }
}

// ------------------------------------------------------------------------
// dlar1v with checkpoints (the singleton rounds).  The three sweeps of
// dlar1v above keep LPLUS, S and UMINUS of every row in per-lane scratch,
// written by one sweep and read back in the opposite order by the next: for
// a batch that is several bytes of scratch traffic per row and lane, all of
// it through DRAM.  Here a sweep keeps only its state at the start of every
// block of CK_K rows (block j = rows j*CK_K+1 .. (j+1)*CK_K); a consumer
// that needs a block's values recomputes them from the checkpoint with the
// same operations, in registers, and uses them in its own order.  The
// recomputed values are the stored values, bit for bit; the recurrences are
// run about twice, and the scratch traffic falls to three doubles per block.
// The back-substitution writes the normalised eigenvector straight to its
// column of Z when asked to (a second call after the vector is accepted).
// ------------------------------------------------------------------------
#ifndef CK_K
#define CK_K 2   // 4 keeps a quarter of the checkpoints but spills in the search sweep
#endif
// 1: the progressive sweep double-buffers the next block's rows in
// registers; 0: it loads a block's rows when it reaches it, prefetched into
// L1 two blocks ahead (fewer registers)
#ifndef MR3_PROGR_DB
#define MR3_PROGR_DB 1
#endif
// checkpoint blocks prefetched ahead (into L1) by the progressive sweep and
// the back-substitution: the checkpoints of a round's warps are far larger
// than L2, so each block's checkpoint comes from DRAM (0: none)
#ifndef MR3_CKPF
#define MR3_CKPF 0
#endif

// One lane's checkpoints; element j of each array at [j * 32].
struct r1c_ck {
  double *S;   // s entering block j (s = -lambda for j = 0)
  double *I;   // stationary value SI of row j*CK_K (0 for j = 0)
  double *P;   // p entering the highest row of block j that the progressive
               // sweep processed
};

struct r1c_state {
  int r;
  double mingma;
  bool sawnan, slowA, slowB;   // NaN seen; stationary / progressive sweep
                               // used the NaN-safe formulas
};

// Stationary sweep (rows 1..r2-1) of one lane with checkpoints, rows read
// in register chunks of MR3_U (next chunk loaded before the current one is
// computed).  SLOW selects the NaN-safe formulas.  Returns whether a NaN
// calls for the NaN-safe rerun; sr1 = SI of row r1-1 (0 for r1 = 1),
// silast = SI of row r2-1.
template <bool SLOW>
static __device__ __noinline__ bool dv_r1c_statio(double lambda, const double2 *__restrict__ P,
                                           const double2 *__restrict__ Q, int ps, double pivmin,
                                           int r1, int r2, double *__restrict__ ckS,
                                           double *__restrict__ ckI, int *neg1o, double *sr1o,
                                           double *silasto) {
  constexpr int U = (MR3_U < CK_K) ? MR3_U : CK_K;
  static_assert(CK_K % U == 0, "chunks must not straddle checkpoint blocks");
  const int last = r2 - 1;
  int neg1 = 0;
  double s = 0.0 - lambda, siv = 0.0, sr1 = 0.0;
  bool sawnan = false;
  if (last >= 1) {
    double2 cp[U], cq[U], np_[U], nq[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int i = d_imin(1 + u, last);
      cp[u] = P[(size_t)(i - 1) * ps];
      cq[u] = Q[(size_t)(i - 1) * ps];
    }
    for (int i0 = 1; i0 <= last; i0 += U) {
      if (((i0 - 1) & (CK_K - 1)) == 0) {
        const int j = (i0 - 1) / CK_K;
        ckS[(size_t)j * 32] = s;
        ckI[(size_t)j * 32] = siv;
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int i = d_imin(i0 + U + u, last);
        np_[u] = P[(size_t)(i - 1) * ps];
        nq[u] = Q[(size_t)(i - 1) * ps];
        if (MR3_PF && i0 + u + MR3_PF <= last) {
          pf_l1(&P[(size_t)(i0 + u + MR3_PF - 1) * ps]);
          pf_l1(&Q[(size_t)(i0 + u + MR3_PF - 1) * ps]);
        }
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int i = i0 + u;
        if (i <= last) {
          double dplus = cp[u].x + s;
          if (SLOW && fabs(dplus) < pivmin) dplus = -pivmin;
          const double lp = cq[u].y / dplus;
          if (i <= r1 - 1) neg1 += (dplus < 0.0);
          double si = s * lp * cq[u].x;
          if (SLOW && lp == 0.0) si = cp[u].y;
          s = si - lambda;
          siv = si;
          if (i == r1 - 1) {
            sr1 = si;
            if (!SLOW && isnan(s)) sawnan = true;
          }
        }
      }
      if (sawnan) break;
#pragma unroll
      for (int u = 0; u < U; u++) { cp[u] = np_[u]; cq[u] = nq[u]; }
    }
  }
  if (!SLOW && !sawnan) sawnan = isnan(s);
  *neg1o = neg1;
  *sr1o = sr1;
  *silasto = siv;
  return !SLOW && sawnan;
}

// Progressive sweep (rows n-1..r1) with the twist search of r1..r2, for the
// whole warp: the lanes sweep the blocks by absolute index from the largest
// N-1 down to the smallest R1, each lane on its own rows, so the per-lane
// checkpoint rows stay aligned.  The twist search needs the stationary SI of
// row i-1 at row i: in search mode a block's SI values are recomputed from
// its stationary checkpoint first.  Returns P(R1-1).
template <bool SLOW, bool SEARCH>
static __device__ __noinline__ double dv_r1c_progr(bool active, int n, double lambda,
                                            const double2 *__restrict__ P,
                                            const double2 *__restrict__ Q, int ps, double pivmin,
                                            int r1, int r2, bool slowA, const double *__restrict__ ckS,
                                            const double *__restrict__ ckI, double *__restrict__ ckP,
                                            double silast, int *neg2o, int *rbest_o, double *best_o,
                                            bool *have_o) {
  const double eps = MR3_EPS;
  int neg2 = 0, rbest = 0;
  double p = 0.0, best = 0.0;
  bool have = false;
  const int top = n - 1;
  if (active) {
    p = P[(size_t)(n - 1) * ps].x - lambda;   // P(n-1)
    if (r2 == n && n > r1) {                  // candidate r = n
      double c = silast + p;
      if (c == 0.0) c = eps * silast;
      best = c; rbest = n; have = true;
    }
  }
  const bool work = active && top >= r1;
  // SEARCH = false: no lane of the warp searches the twist index (the rows'
  // Q halves and the stationary recompute are not needed)
  const bool search = SEARCH && r2 > r1;
  const int topw = __reduce_max_sync(0xffffffffu, work ? top : 0);
  const int r1w = __reduce_min_sync(0xffffffffu, work ? r1 : 0x7fffffff);
  if (topw >= 1) {
    const int jtop = (topw - 1) / CK_K, jbot = (r1w - 1) / CK_K;
    // a block's rows (P; Q for the search's stationary recompute) are
    // loaded one block ahead of its arithmetic
    double2 cp[CK_K], cq[CK_K], np_[CK_K], nq[CK_K];
    // the search's stationary checkpoints, also one block ahead
    double ckSv = 0.0, ckIv = 0.0, nckS = 0.0, nckI = 0.0;
    if (work && search) { ckSv = ckS[(size_t)jtop * 32]; ckIv = ckI[(size_t)jtop * 32]; }
    auto load = [&](int jb, double2 *bp, double2 *bq) {
      const int base = jb * CK_K + 1;
      const int hi = d_imin(base + CK_K - 1, top), lo = d_imax(base, r1);
      if (work && lo <= hi) {
#pragma unroll
        for (int u = 0; u < CK_K; u++) {
          const int i = d_imax(d_imin(base + u, hi), lo);
          bp[u] = P[(size_t)(i - 1) * ps];
          if (SEARCH && search) bq[u] = Q[(size_t)(i - 1) * ps];
        }
      }
    };
#if MR3_PROGR_DB
    load(jtop, cp, cq);
#endif
    for (int jb = jtop; jb >= jbot; jb--) {
#if MR3_CKPF > 0
      // only blocks inside this lane's own rows [r1, top]
      if (work && (jb - MR3_CKPF) * CK_K + 1 >= r1 && (jb - MR3_CKPF + 1) * CK_K <= top) {
        const int jf = jb - MR3_CKPF, bf = jf * CK_K + 1;
        pf_l1(&P[(size_t)(bf - 1) * ps]);
        pf_l1(&P[(size_t)(bf + CK_K - 2) * ps]);
        if (SEARCH && search) {
          pf_l1(&Q[(size_t)(bf - 1) * ps]);
          pf_l1(&Q[(size_t)(bf + CK_K - 2) * ps]);
          pf_l1(&ckS[(size_t)jf * 32]);
          pf_l1(&ckI[(size_t)jf * 32]);
        }
      }
#endif
#if MR3_PROGR_DB
      if (jb - 1 >= jbot) {
        load(jb - 1, np_, nq);
        if (work && search) { nckS = ckS[(size_t)(jb - 1) * 32]; nckI = ckI[(size_t)(jb - 1) * 32]; }
      }
#else
      // rows loaded at the block (L1 hits: prefetched two blocks ahead)
      load(jb, cp, cq);
      if (work && search) { ckSv = ckS[(size_t)jb * 32]; ckIv = ckI[(size_t)jb * 32]; }
      if (work && jb - 2 >= jbot) {
        const int b2 = (jb - 2) * CK_K + 1;
#pragma unroll
        for (int u = 0; u < CK_K; u += 2) {
          pf_l1(&P[(size_t)(b2 + u - 1) * ps]);
          if (SEARCH && search) pf_l1(&Q[(size_t)(b2 + u - 1) * ps]);
        }
      }
#endif
      const int base = jb * CK_K + 1;
      const int hi = d_imin(base + CK_K - 1, top), lo = d_imax(base, r1);
      const bool bw = work && lo <= hi;
      double sia[CK_K];
      if (SEARCH && bw && search) {
        // SI of rows base-1 .. base+CK_K-2 (those of twist candidates only);
        // in search mode r1 = 1, so the block's rows were loaded unclamped
        sia[0] = ckIv;
        double s = ckSv;
        const int rmax = d_imin(hi - 1, r2 - 1);
#pragma unroll
        for (int u = 1; u < CK_K; u++) {
          const int i = base + u - 1;
          if (i <= rmax) {
            double dplus = cp[u - 1].x + s;
            if (slowA && fabs(dplus) < pivmin) dplus = -pivmin;
            const double lp = cq[u - 1].y / dplus;
            double si = s * lp * cq[u - 1].x;
            if (slowA && lp == 0.0) si = cp[u - 1].y;
            s = si - lambda;
            sia[u] = si;
          }
        }
      }
      if (bw) ckP[(size_t)jb * 32] = p;
#pragma unroll
      for (int u = CK_K - 1; u >= 0; u--) {
        const int i = base + u;
        if (bw && i >= lo && i <= hi) {
          double dminus = cp[u].y + p;
          if (SLOW && fabs(dminus) < pivmin) dminus = -pivmin;
          const double tmp = cp[u].x / dminus;
          neg2 += (dminus < 0.0);
          double pn = p * tmp - lambda;
          if (SLOW && tmp == 0.0) pn = cp[u].x - lambda;
          p = pn;
          if (SEARCH && i > r1 && i <= r2) {   // candidate r = i: S(i-1) + P(i-1)
            const double sprev = sia[u];
            double c = sprev + p;
            if (c == 0.0) c = eps * sprev;
            if (!have || fabs(c) < fabs(best)) { best = c; rbest = i; have = true; }
          }
        }
      }
#if MR3_PROGR_DB
      #pragma unroll
      for (int u = 0; u < CK_K; u++) {
        cp[u] = np_[u];
        if (SEARCH) cq[u] = nq[u];
      }
      ckSv = nckS;
      ckIv = nckI;
#endif
    }
  }
  *neg2o = neg2;
  *rbest_o = rbest;
  *best_o = best;
  *have_o = have;
  return p;
}

// The two factorisation sweeps and the twist choice of dlar1v (as
// dv_r1v_factor), for the whole warp.
static __device__ __noinline__ void dv_r1c_factor(bool active, int n, double lambda,
                                           const double2 *__restrict__ P,
                                           const double2 *__restrict__ Q, int ps, double pivmin,
                                           bool wantnc, int r_in, r1c_ck ck, int *negcnt,
                                           r1c_state *st) {
  const double eps = MR3_EPS;
  int r1 = 1, r2 = n, neg1 = 0, neg2 = 0, rbest = 0;
  if (r_in != 0) { r1 = r_in; r2 = r_in; }
  bool sawnan1 = false;
  double sr1 = 0.0, silast = 0.0;
  if (active) {
    sawnan1 = dv_r1c_statio<false>(lambda, P, Q, ps, pivmin, r1, r2, ck.S, ck.I, &neg1, &sr1, &silast);
    // odr1v.f:199-205: rerun with the NaN-safe formulas
    if (sawnan1) dv_r1c_statio<true>(lambda, P, Q, ps, pivmin, r1, r2, ck.S, ck.I, &neg1, &sr1, &silast);
  }
  double best = 0.0;
  bool have = false;
  // the search form only when a lane of the warp searches its twist index
  const bool anysearch = __any_sync(0xffffffffu, active && r2 > r1);
  double pr1 = anysearch
      ? dv_r1c_progr<false, true>(active, n, lambda, P, Q, ps, pivmin, r1, r2, sawnan1, ck.S,
                                  ck.I, ck.P, silast, &neg2, &rbest, &best, &have)
      : dv_r1c_progr<false, false>(active, n, lambda, P, Q, ps, pivmin, r1, r2, sawnan1, ck.S,
                                   ck.I, ck.P, silast, &neg2, &rbest, &best, &have);
  bool sawnan2 = active && isnan(pr1);
  if (__any_sync(0xffffffffu, sawnan2)) {
    // odr1v.f:234-250: the progressive sweep again with the NaN-safe
    // formulas (the stationary checkpoints are unchanged)
    int n2b = 0, rbb = 0;
    double bb = 0.0;
    bool hb = false;
    double pb = dv_r1c_progr<true, true>(sawnan2, n, lambda, P, Q, ps, pivmin, r1, r2, sawnan1,
                                         ck.S, ck.I, ck.P, silast, &n2b, &rbb, &bb, &hb);
    if (sawnan2) { pr1 = pb; neg2 = n2b; rbest = rbb; best = bb; have = hb; }
  }
  if (!active) return;
  double mg = sr1 + pr1;
  if (mg < 0.0) neg1++;
  *negcnt = wantnc ? neg1 + neg2 : -1;
  if (fabs(mg) == 0.0) mg = eps * sr1;
  int r = r1;
  if (have && fabs(best) <= fabs(mg)) { mg = best; r = rbest; }
  st->mingma = mg;
  st->r = r;
  st->sawnan = sawnan1 || sawnan2;
  st->slowA = sawnan1;
  st->slowB = sawnan2;
}

// Back-substitution of dlar1v (as dv_r1v_solve) for one lane, on its own
// rows only (no lock-step: a localised eigenvector costs its support, not
// the span of its warp's twist indices), with the factors recomputed block
// by block from the checkpoints: upward from the twist, LPLUS of a block
// from its stationary checkpoint; downward, UMINUS from its progressive
// checkpoint.  With zout (the lane's column of Z at the block's first row)
// the normalised z (times nv) of the rows in the support is written there;
// rows outside the support are not touched.
static __device__ __noinline__ void dv_r1c_solve(int n, double lambda, const double2 *__restrict__ P,
                                          const double2 *__restrict__ Q, int ps, double pivmin,
                                          double gaptol, int r, bool slow, bool slowA, bool slowB,
                                          const double *__restrict__ ckS,
                                          const double *__restrict__ ckP, double mingma,
                                          double *zout, double nv, dlar1v_out *o) {
  int is1 = 1, is2 = n;
  double ztz = 1.0;
  if (zout) zout[r - 1] = 1.0 * nv;
  // upward solve: i = r-1 .. 1
  {
    double zp = 1.0, zpp = 0.0;   // z(i+1), z(i+2)
    bool go = r - 1 >= 1;
    // each block's checkpoint is loaded one block ahead
    double s_next = go ? ckS[(size_t)((r - 2) / CK_K) * 32] : 0.0;
    for (int jb = (r - 2) / CK_K; go && jb >= 0; jb--) {
      const int base = jb * CK_K + 1;
      const int hi = d_imin(base + CK_K - 1, r - 1);
      double lpa[CK_K], lda[CK_K];
      double s = s_next;
      if (jb > 0) s_next = ckS[(size_t)(jb - 1) * 32];
#if MR3_CKPF > 0
      if (jb - MR3_CKPF >= 0) pf_l1(&ckS[(size_t)(jb - MR3_CKPF) * 32]);
#endif
#pragma unroll
      for (int u = 0; u < CK_K; u++) {
        const int i = base + u;
        if (i <= hi) {
          const double2 pp = P[(size_t)(i - 1) * ps];
          const double2 q = Q[(size_t)(i - 1) * ps];
          double dplus = pp.x + s;
          if (slowA && fabs(dplus) < pivmin) dplus = -pivmin;
          const double lp = q.y / dplus;
          double si = s * lp * q.x;
          if (slowA && lp == 0.0) si = pp.y;
          s = si - lambda;
          lpa[u] = lp;
          lda[u] = q.y;
        }
      }
      if (base > 1)
        for (int i = d_imax(base - CK_K, 1); i <= base - 1; i++) {
          pf_l1(&P[(size_t)(i - 1) * ps]);
          pf_l1(&Q[(size_t)(i - 1) * ps]);
        }
#pragma unroll
      for (int u = CK_K - 1; u >= 0; u--) {
        const int i = base + u;
        if (go && i <= hi) {
          const double ldi = lda[u];
          double zi;
          if (!slow) zi = -(lpa[u] * zp);
          else if (zp == 0.0) zi = -(Q[(size_t)i * ps].y / ldi) * zpp;
          else zi = -(lpa[u] * zp);
          if ((fabs(zi) + fabs(zp)) * fabs(ldi) < gaptol) {
            is1 = i + 1;
            go = false;
          } else {
            ztz = ztz + zi * zi;
            if (zout) zout[i - 1] = zi * nv;
            zpp = zp;
            zp = zi;
          }
        }
      }
    }
  }
  // downward solve: i = r .. n-1, z(i+1) from z(i)
  {
    double zc = 1.0, zcp = 0.0;   // z(i), z(i-1)
    bool go = r <= n - 1;
    const int jlast = (n - 2) / CK_K;
    double p_next = go ? ckP[(size_t)((r - 1) / CK_K) * 32] : 0.0;
    for (int jb = (r - 1) / CK_K; go && jb <= jlast; jb++) {
      const int base = jb * CK_K + 1;
      const int lo = d_imax(base, r), hi = d_imin(base + CK_K - 1, n - 1);
      double uma[CK_K], lda[CK_K];
      double p = p_next;
      if (jb < jlast) p_next = ckP[(size_t)(jb + 1) * 32];
#if MR3_CKPF > 0
      if (jb + MR3_CKPF <= jlast) pf_l1(&ckP[(size_t)(jb + MR3_CKPF) * 32]);
#endif
#pragma unroll
      for (int u = CK_K - 1; u >= 0; u--) {
        const int i = base + u;
        if (i >= lo && i <= hi) {
          const double2 pp = P[(size_t)(i - 1) * ps];
          const double2 q = Q[(size_t)(i - 1) * ps];
          double dminus = pp.y + p;
          if (slowB && fabs(dminus) < pivmin) dminus = -pivmin;
          const double tmp = pp.x / dminus;
          uma[u] = q.x * tmp;
          lda[u] = q.y;
          double pn = p * tmp - lambda;
          if (slowB && tmp == 0.0) pn = pp.x - lambda;
          p = pn;
        }
      }
      if (base + CK_K <= n - 1)
        for (int i = base + CK_K; i <= d_imin(base + 2 * CK_K - 1, n - 1); i++) {
          pf_l1(&P[(size_t)(i - 1) * ps]);
          pf_l1(&Q[(size_t)(i - 1) * ps]);
        }
#pragma unroll
      for (int u = 0; u < CK_K; u++) {
        const int i = base + u;
        if (go && i >= lo && i <= hi) {
          const double ldi = lda[u];
          double zn;
          if (!slow) zn = -(uma[u] * zc);
          else if (zc == 0.0) zn = -(Q[(size_t)(i - 2) * ps].y / ldi) * zcp;
          else zn = -(uma[u] * zc);
          if ((fabs(zc) + fabs(zn)) * fabs(ldi) < gaptol) {
            is2 = i;
            go = false;
          } else {
            ztz = ztz + zn * zn;
            if (zout) zout[i] = zn * nv;
            zcp = zc;
            zc = zn;
          }
        }
      }
    }
  }
  o->r = r;
  o->mingma = mingma;
  o->isupp1 = is1;
  o->isupp2 = is2;
  o->ztz = ztz;
  const double tmp = 1.0 / ztz;
  o->nrminv = sqrt(tmp);
  o->resid = fabs(mingma) * o->nrminv;
  o->rqcorr = mingma * tmp;
  o->sawnan = slow;
}

// Back-substitution of dlar1v (as dv_r1c_solve) for the whole warp in
// lock-step: the lanes visit the same absolute rows at the same time (the
// upward solve from the largest twist index down, the downward one from the
// smallest up), each lane working only inside its own range, so that a
// checkpoint access is one 256-byte row across the lanes and lanes that
// share a representation read its rows once.  With `write`, the lanes' z
// values go to a shared-memory tile of 32 rows x 32 lanes (tile[row * 33 +
// lane], 8448 bytes per warp); a tile is written out when the sweep leaves
// it, one column at a time by the whole warp (lane k writes row k of the
// tile's segment of that column): coalesced 256-byte segments instead of
// one 8-byte store per lane and row.  A block of CK_K rows never straddles
// two tiles (upward tiles cover rows 32t+1 .. 32t+32, downward ones, whose
// block j writes z of rows 4j+2 .. 4j+5, rows 32t+2 .. 32t+33).  zout is the
// lane's column of Z at the block's first row; z is written unscaled.  Every
// value and every test is the one of dv_r1c_solve, in the same order per
// lane.
#define R1W_T 32
static __device__ __noinline__ void dv_r1w_solve(bool active, int n, double lambda,
                                          const double2 *__restrict__ P,
                                          const double2 *__restrict__ Q, int ps, double pivmin,
                                          double gaptol, int r, bool slow, bool slowA, bool slowB,
                                          const double *__restrict__ ckS,
                                          const double *__restrict__ ckP, double mingma,
                                          double *zout, bool write, double *tile,
                                          dlar1v_out *o) {
  static_assert(R1W_T == 32 && R1W_T % CK_K == 0, "tiles hold whole blocks");
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  int is1 = 1, is2 = n;
  double ztz = 1.0;
  const bool wr = active && write;
  if (wr) zout[r - 1] = 1.0;
  const bool anyw = __any_sync(full, wr);
  // rows [tlo, thi] (1-based) of the current tile hold this lane's values
  int tbase = 0, tlo = 1, thi = 0;
  auto flush = [&]() {   // warp-uniform call sites only
    __syncwarp();
    unsigned m = __ballot_sync(full, wr && tlo <= thi);
    while (m) {
      const int c = __ffs(m) - 1;
      m &= m - 1;
      const int lo = __shfl_sync(full, tlo, c), hi = __shfl_sync(full, thi, c);
      double *zc = (double *)__shfl_sync(full, (unsigned long long)zout, c);
      const int row = tbase + lane;
      if (row >= lo && row <= hi) zc[row - 1] = tile[lane * 33 + c];
    }
    __syncwarp();
    tlo = 1;
    thi = 0;
  };
  auto put = [&](int row, double z) {
    tile[(row - tbase) * 33 + lane] = z;
    if (tlo > thi) { tlo = row; thi = row; }
    else { tlo = d_imin(tlo, row); thi = d_imax(thi, row); }
  };
  // upward solve: i = r-1 .. 1, blocks from the warp's largest r down
  {
    double zp = 1.0, zpp = 0.0;   // z(i+1), z(i+2)
    bool go = active && r - 1 >= 1;
    const int jtop = __reduce_max_sync(full, go ? (r - 2) / CK_K : -1);
    int cur_tile = -1;
    for (int jb = jtop; jb >= 0; jb--) {
      if (!__any_sync(full, go)) break;
      const int base = jb * CK_K + 1;
      if (anyw && jb * CK_K / R1W_T != cur_tile) {
        if (cur_tile >= 0) flush();
        cur_tile = jb * CK_K / R1W_T;
        tbase = cur_tile * R1W_T + 1;
      }
      const int hi = d_imin(base + CK_K - 1, r - 1);
      if (go && jb <= (r - 2) / CK_K) {
        double lpa[CK_K], lda[CK_K];
        double s = ckS[(size_t)jb * 32];
#pragma unroll
        for (int u = 0; u < CK_K; u++) {
          const int i = base + u;
          if (i <= hi) {
            const double2 pp = P[(size_t)(i - 1) * ps];
            const double2 q = Q[(size_t)(i - 1) * ps];
            double dplus = pp.x + s;
            if (slowA && fabs(dplus) < pivmin) dplus = -pivmin;
            const double lp = q.y / dplus;
            double si = s * lp * q.x;
            if (slowA && lp == 0.0) si = pp.y;
            s = si - lambda;
            lpa[u] = lp;
            lda[u] = q.y;
          }
        }
#pragma unroll
        for (int u = CK_K - 1; u >= 0; u--) {
          const int i = base + u;
          if (go && i <= hi) {
            const double ldi = lda[u];
            double zi;
            if (!slow) zi = -(lpa[u] * zp);
            else if (zp == 0.0) zi = -(Q[(size_t)i * ps].y / ldi) * zpp;
            else zi = -(lpa[u] * zp);
            if ((fabs(zi) + fabs(zp)) * fabs(ldi) < gaptol) {
              is1 = i + 1;
              go = false;
            } else {
              ztz = ztz + zi * zi;
              if (wr) put(i, zi);
              zpp = zp;
              zp = zi;
            }
          }
        }
      }
    }
    if (anyw && cur_tile >= 0) flush();
  }
  // downward solve: i = r .. n-1 (z of row i+1 from z of row i), blocks from
  // the warp's smallest r up
  {
    double zc = 1.0, zcp = 0.0;   // z(i), z(i-1)
    bool go = active && r <= n - 1;
    const int jbot = __reduce_min_sync(full, go ? (r - 1) / CK_K : 0x7fffffff);
    const int jend = __reduce_max_sync(full, go ? (n - 2) / CK_K : -1);
    int cur_tile = -1;
    for (int jb = jbot; jb <= jend; jb++) {
      if (!__any_sync(full, go)) break;
      const int base = jb * CK_K + 1;
      if (anyw && jb * CK_K / R1W_T != cur_tile) {
        if (cur_tile >= 0) flush();
        cur_tile = jb * CK_K / R1W_T;
        tbase = cur_tile * R1W_T + 2;
      }
      const int lo = d_imax(base, r), hi = d_imin(base + CK_K - 1, n - 1);
      if (go && jb >= (r - 1) / CK_K && lo <= hi) {
        double uma[CK_K], lda[CK_K];
        double p = ckP[(size_t)jb * 32];
#pragma unroll
        for (int u = CK_K - 1; u >= 0; u--) {
          const int i = base + u;
          if (i >= lo && i <= hi) {
            const double2 pp = P[(size_t)(i - 1) * ps];
            const double2 q = Q[(size_t)(i - 1) * ps];
            double dminus = pp.y + p;
            if (slowB && fabs(dminus) < pivmin) dminus = -pivmin;
            const double tmp = pp.x / dminus;
            uma[u] = q.x * tmp;
            lda[u] = q.y;
            double pn = p * tmp - lambda;
            if (slowB && tmp == 0.0) pn = pp.x - lambda;
            p = pn;
          }
        }
#pragma unroll
        for (int u = 0; u < CK_K; u++) {
          const int i = base + u;
          if (go && i >= lo && i <= hi) {
            const double ldi = lda[u];
            double zn;
            if (!slow) zn = -(uma[u] * zc);
            else if (zc == 0.0) zn = -(Q[(size_t)(i - 2) * ps].y / ldi) * zcp;
            else zn = -(uma[u] * zc);
            if ((fabs(zc) + fabs(zn)) * fabs(ldi) < gaptol) {
              is2 = i;
              go = false;
            } else {
              ztz = ztz + zn * zn;
              if (wr) put(i + 1, zn);
              zcp = zc;
              zc = zn;
            }
          }
        }
      }
    }
    if (anyw && cur_tile >= 0) flush();
  }
  o->r = r;
  o->mingma = mingma;
  o->isupp1 = is1;
  o->isupp2 = is2;
  o->ztz = ztz;
  const double tmp = 1.0 / ztz;
  o->nrminv = sqrt(tmp);
  o->resid = fabs(mingma) * o->nrminv;
  o->rqcorr = mingma * tmp;
  o->sawnan = slow;
}

// ------------------------------------------------------------------------
// dlar1v for one eigenvector on a whole warp (the short lists at the end of
// a level, where latency rather than throughput counts).  The stationary
// sweep (lane 0) and the progressive sweep (lane 1) are independent chains
// and run at the same time, each keeping every row's values in the warp's
// scratch (SI and LPLUS of the stationary rows, P and UMINUS of the
// progressive ones); the twist index is then chosen by all 32 lanes (the
// smallest |gamma(i)|, the largest i among equal ones: what odr1v.f's upward
// scan with .LE. selects); the back-substitution runs upward on lane 0 and
// downward on lane 1, and lane 0 adds the downward squares to ztz after its
// own, in odr1v.f's order.  Every value is computed by the operations of
// odr1v.f:158-362 in their order, so the results are those of
// dv_r1c_factor + dv_r1c_solve bit for bit.
// Scratch per warp (nmax doubles each): SI, LP, PA, UM, ZV, rows 1-based at
// [row]: SI[i], LP[i] of stationary row i; PA[i] the progressive value after
// row i (PA[n] = D(n) - lambda); UM[i] of row i; ZV[i] the vector.
// ------------------------------------------------------------------------
struct r1s_buf {
  double *SI, *LP, *PA, *UM, *ZV;
};

// Rows the split form's sweeping lanes prefetch ahead of their arithmetic
// (0: none).  A lane sweeps alone, so nothing else hides the latency of its
// loads; the child representations live in DRAM.
#ifndef MR3_R1S_PF
#define MR3_R1S_PF 32
#endif
static __device__ __forceinline__ void pf_l2(const void *p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

static __device__ __noinline__ void dv_r1s_call(int n, double lambda, const double2 *__restrict__ P,
                                         const double2 *__restrict__ Q, int ps, double pivmin,
                                         bool wantnc, int r_in, double gaptol, r1s_buf b,
                                         int *negcnt_o, dlar1v_out *o) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const double eps = MR3_EPS;
  int r1 = 1, r2 = n;
  if (r_in != 0) { r1 = r_in; r2 = r_in; }
  // ---- the two sweeps, rerun with the NaN-safe formulas where needed
  int neg1 = 0, neg2 = 0;
  bool slowA = false, slowB = false;
  double sr1 = 0.0;   // SI of row r1-1 (0 for r1 = 1)
  if (lane == 0) {
    for (int pass = 0; pass < 2; pass++) {
      const bool SLOW = pass == 1;
      double s = 0.0 - lambda;
      bool sawnan = false;
      neg1 = 0;
      sr1 = 0.0;
#pragma unroll 4
      for (int i = 1; i <= r2 - 1; i++) {
        if (MR3_R1S_PF && i + MR3_R1S_PF <= r2 - 1) {
          pf_l2(&P[(size_t)(i + MR3_R1S_PF - 1) * ps]);
          pf_l2(&Q[(size_t)(i + MR3_R1S_PF - 1) * ps]);
        }
        const double2 pp = P[(size_t)(i - 1) * ps], q = Q[(size_t)(i - 1) * ps];
        double dplus = pp.x + s;
        if (SLOW && fabs(dplus) < pivmin) dplus = -pivmin;
        const double lp = q.y / dplus;
        if (i <= r1 - 1) neg1 += (dplus < 0.0);
        double si = s * lp * q.x;
        if (SLOW && lp == 0.0) si = pp.y;
        s = si - lambda;
        b.LP[i] = lp;
        b.SI[i] = si;
        if (i == r1 - 1) {
          sr1 = si;
          if (!SLOW && isnan(s)) sawnan = true;
        }
        if (sawnan) break;
      }
      if (!SLOW && !sawnan) sawnan = isnan(s);
      if (SLOW || !sawnan) break;
      slowA = true;
    }
  } else if (lane == 1) {
    for (int pass = 0; pass < 2; pass++) {
      const bool SLOW = pass == 1;
      double p = P[(size_t)(n - 1) * ps].x - lambda;
      b.PA[n] = p;
      neg2 = 0;
#pragma unroll 4
      for (int i = n - 1; i >= r1; i--) {
        if (MR3_R1S_PF && i - MR3_R1S_PF >= r1) {
          pf_l2(&P[(size_t)(i - MR3_R1S_PF - 1) * ps]);
          pf_l2(&Q[(size_t)(i - MR3_R1S_PF - 1) * ps]);
        }
        const double2 pp = P[(size_t)(i - 1) * ps];
        double dminus = pp.y + p;
        if (SLOW && fabs(dminus) < pivmin) dminus = -pivmin;
        const double tmp = pp.x / dminus;
        neg2 += (dminus < 0.0);
        b.UM[i] = Q[(size_t)(i - 1) * ps].x * tmp;
        double pn = p * tmp - lambda;
        if (SLOW && tmp == 0.0) pn = pp.x - lambda;
        p = pn;
        b.PA[i] = p;
      }
      if (SLOW || !isnan(p)) break;
      slowB = true;
    }
  }
  neg1 = __shfl_sync(full, neg1, 0);
  sr1 = __shfl_sync(full, sr1, 0);
  slowA = __shfl_sync(full, slowA, 0);
  neg2 = __shfl_sync(full, neg2, 1);
  slowB = __shfl_sync(full, slowB, 1);
  __syncwarp();
  // ---- the twist index: gamma(i) = SI(i-1) + P(i-1) for i in (r1, r2]
  double best = 0.0;
  int rbest = 0;
  for (int i = r1 + 1 + lane; i <= r2; i += 32) {
    const double sprev = b.SI[i - 1];
    double c = sprev + b.PA[i];
    if (c == 0.0) c = eps * sprev;
    if (isnan(c)) continue;
    if (rbest == 0 || fabs(c) <= fabs(best)) { best = c; rbest = i; }   // i increases
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double ob = __shfl_xor_sync(full, best, o);
    const int orb = __shfl_xor_sync(full, rbest, o);
    if (orb != 0 && (rbest == 0 || fabs(ob) < fabs(best) || (fabs(ob) == fabs(best) && orb > rbest))) {
      best = ob;
      rbest = orb;
    }
  }
  const double pr1 = b.PA[r1];
  double mg = sr1 + pr1;
  if (mg < 0.0) neg1++;
  *negcnt_o = wantnc ? neg1 + neg2 : -1;
  if (fabs(mg) == 0.0) mg = eps * sr1;
  int r = r1;
  if (rbest != 0 && fabs(best) <= fabs(mg)) { mg = best; r = rbest; }
  const bool slow = slowA || slowB;
  // ---- back-substitution: upward on lane 0, downward on lane 1
  int is1 = 1, is2 = n;
  double ztz = 1.0;
  if (lane == 0) {
    b.ZV[r] = 1.0;
    double zp = 1.0, zpp = 0.0;
    for (int i = r - 1; i >= 1; i--) {
      if (MR3_R1S_PF && i - 16 >= 1) {   // the rows ahead into L1
        pf_l1(&Q[(size_t)(i - 17) * ps]);
        pf_l1(&b.LP[i - 16]);
      }
      const double ldi = Q[(size_t)(i - 1) * ps].y;
      double zi;
      if (!slow) zi = -(b.LP[i] * zp);
      else if (zp == 0.0) zi = -(Q[(size_t)i * ps].y / ldi) * zpp;
      else zi = -(b.LP[i] * zp);
      if ((fabs(zi) + fabs(zp)) * fabs(ldi) < gaptol) { is1 = i + 1; break; }
      ztz = ztz + zi * zi;
      b.ZV[i] = zi;
      zpp = zp;
      zp = zi;
    }
  } else if (lane == 1) {
    double zc = 1.0, zcp = 0.0;
    for (int i = r; i <= n - 1; i++) {
      if (MR3_R1S_PF && i + 16 <= n - 1) {
        pf_l1(&Q[(size_t)(i + 15) * ps]);
        pf_l1(&b.UM[i + 16]);
      }
      const double ldi = Q[(size_t)(i - 1) * ps].y;
      double zn;
      if (!slow) zn = -(b.UM[i] * zc);
      else if (zc == 0.0) zn = -(Q[(size_t)(i - 2) * ps].y / ldi) * zcp;
      else zn = -(b.UM[i] * zc);
      if ((fabs(zc) + fabs(zn)) * fabs(ldi) < gaptol) { is2 = i; break; }
      b.ZV[i + 1] = zn;
      zcp = zc;
      zc = zn;
    }
  }
  is2 = __shfl_sync(full, is2, 1);
  __syncwarp();
  if (lane == 0)
    for (int i = r + 1; i <= is2; i++) ztz = ztz + b.ZV[i] * b.ZV[i];
  ztz = __shfl_sync(full, ztz, 0);
  is1 = __shfl_sync(full, is1, 0);
  o->r = r;
  o->mingma = mg;
  o->isupp1 = is1;
  o->isupp2 = is2;
  o->ztz = ztz;
  const double tmp = 1.0 / ztz;
  o->nrminv = sqrt(tmp);
  o->resid = fabs(mg) * o->nrminv;
  o->rqcorr = mg * tmp;
  o->sawnan = slow;
}

// The factorisation L+ D+ L+^T = L D L^T - sigma I of dlarrf
// (SRC/LAPACK/odrrf.f:226-252) for one shift: DPLUS into dp[i*os], LPLUS
// into lp[i*os]; returns max |DPLUS|, sawnan when a pivot was replaced by
// -pivmin.  The running pivot stays in a register (it is written out, never
// read back) and the rows are read in chunks of MR3_U issued one chunk
// ahead of the arithmetic.
static __device__ __forceinline__ double rrf_sweep(int n, const double2 *__restrict__ P,
                                                   const double2 *__restrict__ Q, int ps,
                                                   double sig, double pivmin, double *dp,
                                                   double *lp, int os, bool *sawnan) {
  constexpr int U = MR3_U;
  double s = -sig;
  double d = P[0].x + s;
  if (fabs(d) < pivmin) { d = -pivmin; *sawnan = true; }
  dp[0] = d;
  double mx = fabs(d);
  const int last = n - 2;   // rows i = 0..n-2 produce LPLUS(i), DPLUS(i+1)
  if (last >= 0) {
    double2 cq[U], nq[U];
    double cp[U], np_[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int i = d_imin(u, last);
      cq[u] = Q[(size_t)i * ps];
      cp[u] = P[(size_t)(i + 1) * ps].x;
    }
    for (int i0 = 0; i0 <= last; i0 += U) {
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int i = d_imin(i0 + U + u, last);
        nq[u] = Q[(size_t)i * ps];
        np_[u] = P[(size_t)(i + 1) * ps].x;
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int i = i0 + u;
        if (i <= last) {
          const double l = cq[u].y / d;
          lp[(size_t)i * os] = l;
          s = s * l * cq[u].x - sig;
          d = cp[u] + s;
          if (fabs(d) < pivmin) { d = -pivmin; *sawnan = true; }
          dp[(size_t)(i + 1) * os] = d;
          mx = fmax(mx, fabs(d));
        }
      }
#pragma unroll
      for (int u = 0; u < U; u++) { cq[u] = nq[u]; cp[u] = np_[u]; }
    }
  }
  return mx;
}

// dlarrf, LAPACK 3.2.2 with NOFAIL (SRC/LAPACK/odrrf.f:140-378), one thread.
// Parent rows: d = P[i].x, l = Q[i].x, ld = Q[i].y.  w/wgap/werr point at the
// cluster's first eigenvalue (CLSTRT = 1, CLEND = clend).  dplus, lplus: out;
// work: 2n scratch.  Returns the shift sigma.
// PAIR: two lanes (an even lane and the next odd one) per cluster, with the
// same arguments; the even lane sweeps the left shift while the odd one
// sweeps the right shift, so that a try costs one sweep's time instead of
// two when the left shift fails.  The right sweep is run even when the left
// one is accepted; its output (the work array) is then not used, so the
// result -- the shift and the representation in dplus/lplus -- is the
// sequential one bit for bit.  Both lanes return the shift.
template <bool PAIR>
static __device__ __noinline__ double dv_dlarrf(int n, const double2 *__restrict__ P,
                                         const double2 *__restrict__ Q, int ps, int clend,
                                         const double *w, const double *wgap, const double *werr,
                                         double spdiam, double clgapl, double clgapr,
                                         double pivmin, double *dp_, double *lp_, double *wk_,
                                         int os) {
#define dplus(i) dp_[(size_t)(i) * os]
#define lplus(i) lp_[(size_t)(i) * os]
#define work(i) wk_[(size_t)(i) * os]
  const double maxgrowth1 = 8.0, maxgrowth2 = 8.0, eps = MR3_EPS, fact = 2.0;
  const int ktrymax = 1;
  int shift = 0, indx = 0, ktry = 0;
  bool forcer = false;
  double sigma = 0.0;
  double clwdth = fabs(w[clend - 1] - w[0]) + werr[clend - 1] + werr[0];
  double avgap = clwdth / (double)(clend - 1);
  double mingap = fmin(clgapl, clgapr);
  double lsigma = fmin(w[0], w[clend - 1]) - werr[0];
  double rsigma = fmax(w[0], w[clend - 1]) + werr[clend - 1];
  lsigma = lsigma - fabs(lsigma) * 4.0 * eps;
  rsigma = rsigma + fabs(rsigma) * 4.0 * eps;
  double ldmax = 0.25 * mingap + 2.0 * pivmin;
  double rdmax = 0.25 * mingap + 2.0 * pivmin;
  double ldelta = fmax(avgap, wgap[0]) / fact;
  double rdelta = fmax(avgap, wgap[clend - 2]) / fact;
  double smlgrowth = 1.0 / MR3_SAFMIN;
  double fail = (double)(n - 1) * mingap / (spdiam * eps);
  double fail2 = (double)(n - 1) * mingap / (spdiam * sqrt(eps));
  double bestshift = lsigma;
  double growthbound = maxgrowth1 * spdiam;
  double max1 = 0.0, max2 = 0.0;
  for (int guard = 0; guard < 8; guard++) {
    bool sawnan1 = false, sawnan2 = false;
    ldelta = fmin(ldmax, ldelta);
    rdelta = fmin(rdmax, rdelta);
    if (PAIR) {
      const unsigned pm = 3u << ((threadIdx.x & 31) & ~1);   // this lane pair
      const bool right = (threadIdx.x & 1) != 0;
      bool sn = false;
      const double mx = right ? rrf_sweep(n, P, Q, ps, rsigma, pivmin, wk_, wk_ + (size_t)n * os,
                                          os, &sn)
                              : rrf_sweep(n, P, Q, ps, lsigma, pivmin, dp_, lp_, os, &sn);
      const int src = (threadIdx.x & 31) & ~1;
      max1 = __shfl_sync(pm, mx, src);
      sawnan1 = __shfl_sync(pm, (int)sn, src) != 0;
      max2 = __shfl_sync(pm, mx, src + 1);
      sawnan2 = __shfl_sync(pm, (int)sn, src + 1) != 0;
      __syncwarp(pm);   // both sweeps' stores visible to both lanes
      sawnan1 = sawnan1 || isnan(max1);
      if (forcer || (max1 <= growthbound && !sawnan1)) { sigma = lsigma; shift = 1; break; }
      sawnan2 = sawnan2 || isnan(max2);
      if (forcer || (max2 <= growthbound && !sawnan2)) { sigma = rsigma; shift = 2; break; }
    } else {
      max1 = rrf_sweep(n, P, Q, ps, lsigma, pivmin, dp_, lp_, os, &sawnan1);
      sawnan1 = sawnan1 || isnan(max1);
      if (forcer || (max1 <= growthbound && !sawnan1)) { sigma = lsigma; shift = 1; break; }

      max2 = rrf_sweep(n, P, Q, ps, rsigma, pivmin, wk_, wk_ + (size_t)n * os, os, &sawnan2);
      sawnan2 = sawnan2 || isnan(max2);
      if (forcer || (max2 <= growthbound && !sawnan2)) { sigma = rsigma; shift = 2; break; }
    }

    if (!(sawnan1 && sawnan2)) {
      if (!sawnan1) {
        indx = 1;
        if (max1 <= smlgrowth) { smlgrowth = max1; bestshift = lsigma; }
      }
      if (!sawnan2) {
        if (sawnan1 || max2 <= max1) indx = 2;
        if (max2 <= smlgrowth) { smlgrowth = max2; bestshift = rsigma; }
      }
      bool dorrr1 = (clwdth < mingap / 128.0) && (fmin(max1, max2) < fail2) && !sawnan1 &&
                    !sawnan2;
      if (dorrr1) {
        if (indx == 1) {
          double tmp = fabs(dplus(n - 1)), znm2 = 1.0, prod = 1.0, oldp = 1.0;
          for (int i = n - 1; i >= 1; i--) {
            if (prod <= eps)
              prod = ((dplus(i) * work(n + i)) / (dplus(i - 1) * work(n + i - 1))) * oldp;
            else
              prod = prod * fabs(work(n + i - 1));
            oldp = prod;
            znm2 = znm2 + prod * prod;
            tmp = fmax(tmp, fabs(dplus(i - 1) * prod));
          }
          double rrr1 = tmp / (spdiam * sqrt(znm2));
          if (rrr1 <= maxgrowth2) { sigma = lsigma; shift = 1; break; }
        } else if (indx == 2) {
          double tmp = fabs(work(n - 1)), znm2 = 1.0, prod = 1.0, oldp = 1.0;
          for (int i = n - 1; i >= 1; i--) {
            if (prod <= eps)
              prod = ((work(i) * lplus(i)) / (work(i - 1) * lplus(i - 1))) * oldp;
            else
              prod = prod * fabs(lplus(i - 1));
            oldp = prod;
            znm2 = znm2 + prod * prod;
            tmp = fmax(tmp, fabs(work(i - 1) * prod));
          }
          double rrr2 = tmp / (spdiam * sqrt(znm2));
          if (rrr2 <= maxgrowth2) { sigma = rsigma; shift = 2; break; }
        }
      }
    }
    if (ktry < ktrymax) {
      lsigma = fmax(lsigma - ldelta, lsigma - ldmax);
      rsigma = fmin(rsigma + rdelta, rsigma + rdmax);
      ldelta = 2.0 * ldelta;
      rdelta = 2.0 * rdelta;
      ktry++;
      continue;
    }
    (void)fail;   // NOFAIL: the best shift is always accepted
    lsigma = bestshift;
    rsigma = bestshift;
    forcer = true;
  }
  if (shift == 2) {
    // PAIR: the even lane copies DPLUS, the odd one LPLUS
    if (!PAIR || (threadIdx.x & 1) == 0)
      for (int i = 0; i < n; i++) dplus(i) = work(i);
    if (!PAIR || (threadIdx.x & 1) != 0)
      for (int i = 0; i < n - 1; i++) lplus(i) = work(n + i);
  }
  return sigma;
#undef dplus
#undef lplus
#undef work
}

// One interval of dlarrj (SRC/LAPACK/odrrj.f:100-281): bisection on T to
// relative tolerance rtol.  Intervals are independent (no gaps involved).
// tp[j] = (d[j], e2[j-1]) of the unshifted matrix.
static __device__ __forceinline__ int dv_count_rrj(int n, const double2 *__restrict__ tp, double s) {
  double dplus = tp[0].x - s;
  int cnt = (dplus < 0.0);
  for (int j = 1; j < n; j++) {
    const double2 v = tp[j];
    dplus = v.x - s - v.y / dplus;
    cnt += (dplus < 0.0);
  }
  return cnt;
}

static __device__ __noinline__ void dv_dlarrj_one(int n, const double2 *__restrict__ tp, int i,
                                           double rtol, int maxitr, double *w, double *werr) {
  double left = *w - *werr, mid = *w, right = *w + *werr;
  double width = right - mid;
  double tmp = fmax(fabs(left), fabs(right));
  if (width < rtol * tmp) return;
  double fac = 1.0;
  for (int cap = 0; cap < MR3_EXPAND_CAP; cap++) {
    if (dv_count_rrj(n, tp, left) > i - 1) { left = left - *werr * fac; fac = 2.0 * fac; }
    else break;
  }
  fac = 1.0;
  for (int cap = 0; cap < MR3_EXPAND_CAP; cap++) {
    if (dv_count_rrj(n, tp, right) < i) { right = right + *werr * fac; fac = 2.0 * fac; }
    else break;
  }
  for (int iter = 0; iter <= maxitr; iter++) {
    mid = 0.5 * (left + right);
    width = right - mid;
    tmp = fmax(fabs(left), fabs(right));
    if (width < rtol * tmp || iter == maxitr) break;
    int cnt = dv_count_rrj(n, tp, mid);
    if (cnt <= i - 1) left = mid; else right = mid;
  }
  *w = 0.5 * (left + right);
  *werr = right - *w;
}
