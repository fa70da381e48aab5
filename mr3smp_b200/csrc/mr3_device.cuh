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

// Sturm count of T - x, IJOB=1 rule of dlaebz (SRC/LAPACK/odebz.f:255-270).
// tp[j] = (d[j], e2[j-1]); tp[0].y unused.
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

// The interval of eigenvalue j under dlaebz IJOB=2 started from [a,b] with
// counts (na,nb): midpoint bisection of that one interval (odebz.f 90-120).
static __device__ __noinline__ int dv_bisect_one(int n, const double2 *__restrict__ tp, double pivmin,
                                          double abstol, double reltol, int itmax, int j,
                                          double *a, double *b, int na, int nb, int *iters) {
  double c = 0.5 * (*a + *b);
  for (int it = 1; it <= itmax; it++) {
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

// dlaneg (SRC/LAPACK/odneg.f:98-163) on packed rows P[(i)*ps]; r is 1-based.
static __device__ __noinline__ int dv_dlaneg(int n, const double2 *__restrict__ P, int ps, double sigma,
                                      int r) {
  const int blklen = 128;
  int negcnt = 0;
  double t = -sigma;
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

// One interval of dlarrb (SRC/LAPACK/odrrb.f:136-293).  Intervals of one
// dlarrb call never read each other's state: the convergence test reads the
// gaps of the input WGAP, which dlarrb rewrites only after every interval has
// converged.  So one thread per interval yields the sequential result.
//   i      : 1-based eigenvalue index of this interval (IFIRST..ILAST)
//   first  : i == IFIRST (initial-phase left gap is then the own right gap)
//   has_left: II > 1 (main-loop left gap is WGAP(II-1))
//   w, werr: in/out; updated only if the interval went through the main loop
// Returns the number of counts spent, or -1 if a widening loop hit its cap.
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
    negcnt = dv_dlaneg(n, R, ps, left, r);
    nc++;
    if (negcnt > i - 1) { left = left - back; back = 2.0 * back; } else break;
  }
  if (cap == MR3_EXPAND_CAP) status = -1;
  back = *werr;
  for (cap = 0; cap < MR3_EXPAND_CAP; cap++) {
    negcnt = dv_dlaneg(n, R, ps, right, r);
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
    negcnt = dv_dlaneg(n, R, ps, mid, r);
    *ncount += 1;
    if (negcnt <= i - 1) left = mid; else right = mid;
  }
  *w = 0.5 * (left + right);
  *werr = right - *w;
  return status;
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

#define MR3_PF 16   // prefetch distance in rows

// dlar1v (SRC/LAPACK/odr1v.f:158-362) with B1 = 1, BN = n.  Each lane of a
// warp runs its own eigenvector; the three sweeps (stationary transform,
// progressive transform, back-substitution) run over the rows in lock-step
// so every per-lane scratch access is one coalesced 256-byte row.
// Scratch per lane: X[i*stride], Y[i*stride], i < n.
//   stationary  : X[i] = LPLUS(i), Y[i] = S(i)
//   progressive : Y[i] = UMINUS(i) once S(i) has been used; the twist search
//                 runs inside this sweep from the top index down with a strict
//                 '<', which selects the same index as the Fortran's upward
//                 scan with '<='
//   solve       : z(k) for k < r in X[k], z(r) = 1, z(k) for k > r in Y[k-1]
// r_in = 0 means "search the twist index over 1..n".
struct dlar1v_out {
  int negcnt, r, isupp1, isupp2;
  double ztz, mingma, nrminv, resid, rqcorr;
  bool sawnan;
};

static __device__ __forceinline__ double dv_zget(const double *X, const double *Y, int stride, int r,
                                          int k) {
  return k < r ? X[(size_t)k * stride] : (k == r ? 1.0 : Y[(size_t)(k - 1) * stride]);
}

static __device__ __noinline__ bool dv_r1v_passA(int n, double lambda, const double2 *__restrict__ P,
                                          const double2 *__restrict__ Q, int ps, double pivmin, int r1,
                                          int r2, double *X, double *Y, int stride, int *neg1o) {
  int neg1 = 0;
  double s = 0.0 - lambda;
  Y[0] = 0.0;
  bool sawnan = false;
  for (int i = 1; i <= r2 - 1; i++) {
    if (i + MR3_PF <= n - 1) { pf_l1(&P[(size_t)(i + MR3_PF - 1) * ps]); pf_l1(&Q[(size_t)(i + MR3_PF - 1) * ps]); }
    const double dd = P[(size_t)(i - 1) * ps].x;
    const double2 q = Q[(size_t)(i - 1) * ps];
    double dplus = dd + s;
    double lp = q.y / dplus;
    X[(size_t)i * stride] = lp;
    if (i <= r1 - 1) neg1 += (dplus < 0.0);
    double si = s * lp * q.x;
    Y[(size_t)i * stride] = si;
    s = si - lambda;
    if (i == r1 - 1 && isnan(s)) { sawnan = true; break; }
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
      X[(size_t)i * stride] = lp;
      if (i <= r1 - 1) neg1 += (dplus < 0.0);
      double si = s * lp * q.x;
      if (lp == 0.0) si = pp.y;
      Y[(size_t)i * stride] = si;
      s = si - lambda;
    }
  }
  *neg1o = neg1;
  return sawnan;
}

// Progressive transform with the fused twist search.  Returns P(R1-1).
static __device__ __noinline__ double dv_r1v_passB(int n, double lambda, const double2 *__restrict__ P,
                                            const double2 *__restrict__ Q, int ps, double pivmin, int r1,
                                            int r2, bool slow, double *Y, int stride, int *neg2o,
                                            int *rbest, double *best, bool *have) {
  const double eps = MR3_EPS;
  int neg2 = 0;
  double p = P[(size_t)(n - 1) * ps].x - lambda;   // P(n-1)
  *have = false;
  if (r2 == n && n > r1) {          // candidate r = n
    double s = Y[(size_t)(n - 1) * stride];
    double c = s + p;
    if (c == 0.0) c = eps * s;
    *best = c; *rbest = n; *have = true;
  }
  for (int i = n - 1; i >= r1; i--) {
    if (i - MR3_PF >= 1) {
      pf_l1(&P[(size_t)(i - MR3_PF - 1) * ps]);
      pf_l1(&Q[(size_t)(i - MR3_PF - 1) * ps]);
      pf_l1(&Y[(size_t)(i - MR3_PF - 1) * stride]);
    }
    const double2 pp = P[(size_t)(i - 1) * ps];
    const double2 q = Q[(size_t)(i - 1) * ps];
    const double sprev = Y[(size_t)(i - 1) * stride];
    double dminus = pp.y + p;
    if (slow && fabs(dminus) < pivmin) dminus = -pivmin;
    double tmp = pp.x / dminus;
    neg2 += (dminus < 0.0);
    double um = q.x * tmp;
    double pn = p * tmp - lambda;
    if (slow && tmp == 0.0) pn = pp.x - lambda;
    Y[(size_t)i * stride] = um;
    p = pn;
    if (i > r1 && i <= r2) {        // candidate r = i: S(i-1) + P(i-1)
      double c = sprev + p;
      if (c == 0.0) c = eps * sprev;
      if (!*have || fabs(c) < fabs(*best)) { *best = c; *rbest = i; *have = true; }
    }
  }
  *neg2o = neg2;
  return p;
}

// The two factorisation sweeps and the twist choice of dlar1v.  Leaves the
// lane's state for dv_r1v_solve.
struct r1v_state {
  int r;
  double mingma;
  bool sawnan;
};

static __device__ __noinline__ void dv_r1v_factor(int n, double lambda, const double2 *__restrict__ P,
                                           const double2 *__restrict__ Q, int ps, double pivmin,
                                           bool wantnc, int r_in, double *X, double *Y,
                                           int stride, int *negcnt, r1v_state *st) {
  const double eps = MR3_EPS;
  int r1, r2, neg1, neg2, rbest = 0;
  if (r_in == 0) { r1 = 1; r2 = n; } else { r1 = r_in; r2 = r_in; }
  bool sawnan1 = dv_r1v_passA(n, lambda, P, Q, ps, pivmin, r1, r2, X, Y, stride, &neg1);
  double best = 0.0;
  bool have;
  double pr1 = dv_r1v_passB(n, lambda, P, Q, ps, pivmin, r1, r2, false, Y, stride, &neg2, &rbest,
                            &best, &have);
  bool sawnan2 = isnan(pr1);
  if (sawnan2) {
    // S was overwritten by UMINUS; recompute the stationary sweep (same bits)
    // and run the slow progressive sweep
    dv_r1v_passA(n, lambda, P, Q, ps, pivmin, r1, r2, X, Y, stride, &neg1);
    pr1 = dv_r1v_passB(n, lambda, P, Q, ps, pivmin, r1, r2, true, Y, stride, &neg2, &rbest, &best,
                       &have);
  }
  double sr1 = Y[(size_t)(r1 - 1) * stride];
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
// solve) and then from the smallest up (downward solve); a lane works on the
// rows where it is active.  `active` says whether this lane has a solve to do.
// Writes z over X/Y as described above and returns the outputs.
static __device__ __noinline__ void dv_r1v_solve(bool active, int n, const double2 *__restrict__ Q, int ps,
                                          double gaptol, double *X, double *Y, int stride,
                                          const r1v_state &st, dlar1v_out *o) {
  const int r = active ? st.r : 0;
  const int rmax = __reduce_max_sync(0xffffffffu, active ? r : 0);
  int rmin = __reduce_min_sync(0xffffffffu, active ? r : 0x7fffffff);
  int is1 = 1, is2 = n;
  double ztz = 1.0;
  const bool slow = active && st.sawnan;
  // upward solve: i = r-1 .. 1
  bool go = active;
  double zp = 1.0;
  for (int i = rmax - 1; i >= 1; i--) {
    if (!__any_sync(0xffffffffu, go)) break;
    if (i - MR3_PF >= 1) pf_l1(&X[(size_t)(i - MR3_PF) * stride]);
    if (go && i < r) {
      double zi;
      if (!slow) {
        zi = -(X[(size_t)i * stride] * zp);
      } else {
        double zi1 = dv_zget(X, Y, stride, r, i + 1);
        if (zi1 == 0.0) zi = -(Q[(size_t)i * ps].y / Q[(size_t)(i - 1) * ps].y) * dv_zget(X, Y, stride, r, i + 2);
        else zi = -(X[(size_t)i * stride] * zi1);
        zp = zi1;
      }
      if ((fabs(zi) + fabs(zp)) * fabs(Q[(size_t)(i - 1) * ps].y) < gaptol) {
        X[(size_t)i * stride] = 0.0;
        is1 = i + 1;
        go = false;
      } else {
        ztz = ztz + zi * zi;
        X[(size_t)i * stride] = zi;
        zp = zi;
      }
    }
  }
  // downward solve: i = r .. n-1
  go = active;
  double zc = 1.0;
  if (rmin == 0x7fffffff) rmin = n;
  for (int i = rmin; i <= n - 1; i++) {
    if (!__any_sync(0xffffffffu, go)) break;
    if (i + MR3_PF <= n - 1) pf_l1(&Y[(size_t)(i + MR3_PF) * stride]);
    if (go && i >= r) {
      double zn;
      if (!slow) {
        zn = -(Y[(size_t)i * stride] * zc);
      } else {
        double zci = dv_zget(X, Y, stride, r, i);
        if (zci == 0.0) zn = -(Q[(size_t)(i - 2) * ps].y / Q[(size_t)(i - 1) * ps].y) * dv_zget(X, Y, stride, r, i - 1);
        else zn = -(Y[(size_t)i * stride] * zci);
        zc = zci;
      }
      if ((fabs(zc) + fabs(zn)) * fabs(Q[(size_t)(i - 1) * ps].y) < gaptol) {
        Y[(size_t)i * stride] = 0.0;
        is2 = i;
        go = false;
      } else {
        ztz = ztz + zn * zn;
        Y[(size_t)i * stride] = zn;
        zc = zn;
      }
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

// dlarrf, LAPACK 3.2.2 with NOFAIL (SRC/LAPACK/odrrf.f:140-378), one thread.
// Parent rows: d = P[i].x, l = Q[i].x, ld = Q[i].y.  w/wgap/werr point at the
// cluster's first eigenvalue (CLSTRT = 1, CLEND = clend).  dplus, lplus: out;
// work: 2n scratch.  Returns the shift sigma.
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
    double s = -lsigma;
    dplus(0) = P[0].x + s;
    if (fabs(dplus(0)) < pivmin) { dplus(0) = -pivmin; sawnan1 = true; }
    max1 = fabs(dplus(0));
    for (int i = 0; i < n - 1; i++) {
      const double2 q = Q[(size_t)i * ps];
      lplus(i) = q.y / dplus(i);
      s = s * lplus(i) * q.x - lsigma;
      double dp = P[(size_t)(i + 1) * ps].x + s;
      if (fabs(dp) < pivmin) { dp = -pivmin; sawnan1 = true; }
      dplus(i + 1) = dp;
      max1 = fmax(max1, fabs(dp));
    }
    sawnan1 = sawnan1 || isnan(max1);
    if (forcer || (max1 <= growthbound && !sawnan1)) { sigma = lsigma; shift = 1; break; }

    s = -rsigma;
    work(0) = P[0].x + s;
    if (fabs(work(0)) < pivmin) { work(0) = -pivmin; sawnan2 = true; }
    max2 = fabs(work(0));
    for (int i = 0; i < n - 1; i++) {
      const double2 q = Q[(size_t)i * ps];
      work(n + i) = q.y / work(i);
      s = s * work(n + i) * q.x - rsigma;
      double dp = P[(size_t)(i + 1) * ps].x + s;
      if (fabs(dp) < pivmin) { dp = -pivmin; sawnan2 = true; }
      work(i + 1) = dp;
      max2 = fmax(max2, fabs(dp));
    }
    sawnan2 = sawnan2 || isnan(max2);
    if (forcer || (max2 <= growthbound && !sawnan2)) { sigma = rsigma; shift = 2; break; }

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
    for (int i = 0; i < n; i++) dplus(i) = work(i);
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
