/*
 * mr3_oracle.c -- CPU restatement of the MR3-SMP MRRR path.
 *
 * TEST INFRASTRUCTURE ONLY: the tests, the smoke check and the CPU-baseline leg
 * of bench.py load this file's shared library as the checker.  The product
 * (mr3smp_b200/) never links, loads or calls it.
 *
 * Every routine names the reference file:line range it restates.  Fortran
 * index conventions (1-based IFIRST/ILAST/OFFSET/TWIST/R) are kept at the
 * interfaces so the code can be read against the .f files line by line.
 * The execution order that makes the result deterministic is described in
 * mr3_oracle.h.  Build with -ffp-contract=off: the arithmetic must be plain
 * IEEE double with no fused multiply-add, exactly as the vendored Fortran.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "mr3_oracle.h"

#define OR_EPS    DBL_EPSILON   /* dlamch('P'), SRC/LAPACK/odmch.f */
#define OR_SAFMIN DBL_MIN       /* dlamch('S') == dlamch('U') */

/* Tuning constants of the reference (INCLUDE/mrrr.h:154-200). */
#define MAX_GROWTH      64.0
#define MIN_RELGAP      1e-3
#define MAX_TRY_ROOT    6
#define MAXITER         10      /* SRC/process_singleton.c:57 */
#define EXPAND_CAP      4096    /* bound on the interval-widening loops */
#define DEPTH_CAP       512     /* bound on the representation-tree depth */

static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }

/* ------------------------------------------------------------------------ */
/* Deterministic natural logarithm.                                          */
/* log(x) = e*ln2 + 2*atanh(s), s = (m-1)/(m+1), m in [sqrt(1/2), sqrt(2)),  */
/* atanh by its Taylor series to s^25 (|s| <= 0.1716, truncation < 1e-19),   */
/* ln2 split into the fdlibm hi/lo pair.  Plain +,-,*,/ only, so the device  */
/* copy of this function returns the same bits.  Accurate to about 1 ulp;    */
/* the reference uses libm log, which agrees to within an ulp.              */
/* ------------------------------------------------------------------------ */
double or_log(double x)
{
  const double ln2_hi = 6.93147180369123816490e-01;
  const double ln2_lo = 1.90821492927058770002e-10;
  int e;
  double m, s, s2, p, r;
  if (isnan(x) || x < 0.0) return NAN;
  if (x == 0.0) return -INFINITY;
  if (isinf(x)) return INFINITY;
  m = frexp(x, &e);                         /* x = m * 2^e, m in [0.5, 1) */
  if (m < 0.70710678118654752440) { m = m * 2.0; e = e - 1; }
  s  = (m - 1.0) / (m + 1.0);
  s2 = s * s;
  p  = 1.0 / 25.0;
  p  = 1.0 / 23.0 + s2 * p;
  p  = 1.0 / 21.0 + s2 * p;
  p  = 1.0 / 19.0 + s2 * p;
  p  = 1.0 / 17.0 + s2 * p;
  p  = 1.0 / 15.0 + s2 * p;
  p  = 1.0 / 13.0 + s2 * p;
  p  = 1.0 / 11.0 + s2 * p;
  p  = 1.0 / 9.0  + s2 * p;
  p  = 1.0 / 7.0  + s2 * p;
  p  = 1.0 / 5.0  + s2 * p;
  p  = 1.0 / 3.0  + s2 * p;
  r  = s + (s * s2) * p;                    /* atanh(s) */
  return (double)e * ln2_hi + (2.0 * r + (double)e * ln2_lo);
}

/* INT((LOG(a)-LOG(b))/LOG(TWO)) + 2, the iteration cap of the bisections. */
static int or_itmax(double a, double b)
{
  return (int)((or_log(a) - or_log(b)) / or_log(2.0)) + 2;
}

/* dlanst('M'): SRC/LAPACK/odnst.f ('M' branch). */
double or_dlanst_m(int n, const double *d, const double *e)
{
  double anorm;
  int i;
  if (n <= 0) return 0.0;
  anorm = fabs(d[n - 1]);
  for (i = 0; i < n - 1; i++) {
    anorm = fmax(anorm, fabs(d[i]));
    anorm = fmax(anorm, fabs(e[i]));
  }
  return anorm;
}

/* dlarrr: SRC/LAPACK/odrrr.f:60-146.  Returns INFO (0 = relative accuracy
 * is warranted). */
int or_dlarrr(int n, const double *d, const double *e)
{
  const double relcond = 0.999;
  double smlnum = OR_SAFMIN / OR_EPS;
  double rmin = sqrt(smlnum);
  double offdig = 0.0, offdig2, tmp, tmp2;
  int i;
  if (n <= 0) return 0;
  tmp = sqrt(fabs(d[0]));
  if (tmp < rmin) return 1;
  for (i = 1; i < n; i++) {
    tmp2 = sqrt(fabs(d[i]));
    if (tmp2 < rmin) return 1;
    offdig2 = fabs(e[i - 1]) / (tmp * tmp2);
    if (offdig + offdig2 >= relcond) return 1;
    tmp = tmp2;
    offdig = offdig2;
  }
  return 0;
}

/* dlarra: SRC/LAPACK/odrra.f:98-125.  isplit holds 1-based block ends. */
void or_dlarra(int n, const double *d, double *e, double *e2, double spltol,
               double tnrm, int *nsplit, int *isplit)
{
  int i, ns = 1;
  if (spltol < 0.0) {
    double tmp1 = fabs(spltol) * tnrm;
    for (i = 0; i < n - 1; i++) {
      if (fabs(e[i]) <= tmp1) {
        e[i] = 0.0; e2[i] = 0.0; isplit[ns - 1] = i + 1; ns++;
      }
    }
  } else {
    for (i = 0; i < n - 1; i++) {
      if (fabs(e[i]) <= spltol * sqrt(fabs(d[i])) * sqrt(fabs(d[i + 1]))) {
        e[i] = 0.0; e2[i] = 0.0; isplit[ns - 1] = i + 1; ns++;
      }
    }
  }
  isplit[ns - 1] = n;
  *nsplit = ns;
}

/* Sturm count of T - x with the IJOB=1 rule of dlaebz
 * (SRC/LAPACK/odebz.f:255-270): |pivot| < pivmin -> -pivmin, count pivot <= 0. */
int or_count_ijob1(int n, const double *d, const double *e2, double pivmin,
                   double x)
{
  double tmp = d[0] - x;
  int j, cnt;
  if (fabs(tmp) < pivmin) tmp = -pivmin;
  cnt = (tmp <= 0.0);
  for (j = 1; j < n; j++) {
    tmp = d[j] - e2[j - 1] / tmp - x;
    if (fabs(tmp) < pivmin) tmp = -pivmin;
    if (tmp <= 0.0) cnt++;
  }
  return cnt;
}

/* Sturm count with the IJOB=2/3 rule of dlaebz's serial loop
 * (SRC/LAPACK/odebz.f, loop 90): count pivot <= pivmin, then clamp it to
 * min(pivot, -pivmin). */
int or_count_bisect(int n, const double *d, const double *e2, double pivmin,
                    double c)
{
  double tmp2 = d[0] - c;
  int j, cnt = 0;
  if (tmp2 <= pivmin) { cnt = 1; tmp2 = fmin(tmp2, -pivmin); }
  for (j = 1; j < n; j++) {
    tmp2 = d[j] - e2[j - 1] / tmp2 - c;
    if (tmp2 <= pivmin) { cnt++; tmp2 = fmin(tmp2, -pivmin); }
  }
  return cnt;
}

/* One interval of dlaebz IJOB=3 (binary search for N(w) = nval), from the
 * user-supplied starting point c.  Intervals of IJOB=3 never interact, so one
 * at a time gives the same endpoints (SRC/LAPACK/odebz.f loops 100/110/120). */
static void or_ijob3(int n, const double *d, const double *e2, double pivmin,
                     double abstol, double reltol, int nitmax, int nval,
                     double c, double *a, double *b, int *na, int *nb)
{
  int it;
  for (it = 1; it <= nitmax; it++) {
    int cnt = or_count_bisect(n, d, e2, pivmin, c);
    double w, t;
    if (cnt <= nval) { *a = c; *na = cnt; }
    if (cnt >= nval) { *b = c; *nb = cnt; }
    w = fabs(*b - *a);
    t = fmax(fabs(*b), fabs(*a));
    if (w < fmax(fmax(abstol, pivmin), reltol * t) || *na >= *nb) break;
    c = 0.5 * (*a + *b);
  }
}

/* The interval of eigenvalue j (1-based) under dlaebz IJOB=2, started from
 * [a,b] with counts (na,nb).  dlaebz splits and shrinks intervals by their
 * midpoints, so the interval that holds eigenvalue j evolves exactly as a
 * bisection for j alone (SRC/LAPACK/odebz.f loops 90-120).  Returns 1 if the
 * interval converged within itmax steps. */
static int or_bisect_one(int n, const double *d, const double *e2,
                         double pivmin, double abstol, double reltol,
                         int itmax, int j, double *a, double *b, int na,
                         int nb)
{
  double c = 0.5 * (*a + *b);
  int it;
  for (it = 1; it <= itmax; it++) {
    int cnt = or_count_bisect(n, d, e2, pivmin, c);
    double w, t;
    cnt = imin(nb, imax(na, cnt));
    if (j <= cnt) { *b = c; nb = cnt; } else { *a = c; na = cnt; }
    w = fabs(*b - *a);
    t = fmax(fabs(*b), fabs(*a));
    if (w < fmax(fmax(abstol, pivmin), reltol * t) || na >= nb) return 1;
    c = 0.5 * (*a + *b);
  }
  return 0;
}

/* dlarrd("I","B") on one irreducible block (NSPLIT=1): initial eigenvalue
 * approximations il..iu to relative tolerance reltol.
 * Restates SRC/LAPACK/odrrd.f:283-700 for this call pattern, the one used by
 * find_eigval_irreducible (SRC/mrrr_val.c:1293-1296).  Returns INFO. */
static int or_dlarrd_block(int n, int il, int iu, const double *gers,
                           double reltol, const double *d, const double *e2,
                           double pivmin, int *m, double *w, double *werr,
                           int *indexw)
{
  const int ALLRNG = 1, INDRNG = 3;
  int irange = INDRNG, info = 0, ncnvrg = 0, toofew = 0;
  double gl, gu, tnorm, rtoli, atoli, wl = 0, wu = 0, wlu = 0, wul = 0;
  int nwl = 0, nwu = 0, i, j;
  int *iblk;
  *m = 0;
  if (n <= 0) return 0;
  if (il == 1 && iu == n) irange = ALLRNG;
  if (n == 1) {
    if (irange == ALLRNG || (il == 1 && iu == 1)) {
      *m = 1; w[0] = d[0]; werr[0] = 0.0; indexw[0] = 1;
    }
    return 0;
  }
  gl = d[0]; gu = d[0];
  for (i = 0; i < n; i++) { gl = fmin(gl, gers[2 * i]); gu = fmax(gu, gers[2 * i + 1]); }
  tnorm = fmax(fabs(gl), fabs(gu));
  gl = gl - 2.0 * tnorm * OR_EPS * n - 2.0 * 2.0 * pivmin;
  gu = gu + 2.0 * tnorm * OR_EPS * n + 2.0 * 2.0 * pivmin;
  rtoli = reltol;
  atoli = 2.0 * 2.0 * OR_SAFMIN + 2.0 * 2.0 * pivmin;

  if (irange == INDRNG) {
    int itmax = or_itmax(tnorm + pivmin, pivmin);
    double a1 = gl, b1 = gu, a2 = gl, b2 = gu;
    int na1 = -1, nb1 = n + 1, na2 = -1, nb2 = n + 1;
    or_ijob3(n, d, e2, pivmin, atoli, rtoli, itmax, il - 1, gl, &a1, &b1, &na1, &nb1);
    or_ijob3(n, d, e2, pivmin, atoli, rtoli, itmax, iu, gu, &a2, &b2, &na2, &nb2);
    wl = a1; wlu = b1; nwl = na1;
    wul = a2; wu = b2; nwu = nb2;
    if (nwl < 0 || nwl >= n || nwu < 1 || nwu > n) return 4;
  } else {
    wl = gl; wu = gu;
  }

  /* The single block (odrrd.f loop 70 with NSPLIT=1, IN=N >= 2). */
  nwl = 0; nwu = 0;
  {
    double bgl = d[0], bgu = d[0];
    int nab1, nab2, iwoff;
    for (j = 0; j < n; j++) { bgl = fmin(bgl, gers[2 * j]); bgu = fmax(bgu, gers[2 * j + 1]); }
    bgl = bgl - 2.0 * tnorm * OR_EPS * n - 2.0 * pivmin;
    bgu = bgu + 2.0 * tnorm * OR_EPS * n + 2.0 * pivmin;
    if (irange > 1) {
      if (bgu < wl) { nwl += n; nwu += n; goto discard; }
      bgl = fmax(bgl, wl);
      bgu = fmin(bgu, wu);
      if (bgl >= bgu) goto discard;
    }
    nab1 = or_count_ijob1(n, d, e2, pivmin, bgl);
    nab2 = or_count_ijob1(n, d, e2, pivmin, bgu);
    nwl += nab1; nwu += nab2;
    iwoff = *m - nab1;
    {
      int itmax = or_itmax(bgu - bgl + pivmin, pivmin);
      for (j = nab1 + 1; j <= nab2; j++) {
        double a = bgl, b = bgu;
        int je = j + iwoff;               /* 1-based position in w */
        if (!or_bisect_one(n, d, e2, pivmin, atoli, rtoli, itmax, j, &a, &b, nab1, nab2))
          ncnvrg = 1;
        w[je - 1] = 0.5 * (a + b);
        werr[je - 1] = 0.5 * fabs(a - b);
        indexw[je - 1] = je - iwoff;
      }
      *m += nab2 - nab1;
    }
  }

discard:
  if (irange == INDRNG) {
    int idiscl = il - 1 - nwl, idiscu = nwu - iu, im, je, jee;
    iblk = (int *)malloc(sizeof(int) * (size_t)imax(*m, 1));
    for (je = 0; je < *m; je++) iblk[je] = 1;
    if (idiscl > 0) {
      im = 0;
      for (je = 0; je < *m; je++) {
        if (w[je] <= wlu && idiscl > 0) {
          idiscl--;
        } else {
          w[im] = w[je]; werr[im] = werr[je]; indexw[im] = indexw[je]; iblk[im] = iblk[je]; im++;
        }
      }
      *m = im;
    }
    if (idiscu > 0) {
      im = *m;
      for (je = *m - 1; je >= 0; je--) {
        if (w[je] >= wul && idiscu > 0) {
          idiscu--;
        } else {
          im--;
          w[im] = w[je]; werr[im] = werr[je]; indexw[im] = indexw[je]; iblk[im] = iblk[je];
        }
      }
      jee = 0;
      for (je = im; je < *m; je++) {
        w[jee] = w[je]; werr[jee] = werr[je]; indexw[jee] = indexw[je]; iblk[jee] = iblk[je]; jee++;
      }
      *m = *m - im;
    }
    if (idiscl > 0 || idiscu > 0) {
      int jdisc, iw;
      double wkill;
      if (idiscl > 0) {
        wkill = wu;
        for (jdisc = 0; jdisc < idiscl; jdisc++) {
          iw = -1;
          for (je = 0; je < *m; je++)
            if (iblk[je] != 0 && (w[je] < wkill || iw == -1)) { iw = je; wkill = w[je]; }
          iblk[iw] = 0;
        }
      }
      if (idiscu > 0) {
        wkill = wl;
        for (jdisc = 0; jdisc < idiscu; jdisc++) {
          iw = -1;
          for (je = 0; je < *m; je++)
            if (iblk[je] != 0 && (w[je] >= wkill || iw == -1)) { iw = je; wkill = w[je]; }
          iblk[iw] = 0;
        }
      }
      im = 0;
      for (je = 0; je < *m; je++) {
        if (iblk[je] != 0) {
          w[im] = w[je]; werr[im] = werr[je]; indexw[im] = indexw[je]; im++;
        }
      }
      *m = im;
    }
    if (idiscl < 0 || idiscu < 0) toofew = 1;
    free(iblk);
  }
  if ((irange == ALLRNG && *m != n) || (irange == INDRNG && *m != iu - il + 1))
    toofew = 1;
  info = 0;
  if (ncnvrg) info += 1;
  if (toofew) info += 2;
  return info;
}

/* dlarrc('T'): SRC/LAPACK/odrrc.f:100-123. */
void or_dlarrc_t(int n, double vl, double vu, const double *d, const double *e,
                 double pivmin, int *eigcnt, int *lcnt, int *rcnt)
{
  double lpivot = d[0] - vl, rpivot = d[0] - vu, tmp;
  int i, lc = 0, rc = 0;
  (void)pivmin;
  if (lpivot <= 0.0) lc++;
  if (rpivot <= 0.0) rc++;
  for (i = 0; i < n - 1; i++) {
    tmp = e[i] * e[i];
    lpivot = (d[i + 1] - vl) - tmp / lpivot;
    rpivot = (d[i + 1] - vu) - tmp / rpivot;
    if (lpivot <= 0.0) lc++;
    if (rpivot <= 0.0) rc++;
  }
  *lcnt = lc; *rcnt = rc; *eigcnt = rc - lc;
}

/* dlaneg: SRC/LAPACK/odneg.f:98-163.  Sturm count of L D L^T - sigma I by a
 * stationary transform down to the twist index r and a progressive one up to
 * it, re-running any 128-block whose result is NaN with 0/0 read as 1. */
int or_dlaneg(int n, const double *d, const double *lld, double sigma,
              double pivmin, int r)
{
  const int blklen = 128;
  int negcnt = 0, bj, j, neg1, neg2;
  double t, p, bsav, dplus, dminus, tmp, gamma;
  (void)pivmin;
  t = -sigma;
  for (bj = 1; bj <= r - 1; bj += blklen) {
    int jend = imin(bj + blklen - 1, r - 1);
    neg1 = 0; bsav = t;
    for (j = bj; j <= jend; j++) {
      dplus = d[j - 1] + t;
      if (dplus < 0.0) neg1++;
      tmp = t / dplus;
      t = tmp * lld[j - 1] - sigma;
    }
    if (isnan(t)) {
      neg1 = 0; t = bsav;
      for (j = bj; j <= jend; j++) {
        dplus = d[j - 1] + t;
        if (dplus < 0.0) neg1++;
        tmp = t / dplus;
        if (isnan(tmp)) tmp = 1.0;
        t = tmp * lld[j - 1] - sigma;
      }
    }
    negcnt += neg1;
  }
  p = d[n - 1] - sigma;
  for (bj = n - 1; bj >= r; bj -= blklen) {
    int jend = imax(bj - blklen + 1, r);
    neg2 = 0; bsav = p;
    for (j = bj; j >= jend; j--) {
      dminus = lld[j - 1] + p;
      if (dminus < 0.0) neg2++;
      tmp = p / dminus;
      p = tmp * d[j - 1] - sigma;
    }
    if (isnan(p)) {
      neg2 = 0; p = bsav;
      for (j = bj; j >= jend; j--) {
        dminus = lld[j - 1] + p;
        if (dminus < 0.0) neg2++;
        tmp = p / dminus;
        if (isnan(tmp)) tmp = 1.0;
        p = tmp * d[j - 1] - sigma;
      }
    }
    negcnt += neg2;
  }
  gamma = (t + sigma) + p;
  if (gamma < 0.0) negcnt++;
  return negcnt;
}

/* dlarrb: SRC/LAPACK/odrrb.f:136-293.  work[2n], iwork[2n]. */
void or_dlarrb(int n, const double *d, const double *lld, int ifirst,
               int ilast, double rtol1, double rtol2, int offset, double *w,
               double *wgap, double *werr, double *work, int *iwork,
               double pivmin, double spdiam, int twist, int *info)
{
  int maxitr = or_itmax(spdiam + pivmin, pivmin);
  double mnwdth = 2.0 * pivmin;
  int r = twist, i1, nint, prev, i, k, ii, iter, olnint, ip, next, negcnt, cap;
  double lgap, rgap, gap, left, right, back, width, tmp, cvrgd, mid;
  *info = 0;
  if (r < 1 || r > n) r = n;
  i1 = ifirst; nint = 0; prev = 0;
  rgap = wgap[i1 - offset - 1];
  for (i = i1; i <= ilast; i++) {
    k = 2 * i; ii = i - offset;
    left = w[ii - 1] - werr[ii - 1];
    right = w[ii - 1] + werr[ii - 1];
    lgap = rgap; rgap = wgap[ii - 1];
    gap = fmin(lgap, rgap);
    back = werr[ii - 1];
    for (cap = 0; cap < EXPAND_CAP; cap++) {
      negcnt = or_dlaneg(n, d, lld, left, pivmin, r);
      if (negcnt > i - 1) { left = left - back; back = 2.0 * back; } else break;
    }
    if (cap == EXPAND_CAP) *info = -1;
    back = werr[ii - 1];
    for (cap = 0; cap < EXPAND_CAP; cap++) {
      negcnt = or_dlaneg(n, d, lld, right, pivmin, r);
      if (negcnt < i) { right = right + back; back = 2.0 * back; } else break;
    }
    if (cap == EXPAND_CAP) *info = -1;
    width = 0.5 * fabs(left - right);
    tmp = fmax(fabs(left), fabs(right));
    cvrgd = fmax(rtol1 * gap, rtol2 * tmp);
    if (width <= cvrgd || width <= mnwdth) {
      iwork[k - 2] = -1;
      if (i == i1 && i < ilast) i1 = i + 1;
      if (prev >= i1 && i <= ilast) iwork[2 * prev - 2] = i + 1;
    } else {
      prev = i; nint++;
      iwork[k - 2] = i + 1;
      iwork[k - 1] = negcnt;
    }
    work[k - 2] = left;
    work[k - 1] = right;
  }
  iter = 0;
  for (;;) {
    prev = i1 - 1; i = i1; olnint = nint;
    for (ip = 1; ip <= olnint; ip++) {
      k = 2 * i; ii = i - offset;
      rgap = wgap[ii - 1];
      lgap = rgap;
      if (ii > 1) lgap = wgap[ii - 2];
      gap = fmin(lgap, rgap);
      next = iwork[k - 2];
      left = work[k - 2]; right = work[k - 1];
      mid = 0.5 * (left + right);
      width = right - mid;
      tmp = fmax(fabs(left), fabs(right));
      cvrgd = fmax(rtol1 * gap, rtol2 * tmp);
      if (width <= cvrgd || width <= mnwdth || iter == maxitr) {
        nint--;
        iwork[k - 2] = 0;
        if (i1 == i) i1 = next;
        else if (prev >= i1) iwork[2 * prev - 2] = next;
        i = next;
        continue;
      }
      prev = i;
      negcnt = or_dlaneg(n, d, lld, mid, pivmin, r);
      if (negcnt <= i - 1) work[k - 2] = mid; else work[k - 1] = mid;
      i = next;
    }
    iter++;
    if (!(nint > 0 && iter <= maxitr)) break;
  }
  for (i = ifirst; i <= ilast; i++) {
    k = 2 * i; ii = i - offset;
    if (iwork[k - 2] == 0) {
      w[ii - 1] = 0.5 * (work[k - 2] + work[k - 1]);
      werr[ii - 1] = work[k - 1] - w[ii - 1];
    }
  }
  for (i = ifirst + 1; i <= ilast; i++) {
    ii = i - offset;
    wgap[ii - 2] = fmax(0.0, w[ii - 1] - werr[ii - 1] - w[ii - 2] - werr[ii - 2]);
  }
}

/* dlar1v: SRC/LAPACK/odr1v.f:158-362.  work[4n]; z and isuppz are 1-based
 * relative to the block (z[0] is row B1=1). */
void or_dlar1v(int n, int b1, int bn, double lambda, const double *d,
               const double *l, const double *ld, const double *lld,
               double pivmin, double gaptol, double *z, int wantnc,
               int *negcnt, double *ztz, double *mingma, int *r, int *isuppz,
               double *nrminv, double *resid, double *rqcorr, double *work)
{
  /* Fortran 1-based views: D(i) = d[i-1], WORK(k) = work[k-1], Z(i) = z[i-1]. */
#define D_(i)    d[(i) - 1]
#define L_(i)    l[(i) - 1]
#define LD_(i)   ld[(i) - 1]
#define LLD_(i)  lld[(i) - 1]
#define WK(k)    work[(k) - 1]
#define Z_(i)    z[(i) - 1]
  const double eps = OR_EPS;
  int r1, r2, indlpl, indumn, inds, indp, i, neg1, neg2, sawnan1, sawnan2;
  double s, dplus, dminus, tmp;
  if (*r == 0) { r1 = b1; r2 = bn; } else { r1 = *r; r2 = *r; }
  indlpl = 0; indumn = n; inds = 2 * n + 1; indp = 3 * n + 1;
  if (b1 == 1) WK(inds) = 0.0; else WK(inds + b1 - 1) = LLD_(b1 - 1);

  sawnan1 = 0; neg1 = 0;
  s = WK(inds + b1 - 1) - lambda;
  for (i = b1; i <= r1 - 1; i++) {
    dplus = D_(i) + s;
    WK(indlpl + i) = LD_(i) / dplus;
    if (dplus < 0.0) neg1++;
    WK(inds + i) = s * WK(indlpl + i) * L_(i);
    s = WK(inds + i) - lambda;
  }
  sawnan1 = isnan(s);
  if (!sawnan1) {
    for (i = r1; i <= r2 - 1; i++) {
      dplus = D_(i) + s;
      WK(indlpl + i) = LD_(i) / dplus;
      WK(inds + i) = s * WK(indlpl + i) * L_(i);
      s = WK(inds + i) - lambda;
    }
    sawnan1 = isnan(s);
  }
  if (sawnan1) {
    neg1 = 0;
    s = WK(inds + b1 - 1) - lambda;
    for (i = b1; i <= r1 - 1; i++) {
      dplus = D_(i) + s;
      if (fabs(dplus) < pivmin) dplus = -pivmin;
      WK(indlpl + i) = LD_(i) / dplus;
      if (dplus < 0.0) neg1++;
      WK(inds + i) = s * WK(indlpl + i) * L_(i);
      if (WK(indlpl + i) == 0.0) WK(inds + i) = LLD_(i);
      s = WK(inds + i) - lambda;
    }
    for (i = r1; i <= r2 - 1; i++) {
      dplus = D_(i) + s;
      if (fabs(dplus) < pivmin) dplus = -pivmin;
      WK(indlpl + i) = LD_(i) / dplus;
      WK(inds + i) = s * WK(indlpl + i) * L_(i);
      if (WK(indlpl + i) == 0.0) WK(inds + i) = LLD_(i);
      s = WK(inds + i) - lambda;
    }
  }

  sawnan2 = 0; neg2 = 0;
  WK(indp + bn - 1) = D_(bn) - lambda;
  for (i = bn - 1; i >= r1; i--) {
    dminus = LLD_(i) + WK(indp + i);
    tmp = D_(i) / dminus;
    if (dminus < 0.0) neg2++;
    WK(indumn + i) = L_(i) * tmp;
    WK(indp + i - 1) = WK(indp + i) * tmp - lambda;
  }
  tmp = WK(indp + r1 - 1);
  sawnan2 = isnan(tmp);
  if (sawnan2) {
    neg2 = 0;
    for (i = bn - 1; i >= r1; i--) {
      dminus = LLD_(i) + WK(indp + i);
      if (fabs(dminus) < pivmin) dminus = -pivmin;
      tmp = D_(i) / dminus;
      if (dminus < 0.0) neg2++;
      WK(indumn + i) = L_(i) * tmp;
      WK(indp + i - 1) = WK(indp + i) * tmp - lambda;
      if (tmp == 0.0) WK(indp + i - 1) = D_(i) - lambda;
    }
  }

  *mingma = WK(inds + r1 - 1) + WK(indp + r1 - 1);
  if (*mingma < 0.0) neg1++;
  *negcnt = wantnc ? neg1 + neg2 : -1;
  if (fabs(*mingma) == 0.0) *mingma = eps * WK(inds + r1 - 1);
  *r = r1;
  for (i = r1; i <= r2 - 1; i++) {
    tmp = WK(inds + i) + WK(indp + i);
    if (tmp == 0.0) tmp = eps * WK(inds + i);
    if (fabs(tmp) <= fabs(*mingma)) { *mingma = tmp; *r = i + 1; }
  }

  isuppz[0] = b1; isuppz[1] = bn;
  Z_(*r) = 1.0;
  *ztz = 1.0;
  if (!sawnan1 && !sawnan2) {
    for (i = *r - 1; i >= b1; i--) {
      Z_(i) = -(WK(indlpl + i) * Z_(i + 1));
      if ((fabs(Z_(i)) + fabs(Z_(i + 1))) * fabs(LD_(i)) < gaptol) {
        Z_(i) = 0.0; isuppz[0] = i + 1; break;
      }
      *ztz = *ztz + Z_(i) * Z_(i);
    }
  } else {
    for (i = *r - 1; i >= b1; i--) {
      if (Z_(i + 1) == 0.0) Z_(i) = -(LD_(i + 1) / LD_(i)) * Z_(i + 2);
      else Z_(i) = -(WK(indlpl + i) * Z_(i + 1));
      if ((fabs(Z_(i)) + fabs(Z_(i + 1))) * fabs(LD_(i)) < gaptol) {
        Z_(i) = 0.0; isuppz[0] = i + 1; break;
      }
      *ztz = *ztz + Z_(i) * Z_(i);
    }
  }
  if (!sawnan1 && !sawnan2) {
    for (i = *r; i <= bn - 1; i++) {
      Z_(i + 1) = -(WK(indumn + i) * Z_(i));
      if ((fabs(Z_(i)) + fabs(Z_(i + 1))) * fabs(LD_(i)) < gaptol) {
        Z_(i + 1) = 0.0; isuppz[1] = i; break;
      }
      *ztz = *ztz + Z_(i + 1) * Z_(i + 1);
    }
  } else {
    for (i = *r; i <= bn - 1; i++) {
      if (Z_(i) == 0.0) Z_(i + 1) = -(LD_(i - 1) / LD_(i)) * Z_(i - 1);
      else Z_(i + 1) = -(WK(indumn + i) * Z_(i));
      if ((fabs(Z_(i)) + fabs(Z_(i + 1))) * fabs(LD_(i)) < gaptol) {
        Z_(i + 1) = 0.0; isuppz[1] = i; break;
      }
      *ztz = *ztz + Z_(i + 1) * Z_(i + 1);
    }
  }
  tmp = 1.0 / *ztz;
  *nrminv = sqrt(tmp);
  *resid = fabs(*mingma) * *nrminv;
  *rqcorr = *mingma * tmp;
#undef D_
#undef L_
#undef LD_
#undef LLD_
#undef WK
#undef Z_
}

/* dlarrf (LAPACK 3.2.2, NOFAIL): SRC/LAPACK/odrrf.f:140-378.
 * clstrt/clend are 1-based into w/wgap/werr.  work[2n]. */
void or_dlarrf(int n, const double *d, const double *l, const double *ld,
               int clstrt, int clend, const double *w, const double *wgap,
               const double *werr, double spdiam, double clgapl,
               double clgapr, double pivmin, double *sigma, double *dplus,
               double *lplus, double *work, int *info)
{
  const double maxgrowth1 = 8.0, maxgrowth2 = 8.0;
  const int ktrymax = 1, sleft = 1, sright = 2;
  double eps = OR_EPS, fact = 2.0;   /* DBLE(2**KTRYMAX) */
  int shift = 0, forcer = 0, nofail = 1, sawnan1, sawnan2, indx = 0, ktry, i, dorrr1;
  double clwdth, avgap, mingap, lsigma, rsigma, ldmax, rdmax, ldelta, rdelta;
  double smlgrowth, fail, fail2, bestshift, growthbound, s, max1, max2;
  double tmp, znm2, prod, oldp, rrr1, rrr2;
#define W_(i)    w[(i) - 1]
#define WERR_(i) werr[(i) - 1]
#define WGAP_(i) wgap[(i) - 1]
  *info = 0;
  clwdth = fabs(W_(clend) - W_(clstrt)) + WERR_(clend) + WERR_(clstrt);
  avgap = clwdth / (double)(clend - clstrt);
  mingap = fmin(clgapl, clgapr);
  lsigma = fmin(W_(clstrt), W_(clend)) - WERR_(clstrt);
  rsigma = fmax(W_(clstrt), W_(clend)) + WERR_(clend);
  lsigma = lsigma - fabs(lsigma) * 4.0 * eps;
  rsigma = rsigma + fabs(rsigma) * 4.0 * eps;
  ldmax = 0.25 * mingap + 2.0 * pivmin;
  rdmax = 0.25 * mingap + 2.0 * pivmin;
  ldelta = fmax(avgap, WGAP_(clstrt)) / fact;
  rdelta = fmax(avgap, WGAP_(clend - 1)) / fact;
  smlgrowth = 1.0 / OR_SAFMIN;
  fail = (double)(n - 1) * mingap / (spdiam * eps);
  fail2 = (double)(n - 1) * mingap / (spdiam * sqrt(eps));
  bestshift = lsigma;
  ktry = 0;
  growthbound = maxgrowth1 * spdiam;

  for (;;) {   /* label 5 */
    sawnan1 = 0; sawnan2 = 0;
    ldelta = fmin(ldmax, ldelta);
    rdelta = fmin(rdmax, rdelta);

    s = -lsigma;
    dplus[0] = d[0] + s;
    if (fabs(dplus[0]) < pivmin) { dplus[0] = -pivmin; sawnan1 = 1; }
    max1 = fabs(dplus[0]);
    for (i = 0; i < n - 1; i++) {
      lplus[i] = ld[i] / dplus[i];
      s = s * lplus[i] * l[i] - lsigma;
      dplus[i + 1] = d[i + 1] + s;
      if (fabs(dplus[i + 1]) < pivmin) { dplus[i + 1] = -pivmin; sawnan1 = 1; }
      max1 = fmax(max1, fabs(dplus[i + 1]));
    }
    sawnan1 = sawnan1 || isnan(max1);
    if (forcer || (max1 <= growthbound && !sawnan1)) {
      *sigma = lsigma; shift = sleft; break;
    }

    s = -rsigma;
    work[0] = d[0] + s;
    if (fabs(work[0]) < pivmin) { work[0] = -pivmin; sawnan2 = 1; }
    max2 = fabs(work[0]);
    for (i = 0; i < n - 1; i++) {
      work[n + i] = ld[i] / work[i];
      s = s * work[n + i] * l[i] - rsigma;
      work[i + 1] = d[i + 1] + s;
      if (fabs(work[i + 1]) < pivmin) { work[i + 1] = -pivmin; sawnan2 = 1; }
      max2 = fmax(max2, fabs(work[i + 1]));
    }
    sawnan2 = sawnan2 || isnan(max2);
    if (forcer || (max2 <= growthbound && !sawnan2)) {
      *sigma = rsigma; shift = sright; break;
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
      dorrr1 = (clwdth < mingap / 128.0) && (fmin(max1, max2) < fail2) && !sawnan1 && !sawnan2;
      if (dorrr1) {
        if (indx == 1) {
          tmp = fabs(dplus[n - 1]);
          znm2 = 1.0; prod = 1.0; oldp = 1.0;
          for (i = n - 1; i >= 1; i--) {     /* Fortran I = N-1..1 */
            if (prod <= eps)
              prod = ((dplus[i] * work[n + i]) / (dplus[i - 1] * work[n + i - 1])) * oldp;
            else
              prod = prod * fabs(work[n + i - 1]);
            oldp = prod;
            znm2 = znm2 + prod * prod;
            tmp = fmax(tmp, fabs(dplus[i - 1] * prod));
          }
          rrr1 = tmp / (spdiam * sqrt(znm2));
          if (rrr1 <= maxgrowth2) { *sigma = lsigma; shift = sleft; break; }
        } else if (indx == 2) {
          tmp = fabs(work[n - 1]);
          znm2 = 1.0; prod = 1.0; oldp = 1.0;
          for (i = n - 1; i >= 1; i--) {
            if (prod <= eps)
              prod = ((work[i] * lplus[i]) / (work[i - 1] * lplus[i - 1])) * oldp;
            else
              prod = prod * fabs(lplus[i - 1]);
            oldp = prod;
            znm2 = znm2 + prod * prod;
            tmp = fmax(tmp, fabs(work[i - 1] * prod));
          }
          rrr2 = tmp / (spdiam * sqrt(znm2));
          if (rrr2 <= maxgrowth2) { *sigma = rsigma; shift = sright; break; }
        }
      }
    }
    /* label 50 */
    if (ktry < ktrymax) {
      lsigma = fmax(lsigma - ldelta, lsigma - ldmax);
      rsigma = fmin(rsigma + rdelta, rsigma + rdmax);
      ldelta = 2.0 * ldelta;
      rdelta = 2.0 * rdelta;
      ktry++;
      continue;
    }
    if (smlgrowth < fail || nofail) {
      lsigma = bestshift; rsigma = bestshift; forcer = 1;
      continue;
    }
    *info = 1;
    return;
  }
  if (shift == sright) {
    memcpy(dplus, work, sizeof(double) * (size_t)n);
    memcpy(lplus, work + n, sizeof(double) * (size_t)(n - 1));
  }
#undef W_
#undef WERR_
#undef WGAP_
}

/* dlarrj: SRC/LAPACK/odrrj.f:100-281 (bisection on T to relative rtol). */
void or_dlarrj(int n, const double *d, const double *e2, int ifirst,
               int ilast, double rtol, int offset, double *w, double *werr,
               double *work, int *iwork, double pivmin, double spdiam,
               int *info)
{
  int maxitr = or_itmax(spdiam + pivmin, pivmin);
  int i1 = ifirst, i2 = ilast, nint = 0, prev = 0, i, k, ii, cnt, j, savi1, iter, olnint, p, next, cap;
  double left, mid, right, width, tmp, s, dplus, fac;
  *info = 0;
  for (i = i1; i <= i2; i++) {
    k = 2 * i; ii = i - offset;
    left = w[ii - 1] - werr[ii - 1];
    mid = w[ii - 1];
    right = w[ii - 1] + werr[ii - 1];
    width = right - mid;
    tmp = fmax(fabs(left), fabs(right));
    if (width < rtol * tmp) {
      iwork[k - 2] = -1;
      if (i == i1 && i < i2) i1 = i + 1;
      if (prev >= i1 && i <= i2) iwork[2 * prev - 2] = i + 1;
    } else {
      prev = i;
      fac = 1.0;
      for (cap = 0; cap < EXPAND_CAP; cap++) {
        cnt = 0; s = left;
        dplus = d[0] - s;
        if (dplus < 0.0) cnt++;
        for (j = 1; j < n; j++) {
          dplus = d[j] - s - e2[j - 1] / dplus;
          if (dplus < 0.0) cnt++;
        }
        if (cnt > i - 1) { left = left - werr[ii - 1] * fac; fac = 2.0 * fac; } else break;
      }
      fac = 1.0;
      for (cap = 0; cap < EXPAND_CAP; cap++) {
        cnt = 0; s = right;
        dplus = d[0] - s;
        if (dplus < 0.0) cnt++;
        for (j = 1; j < n; j++) {
          dplus = d[j] - s - e2[j - 1] / dplus;
          if (dplus < 0.0) cnt++;
        }
        if (cnt < i) { right = right + werr[ii - 1] * fac; fac = 2.0 * fac; } else break;
      }
      nint++;
      iwork[k - 2] = i + 1;
      iwork[k - 1] = cnt;
    }
    work[k - 2] = left;
    work[k - 1] = right;
  }
  savi1 = i1;
  iter = 0;
  for (;;) {
    prev = i1 - 1; i = i1; olnint = nint;
    for (p = 1; p <= olnint; p++) {
      k = 2 * i; ii = i - offset;
      next = iwork[k - 2];
      left = work[k - 2]; right = work[k - 1];
      mid = 0.5 * (left + right);
      width = right - mid;
      tmp = fmax(fabs(left), fabs(right));
      if (width < rtol * tmp || iter == maxitr) {
        nint--;
        iwork[k - 2] = 0;
        if (i1 == i) i1 = next;
        else if (prev >= i1) iwork[2 * prev - 2] = next;
        i = next;
        continue;
      }
      prev = i;
      cnt = 0; s = mid;
      dplus = d[0] - s;
      if (dplus < 0.0) cnt++;
      for (j = 1; j < n; j++) {
        dplus = d[j] - s - e2[j - 1] / dplus;
        if (dplus < 0.0) cnt++;
      }
      if (cnt <= i - 1) work[k - 2] = mid; else work[k - 1] = mid;
      i = next;
    }
    iter++;
    if (!(nint > 0 && iter <= maxitr)) break;
  }
  for (i = savi1; i <= ilast; i++) {
    k = 2 * i; ii = i - offset;
    if (iwork[k - 2] == 0) {
      w[ii - 1] = 0.5 * (work[k - 2] + work[k - 1]);
      werr[ii - 1] = work[k - 1] - w[ii - 1];
    }
  }
}

/* dlarnv(IDIST=2) through dlaruv: SRC/LAPACK/odrnv.f, SRC/LAPACK/odruv.f.
 * dlaruv's multiplier table holds the powers a^i mod 2^48 of
 * a = 33952834046453, so the k-th number of a stream that starts at seed s is
 * (s * a^k mod 2^48) / 2^48, mapped to (-1,1) by 2u-1.  The new seed is
 * s * a^n. */
void or_dlarnv2(int iseed[4], int n, double *x)
{
  const uint64_t a = 33952834046453ULL, mask = (1ULL << 48) - 1ULL;
  uint64_t s = ((uint64_t)iseed[0] << 36) | ((uint64_t)iseed[1] << 24) |
               ((uint64_t)iseed[2] << 12) | (uint64_t)iseed[3];
  int k;
  for (k = 0; k < n; k++) {
    s = (s * a) & mask;
    x[k] = 2.0 * ((double)s * 0x1p-48) - 1.0;
  }
  iseed[0] = (int)((s >> 36) & 4095); iseed[1] = (int)((s >> 24) & 4095);
  iseed[2] = (int)((s >> 12) & 4095); iseed[3] = (int)(s & 4095);
}

/* ======================================================================== */
/* The solver.                                                               */
/* ======================================================================== */

typedef struct {
  int n, nsplit;
  double *D, *E, *E2;
  int *isplit;            /* 1-based block ends */
  double spdiam;
} or_in_t;

typedef struct {
  int n, m;
  double *vlp, *vup;
  int *ilp, *iup, *mp;
  double *W, *Werr, *Wgap, *Wshifted, *gersch;
  int *Windex, *iblock;
} or_val_t;

typedef struct {
  double split, rtol1, rtol2, RQtol, pivmin, bsrtol;
} or_tol_t;

/* compute_root_rrr, bisection branch: SRC/mrrr_val.c:717-948 with
 * allrng_no_bisec = useDQDS = false. */
/* dlarrk (SRC/LAPACK/odrrk.f:120-161): the iw-th eigenvalue of T by
 * bisection on [gl, gu] to relative tolerance reltol; w, werr. */
static void or_dlarrk(int n, int iw, double gl, double gu, const double *d, const double *e2,
                      double pivmin, double reltol, double *w, double *werr)
{
  const double eps = OR_EPS, fudge = 2.0;
  const double tnorm = fmax(fabs(gl), fabs(gu)), atoli = fudge * 2.0 * pivmin;
  const int itmax = (int)((or_log(tnorm + pivmin) - or_log(pivmin)) / or_log(2.0)) + 2;
  double left = gl - fudge * tnorm * eps * n - fudge * 2.0 * pivmin;
  double right = gu + fudge * tnorm * eps * n + fudge * 2.0 * pivmin;
  int it = 0, i, negcnt;
  for (;;) {
    double tmp1 = fabs(right - left), tmp2 = fmax(fabs(right), fabs(left)), mid;
    if (tmp1 < fmax(fmax(atoli, pivmin), reltol * tmp2)) break;
    if (it > itmax) break;
    it++;
    mid = 0.5 * (left + right);
    negcnt = 0;
    tmp1 = d[0] - mid;
    if (fabs(tmp1) < pivmin) tmp1 = -pivmin;
    if (tmp1 <= 0.0) negcnt++;
    for (i = 2; i <= n; i++) {
      tmp1 = d[i - 1] - e2[i - 2] / tmp1 - mid;
      if (fabs(tmp1) < pivmin) tmp1 = -pivmin;
      if (tmp1 <= 0.0) negcnt++;
    }
    if (negcnt >= iw) right = mid;
    else left = mid;
  }
  *w = 0.5 * (left + right);
  *werr = 0.5 * fabs(right - left);
}

/* compute_root_rrr (SRC/mrrr_val.c:717-948).  allrng_no_bisec / useDQDS:
 * the branches of the dqds route (extremal eigenvalues by dlarrk, the shift
 * at an end of [isleft, isright], a definite representation). */
static int or_root_rrr(int allrng_no_bisec, int useDQDS, int ibgn, int iend, int wbgn,
                       int wend, int ilow, int iupp, double gl, double gu, or_in_t *Ds,
                       or_val_t *Ws, or_tol_t *tol, double *work, int *sgndefp,
                       double *sigmap, double *spdiamp)
{
  int nbl = iend - ibgn + 1, mbl = wend - wbgn + 1, n = Ds->n, i, j, jtry;
  double *D = Ds->D, *E = Ds->E, *W = Ws->W, *Werr = Ws->Werr, *Wgap = Ws->Wgap;
  double pivmin = tol->pivmin, isleft, isright, spdiam, tmp0, tmp1, s1, s2, sigma;
  double clwdth, avgap, tau, Dpivot, Dmax;
  int cnt = 0, negcnt_lft = 0, negcnt_rgt = 0, sgndef, noREP;
  int off_L = n, off_invD = 2 * n;

  if (allrng_no_bisec || useDQDS) {
    const double rtl = sqrt(OR_EPS);
    or_dlarrk(nbl, 1, gl, gu, &D[ibgn], &Ds->E2[ibgn], pivmin, rtl, &tmp0, &tmp1);
    isleft = fmax(gl, (tmp0 - tmp1) - 100.0 * OR_EPS * fabs(tmp0 - tmp1));
    or_dlarrk(nbl, nbl, gl, gu, &D[ibgn], &Ds->E2[ibgn], pivmin, rtl, &tmp0, &tmp1);
    isright = fmin(gu, (tmp0 + tmp1) + 100.0 * OR_EPS * fabs(tmp0 + tmp1));
    spdiam = isright - isleft;
  } else {
    isleft = fmax(gl, (W[wbgn] - Werr[wbgn]) - 100.0 * OR_EPS * fabs(W[wbgn] - Werr[wbgn]));
    isright = fmin(gu, (W[wend] + Werr[wend]) + 100.0 * OR_EPS * fabs(W[wend] - Werr[wend]));
    spdiam = gu - gl;
  }
  if (allrng_no_bisec || useDQDS) {
    s1 = isleft + 0.25 * spdiam;
    s2 = isright - 0.25 * spdiam;
  } else {
    tmp0 = fmin(isright, *Ws->vup) - fmax(isleft, *Ws->vlp);
    s1 = fmax(isleft, *Ws->vlp) + 0.25 * tmp0;
    s2 = fmin(isright, *Ws->vup) - 0.25 * tmp0;
  }
  if (mbl > 1)
    or_dlarrc_t(nbl, s1, s2, &D[ibgn], &E[ibgn], pivmin, &cnt, &negcnt_lft, &negcnt_rgt);
  if (mbl == 1) {
    sigma = gl; sgndef = 1;
  } else if ((negcnt_lft - ilow) >= (iupp - negcnt_rgt)) {
    if (allrng_no_bisec) sigma = fmax(isleft, gl);
    else if (useDQDS) sigma = isleft;
    else sigma = fmax(isleft, *Ws->vlp);
    sgndef = 1;
  } else {
    if (allrng_no_bisec) sigma = fmin(isright, gu);
    else if (useDQDS) sigma = isright;
    else sigma = fmin(isright, *Ws->vup);
    sgndef = -1;
  }
  if (useDQDS) {
    tau = spdiam * OR_EPS * nbl + 2.0 * pivmin;
    tau = fmax(tau, 2 * OR_EPS * fabs(sigma));
  } else if (mbl > 1) {
    clwdth = W[wend] + Werr[wend] - W[wbgn] - Werr[wbgn];
    avgap = fabs(clwdth / (double)(wend - wbgn));
    if (sgndef > 0) {
      tau = fmax(Wgap[wbgn], avgap); tau *= 0.5; tau = fmax(tau, Werr[wbgn]);
    } else {
      tau = fmax(Wgap[wend - 1], avgap); tau *= 0.5; tau = fmax(tau, Werr[wend]);
    }
  } else {
    tau = Werr[wbgn];
  }
  for (jtry = 0; jtry < MAX_TRY_ROOT; jtry++) {
    Dpivot = D[ibgn] - sigma;
    work[0] = Dpivot;
    Dmax = fabs(work[0]);
    j = ibgn;
    for (i = 0; i < nbl - 1; i++) {
      work[i + off_invD] = 1.0 / work[i];
      tmp0 = E[j] * work[i + off_invD];
      work[i + off_L] = tmp0;
      Dpivot = (D[j + 1] - sigma) - tmp0 * E[j];
      work[i + 1] = Dpivot;
      Dmax = fmax(Dmax, fabs(Dpivot));
      j++;
    }
    noREP = (Dmax > MAX_GROWTH * spdiam);
    if (useDQDS && !noREP)   /* dqds needs a definite representation */
      for (i = 0; i < nbl; i++)
        if (sgndef * work[i] < 0.0) noREP = 1;
    if (noREP) {
      if (jtry == MAX_TRY_ROOT - 2) {
        if (sgndef == 1)
          sigma = gl - 2.0 * spdiam * OR_EPS * nbl - 2.0 * 2.0 * pivmin;
        else
          sigma = gu + 2.0 * spdiam * OR_EPS * nbl + 2.0 * 2.0 * pivmin;
      } else if (jtry == MAX_TRY_ROOT - 1) {
        return 2;
      } else {
        sigma -= sgndef * tau;
        tau *= 2.0;
        continue;
      }
    } else {
      break;
    }
  }
  E[iend] = sigma;
  memcpy(&D[ibgn], &work[0], sizeof(double) * (size_t)nbl);
  if (nbl > 1) memcpy(&E[ibgn], &work[n], sizeof(double) * (size_t)(nbl - 1));
  if (mbl > 1) {
    int iseed[4] = {1, 1, 1, 1};
    or_dlarnv2(iseed, 2 * nbl, work);
    for (i = 0; i < nbl - 1; i++) {
      D[i + ibgn] *= 1.0 + OR_EPS * 8.0 * work[i];
      E[i + ibgn] *= 1.0 + OR_EPS * 8.0 * work[i + nbl];
    }
    D[iend] *= 1.0 + OR_EPS * 8.0 * work[2 * nbl - 1];
  }
  *sgndefp = sgndef;
  *sigmap = sigma;
  *spdiamp = spdiam;
  return 0;
}

/* mrrr_val with force_bisection: SRC/mrrr_val.c:110-639. */
/* mrrr_val (SRC/mrrr_val.c:110-639).  nthreads plays the part of the
 * reference's thread count in its route choice (SRC/mrrr_val.c:279-285,
 * 409-412): bisection is forced when nthreads > ceil(12 nvals / n); else a
 * block with more than half of its eigenvalues wanted takes dqds. */
static int or_mrrr_val(const char *jobz, const char *range, or_in_t *Ds,
                       or_val_t *Ws, or_tol_t *tol, int nthreads)
{
  int n = Ds->n, i, info = 0;
  double *D = Ds->D, *E = Ds->E, *E2, *work, *Wcopy;
  double *W = Ws->W, *Werr = Ws->Werr, *Wgap = Ws->Wgap, *gersch = Ws->gersch;
  int *iblock = Ws->iblock, *Windex = Ws->Windex, *isplit = Ds->isplit;
  int *mp = Ws->mp;
  enum { allrng = 1, valrng = 2, indrng = 3 } irange;
  double gl, gu, eold, emax, eabs, tmp1, tnorm, wl = 0, wu = 0, wlu = 0, wul = 0;
  int nwl = 0, nwu = 0, nvals, ibgn, wbgn, jbl, force_bisection = 1;

  if (range[0] == 'A' || range[0] == 'a') irange = allrng;
  else if (range[0] == 'V' || range[0] == 'v') irange = valrng;
  else irange = indrng;
  if (irange == indrng && *Ws->ilp == 1 && *Ws->iup == n) irange = allrng;

  E2 = (double *)malloc(sizeof(double) * (size_t)n);
  Wcopy = (double *)malloc(sizeof(double) * (size_t)n);
  work = (double *)malloc(sizeof(double) * (size_t)(4 * n));
  Ds->E2 = E2;

  for (i = 0; i < n; i++) E2[i] = E[i] * E[i];
  gl = D[0]; gu = D[0]; eold = 0.0; emax = 0.0;
  E[n - 1] = 0.0;
  for (i = 0; i < n; i++) {
    eabs = fabs(E[i]);
    if (eabs >= emax) emax = eabs;
    tmp1 = eabs + eold;
    gersch[2 * i] = D[i] - tmp1;
    gl = fmin(gl, gersch[2 * i]);
    gersch[2 * i + 1] = D[i] + tmp1;
    gu = fmax(gu, gersch[2 * i + 1]);
    eold = eabs;
  }
  tol->pivmin = OR_SAFMIN * fmax(1.0, emax * emax);
  Ds->spdiam = gu - gl;
  tnorm = fmax(fabs(gl), fabs(gu));
  gl = gl - 2 * tnorm * OR_EPS * n - 4 * tol->pivmin;
  gu = gu + 2 * tnorm * OR_EPS * n + 4 * tol->pivmin;
  if (irange == valrng && *Ws->vlp < gl && *Ws->vup >= gu) irange = allrng;

  or_dlarra(n, D, E, E2, tol->split, Ds->spdiam, &Ds->nsplit, isplit);

  if (irange == allrng) {
    *Ws->ilp = 1; *Ws->iup = n;
  } else if (irange == valrng) {
    int c0 = or_count_ijob1(n, D, E2, tol->pivmin, *Ws->vlp);
    int c1 = or_count_ijob1(n, D, E2, tol->pivmin, *Ws->vup);
    *Ws->ilp = c0 + 1; *Ws->iup = c1;
  }
  nvals = *Ws->iup - *Ws->ilp + 1;
  *mp = nvals;
  if (jobz[0] == 'C' || jobz[0] == 'c') { info = 0; goto done; }
  force_bisection = (double)nthreads > ceil(12.0 * nvals / (double)n);

  if (irange == indrng) {
    int itmax = (int)((or_log(tnorm + tol->pivmin) - or_log(tol->pivmin)) / or_log(2.0) + 2);
    double atoli = 2 * (2 * OR_SAFMIN + 2 * tol->pivmin);
    double a1 = gl, b1 = gu, a2 = gl, b2 = gu;
    int na1 = -1, nb1 = n + 1, na2 = -1, nb2 = n + 1;
    or_ijob3(n, D, E2, tol->pivmin, atoli, tol->RQtol, itmax, *Ws->ilp - 1, gl, &a1, &b1, &na1, &nb1);
    or_ijob3(n, D, E2, tol->pivmin, atoli, tol->RQtol, itmax, *Ws->iup, gu, &a2, &b2, &na2, &nb2);
    wl = a1; wlu = b1; nwl = na1;
    wul = a2; wu = b2; nwu = nb2;
    *Ws->vlp = wl; *Ws->vup = wu;
  } else if (irange == valrng) {
    wl = *Ws->vlp; wu = *Ws->vup;
  } else {
    wl = gl; wu = gu; *Ws->vlp = gl; *Ws->vup = gu;
  }

  *mp = 0; ibgn = 0; wbgn = 0;
  for (jbl = 0; jbl < Ds->nsplit; jbl++) {
    int iend = isplit[jbl] - 1, nbl = iend - ibgn + 1, ilow, iupp, mbl, wend, m_bl;
    double bgl, bgu, spdiam, sigma;
    if (nbl == 1) {
      if (irange == allrng || (irange == valrng && D[ibgn] > wl && D[ibgn] <= wu) ||
          (irange == indrng && (D[ibgn] + tol->pivmin) > wl && (D[ibgn] - tol->pivmin) <= wu)) {
        W[*mp] = D[ibgn]; Wcopy[*mp] = D[ibgn]; Werr[*mp] = 0.0;
        iblock[*mp] = jbl + 1; Windex[*mp] = 1;
        (*mp)++; wbgn++;
      }
      E[iend] = 0.0;
      ibgn = iend + 1;
      continue;
    }
    bgl = D[ibgn]; bgu = D[ibgn];
    for (i = ibgn; i <= iend; i++) { bgl = fmin(bgl, gersch[2 * i]); bgu = fmax(bgu, gersch[2 * i + 1]); }
    spdiam = bgu - bgl;
    bgl = bgl - 2 * tnorm * OR_EPS * nbl - 4 * tol->pivmin;
    bgu = bgu + 2 * tnorm * OR_EPS * nbl + 4 * tol->pivmin;
    if (irange == allrng) {
      ilow = 1; iupp = nbl;
    } else {
      ilow = or_count_ijob1(nbl, &D[ibgn], &E2[ibgn], tol->pivmin, fmax(wl, bgl)) + 1;
      iupp = or_count_ijob1(nbl, &D[ibgn], &E2[ibgn], tol->pivmin, fmin(wu, bgu));
    }
    mbl = iupp - ilow + 1;
    *mp += mbl;
    if (mbl == 0) { E[iend] = 0.0; ibgn = iend + 1; continue; }
    wend = wbgn + mbl - 1;
    for (i = wbgn; i <= wend; i++) iblock[i] = jbl + 1;
    info = or_dlarrd_block(nbl, ilow, iupp, &gersch[2 * ibgn], tol->bsrtol, &D[ibgn],
                           &E2[ibgn], tol->pivmin, &m_bl, &W[wbgn], &Werr[wbgn], &Windex[wbgn]);
    if (info != 0 && info != 1) { info = 2; goto done; }   /* TOOFEW or bad bounds */
    info = 0;
    for (i = wbgn; i <= wend; i++) Wcopy[i] = W[i];
    for (i = wbgn; i < wend; i++) Wgap[i] = fmax(0.0, (W[i + 1] - Werr[i + 1]) - (W[i] + Werr[i]));
    Wgap[wend] = fmax(0.0, wu - (W[wend] + Werr[wend]));

    {
      const int useDQDS = mbl > 0.5 * nbl && !force_bisection;
      const int allrng_no_bisec = irange == allrng && !force_bisection;
      int sgndef = 1;
      if (or_root_rrr(allrng_no_bisec, useDQDS, ibgn, iend, wbgn, wend, ilow, iupp, bgl, bgu,
                      Ds, Ws, tol, work, &sgndef, &sigma, &spdiam)) {
        info = 2; goto done;
      }
      if (useDQDS) {
        /* all eigenvalues of the definite root representation by dqds:
         * SRC/mrrr_val.c:459-506 (the tolerance's log is or_log) */
        const double rtol = 4.0 * or_log((double)nbl) * OR_EPS;
        int j = ibgn, je = wbgn, qinfo = 0;
        for (i = 0; i < nbl - 1; i++) {
          work[2 * i] = fabs(D[j]);
          work[2 * i + 1] = E[j] * E[j] * work[2 * i];
          j++;
        }
        work[2 * (nbl - 1)] = fabs(D[iend]);
        work[2 * (nbl - 1) + 1] = 0.0;
        or_dlasq2(nbl, work, &qinfo);
        if (qinfo != 0) { info = 2; goto done; }
        for (i = ilow; i <= iupp; i++, je++) {
          W[je] = sgndef > 0 ? work[nbl - i] : -work[i - 1];
          iblock[je] = jbl + 1;
          Windex[je] = i;
        }
        for (i = wbgn; i <= wend; i++) Werr[i] = rtol * fabs(W[i]);
        for (i = wbgn; i < wend; i++) Wgap[i] = fmax(0.0, (W[i + 1] - Werr[i + 1]) - (W[i] + Werr[i]));
        Wgap[wend] = fmax(0.0, (*Ws->vup - sigma) - (W[wend] + Werr[wend]));
        ibgn = iend + 1;
        wbgn = wend + 1;
        continue;
      }
    }
    /* refine_eigval_approx, unchunked branch: SRC/mrrr_val.c:992-1001, 1070-1082 */
    for (i = wbgn; i <= wend; i++) { W[i] -= sigma; Werr[i] += fabs(W[i]) * OR_EPS; }
    {
      double *DE2 = work + 2 * n;
      int *iwork = (int *)malloc(sizeof(int) * (size_t)(2 * nbl));
      int rinfo;
      for (i = ibgn; i < iend; i++) DE2[i] = D[i] * E[i] * E[i];
      or_dlarrb(nbl, &D[ibgn], &DE2[ibgn], ilow, iupp, tol->rtol1, tol->rtol2, ilow - 1,
                &W[wbgn], &Wgap[wbgn], &Werr[wbgn], work, iwork, tol->pivmin, spdiam, nbl, &rinfo);
      free(iwork);
      Wgap[wend] = fmax(0.0, (*Ws->vup - sigma) - (W[wend] + Werr[wend]));
    }
    ibgn = iend + 1;
    wbgn = wend + 1;
  }

  /* Discard surplus eigenvalues of range I: SRC/mrrr_val.c:520-626. */
  if (*mp > nvals && irange == indrng) {
    int idiscl = *Ws->ilp - 1 - nwl, idiscu = nwu - *Ws->iup, im, je, jee;
    if (idiscl > 0) {
      im = 0;
      for (je = 0; je < *mp; je++) {
        if (Wcopy[je] < wlu && idiscl > 0) {
          idiscl--;
        } else {
          W[im] = W[je]; Wcopy[im] = Wcopy[je]; Werr[im] = Werr[je]; Wgap[im] = Wgap[je];
          Windex[im] = Windex[je]; iblock[im] = iblock[je]; im++;
        }
      }
      *mp = im;
    }
    if (idiscu > 0) {
      im = *mp;
      for (je = *mp - 1; je >= 0; je--) {
        if (Wcopy[je] > wul && idiscu > 0) {
          idiscu--;
        } else {
          im--;
          W[im] = W[je]; Wcopy[im] = Wcopy[je]; Werr[im] = Werr[je]; Wgap[im] = Wgap[je];
          Windex[im] = Windex[je]; iblock[im] = iblock[je];
        }
      }
      jee = 0;
      for (je = im; je < *mp; je++) {
        W[jee] = W[je]; Wcopy[jee] = Wcopy[je]; Werr[jee] = Werr[je]; Wgap[jee] = Wgap[je];
        Windex[jee] = Windex[je]; iblock[jee] = iblock[je]; jee++;
      }
      *mp -= im;
    }
    if (idiscl > 0 || idiscu > 0) {
      int jdisc, iw;
      double wkill;
      if (idiscl > 0) {
        wkill = wu;
        for (jdisc = 0; jdisc < idiscl; jdisc++) {
          iw = -1;
          for (je = 0; je < *mp; je++)
            if (iblock[je] != 0 && (Wcopy[je] < wkill || iw == -1)) { iw = je; wkill = Wcopy[je]; }
          iblock[iw] = 0;
        }
      }
      if (idiscu > 0) {
        wkill = wl;
        for (jdisc = 0; jdisc < idiscu; jdisc++) {
          iw = -1;
          for (je = 0; je < *mp; je++)
            if (iblock[je] != 0 && (Wcopy[je] > wkill || iw == -1)) { iw = je; wkill = Wcopy[je]; }
          iblock[iw] = 0;
        }
      }
      im = 0;
      for (je = 0; je < *mp; je++) {
        if (iblock[je] != 0) {
          W[im] = W[je]; Wcopy[im] = Wcopy[je]; Werr[im] = Werr[je]; Wgap[im] = Wgap[je];
          Windex[im] = Windex[je]; iblock[im] = iblock[je]; im++;
        }
      }
      *mp = im;
    }
  }
  Ws->m = *mp;
  if (*mp < nvals) info = 3;

done:
  free(Wcopy);
  free(work);
  return info;
}

/* ---- eigenvector stage ---------------------------------------------------- */

typedef struct {
  int begin, end, depth, bl_begin, bl_end, bl_W_begin, bl_W_end;
  double bl_spdiam, lgap;
  double *D, *L;          /* parent representation (rows bl_begin..bl_end) */
  int owns;               /* D/L were allocated for this task */
} or_task_t;

typedef struct {
  or_task_t *v;
  int head, tail, cap;
} or_queue_t;

static void or_push(or_queue_t *q, or_task_t t)
{
  if (q->tail == q->cap) {
    q->cap = q->cap ? 2 * q->cap : 64;
    q->v = (or_task_t *)realloc(q->v, sizeof(or_task_t) * (size_t)q->cap);
  }
  q->v[q->tail++] = t;
}

typedef struct {
  int n, ldz;
  double *Z;
  int *Zsupp, *Zindex;
} or_vec_t;

/* One singleton: SRC/process_singleton.c:65-317 for a task of size 1. */
static void or_singleton(int i, const or_task_t *sng, const double *D,
                         const double *L, const double *DL, const double *DLL,
                         or_val_t *Ws, or_vec_t *Zs, or_tol_t *tol,
                         double *work, int *iwork)
{
  int bl_begin = sng->bl_begin, bl_end = sng->bl_end;
  int bl_size = bl_end - bl_begin + 1, n = Zs->n, ldz = Zs->ldz;
  double *W = Ws->W, *Werr = Ws->Werr, *Wgap = Ws->Wgap, *Wshifted = Ws->Wshifted;
  int *Windex = Ws->Windex, *isuppZ = Zs->Zsupp;
  double *Zc;
  double pivmin = tol->pivmin, twoeps = 2 * OR_EPS, RQtol = 2 * OR_EPS;
  double tolr = 4.0 * or_log((double)bl_size) * OR_EPS;
  double lambda, left, right, lgap, rgap, gap, gaptol, savedgap, tmp;
  double residual = 0, bstres = 0, bstw = 0, RQcorr = 0, ztz, norminv = 0, mingma, sigma;
  int i_local, r, k, itmp, usedBS, usedRQ, needBS, wantNC, step2II, negcount = 0;
  int i_supmn, i_supmx, sgndef, i_Zfrom, i_Zto, info;
  size_t zind = (size_t)Zs->Zindex[i];

  Zc = &Zs->Z[zind * (size_t)ldz];
  if (bl_size == 1) {
    memset(Zc, 0, sizeof(double) * (size_t)n);
    Zc[bl_begin] = 1.0;
    isuppZ[2 * zind] = bl_begin + 1;
    isuppZ[2 * zind + 1] = bl_begin + 1;
    return;
  }
  lambda = Wshifted[i];
  left = Wshifted[i] - Werr[i];
  right = Wshifted[i] + Werr[i];
  i_local = Windex[i];
  r = 0;
  if (i == bl_begin) lgap = OR_EPS * fmax(fabs(left), fabs(right));
  else if (i == sng->begin) lgap = sng->lgap;
  else lgap = Wgap[i - 1];
  if (i == bl_end) rgap = OR_EPS * fmax(fabs(left), fabs(right));
  else rgap = Wgap[i];
  gap = fmin(lgap, rgap);
  gaptol = (i == bl_begin || i == bl_end) ? 0.0 : gap * OR_EPS;
  i_supmn = bl_size; i_supmx = 1;
  savedgap = Wgap[i];
  Wgap[i] = gap;
  usedBS = 0; usedRQ = 0; needBS = 0;
  memset(Zc, 0, sizeof(double) * (size_t)n);
  for (k = 1; k <= MAXITER; k++) {
    if (needBS) {
      usedBS = 1;
      itmp = r;
      tmp = Wgap[i];
      Wgap[i] = 0.0;
      or_dlarrb(bl_size, D, DLL, i_local, i_local, 0.0, twoeps, Windex[i] - 1,
                &Wshifted[i], &Wgap[i], &Werr[i], work, iwork, pivmin, sng->bl_spdiam,
                itmp, &info);
      Wgap[i] = tmp;
      lambda = Wshifted[i];
      r = 0;
    }
    wantNC = !usedBS;
    or_dlar1v(bl_size, 1, bl_size, lambda, D, L, DL, DLL, pivmin, gaptol, Zc + bl_begin,
              wantNC, &negcount, &ztz, &mingma, &r, &isuppZ[2 * zind], &norminv,
              &residual, &RQcorr, work);
    if (k == 1 || residual < bstres) { bstres = residual; bstw = lambda; }
    i_supmn = imin(i_supmn, isuppZ[2 * zind]);
    i_supmx = imax(i_supmx, isuppZ[2 * zind + 1]);
    if (!usedBS && residual > tolr * gap && fabs(RQcorr) > RQtol * fabs(lambda)) {
      sgndef = (i_local <= negcount) ? -1 : 1;
      if (RQcorr * sgndef >= 0.0 && lambda + RQcorr <= right && lambda + RQcorr >= left) {
        usedRQ = 1;
        if (sgndef == 1) left = lambda; else right = lambda;
        Wshifted[i] = 0.5 * (left + right);
        lambda += RQcorr;
      } else {
        needBS = 1;
      }
      if (right - left < RQtol * fabs(lambda)) usedBS = 1;
      else if (k == MAXITER - 1) needBS = 1;
    } else {
      break;
    }
  }
  step2II = (usedRQ && usedBS && (bstres <= residual));
  if (step2II) {
    lambda = bstw;
    or_dlar1v(bl_size, 1, bl_size, lambda, D, L, DL, DLL, pivmin, gaptol, Zc + bl_begin,
              wantNC, &negcount, &ztz, &mingma, &r, &isuppZ[2 * zind], &norminv,
              &residual, &RQcorr, work);
  }
  Wshifted[i] = lambda;
  isuppZ[2 * zind] += bl_begin;
  isuppZ[2 * zind + 1] += bl_begin;
  i_Zfrom = isuppZ[2 * zind] - 1;
  i_Zto = isuppZ[2 * zind + 1] - 1;
  i_supmn += bl_begin - 1;
  i_supmx += bl_begin - 1;
  for (k = i_supmn; k < i_Zfrom; k++) Zc[k] = 0.0;
  for (k = i_Zto + 1; k <= i_supmx; k++) Zc[k] = 0.0;
  for (k = i_Zfrom; k <= i_Zto; k++) Zc[k] *= norminv;
  sigma = L[bl_size - 1];
  W[i] = lambda + sigma;
  (void)savedgap;  /* size-1 task: Wgap[i] keeps gap (process_singleton.c:308) */
}

/* create_subtasks with one singleton per S-task: SRC/process_cluster.c:438-629.
 * The whole cluster is classified first and its singletons run afterwards,
 * as if every S-task were enqueued; a singleton rewrites the gap to its right
 * (SRC/process_singleton.c:169-170), so running one inline would change the
 * left gap a later sibling cluster records. */
static void or_subtasks(const or_task_t *cl, const double *D, const double *L,
                        const double *DL, const double *DLL, or_queue_t *cq,
                        or_val_t *Ws, or_vec_t *Zs, or_tol_t *tol,
                        double *work, int *iwork)
{
  int cl_begin = cl->begin, cl_end = cl->end, depth = cl->depth;
  int bl_size = cl->bl_end - cl->bl_begin + 1, i, k, ns = 0;
  double *Wgap = Ws->Wgap, *Wshifted = Ws->Wshifted;
  int new_first = cl_begin, new_last, new_size;
  or_task_t *sng = (or_task_t *)malloc(sizeof(or_task_t) * (size_t)(cl_end - cl_begin + 1));
  for (i = cl_begin; i <= cl_end; i++) {
    if (i == cl_end) new_last = i;
    else if (Wgap[i] >= MIN_RELGAP * fabs(Wshifted[i])) new_last = i;
    else continue;
    new_size = new_last - new_first + 1;
    if (new_size == 1) {
      or_task_t s = *cl;
      s.begin = new_first; s.end = new_first; s.depth = depth + 1;
      s.lgap = (new_first == cl_begin) ? cl->lgap : Wgap[new_first - 1];
      s.owns = 0;
      sng[ns++] = s;
    } else if (depth == 0 && new_size > 3) {
      int cl_first = new_first, cl_last = new_last;
      double avggap = cl->bl_spdiam / (bl_size - 1);
      for (k = new_first + 1; k < new_last; k++) {
        or_task_t c;
        if (k == new_last - 1) cl_last = new_last;
        else if (k != cl_first && Wgap[k] > 2.0 * avggap) cl_last = k;
        else continue;
        c = *cl;
        c.begin = cl_first; c.end = cl_last; c.depth = depth + 1;
        c.lgap = (cl_first == cl_begin) ? cl->lgap : Wgap[cl_first - 1];
        c.D = (double *)D; c.L = (double *)L; c.owns = 0;
        or_push(cq, c);
        cl_first = k + 1;
      }
    } else {
      or_task_t c = *cl;
      c.begin = new_first; c.end = new_last; c.depth = depth + 1;
      c.lgap = (new_first == cl_begin) ? cl->lgap : Wgap[new_first - 1];
      if (depth == 0) {
        c.D = (double *)D; c.L = (double *)L; c.owns = 0;
      } else {
        c.D = (double *)malloc(sizeof(double) * (size_t)bl_size);
        c.L = (double *)malloc(sizeof(double) * (size_t)bl_size);
        memcpy(c.D, D, sizeof(double) * (size_t)bl_size);
        memcpy(c.L, L, sizeof(double) * (size_t)bl_size);
        c.owns = 1;
      }
      or_push(cq, c);
    }
    new_first = i + 1;
  }
  for (k = 0; k < ns; k++)
    or_singleton(sng[k].begin, &sng[k], D, L, DL, DLL, Ws, Zs, tol, work, iwork);
  free(sng);
}

/* One cluster task: SRC/process_cluster.c:75-433 (never split into R-tasks). */
static int or_cluster(or_task_t *cl, or_queue_t *cq, or_val_t *Ws, or_vec_t *Zs,
                      or_tol_t *tol, const double *gersch, double *work, int *iwork)
{
  int cl_begin = cl->begin, cl_end = cl->end, cl_size = cl_end - cl_begin + 1;
  int bl_size = cl->bl_end - cl->bl_begin + 1, depth = cl->depth, i, k, info;
  double *W = Ws->W, *Werr = Ws->Werr, *Wgap = Ws->Wgap, *Wshifted = Ws->Wshifted;
  int *Windex = Ws->Windex;
  double *D, *L, *DL, *DLL, sigma;
  DL = (double *)malloc(sizeof(double) * (size_t)bl_size);
  DLL = (double *)malloc(sizeof(double) * (size_t)bl_size);
  if (depth == 0) {
    D = cl->D; L = cl->L;
  } else {
    double *Dp = cl->D, *Lp = cl->L, tau, fudge, savegap, lgap, rgap;
    int p, offset;
    D = (double *)malloc(sizeof(double) * (size_t)bl_size);
    L = (double *)malloc(sizeof(double) * (size_t)bl_size);
    for (i = 0; i < bl_size - 1; i++) { double t = Dp[i] * Lp[i]; DL[i] = t; DLL[i] = t * Lp[i]; }
    for (k = 0; k < 2; k++) {
      int ix = (k == 0) ? cl_begin : cl_end;
      p = Windex[ix];
      savegap = Wgap[ix];
      Wgap[ix] = 0.0;
      offset = Windex[cl_begin] - 1;
      or_dlarrb(bl_size, Dp, DLL, p, p, tol->RQtol, tol->RQtol, offset, &Wshifted[cl_begin],
                &Wgap[cl_begin], &Werr[cl_begin], work, iwork, tol->pivmin, cl->bl_spdiam,
                bl_size, &info);
      if (k == 0)
        Wgap[cl_begin] = fmax(0, (Wshifted[cl_begin + 1] - Werr[cl_begin + 1]) -
                                     (Wshifted[cl_begin] + Werr[cl_begin]));
      else
        Wgap[cl_end] = savegap;
    }
    lgap = cl->lgap;
    rgap = Wgap[cl_end];
    or_dlarrf(bl_size, Dp, Lp, DL, 1, cl_size, &Wshifted[cl_begin], &Wgap[cl_begin],
              &Werr[cl_begin], cl->bl_spdiam, lgap, rgap, tol->pivmin, &tau, D, L, work, &info);
    L[bl_size - 1] = Lp[bl_size - 1] + tau;
    for (k = cl_begin; k <= cl_end; k++) {
      fudge = 3.0 * OR_EPS * fabs(Wshifted[k]);
      Wshifted[k] -= tau;
      fudge += 4.0 * OR_EPS * fabs(Wshifted[k]);
      Werr[k] += fudge;
    }
    if (cl->owns) { free(cl->D); free(cl->L); cl->owns = 0; }
  }
  for (i = 0; i < bl_size - 1; i++) { double t = D[i] * L[i]; DL[i] = t; DLL[i] = t * L[i]; }

  if (depth == 0) {
    int bl_begin = cl->bl_begin, bl_end = cl->bl_end, mbl = cl->bl_W_end - cl->bl_W_begin + 1;
    double gl = gersch[2 * bl_begin], gu = gersch[2 * bl_begin + 1];
    for (i = bl_begin + 1; i < bl_end; i++) { gl = fmin(gl, gersch[2 * i]); gu = fmax(gu, gersch[2 * i + 1]); }
    cl->bl_spdiam = gu - gl;
    sigma = L[bl_size - 1];
    memcpy(&Wshifted[cl_begin], &W[cl_begin], sizeof(double) * (size_t)mbl);
    for (i = 0; i < mbl; i++) W[cl_begin + i] += sigma;
  } else {
    int p = Windex[cl_begin], q = Windex[cl_end], offset = p - 1;
    double savegap = 0;
    if (p == q) { savegap = Wgap[cl_begin]; Wgap[cl_begin] = 0.0; }
    or_dlarrb(bl_size, D, DLL, p, q, tol->rtol1, tol->rtol2, offset, &Wshifted[cl_begin],
              &Wgap[cl_begin], &Werr[cl_begin], work, iwork, tol->pivmin, cl->bl_spdiam,
              bl_size, &info);
    if (p == q) Wgap[cl_begin] = savegap;
    sigma = L[bl_size - 1];
    for (k = cl_begin; k <= cl_end; k++) W[k] = Wshifted[k] + sigma;
  }
  or_subtasks(cl, D, L, DL, DLL, cq, Ws, Zs, tol, work, iwork);
  /* Child clusters at depth 0 point at the root (not owned); deeper ones got
   * their own copies, so D/L of this level can be released now. */
  if (depth > 0) { free(D); free(L); }
  free(DL); free(DLL);
  return 0;
}

/* Output column of each eigenvalue (SRC/mrrr_vec.c:380-416).  The reference
 * sorts with a comparator that orders by local index inside a block and by
 * value across blocks.  Here the value used across blocks is the running
 * maximum of the block's values in local-index order, which orders a block's
 * eigenvalues by local index even where rounding makes two neighbours
 * non-monotone, and equals the reference's order wherever that order is
 * well defined. */
typedef struct { double key; int ilocal, iblock, ind; } or_sort_t;
static int or_cmp_key(const void *a, const void *b)
{
  const or_sort_t *x = (const or_sort_t *)a, *y = (const or_sort_t *)b;
  if (x->key < y->key) return -1;
  if (x->key > y->key) return 1;
  if (x->ilocal != y->ilocal) return x->ilocal < y->ilocal ? -1 : 1;
  if (x->iblock != y->iblock) return x->iblock < y->iblock ? -1 : 1;
  return 0;
}

static void or_init_zindex(or_in_t *Ds, or_val_t *Ws, int *Zindex)
{
  int m = Ws->m, i;
  or_sort_t *a = (or_sort_t *)malloc(sizeof(or_sort_t) * (size_t)(m > 0 ? m : 1));
  double runmax = 0;
  for (i = 0; i < m; i++) {
    int iblk = Ws->iblock[i];
    double sigma = Ds->E[Ds->isplit[iblk - 1] - 1];
    double lam = Ws->W[i] + sigma;
    if (i == 0 || Ws->iblock[i - 1] != iblk) runmax = lam;
    else runmax = fmax(runmax, lam);
    a[i].key = runmax; a[i].ilocal = Ws->Windex[i]; a[i].iblock = iblk; a[i].ind = i;
  }
  qsort(a, (size_t)m, sizeof(or_sort_t), or_cmp_key);
  for (i = 0; i < m; i++) Zindex[a[i].ind] = i;
  free(a);
}

/* mrrr_vec: SRC/mrrr_vec.c:75-374, tasks drained in FIFO order. */
static int or_mrrr_vec(or_in_t *Ds, or_val_t *Ws, or_vec_t *Zs, or_tol_t *tol)
{
  int n = Ds->n, m = Ws->m, j, begin = 0, Wbegin = 0, rc = 0;
  double *work = (double *)malloc(sizeof(double) * (size_t)(4 * n));
  int *iwork = (int *)malloc(sizeof(int) * (size_t)(2 * n));
  or_queue_t cq = {0, 0, 0, 0};
  Ws->Wshifted = (double *)malloc(sizeof(double) * (size_t)n);
  or_init_zindex(Ds, Ws, Zs->Zindex);

  for (j = 0; j < Ds->nsplit; j++) {
    int end = Ds->isplit[j] - 1, Wend = Wbegin - 1, nbl;
    double sigma = Ds->E[end];
    while (Wend < m - 1 && Ws->iblock[Wend + 1] == j + 1) Wend++;
    if (Wend < Wbegin) { begin = end + 1; continue; }
    nbl = end - begin + 1;
    {
      or_task_t t;
      t.begin = Wbegin; t.end = Wend; t.depth = 0; t.bl_begin = begin; t.bl_end = end;
      t.bl_W_begin = Wbegin; t.bl_W_end = Wend; t.bl_spdiam = 0.0;
      t.D = &Ds->D[begin]; t.L = &Ds->E[begin]; t.owns = 0;
      if (nbl == 1) {
        t.lgap = 0.0;
        or_singleton(Wbegin, &t, t.D, t.L, NULL, NULL, Ws, Zs, tol, work, iwork);
      } else {
        t.lgap = fmax(0.0, (Ws->W[Wbegin] + sigma) - Ws->Werr[Wbegin] - (*Ws->vlp));
        or_push(&cq, t);
      }
    }
    begin = end + 1;
    Wbegin = Wend + 1;
  }
  while (cq.head < cq.tail) {
    or_task_t t = cq.v[cq.head++];
    if (t.depth >= DEPTH_CAP) { rc = 2; if (t.owns) { free(t.D); free(t.L); } continue; }
    or_cluster(&t, &cq, Ws, Zs, tol, Ws->gersch, work, iwork);
  }
  free(cq.v);
  free(Ws->Wshifted);
  free(work);
  free(iwork);
  return rc;
}

/* refine_to_highrac: SRC/mrrr.c:452-520. */
static void or_refine_highrac(double *D, double *E2, or_in_t *Ds, or_val_t *Ws,
                              or_tol_t *tol)
{
  int n = Ds->n, j, i, begin = 0, Wbegin = 0;
  double *work = (double *)malloc(sizeof(double) * (size_t)(2 * n));
  int *iwork = (int *)malloc(sizeof(int) * (size_t)(2 * n));
  for (j = 0; j < Ds->nsplit; j++) {
    int end = Ds->isplit[j] - 1, nbl = end - begin + 1, mbl = 0, ilow = n, iupp = 1, info;
    for (i = Wbegin; i < *Ws->mp; i++) {
      if (Ws->iblock[i] == j + 1) { mbl++; ilow = imin(ilow, Ws->Windex[i]); iupp = imax(iupp, Ws->Windex[i]); }
      else break;
    }
    if (mbl == 0) { begin = end + 1; continue; }
    or_dlarrj(nbl, &D[begin], &E2[begin], ilow, iupp, 4 * OR_EPS, ilow - 1, &Ws->W[Wbegin],
              &Ws->Werr[Wbegin], work, iwork, tol->pivmin, Ds->spdiam, &info);
    begin = end + 1;
    Wbegin = Wbegin + mbl;
  }
  free(work);
  free(iwork);
}

static int or_cmp_double(const void *a, const void *b)
{
  double x = *(const double *)a, y = *(const double *)b;
  return (x < y) ? -1 : (x > y) ? 1 : 0;
}

/* mrrr: SRC/mrrr.c:87-296 (no dstemr route; see mr3_oracle.h). */
int or_mrrr(const char *jobz, const char *range, int *np, double *D, double *E,
            double *vlp, double *vup, int *ilp, int *iup, int *tryracp, int *mp,
            double *W, double *Z, int *ldz, int *Zsupp)
{
  int n = *np, i, info, rc = 0;
  int onlyW = (jobz[0] == 'N' || jobz[0] == 'n');
  int wantZ = (jobz[0] == 'V' || jobz[0] == 'v');
  int cntval = (jobz[0] == 'C' || jobz[0] == 'c');
  int alleig = (range[0] == 'A' || range[0] == 'a');
  int valeig = (range[0] == 'V' || range[0] == 'v');
  int indeig = (range[0] == 'I' || range[0] == 'i');
  double scale = 1.0, *Dcopy = NULL, *E2copy = NULL;
  or_in_t Ds;
  or_val_t Ws;
  or_vec_t Zs;
  or_tol_t tol;

  if (!(onlyW || wantZ || cntval)) return 1;
  if (!(alleig || valeig || indeig)) return 1;
  if (n <= 0) return 1;
  if (valeig) { if (*vup <= *vlp) return 1; }
  else if (indeig) { if (*ilp < 1 || *ilp > n || *iup < *ilp || *iup > n) return 1; }
  if (cntval) {
    if (alleig) { *mp = n; return 0; }
    if (indeig) { *mp = *iup - *ilp + 1; return 0; }
  }
  if (wantZ && *ldz < n) return 1;

  if (n == 1) {
    int take = alleig || indeig || (valeig && D[0] > *vlp && D[0] <= *vup);
    *mp = take ? 1 : 0;
    if (cntval) return 0;
    if (take) {
      W[0] = D[0];
      if (wantZ) { Z[0] = 1.0; Zsupp[0] = 1; Zsupp[1] = 1; }
    }
    return 0;
  }

  memset(&Ds, 0, sizeof(Ds)); memset(&Ws, 0, sizeof(Ws));
  Ws.Werr = (double *)malloc(sizeof(double) * (size_t)n);
  Ws.Wgap = (double *)malloc(sizeof(double) * (size_t)n);
  Ws.gersch = (double *)malloc(sizeof(double) * (size_t)(2 * n));
  Ws.iblock = (int *)calloc((size_t)n, sizeof(int));
  Ws.Windex = (int *)malloc(sizeof(int) * (size_t)n);
  Ds.isplit = (int *)malloc(sizeof(int) * (size_t)n);
  Zs.Zindex = (int *)malloc(sizeof(int) * (size_t)n);
  Ds.n = n; Ds.D = D; Ds.E = E;
  Ws.n = n; Ws.vlp = vlp; Ws.vup = vup; Ws.ilp = ilp; Ws.iup = iup; Ws.mp = mp; Ws.W = W;
  Zs.n = n; Zs.ldz = wantZ ? *ldz : n; Zs.Z = Z; Zs.Zsupp = Zsupp;

  /* scale_matrix: SRC/mrrr.c:325-365 */
  {
    double smlnum = DBL_MIN / DBL_EPSILON, bignum = 1.0 / smlnum;
    double rmin = sqrt(smlnum), rmax = fmin(sqrt(bignum), 1.0 / sqrt(sqrt(DBL_MIN)));
    double tn = or_dlanst_m(n, D, E);
    if (tn > 0 && tn < rmin) scale = rmin / tn;
    else if (tn > rmax) scale = rmax / tn;
    if (scale != 1.0) {
      for (i = 0; i < n; i++) D[i] *= scale;
      for (i = 0; i < n - 1; i++) E[i] *= scale;
      if (valeig) { *vlp *= scale; *vup *= scale; }
    }
  }
  info = (*tryracp) ? or_dlarrr(n, D, E) : -1;
  if (info == 0) {
    tol.split = DBL_EPSILON;
    Dcopy = (double *)malloc(sizeof(double) * (size_t)n);
    E2copy = (double *)malloc(sizeof(double) * (size_t)n);
    memcpy(Dcopy, D, sizeof(double) * (size_t)n);
    for (i = 0; i < n - 1; i++) E2copy[i] = E[i] * E[i];
  } else {
    tol.split = -DBL_EPSILON;
    *tryracp = 0;
  }
  if (!wantZ) {
    tol.rtol1 = 4.0 * DBL_EPSILON;
    tol.rtol2 = 4.0 * DBL_EPSILON;
  } else {
    tol.rtol1 = sqrt(DBL_EPSILON);
    tol.rtol1 = fmin(tol.rtol1, 1e-2 * MIN_RELGAP);
    tol.rtol2 = tol.rtol1 * 5.0E-3;
    tol.rtol2 = fmin(tol.rtol2, MIN_RELGAP * 5.0E-6);
    tol.rtol2 = fmax(tol.rtol2, 4.0 * DBL_EPSILON);
  }
  tol.bsrtol = fmin(MIN_RELGAP * 1.0E-2, sqrt(DBL_EPSILON));
  tol.RQtol = 2.0 * DBL_EPSILON;

  {
    /* the thread count of the reference's route choice: MR3_NTHREADS, as
     * the product reads it; unset, bisection (a GPU's parallelism) */
    const char *ev = getenv("MR3_NTHREADS");
    const int nthreads = (ev && *ev) ? atoi(ev) : 1 << 30;
    info = or_mrrr_val(jobz, range, &Ds, &Ws, &tol, nthreads);
  }
  if (info != 0) { rc = 2; goto out; }
  if (cntval) goto out;
  if (wantZ) {
    if (or_mrrr_vec(&Ds, &Ws, &Zs, &tol) != 0) { rc = 2; goto out; }
  } else {
    for (i = 0; i < *mp; i++) W[i] += E[Ds.isplit[Ws.iblock[i] - 1] - 1];
  }
  if (*tryracp) or_refine_highrac(Dcopy, E2copy, &Ds, &Ws, &tol);
  if (scale != 1.0) {
    double inv = 1.0 / scale;
    *vlp *= inv; *vup *= inv;
    for (i = 0; i < *mp; i++) W[i] *= inv;
  }
  if (wantZ) {
    /* sort_eigenpairs: SRC/mrrr.c:525-588 */
    int m = Ws.m, sorted = 0;
    double *Wt = (double *)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
    double *col = (double *)malloc(sizeof(double) * (size_t)n);
    for (i = 0; i < m; i++) Wt[Zs.Zindex[i]] = W[i];
    memcpy(W, Wt, sizeof(double) * (size_t)m);
    while (!sorted) {
      sorted = 1;
      for (i = 0; i < m - 1; i++) {
        if (W[i] > W[i + 1]) {
          double t = W[i]; int it;
          size_t a = (size_t)i * (size_t)*ldz, b = (size_t)(i + 1) * (size_t)*ldz;
          sorted = 0;
          W[i] = W[i + 1]; W[i + 1] = t;
          it = Zsupp[2 * i]; Zsupp[2 * i] = Zsupp[2 * (i + 1)]; Zsupp[2 * (i + 1)] = it;
          it = Zsupp[2 * i + 1]; Zsupp[2 * i + 1] = Zsupp[2 * (i + 1) + 1]; Zsupp[2 * (i + 1) + 1] = it;
          memcpy(col, &Z[a], sizeof(double) * (size_t)n);
          memcpy(&Z[a], &Z[b], sizeof(double) * (size_t)n);
          memcpy(&Z[b], col, sizeof(double) * (size_t)n);
        }
      }
    }
    free(Wt); free(col);
  } else {
    qsort(W, (size_t)*mp, sizeof(double), or_cmp_double);
  }
out:
  free(Ws.Werr); free(Ws.Wgap); free(Ws.gersch); free(Ws.iblock); free(Ws.Windex);
  free(Ds.isplit); free(Zs.Zindex); free(Ds.E2);
  free(Dcopy); free(E2copy);
  return rc;
}

/* ------------------------------------------------------------------------
 * dqds: all eigenvalues of a positive definite L D L^T to high relative
 * accuracy (LAPACK 3.2.2 dlasq2-dlasq6, vendored as SRC/LAPACK/odsq2.f -
 * odsq6.f; the reference calls it at SRC/mrrr_val.c:464-477).  Z is the qd
 * array in Fortran's 1-based numbering, Zq(i) = z[i-1].  IEEE arithmetic is
 * assumed (odsq2.f's IEEE flag from ilaenv 10/11 is true on this hardware);
 * MIN and MAX propagate a NaN so that dlasq3's NaN test sees it.
 * ------------------------------------------------------------------------ */
#define Zq(i) z[(i) - 1]

static double or_fmin2(double a, double b) { return (a != a || b != b) ? NAN : (a < b ? a : b); }
static double or_fmax2(double a, double b) { return (a != a || b != b) ? NAN : (a > b ? a : b); }

/* odsq5.f: one dqds transform with shift tau (IEEE form). */
static void or_dlasq5(int i0, int n0, double *z, int pp, double tau, double *dmin,
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
      *dmin = or_fmin2(*dmin, d);
      Zq(j4) = Zq(j4 - 1) * temp;
      emin = or_fmin2(Zq(j4), emin);
    }
  } else {
    for (j4 = 4 * i0; j4 <= 4 * (n0 - 3); j4 += 4) {
      Zq(j4 - 3) = d + Zq(j4);
      temp = Zq(j4 + 2) / Zq(j4 - 3);
      d = d * temp - tau;
      *dmin = or_fmin2(*dmin, d);
      Zq(j4 - 1) = Zq(j4) * temp;
      emin = or_fmin2(Zq(j4 - 1), emin);
    }
  }
  *dnm2 = d;
  *dmin2 = *dmin;
  j4 = 4 * (n0 - 2) - pp;
  j4p2 = j4 + 2 * pp - 1;
  Zq(j4 - 2) = *dnm2 + Zq(j4p2);
  Zq(j4) = Zq(j4p2 + 2) * (Zq(j4p2) / Zq(j4 - 2));
  *dnm1 = Zq(j4p2 + 2) * (*dnm2 / Zq(j4 - 2)) - tau;
  *dmin = or_fmin2(*dmin, *dnm1);
  *dmin1 = *dmin;
  j4 = j4 + 4;
  j4p2 = j4 + 2 * pp - 1;
  Zq(j4 - 2) = *dnm1 + Zq(j4p2);
  Zq(j4) = Zq(j4p2 + 2) * (Zq(j4p2) / Zq(j4 - 2));
  *dn = Zq(j4p2 + 2) * (*dnm1 / Zq(j4 - 2)) - tau;
  *dmin = or_fmin2(*dmin, *dn);
  Zq(j4 + 2) = *dn;
  Zq(4 * n0 - pp) = emin;
}

/* odsq6.f: one dqd transform (no shift), guarded against underflow. */
static void or_dlasq6(int i0, int n0, double *z, int pp, double *dmin, double *dmin1,
                      double *dmin2, double *dn, double *dnm1, double *dnm2)
{
  int j4, j4p2;
  double d, emin, temp;
  const double safmin = OR_SAFMIN;
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
      *dmin = or_fmin2(*dmin, d);
      emin = or_fmin2(emin, Zq(j4));
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
      *dmin = or_fmin2(*dmin, d);
      emin = or_fmin2(emin, Zq(j4 - 1));
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
  *dmin = or_fmin2(*dmin, *dnm1);
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
  *dmin = or_fmin2(*dmin, *dn);
  Zq(j4 + 2) = *dn;
  Zq(4 * n0 - pp) = emin;
}

/* dqds shift state carried between calls of dlasq3 (odsq2.f's locals). */
typedef struct {
  int ttype;
  double dmin1, dmin2, dn, dn1, dn2, g, tau;
} or_sq_t;

/* odsq4.f: the shift. */
static void or_dlasq4(int i0, int n0, const double *z, int pp, int n0in, double dmin,
                      or_sq_t *q)
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
          s = or_fmax2(dn - (b1 / gap1) * b1, half * dmin);
          q->ttype = -2;
        } else {
          s = 0.0;
          if (dn > b1) s = dn - b1;
          if (a2 > (b1 + b2)) s = or_fmin2(s, a2 - (b1 + b2));
          s = or_fmax2(s, third * dmin);
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
          if (hundrd * or_fmax2(b2, b1) < a2 || cnst1 < a2) break;
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
          if (hundrd * or_fmax2(b2, b1) < a2 || cnst1 < a2) break;
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
          if (hundrd * or_fmax2(b1, a2) < b2) break;
        }
      }
      b2 = sqrt(cnst3 * b2);
      a2 = dmin1 / (1.0 + b2 * b2);
      gap2 = half * dmin2 - a2;
      if (gap2 > 0.0 && gap2 > b2 * a2) {
        s = or_fmax2(s, a2 * (1.0 - cnst2 * a2 * (b2 / gap2) * b2));
      } else {
        s = or_fmax2(s, a2 * (1.0 - cnst2 * b2));
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
      if (gap2 > 0.0 && gap2 > b2 * a2) s = or_fmax2(s, a2 * (1.0 - cnst2 * a2 * (b2 / gap2) * b2));
      else s = or_fmax2(s, a2 * (1.0 - cnst2 * b2));
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
static void or_dlasq3(int i0, int *n0p, double *z, int *ppp, double *dminp, double *sigmap,
                      double *desigp, double *qmaxp, int *nfail, int *iter, int *ndiv,
                      or_sq_t *q)
{
  const double cbias = 1.50, qurtr = 0.250, half = 0.5, hundrd = 100.0;
  const double eps = OR_EPS, tol = eps * hundrd, tol2 = tol * tol;
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
      q->dmin2 = or_fmin2(q->dmin2, Zq(4 * n0 + pp - 1));
      Zq(4 * n0 + pp - 1) =
          or_fmin2(or_fmin2(Zq(4 * n0 + pp - 1), Zq(4 * i0 + pp - 1)), Zq(4 * i0 + pp + 3));
      Zq(4 * n0 - pp) = or_fmin2(or_fmin2(Zq(4 * n0 - pp), Zq(4 * i0 - pp)), Zq(4 * i0 - pp + 4));
      qmax = or_fmax2(or_fmax2(qmax, Zq(4 * i0 + pp - 3)), Zq(4 * i0 + pp + 1));
      dmin = -0.0;
    }
  }
  or_dlasq4(i0, n0, z, pp, n0in, dmin, q);
  for (;;) {   /* label 70 */
    or_dlasq5(i0, n0, z, pp, q->tau, &dmin, &q->dmin1, &q->dmin2, &q->dn, &q->dn1, &q->dn2);
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
  or_dlasq6(i0, n0, z, pp, &dmin, &q->dmin1, &q->dmin2, &q->dn, &q->dn1, &q->dn2);
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
 * the order of equal values is immaterial). */
static int or_cmp_desc(const void *a, const void *b)
{
  const double x = *(const double *)a, y = *(const double *)b;
  return (x < y) - (x > y);
}

/* odsq2.f: the eigenvalues of the qd array z (z[2k-2] = q_k, z[2k-1] = e_k,
 * 4n doubles of room) in z[0..n-1], decreasing; info as LAPACK's. */
void or_dlasq2(int n, double *z, int *info)
{
  const double cbias = 1.50, half = 0.5, four = 4.0, hundrd = 100.0;
  const double eps = OR_EPS, safmin = OR_SAFMIN, tol = eps * hundrd, tol2 = tol * tol;
  int i0, i4, ipn4, iter, iwhila, iwhilb, k, kmin, n0, n1, i1, nbig, ndiv, nfail, pp, splt;
  double d, dee, deemin, desig, dmin, e, emax, emin, oldemn, qmax, qmin, s, sigma, t, temp,
      trace, zmax, tempe, tempq;
  or_sq_t q;
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
    qmax = or_fmax2(qmax, Zq(k));
    emin = or_fmin2(emin, Zq(k + 1));
    zmax = or_fmax2(or_fmax2(qmax, zmax), Zq(k + 1));
  }
  if (Zq(2 * n - 1) < 0.0) { *info = -(200 + 2 * n - 1); return; }
  d = d + Zq(2 * n - 1);
  qmax = or_fmax2(qmax, Zq(2 * n - 1));
  zmax = or_fmax2(qmax, zmax);
  if (e == 0.0) {
    for (k = 2; k <= n; k++) Zq(k) = Zq(2 * k - 1);
    qsort(z, (size_t)n, sizeof(double), or_cmp_desc);
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
      emin = or_fmin2(emin, Zq(i4 - 2 * pp));
    }
    Zq(4 * n0 - pp - 2) = d;
    qmax = Zq(4 * i0 - pp - 2);
    for (i4 = 4 * i0 - pp + 2; i4 <= 4 * n0 - pp - 2; i4 += 4) qmax = or_fmax2(qmax, Zq(i4));
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
        qmin = or_fmin2(qmin, Zq(i4 - 3));
        emax = or_fmax2(emax, Zq(i4 - 5));
      }
      qmax = or_fmax2(qmax, Zq(i4 - 7) + Zq(i4 - 5));
      emin = or_fmin2(emin, Zq(i4 - 5));
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
    dmin = -or_fmax2(0.0, qmin - 2.0 * sqrt(qmin) * sqrt(emax));
    nbig = 100 * (n0 - i0 + 1);
    for (iwhilb = 1; iwhilb <= nbig; iwhilb++) {
      if (i0 > n0) goto l150;
      or_dlasq3(i0, &n0, z, &pp, &dmin, &sigma, &desig, &qmax, &nfail, &iter, &ndiv, &q);
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
              qmax = or_fmax2(qmax, Zq(i4 + 1));
              emin = or_fmin2(emin, Zq(i4 - 1));
              oldemn = or_fmin2(oldemn, Zq(i4));
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
  qsort(z, (size_t)n, sizeof(double), or_cmp_desc);
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
