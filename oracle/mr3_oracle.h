/*
 * mr3_oracle.h -- CPU restatement of the MR3-SMP MRRR path (TEST INFRASTRUCTURE ONLY).
 *
 * This header declares the oracle: a sequential C restatement of the reference's
 * tridiagonal eigensolver `mrrr()` (SRC/mrrr.c, SRC/mrrr_val.c, SRC/mrrr_vec.c,
 * SRC/process_{cluster,singleton,refinement}.c) and of the vendored LAPACK 3.2.x
 * kernels it calls (SRC/LAPACK/od*.f).  Only the test suite, the smoke check and
 * the CPU-baseline leg of bench.py use it, always as the checker, never as the
 * thing measured or shipped.
 *
 * Execution order.  The reference's results depend on its thread count and on
 * timing: bisection and refinement are chunked per thread
 * (SRC/mrrr_val.c:1230-1277, :1003-1060), singleton tasks are batched by a live
 * counter (SRC/process_cluster.c:477-478) and cluster refinement is split into
 * R-tasks by the same counter (SRC/process_cluster.c:302-306).  The oracle fixes
 * one deterministic order of the same algorithm:
 *   - bisection for the initial approximations (dlarrd) and the root refinement
 *     (dlarrb) run unchunked over the whole block, which is the reference's
 *     nthreads==1 branch of those two functions;
 *   - the eigenvalue stage always uses bisection, never dqds, which is what the
 *     reference does once nthreads > 12*m/n (SRC/mrrr_val.c:281-285);
 *   - there is no dstemr route for n < 500 (SRC/mrrr.c:149-153);
 *   - every singleton is its own S-task (max_size = 1 in
 *     SRC/process_cluster.c:477), and cluster refinement is never split;
 *   - logarithms use or_log(), a deterministic log (see mr3_oracle.c).
 * With these choices the result does not depend on the order tasks run in, so a
 * massively parallel implementation can reproduce it bit for bit.
 */
#ifndef MR3_ORACLE_H
#define MR3_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Full solver, same argument contract as the reference (INCLUDE/mrrr.h:62-149). */
int or_mrrr(const char *jobz, const char *range, int *n, double *D, double *E,
            double *vl, double *vu, int *il, int *iu, int *tryrac, int *m,
            double *W, double *Z, int *ldz, int *Zsupp);

/* Kernel restatements (1-based index arguments as in the Fortran). */
double or_log(double x);
int    or_dlaneg(int n, const double *d, const double *lld, double sigma,
                 double pivmin, int r);
void   or_dlarrb(int n, const double *d, const double *lld, int ifirst,
                 int ilast, double rtol1, double rtol2, int offset, double *w,
                 double *wgap, double *werr, double *work, int *iwork,
                 double pivmin, double spdiam, int twist, int *info);
void   or_dlar1v(int n, int b1, int bn, double lambda, const double *d,
                 const double *l, const double *ld, const double *lld,
                 double pivmin, double gaptol, double *z, int wantnc,
                 int *negcnt, double *ztz, double *mingma, int *r, int *isuppz,
                 double *nrminv, double *resid, double *rqcorr, double *work);
void   or_dlarrf(int n, const double *d, const double *l, const double *ld,
                 int clstrt, int clend, const double *w, const double *wgap,
                 const double *werr, double spdiam, double clgapl,
                 double clgapr, double pivmin, double *sigma, double *dplus,
                 double *lplus, double *work, int *info);
void   or_dlarrc_t(int n, double vl, double vu, const double *d,
                   const double *e, double pivmin, int *eigcnt, int *lcnt,
                   int *rcnt);
int    or_count_ijob1(int n, const double *d, const double *e2, double pivmin,
                      double x);
int    or_count_bisect(int n, const double *d, const double *e2,
                       double pivmin, double x);
void   or_dlarnv2(int iseed[4], int n, double *x);
void   or_dlasq2(int n, double *z, int *info);
int    or_dlarrr(int n, const double *d, const double *e);
void   or_dlarra(int n, const double *d, double *e, double *e2, double spltol,
                 double tnrm, int *nsplit, int *isplit);
void   or_dlarrj(int n, const double *d, const double *e2, int ifirst,
                 int ilast, double rtol, int offset, double *w, double *werr,
                 double *work, int *iwork, double pivmin, double spdiam,
                 int *info);
double or_dlanst_m(int n, const double *d, const double *e);

#ifdef __cplusplus
}
#endif
#endif
