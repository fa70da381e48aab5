// solver.cu -- batched MRRR tridiagonal eigensolver for sm_100a.
//
// One pass solves a whole batch: every kernel runs over all problems, blocks,
// eigenvalues or clusters of the batch at once.  The algorithm is the one of
// MR3-SMP (SRC/mrrr.c, SRC/mrrr_val.c, SRC/mrrr_vec.c,
// SRC/process_{cluster,singleton,refinement}.c) executed in one fixed,
// order-independent way, so the output does not depend on how the GPU
// schedules the work:
//   - bisection (dlarrd) and root refinement (dlarrb) are not chunked: one
//     thread per eigenvalue gives exactly the unchunked sequential result;
//   - the eigenvalue stage always bisects (the reference's choice once
//     nthreads > 12*m/n, SRC/mrrr_val.c:281-285); there is no dqds;
//   - every singleton is its own task and cluster refinement is never split;
//     a cluster is classified completely before its singletons run.
// The pthread task queue becomes a device work queue drained level by level:
// a level's clusters compute their child representations and refine their
// eigenvalues; a classification kernel appends child clusters and singleton
// tasks to device queues with atomics; persistent warps pull singleton tasks.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <string>
#include <vector>

#include "mr3_cuda.h"
#include "mr3_device.cuh"

#define MR3_THREADS 256
// resident 128-thread blocks per SM that the bisection and refinement
// kernels' register budgets are sized for (0: the compiler's choice)
#ifndef MR3_BIS_MINB
#define MR3_BIS_MINB 0
#endif
#ifndef MR3_REF_MINB
#define MR3_REF_MINB 0
#endif
#if MR3_BIS_MINB > 0
#define LB_BIS __launch_bounds__(128, MR3_BIS_MINB)
#else
#define LB_BIS __launch_bounds__(128)
#endif
#if MR3_REF_MINB > 0
#define LB_REF __launch_bounds__(128, MR3_REF_MINB)
#else
#define LB_REF __launch_bounds__(128)
#endif
#ifndef MR3_RRF_MINB
#define MR3_RRF_MINB 0
#endif
#if MR3_RRF_MINB > 0
#define LB_RRF __launch_bounds__(128, MR3_RRF_MINB)
#else
#define LB_RRF __launch_bounds__(128)
#endif

// ------------------------------------------------------------------------
// Device-side records
// ------------------------------------------------------------------------
struct ProbDev {
  // inputs
  int n, off, jobz, range, il, iu, tryrac, ldz;
  double vl, vu;
  double *Z;
  int *Zsupp;
  // state and outputs
  int status, m, nvals, nsplit, irange, nwl, nwu, il_out, iu_out, tryrac_out, trivial;
  int zleft;                    // eigenvector columns not yet written
  int force_bis;                // the reference's route choice forces bisection
  int tbase;                    // first column tile in the tile counters (-1: none)
  double scale, pivmin, spdiam, tnorm, gl, gu, wl, wu, wlu, wul, vl_out, vu_out, split;
};

struct BlockDev {
  int prob, ibgn, iend, nbl;    // global rows
  int ilow, iupp, mbl, wbgn;    // block-local indices, global W slot
  int irange, nab1, nab2, itmax2, nwl, nwu, none;
  double bgl, bgu;              // fudged block bounds of mrrr_val (gl, gu)
  double gl3, gu3, atoli;       // dlarrd bisection start and abstol
  double wlu, wul;              // dlarrd discard thresholds
  double sigma, spdiam, bl_spdiam;
  int dqds, sgndef;             // eigenvalues by dqds; sign of the root's definiteness
};

// A cluster of one level.  Sibling clusters (children of one parent, hence
// of one block) are stored in groups of up to 32 whose representations are
// interleaved row by row in the level's arena: row i of member g of a group
// with G members sits at index i*G + g of each field.  Group layout, in
// doubles from the group's base: P (2*nb*G), Q (2*nb*G), dplus (nb*G),
// lplus (nb*G), dlarrf work (2*nb*G): 8*nb*G doubles in all.
struct ClusterDev {
  int begin, end, depth, blk;   // W slots (global), depth, block
  double bl_spdiam, lgap;
  long long par_off;            // -1: parent is the block's root; else parent group's base
  int pG, pg;                   // parent's group size and position
  long long grp_off;            // this cluster's group base in the current arena (depth >= 1)
  int G, g;                     // group size and position
  double par_sigma, sigma, tau;
};

struct SngDev {
  int slot, cl;
  double lgap;
};


// Clusters of one level and their arena need (one record per level parity).
struct LevelCounters {
  int n_cl, err;
  unsigned long long arena_need;
};

// Singleton queue of the level being processed.
struct SngCounters {
  int n_sng, n_unit;
  int act_n[2], act_next[2];   // round lists: entries, next entry to take
  int bs_n, bs_next, err, nin; // bisection list; err: a list outlived the
                               // rounds; nin: entries of this round's list
  int done_n, done_exp;        // finished column tiles: listed, exported to the host
  int mode, fin_ctas;          // 0 rounds; 1 the next list is finished by k_sng_finish;
                               // 3 by k_sng_round<SNG_ITER>; 2 finished (later
                               // rounds are empty)
};

// Output column zind of a problem is written.  Columns are counted in tiles
// of ZT_COLS; a tile whose last column is written is listed as
// (problem, tile), so that its copy can start while the solve goes on.
#define ZT_COLS 256
__device__ __forceinline__ void column_done(ProbDev *p, int prob, int zind, SngCounters *sc,
                                            int2 *done_list, int *tile_left) {
  atomicSub(&p->zleft, 1);
  if (p->tbase < 0) return;
  const int t = zind / ZT_COLS;
  if (atomicSub(&tile_left[p->tbase + t], 1) == 1)
    done_list[atomicAdd(&sc->done_n, 1)] = make_int2(prob, t);
}

// The level and singleton counters (hlc, hsc), and the column tiles listed
// since the last export (hdone, with their count so far in *hsnap), written
// by the SMs straight into pinned host memory; null targets are skipped.
// A copy-engine transfer would queue behind the eigenvector copies of
// finished tiles that the caller may have started meanwhile.
__global__ void k_export(const LevelCounters *lc, LevelCounters *hlc, SngCounters *sc,
                         SngCounters *hsc, const int2 *done_list, int2 *hdone, int *hsnap) {
  const int t = threadIdx.x, from = sc->done_exp, to = sc->done_n;
  if (t == 0) {
    if (hlc) *hlc = *lc;
    if (hsc) *hsc = *sc;
    if (hsnap) *hsnap = to;
  }
  if (hdone)
    for (int i = from + t; i < to; i += blockDim.x) hdone[i] = done_list[i];
  __syncthreads();
  if (t == 0 && hdone) sc->done_exp = to;
}

struct Tol {
  double rtol1, rtol2, bsrtol, rqtol;
  int nthreads;                 // thread count of the reference's route choice
};

// ------------------------------------------------------------------------
// Small helpers
// ------------------------------------------------------------------------
__device__ __forceinline__ double warp_min(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Inclusive scan of ints over a 256-thread CTA; returns the exclusive prefix
// and stores the total in *total.
__device__ int cta_exscan(int v, int *sh, int *total) {
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int t = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    sh[lane] = t;
  }
  __syncthreads();
  int base = (wid > 0) ? sh[wid - 1] : 0;
  *total = sh[(blockDim.x >> 5) - 1];
  __syncthreads();
  return base + x - v;
}

__device__ __forceinline__ void set_status(ProbDev *p, int s) { atomicMax(&p->status, s); }

// Device work counters for the roofline: stats[kernel * 4 + kind], kinds
// 0 = Sturm-count steps on T, 1 = Sturm-count steps on L D L^T (dlaneg),
// 2 = twisted-factorisation rows (dlar1v), 3 = dlarrf rows.  Every lane of a
// warp must call stat_add (it reduces over the full warp).
enum { KID_BISECT = 0, KID_REFROOT, KID_NEWRRR, KID_REFCL, KID_SNG, KID_OTHER, KID_COUNT };
__device__ __forceinline__ void stat_add(unsigned long long *stats, int slot, unsigned long long v) {
  if (stats == nullptr) return;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(&stats[slot], v);
}

// ------------------------------------------------------------------------
// Stage A0: per-problem prologue (SRC/mrrr.c:206-243, SRC/mrrr_val.c:167-329)
// ------------------------------------------------------------------------
__global__ void k_gather(ProbDev *probs, const double *const *Din, const double *const *Ein,
                         double *D, double *E, int *prob_of_slot, int *iblk) {
  ProbDev *p = &probs[blockIdx.x];
  const double *di = Din[blockIdx.x], *ei = Ein[blockIdx.x];
  for (int i = threadIdx.x; i < p->n; i += blockDim.x) {
    D[p->off + i] = di[i];
    E[p->off + i] = ei[i];
    prob_of_slot[p->off + i] = blockIdx.x;
    iblk[p->off + i] = -1;
  }
}

// Non-finite entries among the values a problem's solve reads (D[0..n-1],
// E[0..n-2]): flag[k] = 1.  Such a problem is refused before the solve.
__global__ void k_finite(const ProbDev *probs, const double *const *Din, const double *const *Ein,
                         int *flag) {
  __shared__ int bad;
  const int n = probs[blockIdx.x].n;
  const double *d = Din[blockIdx.x], *e = Ein[blockIdx.x];
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  int b = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    b |= !isfinite(d[i]);
    if (i < n - 1) b |= !isfinite(e[i]);
  }
  if (b) bad = 1;
  __syncthreads();
  if (threadIdx.x == 0) flag[blockIdx.x] = bad;
}

__global__ void __launch_bounds__(MR3_THREADS)
k_prologue(ProbDev *probs, BlockDev *blocks, int *blk_of_row, double *D, double *E, double *E2,
           double2 *gers, double2 *TP, double2 *TPc, Tol tol) {
  __shared__ double sred[32];
  __shared__ int sint[64];
  __shared__ int sflag;
  ProbDev *p = &probs[blockIdx.x];
  const int n = p->n, off = p->off, tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, wid = tid >> 5;
  double *d = D + off, *e = E + off, *e2 = E2 + off;
  if (p->trivial) return;   // handled on the host side (n == 1 or counting only)

  // ---- scale_matrix (SRC/mrrr.c:325-365): dlanst('M') by a max-reduction
  double tn = 0.0;
  for (int i = tid; i < n; i += nt) {
    tn = fmax(tn, fabs(d[i]));
    if (i < n - 1) tn = fmax(tn, fabs(e[i]));
  }
  tn = warp_max(tn);
  if (lane == 0) sred[wid] = tn;
  __syncthreads();
  if (tid == 0) {
    double t = 0.0;
    for (int w = 0; w < (nt >> 5); w++) t = fmax(t, sred[w]);
    double smlnum = MR3_SAFMIN / MR3_EPS, bignum = 1.0 / smlnum;
    double rmin = sqrt(smlnum), rmax = fmin(sqrt(bignum), 1.0 / sqrt(sqrt(MR3_SAFMIN)));
    double scale = 1.0;
    if (t > 0 && t < rmin) scale = rmin / t;
    else if (t > rmax) scale = rmax / t;
    p->scale = scale;
    if (scale != 1.0 && p->range == MR3_RANGE_V) { p->vl *= scale; p->vu *= scale; }
  }
  __syncthreads();
  const double scale = p->scale;
  if (scale != 1.0) {
    for (int i = tid; i < n; i += nt) {
      d[i] *= scale;
      if (i < n - 1) e[i] *= scale;
    }
  }
  __syncthreads();

  // ---- dlarrr (SRC/LAPACK/odrrr.f): the sequential test is an AND of
  // independent per-row conditions, so it is evaluated in parallel.
  if (tid == 0) sflag = 0;
  __syncthreads();
  int tryrac = p->tryrac;
  if (tryrac) {
    // fail if some sqrt|d(i)| < rmin, or od(i-1) + od(i) >= 0.999 with
    // od(i) = |e(i-1)| / (sqrt|d(i-1)| sqrt|d(i)|) and od(0) = 0
    const double rmin = sqrt(MR3_SAFMIN / MR3_EPS);
    int bad = 0;
    for (int i = tid; i < n; i += nt) {
      double t2 = sqrt(fabs(d[i]));
      if (t2 < rmin) bad = 1;
      if (i >= 1) {
        double t1 = sqrt(fabs(d[i - 1]));
        double od = fabs(e[i - 1]) / (t1 * t2);
        double odp = (i >= 2) ? fabs(e[i - 2]) / (sqrt(fabs(d[i - 2])) * t1) : 0.0;
        if (odp + od >= 0.999) bad = 1;
      }
    }
    if (bad) atomicOr(&sflag, 1);
    __syncthreads();
    tryrac = (sflag == 0);
  }
  if (tid == 0) {
    p->tryrac_out = tryrac;
    p->split = tryrac ? MR3_EPS : -MR3_EPS;
  }
  if (tryrac) {   // Dcopy, E2copy for refine_to_highrac (SRC/mrrr.c:217-222)
    for (int i = tid; i < n; i += nt) {
      double e2c = (i >= 1) ? e[i - 1] * e[i - 1] : 0.0;
      TPc[off + i] = make_double2(d[i], e2c);
    }
  }
  __syncthreads();

  // ---- E2, Gershgorin discs, pivmin, spdiam (SRC/mrrr_val.c:213-241)
  for (int i = tid; i < n; i += nt) e2[i] = e[i] * e[i];
  __syncthreads();
  if (tid == 0) e[n - 1] = 0.0;
  __syncthreads();
  double gl = d[0], gu = d[0], emax = 0.0;
  for (int i = tid; i < n; i += nt) {
    double eabs = fabs(e[i]);
    double eold = (i > 0) ? fabs(e[i - 1]) : 0.0;
    double t1 = eabs + eold;
    double lo = d[i] - t1, hi = d[i] + t1;
    gers[off + i] = make_double2(lo, hi);
    gl = fmin(gl, lo);
    gu = fmax(gu, hi);
    emax = fmax(emax, eabs);
  }
  gl = warp_min(gl);
  gu = warp_max(gu);
  emax = warp_max(emax);
  __shared__ double sgl[8], sgu[8], sem[8];
  if (lane == 0) { sgl[wid] = gl; sgu[wid] = gu; sem[wid] = emax; }
  __syncthreads();
  if (tid == 0) {
    for (int w = 1; w < (nt >> 5); w++) {
      sgl[0] = fmin(sgl[0], sgl[w]);
      sgu[0] = fmax(sgu[0], sgu[w]);
      sem[0] = fmax(sem[0], sem[w]);
    }
    double pivmin = MR3_SAFMIN * fmax(1.0, sem[0] * sem[0]);
    double g0 = sgl[0], g1 = sgu[0];
    p->pivmin = pivmin;
    p->spdiam = g1 - g0;
    double tnorm = fmax(fabs(g0), fabs(g1));
    p->tnorm = tnorm;
    g0 = g0 - 2 * tnorm * MR3_EPS * n - 4 * pivmin;
    g1 = g1 + 2 * tnorm * MR3_EPS * n + 4 * pivmin;
    p->gl = g0;
    p->gu = g1;
    int irange = p->range;
    if (irange == MR3_RANGE_I && p->il == 1 && p->iu == n) irange = MR3_RANGE_A;
    if (irange == MR3_RANGE_V && p->vl < g0 && p->vu >= g1) irange = MR3_RANGE_A;
    p->irange = irange;
  }
  __syncthreads();

  // ---- dlarra splitting (SRC/LAPACK/odrra.f:98-125) and the block list
  const double split = p->split, spd = p->spdiam;
  int chunk = (n + nt - 1) / nt;
  int c0 = tid * chunk, c1 = min(n, c0 + chunk);
  int cnt = 0;
  for (int i = c0; i < c1; i++) {
    if (i < n - 1) {
      double eabs = fabs(e[i]);
      bool sp = (split < 0.0) ? (eabs <= fabs(split) * spd)
                              : (eabs <= split * sqrt(fabs(d[i])) * sqrt(fabs(d[i + 1])));
      if (sp) { e[i] = 0.0; e2[i] = 0.0; cnt++; }
    }
  }
  __syncthreads();
  int total;
  int base = cta_exscan(cnt, sint, &total);
  // splits are recognised again by e[i] == 0.0 && e2[i] == 0.0 only where we
  // set them; recount with the same predicate outcome stored in a flag pass.
  int b = base;
  for (int i = c0; i < c1; i++) {
    blk_of_row[off + i] = off + b;
    if (i < n - 1) {
      double eabs = fabs(e[i]);
      // after zeroing, a split row has e[i] == 0 exactly; rows that were
      // already zero also satisfy the split test, so the test is repeated on
      // the stored value, which gives the same decision.
      bool sp = (split < 0.0) ? (eabs <= fabs(split) * spd)
                              : (eabs <= split * sqrt(fabs(d[i])) * sqrt(fabs(d[i + 1])));
      if (sp) {
        blocks[off + b].iend = off + i;
        blocks[off + b + 1].ibgn = off + i + 1;
        b++;
      }
    }
  }
  if (tid == 0) {
    blocks[off].ibgn = off;
    blocks[off + total].iend = off + n - 1;
    p->nsplit = total + 1;
  }
  __syncthreads();
  for (int bb = tid; bb <= total; bb += nt) {
    BlockDev *B = &blocks[off + bb];
    B->prob = blockIdx.x;
    B->nbl = B->iend - B->ibgn + 1;
  }
  // packed T rows for the Sturm counts: (d[j], e2[j-1])
  for (int i = tid; i < n; i += nt) TP[off + i] = make_double2(d[i], (i > 0) ? e2[i - 1] : 0.0);
  __syncthreads();

  // ---- number of wanted eigenvalues (SRC/mrrr_val.c:252-270)
  const int irange = p->irange;
  const double pivmin = p->pivmin;
  if (irange == MR3_RANGE_A) {
    if (tid == 0) { p->il_out = 1; p->iu_out = n; }
  } else if (irange == MR3_RANGE_V) {
    if (tid == 0) p->il_out = dv_count_ijob1(n, TP + off, pivmin, p->vl) + 1;
    if (tid == 32) p->iu_out = dv_count_ijob1(n, TP + off, pivmin, p->vu);
  } else {
    if (tid == 0) { p->il_out = p->il; p->iu_out = p->iu; }
  }
  __syncthreads();
  if (tid == 0) {
    p->nvals = p->iu_out - p->il_out + 1;
    p->m = p->nvals;
    // SRC/mrrr_val.c:279-282: bisection unless few threads per eigenvalue
    p->force_bis = (double)tol.nthreads > ceil(12.0 * p->nvals / (double)n);
    if (irange == MR3_RANGE_V) { p->wl = p->vl; p->wu = p->vu; p->vl_out = p->vl; p->vu_out = p->vu; }
    if (irange == MR3_RANGE_A) { p->wl = p->gl; p->wu = p->gu; p->vl_out = p->gl; p->vu_out = p->gu; }
  }
  if (p->jobz == MR3_JOB_C) return;
  // ---- range I: the interval holding eigenvalues il..iu (SRC/mrrr_val.c:295-319),
  // the two searches by warps 0 and 1, each with the tree form
  if (irange == MR3_RANGE_I && tid < 64) {
    int itmax = (int)((dv_log(p->tnorm + pivmin) - dv_log(pivmin)) / dv_log(2.0) + 2);
    double atoli = 2 * (2 * MR3_SAFMIN + 2 * pivmin);
    double a = p->gl, bq = p->gu;
    int na = -1, nb = n + 1;
    if (tid < 32) {
      dv_ijob3_tree(32, n, TP + off, pivmin, atoli, tol.rqtol, itmax, p->il - 1, p->gl, &a, &bq,
                    &na, &nb);
      if (tid == 0) { p->wl = a; p->wlu = bq; p->nwl = na; p->vl_out = a; }
    } else {
      dv_ijob3_tree(32, n, TP + off, pivmin, atoli, tol.rqtol, itmax, p->iu, p->gu, &a, &bq, &na,
                    &nb);
      if (tid == 32) { p->wul = a; p->wu = bq; p->nwu = nb; p->vu_out = bq; }
    }
  }
}

// ------------------------------------------------------------------------
// Stage A1: per-block setup (SRC/mrrr_val.c:340-412 and the set-up part of
// dlarrd, SRC/LAPACK/odrrd.f:283-450).  One warp per block.
// ------------------------------------------------------------------------
__global__ void __launch_bounds__(MR3_THREADS)
k_blocks(ProbDev *probs, BlockDev *blocks, const double *D, double *E, const double2 *gers,
         const double2 *TP, Tol tol) {
  ProbDev *p = &probs[blockIdx.x];
  if (p->trivial || p->jobz == MR3_JOB_C) return;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const double pivmin = p->pivmin, tnorm = p->tnorm, wl = p->wl, wu = p->wu;
  const int irange = p->irange;
  for (int b = wid; b < p->nsplit; b += nw) {
    BlockDev *B = &blocks[p->off + b];
    const int ibgn = B->ibgn, iend = B->iend, nbl = B->nbl;
    if (nbl == 1) {
      if (lane == 0) {
        double dv = D[ibgn];
        bool take = (irange == MR3_RANGE_A) || (irange == MR3_RANGE_V && dv > wl && dv <= wu) ||
                    (irange == MR3_RANGE_I && (dv + pivmin) > wl && (dv - pivmin) <= wu);
        B->mbl = take ? 1 : 0;
        B->ilow = 1; B->iupp = take ? 1 : 0;
        B->nab1 = 0; B->nab2 = 0; B->none = 1;
        B->sigma = 0.0;
        E[iend] = 0.0;
      }
      continue;
    }
    double bgl = D[ibgn], bgu = D[ibgn];
    for (int i = ibgn + lane; i <= iend; i += 32) {
      double2 g = gers[i];
      bgl = fmin(bgl, g.x);
      bgu = fmax(bgu, g.y);
    }
    bgl = warp_min(bgl);
    bgu = warp_max(bgu);
    const double bglf = bgl - 2 * tnorm * MR3_EPS * nbl - 4 * pivmin;
    const double bguf = bgu + 2 * tnorm * MR3_EPS * nbl + 4 * pivmin;
    int ilow = 1, iupp = nbl;
    if (irange != MR3_RANGE_A) {
      int c = 0;
      if (lane == 0) c = dv_count_ijob1(nbl, TP + ibgn, pivmin, fmax(wl, bglf)) + 1;
      if (lane == 1) c = dv_count_ijob1(nbl, TP + ibgn, pivmin, fmin(wu, bguf));
      ilow = __shfl_sync(0xffffffffu, c, 0);
      iupp = __shfl_sync(0xffffffffu, c, 1);
    }
    const int mbl = iupp - ilow + 1;
    if (lane == 0) {
      B->bgl = bglf; B->bgu = bguf; B->spdiam = bguf - bglf;
      B->ilow = ilow; B->iupp = iupp; B->mbl = mbl;
      B->none = 1; B->nab1 = 0; B->nab2 = 0;
      if (mbl < 0) set_status(p, MR3_EMISC);
      if (mbl <= 0) E[iend] = 0.0;
    }
    if (mbl <= 0) continue;
    // dlarrd("I","B") set-up on this block
    const int brange = (ilow == 1 && iupp == nbl) ? MR3_RANGE_A : MR3_RANGE_I;
    const double tnb = fmax(fabs(bgl), fabs(bgu));
    const double gl2 = bgl - 2.0 * tnb * MR3_EPS * nbl - 2.0 * 2.0 * pivmin;
    const double gu2 = bgu + 2.0 * tnb * MR3_EPS * nbl + 2.0 * 2.0 * pivmin;
    const double atoli = 2.0 * 2.0 * MR3_SAFMIN + 2.0 * 2.0 * pivmin;
    double wlb = gl2, wub = gu2, wlub = 0.0, wulb = 0.0;
    int bad = 0;
    if (brange == MR3_RANGE_I) {
      int itmax = dv_itmax(tnb + pivmin, pivmin);
      double a = gl2, bq = gu2;
      int na = -1, nb = nbl + 1;
      // the two searches by half-warps, each with the tree form
      if (lane < 16)
        dv_ijob3_tree(16, nbl, TP + ibgn, pivmin, atoli, tol.bsrtol, itmax, ilow - 1, gl2, &a, &bq,
                      &na, &nb);
      else
        dv_ijob3_tree(16, nbl, TP + ibgn, pivmin, atoli, tol.bsrtol, itmax, iupp, gu2, &a, &bq,
                      &na, &nb);
      double a0 = __shfl_sync(0xffffffffu, a, 0), b0 = __shfl_sync(0xffffffffu, bq, 0);
      double a1 = __shfl_sync(0xffffffffu, a, 16), b1 = __shfl_sync(0xffffffffu, bq, 16);
      int nwl = __shfl_sync(0xffffffffu, na, 0), nwu = __shfl_sync(0xffffffffu, nb, 16);
      wlb = a0; wlub = b0; wulb = a1; wub = b1;
      if (nwl < 0 || nwl >= nbl || nwu < 1 || nwu > nbl) bad = 1;
    }
    double gl3 = bgl - 2.0 * tnb * MR3_EPS * nbl - 2.0 * pivmin;
    double gu3 = bgu + 2.0 * tnb * MR3_EPS * nbl + 2.0 * pivmin;
    int none = 0, nwlb = 0, nwub = 0;
    if (brange == MR3_RANGE_I) {
      if (gu3 < wlb) { none = 1; nwlb = nbl; nwub = nbl; }
      else {
        gl3 = fmax(gl3, wlb);
        gu3 = fmin(gu3, wub);
        if (gl3 >= gu3) none = 1;
      }
    }
    int nab1 = 0, nab2 = 0;
    if (!none) {
      int c = 0;
      if (lane == 0) c = dv_count_ijob1(nbl, TP + ibgn, pivmin, gl3);
      if (lane == 1) c = dv_count_ijob1(nbl, TP + ibgn, pivmin, gu3);
      nab1 = __shfl_sync(0xffffffffu, c, 0);
      nab2 = __shfl_sync(0xffffffffu, c, 1);
      nwlb = nab1; nwub = nab2;
    }
    if (lane == 0) {
      B->irange = brange;
      B->gl3 = gl3; B->gu3 = gu3; B->atoli = atoli;
      B->wlu = wlub; B->wul = wulb;
      B->none = none; B->nab1 = nab1; B->nab2 = nab2; B->nwl = nwlb; B->nwu = nwub;
      B->itmax2 = none ? 0 : dv_itmax(gu3 - gl3 + pivmin, pivmin);
      if (bad) set_status(p, MR3_EMISC);
    }
  }
}

// ------------------------------------------------------------------------
// Stage A2: initial approximations by bisection, one thread per eigenvalue
// (dlarrd/dlaebz IJOB=2, SRC/LAPACK/odrrd.f:450-520).  Thread k of a block
// bisects eigenvalue nab1+1+k; a block never has more than nbl of them.
// ------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long bisect_body(int g, const ProbDev *probs,
                                                          const BlockDev *blocks,
                                                          const int *blk_of_row, const double2 *TP,
                                                          double *Wt, double *Et, int *It, Tol tol) {
  const BlockDev *B = &blocks[blk_of_row[g]];
  const ProbDev *p = &probs[B->prob];
  if (p->trivial || p->jobz == MR3_JOB_C || p->status) return 0;
  int k = g - B->ibgn;
  if (B->nbl < 2 || B->mbl <= 0 || B->none || k >= B->nab2 - B->nab1) return 0;
  int j = B->nab1 + 1 + k;
  double a = B->gl3, b = B->gu3;
  int it = 0;
  dv_bisect_one(B->nbl, TP + B->ibgn, p->pivmin, B->atoli, tol.bsrtol, B->itmax2, j, &a, &b,
                B->nab1, B->nab2, &it);
  Wt[g] = 0.5 * (a + b);
  Et[g] = 0.5 * fabs(a - b);
  It[g] = j;
  return (unsigned long long)it * (unsigned long long)B->nbl;
}

// TREE = false: a thread per eigenvalue (L = 1).  The two forms are separate
// instantiations so that the thread form keeps its own register budget.
template <bool TREE>
__global__ void __launch_bounds__(128)
k_bisect(int N, int L, const ProbDev *probs, const BlockDev *blocks, const int *blk_of_row,
         const double2 *TP, double *Wt, double *Et, int *It, Tol tol, unsigned long long *stats) {
  const long long gt = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  unsigned long long work = 0;
  if (!TREE) {
    if (gt < N) work = bisect_body((int)gt, probs, blocks, blk_of_row, TP, Wt, Et, It, tol);
  } else if (gt / L < N) {
    // L lanes per eigenvalue (few eigenvalues: single large problems)
    const int g = (int)(gt / L);
    const BlockDev *B = &blocks[blk_of_row[g]];
    const ProbDev *p = &probs[B->prob];
    const int k = g - B->ibgn;
    if (!(p->trivial || p->jobz == MR3_JOB_C || p->status) &&
        !(B->nbl < 2 || B->mbl <= 0 || B->none || k >= B->nab2 - B->nab1)) {
      const int j = B->nab1 + 1 + k;
      double a = B->gl3, b = B->gu3;
      int itc = 0;
      dv_bisect_tree(L, B->nbl, TP + B->ibgn, p->pivmin, B->atoli, tol.bsrtol, B->itmax2, j, &a, &b,
                     B->nab1, B->nab2, &itc);
      if ((gt % L) == 0) {
        Wt[g] = 0.5 * (a + b);
        Et[g] = 0.5 * fabs(a - b);
        It[g] = j;
        work = (unsigned long long)itc * (unsigned long long)B->nbl;
      }
    }
  }
  stat_add(stats, KID_BISECT * 4 + 0, work);
}

// ------------------------------------------------------------------------
// Stage A2 with shared intervals (the thread form's replacement for many
// eigenvalues).  The bisection of eigenvalue j (dv_bisect_one from
// [gl3, gu3]) visits the same intervals as every other eigenvalue of its
// block until a Sturm count separates them: its state (a, b, na, nb) after
// k steps is a node of a binary tree rooted at the block's start interval.
// The tree's levels run breadth-first with one Sturm count per node, and a
// node's eigenvalues continue in its children.  A child holding one
// eigenvalue leaves the tree with its state (k_bisect_cont continues it, a
// thread per eigenvalue); a converged child, or one at the iteration
// limit, writes its eigenvalues' results.  Every eigenvalue sees the
// operations of dv_bisect_one in the same order, so the results are those
// of the thread form bit for bit, and the first levels, which all of a
// block's eigenvalues share, are counted once per node.
// ------------------------------------------------------------------------
struct BisNode {
  double a, b;
  int na, nb, it, blk;   // counts at a and b, steps done, block
};
struct BisState {
  int na, nb, it, pad;   // a single eigenvalue's state (a, b in Wt, Et); it < 0: none
};
#define BIS_DEPTH 16     // tree levels before the remaining nodes are split up

__device__ __forceinline__ bool bis_block_ok(const BlockDev *B, const ProbDev *p) {
  return !(p->trivial || p->jobz == MR3_JOB_C || p->status) &&
         !(B->nbl < 2 || B->mbl <= 0 || B->none) && B->nab2 > B->nab1;
}

// Eigenvalues na+1..nb of an interval: results (done) or single states.
__device__ __forceinline__ void bis_finish(const BlockDev *B, double a, double b, int na, int nb,
                                           int it, bool done, double *Wt, double *Et, int *It,
                                           BisState *st) {
  for (int j = na + 1; j <= nb; j++) {
    const int g = B->ibgn + (j - B->nab1 - 1);
    if (done) {
      Wt[g] = 0.5 * (a + b);
      Et[g] = 0.5 * fabs(a - b);
      It[g] = j;
    } else {
      Wt[g] = a;
      Et[g] = b;
      BisState q;
      q.na = na; q.nb = nb; q.it = it; q.pad = 0;
      st[g] = q;
    }
  }
}

// The children of a node after its count cnt (already clamped to [na, nb]):
// kind 0 empty, 1 done, 2 one eigenvalue, 3 a node of the next level.
__device__ __forceinline__ int bis_child(const BisNode &nd, int cnt, int side, double pivmin,
                                         double abstol, double reltol, int itmax, BisNode *ch) {
  const double c = 0.5 * (nd.a + nd.b);
  ch->a = side ? c : nd.a;
  ch->b = side ? nd.b : c;
  ch->na = side ? cnt : nd.na;
  ch->nb = side ? nd.nb : cnt;
  ch->it = nd.it + 1;
  ch->blk = nd.blk;
  if (ch->nb <= ch->na) return 0;
  const double w = fabs(ch->b - ch->a), t = fmax(fabs(ch->b), fabs(ch->a));
  if (w < fmax(fmax(abstol, pivmin), reltol * t) || ch->it >= itmax) return 1;
  return ch->nb - ch->na == 1 ? 2 : 3;
}

__global__ void __launch_bounds__(256)
k_bis_roots(int N, const ProbDev *probs, const BlockDev *blocks, const int *blk_of_row,
            BisNode *out, int *n_out, double *Wt, double *Et, int *It, BisState *st) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= N) return;
  const int bk = blk_of_row[g];
  const BlockDev *B = &blocks[bk];
  if (g != B->ibgn) return;
  const ProbDev *p = &probs[B->prob];
  if (!bis_block_ok(B, p)) return;
  if (B->itmax2 <= 0) {
    bis_finish(B, B->gl3, B->gu3, B->nab1, B->nab2, 0, true, Wt, Et, It, st);
  } else if (B->nab2 - B->nab1 == 1) {
    bis_finish(B, B->gl3, B->gu3, B->nab1, B->nab2, 0, false, Wt, Et, It, st);
  } else {
    BisNode nd;
    nd.a = B->gl3; nd.b = B->gu3; nd.na = B->nab1; nd.nb = B->nab2; nd.it = 0; nd.blk = bk;
    out[atomicAdd(n_out, 1)] = nd;
  }
}

// One level: a Sturm count per node; done and single children written out,
// the number of next-level children per CTA in bcnt.
__global__ void __launch_bounds__(256)
k_bis_count(const BisNode *in, const int *n_in_dev, const ProbDev *probs, const BlockDev *blocks,
            const double2 *TP, Tol tol, int *ccnt, int *bcnt, double *Wt, double *Et, int *It,
            BisState *st, unsigned long long *stats) {
  __shared__ int sint[32];
  // the level's length is on the device (the grid covers its bound, N/2)
  const int n_in = *n_in_dev;
  if (blockIdx.x * blockDim.x >= n_in) {
    if (threadIdx.x == 0) bcnt[blockIdx.x] = 0;
    return;
  }
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int nnext = 0;
  unsigned long long work = 0;
  if (i < n_in) {
    const BisNode nd = in[i];
    const BlockDev *B = &blocks[nd.blk];
    const double pivmin = probs[B->prob].pivmin;
    int cnt = dv_count_bisect(B->nbl, TP + B->ibgn, pivmin, 0.5 * (nd.a + nd.b));
    cnt = d_imin(nd.nb, d_imax(nd.na, cnt));
    ccnt[i] = cnt;
    work = (unsigned long long)B->nbl;
    for (int side = 0; side < 2; side++) {
      BisNode ch;
      const int kind = bis_child(nd, cnt, side, pivmin, B->atoli, tol.bsrtol, B->itmax2, &ch);
      if (kind == 1 || kind == 2)
        bis_finish(B, ch.a, ch.b, ch.na, ch.nb, ch.it, kind == 1, Wt, Et, It, st);
      else if (kind == 3)
        nnext++;
    }
  }
  int total;
  cta_exscan(nnext, sint, &total);
  if (threadIdx.x == 0) bcnt[blockIdx.x] = total;
  stat_add(stats, KID_BISECT * 4 + 0, work);
}

// Exclusive scan of the per-CTA counts (one CTA of 1024 threads); the total
// is the next level's length.
__global__ void __launch_bounds__(1024) k_bis_scan(int nblk, int *bcnt, int *n_out) {
  __shared__ int sint[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int b0 = 0; b0 < nblk; b0 += 1024) {
    const int b = b0 + threadIdx.x;
    const int v = b < nblk ? bcnt[b] : 0;
    int total;
    const int ex = cta_exscan(v, sint, &total);
    if (b < nblk) bcnt[b] = carry + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) *n_out = carry;
}

// The next level's nodes, in the order of their parents (a block's nodes
// stay together).  split: the depth limit is reached and the nodes' eigenvalues
// leave the tree as single states instead.
__global__ void __launch_bounds__(256)
k_bis_scatter(const BisNode *in, const int *n_in_dev, const ProbDev *probs, const BlockDev *blocks,
              Tol tol, const int *ccnt, const int *bcnt, BisNode *out, int split, double *Wt,
              double *Et, int *It, BisState *st) {
  __shared__ int sint[32];
  const int n_in = *n_in_dev;
  if (blockIdx.x * blockDim.x >= n_in) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  BisNode ch[2];
  int kind[2] = {0, 0}, nnext = 0;
  const BlockDev *B = nullptr;
  if (i < n_in) {
    const BisNode nd = in[i];
    B = &blocks[nd.blk];
    const double pivmin = probs[B->prob].pivmin;
    for (int side = 0; side < 2; side++) {
      kind[side] = bis_child(nd, ccnt[i], side, pivmin, B->atoli, tol.bsrtol, B->itmax2, &ch[side]);
      nnext += kind[side] == 3;
    }
  }
  int total;
  int pos = bcnt[blockIdx.x] + cta_exscan(split ? 0 : nnext, sint, &total);
  for (int side = 0; side < 2; side++)
    if (kind[side] == 3) {
      if (split) bis_finish(B, ch[side].a, ch[side].b, ch[side].na, ch[side].nb, ch[side].it, false,
                            Wt, Et, It, st);
      else out[pos++] = ch[side];
    }
}

// The single eigenvalues that left the tree, a thread each, continued with
// dv_bisect_one from their state.
__global__ void LB_BIS
k_bisect_cont(int N, const ProbDev *probs, const BlockDev *blocks, const int *blk_of_row,
              const double2 *TP, double *Wt, double *Et, int *It, const BisState *st, Tol tol,
              unsigned long long *stats) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long work = 0;
  if (g < N) {
    const BisState q = st[g];
    if (q.it >= 0) {
      const BlockDev *B = &blocks[blk_of_row[g]];
      const ProbDev *p = &probs[B->prob];
      const int j = B->nab1 + 1 + (g - B->ibgn);
      double a = Wt[g], b = Et[g];
      int it = q.it;
      dv_bisect_one(B->nbl, TP + B->ibgn, p->pivmin, B->atoli, tol.bsrtol, B->itmax2, j, &a, &b,
                    q.na, q.nb, &it, q.it);
      Wt[g] = 0.5 * (a + b);
      Et[g] = 0.5 * fabs(a - b);
      It[g] = j;
      work = (unsigned long long)(it - q.it) * (unsigned long long)B->nbl;
    }
  }
  stat_add(stats, KID_BISECT * 4 + 0, work);
}

// ------------------------------------------------------------------------
// Stage A3: per problem, place each block's approximations in W after the
// dlarrd discard of range I (SRC/LAPACK/odrrd.f:520-640).
// ------------------------------------------------------------------------
__global__ void __launch_bounds__(MR3_THREADS)
k_compact(ProbDev *probs, BlockDev *blocks, const double *D, double *Wt, double *Et, int *It,
          double *W, double *Werr, int *Windex, int *iblk, double *Wcopy, int *tile_left) {
  __shared__ int sint[64];
  ProbDev *p = &probs[blockIdx.x];
  if (p->trivial || p->jobz == MR3_JOB_C) return;
  const int tid = threadIdx.x, nt = blockDim.x, off = p->off, ns = p->nsplit;
  // W slot of each block: exclusive prefix of mbl over the blocks
  int chunk = (ns + nt - 1) / nt, c0 = tid * chunk, c1 = min(ns, c0 + chunk), s = 0;
  for (int b = c0; b < c1; b++) s += max(blocks[off + b].mbl, 0);
  int total, base = cta_exscan(s, sint, &total);
  for (int b = c0; b < c1; b++) {
    blocks[off + b].wbgn = off + base;
    base += max(blocks[off + b].mbl, 0);
  }
  if (tid == 0) {
    p->m = total;
    p->zleft = (p->jobz == MR3_JOB_V) ? total : 0;
    // the host sized the tiles for iu-il+1 (range I) or n (range A) columns
    if (total != (p->range == MR3_RANGE_I ? p->iu - p->il + 1 : p->n)) p->tbase = -1;
  }
  __syncthreads();
  // column tiles of ZT_COLS output columns, each counting its unwritten columns
  if (p->tbase >= 0 && p->jobz == MR3_JOB_V)
    for (int t = tid; t * ZT_COLS < total; t += nt)
      tile_left[p->tbase + t] = min(ZT_COLS, total - t * ZT_COLS);
  __syncthreads();
  const int lane = tid & 31, wid = tid >> 5, nw = nt >> 5;
  for (int b = wid; b < ns; b += nw) {
    BlockDev *B = &blocks[off + b];
    const int mbl = B->mbl, wb = B->wbgn, ib = B->ibgn;
    if (mbl <= 0) continue;
    if (B->nbl == 1) {
      if (lane == 0) {
        W[wb] = D[ib]; Werr[wb] = 0.0; Windex[wb] = 1; iblk[wb] = off + b; Wcopy[wb] = D[ib];
      }
      continue;
    }
    int mcnt = B->nab2 - B->nab1;
    if (B->irange == MR3_RANGE_I && lane == 0) {
      // discard surplus values from both ends, in place on the row scratch
      double *w = Wt + ib, *we = Et + ib;
      int *ix = It + ib;
      int idiscl = B->ilow - 1 - B->nwl, idiscu = B->nwu - B->iupp, im;
      if (idiscl > 0) {
        im = 0;
        for (int je = 0; je < mcnt; je++) {
          if (w[je] <= B->wlu && idiscl > 0) idiscl--;
          else { w[im] = w[je]; we[im] = we[je]; ix[im] = ix[je]; im++; }
        }
        mcnt = im;
      }
      if (idiscu > 0) {
        im = mcnt;
        for (int je = mcnt - 1; je >= 0; je--) {
          if (w[je] >= B->wul && idiscu > 0) idiscu--;
          else { im--; w[im] = w[je]; we[im] = we[je]; ix[im] = ix[je]; }
        }
        int jee = 0;
        for (int je = im; je < mcnt; je++) { w[jee] = w[je]; we[jee] = we[je]; ix[jee] = ix[je]; jee++; }
        mcnt = mcnt - im;
      }
      if (idiscl > 0 || idiscu > 0) {
        // kill-off path of dlarrd (bad arithmetic): mark by index = 0
        if (idiscl > 0) {
          double wkill = 0.0;
          for (int jd = 0; jd < idiscl; jd++) {
            int iw = -1;
            for (int je = 0; je < mcnt; je++)
              if (ix[je] != 0 && (iw == -1 || w[je] < wkill)) { iw = je; wkill = w[je]; }
            if (iw >= 0) ix[iw] = 0;
          }
        }
        if (idiscu > 0) {
          double wkill = 0.0;
          for (int jd = 0; jd < idiscu; jd++) {
            int iw = -1;
            for (int je = 0; je < mcnt; je++)
              if (ix[je] != 0 && (iw == -1 || w[je] >= wkill)) { iw = je; wkill = w[je]; }
            if (iw >= 0) ix[iw] = 0;
          }
        }
        im = 0;
        for (int je = 0; je < mcnt; je++)
          if (ix[je] != 0) { w[im] = w[je]; we[im] = we[je]; ix[im] = ix[je]; im++; }
        mcnt = im;
      }
      B->nab2 = B->nab1 + mcnt;   // remember the kept count
    }
    __syncwarp();
    mcnt = B->nab2 - B->nab1;
    if (mcnt != mbl) {
      if (lane == 0) set_status(p, MR3_EMISC);
      continue;
    }
    for (int k = lane; k < mbl; k += 32) {
      W[wb + k] = Wt[ib + k];
      Werr[wb + k] = Et[ib + k];
      Windex[wb + k] = It[ib + k];
      iblk[wb + k] = off + b;
      Wcopy[wb + k] = Wt[ib + k];
    }
  }
}

// Gaps after the initial approximations (SRC/mrrr_val.c:431-435).
__global__ void k_gaps_init(int N, const ProbDev *probs, const BlockDev *blocks, const int *iblk,
                            const double *W, const double *Werr, double *Wgap) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= N || iblk[s] < 0) return;
  const BlockDev *B = &blocks[iblk[s]];
  if (B->nbl < 2) return;
  const ProbDev *p = &probs[B->prob];
  int wend = B->wbgn + B->mbl - 1;
  if (s < wend) Wgap[s] = fmax(0.0, (W[s + 1] - Werr[s + 1]) - (W[s] + Werr[s]));
  else Wgap[s] = fmax(0.0, p->wu - (W[s] + Werr[s]));
}

// ------------------------------------------------------------------------
// Stage A4: root representation L D L^T = T - sigma I of each block
// (compute_root_rrr, bisection branch, SRC/mrrr_val.c:717-948).
// One warp per block; the factorisation tries are serial on lane 0.
// ------------------------------------------------------------------------
__global__ void __launch_bounds__(MR3_THREADS)
k_root(ProbDev *probs, BlockDev *blocks, double *D, double *E, const double2 *TP, double *Dt,
       double *Lt, const double *W, const double *Werr, const double *Wgap, double2 *RP,
       double2 *RQ) {
  ProbDev *p = &probs[blockIdx.x];
  if (p->trivial || p->jobz == MR3_JOB_C || p->status) return;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const double pivmin = p->pivmin, vlp = p->vl_out, vup = p->vu_out;
  for (int b = wid; b < p->nsplit; b += nw) {
    BlockDev *B = &blocks[p->off + b];
    const int nbl = B->nbl, mbl = B->mbl, ibgn = B->ibgn, iend = B->iend;
    if (nbl < 2 || mbl <= 0) continue;
    const int wbgn = B->wbgn, wend = wbgn + mbl - 1;
    const double gl = B->bgl, gu = B->bgu;
    // the dqds route (SRC/mrrr_val.c:409-412, 758-781): extremal eigenvalues
    // by dlarrk (lanes 0 and 1), quarter points of [isleft, isright]
    const bool dqds = mbl > 0.5 * nbl && !p->force_bis;
    const bool allno = p->irange == MR3_RANGE_A && !p->force_bis;
    double isleft, isright, spdiam, s1, s2;
    if (dqds || allno) {
      double w = 0.0, we = 0.0;
      if (lane < 2)
        dv_dlarrk(nbl, lane == 0 ? 1 : nbl, gl, gu, TP + ibgn, pivmin, sqrt(MR3_EPS), &w, &we);
      const double w0 = __shfl_sync(0xffffffffu, w, 0), e0 = __shfl_sync(0xffffffffu, we, 0);
      const double w1 = __shfl_sync(0xffffffffu, w, 1), e1 = __shfl_sync(0xffffffffu, we, 1);
      isleft = fmax(gl, (w0 - e0) - 100.0 * MR3_EPS * fabs(w0 - e0));
      isright = fmin(gu, (w1 + e1) + 100.0 * MR3_EPS * fabs(w1 + e1));
      spdiam = isright - isleft;
      s1 = isleft + 0.25 * spdiam;
      s2 = isright - 0.25 * spdiam;
    } else {
      isleft = fmax(gl, (W[wbgn] - Werr[wbgn]) - 100.0 * MR3_EPS * fabs(W[wbgn] - Werr[wbgn]));
      isright = fmin(gu, (W[wend] + Werr[wend]) + 100.0 * MR3_EPS * fabs(W[wend] - Werr[wend]));
      spdiam = gu - gl;
      const double tmp0 = fmin(isright, vup) - fmax(isleft, vlp);
      s1 = fmax(isleft, vlp) + 0.25 * tmp0;
      s2 = fmin(isright, vup) - 0.25 * tmp0;
    }
    int cnt = 0;
    if (mbl > 1 && lane < 2) {   // dlarrc('T'): lane 0 counts at s1, lane 1 at s2
      const double x = (lane == 0) ? s1 : s2;
      const double2 *tp = TP + ibgn;
      double piv = tp[0].x - x;
      cnt = (piv <= 0.0);
      for (int i = 0; i < nbl - 1; i++) {
        double ee = E[ibgn + i];
        double t = ee * ee;
        piv = (tp[i + 1].x - x) - t / piv;
        cnt += (piv <= 0.0);
      }
    }
    int lcnt = __shfl_sync(0xffffffffu, cnt, 0), rcnt = __shfl_sync(0xffffffffu, cnt, 1);
    int ok = 1;
    double sigma = 0.0;
    if (lane == 0) {
      int sgndef;
      if (mbl == 1) { sigma = gl; sgndef = 1; }
      else if ((lcnt - B->ilow) >= (B->iupp - rcnt)) {
        sigma = allno ? fmax(isleft, gl) : (dqds ? isleft : fmax(isleft, vlp));
        sgndef = 1;
      } else {
        sigma = allno ? fmin(isright, gu) : (dqds ? isright : fmin(isright, vup));
        sgndef = -1;
      }
      double tau;
      if (dqds) {
        tau = spdiam * MR3_EPS * nbl + 2.0 * pivmin;
        tau = fmax(tau, 2 * MR3_EPS * fabs(sigma));
      } else if (mbl > 1) {
        double clwdth = W[wend] + Werr[wend] - W[wbgn] - Werr[wbgn];
        double avgap = fabs(clwdth / (double)(wend - wbgn));
        if (sgndef > 0) { tau = fmax(Wgap[wbgn], avgap); tau *= 0.5; tau = fmax(tau, Werr[wbgn]); }
        else { tau = fmax(Wgap[wend - 1], avgap); tau *= 0.5; tau = fmax(tau, Werr[wend]); }
      } else {
        tau = Werr[wbgn];
      }
      ok = 0;
      for (int jtry = 0; jtry < MR3_MAX_TRY_ROOT; jtry++) {
        double dpiv = D[ibgn] - sigma;
        Dt[ibgn] = dpiv;
        double dmax = fabs(dpiv);
        for (int i = 0; i < nbl - 1; i++) {
          int j = ibgn + i;
          double ej = E[j];
          double inv = 1.0 / dpiv;
          double t0 = ej * inv;
          Lt[j] = t0;
          dpiv = (D[j + 1] - sigma) - t0 * ej;
          Dt[j + 1] = dpiv;
          dmax = fmax(dmax, fabs(dpiv));
        }
        bool norep = dmax > MR3_MAX_GROWTH * spdiam;
        if (dqds && !norep)   // dqds needs a definite representation
          for (int i = 0; i < nbl; i++)
            if (sgndef * Dt[ibgn + i] < 0.0) norep = true;
        if (!norep) { ok = 1; break; }
        if (jtry == MR3_MAX_TRY_ROOT - 2) {
          if (sgndef == 1) sigma = gl - 2.0 * spdiam * MR3_EPS * nbl - 2.0 * 2.0 * pivmin;
          else sigma = gu + 2.0 * spdiam * MR3_EPS * nbl + 2.0 * 2.0 * pivmin;
        } else if (jtry == MR3_MAX_TRY_ROOT - 1) {
          break;
        } else {
          sigma -= sgndef * tau;
          tau *= 2.0;
        }
      }
      if (!ok) set_status(p, MR3_EMISC);
      B->sigma = sigma;
      B->spdiam = spdiam;
      B->dqds = dqds;
      B->sgndef = sgndef;
    }
    ok = __shfl_sync(0xffffffffu, ok, 0);
    sigma = __shfl_sync(0xffffffffu, sigma, 0);
    __syncwarp();
    if (!ok) continue;
    // store the root, perturb it by 8*eps relative noise from dlarnv(2) with
    // seed (1,1,1,1) (SRC/mrrr_val.c:927-941), and pack its rows
    const unsigned long long seed = (1ULL << 36) | (1ULL << 24) | (1ULL << 12) | 1ULL;
    for (int i = lane; i < nbl; i += 32) {
      double dv = Dt[ibgn + i];
      double lv = (i < nbl - 1) ? Lt[ibgn + i] : sigma;
      if (mbl > 1) {
        if (i < nbl - 1) {
          dv *= 1.0 + MR3_EPS * 8.0 * dv_lcg_uniform(seed, (unsigned long long)(i + 1));
          lv *= 1.0 + MR3_EPS * 8.0 * dv_lcg_uniform(seed, (unsigned long long)(i + 1 + nbl));
        } else {
          dv *= 1.0 + MR3_EPS * 8.0 * dv_lcg_uniform(seed, (unsigned long long)(2 * nbl));
        }
      }
      D[ibgn + i] = dv;
      E[ibgn + i] = lv;
      if (i < nbl - 1) {
        double ld = dv * lv;
        RP[ibgn + i] = make_double2(dv, ld * lv);
        RQ[ibgn + i] = make_double2(lv, ld);
      } else {
        RP[ibgn + i] = make_double2(dv, 0.0);
        RQ[ibgn + i] = make_double2(sigma, 0.0);
      }
    }
  }
}

// ------------------------------------------------------------------------
// Stage A5: refine the approximations w.r.t. the root representation
// (refine_eigval_approx, unchunked dlarrb, SRC/mrrr_val.c:992-1082).
// ------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long refine_root_body(int s, const ProbDev *probs,
                                                               const BlockDev *blocks,
                                                               const int *iblk, const double2 *RP,
                                                               double *W, double *Werr,
                                                               const double *Wgap, Tol tol) {
  if (iblk[s] < 0) return 0;
  const BlockDev *B = &blocks[iblk[s]];
  const ProbDev *p = &probs[B->prob];
  if (p->status || B->nbl < 2 || B->dqds) return 0;
  const bool onlyW = (p->jobz == MR3_JOB_N);   // rtol1 = rtol2 = 4 eps (SRC/mrrr.c:230-232)
  const int II = s - B->wbgn + 1;
  const int i = B->ilow + II - 1;
  double w = W[s] - B->sigma;
  double werr = Werr[s] + fabs(w) * MR3_EPS;
  const double rgap = Wgap[s];
  const double lgap = (II > 1) ? Wgap[s - 1] : rgap;
  const int maxitr = dv_itmax(B->spdiam + p->pivmin, p->pivmin);
  const double rtol1 = onlyW ? 4.0 * MR3_EPS : tol.rtol1;
  const double rtol2 = onlyW ? 4.0 * MR3_EPS : tol.rtol2;
  int nc = 0;
  dv_dlarrb_one<1>(B->nbl, RP + B->ibgn, 1, i, II == 1, II > 1, rgap, lgap, rtol1, rtol2, p->pivmin,
                maxitr, B->nbl, &w, &werr, &nc);
  W[s] = w;
  Werr[s] = werr;
  return (unsigned long long)nc * (unsigned long long)B->nbl;
}

template <bool TREE>
__global__ void LB_REF
k_refine_root(int N, int L, const ProbDev *probs, const BlockDev *blocks, const int *iblk,
              const double2 *RP, double *W, double *Werr, const double *Wgap, Tol tol,
              unsigned long long *stats) {
  const long long gt = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  unsigned long long work = 0;
  if (!TREE) {
    if (gt < N) work = refine_root_body((int)gt, probs, blocks, iblk, RP, W, Werr, Wgap, tol);
  } else if (gt / L < N) {
    // L lanes per eigenvalue (few eigenvalues: single large problems)
    const int s = (int)(gt / L);
    const bool ok = iblk[s] >= 0;
    const BlockDev *B = ok ? &blocks[iblk[s]] : nullptr;
    const ProbDev *p = ok ? &probs[B->prob] : nullptr;
    if (ok && !p->status && B->nbl >= 2 && !B->dqds) {
      const bool onlyW = (p->jobz == MR3_JOB_N);
      const int II = s - B->wbgn + 1;
      const int i = B->ilow + II - 1;
      double w = W[s] - B->sigma;
      double werr = Werr[s] + fabs(w) * MR3_EPS;
      const double rgap = Wgap[s];
      const double lgap = (II > 1) ? Wgap[s - 1] : rgap;
      const int maxitr = dv_itmax(B->spdiam + p->pivmin, p->pivmin);
      const double rtol1 = onlyW ? 4.0 * MR3_EPS : tol.rtol1;
      const double rtol2 = onlyW ? 4.0 * MR3_EPS : tol.rtol2;
      int nc = 0;
      dv_dlarrb_tree(L, B->nbl, RP + B->ibgn, 1, i, II == 1, II > 1, rgap, lgap, rtol1, rtol2,
                     p->pivmin, maxitr, B->nbl, &w, &werr, &nc);
      if ((gt % L) == 0) {
        W[s] = w;
        Werr[s] = werr;
        work = (unsigned long long)nc * (unsigned long long)B->nbl;
      }
    }
  }
  stat_add(stats, KID_REFROOT * 4 + 1, work);
}

// The eigenvalues of a dqds block (SRC/mrrr_val.c:459-506): one thread per
// block builds the qd array of its definite root representation in qd
// (4 doubles per row of the block), runs dqds, and writes the wanted ones,
// shifted as the refined ones are, with Werr = 4 log(nbl) eps |W|.
__global__ void k_dqds(int N, ProbDev *probs, const BlockDev *blocks, const int *blk_of_row,
                       const double *D, const double *E, double *W, double *Werr, double *qd) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= N) return;
  const BlockDev *B = &blocks[blk_of_row[g]];
  if (g != B->ibgn || !B->dqds || B->nbl < 2 || B->mbl <= 0) return;
  ProbDev *p = &probs[B->prob];
  if (p->status || p->trivial || p->jobz == MR3_JOB_C) return;
  const int nbl = B->nbl, ibgn = B->ibgn;
  double *z = qd + 4 * (size_t)ibgn;
  for (int i = 0; i < nbl - 1; i++) {
    z[2 * i] = fabs(D[ibgn + i]);
    z[2 * i + 1] = E[ibgn + i] * E[ibgn + i] * z[2 * i];
  }
  z[2 * (nbl - 1)] = fabs(D[B->iend]);
  z[2 * (nbl - 1) + 1] = 0.0;
  int info = 0;
  dv_dlasq2(nbl, z, &info);
  if (info != 0) { set_status(p, MR3_EMISC); return; }
  const double rtol = 4.0 * dv_log((double)nbl) * MR3_EPS;
  for (int i = B->ilow, je = B->wbgn; i <= B->iupp; i++, je++) {
    const double w = B->sgndef > 0 ? z[nbl - i] : -z[i - 1];
    W[je] = w;
    Werr[je] = rtol * fabs(w);
  }
}

// Final gaps of the root refinement (dlarrb loop 111) or of a dqds block, and
// the last gap of the block (SRC/mrrr_val.c:1080-1082).
__global__ void k_gaps_root(int N, const ProbDev *probs, const BlockDev *blocks, const int *iblk,
                            const double *W, const double *Werr, double *Wgap) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= N || iblk[s] < 0) return;
  const BlockDev *B = &blocks[iblk[s]];
  const ProbDev *p = &probs[B->prob];
  if (p->status || B->nbl < 2) return;
  int wend = B->wbgn + B->mbl - 1;
  // dlarrb's loop 111 subtracts term by term; the dqds branch groups the
  // bounds (SRC/mrrr_val.c:501-503)
  if (s < wend) Wgap[s] = B->dqds ? fmax(0.0, (W[s + 1] - Werr[s + 1]) - (W[s] + Werr[s]))
                                  : fmax(0.0, W[s + 1] - Werr[s + 1] - W[s] - Werr[s]);
  else Wgap[s] = fmax(0.0, (p->vu_out - B->sigma) - (W[s] + Werr[s]));
}

// ------------------------------------------------------------------------
// Range I: drop surplus eigenvalues found near wl/wu
// (SRC/mrrr_val.c:515-626).  One thread per problem; runs only when the
// blocks together produced more than nvals values.
// ------------------------------------------------------------------------
__global__ void k_discard(ProbDev *probs, int nprob, BlockDev *blocks, double *W, double *Werr,
                          double *Wgap, int *Windex, int *iblk, double *Wcopy) {
  int pi = blockIdx.x * blockDim.x + threadIdx.x;
  if (pi >= nprob) return;
  ProbDev *p = &probs[pi];
  if (p->trivial || p->jobz == MR3_JOB_C || p->status) return;
  int mp = p->m;
  if (!(mp > p->nvals && p->irange == MR3_RANGE_I)) {
    if (mp < p->nvals) set_status(p, MR3_EMISC);
    return;
  }
  const int o = p->off;
  double *w = W + o, *we = Werr + o, *wg = Wgap + o, *wc = Wcopy + o;
  int *wi = Windex + o, *ib = iblk + o;
  int idiscl = p->il_out - 1 - p->nwl, idiscu = p->nwu - p->iu_out, im;
#define MOVE(dst, src) { w[dst] = w[src]; wc[dst] = wc[src]; we[dst] = we[src]; wg[dst] = wg[src]; \
                         wi[dst] = wi[src]; ib[dst] = ib[src]; }
  if (idiscl > 0) {
    im = 0;
    for (int je = 0; je < mp; je++) {
      if (wc[je] < p->wlu && idiscl > 0) idiscl--;
      else { MOVE(im, je); im++; }
    }
    mp = im;
  }
  if (idiscu > 0) {
    im = mp;
    for (int je = mp - 1; je >= 0; je--) {
      if (wc[je] > p->wul && idiscu > 0) idiscu--;
      else { im--; MOVE(im, je); }
    }
    int jee = 0;
    for (int je = im; je < mp; je++) { MOVE(jee, je); jee++; }
    mp -= im;
  }
  if (idiscl > 0 || idiscu > 0) {
    if (idiscl > 0) {
      double wkill = p->wu;
      for (int jd = 0; jd < idiscl; jd++) {
        int iw = -1;
        for (int je = 0; je < mp; je++)
          if (ib[je] >= 0 && (wc[je] < wkill || iw == -1)) { iw = je; wkill = wc[je]; }
        if (iw >= 0) ib[iw] = -2;
      }
    }
    if (idiscu > 0) {
      double wkill = p->wl;
      for (int jd = 0; jd < idiscu; jd++) {
        int iw = -1;
        for (int je = 0; je < mp; je++)
          if (ib[je] >= 0 && (wc[je] > wkill || iw == -1)) { iw = je; wkill = wc[je]; }
        if (iw >= 0) ib[iw] = -2;
      }
    }
    im = 0;
    for (int je = 0; je < mp; je++)
      if (ib[je] >= 0) { MOVE(im, je); im++; }
    mp = im;
  }
#undef MOVE
  for (int je = mp; je < p->m; je++) ib[je] = -1;
  p->m = mp;
  if (mp < p->nvals) set_status(p, MR3_EMISC);
  // block W ranges after the removal: recomputed from iblk (SRC/mrrr_vec.c:335-338)
  for (int b = 0; b < p->nsplit; b++) blocks[o + b].mbl = 0;
  for (int je = 0; je < mp; je++) {
    BlockDev *B = &blocks[ib[je]];
    if (B->mbl == 0) B->wbgn = o + je;
    B->mbl++;
  }
}

// ------------------------------------------------------------------------
// Eigenvalues only: W += sigma of the block (SRC/mrrr.c:262-269).
// ------------------------------------------------------------------------
__global__ void k_shift_w(int N, const ProbDev *probs, const BlockDev *blocks, const int *iblk,
                          const double *E, double *W) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= N || iblk[s] < 0) return;
  const BlockDev *B = &blocks[iblk[s]];
  const ProbDev *p = &probs[B->prob];
  if (p->status || p->jobz != MR3_JOB_N) return;
  W[s] += E[B->iend];
}

// refine_to_highrac (SRC/mrrr.c:452-520): dlarrj on the scaled input T,
// one thread per eigenvalue.
__global__ void k_highrac(int N, const ProbDev *probs, const BlockDev *blocks, const int *iblk,
                          const int *Windex, const double2 *TPc, double *W, double *Werr) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= N || iblk[s] < 0) return;
  const BlockDev *B = &blocks[iblk[s]];
  const ProbDev *p = &probs[B->prob];
  if (p->status || !p->tryrac_out || p->jobz == MR3_JOB_C) return;
  // ilow = smallest local index of the block's values; values are stored in
  // increasing local index, so it is the index of the first one.
  const int i = Windex[B->wbgn] + (s - B->wbgn);
  const int maxitr = dv_itmax(p->spdiam + p->pivmin, p->pivmin);
  double w = W[s], we = Werr[s];
  dv_dlarrj_one(B->nbl, TPc + B->ibgn, i, 4.0 * MR3_EPS, maxitr, &w, &we);
  W[s] = w;
  Werr[s] = we;
}

__global__ void k_invscale(int N, const ProbDev *probs, const BlockDev *blocks, const int *iblk,
                           double *W) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= N || iblk[s] < 0) return;
  const ProbDev *p = &probs[blocks[iblk[s]].prob];
  if (p->status || p->scale == 1.0) return;
  W[s] = (1.0 / p->scale) * W[s];
}

// ------------------------------------------------------------------------
// Sorting: per-problem bottom-up merge sort of (key, sec, idx) by the
// lexicographic order, one element per thread and pass.
// ------------------------------------------------------------------------
struct SortRec {
  double key;
  long long sec;
  int idx, pad;
};
__device__ __forceinline__ bool rec_less(const SortRec &a, const SortRec &b) {
  if (a.key < b.key) return true;
  if (a.key > b.key) return false;
  if (a.sec != b.sec) return a.sec < b.sec;
  return a.idx < b.idx;
}
__global__ void k_merge_pass(int N, const ProbDev *probs, const int *prob_of_slot, const SortRec *in,
                             SortRec *out, int width, int want_job, const int *flag) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= N) return;
  int pi = prob_of_slot[s];
  if (pi < 0) return;
  const ProbDev *p = &probs[pi];
  if (p->trivial || p->status || p->jobz != want_job) return;
  if (flag && !flag[pi]) return;
  int m = p->m, o = p->off, k = s - o;
  if (k >= m) return;
  int run0 = (k / (2 * width)) * (2 * width);
  int a0 = run0, a1 = min(run0 + width, m), b1 = min(run0 + 2 * width, m);
  SortRec r = in[s];
  int pos;
  if (k < a1) {   // element of run A: count run-B elements smaller
    int lo = a1, hi = b1;
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if (rec_less(in[o + mid], r)) lo = mid + 1; else hi = mid;
    }
    pos = run0 + (k - a0) + (lo - a1);
  } else {        // element of run B: count run-A elements smaller
    int lo = a0, hi = a1;
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if (rec_less(in[o + mid], r)) lo = mid + 1; else hi = mid;
    }
    pos = run0 + (k - a1) + (lo - a0);
  }
  out[o + pos] = r;
}

// Keys of init_zindex (SRC/mrrr_vec.c:380-416): the running maximum of
// W + sigma inside each block; one warp per block.
__global__ void k_zkeys(ProbDev *probs, const BlockDev *blocks, const double *W, const double *E,
                        const int *Windex, SortRec *rec) {
  ProbDev *p = &probs[blockIdx.x];
  if (p->trivial || p->status || p->jobz != MR3_JOB_V) return;
  const int o = p->off;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const double ninf = -__longlong_as_double(0x7ff0000000000000LL);
  for (int b = wid; b < p->nsplit; b += nw) {
    const BlockDev *B = &blocks[o + b];
    if (B->mbl <= 0) continue;
    const double sigma = E[B->iend];
    double run = ninf;
    for (int c = 0; c < B->mbl; c += 32) {
      const int k = c + lane;
      double v = (k < B->mbl) ? W[B->wbgn + k] + sigma : ninf;
      for (int sh = 1; sh < 32; sh <<= 1) {
        double u = __shfl_up_sync(0xffffffffu, v, sh);
        if (lane >= sh) v = fmax(v, u);
      }
      v = fmax(v, run);
      if (k < B->mbl) {
        const int s = B->wbgn + k;
        rec[s].key = v;
        rec[s].sec = ((long long)Windex[s] << 32) | (long long)b;
        rec[s].idx = s - o;
      }
      run = __shfl_sync(0xffffffffu, v, 31);
    }
  }
}

// Keys for the final ascending sort of eigenvalues-only results (qsort in
// SRC/mrrr.c:284) and of the bubble fix-up of sort_eigenpairs
// (SRC/mrrr.c:560-585), which yields the stable order by value.
__global__ void k_wkeys(int N, const ProbDev *probs, const int *prob_of_slot, const double *Wv,
                        SortRec *rec, int want_job, const int *flag) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= N) return;
  int pi = prob_of_slot[s];
  if (pi < 0) return;
  const ProbDev *p = &probs[pi];
  if (p->trivial || p->status || p->jobz != want_job) return;
  if (flag && !flag[pi]) return;
  int k = s - p->off;
  if (k >= p->m) return;
  rec[s].key = Wv[s];
  rec[s].sec = 0;
  rec[s].idx = k;
}

__global__ void k_zindex_from_sorted(int N, const ProbDev *probs, const int *prob_of_slot,
                                     const SortRec *rec, int *Zindex) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= N) return;
  int pi = prob_of_slot[s];
  if (pi < 0) return;
  const ProbDev *p = &probs[pi];
  int k = s - p->off;
  if (k >= p->m || p->jobz != MR3_JOB_V || p->status) return;
  Zindex[p->off + rec[s].idx] = k;
}

// ------------------------------------------------------------------------
// Stage B, level 0: one cluster per block (init_workQ, SRC/mrrr_vec.c:304-374,
// and the depth-0 branch of refine_eigvals, SRC/process_cluster.c:278-297).
// ------------------------------------------------------------------------
__global__ void k_level0(ProbDev *probs, BlockDev *blocks, const double *E, const double2 *gers,
                         double *W, const double *Werr, double *Wsh, ClusterDev *cl,
                         LevelCounters *lc, SngCounters *sc, int *unit_list) {
  ProbDev *p = &probs[blockIdx.x];
  if (p->trivial || p->status || p->jobz != MR3_JOB_V) return;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int b = wid; b < p->nsplit; b += nw) {
    BlockDev *B = &blocks[p->off + b];
    if (B->mbl <= 0) continue;
    if (B->nbl == 1) {   // the eigenvector of a 1x1 block is a unit vector
      if (lane == 0) unit_list[atomicAdd(&sc->n_unit, 1)] = B->wbgn;
      continue;
    }
    const double sigma = E[B->iend];
    const int wb = B->wbgn, we = wb + B->mbl - 1;
    const double lgap = fmax(0.0, (W[wb] + sigma) - Werr[wb] - p->vl_out);
    // spectral diameter of the block as refine_eigvals computes it at depth 0:
    // discs of its first row and of rows bl_begin+1 .. bl_end-1
    double gl = gers[B->ibgn].x, gu = gers[B->ibgn].y;
    for (int i = B->ibgn + 1 + lane; i < B->iend; i += 32) {
      gl = fmin(gl, gers[i].x);
      gu = fmax(gu, gers[i].y);
    }
    gl = warp_min(gl);
    gu = warp_max(gu);
    __syncwarp();
    for (int s = wb + lane; s <= we; s += 32) {
      Wsh[s] = W[s];
      W[s] = W[s] + sigma;
    }
    if (lane == 0) {
      B->bl_spdiam = gu - gl;
      int c = atomicAdd(&lc->n_cl, 1);
      ClusterDev C;
      C.begin = wb; C.end = we; C.depth = 0; C.blk = p->off + b;
      C.bl_spdiam = gu - gl; C.lgap = lgap; C.par_off = -1; C.pG = 1; C.pg = 0;
      C.grp_off = -1; C.G = 1; C.g = 0;
      C.par_sigma = sigma; C.sigma = sigma; C.tau = 0.0;
      cl[c] = C;
    }
  }
}

// ------------------------------------------------------------------------
// Child representation of each cluster of depth >= 1
// (compute_new_rrr, SRC/process_cluster.c:105-235).  One warp per cluster.
// ------------------------------------------------------------------------
// Parent representation of a cluster: rows P[i*ps], Q[i*ps].
__device__ __forceinline__ void par_rrr(const ClusterDev &C, const BlockDev &B, const double2 *RP,
                                        const double2 *RQ, const double *arena,
                                        const double2 **P, const double2 **Q, int *ps) {
  if (C.par_off < 0) { *P = RP + B.ibgn; *Q = RQ + B.ibgn; *ps = 1; }
  else {
    *P = reinterpret_cast<const double2 *>(arena + C.par_off) + C.pg;
    *Q = reinterpret_cast<const double2 *>(arena + C.par_off + 2LL * B.nbl * C.pG) + C.pg;
    *ps = C.pG;
  }
}

// The cluster's own representation (the root for depth 0).
__device__ __forceinline__ void own_rrr(const ClusterDev &C, const BlockDev &B, const double2 *RP,
                                        const double2 *RQ, const double *arena,
                                        const double2 **P, const double2 **Q, int *ps) {
  if (C.depth == 0) { *P = RP + B.ibgn; *Q = RQ + B.ibgn; *ps = 1; }
  else {
    *P = reinterpret_cast<const double2 *>(arena + C.grp_off) + C.g;
    *Q = reinterpret_cast<const double2 *>(arena + C.grp_off + 2LL * B.nbl * C.G) + C.g;
    *ps = C.G;
  }
}

// (a) the two extremal eigenvalues of each cluster refined to full accuracy
// (dlarrb with RQtol, SRC/process_cluster.c:170-195), one thread per end.
// Both calls see a zero right gap, so their convergence test does not depend
// on any other gap and the two ends are independent.
template <bool TREE>
__global__ void LB_REF
k_cl_ext(int ncl, int L, const ClusterDev *cl, const ProbDev *probs, const BlockDev *blocks,
         const double2 *RP, const double2 *RQ, const double *arena_prev, const double *Wsh,
         const double *Werr, const int *Windex, double *xw, double *xe, Tol tol,
         unsigned long long *stats) {
  // L lanes per cluster end (L = 1: a thread; L >= 4: dv_dlarrb_tree, for
  // launches with few clusters, where the sequential steps are the cost)
  const long long gt = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const bool valid = gt / L < 2LL * ncl;
  const int t = valid ? (int)(gt / L) : 2 * ncl - 1;   // spare lanes mirror the last end
  const int w = t >> 1;
  unsigned long long work = 0;
  {
    const ClusterDev C = cl[w];
    const BlockDev &B = blocks[C.blk];
    const ProbDev *p = &probs[B.prob];
    const int nb = B.nbl;
    const double2 *Pp, *Qp;
    int ps;
    par_rrr(C, B, RP, RQ, arena_prev, &Pp, &Qp, &ps);
    const int sx = (t & 1) ? C.end : C.begin;
    const int i = Windex[sx], II = i - (Windex[C.begin] - 1);
    const int maxitr = dv_itmax(C.bl_spdiam + p->pivmin, p->pivmin);
    double wv = Wsh[sx], ev = Werr[sx];
    int nc = 0;
    if (!TREE) {
      if (valid)
        dv_dlarrb_one<MR3_U>(nb, Pp, ps, i, 1, II > 1, 0.0, 0.0, tol.rqtol, tol.rqtol, p->pivmin,
                             maxitr, nb, &wv, &ev, &nc);
    } else {
      dv_dlarrb_tree(L, nb, Pp, ps, i, 1, II > 1, 0.0, 0.0, tol.rqtol, tol.rqtol, p->pivmin, maxitr,
                     nb, &wv, &ev, &nc);
    }
    if (valid && (gt % L) == 0) {
      xw[t] = wv;
      xe[t] = ev;
      work = (unsigned long long)nc * nb;
    }
  }
  stat_add(stats, KID_NEWRRR * 4 + 1, work);
}

// (b) child representation by dlarrf (SRC/process_cluster.c:197-210), one
// thread per cluster, after storing the refined extremes and the gap right of
// the first eigenvalue (computed against its neighbour's value before the
// second extreme was refined).
// PAIR (launches with few clusters, where each cluster's sweeps are the
// cost): two lanes per cluster, the left and right shifts of each try swept
// at once (dv_dlarrf<true>); the even lane writes the results.
template <bool PAIR>
__global__ void LB_RRF
k_cl_rrf(int ncl, ClusterDev *cl, const ProbDev *probs, const BlockDev *blocks, const double2 *RP,
         const double2 *RQ, const double *arena_prev, double *arena_cur, const double *xw,
         const double *xe, double *Wsh, double *Werr, double *Wgap, unsigned long long *stats) {
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int w = PAIR ? gt >> 1 : gt;
  const bool lead = !PAIR || (gt & 1) == 0;
  unsigned long long work = 0;
  if (w < ncl) {
    const ClusterDev C = cl[w];
    const BlockDev &B = blocks[C.blk];
    const ProbDev *p = &probs[B.prob];
    const int nb = B.nbl, cb = C.begin, ce = C.end;
    const double2 *Pp, *Qp;
    int ps;
    par_rrr(C, B, RP, RQ, arena_prev, &Pp, &Qp, &ps);
    double *grp = arena_cur + C.grp_off;
    const long long nG = (long long)nb * C.G;
    double *dplus = grp + 4 * nG + C.g, *lplus = grp + 5 * nG + C.g, *wk = grp + 6 * nG + C.g;
    const double w0 = xw[2 * w], e0 = xe[2 * w], w1 = xw[2 * w + 1], e1 = xe[2 * w + 1];
    const double nw_ = Wsh[cb + 1], ne_ = Werr[cb + 1];
    if (PAIR) __syncwarp(3u << ((threadIdx.x & 31) & ~1));   // both lanes read nw_, ne_ first
    if (lead) {
      Wgap[cb] = fmax(0.0, (nw_ - ne_) - (w0 + e0));
      Wsh[cb] = w0; Werr[cb] = e0;
      Wsh[ce] = w1; Werr[ce] = e1;
    }
    if (PAIR) __syncwarp(3u << ((threadIdx.x & 31) & ~1));
    const double tau = dv_dlarrf<PAIR>(nb, Pp, Qp, ps, ce - cb + 1, Wsh + cb, Wgap + cb,
                                       Werr + cb, C.bl_spdiam, C.lgap, Wgap[ce], p->pivmin, dplus,
                                       lplus, wk, C.G);
    if (lead) {
      cl[w].tau = tau;
      cl[w].sigma = C.par_sigma + tau;
      work = 2ull * nb;
    }
  }
  stat_add(stats, KID_NEWRRR * 4 + 3, work);
}

// (c) shift the cluster's eigenvalues and errors by tau
// (SRC/process_cluster.c:212-218) and pack the new representations' rows;
// one CTA per sibling group, rows of the group's members interleaved.
__global__ void k_cl_pack(int ncl, const ClusterDev *cl, const BlockDev *blocks, double *arena_cur,
                          double *Wsh, double *Werr, int *cl_of_slot, int *lvl_of_slot, int level,
                          int *rl_n) {
  for (int w = blockIdx.x; w < ncl; w += gridDim.x) {
    const ClusterDev L0 = cl[w];
    if (L0.g != 0) continue;   // the group's first member packs the group
    const int G = L0.G, nb = blocks[L0.blk].nbl;
    const long long nG = (long long)nb * G;
    double *grp = arena_cur + L0.grp_off;
    double2 *Pn = reinterpret_cast<double2 *>(grp);
    double2 *Qn = reinterpret_cast<double2 *>(grp + 2 * nG);
    const double *dplus = grp + 4 * nG, *lplus = grp + 5 * nG;
    for (int m = 0; m < G; m++) {
      const ClusterDev C = cl[w + m];
      const double tau = C.tau;
      for (int k = C.begin + threadIdx.x; k <= C.end; k += blockDim.x) {
        double f = 3.0 * MR3_EPS * fabs(Wsh[k]);
        double x = Wsh[k] - tau;
        Wsh[k] = x;
        f += 4.0 * MR3_EPS * fabs(x);
        Werr[k] += f;
        cl_of_slot[k] = w + m;
        lvl_of_slot[k] = level;
      }
      // the level's refinement list is built in slot order from
      // lvl_of_slot afterwards (k_rl_*); here only its length
      if (threadIdx.x == 0) atomicAdd(rl_n, C.end - C.begin + 1);
    }
    for (long long idx = threadIdx.x; idx < nG; idx += blockDim.x) {
      const int i = (int)(idx / G);
      double dv = dplus[idx];
      if (i < nb - 1) {
        double lv = lplus[idx];
        double ld = dv * lv;
        Pn[idx] = make_double2(dv, ld * lv);
        Qn[idx] = make_double2(lv, ld);
      } else {
        Pn[idx] = make_double2(dv, 0.0);
        Qn[idx] = make_double2(cl[w + (int)(idx % G)].sigma, 0.0);
      }
    }
  }
}

// Refinement of a level's clusters w.r.t. their new representation
// (refine_eigvals without R-tasks, SRC/process_cluster.c:394-428).
__device__ __forceinline__ unsigned long long refine_cl_body(
    int s, const ClusterDev *cl, const ProbDev *probs, const BlockDev *blocks,
    const double *arena_cur, double *Wsh, double *Werr, const double *Wgap, const int *Windex,
    const int *cl_of_slot, const int *lvl_of_slot, int level, Tol tol) {
  if (lvl_of_slot[s] != level) return 0;
  const ClusterDev C = cl[cl_of_slot[s]];
  const BlockDev &B = blocks[C.blk];
  const ProbDev *p = &probs[B.prob];
  const int pidx = Windex[C.begin], i = Windex[s], II = i - (pidx - 1);
  const double2 *P, *Q;
  int ps;
  own_rrr(C, B, nullptr, nullptr, arena_cur, &P, &Q, &ps);
  const double rgap = Wgap[s];
  const double lgap = (II > 1) ? Wgap[s - 1] : rgap;
  const int maxitr = dv_itmax(C.bl_spdiam + p->pivmin, p->pivmin);
  double w = Wsh[s], e = Werr[s];
  int nc = 0;
  dv_dlarrb_one<MR3_U>(B.nbl, P, ps, i, i == pidx, II > 1, rgap, lgap, tol.rtol1, tol.rtol2, p->pivmin,
                maxitr, B.nbl, &w, &e, &nc);
  Wsh[s] = w;
  Werr[s] = e;
  return (unsigned long long)nc * (unsigned long long)B.nbl;
}

// Threads per SM that the tree forms may fill (a launch of few intervals
// gets as many lanes per interval as fit; more than the resident threads
// run in waves, which the tree's steps per count outweigh)
#ifndef MR3_TREE_BUDGET
#define MR3_TREE_BUDGET 2048
#endif

// Lanes per interval for a launch of `items` independent dlarrb intervals:
// a thread each when they fill the GPU, else groups of 4..32 lanes running
// the tree bisection (the same intervals, fewer sequential sweeps).
__host__ __device__ __forceinline__ int tree_lanes(long long items, long long lanes,
                                                   int maxL = 32) {
  if (maxL < 4) return 1;
  int L = maxL > 32 ? 32 : maxL;
  while (L > 4 && items * L > lanes) L >>= 1;
  return items * L > lanes ? 1 : L;
}

template <bool TREE>
__global__ void LB_REF
k_refine_cl(const int *rl, const int *rl_n, const ClusterDev *cl, const ProbDev *probs,
            const BlockDev *blocks, const double *arena_cur, double *Wsh, double *Werr,
            const double *Wgap, const int *Windex, const int *cl_of_slot, const int *lvl_of_slot,
            int level, Tol tol, long long lanes, int tree_max, unsigned long long *stats) {
  const int cnt = *rl_n;
  unsigned long long work = 0;
  const int L0 = cnt > 0 ? tree_lanes(cnt, lanes, tree_max) : 1;
  if (cnt > 0 && (L0 > 1) == TREE) {   // the other instantiation has the other form
    const int L = L0;
    const long long gt = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long per = ((long long)gridDim.x * blockDim.x) / L;
    for (long long b0 = 0; b0 < cnt; b0 += per) {
      const long long it = b0 + gt / L;
      const bool valid = it < cnt;
      const int s = rl[valid ? it : cnt - 1];
      if (!TREE) {
        if (valid)
          work += refine_cl_body(s, cl, probs, blocks, arena_cur, Wsh, Werr, Wgap, Windex,
                                 cl_of_slot, lvl_of_slot, level, tol);
        continue;
      }
      const ClusterDev C = cl[cl_of_slot[s]];
      const BlockDev &B = blocks[C.blk];
      const ProbDev *p = &probs[B.prob];
      const int pidx = Windex[C.begin], i = Windex[s], II = i - (pidx - 1);
      const double2 *P, *Q;
      int ps;
      own_rrr(C, B, nullptr, nullptr, arena_cur, &P, &Q, &ps);
      const double rgap = Wgap[s];
      const double lgap = (II > 1) ? Wgap[s - 1] : rgap;
      const int maxitr = dv_itmax(C.bl_spdiam + p->pivmin, p->pivmin);
      double w = Wsh[s], e = Werr[s];
      int nc = 0;
      dv_dlarrb_tree(L, B.nbl, P, ps, i, i == pidx, II > 1, rgap, lgap, tol.rtol1, tol.rtol2,
                     p->pivmin, maxitr, B.nbl, &w, &e, &nc);
      if (valid && (gt % L) == 0) {
        Wsh[s] = w;
        Werr[s] = e;
        work += (unsigned long long)nc * (unsigned long long)B.nbl;
      }
    }
  }
  stat_add(stats, KID_REFCL * 4 + 1, work);
}

// The level's refinement list in slot order: the slots that k_cl_pack
// marked with this level.  Consecutive threads of k_refine_cl then take
// neighbouring eigenvalues -- of one cluster, or of sibling clusters whose
// representations are interleaved row by row in the arena -- so that a
// warp's Sturm sweeps read common or adjacent rows, instead of the rows of
// a dozen unrelated representations.  Count per 1024 slots, exclusive scan,
// stable scatter.
#define RL_T 1024
__global__ void __launch_bounds__(256) k_rl_count(int N, const int *lvl, int level, int *bcnt) {
  __shared__ int red[8];
  const int base = blockIdx.x * RL_T;
  int c = 0;
  for (int q = 0; q < RL_T / 256; q++) {
    const int k = base + q * 256 + threadIdx.x;
    c += (k < N && lvl[k] == level);
  }
  c = __reduce_add_sync(0xffffffffu, c);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int a = 0;
    for (int w = 0; w < 8; w++) a += red[w];
    bcnt[blockIdx.x] = a;
  }
}

__global__ void __launch_bounds__(1024) k_rl_scan(int nblk, int *bcnt) {
  __shared__ int wsum[32];
  __shared__ int carry;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int b0 = 0; b0 < nblk; b0 += 1024) {
    const int b = b0 + threadIdx.x;
    const int a = b < nblk ? bcnt[b] : 0;
    int x = a;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[wid] = x;
    __syncthreads();
    if (wid == 0) {
      int v = wsum[lane];
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += y;
      }
      wsum[lane] = v;
    }
    __syncthreads();
    if (b < nblk) bcnt[b] = carry + (wid ? wsum[wid - 1] : 0) + x - a;
    __syncthreads();
    if (threadIdx.x == 0) carry += wsum[31];
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256) k_rl_scatter(int N, const int *lvl, int level,
                                                    const int *bcnt, int *rl) {
  __shared__ int wcnt[8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int base = blockIdx.x * RL_T;
  int pos = bcnt[blockIdx.x];
  for (int q = 0; q < RL_T / 256; q++) {
    const int k = base + q * 256 + threadIdx.x;
    const bool f = k < N && lvl[k] == level;
    const unsigned b = __ballot_sync(0xffffffffu, f);
    if (lane == 0) wcnt[wid] = __popc(b);
    __syncthreads();
    int before = 0, total = 0;
    for (int w = 0; w < 8; w++) {
      before += (w < wid) ? wcnt[w] : 0;
      total += wcnt[w];
    }
    if (f) rl[pos + before + __popc(b & ((1u << lane) - 1u))] = k;
    pos += total;
    __syncthreads();
  }
}

__global__ void k_gaps_cl(int N, const ClusterDev *cl, const double *Wsh, const double *Werr,
                          double *Wgap, double *W, const int *cl_of_slot, const int *lvl_of_slot,
                          int level) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= N || lvl_of_slot[s] != level) return;
  const ClusterDev C = cl[cl_of_slot[s]];
  if (s < C.end) Wgap[s] = fmax(0.0, Wsh[s + 1] - Werr[s + 1] - Wsh[s] - Werr[s]);
  W[s] = Wsh[s] + C.sigma;
}

// ------------------------------------------------------------------------
// Classification of a cluster's eigenvalues into singletons and child
// clusters (PMR_create_subtasks, SRC/process_cluster.c:438-629).  One warp
// per cluster.  Three launches: count (and reserve the children and their
// arena), allocate the singleton records of each sibling group contiguously
// and cut them into warp tasks, then write the records.
// ------------------------------------------------------------------------
struct ClsScratch {
  int *ns;          // singletons of each cluster
  int *soff;        // first singleton record of each cluster
  int *cbase;       // first child of each cluster in the next level's list
  long long *abase; // arena base of each cluster's children
};

// Child cluster number `rank` of `nc` children, all of block size nb: its
// group and its position in the group (groups of 32 consecutive children).
__device__ __forceinline__ void child_group(ClusterDev &c, int rank, int nc, int nb,
                                            long long a_base) {
  const int grp = rank >> 5;
  c.G = min(32, nc - 32 * grp);
  c.g = rank & 31;
  c.grp_off = a_base + 8LL * nb * 32 * grp;
}

// Children of a segment [first, last] of a depth-0 cluster with more than
// three members, split where the gap exceeds twice the average gap
// (SRC/process_cluster.c:542-577).  Returns their number; writes them if out.
__device__ int split_children(int first, int last, const ClusterDev &parent, double avggap,
                              const double *Wgap, ClusterDev proto, ClusterDev *out,
                              int crank, int nc, int nb, long long a_base) {
  int cnt = 0, cl_first = first;
  for (int k = first + 1; k < last; k++) {
    int cl_last;
    if (k == last - 1) cl_last = last;
    else if (k != cl_first && Wgap[k] > 2.0 * avggap) cl_last = k;
    else continue;
    if (out) {
      ClusterDev c = proto;
      c.begin = cl_first; c.end = cl_last;
      c.lgap = (cl_first == parent.begin) ? parent.lgap : Wgap[cl_first - 1];
      child_group(c, crank + cnt, nc, nb, a_base);
      out[crank + cnt] = c;
    }
    cnt++;
    cl_first = k + 1;
  }
  return cnt;
}

template <int PASS>
__global__ void __launch_bounds__(MR3_THREADS)
k_classify(int ncl, const ClusterDev *cl, const BlockDev *blocks, const double *Wsh,
           const double *Wgap, ClusterDev *cl_next, SngDev *sng, LevelCounters *lcn,
           ClsScratch xs, int cap) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= ncl) return;
  const ClusterDev C = cl[w];
  const BlockDev &B = blocks[C.blk];
  const int cb = C.begin, ce = C.end, depth = C.depth, nb = B.nbl;
  const double avggap = C.bl_spdiam / (nb - 1);
  ClusterDev proto;
  proto.begin = 0; proto.end = 0; proto.lgap = 0.0;
  proto.depth = depth + 1; proto.blk = C.blk; proto.bl_spdiam = C.bl_spdiam;
  proto.par_off = (depth == 0) ? -1 : C.grp_off;
  proto.pG = C.G; proto.pg = C.g;
  proto.par_sigma = C.sigma; proto.sigma = 0.0; proto.tau = 0.0;
  proto.grp_off = 0; proto.G = 1; proto.g = 0;
  int s_base = 0, c_base = 0, nc_tot = 0;
  long long a_base = 0;
  if (PASS == 1) {
    s_base = xs.soff[w]; c_base = xs.cbase[w]; a_base = xs.abase[w];
    nc_tot = -1;   // filled from the count of pass 0 below
  }
  int ns = 0, nc = 0, prev_end = cb - 1;
  // PASS 1 needs the total child count for the group sizes: recount first
  if (PASS == 1) {
    int tot = 0, pe = cb - 1;
    for (int c0 = cb; c0 <= ce; c0 += 32) {
      const int s = c0 + lane;
      bool flag = false;
      if (s <= ce) flag = (s == ce) || (Wgap[s] >= MR3_MIN_RELGAP * fabs(Wsh[s]));
      const unsigned bal = __ballot_sync(0xffffffffu, flag);
      const unsigned below = bal & ((1u << lane) - 1u);
      const int first = below ? (c0 + 31 - __clz(below)) + 1 : pe + 1;
      int nchild = 0;
      if (flag && s != first)
        nchild = (depth == 0 && s - first + 1 > 3)
                     ? split_children(first, s, C, avggap, Wgap, proto, nullptr, 0, 0, nb, 0)
                     : 1;
      for (int o = 16; o > 0; o >>= 1) nchild += __shfl_xor_sync(0xffffffffu, nchild, o);
      tot += nchild;
      pe = bal ? (c0 + 31 - __clz(bal)) : pe;
    }
    nc_tot = tot;
  }
  for (int c0 = cb; c0 <= ce; c0 += 32) {
    const int s = c0 + lane;
    bool flag = false;
    if (s <= ce) flag = (s == ce) || (Wgap[s] >= MR3_MIN_RELGAP * fabs(Wsh[s]));
    const unsigned bal = __ballot_sync(0xffffffffu, flag);
    const unsigned below = bal & ((1u << lane) - 1u);
    const int first = below ? (c0 + 31 - __clz(below)) + 1 : prev_end + 1;
    int is_sng = 0, nchild = 0;
    const bool split = flag && depth == 0 && (s - first + 1) > 3;
    if (flag) {
      if (s == first) is_sng = 1;
      else if (split)
        nchild = split_children(first, s, C, avggap, Wgap, proto, nullptr, 0, 0, nb, 0);
      else nchild = 1;
    }
    int sr = is_sng, cr = nchild;
    for (int o = 1; o < 32; o <<= 1) {
      int a = __shfl_up_sync(0xffffffffu, sr, o), b = __shfl_up_sync(0xffffffffu, cr, o);
      if (lane >= o) { sr += a; cr += b; }
    }
    if (PASS == 1 && flag) {
      const int srank = ns + sr - is_sng, crank = nc + cr - nchild;
      if (is_sng) {
        SngDev r;
        r.slot = s; r.cl = w;
        r.lgap = (s == cb) ? C.lgap : Wgap[s - 1];
        sng[s_base + srank] = r;
      } else if (split) {
        split_children(first, s, C, avggap, Wgap, proto, cl_next + c_base, crank, nc_tot, nb,
                       a_base);
      } else {
        ClusterDev c = proto;
        c.begin = first; c.end = s;
        c.lgap = (first == cb) ? C.lgap : Wgap[first - 1];
        child_group(c, crank, nc_tot, nb, a_base);
        cl_next[c_base + crank] = c;
      }
    }
    ns += __shfl_sync(0xffffffffu, sr, 31);
    nc += __shfl_sync(0xffffffffu, cr, 31);
    prev_end = bal ? (c0 + 31 - __clz(bal)) : prev_end;
  }
  if (PASS == 0 && lane == 0) {
    xs.ns[w] = ns;
    const int cb0 = atomicAdd(&lcn->n_cl, nc);
    // groups of 32 children; only the last group can be smaller
    const long long need = 8LL * nb * nc;
    const long long ab = (long long)atomicAdd(&lcn->arena_need, (unsigned long long)need);
    xs.cbase[w] = cb0;
    xs.abase[w] = ab;
    if (cb0 + nc > cap) atomicOr(&lcn->err, 1);
  }
}

// Per sibling group (led by the member with g == 0): reserve the group's
// singleton records contiguously, so that consecutive records share a block
// (and the size of their sweeps).  The level's list is ordered by block size,
// largest first (16 log2 buckets): a round's costliest chunks start first
// and the small ones fill in behind them.  PASS 0 counts per bucket, PASS 1
// reserves inside the buckets laid out by k_bucket_scan.
#define SNG_BUCKETS 16
__device__ __forceinline__ int size_bucket(int nb) {
  const int b = 31 - __clz(nb > 0 ? nb : 1);
  return b < SNG_BUCKETS ? b : SNG_BUCKETS - 1;
}

template <int PASS>
__global__ void k_group_tasks(int ncl, const ClusterDev *cl, const BlockDev *blocks, ClsScratch xs,
                              SngCounters *sc, int *bk, LevelCounters *lcn, int cap) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= ncl) return;
  const ClusterDev C = cl[w];
  if (C.g != 0) return;
  int tot = 0;
  for (int m = 0; m < C.G; m++) tot += xs.ns[w + m];
  if (tot == 0) return;
  const int b = size_bucket(blocks[C.blk].nbl);
  if (PASS == 0) {
    atomicAdd(&bk[b], tot);
    atomicAdd(&sc->n_sng, tot);
    return;
  }
  const int base = bk[SNG_BUCKETS + b] + atomicAdd(&bk[2 * SNG_BUCKETS + b], tot);
  if (base + tot > cap) { atomicOr(&lcn->err, 1); return; }
  int o = base;
  for (int m = 0; m < C.G; m++) { xs.soff[w + m] = o; o += xs.ns[w + m]; }
}

// bk[0..15]: counts per bucket; bk[16..31]: first record of each bucket,
// largest blocks first; bk[32..47]: fill counters (zeroed with the counts).
__global__ void k_bucket_scan(int *bk) {
  int run = 0;
  for (int b = SNG_BUCKETS - 1; b >= 0; b--) {
    bk[SNG_BUCKETS + b] = run;
    run += bk[b];
  }
}

// ------------------------------------------------------------------------
// Singletons (PMR_process_s_task, SRC/process_singleton.c:65-317), in
// rounds.  A singleton's Rayleigh-quotient loop is a sequence of dlar1v
// calls whose only carried state is a handful of scalars (SngState).  Each
// round gives every unfinished singleton of the level one dlar1v: persistent
// warps take 32 singletons at a time from the round's list, one lane each,
// and the singletons that need another call are compacted into the next
// round's list; those that need a bisection first (needBS) go to a list that
// k_sng_bisect serves between rounds.  So no lane waits for another lane's
// extra iterations, and the warps stay full in every round.
//
// A lane's dlar1v keeps only checkpoints (dv_r1c_*): each warp owns scratch
// of 3 x (nmax/CK_K + 1) x 32 doubles laid out [array][block][lane], and the
// lanes sweep the blocks by absolute index, so a checkpoint access is one
// coalesced 256-byte row.  Consecutive records of a list mostly share a
// block; a warp whose lanes hold blocks of different sizes sweeps the
// largest.  A call after a singleton's first writes z of its support to the
// lane's column of Z as it goes; when the vector is accepted the warp scales
// the support and zeroes the rows outside it in coalesced rows.  (A first
// call, practically never accepted, writes nothing; if it is accepted the
// next round repeats it and writes.)
// ------------------------------------------------------------------------
#define SNG_WARPS 8
#ifndef SNG_MINB
#define SNG_MINB 2     // resident round blocks per SM the register budget is sized for
#endif
#define SNG_ROUNDS (MR3_MAXITER + 1)   // MAXITER loop calls and the step-2 call
// The back-substitution of a round: each lane on its own rows from its own
// twist index (default), or the warp in lock-step through shared-memory z
// tiles written as coalesced column segments (MR3_SNG_LOCKSTEP=1).  The
// lock-step form sweeps the union of its lanes' ranges; with the localized
// supports of most eigenvectors that is many times each lane's own range.
#ifndef MR3_SNG_LOCKSTEP
#define MR3_SNG_LOCKSTEP 0
#endif
#if MR3_SNG_LOCKSTEP
#define SNG_TILE_BYTES (SNG_WARPS * 32 * 33 * (int)sizeof(double))   // k_sng_round's z tiles
#else
#define SNG_TILE_BYTES 0
#endif
enum { SF_USEDBS = 1, SF_USEDRQ = 2, SF_NEEDBS = 4, SF_STEP2 = 8, SF_REWRITE = 16 };

// Loop variables of one singleton between rounds
// (SRC/process_singleton.c:159-292: lambda, Wshifted[i], Werr[i], left,
// right, bstres, bstw, residual, gap, gaptol, r, k and the flags).
struct SngState {
  double lambda, wsh, werr, left, right, bstres, bstw, resid, gap, gaptol;
  int r, k, flags, pad;
};

__global__ void k_round_reset(SngCounters *sc, int in, int first) {
  sc->nin = first ? sc->n_sng : sc->act_n[in];
  sc->act_next[in] = 0;
  sc->bs_next = 0;
  if (first) { sc->mode = 0; sc->fin_ctas = 0; }
}

// Stable compaction of a round's list: entry j of the list leaves the round
// with flag[j] = 0 (finished), 1 (next round) or 2 (bisection first).  The
// survivors keep their order, so the warps of the next round again take
// neighbouring singletons (mostly of one block and one representation).
// The next round's list ordered within windows of LSORT_W entries by
// (cluster, twist index), so that the 32 lanes of a warp take neighbouring
// twist indices of one representation: the lock-step sweeps of a warp span
// its lanes' twist indices (stationary rows up to the largest, progressive
// rows down to the smallest), and neighbouring twists keep that span short.
// Each singleton's result does not depend on the order.  Bitonic sort of
// (cluster, twist, position) keys in shared memory, one window per block.
#define LSORT_W 4096
__global__ void __launch_bounds__(1024) k_list_sort(const SngCounters *sc, int out, int *act0,
                                                    int *act1, const SngDev *sng,
                                                    const SngState *sst) {
  __shared__ unsigned long long key[LSORT_W];
  __shared__ int val[LSORT_W];
  const int cnt = sc->act_n[out], start = blockIdx.x * LSORT_W;
  if (start >= cnt) return;
  int *A = out ? act1 : act0;
  const int m = min(LSORT_W, cnt - start);
  const unsigned cap = (1u << 22) - 1;
  for (int j = threadIdx.x; j < LSORT_W; j += blockDim.x) {
    unsigned long long k = ~0ull;
    if (j < m) {
      const int idx = A[start + j];
      val[j] = idx;
      const unsigned c = min((unsigned)sng[idx].cl, cap), r = min((unsigned)sst[idx].r, cap);
      k = ((unsigned long long)c << 34) | ((unsigned long long)r << 12) | (unsigned)j;
    }
    key[j] = k;
  }
  __syncthreads();
  for (int size = 2; size <= LSORT_W; size <<= 1)
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int t = threadIdx.x; t < LSORT_W / 2; t += blockDim.x) {
        const int lo = 2 * t - (t & (stride - 1)), hi = lo + stride;
        const unsigned long long a = key[lo], b = key[hi];
        if ((a > b) == ((lo & size) == 0)) { key[lo] = b; key[hi] = a; }
      }
      __syncthreads();
    }
  for (int j = threadIdx.x; j < m; j += blockDim.x) A[start + j] = val[key[j] & (LSORT_W - 1)];
}

#define LIST_T 1024   // entries per block: 256 threads x 4
__global__ void __launch_bounds__(256) k_list_count(const SngCounters *sc,
                                                    const unsigned char *flag, int *bcnt) {
  __shared__ int red[2][8];
  const int nin = sc->nin, base = blockIdx.x * LIST_T;
  int c1 = 0, c2 = 0;
  for (int q = 0; q < 4; q++) {
    const int j = base + threadIdx.x * 4 + q;
    if (j < nin) { const int f = flag[j]; c1 += f == 1; c2 += f == 2; }
  }
  for (int o = 16; o > 0; o >>= 1) {
    c1 += __shfl_xor_sync(0xffffffffu, c1, o);
    c2 += __shfl_xor_sync(0xffffffffu, c2, o);
  }
  if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = c1; red[1][threadIdx.x >> 5] = c2; }
  __syncthreads();
  if (threadIdx.x == 0) {
    int a = 0, b = 0;
    for (int w = 0; w < 8; w++) { a += red[0][w]; b += red[1][w]; }
    bcnt[2 * blockIdx.x] = a;
    bcnt[2 * blockIdx.x + 1] = b;
  }
}

// Exclusive scan of the block counts (one block of 1024 threads); the totals
// become the next list's length and the bisection list's length.
__global__ void __launch_bounds__(1024) k_list_scan(int nblk, SngCounters *sc, int *bcnt, int out,
                                                    int last_round, int finish_max, int iter_max) {
  __shared__ int wa[32], wb[32];
  __shared__ int carry[2];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (threadIdx.x == 0) { carry[0] = 0; carry[1] = 0; }
  __syncthreads();
  for (int b0 = 0; b0 < nblk; b0 += 1024) {
    const int b = b0 + threadIdx.x;
    const int a = b < nblk ? bcnt[2 * b] : 0, c = b < nblk ? bcnt[2 * b + 1] : 0;
    int ia = a, ic = c;
    for (int o = 1; o < 32; o <<= 1) {
      const int x = __shfl_up_sync(0xffffffffu, ia, o), y = __shfl_up_sync(0xffffffffu, ic, o);
      if (lane >= o) { ia += x; ic += y; }
    }
    if (lane == 31) { wa[wid] = ia; wb[wid] = ic; }
    __syncthreads();
    if (wid == 0) {
      int xa = wa[lane], xc = wb[lane];
      for (int o = 1; o < 32; o <<= 1) {
        const int x = __shfl_up_sync(0xffffffffu, xa, o), y = __shfl_up_sync(0xffffffffu, xc, o);
        if (lane >= o) { xa += x; xc += y; }
      }
      wa[lane] = xa; wb[lane] = xc;
    }
    __syncthreads();
    const int pa = carry[0] + (wid ? wa[wid - 1] : 0) + ia - a;
    const int pc = carry[1] + (wid ? wb[wid - 1] : 0) + ic - c;
    if (b < nblk) { bcnt[2 * b] = pa; bcnt[2 * b + 1] = pc; }
    __syncthreads();
    if (threadIdx.x == 0) { carry[0] += wa[31]; carry[1] += wb[31]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    sc->act_n[out] = carry[0];
    sc->bs_n = carry[1];
    if (last_round && (carry[0] | carry[1])) sc->err = 1;
    // a short list is finished in one launch, a warp per singleton (mode 1)
    // or a lane per singleton (mode 3: no more than a chunk per warp)
    const int left = carry[0] + carry[1];
    if (!last_round && sc->mode == 0 && left > 0) {
      if (left <= finish_max) sc->mode = 1;
      else if (left <= iter_max) sc->mode = 3;
    }
  }
}

__global__ void __launch_bounds__(256) k_list_scatter(int first, const SngCounters *sc,
                                                      const unsigned char *flag, const int *bcnt,
                                                      const int *act0, const int *act1, int in,
                                                      int *bsl) {
  __shared__ int wa[8], wb[8];
  const int nin = sc->nin, base = blockIdx.x * LIST_T;
  if (base >= nin) return;
  const int *Ain = in ? act1 : act0;
  int *Aout = const_cast<int *>(in ? act0 : act1);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int f[4], c1 = 0, c2 = 0;
  for (int q = 0; q < 4; q++) {
    const int j = base + threadIdx.x * 4 + q;
    f[q] = j < nin ? flag[j] : 0;
    c1 += f[q] == 1;
    c2 += f[q] == 2;
  }
  int i1 = c1, i2 = c2;
  for (int o = 1; o < 32; o <<= 1) {
    const int x = __shfl_up_sync(0xffffffffu, i1, o), y = __shfl_up_sync(0xffffffffu, i2, o);
    if (lane >= o) { i1 += x; i2 += y; }
  }
  if (lane == 31) { wa[wid] = i1; wb[wid] = i2; }
  __syncthreads();
  int p1 = bcnt[2 * blockIdx.x] + i1 - c1, p2 = bcnt[2 * blockIdx.x + 1] + i2 - c2;
  for (int w = 0; w < wid; w++) { p1 += wa[w]; p2 += wb[w]; }
  for (int q = 0; q < 4; q++) {
    const int j = base + threadIdx.x * 4 + q;
    if (f[q] == 0) continue;
    const int idx = first ? j : Ain[j];
    if (f[q] == 1) Aout[p1++] = idx; else bsl[p2++] = idx;
  }
}

// ITER (SngCounters.mode 3, a level's tail): every lane runs its singleton's
// remaining Rayleigh-quotient loop to the end in this launch -- one dlar1v
// call per pass of the warp, a bisection (SRC/process_singleton.c:178-192)
// by the whole warp with the tree bisection when a lane's step left its
// interval -- instead of one call per round.  A tail round lasts as long as
// the largest block's dlar1v whatever the list's length; here the tail's
// calls follow one another without the rounds' launches between them.
// Every call and state update is the one the rounds make (the same bits).
// The last block to finish empties the list (mode 2).
// KIND: SNG_LATER (rounds after the first), SNG_FIRST (the first round of a
// level: the state starts from the eigenvalue's refinement), SNG_ITER.
enum { SNG_LATER = 0, SNG_FIRST = 1, SNG_ITER = 2 };
template <int KIND>
__global__ void __launch_bounds__(SNG_WARPS * 32, SNG_MINB)
k_sng_round(int in, const SngDev *sng, const ClusterDev *cl, ProbDev *probs,
            const BlockDev *blocks, const double2 *RP, const double2 *RQ, const double *arena,
            double *W, double *Wsh, double *Werr, double *Wgap, const int *Windex,
            const int *Zindex, SngState *sst, const int *act0, const int *act1,
            unsigned char *flag, SngCounters *sc, double *scratch, long long nmax,
            int2 *done_list, int *tile_left, unsigned long long *stats) {
  constexpr bool FIRST = KIND == SNG_FIRST, ITER = KIND == SNG_ITER;
  if (ITER && sc->mode != 3) return;
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const long long gw = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nck = nmax / CK_K + 1;   // checkpoint blocks per lane
  r1c_ck ck;
  ck.S = scratch + gw * 3 * nck * 32 + lane;
  ck.I = ck.S + nck * 32;
  ck.P = ck.I + nck * 32;
  const int *Ain = in ? act1 : act0;
  const int nin = sc->nin;
  const double rqtol = 2.0 * MR3_EPS;
  __shared__ SngState sm_st[SNG_WARPS * 32];
#if MR3_SNG_LOCKSTEP
  extern __shared__ double ztile[];   // SNG_WARPS tiles of 32 x 33 doubles
#endif
  unsigned long long w_r1v = 0, w_sweep = 0, w_chunks = 0, w_neg = 0;
  for (;;) {
    int base = 0;
    if (lane == 0) base = atomicAdd(&sc->act_next[in], 32);
    base = __shfl_sync(full, base, 0);
    if (base >= nin) break;
    const bool active = base + lane < nin;
    // lanes without a singleton mirror the chunk's first one (valid
    // pointers) and do no work
    const int j = active ? base + lane : base;
    const int idx = FIRST ? j : Ain[j];
    const int s = sng[idx].slot;
    bool live = active;   // ITER: this lane's singleton is not finished yet
    do {
    int nb;
    double pivmin, lam_call, gaptol, bspd;
    const double2 *P, *Q;
    double *zcol;   // the eigenvector's column of Z at the block's first row
    int ps, r_in;
    bool usedBS, write;
    {
      // the loop state waits in shared memory while the sweeps run, so that
      // they have the registers to themselves
      const SngDev S = sng[idx];
      const ClusterDev C = cl[S.cl];
      const BlockDev &B = blocks[C.blk];
      nb = B.nbl;
      const ProbDev *pd = &probs[B.prob];
      pivmin = pd->pivmin;
      bspd = C.bl_spdiam;
      zcol = pd->Z + (size_t)Zindex[s] * pd->ldz + (B.ibgn - pd->off);
      own_rrr(C, B, RP, RQ, arena, &P, &Q, &ps);
      SngState st;
      if (FIRST) {
        st.lambda = Wsh[s]; st.wsh = st.lambda; st.werr = Werr[s];
        st.left = st.lambda - st.werr; st.right = st.lambda + st.werr;
        // the reference compares the eigenvalue index with the block's first
        // and last row (SRC/process_singleton.c:142-157); W slots and rows of
        // a problem start at the same offset, so the same comparison is s == row
        const double lgap = (s == B.ibgn) ? MR3_EPS * fmax(fabs(st.left), fabs(st.right)) : S.lgap;
        const double rgap = (s == B.iend) ? MR3_EPS * fmax(fabs(st.left), fabs(st.right)) : Wgap[s];
        st.gap = fmin(lgap, rgap);
        st.gaptol = (s == B.ibgn || s == B.iend) ? 0.0 : st.gap * MR3_EPS;
        st.bstres = 0.0; st.bstw = 0.0; st.resid = 0.0;
        st.r = 0; st.k = 1; st.flags = 0; st.pad = 0;
      } else {
        st = sst[idx];
      }
      sm_st[threadIdx.x] = st;
      usedBS = (st.flags & SF_USEDBS) != 0;
      lam_call = (st.flags & SF_STEP2) ? st.bstw : st.lambda;
      // a rewrite repeats the accepted first call (twist searched, r = 0)
      r_in = (st.flags & SF_REWRITE) ? 0 : st.r;
      gaptol = st.gaptol;
      // the first call of a Rayleigh-quotient iteration (no bisection
      // before it) is practically never accepted: its eigenvalue carries
      // the refinement's error, far above the acceptance test's tolerance.
      // Its vector is not written; in the rare case that it is accepted,
      // the next call repeats the identical call and writes the vector.
      write = (st.flags & (SF_REWRITE | SF_STEP2 | SF_USEDBS)) || st.k > 1;
    }
    r1c_state rs;
    rs.r = 0; rs.mingma = 0.0; rs.sawnan = false; rs.slowA = false; rs.slowB = false;
    int negc = 0;
    dv_r1c_factor(live, nb, lam_call, P, Q, ps, pivmin, !usedBS, r_in, ck, &negc, &rs);
    dlar1v_out o;
    o.isupp1 = 1; o.isupp2 = nb; o.nrminv = 0.0; o.r = 0; o.resid = 0.0; o.rqcorr = 0.0;
    // z of the support goes to the column unscaled; an accepted vector is
    // scaled below (z * nrminv, the reference's dscal after dlar1v)
#if MR3_SNG_LOCKSTEP
    dv_r1w_solve(live, nb, lam_call, P, Q, ps, pivmin, gaptol, rs.r, rs.sawnan, rs.slowA,
                 rs.slowB, ck.S, ck.P, rs.mingma, zcol, write, ztile + (threadIdx.x >> 5) * 32 * 33,
                 &o);
#else
    if (live)
      dv_r1c_solve(nb, lam_call, P, Q, ps, pivmin, gaptol, rs.r, rs.sawnan, rs.slowA, rs.slowB,
                   ck.S, ck.P, rs.mingma, write ? zcol : nullptr, 1.0, &o);
#endif
    SngState st = sm_st[threadIdx.x];
    const bool step2 = (st.flags & SF_STEP2) != 0;
    const bool rewrite = (st.flags & SF_REWRITE) != 0;
    const int nb_sweep = __reduce_max_sync(full, live ? nb : 0);
    if (lane == 0) { w_chunks++; w_sweep += nb_sweep; }
    bool done = false, tobs = false;
    if (live) {
      w_r1v += nb;
      st.r = o.r;
      if (rewrite) {
        done = true;   // the decision was taken in the call before
      } else if (step2) {
        st.lambda = st.bstw;
        done = true;
      } else {
        const double tolr = 4.0 * dv_log((double)nb) * MR3_EPS;
        st.resid = o.resid;
        if (st.k == 1 || o.resid < st.bstres) { st.bstres = o.resid; st.bstw = st.lambda; }
        bool more = false;
        if (!usedBS && o.resid > tolr * st.gap && fabs(o.rqcorr) > rqtol * fabs(st.lambda)) {
          const int sgndef = (Windex[s] <= negc) ? -1 : 1;
          if (o.rqcorr * sgndef >= 0.0 && st.lambda + o.rqcorr <= st.right &&
              st.lambda + o.rqcorr >= st.left) {
            st.flags |= SF_USEDRQ;
            if (sgndef == 1) st.left = st.lambda; else st.right = st.lambda;
            st.wsh = 0.5 * (st.left + st.right);
            st.lambda += o.rqcorr;
          } else {
            st.flags |= SF_NEEDBS;
          }
          if (st.right - st.left < rqtol * fabs(st.lambda)) st.flags |= SF_USEDBS;
          else if (st.k == MR3_MAXITER - 1) st.flags |= SF_NEEDBS;
          st.k++;
          more = (st.k <= MR3_MAXITER);
        }
        if (!more) {
          if ((st.flags & SF_USEDRQ) && (st.flags & SF_USEDBS) && st.bstres <= st.resid)
            st.flags |= SF_STEP2;
          else if (write)
            done = true;
          else
            st.flags |= SF_REWRITE;   // accepted, vector not written yet
        } else if (st.flags & SF_NEEDBS) {
          tobs = true;
        }
      }
    }
    if (!ITER) {
      // unfinished singletons: state saved, flagged for the next round's
      // list (or the bisection list); the compaction keeps the list order
      if (live && !done) sst[idx] = st;
      if (live) flag[base + lane] = done ? 0 : (tobs ? 2 : 1);
    } else {
      // the bisections the rounds would send to k_sng_bisect, one lane's
      // singleton at a time by the whole warp (same bits as k_sng_bisect)
      for (unsigned bm = __ballot_sync(full, tobs); bm; bm &= bm - 1) {
        const int v = __ffs(bm) - 1;
        const int nbv = __shfl_sync(full, nb, v), psv = __shfl_sync(full, ps, v);
        const int wiv = __shfl_sync(full, Windex[s], v);
        const double pvm = __shfl_sync(full, pivmin, v), spd = __shfl_sync(full, bspd, v);
        const double2 *Pv = (const double2 *)__shfl_sync(full, (unsigned long long)P, v);
        const int rv = __shfl_sync(full, st.r, v);
        double wsh = __shfl_sync(full, st.wsh, v), werr = __shfl_sync(full, st.werr, v);
        const int maxitr = dv_itmax(spd + pvm, pvm);
        const int tw = (rv < 1 || rv > nbv) ? nbv : rv;
        int nc = 0;
        dv_dlarrb_tree(32, nbv, Pv, psv, wiv, 1, 0, 0.0, 0.0, 0.0, 2.0 * MR3_EPS, pvm, maxitr, tw,
                       &wsh, &werr, &nc);
        wsh = __shfl_sync(full, wsh, 0);
        werr = __shfl_sync(full, werr, 0);
        if (lane == 0) w_neg += (unsigned long long)nc * nbv;
        if (lane == v) {
          st.wsh = wsh;
          st.werr = werr;
          st.flags = (st.flags | SF_USEDBS) & ~SF_NEEDBS;
          st.lambda = st.wsh;
          st.r = 0;
        }
      }
      if (live && !done) sst[idx] = st;
    }
    // finished eigenvectors out
    const unsigned fin = __ballot_sync(full, done);
    live = live && !done;
    if (fin) {
      const ClusterDev &Cf = cl[sng[idx].cl];
      const BlockDev &B = blocks[Cf.blk];
      ProbDev *p = &probs[B.prob];
      const int bl0 = B.ibgn - p->off;   // block's first row inside the problem
      int zind = 0;
      if (done) {
        Wsh[s] = st.lambda;
        Werr[s] = st.werr;
        Wgap[s] = st.gap;
        W[s] = st.lambda + Cf.sigma;
        zind = Zindex[s];
        p->Zsupp[2 * (size_t)zind] = o.isupp1 + bl0;
        p->Zsupp[2 * (size_t)zind + 1] = o.isupp2 + bl0;
      }
      // the accepted vectors, one column at a time by the whole warp: the
      // support scaled by nrminv, the rows outside the support (and outside
      // the block) zero
      const int ldz = p->ldz, np = p->n;
      const int z1 = bl0 + o.isupp1 - 1, z2 = bl0 + o.isupp2;   // support rows [z1, z2)
      __syncwarp();
      for (unsigned m = fin; m; m &= m - 1) {
        const int v = __ffs(m) - 1;
        const int npv = __shfl_sync(full, np, v), zc = __shfl_sync(full, zind, v);
        const int a = __shfl_sync(full, z1, v), b = __shfl_sync(full, z2, v);
        const int ldv = __shfl_sync(full, ldz, v);
        const double nv = __shfl_sync(full, o.nrminv, v);
        double *Zc = (double *)__shfl_sync(full, (unsigned long long)p->Z, v) + (size_t)zc * ldv;
        for (int row = lane; row < a; row += 32) Zc[row] = 0.0;
        for (int row = a + lane; row < b; row += 32) Zc[row] = Zc[row] * nv;
        for (int row = b + lane; row < npv; row += 32) Zc[row] = 0.0;
      }
      __syncwarp();
      if (done) {   // this lane's column is complete (its zero rows included)
        __threadfence();
        column_done(p, B.prob, zind, sc, done_list, tile_left);
      }
    }
    } while (ITER && __any_sync(full, live));
  }
  stat_add(stats, KID_SNG * 4 + 2, w_r1v);
  if (ITER) stat_add(stats, KID_SNG * 4 + 1, w_neg);
  // diagnostics: warp-level row sweeps and warp chunks
  stat_add(stats, KID_OTHER * 4 + 0, w_sweep);
  stat_add(stats, KID_OTHER * 4 + 1, w_chunks);
  if (ITER) {
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      if (atomicAdd(&sc->fin_ctas, 1) == (int)gridDim.x - 1) {
        sc->nin = 0;
        sc->mode = 2;
      }
    }
  }
}

// The bisection of a singleton whose Rayleigh-quotient step left its
// interval (SRC/process_singleton.c:178-192: dlarrb to 2*eps with the twist
// index of the last dlar1v), by a group of L lanes with the tree bisection
// of dv_dlarrb_tree.  L is the largest of 32, 16, 8, 4 with which the list
// still fits the resident lanes, so few singletons get short latency and
// many get little redundant work.  The singleton joins the next round's list
// (at its end).
__global__ void __launch_bounds__(256)
k_sng_bisect(int out, const SngDev *sng, const ClusterDev *cl, const ProbDev *probs,
             const BlockDev *blocks, const double2 *RP, const double2 *RQ, const double *arena,
             const int *Windex, SngState *sst, const int *bsl, int *act0, int *act1,
             SngCounters *sc, unsigned long long *stats) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  int *Aout = out ? act1 : act0;
  const int nbs = sc->bs_n;
  if (nbs == 0) return;
  const long long lanes = (long long)gridDim.x * blockDim.x;
  int L = 32;
  while (L > 4 && (long long)nbs * L > lanes) L >>= 1;
  const int G = 32 / L, gi = lane / L, t = lane & (L - 1);
  unsigned long long w_neg = 0;
  for (;;) {
    int t0 = 0;
    if (lane == 0) t0 = atomicAdd(&sc->bs_next, G);
    t0 = __shfl_sync(full, t0, 0);
    if (t0 >= nbs) break;
    const bool valid = t0 + gi < nbs;
    const int idx = bsl[valid ? t0 + gi : t0];   // spare groups mirror a valid one
    const SngDev S = sng[idx];
    const ClusterDev C = cl[S.cl];
    const BlockDev &B = blocks[C.blk];
    const ProbDev *p = &probs[B.prob];
    const int nb = B.nbl;
    const double pivmin = p->pivmin;
    const double2 *P, *Q;
    int ps;
    own_rrr(C, B, RP, RQ, arena, &P, &Q, &ps);
    SngState st = sst[idx];
    const int maxitr = dv_itmax(C.bl_spdiam + pivmin, pivmin);
    const int tw = (st.r < 1 || st.r > nb) ? nb : st.r;
    int nc = 0;
    dv_dlarrb_tree(L, nb, P, ps, Windex[S.slot], 1, 0, 0.0, 0.0, 0.0, 2.0 * MR3_EPS, pivmin, maxitr,
                   tw, &st.wsh, &st.werr, &nc);
    st.flags = (st.flags | SF_USEDBS) & ~SF_NEEDBS;
    st.lambda = st.wsh;
    st.r = 0;
    if (valid && t == 0) {
      w_neg += (unsigned long long)nc * nb;
      sst[idx] = st;
      Aout[atomicAdd(&sc->act_n[out], 1)] = idx;
    }
    __syncwarp();
  }
  stat_add(stats, KID_SNG * 4 + 1, w_neg);
}

// The rest of a level's singletons when few are left (SngCounters.mode 1):
// a warp per singleton (the warps take them in turn) runs its remaining
// Rayleigh-quotient loop (SRC/process_singleton.c:159-292) to the end in one
// launch -- each dlar1v on lanes 0 and 1 (SPLIT, the default) or on lane 0
// with its checkpoints, a bisection by all 32 lanes with the tree
// bisection -- instead of one call per round with a launch
// sequence (round, compaction, bisection, sort) between calls.  Every call
// and every state update is the one the rounds make, so the results are the
// same bits.  The last block to finish empties the list (mode 2).
// SPLIT: each dlar1v is dv_r1s_call (the two sweeps on two lanes at once,
// the twist chosen by the warp, the vector in the warp's row scratch
// fscratch, 5 (nmax + 2) doubles per warp) instead of lane 0's checkpointed
// dlar1v; the results are the same bits.
template <bool SPLIT>
__global__ void __launch_bounds__(SNG_WARPS * 32, 2)
k_sng_finish(int in, const SngDev *sng, const ClusterDev *cl, ProbDev *probs,
             const BlockDev *blocks, const double2 *RP, const double2 *RQ, const double *arena,
             double *W, double *Wsh, double *Werr, double *Wgap, const int *Windex,
             const int *Zindex, SngState *sst, const int *act0, const int *act1, SngCounters *sc,
             double *scratch, double *fscratch, long long nmax, int2 *done_list, int *tile_left,
             unsigned long long *stats) {
  if (sc->mode != 1) return;
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const long long gw = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nck = nmax / CK_K + 1;
  r1c_ck ck;
  ck.S = scratch + gw * 3 * nck * 32 + lane;
  ck.I = ck.S + nck * 32;
  ck.P = ck.I + nck * 32;
  r1s_buf rb;
  {
    const long long len = nmax + 2;
    rb.SI = (SPLIT ? fscratch : scratch) + gw * 5 * len;
    rb.LP = rb.SI + len;
    rb.PA = rb.LP + len;
    rb.UM = rb.PA + len;
    rb.ZV = rb.UM + len;
  }
  const int *Ain = in ? act1 : act0;
  const int nin = sc->nin;
  const double rqtol = 2.0 * MR3_EPS;
  unsigned long long w_r1v = 0, w_neg = 0;
  for (;;) {
    int j = 0;
    if (lane == 0) j = atomicAdd(&sc->act_next[in], 1);
    j = __shfl_sync(full, j, 0);
    if (j >= nin) break;
    const int idx = Ain[j];
    const SngDev S = sng[idx];
    const int s = S.slot;
    const ClusterDev C = cl[S.cl];
    const BlockDev &B = blocks[C.blk];
    ProbDev *p = &probs[B.prob];
    const int nb = B.nbl;
    const double pivmin = p->pivmin;
    const double2 *P, *Q;
    int ps;
    own_rrr(C, B, RP, RQ, arena, &P, &Q, &ps);
    double *zcol = p->Z + (size_t)Zindex[s] * p->ldz + (B.ibgn - p->off);
    const int wi = Windex[s];
    SngState st = sst[idx];   // identical in every lane
    dlar1v_out o;
    for (;;) {
      // the bisection a round would have sent this singleton to (a second
      // step or a rewrite follows the loop's end: no bisection then)
      if ((st.flags & SF_NEEDBS) && !(st.flags & (SF_STEP2 | SF_REWRITE))) {
        const int maxitr = dv_itmax(C.bl_spdiam + pivmin, pivmin);
        const int tw = (st.r < 1 || st.r > nb) ? nb : st.r;
        int nc = 0;
        dv_dlarrb_tree(32, nb, P, ps, wi, 1, 0, 0.0, 0.0, 0.0, 2.0 * MR3_EPS, pivmin, maxitr, tw,
                       &st.wsh, &st.werr, &nc);
        st.flags = (st.flags | SF_USEDBS) & ~SF_NEEDBS;
        st.lambda = st.wsh;
        st.r = 0;
        if (lane == 0) w_neg += (unsigned long long)nc * nb;
      }
      const bool usedBS = (st.flags & SF_USEDBS) != 0;
      const double lam_call = (st.flags & SF_STEP2) ? st.bstw : st.lambda;
      const int r_in = (st.flags & SF_REWRITE) ? 0 : st.r;
      const bool write = (st.flags & (SF_REWRITE | SF_STEP2 | SF_USEDBS)) || st.k > 1;
      int negc = 0;
      o.isupp1 = 1; o.isupp2 = nb; o.nrminv = 0.0; o.r = 0; o.resid = 0.0; o.rqcorr = 0.0;
      if (SPLIT) {
        dv_r1s_call(nb, lam_call, P, Q, ps, pivmin, !usedBS, r_in, st.gaptol, rb, &negc, &o);
      } else {
        r1c_state rs;
        rs.r = 0; rs.mingma = 0.0; rs.sawnan = false; rs.slowA = false; rs.slowB = false;
        dv_r1c_factor(lane == 0, nb, lam_call, P, Q, ps, pivmin, !usedBS, r_in, ck, &negc, &rs);
        if (lane == 0)
          dv_r1c_solve(nb, lam_call, P, Q, ps, pivmin, st.gaptol, rs.r, rs.sawnan, rs.slowA,
                       rs.slowB, ck.S, ck.P, rs.mingma, write ? zcol : nullptr, 1.0, &o);
      }
      o.r = __shfl_sync(full, o.r, 0);
      o.isupp1 = __shfl_sync(full, o.isupp1, 0);
      o.isupp2 = __shfl_sync(full, o.isupp2, 0);
      o.nrminv = __shfl_sync(full, o.nrminv, 0);
      o.resid = __shfl_sync(full, o.resid, 0);
      o.rqcorr = __shfl_sync(full, o.rqcorr, 0);
      negc = __shfl_sync(full, negc, 0);
      if (lane == 0) w_r1v += nb;
      // the state update of k_sng_round, in every lane
      bool done = false;
      const bool step2 = (st.flags & SF_STEP2) != 0;
      st.r = o.r;
      if (st.flags & SF_REWRITE) {
        done = true;
      } else if (step2) {
        st.lambda = st.bstw;
        done = true;
      } else {
        const double tolr = 4.0 * dv_log((double)nb) * MR3_EPS;
        st.resid = o.resid;
        if (st.k == 1 || o.resid < st.bstres) { st.bstres = o.resid; st.bstw = st.lambda; }
        bool more = false;
        if (!usedBS && o.resid > tolr * st.gap && fabs(o.rqcorr) > rqtol * fabs(st.lambda)) {
          const int sgndef = (wi <= negc) ? -1 : 1;
          if (o.rqcorr * sgndef >= 0.0 && st.lambda + o.rqcorr <= st.right &&
              st.lambda + o.rqcorr >= st.left) {
            st.flags |= SF_USEDRQ;
            if (sgndef == 1) st.left = st.lambda; else st.right = st.lambda;
            st.wsh = 0.5 * (st.left + st.right);
            st.lambda += o.rqcorr;
          } else {
            st.flags |= SF_NEEDBS;
          }
          if (st.right - st.left < rqtol * fabs(st.lambda)) st.flags |= SF_USEDBS;
          else if (st.k == MR3_MAXITER - 1) st.flags |= SF_NEEDBS;
          st.k++;
          more = (st.k <= MR3_MAXITER);
        }
        if (!more) {
          if ((st.flags & SF_USEDRQ) && (st.flags & SF_USEDBS) && st.bstres <= st.resid)
            st.flags |= SF_STEP2;
          else if (write)
            done = true;
          else
            st.flags |= SF_REWRITE;
        }
      }
      if (done) break;
    }
    // outputs and the finished column (support scaled, the rest zero)
    const int bl0 = B.ibgn - p->off;
    const int zind = Zindex[s];
    if (lane == 0) {
      Wsh[s] = st.lambda;
      Werr[s] = st.werr;
      Wgap[s] = st.gap;
      W[s] = st.lambda + C.sigma;
      p->Zsupp[2 * (size_t)zind] = o.isupp1 + bl0;
      p->Zsupp[2 * (size_t)zind + 1] = o.isupp2 + bl0;
    }
    const int a = bl0 + o.isupp1 - 1, b = bl0 + o.isupp2;
    double *Zc = p->Z + (size_t)zind * p->ldz;
    __syncwarp();
    for (int row = lane; row < a; row += 32) Zc[row] = 0.0;
    if (SPLIT)   // the vector is in the warp's scratch (rows of the block, 1-based)
      for (int row = a + lane; row < b; row += 32) Zc[row] = rb.ZV[row - bl0 + 1] * o.nrminv;
    else
      for (int row = a + lane; row < b; row += 32) Zc[row] = Zc[row] * o.nrminv;
    for (int row = b + lane; row < p->n; row += 32) Zc[row] = 0.0;
    __syncwarp();
    if (lane == 0) {
      __threadfence();
      column_done(p, B.prob, zind, sc, done_list, tile_left);
    }
  }
  stat_add(stats, KID_SNG * 4 + 2, w_r1v);
  stat_add(stats, KID_SNG * 4 + 1, w_neg);
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&sc->fin_ctas, 1) == (int)gridDim.x - 1) {
      sc->nin = 0;
      sc->mode = 2;
    }
  }
}

// Unit vectors of 1x1 blocks (SRC/process_singleton.c:125-133).
__global__ void k_unitvec(const int *list, SngCounters *sc, ProbDev *probs,
                          const BlockDev *blocks, const int *iblk, const int *Zindex,
                          int2 *done_list, int *tile_left) {
  int t = blockIdx.x;
  if (t >= sc->n_unit) return;
  int s = list[t];
  const BlockDev &B = blocks[iblk[s]];
  ProbDev *p = &probs[B.prob];
  int zind = Zindex[s];
  double *Zc = p->Z + (size_t)zind * (size_t)p->ldz;
  int row0 = B.ibgn - p->off;
  for (int row = threadIdx.x; row < p->n; row += blockDim.x) Zc[row] = (row == row0) ? 1.0 : 0.0;
  __syncthreads();
  if (threadIdx.x == 0) {
    p->Zsupp[2 * (size_t)zind] = row0 + 1;
    p->Zsupp[2 * (size_t)zind + 1] = row0 + 1;
    __threadfence();
    column_done(p, B.prob, zind, sc, done_list, tile_left);
  }
}

// ------------------------------------------------------------------------
// Output ordering (sort_eigenpairs, SRC/mrrr.c:525-588) and copy-out.
// ------------------------------------------------------------------------
__global__ void k_place_w(int N, const ProbDev *probs, const int *prob_of_slot, const double *W,
                          const int *Zindex, double *Wout) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= N) return;
  int pi = prob_of_slot[s];
  if (pi < 0) return;
  const ProbDev *p = &probs[pi];
  int k = s - p->off;
  if (k >= p->m || p->status) return;
  if (p->jobz == MR3_JOB_V) Wout[p->off + Zindex[s]] = W[s];
  else Wout[s] = W[s];
}

__global__ void k_check_sorted(int N, ProbDev *probs, const int *prob_of_slot, const double *Wout,
                               int *unsorted) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= N) return;
  int pi = prob_of_slot[s];
  if (pi < 0) return;
  const ProbDev *p = &probs[pi];
  int k = s - p->off;
  if (k + 1 >= p->m || p->status || p->jobz == MR3_JOB_C) return;
  if (Wout[s] > Wout[s + 1]) atomicOr(&unsorted[pi], 1);
}

__global__ void k_scatter(const ProbDev *probs, double *const *Wp, double *const *Dp,
                          double *const *Ep, const double *Wout, const double *D, const double *E) {
  const ProbDev *p = &probs[blockIdx.x];
  if (p->trivial) return;
  for (int i = threadIdx.x; i < p->n; i += blockDim.x) {
    if (i < p->m && p->jobz != MR3_JOB_C && !p->status) Wp[blockIdx.x][i] = Wout[p->off + i];
    Dp[blockIdx.x][i] = D[p->off + i];
    Ep[blockIdx.x][i] = E[p->off + i];
  }
}

__global__ void k_sorted_to_w(int N, const ProbDev *probs, const int *prob_of_slot,
                              const SortRec *rec, double *Wout, int want_job, const int *flag) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= N) return;
  int pi = prob_of_slot[s];
  if (pi < 0) return;
  const ProbDev *p = &probs[pi];
  if (p->trivial || p->status || p->jobz != want_job) return;
  if (flag && !flag[pi]) return;
  if (s - p->off < p->m) Wout[s] = rec[s].key;
}

// Apply the permutation of the bubble fix-up to Zsupp (new column k takes
// old column rec[k].idx); W was already rewritten from the sorted keys.
__global__ void k_perm_zsupp(int N, const ProbDev *probs, const int *prob_of_slot,
                             const SortRec *rec, const int *flag, int *tmp2) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= N) return;
  int pi = prob_of_slot[s];
  if (pi < 0 || !flag[pi]) return;
  const ProbDev *p = &probs[pi];
  int k = s - p->off;
  if (k >= p->m) return;
  int src = rec[s].idx;
  tmp2[2 * (size_t)s] = p->Zsupp[2 * (size_t)src];
  tmp2[2 * (size_t)s + 1] = p->Zsupp[2 * (size_t)src + 1];
}
__global__ void k_perm_zsupp2(int N, const ProbDev *probs, const int *prob_of_slot, const int *flag,
                              const int *tmp2) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= N) return;
  int pi = prob_of_slot[s];
  if (pi < 0 || !flag[pi]) return;
  const ProbDev *p = &probs[pi];
  int k = s - p->off;
  if (k >= p->m) return;
  p->Zsupp[2 * (size_t)k] = tmp2[2 * (size_t)s];
  p->Zsupp[2 * (size_t)k + 1] = tmp2[2 * (size_t)s + 1];
}

// ========================================================================
// Host side
// ========================================================================
struct mr3_cuda_ctx {
  int device = 0, nsm = 148;
  int sng_ctas_per_sm = 2;                  // resident k_sng_round CTAs per SM
  cudaStream_t own = nullptr;
  cudaStream_t aux = nullptr;               // copies that overlap the solves
  cudaStream_t rnd = nullptr;               // a level's singleton rounds
  cudaEvent_t rnd_done = nullptr;           // and their end
  cudaEvent_t xev[MR3_CUDA_EVENTS] = {nullptr};
  void *hws = nullptr;                      // page-locked staging buffer
  size_t hws_cap = 0;
  char err[256] = {0};
  long long launches = 0;
  size_t capN = 0, capP = 0, capScratch = 0, capArena[2] = {0, 0};
  ProbDev *probs = nullptr;
  BlockDev *blocks = nullptr;
  int *blk_of_row = nullptr, *Windex = nullptr, *iblk = nullptr, *It = nullptr, *Zindex = nullptr;
  int *prob_of_slot = nullptr, *cl_of_slot = nullptr, *lvl_of_slot = nullptr, *unit_list = nullptr;
  int *flag = nullptr, *tmp2 = nullptr;
  int *cls_ns = nullptr, *cls_soff = nullptr, *cls_cbase = nullptr;
  long long *cls_abase = nullptr;
  double *D = nullptr, *E = nullptr, *E2 = nullptr, *Wt = nullptr, *Et = nullptr, *W = nullptr;
  double *Werr = nullptr, *Wgap = nullptr, *Wcopy = nullptr, *Wsh = nullptr, *Dt = nullptr;
  double *Lt = nullptr, *Wout = nullptr;
  double2 *gers = nullptr, *TP = nullptr, *TPc = nullptr, *RP = nullptr, *RQ = nullptr;
  SortRec *rec0 = nullptr, *rec1 = nullptr;
  ClusterDev *cl[2] = {nullptr, nullptr};
  SngDev *sng = nullptr;
  SngState *sst = nullptr;
  int *act[2] = {nullptr, nullptr}, *bsl = nullptr, *sbcnt = nullptr, *rlcnt = nullptr;
  int *rl = nullptr, *rl_n = nullptr;       // a level's cluster eigenvalues to refine
  int *sbk = nullptr;                       // singleton size buckets (3 x 16)
  BisNode *bis_nodes[2] = {nullptr, nullptr}; // shared-interval bisection: levels
  int *bis_cnt = nullptr, *bis_bcnt = nullptr, *bis_n = nullptr;
  BisState *bis_st = nullptr;
  int2 *done_list = nullptr;                // finished column tiles (problem, tile)
  int *tile_left = nullptr;                 // unwritten columns of each tile
  size_t capTiles = 0;
  int2 *h_done = nullptr, *d_hdone = nullptr;   // pinned copy of done_list (host, device view)
  int *h_snap = nullptr, *d_hsnap = nullptr;    // done_n after each singleton round
  cudaEvent_t rev[SNG_ROUNDS] = {};             // and the rounds' completion
  std::vector<int2> h_runs;
  std::vector<int> h_dprob, h_dcol, h_dcnt;
  unsigned char *sflag = nullptr;
  LevelCounters *lc = nullptr;
  SngCounters *sc = nullptr;
  double *scratch = nullptr, *arena[2] = {nullptr, nullptr};
  double *qd = nullptr;                     // dqds arrays (4 doubles per row)
  double *fscratch = nullptr;               // row scratch of the split finish
  size_t capFscratch = 0;
  size_t round_scratch = (size_t)8 << 30;   // bound of the round warps' checkpoint scratch
  const double **Din = nullptr, **Ein = nullptr;
  double **Wp = nullptr, **Dp = nullptr, **Ep = nullptr;
  // pinned host mirrors
  ProbDev *h_probs = nullptr;
  void **h_ptrs = nullptr;
  LevelCounters *h_lc = nullptr, *d_hlc = nullptr;   // host pointer, device view
  SngCounters *h_sc = nullptr, *d_hsc = nullptr;
  int *h_flag = nullptr;
  double *h_const = nullptr;   // {1.0}
  int *h_iconst = nullptr;     // {1, 1}
  int *h_bisn = nullptr;       // a level's node count of the shared-interval bisection
  void *ws[MR3_CUDA_WS_SLOTS] = {nullptr};
  size_t ws_cap[MR3_CUDA_WS_SLOTS] = {0};
  // profiling: per-kernel CUDA-event timing and device work counters
  int prof = 0;
  unsigned long long *stats = nullptr;
  std::vector<cudaEvent_t> evpool;
  size_t evnext = 0;
  struct Pending { const char *name; cudaEvent_t a, b; };
  std::vector<Pending> pending;
  std::vector<std::string> knames;
  std::vector<double> kms;
  std::vector<long long> kcount;
};

static cudaEvent_t prof_event(mr3_cuda_ctx *c) {
  if (c->evnext == c->evpool.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    c->evpool.push_back(e);
  }
  return c->evpool[c->evnext++];
}

static void prof_flush(mr3_cuda_ctx *c) {
  for (auto &q : c->pending) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, q.a, q.b);
    size_t k = 0;
    while (k < c->knames.size() && c->knames[k] != q.name) k++;
    if (k == c->knames.size()) {
      c->knames.emplace_back(q.name);
      c->kms.push_back(0.0);
      c->kcount.push_back(0);
    }
    c->kms[k] += ms;
    c->kcount[k] += 1;
  }
  c->pending.clear();
  c->evnext = 0;
}

#define CK(call, what)                                                    \
  do {                                                                    \
    cudaError_t e_ = (call);                                              \
    if (e_ != cudaSuccess) {                                              \
      snprintf(c->err, sizeof(c->err), "%s: %s", what, cudaGetErrorString(e_)); \
      return MR3_EMISC;                                                   \
    }                                                                     \
  } while (0)

#define LAUNCH(kern, grid, block, ...) LAUNCH_SMEM(kern, grid, block, 0, __VA_ARGS__)
#define LAUNCH_SMEM(kern, grid, block, smem, ...)                         \
  do {                                                                    \
    if ((grid) > 0) {                                                     \
      cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;                         \
      if (c->prof) {                                                      \
        ev0_ = prof_event(c);                                             \
        ev1_ = prof_event(c);                                             \
        cudaEventRecord(ev0_, st);                                        \
      }                                                                   \
      kern<<<(grid), (block), (smem), st>>>(__VA_ARGS__);                 \
      c->launches++;                                                      \
      CK(cudaGetLastError(), #kern);                                      \
      if (c->prof) {                                                      \
        cudaEventRecord(ev1_, st);                                        \
        c->pending.push_back({#kern, ev0_, ev1_});                        \
      }                                                                   \
    }                                                                     \
  } while (0)

template <typename T>
static cudaError_t regrow(T **p, size_t count) {
  if (*p) cudaFree(*p);
  *p = nullptr;
  return cudaMalloc((void **)p, std::max<size_t>(count, 1) * sizeof(T));
}

static int ensure_rows(mr3_cuda_ctx *c, size_t N, size_t P) {
  if (N > c->capN) {
    size_t n = std::max(N, c->capN + c->capN / 2);
    CK(regrow(&c->blocks, n), "blocks");
    CK(regrow(&c->blk_of_row, n), "blk_of_row");
    CK(regrow(&c->Windex, n), "Windex");
    CK(regrow(&c->iblk, n), "iblk");
    CK(regrow(&c->It, n), "It");
    CK(regrow(&c->Zindex, n), "Zindex");
    CK(regrow(&c->prob_of_slot, n), "prob_of_slot");
    CK(regrow(&c->cl_of_slot, n), "cl_of_slot");
    CK(regrow(&c->lvl_of_slot, n), "lvl_of_slot");
    CK(regrow(&c->unit_list, n), "unit_list");
    CK(regrow(&c->tmp2, 2 * n), "tmp2");
    CK(regrow(&c->cls_ns, n), "cls_ns");
    CK(regrow(&c->cls_soff, n), "cls_soff");
    CK(regrow(&c->cls_cbase, n), "cls_cbase");
    CK(regrow(&c->cls_abase, n), "cls_abase");
    double **dd[] = {&c->D, &c->E, &c->E2, &c->Wt, &c->Et, &c->W, &c->Werr, &c->Wgap,
                     &c->Wcopy, &c->Wsh, &c->Dt, &c->Lt, &c->Wout};
    for (double **q : dd) CK(regrow(q, n), "rows");
    double2 **d2[] = {&c->gers, &c->TP, &c->TPc, &c->RP, &c->RQ};
    for (double2 **q : d2) CK(regrow(q, n), "rows2");
    CK(regrow(&c->rec0, n), "rec0");
    CK(regrow(&c->rec1, n), "rec1");
    CK(regrow(&c->cl[0], n), "cl0");
    CK(regrow(&c->cl[1], n), "cl1");
    CK(regrow(&c->sng, n), "sng");
    CK(regrow(&c->sst, n), "sst");
    CK(regrow(&c->act[0], n), "act0");
    CK(regrow(&c->act[1], n), "act1");
    CK(regrow(&c->bsl, n), "bsl");
    CK(regrow(&c->rl, n), "rl");
    CK(regrow(&c->sflag, n), "sflag");
    CK(regrow(&c->sbcnt, 2 * (n / LIST_T + 1)), "sbcnt");
    CK(regrow(&c->rlcnt, n / RL_T + 1), "rlcnt");
    CK(regrow(&c->bis_nodes[0], n / 2 + 1), "bis nodes");
    CK(regrow(&c->bis_nodes[1], n / 2 + 1), "bis nodes");
    CK(regrow(&c->bis_cnt, n / 2 + 1), "bis cnt");
    CK(regrow(&c->bis_bcnt, (n / 2 + 1) / 256 + 1), "bis bcnt");
    CK(regrow(&c->bis_st, n), "bis st");
    CK(regrow(&c->qd, 4 * n), "qd");
    c->capN = n;
  }
  if (P > c->capP) {
    size_t p = std::max(P, c->capP + c->capP / 2);
    CK(regrow(&c->probs, p), "probs");
    CK(regrow(&c->flag, p), "flag");

    CK(regrow(&c->Din, p), "Din");
    CK(regrow(&c->Ein, p), "Ein");
    CK(regrow(&c->Wp, p), "Wp");
    CK(regrow(&c->Dp, p), "Dp");
    CK(regrow(&c->Ep, p), "Ep");
    if (c->h_probs) cudaFreeHost(c->h_probs);
    if (c->h_ptrs) cudaFreeHost(c->h_ptrs);
    if (c->h_flag) cudaFreeHost(c->h_flag);
    CK(cudaMallocHost((void **)&c->h_probs, p * sizeof(ProbDev)), "h_probs");
    CK(cudaMallocHost((void **)&c->h_ptrs, 5 * p * sizeof(void *)), "h_ptrs");
    CK(cudaMallocHost((void **)&c->h_flag, p * sizeof(int)), "h_flag");
    c->capP = p;
  }
  return MR3_OK;
}

extern "C" int mr3_cuda_ctx_create(int device, mr3_cuda_ctx **out) {
  return mr3_cuda_ctx_create_prio(device, 0, out);
}

extern "C" int mr3_cuda_ctx_create_prio(int device, int high, mr3_cuda_ctx **out) {
  if (!out) return MR3_EARG;
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return MR3_EMISC;
  int prio_lo = 0, prio_hi = 0;
  if (high && cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi) != cudaSuccess) prio_hi = 0;
  const int prio = high ? prio_hi : 0;
  mr3_cuda_ctx *c = new mr3_cuda_ctx();
  c->device = device;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) c->nsm = prop.multiProcessorCount;
  bool evok = true;
  for (int i = 0; i < MR3_CUDA_EVENTS; i++)
    evok = evok && cudaEventCreateWithFlags(&c->xev[i], cudaEventDisableTiming) == cudaSuccess;
  for (int i = 0; i < SNG_ROUNDS; i++)
    evok = evok && cudaEventCreateWithFlags(&c->rev[i], cudaEventDisableTiming) == cudaSuccess;
  if (!evok || cudaStreamCreateWithPriority(&c->own, cudaStreamNonBlocking, prio) != cudaSuccess ||
      cudaStreamCreateWithPriority(&c->aux, cudaStreamNonBlocking, prio) != cudaSuccess ||
      cudaStreamCreateWithPriority(&c->rnd, cudaStreamNonBlocking, prio) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->rnd_done, cudaEventDisableTiming) != cudaSuccess ||
      cudaMalloc((void **)&c->lc, 2 * sizeof(LevelCounters)) != cudaSuccess ||
      cudaMalloc((void **)&c->sc, sizeof(SngCounters)) != cudaSuccess ||
      cudaMalloc((void **)&c->rl_n, sizeof(int)) != cudaSuccess ||
      cudaMalloc((void **)&c->bis_n, 2 * sizeof(int)) != cudaSuccess ||
      cudaMalloc((void **)&c->sbk, 3 * SNG_BUCKETS * sizeof(int)) != cudaSuccess ||
      cudaMallocHost((void **)&c->h_lc, 2 * sizeof(LevelCounters)) != cudaSuccess ||
      cudaMallocHost((void **)&c->h_sc, sizeof(SngCounters)) != cudaSuccess ||
      cudaMallocHost((void **)&c->h_snap, SNG_ROUNDS * sizeof(int)) != cudaSuccess ||
      cudaMallocHost((void **)&c->h_const, sizeof(double)) != cudaSuccess ||
      cudaMallocHost((void **)&c->h_iconst, 2 * sizeof(int)) != cudaSuccess ||
      cudaMallocHost((void **)&c->h_bisn, sizeof(int)) != cudaSuccess ||
      cudaMalloc((void **)&c->stats, KID_COUNT * 4 * sizeof(unsigned long long)) != cudaSuccess ||
      cudaHostGetDevicePointer((void **)&c->d_hlc, c->h_lc, 0) != cudaSuccess ||
      cudaHostGetDevicePointer((void **)&c->d_hsc, c->h_sc, 0) != cudaSuccess ||
      cudaHostGetDevicePointer((void **)&c->d_hsnap, c->h_snap, 0) != cudaSuccess) {
    mr3_cuda_ctx_destroy(c);
    return MR3_EMISC;
  }
  int nb = 0;
  if (cudaFuncSetAttribute(k_sng_round<SNG_LATER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           SNG_TILE_BYTES) != cudaSuccess ||
      cudaFuncSetAttribute(k_sng_round<SNG_ITER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           SNG_TILE_BYTES) != cudaSuccess ||
      cudaFuncSetAttribute(k_sng_round<SNG_FIRST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           SNG_TILE_BYTES) != cudaSuccess) {
    mr3_cuda_ctx_destroy(c);
    return MR3_EMISC;
  }
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_sng_round<SNG_LATER>, SNG_WARPS * 32,
                                                    SNG_TILE_BYTES) == cudaSuccess &&
      nb > 0)
    c->sng_ctas_per_sm = nb;
  c->h_const[0] = 1.0;
  c->h_iconst[0] = 1;
  c->h_iconst[1] = 1;
  *out = c;
  return MR3_OK;
}

extern "C" void mr3_cuda_ctx_destroy(mr3_cuda_ctx *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  void *dev[] = {c->probs, c->blocks, c->blk_of_row, c->Windex, c->iblk, c->It, c->Zindex,
                 c->prob_of_slot, c->cl_of_slot, c->lvl_of_slot, c->unit_list, c->flag, c->tmp2,
                 c->D, c->E, c->E2, c->Wt, c->Et, c->W, c->Werr, c->Wgap, c->Wcopy, c->Wsh,
                 c->Dt, c->Lt, c->Wout, c->gers, c->TP, c->TPc, c->RP, c->RQ, c->rec0, c->rec1,
                 c->cl[0], c->cl[1], c->sng, c->sst, c->act[0], c->act[1], c->bsl, c->sflag, c->sbcnt, c->rlcnt, c->rl, c->rl_n, c->sbk, c->done_list, c->tile_left,
                 c->bis_nodes[0], c->bis_nodes[1], c->bis_cnt, c->bis_bcnt, c->bis_n, c->bis_st, c->lc, c->sc, c->scratch, c->arena[0],
                 c->cls_ns, c->cls_soff, c->cls_cbase, c->cls_abase, c->qd, c->fscratch,
                 c->arena[1], (void *)c->Din, (void *)c->Ein, c->Wp, c->Dp, c->Ep};
  for (void *q : dev)
    if (q) cudaFree(q);
  for (int i = 0; i < MR3_CUDA_WS_SLOTS; i++)
    if (c->ws[i]) cudaFree(c->ws[i]);
  void *host[] = {c->h_probs, c->h_ptrs, c->h_lc, c->h_sc, c->h_flag, c->h_const, c->h_iconst, c->h_bisn,
                  c->h_done, c->h_snap};
  for (void *q : host)
    if (q) cudaFreeHost(q);
  if (c->stats) cudaFree(c->stats);
  for (cudaEvent_t e : c->evpool) cudaEventDestroy(e);
  for (int i = 0; i < MR3_CUDA_EVENTS; i++)
    if (c->xev[i]) cudaEventDestroy(c->xev[i]);
  for (int i = 0; i < SNG_ROUNDS; i++)
    if (c->rev[i]) cudaEventDestroy(c->rev[i]);
  if (c->hws) cudaFreeHost(c->hws);
  if (c->aux) cudaStreamDestroy(c->aux);
  if (c->rnd) cudaStreamDestroy(c->rnd);
  if (c->rnd_done) cudaEventDestroy(c->rnd_done);
  if (c->own) cudaStreamDestroy(c->own);
  delete c;
}

extern "C" int mr3_cuda_ctx_set_round_scratch(mr3_cuda_ctx *c, size_t bytes) {
  if (!c || bytes < ((size_t)64 << 20)) return MR3_EARG;
  c->round_scratch = bytes;
  return MR3_OK;
}

extern "C" void *mr3_cuda_ws(mr3_cuda_ctx *c, int slot, size_t bytes) {
  if (!c || slot < 0 || slot >= MR3_CUDA_WS_SLOTS) return nullptr;
  if (bytes > c->ws_cap[slot] || !c->ws[slot]) {
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->own);
    cudaStreamSynchronize(c->aux);
    if (c->ws[slot]) cudaFree(c->ws[slot]);
    c->ws[slot] = nullptr;
    c->ws_cap[slot] = 0;
    size_t sz = std::max<size_t>(bytes, 256);
    if (cudaMalloc(&c->ws[slot], sz) != cudaSuccess) {
      snprintf(c->err, sizeof(c->err), "workspace of %zu bytes", sz);
      return nullptr;
    }
    c->ws_cap[slot] = sz;
  }
  return c->ws[slot];
}

extern "C" int mr3_cuda_copy(mr3_cuda_ctx *c, void *dst, const void *src, size_t bytes, int dir) {
  if (!c) return MR3_EMISC;
  if (bytes == 0) return MR3_OK;
  CK(cudaMemcpyAsync(dst, src, bytes, dir == 0 ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost,
                     c->own), "copy");
  return MR3_OK;
}

extern "C" int mr3_cuda_copy2d(mr3_cuda_ctx *c, void *dst, size_t dpitch, const void *src,
                               size_t spitch, size_t width, size_t height, int dir) {
  if (!c) return MR3_EMISC;
  if (width == 0 || height == 0) return MR3_OK;
  CK(cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, height,
                       dir == 0 ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost, c->own),
     "copy2d");
  return MR3_OK;
}

extern "C" int mr3_cuda_sync(mr3_cuda_ctx *c) {
  if (!c) return MR3_EMISC;
  CK(cudaStreamSynchronize(c->own), "sync");
  return MR3_OK;
}

extern "C" int mr3_cuda_set_device(mr3_cuda_ctx *c) {
  if (!c) return MR3_EMISC;
  return cudaSetDevice(c->device) == cudaSuccess ? MR3_OK : MR3_EMISC;
}

static cudaStream_t ctx_stream(mr3_cuda_ctx *c, int which) {
  return which == MR3_STREAM_COPY ? c->aux : c->own;
}

extern "C" int mr3_cuda_copy_on(mr3_cuda_ctx *c, int stream, void *dst, const void *src,
                                size_t bytes, int dir) {
  if (!c || (stream != MR3_STREAM_MAIN && stream != MR3_STREAM_COPY)) return MR3_EMISC;
  if (bytes == 0) return MR3_OK;
  CK(cudaMemcpyAsync(dst, src, bytes, dir == 0 ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost,
                     ctx_stream(c, stream)), "copy_on");
  return MR3_OK;
}

extern "C" int mr3_cuda_copy2d_on(mr3_cuda_ctx *c, int stream, void *dst, size_t dpitch,
                                  const void *src, size_t spitch, size_t width, size_t height,
                                  int dir) {
  if (!c || (stream != MR3_STREAM_MAIN && stream != MR3_STREAM_COPY)) return MR3_EMISC;
  if (width == 0 || height == 0) return MR3_OK;
  CK(cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, height,
                       dir == 0 ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost,
                       ctx_stream(c, stream)),
     "copy2d_on");
  return MR3_OK;
}

extern "C" int mr3_cuda_event(mr3_cuda_ctx *c, int ev, int record_on, int wait_on) {
  if (!c || ev < 0 || ev >= MR3_CUDA_EVENTS || record_on > MR3_STREAM_COPY ||
      wait_on > MR3_STREAM_COPY)
    return MR3_EMISC;
  if (record_on >= 0) CK(cudaEventRecord(c->xev[ev], ctx_stream(c, record_on)), "event record");
  if (wait_on >= 0) CK(cudaStreamWaitEvent(ctx_stream(c, wait_on), c->xev[ev], 0), "event wait");
  return MR3_OK;
}

extern "C" int mr3_cuda_sync_all(mr3_cuda_ctx *c) {
  if (!c) return MR3_EMISC;
  CK(cudaStreamSynchronize(c->own), "sync main");
  CK(cudaStreamSynchronize(c->aux), "sync copy");
  return MR3_OK;
}

extern "C" void *mr3_cuda_host_ws(mr3_cuda_ctx *c, size_t bytes) {
  if (!c) return nullptr;
  if (bytes > c->hws_cap || !c->hws) {
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->own);
    cudaStreamSynchronize(c->aux);
    if (c->hws) cudaFreeHost(c->hws);
    c->hws = nullptr;
    c->hws_cap = 0;
    size_t sz = std::max<size_t>(bytes, 4096);
    if (cudaMallocHost(&c->hws, sz) != cudaSuccess) {
      c->hws = nullptr;
      snprintf(c->err, sizeof(c->err), "page-locked buffer of %zu bytes", sz);
      return nullptr;
    }
    c->hws_cap = sz;
  }
  return c->hws;
}

extern "C" void mr3_cuda_profile(mr3_cuda_ctx *c, int on) {
  if (!c) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->own);
  c->prof = on;
  c->pending.clear();
  c->evnext = 0;
  c->knames.clear();
  c->kms.clear();
  c->kcount.clear();
  cudaMemset(c->stats, 0, KID_COUNT * 4 * sizeof(unsigned long long));
  cudaDeviceSynchronize();
}

extern "C" int mr3_cuda_profile_read(mr3_cuda_ctx *c, int max, char *names, double *ms,
                                     long long *launches, unsigned long long *counters) {
  if (!c) return 0;
  int k = (int)std::min<size_t>((size_t)max, c->knames.size());
  for (int i = 0; i < k; i++) {
    strncpy(names + 32 * i, c->knames[i].c_str(), 31);
    names[32 * i + 31] = 0;
    ms[i] = c->kms[i];
    launches[i] = c->kcount[i];
  }
  if (counters)
    cudaMemcpy(counters, c->stats, KID_COUNT * 4 * sizeof(unsigned long long),
               cudaMemcpyDeviceToHost);
  return k;
}

extern "C" long long mr3_cuda_last_launches(const mr3_cuda_ctx *c) { return c ? c->launches : 0; }
extern "C" const char *mr3_cuda_last_error(const mr3_cuda_ctx *c) { return c ? c->err : ""; }

static int valid_prob(const mr3_cuda_prob &q) {
  if (q.jobz < MR3_JOB_N || q.jobz > MR3_JOB_C) return 0;
  if (q.range < MR3_RANGE_A || q.range > MR3_RANGE_I) return 0;
  if (q.n <= 0) return 0;
  if (q.range == MR3_RANGE_V && !(q.vu > q.vl)) return 0;
  if (q.range == MR3_RANGE_I && (q.il < 1 || q.il > q.n || q.iu < q.il || q.iu > q.n)) return 0;
  if (q.jobz == MR3_JOB_V && q.ldz < q.n) return 0;
  return 1;
}

// Sort the records of the problems selected by (want_job, flag) in place in
// rec0/rec1; returns the buffer holding the result.
static int merge_sort_impl(mr3_cuda_ctx *c, cudaStream_t st, int N, int mmax, int want_job,
                           const int *flag, SortRec **result) {
  SortRec *in = c->rec0, *out = c->rec1;
  // every pass writes every element of every selected problem
  for (int width = 1; width < mmax; width *= 2) {
    LAUNCH(k_merge_pass, (N + 255) / 256, 256, N, c->probs, c->prob_of_slot, in, out, width,
           want_job, flag);
    std::swap(in, out);
  }
  *result = in;
  return MR3_OK;
}

static SortRec *merge_sort(mr3_cuda_ctx *c, cudaStream_t st, int N, int mmax, int want_job,
                           const int *flag, int *rc) {
  SortRec *r = c->rec0;
  *rc = merge_sort_impl(c, st, N, mmax, want_job, flag, &r);
  return r;
}

extern "C" int mr3_cuda_solve(mr3_cuda_ctx *c, int P, mr3_cuda_prob *pr, void *stream) {
  return mr3_cuda_solve_cb(c, P, pr, stream, nullptr, nullptr);
}

extern "C" int mr3_cuda_solve_cb(mr3_cuda_ctx *c, int P, mr3_cuda_prob *pr, void *stream,
                                 mr3_cuda_done_fn done_fn, void *user) {
  if (!c) return MR3_EMISC;
  cudaStream_t st = stream ? (cudaStream_t)stream : c->own;
  // MR3_TREE_LANES caps the lanes per bisection interval (1: a thread each);
  // tests use it to run both forms on small problems
  int tree_max = 32;
  if (const char *ev = getenv("MR3_TREE_LANES")) tree_max = atoi(ev);
  c->launches = 0;
  c->err[0] = 0;
  CK(cudaSetDevice(c->device), "cudaSetDevice");
  if (P <= 0) return MR3_OK;
  // rounds of an earlier solve that ended early (an error) finish first
  CK(cudaStreamWaitEvent(st, c->rnd_done, 0), "rounds wait");

  // ---- host-side triage: invalid and trivial problems
  size_t N = 0;
  int nmaxV = 0, mmax = 0, nlive = 0;
  bool anyV = false, anyN = false, anyTry = false;
  std::vector<int> off(P), live(P, 0);
  for (int i = 0; i < P; i++) {
    mr3_cuda_prob &q = pr[i];
    q.m = 0;
    q.info = MR3_OK;
    q.il_out = q.il; q.iu_out = q.iu; q.vl_out = q.vl; q.vu_out = q.vu; q.tryrac_out = q.tryrac;
    off[i] = (int)N;
    if (!valid_prob(q)) { q.info = MR3_EARG; continue; }
    if (q.jobz == MR3_JOB_C && q.range != MR3_RANGE_V) {   // SRC/mrrr.c:130-138
      q.m = (q.range == MR3_RANGE_A) ? q.n : q.iu - q.il + 1;
      continue;
    }
    if (q.n == 1) {   // a 1x1 matrix: its entry is the eigenvalue
      double d0;
      CK(cudaMemcpyAsync(&d0, q.D, sizeof(double), cudaMemcpyDeviceToHost, st), "n1 D");
      CK(cudaStreamSynchronize(st), "n1 sync");
      bool take = q.range != MR3_RANGE_V || (d0 > q.vl && d0 <= q.vu);
      q.m = take ? 1 : 0;
      if (take && q.jobz != MR3_JOB_C) {
        CK(cudaMemcpyAsync(q.W, q.D, sizeof(double), cudaMemcpyDeviceToDevice, st), "n1 W");
        if (q.jobz == MR3_JOB_V) {
          CK(cudaMemcpyAsync(q.Z, c->h_const, sizeof(double), cudaMemcpyHostToDevice, st), "n1 Z");
          CK(cudaMemcpyAsync(q.Zsupp, c->h_iconst, 2 * sizeof(int), cudaMemcpyHostToDevice, st),
             "n1 Zsupp");
        }
      }
      continue;
    }
    live[i] = 1;
    nlive++;
    N += (size_t)q.n;
    mmax = std::max(mmax, q.n);
    if (q.jobz == MR3_JOB_V) { anyV = true; nmaxV = std::max(nmaxV, q.n); }
    if (q.jobz == MR3_JOB_N) anyN = true;
    if (q.tryrac) anyTry = true;
  }
  if (nlive == 0) return cudaStreamSynchronize(st) == cudaSuccess ? MR3_OK : MR3_EMISC;

  // compact the live problems
  std::vector<int> idx;
  idx.reserve(nlive);
  for (int i = 0; i < P; i++)
    if (live[i]) idx.push_back(i);
  int rc = ensure_rows(c, 0, (size_t)nlive);
  if (rc != MR3_OK) return rc;
  {
    // a problem with a non-finite entry is refused (info 2) before the
    // solve, so that it cannot disturb the others of the batch
    const int Lc = nlive;
    for (int k = 0; k < Lc; k++) {
      c->h_probs[k].n = pr[idx[k]].n;
      c->h_ptrs[k] = (void *)pr[idx[k]].D;
      c->h_ptrs[Lc + k] = (void *)pr[idx[k]].E;
    }
    CK(cudaMemcpyAsync(c->probs, c->h_probs, Lc * sizeof(ProbDev), cudaMemcpyHostToDevice, st),
       "screen probs");
    CK(cudaMemcpyAsync(c->Din, c->h_ptrs, Lc * sizeof(void *), cudaMemcpyHostToDevice, st),
       "screen D");
    CK(cudaMemcpyAsync(c->Ein, c->h_ptrs + Lc, Lc * sizeof(void *), cudaMemcpyHostToDevice, st),
       "screen E");
    LAUNCH(k_finite, Lc, 256, c->probs, c->Din, c->Ein, c->flag);
    CK(cudaMemcpyAsync(c->h_flag, c->flag, Lc * sizeof(int), cudaMemcpyDeviceToHost, st),
       "screen flags");
    CK(cudaStreamSynchronize(st), "screen sync");
    int kept = 0;
    for (int k = 0; k < Lc; k++) {
      mr3_cuda_prob &q = pr[idx[k]];
      if (c->h_flag[k]) {
        q.info = MR3_EMISC;
        N -= (size_t)q.n;
        nlive--;
      } else {
        idx[kept++] = idx[k];
      }
    }
    idx.resize(kept);
    if (nlive == 0) return MR3_OK;
    mmax = 0; nmaxV = 0; anyV = anyN = anyTry = false;
    for (int i : idx) {
      const mr3_cuda_prob &q = pr[i];
      mmax = std::max(mmax, q.n);
      if (q.jobz == MR3_JOB_V) { anyV = true; nmaxV = std::max(nmaxV, q.n); }
      if (q.jobz == MR3_JOB_N) anyN = true;
      if (q.tryrac) anyTry = true;
    }
  }
  const int L = nlive;
  rc = ensure_rows(c, N, (size_t)L);
  if (rc != MR3_OK) return rc;
  // column tiles of the problems whose column count is known up front
  // (jobz V, range A or I); finished tiles are reported to done_fn at the
  // host's syncs (the kernels that wrote them have finished)
  std::vector<int> mest(L, 0);
  size_t ntiles = 0;
  for (int k = 0; k < L; k++) {
    const mr3_cuda_prob &q = pr[idx[k]];
    if (q.jobz == MR3_JOB_V && q.range != MR3_RANGE_V)
      mest[k] = q.range == MR3_RANGE_I ? q.iu - q.il + 1 : q.n;
    ntiles += (mest[k] + ZT_COLS - 1) / ZT_COLS;
  }
  if (done_fn && ntiles > c->capTiles) {
    CK(cudaStreamSynchronize(st), "tiles sync");
    CK(regrow(&c->tile_left, ntiles), "tile_left");
    CK(regrow(&c->done_list, ntiles), "done_list");
    if (c->h_done) cudaFreeHost(c->h_done);
    c->h_done = nullptr;
    CK(cudaMallocHost((void **)&c->h_done, ntiles * sizeof(int2)), "h_done");
    CK(cudaHostGetDevicePointer((void **)&c->d_hdone, c->h_done, 0), "h_done view");
    c->capTiles = ntiles;
  }
  const bool tiles = done_fn && ntiles > 0;
  int reported = 0;
  auto report_upto = [&](int upto) -> int {
    if (!tiles || upto <= reported) return MR3_OK;
    // the new tiles in (problem, tile) order, adjacent tiles of a problem
    // merged into one range
    c->h_runs.assign(c->h_done + reported, c->h_done + upto);
    std::sort(c->h_runs.begin(), c->h_runs.end(), [](int2 a, int2 b) {
      return a.x != b.x ? a.x < b.x : a.y < b.y;
    });
    c->h_dprob.clear();
    c->h_dcol.clear();
    c->h_dcnt.clear();
    for (size_t t = 0; t < c->h_runs.size();) {
      size_t u = t + 1;
      while (u < c->h_runs.size() && c->h_runs[u].x == c->h_runs[t].x &&
             c->h_runs[u].y == c->h_runs[u - 1].y + 1)
        u++;
      const int k = c->h_runs[t].x, c0 = c->h_runs[t].y * ZT_COLS;
      c->h_dprob.push_back(idx[k]);
      c->h_dcol.push_back(c0);
      c->h_dcnt.push_back(std::min((c->h_runs[u - 1].y + 1) * ZT_COLS, mest[k]) - c0);
      t = u;
    }
    done_fn(user, c->h_dprob.data(), c->h_dcol.data(), c->h_dcnt.data(), (int)c->h_dprob.size());
    reported = upto;
    return MR3_OK;
  };
  auto report_done = [&]() -> int { return report_upto(c->h_sc->done_n); };
  // singleton rounds whose finished tiles are exported but not yet reported
  int npend = 0;
  // the counters (and the tiles finished since the last export) go to the
  // host through k_export; the host waits for it, reporting the tiles of
  // the rounds before it as they complete
  auto sync_counters = [&](LevelCounters *lc, const char *what) -> int {
    LAUNCH(k_export, 1, 256, lc, lc ? c->d_hlc : nullptr, c->sc, c->d_hsc, c->done_list,
           tiles ? c->d_hdone : nullptr, nullptr);
    for (int i = 0; i < npend; i++) {
      CK(cudaEventSynchronize(c->rev[i]), "round event");
      int rc2 = report_upto(c->h_snap[i]);
      if (rc2 != MR3_OK) return rc2;
    }
    npend = 0;
    CK(cudaStreamSynchronize(st), what);
    return MR3_OK;
  };
  const int NN = (int)N;
  {
    int o = 0, tb = 0;
    for (int k = 0; k < L; k++) {
      const mr3_cuda_prob &q = pr[idx[k]];
      ProbDev &h = c->h_probs[k];
      memset(&h, 0, sizeof(ProbDev));
      h.tbase = (done_fn && mest[k] > 0) ? tb : -1;
      if (h.tbase >= 0) tb += (mest[k] + ZT_COLS - 1) / ZT_COLS;
      h.n = q.n; h.off = o; h.jobz = q.jobz; h.range = q.range; h.il = q.il; h.iu = q.iu;
      h.tryrac = q.tryrac; h.ldz = q.ldz; h.vl = q.vl; h.vu = q.vu; h.Z = q.Z; h.Zsupp = q.Zsupp;
      h.scale = 1.0;
      o += q.n;
      c->h_ptrs[k] = (void *)q.D;
      c->h_ptrs[L + k] = (void *)q.E;
      c->h_ptrs[2 * L + k] = (void *)q.W;
      c->h_ptrs[3 * L + k] = (void *)q.D;
      c->h_ptrs[4 * L + k] = (void *)q.E;
    }
  }
  CK(cudaMemcpyAsync(c->probs, c->h_probs, L * sizeof(ProbDev), cudaMemcpyHostToDevice, st), "probs");
  CK(cudaMemcpyAsync(c->Din, c->h_ptrs, L * sizeof(void *), cudaMemcpyHostToDevice, st), "Din");
  CK(cudaMemcpyAsync(c->Ein, c->h_ptrs + L, L * sizeof(void *), cudaMemcpyHostToDevice, st), "Ein");
  CK(cudaMemcpyAsync(c->Wp, c->h_ptrs + 2 * L, L * sizeof(void *), cudaMemcpyHostToDevice, st), "Wp");
  CK(cudaMemcpyAsync(c->Dp, c->h_ptrs + 3 * L, L * sizeof(void *), cudaMemcpyHostToDevice, st), "Dp");
  CK(cudaMemcpyAsync(c->Ep, c->h_ptrs + 4 * L, L * sizeof(void *), cudaMemcpyHostToDevice, st), "Ep");

  Tol tol;
  tol.rtol1 = fmin(sqrt(2.220446049250313e-16), 1e-2 * 1e-3);
  tol.rtol2 = fmax(fmin(tol.rtol1 * 5.0E-3, 1e-3 * 5.0E-6), 4.0 * 2.220446049250313e-16);
  tol.bsrtol = fmin(1e-3 * 1.0E-2, sqrt(2.220446049250313e-16));
  tol.rqtol = 2.0 * 2.220446049250313e-16;
  // the reference picks dqds over bisection when its thread count is low
  // (SRC/mrrr_val.c:279-285); MR3_NTHREADS sets the count that choice sees,
  // unset the GPU's parallelism, for which the reference bisects
  tol.nthreads = 1 << 30;
  if (const char *ev = getenv("MR3_NTHREADS"))
    if (*ev) tol.nthreads = atoi(ev);
  const int gN = (NN + 255) / 256, gN128 = (NN + 127) / 128;

  // ---- stage A: eigenvalues
  LAUNCH(k_gather, L, 256, c->probs, c->Din, c->Ein, c->D, c->E, c->prob_of_slot, c->iblk);
  LAUNCH(k_prologue, L, MR3_THREADS, c->probs, c->blocks, c->blk_of_row, c->D, c->E, c->E2,
         c->gers, c->TP, c->TPc, tol);
  LAUNCH(k_blocks, L, MR3_THREADS, c->probs, c->blocks, c->D, c->E, c->gers, c->TP, tol);
  unsigned long long *stats = c->prof ? c->stats : nullptr;
  {
    const int Lb = tree_lanes(NN, (long long)c->nsm * MR3_TREE_BUDGET, tree_max);
    if (Lb == 1) {
      // shared intervals breadth-first, then a thread per eigenvalue
      CK(cudaMemsetAsync(c->bis_st, 0xff, N * sizeof(BisState), st), "bis st");
      CK(cudaMemsetAsync(c->bis_n, 0, 2 * sizeof(int), st), "bis n");
      LAUNCH(k_bis_roots, gN, 256, NN, c->probs, c->blocks, c->blk_of_row, c->bis_nodes[0],
             c->bis_n, c->Wt, c->Et, c->It, c->bis_st);
      // BIS_DEPTH levels without a host synchronisation: each level's length
      // stays on the device (bis_n[level parity]); a node holds at least two
      // eigenvalues, so no level exceeds N/2 nodes, the grid's bound
      const int nbmax = (int)((N / 2 + 1 + 255) / 256);
      int cur = 0;
      for (int depth = 0; depth < BIS_DEPTH; depth++) {
        const int split = depth + 1 >= BIS_DEPTH;
        LAUNCH(k_bis_count, nbmax, 256, c->bis_nodes[cur], c->bis_n + cur, c->probs, c->blocks,
               c->TP, tol, c->bis_cnt, c->bis_bcnt, c->Wt, c->Et, c->It, c->bis_st, stats);
        if (!split) LAUNCH(k_bis_scan, 1, 1024, nbmax, c->bis_bcnt, c->bis_n + (cur ^ 1));
        LAUNCH(k_bis_scatter, nbmax, 256, c->bis_nodes[cur], c->bis_n + cur, c->probs, c->blocks,
               tol, c->bis_cnt, c->bis_bcnt, c->bis_nodes[cur ^ 1], split, c->Wt, c->Et, c->It,
               c->bis_st);
        cur ^= 1;
      }
      LAUNCH(k_bisect_cont, gN128, 128, NN, c->probs, c->blocks, c->blk_of_row, c->TP, c->Wt,
             c->Et, c->It, c->bis_st, tol, stats);
    } else
      LAUNCH(k_bisect<true>, (int)(((long long)NN * Lb + 127) / 128), 128, NN, Lb, c->probs,
             c->blocks, c->blk_of_row, c->TP, c->Wt, c->Et, c->It, tol, stats);
  }
  LAUNCH(k_compact, L, MR3_THREADS, c->probs, c->blocks, c->D, c->Wt, c->Et, c->It, c->W, c->Werr,
         c->Windex, c->iblk, c->Wcopy, c->tile_left);
  LAUNCH(k_gaps_init, gN, 256, NN, c->probs, c->blocks, c->iblk, c->W, c->Werr, c->Wgap);
  LAUNCH(k_root, L, MR3_THREADS, c->probs, c->blocks, c->D, c->E, c->TP, c->Dt, c->Lt, c->W,
         c->Werr, c->Wgap, c->RP, c->RQ);
  {
    const int Lr = tree_lanes(NN, (long long)c->nsm * MR3_TREE_BUDGET, tree_max);
    if (Lr == 1)
      LAUNCH(k_refine_root<false>, gN128, 128, NN, 1, c->probs, c->blocks, c->iblk, c->RP, c->W,
             c->Werr, c->Wgap, tol, stats);
    else
      LAUNCH(k_refine_root<true>, (int)(((long long)NN * Lr + 127) / 128), 128, NN, Lr, c->probs,
             c->blocks, c->iblk, c->RP, c->W, c->Werr, c->Wgap, tol, stats);
  }
  if (tol.nthreads < (1 << 30))
    LAUNCH(k_dqds, gN, 256, NN, c->probs, c->blocks, c->blk_of_row, c->D, c->E, c->W, c->Werr,
           c->qd);
  LAUNCH(k_gaps_root, gN, 256, NN, c->probs, c->blocks, c->iblk, c->W, c->Werr, c->Wgap);
  LAUNCH(k_discard, (L + 127) / 128, 128, c->probs, L, c->blocks, c->W, c->Werr, c->Wgap,
         c->Windex, c->iblk, c->Wcopy);

  // ---- stage B: eigenvectors
  if (anyV) {
    LAUNCH(k_zkeys, L, MR3_THREADS, c->probs, c->blocks, c->W, c->E, c->Windex, c->rec0);
    SortRec *sorted = merge_sort(c, st, NN, mmax, MR3_JOB_V, nullptr, &rc);
    if (rc != MR3_OK) { snprintf(c->err, sizeof(c->err), "merge sort"); return rc; }
    LAUNCH(k_zindex_from_sorted, gN, 256, NN, c->probs, c->prob_of_slot, sorted, c->Zindex);
    CK(cudaMemsetAsync(c->lc, 0, 2 * sizeof(LevelCounters), st), "lc");
    CK(cudaMemsetAsync(c->sc, 0, sizeof(SngCounters), st), "sc");
    CK(cudaMemsetAsync(c->lvl_of_slot, 0xff, N * sizeof(int), st), "lvl");
    LAUNCH(k_level0, L, MR3_THREADS, c->probs, c->blocks, c->E, c->gers, c->W, c->Werr, c->Wsh,
           c->cl[0], &c->lc[0], c->sc, c->unit_list);
    if ((rc = sync_counters(c->lc, "level0 sync")) != MR3_OK) return rc;
    if (c->h_sc->n_unit > 0)
      LAUNCH(k_unitvec, c->h_sc->n_unit, 256, c->unit_list, c->sc, c->probs, c->blocks, c->iblk,
             c->Zindex, c->done_list, c->tile_left);
    // singleton scratch: the checkpoints of 32 lanes per persistent warp
    const size_t per_warp = 3ull * ((size_t)nmaxV / CK_K + 1) * 32ull;
    const size_t budget = c->round_scratch;   // bytes
    // persistent warps: no more than can be resident at once
    const size_t resident = (size_t)c->nsm * (size_t)c->sng_ctas_per_sm * SNG_WARPS;
    size_t nwarps = std::min<size_t>(resident, std::max<size_t>(c->nsm, budget / (per_warp * 8)));
    nwarps = (nwarps + SNG_WARPS - 1) / SNG_WARPS * SNG_WARPS;
    if (nwarps * per_warp > c->capScratch) {
      CK(regrow(&c->scratch, nwarps * per_warp), "scratch");
      c->capScratch = nwarps * per_warp;
    }
    int ncl = c->h_lc[0].n_cl;
    const int DEPTH_CAP = 512;
    ClsScratch xs;
    xs.ns = c->cls_ns; xs.soff = c->cls_soff; xs.cbase = c->cls_cbase; xs.abase = c->cls_abase;
    const long long lanes = (long long)c->nsm * MR3_TREE_BUDGET;   // lanes a launch can keep busy
    bool rounds_pending = false;
    for (int level = 0; ncl > 0; level++) {
      if (level >= DEPTH_CAP) { snprintf(c->err, sizeof(c->err), "representation tree too deep"); return MR3_EMISC; }
      const int cur = level & 1, nxt = cur ^ 1;
      const int gW = (ncl * 32 + MR3_THREADS - 1) / MR3_THREADS;
      if (level > 0) {
        const int Lx = tree_lanes(2LL * ncl, lanes, tree_max);
        if (Lx == 1)
          LAUNCH(k_cl_ext<false>, (int)((2LL * ncl + 127) / 128), 128, ncl, 1, c->cl[cur], c->probs,
                 c->blocks, c->RP, c->RQ, c->arena[nxt], c->Wsh, c->Werr, c->Windex, c->Wt, c->Et,
                 tol, stats);
        else
          LAUNCH(k_cl_ext<true>, (int)((2LL * ncl * Lx + 127) / 128), 128, ncl, Lx, c->cl[cur],
                 c->probs, c->blocks, c->RP, c->RQ, c->arena[nxt], c->Wsh, c->Werr, c->Windex, c->Wt,
                 c->Et, tol, stats);
        // two lanes per cluster when the clusters leave lanes idle
        if (2LL * ncl <= lanes)
          LAUNCH(k_cl_rrf<true>, (int)((2LL * ncl + 127) / 128), 128, ncl, c->cl[cur], c->probs,
                 c->blocks, c->RP, c->RQ, c->arena[nxt], c->arena[cur], c->Wt, c->Et, c->Wsh,
                 c->Werr, c->Wgap, stats);
        else
          LAUNCH(k_cl_rrf<false>, (ncl + 127) / 128, 128, ncl, c->cl[cur], c->probs, c->blocks,
                 c->RP, c->RQ, c->arena[nxt], c->arena[cur], c->Wt, c->Et, c->Wsh, c->Werr,
                 c->Wgap, stats);
        CK(cudaMemsetAsync(c->rl_n, 0, sizeof(int), st), "rl_n");
        LAUNCH(k_cl_pack, std::min(ncl, 65535 * 16), 256, ncl, c->cl[cur], c->blocks, c->arena[cur],
               c->Wsh, c->Werr, c->cl_of_slot, c->lvl_of_slot, level, c->rl_n);
        {
          const int nrb = (int)((NN + RL_T - 1) / RL_T);
          LAUNCH(k_rl_count, nrb, 256, NN, c->lvl_of_slot, level, c->rlcnt);
          LAUNCH(k_rl_scan, 1, 1024, nrb, c->rlcnt);
          LAUNCH(k_rl_scatter, nrb, 256, NN, c->lvl_of_slot, level, c->rlcnt, c->rl);
        }
        // both forms are launched; the one that does not match the list's
        // length returns at once (the length is known on the device only)
        LAUNCH(k_refine_cl<false>, gN128, 128, c->rl, c->rl_n, c->cl[cur], c->probs, c->blocks,
               c->arena[cur], c->Wsh, c->Werr, c->Wgap, c->Windex, c->cl_of_slot, c->lvl_of_slot,
               level, tol, lanes, tree_max, stats);
        LAUNCH(k_refine_cl<true>, (int)(lanes / 128), 128, c->rl, c->rl_n, c->cl[cur], c->probs,
               c->blocks, c->arena[cur], c->Wsh, c->Werr, c->Wgap, c->Windex, c->cl_of_slot,
               c->lvl_of_slot, level, tol, lanes, tree_max, stats);
        LAUNCH(k_gaps_cl, gN, 256, NN, c->cl[cur], c->Wsh, c->Werr, c->Wgap, c->W, c->cl_of_slot,
               c->lvl_of_slot, level);
      }
      // the classification below rewrites the singleton records and the
      // cluster records that the previous level's rounds read
      if (rounds_pending) {
        CK(cudaStreamWaitEvent(st, c->rnd_done, 0), "rounds wait");
        rounds_pending = false;
      }
      CK(cudaMemsetAsync(&c->lc[nxt], 0, sizeof(LevelCounters), st), "lcn");
      CK(cudaMemsetAsync(&c->sc->n_sng, 0, sizeof(int), st), "scn");
      LAUNCH(k_classify<0>, gW, MR3_THREADS, ncl, c->cl[cur], c->blocks, c->Wsh, c->Wgap,
             c->cl[nxt], c->sng, &c->lc[nxt], xs, NN);
      CK(cudaMemsetAsync(c->sbk, 0, 3 * SNG_BUCKETS * sizeof(int), st), "sbk");
      LAUNCH(k_group_tasks<0>, (ncl + 127) / 128, 128, ncl, c->cl[cur], c->blocks, xs, c->sc, c->sbk,
             &c->lc[nxt], NN);
      LAUNCH(k_bucket_scan, 1, 1, c->sbk);
      LAUNCH(k_group_tasks<1>, (ncl + 127) / 128, 128, ncl, c->cl[cur], c->blocks, xs, c->sc, c->sbk,
             &c->lc[nxt], NN);
      LAUNCH(k_classify<1>, gW, MR3_THREADS, ncl, c->cl[cur], c->blocks, c->Wsh, c->Wgap,
             c->cl[nxt], c->sng, &c->lc[nxt], xs, NN);
      if ((rc = sync_counters(&c->lc[nxt], "level sync")) != MR3_OK) return rc;
      if (c->h_lc->err) { snprintf(c->err, sizeof(c->err), "queue overflow"); return MR3_EMISC; }
      if ((rc = report_done()) != MR3_OK) return rc;
      if (c->h_sc->err) { snprintf(c->err, sizeof(c->err), "singleton rounds exhausted"); return MR3_EMISC; }
      if (c->h_sc->n_sng > 0) {
        // the level's singletons in rounds (see k_sng_round), on their own
        // stream: the next level's cluster kernels (which read and write
        // neither their records nor their eigenvalue slots) run beside the
        // rounds' short tail.  Profiling with serialised streams (prof 2)
        // keeps them on the solve's stream, so that every kernel's events
        // bracket that kernel alone.
        const cudaStream_t st_solve = st;
        cudaStream_t st = (c->prof == 2) ? st_solve : c->rnd;
        rounds_pending = true;
        const int nsng = c->h_sc->n_sng;
        const int ctas_all = (int)(nwarps / SNG_WARPS);
        const int ctas_first = std::min(ctas_all, (nsng + 32 * SNG_WARPS - 1) / (32 * SNG_WARPS));
        const size_t smem = SNG_TILE_BYTES;
        const int bis_ctas = c->nsm * 4;
        const int nblk = (nsng + LIST_T - 1) / LIST_T;
        // a list of at most this many singletons (four per persistent warp)
        // is finished in one launch (k_sng_finish), a warp each in turn;
        // MR3_FINISH_MAX overrides it (0: never).  A level's last few
        // thousand singletons are mostly ones that run all MAXITER calls and
        // the bisection; one round per call for them cost more than their
        // warps running the calls back to back (4096-problem batch: 44 ms
        // less per step with four per warp than with one)
        int finish_max = (int)std::min<size_t>(4 * nwarps, 1u << 30);
        if (const char *ev = getenv("MR3_FINISH_MAX")) finish_max = atoi(ev);
        // MR3_ITER_MAX: a list of at most this many is finished in one launch,
        // a lane each (k_sng_round<SNG_ITER>).  Off by default: a warp then
        // waits for its slowest lane and runs its lanes' bisections one after
        // another, and the step took longer than with the rounds (1049 ms
        // against 1009 ms on the 4096-problem batch, 279 ms against 178 ms on
        // a 256-problem one).
        int iter_max = 0;
        if (const char *ev = getenv("MR3_ITER_MAX")) iter_max = atoi(ev);
        // the split form of the finish (two sweeps at once, about half the
        // latency of a call); MR3_FINISH_SPLIT=0 gives lane 0's checkpointed
        // form
        bool split = true;
        if (const char *ev = getenv("MR3_FINISH_SPLIT")) split = atoi(ev) != 0;
        int fin_ctas = ctas_all;
        if (split) {
          // warps of the split finish: their row scratch (5 (nmax + 2) doubles
          // each) kept within 2 GB, at least one CTA per SM
          const size_t per = 5ull * ((size_t)nmaxV + 2) * sizeof(double);
          size_t fw = std::min<size_t>(nwarps, std::max<size_t>((size_t)c->nsm * SNG_WARPS,
                                                                ((size_t)2 << 30) / per));
          fw = fw / SNG_WARPS * SNG_WARPS;
          fin_ctas = (int)(fw / SNG_WARPS);
          if (fw * per > c->capFscratch) {
            CK(cudaStreamSynchronize(c->own), "fscratch sync");
            CK(cudaStreamSynchronize(c->rnd), "fscratch sync");
            CK(regrow(&c->fscratch, fw * per / sizeof(double)), "fscratch");
            c->capFscratch = fw * per;
          }
        }
        const bool trace_rounds = getenv("MR3_TRACE_ROUNDS") != nullptr;
        auto trace_t0 = std::chrono::steady_clock::now();
        if (trace_rounds) CK(cudaStreamSynchronize(st), "trace sync");
        trace_t0 = std::chrono::steady_clock::now();
        for (int rd = 0; rd < SNG_ROUNDS; rd++) {
          const int in = rd & 1, last = rd == SNG_ROUNDS - 1;
          LAUNCH(k_round_reset, 1, 1, c->sc, in, rd == 0);
          if (rd > 0 && split)
            LAUNCH(k_sng_finish<true>, fin_ctas, SNG_WARPS * 32, in, c->sng, c->cl[cur],
                   c->probs, c->blocks, c->RP, c->RQ, c->arena[cur], c->W, c->Wsh, c->Werr,
                   c->Wgap, c->Windex, c->Zindex, c->sst, c->act[0], c->act[1], c->sc,
                   c->scratch, c->fscratch, (long long)nmaxV, c->done_list, c->tile_left, stats);
          else if (rd > 0)
            LAUNCH(k_sng_finish<false>, ctas_all, SNG_WARPS * 32, in, c->sng, c->cl[cur],
                   c->probs, c->blocks, c->RP, c->RQ, c->arena[cur], c->W, c->Wsh, c->Werr,
                   c->Wgap, c->Windex, c->Zindex, c->sst, c->act[0], c->act[1], c->sc,
                   c->scratch, nullptr, (long long)nmaxV, c->done_list, c->tile_left, stats);
          if (rd > 0)
            LAUNCH_SMEM(k_sng_round<SNG_ITER>, ctas_all, SNG_WARPS * 32, smem, in, c->sng,
                        c->cl[cur], c->probs, c->blocks, c->RP, c->RQ, c->arena[cur], c->W, c->Wsh,
                        c->Werr, c->Wgap, c->Windex, c->Zindex, c->sst, c->act[0], c->act[1],
                        c->sflag, c->sc, c->scratch, (long long)nmaxV, c->done_list, c->tile_left,
                        stats);
          if (rd == 0)
            LAUNCH_SMEM(k_sng_round<SNG_FIRST>, ctas_first, SNG_WARPS * 32, smem, in, c->sng,
                        c->cl[cur], c->probs, c->blocks, c->RP, c->RQ, c->arena[cur], c->W, c->Wsh,
                        c->Werr, c->Wgap, c->Windex, c->Zindex, c->sst, c->act[0], c->act[1],
                        c->sflag, c->sc, c->scratch, (long long)nmaxV, c->done_list, c->tile_left,
                        stats);
          else
            LAUNCH_SMEM(k_sng_round<SNG_LATER>, ctas_all, SNG_WARPS * 32, smem, in, c->sng,
                        c->cl[cur], c->probs, c->blocks, c->RP, c->RQ, c->arena[cur], c->W, c->Wsh,
                        c->Werr, c->Wgap, c->Windex, c->Zindex, c->sst, c->act[0], c->act[1],
                        c->sflag, c->sc, c->scratch, (long long)nmaxV, c->done_list, c->tile_left,
                        stats);
          if (tiles) {
            LAUNCH(k_export, 1, 256, nullptr, nullptr, c->sc, nullptr, c->done_list, c->d_hdone,
                   c->d_hsnap + npend);
            CK(cudaEventRecord(c->rev[npend], st), "round record");
            npend++;
          }
          LAUNCH(k_list_count, nblk, 256, c->sc, c->sflag, c->sbcnt);
          LAUNCH(k_list_scan, 1, 1024, nblk, c->sc, c->sbcnt, in ^ 1, last, finish_max, iter_max);
          if (trace_rounds) {
            // MR3_TRACE_ROUNDS=1: each round's list lengths and wall time on
            // stderr (synchronises after every round; diagnostics only)
            SngCounters h;
            CK(cudaStreamSynchronize(st), "trace sync");
            CK(cudaMemcpy(&h, c->sc, sizeof(SngCounters), cudaMemcpyDeviceToHost), "trace copy");
            const auto now = std::chrono::steady_clock::now();
            fprintf(stderr, "mr3 trace: level %d round %d: in %d, next %d, bisection %d, mode %d, "
                    "%.2f ms\n", level, rd, h.nin, h.act_n[in ^ 1], h.bs_n, h.mode,
                    std::chrono::duration<double, std::milli>(now - trace_t0).count());
            trace_t0 = now;
          }
          LAUNCH(k_list_scatter, nblk, 256, rd == 0, c->sc, c->sflag, c->sbcnt, c->act[0],
                 c->act[1], in, c->bsl);
          if (!last) {
            LAUNCH(k_sng_bisect, bis_ctas, 256, in ^ 1, c->sng, c->cl[cur], c->probs, c->blocks,
                   c->RP, c->RQ, c->arena[cur], c->Windex, c->sst, c->bsl, c->act[0], c->act[1],
                   c->sc, stats);
            LAUNCH(k_list_sort, (nsng + LSORT_W - 1) / LSORT_W, 1024, c->sc, in ^ 1, c->act[0],
                   c->act[1], c->sng, c->sst);
          }
        }
        CK(cudaEventRecord(c->rnd_done, st), "rounds record");
      }
      ncl = c->h_lc->n_cl;
      const size_t need = (size_t)c->h_lc->arena_need;
      if (ncl > 0 && need > c->capArena[nxt]) {
        CK(cudaStreamSynchronize(st), "arena sync");
        size_t nsz = std::max(need, c->capArena[nxt] + c->capArena[nxt] / 2);
        CK(regrow(&c->arena[nxt], nsz), "arena");
        c->capArena[nxt] = nsz;
      }
    }
    if (rounds_pending) CK(cudaStreamWaitEvent(st, c->rnd_done, 0), "rounds wait");
    if ((rc = sync_counters(nullptr, "rounds sync")) != MR3_OK) return rc;
    if (c->h_sc->err) { snprintf(c->err, sizeof(c->err), "singleton rounds exhausted"); return MR3_EMISC; }
    if ((rc = report_done()) != MR3_OK) return rc;
  }

  // ---- post-processing (SRC/mrrr.c:262-285)
  if (anyN) LAUNCH(k_shift_w, gN, 256, NN, c->probs, c->blocks, c->iblk, c->E, c->W);
  if (anyTry)
    LAUNCH(k_highrac, gN128, 128, NN, c->probs, c->blocks, c->iblk, c->Windex, c->TPc, c->W,
           c->Werr);
  LAUNCH(k_invscale, gN, 256, NN, c->probs, c->blocks, c->iblk, c->W);
  if (anyV) {
    LAUNCH(k_place_w, gN, 256, NN, c->probs, c->prob_of_slot, c->W, c->Zindex, c->Wout);
    CK(cudaMemsetAsync(c->flag, 0, L * sizeof(int), st), "flag");
    LAUNCH(k_check_sorted, gN, 256, NN, c->probs, c->prob_of_slot, c->Wout, c->flag);
    CK(cudaMemcpyAsync(c->h_flag, c->flag, L * sizeof(int), cudaMemcpyDeviceToHost, st), "flag d2h");
    CK(cudaStreamSynchronize(st), "flag sync");
    bool anyUnsorted = false;
    for (int k = 0; k < L; k++) anyUnsorted |= (c->h_flag[k] != 0);
    if (anyUnsorted) {
      // bubble fix-up of sort_eigenpairs == stable sort by value of the
      // columns in output order; permute W, Zsupp and the Z columns
      LAUNCH(k_wkeys, gN, 256, NN, c->probs, c->prob_of_slot, c->Wout, c->rec0, MR3_JOB_V, c->flag);
      SortRec *sorted = merge_sort(c, st, NN, mmax, MR3_JOB_V, c->flag, &rc);
      if (rc != MR3_OK) return rc;
      LAUNCH(k_sorted_to_w, gN, 256, NN, c->probs, c->prob_of_slot, sorted, c->Wout, MR3_JOB_V, c->flag);
      LAUNCH(k_perm_zsupp, gN, 256, NN, c->probs, c->prob_of_slot, sorted, c->flag, c->tmp2);
      LAUNCH(k_perm_zsupp2, gN, 256, NN, c->probs, c->prob_of_slot, c->flag, c->tmp2);
      std::vector<SortRec> hrec(N);
      CK(cudaMemcpyAsync(hrec.data(), sorted, N * sizeof(SortRec), cudaMemcpyDeviceToHost, st), "perm d2h");
      CK(cudaMemcpyAsync(c->h_probs, c->probs, L * sizeof(ProbDev), cudaMemcpyDeviceToHost, st), "probs m");
      CK(cudaStreamSynchronize(st), "perm sync");
      for (int k = 0; k < L; k++) {
        if (!c->h_flag[k]) continue;
        const ProbDev &h = c->h_probs[k];
        std::vector<int> moved;
        for (int j = 0; j < h.m; j++)
          if (hrec[h.off + j].idx != j) moved.push_back(j);
        if (moved.empty()) continue;
        double *tmp = nullptr;
        size_t colsz = (size_t)h.n;
        CK(cudaMalloc((void **)&tmp, moved.size() * colsz * sizeof(double)), "perm tmp");
        for (size_t t = 0; t < moved.size(); t++)
          CK(cudaMemcpyAsync(tmp + t * colsz, h.Z + (size_t)hrec[h.off + moved[t]].idx * h.ldz,
                             colsz * sizeof(double), cudaMemcpyDeviceToDevice, st), "perm gather");
        for (size_t t = 0; t < moved.size(); t++)
          CK(cudaMemcpyAsync(h.Z + (size_t)moved[t] * h.ldz, tmp + t * colsz,
                             colsz * sizeof(double), cudaMemcpyDeviceToDevice, st), "perm scatter");
        CK(cudaStreamSynchronize(st), "perm done");
        cudaFree(tmp);
      }
      // columns were reordered: report these problems' columns again
      if (done_fn) {
        c->h_dprob.clear();
        c->h_dcol.clear();
        c->h_dcnt.clear();
        for (int k = 0; k < L; k++)
          if (c->h_flag[k] && c->h_probs[k].m > 0) {
            c->h_dprob.push_back(idx[k]);
            c->h_dcol.push_back(0);
            c->h_dcnt.push_back(c->h_probs[k].m);
          }
        if (!c->h_dprob.empty())
          done_fn(user, c->h_dprob.data(), c->h_dcol.data(), c->h_dcnt.data(),
                  (int)c->h_dprob.size());
      }
    }
  }
  if (anyN) {
    LAUNCH(k_wkeys, gN, 256, NN, c->probs, c->prob_of_slot, c->W, c->rec0, MR3_JOB_N, nullptr);
    SortRec *sorted = merge_sort(c, st, NN, mmax, MR3_JOB_N, nullptr, &rc);
    if (rc != MR3_OK) return rc;
    LAUNCH(k_sorted_to_w, gN, 256, NN, c->probs, c->prob_of_slot, sorted, c->Wout, MR3_JOB_N, nullptr);
  }
  LAUNCH(k_scatter, L, 256, c->probs, c->Wp, c->Dp, c->Ep, c->Wout, c->D, c->E);
  CK(cudaMemcpyAsync(c->h_probs, c->probs, L * sizeof(ProbDev), cudaMemcpyDeviceToHost, st), "probs d2h");
  CK(cudaStreamSynchronize(st), "final sync");
  if (c->prof) prof_flush(c);

  for (int k = 0; k < L; k++) {
    const ProbDev &h = c->h_probs[k];
    mr3_cuda_prob &q = pr[idx[k]];
    q.info = h.status ? MR3_EMISC : MR3_OK;
    q.m = h.m;
    q.tryrac_out = h.tryrac_out;
    // count-only calls return before the bounds are scaled back (SRC/mrrr.c:250-254)
    const bool unscale = (h.scale != 1.0) && q.jobz != MR3_JOB_C;
    const double inv = 1.0 / h.scale;
    q.vl_out = unscale ? h.vl_out * inv : h.vl_out;
    q.vu_out = unscale ? h.vu_out * inv : h.vu_out;
    if (q.jobz == MR3_JOB_C) { q.m = h.nvals; q.vl_out = h.vl; q.vu_out = h.vu; }
    q.il_out = h.il_out;
    q.iu_out = h.iu_out;
  }
  return MR3_OK;
}
