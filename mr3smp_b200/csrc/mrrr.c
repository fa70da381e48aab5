/*
 * mrrr.c -- C host library: the reference-compatible entry points.
 *
 * mrrr()/mrrr_() keep the argument contract of INCLUDE/mrrr.h:62-149 and the
 * argument checks of SRC/mrrr.c:119-138.  The solve itself runs on the GPU
 * through the C ABI of mr3_cuda.h; there is no CPU path.  Calls are reentrant:
 * each calling thread borrows a solver context from a small pool.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "mr3_b200.h"

#define POOL_MAX 64

typedef struct {
  mr3_cuda_ctx *ctx;
  int busy;
} pool_slot;

static pool_slot g_pool[POOL_MAX];
static pthread_mutex_t g_pool_mu = PTHREAD_MUTEX_INITIALIZER;
static __thread long long t_launches;
static __thread char t_err[256];

static int device_id(void)
{
  const char *s = getenv("MR3_DEVICE");
  return s ? atoi(s) : 0;
}

static int pool_acquire(void)
{
  int i, slot = -1;
  pthread_mutex_lock(&g_pool_mu);
  for (i = 0; i < POOL_MAX; i++) {
    if (g_pool[i].ctx && !g_pool[i].busy) { slot = i; break; }
  }
  if (slot < 0) {
    for (i = 0; i < POOL_MAX; i++) {
      if (!g_pool[i].ctx) {
        if (mr3_cuda_ctx_create(device_id(), &g_pool[i].ctx) == MR3_OK) slot = i;
        break;
      }
    }
  }
  if (slot >= 0) g_pool[slot].busy = 1;
  pthread_mutex_unlock(&g_pool_mu);
  return slot;
}

static void pool_release(int slot)
{
  const char *e = mr3_cuda_last_error(g_pool[slot].ctx);
  t_launches = mr3_cuda_last_launches(g_pool[slot].ctx);
  strncpy(t_err, e ? e : "", sizeof(t_err) - 1);
  t_err[sizeof(t_err) - 1] = 0;
  pthread_mutex_lock(&g_pool_mu);
  g_pool[slot].busy = 0;
  pthread_mutex_unlock(&g_pool_mu);
}

long long mr3_last_launches(void) { return t_launches; }
const char *mr3_last_error(void) { return t_err; }

static int job_code(char c)
{
  if (c == 'N' || c == 'n') return MR3_JOB_N;
  if (c == 'V' || c == 'v') return MR3_JOB_V;
  if (c == 'C' || c == 'c') return MR3_JOB_C;
  return -1;
}

static int range_code(char c)
{
  if (c == 'A' || c == 'a') return MR3_RANGE_A;
  if (c == 'V' || c == 'v') return MR3_RANGE_V;
  if (c == 'I' || c == 'i') return MR3_RANGE_I;
  return -1;
}

/* Number of eigenvector columns to reserve on the device for one problem. */
static int ncols_of(const mr3_host_prob *h, int jz, int rg)
{
  if (jz != MR3_JOB_V) return 0;
  if (rg == MR3_RANGE_I) return h->iu - h->il + 1;
  return h->n;
}

static size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

/* Whether the matrix entries the solver reads (D[0..n-1], E[0..n-2]) are
 * all finite.  The reference does not check; a NaN or infinity there makes
 * its bisection loop on meaningless counts.  Here such a problem is refused
 * before any launch with info = 2 and the other problems of its batch are
 * solved as if it were absent. */
int mr3__finite_input(const double *D, const double *E, int n)
{
  int i, ok = 1;
  for (i = 0; i < n; i++) ok &= isfinite(D[i]) != 0;
  for (i = 0; i + 1 < n; i++) ok &= isfinite(E[i]) != 0;
  return ok;
}

/* Batches whose eigenvectors exceed PIPE_MIN_BYTES are solved in chunks of
 * consecutive problems holding about PIPE_CHUNK_BYTES of Z each, so that the
 * device Z buffers stay within memory; the device-to-host copy of one
 * chunk's Z (on the context's copy stream) runs while the next chunk is
 * solved.  Two device Z buffers alternate; a chunk's solve waits for the
 * copies out of the buffer it reuses.  The device solves a large batch much
 * faster per eigenpair than a small one, so smaller chunks lose more in the
 * solves than the overlap wins (a 56 GB batch took 2.5 s whole and 3.1 s in
 * three chunks); chunking is for capacity only.  MR3_PIPE_BYTES in the
 * environment replaces both sizes (tests use it to chunk small batches). */
#define PIPE_MIN_BYTES ((size_t)80 << 30)
#define PIPE_CHUNK_BYTES ((size_t)40 << 30)
#define PIPE_MAX_CHUNKS 16

/* Columns c0 .. c0+m-1 of one problem's Z to the caller's array, on the
 * copy stream: one contiguous copy when the caller's Z has no padding
 * between columns (a pitched copy into pageable memory goes column by
 * column). */
static int copy_z(mr3_cuda_ctx *ctx, const mr3_host_prob *h, const mr3_cuda_prob *q, int c0, int m)
{
  double *dst = h->Z + (size_t)c0 * (size_t)h->ldz;
  const double *src = q->Z + (size_t)c0 * (size_t)q->ldz;
  if (h->ldz == q->ldz)
    return mr3_cuda_copy_on(ctx, MR3_STREAM_COPY, dst, src,
                            (size_t)h->ldz * (size_t)m * sizeof(double), 1);
  return mr3_cuda_copy2d_on(ctx, MR3_STREAM_COPY, dst, (size_t)h->ldz * sizeof(double), src,
                            (size_t)q->ldz * sizeof(double), (size_t)h->n * sizeof(double),
                            (size_t)m, 1);
}

/* Eigenvector copies started while the solve goes on: the solver reports
 * column tiles whose Z columns are complete (mr3_cuda_solve_cb). */
typedef struct {
  mr3_cuda_ctx *ctx;
  mr3_host_prob *hp;
  mr3_cuda_prob *dp;
  int *copied;   /* columns copied so far, per problem */
  int rc;
} early_copy;

static void on_done(void *user, const int *probs, const int *col0, const int *ncols, int count)
{
  early_copy *e = (early_copy *)user;
  int t;
  for (t = 0; t < count; t++) {
    const int i = probs[t];
    if (e->dp[i].jobz != MR3_JOB_V || ncols[t] <= 0) continue;
    if (copy_z(e->ctx, &e->hp[i], &e->dp[i], col0[t], ncols[t]) != MR3_OK) e->rc = MR3_EMISC;
    e->copied[i] += ncols[t];
  }
}

/* One batched solve of host problems on a given context (the body of
 * mr3_batched, also used by the serving workers, which own their contexts). */
__attribute__((visibility("hidden"))) int mr3__batched_on(mr3_cuda_ctx *ctx, int nprob, mr3_host_prob *hp)
{
  int i, c, rc = MR3_OK, worst = 0, nchunk = 1;
  int cbeg[PIPE_MAX_CHUNKS + 1];
  mr3_cuda_prob *dp;
  size_t nrow = 0, nzs = 0, ztot = 0, zmax = 0, small, pipe_min, pipe_chunk;
  size_t *zb, *orow, *ozs;
  int *copied;
  early_copy ec;
  char *base, *stage;
  double *dD, *dE, *dW, *dZb[2] = {NULL, NULL};
  int *dZs;
  if (nprob <= 0) return 0;
  dp = (mr3_cuda_prob *)calloc((size_t)nprob, sizeof(mr3_cuda_prob));
  zb = (size_t *)calloc(3 * (size_t)nprob, sizeof(size_t));
  copied = (int *)calloc((size_t)nprob, sizeof(int));
  if (!dp || !zb || !copied) { free(dp); free(zb); free(copied); return MR3_EMISC; }
  orow = zb + nprob;
  ozs = orow + nprob;
  for (i = 0; i < nprob; i++) {
    mr3_host_prob *h = &hp[i];
    int jz = job_code(h->jobz), rg = range_code(h->range);
    int ok = jz >= 0 && rg >= 0 && h->n > 0;
    if (ok && rg == MR3_RANGE_V) ok = h->vu > h->vl;
    if (ok && rg == MR3_RANGE_I) ok = h->il >= 1 && h->il <= h->n && h->iu >= h->il && h->iu <= h->n;
    if (ok && jz == MR3_JOB_V) ok = h->ldz >= h->n;
    dp[i].jobz = ok ? jz : -1;
    dp[i].range = ok ? rg : -1;
    if (!ok) continue;
    if (!(jz == MR3_JOB_C && rg != MR3_RANGE_V) && !mr3__finite_input(h->D, h->E, h->n)) {
      dp[i].jobz = -2;   /* non-finite input: info 2, not solved */
      continue;
    }
    orow[i] = nrow;
    ozs[i] = nzs;
    nrow += align_up((size_t)h->n, 32);
    nzs += align_up(2 * (size_t)h->n, 64);
    zb[i] = (size_t)h->n * (size_t)ncols_of(h, jz, rg) * sizeof(double);
    ztot += zb[i];
  }
  /* chunk boundaries: consecutive problems, about equal Z bytes */
  cbeg[0] = 0;
  {
    const char *ev = getenv("MR3_PIPE_BYTES");
    long long v = ev ? atoll(ev) : 0;
    pipe_min = v > 0 ? (size_t)v : PIPE_MIN_BYTES;
    pipe_chunk = v > 0 ? (size_t)v : PIPE_CHUNK_BYTES;
  }
  if (ztot > pipe_min) {
    size_t acc = 0, target;
    nchunk = (int)((ztot + pipe_chunk - 1) / pipe_chunk);
    if (nchunk > PIPE_MAX_CHUNKS) nchunk = PIPE_MAX_CHUNKS;
    if (nchunk > nprob) nchunk = nprob;
    target = ztot / (size_t)nchunk;
    c = 1;
    for (i = 0; i < nprob && c < nchunk; i++) {
      acc += zb[i];
      if (acc >= target * (size_t)c) cbeg[c++] = i + 1;
    }
    nchunk = c;
  }
  cbeg[nchunk] = nprob;
  for (c = 0; c < nchunk; c++) {
    size_t z = 0;
    for (i = cbeg[c]; i < cbeg[c + 1]; i++) z += zb[i];
    if (z > zmax) zmax = z;
  }
  if (!ctx) { free(dp); free(zb); free(copied); return MR3_EMISC; }
  /* device layout of the small arrays, mirrored by the staging buffer:
   * D | E | W (nrow doubles each) | Zsupp (nzs ints) */
  small = 3 * nrow * sizeof(double) + nzs * sizeof(int);
  base = (char *)mr3_cuda_ws(ctx, 0, small + 1024);
  dZb[0] = (double *)mr3_cuda_ws(ctx, 1, zmax + 256);
  if (nchunk > 1) dZb[1] = (double *)mr3_cuda_ws(ctx, 2, zmax + 256);
  stage = (char *)mr3_cuda_host_ws(ctx, small + 1024);
  if (!base || !dZb[0] || (nchunk > 1 && !dZb[1]) || !stage) { rc = MR3_EMISC; goto done; }
  dD = (double *)base;
  dE = dD + nrow;
  dW = dE + nrow;
  dZs = (int *)(dW + nrow);
  for (i = 0; i < nprob; i++) {
    mr3_host_prob *h = &hp[i];
    mr3_cuda_prob *q = &dp[i];
    q->n = h->n;
    q->il = h->il; q->iu = h->iu; q->tryrac = h->tryrac;
    q->vl = h->vl; q->vu = h->vu;
    if (q->jobz < 0) continue;
    q->D = dD + orow[i]; q->E = dE + orow[i]; q->W = dW + orow[i];
    q->ldz = h->n;
    q->Zsupp = (q->jobz == MR3_JOB_V) ? dZs + ozs[i] : NULL;
    memcpy((double *)stage + orow[i], h->D, (size_t)h->n * sizeof(double));
    memcpy((double *)stage + nrow + orow[i], h->E, (size_t)h->n * sizeof(double));
  }
  if (mr3_cuda_copy(ctx, base, stage, 2 * nrow * sizeof(double), 0) != MR3_OK) {
    rc = MR3_EMISC;
    goto done;
  }
  for (c = 0; c < nchunk; c++) {
    double *zbuf = dZb[c & 1];
    size_t oz = 0;
    for (i = cbeg[c]; i < cbeg[c + 1]; i++) {
      if (dp[i].jobz < 0) continue;
      dp[i].Z = (dp[i].jobz == MR3_JOB_V) ? zbuf + oz / sizeof(double) : NULL;
      oz += zb[i];
    }
    /* the buffer's previous chunk must have left it */
    if (c >= 2 && mr3_cuda_event(ctx, c & 1, -1, MR3_STREAM_MAIN) != MR3_OK) {
      rc = MR3_EMISC;
      goto done;
    }
    ec.ctx = ctx;
    ec.hp = hp + cbeg[c];
    ec.dp = dp + cbeg[c];
    ec.copied = copied + cbeg[c];
    ec.rc = MR3_OK;
    if (mr3_cuda_solve_cb(ctx, cbeg[c + 1] - cbeg[c], dp + cbeg[c], NULL, on_done, &ec) != MR3_OK ||
        ec.rc != MR3_OK || mr3_cuda_event(ctx, 2, MR3_STREAM_MAIN, MR3_STREAM_COPY) != MR3_OK) {
      rc = MR3_EMISC;
      goto done;
    }
    for (i = cbeg[c]; i < cbeg[c + 1]; i++) {
      mr3_host_prob *h = &hp[i];
      mr3_cuda_prob *q = &dp[i];
      /* the columns that were not all copied during the solve */
      if (q->jobz != MR3_JOB_V || q->info != MR3_OK || q->m <= 0 || copied[i] >= q->m) continue;
      if (copy_z(ctx, h, q, 0, q->m) != MR3_OK) {
        rc = MR3_EMISC;
        goto done;
      }
    }
    if (mr3_cuda_event(ctx, c & 1, MR3_STREAM_COPY, -1) != MR3_OK) { rc = MR3_EMISC; goto done; }
  }
  /* W, D, E and Zsupp of all problems in one copy, then to the callers' arrays */
  if (mr3_cuda_copy(ctx, stage, base, small, 1) != MR3_OK || mr3_cuda_sync_all(ctx) != MR3_OK) {
    rc = MR3_EMISC;
    goto done;
  }
  for (i = 0; i < nprob; i++) {
    mr3_host_prob *h = &hp[i];
    mr3_cuda_prob *q = &dp[i];
    h->m = 0;
    if (q->jobz < 0) { h->info = q->jobz == -2 ? MR3_EMISC : MR3_EARG; continue; }
    h->info = q->info;
    h->m = q->m;
    h->vl_out = q->vl_out; h->vu_out = q->vu_out;
    h->il_out = q->il_out; h->iu_out = q->iu_out;
    h->tryrac_out = q->tryrac_out;
    if (q->info != MR3_OK || q->jobz == MR3_JOB_C) continue;
    if (q->m > 0) memcpy(h->W, (double *)stage + 2 * nrow + orow[i], (size_t)q->m * sizeof(double));
    if (h->n > 1) {   /* a 1x1 problem's D and E are left as they were */
      memcpy(h->D, (double *)stage + orow[i], (size_t)h->n * sizeof(double));
      memcpy(h->E, (double *)stage + nrow + orow[i], (size_t)h->n * sizeof(double));
    }
    if (q->jobz == MR3_JOB_V && q->m > 0)
      memcpy(h->Zsupp, (int *)((double *)stage + 3 * nrow) + ozs[i], 2 * (size_t)q->m * sizeof(int));
  }
done:
  if (rc != MR3_OK) mr3_cuda_sync_all(ctx);
  for (i = 0; i < nprob; i++) {
    if (rc != MR3_OK) hp[i].info = dp[i].jobz == -1 ? MR3_EARG : MR3_EMISC;
    if (hp[i].info > worst) worst = hp[i].info;
  }
  free(dp);
  free(zb);
  free(copied);
  return worst;
}

int mr3_batched(int nprob, mr3_host_prob *hp)
{
  int rc, slot;
  if (nprob <= 0) return 0;
  slot = pool_acquire();
  if (slot < 0) return MR3_EMISC;
  rc = mr3__batched_on(g_pool[slot].ctx, nprob, hp);
  pool_release(slot);
  return rc;
}

int mr3_batched_device(int nprob, mr3_cuda_prob *probs, void *stream)
{
  int i, rc, worst = 0, slot = pool_acquire();
  if (slot < 0) return MR3_EMISC;
  rc = mr3_cuda_solve(g_pool[slot].ctx, nprob, probs, stream);
  pool_release(slot);
  if (rc != MR3_OK) return rc;
  for (i = 0; i < nprob; i++)
    if (probs[i].info > worst) worst = probs[i].info;
  return worst;
}

int mrrr(char *jobz, char *range, int *np, double *D, double *E, double *vl,
         double *vu, int *il, int *iu, int *tryrac, int *m, double *W,
         double *Z, int *ldz, int *Zsupp)
{
  int n = *np, jz = job_code(jobz[0]), rg = range_code(range[0]);
  mr3_host_prob h;
  /* argument checks of SRC/mrrr.c:119-126 */
  if (jz < 0 || rg < 0) return 1;
  if (n <= 0) return 1;
  if (rg == MR3_RANGE_V) {
    if (*vu <= *vl) return 1;
  } else if (rg == MR3_RANGE_I) {
    if (*il < 1 || *il > n || *iu < *il || *iu > n) return 1;
  }
  /* counting with range A or I needs no work (SRC/mrrr.c:130-138) */
  if (jz == MR3_JOB_C) {
    if (rg == MR3_RANGE_A) { *m = n; return 0; }
    if (rg == MR3_RANGE_I) { *m = *iu - *il + 1; return 0; }
  }
  if (jz == MR3_JOB_V && *ldz < n) return 1;
  if (!mr3__finite_input(D, E, n)) return 2;
  memset(&h, 0, sizeof(h));
  h.jobz = jobz[0]; h.range = range[0]; h.n = n;
  h.il = *il; h.iu = *iu; h.tryrac = *tryrac; h.ldz = (jz == MR3_JOB_V) ? *ldz : n;
  h.vl = *vl; h.vu = *vu;
  h.D = D; h.E = E; h.W = W; h.Z = Z; h.Zsupp = Zsupp;
  mr3_batched(1, &h);
  if (h.info != MR3_OK) return h.info;
  *m = h.m;
  if (n > 1) {
    *vl = h.vl_out; *vu = h.vu_out;
    *il = h.il_out; *iu = h.iu_out;
    *tryrac = h.tryrac_out;
  }
  return 0;
}

void mrrr_(char *jobz, char *range, int *n, double *D, double *E, double *vl,
           double *vu, int *il, int *iu, int *tryrac, int *m, double *W,
           double *Z, int *ldz, int *Zsupp, int *info)
{
  *info = mrrr(jobz, range, n, D, E, vl, vu, il, iu, tryrac, m, W, Z, ldz, Zsupp);
}
