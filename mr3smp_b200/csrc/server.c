/*
 * server.c -- serving front end: a stream of independent requests solved
 * with continuous batching.
 *
 * The reference answers one call at a time (mrrr, SRC/mrrr.c:87-296).  A
 * serving process instead receives a stream of requests (tridiagonal
 * problems of mixed sizes) and wants each answered soon after it arrives.
 *
 * The server runs several lanes.  A lane is a worker thread with its own
 * solver context, hence its own CUDA streams, so the batches of different
 * lanes run on the device at the same time.  All lanes admit from one FIFO
 * of pending requests: a lane that becomes free takes, in arrival order,
 * the queued requests that fit (a) the device-memory budget -- the bytes
 * held by all requests in flight on every lane (their eigenvectors plus the
 * solver's per-row arrays) stay within the server's budget -- and (b) the
 * lane's work cap, which keeps a batch short so that later arrivals are
 * admitted soon, and solves them in one batched pass.  A request that
 * arrives while other batches are on the GPU is admitted by the next lane
 * that frees up, and its batch overlaps theirs on the device.  The first
 * lanes are reserved for small requests (n <= MR3_SERVE_SMALL_N) and run
 * on high-priority streams, so that a large solve in flight holds them
 * back as little as possible; the others take requests of any size.
 *
 * Requests come in two kinds.  A host request (mr3_host_prob, meaning as
 * for mr3_batched) has its inputs and outputs in host memory; its
 * eigenvectors are copied back.  A device request (mr3_cuda_prob, meaning
 * as for mr3_batched_device) has D, E, W, Z and Zsupp resident in device
 * memory: nothing crosses PCIe and the results stay where the caller's next
 * device step reads them.  Either way the arrays must stay valid and
 * untouched until poll reports the request done.  Every request is solved
 * exactly as it would be alone: batching never changes a result (each
 * problem's computation is independent of the others in its batch).
 *
 * Settings (environment, read at create): MR3_SERVE_LANES (lanes, default
 * 4, at most 16), MR3_SERVE_SMALL_LANES (lanes reserved for small
 * requests, default 2), MR3_SERVE_BATCH_WORK (work cap of a batch in units
 * of eigenvector entries n*m, default 2^27, for the small-request lanes;
 * the other lanes take 8 times as much, so that several large solves --
 * each latency-bound alone -- share one pass).
 */
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "mr3_b200.h"

__attribute__((visibility("hidden"))) int mr3__batched_on(mr3_cuda_ctx *ctx, int nprob,
                                                       mr3_host_prob *hp);   /* mrrr.c */

#define SRV_MAXLANES 16
#define SRV_MAXBATCH 4096
#define SRV_SCAN 512                   /* queued requests a lane looks at */
#define SRV_SMALL_N 2048
#define SRV_DEFAULT_BUDGET ((size_t)120 << 30)
#define SRV_DEFAULT_WORK ((double)(1 << 27))

enum { T_QUEUED = 1, T_RUNNING = 2, T_DONE = 3 };
enum { K_HOST = 0, K_DEVICE = 1 };

/* One queued request as admission sees it. */
typedef struct {
  int kind, n;
  size_t bytes;
  double work;
} mr3__srv_view;

typedef struct {
  int kind, n;
  mr3_host_prob *hreq;
  mr3_cuda_prob *dreq;
  size_t bytes;
  double work;
  double t_submit, t_admit, t_done;
  int state;
} srv_ticket;

typedef struct {
  mr3_cuda_ctx *ctx;
  pthread_t th;
  int started, small_only;
  mr3_host_prob *hbatch;
  mr3_cuda_prob *dbatch;
  long long *ids;
  mr3__srv_view *view;   /* the queued requests admission looks at */
  long long *vpos;       /* and their queue positions */
  int *pick;
} srv_lane;

struct mr3_server {
  int device, nlanes;
  pthread_mutex_t mu;
  pthread_cond_t cv_work, cv_done;
  srv_ticket *t;          /* ticket k at t[k - 1] */
  long long nt, cap;
  long long *q;           /* FIFO of ticket ids; entries no longer queued are skipped */
  long long qhead, qtail, qcap;
  size_t budget, used;
  double work_cap;
  srv_lane lane[SRV_MAXLANES];
  int busy;               /* lanes with a batch in flight */
  int stop;
  long long batches, solved, overlapped;
};

static double now_ms(void)
{
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec * 1e3 + ts.tv_nsec * 1e-6;
}

static int env_int(const char *name, int dflt)
{
  const char *s = getenv(name);
  return s && *s ? atoi(s) : dflt;
}

static int is_v(int kind, const void *r)
{
  if (kind == K_HOST) {
    const char j = ((const mr3_host_prob *)r)->jobz;
    return j == 'V' || j == 'v';
  }
  return ((const mr3_cuda_prob *)r)->jobz == MR3_JOB_V;
}

/* Eigenvector columns a request produces. */
static size_t req_cols(int kind, const void *r)
{
  int n, il, iu, range_i;
  if (!is_v(kind, r)) return 0;
  if (kind == K_HOST) {
    const mr3_host_prob *h = (const mr3_host_prob *)r;
    n = h->n; il = h->il; iu = h->iu; range_i = h->range == 'I' || h->range == 'i';
  } else {
    const mr3_cuda_prob *d = (const mr3_cuda_prob *)r;
    n = d->n; il = d->il; iu = d->iu; range_i = d->range == MR3_RANGE_I;
  }
  return range_i ? (size_t)(iu - il + 1) : (size_t)n;
}

/* Device bytes a request holds while in flight: its eigenvectors and the
 * solver's per-row work arrays (about 70 doubles per row). */
static size_t request_bytes(int kind, const void *r, int n)
{
  return 8 * (size_t)n * req_cols(kind, r) + 560 * (size_t)n;
}

/* Work of a request in eigenvector entries (n per column), plus the
 * eigenvalue stage. */
static double request_work(int kind, const void *r, int n)
{
  return (double)n * (double)req_cols(kind, r) + 64.0 * n;
}

static int q_push(mr3_server *s, long long id)
{
  if (s->qtail == s->qcap) {
    long long live = s->qtail - s->qhead, ncap;
    long long *nv;
    if (s->qhead > 0 && live < s->qcap / 2) {
      memmove(s->q, s->q + s->qhead, (size_t)live * sizeof(long long));
      s->qtail = live;
      s->qhead = 0;
    } else {
      ncap = s->qcap ? 2 * s->qcap : 4096;
      nv = (long long *)realloc(s->q, (size_t)ncap * sizeof(long long));
      if (!nv) return -1;
      s->q = nv;
      s->qcap = ncap;
    }
  }
  s->q[s->qtail++] = id;
  return 0;
}

/* Advances the head past entries that are no longer queued. */
static void q_trim(mr3_server *s)
{
  while (s->qhead < s->qtail && s->t[s->q[s->qhead] - 1].state != T_QUEUED) s->qhead++;
}

static int lane_wants(const srv_lane *L, const srv_ticket *t)
{
  return !L->small_only || t->n <= SRV_SMALL_N;
}

/* Whether a request this lane may take is queued. */
static int q_has_work(mr3_server *s, const srv_lane *L)
{
  long long i, seen = 0;
  for (i = s->qhead; i < s->qtail && seen < SRV_SCAN; i++) {
    const srv_ticket *t = &s->t[s->q[i] - 1];
    if (t->state != T_QUEUED) continue;
    seen++;
    if (lane_wants(L, t)) return 1;
  }
  return 0;
}

/* Admission of one batch, on its own so that it can be tested without a
 * device: from nq queued requests in arrival order, the positions (in out,
 * at most maxk) of those a lane takes -- requests of the kind of the first
 * one taken, that the lane may take (small_only: n <= SRV_SMALL_N), that fit
 * the budget left (budget - used) and that keep the batch's work within
 * work_cap (the first one always does).  Returns their number. */
int mr3__srv_admit(const mr3__srv_view *v, int nq, int small_only, size_t budget, size_t used,
                   double work_cap, int maxk, int *out)
{
  int i, k = 0, kind = -1;
  double work = 0.0;
  for (i = 0; i < nq && k < maxk; i++) {
    if (small_only && v[i].n > SRV_SMALL_N) continue;
    if (kind >= 0 && v[i].kind != kind) continue;
    if (used + v[i].bytes > budget) continue;
    if (k > 0 && work + v[i].work > work_cap) continue;
    kind = v[i].kind;
    used += v[i].bytes;
    work += v[i].work;
    out[k++] = i;
  }
  return k;
}

typedef struct {
  mr3_server *s;
  int lane;
} lane_arg;

static void *lane_main(void *p)
{
  lane_arg *a = (lane_arg *)p;
  mr3_server *s = a->s;
  srv_lane *L = &s->lane[a->lane];
  free(a);
  mr3_cuda_set_device(L->ctx);
  pthread_mutex_lock(&s->mu);
  for (;;) {
    int k = 0, i, kind = -1;
    size_t bytes = 0;
    double work = 0.0, t0;
    long long j, seen = 0;
    q_trim(s);
    while (!s->stop && !q_has_work(s, L)) {
      pthread_cond_wait(&s->cv_work, &s->mu);
      q_trim(s);
    }
    if (s->stop && !q_has_work(s, L)) break;   /* stopping and nothing left for this lane */
    /* admission: queued requests in arrival order, of one kind, that fit the
     * budget left and the batch's work cap; a batch takes at least one */
    t0 = now_ms();
    for (j = s->qhead; j < s->qtail && seen < SRV_SCAN; j++) {
      const srv_ticket *t = &s->t[s->q[j] - 1];
      if (t->state != T_QUEUED) continue;
      L->view[seen].kind = t->kind;
      L->view[seen].n = t->n;
      L->view[seen].bytes = t->bytes;
      L->view[seen].work = t->work;
      L->vpos[seen] = j;
      seen++;
    }
    /* large requests are latency-bound solves that batch well together:
     * lanes of any size take 8 times the work of the small-request lanes */
    k = mr3__srv_admit(L->view, (int)seen, L->small_only, s->budget, s->used,
                       L->small_only ? s->work_cap : 8.0 * s->work_cap, SRV_MAXBATCH, L->pick);
    for (i = 0; i < k; i++) {
      const long long id = s->q[L->vpos[L->pick[i]]];
      srv_ticket *t = &s->t[id - 1];
      kind = t->kind;
      t->state = T_RUNNING;
      t->t_admit = t0;
      s->used += t->bytes;
      bytes += t->bytes;
      work += t->work;
      L->ids[i] = id;
      if (kind == K_HOST) L->hbatch[i] = *t->hreq;
      else L->dbatch[i] = *t->dreq;
    }
    if (k == 0) {
      /* everything this lane may take waits for budget: sleep until a
       * batch finishes (or a request arrives) */
      pthread_cond_wait(&s->cv_work, &s->mu);
      continue;
    }
    if (s->busy > 0) s->overlapped++;
    s->busy++;
    pthread_mutex_unlock(&s->mu);
    if (kind == K_HOST) {
      mr3__batched_on(L->ctx, k, L->hbatch);
    } else {
      if (mr3_cuda_solve(L->ctx, k, L->dbatch, NULL) != MR3_OK)
        for (i = 0; i < k; i++) L->dbatch[i].info = MR3_EMISC;
    }
    pthread_mutex_lock(&s->mu);
    {
      const double t1 = now_ms();
      for (i = 0; i < k; i++) {
        srv_ticket *t = &s->t[L->ids[i] - 1];
        if (kind == K_HOST) {
          mr3_host_prob *r = t->hreq;
          const mr3_host_prob *b = &L->hbatch[i];
          r->m = b->m; r->info = b->info;
          r->vl_out = b->vl_out; r->vu_out = b->vu_out;
          r->il_out = b->il_out; r->iu_out = b->iu_out;
          r->tryrac_out = b->tryrac_out;
        } else {
          mr3_cuda_prob *r = t->dreq;
          const mr3_cuda_prob *b = &L->dbatch[i];
          r->m = b->m; r->info = b->info;
          r->vl_out = b->vl_out; r->vu_out = b->vu_out;
          r->il_out = b->il_out; r->iu_out = b->iu_out;
          r->tryrac_out = b->tryrac_out;
        }
        t->t_done = t1;
        t->state = T_DONE;
      }
      s->used -= bytes;
      s->busy--;
      s->batches++;
      s->solved += k;
      pthread_cond_broadcast(&s->cv_done);
      pthread_cond_broadcast(&s->cv_work);   /* budget freed */
    }
  }
  pthread_mutex_unlock(&s->mu);
  return NULL;
}

int mr3_server_create(int device, size_t budget_bytes, mr3_server **out)
{
  mr3_server *s;
  int c, nsmall;
  if (!out) return MR3_EARG;
  *out = NULL;
  s = (mr3_server *)calloc(1, sizeof(mr3_server));
  if (!s) return MR3_EMISC;
  s->device = device;
  s->budget = budget_bytes ? budget_bytes : SRV_DEFAULT_BUDGET;
  s->nlanes = env_int("MR3_SERVE_LANES", 4);
  if (s->nlanes < 1) s->nlanes = 1;
  if (s->nlanes > SRV_MAXLANES) s->nlanes = SRV_MAXLANES;
  nsmall = env_int("MR3_SERVE_SMALL_LANES", 2);
  if (nsmall > s->nlanes - 1) nsmall = s->nlanes - 1;   /* at least one lane takes any size */
  if (nsmall < 0) nsmall = 0;
  {
    const char *w = getenv("MR3_SERVE_BATCH_WORK");
    s->work_cap = (w && *w) ? atof(w) : SRV_DEFAULT_WORK;
    if (s->work_cap < 1.0) s->work_cap = SRV_DEFAULT_WORK;
  }
  pthread_mutex_init(&s->mu, NULL);
  pthread_cond_init(&s->cv_work, NULL);
  pthread_cond_init(&s->cv_done, NULL);
  for (c = 0; c < s->nlanes; c++) {
    srv_lane *L = &s->lane[c];
    lane_arg *a;
    L->small_only = c < nsmall;
    L->hbatch = (mr3_host_prob *)malloc(SRV_MAXBATCH * sizeof(mr3_host_prob));
    L->dbatch = (mr3_cuda_prob *)malloc(SRV_MAXBATCH * sizeof(mr3_cuda_prob));
    L->ids = (long long *)malloc(SRV_MAXBATCH * sizeof(long long));
    L->view = (mr3__srv_view *)malloc(SRV_SCAN * sizeof(mr3__srv_view));
    L->vpos = (long long *)malloc(SRV_SCAN * sizeof(long long));
    L->pick = (int *)malloc(SRV_SCAN * sizeof(int));
    if (!L->hbatch || !L->dbatch || !L->ids || !L->view || !L->vpos || !L->pick) goto fail;
    if (mr3_cuda_ctx_create_prio(device, L->small_only ? 1 : 0, &L->ctx) != MR3_OK) goto fail;
    /* several lanes share the device: 2 GB of round scratch each (enough
     * warps for a 16384-row request's singletons) */
    mr3_cuda_ctx_set_round_scratch(L->ctx, (size_t)2 << 30);
    a = (lane_arg *)malloc(sizeof(lane_arg));
    if (!a) goto fail;
    a->s = s;
    a->lane = c;
    if (pthread_create(&L->th, NULL, lane_main, a) != 0) { free(a); goto fail; }
    L->started = 1;
  }
  *out = s;
  return MR3_OK;
fail:
  mr3_server_destroy(s);
  return MR3_EMISC;
}

static long long submit(mr3_server *s, int kind, void *req, int n)
{
  srv_ticket *t;
  long long id;
  size_t bytes = request_bytes(kind, req, n);
  pthread_mutex_lock(&s->mu);
  if (s->stop) { pthread_mutex_unlock(&s->mu); return -3; }
  if (bytes > s->budget) { pthread_mutex_unlock(&s->mu); return -2; }
  if (s->nt == s->cap) {
    long long ncap = s->cap ? 2 * s->cap : 4096;
    srv_ticket *nt = (srv_ticket *)realloc(s->t, (size_t)ncap * sizeof(srv_ticket));
    if (!nt) { pthread_mutex_unlock(&s->mu); return -4; }
    s->t = nt;
    s->cap = ncap;
  }
  t = &s->t[s->nt];
  memset(t, 0, sizeof(*t));
  t->kind = kind;
  t->n = n;
  t->hreq = kind == K_HOST ? (mr3_host_prob *)req : NULL;
  t->dreq = kind == K_DEVICE ? (mr3_cuda_prob *)req : NULL;
  t->bytes = bytes;
  t->work = request_work(kind, req, n);
  t->t_submit = now_ms();
  t->state = T_QUEUED;
  if (q_push(s, s->nt + 1) != 0) { pthread_mutex_unlock(&s->mu); return -4; }
  id = ++s->nt;
  pthread_cond_broadcast(&s->cv_work);
  pthread_mutex_unlock(&s->mu);
  return id;
}

long long mr3_server_submit(mr3_server *s, mr3_host_prob *req)
{
  if (!s || !req || req->n < 1 || !req->D || !req->E || !req->W) return -1;
  if ((req->jobz == 'V' || req->jobz == 'v') && (!req->Z || !req->Zsupp || req->ldz < req->n)) return -1;
  if ((req->range == 'I' || req->range == 'i') &&
      (req->il < 1 || req->iu < req->il || req->iu > req->n))
    return -1;
  return submit(s, K_HOST, req, req->n);
}

long long mr3_server_submit_device(mr3_server *s, mr3_cuda_prob *req)
{
  if (!s || !req || req->n < 1 || !req->D || !req->E || !req->W) return -1;
  if (req->jobz < MR3_JOB_N || req->jobz > MR3_JOB_C) return -1;
  if (req->range < MR3_RANGE_A || req->range > MR3_RANGE_I) return -1;
  if (req->jobz == MR3_JOB_V && (!req->Z || !req->Zsupp || req->ldz < req->n)) return -1;
  if (req->range == MR3_RANGE_I && (req->il < 1 || req->iu < req->il || req->iu > req->n))
    return -1;
  return submit(s, K_DEVICE, req, req->n);
}

int mr3_server_poll(mr3_server *s, long long ticket, int wait, double *latency_ms)
{
  srv_ticket *t;
  int done;
  if (!s) return -1;
  pthread_mutex_lock(&s->mu);
  if (ticket < 1 || ticket > s->nt) { pthread_mutex_unlock(&s->mu); return -1; }
  while (wait && s->t[ticket - 1].state != T_DONE) pthread_cond_wait(&s->cv_done, &s->mu);
  t = &s->t[ticket - 1];
  done = t->state == T_DONE;
  if (done && latency_ms) *latency_ms = t->t_done - t->t_submit;
  pthread_mutex_unlock(&s->mu);
  return done ? 1 : 0;
}

int mr3_server_timing(mr3_server *s, long long ticket, double *queued_ms, double *solve_ms)
{
  int done;
  if (!s) return -1;
  pthread_mutex_lock(&s->mu);
  if (ticket < 1 || ticket > s->nt) { pthread_mutex_unlock(&s->mu); return -1; }
  {
    const srv_ticket *t = &s->t[ticket - 1];
    done = t->state == T_DONE;
    if (done && queued_ms) *queued_ms = t->t_admit - t->t_submit;
    if (done && solve_ms) *solve_ms = t->t_done - t->t_admit;
  }
  pthread_mutex_unlock(&s->mu);
  return done ? 1 : 0;
}

int mr3_server_stats(mr3_server *s, long long *submitted, long long *solved, long long *batches)
{
  if (!s) return MR3_EARG;
  pthread_mutex_lock(&s->mu);
  if (submitted) *submitted = s->nt;
  if (solved) *solved = s->solved;
  if (batches) *batches = s->batches;
  pthread_mutex_unlock(&s->mu);
  return MR3_OK;
}

int mr3_server_stats2(mr3_server *s, long long *overlapped, int *lanes, size_t *budget_bytes)
{
  if (!s) return MR3_EARG;
  pthread_mutex_lock(&s->mu);
  if (overlapped) *overlapped = s->overlapped;
  if (lanes) *lanes = s->nlanes;
  if (budget_bytes) *budget_bytes = s->budget;
  pthread_mutex_unlock(&s->mu);
  return MR3_OK;
}

void mr3_server_destroy(mr3_server *s)
{
  int c;
  if (!s) return;
  pthread_mutex_lock(&s->mu);
  s->stop = 1;
  pthread_cond_broadcast(&s->cv_work);
  pthread_mutex_unlock(&s->mu);
  for (c = 0; c < s->nlanes; c++)
    if (s->lane[c].started) pthread_join(s->lane[c].th, NULL);
  for (c = 0; c < s->nlanes; c++) {
    srv_lane *L = &s->lane[c];
    if (L->ctx) mr3_cuda_ctx_destroy(L->ctx);
    free(L->hbatch);
    free(L->dbatch);
    free(L->ids);
    free(L->view);
    free(L->vpos);
    free(L->pick);
  }
  free(s->q);
  free(s->t);
  pthread_cond_destroy(&s->cv_work);
  pthread_cond_destroy(&s->cv_done);
  pthread_mutex_destroy(&s->mu);
  free(s);
}
