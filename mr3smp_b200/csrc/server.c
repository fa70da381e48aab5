/*
 * server.c -- serving front end: many independent requests, solved in
 * batches as they arrive (continuous batching).
 *
 * The reference answers one call at a time (mrrr, SRC/mrrr.c:87-296).  A
 * serving process instead receives a stream of requests (tridiagonal
 * problems of mixed sizes) and wants each answered soon after it arrives.
 * The server keeps one queue per size class and one worker thread per
 * class; a worker owns a solver context and, whenever it is idle, takes the
 * oldest queued requests of its class that fit the class's share of the
 * device-memory budget and solves them in one batched pass (the path of
 * mr3_batched).  Requests that arrive meanwhile wait for the next pass.
 * Small requests get their own class so that a large problem in flight
 * does not hold them back.
 *
 * A request is an mr3_host_prob with the meaning it has for mr3_batched;
 * its arrays must stay valid and untouched until poll reports it done.
 * Every request is solved exactly as it would be alone: batching never
 * changes a result (each problem's computation is independent of the
 * others in the batch).
 */
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "mr3_b200.h"

__attribute__((visibility("hidden"))) int mr3__batched_on(mr3_cuda_ctx *ctx, int nprob,
                                                       mr3_host_prob *hp);   /* mrrr.c */

#define SRV_CLASSES 2
#define SRV_MAXBATCH 4096
#define SRV_SMALL_N 2048          /* n <= this: class 0 */
#define SRV_SMALL_SHARE 8         /* class 0 budget: budget / 8, at most 16 GB */
#define SRV_DEFAULT_BUDGET ((size_t)120 << 30)

enum { T_QUEUED = 1, T_RUNNING = 2, T_DONE = 3 };

typedef struct {
  mr3_host_prob *req;
  size_t bytes;
  double t_submit, t_done;
  int state, cls;
} srv_ticket;

typedef struct {
  long long *ids;
  long long head, tail, cap;
} srv_queue;

struct mr3_server {
  int device;
  pthread_mutex_t mu;
  pthread_cond_t cv_work, cv_done;
  srv_ticket *t;          /* ticket k at t[k - 1] */
  long long nt, cap;
  srv_queue q[SRV_CLASSES];
  size_t budget[SRV_CLASSES];
  mr3_cuda_ctx *ctx[SRV_CLASSES];
  pthread_t th[SRV_CLASSES];
  mr3_host_prob *batch[SRV_CLASSES];   /* a worker's batch (copies of the requests) */
  long long *ids[SRV_CLASSES];         /* and their tickets */
  int started[SRV_CLASSES];
  int stop;
  long long batches, solved;
};

static double now_ms(void)
{
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec * 1e3 + ts.tv_nsec * 1e-6;
}

/* Device bytes a request holds while its batch runs: its eigenvectors and
 * the per-row work arrays of the solver (about 70 doubles per row). */
static size_t request_bytes(const mr3_host_prob *h)
{
  size_t n = (size_t)h->n, cols = 0;
  if (h->jobz == 'V' || h->jobz == 'v') {
    if (h->range == 'I' || h->range == 'i') cols = (size_t)(h->iu - h->il + 1);
    else cols = n;
  }
  return 8 * n * cols + 560 * n;
}

static int q_push(srv_queue *q, long long id)
{
  if (q->tail == q->cap) {
    long long live = q->tail - q->head, ncap;
    long long *nv;
    if (q->head > 0 && live < q->cap / 2) {
      memmove(q->ids, q->ids + q->head, (size_t)live * sizeof(long long));
      q->tail = live;
      q->head = 0;
    } else {
      ncap = q->cap ? 2 * q->cap : 1024;
      nv = (long long *)realloc(q->ids, (size_t)ncap * sizeof(long long));
      if (!nv) return -1;
      q->ids = nv;
      q->cap = ncap;
    }
  }
  q->ids[q->tail++] = id;
  return 0;
}

typedef struct {
  mr3_server *s;
  int cls;
} worker_arg;

static void *worker(void *p)
{
  worker_arg *a = (worker_arg *)p;
  mr3_server *s = a->s;
  const int c = a->cls;
  long long *ids = s->ids[c];
  mr3_host_prob *batch = s->batch[c];
  free(a);
  pthread_mutex_lock(&s->mu);
  for (;;) {
    srv_queue *q = &s->q[c];
    int k = 0, i;
    size_t used = 0;
    while (!s->stop && q->head == q->tail) pthread_cond_wait(&s->cv_work, &s->mu);
    if (q->head == q->tail) break;   /* stopping and nothing left */
    /* the oldest requests of the class that fit the budget (at least one) */
    while (q->head < q->tail && k < SRV_MAXBATCH) {
      srv_ticket *t = &s->t[q->ids[q->head] - 1];
      if (k > 0 && used + t->bytes > s->budget[c]) break;
      used += t->bytes;
      t->state = T_RUNNING;
      ids[k] = q->ids[q->head];
      batch[k] = *t->req;
      k++;
      q->head++;
    }
    pthread_mutex_unlock(&s->mu);
    if (k > 0) mr3_cuda_set_device(s->ctx[c]);
    if (k > 0) mr3__batched_on(s->ctx[c], k, batch);
    pthread_mutex_lock(&s->mu);
    {
      const double t1 = now_ms();
      for (i = 0; i < k; i++) {
        srv_ticket *t = &s->t[ids[i] - 1];
        mr3_host_prob *r = t->req;
        r->m = batch[i].m;
        r->info = batch[i].info;
        r->vl_out = batch[i].vl_out;
        r->vu_out = batch[i].vu_out;
        r->il_out = batch[i].il_out;
        r->iu_out = batch[i].iu_out;
        r->tryrac_out = batch[i].tryrac_out;
        t->t_done = t1;
        t->state = T_DONE;
      }
      if (k > 0) { s->batches++; s->solved += k; }
      pthread_cond_broadcast(&s->cv_done);
    }
  }
  pthread_mutex_unlock(&s->mu);
  return NULL;
}

int mr3_server_create(int device, size_t budget_bytes, mr3_server **out)
{
  mr3_server *s;
  int c;
  if (!out) return MR3_EARG;
  *out = NULL;
  s = (mr3_server *)calloc(1, sizeof(mr3_server));
  if (!s) return MR3_EMISC;
  s->device = device;
  if (budget_bytes == 0) budget_bytes = SRV_DEFAULT_BUDGET;
  s->budget[0] = budget_bytes / SRV_SMALL_SHARE;
  if (s->budget[0] > ((size_t)16 << 30)) s->budget[0] = (size_t)16 << 30;
  s->budget[1] = budget_bytes - s->budget[0];
  pthread_mutex_init(&s->mu, NULL);
  pthread_cond_init(&s->cv_work, NULL);
  pthread_cond_init(&s->cv_done, NULL);
  for (c = 0; c < SRV_CLASSES; c++) {
    worker_arg *a;
    s->batch[c] = (mr3_host_prob *)malloc(SRV_MAXBATCH * sizeof(mr3_host_prob));
    s->ids[c] = (long long *)malloc(SRV_MAXBATCH * sizeof(long long));
    if (!s->batch[c] || !s->ids[c]) goto fail;
    if (mr3_cuda_ctx_create(device, &s->ctx[c]) != MR3_OK) goto fail;
    a = (worker_arg *)malloc(sizeof(worker_arg));
    if (!a) goto fail;
    a->s = s;
    a->cls = c;
    if (pthread_create(&s->th[c], NULL, worker, a) != 0) { free(a); goto fail; }
    s->started[c] = 1;
  }
  *out = s;
  return MR3_OK;
fail:
  mr3_server_destroy(s);
  return MR3_EMISC;
}

long long mr3_server_submit(mr3_server *s, mr3_host_prob *req)
{
  srv_ticket *t;
  long long id;
  int c;
  if (!s || !req || req->n < 1 || !req->D || !req->E || !req->W) return -1;
  if ((req->jobz == 'V' || req->jobz == 'v') && (!req->Z || !req->Zsupp || req->ldz < req->n)) return -1;
  if ((req->range == 'I' || req->range == 'i') &&
      (req->il < 1 || req->iu < req->il || req->iu > req->n))
    return -1;
  c = req->n <= SRV_SMALL_N ? 0 : 1;
  pthread_mutex_lock(&s->mu);
  if (s->stop) { pthread_mutex_unlock(&s->mu); return -3; }
  if (request_bytes(req) > s->budget[c]) { pthread_mutex_unlock(&s->mu); return -2; }
  if (s->nt == s->cap) {
    long long ncap = s->cap ? 2 * s->cap : 4096;
    srv_ticket *nt = (srv_ticket *)realloc(s->t, (size_t)ncap * sizeof(srv_ticket));
    if (!nt) { pthread_mutex_unlock(&s->mu); return -4; }
    s->t = nt;
    s->cap = ncap;
  }
  t = &s->t[s->nt];
  t->req = req;
  t->bytes = request_bytes(req);
  t->t_submit = now_ms();
  t->t_done = 0.0;
  t->state = T_QUEUED;
  t->cls = c;
  if (q_push(&s->q[c], s->nt + 1) != 0) { pthread_mutex_unlock(&s->mu); return -4; }
  id = ++s->nt;
  pthread_cond_broadcast(&s->cv_work);
  pthread_mutex_unlock(&s->mu);
  return id;
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

void mr3_server_destroy(mr3_server *s)
{
  int c;
  if (!s) return;
  pthread_mutex_lock(&s->mu);
  s->stop = 1;
  pthread_cond_broadcast(&s->cv_work);
  pthread_mutex_unlock(&s->mu);
  for (c = 0; c < SRV_CLASSES; c++)
    if (s->started[c]) pthread_join(s->th[c], NULL);
  for (c = 0; c < SRV_CLASSES; c++)
    if (s->ctx[c]) mr3_cuda_ctx_destroy(s->ctx[c]);
  for (c = 0; c < SRV_CLASSES; c++) {
    free(s->q[c].ids);
    free(s->batch[c]);
    free(s->ids[c]);
  }
  free(s->t);
  pthread_cond_destroy(&s->cv_work);
  pthread_cond_destroy(&s->cv_done);
  pthread_mutex_destroy(&s->mu);
  free(s);
}
