/*
 * mr3_cuda.h -- C ABI of the CUDA layer of the B200 MRRR solver.
 *
 * The host library (mrrr(), the batched and serving APIs in mr3_b200.h) calls
 * only these functions.  No CUDA or torch types cross this boundary: streams
 * are passed as void*, buffers as plain device pointers.
 *
 * This layer replaces the reference's eigenvalue stage and task runtime:
 *   mrrr_val()  SRC/mrrr_val.c:110-639      (scaling, splitting, bisection,
 *                                             root representation, refinement)
 *   mrrr_vec()  SRC/mrrr_vec.c:75-143       (representation tree and the
 *               SRC/process_cluster.c        pthread task queue; here a
 *               SRC/process_singleton.c      device work queue drained level by
 *               SRC/process_refinement.c     level)
 *   and the post-processing of mrrr() in SRC/mrrr.c:257-285.
 */
#ifndef MR3_CUDA_H
#define MR3_CUDA_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Job and range codes (first character of the reference's jobz/range). */
enum { MR3_JOB_N = 0, MR3_JOB_V = 1, MR3_JOB_C = 2 };
enum { MR3_RANGE_A = 1, MR3_RANGE_V = 2, MR3_RANGE_I = 3 };

/* Status codes, the reference's return values (INCLUDE/mrrr.h:133-137). */
enum { MR3_OK = 0, MR3_EARG = 1, MR3_EMISC = 2 };

/* One tridiagonal problem whose arrays are resident on the device.
 * Inputs mirror the arguments of mrrr() (INCLUDE/mrrr.h:62-65); D and E are
 * overwritten with the root representation as the reference does. */
typedef struct mr3_cuda_prob {
  int     n;            /* order */
  int     jobz;         /* MR3_JOB_* */
  int     range;        /* MR3_RANGE_* */
  int     il, iu;       /* 1-based index range (range I) */
  int     tryrac;       /* try high relative accuracy */
  int     ldz;          /* leading dimension of Z (>= n when jobz = V) */
  double  vl, vu;       /* value range (vl, vu] (range V) */
  double *D, *E;        /* device, n each (in/out) */
  double *W;            /* device, n: first m entries ascending */
  double *Z;            /* device, ldz*m (jobz = V), column-major */
  int    *Zsupp;        /* device, 2*m (jobz = V), 1-based supports */
  /* outputs */
  int     m, info, il_out, iu_out, tryrac_out;
  double  vl_out, vu_out;
} mr3_cuda_prob;

typedef struct mr3_cuda_ctx mr3_cuda_ctx;

/* Per-device solver context with a grow-only workspace.  One context serves
 * one host thread at a time. */
int  mr3_cuda_ctx_create(int device, mr3_cuda_ctx **out);

/* mr3_cuda_ctx_create whose streams run at the device's highest stream
 * priority when high != 0: the block scheduler starts their kernels'
 * blocks ahead of those of normal-priority streams (no preemption of
 * blocks already running).  The serving lanes for small requests use it. */
int  mr3_cuda_ctx_create_prio(int device, int high, mr3_cuda_ctx **out);

/* Bound (bytes, at least 64 MB; default 8 GB) of the checkpoint scratch of
 * the eigenvector rounds' persistent warps: fewer warps run the rounds when
 * 3 (n_max/4 + 1) 32 doubles per warp do not fit it.  Serving lanes, several
 * contexts on one device, use a smaller bound. */
int  mr3_cuda_ctx_set_round_scratch(mr3_cuda_ctx *ctx, size_t bytes);
void mr3_cuda_ctx_destroy(mr3_cuda_ctx *ctx);

/* Solve nprob problems in one batched pass on `stream` (a cudaStream_t, or
 * NULL for the context's own stream).  Returns MR3_OK when the launch
 * sequence ran; per-problem outcomes are in probs[i].info and .m.  The call
 * returns after the results (m, info, ...) have been copied to probs. */
int  mr3_cuda_solve(mr3_cuda_ctx *ctx, int nprob, mr3_cuda_prob *probs, void *stream);

/* mr3_cuda_solve with a report of finished eigenvectors: done(user, probs,
 * col0, ncols, count) is called on the calling thread, during the solve,
 * with `count` column ranges: columns col0[t] .. col0[t]+ncols[t]-1 of
 * problem probs[t] (an index into probs) are written in device memory, so
 * that their copies can start while the rest is solved.  Columns come in
 * tiles of 256, for problems with jobz V and range A or I.  Columns are
 * reported again if they were reordered afterwards (the rare order fix-up
 * of sort_eigenpairs); the last report holds. */
typedef void (*mr3_cuda_done_fn)(void *user, const int *probs, const int *col0, const int *ncols,
                                 int count);
int  mr3_cuda_solve_cb(mr3_cuda_ctx *ctx, int nprob, mr3_cuda_prob *probs, void *stream,
                       mr3_cuda_done_fn done, void *user);

/* Grow-only device buffer `slot` (0..MR3_CUDA_WS_SLOTS-1) of this context,
 * at least `bytes` long and 256-byte aligned; NULL on allocation failure.
 * Its contents do not survive a call that grows it. */
#define MR3_CUDA_WS_SLOTS 8
void *mr3_cuda_ws(mr3_cuda_ctx *ctx, int slot, size_t bytes);

/* Copies on the context's stream; dir 0 = host to device, 1 = device to host.
 * mr3_cuda_copy2d copies `height` rows of `width` bytes between pitched
 * buffers (used for column-major Z with different leading dimensions). */
int  mr3_cuda_copy(mr3_cuda_ctx *ctx, void *dst, const void *src, size_t bytes, int dir);
int  mr3_cuda_copy2d(mr3_cuda_ctx *ctx, void *dst, size_t dpitch, const void *src,
                     size_t spitch, size_t width, size_t height, int dir);
int  mr3_cuda_sync(mr3_cuda_ctx *ctx);

/* Makes the context's device current for the calling thread. */
int  mr3_cuda_set_device(mr3_cuda_ctx *ctx);

/* Second stream of the context for copies that overlap the solves, and the
 * events that order the two.  stream: MR3_STREAM_MAIN (the stream of the
 * copies above and of solves given stream NULL) or MR3_STREAM_COPY.
 * mr3_cuda_event: ev in 0..MR3_CUDA_EVENTS-1; when record_on >= 0 the event
 * is recorded on that stream, then when wait_on >= 0 that stream waits for
 * the event's last recording.  mr3_cuda_sync_all waits for both streams.
 * mr3_cuda_host_ws: grow-only page-locked host buffer of the context (NULL
 * on failure); its contents do not survive a call that grows it. */
#define MR3_STREAM_MAIN 0
#define MR3_STREAM_COPY 1
#define MR3_CUDA_EVENTS 4
int  mr3_cuda_copy_on(mr3_cuda_ctx *ctx, int stream, void *dst, const void *src, size_t bytes,
                      int dir);
int  mr3_cuda_copy2d_on(mr3_cuda_ctx *ctx, int stream, void *dst, size_t dpitch, const void *src,
                        size_t spitch, size_t width, size_t height, int dir);
int  mr3_cuda_event(mr3_cuda_ctx *ctx, int ev, int record_on, int wait_on);
int  mr3_cuda_sync_all(mr3_cuda_ctx *ctx);
void *mr3_cuda_host_ws(mr3_cuda_ctx *ctx, size_t bytes);

/* Profiling switch: with on = 1 every kernel launch is bracketed by CUDA
 * events on the solve's stream and the kernels add their work to device
 * counters; the accumulators are reset by every call of this function.
 * on = 2 also serialises the streams (the singleton rounds run on the
 * solve's stream instead of beside the next level's cluster kernels), so
 * that each kernel's time is its own, not shared with a concurrent one. */
void mr3_cuda_profile(mr3_cuda_ctx *ctx, int on);

/* Accumulated profile: up to `max` kernels (names as 32-byte strings, total
 * milliseconds, launch counts) and 24 work counters: counters[4*k + kind] for
 * kernel group k (bisection, root refinement, child representation, cluster
 * refinement, singletons, other) and kind (0 Sturm steps on T, 1 Sturm steps
 * on L D L^T, 2 twisted-factorisation rows, 3 dlarrf rows). */
int  mr3_cuda_profile_read(mr3_cuda_ctx *ctx, int max, char *names, double *ms,
                           long long *launches, unsigned long long *counters);

/* Measures FP64 fused multiply-add throughput (TFLOP/s, 2 flops per FMA)
 * and IEEE double division throughput (G divisions/s) on `device` with short
 * kernels of many independent chains: the roofline denominators of the
 * division-bound Sturm-count kernels. */
int  mr3_cuda_fp64_peaks(int device, double *fma_tflops, double *div_gops);

/* Eigenvectors of an L D L^T representation without any allocation.
 * No counterpart in the reference.  For callers that cannot call cudaMalloc:
 * code inside a device-memory budget owned by another allocator, or
 * latency-critical loops that cannot afford cudaMalloc's implicit device
 * synchronisation.  One twisted factorisation (dlar1v, twist index searched
 * over 1..n) per eigenvalue lambda[j] of L D L^T; column j of Z gets the unit
 * eigenvector, zero outside its support, Zsupp[2j..2j+1] the 1-based support.
 * D (n), L (n-1), lambda (m), Z (ldz*m), Zsupp (2m) are device pointers;
 * gaptol is dlar1v's support-truncation tolerance (0 keeps every entry).
 * The pivot threshold is derived from the representation as the solver
 * derives it from T: DBL_MIN * max(1, max_i (D(i) L(i))^2).  n = 1 gives
 * unit vectors.  Scratch is one static device array of the library (16.8 MB per GPU), so
 * n <= MR3_NOALLOC_NMAX; larger n, m < 0 or ldz < n return 1.  The first call
 * on a device looks the array up (cudaGetSymbolAddress); make that first call
 * before any stream capture.  All calls share the array: calls that overlap
 * on the GPU race.  Returns 0 when the kernels were queued on `stream`. */
#define MR3_NOALLOC_NMAX 2048
int  mr3_cuda_eigvec_noalloc(int n, const double *D, const double *L, int m,
                             const double *lambda, double gaptol, double *Z, int ldz,
                             int *Zsupp, void *stream);

/* Number of kernels launched by the last mr3_cuda_solve on this context. */
long long mr3_cuda_last_launches(const mr3_cuda_ctx *ctx);

/* Last CUDA error text of this context (empty if none). */
const char *mr3_cuda_last_error(const mr3_cuda_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif
