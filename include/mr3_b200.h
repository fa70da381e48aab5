/*
 * mr3_b200.h -- public C ABI of the B200 MRRR tridiagonal eigensolver.
 *
 * Drop-in replacement for the entry points of MR3-SMP: the tridiagonal
 * solver mrrr() and the dense drivers of SRC/dense.c built on it.  All
 * arguments keep the reference's meaning; host pointers throughout.
 */
#ifndef MR3_B200_H
#define MR3_B200_H

#include "mr3_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces int mrrr(...) of INCLUDE/mrrr.h:62-65 (implementation
 * SRC/mrrr.c:87-296); same argument contract (INCLUDE/mrrr.h:67-149):
 *   jobz  "N" eigenvalues, "V" eigenpairs, "C" count only (first char, any case)
 *   range "A" all, "V" (vl,vu], "I" il..iu (1-based)
 *   D, E  n doubles each (E[n-1] arbitrary); overwritten with the root
 *         representation L D L^T of each block and its shift, as the
 *         reference does
 *   vl, vu, il, iu  refined on output; tryrac reset to 0 if relative
 *         accuracy cannot be guaranteed
 *   m     number of eigenpairs; W[0..m-1] ascending
 *   Z     column j at Z[j*ldz], rows 0..n-1 written; Zsupp[2j], Zsupp[2j+1]
 *         its 1-based support
 * Returns 0 on success, 1 for a bad argument, 2 on an internal failure. */
int mrrr(char *jobz, char *range, int *n, double *D, double *E, double *vl,
         double *vu, int *il, int *iu, int *tryrac, int *m, double *W,
         double *Z, int *ldz, int *Zsupp);

/* Replaces the Fortran binding mrrr_ of SRC/mrrr.c:630-637. */
void mrrr_(char *jobz, char *range, int *n, double *D, double *E, double *vl,
           double *vu, int *il, int *iu, int *tryrac, int *m, double *W,
           double *Z, int *ldz, int *Zsupp, int *info);

/* One problem of a batched call with host arrays (no counterpart in the
 * reference, which has no batch API; each entry means what the arguments of
 * mrrr() mean). */
typedef struct mr3_host_prob {
  char    jobz, range;
  int     n, il, iu, tryrac, ldz;
  double  vl, vu;
  double *D, *E;       /* in/out, n each */
  double *W;           /* out, n */
  double *Z;           /* out, ldz*m (jobz 'V') */
  int    *Zsupp;       /* out, 2*m  (jobz 'V') */
  int     m, info;     /* out */
  double  vl_out, vu_out;
  int     il_out, iu_out, tryrac_out;
} mr3_host_prob;

/* Solves all problems in one batched device pass (arrays in host memory).
 * Returns 0 if every problem succeeded, else the largest info. */
int mr3_batched(int nprob, mr3_host_prob *probs);

/* Same with arrays already resident in device memory on `stream`
 * (a cudaStream_t or NULL). */
int mr3_batched_device(int nprob, mr3_cuda_prob *probs, void *stream);

/* Serving (no counterpart in the reference, which answers one call at a
 * time; SRC/mrrr.c:87-296 is the per-request computation).  A server takes
 * a stream of independent requests and solves them with continuous
 * batching: several lanes (worker threads, each with its own solver
 * context and streams) admit queued requests in arrival order whenever
 * they free up, as long as the device bytes of all requests in flight
 * (eigenvectors plus per-row work arrays) stay within the budget
 * (budget_bytes; 0 = 120 GB) and the batch stays under a work cap; batches
 * of different lanes run on the device at the same time, and lanes
 * reserved for small requests (n <= 2048) run at high stream priority.
 * Results are those of a call alone.  Environment (read at create):
 * MR3_SERVE_LANES (default 4), MR3_SERVE_SMALL_LANES (default 2),
 * MR3_SERVE_BATCH_WORK (work cap in eigenvector entries, default 2^27).
 *
 * mr3_server_submit: a host request (an mr3_host_prob as for mr3_batched);
 * eigenvectors are copied back to its host arrays.
 * mr3_server_submit_device: a device request (an mr3_cuda_prob as for
 * mr3_batched_device): D, E, W, Z, Zsupp stay resident in device memory and
 * nothing crosses PCIe.
 * The request struct and its arrays must stay valid and untouched until
 * poll reports it done.  Both return a ticket >= 1, or -1 bad arguments,
 * -2 request larger than the budget, -3 server stopping, -4 out of host
 * memory.
 * mr3_server_poll: 1 done (the request's info, m, ... are set), 0 pending,
 * -1 unknown ticket; wait = 1 blocks until done; latency_ms (or NULL)
 * receives the submit-to-done time.
 * mr3_server_timing: of a done request, the time it waited for admission
 * and the time from admission to done (1 done, 0 pending, -1 unknown).
 * mr3_server_stats2: batches admitted while another lane's batch was on
 * the device, the number of lanes and the budget.
 * mr3_server_destroy finishes every queued request, then stops. */
typedef struct mr3_server mr3_server;
int  mr3_server_create(int device, size_t budget_bytes, mr3_server **out);
long long mr3_server_submit(mr3_server *s, mr3_host_prob *req);
long long mr3_server_submit_device(mr3_server *s, mr3_cuda_prob *req);
int  mr3_server_poll(mr3_server *s, long long ticket, int wait, double *latency_ms);
int  mr3_server_timing(mr3_server *s, long long ticket, double *queued_ms, double *solve_ms);
int  mr3_server_stats(mr3_server *s, long long *submitted, long long *solved, long long *batches);
int  mr3_server_stats2(mr3_server *s, long long *overlapped, int *lanes, size_t *budget_bytes);
void mr3_server_destroy(mr3_server *s);

/* Replaces int dsyeig(...) of INCLUDE/mrrr.h:270-272 (implementation
 * SRC/dense.c:151-232): all or some eigenpairs of the dense symmetric n x n
 * matrix A (column-major, leading dimension lda; uplo "L" or "U" selects the
 * stored triangle).  jobz, range, vl, vu, il, iu, m, W and Z (leading
 * dimension ldz) mean what they mean for mrrr(); A is scaled, reduced to
 * tridiagonal form, solved and back-transformed on the device (A on the host
 * is left unchanged; the reference's contract allows it to be overwritten).
 * Returns 0, 1 for a bad argument (also lda < n, or ldz < n with jobz "V"),
 * 2 on an internal failure (also when the device's LAPACK library, cuSOLVER,
 * cannot be loaded). */
int dsyeig(char *jobz, char *range, char *uplo, int *n, double *A, int *lda,
           double *vl, double *vu, int *il, int *iu, int *m, double *W,
           double *Z, int *ldz);

/* Replaces the Fortran binding dsyeig_ of SRC/dense.c:1037-1043. */
void dsyeig_(char *jobz, char *range, char *uplo, int *n, double *A, int *lda,
             double *vl, double *vu, int *il, int *iu, int *m, double *W,
             double *Z, int *ldz, int *info);

/* Replaces int dspeig(...) of INCLUDE/mrrr.h:444-446 (implementation
 * SRC/dense.c:319-398): dsyeig with A in LAPACK packed storage AP
 * (n(n+1)/2 doubles, the uplo triangle column by column); AP on the host is
 * left unchanged.  Same returns as dsyeig. */
int dspeig(char *jobz, char *range, char *uplo, int *n, double *AP,
           double *vl, double *vu, int *il, int *iu, int *m, double *W,
           double *Z, int *ldz);
void dspeig_(char *jobz, char *range, char *uplo, int *n, double *AP,
             double *vl, double *vu, int *il, int *iu, int *m, double *W,
             double *Z, int *ldz, int *info);   /* SRC/dense.c:1056-1062 */

/* Replaces int dsygeig(...) of INCLUDE/mrrr.h:352-354 (implementation
 * SRC/dense.c:236-313): the generalized symmetric-definite problem,
 * itype 1 A x = lambda B x, 2 A B x = lambda x, 3 B A x = lambda x, B
 * positive definite (leading dimension ldb).  On return B holds its
 * Cholesky factor (uplo triangle) and, for jobz "V", the first m columns of
 * A the eigenvectors, as in the reference.  n <= 1 is a bad argument there
 * and here.  Returns 2 also when B is not positive definite. */
int dsygeig(int *itype, char *jobz, char *range, char *uplo, int *n,
            double *A, int *lda, double *B, int *ldb, double *vl,
            double *vu, int *il, int *iu, int *m, double *W);
void dsygeig_(int *itype, char *jobz, char *range, char *uplo, int *n,
              double *A, int *lda, double *B, int *ldb, double *vl,
              double *vu, int *il, int *iu, int *m, double *W,
              int *info);   /* SRC/dense.c:1046-1053 */

/* Replaces int dspgeig(...) of INCLUDE/mrrr.h:526-529 (implementation
 * SRC/dense.c:403-470): dsygeig with A and B in packed storage; the
 * eigenvectors go to Z (leading dimension ldz) and BP returns the packed
 * Cholesky factor. */
int dspgeig(int *itype, char *jobz, char *range, char *uplo, int *n,
            double *AP, double *BP, double *vl, double *vu, int *il,
            int *iu, int *m, double *W, double *Z, int *ldz);
void dspgeig_(int *itype, char *jobz, char *range, char *uplo, int *n,
              double *AP, double *BP, double *vl, double *vu, int *il,
              int *iu, int *m, double *W, double *Z, int *ldz,
              int *info);   /* SRC/dense.c:1065-1072 */

/* The complex Hermitian drivers, which the reference compiles only with its
 * COMPLEX_SUPPORTED switch.  Complex arrays (A, B, AP, BP, Z) are
 * column-major with interleaved (re, im) doubles -- the layout of C99
 * double complex -- and are passed as void * so that C and C++ callers
 * can hand in double complex or std::complex<double> arrays alike; W, vl
 * and vu are real.  Arguments, outputs and returns are those of the real
 * drivers above, with conjugate transposes in place of transposes:
 *   zheeig  replaces INCLUDE/mrrr.h:538-541 (SRC/dense.c:568-671);
 *   zhegeig replaces INCLUDE/mrrr.h:624-627 (SRC/dense.c:676-754);
 *   zhpeig  replaces INCLUDE/mrrr.h:718-721 (SRC/dense.c:760-862);
 *   zhpgeig replaces INCLUDE/mrrr.h:802-805 (SRC/dense.c:869-936);
 * and the _ bindings replace SRC/dense.c:1076-1113.  zhegeig and zhpgeig
 * refuse n <= 1, as the reference does. */
int zheeig(char *jobz, char *range, char *uplo, int *n, void *A, int *lda,
           double *vl, double *vu, int *il, int *iu, int *m, double *W,
           void *Z, int *ldz);
int zhegeig(int *itype, char *jobz, char *range, char *uplo, int *n,
            void *A, int *lda, void *B, int *ldb, double *vl, double *vu,
            int *il, int *iu, int *m, double *W);
int zhpeig(char *jobz, char *range, char *uplo, int *n, void *AP,
           double *vl, double *vu, int *il, int *iu, int *m, double *W,
           void *Z, int *ldz);
int zhpgeig(int *itype, char *jobz, char *range, char *uplo, int *n,
            void *AP, void *BP, double *vl, double *vu, int *il, int *iu,
            int *m, double *W, void *Z, int *ldz);
void zheeig_(char *jobz, char *range, char *uplo, int *n, void *A, int *lda,
             double *vl, double *vu, int *il, int *iu, int *m, double *W,
             void *Z, int *ldz, int *info);
void zhegeig_(int *itype, char *jobz, char *range, char *uplo, int *n,
              void *A, int *lda, void *B, int *ldb, double *vl, double *vu,
              int *il, int *iu, int *m, double *W, int *info);
void zhpeig_(char *jobz, char *range, char *uplo, int *n, void *AP,
             double *vl, double *vu, int *il, int *iu, int *m, double *W,
             void *Z, int *ldz, int *info);
void zhpgeig_(int *itype, char *jobz, char *range, char *uplo, int *n,
              void *AP, void *BP, double *vl, double *vu, int *il, int *iu,
              int *m, double *W, void *Z, int *ldz, int *info);

/* Kernels launched by the calling thread's last solve (diagnostics). */
long long mr3_last_launches(void);

/* Text of the last CUDA error seen by the calling thread's last solve. */
const char *mr3_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
