/*
 * ilobpcg_shim.c -- the external "LOBPCG" library that pstuermer/BDG_LOBPCG
 * links (src/solver.c:2, Makefile:13-14, 32-33; not vendored, no version
 * pinned), restated for the oracle build: linop wrappers and d_/z_ilobpcg.
 *
 * TEST INFRASTRUCTURE ONLY.  The iteration (ilobpcg_impl.inc) follows
 * oracle/bdg_oracle.py:ilobpcg step for step: Kressner, Miloloza Pandur &
 * Shao, "An indefinite variant of LOBPCG for definite matrix pencils",
 * Numer. Algorithms 66 (2014), in block form with soft locking and SVQB
 * (Stathopoulos & Wu 2002).  BLAS/LAPACK come from the OpenBLAS build that
 * scipy ships (its symbols carry a scipy_ prefix).
 *
 * Options the reference's ABI has no field for (convergence criterion,
 * Goldstone deflation, guard levels) are set with ilobpcg_shim_set; a
 * per-iteration timeline (wall clock, Ritz values, convergence measures) is
 * kept for the timed CPU baseline and read with ilobpcg_shim_timeline.
 */
#define _GNU_SOURCE
#include "lobpcg.h"

#include <complex.h>
#include <math.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ---- BLAS / LAPACK (Fortran ABI, 32-bit integers) ------------------------ */
void scipy_dgemm_(const char *ta, const char *tb, const int *m, const int *n, const int *k, const double *alpha,
                  const double *a, const int *lda, const double *b, const int *ldb, const double *beta, double *c,
                  const int *ldc, size_t, size_t);
void scipy_zgemm_(const char *ta, const char *tb, const int *m, const int *n, const int *k, const c64 *alpha,
                  const c64 *a, const int *lda, const c64 *b, const int *ldb, const c64 *beta, c64 *c,
                  const int *ldc, size_t, size_t);
void scipy_dsyevd_(const char *jobz, const char *uplo, const int *n, double *a, const int *lda, double *w,
                   double *work, const int *lwork, int *iwork, const int *liwork, int *info, size_t, size_t);
void scipy_zheevd_(const char *jobz, const char *uplo, const int *n, c64 *a, const int *lda, double *w, c64 *work,
                   const int *lwork, double *rwork, const int *lrwork, int *iwork, const int *liwork, int *info,
                   size_t, size_t);
void scipy_openblas_set_num_threads(int);

/* ---- reference operators and context helpers (ref_helpers.c) -------------- */
void matmulK_d(void *ctx, const f64 *x, f64 *y);
void matmulM_d(void *ctx, const f64 *x, f64 *y);
void matmulK_z(void *ctx, const c64 *x, c64 *y);
void matmulM_z(void *ctx, const c64 *x, c64 *y);
const void *ref_helper_wf(void *ctx);
double ref_helper_anorm(void *ctx);

/* ---- options ------------------------------------------------------------- */
typedef struct {
  int criterion; /* 0: backward error, 1: true residual ||K M v - lam^2 v|| / ||v|| */
  int lock;
  int deflate;
  int stall_win;
  double drop, guard, guard_strict, true_gate;
  int norm_p; /* SVQB-normalise the projected P (off: as the GPU solver) */
} shim_opts_t;

static shim_opts_t g_opt = {0, 1, 0, 10, 1e-13, 1e-4, 1e-12, 1e-7, 0};

/* Capture mode: the next solve copies the initial block that the caller's
 * init switch wrote into alg->S (src/solver.c:167-259) to this buffer and
 * returns without iterating (converged = 0, iterations = 0). */
static void *g_capture;

void ilobpcg_shim_capture_init(void *dst) { g_capture = dst; }

void ilobpcg_shim_set(int criterion, int deflate, int lock, double guard, double guard_strict, int stall_win,
                      double true_gate) {
  g_opt.criterion = criterion;
  g_opt.deflate = deflate;
  g_opt.lock = lock;
  g_opt.guard = guard;
  g_opt.guard_strict = guard_strict;
  g_opt.stall_win = stall_win > 0 && stall_win < 64 ? stall_win : 10;
  g_opt.true_gate = true_gate;
}

void ilobpcg_shim_set_pnorm(int on) { g_opt.norm_p = on != 0; }

void ilobpcg_shim_threads(int nthreads) {
  scipy_openblas_set_num_threads(nthreads);
  omp_set_num_threads(nthreads);
}

/* ---- timeline -------------------------------------------------------------- *
 * t[0]: entry; t[1]: loop start (after the Rayleigh-Ritz of span X0);
 * t[2 + i]: end of iteration i.  Ritz values and measures of the wanted
 * pairs per iteration (first TL_NEV). */
#define TL_CAP 4096
#define TL_NEV 64
static double g_t[TL_CAP + 2];
static int g_nt;
static double g_lam[TL_CAP][TL_NEV], g_res[TL_CAP][TL_NEV];
static int g_nrec, g_iters, g_nconv;

static void shim_tl_reset(void) {
  g_nt = 0;
  g_nrec = 0;
  g_iters = 0;
  g_nconv = 0;
  g_t[g_nt++] = omp_get_wtime();
}

static void shim_tl_mark(void) {
  if (g_nt < TL_CAP + 2) g_t[g_nt++] = omp_get_wtime();
}

static void shim_tl_record(uint64_t it, const double *lam, const double *res, int nev) {
  if (it >= TL_CAP) return;
  for (int j = 0; j < nev && j < TL_NEV; j++) {
    g_lam[it][j] = lam[j];
    g_res[it][j] = res[j];
  }
  g_nrec = (int)it + 1;
}

static void shim_tl_finish(uint64_t iters, int nconv) {
  g_iters = (int)iters;
  g_nconv = nconv;
}

/* Copies the timestamps (up to cap) and returns how many there are; iters
 * and nconv of the last solve through the pointers. */
int ilobpcg_shim_timeline(double *t, int cap, int *iters, int *nconv) {
  const int c = g_nt < cap ? g_nt : cap;
  memcpy(t, g_t, (size_t)c * sizeof(double));
  if (iters) *iters = g_iters;
  if (nconv) *nconv = g_nconv;
  return g_nt;
}

/* Ritz values and convergence measures of the first nev wanted pairs at
 * iteration it (0 .. records-1); returns the count of records. */
int ilobpcg_shim_history(int it, int nev, double *lam, double *res) {
  if (it >= 0 && it < g_nrec)
    for (int j = 0; j < nev && j < TL_NEV; j++) {
      lam[j] = g_lam[it][j];
      res[j] = g_res[it][j];
    }
  return g_nrec;
}

/* ---- linops ---------------------------------------------------------------- */
LinearOperator_d_t *linop_create_d(uint64_t rows, uint64_t cols, linop_matvec_d_fn matvec, linop_cleanup_fn cleanup,
                                   linop_ctx_t *ctx) {
  LinearOperator_d_t *op = (LinearOperator_d_t *)calloc(1, sizeof *op);
  op->rows = rows;
  op->cols = cols;
  op->matvec = matvec;
  op->cleanup = cleanup;
  op->ctx = ctx;
  return op;
}

LinearOperator_z_t *linop_create_z(uint64_t rows, uint64_t cols, linop_matvec_z_fn matvec, linop_cleanup_fn cleanup,
                                   linop_ctx_t *ctx) {
  LinearOperator_z_t *op = (LinearOperator_z_t *)calloc(1, sizeof *op);
  op->rows = rows;
  op->cols = cols;
  op->matvec = matvec;
  op->cleanup = cleanup;
  op->ctx = ctx;
  return op;
}

void linop_destroy_d(LinearOperator_d_t **op) {
  if (!op || !*op) return;
  if ((*op)->cleanup) (*op)->cleanup((*op)->ctx);
  free(*op);
  *op = NULL;
}

void linop_destroy_z(LinearOperator_z_t **op) {
  if (!op || !*op) return;
  if ((*op)->cleanup) (*op)->cleanup((*op)->ctx);
  free(*op);
  *op = NULL;
}

/* ---- the two instantiations -------------------------------------------------- */
#define SC f64
#define FN(x) d_##x
#define CJ(x) (x)
#define RE(x) (x)
#define OPC 'T'
#define GEMM_F scipy_dgemm_
#define HEEV_F scipy_dsyevd_
#define MATMUL_K(c, x, y) matmulK_d((c), (x), (y))
#define MATMUL_M(c, x, y) matmulM_d((c), (x), (y))
#define ALG_T d_lobpcg_t
#define LINOP_T LinearOperator_d_t
#include "ilobpcg_impl.inc"
#undef SC
#undef FN
#undef CJ
#undef RE
#undef OPC
#undef GEMM_F
#undef HEEV_F
#undef MATMUL_K
#undef MATMUL_M
#undef ALG_T
#undef LINOP_T

#define SHIM_COMPLEX 1
#define SC c64
#define FN(x) z_##x
#define CJ(x) conj(x)
#define RE(x) creal(x)
#define OPC 'C'
#define GEMM_F scipy_zgemm_
#define HEEV_F scipy_zheevd_
#define MATMUL_K(c, x, y) matmulK_z((c), (x), (y))
#define MATMUL_M(c, x, y) matmulM_z((c), (x), (y))
#define ALG_T z_lobpcg_t
#define LINOP_T LinearOperator_z_t
#include "ilobpcg_impl.inc"
