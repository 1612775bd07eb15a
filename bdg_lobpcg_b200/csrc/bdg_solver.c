/*
 * bdg_solver.c -- the iLOBPCG iteration on the GPU, driven from host C.
 *
 * Replaces the reference's solver adapter + external eigensolver
 * (pstuermer/BDG_LOBPCG src/solver.c:134-441 calling d_ilobpcg/z_ilobpcg of
 * an unvendored "LOBPCG" library).  The iteration is restated from the
 * published method (Kressner, Miloloza Pandur & Shao, "An indefinite variant
 * of LOBPCG for definite matrix pencils", Numer. Algorithms 66, 2014) in
 * block form for the pencil (A, B) = (diag(K, M), swap):
 *
 *   X0 (B-positive) -> AX = A X -> Rayleigh-Ritz on span X
 *   repeat:  R = AX - B X diag(lam)          (swap folded into the kernel)
 *            test the nev wanted pairs       (backward error or ||KMv - w^2 v||)
 *            W = T R,  AW = A W              (batched FFT operator kernels)
 *            Gram blocks of S = [X W P]      (FP64 tensor-core contraction)
 *            Rayleigh-Ritz on the projected definite pencil:
 *              S^H S = Guu + Gvv -> implicit orthonormalisation (small
 *              directions dropped), A_s = Q D Q^H (D clamped so a Goldstone
 *              null direction stays finite), H = D^-1/2 Q^H B_s Q D^-1/2,
 *              theta = eig(H), lam = 1/theta, the m largest positive theta
 *            X <- S C,  P <- [W P] C_wp  (and AX, AP alike, no extra apply)
 *
 * Everything block-sized stays in HBM for the whole solve; the host sees
 * only the k x k eigenvalue counts and the convergence norms each iteration.
 * Block updates are plain GEMMs (cuBLAS); the k x k eigenproblems use
 * cuSOLVER syevd/heevd.
 */
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>
#include <math.h>
#include <string.h>
#include <time.h>

#include "bdg/bdg_cuda.h"
#include "bdg/bdg_internal.h"
#include "bdg_blas.h"

#define RR_DROP_F64 1e-13
#define RR_DROP_F32 1e-6
#define RR_CLAMP 1e-14

typedef struct {
  uint64_t S, n, m, nev, kmax;
  int cplx;
  int prec;      /* BDGD_F64 / BDGD_F32 storage of the current blocks */
  size_t esz;    /* bytes per block element */
  void *S0, *S1, *AS0, *AS1, *R, *TR, *X64; /* TR: S x nev; X64: FP64 copy for refinement */
  double *lam, *work, *norms, *gram, *Gs, *Gb, *Ga, *dsc, *Z, *T1, *T2, *Ga2, *Gb2, *Y, *H, *V, *C64, *wG, *wA, *wH;
  float *C32;
  double *defl; /* deflation vectors psi0 and w (FP64, [2][n_half*es]) */
  cublasHandle_t blas;
  cusolverDnHandle_t sol;
  void *swork;
  int lwork;
  int *info;
  size_t bytes_blocks;
  uint64_t cap_S, cap_m, cap_nev;
  int cap_cplx, cap_prec;
  cudaEvent_t ev[16];
} ws_t;

static void ws_free(ws_t *w) {
  if (!w) return;
  void *bufs[] = {w->S0, w->S1, w->AS0, w->AS1, w->R, w->TR, w->X64, w->lam, w->work, w->norms, w->gram, w->Gs,
                  w->Gb, w->Ga, w->dsc, w->Z,   w->T1, w->T2, w->Ga2, w->Gb2, w->Y, w->H, w->V, w->C64, w->wG,
                  w->wA, w->wH, w->C32, w->defl, w->swork, w->info};
  for (size_t i = 0; i < sizeof bufs / sizeof bufs[0]; i++)
    if (bufs[i]) cudaFree(bufs[i]);
  if (w->blas) cublasDestroy(w->blas);
  if (w->sol) cusolverDnDestroy(w->sol);
  for (int i = 0; i < 16; i++)
    if (w->ev[i]) cudaEventDestroy(w->ev[i]);
  memset(w, 0, sizeof *w);
}

void bdg_solver_release(bdg_t *bdg) {
  if (bdg->solver_ws) {
    ws_free((ws_t *)bdg->solver_ws);
    free(bdg->solver_ws);
    bdg->solver_ws = NULL;
  }
  safe_free(&bdg->block);
}

const void *bdg_solver_block(const bdg_t *bdg) { return bdg->block; }

#define CUDA_TRY(x)                                                                     \
  do {                                                                                  \
    cudaError_t _e = (x);                                                               \
    if (_e != cudaSuccess) {                                                            \
      fprintf(stderr, "bdg_solve: %s failed: %s\n", #x, cudaGetErrorString(_e));        \
      return -1;                                                                        \
    }                                                                                   \
  } while (0)
#define BLAS_TRY(x)                                                                     \
  do {                                                                                  \
    cublasStatus_t _s = (x);                                                            \
    if (_s != CUBLAS_STATUS_SUCCESS) {                                                  \
      fprintf(stderr, "bdg_solve: %s failed: %d\n", #x, (int)_s);                       \
      return -2;                                                                        \
    }                                                                                   \
  } while (0)
#define SOL_TRY(x)                                                                      \
  do {                                                                                  \
    cusolverStatus_t _s = (x);                                                          \
    if (_s != CUSOLVER_STATUS_SUCCESS) {                                                \
      fprintf(stderr, "bdg_solve: %s failed: %d\n", #x, (int)_s);                       \
      return -3;                                                                        \
    }                                                                                   \
  } while (0)
#define DEV_TRY(x)                                                                      \
  do {                                                                                  \
    int _r = (x);                                                                       \
    if (_r) {                                                                           \
      fprintf(stderr, "bdg_solve: %s failed (%d): %s\n", #x, _r, bdgd_last_error());    \
      return _r;                                                                        \
    }                                                                                   \
  } while (0)

static int dmalloc(void **p, size_t bytes) {
  CUDA_TRY(cudaMalloc(p, bytes ? bytes : 16));
  return 0;
}

static int ws_setup(ws_t *w, bdgd_ctx *dev, uint64_t S, uint64_t m, uint64_t nev, int cplx, int prec) {
  if (w->S0 && w->cap_S == S && w->cap_m == m && w->cap_nev == nev && w->cap_cplx == cplx && w->cap_prec == prec)
    return 0;
  ws_free(w);
  w->S = S;
  w->n = 2 * S;
  w->m = m;
  w->nev = nev;
  w->kmax = 3 * m;
  w->cplx = cplx;
  w->prec = prec;
  w->esz = (prec == BDGD_F32 ? 4 : 8) * (cplx ? 2 : 1);
  const size_t blk = w->n * w->kmax * w->esz;
  int rc;
  if ((rc = dmalloc(&w->S0, blk)) || (rc = dmalloc(&w->S1, blk)) || (rc = dmalloc(&w->AS0, blk)) ||
      (rc = dmalloc(&w->AS1, blk)) || (rc = dmalloc(&w->R, w->n * m * w->esz)) ||
      (rc = dmalloc(&w->TR, S * nev * w->esz)))
    return rc;
  const size_t es = cplx ? 2 : 1;
  const size_t kk = w->kmax * w->kmax * es * sizeof(double);
  void **small[] = {(void **)&w->Gs, (void **)&w->Gb, (void **)&w->Ga, (void **)&w->Z, (void **)&w->T1,
                    (void **)&w->T2, (void **)&w->Ga2, (void **)&w->Gb2, (void **)&w->Y, (void **)&w->H,
                    (void **)&w->V, (void **)&w->C64};
  for (size_t i = 0; i < sizeof small / sizeof small[0]; i++)
    if ((rc = dmalloc(small[i], kk))) return rc;
  if ((rc = dmalloc((void **)&w->C32, kk)) || (rc = dmalloc((void **)&w->gram, 4 * kk)) ||
      (rc = dmalloc((void **)&w->lam, w->kmax * sizeof(double))) ||
      (rc = dmalloc((void **)&w->work, 2 * 64 * w->kmax * sizeof(double))) ||
      (rc = dmalloc((void **)&w->norms, 4 * w->kmax * sizeof(double))) ||
      (rc = dmalloc((void **)&w->dsc, w->kmax * sizeof(double))) ||
      (rc = dmalloc((void **)&w->wG, w->kmax * sizeof(double))) ||
      (rc = dmalloc((void **)&w->wA, w->kmax * sizeof(double))) ||
      (rc = dmalloc((void **)&w->wH, w->kmax * sizeof(double))) || (rc = dmalloc((void **)&w->info, sizeof(int))))
    return rc;
  BLAS_TRY(cublasCreate(&w->blas));
  BLAS_TRY(cublasSetStream(w->blas, (cudaStream_t)bdgd_stream(dev)));
  SOL_TRY(cusolverDnCreate(&w->sol));
  SOL_TRY(cusolverDnSetStream(w->sol, (cudaStream_t)bdgd_stream(dev)));
  int lw = 0;
  const int K = (int)w->kmax;
  if (cplx) {
    SOL_TRY(cusolverDnZheevd_bufferSize(w->sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, K,
                                        (cuDoubleComplex *)w->Gs, K, w->wG, &lw));
    w->lwork = lw;
    if ((rc = dmalloc(&w->swork, (size_t)lw * sizeof(cuDoubleComplex)))) return rc;
  } else {
    SOL_TRY(cusolverDnDsyevd_bufferSize(w->sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, K, w->Gs, K,
                                        w->wG, &lw));
    w->lwork = lw;
    if ((rc = dmalloc(&w->swork, (size_t)lw * sizeof(double)))) return rc;
  }
  for (int i = 0; i < 16; i++) CUDA_TRY(cudaEventCreate(&w->ev[i]));
  w->cap_S = S;
  w->cap_m = m;
  w->cap_nev = nev;
  w->cap_cplx = cplx;
  w->cap_prec = prec;
  return 0;
}

/* Hermitian eigen-decomposition in place (eigenvalues ascending). */
static int heev(ws_t *w, double *A, int k, double *wout) {
  if (w->cplx)
    SOL_TRY(cusolverDnZheevd(w->sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, k, (cuDoubleComplex *)A, k,
                             wout, (cuDoubleComplex *)w->swork, w->lwork, w->info));
  else
    SOL_TRY(cusolverDnDsyevd(w->sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, k, A, k, wout,
                             (double *)w->swork, w->lwork, w->info));
  return 0;
}

/* small FP64 GEMM: C = op(A) op(B), op = N or H */
static int sgemm_small(ws_t *w, int ha, int hb, int M, int N, int K, const double *A, int lda, const double *B,
                       int ldb, double *C, int ldc) {
  if (w->cplx) {
    const cuDoubleComplex one = {1.0, 0.0}, zero = {0.0, 0.0};
    BLAS_TRY(cublasZgemm(w->blas, ha ? CUBLAS_OP_C : CUBLAS_OP_N, hb ? CUBLAS_OP_C : CUBLAS_OP_N, M, N, K, &one,
                         (const cuDoubleComplex *)A, lda, (const cuDoubleComplex *)B, ldb, &zero,
                         (cuDoubleComplex *)C, ldc));
  } else {
    const double one = 1.0, zero = 0.0;
    BLAS_TRY(cublasDgemm(w->blas, ha ? CUBLAS_OP_T : CUBLAS_OP_N, hb ? CUBLAS_OP_T : CUBLAS_OP_N, M, N, K, &one, A,
                         lda, B, ldb, &zero, C, ldc));
  }
  return 0;
}

/* Rayleigh-Ritz on the Gram blocks in w->gram (k x k).  On return w->C64
 * holds C (k x m), lam_host the m eigenvalues (ascending), *nsel the number
 * selected. */
static int rayleigh_ritz(ws_t *w, bdgd_ctx *dev, int k, int m, double drop, double *lam_host, int *nsel) {
  cudaStream_t st = (cudaStream_t)bdgd_stream(dev);
  const int cplx = w->cplx;
  const size_t es = cplx ? 2 : 1;
  DEV_TRY(bdgd_rr_prepare(dev, w->gram, k, cplx, w->Gs, w->Gb, w->Ga, w->dsc));
  int rc;
  if ((rc = heev(w, w->Gs, k, w->wG))) return rc;
  double hw[3 * 1024];
  if (k > 3 * 1024) return -4;
  CUDA_TRY(cudaMemcpyAsync(hw, w->wG, k * sizeof(double), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  const double smax = hw[k - 1];
  int keep = 0;
  for (int i = 0; i < k; i++)
    if (hw[i] > drop * smax) keep++;
  if (keep < m) keep = (m <= k) ? m : k;
  /* Z = D Q[:, k-keep:] diag(s^-1/2) */
  DEV_TRY(bdgd_scale_cols(dev, w->Gs, k, k - keep, keep, cplx, w->dsc, w->wG, 1, 0, w->Z));
  if ((rc = sgemm_small(w, 0, 0, k, keep, k, w->Ga, k, w->Z, k, w->T1, k))) return rc;
  if ((rc = sgemm_small(w, 1, 0, keep, keep, k, w->Z, k, w->T1, k, w->Ga2, keep))) return rc;
  if ((rc = sgemm_small(w, 0, 0, k, keep, k, w->Gb, k, w->Z, k, w->T1, k))) return rc;
  if ((rc = sgemm_small(w, 1, 0, keep, keep, k, w->Z, k, w->T1, k, w->Gb2, keep))) return rc;
  DEV_TRY(bdgd_hermitize(dev, w->Ga2, keep, cplx));
  DEV_TRY(bdgd_hermitize(dev, w->Gb2, keep, cplx));
  if ((rc = heev(w, w->Ga2, keep, w->wA))) return rc;
  DEV_TRY(bdgd_clamp(dev, w->wA, keep, RR_CLAMP));
  /* Y = Q2 diag(dA^-1/2); H = Y^H Gb2 Y */
  DEV_TRY(bdgd_scale_cols(dev, w->Ga2, keep, 0, keep, cplx, NULL, w->wA, 1, 0, w->Y));
  if ((rc = sgemm_small(w, 0, 0, keep, keep, keep, w->Gb2, keep, w->Y, keep, w->T1, keep))) return rc;
  if ((rc = sgemm_small(w, 1, 0, keep, keep, keep, w->Y, keep, w->T1, keep, w->H, keep))) return rc;
  DEV_TRY(bdgd_hermitize(dev, w->H, keep, cplx));
  if ((rc = heev(w, w->H, keep, w->wH))) return rc;
  CUDA_TRY(cudaMemcpyAsync(hw, w->wH, keep * sizeof(double), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  int npos = 0;
  for (int i = 0; i < keep; i++)
    if (hw[i] > 0) npos++;
  const int sel = npos < m ? npos : m;
  *nsel = sel;
  if (sel == 0) return 0;
  /* V = Q3[:, largest theta first] diag(theta^-1/2); C = Z Y V */
  DEV_TRY(bdgd_scale_cols(dev, w->H, keep, keep - sel, sel, cplx, NULL, w->wH, 1, 1, w->V));
  if ((rc = sgemm_small(w, 0, 0, keep, sel, keep, w->Y, keep, w->V, keep, w->T2, keep))) return rc;
  if ((rc = sgemm_small(w, 0, 0, k, sel, keep, w->Z, k, w->T2, keep, w->C64, k))) return rc;
  for (int j = 0; j < sel; j++) lam_host[j] = 1.0 / hw[keep - 1 - j];
  (void)es;
  return 0;
}

/* Y[:, 0:ncol] = X[:, 0:k] C (C is k x ncol FP64 on device, leading dim ldc).
 * X, Y blocks of the current precision with leading dimension n. */
static int block_gemm(ws_t *w, bdgd_ctx *dev, const void *X, int k, const double *C, int ldc, int ncol, void *Y) {
  const int n = (int)w->n;
  if (w->prec == BDGD_F32) {
    /* C -> float (k x ncol, leading dim k) */
    DEV_TRY(bdgd_scale_cols(dev, C, ldc, 0, ncol, w->cplx, NULL, NULL, 0, 0, w->T1));
    DEV_TRY(bdgd_convert(dev, 1, w->T1, w->C32, (uint64_t)ldc * ncol * (w->cplx ? 2 : 1)));
    if (w->cplx) {
      const cuComplex one = {1.f, 0.f}, zero = {0.f, 0.f};
      BLAS_TRY(cublasCgemm(w->blas, CUBLAS_OP_N, CUBLAS_OP_N, n, ncol, k, &one, (const cuComplex *)X, n,
                           (const cuComplex *)w->C32, ldc, &zero, (cuComplex *)Y, n));
    } else {
      const float one = 1.f, zero = 0.f;
      BLAS_TRY(cublasSgemm(w->blas, CUBLAS_OP_N, CUBLAS_OP_N, n, ncol, k, &one, (const float *)X, n, w->C32, ldc,
                           &zero, (float *)Y, n));
    }
  } else if (w->cplx) {
    const cuDoubleComplex one = {1.0, 0.0}, zero = {0.0, 0.0};
    BLAS_TRY(cublasZgemm(w->blas, CUBLAS_OP_N, CUBLAS_OP_N, n, ncol, k, &one, (const cuDoubleComplex *)X, n,
                         (const cuDoubleComplex *)C, ldc, &zero, (cuDoubleComplex *)Y, n));
  } else {
    const double one = 1.0, zero = 0.0;
    BLAS_TRY(cublasDgemm(w->blas, CUBLAS_OP_N, CUBLAS_OP_N, n, ncol, k, &one, (const double *)X, n, C, ldc, &zero,
                         (double *)Y, n));
  }
  return 0;
}

static inline void *col_ptr(ws_t *w, void *base, uint64_t col) { return (char *)base + col * w->n * w->esz; }

static double now_s(void) {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

static float ev_ms(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  return ms;
}

/* ||A|| bound: max kinetic energy + largest local term (+ dipolar exchange). */
static double anorm_estimate(const matmul_ctx_t *ctx) {
  double kin = 0.0;
  for (uint64_t d = 0; d < ctx->dim; d++) {
    double mx = 0.0;
    for (uint64_t j = 0; j < ctx->N[d]; j++) mx = fmax(mx, ctx->kx2[d][j]);
    kin += 0.5 * mx;
  }
  double aK = 0.0, aM = 0.0;
  for (uint64_t i = 0; i < ctx->size; i++) {
    aK = fmax(aK, fabs(ctx->localTermK[i]));
    aM = fmax(aM, fabs(ctx->localTermM[i]));
  }
  if (ctx->dipolar && ctx->dim == 3 && ctx->wf && ctx->longRngInt) {
    double wmax = 0.0, vmax = 0.0;
    for (uint64_t i = 0; i < ctx->size; i++) {
      const double a = ctx->complex_psi0 ? cabs(((const c64 *)ctx->wf)[i]) : fabs(((const f64 *)ctx->wf)[i]);
      wmax = fmax(wmax, a);
    }
    for (uint64_t i = 0; i < ctx->k_size; i++) vmax = fmax(vmax, fabs(ctx->longRngInt[i]));
    aM += 2.0 * fabs(ctx->g_ddi) * wmax * wmax * vmax;
  }
  return kin + fmax(aK, aM);
}

/* Evaluate the convergence measure of the first nev columns; writes
 * res_host[nev]; returns the number converged. */
static int check_convergence(ws_t *w, bdgd_ctx *dev, bdg_t *bdg, const void *X, const void *AX, double anorm,
                             const double *lam_host, double *res_host, double *tres_host, int want_true) {
  cudaStream_t st = (cudaStream_t)bdgd_stream(dev);
  const int nev = (int)w->nev;
  double h[4 * 1024];
  DEV_TRY(bdgd_residual(dev, w->prec, w->cplx, w->S, w->m, X, AX, w->n, w->R, w->n, w->lam, w->work, w->norms,
                        w->norms + w->kmax));
  const int tr = want_true || bdg->criterion == BDG_CONV_TRUE_RESIDUAL;
  if (tr) {
    /* K (M v): M v is the lower half of AX */
    const char *Mv = (const char *)AX + w->S * w->esz;
    DEV_TRY(bdgd_apply(dev, BDGD_OP_K, w->prec, Mv, w->n, w->TR, w->S, (uint64_t)nev));
    DEV_TRY(bdgd_true_residual(dev, w->prec, w->cplx, w->S, (uint64_t)nev, w->TR, w->S, X, w->n, w->lam, w->work,
                               w->norms + 2 * w->kmax, w->norms + 3 * w->kmax));
  }
  CUDA_TRY(cudaMemcpyAsync(h, w->norms, 4 * w->kmax * sizeof(double), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  int nconv = 0;
  for (int j = 0; j < nev; j++) {
    const double rr = sqrt(h[j]), xx = sqrt(h[w->kmax + j]);
    const double back = rr / ((anorm + fabs(lam_host[j])) * (xx > 0 ? xx : 1e-300));
    double tres = NAN;
    if (tr) {
      const double tt = sqrt(h[2 * w->kmax + j]), vv = sqrt(h[3 * w->kmax + j]);
      tres = tt / (vv > 0 ? vv : 1e-300);
    }
    res_host[j] = (bdg->criterion == BDG_CONV_TRUE_RESIDUAL) ? tres : back;
    if (tres_host) tres_host[j] = tres;
    if (res_host[j] <= bdg->tol) nconv++;
  }
  return nconv;
}

/* One full iLOBPCG run with blocks of the workspace precision, starting from
 * X in S0[:, 0:m].  Returns 0 or an error; leaves X, AX in S0/AS0. */
static int run_loop(ws_t *w, bdgd_ctx *dev, bdg_t *bdg, uint64_t maxit, double anorm, double *lam_host,
                    uint64_t *iters, int *nconv_out, double *res_host) {
  cudaStream_t st = (cudaStream_t)bdgd_stream(dev);
  const uint64_t m = w->m, S = w->S;
  const double drop = (w->prec == BDGD_F32) ? RR_DROP_F32 : RR_DROP_F64;
  int rc, nsel = 0;
  bdg_solve_stats_t *ss = &bdg->stats;
  /* AX = A X, Rayleigh-Ritz on span X */
  cudaEventRecord(w->ev[0], st);
  DEV_TRY(bdgd_apply(dev, BDGD_OP_LREP, w->prec, w->S0, w->n, w->AS0, w->n, m));
  cudaEventRecord(w->ev[1], st);
  DEV_TRY(bdgd_gram(dev, w->prec, w->cplx, S, m, w->S0, w->n, w->AS0, w->n, w->gram));
  if ((rc = rayleigh_ritz(w, dev, (int)m, (int)m, drop, lam_host, &nsel))) return rc;
  if (nsel < (int)m) {
    fprintf(stderr, "bdg_solve: initial block is not B-positive (%d of %lu positive-type)\n", nsel,
            (unsigned long)m);
    return -5;
  }
  if ((rc = block_gemm(w, dev, w->S0, (int)m, w->C64, (int)m, (int)m, w->S1))) return rc;
  if ((rc = block_gemm(w, dev, w->AS0, (int)m, w->C64, (int)m, (int)m, w->AS1))) return rc;
  void *t;
  t = w->S0; w->S0 = w->S1; w->S1 = t;
  t = w->AS0; w->AS0 = w->AS1; w->AS1 = t;
  CUDA_TRY(cudaMemcpyAsync(w->lam, lam_host, m * sizeof(double), cudaMemcpyHostToDevice, st));
  ss->ms_apply_A += ev_ms(w->ev[0], w->ev[1]);
  ss->cols_apply_A += m;
  int have_p = 0;
  uint64_t it = 0;
  int nconv = 0;
  for (;;) {
    cudaEventRecord(w->ev[2], st);
    nconv = check_convergence(w, dev, bdg, w->S0, w->AS0, anorm, lam_host, res_host, NULL, 0);
    if (nconv < 0) return nconv;
    cudaEventRecord(w->ev[3], st);
    if (nconv >= (int)w->nev || it >= maxit) break;
    /* W = T R into the W slot, AW = A W */
    void *W = col_ptr(w, w->S0, m), *AW = col_ptr(w, w->AS0, m);
    DEV_TRY(bdgd_apply(dev, BDGD_OP_TLREP, w->prec, w->R, w->n, W, w->n, m));
    cudaEventRecord(w->ev[4], st);
    DEV_TRY(bdgd_apply(dev, BDGD_OP_LREP, w->prec, W, w->n, AW, w->n, m));
    cudaEventRecord(w->ev[5], st);
    const int k = have_p ? (int)(3 * m) : (int)(2 * m);
    DEV_TRY(bdgd_gram(dev, w->prec, w->cplx, S, (uint64_t)k, w->S0, w->n, w->AS0, w->n, w->gram));
    cudaEventRecord(w->ev[6], st);
    if ((rc = rayleigh_ritz(w, dev, k, (int)m, drop, lam_host, &nsel))) return rc;
    cudaEventRecord(w->ev[7], st);
    if (nsel < (int)m) {
      fprintf(stderr, "bdg_solve: search space lost B-positivity (%d of %lu)\n", nsel, (unsigned long)m);
      return -6;
    }
    /* X <- S C ; P <- S[:, m:k] C[m:k, :] (same for AS) */
    const size_t cel = w->cplx ? 2 : 1;
    const double *Cwp = w->C64 + m * cel;
    if ((rc = block_gemm(w, dev, w->S0, k, w->C64, k, (int)m, w->S1))) return rc;
    if ((rc = block_gemm(w, dev, W, k - (int)m, Cwp, k, (int)m, col_ptr(w, w->S1, 2 * m)))) return rc;
    if ((rc = block_gemm(w, dev, w->AS0, k, w->C64, k, (int)m, w->AS1))) return rc;
    if ((rc = block_gemm(w, dev, AW, k - (int)m, Cwp, k, (int)m, col_ptr(w, w->AS1, 2 * m)))) return rc;
    cudaEventRecord(w->ev[8], st);
    t = w->S0; w->S0 = w->S1; w->S1 = t;
    t = w->AS0; w->AS0 = w->AS1; w->AS1 = t;
    CUDA_TRY(cudaMemcpyAsync(w->lam, lam_host, m * sizeof(double), cudaMemcpyHostToDevice, st));
    have_p = 1;
    it++;
    CUDA_TRY(cudaEventSynchronize(w->ev[8]));
    ss->ms_residual += ev_ms(w->ev[2], w->ev[3]);
    ss->ms_apply_T += ev_ms(w->ev[3], w->ev[4]);
    ss->ms_apply_A += ev_ms(w->ev[4], w->ev[5]);
    ss->ms_gram += ev_ms(w->ev[5], w->ev[6]);
    ss->ms_small_dense += ev_ms(w->ev[6], w->ev[7]);
    ss->ms_update += ev_ms(w->ev[7], w->ev[8]);
    ss->cols_apply_A += m;
    ss->cols_apply_T += m;
  }
  *iters = it;
  *nconv_out = nconv;
  return 0;
}

static int solve_gpu(bdg_t *bdg) {
  const double t0 = now_s();
  matmul_ctx_t *ctx = bdg->ctx;
  const int cplx = bdg->complex_psi0;
  const uint64_t S = ctx->size, n = 2 * S, m = bdg->sizeSub, nev = bdg->nev;
  memset(&bdg->stats, 0, sizeof bdg->stats);
  if (nev == 0 || m < nev) {
    fprintf(stderr, "bdg_solve: need 0 < nev <= sizeSub\n");
    return -7;
  }
  safe_free((void **)&bdg->eigvals);
  safe_free(&bdg->modes_u);
  safe_free(&bdg->modes_v);
  /* mirror every operator field on the device */
  int rc = bdg_ctx_sync_device(ctx, BDGD_OP_LREP);
  if (!rc) rc = bdg_ctx_sync_device(ctx, BDGD_OP_TLREP);
  if (rc) {
    fprintf(stderr, "bdg_solve: device setup failed (%d): %s\n", rc, bdgd_last_error());
    return rc;
  }
  bdgd_ctx *dev = ctx->dev;
  cudaStream_t st = (cudaStream_t)bdgd_stream(dev);
  if (!bdg->solver_ws) bdg->solver_ws = xcalloc(1, sizeof(ws_t));
  ws_t *w = (ws_t *)bdg->solver_ws;
  const int prec = (bdg->precision == BDG_PREC_MIXED) ? BDGD_F32 : BDGD_F64;
  if ((rc = ws_setup(w, dev, S, m, nev, cplx, prec))) return rc;
  /* initial block on the host, then to the device */
  const size_t hesz = cplx ? sizeof(c64) : sizeof(f64);
  void *X0 = xcalloc(n * m, hesz);
  bdg_fill_initial_block(bdg, X0);
  if (prec == BDGD_F32) {
    void *tmp = NULL;
    if ((rc = dmalloc(&tmp, n * m * hesz))) return rc;
    CUDA_TRY(cudaMemcpyAsync(tmp, X0, n * m * hesz, cudaMemcpyHostToDevice, st));
    DEV_TRY(bdgd_convert(dev, 1, tmp, w->S0, n * m * (cplx ? 2 : 1)));
    CUDA_TRY(cudaStreamSynchronize(st));
    cudaFree(tmp);
  } else {
    CUDA_TRY(cudaMemcpyAsync(w->S0, X0, n * m * hesz, cudaMemcpyHostToDevice, st));
  }
  const double anorm = anorm_estimate(ctx);
  double *lam = xcalloc(3 * m, sizeof(double));
  double *res = xcalloc(nev, sizeof(double));
  uint64_t iters = 0;
  int nconv = 0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  rc = run_loop(w, dev, bdg, bdg->maxIter, anorm, lam, &iters, &nconv, res);
  cudaEventRecord(e1, st);
  cudaEventSynchronize(e1);
  bdg->stats.seconds_device = 1e-3 * ev_ms(e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  bdg->stats.iterations = iters;
  if (rc) {
    bdg->stats.status = rc;
    free(X0);
    free(lam);
    free(res);
    return rc;
  }
  /* final true residual of the wanted pairs (reported in the stats) */
  double *tres = xcalloc(nev, sizeof(double));
  {
    double *tmp = xcalloc(nev, sizeof(double));
    check_convergence(w, dev, bdg, w->S0, w->AS0, anorm, lam, tmp, tres, 1);
    double mx = 0.0, mt = 0.0;
    for (uint64_t j = 0; j < nev; j++) {
      mx = fmax(mx, res[j]);
      mt = fmax(mt, tres[j]);
    }
    bdg->stats.max_residual = mx;
    bdg->stats.max_true_residual = mt;
    free(tmp);
  }
  /* results: eigenvalues, modes, full block */
  bdg->converged = (uint64_t)nconv;
  bdg->eigvals = xcalloc(nev, sizeof(f64));
  memcpy(bdg->eigvals, lam, nev * sizeof(f64));
  safe_free(&bdg->block);
  bdg->block = xcalloc(n * m, hesz);
  if (prec == BDGD_F32) {
    void *tmp = NULL;
    if ((rc = dmalloc(&tmp, n * m * hesz))) return rc;
    DEV_TRY(bdgd_convert(dev, 0, w->S0, tmp, n * m * (cplx ? 2 : 1)));
    CUDA_TRY(cudaMemcpyAsync(bdg->block, tmp, n * m * hesz, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    cudaFree(tmp);
  } else {
    CUDA_TRY(cudaMemcpyAsync(bdg->block, w->S0, n * m * hesz, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
  }
  char *mu = xcalloc(S * nev, hesz), *mv = xcalloc(S * nev, hesz);
  for (uint64_t j = 0; j < nev; j++) {
    memcpy(mu + j * S * hesz, (char *)bdg->block + j * n * hesz, S * hesz);
    memcpy(mv + j * S * hesz, (char *)bdg->block + (j * n + S) * hesz, S * hesz);
  }
  bdg->modes_u = mu;
  bdg->modes_v = mv;
  free(X0);
  free(lam);
  free(res);
  free(tres);
  bdg->stats.seconds_total = now_s() - t0;
  return 0;
}

int bdg_solve_d(bdg_t *bdg) { return solve_gpu(bdg); }
int bdg_solve_z(bdg_t *bdg) { return solve_gpu(bdg); }
