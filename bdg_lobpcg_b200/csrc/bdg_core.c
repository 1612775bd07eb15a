/*
 * bdg_core.c -- operator context and the reference's single-column operator
 * entry points, served by the GPU.
 *
 * Reference counterparts (pstuermer/BDG_LOBPCG): src/matmul_ctx.c (context,
 * k tables), src/kinetic_impl.inc, src/matmulK_impl.inc, src/matmulM_impl.inc,
 * src/matmulLrep_impl.inc, src/matmulSwap_impl.inc, src/precond_impl.inc,
 * src/dipolar_conv_impl.inc, src/dipolar.c, src/dipolar_meanfield_impl.inc.
 *
 * The host context keeps the reference's arrays (tests write them directly);
 * every operator call mirrors the arrays it reads onto the device and runs
 * the batched kernels of bdg_ops.cu on one column.
 */
#include <math.h>
#include <stdarg.h>
#include <string.h>
#include <unistd.h>

#include "bdg/bdg_cuda.h"
#include "bdg/bdg_internal.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ---- logging (reference src/bdg_log.h: errors exit with EXIT_FAILURE) --- */
static int use_color(void) {
  static int cached = -1; /* idempotent; atomic loads/stores as several threads may log */
  int c = __atomic_load_n(&cached, __ATOMIC_RELAXED);
  if (c < 0) {
    c = isatty(STDERR_FILENO);
    __atomic_store_n(&cached, c, __ATOMIC_RELAXED);
  }
  return c;
}

void bdg_fatal(const char *file, int line, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  fprintf(stderr, use_color() ? "\033[1;31mERROR\033[0m [%s:%d] " : "ERROR [%s:%d] ", file, line);
  vfprintf(stderr, fmt, ap);
  fprintf(stderr, "\n");
  va_end(ap);
  exit(EXIT_FAILURE);
}

void bdg_warn(const char *file, int line, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  fprintf(stderr, use_color() ? "\033[1;33mWARN\033[0m [%s:%d] " : "WARN [%s:%d] ", file, line);
  vfprintf(stderr, fmt, ap);
  fprintf(stderr, "\n");
  va_end(ap);
}

/* ---- context --------------------------------------------------------------- */
matmul_ctx_t *matmul_ctx_alloc(uint64_t dim, const uint64_t *N, const f64 *L) {
  if (dim < 1 || dim > 3) BDG_ERROR("matmul_ctx_alloc: dim must be 1, 2 or 3 (got %lu)", (unsigned long)dim);
  matmul_ctx_t *ctx = xcalloc(1, sizeof(matmul_ctx_t));
  ctx->dim = dim;
  ctx->N = xcalloc(dim, sizeof(uint64_t));
  ctx->L = xcalloc(dim, sizeof(f64));
  ctx->size = 1;
  for (uint64_t d = 0; d < dim; d++) {
    if (N[d] == 0) BDG_ERROR("matmul_ctx_alloc: N[%lu] is zero", (unsigned long)d);
    ctx->N[d] = N[d];
    ctx->L[d] = L[d];
    ctx->size *= N[d];
  }
  ctx->localTermK = xcalloc(ctx->size, sizeof(f64));
  ctx->localTermM = xcalloc(ctx->size, sizeof(f64));
  ctx->prec = BDG_PREC_F64;
  return ctx;
}

void matmul_ctx_free(matmul_ctx_t **pctx) {
  if (!pctx || !*pctx) return;
  matmul_ctx_t *ctx = *pctx;
  if (ctx->dev) bdgd_destroy(&ctx->dev);
  safe_free(&ctx->fwd_plan);
  safe_free(&ctx->bwd_plan);
  if (ctx->kx2) {
    for (uint64_t d = 0; d < ctx->dim; d++) safe_free((void **)&ctx->kx2[d]);
    safe_free((void **)&ctx->kx2);
  }
  safe_free((void **)&ctx->k2);
  safe_free((void **)&ctx->localTermK);
  safe_free((void **)&ctx->localTermM);
  safe_free((void **)&ctx->longRngInt);
  safe_free(&ctx->wf);
  safe_free((void **)&ctx->precond_sqrtK);
  safe_free((void **)&ctx->precond_sqrtM);
  safe_free(&ctx->f_wrk);
  safe_free(&ctx->c_wrk1);
  safe_free(&ctx->c_wrk2);
  safe_free((void **)&ctx->N);
  safe_free((void **)&ctx->L);
  safe_free((void **)pctx);
}

/* Plan handle stored in fwd_plan / bwd_plan: names the device transform of
 * this context in one direction. */
typedef struct {
  matmul_ctx_t *ctx;
  int forward;
} bdg_fft_plan_t;

void matmul_ctx_set_system(matmul_ctx_t *ctx, int complex_psi0) {
  ctx->complex_psi0 = complex_psi0;
  /* k_size (reference src/matmul_ctx.c:94-101) */
  if (complex_psi0) {
    ctx->k_size = ctx->size;
  } else {
    ctx->k_size = ctx->N[0] / 2 + 1;
    for (uint64_t d = 1; d < ctx->dim; d++) ctx->k_size *= ctx->N[d];
  }
  /* kx2[d][j] = (dk * wrapped j)^2 (reference :103-113) */
  ctx->kx2 = xcalloc(ctx->dim, sizeof(f64 *));
  for (uint64_t d = 0; d < ctx->dim; d++) {
    ctx->kx2[d] = xcalloc(ctx->N[d], sizeof(f64));
    const f64 dk = 2.0 * M_PI / ctx->L[d];
    for (uint64_t j = 0; j < ctx->N[d]; j++) {
      const f64 kj = (j <= ctx->N[d] / 2) ? dk * (f64)j : dk * (f64)((int64_t)j - (int64_t)ctx->N[d]);
      ctx->kx2[d][j] = kj * kj;
    }
  }
  /* k2 flat on the spectrum layout, x fastest (reference :116-132) */
  const uint64_t n0k = complex_psi0 ? ctx->N[0] : ctx->N[0] / 2 + 1;
  const uint64_t ny = ctx->dim > 1 ? ctx->N[1] : 1;
  const uint64_t nz = ctx->dim > 2 ? ctx->N[2] : 1;
  ctx->k2 = xcalloc(ctx->k_size, sizeof(f64));
  for (uint64_t iz = 0; iz < nz; iz++)
    for (uint64_t iy = 0; iy < ny; iy++)
      for (uint64_t ix = 0; ix < n0k; ix++) {
        f64 v = ctx->kx2[0][ix];
        if (ctx->dim > 1) v += ctx->kx2[1][iy];
        if (ctx->dim > 2) v += ctx->kx2[2][iz];
        ctx->k2[(iz * ny + iy) * n0k + ix] = v;
      }
  /* host scratch of the reference's shapes (reference :143-146) */
  const uint64_t wrk = ctx->size > ctx->k_size ? ctx->size : ctx->k_size;
  ctx->f_wrk = xcalloc(ctx->k_size, 2 * sizeof(f64));
  ctx->c_wrk1 = xcalloc(wrk, 2 * sizeof(f64));
  ctx->c_wrk2 = xcalloc(wrk, 2 * sizeof(f64));
  bdg_fft_plan_t *fp = xcalloc(1, sizeof(bdg_fft_plan_t));
  bdg_fft_plan_t *bp = xcalloc(1, sizeof(bdg_fft_plan_t));
  fp->ctx = ctx;
  fp->forward = 1;
  bp->ctx = ctx;
  bp->forward = 0;
  ctx->fwd_plan = fp;
  ctx->bwd_plan = bp;
  /* the device context (and its FFT tables) is built on first GPU use */
}

static int op_reads_fields(int op, int *lt, int *wf, int *pre, int *dip) {
  *lt = (op == BDGD_OP_K || op == BDGD_OP_M || op == BDGD_OP_LREP);
  *pre = (op == BDGD_OP_TK || op == BDGD_OP_TM || op == BDGD_OP_TLREP);
  *dip = (op == BDGD_OP_DIPCONV || op == BDGD_OP_M || op == BDGD_OP_LREP);
  *wf = *dip;
  return 0;
}

int bdg_ctx_sync_device(matmul_ctx_t *ctx, int op) {
  if (ctx->k2 == NULL) {
    fprintf(stderr, "bdg: operator applied before matmul_ctx_set_system\n");
    return BDGD_ERR_STATE;
  }
  int rc;
  if (ctx->dev == NULL) {
    rc = bdgd_create(&ctx->dev, ctx->dim, ctx->N, ctx->L, ctx->complex_psi0);
    if (rc) return rc;
  }
  int lt, wf, pre, dip;
  op_reads_fields(op, &lt, &wf, &pre, &dip);
  if (lt && (rc = bdgd_set_local_terms(ctx->dev, ctx->localTermK, ctx->localTermM))) return rc;
  const int dip_on = (op == BDGD_OP_DIPCONV) || (ctx->dipolar && ctx->dim == 3);
  if (wf && dip_on && ctx->wf && (rc = bdgd_set_wavefunction(ctx->dev, ctx->wf))) return rc;
  if (pre && (rc = bdgd_set_precond(ctx->dev, ctx->precond_sqrtK, ctx->precond_sqrtM, ctx->mu))) return rc;
  if (dip) {
    rc = bdgd_set_dipolar(ctx->dev, dip_on ? ctx->longRngInt : NULL, ctx->g_ddi,
                          (int)(ctx->dipolar && ctx->dim == 3));
    if (rc) return rc;
  }
  return BDGD_OK;
}

void bdg_ctx_apply_host(matmul_ctx_t *ctx, int op, const void *x, void *y, uint64_t ncol, const char *caller) {
  int rc = bdg_ctx_sync_device(ctx, op);
  if (rc == 0) rc = bdgd_apply_host(ctx->dev, op, x, y, ncol);
  if (rc) BDG_ERROR("%s: GPU apply failed (%d): %s", caller, rc, bdgd_last_error());
}

/* ---- single-column operators on host pointers ----------------------------- */
#define DEF_OP(name, op)                                                  \
  void name##_d(matmul_ctx_t *ctx, const f64 *x, f64 *y) {               \
    if (ctx->complex_psi0) BDG_ERROR(#name "_d: context is complex");     \
    bdg_ctx_apply_host(ctx, op, x, y, 1, #name "_d");                     \
  }                                                                       \
  void name##_z(matmul_ctx_t *ctx, const c64 *x, c64 *y) {               \
    if (!ctx->complex_psi0) BDG_ERROR(#name "_z: context is real");       \
    bdg_ctx_apply_host(ctx, op, x, y, 1, #name "_z");                     \
  }

DEF_OP(kinetic, BDGD_OP_KINETIC)
DEF_OP(matmulK, BDGD_OP_K)
DEF_OP(matmulM, BDGD_OP_M)
DEF_OP(matmulLrep, BDGD_OP_LREP)
DEF_OP(precondK, BDGD_OP_TK)
DEF_OP(precondM, BDGD_OP_TM)
DEF_OP(precondLrep, BDGD_OP_TLREP)
DEF_OP(dipolar_conv, BDGD_OP_DIPCONV)

/* Swap needs no set_system (the reference tests call it on a bare context),
 * so the host side handles contexts without k tables by a plain copy. */
static void swap_host(matmul_ctx_t *ctx, const void *x, void *y, size_t esz) {
  const size_t hb = ctx->size * esz;
  if (ctx->k2 == NULL) {
    memcpy(y, (const char *)x + hb, hb);
    memcpy((char *)y + hb, x, hb);
    return;
  }
  bdg_ctx_apply_host(ctx, BDGD_OP_SWAP, x, y, 1, "matmulSwap");
}

void matmulSwap_d(matmul_ctx_t *ctx, const f64 *x, f64 *y) { swap_host(ctx, x, y, sizeof(f64)); }
void matmulSwap_z(matmul_ctx_t *ctx, const c64 *x, c64 *y) { swap_host(ctx, x, y, sizeof(c64)); }

/* ---- dipolar kernel (setup time, host; reference src/dipolar.c:21-72) ----- */
void dipolar_set_kernel(matmul_ctx_t *ctx, f64 g_ddi, const f64 *dipole_dir, f64 cutoff_radius) {
  if (ctx->dim != 3) BDG_ERROR("dipolar_set_kernel: requires dim == 3");
  if (ctx->k2 == NULL) BDG_ERROR("dipolar_set_kernel: call matmul_ctx_set_system first");
  ctx->g_ddi = g_ddi;
  const uint64_t Nx = ctx->N[0], Ny = ctx->N[1], Nz = ctx->N[2];
  const uint64_t n0k = ctx->complex_psi0 ? Nx : Nx / 2 + 1;
  const f64 dkx = 2.0 * M_PI / ctx->L[0];
  const f64 dky = 2.0 * M_PI / ctx->L[1];
  const f64 dkz = 2.0 * M_PI / ctx->L[2];
  const f64 dir_sq = dipole_dir[0] * dipole_dir[0] + dipole_dir[1] * dipole_dir[1] + dipole_dir[2] * dipole_dir[2];
  safe_free((void **)&ctx->longRngInt);
  ctx->longRngInt = xcalloc(ctx->k_size, sizeof(f64));
  for (uint64_t iz = 0; iz < Nz; iz++) {
    const int64_t fz = (iz <= Nz / 2) ? (int64_t)iz : (int64_t)iz - (int64_t)Nz;
    const f64 kz = dkz * (f64)fz;
    for (uint64_t iy = 0; iy < Ny; iy++) {
      const int64_t fy = (iy <= Ny / 2) ? (int64_t)iy : (int64_t)iy - (int64_t)Ny;
      const f64 ky = dky * (f64)fy;
      for (uint64_t ix = 0; ix < n0k; ix++) {
        const int64_t fx = (ctx->complex_psi0 && ix > Nx / 2) ? (int64_t)ix - (int64_t)Nx : (int64_t)ix;
        const f64 kx = dkx * (f64)fx;
        const uint64_t idx = (iz * Ny + iy) * n0k + ix;
        const f64 ksq = kx * kx + ky * ky + kz * kz;
        if (ksq < 1e-50) {
          ctx->longRngInt[idx] = 0.0;
          continue;
        }
        const f64 kd = kx * dipole_dir[0] + ky * dipole_dir[1] + kz * dipole_dir[2];
        const f64 cos2 = (kd * kd) / (ksq * dir_sq);
        const f64 kR = sqrt(ksq) * cutoff_radius;
        const f64 kR2 = kR * kR;
        const f64 cut = 1.0 + 3.0 * cos(kR) / kR2 - 3.0 * sin(kR) / (kR2 * kR);
        ctx->longRngInt[idx] = (3.0 * cos2 - 1.0) * cut;
      }
    }
  }
}

/* Phi_dd = g F^-1[kernel/size F|psi|^2], added to both local terms
 * (reference src/dipolar_meanfield_impl.inc:20-55); the transforms run on
 * the GPU. */
static void meanfield(matmul_ctx_t *ctx, const char *caller) {
  if (!ctx->wf || !ctx->longRngInt) BDG_ERROR("%s: needs wavefunction and kernel", caller);
  int rc = bdg_ctx_sync_device(ctx, BDGD_OP_KINETIC);
  if (!rc) rc = bdgd_set_wavefunction(ctx->dev, ctx->wf);
  if (!rc) rc = bdgd_set_dipolar(ctx->dev, ctx->longRngInt, ctx->g_ddi, 0);
  f64 *phi = xcalloc(ctx->size, sizeof(f64));
  if (!rc) rc = bdgd_dipolar_meanfield(ctx->dev, phi);
  if (rc) BDG_ERROR("%s: GPU mean field failed (%d): %s", caller, rc, bdgd_last_error());
  for (uint64_t i = 0; i < ctx->size; i++) {
    ctx->localTermK[i] += phi[i];
    ctx->localTermM[i] += phi[i];
  }
  safe_free((void **)&phi);
}

void dipolar_add_meanfield_d(matmul_ctx_t *ctx) { meanfield(ctx, "dipolar_add_meanfield_d"); }
void dipolar_add_meanfield_z(matmul_ctx_t *ctx) { meanfield(ctx, "dipolar_add_meanfield_z"); }
void dipolar_add_meanfield(matmul_ctx_t *ctx) {
  if (ctx->complex_psi0)
    dipolar_add_meanfield_z(ctx);
  else
    dipolar_add_meanfield_d(ctx);
}

/* Execute a plan handle of ctx->fwd_plan / ctx->bwd_plan on host arrays:
 * unnormalised, FFTW layout (r2c half spectrum along x, or c2c). */
int bdg_fft_execute(void *plan, const void *in, void *out) {
  bdg_fft_plan_t *p = (bdg_fft_plan_t *)plan;
  if (!p || !p->ctx) return BDGD_ERR_ARG;
  int rc = bdg_ctx_sync_device(p->ctx, BDGD_OP_KINETIC);
  if (rc) return rc;
  return bdgd_fft_host(p->ctx->dev, p->forward, in, out, 1);
}
