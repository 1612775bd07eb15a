/*
 * bdg_api.c -- problem lifecycle, physics setup, solver options.
 *
 * Same call order, state checks, defaults and arithmetic as the reference
 * (pstuermer/BDG_LOBPCG src/bdg.c:17-238 and src/setup.c:17-197).  Setup is
 * host work (the trap and interaction callbacks are host function
 * pointers); the dipolar mean field runs its transforms on the GPU.
 */
#include <inttypes.h>
#include <math.h>
#include <string.h>

#include "bdg/bdg_cuda.h"
#include "bdg/bdg_learn.h"
#include "bdg/bdg_internal.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ---- lifecycle (reference src/bdg.c:17-84) -------------------------------- */
bdg_t *bdg_alloc(uint64_t dim, const uint64_t *N, const f64 *L, int complex_psi0) {
  bdg_t *bdg = xcalloc(1, sizeof(bdg_t));
  bdg->complex_psi0 = complex_psi0;
  bdg->ctx = matmul_ctx_alloc(dim, N, L);
  bdg->ctx->complex_psi0 = complex_psi0;
  bdg->nev = 3;
  bdg->sizeSub = 6;
  bdg->maxIter = 500;
  bdg->tol = 1e-6;
  bdg->precision = BDG_PREC_F64;
  bdg->criterion = BDG_CONV_BACKWARD;
  bdg->deflate = 0;
  bdg->refine_iters = 3;
  return bdg;
}

void bdg_free(bdg_t **pb) {
  if (!pb || !*pb) return;
  bdg_t *b = *pb;
  safe_free((void **)&b->eigvals);
  safe_free(&b->modes_u);
  safe_free(&b->modes_v);
  safe_free(&b->reuse_buf);
  extern void bdg_solver_release(bdg_t *);
  bdg_solver_release(b);
  matmul_ctx_free(&b->ctx);
  safe_free((void **)pb);
}

void bdg_reset(bdg_t *bdg) {
  BDG_REQUIRE(bdg, BDG_HAS_SYSTEM, "bdg_reset");
  matmul_ctx_t *ctx = bdg->ctx;
  safe_free(&ctx->wf);
  safe_free((void **)&ctx->longRngInt);
  safe_free((void **)&ctx->precond_sqrtK);
  safe_free((void **)&ctx->precond_sqrtM);
  memset(ctx->localTermK, 0, ctx->size * sizeof(f64));
  memset(ctx->localTermM, 0, ctx->size * sizeof(f64));
  ctx->mu = 0.0;
  ctx->g_ddi = 0.0;
  ctx->dipolar = 0;
  ctx->wf_size = 0;
  safe_free((void **)&bdg->eigvals);
  safe_free(&bdg->modes_u);
  safe_free(&bdg->modes_v);
  safe_free(&bdg->block);
  bdg->modes_bytes = 0;
  bdg->block_ws = -1;
  bdg->converged = 0;
  bdg->state = BDG_HAS_SYSTEM;
}

void bdg_set_system(bdg_t *bdg) {
  matmul_ctx_set_system(bdg->ctx, bdg->complex_psi0);
  bdg->state |= BDG_HAS_SYSTEM;
}

void bdg_set_solver_params(bdg_t *bdg, uint64_t nev, uint64_t sizeSub, uint64_t maxIter, f64 tol) {
  bdg->nev = nev;
  bdg->sizeSub = sizeSub;
  bdg->maxIter = maxIter;
  bdg->tol = tol;
}

static void init_from_host_block(const bdg_t *bdg, void *X, uint64_t n, uint64_t sizeSub, void *param);

void bdg_set_init_mode(bdg_t *bdg, bdg_init_mode_t mode, bdg_init_fn fn, void *param) {
  if (fn != init_from_host_block) bdg->init_block = NULL; /* another init source replaces the stored block */
  bdg->init_mode = mode;
  bdg->custom_init_fn = fn;
  bdg->custom_init_param = param;
}

/* CUSTOM fill from the block given to bdg_set_initial_block */
static void init_from_host_block(const bdg_t *bdg, void *X, uint64_t n, uint64_t sizeSub, void *param) {
  (void)param;
  const size_t esz = bdg->complex_psi0 ? sizeof(c64) : sizeof(f64);
  if (bdg->init_block == NULL || n != bdg->init_block_n || sizeSub != bdg->init_block_m) {
    fprintf(stderr, "bdg_solve: the block of bdg_set_initial_block is %llu x %llu, the solve needs %llu x %llu\n",
            (unsigned long long)bdg->init_block_n, (unsigned long long)bdg->init_block_m, (unsigned long long)n,
            (unsigned long long)sizeSub);
    memset(X, 0, (size_t)(n * sizeSub) * esz);
    return;
  }
  memcpy(X, bdg->init_block, (size_t)(n * sizeSub) * esz);
}

int bdg_set_initial_block(bdg_t *bdg, const void *X, uint64_t n, uint64_t sizeSub) {
  BDG_REQUIRE(bdg, BDG_HAS_SYSTEM, "bdg_set_initial_block");
  if (X == NULL || n != 2 * bdg->ctx->size || sizeSub == 0 || sizeSub != bdg->sizeSub) return -2;
  bdg->init_block = X;
  bdg->init_block_n = n;
  bdg->init_block_m = sizeSub;
  bdg_set_init_mode(bdg, BDG_INIT_CUSTOM, init_from_host_block, NULL);
  return 0;
}

/* ---- setup (reference src/setup.c) ----------------------------------------- */
void bdg_set_trap(bdg_t *bdg, f64 (*V_trap)(uint64_t dim, const f64 *r, const void *param), const void *param) {
  BDG_REQUIRE(bdg, BDG_HAS_SYSTEM, "bdg_set_trap");
  if (V_trap == NULL) {
    BDG_WARN("bdg_set_trap: V_trap is NULL, skipping");
    return;
  }
  matmul_ctx_t *ctx = bdg->ctx;
  const uint64_t dim = ctx->dim;
  const uint64_t Nx = ctx->N[0];
  const uint64_t Ny = dim > 1 ? ctx->N[1] : 1;
  const uint64_t Nz = dim > 2 ? ctx->N[2] : 1;
  /* r_d = (i_d - N_d/2) * L_d / N_d, box [-L/2, L/2) (reference setup.c:35) */
  for (uint64_t iz = 0; iz < Nz; iz++) {
    const f64 z = dim > 2 ? ((f64)iz - 0.5 * (f64)Nz) * ctx->L[2] / (f64)Nz : 0.0;
    for (uint64_t iy = 0; iy < Ny; iy++) {
      const f64 y = dim > 1 ? ((f64)iy - 0.5 * (f64)Ny) * ctx->L[1] / (f64)Ny : 0.0;
      for (uint64_t ix = 0; ix < Nx; ix++) {
        const f64 x = ((f64)ix - 0.5 * (f64)Nx) * ctx->L[0] / (f64)Nx;
        const f64 r[3] = {x, y, z};
        const uint64_t idx = (iz * Ny + iy) * Nx + ix;
        const f64 V = V_trap(dim, r, param);
        ctx->localTermK[idx] += V;
        ctx->localTermM[idx] += V;
      }
    }
  }
  bdg->state |= BDG_HAS_TRAP;
}

void bdg_set_wavefunction(bdg_t *bdg, const void *wf, uint64_t wf_size) {
  BDG_REQUIRE(bdg, BDG_HAS_SYSTEM, "bdg_set_wavefunction");
  matmul_ctx_t *ctx = bdg->ctx;
  if (wf == NULL) BDG_ERROR("bdg_set_wavefunction: wf is NULL");
  if (wf_size != ctx->size)
    BDG_ERROR("bdg_set_wavefunction: wf_size (%" PRIu64 ") != grid size (%" PRIu64 ")", wf_size, ctx->size);
  safe_free(&ctx->wf);
  const size_t esz = bdg->complex_psi0 ? sizeof(c64) : sizeof(f64);
  ctx->wf = xcalloc(ctx->size, esz);
  memcpy(ctx->wf, wf, ctx->size * esz);
  ctx->wf_size = ctx->size;
  bdg->state |= BDG_HAS_WF;
}

void bdg_set_local_interactions(bdg_t *bdg, f64 (*U_intK)(const void *param, f64 density),
                                f64 (*U_intM)(const void *param, f64 density), const void *param) {
  BDG_REQUIRE(bdg, BDG_HAS_WF, "bdg_set_local_interactions");
  BDG_FORBID(bdg, BDG_HAS_INTERACTIONS, "bdg_set_local_interactions");
  matmul_ctx_t *ctx = bdg->ctx;
  for (uint64_t i = 0; i < ctx->size; i++) {
    f64 n;
    if (bdg->complex_psi0) {
      const c64 p = ((const c64 *)ctx->wf)[i];
      n = creal(p) * creal(p) + cimag(p) * cimag(p);
    } else {
      const f64 p = ((const f64 *)ctx->wf)[i];
      n = p * p;
    }
    const f64 uK = U_intK(param, n);
    const f64 uM = U_intM(param, n);
    ctx->localTermK[i] += uK;
    ctx->localTermM[i] += uK + 2.0 * uM;
  }
  bdg->state |= BDG_HAS_INTERACTIONS;
}

void bdg_set_mu(bdg_t *bdg, f64 mu) {
  BDG_REQUIRE(bdg, BDG_HAS_SYSTEM, "bdg_set_mu");
  matmul_ctx_t *ctx = bdg->ctx;
  if (ctx->precond_sqrtK == NULL) ctx->precond_sqrtK = xcalloc(ctx->size, sizeof(f64));
  if (ctx->precond_sqrtM == NULL) ctx->precond_sqrtM = xcalloc(ctx->size, sizeof(f64));
  /* preconditioner scalings from the local terms before mu is subtracted
   * (reference setup.c:161-168) */
  for (uint64_t i = 0; i < ctx->size; i++) {
    ctx->precond_sqrtK[i] = 1.0 / sqrt(fmax(1e-8, ctx->localTermK[i]));
    ctx->precond_sqrtM[i] = 1.0 / sqrt(fmax(1e-8, ctx->localTermM[i]));
  }
  for (uint64_t i = 0; i < ctx->size; i++) {
    ctx->localTermK[i] -= mu;
    ctx->localTermM[i] -= mu;
  }
  ctx->mu = mu;
  bdg->state |= BDG_HAS_MU;
}

void bdg_set_dipolar(bdg_t *bdg, f64 g_ddi, const f64 *dipole_dir, f64 cutoff_radius) {
  BDG_REQUIRE(bdg, BDG_HAS_WF, "bdg_set_dipolar");
  BDG_FORBID(bdg, BDG_HAS_MU, "bdg_set_dipolar");
  matmul_ctx_t *ctx = bdg->ctx;
  if (ctx->dim != 3)
    BDG_ERROR("bdg_set_dipolar: dipolar interactions require dim == 3 (got %" PRIu64 ")", ctx->dim);
  dipolar_set_kernel(ctx, g_ddi, dipole_dir, cutoff_radius);
  dipolar_add_meanfield(ctx);
  ctx->dipolar = 1;
  bdg->state |= BDG_HAS_DIPOLAR;
}

/* ---- warm start (reference src/bdg.c:112-207) ------------------------------ */
static void box_muller(uint32_t *seed, f64 *z0, f64 *z1) {
  f64 u1 = xrand(seed);
  f64 u2 = xrand(seed);
  u1 = fmax(u1, 1e-10);
  const f64 rad = sqrt(-2.0 * log(u1));
  *z0 = rad * cos(2.0 * M_PI * u2);
  *z1 = rad * sin(2.0 * M_PI * u2);
}

int bdg_reuse_modes(bdg_t *bdg, f64 noise_frac) {
  if (bdg->modes_u == NULL || bdg->modes_v == NULL) return -3;
  const uint64_t size = bdg->ctx->size, n = 2 * size, nev = bdg->nev, m = bdg->sizeSub;
  const int cplx = bdg->complex_psi0;
  safe_free(&bdg->reuse_buf);
  bdg->reuse_buf = xcalloc(n * m, cplx ? sizeof(c64) : sizeof(f64));
  bdg->reuse_n = n;
  bdg->reuse_cols = m;
  uint32_t seed = 12345;
  for (uint64_t j = 0; j < nev && j < m; j++) {
    f64 nrm = 0.0;
    for (uint64_t i = 0; i < size; i++) {
      if (cplx) {
        const f64 a = cabs(((const c64 *)bdg->modes_u)[j * size + i]);
        const f64 b = cabs(((const c64 *)bdg->modes_v)[j * size + i]);
        nrm += a * a;
        nrm += b * b;
      } else {
        const f64 a = ((const f64 *)bdg->modes_u)[j * size + i];
        const f64 b = ((const f64 *)bdg->modes_v)[j * size + i];
        nrm += a * a;
        nrm += b * b;
      }
    }
    const f64 sigma = noise_frac * sqrt(nrm);
    for (uint64_t i = 0; i < size; i++) {
      f64 z0, z1;
      box_muller(&seed, &z0, &z1);
      if (cplx) {
        c64 *buf = (c64 *)bdg->reuse_buf;
        buf[i + j * n] = ((const c64 *)bdg->modes_u)[j * size + i] + sigma * z0;
        buf[i + size + j * n] = ((const c64 *)bdg->modes_v)[j * size + i] + sigma * z1;
      } else {
        f64 *buf = (f64 *)bdg->reuse_buf;
        buf[i + j * n] = ((const f64 *)bdg->modes_u)[j * size + i] + sigma * z0;
        buf[i + size + j * n] = ((const f64 *)bdg->modes_v)[j * size + i] + sigma * z1;
      }
    }
  }
  for (uint64_t j = nev; j < m; j++) {
    for (uint64_t i = 0; i < size; i++) {
      f64 z0, z1;
      box_muller(&seed, &z0, &z1);
      f64 w = 1.0;
      if (bdg->ctx->wf) w = cplx ? cabs(((const c64 *)bdg->ctx->wf)[i]) : fabs(((const f64 *)bdg->ctx->wf)[i]);
      const f64 val = fabs(z0) * w;
      if (cplx) {
        ((c64 *)bdg->reuse_buf)[i + j * n] = val;
        ((c64 *)bdg->reuse_buf)[i + size + j * n] = val;
      } else {
        ((f64 *)bdg->reuse_buf)[i + j * n] = val;
        ((f64 *)bdg->reuse_buf)[i + size + j * n] = val;
      }
    }
  }
  bdg->init_mode = BDG_INIT_REUSE;
  return 0;
}

/* ---- solve dispatch and results (reference src/bdg.c:212-238) ------------- */
int bdg_solve(bdg_t *bdg) {
  BDG_REQUIRE(bdg, BDG_HAS_SYSTEM, "bdg_solve");
  BDG_REQUIRE(bdg, BDG_HAS_MU, "bdg_solve");
  return bdg->complex_psi0 ? bdg_solve_z(bdg) : bdg_solve_d(bdg);
}

uint64_t bdg_converged(const bdg_t *bdg) { return bdg->converged; }
const f64 *bdg_eigenvalues(const bdg_t *bdg) { return bdg->eigvals; }
const void *bdg_modes_u(const bdg_t *bdg) { return bdg->modes_u; }
const void *bdg_modes_v(const bdg_t *bdg) { return bdg->modes_v; }

/* ---- options without a reference counterpart (bdg/bdg_b200.h) --------------- */
void bdg_set_precision(bdg_t *bdg, int precision) {
  if (precision != BDG_PREC_F64 && precision != BDG_PREC_MIXED)
    BDG_ERROR("bdg_set_precision: unknown precision %d", precision);
  bdg->precision = precision;
}

void bdg_set_convergence(bdg_t *bdg, int criterion) {
  if (criterion != BDG_CONV_BACKWARD && criterion != BDG_CONV_TRUE_RESIDUAL)
    BDG_ERROR("bdg_set_convergence: unknown criterion %d", criterion);
  bdg->criterion = criterion;
}

void bdg_set_goldstone_deflation(bdg_t *bdg, int enable) { bdg->deflate = enable ? 1 : 0; }

void bdg_set_refinement(bdg_t *bdg, int max_iters) { bdg->refine_iters = max_iters < 0 ? 0 : max_iters; }

const bdg_solve_stats_t *bdg_solve_stats(const bdg_t *bdg) { return &bdg->stats; }

/* ---- learned preconditioner and residual harvesting (bdg/bdg_learn.h) ---- */
int bdg_set_learned_precond(bdg_t *bdg, bdg_lp *lp, int stall_window) {
  if (bdg == NULL) return -1;
  if (bdg->complex_psi0 && lp != NULL) {
    fprintf(stderr, "bdg_set_learned_precond: the learned preconditioner is for real (_d) problems\n");
    return -2;
  }
  bdg->learned = lp;
  bdg->learned_stall = stall_window > 0 ? stall_window : 12;
  bdg->learned_fallback = -1;
  return 0;
}

int64_t bdg_learned_fallback_iteration(const bdg_t *bdg) { return bdg ? bdg->learned_fallback : -1; }

int bdg_set_residual_harvest(bdg_t *bdg, double *d_buf, uint64_t cap_cols) {
  if (bdg == NULL) return -1;
  bdg->harvest = d_buf;
  bdg->harvest_cap = d_buf ? cap_cols : 0;
  bdg->harvest_n = 0;
  return 0;
}

uint64_t bdg_residual_harvest_count(const bdg_t *bdg) { return bdg ? bdg->harvest_n : 0; }

bdgd_ctx *bdg_device_context(bdg_t *bdg) {
  if (bdg == NULL || bdg->ctx == NULL) return NULL;
  if (bdg_ctx_sync_device(bdg->ctx, BDGD_OP_LREP) || bdg_ctx_sync_device(bdg->ctx, BDGD_OP_TLREP)) return NULL;
  return bdg->ctx->dev;
}

void bdg_set_trap_grid(bdg_t *bdg, const double *V) {
  BDG_REQUIRE(bdg, BDG_HAS_SYSTEM, "bdg_set_trap_grid");
  if (V == NULL) BDG_ERROR("bdg_set_trap_grid: V is NULL");
  matmul_ctx_t *ctx = bdg->ctx;
  for (uint64_t i = 0; i < ctx->size; i++) {
    ctx->localTermK[i] += V[i];
    ctx->localTermM[i] += V[i];
  }
  bdg->state |= BDG_HAS_TRAP;
}

void bdg_set_local_interactions_grid(bdg_t *bdg, const double *uK, const double *uM) {
  BDG_REQUIRE(bdg, BDG_HAS_WF, "bdg_set_local_interactions_grid");
  BDG_FORBID(bdg, BDG_HAS_INTERACTIONS, "bdg_set_local_interactions_grid");
  if (uK == NULL || uM == NULL) BDG_ERROR("bdg_set_local_interactions_grid: NULL array");
  matmul_ctx_t *ctx = bdg->ctx;
  for (uint64_t i = 0; i < ctx->size; i++) {
    ctx->localTermK[i] += uK[i];
    ctx->localTermM[i] += uK[i] + 2.0 * uM[i];
  }
  bdg->state |= BDG_HAS_INTERACTIONS;
}

/* ---- ground-state producer (no reference counterpart) ---------------------- */
int bdg_ground_state(uint64_t dim, const uint64_t *N, const double *L, const double *V, double g, double g_ddi,
                     const double *dipole_dir, double cutoff_radius, double dt, double tol, uint64_t max_steps,
                     int newton_steps, double *psi_inout, double *mu_out, uint64_t *steps_out,
                     double *stationarity_out) {
  matmul_ctx_t *ctx = matmul_ctx_alloc(dim, N, L);
  matmul_ctx_set_system(ctx, 0);
  if (g_ddi != 0.0 && dim == 3) dipolar_set_kernel(ctx, g_ddi, dipole_dir, cutoff_radius);
  int rc = bdg_ctx_sync_device(ctx, BDGD_OP_KINETIC);
  if (!rc && ctx->longRngInt) rc = bdgd_set_dipolar(ctx->dev, ctx->longRngInt, g_ddi, 1);
  int steps = 0;
  if (!rc)
    rc = bdgd_ground_state(ctx->dev, V, g, dt, tol, (int)max_steps, newton_steps, psi_inout, mu_out, &steps,
                           stationarity_out);
  if (rc) fprintf(stderr, "bdg_ground_state: %s\n", bdgd_last_error());
  if (steps_out) *steps_out = (uint64_t)steps;
  matmul_ctx_free(&ctx);
  return rc;
}
