/*
 * bdg_init.c -- initial iLOBPCG block per init mode, host side.
 *
 * Same modes, seeds and formulas as the reference's solver adapter
 * (pstuermer/BDG_LOBPCG src/solver.c:68-259 real path, :321-414 complex):
 *   PLANEWAVE    cos/sin pairs of the lowest-|k|^2 plane waves (per geometry
 *                hint) times |psi0| plus 1e-4 xorshift noise, u = v;
 *   WF_WEIGHTED  |gaussian| * |psi0|, u = v (real path seeded by time() via
 *                rand_r as in the reference, complex path xorshift seed 42);
 *   REUSE        buffer from bdg_reuse_modes when its shape matches, else
 *                falls through to WF_WEIGHTED;
 *   CUSTOM       the user callback.
 * The block is n x sizeSub column-major, n = 2*size.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "bdg/bdg_cuda.h"
#include "bdg/bdg_internal.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

typedef struct {
  f64 k2;
  uint64_t idx[3];
} kvec_t;

static int kvec_cmp(const void *a, const void *b) {
  const f64 x = ((const kvec_t *)a)->k2, y = ((const kvec_t *)b)->k2;
  return (x > y) - (x < y);
}

/* lowest |k|^2 wave vectors within the hinted ranges (reference :76-129) */
static kvec_t *enumerate_kvecs(const matmul_ctx_t *ctx, bdg_geom_hint_t hint, uint64_t need, uint64_t *n_out) {
  const uint64_t dim = ctx->dim;
  uint64_t range[3] = {1, 1, 1};
  if (hint == BDG_GEOM_ELONGATED) {
    uint64_t ld = 0;
    for (uint64_t d = 1; d < dim; d++)
      if (ctx->L[d] > ctx->L[ld]) ld = d;
    range[ld] = ctx->N[ld] < 2 * need ? ctx->N[ld] : 2 * need;
  } else if (hint == BDG_GEOM_RING) {
    for (uint64_t d = 0; d < dim && d < 2; d++) range[d] = ctx->N[d] < 2 * need ? ctx->N[d] : 2 * need;
  } else {
    for (uint64_t d = 0; d < dim; d++) range[d] = ctx->N[d] < 2 * need ? ctx->N[d] : 2 * need;
  }
  const uint64_t total = range[0] * range[1] * range[2];
  kvec_t *e = xcalloc(total, sizeof(kvec_t));
  uint64_t c = 0;
  for (uint64_t iz = 0; iz < range[2]; iz++) {
    const f64 kz2 = dim > 2 ? ctx->kx2[2][iz] : 0.0;
    for (uint64_t iy = 0; iy < range[1]; iy++) {
      const f64 ky2 = dim > 1 ? ctx->kx2[1][iy] : 0.0;
      for (uint64_t ix = 0; ix < range[0]; ix++) {
        e[c].k2 = ctx->kx2[0][ix] + ky2 + kz2;
        e[c].idx[0] = ix;
        e[c].idx[1] = iy;
        e[c].idx[2] = iz;
        c++;
      }
    }
  }
  qsort(e, c, sizeof(kvec_t), kvec_cmp);
  *n_out = c < need ? c : need;
  return e;
}

static inline f64 wf_abs(const matmul_ctx_t *ctx, int cplx, uint64_t i) {
  if (ctx->wf == NULL) return 1.0;
  return cplx ? cabs(((const c64 *)ctx->wf)[i]) : fabs(((const f64 *)ctx->wf)[i]);
}

static inline void put(void *S, int cplx, uint64_t at, f64 v) {
  if (cplx)
    ((c64 *)S)[at] = v;
  else
    ((f64 *)S)[at] = v;
}

static void fill_wf_weighted(bdg_t *bdg, void *S) {
  const matmul_ctx_t *ctx = bdg->ctx;
  const uint64_t size = ctx->size, n = 2 * size, m = bdg->sizeSub;
  const int cplx = bdg->complex_psi0;
  if (!cplx) {
    /* reference :178-189: rand_r seeded with time(NULL) */
    unsigned int seed = (unsigned int)time(NULL);
    for (uint64_t j = 0; j < m; j++)
      for (uint64_t i = 0; i < size; i++) {
        f64 u1 = (f64)rand_r(&seed) / RAND_MAX;
        f64 u2 = (f64)rand_r(&seed) / RAND_MAX;
        u1 = fmax(u1, 1e-10);
        const f64 v = fabs(sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2)) * wf_abs(ctx, 0, i);
        put(S, 0, i + j * n, v);
        put(S, 0, i + size + j * n, v);
      }
  } else {
    uint32_t seed = 42; /* reference :334 */
    for (uint64_t j = 0; j < m; j++)
      for (uint64_t i = 0; i < size; i++) {
        f64 u1 = xrand(&seed);
        f64 u2 = xrand(&seed);
        u1 = fmax(u1, 1e-10);
        const f64 v = fabs(sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2)) * wf_abs(ctx, 1, i);
        put(S, 1, i + j * n, v);
        put(S, 1, i + size + j * n, v);
      }
  }
}

static void fill_planewave(bdg_t *bdg, void *S) {
  const matmul_ctx_t *ctx = bdg->ctx;
  const uint64_t size = ctx->size, n = 2 * size, m = bdg->sizeSub;
  const int cplx = bdg->complex_psi0;
  uint32_t seed = 42;
  const bdg_geom_hint_t hint =
      bdg->custom_init_param ? (bdg_geom_hint_t)(intptr_t)bdg->custom_init_param : BDG_GEOM_AUTO;
  const uint64_t need = (m + 1) / 2;
  uint64_t nk = 0;
  kvec_t *kv = enumerate_kvecs(ctx, hint, need, &nk);
  for (uint64_t j = 0; j < m; j++) {
    const uint64_t kvi = (j + 1) / 2; /* 0,1,1,2,2,... */
    const int use_sin = (j % 2 == 1);
    if (kvi >= nk) {
      for (uint64_t i = 0; i < size; i++) {
        const f64 v = (xrand(&seed) - 0.5) * wf_abs(ctx, cplx, i);
        put(S, cplx, i + j * n, v);
        put(S, cplx, i + size + j * n, v);
      }
      continue;
    }
    f64 freq[3] = {0.0, 0.0, 0.0};
    for (uint64_t d = 0; d < ctx->dim; d++) {
      const uint64_t kd = kv[kvi].idx[d];
      const int64_t f = kd <= ctx->N[d] / 2 ? (int64_t)kd : (int64_t)kd - (int64_t)ctx->N[d];
      freq[d] = 2.0 * M_PI * (f64)f / ctx->L[d];
    }
    uint64_t stride[3] = {1, 1, 1};
    for (uint64_t d = 1; d < ctx->dim; d++) stride[d] = stride[d - 1] * ctx->N[d - 1];
    for (uint64_t i = 0; i < size; i++) {
      f64 kr = 0.0;
      for (uint64_t d = 0; d < ctx->dim; d++) {
        const uint64_t id = (i / stride[d]) % ctx->N[d];
        kr += freq[d] * ((f64)id * ctx->L[d] / (f64)ctx->N[d]);
      }
      const f64 pw = use_sin ? sin(kr) : cos(kr);
      const f64 pert = 1e-4 * (xrand(&seed) - 0.5);
      const f64 v = (pw + pert) * wf_abs(ctx, cplx, i);
      put(S, cplx, i + j * n, v);
      put(S, cplx, i + size + j * n, v);
    }
  }
  safe_free((void **)&kv);
}

/* The same block generated on the device (bdg_initd.cu): 0 when d_S (n x
 * sizeSub, leading dim n, FP64 or FP32 per prec) was filled, 1 when the
 * mode needs the host fill (CUSTOM, or REUSE with a stored buffer), < 0 on
 * a device error. */
int bdg_fill_initial_block_device(bdg_t *bdg, void *d_S, int prec) {
  matmul_ctx_t *ctx = bdg->ctx;
  if (ctx == NULL || ctx->dev == NULL) return 1;
  const uint64_t n = 2 * ctx->size, m = bdg->sizeSub;
  const int cplx = bdg->complex_psi0;
  if (bdg->init_mode == BDG_INIT_CUSTOM) return 1;
  if (bdg->init_mode == BDG_INIT_REUSE && bdg->reuse_buf && bdg->reuse_n == n && bdg->reuse_cols == m) return 1;
  /* the |psi0| weights: the operators upload psi0 only when the dipolar term
   * needs it, so bring the current one to the device here */
  if (ctx->wf) {
    const int rc = bdgd_set_wavefunction(ctx->dev, ctx->wf);
    if (rc) return rc;
  }
  switch (bdg->init_mode) {
    case BDG_INIT_CUSTOM:
      return 1;
    case BDG_INIT_REUSE:
      if (bdg->reuse_buf && bdg->reuse_n == n && bdg->reuse_cols == m) return 1;
      /* fall through */
    case BDG_INIT_WF_WEIGHTED: {
      uint32_t seed = 42;
      if (!cplx) {
        seed = (uint32_t)time(NULL);
        if (seed == 0) seed = 1;
      }
      return bdgd_init_block(ctx->dev, prec, 1, seed, (int)m, NULL, d_S, n);
    }
    case BDG_INIT_PLANEWAVE:
    default: {
      const bdg_geom_hint_t hint =
          bdg->custom_init_param ? (bdg_geom_hint_t)(intptr_t)bdg->custom_init_param : BDG_GEOM_AUTO;
      uint64_t nk = 0;
      kvec_t *kv = enumerate_kvecs(ctx, hint, (m + 1) / 2, &nk);
      f64 *cols = xcalloc(4 * m, sizeof(f64));
      for (uint64_t j = 0; j < m; j++) {
        const uint64_t kvi = (j + 1) / 2;
        if (kvi >= nk) continue; /* kind 0: noise column */
        cols[4 * j] = (j % 2 == 1) ? 2.0 : 1.0;
        for (uint64_t d = 0; d < ctx->dim; d++) {
          const uint64_t kd = kv[kvi].idx[d];
          const int64_t f = kd <= ctx->N[d] / 2 ? (int64_t)kd : (int64_t)kd - (int64_t)ctx->N[d];
          cols[4 * j + 1 + d] = 2.0 * M_PI * (f64)f / ctx->L[d];
        }
      }
      safe_free((void **)&kv);
      const int rc = bdgd_init_block(ctx->dev, prec, 0, 42u, (int)m, cols, d_S, n);
      free(cols);
      return rc;
    }
  }
}

void bdg_fill_initial_block(bdg_t *bdg, void *S) {
  const uint64_t n = 2 * bdg->ctx->size, m = bdg->sizeSub;
  const size_t esz = bdg->complex_psi0 ? sizeof(c64) : sizeof(f64);
  switch (bdg->init_mode) {
    case BDG_INIT_REUSE:
      if (bdg->reuse_buf && bdg->reuse_n == n && bdg->reuse_cols == m) {
        memcpy(S, bdg->reuse_buf, n * m * esz);
        safe_free(&bdg->reuse_buf);
        bdg->init_mode = BDG_INIT_WF_WEIGHTED;
        return;
      }
      /* fall through */
    case BDG_INIT_WF_WEIGHTED:
      fill_wf_weighted(bdg, S);
      return;
    case BDG_INIT_CUSTOM:
      if (bdg->custom_init_fn) bdg->custom_init_fn(bdg, S, n, m, bdg->custom_init_param);
      return;
    case BDG_INIT_PLANEWAVE:
    default:
      fill_planewave(bdg, S);
      return;
  }
}
