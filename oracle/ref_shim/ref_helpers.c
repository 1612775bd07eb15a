/*
 * ref_helpers.c -- field access into the reference's own structs for the
 * oracle build (compiled against pstuermer/BDG_LOBPCG src/bdg_internal.h).
 *
 * TEST INFRASTRUCTURE ONLY.  The Python binding (oracle/ref.py) reaches the
 * reference's matmul_ctx_t fields through these accessors, the way the
 * reference's unit tests poke them (e.g. tests/test_matmulM.c:166-186); the
 * shim's iLOBPCG reads psi0 and the operator-norm bound through them.
 */
#include "bdg_internal.h"

#include <complex.h>
#include <math.h>
#include <string.h>

const void *ref_helper_wf(void *vctx) { return ((matmul_ctx_t *)vctx)->wf; }

/* Upper bound of ||A|| = max(||K||, ||M||): max kinetic energy of the grid
 * plus the largest local term (plus the dipolar exchange bound), the scale
 * of the backward-error convergence test (oracle/bdg_oracle.py:anorm_estimate). */
double ref_helper_anorm(void *vctx) {
  const matmul_ctx_t *ctx = (const matmul_ctx_t *)vctx;
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

matmul_ctx_t *ref_helper_ctx(bdg_t *bdg) { return bdg->ctx; }

/* Address of an array field of ctx (NULL if unknown or unset). */
void *ref_helper_field(matmul_ctx_t *ctx, const char *name) {
  if (!strcmp(name, "k2")) return ctx->k2;
  if (!strcmp(name, "localTermK")) return ctx->localTermK;
  if (!strcmp(name, "localTermM")) return ctx->localTermM;
  if (!strcmp(name, "longRngInt")) return ctx->longRngInt;
  if (!strcmp(name, "wf")) return ctx->wf;
  if (!strcmp(name, "precond_sqrtK")) return ctx->precond_sqrtK;
  if (!strcmp(name, "precond_sqrtM")) return ctx->precond_sqrtM;
  if (!strncmp(name, "kx2_", 4)) {
    const int d = name[4] - '0';
    return (ctx->kx2 && d >= 0 && (uint64_t)d < ctx->dim) ? ctx->kx2[d] : NULL;
  }
  return NULL;
}

/* Allocate (zeroed, replacing any previous) an array field that the setup
 * path allocates lazily (wf, longRngInt, precond_sqrtK/M); returns it. */
void *ref_helper_alloc(matmul_ctx_t *ctx, const char *name, uint64_t count, uint64_t elem) {
  void **slot = NULL;
  if (!strcmp(name, "wf")) slot = &ctx->wf;
  else if (!strcmp(name, "longRngInt")) slot = (void **)&ctx->longRngInt;
  else if (!strcmp(name, "precond_sqrtK")) slot = (void **)&ctx->precond_sqrtK;
  else if (!strcmp(name, "precond_sqrtM")) slot = (void **)&ctx->precond_sqrtM;
  if (!slot) return NULL;
  safe_free(slot);
  *slot = xcalloc(count, elem);
  if (!strcmp(name, "wf")) ctx->wf_size = count;
  return *slot;
}

double ref_helper_get(const matmul_ctx_t *ctx, const char *name) {
  if (!strcmp(name, "mu")) return ctx->mu;
  if (!strcmp(name, "g_ddi")) return ctx->g_ddi;
  if (!strcmp(name, "dipolar")) return (double)ctx->dipolar;
  if (!strcmp(name, "size")) return (double)ctx->size;
  if (!strcmp(name, "k_size")) return (double)ctx->k_size;
  if (!strcmp(name, "complex_psi0")) return (double)ctx->complex_psi0;
  return NAN;
}

void ref_helper_set(matmul_ctx_t *ctx, const char *name, double v) {
  if (!strcmp(name, "mu")) ctx->mu = v;
  else if (!strcmp(name, "g_ddi")) ctx->g_ddi = v;
  else if (!strcmp(name, "dipolar")) ctx->dipolar = (unsigned)v;
}

uint64_t ref_helper_bdg_state(const bdg_t *bdg) { return bdg->state; }

/* ---- C callbacks for the reference's setup API ------------------------------ */
/* Trap from a table: the reference visits the grid in index order
 * (src/setup.c:17-84, idx = (iz * Ny + iy) * Nx + ix), so the callback
 * returns the table's entries one after another. */
typedef struct {
  const double *V;
  uint64_t next;
} ref_trap_table_t;

f64 ref_cb_trap_table(uint64_t dim, const f64 *r, const void *param) {
  (void)dim;
  (void)r;
  ref_trap_table_t *t = (ref_trap_table_t *)param;
  return t->V[t->next++];
}

/* contact interaction U(n) = g n, param -> g */
f64 ref_cb_contact(const void *param, f64 density) { return *(const double *)param * density; }

/* BDG_INIT_CUSTOM callback copying a prepared n x sizeSub block (param) */
void ref_cb_init_copy(const bdg_t *bdg, void *X, uint64_t n, uint64_t sizeSub, void *param) {
  const size_t esz = bdg->complex_psi0 ? sizeof(c64) : sizeof(f64);
  memcpy(X, param, n * sizeSub * esz);
}
