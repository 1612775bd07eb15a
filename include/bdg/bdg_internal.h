/*
 * bdg_internal.h -- library-internal ABI of the B200 BdG library.
 *
 * Mirrors the internal ABI of pstuermer/BDG_LOBPCG that its unit tests link
 * against (src/bdg_internal.h:71-222 of that project): the matmul_ctx_t and
 * bdg_t structs keep the reference's field names, order and meaning (tests
 * allocate and poke ctx fields directly), and the single-column operator
 * entry points keep their signatures.  Those entry points take HOST pointers
 * for one column, as the reference's do; each call copies the context's
 * arrays and the column to the GPU, applies the operator there and copies
 * the result back.  The block/device entry points in bdg/bdg_cuda.h are the
 * fast path.
 *
 * Differences in layout, all appended after the reference fields:
 *   - fwd_plan / bwd_plan are opaque handles of the GPU FFT plan (the
 *     reference holds FFTW plans);
 *   - matmul_ctx_t gains `dev` (the device-side context, created lazily on
 *     the first GPU use) and `prec` (operator precision);
 *   - bdg_t gains the solver options of bdg/bdg_b200.h and solve statistics.
 */
#ifndef BDG_INTERNAL_H
#define BDG_INTERNAL_H

#include "bdg/bdg.h"
#include "bdg/bdg_b200.h"
#include "bdg/memory.h"
#include "lobpcg/types.h"
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- setup state bits (reference src/bdg_internal.h:25-32) -------------- */
enum {
  BDG_HAS_SYSTEM = 1u << 0,
  BDG_HAS_TRAP = 1u << 1,
  BDG_HAS_WF = 1u << 2,
  BDG_HAS_INTERACTIONS = 1u << 3,
  BDG_HAS_DIPOLAR = 1u << 4,
  BDG_HAS_MU = 1u << 5
};

/* Fatal setup-order errors print and exit(EXIT_FAILURE), as the reference's
 * BDG_ERROR does (src/bdg_log.h:29-37); tests rely on the exit status. */
void bdg_fatal(const char *file, int line, const char *fmt, ...);
void bdg_warn(const char *file, int line, const char *fmt, ...);
#define BDG_ERROR(...) bdg_fatal(__FILE__, __LINE__, __VA_ARGS__)
#define BDG_WARN(...) bdg_warn(__FILE__, __LINE__, __VA_ARGS__)

#define BDG_REQUIRE(bdg, flag, caller)                                        \
  do {                                                                        \
    if (0 == ((bdg)->state & (flag)))                                         \
      BDG_ERROR("%s: prerequisite %s not satisfied", caller, #flag);          \
  } while (0)

#define BDG_FORBID(bdg, flag, caller)                                         \
  do {                                                                        \
    if (0 != ((bdg)->state & (flag)))                                         \
      BDG_ERROR("%s: %s already set (double-call forbidden)", caller, #flag); \
  } while (0)

/* |x| < 1e-8 clamps to 1e-8 (reference src/bdg_internal.h:47-50). */
static inline f64 safe_val(f64 x) { return (fabs(x) < 1e-8) ? 1e-8 : x; }

/* xorshift32 and its (0,1] uniform (reference src/bdg_internal.h:52-65). */
static inline uint32_t xorshift32(uint32_t *state) {
  uint32_t x = *state;
  x ^= x << 13;
  x ^= x >> 17;
  x ^= x << 5;
  *state = x;
  return x;
}

static inline f64 xrand(uint32_t *state) {
  return (f64)(xorshift32(state) & 0x7FFFFFFF) / (f64)0x7FFFFFFF;
}

struct bdgd_ctx;

/* Operator context (reference src/bdg_internal.h:71-115, same fields). */
typedef struct {
  uint64_t dim;
  uint64_t *N;
  f64 *L;
  uint64_t size;
  uint64_t k_size;

  f64 *k2;
  f64 **kx2;

  f64 *localTermK;
  f64 *localTermM;
  f64 *longRngInt;
  f64 g_ddi;
  f64 mu;
  unsigned int dipolar;

  void *wf;
  uint64_t wf_size;

  void *fwd_plan; /* GPU FFT plan handle (forward) */
  void *bwd_plan; /* GPU FFT plan handle (backward) */

  /* Host scratch of the reference's shapes: f_wrk c64[k_size],
   * c_wrk1/c_wrk2 max(size, k_size) c64.  Kept so code that indexes them
   * keeps working; the operators use device scratch. */
  void *f_wrk;
  void *c_wrk1;
  void *c_wrk2;

  f64 *precond_sqrtK;
  f64 *precond_sqrtM;

  int complex_psi0;

  /* ---- appended ---- */
  struct bdgd_ctx *dev; /* device context, created on first GPU use */
  int prec;             /* BDG_PREC_F64 or BDG_PREC_MIXED */
} matmul_ctx_t;

/* Problem handle (reference src/bdg_internal.h:121-145, same fields). */
struct bdg_t {
  matmul_ctx_t *ctx;
  uint32_t state;

  uint64_t nev;
  uint64_t sizeSub;
  uint64_t maxIter;
  f64 tol;
  int complex_psi0;

  f64 *eigvals;
  void *modes_u;
  void *modes_v;
  uint64_t converged;

  bdg_init_mode_t init_mode;
  bdg_init_fn custom_init_fn;
  void *custom_init_param;
  void *reuse_buf;
  uint64_t reuse_n;
  uint64_t reuse_cols;

  /* ---- appended (bdg/bdg_b200.h options and statistics) ---- */
  int precision;       /* BDG_PREC_F64 (default) or BDG_PREC_MIXED */
  int criterion;       /* BDG_CONV_BACKWARD (default) or BDG_CONV_TRUE_RESIDUAL */
  int deflate;         /* Goldstone deflation on/off (default off) */
  int refine_iters;    /* FP64 refinement iterations after a mixed solve */
  bdg_solve_stats_t stats;
  void *solver_ws;     /* cached device workspace of the GPU solver */
  void *block;         /* last solver block (host, n x sizeSub) */
  /* learned preconditioner (bdg/bdg_learn.h) and residual harvesting */
  void *learned;            /* struct bdg_lp *, or NULL for the plain preconditioner */
  int learned_stall;        /* stall window (iterations) before the fallback */
  int64_t learned_fallback; /* iteration of the last fallback, or -1 */
  double *harvest;          /* device buffer of residual columns, or NULL */
  uint64_t harvest_cap, harvest_n;
  int block_ws;             /* workspace holding the last solve's block (0/1), or -1 */
  size_t modes_bytes;       /* allocation size of modes_u / modes_v (reused across solves) */
  const void *init_block;   /* caller's initial block (bdg_set_initial_block), borrowed */
  uint64_t init_block_n, init_block_m;
};

/* ---- context lifecycle (reference src/bdg_internal.h:151-153) ------------ */
matmul_ctx_t *matmul_ctx_alloc(uint64_t dim, const uint64_t *N, const f64 *L);
void matmul_ctx_free(matmul_ctx_t **ctx);
void matmul_ctx_set_system(matmul_ctx_t *ctx, int complex_psi0);

/* ---- single-column operators on host pointers (reference :159-207) ------- */
void kinetic_d(matmul_ctx_t *ctx, const f64 *x, f64 *y);
void matmulK_d(matmul_ctx_t *ctx, const f64 *x, f64 *y);
void matmulM_d(matmul_ctx_t *ctx, const f64 *x, f64 *y);
void matmulLrep_d(matmul_ctx_t *ctx, const f64 *x, f64 *y);
void matmulSwap_d(matmul_ctx_t *ctx, const f64 *x, f64 *y);
void precondK_d(matmul_ctx_t *ctx, const f64 *x, f64 *y);
void precondM_d(matmul_ctx_t *ctx, const f64 *x, f64 *y);
void precondLrep_d(matmul_ctx_t *ctx, const f64 *x, f64 *y);
void dipolar_conv_d(matmul_ctx_t *ctx, const f64 *v, f64 *out);
#ifndef __cplusplus
void kinetic_z(matmul_ctx_t *ctx, const c64 *x, c64 *y);
void matmulK_z(matmul_ctx_t *ctx, const c64 *x, c64 *y);
void matmulM_z(matmul_ctx_t *ctx, const c64 *x, c64 *y);
void matmulLrep_z(matmul_ctx_t *ctx, const c64 *x, c64 *y);
void matmulSwap_z(matmul_ctx_t *ctx, const c64 *x, c64 *y);
void precondK_z(matmul_ctx_t *ctx, const c64 *x, c64 *y);
void precondM_z(matmul_ctx_t *ctx, const c64 *x, c64 *y);
void precondLrep_z(matmul_ctx_t *ctx, const c64 *x, c64 *y);
void dipolar_conv_z(matmul_ctx_t *ctx, const c64 *v, c64 *out);
#endif

/* ---- dipolar (reference :213-224) ---------------------------------------- */
void dipolar_set_kernel(matmul_ctx_t *ctx, f64 g_ddi, const f64 *dipole_dir,
                        f64 cutoff_radius);
void dipolar_add_meanfield(matmul_ctx_t *ctx);
void dipolar_add_meanfield_d(matmul_ctx_t *ctx);
void dipolar_add_meanfield_z(matmul_ctx_t *ctx);

/* Run a plan handle of ctx->fwd_plan / ctx->bwd_plan on host arrays (the
 * counterpart of the reference tests' fftw_execute_dft{,_r2c,_c2r} on those
 * fields, tests/test_setup.c:192-286): unnormalised, FFTW layout.  Returns 0
 * or a negative device error. */
int bdg_fft_execute(void *plan, const void *in, void *out);

/* FFTW names for code that runs ctx->fwd_plan / ctx->bwd_plan through the
 * FFTW execute calls, as the reference's tests do (tests/test_setup.c:208-271
 * calls fftw_execute_dft{,_r2c,_c2r} on those fields): the three calls map
 * onto bdg_fft_execute, so such code compiles unchanged against this header.
 * Macros rather than exported functions, so the library exports no FFTW
 * symbol; skipped when the real fftw3.h came first (its FFTW3_H guard) or
 * with BDG_NO_FFTW_COMPAT. */
#if !defined(FFTW3_H) && !defined(BDG_NO_FFTW_COMPAT)
typedef double fftw_complex[2];
typedef void *fftw_plan;
#define fftw_execute_dft(p, in, out) ((void)bdg_fft_execute((p), (in), (out)))
#define fftw_execute_dft_r2c(p, in, out) ((void)bdg_fft_execute((p), (in), (out)))
#define fftw_execute_dft_c2r(p, in, out) ((void)bdg_fft_execute((p), (in), (out)))
#endif

/* ---- solver (reference :220-221) ----------------------------------------- */
int bdg_solve_d(bdg_t *bdg);
int bdg_solve_z(bdg_t *bdg);

/* ---- helpers shared by the host C files ---------------------------------- */
/* Create ctx->dev if needed and upload every ctx array the operator `op`
 * reads (the host arrays may have been replaced by the caller since the last
 * call).  Returns 0 or a negative error. */
int bdg_ctx_sync_device(matmul_ctx_t *ctx, int op);
/* Run `op` on ncol host columns through the device (synchronous). */
void bdg_ctx_apply_host(matmul_ctx_t *ctx, int op, const void *x, void *y,
                        uint64_t ncol, const char *caller);
/* Fill the initial block S (n x sizeSub, host) per bdg->init_mode. */
void bdg_fill_initial_block(bdg_t *bdg, void *S);
/* The same block generated on the device into d_S (n x sizeSub, leading dim
 * n; FP64 or FP32 per prec, complex on the _z path): 0 when filled, 1 when
 * the mode needs the host fill (CUSTOM, or REUSE with a stored buffer), < 0
 * on a device error.  The wavefunction must be on the device
 * (bdg_device_context). */
int bdg_fill_initial_block_device(bdg_t *bdg, void *d_S, int prec);

#ifdef __cplusplus
}
#endif

#endif /* BDG_INTERNAL_H */
