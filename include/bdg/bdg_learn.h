/* bdg_learn.h -- learned SPD preconditioner for the BdG solver (B200).
 *
 * No counterpart in the reference: pstuermer/BDG_LOBPCG preconditions with
 * the diagonal k-space operator of src/precond_impl.inc:21-118 only.  This
 * component replaces it, optionally, by
 *
 *     T = S^T S + exp(eta) P0          (one network per half, K and M)
 *
 * where P0 is that plain preconditioner and S is a linear map of the
 * residual onto 16 channels on the 2x coarsened grid: 2x2x2 average pooling,
 * a lift conditioned on psi0, the trap, eps_dd and lambda, and 4 residual
 * layers z <- z + SC(z) + PM(z) (SC a spectral convolution over the lowest
 * 12 wave numbers per axis with an even filter, PM a pointwise channel mix
 * with a conditioned diagonal).  T is symmetric positive definite by
 * construction.  Weights are FP32; the network runs in FP32 on the GPU.
 *
 * Training minimises ||T r - e||^2 / ||e||^2 over (residual, correction)
 * pairs: r are residual columns harvested from solves
 * (bdg_set_residual_harvest), e = (K + sigma)^-1 r or (M + sigma)^-1 r from
 * an inner conjugate-gradient solve (bdg_lp_cg).  Forward, adjoint,
 * gradient and Adam kernels are the library's own (bdg_learn.cu).
 *
 * In bdg_solve (bdg_set_learned_precond) the solver falls back to the plain
 * preconditioner when the worst wanted residual stalls.
 */
#ifndef BDG_LEARN_H
#define BDG_LEARN_H

#include <stdint.h>

#include "bdg/bdg.h"
#include "bdg/bdg_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bdg_lp bdg_lp;

enum { BDG_LP_HALF_K = 0, BDG_LP_HALF_M = 1 };

/* Create a preconditioner for the fine 3D grid N (even extents >= 8) with
 * channels C (1, 2, 4, 8 or 16), layers L and retained wave numbers `modes`
 * per axis (modes <= N/4).  Parameters start at the plain preconditioner (S = 0, eta = 0).
 * Returns 0 or a BDGD_ERR_* code (bdgd_last_error explains). */
int bdg_lp_create(bdg_lp **out, const uint64_t N[3], int C, int L, int modes);
void bdg_lp_free(bdg_lp **lp);

/* Parameter vector of one half (FP32, count bdg_lp_nparams): the lift A
 * [C][5], then per layer the filters W [L][C][modes]^3, the mixes B [L][C][C],
 * the conditioned diagonals Dg [L][C][5], and eta. */
uint64_t bdg_lp_nparams(const bdg_lp *lp);
int bdg_lp_get_params(const bdg_lp *lp, int half, float *host_out);
int bdg_lp_set_params(bdg_lp *lp, int half, const float *host_in);

/* Random initial lift weights (scale `amp`, seed) for both halves; the rest
 * stays zero.  Resets the Adam state. */
int bdg_lp_init_random(bdg_lp *lp, double amp, uint64_t seed);

/* Binary save / load of both halves' parameters (and the shape, checked on
 * load against C, L and modes; the grid may differ). */
int bdg_lp_save(const bdg_lp *lp, const char *path);
int bdg_lp_load(bdg_lp *lp, const char *path);

/* Conditioning of the problem the preconditioner is used on: psi0 (real,
 * fine grid), the trap potential V (fine grid), eps_dd and the trap aspect
 * lambda.  Must precede apply and training steps. */
int bdg_lp_condition(bdg_lp *lp, const double *psi0, const double *V, double eps_dd, double lambda);

/* Move the preconditioner to another fine grid (same C, L, modes): keeps the
 * parameters, drops the conditioning. */
int bdg_lp_regrid(bdg_lp *lp, const uint64_t N[3]);

/* y <- exp(eta_h) y + S_h^T S_h x for ncol columns of one half h; x and y
 * device columns of length N0 N1 N2 (FP64 if prec == BDGD_F64, else FP32),
 * y holding P0 x on entry.  Work is queued on the stream of dev. */
int bdg_lp_apply_half(bdg_lp *lp, bdgd_ctx *dev, int half, int prec, const void *d_x, uint64_t ldx, void *d_y,
                      uint64_t ldy, uint64_t ncol);

/* Applies run the basis contractions of the spectral convolutions as TF32
 * tensor-core GEMMs (on = 1, the default; about 1e-3 relative error, ample
 * for a preconditioner) or in exact FP32 (on = 0).  Training steps are
 * always exact FP32. */
int bdg_lp_set_fast_math(bdg_lp *lp, int on);

/* Full T on [u; v] columns: y = T x with P0 = the plain T_Lrep of dev. */
int bdg_lp_apply(bdg_lp *lp, bdgd_ctx *dev, int prec, const void *d_x, uint64_t ldx, void *d_y, uint64_t ldy,
                 uint64_t ncol);

/* Loss and gradient of one half on ncol pairs (device FP64 columns r, e,
 * P0 r, leading dimension ld): loss_out = mean ||T r - e||^2 / ||e||^2,
 * grad_out (host, nparams floats, may be NULL) the gradient of that mean. */
int bdg_lp_loss_grad(bdg_lp *lp, bdgd_ctx *dev, int half, const double *d_r, const double *d_e,
                     const double *d_p0r, uint64_t ld, uint64_t ncol, double *loss_out, float *grad_out);

/* Loss of bdg_lp_loss_grad / bdg_lp_train_step: sigma < 0 selects the L2
 * loss above (the default); sigma >= 0 the energy norm
 * ||T r - e||_A^2 / ||e||_A^2 of A = Op + sigma (Op = K for half 0, M for
 * half 1, applied through the dev passed to those calls), which needs
 * e = A^-1 r only in <r, e>. */
int bdg_lp_set_energy_loss(bdg_lp *lp, double sigma);

/* One Adam step (lr; beta1 0.9, beta2 0.999, eps 1e-8) of one half on ncol
 * pairs; loss_out (may be NULL) receives the loss before the step. */
int bdg_lp_train_step(bdg_lp *lp, bdgd_ctx *dev, int half, const double *d_r, const double *d_e,
                      const double *d_p0r, uint64_t ld, uint64_t ncol, double lr, double *loss_out);

/* Inner conjugate gradients for training targets: e = (Op + sigma)^-1 r
 * for ncol device FP64 columns of one half (Op = BDGD_OP_K or BDGD_OP_M of
 * dev, which must be SPD after the shift), to relative residual tol or
 * maxit iterations.  iters_out (may be NULL): iterations run. */
int bdg_lp_cg(bdgd_ctx *dev, int op, double sigma, const double *d_r, double *d_e, uint64_t ld, uint64_t ncol,
              double tol, int maxit, int *iters_out);

/* Solver hooks (bdg_t of bdg.h). */
/* Use lp as the preconditioner of bdg_solve (NULL: plain).  lp must be
 * conditioned on the same problem; the solver falls back to the plain
 * preconditioner for the rest of a solve when the worst backward error of the
 * wanted pairs is not finite or has not fallen by 10% over `stall_window`
 * iterations (0: 12). */
int bdg_set_learned_precond(bdg_t *bdg, bdg_lp *lp, int stall_window);
/* Iteration at which the last solve fell back to the plain preconditioner,
 * or -1. */
int64_t bdg_learned_fallback_iteration(const bdg_t *bdg);
/* Copy residual columns (FP64 [u; v], length 2 N0 N1 N2 each) of FP64
 * solves into d_buf until cap_cols columns are stored. */
int bdg_set_residual_harvest(bdg_t *bdg, double *d_buf, uint64_t cap_cols);
uint64_t bdg_residual_harvest_count(const bdg_t *bdg);
/* The device context of a set-up problem (operator fields uploaded), for
 * bdg_lp_cg and P0 applies on its grid; owned by bdg.  NULL on failure. */
bdgd_ctx *bdg_device_context(bdg_t *bdg);

#ifdef __cplusplus
}
#endif

#endif
