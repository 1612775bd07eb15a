/* bdg_blas.h -- device helpers of the iLOBPCG driver (defined in
 * bdg_blas.cu); internal to the library. */
#ifndef BDG_BLAS_H
#define BDG_BLAS_H

#include <stdint.h>

#include "bdg/bdg_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

/* R = AX - diag(lam) swap(X) (R may be NULL); per-column |R|^2 -> d_rr and
 * |X|^2 -> d_xx.  Blocks of `ncol` columns, leading dimension ld. */
int bdgd_residual(bdgd_ctx *c, int prec, int cplx, uint64_t half, uint64_t ncol, const void *d_X, const void *d_AX,
                  uint64_t ld, void *d_R, uint64_t ldr, const double *d_lam, double *d_work, double *d_rr,
                  double *d_xx, const int *d_colmap);
/* |KMv - lam^2 v|^2 -> d_tt and |v|^2 -> d_vv per column. */
int bdgd_true_residual(bdgd_ctx *c, int prec, int cplx, uint64_t half, uint64_t ncol, const void *d_KMv,
                       uint64_t ldk, const void *d_X, uint64_t ld, const double *d_lam, double *d_work,
                       double *d_tt, double *d_vv);
int bdgd_convert(bdgd_ctx *c, int to_f32, const void *src, void *dst, uint64_t n_scalars);
int bdgd_rr_prepare(bdgd_ctx *c, const double *G, const double *Ga_in, const double *Guv, int k, int ldo, int cplx,
                    double *Gs, double *Gb, double *Ga, double *d);
int bdgd_set_ritz_block(bdgd_ctx *c, double *Ga, double *Guv, int ldo, int m, int cplx, const double *d_lam);
int bdgd_vec_pow(bdgd_ctx *c, const double *in, int n, double e, double *out);
int bdgd_gather_cols(bdgd_ctx *c, const double *In, int ldi, int rows, const int *d_cols, int ncols, int cplx,
                     double *Out, int ldo);
int bdgd_scale_cols(bdgd_ctx *c, const double *In, int rows, int col0, int ncols, int cplx, const double *rowscale,
                    const double *colval, int invsqrt, int reverse, double *Out);
int bdgd_hermitize(bdgd_ctx *c, double *A, int k, int cplx);
int bdgd_clamp(bdgd_ctx *c, double *w, int n, double floor_rel);

#ifdef __cplusplus
}
#endif

#endif
