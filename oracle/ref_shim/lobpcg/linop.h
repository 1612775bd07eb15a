/*
 * lobpcg/linop.h -- linear-operator wrapper of the external "LOBPCG" library,
 * with the ABI its caller implies (pstuermer/BDG_LOBPCG src/solver.c:26-62,
 * :152-157, :280-282): a matvec callback void(const op *, x, y) on one
 * column, a user context { data, data_size } reached as op->ctx->data, and an
 * optional cleanup hook (NULL there, so destroy frees only the wrapper).
 * TEST INFRASTRUCTURE ONLY (oracle build of the reference library).
 */
#ifndef LOBPCG_LINOP_H
#define LOBPCG_LINOP_H
#include <stddef.h>
#include <stdint.h>
#include "lobpcg/types.h"

typedef struct {
  void *data;
  size_t data_size;
} linop_ctx_t;

typedef struct LinearOperator_d_s LinearOperator_d_t;
typedef struct LinearOperator_z_s LinearOperator_z_t;
typedef void (*linop_matvec_d_fn)(const LinearOperator_d_t *op, f64 *restrict x, f64 *restrict y);
typedef void (*linop_matvec_z_fn)(const LinearOperator_z_t *op, c64 *restrict x, c64 *restrict y);
typedef void (*linop_cleanup_fn)(linop_ctx_t *ctx);

struct LinearOperator_d_s {
  uint64_t rows, cols;
  linop_matvec_d_fn matvec;
  linop_cleanup_fn cleanup;
  linop_ctx_t *ctx;
};

struct LinearOperator_z_s {
  uint64_t rows, cols;
  linop_matvec_z_fn matvec;
  linop_cleanup_fn cleanup;
  linop_ctx_t *ctx;
};

LinearOperator_d_t *linop_create_d(uint64_t rows, uint64_t cols, linop_matvec_d_fn matvec,
                                   linop_cleanup_fn cleanup, linop_ctx_t *ctx);
LinearOperator_z_t *linop_create_z(uint64_t rows, uint64_t cols, linop_matvec_z_fn matvec,
                                   linop_cleanup_fn cleanup, linop_ctx_t *ctx);
void linop_destroy_d(LinearOperator_d_t **op);
void linop_destroy_z(LinearOperator_z_t **op);
#endif
