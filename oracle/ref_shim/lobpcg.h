/*
 * lobpcg.h -- the indefinite-LOBPCG entry points of the external "LOBPCG"
 * library, with the ABI its caller implies (pstuermer/BDG_LOBPCG
 * src/solver.c:147-164, :262-283 and :304-320, :417-438): alloc(n, nev,
 * sizeSub) returns a state whose S block (n x sizeSub, column-major) carries
 * the initial guess in and the Ritz vectors out, eigVals the Ritz values,
 * converged the count of converged wanted pairs; A, B, T, maxIter, tol are set
 * by the caller.  The solver behind it (ilobpcg_shim.c) is this project's C
 * restatement of the published method (Kressner, Miloloza Pandur & Shao 2014),
 * step for step the iteration of oracle/bdg_oracle.py:ilobpcg.
 * TEST INFRASTRUCTURE ONLY (oracle build of the reference library).
 */
#ifndef LOBPCG_H
#define LOBPCG_H
#include "lobpcg/linop.h"
#include "lobpcg/types.h"

typedef struct {
  uint64_t n, nev, sizeSub;
  LinearOperator_d_t *A, *B, *T;
  uint64_t maxIter;
  f64 tol;
  f64 *S;
  f64 *eigVals;
  uint64_t converged;
  uint64_t iterations;
} d_lobpcg_t;

typedef struct {
  uint64_t n, nev, sizeSub;
  LinearOperator_z_t *A, *B, *T;
  uint64_t maxIter;
  f64 tol;
  c64 *S;
  f64 *eigVals;
  uint64_t converged;
  uint64_t iterations;
} z_lobpcg_t;

d_lobpcg_t *d_ilobpcg_alloc(uint64_t n, uint64_t nev, uint64_t sizeSub);
void d_ilobpcg(d_lobpcg_t *alg);
void d_lobpcg_free(d_lobpcg_t **alg);
z_lobpcg_t *z_ilobpcg_alloc(uint64_t n, uint64_t nev, uint64_t sizeSub);
void z_ilobpcg(z_lobpcg_t *alg);
void z_lobpcg_free(z_lobpcg_t **alg);
#endif
