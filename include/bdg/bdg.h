/*
 * bdg.h -- public C API of the B200 BdG library.
 *
 * Drop-in for the public API of pstuermer/BDG_LOBPCG (include/bdg/bdg.h:23-244
 * of that project): the same 22 functions, the same types and enum values,
 * the same call order and error behaviour.  Behind the API every operator
 * apply and the whole iLOBPCG iteration run on one NVIDIA B200 (sm_100a);
 * the host keeps only setup, bookkeeping and I/O.
 *
 * Problem: the Bogoliubov-de Gennes (BdG) excitations of a (dipolar) BEC on
 * a periodic 1D/2D/3D grid in the K/M form
 *     A x = omega B x,   A = diag(K, M),   B = [[0, I], [I, 0]],   x = [u; v],
 * K = -1/2 lap + localTermK, M = -1/2 lap + localTermM + 2 (dipolar exchange).
 * Real psi0 runs the real (_d, f64) path, complex psi0 the complex (_z, c64)
 * path.
 *
 * Extensions that have no counterpart in the reference (precision mode,
 * convergence criterion, Goldstone deflation, device block entry points)
 * are declared in bdg/bdg_b200.h so this header keeps the reference surface.
 */
#ifndef BDG_H
#define BDG_H

#include "lobpcg/types.h"
#include <stdarg.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Opaque problem handle (reference: include/bdg/bdg.h:23). */
typedef struct bdg_t bdg_t;

/* Initial-block strategy (reference: include/bdg/bdg.h:29-34); values fixed. */
typedef enum {
  BDG_INIT_PLANEWAVE,   /* 0: cos/sin of the lowest |k| plane waves times |psi0| */
  BDG_INIT_WF_WEIGHTED, /* 1: |gaussian| * |psi0|, u = v */
  BDG_INIT_REUSE,       /* 2: previous modes + noise (bdg_reuse_modes) */
  BDG_INIT_CUSTOM       /* 3: user callback fills the block */
} bdg_init_mode_t;

/* k-vector selection for BDG_INIT_PLANEWAVE (reference: :36-40). */
typedef enum {
  BDG_GEOM_AUTO,      /* lowest |k|^2 over all axes */
  BDG_GEOM_ELONGATED, /* k along the longest box axis only */
  BDG_GEOM_RING       /* (kx, ky) pairs, kz = 0 */
} bdg_geom_hint_t;

/*
 * Custom initial-block callback (reference: :42-54).  X is the solver's
 * block, n x sizeSub column-major, n = 2*size; column j holds u in rows
 * [0, size) and v in rows [size, n).  Element type f64 (real path) or c64
 * (complex path).  The block must be B-positive (u^H v > 0 per column; the
 * usual way is u = v).
 */
typedef void (*bdg_init_fn)(const bdg_t *bdg, void *X, uint64_t n,
                            uint64_t sizeSub, void *param);

/* ---- lifecycle ---------------------------------------------------------- */

/* Allocate a problem on an N[0] x ... x N[dim-1] grid of box lengths L
 * (x fastest).  complex_psi0 selects the complex path. */
bdg_t *bdg_alloc(uint64_t dim, const uint64_t *N, const f64 *L, int complex_psi0);

/* Release host and device resources; sets *bdg to NULL. */
void bdg_free(bdg_t **bdg);

/* Drop all physics state and results, keep grid, k tables, FFT plans,
 * device buffers and solver parameters.  State returns to "system set". */
void bdg_reset(bdg_t *bdg);

/* ---- setup, in this order ------------------------------------------------ */

/* k tables (k2, kx2) and FFT plans; required before any operator apply. */
void bdg_set_system(bdg_t *bdg);

/* Add V(r) at r_i = (i - N/2) L/N to both local terms (may be repeated). */
void bdg_set_trap(bdg_t *bdg,
                  f64 (*V_trap)(uint64_t dim, const f64 *r, const void *param),
                  const void *param);

/* Copy the condensate wavefunction (f64 or c64 per the path). */
void bdg_set_wavefunction(bdg_t *bdg, const void *wf, uint64_t wf_size);

/* localTermK += U_K(|psi|^2); localTermM += U_K(|psi|^2) + 2 U_M(|psi|^2). */
void bdg_set_local_interactions(bdg_t *bdg,
                                f64 (*U_intK)(const void *param, f64 density),
                                f64 (*U_intM)(const void *param, f64 density),
                                const void *param);

/* Store mu, build the preconditioner scalings from the local terms, then
 * subtract mu from both local terms. */
void bdg_set_mu(bdg_t *bdg, f64 mu);

/* 3D only, before bdg_set_mu: dipolar kernel and mean field. */
void bdg_set_dipolar(bdg_t *bdg, f64 g_ddi, const f64 *dipole_dir, f64 cutoff_radius);

/* ---- solver -------------------------------------------------------------- */

void bdg_set_solver_params(bdg_t *bdg, uint64_t nev, uint64_t sizeSub,
                           uint64_t maxIter, f64 tol);

/* For BDG_INIT_PLANEWAVE pass fn = NULL and param = (void*)(intptr_t)hint. */
void bdg_set_init_mode(bdg_t *bdg, bdg_init_mode_t mode,
                       bdg_init_fn fn, void *param);

/* Keep the current modes (+ noise_frac * ||column|| gaussian noise) as the
 * next initial block; returns 0, or -3 when there are no results. */
int bdg_reuse_modes(bdg_t *bdg, f64 noise_frac);

/* Run iLOBPCG on the GPU; 0 on success, nonzero on a CUDA/solver failure. */
int bdg_solve(bdg_t *bdg);

/* ---- results (valid after bdg_solve returned 0) --------------------------- */

uint64_t bdg_converged(const bdg_t *bdg);
const f64 *bdg_eigenvalues(const bdg_t *bdg);
const void *bdg_modes_u(const bdg_t *bdg);
const void *bdg_modes_v(const bdg_t *bdg);

/* ---- text I/O ------------------------------------------------------------- */

/* One "re im" pair per line; 0 ok, -1 file error, -2 format/size error. */
int bdg_load_wavefunction(bdg_t *bdg, const char *filename);
int bdg_load_wavefunction_fmt(bdg_t *bdg, const char *fmt, ...);
/* Append one line of nev "%.8e" values separated by tabs; -3 no results. */
int bdg_write_eigenvalues(const bdg_t *bdg, const char *filename);
/* basename_u_<idx>.dat / basename_v_<idx>.dat; -2 index out of range. */
int bdg_write_mode_u(const bdg_t *bdg, uint64_t mode_idx, const char *basename);
int bdg_write_mode_v(const bdg_t *bdg, uint64_t mode_idx, const char *basename);

#ifdef __cplusplus
}
#endif

#endif /* BDG_H */
