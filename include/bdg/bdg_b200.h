/*
 * bdg_b200.h -- options and statistics of the B200 library that have no
 * counterpart in the reference API (pstuermer/BDG_LOBPCG include/bdg/bdg.h).
 * All default to the reference's behaviour, so code that never calls them
 * gets the reference semantics.
 */
#ifndef BDG_B200_H
#define BDG_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bdg_t bdg_t;

/* Operator/preconditioner arithmetic inside the solver. */
enum {
  BDG_PREC_F64 = 0,  /* everything FP64 (default) */
  BDG_PREC_MIXED = 1 /* FP32 operator + preconditioner applies and FP32
                        blocks; FP64 Gram accumulation, small dense work,
                        final residual check and FP64 refinement */
};

/* Meaning of the solver tolerance `tol`.  The reference delegates it to an
 * external library whose definition is not available. */
enum {
  BDG_CONV_BACKWARD = 0,     /* ||A x - w B x|| / ((||A||_est + |w|) ||x||) <= tol
                                for each of the nev wanted pairs (default) */
  BDG_CONV_TRUE_RESIDUAL = 1 /* ||K M v - w^2 v|| / ||v|| <= tol */
};

typedef struct {
  uint64_t iterations;     /* iLOBPCG iterations of the last solve */
  uint64_t refine_iterations;
  double seconds_total;    /* wall time of bdg_solve (upload to download) */
  double seconds_device;   /* device time of the iteration loop (CUDA events) */
  double ms_apply_A;       /* accumulated device ms per stage */
  double ms_apply_T;
  double ms_residual;
  double ms_gram;
  double ms_small_dense;
  double ms_update;
  uint64_t cols_apply_A;   /* columns pushed through A and T */
  uint64_t cols_apply_T;
  double max_residual;     /* final convergence measure over the nev pairs */
  double max_true_residual;/* final ||KMv - w^2 v||/||v|| over the nev pairs */
  int status;              /* 0 ok, <0 CUDA / numerical failure */
  double seconds_setup;    /* wall time before the loop: fields, workspace, deflation, X0 fill and upload */
  double seconds_output;   /* wall time after the loop: final measures, block and modes download */
} bdg_solve_stats_t;

void bdg_set_precision(bdg_t *bdg, int precision);
void bdg_set_convergence(bdg_t *bdg, int criterion);
/* Restrict the search to the B-orthogonal complement of the Goldstone
 * Jordan chain {[psi0; 0], [0; M^-1 psi0]} (real or complex psi0 with
 * K psi0 = 0), so the nev wanted pairs are the lowest nonzero modes. */
void bdg_set_goldstone_deflation(bdg_t *bdg, int enable);
/* FP64 iterations appended to a BDG_PREC_MIXED solve (default 3 max). */
void bdg_set_refinement(bdg_t *bdg, int max_iters);
const bdg_solve_stats_t *bdg_solve_stats(const bdg_t *bdg);
/* bdg_set_trap with the potential already evaluated on the grid
 * (V[size], x fastest, at r_i = (i - N/2) L / N); same state rules. */
void bdg_set_trap_grid(bdg_t *bdg, const double *V);
/* bdg_set_local_interactions with U_K(|psi_i|^2) and U_M(|psi_i|^2) already
 * evaluated per grid point; same state rules and accumulation. */
void bdg_set_local_interactions_grid(bdg_t *bdg, const double *uK, const double *uM);
/* Full solver block after a solve: n x sizeSub column-major (host), or NULL.
 * Downloaded on the first call after a solve (the solve itself only brings
 * back the nev wanted modes); NULL once the device workspace is released. */
const void *bdg_solver_block(const bdg_t *bdg);

/* Stationary real condensate on the GPU: split-step imaginary-time
 * propagation from psi_inout (dt, until |delta mu| per step < tol or
 * max_steps), then newton_steps bordered Newton steps (CG on the BdG
 * operator M) to the exact discrete stationary state.  H = -1/2 lap + V +
 * g |psi|^2 (+ g_ddi Phi_dd with the reference's truncated dipolar kernel,
 * 3D), psi normalised to sum |psi|^2 dV = 1.  Writes psi, mu, the ITP step
 * count and ||H psi - mu psi|| (L2 with dV).  0 or a negative error. */
int bdg_ground_state(uint64_t dim, const uint64_t *N, const double *L, const double *V, double g, double g_ddi,
                     const double *dipole_dir, double cutoff_radius, double dt, double tol, uint64_t max_steps,
                     int newton_steps, double *psi_inout, double *mu_out, uint64_t *steps_out,
                     double *stationarity_out);

/* Solve n independent, fully set-up problems on one GPU (no counterpart in
 * the reference, which solves one problem per call).  Up to `concurrency`
 * solves run at once, each on its own host thread and CUDA stream; with
 * `graphs` set their operator applies replay CUDA graphs (bdgd_set_graphs).
 * After each solve the problem's device workspace is released
 * (bdg_release_device_memory); results stay in the problem.  rcs_out[i]
 * (may be NULL) receives bdg_solve's return code, seconds_out[i] (may be
 * NULL) the wall time of that solve.  Returns 0 when every solve returned 0.
 * Problems must be distinct handles. */
int bdg_solve_batch(bdg_t **problems, int n, int concurrency, int graphs, int *rcs_out, double *seconds_out);

/* Free a problem's solver workspace and device scratch (results and the
 * problem's set-up stay; the next bdg_solve reallocates them). */
void bdg_release_device_memory(bdg_t *bdg);

/* Initial block from a host array (no counterpart in the reference, where
 * a BDG_INIT_CUSTOM callback fills it): X is n x sizeSub, column-major
 * (n = 2 * grid size, u rows then v rows; f64, or c64 on the complex
 * path), after bdg_set_solver_params.  The library borrows X: it must stay
 * valid and unchanged until the last bdg_solve that uses it (each solve
 * copies it).  Same as bdg_set_init_mode(BDG_INIT_CUSTOM, ...) with a callback
 * that copies X, but no caller code runs inside bdg_solve, which matters on
 * the solver threads of bdg_solve_batch.  Returns 0, or -2 when X is NULL or
 * the shape is not the problem's. */
int bdg_set_initial_block(bdg_t *bdg, const void *X, uint64_t n, uint64_t sizeSub);

/* Binary files (no counterpart in the reference; its text files,
 * src/io.c:13-165, stay as they are).  The text formats keep 8 significant
 * digits and write one value per fprintf; these keep the exact doubles and
 * write each array at once.  Layout: a 64-byte bdg_bin_header_t, then
 * `count` consecutive fields of N[0]*N[1]*N[2] values each (f64, or
 * interleaved re, im for c128), x fastest, in the host's byte order.
 * Return codes as the text functions: 0 ok, -1 file error, -2 format or
 * grid mismatch (or a bad `part`), -3 nothing to write. */
#define BDG_BIN_MAGIC "BDGBIN01"
#define BDG_BIN_VERSION 1u
enum { BDG_BIN_WAVEFUNCTION = 0, BDG_BIN_MODES_U = 1, BDG_BIN_MODES_V = 2, BDG_BIN_EIGENVALUES = 3 };
enum { BDG_BIN_F64 = 0, BDG_BIN_C128 = 1 };

typedef struct {
  char magic[8];     /* "BDGBIN01" */
  uint32_t version;  /* BDG_BIN_VERSION */
  uint32_t kind;     /* BDG_BIN_WAVEFUNCTION, _MODES_U, _MODES_V, _EIGENVALUES */
  uint32_t dtype;    /* BDG_BIN_F64 or BDG_BIN_C128 */
  uint32_t dim;      /* grid dimension; N[d] = 1 for d >= dim */
  uint64_t N[3];
  uint64_t count;    /* fields (1 for psi0, nev for modes); eigenvalues: nev values */
  uint64_t reserved;
} bdg_bin_header_t;

int bdg_write_wavefunction_bin(const bdg_t *bdg, const char *filename);
/* all nev modes of the last solve: part 0 = u, 1 = v */
int bdg_write_modes_bin(const bdg_t *bdg, int part, const char *filename);
int bdg_write_eigenvalues_bin(const bdg_t *bdg, const char *filename);
/* psi0 from a file written by bdg_write_wavefunction_bin for the same grid
 * and path (real or complex); as bdg_set_wavefunction afterwards */
int bdg_load_wavefunction_bin(bdg_t *bdg, const char *filename);

#ifdef __cplusplus
}
#endif

#endif /* BDG_B200_H */
