/*
 * bdg_cuda.h -- the thin C ABI between the host C library and the sm_100a
 * kernels.  Plain pointers and sizes only.  Device pointers are expected
 * where a name says `d_`; all device work is ordered on the context's own
 * CUDA stream (bdgd_stream).
 *
 * These entry points replace, as block (many-column) device calls, the
 * reference's single-column host operators of pstuermer/BDG_LOBPCG:
 *   BDGD_OP_KINETIC  kinetic_{d,z}      src/kinetic_impl.inc:17-30
 *   BDGD_OP_K        matmulK_{d,z}      src/matmulK_impl.inc:11-28
 *   BDGD_OP_M        matmulM_{d,z}      src/matmulM_impl.inc:14-44
 *   BDGD_OP_LREP     matmulLrep_{d,z}   src/matmulLrep_impl.inc:13-18
 *   BDGD_OP_SWAP     matmulSwap_{d,z}   src/matmulSwap_impl.inc:14-26
 *   BDGD_OP_TK/TM    precondK/M_{d,z}   src/precond_impl.inc:21-111
 *   BDGD_OP_TLREP    precondLrep_{d,z}  src/precond_impl.inc:113-118
 *   BDGD_OP_DIPCONV  dipolar_conv_{d,z} src/dipolar_conv_impl.inc:22-52
 * and the dense Gram work of the external iLOBPCG (call site
 * src/solver.c:262).
 */
#ifndef BDG_CUDA_H
#define BDG_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bdgd_ctx bdgd_ctx;

enum {
  BDGD_OP_KINETIC = 0,
  BDGD_OP_K = 1,
  BDGD_OP_M = 2,
  BDGD_OP_LREP = 3,
  BDGD_OP_SWAP = 4,
  BDGD_OP_TK = 5,
  BDGD_OP_TM = 6,
  BDGD_OP_TLREP = 7,
  BDGD_OP_DIPCONV = 8
};

enum { BDGD_F64 = 0, BDGD_F32 = 1 };

enum {
  BDGD_OK = 0,
  BDGD_ERR_CUDA = -1,
  BDGD_ERR_ARG = -2,
  BDGD_ERR_UNSUPPORTED = -3,
  BDGD_ERR_STATE = -4
};

/* Message of the last failing call of this thread. */
const char *bdgd_last_error(void);
/* Kernels this library has launched since load (all contexts). */
unsigned long long bdgd_launch_count(void);

/* Number of visible CUDA devices (0 without a GPU); never fails. */
int bdgd_device_count(void);

/* Grid N[0..dim-1] (x fastest), box L; complex_psi0 selects c2c transforms. */
int bdgd_create(bdgd_ctx **out, uint64_t dim, const uint64_t *N, const double *L,
                int complex_psi0);
void bdgd_destroy(bdgd_ctx **ctx);
void *bdgd_stream(bdgd_ctx *ctx);
int bdgd_synchronize(bdgd_ctx *ctx);

/* Physics arrays from host memory (size doubles each; wf is size f64 or size
 * interleaved (re, im) pairs on the complex path; vdd has k_size doubles in
 * the spectrum layout).  NULL leaves an array unchanged. */
int bdgd_set_local_terms(bdgd_ctx *ctx, const double *ltK, const double *ltM);
int bdgd_set_wavefunction(bdgd_ctx *ctx, const void *wf);
int bdgd_set_precond(bdgd_ctx *ctx, const double *sqrtK, const double *sqrtM,
                     double mu);
int bdgd_set_dipolar(bdgd_ctx *ctx, const double *vdd, double g_ddi, int enabled);

/* y = op(x) for ncol columns of device memory.  Column j of x starts at
 * x + j*ldx elements (f64, c64 or, with prec = BDGD_F32, f32 / c32).
 * LREP/TLREP/SWAP columns are [u; v] of 2*size elements, the others size
 * elements.  x and y must not overlap. */
int bdgd_apply(bdgd_ctx *ctx, int op, int prec, const void *d_x, uint64_t ldx,
               void *d_y, uint64_t ldy, uint64_t ncol);

/* Replay operator applies as CUDA graphs (on = 1): the first apply of a
 * given (operator, precision, pointers, leading dimensions, columns) runs
 * directly, the second is captured, later ones launch the graph.  Every
 * field setter invalidates the recorded graphs.  Off by default; the
 * environment variable BDG_GRAPHS=1 turns it on for new contexts.  (No
 * counterpart in the reference, which applies one column per FFTW call.) */
int bdgd_set_graphs(bdgd_ctx *ctx, int on);

/* Free the context's apply scratch (spectra, staging, Gram partials) and its
 * recorded graphs; they are reallocated on the next use. */
int bdgd_trim(bdgd_ctx *ctx);

/* FFT pass family the autotuner chose for (op, prec) on this context: 0 not
 * tuned yet, 1 register-resident line transforms, 2 compile-time
 * shared-memory stages; ms_out (2 floats, may be NULL) receives the timed
 * milliseconds of both.  Tuning happens on the first apply of >= 4 columns
 * unless BDG_FFT_PATH or BDG_GENERIC_FFT fixes the family. */
int bdgd_fft_tuning(bdgd_ctx *ctx, int op, int prec, int *path_out, float *ms_out);

/* Same as bdgd_apply on host memory (copies in, applies, copies out). */
int bdgd_apply_host(bdgd_ctx *ctx, int op, const void *x, void *y, uint64_t ncol);

/* Dipolar mean field phi = g_ddi * F^-1[vdd/size F(|wf|^2)] (real part) of
 * the uploaded wavefunction and kernel, written to host phi_out[size]. */
int bdgd_dipolar_meanfield(bdgd_ctx *ctx, double *phi_out);

/* Unnormalised forward/backward transform of ncol host fields, for plan
 * round-trip checks: forward maps size reals (or complex) to k_size complex
 * values in the FFTW r2c (or c2c) layout, backward the reverse. */
int bdgd_fft_host(bdgd_ctx *ctx, int forward, const void *in, void *out,
                  uint64_t ncol);

/* ---- Gram contraction of the iLOBPCG Rayleigh-Ritz step ----------------
 * For a block S (n x k, column-major, leading dimension lds, n = 2*half)
 * and AS (n x k, leading dimension ldas), writes four k x k column-major
 * FP64 matrices to d_out (leading dimension k, consecutive):
 *   Guu = S_u^H S_u, Gvv = S_v^H S_v, Guv = S_u^H S_v, Ga = S^H AS
 * where S_u are rows [0, half) and S_v rows [half, n).  With B = swap,
 * S^H S = Guu + Gvv and S^H B S = Guv + Guv^H.  Accumulation is FP64
 * (DMMA); prec selects FP64 or FP32 inputs; cplx selects complex data. */
int bdgd_gram(bdgd_ctx *ctx, int prec, int cplx, uint64_t half, uint64_t k,
              const void *d_S, uint64_t lds, const void *d_AS, uint64_t ldas,
              double *d_out);

/* General Gram task list: task t computes C = A^H B (rows x ka by rows x kb,
 * column-major, leading dimensions in elements) into output matrix `out`
 * (ldo x ldo, column-major, FP64 or interleaved complex) at rows i0.., columns
 * j0...  `sym` marks a diagonal block A == B (upper tiles computed, lower
 * filled by symmetry); `mirror` also writes C^H at (j0.., i0..).  Up to 48
 * tasks per call; all tasks in one launch. */
typedef struct {
  const void *a;
  const void *b;
  uint64_t lda, ldb, rows;
  int ka, kb, out, i0, j0, sym, mirror;
} bdgd_gram_task;

int bdgd_gram_tasks(bdgd_ctx *ctx, int prec, int cplx, int ntask, const bdgd_gram_task *tasks, int ldo,
                    double *d_out);

/* Integer tensor-core GEMM tile building block (no counterpart in the
 * reference): D = A B^T with A (M x K) and B (N x K) int8, rows K-contiguous
 * (leading dimensions in elements, multiples of 16, 16-byte aligned), D
 * (M x N) int32 row-major with leading dimension ldd.  M a multiple of 128,
 * N of 64, K of 32.  tcgen05 MMA (kind::i8) with the accumulator in tensor
 * memory, on `stream` (a cudaStream_t).  *d_err (device int) is set to 1 if a
 * wait on the tensor core timed out.  It exists so that the layouts of the
 * FP64-emulation kernels are checked against exact integer arithmetic. */
int bdgd_tc_i8_gemm(void *stream, const int8_t *A, uint64_t lda, const int8_t *B, uint64_t ldb, int32_t *D,
                    uint64_t ldd, uint64_t M, uint64_t N, uint64_t K, int *d_err);

/* Block update (no counterpart in the reference; it replaces the BLAS-3
 * basis updates of the external solver): for each of `nout` outputs,
 *   Y = alpha * sum_b S_b C_b + beta * Y
 * with S_b n x k_b (column-major, leading dimension ld, 16-byte aligned),
 * C_b a k_b x ncol device matrix (column-major, leading dimension ldc >= k_b,
 * any alignment of FP64), Y n x ncol (leading dimension ld).  Up to 4
 * outputs of up to 3 terms each, at most 16 column tiles of 64 in all, in
 * one launch; beta == 0 does not read Y, and an output whose terms all have
 * k_b = 0 is left untouched.  Y must not overlap any S_b.  Real
 * FP64 only (FP64 tensor cores); other precisions, complex data or a layout
 * outside these limits return BDGD_ERR_UNSUPPORTED without launching. */
typedef struct {
  const void *s;
  const double *c;
  int k, ldc;
} bdgd_update_term;

typedef struct {
  void *y;
  int ncol, nterm;
  double alpha, beta;
  bdgd_update_term term[3];
} bdgd_update_out;

int bdgd_block_update(bdgd_ctx *ctx, int prec, int cplx, uint64_t n, uint64_t ld, int nout,
                      const bdgd_update_out *outs);

/* Initial iLOBPCG block on the device (no counterpart in the reference,
 * which fills it on the host, src/solver.c:68-259 and :321-414): columns
 * 0..ncols-1 of d_S (2*size rows, leading dimension ld, FP64 or FP32 per
 * prec, complex when the context is), u = v.  mode 0: plane-wave columns,
 * cols_host = ncols x {kind, fx, fy, fz} (kind 0 noise, 1 cos, 2 sin;
 * f the angular wave numbers), value (wave + 1e-4 (xrand - 0.5)) |psi0| or
 * (xrand - 0.5) |psi0|, one xorshift32 draw per element; mode 1:
 * |sqrt(-2 log u1) cos(2 pi u2)| |psi0|, two draws per element.  The draws
 * follow one xorshift32 stream from `seed` (nonzero), column after column,
 * row after row, so the block equals the reference's host fill with the same
 * seed up to the rounding of sin, cos, log and sqrt. */
int bdgd_init_block(bdgd_ctx *ctx, int prec, int mode, uint32_t seed, int ncols, const double *cols_host, void *d_S,
                    uint64_t ld);

/* Gram contraction that allocates nothing (no counterpart in the reference).
 *
 * Same inputs and output as bdgd_gram (Guu, Gvv, Guv, Ga of a block S and
 * its image AS, four k x k FP64 matrices, column-major, consecutive), for
 * callers that may not allocate device memory when they need it: code
 * running inside a memory pool or arena it does not own, or a framework
 * that bans cudaMalloc/cudaFree on its hot path because they synchronise the
 * device.  Nothing is allocated: no context is needed (work goes to `stream`,
 * NULL for the default stream), and the split partial sums live in one
 * static 8 MiB device array that each GPU using the library keeps until the
 * process exits.
 *
 * Limits: the partials of one split need 4 k^2 doubles (8 k^2 complex), so k
 * is at most 512 (real) or 362 (complex); larger k returns BDGD_ERR_ARG with
 * a message and launches nothing.  The first call on each device looks up
 * the array's device address; make that first call before any stream
 * capture.  Every call reuses the same array: calls that may run at the same
 * time on the GPU (other streams, other host threads) race on it and must
 * be serialised by the caller.  Each call writes every partial it reads, so
 * nothing left over from an earlier call is used.  The looked-up address is
 * kept per device ordinal for the primary context: after cudaDeviceReset,
 * or from a context other than the primary one, do not call it again. */
int bdgd_gram_noalloc(void *stream, int prec, int cplx, uint64_t half, uint64_t k, const void *d_S, uint64_t lds,
                      const void *d_AS, uint64_t ldas, double *d_out);

/* Ground-state producer on the context's grid (real path): split-step
 * imaginary-time propagation then bordered Newton polish; V on the host.
 * The dipolar kernel, when wanted, is uploaded first with
 * bdgd_set_dipolar(enabled = 1).  See bdg_ground_state in bdg/bdg_b200.h. */
int bdgd_ground_state(bdgd_ctx *ctx, const double *V_host, double g, double dt, double tol, int max_steps,
                      int newton_steps, double *psi_inout, double *mu_out, int *steps_out,
                      double *stationarity_out);

#ifdef __cplusplus
}
#endif

#endif /* BDG_CUDA_H */
