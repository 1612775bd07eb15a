// bdg_dev.h -- device context shared by the CUDA translation units.
// Not installed; the public C ABI is include/bdg/bdg_cuda.h.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "bdg/bdg_cuda.h"

#define BDGD_MAX_STAGES 12

struct AxisDev {
  int n;                    // line length
  int nst;                  // number of Stockham stages
  int rad[BDGD_MAX_STAGES]; // radix per stage
  const double2 *r64;       // exp(-2 pi i m / n), m < n
  const float2 *r32;
};

struct GeoDev {
  int dim;
  int cplx;   // complex (c2c) path
  int N[3];   // N[0] = x (fastest)
  int nxk;    // spectrum x extent: N[0]/2+1 (r2c) or N[0] (c2c)
  int nrows;  // real-space rows along x = size / N[0]
  long long S;  // real-space points
  long long H;  // spectrum points per field
  AxisDev ax[3];
  const double *kx2[3];  // per-axis k^2 tables (N[d] entries)
};

struct FieldsDev {
  // precision-specific copies; `w` is the wavefunction (real or interleaved complex)
  const void *ltK, *ltM, *pK, *pM, *w;
  const double *vdd;  // dipolar kernel (k_size doubles, spectrum layout)
  double g_ddi;
  double mu;
  double inv_size;
  double kin_dt;  // exp(-kin_dt k^2) multiplier of the imaginary-time step
  const double *ptab;  // preconditioner multiplier per spectrum point (H), or null
};

struct bdgd_ctx {
  int dim;
  int cplx;
  int N[3];
  double L[3];
  long long S, H;
  int nxk;
  int device;
  cudaStream_t stream;
  GeoDev geo;
  // tables
  double2 *d_roots64[3];
  float2 *d_roots32[3];
  double *d_kx2[3];
  // physics (FP64 and FP32 copies)
  double *ltK64, *ltM64, *pK64, *pM64;
  float *ltK32, *ltM32, *pK32, *pM32;
  void *wf64, *wf32;
  double *vdd;
  double g_ddi, mu;
  int dipolar;
  int has_wf, has_precond;
  // scratch
  void *spec;
  size_t spec_bytes;
  void *io;   // staging for host applies
  size_t io_bytes;
  double *gram_part;
  size_t gram_part_bytes;
  void *oz_buf;        // tensor-core Gram: column maxima of its operands + error flag (stream-ordered)
  size_t oz_buf_bytes;
  size_t spec_cap;  // max scratch bytes per apply chunk
  double kin_dt;
  double *ptab;     // (1/size) / safe_val(mu + k^2/2) per spectrum point, for the current mu
  // FFT pass family per (operator, precision) chosen by the autotuner:
  // 0 not tuned, 1 register lines, 2 compile-time shared-memory stages
  signed char tune[16][2];
  float tune_ms[16][2][2];
  int force_path;   // set while the autotuner times one family
  // CUDA graphs of operator applies (bdgd_set_graphs)
  int graphs_on;
  unsigned version; // bumped by every setter and scratch reallocation
  struct bdgd_graph *graphs;
  int ngraphs;
};

// launches inside a stream capture skip per-launch attribute calls
extern thread_local int bdgd_capturing;

int bdgd_run_internal(bdgd_ctx *c, int kind, const void *d_x, long long ldx, void *d_y, long long ldy, int ncol);

// kernel launch counter (defined in bdg_ops.cu)
void bdgd_count_launch(void);

// error helpers (defined in bdg_ops.cu)
void bdgd_set_error(const char *fmt, ...);
int bdgd_check(cudaError_t e, const char *what);
int bdgd_ensure(cudaStream_t st, void **ptr, size_t *have, size_t want);

#define BDGD_CK(call)                                   \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return bdgd_check(_e, #call); \
  } while (0)
