// bdg_initd.cu -- the iLOBPCG initial block generated on the device.
//
// The reference fills the n x sizeSub initial block on the host, one element
// after another (pstuermer/BDG_LOBPCG src/solver.c:68-259 real path,
// :321-414 complex path); at 128^3 with sizeSub 64 that is 2.1 GB of
// transcendentals and random draws before the upload.  Here every element is
// computed where it is stored, with the same formulas and the same random
// stream:
//
//   PLANEWAVE    column j: (cos or sin (k_j . r) + 1e-4 (xrand - 0.5)) |psi0|,
//                or (xrand - 0.5) |psi0| past the enumerated wave vectors;
//                one draw per element, stream xorshift32 seeded 42, columns
//                in order, rows in order within a column;
//   WF_WEIGHTED  |sqrt(-2 log u1) cos(2 pi u2)| |psi0|, two draws per
//                element from xorshift32 (seed 42 on the complex path, as the
//                reference; the reference's real path seeds rand_r with the
//                time, so its stream is not reproducible, and the device uses
//                xorshift32 seeded with the time instead);
//   u = v for every column.
//
// xorshift32 is linear over GF(2): the state after p steps is T^p s0 with T a
// 32 x 32 bit matrix.  The host builds T^(2^b), b < 32, once; a thread jumps
// to the first draw of its chunk with at most 32 matrix-vector products
// (p taken modulo the period 2^32 - 1) and steps from there, so the device
// block reproduces the host stream draw for draw.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "bdg_dev.h"

#define IB_T 256  // threads per block
#define IB_C 16   // consecutive rows per thread

struct XsJump {
  uint32_t m[32][32];  // m[b][i] = T^(2^b) e_i (column i)
};

struct IArgs {
  XsJump jump;
  const void *wf;  // |psi0| weights (real or interleaved complex), or null
  int cplx_wf;
  int dim, N[3];
  double L[3];
  long long size, ld;
  uint32_t seed;
  int mode;        // 0 plane waves, 1 |gaussian| weighted
  const double *cols;  // mode 0: per column {kind, fx, fy, fz}; kind 0 noise, 1 cos, 2 sin
};

static uint32_t xs_step_h(uint32_t x) {
  x ^= x << 13;
  x ^= x >> 17;
  x ^= x << 5;
  return x;
}

__device__ __forceinline__ uint32_t xs_step(uint32_t x) {
  x ^= x << 13;
  x ^= x >> 17;
  x ^= x << 5;
  return x;
}

// (0, 1] uniform of a state, as xrand
__device__ __forceinline__ double xs_unit(uint32_t x) { return (double)(x & 0x7FFFFFFFu) / (double)0x7FFFFFFF; }

static uint32_t mat_vec_h(const uint32_t *m, uint32_t v) {
  uint32_t r = 0;
  for (int i = 0; i < 32; ++i)
    if (v >> i & 1u) r ^= m[i];
  return r;
}

static XsJump build_jump_tables() {
  XsJump J;
  for (int i = 0; i < 32; ++i) J.m[0][i] = xs_step_h(1u << i);
  for (int b = 1; b < 32; ++b)
    for (int i = 0; i < 32; ++i) J.m[b][i] = mat_vec_h(J.m[b - 1], J.m[b - 1][i]);
  return J;
}

// built once; a function-local static is initialised exactly once even when
// several solver threads (bdg_solve_batch) reach it together
static const XsJump &jump_tables() {
  static const XsJump J = build_jump_tables();
  return J;
}

// state after p steps from s
__device__ __forceinline__ uint32_t xs_jump(const XsJump &J, uint32_t s, unsigned long long p) {
  p %= 0xFFFFFFFFull;  // period of xorshift32 on nonzero states
  for (int b = 0; b < 32 && p; ++b, p >>= 1) {
    if (!(p & 1ull)) continue;
    uint32_t r = 0;
#pragma unroll 8
    for (int i = 0; i < 32; ++i)
      if (s >> i & 1u) r ^= J.m[b][i];
    s = r;
  }
  return s;
}

template <typename O> __device__ __forceinline__ O out_of(double v);
template <> __device__ __forceinline__ double out_of<double>(double v) { return v; }
template <> __device__ __forceinline__ float out_of<float>(double v) { return (float)v; }
template <> __device__ __forceinline__ double2 out_of<double2>(double v) { return make_double2(v, 0.0); }
template <> __device__ __forceinline__ float2 out_of<float2>(double v) { return make_float2((float)v, 0.f); }

// grid (row chunks, columns); each thread IB_C consecutive rows of column
// blockIdx.y, values staged in shared memory and stored coalesced to both
// halves (u = v)
template <typename O>
__global__ void __launch_bounds__(IB_T) k_init_block(IArgs a, O *__restrict__ S) {
  __shared__ double vals[IB_C][IB_T + 1];
  const int j = blockIdx.y;
  const long long base = (long long)blockIdx.x * IB_T * IB_C;
  const long long i0 = base + (long long)threadIdx.x * IB_C;
  const int draws = a.mode == 0 ? 1 : 2;
  double kind = 0.0, fr[3] = {0.0, 0.0, 0.0};
  if (a.mode == 0) {
    kind = a.cols[4 * j];
    fr[0] = a.cols[4 * j + 1];
    fr[1] = a.cols[4 * j + 2];
    fr[2] = a.cols[4 * j + 3];
  }
  if (i0 < a.size) {
    uint32_t s = xs_jump(a.jump, a.seed, (unsigned long long)draws * ((unsigned long long)j * a.size + i0));
    for (int c = 0; c < IB_C; ++c) {
      const long long i = i0 + c;
      if (i >= a.size) break;
      double w = 1.0;
      if (a.wf) {
        if (a.cplx_wf) {
          const double2 z = ((const double2 *)a.wf)[i];
          w = hypot(z.x, z.y);
        } else {
          w = fabs(((const double *)a.wf)[i]);
        }
      }
      double v;
      if (a.mode == 0) {
        s = xs_step(s);
        const double r = xs_unit(s);
        if (kind == 0.0) {
          v = (r - 0.5) * w;
        } else {
          double kr = 0.0;
          long long stride = 1;
          for (int d = 0; d < a.dim; ++d) {
            const long long id = (i / stride) % a.N[d];
            kr += fr[d] * ((double)id * a.L[d] / (double)a.N[d]);
            stride *= a.N[d];
          }
          const double pw = kind == 2.0 ? sin(kr) : cos(kr);
          const double pert = 1e-4 * (r - 0.5);
          v = (pw + pert) * w;
        }
      } else {
        s = xs_step(s);
        double u1 = xs_unit(s);
        s = xs_step(s);
        const double u2 = xs_unit(s);
        u1 = fmax(u1, 1e-10);
        v = fabs(sqrt(-2.0 * log(u1)) * cos(2.0 * 3.14159265358979323846 * u2)) * w;
      }
      vals[c][threadIdx.x] = v;
    }
  }
  __syncthreads();
  for (int q = threadIdx.x; q < IB_T * IB_C; q += IB_T) {
    const long long i = base + q;
    if (i >= a.size) break;
    const O o = out_of<O>(vals[q % IB_C][q / IB_C]);
    S[(long long)j * a.ld + i] = o;
    S[(long long)j * a.ld + a.size + i] = o;
  }
}

extern "C" int bdgd_init_block(bdgd_ctx *c, int prec, int mode, uint32_t seed, int ncols, const double *cols_host,
                               void *d_S, uint64_t ld) {
  if (ncols <= 0) return BDGD_OK;
  if ((mode != 0 && mode != 1) || d_S == NULL || ld < 2 * (uint64_t)c->S || seed == 0 || ncols > 65535 ||
      (mode == 0 && cols_host == NULL)) {
    bdgd_set_error("bdgd_init_block: bad arguments");
    return BDGD_ERR_ARG;
  }
  static thread_local IArgs a;  // 4 KB of jump tables: host-side staging of the kernel parameters
  memset(&a, 0, sizeof a);
  a.jump = jump_tables();
  a.wf = c->has_wf ? c->wf64 : NULL;
  a.cplx_wf = c->cplx;
  a.dim = c->dim;
  for (int d = 0; d < 3; ++d) {
    a.N[d] = c->N[d] > 0 ? c->N[d] : 1;
    a.L[d] = c->L[d];
  }
  a.size = c->S;
  a.ld = (long long)ld;
  a.seed = seed;
  a.mode = mode;
  if (mode == 0) {
    const size_t cb = sizeof(double) * 4 * (size_t)ncols;
    int rc = bdgd_ensure(c->stream, &c->io, &c->io_bytes, cb);
    if (rc) return rc;
    BDGD_CK(cudaMemcpyAsync(c->io, cols_host, cb, cudaMemcpyHostToDevice, c->stream));
    a.cols = (const double *)c->io;
  }
  const long long nb = (c->S + (long long)IB_T * IB_C - 1) / ((long long)IB_T * IB_C);
  if (nb > 0x7fffffffLL) return BDGD_ERR_UNSUPPORTED;
  dim3 grid((unsigned)nb, (unsigned)ncols);
  bdgd_count_launch();
  if (prec == BDGD_F32) {
    if (c->cplx) k_init_block<float2><<<grid, IB_T, 0, c->stream>>>(a, (float2 *)d_S);
    else k_init_block<float><<<grid, IB_T, 0, c->stream>>>(a, (float *)d_S);
  } else {
    if (c->cplx) k_init_block<double2><<<grid, IB_T, 0, c->stream>>>(a, (double2 *)d_S);
    else k_init_block<double><<<grid, IB_T, 0, c->stream>>>(a, (double *)d_S);
  }
  BDGD_CK(cudaGetLastError());
  // the column table lives in the context's staging buffer until the kernel has read it
  if (mode == 0) BDGD_CK(cudaStreamSynchronize(c->stream));
  return BDGD_OK;
}
