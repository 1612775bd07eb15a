// bdg_blas.cu -- dense block kernels of the GPU iLOBPCG.
//
// * Gram contraction: the four k x k blocks of [X, W, P] needed by the
//   Rayleigh-Ritz step of iLOBPCG (the BLAS-3 work of the external solver
//   the reference links, call site pstuermer/BDG_LOBPCG src/solver.c:262).
//   Tall-skinny C = A^T B over the grid dimension, split over row chunks,
//   FP64 tensor cores (mma.sync m8n8k4 f64; tcgen05 has no FP64 kind),
//   deterministic two-stage reduction.  FP32 inputs are widened to FP64 when
//   staged, so the mixed mode still accumulates in FP64.  The swap operator
//   B never touches memory: S^T B S = Guu... + Guv + Guv^T is formed from
//   the u/v row halves of S.
// * residual / norm kernels and small-matrix helpers for the Rayleigh-Ritz
//   step.
#include <cuda_runtime.h>

#include <atomic>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "bdg_dev.h"
#include "bdg_blas.h"

// ---------------------------------------------------------------------------
// Gram contraction: a list of tasks C_t = A_t^H B_t (tall-skinny, FP64 acc.)
// ---------------------------------------------------------------------------
#define GT 64    // output tile (GT x GT)
#define GRK 32   // contraction rows per shared-memory stage
#define GLD (GRK + 4)
#define GMAXT 48

struct GTask {
  const void *a, *b;
  long long lda, ldb;  // leading dimensions in elements
  long long rows;
  int ka, kb, out, i0, j0, sym, mirror;
  int ta, tb;          // tiles along a, b
  int tile0;           // first global tile of this task
  long long part0;     // offset of this task's partials (doubles)
  long long rowsP;     // rows rounded up to the stage height (stream-K work per tile)
  long long wbase;     // start of this task's tiles on the stream-K work line
};

struct GArgs {
  GTask t[GMAXT];
  int nt;
  int ntiles;
  int nsplit;
  long long chunk;
  double *part;
};

__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// stage a GT x GRK tile: sm[c][r] (component comp of column c0+c, rows r0..)
template <typename T, int ES>
__device__ __forceinline__ void stage_tile(double *sm, const T *__restrict__ base, long long ld, int comp, int c0,
                                           int kc, long long r0, long long rend) {
  for (int q = threadIdx.x; q < GT * GRK; q += blockDim.x) {
    const int c = q / GRK, r = q - c * GRK;
    const long long rr = r0 + r;
    double v = 0.0;
    if (c0 + c < kc && rr < rend) v = (double)base[((long long)(c0 + c) * ld + rr) * ES + comp];
    sm[c * GLD + r] = v;
  }
}

template <typename T, bool CPLX>
__global__ void __launch_bounds__(128) k_gram_tasks(GArgs g) {
  extern __shared__ __align__(16) double gsm[];
  double *sAr = gsm, *sBr = gsm + GT * GLD;
  double *sAi = gsm + 2 * GT * GLD, *sBi = gsm + 3 * GT * GLD;
  // locate task and tile
  int t = 0;
  while (t + 1 < g.nt && (int)blockIdx.x >= g.t[t + 1].tile0) ++t;
  const GTask tk = g.t[t];
  int local = blockIdx.x - tk.tile0, ti, tj;
  if (tk.sym) {  // upper-triangular tiles ti <= tj, row by row
    ti = 0;
    int rowlen = tk.tb;
    while (local >= rowlen) {
      local -= rowlen;
      ++ti;
      rowlen = tk.tb - ti;
    }
    tj = ti + local;
  } else {
    ti = local / tk.tb;
    tj = local - ti * tk.tb;
  }
  const int split = blockIdx.y;
  const long long rbeg = (long long)split * g.chunk;
  long long rend = rbeg + g.chunk;
  if (rend > tk.rows) rend = tk.rows;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wi = warp & 1, wj = warp >> 1;
  const int lr = lane & 3, lc = lane >> 2;
  double acc[4][4][2], aci[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      acc[a][b][0] = acc[a][b][1] = 0.0;
      aci[a][b][0] = aci[a][b][1] = 0.0;
    }
  const T *A = (const T *)tk.a;
  const T *B = (const T *)tk.b;
  constexpr int ES = CPLX ? 2 : 1;
  for (long long r0 = rbeg; r0 < rend; r0 += GRK) {
    stage_tile<T, ES>(sAr, A, tk.lda, 0, ti * GT, tk.ka, r0, rend);
    stage_tile<T, ES>(sBr, B, tk.ldb, 0, tj * GT, tk.kb, r0, rend);
    if (CPLX) {
      stage_tile<T, ES>(sAi, A, tk.lda, 1, ti * GT, tk.ka, r0, rend);
      stage_tile<T, ES>(sBi, B, tk.ldb, 1, tj * GT, tk.kb, r0, rend);
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < GRK; kk += 4) {
      double ar[4], br[4];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi) ar[mi] = sAr[(wi * 32 + mi * 8 + lc) * GLD + kk + lr];
#pragma unroll
      for (int nj = 0; nj < 4; ++nj) br[nj] = sBr[(wj * 32 + nj * 8 + lc) * GLD + kk + lr];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int nj = 0; nj < 4; ++nj) dmma(acc[mi][nj][0], acc[mi][nj][1], ar[mi], br[nj]);
      if (CPLX) {
        // conj(A)^T B: re += Ar Br + Ai Bi ; im += Ar Bi - Ai Br
        double ai[4], bi[4], nai[4];
#pragma unroll
        for (int mi = 0; mi < 4; ++mi) {
          ai[mi] = sAi[(wi * 32 + mi * 8 + lc) * GLD + kk + lr];
          nai[mi] = -ai[mi];
        }
#pragma unroll
        for (int nj = 0; nj < 4; ++nj) bi[nj] = sBi[(wj * 32 + nj * 8 + lc) * GLD + kk + lr];
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
          for (int nj = 0; nj < 4; ++nj) {
            dmma(acc[mi][nj][0], acc[mi][nj][1], ai[mi], bi[nj]);
            dmma(aci[mi][nj][0], aci[mi][nj][1], ar[mi], bi[nj]);
            dmma(aci[mi][nj][0], aci[mi][nj][1], nai[mi], br[nj]);
          }
      }
    }
    __syncthreads();
  }
  // D fragment: row = lane >> 2, cols 2*(lane & 3) + {0, 1}; partials [split][kb][ka] (col-major)
  double *out = g.part + tk.part0 + (long long)split * tk.ka * tk.kb * ES;
#pragma unroll
  for (int mi = 0; mi < 4; ++mi)
#pragma unroll
    for (int nj = 0; nj < 4; ++nj)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int i = ti * GT + wi * 32 + mi * 8 + lc;
        const int j = tj * GT + wj * 32 + nj * 8 + 2 * lr + e;
        if (i < tk.ka && j < tk.kb) {
          const long long o = ((long long)j * tk.ka + i) * ES;
          out[o] = acc[mi][nj][e];
          if (CPLX) out[o + 1] = aci[mi][nj][e];
        }
      }
}

// ---------------------------------------------------------------------------
// Pipelined Gram kernel: tiles staged with 16-byte cp.async, two stages in
// flight, so the loads of rows r0+RK.. overlap the DMMA work on rows r0..
// Needs 16-byte aligned column starts (checked on the host; the kernel above
// is the fallback).
// ---------------------------------------------------------------------------
template <typename T, bool CPLX> struct GStage;
template <> struct GStage<double, false> { typedef double E; static constexpr int RK = 32, LDE = 36; };
template <> struct GStage<float, false> { typedef float E; static constexpr int RK = 32, LDE = 36; };
template <> struct GStage<double, true> { typedef double2 E; static constexpr int RK = 16, LDE = 18; };
template <> struct GStage<float, true> { typedef float2 E; static constexpr int RK = 16, LDE = 18; };
// stage shapes per kernel variant: V = 0 the shapes above; V = 1 half-height
// stages (half the shared memory, so four 128-thread blocks fit an SM)
template <typename T, bool CPLX, int V> struct GStageV : GStage<T, CPLX> {};
template <typename T> struct GStageV<T, false, 1> { typedef typename GStage<T, false>::E E; static constexpr int RK = 16, LDE = 20; };
template <typename T> struct GStageV<T, true, 1> { typedef typename GStage<T, true>::E E; static constexpr int RK = 8, LDE = 10; };
// V = 3 (real, BDG_GRAM_VARIANT=3): a ring of three 16-row stages with one
// barrier per stage, the loads two stages ahead of the DMMA work (60 KB,
// three blocks per SM).  At 128^3, k = 192: 24.0 against 24.6 ms for V = 1;
// four-stage rings (8 rows at four blocks per SM, 16 rows at two) measured
// 36.4 and 25.8 ms.
template <typename T> struct GStageV<T, false, 3> { typedef typename GStage<T, false>::E E; static constexpr int RK = 16, LDE = 20; };
template <int V> constexpr int gram_nstage() { return V == 3 ? 3 : 2; }

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int src_bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <typename E> __device__ __forceinline__ double re_of(E v);
template <> __device__ __forceinline__ double re_of<double>(double v) { return v; }
template <> __device__ __forceinline__ double re_of<float>(float v) { return (double)v; }
template <> __device__ __forceinline__ double re_of<double2>(double2 v) { return v.x; }
template <> __device__ __forceinline__ double re_of<float2>(float2 v) { return (double)v.x; }
template <typename E> __device__ __forceinline__ double im_of(E v) { return 0.0; }
template <> __device__ __forceinline__ double im_of<double2>(double2 v) { return v.y; }
template <> __device__ __forceinline__ double im_of<float2>(float2 v) { return (double)v.y; }

template <typename T, bool CPLX, int V = 0>
__device__ __forceinline__ void stage_async(typename GStageV<T, CPLX, V>::E *sm, const T *__restrict__ base, long long ld,
                                            int c0, int kc, long long r0, long long rend) {
  typedef typename GStageV<T, CPLX, V>::E E;
  constexpr int RK = GStageV<T, CPLX, V>::RK, LDE = GStageV<T, CPLX, V>::LDE;
  constexpr int EB = (int)sizeof(E);
  constexpr int RPC = 16 / EB;          // rows per 16-byte chunk
  constexpr int CPC = RK / RPC;         // chunks per column
  constexpr int ES = CPLX ? 2 : 1;
  for (int q = threadIdx.x; q < GT * CPC; q += blockDim.x) {
    const int c = q / CPC, ch = q - c * CPC;
    const int r = ch * RPC;
    const long long rr = r0 + r;
    long long nvalid = rend - rr;
    nvalid = nvalid < 0 ? 0 : (nvalid > RPC ? RPC : nvalid);
    const bool colok = (c0 + c) < kc;
    const T *src = colok && nvalid > 0 ? base + ((long long)(c0 + c) * ld + rr) * ES : base;
    cp_async16(sm + c * LDE + r, src, colok ? (int)(nvalid * EB) : 0);
  }
}

template <typename T, bool CPLX>
__global__ void __launch_bounds__(128) k_gram_tasks2(GArgs g) {
  typedef typename GStage<T, CPLX>::E E;
  constexpr int RK = GStage<T, CPLX>::RK, LDE = GStage<T, CPLX>::LDE;
  constexpr int ES = CPLX ? 2 : 1;
  extern __shared__ __align__(16) unsigned char gsm2[];
  E *buf = (E *)gsm2;  // [stage][A|B][GT][LDE]
  int t = 0;
  while (t + 1 < g.nt && (int)blockIdx.x >= g.t[t + 1].tile0) ++t;
  const GTask tk = g.t[t];
  int local = blockIdx.x - tk.tile0, ti, tj;
  if (tk.sym) {
    ti = 0;
    int rowlen = tk.tb;
    while (local >= rowlen) {
      local -= rowlen;
      ++ti;
      rowlen = tk.tb - ti;
    }
    tj = ti + local;
  } else {
    ti = local / tk.tb;
    tj = local - ti * tk.tb;
  }
  const int split = blockIdx.y;
  const long long rbeg = (long long)split * g.chunk;
  long long rend = rbeg + g.chunk;
  if (rend > tk.rows) rend = tk.rows;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wi = warp & 1, wj = warp >> 1;
  const int lr = lane & 3, lc = lane >> 2;
  double acc[4][4][2], aci[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      acc[a][b][0] = acc[a][b][1] = 0.0;
      aci[a][b][0] = aci[a][b][1] = 0.0;
    }
  const T *A = (const T *)tk.a;
  const T *B = (const T *)tk.b;
  const long long nst = rend > rbeg ? (rend - rbeg + RK - 1) / RK : 0;
  if (nst > 0) {
    stage_async<T, CPLX>(buf, A, tk.lda, ti * GT, tk.ka, rbeg, rend);
    stage_async<T, CPLX>(buf + GT * LDE, B, tk.ldb, tj * GT, tk.kb, rbeg, rend);
    cp_async_commit();
  }
  for (long long s = 0; s < nst; ++s) {
    E *cur = buf + (s & 1) * 2 * GT * LDE;
    if (s + 1 < nst) {
      E *nxt = buf + ((s + 1) & 1) * 2 * GT * LDE;
      const long long r0 = rbeg + (s + 1) * RK;
      stage_async<T, CPLX>(nxt, A, tk.lda, ti * GT, tk.ka, r0, rend);
      stage_async<T, CPLX>(nxt + GT * LDE, B, tk.ldb, tj * GT, tk.kb, r0, rend);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const E *sA = cur, *sB = cur + GT * LDE;
#pragma unroll
    for (int kk = 0; kk < RK; kk += 4) {
      double ar[4], br[4], ai[4], bi[4];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi) {
        const E v = sA[(wi * 32 + mi * 8 + lc) * LDE + kk + lr];
        ar[mi] = re_of<E>(v);
        ai[mi] = im_of<E>(v);
      }
#pragma unroll
      for (int nj = 0; nj < 4; ++nj) {
        const E v = sB[(wj * 32 + nj * 8 + lc) * LDE + kk + lr];
        br[nj] = re_of<E>(v);
        bi[nj] = im_of<E>(v);
      }
#pragma unroll
      for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int nj = 0; nj < 4; ++nj) dmma(acc[mi][nj][0], acc[mi][nj][1], ar[mi], br[nj]);
      if (CPLX) {
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
          for (int nj = 0; nj < 4; ++nj) {
            dmma(acc[mi][nj][0], acc[mi][nj][1], ai[mi], bi[nj]);
            dmma(aci[mi][nj][0], aci[mi][nj][1], ar[mi], bi[nj]);
            dmma(aci[mi][nj][0], aci[mi][nj][1], -ai[mi], br[nj]);
          }
      }
    }
    __syncthreads();
  }
  double *out = g.part + tk.part0 + (long long)split * tk.ka * tk.kb * ES;
#pragma unroll
  for (int mi = 0; mi < 4; ++mi)
#pragma unroll
    for (int nj = 0; nj < 4; ++nj)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int i = ti * GT + wi * 32 + mi * 8 + lc;
        const int j = tj * GT + wj * 32 + nj * 8 + 2 * lr + e;
        if (i < tk.ka && j < tk.kb) {
          const long long o = ((long long)j * tk.ka + i) * ES;
          out[o] = acc[mi][nj][e];
          if (CPLX) out[o + 1] = aci[mi][nj][e];
        }
      }
}

// ---------------------------------------------------------------------------
// Stream-K schedule of the pipelined Gram kernel.  The (tile, row) work of
// all tasks is laid on one line -- task after task, tile after tile, each
// tile's rows rounded up to a multiple of the stage height -- and cut into
// equal pieces, one per resident block, so every block has the same work
// whatever the mix of task sizes (tasks over the u or v half have half the
// rows of those over all n).  A block writes one GT x GT partial per tile
// segment it covers; a tile's partials are summed in a fixed order by the
// reduction, so the result is deterministic.
// ---------------------------------------------------------------------------
#define GSK_STEP 32        // work-line granularity (multiple of every stage height)
#define GMAXTILES 1024

struct GArgsSK {
  GTask t[GMAXT];
  int nt;
  int ntiles;
  long long per;  // work-line rows per block (multiple of GSK_STEP)
  long long W;    // work-line length
  double *part;
  int segbase[GMAXTILES + 1];  // first partial slot of each tile
};

__device__ __forceinline__ void gram_tile_of(const GTask &tk, int local, int &ti, int &tj) {
  if (tk.sym) {
    ti = 0;
    int rowlen = tk.tb;
    while (local >= rowlen) {
      local -= rowlen;
      ++ti;
      rowlen = tk.tb - ti;
    }
    tj = ti + local;
  } else {
    ti = local / tk.tb;
    tj = local - ti * tk.tb;
  }
}

// One tile of A^H B over rows [rbeg, rend): the two-stage cp.async pipeline
// of k_gram_tasks2; writes the GT x GT partial to out (column-major, tile-local).
template <typename T, bool CPLX, int V = 0>
__device__ __forceinline__ void gram_tile_rows(const GTask &tk, int ti, int tj, long long rbeg, long long rend,
                                               double *__restrict__ out, typename GStageV<T, CPLX, V>::E *buf) {
  typedef typename GStageV<T, CPLX, V>::E E;
  constexpr int RK = GStageV<T, CPLX, V>::RK, LDE = GStageV<T, CPLX, V>::LDE;
  constexpr int ES = CPLX ? 2 : 1;
  // SPLIT (complex, V = 2, 256 threads): warps 0-3 accumulate the real parts
  // and warps 4-7 the imaginary parts of the same four 32 x 32 quadrants, one
  // accumulator set per warp
  constexpr bool SPLIT = CPLX && V == 2;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int part = SPLIT ? (warp >> 2) : 0;
  const int wi = warp & 1, wj = (warp >> 1) & 1;
  const int lr = lane & 3, lc = lane >> 2;
  double acc[4][4][2], aci[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      acc[a][b][0] = acc[a][b][1] = 0.0;
      aci[a][b][0] = aci[a][b][1] = 0.0;
    }
  const T *A = (const T *)tk.a;
  const T *B = (const T *)tk.b;
  const long long nst = rend > rbeg ? (rend - rbeg + RK - 1) / RK : 0;
  constexpr int NS = gram_nstage<V>();
  if constexpr (NS > 2) {
    // ring of NS stages: stages 0 .. NS-2 in flight before the first; one
    // (possibly empty) commit group per stage keeps the wait counts uniform
#pragma unroll
    for (int q = 0; q < NS - 1; ++q) {
      if (q < nst) {
        E *st = buf + q * 2 * GT * LDE;
        stage_async<T, CPLX, V>(st, A, tk.lda, ti * GT, tk.ka, rbeg + q * RK, rend);
        stage_async<T, CPLX, V>(st + GT * LDE, B, tk.ldb, tj * GT, tk.kb, rbeg + q * RK, rend);
      }
      cp_async_commit();
    }
  } else if (nst > 0) {
    stage_async<T, CPLX, V>(buf, A, tk.lda, ti * GT, tk.ka, rbeg, rend);
    stage_async<T, CPLX, V>(buf + GT * LDE, B, tk.ldb, tj * GT, tk.kb, rbeg, rend);
    cp_async_commit();
  }
  for (long long s = 0; s < nst; ++s) {
    E *cur;
    if constexpr (NS > 2) {
      cur = buf + (int)(s % NS) * 2 * GT * LDE;
      cp_async_wait<NS - 2>();  // this thread's copies of stage s have landed
      __syncthreads();          // everyone's, and stage s - 1 is consumed by all warps
      const long long q = s + NS - 1;
      if (q < nst) {
        E *st = buf + (int)(q % NS) * 2 * GT * LDE;
        stage_async<T, CPLX, V>(st, A, tk.lda, ti * GT, tk.ka, rbeg + q * RK, rend);
        stage_async<T, CPLX, V>(st + GT * LDE, B, tk.ldb, tj * GT, tk.kb, rbeg + q * RK, rend);
      }
      cp_async_commit();
    } else {
      cur = buf + (s & 1) * 2 * GT * LDE;
      if (s + 1 < nst) {
        E *nxt = buf + ((s + 1) & 1) * 2 * GT * LDE;
        const long long r0 = rbeg + (s + 1) * RK;
        stage_async<T, CPLX, V>(nxt, A, tk.lda, ti * GT, tk.ka, r0, rend);
        stage_async<T, CPLX, V>(nxt + GT * LDE, B, tk.ldb, tj * GT, tk.kb, r0, rend);
        cp_async_commit();
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
      __syncthreads();
    }
    const E *sA = cur, *sB = cur + GT * LDE;
#pragma unroll
    for (int kk = 0; kk < RK; kk += 4) {
      double ar[4], br[4], ai[4], bi[4];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi) {
        const E v = sA[(wi * 32 + mi * 8 + lc) * LDE + kk + lr];
        ar[mi] = re_of<E>(v);
        ai[mi] = im_of<E>(v);
      }
#pragma unroll
      for (int nj = 0; nj < 4; ++nj) {
        const E v = sB[(wj * 32 + nj * 8 + lc) * LDE + kk + lr];
        br[nj] = re_of<E>(v);
        bi[nj] = im_of<E>(v);
      }
      if constexpr (SPLIT) {
        if (part == 0) {
#pragma unroll
          for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int nj = 0; nj < 4; ++nj) {
              dmma(acc[mi][nj][0], acc[mi][nj][1], ar[mi], br[nj]);
              dmma(acc[mi][nj][0], acc[mi][nj][1], ai[mi], bi[nj]);
            }
        } else {
#pragma unroll
          for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int nj = 0; nj < 4; ++nj) {
              dmma(acc[mi][nj][0], acc[mi][nj][1], ar[mi], bi[nj]);
              dmma(acc[mi][nj][0], acc[mi][nj][1], -ai[mi], br[nj]);
            }
        }
      } else {
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
          for (int nj = 0; nj < 4; ++nj) dmma(acc[mi][nj][0], acc[mi][nj][1], ar[mi], br[nj]);
        if (CPLX) {
#pragma unroll
          for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int nj = 0; nj < 4; ++nj) {
              dmma(acc[mi][nj][0], acc[mi][nj][1], ai[mi], bi[nj]);
              dmma(aci[mi][nj][0], aci[mi][nj][1], ar[mi], bi[nj]);
              dmma(aci[mi][nj][0], aci[mi][nj][1], -ai[mi], br[nj]);
            }
        }
      }
    }
    if constexpr (NS == 2) __syncthreads();
  }
  if constexpr (NS > 2) {
    // the next segment's prologue refills the ring: every warp done with it
    cp_async_wait<0>();
    __syncthreads();
  }
#pragma unroll
  for (int mi = 0; mi < 4; ++mi)
#pragma unroll
    for (int nj = 0; nj < 4; ++nj)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int il = wi * 32 + mi * 8 + lc;
        const int jl = wj * 32 + nj * 8 + 2 * lr + e;
        const long long o = ((long long)jl * GT + il) * ES;
        if constexpr (SPLIT) {
          out[o + part] = acc[mi][nj][e];
        } else {
          out[o] = acc[mi][nj][e];
          if (CPLX) out[o + 1] = aci[mi][nj][e];
        }
      }
}

// threads per block of a k_gram_sk variant (V = 2 splits real and imaginary
// accumulation over twice the warps)
template <int V> constexpr int gram_threads() { return V == 2 ? 256 : 128; }
template <int V> constexpr int gram_min_blocks() { return V == 1 ? 4 : V == 3 ? 3 : V == 2 ? 2 : 1; }

template <typename T, bool CPLX, int V>
__global__ void __launch_bounds__(gram_threads<V>(), gram_min_blocks<V>()) k_gram_sk(GArgsSK g) {
  typedef typename GStageV<T, CPLX, V>::E E;
  constexpr int ES = CPLX ? 2 : 1;
  extern __shared__ __align__(16) unsigned char gsm3[];
  E *buf = (E *)gsm3;
  const long long start = (long long)blockIdx.x * g.per;
  long long end = start + g.per;
  if (end > g.W) end = g.W;
  long long pos = start;
  int t = 0;
  while (pos < end) {
    while (t + 1 < g.nt && pos >= g.t[t + 1].wbase) ++t;
    const GTask &tk = g.t[t];
    const long long rel = pos - tk.wbase;
    const int lt = (int)(rel / tk.rowsP);
    const long long r0 = rel - (long long)lt * tk.rowsP;
    long long seglen = tk.rowsP - r0;
    if (seglen > end - pos) seglen = end - pos;
    long long r1 = r0 + seglen;
    if (r1 > tk.rows) r1 = tk.rows;
    int ti, tj;
    gram_tile_of(tk, lt, ti, tj);
    const int tau = tk.tile0 + lt;
    const long long first = (tk.wbase + (long long)lt * tk.rowsP) / g.per;
    const int slot = g.segbase[tau] + (int)((long long)blockIdx.x - first);
    gram_tile_rows<T, CPLX, V>(tk, ti, tj, r0, r1, g.part + (long long)slot * GT * GT * ES, buf);
    pos += seglen;
  }
}

// Sum the segment partials of every tile into the output block (and its
// mirror); symmetric tasks take the lower triangle from the upper tiles.
__global__ void k_gram_sk_reduce(GArgsSK g, int cplx, int ldo, double *__restrict__ outbuf) {
  const int es = cplx ? 2 : 1;
  const int t = blockIdx.y;
  const GTask &tk = g.t[t];
  const long long kk = (long long)tk.ka * tk.kb;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < kk; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % tk.ka), j = (int)(q / tk.ka);
    int si = i, sj = j;
    bool conj = false;
    if (tk.sym && (i / GT) > (j / GT)) {
      si = j;
      sj = i;
      conj = true;
    }
    const int ti = si / GT, tj = sj / GT;
    const int lt = tk.sym ? (ti * tk.tb - ti * (ti - 1) / 2 + (tj - ti)) : (ti * tk.tb + tj);
    const int tau = tk.tile0 + lt;
    const long long el = ((long long)(sj - tj * GT) * GT + (si - ti * GT)) * es;
    double re = 0.0, im = 0.0;
    for (int sg = g.segbase[tau]; sg < g.segbase[tau + 1]; ++sg) {
      const double *pp = g.part + (long long)sg * GT * GT * es + el;
      re += pp[0];
      if (cplx) im += pp[1];
    }
    if (conj) im = -im;
    double *o = outbuf + (long long)tk.out * ldo * ldo * es;
    const long long dst = ((long long)(tk.j0 + j) * ldo + tk.i0 + i) * es;
    o[dst] = re;
    if (cplx) o[dst + 1] = im;
    if (tk.mirror) {
      const long long mdst = ((long long)(tk.i0 + i) * ldo + tk.j0 + j) * es;
      o[mdst] = re;
      if (cplx) o[mdst + 1] = -im;
    }
  }
}

// resident blocks of k_gram_sk<T, CPLX> on this device (cached per device)
template <typename T, bool CPLX, int V>
static int gram_sk_slots(bdgd_ctx *c, size_t sm) {
  static std::atomic<int> cached[64];  // written by several solver threads: idempotent, atomic
  const int dev = c->device < 64 ? c->device : 63;
  if (const int v = cached[dev].load(std::memory_order_relaxed)) return v;
  int nsm = 0, nb = 0;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_gram_sk<T, CPLX, V>, gram_threads<V>(), sm) != cudaSuccess || nb < 1 ||
      nsm < 1) {
    cudaGetLastError();
    return 148;
  }
  cached[dev].store(nb * nsm, std::memory_order_relaxed);
  return nb * nsm;
}

// Stream-K launch of the task list; returns BDGD_ERR_UNSUPPORTED when the
// tile count exceeds GMAXTILES (the caller then uses the row-split kernels).
template <typename T, bool CPLX, int V>
static int launch_gram_sk(bdgd_ctx *c, const GArgs &ga, int cplx, int ldo, double *d_out) {
  typedef typename GStageV<T, CPLX, V>::E E;
  const int es = cplx ? 2 : 1;
  if (ga.ntiles > GMAXTILES) return BDGD_ERR_UNSUPPORTED;
  const size_t sm = sizeof(E) * gram_nstage<V>() * 2 * GT * GStageV<T, CPLX, V>::LDE;
  if (sm > 48 * 1024)
    BDGD_CK(cudaFuncSetAttribute(k_gram_sk<T, CPLX, V>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  static thread_local GArgsSK g;  // large; host-side staging of the kernel parameters
  memset(&g, 0, sizeof g);
  g.nt = ga.nt;
  g.ntiles = ga.ntiles;
  long long W = 0;
  for (int i = 0; i < ga.nt; ++i) {
    g.t[i] = ga.t[i];
    GTask &t = g.t[i];
    t.rowsP = (t.rows + GSK_STEP - 1) / GSK_STEP * GSK_STEP;
    t.wbase = W;
    const int nti = t.sym ? t.ta * (t.ta + 1) / 2 : t.ta * t.tb;
    W += (long long)nti * t.rowsP;
  }
  if (W == 0) return BDGD_OK;
  const int slots = gram_sk_slots<T, CPLX, V>(c, sm);
  long long per = (W + slots - 1) / slots;
  per = (per + GSK_STEP - 1) / GSK_STEP * GSK_STEP;
  const long long nblk = (W + per - 1) / per;
  g.per = per;
  g.W = W;
  int sb = 0;
  for (int i = 0; i < g.nt; ++i) {
    const GTask &t = g.t[i];
    const int nti = t.sym ? t.ta * (t.ta + 1) / 2 : t.ta * t.tb;
    for (int lt = 0; lt < nti; ++lt) {
      const long long b0 = t.wbase + (long long)lt * t.rowsP;
      const long long f = b0 / per, l = (b0 + t.rowsP - 1) / per;
      g.segbase[t.tile0 + lt] = sb;
      if (t.rowsP > 0) sb += (int)(l - f + 1);  // a task without rows has no segments (its blocks are zero)
    }
  }
  g.segbase[g.ntiles] = sb;
  int rc = bdgd_ensure(c->stream, (void **)&c->gram_part, &c->gram_part_bytes, sizeof(double) * (size_t)sb * GT * GT * es);
  if (rc) return rc;
  g.part = c->gram_part;
  bdgd_count_launch();
  k_gram_sk<T, CPLX, V><<<(unsigned)nblk, gram_threads<V>(), sm, c->stream>>>(g);
  BDGD_CK(cudaGetLastError());
  bdgd_count_launch();
  k_gram_sk_reduce<<<dim3(32, g.nt), 256, 0, c->stream>>>(g, cplx, ldo, d_out);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}

template <typename T, bool CPLX>
static int launch_gram2(bdgd_ctx *c, const GArgs &g, dim3 grid) {
  typedef typename GStage<T, CPLX>::E E;
  const size_t sm = sizeof(E) * 2 * 2 * GT * GStage<T, CPLX>::LDE;
  if (sm > 48 * 1024)
    BDGD_CK(cudaFuncSetAttribute(k_gram_tasks2<T, CPLX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  bdgd_count_launch();
  k_gram_tasks2<T, CPLX><<<grid, 128, sm, c->stream>>>(g);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}

// Sum the split partials of every task into its output block (and its
// mirror); sym tasks read the lower triangle from the computed upper tiles.
__global__ void k_gram_tasks_reduce(GArgs g, int cplx, int ldo, double *__restrict__ outbuf) {
  const int es = cplx ? 2 : 1;
  const int t = blockIdx.y;
  const GTask tk = g.t[t];
  const long long kk = (long long)tk.ka * tk.kb;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < kk; q += (long long)gridDim.x * blockDim.x) {
    int i = (int)(q % tk.ka), j = (int)(q / tk.ka);
    bool conj = false;
    int si = i, sj = j;
    if (tk.sym && (i / GT) > (j / GT)) {  // lower tile: take the transpose element
      si = j;
      sj = i;
      conj = true;
    }
    double re = 0.0, im = 0.0;
    const double *pp = g.part + tk.part0 + ((long long)sj * tk.ka + si) * es;
    for (int sp = 0; sp < g.nsplit; ++sp) {
      re += pp[(long long)sp * kk * es];
      if (cplx) im += pp[(long long)sp * kk * es + 1];
    }
    if (conj) im = -im;
    double *o = outbuf + (long long)tk.out * ldo * ldo * es;
    const long long dst = ((long long)(tk.j0 + j) * ldo + tk.i0 + i) * es;
    o[dst] = re;
    if (cplx) o[dst + 1] = im;
    if (tk.mirror) {
      const long long mdst = ((long long)(tk.i0 + i) * ldo + tk.j0 + j) * es;
      o[mdst] = re;
      if (cplx) o[mdst + 1] = -im;
    }
  }
}

extern "C" int bdgd_gram_oz(bdgd_ctx *c, int prec, int ntask, const bdgd_gram_task *tasks, int ldo, double *d_out);
#define BDG_GRAM_TC_F32_DEFAULT 1  // 13.9 against 21.9 ms at 128^3, k = 192; mixed solve 3.34 against 3.49 s

// Tensor-core (int8 digits, tcgen05) Gram for real FP64 or FP32 blocks:
// BDG_GRAM_TC=1 turns it on for both, BDG_GRAM_TC=0 off for both; unset, it
// serves the FP32 blocks (faster than DMMA there) and not the FP64 ones (on
// a par with DMMA per iteration at 128^3)
static bool gram_tc_on(int prec) {
  const char *e = getenv("BDG_GRAM_TC");
  if (e && e[0]) return e[0] == '1';
  return prec == BDGD_F32 && BDG_GRAM_TC_F32_DEFAULT;
}

extern "C" int bdgd_gram_tasks(bdgd_ctx *c, int prec, int cplx, int ntask, const bdgd_gram_task *tasks, int ldo,
                               double *d_out) {
  if (ntask <= 0) return BDGD_OK;
  if ((prec == BDGD_F64 || prec == BDGD_F32) && !cplx && gram_tc_on(prec)) {
    const int rc = bdgd_gram_oz(c, prec, ntask, tasks, ldo, d_out);
    if (rc != BDGD_ERR_UNSUPPORTED) return rc;
  }
  if (ntask > GMAXT) {
    bdgd_set_error("bdgd_gram_tasks: at most %d tasks", GMAXT);
    return BDGD_ERR_ARG;
  }
  const int es = cplx ? 2 : 1;
  GArgs g;
  memset(&g, 0, sizeof g);
  g.nt = ntask;
  long long maxrows = 0;
  int tiles = 0;
  for (int i = 0; i < ntask; ++i) {
    GTask &t = g.t[i];
    const bdgd_gram_task &s = tasks[i];
    t.a = s.a;
    t.b = s.b;
    t.lda = (long long)s.lda;
    t.ldb = (long long)s.ldb;
    t.rows = (long long)s.rows;
    t.ka = s.ka;
    t.kb = s.kb;
    t.out = s.out;
    t.i0 = s.i0;
    t.j0 = s.j0;
    t.sym = s.sym && s.ka == s.kb;
    t.mirror = s.mirror;
    t.ta = (s.ka + GT - 1) / GT;
    t.tb = (s.kb + GT - 1) / GT;
    t.tile0 = tiles;
    tiles += t.sym ? t.ta * (t.ta + 1) / 2 : t.ta * t.tb;
    if (t.rows > maxrows) maxrows = t.rows;
  }
  g.ntiles = tiles;
  int nsplit = (4 * 148 + tiles - 1) / tiles;
  const long long maxsplit = (maxrows + 8 * GRK - 1) / (8 * GRK);
  if (nsplit > maxsplit) nsplit = (int)maxsplit;
  if (nsplit < 1) nsplit = 1;
  long long chunk = (maxrows + nsplit - 1) / nsplit;
  chunk = (chunk + GRK - 1) / GRK * GRK;
  if (chunk < GRK) chunk = GRK;
  nsplit = (int)((maxrows + chunk - 1) / chunk);
  if (nsplit < 1) nsplit = 1;
  g.nsplit = nsplit;
  g.chunk = chunk;
  long long off = 0;
  for (int i = 0; i < ntask; ++i) {
    g.t[i].part0 = off;
    off += (long long)nsplit * g.t[i].ka * g.t[i].kb * es;
  }
  int rc = bdgd_ensure(c->stream, (void **)&c->gram_part, &c->gram_part_bytes, sizeof(double) * off);
  if (rc) return rc;
  g.part = c->gram_part;
  // tasks with fewer rows than nsplit*chunk simply see empty splits (zeros)
  const size_t sm = sizeof(double) * GT * GLD * (cplx ? 4 : 2);
  dim3 grid(tiles, nsplit);
  bool aligned = !getenv("BDG_GRAM_SIMPLE");
  {
    const size_t eb = (size_t)(prec == BDGD_F32 ? 4 : 8) * (cplx ? 2 : 1);
    for (int i = 0; i < ntask && aligned; ++i)
      if (((uintptr_t)g.t[i].a | (uintptr_t)g.t[i].b) % 16 || (g.t[i].lda * eb) % 16 || (g.t[i].ldb * eb) % 16)
        aligned = false;
  }
  if (aligned && !getenv("BDG_GRAM_SPLIT")) {
    // real FP64: half-height stages, four blocks per SM (BDG_GRAM_VARIANT=0 for
    // the full-height stages at three blocks per SM)
    const char *gv = getenv("BDG_GRAM_VARIANT");
    const bool half = !(gv && gv[0] == '0');
    const int ring = gv ? atoi(gv) : 0;  // 3: the three-stage ring (real FP64)
    // complex FP64: real and imaginary parts on separate warps (29.8 against
    // 28.9 TF/s at 128^3, k = 192; in FP32 the one-warp form is faster)
    if (prec == BDGD_F32) rc = cplx ? launch_gram_sk<float, true, 0>(c, g, cplx, ldo, d_out)
                                    : launch_gram_sk<float, false, 0>(c, g, cplx, ldo, d_out);
    else if (cplx) rc = half ? launch_gram_sk<double, true, 2>(c, g, cplx, ldo, d_out)
                             : launch_gram_sk<double, true, 0>(c, g, cplx, ldo, d_out);
    else if (ring == 3) rc = launch_gram_sk<double, false, 3>(c, g, cplx, ldo, d_out);
    else rc = half ? launch_gram_sk<double, false, 1>(c, g, cplx, ldo, d_out)
                   : launch_gram_sk<double, false, 0>(c, g, cplx, ldo, d_out);
    if (rc != BDGD_ERR_UNSUPPORTED) return rc;
  }
  if (aligned) {
    if (prec == BDGD_F32) rc = cplx ? launch_gram2<float, true>(c, g, grid) : launch_gram2<float, false>(c, g, grid);
    else rc = cplx ? launch_gram2<double, true>(c, g, grid) : launch_gram2<double, false>(c, g, grid);
    if (rc) return rc;
  } else if (prec == BDGD_F32) {
    if (cplx) {
      BDGD_CK(cudaFuncSetAttribute(k_gram_tasks<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      bdgd_count_launch();
      k_gram_tasks<float, true><<<grid, 128, sm, c->stream>>>(g);
    } else {
      bdgd_count_launch();
      k_gram_tasks<float, false><<<grid, 128, sm, c->stream>>>(g);
    }
  } else {
    if (cplx) {
      BDGD_CK(cudaFuncSetAttribute(k_gram_tasks<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      bdgd_count_launch();
      k_gram_tasks<double, true><<<grid, 128, sm, c->stream>>>(g);
    } else {
      bdgd_count_launch();
      k_gram_tasks<double, false><<<grid, 128, sm, c->stream>>>(g);
    }
  }
  BDGD_CK(cudaGetLastError());
  bdgd_count_launch();
  k_gram_tasks_reduce<<<dim3(32, ntask), 256, 0, c->stream>>>(g, cplx, ldo, d_out);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}

// The four Rayleigh-Ritz blocks of one contiguous block S (kept for direct
// checks of the contraction): Guu, Gvv, Guv, Ga.
extern "C" int bdgd_gram(bdgd_ctx *c, int prec, int cplx, uint64_t half, uint64_t k, const void *d_S, uint64_t lds,
                         const void *d_AS, uint64_t ldas, double *d_out) {
  if (k == 0) return BDGD_OK;
  const size_t esz = (size_t)(prec == BDGD_F32 ? 4 : 8) * (cplx ? 2 : 1);
  const char *S = (const char *)d_S, *AS = (const char *)d_AS;
  bdgd_gram_task t[5];
  memset(t, 0, sizeof t);
  const void *as[5] = {S, S + half * esz, S, S, S + half * esz};
  const void *bs[5] = {S, S + half * esz, S + half * esz, AS, AS + half * esz};
  const int outs[5] = {0, 1, 2, 3, 4};
  for (int i = 0; i < 5; ++i) {
    t[i].a = as[i];
    t[i].b = bs[i];
    t[i].lda = lds;
    t[i].ldb = (i >= 3) ? ldas : lds;
    t[i].rows = half;
    t[i].ka = t[i].kb = (int)k;
    t[i].out = outs[i];
    t[i].sym = (i < 2);
  }
  // Ga = Su^H ASu + Sv^H ASv: contract over all n rows in one task instead
  t[3].rows = 2 * half;
  int rc = bdgd_gram_tasks(c, prec, cplx, 4, t, (int)k, d_out);
  return rc;
}
// ---------------------------------------------------------------------------
// residuals and column norms
// ---------------------------------------------------------------------------
// Block reduction of sums of squares into part[col * nb + blockIdx.x].
template <typename T>
__device__ __forceinline__ void block_store(double v, double *part, int col, int nb) {
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    v = (l < (int)(blockDim.x >> 5)) ? red[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (l == 0) part[(long long)col * nb + blockIdx.x] = v;
  }
}

// R = AX - lam * swap(X) over columns; partial sums of |R|^2 and |X|^2.
// Elements are scalars of type T (complex data passed as 2*n reals with
// es = 2: the swap and the real lambda act on both components alike).
template <typename T>
__global__ void k_residual(const T *__restrict__ X, const T *__restrict__ AX, long long ld, T *__restrict__ Rout,
                           long long ldr, const double *__restrict__ lam, long long half_el, double *part_r,
                           double *part_x, const int *__restrict__ colmap) {
  const int col = blockIdx.y;
  const int src = colmap ? colmap[col] : col;
  const int nb = gridDim.x;
  const T *x = X + src * ld;
  const T *ax = AX + src * ld;
  T *r = Rout ? Rout + col * ldr : nullptr;
  const double l = lam[src];
  const long long n_el = 2 * half_el;
  double sr = 0.0, sx = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n_el; i += (long long)nb * blockDim.x) {
    const long long sw = (i < half_el) ? i + half_el : i - half_el;
    const double xv = (double)x[i];
    const double rv = (double)ax[i] - l * (double)x[sw];
    if (r) r[i] = (T)rv;
    sr += rv * rv;
    sx += xv * xv;
  }
  block_store<T>(sr, part_r, col, nb);
  block_store<T>(sx, part_x, col, nb);
}

// t = KMv - lam^2 v for the v rows of X (v at X + half_el, ld); partial
// sums of |t|^2 and |v|^2.
template <typename T>
__global__ void k_true_residual(const T *__restrict__ KMv, long long ldk, const T *__restrict__ X, long long ld,
                                const double *__restrict__ lam, long long half_el, double *part_t, double *part_v) {
  const int col = blockIdx.y;
  const int nb = gridDim.x;
  const T *km = KMv + col * ldk;
  const T *v = X + col * ld + half_el;
  const double l2 = lam[col] * lam[col];
  double st = 0.0, sv = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < half_el; i += (long long)nb * blockDim.x) {
    const double vv = (double)v[i];
    const double t = (double)km[i] - l2 * vv;
    st += t * t;
    sv += vv * vv;
  }
  block_store<T>(st, part_t, col, nb);
  block_store<T>(sv, part_v, col, nb);
}

__global__ void k_sum_parts(const double *__restrict__ part, int nb, int ncol, double *__restrict__ out) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= ncol) return;
  double s = 0.0;
  for (int b = 0; b < nb; ++b) s += part[(long long)col * nb + b];
  out[col] = s;
}

static int norm_blocks(long long n) {
  long long nb = (n + 255) / 256;
  if (nb > 64) nb = 64;
  return (int)(nb < 1 ? 1 : nb);
}

extern "C" int bdgd_residual(bdgd_ctx *c, int prec, int cplx, uint64_t half, uint64_t ncol, const void *d_X,
                             const void *d_AX, uint64_t ld, void *d_R, uint64_t ldr, const double *d_lam,
                             double *d_work, double *d_rr, double *d_xx, const int *d_colmap) {
  const int es = cplx ? 2 : 1;
  const long long half_el = (long long)half * es;
  const int nb = norm_blocks(2 * half_el);
  double *pr = d_work, *px = d_work + (long long)nb * ncol;
  dim3 grid(nb, (unsigned)ncol);
  bdgd_count_launch();
  if (prec == BDGD_F32)
    k_residual<float><<<grid, 256, 0, c->stream>>>((const float *)d_X, (const float *)d_AX, (long long)ld * es,
                                                   (float *)d_R, (long long)ldr * es, d_lam, half_el, pr, px, d_colmap);
  else
    k_residual<double><<<grid, 256, 0, c->stream>>>((const double *)d_X, (const double *)d_AX, (long long)ld * es,
                                                    (double *)d_R, (long long)ldr * es, d_lam, half_el, pr, px, d_colmap);
  BDGD_CK(cudaGetLastError());
  bdgd_count_launch();
  k_sum_parts<<<((int)ncol + 127) / 128, 128, 0, c->stream>>>(pr, nb, (int)ncol, d_rr);
  bdgd_count_launch();
  k_sum_parts<<<((int)ncol + 127) / 128, 128, 0, c->stream>>>(px, nb, (int)ncol, d_xx);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}

extern "C" int bdgd_true_residual(bdgd_ctx *c, int prec, int cplx, uint64_t half, uint64_t ncol, const void *d_KMv,
                                  uint64_t ldk, const void *d_X, uint64_t ld, const double *d_lam, double *d_work,
                                  double *d_tt, double *d_vv) {
  const int es = cplx ? 2 : 1;
  const long long half_el = (long long)half * es;
  const int nb = norm_blocks(half_el);
  double *pt = d_work, *pv = d_work + (long long)nb * ncol;
  dim3 grid(nb, (unsigned)ncol);
  bdgd_count_launch();
  if (prec == BDGD_F32)
    k_true_residual<float><<<grid, 256, 0, c->stream>>>((const float *)d_KMv, (long long)ldk * es,
                                                        (const float *)d_X, (long long)ld * es, d_lam, half_el, pt,
                                                        pv);
  else
    k_true_residual<double><<<grid, 256, 0, c->stream>>>((const double *)d_KMv, (long long)ldk * es,
                                                         (const double *)d_X, (long long)ld * es, d_lam, half_el, pt,
                                                         pv);
  BDGD_CK(cudaGetLastError());
  bdgd_count_launch();
  k_sum_parts<<<((int)ncol + 127) / 128, 128, 0, c->stream>>>(pt, nb, (int)ncol, d_tt);
  bdgd_count_launch();
  k_sum_parts<<<((int)ncol + 127) / 128, 128, 0, c->stream>>>(pv, nb, (int)ncol, d_vv);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}

// ---------------------------------------------------------------------------
// precision conversion
// ---------------------------------------------------------------------------
__global__ void k_d2f(const double *__restrict__ a, float *__restrict__ b, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}
__global__ void k_f2d(const float *__restrict__ a, double *__restrict__ b, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = (double)a[i];
}

extern "C" int bdgd_convert(bdgd_ctx *c, int to_f32, const void *src, void *dst, uint64_t n_scalars) {
  long long nb = ((long long)n_scalars + 255) / 256;
  if (nb > 8192) nb = 8192;
  if (nb < 1) nb = 1;
  bdgd_count_launch();
  if (to_f32)
    k_d2f<<<(int)nb, 256, 0, c->stream>>>((const double *)src, (float *)dst, (long long)n_scalars);
  else
    k_f2d<<<(int)nb, 256, 0, c->stream>>>((const float *)src, (double *)dst, (long long)n_scalars);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}

// ---------------------------------------------------------------------------
// small dense helpers for the Rayleigh-Ritz step (k <= a few hundred)
// matrices column-major, leading dimension = rows; complex interleaved.
// ---------------------------------------------------------------------------
// From the Gram outputs G = S^H S, Ga = S^H A S, Guv = S_u^H S_v (k x k,
// leading dimension ldo): Gs = D G D with D = diag(G)^-1/2 (d returned),
// Gb = Guv + Guv^H, Ga <- (Ga + Ga^H)/2.  G may be null when only the
// scaling of another matrix is wanted (then d is computed from Gs input).
__global__ void k_rr_prepare(const double *__restrict__ G, const double *__restrict__ Gain,
                             const double *__restrict__ Guv, int k, int ldo, int cplx, double *__restrict__ Gs,
                             double *__restrict__ Gb, double *__restrict__ Ga, double *__restrict__ d) {
  const long long kk = (long long)k * k;
  const int es = cplx ? 2 : 1;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < kk; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % k), j = (int)(q / k);
    const long long ij = (long long)j * ldo + i, ji = (long long)i * ldo + j;
    const long long oij = (long long)j * k + i;
    const double gii = G[((long long)i * ldo + i) * es], gjj = G[((long long)j * ldo + j) * es];
    const double di = gii > 0 ? 1.0 / sqrt(gii) : 1.0;
    const double dj = gjj > 0 ? 1.0 / sqrt(gjj) : 1.0;
    if (j == 0) d[i] = di;
    if (!cplx) {
      Gs[oij] = di * (0.5 * (G[ij] + G[ji])) * dj;
      if (Gb) Gb[oij] = Guv[ij] + Guv[ji];
      if (Ga) Ga[oij] = 0.5 * (Gain[ij] + Gain[ji]);
    } else {
      Gs[2 * oij] = di * (0.5 * (G[2 * ij] + G[2 * ji])) * dj;
      Gs[2 * oij + 1] = di * (0.5 * (G[2 * ij + 1] - G[2 * ji + 1])) * dj;
      if (Gb) {
        Gb[2 * oij] = Guv[2 * ij] + Guv[2 * ji];
        Gb[2 * oij + 1] = Guv[2 * ij + 1] - Guv[2 * ji + 1];
      }
      if (Ga) {
        Ga[2 * oij] = 0.5 * (Gain[2 * ij] + Gain[2 * ji]);
        Ga[2 * oij + 1] = 0.5 * (Gain[2 * ij + 1] - Gain[2 * ji + 1]);
      }
    }
  }
}

// Out[:, j] = diag(rowscale) * In[:, col0 + j] * colscale[col0 + j] (colscale^-1/2 applied
// when invsqrt); rowscale may be null.
__global__ void k_scale_cols(const double *__restrict__ In, int rows, int col0, int ncols, int cplx,
                             const double *__restrict__ rowscale, const double *__restrict__ colval, int invsqrt,
                             int reverse, double *__restrict__ Out) {
  const int es = cplx ? 2 : 1;
  const long long tot = (long long)rows * ncols;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % rows), j = (int)(q / rows);
    const int src = reverse ? (col0 + ncols - 1 - j) : (col0 + j);
    double s = 1.0;
    if (colval) s = invsqrt ? 1.0 / sqrt(colval[src]) : colval[src];
    if (rowscale) s *= rowscale[i];
    for (int e = 0; e < es; ++e) Out[((long long)j * rows + i) * es + e] = In[((long long)src * rows + i) * es + e] * s;
  }
}

__global__ void k_hermitize(double *__restrict__ A, int k, int cplx) {
  const long long kk = (long long)k * k;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < kk; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % k), j = (int)(q / k);
    if (i >= j) continue;
    const long long ij = (long long)j * k + i, ji = (long long)i * k + j;
    if (!cplx) {
      const double v = 0.5 * (A[ij] + A[ji]);
      A[ij] = v;
      A[ji] = v;
    } else {
      const double re = 0.5 * (A[2 * ij] + A[2 * ji]);
      const double im = 0.5 * (A[2 * ij + 1] - A[2 * ji + 1]);
      A[2 * ij] = re;
      A[2 * ij + 1] = im;
      A[2 * ji] = re;
      A[2 * ji + 1] = -im;
    }
  }
}

// lam[j] = 1/theta of the selected (descending theta) eigenvalues
__global__ void k_clamp(double *__restrict__ w, int n, double floor_rel) {
  __shared__ double mx;
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int i = 0; i < n; ++i) m = fmax(m, w[i]);
    mx = m;
  }
  __syncthreads();
  const double fl = floor_rel * mx;
  for (int i = threadIdx.x; i < n; i += blockDim.x) w[i] = fmax(w[i], fl);
}

static int grid_for(long long n) {
  long long b = (n + 255) / 256;
  if (b > 1024) b = 1024;
  return (int)(b < 1 ? 1 : b);
}

extern "C" int bdgd_rr_prepare(bdgd_ctx *c, const double *G, const double *Ga_in, const double *Guv, int k, int ldo,
                               int cplx, double *Gs, double *Gb, double *Ga, double *d) {
  bdgd_count_launch();
  k_rr_prepare<<<grid_for((long long)k * k), 256, 0, c->stream>>>(G, Ga_in, Guv, k, ldo, cplx, Gs, Gb, Ga, d);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}

extern "C" int bdgd_scale_cols(bdgd_ctx *c, const double *In, int rows, int col0, int ncols, int cplx,
                               const double *rowscale, const double *colval, int invsqrt, int reverse, double *Out) {
  bdgd_count_launch();
  k_scale_cols<<<grid_for((long long)rows * ncols), 256, 0, c->stream>>>(In, rows, col0, ncols, cplx, rowscale,
                                                                          colval, invsqrt, reverse, Out);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}

extern "C" int bdgd_hermitize(bdgd_ctx *c, double *A, int k, int cplx) {
  bdgd_count_launch();
  k_hermitize<<<grid_for((long long)k * k), 256, 0, c->stream>>>(A, k, cplx);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}

extern "C" int bdgd_clamp(bdgd_ctx *c, double *w, int n, double floor_rel) {
  bdgd_count_launch();
  k_clamp<<<1, 256, 0, c->stream>>>(w, n, floor_rel);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}

// out[i] = in[i]^e for in[i] > 0, else 0
__global__ void k_vec_pow(const double *__restrict__ in, int n, double e, double *__restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = in[i] > 0 ? pow(in[i], e) : 0.0;
}

extern "C" int bdgd_vec_pow(bdgd_ctx *c, const double *in, int n, double e, double *out) {
  bdgd_count_launch();
  k_vec_pow<<<(n + 255) / 256, 256, 0, c->stream>>>(in, n, e, out);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}

// Out[:, j] = In[:, cols[j]] (rows x ncols, FP64 or complex, leading dims ldi / ldo)
__global__ void k_gather_cols(const double *__restrict__ In, int ldi, int rows, const int *__restrict__ cols,
                              int ncols, int cplx, double *__restrict__ Out, int ldo) {
  const int es = cplx ? 2 : 1;
  const long long tot = (long long)rows * ncols;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % rows), j = (int)(q / rows);
    for (int e = 0; e < es; ++e) Out[((long long)j * ldo + i) * es + e] = In[((long long)cols[j] * ldi + i) * es + e];
  }
}

extern "C" int bdgd_gather_cols(bdgd_ctx *c, const double *In, int ldi, int rows, const int *d_cols, int ncols,
                                int cplx, double *Out, int ldo) {
  bdgd_count_launch();
  k_gather_cols<<<grid_for((long long)rows * ncols), 256, 0, c->stream>>>(In, ldi, rows, d_cols, ncols, cplx, Out,
                                                                           ldo);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}

// ---------------------------------------------------------------------------
// Gram contraction without any allocation
// ---------------------------------------------------------------------------
// Some callers cannot allocate device memory at the time they need the Gram
// blocks: code that runs under a memory pool or arena it does not own, a
// host framework that forbids cudaMalloc/cudaFree on its hot path (they
// synchronise the device), or a process that has handed all device memory to
// another allocator.  For them the split partial sums live in this fixed
// array, which every GPU that loads the library holds until exit.
#define BDGD_NOALLOC_SCRATCH_DOUBLES (1u << 20) /* 8 MiB */
static __device__ __align__(256) double g_gram_noalloc_scratch[BDGD_NOALLOC_SCRATCH_DOUBLES];

#define BDGD_NOALLOC_MAX_DEVICES 64
static std::atomic<double *> g_noalloc_ptr[BDGD_NOALLOC_MAX_DEVICES];

// Device address of the scratch array on the current device, looked up once
// per device (the host-side symbol is not a device address).
static int noalloc_scratch(double **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return bdgd_check(e, "cudaGetDevice");
  if (dev < 0 || dev >= BDGD_NOALLOC_MAX_DEVICES) {
    bdgd_set_error("bdgd_gram_noalloc: device ordinal %d above %d", dev, BDGD_NOALLOC_MAX_DEVICES);
    return BDGD_ERR_UNSUPPORTED;
  }
  if (!g_noalloc_ptr[dev]) {
    double *p = nullptr;
    e = cudaGetSymbolAddress((void **)&p, g_gram_noalloc_scratch);
    if (e != cudaSuccess) return bdgd_check(e, "cudaGetSymbolAddress(g_gram_noalloc_scratch)");
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return BDGD_OK;
}

extern "C" int bdgd_gram_noalloc(void *stream, int prec, int cplx, uint64_t half, uint64_t k, const void *d_S,
                                 uint64_t lds, const void *d_AS, uint64_t ldas, double *d_out) {
  if (k == 0) return BDGD_OK;
  if (!d_S || !d_AS || !d_out) {
    bdgd_set_error("bdgd_gram_noalloc: null pointer");
    return BDGD_ERR_ARG;
  }
  const int es = cplx ? 2 : 1;
  const unsigned long long per_split = 4ull * k * k * (unsigned long long)es;
  if (per_split > BDGD_NOALLOC_SCRATCH_DOUBLES) {
    bdgd_set_error("bdgd_gram_noalloc: k = %llu needs %llu bytes of scratch, above the %u-byte static buffer",
                   (unsigned long long)k, per_split * 8ull, BDGD_NOALLOC_SCRATCH_DOUBLES * 8u);
    return BDGD_ERR_ARG;
  }
  double *scratch = nullptr;
  int rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  const size_t esz = (size_t)(prec == BDGD_F32 ? 4 : 8) * (cplx ? 2 : 1);
  const char *S = (const char *)d_S, *AS = (const char *)d_AS;
  // tasks: Guu = Su^H Su, Gvv = Sv^H Sv, Guv = Su^H Sv, Ga = S^H AS
  GArgs g;
  memset(&g, 0, sizeof g);
  g.nt = 4;
  const void *as[4] = {S, S + half * esz, S, S};
  const void *bs[4] = {S, S + half * esz, S + half * esz, AS};
  long long maxrows = 0;
  int tiles = 0;
  for (int i = 0; i < 4; ++i) {
    GTask &t = g.t[i];
    t.a = as[i];
    t.b = bs[i];
    t.lda = (long long)lds;
    t.ldb = (long long)(i == 3 ? ldas : lds);
    t.rows = (long long)(i == 3 ? 2 * half : half);
    t.ka = t.kb = (int)k;
    t.out = i;
    t.sym = (i < 2);
    t.ta = t.tb = (int)((k + GT - 1) / GT);
    t.tile0 = tiles;
    tiles += t.sym ? t.ta * (t.ta + 1) / 2 : t.ta * t.tb;
    if (t.rows > maxrows) maxrows = t.rows;
  }
  g.ntiles = tiles;
  int nsplit = (4 * 148 + tiles - 1) / tiles;
  const int fit = (int)(BDGD_NOALLOC_SCRATCH_DOUBLES / per_split);
  if (nsplit > fit) nsplit = fit;
  const long long maxsplit = (maxrows + 8 * GRK - 1) / (8 * GRK);
  if (nsplit > maxsplit) nsplit = (int)maxsplit;
  if (nsplit < 1) nsplit = 1;
  long long chunk = (maxrows + nsplit - 1) / nsplit;
  chunk = (chunk + GRK - 1) / GRK * GRK;
  if (chunk < GRK) chunk = GRK;
  nsplit = (int)((maxrows + chunk - 1) / chunk);
  if (nsplit < 1) nsplit = 1;
  g.nsplit = nsplit;
  g.chunk = chunk;
  long long off = 0;
  for (int i = 0; i < 4; ++i) {
    g.t[i].part0 = off;
    off += (long long)nsplit * g.t[i].ka * g.t[i].kb * es;
  }
  g.part = scratch;
  cudaStream_t st = (cudaStream_t)stream;
  const size_t sm = sizeof(double) * GT * GLD * (cplx ? 4 : 2);
  dim3 grid(tiles, nsplit);
  if (prec == BDGD_F32) {
    if (cplx) {
      BDGD_CK(cudaFuncSetAttribute(k_gram_tasks<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      bdgd_count_launch();
      k_gram_tasks<float, true><<<grid, 128, sm, st>>>(g);
    } else {
      bdgd_count_launch();
      k_gram_tasks<float, false><<<grid, 128, sm, st>>>(g);
    }
  } else {
    if (cplx) {
      BDGD_CK(cudaFuncSetAttribute(k_gram_tasks<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      bdgd_count_launch();
      k_gram_tasks<double, true><<<grid, 128, sm, st>>>(g);
    } else {
      bdgd_count_launch();
      k_gram_tasks<double, false><<<grid, 128, sm, st>>>(g);
    }
  }
  BDGD_CK(cudaGetLastError());
  bdgd_count_launch();
  k_gram_tasks_reduce<<<dim3(32, 4), 256, 0, st>>>(g, cplx, (int)k, d_out);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}

// X-X blocks of the Rayleigh-Ritz Grams for a Ritz block X (B-orthonormal,
// A-diagonal): Ga(0:m, 0:m) = diag(lam), Guv(0:m, 0:m) = I/2 (so that
// Guv + Guv^H = X^H B X = I).  Leading dimension ldo.
__global__ void k_set_ritz_block(double *__restrict__ Ga, double *__restrict__ Guv, int ldo, int m, int cplx,
                                 const double *__restrict__ lam) {
  const int es = cplx ? 2 : 1;
  const long long mm = (long long)m * m;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < mm; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % m), j = (int)(q / m);
    const long long o = ((long long)j * ldo + i) * es;
    Ga[o] = (i == j) ? lam[i] : 0.0;
    Guv[o] = (i == j) ? 0.5 : 0.0;
    if (cplx) {
      Ga[o + 1] = 0.0;
      Guv[o + 1] = 0.0;
    }
  }
}

extern "C" int bdgd_set_ritz_block(bdgd_ctx *c, double *Ga, double *Guv, int ldo, int m, int cplx,
                                   const double *d_lam) {
  bdgd_count_launch();
  k_set_ritz_block<<<grid_for((long long)m * m), 256, 0, c->stream>>>(Ga, Guv, ldo, m, cplx, d_lam);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}

// ---------------------------------------------------------------------------
// Block update Y_o = alpha_o * sum_b S_ob C_ob + beta_o * Y_o (FP64, real).
//
// The basis updates of iLOBPCG (X <- [X, P, W] C_x, P <- [P, W] C_p and their
// A-images, the projections P -= X (X^H X)^+ X^H P and W -= Q (...), the SVQB
// rotations) are n x k by k x ncol products with n = 2 N^3 rows and k, ncol
// at most a few hundred: the other half of the solver's FP64 work beside the
// Gram.  One launch serves up to UMAXO outputs, each a sum of up to three
// terms, so X, AX, P, AP of the update step come out of one pass.  Tiles: 64
// rows x 64 output columns per 128-thread block (four warps of 32 x 32), the
// contraction walked in 16-column stages through a cp.async ring: the S
// stage as [16 columns][64 rows] (16-byte copies along the contiguous rows),
// the small matrix C as [64 output columns][16] (8-byte copies, it may have
// any leading dimension).  Products on the FP64 tensor cores (mma.sync
// m8n8k4).  The blocks are persistent; each takes the output column tasks of
// its row tiles in turn, so S tiles shared by several outputs come from L2.
// ---------------------------------------------------------------------------
#define UMAXO 4
#define UMAXCT 16
#define UKC 16   // contraction columns per stage
#define ULDM 68  // S stage row: 64 rows + 4 (the 16 fragment addresses of a half-warp fall in distinct banks)
#define ULDK 20  // C stage row: UKC + 4

struct UTerm {
  const double *s;
  const double *c;
  int k, ldc;
};
struct UOut {
  double *y;
  int ncol, nterm;
  double alpha, beta;
  UTerm t[3];
};
struct UArgs {
  UOut o[UMAXO];
  long long n, ld;
  int nct;
  signed char ct_out[UMAXCT], ct_col[UMAXCT];
};

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, int src_bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}

// stage j of term tm: S columns [UKC j, UKC j + UKC) of rows [r0, r0 + 64) as
// sA[column][row], and the matching UKC rows of C for output columns
// [c0, c0 + 64) as sB[output column][k]; out-of-range entries are zero-filled
__device__ __forceinline__ void upd_stage(double *sA, double *sB, const UTerm &tm, int j, long long r0, long long n,
                                          long long ld, int c0, int ncol) {
  const int kc0 = UKC * j;
  for (int q = threadIdx.x; q < UKC * 32; q += 128) {
    const int col = q >> 5, ch = q & 31;
    const long long row = r0 + 2 * ch;
    long long nv = n - row;
    nv = nv < 0 ? 0 : (nv > 2 ? 2 : nv);
    const bool ok = (kc0 + col) < tm.k && nv > 0;
    const double *src = ok ? tm.s + (long long)(kc0 + col) * ld + row : tm.s;
    cp_async16(sA + col * ULDM + 2 * ch, src, ok ? (int)(nv * 8) : 0);
  }
  for (int q = threadIdx.x; q < 64 * UKC; q += 128) {
    const int oc = q / UKC, kk = q % UKC;
    const bool ok = (c0 + oc) < ncol && (kc0 + kk) < tm.k;
    const double *src = ok ? tm.c + (long long)(c0 + oc) * tm.ldc + kc0 + kk : tm.c;
    cp_async8(sB + oc * ULDK + kk, src, ok ? 8 : 0);
  }
}

// stages of output column task ct (sum over its terms of ceil(k / UKC))
__device__ __forceinline__ int upd_nst(const UArgs &u, int ct) {
  const UOut &o = u.o[u.ct_out[ct]];
  int n = 0;
  for (int b = 0; b < o.nterm; ++b) n += (o.t[b].k + UKC - 1) / UKC;
  return n;
}

// Persistent: block b takes row tiles b, b + grid, ... and, for each, the
// column tasks 0..nct-1 in turn (their S tiles are shared through L2); all
// stages run through one USTG-deep cp.async ring (USTG - 1 stages loading
// while one is multiplied), so the loads of a tile's first stages overlap the
// previous tile's last products and its stores.
// With beta != 0 the accumulators start at (beta / alpha) Y, loaded together
// at the start of the tile (exact for the solver's alpha = +-1, beta = 1).
template <int USTG, int MINB>
__global__ void __launch_bounds__(128, MINB) k_block_update(UArgs u, long long nrt) {
  extern __shared__ __align__(16) unsigned char usm[];
  double *buf = (double *)usm;  // [USTG][A: UKC x ULDM | B: 64 x ULDK]
  constexpr int STG = UKC * ULDM + 64 * ULDK;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wi = warp & 1, wj = warp >> 1;
  const int lr = lane & 3, lc = lane >> 2;
  // load cursor: row tile lrt, column task lct, term lb, stage lj within the term
  long long lrt = blockIdx.x;
  int lct = 0, lb = 0, lj = 0;
  auto issue = [&](int slot) {
    // the next stage of the load cursor into ring slot `slot` (an empty group when done)
    if (lrt < nrt) {
      const UOut &o = u.o[u.ct_out[lct]];
      double *dst = buf + slot * STG;
      upd_stage(dst, dst + UKC * ULDM, o.t[lb], lj, lrt * 64, u.n, u.ld, 64 * u.ct_col[lct], o.ncol);
      if (++lj == (o.t[lb].k + UKC - 1) / UKC) {
        lj = 0;
        if (++lb == o.nterm) {
          lb = 0;
          if (++lct == u.nct) lct = 0, lrt += gridDim.x;
        }
      }
    }
    cp_async_commit();
  };
#pragma unroll
  for (int q = 0; q < USTG - 1; ++q) issue(q);
  double acc[4][4][2];
  int slot = 0;
  for (long long rt = blockIdx.x; rt < nrt; rt += gridDim.x)
    for (int ct = 0; ct < u.nct; ++ct) {
      const long long r0 = rt * 64;
      const UOut &o = u.o[u.ct_out[ct]];
      const int c0 = 64 * u.ct_col[ct];
      const int nst = upd_nst(u, ct);
      const double alpha = o.alpha, beta = o.beta;
      double *y = o.y;
      if (beta != 0.0) {
        const double sc = beta / alpha;
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
          for (int nj = 0; nj < 4; ++nj)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              const long long row = r0 + wi * 32 + mi * 8 + lc;
              const int col = c0 + wj * 32 + nj * 8 + 2 * lr + e;
              acc[mi][nj][e] = (row < u.n && col < o.ncol) ? sc * __ldcs(y + (long long)col * u.ld + row) : 0.0;
            }
      } else {
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
          for (int nj = 0; nj < 4; ++nj) acc[mi][nj][0] = acc[mi][nj][1] = 0.0;
      }
      for (int s = 0; s < nst; ++s) {
        cp_async_wait<USTG - 2>();
        __syncthreads();  // stage `slot` visible to all; the slot refilled below is no longer read
        issue((slot + USTG - 1) % USTG);
        const double *sA = buf + slot * STG, *sB = sA + UKC * ULDM;
#pragma unroll
        for (int kk = 0; kk < UKC; kk += 4) {
          double ar[4], br[4];
#pragma unroll
          for (int mi = 0; mi < 4; ++mi) ar[mi] = sA[(kk + lr) * ULDM + wi * 32 + mi * 8 + lc];
#pragma unroll
          for (int nj = 0; nj < 4; ++nj) br[nj] = sB[(wj * 32 + nj * 8 + lc) * ULDK + kk + lr];
#pragma unroll
          for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int nj = 0; nj < 4; ++nj) dmma(acc[mi][nj][0], acc[mi][nj][1], ar[mi], br[nj]);
        }
        slot = slot == USTG - 1 ? 0 : slot + 1;
      }
#pragma unroll
      for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int nj = 0; nj < 4; ++nj)
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const long long row = r0 + wi * 32 + mi * 8 + lc;
            const int col = c0 + wj * 32 + nj * 8 + 2 * lr + e;
            if (row < u.n && col < o.ncol) __stcs(y + (long long)col * u.ld + row, alpha * acc[mi][nj][e]);
          }
    }
  cp_async_wait<0>();
}

// resident blocks of a k_block_update variant on this device (queried once per device)
template <int USTG, int MINB>
static int upd_slots(size_t sm) {
  static std::atomic<int> cache[64];  // written by several solver threads: idempotent, atomic
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  if (cache[dev].load(std::memory_order_relaxed) <= 0) {
    int nb = 0, nsm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_block_update<USTG, MINB>, 128, sm) != cudaSuccess ||
        nb < 1)
      nb = 1;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm < 1) nsm = 148;
    cache[dev].store(nb * nsm, std::memory_order_relaxed);
  }
  return cache[dev].load(std::memory_order_relaxed);
}

template <int USTG, int MINB>
static int launch_update(bdgd_ctx *c, const UArgs &u, long long nrt) {
  const size_t sm = sizeof(double) * USTG * (UKC * ULDM + 64 * ULDK);
  if (!bdgd_capturing)
    BDGD_CK(cudaFuncSetAttribute(k_block_update<USTG, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  const long long slots = upd_slots<USTG, MINB>(sm);
  const long long nblk = nrt < slots ? nrt : slots;
  bdgd_count_launch();
  k_block_update<USTG, MINB><<<(unsigned)nblk, 128, sm, c->stream>>>(u, nrt);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}

extern "C" int bdgd_block_update_oz(bdgd_ctx *c, uint64_t n, uint64_t ld, int nout, const bdgd_update_out *outs);

// Tensor-core (int8 digits, tcgen05) FP64 update: on with BDG_UPDATE_TC=1
static bool update_tc_on() {
  const char *e = getenv("BDG_UPDATE_TC");
  return e && e[0] == '1';
}

extern "C" int bdgd_block_update(bdgd_ctx *c, int prec, int cplx, uint64_t n, uint64_t ld, int nout,
                                 const bdgd_update_out *outs) {
  if (nout <= 0 || n == 0) return BDGD_OK;
  if (prec == BDGD_F64 && !cplx && update_tc_on()) {
    const int rc = bdgd_block_update_oz(c, n, ld, nout, outs);
    if (rc != BDGD_ERR_UNSUPPORTED) return rc;
  }
  if (prec != BDGD_F64 || cplx || nout > UMAXO || ld < n || (ld & 1)) return BDGD_ERR_UNSUPPORTED;
  UArgs u;
  memset(&u, 0, sizeof u);
  u.n = (long long)n;
  u.ld = (long long)ld;
  int nct = 0;
  for (int i = 0; i < nout; ++i) {
    const bdgd_update_out &s = outs[i];
    if (s.nterm < 0 || s.nterm > 3 || s.ncol < 0 || ((uintptr_t)s.y % 8)) return BDGD_ERR_UNSUPPORTED;
    UOut &o = u.o[i];
    o.y = (double *)s.y;
    o.ncol = s.ncol;
    o.nterm = 0;
    o.alpha = s.alpha;
    o.beta = s.beta;
    for (int b = 0; b < s.nterm; ++b) {
      if (s.term[b].k <= 0) continue;
      if (((uintptr_t)s.term[b].s % 16) || s.term[b].ldc < s.term[b].k || ((uintptr_t)s.term[b].c % 8))
        return BDGD_ERR_UNSUPPORTED;
      UTerm &t = o.t[o.nterm++];
      t.s = (const double *)s.term[b].s;
      t.c = s.term[b].c;
      t.k = s.term[b].k;
      t.ldc = s.term[b].ldc;
    }
    for (int j = 0; o.nterm > 0 && j * 64 < s.ncol; ++j) {  // no terms: Y untouched
      if (nct == UMAXCT) return BDGD_ERR_UNSUPPORTED;
      u.ct_out[nct] = (signed char)i;
      u.ct_col[nct] = (signed char)j;
      nct++;
    }
  }
  if (nct == 0) return BDGD_OK;
  u.nct = nct;
  const long long nrt = ((long long)n + 63) / 64;
  // four-deep ring at three blocks per SM: inside the 128^3 solve its update
  // stage took 778 ms against 822 ms for the double-buffered ring at four
  // blocks per SM (BDG_UPDATE_VARIANT=2), although the latter times faster
  // alone (12.8 against 13.5 ms per update)
  const char *v = getenv("BDG_UPDATE_VARIANT");
  if (v && v[0] == '2') return launch_update<2, 4>(c, u, nrt);
  return launch_update<4, 3>(c, u, nrt);
}
