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
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "bdg_dev.h"
#include "bdg_blas.h"

// ---------------------------------------------------------------------------
// Gram contraction
// ---------------------------------------------------------------------------
#define GT 64    // output tile (GT x GT)
#define GRK 32   // contraction rows per shared-memory stage
#define GLD (GRK + 4)

struct GramProb {
  const void *a;   // A base (element (r, i) at a[(i*lda + r)*es + comp])
  const void *b;
  long long lda, ldb;
  long long rows;  // contraction length
  int comp_a, comp_b;
};

struct GramArgs {
  GramProb pr[20];
  int nprob;
  int k;
  int es;          // 1 real, 2 complex (interleaved)
  int nsplit;
  long long chunk; // rows per split (multiple of GRK)
  double *part;    // [nprob][nsplit][k][k]
};

__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

template <typename T>
__device__ __forceinline__ void stage_tile(double *sm, const T *__restrict__ base, long long ld, int es, int comp,
                                           int c0, int k, long long r0, long long rend) {
  // sm[c][r], c < GT, r < GRK; column c of the operand is contiguous along r
  for (int q = threadIdx.x; q < GT * GRK; q += blockDim.x) {
    const int c = q / GRK, r = q - c * GRK;
    const long long rr = r0 + r;
    double v = 0.0;
    if (c0 + c < k && rr < rend) v = (double)base[((long long)(c0 + c) * ld + rr) * es + comp];
    sm[c * GLD + r] = v;
  }
}

template <typename T>
__global__ void __launch_bounds__(128) k_gram(GramArgs g) {
  __shared__ __align__(16) double sA[GT * GLD];
  __shared__ __align__(16) double sB[GT * GLD];
  const int ntile = (g.k + GT - 1) / GT;
  const int ti = blockIdx.x % ntile, tj = blockIdx.x / ntile;
  const int split = blockIdx.y, p = blockIdx.z;
  const GramProb pr = g.pr[p];
  const long long rbeg = (long long)split * g.chunk;
  long long rend = rbeg + g.chunk;
  if (rend > pr.rows) rend = pr.rows;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wi = warp & 1, wj = warp >> 1;  // 2 x 2 warps, 32 x 32 each
  double acc[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
  const T *A = (const T *)pr.a;
  const T *B = (const T *)pr.b;
  const int lr = lane & 3, lc = lane >> 2;
  for (long long r0 = rbeg; r0 < rend; r0 += GRK) {
    stage_tile<T>(sA, A, pr.lda, g.es, pr.comp_a, ti * GT, g.k, r0, rend);
    stage_tile<T>(sB, B, pr.ldb, g.es, pr.comp_b, tj * GT, g.k, r0, rend);
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < GRK; kk += 4) {
      double af[4], bf[4];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi) af[mi] = sA[(wi * 32 + mi * 8 + lc) * GLD + kk + lr];
#pragma unroll
      for (int nj = 0; nj < 4; ++nj) bf[nj] = sB[(wj * 32 + nj * 8 + lc) * GLD + kk + lr];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int nj = 0; nj < 4; ++nj) dmma(acc[mi][nj][0], acc[mi][nj][1], af[mi], bf[nj]);
    }
    __syncthreads();
  }
  // D fragment: row = lane >> 2, cols 2*(lane & 3) + {0, 1}
  double *out = g.part + ((long long)p * g.nsplit + split) * (long long)g.k * g.k;
#pragma unroll
  for (int mi = 0; mi < 4; ++mi)
#pragma unroll
    for (int nj = 0; nj < 4; ++nj)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int i = ti * GT + wi * 32 + mi * 8 + lc;
        const int j = tj * GT + wj * 32 + nj * 8 + 2 * lr + e;
        if (i < g.k && j < g.k) out[(long long)j * g.k + i] = acc[mi][nj][e];  // column-major
      }
}

// out[b] (k x k, column-major, real or interleaved complex) =
//   sum over terms t of block b/component c: sign * sum_split part[prob]
struct GramReduce {
  int nterm[8];        // per (block, comp) slot: block*2 + comp
  int prob[8][4];
  double sign[8][4];
  int nblk, cplx, k, nsplit;
};

__global__ void k_gram_reduce(GramReduce R, const double *__restrict__ part, double *__restrict__ out) {
  const long long kk = (long long)R.k * R.k;
  const int ncomp = R.cplx ? 2 : 1;
  const long long total = kk * R.nblk * ncomp;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const long long e = q % kk;
    const long long bc = q / kk;  // block*ncomp + comp
    const int blk = (int)(bc / ncomp), comp = (int)(bc % ncomp);
    const int slot = blk * 2 + comp;
    double s = 0.0;
    for (int t = 0; t < R.nterm[slot]; ++t) {
      const double *pp = part + (long long)R.prob[slot][t] * R.nsplit * kk + e;
      double a = 0.0;
      for (int sp = 0; sp < R.nsplit; ++sp) a += pp[(long long)sp * kk];
      s += R.sign[slot][t] * a;
    }
    if (R.cplx)
      out[(blk * kk + e) * 2 + comp] = s;
    else
      out[blk * kk + e] = s;
  }
}

extern "C" int bdgd_gram(bdgd_ctx *c, int prec, int cplx, uint64_t half, uint64_t k, const void *d_S, uint64_t lds,
                         const void *d_AS, uint64_t ldas, double *d_out) {
  if (k == 0) return BDGD_OK;
  const int es = cplx ? 2 : 1;
  const size_t esz = (prec == BDGD_F32 ? 4 : 8);
  GramArgs g;
  memset(&g, 0, sizeof g);
  g.k = (int)k;
  g.es = es;
  GramReduce R;
  memset(&R, 0, sizeof R);
  R.nblk = 4;
  R.cplx = cplx;
  R.k = (int)k;
  // real contractions over rows [0, half): (A, B) pairs per output block
  //   0 Guu = Su^T Su   1 Gvv = Sv^T Sv   2 Guv = Su^T Sv   3 Ga = Su^T ASu + Sv^T ASv
  const char *S = (const char *)d_S;
  const char *AS = (const char *)d_AS;
  const char *Su = S, *Sv = S + half * es * esz;
  const char *Au = AS, *Av = AS + half * es * esz;
  struct Pair { const char *a, *b; long long la, lb; int blk; };
  Pair pairs[5] = {{Su, Su, (long long)lds, (long long)lds, 0},
                   {Sv, Sv, (long long)lds, (long long)lds, 1},
                   {Su, Sv, (long long)lds, (long long)lds, 2},
                   {Su, Au, (long long)lds, (long long)ldas, 3},
                   {Sv, Av, (long long)lds, (long long)ldas, 3}};
  int np = 0;
  for (int pi = 0; pi < 5; ++pi) {
    if (!cplx) {
      GramProb &q = g.pr[np];
      q.a = pairs[pi].a; q.b = pairs[pi].b; q.lda = pairs[pi].la; q.ldb = pairs[pi].lb;
      q.rows = (long long)half; q.comp_a = q.comp_b = 0;
      const int slot = pairs[pi].blk * 2;
      R.prob[slot][R.nterm[slot]] = np;
      R.sign[slot][R.nterm[slot]++] = 1.0;
      ++np;
    } else {
      // (Ar - i Ai)^T (Br + i Bi): re = Ar Br + Ai Bi, im = Ar Bi - Ai Br
      const int ca[4] = {0, 1, 0, 1}, cb[4] = {0, 1, 1, 0};
      const int comp[4] = {0, 0, 1, 1};
      const double sg[4] = {1.0, 1.0, 1.0, -1.0};
      for (int t = 0; t < 4; ++t) {
        GramProb &q = g.pr[np];
        q.a = pairs[pi].a; q.b = pairs[pi].b; q.lda = pairs[pi].la; q.ldb = pairs[pi].lb;
        q.rows = (long long)half; q.comp_a = ca[t]; q.comp_b = cb[t];
        const int slot = pairs[pi].blk * 2 + comp[t];
        R.prob[slot][R.nterm[slot]] = np;
        R.sign[slot][R.nterm[slot]++] = sg[t];
        ++np;
      }
    }
  }
  g.nprob = np;
  const int ntile = (int)((k + GT - 1) / GT);
  const int ctas_per_split = ntile * ntile * np;
  int nsplit = (4 * 148 + ctas_per_split - 1) / ctas_per_split;
  const long long maxsplit = ((long long)half + 4 * GRK - 1) / (4 * GRK);
  if (nsplit > maxsplit) nsplit = (int)maxsplit;
  if (nsplit < 1) nsplit = 1;
  long long chunk = ((long long)half + nsplit - 1) / nsplit;
  chunk = (chunk + GRK - 1) / GRK * GRK;
  nsplit = (int)(((long long)half + chunk - 1) / chunk);
  g.nsplit = nsplit;
  g.chunk = chunk;
  R.nsplit = nsplit;
  int rc = bdgd_ensure((void **)&c->gram_part, &c->gram_part_bytes, sizeof(double) * np * nsplit * k * k);
  if (rc) return rc;
  g.part = c->gram_part;
  dim3 grid(ntile * ntile, nsplit, np);
  if (prec == BDGD_F32)
    k_gram<float><<<grid, 128, 0, c->stream>>>(g);
  else
    k_gram<double><<<grid, 128, 0, c->stream>>>(g);
  BDGD_CK(cudaGetLastError());
  const long long tot = (long long)k * k * 4 * (cplx ? 2 : 1);
  int nb = (int)((tot + 255) / 256);
  if (nb > 2048) nb = 2048;
  k_gram_reduce<<<nb, 256, 0, c->stream>>>(R, c->gram_part, d_out);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
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
                           double *part_x) {
  const int col = blockIdx.y;
  const int nb = gridDim.x;
  const T *x = X + col * ld;
  const T *ax = AX + col * ld;
  T *r = Rout ? Rout + col * ldr : nullptr;
  const double l = lam[col];
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
                             double *d_work, double *d_rr, double *d_xx) {
  const int es = cplx ? 2 : 1;
  const long long half_el = (long long)half * es;
  const int nb = norm_blocks(2 * half_el);
  double *pr = d_work, *px = d_work + (long long)nb * ncol;
  dim3 grid(nb, (unsigned)ncol);
  if (prec == BDGD_F32)
    k_residual<float><<<grid, 256, 0, c->stream>>>((const float *)d_X, (const float *)d_AX, (long long)ld * es,
                                                   (float *)d_R, (long long)ldr * es, d_lam, half_el, pr, px);
  else
    k_residual<double><<<grid, 256, 0, c->stream>>>((const double *)d_X, (const double *)d_AX, (long long)ld * es,
                                                    (double *)d_R, (long long)ldr * es, d_lam, half_el, pr, px);
  BDGD_CK(cudaGetLastError());
  k_sum_parts<<<((int)ncol + 127) / 128, 128, 0, c->stream>>>(pr, nb, (int)ncol, d_rr);
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
  if (prec == BDGD_F32)
    k_true_residual<float><<<grid, 256, 0, c->stream>>>((const float *)d_KMv, (long long)ldk * es,
                                                        (const float *)d_X, (long long)ld * es, d_lam, half_el, pt,
                                                        pv);
  else
    k_true_residual<double><<<grid, 256, 0, c->stream>>>((const double *)d_KMv, (long long)ldk * es,
                                                         (const double *)d_X, (long long)ld * es, d_lam, half_el, pt,
                                                         pv);
  BDGD_CK(cudaGetLastError());
  k_sum_parts<<<((int)ncol + 127) / 128, 128, 0, c->stream>>>(pt, nb, (int)ncol, d_tt);
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
// G = Guu + Gvv, Gb = Guv + Guv^H, Ga = (Ga + Ga^H)/2, Gs = D G D with
// D = diag(G)^-1/2 (d returned).
__global__ void k_rr_prepare(const double *__restrict__ gram, int k, int cplx, double *__restrict__ Gs,
                             double *__restrict__ Gb, double *__restrict__ Ga, double *__restrict__ d) {
  const long long kk = (long long)k * k;
  const int es = cplx ? 2 : 1;
  const double *Guu = gram, *Gvv = gram + kk * es, *Guv = gram + 2 * kk * es, *Gaa = gram + 3 * kk * es;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < kk; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % k), j = (int)(q / k);
    const long long ij = (long long)j * k + i, ji = (long long)i * k + j;
    const double dii = Guu[((long long)i * k + i) * es] + Gvv[((long long)i * k + i) * es];
    const double djj = Guu[((long long)j * k + j) * es] + Gvv[((long long)j * k + j) * es];
    const double di = dii > 0 ? 1.0 / sqrt(dii) : 1.0;
    const double dj = djj > 0 ? 1.0 / sqrt(djj) : 1.0;
    if (j == 0) d[i] = di;
    if (!cplx) {
      const double g = 0.5 * ((Guu[ij] + Gvv[ij]) + (Guu[ji] + Gvv[ji]));
      Gs[ij] = di * g * dj;
      Gb[ij] = Guv[ij] + Guv[ji];
      Ga[ij] = 0.5 * (Gaa[ij] + Gaa[ji]);
    } else {
      // Hermitian parts: (M + M^H)/2, and Guv + Guv^H
      const double gre = 0.5 * ((Guu[2 * ij] + Gvv[2 * ij]) + (Guu[2 * ji] + Gvv[2 * ji]));
      const double gim = 0.5 * ((Guu[2 * ij + 1] + Gvv[2 * ij + 1]) - (Guu[2 * ji + 1] + Gvv[2 * ji + 1]));
      Gs[2 * ij] = di * gre * dj;
      Gs[2 * ij + 1] = di * gim * dj;
      Gb[2 * ij] = Guv[2 * ij] + Guv[2 * ji];
      Gb[2 * ij + 1] = Guv[2 * ij + 1] - Guv[2 * ji + 1];
      Ga[2 * ij] = 0.5 * (Gaa[2 * ij] + Gaa[2 * ji]);
      Ga[2 * ij + 1] = 0.5 * (Gaa[2 * ij + 1] - Gaa[2 * ji + 1]);
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

extern "C" int bdgd_rr_prepare(bdgd_ctx *c, const double *gram, int k, int cplx, double *Gs, double *Gb, double *Ga,
                               double *d) {
  k_rr_prepare<<<grid_for((long long)k * k), 256, 0, c->stream>>>(gram, k, cplx, Gs, Gb, Ga, d);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}

extern "C" int bdgd_scale_cols(bdgd_ctx *c, const double *In, int rows, int col0, int ncols, int cplx,
                               const double *rowscale, const double *colval, int invsqrt, int reverse, double *Out) {
  k_scale_cols<<<grid_for((long long)rows * ncols), 256, 0, c->stream>>>(In, rows, col0, ncols, cplx, rowscale,
                                                                          colval, invsqrt, reverse, Out);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}

extern "C" int bdgd_hermitize(bdgd_ctx *c, double *A, int k, int cplx) {
  k_hermitize<<<grid_for((long long)k * k), 256, 0, c->stream>>>(A, k, cplx);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}

extern "C" int bdgd_clamp(bdgd_ctx *c, double *w, int n, double floor_rel) {
  k_clamp<<<1, 256, 0, c->stream>>>(w, n, floor_rel);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}
