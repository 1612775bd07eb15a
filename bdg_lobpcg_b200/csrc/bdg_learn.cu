// bdg_learn.cu -- learned SPD preconditioner T = S^T S + exp(eta) P0:
// forward, adjoint, gradient and Adam kernels, inner CG for training
// targets.  The definitions (pooling, lift, spectral convolution in the
// real cos/sin basis, pointwise mix, loss and gradient) are those written
// out in include/bdg/bdg_learn.h; everything runs in FP32 except the fine
// grid vectors of the loss (FP64).
//
// Layouts (FP32, x fastest):
//   coarse fields    [batch][C][nz][ny][nx]
//   coefficients     [batch][C][R][R][R]        R = 2 modes - 1 rows per axis
//   axis basis E_d   [R][n_d]: rows cos(2 pi a x/n), a < modes, then
//                    sin(2 pi a x/n), 1 <= a < modes
//   parameters       A [C][F] | W [L][C][M][M][M] | B [L][C][C] | Dg [L][C][F] | eta
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "bdg/bdg_learn.h"
#include "bdg_dev.h"

#define LP_F 5       // conditioning fields
#define LP_CMAX 16   // channels (upper bound)

struct LPHalf {
  float *p, *g, *m, *v;
  int step;
};

struct bdg_lp {
  int N[3], n[3];
  long long S, nc;
  int C, L, M, R;
  long long np, oA, oW, oB, oD, oEta;
  int device;
  float *E[3];
  float *phi;
  int conditioned;
  LPHalf h[2];
  // workspace
  long long wsB;
  int wsTrain;
  float *rc[2], *acts[2], *gbuf[2], *sbuf, *co[2], *ax1, *ax2, *part;
  double *tr, *tq, *dots, *fac;
  long long part_n;
  // loss: L2 (energy = 0) or the energy norm of A = Op + esigma (energy = 1)
  int energy;
  double esigma;
  cublasHandle_t blas;  // axis contractions of the spectral convolutions (plain FP32 GEMMs)
  int fast;             // applies use TF32 tensor-core GEMMs (training always exact FP32)
};

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
__device__ __forceinline__ int lp_mode(int row, int M) { return row < M ? row : row - M + 1; }
__device__ __forceinline__ float lp_mult(int row, int M) { return lp_mode(row, M) == 0 ? 1.0f : 2.0f; }

#define GSTRIDE(i, n) for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

static unsigned lp_blocks(long long n) {
  long long b = (n + 255) / 256;
  if (b > 8192) b = 8192;
  if (b < 1) b = 1;
  return (unsigned)b;
}

// 2x2x2 average pooling of half-columns: rc[b][p]
template <typename TI>
__global__ void k_lp_pool(const TI *__restrict__ x, long long ldx, int B, int N0, int N1, int n0, int n1, int n2,
                          float *__restrict__ rc) {
  const long long nc = (long long)n0 * n1 * n2;
  GSTRIDE(i, (long long)B * nc) {
    const long long b = i / nc, p = i - b * nc;
    const int X = (int)(p % n0), Y = (int)((p / n0) % n1), Z = (int)(p / ((long long)n0 * n1));
    const TI *s = x + b * ldx;
    double acc = 0.0;
    for (int dz = 0; dz < 2; ++dz)
      for (int dy = 0; dy < 2; ++dy)
        for (int dx = 0; dx < 2; ++dx)
          acc += (double)s[((long long)(2 * Z + dz) * N1 + (2 * Y + dy)) * N0 + 2 * X + dx];
    rc[i] = (float)(acc * 0.125);
  }
}

// y = exp(eta) y + pool^T(rc) (replicate / 8) on half-columns
template <typename TO>
__global__ void k_lp_poolt_axpy(const float *__restrict__ rc, TO *__restrict__ y, long long ldy, int B, int N0, int N1,
                                int N2, const float *__restrict__ eta) {
  const long long S = (long long)N0 * N1 * N2;
  const int n0 = N0 / 2, n1 = N1 / 2;
  const long long nc = S / 8;
  const double s = exp((double)*eta);
  GSTRIDE(i, (long long)B * S) {
    const long long b = i / S, q = i - b * S;
    const int x = (int)(q % N0), yy = (int)((q / N0) % N1), z = (int)(q / ((long long)N0 * N1));
    const long long p = ((long long)(z / 2) * n1 + yy / 2) * n0 + x / 2;
    TO *d = y + b * ldy + q;
    *d = (TO)(s * (double)*d + 0.125 * (double)rc[b * nc + p]);
  }
}

// z0[b][c][p] = (sum_f A[c][f] phi[f][p]) rc[b][p]
__global__ void k_lp_lift(const float *__restrict__ rc, const float *__restrict__ A, const float *__restrict__ phi,
                          int B, int C, long long nc, float *__restrict__ z) {
  GSTRIDE(i, (long long)B * C * nc) {
    const long long p = i % nc, bc = i / nc;
    const int c = (int)(bc % C);
    const long long b = bc / C;
    float a = 0.f;
#pragma unroll
    for (int f = 0; f < LP_F; ++f) a += A[c * LP_F + f] * phi[f * nc + p];
    z[i] = a * rc[b * nc + p];
  }
}

// rc[b][p] = sum_c a_c(p) g[b][c][p]   (adjoint of the lift)
__global__ void k_lp_lift_adj(const float *__restrict__ g, const float *__restrict__ A, const float *__restrict__ phi,
                              int B, int C, long long nc, float *__restrict__ rc) {
  GSTRIDE(i, (long long)B * nc) {
    const long long b = i / nc, p = i - b * nc;
    float acc = 0.f;
    for (int c = 0; c < C; ++c) {
      float a = 0.f;
#pragma unroll
      for (int f = 0; f < LP_F; ++f) a += A[c * LP_F + f] * phi[f * nc + p];
      acc += a * g[(b * C + c) * nc + p];
    }
    rc[i] = acc;
  }
}

// co *= w_l[c] (filter of one layer, W = this layer's [C][M][M][M])
__global__ void k_lp_filter(float *__restrict__ co, const float *__restrict__ W, int B, int C, int R, int M,
                            float inv_nc) {
  const long long R3 = (long long)R * R * R;
  GSTRIDE(idx, (long long)B * C * R3) {
    const int ri = (int)(idx % R), rj = (int)((idx / R) % R), rk = (int)((idx / ((long long)R * R)) % R);
    const int c = (int)((idx / R3) % C);
    const float w = W[(((long long)c * M + lp_mode(rk, M)) * M + lp_mode(rj, M)) * M + lp_mode(ri, M)] *
                    lp_mult(rk, M) * lp_mult(rj, M) * lp_mult(ri, M) * inv_nc;
    co[idx] *= w;
  }
}

// gW[c][az][ay][ax] += sum_b sum_rows pz * pg * mult / nc (one writer per entry)
__global__ void k_lp_filter_grad(const float *__restrict__ pz, const float *__restrict__ pg, float *__restrict__ gW,
                                 int B, int C, int R, int M, float inv_nc) {
  const long long R3 = (long long)R * R * R;
  GSTRIDE(idx, (long long)C * M * M * M) {
    const int ax = (int)(idx % M), ay = (int)((idx / M) % M), az = (int)((idx / ((long long)M * M)) % M);
    const int c = (int)(idx / ((long long)M * M * M));
    int rz[2], ry[2], rx[2];
    const int nz = az ? 2 : 1, ny = ay ? 2 : 1, nx = ax ? 2 : 1;
    rz[0] = az;
    rz[1] = M - 1 + az;
    ry[0] = ay;
    ry[1] = M - 1 + ay;
    rx[0] = ax;
    rx[1] = M - 1 + ax;
    const float mult = (az ? 2.f : 1.f) * (ay ? 2.f : 1.f) * (ax ? 2.f : 1.f) * inv_nc;
    double acc = 0.0;
    for (int b = 0; b < B; ++b) {
      const long long base = ((long long)b * C + c) * R3;
      for (int u = 0; u < nz; ++u)
        for (int v = 0; v < ny; ++v)
          for (int w = 0; w < nx; ++w) {
            const long long e = base + ((long long)rz[u] * R + ry[v]) * R + rx[w];
            acc += (double)pz[e] * (double)pg[e];
          }
    }
    gW[idx] += (float)(acc * mult);
  }
}

// out = z + s + PM(z)  (transpose: PM^T), PM(z)[c] = sum_c' Bm[c][c'] z[c'] + (sum_f Dg[c][f] phi_f) z[c]
// C is a compile-time channel count (the channel values stay in registers);
// the layer's mix weights are staged in shared memory.
template <int C>
__global__ void __launch_bounds__(256) k_lp_layer(const float *__restrict__ z, const float *__restrict__ s,
                                                  float *__restrict__ out, const float *__restrict__ Bm,
                                                  const float *__restrict__ Dg, const float *__restrict__ phi, int B,
                                                  long long nc, int transpose) {
  __shared__ float sB[C * C], sD[C * LP_F];
  for (int i = threadIdx.x; i < C * C; i += blockDim.x) {
    const int r = i / C, q = i - r * C;
    sB[i] = transpose ? Bm[q * C + r] : Bm[i];
  }
  for (int i = threadIdx.x; i < C * LP_F; i += blockDim.x) sD[i] = Dg[i];
  __syncthreads();
  GSTRIDE(i, (long long)B * nc) {
    const long long b = i / nc, p = i - b * nc;
    const float *zb = z + b * C * nc + p;
    float ph[LP_F], acc[C];
#pragma unroll
    for (int f = 0; f < LP_F; ++f) ph[f] = phi[f * nc + p];
#pragma unroll
    for (int c = 0; c < C; ++c) acc[c] = s[(b * C + c) * nc + p];
    // one input channel at a time: acc[c] += B[c][c2] z[c2], plus the
    // identity and conditioned diagonal on c = c2
#pragma unroll 2
    for (int c2 = 0; c2 < C; ++c2) {
      const float zv = zb[(long long)c2 * nc];
      float d = 1.f;
#pragma unroll
      for (int f = 0; f < LP_F; ++f) d += sD[c2 * LP_F + f] * ph[f];
#pragma unroll
      for (int c = 0; c < C; ++c) acc[c] += (sB[c * C + c2] + (c == c2 ? d : 0.f)) * zv;
    }
#pragma unroll
    for (int c = 0; c < C; ++c) out[(b * C + c) * nc + p] = acc[c];
  }
}

// launch k_lp_layer for the channel counts the library builds (1, 2, 4, 8, 16)
static int lp_layer_launch(cudaStream_t st, int C, const float *z, const float *s, float *out, const float *Bm,
                           const float *Dg, const float *phi, int B, long long nc, int transpose) {
  const unsigned nb = lp_blocks((long long)B * nc);
  switch (C) {
    case 1: k_lp_layer<1><<<nb, 256, 0, st>>>(z, s, out, Bm, Dg, phi, B, nc, transpose); break;
    case 2: k_lp_layer<2><<<nb, 256, 0, st>>>(z, s, out, Bm, Dg, phi, B, nc, transpose); break;
    case 4: k_lp_layer<4><<<nb, 256, 0, st>>>(z, s, out, Bm, Dg, phi, B, nc, transpose); break;
    case 8: k_lp_layer<8><<<nb, 256, 0, st>>>(z, s, out, Bm, Dg, phi, B, nc, transpose); break;
    case 16: k_lp_layer<16><<<nb, 256, 0, st>>>(z, s, out, Bm, Dg, phi, B, nc, transpose); break;
    default:
      bdgd_set_error("bdg_lp: channel count %d not built (1, 2, 4, 8 or 16)", C);
      return BDGD_ERR_UNSUPPORTED;
  }
  bdgd_count_launch();
  return BDGD_OK;
}

// Partial sums (block per (row c, split)) of
//   gB[c][c'] = sum g[b][c][p] z[b][c'][p],  gD[c][f] = sum g[b][c][p] z[b][c][p] phi[f][p]
// into part[split][c][C + F]; mode 1 (lift): gA[c][f] = sum g[b][c][p] phi[f][p] rc[b][p]
// into part[split][c][F].
__global__ void __launch_bounds__(256) k_lp_mix_grad_part(const float *__restrict__ g, const float *__restrict__ z,
                                                          const float *__restrict__ rc,
                                                          const float *__restrict__ phi, int B, int C, long long nc,
                                                          int nsplit, int lift, float *__restrict__ part) {
  const int c = blockIdx.x, split = blockIdx.y;
  const long long total = (long long)B * nc;
  const long long chunk = (total + nsplit - 1) / nsplit;
  const long long i0 = (long long)split * chunk, i1 = min(total, i0 + chunk);
  const int NV = lift ? LP_F : C + LP_F;
  float acc[LP_CMAX + LP_F];
#pragma unroll
  for (int j = 0; j < LP_CMAX + LP_F; ++j) acc[j] = 0.f;
  for (long long i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
    const long long b = i / nc, p = i - b * nc;
    const float gv = g[(b * C + c) * nc + p];
    if (lift) {
      const float r = gv * rc[b * nc + p];
#pragma unroll
      for (int f = 0; f < LP_F; ++f) acc[f] += r * phi[f * nc + p];
    } else {
#pragma unroll
      for (int c2 = 0; c2 < LP_CMAX; ++c2)
        if (c2 < C) acc[c2] += gv * z[(b * C + c2) * nc + p];
      const float gz = gv * z[(b * C + c) * nc + p];
#pragma unroll
      for (int f = 0; f < LP_F; ++f) acc[LP_CMAX + f] += gz * phi[f * nc + p];
    }
  }
  __shared__ float red[8][LP_CMAX + LP_F];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < LP_CMAX + LP_F; ++j) {
    float v = acc[j];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[w][j] = v;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    const int j = threadIdx.x;
    // map the output slot to the accumulator index
    const int a = lift ? j : (j < C ? j : LP_CMAX + (j - C));
    float v = 0.f;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) v += red[k][a];
    part[((long long)split * C + c) * NV + j] = v;
  }
}

// sum the split partials: mode 0 -> gB (C x C) and gD (C x F); mode 1 -> gA (C x F)
__global__ void k_lp_mix_grad_sum(const float *__restrict__ part, int nsplit, int C, int lift, float *__restrict__ g1,
                                  float *__restrict__ g2) {
  const int NV = lift ? LP_F : C + LP_F;
  GSTRIDE(i, (long long)C * NV) {
    const int c = (int)(i / NV), j = (int)(i % NV);
    double v = 0.0;
    for (int s = 0; s < nsplit; ++s) v += part[((long long)s * C + c) * NV + j];
    if (lift) g1[c * LP_F + j] += (float)v;
    else if (j < C) g1[c * C + j] += (float)v;
    else g2[c * LP_F + (j - C)] += (float)v;
  }
}

__global__ void k_lp_scale_cols(float *__restrict__ a, const double *__restrict__ fac, int B, long long per) {
  GSTRIDE(i, (long long)B * per) a[i] *= (float)fac[i / per];
}

// per column: dd = d.d, ee = e.e, dp = d.p0r (one block per column)
__global__ void k_lp_coldots(const double *__restrict__ d, long long ldd, const double *__restrict__ e,
                             const double *__restrict__ p, long long ld, long long S, double *__restrict__ out) {
  const int b = blockIdx.x;
  double a0 = 0, a1 = 0, a2 = 0;
  for (long long i = threadIdx.x; i < S; i += blockDim.x) {
    const double dv = d[b * ldd + i], ev = e[b * ld + i], pv = p[b * ld + i];
    a0 += dv * dv;
    a1 += ev * ev;
    a2 += dv * pv;
  }
  __shared__ double red[3][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) {
    a0 += __shfl_xor_sync(0xffffffffu, a0, o);
    a1 += __shfl_xor_sync(0xffffffffu, a1, o);
    a2 += __shfl_xor_sync(0xffffffffu, a2, o);
  }
  if (lane == 0) {
    red[0][w] = a0;
    red[1][w] = a1;
    red[2][w] = a2;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double v = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) v += red[threadIdx.x][k];
    out[b * 3 + threadIdx.x] = v;
  }
}

// Energy loss terms per column, with q = A T r (Op applied, shift added here):
// a0 = <Tr, q>, a1 = <r, Tr>, a2 = <r, e>; then q <- d = q - r and
// a3 = <d, P0 r>.  tr, q leading dim S; r, e, p leading dim ld.
__global__ void k_lp_edots(const double *__restrict__ tr, double *__restrict__ q, const double *__restrict__ r,
                           const double *__restrict__ e, const double *__restrict__ p, double sigma, long long ld,
                           long long S, double *__restrict__ out) {
  const int b = blockIdx.x;
  double a[4] = {0, 0, 0, 0};
  for (long long i = threadIdx.x; i < S; i += blockDim.x) {
    const double t = tr[b * S + i], rv = r[b * ld + i];
    const double qv = q[b * S + i] + sigma * t;
    a[0] += t * qv;
    a[1] += rv * t;
    a[2] += rv * e[b * ld + i];
    const double dv = qv - rv;
    q[b * S + i] = dv;
    a[3] += dv * p[b * ld + i];
  }
  __shared__ double red[4][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    double v = a[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[k][w] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double v = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) v += red[threadIdx.x][k];
    out[b * 4 + threadIdx.x] = v;
  }
}

// tr <- tr - e (tr holds T r), column-wise with leading dims
__global__ void k_lp_sub(double *__restrict__ tr, long long ldt, const double *__restrict__ e, long long lde, int B,
                         long long S) {
  GSTRIDE(i, (long long)B * S) {
    const long long b = i / S, q = i - b * S;
    tr[b * ldt + q] -= e[b * lde + q];
  }
}

__global__ void k_lp_copy_cols(const double *__restrict__ src, long long lds, double *__restrict__ dst,
                               long long ldd, int B, long long S) {
  GSTRIDE(i, (long long)B * S) {
    const long long b = i / S, q = i - b * S;
    dst[b * ldd + q] = src[b * lds + q];
  }
}

__global__ void k_lp_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                          float *__restrict__ v, long long n, float lr, float c1, float c2) {
  GSTRIDE(i, n) {
    const float gi = g[i];
    const float mi = 0.9f * m[i] + 0.1f * gi;
    const float vi = 0.999f * v[i] + 0.001f * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
  }
}

// ---------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------
#define LP_CK(call)                                      \
  do {                                                   \
    cudaError_t _e = (call);                             \
    if (_e != cudaSuccess) return bdgd_check(_e, #call); \
  } while (0)

static int lp_alloc(void **p, size_t bytes) {
  LP_CK(cudaMalloc(p, bytes));
  return BDGD_OK;
}

static void lp_free_ws(bdg_lp *lp) {
  void *bufs[] = {lp->rc[0], lp->rc[1], lp->acts[0], lp->acts[1], lp->gbuf[0], lp->gbuf[1], lp->sbuf,
                  lp->co[0], lp->co[1], lp->ax1,     lp->ax2,     lp->part,    lp->tr,      lp->dots,
                  lp->fac,   lp->tq};
  for (void *b : bufs)
    if (b) cudaFree(b);
  lp->rc[0] = lp->rc[1] = lp->acts[0] = lp->acts[1] = lp->gbuf[0] = lp->gbuf[1] = lp->sbuf = nullptr;
  lp->co[0] = lp->co[1] = lp->ax1 = lp->ax2 = lp->part = nullptr;
  lp->tr = lp->tq = lp->dots = lp->fac = nullptr;
  lp->wsB = 0;
  lp->wsTrain = 0;
}

static const int kLpSplit = 64;

static int lp_workspace(bdg_lp *lp, long long B, int train) {
  if (lp->wsB >= B && (lp->wsTrain || !train)) return BDGD_OK;
  lp_free_ws(lp);
  const long long nc = lp->nc, C = lp->C, R = lp->R;
  const long long field = B * C * nc;
  int rc;
  const int nsets = train ? 2 : 1;
  for (int s = 0; s < nsets; ++s) {
    if ((rc = lp_alloc((void **)&lp->rc[s], sizeof(float) * B * nc))) return rc;
    if ((rc = lp_alloc((void **)&lp->acts[s], sizeof(float) * field * (train ? lp->L + 1 : 2)))) return rc;
  }
  for (int s = 0; s < 2; ++s) {
    if ((rc = lp_alloc((void **)&lp->gbuf[s], sizeof(float) * field))) return rc;
    if ((rc = lp_alloc((void **)&lp->co[s], sizeof(float) * B * C * R * R * R))) return rc;
  }
  if ((rc = lp_alloc((void **)&lp->sbuf, sizeof(float) * field))) return rc;
  if ((rc = lp_alloc((void **)&lp->ax1, sizeof(float) * B * C * lp->n[2] * lp->n[1] * R))) return rc;
  if ((rc = lp_alloc((void **)&lp->ax2, sizeof(float) * B * C * lp->n[2] * R * R))) return rc;
  lp->part_n = (long long)kLpSplit * C * (C + LP_F);
  if ((rc = lp_alloc((void **)&lp->part, sizeof(float) * lp->part_n))) return rc;
  if (train) {
    if ((rc = lp_alloc((void **)&lp->tr, sizeof(double) * B * lp->S))) return rc;
    if ((rc = lp_alloc((void **)&lp->tq, sizeof(double) * B * lp->S))) return rc;
    if ((rc = lp_alloc((void **)&lp->dots, sizeof(double) * B * 4))) return rc;
    if ((rc = lp_alloc((void **)&lp->fac, sizeof(double) * B))) return rc;
  }
  lp->wsB = B;
  lp->wsTrain = train;
  return BDGD_OK;
}

// Contraction of the middle axis of in[outer][lin][inner] with the basis:
// out[o][i][q] = sum_m Mat(i, m) in[o][m][q], Mat = E (forward, R x n) or
// E^T (adjoint).  Plain FP32 GEMMs (cuBLAS, column-major view): one GEMM when
// inner == 1, else one strided batch over `outer`.
static int lp_axis(bdg_lp *lp, const float *in, float *out, const float *E, long long outer, int lin, int lout,
                   long long inner, int n, int adj) {
  const float one = 1.f, zero = 0.f;
  cublasStatus_t st;
  if (inner == 1) {
    // C(lout x outer) = op(E_cm) (lout x lin) * in_cm (lin x outer)
    st = cublasSgemm(lp->blas, adj ? CUBLAS_OP_N : CUBLAS_OP_T, CUBLAS_OP_N, lout, (int)outer, lin, &one, E, n, in,
                     lin, &zero, out, lout);
  } else {
    // per o: C_o (inner x lout) = in_o (inner x lin) * op(E_cm) (lin x lout)
    st = cublasSgemmStridedBatched(lp->blas, CUBLAS_OP_N, adj ? CUBLAS_OP_T : CUBLAS_OP_N, (int)inner, lout, lin, &one,
                                   in, (int)inner, (long long)lin * inner, E, n, 0, &zero, out, (int)inner,
                                   (long long)lout * inner, (int)outer);
  }
  if (st != CUBLAS_STATUS_SUCCESS) {
    bdgd_set_error("bdg_lp: cuBLAS GEMM failed (%d)", (int)st);
    return BDGD_ERR_CUDA;
  }
  bdgd_count_launch();
  return BDGD_OK;
}

// coefficients co = P z for B*C fields
static int lp_P(bdg_lp *lp, const float *z, float *co, long long BC) {
  const int R = lp->R, n0 = lp->n[0], n1 = lp->n[1], n2 = lp->n[2];
  int rc = lp_axis(lp, z, lp->ax1, lp->E[0], BC * n2 * n1, n0, R, 1, n0, 0);
  if (!rc) rc = lp_axis(lp, lp->ax1, lp->ax2, lp->E[1], BC * n2, n1, R, R, n1, 0);
  if (!rc) rc = lp_axis(lp, lp->ax2, co, lp->E[2], BC, n2, R, (long long)R * R, n2, 0);
  return rc;
}

// z = P^T co
static int lp_Pt(bdg_lp *lp, const float *co, float *z, long long BC) {
  const int R = lp->R, n0 = lp->n[0], n1 = lp->n[1], n2 = lp->n[2];
  int rc = lp_axis(lp, co, lp->ax2, lp->E[2], BC, R, n2, (long long)R * R, n2, 1);
  if (!rc) rc = lp_axis(lp, lp->ax2, lp->ax1, lp->E[1], BC * n2, R, n1, R, n1, 1);
  if (!rc) rc = lp_axis(lp, lp->ax1, z, lp->E[0], BC * n2 * n1, R, n0, 1, n0, 1);
  return rc;
}

static const float *lpW(bdg_lp *lp, int h, int l) { return lp->h[h].p + lp->oW + (long long)l * lp->C * lp->M * lp->M * lp->M; }
static const float *lpB(bdg_lp *lp, int h, int l) { return lp->h[h].p + lp->oB + (long long)l * lp->C * lp->C; }
static const float *lpD(bdg_lp *lp, int h, int l) { return lp->h[h].p + lp->oD + (long long)l * lp->C * LP_F; }

// One layer step on z (B columns): out = z + SC(z) + PM(z) (transpose: PM^T).
// If co_given, co already holds P z (consumed).
static int lp_layer(bdg_lp *lp, cudaStream_t st, int h, int l, int B, const float *z, float *out, int transpose,
                    float *co) {
  const long long BC = (long long)B * lp->C;
  const float inv_nc = 1.0f / (float)lp->nc;
  int rc = lp_P(lp, z, co, BC);
  if (rc) return rc;
  k_lp_filter<<<lp_blocks(BC * lp->R * lp->R * lp->R), 256, 0, st>>>(co, lpW(lp, h, l), B, lp->C, lp->R, lp->M,
                                                                     inv_nc);
  bdgd_count_launch();
  if ((rc = lp_Pt(lp, co, lp->sbuf, BC))) return rc;
  if ((rc = lp_layer_launch(st, lp->C, z, lp->sbuf, out, lpB(lp, h, l), lpD(lp, h, l), lp->phi, B, lp->nc,
                            transpose)))
    return rc;
  LP_CK(cudaGetLastError());
  return BDGD_OK;
}

// forward S of pooled input rc (B columns): keep = all layer inputs in acts
// (L+1 fields) else ping-pong in acts[0..1]; returns pointer to S x.
static float *lp_forward(bdg_lp *lp, cudaStream_t st, int h, int B, const float *rc, float *acts, int keep, int *err) {
  const long long field = (long long)B * lp->C * lp->nc;
  k_lp_lift<<<lp_blocks(field), 256, 0, st>>>(rc, lp->h[h].p + lp->oA, lp->phi, B, lp->C, lp->nc, acts);
  bdgd_count_launch();
  float *cur = acts;
  for (int l = 0; l < lp->L; ++l) {
    float *nxt = keep ? acts + (l + 1) * field : acts + ((l + 1) & 1) * field;
    if ((*err = lp_layer(lp, st, h, l, B, cur, nxt, 0, lp->co[0]))) return nullptr;
    cur = nxt;
  }
  return cur;
}

// adjoint S^T applied to g (B columns, overwritten) -> rc_out (coarse)
static int lp_adjoint(bdg_lp *lp, cudaStream_t st, int h, int B, float *g, float *rc_out) {
  float *a = g, *b = lp->gbuf[1] == g ? lp->gbuf[0] : lp->gbuf[1];
  for (int l = lp->L - 1; l >= 0; --l) {
    int rc = lp_layer(lp, st, h, l, B, a, b, 1, lp->co[0]);
    if (rc) return rc;
    float *t = a;
    a = b;
    b = t;
  }
  k_lp_lift_adj<<<lp_blocks((long long)B * lp->nc), 256, 0, st>>>(a, lp->h[h].p + lp->oA, lp->phi, B, lp->C, lp->nc,
                                                                  rc_out);
  bdgd_count_launch();
  LP_CK(cudaGetLastError());
  return BDGD_OK;
}

// gradient of <u, S v> accumulated into lp->h[h].g; acts = layer inputs of v
// (L+1 fields), rcv = pooled v, u (B columns) is overwritten.
static int lp_backprop(bdg_lp *lp, cudaStream_t st, int h, int B, const float *acts, const float *rcv, float *u) {
  const long long field = (long long)B * lp->C * lp->nc;
  const long long BC = (long long)B * lp->C;
  const float inv_nc = 1.0f / (float)lp->nc;
  float *g = u, *gn = (u == lp->gbuf[0]) ? lp->gbuf[1] : lp->gbuf[0];
  float *gr = lp->h[h].g;
  for (int l = lp->L - 1; l >= 0; --l) {
    const float *z = acts + l * field;
    int rc = lp_P(lp, z, lp->co[0], BC);
    if (!rc) rc = lp_P(lp, g, lp->co[1], BC);
    if (rc) return rc;
    k_lp_filter_grad<<<lp_blocks((long long)lp->C * lp->M * lp->M * lp->M), 256, 0, st>>>(
        lp->co[0], lp->co[1], gr + lp->oW + (long long)l * lp->C * lp->M * lp->M * lp->M, B, lp->C, lp->R, lp->M,
        inv_nc);
    k_lp_mix_grad_part<<<dim3(lp->C, kLpSplit), 256, 0, st>>>(g, z, nullptr, lp->phi, B, lp->C, lp->nc, kLpSplit, 0,
                                                              lp->part);
    k_lp_mix_grad_sum<<<lp_blocks((long long)lp->C * (lp->C + LP_F)), 256, 0, st>>>(
        lp->part, kLpSplit, lp->C, 0, gr + lp->oB + (long long)l * lp->C * lp->C, gr + lp->oD + (long long)l * lp->C * LP_F);
    for (int k = 0; k < 3; ++k) bdgd_count_launch();
    // g <- g + SC(g) + PM^T(g), reusing P g
    k_lp_filter<<<lp_blocks(BC * lp->R * lp->R * lp->R), 256, 0, st>>>(lp->co[1], lpW(lp, h, l), B, lp->C, lp->R,
                                                                       lp->M, inv_nc);
    if ((rc = lp_Pt(lp, lp->co[1], lp->sbuf, BC))) return rc;
    if ((rc = lp_layer_launch(st, lp->C, g, lp->sbuf, gn, lpB(lp, h, l), lpD(lp, h, l), lp->phi, B, lp->nc, 1)))
      return rc;
    bdgd_count_launch();
    float *t = g;
    g = gn;
    gn = t;
  }
  k_lp_mix_grad_part<<<dim3(lp->C, kLpSplit), 256, 0, st>>>(g, nullptr, rcv, lp->phi, B, lp->C, lp->nc, kLpSplit, 1,
                                                            lp->part);
  k_lp_mix_grad_sum<<<lp_blocks((long long)lp->C * LP_F), 256, 0, st>>>(lp->part, kLpSplit, lp->C, 1, gr + lp->oA,
                                                                       nullptr);
  for (int k = 0; k < 2; ++k) bdgd_count_launch();
  LP_CK(cudaGetLastError());
  return BDGD_OK;
}

// ---------------------------------------------------------------------------
// API
// ---------------------------------------------------------------------------
static int lp_set_geometry(bdg_lp *lp, const uint64_t N[3]) {
  for (int d = 0; d < 3; ++d) {
    if (N[d] < 8 || (N[d] % 2) || (int)(N[d] / 4) < lp->M) {
      bdgd_set_error("bdg_lp: grid extents must be even, >= 8 and >= 4*modes");
      return BDGD_ERR_ARG;
    }
  }
  for (int d = 0; d < 3; ++d) {
    lp->N[d] = (int)N[d];
    lp->n[d] = (int)N[d] / 2;
    if (lp->E[d]) cudaFree(lp->E[d]);
    lp->E[d] = nullptr;
  }
  lp->S = (long long)lp->N[0] * lp->N[1] * lp->N[2];
  lp->nc = lp->S / 8;
  for (int d = 0; d < 3; ++d) {
    const int n = lp->n[d];
    float *h = (float *)malloc(sizeof(float) * lp->R * n);
    for (int r = 0; r < lp->R; ++r) {
      const int a = r < lp->M ? r : r - lp->M + 1;
      for (int x = 0; x < n; ++x) {
        const double ang = 2.0 * M_PI * (double)a * (double)x / (double)n;
        h[r * n + x] = (float)(r < lp->M ? cos(ang) : sin(ang));
      }
    }
    int rc = lp_alloc((void **)&lp->E[d], sizeof(float) * lp->R * n);
    if (!rc) {
      cudaError_t e = cudaMemcpy(lp->E[d], h, sizeof(float) * lp->R * n, cudaMemcpyHostToDevice);
      if (e != cudaSuccess) rc = bdgd_check(e, "upload basis");
    }
    free(h);
    if (rc) return rc;
  }
  if (lp->phi) cudaFree(lp->phi);
  lp->phi = nullptr;
  lp->conditioned = 0;
  lp_free_ws(lp);
  return BDGD_OK;
}

extern "C" int bdg_lp_create(bdg_lp **out, const uint64_t N[3], int C, int L, int modes) {
  *out = nullptr;
  if ((C != 1 && C != 2 && C != 4 && C != 8 && C != 16) || L < 1 || L > 16 || modes < 1) {
    bdgd_set_error("bdg_lp_create: need C in {1, 2, 4, 8, 16}, 1 <= L <= 16, modes >= 1");
    return BDGD_ERR_ARG;
  }
  bdg_lp *lp = (bdg_lp *)calloc(1, sizeof(bdg_lp));
  if (cublasCreate(&lp->blas) != CUBLAS_STATUS_SUCCESS) {
    free(lp);
    bdgd_set_error("bdg_lp_create: cublasCreate failed");
    return BDGD_ERR_CUDA;
  }
  cublasSetMathMode(lp->blas, CUBLAS_PEDANTIC_MATH);  // true FP32 (no TF32 down-conversion)
  lp->fast = 1;
  lp->C = C;
  lp->L = L;
  lp->M = modes;
  lp->R = 2 * modes - 1;
  cudaGetDevice(&lp->device);
  lp->oA = 0;
  lp->oW = lp->oA + (long long)C * LP_F;
  lp->oB = lp->oW + (long long)L * C * modes * modes * modes;
  lp->oD = lp->oB + (long long)L * C * C;
  lp->oEta = lp->oD + (long long)L * C * LP_F;
  lp->np = lp->oEta + 1;
  int rc = lp_set_geometry(lp, N);
  for (int h = 0; h < 2 && !rc; ++h) {
    LPHalf &H = lp->h[h];
    if ((rc = lp_alloc((void **)&H.p, sizeof(float) * lp->np))) break;
    if ((rc = lp_alloc((void **)&H.g, sizeof(float) * lp->np))) break;
    if ((rc = lp_alloc((void **)&H.m, sizeof(float) * lp->np))) break;
    if ((rc = lp_alloc((void **)&H.v, sizeof(float) * lp->np))) break;
    cudaMemset(H.p, 0, sizeof(float) * lp->np);
    cudaMemset(H.m, 0, sizeof(float) * lp->np);
    cudaMemset(H.v, 0, sizeof(float) * lp->np);
    H.step = 0;
  }
  if (rc) {
    bdg_lp_free(&lp);
    return rc;
  }
  *out = lp;
  return BDGD_OK;
}

extern "C" void bdg_lp_free(bdg_lp **plp) {
  if (!plp || !*plp) return;
  bdg_lp *lp = *plp;
  cudaDeviceSynchronize();
  lp_free_ws(lp);
  for (int d = 0; d < 3; ++d)
    if (lp->E[d]) cudaFree(lp->E[d]);
  if (lp->phi) cudaFree(lp->phi);
  if (lp->blas) cublasDestroy(lp->blas);
  for (int h = 0; h < 2; ++h) {
    cudaFree(lp->h[h].p);
    cudaFree(lp->h[h].g);
    cudaFree(lp->h[h].m);
    cudaFree(lp->h[h].v);
  }
  free(lp);
  *plp = nullptr;
}

extern "C" uint64_t bdg_lp_nparams(const bdg_lp *lp) { return lp ? (uint64_t)lp->np : 0; }

extern "C" int bdg_lp_get_params(const bdg_lp *lp, int half, float *host_out) {
  if (!lp || half < 0 || half > 1 || !host_out) return BDGD_ERR_ARG;
  LP_CK(cudaMemcpy(host_out, lp->h[half].p, sizeof(float) * lp->np, cudaMemcpyDeviceToHost));
  return BDGD_OK;
}

extern "C" int bdg_lp_set_params(bdg_lp *lp, int half, const float *host_in) {
  if (!lp || half < 0 || half > 1 || !host_in) return BDGD_ERR_ARG;
  LP_CK(cudaMemcpy(lp->h[half].p, host_in, sizeof(float) * lp->np, cudaMemcpyHostToDevice));
  LP_CK(cudaMemset(lp->h[half].m, 0, sizeof(float) * lp->np));
  LP_CK(cudaMemset(lp->h[half].v, 0, sizeof(float) * lp->np));
  lp->h[half].step = 0;
  return BDGD_OK;
}

extern "C" int bdg_lp_init_random(bdg_lp *lp, double amp, uint64_t seed) {
  if (!lp) return BDGD_ERR_ARG;
  float *p = (float *)calloc(lp->np, sizeof(float));
  uint64_t s = seed * 2654435761ull + 12345ull;
  for (int h = 0; h < 2; ++h) {
    memset(p, 0, sizeof(float) * lp->np);
    for (long long i = 0; i < (long long)lp->C * LP_F; ++i) {
      s = s * 6364136223846793005ull + 1442695040888963407ull;  // 64-bit LCG (Knuth's MMIX constants)
      const double u = (double)(s >> 11) / 9007199254740992.0;
      p[lp->oA + i] = (float)(amp * (2.0 * u - 1.0));
    }
    int rc = bdg_lp_set_params(lp, h, p);
    if (rc) {
      free(p);
      return rc;
    }
  }
  free(p);
  return BDGD_OK;
}

struct LPFileHeader {
  char magic[8];
  int C, L, M, F;
  long long np;
};

extern "C" int bdg_lp_save(const bdg_lp *lp, const char *path) {
  if (!lp || !path) return BDGD_ERR_ARG;
  FILE *f = fopen(path, "wb");
  if (!f) {
    bdgd_set_error("bdg_lp_save: cannot open %s", path);
    return BDGD_ERR_ARG;
  }
  LPFileHeader hd;
  memset(&hd, 0, sizeof hd);
  memcpy(hd.magic, "BDGLP01", 8);
  hd.C = lp->C;
  hd.L = lp->L;
  hd.M = lp->M;
  hd.F = LP_F;
  hd.np = lp->np;
  float *buf = (float *)malloc(sizeof(float) * lp->np);
  int rc = (fwrite(&hd, sizeof hd, 1, f) == 1) ? BDGD_OK : BDGD_ERR_ARG;
  for (int h = 0; h < 2 && !rc; ++h) {
    rc = bdg_lp_get_params(lp, h, buf);
    if (!rc && fwrite(buf, sizeof(float), lp->np, f) != (size_t)lp->np) rc = BDGD_ERR_ARG;
  }
  free(buf);
  fclose(f);
  if (rc) bdgd_set_error("bdg_lp_save: write failed");
  return rc;
}

extern "C" int bdg_lp_load(bdg_lp *lp, const char *path) {
  if (!lp || !path) return BDGD_ERR_ARG;
  FILE *f = fopen(path, "rb");
  if (!f) {
    bdgd_set_error("bdg_lp_load: cannot open %s", path);
    return BDGD_ERR_ARG;
  }
  LPFileHeader hd;
  int rc = BDGD_OK;
  if (fread(&hd, sizeof hd, 1, f) != 1 || memcmp(hd.magic, "BDGLP01", 8) || hd.C != lp->C || hd.L != lp->L ||
      hd.M != lp->M || hd.F != LP_F || hd.np != lp->np) {
    bdgd_set_error("bdg_lp_load: %s does not hold a C=%d L=%d modes=%d preconditioner", path, lp->C, lp->L, lp->M);
    rc = BDGD_ERR_ARG;
  }
  float *buf = (float *)malloc(sizeof(float) * lp->np);
  for (int h = 0; h < 2 && !rc; ++h) {
    if (fread(buf, sizeof(float), lp->np, f) != (size_t)lp->np) {
      bdgd_set_error("bdg_lp_load: %s is truncated", path);
      rc = BDGD_ERR_ARG;
    } else {
      rc = bdg_lp_set_params(lp, h, buf);
    }
  }
  free(buf);
  fclose(f);
  return rc;
}

extern "C" int bdg_lp_set_fast_math(bdg_lp *lp, int on) {
  if (!lp) return BDGD_ERR_ARG;
  lp->fast = on ? 1 : 0;
  return BDGD_OK;
}

extern "C" int bdg_lp_set_energy_loss(bdg_lp *lp, double sigma) {
  if (!lp) return BDGD_ERR_ARG;
  lp->energy = sigma >= 0.0;
  lp->esigma = sigma >= 0.0 ? sigma : 0.0;
  return BDGD_OK;
}

extern "C" int bdg_lp_regrid(bdg_lp *lp, const uint64_t N[3]) {
  if (!lp) return BDGD_ERR_ARG;
  return lp_set_geometry(lp, N);
}

extern "C" int bdg_lp_condition(bdg_lp *lp, const double *psi0, const double *V, double eps_dd, double lambda) {
  if (!lp || !psi0 || !V) return BDGD_ERR_ARG;
  const long long nc = lp->nc;
  const int N0 = lp->N[0], N1 = lp->N[1];
  const int n0 = lp->n[0], n1 = lp->n[1], n2 = lp->n[2];
  double *dens = (double *)calloc(nc, sizeof(double)), *vc = (double *)calloc(nc, sizeof(double));
  for (int Z = 0; Z < n2; ++Z)
    for (int Y = 0; Y < n1; ++Y)
      for (int X = 0; X < n0; ++X) {
        double sd = 0, sv = 0;
        for (int dz = 0; dz < 2; ++dz)
          for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx) {
              const long long q = ((long long)(2 * Z + dz) * N1 + 2 * Y + dy) * N0 + 2 * X + dx;
              sd += psi0[q] * psi0[q];
              sv += V[q];
            }
        const long long p = ((long long)Z * n1 + Y) * n0 + X;
        dens[p] = 0.125 * sd;
        vc[p] = 0.125 * sv;
      }
  double dmax = 1e-300, vmax = 1e-300;
  for (long long p = 0; p < nc; ++p) {
    dmax = fmax(dmax, dens[p]);
    vmax = fmax(vmax, fabs(vc[p]));
  }
  float *phi = (float *)malloc(sizeof(float) * LP_F * nc);
  for (long long p = 0; p < nc; ++p) {
    phi[p] = 1.0f;
    phi[nc + p] = (float)(dens[p] / dmax);
    phi[2 * nc + p] = (float)(vc[p] / vmax);
    phi[3 * nc + p] = (float)eps_dd;
    phi[4 * nc + p] = (float)(lambda / 4.0);
  }
  free(dens);
  free(vc);
  int rc = BDGD_OK;
  if (!lp->phi) rc = lp_alloc((void **)&lp->phi, sizeof(float) * LP_F * nc);
  if (!rc) {
    cudaError_t e = cudaMemcpy(lp->phi, phi, sizeof(float) * LP_F * nc, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) rc = bdgd_check(e, "upload conditioning");
  }
  free(phi);
  if (!rc) lp->conditioned = 1;
  return rc;
}

static int lp_check(bdg_lp *lp, bdgd_ctx *dev) {
  if (!lp || !dev) return BDGD_ERR_ARG;
  cublasSetStream(lp->blas, dev->stream);
  if (!lp->conditioned) {
    bdgd_set_error("bdg_lp: not conditioned (call bdg_lp_condition)");
    return BDGD_ERR_STATE;
  }
  if (dev->dim != 3 || dev->cplx || dev->N[0] != lp->N[0] || dev->N[1] != lp->N[1] || dev->N[2] != lp->N[2]) {
    bdgd_set_error("bdg_lp: the context is not the real 3D grid of the preconditioner");
    return BDGD_ERR_ARG;
  }
  return BDGD_OK;
}

static const long long kLpChunk = 16;  // columns per apply chunk (bounds the workspace)

extern "C" int bdg_lp_apply_half(bdg_lp *lp, bdgd_ctx *dev, int half, int prec, const void *d_x, uint64_t ldx,
                                 void *d_y, uint64_t ldy, uint64_t ncol) {
  int rc = lp_check(lp, dev);
  if (rc) return rc;
  if (half < 0 || half > 1) return BDGD_ERR_ARG;
  cudaStream_t st = dev->stream;
  cublasSetMathMode(lp->blas, lp->fast ? CUBLAS_TF32_TENSOR_OP_MATH : CUBLAS_PEDANTIC_MATH);
  for (uint64_t c0 = 0; c0 < ncol; c0 += kLpChunk) {
    const int B = (int)((ncol - c0) < (uint64_t)kLpChunk ? (ncol - c0) : kLpChunk);
    if ((rc = lp_workspace(lp, kLpChunk, lp->wsTrain))) return rc;
    const size_t es = prec == BDGD_F32 ? 4 : 8;
    const char *x = (const char *)d_x + c0 * ldx * es;
    char *y = (char *)d_y + c0 * ldy * es;
    if (prec == BDGD_F32)
      k_lp_pool<float><<<lp_blocks((long long)B * lp->nc), 256, 0, st>>>((const float *)x, (long long)ldx, B, lp->N[0],
                                                                         lp->N[1], lp->n[0], lp->n[1], lp->n[2],
                                                                         lp->rc[0]);
    else
      k_lp_pool<double><<<lp_blocks((long long)B * lp->nc), 256, 0, st>>>((const double *)x, (long long)ldx, B,
                                                                          lp->N[0], lp->N[1], lp->n[0], lp->n[1],
                                                                          lp->n[2], lp->rc[0]);
    bdgd_count_launch();
    float *sx = lp_forward(lp, st, half, B, lp->rc[0], lp->acts[0], 0, &rc);
    if (rc) return rc;
    // S^T S x: the adjoint consumes a copy of S x in gbuf[0]
    LP_CK(cudaMemcpyAsync(lp->gbuf[0], sx, sizeof(float) * (size_t)B * lp->C * lp->nc, cudaMemcpyDeviceToDevice, st));
    if ((rc = lp_adjoint(lp, st, half, B, lp->gbuf[0], lp->rc[0]))) return rc;
    const float *eta = lp->h[half].p + lp->oEta;
    if (prec == BDGD_F32)
      k_lp_poolt_axpy<float><<<lp_blocks((long long)B * lp->S), 256, 0, st>>>(lp->rc[0], (float *)y, (long long)ldy, B,
                                                                              lp->N[0], lp->N[1], lp->N[2], eta);
    else
      k_lp_poolt_axpy<double><<<lp_blocks((long long)B * lp->S), 256, 0, st>>>(lp->rc[0], (double *)y, (long long)ldy,
                                                                               B, lp->N[0], lp->N[1], lp->N[2], eta);
    bdgd_count_launch();
    LP_CK(cudaGetLastError());
  }
  return BDGD_OK;
}

extern "C" int bdg_lp_apply(bdg_lp *lp, bdgd_ctx *dev, int prec, const void *d_x, uint64_t ldx, void *d_y,
                            uint64_t ldy, uint64_t ncol) {
  int rc = lp_check(lp, dev);
  if (rc) return rc;
  if ((rc = bdgd_apply(dev, BDGD_OP_TLREP, prec, d_x, ldx, d_y, ldy, ncol))) return rc;
  const size_t es = prec == BDGD_F32 ? 4 : 8;
  for (int h = 0; h < 2; ++h) {
    const char *x = (const char *)d_x + (size_t)h * lp->S * es;
    char *y = (char *)d_y + (size_t)h * lp->S * es;
    if ((rc = bdg_lp_apply_half(lp, dev, h, prec, x, ldx, y, ldy, ncol))) return rc;
  }
  return BDGD_OK;
}

extern "C" int bdg_lp_loss_grad(bdg_lp *lp, bdgd_ctx *dev, int half, const double *d_r, const double *d_e,
                                const double *d_p0r, uint64_t ld, uint64_t ncol, double *loss_out,
                                float *grad_out) {
  int rc = lp_check(lp, dev);
  if (rc) return rc;
  if (half < 0 || half > 1 || ncol == 0) return BDGD_ERR_ARG;
  if ((rc = lp_workspace(lp, (long long)ncol, 1))) return rc;
  cudaStream_t st = dev->stream;
  cublasSetMathMode(lp->blas, CUBLAS_PEDANTIC_MATH);  // gradients in exact FP32
  const int B = (int)ncol;
  const long long S = lp->S, field = (long long)B * lp->C * lp->nc;
  LPHalf &H = lp->h[half];
  LP_CK(cudaMemsetAsync(H.g, 0, sizeof(float) * lp->np, st));
  // forward S r (kept), T r = S^T S r + exp(eta) P0 r, d = T r - e
  k_lp_pool<double><<<lp_blocks((long long)B * lp->nc), 256, 0, st>>>(d_r, (long long)ld, B, lp->N[0], lp->N[1],
                                                                      lp->n[0], lp->n[1], lp->n[2], lp->rc[0]);
  bdgd_count_launch();
  float *sr = lp_forward(lp, st, half, B, lp->rc[0], lp->acts[0], 1, &rc);
  if (rc) return rc;
  LP_CK(cudaMemcpyAsync(lp->gbuf[0], sr, sizeof(float) * field, cudaMemcpyDeviceToDevice, st));
  if ((rc = lp_adjoint(lp, st, half, B, lp->gbuf[0], lp->rc[1]))) return rc;
  k_lp_copy_cols<<<lp_blocks((long long)B * S), 256, 0, st>>>(d_p0r, (long long)ld, lp->tr, S, B, S);
  k_lp_poolt_axpy<double><<<lp_blocks((long long)B * S), 256, 0, st>>>(lp->rc[1], lp->tr, S, B, lp->N[0], lp->N[1],
                                                                       lp->N[2], H.p + lp->oEta);
  const double *dvec;  // d of the gradient formula (leading dim S)
  if (lp->energy) {
    // q = Op T r (+ sigma T r in the dots kernel), d = q - r
    if ((rc = bdgd_apply(dev, half ? BDGD_OP_M : BDGD_OP_K, BDGD_F64, lp->tr, (uint64_t)S, lp->tq, (uint64_t)S,
                         (uint64_t)B)))
      return rc;
    k_lp_edots<<<B, 256, 0, st>>>(lp->tr, lp->tq, d_r, d_e, d_p0r, lp->esigma, (long long)ld, S, lp->dots);
    bdgd_count_launch();
    dvec = lp->tq;
  } else {
    k_lp_sub<<<lp_blocks((long long)B * S), 256, 0, st>>>(lp->tr, S, d_e, (long long)ld, B, S);
    k_lp_coldots<<<B, 256, 0, st>>>(lp->tr, S, d_e, d_p0r, (long long)ld, S, lp->dots);
    for (int k = 0; k < 2; ++k) bdgd_count_launch();
    dvec = lp->tr;
  }
  for (int k = 0; k < 2; ++k) bdgd_count_launch();
  LP_CK(cudaGetLastError());
  const int nd = lp->energy ? 4 : 3;
  double *dots = (double *)malloc(sizeof(double) * B * 4), *fac = (double *)malloc(sizeof(double) * B);
  float eta = 0.f;
  cudaError_t e1 = cudaMemcpyAsync(dots, lp->dots, sizeof(double) * B * nd, cudaMemcpyDeviceToHost, st);
  cudaError_t e2 = cudaMemcpyAsync(&eta, H.p + lp->oEta, sizeof(float), cudaMemcpyDeviceToHost, st);
  cudaError_t e3 = cudaStreamSynchronize(st);
  if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
    free(dots);
    free(fac);
    return bdgd_check(e3 != cudaSuccess ? e3 : (e1 != cudaSuccess ? e1 : e2), "bdg_lp_loss_grad");
  }
  double loss = 0.0, geta = 0.0;
  for (int b = 0; b < B; ++b) {
    if (lp->energy) {
      const double *a = dots + b * 4;
      const double re = a[2] > 0 ? a[2] : 1e-300;
      loss += (a[0] - 2.0 * a[1] + a[2]) / re;
      fac[b] = 2.0 / (re * B);
      geta += 2.0 * exp((double)eta) * a[3] / (re * B);
    } else {
      const double ee = dots[b * 3 + 1] > 0 ? dots[b * 3 + 1] : 1e-300;
      loss += dots[b * 3] / ee;
      fac[b] = 2.0 / (ee * B);
      geta += 2.0 * exp((double)eta) * dots[b * 3 + 2] / (ee * B);
    }
  }
  loss /= B;
  if (loss_out) *loss_out = loss;
  cudaError_t e4 = cudaMemcpyAsync(lp->fac, fac, sizeof(double) * B, cudaMemcpyHostToDevice, st);
  cudaError_t e5 = cudaStreamSynchronize(st);
  free(dots);
  free(fac);
  if (e4 != cudaSuccess || e5 != cudaSuccess) return bdgd_check(e4 != cudaSuccess ? e4 : e5, "bdg_lp_loss_grad");
  // forward S d (kept)
  k_lp_pool<double><<<lp_blocks((long long)B * lp->nc), 256, 0, st>>>(dvec, S, B, lp->N[0], lp->N[1], lp->n[0],
                                                                      lp->n[1], lp->n[2], lp->rc[1]);
  bdgd_count_launch();
  float *sd = lp_forward(lp, st, half, B, lp->rc[1], lp->acts[1], 1, &rc);
  if (rc) return rc;
  // grad <S d, S r> = J(d)^T (S r) + J(r)^T (S d), upstreams scaled by 2 / (||e||^2 B)
  LP_CK(cudaMemcpyAsync(lp->gbuf[0], sr, sizeof(float) * field, cudaMemcpyDeviceToDevice, st));
  k_lp_scale_cols<<<lp_blocks(field), 256, 0, st>>>(lp->gbuf[0], lp->fac, B, (long long)lp->C * lp->nc);
  bdgd_count_launch();
  if ((rc = lp_backprop(lp, st, half, B, lp->acts[1], lp->rc[1], lp->gbuf[0]))) return rc;
  LP_CK(cudaMemcpyAsync(lp->gbuf[0], sd, sizeof(float) * field, cudaMemcpyDeviceToDevice, st));
  k_lp_scale_cols<<<lp_blocks(field), 256, 0, st>>>(lp->gbuf[0], lp->fac, B, (long long)lp->C * lp->nc);
  bdgd_count_launch();
  if ((rc = lp_backprop(lp, st, half, B, lp->acts[0], lp->rc[0], lp->gbuf[0]))) return rc;
  const float ge = (float)geta;
  LP_CK(cudaMemcpyAsync(H.g + lp->oEta, &ge, sizeof(float), cudaMemcpyHostToDevice, st));
  if (grad_out) {
    LP_CK(cudaMemcpyAsync(grad_out, H.g, sizeof(float) * lp->np, cudaMemcpyDeviceToHost, st));
  }
  LP_CK(cudaStreamSynchronize(st));
  return BDGD_OK;
}

extern "C" int bdg_lp_train_step(bdg_lp *lp, bdgd_ctx *dev, int half, const double *d_r, const double *d_e,
                                 const double *d_p0r, uint64_t ld, uint64_t ncol, double lr, double *loss_out) {
  int rc = bdg_lp_loss_grad(lp, dev, half, d_r, d_e, d_p0r, ld, ncol, loss_out, nullptr);
  if (rc) return rc;
  LPHalf &H = lp->h[half];
  H.step += 1;
  const float c1 = (float)(1.0 - pow(0.9, H.step)), c2 = (float)(1.0 - pow(0.999, H.step));
  k_lp_adam<<<lp_blocks(lp->np), 256, 0, dev->stream>>>(H.p, H.g, H.m, H.v, lp->np, (float)lr, c1, c2);
  bdgd_count_launch();
  LP_CK(cudaGetLastError());
  return BDGD_OK;
}

// ---------------------------------------------------------------------------
// inner CG for training targets
// ---------------------------------------------------------------------------
// per column: out[b] = <a_b, c_b>
__global__ void k_lp_dotc(const double *__restrict__ a, const double *__restrict__ c, long long ld, long long S,
                          double *__restrict__ out) {
  const int b = blockIdx.x;
  double acc = 0;
  for (long long i = threadIdx.x; i < S; i += blockDim.x) acc += a[b * ld + i] * c[b * ld + i];
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) v += red[k];
    out[b] = v;
  }
}

// CG update with per-column scalars (alpha = rr / pq; inactive columns have alpha 0)
__global__ void k_lp_cg_update(double *__restrict__ e, double *__restrict__ res, const double *__restrict__ p,
                               const double *__restrict__ q, const double *__restrict__ alpha, long long ld, int B,
                               long long S) {
  GSTRIDE(i, (long long)B * S) {
    const long long b = i / S, k = b * ld + (i - b * S);
    e[k] += alpha[b] * p[k];
    res[k] -= alpha[b] * q[k];
  }
}
__global__ void k_lp_cg_dir(double *__restrict__ p, const double *__restrict__ res, const double *__restrict__ beta,
                            long long ld, int B, long long S) {
  GSTRIDE(i, (long long)B * S) {
    const long long b = i / S, k = b * ld + (i - b * S);
    p[k] = res[k] + beta[b] * p[k];
  }
}
__global__ void k_lp_shift_add(double *__restrict__ q, const double *__restrict__ p, double sigma, long long ld, int B,
                               long long S) {
  GSTRIDE(i, (long long)B * S) {
    const long long b = i / S, k = b * ld + (i - b * S);
    q[k] += sigma * p[k];
  }
}

extern "C" int bdg_lp_cg(bdgd_ctx *dev, int op, double sigma, const double *d_r, double *d_e, uint64_t ld,
                         uint64_t ncol, double tol, int maxit, int *iters_out) {
  if (!dev || (op != BDGD_OP_K && op != BDGD_OP_M) || ncol == 0) return BDGD_ERR_ARG;
  cudaStream_t st = dev->stream;
  const long long S = dev->S;
  const int B = (int)ncol;
  double *res = nullptr, *p = nullptr, *q = nullptr, *sc = nullptr;
  int rc = BDGD_OK;
  const size_t bytes = sizeof(double) * (size_t)ld * B;
  if ((rc = lp_alloc((void **)&res, bytes)) || (rc = lp_alloc((void **)&p, bytes)) ||
      (rc = lp_alloc((void **)&q, bytes)) || (rc = lp_alloc((void **)&sc, sizeof(double) * 4 * B))) {
    cudaFree(res);
    cudaFree(p);
    cudaFree(q);
    return rc;
  }
  double *h = (double *)malloc(sizeof(double) * 4 * B);
  double *rr = h, *rr0 = h + B, *al = h + 2 * B, *pq = h + 3 * B;
  int it = 0;
  cudaError_t ce = cudaSuccess;
  ce = cudaMemsetAsync(d_e, 0, bytes, st);
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(res, d_r, bytes, cudaMemcpyDeviceToDevice, st);
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(p, d_r, bytes, cudaMemcpyDeviceToDevice, st);
  if (ce != cudaSuccess) rc = bdgd_check(ce, "bdg_lp_cg");
  if (!rc) {
    k_lp_dotc<<<B, 256, 0, st>>>(res, res, (long long)ld, S, sc);
    bdgd_count_launch();
    ce = cudaMemcpyAsync(rr, sc, sizeof(double) * B, cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) rc = bdgd_check(ce, "bdg_lp_cg");
    for (int b = 0; b < B; ++b) rr0[b] = rr[b] > 0 ? rr[b] : 1e-300;
  }
  for (; !rc && it < maxit; ++it) {
    int active = 0;
    for (int b = 0; b < B; ++b)
      if (rr[b] > tol * tol * rr0[b]) active = 1;
    if (!active) break;
    if ((rc = bdgd_apply(dev, op, BDGD_F64, p, ld, q, ld, (uint64_t)B))) break;
    k_lp_shift_add<<<lp_blocks((long long)B * S), 256, 0, st>>>(q, p, sigma, (long long)ld, B, S);
    k_lp_dotc<<<B, 256, 0, st>>>(p, q, (long long)ld, S, sc);
    for (int k = 0; k < 2; ++k) bdgd_count_launch();
    ce = cudaMemcpyAsync(pq, sc, sizeof(double) * B, cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) {
      rc = bdgd_check(ce, "bdg_lp_cg");
      break;
    }
    for (int b = 0; b < B; ++b) al[b] = (rr[b] > tol * tol * rr0[b] && pq[b] > 0) ? rr[b] / pq[b] : 0.0;
    ce = cudaMemcpyAsync(sc + B, al, sizeof(double) * B, cudaMemcpyHostToDevice, st);
    if (ce != cudaSuccess) {
      rc = bdgd_check(ce, "bdg_lp_cg");
      break;
    }
    k_lp_cg_update<<<lp_blocks((long long)B * S), 256, 0, st>>>(d_e, res, p, q, sc + B, (long long)ld, B, S);
    k_lp_dotc<<<B, 256, 0, st>>>(res, res, (long long)ld, S, sc);
    for (int k = 0; k < 2; ++k) bdgd_count_launch();
    ce = cudaMemcpyAsync(pq, sc, sizeof(double) * B, cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) {
      rc = bdgd_check(ce, "bdg_lp_cg");
      break;
    }
    for (int b = 0; b < B; ++b) {
      al[b] = (al[b] != 0.0 && rr[b] > 0) ? pq[b] / rr[b] : 0.0;  // beta
      if (al[b] != 0.0) rr[b] = pq[b];
    }
    ce = cudaMemcpyAsync(sc + 2 * B, al, sizeof(double) * B, cudaMemcpyHostToDevice, st);
    if (ce != cudaSuccess) {
      rc = bdgd_check(ce, "bdg_lp_cg");
      break;
    }
    k_lp_cg_dir<<<lp_blocks((long long)B * S), 256, 0, st>>>(p, res, sc + 2 * B, (long long)ld, B, S);
    bdgd_count_launch();
  }
  if (!rc) {
    ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) rc = bdgd_check(ce, "bdg_lp_cg");
  }
  if (iters_out) *iters_out = it;
  free(h);
  cudaFree(res);
  cudaFree(p);
  cudaFree(q);
  cudaFree(sc);
  return rc;
}
