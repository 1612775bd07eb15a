// bdg_ops.cu -- batched BdG operator applies on sm_100a.
//
// Every operator of the reference (pstuermer/BDG_LOBPCG) operator layer is a
// pointwise prologue, an unnormalised 3D FFT, a k-space multiply, an inverse
// FFT and a pointwise epilogue, applied there one column at a time through
// FFTW (src/kinetic_impl.inc:17-30, src/matmulK_impl.inc:11-28,
// src/matmulM_impl.inc:14-44, src/dipolar_conv_impl.inc:22-52,
// src/precond_impl.inc:21-118).  Here one launch per FFT pass handles all
// columns (and both halves [u; v]) of a block:
//
//   pass X-fwd   rows along x: prologue (p*x, conj(psi0)*x) + forward FFT
//   pass Y-fwd   pencils along y (3D only)
//   pass Z-fused pencils along the last axis: forward FFT, k-space multiply
//                (k^2/2, dipolar kernel, 1/(mu + k^2/2)), inverse FFT
//   pass Y-inv   (3D only)
//   pass X-inv   rows: inverse FFT of every spectrum of the half + epilogue
//                (+ localTerm*x, + 2 g psi0 * exchange, * p)
//
// Each pass stages its lines in shared memory and runs a mixed-radix
// Stockham FFT (radix 8/4/2/3 butterflies in registers, generic radix for
// other small primes).  Real fields use the r2c half spectrum (x extent
// N/2+1) between passes, so the spectrum traffic is that of FFTW's r2c.
#include <cuda_runtime.h>

#include <atomic>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "bdg_dev.h"
#include "bdg_kern.cuh"
#include "bdg_lines.h"

static void graphs_clear(bdgd_ctx *c);

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local char g_err[512] = "";

void bdgd_set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
}

int bdgd_check(cudaError_t e, const char *what) {
  bdgd_set_error("%s: %s", what, cudaGetErrorString(e));
  return BDGD_ERR_CUDA;
}

extern "C" const char *bdgd_last_error(void) { return g_err; }

static unsigned long long g_launches = 0;
thread_local int bdgd_capturing = 0;
void bdgd_count_launch(void) { __atomic_add_fetch(&g_launches, 1ULL, __ATOMIC_RELAXED); }
static void count_launches(unsigned long long n) { __atomic_add_fetch(&g_launches, n, __ATOMIC_RELAXED); }
extern "C" unsigned long long bdgd_launch_count(void) { return __atomic_load_n(&g_launches, __ATOMIC_RELAXED); }

extern "C" int bdgd_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

// Grow a scratch buffer, stream-ordered on st (no device-wide sync, so
// solves on other streams keep running).
int bdgd_ensure(cudaStream_t st, void **ptr, size_t *have, size_t want) {
  if (*have >= want && *ptr) return BDGD_OK;
  if (*ptr) BDGD_CK(cudaFreeAsync(*ptr, st));
  *ptr = nullptr;
  *have = 0;
  if (want == 0) return BDGD_OK;
  BDGD_CK(cudaMallocAsync(ptr, want, st));
  *have = want;
  return BDGD_OK;
}


// One Stockham stage of radix R over `nlines` lines of length n in shared
// memory (line l at a + l*ls), a -> b.
template <int R, typename C>
__device__ __forceinline__ void stage_r(const C *__restrict__ a, C *__restrict__ b, int nlines,
                                        int ls, int n, int Ns, const C *roots, int sgn) {
  const int nb = n / R;
  const int tot = nlines * nb;
  const int tw = n / (Ns * R);
  for (int t = threadIdx.x; t < tot; t += blockDim.x) {
    const int line = t / nb;
    const int j = t - line * nb;
    const C *src = a + line * ls;
    C *dst = b + line * ls;
    const int k = j % Ns;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[j + r * nb];
    if (k) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], rootv(roots, r * k * tw, sgn));
    }
    Bfly<R, C>::run(v, sgn);
    const int base = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[base + r * Ns] = v[r];
  }
}

// Generic odd prime radix (5, 7, 11, 13): direct DFT with table roots.
template <typename C>
__device__ void stage_gen(const C *__restrict__ a, C *__restrict__ b, int nlines, int ls, int n,
                          int Ns, int R, const C *roots, int sgn) {
  const int nb = n / R;
  const int tot = nlines * nb;
  const int tw = n / (Ns * R);
  const int wstep = n / R;
  for (int t = threadIdx.x; t < tot; t += blockDim.x) {
    const int line = t / nb;
    const int j = t - line * nb;
    const C *src = a + line * ls;
    C *dst = b + line * ls;
    const int k = j % Ns;
    C v[16];
    for (int r = 0; r < R; ++r) {
      v[r] = src[j + r * nb];
      if (k && r) v[r] = cmul(v[r], rootv(roots, r * k * tw, sgn));
    }
    const int base = (j / Ns) * Ns * R + k;
    for (int q = 0; q < R; ++q) {
      C acc = v[0];
      for (int r = 1; r < R; ++r) acc = cadd(acc, cmul(v[r], rootv(roots, ((r * q) % R) * wstep, sgn)));
      dst[base + q * Ns] = acc;
    }
  }
}

// Full FFT of `nlines` lines held in shared memory buffer a (scratch b).
// Caller synchronises before; returns the buffer that holds the result
// (synchronised).
template <typename C>
__device__ C *smem_fft(C *a, C *b, int nlines, int ls, const AxisDev &ax, int sgn) {
  const C *roots = roots_of<C>(ax);
  int Ns = 1;
  for (int s = 0; s < ax.nst; ++s) {
    const int R = ax.rad[s];
    switch (R) {
      case 8: stage_r<8>(a, b, nlines, ls, ax.n, Ns, roots, sgn); break;
      case 4: stage_r<4>(a, b, nlines, ls, ax.n, Ns, roots, sgn); break;
      case 2: stage_r<2>(a, b, nlines, ls, ax.n, Ns, roots, sgn); break;
      case 3: stage_r<3>(a, b, nlines, ls, ax.n, Ns, roots, sgn); break;
      default: stage_gen(a, b, nlines, ls, ax.n, Ns, R, roots, sgn); break;
    }
    __syncthreads();
    C *t = a;
    a = b;
    b = t;
    Ns *= R;
  }
  return a;
}


static Prog make_prog(int op, int dipolar) {
  Prog p;
  memset(&p, 0, sizeof p);
  auto set_half = [&](int h, int kind) {
    switch (kind) {
      case BDGD_OP_KINETIC:
        p.nf[h] = 1; p.pre[h][0] = PRE_NONE; p.mul[h][0] = MUL_KIN; p.post[h] = POST_RAW; break;
      case BDGD_OP_K:
        p.nf[h] = 1; p.pre[h][0] = PRE_NONE; p.mul[h][0] = MUL_KIN; p.post[h] = POST_K; break;
      case BDGD_OP_M:
        p.nf[h] = dipolar ? 2 : 1;
        p.pre[h][0] = PRE_NONE; p.mul[h][0] = MUL_KIN;
        p.pre[h][1] = PRE_CONJWF; p.mul[h][1] = MUL_DIP;
        p.post[h] = POST_M; break;
      case BDGD_OP_TK:
        p.nf[h] = 1; p.pre[h][0] = PRE_PK; p.mul[h][0] = MUL_PRE; p.post[h] = POST_TK; break;
      case BDGD_OP_TM:
        p.nf[h] = 1; p.pre[h][0] = PRE_PM; p.mul[h][0] = MUL_PRE; p.post[h] = POST_TM; break;
      case BDGD_OP_DIPCONV:
        p.nf[h] = 1; p.pre[h][0] = PRE_CONJWF; p.mul[h][0] = MUL_DIP; p.post[h] = POST_DIPCONV; break;
      case 100:  // dipolar mean field of |psi0|^2
        p.nf[h] = 1; p.pre[h][0] = PRE_DENS; p.mul[h][0] = MUL_DIP; p.post[h] = POST_PHI; break;
      case 101:  // exp(-kin_dt k^2) propagator (imaginary-time kinetic half step)
        p.nf[h] = 1; p.pre[h][0] = PRE_NONE; p.mul[h][0] = MUL_EXPKIN; p.post[h] = POST_RAW; break;
      case 102:  // dipolar mean field of the input field |x|^2
        p.nf[h] = 1; p.pre[h][0] = PRE_XDENS; p.mul[h][0] = MUL_DIP; p.post[h] = POST_PHI; break;
    }
  };
  if (op == BDGD_OP_LREP) {
    p.nh = 2; set_half(0, BDGD_OP_K); set_half(1, BDGD_OP_M);
  } else if (op == BDGD_OP_TLREP) {
    p.nh = 2; set_half(0, BDGD_OP_TK); set_half(1, BDGD_OP_TM);
  } else {
    p.nh = 1; set_half(0, op);
  }
  int j = 0;
  for (int h = 0; h < p.nh; ++h) {
    p.j0[h] = j;
    for (int f = 0; f < p.nf[h]; ++f) { p.jh[j] = h; p.jf[j] = f; ++j; }
  }
  p.J = j;
  return p;
}


// ---------------------------------------------------------------------------
// pass kernels
// ---------------------------------------------------------------------------
// Rows along x, forward.  grid.x: row blocks, grid.y: ncol*J jobs.
template <typename T, bool CPLX>
__global__ void __launch_bounds__(256) k_row_fwd(GeoDev g, Prog p, FieldsDev f, const void *__restrict__ xin,
                                                 long long ldx, typename Cx<T>::t *__restrict__ spec, int rpb) {
  typedef typename El<T, CPLX>::C C;
  typedef typename El<T, CPLX>::V V;
  extern __shared__ __align__(16) unsigned char smraw[];
  C *a = (C *)smraw;
  const int Nx = g.N[0];
  C *b = a + rpb * Nx;
  const int job = blockIdx.y;
  const int col = job / p.J;
  const int jj = job - col * p.J;
  const int h = p.jh[jj], fi = p.jf[jj];
  const int pre = p.pre[h][fi];
  const V *src = (const V *)xin + (long long)col * ldx + (long long)h * g.S;
  const int row0 = blockIdx.x * rpb;
  const int nr = min(rpb, g.nrows - row0);
  for (int q = threadIdx.x; q < nr * Nx; q += blockDim.x) {
    const long long r = (long long)row0 * Nx + q;
    a[q] = prologue<T, CPLX>(f, pre, src[r], r);
  }
  __syncthreads();
  C *res = smem_fft(a, b, nr, Nx, g.ax[0], -1);
  C *dst = spec + (long long)job * g.H + (long long)row0 * g.nxk;
  const int nxk = g.nxk;
  for (int q = threadIdx.x; q < nr * nxk; q += blockDim.x) {
    const int rr = q / nxk, kx = q - rr * nxk;
    dst[q] = res[rr * Nx + kx];
  }
}

// Pencils along y (axis 1) or z (axis 2).  mode 0 forward, 1 inverse,
// 2 fused forward + multiply + inverse.  grid.x: kx tiles * outer, grid.y: jobs.
template <typename T>
__global__ void __launch_bounds__(256) k_col_pass(GeoDev g, Prog p, FieldsDev f,
                                                  typename Cx<T>::t *__restrict__ spec, int axis, int mode,
                                                  int tx) {
  typedef typename Cx<T>::t C;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int n = g.N[axis];
  const int ld = n + 1;
  C *a = (C *)smraw;
  C *b = a + tx * ld;
  const int nxk = g.nxk;
  const int ntx = (nxk + tx - 1) / tx;
  const int tile = blockIdx.x % ntx;
  const int outer = blockIdx.x / ntx;
  const int kx0 = tile * tx;
  const int nt = min(tx, nxk - kx0);
  long long ls, os;
  if (axis == 1) {
    ls = nxk;
    os = (long long)nxk * g.N[1];
  } else {
    ls = (long long)nxk * g.N[1];
    os = nxk;
  }
  const int job = blockIdx.y;
  C *base = spec + (long long)job * g.H + (long long)outer * os + kx0;
  for (int q = threadIdx.x; q < n * tx; q += blockDim.x) {
    const int i = q / tx, t = q - i * tx;
    if (t < nt) a[t * ld + i] = base[(long long)i * ls + t];
  }
  __syncthreads();
  C *res = smem_fft(a, b, nt, ld, g.ax[axis], mode == 1 ? +1 : -1);
  if (mode == 2) {
    const int col = job / p.J;
    const int jj = job - col * p.J;
    const int kind = p.mul[p.jh[jj]][p.jf[jj]];
    for (int q = threadIdx.x; q < n * nt; q += blockDim.x) {
      const int t = q / n, i = q - t * n;
      const int ix = kx0 + t;
      int iy, iz;
      if (axis == 1) {
        iy = i;
        iz = outer;
      } else {
        iy = outer;
        iz = i;
      }
      const long long kidx = ((long long)iz * g.N[1] + iy) * nxk + ix;
      const double m = kmult(g, f, kind, ix, iy, iz, kidx);
      res[t * ld + i] = cscale(res[t * ld + i], (T)m);
    }
    __syncthreads();
    C *other = (res == a) ? b : a;
    res = smem_fft(res, other, nt, ld, g.ax[axis], +1);
  }
  for (int q = threadIdx.x; q < n * tx; q += blockDim.x) {
    const int i = q / tx, t = q - i * tx;
    if (t < nt) base[(long long)i * ls + t] = res[t * ld + i];
  }
}


// Rows along x, inverse + epilogue.  grid.x: row blocks, grid.y: ncol*nh units.
template <typename T, bool CPLX>
__global__ void __launch_bounds__(256) k_row_inv(GeoDev g, Prog p, FieldsDev f,
                                                 const typename Cx<T>::t *__restrict__ spec,
                                                 const void *__restrict__ xin, long long ldx, void *__restrict__ yout,
                                                 long long ldy, int rpb) {
  typedef typename El<T, CPLX>::C C;
  typedef typename El<T, CPLX>::V V;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int Nx = g.N[0];
  const int nxk = g.nxk;
  const int unit = blockIdx.y;
  const int col = unit / p.nh;
  const int h = unit - col * p.nh;
  const int nf = p.nf[h];
  const int row0 = blockIdx.x * rpb;
  const int nr = min(rpb, g.nrows - row0);
  C *buf = (C *)smraw;
  C *res[2] = {nullptr, nullptr};
  for (int fi = 0; fi < nf; ++fi) {
    C *a = buf + (2 * fi) * rpb * Nx;
    C *b = a + rpb * Nx;
    const C *src = spec + ((long long)col * p.J + p.j0[h] + fi) * g.H + (long long)row0 * nxk;
    for (int q = threadIdx.x; q < nr * Nx; q += blockDim.x) {
      const int rr = q / Nx, kx = q - rr * Nx;
      C v;
      if (CPLX || kx < nxk) {
        v = src[rr * nxk + kx];
      } else {
        v = cconj(src[rr * nxk + (Nx - kx)]);
      }
      a[q] = v;
    }
    __syncthreads();
    res[fi] = smem_fft(a, b, nr, Nx, g.ax[0], +1);
  }
  const V *xs = (const V *)xin + (long long)col * ldx + (long long)h * g.S;
  V *ys = (V *)yout + (long long)col * ldy + (long long)h * g.S;
  const int post = p.post[h];
  for (int q = threadIdx.x; q < nr * Nx; q += blockDim.x) {
    const long long r = (long long)row0 * Nx + q;
    C o0 = res[0][q];
    C o1 = (nf > 1) ? res[1][q] : o0;
    V xv = (post == POST_K || post == POST_M) ? xs[r] : V();
    ys[r] = epilogue<T, CPLX>(f, post, nf, o0, o1, xv, r);
  }
}

// 1D problems: one kernel does prologue, forward, multiply, inverse and
// epilogue per row.  grid.y: units.
template <typename T, bool CPLX>
__global__ void __launch_bounds__(256) k_row_fused1d(GeoDev g, Prog p, FieldsDev f, const void *__restrict__ xin,
                                                     long long ldx, void *__restrict__ yout, long long ldy) {
  typedef typename El<T, CPLX>::C C;
  typedef typename El<T, CPLX>::V V;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int Nx = g.N[0];
  const int unit = blockIdx.y;
  const int col = unit / p.nh;
  const int h = unit - col * p.nh;
  const int nf = p.nf[h];
  C *buf = (C *)smraw;
  C *res[2] = {nullptr, nullptr};
  const V *xs = (const V *)xin + (long long)col * ldx + (long long)h * g.S;
  V *ys = (V *)yout + (long long)col * ldy + (long long)h * g.S;
  for (int fi = 0; fi < nf; ++fi) {
    C *a = buf + (2 * fi) * Nx;
    C *b = a + Nx;
    const int pre = p.pre[h][fi];
    for (int q = threadIdx.x; q < Nx; q += blockDim.x) a[q] = prologue<T, CPLX>(f, pre, xs[q], q);
    __syncthreads();
    C *r = smem_fft(a, b, 1, Nx, g.ax[0], -1);
    const int kind = p.mul[h][fi];
    for (int q = threadIdx.x; q < Nx; q += blockDim.x) {
      // full-length spectrum: kx2 is defined on all N entries (wrapped k)
      const int kk = (CPLX || q < g.nxk) ? q : (Nx - q);
      const double m = kmult(g, f, kind, q, 0, 0, kk);
      r[q] = cscale(r[q], (T)m);
    }
    __syncthreads();
    C *o = (r == a) ? b : a;
    res[fi] = smem_fft(r, o, 1, Nx, g.ax[0], +1);
  }
  const int post = p.post[h];
  for (int q = threadIdx.x; q < Nx; q += blockDim.x) {
    C o0 = res[0][q];
    C o1 = (nf > 1) ? res[1][q] : o0;
    V xv = (post == POST_K || post == POST_M) ? xs[q] : V();
    ys[q] = epilogue<T, CPLX>(f, post, nf, o0, o1, xv, q);
  }
}

// ---------------------------------------------------------------------------
// compile-time sized passes (line lengths 16..256 with radices 8/4/2/3)
// ---------------------------------------------------------------------------
// s-th radix of the compile-time plan: 8s first, then 4, 2, 3
__host__ __device__ constexpr int ct_factor(int n, int s) {
  int idx = 0;
  while (n > 1) {
    const int r = (n % 8 == 0) ? 8 : (n % 4 == 0) ? 4 : (n % 2 == 0) ? 2 : (n % 3 == 0) ? 3 : n;
    if (idx == s) return r;
    n /= r;
    ++idx;
  }
  return 1;
}
__host__ __device__ constexpr int ct_nst(int n) {
  int c = 0;
  while (n > 1) {
    const int r = (n % 8 == 0) ? 8 : (n % 4 == 0) ? 4 : (n % 2 == 0) ? 2 : (n % 3 == 0) ? 3 : n;
    n /= r;
    ++c;
  }
  return c;
}
__host__ __device__ constexpr int ct_ns(int n, int s) {
  int p = 1;
  for (int i = 0; i < s; ++i) p *= ct_factor(n, i);
  return p;
}
// threads per line: butterflies of the first (largest-radix) stage
__host__ __device__ constexpr int ct_tpl(int n) { return n / ct_factor(n, 0); }

static bool ct_supported(int n) {
  return n == 16 || n == 32 || n == 48 || n == 64 || n == 96 || n == 128 || n == 256;
}

// Shared-memory index of line element i: one pad slot every 8 elements
// breaks the stride-R bank conflicts of the Stockham writes.
__host__ __device__ constexpr int ct_pad(int i) { return i + (i >> 3); }
__host__ __device__ constexpr int ct_line(int n) { return ct_pad(n - 1) + 1; }

// One in-place Stockham stage: every thread first reads all the inputs of
// its butterflies into registers, the block synchronises, then it writes.
template <typename C, int N, int S, int TPL>
__device__ __forceinline__ void ct_stage(C *__restrict__ a, int lt, const C *roots, int sgn, bool on) {
  constexpr int R = ct_factor(N, S);
  constexpr int Ns = ct_ns(N, S);
  constexpr int nb = N / R;
  constexpr int tw = N / (Ns * R);
  constexpr int iters = (nb + TPL - 1) / TPL;
  C v[iters][R];
  if (on) {
#pragma unroll
    for (int it = 0; it < iters; ++it) {
      const int j = lt + it * TPL;
      if ((nb % TPL == 0) || j < nb) {
#pragma unroll
        for (int r = 0; r < R; ++r) v[it][r] = a[ct_pad(j + r * nb)];
      }
    }
  }
  __syncthreads();
  if (on) {
#pragma unroll
    for (int it = 0; it < iters; ++it) {
      const int j = lt + it * TPL;
      if ((nb % TPL == 0) || j < nb) {
        const int k = j % Ns;
        if (Ns > 1 && k) {
#pragma unroll
          for (int r = 1; r < R; ++r) v[it][r] = cmul(v[it][r], rootv(roots, r * k * tw, sgn));
        }
        Bfly<R, C>::run(v[it], sgn);
        const int base = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) a[ct_pad(base + r * Ns)] = v[it][r];
      }
    }
  }
  __syncthreads();
}

// All threads of the block call this; the result is in place in `a`
// (this thread's line, padded layout).
template <typename C, int N, int TPL, int S = 0>
__device__ __forceinline__ void ct_fft(C *a, int lt, const C *roots, int sgn, bool on) {
  if constexpr (S < ct_nst(N)) {
    ct_stage<C, N, S, TPL>(a, lt, roots, sgn, on);
    ct_fft<C, N, TPL, S + 1>(a, lt, roots, sgn, on);
  }
}


// Rows along x, forward, all NF spectra of one half per CTA (x read once).
// grid.x: row blocks, grid.y: columns; half h fixed per launch.
template <typename T, bool CPLX, int NX, int NF>
__global__ void __launch_bounds__(256, 4) k_row_fwd_ct(GeoDev g, Prog p, FieldsDev f, const void *__restrict__ xin,
                                                       long long ldx, typename Cx<T>::t *__restrict__ spec, int h) {
  typedef typename El<T, CPLX>::C C;
  typedef typename El<T, CPLX>::V V;
  constexpr int TPL = ct_tpl(NX);
  constexpr int LPG = (256 / NF) / TPL;  // rows per CTA
  constexpr int LN = ct_line(NX);        // padded line length
  extern __shared__ __align__(16) unsigned char smraw[];
  C *a = (C *)smraw;                     // [NF][LPG][LN]
  const int col = blockIdx.y;
  const V *src = (const V *)xin + (long long)col * ldx + (long long)h * g.S;
  const int row0 = blockIdx.x * LPG;
  const int nr = min(LPG, g.nrows - row0);
  for (int q = threadIdx.x; q < nr * NX; q += blockDim.x) {
    const int rr = q / NX, ix = q - rr * NX;
    const long long r = (long long)row0 * NX + q;
    const V xv = src[r];
#pragma unroll
    for (int fi = 0; fi < NF; ++fi) a[(fi * LPG + rr) * LN + ct_pad(ix)] = prologue<T, CPLX>(f, p.pre[h][fi], xv, r);
  }
  __syncthreads();
  const int t = threadIdx.x;
  const int grp = t / (LPG * TPL);  // field
  const int tl = t - grp * LPG * TPL;
  const int line = tl / TPL, lt = tl - line * TPL;
  const bool act = grp < NF;
  const int li = act ? (grp * LPG + line) : 0;
  ct_fft<C, NX, TPL>(a + li * LN, lt, roots_of<C>(g.ax[0]), -1, act);
  const int nxk = g.nxk;
#pragma unroll
  for (int fi = 0; fi < NF; ++fi) {
    C *dst = spec + ((long long)col * p.J + p.j0[h] + fi) * g.H + (long long)row0 * nxk;
    for (int q = threadIdx.x; q < nr * nxk; q += blockDim.x) {
      const int rr = q / nxk, kx = q - rr * nxk;
      dst[q] = a[(fi * LPG + rr) * LN + ct_pad(kx)];
    }
  }
}

// Pencils along y / z with compile-time length N (see k_col_pass).
template <typename T, int N>
__global__ void __launch_bounds__(256, 4) k_col_pass_ct(GeoDev g, Prog p, FieldsDev f,
                                                        typename Cx<T>::t *__restrict__ spec, int axis, int mode) {
  typedef typename Cx<T>::t C;
  constexpr int TPL = ct_tpl(N);
  constexpr int TX = 256 / TPL;         // lines (kx values) per CTA
  constexpr int LD = ct_line(N) | 1;    // odd line stride for the transposed loads
  extern __shared__ __align__(16) unsigned char smraw[];
  C *a = (C *)smraw;                    // [TX][LD]
  const int nxk = g.nxk;
  const int ntx = (nxk + TX - 1) / TX;
  const int tile = blockIdx.x % ntx;
  const int outer = blockIdx.x / ntx;
  const int kx0 = tile * TX;
  const int nt = min(TX, nxk - kx0);
  long long ls, os;
  if (axis == 1) {
    ls = nxk;
    os = (long long)nxk * g.N[1];
  } else {
    ls = (long long)nxk * g.N[1];
    os = nxk;
  }
  const int job = blockIdx.y;
  C *base = spec + (long long)job * g.H + (long long)outer * os + kx0;
  for (int q = threadIdx.x; q < N * TX; q += blockDim.x) {
    const int i = q / TX, t = q - i * TX;
    if (t < nt) a[t * LD + ct_pad(i)] = base[(long long)i * ls + t];
  }
  __syncthreads();
  const int line = threadIdx.x / TPL, lt = threadIdx.x - line * TPL;
  const bool on = line < TX;
  const int ln = on ? line : 0;
  const C *roots = roots_of<C>(g.ax[axis]);
  ct_fft<C, N, TPL>(a + ln * LD, lt, roots, mode == 1 ? +1 : -1, on);
  if (mode == 2) {
    const int col = job / p.J;
    const int jj = job - col * p.J;
    const int kind = p.mul[p.jh[jj]][p.jf[jj]];
    for (int q = threadIdx.x; q < N * nt; q += blockDim.x) {
      const int t = q / N, i = q - t * N;
      const int ix = kx0 + t;
      int iy, iz;
      if (axis == 1) {
        iy = i;
        iz = outer;
      } else {
        iy = outer;
        iz = i;
      }
      const long long kidx = ((long long)iz * g.N[1] + iy) * nxk + ix;
      const double m = kmult(g, f, kind, ix, iy, iz, kidx);
      C &e = a[t * LD + ct_pad(i)];
      e = cscale(e, (T)m);
    }
    __syncthreads();
    ct_fft<C, N, TPL>(a + ln * LD, lt, roots, +1, on);
  }
  for (int q = threadIdx.x; q < N * TX; q += blockDim.x) {
    const int i = q / TX, t = q - i * TX;
    if (t < nt) base[(long long)i * ls + t] = a[t * LD + ct_pad(i)];
  }
}

// Rows along x, inverse of the NF spectra of one half + epilogue.
// grid.x: row blocks, grid.y: columns; half h fixed per launch.
template <typename T, bool CPLX, int NX, int NF>
__global__ void __launch_bounds__(256, 4) k_row_inv_ct(GeoDev g, Prog p, FieldsDev f,
                                                       const typename Cx<T>::t *__restrict__ spec,
                                                       const void *__restrict__ xin, long long ldx,
                                                       void *__restrict__ yout, long long ldy, int h) {
  typedef typename El<T, CPLX>::C C;
  typedef typename El<T, CPLX>::V V;
  constexpr int TPL = ct_tpl(NX);
  constexpr int LPG = (256 / NF) / TPL;
  constexpr int LN = ct_line(NX);
  extern __shared__ __align__(16) unsigned char smraw[];
  C *a = (C *)smraw;  // [NF][LPG][LN]
  const int nxk = g.nxk;
  const int col = blockIdx.y;
  const int row0 = blockIdx.x * LPG;
  const int nr = min(LPG, g.nrows - row0);
#pragma unroll
  for (int fi = 0; fi < NF; ++fi) {
    const C *src = spec + ((long long)col * p.J + p.j0[h] + fi) * g.H + (long long)row0 * nxk;
    for (int q = threadIdx.x; q < nr * NX; q += blockDim.x) {
      const int rr = q / NX, kx = q - rr * NX;
      C v;
      if (CPLX || kx < nxk)
        v = src[rr * nxk + kx];
      else
        v = cconj(src[rr * nxk + (NX - kx)]);
      a[(fi * LPG + rr) * LN + ct_pad(kx)] = v;
    }
  }
  __syncthreads();
  const int t = threadIdx.x;
  const int grp = t / (LPG * TPL);
  const int tl = t - grp * LPG * TPL;
  const int line = tl / TPL, lt = tl - line * TPL;
  const bool act = grp < NF;
  const int li = act ? (grp * LPG + line) : 0;
  ct_fft<C, NX, TPL>(a + li * LN, lt, roots_of<C>(g.ax[0]), +1, act);
  const V *xs = (const V *)xin + (long long)col * ldx + (long long)h * g.S;
  V *ys = (V *)yout + (long long)col * ldy + (long long)h * g.S;
  const int post = p.post[h];
  for (int q = threadIdx.x; q < nr * NX; q += blockDim.x) {
    const int rr = q / NX, ix = q - rr * NX;
    const long long r = (long long)row0 * NX + q;
    const C o0 = a[rr * LN + ct_pad(ix)];
    const C o1 = (NF > 1) ? a[(LPG + rr) * LN + ct_pad(ix)] : o0;
    const V xv = (post == POST_K || post == POST_M) ? xs[r] : V();
    ys[r] = epilogue<T, CPLX>(f, post, NF, o0, o1, xv, r);
  }
}

// Swap: y = [x_v; x_u] (src/matmulSwap_impl.inc:18-22), copied in words of W.
template <typename W>
__global__ void k_swap(const unsigned char *__restrict__ x, long long ldxb, unsigned char *__restrict__ y,
                       long long ldyb, long long halfb) {
  const long long nw = halfb / (long long)sizeof(W);
  const long long col = blockIdx.y;
  const W *xs = (const W *)(x + col * ldxb);
  W *ys = (W *)(y + col * ldyb);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nw;
       i += (long long)gridDim.x * blockDim.x) {
    ys[i] = xs[nw + i];
    ys[nw + i] = xs[i];
  }
}

// ---------------------------------------------------------------------------
// host side: context
// ---------------------------------------------------------------------------
static int factorize(int n, int *rad) {
  int k = 0;
  if (n == 1) return 0;
  while (n % 8 == 0 && n > 8 && k < BDGD_MAX_STAGES) { rad[k++] = 8; n /= 8; }
  while (n % 4 == 0 && k < BDGD_MAX_STAGES) { rad[k++] = 4; n /= 4; }
  while (n % 2 == 0 && k < BDGD_MAX_STAGES) { rad[k++] = 2; n /= 2; }
  while (n % 8 == 0 && k < BDGD_MAX_STAGES) { rad[k++] = 8; n /= 8; }
  const int primes[] = {3, 5, 7, 11, 13};
  for (int pi = 0; pi < 5; ++pi)
    while (n % primes[pi] == 0 && k < BDGD_MAX_STAGES) { rad[k++] = primes[pi]; n /= primes[pi]; }
  if (n != 1) return -1;
  return k;
}

// Stage order: radix 8 first (largest butterflies on the Ns = 1 stage).
static int plan_axis(int n, int *rad) {
  int tmp[BDGD_MAX_STAGES];
  int k = factorize(n, tmp);
  if (k < 0) return -1;
  // pull 8s together: factorize returns 8s only when n has 16 | n; recombine 4*2 -> 8
  int c8 = 0, c4 = 0, c2 = 0, cnt = 0;
  int others[BDGD_MAX_STAGES];
  int no = 0;
  for (int i = 0; i < k; ++i) {
    if (tmp[i] == 8) c8++;
    else if (tmp[i] == 4) c4++;
    else if (tmp[i] == 2) c2++;
    else others[no++] = tmp[i];
  }
  int p2 = 3 * c8 + 2 * c4 + c2;  // power of two exponent
  while (p2 >= 3) { rad[cnt++] = 8; p2 -= 3; }
  if (p2 == 2) rad[cnt++] = 4;
  if (p2 == 1) rad[cnt++] = 2;
  for (int i = 0; i < no; ++i) rad[cnt++] = others[i];
  return cnt;
}

extern "C" int bdgd_create(bdgd_ctx **out, uint64_t dim, const uint64_t *N, const double *L,
                           int complex_psi0) {
  *out = nullptr;
  if (dim < 1 || dim > 3) {
    bdgd_set_error("bdgd_create: dim must be 1, 2 or 3");
    return BDGD_ERR_ARG;
  }
  bdgd_ctx *c = (bdgd_ctx *)calloc(1, sizeof(bdgd_ctx));
  if (!c) return BDGD_ERR_ARG;
  c->dim = (int)dim;
  c->cplx = complex_psi0 ? 1 : 0;
  for (int d = 0; d < 3; ++d) {
    c->N[d] = d < (int)dim ? (int)N[d] : 1;
    c->L[d] = d < (int)dim ? L[d] : 1.0;
  }
  c->S = (long long)c->N[0] * c->N[1] * c->N[2];
  c->nxk = c->cplx ? c->N[0] : c->N[0] / 2 + 1;
  c->H = (long long)c->nxk * c->N[1] * c->N[2];
  c->spec_cap = (size_t)4 << 30;
  c->graphs_on = getenv("BDG_GRAPHS") && atoi(getenv("BDG_GRAPHS")) != 0;
  if (const char *e = getenv("BDG_SPEC_CAP_MB")) c->spec_cap = (size_t)atoll(e) << 20;
  if (cudaGetDevice(&c->device) != cudaSuccess) {
    cudaGetLastError();
    free(c);
    bdgd_set_error("bdgd_create: no CUDA device");
    return BDGD_ERR_CUDA;
  }
  {
    // keep freed stream-ordered scratch in the device pool for reuse
    static std::atomic<int> pool_done[64];  // several solver threads create contexts at once
    if (c->device >= 0 && c->device < 64 && !pool_done[c->device].exchange(1)) {
      cudaMemPool_t pool;
      if (cudaDeviceGetDefaultMemPool(&pool, c->device) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
      }
      cudaGetLastError();
    }
  }
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    free(c);
    return bdgd_check(e, "cudaStreamCreateWithFlags");
  }
  GeoDev &g = c->geo;
  memset(&g, 0, sizeof g);
  g.dim = c->dim;
  g.cplx = c->cplx;
  for (int d = 0; d < 3; ++d) g.N[d] = c->N[d];
  g.nxk = c->nxk;
  g.nrows = (int)(c->S / c->N[0]);
  g.S = c->S;
  g.H = c->H;
  for (int d = 0; d < 3; ++d) {
    const int n = c->N[d];
    int nst = plan_axis(n, g.ax[d].rad);
    if (nst < 0) {
      bdgd_set_error("bdgd_create: N[%d] = %d has a prime factor above 13", d, n);
      bdgd_destroy(&c);
      return BDGD_ERR_UNSUPPORTED;
    }
    g.ax[d].n = n;
    g.ax[d].nst = nst;
    double2 *h64 = (double2 *)malloc(sizeof(double2) * n);
    float2 *h32 = (float2 *)malloc(sizeof(float2) * n);
    double *hk = (double *)malloc(sizeof(double) * n);
    const long double tau = 6.283185307179586476925286766559L;
    for (int m = 0; m < n; ++m) {
      // exp(-2 pi i m/n), reduced to the first octant's symmetric angle for accuracy
      long double ang = tau * (long double)m / (long double)n;
      h64[m].x = (double)cosl(ang);
      h64[m].y = (double)-sinl(ang);
      h32[m].x = (float)h64[m].x;
      h32[m].y = (float)h64[m].y;
      // k_j^2 as the reference builds kx2 (src/matmul_ctx.c:103-113)
      const double dk = 2.0 * M_PI / c->L[d];
      const double kj = (m <= n / 2) ? (dk * (double)m) : (dk * (double)(m - n));
      hk[m] = kj * kj;
    }
    cudaError_t e1 = cudaMalloc(&c->d_roots64[d], sizeof(double2) * n);
    cudaError_t e2 = cudaMalloc(&c->d_roots32[d], sizeof(float2) * n);
    cudaError_t e3 = cudaMalloc(&c->d_kx2[d], sizeof(double) * n);
    if (e1 == cudaSuccess && e2 == cudaSuccess && e3 == cudaSuccess) {
      cudaMemcpy(c->d_roots64[d], h64, sizeof(double2) * n, cudaMemcpyHostToDevice);
      cudaMemcpy(c->d_roots32[d], h32, sizeof(float2) * n, cudaMemcpyHostToDevice);
      cudaMemcpy(c->d_kx2[d], hk, sizeof(double) * n, cudaMemcpyHostToDevice);
    }
    free(h64);
    free(h32);
    free(hk);
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
      bdgd_destroy(&c);
      return bdgd_check(cudaErrorMemoryAllocation, "cudaMalloc(tables)");
    }
    g.ax[d].r64 = c->d_roots64[d];
    g.ax[d].r32 = c->d_roots32[d];
    g.kx2[d] = c->d_kx2[d];
  }
  *out = c;
  return BDGD_OK;
}

extern "C" void bdgd_destroy(bdgd_ctx **pc) {
  if (!pc || !*pc) return;
  bdgd_ctx *c = *pc;
  if (c->stream) cudaStreamSynchronize(c->stream);
  graphs_clear(c);
  for (int d = 0; d < 3; ++d) {
    cudaFree(c->d_roots64[d]);
    cudaFree(c->d_roots32[d]);
    cudaFree(c->d_kx2[d]);
  }
  void *bufs[] = {c->ltK64, c->ltM64, c->pK64, c->pM64, c->ltK32, c->ltM32, c->pK32, c->pM32,
                  c->wf64,  c->wf32,  c->vdd,  c->ptab};
  for (void *b : bufs)
    if (b) cudaFree(b);
  void *sbufs[] = {c->spec, c->io, c->gram_part, c->oz_buf};  // stream-ordered (bdgd_ensure)
  for (void *b : sbufs)
    if (b) cudaFreeAsync(b, c->stream);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->stream) cudaStreamDestroy(c->stream);
  free(c);
  *pc = nullptr;
}

extern "C" void *bdgd_stream(bdgd_ctx *c) { return c ? (void *)c->stream : nullptr; }

extern "C" int bdgd_synchronize(bdgd_ctx *c) {
  BDGD_CK(cudaStreamSynchronize(c->stream));
  return BDGD_OK;
}

// Preconditioner multiplier table for the current mu: the k-space factor of
// T at every spectrum point, computed by kmult itself (bit-identical to the
// on-the-fly value); read once per spectrum pass instead of a division per
// element.
__global__ void k_ptab(GeoDev g, FieldsDev f, double *__restrict__ out) {
  const long long n = g.H;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(i % g.nxk);
    const long long r = i / g.nxk;
    const int iy = g.dim > 1 ? (int)(r % g.N[1]) : 0;
    const int iz = g.dim > 2 ? (int)(r / g.N[1]) : 0;
    out[i] = kmult(g, f, MUL_PRE, ix, iy, iz, i);
  }
}

static int build_ptab(bdgd_ctx *c) {
  if (!c->ptab) BDGD_CK(cudaMalloc((void **)&c->ptab, sizeof(double) * c->H));
  FieldsDev f;
  memset(&f, 0, sizeof f);
  f.mu = c->mu;
  f.inv_size = 1.0 / (double)c->S;
  f.ptab = nullptr;
  long long blocks = (c->H + 255) / 256;
  if (blocks > 4096) blocks = 4096;
  bdgd_count_launch();
  k_ptab<<<(unsigned)blocks, 256, 0, c->stream>>>(c->geo, f, c->ptab);
  BDGD_CK(cudaGetLastError());
  BDGD_CK(cudaStreamSynchronize(c->stream));
  return BDGD_OK;
}

// upload a host double array and its float copy
static int upload_pair(bdgd_ctx *c, double **d64, float **d32, const double *h, long long n) {
  if (!*d64) BDGD_CK(cudaMalloc((void **)d64, sizeof(double) * n));
  if (!*d32) BDGD_CK(cudaMalloc((void **)d32, sizeof(float) * n));
  BDGD_CK(cudaMemcpyAsync(*d64, h, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
  float *tmp = (float *)malloc(sizeof(float) * n);
  for (long long i = 0; i < n; ++i) tmp[i] = (float)h[i];
  cudaError_t e = cudaMemcpyAsync(*d32, tmp, sizeof(float) * n, cudaMemcpyHostToDevice, c->stream);
  cudaError_t e2 = cudaStreamSynchronize(c->stream);
  free(tmp);
  if (e != cudaSuccess) return bdgd_check(e, "upload");
  if (e2 != cudaSuccess) return bdgd_check(e2, "upload sync");
  return BDGD_OK;
}

extern "C" int bdgd_set_local_terms(bdgd_ctx *c, const double *ltK, const double *ltM) {
  c->version++;
  int rc;
  if (ltK && (rc = upload_pair(c, &c->ltK64, &c->ltK32, ltK, c->S))) return rc;
  if (ltM && (rc = upload_pair(c, &c->ltM64, &c->ltM32, ltM, c->S))) return rc;
  return BDGD_OK;
}

extern "C" int bdgd_set_precond(bdgd_ctx *c, const double *sK, const double *sM, double mu) {
  c->version++;
  int rc;
  if (sK && (rc = upload_pair(c, &c->pK64, &c->pK32, sK, c->S))) return rc;
  if (sM && (rc = upload_pair(c, &c->pM64, &c->pM32, sM, c->S))) return rc;
  c->mu = mu;
  c->has_precond = (sK && sM) ? 1 : c->has_precond;
  return build_ptab(c);
}

extern "C" int bdgd_set_wavefunction(bdgd_ctx *c, const void *wf) {
  c->version++;
  if (!wf) return BDGD_OK;
  const long long n = c->S * (c->cplx ? 2 : 1);
  double *d64 = (double *)c->wf64;
  float *d32 = (float *)c->wf32;
  int rc = upload_pair(c, &d64, &d32, (const double *)wf, n);
  c->wf64 = d64;
  c->wf32 = d32;
  if (rc) return rc;
  c->has_wf = 1;
  return BDGD_OK;
}

extern "C" int bdgd_set_dipolar(bdgd_ctx *c, const double *vdd, double g_ddi, int enabled) {
  c->version++;
  c->g_ddi = g_ddi;
  c->dipolar = enabled && c->dim == 3;
  if (vdd) {
    if (!c->vdd) BDGD_CK(cudaMalloc((void **)&c->vdd, sizeof(double) * c->H));
    BDGD_CK(cudaMemcpyAsync(c->vdd, vdd, sizeof(double) * c->H, cudaMemcpyHostToDevice, c->stream));
    BDGD_CK(cudaStreamSynchronize(c->stream));
  }
  return BDGD_OK;
}

// ---------------------------------------------------------------------------
// host side: apply
// ---------------------------------------------------------------------------
static const int kThreads = 256;

static int rows_per_block(int Nx) {
  int r = 1024 / Nx;
  return r < 1 ? 1 : r;
}


// ---- host launchers of the compile-time kernels ----
template <typename T, bool CPLX, int NX, int NF>
static int launch_row_fwd_ct(bdgd_ctx *c, const Prog &p, const FieldsDev &fd, const void *x, long long ldx,
                             typename Cx<T>::t *spec, int nc, int h) {
  typedef typename Cx<T>::t C;
  constexpr int LPG = (256 / NF) / ct_tpl(NX);
  const size_t sm = sizeof(C) * NF * LPG * ct_line(NX);
  if (sm > 48 * 1024)
    { const int _ra = bdgd_smem_attr(k_row_fwd_ct<T, CPLX, NX, NF>, sm); if (_ra) return _ra; }
  const int nrb = (c->geo.nrows + LPG - 1) / LPG;
  bdgd_count_launch();
  k_row_fwd_ct<T, CPLX, NX, NF><<<dim3(nrb, nc), 256, sm, c->stream>>>(c->geo, p, fd, x, ldx, spec, h);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}

template <typename T, bool CPLX, int NX, int NF>
static int launch_row_inv_ct(bdgd_ctx *c, const Prog &p, const FieldsDev &fd, const typename Cx<T>::t *spec,
                             const void *x, long long ldx, void *y, long long ldy, int nc, int h) {
  typedef typename Cx<T>::t C;
  constexpr int LPG = (256 / NF) / ct_tpl(NX);
  const size_t sm = sizeof(C) * NF * LPG * ct_line(NX);
  if (sm > 48 * 1024)
    { const int _ra = bdgd_smem_attr(k_row_inv_ct<T, CPLX, NX, NF>, sm); if (_ra) return _ra; }
  const int nrb = (c->geo.nrows + LPG - 1) / LPG;
  bdgd_count_launch();
  k_row_inv_ct<T, CPLX, NX, NF><<<dim3(nrb, nc), 256, sm, c->stream>>>(c->geo, p, fd, spec, x, ldx, y, ldy, h);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}

template <typename T, int N>
static int launch_col_ct(bdgd_ctx *c, const Prog &p, const FieldsDev &fd, typename Cx<T>::t *spec, int njobs,
                         int axis, int mode) {
  typedef typename Cx<T>::t C;
  constexpr int TX = 256 / ct_tpl(N);
  const size_t sm = sizeof(C) * TX * (ct_line(N) | 1);
  if (sm > 48 * 1024)
    { const int _ra = bdgd_smem_attr(k_col_pass_ct<T, N>, sm); if (_ra) return _ra; }
  const int ntx = (c->nxk + TX - 1) / TX;
  const int outer = (axis == 1) ? c->N[2] : c->N[1];
  bdgd_count_launch();
  k_col_pass_ct<T, N><<<dim3(ntx * outer, njobs), 256, sm, c->stream>>>(c->geo, p, fd, spec, axis, mode);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}

#define CT_SWITCH(n, CALL) \
  switch (n) {             \
    case 16: CALL(16);     \
    case 32: CALL(32);     \
    case 48: CALL(48);     \
    case 64: CALL(64);     \
    case 96: CALL(96);     \
    case 128: CALL(128);   \
    case 256: CALL(256);   \
    default: break;        \
  }

template <typename T, bool CPLX>
static int rows_fwd_ct(bdgd_ctx *c, const Prog &p, const FieldsDev &fd, const void *x, long long ldx,
                       typename Cx<T>::t *spec, int nc, int h) {
#define RF(NXV) return p.nf[h] == 2 ? launch_row_fwd_ct<T, CPLX, NXV, 2>(c, p, fd, x, ldx, spec, nc, h) \
                                    : launch_row_fwd_ct<T, CPLX, NXV, 1>(c, p, fd, x, ldx, spec, nc, h)
  CT_SWITCH(c->N[0], RF)
#undef RF
  return BDGD_ERR_UNSUPPORTED;
}

template <typename T, bool CPLX>
static int rows_inv_ct(bdgd_ctx *c, const Prog &p, const FieldsDev &fd, const typename Cx<T>::t *spec, const void *x,
                       long long ldx, void *y, long long ldy, int nc, int h) {
#define RI(NXV) return p.nf[h] == 2 ? launch_row_inv_ct<T, CPLX, NXV, 2>(c, p, fd, spec, x, ldx, y, ldy, nc, h) \
                                    : launch_row_inv_ct<T, CPLX, NXV, 1>(c, p, fd, spec, x, ldx, y, ldy, nc, h)
  CT_SWITCH(c->N[0], RI)
#undef RI
  return BDGD_ERR_UNSUPPORTED;
}

template <typename T>
static int cols_ct(bdgd_ctx *c, const Prog &p, const FieldsDev &fd, typename Cx<T>::t *spec, int njobs, int axis,
                   int mode) {
#define CC(NV) return launch_col_ct<T, NV>(c, p, fd, spec, njobs, axis, mode)
  CT_SWITCH(c->N[axis], CC)
#undef CC
  return BDGD_ERR_UNSUPPORTED;
}

// FFT pass family: register line transforms (default), compile-time sized
// shared-memory stages, or the generic runtime-sized kernels.  BDG_FFT_PATH
// = reg | ct | generic overrides (BDG_GENERIC_FFT=1 is the same as generic).
enum { FFT_PATH_REG = 0, FFT_PATH_CT = 1, FFT_PATH_GENERIC = 2 };
static int fft_path(const bdgd_ctx *c) {
  if (c->force_path) return c->force_path == 2 ? FFT_PATH_CT : FFT_PATH_REG;
  if (getenv("BDG_GENERIC_FFT")) return FFT_PATH_GENERIC;
  const char *e = getenv("BDG_FFT_PATH");
  if (e) {
    if (!strcmp(e, "ct")) return FFT_PATH_CT;
    if (!strcmp(e, "generic")) return FFT_PATH_GENERIC;
  }
  return FFT_PATH_REG;
}

template <typename T, bool CPLX>
static int run_program(bdgd_ctx *c, const Prog &p, const void *x, long long ldx, void *y, long long ldy,
                       int ncol, int only_fwd, int only_bwd) {
  typedef typename Cx<T>::t C;
  const bool f32 = sizeof(T) == 4;
  FieldsDev fd;
  fd.ltK = f32 ? (const void *)c->ltK32 : (const void *)c->ltK64;
  fd.ltM = f32 ? (const void *)c->ltM32 : (const void *)c->ltM64;
  fd.pK = f32 ? (const void *)c->pK32 : (const void *)c->pK64;
  fd.pM = f32 ? (const void *)c->pM32 : (const void *)c->pM64;
  fd.w = f32 ? c->wf32 : c->wf64;
  fd.vdd = c->vdd;
  fd.g_ddi = c->g_ddi;
  fd.mu = c->mu;
  fd.inv_size = 1.0 / (double)c->S;
  fd.kin_dt = c->kin_dt;
  fd.ptab = c->ptab;
  const GeoDev &g = c->geo;
  const int Nx = c->N[0];
  const int rpb = rows_per_block(Nx);
  const int nrb = (g.nrows + rpb - 1) / rpb;
  if (c->dim == 1 && !only_fwd && !only_bwd) {
    int maxnf = p.nf[0] > p.nf[p.nh - 1] ? p.nf[0] : p.nf[p.nh - 1];
    size_t sm = sizeof(C) * 2 * maxnf * Nx;
    if (sm > 48 * 1024)
      { const int _ra = bdgd_smem_attr(k_row_fused1d<T, CPLX>, sm); if (_ra) return _ra; }
    dim3 grid(1, ncol * p.nh);
    bdgd_count_launch();
    k_row_fused1d<T, CPLX><<<grid, kThreads, sm, c->stream>>>(g, p, fd, x, ldx, y, ldy);
    BDGD_CK(cudaGetLastError());
    return BDGD_OK;
  }
  // column chunking bounded by the scratch cap
  const size_t per_col = sizeof(C) * (size_t)p.J * (size_t)g.H;
  int chunk = ncol;
  if (per_col * (size_t)chunk > c->spec_cap) {
    chunk = (int)(c->spec_cap / per_col);
    if (chunk < 1) chunk = 1;
  }
  if (only_fwd || only_bwd) chunk = ncol;  // raw transforms use the whole scratch as I/O
  void *spec_before = c->spec;
  int rc = bdgd_ensure(c->stream, &c->spec, &c->spec_bytes, per_col * (size_t)chunk);
  if (rc) return rc;
  if (c->spec != spec_before) c->version++;  // captured graphs hold the old scratch
  C *spec = (C *)c->spec;
  const int tx = f32 ? 16 : 8;
  if (!only_fwd && !only_bwd && fft_path(c) == FFT_PATH_REG && bdgd_lines_usable(c, p)) {
    for (int c0 = 0; c0 < ncol; c0 += chunk) {
      const int nc = (ncol - c0) < chunk ? (ncol - c0) : chunk;
      const size_t esz = CPLX ? sizeof(C) : sizeof(T);
      const void *xc = (const char *)x + (size_t)c0 * ldx * esz;
      void *yc = (char *)y + (size_t)c0 * ldy * esz;
      int rc = bdgd_lines_apply(c, p, fd, f32 ? BDGD_F32 : BDGD_F64, xc, ldx, yc, ldy, spec, nc);
      if (rc) return rc;
    }
    return BDGD_OK;
  }
  const bool ct = (c->dim >= 2) && ct_supported(c->N[0]) && ct_supported(c->N[1]) &&
                  (c->dim < 3 || ct_supported(c->N[2])) && fft_path(c) != FFT_PATH_GENERIC;
  if (ct) {
    for (int c0 = 0; c0 < ncol; c0 += chunk) {
      const int nc = (ncol - c0) < chunk ? (ncol - c0) : chunk;
      const size_t esz = CPLX ? sizeof(C) : sizeof(T);
      const void *xc = (const char *)x + (size_t)c0 * ldx * esz;
      void *yc = (char *)y + (size_t)c0 * ldy * esz;
      int rc;
      if (!only_bwd)
        for (int h = 0; h < p.nh; ++h)
          if ((rc = rows_fwd_ct<T, CPLX>(c, p, fd, xc, ldx, spec, nc, h))) return rc;
      for (int ax = 1; ax < c->dim && !only_bwd; ++ax) {
        const int last = (ax == c->dim - 1);
        if ((rc = cols_ct<T>(c, p, fd, spec, nc * p.J, ax, (last && !only_fwd) ? 2 : 0))) return rc;
      }
      if (only_fwd) break;
      for (int ax = only_bwd ? c->dim - 1 : c->dim - 2; ax >= 1; --ax)
        if ((rc = cols_ct<T>(c, p, fd, spec, nc * p.J, ax, 1))) return rc;
      for (int h = 0; h < p.nh; ++h)
        if ((rc = rows_inv_ct<T, CPLX>(c, p, fd, spec, xc, ldx, yc, ldy, nc, h))) return rc;
    }
    return BDGD_OK;
  }
  for (int c0 = 0; c0 < ncol; c0 += chunk) {
    const int nc = (ncol - c0) < chunk ? (ncol - c0) : chunk;
    const size_t esz = CPLX ? sizeof(C) : sizeof(T);
    const void *xc = (const char *)x + (size_t)c0 * ldx * esz;
    void *yc = (char *)y + (size_t)c0 * ldy * esz;
    if (!only_bwd) {
      size_t sm = sizeof(C) * 2 * rpb * Nx;
      if (sm > 48 * 1024)
        { const int _ra = bdgd_smem_attr(k_row_fwd<T, CPLX>, sm); if (_ra) return _ra; }
      bdgd_count_launch();
      k_row_fwd<T, CPLX><<<dim3(nrb, nc * p.J), kThreads, sm, c->stream>>>(g, p, fd, xc, ldx, spec, rpb);
      BDGD_CK(cudaGetLastError());
    }
    // middle / last axes
    for (int ax = 1; ax < c->dim && !only_bwd; ++ax) {
      const int last = (ax == c->dim - 1);
      const int mode = (last && !only_fwd) ? 2 : 0;
      const int n = c->N[ax];
      const int ntx = (c->nxk + tx - 1) / tx;
      const int outer = (ax == 1) ? c->N[2] : c->N[1];
      size_t sm = sizeof(C) * 2 * tx * (n + 1);
      if (sm > 48 * 1024)
        { const int _ra = bdgd_smem_attr(k_col_pass<T>, sm); if (_ra) return _ra; }
      bdgd_count_launch();
      k_col_pass<T><<<dim3(ntx * outer, nc * p.J), kThreads, sm, c->stream>>>(g, p, fd, spec, ax, mode, tx);
      BDGD_CK(cudaGetLastError());
    }
    if (only_fwd) break;
    const int first_inv = only_bwd ? c->dim - 1 : c->dim - 2;
    for (int ax = first_inv; ax >= 1; --ax) {
      const int n = c->N[ax];
      const int ntx = (c->nxk + tx - 1) / tx;
      const int outer = (ax == 1) ? c->N[2] : c->N[1];
      size_t sm = sizeof(C) * 2 * tx * (n + 1);
      if (sm > 48 * 1024)
        { const int _ra = bdgd_smem_attr(k_col_pass<T>, sm); if (_ra) return _ra; }
      bdgd_count_launch();
      k_col_pass<T><<<dim3(ntx * outer, nc * p.J), kThreads, sm, c->stream>>>(g, p, fd, spec, ax, 1, tx);
      BDGD_CK(cudaGetLastError());
    }
    {
      int maxnf = 1;
      for (int h = 0; h < p.nh; ++h) maxnf = p.nf[h] > maxnf ? p.nf[h] : maxnf;
      size_t sm = sizeof(C) * 2 * maxnf * rpb * Nx;
      if (sm > 48 * 1024)
        { const int _ra = bdgd_smem_attr(k_row_inv<T, CPLX>, sm); if (_ra) return _ra; }
      bdgd_count_launch();
      k_row_inv<T, CPLX><<<dim3(nrb, nc * p.nh), kThreads, sm, c->stream>>>(g, p, fd, spec, xc, ldx, yc, ldy, rpb);
      BDGD_CK(cudaGetLastError());
    }
  }
  return BDGD_OK;
}

static int check_ready(bdgd_ctx *c, int op) {
  const bool needs_lt = op == BDGD_OP_K || op == BDGD_OP_M || op == BDGD_OP_LREP;
  const bool needs_p = op == BDGD_OP_TK || op == BDGD_OP_TM || op == BDGD_OP_TLREP;
  const bool needs_wf = op == BDGD_OP_DIPCONV || ((op == BDGD_OP_M || op == BDGD_OP_LREP) && c->dipolar);
  if (needs_lt && (!c->ltK64 || !c->ltM64)) {
    bdgd_set_error("operator needs localTermK/localTermM");
    return BDGD_ERR_STATE;
  }
  if (needs_p && (!c->pK64 || !c->pM64)) {
    bdgd_set_error("preconditioner needs precond_sqrtK/M (bdg_set_mu)");
    return BDGD_ERR_STATE;
  }
  if (needs_wf && !c->wf64) {
    bdgd_set_error("operator needs the wavefunction");
    return BDGD_ERR_STATE;
  }
  if ((op == BDGD_OP_DIPCONV || (c->dipolar && (op == BDGD_OP_M || op == BDGD_OP_LREP))) && !c->vdd) {
    bdgd_set_error("dipolar operator needs the dipolar kernel");
    return BDGD_ERR_STATE;
  }
  return BDGD_OK;
}

static int dispatch(bdgd_ctx *c, const Prog &p, int prec, const void *x, long long ldx, void *y, long long ldy,
                    int ncol, int only_fwd, int only_bwd) {
  if (prec == BDGD_F32) {
    if (c->cplx) return run_program<float, true>(c, p, x, ldx, y, ldy, ncol, only_fwd, only_bwd);
    return run_program<float, false>(c, p, x, ldx, y, ldy, ncol, only_fwd, only_bwd);
  }
  if (c->cplx) return run_program<double, true>(c, p, x, ldx, y, ldy, ncol, only_fwd, only_bwd);
  return run_program<double, false>(c, p, x, ldx, y, ldy, ncol, only_fwd, only_bwd);
}

// ---------------------------------------------------------------------------
// CUDA graphs of operator applies and the FFT pass-family autotuner
// ---------------------------------------------------------------------------
struct bdgd_graph {
  int op, prec, ncol, path;
  const void *x;
  void *y;
  long long ldx, ldy;
  unsigned version;
  cudaGraphExec_t exec;  // null after the first (uncaptured) use
  unsigned long long nkern, stamp;
};
#define BDGD_MAX_GRAPHS 48
static std::atomic<unsigned long long> g_graph_clock{0};  // LRU stamps from several threads

static void graphs_clear(bdgd_ctx *c) {
  for (int i = 0; i < c->ngraphs; ++i)
    if (c->graphs[i].exec) cudaGraphExecDestroy(c->graphs[i].exec);
  free(c->graphs);
  c->graphs = nullptr;
  c->ngraphs = 0;
}

extern "C" int bdgd_trim(bdgd_ctx *c) {
  if (!c) return BDGD_ERR_ARG;
  BDGD_CK(cudaStreamSynchronize(c->stream));
  graphs_clear(c);
  void **bufs[] = {&c->spec, &c->io, (void **)&c->gram_part, &c->oz_buf};
  size_t *sizes[] = {&c->spec_bytes, &c->io_bytes, &c->gram_part_bytes, &c->oz_buf_bytes};
  for (int i = 0; i < 4; ++i) {
    if (*bufs[i]) BDGD_CK(cudaFreeAsync(*bufs[i], c->stream));
    *bufs[i] = nullptr;
    *sizes[i] = 0;
  }
  c->version++;
  return BDGD_OK;
}

extern "C" int bdgd_set_graphs(bdgd_ctx *c, int on) {
  if (!c) return BDGD_ERR_ARG;
  c->graphs_on = on ? 1 : 0;
  if (!on) graphs_clear(c);
  return BDGD_OK;
}

extern "C" int bdgd_fft_tuning(bdgd_ctx *c, int op, int prec, int *path_out, float *ms_out) {
  if (!c || op < 0 || op >= 16) return BDGD_ERR_ARG;
  const int pi = prec == BDGD_F32 ? 1 : 0;
  if (path_out) *path_out = c->tune[op][pi];
  if (ms_out) {
    ms_out[0] = c->tune_ms[op][pi][0];
    ms_out[1] = c->tune_ms[op][pi][1];
  }
  return BDGD_OK;
}

// Run one apply through a cached graph: the first use of a key runs
// uncaptured (allocations, attributes), the second captures and launches
// the graph, later uses replay it.  Keys include the context version, which
// every setter and scratch reallocation bumps.
static int apply_graph(bdgd_ctx *c, int op, const Prog &p, int prec, const void *x, long long ldx, void *y,
                       long long ldy, int ncol) {
  bdgd_graph *g = nullptr;
  for (int i = 0; i < c->ngraphs; ++i) {
    bdgd_graph &e = c->graphs[i];
    if (e.op == op && e.prec == prec && e.ncol == ncol && e.x == x && e.y == y && e.ldx == ldx && e.ldy == ldy &&
        e.path == c->force_path && e.version == c->version) {
      g = &e;
      break;
    }
  }
  if (g && g->exec) {
    g->stamp = ++g_graph_clock;
    BDGD_CK(cudaGraphLaunch(g->exec, c->stream));
    count_launches(g->nkern);
    return BDGD_OK;
  }
  if (!g) {
    if (!c->graphs) c->graphs = (bdgd_graph *)calloc(BDGD_MAX_GRAPHS, sizeof(bdgd_graph));
    if (c->ngraphs < BDGD_MAX_GRAPHS) {
      g = &c->graphs[c->ngraphs++];
    } else {  // replace the least recently used entry
      g = &c->graphs[0];
      for (int i = 1; i < c->ngraphs; ++i)
        if (c->graphs[i].stamp < g->stamp) g = &c->graphs[i];
      if (g->exec) cudaGraphExecDestroy(g->exec);
    }
    memset(g, 0, sizeof *g);
    g->op = op;
    g->prec = prec;
    g->ncol = ncol;
    g->x = x;
    g->y = y;
    g->ldx = ldx;
    g->ldy = ldy;
    g->path = c->force_path;
    g->version = c->version;
    g->stamp = ++g_graph_clock;
    return dispatch(c, p, prec, x, ldx, y, ldy, ncol, 0, 0);
  }
  // second use: capture
  const unsigned long long l0 = bdgd_launch_count();
  cudaGraph_t gr = nullptr;
  BDGD_CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  bdgd_capturing = 1;
  int rc = dispatch(c, p, prec, x, ldx, y, ldy, ncol, 0, 0);
  bdgd_capturing = 0;
  cudaError_t e = cudaStreamEndCapture(c->stream, &gr);
  const unsigned long long nk = bdgd_launch_count() - l0;
  cudaGraphExec_t ex = nullptr;
  if (!rc && e == cudaSuccess && gr) e = cudaGraphInstantiate(&ex, gr, 0);
  if (gr) cudaGraphDestroy(gr);
  if (rc || e != cudaSuccess || !ex) {
    // not capturable here: run it directly (nothing of the capture ran)
    cudaGetLastError();
    __atomic_sub_fetch(&g_launches, nk, __ATOMIC_RELAXED);
    g->version = c->version - 1;  // never matches again
    return dispatch(c, p, prec, x, ldx, y, ldy, ncol, 0, 0);
  }
  g->exec = ex;
  g->nkern = nk;
  BDGD_CK(cudaGraphLaunch(ex, c->stream));  // the recorded launches are counted already
  return BDGD_OK;
}

// Choose the FFT pass family of (op, prec) on this context by timing both
// (each run twice, the second timed) on its first apply of >= 4 columns;
// later applies use the faster one.  BDG_FFT_PATH / BDG_GENERIC_FFT override.
static int apply_tuned(bdgd_ctx *c, int op, const Prog &p, int prec, const void *x, long long ldx, void *y,
                       long long ldy, int ncol) {
  const int pi = prec == BDGD_F32 ? 1 : 0;
  const bool env = getenv("BDG_FFT_PATH") || getenv("BDG_GENERIC_FFT");
  const bool tunable = !env && bdgd_lines_usable(c, p) && op < 16;
  if (tunable && c->tune[op][pi] == 0 && ncol >= 4 && !bdgd_capturing) {
    float ms[2] = {0.f, 0.f};
    cudaEvent_t e0, e1;
    BDGD_CK(cudaEventCreate(&e0));
    BDGD_CK(cudaEventCreate(&e1));
    int rc = BDGD_OK;
    for (int k = 0; k < 2 && !rc; ++k) {
      c->force_path = k + 1;
      rc = dispatch(c, p, prec, x, ldx, y, ldy, ncol, 0, 0);
      if (!rc) {
        cudaEventRecord(e0, c->stream);
        rc = dispatch(c, p, prec, x, ldx, y, ldy, ncol, 0, 0);
        cudaEventRecord(e1, c->stream);
        cudaError_t ce = cudaEventSynchronize(e1);
        if (ce != cudaSuccess) rc = bdgd_check(ce, "autotune");
        else cudaEventElapsedTime(&ms[k], e0, e1);
      }
    }
    c->force_path = 0;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    c->tune[op][pi] = ms[0] <= ms[1] ? 1 : 2;
    c->tune_ms[op][pi][0] = ms[0];
    c->tune_ms[op][pi][1] = ms[1];
    return BDGD_OK;  // y holds the result of the last run
  }
  if (tunable && c->tune[op][pi]) c->force_path = c->tune[op][pi];
  const int rc = (c->graphs_on && !bdgd_capturing) ? apply_graph(c, op, p, prec, x, ldx, y, ldy, ncol)
                                                   : dispatch(c, p, prec, x, ldx, y, ldy, ncol, 0, 0);
  c->force_path = 0;
  return rc;
}

extern "C" int bdgd_apply(bdgd_ctx *c, int op, int prec, const void *d_x, uint64_t ldx, void *d_y, uint64_t ldy,
                          uint64_t ncol) {
  if (!c || !d_x || !d_y) {
    bdgd_set_error("bdgd_apply: null argument");
    return BDGD_ERR_ARG;
  }
  if (ncol == 0) return BDGD_OK;
  if (op < 0 || op > BDGD_OP_DIPCONV) {
    bdgd_set_error("bdgd_apply: unknown operator %d", op);
    return BDGD_ERR_ARG;
  }
  const size_t esz = (prec == BDGD_F32 ? 4 : 8) * (c->cplx ? 2 : 1);
  if (op == BDGD_OP_SWAP) {
    const long long halfb = c->S * (long long)esz;
    const long long ldxb = (long long)ldx * esz, ldyb = (long long)ldy * esz;
    const uintptr_t al = (uintptr_t)d_x | (uintptr_t)d_y | (uintptr_t)halfb | (uintptr_t)ldxb | (uintptr_t)ldyb;
    const int wsz = (al % 16 == 0) ? 16 : (al % 8 == 0) ? 8 : 4;
    long long blocks = (halfb / wsz + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    if (blocks < 1) blocks = 1;
    dim3 grid((unsigned)blocks, (unsigned)ncol);
    const unsigned char *xb = (const unsigned char *)d_x;
    unsigned char *yb = (unsigned char *)d_y;
    if (wsz == 16) { bdgd_count_launch(); k_swap<uint4><<<grid, 256, 0, c->stream>>>(xb, ldxb, yb, ldyb, halfb); }
    else if (wsz == 8) { bdgd_count_launch(); k_swap<unsigned long long><<<grid, 256, 0, c->stream>>>(xb, ldxb, yb, ldyb, halfb); }
    else { bdgd_count_launch(); k_swap<unsigned int><<<grid, 256, 0, c->stream>>>(xb, ldxb, yb, ldyb, halfb); }
    BDGD_CK(cudaGetLastError());
    return BDGD_OK;
  }
  int rc = check_ready(c, op);
  if (rc) return rc;
  if (op == BDGD_OP_DIPCONV && c->dim != 3) {
    bdgd_set_error("dipolar convolution requires dim == 3");
    return BDGD_ERR_ARG;
  }
  Prog p = make_prog(op, c->dipolar && c->dim == 3);
  return apply_tuned(c, op, p, prec, d_x, (long long)ldx, d_y, (long long)ldy, (int)ncol);
}

extern "C" int bdgd_apply_host(bdgd_ctx *c, int op, const void *x, void *y, uint64_t ncol) {
  const int two = (op == BDGD_OP_LREP || op == BDGD_OP_TLREP || op == BDGD_OP_SWAP) ? 2 : 1;
  const size_t esz = c->cplx ? 16 : 8;
  const size_t colb = (size_t)c->S * two * esz;
  int rc = bdgd_ensure(c->stream, &c->io, &c->io_bytes, 2 * colb * ncol);
  if (rc) return rc;
  char *dx = (char *)c->io;
  char *dy = dx + colb * ncol;
  BDGD_CK(cudaMemcpyAsync(dx, x, colb * ncol, cudaMemcpyHostToDevice, c->stream));
  rc = bdgd_apply(c, op, BDGD_F64, dx, (uint64_t)c->S * two, dy, (uint64_t)c->S * two, ncol);
  if (rc) return rc;
  BDGD_CK(cudaMemcpyAsync(y, dy, colb * ncol, cudaMemcpyDeviceToHost, c->stream));
  BDGD_CK(cudaStreamSynchronize(c->stream));
  return BDGD_OK;
}

extern "C" int bdgd_dipolar_meanfield(bdgd_ctx *c, double *phi_out) {
  if (!c->wf64 || !c->vdd) {
    bdgd_set_error("dipolar mean field needs wavefunction and kernel");
    return BDGD_ERR_STATE;
  }
  Prog p = make_prog(100, 0);
  const size_t esz = c->cplx ? 16 : 8;
  int rc = bdgd_ensure(c->stream, &c->io, &c->io_bytes, 2 * esz * c->S);
  if (rc) return rc;
  char *dx = (char *)c->io;
  char *dy = dx + esz * c->S;
  BDGD_CK(cudaMemsetAsync(dx, 0, esz * c->S, c->stream));
  rc = dispatch(c, p, BDGD_F64, dx, c->S, dy, c->S, 1, 0, 0);
  if (rc) return rc;
  if (c->cplx) {
    BDGD_CK(cudaMemcpy2DAsync(phi_out, sizeof(double), dy, 2 * sizeof(double), sizeof(double), c->S,
                              cudaMemcpyDeviceToHost, c->stream));
  } else {
    BDGD_CK(cudaMemcpyAsync(phi_out, dy, sizeof(double) * c->S, cudaMemcpyDeviceToHost, c->stream));
  }
  BDGD_CK(cudaStreamSynchronize(c->stream));
  return BDGD_OK;
}

extern "C" int bdgd_fft_host(bdgd_ctx *c, int forward, const void *in, void *out, uint64_t ncol) {
  Prog p = make_prog(BDGD_OP_KINETIC, 0);
  p.post[0] = POST_RAW;
  p.mul[0][0] = MUL_ONE;
  const size_t esz = c->cplx ? 16 : 8;
  const size_t rb = esz * (size_t)c->S * ncol;
  const size_t kb = 16 * (size_t)c->H * ncol;
  int rc = bdgd_ensure(c->stream, &c->io, &c->io_bytes, rb);
  if (rc) return rc;
  rc = bdgd_ensure(c->stream, &c->spec, &c->spec_bytes, kb);
  if (rc) return rc;
  if (forward) {
    BDGD_CK(cudaMemcpyAsync(c->io, in, rb, cudaMemcpyHostToDevice, c->stream));
    rc = dispatch(c, p, BDGD_F64, c->io, c->S, c->io, c->S, (int)ncol, 1, 0);
    if (rc) return rc;
    if (c->dim == 1) {
      // 1D: the row pass wrote the spectrum already
    }
    BDGD_CK(cudaMemcpyAsync(out, c->spec, kb, cudaMemcpyDeviceToHost, c->stream));
  } else {
    BDGD_CK(cudaMemcpyAsync(c->spec, in, kb, cudaMemcpyHostToDevice, c->stream));
    rc = dispatch(c, p, BDGD_F64, c->io, c->S, c->io, c->S, (int)ncol, 0, 1);
    if (rc) return rc;
    BDGD_CK(cudaMemcpyAsync(out, c->io, rb, cudaMemcpyDeviceToHost, c->stream));
  }
  BDGD_CK(cudaStreamSynchronize(c->stream));
  return BDGD_OK;
}

// Internal programs of the ground-state producer (bdg_gs.cu): 101
// imaginary-time kinetic propagator exp(-kin_dt k^2), 102 dipolar mean field
// of the input field.  FP64, device pointers.
int bdgd_run_internal(bdgd_ctx *c, int kind, const void *d_x, long long ldx, void *d_y, long long ldy, int ncol) {
  Prog p = make_prog(kind, 0);
  return dispatch(c, p, BDGD_F64, d_x, ldx, d_y, ldy, ncol, 0, 0);
}
