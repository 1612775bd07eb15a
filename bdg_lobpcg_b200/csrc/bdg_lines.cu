// bdg_lines.cu -- FFT pass kernels whose line transforms live in registers.
//
// Same five passes as the shared-memory kernels in bdg_ops.cu (x forward
// with the prologue, y, last axis fused with the k-space multiply, y
// inverse, x inverse with the epilogue), but each line of length
// N = N1 * N2 is transformed by N2 threads in two register phases:
//
//   phase 1  thread t holds x[N2*n1 + t], n1 < N1, loaded straight from
//            global memory; DFT of size N1 in registers, twiddle w_N^(t*k1)
//   exchange one write and one read through shared memory
//   phase 2  thread t takes k1 = t + N2*j (j < N1/N2) and runs the DFTs of
//            size N2 over n2; it ends holding X[k1 + N1*k2]
//
// so a pass costs one shared-memory round trip instead of one per radix
// stage, and all loads of a tile are in flight at once.  The last-axis pass
// multiplies in that phase-2 order and runs the inverse as the transposed
// decomposition, which returns the data to the phase-1 positions.
//
// Real fields are transformed two at a time as one complex line
// z = a + i b (two x rows, or the two prologue fields of the M half), and
// split with A[k] = (Z[k] + conj Z[N-k]) / 2, B[k] = (Z[k] - conj Z[N-k]) / 2i.
// The inverse packs Z = A + i B with the Hermitian extension of each half
// spectrum, so one complex inverse returns a = Re z and b = Im z.  The half
// spectrum layout (x extent N/2+1, x fastest) is that of the other kernels
// and of FFTW's r2c (src/fft_helpers_impl.inc:24-82 of the reference).
//
// Grids run the spectra (or columns) along grid.x and the line blocks along
// grid.y, so the blocks of all columns that share a tile of coefficient or
// multiplier entries are resident together and those entries come from L2.
#include <type_traits>

#include "bdg_lines.h"

// ---------------------------------------------------------------------------
// compile-time trigonometry for the in-register DFT twiddles
// ---------------------------------------------------------------------------
// Taylor series on [0, pi/2) after an exact reduction of the angle 2*pi*j/n
// to a quadrant; absolute error a few units of the last place.
__host__ __device__ constexpr double cx_sin_poly(double x) {
  double t = x, s = x;
  for (int i = 1; i < 16; ++i) {
    t *= -x * x / ((2.0 * i) * (2.0 * i + 1.0));
    s += t;
  }
  return s;
}
__host__ __device__ constexpr double cx_cos_poly(double x) {
  double t = 1.0, s = 1.0;
  for (int i = 1; i < 16; ++i) {
    t *= -x * x / ((2.0 * i - 1.0) * (2.0 * i));
    s += t;
  }
  return s;
}
__host__ __device__ constexpr int cx_quadrant(int j, int n) { return (4 * j) / n; }
__host__ __device__ constexpr double cx_rem(int j, int n) {
  return 6.283185307179586476925 * (double)(4 * j - cx_quadrant(j, n) * n) / (4.0 * (double)n);
}
// cos(2 pi j / n), sin(2 pi j / n) for 0 <= j < n
__host__ __device__ constexpr double cx_cos(int j, int n) {
  const int q = cx_quadrant(j, n);
  const double r = cx_rem(j, n);
  return q == 0 ? cx_cos_poly(r) : q == 1 ? -cx_sin_poly(r) : q == 2 ? -cx_cos_poly(r) : cx_sin_poly(r);
}
__host__ __device__ constexpr double cx_sin(int j, int n) {
  const int q = cx_quadrant(j, n);
  const double r = cx_rem(j, n);
  return q == 0 ? cx_sin_poly(r) : q == 1 ? cx_cos_poly(r) : q == 2 ? -cx_sin_poly(r) : -cx_cos_poly(r);
}

#define CV(I) decltype(I)::value

template <int B, int E, typename F>
__device__ __forceinline__ void sfor(F &&f) {
  if constexpr (B < E) {
    f(std::integral_constant<int, B>{});
    sfor<B + 1, E>(f);
  }
}

// a * w_R^M with w_R = exp(SGN * 2 pi i / R), M a compile-time constant
template <int M, int R, int SGN, typename C>
__device__ __forceinline__ C ctw(C a) {
  constexpr int m = ((M % R) + R) % R;
  if constexpr (m == 0) {
    return a;
  } else if constexpr (2 * m == R) {
    a.x = -a.x;
    a.y = -a.y;
    return a;
  } else if constexpr (4 * m == R) {
    return cmul_si(a, SGN);
  } else if constexpr (4 * m == 3 * R) {
    return cmul_si(a, -SGN);
  } else {
    typedef decltype(a.x) E;
    constexpr double c = cx_cos(m, R), s = SGN * cx_sin(m, R);
    C r;
    r.x = a.x * (E)c - a.y * (E)s;
    r.y = a.x * (E)s + a.y * (E)c;
    return r;
  }
}

template <int R>
__host__ __device__ constexpr int rdft_split() {
  return (R % 16 == 0) ? 4 : (R % 8 == 0) ? 8 : (R % 4 == 0) ? 4 : (R % 2 == 0) ? 2 : 3;
}

// In-register DFT of size R (natural order in and out), sign SGN.
template <int R, int SGN, typename C>
__device__ __forceinline__ void rdft(C *v) {
  if constexpr (R == 1) {
  } else if constexpr (R == 2) {
    bfly2(v);
  } else if constexpr (R == 3) {
    bfly3(v, SGN);
  } else if constexpr (R == 4) {
    bfly4(v[0], v[1], v[2], v[3], SGN);
  } else if constexpr (R == 8) {
    bfly8(v, SGN);
  } else {
    constexpr int R1 = rdft_split<R>(), R2 = R / R1;
    // n = R2*n1 + n2, k = k1 + R1*k2
    sfor<0, R2>([&](auto I2) {
      constexpr int n2 = CV(I2);
      C u[R1];
      sfor<0, R1>([&](auto I1) { u[CV(I1)] = v[R2 * CV(I1) + n2]; });
      rdft<R1, SGN>(u);
      sfor<0, R1>([&](auto K1) { v[R2 * CV(K1) + n2] = ctw<n2 * CV(K1), R, SGN>(u[CV(K1)]); });
    });
    C w[R];
    sfor<0, R1>([&](auto K1) {
      constexpr int k1 = CV(K1);
      C u[R2];
      sfor<0, R2>([&](auto I2) { u[CV(I2)] = v[R2 * k1 + CV(I2)]; });
      rdft<R2, SGN>(u);
      sfor<0, R2>([&](auto K2) { w[k1 + R1 * CV(K2)] = u[CV(K2)]; });
    });
    sfor<0, R>([&](auto I) { v[CV(I)] = w[CV(I)]; });
  }
}

// ---------------------------------------------------------------------------
// line plans: N = N1 * N2, N2 threads per line, N1 / N2 phase-2 DFTs each
// ---------------------------------------------------------------------------
template <int N>
struct LPlan {
  static constexpr int N1 = N == 16 ? 4 : N == 32 ? 8 : N == 48 ? 12 : N == 64 ? 8 : N == 96 ? 24
                          : N == 128 ? 16 : N == 256 ? 16 : 0;
  static constexpr int N2 = N1 ? N / N1 : 1;
  static constexpr int Q = N1 / N2;
  static constexpr int LS = N1 * (N2 + 1) + 1;  // exchange stride per line (odd, >= N)
  static constexpr int TX = 128 / N2;           // lines per 128-thread block
  static_assert(N1 == 0 || (N1 % N2 == 0 && LS >= N), "line plan");
};

bool bdgd_lines_size_ok(int n) {
  return n == 16 || n == 32 || n == 48 || n == 64 || n == 96 || n == 128 || n == 256;
}

// Forward (SGN = -1) or inverse (SGN = +1) transform of one line.
// In:  v[n1] = x[N2*n1 + t].  Out: v[j*N2 + k2] = X[k1 + N1*k2], k1 = t + N2*j.
// buf: this line's exchange area (LS elements).  Every thread of the block
// must call it (it synchronises).
template <typename C, int N, int SGN>
__device__ __forceinline__ void line_dft(C *v, C *buf, int t, const C *roots) {
  typedef LPlan<N> P;
  rdft<P::N1, SGN>(v);
#pragma unroll
  for (int k1 = 1; k1 < P::N1; ++k1) v[k1] = cmul(v[k1], rootv(roots, t * k1, SGN));
#pragma unroll
  for (int k1 = 0; k1 < P::N1; ++k1) buf[k1 * (P::N2 + 1) + t] = v[k1];
  __syncthreads();
#pragma unroll
  for (int j = 0; j < P::Q; ++j) {
    C u[P::N2];
    const int k1 = t + P::N2 * j;
#pragma unroll
    for (int n2 = 0; n2 < P::N2; ++n2) u[n2] = buf[k1 * (P::N2 + 1) + n2];
    rdft<P::N2, SGN>(u);
#pragma unroll
    for (int k2 = 0; k2 < P::N2; ++k2) v[j * P::N2 + k2] = u[k2];
  }
}

// Transform back from the phase-2 order (the transposed decomposition).
// In:  v[j*N2 + k2] = X[k1 + N1*k2].  Out: v[n1] = x[N2*n1 + t].
template <typename C, int N, int SGN>
__device__ __forceinline__ void line_dit(C *v, C *buf, int t, const C *roots) {
  typedef LPlan<N> P;
#pragma unroll
  for (int j = 0; j < P::Q; ++j) {
    C u[P::N2];
#pragma unroll
    for (int k2 = 0; k2 < P::N2; ++k2) u[k2] = v[j * P::N2 + k2];
    rdft<P::N2, SGN>(u);
    const int k1 = t + P::N2 * j;
#pragma unroll
    for (int n2 = 0; n2 < P::N2; ++n2)
      buf[k1 * (P::N2 + 1) + n2] = n2 ? cmul(u[n2], rootv(roots, n2 * k1, SGN)) : u[n2];
  }
  __syncthreads();
#pragma unroll
  for (int k1 = 0; k1 < P::N1; ++k1) v[k1] = buf[k1 * (P::N2 + 1) + t];
  rdft<P::N1, SGN>(v);
}

template <typename C>
__device__ __forceinline__ C czero() {
  C z;
  z.x = 0;
  z.y = 0;
  return z;
}


// ---------------------------------------------------------------------------
// prologue / epilogue with the coefficient loads hoisted: the operator kind
// is uniform over a launch, so the array it reads is chosen once and every
// load of a row chunk is issued before the arithmetic (a per-element switch
// with the load inside would expose one memory latency per element).  The
// arithmetic is that of prologue() and epilogue() in bdg_kern.cuh.
// ---------------------------------------------------------------------------
// real-valued coefficient array of a prologue kind (pK, pM; the wavefunction
// for the real path), or null
__device__ __forceinline__ const void *pre_coef(const FieldsDev &f, int kind) {
  switch (kind) {
    case PRE_PK: return f.pK;
    case PRE_PM: return f.pM;
    case PRE_CONJWF:
    case PRE_DENS: return f.w;
    default: return nullptr;
  }
}
template <typename T>
__device__ __forceinline__ T pre_real(int kind, T x, T c) {
  switch (kind) {
    case PRE_PK:
    case PRE_PM:
    case PRE_CONJWF: return c * x;
    case PRE_DENS: {
      const T a = fabs(c);
      return a * a;
    }
    case PRE_XDENS: return x * x;
    default: return x;
  }
}
// complex path: c is the real coefficient (pK, pM), w the wavefunction value
template <typename T, typename C>
__device__ __forceinline__ C pre_cplx(int kind, C x, T c, C w) {
  switch (kind) {
    case PRE_PK:
    case PRE_PM: return cscale(x, c);
    case PRE_CONJWF: return cmul(cconj(w), x);
    case PRE_DENS: {
      const T a = hypot(w.x, w.y);
      return cmk<C>(a * a, 0.0);
    }
    case PRE_XDENS: return cmk<C>(x.x * x.x + x.y * x.y, 0.0);
    default: return x;
  }
}
// real-valued coefficient array of an epilogue kind (ltK, ltM, pK, pM), or null
__device__ __forceinline__ const void *post_coef(const FieldsDev &f, int post) {
  switch (post) {
    case POST_K: return f.ltK;
    case POST_M: return f.ltM;
    case POST_TK: return f.pK;
    case POST_TM: return f.pM;
    default: return nullptr;
  }
}
template <typename T>
__device__ __forceinline__ T epi_real(int post, int nf, T y0, T y1, T x, T c, T w, T g) {
  switch (post) {
    case POST_K: return y0 + c * x;
    case POST_M:
      if (nf > 1) {
        const T dc = (g * w) * y1;
        return y0 + (c * x + (T)2 * dc);
      }
      return y0 + c * x;
    case POST_TK:
    case POST_TM: return y0 * c;
    case POST_DIPCONV: return (g * w) * y0;
    case POST_PHI: return g * y0;
    default: return y0;
  }
}
template <typename T, typename C>
__device__ __forceinline__ C epi_cplx(int post, int nf, C o0, C o1, C x, T c, C w, T g) {
  switch (post) {
    case POST_K: return cadd(o0, cscale(x, c));
    case POST_M:
      if (nf > 1) {
        const C dc = cmul(cscale(w, g), o1);
        return cadd(o0, cadd(cscale(x, c), cscale(dc, (T)2)));
      }
      return cadd(o0, cscale(x, c));
    case POST_TK:
    case POST_TM: return cscale(o0, c);
    case POST_DIPCONV: return cmul(cscale(w, g), o0);
    case POST_PHI: return cmk<C>(g * o0.x, 0.0);
    default: return o0;
  }
}
// elements per load batch of the epilogue (bounds the registers in flight)
constexpr int kEpiBatch = 8;

// ---------------------------------------------------------------------------
// pencil pass along axis 1 or 2 (MODE 0 forward, 1 inverse, 2 forward *
// k-space multiplier * inverse).  Lines are the spectrum lines along the
// axis, numbered L = outer * inner + in, element e at
// outer*inner*N + in + e*inner; consecutive L are consecutive addresses
// within an x row, and the block's lanes run over L first (coalesced).
// grid.x: spectra (column * J + job), grid.y: line blocks.
// ---------------------------------------------------------------------------
template <typename T, int N, int MODE>
__global__ void __launch_bounds__(128, 3) k_cols_reg(GeoDev g, Prog p, FieldsDev f,
                                                     typename Cx<T>::t *__restrict__ spec, int axis,
                                                     long long nlines, long long inner) {
  typedef typename Cx<T>::t C;
  typedef LPlan<N> P;
  extern __shared__ __align__(16) unsigned char smraw[];
  C *buf = (C *)smraw;
  const int l = threadIdx.x % P::TX, t = threadIdx.x / P::TX;
  const long long L = (long long)blockIdx.y * P::TX + l;
  const bool on = L < nlines;
  const long long Lc = on ? L : 0;
  const long long outer = Lc / inner, in = Lc - outer * inner;
  const long long off = outer * inner * N + in;
  C *base = spec + (long long)blockIdx.x * g.H + off;
  C v[P::N1];
#pragma unroll
  for (int n1 = 0; n1 < P::N1; ++n1) v[n1] = on ? base[(long long)(P::N2 * n1 + t) * inner] : czero<C>();
  C *lb = buf + l * P::LS;
  const C *roots = roots_of<C>(g.ax[axis]);
  if constexpr (MODE == 1)
    line_dft<C, N, +1>(v, lb, t, roots);
  else
    line_dft<C, N, -1>(v, lb, t, roots);
  if constexpr (MODE == 2) {
    const int job = blockIdx.x;
    const int col = job / p.J;
    const int jj = job - col * p.J;
    const int kind = p.mul[p.jh[jj]][p.jf[jj]];
    // the multiplied axis is the last one: (ix, iy) from `in`, the axis index from k
    int ix, iy;
    if (g.dim == 3) {
      iy = (int)(in / g.nxk);
      ix = (int)(in - (long long)iy * g.nxk);
    } else {
      iy = 0;
      ix = (int)in;
    }
    if (kind == MUL_DIP || (kind == MUL_PRE && f.ptab)) {
      // tabulated multiplier (dipolar kernel or preconditioner factor)
      const double *tab = (kind == MUL_DIP) ? f.vdd : f.ptab;
      const double sc = (kind == MUL_DIP) ? f.inv_size : 1.0;
#pragma unroll
      for (int j = 0; j < P::Q; ++j)
#pragma unroll
        for (int k2 = 0; k2 < P::N2; ++k2) {
          const int k = t + P::N2 * j + P::N1 * k2;
          const double m = __ldg(tab + off + (long long)k * inner) * sc;
          v[j * P::N2 + k2] = cscale(v[j * P::N2 + k2], (T)m);
        }
    } else {
      // k^2 = kx2[0][ix] + kx2[1][iy] + kx2[2][iz] summed in that order; the
      // line-constant part is added once
      const double *kl = g.kx2[g.dim - 1];
      const double kxy = (g.dim == 3) ? __ldg(g.kx2[0] + ix) + __ldg(g.kx2[1] + iy) : __ldg(g.kx2[0] + ix);
#pragma unroll
      for (int j = 0; j < P::Q; ++j)
#pragma unroll
        for (int k2 = 0; k2 < P::N2; ++k2) {
          const int k = t + P::N2 * j + P::N1 * k2;
          const double m = kmult_k2(f, kind, kxy + __ldg(kl + k));
          v[j * P::N2 + k2] = cscale(v[j * P::N2 + k2], (T)m);
        }
    }
    __syncthreads();
    line_dit<C, N, +1>(v, lb, t, roots);
    if (on) {
#pragma unroll
      for (int n1 = 0; n1 < P::N1; ++n1) base[(long long)(P::N2 * n1 + t) * inner] = v[n1];
    }
  } else {
    if (on) {
#pragma unroll
      for (int j = 0; j < P::Q; ++j)
#pragma unroll
        for (int k2 = 0; k2 < P::N2; ++k2)
          base[(long long)(t + P::N2 * j + P::N1 * k2) * inner] = v[j * P::N2 + k2];
    }
  }
}

// ---------------------------------------------------------------------------
// x rows, forward, with the prologue.  Half h of every column; lanes run
// over the N2 threads of a line first (row elements, coalesced).
//   real, NF = 1: line L = rows 2L and 2L+1 of the half
//   real, NF = 2: line L = row L, fields 0 and 1
//   complex:      line L = row L / NF, field L % NF
// grid.x: columns, grid.y: line blocks.
// ---------------------------------------------------------------------------
template <typename T, bool CPLX, int N, int NF>
__global__ void __launch_bounds__(128, 3) k_rows_fwd_reg(GeoDev g, Prog p, FieldsDev f,
                                                         const void *__restrict__ xin, long long ldx,
                                                         typename Cx<T>::t *__restrict__ spec, int h,
                                                         long long nlines) {
  typedef typename El<T, CPLX>::C C;
  typedef typename El<T, CPLX>::V V;
  typedef LPlan<N> P;
  extern __shared__ __align__(16) unsigned char smraw[];
  C *buf = (C *)smraw;
  const int t = threadIdx.x % P::N2, l = threadIdx.x / P::N2;
  const long long L = (long long)blockIdx.y * P::TX + l;
  const bool on = L < nlines;
  const long long Lc = on ? L : 0;
  const int col = blockIdx.x;
  const V *src = (const V *)xin + (long long)col * ldx + (long long)h * g.S;
  const C *roots = roots_of<C>(g.ax[0]);
  C *lb = buf + l * P::LS;
  C v[P::N1];
  if constexpr (!CPLX) {
    const long long ra = (NF == 1 ? 2 * Lc : Lc) * N;
    const long long rb = (NF == 1) ? ra + N : ra;
    const int ka = p.pre[h][0], kb = p.pre[h][NF == 1 ? 0 : 1];
    const T *ca = (const T *)pre_coef(f, ka), *cb = (const T *)pre_coef(f, kb);
    T xa[P::N1], xb[P::N1], wa[P::N1], wb[P::N1];
#pragma unroll
    for (int n1 = 0; n1 < P::N1; ++n1) {
      xa[n1] = xb[n1] = wa[n1] = wb[n1] = (T)0;
    }
    if (on) {
#pragma unroll
      for (int n1 = 0; n1 < P::N1; ++n1) xa[n1] = src[ra + P::N2 * n1 + t];
      if (NF == 1) {
#pragma unroll
        for (int n1 = 0; n1 < P::N1; ++n1) xb[n1] = src[rb + P::N2 * n1 + t];
      }
      if (ca) {
#pragma unroll
        for (int n1 = 0; n1 < P::N1; ++n1) wa[n1] = __ldg(ca + ra + P::N2 * n1 + t);
      }
      if (cb) {
#pragma unroll
        for (int n1 = 0; n1 < P::N1; ++n1) wb[n1] = __ldg(cb + rb + P::N2 * n1 + t);
      }
    }
#pragma unroll
    for (int n1 = 0; n1 < P::N1; ++n1) {
      v[n1].x = pre_real<T>(ka, xa[n1], wa[n1]);
      v[n1].y = pre_real<T>(kb, (NF == 1) ? xb[n1] : xa[n1], wb[n1]);
    }
    line_dft<C, N, -1>(v, lb, t, roots);
    __syncthreads();  // phase-2 reads done before the line area is reused
#pragma unroll
    for (int j = 0; j < P::Q; ++j)
#pragma unroll
      for (int k2 = 0; k2 < P::N2; ++k2) lb[t + P::N2 * j + P::N1 * k2] = v[j * P::N2 + k2];
    __syncthreads();
    if (on) {
      const int nxk = g.nxk;
      C *sa, *sb;
      C *s0 = spec + ((long long)col * p.J + p.j0[h]) * g.H;
      if (NF == 1) {
        sa = s0 + 2 * Lc * nxk;
        sb = sa + nxk;
      } else {
        sa = s0 + Lc * nxk;
        sb = sa + g.H;
      }
      for (int k = t; k <= N / 2; k += P::N2) {
        const C zk = lb[k], zm = lb[k ? N - k : 0];
        C a, b;
        a.x = (T)0.5 * (zk.x + zm.x);
        a.y = (T)0.5 * (zk.y - zm.y);
        b.x = (T)0.5 * (zk.y + zm.y);
        b.y = (T)0.5 * (zm.x - zk.x);
        sa[k] = a;
        sb[k] = b;
      }
    }
  } else {
    const long long row = Lc / NF;
    const int fi = (int)(Lc - row * NF);
    const int kind = p.pre[h][fi];
    const long long r0 = row * N;
    const T *cr = (kind == PRE_PK || kind == PRE_PM) ? (const T *)pre_coef(f, kind) : nullptr;
    const C *cw = (kind == PRE_CONJWF || kind == PRE_DENS) ? (const C *)f.w : nullptr;
    C xv[P::N1], wv[P::N1];
    T rv[P::N1];
#pragma unroll
    for (int n1 = 0; n1 < P::N1; ++n1) {
      xv[n1] = wv[n1] = czero<C>();
      rv[n1] = (T)0;
    }
    if (on) {
#pragma unroll
      for (int n1 = 0; n1 < P::N1; ++n1) xv[n1] = src[r0 + P::N2 * n1 + t];
      if (cr) {
#pragma unroll
        for (int n1 = 0; n1 < P::N1; ++n1) rv[n1] = __ldg(cr + r0 + P::N2 * n1 + t);
      }
      if (cw) {
#pragma unroll
        for (int n1 = 0; n1 < P::N1; ++n1) wv[n1] = cw[r0 + P::N2 * n1 + t];
      }
    }
#pragma unroll
    for (int n1 = 0; n1 < P::N1; ++n1) v[n1] = on ? pre_cplx<T, C>(kind, xv[n1], rv[n1], wv[n1]) : czero<C>();
    line_dft<C, N, -1>(v, lb, t, roots);
    if (on) {
      C *s = spec + ((long long)col * p.J + p.j0[h] + fi) * g.H + row * N;
#pragma unroll
      for (int j = 0; j < P::Q; ++j)
#pragma unroll
        for (int k2 = 0; k2 < P::N2; ++k2) s[t + P::N2 * j + P::N1 * k2] = v[j * P::N2 + k2];
    }
  }
}

// ---------------------------------------------------------------------------
// x rows, inverse, with the epilogue.  Line numbering as k_rows_fwd_reg,
// except that complex lines are whole rows (both fields in one thread).
// ---------------------------------------------------------------------------
template <typename T, bool CPLX, int N, int NF>
__global__ void __launch_bounds__(128, 3) k_rows_inv_reg(GeoDev g, Prog p, FieldsDev f,
                                                         const typename Cx<T>::t *__restrict__ spec,
                                                         const void *__restrict__ xin, long long ldx,
                                                         void *__restrict__ yout, long long ldy, int h,
                                                         long long nlines) {
  typedef typename El<T, CPLX>::C C;
  typedef typename El<T, CPLX>::V V;
  typedef LPlan<N> P;
  extern __shared__ __align__(16) unsigned char smraw[];
  C *buf = (C *)smraw;
  const int t = threadIdx.x % P::N2, l = threadIdx.x / P::N2;
  const long long L = (long long)blockIdx.y * P::TX + l;
  const bool on = L < nlines;
  const long long Lc = on ? L : 0;
  const int col = blockIdx.x;
  const C *roots = roots_of<C>(g.ax[0]);
  C *lb = buf + l * P::LS;
  const V *xs = (const V *)xin + (long long)col * ldx + (long long)h * g.S;
  V *ys = (V *)yout + (long long)col * ldy + (long long)h * g.S;
  const int post = p.post[h];
  const bool needx = (post == POST_K || post == POST_M);
  const C *s0 = spec + ((long long)col * p.J + p.j0[h]) * g.H;
  C v[P::N1];
  if constexpr (!CPLX) {
    const int nxk = g.nxk;
    const C *sa, *sb;
    if (NF == 1) {
      sa = s0 + 2 * Lc * nxk;
      sb = sa + nxk;
    } else {
      sa = s0 + Lc * nxk;
      sb = sa + g.H;
    }
#pragma unroll
    for (int n1 = 0; n1 < P::N1; ++n1) {
      const int k = P::N2 * n1 + t;
      C z = czero<C>();
      if (on) {
        if (k <= N / 2) {
          C a = sa[k], b = sb[k];
          if (k == 0 || 2 * k == N) {
            // a real row's DC and Nyquist terms are real: drop the imaginary
            // parts (as a c2r transform does) rather than leak them into
            // the partner field
            a.y = 0;
            b.y = 0;
          }
          z.x = a.x - b.y;
          z.y = a.y + b.x;
        } else {
          const C a = sa[N - k], b = sb[N - k];
          z.x = a.x + b.y;
          z.y = b.x - a.y;
        }
      }
      v[n1] = z;
    }
    line_dft<C, N, +1>(v, lb, t, roots);
    if (on) {
      const long long ra = (NF == 1 ? 2 * Lc : Lc) * N;
      const T *cl = (const T *)post_coef(f, post);
      const bool needw = (post == POST_M && NF > 1) || post == POST_DIPCONV;
      const T *wr = (const T *)f.w;
      const T gg = (T)f.g_ddi;
      // NF = 1: rows ra (real parts) and ra + N (imaginary parts); NF = 2: row ra
#pragma unroll
      for (int rr = 0; rr < (NF == 1 ? 2 : 1); ++rr) {
        const long long ro = ra + rr * N;
#pragma unroll
        for (int e0 = 0; e0 < P::N1; e0 += kEpiBatch) {
          T xv[kEpiBatch], cv[kEpiBatch], wv[kEpiBatch];
#pragma unroll
          for (int b = 0; b < kEpiBatch; ++b) {
            const int e = e0 + b;
            const int n = t + P::N2 * (e / P::N2) + P::N1 * (e % P::N2);
            xv[b] = (needx && e < P::N1) ? xs[ro + n] : (T)0;
            cv[b] = (cl && e < P::N1) ? __ldg(cl + ro + n) : (T)0;
            wv[b] = (needw && e < P::N1) ? wr[ro + n] : (T)0;
          }
#pragma unroll
          for (int b = 0; b < kEpiBatch; ++b) {
            const int e = e0 + b;
            if (e < P::N1) {
              const int n = t + P::N2 * (e / P::N2) + P::N1 * (e % P::N2);
              const T y0 = rr ? v[e].y : v[e].x;
              ys[ro + n] = epi_real<T>(post, NF, y0, v[e].y, xv[b], cv[b], wv[b], gg);
            }
          }
        }
      }
    }
  } else {
    const long long r0 = Lc * N;
    const C *sr = s0 + Lc * N;
#pragma unroll
    for (int n1 = 0; n1 < P::N1; ++n1) v[n1] = on ? sr[P::N2 * n1 + t] : czero<C>();
    line_dft<C, N, +1>(v, lb, t, roots);
    C w[(NF > 1) ? P::N1 : 1];
    if constexpr (NF > 1) {
      __syncthreads();
      const C *sr1 = sr + g.H;
#pragma unroll
      for (int n1 = 0; n1 < P::N1; ++n1) w[n1] = on ? sr1[P::N2 * n1 + t] : czero<C>();
      line_dft<C, N, +1>(w, lb, t, roots);
    }
    if (on) {
      const T *cl = (const T *)post_coef(f, post);
      const bool needw = (post == POST_M && NF > 1) || post == POST_DIPCONV;
      const C *wc = (const C *)f.w;
      const T gg = (T)f.g_ddi;
#pragma unroll
      for (int e0 = 0; e0 < P::N1; e0 += kEpiBatch) {
        C xv[kEpiBatch], wv[kEpiBatch];
        T cv[kEpiBatch];
#pragma unroll
        for (int b = 0; b < kEpiBatch; ++b) {
          const int e = e0 + b;
          const int n = t + P::N2 * (e / P::N2) + P::N1 * (e % P::N2);
          xv[b] = (needx && e < P::N1) ? xs[r0 + n] : czero<C>();
          cv[b] = (cl && e < P::N1) ? __ldg(cl + r0 + n) : (T)0;
          wv[b] = (needw && e < P::N1) ? wc[r0 + n] : czero<C>();
        }
#pragma unroll
        for (int b = 0; b < kEpiBatch; ++b) {
          const int e = e0 + b;
          if (e < P::N1) {
            const int n = t + P::N2 * (e / P::N2) + P::N1 * (e % P::N2);
            const C o0 = v[e];
            const C o1 = (NF > 1) ? w[(NF > 1) ? e : 0] : o0;
            ys[r0 + n] = epi_cplx<T, C>(post, NF, o0, o1, xv[b], cv[b], wv[b], gg);
          }
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
template <typename C, int N>
static size_t lines_smem() {
  return sizeof(C) * (size_t)LPlan<N>::TX * LPlan<N>::LS;
}

// Opt in to more than 48 KB of dynamic shared memory (per device, so on
// every launch that needs it).
template <typename K>
static int set_smem(K kern, size_t sm) {
  if (sm > 48 * 1024) { const int _ra = bdgd_smem_attr(kern, sm); if (_ra) return _ra; }
  return BDGD_OK;
}

template <typename T, int N, int MODE>
static int launch_cols(bdgd_ctx *c, const Prog &p, const FieldsDev &fd, typename Cx<T>::t *spec, int njobs,
                       int axis) {
  typedef typename Cx<T>::t C;
  const size_t sm = lines_smem<C, N>();
  int rc = set_smem(k_cols_reg<T, N, MODE>, sm);
  if (rc) return rc;
  long long inner = c->nxk;
  for (int d = 1; d < axis; ++d) inner *= c->N[d];
  const long long nlines = c->H / c->N[axis];
  const long long nb = (nlines + LPlan<N>::TX - 1) / LPlan<N>::TX;
  bdgd_count_launch();
  k_cols_reg<T, N, MODE><<<dim3(njobs, (unsigned)nb), 128, sm, c->stream>>>(c->geo, p, fd, spec, axis, nlines,
                                                                           inner);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}

static long long row_lines(const bdgd_ctx *c, int cplx, int nf) {
  const long long nrows = c->S / c->N[0];
  if (cplx) return nrows * nf;
  return nf == 1 ? nrows / 2 : nrows;
}

template <typename T, bool CPLX, int N, int NF>
static int launch_rows_fwd(bdgd_ctx *c, const Prog &p, const FieldsDev &fd, const void *x, long long ldx,
                           typename Cx<T>::t *spec, int nc, int h) {
  typedef typename Cx<T>::t C;
  const size_t sm = lines_smem<C, N>();
  int rc = set_smem(k_rows_fwd_reg<T, CPLX, N, NF>, sm);
  if (rc) return rc;
  const long long nlines = row_lines(c, CPLX, NF);
  const long long nb = (nlines + LPlan<N>::TX - 1) / LPlan<N>::TX;
  bdgd_count_launch();
  k_rows_fwd_reg<T, CPLX, N, NF><<<dim3(nc, (unsigned)nb), 128, sm, c->stream>>>(c->geo, p, fd, x, ldx, spec, h,
                                                                                nlines);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}

template <typename T, bool CPLX, int N, int NF>
static int launch_rows_inv(bdgd_ctx *c, const Prog &p, const FieldsDev &fd, const typename Cx<T>::t *spec,
                           const void *x, long long ldx, void *y, long long ldy, int nc, int h) {
  typedef typename Cx<T>::t C;
  const size_t sm = lines_smem<C, N>();
  int rc = set_smem(k_rows_inv_reg<T, CPLX, N, NF>, sm);
  if (rc) return rc;
  // complex lines of the inverse are whole rows (both fields per thread)
  const long long nlines = CPLX ? c->S / c->N[0] : row_lines(c, CPLX, NF);
  const long long nb = (nlines + LPlan<N>::TX - 1) / LPlan<N>::TX;
  bdgd_count_launch();
  k_rows_inv_reg<T, CPLX, N, NF><<<dim3(nc, (unsigned)nb), 128, sm, c->stream>>>(c->geo, p, fd, spec, x, ldx, y,
                                                                                ldy, h, nlines);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}

#define LINES_SWITCH(n, CALL) \
  switch (n) {                \
    case 16: CALL(16);        \
    case 32: CALL(32);        \
    case 48: CALL(48);        \
    case 64: CALL(64);        \
    case 96: CALL(96);        \
    case 128: CALL(128);      \
    case 256: CALL(256);      \
    default: break;           \
  }

template <typename T, bool CPLX>
static int rows_fwd(bdgd_ctx *c, const Prog &p, const FieldsDev &fd, const void *x, long long ldx,
                    typename Cx<T>::t *spec, int nc, int h) {
#define RF(NV) return p.nf[h] == 2 ? launch_rows_fwd<T, CPLX, NV, 2>(c, p, fd, x, ldx, spec, nc, h) \
                                   : launch_rows_fwd<T, CPLX, NV, 1>(c, p, fd, x, ldx, spec, nc, h)
  LINES_SWITCH(c->N[0], RF)
#undef RF
  return BDGD_ERR_UNSUPPORTED;
}

template <typename T, bool CPLX>
static int rows_inv(bdgd_ctx *c, const Prog &p, const FieldsDev &fd, const typename Cx<T>::t *spec, const void *x,
                    long long ldx, void *y, long long ldy, int nc, int h) {
#define RI(NV) return p.nf[h] == 2 ? launch_rows_inv<T, CPLX, NV, 2>(c, p, fd, spec, x, ldx, y, ldy, nc, h) \
                                   : launch_rows_inv<T, CPLX, NV, 1>(c, p, fd, spec, x, ldx, y, ldy, nc, h)
  LINES_SWITCH(c->N[0], RI)
#undef RI
  return BDGD_ERR_UNSUPPORTED;
}

template <typename T>
static int cols(bdgd_ctx *c, const Prog &p, const FieldsDev &fd, typename Cx<T>::t *spec, int njobs, int axis,
                int mode) {
#define CC(NV)                                                                      \
  return mode == 0   ? launch_cols<T, NV, 0>(c, p, fd, spec, njobs, axis)           \
         : mode == 1 ? launch_cols<T, NV, 1>(c, p, fd, spec, njobs, axis)           \
                     : launch_cols<T, NV, 2>(c, p, fd, spec, njobs, axis)
  LINES_SWITCH(c->N[axis], CC)
#undef CC
  return BDGD_ERR_UNSUPPORTED;
}

// lines per block for line length n (LPlan<n>::TX)
static int lines_tx(int n) {
  switch (n) {
    case 16: return LPlan<16>::TX;
    case 32: return LPlan<32>::TX;
    case 48: return LPlan<48>::TX;
    case 64: return LPlan<64>::TX;
    case 96: return LPlan<96>::TX;
    case 128: return LPlan<128>::TX;
    case 256: return LPlan<256>::TX;
    default: return 0;
  }
}

bool bdgd_lines_usable(const bdgd_ctx *c, const Prog &p) {
  if (c->dim < 2) return false;
  for (int d = 0; d < c->dim; ++d)
    if (!bdgd_lines_size_ok(c->N[d])) return false;
  // line blocks run along grid.y (at most 65535)
  const long long rows = c->S / c->N[0];
  if ((rows * 2 + lines_tx(c->N[0]) - 1) / lines_tx(c->N[0]) > 65535) return false;
  for (int d = 1; d < c->dim; ++d)
    if ((c->H / c->N[d] + lines_tx(c->N[d]) - 1) / lines_tx(c->N[d]) > 65535) return false;
  if (!c->cplx) {
    for (int h = 0; h < p.nh; ++h)
      if (p.nf[h] == 1 && (rows % 2)) return false;
  }
  return true;
}

template <typename T, bool CPLX>
static int apply_t(bdgd_ctx *c, const Prog &p, const FieldsDev &fd, const void *x, long long ldx, void *y,
                   long long ldy, typename Cx<T>::t *spec, int nc) {
  int rc;
  for (int h = 0; h < p.nh; ++h)
    if ((rc = rows_fwd<T, CPLX>(c, p, fd, x, ldx, spec, nc, h))) return rc;
  for (int ax = 1; ax < c->dim; ++ax)
    if ((rc = cols<T>(c, p, fd, spec, nc * p.J, ax, ax == c->dim - 1 ? 2 : 0))) return rc;
  for (int ax = c->dim - 2; ax >= 1; --ax)
    if ((rc = cols<T>(c, p, fd, spec, nc * p.J, ax, 1))) return rc;
  for (int h = 0; h < p.nh; ++h)
    if ((rc = rows_inv<T, CPLX>(c, p, fd, spec, x, ldx, y, ldy, nc, h))) return rc;
  return BDGD_OK;
}

int bdgd_lines_apply(bdgd_ctx *c, const Prog &p, const FieldsDev &fd, int prec, const void *x, long long ldx,
                     void *y, long long ldy, void *spec, int nc) {
  if (prec == BDGD_F32) {
    if (c->cplx) return apply_t<float, true>(c, p, fd, x, ldx, y, ldy, (float2 *)spec, nc);
    return apply_t<float, false>(c, p, fd, x, ldx, y, ldy, (float2 *)spec, nc);
  }
  if (c->cplx) return apply_t<double, true>(c, p, fd, x, ldx, y, ldy, (double2 *)spec, nc);
  return apply_t<double, false>(c, p, fd, x, ldx, y, ldy, (double2 *)spec, nc);
}
