// bdg_kern.cuh -- device helpers shared by the operator kernels: complex
// arithmetic, small in-register DFTs, operator programs (prologue, k-space
// multiplier, epilogue).  Internal to the library.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

#include "bdg_dev.h"

// Opt a kernel in to sm bytes of dynamic shared memory; skipped while a
// stream capture records the launches (the attribute is already set by the
// uncaptured first run of the same apply).
template <typename K>
static inline int bdgd_smem_attr(K kern, size_t sm) {
  if (bdgd_capturing) return BDGD_OK;
  BDGD_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  return BDGD_OK;
}

// ---------------------------------------------------------------------------
// complex helpers
// ---------------------------------------------------------------------------
template <typename T> struct Cx;
template <> struct Cx<double> { typedef double2 t; };
template <> struct Cx<float> { typedef float2 t; };

template <typename C> __device__ __forceinline__ C cmk(double a, double b) {
  C r;
  r.x = a;
  r.y = b;
  return r;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) {
  C r;
  r.x = a.x + b.x;
  r.y = a.y + b.y;
  return r;
}
template <typename C> __device__ __forceinline__ C csub(C a, C b) {
  C r;
  r.x = a.x - b.x;
  r.y = a.y - b.y;
  return r;
}
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  C r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <typename C> __device__ __forceinline__ C cconj(C a) {
  a.y = -a.y;
  return a;
}
template <typename C, typename T> __device__ __forceinline__ C cscale(C a, T s) {
  a.x *= s;
  a.y *= s;
  return a;
}
// (x + i y) * (sgn * i)
template <typename C> __device__ __forceinline__ C cmul_si(C a, int sgn) {
  C r;
  if (sgn > 0) {
    r.x = -a.y;
    r.y = a.x;
  } else {
    r.x = a.y;
    r.y = -a.x;
  }
  return r;
}

template <typename C> __device__ __forceinline__ const C *roots_of(const AxisDev &ax);
template <> __device__ __forceinline__ const double2 *roots_of<double2>(const AxisDev &ax) {
  return ax.r64;
}
template <> __device__ __forceinline__ const float2 *roots_of<float2>(const AxisDev &ax) {
  return ax.r32;
}

// root(m) = exp(sgn * 2 pi i m / n)
template <typename C> __device__ __forceinline__ C rootv(const C *r, int m, int sgn) {
  C w = __ldg(r + m);
  if (sgn > 0) w.y = -w.y;
  return w;
}

// ---------------------------------------------------------------------------
// small DFT butterflies (in registers)
// ---------------------------------------------------------------------------
template <typename C> __device__ __forceinline__ void bfly2(C *v) {
  C a = v[0];
  v[0] = cadd(a, v[1]);
  v[1] = csub(a, v[1]);
}

template <typename C> __device__ __forceinline__ void bfly4(C &v0, C &v1, C &v2, C &v3, int sgn) {
  C a0 = cadd(v0, v2), a1 = csub(v0, v2);
  C a2 = cadd(v1, v3), a3 = cmul_si(csub(v1, v3), sgn);
  v0 = cadd(a0, a2);
  v2 = csub(a0, a2);
  v1 = cadd(a1, a3);
  v3 = csub(a1, a3);
}

template <typename C> __device__ __forceinline__ void bfly8(C *v, int sgn) {
  // even/odd split: E = DFT4(v0 v2 v4 v6), O = DFT4(v1 v3 v5 v7)
  bfly4(v[0], v[2], v[4], v[6], sgn);
  bfly4(v[1], v[3], v[5], v[7], sgn);
  typedef decltype(v[0].x) E;
  const E h = (E)0.70710678118654752440;
  C o1 = v[3], o2 = v[5], o3 = v[7];
  // o1 * exp(sgn i pi/4) = h (x - sgn y) + i h (sgn x + y)
  C t1, t3;
  t1.x = h * (o1.x - sgn * o1.y);
  t1.y = h * (sgn * o1.x + o1.y);
  C t2 = cmul_si(o2, sgn);
  // o3 * exp(sgn i 3pi/4) = h(-x - sgn y) + i h(sgn x - y)
  t3.x = h * (-o3.x - sgn * o3.y);
  t3.y = h * (sgn * o3.x - o3.y);
  C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  C o0 = v[1];
  v[0] = cadd(e0, o0);
  v[4] = csub(e0, o0);
  v[1] = cadd(e1, t1);
  v[5] = csub(e1, t1);
  v[2] = cadd(e2, t2);
  v[6] = csub(e2, t2);
  v[3] = cadd(e3, t3);
  v[7] = csub(e3, t3);
}

template <typename C> __device__ __forceinline__ void bfly3(C *v, int sgn) {
  typedef decltype(v[0].x) E;
  const E h = (E)0.86602540378443864676;
  C t1 = cadd(v[1], v[2]);
  C t2;
  t2.x = v[0].x - (E)0.5 * t1.x;
  t2.y = v[0].y - (E)0.5 * t1.y;
  C t3 = cscale(cmul_si(csub(v[1], v[2]), sgn), h);
  v[0] = cadd(v[0], t1);
  v[1] = cadd(t2, t3);
  v[2] = csub(t2, t3);
}

template <int R, typename C> struct Bfly {
  static __device__ __forceinline__ void run(C *v, int sgn) {}
};
template <typename C> struct Bfly<2, C> {
  static __device__ __forceinline__ void run(C *v, int) { bfly2(v); }
};
template <typename C> struct Bfly<3, C> {
  static __device__ __forceinline__ void run(C *v, int sgn) { bfly3(v, sgn); }
};
template <typename C> struct Bfly<4, C> {
  static __device__ __forceinline__ void run(C *v, int sgn) { bfly4(v[0], v[1], v[2], v[3], sgn); }
};
template <typename C> struct Bfly<8, C> {
  static __device__ __forceinline__ void run(C *v, int sgn) { bfly8(v, sgn); }
};

// ---------------------------------------------------------------------------
// operator programs
// ---------------------------------------------------------------------------
enum { PRE_NONE = 0, PRE_PK, PRE_PM, PRE_CONJWF, PRE_DENS, PRE_XDENS };
enum { MUL_KIN = 0, MUL_DIP, MUL_PRE, MUL_ONE, MUL_EXPKIN };
enum { POST_RAW = 0, POST_K, POST_M, POST_TK, POST_TM, POST_DIPCONV, POST_PHI };

struct Prog {
  int nh;         // halves per column (1, or 2 for [u; v])
  int J;          // spectra (jobs) per column
  int nf[2];      // spectra per half
  int j0[2];      // first job of each half
  int pre[2][2];  // prologue per half, field
  int mul[2][2];  // k-space multiplier per half, field
  int post[2];    // epilogue per half
  int jh[4], jf[4];
};

// k-space multiplier of spectrum element (ix, iy, iz), flat index kidx.
// Same arithmetic as the reference loops: k2 = kx2[0][ix] + kx2[1][iy] +
// kx2[2][iz]; kinetic k2 * (0.5/size) (src/kinetic_impl.inc:25-27); dipolar
// kernel * (1/size) (src/dipolar_conv_impl.inc:41-43); preconditioner
// (1/size) / safe_val(mu + 0.5 k2) (src/precond_impl.inc:45-48).
__device__ __forceinline__ double kmult(const GeoDev &g, const FieldsDev &f, int kind, int ix, int iy,
                                        int iz, long long kidx) {
  if (kind == MUL_DIP) return __ldg(f.vdd + kidx) * f.inv_size;
  if (kind == MUL_ONE) return 1.0;
  if (kind == MUL_PRE && f.ptab) return __ldg(f.ptab + kidx);
  double k2 = __ldg(g.kx2[0] + ix);
  if (g.dim > 1) k2 += __ldg(g.kx2[1] + iy);
  if (g.dim > 2) k2 += __ldg(g.kx2[2] + iz);
  if (kind == MUL_KIN) return k2 * (0.5 * f.inv_size);
  if (kind == MUL_EXPKIN) return exp(-f.kin_dt * k2) * f.inv_size;
  double d = f.mu + 0.5 * k2;
  if (fabs(d) < 1e-8) d = 1e-8;
  return f.inv_size / d;
}

// kmult for a kind other than MUL_DIP/MUL_PRE-with-table, given k2 already
// summed in the reference order (kx2[0][ix] + kx2[1][iy] + kx2[2][iz]).
__device__ __forceinline__ double kmult_k2(const FieldsDev &f, int kind, double k2) {
  if (kind == MUL_ONE) return 1.0;
  if (kind == MUL_KIN) return k2 * (0.5 * f.inv_size);
  if (kind == MUL_EXPKIN) return exp(-f.kin_dt * k2) * f.inv_size;
  double d = f.mu + 0.5 * k2;
  if (fabs(d) < 1e-8) d = 1e-8;
  return f.inv_size / d;
}

// ---------------------------------------------------------------------------
// element access helpers for the real (T) and complex (C) paths
// ---------------------------------------------------------------------------
template <typename T, bool CPLX> struct El;
template <typename T> struct El<T, false> {
  typedef typename Cx<T>::t C;
  typedef T V;
  static __device__ __forceinline__ C to_c(V v) { return cmk<C>(v, 0.0); }
  static __device__ __forceinline__ V from_c(C c) { return c.x; }
};
template <typename T> struct El<T, true> {
  typedef typename Cx<T>::t C;
  typedef C V;
  static __device__ __forceinline__ C to_c(V v) { return v; }
  static __device__ __forceinline__ V from_c(C c) { return c; }
};

template <typename T, bool CPLX>
__device__ __forceinline__ typename El<T, CPLX>::C prologue(const FieldsDev &f, int kind,
                                                            typename El<T, CPLX>::V x, long long r) {
  typedef typename El<T, CPLX>::C C;
  typedef typename El<T, CPLX>::V V;
  const T *pK = (const T *)f.pK;
  const T *pM = (const T *)f.pM;
  const V *w = (const V *)f.w;
  if constexpr (CPLX) {
    switch (kind) {
      case PRE_PK: return cscale(x, __ldg(pK + r));
      case PRE_PM: return cscale(x, __ldg(pM + r));
      case PRE_CONJWF: return cmul(cconj(w[r]), x);
      case PRE_DENS: {
        // |psi|^2 as cabs(psi)^2 (src/dipolar_meanfield_impl.inc:33-35)
        C z = w[r];
        T a = hypot(z.x, z.y);
        return cmk<C>(a * a, 0.0);
      }
      case PRE_XDENS: return cmk<C>(x.x * x.x + x.y * x.y, 0.0);
      default: return x;
    }
  } else {
    switch (kind) {
      case PRE_PK: return cmk<C>(__ldg(pK + r) * x, 0.0);
      case PRE_PM: return cmk<C>(__ldg(pM + r) * x, 0.0);
      case PRE_CONJWF: return cmk<C>(w[r] * x, 0.0);
      case PRE_DENS: {
        T a = fabs(w[r]);
        return cmk<C>(a * a, 0.0);
      }
      case PRE_XDENS: return cmk<C>(x * x, 0.0);
      default: return cmk<C>(x, 0.0);
    }
  }
}

// Epilogue of one half at real-space point r given the inverse transforms
// o0 (and o1 for M with dipolar exchange).  Reference arithmetic order:
//   K: y = kin + ltK*x                      (src/matmulK_impl.inc:21-23)
//   M: y = kin + (ltM*x + 2*(g*wf*buf))     (src/matmulM_impl.inc:30-32, dipolar_conv :49-51)
//   T: y = out * p                          (src/precond_impl.inc:56-60)
template <typename T, bool CPLX>
__device__ __forceinline__ typename El<T, CPLX>::V epilogue(const FieldsDev &f, int post, int nf,
                                                            typename El<T, CPLX>::C o0,
                                                            typename El<T, CPLX>::C o1,
                                                            typename El<T, CPLX>::V x, long long r) {
  typedef typename El<T, CPLX>::V V;
  typedef typename El<T, CPLX>::C C;
  const T *ltK = (const T *)f.ltK;
  const T *ltM = (const T *)f.ltM;
  const T *pK = (const T *)f.pK;
  const T *pM = (const T *)f.pM;
  const V *w = (const V *)f.w;
  const T g = (T)f.g_ddi;
  if constexpr (CPLX) {
    switch (post) {
      case POST_K: return cadd(o0, cscale(x, __ldg(ltK + r)));
      case POST_M:
        if (nf > 1) {
          C dc = cmul(cscale(w[r], g), o1);
          return cadd(o0, cadd(cscale(x, __ldg(ltM + r)), cscale(dc, (T)2)));
        }
        return cadd(o0, cscale(x, __ldg(ltM + r)));
      case POST_TK: return cscale(o0, __ldg(pK + r));
      case POST_TM: return cscale(o0, __ldg(pM + r));
      case POST_DIPCONV: return cmul(cscale(w[r], g), o0);
      case POST_PHI: return cmk<C>(g * o0.x, 0.0);
      default: return o0;
    }
  } else {
    const T y0 = o0.x;
    switch (post) {
      case POST_K: return y0 + __ldg(ltK + r) * x;
      case POST_M:
        if (nf > 1) {
          const T dc = (g * w[r]) * o1.x;
          return y0 + (__ldg(ltM + r) * x + (T)2 * dc);
        }
        return y0 + __ldg(ltM + r) * x;
      case POST_TK: return y0 * __ldg(pK + r);
      case POST_TM: return y0 * __ldg(pM + r);
      case POST_DIPCONV: return (g * w[r]) * o0.x;
      case POST_PHI: return g * o0.x;
      default: return y0;
    }
  }
}
