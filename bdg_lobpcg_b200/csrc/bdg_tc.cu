// bdg_tc.cu -- tensor-core (tcgen05, sm_100a) kernels of the solver's FP64
// and FP32 contractions (Gram and basis update through int8 digits).
//
// k_tc_i8_gemm: D = A B^T with int8 A (M x K) and B (N x K), K contiguous,
// int32 D; one 128 x 64 output tile per CTA, K in steps of 32 through a
// two-stage shared-memory ring, the accumulator in TMEM.  It is the building
// block the FP64 emulation is made of, exported (bdgd_tc_i8_gemm) so that its
// layouts and descriptors are checked on their own against integer
// arithmetic.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "bdg/bdg_cuda.h"
#include "bdg_dev.h"
#include "bdg_tc.cuh"

using namespace bdgtc;

// spin limit of every mbarrier wait (~seconds); past it the kernel records
// an error and returns instead of hanging
#define TC_WAIT_LIMIT (1LL << 26)

__global__ void __launch_bounds__(128) k_tc_i8_gemm(const int8_t *__restrict__ A, long long lda,
                                                     const int8_t *__restrict__ Bm, long long ldb,
                                                     int32_t *__restrict__ D, long long ldd, int K,
                                                     int *__restrict__ err) {
  __shared__ __align__(128) int8_t sa[2][128 * 32];
  __shared__ __align__(128) int8_t sb[2][64 * 32];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ uint32_t tbase;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) tmem_alloc(&tbase, 64);
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init_fence();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tbase;
  const long long m0 = (long long)blockIdx.x * 128, n0 = (long long)blockIdx.y * 64;
  const int nk = K / 32;
  uint32_t phase0 = 0, phase1 = 0;
  int failed = 0;
  for (int ks = 0; ks < nk; ++ks) {
    const int s = ks & 1;
    if (ks >= 2) {  // the MMA committed two steps ago read this stage
      uint32_t &ph = s ? phase1 : phase0;
      const bool ok = mbar_wait(&bar[s], ph, TC_WAIT_LIMIT);
      ph ^= 1;
      failed = __syncthreads_or(!ok);
      if (failed) break;
    }
    {
      const int4 *src = reinterpret_cast<const int4 *>(A + (m0 + tid) * lda + (long long)ks * 32);
      int8_t *dst = sa[s] + (tid & 7) * 16 + (tid >> 3) * 256;
      *reinterpret_cast<int4 *>(dst) = src[0];
      *reinterpret_cast<int4 *>(dst + 128) = src[1];
    }
    if (tid < 64) {
      const int4 *src = reinterpret_cast<const int4 *>(Bm + (n0 + tid) * ldb + (long long)ks * 32);
      int8_t *dst = sb[s] + (tid & 7) * 16 + (tid >> 3) * 256;
      *reinterpret_cast<int4 *>(dst) = src[0];
      *reinterpret_cast<int4 *>(dst + 128) = src[1];
    }
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      mma_i8(tmem, smem_desc(smem_u32(sa[s])), smem_desc(smem_u32(sb[s])), idesc_i8(64), ks > 0 ? 1u : 0u);
      mma_commit(&bar[s]);
    }
  }
  if (!failed && nk > 0) {  // the last commit covers every MMA issued before it
    const int s = (nk - 1) & 1;
    const bool ok = mbar_wait(&bar[s], s ? phase1 : phase0, TC_WAIT_LIMIT);
    failed = __syncthreads_or(!ok);
  }
  tc_fence_after();
  if (!failed) {
    const long long row = m0 + warp * 32 + lane;
    for (int c = 0; c < 64; c += 16) {
      int32_t v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) D[row * ldd + n0 + c + i] = v[i];
    }
  } else if (tid == 0) {
    atomicExch(err, 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_free(tmem, 64);
}

extern "C" int bdgd_tc_i8_gemm(void *stream, const int8_t *A, uint64_t lda, const int8_t *B, uint64_t ldb,
                               int32_t *D, uint64_t ldd, uint64_t M, uint64_t N, uint64_t K, int *d_err) {
  if (M % 128 || N % 64 || K % 32 || M == 0 || N == 0 || K == 0) {
    bdgd_set_error("bdgd_tc_i8_gemm: M must be a multiple of 128, N of 64, K of 32");
    return BDGD_ERR_ARG;
  }
  if (((uintptr_t)A | (uintptr_t)B) % 16 || lda % 16 || ldb % 16 || lda < K || ldb < K || ldd < N || !d_err) {
    bdgd_set_error("bdgd_tc_i8_gemm: operands must be 16-byte aligned with K-contiguous rows");
    return BDGD_ERR_ARG;
  }
  bdgd_count_launch();
  k_tc_i8_gemm<<<dim3((unsigned)(M / 128), (unsigned)(N / 64)), 128, 0, (cudaStream_t)stream>>>(
      A, (long long)lda, B, (long long)ldb, D, (long long)ldd, (int)K, d_err);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}

// ---------------------------------------------------------------------------
// FP64 contractions on the integer tensor cores (Ozaki-style splitting).
//
// A value x of a column (or row) whose magnitudes stay below 2^(S-1) is
// written as the integer X = rint(x 2^(55 - S)), |X| < 2^54, in 7 signed
// 8-bit digits: X = sum_{t<6} d_t 256^t + d_6 256^6, taken from the bytes of
// X + 0x808080808080 (the offset makes the six low digits signed).  A dot
// product of two such sequences is
//   sum_r a_r b_r = 2^(S_a + S_b - 110) sum_{t,u} 256^(t+u) sum_r d_t d'_u,
// each inner sum an exact int32 dot product of int8 digits on the tensor
// cores (tcgen05.mma kind::i8).  Diagonals t + u >= 5 are kept (34 MMAs per
// 32-deep step); the dropped ones are below 2^-57 of max|a| max|b| per term.
// The 8 kept diagonals accumulate in 8 int32 TMEM accumulators (128 x 64
// each: all 512 TMEM columns); a diagonal sums at most 7 products of
// |d| <= 128 per term, so 16384 terms stay exact in int32.
// ---------------------------------------------------------------------------
#define OZ_CHUNK 16384
#define OZ_MAXT 48
#define OZ_THREADS 512              // digit threads of the update
#define OZ_DTHREADS 512             // digit threads of the Gram (warps 0-15)
#define OZ_BLOCK (OZ_DTHREADS + 32) // + the Gram's MMA warp
#define OZ_ND 7          // digits per value
#define OZ_DMIN 5        // lowest kept diagonal t + u
#define OZ_NDIAG 8       // kept diagonals 5..12
#define OZ_P 55          // X = rint(a * 2^(OZ_P - S))
#define OZ_STAGE_A (OZ_ND * 128 * 32)
#define OZ_STAGE_B (OZ_ND * 64 * 32)
#define OZ_STAGE (OZ_STAGE_A + OZ_STAGE_B)

// scale = 2^(P - S) with 2^(S - 1) above the column's largest |x|, the
// exponent clamped to [pmin, pmax] (the scale's own range)
__device__ __forceinline__ void oz_scale(unsigned long long bits, double &scale, int &S, bool &finite, int P = OZ_P,
                                         int pmin = -1022, int pmax = 1023) {
  const double m = __longlong_as_double((long long)bits);
  finite = isfinite(m);
  if (!(m > 0.0) || !finite) {  // zero column (or not finite: flagged at the flush)
    scale = 1.0;
    S = 0;
    return;
  }
  int E = 0;
  frexp(m, &E);  // m = f 2^E, f in [0.5, 1): |x| < 2^E
  S = E + 1;
  int p = P - S;
  if (p > pmax) p = pmax;
  if (p < pmin) p = pmin;
  scale = ldexp(1.0, p);
}

// digit words of 4 consecutive values: w[t] holds digit t of the four
__device__ __forceinline__ void oz_digits4(double v0, double v1, double v2, double v3, double scale,
                                           uint32_t (&w)[OZ_ND]) {
  uint32_t lo[4], hi[4];
  const double v[4] = {v0, v1, v2, v3};
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const long long X = __double2ll_rn(v[q] * scale) + 0x808080808080LL;
    lo[q] = (uint32_t)X ^ 0x80808080u;
    hi[q] = (uint32_t)((unsigned long long)X >> 32) ^ 0x8080u;
  }
  // 4 x 4 byte transposes
  const uint32_t a0 = __byte_perm(lo[0], lo[1], 0x5140), a1 = __byte_perm(lo[2], lo[3], 0x5140);
  const uint32_t a2 = __byte_perm(lo[0], lo[1], 0x7362), a3 = __byte_perm(lo[2], lo[3], 0x7362);
  const uint32_t b0 = __byte_perm(hi[0], hi[1], 0x5140), b1 = __byte_perm(hi[2], hi[3], 0x5140);
  const uint32_t b2 = __byte_perm(hi[0], hi[1], 0x7362), b3 = __byte_perm(hi[2], hi[3], 0x7362);
  w[0] = __byte_perm(a0, a1, 0x5410);
  w[1] = __byte_perm(a0, a1, 0x7632);
  w[2] = __byte_perm(a2, a3, 0x5410);
  w[3] = __byte_perm(a2, a3, 0x7632);
  w[4] = __byte_perm(b0, b1, 0x5410);
  w[5] = __byte_perm(b0, b1, 0x7632);
  w[6] = __byte_perm(b2, b3, 0x5410);
}

// FP32 values (the FP32 phase of the mixed form): X = rint(x 2^(31 - S)),
// |X| < 2^30, in 4 signed 8-bit digits from the bytes of X + 0x808080;
// w[t] holds digit t of the four values
__device__ __forceinline__ void oz_digits4f(float v0, float v1, float v2, float v3, float scale,
                                            uint32_t (&w)[4]) {
  uint32_t lo[4];
  const float v[4] = {v0, v1, v2, v3};
#pragma unroll
  for (int q = 0; q < 4; ++q) lo[q] = (uint32_t)(__float2int_rn(v[q] * scale) + 0x808080) ^ 0x808080u;
  const uint32_t a0 = __byte_perm(lo[0], lo[1], 0x5140), a1 = __byte_perm(lo[2], lo[3], 0x5140);
  const uint32_t a2 = __byte_perm(lo[0], lo[1], 0x7362), a3 = __byte_perm(lo[2], lo[3], 0x7362);
  w[0] = __byte_perm(a0, a1, 0x5410);
  w[1] = __byte_perm(a0, a1, 0x7632);
  w[2] = __byte_perm(a2, a3, 0x5410);
  w[3] = __byte_perm(a2, a3, 0x7632);
}

// digit formats of the Gram per input type: digits per value, lowest kept
// diagonal, kept diagonals, fixed-point bits, range of the scale exponent
template <typename T>
struct OzFmt;
template <>
struct OzFmt<double> {
  static constexpr int ND = 7, DMIN = 5, NDIAG = 8, P = 55, PMIN = -1022, PMAX = 1023;
};
template <>
struct OzFmt<float> {
  // diagonals t + u >= 2 of 4 x 4 (13 products); the dropped ones are below
  // 2^-33 of max|a| max|b| per term, under the FP32 inputs' own rounding
  static constexpr int ND = 4, DMIN = 2, NDIAG = 5, P = 31, PMIN = -126, PMAX = 127;
};

struct OzTask {
  const void *a, *b;
  long long lda, ldb, rows;
  int ka, kb, out, i0, j0, sym, mirror;
  int nsp;                // row chunks of this task
  int ma, mb;             // offsets of the operands' column maxima
  long long part0;        // offset of the task's chunk partials (doubles)
};

// A 128 x 64 output tile: two 64-column slices of A operands (of one task or
// of two tasks that share the B operand, its rows and its columns) against
// one 64-column tile of B, so that tasks of 64 columns fill whole tiles.
struct OzTile {
  short ta[2], sa[2];     // task and 64-column slice of each half (ta = -1: empty)
  short tb, jb;           // task of the B operand and rows, B column tile
  int nsp;                // row chunks
};
#define OZ_MAXTILES 640
struct OzArgs {
  OzTask t[OZ_MAXT];
  OzTile p[OZ_MAXTILES];  // sorted by nsp, largest first
  int nt, np;
  const unsigned long long *colmax;  // |x| maxima as FP64 bit patterns
  double *part;
  int *err;
};

// Digit stages in shared memory (MMA operands, 6144 bytes per digit: 43008
// for FP64 values, 24576 for FP32) and the per-step raw values of a digit
// thread, held in registers: 8 rows of its A column and 4 rows of its B
// column.
#define OZ_NS 4
template <typename T>
constexpr int oz_smem_bytes() {
  return OZ_NS * OzFmt<T>::ND * 6144 + 4096;
}

template <typename T>
struct OzRaw;
template <>
struct OzRaw<double> {
  double2 a[4], b[2];
};
template <>
struct OzRaw<float> {
  float4 a[2], b;
};

__device__ __forceinline__ void oz_load(OzRaw<float> &x, const float *pa, const float *pb) {
  const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
  if (pa) {
    const float4 *p = reinterpret_cast<const float4 *>(pa);
    x.a[0] = __ldg(p);
    x.a[1] = __ldg(p + 1);
  } else {
    x.a[0] = x.a[1] = z;
  }
  x.b = pb ? __ldg(reinterpret_cast<const float4 *>(pb)) : z;
}

// the step's digits of a digit thread: w0 / w1 the A rows 0-3 / 4-7, wb the B rows
__device__ __forceinline__ void oz_step_digits(const OzRaw<double> &x, double sa, double sb, uint32_t (&w0)[7],
                                               uint32_t (&w1)[7], uint32_t (&wb)[7]) {
  oz_digits4(x.a[0].x, x.a[0].y, x.a[1].x, x.a[1].y, sa, w0);
  oz_digits4(x.a[2].x, x.a[2].y, x.a[3].x, x.a[3].y, sa, w1);
  oz_digits4(x.b[0].x, x.b[0].y, x.b[1].x, x.b[1].y, sb, wb);
}
__device__ __forceinline__ void oz_step_digits(const OzRaw<float> &x, double sa, double sb, uint32_t (&w0)[4],
                                               uint32_t (&w1)[4], uint32_t (&wb)[4]) {
  oz_digits4f(x.a[0].x, x.a[0].y, x.a[0].z, x.a[0].w, (float)sa, w0);
  oz_digits4f(x.a[1].x, x.a[1].y, x.a[1].z, x.a[1].w, (float)sa, w1);
  oz_digits4f(x.b.x, x.b.y, x.b.z, x.b.w, (float)sb, wb);
}

__device__ __forceinline__ void oz_load(OzRaw<double> &x, const double *pa, const double *pb) {
  const double2 z = make_double2(0.0, 0.0);
  if (pa) {
    const double2 *p = reinterpret_cast<const double2 *>(pa);
#pragma unroll
    for (int i = 0; i < 4; ++i) x.a[i] = __ldg(p + i);
  } else {
#pragma unroll
    for (int i = 0; i < 4; ++i) x.a[i] = z;
  }
  if (pb) {
    const double2 *p = reinterpret_cast<const double2 *>(pb);
    x.b[0] = __ldg(p);
    x.b[1] = __ldg(p + 1);
  } else {
    x.b[0] = x.b[1] = z;
  }
}

// unit -> (tile, chunk): chunks ascending; in chunk range [nsp_{i+1},
// nsp_i) the tiles 0..i (sorted by nsp, largest first) are active
__device__ __forceinline__ void oz_unit(const OzArgs &g, int unit, int &tile, int &split) {
  int u = unit;
  tile = split = 0;
  for (int i = g.np - 1; i >= 0; --i) {
    const int lo = (i == g.np - 1) ? 0 : g.p[i + 1].nsp, hi = g.p[i].nsp;
    const int cnt = (hi - lo) * (i + 1);
    if (u < cnt) {
      split = lo + u / (i + 1);
      tile = u - (u / (i + 1)) * (i + 1);
      return;
    }
    u -= cnt;
  }
}

// C = A^T B over a long row range, A (rows x ka) and B (rows x kb) FP64 or
// FP32, column-major, each column scaled by its maximum over all rows
// (pre-pass).  Persistent: one CTA per SM walks the work units (packed
// 128 x 64 output tile, 16384-row chunk) chunk by chunk, so that the CTAs
// working at one time share rows in L2.  A tile's two 64-row halves are
// 64-column slices of A operands that share the tile's B operand (see
// OzTile).  Warp-specialised per unit:
//  * 16 digit warps: each thread loads 8 rows of one A column and 4 rows of
//    one B column straight into registers two steps ahead, turns them into
//    digits and stores them into a digit stage (thread-to-column mapping
//    chosen so that each warp's stores hit 32 distinct banks), then signals
//    the stage;
//  * one MMA warp: waits for each digit stage and issues its products, whose
//    commit frees the stage.  The 34 digit products of a step are grouped by
//    A digit t over consecutive B digits u (N = 64 per digit, up to 256): the
//    B digits of a stage are contiguous and the accumulator of diagonal
//    t + u sits at TMEM column 64 (t + u - 5), so one MMA with N = 64 c adds
//    A_t [B_u .. B_u+c-1] into diagonals t + u .. t + u + c - 1 (11 MMAs per
//    step, which cuts the operand reads from shared memory from 204 KB to
//    112 KB).  The first step of a unit initialises each diagonal with
//    single-digit MMAs instead.
// TMEM accumulates the unit; the digit warps flush its FP64 chunk partial.
__device__ __forceinline__ bool oz_wait(uint64_t *bar, uint32_t &bits, int s, volatile int *fail) {
  const uint32_t ph = (bits >> s) & 1u;
  bits ^= 1u << s;
  if (*fail) return false;
  const bool ok = mbar_wait(bar, ph, TC_WAIT_LIMIT);
  if (!ok) *fail = 1;
  return ok;
}

template <typename T>
__global__ void __launch_bounds__(OZ_BLOCK, 1) k_gram_oz(OzArgs g, long long chunk, int nunits) {
  constexpr int ND = OzFmt<T>::ND, DMIN = OzFmt<T>::DMIN, NDIAG = OzFmt<T>::NDIAG, P = OzFmt<T>::P;
  constexpr int STAGE_A = ND * 4096, STAGE = ND * 6144;  // A: 128 x 32 bytes, B: 64 x 32 bytes per digit
  extern __shared__ __align__(1024) uint8_t oz_smem[];
  uint8_t *dig0 = oz_smem;  // [OZ_NS][STAGE]
  uint8_t *misc = dig0 + OZ_NS * STAGE;
  double *scaleA = reinterpret_cast<double *>(misc);
  double *scaleB = scaleA + 128;
  int *SA = reinterpret_cast<int *>(scaleB + 64);
  int *SB = SA + 128;
  int *badA = SB + 64;
  int *badB = badA + 128;
  uint64_t *dfull = reinterpret_cast<uint64_t *>(badB + 64);  // [OZ_NS] digit stage written (16 warp arrivals)
  uint64_t *mdone = dfull + OZ_NS;                            // [OZ_NS] MMAs of a digit stage done (commit)
  uint64_t *fin = mdone + OZ_NS;                              // every MMA of the CTA done (exit path)
  uint32_t *tslot = reinterpret_cast<uint32_t *>(fin + 1);
  volatile int *fail = reinterpret_cast<volatile int *>(tslot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const bool mma_warp = warp == OZ_DTHREADS / 32;
  if (warp == 0) tmem_alloc(tslot, 512);
  if (tid == 0) {
    for (int i = 0; i < OZ_NS; ++i) {
      mbar_init(&dfull[i], OZ_DTHREADS / 32);
      mbar_init(&mdone[i], 1);
    }
    mbar_init(fin, 1);
    *fail = 0;
    mbar_init_fence();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  uint32_t dbits = 0u, mbits = 0u;  // mbarrier phases per stage

  // digit roles (warp w, lane l): A column ca, rows [8 hq, 8 hq + 8) of the
  // step; B column cb, rows [4 he, 4 he + 4).  Within a warp the A stores
  // (8 bytes) of each half-warp and the B stores (4 bytes) cover one 128-byte
  // row group of the K-major layout exactly once.
  const int ca = (warp & 7) * 16 + ((lane >> 4) & 1) * 8 + (lane & 7), hq = ((warp >> 3) & 1) * 2 + ((lane >> 3) & 1);
  const int cb = (warp & 7) * 8 + (lane & 7), he = ((warp >> 3) & 1) * 4 + (lane >> 3);
  const int offA = (ca & 7) * 16 + (ca >> 3) * 256 + (hq >> 1) * 128 + (hq & 1) * 8;
  const int offB = (cb & 7) * 16 + (cb >> 3) * 256 + (he >> 2) * 128 + (he & 3) * 4;

  for (int unit = blockIdx.x; unit < nunits; unit += gridDim.x) {
    int pt, split;
    oz_unit(g, unit, pt, split);
    const OzTile tile = g.p[pt];
    const OzTask &tk = g.t[tile.tb];  // the B operand and the row range
    const int jb = tile.jb;
    const long long r0 = (long long)split * chunk;
    const long long r1 = min(tk.rows, r0 + chunk);
    const int nsteps = r1 > r0 ? (int)((r1 - r0) / 32) : 0;  // rows are a multiple of 32

    if (tid < 128) {
      // A column tid: half tid / 64 of the tile, column 64 sa + tid % 64 of its task
      const int h = tid >> 6, tA = tile.ta[h];
      const int c = tile.sa[h] * 64 + (tid & 63);
      double s = 1.0;
      int S = 0;
      bool fin_ = true;
      if (tA >= 0 && c < g.t[tA].ka) oz_scale(g.colmax[g.t[tA].ma + c], s, S, fin_, P, OzFmt<T>::PMIN, OzFmt<T>::PMAX);
      scaleA[tid] = s;
      SA[tid] = S;
      badA[tid] = !fin_;
    } else if (tid < 192) {
      const int c = jb * 64 + tid - 128;
      double s = 1.0;
      int S = 0;
      bool fin_ = true;
      if (c < tk.kb) oz_scale(g.colmax[tk.mb + c], s, S, fin_, P, OzFmt<T>::PMIN, OzFmt<T>::PMAX);
      scaleB[tid - 128] = s;
      SB[tid - 128] = S;
      badB[tid - 128] = !fin_;
    }
    __syncthreads();
    if (!mma_warp) {
      const int tA = tile.ta[ca >> 6], colA = tile.sa[ca >> 6] * 64 + (ca & 63);
      const T *pa = nullptr;
      if (tA >= 0 && colA < g.t[tA].ka)
        pa = static_cast<const T *>(g.t[tA].a) + (long long)colA * g.t[tA].lda + r0 + 8 * hq;
      const T *pb = jb * 64 + cb < tk.kb
                        ? static_cast<const T *>(tk.b) + (long long)(jb * 64 + cb) * tk.ldb + r0 + 4 * he
                        : nullptr;
      const double sa = scaleA[ca], sb = scaleB[cb];
      auto load = [&](OzRaw<T> &x, int ks) { oz_load(x, pa ? pa + 32LL * ks : nullptr, pb ? pb + 32LL * ks : nullptr); };
      auto step = [&](const OzRaw<T> &x, int ks) {
        const int s = ks & (OZ_NS - 1);
        uint8_t *dig = dig0 + s * STAGE;
        uint32_t w0[ND], w1[ND], wb[ND];
        oz_step_digits(x, sa, sb, w0, w1, wb);
        if (ks >= OZ_NS) oz_wait(&mdone[s], mbits, s, fail);  // the MMAs of step ks - OZ_NS read this stage
#pragma unroll
        for (int t = 0; t < ND; ++t) {
          *reinterpret_cast<uint2 *>(dig + t * 4096 + offA) = make_uint2(w0[t], w1[t]);
          *reinterpret_cast<uint32_t *>(dig + STAGE_A + t * 2048 + offB) = wb[t];
        }
        fence_async_smem();
        __syncwarp();
        if (lane == 0) mbar_arrive(&dfull[s]);
      };
      OzRaw<T> x0, x1;
      if (nsteps > 0) load(x0, 0);
      if (nsteps > 1) load(x1, 1);
      for (int ks = 0; ks < nsteps; ks += 2) {
        step(x0, ks);
        if (ks + 2 < nsteps) load(x0, ks + 2);
        if (ks + 1 < nsteps) {
          step(x1, ks + 1);
          if (ks + 3 < nsteps) load(x1, ks + 3);
        }
      }
      // the unit's accumulators are complete once the last commits arrived
      for (int k = nsteps > OZ_NS ? nsteps - OZ_NS : 0; k < nsteps; ++k)
        oz_wait(&mdone[k & (OZ_NS - 1)], mbits, k & (OZ_NS - 1), fail);
    } else {
      for (int ks = 0; ks < nsteps; ++ks) {
        const int s = ks & (OZ_NS - 1);
        if (lane == 0) {
          const bool ok = oz_wait(&dfull[s], dbits, s, fail);
          tc_fence_after();
          const uint32_t base = smem_u32(dig0 + s * STAGE);
          if (ok && ks == 0) {
#pragma unroll
            for (int t = 0; t < ND; ++t)
#pragma unroll
              for (int u = 0; u < ND; ++u) {
                const int D = t + u;
                if (D < DMIN) continue;
                const int first_t = D - (ND - 1) > 0 ? D - (ND - 1) : 0;
                mma_i8(tmem + (uint32_t)((D - DMIN) * 64), smem_desc(base + t * 4096),
                       smem_desc(base + STAGE_A + u * 2048), idesc_i8(64), t > first_t ? 1u : 0u);
              }
          } else if (ok) {
#pragma unroll
            for (int t = 0; t < ND; ++t)
#pragma unroll
              for (int u0 = (DMIN - t > 0 ? DMIN - t : 0); u0 < ND; u0 += 4) {
                const int cnt = ND - u0 < 4 ? ND - u0 : 4;
                mma_i8(tmem + (uint32_t)((t + u0 - DMIN) * 64), smem_desc(base + t * 4096),
                       smem_desc(base + STAGE_A + u0 * 2048), idesc_i8(64 * cnt), 1u);
              }
          }
          mma_commit(&mdone[s]);
        }
        __syncwarp();
      }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (!mma_warp) {
      // flush: warp w reads TMEM lanes 32 (w % 4).., columns 16 (w / 4)..
      const int row = 32 * (warp & 3) + lane;
      const int tA = tile.ta[row >> 6];
      const OzTask &to = g.t[tA >= 0 ? tA : tile.tb];  // the task this row's output belongs to
      const int i = tile.sa[row >> 6] * 64 + (row & 63);
      const long long kk = (long long)to.ka * to.kb;
      double *part = g.part + to.part0 + (long long)split * kk;
      const int c0 = 16 * (warp >> 2);
      double acc[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) acc[q] = 0.0;
      if (nsteps > 0) {
#pragma unroll
        for (int d = 0; d < NDIAG; ++d) {
          int32_t v[16];
          tmem_ld16(tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(d * 64 + c0), v);
          const double w = ldexp(1.0, 8 * (d + DMIN) - 2 * P);
#pragma unroll
          for (int q = 0; q < 16; ++q) acc[q] = fma((double)v[q], w, acc[q]);
        }
      }
      if (tA >= 0 && i < to.ka) {
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          const int j = jb * 64 + c0 + q;
          if (j < to.kb) {
            double val = ldexp(acc[q], SA[row] + SB[c0 + q]);
            if (badA[row] || badB[c0 + q]) val = __longlong_as_double(0x7ff8000000000000LL);
            part[(long long)j * to.ka + i] = val;
          }
        }
      }
    }
    // TMEM and scale reads done before the next unit reuses them
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (*fail) break;
  }
  // MMAs still in flight after a timeout end before TMEM is freed
  if (mma_warp && lane == 0) {
    mma_commit(fin);
    if (!mbar_wait(fin, 0, TC_WAIT_LIMIT)) *fail = 1;
  }
  tc_fence_before();
  __syncthreads();
  if (*fail && tid == 0) atomicExch(g.err, 1);
  if (warp == 0) tmem_free(tmem, 512);
}

// |x| maxima of the columns of an operand (FP64 bit patterns, atomic max;
// the target starts at zero)
template <typename T>
__global__ void k_oz_colmax(const T *__restrict__ a, long long lda, long long rows, long long span,
                            unsigned long long *__restrict__ out) {
  const int c = blockIdx.x;
  const long long rb = (long long)blockIdx.y * span, re = min(rows, rb + span);
  const T *col = a + (long long)c * lda;
  double m = 0.0;
  for (long long r = rb + threadIdx.x; r < re; r += blockDim.x) {
    const double x = fabs((double)__ldg(col + r));
    m = (x > m || x != x) ? x : m;  // NaN propagates
  }
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) {
    const double y = __shfl_xor_sync(0xffffffffu, m, o);
    m = (y > m || y != y) ? y : m;
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = (red[w] > m || red[w] != red[w]) ? red[w] : m;
    atomicMax(out + c, (unsigned long long)__double_as_longlong(m));
  }
}

// sum of the chunk partials in fixed order; symmetric tasks take the
// transposed element where its tile was not computed; mirror writes C^T too
__global__ void k_oz_reduce(OzArgs g, int ldo, double *__restrict__ outbuf) {
  const OzTask &tk = g.t[blockIdx.y];
  const long long kk = (long long)tk.ka * tk.kb;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < kk; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % tk.ka), j = (int)(q / tk.ka);
    int si = i, sj = j;
    if (tk.sym && i / 64 > j / 64) {  // below the computed 64 x 64 blocks: the transpose
      si = j;
      sj = i;
    }
    const double *pp = g.part + tk.part0 + (long long)sj * tk.ka + si;
    double s = 0.0;
    for (int sp = 0; sp < tk.nsp; ++sp) s += pp[(long long)sp * kk];
    double *o = outbuf + (long long)tk.out * ldo * ldo;
    o[(long long)(tk.j0 + j) * ldo + tk.i0 + i] = s;
    if (tk.mirror) o[(long long)(tk.i0 + i) * ldo + tk.j0 + j] = s;
  }
}

static int oz_sm_count(bdgd_ctx *c) {
  int nsm = 148;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device) != cudaSuccess || nsm < 1) {
    cudaGetLastError();
    nsm = 148;
  }
  return nsm;
}

// Real FP64 task list on the tensor cores; BDGD_ERR_UNSUPPORTED (nothing
// launched) for layouts outside the kernel's limits.
template <typename T>
static int gram_oz_launch(bdgd_ctx *c, const OzArgs &g, long long chunk, int nunits, int nsm) {
  if (!bdgd_capturing)
    BDGD_CK(cudaFuncSetAttribute(k_gram_oz<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, oz_smem_bytes<T>()));
  bdgd_count_launch();
  k_gram_oz<T><<<(unsigned)(nunits < nsm ? nunits : nsm), OZ_BLOCK, oz_smem_bytes<T>(), c->stream>>>(g, chunk, nunits);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}

// prec: BDGD_F64 (FP64 blocks) or BDGD_F32 (FP32 blocks, FP64 results)
extern "C" int bdgd_gram_oz(bdgd_ctx *c, int prec, int ntask, const bdgd_gram_task *tasks, int ldo, double *d_out) {
  if (ntask <= 0) return BDGD_OK;
  if (ntask > OZ_MAXT || (prec != BDGD_F64 && prec != BDGD_F32)) return BDGD_ERR_UNSUPPORTED;
  const uint64_t vec = prec == BDGD_F64 ? 2 : 4;  // elements per 16 bytes
  long long maxrows = 0;
  for (int i = 0; i < ntask; ++i) {
    const bdgd_gram_task &s = tasks[i];
    if (((uintptr_t)s.a | (uintptr_t)s.b) % 16 || s.lda % vec || s.ldb % vec || s.ka <= 0 || s.kb <= 0 ||
        s.rows % 32)
      return BDGD_ERR_UNSUPPORTED;
    if ((long long)s.rows > maxrows) maxrows = (long long)s.rows;
  }
  OzArgs g;
  memset(&g, 0, sizeof g);
  g.nt = ntask;
  // tasks in order of decreasing rows (so that chunk counts decrease)
  int order[OZ_MAXT];
  for (int i = 0; i < ntask; ++i) order[i] = i;
  for (int i = 1; i < ntask; ++i)
    for (int j = i; j > 0 && tasks[order[j]].rows > tasks[order[j - 1]].rows; --j) {
      const int t = order[j];
      order[j] = order[j - 1];
      order[j - 1] = t;
    }
  // unique operands (pointer, leading dimension, rows, columns) -> column maxima
  struct Op {
    const void *p;
    long long ld, rows;
    int k, off;
  } ops[2 * OZ_MAXT];
  int nops = 0, moff = 0;
  auto op_index = [&](const void *p, uint64_t ld, uint64_t rows, int k) -> int {
    for (int i = 0; i < nops; ++i)
      if (ops[i].p == p && ops[i].ld == (long long)ld && ops[i].rows == (long long)rows && ops[i].k == k)
        return ops[i].off;
    ops[nops] = {p, (long long)ld, (long long)rows, k, moff};
    moff += k;
    return ops[nops++].off;
  };
  for (int q = 0; q < ntask; ++q) {
    const bdgd_gram_task &s = tasks[order[q]];
    OzTask &t = g.t[q];
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
    t.sym = s.sym && s.ka == s.kb;  // a symmetric result: the 64 x 64 blocks on and above the diagonal
    t.mirror = s.mirror;
    t.ma = op_index(s.a, s.lda, s.rows, s.ka);
    t.mb = op_index(s.b, s.ldb, s.rows, s.kb);
  }
  // 64 x 64 output blocks (task, A slice, B tile), grouped by B operand and B
  // tile (operands are identified by their column-maxima slot, which is
  // unique per pointer, leading dimension, rows and columns); consecutive
  // blocks of a group share one 128 x 64 tile
  struct Blk {
    int t, s, jb, key;
  };
  static thread_local Blk blk[OZ_MAXTILES * 2];
  int nblk = 0;
  for (int q = 0; q < ntask; ++q) {
    const OzTask &t = g.t[q];
    const int sa = (t.ka + 63) / 64, tb = (t.kb + 63) / 64;
    for (int jb = 0; jb < tb; ++jb)
      for (int sl = 0; sl < sa; ++sl) {
        if (t.sym && sl > jb) continue;
        if (nblk >= OZ_MAXTILES * 2) return BDGD_ERR_UNSUPPORTED;
        blk[nblk++] = {q, sl, jb, t.mb * 1024 + jb};
      }
  }
  // stable order by key (tasks already in order of decreasing rows)
  for (int i = 1; i < nblk; ++i)
    for (int j = i; j > 0 && blk[j].key < blk[j - 1].key; --j) {
      const Blk x = blk[j];
      blk[j] = blk[j - 1];
      blk[j - 1] = x;
    }
  int tiles = 0;
  for (int i = 0; i < nblk;) {
    if (tiles >= OZ_MAXTILES) return BDGD_ERR_UNSUPPORTED;
    OzTile &p = g.p[tiles++];
    p.ta[0] = (short)blk[i].t;
    p.sa[0] = (short)blk[i].s;
    p.tb = (short)blk[i].t;
    p.jb = (short)blk[i].jb;
    if (i + 1 < nblk && blk[i + 1].key == blk[i].key) {
      p.ta[1] = (short)blk[i + 1].t;
      p.sa[1] = (short)blk[i + 1].s;
      i += 2;
    } else {
      p.ta[1] = -1;
      p.sa[1] = 0;
      i += 1;
    }
  }
  g.np = tiles;
  // row chunks: at most OZ_CHUNK rows (int32 exactness), enough units to fill the GPU
  const int nsm = oz_sm_count(c);
  long long nsplit = (2LL * nsm + tiles - 1) / tiles;
  const long long minsplit = (maxrows + OZ_CHUNK - 1) / OZ_CHUNK;
  const long long maxsplit = (maxrows + 255) / 256;
  if (nsplit < minsplit) nsplit = minsplit;
  if (nsplit > maxsplit) nsplit = maxsplit > minsplit ? maxsplit : minsplit;
  if (nsplit < 1) nsplit = 1;
  long long chunk = (maxrows + nsplit - 1) / nsplit;
  chunk = (chunk + 31) / 32 * 32;
  long long off = 0;
  for (int q = 0; q < ntask; ++q) {
    OzTask &t = g.t[q];
    t.nsp = (int)((t.rows + chunk - 1) / chunk);
    t.part0 = off;
    off += (long long)t.nsp * t.ka * t.kb;
  }
  int nunits = 0;
  for (int i = 0; i < tiles; ++i) {
    g.p[i].nsp = g.t[g.p[i].tb].nsp;
    nunits += g.p[i].nsp;
  }
  // tiles in order of decreasing chunk count (stable)
  for (int i = 1; i < tiles; ++i)
    for (int j = i; j > 0 && g.p[j].nsp > g.p[j - 1].nsp; --j) {
      const OzTile x = g.p[j];
      g.p[j] = g.p[j - 1];
      g.p[j - 1] = x;
    }
  int rc = bdgd_ensure(c->stream, (void **)&c->gram_part, &c->gram_part_bytes, sizeof(double) * off);
  if (rc) return rc;
  // oz_buf: the error flag (16 bytes), then the column maxima
  const size_t mbytes = 16 + sizeof(unsigned long long) * (size_t)moff;
  rc = bdgd_ensure(c->stream, &c->oz_buf, &c->oz_buf_bytes, mbytes);
  if (rc) return rc;
  unsigned long long *colmax = (unsigned long long *)((char *)c->oz_buf + 16);
  g.colmax = colmax;
  g.err = (int *)c->oz_buf;
  g.part = c->gram_part;
  BDGD_CK(cudaMemsetAsync(c->oz_buf, 0, mbytes, c->stream));
  for (int i = 0; i < nops; ++i) {
    const long long span = 65536;
    const unsigned ny = (unsigned)((ops[i].rows + span - 1) / span);
    bdgd_count_launch();
    const dim3 grid((unsigned)ops[i].k, ny ? ny : 1);
    if (prec == BDGD_F64)
      k_oz_colmax<double><<<grid, 256, 0, c->stream>>>((const double *)ops[i].p, ops[i].ld, ops[i].rows, span,
                                                       colmax + ops[i].off);
    else
      k_oz_colmax<float><<<grid, 256, 0, c->stream>>>((const float *)ops[i].p, ops[i].ld, ops[i].rows, span,
                                                      colmax + ops[i].off);
    BDGD_CK(cudaGetLastError());
  }
  rc = prec == BDGD_F64 ? gram_oz_launch<double>(c, g, chunk, nunits, nsm)
                        : gram_oz_launch<float>(c, g, chunk, nunits, nsm);
  if (rc) return rc;
  bdgd_count_launch();
  k_oz_reduce<<<dim3(32, ntask), 256, 0, c->stream>>>(g, ldo, d_out);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}

// the error flag of the last tensor-core Gram or update on this context (1:
// a wait on the tensor core timed out); reads it synchronously
extern "C" int bdgd_gram_oz_error(bdgd_ctx *c) {
  if (!c->oz_buf || c->oz_buf_bytes < 16) return 0;
  int h = 0;
  if (cudaMemcpyAsync(&h, c->oz_buf, sizeof h, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess)
    return -1;
  return h;
}

// ---------------------------------------------------------------------------
// Basis update on the integer tensor cores: Y = alpha sum_b S_b C_b + beta Y
// for real FP64 blocks (the interface of bdgd_block_update).
//
// With S = [S_1 .. S_nt] (n x K) and C stacked (K x ncol):  Y = (S D^-1)(D C)
// with D = diag(2^S_j) from the column maxima of S: every column of S D^-1
// is written in the digits above with its own power of two, and each column
// c of D C gets its own power of two f_c, so that
//   Y_rc = 2^(f_c - 110) sum_{t,u} 256^(t+u) sum_j d_t(X_rj) d_u(X'_jc);
// the error is about K 2^-55 of the largest term, that of an FP64 dot
// product of length K.  Persistent CTAs: each owns one (output, 64-column
// tile), keeps the digits of its D C block in shared memory and walks row
// tiles of 128 rows (the CTAs that share a row tile run together, so S comes
// from L2 after the first); S streams in by cp.async (32 columns x 128 rows
// per K step), the next row tile's first steps during the current flush.
// ---------------------------------------------------------------------------
#define OZU_MAXK 192                       // K = sum k_b limit (6 steps of 32)
#define OZU_RAW_LD 1040                    // bytes per raw column (128 rows + 16 bytes)
#define OZU_RAW_STAGE (32 * OZU_RAW_LD)
#define OZU_SMEM_C (6 * OZ_ND * 64 * 32)   // D C digits of up to 6 K steps
#define OZU_SMEM_A (2 * OZ_ND * 128 * 32)  // two stages of S digits
#define OZU_SMEM (OZU_SMEM_C + OZU_SMEM_A + 2 * OZU_RAW_STAGE + 8192)

struct OzuTerm {
  const double *s, *c;
  int k, ldc, nst;  // columns, C leading dim, K steps of 32
  int mx;           // offset of the column maxima of s
};
struct OzuOut {
  double *y;
  int ncol, nterm;
  double alpha, beta;
  OzuTerm t[3];
  int nst, ktot;
};
struct OzuArgs {
  OzuOut o[4];
  int nout;
  int ct_out[64], ct_col[64], nct;  // (output, 64-column tile) pairs
  long long n, ld, nrt;
  const unsigned long long *colmax;
  int *err;
};

// K step `st` of output o: its term b and first column j0 inside the term
__device__ __forceinline__ void ozu_step_term(const OzuOut &o, int st, int &b, int &j0) {
  b = 0;
  while (b + 1 < o.nterm && st >= o.t[b].nst) {
    st -= o.t[b].nst;
    ++b;
  }
  j0 = 32 * st;
}

// copies of K step st (32 columns x 128 rows of S) into a raw stage, by all
// threads in 16-byte pieces (64 per column), then one commit group
__device__ __forceinline__ void ozu_issue_step(const OzuOut &o, int st, long long r0, long long ld, uint8_t *raw,
                                               int tid) {
  int b, j0;
  ozu_step_term(o, st, b, j0);
  const OzuTerm &tm = o.t[b];
  const int nj = min(32, tm.k - j0);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int seg = tid + OZ_THREADS * k;
    const int j = seg >> 6, piece = seg & 63;
    if (j < nj) cp_async16(raw + j * OZU_RAW_LD + piece * 16, tm.s + (long long)(j0 + j) * ld + r0 + 2 * piece);
  }
  cp_async_commit();
}

__global__ void __launch_bounds__(OZ_THREADS, 1) k_update_oz(OzuArgs u) {
  extern __shared__ __align__(1024) uint8_t oz_smem[];
  uint8_t *cdig = oz_smem;                                   // [step][digit][64 x 32]
  uint8_t *adig = oz_smem + OZU_SMEM_C;                      // [stage][digit][128 x 32]
  uint8_t *raw0 = adig + OZU_SMEM_A;                         // [stage][32 columns][128 rows]
  double *sS = reinterpret_cast<double *>(raw0 + 2 * OZU_RAW_STAGE);  // [192] 2^(55 - S_j)
  double *cm = sS + OZU_MAXK;                                // [8][64] partial column maxima of D C
  int *fexp = reinterpret_cast<int *>(cm + 512);             // [64]
  int *fbad = fexp + 64;                                     // [64]
  double *fsc = reinterpret_cast<double *>(fbad + 64);       // [64] 2^(55 - f_c)
  uint64_t *mdone = reinterpret_cast<uint64_t *>(fsc + 64);  // [2] MMAs of a digit stage done
  uint32_t *tslot = reinterpret_cast<uint32_t *>(mdone + 2);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ct = blockIdx.x % u.nct;
  const int rstep = gridDim.x / u.nct;  // CTAs per (output, column tile)
  const int rfirst = blockIdx.x / u.nct;
  const OzuOut &o = u.o[u.ct_out[ct]];
  const int c0 = 64 * u.ct_col[ct];
  const long long n = u.n, ld = u.ld;
  const int nst = o.nst;

  if (warp == 0) tmem_alloc(tslot, 512);
  if (tid == 0) {
    for (int i = 0; i < 2; ++i) mbar_init(&mdone[i], 1);
    mbar_init_fence();
  }
  // the first row tile's first two K steps start loading now
  long long G = 0;  // K steps issued so far, over this CTA's row tiles
  auto issue_global = [&](long long Gs) {
    const long long rt = rfirst + (Gs / nst) * rstep;
    if (rt < u.nrt) ozu_issue_step(o, (int)(Gs % nst), rt * 128, ld, raw0 + (Gs & 1) * OZU_RAW_STAGE, tid);
    else cp_async_commit();
  };
  issue_global(0);
  issue_global(1);
  // column scales of S: 2^(55 - S_j) per stacked column j; a non-finite
  // column makes the whole output NaN through D C below
  for (int j = tid; j < OZU_MAXK; j += blockDim.x) {
    double sc = 1.0;
    int E = 0;
    bool fin = true;
    int b = 0, jj = j;
    while (b < o.nterm && jj >= o.t[b].k) {
      jj -= o.t[b].k;
      ++b;
    }
    if (b < o.nterm) oz_scale(u.colmax[o.t[b].mx + jj], sc, E, fin);
    sS[j] = fin ? sc : __longlong_as_double(0x7ff8000000000000LL);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  // D C for this CTA's 64 columns: (D C)_jc = C_jc 2^S_j = C_jc 2^55 / sS_j,
  // exact; column maxima, then the digits of every K step
  const int cc = tid & 63, cp = tid >> 6;  // column, part 0..7
  const bool vc = c0 + cc < o.ncol;
  {
    double m = 0.0;
    if (vc) {
      int jg = 0;
      for (int b = 0; b < o.nterm; ++b) {
        const OzuTerm &tm = o.t[b];
        const double *col = tm.c + (long long)(c0 + cc) * tm.ldc;
        for (int j = cp; j < tm.k; j += 8) {
          const double x = fabs(col[j] * 0x1p55 / sS[jg + j]);
          m = (x > m || x != x) ? x : m;
        }
        jg += tm.k;
      }
    }
    cm[cp * 64 + cc] = m;
  }
  __syncthreads();
  if (tid < 64) {
    double mc = 0.0;
    for (int q = 0; q < 8; ++q) {
      const double a = cm[q * 64 + tid];
      mc = (a > mc || a != a) ? a : mc;
    }
    double fs = 1.0;
    int F = 0;
    bool fin = true;
    oz_scale((unsigned long long)__double_as_longlong(mc), fs, F, fin);
    fexp[tid] = F;
    fbad[tid] = !fin;
    fsc[tid] = fs;
  }
  __syncthreads();
  {  // thread (cc, cp): K rows [4 cp, 4 cp + 4) of every step
    const double fs = fsc[cc];
    const int off = (cc & 7) * 16 + (cc >> 3) * 256 + (cp >> 2) * 128 + (cp & 3) * 4;
    int st = 0, jg = 0;
    for (int b = 0; b < o.nterm; ++b) {
      const OzuTerm &tm = o.t[b];
      const double *col = tm.c + (long long)(c0 + cc) * tm.ldc;
      for (int s = 0; s < tm.nst; ++s, ++st) {
        double v[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int j = 32 * s + 4 * cp + q;
          v[q] = (vc && j < tm.k) ? col[j] * 0x1p55 / sS[jg + j] : 0.0;
        }
        uint32_t w[OZ_ND];
        oz_digits4(v[0], v[1], v[2], v[3], fs, w);
#pragma unroll
        for (int t = 0; t < OZ_ND; ++t) *reinterpret_cast<uint32_t *>(cdig + (st * OZ_ND + t) * 2048 + off) = w[t];
      }
      jg += tm.k;
    }
  }
  __syncthreads();

  // S digits role: row rr of the tile, K columns [8 q4, 8 q4 + 8) of a step
  const int rr = tid & 127, q4 = tid >> 7;
  const int offA = (rr & 7) * 16 + (rr >> 3) * 256 + (q4 >> 1) * 128 + (q4 & 1) * 8;
  uint32_t mph[2] = {0u, 0u};
  int failed = 0;
  for (long long rt = rfirst; rt < u.nrt && !failed; rt += rstep) {
    const long long r0 = rt * 128;
    for (int st = 0; st < nst; ++st, ++G) {
      const int s = st & 1;
      const uint8_t *raw = raw0 + (G & 1) * OZU_RAW_STAGE;
      uint8_t *dig = adig + s * (OZ_ND * 4096);
      cp_async_wait<1>();  // this thread's copies of step G are done (the newest group is G + 1)
      bool ok = true;
      if (st >= 2) {
        ok = mbar_wait(&mdone[s], mph[s], TC_WAIT_LIMIT);
        mph[s] ^= 1u;
      }
      failed = __syncthreads_or(!ok);
      if (failed) break;
      {
        int b, j0;
        ozu_step_term(o, st, b, j0);
        int jg = j0;
        for (int q = 0; q < b; ++q) jg += o.t[q].k;
        const int kb = o.t[b].k;
        double v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int j = 8 * q4 + q;
          v[q] = (j0 + j < kb) ? *reinterpret_cast<const double *>(raw + j * OZU_RAW_LD + rr * 8) * sS[jg + j] : 0.0;
        }
        uint32_t w0[OZ_ND], w1[OZ_ND];
        oz_digits4(v[0], v[1], v[2], v[3], 1.0, w0);
        oz_digits4(v[4], v[5], v[6], v[7], 1.0, w1);
#pragma unroll
        for (int t = 0; t < OZ_ND; ++t) *reinterpret_cast<uint2 *>(dig + t * 4096 + offA) = make_uint2(w0[t], w1[t]);
      }
      fence_async_smem();
      __syncthreads();
      if (tid == 0) {
        tc_fence_after();
        const uint32_t id = idesc_i8(64);
        const uint32_t abase = smem_u32(dig), bbase = smem_u32(cdig + st * OZ_ND * 2048);
#pragma unroll
        for (int t = 0; t < OZ_ND; ++t)
#pragma unroll
          for (int q = 0; q < OZ_ND; ++q) {
            const int D = t + q;
            if (D < OZ_DMIN) continue;
            const int first_t = D - (OZ_ND - 1) > 0 ? D - (OZ_ND - 1) : 0;
            mma_i8(tmem + (uint32_t)((D - OZ_DMIN) * 64), smem_desc(abase + t * 4096),
                   smem_desc(bbase + q * 2048), id, (st > 0 || t > first_t) ? 1u : 0u);
          }
        mma_commit(&mdone[s]);
      }
      // the raw stage of step G is consumed: refill it with step G + 2 (maybe
      // of the next row tile, loading while this tile is flushed)
      issue_global(G + 2);
    }
    if (failed) break;
    {  // the last commit of each digit stage of this row tile
      bool ok = true;
      for (int k = nst >= 2 ? nst - 2 : 0; k < nst && ok; ++k) {
        const int s = k & 1;
        ok = mbar_wait(&mdone[s], mph[s], TC_WAIT_LIMIT);
        mph[s] ^= 1u;
      }
      failed = __syncthreads_or(!ok);
      if (failed) break;
    }
    tc_fence_after();
    // flush: warp w has TMEM lanes (rows) 32 (w % 4).., output columns 16 (w / 4)..
    const int row = 32 * (warp & 3) + lane;
    const long long r = r0 + row;
    const int cl = 16 * (warp >> 2);
    double acc[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) acc[q] = 0.0;
#pragma unroll
    for (int d = 0; d < OZ_NDIAG; ++d) {
      int32_t v[16];
      tmem_ld16(tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(d * 64 + cl), v);
      const double w = ldexp(1.0, 8 * (d + OZ_DMIN) - 2 * OZ_P);
#pragma unroll
      for (int q = 0; q < 16; ++q) acc[q] = fma((double)v[q], w, acc[q]);
    }
    if (r < n) {
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const int c = c0 + cl + q;
        if (c < o.ncol) {
          double val = o.alpha * ldexp(acc[q], fexp[cl + q]);
          if (fbad[cl + q]) val = __longlong_as_double(0x7ff8000000000000LL);
          double *yp = o.y + (long long)c * ld + r;
          if (o.beta != 0.0) val += o.beta * *yp;
          *yp = val;
        }
      }
    }
    // TMEM reads done before the next row tile's MMAs overwrite it
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  }
  cp_async_wait<0>();
  if (failed && tid == 0) atomicExch(u.err, 1);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_free(tmem, 512);
}

// Real FP64 block update on the tensor cores (bdgd_block_update's interface);
// BDGD_ERR_UNSUPPORTED (nothing launched) outside its limits.
extern "C" int bdgd_block_update_oz(bdgd_ctx *c, uint64_t n, uint64_t ld, int nout, const bdgd_update_out *outs) {
  if (nout <= 0 || n == 0) return BDGD_OK;
  if (nout > 4 || ld < n || n % 128 || ld % 2) return BDGD_ERR_UNSUPPORTED;
  OzuArgs u;
  memset(&u, 0, sizeof u);
  u.n = (long long)n;
  u.ld = (long long)ld;
  u.nout = nout;
  struct Op {
    const double *p;
    int k, off;
  } ops[12];
  int nops = 0, moff = 0;
  for (int i = 0; i < nout; ++i) {
    const bdgd_update_out &s = outs[i];
    if (s.nterm < 0 || s.nterm > 3 || s.ncol < 0 || ((uintptr_t)s.y % 8)) return BDGD_ERR_UNSUPPORTED;
    OzuOut &o = u.o[i];
    o.y = (double *)s.y;
    o.ncol = s.ncol;
    o.alpha = s.alpha;
    o.beta = s.beta;
    for (int b = 0; b < s.nterm; ++b) {
      if (s.term[b].k <= 0) continue;
      if (((uintptr_t)s.term[b].s % 16) || s.term[b].ldc < s.term[b].k || ((uintptr_t)s.term[b].c % 8))
        return BDGD_ERR_UNSUPPORTED;
      OzuTerm &t = o.t[o.nterm++];
      t.s = (const double *)s.term[b].s;
      t.c = s.term[b].c;
      t.k = s.term[b].k;
      t.ldc = s.term[b].ldc;
      t.nst = (t.k + 31) / 32;
      o.nst += t.nst;
      o.ktot += t.k;
      int found = -1;
      for (int q = 0; q < nops; ++q)
        if (ops[q].p == t.s && ops[q].k == t.k) found = ops[q].off;
      if (found < 0) {
        ops[nops] = {t.s, t.k, moff};
        found = moff;
        moff += t.k;
        nops++;
      }
      t.mx = found;
    }
    if (o.nst > 6 || o.ktot > OZU_MAXK) return BDGD_ERR_UNSUPPORTED;
    for (int j = 0; o.nterm > 0 && j * 64 < s.ncol; ++j) {  // no terms: Y untouched
      if (u.nct == 64) return BDGD_ERR_UNSUPPORTED;
      u.ct_out[u.nct] = i;
      u.ct_col[u.nct] = j;
      u.nct++;
    }
  }
  if (u.nct == 0) return BDGD_OK;
  u.nrt = (long long)n / 128;
  const size_t mbytes = 16 + sizeof(unsigned long long) * (size_t)moff;
  int rc = bdgd_ensure(c->stream, &c->oz_buf, &c->oz_buf_bytes, mbytes);
  if (rc) return rc;
  u.err = (int *)c->oz_buf;
  unsigned long long *colmax = (unsigned long long *)((char *)c->oz_buf + 16);
  u.colmax = colmax;
  BDGD_CK(cudaMemsetAsync(c->oz_buf, 0, mbytes, c->stream));
  for (int i = 0; i < nops; ++i) {
    const long long span = 65536;
    const unsigned ny = (unsigned)(((long long)n + span - 1) / span);
    bdgd_count_launch();
    k_oz_colmax<double><<<dim3((unsigned)ops[i].k, ny), 256, 0, c->stream>>>(ops[i].p, (long long)ld, (long long)n, span,
                                                                    colmax + ops[i].off);
    BDGD_CK(cudaGetLastError());
  }
  // persistent CTAs: the same count for every (output, column tile), at most one per SM
  const int nsm = oz_sm_count(c);
  int per = nsm / u.nct;
  if (per < 1) per = 1;
  if ((long long)per > u.nrt) per = (int)u.nrt;
  if (!bdgd_capturing)
    BDGD_CK(cudaFuncSetAttribute(k_update_oz, cudaFuncAttributeMaxDynamicSharedMemorySize, OZU_SMEM));
  bdgd_count_launch();
  k_update_oz<<<(unsigned)(per * u.nct), OZ_THREADS, OZU_SMEM, c->stream>>>(u);
  BDGD_CK(cudaGetLastError());
  return BDGD_OK;
}
