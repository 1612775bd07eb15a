// bdg_tc.cu -- tensor-core (tcgen05, sm_100a) kernels of the solver's FP64
// contractions.
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
  return bdgd_check(cudaGetLastError(), "k_tc_i8_gemm");
}
