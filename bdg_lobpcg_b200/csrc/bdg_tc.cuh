// bdg_tc.cuh -- Blackwell (sm_100a) tensor-core building blocks: tcgen05 MMA
// with int8 operands in shared memory and int32 accumulators in tensor memory
// (TMEM), the mbarrier handshake with the asynchronous tensor core, and TMEM
// loads.  Inline PTX; the descriptor formats follow the sm100 UMMA
// descriptors (shared-memory matrix descriptor and instruction descriptor).
//
// Operand layout in shared memory ("K-major, no swizzle"): a tile of R rows
// (M or N) by 32 bytes of K (one kind::i8 MMA step) is stored as 8-row core
// matrices of 8 x 16 bytes (128 contiguous bytes, row r_in at r_in * 16);
// the two 16-byte K halves of a row group are adjacent (leading byte offset
// 128) and row groups follow each other every 256 bytes (stride byte offset):
//   byte(r, k) = (r % 8) * 16 + (r / 8) * 256 + (k / 16) * 128 + k % 16.
#pragma once
#include <cstdint>

namespace bdgtc {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// offset of int8 element (row r, k in [0, 32)) inside a K-major tile
__device__ __forceinline__ int tile_off(int r, int k) {
  return (r & 7) * 16 + (r >> 3) * 256 + (k >> 4) * 128 + (k & 15);
}

// shared-memory matrix descriptor: start address, LBO = 128 B, SBO = 256 B,
// version 1 (sm100), no swizzle, base offset 0
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)((128 >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((256 >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// instruction descriptor: kind::i8, A and B signed int8, D int32, both
// K-major, M = 128, N = n (multiple of 16, 16..256)
__host__ __device__ constexpr uint32_t idesc_i8(int n) {
  return (2u << 4)                        // D format: S32
         | (1u << 7)                      // A format: signed 8-bit
         | (1u << 10)                     // B format: signed 8-bit
         | ((uint32_t)(n >> 3) << 17)     // N >> 3
         | ((uint32_t)(128 >> 4) << 24);  // M >> 4
}

// D[tmem] (+)= A[smem] * B[smem]^T; accumulate != 0 adds to D
__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

// arrive on the mbarrier once every MMA issued so far by this thread is done
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// bounded wait for phase `parity` of the mbarrier; returns false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, long long max_iter) {
  const uint32_t a = smem_u32(bar);
  for (long long i = 0; i < max_iter; ++i) {
    uint32_t done = 0;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 16-byte asynchronous copy global -> shared (L2 only), grouped completion
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// one arrival of this thread on the mbarrier (release: its prior writes are
// visible to the thread that observes the phase)
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// generic-proxy shared-memory writes become visible to the tensor core
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// TMEM allocation by one full warp; the base address is written to *slot
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols) : "memory");
}

// 16 consecutive 32-bit TMEM columns of this warp's 32 lanes (thread = lane)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, int32_t (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = (int32_t)r[i];
}

}  // namespace bdgtc
