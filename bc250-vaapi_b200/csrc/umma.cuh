// umma.cuh - tcgen05 (5th-generation tensor core) building blocks for sm_100a:
// shared-memory matrix descriptors in the canonical K-major no-swizzle layout,
// the kind::f16 (BF16) and kind::f8f6f4 (E4M3) instruction descriptors, MMA
// issue/commit, bounded mbarrier waits, plain 2-D TMA loads and TMEM loads.
//
// Canonical K-major no-swizzle layout of an operand tile of `rows` rows
// (rows a multiple of 8): core matrices of 8 rows x 16 bytes (8 BF16), rows
// of a core matrix 16 B apart, 8-row groups 128 B apart (stride byte offset),
// 8-element K chunks rows*16 B apart (leading byte offset):
//   element (r, k) at ((k/8) * rows/8 + r/8) * 64 + (r%8) * 8 + k%8.
#pragma once
#include <cuda_bf16.h>

#include "common.cuh"

namespace b200enc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__host__ __device__ constexpr int canon_off(int r, int k, int rows) {
  return ((k >> 3) * (rows >> 3) + (r >> 3)) * 64 + (r & 7) * 8 + (k & 7);
}

// Shared-memory matrix descriptor, K-major, no swizzle (layout type 0),
// Blackwell version 1: start address, leading byte offset (between K
// chunks) and stride byte offset (between 8-row groups), all >> 4.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;  // version
  return d;
}

// Descriptor of the 16-wide K step starting at element k0 of a canonical
// tile of `rows` rows at shared address base.
__device__ __forceinline__ uint64_t canon_desc(uint32_t base, int rows, int k0) {
  return umma_desc(base + (uint32_t)((k0 >> 3) * (rows >> 3) * 128), (uint32_t)rows * 16u, 128u);
}

// Instruction descriptor of kind::f16: D F32, A and B BF16, both K-major.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
  return (1u << 4)                        // c_format F32
         | (1u << 7)                      // a_format BF16
         | (1u << 10)                     // b_format BF16
         | ((uint32_t)(N >> 3) << 17)     // n_dim
         | ((uint32_t)(M >> 4) << 24);    // m_dim
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc)
      : "memory");
}

// The same layout for 8-bit operands (FP8 E4M3): a core matrix row is 16
// bytes = 16 elements, so K chunks are 16 elements wide:
//   element (r, k) at byte ((k/16) * rows/8 + r/8) * 128 + (r%8) * 16 + k%16.
__host__ __device__ constexpr int canon_off8(int r, int k, int rows) {
  return ((k >> 4) * (rows >> 3) + (r >> 3)) * 128 + (r & 7) * 16 + (k & 15);
}

// Descriptor of the 32-wide K step (one kind::f8f6f4 MMA) starting at
// element k0 (a multiple of 16) of an 8-bit canonical tile.
__device__ __forceinline__ uint64_t canon_desc8(uint32_t base, int rows, int k0) {
  return umma_desc(base + (uint32_t)((k0 >> 4) * (rows >> 3) * 128), (uint32_t)rows * 16u, 128u);
}

// Instruction descriptor of kind::f8f6f4: D F32, A and B E4M3 (format 0),
// both K-major.
__host__ __device__ constexpr uint32_t umma_idesc_e4m3(int M, int N) {
  return (1u << 4)                        // c_format F32
         | (0u << 7)                      // a_format E4M3
         | (0u << 10)                     // b_format E4M3
         | ((uint32_t)(N >> 3) << 17)     // n_dim
         | ((uint32_t)(M >> 4) << 24);    // m_dim
}

__device__ __forceinline__ void umma_f8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Arrive on an mbarrier and add `bytes` to the transaction count its
// current phase waits for (the issuing thread of a TMA copy).
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// 2-D tiled TMA load of the tensor map's box at element coordinates (x, y)
// into shared memory, completing `bar`'s transaction count. The map lives in
// kernel parameter space (__grid_constant__). Plain load: no cluster
// multicast. x times the element size must be a multiple of 16 bytes.
__device__ __forceinline__ void tma_load_2d(void* dst, const void* tmap, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// Bounded wait on an mbarrier phase; false after ~max_ns without completion.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, uint64_t max_ns) {
  const uint32_t a = smem_u32(bar);
  const uint64_t t0 = global_ns();
  for (;;) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(phase)
        : "memory");
    if (ok) return true;
    if (global_ns() - t0 > max_ns) return false;
  }
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
// 16 accumulator columns of TMEM lane 32*quad + lane (a warp reads its own
// lane quadrant), columns col .. col+15; waits for the load.
__device__ __forceinline__ void tmem_row16(uint32_t tmem, int quad, int col, uint32_t (&v)[16]) {
  tmem_ld16(tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)col, v);
  tmem_wait_ld();
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Warp-wide TMEM allocation of `cols` columns (a power of two >= 32); the
// address is written to *dst in shared memory.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(cols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

}  // namespace b200enc
