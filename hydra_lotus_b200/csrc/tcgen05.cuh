// SPDX-License-Identifier: Apache-2.0
// Blackwell tensor-core primitives used by the radiance cache's network:
// tensor-memory allocation, tcgen05.mma of BF16 operands in shared memory
// with an FP32 accumulator in tensor memory, completion through an
// mbarrier, and accumulator loads back to registers. One CTA (cta_group::1),
// operands in the no-swizzle canonical layout.
//
// Operand layout. A K-major operand tile of R rows by 64 BF16 columns is
// stored as 8x8 "core matrices" (8 rows of 16 contiguous bytes, 128 bytes
// each): element (r, c) sits at byte
//   (r / 8) * 1024 + (c / 8) * 128 + (r % 8) * 16 + (c % 8) * 2,
// so core matrices adjacent along K are 128 bytes apart (the leading byte
// offset) and adjacent 8-row groups 1024 bytes apart (the stride byte
// offset). The same bytes read as an MN-major operand (rows become K,
// columns M or N) have core matrices adjacent along M/N 128 bytes apart and
// along K 1024 bytes apart.
#pragma once

#include <cstdint>

namespace lotus {
namespace tc {

constexpr uint32_t kTileBytes64 = 128 * 64 * 2;  // 128 x 64 BF16 tile

__device__ __forceinline__ uint32_t tile_offset(uint32_t row, uint32_t col) {
  return (row >> 3) * 1024u + (col >> 3) * 128u + (row & 7u) * 16u + (col & 7u) * 2u;
}

// The same layout for a tile of `cols` (a multiple of 8) columns: 8-row
// groups are cols * 16 bytes apart.
__host__ __device__ __forceinline__ uint32_t tile_offset_n(uint32_t row, uint32_t col, uint32_t cols) {
  return (row >> 3) * (cols * 16u) + (col >> 3) * 128u + (row & 7u) * 16u + (col & 7u) * 2u;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (no swizzle, version 1): start address,
// leading and stride byte offsets, all in 16-byte units.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// K-major view of a tile of `cols` columns at K offset k (a multiple of 16).
__device__ __forceinline__ uint64_t desc_k_major(uint32_t base, uint32_t k, uint32_t cols = 64) {
  return smem_desc(base + (k >> 3) * 128u, 128u, cols * 16u);
}

// MN-major view of the same storage at K offset k, K running over rows.
__device__ __forceinline__ uint64_t desc_mn_major(uint32_t base, uint32_t k, uint32_t cols = 64) {
  return smem_desc(base + (k >> 3) * (cols * 16u), cols * 16u, 128u);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B,
// each K-major (0) or MN-major (1), shape M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t m, uint32_t n, uint32_t a_mn_major,
    uint32_t b_mn_major) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (a_mn_major << 15) | (b_mn_major << 16) | ((n >> 3) << 17) |
         ((m >> 4) << 24);
}

// D (+)= A * B, issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
    uint32_t accumulate) {
  const uint32_t no_mask = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n"
      :
      : "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(no_mask)
      : "memory");
}

// Arrives on the mbarrier once every MMA this thread issued has completed.
__device__ __forceinline__ void commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Orders this thread's generic-proxy shared-memory writes before the
// tensor core's (async-proxy) reads of them.
__device__ __forceinline__ void fence_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Tensor-memory allocation by one full warp; the address lands in smem.
__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t columns) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(columns)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t tmem, uint32_t columns) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(columns) : "memory");
}

// 32 lanes x 16 consecutive 32-bit columns into each lane's registers
// (warp-collective; lanes 32 * (warp % 4) ...).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
      "%14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Waits for the mbarrier's phase `parity` to complete, at most `limit`
// polls; false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, uint32_t limit) {
  for (uint32_t i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

}  // namespace tc
}  // namespace lotus
