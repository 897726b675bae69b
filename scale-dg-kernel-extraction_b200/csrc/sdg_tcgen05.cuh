// Fifth-generation tensor-core (tcgen05) helpers for the TF32 line
// contractions of the mixed form at Nq = 8 (kernel variant kVariantTensor).
//
// The x-line contraction of a tile of two elements is, per line (j, k, e),
// out_x(i) = sum_l D(i, l) F_x(l, j, k, e): as a matrix product
// OUT[m, i] = sum_l A[m, l] B[l, i] with m = (j, k, e) the 128 lines (one per
// thread of the tile, the thread that owns x-line (j, k) of element e),
// A[m, l] = F_x(l, j, k, e) and B[l, i] = D(i, l); the y lines likewise with
// m = (i, k, e) and A[m, l] = F_y(i, l, k, e).  One tcgen05.mma of shape
// M = 128, N = 8, K = 8 (kind::tf32) per pass and direction, accumulated in
// tensor memory (TMEM lane m, 8 columns); thread m reads its line's eight
// results back with one tcgen05.ld.
//
// TF32 keeps 10 mantissa bits, so each operand is split into hi = tf32(x)
// and lo = tf32(x - hi) and three passes accumulate hi*hi + lo*hi + hi*lo
// (the lo*lo term is below FP32 rounding of the sum).
//
// Operands sit in shared memory in the canonical K-major layout without
// swizzle: 8-row x 16-byte core matrices, rows 16 bytes apart, the two
// 16-byte K halves (l = 0..3, 4..7) kLbo bytes apart and successive 8-row
// groups kSbo bytes apart.  Descriptor bit fields follow the sm_100
// shared-memory and instruction descriptor formats of the PTX ISA
// (tcgen05 matrix descriptors).
#pragma once

#include <stdint.h>

namespace sdg {
namespace tc {

constexpr uint32_t kLbo = 128;  // bytes between the two K halves of a core row
constexpr uint32_t kSbo = 256;  // bytes between 8-row groups
constexpr uint32_t kOperandBytes = 16 * kSbo;  // 128 rows x 8 TF32
constexpr uint32_t kBBytes = 2 * kLbo;         // 8 rows x 8 TF32
constexpr int kTmemCols = 32;                  // smallest allocation

// Byte offset of element (row m, k) in a K-major operand.
__host__ __device__ constexpr uint32_t offset(int m, int k) {
  return (m >> 3) * kSbo + (m & 7) * 16 + (k >> 2) * kLbo + (k & 3) * 4;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: start address, leading and stride byte
// offsets (all >> 4), version 1, no base offset, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(const void* p) {
  uint64_t d = static_cast<uint64_t>((smem_addr(p) >> 4) & 0x3FFF);
  d |= static_cast<uint64_t>((kLbo >> 4) & 0x3FFF) << 16;
  d |= static_cast<uint64_t>((kSbo >> 4) & 0x3FFF) << 32;
  d |= static_cast<uint64_t>(1) << 46;
  return d;
}

// Instruction descriptor: FP32 accumulator, TF32 A and B, both K-major,
// N = 8, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((8u >> 3) << 17) |
                            ((128u >> 4) << 24);

// x rounded to TF32 (round to nearest, ties away), kept in a 32-bit word.
__device__ __forceinline__ float to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// One warp allocates kTmemCols columns and writes the address to *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_addr(slot)),
               "n"(kTmemCols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr),
               "n"(kTmemCols)
               : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// D[tmem] (+)= A * B, one thread.
__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t a, uint64_t b,
                                         bool accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
      "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate ? 1u : 0u)
      : "memory");
}

// The MMAs issued so far by this thread arrive on `bar` when complete.
__device__ __forceinline__ void commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_addr(bar))
      : "memory");
}

// Eight 32-bit columns of this thread's TMEM lane (warp w reads lanes
// 32 w .. 32 w + 31), waited for.
__device__ __forceinline__ void ld8(uint32_t taddr, float* r) {
  uint32_t v[8];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int c = 0; c < 8; ++c) r[c] = __uint_as_float(v[c]);
}

}  // namespace tc
}  // namespace sdg
