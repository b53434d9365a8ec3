// 5th-generation tensor core (tcgen05) helpers for sm_100a.
//
//   * tensor memory (TMEM): allocation by one warp, relinquish, release;
//   * shared-memory matrix descriptors for K-major operands in the canonical
//     layout without swizzle: "core matrices" of 8 rows x 16 bytes stored as
//     128 contiguous bytes; LBO is the byte distance between the two core
//     matrices that are adjacent along K, SBO the distance between core
//     matrices adjacent along M (or N);
//   * kind::tf32 MMAs (A and B read from shared memory, D = A x B^T summed
//     into an FP32 accumulator in TMEM), issued by one thread;
//   * tcgen05.commit to an mbarrier (arrives when every MMA the thread issued
//     before it has completed);
//   * 32 lanes x 32-bit TMEM loads for the epilogue (warp w of a CTA may read
//     TMEM lanes 32 (w mod 4) .. 32 (w mod 4) + 31).
//
// The descriptor bit layouts follow the PTX ISA (tcgen05 matrix and
// instruction descriptors), as CUTLASS's cute/arch/mma_sm100_desc.hpp also
// encodes them.  Only CTA-local forms are used (cta_group::1, no multicast).
#pragma once

#include <stdint.h>

#include "tma.cuh"

namespace drb {

// Allocates ncols (a power of two >= 32) TMEM columns; the whole warp executes it.  The TMEM address of the
// allocation is written to *dst.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst)), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// Order tcgen05 operations against thread synchronisation (barriers, mbarrier waits).
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Matrix descriptor: start address, LBO and SBO in 16-byte units (14 bits each), descriptor version 1 at bits
// 46-47, base offset 0, absolute LBO mode, layout type 0 (no swizzle) at bits 61-63.
__device__ __forceinline__ uint64_t sdesc_kmajor(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor for kind::tf32: D format F32 (bits 4-5 = 1), A and B format TF32 (bits 7-9, 10-12 = 2),
// both K-major (bits 15, 16 = 0), N / 8 at bits 17-22, M / 16 at bits 24-28.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A x B^T; accumulate == 0 overwrites D.
__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// One arrival on *bar once all MMAs previously issued by this thread have completed.
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
               : "memory");
}

// Thread i of the warp receives TMEM lane (lane field of taddr) + i, columns (column field) .. + 15.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// x = hi + lo with hi holding the sign, exponent and top 10 mantissa bits of x (the bits a TF32 operand keeps) and
// lo = x - hi exact; hi x hi + hi x lo + lo x hi then carries about 21 bits of each product.
__device__ __forceinline__ float tf32_hi(float x) { return __uint_as_float(__float_as_uint(x) & 0xFFFFE000u); }

}  // namespace drb
