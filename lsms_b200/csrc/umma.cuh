// tcgen05 (5th-generation tensor core) helpers: shared-memory matrix descriptors, kind::tf32
// MMAs with the accumulator in tensor memory, commits to mbarriers, TMEM allocation and loads.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace b200 {
namespace um {

// Shared-memory layouts of a matrix descriptor (bits 61-63).
constexpr uint32_t kSw128Base32b = 1;  // 128-byte swizzle on 32-byte atoms: MN-major TF32 operands
constexpr uint32_t kSw128 = 2;         // 128-byte swizzle: K-major operands, 8-row groups of 128-byte rows

// Descriptor of an operand at shared address `addr`: leading and stride byte offsets (LBO, SBO),
// descriptor version 1, base offset 0 (the swizzle pattern starts on a 1024-byte boundary).
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo, uint32_t layout) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)layout << 61;
  return d;
}

// Instruction descriptor of kind::tf32 with an F32 accumulator: M x N, A and B each K-major
// (false) or MN-major (true).
constexpr uint32_t idesc_tf32(int m, int n, bool a_mn, bool b_mn) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
         ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// D[tmem] (+)= A B, one CTA; `accumulate` 0 overwrites D.
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{ .reg .pred p; setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p; }" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}
// One arrival on `bar` once every tcgen05 operation this thread issued before has completed.
__device__ __forceinline__ void commit(unsigned long long *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   static_cast<unsigned>(__cvta_generic_to_shared(bar)))
               : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Whole warp: allocates `cols` TMEM columns (a power of two >= 32), address into *dst.
__device__ __forceinline__ void alloc(unsigned *dst, unsigned cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   static_cast<unsigned>(__cvta_generic_to_shared(dst))),
               "r"(cols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void dealloc(uint32_t tmem, unsigned cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(cols) : "memory");
}

// Whole warp: lane i reads TMEM lane (addr >> 16) + i, columns (addr & 0xffff) .. + 7.
__device__ __forceinline__ void ld_32x32b_x8(uint32_t addr, uint32_t (&v)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
               : "r"(addr)
               : "memory");
}
__device__ __forceinline__ void wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// FP32 rounded to the nearest TF32 value (ties away from zero), returned as FP32.
__device__ __forceinline__ float tf32_round(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// The same value computed on the integer pipe, for finite inputs: half a TF32 unit in the last
// place added to the magnitude bits, then the 13 bits below the TF32 mantissa cleared.
__device__ __forceinline__ float tf32_round_int(float x) {
  return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xffffe000u);
}

}  // namespace um
}  // namespace b200
