// 5th-generation tensor cores (tcgen05) for the mixed form's volume
// contraction: D[128 x N] (FP32, in tensor memory) = A[128 x K] B[K x N] with
// A and B TF32 operands in shared memory, K-major, no swizzle.  Operands are
// split into a TF32 high part and a TF32 remainder and the three products
// hi*hi + hi*lo + lo*hi accumulate into D, which keeps the contraction at
// FP32 accuracy.  One elected thread issues the MMAs; completion arrives on an
// mbarrier through tcgen05.commit; each warp reads its 32 lanes of D.
#pragma once

#include <cstdint>

#include "dgp_tma.cuh"

namespace dgp {

// K-major, no-swizzle operand layout: 8-row x 16-byte core matrices; the
// core matrices of one 8-row group lie 128 bytes apart along K (leading
// byte offset) and the 8-row groups `sbo` bytes apart (stride byte offset).
// Byte offset of element (row, k) of a 4-byte operand with Kpad columns:
__host__ __device__ constexpr uint32_t umma_off(int row, int k, int kpad) {
  return (uint32_t)((row >> 3) * (kpad / 4) * 128 + (k >> 2) * 128 + (row & 7) * 16 + (k & 3) * 4);
}

// shared-memory matrix descriptor (tcgen05): start address, leading and
// stride byte offsets (all >> 4), descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t umma_desc(const void* smem, uint32_t lbo, uint32_t sbo) {
  const uint32_t a = smem_u32(smem);
  return (uint64_t)((a >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor of kind::tf32: F32 accumulator, TF32 A and B, both
// K-major, N >> 3 at bit 17, M >> 4 at bit 24
constexpr uint32_t umma_idesc_tf32(int m, int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// x = hi + lo to about 2^-22 relative: hi its TF32 rounding, lo the TF32
// rounding of the remainder
__device__ __forceinline__ void tf32_split(float x, uint32_t& hi, uint32_t& lo) {
  hi = to_tf32(x);
  lo = to_tf32(x - __uint_as_float(hi));
}

// tensor-memory allocation by one whole warp: the address lands in *dst
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// D (+)= A B, one MMA of M x N x 8 (TF32)
__device__ __forceinline__ void umma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// the MMAs issued so far by this thread arrive on the mbarrier when done
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

// 16 consecutive 32-bit columns of this warp's 32 lanes (lane = thread)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// host: the TF32 rounding (10 explicit mantissa bits, to nearest) of a value
// that is exact in FP32
inline float host_tf32(float x) {
  uint32_t u;
  __builtin_memcpy(&u, &x, 4);
  if ((u & 0x7F800000u) == 0x7F800000u) return x;
  u = (u + 0x1000u) & 0xFFFFE000u;
  float r;
  __builtin_memcpy(&r, &u, 4);
  return r;
}

}  // namespace dgp
