// tc_common.cuh -- inline PTX helpers for the 5th-generation tensor cores
// (tcgen05) shared by the tensor-core kernels: shared-memory matrix
// descriptors, the TF32 head of an FP32 value, bounded mbarrier waits, the
// kind::tf32 MMA and its commit.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace efmm {
namespace {

constexpr long long TC_WAIT_CYCLES = 4000000000LL;  // about 2 s at 2 GHz

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// no-swizzle shared-memory matrix descriptor (version 1)
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// instruction descriptor: F32 accumulate, TF32 A and B (both K-major), M x N
__host__ __device__ constexpr uint32_t tc_idesc_mn(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | (0u << 15) | (0u << 16) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

// TF32 value nearest to x, ties away from zero (what cvt.rna.tf32.f32
// gives), in integer operations: the conversion instruction issues on the XU
// pipe, which splitting every staged operand element would saturate.
// Infinities and NaNs pass unchanged.
__device__ __forceinline__ float tf32_head(float x) {
  const uint32_t u = __float_as_uint(x);
  return (u & 0x7f800000u) == 0x7f800000u ? x : __uint_as_float((u + 0x1000u) & ~0x1FFFu);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait for phase `parity` of the barrier; false when it ran out
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  const long long t0 = clock64();
  while (!mbar_try(bar, parity))
    if (clock64() - t0 > TC_WAIT_CYCLES) return false;
  return true;
}

__device__ __forceinline__ void mma_tf32(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(dtmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

}  // namespace
}  // namespace efmm
