// tcgen05 building blocks shared by the predictor's tensor-core kernels: the UMMA canonical K-major shared-memory
// layout without swizzle and its descriptor, the kind::f16 instruction descriptor, MMA issue and commit, bounded
// mbarrier waits, TMEM loads and the tcgen05 fences (PTX ISA, tcgen05 family; bit layouts as in CUTLASS's
// cute/arch/mma_sm100_desc.hpp).
#pragma once
#include <stdint.h>

namespace rsx {
namespace tc {

constexpr long long kWaitCycles = 1ll << 28;

// byte offset of element (r, k) of a K-major operand with K columns in the canonical no-swizzle layout
__device__ __forceinline__ uint32_t canon(uint32_t r, uint32_t k, uint32_t K) {
  return (r >> 3) * (K / 8 * 128) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

// shared-memory matrix descriptor (SM100 UMMA): start >> 4 in bits 0-13, leading-dimension byte offset (the K
// direction between 8-element core matrices) >> 4 in bits 16-29, stride byte offset (between 8-row groups) >> 4 in
// bits 32-45, version 1 in bits 46-47, no swizzle (layout type 0 in bits 61-63)
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) | ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) |
         (1ull << 46);
}
// instruction descriptor, kind::f16: FP32 accumulate (bits 4-5 = 1), A and B BF16 (bits 7-9, 10-12 = 1), both K-major,
// N >> 3 in bits 17-22, M >> 4 in bits 24-28
__host__ __device__ constexpr uint32_t instr_desc(uint32_t M, uint32_t N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d), "l"(a),
      "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  const long long t0 = clock64();
  for (;;) {
    uint32_t done;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(done)
                 : "r"(mbar), "r"(parity)
                 : "memory");
    if (done) return true;
    if (clock64() - t0 > kWaitCycles) return false;
  }
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]),
        "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_smem_to_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }


}  // namespace tc
}  // namespace rsx
