// The contact predictor's inference on the 5th-generation tensor cores: the 48 -> 128 -> 128 -> 128 -> 6 MLP forward
// for tiles of 128 arenas with tcgen05.mma (BF16 operands from shared memory, FP32 accumulators in tensor memory),
// the epilogues (bias, ReLU, BF16) read back with tcgen05.ld.  Same parameters and outputs as k_pred_forward (the
// mma.sync version), including the saved activations that training's backward pass reads; the logits agree to FP32
// rounding of the same BF16 products.
//
// Per CTA (128 threads, one per accumulator row / TMEM lane): the four weight matrices are staged once in shared
// memory in the UMMA canonical K-major layout without swizzle (8 x 16-byte core matrices: element (r, k) at
// (r / 8) * SBO + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2 bytes, SBO = K / 8 * 128), then the CTA loops over
// 128-arena tiles: the feature tile is written in the same layout (K padded 48 -> 64 with zeros), one thread issues
// the layer's MMAs (K / 16 of them, 128 x N x 16 each) and commits them to an mbarrier; every warp waits, loads its
// 32 accumulator rows from TMEM, applies bias and ReLU and writes the next layer's operand tile.  The output layer is
// N = 16 (outputs 8..15 zero weights).  Waits are bounded by a clock limit: on expiry the kernel raises *err, waits
// (bounded) for its MMAs in flight, frees its TMEM and returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/rsx.h"

namespace {

constexpr int kIn = RSX_PRED_FEATURES, kInPad = 64, kHid = 128, kOutPad = 8, kOutMma = 16;
constexpr int oW1 = 0, ob1 = oW1 + kHid * kIn, oW2 = ob1 + kHid, ob2 = oW2 + kHid * kHid, oW3 = ob2 + kHid, ob3 = oW3 + kHid * kHid,
              oW4 = ob3 + kHid, ob4 = oW4 + kOutPad * kHid;
constexpr int kRows = 128;             // arenas per tile = MMA M = threads per CTA = TMEM lanes
constexpr uint32_t kTmemCols = 128;    // one FP32 accumulator of N <= 128
constexpr long long kWaitCycles = 1ll << 28;

// shared memory (bytes; every operand tile 1024-aligned)
constexpr uint32_t kW1 = 0, kW1Bytes = kHid * kInPad * 2;
constexpr uint32_t kW2 = kW1 + kW1Bytes, kW2Bytes = kHid * kHid * 2;
constexpr uint32_t kW3 = kW2 + kW2Bytes;
constexpr uint32_t kW4 = kW3 + kW2Bytes, kW4Bytes = kOutMma * kHid * 2;
constexpr uint32_t kAct = kW4 + kW4Bytes, kActBytes = kRows * kHid * 2;
constexpr uint32_t kBias = kAct + kActBytes, kBiasBytes = (3 * kHid + kOutMma) * 4;
constexpr uint32_t kMisc = kBias + kBiasBytes;  // mbarrier (8 bytes), TMEM address (4 bytes)
constexpr uint32_t kSmemBytes = kMisc + 16 + 1024;  // + alignment slack

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

}  // namespace

extern "C" __global__ void __launch_bounds__(kRows, 1) k_pred_forward_tc(const __nv_bfloat16* __restrict__ wb, const float* __restrict__ wf,
                                                                         const __nv_bfloat16* __restrict__ X, uint32_t n, float* __restrict__ logits,
                                                                         __nv_bfloat16* __restrict__ save, uint32_t* err) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* sm = reinterpret_cast<unsigned char*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(sm);
  const uint32_t tid = threadIdx.x, warp = tid >> 5;
  float* bias = reinterpret_cast<float*>(sm + kBias);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + kMisc + 8);
  const uint32_t mbar = sbase + kMisc;

  // weights and biases into the canonical layout (zero padding: W1's K 48..63, W4's rows 8..15)
  const __nv_bfloat16 zero = __float2bfloat16_rn(0.0f);
  for (uint32_t i = tid; i < (uint32_t)(kHid * kInPad); i += kRows) {
    uint32_t r = i / kInPad, k = i % kInPad;
    *reinterpret_cast<__nv_bfloat16*>(sm + kW1 + canon(r, k, kInPad)) = k < (uint32_t)kIn ? wb[oW1 + r * kIn + k] : zero;
  }
  for (uint32_t i = tid; i < (uint32_t)(kHid * kHid); i += kRows) {
    uint32_t r = i / kHid, k = i % kHid;
    *reinterpret_cast<__nv_bfloat16*>(sm + kW2 + canon(r, k, kHid)) = wb[oW2 + i];
    *reinterpret_cast<__nv_bfloat16*>(sm + kW3 + canon(r, k, kHid)) = wb[oW3 + i];
  }
  for (uint32_t i = tid; i < (uint32_t)(kOutMma * kHid); i += kRows) {
    uint32_t r = i / kHid, k = i % kHid;
    *reinterpret_cast<__nv_bfloat16*>(sm + kW4 + canon(r, k, kHid)) = r < (uint32_t)kOutPad ? wb[oW4 + r * kHid + k] : zero;
  }
  for (uint32_t i = tid; i < (uint32_t)kHid; i += kRows) {
    bias[i] = wf[ob1 + i];
    bias[kHid + i] = wf[ob2 + i];
    bias[2 * kHid + i] = wf[ob3 + i];
  }
  if (tid < (uint32_t)kOutMma) bias[3 * kHid + tid] = tid < (uint32_t)kOutPad ? wf[ob4 + tid] : 0.0f;
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sbase + kMisc + 8), "r"(kTmemCols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t lane_base = (warp * 32u) << 16;  // this warp's 32 TMEM lanes
  uint32_t phase = 0;
  bool ok = true;

  const uint32_t tiles = (n + kRows - 1) / kRows;
  for (uint32_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
    const uint32_t row = tile * kRows + tid;
    const bool live = row < n;
    // the feature tile (K 48 padded to 64)
#pragma unroll 4
    for (uint32_t k = 0; k < (uint32_t)kInPad; k += 8) {
      uint32_t w[4] = {0u, 0u, 0u, 0u};
      if (live && k < (uint32_t)kIn) {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(X + (size_t)row * kIn + k);
        w[0] = src[0];
        w[1] = src[1];
        w[2] = src[2];
        w[3] = src[3];
      }
      *reinterpret_cast<uint4*>(sm + kAct + canon(tid, k, kInPad)) = make_uint4(w[0], w[1], w[2], w[3]);
    }
    // four layers: (operand K, weights, N, bias)
#pragma unroll 1
    for (int layer = 0; layer < 4 && ok; ++layer) {
      const uint32_t K = layer == 0 ? kInPad : kHid;
      const uint32_t N = layer == 3 ? kOutMma : kHid;
      const uint32_t wofs = layer == 0 ? kW1 : layer == 1 ? kW2 : layer == 2 ? kW3 : kW4;
      fence_smem_to_async();
      fence_before();
      __syncthreads();
      fence_after();
      if (tid == 0) {
        const uint32_t sbo = K / 8 * 128;
#pragma unroll 1
        for (uint32_t s = 0; s < K / 16; ++s)
          mma_bf16(tmem, smem_desc(sbase + kAct + s * 256, 128, sbo), smem_desc(sbase + wofs + s * 256, 128, sbo), instr_desc(kRows, N),
                   s > 0 ? 1u : 0u);
        mma_commit(mbar);
      }
      __syncwarp();
      // every thread waits for the layer's MMAs; the block agrees on the outcome so that all take the same path
      if (!__syncthreads_and(mbar_wait(mbar, phase) ? 1 : 0)) {
        ok = false;
        break;
      }
      phase ^= 1u;
      fence_after();
      if (layer < 3) {
        // bias, ReLU, BF16: this thread's row of the next operand tile (K = 128)
        const float* b = bias + layer * kHid;
#pragma unroll 1
        for (uint32_t c0 = 0; c0 < (uint32_t)kHid; c0 += 16) {
          float v[16];
          tmem_ld16(tmem + lane_base + c0, v);
          uint32_t pk[8];
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            float lo = fmaxf(v[2 * i] + b[c0 + 2 * i], 0.0f), hi = fmaxf(v[2 * i + 1] + b[c0 + 2 * i + 1], 0.0f);
            __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
            pk[i] = *reinterpret_cast<uint32_t*>(&h);
          }
          *reinterpret_cast<uint4*>(sm + kAct + canon(tid, c0, kHid)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
          *reinterpret_cast<uint4*>(sm + kAct + canon(tid, c0 + 8, kHid)) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
          if (save && live) {  // the activations for the backward pass: [layer][n][128] BF16, row-major
            uint4* dst = reinterpret_cast<uint4*>(save + ((size_t)layer * n + row) * kHid + c0);
            dst[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
            dst[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
          }
        }
      } else {
        float v[16];
        tmem_ld16(tmem + lane_base, v);
        if (live) {
          float4* dst = reinterpret_cast<float4*>(logits + (size_t)row * kOutPad);
          const float* b = bias + 3 * kHid;
          dst[0] = make_float4(v[0] + b[0], v[1] + b[1], v[2] + b[2], v[3] + b[3]);
          dst[1] = make_float4(v[4] + b[4], v[5] + b[5], v[6] + b[6], v[7] + b[7]);
        }
      }
    }
  }
  if (!ok) {
    if (tid == 0) atomicExch(err, 1u);
    mbar_wait(mbar, phase);  // the MMAs in flight, bounded again
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

cudaError_t rsx_launch_pred_forward_tc(const void* wb, const float* wf, const void* X, uint32_t n, float* logits, void* save, uint32_t* err,
                                       cudaStream_t s) {
  static int configured[64];
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64 || !configured[dev]) {
    e = cudaFuncSetAttribute((const void*)k_pred_forward_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < 64) configured[dev] = 1;
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const uint32_t tiles = (n + kRows - 1) / kRows;
  const uint32_t grid = tiles < (uint32_t)sms ? tiles : (uint32_t)sms;
  k_pred_forward_tc<<<grid, kRows, kSmemBytes, s>>>((const __nv_bfloat16*)wb, wf, (const __nv_bfloat16*)X, n, logits, (__nv_bfloat16*)save, err);
  return cudaGetLastError();
}
