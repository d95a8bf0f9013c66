// The contact predictor on the 5th-generation tensor cores: the 48 -> 128 -> 128 -> 128 -> 6 MLP forward for tiles
// of 128 arenas with tcgen05.mma (BF16 operands from shared memory, FP32 accumulators in tensor memory), the epilogues
// (bias, ReLU, BF16) read back with tcgen05.ld; and training's backward through the layers and weight gradients, below.  Same parameters and outputs as k_pred_forward (the
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
#include "tcgen05.cuh"

using namespace rsx::tc;

namespace {

constexpr int kIn = RSX_PRED_FEATURES, kInPad = 64, kHid = 128, kOutPad = 8, kOutMma = 16, kOut = RSX_PRED_LABELS;
constexpr int oW1 = 0, ob1 = oW1 + kHid * kIn, oW2 = ob1 + kHid, ob2 = oW2 + kHid * kHid, oW3 = ob2 + kHid, ob3 = oW3 + kHid * kHid,
              oW4 = ob3 + kHid, ob4 = oW4 + kOutPad * kHid;
constexpr int kRows = 128;             // arenas per tile = MMA M = threads per CTA = TMEM lanes
constexpr uint32_t kTmemCols = 128;    // one FP32 accumulator of N <= 128

// shared memory (bytes; every operand tile 1024-aligned)
constexpr uint32_t kW1 = 0, kW1Bytes = kHid * kInPad * 2;
constexpr uint32_t kW2 = kW1 + kW1Bytes, kW2Bytes = kHid * kHid * 2;
constexpr uint32_t kW3 = kW2 + kW2Bytes;
constexpr uint32_t kW4 = kW3 + kW2Bytes, kW4Bytes = kOutMma * kHid * 2;
constexpr uint32_t kAct = kW4 + kW4Bytes, kActBytes = kRows * kHid * 2;
constexpr uint32_t kBias = kAct + kActBytes, kBiasBytes = (3 * kHid + kOutMma) * 4;
constexpr uint32_t kMisc = kBias + kBiasBytes;  // mbarrier (8 bytes), TMEM address (4 bytes)
constexpr uint32_t kSmemBytes = kMisc + 16 + 1024;  // + alignment slack

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

// ---- backward through the layers on tcgen05: dZ = (sigmoid(z) - y) / n on the six outputs, then dH3 = (dZ . W4)
// masked by H3 > 0, dH2 = (dH3 . W3) masked by H2 > 0, dH1 = (dH2 . W2) masked by H1 > 0 (BF16; [n][8] and
// [3][n][128], the layout the weight-gradient kernels read), and the loss sum.  The weights are staged transposed
// (B operand element (i, o) = W[o][i], K-major), the dZ / dH tiles are the A operands. ----
namespace {
constexpr uint32_t bW4T = 0, bW4TBytes = kHid * 16 * 2;                 // N = 128 x K = 16 (outputs 8..15 zero)
constexpr uint32_t bW3T = bW4T + bW4TBytes, bW3TBytes = kHid * kHid * 2;
constexpr uint32_t bW2T = bW3T + bW3TBytes;
constexpr uint32_t bAct = bW2T + bW3TBytes;
constexpr uint32_t bMisc = bAct + kActBytes;
constexpr uint32_t kBwdSmemBytes = bMisc + 16 + 1024;
}  // namespace

extern "C" __global__ void __launch_bounds__(kRows, 1) k_pred_backward_tc(const __nv_bfloat16* __restrict__ wb, const float* __restrict__ logits,
                                                                          const uint8_t* __restrict__ Y, const __nv_bfloat16* __restrict__ save,
                                                                          uint32_t n, float inv_scale, __nv_bfloat16* __restrict__ dz,
                                                                          __nv_bfloat16* __restrict__ dsave, float* loss_sum, uint32_t* err) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* sm = reinterpret_cast<unsigned char*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(sm);
  const uint32_t tid = threadIdx.x, warp = tid >> 5;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + bMisc + 8);
  const uint32_t mbar = sbase + bMisc;
  const __nv_bfloat16 zero = __float2bfloat16_rn(0.0f);
  for (uint32_t i = tid; i < (uint32_t)(kHid * 16); i += kRows) {  // element (i, o) of W4^T
    uint32_t r = i / 16, o = i % 16;
    *reinterpret_cast<__nv_bfloat16*>(sm + bW4T + canon(r, o, 16)) = o < (uint32_t)kOutPad ? wb[oW4 + o * kHid + r] : zero;
  }
  for (uint32_t i = tid; i < (uint32_t)(kHid * kHid); i += kRows) {  // W[o][i] -> element (i, o)
    uint32_t o = i / kHid, r = i % kHid;
    *reinterpret_cast<__nv_bfloat16*>(sm + bW3T + canon(r, o, kHid)) = wb[oW3 + i];
    *reinterpret_cast<__nv_bfloat16*>(sm + bW2T + canon(r, o, kHid)) = wb[oW2 + i];
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sbase + bMisc + 8), "r"(kTmemCols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t lane_base = (warp * 32u) << 16;
  uint32_t phase = 0;
  bool ok = true;
  float loss = 0.0f;

  const uint32_t tiles = (n + kRows - 1) / kRows;
  for (uint32_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
    const uint32_t row = tile * kRows + tid;
    const bool live = row < n;
    // dZ (K = 16: outputs 0..5, zero elsewhere) into the A tile and, for outputs 0..7, into dz
    uint32_t pk[8];
#pragma unroll
    for (int o2 = 0; o2 < 8; ++o2) {
      float d2[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int o = 2 * o2 + h;
        float d = 0.0f;
        if (live && o < kOut) {
          const float zz = logits[(size_t)row * kOutPad + o];
          const float y = (Y[row] >> o) & 1u ? 1.0f : 0.0f;
          const float p = 1.0f / (1.0f + expf(-zz));
          d = (p - y) * inv_scale;
          loss += fmaxf(zz, 0.0f) - zz * y + log1pf(expf(-fabsf(zz)));
        }
        d2[h] = d;
      }
      __nv_bfloat162 hv = __floats2bfloat162_rn(d2[0], d2[1]);
      pk[o2] = *reinterpret_cast<uint32_t*>(&hv);
    }
    *reinterpret_cast<uint4*>(sm + bAct + canon(tid, 0, 16)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    *reinterpret_cast<uint4*>(sm + bAct + canon(tid, 8, 16)) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
    if (live) *reinterpret_cast<uint4*>(dz + (size_t)row * kOutPad) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    // three layers down: (operand K, transposed weights, saved activation layer = mask, gradient layer)
#pragma unroll 1
    for (int step = 0; step < 3 && ok; ++step) {
      const uint32_t K = step == 0 ? 16u : (uint32_t)kHid;
      const uint32_t wofs = step == 0 ? bW4T : step == 1 ? bW3T : bW2T;
      const int layer = 2 - step;  // H3, H2, H1 and dH3, dH2, dH1
      fence_smem_to_async();
      fence_before();
      __syncthreads();
      fence_after();
      if (tid == 0) {
        const uint32_t sbo = K / 8 * 128;
#pragma unroll 1
        for (uint32_t s = 0; s < K / 16; ++s)
          mma_bf16(tmem, smem_desc(sbase + bAct + s * 256, 128, sbo), smem_desc(sbase + wofs + s * 256, 128, sbo), instr_desc(kRows, kHid),
                   s > 0 ? 1u : 0u);
        mma_commit(mbar);
      }
      __syncwarp();
      if (!__syncthreads_and(mbar_wait(mbar, phase) ? 1 : 0)) {
        ok = false;
        break;
      }
      phase ^= 1u;
      fence_after();
      const __nv_bfloat16* hrow = save + ((size_t)layer * n + row) * kHid;
      __nv_bfloat16* grow = dsave + ((size_t)layer * n + row) * kHid;
#pragma unroll 1
      for (uint32_t c0 = 0; c0 < (uint32_t)kHid; c0 += 16) {
        float v[16];
        tmem_ld16(tmem + lane_base + c0, v);
        uint4 hm[2] = {make_uint4(0u, 0u, 0u, 0u), make_uint4(0u, 0u, 0u, 0u)};
        if (live) {
          hm[0] = reinterpret_cast<const uint4*>(hrow + c0)[0];
          hm[1] = reinterpret_cast<const uint4*>(hrow + c0)[1];
        }
        const __nv_bfloat16* hb = reinterpret_cast<const __nv_bfloat16*>(hm);
        uint32_t q[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const float lo = __bfloat162float(hb[2 * i]) > 0.0f ? v[2 * i] : 0.0f;
          const float hi = __bfloat162float(hb[2 * i + 1]) > 0.0f ? v[2 * i + 1] : 0.0f;
          __nv_bfloat162 h2v = __floats2bfloat162_rn(lo, hi);
          q[i] = *reinterpret_cast<uint32_t*>(&h2v);
        }
        if (step < 2) {
          *reinterpret_cast<uint4*>(sm + bAct + canon(tid, c0, kHid)) = make_uint4(q[0], q[1], q[2], q[3]);
          *reinterpret_cast<uint4*>(sm + bAct + canon(tid, c0 + 8, kHid)) = make_uint4(q[4], q[5], q[6], q[7]);
        }
        if (live) {
          reinterpret_cast<uint4*>(grow + c0)[0] = make_uint4(q[0], q[1], q[2], q[3]);
          reinterpret_cast<uint4*>(grow + c0)[1] = make_uint4(q[4], q[5], q[6], q[7]);
        }
      }
    }
  }
  if (!ok) {
    if (tid == 0) atomicExch(err, 1u);
    mbar_wait(mbar, phase);
  }
  for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xFFFFFFFFu, loss, o);
  if ((tid & 31) == 0 && loss_sum) atomicAdd(loss_sum, loss);
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

cudaError_t rsx_launch_pred_backward_tc(const void* wb, const float* logits, const uint8_t* Y, const void* save, uint32_t n, float inv_scale,
                                        void* dz, void* dsave, float* loss_sum, uint32_t* err, cudaStream_t s) {
  static int configured[64];
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64 || !configured[dev]) {
    e = cudaFuncSetAttribute((const void*)k_pred_backward_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBwdSmemBytes);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < 64) configured[dev] = 1;
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const uint32_t tiles = (n + kRows - 1) / kRows;
  const uint32_t grid = tiles < (uint32_t)sms ? tiles : (uint32_t)sms;
  k_pred_backward_tc<<<grid, kRows, kBwdSmemBytes, s>>>((const __nv_bfloat16*)wb, logits, Y, (const __nv_bfloat16*)save, n, inv_scale,
                                                        (__nv_bfloat16*)dz, (__nv_bfloat16*)dsave, loss_sum, err);
  return cudaGetLastError();
}

// ---- weight gradients on tcgen05: dW[o][i] += sum_b G[b][o] Act[b][i] and db[o] += sum_b G[b][o] over a slice of
// the batch, the batch as the MMA's K (64 arenas per staged chunk, both operands transposed into K-major tiles while
// staging).  The 128-wide side is the MMA's M: o for W3, W2, W1 (G = dH3, dH2, dH1; N = i = 128, 128, 48), i for W4
// (A = H3, B = dZ with N = 16, so D holds dW4 transposed).  Partial sums of each slice are added with atomics. ----
namespace {
constexpr uint32_t kChunk = 64;                      // batch rows per staged chunk (MMA K 64 = 4 instructions)
constexpr uint32_t gA = 0, gABytes = kRows * kChunk * 2;
constexpr uint32_t gB = gA + gABytes, gBBytes = kRows * kChunk * 2;
constexpr uint32_t gMisc = gB + gBBytes;
constexpr uint32_t kWgradSmemBytes = 56 * 1024;      // at most 4 CTAs per SM: their 128 TMEM columns each always fit
static_assert(gMisc + 16 + 1024 <= kWgradSmemBytes, "wgrad shared memory");
}  // namespace

extern "C" __global__ void __launch_bounds__(kRows) k_pred_wgrad_tc(const __nv_bfloat16* __restrict__ X, const __nv_bfloat16* __restrict__ dz,
                                                                    const __nv_bfloat16* __restrict__ save, const __nv_bfloat16* __restrict__ dsave,
                                                                    uint32_t n, uint32_t slice, float* __restrict__ grad, uint32_t* err) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* sm = reinterpret_cast<unsigned char*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(sm);
  const uint32_t tid = threadIdx.x, warp = tid >> 5;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + gMisc + 8);
  const uint32_t mbar = sbase + gMisc;
  const int layer = blockIdx.y;  // 0: W4, 1: W3, 2: W2, 3: W1
  // A operand (the 128-wide side) and B operand sources: element (row r, batch b) = src[b * stride + r]
  const __nv_bfloat16* asrc;
  const __nv_bfloat16* bsrc;
  uint32_t bstride, N, nb_live;  // B row count in the MMA (N), B rows that exist in the source
  float* dW;
  float* db;
  if (layer == 0) {
    asrc = save + (size_t)2 * n * kHid;  // H3
    bsrc = dz;
    bstride = kOutPad;
    N = kOutMma;
    nb_live = kOut;
    dW = grad + oW4;
    db = grad + ob4;
  } else {
    asrc = dsave + (size_t)(3 - layer) * n * kHid;  // dH3, dH2, dH1
    bsrc = layer == 3 ? X : save + (size_t)(2 - layer) * n * kHid;  // H2, H1, X
    bstride = layer == 3 ? kIn : kHid;
    N = layer == 3 ? kIn : kHid;
    nb_live = N;
    dW = grad + (layer == 1 ? oW3 : layer == 2 ? oW2 : oW1);
    db = grad + (layer == 1 ? ob3 : layer == 2 ? ob2 : ob1);
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sbase + gMisc + 8), "r"(kTmemCols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t b_lo = blockIdx.x * slice, b_hi = min(n, b_lo + slice);
  const __nv_bfloat16 zero = __float2bfloat16_rn(0.0f);
  uint32_t phase = 0;
  bool ok = true, first = true;
  float bias_acc = 0.0f;  // layers 1..3: db of row o = tid
  float bias_w4 = 0.0f;   // layer 0: this thread's share of db4[tid % 16]
#pragma unroll 1
  for (uint32_t c = b_lo; c < b_hi && ok; c += kChunk) {
    // stage the chunk, transposing: A element (r, b) for r < 128, B element (r, b) for r < N
    for (uint32_t idx = tid; idx < (uint32_t)kRows * kChunk; idx += kRows) {
      const uint32_t b = idx / kRows, r = idx % kRows, gb = c + b;
      __nv_bfloat16 v = gb < b_hi ? asrc[(size_t)gb * kHid + r] : zero;
      *reinterpret_cast<__nv_bfloat16*>(sm + gA + canon(r, b, kChunk)) = v;
      if (layer != 0) bias_acc += __bfloat162float(v);
    }
    for (uint32_t idx = tid; idx < N * kChunk; idx += kRows) {
      const uint32_t b = idx / N, r = idx % N, gb = c + b;
      __nv_bfloat16 v = (gb < b_hi && r < nb_live) ? bsrc[(size_t)gb * bstride + r] : zero;
      *reinterpret_cast<__nv_bfloat16*>(sm + gB + canon(r, b, kChunk)) = v;
      if (layer == 0) bias_w4 += __bfloat162float(v);
    }
    fence_smem_to_async();
    fence_before();
    __syncthreads();
    fence_after();
    if (tid == 0) {
      const uint32_t sbo = kChunk / 8 * 128;
#pragma unroll 1
      for (uint32_t s = 0; s < kChunk / 16; ++s)
        mma_bf16(tmem, smem_desc(sbase + gA + s * 256, 128, sbo), smem_desc(sbase + gB + s * 256, 128, sbo), instr_desc(kRows, N),
                 (first && s == 0) ? 0u : 1u);
      mma_commit(mbar);
    }
    first = false;
    __syncwarp();
    if (!__syncthreads_and(mbar_wait(mbar, phase) ? 1 : 0)) {
      ok = false;
      break;
    }
    phase ^= 1u;
    fence_after();
  }
  if (ok && !first) {
    // this thread's accumulator row r = tid: W3 / W2 / W1 row o = r (columns i); W4 column i = r (rows o = columns)
    const uint32_t lane_base = (warp * 32u) << 16;
#pragma unroll 1
    for (uint32_t c0 = 0; c0 < N; c0 += 16) {
      float v[16];
      tmem_ld16(tmem + lane_base + c0, v);
      for (int j = 0; j < 16; ++j) {
        const uint32_t col = c0 + j;
        if (layer == 0) {
          if (col < (uint32_t)kOut) atomicAdd(&dW[col * kHid + tid], v[j]);
        } else if (col < N) {
          atomicAdd(&dW[tid * N + col], v[j]);
        }
      }
    }
  }
  if (layer != 0) {
    atomicAdd(&db[tid], bias_acc);
  } else {
    // thread tid staged the dZ column tid % 16 (N = 16 divides 128)
    if (tid % kOutMma < (uint32_t)kOut) atomicAdd(&db[tid % kOutMma], bias_w4);
  }
  if (!ok) {
    if (tid == 0) atomicExch(err, 1u);
    mbar_wait(mbar, phase);
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

cudaError_t rsx_launch_pred_wgrads_tc(const void* X, const void* dz, const void* save, const void* dsave, uint32_t n, float* grad, uint32_t* err,
                                      cudaStream_t s) {
  static int configured[64];
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64 || !configured[dev]) {
    e = cudaFuncSetAttribute((const void*)k_pred_wgrad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kWgradSmemBytes);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < 64) configured[dev] = 1;
  }
  const uint32_t slice = 512, slices = (n + slice - 1) / slice;
  k_pred_wgrad_tc<<<dim3(slices, 4), kRows, kWgradSmemBytes, s>>>((const __nv_bfloat16*)X, (const __nv_bfloat16*)dz, (const __nv_bfloat16*)save,
                                                                  (const __nv_bfloat16*)dsave, n, slice, grad, err);
  return cudaGetLastError();
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
