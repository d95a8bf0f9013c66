// The contact predictor: per-arena features, a 48 -> 128 -> 128 -> 128 -> 6 ReLU MLP with sigmoid outputs (BF16
// weights and activations, FP32 accumulation), Adam on the FP32 master weights, and the orders of arenas (two bins,
// cost levels) for the persistent decision kernels.  The MLP's products run on tcgen05 (predictor_tc.cu: forward,
// backward, weight gradients); the forward here, on mma.sync m16n8k16, is kept as the check of that one.
//
// It only schedules work: the decision kernels give the same words whatever order they take arenas in, so a wrong
// prediction costs time, never correctness.  The six labels are the decision's event OR (the decision kernels'
// ev_or output): car 0 - ball (event bit 0), car 1 - ball (1), car - car bump or demo (2..5), ball - world (12, 14),
// car 0 - world (10), car 1 - world (11).
//
// Parameter layout (floats; the BF16 copy has the same indexing, biases are read from the FP32 master):
//   W1[128][48] b1[128] W2[128][128] b2[128] W3[128][128] b3[128] W4[8][128] b4[8]   (rows 6, 7 of W4 stay zero)
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/rsx.h"
#include "state.cuh"

using namespace rsx;

namespace {

constexpr int kIn = RSX_PRED_FEATURES, kHid = 128, kOutPad = 8, kOut = RSX_PRED_LABELS;
constexpr int oW1 = 0, ob1 = oW1 + kHid * kIn, oW2 = ob1 + kHid, ob2 = oW2 + kHid * kHid, oW3 = ob2 + kHid, ob3 = oW3 + kHid * kHid,
              oW4 = ob3 + kHid, ob4 = oW4 + kOutPad * kHid, kParams = ob4 + kOutPad;
static_assert(kParams == RSX_PRED_PARAMS, "parameter count");

// padded shared-memory row strides (bf16 elements): conflict-free 32-bit fragment loads
constexpr int sIn = kIn + 8, sHid = kHid + 8;
constexpr int kWarps = 4;

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}
__device__ __forceinline__ uint32_t ld32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

// D = A(16x16, row) * B(16x8, col) + D, BF16 inputs, FP32 accumulate
__device__ __forceinline__ void mma16816(float c[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

struct Smem {
  __nv_bfloat16 w1[kHid * sIn], w2[kHid * sHid], w3[kHid * sHid], w4[kOutPad * sHid];
  float b1[kHid], b2[kHid], b3[kHid], b4[kOutPad];
  __nv_bfloat16 act[kWarps][2][16 * sHid];
};

__device__ void load_weights(Smem& sm, const __nv_bfloat16* wb, const float* wf) {
  for (int i = threadIdx.x; i < kHid * kIn; i += blockDim.x) sm.w1[(i / kIn) * sIn + i % kIn] = wb[oW1 + i];
  for (int i = threadIdx.x; i < kHid * kHid; i += blockDim.x) {
    sm.w2[(i / kHid) * sHid + i % kHid] = wb[oW2 + i];
    sm.w3[(i / kHid) * sHid + i % kHid] = wb[oW3 + i];
  }
  for (int i = threadIdx.x; i < kOutPad * kHid; i += blockDim.x) sm.w4[(i / kHid) * sHid + i % kHid] = wb[oW4 + i];
  for (int i = threadIdx.x; i < kHid; i += blockDim.x) {
    sm.b1[i] = wf[ob1 + i];
    sm.b2[i] = wf[ob2 + i];
    sm.b3[i] = wf[ob3 + i];
  }
  for (int i = threadIdx.x; i < kOutPad; i += blockDim.x) sm.b4[i] = wf[ob4 + i];
  __syncthreads();
}

// one dense layer for a warp's 16 rows: out(16 x N) = relu?(in(16 x K) . W^T + b), W[N][K] in shared memory
template <int K, int N, int SIN, int SW, bool RELU>
__device__ void layer_fwd(const __nv_bfloat16* in, const __nv_bfloat16* w, const float* bias, __nv_bfloat16* out, int sout,
                          __nv_bfloat16* save, float* logits, int rows_left) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  uint32_t a[K / 16][4];
#pragma unroll
  for (int ks = 0; ks < K / 16; ++ks) {
    const int k0 = ks * 16 + 2 * t;
    a[ks][0] = ld32(in + g * SIN + k0);
    a[ks][1] = ld32(in + (g + 8) * SIN + k0);
    a[ks][2] = ld32(in + g * SIN + k0 + 8);
    a[ks][3] = ld32(in + (g + 8) * SIN + k0 + 8);
  }
#pragma unroll 1
  for (int nt = 0; nt < N / 8; ++nt) {
    const int n0 = nt * 8;
    float c[4] = {bias[n0 + 2 * t], bias[n0 + 2 * t + 1], bias[n0 + 2 * t], bias[n0 + 2 * t + 1]};
#pragma unroll
    for (int ks = 0; ks < K / 16; ++ks) {
      uint32_t b[2] = {ld32(w + (n0 + g) * SW + ks * 16 + 2 * t), ld32(w + (n0 + g) * SW + ks * 16 + 2 * t + 8)};
      mma16816(c, a[ks], b);
    }
    if (logits) {
      if (g < rows_left) {
        logits[g * kOutPad + n0 + 2 * t] = c[0];
        logits[g * kOutPad + n0 + 2 * t + 1] = c[1];
      }
      if (g + 8 < rows_left) {
        logits[(g + 8) * kOutPad + n0 + 2 * t] = c[2];
        logits[(g + 8) * kOutPad + n0 + 2 * t + 1] = c[3];
      }
      continue;
    }
    if (RELU)
      for (int i = 0; i < 4; ++i) c[i] = fmaxf(c[i], 0.0f);
    uint32_t lo = pack2(__float2bfloat16_rn(c[0]), __float2bfloat16_rn(c[1]));
    uint32_t hi = pack2(__float2bfloat16_rn(c[2]), __float2bfloat16_rn(c[3]));
    *reinterpret_cast<uint32_t*>(out + g * sout + n0 + 2 * t) = lo;
    *reinterpret_cast<uint32_t*>(out + (g + 8) * sout + n0 + 2 * t) = hi;
    if (save) {
      if (g < rows_left) *reinterpret_cast<uint32_t*>(save + g * kHid + n0 + 2 * t) = lo;
      if (g + 8 < rows_left) *reinterpret_cast<uint32_t*>(save + (g + 8) * kHid + n0 + 2 * t) = hi;
    }
  }
  __syncwarp();
}

}  // namespace

// ---- features: 48 per arena from the tick-boundary state (AoSoA-32), its StaticData and its controls ----
__device__ __forceinline__ float sw(const uint32_t* st, uint32_t a, size_t byte_off) {
  return __uint_as_float(st[aosoa_index(a, (int)(byte_off / 4))]);
}
__device__ __forceinline__ uint32_t uw(const uint32_t* st, uint32_t a, size_t byte_off) { return st[aosoa_index(a, (int)(byte_off / 4))]; }

__device__ __forceinline__ float boundary_dist(float x, float y, float z) {
  return fminf(fminf(4096.0f - fabsf(x), 5120.0f - fabsf(y)), fminf(z, 2044.0f - z));
}

extern "C" __global__ void k_pred_features(const uint32_t* states, const StaticData* sds, const uint8_t* sd_index, const Controls* controls,
                                           uint32_t n, __nv_bfloat16* X) {
  uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  const StaticData& D = sds[sd_index ? sd_index[a] : 0];
  float f[kIn];
  const size_t ob = offsetof(ArenaState, ball);
  float bp[3], bv[3];
  for (int i = 0; i < 3; ++i) {
    bp[i] = sw(states, a, ob + offsetof(Ball, pos) + 4 * i);
    bv[i] = sw(states, a, ob + offsetof(Ball, vel) + 4 * i);
    f[i] = bp[i] * (1.0f / 4096.0f);
    f[3 + i] = bv[i] * (1.0f / 6000.0f);
    f[6 + i] = sw(states, a, ob + offsetof(Ball, ang_vel) + 4 * i) * (1.0f / 6.0f);
  }
  float cp[2][3], cv[2][3];
  for (int c = 0; c < kCars; ++c) {
    const size_t oc = offsetof(ArenaState, cars) + c * sizeof(Car);
    float* g = f + 9 + 14 * c;
    for (int i = 0; i < 3; ++i) {
      cp[c][i] = sw(states, a, oc + offsetof(Car, pos) + 4 * i);
      cv[c][i] = sw(states, a, oc + offsetof(Car, vel) + 4 * i);
      g[i] = cp[c][i] * (1.0f / 4096.0f);
      g[3 + i] = cv[c][i] * (1.0f / 2300.0f);
      g[6 + i] = sw(states, a, oc + offsetof(Car, ang_vel) + 4 * i) * (1.0f / 5.5f);
      g[9 + i] = sw(states, a, oc + offsetof(Car, rot) + offsetof(M3, c2) + 4 * i);
    }
    g[12] = uw(states, a, oc + offsetof(Car, on_ground)) ? 1.0f : 0.0f;
    g[13] = sw(states, a, oc + offsetof(Car, boost)) * 0.01f;
  }
  auto dist = [](const float* p, const float* q) {
    float dx = p[0] - q[0], dy = p[1] - q[1], dz = p[2] - q[2];
    return sqrtf(dx * dx + dy * dy + dz * dz);
  };
  float dcc = dist(cp[0], cp[1]);
  f[37] = dcc * (1.0f / 4096.0f);
  f[38] = dist(cp[0], bp) * (1.0f / 4096.0f);
  f[39] = dist(cp[1], bp) * (1.0f / 4096.0f);
  f[40] = boundary_dist(bp[0], bp[1], bp[2]) * 0.001f;
  f[41] = boundary_dist(cp[0][0], cp[0][1], cp[0][2]) * 0.001f;
  f[42] = boundary_dist(cp[1][0], cp[1][1], cp[1][2]) * 0.001f;
  for (int c = 0; c < kCars; ++c) {
    float best = 1e30f;
    for (int p = 0; p < kPads; ++p) {
      const V3 q = D.pads[p].pos;
      float pq[3] = {q.x, q.y, q.z};
      best = fminf(best, dist(cp[c], pq));
    }
    f[43 + c] = fminf(best, 4096.0f) * 0.001f;
    f[45 + c] = controls[(size_t)a * kCars + c].jump ? 1.0f : 0.0f;
  }
  float rel = (cv[1][0] - cv[0][0]) * (cp[0][0] - cp[1][0]) + (cv[1][1] - cv[0][1]) * (cp[0][1] - cp[1][1]) +
              (cv[1][2] - cv[0][2]) * (cp[0][2] - cp[1][2]);
  f[47] = rel / fmaxf(dcc, 1.0f) * (1.0f / 2300.0f);
  for (int i = 0; i < kIn; ++i) X[(size_t)a * kIn + i] = __float2bfloat16_rn(f[i]);
}

// ---- labels from the decision's event OR ----
extern "C" __global__ void k_pred_labels(const uint32_t* ev, uint32_t n, uint8_t* Y) {
  uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  uint32_t e = ev[a];
  uint32_t y = (e & 1u) | (e & 2u) | (((e >> 2) & 15u) ? 4u : 0u) | ((e & ((1u << 12) | (1u << 14))) ? 8u : 0u) | (((e >> 10) & 1u) << 4) |
               (((e >> 11) & 1u) << 5);
  Y[a] = (uint8_t)y;
}

// ---- forward: logits[n][8] (FP32); with `save`, the BF16 activations H1, H2, H3 ([3][n][128]) for training ----
extern "C" __global__ void __launch_bounds__(kWarps * 32) k_pred_forward(const __nv_bfloat16* wb, const float* wf, const __nv_bfloat16* X,
                                                                        uint32_t n, float* logits, __nv_bfloat16* save) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem& sm = *reinterpret_cast<Smem*>(smem_raw);
  load_weights(sm, wb, wf);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __nv_bfloat16* A = sm.act[warp][0];
  __nv_bfloat16* B = sm.act[warp][1];
  const uint32_t tiles = (n + 15) / 16;
  for (uint32_t tile = blockIdx.x * kWarps + warp; tile < tiles; tile += gridDim.x * kWarps) {
    const uint32_t r0 = tile * 16;
    const int rows = (int)min(16u, n - r0);
    for (int i = lane; i < 16 * kIn; i += 32) {
      int r = i / kIn, k = i % kIn;
      A[r * sIn + k] = r < rows ? X[(size_t)(r0 + r) * kIn + k] : __float2bfloat16_rn(0.0f);
    }
    __syncwarp();
    __nv_bfloat16* s1 = save ? save + (size_t)r0 * kHid : nullptr;
    __nv_bfloat16* s2 = save ? save + (size_t)n * kHid + (size_t)r0 * kHid : nullptr;
    __nv_bfloat16* s3 = save ? save + (size_t)2 * n * kHid + (size_t)r0 * kHid : nullptr;
    layer_fwd<kIn, kHid, sIn, sIn, true>(A, sm.w1, sm.b1, B, sHid, s1, nullptr, rows);
    layer_fwd<kHid, kHid, sHid, sHid, true>(B, sm.w2, sm.b2, A, sHid, s2, nullptr, rows);
    layer_fwd<kHid, kHid, sHid, sHid, true>(A, sm.w3, sm.b3, B, sHid, s3, nullptr, rows);
    layer_fwd<kHid, kOutPad, sHid, sHid, false>(B, sm.w4, sm.b4, nullptr, 0, nullptr, logits + (size_t)r0 * kOutPad, rows);
  }
}

// ---- Adam on the FP32 master weights, BF16 copy refreshed ----
extern "C" __global__ void k_pred_adam(float* w, __nv_bfloat16* wb, float* m, float* v, const float* grad, uint32_t count, float lr, float b1,
                                       float b2, float eps, float c1, float c2) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  float gr = grad[i];
  float mi = b1 * m[i] + (1.0f - b1) * gr;
  float vi = b2 * v[i] + (1.0f - b2) * gr * gr;
  m[i] = mi;
  v[i] = vi;
  float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  wb[i] = __float2bfloat16_rn(wi);
}

extern "C" __global__ void k_pred_to_bf16(const float* w, __nv_bfloat16* wb, uint32_t count) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) wb[i] = __float2bfloat16_rn(w[i]);
}

// ---- binning: an arena is contact-heavy when any output of `mask` has its logit above `threshold_logit`; the order lists the
// heavy arenas first (longest work first), each bin in arena order.  Two passes over blocks of 1024 arenas. ----
extern "C" __global__ void __launch_bounds__(1024) k_pred_bin_count(const float* logits, uint32_t n, float thr, uint32_t mask,
                                                                   uint32_t* block_heavy) {
  __shared__ uint32_t warp_cnt[32];
  uint32_t a = blockIdx.x * 1024 + threadIdx.x;
  bool heavy = false;
  if (a < n)
    for (int o = 0; o < kOut; ++o) heavy |= ((mask >> o) & 1u) && logits[(size_t)a * kOutPad + o] > thr;
  uint32_t m = __ballot_sync(0xFFFFFFFFu, heavy);
  if ((threadIdx.x & 31) == 0) warp_cnt[threadIdx.x >> 5] = __popc(m);
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t s = 0;
    for (int w = 0; w < 32; ++w) s += warp_cnt[w];
    block_heavy[blockIdx.x] = s;
  }
}

extern "C" __global__ void __launch_bounds__(1024) k_pred_bin_scatter(const float* logits, uint32_t n, float thr, uint32_t mask,
                                                                     const uint32_t* block_heavy, uint32_t nblocks, uint32_t* order,
                                                                     uint32_t* heavy_total) {
  __shared__ uint32_t warp_heavy[32], warp_quiet[32], base[2];
  uint32_t a = blockIdx.x * 1024 + threadIdx.x;
  bool live = a < n, heavy = false;
  if (live)
    for (int o = 0; o < kOut; ++o) heavy |= ((mask >> o) & 1u) && logits[(size_t)a * kOutPad + o] > thr;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t mh = __ballot_sync(0xFFFFFFFFu, live && heavy), mq = __ballot_sync(0xFFFFFFFFu, live && !heavy);
  if (lane == 0) {
    warp_heavy[warp] = __popc(mh);
    warp_quiet[warp] = __popc(mq);
  }
  if (threadIdx.x == 0) {
    uint32_t before = 0, total = 0;
    for (uint32_t b = 0; b < nblocks; ++b) {
      if (b < blockIdx.x) before += block_heavy[b];
      total += block_heavy[b];
    }
    uint32_t first = blockIdx.x * 1024;
    base[0] = before;                               // heavy arenas of earlier blocks
    base[1] = total + (first - before);             // quiet arenas of earlier blocks (all earlier blocks are full)
    if (blockIdx.x == 0) *heavy_total = total;
  }
  __syncthreads();
  if (!live) return;
  uint32_t hb = base[0], qb = base[1];
  for (uint32_t w = 0; w < warp; ++w) {
    hb += warp_heavy[w];
    qb += warp_quiet[w];
  }
  uint32_t below = (1u << lane) - 1u;
  uint32_t at = heavy ? hb + __popc(mh & below) : qb + __popc(mq & below);
  if (at < n) order[at] = a;  // always true when both passes read the same logits
}

// ---- cost levels: an arena's expected contact count e = sum_k w_k * sigmoid(logit_k) over the six outputs, quantised
// to `levels` levels of e / max(e) (the maximum over this batch); the order lists the arenas by level, highest first,
// each level in arena order (a stable counting sort).  Three passes over blocks of 1024 arenas: the maximum, per-block
// level counts, then the scatter. ----
constexpr int kMaxLevels = 32;
struct LevelWeights {
  float w[kOut];
};
__device__ __forceinline__ float expected_contacts(const float* logits, uint32_t a, const LevelWeights& lw) {
  float e = 0.0f;
  for (int o = 0; o < kOut; ++o) e += lw.w[o] / (1.0f + expf(-logits[(size_t)a * kOutPad + o]));
  return e;
}
__device__ __forceinline__ int level_of(float e, float emax, int levels) {
  if (!(emax > 0.0f)) return 0;
  int l = (int)(e / emax * (float)levels);
  return l < 0 ? 0 : (l >= levels ? levels - 1 : l);
}

extern "C" __global__ void __launch_bounds__(1024) k_pred_level_max(const float* logits, uint32_t n, LevelWeights lw, uint32_t* emax_bits) {
  uint32_t a = blockIdx.x * 1024 + threadIdx.x;
  float e = a < n ? expected_contacts(logits, a, lw) : 0.0f;
  for (int d = 16; d > 0; d >>= 1) e = fmaxf(e, __shfl_xor_sync(0xFFFFFFFFu, e, d));
  if ((threadIdx.x & 31) == 0 && e > 0.0f) atomicMax(emax_bits, __float_as_uint(e));  // non-negative floats order as integers
}

extern "C" __global__ void __launch_bounds__(1024) k_pred_level_count(const float* logits, uint32_t n, LevelWeights lw, int levels,
                                                                     const uint32_t* emax_bits, uint32_t* block_hist) {
  __shared__ uint32_t hist[kMaxLevels];
  if (threadIdx.x < kMaxLevels) hist[threadIdx.x] = 0;
  __syncthreads();
  uint32_t a = blockIdx.x * 1024 + threadIdx.x;
  if (a < n) atomicAdd(&hist[level_of(expected_contacts(logits, a, lw), __uint_as_float(*emax_bits), levels)], 1u);
  __syncthreads();
  if (threadIdx.x < (uint32_t)levels) block_hist[(size_t)blockIdx.x * levels + threadIdx.x] = hist[threadIdx.x];
}

extern "C" __global__ void __launch_bounds__(1024) k_pred_level_scatter(const float* logits, uint32_t n, LevelWeights lw, int levels,
                                                                       const uint32_t* emax_bits, const uint32_t* block_hist,
                                                                       uint32_t nblocks, uint32_t* order) {
  __shared__ uint32_t total[kMaxLevels], before[kMaxLevels], base[kMaxLevels], warp_cnt[32][kMaxLevels];
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x < (uint32_t)levels) {
    uint32_t t = 0, b = 0;
    for (uint32_t k = 0; k < nblocks; ++k) {
      uint32_t c = block_hist[(size_t)k * levels + threadIdx.x];
      t += c;
      if (k < blockIdx.x) b += c;
    }
    total[threadIdx.x] = t;
    before[threadIdx.x] = b;
  }
  __syncthreads();
  if (threadIdx.x < (uint32_t)levels) {
    uint32_t higher = 0;  // arenas of the levels above, which come first
    for (int l = levels - 1; l > (int)threadIdx.x; --l) higher += total[l];
    base[threadIdx.x] = higher + before[threadIdx.x];
  }
  const uint32_t a = blockIdx.x * 1024 + threadIdx.x;
  const bool live = a < n;
  const int lv = live ? level_of(expected_contacts(logits, a, lw), __uint_as_float(*emax_bits), levels) : -1;
  uint32_t mine = 0;
  for (int l = 0; l < levels; ++l) {
    uint32_t m = __ballot_sync(0xFFFFFFFFu, lv == l);
    if (lane == 0) warp_cnt[warp][l] = __popc(m);
    if (lv == l) mine = m;
  }
  __syncthreads();
  if (!live) return;
  uint32_t at = base[lv];
  for (uint32_t w = 0; w < warp; ++w) at += warp_cnt[w][lv];
  at += __popc(mine & ((1u << lane) - 1u));
  if (at < n) order[at] = a;  // always true when all three passes read the same logits
}

// ---- launchers ----
static size_t pred_smem() { return sizeof(Smem); }

cudaError_t rsx_launch_pred_features(const uint32_t* states, const void* sds, const uint8_t* sd_index, const void* controls, uint32_t n,
                                     void* X, cudaStream_t s) {
  k_pred_features<<<(n + 127) / 128, 128, 0, s>>>(states, (const StaticData*)sds, sd_index, (const Controls*)controls, n, (__nv_bfloat16*)X);
  return cudaGetLastError();
}
cudaError_t rsx_launch_pred_labels(const uint32_t* ev, uint32_t n, uint8_t* Y, cudaStream_t s) {
  k_pred_labels<<<(n + 255) / 256, 256, 0, s>>>(ev, n, Y);
  return cudaGetLastError();
}
// the shared-memory opt-in of the forward / backward kernels, once per process and device (kept out of the launch path,
// so that launches can be captured into CUDA graphs)
static cudaError_t set_smem(const void* fn) {
  static int done[64];
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev >= 0 && dev < 64 && done[dev]) return cudaSuccess;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pred_smem());
  if (e == cudaSuccess && dev >= 0 && dev < 64) done[dev] = 1;
  return e;
}
cudaError_t rsx_launch_pred_forward(const void* wb, const float* wf, const void* X, uint32_t n, float* logits, void* save, cudaStream_t s) {
  cudaError_t e = set_smem((const void*)k_pred_forward);
  if (e != cudaSuccess) return e;
  uint32_t tiles = (n + 15) / 16, grid = min((tiles + kWarps - 1) / kWarps, 148u * 4u);
  k_pred_forward<<<grid, kWarps * 32, pred_smem(), s>>>((const __nv_bfloat16*)wb, wf, (const __nv_bfloat16*)X, n, logits, (__nv_bfloat16*)save);
  return cudaGetLastError();
}
cudaError_t rsx_launch_pred_adam(float* w, void* wb, float* m, float* v, const float* grad, float lr, float b1, float b2, float eps, float c1,
                                 float c2, cudaStream_t s) {
  k_pred_adam<<<(kParams + 255) / 256, 256, 0, s>>>(w, (__nv_bfloat16*)wb, m, v, grad, kParams, lr, b1, b2, eps, c1, c2);
  return cudaGetLastError();
}
cudaError_t rsx_launch_pred_to_bf16(const float* w, void* wb, cudaStream_t s) {
  k_pred_to_bf16<<<(kParams + 255) / 256, 256, 0, s>>>(w, (__nv_bfloat16*)wb, kParams);
  return cudaGetLastError();
}
cudaError_t rsx_launch_pred_levels(const float* logits, uint32_t n, const float* weights, int levels, uint32_t* scratch, uint32_t* order,
                                   cudaStream_t s) {
  LevelWeights lw;
  for (int o = 0; o < kOut; ++o) lw.w[o] = weights[o];
  const uint32_t nb = (n + 1023) / 1024;
  cudaError_t e = cudaMemsetAsync(scratch, 0, 4, s);
  if (e != cudaSuccess) return e;
  k_pred_level_max<<<nb, 1024, 0, s>>>(logits, n, lw, scratch);
  k_pred_level_count<<<nb, 1024, 0, s>>>(logits, n, lw, levels, scratch, scratch + 1);
  k_pred_level_scatter<<<nb, 1024, 0, s>>>(logits, n, lw, levels, scratch, scratch + 1, nb, order);
  return cudaGetLastError();
}
cudaError_t rsx_launch_pred_bin(const float* logits, uint32_t n, float thr, uint32_t mask, uint32_t* block_scratch, uint32_t* order,
                                uint32_t* heavy_total, cudaStream_t s) {
  uint32_t nb = (n + 1023) / 1024;
  k_pred_bin_count<<<nb, 1024, 0, s>>>(logits, n, thr, mask, block_scratch);
  k_pred_bin_scatter<<<nb, 1024, 0, s>>>(logits, n, thr, mask, block_scratch, nb, order, heavy_total);
  return cudaGetLastError();
}
