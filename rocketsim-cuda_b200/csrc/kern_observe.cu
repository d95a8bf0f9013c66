// Observations and rewards for a learner, straight from the AoSoA-32 state buffer: one FP16 row of kObsDim values
// and one FP32 reward per car, written after a decision so a policy and a trainer read them without the states ever
// leaving the device.  The reference defines no observation (its training loop is not part of it; it ships only the
// FP16 conversion such a kernel uses, cuda/common/hd.cuh:167-176: round to nearest even, as cvt.rn.f16.f32); the
// layout below is this library's, fixed in include/rsx.h.
//
// Per car c (the opponent is o = 1 - c), seen from c's side: car 1's values are turned 180 degrees about z (x and y
// negated, exact) and its pads listed in mirrored order, so both cars see themselves attacking +y.  Positions and
// velocities are scaled by 1/2300, angular velocities by 1/pi, boost by 1/100; differences are taken before scaling.
// Every value is one FP32 operation sequence in a fixed order (explicit _rn intrinsics), then rounded once to FP16.
//
// One thread per arena, both cars; each warp assembles its 64 rows in shared memory and stores them as 16-byte
// vectors, so the row-major output is written with whole sectors.
#include <cuda_fp16.h>
#include "state.cuh"

using namespace rsx;

namespace {

constexpr int kObsDim = 104;          // FP16 values per car row (208 bytes, 13 x 16)
constexpr int kRewardTerms = 8;
constexpr float kPosScale = 1.0f / 2300.0f;
constexpr float kAngScale = 0.318309886183790671538f;  // 1/pi, rounded to FP32
constexpr float kBoostScale = 0.01f;
constexpr int kWarps = 2;             // warps per block (64 arenas)

struct Weights {
  float w[kRewardTerms];
};

struct Rd {
  const uint32_t* base;  // word 0 of this arena (lane-strided)
  __device__ uint32_t u(size_t w) const { return base[w * kLanes]; }
  __device__ float f(size_t w) const { return __uint_as_float(base[w * kLanes]); }
};

#define W_OF(field) (offsetof(ArenaState, field) / 4)

struct CarWords {
  size_t at;
  __device__ explicit CarWords(int c) : at(offsetof(ArenaState, cars) / 4 + (size_t)c * (sizeof(Car) / 4)) {}
  __device__ size_t w(size_t car_off) const { return at + car_off / 4; }
};

// the view of one value from car `side`: x and y negated for car 1
__device__ __forceinline__ float sx(float v, int side) { return side ? -v : v; }

struct V3f {
  float x, y, z;
};

__device__ __forceinline__ V3f load3(const Rd& r, size_t w) { return V3f{r.f(w), r.f(w + 1), r.f(w + 2)}; }

__device__ __forceinline__ void put3(__half* row, int k, V3f v, int side, float scale) {
  row[k] = __float2half_rn(__fmul_rn(sx(v.x, side), scale));
  row[k + 1] = __float2half_rn(__fmul_rn(sx(v.y, side), scale));
  row[k + 2] = __float2half_rn(__fmul_rn(v.z, scale));
}

__device__ __forceinline__ void put_diff3(__half* row, int k, V3f a, V3f b, int side, float scale) {
  row[k] = __float2half_rn(__fmul_rn(sx(__fsub_rn(a.x, b.x), side), scale));
  row[k + 1] = __float2half_rn(__fmul_rn(sx(__fsub_rn(a.y, b.y), side), scale));
  row[k + 2] = __float2half_rn(__fmul_rn(__fsub_rn(a.z, b.z), scale));
}

__device__ __forceinline__ float flag01(uint32_t v) { return v ? 1.0f : 0.0f; }

}  // namespace

extern "C" __global__ void __launch_bounds__(kWarps * 32) k_observe(const uint32_t* __restrict__ states, uint32_t n,
                                                                    const StaticData* __restrict__ sds, const uint8_t* __restrict__ sd_index,
                                                                    const uint8_t* __restrict__ pad_mirror, const uint32_t* __restrict__ result,
                                                                    const uint32_t* __restrict__ event_or, Weights wt, __half* __restrict__ obs,
                                                                    float* __restrict__ reward) {
  __shared__ __align__(16) __half rows[kWarps][64 * kObsDim];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t a0 = (blockIdx.x * kWarps + warp) * 32;
  if (a0 >= n) return;
  const uint32_t a = a0 + lane;
  const bool live = a < n;
  if (live) {
    Rd r{states + (size_t)(a / kLanes) * aosoa_block_words() + (a % kLanes)};
    const uint32_t si = sd_index ? sd_index[a] : 0u;
    const StaticData& D = sds[si];
    const V3f bpos = load3(r, W_OF(ball.pos)), bvel = load3(r, W_OF(ball.vel)), bang = load3(r, W_OF(ball.ang_vel));
    const int64_t tick = (int64_t)((uint64_t)r.u(W_OF(tick_count.hi)) << 32 | r.u(W_OF(tick_count.lo)));
    // pad activity, the game's own test (P8): active unless it gave boost less than its cooldown ago
    uint64_t active = 0;
    for (int p = 0; p < kPads; ++p) {
      size_t w = W_OF(pad_gave) + (size_t)p * (sizeof(Opt<U64W>) / 4);
      bool on = true;
      if (r.u(w)) {
        int64_t last = (int64_t)((uint64_t)r.u(w + 2) << 32 | r.u(w + 1));
        on = !(__fmul_rn(ll2f(tick - last), 1.0f / 120.0f) < D.pads[p].cooldown);
      }
      active |= (uint64_t)on << p;
    }
    const uint32_t res = result ? result[a] : 0u;
    const uint32_t ev = event_or ? event_or[a] : 0u;
    for (int c = 0; c < kCars; ++c) {
      const int o = 1 - c, side = c;
      const CarWords cs(c), co(o);
      __half* row = &rows[warp][(lane * 2 + c) * kObsDim];
      const V3f pos = load3(r, cs.w(offsetof(Car, pos))), vel = load3(r, cs.w(offsetof(Car, vel)));
      const V3f ang = load3(r, cs.w(offsetof(Car, ang_vel)));
      const V3f fwd = load3(r, cs.w(offsetof(Car, rot) + offsetof(M3, c0))), up = load3(r, cs.w(offsetof(Car, rot) + offsetof(M3, c2)));
      const V3f opos = load3(r, co.w(offsetof(Car, pos))), ovel = load3(r, co.w(offsetof(Car, vel)));
      const V3f oang = load3(r, co.w(offsetof(Car, ang_vel)));
      const V3f ofwd = load3(r, co.w(offsetof(Car, rot) + offsetof(M3, c0))), oup = load3(r, co.w(offsetof(Car, rot) + offsetof(M3, c2)));
      put3(row, 0, bpos, side, kPosScale);
      put3(row, 3, bvel, side, kPosScale);
      put3(row, 6, bang, side, kAngScale);
      put3(row, 9, pos, side, kPosScale);
      put3(row, 12, fwd, side, 1.0f);
      put3(row, 15, up, side, 1.0f);
      put3(row, 18, vel, side, kPosScale);
      put3(row, 21, ang, side, kAngScale);
      row[24] = __float2half_rn(__fmul_rn(r.f(cs.w(offsetof(Car, boost))), kBoostScale));
      row[25] = __float2half_rn(flag01(r.u(cs.w(offsetof(Car, on_ground)))));
      row[26] = __float2half_rn(flag01(r.u(cs.w(offsetof(Car, has_jumped)))));
      row[27] = __float2half_rn(flag01(r.u(cs.w(offsetof(Car, has_double_jumped)))));
      row[28] = __float2half_rn(flag01(r.u(cs.w(offsetof(Car, has_flipped)))));
      row[29] = __float2half_rn(flag01(r.u(cs.w(offsetof(Car, is_demoed)))));
      put_diff3(row, 30, bpos, pos, side, kPosScale);
      put_diff3(row, 33, bvel, vel, side, kPosScale);
      put3(row, 36, opos, side, kPosScale);
      put3(row, 39, ofwd, side, 1.0f);
      put3(row, 42, oup, side, 1.0f);
      put3(row, 45, ovel, side, kPosScale);
      put3(row, 48, oang, side, kAngScale);
      row[51] = __float2half_rn(__fmul_rn(r.f(co.w(offsetof(Car, boost))), kBoostScale));
      row[52] = __float2half_rn(flag01(r.u(co.w(offsetof(Car, on_ground)))));
      row[53] = __float2half_rn(flag01(r.u(co.w(offsetof(Car, is_demoed)))));
      put_diff3(row, 54, opos, pos, side, kPosScale);
      put_diff3(row, 57, ovel, vel, side, kPosScale);
      const size_t ctl = cs.w(offsetof(Car, controls));
      for (int k = 0; k < 5; ++k) row[60 + k] = __float2half_rn(r.f(ctl + k));
      for (int k = 5; k < 8; ++k) row[60 + k] = __float2half_rn(flag01(r.u(ctl + k)));
      for (int p = 0; p < kPads; ++p) {
        int q = (side && pad_mirror) ? pad_mirror[si * kPads + p] : p;
        row[68 + p] = __float2half_rn((active >> q & 1u) ? 1.0f : 0.0f);
      }
      row[102] = row[103] = __float2half_rn(0.0f);

      // reward terms: goal, touch, bump given, demo given, demoed, boost pickup, speed toward the ball, ball speed
      // toward the opponent's goal (team 0 attacks +y)
      const uint32_t team = D.cars[c].team;
      const bool scored = (res & kScoredMask) != 0u;
      const float goal = scored ? (((bpos.y > 0.0f) == (team == 0u)) ? 1.0f : -1.0f) : 0.0f;
      const float dx = __fsub_rn(bpos.x, pos.x), dy = __fsub_rn(bpos.y, pos.y), dz = __fsub_rn(bpos.z, pos.z);
      const float len = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)));
      const float dot = __fadd_rn(__fadd_rn(__fmul_rn(vel.x, dx), __fmul_rn(vel.y, dy)), __fmul_rn(vel.z, dz));
      const float toward = len > 0.0f ? __fmul_rn(__fdiv_rn(dot, len), kPosScale) : 0.0f;
      const float ball_goal = __fmul_rn(team == 0u ? bvel.y : -bvel.y, kPosScale);
      const float term[kRewardTerms] = {goal,
                                        flag01(ev >> (EV_CAR_HIT_BALL + c) & 1u),
                                        flag01(ev >> (EV_BUMP + o) & 1u),
                                        flag01(ev >> (EV_DEMO + o) & 1u),
                                        flag01(ev >> (EV_DEMO + c) & 1u),
                                        flag01(ev >> (EV_PICKUP + c) & 1u),
                                        toward,
                                        ball_goal};
      float total = __fmul_rn(wt.w[0], term[0]);
      for (int k = 1; k < kRewardTerms; ++k) total = __fadd_rn(total, __fmul_rn(wt.w[k], term[k]));
      if (reward) reward[(size_t)a * 2 + c] = total;
    }
  }
  __syncwarp();
  // the warp's rows are contiguous in the output: 16-byte stores across the lanes
  const uint32_t rows_here = 2u * ((n - a0) < 32u ? (n - a0) : 32u);
  const int4* src = reinterpret_cast<const int4*>(rows[warp]);
  int4* dst = reinterpret_cast<int4*>(obs + (size_t)a0 * 2 * kObsDim);
  const uint32_t vecs = rows_here * (kObsDim * 2 / 16);
  for (uint32_t k = lane; k < vecs; k += 32) dst[k] = src[k];
}

cudaError_t rsx_launch_observe(const uint32_t* states, uint32_t n, const void* sds, const uint8_t* sd_index, const uint8_t* pad_mirror,
                               const uint32_t* result, const uint32_t* event_or, const float* weights, uint16_t* obs, float* reward,
                               cudaStream_t s) {
  Weights w;
  for (int k = 0; k < kRewardTerms; ++k) w.w[k] = weights ? weights[k] : 0.0f;
  const uint32_t per_block = kWarps * 32;
  k_observe<<<(n + per_block - 1) / per_block, per_block, 0, s>>>(states, n, (const StaticData*)sds, sd_index, pad_mirror, result, event_or,
                                                                   w, reinterpret_cast<__half*>(obs), reward);
  return cudaGetLastError();
}
