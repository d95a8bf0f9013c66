// Device helpers shared by the decision kernels: the AoSoA-32 copy-in / copy-out of one arena's tick-boundary words,
// the tick hooks (goal store, per-tick trace, event OR) and one decision of one arena.  Every kernel translation unit
// includes this and the simulator, and compiles them into its own module (the build runs them in parallel).
#pragma once
#include <cuda_runtime.h>
#include "../../include/rsx.h"
#include "state.cuh"
#include "sim/physics.cuh"

using namespace rsx;

namespace {

constexpr int kMaxBlock = 64;

// (unrolled 32 deep: the copy is a chain of dependent-latency groups, one group of loads in flight at a time)
__device__ __forceinline__ void load_tick(ArenaState* s, const uint32_t* buf, uint32_t a) {
  uint32_t* d = reinterpret_cast<uint32_t*>(s);
  const uint32_t* src = buf + (size_t)(a / kLanes) * aosoa_block_words() + (a % kLanes);
#pragma unroll 32
  for (int w = 0; w < kTickWords; ++w) d[w] = src[(size_t)w * kLanes];
#pragma unroll 8
  for (int w = kTickWords; w < kArenaWords; ++w) d[w] = 0u;
}
__device__ __forceinline__ void store_tick(uint32_t* buf, uint32_t a, const ArenaState* s) {
  const uint32_t* d = reinterpret_cast<const uint32_t*>(s);
  uint32_t* dst = buf + (size_t)(a / kLanes) * aosoa_block_words() + (a % kLanes);
#pragma unroll 32
  for (int w = 0; w < kTickWords; ++w) dst[(size_t)w * kLanes] = d[w];
}

struct GoalStore {
  uint32_t* states;
  uint32_t a;
  bool* ovf;
  __device__ void operator()(uint32_t, const ArenaState& s) const {
    store_tick(states, a, &s);
    *ovf = sim::any_overflow(s);
  }
};
struct TraceStore {
  uint32_t* trace;
  size_t words;
  uint32_t a;
  __device__ void operator()(uint32_t t, const ArenaState& s) const {
    if (trace) store_tick(trace + (size_t)(t - 1) * words, a, &s);
  }
};
struct EventOr {
  uint32_t* acc;
  __device__ void operator()(uint32_t, const ArenaState& s) const { *acc |= s.events; }
};

// one decision of arena a (state in the buffer at index a); returns the result word
__device__ __forceinline__ uint32_t decide_arena(uint32_t* states, const StaticData& D, const Controls* controls, uint32_t a,
                                                  uint32_t* trace, size_t trace_words, uint32_t* ev_out) {
  ArenaState s;
  load_tick(&s, states, a);
  Controls ctl[kCars];
  ctl[0] = controls[(size_t)a * kCars];
  ctl[1] = controls[(size_t)a * kCars + 1];
  bool ovf = false;
  uint32_t ev = 0;
  uint32_t r;
  if (trace) {
    r = sim::decide(s, D, ctl, kTicksPerDecision, GoalStore{states, a, &ovf}, TraceStore{trace, trace_words, a});
  } else {
    r = sim::decide(s, D, ctl, kTicksPerDecision, GoalStore{states, a, &ovf}, EventOr{&ev});
  }
  if ((r & kScoredMask) == 0) {
    store_tick(states, a, &s);
    ovf = sim::any_overflow(s);
  }
  if (ev_out) ev_out[a] = ev;
  return r | (ovf ? kOverflow : 0u);
}

// The claim loop of the persistent kernels without barriers: each warp takes 32 * gran consecutive entries of `order`
// (arena indices; identity when null) with one atomicAdd on `counter` (zero at launch) until a claim starts past n, and
// runs `arena(a)` for each entry below n whose arena index is below n.  The counter overshoots n by at most gridDim.x * blockDim.x * gran, which the
// launchers keep below 2^32 - n.
template <class Arena>
__device__ __forceinline__ void persistent_claims(uint32_t* counter, uint32_t n, uint32_t gran, const uint32_t* order, const Arena& arena) {
  const uint32_t lane = threadIdx.x & 31u;
  for (;;) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(counter, 32u * gran);
    base = __shfl_sync(0xFFFFFFFFu, base, 0);
    if (base >= n) break;
    for (uint32_t g = 0; g < gran; ++g) {
      uint32_t i = base + g * 32u + lane;
      uint32_t a = i < n ? (order ? order[i] : i) : n;
      if (a < n) arena(a);  // an order entry past n (not a permutation) is skipped, never dereferenced
    }
  }
}

}  // namespace

