// Arena resets on the device: fresh seeded start states written into the AoSoA-32 buffer for the arenas a caller marks
// (or those whose last decision scored a goal), so a rollout can restart its finished episodes without a round trip to
// the host.  The states are the host generator's (sim/start.cuh) for the same (seed, arena index, StaticData), word
// for word.  No counterpart kernel in the reference (its on-device reset helpers are referenced but absent).
#include "kern_common.cuh"
#include "sim/start.cuh"

struct Mix5 {
  float v[5];
};

extern "C" __global__ void __launch_bounds__(64) k_reset_arenas(uint32_t* states, uint32_t n, const StaticData* sds, const uint8_t* sd_index,
                                                                uint64_t seed, Mix5 mix, const uint32_t* result, const uint8_t* mask,
                                                                uint32_t* reset_count) {
  uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  bool go = true;
  if (mask) go = mask[a] != 0;
  if (result) go = go && (result[a] & kScoredMask) != 0;
  if (!go) return;
  ArenaState s;
  world::make_state(sds[sd_index ? sd_index[a] : 0], s, a, seed, mix.v);
  const uint32_t* d = reinterpret_cast<const uint32_t*>(&s);
  uint32_t* dst = states + (size_t)(a / kLanes) * aosoa_block_words() + (a % kLanes);
  for (int w = 0; w < kArenaWords; ++w) dst[(size_t)w * kLanes] = d[w];
  if (reset_count) atomicAdd(reset_count, 1u);
}

cudaError_t rsx_launch_reset_arenas(uint32_t* states, uint32_t n, const void* sds, const uint8_t* sd_index, uint64_t seed, const float* mix,
                                    const uint32_t* result, const uint8_t* mask, uint32_t* reset_count, cudaStream_t s) {
  Mix5 m;
  for (int k = 0; k < 5; ++k) m.v[k] = mix[k];
  k_reset_arenas<<<(n + 63) / 64, 64, 0, s>>>(states, n, (const StaticData*)sds, sd_index, seed, m, result, mask, reset_count);
  return cudaGetLastError();
}
