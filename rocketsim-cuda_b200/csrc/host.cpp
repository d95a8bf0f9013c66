// Host-side entry points of the C ABI (include/rsx.h): layout queries, AoSoA pack / unpack, the synthetic world and
// start states, and the simulator's host build for debugging.  Compiled with -ffp-contract=off and no FMA target, so
// the host build computes the same bits as the device.
#include <string.h>
#include "../../include/rsx.h"
#include "state.cuh"
#include "sim/physics.cuh"
#include "sim/start.cuh"

namespace rsx {
namespace world {
int build_static(StaticData* sd, uint64_t seed, int preset0, int preset1);
void make_states(const StaticData& sd, ArenaState* out, uint32_t n, uint64_t seed, const float* mix);
void make_states_multi(const StaticData* sds, const uint8_t* idx, ArenaState* out, uint32_t n, uint64_t seed, const float* mix);
}  // namespace world
}  // namespace rsx

using namespace rsx;

extern "C" {

uint64_t rsx_arena_words(void) { return kArenaWords; }
uint64_t rsx_tick_words(void) { return kTickWords; }
uint64_t rsx_static_words(void) { return kStaticWords; }
uint64_t rsx_aosoa_words(uint32_t n) { return aosoa_words(n); }
uint64_t rsx_aosoa_index(uint32_t a, uint32_t w) { return aosoa_index(a, (int)w); }

void rsx_aosoa_pack(const uint32_t* states, uint32_t n, uint32_t* out) {
  memset(out, 0, aosoa_words(n) * 4);
  for (uint32_t a = 0; a < n; ++a)
    for (int w = 0; w < kArenaWords; ++w) out[aosoa_index(a, w)] = states[(size_t)a * kArenaWords + w];
}
void rsx_aosoa_unpack(const uint32_t* in, uint32_t n, uint32_t* states) {
  for (uint32_t a = 0; a < n; ++a)
    for (int w = 0; w < kArenaWords; ++w) states[(size_t)a * kArenaWords + w] = in[aosoa_index(a, w)];
}

int rsx_build_static(uint32_t* words, uint64_t seed, int preset0, int preset1) {
  if (!words || preset0 < 0 || preset0 > 6 || preset1 < 0 || preset1 > 6) return RSX_E_ARG;
  int r = world::build_static(reinterpret_cast<StaticData*>(words), seed, preset0, preset1);
  return r < 0 ? RSX_E_ARG : r;
}

int rsx_make_states(const uint32_t* static_words, uint32_t* states, uint32_t n, uint64_t seed, const float* mix) {
  if (!static_words || !states || !mix) return RSX_E_ARG;
  world::make_states(*reinterpret_cast<const StaticData*>(static_words), reinterpret_cast<ArenaState*>(states), n, seed, mix);
  return RSX_OK;
}

int rsx_make_states_multi(const uint32_t* statics, uint32_t count, const uint8_t* sd_index, uint32_t* states, uint32_t n, uint64_t seed,
                          const float* mix) {
  if (!statics || !sd_index || !states || !mix) return RSX_E_ARG;
  for (uint32_t a = 0; a < n; ++a)
    if (sd_index[a] >= count) return RSX_E_ARG;
  world::make_states_multi(reinterpret_cast<const StaticData*>(statics), sd_index, reinterpret_cast<ArenaState*>(states), n, seed, mix);
  return RSX_OK;
}

int rsx_pad_mirror(const uint32_t* statics, uint32_t count, uint8_t* out) {
  if (!statics || !out) return RSX_E_ARG;
  for (uint32_t k = 0; k < count; ++k) {
    const StaticData& sd = reinterpret_cast<const StaticData*>(statics)[k];
    for (int p = 0; p < kPads; ++p) {
      const V3 m = V3{-sd.pads[p].pos.x, -sd.pads[p].pos.y, sd.pads[p].pos.z};
      int q = p;  // a pad with no mirror image keeps its own place
      for (int j = 0; j < kPads; ++j)
        if (sd.pads[j].pos.x == m.x && sd.pads[j].pos.y == m.y && sd.pads[j].pos.z == m.z) {
          q = j;
          break;
        }
      out[(size_t)k * kPads + p] = (uint8_t)q;
    }
  }
  return RSX_OK;
}

int rsx_make_states_at(const uint32_t* statics, uint32_t count, const uint8_t* sd_index, const uint32_t* arena_index, uint32_t k,
                       uint64_t seed, const float* mix, uint32_t* states) {
  if (!statics || !sd_index || !arena_index || !states || !mix) return RSX_E_ARG;
  for (uint32_t j = 0; j < k; ++j)
    if (sd_index[j] >= count) return RSX_E_ARG;
  const StaticData* sds = reinterpret_cast<const StaticData*>(statics);
  ArenaState* out = reinterpret_cast<ArenaState*>(states);
  for (uint32_t j = 0; j < k; ++j) world::make_state(sds[sd_index[j]], out[j], arena_index[j], seed, mix);
  return RSX_OK;
}

int rsx_host_phase(int k, uint32_t* state_words, const uint32_t* static_words) {
  return sim::run_phase(k, *reinterpret_cast<ArenaState*>(state_words), *reinterpret_cast<const StaticData*>(static_words));
}

uint32_t rsx_host_decide(uint32_t* state_words, const uint32_t* static_words, const rsx_controls* controls2) {
  ArenaState& S = *reinterpret_cast<ArenaState*>(state_words);
  const StaticData& D = *reinterpret_cast<const StaticData*>(static_words);
  static thread_local ArenaState goal;
  bool have_goal = false;
  uint32_t r = sim::decide(
      S, D, reinterpret_cast<const Controls*>(controls2), kTicksPerDecision,
      [&](uint32_t, const ArenaState& s) {
        goal = s;
        have_goal = true;
      },
      sim::NoHook{});
  if (have_goal) S = goal;
  return r | (sim::any_overflow(S) ? kOverflow : 0u);
}

}  // extern "C"
