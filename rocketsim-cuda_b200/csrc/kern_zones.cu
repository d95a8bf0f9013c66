// Zone-timer build of the lockstep decision (profiling only; not part of librsx.so).  Built with RSX_ZONES by
// `make zones` into librsx_zones.so (phase-level zones: RSX_ZONES_MIN=40) and librsx_zones_all.so (every zone marker in
// the simulator, which inflates the enclosing phases by the markers' own cost).  Zone ids: 0-39 the simulator's
// markers (sim/car.cuh, sim/ray.cuh, sim/narrow.cuh), 40 + k phase k's body, 50 + k the barrier after phase k,
// 60 / 61 the copy-in / copy-out of the tick words.  The sums are warp cycles (clock64) per zone over all warps.
#include <stdio.h>
#include <cuda_runtime.h>
#include <stdint.h>
__device__ unsigned long long rsx_zone_acc[148 * 16][64];
#include "kern_common.cuh"

__global__ void __launch_bounds__(448, 1) k_sim8_zones(uint32_t* states, const StaticData* sds, const uint8_t* sd_index,
                                                      const Controls* controls, uint32_t* result, uint32_t* ev_or, uint32_t* counter,
                                                      uint32_t n) {
  const uint32_t lane = threadIdx.x & 31u;
  ArenaState s;
  Controls c0, c1;
  const StaticData* D = sds;
  uint32_t a = 0, t = 0, scored = 0, unimpl = 0, ev = 0;
  bool live = false, have = false, ovf = false;
  for (;;) {
    if (!have) {
      uint32_t base = 0;
      if (lane == 0) base = atomicAdd(counter, 32u);
      base = __shfl_sync(0xFFFFFFFFu, base, 0);
      if (base < n) {
        uint32_t i = base + lane;
        live = i < n;
        a = live ? i : base;
        D = sds + (sd_index ? sd_index[a] : 0);
        RSX_ZONE_BEGIN(zl);
        load_tick(&s, states, a);
        RSX_ZONE_END(zl, 60);
        c0 = controls[(size_t)a * kCars];
        c1 = controls[(size_t)a * kCars + 1];
        t = 1;
        scored = unimpl = ev = 0;
        ovf = false;
        have = true;
      }
    }
    if (!__syncthreads_or(have)) break;
    int un = 0;
    if (have) {
      s.cars[0].controls = c0;
      s.cars[1].controls = c1;
    }
#pragma unroll 1
    for (int k = 0; k < sim::kPhases; ++k) {
      if (have) {
        RSX_ZONE_BEGIN(zp);
        if (sim::run_phase(k, s, *D) != sim::PHASE_OK) un = 1;
        RSX_ZONE_END(zp, 40 + k);
      }
      RSX_ZONE_BEGIN(zb);
      __syncthreads();
      RSX_ZONE_END(zb, 50 + k);
    }
    if (have) {
      if (scored == 0) {
        if (un) unimpl = kUnimplemented;
        ev |= s.events;
        if (sim::ball_scored(s, *D)) {
          scored = t;
          if (live) store_tick(states, a, &s);
          ovf = sim::any_overflow(s);
        }
      }
      if (t == kTicksPerDecision) {
        RSX_ZONE_BEGIN(zs);
        if (scored == 0) {
          if (live) store_tick(states, a, &s);
          ovf = sim::any_overflow(s);
        }
        RSX_ZONE_END(zs, 61);
        if (live) {
          if (ev_or) ev_or[a] = ev;
          result[a] = scored | unimpl | (ovf ? kOverflow : 0u);
        }
        have = false;
      }
      ++t;
    }
  }
}

// one decision with zone timers; zone_cycles[64] receives the sums over all warps.  Synchronous.
extern "C" int rsx_zones_decision(uint32_t* d_states, uint32_t n, const void* d_statics, const uint8_t* d_sd_index, const void* d_controls,
                                  uint32_t* d_result, uint32_t* d_counter, unsigned long long* zone_cycles) {
  static unsigned long long acc[148 * 16][64];
  memset(acc, 0, sizeof(acc));
  if (cudaMemcpyToSymbol(rsx_zone_acc, acc, sizeof(acc)) != cudaSuccess) return -2;
  if (cudaMemset(d_counter, 0, 4) != cudaSuccess) return -2;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  k_sim8_zones<<<sms < 148 ? sms : 148, 448>>>(d_states, (const StaticData*)d_statics, d_sd_index, (const Controls*)d_controls, d_result,
                                               nullptr, d_counter, n);
  if (cudaDeviceSynchronize() != cudaSuccess) return -2;
  if (cudaMemcpyFromSymbol(acc, rsx_zone_acc, sizeof(acc)) != cudaSuccess) return -2;
  for (int z = 0; z < 64; ++z) {
    zone_cycles[z] = 0;
    for (int w = 0; w < 148 * 16; ++w) zone_cycles[z] += acc[w][z];
  }
  return 0;
}
