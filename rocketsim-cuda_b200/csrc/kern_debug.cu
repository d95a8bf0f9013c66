// Per-tick and per-phase kernels and the layout round trip (the reference's sim.cu:9-53: sim_identity[_tick], phase_k,
// step_tick_k).
#include "kern_common.cuh"

extern "C" __global__ void k_identity(const uint32_t* in, uint32_t* out, uint32_t n, int tick_only) {
  uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  ArenaState s;
  uint32_t* d = reinterpret_cast<uint32_t*>(&s);
  int words = tick_only ? kTickWords : kArenaWords;
  for (int w = 0; w < kArenaWords; ++w) d[w] = w < words ? in[aosoa_index(a, w)] : 0u;
  for (int w = 0; w < words; ++w) out[aosoa_index(a, w)] = d[w];
}

extern "C" __global__ void __launch_bounds__(128) k_phase(int k, uint32_t* buf, const StaticData* sd, uint32_t n, int32_t* status) {
  uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  ArenaState s;
  uint32_t* d = reinterpret_cast<uint32_t*>(&s);
  for (int w = 0; w < kArenaWords; ++w) d[w] = buf[aosoa_index(a, w)];
  status[a] = sim::run_phase(k, s, *sd);
  for (int w = 0; w < kArenaWords; ++w) buf[aosoa_index(a, w)] = d[w];
}

extern "C" __global__ void __launch_bounds__(kMaxBlock, 1) k_step_tick(uint32_t* buf, const StaticData* sd, uint32_t n, int32_t* status) {
  uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  ArenaState s;
  load_tick(&s, buf, a);
  status[a] = sim::step_tick(s, *sd);
  store_tick(buf, a, &s);
}

cudaError_t rsx_launch_identity(const uint32_t* in, uint32_t* out, uint32_t n, int tick_only, cudaStream_t s) {
  k_identity<<<(n + 127) / 128, 128, 0, s>>>(in, out, n, tick_only);
  return cudaGetLastError();
}
cudaError_t rsx_launch_phase(int k, uint32_t* buf, const void* sd, uint32_t n, int32_t* status, cudaStream_t s) {
  k_phase<<<(n + 127) / 128, 128, 0, s>>>(k, buf, (const StaticData*)sd, n, status);
  return cudaGetLastError();
}
cudaError_t rsx_launch_step_tick(uint32_t* buf, const void* sd, uint32_t n, int32_t* status, cudaStream_t s) {
  k_step_tick<<<(n + 31) / 32, 32, 0, s>>>(buf, (const StaticData*)sd, n, status);
  return cudaGetLastError();
}

// Phase profile of one decision: the tick loop of decide() with clock64() read around each of the ten phases.  Lane 0
// of every warp adds its warp's cycles per phase to prof[0..9] (cycles the warp spent in the phase, all lanes together,
// so the shares show where the decision's time goes).  Lanes past n step the last arena and store nothing, so the warp
// keeps its shape.  Tick-boundary words are written back as by the decision kernels (goal state not kept: profiling only).
extern "C" __global__ void __launch_bounds__(kMaxBlock, 1) k_sim8_profile(uint32_t* states, const StaticData* sds, const uint8_t* sd_index,
                                                                          const Controls* controls, uint32_t n,
                                                                          unsigned long long* prof) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (blockIdx.x * blockDim.x >= n) return;
  uint32_t a = i < n ? i : n - 1;
  const StaticData& D = sds[sd_index ? sd_index[a] : 0];
  ArenaState s;
  load_tick(&s, states, a);
  unsigned long long acc[sim::kPhases];
  for (int k = 0; k < sim::kPhases; ++k) acc[k] = 0;
#pragma unroll 1
  for (uint32_t t = 1; t <= kTicksPerDecision; ++t) {
    s.cars[0].controls = controls[(size_t)a * kCars];
    s.cars[1].controls = controls[(size_t)a * kCars + 1];
#pragma unroll 1
    for (int k = 0; k < sim::kPhases; ++k) {
      __syncwarp();
      long long t0 = clock64();
      sim::run_phase(k, s, D);
      __syncwarp();
      acc[k] += (unsigned long long)(clock64() - t0);
    }
  }
  if (i < n) store_tick(states, a, &s);
  if ((threadIdx.x & 31u) == 0)
    for (int k = 0; k < sim::kPhases; ++k) atomicAdd(prof + k, acc[k]);
}

cudaError_t rsx_launch_sim8_profile(uint32_t* states, const void* sds, const uint8_t* sd_index, const void* controls, uint32_t n,
                                    unsigned long long* prof, cudaStream_t s) {
  k_sim8_profile<<<(n + 31) / 32, 32, 0, s>>>(states, (const StaticData*)sds, sd_index, (const Controls*)controls, n, prof);
  return cudaGetLastError();
}
