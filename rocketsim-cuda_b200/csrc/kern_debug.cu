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
