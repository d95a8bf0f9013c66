// The reference's decision kernel (cuda/sim/sim.cu:95-112, sim8 / sim8_trace): one thread per arena, one StaticData.
#include "kern_common.cuh"

extern "C" __global__ void __launch_bounds__(kMaxBlock, 1) k_sim8(uint32_t* states, const StaticData* sd, const Controls* controls,
                                                                  uint32_t* result, uint32_t n, uint32_t* trace) {
  uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  result[a] = decide_arena(states, *sd, controls, a, trace, aosoa_words(n), nullptr);
}

cudaError_t rsx_launch_sim8(uint32_t* states, const void* sd, const void* controls, uint32_t* result, uint32_t n, uint32_t* trace,
                            uint32_t block, cudaStream_t s) {
  k_sim8<<<(n + block - 1) / block, block, 0, s>>>(states, (const StaticData*)sd, (const Controls*)controls, result, n, trace);
  return cudaGetLastError();
}
