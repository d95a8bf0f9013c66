// The decision with a StaticData per arena (all 7 x 7 car pairings in one launch) and the OR of each arena's event words
// over the decision (the contact labels of the binning predictor).  No counterpart kernel in the reference.
#include "kern_common.cuh"

extern "C" __global__ void __launch_bounds__(kMaxBlock, 1) k_sim8_multi(uint32_t* states, const StaticData* sds, const uint8_t* sd_index,
                                                                        const Controls* controls, uint32_t* result, uint32_t* ev_or,
                                                                        uint32_t n) {
  uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  const StaticData& D = sds[sd_index ? sd_index[a] : 0];
  result[a] = decide_arena(states, D, controls, a, nullptr, 0, ev_or);
}

cudaError_t rsx_launch_sim8_multi(uint32_t* states, const void* sds, const uint8_t* sd_index, const void* controls, uint32_t* result,
                                  uint32_t* ev_or, uint32_t n, uint32_t block, cudaStream_t s) {
  k_sim8_multi<<<(n + block - 1) / block, block, 0, s>>>(states, (const StaticData*)sds, sd_index, (const Controls*)controls, result, ev_or, n);
  return cudaGetLastError();
}
