// The persistent decision kernel: `gridDim.x` resident blocks, each warp repeatedly claiming 32 * `gran` consecutive
// entries of `order` (arena indices; identity when null) with one atomicAdd on a device counter.  With a binned order
// (arenas sorted by predicted cost), the lanes of a warp step arenas of like cost.  Nothing waits on another block: a
// claim past n ends the warp.  The counter must be zero at launch.
//
// Compiled once per register budget (RSX_MINB blocks of 64 threads per SM: 1 -> 255 registers, 8 -> 128, 12 -> 80,
// 16 -> 64) into separately named kernels; the autotuner picks one.  `cost[a]`, when non-null, receives the clock
// cycles arena a's decision took (>> 8): the measured labels of the cost binning.
#include "kern_common.cuh"

#ifndef RSX_MINB
#define RSX_MINB 1
#endif
#define RSX_CAT2(a, b) a##b
#define RSX_CAT(a, b) RSX_CAT2(a, b)
#define K_NAME RSX_CAT(k_sim8_persistent_b, RSX_MINB)
#define L_NAME RSX_CAT(rsx_launch_sim8_persistent_b, RSX_MINB)

extern "C" __global__ void __launch_bounds__(kMaxBlock, RSX_MINB) K_NAME(uint32_t* states, const StaticData* sds, const uint8_t* sd_index,
                                                                        const Controls* controls, uint32_t* result, uint32_t* ev_or,
                                                                        const uint32_t* order, uint32_t* counter, uint32_t n,
                                                                        uint32_t gran, uint32_t* cost) {
  persistent_claims(counter, n, gran, order, [&](uint32_t a) {
    const StaticData& D = sds[sd_index ? sd_index[a] : 0];
    long long t0 = clock64();
    result[a] = decide_arena(states, D, controls, a, nullptr, 0, ev_or);
    if (cost) cost[a] = (uint32_t)((clock64() - t0) >> 8);
  });
}

cudaError_t L_NAME(uint32_t* states, const void* sds, const uint8_t* sd_index, const void* controls, uint32_t* result, uint32_t* ev_or,
                   const uint32_t* order, uint32_t* counter, uint32_t n, uint32_t gran, uint32_t grid, uint32_t block, uint32_t* cost,
                   cudaStream_t s) {
  K_NAME<<<grid, block, 0, s>>>(states, (const StaticData*)sds, sd_index, (const Controls*)controls, result, ev_or, order, counter, n, gran,
                                cost);
  return cudaGetLastError();
}
