// Verification entry points of the correctly rounded libm (crmath.cuh): batch evaluation on the host, and a device
// kernel that hashes f(x) over chunks of 2^24 consecutive input bit patterns, so that all 2^32 inputs of sin, cos and
// tan can be compared with hashes of the reference's values made once on a CPU.  The hash of a chunk is the wrapping
// sum of mix64((x_bits << 32) | f(x)_bits) over its inputs: independent of evaluation order.
#include <cuda_runtime.h>
#include "../../include/rsx.h"
#include "crmath.cuh"

using namespace rsx;

namespace {
__host__ __device__ inline uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__host__ __device__ inline float eval1(int fn, float x) { return fn == 0 ? cr_sin(x) : fn == 1 ? cr_cos(x) : cr_tan(x); }
}  // namespace

// one block per chunk slice: blockIdx.y = chunk, grid.x * blockDim.x threads stride over its 2^24 inputs
extern "C" __global__ void __launch_bounds__(256) k_libm_hash(int fn, uint32_t first_chunk, unsigned long long* hashes) {
  uint32_t chunk = first_chunk + blockIdx.y;
  uint64_t local = 0;
  uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < (1u << 24); i += stride) {
    uint32_t xb = (chunk << 24) | i;
    uint32_t yb = bits(eval1(fn, from_bits(xb)));
    if ((yb & 0x7FFFFFFFu) > 0x7F800000u) yb = 0x7FC00000u;
    local += mix64(((uint64_t)xb << 32) | yb);
  }
  // warp reduce then one atomic per warp
  for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xFFFFFFFFu, local, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(&hashes[blockIdx.y], (unsigned long long)local);
}

extern "C" {

// out[i] = f(a[i]) (fn 0 sin, 1 cos, 2 tan) or f(a[i], b[i]) (fn 3 atan2, 4 pow, 5 float(atan2 as double),
// 6 float(hypot as double)), on the host
int rsx_libm_host(int fn, const float* a, const float* b, float* out, uint64_t n) {
  if (!a || !out || fn < 0 || fn > 6 || (fn >= 3 && !b)) return RSX_E_ARG;
  for (uint64_t i = 0; i < n; ++i) {
    switch (fn) {
      case 0: out[i] = cr_sin(a[i]); break;
      case 1: out[i] = cr_cos(a[i]); break;
      case 2: out[i] = cr_tan(a[i]); break;
      case 3: out[i] = cr_atan2(a[i], b[i]); break;
      case 4: out[i] = cr_pow(a[i], b[i]); break;
      case 5: out[i] = crm::atan2_via_double(a[i], b[i]); break;
      default: out[i] = crm::hypot_via_double(a[i], b[i]); break;
    }
  }
  return RSX_OK;
}

// the same hash on the host for a range of inputs (tests compare a few chunks host vs device)
uint64_t rsx_libm_hash_host(int fn, uint32_t first_bits, uint32_t count) {
  uint64_t h = 0;
  for (uint32_t k = 0; k < count; ++k) {
    uint32_t xb = first_bits + k;
    uint32_t yb = bits(eval1(fn, from_bits(xb)));
    if ((yb & 0x7FFFFFFFu) > 0x7F800000u) yb = 0x7FC00000u;
    h += mix64(((uint64_t)xb << 32) | yb);
  }
  return h;
}

// hashes[c] for chunks first_chunk .. first_chunk + nchunks - 1 (d_hashes: nchunks u64 on the device, zeroed here)
int rsx_libm_chunk_hashes(int fn, uint32_t first_chunk, uint32_t nchunks, uint64_t* d_hashes, void* stream) {
  if (fn < 0 || fn > 2 || !d_hashes || first_chunk + nchunks > 256u) return RSX_E_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemsetAsync(d_hashes, 0, (size_t)nchunks * 8, s) != cudaSuccess) return RSX_E_CUDA;
  dim3 grid(592, nchunks);
  k_libm_hash<<<grid, 256, 0, s>>>(fn, first_chunk, (unsigned long long*)d_hashes);
  return cudaGetLastError() == cudaSuccess ? RSX_OK : RSX_E_CUDA;
}

}  // extern "C"
