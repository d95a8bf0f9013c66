// Device side: the decision kernels for sm_100a and the device entry points of the C ABI (include/rsx.h).
//
// One thread owns one arena for a whole decision: its tick-boundary words are copied from the AoSoA-32 buffer into a
// thread-local ArenaState (lanes of a warp read 32 consecutive words per instruction when the warp covers one AoSoA
// block), the 8 ticks run on it, and the words are written back (at the goal tick when the ball is scored).  No
// arithmetic crosses arenas, so no result depends on block size, grid, arena order, queue granularity or binning.
//
// Kernels:
//   k_identity       copy-in / copy-out round trip (the layout check; reference sim.cu:9-24)
//   k_phase          one phase of every arena (sim.cu:27-34)
//   k_step_tick      one full tick (sim.cu:46-53)
//   k_sim8           one decision, one StaticData, optional per-tick trace (sim.cu:95-112)
//   k_sim8_multi     one decision with a per-arena StaticData (7 x 7 car pairings in one launch) and the OR of the
//                    decision's event words (the contact labels of the predictor)
//   k_sim8_persistent  resident blocks pull arenas from a device counter over an order array (binned or identity)
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>
#include <mutex>
#include "../../include/rsx.h"
#include "state.cuh"
#include "sim/physics.cuh"

using namespace rsx;

namespace {

constexpr int kMaxBlock = 64;

__device__ __forceinline__ void load_tick(ArenaState* s, const uint32_t* buf, uint32_t a) {
  uint32_t* d = reinterpret_cast<uint32_t*>(s);
  const uint32_t* src = buf + (size_t)(a / kLanes) * aosoa_block_words() + (a % kLanes);
#pragma unroll 8
  for (int w = 0; w < kTickWords; ++w) d[w] = src[(size_t)w * kLanes];
#pragma unroll 8
  for (int w = kTickWords; w < kArenaWords; ++w) d[w] = 0u;
}
__device__ __forceinline__ void store_tick(uint32_t* buf, uint32_t a, const ArenaState* s) {
  const uint32_t* d = reinterpret_cast<const uint32_t*>(s);
  uint32_t* dst = buf + (size_t)(a / kLanes) * aosoa_block_words() + (a % kLanes);
#pragma unroll 8
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

}  // namespace

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

extern "C" __global__ void __launch_bounds__(kMaxBlock, 1) k_sim8(uint32_t* states, const StaticData* sd, const Controls* controls,
                                                                  uint32_t* result, uint32_t n, uint32_t* trace) {
  uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  result[a] = decide_arena(states, *sd, controls, a, trace, aosoa_words(n), nullptr);
}

extern "C" __global__ void __launch_bounds__(kMaxBlock, 1) k_sim8_multi(uint32_t* states, const StaticData* sds, const uint8_t* sd_index,
                                                                        const Controls* controls, uint32_t* result, uint32_t* ev_or,
                                                                        uint32_t n) {
  uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  const StaticData& D = sds[sd_index ? sd_index[a] : 0];
  result[a] = decide_arena(states, D, controls, a, nullptr, 0, ev_or);
}

// Persistent decision kernel: `gridDim.x` resident blocks; each warp repeatedly takes `gran` consecutive entries of
// `order` (arena indices) from the device counter.  The counter must be zero at launch (the host clears it in the same
// stream) and ends at >= n.  No wait on another block or grid: each claim is one atomicAdd.
extern "C" __global__ void __launch_bounds__(kMaxBlock, 1) k_sim8_persistent(uint32_t* states, const StaticData* sds, const uint8_t* sd_index,
                                                                             const Controls* controls, uint32_t* result, uint32_t* ev_or,
                                                                             const uint32_t* order, uint32_t* counter, uint32_t n,
                                                                             uint32_t gran) {
  const uint32_t lane = threadIdx.x & 31u;
  for (;;) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(counter, 32u * gran);
    base = __shfl_sync(0xFFFFFFFFu, base, 0);
    if (base >= n) break;
    for (uint32_t g = 0; g < gran; ++g) {
      uint32_t i = base + g * 32u + lane;
      if (i < n) {
        uint32_t a = order ? order[i] : i;
        const StaticData& D = sds[sd_index ? sd_index[a] : 0];
        result[a] = decide_arena(states, D, controls, a, nullptr, 0, ev_or);
      }
    }
  }
}

// ---------------------------------------------------------------------------------------------------------------------
// The device entry points of the C ABI.

struct rsx_device {
  int ordinal;
  cudaStream_t stream;
};
struct rsx_static {
  rsx_device* dev;
  void* d;
  uint32_t count;
};
struct rsx_states {
  rsx_device* dev;
  uint32_t* d;
  uint32_t n;
};

static thread_local char g_err[256] = "";
static int fail(cudaError_t e, const char* where) {
  snprintf(g_err, sizeof(g_err), "%s: %s", where, cudaGetErrorString(e));
  return RSX_E_CUDA;
}
#define RSX_CK(x)                          \
  do {                                     \
    cudaError_t e_ = (x);                  \
    if (e_ != cudaSuccess) return fail(e_, #x); \
  } while (0)

static int configure_current(void) {
  static std::once_flag once[64];
  int dev = 0;
  RSX_CK(cudaGetDevice(&dev));
  static int status[64];
  std::call_once(once[dev & 63], [&] {
    // the phases run as calls with large frames (the solver's rows, the narrowphase jobs): reserve the stack they need
    size_t want = 32 * 1024;
    cudaError_t e = cudaDeviceSetLimit(cudaLimitStackSize, want);
    status[dev & 63] = e == cudaSuccess ? RSX_OK : fail(e, "cudaDeviceSetLimit(stack)");
  });
  return status[dev & 63];
}

extern "C" {

const char* rsx_last_error(void) { return g_err; }

int rsx_device_create(int ordinal, rsx_device** out) {
  if (!out) return RSX_E_ARG;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0 || ordinal < 0 || ordinal >= count) {
    snprintf(g_err, sizeof(g_err), "no CUDA device %d", ordinal);
    return RSX_E_NODEV;
  }
  cudaDeviceProp p;
  RSX_CK(cudaGetDeviceProperties(&p, ordinal));
  if (p.major != 10) {
    snprintf(g_err, sizeof(g_err), "device %d is sm_%d%d; this library is built for sm_100a", ordinal, p.major, p.minor);
    return RSX_E_NODEV;
  }
  RSX_CK(cudaSetDevice(ordinal));
  int c = configure_current();
  if (c != RSX_OK) return c;
  rsx_device* d = new rsx_device;
  d->ordinal = ordinal;
  cudaError_t e = cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete d;
    return fail(e, "cudaStreamCreate");
  }
  *out = d;
  return RSX_OK;
}

int rsx_device_destroy(rsx_device* dev) {
  if (!dev) return RSX_E_ARG;
  cudaStreamSynchronize(dev->stream);
  cudaStreamDestroy(dev->stream);
  delete dev;
  return RSX_OK;
}

int rsx_sync(rsx_device* dev) {
  if (!dev) return RSX_E_ARG;
  RSX_CK(cudaStreamSynchronize(dev->stream));
  return RSX_OK;
}

void* rsx_device_stream(rsx_device* dev) { return dev ? (void*)dev->stream : nullptr; }

int rsx_static_upload(rsx_device* dev, const uint32_t* words, uint32_t count, rsx_static** out) {
  if (!dev || !words || !out || count == 0) return RSX_E_ARG;
  RSX_CK(cudaSetDevice(dev->ordinal));
  size_t bytes = sizeof(StaticData) * (size_t)count;
  void* d = nullptr;
  RSX_CK(cudaMalloc(&d, bytes));
  cudaError_t e = cudaMemcpyAsync(d, words, bytes, cudaMemcpyHostToDevice, dev->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(dev->stream);
  if (e != cudaSuccess) {
    cudaFree(d);
    return fail(e, "static upload");
  }
  *out = new rsx_static{dev, d, count};
  return RSX_OK;
}
int rsx_static_free(rsx_static* sd) {
  if (!sd) return RSX_E_ARG;
  cudaFree(sd->d);
  delete sd;
  return RSX_OK;
}
const void* rsx_static_device_ptr(rsx_static* sd) { return sd ? sd->d : nullptr; }

int rsx_states_alloc(rsx_device* dev, uint32_t n, rsx_states** out) {
  if (!dev || !out || n == 0) return RSX_E_ARG;
  RSX_CK(cudaSetDevice(dev->ordinal));
  uint32_t* d = nullptr;
  RSX_CK(cudaMalloc(&d, aosoa_words(n) * 4));
  RSX_CK(cudaMemsetAsync(d, 0, aosoa_words(n) * 4, dev->stream));
  *out = new rsx_states{dev, d, n};
  return RSX_OK;
}
int rsx_states_free(rsx_states* st) {
  if (!st) return RSX_E_ARG;
  cudaFree(st->d);
  delete st;
  return RSX_OK;
}
int rsx_states_upload(rsx_device* dev, rsx_states* st, const uint32_t* aosoa) {
  if (!dev || !st || !aosoa) return RSX_E_ARG;
  RSX_CK(cudaMemcpyAsync(st->d, aosoa, aosoa_words(st->n) * 4, cudaMemcpyHostToDevice, dev->stream));
  RSX_CK(cudaStreamSynchronize(dev->stream));
  return RSX_OK;
}
int rsx_states_download(rsx_device* dev, rsx_states* st, uint32_t* aosoa) {
  if (!dev || !st || !aosoa) return RSX_E_ARG;
  RSX_CK(cudaMemcpyAsync(aosoa, st->d, aosoa_words(st->n) * 4, cudaMemcpyDeviceToHost, dev->stream));
  RSX_CK(cudaStreamSynchronize(dev->stream));
  return RSX_OK;
}
uint32_t* rsx_states_device_ptr(rsx_states* st) { return st ? st->d : nullptr; }

int rsx_sim8_raw(uint32_t* d_states, uint32_t n, const void* d_static, const rsx_controls* d_controls, uint32_t* d_result, uint32_t block,
                 uint32_t* d_trace, void* stream) {
  if (!d_states || !d_static || !d_controls || !d_result || block < 1 || block > RSX_MAX_BLOCK) return RSX_E_ARG;
  if (n == 0) return RSX_OK;
  int c = configure_current();
  if (c != RSX_OK) return c;
  k_sim8<<<(n + block - 1) / block, block, 0, (cudaStream_t)stream>>>(d_states, (const StaticData*)d_static, (const Controls*)d_controls,
                                                                        d_result, n, d_trace);
  RSX_CK(cudaGetLastError());
  return RSX_OK;
}

int rsx_sim8(rsx_device* dev, rsx_states* st, rsx_static* sd, const rsx_controls* d_controls, uint32_t* d_result, uint32_t block,
             uint32_t* d_trace) {
  if (!dev || !st || !sd) return RSX_E_ARG;
  return rsx_sim8_raw(st->d, st->n, sd->d, d_controls, d_result, block, d_trace, dev->stream);
}

int rsx_step_tick(rsx_device* dev, rsx_states* st, rsx_static* sd, int32_t* d_status) {
  if (!dev || !st || !sd || !d_status) return RSX_E_ARG;
  k_step_tick<<<(st->n + 31) / 32, 32, 0, dev->stream>>>(st->d, (const StaticData*)sd->d, st->n, d_status);
  RSX_CK(cudaGetLastError());
  return RSX_OK;
}

int rsx_phase(rsx_device* dev, int k, rsx_states* st, rsx_static* sd, int32_t* d_status) {
  if (!dev || !st || !sd || !d_status || k < 0 || k >= sim::kPhases) return RSX_E_ARG;
  k_phase<<<(st->n + 127) / 128, 128, 0, dev->stream>>>(k, st->d, (const StaticData*)sd->d, st->n, d_status);
  RSX_CK(cudaGetLastError());
  return RSX_OK;
}

int rsx_identity(rsx_device* dev, const uint32_t* d_in, uint32_t* d_out, uint32_t n, int tick_only) {
  if (!dev || !d_in || !d_out) return RSX_E_ARG;
  if (n == 0) return RSX_OK;
  k_identity<<<(n + 127) / 128, 128, 0, dev->stream>>>(d_in, d_out, n, tick_only);
  RSX_CK(cudaGetLastError());
  return RSX_OK;
}

int rsx_sim8_multi_raw(uint32_t* d_states, uint32_t n, const void* d_statics, const uint8_t* d_sd_index, const rsx_controls* d_controls,
                       uint32_t* d_result, uint32_t* d_event_or, uint32_t block, void* stream) {
  if (!d_states || !d_statics || !d_controls || !d_result || block < 1 || block > RSX_MAX_BLOCK) return RSX_E_ARG;
  if (n == 0) return RSX_OK;
  int c = configure_current();
  if (c != RSX_OK) return c;
  k_sim8_multi<<<(n + block - 1) / block, block, 0, (cudaStream_t)stream>>>(d_states, (const StaticData*)d_statics, d_sd_index,
                                                                             (const Controls*)d_controls, d_result, d_event_or, n);
  RSX_CK(cudaGetLastError());
  return RSX_OK;
}

int rsx_sim8_persistent_raw(uint32_t* d_states, uint32_t n, const void* d_statics, const uint8_t* d_sd_index, const rsx_controls* d_controls,
                            uint32_t* d_result, uint32_t* d_event_or, const uint32_t* d_order, uint32_t* d_queue_counter, uint32_t grid,
                            uint32_t block, uint32_t granularity, void* stream) {
  if (!d_states || !d_statics || !d_controls || !d_result || !d_queue_counter || block < 32 || block > RSX_MAX_BLOCK || (block & 31) ||
      grid == 0 || granularity == 0)
    return RSX_E_ARG;
  if (n == 0) return RSX_OK;
  int c = configure_current();
  if (c != RSX_OK) return c;
  RSX_CK(cudaMemsetAsync(d_queue_counter, 0, 4, (cudaStream_t)stream));
  k_sim8_persistent<<<grid, block, 0, (cudaStream_t)stream>>>(d_states, (const StaticData*)d_statics, d_sd_index,
                                                              (const Controls*)d_controls, d_result, d_event_or, d_order, d_queue_counter,
                                                              n, granularity);
  RSX_CK(cudaGetLastError());
  return RSX_OK;
}

}  // extern "C"
