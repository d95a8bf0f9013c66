// The persistent decision kernel for callers that cannot allocate device memory.
//
// rsx_sim8_persistent_raw needs one word of scratch, the work-queue counter that the warps of the persistent kernel
// claim arenas from, and takes it from the caller.  Some callers have no way to provide it: a host program whose device
// memory is owned by another allocator (a framework that reserved the GPU's memory up front, so that cudaMalloc fails
// or would fragment it), a real-time loop that must not call cudaMalloc / cudaFree because they can synchronise the
// whole device, or a foreign-language binding that only ever receives the buffers of states, controls and results.
// rsx_sim8_persistent_noalloc runs the same decision with the counter in a file-scope device array instead.
//
// The scratch: kNoallocScratchWords words (256 bytes), of which one launch uses word 0 as the queue counter.  Every GPU
// that loads this library holds the array until the process exits.  It is shared by every call on that device and keeps
// the last call's contents, so each call clears the counter on the caller's stream before its launch; two calls whose
// launches overlap on the GPU (different streams, no ordering between them) race on the counter and may skip or repeat
// arenas.  Calls on one stream are ordered and safe.
//
// Set-up: the first call on a device (the device current at the call) looks up the array's device address with
// cudaGetSymbolAddress and keeps it, with the unique ID of the device's CUDA context; make that first call before any
// stream capture on the device.  A later call whose current context has another ID (the device was reset, which
// reloads the module, possibly at another address) looks the address up again, so make the first call after a reset
// before any capture too.  The caller's current device must be the one that holds the buffers and the stream.
//
// Limit: at most kNoallocMaxArenas (2^24) arenas per call, granularity at most 256 and grid at most 65,535, so that the
// 32-bit counter, which overshoots n by up to grid x block x granularity claims, cannot wrap.
#include <stdio.h>
#include <mutex>
#include "kern_common.cuh"

namespace {
constexpr uint32_t kNoallocScratchWords = 64;
constexpr uint32_t kNoallocMaxArenas = kQueueMaxArenas;
constexpr uint32_t kNoallocMaxGran = kQueueMaxGran;
constexpr uint32_t kNoallocMaxGrid = kQueueMaxGrid;
constexpr int kNoallocMaxDevices = 64;
}  // namespace

static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoallocScratchWords];

// The persistent kernel of kern_persist.cu (255-register budget) with its counter at `counter` (the scratch array's
// device address) and no cost output.
extern "C" __global__ void __launch_bounds__(kMaxBlock, 1) k_sim8_persistent_noalloc(uint32_t* states, const StaticData* sds,
                                                                                     const uint8_t* sd_index, const Controls* controls,
                                                                                     uint32_t* result, uint32_t* ev_or, const uint32_t* order,
                                                                                     uint32_t* counter, uint32_t n, uint32_t gran) {
  persistent_claims(counter, n, gran, order, [&](uint32_t a) {
    const StaticData& D = sds[sd_index ? sd_index[a] : 0];
    result[a] = decide_arena(states, D, controls, a, nullptr, 0, ev_or);
  });
}

static std::mutex g_noalloc_mu;
static uint32_t* g_noalloc_ptr[kNoallocMaxDevices];
static unsigned long long g_noalloc_ctx[kNoallocMaxDevices];

// The unique ID of the calling thread's current CUDA context (cuCtxGetCurrent + cuCtxGetId through the runtime's driver
// entry points, so the library needs no link to the driver library); 0 when there is none or the driver lacks the call.
typedef int (*CtxGetCurrentFn)(void** ctx);
typedef int (*CtxGetIdFn)(void* ctx, unsigned long long* id);
static unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", (void**)&get_current, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      get_current = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", (void**)&get_id, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
      get_id = nullptr;
    (void)cudaGetLastError();
  });
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (get_current && get_id && get_current(&ctx) == 0 && ctx && get_id(ctx, &id) == 0) return id;
  return 0;
}

// The scratch array's device address on the current device (cudaGetSymbolAddress; in host code the array's name is only
// a host-side stand-in, never a device address): looked up by the first call on the device, and again when the current
// context is no longer the one it was looked up in.
static cudaError_t noalloc_scratch(uint32_t** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kNoallocMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev] || current_context_id() != g_noalloc_ctx[dev]) {
    uint32_t* p = nullptr;
    e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_ptr[dev] = p;
    g_noalloc_ctx[dev] = current_context_id();  // the lookup made the device's context current
  }
  *out = g_noalloc_ptr[dev];
  return cudaSuccess;
}

int rsx_set_last_error(int code, const char* msg);  // capi.cu: the message rsx_last_error() returns

extern "C" int rsx_sim8_persistent_noalloc(uint32_t* d_states, uint32_t n, const void* d_statics, const uint8_t* d_sd_index,
                                           const rsx_controls* d_controls, uint32_t* d_result, uint32_t* d_event_or,
                                           const uint32_t* d_order, uint32_t grid, uint32_t block, uint32_t granularity, void* stream) {
  if (!d_states || !d_statics || !d_controls || !d_result || block < 32 || block > RSX_MAX_BLOCK || (block & 31) || grid == 0 ||
      granularity == 0)
    return rsx_set_last_error(RSX_E_ARG, "rsx_sim8_persistent_noalloc: null buffer, or block not 32/64, or grid / granularity 0");
  if (n > kNoallocMaxArenas || granularity > kNoallocMaxGran || grid > kNoallocMaxGrid)
    return rsx_set_last_error(RSX_E_ARG,
                            "rsx_sim8_persistent_noalloc: at most 16,777,216 arenas, granularity 256 and grid 65,535 per call "
                            "(the 32-bit queue counter in its fixed scratch must not wrap)");
  if (n == 0) return RSX_OK;
  uint32_t* counter = nullptr;
  cudaError_t e = noalloc_scratch(&counter);
  if (e == cudaSuccess) e = cudaMemsetAsync(counter, 0, sizeof(uint32_t), (cudaStream_t)stream);
  if (e == cudaSuccess) {
    k_sim8_persistent_noalloc<<<grid, block, 0, (cudaStream_t)stream>>>(d_states, (const StaticData*)d_statics, d_sd_index,
                                                                        (const Controls*)d_controls, d_result, d_event_or, d_order,
                                                                        counter, n, granularity);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    char msg[200];
    snprintf(msg, sizeof(msg), "rsx_sim8_persistent_noalloc: %s", cudaGetErrorString(e));
    return rsx_set_last_error(RSX_E_CUDA, msg);
  }
  return RSX_OK;
}
