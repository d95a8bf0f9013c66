// The device entry points of the C ABI (include/rsx.h): the handles (device + stream, static data, states), uploads and
// downloads, and the launches of the decision kernels (kern_*.cu).  Status codes, never exceptions, cross the ABI.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>
#include <mutex>
#include "../../include/rsx.h"
#include "state.cuh"

using namespace rsx;

cudaError_t rsx_launch_sim8(uint32_t* states, const void* sd, const void* controls, uint32_t* result, uint32_t n, uint32_t* trace,
                            uint32_t block, cudaStream_t s);
cudaError_t rsx_launch_sim8_multi(uint32_t* states, const void* sds, const uint8_t* sd_index, const void* controls, uint32_t* result,
                                  uint32_t* ev_or, uint32_t n, uint32_t block, cudaStream_t s);
#define RSX_DECL_PERSIST(B)                                                                                               \
  cudaError_t rsx_launch_sim8_persistent_b##B(uint32_t* states, const void* sds, const uint8_t* sd_index, const void* controls,        \
                                              uint32_t* result, uint32_t* ev_or, const uint32_t* order, uint32_t* counter, uint32_t n, \
                                              uint32_t gran, uint32_t grid, uint32_t block, uint32_t* cost, cudaStream_t s);
RSX_DECL_PERSIST(1)
RSX_DECL_PERSIST(8)
RSX_DECL_PERSIST(12)
RSX_DECL_PERSIST(16)
#define RSX_DECL_LOCKSTEP(T)                                                                                                \
  cudaError_t rsx_launch_sim8_lockstep_t##T(uint32_t* states, const void* sds, const uint8_t* sd_index, const void* controls,         \
                                            uint32_t* result, uint32_t* ev_or, const uint32_t* order, uint32_t* counter, uint32_t n,  \
                                            uint32_t grid, uint32_t block, int split, uint32_t t_first, uint32_t t_last,                \
                                            cudaStream_t s);
RSX_DECL_LOCKSTEP(448)
RSX_DECL_LOCKSTEP(512)
cudaError_t rsx_launch_pred_features(const uint32_t* states, const void* sds, const uint8_t* sd_index, const void* controls, uint32_t n,
                                     void* X, cudaStream_t s);
cudaError_t rsx_launch_pred_labels(const uint32_t* ev, uint32_t n, uint8_t* Y, cudaStream_t s);
cudaError_t rsx_launch_pred_forward(const void* wb, const float* wf, const void* X, uint32_t n, float* logits, void* save, cudaStream_t s);
cudaError_t rsx_launch_pred_adam(float* w, void* wb, float* m, float* v, const float* grad, float lr, float b1, float b2, float eps, float c1,
                                 float c2, cudaStream_t s);
cudaError_t rsx_launch_pred_to_bf16(const float* w, void* wb, cudaStream_t s);
cudaError_t rsx_launch_pred_forward_tc(const void* wb, const float* wf, const void* X, uint32_t n, float* logits, void* save, uint32_t* err,
                                       cudaStream_t s);
cudaError_t rsx_launch_pred_backward_tc(const void* wb, const float* logits, const uint8_t* Y, const void* save, uint32_t n, float inv_scale,
                                        void* dz, void* dsave, float* loss_sum, uint32_t* err, cudaStream_t s);
cudaError_t rsx_launch_pred_wgrads_tc(const void* X, const void* dz, const void* save, const void* dsave, uint32_t n, float* grad, uint32_t* err,
                                      cudaStream_t s);
cudaError_t rsx_launch_pred_levels(const float* logits, uint32_t n, const float* weights, int levels, uint32_t* scratch, uint32_t* order,
                                   cudaStream_t s);
cudaError_t rsx_launch_pred_bin(const float* logits, uint32_t n, float thr, uint32_t mask, uint32_t* block_scratch, uint32_t* order,
                                uint32_t* heavy_total, cudaStream_t s);
cudaError_t rsx_launch_observe(const uint32_t* states, uint32_t n, const void* sds, const uint8_t* sd_index, const uint8_t* pad_mirror,
                               const uint32_t* result, const uint32_t* event_or, const float* weights, uint16_t* obs, float* reward,
                               cudaStream_t s);
cudaError_t rsx_launch_reset_arenas(uint32_t* states, uint32_t n, const void* sds, const uint8_t* sd_index, uint64_t seed, const float* mix,
                                    const uint32_t* result, const uint8_t* mask, uint32_t* reset_count, cudaStream_t s);
cudaError_t rsx_launch_identity(const uint32_t* in, uint32_t* out, uint32_t n, int tick_only, cudaStream_t s);
cudaError_t rsx_launch_phase(int k, uint32_t* buf, const void* sd, uint32_t n, int32_t* status, cudaStream_t s);
cudaError_t rsx_launch_step_tick(uint32_t* buf, const void* sd, uint32_t n, int32_t* status, cudaStream_t s);
cudaError_t rsx_launch_sim8_profile(uint32_t* states, const void* sds, const uint8_t* sd_index, const void* controls, uint32_t n,
                                    unsigned long long* prof, cudaStream_t s);


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
int rsx_set_last_error(int code, const char* msg) {
  snprintf(g_err, sizeof(g_err), "%s", msg);
  return code;
}
#define RSX_CK(x)                          \
  do {                                     \
    cudaError_t e_ = (x);                  \
    if (e_ != cudaSuccess) return fail(e_, #x); \
  } while (0)

// Local memory: the kernels' call chains are known at compile time (no recursion), so the runtime sizes each thread's
// local memory (about 20 KB: the arena state and the solver's rows) by itself; nothing to configure per device.
static int configure_current(void) { return RSX_OK; }

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
  // a blocking stream: ordered with work the caller puts on the legacy default stream (torch's, for one), as the
  // reference's cudarc context with event tracking off leaves ordering to the caller's stream use
  cudaError_t e = cudaStreamCreate(&d->stream);
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
  RSX_CK(rsx_launch_sim8(d_states, d_static, d_controls, d_result, n, d_trace, block, (cudaStream_t)stream));
  return RSX_OK;
}

int rsx_sim8(rsx_device* dev, rsx_states* st, rsx_static* sd, const rsx_controls* d_controls, uint32_t* d_result, uint32_t block,
             uint32_t* d_trace) {
  if (!dev || !st || !sd) return RSX_E_ARG;
  return rsx_sim8_raw(st->d, st->n, sd->d, d_controls, d_result, block, d_trace, dev->stream);
}

int rsx_step_tick(rsx_device* dev, rsx_states* st, rsx_static* sd, int32_t* d_status) {
  if (!dev || !st || !sd || !d_status) return RSX_E_ARG;
  RSX_CK(rsx_launch_step_tick(st->d, sd->d, st->n, d_status, dev->stream));
  return RSX_OK;
}

int rsx_phase(rsx_device* dev, int k, rsx_states* st, rsx_static* sd, int32_t* d_status) {
  if (!dev || !st || !sd || !d_status || k < 0 || k >= 10) return RSX_E_ARG;
  RSX_CK(rsx_launch_phase(k, st->d, sd->d, st->n, d_status, dev->stream));
  return RSX_OK;
}

int rsx_identity(rsx_device* dev, const uint32_t* d_in, uint32_t* d_out, uint32_t n, int tick_only) {
  if (!dev || !d_in || !d_out) return RSX_E_ARG;
  if (n == 0) return RSX_OK;
  RSX_CK(rsx_launch_identity(d_in, d_out, n, tick_only, dev->stream));
  return RSX_OK;
}

int rsx_sim8_multi_raw(uint32_t* d_states, uint32_t n, const void* d_statics, const uint8_t* d_sd_index, const rsx_controls* d_controls,
                       uint32_t* d_result, uint32_t* d_event_or, uint32_t block, void* stream) {
  if (!d_states || !d_statics || !d_controls || !d_result || block < 1 || block > RSX_MAX_BLOCK) return RSX_E_ARG;
  if (n == 0) return RSX_OK;
  int c = configure_current();
  if (c != RSX_OK) return c;
  RSX_CK(rsx_launch_sim8_multi(d_states, d_statics, d_sd_index, d_controls, d_result, d_event_or, n, block, (cudaStream_t)stream));
  return RSX_OK;
}

int rsx_sim8_persistent_raw(uint32_t* d_states, uint32_t n, const void* d_statics, const uint8_t* d_sd_index, const rsx_controls* d_controls,
                            uint32_t* d_result, uint32_t* d_event_or, const uint32_t* d_order, uint32_t* d_queue_counter, uint32_t grid,
                            uint32_t block, uint32_t granularity, void* stream) {
  return rsx_sim8_persistent_ex(d_states, n, d_statics, d_sd_index, d_controls, d_result, d_event_or, d_order, d_queue_counter, grid, block,
                                granularity, 1, nullptr, stream);
}

int rsx_sim8_persistent_ex(uint32_t* d_states, uint32_t n, const void* d_statics, const uint8_t* d_sd_index, const rsx_controls* d_controls,
                           uint32_t* d_result, uint32_t* d_event_or, const uint32_t* d_order, uint32_t* d_queue_counter, uint32_t grid,
                           uint32_t block, uint32_t granularity, uint32_t min_blocks, uint32_t* d_cost, void* stream) {
  if (!d_states || !d_statics || !d_controls || !d_result || !d_queue_counter || block < 32 || block > RSX_MAX_BLOCK || (block & 31) ||
      grid == 0 || granularity == 0)
    return rsx_set_last_error(RSX_E_ARG, "rsx_sim8_persistent_ex: null buffer, or block not 32/64, or grid / granularity 0");
  if (min_blocks != 1 && min_blocks != 8 && min_blocks != 12 && min_blocks != 16)
    return rsx_set_last_error(RSX_E_ARG, "rsx_sim8_persistent_ex: min_blocks not 1, 8, 12 or 16");
  // the 32-bit queue counter ends at most grid x block x granularity claims past n: it must not wrap
  if (n > kQueueMaxArenas || granularity > kQueueMaxGran || grid > kQueueMaxGrid ||
      (uint64_t)n + (uint64_t)grid * block * granularity >= (1ull << 32))
    return rsx_set_last_error(RSX_E_ARG, "rsx_sim8_persistent_ex: at most 16,777,216 arenas, granularity 256 and grid 65,535 per call "
                                         "(the 32-bit queue counter must not wrap)");
  if (n == 0) return RSX_OK;
  cudaStream_t s = (cudaStream_t)stream;
  RSX_CK(cudaMemsetAsync(d_queue_counter, 0, 4, s));
  cudaError_t e;
  switch (min_blocks) {
    case 8: e = rsx_launch_sim8_persistent_b8(d_states, d_statics, d_sd_index, d_controls, d_result, d_event_or, d_order, d_queue_counter, n,
                                              granularity, grid, block, d_cost, s); break;
    case 12: e = rsx_launch_sim8_persistent_b12(d_states, d_statics, d_sd_index, d_controls, d_result, d_event_or, d_order, d_queue_counter, n,
                                                granularity, grid, block, d_cost, s); break;
    case 16: e = rsx_launch_sim8_persistent_b16(d_states, d_statics, d_sd_index, d_controls, d_result, d_event_or, d_order, d_queue_counter, n,
                                                granularity, grid, block, d_cost, s); break;
    default: e = rsx_launch_sim8_persistent_b1(d_states, d_statics, d_sd_index, d_controls, d_result, d_event_or, d_order, d_queue_counter, n,
                                               granularity, grid, block, d_cost, s); break;
  }
  RSX_CK(e);
  return RSX_OK;
}

int rsx_sim8_lockstep_raw(uint32_t* d_states, uint32_t n, const void* d_statics, const uint8_t* d_sd_index, const rsx_controls* d_controls,
                          uint32_t* d_result, uint32_t* d_event_or, const uint32_t* d_order, uint32_t* d_queue_counter, uint32_t grid,
                          uint32_t block, uint32_t split, void* stream) {
  return rsx_sim8_lockstep_ex(d_states, n, d_statics, d_sd_index, d_controls, d_result, d_event_or, d_order, d_queue_counter, grid, block,
                              split, RSX_TICKS_PER_DECISION, stream);
}

int rsx_sim8_lockstep_ex(uint32_t* d_states, uint32_t n, const void* d_statics, const uint8_t* d_sd_index, const rsx_controls* d_controls,
                         uint32_t* d_result, uint32_t* d_event_or, const uint32_t* d_order, uint32_t* d_queue_counter, uint32_t grid,
                         uint32_t block, uint32_t split, uint32_t ticks_per_launch, void* stream) {
  if (!d_states || !d_statics || !d_controls || !d_result || !d_queue_counter || block < 32 || block > RSX_LOCKSTEP_MAX_BLOCK ||
      (block & 31) || grid == 0 || (split > 11 && split != 14 && split != 15))
    return rsx_set_last_error(RSX_E_ARG, "rsx_sim8_lockstep: null buffer, block not a multiple of 32 in 32..512, grid 0 or split not in 0..11, 14, 15");
  if (ticks_per_launch == 0 || RSX_TICKS_PER_DECISION % ticks_per_launch != 0)
    return rsx_set_last_error(RSX_E_ARG, "rsx_sim8_lockstep_ex: ticks_per_launch must divide 8 (1, 2, 4 or 8)");
  // idle warps claim 32 entries once per tick until their block ends: n plus that overshoot must stay below 2^32
  if (n > kQueueMaxArenas || grid > kQueueMaxGrid)
    return rsx_set_last_error(RSX_E_ARG, "rsx_sim8_lockstep: at most 16,777,216 arenas and grid 65,535 per call "
                                         "(the 32-bit queue counter must not wrap)");
  if (n == 0) return RSX_OK;
  cudaStream_t s = (cudaStream_t)stream;
  for (uint32_t t0 = 1; t0 <= RSX_TICKS_PER_DECISION; t0 += ticks_per_launch) {
    const uint32_t t1 = t0 + ticks_per_launch - 1;
    RSX_CK(cudaMemsetAsync(d_queue_counter, 0, 4, s));
    cudaError_t e;
    if (block <= 448)
      e = rsx_launch_sim8_lockstep_t448(d_states, d_statics, d_sd_index, d_controls, d_result, d_event_or, d_order, d_queue_counter, n, grid,
                                        block, (int)split, t0, t1, s);
    else
      e = rsx_launch_sim8_lockstep_t512(d_states, d_statics, d_sd_index, d_controls, d_result, d_event_or, d_order, d_queue_counter, n, grid,
                                        block, (int)split, t0, t1, s);
    RSX_CK(e);
  }
  return RSX_OK;
}

int rsx_copy_raw(void* d_dst, const void* d_src, uint64_t bytes, void* stream) {
  if (!d_dst || !d_src) return RSX_E_ARG;
  if (bytes == 0) return RSX_OK;
  RSX_CK(cudaMemcpyAsync(d_dst, d_src, bytes, cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
  return RSX_OK;
}

int rsx_reset_arenas_raw(uint32_t* d_states, uint32_t n, const void* d_statics, const uint8_t* d_sd_index, uint64_t seed, const float* mix,
                         const uint32_t* d_result, const uint8_t* d_mask, uint32_t* d_reset_count, void* stream) {
  if (!d_states || !d_statics || !mix) return RSX_E_ARG;
  if (n == 0) return RSX_OK;
  RSX_CK(rsx_launch_reset_arenas(d_states, n, d_statics, d_sd_index, seed, mix, d_result, d_mask, d_reset_count, (cudaStream_t)stream));
  return RSX_OK;
}

int rsx_observe_raw(const uint32_t* d_states, uint32_t n, const void* d_statics, const uint8_t* d_sd_index, const uint8_t* d_pad_mirror,
                    const uint32_t* d_result, const uint32_t* d_event_or, const float* weights, uint16_t* d_obs, float* d_reward, void* stream) {
  if (!d_states || !d_statics || !d_obs || ((uintptr_t)d_obs & 15u) != 0)
    return rsx_set_last_error(RSX_E_ARG, "rsx_observe_raw: null buffer or an observation buffer not 16-byte aligned");
  if (n == 0) return RSX_OK;
  RSX_CK(rsx_launch_observe(d_states, n, d_statics, d_sd_index, d_pad_mirror, d_result, d_event_or, weights, d_obs, d_reward,
                            (cudaStream_t)stream));
  return RSX_OK;
}

// L2 residency for the static data: a persisting-access window over [d_ptr, d_ptr + bytes) on `stream` (kernels
// launched there afterwards, and kernel nodes captured from it, keep those lines in the persisting part of L2, which
// the streaming local-memory traffic of the decision kernels cannot evict).  bytes 0 removes the window.  The
// persisting carve-out is a limit of this process's context: it ends with the process.
int rsx_l2_persist_raw(const void* d_ptr, uint64_t bytes, float hit_ratio, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  int dev = 0;
  RSX_CK(cudaGetDevice(&dev));
  cudaStreamAttrValue v;
  memset(&v, 0, sizeof(v));
  if (bytes == 0 || !d_ptr) {
    v.accessPolicyWindow.base_ptr = nullptr;
    v.accessPolicyWindow.num_bytes = 0;
    v.accessPolicyWindow.hitRatio = 0.0f;
    v.accessPolicyWindow.hitProp = cudaAccessPropertyNormal;
    v.accessPolicyWindow.missProp = cudaAccessPropertyNormal;
    RSX_CK(cudaStreamSetAttribute(s, cudaStreamAttributeAccessPolicyWindow, &v));
    return RSX_OK;
  }
  int max_window = 0, max_persist = 0;
  RSX_CK(cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, dev));
  RSX_CK(cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, dev));
  size_t win = bytes < (uint64_t)max_window ? (size_t)bytes : (size_t)max_window;
  size_t carve = win < (size_t)max_persist ? win : (size_t)max_persist;
  RSX_CK(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, carve));
  v.accessPolicyWindow.base_ptr = const_cast<void*>(d_ptr);
  v.accessPolicyWindow.num_bytes = win;
  float hr = hit_ratio > 0.0f ? (hit_ratio < 1.0f ? hit_ratio : 1.0f) : 1.0f;
  if (win > carve) {  // the share of the window the carve-out can hold
    float fit = (float)carve / (float)win;
    hr = hr < fit ? hr : fit;
  }
  v.accessPolicyWindow.hitRatio = hr;
  v.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
  v.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
  RSX_CK(cudaStreamSetAttribute(s, cudaStreamAttributeAccessPolicyWindow, &v));
  return RSX_OK;
}

// ---- the contact predictor ----
uint64_t rsx_pred_scratch_elems(uint32_t n) { return 2ull * (3ull * n + 16) * 128 + (uint64_t)(n + 16) * 8 + 2; }

int rsx_pred_features_raw(const uint32_t* d_states, uint32_t n, const void* d_statics, const uint8_t* d_sd_index, const rsx_controls* d_controls,
                          uint16_t* d_features, void* stream) {
  if (!d_states || !d_statics || !d_controls || !d_features) return RSX_E_ARG;
  if (n == 0) return RSX_OK;
  RSX_CK(rsx_launch_pred_features(d_states, d_statics, d_sd_index, d_controls, n, d_features, (cudaStream_t)stream));
  return RSX_OK;
}

int rsx_pred_labels_raw(const uint32_t* d_event_or, uint32_t n, uint8_t* d_labels, void* stream) {
  if (!d_event_or || !d_labels) return RSX_E_ARG;
  if (n == 0) return RSX_OK;
  RSX_CK(rsx_launch_pred_labels(d_event_or, n, d_labels, (cudaStream_t)stream));
  return RSX_OK;
}

int rsx_pred_forward_raw(const uint16_t* d_w_bf16, const float* d_w_f32, const uint16_t* d_features, uint32_t n, float* d_logits, void* stream) {
  if (!d_w_bf16 || !d_w_f32 || !d_features || !d_logits) return RSX_E_ARG;
  if (n == 0) return RSX_OK;
  RSX_CK(rsx_launch_pred_forward(d_w_bf16, d_w_f32, d_features, n, d_logits, nullptr, (cudaStream_t)stream));
  return RSX_OK;
}

int rsx_pred_gradients_raw(const uint16_t* d_w_bf16, const float* d_w_f32, const uint16_t* d_features, const uint8_t* d_labels, uint32_t n,
                           uint16_t* d_scratch, float* d_logits, float* d_grad, float* d_loss, void* stream) {
  if (!d_w_bf16 || !d_w_f32 || !d_features || !d_labels || !d_scratch || !d_logits || !d_grad || !d_loss || n == 0) return RSX_E_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  uint16_t* save = d_scratch;
  uint16_t* dsave = save + (3ull * n + 16) * 128;
  uint16_t* dz = dsave + (3ull * n + 16) * 128;
  RSX_CK(cudaMemsetAsync(d_grad, 0, RSX_PRED_PARAMS * sizeof(float), s));
  RSX_CK(cudaMemsetAsync(d_loss, 0, sizeof(float), s));
  RSX_CK(cudaMemsetAsync(save + 3ull * n * 128, 0, 16 * 128 * 2, s));  // the rows past n that the last tile reads
  uint32_t* tc_error = reinterpret_cast<uint32_t*>(dz + (uint64_t)(n + 16) * 8);  // the scratch's last two elements
  RSX_CK(rsx_launch_pred_forward_tc(d_w_bf16, d_w_f32, d_features, n, d_logits, save, tc_error, s));
  RSX_CK(rsx_launch_pred_backward_tc(d_w_bf16, d_logits, d_labels, save, n, 1.0f / (float)n, dz, dsave, d_loss, tc_error, s));
  RSX_CK(rsx_launch_pred_wgrads_tc(d_features, dz, save, dsave, n, d_grad, tc_error, s));
  return RSX_OK;
}

int rsx_pred_adam_raw(float* d_w_f32, uint16_t* d_w_bf16, float* d_m, float* d_v, const float* d_grad, uint32_t step, float lr, void* stream) {
  if (!d_w_f32 || !d_w_bf16 || !d_m || !d_v || !d_grad || step == 0) return RSX_E_ARG;
  const float b1 = 0.9f, b2 = 0.999f;
  float p1 = 1.0f, p2 = 1.0f;
  for (uint32_t i = 0; i < step && i < 100000u; ++i) {
    p1 *= b1;
    p2 *= b2;
  }
  RSX_CK(rsx_launch_pred_adam(d_w_f32, d_w_bf16, d_m, d_v, d_grad, lr, b1, b2, 1e-8f, 1.0f - p1, 1.0f - p2, (cudaStream_t)stream));
  return RSX_OK;
}

int rsx_pred_to_bf16_raw(const float* d_w_f32, uint16_t* d_w_bf16, void* stream) {
  if (!d_w_f32 || !d_w_bf16) return RSX_E_ARG;
  RSX_CK(rsx_launch_pred_to_bf16(d_w_f32, d_w_bf16, (cudaStream_t)stream));
  return RSX_OK;
}

int rsx_pred_bin_raw(const float* d_logits, uint32_t n, float threshold_logit, uint32_t label_mask, uint32_t* d_scratch, uint32_t* d_order,
                     uint32_t* d_heavy_count, void* stream) {
  if (!d_logits || !d_scratch || !d_order || !d_heavy_count) return RSX_E_ARG;
  if (n == 0) return RSX_OK;
  RSX_CK(rsx_launch_pred_bin(d_logits, n, threshold_logit, label_mask, d_scratch, d_order, d_heavy_count, (cudaStream_t)stream));
  return RSX_OK;
}

int rsx_pred_forward_tc_raw(const uint16_t* d_w_bf16, const float* d_w_f32, const uint16_t* d_features, uint32_t n, float* d_logits,
                            uint32_t* d_error, void* stream) {
  if (!d_w_bf16 || !d_w_f32 || !d_features || !d_logits || !d_error || ((uintptr_t)d_features & 15u) || ((uintptr_t)d_logits & 15u))
    return rsx_set_last_error(RSX_E_ARG, "rsx_pred_forward_tc_raw: null buffer, or features / logits not 16-byte aligned");
  if (n == 0) return RSX_OK;
  RSX_CK(rsx_launch_pred_forward_tc(d_w_bf16, d_w_f32, d_features, n, d_logits, nullptr, d_error, (cudaStream_t)stream));
  return RSX_OK;
}

int rsx_pred_levels_raw(const float* d_logits, uint32_t n, const float* weights, uint32_t levels, uint32_t* d_scratch, uint32_t* d_order,
                        void* stream) {
  if (!d_logits || !weights || !d_scratch || !d_order || levels < 2 || levels > 32)
    return rsx_set_last_error(RSX_E_ARG, "rsx_pred_levels_raw: null buffer or levels outside 2..32");
  if (n == 0) return RSX_OK;
  RSX_CK(rsx_launch_pred_levels(d_logits, n, weights, (int)levels, d_scratch, d_order, (cudaStream_t)stream));
  return RSX_OK;
}

int rsx_profile_phases_raw(uint32_t* d_states, uint32_t n, const void* d_statics, const uint8_t* d_sd_index, const rsx_controls* d_controls,
                           uint64_t* d_phase_cycles, void* stream) {
  if (!d_states || !d_statics || !d_controls || !d_phase_cycles) return RSX_E_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  RSX_CK(cudaMemsetAsync(d_phase_cycles, 0, 10 * sizeof(uint64_t), s));
  if (n == 0) return RSX_OK;
  RSX_CK(rsx_launch_sim8_profile(d_states, d_statics, d_sd_index, d_controls, n, (unsigned long long*)d_phase_cycles, s));
  return RSX_OK;
}

}  // extern "C"
