/* rsx: the soccar 1v1 8-tick decision step on B200 (sm_100a), as a C ABI.
 *
 * Drop-in for the device path of the reference's Rust host crate (crates/rocketsim-cuda/src/device.rs, SimDevice):
 * arena states in AoSoA-32 buffers of u32 words (word w of arena a at (a/32)*32*2784 + w*32 + a%32), one StaticData
 * of 317,895 words per car pairing, controls as 8 words per car, one result word per arena.  Every entry point returns
 * an int status (RSX_OK or a negative RSX_E*); nothing throws across the ABI.  Launch entry points are asynchronous on
 * the handle's stream; downloads synchronise.  All layouts are the reference's (cuda/sim/arena_state.cuh:42-339).
 */
#ifndef RSX_H
#define RSX_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define RSX_OK 0
#define RSX_E_ARG (-1)      /* a bad argument (null handle, block outside 1..64, buffer too short) */
#define RSX_E_CUDA (-2)     /* a CUDA runtime error (rsx_last_error() names it) */
#define RSX_E_NODEV (-3)    /* no CUDA device / no sm_100 device */
#define RSX_E_TIMEOUT (-4)  /* a bounded device wait gave up (persistent kernel) */
#define RSX_E_FORMAT (-5)   /* a V3 dump that does not import (rsx_last_error() says why, in the reference's words) */

/* ---- constants (device.rs:16-28, arena_step.cuh:16-18) ---- */
#define RSX_TICKS_PER_DECISION 8u
#define RSX_SCORED_MASK 0xFFu
#define RSX_UNIMPLEMENTED 0x80000000u
#define RSX_OVERFLOW 0x40000000u
#define RSX_SIM8_BLOCK 32u
#define RSX_MAX_BLOCK 64u

/* Controls of one car (arena_state.cuh:77-80): throttle, steer, pitch, yaw, roll as f32, then jump, boost, handbrake 0/1. */
typedef struct rsx_controls {
  float throttle, steer, pitch, yaw, roll;
  uint32_t jump, boost, handbrake;
} rsx_controls;

typedef struct rsx_device rsx_device;    /* SimDevice: a device, its stream */
typedef struct rsx_static rsx_static;    /* DeviceStatic: one or more StaticData on the device */
typedef struct rsx_states rsx_states;    /* DeviceStates: n arenas in one AoSoA-32 buffer */

/* ---- layout (layout.rs; lf_arena_words / lf_tick_words / lf_static_words of csrc/phase.cpp:18-22) ---- */
uint64_t rsx_arena_words(void);            /* 2784 */
uint64_t rsx_tick_words(void);             /* 2567: the words that cross a tick */
uint64_t rsx_static_words(void);           /* 317,895 */
uint64_t rsx_aosoa_words(uint32_t n);      /* words of an AoSoA-32 buffer of n arenas (aosoa.cuh:15) */
uint64_t rsx_aosoa_index(uint32_t a, uint32_t w);  /* aosoa.cuh:17 */
/* host-side pack / unpack between n contiguous ArenaStates and AoSoA-32 (aosoa.rs:9-38) */
void rsx_aosoa_pack(const uint32_t* states, uint32_t n, uint32_t* aosoa);
void rsx_aosoa_unpack(const uint32_t* aosoa, uint32_t n, uint32_t* states);
const char* rsx_last_error(void);

/* ---- device (SimDevice::new, device.rs:53-67; cuda.rs:18-28 context with an 8 KiB stack) ---- */
int rsx_device_create(int ordinal, rsx_device** out);
int rsx_device_destroy(rsx_device* dev);
int rsx_sync(rsx_device* dev);
void* rsx_device_stream(rsx_device* dev);  /* the handle's cudaStream_t */

/* ---- static data (SimDevice::upload_static, device.rs:69) ---- */
/* `count` StaticData back to back (count 1 is the reference's single car pairing) */
int rsx_static_upload(rsx_device* dev, const uint32_t* words, uint32_t count, rsx_static** out);
int rsx_static_free(rsx_static* sd);
const void* rsx_static_device_ptr(rsx_static* sd);

/* ---- states (upload_states / alloc_states / download_words, device.rs:74-90) ---- */
int rsx_states_alloc(rsx_device* dev, uint32_t n, rsx_states** out);
int rsx_states_free(rsx_states* st);
int rsx_states_upload(rsx_device* dev, rsx_states* st, const uint32_t* aosoa);     /* rsx_aosoa_words(n) words */
int rsx_states_download(rsx_device* dev, rsx_states* st, uint32_t* aosoa);         /* synchronises */
uint32_t* rsx_states_device_ptr(rsx_states* st);
/* device-to-device copy of `bytes` on a caller stream (snapshots of a state buffer; no counterpart in the reference) */
int rsx_copy_raw(void* d_dst, const void* d_src, uint64_t bytes, void* stream);

/* ---- the decision (SimDevice::sim8, device.rs:155-168; kernel sim.cu:95-104) ----
 * One decision of every arena in place: 8 ticks with controls[a*2+i] (device memory, 16 words per arena), result[a] the
 * scored tick | RSX_UNIMPLEMENTED | RSX_OVERFLOW (device memory).  block: 1..64 threads (RSX_SIM8_BLOCK in production).
 * trace: null, or 8 AoSoA buffers (8 * rsx_aosoa_words(n) words, device memory) that receive the state after each tick. */
int rsx_sim8(rsx_device* dev, rsx_states* st, rsx_static* sd, const rsx_controls* d_controls, uint32_t* d_result, uint32_t block,
             uint32_t* d_trace);
/* the same on raw device pointers and a caller stream (the path torch / CUDA-graph callers use) */
int rsx_sim8_raw(uint32_t* d_states, uint32_t n, const void* d_static, const rsx_controls* d_controls, uint32_t* d_result,
                 uint32_t block, uint32_t* d_trace, void* stream);
/* one full tick (step_tick_k, sim.cu:46-53) and one phase (phase_k, sim.cu:27-34); status[a] is the PhaseStatus */
int rsx_step_tick(rsx_device* dev, rsx_states* st, rsx_static* sd, int32_t* d_status);
int rsx_phase(rsx_device* dev, int k, rsx_states* st, rsx_static* sd, int32_t* d_status);
/* the copy-in / copy-out round trip (sim_identity[_tick], sim.cu:9-24) */
int rsx_identity(rsx_device* dev, const uint32_t* d_in, uint32_t* d_out, uint32_t n, int tick_only);

/* ---- extensions (no counterpart in the reference's kernel set; the functions above are unchanged by them) ----
 * Per-arena car pairing: d_static points at `count` StaticData, sd_index[a] (u8, device memory) selects arena a's. */
int rsx_sim8_multi_raw(uint32_t* d_states, uint32_t n, const void* d_statics, const uint8_t* d_sd_index,
                       const rsx_controls* d_controls, uint32_t* d_result, uint32_t* d_event_or, uint32_t block, void* stream);
/* The persistent kernel: `grid` resident blocks pull work items (32 x `granularity` arenas per warp) from a device
 * queue: entries of d_order (identity when null; a binned order puts arenas of like predicted cost together) claimed
 * with atomics on d_queue_counter (cleared by the call).  At most 2^24 arenas, granularity 256 and grid 65,535 per call
 * (RSX_E_ARG beyond: the 32-bit counter must not wrap).  Results do not depend on grid, block, granularity or order
 * (no cross-arena arithmetic). */
int rsx_sim8_persistent_raw(uint32_t* d_states, uint32_t n, const void* d_statics, const uint8_t* d_sd_index,
                            const rsx_controls* d_controls, uint32_t* d_result, uint32_t* d_event_or,
                            const uint32_t* d_order, uint32_t* d_queue_counter, uint32_t grid, uint32_t block,
                            uint32_t granularity, void* stream);

/* The same with the register budget of the kernel (min_blocks of 64 threads resident per SM: 1 -> 255 registers,
 * 8 -> 128, 12 -> 80, 16 -> 64) and, when d_cost is non-null, each arena's decision cost in clock cycles >> 8. */
int rsx_sim8_persistent_ex(uint32_t* d_states, uint32_t n, const void* d_statics, const uint8_t* d_sd_index,
                           const rsx_controls* d_controls, uint32_t* d_result, uint32_t* d_event_or, const uint32_t* d_order,
                           uint32_t* d_queue_counter, uint32_t grid, uint32_t block, uint32_t granularity, uint32_t min_blocks,
                           uint32_t* d_cost, void* stream);
/* The SM-lockstep persistent decision (no counterpart in the reference): `grid` resident blocks of `block` threads (a
 * multiple of 32, at most RSX_LOCKSTEP_MAX_BLOCK; normally one block per SM) step their warps' arenas phase by phase
 * together, so that all warps of an SM execute one phase's code at a time; each warp claims 32 entries of d_order
 * (identity when null) from d_queue_counter (cleared by the call) when its arenas finish.  split 1 adds a barrier after
 * each car's pre-tick inside P1; split 2 splits each car's P1 into pre-tick head, wheel rays and wheel response; split 3 adds a barrier
 * after every step of P3b's pair / leaf loop; split 4 / 5 drop the barriers from P3b / P4 to P8 (slower: kept for
 * measurement); split 6 is split 2 with P5 (rows, iterations, integration) and P8 (cars, the rest) in parts; split 7 is
 * split 6 with P3a one dynamic body at a time; split 9 is split 7 with P3b's mesh-leaf tests pooled over the block (each
 * round every arena's next BVH leaves are tested by all threads; the owners add the hits in walk order); split 10 is
 * split 9 with the wheel rays' mesh leaves pooled too (per car, every mesh candidate's leaves evaluated by all threads
 * in one round, the owners replaying them in candidate and walk order); split 11 is split 10 with P3a in one piece;
 * split 14 is split 11 with the 47 feature pairs of the box-triangle SATs that reach them computed by the whole block
 * (up to 18 SATs per round); split 15 is split 14 with the wheel rays' mesh walks run by the whole block level by level
 * (their leaves sorted back into each walk's order; the default: the fastest measured).  Register budget by block: up to 448 threads 144 registers, 512 128.  At
 * most 2^24 arenas and grid 65,535 per call.  Results equal rsx_sim8_multi_raw's whatever grid, block, split or order. */
#define RSX_LOCKSTEP_MAX_BLOCK 512u
int rsx_sim8_lockstep_raw(uint32_t* d_states, uint32_t n, const void* d_statics, const uint8_t* d_sd_index,
                          const rsx_controls* d_controls, uint32_t* d_result, uint32_t* d_event_or, const uint32_t* d_order,
                          uint32_t* d_queue_counter, uint32_t grid, uint32_t block, uint32_t split, void* stream);
/* The same decision in 8 / ticks_per_launch launches of ticks_per_launch ticks each (1, 2, 4 or 8; no counterpart in
 * the reference, whose step_ticks takes the tick count, arena_step.cuh:83-105): every launch re-claims the arenas from
 * the queue, and each arena's progress between launches rides in d_result (scored tick, RSX_UNIMPLEMENTED) and
 * d_event_or (the event OR so far); an arena scored in an earlier launch is not stepped again and keeps its goal state.
 * The words after the last launch equal rsx_sim8_lockstep_raw's.  A tuning knob: with several claim rounds, shorter
 * launches re-balance the arenas across SMs more often. */
int rsx_sim8_lockstep_ex(uint32_t* d_states, uint32_t n, const void* d_statics, const uint8_t* d_sd_index,
                         const rsx_controls* d_controls, uint32_t* d_result, uint32_t* d_event_or, const uint32_t* d_order,
                         uint32_t* d_queue_counter, uint32_t grid, uint32_t block, uint32_t split, uint32_t ticks_per_launch,
                         void* stream);

/* The persistent decision without caller scratch (no counterpart in the reference): for callers that cannot allocate
 * device memory (their framework owns it, or cudaMalloc / cudaFree would synchronise a real-time loop), the work-queue
 * counter lives in a fixed 256-byte device array of the library instead of d_queue_counter.  At most 2^24 arenas,
 * granularity 256 and grid 65,535 per call (RSX_E_ARG beyond).  The first call on a device looks the array up (make it
 * before any stream capture), and so does the first call after a device reset; calls share the array, so calls whose
 * launches overlap on the GPU race.  Results equal rsx_sim8_persistent_raw's. */
int rsx_sim8_persistent_noalloc(uint32_t* d_states, uint32_t n, const void* d_statics, const uint8_t* d_sd_index,
                                const rsx_controls* d_controls, uint32_t* d_result, uint32_t* d_event_or, const uint32_t* d_order,
                                uint32_t grid, uint32_t block, uint32_t granularity, void* stream);

/* Phase profile of one decision (no counterpart in the reference): d_phase_cycles[10] receives, per phase P0, P1, P2,
 * P3a, P3b, P4, P5, P6, P7, P8, the clock cycles all warps spent in it over the 8 ticks (zeroed by the call).  The states
 * advance by one decision; the goal state is not kept, so use it on a copy. */
int rsx_profile_phases_raw(uint32_t* d_states, uint32_t n, const void* d_statics, const uint8_t* d_sd_index,
                           const rsx_controls* d_controls, uint64_t* d_phase_cycles, void* stream);

/* L2 residency for the static data (no counterpart in the reference): a persisting-access window over
 * [d_ptr, d_ptr + bytes) on `stream` (bytes 0: remove it), hit_ratio in (0, 1] (scaled down when the window exceeds the
 * device's persisting carve-out).  The carve-out is a limit of the calling process's context. */
int rsx_l2_persist_raw(const void* d_ptr, uint64_t bytes, float hit_ratio, void* stream);

/* Device resets (no counterpart in the reference): the arenas selected by d_mask (u8, nonzero: reset; null: all) and
 * by d_result (the last decision's result words; null: no condition, else only arenas whose decision scored) get the
 * start state rsx_make_states_multi builds for the same seed, arena index, StaticData and mix[5] (host memory),
 * written into the AoSoA-32 buffer (all 2784 words); d_reset_count (nullable) is incremented per reset arena. */
int rsx_reset_arenas_raw(uint32_t* d_states, uint32_t n, const void* d_statics, const uint8_t* d_sd_index, uint64_t seed,
                         const float* mix, const uint32_t* d_result, const uint8_t* d_mask, uint32_t* d_reset_count, void* stream);

/* ---- the contact predictor (no counterpart in the reference: the binning it drives is this library's) ----
 * A 48 -> 128 -> 128 -> 128 -> 6 ReLU MLP (sigmoid outputs) over per-arena features, BF16 weights and activations
 * with FP32 accumulation, trained on the decision kernels' event-OR labels.  Weights: RSX_PRED_PARAMS FP32 master
 * values and a BF16 copy (uint16 words) of the same layout: W1[128][48] b1[128] W2[128][128] b2[128] W3[128][128]
 * b3[128] W4[8][128] b4[8] (rows 6 and 7 of W4 zero).  Labels: bit 0 car 0 - ball, 1 car 1 - ball, 2 car - car,
 * 3 ball - world, 4 car 0 - world, 5 car 1 - world.  All buffers are device memory; calls are asynchronous. */
#define RSX_PRED_FEATURES 48
#define RSX_PRED_LABELS 6
#define RSX_PRED_PARAMS 40328
int rsx_pred_features_raw(const uint32_t* d_states, uint32_t n, const void* d_statics, const uint8_t* d_sd_index,
                          const rsx_controls* d_controls, uint16_t* d_features, void* stream);
int rsx_pred_labels_raw(const uint32_t* d_event_or, uint32_t n, uint8_t* d_labels, void* stream);
/* logits[n][8] (FP32; outputs 6, 7 unused) */
int rsx_pred_forward_raw(const uint16_t* d_w_bf16, const float* d_w_f32, const uint16_t* d_features, uint32_t n, float* d_logits,
                         void* stream);
/* The same forward on the 5th-generation tensor cores (tcgen05.mma, accumulators in tensor memory; 128 arenas per
 * tile, one CTA per SM), the one inference and training use (training's forward also saves the activations).
 * Logits equal rsx_pred_forward_raw's up to FP32 summation order.  d_error[0] is set to 1 if a bounded wait for the
 * tensor cores gave up (the logits are then incomplete); features and logits 16-byte aligned. */
int rsx_pred_forward_tc_raw(const uint16_t* d_w_bf16, const float* d_w_f32, const uint16_t* d_features, uint32_t n, float* d_logits,
                            uint32_t* d_error, void* stream);
/* BF16 elements of the training scratch for a batch of n */
uint64_t rsx_pred_scratch_elems(uint32_t n);
/* gradients of L = (1/n) sum over the batch and the 6 outputs of the binary cross-entropy: d_grad[RSX_PRED_PARAMS]
 * (overwritten), d_loss[0] = n L, d_logits[n][8] the forward's logits.  Forward, backward through the layers and the
 * weight gradients all run on tcgen05 (their wait flag in the scratch's last two elements). */
int rsx_pred_gradients_raw(const uint16_t* d_w_bf16, const float* d_w_f32, const uint16_t* d_features, const uint8_t* d_labels,
                           uint32_t n, uint16_t* d_scratch, float* d_logits, float* d_grad, float* d_loss, void* stream);
/* one Adam step (beta 0.9, 0.999, eps 1e-8) of the FP32 master weights with moments d_m, d_v; refreshes the BF16 copy */
int rsx_pred_adam_raw(float* d_w_f32, uint16_t* d_w_bf16, float* d_m, float* d_v, const float* d_grad, uint32_t step, float lr,
                      void* stream);
int rsx_pred_to_bf16_raw(const float* d_w_f32, uint16_t* d_w_bf16, void* stream);
/* Bins: arena a is contact-heavy when any output in label_mask (bit k: output k; 0x3F all six) has its logit above
 * threshold_logit.  d_order[n] lists the heavy arenas then the quiet ones, each in arena order; d_heavy_count[0] their
 * number; d_scratch ceil(n / 1024) words. */
int rsx_pred_bin_raw(const float* d_logits, uint32_t n, float threshold_logit, uint32_t label_mask, uint32_t* d_scratch,
                     uint32_t* d_order, uint32_t* d_heavy_count, void* stream);
/* Cost levels: e = sum_k weights[k] * sigmoid(logit_k) over the six outputs (weights: 6 host floats), quantised to
 * `levels` (2..32) levels of e / max(e) over the batch; d_order[n] lists the arenas by level, highest first, each level
 * in arena order.  d_scratch 1 + levels * ceil(n / 1024) words.  With several claim rounds of the lockstep kernel
 * (more arenas than its threads), the costliest arenas start first. */
int rsx_pred_levels_raw(const float* d_logits, uint32_t n, const float* weights, uint32_t levels, uint32_t* d_scratch, uint32_t* d_order,
                        void* stream);

/* ---- observations and rewards for a learner (no counterpart in the reference, which defines no observation; its
 * FP16 conversion, cuda/common/hd.cuh:167-176, is the rounding used: nearest even, as cvt.rn.f16.f32) ----
 * After a decision, per arena a and car c (row 2a + c): RSX_OBS_DIM FP16 values, seen from c's side (car 1's x and y
 * negated, its pads in mirrored order), positions and velocities / 2300, angular velocities / pi, boost / 100:
 *   [0,9) ball position, velocity, angular velocity; [9,24) own position, forward (rotation x axis), up (z axis),
 *   velocity, angular velocity; [24] boost; [25..29] on ground, has jumped, has double jumped, has flipped, demoed;
 *   [30,36) ball minus own position and velocity; [36,51) opponent position, forward, up, velocity, angular velocity;
 *   [51..53] opponent boost, on ground, demoed; [54,60) opponent minus own position and velocity; [60,68) own
 *   controls (5 axes, jump, boost, handbrake as 0/1); [68,102) boost pads active (the game's cooldown test) 0/1;
 *   [102,104) zero.
 * Reward per car: sum over k of weights[k] * term[k] (FP32, k ascending): goal (+1 own team scored, -1 conceded, from
 * the result word and the ball's side), ball touch, bump given, demo given, demoed, boost pickup (the decision's event
 * OR; 0 without it), own velocity toward the ball / 2300, ball velocity toward the opponent's goal / 2300.
 * d_obs must be 16-byte aligned; d_pad_mirror (count x 34 bytes from rsx_pad_mirror) and d_reward may be NULL. */
#define RSX_OBS_DIM 104u
#define RSX_REWARD_TERMS 8u
int rsx_pad_mirror(const uint32_t* statics, uint32_t count, uint8_t* out);
int rsx_observe_raw(const uint32_t* d_states, uint32_t n, const void* d_statics, const uint8_t* d_sd_index, const uint8_t* d_pad_mirror,
                    const uint32_t* d_result, const uint32_t* d_event_or, const float* weights, uint16_t* d_obs, float* d_reward,
                    void* stream);

/* ---- host side: the synthetic world and seeded start states (the game's meshes and V3's dumps are absent) ---- */
/* builds one StaticData (317,895 words) for the car pairing (preset0, preset1), presets 0..6; returns the triangle count */
int rsx_build_static(uint32_t* words, uint64_t seed, int preset0, int preset1);
/* n fresh ArenaStates (2784 words each, contiguous): scenario mix[5] = kickoff, open play, head-on, pinch, pad contention */
int rsx_make_states(const uint32_t* static_words, uint32_t* states, uint32_t n, uint64_t seed, const float* mix);
/* per-arena car pairings: statics[count], sd_index[a] < count selects arena a's StaticData */
int rsx_make_states_multi(const uint32_t* statics, uint32_t count, const uint8_t* sd_index, uint32_t* states, uint32_t n,
                          uint64_t seed, const float* mix);
/* the start states of chosen arenas: states[j] is arena arena_index[j]'s state for (seed, statics[sd_index[j]], mix),
 * the words rsx_make_states_multi and the device's rsx_reset_arenas_raw give that arena */
int rsx_make_states_at(const uint32_t* statics, uint32_t count, const uint8_t* sd_index, const uint32_t* arena_index, uint32_t k,
                       uint64_t seed, const float* mix, uint32_t* states);
/* the same source compiled for the host (for debugging and CPU-side checks; the device entry points never call these) */
int rsx_host_phase(int k, uint32_t* state_words, const uint32_t* static_words);
uint32_t rsx_host_decide(uint32_t* state_words, const uint32_t* static_words, const rsx_controls* controls2);

/* ---- V3 dumps (crates/rocketsim-cuda/src/dump.rs:1-1300; the V3 side: v3/rocketsim-dump.patch, src/dump.rs) ----
 * Import and export of the per-arena state ("V3ARENA\0" version 2) and the static collision data ("V3STATIC"
 * version 3, FNV-1a 64 over its payload) that the patched RocketSim V3 writes.  Host functions; buffers are the
 * caller's.  A write returns RSX_E_ARG with the size it needs in *len when out is NULL or cap is short.  An import
 * that the reference refuses (a list over its cap, another game mode's state, constants that differ from StaticData,
 * a truncated or trailing dump) returns RSX_E_FORMAT with the reference's message in rsx_last_error(). */
#define RSX_V3_ARENA_HEADER_LEN 68u   /* magic, version, config hash, 12 u32 counts (dump.rs:18) */
#define RSX_V3_STATIC_HEADER_LEN 76u  /* magic, version, payload hash, payload length, 12 u32 counts (dump.rs:19) */
#define RSX_V3_BODY_RECORD_LEN 219u   /* one BODY record (dump.rs:21) */
/* What an ArenaState leaves out of a V3 arena dump (dump.rs:209-238, Template): the config hash, the BODY records of
 * the static bodies, the sweep-and-prune counters, the manifold table stride and the other modes' ball info. */
typedef struct rsx_v3_template {
  uint64_t config_hash;
  uint8_t static_body[23][RSX_V3_BODY_RECORD_LEN];
  uint16_t num_handles, next_new_handle;
  uint32_t manifold_stride;
  uint8_t ball_other[24];
  uint32_t ball_other_set;
} rsx_v3_template;
uint64_t rsx_v3_fnv1a64(const uint8_t* bytes, size_t len);                          /* dump.rs:30-36 */
int rsx_v3_parse_static(const uint8_t* bytes, size_t len, uint32_t* static_words);  /* parse_static, dump.rs:976-1012 */
/* the static dump of a StaticData (the V3 side's export_static layout); the reference only reads these */
int rsx_v3_write_static(const uint32_t* static_words, uint8_t* out, size_t cap, size_t* len);
/* config_hash of a StaticData: FNV-1a over its static dump's WRLD, BODY, PLAN, CARS and PADS sections */
int rsx_v3_config_hash(const uint32_t* static_words, uint64_t* hash);
/* a template for a StaticData without a V3 dump (unmoving, unrotated static bodies) */
int rsx_v3_template_init(const uint32_t* static_words, rsx_v3_template* t);
/* parse_arena (dump.rs:884-900): one arena dump into 2784 state words and its template */
int rsx_v3_parse_arena(const uint8_t* bytes, size_t len, const uint32_t* static_words, uint32_t* state_words, rsx_v3_template* t);
/* write_arena (dump.rs:902-944) */
int rsx_v3_write_arena(const uint32_t* state_words, const uint32_t* static_words, const rsx_v3_template* t, uint8_t* out, size_t cap,
                       size_t* len);

/* ---- verification of the FP64-free correctly rounded libm (sin, cos, tan, atan2, pow and the auto-flip helpers) ----
 * fn 0 sin, 1 cos, 2 tan, 3 atan2(a, b), 4 pow(a, b), 5 float(double atan2(a, b)), 6 float(double hypot(a, b)) */
int rsx_libm_host(int fn, const float* a, const float* b, float* out, uint64_t n);
/* order-independent hash of f over [first_bits, first_bits + count): sum of mix64((x << 32) | f(x)), NaN canonical */
uint64_t rsx_libm_hash_host(int fn, uint32_t first_bits, uint32_t count);
/* the same hash on the device for chunks of 2^24 inputs (fn 0..2), d_hashes[nchunks] */
int rsx_libm_chunk_hashes(int fn, uint32_t first_chunk, uint32_t nchunks, uint64_t* d_hashes, void* stream);

#ifdef __cplusplus
}
#endif
#endif
