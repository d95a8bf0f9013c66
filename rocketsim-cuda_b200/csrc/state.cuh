// The arena state and the static data of one Soccar 1v1 arena, word for word in the layout the reference's host crate
// exchanges (cuda/sim/arena_state.cuh:42-339; its Rust mirror crates/rocketsim-cuda/src/layout.rs).  This layout is the
// drop-in format: states that a user uploads, downloads or exports are these words, so every field keeps the
// reference's position and meaning.  Every member is a 4-byte word or a struct of them (no padding): an arena is an
// array of u32 words, moved AoSoA-32 by the kernels.
//
//   * flags are u32 0/1; an optional is {u32 some; T v} with v zero when absent; a u64 is {lo, hi};
//   * a list is a count plus a fixed array, with an overflow counter bumped instead of writing past the cap;
//   * the part after `events` is live only inside a tick (zero at a tick boundary): TICK_WORDS words cross a tick.
#pragma once
#include <stddef.h>
#include "vmath.cuh"

namespace rsx {

constexpr int kBodies = 23;       // 16 meshes, 4 planes, ball, 2 cars
constexpr int kDyn = 3;           // ball (body 20), car 0 (21), car 1 (22)
constexpr int kCars = 2;
constexpr int kWheels = 4;
constexpr int kPads = 34;
constexpr int kHandles = 24;      // sweep-and-prune handles: sentinel + 23 bodies
constexpr int kEdges = 2 * kHandles;
constexpr int kMeshes = 16;
constexpr int kPlanes = 4;

constexpr int kMaxManifolds = 16;
constexpr int kMaxPoints = 4;
constexpr int kMaxActive = 16;
constexpr int kMaxRecords = 16;
constexpr int kMaxPairs = 16;
constexpr int kMaxDynCells = 64;

enum Ovf { OVF_MANIFOLDS, OVF_ACTIVE, OVF_RECORDS, OVF_PAIRS, OVF_DYN_CELLS, OVF_PAD_TOUCHING, OVF_COUNT };

// events word: bit (kind + car index)
enum Ev : uint32_t {
  EV_CAR_HIT_BALL = 0, EV_BUMP = 2, EV_DEMO = 4, EV_PICKUP = 6, EV_LANDED = 8, EV_CAR_HIT_WORLD = 10,
  EV_BALL_HIT_WORLD = 12, EV_BALL_WALL = 14,
};

struct U64W { uint32_t lo, hi; };
RSX_F uint64_t u64_of(U64W x) { return ((uint64_t)x.hi << 32) | x.lo; }
RSX_F U64W u64w(uint64_t v) { return U64W{(uint32_t)v, (uint32_t)(v >> 32)}; }
template <class T> struct Opt { uint32_t some; T v; };

struct Controls { float throttle, steer, pitch, yaw, roll; uint32_t jump, boost, handbrake; };
struct HitInfo { V3 hit_point, hit_normal; float hit_fraction; uint32_t user_info; };
struct RayInfo {
  V3 contact_normal, contact_point;
  uint32_t ground_body;
  float suspension_length;
  V3 impulse;
  Opt<V3> ground_stick;
  uint32_t in_contact_with_world;
  float clipped_inv_contact_dot_susp;
  float susp_rel_vel;
};
struct Wheel {
  Opt<RayInfo> ray;
  V3 hard_point, axle_dir;
  float engine_force, brake, steer_angle;
  V3 vel_at_contact;
  float lat_friction, long_friction, extra_pushback;
};
struct Car {
  float dodge_deadzone;
  V3 vel_impulse_cache;
  uint32_t sticky_gate_prev;
  V3 pos;
  M3 rot;
  V3 vel, ang_vel;
  Controls controls;
  uint32_t has_jumped, has_double_jumped, has_flipped;
  V3 flip_rel_torque;
  uint32_t jump_ticks;
  float flip_time;
  uint32_t is_flipping, is_jumping, jump_hold_broken;
  float air_time, air_time_since_jump, boost, handbrake_val;
  uint32_t is_supersonic;
  float supersonic_grace, time_since_boosted, boosting_time;
  uint32_t is_boosting, is_auto_flipping;
  float auto_flip_timer, auto_flip_torque_scale, bump_cooldown;
  Opt<uint32_t> bump_victim;
  Opt<U64W> last_extra_hit_tick;
  uint32_t is_demoed;
  float demo_respawn_timer;
  uint32_t on_ground;
  Opt<HitInfo> wheel_contact[kWheels];
  Opt<V3> world_contact_normal;
  Controls prev_controls;
  Wheel wheels[kWheels];
};
struct PadTouch { uint32_t n; uint32_t car[kCars]; };
struct Ball { V3 pos; M3 rot; V3 vel, ang_vel; U64W ticks_since_kickoff; };
struct Body {
  uint32_t flags;          // collision flags
  uint32_t activation;     // 0 active, 1 sleeping, 2 disabled, 3 wants deactivation
  float deactivation_time;
  Aff xf;                  // world transform (Bullet units)
  Q4 quat;
  Aff pred;                // predicted (interpolation) transform, live P2..P6
  V3 lin_vel, ang_vel;
  M3 inv_inertia_world;
  V3 acc_lin, acc_ang;     // accumulated impulses, live P1..P6
  float damp_cache, damp_cache_dt, damp_cache_value;
};
struct MPoint {
  V3 local_a, local_b, world_b, world_a, normal_b;
  float dist, friction, restitution;
  uint32_t special;
};
struct Manifold { uint32_t body0, body1, n; MPoint pts[kMaxPoints]; };
struct RecPoint { V3 world_b, world_a, normal_b; };
struct Record { uint32_t swapped, body_a, body_b; RecPoint p; };
struct DynProxy { Box3 box; uint32_t cell; uint32_t idx[3]; };
struct HandleEdges { uint16_t lo[3], hi[3]; };
struct Edge { uint16_t pos, handle; };
struct DynCell { uint32_t cell, handle; };
struct Pair { uint32_t h0, h1; };

struct ArenaState {
  U64W tick_count;
  U64W rng;
  Ball ball;
  Car cars[kCars];
  Opt<U64W> pad_gave[kPads];
  PadTouch pad_touch[kPads];
  Body bodies[kDyn];
  uint32_t n_manifolds;
  Manifold manifolds[kMaxManifolds];
  uint32_t n_dyn_cells;
  DynCell dyn_cells[kMaxDynCells];
  DynProxy dyn_proxy[kDyn];
  HandleEdges handle_edges[kHandles];
  Edge edges[3][kEdges];
  uint32_t n_pairs;
  Pair pairs[kMaxPairs];
  uint32_t overflow[OVF_COUNT];
  uint32_t events;
  // ---- mid-tick only (zero at a tick boundary) ----
  uint32_t n_active;
  uint32_t active[kMaxActive];
  uint32_t fold_events;
  V3 fold_car_normal[kCars];
  uint32_t n_records;
  Record records[kMaxRecords];
};

constexpr int kArenaWords = (int)(sizeof(ArenaState) / 4);
constexpr int kTickWords = (int)(offsetof(ArenaState, n_active) / 4);
static_assert(sizeof(ArenaState) % 4 == 0, "an arena is an array of words");

// ---- static data ----
constexpr int kMaxTris = 8020;
constexpr int kMaxNodes = 3754;
constexpr int kMaxLeaves = 8020;
constexpr int kTableSin = 16384;
constexpr int kGridCells = 242;
constexpr int kMaxCellEntries = 1210;
constexpr int kMut = 20;

struct MeshInfo { uint32_t body, tri_first, tri_count, node_first, node_count, leaf_first, leaf_count; Box3 ident_box, root_box; };
struct Tri { V3 p0, p1, p2, n; };
struct WideNode {
  float lo_x[4], lo_y[4], lo_z[4], hi_x[4], hi_y[4], hi_z[4];
  uint32_t child[4];   // bit 31: a leaf
  uint32_t n_child;
  uint32_t valid;      // (1 << n_child) - 1
};
struct Leaf { Box3 box; uint32_t tri; };
struct TriInfo { uint32_t flags; float a01, a12, a20; };
struct Plane { uint32_t body; V3 n; uint32_t single_axis, axis, backwards; Box3 ident_box, box; };
struct BodyConst {
  uint32_t world_idx, user, user_ptr, handle, group, mask;
  float mass, inv_mass;
  V3 inv_inertia_local, inv_mass3;
  float friction, restitution, processing_threshold, breaking_threshold;
  float lin_damping, lin_sleep, ang_sleep;
  Aff pose;
  uint32_t shape;      // 0 mesh, 1 plane, 2 sphere, 3 compound (car box)
  V3 sphere_dim;
  float sphere_margin;
  V3 box_half;
  float box_margin;
  Aff child;
  Box3 compound_box;
  uint32_t mesh_tris;
};
struct WheelConst { V3 connection; float rest_length, radius, force_scale, ray_length; };
struct CarConst { uint32_t car_idx, team, body, three_wheels; V3 hitbox_size, hitbox_offset; WheelConst wheels[kWheels]; };
struct PadConst { V3 pos; uint32_t big; float box_radius, cyl_radius, cooldown, amount; Box3 box; };
struct ProxyConst { uint32_t body, group, mask, uid; Box3 box; uint32_t cell, idx[3]; };
struct CellRange { uint32_t first, count; };

struct StaticData {
  uint32_t game_mode, no_ball_rot, ball_body;
  V3 gravity_uu;
  float mut[kMut];
  uint32_t unlimited_flips, unlimited_double_jumps, recharge_boost;
  float recharge_per_second, recharge_delay;
  uint32_t demo_mode, team_demos;
  float goal_y;
  uint32_t pads_enabled;
  V3 gravity_bt;
  uint32_t dyn_body[kDyn];
  V3 grid_lo, grid_hi;
  float cell_size, cell_size_sq;
  uint32_t grid_n[3];
  V3 sap_lo, sap_quant;
  uint32_t sap_mask, sap_sentinel, sap_max_handles;
  float sap_half_extent;
  float max_pad_z;
  uint32_t dyn_handle[kDyn];
  BodyConst bodies[kBodies];
  Plane planes[kPlanes];
  MeshInfo meshes[kMeshes];
  CarConst cars[kCars];
  PadConst pads[kPads];
  ProxyConst proxies[kHandles];
  CellRange cells[kGridCells];
  uint32_t cell_handles[kMaxCellEntries];
  TriInfo infos[kMaxTris];
  Tri tris[kMaxTris];
  WideNode nodes[kMaxNodes];
  Leaf leaves[kMaxLeaves];
  float table_sin[kTableSin];
};
constexpr int kStaticWords = (int)(sizeof(StaticData) / 4);
static_assert(sizeof(StaticData) % 4 == 0, "static data is an array of words");

// mutator floats (StaticData.mut order)
enum Mut {
  M_CAR_MASS, M_BALL_MASS, M_BALL_MAX_SPEED, M_BALL_DRAG, M_JUMP_ACCEL, M_JUMP_IMMEDIATE, M_BOOST_ACCEL_GROUND,
  M_BOOST_ACCEL_AIR, M_BOOST_PER_SECOND, M_RESPAWN_DELAY, M_BUMP_COOLDOWN, M_MAX_BOOST, M_SPAWN_BOOST, M_PAD_SMALL,
  M_PAD_BIG, M_PAD_COOLDOWN_BIG, M_PAD_COOLDOWN_SMALL, M_HIT_EXTRA_SCALE, M_BUMP_FORCE_SCALE, M_BALL_RADIUS
};

// result word of one decision
constexpr uint32_t kTicksPerDecision = 8;
constexpr uint32_t kScoredMask = 0xFFu;
constexpr uint32_t kUnimplemented = 0x80000000u;
constexpr uint32_t kOverflow = 0x40000000u;

// launch limits of the queue-driven kernels: the 32-bit queue counter must not wrap (n plus the overshoot of the last
// claims; the lockstep kernel's idle warps claim once per tick); 2^24 arenas are 187 GB of AoSoA state, more than a GPU
// holds
constexpr uint32_t kQueueMaxArenas = 1u << 24;
constexpr uint32_t kQueueMaxGran = 256;
constexpr uint32_t kQueueMaxGrid = 65535;

// AoSoA-32: word w of arena a at (a / 32) * 32 * kArenaWords + w * 32 + a % 32
constexpr uint32_t kLanes = 32;
RSX_F size_t aosoa_block_words() { return (size_t)kArenaWords * kLanes; }
RSX_F size_t aosoa_words(uint32_t n) { return (size_t)((n + kLanes - 1) / kLanes) * aosoa_block_words(); }
RSX_F size_t aosoa_index(uint32_t a, int w) { return (size_t)(a / kLanes) * aosoa_block_words() + (size_t)w * kLanes + (a % kLanes); }

}  // namespace rsx
