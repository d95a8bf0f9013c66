// Shared pieces of the tick: constants, body access (a world body index 0..22 is a mesh, a plane, the ball or a car;
// the three dynamic ones live in ArenaState.bodies, the rest in StaticData), and the rigid-body operations.
// Bullet / RocketSim V3 semantics as the reference states them: cuda/sim/consts.cuh, bullet_consts.cuh,
// rigid_body.cuh, rigid_body_p1.cuh, narrowphase.cuh:23-114.  Constant expressions are written as the reference writes
// them, so that the compiler folds them to the same binary32 values.
#pragma once
#include "../state.cuh"
#include "../crmath.cuh"

// Zone timers of profiling builds (RSX_ZONES defined, device code): the lowest active lane of each group of lanes that
// runs a zone adds the zone's clock cycles to its warp's slot rsx_zone_acc[warp][id], so the sums are warp cycles spent in each
// zone.  The including translation unit defines rsx_zone_acc.  Without RSX_ZONES the markers are empty.
#if defined(RSX_ZONES) && defined(__CUDA_ARCH__)
#ifndef RSX_ZONES_MIN
#define RSX_ZONES_MIN 0
#endif
extern __device__ unsigned long long rsx_zone_acc[148 * 16][64];
#define RSX_ZONE_BEGIN(v) long long v = clock64()
#define RSX_ZONE_END(v, id)                                                                              \
  do {                                                                                                   \
    unsigned m_ = __activemask();                                                                        \
    if ((id) >= RSX_ZONES_MIN && (threadIdx.x & 31u) == (unsigned)(__ffs(m_) - 1))                      \
      atomicAdd(&rsx_zone_acc[(blockIdx.x * 16u + (threadIdx.x >> 5)) % (148u * 16u)][id],               \
                (unsigned long long)(clock64() - v));                                                    \
  } while (0)
#elif defined(RSX_HOST_ZONE_COUNTS) && !defined(__CUDA_ARCH__)
// Host profiling builds (RSX_HOST_ZONE_COUNTS defined): each marker's end counts one run of its zone in
// rsx_zone_count[id] of the calling thread, which the including translation unit defines; how often each piece of
// work runs per arena and tick, for the work-distribution statistics of the decision kernels.
extern thread_local unsigned long long rsx_zone_count[64];
#define RSX_ZONE_BEGIN(v) \
  do {                    \
  } while (0)
#define RSX_ZONE_END(v, id) (rsx_zone_count[id] += 1)
#else
#define RSX_ZONE_BEGIN(v) \
  do {                    \
  } while (0)
#define RSX_ZONE_END(v, id) \
  do {                      \
  } while (0)
#endif

namespace rsx {
namespace sim {

// ---- constants (cuda/sim/consts.cuh) ----
constexpr float kBTtoUU = 50.0f;
constexpr float kUUtoBT = 1.0f / 50.0f;
constexpr float kTickTime = 1.0f / 120.0f;
constexpr float kCarMaxSpeed = 2300.0f;
constexpr float kCarMaxAngSpeed = 5.5f;
constexpr float kSupersonicStart = 2200.0f;
constexpr float kSupersonicMaintainMin = 2200.0f - 100.0f;
constexpr float kSupersonicMaintainTime = 1.0f;
constexpr float kDemoYawDeg = 45.572994f, kDemoPitchDeg = 36.869896f;
constexpr uint32_t kJumpRearmTicks = 15;
constexpr float kBumpYawDeg = 70.0f, kBumpPitchDeg = 36.869896f;
constexpr float kBallMaxAngSpeed = 6.0f;
constexpr float kHitForwardScale = 0.65f, kHitMaxDeltaVel = 4600.0f, kHitZScale = 0.35f;
constexpr float kBumpAttackerSpeedMax = 2200.0f;
constexpr float kCylHeight = 95.0f;
constexpr float kPi = 3.14159265358979323846264338327950288f;
constexpr float kEps = 1.1920928955078125e-7f;
constexpr float kFltMax = 3.40282347e+38f;
constexpr float kTau = 6.28318530717958647692f;
constexpr float kBoostMax = 100.0f, kBoostMinTime = 0.1f;
constexpr float kThrottleTorque = 180.0f * 400.0f;
constexpr float kBrakeTorque = 180.0f * (14.25f + (1.0f / 3.0f));
constexpr float kStoppingFwdVel = 25.0f, kCoastBrake = 0.15f, kBrakeNoThrottleThresh = 0.01f, kThrottleDeadzone = 0.01f;
constexpr float kThrottleAirAccel = 200.0f / 3.0f;
constexpr float kPowerslideRise = 5.0f, kPowerslideFall = 2.0f;
constexpr uint32_t kJumpMinTicks = 3, kJumpMaxTicks = 24;
constexpr float kDoubleJumpMaxDelay = 1.25f;
constexpr float kFlipZDamp120 = 0.35f, kFlipZDampStart = 0.15f, kFlipZDampEnd = 0.21f, kFlipTorqueTime = 0.65f;
constexpr float kFlipPitchCancelMin = 0.041f, kFlipPitchLockExtra = 0.3f, kFlipInitVel = 500.0f;
constexpr float kFlipTorqueX = 260.0f, kFlipTorqueY = 224.0f, kFlipTorqueZ = 0.0f;
constexpr float kFlipFwdScale = 1.0f, kFlipSideScale = 1.9f, kFlipBackScale = 2.5f, kFlipBackScaleX = 16.0f / 15.0f;
constexpr float kAirTorqueX = 130.0f, kAirTorqueY = 95.0f, kAirTorqueZ = 400.0f;
constexpr float kAirDampX = 30.0f, kAirDampY = 20.0f, kAirDampZ = 50.0f;
constexpr float kAirTorqueScale = 2.0f * kPi / 65536.0f * 1000.0f;
constexpr float kAutoflipImpulse = 200.0f, kAutoflipAngVel = 1000.0f, kAutoflipTime = 0.4f;
constexpr float kAutoflipNormZ = 0.707106781186547524400844362104849039f, kAutoflipRollThresh = 2.8f;
constexpr float kAutorollForce = 100.0f, kAutorollTorque = 80.0f;
constexpr float kRespawnZ = 36.0f;
constexpr float kSuspStiffness = 500.0f, kDampCompression = 25.0f, kDampRelaxation = 40.0f;
constexpr float kMaxSuspTravel = 12.0f, kSuspSubtract = 0.05f, kPushbackErp = 0.1f;
constexpr float kBreakingThreshold = 0.02f;  // CONTACT_BREAKING_THRESHOLD

// collision flags (rigid_body.rs:51-58)
constexpr uint32_t CF_STATIC = 1u, CF_CUSTOM = 2u, CF_CAN_SLEEP = 4u, CF_NO_RESPONSE = 8u, CF_NO_ANGULAR = 32u;
enum : uint32_t { ACT_ACTIVE = 0, ACT_SLEEPING = 1, ACT_DISABLED = 2, ACT_WANTS_SLEEP = 3 };
enum : uint32_t { USER_NONE = 0, USER_CAR = 1, USER_BALL = 2 };
enum : uint32_t { SHAPE_MESH = 0, SHAPE_PLANE = 1, SHAPE_SPHERE = 2, SHAPE_BOX = 3 };
constexpr uint32_t kNoBody = 0xFFFFFFFFu;

// ---- body access ----
// dynamic slot of world body w (0 ball, 1 car 0, 2 car 1), or -1 for a static body
RSX_F int slot(const StaticData& D, uint32_t w) {
  for (int d = 0; d < kDyn; ++d)
    if (D.dyn_body[d] == w) return d;
  return -1;
}
RSX_F Aff body_xf(const ArenaState& S, const StaticData& D, uint32_t w) {
  int d = slot(D, w);
  return d >= 0 ? S.bodies[d].xf : D.bodies[w].pose;
}
RSX_F uint32_t body_flags(const ArenaState& S, const StaticData& D, uint32_t w) {
  int d = slot(D, w);
  return d >= 0 ? S.bodies[d].flags : CF_STATIC;
}
RSX_F bool body_static(const ArenaState& S, const StaticData& D, uint32_t w) { return (body_flags(S, D, w) & CF_STATIC) != 0; }
RSX_F bool body_responds(const ArenaState& S, const StaticData& D, uint32_t w) { return (body_flags(S, D, w) & CF_NO_RESPONSE) == 0; }
RSX_F bool body_awake(const ArenaState& S, const StaticData& D, uint32_t w) {
  int d = slot(D, w);
  return d >= 0 && S.bodies[d].activation != ACT_SLEEPING && S.bodies[d].activation != ACT_DISABLED;
}
RSX_F bool awake(const Body& b) { return !(b.activation == ACT_SLEEPING || b.activation == ACT_DISABLED); }

// A snapshot of a body as the vehicle code reads it (a static body: its pose, no velocity, no inverse inertia).
struct View {
  Aff xf;
  V3 lin_vel, ang_vel;
  M3 inv_inertia;
  float inv_mass;
  uint32_t flags, user;
};
RSX_F View view(const ArenaState& S, const StaticData& D, uint32_t w) {
  View v;
  int d = slot(D, w);
  const BodyConst& c = D.bodies[w];
  v.user = c.user;
  v.inv_mass = c.inv_mass;
  if (d >= 0) {
    const Body& b = S.bodies[d];
    v.xf = b.xf;
    v.lin_vel = b.lin_vel;
    v.ang_vel = b.ang_vel;
    v.inv_inertia = b.inv_inertia_world;
    v.flags = b.flags;
  } else {
    v.xf = c.pose;
    v.lin_vel = vzero();
    v.ang_vel = vzero();
    v.inv_inertia = M3{vzero(), vzero(), vzero()};
    v.flags = CF_STATIC;
  }
  return v;
}
RSX_F V3 vel_at(const View& v, V3 rel) { return v.lin_vel + cross(v.ang_vel, rel); }
RSX_F float impulse_denom(const View& v, V3 pos, V3 n) {
  V3 r0 = pos - v.xf.t;
  V3 c0 = cross(r0, n);
  V3 vec = cross(mul_t(v.inv_inertia, c0), r0);
  return fadd(v.inv_mass, dot(n, vec));
}
RSX_F float mass_of(const BodyConst& c) { return c.inv_mass == 0.0f ? 0.0f : fdiv(1.0f, c.inv_mass); }

// ---- rigid-body operations (rigid_body.rs) ----
RSX_F void set_activation(Body& b, uint32_t st) {
  if (b.activation != ACT_DISABLED) b.activation = st;
}
RSX_F void set_world_xf(Body& b, const Aff& xf) {
  if ((b.flags & CF_NO_ANGULAR) == 0) b.quat = quat_from_m3(xf.m);
  b.xf = xf;
}
RSX_F M3 inertia_world(const M3& m, V3 inv_local) {
  M3 sc = transpose(m);
  sc.c0 *= inv_local;
  sc.c1 *= inv_local;
  sc.c2 *= inv_local;
  return m * sc;
}
RSX_F void update_inertia(Body& b, const BodyConst& c) { b.inv_inertia_world = inertia_world(b.xf.m, c.inv_inertia_local); }

enum Imp { IMP_LINEAR, IMP_LINEAR_AT, IMP_ANGULAR };
// add_impulse(kind, massed, accum): the zero parts are added too (their -0 + 0 matters)
RSX_F void add_impulse(Body& b, const BodyConst& c, Imp kind, V3 v, V3 rel, bool massed, bool accum) {
  V3 li = vzero(), ai = vzero();
  float ms = massed ? c.inv_mass : 1.0f;
  if (kind == IMP_LINEAR) {
    li = v * ms;
  } else if (kind == IMP_LINEAR_AT) {
    li = v * ms;
    ai = b.inv_inertia_world * cross(rel, v);
    if (!massed) ai *= c.mass;
  } else {
    ai = v * ms;
  }
  if (accum) {
    b.acc_lin += li;
    b.acc_ang += ai;
  } else {
    b.lin_vel += li;
    b.ang_vel += ai;
  }
}
RSX_F void add_linear_accum(Body& b, V3 v) {  // add_impulse(Linear, massed false, accum true)
  b.acc_lin += v * 1.0f;
  b.acc_ang += vzero();
}
RSX_F void add_linear(Body& b, V3 v) {  // add_impulse(Linear, massed false, accum false)
  b.lin_vel += v * 1.0f;
  b.ang_vel += vzero();
}
RSX_F void clear_accum(Body& b) {
  b.acc_lin = vzero();
  b.acc_ang = vzero();
}
RSX_F float powi2(float a) { return fmul(fmul(1.0f, a), a); }  // f32::powi(a, 2): binary exponentiation from 1
RSX_F void limit_vels(Body& b, float max_lin, float max_ang) {
  if (len2(b.lin_vel) > powi2(max_lin)) b.lin_vel = normalize_or_zero(b.lin_vel) * max_lin;
  if (len2(b.ang_vel) > powi2(max_ang)) b.ang_vel = normalize_or_zero(b.ang_vel) * max_ang;
}
RSX_F void force_activate(Body& b) {
  b.activation = ACT_ACTIVE;
  b.deactivation_time = 0.0f;
}

// ---- the quaternion integrator (transform_util.rs) ----
RSX_F float motion_threshold() { return from_bits(0x3F490FDBu); }  // FRAC_PI_4
RSX_HD RSX_NOINL inline void integrate(Aff& xf, Q4& rot, V3 lin_vel, V3 ang_vel, float dt) {
  xf.t = xf.t + lin_vel * dt;
  float angle = len(ang_vel);
  if (fmul(angle, dt) > motion_threshold()) angle = fdiv(motion_threshold(), dt);
  float half = fmul(fmul(angle, dt), 0.5f);
  float k, sh, ch;
  if (angle < 0.001f) {
    float t3 = fmul(fmul(dt, dt), dt);
    k = fsub(fmul(0.5f, dt), fmul(fmul(fmul(t3, 0.020833334f), angle), angle));
    ch = cr_cos(half);
  } else {
    cr_sincos(half, &sh, &ch);
    k = fdiv(sh, angle);
  }
  V3 ax = ang_vel * k;
  Q4 dorn = {ax.x, ax.y, ax.z, ch};
  rot = qnormalize(dorn * rot);
  xf.m = m3_from_quat(rot);
}

// ---- AABBs of the dynamic shapes ----
RSX_F V3 add_s(V3 a, float s) { return a + vs(s); }
RSX_F Box3 sphere_box(float radius, V3 c) {
  V3 e = vs(fadd(radius, 0.08f));
  return {c - e, c + e};
}
RSX_F Box3 compound_box(const BodyConst& c, const Aff& t) {
  V3 he = 0.5f * (c.compound_box.hi - c.compound_box.lo);
  V3 ctr = 0.5f * (c.compound_box.hi + c.compound_box.lo);
  M3 ab = mabs(t.m);
  V3 center = xform_point(t, ctr);
  V3 ext = ab * he;
  return {center - ext, center + ext};
}
RSX_F Box3 box_from_half(V3 half, float margin, const Aff& t) {
  V3 h = add_s(half, margin);
  M3 ab = mabs(t.m);
  V3 ext = ab * h;
  return {t.t - ext, t.t + ext};
}
// a body's own AABB at its current transform (collision_shape.rs:38)
RSX_F Box3 body_box(const ArenaState& S, const StaticData& D, uint32_t w) {
  const BodyConst& c = D.bodies[w];
  Aff t = body_xf(S, D, w);
  if (c.shape == SHAPE_SPHERE) return sphere_box(c.sphere_margin, t.t);
  if (c.shape == SHAPE_PLANE) return D.planes[w - kMeshes].box;
  if (c.shape == SHAPE_MESH) {
    const Box3& id = D.meshes[w].ident_box;
    return {id.lo + t.t, id.hi + t.t};
  }
  return compound_box(c, t);
}
RSX_F Aff child_xf(const ArenaState& S, const StaticData& D, uint32_t w) { return body_xf(S, D, w) * D.bodies[w].child; }
RSX_F Box3 child_box(const ArenaState& S, const StaticData& D, uint32_t w) {
  const BodyConst& c = D.bodies[w];
  return box_from_half(c.box_half, c.box_margin, child_xf(S, D, w));
}

// ---- ray grid cells (grid_broadphase.rs:51-76) ----
RSX_F void cell_indices(const StaticData& D, V3 p, uint32_t out[3]) {
  V3 f = (p - D.grid_lo) / D.cell_size;
  int32_t v[3] = {f2i(f.x), f2i(f.y), f2i(f.z)};
  for (int a = 0; a < 3; ++a) {
    int32_t m = v[a] > 0 ? v[a] : 0;
    uint32_t hi = D.grid_n[a] - 1;
    out[a] = (uint32_t)m < hi ? (uint32_t)m : hi;
  }
}
// the index of the lowest set bit of x (x != 0)
RSX_F int ctz64(uint64_t x) {
#ifdef __CUDA_ARCH__
  return __ffsll((long long)x) - 1;
#else
  return __builtin_ctzll(x);
#endif
}
RSX_F uint32_t cell_of(const StaticData& D, const uint32_t i[3]) { return i[0] * D.grid_n[1] * D.grid_n[2] + i[1] * D.grid_n[2] + i[2]; }
// The first entry of the ray grid's dynamic list at or after cell c.  The list is sorted by cell (broad.cuh dyn_cells_block inserts
// after every entry of a lower or equal cell and removes in place), so a cell's entries are one run from here, in list
// order: the entries a scan of the whole list for the cell meets, in the same order.
RSX_F uint32_t dyn_cells_first(const ArenaState& S, uint32_t c) {
  uint32_t lo = 0, hi = S.n_dyn_cells < (uint32_t)kMaxDynCells ? S.n_dyn_cells : (uint32_t)kMaxDynCells;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (S.dyn_cells[mid].cell < c)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

}  // namespace sim
}  // namespace rsx
