// The game-logic phases and the integration phases of the tick:
//   P0  clear accumulators, limit velocities, UE3 quantisation     (reference: cuda/sim/arena_base.cuh:21-41, quantize.cuh)
//   P2  gravity, damping, predicted transforms                      (discrete_dynamics_world.cuh:45, rigid_body.cuh:52-70)
//   P6  integrate, activation                                       (discrete_dynamics_world.cuh:51)
//   P7  events, ball hits, bumps and demos in record order          (arena_base.cuh:43-208, ball_base.cuh)
//   P8  car post-tick, pad pickups, ball finish, tick count         (arena_base.cuh:210-222, car_base.cuh, boost_pad_grid.cuh)
// and the piecewise-linear curves of RocketSim (linear_piece_curve.cuh).
#pragma once
#include "base.cuh"

namespace rsx {
namespace sim {

// ---- piecewise-linear curves: (x, y) control points, the pieces' slopes recomputed per lookup ----
RSX_F float curve(const float (*p)[2], int n, float in) {
  if (n == 1) return p[0][1];
  if (in <= p[0][0]) return p[0][1];
  int i = 1;
  while (i < n && !(p[i][0] > in)) ++i;
  if (i == n) return p[n - 1][1];
  float dx = fsub(p[i][0], p[i - 1][0]), dy = fsub(p[i][1], p[i - 1][1]);
  return fadd(fmul(dy, fdiv(fsub(in, p[i - 1][0]), dx)), p[i - 1][1]);
}
RSX_F float c_ball_extra(float x) {
  const float p[5][2] = {{0.f, 0.65f}, {500.f, 0.65f}, {1400.f, 0.60f}, {2300.f, 0.55f}, {4600.f, 0.30f}};
  return curve(p, 5, x);
}
RSX_F float c_bump_ground(float x) {
  const float p[3][2] = {{0.f, fdiv(150.0f, 180.0f)}, {1400.f, fdiv(200000.0f, 180.0f)}, {2200.f, fdiv(275000.0f, 180.0f)}};
  return curve(p, 3, x);
}
RSX_F float c_bump_air(float x) {
  const float p[3][2] = {{0.f, fdiv(150.0f, 180.0f)}, {1400.f, fdiv(250000.0f, 180.0f)}, {2200.f, fdiv(350000.0f, 180.0f)}};
  return curve(p, 3, x);
}
RSX_F float c_bump_up(float x) {
  const float p[3][2] = {{0.f, fdiv(50.0f, 180.0f)}, {1400.f, fdiv(50000.0f, 180.0f)}, {2200.f, fdiv(75000.0f, 180.0f)}};
  return curve(p, 3, x);
}
RSX_F float c_steer(float x) {
  const float p[6][2] = {{0.f, 0.53356f}, {500.f, 0.31930f}, {1000.f, 0.18203f}, {1500.f, 0.10570f}, {1750.f, 0.08507f}, {3000.f, 0.03454f}};
  return curve(p, 6, x);
}
RSX_F float c_steer3(float x) {
  const float p[2][2] = {{0.f, 0.342473f}, {2300.f, 0.034837f}};
  return curve(p, 2, x);
}
RSX_F float c_slide_steer(float x) {
  const float p[2][2] = {{0.f, 0.39235f}, {2500.f, 0.12610f}};
  return curve(p, 2, x);
}
RSX_F float c_drive_torque(float x) {
  const float p[3][2] = {{0.f, 1.0f}, {1400.f, 0.1f}, {1410.f, 0.0f}};
  return curve(p, 3, x);
}
RSX_F float c_nonsticky(float x) {
  const float p[3][2] = {{0.f, 0.1f}, {0.7075f, 0.5f}, {1.0f, 1.0f}};
  return curve(p, 3, x);
}
RSX_F float c_lat(float x) {
  const float p[2][2] = {{0.f, 1.0f}, {1.0f, 0.2f}};
  return curve(p, 2, x);
}
RSX_F float c_lat3(float x) {
  const float p[2][2] = {{0.f, 0.30f}, {1.0f, 0.25f}};
  return curve(p, 2, x);
}
RSX_F float c_hb_lat(float) { return 0.1f; }
RSX_F float c_hb_long(float x) {
  const float p[2][2] = {{0.f, 0.5f}, {1.0f, 0.9f}};
  return curve(p, 2, x);
}

// ---- UE3 quantisation (shared/quantize.rs as the reference restates it, quantize.cuh) ----
RSX_F float sse_floor(float v) {  // glam's SSE floor: |v| < 2^23 via truncation
  if ((int32_t)(bits(v) & 0x7FFFFFFFu) < (int32_t)0x4B000000) {
    float t = i2f(f2i(v));
    return fadd(t, t > v ? -1.0f : 0.0f);
  }
  return v;
}
RSX_F V3 sign3(V3 v) {  // signum with zero lanes zero
  V3 s = vsignum(v);
  return {v.x == 0.0f ? 0.0f : s.x, v.y == 0.0f ? 0.0f : s.y, v.z == 0.0f ? 0.0f : s.z};
}
RSX_F V3 quant_pos(V3 v, float scale) {
  V3 w = v * scale + vs(0.5f);
  return V3{sse_floor(w.x), sse_floor(w.y), sse_floor(w.z)} / scale;
}
RSX_F V3 quant_vel(V3 v, float scale) {
  float inv = fdiv(1.0f, scale);
  V3 sc = v * scale;
  V3 r = {fmul(i2f(f2i(sc.x)), inv), fmul(i2f(f2i(sc.y)), inv), fmul(i2f(f2i(sc.z)), inv)};
  float off = fmul(0.1f, inv);
  return r + (sign3(r) * off);
}
RSX_F void quantize(Body& b) {
  V3 p = quant_pos(b.xf.t * kBTtoUU, 100.0f) * kUUtoBT;
  V3 v = quant_vel(b.lin_vel * kBTtoUU, 100.0f) * kUUtoBT;
  V3 w = quant_vel(b.ang_vel, 10000.0f);
  b.xf.t = p;
  b.lin_vel = v;
  b.ang_vel = w;
}
RSX_F float round_even(float v) {  // glam m128_round_ties_even, one lane
  uint32_t sg = bits(v) & 0x80000000u;
  float magic = from_bits(bits(8388608.0f) | sg);
  float r1 = fsub(fadd(v, magic), magic);
  bool small = from_bits(bits(v) & 0x7FFFFFFFu) <= 8388608.0f;
  return from_bits((small ? bits(r1) : 0u) ^ (small ? 0u : bits(v)));
}
RSX_F float round_away(float v) {  // f32::round through glam's m128_round
  float r = round_even(v);
  uint32_t sg = bits(v) & 0x80000000u;
  bool tie_down = fsub(v, r) == from_bits(bits(0.5f) | sg);
  return fadd(r, tie_down ? from_bits(bits(1.0f) | sg) : 0.0f);
}
// the 8-bit input quantisation of the controls (shared/quantize.rs:67, :87)
RSX_F V3 quant_axes(V3 c) {
  V3 cl = vclamp(c, vs(-1.0f), vs(1.0f));
  V3 sc = {cl.x < 0.0f ? 128.0f : 127.0f, cl.y < 0.0f ? 128.0f : 127.0f, cl.z < 0.0f ? 128.0f : 127.0f};
  V3 b = cl * sc + vs(128.0f);
  V3 w = b + b + vs(0.5f);
  int32_t ix = (f2i(round_away(w.x)) >> 1) & 0xFF, iy = (f2i(round_away(w.y)) >> 1) & 0xFF, iz = (f2i(round_away(w.z)) >> 1) & 0xFF;
  V3 s = V3{i2f(ix), i2f(iy), i2f(iz)} - vs(128.0f);
  float inv = fdiv(1.0f, 128.0f);
  return {s.x < 0.0f ? fmul(s.x, inv) : fdiv(s.x, 127.0f), s.y < 0.0f ? fmul(s.y, inv) : fdiv(s.y, 127.0f),
          s.z < 0.0f ? fmul(s.z, inv) : fdiv(s.z, 127.0f)};
}
RSX_F float quant_axis(float x) {
  float c = rclamp(x, -1.0f, 1.0f);
  float y = c < 0.0f ? rmax(fmul(c, 128.0f), -128.0f) : rmin(fmul(c, 127.0f), 127.0f);
  float w = fadd(fadd(fadd(y, 128.0f), fadd(y, 128.0f)), 0.5f);
  uint32_t byte = (uint32_t)((f2i(round_even(w)) >> 1) & 0xFF);
  float s = fsub(u2f(byte), 128.0f);
  return byte < 0x80u ? fmul(s, fdiv(1.0f, 128.0f)) : fdiv(s, 127.0f);
}

// ---- P0 ----
RSX_F void phase0(ArenaState& S, const StaticData& D) {
  S.events = 0;
  for (int d = 0; d < kDyn; ++d) clear_accum(S.bodies[d]);
  for (int ci = 0; ci < kCars; ++ci) {
    Body& b = S.bodies[1 + ci];
    limit_vels(b, fmul(kCarMaxSpeed, kUUtoBT), kCarMaxAngSpeed);
    quantize(b);
    S.cars[ci].vel = b.lin_vel * kBTtoUU;
    S.cars[ci].ang_vel = b.ang_vel;
  }
  Body& ball = S.bodies[0];
  limit_vels(ball, fmul(D.mut[M_BALL_MAX_SPEED], kUUtoBT), kBallMaxAngSpeed);
  quantize(ball);
  S.ball.vel = ball.lin_vel * kBTtoUU;
  S.ball.ang_vel = ball.ang_vel;
}

// ---- P2 / P6 ----
RSX_F Aff predict(const Body& b, float dt) {
  Aff t = b.xf;
  Q4 q = b.quat;
  if (b.flags & CF_NO_ANGULAR) t.t = t.t + b.lin_vel * dt;
  else integrate(t, q, b.lin_vel, b.ang_vel, dt);
  return t;
}
RSX_F void phase2(ArenaState& S, const StaticData& D) {
  const float dt = kTickTime;
  V3 g = D.gravity_bt * dt;
  for (int d = 0; d < kDyn; ++d)
    if (awake(S.bodies[d])) add_linear_accum(S.bodies[d], g);
  for (int d = 0; d < kDyn; ++d) {
    Body& b = S.bodies[d];
    if (b.activation == ACT_SLEEPING) {
      b.pred = b.xf;
      continue;
    }
    const BodyConst& c = D.bodies[D.dyn_body[d]];
    if (c.lin_damping != 0.0f) {
      if (b.damp_cache_dt != dt || b.damp_cache_value != c.lin_damping) {
        b.damp_cache = cr_pow(fsub(1.0f, c.lin_damping), dt);
        b.damp_cache_dt = dt;
        b.damp_cache_value = c.lin_damping;
      }
      b.lin_vel *= b.damp_cache;
    }
    b.pred = predict(b, dt);
  }
}
RSX_F void phase6(ArenaState& S, const StaticData& D) {
  const float dt = kTickTime;
  for (int d = 0; d < kDyn; ++d) {
    Body& b = S.bodies[d];
    if (!awake(b)) continue;
    Aff p = predict(b, dt);
    b.pred = p;
    set_world_xf(b, p);
    update_inertia(b, D.bodies[D.dyn_body[d]]);
  }
  for (int d = 0; d < kDyn; ++d) {
    Body& b = S.bodies[d];
    const BodyConst& c = D.bodies[D.dyn_body[d]];
    if ((b.flags & CF_CAN_SLEEP) == 0) {
      set_activation(b, ACT_ACTIVE);
      continue;
    }
    if (b.activation == ACT_SLEEPING) continue;
    float lt = fmul(c.lin_sleep, c.lin_sleep), at = fmul(c.ang_sleep, c.ang_sleep);
    if (len2(b.lin_vel) < lt && len2(b.ang_vel) < at) {
      b.deactivation_time = fadd(b.deactivation_time, dt);
      if (b.deactivation_time > 2.0f && b.activation == ACT_ACTIVE) set_activation(b, ACT_WANTS_SLEEP);
    } else {
      b.deactivation_time = 0.0f;
      set_activation(b, ACT_ACTIVE);
    }
  }
}

// ---- P7: contact callbacks ----
RSX_F bool in_rect_cone(V3 fwd, V3 right, V3 up, V3 delta, bool reverse, float yaw_deg, float pitch_deg) {
  V3 f0 = reverse ? -fwd : fwd;
  V3 d;
  if (!try_normalize(delta, &d)) return false;
  float f = dot(d, f0);
  if (f <= 0.0f) return false;
  const float rpd = fdiv(kPi, 180.0f);
  return fabs_(dot(d, right)) <= fmul(f, cr_tan(fmul(yaw_deg, rpd))) && fabs_(dot(d, up)) <= fmul(f, cr_tan(fmul(pitch_deg, rpd)));
}

RSX_HD RSX_NOINL inline void ball_hit(ArenaState& S, const StaticData& D, int ci) {
  Car& car = S.cars[ci];
  Body& rb = S.bodies[0];
  V3 fwd = car.rot.c0;
  V3 rel_pos = S.ball.pos - car.pos, rel_vel = S.ball.vel - car.vel;
  float rel_speed = rmin(len(rel_vel), kHitMaxDeltaVel);
  bool can = !car.last_extra_hit_tick.some || (u64_of(car.last_extra_hit_tick.v) + 1 < u64_of(S.tick_count));
  if (rel_speed > 0.0f && can) {
    V3 dir = normalize_or_zero(rel_pos * V3{1.0f, 1.0f, kHitZScale});
    V3 adj = (fwd * dot(dir, fwd)) * fsub(1.0f, kHitForwardScale);
    dir = normalize_or_zero(dir - adj);
    V3 imp = ((dir * rel_speed) * c_ball_extra(rel_speed)) * D.mut[M_HIT_EXTRA_SCALE];
    add_linear(rb, imp * kUUtoBT);
    car.last_extra_hit_tick.some = 1;
    car.last_extra_hit_tick.v = S.tick_count;
  }
}

RSX_HD RSX_NOINL inline void car_car_hit(ArenaState& S, const StaticData& D, int c1, int c2, const RecPoint& mp) {
  int att = c1, vic = c2;
  if (S.cars[vic].is_demoed || S.cars[att].is_demoed) return;
  for (int sw = 0; sw < 2; ++sw) {
    if (sw) {
      int t = att;
      att = vic;
      vic = t;
    }
    Car& A = S.cars[att];
    Car& V = S.cars[vic];
    if (A.bump_cooldown > 0.0f && (!A.bump_victim.some || A.bump_victim.v == (uint32_t)vic)) continue;
    V3 dp = V.pos - A.pos;
    if (dot(A.vel, dp) < 0.0f) continue;
    V3 vdir = normalize_or_zero(A.vel);
    V3 to_v = normalize_or_zero(dp);
    if (dot(A.vel, to_v) <= dot(V.vel, vdir)) continue;
    V3 af = A.rot.c0, ar = A.rot.c1, au = A.rot.c2;
    bool center_in = in_rect_cone(af, ar, au, dp, false, kBumpYawDeg, kBumpPitchDeg);
    V3 on_att = sw ? mp.world_b : mp.world_a;
    V3 on_vic = sw ? mp.world_a : mp.world_b;
    V3 gate = (V.pos - on_vic * kBTtoUU) - (A.pos - on_att * kBTtoUU);
    bool resid_in = in_rect_cone(af, ar, au, gate, false, kBumpYawDeg, kBumpPitchDeg);
    if (!center_in && !resid_in) continue;
    bool demo;
    if (D.demo_mode == 1) demo = true;
    else if (D.demo_mode == 2) demo = false;
    else {
      demo = false;
      if (A.is_supersonic) {
        float fs = dot(A.vel, af);
        demo = fabs_(fs) >= kSupersonicMaintainMin && in_rect_cone(af, ar, au, dp, fs < 0.0f, kDemoYawDeg, kDemoPitchDeg);
      }
    }
    if (demo && !D.team_demos) demo = D.cars[att].team != D.cars[vic].team;
    if (demo) {
      V.is_demoed = 1;
      V.demo_respawn_timer = D.mut[M_RESPAWN_DELAY];
    } else {
      float sp = rmin(len(A.vel), kBumpAttackerSpeedMax);
      if (V.on_ground != 0) {
        float base = c_bump_ground(sp);
        V3 up = V.rot.c2;
        float upf = fmul(c_bump_up(sp), D.mut[M_BUMP_FORCE_SCALE]);
        V3 imp = (vdir * base) + (up * upf);
        V.vel_impulse_cache += imp * kUUtoBT;
      } else {
        V3 imp = vdir * c_bump_air(sp);
        V.vel_impulse_cache += imp * kUUtoBT;
      }
    }
    A.bump_cooldown = D.mut[M_BUMP_COOLDOWN];
    A.bump_victim.some = 1;
    A.bump_victim.v = (uint32_t)vic;
    S.events |= 1u << ((demo ? EV_DEMO : EV_BUMP) + vic);
  }
}

RSX_F void phase7(ArenaState& S, const StaticData& D) {
  S.events |= S.fold_events;
  for (int ci = 0; ci < kCars; ++ci)
    if (S.fold_events & (1u << (EV_CAR_HIT_WORLD + ci))) {
      S.cars[ci].world_contact_normal.some = 1;
      S.cars[ci].world_contact_normal.v = S.fold_car_normal[ci];
    }
  S.fold_events = 0;
  S.fold_car_normal[0] = vzero();
  S.fold_car_normal[1] = vzero();
  uint32_t n = S.n_records;
  for (uint32_t i = 0; i < n; ++i) {
    Record r = S.records[i];
    const BodyConst& a = D.bodies[r.body_a];
    const BodyConst& b = D.bodies[r.body_b];
    if (b.user == USER_BALL) {
      ball_hit(S, D, (int)a.user_ptr);
      S.events |= 1u << (EV_CAR_HIT_BALL + (int)a.user_ptr);
    } else {
      car_car_hit(S, D, (int)a.user_ptr, (int)b.user_ptr, r.p);
    }
  }
  for (uint32_t i = 0; i < S.n_records; ++i) S.records[i] = Record{};
  S.n_records = 0;
}

// ---- P8 ----
RSX_F void car_post_tick(Car& c, const Body& rb) {
  const float start2 = fmul(kSupersonicStart, kSupersonicStart);
  const float keep2 = fmul(kSupersonicMaintainMin, kSupersonicMaintainMin);
  if (c.is_demoed) return;
  c.rot = rb.xf.m;
  float sp2 = len2(rb.lin_vel * kBTtoUU);
  if (c.is_supersonic) {
    if (sp2 >= start2) {
      c.supersonic_grace = 0.0f;
    } else if (sp2 < keep2) {
      c.is_supersonic = 0;
      c.supersonic_grace = 0.0f;
    } else {
      c.supersonic_grace = fadd(c.supersonic_grace, kTickTime);
      if (c.supersonic_grace >= kSupersonicMaintainTime) {
        c.is_supersonic = 0;
        c.supersonic_grace = 0.0f;
      }
    }
  } else if (sp2 >= start2) {
    c.is_supersonic = 1;
    c.supersonic_grace = 0.0f;
  } else {
    c.supersonic_grace = 0.0f;
  }
  if (c.has_jumped && !c.is_jumping && c.on_ground && c.air_time > 0.0f) {
    int contacts = 0;
    bool extending = true;
    for (int w = 0; w < kWheels; ++w) {
      if (!c.wheels[w].ray.some) continue;
      contacts += 1;
      if (!(c.wheels[w].ray.v.susp_rel_vel > 1.0f)) {
        extending = false;
        break;
      }
    }
    if (!(contacts != 0 && extending)) c.has_jumped = 0;
  } else if (c.has_jumped && !c.is_jumping && c.on_ground && c.jump_ticks > kJumpRearmTicks) {
    c.has_jumped = 0;
  }
  c.bump_cooldown = rmax(fsub(c.bump_cooldown, kTickTime), 0.0f);
  c.prev_controls = c.controls;
}
RSX_F void car_finish(Car& c, Body& rb) {
  if (c.is_demoed) return;
  V3 v = c.vel_impulse_cache;
  if (!(v.x == 0.0f && v.y == 0.0f && v.z == 0.0f)) {
    rb.lin_vel += c.vel_impulse_cache;
    c.vel_impulse_cache = vzero();
  }
  c.pos = rb.xf.t * kBTtoUU;
  c.vel = rb.lin_vel * kBTtoUU;
  c.ang_vel = rb.ang_vel;
}

// boost pads: membership in arrival order, pickup by the first member that can take boost
RSX_F bool pad_cyl(V3 pp, float r, V3 pos) {
  float dx = fsub(pp.x, pos.x), dy = fsub(pp.y, pos.y);
  return fadd(fmul(dx, dx), fmul(dy, dy)) < powi2(r) && fabs_(fsub(pos.z, pp.z)) <= kCylHeight;
}
RSX_F bool pad_can_take(const Car& c, float mx) { return !c.is_demoed && !(c.boost >= mx); }
RSX_F bool pad_box(V3 pp, float br, const Car& car, const CarConst& cc) {
  const M3 R = car.rot;
  const V3 center = car.pos + R * cc.hitbox_offset;
  const V3 ca[3] = {R.c0, R.c1, R.c2};
  const V3 ch = cc.hitbox_size * 0.5f;
  const V3 ph = {br, br, 64.0f};
  const V3 delta = center - pp;
  const V3 wa[3] = {{1.0f, 0.0f, 0.0f}, {0.0f, 1.0f, 0.0f}, {0.0f, 0.0f, 1.0f}};
  for (int k = 0; k < 15; ++k) {
    const V3 ax = k < 3 ? wa[k] : (k < 6 ? ca[k - 3] : cross(ca[(k - 6) / 3], wa[(k - 6) % 3]));
    if (len2(ax) <= kEps) continue;
    float pr = dot(ph, V3{fabs_(dot(wa[0], ax)), fabs_(dot(wa[1], ax)), fabs_(dot(wa[2], ax))});
    float cr = dot(ch, V3{fabs_(dot(ca[0], ax)), fabs_(dot(ca[1], ax)), fabs_(dot(ca[2], ax))});
    if (fabs_(dot(delta, ax)) > fadd(pr, cr)) return false;
  }
  return true;
}
RSX_F int pad_winner(const ArenaState& S, int p, float mx) {
  const PadTouch& t = S.pad_touch[p];
  for (uint32_t k = 0; k < t.n; ++k)
    if (pad_can_take(S.cars[t.car[k]], mx)) return (int)t.car[k];
  return -1;
}
RSX_HD RSX_NOINL inline void pads_tick(ArenaState& S, const StaticData& D) {
  const float mx = D.mut[M_MAX_BOOST];
  int touching[kCars] = {-1, -1};
  // the pads whose touching list is not empty (the loop below leaves an empty list as it is), read as independent loads
  static_assert(kPads <= 64, "one bit per pad");
  uint64_t listed_pads = 0;
#pragma unroll
  for (int i = 0; i < kPads; ++i) listed_pads |= (uint64_t)(S.pad_touch[i].n != 0) << i;
  for (; listed_pads != 0; listed_pads &= listed_pads - 1) {
    const int i = ctz64(listed_pads);
    const PadConst& pad = D.pads[i];
    PadTouch& t = S.pad_touch[i];
    uint32_t kept = 0;
    for (uint32_t k = 0; k < t.n; ++k) {
      uint32_t ci = t.car[k];
      const Car& car = S.cars[ci];
      if (!car.is_demoed && touching[ci] < 0 &&
          (pad_cyl(pad.pos, pad.cyl_radius, car.pos) || pad_box(pad.pos, pad.box_radius, car, D.cars[ci]))) {
        touching[ci] = i;
        t.car[kept++] = ci;
      }
    }
    if (kept != t.n) {  // (an unchanged list is left as it is: the same words, no stores)
      for (uint32_t k = kept; k < t.n; ++k) t.car[k] = 0;
      t.n = kept;
    }
  }
  for (int ci = 0; ci < kCars; ++ci) {
    const Car& car = S.cars[ci];
    if (car.is_demoed || car.pos.z > D.max_pad_z || touching[ci] >= 0) continue;
    for (int i = 0; i < kPads; ++i) {
      const PadConst& pad = D.pads[i];
      if (!(all_le(pad.box.lo, car.pos) && all_ge(pad.box.hi, car.pos))) continue;
      if (!pad_cyl(pad.pos, pad.cyl_radius, car.pos)) continue;
      PadTouch& t = S.pad_touch[i];
      bool listed = false;
      for (uint32_t k = 0; k < t.n; ++k) listed |= t.car[k] == (uint32_t)ci;
      if (!listed) {
        if (t.n < (uint32_t)kCars) t.car[t.n++] = (uint32_t)ci;
        else ++S.overflow[OVF_PAD_TOUCHING];
      }
      touching[ci] = i;
      break;
    }
  }
  // Each pad's winner is the first car of its list that can take boost.  A car is listed at one pad at most (its
  // `touching` pad), so a pickup changes only that pad's winner: evaluating the winner of a car's own pad when the car
  // is reached gives what a table made before the loop and refreshed after each pickup would hold.
  for (int ci = 0; ci < kCars; ++ci) {
    Car& car = S.cars[ci];
    if (car.is_demoed || car.boost >= mx) continue;
    int i = touching[ci];
    if (i < 0 || pad_winner(S, i, mx) != ci) continue;
    const PadConst& pad = D.pads[i];
    int64_t tick = (int64_t)u64_of(S.tick_count);
    if (S.pad_gave[i].some) {
      int64_t last = (int64_t)u64_of(S.pad_gave[i].v);
      if (fmul(ll2f(tick - last), kTickTime) < pad.cooldown) continue;
    }
    car.boost = rmin(fadd(car.boost, pad.amount), mx);
    S.pad_gave[i].some = 1;
    S.pad_gave[i].v = u64w((uint64_t)tick);
    S.events |= 1u << (EV_PICKUP + ci);
  }
}

// P8 in two steps a kernel can barrier between (the cars, then pads, ball and tick count); phase8 runs both.
RSX_F void phase8_cars(ArenaState& S) {
  for (int ci = 0; ci < kCars; ++ci) {
    car_post_tick(S.cars[ci], S.bodies[1 + ci]);
    car_finish(S.cars[ci], S.bodies[1 + ci]);
  }
}
RSX_F void phase8_rest(ArenaState& S, const StaticData& D) {
  if (D.pads_enabled) pads_tick(S, D);
  const Body& rb = S.bodies[0];
  S.ball.vel = rb.lin_vel * kBTtoUU;
  S.ball.ang_vel = rb.ang_vel;
  S.ball.pos = rb.xf.t * kBTtoUU;
  S.ball.rot = rb.xf.m;
  S.ball.ticks_since_kickoff = u64w(u64_of(S.ball.ticks_since_kickoff) + 1);
  S.tick_count = u64w(u64_of(S.tick_count) + 1);
}
RSX_F void phase8(ArenaState& S, const StaticData& D) {
  phase8_cars(S);
  phase8_rest(S, D);
}

}  // namespace sim
}  // namespace rsx
