// P1: the car pre-tick and the raycast vehicle.  Reference: cuda/sim/car_pre_tick.cuh (jump, flips, auto-flip,
// air control, auto-roll, boost, demo respawn, contact state), vehicle_rl.cuh (the four wheel rays, per-wheel
// response, suspension then friction), wheel_info.cuh, contact_constraint.cuh, arena_base_p1.cuh (the phase driver).
// Operation order, branch order and tie rules are the reference's (V3's); the structure is this project's.
#pragma once
#include "game.cuh"
#include "ray.cuh"

namespace rsx {
namespace sim {

RSX_F uint32_t wheels_in_contact(const Car& c) {
  uint32_t n = 0;
  for (int i = 0; i < kWheels; ++i) n += c.wheel_contact[i].some ? 1u : 0u;
  return n;
}

// ---- the auto-flip roll sign: integer angle units rebuilt from the 14-bit sine table (car/base.rs:68-118) ----
RSX_F int32_t angle_units(float a0, float a1) {
  float ang = crm::atan2_via_double(a0, a1);
  float u = fdiv(fmul(ang, 32768.0f), kPi);
  float v = fadd(fmul(u, 2.0f), 0.5f);
  return f2i(round_even(v)) >> 1;
}
RSX_HD RSX_NOINL inline float autoflip_sign(const StaticData& D, const M3& r) {
  int32_t yaw = angle_units(r.c0.y, r.c0.x);
  float l = crm::hypot_via_double(r.c0.x, r.c0.y);
  int32_t pitch = angle_units(r.c0.z, l);
  float tp = D.table_sin[(uint32_t)((pitch >> 2) & 0x3FFF)];
  float ty = D.table_sin[(uint32_t)((yaw >> 2) & 0x3FFF)];
  float tr = D.table_sin[0];
  float tpq = D.table_sin[(uint32_t)(((pitch + 0x4000) >> 2) & 0x3FFF)];
  float tyq = D.table_sin[(uint32_t)(((yaw + 0x4000) >> 2) & 0x3FFF)];
  float trq = D.table_sin[0x1000];
  V3 r1 = {fsub(fmul(fmul(tp, tr), tyq), fmul(trq, ty)), fadd(fmul(tyq, trq), fmul(fmul(tp, tr), ty)), fmul(fneg(tr), tpq)};
  int32_t roll = angle_units(dot(r.c2, r1), dot(r.c1, r1));
  return (int16_t)roll > 0 ? 1.0f : -1.0f;
}

// ---- fastrand's WyRand (respawn spot) ----
RSX_F uint64_t mulhi64(uint64_t a, uint64_t b) {
  uint64_t h, l;
  crm::mul64(a, b, &h, &l);
  return h;
}
RSX_F uint64_t wy_next(U64W* st) {
  uint64_t s = u64_of(*st) + 0x2d358dccaa6c78a5ull;
  *st = u64w(s);
  uint64_t o = s ^ 0x8bb84b93962eacc9ull;
  return (s * o) ^ mulhi64(s, o);
}
RSX_F uint64_t wy_mod(U64W* st, uint64_t n) {
  uint64_t r = wy_next(st);
  uint64_t hi = mulhi64(r, n), lo = r * n;
  if (lo < n) {
    uint64_t t = (0ull - n) % n;
    while (lo < t) {
      r = wy_next(st);
      hi = mulhi64(r, n);
      lo = r * n;
    }
  }
  return hi;
}

// Mat3A::from_euler(ZYX, yaw, 0, 0) in glam's order
RSX_F M3 yaw_matrix(float yaw) {
  float si, ci, sj, cj, sh, ch;
  cr_sincos(yaw, &si, &ci);
  cr_sincos(0.0f, &sj, &cj);
  cr_sincos(0.0f, &sh, &ch);
  float cc = fmul(ci, ch), cs = fmul(ci, sh), sc = fmul(si, ch), ss = fmul(si, sh);
  return M3{V3{fmul(cj, ci), fmul(cj, si), fneg(sj)}, V3{fsub(fmul(sj, cs), sc), fadd(fmul(sj, ss), cc), fmul(cj, sh)},
            V3{fadd(fmul(sj, cc), ss), fsub(fmul(sj, sc), cs), fmul(cj, ch)}};
}

RSX_F void sync_car_body(Car& car, Body& rb, const BodyConst& bc) {
  set_world_xf(rb, Aff{car.rot, car.pos * kUUtoBT});
  rb.pred = rb.xf;
  rb.lin_vel = car.vel * kUUtoBT;
  rb.ang_vel = car.ang_vel;
  clear_accum(rb);
  update_inertia(rb, bc);
  car.vel_impulse_cache = vzero();
}

RSX_HD RSX_NOINL inline void respawn(ArenaState& S, const StaticData& D, int ci, float boost) {
  Car& car = S.cars[ci];
  const CarConst& cc = D.cars[ci];
  Body& rb = S.bodies[slot(D, cc.body)];
  const BodyConst& bc = D.bodies[cc.body];
  const float lx[4] = {-2304.0f, -2688.0f, 2304.0f, 2688.0f};
  const float half_pi = 1.57079632679489661923132169163975144f;
  uint32_t k = (uint32_t)wy_mod(&S.rng, 4);
  float ydir = cc.team == 0 ? -1.0f : 1.0f;
  V3 pos = {lx[k], fmul(-4608.0f, fneg(ydir)), kRespawnZ};
  M3 rot = yaw_matrix(fadd(half_pi, cc.team == 0 ? 0.0f : kPi));
  float dz = car.dodge_deadzone;
  V3 vic = car.vel_impulse_cache;
  uint32_t sticky = car.sticky_gate_prev;
  Wheel wh[kWheels];
  for (int i = 0; i < kWheels; ++i) wh[i] = car.wheels[i];
  car = Car{};
  car.dodge_deadzone = dz;
  car.vel_impulse_cache = vic;
  car.sticky_gate_prev = sticky;
  for (int i = 0; i < kWheels; ++i) car.wheels[i] = wh[i];
  car.pos = pos;
  car.rot = rot;
  car.boost = rclamp(boost, 0.0f, kBoostMax);
  car.on_ground = 1;
  sync_car_body(car, rb, bc);
  for (int i = 0; i < kWheels; ++i) {
    Wheel& w = car.wheels[i];
    w = Wheel{};
    w.lat_friction = 1.0f;
    w.long_friction = 1.0f;
  }
  car.sticky_gate_prev = 0;
}

// ---- the vehicle ----
RSX_F V3 upwards_from_contacts(const Car& car, V3 chassis_up) {
  V3 sum = vzero();
  for (int i = 0; i < kWheels; ++i) {
    const Wheel& w = car.wheels[i];
    if (w.ray.some && w.ray.v.in_contact_with_world) sum += w.ray.v.contact_normal;
  }
  V3 out;
  return try_normalize(sum, &out) ? out : chassis_up;
}

RSX_F float resolve_collision(const View& b1, const View& b2, V3 pos, V3 n, float dt, float distance) {
  V3 r1 = pos - b1.xf.t, r2 = pos - b2.xf.t;
  V3 v = vel_at(b1, r1) - vel_at(b2, r2);
  float rel = dot(n, v);
  float perr = fdiv(fmul(kPushbackErp, fneg(distance)), dt);
  float verr = fneg(rel);
  float inv = fdiv(1.0f, fadd(impulse_denom(b1, pos, n), impulse_denom(b2, pos, n)));
  return rmax(fadd(fmul(perr, inv), fmul(verr, inv)), 0.0f);
}
RSX_F float resolve_bilateral_ground(const View& b1, V3 inv_local, V3 pos, V3 n) {
  V3 r1 = pos - b1.xf.t;
  V3 v1 = vel_at(b1, r1);
  V3 aj = mul_t(b1.xf.m, cross(r1, n));
  float jd = fadd(b1.inv_mass, dot(inv_local * aj, aj));
  float inv = fdiv(1.0f, jd);
  return fmul(fmul(-0.2f, dot(n, v1)), inv);
}

RSX_F void wheel_raycast_response(Wheel& w, const WheelConst& wc, const View& ch, const Aff& cxf, V3 front_axle, const WheelHit& hit,
                                  const View& hb, float dt, bool front) {
  V3 cp = hit.point, cn = hit.normal;
  bool world = (hb.flags & CF_STATIC) != 0;
  w.axle_dir = front ? front_axle : cxf.m.c1;
  V3 up = cxf.m.c2;
  float trace = dot(w.hard_point - cp, up);
  float travel = fmul(kMaxSuspTravel, kUUtoBT);
  float max_len = fadd(wc.rest_length, travel);
  w.vel_at_contact = vel_at(ch, cp - cxf.t);
  float pv = dot(cn, w.vel_at_contact);
  float den = dot(cn, up);
  float srv, clip;
  if (den > 0.1f) {
    float inv = fdiv(1.0f, den);
    srv = fmul(pv, inv);
    clip = inv;
  } else {
    srv = 0.0f;
    clip = 10.0f;
  }
  float susp = rmin(fsub(trace, wc.radius), max_len);
  w.extra_pushback = 0.0f;
  if (world || hb.user == USER_CAR) {
    float thresh = fsub(fadd(wc.rest_length, wc.radius), kSuspSubtract);
    if (trace < thresh) {
      float res = resolve_collision(ch, hb, hit.point, hit.normal, dt, fsub(trace, thresh));
      w.extra_pushback = fdiv(res, (float)kWheels);
    }
  }
  RayInfo ri;
  ri.contact_normal = cn;
  ri.contact_point = cp;
  ri.ground_body = hit.body;
  ri.suspension_length = susp;
  ri.impulse = vzero();
  ri.ground_stick.some = world ? 0u : 1u;
  ri.ground_stick.v = world ? vzero() : -cn;
  ri.in_contact_with_world = world ? 1u : 0u;
  ri.clipped_inv_contact_dot_susp = clip;
  ri.susp_rel_vel = srv;
  w.ray.some = 1;
  w.ray.v = ri;
}

RSX_F void wheel_friction_curves(Wheel& w, const View& ch, V3 cxf_t, V3 cn, float hb, float thr, bool three, bool dyn_hit) {
  V3 lat = w.axle_dir;
  V3 lon = cross(lat, cn);
  V3 cv = (cross(ch.ang_vel, w.hard_point - cxf_t) + ch.lin_vel) * kBTtoUU;
  float base = fabs_(dot(cv, lat));
  float in = base > 5.0f ? fdiv(base, fadd(fabs_(dot(cv, lon)), base)) : 0.0f;
  float lf = three ? c_lat3(in) : c_lat(in);
  float lg = 1.0f;
  if (hb != 0.0f) {
    lf = fmul(lf, fadd(1.0f, fmul(fsub(c_hb_lat(in), 1.0f), hb)));
    lg = fmul(lg, fadd(1.0f, fmul(fsub(c_hb_long(in), 1.0f), hb)));
  }
  if (thr == 0.0f || dyn_hit) {
    float ns = c_nonsticky(cn.z);
    lf = fmul(lf, ns);
    lg = fmul(lg, ns);
  }
  w.lat_friction = lf;
  w.long_friction = lg;
}

RSX_F V3 steered_axle(const Aff& cxf, float angle) {
  float s, c;
  cr_sincos(fmul(angle, 0.5f), &s, &c);
  return qrotate(quat_axis_sc(cxf.m.c2, s, c), cxf.m.c1);
}

// the wheels' hard points and the packet of the four wheel rays (the start of vehicle_update's ray query)
RSX_F void vehicle_rays_begin(ArenaState& S, const StaticData& D, int ci, RayPacket& pk) {
  Car& car = S.cars[ci];
  const CarConst& cc = D.cars[ci];
  const uint32_t cidx = cc.body;
  Aff cxf = S.bodies[slot(D, cidx)].xf;
  V3 src[kWheels], tgt[kWheels];
  for (int i = 0; i < kWheels; ++i) {
    Wheel& w = car.wheels[i];
    const WheelConst& wc = cc.wheels[i];
    w.hard_point = xform_point(cxf, wc.connection);
    tgt[i] = w.hard_point - (cxf.m.c2 * wc.ray_length);
    src[i] = w.hard_point;
  }
  wheel_packet_init(pk, src, tgt, cidx);
}
// the wheels' hard points and the four wheel rays against the world (the first half of vehicle_update)
RSX_HD RSX_NOINL inline void vehicle_rays(ArenaState& S, const StaticData& D, int ci, WheelHit hits[kWheels]) {
  RayPacket pk;
  vehicle_rays_begin(S, D, ci, pk);
  RSX_ZONE_BEGIN(z_rays);
  grid_rays(S, D, &pk);
  RSX_ZONE_END(z_rays, 1);
  wheel_packet_hits(S, D, pk, hits);
}

// the wheels' response to the ray hits: suspension, friction and their impulses (the second half of vehicle_update)
RSX_HD RSX_NOINL inline void vehicle_response(ArenaState& S, const StaticData& D, int ci, float dt, float hb, float thr, bool three,
                                              const WheelHit hits[kWheels]) {
  Car& car = S.cars[ci];
  const CarConst& cc = D.cars[ci];
  const uint32_t cidx = cc.body;
  const int cd = slot(D, cidx);
  const BodyConst& cbc = D.bodies[cidx];
  Aff cxf = S.bodies[cd].xf;
  V3 ct = cxf.t;
  float fscale = fdiv(mass_of(cbc), 3.0f);
  RSX_ZONE_BEGIN(z_resp);
  bool have_axle = false;
  float axle_angle = 0.0f;
  V3 axle = vzero();
  int ncontact = 0;
  for (int i = 0; i < kWheels; ++i) {
    Wheel& w = car.wheels[i];
    if (!hits[i].some) {
      w.extra_pushback = 0.0f;
      w.ray = Opt<RayInfo>{};
      continue;
    }
    {
      View ch = view(S, D, cidx);
      View hbody = view(S, D, hits[i].body);
      ncontact += 1;
      bool front = i < 2;
      V3 ad;
      if (front) {
        if (have_axle && axle_angle == w.steer_angle) {
          ad = axle;
        } else {
          axle = steered_axle(cxf, w.steer_angle);
          have_axle = true;
          axle_angle = w.steer_angle;
          ad = axle;
        }
      } else {
        ad = cxf.m.c1;
      }
      wheel_raycast_response(w, cc.wheels[i], ch, cxf, ad, hits[i], hbody, dt, front);
      wheel_friction_curves(w, ch, ct, hits[i].normal, hb, thr, three, (hbody.flags & CF_STATIC) == 0);
    }
    // dynamic effects of this wheel before the next wheel reads velocities
    const RayInfo& ri = w.ray.v;
    if (ri.ground_stick.some) {
      int gd = slot(D, ri.ground_body);
      Body& g = S.bodies[gd];
      add_impulse(g, D.bodies[ri.ground_body], IMP_LINEAR_AT, ri.ground_stick.v, ri.contact_point - g.xf.t, true, false);
    }
    if (w.extra_pushback > 0.0f && D.bodies[ri.ground_body].user == USER_CAR) {
      int vd = slot(D, ri.ground_body);
      Body& vb = S.bodies[vd];
      float full = fmul(w.extra_pushback, (float)kWheels);
      add_impulse(vb, D.bodies[ri.ground_body], IMP_LINEAR_AT, -ri.contact_normal * full, ri.contact_point - vb.xf.t, true, false);
    }
  }
  if (ncontact < 3)
    for (int i = 0; i < kWheels; ++i) car.wheels[i].engine_force = fdiv(car.wheels[i].engine_force, 4.0f);
  // suspension of all wheels
  for (int i = 0; i < kWheels; ++i) {
    Wheel& w = car.wheels[i];
    const WheelConst& wc = cc.wheels[i];
    if (!w.ray.some) continue;
    const RayInfo& ri = w.ray.v;
    float f = fmul(fmul(fsub(wc.rest_length, ri.suspension_length), kSuspStiffness), ri.clipped_inv_contact_dot_susp);
    float dscale = ri.susp_rel_vel < 0.0f ? kDampCompression : kDampRelaxation;
    float sf = fmul(fsub(f, fmul(dscale, ri.susp_rel_vel)), wc.force_scale);
    if (sf <= 0.0f) continue;
    float bscale = fadd(fmul(sf, dt), w.extra_pushback);
    add_impulse(S.bodies[cd], cbc, IMP_LINEAR_AT, ri.contact_normal * bscale, ri.contact_point - ct, true, false);
  }
  // friction impulses of all wheels (computed against the chassis after suspension), then applied
  {
    View ch = view(S, D, cidx);
    for (int i = 0; i < kWheels; ++i) {
      Wheel& w = car.wheels[i];
      if (!w.ray.some) continue;
      V3 cn = w.ray.v.contact_normal, cp = w.ray.v.contact_point;
      V3 axd = normalize_or_zero(w.axle_dir);
      V3 fwd = normalize_or_zero(cross(cn, axd));
      float side = resolve_bilateral_ground(ch, cbc.inv_inertia_local, cp, axd);
      float roll;
      if (w.engine_force == 0.0f) {
        if (w.brake == 0.0f) {
          roll = 0.0f;
        } else {
          float rv = dot(w.vel_at_contact, fwd);
          if (dt > fdiv(1.0f, 80.0f)) {
            float th = fsub(0.8f, fdiv(1.0f, fmul(dt, 150.0f)));
            if (fabs_(rv) < th) rv = 0.0f;
          }
          roll = rclamp(fmul(fneg(rv), 113.73963f), fneg(w.brake), w.brake);
        }
      } else {
        roll = fdiv(fneg(w.engine_force), fscale);
      }
      V3 total = fwd * roll * w.long_friction + axd * side * w.lat_friction;
      w.ray.v.impulse = total * fscale;
    }
  }
  for (int i = 0; i < kWheels; ++i) {
    const Wheel& w = car.wheels[i];
    if (!w.ray.some) continue;
    const RayInfo& ri = w.ray.v;
    V3 off = ri.contact_point - cxf.t;
    float upd = dot(cxf.m.c2, off);
    V3 rel = off - cxf.m.c2 * upd;
    add_impulse(S.bodies[cd], cbc, IMP_LINEAR_AT, ri.impulse * dt, rel, true, false);
  }
  RSX_ZONE_END(z_resp, 2);
}

// vehicle_rl.cuh:56-138: rays, then the response (the rays read body poses only; the response writes velocities)
RSX_F void vehicle_update(ArenaState& S, const StaticData& D, int ci, float dt, float hb, float thr, bool three) {
  WheelHit hits[kWheels];
  vehicle_rays(S, D, ci, hits);
  vehicle_response(S, D, ci, dt, hb, thr, three, hits);
}

// ---- the car's pre-tick ----
struct UpCache {
  bool some;
  V3 dir;
};
RSX_F V3 cached_up(const Car& car, const Body& rb, UpCache& uc) {
  if (uc.some) return uc.dir;
  uc.dir = upwards_from_contacts(car, rb.xf.m.c2);
  uc.some = true;
  return uc.dir;
}

RSX_F void update_wheels(ArenaState& S, const StaticData& D, int ci, Body& rb, float fwd_speed, UpCache& uc) {
  Car& car = S.cars[ci];
  const CarConst& cc = D.cars[ci];
  const BodyConst& bc = D.bodies[cc.body];
  float hbd = fmul(car.controls.handbrake ? kPowerslideRise : -kPowerslideFall, kTickTime);
  car.handbrake_val = rclamp(fadd(car.handbrake_val, hbd), 0.0f, 1.0f);
  float brake = 0.0f;
  float raw_thr = car.controls.throttle;
  V3 q = quant_axes(V3{raw_thr, car.controls.steer, 0.0f});
  bool all4 = wheels_in_contact(car) == (uint32_t)kWheels;
  float thr = (car.controls.boost && car.boost > 0.0f && all4) ? 1.0f : q.x;
  float afs = fabs_(fwd_speed);
  float eng = thr;
  if (!car.controls.handbrake) {
    if (fabs_(thr) > kThrottleDeadzone) {
      if (afs > kStoppingFwdVel && rsignum(thr) != rsignum(fwd_speed)) {
        brake = 1.0f;
        if (afs > kBrakeNoThrottleThresh) eng = 0.0f;
      }
    } else {
      eng = 0.0f;
      brake = afs < kStoppingFwdVel ? 1.0f : kCoastBrake;
    }
  }
  float dss = c_drive_torque(afs);
  float ef = fmul(fmul(eng, kThrottleTorque * kUUtoBT), dss);
  float bf = fmul(brake, kBrakeTorque * kUUtoBT);
  for (int i = 0; i < kWheels; ++i) {
    car.wheels[i].engine_force = ef;
    car.wheels[i].brake = bf;
  }
  float steer = cc.three_wheels ? c_steer3(afs) : c_steer(afs);
  if (car.handbrake_val != 0.0f) steer = fadd(steer, fmul(fsub(c_slide_steer(afs), steer), car.handbrake_val));
  steer = fmul(steer, q.y);
  car.wheels[0].steer_angle = steer;
  car.wheels[1].steer_angle = steer;
  if (car.sticky_gate_prev) {
    V3 up = cached_up(car, rb, uc);
    bool full = raw_thr != 0.0f || afs > kStoppingFwdVel;
    float sc = fmul(cc.three_wheels ? 0.0f : 1.0f, 0.5f);
    if (full) sc = fadd(sc, fsub(1.0f, fabs_(up.z)));
    add_impulse(rb, bc, IMP_LINEAR, up * sc * -fabs_(D.gravity_uu.z) * kTickTime * kUUtoBT, vzero(), false, true);
  }
}

RSX_F void update_air_torque(ArenaState& S, const StaticData& D, int ci, Body& rb, uint32_t nwic, bool prev_flipping, float prev_ft) {
  Car& car = S.cars[ci];
  const BodyConst& bc = D.bodies[D.cars[ci].body];
  bool allow_dodge = nwic < 3, allow_air = nwic == 0;
  if (car.is_flipping && allow_dodge && !is_zero(car.flip_rel_torque)) {
    V3 t = car.flip_rel_torque;
    float ps = 1.0f;
    if (t.y != 0.0f && car.controls.pitch != 0.0f && rsignum(t.y) == rsignum(car.controls.pitch) && prev_ft >= kFlipPitchCancelMin)
      ps = fsub(1.0f, rmin(fabs_(quant_axis(fneg(car.controls.pitch))), 1.0f));
    t.y = fmul(t.y, ps);
    V3 dt = t * V3{kFlipTorqueX, kFlipTorqueY, kFlipTorqueZ} * kTickTime;
    add_impulse(rb, bc, IMP_ANGULAR, rb.xf.m * dt, vzero(), false, true);
  }
  if (allow_air) {
    V3 in = quant_axes(V3{car.controls.pitch, car.controls.yaw, car.controls.roll});
    float pts = 1.0f;
    if (!is_zero(in) && (prev_flipping || car.is_flipping || prev_ft < kFlipPitchLockExtra)) pts = 0.0f;
    M3 dirs = {-car.rot.c1, car.rot.c2, -car.rot.c0};
    V3 sin_ = in * V3{pts, 1.0f, 1.0f};
    V3 torque = !is_zero(in) ? dirs * (sin_ * V3{kAirTorqueX, kAirTorqueY, kAirTorqueZ}) : vzero();
    V3 keep = vs(1.0f) - vabs(sin_);
    keep.z = 1.0f;
    V3 damp = dirs * (mul_t(dirs, car.ang_vel) * V3{kAirDampX, kAirDampY, kAirDampZ} * keep);
    add_impulse(rb, bc, IMP_ANGULAR, (torque - damp) * kAirTorqueScale * kTickTime, vzero(), false, true);
  }
  if (allow_air) {
    float ts = car.is_boosting ? 1.0f : quant_axis(car.controls.throttle);
    if (ts != 0.0f) add_impulse(rb, bc, IMP_LINEAR, car.rot.c0 * ts * kThrottleAirAccel * kUUtoBT * kTickTime, vzero(), false, true);
  }
}

RSX_F void update_jump(ArenaState& S, const StaticData& D, int ci, Body& rb, bool pressed) {
  Car& car = S.cars[ci];
  const BodyConst& bc = D.bodies[D.cars[ci].body];
  V3 up = car.rot.c2;
  if (!car.has_jumped && car.on_ground && pressed) {
    car.is_jumping = 1;
    car.has_jumped = 1;
    car.jump_ticks = 0;
    car.jump_hold_broken = 0;
  }
  car.jump_ticks += 1;
  if (car.is_jumping) {
    if (!car.controls.jump) car.jump_hold_broken = 1;
    car.is_jumping = (car.jump_ticks <= kJumpMinTicks || (!car.jump_hold_broken && car.controls.jump && car.jump_ticks <= kJumpMaxTicks)) ? 1u : 0u;
    if (!car.is_jumping) car.jump_ticks = 1;
  }
  if (car.is_jumping) {
    if (car.jump_ticks == 1) {
      add_impulse(rb, bc, IMP_LINEAR, up * D.mut[M_JUMP_IMMEDIATE] * kUUtoBT, vzero(), false, false);
      limit_vels(rb, fmul(kCarMaxSpeed, kUUtoBT), kCarMaxAngSpeed);
    }
    add_impulse(rb, bc, IMP_LINEAR, up * D.mut[M_JUMP_ACCEL] * (kUUtoBT * kTickTime), vzero(), false, true);
  }
}

RSX_F void update_auto_flip(ArenaState& S, const StaticData& D, int ci, Body& rb, bool pressed) {
  Car& car = S.cars[ci];
  const BodyConst& bc = D.bodies[D.cars[ci].body];
  if (pressed && car.world_contact_normal.some && car.world_contact_normal.v.z > kAutoflipNormZ) {
    float yz = car.rot.c1.z, zz = car.rot.c2.z;
    float cy = fsqrt(fadd(fmul(zz, zz), fmul(yz, yz)));
    float roll = cy > fmul(16.0f, kEps) ? cr_atan2(yz, zz) : 0.0f;
    float ar = fabs_(roll);
    if (ar > kAutoflipRollThresh) {
      car.auto_flip_timer = fmul(kAutoflipTime, fdiv(ar, kPi));
      car.auto_flip_torque_scale = autoflip_sign(D, car.rot);
      car.is_auto_flipping = 1;
      add_impulse(rb, bc, IMP_LINEAR, -car.rot.c2 * (kAutoflipImpulse * kUUtoBT), vzero(), false, false);
    }
  }
  if (car.is_auto_flipping) {
    if (car.auto_flip_timer <= 0.0f) {
      car.is_auto_flipping = 0;
      car.auto_flip_timer = 0.0f;
    } else {
      rb.ang_vel += car.rot.c0 * kAutoflipAngVel * car.auto_flip_torque_scale;
      limit_vels(rb, fmul(kCarMaxSpeed, kUUtoBT), kCarMaxAngSpeed);
      car.auto_flip_timer = fsub(car.auto_flip_timer, kTickTime);
    }
  }
}

RSX_F bool update_double_jump_or_flip(ArenaState& S, const StaticData& D, int ci, Body& rb, bool pressed, float fwd_speed, bool was_jumping) {
  Car& car = S.cars[ci];
  const BodyConst& bc = D.bodies[D.cars[ci].body];
  if (car.on_ground) {
    car.has_double_jumped = 0;
    car.has_flipped = 0;
    car.air_time = 0.0f;
    car.air_time_since_jump = 0.0f;
    car.flip_time = fadd(car.flip_time, kTickTime);
    return false;
  }
  car.air_time = fadd(car.air_time, kTickTime);
  if (car.has_jumped && !was_jumping && !car.is_jumping) car.air_time_since_jump = fadd(car.air_time_since_jump, kTickTime);
  else car.air_time_since_jump = 0.0f;
  if (pressed && car.air_time_since_jump < kDoubleJumpMaxDelay) {
    V3 di = quant_axes(V3{car.controls.pitch, car.controls.yaw, car.controls.roll} * V3{-1.0f, 1.0f, 1.0f});
    float mag = fadd(fadd(fabs_(di.x), fabs_(di.y)), fabs_(di.z));
    bool flip_in = mag >= S.cars[ci].dodge_deadzone;
    bool unlimited = flip_in ? (D.unlimited_flips != 0) : (D.unlimited_double_jumps != 0);
    if ((!car.is_auto_flipping && !car.has_double_jumped && !car.has_flipped) || unlimited) {
      car.has_jumped = 1;
      if (flip_in) {
        car.flip_time = 0.0f;
        car.has_flipped = 1;
        car.is_flipping = 1;
        V3 dd = di;
        dd.y = fadd(dd.y, dd.z);
        if (fabs_(dd.x) < 0.1f && fabs_(dd.y) < 0.1f) {
          dd = vzero();
        } else {
          dd.z = 0.0f;
          dd = normalize_or_zero(dd);
        }
        V3 dz = V3{fabs_(dd.x) < 0.1f ? 0.0f : dd.x, fabs_(dd.y) < 0.1f ? 0.0f : dd.y, fabs_(dd.z) < 0.1f ? 0.0f : dd.z};
        if (len2(dz) > fmul(kEps, kEps)) {
          car.flip_rel_torque = V3{fneg(dd.y), dd.x, 0.0f};
          bool back = fabs_(fwd_speed) < 100.0f ? (bits(dz.x) >> 31) != 0 : rsignum(dz.x) != rsignum(fwd_speed);
          float msx = back ? kFlipBackScale : kFlipFwdScale;
          float ratio = fdiv(fabs_(fwd_speed), kCarMaxSpeed);
          V3 iv = dz * kFlipInitVel;
          iv.x = fmul(iv.x, fadd(fmul(fsub(msx, 1.0f), ratio), 1.0f));
          iv.y = fmul(iv.y, fadd(fmul(fsub(kFlipSideScale, 1.0f), ratio), 1.0f));
          if (back) iv.x = fmul(iv.x, kFlipBackScaleX);
          V3 fd = car.rot.c0;
          fd.z = 0.0f;
          V3 f2 = normalize_or_zero(fd);
          V3 r2 = {fneg(f2.y), f2.x, 0.0f};
          V3 dv = iv.x * f2 + iv.y * r2;
          add_impulse(rb, bc, IMP_LINEAR, dv * kUUtoBT, vzero(), false, false);
          limit_vels(rb, fmul(kCarMaxSpeed, kUUtoBT), kCarMaxAngSpeed);
        }
      } else {
        add_impulse(rb, bc, IMP_LINEAR, car.rot.c2 * D.mut[M_JUMP_IMMEDIATE] * kUUtoBT, vzero(), false, false);
        limit_vels(rb, fmul(kCarMaxSpeed, kUUtoBT), kCarMaxAngSpeed);
        car.has_double_jumped = 1;
      }
    }
  }
  if (car.is_flipping) {
    float ft = car.flip_time;
    bool still = car.has_flipped && ft < kFlipTorqueTime;
    car.is_flipping = still ? 1u : 0u;
    car.flip_time = still ? fadd(ft, kTickTime) : kTickTime;
    return !still;
  }
  car.flip_time = fadd(car.flip_time, kTickTime);
  return false;
}

RSX_F void update_auto_roll(ArenaState& S, const StaticData& D, int ci, Body& rb, uint32_t nwic, UpCache& uc) {
  Car& car = S.cars[ci];
  const BodyConst& bc = D.bodies[D.cars[ci].body];
  if (!car.sticky_gate_prev && !car.world_contact_normal.some) return;
  V3 gu = (car.sticky_gate_prev && nwic > 0) ? cached_up(car, rb, uc) : car.world_contact_normal.v;
  V3 gd = -gu;
  V3 f = car.rot.c0, r = car.rot.c1;
  V3 cr = cross(gu, f);
  V3 cf = cross(gd, cr);
  float rtf = fsub(1.0f, rclamp(dot(r, cr), 0.0f, 1.0f));
  float ftf = fsub(1.0f, rclamp(dot(f, cf), 0.0f, 1.0f));
  V3 tdr = f * fneg(rsignum(dot(r, gu)));
  V3 tdf = r * rsignum(dot(f, gu));
  V3 tr = tdr * rtf, tf = tdf * ftf;
  add_impulse(rb, bc, IMP_LINEAR, gd * (kAutorollForce * kUUtoBT * kTickTime), vzero(), false, true);
  add_impulse(rb, bc, IMP_ANGULAR, (tf + tr) * (kAutorollTorque * kTickTime), vzero(), false, true);
}

RSX_F void update_boost(ArenaState& S, const StaticData& D, int ci, Body& rb) {
  Car& car = S.cars[ci];
  const BodyConst& bc = D.bodies[D.cars[ci].body];
  const float ag = D.mut[M_BOOST_ACCEL_GROUND], aa = D.mut[M_BOOST_ACCEL_AIR];
  auto thrust = [&]() {
    car.is_boosting = 1;
    car.boosting_time = fadd(car.boosting_time, kTickTime);
    car.time_since_boosted = 0.0f;
    float acc = car.on_ground ? ag : aa;
    add_impulse(rb, bc, IMP_LINEAR, acc * car.rot.c0 * (kUUtoBT * kTickTime), vzero(), false, true);
  };
  auto coast = [&]() {
    car.is_boosting = 0;
    car.boosting_time = 0.0f;
    car.time_since_boosted = fadd(car.time_since_boosted, kTickTime);
    if (D.recharge_boost && car.time_since_boosted >= D.recharge_delay)
      car.boost = fadd(car.boost, fmul(D.recharge_per_second, kTickTime));
  };
  if (car.is_boosting) {
    float cost = fmul(D.mut[M_BOOST_PER_SECOND], kTickTime);
    car.boost = rmax(fsub(car.boost, cost), 0.0f);
    bool depleted = car.boost == 0.0f;
    bool expired = !car.controls.boost && car.boosting_time >= kBoostMinTime;
    if (depleted || expired) coast();
    else thrust();
  } else if (car.controls.boost && car.boost > 0.0f) {
    thrust();
  } else {
    coast();
  }
  car.boost = rclamp(car.boost, 0.0f, D.mut[M_MAX_BOOST]);
}

RSX_F void update_contact_state(ArenaState& S, const StaticData& D, int ci) {
  Car& car = S.cars[ci];
  uint32_t num = 0;
  for (int i = 0; i < kWheels; ++i) {
    const Wheel& w = car.wheels[i];
    Opt<HitInfo> h = Opt<HitInfo>{};
    if (w.ray.some) {
      const RayInfo& ri = w.ray.v;
      float tl = len(w.hard_point - ri.contact_point);
      h.some = 1;
      h.v.hit_point = ri.contact_point * kBTtoUU;
      h.v.hit_normal = ri.contact_normal;
      h.v.hit_fraction = fdiv(tl, D.cars[ci].wheels[i].ray_length);
      h.v.user_info = D.bodies[ri.ground_body].user;
    }
    car.wheel_contact[i] = h;
    num += h.some ? 1u : 0u;
  }
  car.on_ground = num >= 3 ? 1u : 0u;
}

RSX_F void flip_zdamp(ArenaState& S, const StaticData& D, int ci) {
  Car& car = S.cars[ci];
  if (car.is_demoed || car.on_ground || !car.is_flipping) return;
  if (!(car.flip_time >= kFlipZDampStart && car.flip_time <= kFlipTorqueTime)) return;
  Body& rb = S.bodies[slot(D, D.cars[ci].body)];
  if (rb.lin_vel.z < 0.0f || car.flip_time < kFlipZDampEnd) rb.lin_vel.z = fmul(rb.lin_vel.z, fsub(1.0f, kFlipZDamp120));
}

// The car's pre-tick up to its vehicle update; false for a demolished car (whose pre-tick ends here).  *rthr receives the
// throttle the vehicle update uses.
// the pre-tick's values that its parts pass on
struct PreTick {
  float fwd, prev_ft;
  uint32_t nwic;
  UpCache uc;
  bool pressed, was_jumping, prev_flipping, flip_ended;
};

// The car's pre-tick up to its vehicle update, in three parts a kernel can barrier between; part 1 returns false for a
// demolished car (whose pre-tick ends there).
// part 1: the demolished car's timer and respawn, else activation, control clamps and the wheels' drive and steer
RSX_F bool car_pre_tick_wheels(ArenaState& S, const StaticData& D, int ci, PreTick& p) {
  Car& car = S.cars[ci];
  const CarConst& cc = D.cars[ci];
  Body& rb = S.bodies[slot(D, cc.body)];
  if (car.is_demoed) {
    car.demo_respawn_timer = rmax(fsub(car.demo_respawn_timer, kTickTime), 0.0f);
    if (car.demo_respawn_timer == 0.0f) respawn(S, D, ci, D.mut[M_SPAWN_BOOST]);
    if (rb.activation != ACT_DISABLED) rb.activation = ACT_DISABLED;
    rb.flags |= CF_NO_RESPONSE;
    return false;
  }
  force_activate(rb);
  rb.flags &= ~CF_NO_RESPONSE;
  car.controls.throttle = rclamp(car.controls.throttle, -1.0f, 1.0f);
  car.controls.steer = rclamp(car.controls.steer, -1.0f, 1.0f);
  car.controls.pitch = rclamp(car.controls.pitch, -1.0f, 1.0f);
  car.controls.yaw = rclamp(car.controls.yaw, -1.0f, 1.0f);
  car.controls.roll = rclamp(car.controls.roll, -1.0f, 1.0f);
  p.fwd = fmul(dot(rb.lin_vel, rb.xf.m.c0), kBTtoUU);
  p.pressed = car.controls.jump && !car.prev_controls.jump;
  p.nwic = wheels_in_contact(car);
  p.uc = UpCache{false, vzero()};
  update_wheels(S, D, ci, rb, p.fwd, p.uc);
  if (car.on_ground) {
    if (car.is_flipping) car.flip_time = 0.0f;
    car.is_flipping = 0;
  }
  return true;
}
// part 2: jump, auto-flip, double jump or flip
RSX_F void car_pre_tick_jumps(ArenaState& S, const StaticData& D, int ci, PreTick& p) {
  Car& car = S.cars[ci];
  Body& rb = S.bodies[slot(D, D.cars[ci].body)];
  p.was_jumping = car.is_jumping != 0;
  update_jump(S, D, ci, rb, p.pressed);
  update_auto_flip(S, D, ci, rb, p.pressed);
  p.prev_flipping = car.is_flipping != 0;
  p.prev_ft = car.flip_time;
  p.flip_ended = update_double_jump_or_flip(S, D, ci, rb, p.pressed, p.fwd, p.was_jumping);
}
// part 3: air torque, auto-roll, boost; returns the throttle the vehicle update uses
RSX_F float car_pre_tick_air(ArenaState& S, const StaticData& D, int ci, PreTick& p) {
  Car& car = S.cars[ci];
  Body& rb = S.bodies[slot(D, D.cars[ci].body)];
  if (!car.on_ground) update_air_torque(S, D, ci, rb, p.nwic, p.prev_flipping, p.prev_ft);
  float qthr = quant_axis(car.controls.throttle);
  if (qthr != 0.0f && !car.is_flipping && !p.flip_ended && ((0 < p.nwic && p.nwic < 4) || car.world_contact_normal.some))
    update_auto_roll(S, D, ci, rb, p.nwic, p.uc);
  car.world_contact_normal = Opt<V3>{};
  update_boost(S, D, ci, rb);
  return (car.controls.boost && car.boost > 0.0f) ? 1.0f : qthr;
}

// the three parts in order; false for a demolished car.  *rthr receives the throttle the vehicle update uses.
RSX_F bool car_pre_tick_head(ArenaState& S, const StaticData& D, int ci, float* rthr_out) {
  RSX_ZONE_BEGIN(z_pre);
  PreTick p;
  if (!car_pre_tick_wheels(S, D, ci, p)) return false;
  car_pre_tick_jumps(S, D, ci, p);
  *rthr_out = car_pre_tick_air(S, D, ci, p);
  RSX_ZONE_END(z_pre, 0);
  return true;
}

// the car's pre-tick after its vehicle update: wheel contact state and the sticky-force gate
RSX_F void car_pre_tick_tail(ArenaState& S, const StaticData& D, int ci) {
  Car& car = S.cars[ci];
  RSX_ZONE_BEGIN(z_post);
  update_contact_state(S, D, ci);
  uint32_t world = 0;
  for (int i = 0; i < kWheels; ++i)
    if (car.wheels[i].ray.some && car.wheels[i].ray.v.in_contact_with_world) world = 1;
  car.sticky_gate_prev = world;
  RSX_ZONE_END(z_post, 3);
}

// car_pre_tick.cuh:638-705
RSX_F void car_pre_tick(ArenaState& S, const StaticData& D, int ci) {
  float rthr;
  if (!car_pre_tick_head(S, D, ci, &rthr)) return;
  vehicle_update(S, D, ci, kTickTime, S.cars[ci].handbrake_val, rthr, D.cars[ci].three_wheels != 0);
  car_pre_tick_tail(S, D, ci);
}

RSX_F void phase1(ArenaState& S, const StaticData& D) {
  for (int ci = 0; ci < kCars; ++ci) flip_zdamp(S, D, ci);
  for (int ci = 0; ci < kCars; ++ci) {
    uint32_t was = S.cars[ci].on_ground;
    car_pre_tick(S, D, ci);
    if (!was && S.cars[ci].on_ground) S.events |= 1u << (EV_LANDED + ci);
  }
}

}  // namespace sim
}  // namespace rsx
