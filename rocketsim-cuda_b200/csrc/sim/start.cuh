// Seeded start states of an arena (host and device from one source): the scenario mix kickoff / open play / head-on /
// corner or wall pinch / boost-pad contention, car and ball poses and velocities, and a consistent broadphase.  The
// host builds the benchmark's and the tests' states with it (csrc/world.cpp); the device resets arenas with it
// (rsx_reset_arenas_raw), giving the same words for the same (seed, arena index, StaticData).
// All arithmetic is binary32 without contraction (the library's float policy), with the correctly rounded sin / cos.
// Every draw from the generator is its own statement, so the draws' order is the same for every compiler (where one
// expression drew twice, the order is the one the host compiler used when the committed fixtures were made).
#pragma once
#include "physics.cuh"

namespace rsx {
namespace world {

constexpr float BT = 1.0f / 50.0f;

// ---- seeded generator (SplitMix64) ----
struct Rng {
  uint64_t s;
  RSX_HD uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  RSX_HD float uni() { return (float)(next() >> 40) * (1.0f / 16777216.0f); }  // [0, 1)
  RSX_HD float range(float a, float b) { return a + (b - a) * uni(); }
};


RSX_HD inline M3 rot_ypr(float yaw, float pitch, float roll) {
  float cy = cr_cos(yaw), sy = cr_sin(yaw), cp = cr_cos(pitch), sp = cr_sin(pitch), cr = cr_cos(roll), sr = cr_sin(roll);
  V3 fwd = {cp * cy, cp * sy, sp};
  V3 right = {cy * sp * sr - cr * sy, sy * sp * sr + cr * cy, -cp * sr};
  V3 up = {-cr * cy * sp - sr * sy, -cr * sy * sp + sr * cy, cp * cr};
  // re-orthonormalise in float
  fwd = normalize(fwd);
  up = normalize(cross(fwd, right));
  right = cross(up, fwd);
  return M3{fwd, right, up};
}

RSX_HD inline V3 rand_dir(Rng& r) {
  for (;;) {
    V3 v = {r.range(-1, 1), r.range(-1, 1), r.range(-1, 1)};
    float l = len2(v);
    if (l > 0.01f && l <= 1.0f) return v / fsqrt(l);
  }
}

struct CarPose { V3 pos, vel, ang; M3 rot; float boost; bool ground; };

RSX_HD inline void init_car(ArenaState& s, const StaticData& sd, int ci, const CarPose& p) {
  Car& c = s.cars[ci];
  c.dodge_deadzone = 0.5f;
  c.pos = p.pos;
  c.rot = p.rot;
  c.vel = p.vel;
  c.ang_vel = p.ang;
  c.boost = p.boost;
  c.on_ground = p.ground ? 1u : 0u;
  for (int w = 0; w < kWheels; ++w) {
    c.wheels[w].lat_friction = 1.0f;
    c.wheels[w].long_friction = 1.0f;
  }
  Body& b = s.bodies[1 + ci];
  b.flags = 2u;  // custom material
  sim::set_body_pose(b, sd.bodies[sd.cars[ci].body], Aff{p.rot, p.pos * BT}, p.vel * BT, p.ang);
}

// arena a's start state: a function of (seed, a) and its StaticData only
RSX_HD inline void make_state(const StaticData& sd, ArenaState& s, uint32_t a, uint64_t seed, const float* mix) {
  const float HXF = 4096.0f - 200.0f, HYF = 5120.0f - 250.0f;
  {
    Rng r{seed * 0x100000001B3ull + a * 0x9E3779B97F4A7C15ull + 17};
    r.next();
    memset(&s, 0, sizeof(ArenaState));
    s.tick_count = u64w(r.next() & 0xFFFFF);
    s.rng = u64w(r.next());
    // scenario
    float u = r.uni(), acc = 0.0f;
    int kind = 4;
    for (int k = 0; k < 5; ++k) {
      acc += mix[k];
      if (u < acc) { kind = k; break; }
    }
    V3 ball_pos = {0.0f, 0.0f, 93.15f}, ball_vel = vzero(), ball_ang = vzero();
    CarPose cp[2];
    auto grounded = [&](V3 pos, float yaw, float speed) {
      CarPose p;
      p.pos = V3{pos.x, pos.y, 17.0f};
      p.rot = rot_ypr(yaw, 0.0f, 0.0f);
      p.vel = p.rot.c0 * speed;
      p.ang = vzero();
      p.boost = r.range(0.0f, 100.0f);
      p.ground = true;
      return p;
    };
    if (kind == 0) {  // kickoff: one of the five spawn pairs
      const float sp[5][3] = {{-2048, -2560, 0.785398f}, {2048, -2560, 2.356194f}, {-256, -3840, 1.570796f},
                              {256, -3840, 1.570796f}, {0, -4608, 1.570796f}};
      int k = (int)(r.next() % 5);
      cp[0] = grounded(V3{sp[k][0], sp[k][1], 17.0f}, sp[k][2], 0.0f);
      cp[1] = grounded(V3{-sp[k][0], -sp[k][1], 17.0f}, sp[k][2] + 3.14159265f, 0.0f);
      cp[0].boost = cp[1].boost = 100.0f / 3.0f;
    } else if (kind == 1) {  // open play
      for (int ci = 0; ci < 2; ++ci) {
        V3 pos = {r.range(-HXF, HXF), r.range(-HYF, HYF), 17.0f};
        float yaw = r.range(-3.14159f, 3.14159f);
        float speed = r.range(0.0f, 2300.0f);
        if (r.uni() < 0.5f) {
          cp[ci] = grounded(pos, yaw, speed);
        } else {
          CarPose p;
          p.pos = V3{pos.x, pos.y, r.range(17.0f, 1800.0f)};
          float roll = r.range(-3.1f, 3.1f);
          float pitch = r.range(-1.5f, 1.5f);
          p.rot = rot_ypr(yaw, pitch, roll);
          p.vel = rand_dir(r) * speed;
          float spin = r.range(0.0f, 5.5f);
          p.ang = rand_dir(r) * spin;
          p.boost = r.range(0.0f, 100.0f);
          p.ground = false;
          cp[ci] = p;
        }
      }
      ball_pos = V3{r.range(-3800.0f, 3800.0f), r.range(-4800.0f, 4800.0f), r.range(93.15f, 1900.0f)};
      float bspeed = r.range(0.0f, 4000.0f);
      ball_vel = rand_dir(r) * bspeed;
      float bspin = r.range(0.0f, 6.0f);
      ball_ang = rand_dir(r) * bspin;
    } else if (kind == 2) {  // head-on
      float dist = r.range(500.0f, 1500.0f), yaw = r.range(-3.14159f, 3.14159f);
      V3 c = {r.range(-3000.0f, 3000.0f), r.range(-3800.0f, 3800.0f), 17.0f};
      V3 d = {cr_cos(yaw), cr_sin(yaw), 0.0f};
      cp[0] = grounded(c - d * (dist * 0.5f), yaw, r.range(1400.0f, 2300.0f));
      cp[1] = grounded(c + d * (dist * 0.5f), yaw + 3.14159265f, r.range(1400.0f, 2300.0f));
      ball_pos = V3{r.range(-3000.0f, 3000.0f), r.range(-4000.0f, 4000.0f), 93.15f};
    } else if (kind == 3) {  // corner / wall pinch
      int corner = (int)(r.next() % 6);
      V3 bp;
      if (corner < 4) bp = V3{(corner & 1 ? 1.0f : -1.0f) * (4096.0f - 91.25f - r.range(0.0f, 200.0f)),
                              (corner & 2 ? 1.0f : -1.0f) * (5120.0f - 91.25f - r.range(0.0f, 200.0f)), r.range(93.15f, 300.0f)};
      else bp = V3{(corner & 1 ? 1.0f : -1.0f) * (4096.0f - 91.25f - r.range(0.0f, 200.0f)), r.range(-3000.0f, 3000.0f),
                   r.range(93.15f, 300.0f)};
      ball_pos = bp;
      V3 toward = normalize(V3{bp.x, bp.y, 0.0f} - V3{bp.x * 0.7f, bp.y * 0.7f, 0.0f});
      float yaw = cr_atan2(toward.y, toward.x);
      V3 start = V3{bp.x, bp.y, 17.0f} - toward * r.range(300.0f, 900.0f);
      cp[0] = grounded(start, yaw, r.range(1000.0f, 2300.0f));
      float speed1 = r.range(0.0f, 2300.0f);
      float yaw1 = r.range(-3.14159f, 3.14159f);
      V3 pos1 = {r.range(-HXF, HXF), r.range(-HYF, HYF), 17.0f};
      cp[1] = grounded(pos1, yaw1, speed1);
    } else {  // boost-pad contention
      int p = (int)(r.next() % kPads);
      V3 pp = sd.pads[p].pos;
      for (int ci = 0; ci < 2; ++ci) {
        float ang = r.range(-3.14159f, 3.14159f), rad = r.range(0.0f, 300.0f);
        V3 pos = {pp.x + rad * cr_cos(ang), pp.y + rad * cr_sin(ang), 17.0f};
        pos.x = rclamp(pos.x, -HXF, HXF);
        pos.y = rclamp(pos.y, -HYF, HYF);
        float speed = r.range(0.0f, 1500.0f);
        float yaw = r.range(-3.14159f, 3.14159f);
        cp[ci] = grounded(pos, yaw, speed);
        cp[ci].boost = r.range(0.0f, 90.0f);
      }
      ball_pos = V3{r.range(-3800.0f, 3800.0f), r.range(-4800.0f, 4800.0f), 93.15f};
    }
    // ball
    s.ball.pos = ball_pos;
    s.ball.rot = m3_identity();
    s.ball.vel = ball_vel;
    s.ball.ang_vel = ball_ang;
    s.bodies[0].flags = 2u | 4u;  // custom material, can sleep
    sim::set_body_pose(s.bodies[0], sd.bodies[20], Aff{m3_identity(), ball_pos * BT}, ball_vel * BT, ball_ang);
    for (int ci = 0; ci < 2; ++ci) init_car(s, sd, ci, cp[ci]);
    sim::init_broadphase(s, sd);
  }
}

}  // namespace world
}  // namespace rsx
