// V3 dump bytes <-> ArenaState / StaticData: import and export of the per-arena state and the static collision data
// in the format the patched RocketSim V3 writes (the reference's crates/rocketsim-cuda/src/dump.rs:1-1300; the V3 side
// of the format is v3/rocketsim-dump.patch, src/dump.rs there).
//
// The format is its traversal order: little-endian fields, a 4-byte ASCII tag in front of each section, a u32 element
// count in front of each sequence, a V3 bool as one byte, an optional as a flag byte followed by its payload at full
// size.  One template traversal per section serves both directions (Reader / Writer below), so what is written is what
// is read.  The importer refuses what the reference refuses (dump.rs:8-9): a list over its cap (bumping the matching
// overflow counter), Heatseeker / Dropshot / Snowday state away from its default, a ball-world contact record, a
// non-empty free list, constants that differ from StaticData; and, where the reference would index out of bounds, a
// body or car index outside the arena.  Host code only (no device work).
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <string>
#include <vector>
#include "../../include/rsx.h"
#include "state.cuh"
#include "sim/physics.cuh"

int rsx_set_last_error(int code, const char* msg);

static_assert(__BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__, "the dump format is little-endian, as is this host");
static_assert(sizeof(rsx_v3_template) == 5088, "rsx_v3_template layout");

namespace rsx {
namespace v3dump {

constexpr uint8_t kArenaMagic[8] = {'V', '3', 'A', 'R', 'E', 'N', 'A', 0};      // dump.rs:14
constexpr uint8_t kStaticMagic[8] = {'V', '3', 'S', 'T', 'A', 'T', 'I', 'C'};   // dump.rs:15
constexpr uint32_t kArenaVersion = 2, kStaticVersion = 3;                        // dump.rs:16-17
constexpr size_t kArenaHeader = RSX_V3_ARENA_HEADER_LEN;                          // magic, version, config hash, 12 counts
constexpr size_t kStaticHeader = RSX_V3_STATIC_HEADER_LEN;                        // + payload length
constexpr size_t kBodyRecord = RSX_V3_BODY_RECORD_LEN;                            // one dynamic or static BODY record
constexpr size_t kCompanionAt = 1;  // the companion_id option (flag + u32) at bytes 1..6 of a body record
constexpr uint32_t kUserNone = 0, kUserCar = 1, kUserBall = 2;                   // V3's UserInfoType

uint64_t fnv1a64(const uint8_t* p, size_t n) {
  uint64_t h = 0xcbf29ce484222325ull;  // FNV-1a 64: offset basis, then xor-multiply by the FNV prime per byte
  for (size_t i = 0; i < n; ++i) h = (h ^ p[i]) * 0x00000100000001b3ull;
  return h;
}

inline uint32_t tag_word(const char* t) {
  return (uint32_t)(uint8_t)t[0] | (uint32_t)(uint8_t)t[1] << 8 | (uint32_t)(uint8_t)t[2] << 16 | (uint32_t)(uint8_t)t[3] << 24;
}

// ---- the two directions of the byte stream ----
struct Writer {
  static constexpr bool kRead = false;
  std::vector<uint8_t> buf;
  std::vector<size_t> marks;  // offset of every section tag, in order
  std::string err;
  void put(const void* p, size_t n) {
    const uint8_t* b = static_cast<const uint8_t*>(p);
    buf.insert(buf.end(), b, b + n);
  }
  void u8(uint8_t& v) { buf.push_back(v); }
  void u16(uint16_t& v) { put(&v, 2); }
  void u32(uint32_t& v) { put(&v, 4); }
  void u64(uint64_t& v) { put(&v, 8); }
  void f32(float& v) { put(&v, 4); }
  void raw(uint8_t* p, size_t n) { put(p, n); }
  void mark() { marks.push_back(buf.size()); }
  void fail(const std::string& m) {
    if (err.empty()) err = m;
  }
  size_t count(size_t n) {
    uint32_t x = (uint32_t)n;
    u32(x);
    return n;
  }
};

struct Reader {
  static constexpr bool kRead = true;
  const uint8_t* b;
  size_t n, at = 0;
  std::string err;
  Reader(const uint8_t* bytes, size_t len) : b(bytes), n(len) {}
  size_t remaining() const { return n - at; }
  void fail(const std::string& m) {
    if (err.empty()) err = m;
  }
  void take(void* dst, size_t k) {
    if (remaining() < k) {
      fail("dump truncated");
      at = n;
      memset(dst, 0, k);
      return;
    }
    memcpy(dst, b + at, k);
    at += k;
  }
  void u8(uint8_t& v) { take(&v, 1); }
  void u16(uint16_t& v) { take(&v, 2); }
  void u32(uint32_t& v) { take(&v, 4); }
  void u64(uint64_t& v) { take(&v, 8); }
  void f32(float& v) { take(&v, 4); }
  void raw(uint8_t* p, size_t k) {
    if (remaining() < k) {
      fail("dump truncated");
      at = n;
      return;
    }
    memcpy(p, b + at, k);
    at += k;
  }
  void mark() {}
  size_t count(size_t) {  // the writer's n is ignored: the stream says
    uint32_t x = 0;
    u32(x);
    if (x > remaining()) {
      fail("count exceeds the bytes left");
      return 0;
    }
    return x;
  }
};

// ---- field codecs (dump.rs:51-108) ----
template <class IO> void tag(IO& io, const char* t) {
  io.mark();
  uint32_t want = tag_word(t), x = want;
  io.u32(x);
  if (x != want) io.fail(std::string("section tag ") + std::string(t, 4) + " expected");
}
template <class IO> void flag(IO& io, uint32_t& v) {  // a V3 bool as one byte, held as a u32
  uint8_t b = v != 0 ? 1 : 0;
  io.u8(b);
  v = b;
}
template <class IO> void byte(IO& io, uint32_t& v) {  // a u8 field held as a u32
  uint8_t b = (uint8_t)v;
  io.u8(b);
  v = b;
}
template <class IO> void vec3(IO& io, V3& v) {
  io.f32(v.x);
  io.f32(v.y);
  io.f32(v.z);
}
template <class IO> void mat3(IO& io, M3& m) {
  vec3(io, m.c0);
  vec3(io, m.c1);
  vec3(io, m.c2);
}
template <class IO> void aff3(IO& io, Aff& a) {
  mat3(io, a.m);
  vec3(io, a.t);
}
template <class IO> void quat(IO& io, Q4& q) {
  io.f32(q.x);
  io.f32(q.y);
  io.f32(q.z);
  io.f32(q.w);
}
template <class IO> void aabb(IO& io, Box3& b) {
  vec3(io, b.lo);
  vec3(io, b.hi);
}
template <class IO> void word64(IO& io, U64W& v) {
  uint64_t x = u64_of(v);
  io.u64(x);
  v = u64w(x);
}
template <class IO> void opt_idx(IO& io, Opt<uint32_t>& o) {
  flag(io, o.some);
  io.u32(o.v);
}
template <class IO> void opt_u64(IO& io, Opt<U64W>& o) {
  flag(io, o.some);
  word64(io, o.v);
}
template <class IO> void opt_vec3(IO& io, Opt<V3>& o) {
  flag(io, o.some);
  vec3(io, o.v);
}

// ---- the arena traversal (dump.rs:241-371, 449-848) ----
template <class IO> void io_controls(IO& io, Controls& c) {
  io.f32(c.throttle);
  io.f32(c.steer);
  io.f32(c.pitch);
  io.f32(c.yaw);
  io.f32(c.roll);
  flag(io, c.jump);
  flag(io, c.boost);
  flag(io, c.handbrake);
}

template <class IO> void io_hit(IO& io, HitInfo& h) {
  vec3(io, h.hit_point);
  vec3(io, h.hit_normal);
  io.f32(h.hit_fraction);
  byte(io, h.user_info);
}

// A manifold point; V3's applied_impulse is always 0 at a dump and is not state.
template <class IO> void io_point(IO& io, MPoint& p) {
  vec3(io, p.local_a);
  vec3(io, p.local_b);
  vec3(io, p.world_b);
  vec3(io, p.world_a);
  vec3(io, p.normal_b);
  io.f32(p.dist);
  io.f32(p.friction);
  io.f32(p.restitution);
  float applied = 0.0f;
  io.f32(applied);
  uint32_t bits;
  memcpy(&bits, &applied, 4);
  if (IO::kRead && bits != 0) io.fail("manifold point with a non-zero applied_impulse");
  flag(io, p.special);
}

template <class IO> void io_wheel(IO& io, Wheel& w) {
  flag(io, w.ray.some);
  RayInfo& r = w.ray.v;
  vec3(io, r.contact_normal);
  vec3(io, r.contact_point);
  io.u32(r.ground_body);
  io.f32(r.suspension_length);
  vec3(io, r.impulse);
  opt_vec3(io, r.ground_stick);
  flag(io, r.in_contact_with_world);
  io.f32(r.clipped_inv_contact_dot_susp);
  io.f32(r.susp_rel_vel);
  vec3(io, w.hard_point);
  vec3(io, w.axle_dir);
  io.f32(w.engine_force);
  io.f32(w.brake);
  io.f32(w.steer_angle);
  vec3(io, w.vel_at_contact);
  io.f32(w.lat_friction);
  io.f32(w.long_friction);
  io.f32(w.extra_pushback);
}

template <class IO> void io_car(IO& io, Car& c) {
  io.f32(c.dodge_deadzone);
  vec3(io, c.vel_impulse_cache);
  flag(io, c.sticky_gate_prev);
  vec3(io, c.pos);
  mat3(io, c.rot);
  vec3(io, c.vel);
  vec3(io, c.ang_vel);
  io_controls(io, c.controls);
  flag(io, c.has_jumped);
  flag(io, c.has_double_jumped);
  flag(io, c.has_flipped);
  vec3(io, c.flip_rel_torque);
  io.u32(c.jump_ticks);
  io.f32(c.flip_time);
  flag(io, c.is_flipping);
  flag(io, c.is_jumping);
  flag(io, c.jump_hold_broken);
  io.f32(c.air_time);
  io.f32(c.air_time_since_jump);
  io.f32(c.boost);
  io.f32(c.handbrake_val);
  flag(io, c.is_supersonic);
  io.f32(c.supersonic_grace);
  io.f32(c.time_since_boosted);
  io.f32(c.boosting_time);
  flag(io, c.is_boosting);
  flag(io, c.is_auto_flipping);
  io.f32(c.auto_flip_timer);
  io.f32(c.auto_flip_torque_scale);
  io.f32(c.bump_cooldown);
  opt_idx(io, c.bump_victim);
  opt_u64(io, c.last_extra_hit_tick);
  flag(io, c.is_demoed);
  io.f32(c.demo_respawn_timer);
  flag(io, c.on_ground);
  for (int k = 0; k < kWheels; ++k) {
    flag(io, c.wheel_contact[k].some);
    io_hit(io, c.wheel_contact[k].v);
  }
  opt_vec3(io, c.world_contact_normal);
  io_controls(io, c.prev_controls);
  for (int k = 0; k < kWheels; ++k) io_wheel(io, c.wheels[k]);
}

// The BODY record of a dynamic body (219 bytes).  companion_id links a body to its solver body; P5's setup reassigns it
// before any read, so it is not state: written as none, ignored on read.
template <class IO> void io_body(IO& io, Body& b) {
  byte(io, b.flags);
  Opt<uint32_t> companion{0, 0};
  opt_idx(io, companion);
  byte(io, b.activation);
  aff3(io, b.xf);
  quat(io, b.quat);
  aff3(io, b.pred);
  io.f32(b.deactivation_time);
  vec3(io, b.lin_vel);
  vec3(io, b.ang_vel);
  mat3(io, b.inv_inertia_world);
  vec3(io, b.acc_lin);
  vec3(io, b.acc_ang);
  io.f32(b.damp_cache);
  io.f32(b.damp_cache_dt);
  io.f32(b.damp_cache_value);
}

inline uint64_t table_index(uint32_t a, uint32_t b) {  // the triangular pair-index table (dump.rs:373-376)
  uint64_t lo = a <= b ? a : b, hi = a <= b ? b : a;
  return hi * (hi + 1) / 2 + lo;
}

inline int dyn_slot_of_body(const StaticData& sd, uint32_t body) {
  for (int d = 0; d < kDyn; ++d)
    if (sd.dyn_body[d] == body) return d;
  return -1;
}
inline int dyn_slot_of_handle(const StaticData& sd, uint32_t h) {
  for (int d = 0; d < kDyn; ++d)
    if (sd.dyn_handle[d] == h) return d;
  return -1;
}

// V3's contact records of a tick, in call order, folded the way P7 reads them (dump.rs:387-422): car - ball and
// car - car records are kept in order; a car - world record sets EV_CAR_HIT_WORLD + car and leaves its normal in
// fold_car_normal[car] (the last one wins); a ball - world record sets EV_BALL_HIT_WORLD, plus EV_BALL_WALL when
// |normal.z| < 0.8; any other record has no effect in P7 and is dropped.
bool fold_records(ArenaState& s, const StaticData& sd, const std::vector<Record>& recs, std::string& err) {
  s.fold_events = 0;
  memset(s.fold_car_normal, 0, sizeof(s.fold_car_normal));
  s.n_records = 0;
  memset(s.records, 0, sizeof(s.records));
  for (const Record& r : recs) {
    if (r.body_a >= (uint32_t)kBodies || r.body_b >= (uint32_t)kBodies) {
      err = "contact record body index out of range";
      return false;
    }
    const BodyConst& a = sd.bodies[r.body_a];
    const BodyConst& b = sd.bodies[r.body_b];
    if (a.user == kUserCar && (b.user == kUserBall || b.user == kUserCar)) {
      if (s.n_records >= (uint32_t)kMaxRecords) {
        err = "stored contact records over the cap";
        return false;
      }
      s.records[s.n_records++] = r;
    } else if (a.user == kUserCar) {
      if (a.user_ptr >= (uint32_t)kCars) {
        err = "contact record of a car index outside the arena";
        return false;
      }
      s.fold_events |= 1u << (EV_CAR_HIT_WORLD + a.user_ptr);
      s.fold_car_normal[a.user_ptr] = r.p.normal_b;
    } else if (a.user == kUserBall && b.user == kUserNone) {
      s.fold_events |= 1u << EV_BALL_HIT_WORLD;
      if (fabsf(r.p.normal_b.z) < 0.8f) s.fold_events |= 1u << EV_BALL_WALL;
    }
  }
  return true;
}

// The inverse for writing: records that P7 turns into the same state (dump.rs:424-447) — one ball - world record whose
// normal gives the same two bits, one car - world record per car with its normal, then the stored records.
std::vector<Record> unfold_records(const ArenaState& s, const StaticData& sd) {
  std::vector<Record> out;
  uint32_t world = 0;
  while (world < (uint32_t)kBodies && sd.bodies[world].user != kUserNone) ++world;
  auto rec = [&](uint32_t a, V3 n) {
    Record r;
    memset(&r, 0, sizeof(r));
    r.body_a = a;
    r.body_b = world;
    r.p.normal_b = n;
    return r;
  };
  if (s.fold_events >> EV_BALL_HIT_WORLD & 1u)
    out.push_back(rec(sd.dyn_body[0], (s.fold_events >> EV_BALL_WALL & 1u) ? V3{1.0f, 0.0f, 0.0f} : V3{0.0f, 0.0f, 1.0f}));
  for (int car = 0; car < kCars; ++car)
    if (s.fold_events >> (EV_CAR_HIT_WORLD + car) & 1u) out.push_back(rec(sd.dyn_body[1 + car], s.fold_car_normal[car]));
  for (uint32_t i = 0; i < s.n_records && i < (uint32_t)kMaxRecords; ++i) out.push_back(s.records[i]);
  return out;
}

// The sections after the header (dump.rs:449-848).  On write, `s` must hold its lists within their caps.
template <class IO> void io_arena(IO& io, ArenaState& s, const StaticData& sd, rsx_v3_template& t) {
  constexpr bool R = IO::kRead;
  if (!R) {
    if (s.n_manifolds > (uint32_t)kMaxManifolds || s.n_active > (uint32_t)kMaxActive || s.n_records > (uint32_t)kMaxRecords ||
        s.n_pairs > (uint32_t)kMaxPairs || s.n_dyn_cells > (uint32_t)kMaxDynCells) {
      io.fail("a list of the state is over its cap");
      return;
    }
  }
  // ARNA
  tag(io, "ARNA");
  word64(io, s.tick_count);
  word64(io, s.rng);
  uint32_t ball_only = 0;
  flag(io, ball_only);
  if (R && ball_only) io.fail("a ball-only arena");
  // BALL
  tag(io, "BALL");
  vec3(io, s.ball.pos);
  mat3(io, s.ball.rot);
  vec3(io, s.ball.vel);
  vec3(io, s.ball.ang_vel);
  uint8_t other[24];  // Heatseeker and Dropshot ball info: other modes, kept from the first dump read
  memcpy(other, t.ball_other, 24);
  io.raw(other, 24);
  if (R) {
    if (!t.ball_other_set) {
      memcpy(t.ball_other, other, 24);
      t.ball_other_set = 1;
    } else if (memcmp(other, t.ball_other, 24) != 0) {
      io.fail("Heatseeker or Dropshot ball info changed between dumps");
    }
  }
  word64(io, s.ball.ticks_since_kickoff);
  uint8_t ground_stick = 0;
  io.u8(ground_stick);
  if (R && ground_stick) io.fail("Snowday ground_stick_applied is set");
  // CARS
  tag(io, "CARS");
  if (io.count(kCars) != (size_t)kCars) {
    io.fail("not a 2-car arena");
    return;
  }
  for (int c = 0; c < kCars; ++c) io_car(io, s.cars[c]);
  // PADS
  tag(io, "PADS");
  if (io.count(kPads) != (size_t)kPads) {
    io.fail("not a 34-pad arena");
    return;
  }
  for (int p = 0; p < kPads; ++p) {
    opt_u64(io, s.pad_gave[p]);
    PadTouch& pt = s.pad_touch[p];
    size_t n = io.count(pt.n);
    if (n > (size_t)kCars) {
      io.fail("a pad touched by more cars than the arena has");
      return;
    }
    pt.n = (uint32_t)n;
    for (size_t k = 0; k < n; ++k) io.u32(pt.car[k]);
  }
  // CONT: every record of the tick in call order; the state holds them folded
  tag(io, "CONT");
  std::vector<Record> list;
  if (!R) list = unfold_records(s, sd);
  size_t nrec = io.count(list.size());
  if (R) list.assign(nrec, Record{});
  for (Record& r : list) {
    flag(io, r.swapped);
    io.u32(r.body_a);
    io.u32(r.body_b);
    MPoint p;  // P7 reads the two world points and the normal; V3's other point fields are not kept (zero on write)
    memset(&p, 0, sizeof(p));
    p.world_b = r.p.world_b;
    p.world_a = r.p.world_a;
    p.normal_b = r.p.normal_b;
    io_point(io, p);
    r.p = RecPoint{p.world_b, p.world_a, p.normal_b};
  }
  if (R && io.err.empty()) {
    std::string e;
    if (!fold_records(s, sd, list, e)) {
      s.overflow[OVF_RECORDS] += 1;
      io.fail(e);
      return;
    }
  }
  if (io.count(0) != 0) {  // ball-world records: ball-only arenas only
    io.fail("ball-world contact records present");
    return;
  }
  uint32_t ball_only_tracker = 0;
  flag(io, ball_only_tracker);
  // BODY
  tag(io, "BODY");
  if (io.count(kBodies) != (size_t)kBodies) {
    io.fail("not a 23-body arena");
    return;
  }
  for (int i = 0; i < kBodies; ++i) {
    int d = dyn_slot_of_body(sd, (uint32_t)i);
    if (d >= 0) {
      io_body(io, s.bodies[d]);
    } else if (R) {
      uint8_t rec[kBodyRecord];
      io.raw(rec, kBodyRecord);
      memset(rec + kCompanionAt, 0, 5);
      bool empty = true;  // static bodies never change: keep the first record seen
      for (size_t k = 0; k < kBodyRecord; ++k) empty = empty && t.static_body[i][k] == 0;
      if (empty) memcpy(t.static_body[i], rec, kBodyRecord);
    } else {
      io.raw(t.static_body[i], kBodyRecord);
    }
  }
  // DISP
  tag(io, "DISP");
  size_t nm = io.count(s.n_manifolds);
  if (R) {
    if (nm > (size_t)kMaxManifolds) {
      s.overflow[OVF_MANIFOLDS] += 1;
      io.fail("retained manifolds over the cap");
      return;
    }
    s.n_manifolds = (uint32_t)nm;
  }
  for (size_t i = 0; i < nm; ++i) {
    Manifold& m = s.manifolds[i];
    io.u32(m.body0);
    io.u32(m.body1);
    uint32_t lo = m.body0 < m.body1 ? m.body0 : m.body1, hi = m.body0 < m.body1 ? m.body1 : m.body0;
    uint64_t key = (uint64_t)lo << 32 | hi, got = key;
    io.u64(got);
    if (R && got != key) io.fail("manifold pair_key is not min << 32 | max");
    if (m.body0 >= (uint32_t)kBodies || m.body1 >= (uint32_t)kBodies) {
      io.fail("manifold body index out of range");
      return;
    }
    // the two thresholds are the min over the manifold's two bodies
    const BodyConst& b0 = sd.bodies[m.body0];
    const BodyConst& b1 = sd.bodies[m.body1];
    float cbt = fminf(b0.breaking_threshold, b1.breaking_threshold), cpt = fminf(b0.processing_threshold, b1.processing_threshold);
    float want_cbt = cbt, want_cpt = cpt;
    io.f32(cbt);
    io.f32(cpt);
    if (R && (memcmp(&cbt, &want_cbt, 4) != 0 || memcmp(&cpt, &want_cpt, 4) != 0)) {
      io.fail("a manifold threshold is not the min over its two bodies");
      return;
    }
    io.u32(m.n);
    if (m.n > (uint32_t)kMaxPoints) {
      io.fail("manifold with more than 4 points");
      return;
    }
    for (int k = 0; k < kMaxPoints; ++k) io_point(io, m.pts[k]);
  }
  size_t na = io.count(s.n_active);
  if (R) {
    if (na > (size_t)kMaxActive) {
      s.overflow[OVF_ACTIVE] += 1;
      io.fail("active manifolds over the cap");
      return;
    }
    s.n_active = (uint32_t)na;
  }
  for (size_t i = 0; i < na; ++i) io.u32(s.active[i]);
  // manifold_stride and the manifold table: a search over the pool, validated on read and rebuilt on write
  uint32_t stride = R ? t.manifold_stride : (nm > 0 ? 32u : t.manifold_stride);
  io.u32(stride);
  uint64_t cells = (uint64_t)stride * stride;
  size_t tl = io.count((size_t)cells);
  if (R) t.manifold_stride = stride;
  if (R && (uint64_t)tl != cells) {
    io.fail("manifold table length is not stride squared");
    return;
  }
  std::vector<uint32_t> table(tl, 0u);
  for (size_t i = 0; i < nm; ++i) {
    const Manifold& m = s.manifolds[i];
    uint32_t lo = m.body0 < m.body1 ? m.body0 : m.body1, hi = m.body0 < m.body1 ? m.body1 : m.body0;
    if (hi >= stride) {
      io.fail("manifold body index outside the table");
      return;
    }
    table[(size_t)lo * stride + hi] = (uint32_t)i + 1;
  }
  for (size_t k = 0; k < tl; ++k) {
    uint32_t e = table[k];
    io.u32(e);
    if (R && e != table[k]) {
      io.fail("manifold table is not the search of the pool");
      return;
    }
  }
  // BROA: the dynamic ray-cell lists (cells ascending; each: the cell, its handles in list order)
  tag(io, "BROA");
  if (R) {
    size_t ncells = io.count(0);
    std::vector<DynCell> entries;
    bool have_last = false;
    uint32_t last = 0;
    for (size_t c = 0; c < ncells && io.err.empty(); ++c) {
      uint32_t cell = 0;
      io.u32(cell);
      if (have_last && last >= cell) {
        io.fail("dynamic ray cells not ascending");
        return;
      }
      have_last = true;
      last = cell;
      size_t nh = io.count(0);
      for (size_t k = 0; k < nh && io.err.empty(); ++k) {
        uint32_t h = 0;
        io.u32(h);
        entries.push_back(DynCell{cell, h});
      }
    }
    if (entries.size() > (size_t)kMaxDynCells) {
      s.overflow[OVF_DYN_CELLS] += 1;
      io.fail("dynamic ray-cell entries over the cap");
      return;
    }
    s.n_dyn_cells = (uint32_t)entries.size();
    memset(s.dyn_cells, 0, sizeof(s.dyn_cells));
    for (size_t k = 0; k < entries.size(); ++k) s.dyn_cells[k] = entries[k];
  } else {
    std::vector<std::pair<uint32_t, std::vector<uint32_t>>> groups;
    for (uint32_t k = 0; k < s.n_dyn_cells; ++k) {
      const DynCell& e = s.dyn_cells[k];
      if (!groups.empty() && groups.back().first == e.cell)
        groups.back().second.push_back(e.handle);
      else
        groups.push_back({e.cell, {e.handle}});
    }
    io.count(groups.size());
    for (auto& g : groups) {
      io.u32(g.first);
      io.count(g.second.size());
      for (uint32_t& h : g.second) io.u32(h);
    }
  }
  // sweep-and-prune handles: the static proxies are StaticData.proxies, the dynamic ones are state
  if (io.count(kHandles) != (size_t)kHandles) {
    io.fail("not a 24-handle broadphase");
    return;
  }
  for (int h = 0; h < kHandles; ++h) {
    const ProxyConst& c = sd.proxies[h];
    ProxyConst p = c;
    int d = dyn_slot_of_handle(sd, (uint32_t)h);
    io.u32(p.body);
    uint8_t g = (uint8_t)p.group, m = (uint8_t)p.mask;
    io.u8(g);
    io.u8(m);
    io.u32(p.uid);
    if (d >= 0) {
      DynProxy& dp = s.dyn_proxy[d];
      aabb(io, dp.box);
      io.u32(dp.cell);
      for (int k = 0; k < 3; ++k) io.u32(dp.idx[k]);
    } else {
      ProxyConst tmp = p;
      aabb(io, tmp.box);
      io.u32(tmp.cell);
      for (int k = 0; k < 3; ++k) io.u32(tmp.idx[k]);
      // float == comparisons (a NaN box never matches; -0 matches +0)
      bool same = tmp.box.lo.x == c.box.lo.x && tmp.box.lo.y == c.box.lo.y && tmp.box.lo.z == c.box.lo.z && tmp.box.hi.x == c.box.hi.x &&
                  tmp.box.hi.y == c.box.hi.y && tmp.box.hi.z == c.box.hi.z && tmp.cell == c.cell && tmp.idx[0] == c.idx[0] &&
                  tmp.idx[1] == c.idx[1] && tmp.idx[2] == c.idx[2];
      if (R && !same) {
        io.fail("a static broadphase proxy differs from StaticData.proxies");
        return;
      }
    }
    if (R && (p.body != c.body || g != c.group || m != c.mask || p.uid != c.uid)) {
      io.fail("a broadphase proxy constant differs from StaticData.proxies");
      return;
    }
  }
  if (io.count(kHandles) != (size_t)kHandles) {
    io.fail("handle_edges length");
    return;
  }
  for (int h = 0; h < kHandles; ++h) {
    for (int k = 0; k < 3; ++k) io.u16(s.handle_edges[h].lo[k]);
    for (int k = 0; k < 3; ++k) io.u16(s.handle_edges[h].hi[k]);
  }
  for (int axis = 0; axis < 3; ++axis) {
    if (io.count(kEdges) != (size_t)kEdges) {
      io.fail("edge array length");
      return;
    }
    for (int e = 0; e < kEdges; ++e) {
      io.u16(s.edges[axis][e].pos);
      io.u16(s.edges[axis][e].handle);
    }
  }
  io.u16(t.num_handles);
  if (io.count(0) != 0) {
    io.fail("free_list is not empty");
    return;
  }
  io.u16(t.next_new_handle);
  size_t np = io.count(s.n_pairs);
  if (R) {
    if (np > (size_t)kMaxPairs) {
      s.overflow[OVF_PAIRS] += 1;
      io.fail("retained pairs over the cap");
      return;
    }
    s.n_pairs = (uint32_t)np;
  }
  for (size_t i = 0; i < np; ++i) {
    io.u32(s.pairs[i].h0);
    io.u32(s.pairs[i].h1);
  }
  // pair_indices: the triangular table as a search over the pair array (length: the largest index in use + 1)
  std::vector<std::pair<uint64_t, uint32_t>> want;
  for (size_t i = 0; i < np; ++i) want.push_back({table_index(s.pairs[i].h0, s.pairs[i].h1), (uint32_t)i + 1});
  if (R) {
    size_t len = io.count(0);
    size_t seen = 0;
    for (size_t i = 0; i < len; ++i) {
      uint32_t g = 0;
      io.u32(g);
      if (g == 0) continue;
      ++seen;
      bool found = false;
      for (auto& w : want) found = found || (w.first == i && w.second == g);
      if (!found) {
        io.fail("pair index table is not the search of the pair array");
        return;
      }
    }
    if (seen != np) {
      io.fail("pair index table and pair array disagree");
      return;
    }
  } else {
    uint64_t len = 0;
    for (auto& w : want) len = len > w.first + 1 ? len : w.first + 1;
    io.count((size_t)len);
    std::vector<uint32_t> pt((size_t)len, 0u);
    for (auto& w : want) pt[(size_t)w.first] = w.second;
    for (uint32_t& e : pt) io.u32(e);
  }
}

// ISLD: the island manager's memo of the manifold sort, skipped on read (two u32, two i64, two u32 sequences and a
// bool), written empty (dump.rs:851-866).
template <class IO> void io_island(IO& io) {
  tag(io, "ISLD");
  const size_t width[6] = {4, 4, 8, 8, 4, 4};
  for (int k = 0; k < 6; ++k) {
    size_t n = io.count(0);
    if (IO::kRead && n) {
      std::vector<uint8_t> junk(n * width[k]);
      io.raw(junk.data(), junk.size());
    }
  }
  uint32_t ball_only = 0;
  flag(io, ball_only);
}

// ---- the static traversal (dump.rs:1024-1300); the reference reads only, the writer here is its inverse ----
template <class IO> bool expect_count(IO& io, size_t got, size_t want, const char* what) {
  if (got != want) {
    io.fail(std::string(what) + ": " + std::to_string(got) + ", StaticData holds " + std::to_string(want));
    return false;
  }
  return true;
}

template <class IO> void io_static(IO& io, StaticData& sd) {
  constexpr bool R = IO::kRead;
  // WRLD
  tag(io, "WRLD");
  byte(io, sd.game_mode);
  flag(io, sd.no_ball_rot);
  io.u32(sd.ball_body);
  vec3(io, sd.gravity_uu);
  for (int k = 0; k < kMut; ++k) io.f32(sd.mut[k]);
  flag(io, sd.unlimited_flips);
  flag(io, sd.unlimited_double_jumps);
  flag(io, sd.recharge_boost);
  io.f32(sd.recharge_per_second);
  io.f32(sd.recharge_delay);
  byte(io, sd.demo_mode);
  flag(io, sd.team_demos);
  io.f32(sd.goal_y);
  flag(io, sd.pads_enabled);
  vec3(io, sd.gravity_bt);
  if (!expect_count(io, io.count(kDyn), kDyn, "dynamic bodies")) return;
  for (int d = 0; d < kDyn; ++d) io.u32(sd.dyn_body[d]);
  vec3(io, sd.grid_lo);
  vec3(io, sd.grid_hi);
  io.f32(sd.cell_size);
  io.f32(sd.cell_size_sq);
  for (int k = 0; k < 3; ++k) io.u32(sd.grid_n[k]);
  vec3(io, sd.sap_lo);
  vec3(io, sd.sap_quant);
  uint32_t* sap16[3] = {&sd.sap_mask, &sd.sap_sentinel, &sd.sap_max_handles};
  for (uint32_t* v : sap16) {
    uint16_t x = (uint16_t)*v;
    io.u16(x);
    *v = x;
  }
  io.f32(sd.sap_half_extent);
  // BODY
  tag(io, "BODY");
  if (!expect_count(io, io.count(kBodies), kBodies, "bodies")) return;
  uint32_t mesh_tris[kBodies] = {};
  for (int i = 0; i < kBodies; ++i) {
    BodyConst& b = sd.bodies[i];
    io.u32(b.world_idx);
    byte(io, b.user);
    io.u32(b.user_ptr);
    io.u32(b.handle);
    byte(io, b.group);
    byte(io, b.mask);
    io.f32(b.mass);
    io.f32(b.inv_mass);
    vec3(io, b.inv_inertia_local);
    vec3(io, b.inv_mass3);
    io.f32(b.friction);
    io.f32(b.restitution);
    io.f32(b.processing_threshold);
    io.f32(b.breaking_threshold);
    io.f32(b.lin_damping);
    io.f32(b.lin_sleep);
    io.f32(b.ang_sleep);
    aff3(io, b.pose);
    byte(io, b.shape);
    switch (b.shape) {
      case 0:
        io.u32(b.mesh_tris);
        mesh_tris[i] = b.mesh_tris;
        break;
      case 1:
        break;
      case 2:
        vec3(io, b.sphere_dim);
        io.f32(b.sphere_margin);
        break;
      case 3:
        vec3(io, b.box_half);
        io.f32(b.box_margin);
        aff3(io, b.child);
        aabb(io, b.compound_box);
        break;
      default:
        io.fail("unknown shape kind");
        return;
    }
  }
  for (int d = 0; d < kDyn; ++d) {
    if (sd.dyn_body[d] >= (uint32_t)kBodies) {
      io.fail("dynamic body index out of range");
      return;
    }
    sd.dyn_handle[d] = sd.bodies[sd.dyn_body[d]].handle;
  }
  // MESH
  tag(io, "MESH");
  if (!expect_count(io, io.count(kMeshes), kMeshes, "meshes")) return;
  size_t tf = 0, nf = 0, lf = 0;
  for (int mi_ = 0; mi_ < kMeshes; ++mi_) {
    MeshInfo& mi = sd.meshes[mi_];
    io.u32(mi.body);
    aabb(io, mi.ident_box);
    size_t nt = io.count(mi.tri_count);
    size_t t0 = R ? tf : mi.tri_first;
    if (t0 + nt > (size_t)kMaxTris) {
      io.fail("triangles over the StaticData size");
      return;
    }
    mi.tri_first = (uint32_t)t0;
    mi.tri_count = (uint32_t)nt;
    for (size_t k = 0; k < nt; ++k) {
      Tri& tr = sd.tris[t0 + k];
      vec3(io, tr.p0);
      vec3(io, tr.p1);
      vec3(io, tr.p2);
      vec3(io, tr.n);
    }
    aabb(io, mi.root_box);
    size_t nn = io.count(mi.node_count);
    size_t n0 = R ? nf : mi.node_first;
    if (n0 + nn > (size_t)kMaxNodes) {
      io.fail("BVH nodes over the StaticData size");
      return;
    }
    mi.node_first = (uint32_t)n0;
    mi.node_count = (uint32_t)nn;
    for (size_t k = 0; k < nn; ++k) {
      WideNode& nd = sd.nodes[n0 + k];
      float* lanes[6] = {nd.lo_x, nd.lo_y, nd.lo_z, nd.hi_x, nd.hi_y, nd.hi_z};
      for (float* l : lanes)
        for (int j = 0; j < 4; ++j) io.f32(l[j]);
      for (int j = 0; j < 4; ++j) io.u32(nd.child[j]);
      byte(io, nd.n_child);
      io.u32(nd.valid);
    }
    size_t nl = io.count(mi.leaf_count);
    size_t l0 = R ? lf : mi.leaf_first;
    if (l0 + nl > (size_t)kMaxLeaves) {
      io.fail("BVH leaves over the StaticData size");
      return;
    }
    mi.leaf_first = (uint32_t)l0;
    mi.leaf_count = (uint32_t)nl;
    for (size_t k = 0; k < nl; ++k) {
      aabb(io, sd.leaves[l0 + k].box);
      io.u32(sd.leaves[l0 + k].tri);
    }
    size_t ni = io.count(nt);
    if (ni != nt) {
      io.fail("one triangle info per triangle expected");
      return;
    }
    for (size_t k = 0; k < ni; ++k) {
      TriInfo& inf = sd.infos[t0 + k];
      byte(io, inf.flags);
      io.f32(inf.a01);
      io.f32(inf.a12);
      io.f32(inf.a20);
    }
    tf = t0 + nt;
    nf = n0 + nn;
    lf = l0 + nl;
  }
  if (R && (tf != (size_t)kMaxTris || nf != (size_t)kMaxNodes || lf != (size_t)kMaxLeaves)) {
    io.fail("mesh totals differ from StaticData sizes");
    return;
  }
  for (int k = 0; k < kMeshes; ++k) {
    const MeshInfo& mi = sd.meshes[k];
    if (mi.body >= (uint32_t)kBodies || mi.tri_count != mesh_tris[mi.body]) {
      io.fail("mesh triangle count differs from its body record");
      return;
    }
  }
  // PLAN
  tag(io, "PLAN");
  if (!expect_count(io, io.count(kPlanes), kPlanes, "planes")) return;
  for (int k = 0; k < kPlanes; ++k) {
    Plane& p = sd.planes[k];
    io.u32(p.body);
    vec3(io, p.n);
    flag(io, p.single_axis);
    io.u32(p.axis);
    flag(io, p.backwards);
    aabb(io, p.ident_box);
    aabb(io, p.box);
  }
  // CELL: the static ray-cell lists of the occupied cells, in cell order
  tag(io, "CELL");
  size_t occupied = 0;
  if (!R)
    for (int c = 0; c < kGridCells; ++c) occupied += sd.cells[c].count > 0;
  size_t m = io.count(occupied);
  size_t first = 0;
  int next_cell = 0;
  for (size_t k = 0; k < m; ++k) {
    uint32_t cell = 0, cnt = 0;
    if (!R) {
      while (sd.cells[next_cell].count == 0) ++next_cell;
      cell = (uint32_t)next_cell++;
      cnt = sd.cells[cell].count;
    }
    io.u32(cell);
    io.u32(cnt);
    size_t at = R ? first : sd.cells[cell].first;
    if (cell >= (uint32_t)kGridCells || at + cnt > (size_t)kMaxCellEntries) {
      io.fail("static ray cells over the StaticData size");
      return;
    }
    sd.cells[cell] = CellRange{(uint32_t)at, cnt};
    for (uint32_t j = 0; j < cnt; ++j) io.u32(sd.cell_handles[at + j]);
    first = at + cnt;
  }
  if (R && first != (size_t)kMaxCellEntries) {
    io.fail("static ray-cell entries differ from StaticData size");
    return;
  }
  // CARS
  tag(io, "CARS");
  if (!expect_count(io, io.count(kCars), kCars, "cars")) return;
  for (int c = 0; c < kCars; ++c) {
    CarConst& cc = sd.cars[c];
    io.u32(cc.car_idx);
    byte(io, cc.team);
    io.u32(cc.body);
    flag(io, cc.three_wheels);
    vec3(io, cc.hitbox_size);
    vec3(io, cc.hitbox_offset);
    for (int w = 0; w < kWheels; ++w) {
      vec3(io, cc.wheels[w].connection);
      io.f32(cc.wheels[w].rest_length);
      io.f32(cc.wheels[w].radius);
      io.f32(cc.wheels[w].force_scale);
      io.f32(cc.wheels[w].ray_length);
    }
  }
  // PADS
  tag(io, "PADS");
  if (!expect_count(io, io.count(kPads), kPads, "pads")) return;
  io.f32(sd.max_pad_z);
  for (int p = 0; p < kPads; ++p) {
    PadConst& pc = sd.pads[p];
    vec3(io, pc.pos);
    flag(io, pc.big);
    io.f32(pc.box_radius);
    io.f32(pc.cyl_radius);
    io.f32(pc.cooldown);
    io.f32(pc.amount);
    aabb(io, pc.box);
  }
  // PROX
  tag(io, "PROX");
  if (!expect_count(io, io.count(kHandles), kHandles, "proxies")) return;
  for (int h = 0; h < kHandles; ++h) {
    ProxyConst& p = sd.proxies[h];
    io.u32(p.body);
    byte(io, p.group);
    byte(io, p.mask);
    io.u32(p.uid);
    aabb(io, p.box);
    io.u32(p.cell);
    for (int k = 0; k < 3; ++k) io.u32(p.idx[k]);
  }
}

// ---- whole dumps ----
void put32(std::vector<uint8_t>& o, uint32_t v) { o.insert(o.end(), (uint8_t*)&v, (uint8_t*)&v + 4); }
void put64(std::vector<uint8_t>& o, uint64_t v) { o.insert(o.end(), (uint8_t*)&v, (uint8_t*)&v + 8); }
uint32_t get32(const uint8_t* p) {
  uint32_t v;
  memcpy(&v, p, 4);
  return v;
}
uint64_t get64(const uint8_t* p) {
  uint64_t v;
  memcpy(&v, p, 8);
  return v;
}

// The static dump of sd (the V3 side's export_static layout: sections WRLD BODY MESH PLAN CELL CARS PADS PROX) and
// its config hash: FNV-1a over the sections other than MESH, CELL and PROX, tags and counts included.
bool write_static(const StaticData& sd_in, std::vector<uint8_t>& out, uint64_t* config_hash, std::string& err) {
  StaticData* sd = new StaticData(sd_in);
  Writer w;
  io_static(w, *sd);
  uint32_t counts[12] = {(uint32_t)kBodies, (uint32_t)kDyn, (uint32_t)kMeshes, 0, 0, 0, 0, (uint32_t)kPlanes, (uint32_t)kCars,
                         (uint32_t)kPads, (uint32_t)kGridCells, 0};
  for (int m = 0; m < kMeshes; ++m) {
    counts[3] += sd->meshes[m].tri_count;
    counts[4] += sd->meshes[m].node_count;
    counts[5] += sd->meshes[m].leaf_count;
    counts[6] += sd->meshes[m].tri_count;
  }
  for (int c = 0; c < kGridCells; ++c) counts[11] += sd->cells[c].count;
  delete sd;
  if (!w.err.empty()) {
    err = w.err;
    return false;
  }
  if (config_hash) {
    // sections in file order: WRLD BODY MESH PLAN CELL CARS PADS PROX
    std::vector<uint8_t> cfg;
    const int keep[5] = {0, 1, 3, 5, 6};
    for (int k : keep) {
      size_t a = w.marks[k], b = (size_t)k + 1 < w.marks.size() ? w.marks[k + 1] : w.buf.size();
      cfg.insert(cfg.end(), w.buf.begin() + a, w.buf.begin() + b);
    }
    *config_hash = fnv1a64(cfg.data(), cfg.size());
  }
  out.clear();
  out.insert(out.end(), kStaticMagic, kStaticMagic + 8);
  put32(out, kStaticVersion);
  put64(out, fnv1a64(w.buf.data(), w.buf.size()));
  put64(out, (uint64_t)w.buf.size());
  for (uint32_t c : counts) put32(out, c);
  out.insert(out.end(), w.buf.begin(), w.buf.end());
  return true;
}

// parse_static (dump.rs:947-1012).  table_sin is filled by this project's correctly rounded generator, the one every
// StaticData here uses (the reference fills it with the importing platform's f64 sin).
bool parse_static(const uint8_t* bytes, size_t len, StaticData& sd, std::string& err) {
  if (len < kStaticHeader || memcmp(bytes, kStaticMagic, 8) != 0) {
    err = "not a static dump (magic)";
    return false;
  }
  uint32_t version = get32(bytes + 8);
  if (version != kStaticVersion) {
    err = "unsupported static dump version " + std::to_string(version) + " (need 3: re-vendor V3)";
    return false;
  }
  uint64_t hash = get64(bytes + 12), plen = get64(bytes + 20);
  if (plen != (uint64_t)(len - kStaticHeader)) {
    err = "static dump payload length mismatch";
    return false;
  }
  if (fnv1a64(bytes + kStaticHeader, len - kStaticHeader) != hash) {
    err = "static dump payload hash mismatch";
    return false;
  }
  const uint32_t want[12] = {(uint32_t)kBodies, (uint32_t)kDyn, (uint32_t)kMeshes, (uint32_t)kMaxTris, (uint32_t)kMaxNodes,
                             (uint32_t)kMaxLeaves, (uint32_t)kMaxTris, (uint32_t)kPlanes, (uint32_t)kCars, (uint32_t)kPads,
                             (uint32_t)kGridCells, (uint32_t)kMaxCellEntries};
  for (int i = 0; i < 12; ++i) {
    uint32_t got = get32(bytes + 28 + 4 * i);
    if (got != want[i]) {
      err = "static dump count " + std::to_string(i) + " is " + std::to_string(got) + "; StaticData is sized for " +
            std::to_string(want[i]) + " (the project's 16 Soccar meshes)";
      return false;
    }
  }
  memset(&sd, 0, sizeof(sd));
  Reader r(bytes + kStaticHeader, len - kStaticHeader);
  io_static(r, sd);
  if (!r.err.empty()) {
    err = r.err;
    return false;
  }
  for (int i = 0; i < kTableSin; ++i) sd.table_sin[i] = sim::table_sin_value(i);
  if (r.remaining() != 0) {
    err = std::to_string(r.remaining()) + " trailing bytes in the static dump";
    return false;
  }
  return true;
}

bool parse_arena(const uint8_t* bytes, size_t len, const StaticData& sd, ArenaState& s, rsx_v3_template& t, std::string& err) {
  if (len < kArenaHeader || memcmp(bytes, kArenaMagic, 8) != 0) {
    err = "not an arena dump (magic)";
    return false;
  }
  uint32_t version = get32(bytes + 8);
  if (version != kArenaVersion) {
    err = "unsupported arena dump version " + std::to_string(version);
    return false;
  }
  memset(&s, 0, sizeof(s));
  memset(&t, 0, sizeof(t));
  t.config_hash = get64(bytes + 12);
  Reader r(bytes + kArenaHeader, len - kArenaHeader);
  io_arena(r, s, sd, t);
  if (r.err.empty()) io_island(r);
  if (!r.err.empty()) {
    err = r.err;
    return false;
  }
  if (r.remaining() != 0) {
    err = std::to_string(r.remaining()) + " trailing bytes";
    return false;
  }
  return true;
}

bool write_arena(const ArenaState& s_in, const StaticData& sd, const rsx_v3_template& t_in, std::vector<uint8_t>& out, std::string& err) {
  ArenaState s = s_in;
  rsx_v3_template t = t_in;
  Writer w;
  io_arena(w, s, sd, t);
  if (w.err.empty()) io_island(w);
  if (!w.err.empty()) {
    err = w.err;
    return false;
  }
  uint32_t points = 0;
  for (uint32_t i = 0; i < s.n_manifolds; ++i) points += s.manifolds[i].n;
  uint32_t stride = s.n_manifolds > 0 ? 32u : t.manifold_stride;
  const uint32_t counts[12] = {(uint32_t)kBodies, s.n_manifolds, s.n_active, points, stride * stride, (uint32_t)kHandles, s.n_pairs,
                               s.n_dyn_cells, (uint32_t)kCars, (uint32_t)kPads, (uint32_t)unfold_records(s, sd).size(), 0u};
  out.clear();
  out.insert(out.end(), kArenaMagic, kArenaMagic + 8);
  put32(out, kArenaVersion);
  put64(out, t.config_hash);
  for (uint32_t c : counts) put32(out, c);
  out.insert(out.end(), w.buf.begin(), w.buf.end());
  return true;
}

// A template for a StaticData that has no V3 dump (the synthetic world): the config hash of its static dump, and for
// each static body the BODY record V3 would hold for an unmoving body — collision flags 1 (static object), activation
// 0, the body's pose as both transforms, the identity quaternion, zero velocities, inertia and damping caches.  The
// broadphase counters are those of 23 bodies added once (num_handles 23, next_new_handle 24); no manifold table.
bool make_template(const StaticData& sd, rsx_v3_template& t, std::string& err) {
  memset(&t, 0, sizeof(t));
  std::vector<uint8_t> dump;
  if (!write_static(sd, dump, &t.config_hash, err)) return false;
  for (int i = 0; i < kBodies; ++i) {
    if (dyn_slot_of_body(sd, (uint32_t)i) >= 0) continue;
    const Aff& pose = sd.bodies[i].pose;
    const M3& r = pose.m;
    bool unrotated = r.c0.x == 1.0f && r.c0.y == 0.0f && r.c0.z == 0.0f && r.c1.x == 0.0f && r.c1.y == 1.0f && r.c1.z == 0.0f &&
                     r.c2.x == 0.0f && r.c2.y == 0.0f && r.c2.z == 1.0f;
    if (!unrotated) {
      err = "a static body with a rotated pose: take the template from a V3 dump";
      return false;
    }
    Body b;
    memset(&b, 0, sizeof(b));
    b.flags = 1;
    b.xf = pose;
    b.pred = pose;
    b.quat = Q4{0.0f, 0.0f, 0.0f, 1.0f};
    Writer w;
    io_body(w, b);
    memcpy(t.static_body[i], w.buf.data(), kBodyRecord);
  }
  t.num_handles = (uint16_t)(kHandles - 1);
  t.next_new_handle = (uint16_t)kHandles;
  t.manifold_stride = 0;
  t.ball_other_set = 1;
  return true;
}

int copy_out(const std::vector<uint8_t>& v, uint8_t* out, size_t cap, size_t* len) {
  if (len) *len = v.size();
  if (!out || cap < v.size()) return rsx_set_last_error(RSX_E_ARG, "output buffer too short (its size is in *len)");
  memcpy(out, v.data(), v.size());
  return RSX_OK;
}

}  // namespace v3dump
}  // namespace rsx

using namespace rsx;

extern "C" {

uint64_t rsx_v3_fnv1a64(const uint8_t* bytes, size_t len) { return v3dump::fnv1a64(bytes, len); }

int rsx_v3_parse_static(const uint8_t* bytes, size_t len, uint32_t* sd_words) {
  if (!bytes || !sd_words) return rsx_set_last_error(RSX_E_ARG, "rsx_v3_parse_static: null buffer");
  StaticData* sd = new StaticData;
  std::string err;
  bool ok = v3dump::parse_static(bytes, len, *sd, err);
  if (ok) memcpy(sd_words, sd, sizeof(StaticData));
  delete sd;
  return ok ? RSX_OK : rsx_set_last_error(RSX_E_FORMAT, err.c_str());
}

int rsx_v3_write_static(const uint32_t* sd_words, uint8_t* out, size_t cap, size_t* len) {
  if (!sd_words || !len) return rsx_set_last_error(RSX_E_ARG, "rsx_v3_write_static: null argument");
  std::vector<uint8_t> v;
  std::string err;
  if (!v3dump::write_static(*reinterpret_cast<const StaticData*>(sd_words), v, nullptr, err)) return rsx_set_last_error(RSX_E_FORMAT, err.c_str());
  return v3dump::copy_out(v, out, cap, len);
}

int rsx_v3_config_hash(const uint32_t* sd_words, uint64_t* hash) {
  if (!sd_words || !hash) return rsx_set_last_error(RSX_E_ARG, "rsx_v3_config_hash: null argument");
  std::vector<uint8_t> v;
  std::string err;
  if (!v3dump::write_static(*reinterpret_cast<const StaticData*>(sd_words), v, hash, err)) return rsx_set_last_error(RSX_E_FORMAT, err.c_str());
  return RSX_OK;
}

int rsx_v3_template_init(const uint32_t* sd_words, rsx_v3_template* t) {
  if (!sd_words || !t) return rsx_set_last_error(RSX_E_ARG, "rsx_v3_template_init: null argument");
  std::string err;
  if (!v3dump::make_template(*reinterpret_cast<const StaticData*>(sd_words), *t, err)) return rsx_set_last_error(RSX_E_FORMAT, err.c_str());
  return RSX_OK;
}

int rsx_v3_parse_arena(const uint8_t* bytes, size_t len, const uint32_t* sd_words, uint32_t* state_words, rsx_v3_template* t) {
  if (!bytes || !sd_words || !state_words || !t) return rsx_set_last_error(RSX_E_ARG, "rsx_v3_parse_arena: null argument");
  ArenaState s;
  rsx_v3_template tt;
  std::string err;
  if (!v3dump::parse_arena(bytes, len, *reinterpret_cast<const StaticData*>(sd_words), s, tt, err)) return rsx_set_last_error(RSX_E_FORMAT, err.c_str());
  memcpy(state_words, &s, sizeof(s));
  *t = tt;
  return RSX_OK;
}

int rsx_v3_write_arena(const uint32_t* state_words, const uint32_t* sd_words, const rsx_v3_template* t, uint8_t* out, size_t cap,
                       size_t* len) {
  if (!state_words || !sd_words || !t || !len) return rsx_set_last_error(RSX_E_ARG, "rsx_v3_write_arena: null argument");
  std::vector<uint8_t> v;
  std::string err;
  if (!v3dump::write_arena(*reinterpret_cast<const ArenaState*>(state_words), *reinterpret_cast<const StaticData*>(sd_words), *t, v, err))
    return rsx_set_last_error(RSX_E_FORMAT, err.c_str());
  return v3dump::copy_out(v, out, cap, len);
}

}  // extern "C"
