// P3b: the narrowphase over the retained broadphase pairs in pair order.  Reference: cuda/sim/collision_dispatcher.cuh
// (near callback, manifold pool), persistent_manifold.cuh, arena_contact_tracker.cuh (records and folded events),
// internal_edge_utility.cuh, convex_plane_collision_alg.cuh, sphere_obb_collision_alg.cuh, obb_obb_collision_alg.cuh,
// sphere_concave_collision_alg.cuh + triangle_shape.cuh (ball vs mesh), compound_collision_alg.cuh (car vs mesh).
// A mesh pair walks its BVH leaf by leaf and adds each leaf's contact in traversal order, which is V3's order.
#pragma once
#include "broad.cuh"
#include "sat.cuh"

namespace rsx {
namespace sim {

struct Ctx {
  ArenaState& S;
  const StaticData& D;
  uint32_t unimplemented;
};

// ---- manifolds ----
RSX_F Manifold manifold_new(uint32_t b0, uint32_t b1) {
  Manifold m = {};
  m.body0 = b0;
  m.body1 = b1;
  return m;
}
RSX_F float breaking(const StaticData& D, const Manifold& m) {
  return rmin(D.bodies[m.body0].breaking_threshold, D.bodies[m.body1].breaking_threshold);
}
RSX_F void point_swap_remove(Manifold& m, uint32_t i) {
  uint32_t last = m.n - 1;
  if (i != last) m.pts[i] = m.pts[last];
  m.pts[last] = MPoint{};
  m.n = last;
}
RSX_F float res_area(V3 p, V3 a, V3 b, V3 c) { return len2(cross(p - a, b - c)); }
RSX_F uint32_t replace_slot(const Manifold& m, const MPoint& np) {
  uint32_t deepest = kMaxPoints;
  float md = np.dist;
  for (uint32_t i = 0; i < m.n; ++i)
    if (m.pts[i].dist < md) {
      deepest = i;
      md = m.pts[i].dist;
    }
  V3 p = np.local_a;
  const MPoint* c = m.pts;
  V4 r;
  r.x = deepest == 0 ? 0.0f : res_area(p, c[1].local_a, c[3].local_a, c[2].local_a);
  r.y = deepest == 1 ? 0.0f : res_area(p, c[0].local_a, c[3].local_a, c[2].local_a);
  r.z = deepest == 2 ? 0.0f : res_area(p, c[0].local_a, c[3].local_a, c[1].local_a);
  r.w = deepest == 3 ? 0.0f : res_area(p, c[0].local_a, c[2].local_a, c[1].local_a);
  uint32_t best = 0;
  float ma = r.x;
  if (r.y > ma) { best = 1; ma = r.y; }
  if (r.z > ma) { best = 2; ma = r.z; }
  if (r.w > ma) best = 3;
  return best;
}
RSX_F int32_t cache_entry(const StaticData& D, const Manifold& m, const MPoint& np) {
  float t = breaking(D, m);
  float shortest = fmul(t, t);
  int32_t near = -1;
  for (uint32_t i = 0; i < m.n; ++i) {
    float d2 = len2(m.pts[i].local_a - np.local_a);
    if (d2 < shortest) {
      shortest = d2;
      near = (int32_t)i;
    }
  }
  return near;
}
RSX_F uint32_t add_point_nocb(const StaticData& D, Manifold& m, const MPoint& np) {
  int32_t at = cache_entry(D, m, np);
  if (at >= 0) {
    m.pts[at] = np;
    return (uint32_t)at;
  }
  if (m.n == (uint32_t)kMaxPoints) {
    uint32_t i = replace_slot(m, np);
    m.pts[i] = np;
    return i;
  }
  m.pts[m.n] = np;
  return m.n++;
}
RSX_HD RSX_NOINL inline void refresh_points(const ArenaState& S, const StaticData& D, Manifold& m, uint32_t b0, uint32_t b1) {
  if (m.n == 0) return;
  Aff ta = body_xf(S, D, b0), tb = body_xf(S, D, b1);
  for (uint32_t i = 0; i < m.n; ++i) {
    MPoint& p = m.pts[i];
    p.world_a = xform_point(ta, p.local_a);
    p.world_b = xform_point(tb, p.local_b);
    p.dist = dot(p.world_a - p.world_b, p.normal_b);
  }
  float cbt = breaking(D, m);
  float cbt2 = fmul(cbt, cbt);
  for (int32_t i = (int32_t)m.n - 1; i >= 0; --i) {
    MPoint p = m.pts[i];
    if (p.dist > cbt) {
      point_swap_remove(m, (uint32_t)i);
      continue;
    }
    V3 proj = p.world_a - p.normal_b * p.dist;
    V3 diff = p.world_b - proj;
    if (dot(diff, diff) > cbt2) point_swap_remove(m, (uint32_t)i);
  }
}
RSX_HD RSX_NOINL inline void merge_points(const StaticData& D, Manifold& m, const Manifold& o) {
  if (m.n == 0) {
    for (uint32_t i = 0; i < o.n; ++i) m.pts[m.n++] = o.pts[i];
  } else {
    for (uint32_t i = 0; i < o.n; ++i) add_point_nocb(D, m, o.pts[i]);
  }
}

// ---- the contact tracker: car-ball / car-car records in call order; world contacts folded into bits ----
RSX_F bool tracker_swap(const StaticData& D, uint32_t a, uint32_t b) {
  uint32_t ua = D.bodies[a].user, ub = D.bodies[b].user;
  return (ua != USER_NONE && ub != USER_NONE) ? ua > ub : ub != USER_NONE;
}
RSX_F void push_record(Ctx& c, bool swapped, uint32_t a, uint32_t b, const MPoint& p) {
  ArenaState& S = c.S;
  const BodyConst& ba = c.D.bodies[a];
  const BodyConst& bb = c.D.bodies[b];
  if (ba.user == USER_CAR) {
    if (bb.user != USER_BALL && bb.user != USER_CAR) {
      uint32_t car = ba.user_ptr;
      S.fold_events |= 1u << (EV_CAR_HIT_WORLD + car);
      S.fold_car_normal[car] = p.normal_b;
      return;
    }
  } else if (ba.user == USER_BALL && bb.user == USER_NONE) {
    S.fold_events |= 1u << EV_BALL_HIT_WORLD;
    if (fabs_(p.normal_b.z) < 0.8f) S.fold_events |= 1u << EV_BALL_WALL;
    return;
  } else {
    return;
  }
  if (S.n_records >= (uint32_t)kMaxRecords) {
    S.overflow[OVF_RECORDS] += 1;
    return;
  }
  Record& r = S.records[S.n_records++];
  r.swapped = swapped ? 1u : 0u;
  r.body_a = a;
  r.body_b = b;
  r.p.world_b = p.world_b;
  r.p.world_a = p.world_a;
  r.p.normal_b = p.normal_b;
}

// ---- internal-edge fix of a mesh contact (Bullet's btAdjustInternalEdgeContacts) ----
RSX_F float edge_angle(V3 ea, V3 na, V3 nb) { return cr_atan2(dot(nb, ea), dot(nb, na)); }
RSX_F V3 nearest_on_line(V3 p, V3 l0, V3 l1) {
  V3 ld = l1 - l0;
  if (len2(ld) < fmul(kEps, kEps)) return l0;
  float d = fdiv(dot(p - l0, ld), dot(ld, ld));
  return l0 + ld * rclamp(d, from_bits(0x3727c5acu), from_bits(0x3f7fff58u));
}
RSX_F bool clamp_normal(V3 edge, V3 tn, V3 ln, float corrected, V3* out) {
  V3 ec = normalize(cross(edge, tn));
  float cur = edge_angle(ec, tn, ln);
  if ((corrected < 0.0f && cur < corrected) || (corrected >= 0.0f && cur > corrected)) {
    float da = fsub(corrected, cur);
    float s, co;
    cr_sincos(fmul(da, 0.5f), &s, &co);
    V3 v = normalize(edge) * vs(s);
    *out = qrotate(Q4{v.x, v.y, v.z, co}, ln);
    return true;
  }
  return false;
}
RSX_F V3 tri_edge_vec(const Tri& t, int i) { return i == 0 ? t.p1 - t.p0 : (i == 1 ? t.p2 - t.p1 : t.p0 - t.p2); }
RSX_HD RSX_NOINL inline void edge_block(MPoint* cp, const Aff& mt, const Tri& tri, int edge_no, float angle, uint32_t flags, uint32_t cflag, uint32_t sflag,
                      V3 lcn, bool recompute, bool* concave) {
  if (angle == 0.0f) {
    *concave = true;
    return;
  }
  bool convex = (flags & cflag) != 0;
  float swf = fsub(fmul(convex ? 1.0f : 0.0f, 2.0f), 1.0f);
  V3 edge = -tri_edge_vec(tri, edge_no);
  V3 na = vs(swf) * tri.n;
  float s, co;
  cr_sincos(fmul(angle, 0.5f), &s, &co);
  V3 axs = normalize(edge) * vs(s);
  V3 cnb = qrotate(Q4{axs.x, axs.y, axs.z, co}, tri.n);
  if (flags & sflag) cnb *= -1.0f;
  V3 nb = vs(swf) * cnb;
  float da = dot(lcn, na), db = dot(lcn, nb);
  if (da < 0.0f && db < 0.0f) {
    *concave = true;
    return;
  }
  V3 ln = recompute ? mul_t(mt.m, cp->normal_b) : lcn;
  V3 cl;
  if (clamp_normal(edge, vs(swf) * tri.n, ln, angle, &cl) && dot(cl, tri.n) > 0.0f) {
    V3 nn = mt.m * cl;
    cp->normal_b = nn;
    cp->world_b = cp->world_a - nn * cp->dist;
    cp->local_b = inv_xform(mt, cp->world_b);
  }
}
RSX_HD RSX_NOINL inline void adjust_internal_edge(const StaticData& D, MPoint* cp, uint32_t mesh_body, uint32_t idx) {
  const MeshInfo& mesh = D.meshes[mesh_body];
  const TriInfo& info = D.infos[mesh.tri_first + idx];
  const Tri& tri = D.tris[mesh.tri_first + idx];
  Aff mt = D.bodies[mesh_body].pose;
  V3 nearest = nearest_on_line(cp->local_b, tri.p0, tri.p1);
  V3 contact = cp->local_b;
  V3 lcn = mul_t(mt.m, cp->normal_b);
  int best = 0;
  float dx = kFltMax, dy = kFltMax, dz = kFltMax, dbest = kFltMax;
  if (fabs_(info.a01) < kTau) {
    dx = len(contact - nearest);
    if (dx < dbest) { best = 1; dbest = dx; }
  }
  if (fabs_(info.a12) < kTau) {
    dy = len(contact - nearest_on_line(cp->local_b, tri.p1, tri.p2));
    if (dy < dbest || (dy == dbest && info.a12 != 0.0f && (info.flags & 2u) == 0)) { best = 2; dbest = dy; }
  }
  if (fabs_(info.a20) < kTau) {
    dz = len(contact - nearest_on_line(cp->local_b, tri.p2, tri.p0));
    if (dz < dbest || (dz == dbest && info.a20 != 0.0f)) best = 3;
  }
  bool processed = false, concave = false;
  if (fabs_(info.a01) < kTau && dx < 0.1f && (best == 1 || (dx < kEps && info.a01 != 0.0f))) {
    processed = true;
    edge_block(cp, mt, tri, 0, info.a01, info.flags, 1u, 8u, lcn, false, &concave);
  }
  if (fabs_(info.a12) < kTau && dy < 0.1f && (best == 2 || (dy < kEps && info.a12 != 0.0f))) {
    processed = true;
    edge_block(cp, mt, tri, 1, info.a12, info.flags, 2u, 16u, lcn, true, &concave);
  }
  if (fabs_(info.a20) < kTau && dz < 0.1f && (best == 3 || (dz < kEps && info.a20 != 0.0f))) {
    processed = true;
    edge_block(cp, mt, tri, 2, info.a20, info.flags, 4u, 32u, lcn, true, &concave);
  }
  if (!processed || !concave) return;
  if (dot(tri.n, lcn) < 0.0f) return;
  cp->normal_b = mt.m * tri.n;
  cp->world_b = cp->world_a - cp->normal_b * cp->dist;
  cp->local_b = inv_xform(mt, cp->world_b);
}

RSX_F void tracker_added(Ctx& c, MPoint* mp, uint32_t a, uint32_t b, int32_t idx) {
  bool sw = tracker_swap(c.D, a, b);
  if (sw) {
    uint32_t t = a;
    a = b;
    b = t;
  }
  uint32_t ua = c.D.bodies[a].user, ub = c.D.bodies[b].user;
  if (ua == USER_CAR) {
    if (ub == USER_BALL) {
      mp->friction = 2.0f;
      mp->restitution = 0.0f;
    } else if (ub == USER_CAR) {
      mp->friction = 0.09f;
      mp->restitution = 0.1f;
    } else {
      mp->friction = 0.3f;
      mp->restitution = 0.3f;
    }
  } else if (ua == USER_BALL && ub == USER_NONE && body_static(c.S, c.D, b)) {
    mp->special = 1;
  }
  push_record(c, sw, a, b, *mp);
  if (idx >= 0) adjust_internal_edge(c.D, mp, b, (uint32_t)idx);
}
RSX_F void tracker_retained(Ctx& c, const MPoint& mp, uint32_t a, uint32_t b) {
  bool sw = tracker_swap(c.D, a, b);
  if (sw) {
    uint32_t t = a;
    a = b;
    b = t;
  }
  uint32_t ua = c.D.bodies[a].user, ub = c.D.bodies[b].user;
  if (ua != USER_CAR || ub == USER_BALL || ub == USER_CAR) return;
  push_record(c, sw, a, b, mp);
}

// add_contact_point: a new point of the pair (body0, body1) into manifold m, with the tracker's callback
RSX_HD RSX_NOINL inline void add_contact(Ctx& c, Manifold& m, uint32_t b0, uint32_t b1, V3 n_b, V3 p_world, float depth, int32_t idx) {
  if (depth > breaking(c.D, m)) return;
  V3 pa = p_world + n_b * depth;
  MPoint np = {};
  np.local_a = inv_xform(body_xf(c.S, c.D, b0), pa);
  np.local_b = inv_xform(body_xf(c.S, c.D, b1), p_world);
  np.normal_b = n_b;
  np.dist = depth;
  np.world_a = pa;
  np.world_b = p_world;
  bool st = body_static(c.S, c.D, b0) || body_static(c.S, c.D, b1);
  float f0 = c.D.bodies[b0].friction, f1 = c.D.bodies[b1].friction;
  float r0 = c.D.bodies[b0].restitution, r1 = c.D.bodies[b1].restitution;
  np.friction = st ? rmin(f0, f1) : fmul(f0, f1);
  np.restitution = st ? rmax(r0, r1) : fmul(r0, r1);
  uint32_t at = add_point_nocb(c.D, m, np);
  if ((body_flags(c.S, c.D, b0) & CF_CUSTOM) || (body_flags(c.S, c.D, b1) & CF_CUSTOM)) tracker_added(c, &m.pts[at], b0, b1, idx);
}

// ---- convex (ball sphere or car box child) against a plane ----
RSX_HD RSX_NOINL inline bool alg_convex_plane(Ctx& c, uint32_t obj, uint32_t plane_obj, const Aff& wt, bool box, Manifold* out) {
  const Plane& pl = c.D.planes[plane_obj - kMeshes];
  const BodyConst& bc = c.D.bodies[obj];
  Box3 cb = box ? box_from_half(bc.box_half, bc.box_margin, wt) : sphere_box(bc.sphere_margin, wt.t);
  if (!box_overlap(cb, pl.box)) return false;
  V3 pn = pl.n;
  Aff pt = body_xf(c.S, c.D, plane_obj);
  M3 pic = transpose(wt.m);
  V3 dir = pic * (-pn);
  V3 vtx;
  if (box) {
    V3 sg = {dir.x < 0.0f ? -1.0f : 1.0f, dir.y < 0.0f ? -1.0f : 1.0f, dir.z < 0.0f ? -1.0f : 1.0f};
    vtx = add_s(bc.box_half, bc.box_margin) * sg;
  } else {
    V3 n;
    try_normalize(dir, &n);
    vtx = vs(bc.sphere_margin) * n;
  }
  V3 vp = xform_point(Aff{wt.m, wt.t - pt.t}, vtx);
  float dist = dot(pn, vp);
  Manifold m = manifold_new(obj, plane_obj);
  if (dist >= breaking(c.D, m)) return false;
  V3 proj = vp - vs(dist) * pn;
  add_contact(c, m, obj, plane_obj, pn, proj + pt.t, dist, -1);
  refresh_points(c.S, c.D, m, obj, plane_obj);
  *out = m;
  return true;
}

// ---- ball against a car box ----
RSX_HD RSX_NOINL inline bool alg_sphere_box(Ctx& c, uint32_t sph, uint32_t car, Manifold* out) {
  Aff st = body_xf(c.S, c.D, sph);
  float radius = c.D.bodies[sph].sphere_margin;
  if (!box_overlap(sphere_box(radius, st.t), body_box(c.S, c.D, car))) return false;
  Aff cw = child_xf(c.S, c.D, car);
  const BodyConst& bx = c.D.bodies[car];
  V3 ext = bx.box_half;
  V3 local = inv_xform(cw, st.t);
  V3 closest = vclamp(local, -ext, ext);
  V3 delta = local - closest;
  float d2 = len2(delta);
  Manifold m = manifold_new(sph, car);
  float inter = fadd(radius, bx.box_margin);
  float cdist = fadd(inter, breaking(c.D, m));
  if (d2 > fmul(cdist, cdist)) return false;
  float dist;
  if (d2 > kEps) {
    dist = fsqrt(d2);
    delta = delta / dist;
  } else {
    // inside: the nearest face, in V3's face order (+x, -x, +y, -y, +z, -z)
    float md = fsub(ext.x, local.x);
    V3 cl = local;
    cl.x = ext.x;
    V3 nn = {1.0f, 0.0f, 0.0f};
    const int axes[5] = {0, 1, 1, 2, 2};
    const float sgn[5] = {-1.0f, 1.0f, -1.0f, 1.0f, -1.0f};
    for (int t = 0; t < 5; ++t) {
      int ax = axes[t];
      float fd = sgn[t] < 0.0f ? fadd(comp(ext, ax), comp(local, ax)) : fsub(comp(ext, ax), comp(local, ax));
      if (fd < md) {
        md = fd;
        cl = local;
        set_comp(cl, ax, fmul(comp(ext, ax), sgn[t]));
        nn = vzero();
        set_comp(nn, ax, sgn[t]);
      }
    }
    dist = fmul(md, -1.0f);
    closest = cl;
    delta = nn;
  }
  V3 nbox = cw.m * delta;
  V3 pbox = xform_point(cw, closest);
  float depth = fsub(dist, inter);
  add_contact(c, m, sph, car, nbox, pbox + nbox * bx.box_margin, depth, -1);
  refresh_points(c.S, c.D, m, sph, car);
  if (m.n == 0) return false;
  *out = m;
  return true;
}

// ---- car box against car box (Bullet's box-box detector) ----
struct Obb { V3 c; M3 ax; V3 ext; };
struct BbHit { float depth; V3 n; uint32_t code; };
struct Poly16 { float p[16][2]; uint32_t n; };

RSX_F float line_closest(V3 pa, V3 ua, V3 pb, V3 ub) {
  V3 p = pb - pa;
  float uaub = dot(ua, ub), q1 = dot(ua, p), q2 = fneg(dot(ub, p));
  float d = fsub(1.0f, fmul(uaub, uaub));
  if (d <= 0.0001f) return 0.0f;
  return fdiv(fadd(fmul(uaub, q1), q2), d);
}
RSX_NOINL RSX_HD inline void clip_rect_quad(const float h[2], const float quad[4][2], Poly16* res) {
  Poly16 q;
  q.n = 4;
  for (int i = 0; i < 4; ++i) {
    q.p[i][0] = quad[i][0];
    q.p[i][1] = quad[i][1];
  }
  for (int dir = 0; dir < 2; ++dir)
    for (int si = 0; si < 2; ++si) {
      float sg = si == 0 ? -1.0f : 1.0f;
      Poly16 r;
      r.n = 0;
      float cv = fmul(sg, h[dir]);
      uint32_t n = q.n;
      for (uint32_t i = 0; i < n; ++i) {
        const float* cur = q.p[i];
        const float* nx = q.p[(i + 1) % n];
        bool in_c = fmul(sg, cur[dir]) < h[dir];
        if (in_c) {
          r.p[r.n][0] = cur[0];
          r.p[r.n][1] = cur[1];
          r.n++;
        }
        bool in_n = fmul(sg, nx[dir]) < h[dir];
        if (in_c != in_n) {
          float p = fadd(cur[1 - dir], fmul(fdiv(fsub(nx[1 - dir], cur[1 - dir]), fsub(nx[dir], cur[dir])), fsub(cv, cur[dir])));
          float p1 = p, p2 = cv;
          if (dir == 0) {
            float t = p1;
            p1 = p2;
            p2 = t;
          }
          r.p[r.n][0] = p1;
          r.p[r.n][1] = p2;
          r.n++;
        }
      }
      q = r;
    }
  *res = q;
}
RSX_NOINL RSX_HD inline void cull_points(const float p[][2], uint32_t n, uint32_t i0, uint32_t m, uint32_t* res) {
  float cx, cy;
  if (n == 1) {
    cx = p[0][0];
    cy = p[0][1];
  } else if (n == 2) {
    cx = fmul(fadd(p[0][0], p[1][0]), 0.5f);
    cy = fmul(fadd(p[0][1], p[1][1]), 0.5f);
  } else {
    float as = 0.0f, xs = 0.0f, ys = 0.0f;
    for (uint32_t i = 0; i + 1 < n; ++i) {
      float x0 = p[i][0], y0 = p[i][1], x1 = p[i + 1][0], y1 = p[i + 1][1];
      float q = fsub(fmul(x0, y1), fmul(x1, y0));
      as = fadd(as, q);
      xs = fadd(xs, fmul(q, fadd(x0, x1)));
      ys = fadd(ys, fmul(q, fadd(y0, y1)));
    }
    float xl = p[n - 1][0], yl = p[n - 1][1], x0 = p[0][0], y0 = p[0][1];
    float ql = fsub(fmul(xl, y0), fmul(x0, yl));
    float area = fadd(as, ql);
    float inv = fabs_(area) > kEps ? fdiv(1.0f, fmul(3.0f, area)) : 1e18f;
    cx = fmul(inv, fadd(xs, fmul(ql, fadd(xl, x0))));
    cy = fmul(inv, fadd(ys, fmul(ql, fadd(yl, y0))));
  }
  float ang[8];
  for (uint32_t i = 0; i < n; ++i) ang[i] = cr_atan2(fsub(p[i][1], cy), fsub(p[i][0], cx));
  bool avail[8] = {false, false, false, false, false, false, false, false};
  for (uint32_t i = 0; i < n; ++i) avail[i] = true;
  avail[i0] = false;
  res[0] = i0;
  for (uint32_t j = 1; j < m; ++j) {
    float tgt = fadd(fmul(u2f(j), fdiv(kTau, u2f(m))), ang[i0]);
    if (tgt > kPi) tgt = fsub(tgt, kTau);
    uint32_t bi = i0;
    float bd = kFltMax;
    for (uint32_t i = 0; i < n; ++i)
      if (avail[i]) {
        float d = fabs_(fsub(ang[i], tgt));
        if (d > kPi) d = fsub(kTau, d);
        if (d < bd) {
          bd = d;
          bi = i;
        }
      }
    avail[bi] = false;
    res[j] = bi;
  }
}
struct BbSat {
  float s, s2;
  bool has_r;
  V3 nr, nc;
  bool inv;
  uint32_t code;
};
RSX_F bool tst_face(BbSat& st, float e1, float e2, V3 n, uint32_t cc) {
  st.s2 = fsub(fabs_(e1), e2);
  if (st.s2 > 0.0f) return false;
  if (st.s2 > st.s) {
    st.s = st.s2;
    st.has_r = true;
    st.nr = n;
    st.inv = e1 < 0.0f;
    st.code = cc;
  }
  return true;
}
RSX_F bool tst_cross(BbSat& st, float e1, float e2, V3 n, uint32_t cc) {
  st.s2 = fsub(fabs_(e1), e2);
  if (st.s2 > kEps) return false;
  float l = len(n);
  if (l > kEps) {
    st.s2 = fdiv(st.s2, l);
    if (fmul(st.s2, 1.05f) > st.s) {
      st.s = st.s2;
      st.has_r = false;
      st.nc = n / l;
      st.inv = e1 < 0.0f;
      st.code = cc;
    }
  }
  return true;
}
RSX_NOINL RSX_HD inline bool box_box_sat(const Obb& o1, const M3& r1t, const Obb& o2, BbHit* hit) {
  V3 p = o2.c - o1.c;
  V3 pp = r1t * p;
  M3 rij = r1t * o2.ax;
  V3 rc[3] = {rij.c0, rij.c1, rij.c2};
  M3 qm = mabs(rij);
  V3 qc[3] = {qm.c0, qm.c1, qm.c2};
  M3 qrm = transpose(qm);
  V3 qr[3] = {qrm.c0, qrm.c1, qrm.c2};
  BbSat st;
  st.s = from_bits(0xFF800000u);
  st.s2 = 0.0f;
  st.has_r = false;
  st.nr = vzero();
  st.nc = vzero();
  st.inv = false;
  st.code = 0;
  V3 a1[3] = {o1.ax.c0, o1.ax.c1, o1.ax.c2};
  for (int i = 0; i < 3; ++i)
    if (!tst_face(st, comp(pp, i), fadd(comp(o1.ext, i), dot(o2.ext, qr[i])), a1[i], (uint32_t)(i + 1))) return false;
  V3 a2[3] = {o2.ax.c0, o2.ax.c1, o2.ax.c2};
  for (int i = 0; i < 3; ++i)
    if (!tst_face(st, dot(a2[i], p), fadd(dot(o1.ext, qc[i]), comp(o2.ext, i)), a2[i], (uint32_t)(i + 4))) return false;
  const V3 fudge = vs(1e-5f);
  for (int i = 0; i < 3; ++i) qc[i] = qc[i] + fudge;
  qrm = transpose(M3{qc[0], qc[1], qc[2]});
  qr[0] = qrm.c0;
  qr[1] = qrm.c1;
  qr[2] = qrm.c2;
  const V3 unit[3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int i = 0; i < 3; ++i) {
    int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
    for (int j = 0; j < 3; ++j) {
      int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
      V3 n = cross(unit[i], rc[j]);
      float e2 = fadd(fadd(fadd(fmul(comp(o1.ext, i1), comp(qc[j], i2)), fmul(comp(o1.ext, i2), comp(qc[j], i1))),
                           fmul(comp(o2.ext, j1), comp(qr[i], j2))),
                      fmul(comp(o2.ext, j2), comp(qr[i], j1)));
      if (!tst_cross(st, dot(pp, n), e2, n, (uint32_t)(7 + i * 3 + j))) return false;
    }
  }
  if (st.code == 0) return false;
  V3 normal = st.has_r ? st.nr : o1.ax * st.nc;
  if (st.inv) normal = -normal;
  hit->depth = fneg(st.s);
  hit->n = normal;
  hit->code = st.code;
  return true;
}
RSX_NOINL RSX_HD inline void box_box_points(Ctx& c, Obb o1, M3 r1t, Obb o2, M3 r2t, const BbHit& hit, Manifold* m, uint32_t b1, uint32_t b2) {
  V3 r1a[3] = {r1t.c0, r1t.c1, r1t.c2};
  V3 r2a[3] = {r2t.c0, r2t.c1, r2t.c2};
  if (hit.code > 6) {
    V3 pa = o1.c;
    for (int i = 0; i < 3; ++i) {
      float sg = fsub(fmul(2.0f, dot(hit.n, r1a[i]) > 0.0f ? 1.0f : 0.0f), 1.0f);
      pa = pa + fmul(sg, comp(o1.ext, i)) * r1a[i];
    }
    V3 pb = o2.c;
    for (int i = 0; i < 3; ++i) {
      float sg = fsub(1.0f, fmul(2.0f, dot(hit.n, r2a[i]) > 0.0f ? 1.0f : 0.0f));
      pb = pb + fmul(sg, comp(o2.ext, i)) * r2a[i];
    }
    V3 ua = r1a[(hit.code - 7) / 3], ub = r2a[(hit.code - 7) % 3];
    float beta = line_closest(pa, ua, pb, ub);
    add_contact(c, *m, b1, b2, -hit.n, pb + ub * beta, fneg(hit.depth), -1);
    return;
  }
  if (hit.code > 3) {
    Obb t = o1;
    o1 = o2;
    o2 = t;
    M3 tm = r1t;
    r1t = r2t;
    r2t = tm;
    for (int i = 0; i < 3; ++i) {
      V3 x = r1a[i];
      r1a[i] = r2a[i];
      r2a[i] = x;
    }
  }
  V3 n2 = hit.code <= 3 ? hit.n : -hit.n;
  V3 nr = mul_t(r2t, n2);
  V3 anr = vabs(nr);
  int lanr, a1, a2;
  if (anr.y > anr.x) {
    if (anr.y > anr.z) { lanr = 1; a1 = 0; a2 = 2; }
    else { lanr = 2; a1 = 0; a2 = 1; }
  } else if (anr.x > anr.z) {
    lanr = 0; a1 = 1; a2 = 2;
  } else {
    lanr = 2; a1 = 0; a2 = 1;
  }
  float inc = comp(nr, lanr) < 0.0f ? comp(o2.ext, lanr) : fneg(comp(o2.ext, lanr));
  V3 center = (o2.c - o1.c) + inc * r2a[lanr];
  uint32_t cn = hit.code <= 3 ? hit.code - 1 : hit.code - 4;
  int c1i = cn == 0 ? 1 : 0, c2i = cn == 2 ? 1 : 2;
  float cc1 = dot(center, r1a[c1i]), cc2 = dot(center, r1a[c2i]);
  V4 mm = {dot(r1a[c1i], r2a[a1]), dot(r1a[c1i], r2a[a2]), dot(r1a[c2i], r2a[a1]), dot(r1a[c2i], r2a[a2])};
  V4 k = {fmul(mm.x, comp(o2.ext, a1)), fmul(mm.y, comp(o2.ext, a2)), fmul(mm.z, comp(o2.ext, a1)), fmul(mm.w, comp(o2.ext, a2))};
  float quad[4][2] = {{fsub(fsub(cc1, k.x), k.y), fsub(fsub(cc2, k.z), k.w)},
                      {fadd(fsub(cc1, k.x), k.y), fadd(fsub(cc2, k.z), k.w)},
                      {fadd(fadd(cc1, k.x), k.y), fadd(fadd(cc2, k.z), k.w)},
                      {fsub(fadd(cc1, k.x), k.y), fsub(fadd(cc2, k.z), k.w)}};
  float rect[2] = {comp(o1.ext, c1i), comp(o1.ext, c2i)};
  Poly16 ret;
  clip_rect_quad(rect, quad, &ret);
  if (ret.n == 0) return;
  float det1 = fdiv(1.0f, fsub(fmul(mm.x, mm.w), fmul(mm.y, mm.z)));
  mm = V4{fmul(mm.x, det1), fmul(mm.y, det1), fmul(mm.z, det1), fmul(mm.w, det1)};
  uint32_t cnum = 0;
  V3 point[16];
  float dep[16];
  for (uint32_t j = 0; j < ret.n; ++j) {
    float k1 = fsub(fmul(mm.w, fsub(ret.p[j][0], cc1)), fmul(mm.y, fsub(ret.p[j][1], cc2)));
    float k2 = fadd(fmul(fneg(mm.z), fsub(ret.p[j][0], cc1)), fmul(mm.x, fsub(ret.p[j][1], cc2)));
    point[cnum] = (center + k1 * r2a[a1]) + k2 * r2a[a2];
    dep[cnum] = fsub(comp(o1.ext, (int)cn), dot(n2, point[cnum]));
    if (dep[cnum] >= 0.0f) {
      ret.p[cnum][0] = ret.p[j][0];
      ret.p[cnum][1] = ret.p[j][1];
      cnum += 1;
    }
  }
  if (cnum == 0) return;
  uint32_t maxc = cnum < (uint32_t)kMaxPoints ? cnum : (uint32_t)kMaxPoints;
  if (cnum <= maxc) {
    for (uint32_t i = 0; i < cnum; ++i) {
      V3 pw = point[i] + o1.c;
      add_contact(c, *m, b1, b2, -hit.n, hit.code < 4 ? pw : pw - hit.n * dep[i], fneg(dep[i]), -1);
    }
    return;
  }
  uint32_t i1 = 0;
  for (uint32_t i = 0; i < cnum; ++i)
    if (dep[i] > dep[i1]) i1 = i;
  uint32_t iret[kMaxPoints];
  cull_points(ret.p, cnum, i1, maxc, iret);
  for (uint32_t t = 0; t < maxc; ++t) {
    uint32_t id = iret[t];
    V3 pw = point[id] + o1.c;
    add_contact(c, *m, b1, b2, -hit.n, hit.code < 4 ? pw : pw - hit.n * dep[id], fneg(dep[id]), -1);
  }
}
RSX_HD RSX_NOINL inline bool alg_box_box(Ctx& c, uint32_t ba, uint32_t bb, Manifold* out) {
  if (!box_overlap(body_box(c.S, c.D, ba), body_box(c.S, c.D, bb))) return false;
  Aff ta = child_xf(c.S, c.D, ba), tb = child_xf(c.S, c.D, bb);
  M3 ainv = transpose(ta.m);
  const BodyConst& c1 = c.D.bodies[ba];
  const BodyConst& c2 = c.D.bodies[bb];
  Obb o1 = {ta.t, ta.m, add_s(c1.box_half, c1.box_margin)};
  Obb o2 = {tb.t, tb.m, add_s(c2.box_half, c2.box_margin)};
  BbHit hit;
  if (!box_box_sat(o1, ainv, o2, &hit)) return false;
  Manifold m = manifold_new(ba, bb);
  box_box_points(c, o1, ta.m, o2, tb.m, hit, &m, ba, bb);
  if (m.n == 0) return false;
  refresh_points(c.S, c.D, m, ba, bb);
  *out = m;
  return true;
}

// ---- mesh jobs: the BVH walk as a resumable cursor ----
struct Cursor {
  uint32_t stack[128];
  int n;
};
RSX_F void cursor_init(Cursor& cu, const MeshInfo& mesh, const Box3& b) {
  cu.n = 0;
  if (!box_overlap(b, mesh.root_box)) return;
  cu.stack[0] = 0;
  cu.n = 1;
}
RSX_F bool cursor_next(Cursor& cu, const StaticData& D, const MeshInfo& mesh, const Box3& b, uint32_t* tri) {
  while (cu.n != 0) {
    uint32_t w = cu.stack[--cu.n];
    if (w & 0x80000000u) {
      *tri = D.leaves[mesh.leaf_first + (w & 0x7FFFFFFFu)].tri;
      return true;
    }
    const WideNode& nd = D.nodes[mesh.node_first + w];
    uint32_t m = node_mask(nd, b);
    for (int l = (int)nd.n_child - 1; l >= 0; --l)
      if ((m & (1u << l)) && cu.n < 128) cu.stack[cu.n++] = nd.child[l];
  }
  return false;
}

// ball against one triangle (front side only)
struct SphereTriHit { V3 normal, point; float depth; };
RSX_F float seg_dist2(V3 from, V3 to, V3 p, V3* nearest) {
  V3 diff = p - from, v = to - from;
  float t = dot(v, diff);
  if (t > 0.0f) {
    float vv = dot(v, v);
    if (t < vv) {
      t = fdiv(t, vv);
      diff -= vs(t) * v;
    } else {
      t = 1.0f;
      diff -= v;
    }
  } else {
    t = 0.0f;
  }
  *nearest = from + vs(t) * v;
  return dot(diff, diff);
}
RSX_HD RSX_NOINL inline bool sphere_triangle(const Tri& t, V3 center, float radius, float rt, float rt2, SphereTriHit* out) {
  V3 to_c = center - t.p0;
  float dp = dot(to_c, t.n);
  if (dp < 0.0f) return false;
  if (dp >= rt) return false;
  V3 otp[3] = {to_c, center - t.p1, center - t.p2};
  V3 cp;
  if (dot(cross(t.p1 - t.p0, otp[0]), t.n) >= 0.0f && dot(cross(t.p2 - t.p1, otp[1]), t.n) >= 0.0f &&
      dot(cross(t.p0 - t.p2, otp[2]), t.n) >= 0.0f) {
    cp = center - t.n * dp;
  } else {
    float md = rt2;
    cp = vzero();
    for (int e = 0; e < 3; ++e) {
      V3 a = e == 0 ? t.p0 : (e == 1 ? t.p1 : t.p2), b = e == 0 ? t.p1 : (e == 1 ? t.p2 : t.p0);
      V3 ne = vzero();
      float d = seg_dist2(a, b, center, &ne);
      if (d < md) {
        md = d;
        cp = ne;
      }
    }
    if (!(md < rt2)) return false;
  }
  V3 tc = center - cp;
  float d2 = len2(tc);
  if (d2 >= rt2) return false;
  if (d2 > kEps) {
    float d = fsqrt(d2);
    out->normal = tc * fdiv(1.0f, d);
    out->depth = fneg(fsub(radius, d));
  } else {
    out->normal = t.n;
    out->depth = fneg(radius);
  }
  out->point = cp;
  return true;
}

struct SphereJob {
  int32_t manifold;  // pool index
  uint32_t sph, mesh_body;
  const MeshInfo* mesh;
  V3 center, mesh_t;
  float radius, rt, rt2;
  Box3 box;
  Cursor cu;
};
struct BoxJob {
  Aff box_xf, mesh_to_box;
  V3 half;
  float margin, maxd;
  Manifold m;
  bool has_m;
  uint32_t car, mesh_body;
  M3 tri_rot;
  const MeshInfo* mesh;
  Box3 box;
  Cursor cu;
};

RSX_F bool sphere_job_begin(Ctx& c, uint32_t sph, uint32_t mb, int32_t mi, SphereJob& j) {
  if (!(mb < (uint32_t)kMeshes && c.D.meshes[mb].body == mb)) {
    c.unimplemented += 1;
    return false;
  }
  const MeshInfo* mesh = &c.D.meshes[mb];
  Aff xs = body_xf(c.S, c.D, sph), xm = body_xf(c.S, c.D, mb);
  V3 cis = xs.t - xm.t;
  float cbt = breaking(c.D, c.S.manifolds[mi]);
  float r = c.D.bodies[sph].sphere_margin;
  float rt = fadd(r, cbt);
  j.manifold = mi;
  j.sph = sph;
  j.mesh_body = mb;
  j.mesh = mesh;
  j.center = cis;
  j.radius = r;
  j.rt = rt;
  j.rt2 = fmul(rt, rt);
  j.mesh_t = xm.t;
  j.box = sphere_box(r, cis);
  cursor_init(j.cu, *mesh, j.box);
  return true;
}
RSX_F bool box_job_begin(Ctx& c, uint32_t car, uint32_t mb, BoxJob& j) {
  if (!(mb < (uint32_t)kMeshes && c.D.meshes[mb].body == mb)) {
    c.unimplemented += 1;
    return false;
  }
  const MeshInfo* mesh = &c.D.meshes[mb];
  const BodyConst& bc = c.D.bodies[car];
  Aff cw = child_xf(c.S, c.D, car);
  Aff ot = body_xf(c.S, c.D, mb);
  Aff x1 = aff_inverse_rigid(ot);
  Aff cin = {x1.m * cw.m, xform_point(x1, cw.t)};
  Box3 bt = box_from_half(bc.box_half, bc.box_margin, cin);
  Aff m2b = aff_inverse_rigid(cw) * ot;
  float br = rmin(bc.breaking_threshold, c.D.bodies[mb].breaking_threshold);
  j.has_m = false;
  j.car = car;
  j.mesh_body = mb;
  j.mesh = mesh;
  j.box = bt;
  j.half = bc.box_half;
  j.margin = bc.box_margin;
  j.maxd = fadd(bc.box_margin, br);
  j.box_xf = cw;
  j.mesh_to_box = m2b;
  j.tri_rot = ot.m;
  cursor_init(j.cu, *mesh, bt);
  return true;
}
RSX_F bool box_job_next(const StaticData& D, BoxJob& j, uint32_t* tri) {
  uint32_t leaf;
  while (cursor_next(j.cu, D, *j.mesh, j.box, &leaf)) {
    const Tri& t = D.tris[j.mesh->tri_first + leaf];
    V3 lo = vmin(vmin(t.p0, t.p1), t.p2), hi = vmax(vmax(t.p0, t.p1), t.p2);
    if (!(all_le(lo, j.box.hi) && all_ge(hi, j.box.lo))) continue;
    *tri = leaf;
    return true;
  }
  return false;
}

// ---- the near callback ----
RSX_F int32_t find_manifold(const ArenaState& S, uint32_t b0, uint32_t b1) {
  uint32_t lo = b0 < b1 ? b0 : b1, hi = b0 < b1 ? b1 : b0;
  for (uint32_t i = 0; i < S.n_manifolds; ++i) {
    uint32_t a = S.manifolds[i].body0, b = S.manifolds[i].body1;
    if ((a < b ? a : b) == lo && (a < b ? b : a) == hi) return (int32_t)i;
  }
  return -1;
}
RSX_F int32_t insert_manifold(ArenaState& S, const Manifold& m) {
  if (S.n_manifolds >= (uint32_t)kMaxManifolds) {
    S.overflow[OVF_MANIFOLDS] += 1;
    return -1;
  }
  S.manifolds[S.n_manifolds] = m;
  return (int32_t)S.n_manifolds++;
}
RSX_F void push_active(ArenaState& S, uint32_t i) {
  if (S.n_active >= (uint32_t)kMaxActive) {
    S.overflow[OVF_ACTIVE] += 1;
    return;
  }
  S.active[S.n_active++] = i;
}
// the second half: merge the fresh manifold into the retained one (or insert it), then mark it active
RSX_HD RSX_NOINL inline void near_tail(Ctx& c, uint32_t rb0, uint32_t rb1, int32_t cached, bool has_fresh, const Manifold& fresh) {
  ArenaState& S = c.S;
  int32_t act;
  if (cached >= 0) {
    Manifold& m = S.manifolds[cached];
    uint32_t b0 = m.body0, b1 = m.body1;
    if (m.n != 0) refresh_points(S, c.D, m, b0, b1);
    if (has_fresh) {
      merge_points(c.D, m, fresh);
    } else {
      for (uint32_t i = 0; i < m.n; ++i) {
        MPoint p = m.pts[i];
        tracker_retained(c, p, b0, b1);
      }
    }
    act = cached;
  } else if (has_fresh) {
    act = insert_manifold(S, fresh);
  } else {
    uint32_t ka = c.D.bodies[rb0].shape, kb = c.D.bodies[rb1].shape;
    bool sw = ka == SHAPE_PLANE || (ka == SHAPE_MESH && kb == SHAPE_SPHERE) || (ka == SHAPE_MESH && kb == SHAPE_BOX) ||
              (ka == SHAPE_BOX && kb == SHAPE_SPHERE);
    act = insert_manifold(S, manifold_new(sw ? rb1 : rb0, sw ? rb0 : rb1));
  }
  if (act < 0) return;
  push_active(S, (uint32_t)act);
}

enum { NEAR_DONE = 0, NEAR_BOX_JOB = 1, NEAR_SPHERE_JOB = 2 };
struct NearPair { uint32_t rb0, rb1; int32_t cached; };

RSX_F int near_head(Ctx& c, uint32_t rb0, uint32_t rb1, NearPair& np, BoxJob& bj, SphereJob& sj) {
  ArenaState& S = c.S;
  if ((!body_awake(S, c.D, rb0) && !body_awake(S, c.D, rb1)) || !body_responds(S, c.D, rb0) || !body_responds(S, c.D, rb1)) return NEAR_DONE;
  int32_t cached = find_manifold(S, rb0, rb1);
  np.rb0 = rb0;
  np.rb1 = rb1;
  np.cached = cached;
  uint32_t k0 = c.D.bodies[rb0].shape, k1 = c.D.bodies[rb1].shape;
  bool cpair = false;
  uint32_t comp_i = 0, other = 0;
  if (k0 == SHAPE_BOX && k1 != SHAPE_BOX) {
    cpair = true;
    comp_i = rb0;
    other = rb1;
  } else if (k1 == SHAPE_BOX && k0 != SHAPE_BOX) {
    cpair = true;
    comp_i = rb1;
    other = rb0;
  }
  if (cpair && !box_overlap(child_box(S, c.D, comp_i), body_box(S, c.D, other))) {
    release_manifold(S, rb0, rb1);
    return NEAR_DONE;
  }
  if ((k0 == SHAPE_SPHERE && k1 == SHAPE_MESH) || (k0 == SHAPE_MESH && k1 == SHAPE_SPHERE)) {
    uint32_t cv = k0 == SHAPE_SPHERE ? rb0 : rb1, cc = k0 == SHAPE_SPHERE ? rb1 : rb0;
    int32_t pi = cached;
    if (pi < 0) pi = insert_manifold(S, manifold_new(cv, cc));
    if (pi < 0) return NEAR_DONE;
    RSX_ZONE_BEGIN(z_sj);
    bool job = sphere_job_begin(c, cv, cc, pi, sj);
    RSX_ZONE_END(z_sj, 21);
    if (job) return NEAR_SPHERE_JOB;
    push_active(S, (uint32_t)pi);
    return NEAR_DONE;
  }
  Manifold fresh = {};
  bool has = false;
  uint32_t ko = c.D.bodies[other].shape;
  if (cpair && (ko == SHAPE_PLANE || ko == SHAPE_MESH)) {
    if (ko == SHAPE_PLANE) {
      RSX_ZONE_BEGIN(z_cp);
      has = alg_convex_plane(c, comp_i, other, child_xf(S, c.D, comp_i), true, &fresh);
      RSX_ZONE_END(z_cp, 17);
    } else {
      RSX_ZONE_BEGIN(z_bj);
      bool job = box_job_begin(c, comp_i, other, bj);
      RSX_ZONE_END(z_bj, 22);
      if (job) return NEAR_BOX_JOB;
    }
  } else if (k0 == SHAPE_PLANE && k1 == SHAPE_SPHERE) {
    has = alg_convex_plane(c, rb1, rb0, body_xf(S, c.D, rb1), false, &fresh);
  } else if (k0 == SHAPE_SPHERE && k1 == SHAPE_PLANE) {
    has = alg_convex_plane(c, rb0, rb1, body_xf(S, c.D, rb0), false, &fresh);
  } else if (k0 == SHAPE_SPHERE && k1 == SHAPE_BOX) {
    RSX_ZONE_BEGIN(z_sb);
    has = alg_sphere_box(c, rb0, rb1, &fresh);
    RSX_ZONE_END(z_sb, 18);
  } else if (k0 == SHAPE_BOX && k1 == SHAPE_SPHERE) {
    RSX_ZONE_BEGIN(z_sb);
    has = alg_sphere_box(c, rb1, rb0, &fresh);
    RSX_ZONE_END(z_sb, 18);
  } else if (k0 == SHAPE_BOX && k1 == SHAPE_BOX) {
    RSX_ZONE_BEGIN(z_bb);
    has = alg_box_box(c, rb0, rb1, &fresh);
    RSX_ZONE_END(z_bb, 19);
  } else {
    c.unimplemented += 1;
  }
  RSX_ZONE_BEGIN(z_nt);
  near_tail(c, rb0, rb1, cached, has, fresh);
  RSX_ZONE_END(z_nt, 23);
  return NEAR_DONE;
}

// P3b driver: pairs in order; a mesh pair's leaves in BVH walk order, each leaf's contact added in that order.  The loop
// is kept as a state (P3bLoop) and a step, so that a kernel can step the loops of many arenas in lockstep; phase3b runs
// the steps to the end.  A step runs the pair heads up to the next mesh job (or the end of the pairs), then one chunk of
// the open job: up to kLeafChunk leaves taken from the walk, tested, and their hits added in walk order; the job's tail
// follows the chunk that exhausts the walk.  Taking the leaves of a chunk before testing them, and testing them before
// adding any, computes what the reference's leaf-by-leaf loop computes (collision_dispatcher.cuh:240-280): the walk
// reads only the job's fixed query box and the static BVH, and a leaf's test reads only the job's fixed transforms and
// the static triangle, so neither depends on the contacts added before it; only the additions are ordered.  Kernels can
// therefore run the tests of a chunk on any lanes (p3b_collect, leaf_test, p3b_add_hit, p3b_close below).
constexpr int kLeafChunk = 32;
struct P3bLoop {
  uint32_t n, i, unimplemented;
  int kind;
  bool walk_done;  // the open job's walk has no leaf left
  NearPair np;
  BoxJob bj;
  SphereJob sj;
};
RSX_F void p3b_begin(const ArenaState& S, P3bLoop& L) {
  L.n = S.n_pairs < (uint32_t)kMaxPairs ? S.n_pairs : (uint32_t)kMaxPairs;
  L.i = 0;
  L.unimplemented = 0;
  L.kind = NEAR_DONE;
  L.walk_done = false;
  L.np = NearPair{};
}
RSX_F bool p3b_more(const P3bLoop& L) { return L.kind != NEAR_DONE || L.i < L.n; }

// The pair heads up to the next mesh job: returns its kind (NEAR_BOX_JOB / NEAR_SPHERE_JOB), or NEAR_DONE when the pairs
// ran out.  A job already open is returned as it is.
RSX_F int p3b_open(ArenaState& S, const StaticData& D, P3bLoop& L) {
  if (L.kind != NEAR_DONE) return L.kind;
  Ctx c = {S, D, L.unimplemented};
  RSX_ZONE_BEGIN(z_head);
  while (L.i < L.n) {
    Pair p = S.pairs[L.i++];
    L.kind = near_head(c, D.proxies[p.h0].body, D.proxies[p.h1].body, L.np, L.bj, L.sj);
    if (L.kind != NEAR_DONE) break;
  }
  RSX_ZONE_END(z_head, 10);
  L.unimplemented = c.unimplemented;
  L.walk_done = false;
  return L.kind;
}

// The next leaves of the open job's walk (at most cap) into tris[], in walk order; sets L.walk_done when the walk ends.
RSX_F int p3b_collect(const StaticData& D, P3bLoop& L, uint32_t* tris, int cap) {
  int k = 0;
  while (k < cap) {
    uint32_t tri;
    bool more;
    if (L.kind == NEAR_BOX_JOB) {
      RSX_ZONE_BEGIN(z_bnext);
      more = box_job_next(D, L.bj, &tri);
      RSX_ZONE_END(z_bnext, 12);
    } else {
      RSX_ZONE_BEGIN(z_snext);
      more = cursor_next(L.sj.cu, D, *L.sj.mesh, L.sj.box, &tri);
      RSX_ZONE_END(z_snext, 14);
    }
    if (!more) {
      L.walk_done = true;
      break;
    }
    tris[k++] = tri;
  }
  return k;
}

// What one leaf's test needs, fixed for the whole job: the box job's car box and the mesh-to-box transform, or the
// sphere job's centre (in the mesh's frame) and radii; and where the mesh's triangles start.
struct LeafJob {
  int kind;
  uint32_t tri_first;
  Aff box_xf, mesh_to_box;
  V3 half;
  float margin, maxd;
  V3 center;
  float radius, rt, rt2;
};
// One leaf's result: box jobs use point (the contact in world) and depth (the distance); sphere jobs normal, point
// (in the mesh's frame) and depth.
struct LeafHit {
  uint32_t found;
  V3 normal, point;
  float depth;
};
RSX_F void leaf_job_of(const P3bLoop& L, LeafJob& j) {
  j.kind = L.kind;
  if (L.kind == NEAR_BOX_JOB) {
    j.tri_first = L.bj.mesh->tri_first;
    j.box_xf = L.bj.box_xf;
    j.mesh_to_box = L.bj.mesh_to_box;
    j.half = L.bj.half;
    j.margin = L.bj.margin;
    j.maxd = L.bj.maxd;
  } else {
    j.tri_first = L.sj.mesh->tri_first;
    j.center = L.sj.center;
    j.radius = L.sj.radius;
    j.rt = L.sj.rt;
    j.rt2 = L.sj.rt2;
  }
}
// The test of one leaf (a pure function of the job and the static triangle).
RSX_F bool leaf_test(const LeafJob& j, const StaticData& D, uint32_t tri, LeafHit* h) {
  const Tri& t = D.tris[j.tri_first + tri];
  if (j.kind == NEAR_BOX_JOB) {
    RSX_ZONE_BEGIN(z_sat);
    V3 q[3] = {xform_point(j.mesh_to_box, t.p0), xform_point(j.mesh_to_box, t.p1), xform_point(j.mesh_to_box, t.p2)};
    SatHit sh;
    bool f = box_triangle_sat(j.box_xf, j.half, j.margin, q, j.maxd, &sh);
    h->found = f;
    h->point = sh.point_world;
    h->depth = sh.distance;
    RSX_ZONE_END(z_sat, 11);
    return f;
  }
  RSX_ZONE_BEGIN(z_stri);
  SphereTriHit sh;
  bool f = sphere_triangle(t, j.center, j.radius, j.rt, j.rt2, &sh);
  h->found = f;
  h->normal = sh.normal;
  h->point = sh.point;
  h->depth = sh.depth;
  RSX_ZONE_END(z_stri, 15);
  return f;
}
// leaf_test in stages, for callers that share a box-triangle SAT's feature pairs among threads: true when the test is
// complete (h set); false when the SAT goes on from f (feat_pair, then leaf_test_back).  Same results as leaf_test.
RSX_F bool leaf_test_front(const LeafJob& j, const StaticData& D, uint32_t tri, LeafHit* h, SatFront* f) {
  if (j.kind != NEAR_BOX_JOB) {  // a sphere-triangle test is always complete (leaf_test's value is whether it found one)
    leaf_test(j, D, tri, h);
    return true;
  }
  const Tri& t = D.tris[j.tri_first + tri];
  V3 q[3] = {xform_point(j.mesh_to_box, t.p0), xform_point(j.mesh_to_box, t.p1), xform_point(j.mesh_to_box, t.p2)};
  SatHit sh;
  const int r = sat_front(j.box_xf, j.half, j.margin, q, j.maxd, &sh, f);
  if (r == SAT_PAIRS) return false;
  h->found = r == SAT_HIT;
  h->point = sh.point_world;
  h->depth = sh.distance;
  return true;
}
RSX_F void leaf_test_back(const SatFront& f, const FeatPair* P, LeafHit* h) {
  SatHit sh;
  h->found = sat_back(f, P, &sh);
  h->point = sh.point_world;
  h->depth = sh.distance;
}
// The contact of a leaf whose test found one, into the job's manifold (in walk order).
RSX_F void p3b_add_hit(ArenaState& S, const StaticData& D, P3bLoop& L, uint32_t tri, const LeafHit& h) {
  Ctx c = {S, D, L.unimplemented};
  if (L.kind == NEAR_BOX_JOB) {
    BoxJob& bj = L.bj;
    const Tri& t = D.tris[bj.mesh->tri_first + tri];
    if (!bj.has_m) {
      bj.m = manifold_new(bj.car, bj.mesh_body);
      bj.has_m = true;
    }
    add_contact(c, bj.m, bj.car, bj.mesh_body, bj.tri_rot * t.n, h.point, h.depth, (int32_t)tri);
  } else {
    SphereJob& sj = L.sj;
    add_contact(c, S.manifolds[sj.manifold], sj.sph, sj.mesh_body, h.normal, h.point + sj.mesh_t, h.depth, (int32_t)tri);
  }
  L.unimplemented = c.unimplemented;
}
// The job's tail once its walk is done: the box job's fresh manifold merged into the pair's (or inserted), the sphere
// job's manifold refreshed and marked active.
RSX_F void p3b_close(ArenaState& S, const StaticData& D, P3bLoop& L) {
  Ctx c = {S, D, L.unimplemented};
  if (L.kind == NEAR_BOX_JOB) {
    RSX_ZONE_BEGIN(z_btail);
    BoxJob& bj = L.bj;
    Manifold fresh = {};
    bool has = false;
    if (bj.has_m) {
      refresh_points(S, D, bj.m, bj.car, bj.mesh_body);
      if (bj.m.n != 0) {
        fresh = bj.m;
        has = true;
      }
    }
    near_tail(c, L.np.rb0, L.np.rb1, L.np.cached, has, fresh);
    RSX_ZONE_END(z_btail, 13);
  } else {
    RSX_ZONE_BEGIN(z_stail);
    SphereJob& sj = L.sj;
    Manifold& m = S.manifolds[sj.manifold];
    if (m.n != 0) refresh_points(S, D, m, sj.sph, sj.mesh_body);
    push_active(S, (uint32_t)sj.manifold);
    RSX_ZONE_END(z_stail, 16);
  }
  L.kind = NEAR_DONE;
  L.unimplemented = c.unimplemented;
}

// one step; false when the phase has no work left
RSX_F bool p3b_step(ArenaState& S, const StaticData& D, P3bLoop& L) {
  if (!p3b_more(L)) return false;
  if (p3b_open(S, D, L) == NEAR_DONE) return false;
  uint32_t tris[kLeafChunk];
  int k = p3b_collect(D, L, tris, kLeafChunk);
  LeafJob j;
  leaf_job_of(L, j);
  for (int i = 0; i < k; ++i) {
    LeafHit h;
    if (leaf_test(j, D, tris[i], &h)) p3b_add_hit(S, D, L, tris[i], h);
  }
  if (L.walk_done) p3b_close(S, D, L);
  return p3b_more(L);
}

RSX_F uint32_t phase3b(ArenaState& S, const StaticData& D) {
  P3bLoop L;
  p3b_begin(S, L);
  while (p3b_step(S, D, L)) {
  }
  return L.unimplemented;
}

}  // namespace sim
}  // namespace rsx
