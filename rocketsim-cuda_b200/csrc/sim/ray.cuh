// The wheel ray query of P1: a packet of the four wheel rays of a car against the world (reference:
// cuda/sim/raycaster.cuh:105-178 grid ray test and cast_rays, quad_ray.cuh slab tests, quad_ray_shapes.cuh the four
// shapes, quad_ray_callbacks.cuh the closest-hit callback).  Candidates are offered in V3's order (the cells of the four
// ray sources, each cell's static then dynamic handles), and a hit replaces the held one only with a strictly smaller
// fraction, so the order decides ties exactly as in the reference.
#pragma once
#include "base.cuh"

namespace rsx {
namespace sim {

constexpr float kWheelMinHitDist2 = 0.116684f;
constexpr uint32_t kFilterDefault = 1u, kFilterDropshot = 16u, kFilterAll = 0xFFu;

struct RayPacket {  // world rays and the running closest hits
  V3 from[4], to[4];
  float frac[4];
  uint32_t body[4];
  V3 normal[4], point[4];
  uint32_t ignore, group, mask;
  float min_dist2;
};

// a body's local rays and the fractions as they were when its test began
struct LocalRays {
  V3 from[4], to[4];
  float frac[4];
  M3 rot;
  uint32_t body;
  RayPacket* pk;
};

struct RayBox {  // QuadRayInfo: rays, per-ray lambda_max, union box
  V3 src[4], tgt[4];
  float lmax[4];
  Box3 box;
};

RSX_F void raybox_init(RayBox& r, const V3* src, const V3* tgt) {
  for (int i = 0; i < 4; ++i) {
    r.src[i] = src[i];
    r.tgt[i] = tgt[i];
    r.lmax[i] = 1.0f;
  }
  r.box.lo = vmin(src[0], tgt[0]);
  r.box.hi = vmax(src[0], tgt[0]);
  for (int i = 1; i < 4; ++i) {
    r.box.lo = vmin(r.box.lo, vmin(src[i], tgt[i]));
    r.box.hi = vmax(r.box.hi, vmax(src[i], tgt[i]));
  }
}
RSX_F void raybox_dirs(const RayBox& r, float o[3][4], float inv[3][4]) {
  for (int l = 0; l < 4; ++l) {
    o[0][l] = r.src[l].x;
    o[1][l] = r.src[l].y;
    o[2][l] = r.src[l].z;
    float a = fdiv(1.0f, fsub(r.tgt[l].x, r.src[l].x));
    float b = fdiv(1.0f, fsub(r.tgt[l].y, r.src[l].y));
    float c = fdiv(1.0f, fsub(r.tgt[l].z, r.src[l].z));
    inv[0][l] = isfinite_(a) ? a : kFltMax;
    inv[1][l] = isfinite_(b) ? b : kFltMax;
    inv[2][l] = isfinite_(c) ? c : kFltMax;
  }
}
// ray l's slab test against a box: the entry and exit fractions
RSX_F void slab1(const float o[3][4], const float inv[3][4], const Box3& b, int l, float* enter, float* exit) {
  float x0 = fmul(fsub(b.lo.x, o[0][l]), inv[0][l]), x1 = fmul(fsub(b.hi.x, o[0][l]), inv[0][l]);
  float y0 = fmul(fsub(b.lo.y, o[1][l]), inv[1][l]), y1 = fmul(fsub(b.hi.y, o[1][l]), inv[1][l]);
  float z0 = fmul(fsub(b.lo.z, o[2][l]), inv[2][l]), z1 = fmul(fsub(b.hi.z, o[2][l]), inv[2][l]);
  *enter = sse_max(sse_max(sse_min(x0, x1), sse_min(y0, y1)), sse_min(z0, z1));
  *exit = sse_min(sse_min(sse_max(x0, x1), sse_max(y0, y1)), sse_max(z0, z1));
}
// bit l set when ray l crosses the box within [0, lmax[l]]
RSX_F uint32_t slab4(const float o[3][4], const float inv[3][4], const Box3& b, const float lmax[4]) {
  uint32_t m = 0;
  for (int l = 0; l < 4; ++l) {
    float enter, exit;
    slab1(o, inv, b, l, &enter, &exit);
    if (enter <= exit && exit >= 0.0f && enter <= lmax[l]) m |= 1u << l;
  }
  return m;
}

// ---- the closest-hit callback ----
RSX_F void pk_add(RayPacket* pk, uint32_t body, V3 n_world, float frac, int r) {
  if (frac >= pk->frac[r]) return;
  float s = fsub(1.0f, frac);
  V3 cand = s * pk->from[r] + frac * pk->to[r];  // interpolate_3
  if (pk->min_dist2 > 0.0f && len2(cand - pk->from[r]) < pk->min_dist2) return;
  pk->frac[r] = frac;
  pk->normal[r] = n_world;
  pk->body[r] = body;
  pk->point[r] = cand;
}
RSX_F void lr_hit_internal(LocalRays* lr, V3 n_local, float frac, int r) { pk_add(lr->pk, lr->body, lr->rot * n_local, frac, r); }
RSX_F void lr_hit(LocalRays* lr, V3 n_local, float frac, int r) {
  if (frac >= lr->frac[r]) return;
  lr_hit_internal(lr, n_local, frac, r);
}

// ---- triangle mesh through the wide BVH ----
// A mesh test walks the BVH with the rays' union box (internal nodes) and tests each reached leaf in walk order: the
// leaf box's slab test against each ray's running limit lmax, then the ray-triangle test of the rays it lets through,
// whose hits update the packet and the limits (the reference's quad_ray_shapes.cuh:377-405, quad_ray.cuh's slab test
// and the closest-hit callback).  Each leaf is split into an evaluation that depends only on the body's local rays and
// the fractions held when the body's test began (ray_leaf_eval: the slab's entry and exit, the triangle's crossing
// fraction and its classification) and a replay of the decisions that depend on the running limits and hits
// (ray_leaf_replay: the slab's limit, the callback).  Evaluating a leaf and replaying it computes what the reference's
// leaf step computes; and since an evaluation reads nothing a replay writes, a kernel may evaluate a walk's leaves on
// any lanes and replay them in walk order on the ray packet's owner.
struct RayMeshJob {      // a mesh body's test: its local rays, their slab terms, the fractions when the test began
  V3 from[4], to[4];
  float o[3][4], inv[3][4];
  float hf[4];
};
struct RayLeaf {         // one leaf's evaluation
  float enter[4], dist[4];
  uint32_t flags;        // bits 0-3: the slab's enter <= exit && exit >= 0; bits 4-7: the ray crosses the triangle's plane
                         // (dist is the crossing fraction); bits 8-11: the crossing is inside the triangle (evaluated only
                         // when dist is below the evaluation's starting fraction); bits 12-15: the ray meets the back side
};
RSX_F void ray_mesh_job(const LocalRays& lr, const RayBox& rb, RayMeshJob& j) {
  raybox_dirs(rb, j.o, j.inv);
  for (int i = 0; i < 4; ++i) {
    j.from[i] = lr.from[i];
    j.to[i] = lr.to[i];
    j.hf[i] = lr.frac[i];
  }
}
// Evaluates leaf `leaf` of `mesh` for the job's rays; with lmax non-null, rays whose slab test fails at those limits
// are not tested further (their replay skips them anyway).  The inside test runs for crossings below the job's
// starting fractions hf; an evaluation made with hf = 1 therefore serves any later starting fraction (fractions only
// fall from 1).
RSX_F void ray_leaf_eval(const RayMeshJob& j, const StaticData& D, const MeshInfo& mesh, uint32_t leaf, const float* lmax, RayLeaf* e) {
  const Leaf& lf = D.leaves[mesh.leaf_first + leaf];
  const Tri& t = D.tris[mesh.tri_first + lf.tri];
  const float tol = -0.0001f;
  const float dist = dot(t.p0, t.n);
  uint32_t flags = 0;
  for (int r = 0; r < 4; ++r) {
    float enter, exit;
    slab1(j.o, j.inv, lf.box, r, &enter, &exit);
    e->enter[r] = enter;
    e->dist[r] = 0.0f;
    const bool ok = enter <= exit && exit >= 0.0f;
    if (ok) flags |= 1u << r;
    if (!ok || (lmax && !(enter <= lmax[r]))) continue;
    float da = fsub(dot(t.n, j.from[r]), dist);
    float db = fsub(dot(t.n, j.to[r]), dist);
    if (fmul(da, db) >= 0.0f) continue;
    float distance = fdiv(da, fsub(da, db));
    e->dist[r] = distance;
    flags |= (1u << (4 + r)) | ((da <= 0.0f ? 1u : 0u) << (12 + r));
    if (distance >= j.hf[r]) continue;
    V3 p = lerp(j.from[r], j.to[r], distance);
    V3 v0 = t.p0 - p, v1 = t.p1 - p;
    if (dot(cross(v0, v1), t.n) < tol) continue;
    V3 v2 = t.p2 - p;
    if (dot(cross(v1, v2), t.n) < tol) continue;
    if (dot(cross(v2, v0), t.n) < tol) continue;
    flags |= 1u << (8 + r);
  }
  e->flags = flags;
}
// The ray-triangle callback's decisions for one evaluated leaf, against the running limits and the fractions the body's
// test began with (lr->frac): a crossing at or past that fraction caps the limit, one before it that lies inside the
// triangle is a hit candidate.
RSX_F void ray_leaf_replay(LocalRays* lr, float lmax[4], const StaticData& D, const MeshInfo& mesh, uint32_t leaf, const RayLeaf& e) {
  for (int r = 0; r < 4; ++r) {
    if (!((e.flags >> r) & 1u) || !(e.enter[r] <= lmax[r])) continue;
    if (!((e.flags >> (4 + r)) & 1u)) continue;
    if (e.dist[r] >= lr->frac[r]) {
      lmax[r] = rmin(lmax[r], lr->frac[r]);
      continue;
    }
    if (!((e.flags >> (8 + r)) & 1u)) continue;
    const Tri& t = D.tris[mesh.tri_first + D.leaves[mesh.leaf_first + leaf].tri];
    float prev = lr->pk->frac[r];
    lr_hit_internal(lr, ((e.flags >> (12 + r)) & 1u) ? -t.n : t.n, e.dist[r], r);
    if (lr->pk->frac[r] < prev) lmax[r] = lr->pk->frac[r];
  }
}
RSX_F uint32_t node_mask(const WideNode& n, const Box3& b) {
  uint32_t m = 0;
  for (int l = 0; l < 4; ++l) {
    bool o = n.lo_x[l] <= b.hi.x && n.hi_x[l] >= b.lo.x && n.lo_y[l] <= b.hi.y && n.hi_y[l] >= b.lo.y && n.lo_z[l] <= b.hi.z &&
             n.hi_z[l] >= b.lo.z;
    m |= (o ? 1u : 0u) << l;
  }
  return m & n.valid;
}
// The leaves of a mesh body's walk, in order, across the body's meshes: resumable (one leaf per call).
struct RayWalk {
  int mesh;  // the mesh being walked (kMeshes: done)
  int n;
  uint32_t stack[128];
};
RSX_F void ray_walk_seek(RayWalk& w, const StaticData& D, uint32_t body, const Box3& box, int from) {
  for (w.mesh = from; w.mesh < kMeshes; ++w.mesh)
    if (D.meshes[w.mesh].body == body && box_overlap(box, D.meshes[w.mesh].root_box)) {
      w.stack[0] = 0;
      w.n = 1;
      return;
    }
  w.n = 0;
}
RSX_F bool ray_walk_next(RayWalk& w, const StaticData& D, uint32_t body, const Box3& box, int* mesh, uint32_t* leaf) {
  while (w.mesh < kMeshes) {
    const MeshInfo& m = D.meshes[w.mesh];
    while (w.n != 0) {
      uint32_t x = w.stack[--w.n];
      if (x & 0x80000000u) {
        *mesh = w.mesh;
        *leaf = x & 0x7FFFFFFFu;
        return true;
      }
      const WideNode& nd = D.nodes[m.node_first + x];
      uint32_t mk = node_mask(nd, box);
      for (int l = (int)nd.n_child - 1; l >= 0; --l)
        if (mk & (1u << l)) w.stack[w.n++] = nd.child[l];
    }
    ray_walk_seek(w, D, body, box, w.mesh + 1);
  }
  return false;
}
// ---- a mesh body's walk level by level, for callers that expand many walks' nodes side by side ----
// An item of the walk is a node of one of the body's meshes with its path key: the mesh index in bits 12-15 and, for
// each level below the mesh's root, the index (0-3) of the child taken, two bits from bit 10 down.  The stack walk of
// ray_walk_next takes the meshes in index order and, within a mesh, a child's whole subtree before the next child's,
// so sorting a walk's leaves by key gives ray_walk_next's order.  Keys hold kWalkLevels levels of children.
constexpr int kWalkLevels = 6;
RSX_F uint32_t walk_root_key(int mesh) { return (uint32_t)mesh << 12; }
// the children of node `node` of mesh m (level 0: the root) whose boxes meet box, in child order: emit(child, key)
template <class Emit>
RSX_F void walk_expand(const StaticData& D, int m, uint32_t node, uint32_t key, int level, const Box3& box, Emit&& emit) {
  const WideNode& nd = D.nodes[D.meshes[m].node_first + node];
  const uint32_t mk = node_mask(nd, box);
  for (int l = 0; l < (int)nd.n_child; ++l)
    if (mk & (1u << l)) emit(nd.child[l], key | ((uint32_t)l << (10 - 2 * level)));
}
// the whole test of a mesh body, leaf by leaf
RSX_HD RSX_NOINL inline void ray_mesh_body(const StaticData& D, uint32_t body, LocalRays* lr, RayBox* rb) {
  RayMeshJob j;
  ray_mesh_job(*lr, *rb, j);
  RayWalk w;
  ray_walk_seek(w, D, body, rb->box, 0);
  int mesh;
  uint32_t leaf;
  while (ray_walk_next(w, D, body, rb->box, &mesh, &leaf)) {
    RayLeaf e;
    ray_leaf_eval(j, D, D.meshes[mesh], leaf, rb->lmax, &e);
    ray_leaf_replay(lr, rb->lmax, D, D.meshes[mesh], leaf, e);
  }
}

// ---- the ball's sphere ----
RSX_F void ray_sphere(float radius, LocalRays* lr, const RayBox& rb) {
  float r2 = fmul(radius, radius);
  bool within[4], any = false;
  for (int l = 0; l < 4; ++l) {
    V3 s = rb.src[l], t = rb.tgt[l];
    float cx = sse_min(sse_max(0.0f, sse_min(s.x, t.x)), sse_max(s.x, t.x));
    float cy = sse_min(sse_max(0.0f, sse_min(s.y, t.y)), sse_max(s.y, t.y));
    float cz = sse_min(sse_max(0.0f, sse_min(s.z, t.z)), sse_max(s.z, t.z));
    within[l] = fadd(fadd(fmul(cx, cx), fmul(cy, cy)), fmul(cz, cz)) <= r2;
    any = any || within[l];
  }
  if (!any) return;
  float dist[4], dx[4], dy[4], dz[4], disc[4];
  bool valid[4];
  any = false;
  for (int l = 0; l < 4; ++l) {
    V3 s = rb.src[l], t = rb.tgt[l];
    float ex = fsub(t.x, s.x), ey = fsub(t.y, s.y), ez = fsub(t.z, s.z);
    dist[l] = fsqrt(fadd(fadd(fmul(ex, ex), fmul(ey, ey)), fmul(ez, ez)));
    dx[l] = fdiv(ex, dist[l]);
    dy[l] = fdiv(ey, dist[l]);
    dz[l] = fdiv(ez, dist[l]);
    float b = fmul(2.0f, fadd(fadd(fmul(s.x, dx[l]), fmul(s.y, dy[l])), fmul(s.z, dz[l])));
    float c = fsub(fadd(fadd(fmul(s.x, s.x), fmul(s.y, s.y)), fmul(s.z, s.z)), r2);
    disc[l] = fsub(fmul(b, b), fmul(4.0f, c));
    valid[l] = disc[l] >= 0.0f && within[l];
    any = any || valid[l];
  }
  if (!any) return;
  float tt[4];
  bool near[4];
  any = false;
  for (int l = 0; l < 4; ++l) {
    V3 s = rb.src[l];
    float b = fmul(2.0f, fadd(fadd(fmul(s.x, dx[l]), fmul(s.y, dy[l])), fmul(s.z, dz[l])));
    float sq = fsqrt(disc[l]);
    float t0 = fdiv(fsub(fneg(b), sq), 2.0f), t1 = fdiv(fadd(fneg(b), sq), 2.0f);
    bool swp = t0 > t1;
    t0 = swp ? t1 : t0;
    t1 = swp ? t0 : t1;  // selects with the updated t0, as the reference's lane code does
    bool n0 = t0 >= 0.0f && t0 <= dist[l];
    bool n1 = t1 >= 0.0f && t1 <= dist[l] && !n0;
    near[l] = valid[l] && (n0 || n1);
    any = any || near[l];
    tt[l] = n0 ? t0 : t1;
  }
  if (!any) return;
  for (int l = 0; l < 4; ++l) {
    if (!near[l]) continue;
    V3 s = rb.src[l];
    float hx = fadd(s.x, fmul(dx[l], tt[l])), hy = fadd(s.y, fmul(dy[l], tt[l])), hz = fadd(s.z, fmul(dz[l], tt[l]));
    lr_hit(lr, V3{fdiv(hx, radius), fdiv(hy, radius), fdiv(hz, radius)}, fdiv(tt[l], dist[l]), l);
  }
}

// ---- a static plane ----
RSX_F void ray_plane(const Plane& pl, LocalRays* lr, const RayBox& rb) {
  if (!box_overlap(rb.box, pl.ident_box)) return;
  float o[3][4], inv[3][4], ddx[4], ddy[4], ddz[4];
  for (int l = 0; l < 4; ++l) {
    V3 s = rb.src[l];
    ddx[l] = fsub(rb.tgt[l].x, s.x);
    ddy[l] = fsub(rb.tgt[l].y, s.y);
    ddz[l] = fsub(rb.tgt[l].z, s.z);
    o[0][l] = s.x; o[1][l] = s.y; o[2][l] = s.z;
    inv[0][l] = fdiv(1.0f, ddx[l]);
    inv[1][l] = fdiv(1.0f, ddy[l]);
    inv[2][l] = fdiv(1.0f, ddz[l]);
  }
  uint32_t ray_m = slab4(o, inv, pl.ident_box, lr->frac);
  if (!ray_m) return;
  V3 n = pl.n;
  float dist[4], align[4], t[4];
  uint32_t am = 0, tm = 0;
  for (int l = 0; l < 4; ++l) {
    dist[l] = fsqrt(fadd(fadd(fmul(ddx[l], ddx[l]), fmul(ddy[l], ddy[l])), fmul(ddz[l], ddz[l])));
    float id = fdiv(1.0f, dist[l]);
    float ux = fmul(ddx[l], id), uy = fmul(ddy[l], id), uz = fmul(ddz[l], id);
    align[l] = fadd(fadd(fmul(ux, n.x), fmul(uy, n.y)), fmul(uz, n.z));
    if (fabs_(align[l]) >= kEps) am |= 1u << l;
  }
  if (!am) return;
  for (int l = 0; l < 4; ++l) {
    V3 s = rb.src[l];
    float ns = fadd(fadd(fmul(s.x, n.x), fmul(s.y, n.y)), fmul(s.z, n.z));
    t[l] = fdiv(fneg(ns), align[l]);
    if (t[l] >= 0.0f && t[l] < dist[l]) tm |= 1u << l;
  }
  uint32_t hm = ray_m & (am & tm);
  for (int l = 0; l < 4; ++l)
    if (hm & (1u << l)) lr_hit(lr, n, fdiv(t[l], dist[l]), l);
}

// ---- a car's box (a compound of one rounded box) ----
RSX_HD RSX_NOINL inline bool rounded_box_solve(V3 src, V3 dir, float dist, V3 inner, float margin, float* t_out, V3* n_out) {
  float pts[8];
  for (int i = 0; i < 8; ++i) pts[i] = 0.0f;
  pts[1] = dist;
  int cnt = 2;
  for (int ax = 0; ax < 3; ++ax) {
    float d = comp(dir, ax);
    if (d == 0.0f) continue;
    float s = comp(src, ax), h = comp(inner, ax);
    for (int bi = 0; bi < 2; ++bi) {
      float t = fdiv(fsub(bi == 0 ? fneg(h) : h, s), d);
      if (t > 0.0f && t < dist && cnt < 8) pts[cnt++] = t;
    }
  }
  for (int i = 1; i < cnt; ++i) {
    float key = pts[i];
    int j = i;
    while (j > 0 && pts[j - 1] > key) {
      pts[j] = pts[j - 1];
      --j;
    }
    pts[j] = key;
  }
  float m2 = fmul(margin, margin);
  for (int i = 0; i < cnt - 1; ++i) {
    float t0 = pts[i], t1 = pts[i + 1];
    if (t1 <= t0) continue;
    float mid = fadd(t0, fmul(fsub(t1, t0), 0.5f));
    V3 pm = src + dir * mid;
    float a = 0.0f, b = 0.0f, c = 0.0f;
    uint32_t outside = 0;
    for (int ax = 0; ax < 3; ++ax) {
      float p = comp(pm, ax), h = comp(inner, ax), bound;
      if (p < fneg(h)) bound = fneg(h);
      else if (p > h) bound = h;
      else continue;
      outside += 1;
      float o = fsub(comp(src, ax), bound), d = comp(dir, ax);
      a = fadd(a, fmul(d, d));
      b = fadd(b, fmul(fmul(2.0f, d), o));
      c = fadd(c, fmul(o, o));
    }
    if (outside == 0) continue;
    float cc = fsub(c, m2);
    float disc = fsub(fmul(b, b), fmul(fmul(4.0f, a), cc));
    if (disc < 0.0f) {
      float scale = fadd(fmul(b, b), fabs_(fmul(fmul(4.0f, a), cc)));
      if (disc > fmul(fneg(kEps), scale)) disc = 0.0f;
      else continue;
    }
    float sq = fsqrt(disc);
    float th;
    if (disc == 0.0f) {
      th = fdiv(fneg(b), fmul(2.0f, a));
    } else {
      float q = fmul(-0.5f, b >= 0.0f ? fadd(b, sq) : fsub(b, sq));
      if (q == 0.0f) th = fdiv(fneg(b), fmul(2.0f, a));
      else {
        float r0 = fdiv(q, a), r1 = fdiv(cc, q);
        th = r0 <= r1 ? r0 : r1;
      }
    }
    if (th <= 0.0f || th > dist || th < t0 || th > t1) continue;
    V3 hit = src + dir * th;
    V3 n = hit - vclamp(hit, -inner, inner);
    float l2 = len2(n);
    if (l2 <= fmul(kEps, kEps)) continue;
    V3 nn = n / fsqrt(l2);
    if (dot(nn, dir) > 0.0f) continue;
    *t_out = th;
    *n_out = nn;
    return true;
  }
  return false;
}
RSX_HD RSX_NOINL inline void ray_box_one(const BodyConst& bc, LocalRays* lr, V3 src, V3 tgt, int ri) {
  const Box3& la = bc.compound_box;
  V3 delta = tgt - src;
  float dist = len(delta);
  V3 dir = delta / dist;
  float tenter = 0.0f, texit = dist;
  int hit_axis = 0;
  V3 inv = 1.0f / dir;
  V3 t1 = (la.lo - src) * inv, t2 = (la.hi - src) * inv;
  V3 tmin = vmin(t1, t2), tmax = vmax(t1, t2);
  uint32_t negm = (bits(tmax.x) >> 31) | ((bits(tmax.y) >> 31) << 1) | ((bits(tmax.z) >> 31) << 2);
  bool fin[3] = {fabs_(inv.x) < from_bits(0x7F800000u), fabs_(inv.y) < from_bits(0x7F800000u), fabs_(inv.z) < from_bits(0x7F800000u)};
  for (int ax = 0; ax < 3; ++ax) {
    if (!fin[ax]) {
      float o = comp(src, ax);
      if (comp(la.lo, ax) > o || o > comp(la.hi, ax)) return;
      continue;
    }
    if (negm & (1u << ax)) return;
    texit = rmin(texit, comp(tmax, ax));
    if (comp(tmin, ax) > tenter) {
      tenter = comp(tmin, ax);
      hit_axis = ax;
    }
    if (tenter > texit) return;
  }
  if (0.0f >= tenter || tenter > dist) return;
  V3 inner = bc.box_half;
  V3 entry = src + dir * tenter;
  V3 loc = entry - bc.child.t;
  bool face = true;
  for (int ax = 0; ax < 3; ++ax) {
    if (ax == hit_axis) continue;
    if (fabs_(comp(loc, ax)) > comp(inner, ax)) {
      face = false;
      break;
    }
  }
  if (face) {
    V3 hn = vzero();
    set_comp(hn, hit_axis, fneg(rsignum(comp(dir, hit_axis))));
    if (len2(hn) > 0.0f) lr_hit(lr, hn, fdiv(rmax(tenter, 0.0f), dist), ri);
    return;
  }
  float th;
  V3 nc;
  if (!rounded_box_solve(src - bc.child.t, dir, dist, bc.box_half, bc.box_margin, &th, &nc)) return;
  nc = nc / len(nc);
  if (dot(nc, dir) > 0.0f) return;
  if (0.0f >= th || th > dist) return;
  lr_hit(lr, nc, fdiv(th, dist), ri);
}
RSX_F void ray_box(const BodyConst& bc, LocalRays* lr, const RayBox& rb) {
  if (!box_overlap(rb.box, bc.compound_box)) return;
  float o[3][4], inv[3][4];
  raybox_dirs(rb, o, inv);
  uint32_t m = slab4(o, inv, bc.compound_box, lr->frac);
  for (int i = 0; i < 4; ++i)
    if (m & (1u << i)) ray_box_one(bc, lr, rb.src[i], rb.tgt[i], i);
}

// ---- one candidate body (collision_world quad_ray_test) ----
// the body's local rays (the packet's rays in the body's frame, their fractions so far) and their box
RSX_F void ray_body_setup(const ArenaState& S, const StaticData& D, uint32_t w, RayPacket* pk, LocalRays& lr, RayBox& rb) {
  View co = view(S, D, w);
  V3 fl[4], tl[4];
  if (m3_is_identity(co.xf.m)) {
    for (int i = 0; i < 4; ++i) {
      fl[i] = pk->from[i] - co.xf.t;
      tl[i] = pk->to[i] - co.xf.t;
    }
  } else {
    Aff inv = aff_inverse_rigid(co.xf);
    for (int i = 0; i < 4; ++i) {
      fl[i] = xform_point(inv, pk->from[i]);
      tl[i] = xform_point(inv, pk->to[i]);
    }
  }
  for (int i = 0; i < 4; ++i) {
    lr.from[i] = fl[i];
    lr.to[i] = tl[i];
    lr.frac[i] = pk->frac[i];
  }
  lr.rot = co.xf.m;
  lr.body = w;
  lr.pk = pk;
  raybox_init(rb, fl, tl);
  for (int i = 0; i < 4; ++i) rb.lmax[i] = lr.frac[i];
}
RSX_HD RSX_NOINL inline void ray_body(const ArenaState& S, const StaticData& D, uint32_t w, RayPacket* pk) {
  RSX_ZONE_BEGIN(z_setup);
  const BodyConst& bc = D.bodies[w];
  LocalRays lr;
  RayBox rb;
  ray_body_setup(S, D, w, pk, lr, rb);
  RSX_ZONE_END(z_setup, 28);
  RSX_ZONE_BEGIN(z_shape);
  if (bc.shape == SHAPE_BOX) {
    ray_box(bc, &lr, rb);
    RSX_ZONE_END(z_shape, 24);
  } else if (bc.shape == SHAPE_SPHERE) {
    ray_sphere(bc.sphere_margin, &lr, rb);
    RSX_ZONE_END(z_shape, 25);
  } else if (bc.shape == SHAPE_PLANE) {
    for (int p = 0; p < kPlanes; ++p)
      if (D.planes[p].body == w) ray_plane(D.planes[p], &lr, rb);
    RSX_ZONE_END(z_shape, 26);
  } else {
    ray_mesh_body(D, w, &lr, &rb);
    RSX_ZONE_END(z_shape, 27);
  }
}

RSX_F Box3 proxy_box(const ArenaState& S, const StaticData& D, uint32_t h) {
  for (int d = 0; d < kDyn; ++d)
    if (D.dyn_handle[d] == h) return S.dyn_proxy[d].box;
  return D.proxies[h].box;
}
// the ray test's filter of a candidate handle: not the ignored body, and group / mask agree both ways
RSX_F bool ray_accepts(const StaticData& D, uint32_t h, const RayPacket* pk) {
  const ProxyConst& px = D.proxies[h];
  if (pk->ignore == px.body) return false;
  return (px.group & pk->mask) != 0 && (pk->group & px.mask) != 0;
}

// the grid's candidate walk: one cell per distinct ray source, its static handles, then its dynamic ones
// the candidate bodies of the packet, in the walk's order (nothing in the walk depends on the hits); returns their count
RSX_F int grid_candidates(const ArenaState& S, const StaticData& D, const RayPacket* pk, uint32_t cand[kHandles]) {
  Box3 rbx;
  rbx.lo = vmin(pk->from[0], pk->to[0]);
  rbx.hi = vmax(pk->from[0], pk->to[0]);
  for (int i = 1; i < 4; ++i) {
    rbx.lo = vmin(rbx.lo, vmin(pk->from[i], pk->to[i]));
    rbx.hi = vmax(rbx.hi, vmax(pk->from[i], pk->to[i]));
  }
  uint32_t cells[4];
  int nc = 0;
  for (int r = 0; r < 4; ++r) {
    uint32_t i3[3];
    cell_indices(D, pk->from[r], i3);
    uint32_t c = cell_of(D, i3);
    bool seen = false;
    for (int k = 0; k < nc; ++k) seen = seen || cells[k] == c;
    if (!seen) cells[nc++] = c;
  }
  uint32_t seen = 0;
  int nk = 0;
  const uint32_t nd = S.n_dyn_cells < (uint32_t)kMaxDynCells ? S.n_dyn_cells : (uint32_t)kMaxDynCells;
  for (int ci = 0; ci < nc; ++ci) {
    uint32_t cell = cells[ci];
    const CellRange& cr = D.cells[cell];
    for (uint32_t e = 0; e < cr.count; ++e) {
      uint32_t h = D.cell_handles[cr.first + e];
      if (seen & (1u << h)) continue;
      seen |= 1u << h;
      if (box_overlap(rbx, proxy_box(S, D, h)) && ray_accepts(D, h, pk)) cand[nk++] = D.proxies[h].body;
    }
    for (uint32_t e = dyn_cells_first(S, cell); e < nd && S.dyn_cells[e].cell == cell; ++e) {
      uint32_t h = S.dyn_cells[e].handle;
      if (seen & (1u << h)) continue;
      seen |= 1u << h;
      if (box_overlap(rbx, proxy_box(S, D, h)) && ray_accepts(D, h, pk)) cand[nk++] = D.proxies[h].body;
    }
  }
  return nk;
}
// the candidates first, then one body test per step, so that the lanes of a warp step through their lists together
RSX_F void grid_rays(const ArenaState& S, const StaticData& D, RayPacket* pk) {
  uint32_t cand[kHandles];
  int nk = grid_candidates(S, D, pk, cand);
  for (int k = 0; k < nk; ++k) ray_body(S, D, cand[k], pk);
}

struct WheelHit {
  uint32_t some;
  V3 point, normal;
  uint32_t body;
};

RSX_F void wheel_packet_init(RayPacket& pk, const V3* from, const V3* to, uint32_t ignore) {
  for (int i = 0; i < 4; ++i) {
    pk.frac[i] = 1.0f;
    pk.body[i] = kNoBody;
    pk.from[i] = from[i];
    pk.to[i] = to[i];
    pk.normal[i] = vzero();
    pk.point[i] = vzero();
  }
  pk.ignore = ignore;
  pk.group = kFilterDefault | kFilterDropshot;
  pk.mask = kFilterAll;
  pk.min_dist2 = kWheelMinHitDist2;
}
RSX_F void wheel_packet_hits(const ArenaState& S, const StaticData& D, const RayPacket& pk, WheelHit out[4]) {
  for (int i = 0; i < 4; ++i) {
    out[i].some = 0;
    out[i].point = vzero();
    out[i].normal = vzero();
    out[i].body = 0;
    if (pk.body[i] != kNoBody) {
      uint32_t b = pk.body[i];
      if ((body_flags(S, D, b) & CF_NO_RESPONSE) == 0) {
        out[i].some = 1;
        out[i].body = b;
        out[i].point = pk.point[i];
        out[i].normal = normalize_or_zero(pk.normal[i]);
      }
    }
  }
}
RSX_F void cast_wheel_rays(const ArenaState& S, const StaticData& D, const V3* from, const V3* to, uint32_t ignore, WheelHit out[4]) {
  RayPacket pk;
  wheel_packet_init(pk, from, to, ignore);
  grid_rays(S, D, &pk);
  wheel_packet_hits(S, D, pk, out);
}

}  // namespace sim
}  // namespace rsx
