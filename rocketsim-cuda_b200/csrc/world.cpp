// Synthetic Soccar world and start states (host only).  The game's collision meshes and RocketSim V3's static dump
// are not available, so this file builds a StaticData of the reference's exact layout from a seeded synthetic arena:
//   * a closed box 8192 x 10240 x 2044 uu with two goal recesses 1786 x 880 x 642 uu and quarter-cylinder fillets of
//     radius 256 uu, every vertex jittered by +-0.5 uu from the seed, split into the 16 mesh bodies the layout has
//     (fillets, back walls, goals and corners), the floor, ceiling and side walls as the 4 static planes;
//   * per mesh a 4-wide BVH (one leaf per triangle), the internal-edge angle map (Bullet's btGenerateInternalEdgeInfo
//     idea: the signed dihedral angle of each shared edge, its convexity and normal-swap flags);
//   * the 11 x 11 x 2 ray grid with its static cell lists, the sweep-and-prune quantisation, body constants, the 34
//     boost pads, the mutator defaults, and the car constants of 7 hitbox presets (synthetic stand-ins for the game's).
// Start states are seeded and self-consistent: poses, velocities, and a broadphase (sorted SAP edges, the overlapping
// pairs, the dynamic ray-grid cells) that satisfies the invariants the incremental sweep-and-prune maintains.
// All arithmetic is binary32 (no FP64), with the library's correctly rounded sin / cos.
#include <stdint.h>
#include <string.h>
#include <stdlib.h>
#include <algorithm>
#include <vector>
#include <map>
#include "state.cuh"
#include "crmath.cuh"
#include "sim/physics.cuh"
#include "sim/start.cuh"

namespace rsx {
namespace world {

// ---- the arena surface --------------------------------------------------------------------------------------------
struct MeshBuild {
  std::vector<V3> verts;                 // uu, jittered
  std::vector<uint32_t> idx;             // 3 per triangle
  std::map<std::pair<int64_t, int64_t>, uint32_t> vmap;  // exact vertex sharing (keyed on 1/64 uu grid)
};

static uint32_t vert(MeshBuild& m, Rng& rng, V3 p) {
  int64_t kx = (int64_t)(p.x * 64.0f), ky = (int64_t)(p.y * 64.0f), kz = (int64_t)(p.z * 64.0f);
  std::pair<int64_t, int64_t> key{kx * 4000000 + ky, kz};
  auto it = m.vmap.find(key);
  if (it != m.vmap.end()) return it->second;
  V3 q = {p.x + rng.range(-0.5f, 0.5f), p.y + rng.range(-0.5f, 0.5f), p.z + rng.range(-0.5f, 0.5f)};
  m.verts.push_back(q);
  uint32_t i = (uint32_t)m.verts.size() - 1;
  m.vmap[key] = i;
  return i;
}

// A grid patch: P(u, v) for u in [0, nu], v in [0, nv]; triangles oriented so that their normal points along `inward`
// (a function of the position).  `skip(u, v)` removes a cell (the goal opening).
template <class Pos, class Inward, class Skip>
static void patch(MeshBuild& m, Rng& rng, int nu, int nv, Pos pos, Inward inward, Skip skip) {
  for (int i = 0; i < nu; ++i)
    for (int j = 0; j < nv; ++j) {
      if (skip(i, j)) continue;
      uint32_t a = vert(m, rng, pos(i, j)), b = vert(m, rng, pos(i + 1, j)), c = vert(m, rng, pos(i + 1, j + 1)),
               d = vert(m, rng, pos(i, j + 1));
      uint32_t t[2][3] = {{a, b, c}, {a, c, d}};
      for (auto& tr : t) {
        V3 p0 = m.verts[tr[0]], p1 = m.verts[tr[1]], p2 = m.verts[tr[2]];
        V3 n = cross(p1 - p0, p2 - p0);
        V3 cen = (p0 + p1 + p2) * (1.0f / 3.0f);
        if (dot(n, inward(cen)) < 0.0f) std::swap(tr[1], tr[2]);
        m.idx.push_back(tr[0]);
        m.idx.push_back(tr[1]);
        m.idx.push_back(tr[2]);
      }
    }
}

constexpr float HX = 4096.0f, HY = 5120.0f, HZ = 2044.0f, R = 256.0f;
constexpr float GW = 893.0f, GD = 880.0f, GH = 642.0f;  // goal half width, depth, height
constexpr int ARC = 8;                                  // segments of a quarter circle

static float cs(float a) { return cr_cos(a); }
static float sn(float a) { return cr_sin(a); }
constexpr float HALF_PI = 1.57079632679f;

// The 16 surfaces (mesh bodies 0-15).
static void build_meshes(std::vector<MeshBuild>& out, Rng& rng) {
  out.assign(16, MeshBuild{});
  auto none = [](int, int) { return false; };
  int k = 0;
  // 0-1: floor-side fillets (x = -HX, +HX), 2-3: ceiling-side fillets; along y, ARC around the edge
  for (int top = 0; top < 2; ++top)
    for (int side = 0; side < 2; ++side, ++k) {
      float sx = side ? 1.0f : -1.0f;
      float cz = top ? HZ - R : R, cx = sx * (HX - R);
      int ny = 40;
      patch(out[k], rng, ARC, ny,
            [&](int i, int j) {
              float a = HALF_PI * (float)i / ARC;  // 0: the wall tangent, pi/2: the floor / ceiling tangent
              float y = -HY + R + (2 * (HY - R)) * (float)j / ny;
              return V3{cx + sx * R * cs(a), y, cz + (top ? 1.0f : -1.0f) * R * sn(a)};
            },
            [&](V3 p) { return V3{cx - p.x, 0.0f, cz - p.z}; }, none);
    }
  // 4-5: floor-back fillets (y = -HY, +HY), 6-7: ceiling-back fillets; along x, the floor ones broken at the goal
  for (int top = 0; top < 2; ++top)
    for (int side = 0; side < 2; ++side, ++k) {
      float sy = side ? 1.0f : -1.0f;
      float cz = top ? HZ - R : R, cy = sy * (HY - R);
      int nx = 32;
      patch(out[k], rng, ARC, nx,
            [&](int i, int j) {
              float a = HALF_PI * (float)i / ARC;
              float x = -HX + R + (2 * (HX - R)) * (float)j / nx;
              return V3{x, cy + sy * R * cs(a), cz + (top ? 1.0f : -1.0f) * R * sn(a)};
            },
            [&](V3 p) { return V3{0.0f, cy - p.y, cz - p.z}; },
            [&](int, int j) {
              if (top) return false;
              float x0 = -HX + R + (2 * (HX - R)) * (float)j / nx, x1 = -HX + R + (2 * (HX - R)) * (float)(j + 1) / nx;
              return x1 > -GW && x0 < GW;
            });
    }
  // 8-9: back walls at y = -HY, +HY between the fillets, with the goal opening
  for (int side = 0; side < 2; ++side, ++k) {
    float sy = side ? 1.0f : -1.0f;
    int nx = 30, nz = 7;
    float x0 = -HX + R, x1 = HX - R, z0 = R, z1 = HZ - R;
    patch(out[k], rng, nx, nz,
          [&](int i, int j) { return V3{x0 + (x1 - x0) * i / nx, sy * HY, z0 + (z1 - z0) * j / nz}; },
          [&](V3) { return V3{0.0f, -sy, 0.0f}; },
          [&](int i, int j) {
            float xa = x0 + (x1 - x0) * i / nx, xb = x0 + (x1 - x0) * (i + 1) / nx, za = z0 + (z1 - z0) * j / nz;
            return xb > -GW && xa < GW && za < GH;
          });
    // the strip below z0 beside the goal: part of the floor-back fillet region, covered there
  }
  // 10-11: goal interiors (sides, back, roof) behind y = -HY, +HY
  for (int side = 0; side < 2; ++side, ++k) {
    float sy = side ? 1.0f : -1.0f;
    float yb = sy * (HY + GD);
    int n1 = 6, n2 = 4;
    MeshBuild& m = out[k];
    for (int wx = 0; wx < 2; ++wx) {  // the two side walls x = -GW, +GW
      float x = wx ? GW : -GW;
      patch(m, rng, n1, n2, [&](int i, int j) { return V3{x, sy * HY + sy * GD * i / n1, GH * j / n2}; },
            [&](V3) { return V3{wx ? -1.0f : 1.0f, 0.0f, 0.0f}; }, none);
    }
    patch(m, rng, 10, n2, [&](int i, int j) { return V3{-GW + 2 * GW * i / 10, yb, GH * j / n2}; },
          [&](V3) { return V3{0.0f, -sy, 0.0f}; }, none);
    patch(m, rng, 10, n1, [&](int i, int j) { return V3{-GW + 2 * GW * i / 10, sy * HY + sy * GD * j / n1, GH}; },
          [&](V3) { return V3{0.0f, 0.0f, -1.0f}; }, none);
  }
  // 12-15: vertical corner fillets at (+-HX, +-HY)
  for (int cxs = 0; cxs < 2; ++cxs)
    for (int cys = 0; cys < 2; ++cys, ++k) {
      float sx = cxs ? 1.0f : -1.0f, sy = cys ? 1.0f : -1.0f;
      float cx = sx * (HX - R), cy = sy * (HY - R);
      int nz = 8;
      patch(out[k], rng, ARC, nz,
            [&](int i, int j) {
              float a = HALF_PI * (float)i / ARC;
              return V3{cx + sx * R * cs(a), cy + sy * R * sn(a), R + (HZ - 2 * R) * j / nz};
            },
            [&](V3 p) { return V3{cx - p.x, cy - p.y, 0.0f}; }, none);
    }
}

// ---- BVH -----------------------------------------------------------------------------------------------------------
struct BvhOut {
  std::vector<WideNode> nodes;
  std::vector<Leaf> leaves;
};

static Box3 tri_box(const Tri& t) {
  return Box3{vmin(vmin(t.p0, t.p1), t.p2), vmax(vmax(t.p0, t.p1), t.p2)};
}
static Box3 box_union(Box3 a, Box3 b) { return Box3{vmin(a.lo, b.lo), vmax(a.hi, b.hi)}; }

// Builds node `ni` over leaves [first, first + count) of `order` (triangle indices local to the mesh); returns its box.
static Box3 build_node(BvhOut& o, const std::vector<Tri>& tris, std::vector<uint32_t>& order, int first, int count, uint32_t ni) {
  WideNode& n0 = o.nodes[ni];
  memset(&n0, 0, sizeof(n0));
  int groups = count <= 4 ? count : 4;
  int bounds[5];
  if (count <= 4) {
    for (int g = 0; g <= groups; ++g) bounds[g] = first + g;
  } else {
    // split along the longest axis of the centroid box into 4 equal parts
    Box3 cb = {vs(1e30f), vs(-1e30f)};
    for (int i = first; i < first + count; ++i) {
      const Tri& t = tris[order[i]];
      V3 c = (t.p0 + t.p1 + t.p2) * (1.0f / 3.0f);
      cb.lo = vmin(cb.lo, c);
      cb.hi = vmax(cb.hi, c);
    }
    V3 ext = cb.hi - cb.lo;
    int axis = ext.x >= ext.y && ext.x >= ext.z ? 0 : (ext.y >= ext.z ? 1 : 2);
    std::sort(order.begin() + first, order.begin() + first + count, [&](uint32_t a, uint32_t b) {
      const Tri& ta = tris[a];
      const Tri& tb = tris[b];
      float ca = comp(ta.p0, axis) + comp(ta.p1, axis) + comp(ta.p2, axis);
      float cb2 = comp(tb.p0, axis) + comp(tb.p1, axis) + comp(tb.p2, axis);
      return ca < cb2 || (ca == cb2 && a < b);
    });
    for (int g = 0; g <= 4; ++g) bounds[g] = first + (int)((int64_t)count * g / 4);
  }
  Box3 total = {vs(1e30f), vs(-1e30f)};
  uint32_t child[4];
  Box3 cbx[4];
  for (int g = 0; g < groups; ++g) {
    int f = bounds[g], c = bounds[g + 1] - bounds[g];
    if (c == 1) {
      Leaf lf;
      lf.tri = order[f];
      lf.box = tri_box(tris[order[f]]);
      o.leaves.push_back(lf);
      child[g] = 0x80000000u | (uint32_t)(o.leaves.size() - 1);
      cbx[g] = lf.box;
    } else {
      uint32_t ci = (uint32_t)o.nodes.size();
      o.nodes.push_back(WideNode{});
      cbx[g] = build_node(o, tris, order, f, c, ci);
      child[g] = ci;
    }
    total = box_union(total, cbx[g]);
  }
  WideNode& n = o.nodes[ni];
  for (int g = 0; g < 4; ++g) {
    bool v = g < groups;
    n.lo_x[g] = v ? cbx[g].lo.x : 0.0f; n.lo_y[g] = v ? cbx[g].lo.y : 0.0f; n.lo_z[g] = v ? cbx[g].lo.z : 0.0f;
    n.hi_x[g] = v ? cbx[g].hi.x : 0.0f; n.hi_y[g] = v ? cbx[g].hi.y : 0.0f; n.hi_z[g] = v ? cbx[g].hi.z : 0.0f;
    n.child[g] = v ? child[g] : 0u;
  }
  n.n_child = (uint32_t)groups;
  n.valid = (1u << groups) - 1u;
  return total;
}

// ---- internal edge angles (per mesh) -------------------------------------------------------------------------------
static void edge_infos(const std::vector<Tri>& tris, const std::vector<uint32_t>& idx, TriInfo* infos) {
  const float TAU = 6.28318530717958647692f;
  size_t nt = tris.size();
  for (size_t t = 0; t < nt; ++t) infos[t] = TriInfo{0u, TAU, TAU, TAU};
  std::map<std::pair<uint32_t, uint32_t>, std::pair<uint32_t, int>> edges;  // (lo, hi vertex) -> (tri, edge no)
  for (size_t t = 0; t < nt; ++t)
    for (int e = 0; e < 3; ++e) {
      uint32_t a = idx[3 * t + e], b = idx[3 * t + (e + 1) % 3];
      std::pair<uint32_t, uint32_t> key{std::min(a, b), std::max(a, b)};
      auto it = edges.find(key);
      if (it == edges.end()) {
        edges[key] = {(uint32_t)t, e};
        continue;
      }
      uint32_t ta = it->second.first;
      int ea = it->second.second;
      // both triangles get the same edge's signed angle from their own side
      for (int side = 0; side < 2; ++side) {
        uint32_t tt = side ? (uint32_t)t : ta, to = side ? ta : (uint32_t)t;
        int ee = side ? e : ea;
        const Tri& A = tris[tt];
        const Tri& B = tris[to];
        V3 pa[3] = {A.p0, A.p1, A.p2};
        V3 v0 = pa[ee], v1 = pa[(ee + 1) % 3], vo = pa[(ee + 2) % 3];
        V3 edge = normalize(v1 - v0);
        V3 pb[3] = {B.p0, B.p1, B.p2};
        V3 other = pb[0];
        for (int q = 0; q < 3; ++q) {
          V3 d = pb[q] - v0, d2 = pb[q] - v1;
          if (len2(d) > 1e-8f && len2(d2) > 1e-8f) other = pb[q];
        }
        V3 ca = normalize(cross(edge, A.n));
        if (dot(ca, other - v0) < 0.0f) ca = -ca;  // points across the edge, into B's side
        V3 cb = normalize(cross(edge, B.n));
        if (dot(cb, vo - v0) < 0.0f) cb = -cb;     // points into A's side
        float dotab = dot(ca, cb);
        float sinv = len(cross(ca, cb));
        float angle = 0.0f;
        bool convex = false;
        if (sinv > 1e-4f) {
          float ang = cr_atan2(sinv, dotab);       // angle between the two in-plane directions
          float bend = 3.14159265f - ang;          // dihedral bend
          convex = dot(A.n, other - v0) < 0.0f;    // B bends away from A's normal side
          angle = convex ? bend : -bend;
        }
        TriInfo& inf = infos[tt];
        uint32_t cflag = 1u << ee, sflag = 8u << ee;
        if (convex) inf.flags |= cflag;
        // swap flag: the edge rotation by `angle` of A's normal is B's normal or its opposite
        float s = cr_sin(angle * 0.5f), c = cr_cos(angle * 0.5f);
        V3 nb = qrotate(quat_axis_sc(-(pa[(ee + 1) % 3] - pa[ee]) / len(pa[(ee + 1) % 3] - pa[ee]), s, c), A.n);
        if (dot(nb, B.n) < 0.0f) inf.flags |= sflag;
        if (ee == 0) inf.a01 = angle; else if (ee == 1) inf.a12 = angle; else inf.a20 = angle;
      }
    }
}

// ---- hitbox presets (uu): size, offset, front / back wheel radius, rest length, connection (x, y, z) ----------------
struct Preset {
  float size[3], off[3];
  float fr, frest, fx, fy, fz;
  float br, brest, bx, by, bz;
};
// Synthetic stand-ins for the game's seven car bodies (Octane's hitbox is the reference's own, consts.cuh:92-94).
static const Preset kPresets[7] = {
    {{120.507f, 86.6994f, 38.6591f}, {13.8757f, 0.0f, 20.755f}, 12.50f, 38.755f, 51.25f, 25.90f, 20.755f, 15.00f, 37.055f, -33.75f, 29.50f, 20.755f},
    {{130.427f, 85.7799f, 33.8f}, {9.0f, 0.0f, 15.75f}, 12.00f, 33.95f, 50.30f, 31.10f, 15.75f, 13.50f, 33.85f, -34.75f, 33.00f, 15.75f},
    {{131.32f, 87.1704f, 31.8944f}, {9.00857f, 0.0f, 12.0942f}, 12.50f, 31.9242f, 49.97f, 27.80f, 12.0942f, 17.00f, 27.9242f, -35.43f, 20.28f, 12.0942f},
    {{133.992f, 83.021f, 32.8f}, {12.5f, 0.0f, 11.75f}, 13.50f, 29.7f, 51.50f, 26.67f, 11.75f, 15.00f, 29.666f, -35.75f, 35.00f, 11.75f},
    {{129.519f, 84.6879f, 36.6591f}, {13.8757f, 0.0f, 20.755f}, 12.50f, 38.755f, 51.25f, 25.90f, 20.755f, 15.00f, 37.055f, -34.00f, 29.50f, 20.755f},
    {{123.22f, 79.2103f, 44.1591f}, {11.3757f, 0.0f, 21.505f}, 15.00f, 39.505f, 51.25f, 25.90f, 21.505f, 15.00f, 39.105f, -33.75f, 29.50f, 21.505f},
    {{127.0f, 82.0f, 36.0f}, {12.0f, 0.0f, 18.0f}, 13.00f, 36.0f, 50.50f, 27.00f, 18.0f, 15.50f, 35.0f, -34.50f, 30.00f, 18.0f},
};

// ---- boost pads (uu) ----
static const float kBigPads[6][2] = {{-3584, 0}, {3584, 0}, {-3072, 4096}, {3072, 4096}, {-3072, -4096}, {3072, -4096}};
static const float kSmallPads[28][2] = {
    {0, -4240}, {-1792, -4184}, {1792, -4184}, {-940, -3308}, {940, -3308}, {0, -2816}, {-3584, -2484},
    {3584, -2484}, {-1788, -2300}, {1788, -2300}, {-2048, -1036}, {0, -1024}, {2048, -1036}, {-1024, 0},
    {1024, 0}, {-2048, 1036}, {0, 1024}, {2048, 1036}, {-1788, 2300}, {1788, 2300}, {-3584, 2484},
    {3584, 2484}, {0, 2816}, {-940, 3310}, {940, 3308}, {-1792, 4184}, {1792, 4184}, {0, 4240}};

int build_static(StaticData* sd, uint64_t seed, int preset0, int preset1) {
  memset(sd, 0, sizeof(StaticData));
  Rng rng{seed};
  std::vector<MeshBuild> meshes;
  build_meshes(meshes, rng);

  // ---- world constants ----
  sd->game_mode = 0;
  sd->no_ball_rot = 0;
  sd->ball_body = 20;
  sd->gravity_uu = V3{0.0f, 0.0f, -650.0f};
  const float mut[kMut] = {180.0f, 30.0f, 6000.0f, 0.03f, 4375.0f / 3.0f, 875.0f / 3.0f, 2975.0f / 3.0f, 3175.0f / 3.0f,
                           100.0f / 3.0f, 3.0f, 0.25f, 100.0f, 100.0f / 3.0f, 12.0f, 100.0f, 10.0f, 4.0f, 1.0f, 1.0f, 91.25f};
  for (int i = 0; i < kMut; ++i) sd->mut[i] = mut[i];
  sd->unlimited_flips = 0;
  sd->unlimited_double_jumps = 0;
  sd->recharge_boost = 0;
  sd->recharge_per_second = 0.0f;
  sd->recharge_delay = 0.25f;
  sd->demo_mode = 0;
  sd->team_demos = 0;
  sd->goal_y = 5124.25f;
  sd->pads_enabled = 1;
  sd->gravity_bt = V3{0.0f, 0.0f, -650.0f * BT};
  for (int d = 0; d < kDyn; ++d) {
    sd->dyn_body[d] = 20 + d;
    sd->dyn_handle[d] = 21 + d;
  }
  sd->cell_size = 24.0f;
  sd->cell_size_sq = 24.0f * 24.0f;
  sd->grid_n[0] = 11; sd->grid_n[1] = 11; sd->grid_n[2] = 2;
  sd->grid_lo = V3{-132.0f, -132.0f, -4.0f};
  sd->grid_hi = V3{132.0f, 132.0f, 44.0f};
  sd->sap_lo = V3{-250.0f, -250.0f, -250.0f};
  sd->sap_quant = vs(65535.0f / 500.0f);
  sd->sap_mask = 0xFFFEu;
  sd->sap_sentinel = 0xFFFFu;
  sd->sap_max_handles = kHandles;
  sd->sap_half_extent = 250.0f;

  // ---- meshes: triangles in BT units, the BVH, the edge map ----
  uint32_t tri_at = 0, node_at = 0, leaf_at = 0;
  for (int m = 0; m < kMeshes; ++m) {
    MeshBuild& mb = meshes[m];
    std::vector<Tri> tris;
    for (size_t t = 0; t < mb.idx.size() / 3; ++t) {
      V3 p0 = mb.verts[mb.idx[3 * t]] * BT, p1 = mb.verts[mb.idx[3 * t + 1]] * BT, p2 = mb.verts[mb.idx[3 * t + 2]] * BT;
      V3 n = normalize(cross(p1 - p0, p2 - p0));
      tris.push_back(Tri{p0, p1, p2, n});
    }
    uint32_t nt = (uint32_t)tris.size();
    if (tri_at + nt > (uint32_t)kMaxTris) return -1;
    BvhOut bo;
    bo.nodes.push_back(WideNode{});
    std::vector<uint32_t> order(nt);
    for (uint32_t i = 0; i < nt; ++i) order[i] = i;
    Box3 root = build_node(bo, tris, order, 0, (int)nt, 0);
    if (node_at + bo.nodes.size() > (size_t)kMaxNodes || leaf_at + bo.leaves.size() > (size_t)kMaxLeaves) return -2;
    for (uint32_t i = 0; i < nt; ++i) sd->tris[tri_at + i] = tris[i];
    edge_infos(tris, mb.idx, &sd->infos[tri_at]);
    for (size_t i = 0; i < bo.nodes.size(); ++i) sd->nodes[node_at + i] = bo.nodes[i];
    for (size_t i = 0; i < bo.leaves.size(); ++i) sd->leaves[leaf_at + i] = bo.leaves[i];
    MeshInfo& mi = sd->meshes[m];
    mi.body = (uint32_t)m;
    mi.tri_first = tri_at; mi.tri_count = nt;
    mi.node_first = node_at; mi.node_count = (uint32_t)bo.nodes.size();
    mi.leaf_first = leaf_at; mi.leaf_count = (uint32_t)bo.leaves.size();
    mi.ident_box = root;
    mi.root_box = root;
    tri_at += nt;
    node_at += (uint32_t)bo.nodes.size();
    leaf_at += (uint32_t)bo.leaves.size();
  }

  // ---- planes (bodies 16-19): floor, ceiling, side walls x = -HX, +HX ----
  const V3 pn[4] = {{0, 0, 1}, {0, 0, -1}, {1, 0, 0}, {-1, 0, 0}};
  const V3 pt[4] = {{0, 0, 0}, {0, 0, HZ * BT}, {-HX * BT, 0, 0}, {HX * BT, 0, 0}};
  const float BIG = 200.0f;
  for (int p = 0; p < kPlanes; ++p) {
    Plane& pl = sd->planes[p];
    pl.body = 16 + p;
    pl.n = pn[p];
    pl.single_axis = 1;
    pl.axis = p < 2 ? 2 : 0;
    pl.backwards = comp(pn[p], (int)pl.axis) < 0.0f ? 1u : 0u;
    Box3 ib = {vs(-BIG), vs(BIG)};
    float s = comp(pn[p], (int)pl.axis);
    if (s > 0.0f) set_comp(ib.hi, (int)pl.axis, 0.0f); else set_comp(ib.lo, (int)pl.axis, 0.0f);
    pl.ident_box = ib;
    pl.box = Box3{ib.lo + pt[p], ib.hi + pt[p]};
  }

  // ---- bodies ----
  const int presets[2] = {preset0, preset1};
  for (int b = 0; b < kBodies; ++b) {
    BodyConst& c = sd->bodies[b];
    c.world_idx = (uint32_t)b;
    c.handle = (uint32_t)b + 1;
    c.pose = aff_identity();
    c.processing_threshold = 1e18f;
    c.lin_sleep = 0.8f;
    c.ang_sleep = 1.0f;
    if (b < 20) {  // static
      c.user = 0;
      c.group = 2;
      c.mask = 0xFD;
      c.friction = 0.6f;
      c.restitution = 0.3f;
      c.breaking_threshold = 1e18f;
      if (b < 16) {
        c.shape = 0;
        c.mesh_tris = sd->meshes[b].tri_count;
      } else {
        c.shape = 1;
        c.pose.t = pt[b - 16];
      }
      continue;
    }
    c.group = 1;
    c.mask = 0xFF;
    if (b == 20) {  // ball
      float r = 91.25f * BT;
      c.user = 2;
      c.shape = 2;
      c.sphere_dim = vs(r);
      c.sphere_margin = r;
      c.mass = 30.0f;
      c.inv_mass = 1.0f / 30.0f;
      float I = 0.4f * 30.0f * r * r;
      c.inv_inertia_local = vs(1.0f / I);
      c.inv_mass3 = vs(c.inv_mass);
      c.friction = 0.35f;
      c.restitution = 0.6f;
      c.breaking_threshold = r * 0.02f;
      c.lin_damping = 0.03f;
      continue;
    }
    int ci = b - 21;
    const Preset& pr = kPresets[presets[ci]];
    c.user = 1;
    c.user_ptr = (uint32_t)ci;
    c.shape = 3;
    c.box_margin = 0.04f;
    V3 half = V3{pr.size[0], pr.size[1], pr.size[2]} * (0.5f * BT);
    c.box_half = half - vs(0.04f);
    c.child = aff_identity();
    c.child.t = V3{pr.off[0], pr.off[1], pr.off[2]} * BT;
    c.compound_box = Box3{c.child.t - half, c.child.t + half};
    c.mass = 180.0f;
    c.inv_mass = 1.0f / 180.0f;
    V3 l = half * 2.0f;
    V3 I = V3{(l.y * l.y + l.z * l.z), (l.x * l.x + l.z * l.z), (l.x * l.x + l.y * l.y)} * (180.0f / 12.0f);
    c.inv_inertia_local = V3{1.0f / I.x, 1.0f / I.y, 1.0f / I.z};
    c.inv_mass3 = vs(c.inv_mass);
    c.friction = 0.3f;
    c.restitution = 0.1f;
    c.breaking_threshold = len(half) * 0.02f;
    c.lin_damping = 0.0f;
  }

  // ---- cars ----
  for (int ci = 0; ci < kCars; ++ci) {
    CarConst& cc = sd->cars[ci];
    const Preset& pr = kPresets[presets[ci]];
    cc.car_idx = (uint32_t)ci;
    cc.team = (uint32_t)ci;
    cc.body = 21 + ci;
    cc.three_wheels = 0;
    cc.hitbox_size = V3{pr.size[0], pr.size[1], pr.size[2]};
    cc.hitbox_offset = V3{pr.off[0], pr.off[1], pr.off[2]};
    for (int w = 0; w < kWheels; ++w) {
      bool front = w < 2, left = (w % 2) == 0;
      WheelConst& wc = cc.wheels[w];
      float r = front ? pr.fr : pr.br, rest = front ? pr.frest : pr.brest;
      float x = front ? pr.fx : pr.bx, y = front ? pr.fy : pr.by, z = front ? pr.fz : pr.bz;
      wc.connection = V3{x, left ? -y : y, z} * BT;
      wc.rest_length = (rest - 12.0f) * BT;
      wc.radius = r * BT;
      wc.force_scale = front ? 35.75f : 54.265f;
      wc.ray_length = wc.rest_length + 12.0f * BT + wc.radius;
    }
  }

  // ---- pads ----
  float max_z = 0.0f;
  for (int i = 0; i < kPads; ++i) {
    PadConst& p = sd->pads[i];
    bool big = i < 6;
    p.big = big ? 1u : 0u;
    p.pos = big ? V3{kBigPads[i][0], kBigPads[i][1], 73.0f} : V3{kSmallPads[i - 6][0], kSmallPads[i - 6][1], 70.0f};
    p.box_radius = big ? 160.0f : 120.0f;
    p.cyl_radius = big ? 208.0f : 144.0f;
    p.cooldown = big ? 10.0f : 4.0f;
    p.amount = big ? 100.0f : 12.0f;
    V3 ext = V3{p.cyl_radius, p.cyl_radius, 95.0f};
    p.box = Box3{p.pos - ext, p.pos + ext};
    max_z = max_z > p.pos.z + 95.0f ? max_z : p.pos.z + 95.0f;
  }
  sd->max_pad_z = max_z;

  // ---- proxies and the static ray-grid cells ----
  auto body_box = [&](int b) -> Box3 {
    if (b < 16) return sd->meshes[b].ident_box;
    if (b < 20) return sd->planes[b - 16].box;
    return Box3{vzero(), vzero()};
  };
  for (int h = 1; h < kHandles; ++h) {
    int b = h - 1;
    ProxyConst& px = sd->proxies[h];
    px.body = (uint32_t)b;
    px.group = sd->bodies[b].group;
    px.mask = sd->bodies[b].mask;
    px.uid = (uint32_t)h;
    if (b < 20) {
      px.box = body_box(b);
      uint32_t idx3[3];
      sim::cell_indices(*sd, px.box.lo, idx3);
      px.cell = sim::cell_of(*sd, idx3);
      px.idx[0] = idx3[0]; px.idx[1] = idx3[1]; px.idx[2] = idx3[2];
    }
  }
  uint32_t at = 0;
  const float margin = 2.0f;
  for (uint32_t i = 0; i < sd->grid_n[0]; ++i)
    for (uint32_t j = 0; j < sd->grid_n[1]; ++j)
      for (uint32_t k = 0; k < sd->grid_n[2]; ++k) {
        uint32_t cell = i * sd->grid_n[1] * sd->grid_n[2] + j * sd->grid_n[2] + k;
        V3 lo = sd->grid_lo + V3{sd->cell_size * i, sd->cell_size * j, sd->cell_size * k} - vs(margin);
        V3 hi = lo + vs(sd->cell_size + 2.0f * margin);
        sd->cells[cell].first = at;
        for (int h = 1; h <= 20; ++h) {
          Box3 bb = sd->proxies[h].box;
          if (box_overlap(bb, Box3{lo, hi})) {
            if (at >= (uint32_t)kMaxCellEntries) return -3;
            sd->cell_handles[at++] = (uint32_t)h;
          }
        }
        sd->cells[cell].count = at - sd->cells[cell].first;
      }

  // ---- the auto-flip sine table: sin(idx * 2 pi / 16384), correctly rounded ----
  for (int i = 0; i < kTableSin; ++i) sd->table_sin[i] = sim::table_sin_value(i);
  return (int)tri_at;
}

// ---- start states: csrc/sim/start.cuh (host and device) ----
void make_states(const StaticData& sd, ArenaState* out, uint32_t n, uint64_t seed, const float* mix) {
  for (uint32_t a = 0; a < n; ++a) make_state(sd, out[a], a, seed, mix);
}
void make_states_multi(const StaticData* sds, const uint8_t* idx, ArenaState* out, uint32_t n, uint64_t seed, const float* mix) {
  for (uint32_t a = 0; a < n; ++a) make_state(sds[idx[a]], out[a], a, seed, mix);
}

}  // namespace world
}  // namespace rsx
