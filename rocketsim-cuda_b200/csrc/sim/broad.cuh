// P3a: the broadphase of the three dynamic bodies: swept AABBs, Bullet's 3-axis sweep-and-prune with u16-quantised
// edges (incremental edge sorts that add and remove overlapping pairs), and the dynamic entries of the ray grid.
// Reference: cuda/sim/collision_world.cuh:34-52, grid_broadphase.cuh, axis_sweep.cuh, overlapping_pair_cache.cuh,
// collision_dispatcher_release.cuh.  Also the construction helpers of a consistent broadphase for fresh states.
#pragma once
#include "base.cuh"

namespace rsx {
namespace sim {

// ---- the pair array (append, swap-remove) ----
RSX_F int find_pair(const ArenaState& S, const StaticData& D, uint32_t id0, uint32_t id1) {
  for (uint32_t i = 0; i < S.n_pairs; ++i)
    if (D.proxies[S.pairs[i].h0].uid == id0 && D.proxies[S.pairs[i].h1].uid == id1) return (int)i;
  return -1;
}
RSX_F void add_pair(ArenaState& S, const StaticData& D, uint32_t h0, uint32_t h1) {
  const ProxyConst& p0 = D.proxies[h0];
  const ProxyConst& p1 = D.proxies[h1];
  if (!((p0.group & p1.mask) != 0 && (p1.group & p0.mask) != 0)) return;
  uint32_t id0, i0, id1, i1;
  if (p0.uid <= p1.uid) { id0 = p0.uid; i0 = h0; id1 = p1.uid; i1 = h1; }
  else { id0 = p1.uid; i0 = h1; id1 = p0.uid; i1 = h0; }
  if (find_pair(S, D, id0, id1) >= 0) return;
  if (S.n_pairs >= (uint32_t)kMaxPairs) {
    S.overflow[OVF_PAIRS] += 1;
    return;
  }
  S.pairs[S.n_pairs++] = Pair{i0, i1};
}

// release_manifold of the pair (body0, body1): the active list loses the index, the pool's last manifold fills the hole
RSX_F void release_manifold(ArenaState& S, uint32_t b0, uint32_t b1) {
  uint32_t lo = b0 < b1 ? b0 : b1, hi = b0 < b1 ? b1 : b0;
  int found = -1;
  for (uint32_t i = 0; i < S.n_manifolds; ++i) {
    uint32_t a = S.manifolds[i].body0, b = S.manifolds[i].body1;
    if ((a < b ? a : b) == lo && (a < b ? b : a) == hi) {
      found = (int)i;
      break;
    }
  }
  if (found < 0) return;
  uint32_t idx = (uint32_t)found, last = S.n_manifolds - 1;
  uint32_t w = 0;
  for (uint32_t r = 0; r < S.n_active; ++r)
    if (S.active[r] != idx) S.active[w++] = S.active[r];
  for (uint32_t r = w; r < S.n_active; ++r) S.active[r] = 0;
  S.n_active = w;
  if (idx != last) {
    S.manifolds[idx] = S.manifolds[last];
    for (uint32_t r = 0; r < S.n_active; ++r)
      if (S.active[r] == last) S.active[r] = idx;
  }
  S.manifolds[last] = Manifold{};
  S.n_manifolds = last;
}

RSX_F void remove_pair(ArenaState& S, const StaticData& D, uint32_t ha, uint32_t hb) {
  uint32_t ua = D.proxies[ha].uid, ub = D.proxies[hb].uid;
  uint32_t id0 = ua < ub ? ua : ub, id1 = ua < ub ? ub : ua;
  int i = find_pair(S, D, id0, id1);
  if (i < 0) return;
  uint32_t last = S.n_pairs - 1;
  Pair p = S.pairs[i];
  if ((uint32_t)i != last) S.pairs[i] = S.pairs[last];
  S.pairs[last] = Pair{0, 0};
  S.n_pairs -= 1;
  release_manifold(S, D.proxies[p.h0].body, D.proxies[p.h1].body);
}

// ---- sweep and prune ----
RSX_F void quantize_point(const StaticData& D, V3 p, uint16_t is_max, uint16_t out[3]) {
  V3 sc = (p - D.sap_lo) * D.sap_quant;
  float top = u2f(D.sap_sentinel);
  V3 cl = {sc.x >= 0.0f ? sse_min(sc.x, top) : 0.0f, sc.y >= 0.0f ? sse_min(sc.y, top) : 0.0f, sc.z >= 0.0f ? sse_min(sc.z, top) : 0.0f};
  out[0] = (uint16_t)(((uint16_t)f2i(cl.x) & D.sap_mask) | is_max);
  out[1] = (uint16_t)(((uint16_t)f2i(cl.y) & D.sap_mask) | is_max);
  out[2] = (uint16_t)(((uint16_t)f2i(cl.z) & D.sap_mask) | is_max);
}
RSX_F bool overlap2d(const ArenaState& S, uint32_t a, uint32_t b, int axis) {
  int a1 = (1 << axis) & 3, a2 = (1 << a1) & 3;
  const HandleEdges& A = S.handle_edges[a];
  const HandleEdges& B = S.handle_edges[b];
  return !(A.hi[a1] < B.lo[a1] || B.hi[a1] < A.lo[a1] || A.hi[a2] < B.lo[a2] || B.hi[a2] < A.lo[a2]);
}
RSX_F bool is_max_edge(Edge e) { return (e.pos & 1) != 0; }
RSX_F void swap_edges(Edge* e, uint32_t i, uint32_t j) {
  Edge t = e[i];
  e[i] = e[j];
  e[j] = t;
}
// an edge moving down (dir -1) or up (+1); `min_edge` says which end of its handle it is
RSX_F void sort_down(ArenaState& S, const StaticData& D, int axis, uint32_t at, bool min_edge) {
  Edge* e = S.edges[axis];
  uint32_t moving = e[at].handle;
  while (at > 0 && e[at].pos < e[at - 1].pos) {
    Edge prev = e[at - 1];
    uint32_t ph = prev.handle;
    if (min_edge) {  // a min edge moving down meets max edges: new overlaps
      if (is_max_edge(prev)) {
        if (overlap2d(S, moving, ph, axis)) add_pair(S, D, moving, ph);
        S.handle_edges[ph].hi[axis] = (uint16_t)(S.handle_edges[ph].hi[axis] + 1);
      } else {
        S.handle_edges[ph].lo[axis] = (uint16_t)(S.handle_edges[ph].lo[axis] + 1);
      }
      S.handle_edges[moving].lo[axis] = (uint16_t)(S.handle_edges[moving].lo[axis] - 1);
    } else {  // a max edge moving down leaves min edges behind: lost overlaps
      if (!is_max_edge(prev)) {
        if (overlap2d(S, moving, ph, axis)) remove_pair(S, D, moving, ph);
        S.handle_edges[ph].lo[axis] = (uint16_t)(S.handle_edges[ph].lo[axis] + 1);
      } else {
        S.handle_edges[ph].hi[axis] = (uint16_t)(S.handle_edges[ph].hi[axis] + 1);
      }
      S.handle_edges[moving].hi[axis] = (uint16_t)(S.handle_edges[moving].hi[axis] - 1);
    }
    swap_edges(e, at, at - 1);
    at -= 1;
  }
}
RSX_F void sort_up(ArenaState& S, const StaticData& D, int axis, uint32_t at, bool min_edge) {
  Edge* e = S.edges[axis];
  uint32_t moving = e[at].handle;
  while (at + 1 < (uint32_t)kEdges && e[at + 1].handle != 0 && e[at].pos >= e[at + 1].pos) {
    Edge next = e[at + 1];
    uint32_t nh = next.handle;
    if (!min_edge) {  // a max edge moving up meets min edges: new overlaps
      if (!is_max_edge(next)) {
        if (overlap2d(S, moving, nh, axis)) add_pair(S, D, moving, nh);
        S.handle_edges[nh].lo[axis] = (uint16_t)(S.handle_edges[nh].lo[axis] - 1);
      } else {
        S.handle_edges[nh].hi[axis] = (uint16_t)(S.handle_edges[nh].hi[axis] - 1);
      }
      S.handle_edges[moving].hi[axis] = (uint16_t)(S.handle_edges[moving].hi[axis] + 1);
    } else {  // a min edge moving up passes max edges: lost overlaps
      if (is_max_edge(next)) {
        if (overlap2d(S, moving, nh, axis)) remove_pair(S, D, moving, nh);
        S.handle_edges[nh].hi[axis] = (uint16_t)(S.handle_edges[nh].hi[axis] - 1);
      } else {
        S.handle_edges[nh].lo[axis] = (uint16_t)(S.handle_edges[nh].lo[axis] - 1);
      }
      S.handle_edges[moving].lo[axis] = (uint16_t)(S.handle_edges[moving].lo[axis] + 1);
    }
    swap_edges(e, at, at + 1);
    at += 1;
  }
}
RSX_F void update_axis(ArenaState& S, const StaticData& D, int axis, uint32_t h, uint16_t qmin, uint16_t qmax) {
  Edge* e = S.edges[axis];
  uint32_t mi = S.handle_edges[h].lo[axis], ma = S.handle_edges[h].hi[axis];
  int32_t dmin = (int32_t)qmin - (int32_t)e[mi].pos, dmax = (int32_t)qmax - (int32_t)e[ma].pos;
  if (dmin == 0 && dmax == 0) return;
  e[mi].pos = qmin;
  e[ma].pos = qmax;
  if (dmin < 0) sort_down(S, D, axis, mi, true);
  if (dmax > 0) sort_up(S, D, axis, ma, false);
  if (dmin > 0) sort_up(S, D, axis, mi, true);
  if (dmax < 0) sort_down(S, D, axis, ma, false);
}

// ---- the ray grid's dynamic entries: sorted by cell, list order within a cell ----
// A body moving to another cell leaves the 3x3x3 block of cells around its old cell and enters the block around its new
// one.  The reference does this cell by cell: a removal finds the first (cell, handle) entry, shifts the tail left and
// zeroes the freed last slot; an insertion (skipped, counting an overflow, when the list is full) goes after every entry
// of a lower or equal cell.  The two passes below give the same list, the same zeroed slots and the same overflow
// count in one sweep each: removal keeps every entry but the first of each block cell for the handle, then zeroes the
// freed slots; insertion merges the block's cells (ascending, the first ones that fit) after equal cells, from the back.
RSX_F void dyn_block_range(const StaticData& D, const uint32_t idx[3], uint32_t lo[3], uint32_t hi[3]) {
  for (int a = 0; a < 3; ++a) {
    uint32_t m = idx[a] > 1 ? idx[a] : 1;
    lo[a] = m - 1;
    uint32_t top = D.grid_n[a] - 1, p = idx[a] + 1;
    hi[a] = top < p ? top : p;
  }
}
// keep_freed (a removal followed at once by the insertion of the same handle): the freed slots are not zeroed here;
// the caller zeroes those the insertion does not refill (dyn_cells_zero_from), which leaves the same words.
RSX_F void dyn_cells_block(ArenaState& S, const StaticData& D, bool add, uint32_t h, const uint32_t idx[3], bool keep_freed = false) {
  uint32_t lo[3], hi[3];
  dyn_block_range(D, idx, lo, hi);
  const uint32_t ny = D.grid_n[1], nz = D.grid_n[2];
  if (!add) {
    uint32_t removed = 0;  // bit (i - lo0) * 9 + (j - lo1) * 3 + (k - lo2): that cell's entry is gone
    uint32_t n = S.n_dyn_cells < (uint32_t)kMaxDynCells ? S.n_dyn_cells : (uint32_t)kMaxDynCells;
    // the list is sorted by cell, and every cell of the block is at least the block's first: the entries before the
    // first at or after that cell stay where they are
    const uint32_t lo3[3] = {lo[0], lo[1], lo[2]};
    uint32_t r0 = dyn_cells_first(S, cell_of(D, lo3));
    if (r0 > n) r0 = n;
    uint32_t w = r0;
    for (uint32_t r = r0; r < n; ++r) {
      DynCell e = S.dyn_cells[r];
      if (e.handle == h) {
        uint32_t i = e.cell / (ny * nz), j = (e.cell / nz) % ny, k = e.cell % nz;
        if (i >= lo[0] && i <= hi[0] && j >= lo[1] && j <= hi[1] && k >= lo[2] && k <= hi[2]) {
          uint32_t bit = 1u << ((i - lo[0]) * 9 + (j - lo[1]) * 3 + (k - lo[2]));
          if (!(removed & bit)) {
            removed |= bit;
            continue;
          }
        }
      }
      if (w != r) S.dyn_cells[w] = e;
      ++w;
    }
    if (!keep_freed)
      for (uint32_t r = w; r < n; ++r) S.dyn_cells[r] = DynCell{0, 0};
    S.n_dyn_cells = w;
    return;
  }
  uint32_t cells[27];
  uint32_t nb = 0;
  for (uint32_t i = lo[0]; i <= hi[0]; ++i)
    for (uint32_t j = lo[1]; j <= hi[1]; ++j)
      for (uint32_t k = lo[2]; k <= hi[2]; ++k) {
        uint32_t c3[3] = {i, j, k};
        cells[nb++] = cell_of(D, c3);
      }
  uint32_t n = S.n_dyn_cells;
  uint32_t room = n < (uint32_t)kMaxDynCells ? (uint32_t)kMaxDynCells - n : 0u;
  uint32_t take = nb < room ? nb : room;
  S.overflow[OVF_DYN_CELLS] += nb - take;
  if (take == 0) return;
  int32_t ia = (int32_t)n - 1, ib = (int32_t)take - 1, out = (int32_t)(n + take) - 1;
  while (ib >= 0) {
    if (ia >= 0 && S.dyn_cells[ia].cell > cells[ib]) {
      S.dyn_cells[out--] = S.dyn_cells[ia--];
    } else {
      S.dyn_cells[out--] = DynCell{cells[ib], h};
      --ib;
    }
  }
  S.n_dyn_cells = n + take;
}

// zero the list's slots [S.n_dyn_cells, end) (end: the count before a keep_freed removal)
RSX_F void dyn_cells_zero_from(ArenaState& S, uint32_t end) {
  for (uint32_t r = S.n_dyn_cells; r < end; ++r) S.dyn_cells[r] = DynCell{0, 0};
}

RSX_F Box3 dyn_shape_box(const BodyConst& c, const Aff& t) {
  return c.shape == SHAPE_SPHERE ? sphere_box(c.sphere_margin, t.t) : compound_box(c, t);
}

// one dynamic body's swept box, sweep-and-prune update and ray-grid cells (phase3a runs the three in order)
RSX_F void phase3a_body(ArenaState& S, const StaticData& D, uint32_t d) {
  const V3 cbt = vs(kBreakingThreshold);
  {
    const BodyConst& c = D.bodies[D.dyn_body[d]];
    const Body& b = S.bodies[d];
    if (b.flags & CF_STATIC) return;
    Box3 bx = dyn_shape_box(c, b.xf);
    bx.lo -= cbt;
    bx.hi += cbt;
    Box3 b2 = dyn_shape_box(c, b.pred);
    b2.lo -= cbt;
    b2.hi += cbt;
    bx.lo = vmin(bx.lo, b2.lo);
    bx.hi = vmax(bx.hi, b2.hi);
    uint32_t h = D.dyn_handle[d];
    S.dyn_proxy[d].box = bx;
    uint16_t qmin[3], qmax[3];
    quantize_point(D, bx.lo, 0, qmin);
    quantize_point(D, bx.hi, 1, qmax);
    for (int ax = 0; ax < 3; ++ax) update_axis(S, D, ax, h, qmin[ax], qmax[ax]);
    uint32_t old = S.dyn_proxy[d].cell, ni[3];
    cell_indices(D, bx.lo, ni);
    uint32_t nc = cell_of(D, ni);
    S.dyn_proxy[d].cell = nc;
    if (nc != old) {
      const uint32_t before = S.n_dyn_cells < (uint32_t)kMaxDynCells ? S.n_dyn_cells : (uint32_t)kMaxDynCells;
      dyn_cells_block(S, D, false, h, S.dyn_proxy[d].idx, true);
      S.dyn_proxy[d].idx[0] = ni[0];
      S.dyn_proxy[d].idx[1] = ni[1];
      S.dyn_proxy[d].idx[2] = ni[2];
      dyn_cells_block(S, D, true, h, ni);
      dyn_cells_zero_from(S, before);
    }
  }
}
RSX_F void phase3a(ArenaState& S, const StaticData& D) {
  for (uint32_t d = 0; d < (uint32_t)kDyn; ++d) phase3a_body(S, D, d);
}

// ---- construction of a consistent broadphase for a fresh state (not a phase) ----
// Bodies at their transforms with no motion: the swept boxes are the shapes' boxes, the edges of every handle are
// sorted (ties by handle), the pairs are exactly the filtered 3-axis overlaps of the sorted edge order (ascending
// handle pairs), and the ray-grid entries are those the blocks of the three bodies add in body order.
RSX_F void set_body_pose(Body& b, const BodyConst& c, const Aff& xf, V3 lin_vel, V3 ang_vel) {
  b.activation = ACT_ACTIVE;
  b.deactivation_time = 0.0f;
  b.quat = quat_from_m3(xf.m);
  b.xf = xf;
  b.pred = xf;
  b.lin_vel = lin_vel;
  b.ang_vel = ang_vel;
  update_inertia(b, c);
  clear_accum(b);
  b.damp_cache = 0.0f;
  b.damp_cache_dt = 0.0f;
  b.damp_cache_value = 0.0f;
}

RSX_HD inline void init_broadphase(ArenaState& S, const StaticData& D) {
  Box3 boxes[kHandles];
  for (int h = 1; h < kHandles; ++h) boxes[h] = D.proxies[h].box;
  const V3 cbt = vs(kBreakingThreshold);
  for (int d = 0; d < kDyn; ++d) {
    Box3 bx = dyn_shape_box(D.bodies[D.dyn_body[d]], S.bodies[d].xf);
    bx.lo -= cbt;
    bx.hi += cbt;
    S.dyn_proxy[d].box = bx;
    boxes[D.dyn_handle[d]] = bx;
  }
  for (int ax = 0; ax < 3; ++ax) {
    struct E { uint16_t pos, h; };
    E es[kEdges];
    int n = 0;
    for (int h = 1; h < kHandles; ++h) {
      uint16_t lo[3], hi[3];
      quantize_point(D, boxes[h].lo, 0, lo);
      quantize_point(D, boxes[h].hi, 1, hi);
      es[n++] = E{lo[ax], (uint16_t)h};
      es[n++] = E{hi[ax], (uint16_t)h};
    }
    for (int i = 1; i < n; ++i) {  // insertion sort by (pos, handle)
      E k = es[i];
      int j = i - 1;
      while (j >= 0 && (es[j].pos > k.pos || (es[j].pos == k.pos && es[j].h > k.h))) {
        es[j + 1] = es[j];
        --j;
      }
      es[j + 1] = k;
    }
    S.edges[ax][0] = Edge{0, 0};
    for (int i = 0; i < n; ++i) {
      S.edges[ax][i + 1] = Edge{es[i].pos, es[i].h};
      if (es[i].pos & 1) S.handle_edges[es[i].h].hi[ax] = (uint16_t)(i + 1);
      else S.handle_edges[es[i].h].lo[ax] = (uint16_t)(i + 1);
    }
    S.edges[ax][kEdges - 1] = Edge{(uint16_t)D.sap_sentinel, 0};
    S.handle_edges[0].lo[ax] = 0;
    S.handle_edges[0].hi[ax] = (uint16_t)(kEdges - 1);
  }
  S.n_pairs = 0;
  for (uint32_t a = 1; a < (uint32_t)kHandles; ++a)
    for (uint32_t b = a + 1; b < (uint32_t)kHandles; ++b) {
      bool ov = true;
      for (int ax = 0; ax < 3; ++ax) {
        const HandleEdges& A = S.handle_edges[a];
        const HandleEdges& B = S.handle_edges[b];
        if (A.hi[ax] < B.lo[ax] || B.hi[ax] < A.lo[ax]) ov = false;
      }
      if (ov) add_pair(S, D, a, b);
    }
  S.n_dyn_cells = 0;
  for (int d = 0; d < kDyn; ++d) {
    uint32_t ni[3];
    cell_indices(D, S.dyn_proxy[d].box.lo, ni);
    S.dyn_proxy[d].cell = cell_of(D, ni);
    S.dyn_proxy[d].idx[0] = ni[0];
    S.dyn_proxy[d].idx[1] = ni[1];
    S.dyn_proxy[d].idx[2] = ni[2];
    dyn_cells_block(S, D, true, D.dyn_handle[d], ni);
  }
}

}  // namespace sim
}  // namespace rsx
