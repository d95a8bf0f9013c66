// P4: islands of the dynamic bodies, sleeping, and the island sort of the active manifolds
//     (reference: cuda/sim/simulation_island_manager.cuh:37-152).
// P5: Bullet's sequential-impulse solver: rows from the active manifolds (special ball-world points as split-only
//     rows plus one synthetic row per body), 10 split-impulse iterations, up to 10 PGS iterations, then the velocity
//     and split-push integration (seq_impulse_constraint_solver.cuh:37-314, solver_constraint.cuh:62-310).
#pragma once
#include "base.cuh"

namespace rsx {
namespace sim {

RSX_F int island_root(int* par, int i) {
  int r = i;
  while (par[r] != r) r = par[r];
  int c = i;
  while (par[c] != r && c != r) {
    int n = par[c];
    par[c] = r;
    c = n;
  }
  return r;
}
// Hoare partition sort of `idx` by keys[idx], V3's recursion order (left range first) with an explicit stack
RSX_F void hoare(uint32_t* idx, int n, const int* keys) {
  if (n <= 1) return;
  int lo_s[32], hi_s[32], sp = 0;
  lo_s[0] = 0;
  hi_s[0] = n - 1;
  sp = 1;
  while (sp > 0) {
    --sp;
    int lo = lo_s[sp], hi = hi_s[sp];
    int i = lo, j = hi;
    int pivot = keys[idx[(lo + hi) / 2]];
    for (;;) {
      while (keys[idx[i]] < pivot) ++i;
      while (pivot < keys[idx[j]]) --j;
      if (i > j) break;
      uint32_t t = idx[i];
      idx[i] = idx[j];
      idx[j] = t;
      ++i;
      if (j == 0) break;
      --j;
      if (i > j) break;
    }
    if (i < hi) { lo_s[sp] = i; hi_s[sp] = hi; ++sp; }
    if (lo < j) { lo_s[sp] = lo; hi_s[sp] = j; ++sp; }
  }
}

RSX_F void phase4(ArenaState& S, const StaticData& D) {
  const int n = (int)S.n_active;
  int par[kDyn];
  for (int d = 0; d < kDyn; ++d) par[d] = d;
  for (uint32_t p = 0; p < S.n_pairs; ++p) {
    const ProxyConst& x0 = D.proxies[S.pairs[p].h0];
    const ProxyConst& x1 = D.proxies[S.pairs[p].h1];
    if ((x0.group & 2u) || (x1.group & 2u)) continue;
    int a = slot(D, x0.body), b = slot(D, x1.body);
    if (a < 0 || b < 0) continue;
    if ((S.bodies[a].flags & CF_NO_RESPONSE) || (S.bodies[b].flags & CF_NO_RESPONSE)) continue;
    int ra = island_root(par, a), rb = island_root(par, b);
    if (ra != rb) par[ra] = rb;
  }
  int tag[kDyn];
  for (int d = 0; d < kDyn; ++d) tag[d] = island_root(par, d);
  bool live[kDyn] = {false, false, false};
  for (int d = 0; d < kDyn; ++d)
    if (S.bodies[d].activation == ACT_ACTIVE) live[tag[d]] = true;
  for (int d = 0; d < kDyn; ++d)
    if (!live[tag[d]] && S.bodies[d].activation == ACT_WANTS_SLEEP) {
      set_activation(S.bodies[d], ACT_SLEEPING);
      S.bodies[d].lin_vel = vzero();
      S.bodies[d].ang_vel = vzero();
    }
  if (n <= 1) return;
  uint32_t idx[kMaxActive];
  for (int i = 0; i < n; ++i) idx[i] = S.active[i];
  for (int i = 1; i < n; ++i) {
    uint32_t v = idx[i];
    int j = i - 1;
    while (j >= 0 && idx[j] > v) {
      idx[j + 1] = idx[j];
      --j;
    }
    idx[j + 1] = v;
  }
  int keys[kMaxManifolds];
  for (int i = 0; i < n; ++i) {
    const Manifold& m = S.manifolds[idx[i]];
    int d0 = slot(D, m.body0), d1 = slot(D, m.body1);
    int t0 = d0 < 0 ? -1 : tag[d0], t1 = d1 < 0 ? -1 : tag[d1];
    keys[idx[i]] = t0 >= 0 ? t0 : t1;
  }
  hoare(idx, n, keys);
  for (int i = 0; i < n; ++i) S.active[i] = idx[i];
}

// ---- P5 ----
constexpr float kErp2 = 0.8f, kSplitThreshold = 1e30f, kSplitTurnErp = 0.1f;
constexpr int kIterations = 10, kMaxRows = 32, kMaxSolverBodies = 8, kNone = -1;

struct SBody {
  V3 dlin, dang, inv_mass, push, turn, lin, ang, ext_f, ext_t;
  int has_orig, orig;
};
struct Row {
  V3 r1xn, n1, r2xn, n2, ang_a, ang_b;
  float push_imp, imp, friction, jinv, rhs, lo, hi, rhs_pen;
  int fric_idx, a, b, split_only;
};
struct CPoint { V3 n; float friction, restitution, dist; };
struct Side { const Body* rb; const BodyConst* c; };
struct Special { int obj; V3 normal; float lever, friction, restitution; uint32_t count; };
struct Solver {
  SBody bodies[kMaxSolverBodies];
  Row contact[kMaxRows];
  Row fric[kMaxRows];
  Special spec[4];
  int nb, nc, nf, ns, fixed;
  int comp[kDyn];
};

RSX_F SBody sbody_fixed() {
  SBody b;
  b.dlin = b.dang = b.inv_mass = b.push = b.turn = b.lin = b.ang = b.ext_f = b.ext_t = vzero();
  b.has_orig = 0;
  b.orig = 0;
  return b;
}
RSX_F SBody sbody_of(const Body& rb, const BodyConst& c, int d) {
  SBody b = sbody_fixed();
  b.inv_mass = c.inv_mass3;
  b.lin = rb.lin_vel;
  b.ang = rb.ang_vel;
  b.ext_f = rb.acc_lin;
  b.ext_t = rb.acc_ang;
  b.has_orig = 1;
  b.orig = d;
  return b;
}
RSX_F float bdot(V3 a, V3 b) {
  V3 r = a * b;
  return fadd(r.x, fadd(r.y, r.z));
}
RSX_F V3 plane_space(V3 n) {
  if (fabs_(n.z) > 0.70710678118654752440f) {
    float a = fadd(fmul(n.y, n.y), fmul(n.z, n.z));
    float k = fdiv(1.0f, fsqrt(a));
    return {0.0f, fmul(fneg(n.z), k), fmul(n.y, k)};
  }
  float a = fadd(fmul(n.x, n.x), fmul(n.y, n.y));
  float k = fdiv(1.0f, fsqrt(a));
  return {fmul(fneg(n.y), k), fmul(n.x, k), 0.0f};
}
RSX_F V3 sb_vel(const SBody& b, V3 rel) { return b.lin + b.ext_f + cross(b.ang + b.ext_t, rel); }
RSX_F V3 lat_dir(const CPoint& cp, const SBody& a, const SBody& b, V3 r1, V3 r2) {
  V3 v = sb_vel(a, r1) - sb_vel(b, r2);
  float rv = dot(cp.n, v);
  V3 lat = v - cp.n * rv;
  float l = len2(lat);
  if (l > 1.1920929e-7f) return lat * fdiv(1.0f, fsqrt(l));
  return plane_space(cp.n);
}
RSX_F Row row0(int a, int b, int fi, float fr, float lo, float hi) {
  Row r;
  r.r1xn = r.n1 = r.r2xn = r.n2 = r.ang_a = r.ang_b = vzero();
  r.push_imp = r.imp = r.jinv = r.rhs = r.rhs_pen = 0.0f;
  r.friction = fr;
  r.lo = lo;
  r.hi = hi;
  r.fric_idx = fi;
  r.a = a;
  r.b = b;
  r.split_only = 0;
  return r;
}
RSX_F Row contact_row(int a, int b, const SBody& sa, const SBody& sb, Side s0, Side s1, V3 r1, V3 r2, const CPoint& cp, int fi, float dt) {
  Row r = row0(a, b, fi, cp.friction, 0.0f, 1e10f);
  float inv_dt = fdiv(1.0f, dt);
  V3 n = cp.n;
  r.imp = 0.0f;
  float den0 = 0.0f, v1n = 0.0f;
  V3 vel0 = vzero();
  if (s0.rb) {
    V3 ta = cross(r1, n);
    r.ang_a = mul_t(s0.rb->inv_inertia_world, ta);
    V3 vec = cross(r.ang_a, r1);
    den0 = fadd(s0.c->inv_mass, dot(n, vec));
    vel0 = s0.rb->lin_vel + cross(s0.rb->ang_vel, r1);
    r.n1 = n;
    r.r1xn = ta;
    v1n = fadd(dot(r.n1, sa.lin + sa.ext_f), dot(r.r1xn, sa.ang + sa.ext_t));
  }
  float den1 = 0.0f, v2n = 0.0f;
  V3 vel1 = vzero();
  if (s1.rb) {
    V3 ta = cross(r2, n);
    r.ang_b = mul_t(s1.rb->inv_inertia_world, -ta);
    V3 vec = cross(-r.ang_b, r2);
    den1 = fadd(s1.c->inv_mass, dot(n, vec));
    vel1 = s1.rb->lin_vel + cross(s1.rb->ang_vel, r2);
    r.n2 = -n;
    r.r2xn = -ta;
    v2n = fadd(dot(r.n2, sb.lin + sb.ext_f), dot(r.r2xn, sb.ang + sb.ext_t));
  }
  r.jinv = fdiv(1.0f, fadd(den0, den1));
  float rel = dot(n, vel0 - vel1);
  float rest = rmax(fmul(cp.restitution, fneg(rel)), 0.0f);
  float pen = cp.dist;
  float perr = pen > 0.0f ? 0.0f : fmul(fmul(fneg(pen), kErp2), inv_dt);
  rel = fadd(v1n, v2n);
  float verr = fsub(rest, rel);
  float pi = fmul(perr, r.jinv), vi = fmul(verr, r.jinv);
  if (pen > kSplitThreshold) {
    r.rhs = fadd(pi, vi);
    r.rhs_pen = 0.0f;
  } else {
    r.rhs = vi;
    r.rhs_pen = pi;
  }
  return r;
}
RSX_F Row split_row(int a, int b, Side s0, Side s1, V3 r1, V3 r2, const CPoint& cp, float dt) {
  Row r = row0(a, b, -1, cp.friction, 0.0f, 1e10f);
  r.split_only = 1;
  V3 n = cp.n;
  float den0 = 0.0f, den1 = 0.0f;
  if (s0.rb) {
    V3 ta = cross(r1, n);
    r.ang_a = mul_t(s0.rb->inv_inertia_world, ta);
    den0 = fadd(s0.c->inv_mass, dot(n, cross(r.ang_a, r1)));
    r.n1 = n;
    r.r1xn = ta;
  }
  if (s1.rb) {
    V3 ta = cross(r2, n);
    r.ang_b = mul_t(s1.rb->inv_inertia_world, -ta);
    den1 = fadd(s1.c->inv_mass, dot(n, cross(-r.ang_b, r2)));
    r.n2 = -n;
    r.r2xn = -ta;
  }
  r.jinv = fdiv(1.0f, fadd(den0, den1));
  float inv_dt = fdiv(1.0f, dt);
  float pen = cp.dist;
  float perr = pen > 0.0f ? 0.0f : fmul(fmul(fneg(pen), kErp2), inv_dt);
  float pi = fmul(perr, r.jinv);
  r.rhs_pen = pen > kSplitThreshold ? 0.0f : pi;
  return r;
}
RSX_F Row friction_row(int a, int b, const SBody& sa, const SBody& sb, Side s0, Side s1, V3 r1, V3 r2, float fr, V3 axis, int fi) {
  Row r = row0(a, b, fi, fr, fneg(fr), fr);
  float v1n = 0.0f, den1 = 0.0f;
  if (s0.rb) {
    r.n1 = axis;
    r.r1xn = cross(r1, r.n1);
    r.ang_a = mul_t(s0.rb->inv_inertia_world, r.r1xn);
    den1 = fadd(s0.c->inv_mass, dot(axis, cross(r.ang_a, r1)));
    v1n = fadd(dot(r.n1, sa.lin + sa.ext_f), dot(r.r1xn, sa.ang));
  }
  float v2n = 0.0f, den2 = 0.0f;
  if (s1.rb) {
    r.n2 = -axis;
    r.r2xn = cross(r2, r.n2);
    r.ang_b = mul_t(s1.rb->inv_inertia_world, r.r2xn);
    den2 = fadd(s1.c->inv_mass, dot(axis, cross(-r.ang_b, r2)));
    v2n = fadd(dot(r.n2, sb.lin + sb.ext_f), dot(r.r2xn, sb.ang));
  }
  r.jinv = fdiv(1.0f, fadd(den1, den2));
  r.rhs = fmul(fneg(fadd(v1n, v2n)), r.jinv);
  return r;
}
RSX_F float resolve_split(Row& c, SBody& a, SBody& b) {
  if (c.rhs_pen == 0.0f) return 0.0f;
  float di = c.rhs_pen;
  float d1 = a.has_orig ? fadd(bdot(c.n1, a.push), bdot(c.r1xn, a.turn)) : 0.0f;
  float d2 = b.has_orig ? fadd(bdot(c.n2, b.push), bdot(c.r2xn, b.turn)) : 0.0f;
  di = fsub(di, fmul(d1, c.jinv));
  di = fsub(di, fmul(d2, c.jinv));
  float sum = fadd(c.push_imp, di);
  if (sum < c.lo) {
    di = fsub(c.lo, c.push_imp);
    c.push_imp = c.lo;
  } else {
    c.push_imp = sum;
  }
  if (a.has_orig) {
    a.push = a.push + c.n1 * a.inv_mass * di;
    a.turn = a.turn + c.ang_a * di;
  }
  if (b.has_orig) {
    b.push = b.push + c.n2 * b.inv_mass * di;
    b.turn = b.turn + c.ang_b * di;
  }
  return fdiv(di, c.jinv);
}
RSX_F float resolve_row(Row& c, SBody& a, SBody& b, bool two_sided) {
  float di = c.rhs;
  float d1 = a.has_orig ? fadd(bdot(c.n1, a.dlin), bdot(c.r1xn, a.dang)) : 0.0f;
  float d2 = b.has_orig ? fadd(bdot(c.n2, b.dlin), bdot(c.r2xn, b.dang)) : 0.0f;
  di = fsub(di, fmul(d1, c.jinv));
  di = fsub(di, fmul(d2, c.jinv));
  float sum = fadd(c.imp, di);
  if (sum < c.lo) {
    di = fsub(c.lo, c.imp);
    c.imp = c.lo;
  } else if (two_sided && sum > c.hi) {
    di = fsub(c.hi, c.imp);
    c.imp = c.hi;
  } else {
    c.imp = sum;
  }
  if (a.has_orig) {
    a.dlin = a.dlin + c.n1 * a.inv_mass * di;
    a.dang = a.dang + c.ang_a * di;
  }
  if (b.has_orig) {
    b.dlin = b.dlin + c.n2 * b.inv_mass * di;
    b.dang = b.dang + c.ang_b * di;
  }
  return fdiv(di, c.jinv);
}

RSX_F int solver_body(Solver& sv, ArenaState& S, const StaticData& D, int d, uint32_t w) {
  if (d < 0) {
    if (sv.fixed >= 0) return sv.fixed;
    int id = sv.nb;
    sv.fixed = id;
    sv.bodies[sv.nb++] = sbody_fixed();
    return id;
  }
  if (sv.comp[d] >= 0) return sv.comp[d];
  int id = sv.nb;
  sv.comp[d] = id;
  sv.bodies[sv.nb++] = sbody_of(S.bodies[d], D.bodies[w], d);
  return id;
}
RSX_F void add_special(Solver& sv, int obj, V3 n, float lever, float fr, float re) {
  for (int i = 0; i < sv.ns; ++i) {
    Special& a = sv.spec[i];
    if (a.obj == obj) {
      a.normal += n;
      a.lever = fadd(a.lever, lever);
      a.friction = fadd(a.friction, fr);
      a.restitution = fadd(a.restitution, re);
      a.count += 1;
      return;
    }
  }
  sv.spec[sv.ns++] = Special{obj, n, lever, fr, re, 1u};
}
RSX_F void emit_special(Solver& sv, ArenaState& S, const StaticData& D, const Special& acc, float dt) {
  float ns = u2f(acc.count);
  V3 mn = normalize_or_zero(acc.normal / ns);
  float ml = fdiv(acc.lever, ns), mf = fdiv(acc.friction, ns), mr = fdiv(acc.restitution, ns);
  int d = acc.obj;
  int ia = sv.comp[d];
  int ib;
  if (sv.fixed >= 0) {
    ib = sv.fixed;
  } else {
    ib = sv.nb;
    sv.fixed = ib;
    sv.bodies[sv.nb++] = sbody_fixed();
  }
  const SBody& sa = sv.bodies[ia];
  const SBody& sb = sv.bodies[ib];
  V3 r1 = mn * fneg(ml), r2 = vzero();
  CPoint cp = {mn, mf, mr, 0.0f};
  Side s0 = {sa.has_orig ? &S.bodies[d] : nullptr, &D.bodies[D.dyn_body[d]]};
  Side s1 = {nullptr, nullptr};
  int fi = sv.nc;
  if (sv.nc >= kMaxRows || sv.nf >= kMaxRows) {
    S.overflow[OVF_ACTIVE]++;
    return;
  }
  sv.contact[sv.nc++] = contact_row(ia, ib, sa, sb, s0, s1, r1, r2, cp, fi, dt);
  V3 lat = lat_dir(cp, sa, sb, r1, r2);
  sv.fric[sv.nf++] = friction_row(ia, ib, sa, sb, s0, s1, r1, r2, cp.friction, lat, fi);
}

// P5 in three steps a kernel can barrier between: the rows (setup), the split-impulse and PGS iterations, and the
// integration of the results (finish); phase5 runs them in order.
RSX_F void phase5_setup(ArenaState& S, const StaticData& D, Solver& sv) {
  const float dt = fdiv(1.0f, 120.0f);
  sv.nb = sv.nc = sv.nf = sv.ns = 0;
  sv.fixed = kNone;
  // bodies: the active dynamic ones first, in order
  for (int d = 0; d < kDyn; ++d) {
    sv.comp[d] = kNone;
    if (!awake(S.bodies[d])) continue;
    sv.comp[d] = sv.nb;
    sv.bodies[sv.nb++] = sbody_of(S.bodies[d], D.bodies[D.dyn_body[d]], d);
  }
  for (uint32_t ai = 0; ai < S.n_active; ++ai) {
    const Manifold& m = S.manifolds[S.active[ai]];
    int d0 = slot(D, m.body0), d1 = slot(D, m.body1);
    int ia = solver_body(sv, S, D, d0, m.body0);
    int ib = solver_body(sv, S, D, d1, m.body1);
    V3 t0 = d0 >= 0 ? S.bodies[d0].xf.t : D.bodies[m.body0].pose.t;
    V3 t1 = d1 >= 0 ? S.bodies[d1].xf.t : D.bodies[m.body1].pose.t;
    for (uint32_t pi = 0; pi < m.n; ++pi) {
      const MPoint& p = m.pts[pi];
      V3 r1 = p.world_a - t0, r2 = p.world_b - t1;
      CPoint cp = {p.normal_b, p.friction, p.restitution, p.dist};
      Side s0 = {sv.bodies[ia].has_orig ? &S.bodies[d0] : nullptr, d0 >= 0 ? &D.bodies[m.body0] : nullptr};
      Side s1 = {sv.bodies[ib].has_orig ? &S.bodies[d1] : nullptr, d1 >= 0 ? &D.bodies[m.body1] : nullptr};
      if (p.special) {
        if (sv.nc >= kMaxRows) S.overflow[OVF_ACTIVE]++;
        else sv.contact[sv.nc++] = split_row(ia, ib, s0, s1, r1, r2, cp, dt);
        int obj = -1;
        V3 lever = vzero();
        if (d0 >= 0) { obj = d0; lever = r1; }
        else if (d1 >= 0) { obj = d1; lever = r2; }
        if (obj >= 0) add_special(sv, obj, p.normal_b, len(lever), p.friction, p.restitution);
        continue;
      }
      int fi = sv.nc;
      V3 lat = lat_dir(cp, sv.bodies[ia], sv.bodies[ib], r1, r2);
      if (sv.nc >= kMaxRows || sv.nf >= kMaxRows) {
        S.overflow[OVF_ACTIVE]++;
        continue;
      }
      sv.contact[sv.nc++] = contact_row(ia, ib, sv.bodies[ia], sv.bodies[ib], s0, s1, r1, r2, cp, fi, dt);
      sv.fric[sv.nf++] = friction_row(ia, ib, sv.bodies[ia], sv.bodies[ib], s0, s1, r1, r2, p.friction, lat, fi);
    }
  }
  S.n_active = 0;
  for (int i = 0; i < kMaxActive; ++i) S.active[i] = 0;
  for (int i = 0; i < sv.ns; ++i) {
    Special acc = sv.spec[i];
    emit_special(sv, S, D, acc, dt);
  }
}

RSX_F void phase5_iterate(Solver& sv) {
  // split-impulse iterations
  {
    bool run[kMaxRows];
    int left = sv.nc;
    for (int i = 0; i < sv.nc; ++i) run[i] = true;
    for (int it = 0; it < kIterations && left != 0; ++it)
      for (int i = 0; i < sv.nc; ++i) {
        if (!run[i]) continue;
        Row& c = sv.contact[i];
        float r = resolve_split(c, sv.bodies[c.a], sv.bodies[c.b]);
        if (fmul(r, r) == 0.0f) {
          run[i] = false;
          --left;
        }
      }
  }
  for (int it = 0; it < kIterations; ++it) {
    float lsr = 0.0f;
    for (int i = 0; i < sv.nc; ++i) {
      Row& c = sv.contact[i];
      if (c.split_only) continue;
      float r = resolve_row(c, sv.bodies[c.a], sv.bodies[c.b], false);
      lsr = rmax(fmul(r, r), lsr);
    }
    for (int i = 0; i < sv.nf; ++i) {
      Row& c = sv.fric[i];
      float tot = sv.contact[c.fric_idx].imp;
      if (tot <= 0.0f) continue;
      float lim = fmul(c.friction, tot);
      c.lo = fneg(lim);
      c.hi = lim;
      float r = resolve_row(c, sv.bodies[c.a], sv.bodies[c.b], true);
      lsr = rmax(fmul(r, r), lsr);
    }
    if (lsr == 0.0f) break;
  }
}

RSX_F void phase5_finish(ArenaState& S, const StaticData& D, Solver& sv) {
  const float dt = fdiv(1.0f, 120.0f);
  // finish
  for (int i = 0; i < sv.nb; ++i) {
    SBody& b = sv.bodies[i];
    if (!b.has_orig) continue;
    Body& body = S.bodies[b.orig];
    b.lin += b.dlin;
    b.ang += b.dang;
    if (len2(b.push) != 0.0f || len2(b.turn) != 0.0f) {
      Aff wt = body.xf;
      if (body.flags & CF_NO_ANGULAR) {
        wt.t += b.push * dt;
      } else {
        Q4 q = body.quat;
        integrate(wt, q, b.push, b.turn * kSplitTurnErp, dt);  // transform_util.rs integrate_trans, the same steps
      }
      if ((body.flags & CF_NO_ANGULAR) == 0) body.quat = quat_from_m3(wt.m);
      body.xf = wt;
    }
    V3 lv = b.lin + b.ext_f, av = b.ang + b.ext_t;
    bool was = body.activation == ACT_SLEEPING;
    body.lin_vel = lv;
    body.ang_vel = av;
    if (was && (lv.x != 0.0f || lv.y != 0.0f || lv.z != 0.0f || av.x != 0.0f || av.y != 0.0f || av.z != 0.0f)) {
      set_activation(body, ACT_WANTS_SLEEP);
      body.deactivation_time = 0.0f;
    }
  }
}

RSX_F void phase5(ArenaState& S, const StaticData& D) {
  Solver sv;
  phase5_setup(S, D, sv);
  phase5_iterate(sv);
  phase5_finish(S, D, sv);
}

}  // namespace sim
}  // namespace rsx
