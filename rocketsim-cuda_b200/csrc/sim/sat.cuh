// The car's box against one arena triangle, in the box's frame (RocketSim V3 box_triangle_sat.rs as the reference
// restates it in cuda/sim/box_triangle_sat.cuh:46-683): separating-axis sweep (3 box faces, the triangle face, 9 edge
// crosses), then either the closest feature pair among 47 candidates (3 clamped vertices, 8 corners, 36 edge-edge
// pairs) with the flat-tie snap, or the penetration witness of the axis kind.  Same axis order, same tie rules.
#pragma once
#include "base.cuh"

namespace rsx {
namespace sim {

constexpr float kTieEps = 1e-4f;
struct SatHit { V3 point_world; float distance; };
struct FeatPair { V3 on_box, on_tri; float d2; };
enum { AX_NONE = 0, AX_TRI = 1, AX_BOX = 2, AX_EDGE = 3 };
struct AxisKind { int tag, box_axis, tri_edge; };
struct Sweep {
  bool has_sep;
  float best_gap;
  V3 sep_axis;
  float best_overlap;
  V3 pen_axis, pen_raw;
  AxisKind kind;
};

RSX_F void gap_overlap(V3 a, const V3 q[3], V3 h, float* gap, float* ov, float* side) {
  float r = fadd(fadd(fmul(h.x, fabs_(a.x)), fmul(h.y, fabs_(a.y))), fmul(h.z, fabs_(a.z)));
  float d0 = dot(q[0], a), d1 = dot(q[1], a), d2 = dot(q[2], a);
  float mn = rmin(rmin(d0, d1), d2), mx = rmax(rmax(d0, d1), d2);
  if (mn > r) {
    *gap = fsub(mn, r); *ov = 0.0f; *side = 1.0f;
  } else if (mx < fneg(r)) {
    *gap = fsub(fneg(r), mx); *ov = 0.0f; *side = -1.0f;
  } else {
    *gap = 0.0f;
    *ov = rmax(rmin(fadd(mx, r), fsub(r, mn)), 0.0f);
    *side = 0.0f;
  }
}
// true when the axis proves the pair apart beyond reach
RSX_NOINL RSX_HD inline bool consider_axis(Sweep* s, V3 a, AxisKind kind, const V3 q[3], V3 h, float margin, float maxd) {
  float gap, ov, side;
  gap_overlap(a, q, h, &gap, &ov, &side);
  if (gap > 0.0f) {
    if (fsub(gap, margin) >= maxd) return true;
    if (!s->has_sep || gap > s->best_gap) {
      s->has_sep = true;
      s->best_gap = gap;
      s->sep_axis = side > 0.0f ? -a : a;
    }
  } else if (!s->has_sep && ov < s->best_overlap) {
    s->best_overlap = ov;
    s->kind = kind;
    s->pen_raw = a;
  }
  return false;
}
RSX_F bool box_face_axis(Sweep* s, float tmin, float tmax, float h, int ax, V3 unit, float margin, float maxd) {
  if (tmin > h) {
    float gap = fsub(tmin, h);
    if (fsub(gap, margin) >= maxd) return true;
    if (!s->has_sep || gap > s->best_gap) {
      s->has_sep = true;
      s->best_gap = gap;
      s->sep_axis = -unit;
    }
  } else if (tmax < fneg(h)) {
    float gap = fsub(fneg(h), tmax);
    if (fsub(gap, margin) >= maxd) return true;
    if (!s->has_sep || gap > s->best_gap) {
      s->has_sep = true;
      s->best_gap = gap;
      s->sep_axis = unit;
    }
  } else if (!s->has_sep) {
    float ov = rmax(rmin(fadd(tmax, h), fsub(h, tmin)), 0.0f);
    if (ov < s->best_overlap) {
      s->best_overlap = ov;
      s->kind = AxisKind{AX_BOX, ax, 0};
      s->pen_raw = unit;
    }
  }
  return false;
}
RSX_F V3 orient_pen(V3 a, V3 to_box, V3 face, bool has_face) {
  float s = dot(a, to_box);
  if (s < 0.0f) return -a;
  if (s > 1e-12f) return a;
  if (has_face && dot(a, face) > 0.0f) return -a;
  return a;
}
RSX_NOINL RSX_HD inline bool sat_sweep(V3 h, const V3 q[3], V3 tmn, V3 tmx, const V3 e[3], V3 face, bool has_face, V3 centroid, float margin,
                                float maxd, Sweep* s) {
  s->has_sep = false;
  s->best_gap = 0.0f;
  s->sep_axis = vzero();
  s->best_overlap = kFltMax;
  s->pen_axis = vzero();
  s->pen_raw = vzero();
  s->kind = AxisKind{AX_NONE, 0, 0};
  V3 to_box = -centroid;
  if (box_face_axis(s, tmn.x, tmx.x, h.x, 0, v3(1.0f, 0.0f, 0.0f), margin, maxd)) return false;
  if (box_face_axis(s, tmn.y, tmx.y, h.y, 1, v3(0.0f, 1.0f, 0.0f), margin, maxd)) return false;
  if (box_face_axis(s, tmn.z, tmx.z, h.z, 2, v3(0.0f, 0.0f, 1.0f), margin, maxd)) return false;
  if (has_face && consider_axis(s, face, AxisKind{AX_TRI, 0, 0}, q, h, margin, maxd)) return false;
  for (int bi = 0; bi < 3; ++bi) {
    V3 ba = bi == 0 ? v3(1.0f, 0.0f, 0.0f) : (bi == 1 ? v3(0.0f, 1.0f, 0.0f) : v3(0.0f, 0.0f, 1.0f));
    for (int ei = 0; ei < 3; ++ei) {
      V3 c = cross(ba, e[ei]);
      float l2 = len2(c);
      if (l2 < 1e-18f) continue;
      if (consider_axis(s, c / fsqrt(l2), AxisKind{AX_EDGE, bi, ei}, q, h, margin, maxd)) return false;
    }
  }
  if (!s->has_sep && s->kind.tag != AX_NONE) s->pen_axis = orient_pen(s->pen_raw, to_box, face, has_face);
  return true;
}
RSX_F V3 tri_support(const V3 q[3], V3 dir) {
  V3 best = q[0];
  float bd = dot(q[0], dir);
  for (int i = 1; i < 3; ++i) {
    float d = dot(q[i], dir);
    if (d > bd) {
      bd = d;
      best = q[i];
    }
  }
  return best;
}
RSX_NOINL RSX_HD inline int clip_half(const V3* in, int n, V3* out, int ax, float bound, bool above) {
  if (n == 0) return 0;
  int o = 0;
  V3 prev = in[n - 1];
  float pc = comp(prev, ax);
  float pd = above ? fsub(pc, bound) : fsub(bound, pc);
  for (int i = 0; i < n; ++i) {
    V3 v = in[i];
    float c = comp(v, ax);
    float d = above ? fsub(c, bound) : fsub(bound, c);
    if (d >= 0.0f) {
      if (pd < 0.0f) {
        float t = fdiv(pd, fsub(pd, d));
        out[o++] = prev + (v - prev) * t;
      }
      out[o++] = v;
    } else if (pd >= 0.0f) {
      float t = fdiv(pd, fsub(pd, d));
      out[o++] = prev + (v - prev) * t;
    }
    prev = v;
    pd = d;
  }
  return o;
}
RSX_NOINL RSX_HD inline bool clipped_centroid(V3 h, const V3 q[3], V3* res) {
  V3 poly[9], tmp[9];
  for (int i = 0; i < 9; ++i) {
    poly[i] = vzero();
    tmp[i] = vzero();
  }
  poly[0] = q[0];
  poly[1] = q[1];
  poly[2] = q[2];
  int n = 3;
  for (int ax = 0; ax < 3; ++ax) {
    float hh = comp(h, ax);
    n = clip_half(poly, n, tmp, ax, fneg(hh), true);
    if (n == 0) return false;
    n = clip_half(tmp, n, poly, ax, hh, false);
    if (n == 0) return false;
  }
  V3 sum = vzero();
  for (int i = 0; i < n; ++i) sum += poly[i];
  *res = sum / i2f(n);
  return true;
}
RSX_F V3 clamp_box(V3 p, V3 h) { return v3(rclamp(p.x, fneg(h.x), h.x), rclamp(p.y, fneg(h.y), h.y), rclamp(p.z, fneg(h.z), h.z)); }
RSX_F V3 closest_on_seg(V3 p, V3 a, V3 b) {
  V3 ab = b - a;
  float den = dot(ab, ab);
  if (den < 1e-30f) return a;
  return a + ab * rclamp(fdiv(dot(p - a, ab), den), 0.0f, 1.0f);
}
RSX_F V3 closest_on_degenerate(V3 p, const V3 q[3]) {
  V3 c0 = closest_on_seg(p, q[0], q[1]), c1 = closest_on_seg(p, q[1], q[2]), c2 = closest_on_seg(p, q[2], q[0]);
  float d0 = len2(p - c0), d1 = len2(p - c1), d2 = len2(p - c2);
  if (d0 <= d1 && d0 <= d2) return c0;
  if (d1 <= d2) return c1;
  return c2;
}
// closest points of segments (p1, q1) and (p2, q2); the parallel case takes the middle of the overlap
RSX_NOINL RSX_HD inline void seg_seg(V3 p1, V3 q1, V3 p2, V3 q2, V3* o1, V3* o2) {
  V3 d1 = q1 - p1, d2 = q2 - p2, r = p1 - p2;
  float a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
  const float eps = 1e-30f;
  float s, t;
  if (a <= eps && e <= eps) {
    *o1 = p1;
    *o2 = p2;
    return;
  }
  if (a <= eps) {
    s = 0.0f;
    t = rclamp(fdiv(f, e), 0.0f, 1.0f);
  } else {
    float c = dot(d1, r);
    if (e <= eps) {
      t = 0.0f;
      s = rclamp(fdiv(fneg(c), a), 0.0f, 1.0f);
    } else {
      float b = dot(d1, d2);
      if (fmul(b, b) > fmul(fmul(0.99900025f, a), e)) {
        float t0 = fdiv(dot(p2 - p1, d1), a), t1 = fdiv(dot(q2 - p1, d1), a);
        float lo = rmax(0.0f, rmin(t0, t1)), hi = rmin(1.0f, rmax(t0, t1));
        if (lo <= hi) {
          float sm = fmul(fadd(lo, hi), 0.5f);
          V3 c1 = p1 + d1 * sm;
          float tm = rclamp(fdiv(dot(c1 - p2, d2), e), 0.0f, 1.0f);
          *o1 = c1;
          *o2 = p2 + d2 * tm;
          return;
        }
      }
      float den = fsub(fmul(a, e), fmul(b, b));
      s = den > eps ? rclamp(fdiv(fsub(fmul(b, f), fmul(c, e)), den), 0.0f, 1.0f) : 0.0f;
      t = fdiv(fadd(fmul(b, s), f), e);
      if (t < 0.0f) {
        t = 0.0f;
        s = rclamp(fdiv(fneg(c), a), 0.0f, 1.0f);
      } else if (t > 1.0f) {
        t = 1.0f;
        s = rclamp(fdiv(fsub(b, c), a), 0.0f, 1.0f);
      }
    }
  }
  *o1 = p1 + d1 * s;
  *o2 = p2 + d2 * t;
}
RSX_F V3 support_corner(V3 h, V3 d) {
  return v3(d.x < 0.0f ? fneg(h.x) : h.x, d.y < 0.0f ? fneg(h.y) : h.y, d.z < 0.0f ? fneg(h.z) : h.z);
}
RSX_F bool in_tri_eps(V3 p, const V3 q[3], V3 n) {
  const float E = 1e-6f;
  bool pos = false, neg = false;
  for (int i = 0; i < 3; ++i) {
    float s = dot(cross(q[(i + 1) % 3] - q[i], p - q[i]), n);
    if (s > E) pos = true;
    else if (s < fneg(E)) neg = true;
    if (pos && neg) return false;
  }
  return true;
}
RSX_F bool clip_seg_box(V3 a, V3 b, V3 h, V3* o0, V3* o1) {
  float t0 = 0.0f, t1 = 1.0f;
  V3 d = b - a;
  for (int ax = 0; ax < 3; ++ax) {
    float hh = comp(h, ax);
    for (int k = 0; k < 2; ++k) {
      bool mn = k == 0;
      float p = mn ? comp(d, ax) : fneg(comp(d, ax));
      float qv = mn ? fadd(comp(a, ax), hh) : fsub(hh, comp(a, ax));
      if (fabs_(p) < kEps) {
        if (qv < 0.0f) return false;
      } else {
        float r = fdiv(qv, p);
        if (p < 0.0f) {
          if (r > t1) return false;
          if (r > t0) t0 = r;
        } else {
          if (r < t0) return false;
          if (r < t1) t1 = r;
        }
      }
    }
  }
  if (t0 > t1) return false;
  *o0 = a + d * t0;
  *o1 = a + d * t1;
  return true;
}
RSX_NOINL RSX_HD inline bool pen_witness(V3 h, const V3 q[3], AxisKind k, V3 n, V3* res) {
  if (k.tag == AX_TRI) {
    float pd = dot(n, q[0]);
    V3 corner = support_corner(h, -n);
    V3 p = corner - n * fsub(dot(n, corner), pd);
    if (in_tri_eps(p, q, n)) {
      *res = p;
      return true;
    }
    return false;
  }
  if (k.tag == AX_BOX) {
    float deep = from_bits(0xFF800000u);
    for (int i = 0; i < 3; ++i) deep = rmax(deep, dot(n, q[i]));
    V3 tied[3];
    int nt = 0;
    for (int i = 0; i < 3; ++i)
      if (fabs_(fsub(dot(n, q[i]), deep)) <= kTieEps) tied[nt++] = q[i];
    if (nt == 0) return false;
    if (nt == 1) {
      *res = tied[0];
      return true;
    }
    if (nt == 2) {
      V3 a, b;
      if (!clip_seg_box(tied[0], tied[1], h, &a, &b)) return false;
      *res = (a + b) * 0.5f;
      return true;
    }
    return clipped_centroid(h, q, res);
  }
  if (k.tag == AX_EDGE) {
    V3 s = vsignum(-n);
    V3 st = h * s, en = h * s;
    set_comp(st, k.box_axis, comp(h, k.box_axis));
    set_comp(en, k.box_axis, fneg(comp(h, k.box_axis)));
    V3 c1, tp;
    seg_seg(st, en, q[k.tri_edge], q[(k.tri_edge + 1) % 3], &c1, &tp);
    *res = tp;
    return true;
  }
  return false;
}
RSX_NOINL RSX_HD inline V3 closest_on_tri(V3 p, const V3 q[3], V3 ab, V3 ac) {
  V3 ap = p - q[0];
  float d1 = dot(ab, ap), d2 = dot(ac, ap);
  if (d1 <= 0.0f && d2 <= 0.0f) return q[0];
  V3 bp = p - q[1];
  float d3 = dot(ab, bp), d4 = dot(ac, bp);
  if (d3 >= 0.0f && d4 <= d3) return q[1];
  float vc = fsub(fmul(d1, d4), fmul(d3, d2));
  if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) return q[0] + ab * fdiv(d1, fsub(d1, d3));
  V3 cp = p - q[2];
  float d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= 0.0f && d5 <= d6) return q[2];
  float vb = fsub(fmul(d5, d2), fmul(d1, d6));
  if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) return q[0] + ac * fdiv(d2, fsub(d2, d6));
  float va = fsub(fmul(d3, d6), fmul(d5, d4));
  if (va <= 0.0f && fsub(d4, d3) >= 0.0f && fsub(d5, d6) >= 0.0f) {
    float w = fdiv(fsub(d4, d3), fadd(fsub(d4, d3), fsub(d5, d6)));
    return q[1] + (q[2] - q[1]) * w;
  }
  float den = fadd(fadd(va, vb), vc);
  if (fabs_(den) < 1e-24f) return closest_on_degenerate(p, q);
  float v = fdiv(vb, den), w = fdiv(vc, den);
  return q[0] + ab * v + ac * w;
}
RSX_NOINL RSX_HD inline void tri_edge_box_edge(V3 tp, V3 td, float ta, V3 b0, V3 b1, V3* o_tri, V3* o_box) {
  V3 d2 = b1 - b0, r = tp - b0;
  float e = dot(d2, d2), f = dot(d2, r);
  const float eps = 1e-30f;
  if (ta <= eps) {
    if (e <= eps) {
      *o_tri = tp;
      *o_box = b0;
      return;
    }
    *o_tri = tp;
    *o_box = b0 + d2 * rclamp(fdiv(f, e), 0.0f, 1.0f);
    return;
  }
  if (e <= eps) {
    float c = dot(td, r);
    *o_tri = tp + td * rclamp(fdiv(fneg(c), ta), 0.0f, 1.0f);
    *o_box = b0;
    return;
  }
  float c = dot(td, r), b = dot(td, d2);
  if (fmul(b, b) > fmul(fmul(0.99900025f, ta), e)) {
    float t0 = fdiv(dot(b0 - tp, td), ta), t1 = fdiv(dot(b1 - tp, td), ta);
    float lo = rmax(0.0f, rmin(t0, t1)), hi = rmin(1.0f, rmax(t0, t1));
    if (lo <= hi) {
      float sm = fmul(fadd(lo, hi), 0.5f);
      V3 c1 = tp + td * sm;
      float tm = rclamp(fdiv(dot(c1 - b0, d2), e), 0.0f, 1.0f);
      *o_tri = c1;
      *o_box = b0 + d2 * tm;
      return;
    }
  }
  float den = fsub(fmul(ta, e), fmul(b, b));
  float s = den > eps ? rclamp(fdiv(fsub(fmul(b, f), fmul(c, e)), den), 0.0f, 1.0f) : 0.0f;
  float t = fdiv(fadd(fmul(b, s), f), e);
  if (t < 0.0f) {
    t = 0.0f;
    s = rclamp(fdiv(fneg(c), ta), 0.0f, 1.0f);
  } else if (t > 1.0f) {
    t = 1.0f;
    s = rclamp(fdiv(fsub(b, c), ta), 0.0f, 1.0f);
  }
  *o_tri = tp + td * s;
  *o_box = b0 + d2 * t;
}
constexpr int kPairs = 47;
RSX_NOINL RSX_HD inline void enum_pairs(V3 h, const V3 q[3], const V3 e[3], FeatPair* P) {
  int k = 0;
  for (int i = 0; i < 3; ++i) {
    V3 pb = clamp_box(q[i], h);
    P[k++] = FeatPair{pb, q[i], len2(pb - q[i])};
  }
  V3 ab = e[0], ac = q[2] - q[0];
  for (int ix = 0; ix < 2; ++ix)
    for (int iy = 0; iy < 2; ++iy)
      for (int iz = 0; iz < 2; ++iz) {
        V3 corner = v3(fmul(ix ? 1.0f : -1.0f, h.x), fmul(iy ? 1.0f : -1.0f, h.y), fmul(iz ? 1.0f : -1.0f, h.z));
        V3 pt = closest_on_tri(corner, q, ab, ac);
        P[k++] = FeatPair{corner, pt, len2(corner - pt)};
      }
  V3 c[8] = {v3(fneg(h.x), fneg(h.y), fneg(h.z)), v3(h.x, fneg(h.y), fneg(h.z)), v3(h.x, h.y, fneg(h.z)), v3(fneg(h.x), h.y, fneg(h.z)),
             v3(fneg(h.x), fneg(h.y), h.z),       v3(h.x, fneg(h.y), h.z),       v3(h.x, h.y, h.z),       v3(fneg(h.x), h.y, h.z)};
  const int be[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6}, {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
  for (int ti = 0; ti < 3; ++ti) {
    V3 tp = q[ti], td = e[ti];
    float ta = dot(td, td);
    for (int j = 0; j < 12; ++j) {
      V3 ot, ob;
      tri_edge_box_edge(tp, td, ta, c[be[j][0]], c[be[j][1]], &ot, &ob);
      P[k++] = FeatPair{ob, ot, len2(ob - ot)};
    }
  }
}
RSX_F FeatPair first_min(const FeatPair* P) {
  FeatPair best = P[0];
  float bd = best.d2;
  for (int i = 1; i < kPairs; ++i)
    if (P[i].d2 < bd) {
      bd = P[i].d2;
      best = P[i];
    }
  return best;
}
RSX_NOINL RSX_HD inline bool flat_tie(V3 h, const FeatPair* P, V3* r0, V3* r1) {
  float link = fmul(0.5f, max_elem(h));
  if (link <= 0.0f || !isfinite_(link)) return false;
  float slope0 = fdiv(kTieEps, link);
  float bd2 = kFltMax;
  for (int i = 0; i < kPairs; ++i)
    if (P[i].d2 < bd2) bd2 = P[i].d2;
  float bd = fsqrt(bd2);
  float link2 = fmul(link, link);
  float td = fadd(bd, kTieEps);
  float td2 = fmul(td, td);
  FeatPair tied[kPairs];
  int nt = 0;
  for (int i = 0; i < kPairs; ++i)
    if (P[i].d2 <= td2) tied[nt++] = P[i];
  if (nt == 0) return false;
  V3 ma = vzero(), mb = vzero();
  for (int i = 0; i < nt; ++i) {
    ma += tied[i].on_box;
    mb += tied[i].on_tri;
  }
  float inv = fdiv(1.0f, i2f(nt));
  ma *= inv;
  mb *= inv;
  float d0 = len(ma - mb);
  bool has_flat = false;
  FeatPair flat = {};
  float best_slope = slope0;
  for (int i = 0; i < kPairs; ++i) {
    const FeatPair& p = P[i];
    float sep2 = len2(p.on_tri - mb);
    if (sep2 <= link2) continue;
    float sep = fsqrt(sep2);
    float slope = fdiv(fsub(fsqrt(p.d2), d0), sep);
    if (slope <= best_slope) {
      V3 mida = (ma + p.on_box) * 0.5f, midb = (mb + p.on_tri) * 0.5f;
      if (len(mida - midb) <= fadd(d0, kTieEps)) {
        best_slope = slope;
        flat = p;
        has_flat = true;
      }
    }
  }
  FeatPair e0 = tied[0], e1 = tied[0];
  float span2 = 0.0f;
  int nc = nt + (has_flat ? 1 : 0);
  for (int ci = 0; ci < nc; ++ci) {
    FeatPair cand = ci < nt ? tied[ci] : flat;
    for (int pi = 0; pi < nc; ++pi) {
      const FeatPair& p = pi < nt ? tied[pi] : flat;
      float s2 = len2(cand.on_tri - p.on_tri);
      if (s2 > span2) {
        span2 = s2;
        e0 = cand;
        e1 = p;
      }
    }
  }
  if (span2 <= link2) return false;
  V3 mida = (e0.on_box + e1.on_box) * 0.5f, midb = (e0.on_tri + e1.on_tri) * 0.5f;
  if (len(mida - midb) > fadd(bd, kTieEps)) return false;
  *r0 = e0.on_tri;
  *r1 = e1.on_tri;
  return true;
}

// The SAT in three stages, for callers that spread the 47 feature pairs of one test over several threads:
// sat_front runs the sweep and returns SAT_NO, SAT_HIT (out set) or SAT_PAIRS (the test goes on from f); the pairs are
// feat_pair(f, 0..46) (enum_pairs' order); sat_back picks the closest pair, snaps flat ties and places the witness.
// The three in a row compute what box_triangle_sat (below, one call, the serial callers' form) computes, bit for bit.
struct SatFront {
  Aff box_xf;
  V3 hu, q[3], e[3], centroid, sep_axis;
  float margin, maxd, best_gap;
};
enum { SAT_NO = 0, SAT_HIT = 1, SAT_PAIRS = 2 };
RSX_F int sat_front(const Aff& box_xf, V3 hu, float margin, const V3 q[3], float maxd, SatHit* out, SatFront* f) {
  V3 tmn = vmin(vmin(q[0], q[1]), q[2]), tmx = vmax(vmax(q[0], q[1]), q[2]);
  for (int ax = 0; ax < 3; ++ax) {
    float a = comp(tmn, ax), b = comp(tmx, ax), h = comp(hu, ax);
    if (a > h) {
      if (fsub(fsub(a, h), margin) >= maxd) return SAT_NO;
    } else if (b < fneg(h) && fsub(fsub(fneg(h), b), margin) >= maxd) {
      return SAT_NO;
    }
  }
  V3 e0 = q[1] - q[0], e1 = q[2] - q[1], e2 = q[0] - q[2];
  V3 fc = cross(e0, -e2);
  float fl2 = len2(fc);
  bool has_face = fl2 > 1e-20f;
  V3 face = has_face ? fc / fsqrt(fl2) : vzero();
  V3 centroid = (q[0] + q[1] + q[2]) * 0.33333334f;
  V3 e[3] = {e0, e1, e2};
  Sweep sw;
  if (!sat_sweep(hu, q, tmn, tmx, e, face, has_face, centroid, margin, maxd, &sw)) return SAT_NO;
  if (sw.has_sep) {
    V3 nw = normalize_or_zero(box_xf.m * sw.sep_axis);
    if (len2(nw) < 0.5f) return SAT_NO;
    f->box_xf = box_xf;
    f->hu = hu;
    for (int i = 0; i < 3; ++i) {
      f->q[i] = q[i];
      f->e[i] = e[i];
    }
    f->centroid = centroid;
    f->sep_axis = sw.sep_axis;
    f->margin = margin;
    f->maxd = maxd;
    f->best_gap = sw.best_gap;
    return SAT_PAIRS;
  }
  if (sw.best_overlap == kFltMax) return SAT_NO;
  V3 n;
  if (len2(sw.pen_axis) > 0.5f) {
    n = sw.pen_axis;
  } else if (has_face) {
    float s = dot(face, -centroid);
    n = s < 0.0f ? -face : face;
  } else {
    return SAT_NO;
  }
  float dist = fsub(fneg(sw.best_overlap), margin);
  if (dist >= maxd) return SAT_NO;
  V3 pb;
  if (!pen_witness(hu, q, sw.kind, n, &pb))
    if (!clipped_centroid(hu, q, &pb)) pb = tri_support(q, n);
  V3 nw = normalize_or_zero(box_xf.m * n);
  if (len2(nw) < 0.5f) return SAT_NO;
  out->point_world = xform_point(box_xf, pb);
  out->distance = dist;
  return SAT_HIT;
}
// pair i of enum_pairs (0-2 clamped vertices, 3-10 corners in x / y / z bit order, 11-46 triangle edge x box edge)
RSX_F FeatPair feat_pair(const SatFront& f, int i) {
  const V3 h = f.hu;
  if (i < 3) {
    V3 pb = clamp_box(f.q[i], h);
    return FeatPair{pb, f.q[i], len2(pb - f.q[i])};
  }
  if (i < 11) {
    const int c = i - 3, ix = c >> 2, iy = (c >> 1) & 1, iz = c & 1;
    V3 corner = v3(fmul(ix ? 1.0f : -1.0f, h.x), fmul(iy ? 1.0f : -1.0f, h.y), fmul(iz ? 1.0f : -1.0f, h.z));
    V3 pt = closest_on_tri(corner, f.q, f.e[0], f.q[2] - f.q[0]);
    return FeatPair{corner, pt, len2(corner - pt)};
  }
  const int c = i - 11, ti = c / 12, j = c % 12;
  // box edge j of enum_pairs' table: corners (bit 0 x, bit 1 y, bit 2 z in its 0..7 numbering) of the edge's two ends
  const int be[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6}, {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
  V3 cn[2];
  for (int k = 0; k < 2; ++k) {
    const int ci = be[j][k];  // enum_pairs' corner order: (-,-,-) (+,-,-) (+,+,-) (-,+,-), then the same at +z
    const bool px = ci == 1 || ci == 2 || ci == 5 || ci == 6, py = ci == 2 || ci == 3 || ci == 6 || ci == 7, pz = ci >= 4;
    cn[k] = v3(px ? h.x : fneg(h.x), py ? h.y : fneg(h.y), pz ? h.z : fneg(h.z));
  }
  V3 tp = f.q[ti], td = f.e[ti];
  float ta = dot(td, td);
  V3 ot, ob;
  tri_edge_box_edge(tp, td, ta, cn[0], cn[1], &ot, &ob);
  return FeatPair{ob, ot, len2(ob - ot)};
}
RSX_F bool sat_back(const SatFront& sf, const FeatPair* P, SatHit* out) {
  FeatPair f = first_min(P);
  if (len2(f.on_box - f.on_tri) > 1e-24f) {
    float pl = len(f.on_box - f.on_tri);
    V3 pb = f.on_tri;
    bool snapped = false;
    V3 s0, s1;
    if (fsub(pl, sf.margin) < 0.0f && flat_tie(sf.hu, P, &s0, &s1)) {
      pb = closest_on_seg(sf.centroid, s0, s1);
      snapped = true;
    }
    float dist = snapped ? fsub(len(clamp_box(pb, sf.hu) - pb), sf.margin) : fsub(pl, sf.margin);
    if (dist >= sf.maxd) return false;
    out->point_world = xform_point(sf.box_xf, pb);
    out->distance = dist;
    return true;
  }
  V3 pb = tri_support(sf.q, sf.sep_axis);
  out->point_world = xform_point(sf.box_xf, pb);
  out->distance = fsub(sf.best_gap, sf.margin);
  return true;
}

RSX_NOINL RSX_HD inline bool box_triangle_sat(const Aff& box_xf, V3 hu, float margin, const V3 q[3], float maxd, SatHit* out) {
  V3 tmn = vmin(vmin(q[0], q[1]), q[2]), tmx = vmax(vmax(q[0], q[1]), q[2]);
  for (int ax = 0; ax < 3; ++ax) {
    float a = comp(tmn, ax), b = comp(tmx, ax), h = comp(hu, ax);
    if (a > h) {
      if (fsub(fsub(a, h), margin) >= maxd) return false;
    } else if (b < fneg(h) && fsub(fsub(fneg(h), b), margin) >= maxd) {
      return false;
    }
  }
  V3 e0 = q[1] - q[0], e1 = q[2] - q[1], e2 = q[0] - q[2];
  V3 fc = cross(e0, -e2);
  float fl2 = len2(fc);
  bool has_face = fl2 > 1e-20f;
  V3 face = has_face ? fc / fsqrt(fl2) : vzero();
  V3 centroid = (q[0] + q[1] + q[2]) * 0.33333334f;
  V3 e[3] = {e0, e1, e2};
  Sweep sw;
  if (!sat_sweep(hu, q, tmn, tmx, e, face, has_face, centroid, margin, maxd, &sw)) return false;
  if (sw.has_sep) {
    V3 nw = normalize_or_zero(box_xf.m * sw.sep_axis);
    if (len2(nw) < 0.5f) return false;
    RSX_ZONE_BEGIN(z_fp);
    FeatPair P[kPairs];
    enum_pairs(hu, q, e, P);
    FeatPair f = first_min(P);
    RSX_ZONE_END(z_fp, 4);
    if (len2(f.on_box - f.on_tri) > 1e-24f) {
      float pl = len(f.on_box - f.on_tri);
      V3 pb = f.on_tri;
      bool snapped = false;
      V3 s0, s1;
      if (fsub(pl, margin) < 0.0f && flat_tie(hu, P, &s0, &s1)) {
        pb = closest_on_seg(centroid, s0, s1);
        snapped = true;
      }
      float dist = snapped ? fsub(len(clamp_box(pb, hu) - pb), margin) : fsub(pl, margin);
      if (dist >= maxd) return false;
      out->point_world = xform_point(box_xf, pb);
      out->distance = dist;
      return true;
    }
    V3 pb = tri_support(q, sw.sep_axis);
    out->point_world = xform_point(box_xf, pb);
    out->distance = fsub(sw.best_gap, margin);
    return true;
  }
  if (sw.best_overlap == kFltMax) return false;
  V3 n;
  if (len2(sw.pen_axis) > 0.5f) {
    n = sw.pen_axis;
  } else if (has_face) {
    float s = dot(face, -centroid);
    n = s < 0.0f ? -face : face;
  } else {
    return false;
  }
  float dist = fsub(fneg(sw.best_overlap), margin);
  if (dist >= maxd) return false;
  V3 pb;
  if (!pen_witness(hu, q, sw.kind, n, &pb))
    if (!clipped_centroid(hu, q, &pb)) pb = tri_support(q, n);
  V3 nw = normalize_or_zero(box_xf.m * n);
  if (len2(nw) < 0.5f) return false;
  out->point_world = xform_point(box_xf, pb);
  out->distance = dist;
  return true;
}

}  // namespace sim
}  // namespace rsx
