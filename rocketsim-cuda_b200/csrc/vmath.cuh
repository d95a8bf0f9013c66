// 3-vectors, column-major 3x3 matrices, affine transforms and quaternions with the exact operation order of glam
// 0.34.1's SSE2 paths (the order the reference reproduces in cuda/common/glam.cuh:27-309, which is RocketSim V3's):
//   dot3 = (x*x' + y*y') + z*z';  M*v = (c0*v.x + c1*v.y) + c2*v.z;  quat product as glam's rtm form;  normalize
//   divides by the length, normalize_or multiplies by the reciprocal.  Nothing is fused.
// The layout of every type is a run of 4-byte floats with no padding: they are the words of the arena state.
#pragma once
#include "fp.cuh"

namespace rsx {

struct V3 { float x, y, z; };
struct V4 { float x, y, z, w; };
struct Q4 { float x, y, z, w; };
struct M3 { V3 c0, c1, c2; };       // columns (glam's x_axis, y_axis, z_axis)
struct Aff { M3 m; V3 t; };         // matrix3, translation
struct Box3 { V3 lo, hi; };         // an axis-aligned box (min, max)

RSX_F V3 v3(float x, float y, float z) { return V3{x, y, z}; }
RSX_F V3 vs(float s) { return V3{s, s, s}; }
RSX_F V3 vzero() { return V3{0.0f, 0.0f, 0.0f}; }
RSX_F V3 operator+(V3 a, V3 b) { return {fadd(a.x, b.x), fadd(a.y, b.y), fadd(a.z, b.z)}; }
RSX_F V3 operator-(V3 a, V3 b) { return {fsub(a.x, b.x), fsub(a.y, b.y), fsub(a.z, b.z)}; }
RSX_F V3 operator*(V3 a, V3 b) { return {fmul(a.x, b.x), fmul(a.y, b.y), fmul(a.z, b.z)}; }
RSX_F V3 operator/(V3 a, V3 b) { return {fdiv(a.x, b.x), fdiv(a.y, b.y), fdiv(a.z, b.z)}; }
RSX_F V3 operator*(V3 a, float s) { return {fmul(a.x, s), fmul(a.y, s), fmul(a.z, s)}; }
RSX_F V3 operator*(float s, V3 a) { return {fmul(s, a.x), fmul(s, a.y), fmul(s, a.z)}; }
RSX_F V3 operator/(V3 a, float s) { return {fdiv(a.x, s), fdiv(a.y, s), fdiv(a.z, s)}; }
RSX_F V3 operator/(float s, V3 a) { return {fdiv(s, a.x), fdiv(s, a.y), fdiv(s, a.z)}; }
RSX_F V3 operator-(V3 a) { return {fneg(a.x), fneg(a.y), fneg(a.z)}; }
RSX_F V3& operator+=(V3& a, V3 b) { return a = a + b; }
RSX_F V3& operator-=(V3& a, V3 b) { return a = a - b; }
RSX_F V3& operator*=(V3& a, V3 b) { return a = a * b; }
RSX_F V3& operator*=(V3& a, float s) { return a = a * s; }
RSX_F float comp(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
RSX_F void set_comp(V3& a, int i, float v) {
  if (i == 0) a.x = v;
  else if (i == 1) a.y = v;
  else a.z = v;
}
RSX_F bool is_zero(V3 a) { return a.x == 0.0f && a.y == 0.0f && a.z == 0.0f; }

RSX_F float dot(V3 a, V3 b) { return fadd(fadd(fmul(a.x, b.x), fmul(a.y, b.y)), fmul(a.z, b.z)); }
RSX_F V3 cross(V3 a, V3 b) {
  return {fsub(fmul(a.y, b.z), fmul(b.y, a.z)), fsub(fmul(a.z, b.x), fmul(b.z, a.x)), fsub(fmul(a.x, b.y), fmul(b.x, a.y))};
}
RSX_F float len2(V3 a) { return dot(a, a); }
RSX_F float len(V3 a) { return fsqrt(dot(a, a)); }
RSX_F V3 normalize(V3 a) { return a / vs(fsqrt(dot(a, a))); }
// glam try_normalize / normalize_or: multiply by 1/length when that is finite and positive
RSX_F bool try_normalize(V3 a, V3* out) {
  float r = fdiv(1.0f, fsqrt(dot(a, a)));
  if (isfinite_(r) && r > 0.0f) {
    *out = a * r;
    return true;
  }
  return false;
}
RSX_F V3 normalize_or_zero(V3 a) {
  V3 r;
  return try_normalize(a, &r) ? r : vzero();
}
RSX_F V3 lerp(V3 a, V3 b, float s) { return a * fsub(1.0f, s) + b * s; }
RSX_F V3 vabs(V3 a) { return {fabs_(a.x), fabs_(a.y), fabs_(a.z)}; }
RSX_F V3 vmin(V3 a, V3 b) { return {sse_min(a.x, b.x), sse_min(a.y, b.y), sse_min(a.z, b.z)}; }
RSX_F V3 vmax(V3 a, V3 b) { return {sse_max(a.x, b.x), sse_max(a.y, b.y), sse_max(a.z, b.z)}; }
RSX_F V3 vclamp(V3 a, V3 lo, V3 hi) { return vmin(vmax(a, lo), hi); }
RSX_F float max_elem(V3 a) { return sse_max(sse_max(a.x, a.z), sse_max(a.y, a.z)); }
// glam signum: sign bit of the lane on 1.0, NaN lanes kept
RSX_F float sgn_lane(float v) { return isnan_(v) ? v : from_bits((bits(v) & 0x80000000u) | 0x3F800000u); }
RSX_F V3 vsignum(V3 a) { return {sgn_lane(a.x), sgn_lane(a.y), sgn_lane(a.z)}; }
RSX_F bool all_le(V3 a, V3 b) { return a.x <= b.x && a.y <= b.y && a.z <= b.z; }
RSX_F bool all_ge(V3 a, V3 b) { return a.x >= b.x && a.y >= b.y && a.z >= b.z; }
RSX_F bool box_overlap(const Box3& a, const Box3& b) { return all_le(a.lo, b.hi) && all_ge(a.hi, b.lo); }

// ---- V4 (quaternion normalisation and the manifold's area choice) ----
RSX_F float dot4(V4 a, V4 b) { return fadd(fadd(fmul(a.x, b.x), fmul(a.z, b.z)), fadd(fmul(a.y, b.y), fmul(a.w, b.w))); }

// ---- M3 ----
RSX_F M3 m3_identity() { return {{1.0f, 0.0f, 0.0f}, {0.0f, 1.0f, 0.0f}, {0.0f, 0.0f, 1.0f}}; }
RSX_F V3 operator*(const M3& m, V3 v) {
  V3 r = m.c0 * vs(v.x);
  r = r + m.c1 * vs(v.y);
  return r + m.c2 * vs(v.z);
}
RSX_F V3 mul_t(const M3& m, V3 v) { return {dot(m.c0, v), dot(m.c1, v), dot(m.c2, v)}; }  // transpose(m) * v
RSX_F M3 operator*(const M3& a, const M3& b) { return {a * b.c0, a * b.c1, a * b.c2}; }
RSX_F M3 transpose(const M3& m) { return {{m.c0.x, m.c1.x, m.c2.x}, {m.c0.y, m.c1.y, m.c2.y}, {m.c0.z, m.c1.z, m.c2.z}}; }
RSX_F M3 mabs(const M3& m) { return {vabs(m.c0), vabs(m.c1), vabs(m.c2)}; }
RSX_F bool m3_is_identity(const M3& m) {
  return m.c0.x == 1.0f && m.c0.y == 0.0f && m.c0.z == 0.0f && m.c1.x == 0.0f && m.c1.y == 1.0f && m.c1.z == 0.0f &&
         m.c2.x == 0.0f && m.c2.y == 0.0f && m.c2.z == 1.0f;
}
RSX_F M3 m3_from_quat(Q4 q) {
  float x2 = fadd(q.x, q.x), y2 = fadd(q.y, q.y), z2 = fadd(q.z, q.z);
  float xx = fmul(q.x, x2), xy = fmul(q.x, y2), xz = fmul(q.x, z2);
  float yy = fmul(q.y, y2), yz = fmul(q.y, z2), zz = fmul(q.z, z2);
  float wx = fmul(q.w, x2), wy = fmul(q.w, y2), wz = fmul(q.w, z2);
  return {{fsub(1.0f, fadd(yy, zz)), fadd(xy, wz), fsub(xz, wy)},
          {fsub(xy, wz), fsub(1.0f, fadd(xx, zz)), fadd(yz, wx)},
          {fadd(xz, wy), fsub(yz, wx), fsub(1.0f, fadd(xx, yy))}};
}

// ---- Aff ----
RSX_F Aff aff_identity() { return {m3_identity(), vzero()}; }
RSX_F V3 xform_point(const Aff& t, V3 p) { return t.m * p + t.t; }
RSX_F Aff operator*(const Aff& a, const Aff& b) { return {a.m * b.m, a.m * b.t + a.t}; }
RSX_F Aff aff_inverse_rigid(const Aff& t) {  // V3 AffineExt::transpose
  M3 r = transpose(t.m);
  return {r, r * (-t.t)};
}
RSX_F V3 inv_xform(const Aff& t, V3 v) { return mul_t(t.m, v - t.t); }

// ---- Q4 ----
RSX_F Q4 qnormalize(Q4 q) {
  V4 v = {q.x, q.y, q.z, q.w};
  float l = fsqrt(dot4(v, v));
  return {fdiv(q.x, l), fdiv(q.y, l), fdiv(q.z, l), fdiv(q.w, l)};
}
RSX_F Q4 operator*(Q4 l, Q4 r) {
  float ax = fadd(fmul(l.x, r.w), fmul(l.w, r.x));
  float ay = fadd(fneg(fmul(l.x, r.z)), fmul(l.w, r.y));
  float az = fadd(fmul(l.x, r.y), fmul(l.w, r.z));
  float aw = fadd(fneg(fmul(l.x, r.x)), fmul(l.w, r.w));
  float bx = fadd(fneg(fmul(l.z, r.y)), fmul(l.y, r.z));
  float by = fadd(fmul(l.z, r.x), fmul(l.y, r.w));
  float bz = fadd(fmul(l.z, r.w), fneg(fmul(l.y, r.x)));
  float bw = fadd(fneg(fmul(l.z, r.z)), fneg(fmul(l.y, r.y)));
  return {fadd(ax, bx), fadd(ay, by), fadd(az, bz), fadd(aw, bw)};
}
RSX_F V3 qrotate(Q4 q, V3 v) {  // glam Quat * Vec3A
  V3 b = {q.x, q.y, q.z};
  float b2 = dot(b, b);
  V3 t1 = v * vs(fsub(fmul(q.w, q.w), b2));
  V3 t2 = b * vs(fmul(dot(v, b), 2.0f));
  V3 t3 = cross(b, v) * vs(fmul(q.w, 2.0f));
  return (t1 + t2) + t3;
}
// glam Quat::from_mat3a (DirectXMath's branch order)
RSX_F Q4 quat_from_m3(const M3& m) {
  float m00 = m.c0.x, m01 = m.c0.y, m02 = m.c0.z, m10 = m.c1.x, m11 = m.c1.y, m12 = m.c1.z, m20 = m.c2.x, m21 = m.c2.y,
        m22 = m.c2.z;
  if (m22 <= 0.0f) {
    float d10 = fsub(m11, m00), om22 = fsub(1.0f, m22);
    if (d10 <= 0.0f) {
      float f = fsub(om22, d10), inv = fdiv(0.5f, fsqrt(f));
      return {fmul(f, inv), fmul(fadd(m01, m10), inv), fmul(fadd(m02, m20), inv), fmul(fsub(m12, m21), inv)};
    }
    float f = fadd(om22, d10), inv = fdiv(0.5f, fsqrt(f));
    return {fmul(fadd(m01, m10), inv), fmul(f, inv), fmul(fadd(m12, m21), inv), fmul(fsub(m20, m02), inv)};
  }
  float s10 = fadd(m11, m00), op22 = fadd(1.0f, m22);
  if (s10 <= 0.0f) {
    float f = fsub(op22, s10), inv = fdiv(0.5f, fsqrt(f));
    return {fmul(fadd(m02, m20), inv), fmul(fadd(m12, m21), inv), fmul(f, inv), fmul(fsub(m01, m10), inv)};
  }
  float f = fadd(op22, s10), inv = fdiv(0.5f, fsqrt(f));
  return {fmul(fsub(m12, m21), inv), fmul(fsub(m20, m02), inv), fmul(fsub(m01, m10), inv), fmul(f, inv)};
}
// glam Quat::from_axis_angle as V3's from_axis_angle_simd: (axis * sin(a/2), cos(a/2)); s, c given
RSX_F Q4 quat_axis_sc(V3 axis, float s, float c) {
  V3 v = axis * vs(s);
  return {v.x, v.y, v.z, c};
}

}  // namespace rsx
