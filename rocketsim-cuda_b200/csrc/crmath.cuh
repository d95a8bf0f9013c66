// Correctly rounded binary32 sin, cos, tan, atan2 and pow without any FP64: every function is evaluated in 128-bit
// integer fixed point (two's complement, 124 fractional bits; absolute error a few units of 2^-124) and rounded once
// to binary32, round to nearest even.  The correctly rounded result of a function is unique, so these equal the
// reference's correctly rounded CPU build (cuda/common/libm_cr.cuh:279 sinf_cr, :329 cosf_cr, :363 tanf_cr, :459
// atan2f_cr, :725 powf_cr, which port CORE-MATH in double precision) bit for bit; the tests check sin, cos and tan on
// all 2^32 inputs and atan2 / pow on large seeded samples.  The auto-flip helpers reproduce the reference's f64 path
// (cuda/sim/car_pre_tick.cuh:39-64: float(atan2_64) and float(hypot64)) with integers: the value is rounded to a
// double first, then to a float, exactly as `(float)` of a correctly rounded double does.
//
// Methods (published textbook algorithms, written for this project; constants from gen_crmath_tables.py):
//   * Payne-Hanek reduction of x by pi/2 against 384 bits of 2/pi;
//   * sin / cos: a 1/64-spaced table of sin and cos, and Taylor series of the remainder (|d| <= 1/128);
//   * tan: sin / cos by restoring long division of the two fixed-point values;
//   * fast paths for sin / cos / tan (|x| in [2^-14, 64]) and atan2 (normal operands): double-float evaluation with a
//     proven error bound and a rounding test; only when the test cannot decide does the fixed-point path run;
//   * atan: a 1/128-spaced table of atan and atan((t - c) / (1 + t c)) by its Taylor series;
//   * pow: 2^(y log2 x): log2 by a table of log2(1 + i/128) and the ln(1 + v) series; exp2 by a table of 2^(j/128)
//     and the exp series; exact results (pow has them) are detected as ties within 2^-100.
// NaN results are the canonical quiet NaN 0x7FC00000.
#pragma once
#include "fp.cuh"

#if defined(__CUDA_ARCH__)
#define RSX_TABLE static __device__ const
#else
#define RSX_TABLE static const
#endif

namespace rsx {
namespace crm {

struct U128 { uint64_t hi, lo; };

#include "crmath_tables.inc"

RSX_F void mul64(uint64_t a, uint64_t b, uint64_t* hi, uint64_t* lo) {
#if defined(__CUDA_ARCH__)
  *hi = __umul64hi(a, b);
  *lo = a * b;
#else
  unsigned __int128 p = (unsigned __int128)a * b;
  *hi = (uint64_t)(p >> 64);
  *lo = (uint64_t)p;
#endif
}
RSX_F int clz64(uint64_t v) {
#if defined(__CUDA_ARCH__)
  return __clzll((long long)v);
#else
  return v ? __builtin_clzll(v) : 64;
#endif
}
RSX_F U128 add(U128 a, U128 b) {
  uint64_t lo = a.lo + b.lo;
  return U128{a.hi + b.hi + (lo < a.lo ? 1u : 0u), lo};
}
RSX_F U128 sub(U128 a, U128 b) {
  uint64_t lo = a.lo - b.lo;
  return U128{a.hi - b.hi - (a.lo < b.lo ? 1u : 0u), lo};
}
RSX_F U128 neg(U128 a) { return sub(U128{0, 0}, a); }
RSX_F bool is_neg(U128 a) { return (a.hi >> 63) != 0; }
RSX_F U128 absv(U128 a) { return is_neg(a) ? neg(a) : a; }
RSX_F bool is_zero(U128 a) { return (a.hi | a.lo) == 0; }
RSX_F bool ult(U128 a, U128 b) { return a.hi < b.hi || (a.hi == b.hi && a.lo < b.lo); }
RSX_F bool eq(U128 a, U128 b) { return a.hi == b.hi && a.lo == b.lo; }
RSX_F U128 shr(U128 a, int n) {  // logical
  if (n <= 0) return a;
  if (n >= 128) return U128{0, 0};
  if (n >= 64) return U128{0, a.hi >> (n - 64)};
  return U128{a.hi >> n, (a.lo >> n) | (a.hi << (64 - n))};
}
RSX_F U128 shl(U128 a, int n) {
  if (n <= 0) return a;
  if (n >= 128) return U128{0, 0};
  if (n >= 64) return U128{a.lo << (n - 64), 0};
  return U128{(a.hi << n) | (a.lo >> (64 - n)), a.lo << n};
}
RSX_F int clz(U128 a) { return a.hi ? clz64(a.hi) : 64 + clz64(a.lo); }
RSX_F U128 one() { return U128{1ull << 60, 0}; }
RSX_F U128 small(uint64_t v, int frac_shift) { return shl(U128{0, v}, frac_shift); }  // v * 2^(frac_shift - 124)

// unsigned (a * b) >> 124 (a, b < 2^127)
RSX_F U128 umulq(U128 a, U128 b) {
  uint64_t p0h, p0l, p1h, p1l, p2h, p2l, p3h, p3l;
  mul64(a.lo, b.lo, &p0h, &p0l);
  mul64(a.lo, b.hi, &p1h, &p1l);
  mul64(a.hi, b.lo, &p2h, &p2l);
  mul64(a.hi, b.hi, &p3h, &p3l);
  (void)p0l;
  uint64_t w1 = p0h, c = 0;
  w1 += p1l; c += w1 < p1l;
  w1 += p2l; c += w1 < p2l;
  uint64_t w2 = p3l + c, c2 = w2 < c;
  w2 += p1h; c2 += w2 < p1h;
  w2 += p2h; c2 += w2 < p2h;
  uint64_t w3 = p3h + c2;
  return U128{(w3 << 4) | (w2 >> 60), (w2 << 4) | (w1 >> 60)};
}
RSX_F U128 mulq(U128 a, U128 b) {  // signed fixed-point product
  bool n = is_neg(a) != is_neg(b);
  U128 p = umulq(absv(a), absv(b));
  return n ? neg(p) : p;
}

// a / b for a, b > 0: the quotient of the two values normalised to [1, 2), in fixed point (in (1/2, 2)), and the
// binary exponent to apply: a / b = q * 2^(*e).  *exact is set when the remainder is zero.
RSX_F U128 udiv_norm(U128 a, U128 b, int* e, bool* exact) {
  int sa = clz(a) - 3, sb = clz(b) - 3;  // leading bits to position 124
  a = sa >= 0 ? shl(a, sa) : shr(a, -sa);
  b = sb >= 0 ? shl(b, sb) : shr(b, -sb);
  *e = sb - sa;
  U128 q = {0, 0}, r = a;
  for (int i = 0; i < 125; ++i) {  // quotient bits of weight 2^0 .. 2^-124
    q = shl(q, 1);
    if (!ult(r, b)) {
      r = sub(r, b);
      q.lo |= 1;
    }
    r = shl(r, 1);
  }
  *exact = is_zero(r);
  return q;
}

// Rounds v * 2^e (v > 0 unsigned fixed point: value = v / 2^124 * 2^e) to binary32, nearest even.  `dir` tells where
// the exact value lies when it is not v: -1 just below, +1 just above, 0 exactly v (or unknown, for a value that is
// not within a unit of a tie).  `pre` > 0 first rounds to a `pre`-bit significand (53: a double), then to binary32.
// `tie_tol` > 0 treats a remainder within tie_tol units of the half-way point as an exact tie.
RSX_F uint32_t round_f32(U128 v, int e, int dir, int pre, uint64_t tie_tol) {
  if (is_zero(v)) return 0u;
  int p = 127 - clz(v);
  if (pre > 0 && p - pre + 1 > 0) {
    int drop = p - pre + 1;
    U128 keep = shr(v, drop);
    U128 rem = sub(v, shl(keep, drop));
    U128 half = shl(U128{0, 1}, drop - 1);
    bool up = ult(half, rem) || (eq(rem, half) && (dir > 0 || (dir == 0 && (keep.lo & 1))));
    v = shl(add(keep, U128{0, up ? 1u : 0u}), drop);
    dir = 0;
    p = 127 - clz(v);
  }
  int E = p - 124 + e;
  if (E > 127) return 0x7F800000u;
  int nb = E >= -126 ? 24 : 24 - (-126 - E);
  if (nb < 0) return 0u;
  int drop = p - nb + 1;  // >= 1 (values carry far more than 24 bits)
  U128 keep = shr(v, drop);
  U128 rem = sub(v, shl(keep, drop));
  U128 half = shl(U128{0, 1}, drop - 1);
  bool up;
  bool tie;
  if (tie_tol) {
    U128 lo = ult(half, U128{0, tie_tol}) ? U128{0, 0} : sub(half, U128{0, tie_tol});
    U128 hi = add(half, U128{0, tie_tol});
    tie = !ult(rem, lo) && !ult(hi, rem);
  } else {
    tie = eq(rem, half);
  }
  if (tie) up = (tie_tol || dir == 0) ? (keep.lo & 1) != 0 : dir > 0;
  else up = ult(half, rem);
  uint64_t k = keep.lo + (up ? 1u : 0u);
  uint64_t b = E >= -126 ? (((uint64_t)(E + 126)) << 23) + k : k;
  return b >= 0x7F800000ull ? 0x7F800000u : (uint32_t)b;
}

// ---- sin, cos, tan -------------------------------------------------------------------------------------------------

// |x| (a finite float >= 2^-14) = n pi/2 + r with |r| <= pi/4: returns r (fixed point), *quadrant = n mod 4.
RSX_F U128 reduce_pio2(uint32_t ax_bits, int* quadrant) {
  int be = (int)(ax_bits >> 23);
  uint32_t m = (ax_bits & 0x7FFFFFu) | 0x800000u;
  int ex = be - 150;                // |x| = m * 2^ex
  int s = ex - 2 > 0 ? ex - 2 : 0;  // bits of 2/pi before s only add multiples of 4
  int k = s >> 5, o = s & 31;
  uint32_t w[5];
  for (int i = 0; i < 5; ++i) {
    uint32_t a = kTwoOverPi[k + i], b = kTwoOverPi[k + i + 1];
    w[i] = o ? (a << o) | (b >> (32 - o)) : a;
  }
  uint32_t P[6];  // m * (the 160-bit window), little-endian limbs; LSB weight 2^(ex - s - 160)
  uint64_t carry = 0;
  for (int i = 4; i >= 0; --i) {
    uint64_t t = (uint64_t)w[i] * m + carry;
    P[4 - i] = (uint32_t)t;
    carry = t >> 32;
  }
  P[5] = (uint32_t)carry;
  int T = 162 + s - ex;  // bits [T-2, T) are the quadrant, [T-126, T-2) the fraction's 124 bits
  U128 f = {0, 0};
  for (int b = T - 3; b >= T - 126; --b) {
    uint32_t bit = (b >= 0 && b < 192) ? (P[b >> 5] >> (b & 31)) & 1u : 0u;
    f = shl(f, 1);
    f.lo |= bit;
  }
  int q = (int)(((T - 2 < 192 ? (P[(T - 2) >> 5] >> ((T - 2) & 31)) & 1u : 0u)) |
                ((T - 1 < 192 ? (P[(T - 1) >> 5] >> ((T - 1) & 31)) & 1u : 0u) << 1));
  if (f.hi >> 59) {  // f >= 1/2: r = (f - 1) pi / 2 in the next quadrant
    f = sub(f, one());
    q += 1;
  }
  *quadrant = q & 3;
  return mulq(f, kPiHalf[0]);
}

// sin and cos of r, |r| <= pi/4, in fixed point.
RSX_F void sincos_fx(U128 r, U128* s_out, U128* c_out) {
  bool rneg = is_neg(r);
  U128 a = absv(r);
  int i = (int)shr(add(a, small(1, 124 - 7)), 124 - 6).lo;  // the nearest multiple of 1/64
  U128 d = sub(a, small((uint64_t)i, 124 - 6));             // |d| <= 1/128
  U128 d2 = mulq(d, d);
  U128 ts = one(), tc = one();
  for (int k = 14; k >= 2; k -= 2) ts = sub(one(), mulq(mulq(d2, kInvPair[k]), ts));  // sin d / d
  for (int k = 15; k >= 1; k -= 2) tc = sub(one(), mulq(mulq(d2, kInvPair[k]), tc));  // cos d
  U128 sd = mulq(d, ts);
  U128 s = add(mulq(kSin64[i], tc), mulq(kCos64[i], sd));
  U128 c = sub(mulq(kCos64[i], tc), mulq(kSin64[i], sd));
  *s_out = rneg ? neg(s) : s;
  *c_out = c;
}

RSX_F uint32_t signed_round(U128 v, int e, uint32_t sign) {
  bool n = is_neg(v);
  uint32_t b = round_f32(absv(v), e, 0, 0, 0);
  return b | ((n ? 0x80000000u : 0u) ^ sign);
}

// which: 0 sin, 1 cos, 2 tan
RSX_F float trig(float x, int which) {
  uint32_t bx = bits(x), ax = bx & 0x7FFFFFFFu, sx = bx & 0x80000000u;
  if (ax >= 0x7F800000u) return from_bits(0x7FC00000u);  // inf or NaN
  if (ax < 0x38800000u) {                                 // |x| < 2^-14: sin x = x, tan x = x, cos x = 1 after rounding
    if (which == 1) return 1.0f;
    // sin x = x - x^3/6 and tan x = x + x^3/3 round to x for |x| < 2^-12 (x is a float, the correction is below half
    // an ulp of x); a subnormal or zero x is exact as well
    return x;
  }
  int q;
  U128 r = reduce_pio2(ax, &q);
  U128 s, c;
  sincos_fx(r, &s, &c);
  if (which == 0) {
    U128 v = (q == 0) ? s : (q == 1) ? c : (q == 2) ? neg(s) : neg(c);
    return from_bits(signed_round(v, 0, sx));
  }
  if (which == 1) {
    U128 v = (q == 0) ? c : (q == 1) ? neg(s) : (q == 2) ? neg(c) : s;
    return from_bits(signed_round(v, 0, 0));
  }
  // tan: q even -> s / c; q odd -> -c / s
  U128 num = (q & 1) ? c : s, den = (q & 1) ? s : c;
  bool n = is_neg(num) != is_neg(den);
  if (q & 1) n = !n;
  if (is_zero(num)) return from_bits(sx);
  int e;
  bool exact;
  U128 qv = udiv_norm(absv(num), absv(den), &e, &exact);
  uint32_t b = round_f32(qv, e, exact ? 0 : 1, 0, 0);
  return from_bits(b | ((n ? 0x80000000u : 0u) ^ sx));
}


// ---- fast path of sin / cos: double-float (binary32 pairs, exact products by FMA) with a rounding test ----------------
// For |x| <= 64: x = k pi/2 + r (Cody-Waite with pi/2 in three parts, the first two short enough that k * part is exact),
// then sin and cos of r by their Taylor polynomials, the leading coefficients as float pairs.  The value carries a proven
// error bound; when the bound does not separate it from the nearest half-way point between two floats, the exact
// fixed-point path above decides.  Coefficients: -1/3!, 1/5!, ... and -1/2!, 1/4!, ... as (hi, lo) float pairs.
RSX_TABLE uint32_t kSinC[7][2] = {{0xbe2aaaabu, 0x31aaaaabu}, {0x3c088889u, 0xafeeeeefu}, {0xb9500d01u, 0x2c3fcbfdu}, {0x3638ef1du, 0x292ad8e6u}, {0xb2d7322bu, 0x00000000u}, {0x2f309231u, 0x00000000u}, {0xab573f9fu, 0x00000000u}};
RSX_TABLE uint32_t kCosC[8][2] = {{0xbf000000u, 0x00000000u}, {0x3d2aaaabu, 0xb0aaaaabu}, {0xbab60b61u, 0x2e13e93fu}, {0x37d00d01u, 0xaabfcbfdu}, {0xb493f27eu, 0x00000000u}, {0x310f76c7u, 0x00000000u}, {0xad49cba5u, 0x00000000u}, {0x29573f9fu, 0x00000000u}};
RSX_TABLE uint32_t kPio2Split[3] = {0x3fc90f80u, 0x37354400u, 0x2e85a309u};  // |pi/2 - sum| < 1.218e-18

struct DF { float h, l; };
RSX_F DF two_prod(float a, float b) {
  float p = fmul(a, b);
  return {p, ffma(a, b, fneg(p))};
}
RSX_F DF two_sum(float a, float b) {
  float s = fadd(a, b), bb = fsub(s, a);
  return {s, fadd(fsub(a, fsub(s, bb)), fsub(b, bb))};
}
RSX_F DF quick_sum(float a, float b) {  // |a| >= |b|
  float s = fadd(a, b);
  return {s, fsub(b, fsub(s, a))};
}
RSX_F DF df_add(DF a, DF b) {
  DF s = two_sum(a.h, b.h);
  return quick_sum(s.h, fadd(s.l, fadd(a.l, b.l)));
}
RSX_F DF df_mul(DF a, DF b) {
  DF p = two_prod(a.h, b.h);
  return quick_sum(p.h, ffma(a.h, b.l, ffma(a.l, b.h, p.l)));
}
RSX_F DF df_mul_f(DF a, float b) {
  DF p = two_prod(a.h, b);
  return quick_sum(p.h, ffma(a.l, b, p.l));
}
RSX_F DF df_c(const uint32_t c[2]) { return {from_bits(c[0]), from_bits(c[1])}; }

// half the gap from |h| to the neighbouring float on the side of l (a quarter ulp below a power of two)
RSX_F float half_gap(float h, float l) {
  uint32_t a = bits(h) & 0x7FFFFFFFu;
  float ulp = from_bits((a & 0x7F800000u) - (23u << 23));
  bool toward_zero = (bits(h) ^ bits(l)) >> 31;
  return ((a & 0x7FFFFFu) == 0 && toward_zero) ? fmul(ulp, 0.25f) : fmul(ulp, 0.5f);
}
// the float nearest to h + l when the exact value is within err of h + l and that decides it; else false
RSX_F bool rounds_to(DF v, float err, float* out) {
  if (fadd(fabs_(v.l), err) < fmul(half_gap(v.h, v.l), 0.9999f)) {
    *out = v.h;
    return true;
  }
  return false;
}

// sin and cos of |x| in [2^-14, 64]: false when the fast path cannot decide one of the two it was asked for
RSX_F float round_nearest(float v) {  // v < 2^22: the nearest integer, ties away (only the quadrant's parity matters)
  return i2f(f2i(fadd(v, 0.5f)));
}
// sin and cos of ax in [2^-14, 64] as float pairs, and the absolute error the reduction adds (each value's own error
// is below |value| * 1e-12 besides)
RSX_F void sincos_df(float ax, DF* s_out, DF* c_out, float* red_err_out) {
  float rh = ax, rl = 0.0f, red_err = 0.0f;
  int q = 0;
  if (ax > 0.78539816f) {
    float kf = round_nearest(fmul(ax, from_bits(0x3f22f983u)));
    q = (int)kf & 3;
    float t1 = ffma(fneg(kf), from_bits(kPio2Split[0]), ax);          // exact
    DF r = two_sum(t1, fneg(fmul(kf, from_bits(kPio2Split[1]))));     // k * part2 exact
    DF p3 = two_prod(kf, from_bits(kPio2Split[2]));
    r = df_add(r, DF{fneg(p3.h), fneg(p3.l)});
    rh = r.h;
    rl = r.l;
    red_err = fmul(kf, 2e-18f);                                        // k (pi/2 - the three parts) and the rounding below
    red_err = fadd(red_err, fmul(fabs_(rh), 1e-14f));
  }
  DF y = two_prod(rh, rh);
  float yh = y.h;
  // sin(rh) = rh + rh * y * Q(y)
  float ts = fadd(from_bits(kSinC[4][0]), fmul(yh, fadd(from_bits(kSinC[5][0]), fmul(yh, from_bits(kSinC[6][0])))));
  DF qs = df_add(df_c(kSinC[3]), df_mul_f(y, ts));
  qs = df_add(df_c(kSinC[2]), df_mul(y, qs));
  qs = df_add(df_c(kSinC[1]), df_mul(y, qs));
  qs = df_add(df_c(kSinC[0]), df_mul(y, qs));
  DF cx = df_mul_f(df_mul(y, qs), rh);
  // cos(rh) = 1 + y * P(y)
  float tc = fadd(from_bits(kCosC[4][0]), fmul(yh, fadd(from_bits(kCosC[5][0]), fmul(yh, fadd(from_bits(kCosC[6][0]), fmul(yh, from_bits(kCosC[7][0])))))));
  DF pc = df_add(df_c(kCosC[3]), df_mul_f(y, tc));
  pc = df_add(df_c(kCosC[2]), df_mul(y, pc));
  pc = df_add(df_c(kCosC[1]), df_mul(y, pc));
  pc = df_add(df_c(kCosC[0]), df_mul(y, pc));
  DF yp = df_mul(y, pc);
  DF C = quick_sum(1.0f, yp.h);
  C = quick_sum(C.h, fadd(C.l, yp.l));
  // the low part of the reduced argument: sin(rh + rl) = sin rh + rl cos rh, cos(rh + rl) = cos rh - rl sin rh
  DF S = two_sum(rh, cx.h);
  S = quick_sum(S.h, fadd(S.l, fadd(cx.l, fmul(rl, C.h))));
  C = quick_sum(C.h, fsub(C.l, fmul(rl, fadd(rh, cx.h))));
  // quadrant
  *s_out = (q == 0) ? S : (q == 1) ? C : (q == 2) ? DF{fneg(S.h), fneg(S.l)} : DF{fneg(C.h), fneg(C.l)};
  *c_out = (q == 0) ? C : (q == 1) ? DF{fneg(S.h), fneg(S.l)} : (q == 2) ? DF{fneg(C.h), fneg(C.l)} : S;
  *red_err_out = red_err;
}
RSX_F bool sincos_fast(float ax, bool want_s, bool want_c, float* s_out, float* c_out) {
  DF vs, vc;
  float red_err;
  sincos_df(ax, &vs, &vc, &red_err);
  bool ok = true;
  if (want_s) ok = ok && rounds_to(vs, fadd(fmul(fabs_(vs.h), 1e-12f), red_err), s_out);
  if (want_c) ok = ok && rounds_to(vc, fadd(fmul(fabs_(vc.h), 1e-12f), red_err), c_out);
  return ok;
}

// a / b in float pairs (Dekker's division: the quotient of the leading parts, corrected by the remainder's quotient);
// relative error below 2^-44 for normal operands
RSX_F DF df_div(DF a, DF b) {
  float q1 = fdiv(a.h, b.h);
  DF p = df_mul_f(b, q1);
  DF r = df_add(a, DF{fneg(p.h), fneg(p.l)});
  float q2 = fdiv(r.h, b.h);
  return quick_sum(q1, q2);
}

// tan of ax in [2^-14, 64] as sin / cos in float pairs; false when the error bound does not decide the rounding (near
// a pole the cosine's relative error grows and the test fails)
RSX_F bool tan_fast(float ax, float* out) {
  DF vs, vc;
  float red_err;
  sincos_df(ax, &vs, &vc, &red_err);
  float as = fabs_(vs.h), ac = fabs_(vc.h);
  if (ac < 1e-6f || as < 1e-30f) return false;
  DF t = df_div(vs, vc);
  float rel = fadd(fadd(fdiv(fadd(fmul(as, 1e-12f), red_err), as), fdiv(fadd(fmul(ac, 1e-12f), red_err), ac)), 1e-12f);
  return rounds_to(t, fmul(fabs_(t.h), rel), out);
}

// ---- atan2 ---------------------------------------------------------------------------------------------------------

// fast path of atan2 for |y|, |x| in [2^-63, 2^64) with exponents at most 60 apart: t = min / max (float pair, the
// remainder of the rounded quotient is exact), c = the nearest multiple of 1/128, atan t = atan c + atan u with
// u = (t - c) / (1 + t c), |u| <= 1/256, atan u = u - u^3/3 + u^5/5 - u^7/7; then pi/2 - . when |y| > |x| and pi - .
// when x < 0.  The error is below 2^-38 of the result; the rounding test uses 2^-36.  The magnitude goes to *out.
RSX_F bool atan2_fast(uint32_t ay, uint32_t ax, bool xneg, float* out) {
  int ey = (int)(ay >> 23), ex = (int)(ax >> 23);
  // operands in [2^-63, 2^64): the quotient's remainder and every product below stay normal (exact where it matters)
  if (ey < 64 || ex < 64 || ey > 190 || ex > 190 || ey - ex > 60 || ex - ey > 60) return false;
  bool swap = ay > ax;
  float num = from_bits(swap ? ax : ay), den = from_bits(swap ? ay : ax);
  float th = fdiv(num, den);
  float tl = fdiv(ffma(fneg(th), den, num), den);
  int i = (int)f2i(fadd(fmul(th, 128.0f), 0.5f));
  float c = fmul(i2f(i), 0.0078125f);
  DF tc = two_prod(th, c);
  tc = quick_sum(tc.h, fadd(tc.l, fmul(tl, c)));
  DF u = df_div(two_sum(fsub(th, c), tl), df_add(DF{1.0f, 0.0f}, tc));
  float p = fmul(u.h, u.h);
  float sfac = fmul(p, fadd(-0.33333334f, fmul(p, fadd(0.2f, fmul(p, -0.14285715f)))));
  DF r = df_add(df_c(kAtan128DF[i]), quick_sum(u.h, fadd(u.l, fmul(u.h, sfac))));
  if (swap) r = df_add(df_c(kPiDF[0]), DF{fneg(r.h), fneg(r.l)});
  if (xneg) r = df_add(df_c(kPiDF[1]), DF{fneg(r.h), fneg(r.l)});
  return rounds_to(r, fmul(fabs_(r.h), 1.5e-11f), out);
}

// atan(t) for t = m * 2^te with m in [1, 2) (fixed point) and t <= 1, as an absolute fixed-point value; for tiny t the
// value is returned relative: *rel = true and the result is m' * 2^(*re) with m' in fixed point.
RSX_F U128 atan_fx(U128 m, int te, bool exact_ratio, bool* rel, int* re, int* rdir) {
  *rel = false;
  *rdir = 0;
  if (te < -50) {  // atan t = t (1 - t^2/3 ...): below t by less than 2^-100 t
    *rel = true;
    *re = te;
    *rdir = exact_ratio ? -1 : 1;
    return m;
  }
  if (te < -8) {  // t < 1/256: t * (1 - t^2/3 + t^4/5 - ...), computed relative to t
    U128 m2 = mulq(m, m);                 // m^2 in [1, 4)
    U128 t2 = shr(m2, -2 * te);           // t^2 (absolute, < 2^-16)
    U128 acc = {0, 0};
    for (int k = 11; k >= 1; --k) acc = mulq(t2, sub(kInvOdd[k], acc));
    U128 fac = sub(one(), acc);
    *rel = true;
    *re = te;
    return mulq(m, fac);
  }
  U128 t = shr(m, -te);  // absolute, in [1/256, 1]
  int i = (int)shr(add(t, small(1, 124 - 8)), 124 - 7).lo;  // nearest multiple of 1/128
  U128 c = small((uint64_t)i, 124 - 7);
  U128 num = sub(t, c);
  U128 den = add(one(), mulq(t, c));
  U128 uabs = {0, 0};
  if (!is_zero(num)) {
    int e;
    bool ex;
    U128 qv = udiv_norm(absv(num), den, &e, &ex);
    uabs = e >= 0 ? shl(qv, e) : shr(qv, -e);
  }
  U128 u2 = mulq(uabs, uabs);
  U128 acc = {0, 0};
  for (int k = 8; k >= 1; --k) acc = mulq(u2, sub(kInvOdd[k], acc));
  U128 au = mulq(uabs, sub(one(), acc));
  return is_neg(num) ? sub(kAtan128[i], au) : add(kAtan128[i], au);
}

// atan2(y, x) of finite floats, both nonzero, as a positive magnitude: (value fixed point, exponent, dir)
RSX_F U128 atan2_mag(uint32_t ay, uint32_t ax, bool xneg, int* e_out, int* dir_out) {
  auto unpack = [](uint32_t b, U128* m, int* e) {  // b = m * 2^e, m in [1, 2) fixed point
    int be = (int)(b >> 23);
    uint32_t mm = b & 0x7FFFFFu;
    if (be == 0) {  // subnormal
      int sh = clz64((uint64_t)mm) - 40;  // to bit 23
      mm <<= sh;
      be = 1 - sh;
    } else {
      mm |= 0x800000u;
    }
    *m = small(mm, 124 - 23);
    *e = be - 127;
  };
  U128 my, mx;
  int ey, ex;
  unpack(ay, &my, &ey);
  unpack(ax, &mx, &ex);
  bool swap = ay > ax;  // |y| > |x|: atan2 = pi/2 - atan(x / y)
  U128 nm = swap ? mx : my, dm = swap ? my : mx;
  int te_base = swap ? ex - ey : ey - ex;
  int e;
  bool exact;
  U128 ratio = udiv_norm(nm, dm, &e, &exact);  // in (1/2, 2): renormalise to [1, 2)
  int te = te_base + e;
  if (ratio.hi >> 60 == 0) {  // below 1
    ratio = shl(ratio, 1);
    te -= 1;
  }
  bool rel;
  int re, rdir;
  U128 a = atan_fx(ratio, te, exact, &rel, &re, &rdir);
  if (!swap && !xneg) {  // the value itself
    *e_out = rel ? re : 0;
    *dir_out = rdir;
    return a;
  }
  U128 aa = rel ? (re >= -124 ? shr(a, -re) : U128{0, 0}) : a;  // absolute
  U128 v = swap ? sub(kPiHalf[0], aa) : aa;
  if (xneg) v = sub(kPi[0], v);
  *e_out = 0;
  *dir_out = 0;
  // a relative tiny part lost below 2^-124 moves the value by less than one unit: not near a tie for these results
  return v;
}

RSX_F float atan2f_cr(float y, float x) {
  uint32_t by = bits(y), bx = bits(x), ay = by & 0x7FFFFFFFu, ax = bx & 0x7FFFFFFFu, sy = by & 0x80000000u;
  bool xneg = (bx >> 31) != 0;
  if (ay > 0x7F800000u || ax > 0x7F800000u) return from_bits(0x7FC00000u);
  const uint32_t PI_B = 0x40490FDBu, PI2_B = 0x3FC90FDBu, PI4_B = 0x3F490FDBu, PI34_B = 0x4016CBE4u;
  if (ay == 0) return from_bits((xneg ? PI_B : 0u) | sy);
  if (ax == 0) return from_bits(PI2_B | sy);
  if (ay == 0x7F800000u) {
    if (ax == 0x7F800000u) return from_bits((xneg ? PI34_B : PI4_B) | sy);
    return from_bits(PI2_B | sy);
  }
  if (ax == 0x7F800000u) return from_bits((xneg ? PI_B : 0u) | sy);
  float fast;
  if (atan2_fast(ay, ax, xneg, &fast)) return from_bits(bits(fast) | sy);
  int e, dir;
  U128 v = atan2_mag(ay, ax, xneg, &e, &dir);
  return from_bits(round_f32(v, e, dir, 0, 0) | sy);
}

// ---- pow -----------------------------------------------------------------------------------------------------------

// 0 not an integer, 1 odd integer, 2 even integer (y finite)
RSX_F int int_kind(uint32_t b) {
  uint32_t a = b & 0x7FFFFFFFu;
  if (a == 0) return 2;
  int be = (int)(a >> 23);
  if (be < 127) return 0;
  if (be >= 150 + 1) return 2;
  int frac_bits = 150 - be;  // bits of the significand below the unit
  uint32_t m = (a & 0x7FFFFFu) | 0x800000u;
  if (frac_bits > 0 && (m & ((1u << frac_bits) - 1u)) != 0) return 0;
  return ((m >> frac_bits) & 1u) ? 1 : 2;
}

RSX_F float powf_cr(float x, float y) {
  uint32_t bx = bits(x), by = bits(y), ax = bx & 0x7FFFFFFFu, ay = by & 0x7FFFFFFFu;
  bool xneg = (bx >> 31) != 0, yneg = (by >> 31) != 0;
  const uint32_t INF = 0x7F800000u, QNAN = 0x7FC00000u;
  if (ay == 0) return 1.0f;
  if (bx == 0x3F800000u) return 1.0f;
  if (ax > INF || ay > INF) return from_bits(QNAN);
  int yk = ay == INF ? 2 : int_kind(by);
  if (ay == INF) {
    if (ax == 0x3F800000u) return 1.0f;  // (-1)^inf
    bool big = ax > 0x3F800000u;
    return from_bits((big != yneg) ? INF : 0u);
  }
  uint32_t rsign = (xneg && yk == 1) ? 0x80000000u : 0u;
  if (ax == 0) return from_bits((yneg ? INF : 0u) | rsign);
  if (ax == INF) return from_bits((yneg ? 0u : INF) | rsign);
  if (xneg && yk == 0) return from_bits(QNAN);
  // |x| = m * 2^ex with m in [0.75, 1.5)
  int be = (int)(ax >> 23);
  uint32_t mm = ax & 0x7FFFFFu;
  if (be == 0) {
    int sh = clz64((uint64_t)mm) - 40;
    mm <<= sh;
    be = 1 - sh;
  } else {
    mm |= 0x800000u;
  }
  int ex = be - 127;
  U128 m = small(mm, 124 - 23);
  if (mm >= 0xC00000u) {  // m >= 1.5: use m / 2
    m = shr(m, 1);
    ex += 1;
  }
  // log2 m = log2 c + ln(1 + v) / ln 2, c = 1 + i/128, v = (m - c) / c
  U128 dm = sub(m, one());
  int i = (int)(is_neg(dm) ? -(int64_t)shr(add(absv(dm), small(1, 124 - 8)), 124 - 7).lo
                           : (int64_t)shr(add(dm, small(1, 124 - 8)), 124 - 7).lo);
  U128 c = add(one(), is_neg(dm) ? neg(small((uint64_t)(-i), 124 - 7)) : small((uint64_t)i, 124 - 7));
  U128 v = mulq(sub(m, c), kInvC[i + 32]);  // |v| <= 1/192
  U128 acc = {0, 0};
  for (int k = 18; k >= 2; --k) acc = mulq(v, sub(kInvInt[k], acc));  // ln(1+v)/v - 1 = -v/2 + v^2/3 ...
  // L = ex + log2 c + v (1 - acc) / ln 2, kept as a magnitude with an exponent: Lm * 2^Le
  U128 lnv = mulq(v, sub(one(), acc));
  U128 Lf = add(kLog2C[i + 32], mulq(lnv, kInvLn2[0]));  // log2 m, |.| <= 0.59 (absolute, 2^-124)
  U128 Lm;
  int Le;
  bool Lneg;
  if (ex == 0) {  // relative precision comes from Lf itself (|Lf| >= ~2^-24 unless m == 1, excluded by x != 1)
    Lneg = is_neg(Lf);
    Lm = absv(Lf);
    Le = 0;
  } else {  // |ex + Lf| >= 0.41: scale by 2^-8 so that ex fits
    U128 L8 = mulq(Lf, small(1, 124 - 8));  // Lf / 256
    U128 ex8 = ex < 0 ? neg(small((uint64_t)(-ex), 124 - 8)) : small((uint64_t)ex, 124 - 8);
    U128 full = add(L8, ex8);
    Lneg = is_neg(full);
    Lm = absv(full);
    Le = 8;
  }
  // t = y * L: y = my * 2^(ey - 23)
  int bey = (int)(ay >> 23);
  uint32_t my = ay & 0x7FFFFFu;
  if (bey == 0) {
    int sh = clz64((uint64_t)my) - 40;
    my <<= sh;
    bey = 1 - sh;
  } else {
    my |= 0x800000u;
  }
  int ey = bey - 127;  // |y| = (my / 2^23) * 2^ey
  bool tneg = Lneg != yneg;
  U128 tm = umulq(Lm, small(my, 124 - 23));  // |t| = tm * 2^(Le + ey)
  int te = Le + ey;
  // normalise tm to [1, 2) * 2^te
  if (is_zero(tm)) return from_bits(0x3F800000u | rsign);  // |x| == 1: (+-1)^y
  int lead = 127 - clz(tm);
  te += lead - 124;
  tm = lead > 124 ? shr(tm, lead - 124) : shl(tm, 124 - lead);
  if (te >= 8) {  // |t| >= 256: overflow or underflow for sure
    return from_bits((tneg ? 0u : INF) | rsign);
  }
  // t absolute with 124 fractional bits: |t| < 256 fits (two's complement range 2^3 ... scale down by 2^8 for the split)
  // integer part n and fraction f in [0, 1)
  U128 tabs8 = te >= -124 ? shr(tm, 8 - te) : U128{0, 0};  // |t| / 256 in fixed point
  // n = floor(|t|), fraction = |t| - n, from |t|/256: integer part is bits [116, 124)
  U128 t_abs_fx;  // |t| mod 1 in fixed point (124 fractional bits)
  int n_abs = (int)(shr(tabs8, 116).lo);
  t_abs_fx = shl(sub(tabs8, shl(U128{0, (uint64_t)n_abs}, 116)), 8);
  // lost bits when shifting |t| down by 8 - te: |t| had bits below 2^-124 only when te < 8 - ... (the shift keeps
  // 124 - 8 + te fractional bits, >= 108 for te >= -8, relative precision of 2^t stays ~2^-108)
  int n;
  U128 f;
  if (!tneg) {
    n = n_abs;
    f = t_abs_fx;
  } else if (is_zero(t_abs_fx)) {
    n = -n_abs;
    f = U128{0, 0};
  } else {
    n = -n_abs - 1;
    f = sub(one(), t_abs_fx);
  }
  // 2^f = 2^(j/128) * exp(w ln 2), w = f - j/128
  int j = (int)shr(add(f, small(1, 124 - 8)), 124 - 7).lo;
  U128 w = sub(f, small((uint64_t)j, 124 - 7));
  U128 z = mulq(w, kLn2[0]);
  U128 ex2 = one();
  for (int k = 16; k >= 1; --k) ex2 = add(one(), mulq(mulq(z, kInvInt[k]), ex2));
  U128 res = mulq(kExp2J[j], ex2);  // in [1, 2]
  uint32_t b = round_f32(res, n, 0, 0, 1ull << 24);
  return from_bits(b | rsign);
}

// ---- the auto-flip helpers: float(correctly rounded double) of atan2 and hypot ---------------------------------------

// (float)(double atan2(a0, a1)) for float a0, a1
RSX_HD RSX_NOINL inline float atan2_via_double(float a0, float a1) {
  uint32_t by = bits(a0), bx = bits(a1), ay = by & 0x7FFFFFFFu, ax = bx & 0x7FFFFFFFu, sy = by & 0x80000000u;
  bool xneg = (bx >> 31) != 0;
  if (ay > 0x7F800000u || ax > 0x7F800000u || ay == 0 || ax == 0 || ay == 0x7F800000u || ax == 0x7F800000u)
    return atan2f_cr(a0, a1);  // the special values are exact doubles whose float rounding is atan2f's
  // the fast path's rounding test keeps a margin of 1e-4 half-gaps, far above the 2^-53 the double rounding can move
  // the value, so its float is also the float of the rounded double
  float fast;
  if (atan2_fast(ay, ax, xneg, &fast)) return from_bits(bits(fast) | sy);
  int e, dir;
  U128 v = atan2_mag(ay, ax, xneg, &e, &dir);
  return from_bits(round_f32(v, e, dir, 53, 0) | sy);
}

// (float)(correctly rounded double hypot(a, b)) for float a, b, by integer square root
RSX_HD RSX_NOINL inline float hypot_via_double(float a, float b) {
  uint32_t ua = bits(a) & 0x7FFFFFFFu, ub = bits(b) & 0x7FFFFFFFu;
  if (ua >= 0x7F800000u || ub >= 0x7F800000u) {
    if (ua == 0x7F800000u || ub == 0x7F800000u) return from_bits(0x7F800000u);
    return from_bits(0x7FC00000u);
  }
  if (ua < ub) { uint32_t t = ua; ua = ub; ub = t; }
  if (ua == 0) return 0.0f;
  if ((ua >> 23) <= 187 && (ub >> 23) >= 91) {
    // fast path, both in [2^-36, 2^61) (the products' low parts stay normal, so they are exact): a^2 + b^2 from exact
    // products as a float pair, its square root corrected by one
    // Newton step (relative error below 2^-44); the rounding test's margin covers the double rounding as above
    float fa = from_bits(ua), fb = from_bits(ub);
    DF s2 = df_add(two_prod(fa, fa), two_prod(fb, fb));
    float r0 = fsqrt(s2.h);
    DF rr = two_prod(r0, r0);
    float d = fadd(fsub(fsub(s2.h, rr.h), rr.l), s2.l);
    DF h = quick_sum(r0, fdiv(d, fmul(2.0f, r0)));
    float fast;
    if (rounds_to(h, fmul(h.h, 1.5e-11f), &fast)) return fast;
  }
  auto unpack = [](uint32_t v, uint64_t* m, int* e) {  // v = m * 2^e, m integer
    int be = (int)(v >> 23);
    uint32_t mm = v & 0x7FFFFFu;
    if (be == 0) { *m = mm; *e = -149; }
    else { *m = mm | 0x800000u; *e = be - 150; }
  };
  uint64_t ma, mb;
  int ea, eb;
  unpack(ua, &ma, &ea);
  unpack(ub, &mb, &eb);
  // S = a^2 + b^2 = (ma^2 << 2(ea - eb) + mb^2) * 2^(2 eb)
  int d = 2 * (ea - eb);
  if (mb == 0 || d > 80) return from_bits(ua);  // (b/a)^2 < 2^-54: the double is |a| exactly
  uint64_t h1, l1;
  mul64(ma, ma, &h1, &l1);
  U128 S = shl(U128{h1, l1}, d);
  uint64_t h2, l2;
  mul64(mb, mb, &h2, &l2);
  S = add(S, U128{h2, l2});
  int se = 2 * eb;
  // scale S by an even power so that its top bit is at 126 or 127: the root then has 64 bits
  int lz = clz(S);
  int sh = lz & ~1;
  S = shl(S, sh);
  se -= sh;
  // integer square root, bit by bit
  uint64_t r = 0;
  for (int bit = 63; bit >= 0; --bit) {
    uint64_t c = r | (1ull << bit);
    uint64_t ph, pl;
    mul64(c, c, &ph, &pl);
    U128 sq = {ph, pl};
    if (!ult(S, sq)) r = c;
  }
  uint64_t ph, pl;
  mul64(r, r, &ph, &pl);
  bool exact = eq(U128{ph, pl}, S);
  // sqrt(S * 2^se) = r * 2^(se / 2): round r (64 bits) to 53, then to 24
  U128 v = shl(U128{0, r}, 60);  // r as fixed point with the binary point at 124: value r * 2^-64 ... exponent below
  int e = se / 2 + 64;
  return from_bits(round_f32(v, e, exact ? 0 : 1, 53, 0));
}

}  // namespace crm

// out of line on the device: one copy of each function serves every call site (the kernels' code must stay small
// enough for the instruction caches of warps in different phases)
RSX_HD RSX_NOINL inline void cr_sincos(float x, float* s, float* c) {
  uint32_t ax = bits(x) & 0x7FFFFFFFu;
  if (ax >= 0x38800000u && ax <= 0x42800000u) {  // 2^-14 <= |x| <= 64
    float ss, cc;
    if (crm::sincos_fast(from_bits(ax), true, true, &ss, &cc)) {
      *s = from_bits(bits(ss) ^ (bits(x) & 0x80000000u));
      *c = cc;
      return;
    }
  }
  *s = crm::trig(x, 0);
  *c = crm::trig(x, 1);
}
RSX_HD RSX_NOINL inline float cr_sin(float x) {
  uint32_t ax = bits(x) & 0x7FFFFFFFu;
  float ss, cc;
  if (ax >= 0x38800000u && ax <= 0x42800000u && crm::sincos_fast(from_bits(ax), true, false, &ss, &cc))
    return from_bits(bits(ss) ^ (bits(x) & 0x80000000u));
  return crm::trig(x, 0);
}
RSX_HD RSX_NOINL inline float cr_cos(float x) {
  uint32_t ax = bits(x) & 0x7FFFFFFFu;
  float ss, cc;
  if (ax >= 0x38800000u && ax <= 0x42800000u && crm::sincos_fast(from_bits(ax), false, true, &ss, &cc)) return cc;
  return crm::trig(x, 1);
}
RSX_HD RSX_NOINL inline float cr_tan(float x) {
  uint32_t ax = bits(x) & 0x7FFFFFFFu;
  if (ax >= 0x38800000u && ax <= 0x42800000u) {  // 2^-14 <= |x| <= 64
    float t;
    if (crm::tan_fast(from_bits(ax), &t)) return from_bits(bits(t) ^ (bits(x) & 0x80000000u));
  }
  return crm::trig(x, 2);
}
RSX_HD RSX_NOINL inline float cr_atan2(float y, float x) { return crm::atan2f_cr(y, x); }
RSX_HD RSX_NOINL inline float cr_pow(float x, float y) { return crm::powf_cr(x, y); }

}  // namespace rsx
