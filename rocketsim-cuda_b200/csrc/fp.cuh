// Float policy of the simulator: every float operation of the physics is one IEEE binary32 operation rounded to
// nearest, never fused.  On the device that is the explicit _rn intrinsics (which nvcc never contracts, whatever the
// flags); on the host it is the plain operator in a translation unit built with -ffp-contract=off and no FMA target.
// The same source therefore computes the same bits on both sides, and the same bits as the reference's correctly
// rounded CPU build (crates/rocketsim-cuda/csrc/phase.cpp over cuda/common/hd.cuh:45-141), which uses the same policy.
//
// Division is IEEE division (__fdiv_rn, the library's correctly rounded quotient), square root is __fsqrt_rn.
#pragma once
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define RSX_HD __host__ __device__
#if defined(RSX_SOFT_INLINE)
#define RSX_INL inline
#else
#define RSX_INL __forceinline__
#endif
#define RSX_NOINL __noinline__
#else
#define RSX_HD
#define RSX_INL inline
#define RSX_NOINL __attribute__((noinline))
#endif
#define RSX_F RSX_HD RSX_INL

#if !defined(__CUDACC__) && (defined(__FMA__) || defined(__AVX2__) || defined(__FP_FAST_FMAF))
#error "the host build of the simulator must not target FMA (build without -march=native / -mfma)"
#endif

namespace rsx {

#if defined(__CUDA_ARCH__)
RSX_F float fadd(float a, float b) { return __fadd_rn(a, b); }
RSX_F float fsub(float a, float b) { return __fsub_rn(a, b); }
RSX_F float fmul(float a, float b) { return __fmul_rn(a, b); }
RSX_F float fdiv(float a, float b) { return __fdiv_rn(a, b); }
RSX_F float fsqrt(float a) { return __fsqrt_rn(a); }
RSX_F uint32_t bits(float a) { return __float_as_uint(a); }
RSX_F float from_bits(uint32_t u) { return __uint_as_float(u); }
RSX_F float i2f(int32_t v) { return __int2float_rn(v); }
RSX_F float u2f(uint32_t v) { return __uint2float_rn(v); }
RSX_F float ull2f(uint64_t v) { return __ull2float_rn(v); }
RSX_F float ffma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
#else
RSX_F float fadd(float a, float b) { return a + b; }
RSX_F float fsub(float a, float b) { return a - b; }
RSX_F float fmul(float a, float b) { return a * b; }
RSX_F float fdiv(float a, float b) { return a / b; }
RSX_F float fsqrt(float a) { return __builtin_sqrtf(a); }
RSX_F uint32_t bits(float a) { uint32_t u; memcpy(&u, &a, 4); return u; }
RSX_F float from_bits(uint32_t u) { float a; memcpy(&a, &u, 4); return a; }
RSX_F float i2f(int32_t v) { return (float)v; }
RSX_F float u2f(uint32_t v) { return (float)v; }
RSX_F float ull2f(uint64_t v) { return (float)v; }
// the correctly rounded fused multiply-add of the C library (the same value as the device's __fmaf_rn)
RSX_F float ffma(float a, float b, float c) { return __builtin_fmaf(a, b, c); }
#endif

// Rust `i64 as f32`: round to nearest even (hd.cuh:144-148 reaches it through the unsigned conversion).
RSX_F float ll2f(int64_t v) {
  if (v >= -2147483648LL && v <= 2147483647LL) return i2f((int32_t)v);
  float m = ull2f(v < 0 ? 0ull - (uint64_t)v : (uint64_t)v);
  return v < 0 ? from_bits(bits(m) ^ 0x80000000u) : m;
}

// ---- scalar helpers with the semantics the reference gives them (cuda/common/glam.cuh:29-70) ----
RSX_F float fneg(float a) { return from_bits(bits(a) ^ 0x80000000u); }
RSX_F float fabs_(float a) { return from_bits(bits(a) & 0x7FFFFFFFu); }
RSX_F bool isnan_(float a) { return (bits(a) & 0x7FFFFFFFu) > 0x7F800000u; }
RSX_F bool isfinite_(float a) { return (bits(a) & 0x7FFFFFFFu) < 0x7F800000u; }
// SSE _mm_min_ps / _mm_max_ps: the second operand wins on NaN and on a tie of zeros.
RSX_F float sse_min(float a, float b) { return a < b ? a : b; }
RSX_F float sse_max(float a, float b) { return a > b ? a : b; }
// Rust f32::min / max: a NaN operand is ignored.
RSX_F float rmin(float a, float b) { return isnan_(a) ? b : isnan_(b) ? a : (a < b ? a : b); }
RSX_F float rmax(float a, float b) { return isnan_(a) ? b : isnan_(b) ? a : (a > b ? a : b); }
// Rust f32::clamp (lower bound first)
RSX_F float rclamp(float x, float lo, float hi) {
  x = x < lo ? lo : x;
  return x > hi ? hi : x;
}
RSX_F float rsignum(float a) { return isnan_(a) ? a : from_bits((bits(a) & 0x80000000u) | 0x3F800000u); }
// Rust `f32 as i32 / u32 / u64`: saturating, NaN to 0.
RSX_F int32_t f2i(float a) {
  if (isnan_(a)) return 0;
  if (a >= 2147483648.0f) return 0x7FFFFFFF;
  if (a <= -2147483648.0f) return (int32_t)0x80000000u;
  return (int32_t)a;
}
RSX_F uint32_t mask_of(bool c) { return c ? 0xFFFFFFFFu : 0u; }
RSX_F float select_bits(uint32_t m, float t, float f) { return from_bits((bits(f) & ~m) | (bits(t) & m)); }

}  // namespace rsx
