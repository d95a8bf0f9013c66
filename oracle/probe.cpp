// Test-only probe of the reference's correctly rounded libm (cuda/common/libm_cr.cuh): the two f64 helpers of the
// auto-flip path (car_pre_tick.cuh:40 atan2_64, :64 hypot64) on float arguments, returned as the float the reference
// keeps of them.  Built by oracle/Makefile into oracle/_ref/ beside the reference's own CPU simulator.
#include "common/libm_cr.cuh"
extern "C" {
float rsref_atan2_64_f(float a0, float a1) { return (float)lfcr::atan2_64_cr((double)a0, (double)a1); }
float rsref_hypot64_f(float a, float b) { return (float)lfcr::hypot64_cr((double)a, (double)b); }
float rsref_sinf(float x) { return lfcr::sinf_cr(x); }
float rsref_cosf(float x) { return lfcr::cosf_cr(x); }
float rsref_tanf(float x) { return lfcr::tanf_cr(x); }
float rsref_atan2f(float y, float x) { return lfcr::atan2f_cr(y, x); }
float rsref_powf(float x, float y) { return lfcr::powf_cr(x, y); }
// the same over arrays (for large test samples)
void rsref_atan2f_batch(const float* y, const float* x, float* out, unsigned long long n) {
  for (unsigned long long i = 0; i < n; ++i) out[i] = lfcr::atan2f_cr(y[i], x[i]);
}
void rsref_atan2_64_f_batch(const float* y, const float* x, float* out, unsigned long long n) {
  for (unsigned long long i = 0; i < n; ++i) out[i] = (float)lfcr::atan2_64_cr((double)y[i], (double)x[i]);
}
void rsref_hypot64_f_batch(const float* a, const float* b, float* out, unsigned long long n) {
  for (unsigned long long i = 0; i < n; ++i) out[i] = (float)lfcr::hypot64_cr((double)a[i], (double)b[i]);
}
void rsref_tanf_batch(const float* x, float* out, unsigned long long n) {
  for (unsigned long long i = 0; i < n; ++i) out[i] = lfcr::tanf_cr(x[i]);
}
}
