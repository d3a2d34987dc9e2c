// GLSL's sin, cos, atan, pow and exp as this library computes them in the
// reference-shading mode, the forward preview's resolve and the
// post-processing passes -- one definition compiled for the device and for the
// host.
//
// GLSL leaves the precision of these built-ins to the implementation (GLSL
// 4.60 section 4.7.1: pow and exp "inherited from exp2 and log2", i.e. up to
// 3 + 2 |y log2 x| ulp); the reference's GL driver supplies its own. CUDA's
// sinf / powf and the host libm differ from each other in the last bits, so a
// device render and its CPU oracle could not agree bit for bit. These
// functions use only IEEE-exact operations -- +, -, *, /, fused multiply-add,
// rounding to an integer, exponent bit manipulation -- each rounded on its own,
// so the device and any host compiled with -ffp-contract=off (the oracle)
// produce the same bits.
//
// Methods (all standard, coefficients fitted by myrt_b200/glmath_fit.py with
// Lawson's iteratively reweighted least squares on Chebyshev nodes):
// * sin / cos: Cody-Waite reduction by pi/2 (Cody and Waite, "Software Manual
//   for the Elementary Functions", 1980) with a three-part float split of pi/2
//   and fused multiply-adds, then odd / even polynomials on [-pi/4, pi/4] and
//   the quadrant. Within 2 ulp for |x| < 10^5 (the shading passes call them on
//   angles in [0, 2 pi]).
// * atan: atan(x) = pi/2 - atan(1/x) for |x| > 1, atan(t) = pi/4 +
//   atan((t - 1) / (t + 1)) above tan(pi/8), an odd polynomial below.
// * pow(x, y) = 2^(y log2 x): log of the mantissa in [sqrt(1/2), sqrt(2)) as
//   2 s + s^3 L(s^2) with s = (m - 1) / (m + 1), y log2 x carried as a
//   float pair through fused multiply-adds and a two-sum, 2^f on [-1/2, 1/2]
//   by a polynomial and the exponent set by bits. exp(x) = 2^(x log2 e) the
//   same way.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

#if defined(__CUDACC__)
#define MYRT_GLM __host__ __device__ __forceinline__
#else
#define MYRT_GLM inline
#endif

namespace myrt_glmath {

// ---- exactly rounded primitives (no contraction on either side) ----
MYRT_GLM float add(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fadd_rn(a, b);
#else
  return a + b;
#endif
}
MYRT_GLM float sub(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fsub_rn(a, b);
#else
  return a - b;
#endif
}
MYRT_GLM float mul(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fmul_rn(a, b);
#else
  return a * b;
#endif
}
MYRT_GLM float div(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fdiv_rn(a, b);
#else
  return a / b;
#endif
}
MYRT_GLM float fma(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
  return __fmaf_rn(a, b, c);
#else
  return std::fmaf(a, b, c);
#endif
}
MYRT_GLM float rint(float a) {  // round half to even
#if defined(__CUDA_ARCH__)
  return rintf(a);
#else
  return std::nearbyintf(a);
#endif
}
MYRT_GLM float floor(float a) {
#if defined(__CUDA_ARCH__)
  return floorf(a);
#else
  return std::floor(a);
#endif
}
MYRT_GLM uint32_t bits(float a) {
#if defined(__CUDA_ARCH__)
  return __float_as_uint(a);
#else
  uint32_t u;
  std::memcpy(&u, &a, 4);
  return u;
#endif
}
MYRT_GLM float from_bits(uint32_t u) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float a;
  std::memcpy(&a, &u, 4);
  return a;
#endif
}
MYRT_GLM bool is_nan(float a) { return a != a; }
MYRT_GLM float abs(float a) { return from_bits(bits(a) & 0x7fffffffu); }
MYRT_GLM float with_sign_of(float mag, float s) {
  return from_bits((bits(mag) & 0x7fffffffu) | (bits(s) & 0x80000000u));
}

// ---- constants: float splits of the exact values ----
constexpr float kPio2_1 = 0x1.921fb6p+0f;  // pi/2 = kPio2_1 + kPio2_2 + kPio2_3 (+ < 2^-74)
constexpr float kPio2_2 = -0x1.777a5cp-25f;
constexpr float kPio2_3 = -0x1.ee59dap-50f;
constexpr float kPio4_hi = 0x1.921fb6p-1f;  // pi/4 = hi + lo
constexpr float kPio4_lo = -0x1.777a5cp-26f;
constexpr float kTwoOverPi = 0x1.45f306p-1f;
constexpr float kTanPi8 = 0x1.a8279ap-2f;
constexpr float kSqrt2 = 0x1.6a09e6p+0f;
constexpr float kLog2e_hi = 0x1.715476p+0f;  // log2(e) = hi + lo
constexpr float kLog2e_lo = 0x1.4ae0c0p-26f;

// ---- polynomial kernels (myrt_b200/glmath_fit.py) ----
MYRT_GLM float sin_kernel(float r) {  // r in [-pi/4, pi/4]
  float const z = mul(r, r);
  float p = fma(z, 2.718274345e-06f, -1.983933180e-04f);
  p = fma(z, p, 8.333329111e-03f);
  p = fma(z, p, -1.666666716e-01f);
  return fma(mul(r, z), p, r);
}
MYRT_GLM float cos_kernel(float r) {
  float const z = mul(r, r);
  float p = fma(z, -2.720577470e-07f, 2.479945942e-05f);
  p = fma(z, p, -1.388888340e-03f);
  p = fma(z, p, 4.166666791e-02f);
  return fma(mul(z, z), p, fma(-0.5f, z, 1.0f));
}
MYRT_GLM float atan_kernel(float u) {  // |u| <= tan(pi/8)
  float const z = mul(u, u);
  float p = fma(z, 4.749976099e-02f, -8.479400724e-02f);
  p = fma(z, p, 1.104531363e-01f);
  p = fma(z, p, -1.428206414e-01f);
  p = fma(z, p, 1.999990642e-01f);
  p = fma(z, p, -3.333333135e-01f);
  return fma(mul(u, z), p, u);
}
MYRT_GLM float exp2_kernel(float f) {  // f in [-1/2, 1/2]: 2^f
  float p = fma(f, 1.518459612e-05f, 1.546698186e-04f);
  p = fma(f, p, 1.333399094e-03f);
  p = fma(f, p, 9.618037380e-03f);
  p = fma(f, p, 5.550410226e-02f);
  p = fma(f, p, 2.402265072e-01f);
  p = fma(f, p, 6.931471825e-01f);
  return fma(f, p, 1.0f);
}
// v * 2^n for v in [1/2, 2] and n in [-151, 129], one rounding (into the
// subnormal range too)
MYRT_GLM float scale2(float v, int n) {
  if (n > 127) return mul(mul(v, from_bits(uint32_t(n - 64 + 127) << 23)), 0x1p64f);
  if (n < -126) return mul(mul(v, from_bits(uint32_t(n + 64 + 127) << 23)), 0x1p-64f);
  return mul(v, from_bits(uint32_t(n + 127) << 23));
}
// 2^(hi + lo), |lo| << 1
MYRT_GLM float exp2_pair(float hi, float lo) {
  if (hi > 128.5f) return from_bits(0x7f800000u);
  if (hi < -150.5f) return 0.0f;
  float const n = rint(hi);
  float const f = add(sub(hi, n), lo);
  return scale2(exp2_kernel(f), int(n));
}
// quadrant of k (k a float integer): k mod 4 in 0..3
MYRT_GLM int quadrant(float k) { return int(sub(k, mul(4.0f, floor(mul(k, 0.25f))))); }

// ---- the GLSL built-ins ----
MYRT_GLM float sin(float x) {
  if (!(abs(x) <= 1e30f)) return sub(x, x);  // inf, nan -> nan
  if (x == 0.0f) return x;
  float const k = rint(mul(x, kTwoOverPi));
  float r = fma(-k, kPio2_1, x);
  r = fma(-k, kPio2_2, r);
  r = fma(-k, kPio2_3, r);
  switch (quadrant(k)) {
    case 0: return sin_kernel(r);
    case 1: return cos_kernel(r);
    case 2: return -sin_kernel(r);
    default: return -cos_kernel(r);
  }
}
MYRT_GLM float cos(float x) {
  if (!(abs(x) <= 1e30f)) return sub(x, x);
  float const k = rint(mul(x, kTwoOverPi));
  float r = fma(-k, kPio2_1, x);
  r = fma(-k, kPio2_2, r);
  r = fma(-k, kPio2_3, r);
  switch (quadrant(k)) {
    case 0: return cos_kernel(r);
    case 1: return -sin_kernel(r);
    case 2: return -cos_kernel(r);
    default: return sin_kernel(r);
  }
}
MYRT_GLM float atan(float x) {
  if (is_nan(x)) return add(x, x);
  float const a = abs(x);
  bool const inv = a > 1.0f;
  float const t = inv ? div(1.0f, a) : a;
  bool const red = t > kTanPi8;
  float const u = red ? div(sub(t, 1.0f), add(t, 1.0f)) : t;
  float r = atan_kernel(u);
  if (red) r = add(kPio4_hi, add(r, kPio4_lo));
  if (inv) r = add(sub(2.0f * kPio4_hi, r), 2.0f * kPio4_lo);
  return with_sign_of(r, x);
}
MYRT_GLM float exp(float x) {
  if (is_nan(x)) return add(x, x);
  if (x > 89.0f) return from_bits(0x7f800000u);
  if (x < -104.0f) return 0.0f;
  float const th = mul(x, kLog2e_hi);
  float tl = fma(x, kLog2e_hi, -th);
  tl = fma(x, kLog2e_lo, tl);
  return exp2_pair(th, tl);
}
MYRT_GLM float pow(float x, float y) {
  if (y == 0.0f || x == 1.0f) return 1.0f;
  if (is_nan(x) || is_nan(y)) return add(x, y);
  if (x < 0.0f) return from_bits(0x7fc00000u);  // undefined in GLSL: nan
  float const inf = from_bits(0x7f800000u);
  if (x == 0.0f) return y > 0.0f ? 0.0f : inf;
  if (x == inf) return y > 0.0f ? inf : 0.0f;
  if (abs(y) == inf) return (x < 1.0f) == (y > 0.0f) ? 0.0f : inf;
  // x = m 2^e, m in [sqrt(1/2), sqrt(2))
  uint32_t b = bits(x);
  int e = 0;
  if (b < 0x00800000u) {  // subnormal
    b = bits(mul(x, 0x1p23f));
    e = -23;
  }
  e += int(b >> 23) - 127;
  float m = from_bits((b & 0x007fffffu) | 0x3f800000u);
  if (m > kSqrt2) {
    m = mul(m, 0.5f);
    e += 1;
  }
  float const s = div(sub(m, 1.0f), add(m, 1.0f));
  float const z = mul(s, s);
  float p = fma(z, 2.357515693e-01f, 2.853771746e-01f);
  p = fma(z, p, 4.000032842e-01f);
  p = fma(z, p, 6.666666865e-01f);
  float const ln_m = fma(mul(s, z), p, add(s, s));
  // y log2 x = y e + y ln_m log2(e), carried as hi + lo
  float const lh = mul(ln_m, kLog2e_hi);
  float const ll = fma(ln_m, kLog2e_lo, fma(ln_m, kLog2e_hi, -lh));
  float const fe = float(e);
  float const eh = mul(y, fe);
  float const el = fma(y, fe, -eh);
  float const ph = mul(y, lh);
  float const pl = fma(y, ll, fma(y, lh, -ph));
  float const hi = add(eh, ph);  // two-sum: hi + err = eh + ph exactly
  float const bv = sub(hi, eh);
  float const err = add(sub(eh, sub(hi, bv)), sub(ph, bv));
  return exp2_pair(hi, add(err, add(el, pl)));
}

}  // namespace myrt_glmath
