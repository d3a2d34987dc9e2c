// Runs the reference's post-processing compute shaders (src/pt/pp_denoise,
// pp_blur, pp_cutoff, pp_add, pp_tonemap, pp_fxaa .comp), rewritten to C++ by
// build_ref.py, on host images. TEST INFRASTRUCTURE ONLY: pins the oracle's
// restatement (oracle_post.cpp) to the reference's own shader code.
//
// The shim below gives the shaders what a GL 4.6 compute dispatch gives them:
// gl_GlobalInvocationID over 8 x 8 groups covering the image (the shaders'
// `pt.x > size.x` check lets the column x = width through: its texelFetch
// reads 0 and its imageStore is dropped, as GL drops stores outside the
// image), texelFetch returning 0 outside the image, texture / textureLod at
// level 0 filtering bilinearly with GL_MIRRORED_REPEAT (the sampler of
// post_process.cpp:41-55), and imageStore into an RGBA16F image (round to
// nearest even). Vector arithmetic rounds every operation separately.
#include <cmath>
#include <cstdint>
#include <cstring>

namespace ppshim {

using uint = uint32_t;
struct vec2;
struct ivec2;
struct uvec2;
struct vec3 {
  float x, y, z;
  vec3() : x(0), y(0), z(0) {}
  explicit vec3(float s) : x(s), y(s), z(s) {}
  vec3(float a, float b, float c) : x(a), y(b), z(c) {}
  vec3& operator+=(vec3 const& o) {
    x += o.x, y += o.y, z += o.z;
    return *this;
  }
};
struct vec4 {
  float x, y, z, w;
  vec4() : x(0), y(0), z(0), w(0) {}
  explicit vec4(float s) : x(s), y(s), z(s), w(s) {}
  vec4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
  vec4(vec3 const& v, float d) : x(v.x), y(v.y), z(v.z), w(d) {}
  vec3 rgb() const { return {x, y, z}; }
  vec3 xyz() const { return {x, y, z}; }
  vec4& operator+=(vec4 const& o) {
    x += o.x, y += o.y, z += o.z, w += o.w;
    return *this;
  }
};
struct bvec4 {
  bool x, y, z, w;
};
struct ivec2 {
  int x, y;
  ivec2() : x(0), y(0) {}
  explicit ivec2(int s) : x(s), y(s) {}
  ivec2(int a, int b) : x(a), y(b) {}
  explicit ivec2(uvec2 const& u);
  explicit ivec2(vec2 const& v);
};
struct uvec2 {
  uint32_t x, y;
  uvec2() : x(0), y(0) {}
  uvec2(uint32_t a, uint32_t b) : x(a), y(b) {}
  explicit uvec2(ivec2 const& v) : x(uint32_t(v.x)), y(uint32_t(v.y)) {}
};
struct vec2 {
  float x, y;
  vec2() : x(0), y(0) {}
  explicit vec2(float s) : x(s), y(s) {}
  vec2(float a, float b) : x(a), y(b) {}
  vec2(int a, int b) : x(float(a)), y(float(b)) {}
  explicit vec2(uvec2 const& u) : x(float(u.x)), y(float(u.y)) {}
  vec2 xy() const { return *this; }
};
inline ivec2::ivec2(uvec2 const& u) : x(int(u.x)), y(int(u.y)) {}
inline ivec2::ivec2(vec2 const& v) : x(int(v.x)), y(int(v.y)) {}
struct uvec3 {
  uint32_t x, y, z;
  uvec2 xy() const { return {x, y}; }
};

inline vec2 operator+(vec2 a, vec2 b) { return {a.x + b.x, a.y + b.y}; }
inline vec2 operator-(vec2 a, vec2 b) { return {a.x - b.x, a.y - b.y}; }
inline vec2 operator*(vec2 a, vec2 b) { return {a.x * b.x, a.y * b.y}; }
inline vec2 operator*(vec2 a, float s) { return {a.x * s, a.y * s}; }
inline vec2 operator*(float s, vec2 a) { return {s * a.x, s * a.y}; }
inline vec2 operator*(int s, vec2 a) { return float(s) * a; }
inline vec2 operator/(vec2 a, vec2 b) { return {a.x / b.x, a.y / b.y}; }
inline vec2 operator/(vec2 a, uvec2 b) { return a / vec2(b); }
inline vec2 operator/(float s, vec2 a) { return {s / a.x, s / a.y}; }
inline vec2 min(vec2 a, vec2 b) { return {b.x < a.x ? b.x : a.x, b.y < a.y ? b.y : a.y}; }
inline vec2 max(vec2 a, vec2 b) { return {a.x < b.x ? b.x : a.x, a.y < b.y ? b.y : a.y}; }
inline ivec2 operator+(ivec2 a, ivec2 b) { return {a.x + b.x, a.y + b.y}; }
inline ivec2 operator-(ivec2 a, int s) { return {a.x - s, a.y - s}; }
inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
inline ivec2 clamp(ivec2 v, ivec2 lo, ivec2 hi) { return {clampi(v.x, lo.x, hi.x), clampi(v.y, lo.y, hi.y)}; }
inline vec3 operator+(vec3 a, vec3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline vec3 operator-(vec3 a, vec3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline vec3 operator-(vec3 a, float s) { return {a.x - s, a.y - s, a.z - s}; }
inline vec3 operator+(vec3 a, float s) { return {a.x + s, a.y + s, a.z + s}; }
inline vec3 operator*(vec3 a, vec3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline vec3 operator*(float s, vec3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline vec3 operator*(vec3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline vec3 operator/(vec3 a, vec3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
inline vec3 operator/(vec3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline float mn(float a, float b) { return b < a ? b : a; }
inline float mx(float a, float b) { return a < b ? b : a; }
inline float min(float a, float b) { return mn(a, b); }
inline float max(float a, float b) { return mx(a, b); }
inline float abs(float v) { return std::fabs(v); }
inline float clamp(float v, float lo, float hi) { return mn(mx(v, lo), hi); }
inline vec3 clamp(vec3 v, float lo, float hi) { return {clamp(v.x, lo, hi), clamp(v.y, lo, hi), clamp(v.z, lo, hi)}; }
inline vec3 max(vec3 a, vec3 b) { return {mx(a.x, b.x), mx(a.y, b.y), mx(a.z, b.z)}; }
inline float dot(vec3 a, vec3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline float exp(float v) { return std::exp(v); }
inline vec3 pow(vec3 a, vec3 b) { return {std::pow(a.x, b.x), std::pow(a.y, b.y), std::pow(a.z, b.z)}; }
inline vec4 operator+(vec4 a, vec4 b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
inline vec4 operator*(float s, vec4 a) { return {s * a.x, s * a.y, s * a.z, s * a.w}; }
inline bvec4 lessThanEqual(vec4 a, vec4 b) { return {a.x <= b.x, a.y <= b.y, a.z <= b.z, a.w <= b.w}; }
inline bvec4 greaterThanEqual(vec4 a, vec4 b) { return {a.x >= b.x, a.y >= b.y, a.z >= b.z, a.w >= b.w}; }
inline vec4 mix(vec4 a, vec4 b, bvec4 s) { return {s.x ? b.x : a.x, s.y ? b.y : a.y, s.z ? b.z : a.z, s.w ? b.w : a.w}; }

float half_rn(float f) {
  uint32_t x;
  std::memcpy(&x, &f, 4);
  uint32_t const sign = x & 0x80000000u, ax = x & 0x7fffffffu;
  if (ax >= 0x7f800000u) return f;
  uint32_t r;
  if (ax >= 0x477ff000u) {
    r = 0x7f800000u;
  } else if (ax < 0x38800000u) {
    float a;
    std::memcpy(&a, &ax, 4);
    float const q = std::nearbyint(a * 16777216.f) * (1.f / 16777216.f);
    std::memcpy(&r, &q, 4);
  } else {
    r = (ax + 0x0fffu + ((ax >> 13) & 1u)) & ~0x1fffu;
  }
  r |= sign;
  float out;
  std::memcpy(&out, &r, 4);
  return out;
}

struct sampler2D {
  float const* p = nullptr;
  int w = 0, h = 0;
};
struct image2D {
  float* p = nullptr;
  int w = 0, h = 0;
};
inline ivec2 textureSize(sampler2D const& s, int) { return {s.w, s.h}; }
inline vec4 texelFetch(sampler2D const& s, ivec2 c, int) {
  if (c.x < 0 || c.y < 0 || c.x >= s.w || c.y >= s.h) return vec4(0.f);
  float const* q = s.p + 4 * (size_t(c.y) * s.w + c.x);
  return {q[0], q[1], q[2], q[3]};
}
inline int mirror_repeat(int i, int size) {
  int m = i % (2 * size);
  if (m < 0) m += 2 * size;
  int const a = m - size;
  return (size - 1) - (a >= 0 ? a : -(1 + a));
}
inline vec4 texture(sampler2D const& s, vec2 uv, float = 0.f) {
  float const u = uv.x * float(s.w) - 0.5f, v = uv.y * float(s.h) - 0.5f;
  float const fu = std::floor(u), fv = std::floor(v);
  float const a = u - fu, b = v - fv;
  int const i0 = int(fu), j0 = int(fv);
  int const x0 = mirror_repeat(i0, s.w), x1 = mirror_repeat(i0 + 1, s.w);
  int const y0 = mirror_repeat(j0, s.h), y1 = mirror_repeat(j0 + 1, s.h);
  float const w00 = (1.f - a) * (1.f - b), w10 = a * (1.f - b), w01 = (1.f - a) * b, w11 = a * b;
  auto t = [&](int x, int y) { return texelFetch(s, ivec2(x, y), 0); };
  return ((w00 * t(x0, y0) + w10 * t(x1, y0)) + w01 * t(x0, y1)) + w11 * t(x1, y1);
}
inline vec4 textureLod(sampler2D const& s, vec2 uv, float) { return texture(s, uv); }
inline void imageStore(image2D const& img, ivec2 c, vec4 v) {
  if (c.x < 0 || c.y < 0 || c.x >= img.w || c.y >= img.h) return;
  float* q = img.p + 4 * (size_t(c.y) * img.w + c.x);
  q[0] = half_rn(v.x), q[1] = half_rn(v.y), q[2] = half_rn(v.z), q[3] = half_rn(v.w);
}

thread_local uvec3 gl_GlobalInvocationID;

}  // namespace ppshim

#define PP_SHADER(NS, FILE) \
  namespace NS {            \
  using namespace ppshim;   \
  _Pragma("GCC diagnostic push") _Pragma("GCC diagnostic ignored \"-Wshadow\"")
#define PP_END _Pragma("GCC diagnostic pop") }

PP_SHADER(pp_denoise, "pp_denoise.comp")
#include "pp_denoise.inc"
PP_END
PP_SHADER(pp_blur, "pp_blur.comp")
#include "pp_blur.inc"
PP_END
PP_SHADER(pp_cutoff, "pp_cutoff.comp")
#include "pp_cutoff.inc"
PP_END
PP_SHADER(pp_add, "pp_add.comp")
#include "pp_add.inc"
PP_END
PP_SHADER(pp_tonemap, "pp_tonemap.comp")
#include "pp_tonemap.inc"
PP_END
PP_SHADER(pp_fxaa, "pp_fxaa.comp")
#include "pp_fxaa.inc"
PP_END

// op numbering as myrt_pp_op (6, the linear blit, has no shader).
extern "C" int ref_post_pass(int op, int const* iparam, float const* fparam, float const* in, int w, int h,
    float const* overlay, int ow, int oh, float* out) {
  using namespace ppshim;
  sampler2D const src{in, w, h};
  image2D const dst{out, w, h};
  auto dispatch = [&](auto&& fn) {
    int const gx = (w + 7) / 8 * 8, gy = (h + 7) / 8 * 8;
    for (int y = 0; y < gy; ++y)
      for (int x = 0; x < gx; ++x) {
        gl_GlobalInvocationID = uvec3{uint32_t(x), uint32_t(y), 0u};
        fn();
      }
  };
  switch (op) {
    case 0:
      pp_denoise::input_image = src, pp_denoise::output_image = dst;
      pp_denoise::exponent = fparam[0], pp_denoise::strength = fparam[1];
      dispatch(pp_denoise::pp_main);
      return 0;
    case 1:
      pp_blur::input_image = src, pp_blur::output_image = dst;
      pp_blur::direction = iparam[0], pp_blur::step = fparam[0];
      dispatch(pp_blur::pp_main);
      return 0;
    case 2:
      pp_cutoff::input_image = src, pp_cutoff::output_image = dst;
      pp_cutoff::value = vec4(fparam[0], fparam[1], fparam[2], fparam[3]);
      pp_cutoff::leave_above = iparam[0] != 0;
      dispatch(pp_cutoff::pp_main);
      return 0;
    case 3:
      pp_add::input_image = src, pp_add::output_image = dst;
      pp_add::overlay_texture = sampler2D{overlay, ow, oh};
      pp_add::factor = fparam[0];
      dispatch(pp_add::pp_main);
      return 0;
    case 4:
      pp_tonemap::input_image = src, pp_tonemap::output_image = dst;
      dispatch(pp_tonemap::pp_main);
      return 0;
    case 5:
      pp_fxaa::input_image = src, pp_fxaa::output_image = dst;
      dispatch(pp_fxaa::pp_main);
      return 0;
    default: return -1;
  }
}
