// GLSL-as-C++ compatibility layer.
//
// TEST INFRASTRUCTURE ONLY. It lets the reference's own shader helper files
// (src/pt/random.glsl, intersect.glsl, ggx.glsl, pbr.glsl, color.glsl,
// transform.glsl, bvh.glsl, bvh.impl.glsl) compile as C++ into oracle/_ref, so
// that the oracle restatement can be pinned against the reference's source
// rather than against a re-reading of it. oracle/build_ref.py applies only
// mechanical rewrites to those files (parameter qualifiers -> references,
// float-literal suffixes, per-invocation globals -> thread_local).
//
// Semantics chosen where GLSL leaves them open (documented, also used by the
// oracle restatement and the CUDA kernels):
//   * dot / cross / matrix products evaluate left to right, no fused multiply-add;
//   * texelFetch outside [0, size) returns 0 (robust buffer access);
//   * int arithmetic wraps (the build passes -fwrapv).
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <type_traits>

namespace glsl {

using uint = std::uint32_t;

struct vec3;
struct vec2;

template <int I0, int I1, int I2, int N> struct swz3 {
  float d[N];
  operator vec3() const;
};
// Readable and writable two-component swizzle (p.xy = p.yx in the Menger fold).
template <int I0, int I1, int N> struct swz2 {
  float d[N];
  operator vec2() const;
  swz2& operator=(vec2 const& v);
  template <int J0, int J1> swz2& operator=(swz2<J0, J1, N> const& o);
};

struct vec2 {
  union {
    struct { float x, y; };
    struct { float r, g; };
    float d[2];
  };
  vec2() : x(0), y(0) {}
  template <typename S> requires std::is_arithmetic_v<S> explicit vec2(S s) : x(float(s)), y(float(s)) {}
  template <typename A, typename B> vec2(A a, B b) : x(float(a)), y(float(b)) {}
  float& operator[](int i) { return d[i]; }
  float operator[](int i) const { return d[i]; }
};

struct vec3 {
  union {
    struct { float x, y, z; };
    struct { float r, g, b; };
    swz3<0, 1, 2, 3> xyz;
    swz3<0, 1, 2, 3> rgb;
    swz2<0, 1, 3> xy;
    swz2<1, 0, 3> yx;
    swz2<0, 2, 3> xz;
    swz2<2, 0, 3> zx;
    swz2<1, 2, 3> yz;
    swz2<2, 1, 3> zy;
    float d[3];
  };
  vec3() : x(0), y(0), z(0) {}
  template <typename S> requires std::is_arithmetic_v<S> explicit vec3(S s) : x(float(s)), y(float(s)), z(float(s)) {}
  template <typename A, typename B, typename C> vec3(A a, B b, C c) : x(float(a)), y(float(b)), z(float(c)) {}
  template <typename S> vec3(vec2 const& v, S s) : x(v.x), y(v.y), z(float(s)) {}
  vec3(vec3 const& o) : x(o.x), y(o.y), z(o.z) {}
  vec3& operator=(vec3 const& o) { x = o.x; y = o.y; z = o.z; return *this; }
  float& operator[](int i) { return d[i]; }
  float operator[](int i) const { return d[i]; }
  vec3& operator+=(vec3 const& o) { x += o.x; y += o.y; z += o.z; return *this; }
  vec3& operator-=(vec3 const& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
  vec3& operator*=(vec3 const& o) { x *= o.x; y *= o.y; z *= o.z; return *this; }
  vec3& operator*=(float s) { x *= s; y *= s; z *= s; return *this; }
  vec3& operator/=(float s) { x /= s; y /= s; z /= s; return *this; }
};

struct vec4 {
  union {
    struct { float x, y, z, w; };
    struct { float r, g, b, a; };
    swz3<0, 1, 2, 4> xyz;
    swz3<0, 1, 2, 4> rgb;
    swz2<0, 1, 4> xy;
    float d[4];
  };
  vec4() : x(0), y(0), z(0), w(0) {}
  template <typename S> requires std::is_arithmetic_v<S> explicit vec4(S s) : x(float(s)), y(float(s)), z(float(s)), w(float(s)) {}
  template <typename A, typename B, typename C, typename D>
  vec4(A a, B b, C c, D e) : x(float(a)), y(float(b)), z(float(c)), w(float(e)) {}
  template <typename S> vec4(vec3 const& v, S s) : x(v.x), y(v.y), z(v.z), w(float(s)) {}
  template <typename A, typename B> vec4(vec2 const& v, A a, B b) : x(v.x), y(v.y), z(float(a)), w(float(b)) {}
  vec4(vec4 const& o) : x(o.x), y(o.y), z(o.z), w(o.w) {}
  vec4& operator=(vec4 const& o) { x = o.x; y = o.y; z = o.z; w = o.w; return *this; }
  float& operator[](int i) { return d[i]; }
  float operator[](int i) const { return d[i]; }
  vec4& operator+=(vec4 const& o) { x += o.x; y += o.y; z += o.z; w += o.w; return *this; }
  vec4& operator*=(vec4 const& o) { x *= o.x; y *= o.y; z *= o.z; w *= o.w; return *this; }
};

template <int I0, int I1, int I2, int N> swz3<I0, I1, I2, N>::operator vec3() const {
  return vec3(d[I0], d[I1], d[I2]);
}
template <int I0, int I1, int N> swz2<I0, I1, N>::operator vec2() const { return vec2(d[I0], d[I1]); }
template <int I0, int I1, int N> swz2<I0, I1, N>& swz2<I0, I1, N>::operator=(vec2 const& v) {
  float const a = v.x, b = v.y;
  d[I0] = a;
  d[I1] = b;
  return *this;
}
template <int I0, int I1, int N>
template <int J0, int J1>
swz2<I0, I1, N>& swz2<I0, I1, N>::operator=(swz2<J0, J1, N> const& o) {
  vec2 const v = o.operator vec2();
  return *this = v;
}

struct ivec2 {
  int x = 0, y = 0;
  ivec2() = default;
  template <typename A, typename B> ivec2(A a, B b) : x(int(a)), y(int(b)) {}
  explicit ivec2(vec2 const& v) : x(int(v.x)), y(int(v.y)) {}
  operator vec2() const { return vec2(x, y); }  // GLSL's implicit ivec2 -> vec2
};
struct uvec2 {
  uint x = 0, y = 0;
  uvec2() = default;
  template <typename S> explicit uvec2(S s) : x(uint(s)), y(uint(s)) {}
  template <typename A, typename B> uvec2(A a, B b) : x(uint(a)), y(uint(b)) {}
  explicit operator vec2() const { return vec2(x, y); }
  explicit operator ivec2() const { return ivec2(int(x), int(y)); }
};
inline bool operator!=(uvec2 a, uvec2 b) { return a.x != b.x || a.y != b.y; }

struct bvec2 { bool x, y; };
struct bvec3 { bool x, y, z; };
inline bool any(bvec2 b) { return b.x || b.y; }
struct bvec4 { bool x, y, z, w; };
inline bool any(bvec3 b) { return b.x || b.y || b.z; }
inline bool any(bvec4 b) { return b.x || b.y || b.z || b.w; }

// ---- vec2 ----
inline vec2 operator+(vec2 a, vec2 b) { return vec2(a.x + b.x, a.y + b.y); }
inline vec2 operator-(vec2 a, vec2 b) { return vec2(a.x - b.x, a.y - b.y); }
inline vec2 operator*(vec2 a, float s) { return vec2(a.x * s, a.y * s); }
inline vec2 operator*(float s, vec2 a) { return vec2(s * a.x, s * a.y); }
inline vec2 operator*(vec2 a, vec2 b) { return vec2(a.x * b.x, a.y * b.y); }
inline vec2 operator/(vec2 a, vec2 b) { return vec2(a.x / b.x, a.y / b.y); }
inline vec2 operator/(vec2 a, float s) { return vec2(a.x / s, a.y / s); }
inline vec2 operator+(vec2 a, float s) { return vec2(a.x + s, a.y + s); }
inline vec2 operator-(vec2 a, float s) { return vec2(a.x - s, a.y - s); }
inline vec2& operator*=(vec2& a, vec2 b) { a.x *= b.x; a.y *= b.y; return a; }
inline bvec2 greaterThanEqual(vec2 a, vec2 b) { return {a.x >= b.x, a.y >= b.y}; }
inline bvec2 lessThan(vec2 a, vec2 b) { return {a.x < b.x, a.y < b.y}; }

// ---- vec3 ----
inline vec3 operator+(vec3 const& a, vec3 const& b) { return vec3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline vec3 operator-(vec3 const& a, vec3 const& b) { return vec3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline vec3 operator*(vec3 const& a, vec3 const& b) { return vec3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline vec3 operator/(vec3 const& a, vec3 const& b) { return vec3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline vec3 operator*(vec3 const& a, float s) { return vec3(a.x * s, a.y * s, a.z * s); }
inline vec3 operator*(float s, vec3 const& a) { return vec3(s * a.x, s * a.y, s * a.z); }
inline vec3 operator/(vec3 const& a, float s) { return vec3(a.x / s, a.y / s, a.z / s); }
inline vec3 operator/(float s, vec3 const& a) { return vec3(s / a.x, s / a.y, s / a.z); }
inline vec3 operator+(vec3 const& a, float s) { return vec3(a.x + s, a.y + s, a.z + s); }
inline vec3 operator+(float s, vec3 const& a) { return vec3(s + a.x, s + a.y, s + a.z); }
inline vec3 operator-(vec3 const& a, float s) { return vec3(a.x - s, a.y - s, a.z - s); }
inline vec3 operator-(vec3 const& a) { return vec3(-a.x, -a.y, -a.z); }
inline bool operator==(vec3 const& a, vec3 const& b) { return a.x == b.x && a.y == b.y && a.z == b.z; }

// ---- vec4 ----
inline vec4 operator+(vec4 const& a, vec4 const& b) { return vec4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
inline vec4 operator*(vec4 const& a, float s) { return vec4(a.x * s, a.y * s, a.z * s, a.w * s); }
inline vec4 operator/(vec4 const& a, float s) { return vec4(a.x / s, a.y / s, a.z / s, a.w / s); }

// ---- scalar helpers ----
inline float min(float a, float b) { return b < a ? b : a; }
inline float max(float a, float b) { return a < b ? b : a; }
inline int min(int a, int b) { return b < a ? b : a; }
inline int max(int a, int b) { return a < b ? b : a; }
inline float min(int a, float b) { return min(float(a), b); }
inline float max(int a, float b) { return max(float(a), b); }
inline float clamp(float v, float lo, float hi) { return min(max(v, lo), hi); }
inline int clamp(int v, int lo, int hi) { return min(max(v, lo), hi); }
inline float abs(float v) { return std::fabs(v); }
inline float sqrt(float v) { return std::sqrt(v); }
inline float pow(float a, float b) { return std::pow(a, b); }
inline float sin(float v) { return std::sin(v); }
inline float cos(float v) { return std::cos(v); }
inline float atan(float v) { return std::atan(v); }
inline float sign(float v) { return v > 0.f ? 1.f : (v < 0.f ? -1.f : 0.f); }
inline bool isnan(float v) { return std::isnan(v); }
inline bool isinf(float v) { return std::isinf(v); }
inline float mix(float a, float b, float t) { return a * (1.f - t) + b * t; }

inline vec2 clamp(vec2 v, vec2 lo, vec2 hi) { return vec2(min(max(v.x, lo.x), hi.x), min(max(v.y, lo.y), hi.y)); }
inline vec3 min(vec3 const& a, vec3 const& b) { return vec3(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)); }
inline vec3 max(vec3 const& a, vec3 const& b) { return vec3(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)); }
inline vec3 clamp(vec3 const& v, float lo, float hi) {
  return vec3(clamp(v.x, lo, hi), clamp(v.y, lo, hi), clamp(v.z, lo, hi));
}
inline vec4 clamp(vec4 const& v, float lo, float hi) {
  return vec4(clamp(v.x, lo, hi), clamp(v.y, lo, hi), clamp(v.z, lo, hi), clamp(v.w, lo, hi));
}
inline vec3 abs(vec3 const& v) { return vec3(abs(v.x), abs(v.y), abs(v.z)); }
inline vec4 pow(vec4 const& a, vec4 const& b) { return vec4(pow(a.x, b.x), pow(a.y, b.y), pow(a.z, b.z), pow(a.w, b.w)); }
inline vec3 pow(vec3 const& a, vec3 const& b) { return vec3(pow(a.x, b.x), pow(a.y, b.y), pow(a.z, b.z)); }
inline bvec3 isnan(vec3 const& v) { return {isnan(v.x), isnan(v.y), isnan(v.z)}; }
inline bvec3 isinf(vec3 const& v) { return {isinf(v.x), isinf(v.y), isinf(v.z)}; }
inline bvec4 isnan(vec4 const& v) { return {isnan(v.x), isnan(v.y), isnan(v.z), isnan(v.w)}; }
inline bvec4 isinf(vec4 const& v) { return {isinf(v.x), isinf(v.y), isinf(v.z), isinf(v.w)}; }

inline vec3 max(vec3 const& a, float s) { return vec3(max(a.x, s), max(a.y, s), max(a.z, s)); }
inline vec3 min(vec3 const& a, float s) { return vec3(min(a.x, s), min(a.y, s), min(a.z, s)); }
inline float length(vec2 const& v) { return sqrt(v.x * v.x + v.y * v.y); }
inline vec3& operator*=(vec3& a, double s) { return a *= float(s); }
inline float dot(vec3 const& a, vec3 const& b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline vec3 cross(vec3 const& a, vec3 const& b) {
  return vec3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline float length(vec3 const& v) { return sqrt(dot(v, v)); }
inline float distance(vec3 const& a, vec3 const& b) { return length(a - b); }
inline vec3 normalize(vec3 const& v) { return v * (1.f / length(v)); }
inline vec3 mix(vec3 const& a, vec3 const& b, float t) { return a * (1.f - t) + b * t; }
inline vec4 mix(vec4 const& a, vec4 const& b, float t) { return a * (1.f - t) + b * t; }
inline vec3 reflect(vec3 const& i, vec3 const& n) { return i - 2.f * dot(n, i) * n; }
inline vec3 refract(vec3 const& i, vec3 const& n, float eta) {
  float const k = 1.f - eta * eta * (1.f - dot(n, i) * dot(n, i));
  if (k < 0.f) return vec3(0.f);
  return eta * i - (eta * dot(n, i) + sqrt(k)) * n;
}
inline vec3 faceforward(vec3 const& n, vec3 const& i, vec3 const& nref) { return dot(nref, i) < 0.f ? n : -n; }

// ---- matrices (column major) ----
struct mat3 {
  vec3 c[3];
  mat3(vec3 const& a, vec3 const& b, vec3 const& d) { c[0] = a; c[1] = b; c[2] = d; }
};
inline vec3 operator*(mat3 const& m, vec3 const& v) {
  return vec3((m.c[0].x * v.x + m.c[1].x * v.y) + m.c[2].x * v.z, (m.c[0].y * v.x + m.c[1].y * v.y) + m.c[2].y * v.z,
      (m.c[0].z * v.x + m.c[1].z * v.y) + m.c[2].z * v.z);
}

struct mat4 {
  vec4 c[4];
  vec4& operator[](int i) { return c[i]; }
  vec4 const& operator[](int i) const { return c[i]; }
};
inline vec4 operator*(mat4 const& m, vec4 const& v) {
  vec4 r;
  for (int k = 0; k < 4; ++k)
    r[k] = ((m.c[0][k] * v.x + m.c[1][k] * v.y) + m.c[2][k] * v.z) + m.c[3][k] * v.w;
  return r;
}
// products summed left to right over k, no fused multiply-add
inline mat4 operator*(mat4 const& a, mat4 const& b) {
  mat4 c;
  for (int col = 0; col < 4; ++col)
    for (int r = 0; r < 4; ++r) {
      float s = a.c[0][r] * b.c[col][0];
      for (int k = 1; k < 4; ++k) s = s + a.c[k][r] * b.c[col][k];
      c.c[col][r] = s;
    }
  return c;
}
// inverse by cofactors in double, rounded once to float (GLSL leaves the method
// to the implementation)
inline mat4 inverse(mat4 const& a) {
  double m[16], inv[16];
  for (int i = 0; i < 16; ++i) m[i] = a.c[i / 4][i % 4];
  inv[0] = m[5] * m[10] * m[15] - m[5] * m[11] * m[14] - m[9] * m[6] * m[15] + m[9] * m[7] * m[14] +
      m[13] * m[6] * m[11] - m[13] * m[7] * m[10];
  inv[4] = -m[4] * m[10] * m[15] + m[4] * m[11] * m[14] + m[8] * m[6] * m[15] - m[8] * m[7] * m[14] -
      m[12] * m[6] * m[11] + m[12] * m[7] * m[10];
  inv[8] = m[4] * m[9] * m[15] - m[4] * m[11] * m[13] - m[8] * m[5] * m[15] + m[8] * m[7] * m[13] +
      m[12] * m[5] * m[11] - m[12] * m[7] * m[9];
  inv[12] = -m[4] * m[9] * m[14] + m[4] * m[10] * m[13] + m[8] * m[5] * m[14] - m[8] * m[6] * m[13] -
      m[12] * m[5] * m[10] + m[12] * m[6] * m[9];
  inv[1] = -m[1] * m[10] * m[15] + m[1] * m[11] * m[14] + m[9] * m[2] * m[15] - m[9] * m[3] * m[14] -
      m[13] * m[2] * m[11] + m[13] * m[3] * m[10];
  inv[5] = m[0] * m[10] * m[15] - m[0] * m[11] * m[14] - m[8] * m[2] * m[15] + m[8] * m[3] * m[14] +
      m[12] * m[2] * m[11] - m[12] * m[3] * m[10];
  inv[9] = -m[0] * m[9] * m[15] + m[0] * m[11] * m[13] + m[8] * m[1] * m[15] - m[8] * m[3] * m[13] -
      m[12] * m[1] * m[11] + m[12] * m[3] * m[9];
  inv[13] = m[0] * m[9] * m[14] - m[0] * m[10] * m[13] - m[8] * m[1] * m[14] + m[8] * m[2] * m[13] +
      m[12] * m[1] * m[10] - m[12] * m[2] * m[9];
  inv[2] = m[1] * m[6] * m[15] - m[1] * m[7] * m[14] - m[5] * m[2] * m[15] + m[5] * m[3] * m[14] +
      m[13] * m[2] * m[7] - m[13] * m[3] * m[6];
  inv[6] = -m[0] * m[6] * m[15] + m[0] * m[7] * m[14] + m[4] * m[2] * m[15] - m[4] * m[3] * m[14] -
      m[12] * m[2] * m[7] + m[12] * m[3] * m[6];
  inv[10] = m[0] * m[5] * m[15] - m[0] * m[7] * m[13] - m[4] * m[1] * m[15] + m[4] * m[3] * m[13] +
      m[12] * m[1] * m[7] - m[12] * m[3] * m[5];
  inv[14] = -m[0] * m[5] * m[14] + m[0] * m[6] * m[13] + m[4] * m[1] * m[14] - m[4] * m[2] * m[13] -
      m[12] * m[1] * m[6] + m[12] * m[2] * m[5];
  inv[3] = -m[1] * m[6] * m[11] + m[1] * m[7] * m[10] + m[5] * m[2] * m[11] - m[5] * m[3] * m[10] -
      m[9] * m[2] * m[7] + m[9] * m[3] * m[6];
  inv[7] = m[0] * m[6] * m[11] - m[0] * m[7] * m[10] - m[4] * m[2] * m[11] + m[4] * m[3] * m[10] +
      m[8] * m[2] * m[7] - m[8] * m[3] * m[6];
  inv[11] = -m[0] * m[5] * m[11] + m[0] * m[7] * m[9] + m[4] * m[1] * m[11] - m[4] * m[3] * m[9] -
      m[8] * m[1] * m[7] + m[8] * m[3] * m[5];
  inv[15] = m[0] * m[5] * m[10] - m[0] * m[6] * m[9] - m[4] * m[1] * m[10] + m[4] * m[2] * m[9] +
      m[8] * m[1] * m[6] - m[8] * m[2] * m[5];
  double const det = m[0] * inv[0] + m[1] * inv[4] + m[2] * inv[8] + m[3] * inv[12];
  mat4 r;
  for (int i = 0; i < 16; ++i) r.c[i / 4][i % 4] = float(inv[i] / det);
  return r;
}
inline mat4 transpose(mat4 const& m) {
  mat4 t;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) t.c[i][j] = m.c[j][i];
  return t;
}

// ---- packing ----
inline uint floatBitsToUint(float f) { uint u; std::memcpy(&u, &f, 4); return u; }
inline float uintBitsToFloat(uint u) { float f; std::memcpy(&f, &u, 4); return f; }
inline uint packUnorm4x8(vec4 const& v) {
  uint r = 0;
  for (int i = 0; i < 4; ++i) {
    float const c = clamp(v[i], 0.f, 1.f);
    r |= uint(std::nearbyint(c * 255.f)) << (8 * i);
  }
  return r;
}
inline vec4 unpackUnorm4x8(uint p) {
  return vec4(float(p & 0xffu) / 255.f, float((p >> 8) & 0xffu) / 255.f, float((p >> 16) & 0xffu) / 255.f,
      float((p >> 24) & 0xffu) / 255.f);
}

// ---- 1-D float texture (the reference's random texture) ----
struct sampler1D {
  float const* data = nullptr;
  int size = 0;
};
inline int textureSize(sampler1D const& s, int) { return s.size; }
inline vec4 texelFetch(sampler1D const& s, int i, int) {
  if (i < 0 || i >= s.size) return vec4(0.f);
  return vec4(s.data[i], 0.f, 0.f, 1.f);
}

}  // namespace glsl
