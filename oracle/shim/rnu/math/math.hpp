// Minimal stand-in for the `rnu` vector-math header that the reference's
// src/pathtracer/bvh.hpp / bvh.cpp include (`rnu` is an unvendored, unpinned
// dependency: the reference's CMakeLists.txt:12-21 clones it at HEAD).
//
// TEST INFRASTRUCTURE ONLY: used to compile the reference's own BVH sources
// into oracle/_ref. It provides exactly the component-wise IEEE operations the
// reference BVH code uses. Evaluation order is fixed and documented:
//   dot(a, b)   = (a.x*b.x + a.y*b.y) + a.z*b.z
//   cross(a, b) = (a.y*b.z - a.z*b.y, a.z*b.x - a.x*b.z, a.x*b.y - a.y*b.x)
// The oracle restatement and the CUDA kernels use the same order, so the
// Moller-Trumbore results are bit-identical across the three.
#pragma once
#include <cmath>
#include <cstdint>
#include <limits>
#include <type_traits>

namespace rnu {

template <typename T, int N> struct vec;

template <typename T> struct vec<T, 2> {
  T x{}, y{};
  constexpr vec() = default;
  constexpr explicit vec(T s) : x(s), y(s) {}
  constexpr vec(T a, T b) : x(a), y(b) {}
  constexpr T& operator[](std::ptrdiff_t i) { return i == 0 ? x : y; }
  constexpr T operator[](std::ptrdiff_t i) const { return i == 0 ? x : y; }
};

template <typename T> struct vec<T, 3> {
  T x{}, y{}, z{};
  constexpr vec() = default;
  constexpr explicit vec(T s) : x(s), y(s), z(s) {}
  constexpr vec(T a, T b, T c) : x(a), y(b), z(c) {}
  template <typename U>
  constexpr explicit vec(vec<U, 3> const& o) : x(static_cast<T>(o.x)), y(static_cast<T>(o.y)), z(static_cast<T>(o.z)) {}
  template <typename U>
  constexpr explicit vec(vec<U, 4> const& o) : x(static_cast<T>(o.x)), y(static_cast<T>(o.y)), z(static_cast<T>(o.z)) {}
  constexpr T& operator[](std::ptrdiff_t i) { return i == 0 ? x : (i == 1 ? y : z); }
  constexpr T operator[](std::ptrdiff_t i) const { return i == 0 ? x : (i == 1 ? y : z); }
  constexpr vec& operator+=(vec const& o) { x += o.x; y += o.y; z += o.z; return *this; }
  constexpr vec& operator-=(vec const& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
  constexpr vec& operator+=(T s) { x += s; y += s; z += s; return *this; }
  constexpr vec& operator-=(T s) { x -= s; y -= s; z -= s; return *this; }
};

template <typename T> struct vec<T, 4> {
  T x{}, y{}, z{}, w{};
  constexpr vec() = default;
  constexpr explicit vec(T s) : x(s), y(s), z(s), w(s) {}
  constexpr vec(T a, T b, T c, T d) : x(a), y(b), z(c), w(d) {}
};

using vec2 = vec<float, 2>;
using vec3 = vec<float, 3>;
using vec4 = vec<float, 4>;
using vec3i = vec<int, 3>;

#define RNU_SHIM_BINOP(OP)                                                                                 \
  template <typename T> constexpr vec<T, 3> operator OP(vec<T, 3> const& a, vec<T, 3> const& b) {        \
    return vec<T, 3>(a.x OP b.x, a.y OP b.y, a.z OP b.z);                                                 \
  }                                                                                                        \
  template <typename T> constexpr vec<T, 3> operator OP(vec<T, 3> const& a, T s) {                       \
    return vec<T, 3>(a.x OP s, a.y OP s, a.z OP s);                                                       \
  }                                                                                                        \
  template <typename T> constexpr vec<T, 3> operator OP(T s, vec<T, 3> const& a) {                       \
    return vec<T, 3>(s OP a.x, s OP a.y, s OP a.z);                                                       \
  }
RNU_SHIM_BINOP(+)
RNU_SHIM_BINOP(-)
RNU_SHIM_BINOP(*)
RNU_SHIM_BINOP(/)
#undef RNU_SHIM_BINOP

template <typename T> constexpr vec<T, 2> operator*(vec<T, 2> const& a, T s) { return vec<T, 2>(a.x * s, a.y * s); }
template <typename T> constexpr vec<T, 2> operator+(vec<T, 2> const& a, vec<T, 2> const& b) {
  return vec<T, 2>(a.x + b.x, a.y + b.y);
}

template <typename T> constexpr T min(T a, T b) requires std::is_arithmetic_v<T> { return b < a ? b : a; }
template <typename T> constexpr T max(T a, T b) requires std::is_arithmetic_v<T> { return a < b ? b : a; }
template <typename T> constexpr T clamp(T v, T lo, T hi) requires std::is_arithmetic_v<T> {
  return min(max(v, lo), hi);
}
template <typename T> constexpr vec<T, 3> min(vec<T, 3> const& a, vec<T, 3> const& b) {
  return vec<T, 3>(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z));
}
template <typename T> constexpr vec<T, 3> max(vec<T, 3> const& a, vec<T, 3> const& b) {
  return vec<T, 3>(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z));
}
template <typename T> constexpr vec<T, 3> clamp(vec<T, 3> const& v, vec<T, 3> const& lo, vec<T, 3> const& hi) {
  return min(max(v, lo), hi);
}
template <typename T> constexpr T dot(vec<T, 3> const& a, vec<T, 3> const& b) {
  return (a.x * b.x + a.y * b.y) + a.z * b.z;
}
template <typename T> constexpr vec<T, 3> cross(vec<T, 3> const& a, vec<T, 3> const& b) {
  return vec<T, 3>(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <typename T> inline T norm(vec<T, 3> const& a) { return std::sqrt(dot(a, a)); }

// 4x4 column-major matrix, used only by the reference's scene::pick restated in the harness.
struct mat4 {
  vec4 col[4];
};
inline vec4 operator*(mat4 const& m, vec4 const& v) {
  vec4 r;
  r.x = ((m.col[0].x * v.x + m.col[1].x * v.y) + m.col[2].x * v.z) + m.col[3].x * v.w;
  r.y = ((m.col[0].y * v.x + m.col[1].y * v.y) + m.col[2].y * v.z) + m.col[3].y * v.w;
  r.z = ((m.col[0].z * v.x + m.col[1].z * v.y) + m.col[2].z * v.z) + m.col[3].z * v.w;
  r.w = ((m.col[0].w * v.x + m.col[1].w * v.y) + m.col[2].w * v.z) + m.col[3].w * v.w;
  return r;
}

}  // namespace rnu
