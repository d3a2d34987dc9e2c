// Device restatement of the reference's shading helpers for the
// "reference shading" wavefront mode:
//   src/pt/random.glsl:14-85          (rng_*)
//   src/pt/ggx.glsl:9-43, pbr.glsl:29-232, transform.glsl:3-15, color.glsl
//   src/pt/material_new.glsl:14-49 + the dispatch material_registry emits
//   (src/material.hpp:39-65) for the single PBR type (7 floats).
// This translation unit is compiled with -fmad=false so every + and * rounds
// separately, as the GLSL reads; random draws happen in the left-to-right
// order GLSL defines for arguments. The transcendentals sin, cos, atan and
// pow are this library's GLSL built-ins (glmath.hpp), which the CPU oracle
// evaluates to the same bits; sqrt and division are IEEE.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "glmath.hpp"

namespace myrt_b200 {
namespace rs {

struct v2 {
  float x, y;
};
struct v3 {
  float x, y, z;
};
__device__ __forceinline__ v3 operator+(v3 a, v3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ v3 operator-(v3 a, v3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ v3 operator-(v3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ v3 operator*(v3 a, v3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ v3 operator*(v3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ v3 operator*(float s, v3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ v3 operator/(v3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ float dot(v3 a, v3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__device__ __forceinline__ v3 cross(v3 a, v3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float length(v3 v) { return sqrtf(dot(v, v)); }
__device__ __forceinline__ v3 normalize(v3 v) { return v * (1.f / length(v)); }
__device__ __forceinline__ float gmin(float a, float b) { return b < a ? b : a; }
__device__ __forceinline__ float gmax(float a, float b) { return a < b ? b : a; }
__device__ __forceinline__ float gclamp(float v, float lo, float hi) { return gmin(gmax(v, lo), hi); }
__device__ __forceinline__ v3 clamp3(v3 v, float lo, float hi) {
  return {gclamp(v.x, lo, hi), gclamp(v.y, lo, hi), gclamp(v.z, lo, hi)};
}
__device__ __forceinline__ float mixf(float a, float b, float t) { return a * (1.f - t) + b * t; }
__device__ __forceinline__ v3 mix3(v3 a, v3 b, float t) { return a * (1.f - t) + b * t; }
__device__ __forceinline__ bool nan3(v3 v) { return isnan(v.x) || isnan(v.y) || isnan(v.z); }
__device__ __forceinline__ bool inf3(v3 v) { return isinf(v.x) || isinf(v.y) || isinf(v.z); }
__device__ __forceinline__ float signf(float v) { return v > 0.f ? 1.f : (v < 0.f ? -1.f : 0.f); }
__device__ __forceinline__ v3 faceforward(v3 n, v3 i, v3 nref) { return dot(nref, i) < 0.f ? n : -n; }
__device__ __forceinline__ v3 reflect(v3 i, v3 n) { return i - 2.f * dot(n, i) * n; }
__device__ __forceinline__ v3 refract(v3 i, v3 n, float eta) {
  float const k = 1.f - eta * eta * (1.f - dot(n, i) * dot(n, i));
  if (k < 0.f) return {0.f, 0.f, 0.f};
  return eta * i - (eta * dot(n, i) + sqrtf(k)) * n;
}

// int(float) with the x86 result for out-of-range inputs (INT_MIN), so the
// device and the reference build agree on the (rare) saturated draws.
__device__ __forceinline__ int f2i(float f) {
  if (!(f > -2147483648.0f && f < 2147483648.0f)) return int(0x80000000u);
  return __float2int_rz(f);
}

__device__ __forceinline__ uint32_t pack_unorm4x8(float x, float y, float z, float w) {
  float const v[4] = {x, y, z, w};
  uint32_t r = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) r |= uint32_t(__float2int_rn(gclamp(v[i], 0.f, 1.f) * 255.f)) << (8 * i);
  return r;
}
__device__ __forceinline__ v3 unpack_rgb(uint32_t p) {
  return {float(p & 0xffu) / 255.f, float((p >> 8) & 0xffu) / 255.f, float((p >> 16) & 0xffu) / 255.f};
}

// ---- random.glsl ---------------------------------------------------------------
struct rng_t {
  uint32_t state;
  int prime;
  float const* tex;  // the pass's 1024-float random texture
};
__device__ __forceinline__ uint32_t wang(uint32_t a) {
  a = (a ^ 61u) ^ (a >> 16);
  a = a + (a << 3);
  a = a ^ (a >> 4);
  a = a * 0x27d4eb2du;
  a = a ^ (a >> 15);
  return a;
}
__device__ __forceinline__ float random_value(rng_t& r, int seed) {
  r.state += wang(uint32_t(seed));
  r.state ^= (r.state << 13);
  r.state ^= (r.state >> 17);
  r.state ^= (r.state << 5);
  return gclamp(float(r.state) * (1.f / 4294967296.f), 0.f, 1.f);
}
__device__ __forceinline__ int random_int(rng_t& r, int seed) { return f2i(random_value(r, seed) * 2147483648.f); }
__device__ __forceinline__ void random_init(rng_t& r, float const* tex, int px, int py, int seed) {
  r.state = uint32_t(seed);
  r.prime = 0;
  r.tex = tex;
  int const a = random_int(r, px ^ 0xba77fa);
  int const b = random_int(r, py ^ 0xcca6df);
  int const c = random_int(r, seed);
  int const seed_base = int(uint32_t(a) * 69019u + uint32_t(b) * 96013u + uint32_t(c));
  int const ti = seed_base % 1024;
  float const t = (ti < 0) ? 0.f : __ldg(tex + ti);
  random_value(r, int(uint32_t(seed_base) + uint32_t(f2i(16756614.f * t))));
}
__device__ __forceinline__ float random_next(rng_t& r) {
  r.prime = r.prime == 5 ? 0 : r.prime + 1;
  return random_value(r, r.prime);
}
// random.glsl:77-85
__device__ __forceinline__ v2 random_uniform_circle(rng_t& r, float radius) {
  float const a = random_next(r) * 2.f * 3.1415926535897f;
  float const b = random_next(r);
  float const s = sqrtf(b) * radius;
  return {s * myrt_glmath::sin(a), s * myrt_glmath::cos(a)};
}

// ---- ggx.glsl / pbr.glsl / transform.glsl ----------------------------------------
constexpr float kPi = 3.1415926535897f;
__device__ __forceinline__ float ggx_distribution(v3 n, v3 h, float alpha) {
  float const ndotm = dot(n, h);
  float const a2 = alpha * alpha;
  float const den = ndotm * ndotm * (a2 - 1.f) + 1.f;
  return a2 / (kPi * den * den);
}
__device__ __forceinline__ v2 ggx_importance_sample(v2 rsm, float roughness) {
  float const phi = rsm.y * 2.f * kPi;
  float const rough2 = roughness * roughness;
  float const theta = myrt_glmath::atan(sqrtf(rough2 * rsm.x / (1.f - rsm.x)));
  return {phi, theta};
}
__device__ __forceinline__ v3 sample_hemisphere(v2 is) {
  float const c = myrt_glmath::cos(is.y), s = myrt_glmath::sin(is.y);
  return {s * myrt_glmath::cos(is.x), s * myrt_glmath::sin(is.x), c};
}
__device__ __forceinline__ v3 transform_local_to_world(v3 v, v3 n) {
  v3 perp{1.f, 0.f, 0.f};
  v3 u = normalize(cross(n, perp));
  if (nan3(u)) {
    perp = {0.f, 1.f, 0.f};
    u = normalize(cross(n, perp));
    if (nan3(u)) {
      perp = {0.f, 0.f, 1.f};
      u = normalize(cross(n, perp));
    }
  }
  v3 const c = cross(n, u);
  v3 const r{(u.x * v.x + c.x * v.y) + n.x * v.z, (u.y * v.x + c.y * v.y) + n.y * v.z,
      (u.z * v.x + c.z * v.y) + n.z * v.z};
  return normalize(r);
}
__device__ __forceinline__ float fresnel(float cos_theta, float ior_in, float ior_out, float metallic) {
  float f0 = fabsf((ior_in - ior_out) / (ior_in + ior_out));
  f0 = mixf(f0 * f0, 1.f, metallic);
  return f0 + (1.f - f0) * myrt_glmath::pow(1.f - cos_theta, 5.f);
}
__device__ __forceinline__ v3 nreflect(v3 tv, v3 n, v3 mn) {
  v3 ray = reflect(-tv, mn);
  float const d = dot(ray, n);
  if (d < 0.f) ray = ray - 2.f * d * n;
  return normalize(ray);
}
__device__ __forceinline__ float schlick(float ndv, float k) { return 1.f / (ndv * (1.f - k) + k); }
__device__ __forceinline__ float smith(v3 N, v3 V, v3 L, float k) {
  float const ndv = fabsf(dot(N, V)), ndl = fabsf(dot(N, L));
  float const g1 = ndl * schlick(ndv, k);
  float const g2 = schlick(ndl, k);
  return g1 * g2;
}

struct matinfo {
  v3 color;
  float ior, roughness, metallic, transmission;
};

// ---- textures (the GL sampling of the reference's textures, level 0) ----------------
// wrap: 0 GL_REPEAT, 1 GL_CLAMP_TO_EDGE, 2 GL_MIRRORED_REPEAT. GL_LINEAR:
// texel coordinates u = s W - 1/2, weights from the fractional parts, summed
// as ((w00 t00 + w10 t10) + w01 t01) + w11 t11.
struct tex2d {
  float4 const* p;
  int w, h, wrap;
};
struct cubemap_dev {
  float4 const* p;  // faces +x, -x, +y, -y, +z, -z, size * size texels each
  int size;
};
__device__ __forceinline__ int wrap_texel(int i, int size, int mode) {
  if (mode == 1) return i < 0 ? 0 : (i >= size ? size - 1 : i);
  if (mode == 2) {
    int m = i % (2 * size);
    if (m < 0) m += 2 * size;
    int const a = m - size;
    return (size - 1) - (a >= 0 ? a : -(1 + a));
  }
  int m = i % size;
  return m < 0 ? m + size : m;
}
__device__ __forceinline__ float4 bilinear_at(float4 const* p, int w, int h, int mode, float s, float t) {
  float const u = s * float(w) - 0.5f, v = t * float(h) - 0.5f;
  float const fu = floorf(u), fv = floorf(v);
  float const a = u - fu, b = v - fv;
  int const i0 = int(fu), j0 = int(fv);
  int const x0 = wrap_texel(i0, w, mode), x1 = wrap_texel(i0 + 1, w, mode);
  int const y0 = wrap_texel(j0, h, mode), y1 = wrap_texel(j0 + 1, h, mode);
  float const w00 = (1.f - a) * (1.f - b), w10 = a * (1.f - b), w01 = (1.f - a) * b, w11 = a * b;
  float4 const t00 = __ldg(p + size_t(y0) * w + x0), t10 = __ldg(p + size_t(y0) * w + x1);
  float4 const t01 = __ldg(p + size_t(y1) * w + x0), t11 = __ldg(p + size_t(y1) * w + x1);
  float4 r;
  r.x = ((w00 * t00.x + w10 * t10.x) + w01 * t01.x) + w11 * t11.x;
  r.y = ((w00 * t00.y + w10 * t10.y) + w01 * t01.y) + w11 * t11.y;
  r.z = ((w00 * t00.z + w10 * t10.z) + w01 * t01.z) + w11 * t11.z;
  r.w = ((w00 * t00.w + w10 * t10.w) + w01 * t01.w) + w11 * t11.w;
  return r;
}
__device__ __forceinline__ float4 tex_sample(tex2d const& t, float s, float tt) {
  return bilinear_at(t.p, t.w, t.h, t.wrap, s, tt);
}
// textureLod(samplerCube, dir, 0): the face of the major axis (GL 4.6 table
// 8.19, ties to x, then y), s = (sc / |ma| + 1) / 2, t = (tc / |ma| + 1) / 2,
// bilinear on that face with clamp to edge.
__device__ __forceinline__ v3 cube_sample(cubemap_dev const& c, v3 d) {
  float const ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
  int face;
  float sc, tc, ma;
  if (ax >= ay && ax >= az) {
    face = d.x >= 0.f ? 0 : 1, ma = ax, sc = d.x >= 0.f ? -d.z : d.z, tc = -d.y;
  } else if (ay >= az) {
    face = d.y >= 0.f ? 2 : 3, ma = ay, sc = d.x, tc = d.y >= 0.f ? d.z : -d.z;
  } else {
    face = d.z >= 0.f ? 4 : 5, ma = az, sc = d.z >= 0.f ? d.x : -d.x, tc = -d.y;
  }
  float const s = (sc / ma + 1.f) / 2.f, t = (tc / ma + 1.f) / 2.f;
  float4 const r = bilinear_at(c.p + size_t(face) * c.size * c.size, c.size, c.size, 1, s, t);
  return {r.x, r.y, r.z};
}
struct pbr_state_t {
  int state;
  bool after_sample;
  float resample;
};
__device__ __forceinline__ void ggx_eval(
    pbr_state_t const& ps, matinfo const& m, float roughness_in, float metallic, v3 tv, v3 tl, v3 n, float i1, float i2,
    v3& refl, float& pdf) {
  float const rough = roughness_in * roughness_in;
  v3 const mn = normalize(tl + tv);
  float const D = (ps.after_sample && rough < 0.01f) ? 1.f : ggx_distribution(n, mn, rough);
  float const G = smith(n, tv, tl, rough);
  float const F = fresnel(dot(tv, mn), i1, i2, metallic);
  float const den = 4.f * fabsf(dot(tv, n)) * fabsf(dot(tl, n));
  float const cos_theta = dot(mn, n);
  v3 const col = mix3(v3{1.f, 1.f, 1.f}, m.color, sqrtf(metallic));
  float mden = G / den;
  mden = isnan(mden) ? 1.f : mden;
  pdf = F * D * cos_theta * mden;
  refl = col * pdf;
}
__device__ __forceinline__ void transmit_eval(
    pbr_state_t const& ps, matinfo const& m, v3 tv, v3 tl, v3 n, float i1, float i2, v3& refl, float& pdf) {
  float const rough = m.roughness * m.roughness;
  v3 mn = normalize(-(i1 * tv + i2 * tl));
  mn = mn * signf(dot(mn, n));
  float const D = (ps.after_sample && rough < 0.01f) ? 1.f : ggx_distribution(n, mn, rough);
  float const G = smith(n, tv, tl, rough);
  float const idoth = dot(tv, mn), odoth = dot(tl, mn);
  float const aidn = fabsf(dot(tv, n)), aodn = fabsf(dot(tl, n));
  float const prefac = (fabsf(idoth) * fabsf(odoth)) / (aidn * aodn);
  float const den = i1 * idoth + i2 * odoth;
  float const F = fresnel(dot(tv, mn), i1, i2, m.metallic);
  float const i2d2 = i2 * i2 / (den * den);
  float const ft = prefac * (1.f - F) * G * D * i2d2;
  float const cos_theta = dot(mn, n);
  pdf = cos_theta * ft;
  refl = m.color * pdf;
}
__device__ __forceinline__ v3 pbr_resample(rng_t& rng, pbr_state_t& ps, v2 rsm, matinfo const& m, v3 tv, v3 n,
    float i1, float i2) {
  float const frand = random_value(rng, int(uint32_t(f2i(19022.f * rsm.x)) * 2909293u));
  float const trand = random_value(rng, int(uint32_t(f2i(23452.f * rsm.y)) * 8994355u));
  v2 is = ggx_importance_sample(rsm, m.roughness * m.roughness);
  v3 hs = sample_hemisphere(is);
  v3 mn = transform_local_to_world(hs, n);
  float const F = fresnel(dot(tv, mn), i1, i2, m.metallic);
  ps.after_sample = true;
  v3 const refracted = refract(-tv, mn, i1 / i2);
  bool const zero = refracted.x == 0.f && refracted.y == 0.f && refracted.z == 0.f;
  if ((m.transmission > 0.f && zero) || F >= frand) {
    ps.state = 0;
    ps.resample = F;
    return nreflect(tv, n, mn);
  } else if (m.transmission >= trand) {
    ps.resample = (1.f - F) * m.transmission;
    ps.state = 1;
    return refracted;
  }
  ps.resample = (1.f - F) * (1.f - m.transmission);
  ps.state = 2;
  is = ggx_importance_sample(rsm, 1.f);
  hs = sample_hemisphere(is);
  mn = transform_local_to_world(hs, n);
  return nreflect(tv, n, mn);
}
__device__ __forceinline__ void pbr_eval(
    pbr_state_t& ps, matinfo const& m, v3 tv, v3 tl, v3 n, float i1, float i2, v3& refl, float& pdf) {
  v3 r;
  float p;
  if (ps.state == 1) {
    transmit_eval(ps, m, tv, tl, n, i1, i2, r, p);
  } else if (ps.state == 2) {
    ggx_eval(ps, m, 1.f, 1.f, tv, tl, n, i1, i2, r, p);
  } else if (ps.state == 0) {
    ggx_eval(ps, m, m.roughness, m.metallic, tv, tl, n, i1, i2, r, p);
  } else {
    r = refl;
    p = pdf;
  }
  ps.after_sample = false;
  pdf = p * ps.resample;
  refl = r * ps.resample;
}

// material_new.glsl for type 0; other type ids behave as the generated
// dispatch does for an unknown id (evaluate -> 0 / pdf 1, bounce -> 0).
struct material_ctx {
  int type;
  matinfo mat;
  pbr_state_t ps;
  uint32_t tex_x, tex_y;  // albedo_texture handle: (slot + 1, 0), (0, 0) = none
};
__device__ __forceinline__ void mat_open(material_ctx& mc, int type, float const* data, int offset) {
  mc.type = type;
  mc.ps = pbr_state_t{-1, false, 1.f};
  if (type != 0) return;
  float const* d = data + offset;
  uint32_t const c = __float_as_uint(__ldg(d));
  mc.mat.color = unpack_rgb(c);
  mc.mat.ior = __ldg(d + 1);
  mc.mat.roughness = __ldg(d + 2);
  mc.mat.metallic = __ldg(d + 3);
  mc.mat.transmission = __ldg(d + 4);
  mc.tex_x = __float_as_uint(__ldg(d + 5));
  mc.tex_y = __float_as_uint(__ldg(d + 6));
}
// material_new.glsl:27-41. With an albedo texture the colour becomes
// pow(texture(albedo, (u, 1 - v)), 2.2) (the context's texture slot tex_x - 1;
// handles outside the table read no texture).
__device__ __forceinline__ void mat_evaluate(material_ctx& mc, v3 n, v3 tl, v3 tv, v3& refl, float& pdf,
    v2 uv = v2{0.f, 0.f}, tex2d const* textures = nullptr, int n_textures = 0) {
  refl = {0.f, 0.f, 0.f};
  pdf = 1.f;
  if (mc.type != 0) return;
  if ((mc.tex_x != 0u || mc.tex_y != 0u) && mc.tex_y == 0u && mc.tex_x <= uint32_t(n_textures) && textures &&
      textures[mc.tex_x - 1u].p) {
    float4 const c = tex_sample(textures[mc.tex_x - 1u], uv.x, 1.f - uv.y);
    mc.mat.color = {myrt_glmath::pow(c.x, 2.2f), myrt_glmath::pow(c.y, 2.2f), myrt_glmath::pow(c.z, 2.2f)};
  }
  bool const incoming = dot(n, -tv) < 0.f;
  float const i1 = incoming ? 1.f : mc.mat.ior;
  float const i2 = incoming ? mc.mat.ior : 1.f;
  v3 r{0.f, 0.f, 0.f};
  float p = 0.f;
  pbr_eval(mc.ps, mc.mat, tv, tl, incoming ? n : -n, i1, i2, r, p);
  refl = r;
  pdf = p;
}
__device__ __forceinline__ v3 mat_bounce(material_ctx& mc, rng_t& rng, v2 rnd, v3 tv, v3 n) {
  if (mc.type != 0) return {0.f, 0.f, 0.f};
  bool const incoming = dot(n, -tv) < 0.f;
  float const i1 = incoming ? 1.f : mc.mat.ior;
  float const i2 = incoming ? mc.mat.ior : 1.f;
  return pbr_resample(rng, mc.ps, rnd, mc.mat, tv, incoming ? n : -n, i1, i2);
}

}  // namespace rs
}  // namespace myrt_b200
