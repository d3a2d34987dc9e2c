// CPU oracle, part 2: the reference's wavefront passes in "reference shading"
// mode, restated from the GLSL and the C++ pass driver.
//
// TEST INFRASTRUCTURE ONLY (checker for the device wavefront). Built into
// liboracle.so with -ffp-contract=off -fwrapv.
//
// Follows, function by function:
//   random.glsl:14-85            rng_* (with the evaluation order GLSL defines:
//                                arguments left to right)
//   ggx.glsl:9-43, pbr.glsl:29-232, transform.glsl:3-15, color.glsl,
//   material_new.glsl:14-49 and the dispatch material_registry::generate_code
//   emits (material.hpp:39-65) for the single PBR type
//   pt_generate.comp:50-84       pass_generate
//   pt_trace.comp:134-226, :311-386 (meshes, then SDF drawables)  pass_trace
//   pt_color.comp:77-202         pass_color (sky gradient, or the cube map)
//   pt_ray_filter.comp:49-64     pass_filter, as a STABLE compaction (slot order
//                                = serial order; the reference's atomicAdd order
//                                is not reproducible)
//   sequential_pathtracer.cpp:10-69, :282-498  frame driver and the host random
//                                stream (std::mt19937 + std distributions, in the
//                                order the passes draw them)
// Scene: world-space triangles with per-corner normals / uvs, one material index
// per triangle. Closest / any hit come from the restated reference BVH
// (oracle.cpp) with canonical ties; see orc_refbvh_* there.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <random>

#include "oracle_glsl_math.hpp"
#include <thread>
#include <vector>

namespace {

struct v2 {
  float x, y;
};
struct v3 {
  float x, y, z;
};
struct v4 {
  float x, y, z, w;
};
inline v3 operator+(v3 a, v3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline v3 operator-(v3 a, v3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline v3 operator-(v3 a) { return {-a.x, -a.y, -a.z}; }
inline v3 operator*(v3 a, v3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline v3 operator*(v3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline v3 operator*(float s, v3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline v3 operator/(v3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline float dot(v3 a, v3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline v3 cross(v3 a, v3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline float length(v3 v) { return std::sqrt(dot(v, v)); }
inline v3 normalize(v3 v) { return v * (1.f / length(v)); }
// GLSL min/max/clamp (NaN goes to the first operand's side as the ternary does)
inline float gmin(float a, float b) { return b < a ? b : a; }
inline float gmax(float a, float b) { return a < b ? b : a; }
inline float gclamp(float v, float lo, float hi) { return gmin(gmax(v, lo), hi); }
inline v3 clamp3(v3 v, float lo, float hi) { return {gclamp(v.x, lo, hi), gclamp(v.y, lo, hi), gclamp(v.z, lo, hi)}; }
inline float mixf(float a, float b, float t) { return a * (1.f - t) + b * t; }
inline v3 mix3(v3 a, v3 b, float t) { return a * (1.f - t) + b * t; }
inline bool nan3(v3 v) { return std::isnan(v.x) || std::isnan(v.y) || std::isnan(v.z); }
inline bool inf3(v3 v) { return std::isinf(v.x) || std::isinf(v.y) || std::isinf(v.z); }
inline bool naninf4(v4 v) {
  return std::isnan(v.x) || std::isnan(v.y) || std::isnan(v.z) || std::isnan(v.w) || std::isinf(v.x) ||
      std::isinf(v.y) || std::isinf(v.z) || std::isinf(v.w);
}
inline float signf(float v) { return v > 0.f ? 1.f : (v < 0.f ? -1.f : 0.f); }
inline v3 faceforward(v3 n, v3 i, v3 nref) { return dot(nref, i) < 0.f ? n : -n; }
inline v3 reflect(v3 i, v3 n) { return i - 2.f * dot(n, i) * n; }
inline v3 refract(v3 i, v3 n, float eta) {
  float const k = 1.f - eta * eta * (1.f - dot(n, i) * dot(n, i));
  if (k < 0.f) return {0.f, 0.f, 0.f};
  return eta * i - (eta * dot(n, i) + std::sqrt(k)) * n;
}

// float -> int with the x86 out-of-range result (INT_MIN), the behaviour the
// reference build on x86 has for int(float) of values >= 2^31.
inline int f2i(float f) {
  if (!(f > -2147483648.0f && f < 2147483648.0f)) return std::numeric_limits<int>::min();
  return int(f);
}
inline std::uint32_t f2u(float f) { return std::uint32_t(f2i(f)); }

inline std::uint32_t pack_unorm4x8(v4 c) {
  float const v[4] = {c.x, c.y, c.z, c.w};
  std::uint32_t r = 0;
  for (int i = 0; i < 4; ++i) r |= std::uint32_t(std::nearbyint(gclamp(v[i], 0.f, 1.f) * 255.f)) << (8 * i);
  return r;
}
inline v4 unpack_unorm4x8(std::uint32_t p) {
  return {float(p & 0xffu) / 255.f, float((p >> 8) & 0xffu) / 255.f, float((p >> 16) & 0xffu) / 255.f,
      float((p >> 24) & 0xffu) / 255.f};
}

// ---- random.glsl -------------------------------------------------------------
struct rng_t {
  std::uint32_t state = 0;
  int prime = 0;
  float const* tex = nullptr;
  int tex_size = 0;
};
constexpr int kPrimes[6] = {69019, 96013, 32159, 22783, 87011, 45263};
inline std::uint32_t wang(std::uint32_t a) {
  a = (a ^ 61u) ^ (a >> 16);
  a = a + (a << 3);
  a = a ^ (a >> 4);
  a = a * 0x27d4eb2du;
  a = a ^ (a >> 15);
  return a;
}
inline std::uint32_t xorshift(rng_t& r) {
  r.state ^= (r.state << 13);
  r.state ^= (r.state >> 17);
  r.state ^= (r.state << 5);
  return r.state;
}
inline float random_value(rng_t& r, int seed) {
  r.state += wang(std::uint32_t(seed));
  return gclamp(float(xorshift(r)) * (1.f / float(0xFFFFFFFFu)), 0.f, 1.f);
}
inline int random_int(rng_t& r, int seed) { return f2i(random_value(r, seed) * float(0x7fffffff)); }
inline float texel(rng_t const& r, int i) { return (i < 0 || i >= r.tex_size) ? 0.f : r.tex[i]; }
inline void random_init(rng_t& r, float const* tex, int tex_size, int px, int py, int seed) {
  r.state = std::uint32_t(seed);
  r.prime = 0;
  r.tex = tex;
  r.tex_size = tex_size;
  int const a = random_int(r, px ^ 0xba77fa);
  int const b = random_int(r, py ^ 0xcca6df);
  int const c = random_int(r, seed);
  int const seed_base = int(std::uint32_t(a) * std::uint32_t(kPrimes[0]) + std::uint32_t(b) * std::uint32_t(kPrimes[1]) +
      std::uint32_t(c));
  random_value(r, int(std::uint32_t(seed_base) + std::uint32_t(f2i(float(0xffaf86) * texel(r, seed_base % tex_size)))));
}
inline float random_next(rng_t& r) {
  r.prime = (r.prime + 1) % 6;
  return random_value(r, r.prime);
}
inline v2 random_uniform_circle(rng_t& r, float radius) {
  float const a = random_next(r) * 2.f * 3.1415926535897f;
  float const b = random_next(r);
  float const s = std::sqrt(b) * radius;
  return {s * orc_glsl::sin(a), s * orc_glsl::cos(a)};
}

// ---- ggx.glsl / pbr.glsl / transform.glsl -------------------------------------
constexpr float kPi = 3.1415926535897f;
inline float ggx_distribution(v3 n, v3 h, float alpha) {
  float const ndotm = dot(n, h);
  float const a2 = alpha * alpha;
  float const den = ndotm * ndotm * (a2 - 1.f) + 1.f;
  return a2 / (kPi * den * den);
}
inline v2 ggx_importance_sample(v2 rs, float roughness) {
  float const phi = rs.y * 2.f * kPi;
  float const rough2 = roughness * roughness;
  float const theta = orc_glsl::atan(std::sqrt(rough2 * rs.x / (1.f - rs.x)));
  return {phi, theta};
}
inline v3 sample_hemisphere(v2 is) {
  float const c = orc_glsl::cos(is.y), s = orc_glsl::sin(is.y);
  return {s * orc_glsl::cos(is.x), s * orc_glsl::sin(is.x), c};
}
inline v3 transform_local_to_world(v3 v, v3 n) {
  v3 perp{1.f, 0.f, 0.f};
  v3 u = normalize(cross(n, perp));
  for (int i = 1; nan3(u) && i < 3; ++i) {
    float* p = &perp.x;
    p[i - 1] = 0.f;
    p[i] = 1.f;
    u = normalize(cross(n, perp));
  }
  v3 const c = cross(n, u);
  v3 const r{(u.x * v.x + c.x * v.y) + n.x * v.z, (u.y * v.x + c.y * v.y) + n.y * v.z, (u.z * v.x + c.z * v.y) + n.z * v.z};
  return normalize(r);
}
inline float fresnel(float cos_theta, float ior_in, float ior_out, float metallic) {
  float f0 = std::fabs((ior_in - ior_out) / (ior_in + ior_out));
  f0 = mixf(f0 * f0, 1.f, metallic);
  return f0 + (1.f - f0) * orc_glsl::pow(1.f - cos_theta, 5.f);
}
inline v3 nreflect(v3 tv, v3 n, v3 mn) {
  v3 ray = reflect(-tv, mn);
  float const d = dot(ray, n);
  if (d < 0.f) ray = ray - 2.f * d * n;
  return normalize(ray);
}
inline float schlick(float ndv, float k) { return 1.f / (ndv * (1.f - k) + k); }
inline float smith(v3 N, v3 V, v3 L, float k) {
  float const ndv = std::fabs(dot(N, V)), ndl = std::fabs(dot(N, L));
  float const g1 = ndl * schlick(ndv, k);
  float const g2 = schlick(ndl, k);
  return g1 * g2;
}
struct matinfo {
  v4 color;
  float ior, roughness, metallic, transmission;
};
struct brdf {
  v3 refl{0, 0, 0};
  float pdf = 0.f;
};
struct pbr_state_t {
  int state = -1;
  bool after_sample = false;
  float resample = 1.f;
};
inline void ggx_eval(pbr_state_t const& ps, matinfo m, v3 tv, v3 tl, v3 n, float i1, float i2, brdf& r) {
  float const rough = m.roughness * m.roughness;
  v3 const mn = normalize(tl + tv);
  float const D = (ps.after_sample && rough < 0.01f) ? 1.f : ggx_distribution(n, mn, rough);
  float const G = smith(n, tv, tl, rough);
  float const F = fresnel(dot(tv, mn), i1, i2, m.metallic);
  float const den = 4.f * std::fabs(dot(tv, n)) * std::fabs(dot(tl, n));
  float const cos_theta = dot(mn, n);
  v3 const col = mix3(v3{1.f, 1.f, 1.f}, v3{m.color.x, m.color.y, m.color.z}, std::sqrt(m.metallic));
  float mden = G / den;
  mden = std::isnan(mden) ? 1.f : mden;
  r.pdf = F * D * cos_theta * mden;
  r.refl = col * r.pdf;
}
inline void transmit_eval(pbr_state_t const& ps, matinfo m, v3 tv, v3 tl, v3 n, float i1, float i2, brdf& r) {
  float const rough = m.roughness * m.roughness;
  v3 mn = normalize(-(i1 * tv + i2 * tl));
  mn = mn * signf(dot(mn, n));
  float const D = (ps.after_sample && rough < 0.01f) ? 1.f : ggx_distribution(n, mn, rough);
  float const G = smith(n, tv, tl, rough);
  float const idoth = dot(tv, mn), odoth = dot(tl, mn);
  float const aidn = std::fabs(dot(tv, n)), aodn = std::fabs(dot(tl, n));
  float const prefac = (std::fabs(idoth) * std::fabs(odoth)) / (aidn * aodn);
  float const den = i1 * idoth + i2 * odoth;
  float const F = fresnel(dot(tv, mn), i1, i2, m.metallic);
  float const i2d2 = i2 * i2 / (den * den);
  float const ft = prefac * (1.f - F) * G * D * i2d2;
  float const cos_theta = dot(mn, n);
  r.pdf = cos_theta * ft;
  r.refl = v3{m.color.x, m.color.y, m.color.z} * r.pdf;
}
inline v3 pbr_resample(rng_t& rng, pbr_state_t& ps, v2 rs, matinfo m, v3 tv, v3 n, float i1, float i2) {
  float const frand = random_value(rng, int(std::uint32_t(f2i(19022.f * rs.x)) * 2909293u));
  float const trand = random_value(rng, int(std::uint32_t(f2i(23452.f * rs.y)) * 8994355u));
  v2 is = ggx_importance_sample(rs, m.roughness * m.roughness);
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
  is = ggx_importance_sample(rs, 1.f);
  hs = sample_hemisphere(is);
  mn = transform_local_to_world(hs, n);
  return nreflect(tv, n, mn);
}
inline void pbr_eval(pbr_state_t& ps, matinfo m, v3 tv, v3 tl, v3 n, float i1, float i2, brdf& r) {
  brdf tr, gl, di;
  transmit_eval(ps, m, tv, tl, n, i1, i2, tr);
  ggx_eval(ps, m, tv, tl, n, i1, i2, gl);
  matinfo md = m;
  md.roughness = 1.f;
  md.metallic = 1.f;
  ggx_eval(ps, md, tv, tl, n, i1, i2, di);
  switch (ps.state) {
    case 1: r = tr; break;
    case 2: r = di; break;
    case 0: r = gl; break;
    default: break;
  }
  ps.after_sample = false;
  r.pdf *= ps.resample;
  r.refl = r.refl * ps.resample;
}

// Textures of the reference mode, sampled as GL samples them at level 0
// (GL_LINEAR, wrap 0 repeat / 1 clamp to edge / 2 mirrored repeat; weights
// summed ((w00 t00 + w10 t10) + w01 t01) + w11 t11), and the cube map
// (GL 4.6 table 8.19 face selection, ties to x then y, clamp to edge).
struct tex_view {
  float const* p = nullptr;  // rgba
  int w = 0, h = 0, wrap = 0;
};
inline int wrap_texel(int i, int size, int mode) {
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
inline v4 bilinear_at(float const* p, int w, int h, int mode, float s, float t) {
  float const u = s * float(w) - 0.5f, v = t * float(h) - 0.5f;
  float const fu = std::floor(u), fv = std::floor(v);
  float const a = u - fu, b = v - fv;
  int const i0 = int(fu), j0 = int(fv);
  int const x0 = wrap_texel(i0, w, mode), x1 = wrap_texel(i0 + 1, w, mode);
  int const y0 = wrap_texel(j0, h, mode), y1 = wrap_texel(j0 + 1, h, mode);
  float const w00 = (1.f - a) * (1.f - b), w10 = a * (1.f - b), w01 = (1.f - a) * b, w11 = a * b;
  float const* t00 = p + 4 * (std::size_t(y0) * w + x0);
  float const* t10 = p + 4 * (std::size_t(y0) * w + x1);
  float const* t01 = p + 4 * (std::size_t(y1) * w + x0);
  float const* t11 = p + 4 * (std::size_t(y1) * w + x1);
  float r[4];
  for (int c = 0; c < 4; ++c) r[c] = ((w00 * t00[c] + w10 * t10[c]) + w01 * t01[c]) + w11 * t11[c];
  return {r[0], r[1], r[2], r[3]};
}
inline v3 cube_sample(float const* faces, int size, v3 d) {
  float const ax = std::fabs(d.x), ay = std::fabs(d.y), az = std::fabs(d.z);
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
  v4 const r = bilinear_at(faces + std::size_t(face) * size * size * 4, size, size, 1, s, t);
  return {r.x, r.y, r.z};
}

// material_new.glsl + generated dispatch (type 0 = PBR, 7 floats)
struct material_ctx {
  int type = -1;
  matinfo mat{};
  bool incoming = false;
  float ior1 = 1.f, ior2 = 1.f;
  pbr_state_t ps;
  std::uint32_t tex_x = 0, tex_y = 0;  // albedo_texture handle (slot + 1, 0)
};
inline std::uint32_t fbits(float f) {
  std::uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}
inline void mat_open(material_ctx& mc, int type, float const* data, int offset) {
  mc.type = type;
  if (type != 0) return;
  float const* d = data + offset;
  mc.mat.color = unpack_unorm4x8(fbits(d[0]));
  mc.mat.ior = d[1];
  mc.mat.roughness = d[2];
  mc.mat.metallic = d[3];
  mc.mat.transmission = d[4];
  mc.tex_x = fbits(d[5]);
  mc.tex_y = fbits(d[6]);
}
// material_new.glsl:27-41: pow(texture(albedo, (u, 1 - v)), 2.2) replaces the colour
inline void mat_evaluate(material_ctx& mc, v3 n, v3 tl, v3 tv, v3& refl, float& pdf, v2 uv = v2{0.f, 0.f},
    tex_view const* textures = nullptr, int n_textures = 0) {
  refl = {0.f, 0.f, 0.f};
  pdf = 1.f;
  if (mc.type != 0) return;
  if ((mc.tex_x != 0u || mc.tex_y != 0u) && mc.tex_y == 0u && mc.tex_x <= std::uint32_t(n_textures) && textures &&
      textures[mc.tex_x - 1u].p) {
    tex_view const& t = textures[mc.tex_x - 1u];
    v4 const c = bilinear_at(t.p, t.w, t.h, t.wrap, uv.x, 1.f - uv.y);
    mc.mat.color = {orc_glsl::pow(c.x, 2.2f), orc_glsl::pow(c.y, 2.2f), orc_glsl::pow(c.z, 2.2f),
        orc_glsl::pow(c.w, 2.2f)};
  }
  mc.incoming = dot(n, -tv) < 0.f;
  mc.ior1 = mc.incoming ? 1.f : mc.mat.ior;
  mc.ior2 = mc.incoming ? mc.mat.ior : 1.f;
  brdf ev;
  pbr_eval(mc.ps, mc.mat, tv, tl, mc.incoming ? n : -n, mc.ior1, mc.ior2, ev);
  refl = ev.refl;
  pdf = ev.pdf;
}
inline v3 mat_bounce(material_ctx& mc, rng_t& rng, v2 rnd, v3 tv, v3 n) {
  if (mc.type != 0) return {0.f, 0.f, 0.f};
  mc.incoming = dot(n, -tv) < 0.f;
  mc.ior1 = mc.incoming ? 1.f : mc.mat.ior;
  mc.ior2 = mc.incoming ? mc.mat.ior : 1.f;
  return pbr_resample(rng, mc.ps, rnd, mc.mat, tv, mc.incoming ? n : -n, mc.ior1, mc.ior2);
}

// ---- SDF drawables (raymarch.glsl, sdf.hpp:399-633, sdf.cpp:122-407) -------------
// Flat post-order programs: modifier instructions move the position of the next
// primitive (innermost first); primitives push (distance, material); operators
// pop two and push one. Opcodes as include/myrt_cuda.h.
struct sdf_scene {
  std::int32_t const* instrs = nullptr;    // (op, param offset) pairs
  std::int32_t const* programs = nullptr;  // (first, count) pairs
  float const* params = nullptr;
  float const* drawables = nullptr;        // 36 floats: mat4, inverse mat4, sdf_index bits, pad
  int n_drawables = 0;
  int steps = 0;
  float eps = 0.f;
};
inline v3 abs3(v3 a) { return {std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }
inline v3 max3s(v3 a, float s) { return {gmax(a.x, s), gmax(a.y, s), gmax(a.z, s)}; }
inline float len2(float x, float y) { return std::sqrt(x * x + y * y); }
struct sdf_ctx {
  sdf_scene const* s;
  rng_t* rng;
  bool load = false;  // g_do_load_materials
  int prog = 0;       // sdf_index_current
};
inline int sdf_ldm(sdf_ctx const& c, int index) { return c.load ? index : -1; }
inline int sdf_mxm(sdf_ctx& c, int a, int b, float t) {
  if (!c.load) return -1;
  return random_next(*c.rng) < t ? b : a;
}
// sdf.hpp: menger_fractal
inline float sd_menger(v3 p) {
  for (int n = 0; n < 4; n++) {
    p = abs3(p);
    if (p.x < p.y) std::swap(p.x, p.y);
    if (p.x < p.z) std::swap(p.x, p.z);
    if (p.y < p.z) std::swap(p.y, p.z);
    p.z -= 1.f / 3.f;
    p.z = -std::fabs(p.z);
    p.z += 1.f / 3.f;
    p = p * 3.f;
    p.x -= 2.f;
    p.y -= 2.f;
  }
  v3 const d = abs3(p) - v3{1.f, 1.f, 1.f};
  float dis = gmin(gmax(d.x, gmax(d.y, d.z)), 0.f) + length(max3s(d, 0.f));
  dis *= std::pow(3.f, float(-4));
  return dis;
}
inline float sdf_map(sdf_ctx& c, v3 p, int& mat) {
  sdf_scene const& s = *c.s;
  auto G = [&](int i) { return s.params[i]; };
  std::int32_t const first = s.programs[2 * c.prog], count = s.programs[2 * c.prog + 1];
  float dist[64];
  int mats[64];
  int sp = 0;
  v3 pos = p;
  float mul = 1.f;
  for (int k = 0; k < count; ++k) {
    int const op = s.instrs[2 * (first + k)], o = s.instrs[2 * (first + k) + 1];
    int m = mat;
    float d = 0.f;
    switch (op) {
      case 32: pos = pos - v3{G(o), G(o + 1), G(o + 2)}; continue;
      case 33: {
        int const ax = int(G(o));
        float* q = &pos.x;
        q[ax] = std::fabs(q[ax]);
        continue;
      }
      case 1: m = sdf_ldm(c, int(G(o + 1))); d = length(pos) - G(o); break;
      case 2: {
        m = sdf_ldm(c, int(G(o + 3)));
        v3 const q = abs3(pos) - v3{G(o), G(o + 1), G(o + 2)};
        d = length(max3s(q, 0.f)) + gmin(gmax(q.x, gmax(q.y, q.z)), 0.f);
        break;
      }
      case 3: m = sdf_ldm(c, int(G(o + 2))); d = len2(len2(pos.x, pos.z) - G(o), pos.y) - G(o + 1); break;
      case 4: {
        m = sdf_ldm(c, int(G(o + 2)));
        v3 q = pos;
        q.y -= gclamp(q.y, 0.f, G(o));
        d = length(q) - G(o + 1);
        break;
      }
      case 5: m = sdf_ldm(c, int(G(o))); d = sd_menger(pos); break;
      default: {
        float const d1 = dist[sp - 1], d0 = dist[sp - 2];
        int const m1 = mats[sp - 1], m0 = mats[sp - 2];
        sp -= 2;
        if (op == 16 || op == 17 || op == 18) {
          float const r = op == 16 ? gmin(d0, d1) : (op == 17 ? gmax(-d0, d1) : gmax(d0, d1));
          m = sdf_mxm(c, m0, m1, float(r == d1));
          d = r;
        } else {  // 19: smooth union
          float const k = G(o);
          float const h = gclamp(0.5f + 0.5f * (d1 - d0) / k, 0.f, 1.f);
          m = sdf_mxm(c, m0, m1, 1.f - h);
          d = mixf(d1, d0, h) - k * h * (1.f - h);
        }
        break;
      }
    }
    dist[sp] = d;
    mats[sp] = m;
    ++sp;
    pos = p;
  }
  mat = mats[sp - 1];
  return mul * dist[sp - 1];
}
inline v4 mat4_vec(float const* m, v4 v) {
  float const in[4] = {v.x, v.y, v.z, v.w};
  float o[4];
  for (int r = 0; r < 4; ++r)
    o[r] = ((m[0 * 4 + r] * in[0] + m[1 * 4 + r] * in[1]) + m[2 * 4 + r] * in[2]) + m[3 * 4 + r] * in[3];
  return {o[0], o[1], o[2], o[3]};
}
struct sdf_hit {
  bool hits = false;
  float t = 0.f;
  v3 position{0, 0, 0}, normal{0, 0, 0};
  v2 uv{0, 0};
  int material = -1;
};
// raymarch.glsl:116-171 for drawable `cur`
inline sdf_hit march_sdf(sdf_scene const& s, rng_t& rng, int cur, v3 oro, v3 ord, float tmax, bool hits_only) {
  sdf_ctx c{&s, &rng, false, 0};
  float const* dr = s.drawables + 36 * cur;
  float const* inv = dr + 16;
  std::int32_t idx;
  std::memcpy(&idx, dr + 32, 4);
  c.prog = idx;
  v4 const ro4 = mat4_vec(inv, v4{oro.x, oro.y, oro.z, 1.f});
  v4 const rd4 = mat4_vec(inv, v4{ord.x, ord.y, ord.z, 0.f});
  v3 const ro{ro4.x, ro4.y, ro4.z}, rd{rd4.x, rd4.y, rd4.z};
  float const len = length(rd);
  float res = -1.f;
  float t = 10.f * s.eps;
  int si = 0;
  for (int i = 0; i < s.steps && t / len < tmax; i++) {
    int mdum = -1;
    float const m = sdf_map(c, ro + rd * t / len, mdum);
    if (si == 0) si = int(signf(m));
    float const h = m;
    if (std::fabs(h) < s.eps) {
      res = t;
      break;
    }
    t += float(si) * h;
  }
  sdf_hit hit;
  if (res < 0.f) return hit;
  hit.hits = true;
  if (hits_only) return hit;
  hit.t = res / len;
  hit.position = oro + res / len * ord;
  v3 const poas = ro + res * rd;
  // nor(): tetrahedral normal, then the material with draws enabled
  v3 n{0.f, 0.f, 0.f};
  for (int i = 0; i < 4; i++) {
    v3 const e = 0.5773f * (2.f * v3{float(((i + 3) >> 1) & 1), float((i >> 1) & 1), float(i & 1)} - v3{1.f, 1.f, 1.f});
    int mdum = -1;
    n = n + e * sdf_map(c, poas + 0.0005f * e / len, mdum) * len;
  }
  v3 const gn = normalize(n);
  c.load = true;
  int mat = -1;
  sdf_map(c, poas, mat);
  // normalize((transpose(inverse) * vec4(nor, 0)).xyz): row r of the transpose = column r of inverse
  float const* m = inv;
  v3 const tn{((m[0] * gn.x + m[1] * gn.y) + m[2] * gn.z) + m[3] * 0.f,
      ((m[4] * gn.x + m[5] * gn.y) + m[6] * gn.z) + m[7] * 0.f,
      ((m[8] * gn.x + m[9] * gn.y) + m[10] * gn.z) + m[11] * 0.f};
  hit.normal = normalize(tn);
  // sample_texture(poas, normal, 0.5): triplanar weights pow(abs(n), k)
  float const wx = std::pow(std::fabs(hit.normal.x), 0.5f), wy = std::pow(std::fabs(hit.normal.y), 0.5f),
              wz = std::pow(std::fabs(hit.normal.z), 0.5f);
  float const sw = (wx + wy) + wz;
  hit.uv = {((poas.y * wx + poas.z * wy) + poas.x * wz) / sw, ((poas.z * wx + poas.x * wy) + poas.y * wz) / sw};
  hit.material = mat;
  return hit;
}

// ---- pass state (pt_*.comp structs) -------------------------------------------
struct gen_t {  // generate_output_t, 80 bytes
  v3 origin;
  float random_value;
  v3 direction;
  float pixel_x;
  v3 reflectance;
  float pixel_y;
  v4 color;
  float pdf, weight, pad[2];
};
struct trace_t {  // trace_output_t, 64 bytes
  v3 point;
  int intersects;
  v3 normal;
  std::uint32_t generated_ray;
  v2 uv;
  int material_index;
  std::uint32_t light_color;
  v3 light_direction;
  float light_strength;
};
static_assert(sizeof(gen_t) == 80 && sizeof(trace_t) == 64);

struct light_t {
  v3 position;
  float radius;
  v3 color;
};
// pt_trace.comp:141-146, products rounded in float as the GLSL computes them
// (6 * 1.8f is 10.79999924, not the float nearest 10.8)
constexpr light_t kLights[2] = {
    {{2.f * 4.f, 2.f * 5.f, 2.f * 4.f}, 1.5f, {6.f * 1.f, 6.f * 1.8f, 6.f * 3.f}},
    {{2.f * -4.f, 2.f * 3.f, 2.f * 5.f}, 1.5f, {8.f * 3.f, 8.f * 1.8f, 8.f * 1.f}},
};

// intersect.glsl:30-39
inline float intersect_sphere(v3 r0, v3 rd, v3 s0, float sr) {
  float const a = dot(rd, rd);
  v3 const s0_r0 = r0 - s0;
  float const b = 2.f * dot(rd, s0_r0);
  float const c = dot(s0_r0, s0_r0) - (sr * sr);
  if (b * b - 4.f * a * c < 0.f) return -1.f;
  return (-b - std::sqrt((b * b) - 4.f * a * c)) / (2.f * a);
}

}  // namespace

// ray queries provided by oracle.cpp
extern "C" void orc_refbvh_traverse(void const* nodes_v, std::uint32_t const* bvh_idx, std::uint32_t const* indices,
    float const* points_xyzw, float const* rays, std::size_t n, int any_hit, int canonical, std::int32_t* prim,
    float* t_out, float* u_out, float* v_out, int nthreads);

namespace {

struct scene_t {
  std::size_t n_tris;
  float const* tris9;       // world positions
  float const* normals9;    // world shading normals per corner (may be null)
  float const* uvs6;        // uvs per corner (may be null)
  std::int32_t const* tri_material;
  std::int32_t const* mat_refs;  // (id, offset) pairs
  std::size_t n_mats;
  float const* mat_data;
  void const* nodes;  // restated reference BVH over the world triangles
  std::uint32_t const* bvh_idx;
  std::vector<std::uint32_t> seq;  // 0..3T-1 (index buffer of the baked soup)
  std::vector<float> pts4;         // points as xyzw
};

template <typename F> void par(std::size_t n, int nthreads, F&& f) {
  if (nthreads <= 1 || n < 2048) {
    f(std::size_t(0), n);
    return;
  }
  std::vector<std::thread> th;
  std::size_t const per = (n + std::size_t(nthreads) - 1) / std::size_t(nthreads);
  for (int i = 0; i < nthreads; ++i) {
    std::size_t const b = std::size_t(i) * per, e = std::min(n, b + per);
    if (b < e) th.emplace_back([&f, b, e] { f(b, e); });
  }
  for (auto& x : th) x.join();
}

struct pass_rng {
  int seed;
  std::vector<float> tex;
};

// mat4 (column major) helpers, GLSL operator order
inline void mat_mul(float const* a, float const* b, float* out) {
  for (int c = 0; c < 4; ++c)
    for (int r = 0; r < 4; ++r)
      out[c * 4 + r] = ((a[0 * 4 + r] * b[c * 4 + 0] + a[1 * 4 + r] * b[c * 4 + 1]) + a[2 * 4 + r] * b[c * 4 + 2]) +
          a[3 * 4 + r] * b[c * 4 + 3];
}
inline v4 mat_vec(float const* m, v4 v) {
  float const in[4] = {v.x, v.y, v.z, v.w};
  float o[4];
  for (int r = 0; r < 4; ++r)
    o[r] = ((m[0 * 4 + r] * in[0] + m[1 * 4 + r] * in[1]) + m[2 * 4 + r] * in[2]) + m[3 * 4 + r] * in[3];
  return {o[0], o[1], o[2], o[3]};
}

struct frame_ctx {
  scene_t* sc;
  int W, H;
  float const* inv_view;
  float const* inv_proj;
  std::vector<v4>* accum;   // debug_image (sum, count)
  std::vector<v4>* display; // output_image
  std::uint32_t sample_index;
  int nthreads;
  sdf_scene const* sdf;     // n_drawables == 0: no SDF drawables
  // reference-mode extras: albedo textures by slot, cube map, depth of field
  tex_view const* textures = nullptr;
  int n_textures = 0;
  float const* cubemap = nullptr;
  int cubemap_size = 0;
  int dof = 0;
  float lens[2] = {0.f, 0.f};
  float focus = 0.f;
  tex_view bokeh{};
};

// pt_generate.comp:50-84
void pass_generate(frame_ctx& f, pass_rng const& pr, std::vector<gen_t>& gen) {
  float vp[16];
  mat_mul(f.inv_view, f.inv_proj, vp);
  gen.resize(std::size_t(f.W) * f.H);
  par(gen.size(), f.nthreads, [&](std::size_t b, std::size_t e) {
    for (std::size_t id = b; id < e; ++id) {
      int const x = int(id % std::size_t(f.W)), y = int(id / std::size_t(f.W));
      rng_t r;
      random_init(r, pr.tex.data(), int(pr.tex.size()), x, y, pr.seed);
      v2 const off = random_uniform_circle(r, 0.7071067812f);
      float const nx = ((off.x + float(x)) / float(f.W)) * 2.f - 1.f;
      float const ny = ((off.y + float(y)) / float(f.H)) * 2.f - 1.f;
      v4 const hom = mat_vec(vp, v4{nx, ny, 1.f, 1.f});
      gen_t g{};
      g.direction = normalize(v3{hom.x, hom.y, hom.z});
      g.origin = v3{f.inv_view[12], f.inv_view[13], f.inv_view[14]};
      v3 tint{1.f, 1.f, 1.f};
      if (f.dof) {
        // bokeh.glsl:15-34 (bokeh_get) and pt_generate.comp:35-48 (apply_bokeh)
        v2 offset = random_uniform_circle(r, 0.49f);
        v3 value{1.f, 1.f, 1.f};
        float amount = 1.f;
        if (f.bokeh.p && f.bokeh.w >= 10) {
          int tries = 8;
          while ((tries == 8 || amount < 1e-5f) && tries-- > 0) {
            v4 const m = bilinear_at(f.bokeh.p, f.bokeh.w, f.bokeh.h, f.bokeh.wrap, 0.5f + offset.x, 0.5f + offset.y);
            value = {m.x, m.y, m.z};
            offset = random_uniform_circle(r, 0.49f);
            amount = gmax(gmax(value.x, value.y), value.z);
          }
        }
        if (!(amount < 1e-5f)) {
          v3 const center = g.origin + f.focus * g.direction;
          v3 const alt = transform_local_to_world(
              normalize(v3{(offset.x * f.lens[0]) / 2.f, (offset.y * f.lens[1]) / 2.f, f.focus}), g.direction);
          tint = value;
          g.origin = center - f.focus * alt;
          g.direction = alt;
        }
      }
      g.random_value = random_next(r);
      g.reflectance = tint;
      g.color = {0.f, 0.f, 0.f, 0.f};
      g.pixel_x = float(x);
      g.pixel_y = float(y);
      g.pdf = 1.f;
      g.weight = 1.f;
      gen[id] = g;
    }
  });
}

// pt_trace.comp:134-226 for meshes
void pass_trace(frame_ctx& f, pass_rng const& pr, std::vector<gen_t> const& gen, std::vector<trace_t>& out) {
  scene_t& sc = *f.sc;
  std::size_t const n = gen.size();
  out.assign(n, trace_t{});
  // closest hits of all rays first (the order of queries does not matter)
  std::vector<float> rays(8 * n);
  for (std::size_t i = 0; i < n; ++i) {
    float* q = &rays[8 * i];
    q[0] = gen[i].origin.x, q[1] = gen[i].origin.y, q[2] = gen[i].origin.z, q[3] = 0.f;
    q[4] = gen[i].direction.x, q[5] = gen[i].direction.y, q[6] = gen[i].direction.z;
    q[7] = std::numeric_limits<float>::infinity();
  }
  std::vector<std::int32_t> prim(n);
  std::vector<float> tt(n), uu(n), vv(n);
  orc_refbvh_traverse(sc.nodes, sc.bvh_idx, sc.seq.data(), sc.pts4.data(), rays.data(), n, 0, 1, prim.data(), tt.data(),
      uu.data(), vv.data(), f.nthreads);
  // per ray: lights, attributes, shadow ray parameters
  std::vector<float> shadow(8 * n, 0.f);
  std::vector<std::uint8_t> wants_shadow(n, 0);
  std::vector<int> light_index(n);
  std::vector<v3> pol(n);
  par(n, f.nthreads, [&](std::size_t b, std::size_t e) {
    for (std::size_t id = b; id < e; ++id) {
      gen_t const& base = gen[id];
      rng_t r;
      random_init(r, pr.tex.data(), int(pr.tex.size()), f2i(base.pixel_x), f2i(base.pixel_y), pr.seed);
      trace_t res{};
      res.uv = {0.f, 0.f};
      res.material_index = 0;
      res.generated_ray = std::uint32_t(id);
      int const li = std::clamp(f2i(2.f * random_next(r)), 0, 1);
      float const rx = random_next(r), ry = random_next(r), rz = random_next(r);
      float const rs = random_next(r);
      v3 const p_on_light = kLights[li].position + normalize(v3{rx, ry, rz}) * kLights[li].radius * std::sqrt(rs);
      bool hits = prim[id] >= 0;
      float ht = tt[id];
      int hits_light = -1;
      // nearest_hit attributes (pt_trace.comp:357-385) of the closest triangle
      // (triangle 0 when nothing was hit, as the reference reads index 0)
      std::size_t const tri = hits ? std::size_t(prim[id]) : 0;
      float const bx = hits ? uu[id] : 0.f, by = hits ? vv[id] : 0.f;
      float const* P = sc.tris9 + 9 * tri;
      v3 const p0{P[0], P[1], P[2]}, p1{P[3], P[4], P[5]}, p2{P[6], P[7], P[8]};
      float const w = (1.f - bx) - by;
      v3 position = (bx * p1 + by * p2) + w * p0;
      v3 normal;
      if (sc.normals9) {
        float const* N = sc.normals9 + 9 * tri;
        v3 const n0{N[0], N[1], N[2]}, n1{N[3], N[4], N[5]}, n2{N[6], N[7], N[8]};
        normal = normalize((bx * n1 + by * n2) + w * n0);
      } else {
        normal = normalize(cross(normalize(p1 - p0), normalize(p2 - p0)));
      }
      v2 uv{0.f, 0.f};
      if (sc.uvs6) {
        float const* U = sc.uvs6 + 6 * tri;
        uv = {(bx * U[2] + by * U[4]) + w * U[0], (bx * U[3] + by * U[5]) + w * U[1]};
      }
      int material = sc.tri_material[tri];
      // SDF drawables after the meshes (pt_trace.comp:342-352)
      for (int d = 0; f.sdf && d < f.sdf->n_drawables; ++d) {
        sdf_hit const sh = march_sdf(*f.sdf, r, d, base.origin, base.direction,
            hits ? ht : std::numeric_limits<float>::infinity(), false);
        if (sh.hits && sh.t < ht) {
          hits = true;
          ht = sh.t;
          position = sh.position;
          normal = sh.normal;
          uv = sh.uv;
          material = sh.material;
        }
      }
      for (int l = 0; l < 2; ++l) {
        float const t_light = intersect_sphere(base.origin, base.direction, kLights[l].position, kLights[l].radius);
        if (t_light > 0.f && (!hits || t_light < ht)) {
          hits = true;
          ht = t_light;
          hits_light = l;
        }
      }
      res.light_direction = {0.f, 0.f, 0.f};
      res.light_color = 0;
      res.light_strength = 0.f;
      if (hits) {
        res.intersects = 1;
        res.point = position;
        res.normal = normal;
        res.uv = uv;
        res.material_index = material;
        if (inf3(res.normal) || nan3(res.normal)) res.intersects = 0;
        v3 const path = p_on_light - position;
        v3 const dir_l = normalize(path);
        float const dist_l = length(path);
        v3 const lnorm = faceforward(normal, base.direction, normal);
        if (hits_light >= 0) {
          res.intersects = 2;
          v3 const col = kLights[hits_light].color;
          res.light_strength = length(col);
          res.light_color = pack_unorm4x8(v4{col.x / res.light_strength, col.y / res.light_strength,
              col.z / res.light_strength, 0.f / res.light_strength});
          res.light_direction = dir_l;
        } else if (dot(dir_l, lnorm) > 0.f) {
          v3 const so = position + lnorm * 0.01f;
          float* q = &shadow[8 * id];
          q[0] = so.x, q[1] = so.y, q[2] = so.z, q[3] = 0.f, q[4] = dir_l.x, q[5] = dir_l.y, q[6] = dir_l.z;
          q[7] = dist_l;
          wants_shadow[id] = 1;
          light_index[id] = li;
        }
        res.generated_ray = std::uint32_t(id);
      } else {
        res.intersects = 0;
        res.point = {0.f, 0.f, 0.f};
        res.normal = {0.f, 0.f, 0.f};
      }
      out[id] = res;
    }
  });
  // shadow rays (any_hit, pt_trace.comp:311-329), then the NEE record
  std::vector<std::int32_t> sp(n);
  std::vector<float> st(n), su(n), sv(n);
  orc_refbvh_traverse(sc.nodes, sc.bvh_idx, sc.seq.data(), sc.pts4.data(), shadow.data(), n, 1, 0, sp.data(), st.data(),
      su.data(), sv.data(), f.nthreads);
  for (std::size_t id = 0; id < n; ++id) {
    if (!wants_shadow[id] || sp[id] >= 0) continue;
    // any_hit's SDF loop (pt_trace.comp:319-327); hits-only marches draw no randoms
    bool sdf_occluded = false;
    if (f.sdf) {
      float const* q = &shadow[8 * id];
      rng_t unused;
      for (int d = 0; !sdf_occluded && d < f.sdf->n_drawables; ++d)
        sdf_occluded = march_sdf(*f.sdf, unused, d, {q[0], q[1], q[2]}, {q[4], q[5], q[6]}, q[7], true).hits;
    }
    if (sdf_occluded) continue;
    trace_t& res = out[id];
    v3 const col = kLights[light_index[id]].color;
    float const strength = length(col);
    res.light_color = pack_unorm4x8(v4{col.x / strength, col.y / strength, col.z / strength, 0.f / strength});
    float const dist_l = shadow[8 * id + 7];
    res.light_strength = strength * (2.f / dist_l);
    res.light_direction = {shadow[8 * id + 4], shadow[8 * id + 5], shadow[8 * id + 6]};
  }
}

// pt_color.comp:77-101
void accumulate(frame_ctx& f, v4 nc, int px, int py) {
  std::size_t const pi = std::size_t(py) * std::size_t(f.W) + std::size_t(px);
  v4& dbg = (*f.accum)[pi];
  v4 last = dbg;
  if (naninf4(nc)) nc = last;
  v4 const actual_last = last;
  if (f.sample_index == 0) last = {nc.x, nc.y, nc.z, 1.f};
  else last = {last.x + nc.x, last.y + nc.y, last.z + nc.z, last.w + 1.f};
  if (naninf4(last)) last = actual_last;
  dbg = last;
  (*f.display)[pi] = {gclamp(last.x / last.w, 0.f, 4.f), gclamp(last.y / last.w, 0.f, 4.f),
      gclamp(last.z / last.w, 0.f, 4.f), 1.f};
}

// pt_color.comp:113-202
void pass_color(frame_ctx& f, pass_rng const& pr, std::vector<gen_t>& gen, std::vector<trace_t>& tr, bool force) {
  scene_t& sc = *f.sc;
  par(gen.size(), f.nthreads, [&](std::size_t b, std::size_t e) {
    for (std::size_t id = b; id < e; ++id) {
      trace_t const trace = tr[id];
      gen_t g = gen[id];
      int const px = f2i(g.pixel_x), py = f2i(g.pixel_y);
      auto acc = [&](v4 c) { accumulate(f, c, px, py); };
      if (trace.intersects != 0) {
        if (trace.intersects == 2) {
          tr[id].intersects = 0;
          v4 const lc = unpack_unorm4x8(trace.light_color);
          v3 const c = v3{lc.x, lc.y, lc.z} * trace.light_strength * g.reflectance / g.pdf;
          acc(v4{c.x + g.color.x, c.y + g.color.y, c.z + g.color.z, 1.f + g.color.w});
          continue;
        }
        rng_t r;
        random_init(r, pr.tex.data(), int(pr.tex.size()), px, py, pr.seed);
        std::uint32_t const uid = std::uint32_t(id);
        random_value(r, int(std::uint32_t(f2i(56128966.f * g.random_value)) + 20945293u * uid));
        random_value(r, int(std::uint32_t(f2i(12233432.f * g.random_value)) + 74867839u * uid));
        material_ctx mc;
        int const mi = trace.material_index;
        bool const valid_mat = mi >= 0 && std::size_t(mi) < sc.n_mats;
        mat_open(mc, valid_mat ? sc.mat_refs[2 * mi] : -1, sc.mat_data, valid_mat ? sc.mat_refs[2 * mi + 1] : 0);
        float const r0 = random_next(r);
        float const r1 = random_next(r);
        v3 const generated = mat_bounce(mc, r, v2{r0, r1}, -g.direction, trace.normal);
        v3 mrefl;
        float mpdf;
        mat_evaluate(mc, trace.normal, generated, -g.direction, mrefl, mpdf, trace.uv, f.textures, f.n_textures);
        {
          float const p = g.pdf * 1.f;
          float const rnd = random_next(r);
          if (rnd > p) {
            tr[id].intersects = 0;
            v3 const c = g.reflectance / g.pdf;
            acc(v4{g.color.x + c.x, g.color.y + c.y, g.color.z + c.z, g.color.w});
            continue;
          }
        }
        if (force || g.pdf < 1e-5f || mpdf < 1e-6f || std::isnan(mpdf) || std::isinf(mpdf) || nan3(mrefl) ||
            inf3(mrefl) || nan3(generated) || inf3(generated)) {
          tr[id].intersects = 0;
          if (nan3(mrefl) || inf3(mrefl) || std::isnan(g.pdf) || std::isinf(g.pdf) || g.pdf < 1e-5f) {
            acc(g.color);
          } else {
            v3 const c = g.reflectance / g.pdf;
            acc(v4{g.color.x + c.x, g.color.y + c.y, g.color.z + c.z, g.color.w});
          }
          continue;
        }
        if (trace.light_strength > 0.f) {
          v3 lrefl{1.f, 1.f, 1.f};
          float lpdf = 1.f;
          mat_evaluate(mc, trace.normal, trace.light_direction, -g.direction, lrefl, lpdf, trace.uv, f.textures,
              f.n_textures);
          if (!inf3(lrefl)) {
            v4 const lc = unpack_unorm4x8(trace.light_color);
            v3 const c = v3{lc.x, lc.y, lc.z} * trace.light_strength * clamp3(lrefl, 0.f, 1.f);
            g.color = {g.color.x + c.x, g.color.y + c.y, g.color.z + c.z, g.color.w};
          }
        }
        g.direction = generated;
        g.origin = trace.point + 1e-4f * faceforward(trace.normal, -g.direction, trace.normal);
        g.pdf *= mpdf;
        g.reflectance = g.reflectance * mrefl;
        // The literal 2341335623 has no suffix: GLSL makes it an int with the same
        // bit pattern (GLSL 4.60, 4.1.3), i.e. -1953631673.
        g.random_value = random_value(r, int(std::uint32_t(f2i(-1953631673.f * g.random_value)) + 357883444u * uid));
        gen[id] = g;
      } else {
        v3 env;
        if (f.cubemap && f.cubemap_size > 10) {  // pt_color.comp:190-199
          env = clamp3(g.reflectance * cube_sample(f.cubemap, f.cubemap_size, g.direction) / g.pdf, 0.f, 16.f);
        } else {
          float const t = (g.direction.y + 1.f) / 2.f;
          v3 const sky = mix3(v3{0.3f, 0.4f, 0.5f}, v3{1.f, 0.98f, 0.96f}, t);
          env = clamp3(g.reflectance * sky / g.pdf, 0.f, 16.f);
        }
        acc(v4{g.color.x + env.x, g.color.y + env.y, g.color.z + env.z, g.color.w});
      }
    }
  });
}

// pt_ray_filter.comp:49-64, stable
void pass_filter(std::vector<gen_t>& gen, std::vector<trace_t> const& tr) {
  std::vector<gen_t> out;
  out.reserve(gen.size());
  for (std::size_t id = 0; id < gen.size(); ++id)
    if (tr[id].intersects == 1) out.push_back(gen[tr[id].generated_ray]);
  gen.swap(out);
}

}  // namespace

namespace orc_glsl {
int mode = 0;
}

extern "C" {

// GLSL built-ins of the restated passes (oracle_glsl_math.hpp): 0 = host libm
// (the pins against oracle/_ref), 1 = the library's glmath.hpp definitions.
void orc_set_glsl_math(int mode) { orc_glsl::mode = mode ? 1 : 0; }

// The library's GLSL built-ins (glmath.hpp) on the host: fn 0 sin, 1 cos,
// 2 atan, 3 exp, 4 pow(x, y).
void orc_glsl_eval(int fn, float const* x, float const* y, std::size_t n, float* out) {
  for (std::size_t i = 0; i < n; ++i) {
    switch (fn) {
      case 0: out[i] = myrt_glmath::sin(x[i]); break;
      case 1: out[i] = myrt_glmath::cos(x[i]); break;
      case 2: out[i] = myrt_glmath::atan(x[i]); break;
      case 3: out[i] = myrt_glmath::exp(x[i]); break;
      default: out[i] = myrt_glmath::pow(x[i], y[i]); break;
    }
  }
}


// Per-pass host randomness in the order sequential_pathtracer draws it for
// `frames` frames of `bounces` bounces from std::mt19937(seed):
//   generate: int then 1024 floats; trace: int then floats; color: floats then int.
// out_seeds: frames * passes ints, out_tex: frames * passes * 1024 floats,
// passes = 2 * bounces + 3 (generate, {trace, color} x (bounces + 1)).
void orc_host_rng(std::uint32_t seed, int frames, int bounces, std::int32_t* out_seeds, float* out_tex) {
  std::mt19937 rng(seed);
  int const passes = 2 * bounces + 3;
  for (int f = 0; f < frames; ++f) {
    for (int p = 0; p < passes; ++p) {
      std::uniform_int_distribution<> dist;
      std::uniform_real_distribution<float> uni(0.f, 1.f);
      std::int32_t& s = out_seeds[f * passes + p];
      float* t = out_tex + (std::size_t(f) * passes + p) * 1024;
      bool const is_color = p >= 1 && ((p - 1) % 2 == 1);
      if (!is_color) s = dist(rng);
      for (int k = 0; k < 1024; ++k) t[k] = uni(rng);
      if (is_color) s = dist(rng);
    }
  }
}

// Renders `frames` frames in reference-shading mode; accum/display are W*H*4
// floats, read and written (accumulation continues from sample_index0).
void orc_render_reference(std::size_t n_tris, float const* tris9, float const* normals9, float const* uvs6,
    std::int32_t const* tri_material, std::int32_t const* mat_refs, std::size_t n_mats, float const* mat_data,
    void const* nodes, std::uint32_t const* bvh_idx, int W, int H, int bounces, int frames,
    std::uint32_t sample_index0, float const* inv_view, float const* inv_proj, std::int32_t const* seeds,
    float const* tex, float* accum, float* display, std::int32_t const* sdf_instrs, std::int32_t const* sdf_programs,
    float const* sdf_params, float const* sdf_drawables, int n_sdf_drawables, int sdf_steps, float sdf_eps,
    int nthreads, int n_textures, float const* const* tex_data, int const* tex_dims, float const* cubemap,
    int cubemap_size, int dof, float lens_x, float lens_y, float focus, int bokeh_texture) {
  std::vector<tex_view> texv(std::size_t(std::max(n_textures, 0)));
  for (int k = 0; k < n_textures; ++k)
    texv[std::size_t(k)] = tex_view{tex_data[k], tex_dims[3 * k], tex_dims[3 * k + 1], tex_dims[3 * k + 2]};
  sdf_scene sdf;
  sdf.instrs = sdf_instrs;
  sdf.programs = sdf_programs;
  sdf.params = sdf_params;
  sdf.drawables = sdf_drawables;
  sdf.n_drawables = n_sdf_drawables;
  sdf.steps = sdf_steps;
  sdf.eps = sdf_eps;
  scene_t sc{n_tris, tris9, normals9, uvs6, tri_material, mat_refs, n_mats, mat_data, nodes, bvh_idx, {}, {}};
  sc.seq.resize(3 * n_tris);
  for (std::size_t i = 0; i < sc.seq.size(); ++i) sc.seq[i] = std::uint32_t(i);
  sc.pts4.resize(4 * 3 * n_tris);
  for (std::size_t i = 0; i < 3 * n_tris; ++i)
    for (int k = 0; k < 3; ++k) sc.pts4[4 * i + k] = tris9[3 * i + k];
  std::vector<v4> acc(std::size_t(W) * H), disp(std::size_t(W) * H);
  std::memcpy(acc.data(), accum, acc.size() * sizeof(v4));
  std::memcpy(disp.data(), display, disp.size() * sizeof(v4));
  int const passes = 2 * bounces + 3;
  for (int fr = 0; fr < frames; ++fr) {
    auto pr = [&](int p) {
      pass_rng r;
      r.seed = seeds[fr * passes + p];
      float const* t = tex + (std::size_t(fr) * passes + p) * 1024;
      r.tex.assign(t, t + 1024);
      return r;
    };
    frame_ctx f{&sc, W, H, inv_view, inv_proj, &acc, &disp, sample_index0 + std::uint32_t(fr), nthreads, &sdf};
    f.textures = texv.empty() ? nullptr : texv.data();
    f.n_textures = n_textures;
    f.cubemap = cubemap;
    f.cubemap_size = cubemap_size;
    f.dof = dof;
    f.lens[0] = lens_x;
    f.lens[1] = lens_y;
    f.focus = focus;
    if (bokeh_texture > 0 && bokeh_texture <= n_textures) f.bokeh = texv[std::size_t(bokeh_texture - 1)];
    std::vector<gen_t> gen;
    std::vector<trace_t> tr;
    pass_generate(f, pr(0), gen);
    int p = 1;
    for (int i = 0; i < bounces; ++i) {
      pass_trace(f, pr(p++), gen, tr);
      pass_color(f, pr(p++), gen, tr, false);
      pass_filter(gen, tr);
    }
    pass_trace(f, pr(p++), gen, tr);
    pass_color(f, pr(p++), gen, tr, true);
  }
  std::memcpy(accum, acc.data(), acc.size() * sizeof(v4));
  std::memcpy(display, disp.data(), disp.size() * sizeof(v4));
}

// Known-answer access to the restated shading functions (for the pins).
// map() of program `prog` at n points; with load_materials the material draws
// consume the random stream started from rng_states[i] (prime index 0).
void orc_sdf_map(std::int32_t const* instrs, std::int32_t const* programs, float const* params, int prog,
    float const* pts, std::size_t n, int load_materials, std::uint32_t const* rng_states, float* out_d, int* out_mat) {
  sdf_scene s;
  s.instrs = instrs;
  s.programs = programs;
  s.params = params;
  for (std::size_t i = 0; i < n; ++i) {
    rng_t r;
    r.state = rng_states ? rng_states[i] : 0u;
    r.prime = 0;
    sdf_ctx c{&s, &r, load_materials != 0, prog};
    int m = -1;
    out_d[i] = sdf_map(c, {pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]}, m);
    out_mat[i] = m;
  }
}

// SDF part of nearest_hit (pt_trace.comp:342-352) / any_hit (:321-326) over all
// drawables; same arguments and outputs as ref_sdf_trace in oracle/_ref.
void orc_sdf_trace(std::int32_t const* instrs, std::int32_t const* programs, float const* params,
    float const* drawables, int n_drawables, float const* rays, std::size_t n, int steps, float eps, int any_hit,
    std::uint32_t const* rng_states, int* out_hit, float* out_t, float* out_n, float* out_uv, int* out_mat,
    int nthreads) {
  sdf_scene s;
  s.instrs = instrs;
  s.programs = programs;
  s.params = params;
  s.drawables = drawables;
  s.n_drawables = n_drawables;
  s.steps = steps;
  s.eps = eps;
  par(n, nthreads, [&](std::size_t b, std::size_t e) {
    for (std::size_t i = b; i < e; ++i) {
      float const* q = rays + 8 * i;
      v3 const ro{q[0], q[1], q[2]}, rd{q[4], q[5], q[6]};
      float const maxd = q[7];
      rng_t r;
      r.state = rng_states ? rng_states[i] : 0u;
      r.prime = 0;
      sdf_hit hit;
      hit.t = maxd;
      if (any_hit) {
        for (int d = 0; d < n_drawables; ++d)
          if (march_sdf(s, r, d, ro, rd, maxd, true).hits) {
            hit.hits = true;
            break;
          }
      } else {
        for (int d = 0; d < n_drawables; ++d) {
          sdf_hit const h = march_sdf(s, r, d, ro, rd, hit.hits ? hit.t : maxd, false);
          if (h.hits && h.t < hit.t) hit = h;
        }
      }
      out_hit[i] = hit.hits ? 1 : 0;
      out_t[i] = hit.hits ? hit.t : maxd;
      out_n[3 * i] = hit.normal.x, out_n[3 * i + 1] = hit.normal.y, out_n[3 * i + 2] = hit.normal.z;
      out_uv[2 * i] = hit.uv.x, out_uv[2 * i + 1] = hit.uv.y;
      out_mat[i] = hit.hits ? hit.material : -1;
    }
  });
}

void orc_random_stream(float const* tex, int tex_size, int px, int py, int seed, int n, float* out,
    std::uint32_t* state_after_init) {
  rng_t r;
  random_init(r, tex, tex_size, px, py, seed);
  if (state_after_init) *state_after_init = r.state;
  for (int i = 0; i < n; ++i) out[i] = random_next(r);
}
std::uint32_t orc_wang_hash(std::uint32_t a) { return wang(a); }
void orc_transform_local_to_world(float const* v, float const* n, float* out) {
  v3 const r = transform_local_to_world({v[0], v[1], v[2]}, {n[0], n[1], n[2]});
  out[0] = r.x, out[1] = r.y, out[2] = r.z;
}
std::uint32_t orc_pack_unorm4x8(float const* v) { return pack_unorm4x8({v[0], v[1], v[2], v[3]}); }
float orc_intersect_sphere(float const* r0, float const* rd, float const* s0, float sr) {
  return intersect_sphere({r0[0], r0[1], r0[2]}, {rd[0], rd[1], rd[2]}, {s0[0], s0[1], s0[2]}, sr);
}
void orc_material_bounce_eval(float const* mat7, std::uint32_t* io_rng, float const* tv, float const* n, float* out_gen,
    float* out_refl, float* out_pdf, int* out_lobe, float* out_resample) {
  rng_t r;
  r.state = io_rng[0];
  r.prime = int(io_rng[1]);
  material_ctx mc;
  mat_open(mc, 0, mat7, 0);
  float const a = random_next(r);
  float const b = random_next(r);
  v3 const t{tv[0], tv[1], tv[2]}, nn{n[0], n[1], n[2]};
  v3 const g = mat_bounce(mc, r, v2{a, b}, t, nn);
  v3 refl;
  float pdf;
  mat_evaluate(mc, nn, g, t, refl, pdf);
  out_gen[0] = g.x, out_gen[1] = g.y, out_gen[2] = g.z;
  out_refl[0] = refl.x, out_refl[1] = refl.y, out_refl[2] = refl.z;
  *out_pdf = pdf;
  *out_lobe = mc.ps.state;
  *out_resample = mc.ps.resample;
  io_rng[0] = r.state;
  io_rng[1] = std::uint32_t(r.prime);
}
void orc_material_eval(float const* mat7, int lobe, float resample, float const* tl, float const* tv, float const* n,
    float* out_refl, float* out_pdf) {
  material_ctx mc;
  mat_open(mc, 0, mat7, 0);
  mc.ps.state = lobe;
  mc.ps.resample = resample;
  mc.ps.after_sample = false;
  v3 refl;
  float pdf;
  mat_evaluate(mc, {n[0], n[1], n[2]}, {tl[0], tl[1], tl[2]}, {tv[0], tv[1], tv[2]}, refl, pdf);
  out_refl[0] = refl.x, out_refl[1] = refl.y, out_refl[2] = refl.z;
  *out_pdf = pdf;
}

}  // extern "C"

// ==== physical shading mode ======================================================
extern "C" void orc_refbvh_query(void const* nodes_v, std::uint32_t const* bvh_idx, std::uint32_t const* indices,
    float const* points_xyzw, float const* rays, std::size_t n, int any_hit, int canonical, int isect,
    std::int32_t* prim, float* t_out, float* u_out, float* v_out, int nthreads);

// Path-at-a-time restatement of the physical mode (GGX + Lambert over the PBR
// record, NEE with the power heuristic to parallelogram lights, Russian
// roulette on the throughput, counter-based random numbers). The method is
// this project's own (the reference has no such mode); this is its checker.
// Only +, -, *, /, sqrt and comparisons: with -ffp-contract=off it reproduces
// the device kernels bit for bit.
namespace {

struct ph_u4 {
  std::uint32_t x, y, z, w;
};
// pcg4d (Jarzynski and Olano, JCGT 9(3) 2020)
ph_u4 ph_pcg4d(std::uint32_t a, std::uint32_t b, std::uint32_t c, std::uint32_t d) {
  ph_u4 v{a * 1664525u + 1013904223u, b * 1664525u + 1013904223u, c * 1664525u + 1013904223u,
      d * 1664525u + 1013904223u};
  v.x += v.y * v.w;
  v.y += v.z * v.x;
  v.z += v.x * v.y;
  v.w += v.y * v.z;
  v.x ^= v.x >> 16;
  v.y ^= v.y >> 16;
  v.z ^= v.z >> 16;
  v.w ^= v.w >> 16;
  v.x += v.y * v.w;
  v.y += v.z * v.x;
  v.z += v.x * v.y;
  v.w += v.y * v.z;
  return v;
}
inline float ph_u01(std::uint32_t x) { return float(x >> 8) * (1.0f / 16777216.0f); }
struct ph_r4 {
  float a, b, c, d;
};
inline ph_r4 ph_rand4(std::uint32_t pix, std::uint32_t sample, std::uint32_t seed, std::uint32_t stream) {
  ph_u4 const h = ph_pcg4d(pix, sample, seed, stream);
  return {ph_u01(h.x), ph_u01(h.y), ph_u01(h.z), ph_u01(h.w)};
}

// sin / cos of 2 pi u: nearest quadrant, Taylor series on [-pi/4, pi/4]
void ph_sincos_turns(float u, float& s, float& c) {
  float const x = u * 4.0f;
  float const k = std::nearbyint(x);
  float const a = (x - k) * 1.57079632679489662f;
  float const a2 = a * a;
  float const sp = a * (1.0f + a2 * (-1.0f / 6.0f + a2 * (1.0f / 120.0f + a2 * (-1.0f / 5040.0f + a2 * (1.0f / 362880.0f)))));
  float const cp = 1.0f + a2 * (-0.5f + a2 * (1.0f / 24.0f + a2 * (-1.0f / 720.0f + a2 * (1.0f / 40320.0f +
                                                                                        a2 * (-1.0f / 3628800.0f)))));
  int const q = int(k) & 3;
  s = q == 0 ? sp : (q == 1 ? cp : (q == 2 ? -sp : -cp));
  c = q == 0 ? cp : (q == 1 ? -sp : (q == 2 ? -cp : sp));
}

inline float ph_lum(v3 c) { return (0.2126f * c.x + 0.7152f * c.y) + 0.0722f * c.z; }
inline float ph_max3(v3 c) { return std::fmax(c.x, std::fmax(c.y, c.z)); }
inline bool ph_finite(v3 c) { return std::isfinite(c.x) && std::isfinite(c.y) && std::isfinite(c.z); }
constexpr float kPhPi = 3.14159265358979324f;
constexpr float kPhInvPi = 0.318309886183790672f;

struct ph_mat {
  v3 diffuse, f0;
  float alpha, p_spec;
};
ph_mat ph_load(float const* data, int off) {
  std::uint32_t bits;
  std::memcpy(&bits, data + off, 4);
  v3 const alb{float(bits & 0xffu) / 255.0f, float((bits >> 8) & 0xffu) / 255.0f, float((bits >> 16) & 0xffu) / 255.0f};
  float const ior = data[off + 1], rough = data[off + 2], metal = data[off + 3];
  float const r = (ior - 1.0f) / (ior + 1.0f);
  float const f0d = r * r;
  ph_mat m;
  m.f0 = v3{f0d, f0d, f0d} * (1.0f - metal) + alb * metal;
  m.diffuse = alb * ((1.0f - metal) * (1.0f - f0d));
  m.alpha = std::fmax(rough * rough, 1e-3f);
  float const ws = ph_lum(m.f0), wd = ph_lum(m.diffuse);
  m.p_spec = wd > 0.0f ? std::fmin(std::fmax(ws / (ws + wd), 0.25f), 0.9f) : 1.0f;
  return m;
}
inline float ph_lambda(float c, float a2) {
  float const c2 = c * c;
  return (std::sqrt(1.0f + a2 * ((1.0f - c2) / c2)) - 1.0f) * 0.5f;
}
struct ph_eval {
  v3 f{0, 0, 0};
  float pdf = 0, cos_i = 0;
};
ph_eval ph_bsdf(ph_mat const& m, v3 ns, v3 ng, v3 wo, v3 wi) {
  ph_eval r;
  float const ci = dot(ns, wi), co = dot(ns, wo);
  if (!(ci > 0.0f) || !(dot(ng, wi) > 0.0f) || !(co > 0.0f)) return r;
  v3 const h = normalize(wo + wi);
  float const ch = dot(ns, h), coh = dot(wo, h);
  float const a2 = m.alpha * m.alpha;
  float const tt = ch * ch * (a2 - 1.0f) + 1.0f;
  float const D = a2 / ((kPhPi * tt) * tt);
  float const lo = ph_lambda(co, a2), li = ph_lambda(ci, a2);
  float const G1 = 1.0f / (1.0f + lo);
  float const G2 = 1.0f / ((1.0f + lo) + li);
  float const om = 1.0f - std::fmax(coh, 0.0f);
  float const om2 = om * om;
  float const w5 = om2 * om2 * om;
  v3 const F = m.f0 + (v3{1.0f, 1.0f, 1.0f} - m.f0) * w5;
  float const spec = (D * G2) / ((4.0f * co) * ci);
  r.f = m.diffuse * kPhInvPi + F * spec;
  float const ps = coh > 0.0f ? (G1 * D) / (4.0f * co) : 0.0f;
  r.pdf = m.p_spec * ps + (1.0f - m.p_spec) * (ci * kPhInvPi);
  r.cos_i = ci;
  return r;
}
void ph_onb(v3 n, v3& t, v3& b) {
  float const sign = n.z >= 0.0f ? 1.0f : -1.0f;
  float const a = -1.0f / (sign + n.z);
  float const bb = n.x * n.y * a;
  t = {1.0f + sign * n.x * n.x * a, sign * bb, -sign * n.x};
  b = {bb, sign + n.y * n.y * a, -n.y};
}
bool ph_sample(ph_mat const& m, v3 ns, v3 wo, float ul, float u1, float u2, v3& wi) {
  v3 t, b;
  ph_onb(ns, t, b);
  float s, c;
  if (ul < m.p_spec) {  // GGX visible normals (Heitz, JCGT 7(4) 2018)
    v3 const wl{dot(wo, t), dot(wo, b), dot(wo, ns)};
    v3 const vh = normalize(v3{m.alpha * wl.x, m.alpha * wl.y, wl.z});
    float const lensq = vh.x * vh.x + vh.y * vh.y;
    v3 T1{1.0f, 0.0f, 0.0f};
    if (lensq > 0.0f) {
      float const il = 1.0f / std::sqrt(lensq);
      T1 = v3{-vh.y * il, vh.x * il, 0.0f};
    }
    v3 const T2 = cross(vh, T1);
    float const r = std::sqrt(u1);
    ph_sincos_turns(u2, s, c);
    float const t1 = r * c;
    float const sh = 0.5f * (1.0f + vh.z);
    float const t2 = (1.0f - sh) * std::sqrt(1.0f - t1 * t1) + sh * (r * s);
    float const nz = std::sqrt(std::fmax(0.0f, (1.0f - t1 * t1) - t2 * t2));
    v3 const nh = (T1 * t1 + T2 * t2) + vh * nz;
    v3 const ne = normalize(v3{m.alpha * nh.x, m.alpha * nh.y, std::fmax(1e-6f, nh.z)});
    v3 const h = (t * ne.x + b * ne.y) + ns * ne.z;
    wi = h * (2.0f * dot(wo, h)) - wo;
  } else {  // cosine-weighted hemisphere
    float const r = std::sqrt(u1);
    ph_sincos_turns(u2, s, c);
    float const z = std::sqrt(std::fmax(0.0f, 1.0f - u1));
    wi = (t * (r * c) + b * (r * s)) + ns * z;
  }
  return dot(wi, ns) > 0.0f;
}

// 24 floats per light: corner, eu, ev, emission, normal, area, du, prob, dv, cdf
struct ph_light {
  v3 c, eu, ev, e, n;
  float area;
  v3 du;
  float prob;
  v3 dv;
  float cdf;
};
bool ph_light_hit(ph_light const& L, v3 o, v3 d, float tmax, float& t) {
  float const den = dot(d, L.n);
  if (!(std::fabs(den) > 1e-12f)) return false;
  float const tt = dot(L.c - o, L.n) / den;
  if (!(tt > 0.0f) || !(tt < tmax)) return false;
  v3 const p = (o + d * tt) - L.c;
  float const a = dot(p, L.du), b = dot(p, L.dv);
  if (!(a >= 0.0f && a <= 1.0f && b >= 0.0f && b <= 1.0f)) return false;
  t = tt;
  return true;
}
inline float ph_power(float a, float b) {
  float const a2 = a * a;
  return a2 / (a2 + b * b);
}

// one watertight query on the restated reference BVH (canonical closest hit)
inline void extern_refbvh_query(scene_t const& sc, float const* ray, int any_hit, std::int32_t& prim, float& t,
    float& u, float& v) {
  orc_refbvh_query(sc.nodes, sc.bvh_idx, sc.seq.data(), sc.pts4.data(), ray, 1, any_hit, 1, 1, &prim, &t, &u, &v, 1);
}

struct ph_scene {
  scene_t* sc;
  sdf_scene const* sdf;
  std::vector<ph_light> lights;
  v3 env;
};

struct ph_hit {
  int kind = -1;  // material >= 0, -1 miss, -2 - l light
  float t = 0;
  v3 pos{0, 0, 0}, ns{0, 0, 0}, ng{0, 0, 0};
};

ph_hit ph_closest(ph_scene const& S, v3 o, v3 d, std::uint32_t sdf_state) {
  scene_t const& sc = *S.sc;
  float const inf = std::numeric_limits<float>::infinity();
  float const ray[8] = {o.x, o.y, o.z, 0.f, d.x, d.y, d.z, inf};
  std::int32_t prim;
  float t, u, v;
  extern_refbvh_query(sc, ray, 0, prim, t, u, v);
  ph_hit h;
  h.t = prim >= 0 ? t : inf;
  if (prim >= 0) {
    float const* P = sc.tris9 + 9 * std::size_t(prim);
    v3 const p0{P[0], P[1], P[2]}, p1{P[3], P[4], P[5]}, p2{P[6], P[7], P[8]};
    float const w = (1.f - u) - v;
    h.pos = (u * p1 + v * p2) + w * p0;
    h.ng = normalize(cross(p1 - p0, p2 - p0));
    if (sc.normals9) {
      float const* N = sc.normals9 + 9 * std::size_t(prim);
      h.ns = normalize((u * v3{N[3], N[4], N[5]} + v * v3{N[6], N[7], N[8]}) + w * v3{N[0], N[1], N[2]});
    } else {
      h.ns = h.ng;
    }
    h.kind = sc.tri_material[prim];
  }
  if (S.sdf && S.sdf->n_drawables > 0) {
    rng_t r;
    r.state = sdf_state;
    r.prime = 0;
    for (int k = 0; k < S.sdf->n_drawables; ++k) {
      sdf_hit const sh = march_sdf(*S.sdf, r, k, o, d, h.t, false);
      if (sh.hits && sh.t < h.t) {
        h.t = sh.t;
        h.pos = sh.position;
        h.ns = h.ng = sh.normal;
        h.kind = sh.material;
      }
    }
  }
  for (std::size_t l = 0; l < S.lights.size(); ++l) {
    float tl;
    if (ph_light_hit(S.lights[l], o, d, h.t, tl)) {
      h.t = tl;
      h.kind = -2 - int(l);
    }
  }
  return h;
}

bool ph_occluded(ph_scene const& S, v3 o, v3 d, float tmax, std::uint32_t sdf_state) {
  float const ray[8] = {o.x, o.y, o.z, 0.f, d.x, d.y, d.z, tmax};
  std::int32_t prim;
  float t, u, v;
  extern_refbvh_query(*S.sc, ray, 1, prim, t, u, v);
  if (prim >= 0) return true;
  if (S.sdf && S.sdf->n_drawables > 0) {
    rng_t r;
    r.state = sdf_state;
    r.prime = 0;
    for (int k = 0; k < S.sdf->n_drawables; ++k)
      if (march_sdf(*S.sdf, r, k, o, d, tmax, true).hits) return true;
  }
  return false;
}

struct ph_params {
  int W, H, max_depth, rr_start;
  std::uint32_t seed, sample;
  float vp[16];
  v3 eye;
};

v3 ph_path(ph_scene const& S, ph_params const& P, std::uint32_t pix) {
  std::uint32_t const x = pix % std::uint32_t(P.W), y = pix / std::uint32_t(P.W);
  ph_r4 const rc = ph_rand4(pix, P.sample, P.seed, 0xffffu);
  float const nx = ((rc.a + float(x)) / float(P.W)) * 2.f - 1.f;
  float const ny = ((rc.b + float(y)) / float(P.H)) * 2.f - 1.f;
  float h[3];
  for (int k = 0; k < 3; ++k) h[k] = ((P.vp[0 * 4 + k] * nx + P.vp[1 * 4 + k] * ny) + P.vp[2 * 4 + k]) + P.vp[3 * 4 + k];
  v3 o = P.eye, d = normalize(v3{h[0], h[1], h[2]});
  v3 T{1.f, 1.f, 1.f}, L{0.f, 0.f, 0.f};
  float prev_pdf = 0.f;
  scene_t const& sc = *S.sc;
  for (int v = 0;; ++v) {
    std::uint32_t const sdf_state = ph_pcg4d(pix, P.sample, P.seed, 4u * std::uint32_t(v) + 2u).x;
    ph_hit const hit = ph_closest(S, o, d, sdf_state);
    if (hit.kind == -1) {
      L = L + T * S.env;
      break;
    }
    if (hit.kind <= -2) {
      ph_light const& lt = S.lights[std::size_t(-2 - hit.kind)];
      float const cl = -dot(d, lt.n);
      if (cl > 0.f) {
        float w = 1.f;
        if (v > 0 && prev_pdf > 0.f) w = ph_power(prev_pdf, (lt.prob * (hit.t * hit.t)) / (lt.area * cl));
        L = L + (T * lt.e) * w;
      }
      break;
    }
    if (v >= P.max_depth) break;
    if (std::size_t(hit.kind) >= sc.n_mats || sc.mat_refs[2 * hit.kind] != 0) break;
    ph_mat const m = ph_load(sc.mat_data, sc.mat_refs[2 * hit.kind + 1]);
    v3 ns = hit.ns, ng = hit.ng;
    v3 const wo = -d;
    float const gdo = dot(ng, wo);
    if (gdo < 0.f) ng = -ng;
    if (dot(ns, ng) < 0.f) ns = -ns;
    if (!(dot(ns, wo) > 0.f)) ns = ng;
    if (gdo == 0.f) break;
    ph_r4 const r0 = ph_rand4(pix, P.sample, P.seed, 4u * std::uint32_t(v));
    ph_r4 const r1 = ph_rand4(pix, P.sample, P.seed, 4u * std::uint32_t(v) + 1u);
    v3 const org = hit.pos + ng * 1e-4f;
    if (!S.lights.empty()) {
      std::size_t l = 0;
      while (l + 1 < S.lights.size() && r1.a >= S.lights[l].cdf) ++l;
      ph_light const& lt = S.lights[l];
      v3 const yy = (lt.c + lt.eu * r1.b) + lt.ev * r1.c;
      v3 const dv = yy - hit.pos;
      float const dist2 = dot(dv, dv);
      float const dist = std::sqrt(dist2);
      v3 const wi = dv * (1.f / dist);
      float const cl = -dot(wi, lt.n);
      if (cl > 0.f && dist > 0.f) {
        ph_eval const bv = ph_bsdf(m, ns, ng, wo, wi);
        if (bv.pdf > 0.f) {
          float const pl = (lt.prob * dist2) / (lt.area * cl);
          float const w = ph_power(pl, bv.pdf);
          v3 const c = ((T * bv.f) * lt.e) * ((bv.cos_i * w) / pl);
          if (ph_max3(c) > 0.f && !ph_occluded(S, org, wi, dist * 0.999f, sdf_state)) L = L + c;
        }
      }
    }
    v3 wi;
    if (!ph_sample(m, ns, wo, r0.a, r0.b, r0.c, wi)) break;
    ph_eval const bv = ph_bsdf(m, ns, ng, wo, wi);
    if (!(bv.pdf > 0.f && bv.cos_i > 0.f)) break;
    v3 Tn = T * (bv.f * (bv.cos_i / bv.pdf));
    if (!(ph_finite(Tn) && ph_max3(Tn) > 0.f)) break;
    if (v >= P.rr_start) {
      float const q = std::fmin(ph_max3(Tn), 0.95f);
      if (r0.d >= q) break;
      Tn = Tn / q;
    }
    o = org;
    d = wi;
    prev_pdf = bv.pdf;
    T = Tn;
  }
  return L;
}

}  // namespace

extern "C" {
// Physical-mode render of samples [sample0, sample0 + spp) into accum (W*H*4;
// float, or double when fp64). lights: 24 floats each (ph_light layout,
// precomputed by the caller). sdf_*: as orc_render_reference (n = 0: none).
void orc_render_physical(std::size_t n_tris, float const* tris9, float const* normals9, std::int32_t const* tri_material,
    std::int32_t const* mat_refs, std::size_t n_mats, float const* mat_data, void const* nodes,
    std::uint32_t const* bvh_idx, float const* lights24, int n_lights, float const* env, int W, int H, int spp,
    std::uint32_t sample0, int max_depth, int rr_start, std::uint32_t seed, float const* vp16, float const* eye,
    std::int32_t const* sdf_instrs, std::int32_t const* sdf_programs, float const* sdf_params,
    float const* sdf_drawables, int n_sdf_drawables, int sdf_steps, float sdf_eps, int fp64, void* accum,
    int nthreads) {
  sdf_scene sdf;
  sdf.instrs = sdf_instrs;
  sdf.programs = sdf_programs;
  sdf.params = sdf_params;
  sdf.drawables = sdf_drawables;
  sdf.n_drawables = n_sdf_drawables;
  sdf.steps = sdf_steps;
  sdf.eps = sdf_eps;
  scene_t sc{n_tris, tris9, normals9, nullptr, tri_material, mat_refs, n_mats, mat_data, nodes, bvh_idx, {}, {}};
  sc.seq.resize(3 * n_tris);
  for (std::size_t i = 0; i < sc.seq.size(); ++i) sc.seq[i] = std::uint32_t(i);
  sc.pts4.resize(4 * 3 * n_tris);
  for (std::size_t i = 0; i < 3 * n_tris; ++i)
    for (int k = 0; k < 3; ++k) sc.pts4[4 * i + k] = tris9[3 * i + k];
  ph_scene S{&sc, &sdf, {}, {env[0], env[1], env[2]}};
  for (int l = 0; l < n_lights; ++l) {
    float const* q = lights24 + 24 * l;
    S.lights.push_back({{q[0], q[1], q[2]}, {q[3], q[4], q[5]}, {q[6], q[7], q[8]}, {q[9], q[10], q[11]},
        {q[12], q[13], q[14]}, q[15], {q[16], q[17], q[18]}, q[19], {q[20], q[21], q[22]}, q[23]});
  }
  std::size_t const WH = std::size_t(W) * H;
  par(WH, nthreads, [&](std::size_t b, std::size_t e) {
    for (std::size_t pix = b; pix < e; ++pix) {
      for (int s = 0; s < spp; ++s) {
        ph_params P{W, H, max_depth, rr_start, seed, sample0 + std::uint32_t(s), {}, eye ? v3{eye[0], eye[1], eye[2]}
                                                                                      : v3{0, 0, 0}};
        std::memcpy(P.vp, vp16, sizeof(P.vp));
        v3 const L = ph_path(S, P, std::uint32_t(pix));
        bool const ok = ph_finite(L);
        if (fp64) {
          double* a = static_cast<double*>(accum) + 4 * pix;
          if (ok) {
            a[0] = a[0] + double(L.x);
            a[1] = a[1] + double(L.y);
            a[2] = a[2] + double(L.z);
          }
          a[3] = a[3] + 1.0;
        } else {
          float* a = static_cast<float*>(accum) + 4 * pix;
          if (ok) {
            a[0] = a[0] + L.x;
            a[1] = a[1] + L.y;
            a[2] = a[2] + L.z;
          }
          a[3] = a[3] + 1.f;
        }
      }
    }
  });
}
}  // extern "C"

// ---- forward (raster preview) renderer ---------------------------------------------------
// forward_renderer.cpp:13-318 with forward/vert.vert, frag.frag, resolve.frag.
// Rasterisation as GL defines it (pixel centres at +0.5, perspective-correct
// attributes, clipping to -w <= z <= w, 24-bit depth, GL_LESS in draw order),
// written as homogeneous rasterisation (Olano & Greer 1997): per triangle the
// edge functions of the homogeneous window coordinates (X, Y, w) =
// ((x + w) W / 2, (y + w) H / 2, w); a pixel centre is covered when the three
// sign-normalised edge functions are positive (zero: top-left rule);
// barycentrics are the edge functions over their sum; z_ndc = sum e_i z_i /
// |det|. Triangles are drawn one after another; a fragment replaces the stored
// one when its (depth, triangle) key is smaller, which is GL_LESS in draw
// order. Every product and sum is rounded separately (-ffp-contract=off), in
// the order the device code writes them.
extern "C" float oracle_half_rn(float f);
namespace {

struct fmat {
  float m[16];
};
fmat fmul(fmat const& a, fmat const& b) {
  fmat c{};
  for (int col = 0; col < 4; ++col)
    for (int r = 0; r < 4; ++r) {
      float s = a.m[r] * b.m[col * 4];
      for (int k = 1; k < 4; ++k) s = s + a.m[k * 4 + r] * b.m[col * 4 + k];
      c.m[col * 4 + r] = s;
    }
  return c;
}
// inverse by cofactors in double, rounded once to float
fmat finverse(fmat const& a) {
  double m[16], inv[16];
  for (int i = 0; i < 16; ++i) m[i] = a.m[i];
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
  fmat r{};
  for (int i = 0; i < 16; ++i) r.m[i] = float(inv[i] / det);
  return r;
}
v4 fmulv(fmat const& a, float x, float y, float z, float w) {
  v4 r;
  float* o = &r.x;
  for (int i = 0; i < 4; ++i) o[i] = ((a.m[i] * x + a.m[4 + i] * y) + a.m[8 + i] * z) + a.m[12 + i] * w;
  return r;
}

struct fwd_tri {
  float e[3][4];  // sign-normalised edge functions (a, b, c) and z_i / |det|
  std::uint32_t flags = 0;
  int x0 = 0, y0 = 0, x1 = -1, y1 = -1;
};
// vert.vert + the rasteriser's triangle set-up
bool fwd_setup(float const* p, fmat const& pv, int W, int H, fwd_tri& t) {
  float const hw = float(W) * 0.5f, hh = float(H) * 0.5f;
  float X[3], Y[3], Wc[3], Z[3];
  bool finite = true, front = true;
  for (int k = 0; k < 3; ++k) {
    v4 const c = fmulv(pv, p[3 * k], p[3 * k + 1], p[3 * k + 2], 1.f);
    X[k] = (c.x + c.w) * hw;
    Y[k] = (c.y + c.w) * hh;
    Z[k] = c.z;
    Wc[k] = c.w;
    finite = finite && std::isfinite(X[k]) && std::isfinite(Y[k]) && std::isfinite(Z[k]) && std::isfinite(Wc[k]);
    front = front && Wc[k] > 0.f;
  }
  float e[3][3];
  for (int i = 0; i < 3; ++i) {
    int const j = (i + 1) % 3, k = (i + 2) % 3;
    e[i][0] = Y[j] * Wc[k] - Wc[j] * Y[k];
    e[i][1] = Wc[j] * X[k] - X[j] * Wc[k];
    e[i][2] = X[j] * Y[k] - Y[j] * X[k];
  }
  float const det = (e[0][0] * X[0] + e[0][1] * Y[0]) + e[0][2] * Wc[0];
  if (!finite || det == 0.f || !std::isfinite(det)) return false;
  float const sg = det > 0.f ? 1.f : -1.f, ad = std::fabs(det);
  t.flags = 0;
  for (int i = 0; i < 3; ++i) {
    float const ea = e[i][0] * sg, eb = e[i][1] * sg, ec = e[i][2] * sg;
    if (ea > 0.f || (ea == 0.f && eb > 0.f)) t.flags |= 1u << i;
    t.e[i][0] = ea, t.e[i][1] = eb, t.e[i][2] = ec, t.e[i][3] = Z[i] / ad;
  }
  int x0 = 0, y0 = 0, x1 = W - 1, y1 = H - 1;
  if (front) {
    float lx = INFINITY, ly = INFINITY, ux = -INFINITY, uy = -INFINITY;
    for (int k = 0; k < 3; ++k) {
      float const sx = X[k] / Wc[k], sy = Y[k] / Wc[k];
      lx = std::fmin(lx, sx), ux = std::fmax(ux, sx), ly = std::fmin(ly, sy), uy = std::fmax(uy, sy);
    }
    x0 = int(std::fmax(std::floor(lx) - 1.f, 0.f)), y0 = int(std::fmax(std::floor(ly) - 1.f, 0.f));
    x1 = int(std::fmin(std::floor(ux) + 1.f, float(W) - 1.f)), y1 = int(std::fmin(std::floor(uy) + 1.f, float(H) - 1.f));
  }
  t.x0 = x0, t.y0 = y0, t.x1 = x1, t.y1 = y1;
  return x1 >= x0 && y1 >= y0;
}
bool fwd_covered(fwd_tri const& t, int x, int y, float* e) {
  float const X = float(x) + 0.5f, Y = float(y) + 0.5f;
  bool in = true;
  for (int i = 0; i < 3; ++i) {
    e[i] = (t.e[i][0] * X + t.e[i][1] * Y) + t.e[i][2];
    in = in && (e[i] > 0.f || (e[i] == 0.f && ((t.flags >> i) & 1u)));
  }
  return in;
}
// draws all triangles into keys (W * H, all ones = empty); tris keeps the set-ups
void fwd_raster(int n, float const* pos, fmat const& pv, int W, int H, std::uint64_t* keys, std::vector<fwd_tri>& tris) {
  std::fill(keys, keys + std::size_t(W) * H, ~std::uint64_t(0));
  tris.assign(std::size_t(n), fwd_tri{});
  for (int t = 0; t < n; ++t) {
    fwd_tri& tr = tris[std::size_t(t)];
    if (!fwd_setup(pos + 9 * std::size_t(t), pv, W, H, tr)) continue;
    for (int y = tr.y0; y <= tr.y1; ++y)
      for (int x = tr.x0; x <= tr.x1; ++x) {
        float e[3];
        if (!fwd_covered(tr, x, y, e)) continue;
        float const zn = (e[0] * tr.e[0][3] + e[1] * tr.e[1][3]) + e[2] * tr.e[2][3];
        if (!(zn >= -1.f && zn <= 1.f)) continue;
        std::uint32_t const d = std::uint32_t(std::nearbyint((zn * 0.5f + 0.5f) * 16777215.f));
        if (d >= 0xffffffu) continue;
        std::uint64_t const key = (std::uint64_t(d) << 32) | std::uint32_t(t);
        std::uint64_t& dst = keys[std::size_t(y) * W + x];
        if (key < dst) dst = key;
      }
  }
}
inline float ld(float const* p) { return *p; }
// frag.frag outputs per pixel: G-buffer layers (half-rounded) or shadow positions
void fwd_attributes(std::vector<fwd_tri> const& tris, std::uint64_t const* keys, int W, int H, float const* pos,
    float const* nrm, float const* uvs, std::int32_t const* mat, float* gbuf, float* smap) {
  std::size_t const plane = std::size_t(W) * H;
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      std::size_t const px = std::size_t(y) * W + x;
      std::uint64_t const key = keys[px];
      if (key == ~std::uint64_t(0)) {
        if (gbuf)
          for (int l = 0; l < 3; ++l) std::fill(gbuf + 4 * (l * plane + px), gbuf + 4 * (l * plane + px) + 4, 0.f);
        else
          std::fill(smap + 4 * px, smap + 4 * px + 4, 0.f);
        continue;
      }
      std::uint32_t const t = std::uint32_t(key & 0xffffffffu);
      float e[3];
      fwd_covered(tris[t], x, y, e);
      float const s = (e[0] + e[1]) + e[2];
      float const l0 = e[0] / s, l1 = e[1] / s, l2 = e[2] / s;
      float const* P = pos + 9 * std::size_t(t);
      v3 const p0{P[0], P[1], P[2]}, p1{P[3], P[4], P[5]}, p2{P[6], P[7], P[8]};
      v3 const q = (l0 * p0 + l1 * p1) + l2 * p2;
      if (!gbuf) {
        float* o = smap + 4 * px;
        o[0] = q.x, o[1] = q.y, o[2] = q.z, o[3] = 1.f;
        continue;
      }
      v3 n;
      if (nrm) {
        float const* N = nrm + 9 * std::size_t(t);  // 3 corners, xyz
        n = normalize((l0 * v3{N[0], N[1], N[2]} + l1 * v3{N[3], N[4], N[5]}) + l2 * v3{N[6], N[7], N[8]});
      } else {
        n = normalize(cross(normalize(p1 - p0), normalize(p2 - p0)));
      }
      float u = 0.f, v = 0.f;
      if (uvs) {
        float const* U = uvs + 6 * std::size_t(t);
        u = (l0 * U[0] + l1 * U[2]) + l2 * U[4];
        v = (l0 * U[1] + l1 * U[3]) + l2 * U[5];
      }
      float const vals[3][4] = {{q.x, q.y, q.z, 1.f}, {u, v, 0.f, 0.f}, {n.x, n.y, n.z, float(mat[t])}};
      for (int l = 0; l < 3; ++l)
        for (int c = 0; c < 4; ++c) gbuf[4 * (l * plane + px) + c] = oracle_half_rn(vals[l][c]);
    }
}
// uint(f) as NVIDIA GPUs convert it (truncation, saturation, NaN -> 0)
inline std::uint32_t f2u_sat(float f) {
  if (!(f > 0.f)) return 0u;
  if (f >= 4294967296.f) return 0xffffffffu;
  return std::uint32_t(f);
}
inline int f2i_idx(float f) { return (f > -2147483648.f && f < 2147483648.f) ? int(f) : 0; }
// random.glsl:52-60
inline void random_init_nt(rng_t& r, int px, int py, int seed) {
  r.state = std::uint32_t(seed);
  r.prime = 0;
  r.tex = nullptr;
  r.tex_size = 0;
  int const a = random_int(r, px ^ 0xba77fa);
  int const b = random_int(r, py ^ 0xcca6df);
  int const c = random_int(r, seed);
  int const seed_base = int(std::uint32_t(a) * 69019u + std::uint32_t(b) * 96013u + std::uint32_t(c));
  int const rem = seed_base % 12352345;
  random_value(r, int(std::uint32_t(seed_base) + 16756614u * std::uint32_t(rem)));
}

}  // namespace

extern "C" {

// forward_renderer::run: G-buffer pass, shadow pass, resolve. Outputs (any may
// be null): vis / svis keys, gbuf (3 layers of H*W*4 half-rounded floats),
// smap (S*S*4), result (H*W*4 half-rounded).
void orc_forward_render(int n, float const* pos, float const* nrm, float const* uvs, std::int32_t const* mat,
    std::int32_t const* refs, int n_refs, float const* mdata, int W, int H, float const* view, float const* proj,
    std::uint32_t seed, int S, float const* shadow_view, float const* shadow_proj, int n_textures,
    float const* const* tex_data, int const* tex_dims, std::uint64_t* vis_out, float* gbuf_out,
    std::uint64_t* svis_out, float* smap_out, float* result) {
  fmat V, P, SV, SP;
  std::memcpy(V.m, view, 64);
  std::memcpy(P.m, proj, 64);
  std::memcpy(SV.m, shadow_view, 64);
  std::memcpy(SP.m, shadow_proj, 64);
  fmat const pv = fmul(P, V), spv = fmul(SP, SV);
  fmat const inv_view = finverse(V);
  fmat const inv_vp = fmul(inv_view, finverse(P));
  fmat const inv_sview = finverse(SV);
  std::size_t const plane = std::size_t(W) * H, splane = std::size_t(S) * S;
  std::vector<std::uint64_t> vis(plane), svis(splane);
  std::vector<float> gbuf(3 * plane * 4), smap(splane * 4);
  std::vector<fwd_tri> tris;
  fwd_raster(n, pos, pv, W, H, vis.data(), tris);
  fwd_attributes(tris, vis.data(), W, H, pos, nrm, uvs, mat, gbuf.data(), nullptr);
  fwd_raster(n, pos, spv, S, S, svis.data(), tris);
  fwd_attributes(tris, svis.data(), S, S, pos, nrm, uvs, mat, nullptr, smap.data());
  if (vis_out) std::copy(vis.begin(), vis.end(), vis_out);
  if (svis_out) std::copy(svis.begin(), svis.end(), svis_out);
  if (gbuf_out) std::copy(gbuf.begin(), gbuf.end(), gbuf_out);
  if (smap_out) std::copy(smap.begin(), smap.end(), smap_out);
  if (!result) return;
  std::vector<tex_view> texv(std::size_t(std::max(n_textures, 0)));
  for (int k = 0; k < n_textures; ++k)
    texv[std::size_t(k)] = tex_view{tex_data[k], tex_dims[3 * k], tex_dims[3 * k + 1], tex_dims[3 * k + 2]};
  v3 const cam{inv_view.m[12], inv_view.m[13], inv_view.m[14]};
  v3 light;
  {
    float const lx = ((inv_sview.m[0] * 0.f + inv_sview.m[4] * 0.f) + inv_sview.m[8] * 1.f) + inv_sview.m[12] * 0.f;
    float const ly = ((inv_sview.m[1] * 0.f + inv_sview.m[5] * 0.f) + inv_sview.m[9] * 1.f) + inv_sview.m[13] * 0.f;
    float const lz = ((inv_sview.m[2] * 0.f + inv_sview.m[6] * 0.f) + inv_sview.m[10] * 1.f) + inv_sview.m[14] * 0.f;
    float const len = std::sqrt((lx * lx + ly * ly) + lz * lz);
    float const inv = 1.f / len;
    light = {lx * inv, ly * inv, lz * inv};
  }
  float const fw = float(W), fh = float(H), fs = float(S);
  auto g = [&](int layer, std::size_t px) { return gbuf.data() + 4 * (std::size_t(layer) * plane + px); };
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      std::size_t const px = std::size_t(y) * W + x;
      float const* g0 = g(0, px);
      float const* g1 = g(1, px);
      float const* g2 = g(2, px);
      float* out = result + 4 * px;
      if (g2[0] == 0.f && g2[1] == 0.f && g2[2] == 0.f) {
        float const nx = (float(x) / fw) * 2.f - 1.f, ny = (float(y) / fh) * 2.f - 1.f;
        v4 const h = fmulv(inv_vp, nx, ny, 1.f, 1.f);
        v3 const d = normalize(v3{h.x, h.y, h.z});
        v3 const c = mix3(v3{0.3f, 0.4f, 0.5f}, v3{1.0f, 0.98f, 0.96f}, (d.y + 1.f) / 2.f);
        out[0] = oracle_half_rn(c.x), out[1] = oracle_half_rn(c.y), out[2] = oracle_half_rn(c.z);
        out[3] = oracle_half_rn(1.f);
        continue;
      }
      v3 const position{g0[0], g0[1], g0[2]};
      v3 const to_cam = normalize(cam - position);
      v3 normal = normalize(v3{g2[0], g2[1], g2[2]});
      normal = faceforward(normal, -to_cam, normal);
      v2 const uv{g1[0], g1[1]};
      int const material = f2i_idx(g2[3]);
      v4 const sp = fmulv(SV, position.x, position.y, position.z, 1.f);
      v4 const spx = fmulv(SP, sp.x, sp.y, sp.z, sp.w);
      float const su = ((spx.x / spx.w) + 1.f) / 2.f, sv = ((spx.y / spx.w) + 1.f) / 2.f;
      rng_t rng;
      std::uint32_t const sd =
          ((seed + 9897584u * f2u_sat(position.x)) ^ f2u_sat(position.y)) ^ f2u_sat(position.z);
      random_init_nt(rng, x, y, int(sd));
      float avg = 0.f;
      int const r = 9;
      for (int i = 0; i < r; ++i) {
        float const qx = random_next(rng);
        float const qy = random_next(rng);
        float const hx = 2.f * qx - 1.f, hy = 2.f * qy - 1.f;
        float const u = su + (2.5f * hx) / fs, v = sv + (2.5f * hy) / fs;
        if (u >= 1.f || v >= 1.f || u < 0.f || v < 0.f) {
          avg += 1.f;
          continue;
        }
        int const tx = int(std::uint32_t(f2i_idx(std::floor(u * fs))) % std::uint32_t(S));
        int const ty = int(std::uint32_t(f2i_idx(std::floor(v * fs))) % std::uint32_t(S));
        float const* m = smap.data() + 4 * (std::size_t(ty) * S + tx);
        v3 const check = position - 100.f * light;
        float const l1 = length(check - v3{m[0], m[1], m[2]});
        avg += (l1 - 100.f < 0.01f) ? 1.f : 0.f;
      }
      float const shadow = avg / float(r);
      material_ctx mc;
      bool const valid = material >= 0 && material < n_refs;
      if (valid) mat_open(mc, refs[2 * material], mdata, refs[2 * material + 1]);
      mc.ps.state = 2;  // s_diffuse
      v3 refl{0.f, 0.f, 0.f};
      float pdf = 1.f;
      mat_evaluate(mc, normal, light, to_cam, refl, pdf, uv, texv.data(), n_textures);
      v3 refgb{0.f, 0.f, 0.f};
      float refpdf = 1.f;
      mc.ps.state = 2;
      mat_evaluate(mc, normal, normal, to_cam, refgb, refpdf, uv, texv.data(), n_textures);
      float freeness = 0.f;
      float dist = 0.1f;
      for (int i = 0; i < 8; ++i) {
        do {
          float const qx = random_next(rng);
          float const qy = random_next(rng);
          v2 const hs{2.f * qx - 1.f, 2.f * qy - 1.f};
          v3 const world = normalize(transform_local_to_world(sample_hemisphere(hs), normal));
          v3 const test = position + world * dist;
          v4 const hom = fmulv(pv, test.x, test.y, test.z, 1.f);
          if (hom.w == 0.f) {
            freeness += 1.f;
            break;
          }
          float const ox = std::fmin(std::fmax((((hom.x / hom.w) + 1.f) / 2.f) * fw, 0.f), fw - 1.f);
          float const oy = std::fmin(std::fmax((((hom.y / hom.w) + 1.f) / 2.f) * fh, 0.f), fh - 1.f);
          std::size_t const o = std::size_t(f2i_idx(oy)) * W + std::size_t(f2i_idx(ox));
          float const* on = g(2, o);
          if (on[0] == 0.f && on[1] == 0.f && on[2] == 0.f) {
            freeness += 1.f;
            break;
          }
          float const* op = g(0, o);
          float const diff = length(cam - v3{op[0], op[1], op[2]}) - length(cam - test);
          if (diff > 0.f) {
            freeness += 1.f;
            break;
          }
          freeness += (diff < -0.2f) ? 1.f : 0.f;
        } while (false);
        dist /= 2.f;
      }
      freeness /= 1.f * 8.f;
      float const lcol = 3.f;
      float const ndl = gmax(0.f, dot(normal, light));
      v3 const direct = (((lcol * refl) / pdf) * shadow) * ndl;
      v3 c = freeness * (refgb / refpdf + direct);
      float const k = 0.7f + 0.4f * random_next(rng);
      c = c * k;
      out[0] = oracle_half_rn(c.x), out[1] = oracle_half_rn(c.y), out[2] = oracle_half_rn(c.z);
      out[3] = oracle_half_rn(1.f * 0.f);
    }
}

}  // extern "C"

// ---- single passes on caller buffers (for pinning against the reference's own
// pt_generate.comp / pt_color.comp compiled as C++) ----------------------------------------
extern "C" {

// pass_color over n rays: gen (80-byte records) and trace (64-byte records)
// are updated in place; accum / display are W x H RGBA float images.
void orc_pass_color(int n, void* gen, void* trace, float* accum, float* display, int width, int height,
    std::uint32_t sample_index, int force, int seed, float const* random_tex, int tex_size, std::int32_t const* refs,
    int n_refs, float const* mdata) {
  scene_t sc{};
  sc.mat_refs = refs;
  sc.n_mats = std::size_t(std::max(n_refs, 0));
  sc.mat_data = mdata;
  std::size_t const px = std::size_t(width) * std::size_t(height);
  std::vector<v4> acc(px), disp(px);
  std::memcpy(acc.data(), accum, px * sizeof(v4));
  std::memcpy(disp.data(), display, px * sizeof(v4));
  sdf_scene const no_sdf{};
  frame_ctx f{&sc, width, height, nullptr, nullptr, &acc, &disp, sample_index, 1, &no_sdf};
  pass_rng const pr{seed, std::vector<float>(random_tex, random_tex + tex_size)};
  std::vector<gen_t> g(static_cast<gen_t*>(gen), static_cast<gen_t*>(gen) + n);
  std::vector<trace_t> t(static_cast<trace_t*>(trace), static_cast<trace_t*>(trace) + n);
  pass_color(f, pr, g, t, force != 0);
  std::memcpy(gen, g.data(), std::size_t(n) * sizeof(gen_t));
  std::memcpy(trace, t.data(), std::size_t(n) * sizeof(trace_t));
  std::memcpy(accum, acc.data(), px * sizeof(v4));
  std::memcpy(display, disp.data(), px * sizeof(v4));
}

// pass_generate over a width x height image into gen (width * height records).
void orc_pass_generate(int width, int height, float const* inv_view, float const* inv_proj, int seed,
    float const* random_tex, int tex_size, int dof, float lens_x, float lens_y, float focus, float const* bokeh,
    int bokeh_w, int bokeh_h, int bokeh_wrap, void* gen) {
  scene_t sc{};
  std::vector<v4> acc, disp;
  sdf_scene const no_sdf{};
  frame_ctx f{&sc, width, height, inv_view, inv_proj, &acc, &disp, 0u, 1, &no_sdf};
  f.dof = dof;
  f.lens[0] = lens_x;
  f.lens[1] = lens_y;
  f.focus = focus;
  if (bokeh) f.bokeh = tex_view{bokeh, bokeh_w, bokeh_h, bokeh_wrap};
  pass_rng const pr{seed, std::vector<float>(random_tex, random_tex + tex_size)};
  std::vector<gen_t> g;
  pass_generate(f, pr, g);
  std::memcpy(gen, g.data(), g.size() * sizeof(gen_t));
}

}  // extern "C"
