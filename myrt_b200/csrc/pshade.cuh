// Physical shading: GGX (height-correlated Smith, Schlick Fresnel) + Lambert
// BSDF over the reference's 7-float PBR record (src/main.cpp:447-464:
// albedo unorm8x4 bits, ior, roughness, metallic, transmission, texture),
// next-event estimation to parallelogram area lights with the power
// heuristic, and a counter-based random stream.
//
// Every function here uses only +, -, *, /, sqrt and comparisons, and the
// translation units that include it are compiled without FMA contraction, so
// a host restatement with -ffp-contract=off reproduces each path bit for bit.
// Angles come from sincos_turns (a Taylor polynomial on one octant), not from
// the math library.
//
// Random numbers: rand4(pixel, sample, seed, stream) is the pcg4d hash of
// Jarzynski and Olano ("Hash Functions for GPU Rendering", JCGT 9(3) 2020);
// a path vertex v draws from streams 4v + {0: bsdf lobe, u1, u2, roulette;
// 1: light pick, u1, u2, guide coin; 2: SDF material stream; 3: guide lobe},
// the camera from stream 0xffff. Results therefore depend only on (pixel,
// sample, seed), not on how rays are queued, compacted or batched.
#pragma once
#include <cstdint>

#include "refshade.cuh"

namespace myrt_b200 {
namespace ps {

using rs::v3;

struct u4 {
  uint32_t x, y, z, w;
};

__device__ __forceinline__ u4 pcg4d(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  u4 v{a * 1664525u + 1013904223u, b * 1664525u + 1013904223u, c * 1664525u + 1013904223u,
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
__device__ __forceinline__ float u01(uint32_t x) { return float(x >> 8) * (1.0f / 16777216.0f); }

struct rnd4 {
  float a, b, c, d;
  uint32_t raw;  // first word, for seeding other streams
};
__device__ __forceinline__ rnd4 rand4(uint32_t pixel, uint32_t sample, uint32_t seed, uint32_t stream) {
  u4 const h = pcg4d(pixel, sample, seed, stream);
  return {u01(h.x), u01(h.y), u01(h.z), u01(h.w), h.x};
}

// sin and cos of 2*pi*u for u in [0, 1]: u*4 split into the nearest quadrant k
// and a remainder r in [-1/2, 1/2] (both exact), the angle r*pi/2 in
// [-pi/4, pi/4] through the Taylor series of sin (to x^9) and cos (to x^10),
// whose truncation error there is below 2e-9, then rotated by k quadrants.
__device__ __forceinline__ void sincos_turns(float u, float& s, float& c) {
  float const x = u * 4.0f;
  float const k = rintf(x);
  float const a = (x - k) * 1.57079632679489662f;
  float const a2 = a * a;
  float const sp = a * (1.0f + a2 * (-1.0f / 6.0f + a2 * (1.0f / 120.0f + a2 * (-1.0f / 5040.0f + a2 * (1.0f / 362880.0f)))));
  float const cp = 1.0f + a2 * (-0.5f + a2 * (1.0f / 24.0f + a2 * (-1.0f / 720.0f + a2 * (1.0f / 40320.0f +
                                                                                        a2 * (-1.0f / 3628800.0f)))));
  int const q = int(k) & 3;
  s = q == 0 ? sp : (q == 1 ? cp : (q == 2 ? -sp : -cp));
  c = q == 0 ? cp : (q == 1 ? -sp : (q == 2 ? -cp : sp));
}

// dot = (x x' + y y') + z z', cross, normalize = v * (1 / sqrt(dot(v, v))):
// rs:: (found by argument lookup on rs::v3).
__device__ __forceinline__ float lum(v3 c) { return (0.2126f * c.x + 0.7152f * c.y) + 0.0722f * c.z; }
__device__ __forceinline__ float max3(v3 c) { return fmaxf(c.x, fmaxf(c.y, c.z)); }
__device__ __forceinline__ bool finite3(v3 c) { return isfinite(c.x) && isfinite(c.y) && isfinite(c.z); }

constexpr float kPi = 3.14159265358979324f;
constexpr float kInvPi = 0.318309886183790672f;

// Orthonormal basis around n (Duff et al., "Building an Orthonormal Basis,
// Revisited", JCGT 6(1) 2017).
__device__ __forceinline__ void onb(v3 n, v3& t, v3& b) {
  float const sign = n.z >= 0.0f ? 1.0f : -1.0f;
  float const a = -1.0f / (sign + n.z);
  float const bb = n.x * n.y * a;
  t = {1.0f + sign * n.x * n.x * a, sign * bb, -sign * n.x};
  b = {bb, sign + n.y * n.y * a, -n.y};
}

struct material {
  v3 albedo;   // diffuse colour (1 - metallic)(1 - F0d) albedo
  v3 f0;       // specular reflectance at normal incidence
  float alpha; // GGX roughness^2, >= 1e-3
  float p_spec;
};

// PBR record at data + offset: albedo bits, ior, roughness, metallic.
__device__ __forceinline__ material load_material(float const* data, int offset) {
  uint32_t const bits = __float_as_uint(data[offset]);
  v3 const alb{float(bits & 0xffu) / 255.0f, float((bits >> 8) & 0xffu) / 255.0f, float((bits >> 16) & 0xffu) / 255.0f};
  float const ior = data[offset + 1], rough = data[offset + 2], metal = data[offset + 3];
  float const r = (ior - 1.0f) / (ior + 1.0f);
  float const f0d = r * r;
  material m;
  m.f0 = v3{f0d, f0d, f0d} * (1.0f - metal) + alb * metal;
  m.albedo = alb * ((1.0f - metal) * (1.0f - f0d));
  m.alpha = fmaxf(rough * rough, 1e-3f);
  float const ws = lum(m.f0), wd = lum(m.albedo);
  m.p_spec = wd > 0.0f ? fminf(fmaxf(ws / (ws + wd), 0.25f), 0.9f) : 1.0f;
  return m;
}

// Smith Lambda for GGX at cos theta = c (> 0).
__device__ __forceinline__ float ggx_lambda(float c, float a2) {
  float const c2 = c * c;
  return (sqrtf(1.0f + a2 * ((1.0f - c2) / c2)) - 1.0f) * 0.5f;
}

struct bsdf_val {
  v3 f;       // BSDF value (without the cosine)
  float pdf;  // solid-angle pdf of the lobe mixture the sampler draws from
  float cos_i;
};

// BSDF and sampling pdf for wo, wi around shading normal ns (geometric ng).
__device__ __forceinline__ bsdf_val bsdf_eval(material const& m, v3 ns, v3 ng, v3 wo, v3 wi) {
  bsdf_val r{{0.0f, 0.0f, 0.0f}, 0.0f, 0.0f};
  float const cos_i = dot(ns, wi), cos_o = dot(ns, wo);
  if (!(cos_i > 0.0f) || !(dot(ng, wi) > 0.0f) || !(cos_o > 0.0f)) return r;
  v3 const h = normalize(wo + wi);
  float const cos_h = dot(ns, h), cos_oh = dot(wo, h);
  float const a2 = m.alpha * m.alpha;
  float const tt = cos_h * cos_h * (a2 - 1.0f) + 1.0f;
  float const D = a2 / ((kPi * tt) * tt);
  float const lo = ggx_lambda(cos_o, a2), li = ggx_lambda(cos_i, a2);
  float const G1 = 1.0f / (1.0f + lo);
  float const G2 = 1.0f / ((1.0f + lo) + li);
  float const om = 1.0f - fmaxf(cos_oh, 0.0f);
  float const om2 = om * om;
  float const w5 = om2 * om2 * om;
  v3 const F = m.f0 + (v3{1.0f, 1.0f, 1.0f} - m.f0) * w5;
  float const spec = (D * G2) / ((4.0f * cos_o) * cos_i);
  r.f = m.albedo * kInvPi + F * spec;
  float const pdf_s = cos_oh > 0.0f ? (G1 * D) / (4.0f * cos_o) : 0.0f;
  float const pdf_d = cos_i * kInvPi;
  r.pdf = m.p_spec * pdf_s + (1.0f - m.p_spec) * pdf_d;
  r.cos_i = cos_i;
  return r;
}

// Draws wi from the lobe mixture: GGX visible normals (Heitz, "Sampling the
// GGX Distribution of Visible Normals", JCGT 7(4) 2018) with probability
// p_spec, else a cosine-weighted hemisphere. Returns false for a direction
// below the surface.
__device__ __forceinline__ bool bsdf_sample(material const& m, v3 ns, v3 wo, float u_lobe, float u1, float u2, v3& wi) {
  v3 t, b;
  onb(ns, t, b);
  float s, c;
  if (u_lobe < m.p_spec) {
    v3 const wl{dot(wo, t), dot(wo, b), dot(wo, ns)};
    v3 const vh = normalize(v3{m.alpha * wl.x, m.alpha * wl.y, wl.z});
    float const lensq = vh.x * vh.x + vh.y * vh.y;
    v3 T1{1.0f, 0.0f, 0.0f};
    if (lensq > 0.0f) {
      float const il = 1.0f / sqrtf(lensq);
      T1 = v3{-vh.y * il, vh.x * il, 0.0f};
    }
    v3 const T2 = cross(vh, T1);
    float const r = sqrtf(u1);
    sincos_turns(u2, s, c);
    float const t1 = r * c;
    float const sh = 0.5f * (1.0f + vh.z);
    float const t2 = (1.0f - sh) * sqrtf(1.0f - t1 * t1) + sh * (r * s);
    float const nz = sqrtf(fmaxf(0.0f, (1.0f - t1 * t1) - t2 * t2));
    v3 const nh = (T1 * t1 + T2 * t2) + vh * nz;
    v3 const ne = normalize(v3{m.alpha * nh.x, m.alpha * nh.y, fmaxf(1e-6f, nh.z)});
    v3 const h = (t * ne.x + b * ne.y) + ns * ne.z;
    float const d = dot(wo, h);
    wi = h * (2.0f * d) - wo;
  } else {
    float const r = sqrtf(u1);
    sincos_turns(u2, s, c);
    float const z = sqrtf(fmaxf(0.0f, 1.0f - u1));
    wi = (t * (r * c) + b * (r * s)) + ns * z;
  }
  return dot(wi, ns) > 0.0f;
}

// Parallelogram area light; host-precomputed normal, area, dual edge vectors
// (for the hit coordinates) and selection probability / cumulative sum.
struct area_light {
  float corner[3], eu[3], ev[3], emission[3];
  float normal[3], area;
  float du[3], prob;
  float dv[3], cdf;
};

__device__ __forceinline__ v3 lv(float const* p) { return {p[0], p[1], p[2]}; }

// Ray / parallelogram: t in (0, tmax) and coordinates in [0, 1]^2.
__device__ __forceinline__ bool light_hit(area_light const& L, v3 o, v3 d, float tmax, float& t) {
  v3 const n = lv(L.normal);
  float const den = dot(d, n);
  if (!(fabsf(den) > 1e-12f)) return false;
  float const tt = dot(lv(L.corner) - o, n) / den;
  if (!(tt > 0.0f) || !(tt < tmax)) return false;
  v3 const p = (o + d * tt) - lv(L.corner);
  float const a = dot(p, lv(L.du)), b = dot(p, lv(L.dv));
  if (!(a >= 0.0f && a <= 1.0f && b >= 0.0f && b <= 1.0f)) return false;
  t = tt;
  return true;
}

__device__ __forceinline__ float power_heuristic(float a, float b) {
  float const a2 = a * a;
  return a2 / (a2 + b * b);
}

}  // namespace ps
}  // namespace myrt_b200
