// Physical and guided wavefront path tracing, for one view or a batch of
// views of many scenes.
//
// Work is organised in waves. A wave holds whole sample rows (all W*H pixels
// of one sample index) of one or more jobs (job = scene + camera +
// resolution + spp + seed); the wave's job table gives each job its rows,
// first sample index and first path slot. Per wave:
//
//   k_pt_camera                 camera rays (box-filtered pixel jitter)
//   for vertex v = 0 .. max_depth:
//     k_pt_extend               closest hit: 8-wide BVH (watertight), SDF
//                               drawables (sphere tracing), area lights
//     [guided: k_guide_gather + k_guide_forward (guide.cu)]
//     k_pt_shade                emission with MIS, NEE toward one light,
//                               BSDF (or guide) sampling, Russian roulette;
//                               survivors and shadow rays are appended to
//                               the next queues with warp-aggregated atomics
//     k_pt_shadow               any-hit for the NEE rays, adds unoccluded
//                               contributions
//   k_pt_resolve (per job)      the job's rows, in sample order, into its
//                               FP32 or FP64 accumulation
//
// Queue order never reaches the result: each path's random numbers are keyed
// by (pixel, sample, seed) and each path's radiance is summed in event order
// in its own slot; rows reach the accumulation in sample order. A job
// therefore renders the same image bit for bit alone or inside any batch,
// with any wave size. A batch's whole frame (all waves) is captured once as
// a CUDA graph; each replay first copies the per-wave job tables (sample
// bases, overwrite flags) from pinned host memory.
// Compiled with -fmad=false (build.py) like the other shading unit.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/myrt_cuda.h"
#include "ctx.hpp"
#include "guide.cuh"
#include "pshade.cuh"
#include "refshade.cuh"
#include "sdf.cuh"
#include "trace.cuh"
#include "rayorder.cuh"

namespace myrt_b200 {

enum : uint32_t {
  ERR_BAD_MATERIAL = 1u << 4,  // material index out of range or unknown type
};

namespace {

using rs::v3;
constexpr int kPtBlock = 128;
constexpr float kOffset = 1e-4f;  // ray origin offset along the geometric normal
constexpr int kMaxLights = 64;
constexpr float kInf = __builtin_huge_valf();

// One scene: geometry, materials, lights, SDF drawables.
struct pt_scene {
  uint4 const* nodes;
  float4 const* tris;
  float4 const* tri_normals;  // may be null
  int32_t const* tri_material;
  int2 const* mat_refs;
  int n_mats;
  float const* mat_data;
  ps::area_light const* lights;
  int n_lights;
  sdfk::sdf_dev sdf;  // steps / eps come from the job
  float3 key_lo, key_scale;  // ray_key's grid over the scene box
};

// One job within one wave.
struct pt_job {
  uint32_t W, H, WH, scene;
  uint32_t seed;
  int max_depth, rr_start;
  uint32_t fp64;
  float vp[16];  // inverse_view * inverse_projection
  float eye[3];
  float env[3];
  int sdf_steps;
  float sdf_eps;
  uint32_t sample_base;  // sample index of the job's first row in this wave
  uint32_t rows;         // rows in this wave (0: none)
  uint32_t path_offset;  // slot of the job's first path in this wave
  uint32_t overwrite;    // 1: the resolve starts a new accumulation
  float4* accum;
  double4* accum64;
  float4* display;
};

struct pt_wave {
  pt_scene const* scenes;
  pt_job const* jobs;
  int n_jobs;
  uint32_t n_paths;
  uint32_t* err;
};

__device__ __forceinline__ v3 xyz(float4 a) { return {a.x, a.y, a.z}; }

__device__ __forceinline__ int find_job(pt_wave const& w, uint32_t g) {
  int j = 0;
  for (int k = 1; k < w.n_jobs; ++k)
    if (g >= w.jobs[k].path_offset && w.jobs[k].rows > 0) j = k;
  return j;
}

__device__ __forceinline__ sdfk::sdf_dev job_sdf(pt_scene const& s, pt_job const& J) {
  sdfk::sdf_dev d = s.sdf;
  d.steps = J.sdf_steps;
  d.eps = J.sdf_eps;
  return d;
}

// Appends one entry per lane with `emit` set; all 32 lanes must call it.
__device__ __forceinline__ uint32_t warp_append(bool emit, uint32_t* count) {
  uint32_t const lane = threadIdx.x & 31u;
  uint32_t const m = __ballot_sync(0xffffffffu, emit);
  uint32_t base = 0;
  if (lane == 0 && m) base = atomicAdd(count, uint32_t(__popc(m)));
  base = __shfl_sync(0xffffffffu, base, 0);
  return base + uint32_t(__popc(m & ((1u << lane) - 1u)));
}

// ---- camera ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kPtBlock) k_pt_camera(pt_wave w, float4* __restrict__ q,
    float4* __restrict__ radiance, uint32_t* __restrict__ count) {
  uint32_t const stride = gridDim.x * blockDim.x;
  if (blockIdx.x == 0 && threadIdx.x == 0) *count = w.n_paths;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < w.n_paths; i += stride) {
    int const j = find_job(w, i);
    pt_job const& J = w.jobs[j];
    uint32_t const p = i - J.path_offset;
    uint32_t const pix = p % J.WH, sample = J.sample_base + p / J.WH;
    uint32_t const x = pix % J.W, y = pix / J.W;
    ps::rnd4 const r = ps::rand4(pix, sample, J.seed, 0xffffu);
    float const nx = ((r.a + float(x)) / float(J.W)) * 2.f - 1.f;
    float const ny = ((r.b + float(y)) / float(J.H)) * 2.f - 1.f;
    float h[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) h[k] = ((J.vp[0 * 4 + k] * nx + J.vp[1 * 4 + k] * ny) + J.vp[2 * 4 + k]) + J.vp[3 * 4 + k];
    v3 const d = rs::normalize(v3{h[0], h[1], h[2]});
    q[3 * size_t(i)] = make_float4(J.eye[0], J.eye[1], J.eye[2], __uint_as_float(i));
    q[3 * size_t(i) + 1] = make_float4(d.x, d.y, d.z, 0.f);
    q[3 * size_t(i) + 2] = make_float4(1.f, 1.f, 1.f, __int_as_float(j));
    radiance[i] = make_float4(0.f, 0.f, 0.f, 1.f);  // w: roulette throughput of guided waves
  }
}

__device__ __forceinline__ void path_key(pt_job const& J, uint32_t path, uint32_t& pix, uint32_t& sample) {
  uint32_t const p = path - J.path_offset;
  pix = p % J.WH;
  sample = J.sample_base + p / J.WH;
}

__device__ __forceinline__ rs::rng_t sdf_stream(pt_job const& J, uint32_t path, int v) {
  uint32_t pix, sample;
  path_key(J, path, pix, sample);
  rs::rng_t r;
  r.state = ps::pcg4d(pix, sample, J.seed, 4u * uint32_t(v) + 2u).x;
  r.prime = 0;
  r.tex = nullptr;
  return r;
}

// ---- extend: closest hit over meshes, SDF drawables and lights ---------------------------
// perm (may be null): the visiting order; thread i takes queue entry perm[i],
// whose hit record is written at that entry's own index.
// hits[3i] = (position, kind): kind >= 0 material index, -1 miss, -2 - l light l;
// hits[3i+1] = (shading normal, t); hits[3i+2] = (geometric normal, 0).
template <bool SDF, int MINB = 8>
__global__ void __launch_bounds__(kPtBlock, MINB) k_pt_extend(pt_wave w, int v, float4 const* __restrict__ q,
    uint32_t const* __restrict__ count, float4* __restrict__ hits, uint32_t* __restrict__ clear_a,
    uint32_t* __restrict__ clear_b, unsigned long long* __restrict__ stats, uint32_t const* __restrict__ perm) {
  uint32_t const n = *count;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *clear_a = 0;
    *clear_b = 0;
    stats[1] += n;
    if (v == 0) stats[0] += n;
  }
  uint32_t const stride = gridDim.x * blockDim.x;
  for (uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += stride) {
    uint32_t const i = perm ? __ldg(perm + i0) : i0;
    float4 const q0 = q[3 * size_t(i)], q1 = q[3 * size_t(i) + 1];
    int const j = __float_as_int(q[3 * size_t(i) + 2].w);
    pt_job const& J = w.jobs[j];
    pt_scene const& s = w.scenes[J.scene];
    v3 const o = xyz(q0), d = xyz(q1);
    hit_rec h;
    uint32_t cn = 0, ct = 0;
    bool const hit =
        traverse<1, false, false>(s.nodes, s.tris, f3{o.x, o.y, o.z}, f3{d.x, d.y, d.z}, 0.f, kInf, h, w.err, cn, ct);
    float t = hit ? h.t : kInf;
    int kind = -1;
    v3 pos{0.f, 0.f, 0.f}, ns{0.f, 0.f, 0.f}, ng{0.f, 0.f, 0.f};
    if (hit) {
      float4 const* tp = s.tris + 3 * size_t(h.leaf);
      v3 const p0 = xyz(__ldg(tp)), p1 = xyz(__ldg(tp + 1)), p2 = xyz(__ldg(tp + 2));
      float const wb = (1.f - h.u) - h.v;
      pos = (h.u * p1 + h.v * p2) + wb * p0;
      ng = rs::normalize(rs::cross(p1 - p0, p2 - p0));
      uint32_t const prim = uint32_t(h.prim);
      if (s.tri_normals) {
        float4 const* np = s.tri_normals + 3 * size_t(prim);
        ns = rs::normalize((h.u * xyz(__ldg(np + 1)) + h.v * xyz(__ldg(np + 2))) + wb * xyz(__ldg(np)));
      } else {
        ns = ng;
      }
      kind = __ldg(s.tri_material + prim);
    }
    if (SDF && s.sdf.n_drawables > 0) {
      sdfk::sdf_dev const sd = job_sdf(s, J);
      rs::rng_t rng = sdf_stream(J, __float_as_uint(q0.w), v);
      for (int k = 0; k < sd.n_drawables; ++k) {
        sdfk::sdf_hit const sh = sdfk::march(sd, k, o, d, t, false, &rng);
        if (sh.hits && sh.t < t) {
          t = sh.t;
          pos = sh.position;
          ns = ng = sh.normal;
          kind = sh.material;
        }
      }
    }
    for (int l = 0; l < s.n_lights; ++l) {
      float tl;
      if (ps::light_hit(s.lights[l], o, d, t, tl)) {
        t = tl;
        kind = -2 - l;
      }
    }
    hits[3 * size_t(i)] = make_float4(pos.x, pos.y, pos.z, __int_as_float(kind));
    hits[3 * size_t(i) + 1] = make_float4(ns.x, ns.y, ns.z, t);
    hits[3 * size_t(i) + 2] = make_float4(ng.x, ng.y, ng.z, 0.f);
  }
}

// Visiting order of an extension queue: each live entry's origin / direction
// cell key in its scene's grid (ray_key), 0xFFFFFF (after every live key) for
// the wave's empty slots.
__global__ void __launch_bounds__(256) k_pt_keys(pt_wave w, float4 const* __restrict__ q,
    uint32_t const* __restrict__ count, uint32_t n_max, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  uint32_t const i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_max) return;
  uint32_t key = 0xFFFFFFu;
  if (i < *count) {
    pt_scene const& s = w.scenes[w.jobs[__float_as_int(q[3 * size_t(i) + 2].w)].scene];
    key = min(ray_key(q[3 * size_t(i)], q[3 * size_t(i) + 1], s.key_lo, s.key_scale), 0xFFFFFEu);
  }
  keys[i] = key;
  vals[i] = i;
}

// ---- shade ------------------------------------------------------------------------------
struct shade_io {
  float4 const* q;
  float4 const* hits;
  uint32_t const* count;
  float4* q_out;
  uint32_t* count_out;
  float4* shadow;
  uint32_t* count_shadow;
  float4* radiance;
  guide_dev guide;  // guide.n_lobes == 0: plain BSDF sampling
  uint32_t const* perm;  // may be null: thread i shades entry perm[i] (the extend kernel's order)
};

// Six resident blocks per SM (80 registers, some spills; 150 unbounded): measured 1.8 % faster per
// frame on a 512x512 64-spp render.
__global__ void __launch_bounds__(kPtBlock, 6) k_pt_shade(pt_wave w, int v, shade_io io) {
  uint32_t const n = *io.count;
  uint32_t const stride = gridDim.x * blockDim.x;
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += stride) {  // warp-uniform trip count
    uint32_t const i0 = base + threadIdx.x;
    bool const active = i0 < n;
    uint32_t const i = active && io.perm ? __ldg(io.perm + i0) : i0;
    bool emit_next = false, emit_shadow = false;
    float4 nq0, nq1, nq2, sq0, sq1, sq2;
    if (active) {
      float4 const q0 = io.q[3 * size_t(i)], q1 = io.q[3 * size_t(i) + 1], q2 = io.q[3 * size_t(i) + 2];
      float4 const h0 = io.hits[3 * size_t(i)], h1 = io.hits[3 * size_t(i) + 1], h2 = io.hits[3 * size_t(i) + 2];
      uint32_t const path = __float_as_uint(q0.w);
      int const j = __float_as_int(q2.w);
      pt_job const& J = w.jobs[j];
      pt_scene const& s = w.scenes[J.scene];
      v3 const d = xyz(q1), T = xyz(q2);
      float const prev_pdf = q1.w;
      int const kind = __float_as_int(h0.w);
      float4 const L0 = io.radiance[path];
      v3 L = xyz(L0);
      bool touched = false;
      if (io.guide.records && v > 0) guide_record_at(io.guide, path, v - 1)[5] = L0;
      if (kind == -1) {
        v3 const env{J.env[0], J.env[1], J.env[2]};
        L = L + T * env;
        touched = true;
      } else if (kind <= -2) {
        ps::area_light const& lt = s.lights[-2 - kind];
        float const cos_l = -rs::dot(d, ps::lv(lt.normal));
        if (cos_l > 0.f) {
          float wm = 1.f;
          if (v > 0 && prev_pdf > 0.f) {
            float const t = h1.w;
            float const pl = (lt.prob * (t * t)) / (lt.area * cos_l);
            wm = ps::power_heuristic(prev_pdf, pl);
          }
          L = L + (T * ps::lv(lt.emission)) * wm;
          touched = true;
        }
      } else if (v < J.max_depth) {
        bool ok = kind < s.n_mats;
        int2 mref{0, 0};
        if (ok) mref = __ldg(s.mat_refs + kind);
        if (!ok || mref.x != 0) {
          atomicOr(w.err, ERR_BAD_MATERIAL);
          ok = false;
        }
        v3 const pos = xyz(h0);
        v3 ns = xyz(h1), ng = xyz(h2);
        v3 const wo = -d;
        float const gdo = rs::dot(ng, wo);
        if (gdo < 0.f) ng = -ng;
        if (rs::dot(ns, ng) < 0.f) ns = -ns;
        if (!(rs::dot(ns, wo) > 0.f)) ns = ng;
        if (ok && gdo != 0.f) {
          ps::material const m = ps::load_material(s.mat_data, mref.y);
          uint32_t pix, sample;
          path_key(J, path, pix, sample);
          ps::rnd4 const r0 = ps::rand4(pix, sample, J.seed, 4u * uint32_t(v));
          ps::rnd4 const r1 = ps::rand4(pix, sample, J.seed, 4u * uint32_t(v) + 1u);
          v3 const org = pos + ng * kOffset;
          guide_lobes gl;
          bool const gwave = io.guide.n_lobes > 0;
          bool const guided = gwave && guide_load(io.guide, i, gl) && io.guide.fraction > 0.f;
          // next-event estimation
          if (s.n_lights > 0) {
            int l = 0;
            while (l < s.n_lights - 1 && r1.a >= s.lights[l].cdf) ++l;
            ps::area_light const& lt = s.lights[l];
            v3 const y = (ps::lv(lt.corner) + ps::lv(lt.eu) * r1.b) + ps::lv(lt.ev) * r1.c;
            v3 const dv = y - pos;
            float const dist2 = rs::dot(dv, dv);
            float const dist = sqrtf(dist2);
            v3 const wi = dv * (1.f / dist);
            float const cos_l = -rs::dot(wi, ps::lv(lt.normal));
            if (cos_l > 0.f && dist > 0.f) {
              ps::bsdf_val const bv = ps::bsdf_eval(m, ns, ng, wo, wi);
              float const pb = guided ? guide_mix_pdf(io.guide, gl, wi, bv.pdf) : bv.pdf;
              if (bv.pdf > 0.f) {
                float const pl = (lt.prob * dist2) / (lt.area * cos_l);
                float const wm = ps::power_heuristic(pl, pb);
                v3 const c = ((T * bv.f) * ps::lv(lt.emission)) * ((bv.cos_i * wm) / pl);
                if (ps::max3(c) > 0.f) {
                  emit_shadow = true;
                  sq0 = make_float4(org.x, org.y, org.z, __uint_as_float(path));
                  sq1 = make_float4(wi.x, wi.y, wi.z, dist * 0.999f);
                  sq2 = make_float4(c.x, c.y, c.z, __int_as_float(j));
                }
              }
            }
          }
          // continuation
          v3 wi;
          bool sampled;
          if (guided && r1.d < io.guide.fraction) {
            ps::rnd4 const r3 = ps::rand4(pix, sample, J.seed, 4u * uint32_t(v) + 3u);
            sampled = guide_sample(gl, r3.a, r3.b, r3.c, wi) && rs::dot(wi, ng) > 0.f;
          } else {
            sampled = ps::bsdf_sample(m, ns, wo, r0.a, r0.b, r0.c, wi);
          }
          if (sampled) {
            ps::bsdf_val const bv = ps::bsdf_eval(m, ns, ng, wo, wi);
            float const pdf = guided ? guide_mix_pdf(io.guide, gl, wi, bv.pdf) : bv.pdf;
            if (pdf > 0.f && bv.cos_i > 0.f) {
              v3 Tn = T * (bv.f * (bv.cos_i / pdf));
              bool alive = ps::finite3(Tn) && ps::max3(Tn) > 0.f;
              // Guided waves: roulette on the throughput the path would carry
              // under BSDF sampling (radiance.w), not on Tn. A guided direction
              // has a large pdf exactly where the incident radiance is large,
              // so a small Tn there does not mean a small contribution.
              float tb = 0.f;
              if (gwave) {
                float const fb = bv.pdf > 0.f ? ps::max3(bv.f * (bv.cos_i / bv.pdf)) : 1.f;
                tb = L0.w * fb;
              }
              if (alive && v >= J.rr_start) {
                float const qq = fminf(gwave ? tb : ps::max3(Tn), 0.95f);
                if (r0.d >= qq) alive = false;
                else {
                  Tn = Tn / qq;
                  tb = tb / qq;
                }
              }
              if (alive && gwave) io.radiance[path].w = tb;
              if (alive) {
                emit_next = true;
                nq0 = make_float4(org.x, org.y, org.z, __uint_as_float(path));
                nq1 = make_float4(wi.x, wi.y, wi.z, pdf);
                nq2 = make_float4(Tn.x, Tn.y, Tn.z, __int_as_float(j));
                if (io.guide.records) {
                  float4* rec = guide_record_at(io.guide, path, v);
                  rec[0] = make_float4(pos.x, pos.y, pos.z, pdf);
                  rec[1] = make_float4(ns.x, ns.y, ns.z, ps::lum(bv.f) * bv.cos_i);
                  rec[2] = make_float4(wo.x, wo.y, wo.z, io.guide.tag);
                  rec[3] = make_float4(wi.x, wi.y, wi.z, 0.f);
                  rec[4] = make_float4(Tn.x, Tn.y, Tn.z, 0.f);
                }
              }
            }
          }
        }
      }
      if (touched) io.radiance[path] = make_float4(L.x, L.y, L.z, L0.w);
    }
    uint32_t const slot = warp_append(emit_next, io.count_out);
    if (emit_next) {
      io.q_out[3 * size_t(slot)] = nq0;
      io.q_out[3 * size_t(slot) + 1] = nq1;
      io.q_out[3 * size_t(slot) + 2] = nq2;
    }
    uint32_t const sslot = warp_append(emit_shadow, io.count_shadow);
    if (emit_shadow) {
      io.shadow[3 * size_t(sslot)] = sq0;
      io.shadow[3 * size_t(sslot) + 1] = sq1;
      io.shadow[3 * size_t(sslot) + 2] = sq2;
    }
  }
}

// ---- shadow ------------------------------------------------------------------------------
template <bool SDF, int MINB = 8>
__global__ void __launch_bounds__(kPtBlock, MINB) k_pt_shadow(pt_wave w, int v, float4 const* __restrict__ sq,
    uint32_t const* __restrict__ count, float4* __restrict__ radiance, unsigned long long* __restrict__ stats) {
  uint32_t const n = *count;
  if (blockIdx.x == 0 && threadIdx.x == 0) stats[2] += n;
  uint32_t const stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    float4 const s0 = sq[3 * size_t(i)], s1 = sq[3 * size_t(i) + 1], s2 = sq[3 * size_t(i) + 2];
    pt_job const& J = w.jobs[__float_as_int(s2.w)];
    pt_scene const& s = w.scenes[J.scene];
    v3 const o = xyz(s0), d = xyz(s1);
    uint32_t const path = __float_as_uint(s0.w);
    hit_rec h;
    uint32_t cn = 0, ct = 0;
    bool occ = traverse<1, true, false>(s.nodes, s.tris, f3{o.x, o.y, o.z}, f3{d.x, d.y, d.z}, 0.f, s1.w, h, w.err,
        cn, ct);
    if (SDF && !occ && s.sdf.n_drawables > 0) {
      sdfk::sdf_dev const sd = job_sdf(s, J);
      rs::rng_t rng = sdf_stream(J, path, v);
      for (int k = 0; !occ && k < sd.n_drawables; ++k) occ = sdfk::march(sd, k, o, d, s1.w, true, &rng).hits;
    }
    if (!occ) {
      float4 const L = radiance[path];
      radiance[path] = make_float4(L.x + s2.x, L.y + s2.y, L.z + s2.z, L.w);
    }
  }
}

// ---- resolve ------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_pt_resolve(pt_job const* __restrict__ jobs, int j,
    float4 const* __restrict__ radiance) {
  pt_job const& J = jobs[j];
  uint32_t const pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= J.WH || J.rows == 0) return;
  float4 const* src = radiance + J.path_offset;
  if (J.fp64) {
    double4 a = J.overwrite ? make_double4(0., 0., 0., 0.) : J.accum64[pix];
    for (uint32_t r = 0; r < J.rows; ++r) {
      float4 const l = src[size_t(r) * J.WH + pix];
      if (isfinite(l.x) && isfinite(l.y) && isfinite(l.z)) {
        a.x = a.x + double(l.x);
        a.y = a.y + double(l.y);
        a.z = a.z + double(l.z);
      }
      a.w = a.w + 1.0;
    }
    J.accum64[pix] = a;
    J.display[pix] = make_float4(float(a.x / a.w), float(a.y / a.w), float(a.z / a.w), 1.f);
  } else {
    float4 a = J.overwrite ? make_float4(0.f, 0.f, 0.f, 0.f) : J.accum[pix];
    for (uint32_t r = 0; r < J.rows; ++r) {
      float4 const l = src[size_t(r) * J.WH + pix];
      if (isfinite(l.x) && isfinite(l.y) && isfinite(l.z)) {
        a.x = a.x + l.x;
        a.y = a.y + l.y;
        a.z = a.z + l.z;
      }
      a.w = a.w + 1.f;
    }
    J.accum[pix] = a;
    J.display[pix] = make_float4(a.x / a.w, a.y / a.w, a.z / a.w, 1.f);
  }
}

void mat_mul4(float const* a, float const* b, float* out) {
  for (int c = 0; c < 4; ++c)
    for (int r = 0; r < 4; ++r)
      out[c * 4 + r] = ((a[0 * 4 + r] * b[c * 4 + 0] + a[1 * 4 + r] * b[c * 4 + 1]) + a[2 * 4 + r] * b[c * 4 + 2]) +
          a[3 * 4 + r] * b[c * 4 + 3];
}

int ensure_queues(myrt_ctx* ctx, physical_state& P, size_t paths) {
  if (P.capacity >= paths && P.queue[0]) return MYRT_OK;
  for (void* p : {static_cast<void*>(P.queue[0]), static_cast<void*>(P.queue[1]), static_cast<void*>(P.hits),
           static_cast<void*>(P.shadow), static_cast<void*>(P.radiance), static_cast<void*>(P.counts),
           static_cast<void*>(P.okeys[0]), static_cast<void*>(P.okeys[1]), static_cast<void*>(P.ovals[0]),
           static_cast<void*>(P.ovals[1]), P.otemp})
    cudaFree(p);
  P.queue[0] = P.queue[1] = P.hits = P.shadow = P.radiance = nullptr;
  P.counts = nullptr;
  P.okeys[0] = P.okeys[1] = P.ovals[0] = P.ovals[1] = nullptr;
  P.otemp = nullptr;
  P.otemp_bytes = 0;
  P.capacity = 0;
  int rc = MYRT_OK;
  auto alloc = [&](void** p, size_t bytes, char const* what) {
    if (!rc) rc = check_cuda(ctx, cudaMalloc(p, bytes), what);
  };
  alloc(reinterpret_cast<void**>(&P.queue[0]), paths * 48, "path queue");
  alloc(reinterpret_cast<void**>(&P.queue[1]), paths * 48, "path queue");
  alloc(reinterpret_cast<void**>(&P.hits), paths * 48, "hit records");
  alloc(reinterpret_cast<void**>(&P.shadow), paths * 48, "shadow queue");
  alloc(reinterpret_cast<void**>(&P.radiance), paths * 16, "path radiance");
  alloc(reinterpret_cast<void**>(&P.counts), 4 * sizeof(uint32_t), "queue counts");
  for (int k = 0; k < 2; ++k) {  // visiting order of the extension queues
    alloc(reinterpret_cast<void**>(&P.okeys[k]), paths * 4, "queue order keys");
    alloc(reinterpret_cast<void**>(&P.ovals[k]), paths * 4, "queue order entries");
  }
  if (!rc)
    rc = check_cuda(ctx, cub::DeviceRadixSort::SortPairs(nullptr, P.otemp_bytes, P.okeys[0], P.okeys[1], P.ovals[0],
                             P.ovals[1], int(paths), 0, kOrderKeyBits, ctx->stream), "queue order size");
  alloc(&P.otemp, std::max<size_t>(P.otemp_bytes, 16), "queue order temporary");
  if (!rc && !P.stats) {
    alloc(reinterpret_cast<void**>(&P.stats), 4 * sizeof(unsigned long long), "ray statistics");
    if (!rc) rc = check_cuda(ctx, cudaMemsetAsync(P.stats, 0, 4 * sizeof(unsigned long long), ctx->stream), "clear");
  }
  if (rc) return rc;
  P.capacity = paths;
  return MYRT_OK;
}

pt_scene scene_of(myrt_ctx const* ctx) {
  device_scene const& S = ctx->scene;
  physical_state const& P = ctx->physical;
  pt_scene r{S.nodes, S.tris, S.tri_normals, S.tri_material, reinterpret_cast<int2 const*>(S.materials),
      int(S.n_materials), S.material_data, static_cast<ps::area_light const*>(P.lights), P.n_lights,
      sdfk::sdf_dev{ctx->sdf.instrs, ctx->sdf.programs, ctx->sdf.params, ctx->sdf.drawables, ctx->sdf.n_drawables,
          0, 0.f, ctx->sdf.skip_sphere, ctx->sdf.skip_next, ctx->sdf.cell_hdr, ctx->sdf.cell_start,
          ctx->sdf.cell_list, ctx->sdf.op_count},
      float3{0.f, 0.f, 0.f}, float3{0.f, 0.f, 0.f}};
  ray_key_grid(S.bounds, r.key_lo, r.key_scale);
  return r;
}

// A job's static description (camera, resolution, spp, ...); the wave planner
// fills sample_base / rows / path_offset / overwrite.
pt_job make_job(uint32_t scene, uint32_t W, uint32_t H, uint32_t seed, int max_depth, int rr_start, uint32_t fp64,
    myrt_camera const& cam, float const* env, int sdf_steps, float sdf_eps) {
  pt_job J{};
  J.W = W;
  J.H = H;
  J.WH = W * H;
  J.scene = scene;
  J.seed = seed;
  J.max_depth = max_depth > 0 ? max_depth : 8;
  J.rr_start = rr_start;
  J.fp64 = fp64;
  mat_mul4(cam.inverse_view, cam.inverse_projection, J.vp);
  J.eye[0] = cam.inverse_view[12];
  J.eye[1] = cam.inverse_view[13];
  J.eye[2] = cam.inverse_view[14];
  for (int k = 0; k < 3; ++k) J.env[k] = env[k];
  J.sdf_steps = sdf_steps;
  J.sdf_eps = sdf_eps;
  return J;
}

struct wave_plan {
  std::vector<pt_job> jobs;  // per job: rows / sample offset / path offset of this wave
  uint32_t n_paths = 0;
  int max_depth = 0;
};

// Packs each job's spp rows into waves of at most `target` paths (a job whose
// single row exceeds the target gets a wave of its own row by row). Rows keep
// their sample order within every job. sample_base holds the row index
// relative to the call's first sample.
std::vector<wave_plan> plan_waves(std::vector<pt_job> const& jobs, std::vector<uint32_t> const& spp, size_t target) {
  std::vector<wave_plan> out;
  std::vector<uint32_t> done(jobs.size(), 0);
  for (;;) {
    wave_plan w;
    w.jobs = jobs;
    size_t used = 0;
    bool any = false;
    for (size_t j = 0; j < jobs.size(); ++j) {
      pt_job& J = w.jobs[j];
      J.rows = 0;
      J.path_offset = uint32_t(used);
      J.sample_base = done[j];
      uint32_t const left = spp[j] - done[j];
      if (left == 0) continue;
      size_t const room = target > used ? (target - used) / J.WH : 0;
      uint32_t rows = uint32_t(std::min<size_t>(left, room));
      if (rows == 0 && used == 0) rows = 1;  // one row always fits an empty wave
      if (rows == 0) continue;
      J.rows = rows;
      done[j] += rows;
      used += size_t(rows) * J.WH;
      w.max_depth = std::max(w.max_depth, J.max_depth);
      any = true;
    }
    if (!any) break;
    w.n_paths = uint32_t(used);
    out.push_back(std::move(w));
  }
  return out;
}

// Waves of one job whose row counts double from 2^first_wave up to what
// `target` paths hold: a guide that is still learning trains after small
// early waves, and later waves run at full size.
std::vector<wave_plan> plan_waves_growing(pt_job const& J, uint32_t spp, size_t target, uint64_t first_wave) {
  std::vector<wave_plan> out;
  uint32_t const cap = uint32_t(std::max<size_t>(1, std::min<size_t>(target / J.WH, 1u << 30)));
  uint32_t done = 0;
  for (uint64_t k = first_wave; done < spp; ++k) {
    uint32_t const grow = k >= 30 ? cap : std::min<uint32_t>(cap, 1u << k);
    uint32_t const rows = std::min(spp - done, grow);
    wave_plan w;
    w.jobs = {J};
    w.jobs[0].rows = rows;
    w.jobs[0].path_offset = 0;
    w.jobs[0].sample_base = done;
    w.n_paths = rows * J.WH;
    w.max_depth = J.max_depth;
    done += rows;
    out.push_back(std::move(w));
  }
  return out;
}

// Launches every wave of a plan. `d_jobs` holds the plan's job tables
// (plan.size() * n_jobs pt_job, already on the device or copied first in
// the same stream). gd: guiding (single views only) or null.
int launch_plan(myrt_ctx* ctx, physical_state& P, cudaStream_t st, pt_scene const* d_scenes, pt_job const* d_jobs,
    std::vector<wave_plan> const& plan, int n_lights_max, bool any_sdf, guide_dev* gd) {
  uint32_t const bps = ctx->tuning.pt_blocks_per_sm ? ctx->tuning.pt_blocks_per_sm : 8u;
  uint32_t const grid = uint32_t(std::max(ctx->sm_count, 1)) * bps;
  size_t const nj = plan.empty() ? 0 : plan[0].jobs.size();
  for (size_t wi = 0; wi < plan.size(); ++wi) {
    wave_plan const& wp = plan[wi];
    pt_wave w{d_scenes, d_jobs + wi * nj, int(nj), wp.n_paths, ctx->d_err};
    // extend / shade / shadow: queue entries (at most the wave's paths) per thread
    bool const per_entry = ctx->tuning.pt_grid != 1;
    uint32_t const qgrid = per_entry
        ? std::max<uint32_t>(1u, uint32_t((uint64_t(wp.n_paths) + kPtBlock - 1) / kPtBlock))
        : grid;
    // one thread per entry: the traversal kernels' 10-blocks register cap unless pt_blocks_per_sm is 1..9
    bool const cap10 = per_entry && (ctx->tuning.pt_blocks_per_sm == 0 || ctx->tuning.pt_blocks_per_sm >= 10);
    if (gd) guide_begin_wave(ctx, *gd);
    k_pt_camera<<<grid, kPtBlock, 0, st>>>(w, P.queue[0], P.radiance, P.counts + 0);
    int cur = 0;
    for (int v = 0; v <= wp.max_depth; ++v) {
      bool const last = v == wp.max_depth;
      // visiting order (trace_order): the first bounces' queues (vertices 1 and 2), whose paths have
      // scattered, sorted by origin / direction cell in waves of at least 1 Mi paths (0); never (1);
      // every vertex after the camera's (2). Results never depend on it.
      uint32_t const order = ctx->tuning.trace_order;
      bool const sorted = per_entry && v >= 1 && wp.n_paths <= P.capacity &&
          (order == 2 || (order == 0 && v <= 2 && wp.n_paths >= (1u << 20)));
      uint32_t const* perm = nullptr;
      if (sorted) {
        k_pt_keys<<<(wp.n_paths + 255) / 256, 256, 0, st>>>(w, P.queue[cur], P.counts + cur, wp.n_paths, P.okeys[0],
            P.ovals[0]);
        size_t tb = P.otemp_bytes;
        int rc = check_cuda(ctx, cub::DeviceRadixSort::SortPairs(P.otemp, tb, P.okeys[0], P.okeys[1], P.ovals[0],
                                     P.ovals[1], int(wp.n_paths), 0, kOrderKeyBits, st), "queue order sort");
        if (rc) return rc;
        perm = P.ovals[1];
      }
      if (any_sdf)
        k_pt_extend<true><<<qgrid, kPtBlock, 0, st>>>(w, v, P.queue[cur], P.counts + cur, P.hits,
            P.counts + (1 - cur), P.counts + 2, P.stats, perm);
      else if (cap10)
        k_pt_extend<false, 10><<<qgrid, kPtBlock, 0, st>>>(w, v, P.queue[cur], P.counts + cur, P.hits,
            P.counts + (1 - cur), P.counts + 2, P.stats, perm);
      else
        k_pt_extend<false><<<qgrid, kPtBlock, 0, st>>>(w, v, P.queue[cur], P.counts + cur, P.hits,
            P.counts + (1 - cur), P.counts + 2, P.stats, perm);
      guide_dev gv = gd ? *gd : guide_dev{};
      if (last) gv.n_lobes = 0;
      if (gv.n_lobes > 0) {
        int rc = guide_infer(ctx, gv, 0, 0, P.queue[cur], P.hits, P.counts + cur, st);
        if (rc) return rc;
      }
      // shading in the same order appends the next queue and the shadow rays in that order too
      shade_io io{P.queue[cur], P.hits, P.counts + cur, P.queue[1 - cur], P.counts + (1 - cur), P.shadow,
          P.counts + 2, P.radiance, gv, perm};
      k_pt_shade<<<qgrid, kPtBlock, 0, st>>>(w, v, io);
      if (!last && n_lights_max > 0) {
        if (any_sdf) k_pt_shadow<true><<<qgrid, kPtBlock, 0, st>>>(w, v, P.shadow, P.counts + 2, P.radiance, P.stats);
        else if (cap10) k_pt_shadow<false, 10><<<qgrid, kPtBlock, 0, st>>>(w, v, P.shadow, P.counts + 2, P.radiance, P.stats);
        else k_pt_shadow<false><<<qgrid, kPtBlock, 0, st>>>(w, v, P.shadow, P.counts + 2, P.radiance, P.stats);
      }
      cur = 1 - cur;
    }
    for (size_t j = 0; j < nj; ++j) {
      if (wp.jobs[j].rows == 0) continue;
      uint32_t const rb = (wp.jobs[j].WH + 255) / 256;
      k_pt_resolve<<<rb, 256, 0, st>>>(d_jobs + wi * nj, int(j), P.radiance);
    }
    if (gd && gd->records) {
      int rc = guide_train(ctx, *gd, wp.n_paths, wp.max_depth, P.radiance, st);
      if (rc) return rc;
    }
    int rc = check_cuda(ctx, cudaGetLastError(), "physical wavefront launch");
    if (rc) return rc;
  }
  return MYRT_OK;
}

int grow_bytes(myrt_ctx* ctx, void** p, size_t& cap, size_t bytes, char const* what) {
  if (cap >= bytes && *p) return MYRT_OK;
  cudaFree(*p);
  *p = nullptr;
  cap = 0;
  int rc = check_cuda(ctx, cudaMalloc(p, bytes), what);
  if (!rc) cap = bytes;
  return rc;
}

}  // namespace

void free_physical(physical_state& P) {
  for (void* p : {static_cast<void*>(P.queue[0]), static_cast<void*>(P.queue[1]), static_cast<void*>(P.hits),
           static_cast<void*>(P.shadow), static_cast<void*>(P.radiance), static_cast<void*>(P.counts), P.lights,
           static_cast<void*>(P.stats), P.tables, static_cast<void*>(P.okeys[0]), static_cast<void*>(P.okeys[1]),
           static_cast<void*>(P.ovals[0]), static_cast<void*>(P.ovals[1]), P.otemp})
    cudaFree(p);
  P = physical_state{};
}

int get_render_stats(myrt_ctx* ctx, myrt_render_stats* out) {
  unsigned long long s[4] = {0, 0, 0, 0};
  if (ctx->physical.stats) {
    int rc = check_cuda(ctx, cudaMemcpyAsync(s, ctx->physical.stats, sizeof(s), cudaMemcpyDeviceToHost, ctx->stream),
        "read statistics");
    if (!rc) rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "read statistics");
    if (rc) return rc;
  }
  out->paths = s[0];
  out->extension_rays = s[1];
  out->shadow_rays = s[2];
  out->reserved = 0;
  return MYRT_OK;
}

int set_area_lights(myrt_ctx* ctx, myrt_area_light const* lights, uint32_t n) {
  if (n > uint32_t(kMaxLights)) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "at most 64 area lights");
  if (n && !lights) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "null lights");
  std::vector<ps::area_light> L(n);
  double total = 0.0;
  std::vector<double> power(n);
  for (uint32_t i = 0; i < n; ++i) {
    myrt_area_light const& a = lights[i];
    ps::area_light& l = L[i];
    std::memcpy(l.corner, a.corner, 12);
    std::memcpy(l.eu, a.edge_u, 12);
    std::memcpy(l.ev, a.edge_v, 12);
    std::memcpy(l.emission, a.emission, 12);
    // normal = cross(eu, ev) / |cross|; dual vectors du, dv with du.eu = 1,
    // du.ev = 0, dv.ev = 1, dv.eu = 0 (both orthogonal to the normal)
    double const u[3] = {a.edge_u[0], a.edge_u[1], a.edge_u[2]}, w[3] = {a.edge_v[0], a.edge_v[1], a.edge_v[2]};
    double c[3] = {u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]};
    double const area = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    if (!(area > 0.0) || !std::isfinite(area))
      return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "degenerate area light");
    double nn[3] = {c[0] / area, c[1] / area, c[2] / area};
    auto cross = [](double const* x, double const* y, double* o) {
      o[0] = x[1] * y[2] - x[2] * y[1];
      o[1] = x[2] * y[0] - x[0] * y[2];
      o[2] = x[0] * y[1] - x[1] * y[0];
    };
    double a1[3], b1[3];
    cross(w, nn, a1);  // orthogonal to ev and n
    cross(nn, u, b1);  // orthogonal to eu and n
    double const sa = a1[0] * u[0] + a1[1] * u[1] + a1[2] * u[2];
    double const sb = b1[0] * w[0] + b1[1] * w[1] + b1[2] * w[2];
    for (int k = 0; k < 3; ++k) {
      l.normal[k] = float(nn[k]);
      l.du[k] = float(a1[k] / sa);
      l.dv[k] = float(b1[k] / sb);
    }
    l.area = float(area);
    double const lum = 0.2126 * a.emission[0] + 0.7152 * a.emission[1] + 0.0722 * a.emission[2];
    if (!(lum >= 0.0)) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "negative light emission");
    power[i] = lum * area;
    total += power[i];
  }
  double run = 0.0;
  for (uint32_t i = 0; i < n; ++i) {
    double const p = total > 0.0 ? power[i] / total : 1.0 / n;
    run += p;
    L[i].prob = float(p);
    L[i].cdf = i + 1 == n ? 1.0f : float(run);
  }
  physical_state& P = ctx->physical;
  cudaFree(P.lights);
  P.lights = nullptr;
  P.n_lights = 0;
  if (n) {
    int rc = check_cuda(ctx, cudaMalloc(&P.lights, n * sizeof(ps::area_light)), "area lights");
    if (!rc)
      rc = check_cuda(ctx, cudaMemcpy(P.lights, L.data(), n * sizeof(ps::area_light), cudaMemcpyHostToDevice),
          "area lights upload");
    if (rc) return rc;
  }
  P.n_lights = int(n);
  ctx->render.sample_counter = 0;
  return MYRT_OK;
}

int render_physical_frames(myrt_ctx* ctx, myrt_camera const* cam, myrt_render_params const* p) {
  uint32_t const W = p->width, H = p->height;
  int rc = ensure_images(ctx, W, H);
  if (rc) return rc;
  render_state& R = ctx->render;
  physical_state& P = ctx->physical;
  size_t const WH = size_t(W) * H;
  uint32_t const spp = p->frames;
  if (p->accum_fp64 && !R.accum64) {
    rc = check_cuda(ctx, cudaMalloc(reinterpret_cast<void**>(&R.accum64), WH * sizeof(double4)), "FP64 image");
    if (rc) return rc;
  }
  bool const guided = p->shading == MYRT_SHADE_GUIDED;
  uint64_t trained = 0;
  bool training = false;
  if (guided) {
    rc = guide_schedule(ctx, &trained, &training);
    if (rc) return rc;
  }
  // default wave: 16 Mi paths (fewer, fuller launches at the late, sparse vertices: 439 -> 513 M
  // samples/s on a 512x512 64-spp frame against 4 Mi), 4 Mi while a guide is training, since it
  // trains after every wave
  size_t const target = p->wave_paths ? p->wave_paths
      : (ctx->tuning.wave_paths ? ctx->tuning.wave_paths : (guided && training ? 4u << 20 : 16u << 20));
  pt_job J = make_job(0, W, H, p->seed, p->max_depth, p->rr_start, p->accum_fp64, *cam, p->env_radiance,
      p->sdf_marching_steps, p->sdf_marching_epsilon);
  J.accum = R.accum;
  J.accum64 = R.accum64;
  J.display = R.display;
  std::vector<wave_plan> plan;
  if (guided && training) plan = plan_waves_growing(J, spp, target, trained);
  else plan = plan_waves({J}, {spp}, target);
  size_t max_paths = 0;
  for (auto& w : plan) {
    max_paths = std::max<size_t>(max_paths, w.n_paths);
    pt_job& jj = w.jobs[0];
    jj.overwrite = ((R.sample_counter == 0 || R.restart) && jj.sample_base == 0) ? 1u : 0u;
    jj.sample_base += R.sample_counter;
  }
  rc = ensure_queues(ctx, P, max_paths);
  if (rc) return rc;
  guide_dev gd{};
  if (guided) {
    rc = guide_prepare(ctx, max_paths, p, gd);
    if (rc) return rc;
  }
  // scene table (1) + job tables (one per wave)
  pt_scene const sc = scene_of(ctx);
  size_t const bytes = sizeof(pt_scene) + plan.size() * sizeof(pt_job);
  rc = grow_bytes(ctx, &P.tables, P.tables_cap, bytes, "wave tables");
  if (rc) return rc;
  std::vector<unsigned char> host(bytes);
  std::memcpy(host.data(), &sc, sizeof(pt_scene));
  for (size_t i = 0; i < plan.size(); ++i)
    std::memcpy(host.data() + sizeof(pt_scene) + i * sizeof(pt_job), &plan[i].jobs[0], sizeof(pt_job));
  cudaStream_t const st = ctx->stream;
  rc = check_cuda(ctx, cudaMemcpyAsync(P.tables, host.data(), bytes, cudaMemcpyHostToDevice, st), "wave tables");
  if (rc) return rc;
  auto* base = static_cast<unsigned char*>(P.tables);
  rc = launch_plan(ctx, P, st, reinterpret_cast<pt_scene const*>(base),
      reinterpret_cast<pt_job const*>(base + sizeof(pt_scene)), plan, P.n_lights, ctx->sdf.n_drawables > 0,
      guided ? &gd : nullptr);
  if (rc) return rc;
  R.sample_counter += spp;
  return MYRT_OK;
}

}  // namespace myrt_b200

// ==== batches: many jobs over many scenes, one CUDA graph per frame ===========================
using namespace myrt_b200;

struct myrt_batch {
  myrt_ctx* ctx = nullptr;  // scenes[0]: stream, tuning, error word
  std::vector<myrt_ctx*> scenes;
  std::vector<myrt_batch_job> jobs;
  std::vector<pt_job> base_jobs;  // static job descriptions with image pointers
  std::vector<wave_plan> plan;
  physical_state queues;          // the batch's own queues
  void* d_scenes = nullptr;
  void* d_jobs = nullptr;
  size_t d_jobs_cap = 0;
  pt_job* h_jobs = nullptr;       // pinned: per-wave job tables refreshed by each replay
  std::vector<void*> images;
  std::vector<uint32_t> samples;  // accumulated samples per job
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint32_t wave_paths = 0, blocks_per_sm = 0;
  int n_lights_max = 0;
  bool any_sdf = false;
};

namespace {

void drop_graph(myrt_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

// (Re)plans the waves for the current wave size and captures the frame graph.
int build_graph(myrt_batch* b) {
  myrt_ctx* ctx = b->ctx;
  drop_graph(b);
  size_t const target = b->wave_paths ? b->wave_paths : (ctx->tuning.wave_paths ? ctx->tuning.wave_paths : (4u << 20));
  std::vector<uint32_t> spp;
  for (auto const& j : b->jobs) spp.push_back(j.spp);
  b->plan = plan_waves(b->base_jobs, spp, target);
  size_t max_paths = 0;
  for (auto const& w : b->plan) max_paths = std::max<size_t>(max_paths, w.n_paths);
  int rc = ensure_queues(ctx, b->queues, max_paths);
  if (rc) return rc;
  size_t const nj = b->jobs.size();
  size_t const bytes = b->plan.size() * nj * sizeof(pt_job);
  if (b->d_jobs_cap < bytes) {
    cudaFree(b->d_jobs);
    cudaFreeHost(b->h_jobs);
    b->d_jobs = nullptr;
    b->h_jobs = nullptr;
    b->d_jobs_cap = 0;
    rc = check_cuda(ctx, cudaMalloc(&b->d_jobs, bytes), "batch job tables");
    if (!rc) rc = check_cuda(ctx, cudaMallocHost(reinterpret_cast<void**>(&b->h_jobs), bytes), "batch job tables");
    if (rc) return rc;
    b->d_jobs_cap = bytes;
  }
  for (size_t w = 0; w < b->plan.size(); ++w)
    std::memcpy(b->h_jobs + w * nj, b->plan[w].jobs.data(), nj * sizeof(pt_job));
  cudaStream_t const st = ctx->stream;
  rc = check_cuda(ctx, cudaStreamSynchronize(st), "batch graph");
  if (rc) return rc;
  myrt_tuning const saved = ctx->tuning;
  if (b->blocks_per_sm) ctx->tuning.pt_blocks_per_sm = b->blocks_per_sm;
  rc = check_cuda(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "graph capture");
  if (!rc) {
    cudaMemcpyAsync(b->d_jobs, b->h_jobs, bytes, cudaMemcpyHostToDevice, st);
    int lrc = launch_plan(ctx, b->queues, st, static_cast<pt_scene const*>(b->d_scenes),
        static_cast<pt_job const*>(b->d_jobs), b->plan, b->n_lights_max, b->any_sdf, nullptr);
    cudaError_t const e = cudaStreamEndCapture(st, &b->graph);
    rc = lrc ? lrc : check_cuda(ctx, e, "graph capture");
  }
  ctx->tuning = saved;
  if (!rc) rc = check_cuda(ctx, cudaGraphInstantiate(&b->exec, b->graph, 0), "graph instantiate");
  if (rc) drop_graph(b);
  return rc;
}

}  // namespace

extern "C" {

int myrt_batch_create(myrt_ctx* const* scenes, uint32_t n_scenes, myrt_batch_job const* jobs, uint32_t n_jobs,
    myrt_batch** out) {
  if (!scenes || !jobs || !out || n_scenes == 0 || n_jobs == 0 || n_jobs > 4096) return MYRT_ERR_INVALID_ARGUMENT;
  myrt_ctx* ctx = scenes[0];
  if (!ctx) return MYRT_ERR_INVALID_ARGUMENT;
  for (uint32_t i = 0; i < n_scenes; ++i) {
    if (!scenes[i] || scenes[i]->device != ctx->device)
      return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "batch scenes must be contexts on one device");
    if (!scenes[i]->scene.valid) return set_error(ctx, MYRT_ERR_NO_SCENE, "a batch scene has no uploaded scene");
  }
  for (uint32_t j = 0; j < n_jobs; ++j) {
    myrt_batch_job const& J = jobs[j];
    if (J.scene >= n_scenes || J.width == 0 || J.height == 0 || uint64_t(J.width) * J.height > (1u << 26) ||
        J.spp == 0 || J.spp > 65536 || J.max_depth < 0 || J.max_depth > 64 || J.rr_start < 0 || J.accum_fp64 > 1)
      return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "batch job out of range");
  }
  int rc = check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  if (rc) return rc;
  auto* b = new myrt_batch();
  b->ctx = ctx;
  b->scenes.assign(scenes, scenes + n_scenes);
  b->jobs.assign(jobs, jobs + n_jobs);
  std::vector<pt_scene> sc;
  for (auto* s : b->scenes) {
    sc.push_back(scene_of(s));
    b->n_lights_max = std::max(b->n_lights_max, s->physical.n_lights);
    b->any_sdf = b->any_sdf || s->sdf.n_drawables > 0;
  }
  rc = check_cuda(ctx, cudaMalloc(&b->d_scenes, sc.size() * sizeof(pt_scene)), "batch scene table");
  if (!rc)
    rc = check_cuda(ctx, cudaMemcpy(b->d_scenes, sc.data(), sc.size() * sizeof(pt_scene), cudaMemcpyHostToDevice),
        "batch scene table");
  for (uint32_t j = 0; !rc && j < n_jobs; ++j) {
    myrt_batch_job const& bj = jobs[j];
    size_t const WH = size_t(bj.width) * bj.height;
    void *acc = nullptr, *disp = nullptr;
    rc = check_cuda(ctx, cudaMalloc(&acc, WH * (bj.accum_fp64 ? 32 : 16)), "batch images");
    if (!rc) rc = check_cuda(ctx, cudaMalloc(&disp, WH * 16), "batch images");
    b->images.push_back(acc);
    b->images.push_back(disp);
    if (rc) break;
    pt_job J = make_job(bj.scene, bj.width, bj.height, bj.seed, bj.max_depth, bj.rr_start, bj.accum_fp64, bj.camera,
        bj.env_radiance, bj.sdf_marching_steps, bj.sdf_marching_epsilon);
    if (bj.accum_fp64) J.accum64 = static_cast<double4*>(acc);
    else J.accum = static_cast<float4*>(acc);
    J.display = static_cast<float4*>(disp);
    b->base_jobs.push_back(J);
  }
  b->samples.assign(n_jobs, 0);
  if (rc) {
    myrt_batch_destroy(b);
    return rc;
  }
  *out = b;
  return MYRT_OK;
}

int myrt_batch_set_tuning(myrt_batch* b, uint32_t wave_paths, uint32_t blocks_per_sm) {
  if (!b) return MYRT_ERR_INVALID_ARGUMENT;
  if ((wave_paths != 0 && wave_paths < 1024) || blocks_per_sm > 16)
    return set_error(b->ctx, MYRT_ERR_INVALID_ARGUMENT, "batch tuning out of range");
  b->wave_paths = wave_paths;
  b->blocks_per_sm = blocks_per_sm;
  drop_graph(b);
  return MYRT_OK;
}

int myrt_batch_render(myrt_batch* b) {
  if (!b) return MYRT_ERR_INVALID_ARGUMENT;
  myrt_ctx* ctx = b->ctx;
  int rc = check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  if (!rc && !b->exec) rc = build_graph(b);
  if (rc) return rc;
  // the previous replay must have consumed the pinned tables before they change
  rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "batch render");
  if (rc) return rc;
  size_t const nj = b->jobs.size();
  for (size_t w = 0; w < b->plan.size(); ++w)
    for (size_t j = 0; j < nj; ++j) {
      pt_job& J = b->h_jobs[w * nj + j];
      uint32_t const row = b->plan[w].jobs[j].sample_base;  // row index within the frame
      J.sample_base = b->samples[j] + row;
      J.overwrite = (b->samples[j] == 0 && row == 0) ? 1u : 0u;
    }
  rc = check_cuda(ctx, cudaGraphLaunch(b->exec, ctx->stream), "batch graph launch");
  if (rc) return rc;
  for (size_t j = 0; j < nj; ++j) b->samples[j] += b->jobs[j].spp;
  return MYRT_OK;
}

int myrt_batch_read(myrt_batch* b, uint32_t job, float* rgba, double* rgba64) {
  if (!b || job >= b->jobs.size()) return MYRT_ERR_INVALID_ARGUMENT;
  myrt_ctx* ctx = b->ctx;
  myrt_batch_job const& bj = b->jobs[job];
  size_t const WH = size_t(bj.width) * bj.height;
  if (b->samples[job] == 0) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "nothing rendered yet");
  int rc = MYRT_OK;
  if (rgba64) {
    if (!bj.accum_fp64) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "job has no FP64 accumulation");
    rc = check_cuda(ctx, cudaMemcpyAsync(rgba64, b->images[2 * job], WH * 32, cudaMemcpyDeviceToHost, ctx->stream),
        "read");
  }
  if (!rc && rgba) {
    void const* src = bj.accum_fp64 ? b->images[2 * job + 1] : b->images[2 * job];
    rc = check_cuda(ctx, cudaMemcpyAsync(rgba, src, WH * 16, cudaMemcpyDeviceToHost, ctx->stream), "read");
  }
  if (!rc) rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "read");
  return rc;
}

int myrt_batch_reset(myrt_batch* b) {
  if (!b) return MYRT_ERR_INVALID_ARGUMENT;
  std::fill(b->samples.begin(), b->samples.end(), 0u);
  return MYRT_OK;
}

int myrt_batch_get_stats(myrt_batch* b, myrt_render_stats* out) {
  if (!b || !out) return MYRT_ERR_INVALID_ARGUMENT;
  myrt_ctx* ctx = b->ctx;
  unsigned long long s[4] = {0, 0, 0, 0};
  if (b->queues.stats) {
    int rc = check_cuda(ctx, cudaMemcpyAsync(s, b->queues.stats, sizeof(s), cudaMemcpyDeviceToHost, ctx->stream),
        "read batch statistics");
    if (!rc) rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "read batch statistics");
    if (rc) return rc;
  }
  out->paths = s[0];
  out->extension_rays = s[1];
  out->shadow_rays = s[2];
  out->reserved = 0;
  return MYRT_OK;
}

int myrt_batch_get_info(myrt_batch* b, myrt_batch_info* info) {
  if (!b || !info) return MYRT_ERR_INVALID_ARGUMENT;
  int rc = MYRT_OK;
  if (!b->exec) rc = build_graph(b);
  if (rc) return rc;
  std::memset(info, 0, sizeof(*info));
  info->waves = uint32_t(b->plan.size());
  uint64_t total = 0;
  uint32_t mx = 0;
  for (auto const& w : b->plan) {
    total += w.n_paths;
    mx = std::max(mx, w.n_paths);
  }
  info->paths_per_frame = total;
  info->max_wave_paths = mx;
  size_t nodes = 0;
  if (b->graph) cudaGraphGetNodes(b->graph, nullptr, &nodes);
  info->graph_nodes = uint32_t(nodes);
  info->wave_paths = b->wave_paths;
  info->blocks_per_sm = b->blocks_per_sm;
  return MYRT_OK;
}

int myrt_batch_destroy(myrt_batch* b) {
  if (!b) return MYRT_ERR_INVALID_ARGUMENT;
  cudaSetDevice(b->ctx->device);
  cudaStreamSynchronize(b->ctx->stream);
  drop_graph(b);
  free_physical(b->queues);
  cudaFree(b->d_scenes);
  cudaFree(b->d_jobs);
  cudaFreeHost(b->h_jobs);
  for (void* p : b->images) cudaFree(p);
  delete b;
  return MYRT_OK;
}

}  // extern "C"
