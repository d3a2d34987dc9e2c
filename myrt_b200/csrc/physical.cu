// Physical and guided wavefront path tracing.
//
// One call renders `spp` samples per pixel in waves of k full-image sample
// rows (k * W * H paths). Per wave:
//
//   k_pt_camera                 camera rays (box-filtered pixel jitter)
//   for vertex v = 0 .. max_depth:
//     k_pt_extend               closest hit: 8-wide BVH (watertight), SDF
//                               drawables (sphere tracing), area lights
//     [guided: k_guide_features + the MLP forward (guide.cu)]
//     k_pt_shade                emission with MIS, NEE toward one light,
//                               BSDF (or guide) sampling, Russian roulette;
//                               survivors and shadow rays are appended to
//                               the next queues with warp-aggregated atomics
//     k_pt_shadow               any-hit for the NEE rays, adds unoccluded
//                               contributions
//   k_pt_resolve                per pixel, the wave's samples in sample order
//                               into the FP32 or FP64 accumulation
//
// Queue order never reaches the result: each path's random numbers are keyed
// by (pixel, sample, seed) and each path's radiance is summed in event order
// in its own slot, so the image equals a path-at-a-time render bit for bit.
// Compiled with -fmad=false (build.py) like the other shading unit.
#include <cuda_runtime.h>

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
  sdfk::sdf_dev sdf;
  uint32_t* err;
  float env[3];
};

struct pt_frame {
  uint32_t W, H, WH;
  uint32_t sample_base;  // sample index of the wave's first row
  uint32_t seed;
  int max_depth, rr_start;
  float vp[16];
  float eye[3];
};

__device__ __forceinline__ v3 xyz(float4 a) { return {a.x, a.y, a.z}; }

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
__global__ void __launch_bounds__(kPtBlock) k_pt_camera(pt_frame f, uint32_t n, float4* __restrict__ q,
    float4* __restrict__ radiance, uint32_t* __restrict__ count) {
  uint32_t const stride = gridDim.x * blockDim.x;
  if (blockIdx.x == 0 && threadIdx.x == 0) *count = n;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    uint32_t const pix = i % f.WH, sample = f.sample_base + i / f.WH;
    uint32_t const x = pix % f.W, y = pix / f.W;
    ps::rnd4 const r = ps::rand4(pix, sample, f.seed, 0xffffu);
    float const nx = ((r.a + float(x)) / float(f.W)) * 2.f - 1.f;
    float const ny = ((r.b + float(y)) / float(f.H)) * 2.f - 1.f;
    float h[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) h[k] = ((f.vp[0 * 4 + k] * nx + f.vp[1 * 4 + k] * ny) + f.vp[2 * 4 + k]) + f.vp[3 * 4 + k];
    v3 const d = rs::normalize(v3{h[0], h[1], h[2]});
    q[3 * size_t(i)] = make_float4(f.eye[0], f.eye[1], f.eye[2], __uint_as_float(i));
    q[3 * size_t(i) + 1] = make_float4(d.x, d.y, d.z, 0.f);
    q[3 * size_t(i) + 2] = make_float4(1.f, 1.f, 1.f, 0.f);
    radiance[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

__device__ __forceinline__ rs::rng_t sdf_stream(pt_frame const& f, uint32_t path, int v) {
  uint32_t const pix = path % f.WH, sample = f.sample_base + path / f.WH;
  rs::rng_t r;
  r.state = ps::pcg4d(pix, sample, f.seed, 4u * uint32_t(v) + 2u).x;
  r.prime = 0;
  r.tex = nullptr;
  return r;
}

// ---- extend: closest hit over meshes, SDF drawables and lights ---------------------------
// hits[3i] = (position, kind): kind >= 0 material index, -1 miss, -2 - l light l;
// hits[3i+1] = (shading normal, t); hits[3i+2] = (geometric normal, 0).
__global__ void __launch_bounds__(kPtBlock, 8) k_pt_extend(pt_scene s, pt_frame f, int v, float4 const* __restrict__ q,
    uint32_t const* __restrict__ count, float4* __restrict__ hits, uint32_t* __restrict__ clear_a,
    uint32_t* __restrict__ clear_b, unsigned long long* __restrict__ stats) {
  uint32_t const n = *count;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *clear_a = 0;
    *clear_b = 0;
    stats[1] += n;
    if (v == 0) stats[0] += n;
  }
  uint32_t const stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    float4 const q0 = q[3 * size_t(i)], q1 = q[3 * size_t(i) + 1];
    v3 const o = xyz(q0), d = xyz(q1);
    hit_rec h;
    uint32_t cn = 0, ct = 0;
    bool const hit =
        traverse<1, false, false>(s.nodes, s.tris, f3{o.x, o.y, o.z}, f3{d.x, d.y, d.z}, 0.f, kInf, h, s.err, cn, ct);
    float t = hit ? h.t : kInf;
    int kind = -1;
    v3 pos{0.f, 0.f, 0.f}, ns{0.f, 0.f, 0.f}, ng{0.f, 0.f, 0.f};
    if (hit) {
      float4 const* tp = s.tris + 3 * size_t(h.leaf);
      v3 const p0 = xyz(__ldg(tp)), p1 = xyz(__ldg(tp + 1)), p2 = xyz(__ldg(tp + 2));
      float const w = (1.f - h.u) - h.v;
      pos = (h.u * p1 + h.v * p2) + w * p0;
      ng = rs::normalize(rs::cross(p1 - p0, p2 - p0));
      uint32_t const prim = uint32_t(h.prim);
      if (s.tri_normals) {
        float4 const* np = s.tri_normals + 3 * size_t(prim);
        ns = rs::normalize((h.u * xyz(__ldg(np + 1)) + h.v * xyz(__ldg(np + 2))) + w * xyz(__ldg(np)));
      } else {
        ns = ng;
      }
      kind = __ldg(s.tri_material + prim);
    }
    if (s.sdf.n_drawables > 0) {
      rs::rng_t rng = sdf_stream(f, __float_as_uint(q0.w), v);
      for (int k = 0; k < s.sdf.n_drawables; ++k) {
        sdfk::sdf_hit const sh = sdfk::march(s.sdf, k, o, d, t, false, &rng);
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
};

__global__ void __launch_bounds__(kPtBlock) k_pt_shade(pt_scene s, pt_frame f, int v, shade_io io) {
  uint32_t const n = *io.count;
  uint32_t const stride = gridDim.x * blockDim.x;
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += stride) {  // warp-uniform trip count
    uint32_t const i = base + threadIdx.x;
    bool const active = i < n;
    bool emit_next = false, emit_shadow = false;
    float4 nq0, nq1, nq2, sq0, sq1, sq2;
    if (active) {
      float4 const q0 = io.q[3 * size_t(i)], q1 = io.q[3 * size_t(i) + 1], q2 = io.q[3 * size_t(i) + 2];
      float4 const h0 = io.hits[3 * size_t(i)], h1 = io.hits[3 * size_t(i) + 1], h2 = io.hits[3 * size_t(i) + 2];
      uint32_t const path = __float_as_uint(q0.w);
      v3 const d = xyz(q1), T = xyz(q2);
      float const prev_pdf = q1.w;
      int const kind = __float_as_int(h0.w);
      float4 const L0 = io.radiance[path];
      v3 L = xyz(L0);
      bool touched = false;
      if (io.guide.records && v > 0) guide_record_at(io.guide, path, v - 1)[5] = L0;
      if (kind == -1) {
        v3 const env{s.env[0], s.env[1], s.env[2]};
        L = L + T * env;
        touched = true;
      } else if (kind <= -2) {
        ps::area_light const& lt = s.lights[-2 - kind];
        float const cos_l = -rs::dot(d, ps::lv(lt.normal));
        if (cos_l > 0.f) {
          float w = 1.f;
          if (v > 0 && prev_pdf > 0.f) {
            float const t = h1.w;
            float const pl = (lt.prob * (t * t)) / (lt.area * cos_l);
            w = ps::power_heuristic(prev_pdf, pl);
          }
          L = L + (T * ps::lv(lt.emission)) * w;
          touched = true;
        }
      } else if (v < f.max_depth) {
        bool ok = kind < s.n_mats;
        int2 mref{0, 0};
        if (ok) mref = __ldg(s.mat_refs + kind);
        if (!ok || mref.x != 0) {
          atomicOr(s.err, ERR_BAD_MATERIAL);
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
          uint32_t const pix = path % f.WH, sample = f.sample_base + path / f.WH;
          ps::rnd4 const r0 = ps::rand4(pix, sample, f.seed, 4u * uint32_t(v));
          ps::rnd4 const r1 = ps::rand4(pix, sample, f.seed, 4u * uint32_t(v) + 1u);
          v3 const org = pos + ng * kOffset;
          guide_lobes gl;
          bool const guided = io.guide.n_lobes > 0 && guide_load(io.guide, i, gl) && io.guide.fraction > 0.f;
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
                float const w = ps::power_heuristic(pl, pb);
                v3 const c = ((T * bv.f) * ps::lv(lt.emission)) * ((bv.cos_i * w) / pl);
                if (ps::max3(c) > 0.f) {
                  emit_shadow = true;
                  sq0 = make_float4(org.x, org.y, org.z, __uint_as_float(path));
                  sq1 = make_float4(wi.x, wi.y, wi.z, dist * 0.999f);
                  sq2 = make_float4(c.x, c.y, c.z, 0.f);
                }
              }
            }
          }
          // continuation
          v3 wi;
          bool sampled;
          if (guided && r1.d < io.guide.fraction) {
            ps::rnd4 const r3 = ps::rand4(pix, sample, f.seed, 4u * uint32_t(v) + 3u);
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
              if (alive && v >= f.rr_start) {
                float const qq = fminf(ps::max3(Tn), 0.95f);
                if (r0.d >= qq) alive = false;
                else Tn = Tn / qq;
              }
              if (alive) {
                emit_next = true;
                nq0 = make_float4(org.x, org.y, org.z, __uint_as_float(path));
                nq1 = make_float4(wi.x, wi.y, wi.z, pdf);
                nq2 = make_float4(Tn.x, Tn.y, Tn.z, 0.f);
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
      if (touched) io.radiance[path] = make_float4(L.x, L.y, L.z, 0.f);
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
__global__ void __launch_bounds__(kPtBlock, 8) k_pt_shadow(pt_scene s, pt_frame f, int v,
    float4 const* __restrict__ sq, uint32_t const* __restrict__ count, float4* __restrict__ radiance,
    unsigned long long* __restrict__ stats) {
  uint32_t const n = *count;
  if (blockIdx.x == 0 && threadIdx.x == 0) stats[2] += n;
  uint32_t const stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    float4 const s0 = sq[3 * size_t(i)], s1 = sq[3 * size_t(i) + 1], s2 = sq[3 * size_t(i) + 2];
    v3 const o = xyz(s0), d = xyz(s1);
    uint32_t const path = __float_as_uint(s0.w);
    hit_rec h;
    uint32_t cn = 0, ct = 0;
    bool occ = traverse<1, true, false>(s.nodes, s.tris, f3{o.x, o.y, o.z}, f3{d.x, d.y, d.z}, 0.f, s1.w, h, s.err,
        cn, ct);
    if (!occ && s.sdf.n_drawables > 0) {
      rs::rng_t rng = sdf_stream(f, path, v);
      for (int k = 0; !occ && k < s.sdf.n_drawables; ++k) occ = sdfk::march(s.sdf, k, o, d, s1.w, true, &rng).hits;
    }
    if (!occ) {
      float4 const L = radiance[path];
      radiance[path] = make_float4(L.x + s2.x, L.y + s2.y, L.z + s2.z, 0.f);
    }
  }
}

// ---- resolve ------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_pt_resolve(uint32_t WH, uint32_t rows, float4 const* __restrict__ radiance,
    int overwrite, float4* __restrict__ accum, float4* __restrict__ display) {
  uint32_t const pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= WH) return;
  float4 a = overwrite ? make_float4(0.f, 0.f, 0.f, 0.f) : accum[pix];
  for (uint32_t j = 0; j < rows; ++j) {
    float4 const l = radiance[size_t(j) * WH + pix];
    if (isfinite(l.x) && isfinite(l.y) && isfinite(l.z)) {
      a.x = a.x + l.x;
      a.y = a.y + l.y;
      a.z = a.z + l.z;
    }
    a.w = a.w + 1.f;
  }
  accum[pix] = a;
  display[pix] = make_float4(a.x / a.w, a.y / a.w, a.z / a.w, 1.f);
}

__global__ void __launch_bounds__(256) k_pt_resolve64(uint32_t WH, uint32_t rows, float4 const* __restrict__ radiance,
    int overwrite, double4* __restrict__ accum, float4* __restrict__ display) {
  uint32_t const pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= WH) return;
  double4 a = overwrite ? make_double4(0., 0., 0., 0.) : accum[pix];
  for (uint32_t j = 0; j < rows; ++j) {
    float4 const l = radiance[size_t(j) * WH + pix];
    if (isfinite(l.x) && isfinite(l.y) && isfinite(l.z)) {
      a.x = a.x + double(l.x);
      a.y = a.y + double(l.y);
      a.z = a.z + double(l.z);
    }
    a.w = a.w + 1.0;
  }
  accum[pix] = a;
  display[pix] = make_float4(float(a.x / a.w), float(a.y / a.w), float(a.z / a.w), 1.f);
}

void mat_mul4(float const* a, float const* b, float* out) {
  for (int c = 0; c < 4; ++c)
    for (int r = 0; r < 4; ++r)
      out[c * 4 + r] = ((a[0 * 4 + r] * b[c * 4 + 0] + a[1 * 4 + r] * b[c * 4 + 1]) + a[2 * 4 + r] * b[c * 4 + 2]) +
          a[3 * 4 + r] * b[c * 4 + 3];
}

int ensure_queues(myrt_ctx* ctx, size_t paths) {
  physical_state& P = ctx->physical;
  if (P.capacity >= paths && P.queue[0]) return MYRT_OK;
  for (void* p : {static_cast<void*>(P.queue[0]), static_cast<void*>(P.queue[1]), static_cast<void*>(P.hits),
           static_cast<void*>(P.shadow), static_cast<void*>(P.radiance), static_cast<void*>(P.counts)})
    cudaFree(p);
  P.queue[0] = P.queue[1] = P.hits = P.shadow = P.radiance = nullptr;
  P.counts = nullptr;
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
  if (!rc && !P.stats) {
    alloc(reinterpret_cast<void**>(&P.stats), 4 * sizeof(unsigned long long), "ray statistics");
    if (!rc) rc = check_cuda(ctx, cudaMemsetAsync(P.stats, 0, 4 * sizeof(unsigned long long), ctx->stream), "clear");
  }
  if (rc) return rc;
  P.capacity = paths;
  return MYRT_OK;
}

}  // namespace

void free_physical(physical_state& P) {
  for (void* p : {static_cast<void*>(P.queue[0]), static_cast<void*>(P.queue[1]), static_cast<void*>(P.hits),
           static_cast<void*>(P.shadow), static_cast<void*>(P.radiance), static_cast<void*>(P.counts), P.lights,
           static_cast<void*>(P.stats)})
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
  device_scene const& S = ctx->scene;
  size_t const WH = size_t(W) * H;
  uint32_t const spp = p->frames;
  if (p->accum_fp64 && !R.accum64) {
    rc = check_cuda(ctx, cudaMalloc(reinterpret_cast<void**>(&R.accum64), WH * sizeof(double4)), "FP64 image");
    if (rc) return rc;
  }
  size_t const target = p->wave_paths ? p->wave_paths : (ctx->tuning.wave_paths ? ctx->tuning.wave_paths : (4u << 20));
  uint32_t const rows_per_wave = uint32_t(std::max<size_t>(1, std::min<size_t>(spp, target / WH)));
  rc = ensure_queues(ctx, size_t(rows_per_wave) * WH);
  if (rc) return rc;
  guide_dev gd{};
  if (p->shading == MYRT_SHADE_GUIDED) {
    rc = guide_prepare(ctx, size_t(rows_per_wave) * WH, p, gd);
    if (rc) return rc;
  }

  pt_scene sc{S.nodes, S.tris, S.tri_normals, S.tri_material, reinterpret_cast<int2 const*>(S.materials),
      int(S.n_materials), S.material_data, static_cast<ps::area_light const*>(P.lights), P.n_lights,
      sdfk::sdf_dev{ctx->sdf.instrs, ctx->sdf.programs, ctx->sdf.params, ctx->sdf.drawables, ctx->sdf.n_drawables,
          p->sdf_marching_steps, p->sdf_marching_epsilon},
      ctx->d_err, {p->env_radiance[0], p->env_radiance[1], p->env_radiance[2]}};
  pt_frame fr{};
  fr.W = W;
  fr.H = H;
  fr.WH = uint32_t(WH);
  fr.seed = p->seed;
  fr.max_depth = p->max_depth > 0 ? p->max_depth : 8;
  fr.rr_start = p->rr_start;
  mat_mul4(cam->inverse_view, cam->inverse_projection, fr.vp);
  fr.eye[0] = cam->inverse_view[12];
  fr.eye[1] = cam->inverse_view[13];
  fr.eye[2] = cam->inverse_view[14];

  cudaStream_t const st = ctx->stream;
  uint32_t const bps = ctx->tuning.pt_blocks_per_sm ? ctx->tuning.pt_blocks_per_sm : 8u;
  uint32_t const grid = uint32_t(std::max(ctx->sm_count, 1)) * bps;
  for (uint32_t s0 = 0; s0 < spp; s0 += rows_per_wave) {
    uint32_t const rows = std::min(rows_per_wave, spp - s0);
    uint32_t const n = uint32_t(rows * WH);
    fr.sample_base = R.sample_counter + s0;
    if (p->shading == MYRT_SHADE_GUIDED) guide_begin_wave(ctx, gd);
    k_pt_camera<<<grid, kPtBlock, 0, st>>>(fr, n, P.queue[0], P.radiance, P.counts + 0);
    int cur = 0;
    for (int v = 0; v <= fr.max_depth; ++v) {
      bool const last = v == fr.max_depth;
      k_pt_extend<<<grid, kPtBlock, 0, st>>>(sc, fr, v, P.queue[cur], P.counts + cur, P.hits, P.counts + (1 - cur),
          P.counts + 2, P.stats);
      guide_dev gv = gd;
      if (last) gv.n_lobes = 0;
      shade_io io{P.queue[cur], P.hits, P.counts + cur, P.queue[1 - cur], P.counts + (1 - cur), P.shadow,
          P.counts + 2, P.radiance, gv};
      if (gv.n_lobes > 0) {
        rc = guide_infer(ctx, gd, fr.WH, fr.sample_base, P.queue[cur], P.hits, P.counts + cur, st);
        if (rc) return rc;
      }
      k_pt_shade<<<grid, kPtBlock, 0, st>>>(sc, fr, v, io);
      if (!last && P.n_lights > 0)
        k_pt_shadow<<<grid, kPtBlock, 0, st>>>(sc, fr, v, P.shadow, P.counts + 2, P.radiance, P.stats);
      cur = 1 - cur;
    }
    int const overwrite = (R.sample_counter == 0 && s0 == 0) ? 1 : 0;
    uint32_t const rb = uint32_t((WH + 255) / 256);
    if (p->accum_fp64)
      k_pt_resolve64<<<rb, 256, 0, st>>>(fr.WH, rows, P.radiance, overwrite, R.accum64, R.display);
    else
      k_pt_resolve<<<rb, 256, 0, st>>>(fr.WH, rows, P.radiance, overwrite, R.accum, R.display);
    if (gd.records) {
      rc = guide_train(ctx, gd, n, fr.max_depth, P.radiance, st);
      if (rc) return rc;
    }
    rc = check_cuda(ctx, cudaGetLastError(), "physical wavefront launch");
    if (rc) return rc;
  }
  R.sample_counter += spp;
  return MYRT_OK;
}

}  // namespace myrt_b200
