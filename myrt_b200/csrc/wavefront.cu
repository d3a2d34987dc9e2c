// Wavefront path tracing, "reference shading" mode: the reference's
// generate -> {trace, color, filter} x bounces -> trace, color frame
// (src/pathtracer/sequential_pathtracer.cpp:10-69, :282-498) as sm_100a kernels.
//
//   k_generate     pt_generate.comp:50-84
//   k_trace_pass   pt_trace.comp:134-226, nearest_hit :331-386 (meshes), any_hit
//                  :311-329 for the NEE shadow ray; both walk the 8-wide BVH
//   k_shadow_pass  that any_hit for mesh-only scenes, over the queue of shadow
//                  rays k_trace_pass leaves, so that every lane walks one
//   k_color_pass   pt_color.comp:77-202 (sky gradient, no cubemap), plus a
//                  per-block count of surviving rays for the compaction
//   k_gen_keys     visiting order of the first two trace passes (ray_key)
//   k_resolve_frames  the frames in flight into the accumulation, in order
//   k_scan_blocks + k_scatter
//                  pt_ray_filter.comp:49-64 as a STABLE compaction: survivors
//                  keep their relative order, so slot ids (which feed the
//                  random stream, pt_color.comp:134-135) are reproducible
//
// Ray state keeps the reference's record layouts: generate_output_t = 80 bytes
// (five float4), trace_output_t = 64 bytes (four float4). The per-pass host
// randomness (an int seed and a 1024-float texture per pass, drawn from
// std::mt19937 in the reference's order) is generated for all frames of a
// call up front and copied to the device once.
//
// Frames in flight: the reference renders a call's frames one after another,
// each pass over one image of rays. Here up to kMaxFramesInFlight frames of a
// call run their passes together (about 16 Mi rays per launch instead of one
// image's), each in its own region of ray slots with its own ray counts,
// compaction, pass randomness and slot ids, so every ray sees exactly what it
// would see alone. A path's final colour is kept per frame and pixel, and
// k_resolve_frames then accumulates the frames in their order, pixel by pixel:
// the images equal the sequential ones bit for bit.
//
// Compiled with -fmad=false (see build.py): the shading arithmetic rounds every
// operation as written, like the CPU oracle.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <random>
#include <vector>

#include <cub/device/device_radix_sort.cuh>

#include "../../include/myrt_cuda.h"
#include "ctx.hpp"
#include "rayorder.cuh"
#include "refshade.cuh"
#include "sdf.cuh"
#include "trace.cuh"

namespace myrt_b200 {
namespace {

using rs::v2;
using rs::v3;

constexpr int kBlock = 256;
constexpr int kTexSize = 1024;
constexpr int kMaxFramesInFlight = 64;

// One pass's randomness for every frame in flight: frame f's texture at
// tex + f * tex_stride, its seed in seed[f].
struct pass_rand {
  float const* tex;
  uint32_t tex_stride;  // floats
  int seed[kMaxFramesInFlight];
};

// Frame and slot of this thread when each frame in flight owns `nb`
// consecutive blocks (its region of ray slots).
struct frame_slot {
  uint32_t f, id;
};
__device__ __forceinline__ frame_slot frame_of(uint32_t nb) {
  uint32_t const f = blockIdx.x / nb;
  return {f, (blockIdx.x - f * nb) * blockDim.x + threadIdx.x};
}

struct scene_dev {
  uint4 const* nodes;
  float4 const* tris;
  float4 const* tri_normals;  // 3 per prim, may be null
  float2 const* tri_uvs;      // 3 per prim, may be null
  int32_t const* tri_material;
  int2 const* mat_refs;  // (id, offset)
  int n_mats;
  float const* mat_data;
  uint32_t* err;
  sdfk::sdf_dev sdf;  // n_drawables == 0: no SDF drawables
};

sdfk::sdf_dev make_sdf_dev(myrt_ctx const* ctx, int steps, float eps) {
  device_sdf const& D = ctx->sdf;
  return sdfk::sdf_dev{D.instrs, D.programs, D.params, D.drawables, D.n_drawables, steps, eps, D.skip_sphere,
      D.skip_next, D.cell_hdr, D.cell_start, D.cell_list, D.op_count};
}

struct camera_dev {
  float vp[16];  // inverse_view * inverse_projection (column major), computed on the host
  float eye[3];
  int dof;       // pt_generate.comp dof_active
  float lens[2], focus;
  rs::tex2d bokeh;  // bokeh_shape; p = null (or width < 10) = no mask
};

struct light_t {
  float px, py, pz, r, cx, cy, cz;
};
// pt_trace.comp:141-146 (float products, as the GLSL folds them)
__constant__ light_t c_lights[2] = {
    {2.f * 4.f, 2.f * 5.f, 2.f * 4.f, 1.5f, 6.f * 1.f, 6.f * 1.8f, 6.f * 3.f},
    {2.f * -4.f, 2.f * 3.f, 2.f * 5.f, 1.5f, 8.f * 3.f, 8.f * 1.8f, 8.f * 1.f},
};

__device__ __forceinline__ v3 xyz(float4 a) { return {a.x, a.y, a.z}; }

// intersect.glsl:30-39
__device__ __forceinline__ float intersect_sphere(v3 r0, v3 rd, v3 s0, float sr) {
  float const a = rs::dot(rd, rd);
  v3 const s0_r0 = r0 - s0;
  float const b = 2.f * rs::dot(rd, s0_r0);
  float const c = rs::dot(s0_r0, s0_r0) - (sr * sr);
  if (b * b - 4.f * a * c < 0.f) return -1.f;
  return (-b - sqrtf((b * b) - 4.f * a * c)) / (2.f * a);
}

// ---- pt_generate.comp -----------------------------------------------------------
// gen: the frames' regions of W * H slots; count[f] = W * H.
__global__ void __launch_bounds__(kBlock) k_generate(uint32_t W, uint32_t H, uint32_t nb, pass_rand pr,
    camera_dev cam, float4* __restrict__ gen, uint32_t* __restrict__ count) {
  frame_slot const fs = frame_of(nb);
  uint32_t const id = fs.id;
  float const* const tex = pr.tex + fs.f * pr.tex_stride;
  int const seed = pr.seed[fs.f];
  gen += 5 * size_t(fs.f) * W * H;
  if (id == 0) count[fs.f] = W * H;
  if (id >= W * H) return;
  int const x = int(id % W), y = int(id / W);
  rs::rng_t r;
  rs::random_init(r, tex, x, y, seed);
  // random_uniform_circle(0.7071067812) (random.glsl:77-85)
  float const a = rs::random_next(r) * 2.f * 3.1415926535897f;
  float const b = rs::random_next(r);
  float const s = sqrtf(b) * 0.7071067812f;
  v2 const off{s * myrt_glmath::sin(a), s * myrt_glmath::cos(a)};
  float const nx = ((off.x + float(x)) / float(W)) * 2.f - 1.f;
  float const ny = ((off.y + float(y)) / float(H)) * 2.f - 1.f;
  float h[3];
#pragma unroll
  for (int k = 0; k < 3; ++k)
    h[k] = ((cam.vp[0 * 4 + k] * nx + cam.vp[1 * 4 + k] * ny) + cam.vp[2 * 4 + k] * 1.f) + cam.vp[3 * 4 + k] * 1.f;
  v3 dir = rs::normalize(v3{h[0], h[1], h[2]});
  v3 origin{cam.eye[0], cam.eye[1], cam.eye[2]};
  v3 tint{1.f, 1.f, 1.f};
  if (cam.dof) {
    // bokeh.glsl:15-34 bokeh_get: the value is read at the previous offset,
    // then a new offset is drawn (the returned offset was never sampled)
    v2 offset = rs::random_uniform_circle(r, 0.49f);
    v3 value{1.f, 1.f, 1.f};
    float amount = 1.f;
    if (cam.bokeh.p && cam.bokeh.w >= 10) {
      int tries = 8;
      while ((tries == 8 || amount < 1e-5f) && tries-- > 0) {
        float4 const m = rs::tex_sample(cam.bokeh, 0.5f + offset.x, 0.5f + offset.y);
        value = {m.x, m.y, m.z};
        offset = rs::random_uniform_circle(r, 0.49f);
        amount = rs::gmax(rs::gmax(value.x, value.y), value.z);
      }
    }
    // pt_generate.comp:35-48 apply_bokeh
    if (!(amount < 1e-5f)) {
      v3 const center = origin + cam.focus * dir;
      v3 const alt = rs::transform_local_to_world(
          rs::normalize(v3{(offset.x * cam.lens[0]) / 2.f, (offset.y * cam.lens[1]) / 2.f, cam.focus}), dir);
      tint = value;
      origin = center - cam.focus * alt;
      dir = alt;
    }
  }
  float const rv = rs::random_next(r);
  float4* g = gen + 5 * size_t(id);
  g[0] = make_float4(origin.x, origin.y, origin.z, rv);
  g[1] = make_float4(dir.x, dir.y, dir.z, float(x));
  g[2] = make_float4(tint.x, tint.y, tint.z, float(y));
  g[3] = make_float4(0.f, 0.f, 0.f, 0.f);
  g[4] = make_float4(1.f, 1.f, 0.f, 0.f);
}

// ---- pt_trace.comp --------------------------------------------------------------
// One thread per ray of the pass. The steps are ordered so that little state
// is live across the two tree walks: the closest-hit walk needs only the ray;
// pt_trace.comp:134-146's random draws (light choice, point on the light) come
// after it -- the walk draws nothing, and the SDF marches, which do draw, still
// follow them as in the reference; the trace record is written before the
// shadow walk, which then only adds the light term. Same operations, same
// results as the reference's order.
// Visiting order of a trace pass over the frames in flight: for every thread
// of the pass's grid, the origin / direction cell key of its ray slot
// (ray_key), or 0xFFFFFF, after every live key, for an empty slot.
__global__ void __launch_bounds__(kBlock) k_gen_keys(float4 const* __restrict__ gen, uint32_t const* __restrict__ count,
    uint32_t slots, uint32_t nb, float3 lo, float3 cell_scale, uint32_t* __restrict__ keys,
    uint32_t* __restrict__ vals) {
  frame_slot const fs = frame_of(nb);
  uint32_t const t = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t key = 0xFFFFFFu;
  if (fs.id < count[fs.f]) {
    float4 const* g = gen + 5 * (size_t(fs.f) * slots + fs.id);
    key = min(ray_key(g[0], g[1], lo, cell_scale), 0xFFFFFEu);
  }
  keys[t] = key;
  vals[t] = t;
}

// gen / trace: the frames' regions of `slots` rays; count[f]: frame f's rays.
// perm (may be null): thread t takes the ray slot of thread perm[t] of the grid.
// shadow_q (may be null): without SDF drawables, the NEE shadow rays are
// appended there (2 float4 each, *shadow_count of them) for k_shadow_pass
// instead of being walked here.
// Four resident blocks per SM (64 registers; the unbounded build used 80 and spilled as much): with
// frames in flight the pass is issue-bound, and the extra warps measured 12 % faster together with
// the same cap on k_color_pass (0.373 -> 0.330 ms per 512x512 frame).
__global__ void __launch_bounds__(kBlock, 4) k_trace_pass(scene_dev s, pass_rand pr, float4 const* __restrict__ gen,
    float4* __restrict__ trace, uint32_t const* __restrict__ count, uint32_t slots, uint32_t nb,
    uint32_t const* __restrict__ perm, float4* __restrict__ shadow_q, uint32_t* __restrict__ shadow_count) {
  uint32_t thread = blockIdx.x * blockDim.x + threadIdx.x;
  if (perm) thread = __ldg(perm + thread);
  frame_slot fs;
  fs.f = thread / (nb * kBlock);
  fs.id = thread - fs.f * nb * kBlock;
  uint32_t const id = fs.id;
  if (id >= count[fs.f]) return;
  float const* const tex = pr.tex + fs.f * pr.tex_stride;
  int const seed = pr.seed[fs.f];
  gen += 5 * size_t(fs.f) * slots;
  trace += 4 * size_t(fs.f) * slots;
  float4 const g0 = gen[5 * size_t(id) + 0];
  float4 const g1 = gen[5 * size_t(id) + 1];
  v3 const ro = xyz(g0), rd = xyz(g1);

  hit_rec h;
  uint32_t cn = 0, ct = 0;
  bool hits = traverse<0, false, false>(s.nodes, s.tris, f3{ro.x, ro.y, ro.z}, f3{rd.x, rd.y, rd.z}, 0.f,
      __int_as_float(0x7f800000), h, s.err, cn, ct);
  float ht = h.t;
  int hits_light = -1;
  v3 position{0.f, 0.f, 0.f}, normal{0.f, 0.f, 0.f};
  v2 uv{0.f, 0.f};
  int material = 0;
  if (hits) {
    float4 const* tp = s.tris + 3 * size_t(h.leaf);
    v3 const p0 = xyz(__ldg(tp)), p1 = xyz(__ldg(tp + 1)), p2 = xyz(__ldg(tp + 2));
    float const bx = h.u, by = h.v;
    float const w = (1.f - bx) - by;
    position = (bx * p1 + by * p2) + w * p0;
    uint32_t const prim = uint32_t(h.prim);
    if (s.tri_normals) {
      v3 const n0 = xyz(__ldg(s.tri_normals + 3 * size_t(prim))), n1 = xyz(__ldg(s.tri_normals + 3 * size_t(prim) + 1)),
               n2 = xyz(__ldg(s.tri_normals + 3 * size_t(prim) + 2));
      normal = rs::normalize((bx * n1 + by * n2) + w * n0);
    } else {
      normal = rs::normalize(rs::cross(rs::normalize(p1 - p0), rs::normalize(p2 - p0)));
    }
    if (s.tri_uvs) {
      float2 const u0 = __ldg(s.tri_uvs + 3 * size_t(prim)), u1 = __ldg(s.tri_uvs + 3 * size_t(prim) + 1),
                   u2 = __ldg(s.tri_uvs + 3 * size_t(prim) + 2);
      uv = {(bx * u1.x + by * u2.x) + w * u0.x, (bx * u1.y + by * u2.y) + w * u0.y};
    }
    material = __ldg(s.tri_material + prim);
  }

  float4 const g2 = gen[5 * size_t(id) + 2];
  rs::rng_t r;
  rs::random_init(r, tex, rs::f2i(g1.w), rs::f2i(g2.w), seed);
  int const li = min(max(rs::f2i(2.f * rs::random_next(r)), 0), 1);
  float const rx = rs::random_next(r);
  float const ry = rs::random_next(r);
  float const rz = rs::random_next(r);
  float const rq = rs::random_next(r);
  v3 p_on_light;
  {
    light_t const L = c_lights[li];
    p_on_light = v3{L.px, L.py, L.pz} + rs::normalize(v3{rx, ry, rz}) * L.r * sqrtf(rq);
  }

  // SDF drawables after the meshes (pt_trace.comp:342-352): a closer march hit
  // replaces the mesh hit and its attributes.
  for (int dsdf = 0; dsdf < s.sdf.n_drawables; ++dsdf) {
    sdfk::sdf_hit const sh =
        sdfk::march(s.sdf, dsdf, ro, rd, hits ? ht : __int_as_float(0x7f800000), false, &r);
    if (sh.hits && sh.t < ht) {
      hits = true;
      ht = sh.t;
      position = sh.position;
      normal = sh.normal;
      uv = v2{sh.u, sh.v};
      material = sh.material;
    }
  }
#pragma unroll
  for (int l = 0; l < 2; ++l) {
    float const tl = intersect_sphere(ro, rd, v3{c_lights[l].px, c_lights[l].py, c_lights[l].pz}, c_lights[l].r);
    if (tl > 0.f && (!hits || tl < ht)) {
      hits = true;
      ht = tl;
      hits_light = l;
    }
  }
  int intersects = 0;
  uint32_t light_color = 0;
  v3 light_dir{0.f, 0.f, 0.f};
  float light_strength = 0.f;
  bool shadow = false;
  v3 so{0.f, 0.f, 0.f}, dir_l{0.f, 0.f, 0.f};
  float dist_l = 0.f;
  if (hits) {
    intersects = 1;
    if (rs::inf3(normal) || rs::nan3(normal)) intersects = 0;
    v3 const path = p_on_light - position;
    dir_l = rs::normalize(path);
    dist_l = rs::length(path);
    v3 const lnorm = rs::faceforward(normal, rd, normal);
    if (hits_light >= 0) {
      intersects = 2;
      v3 const col{c_lights[hits_light].cx, c_lights[hits_light].cy, c_lights[hits_light].cz};
      light_strength = rs::length(col);
      light_color = rs::pack_unorm4x8(col.x / light_strength, col.y / light_strength, col.z / light_strength,
          0.f / light_strength);
      light_dir = dir_l;
    } else if (rs::dot(dir_l, lnorm) > 0.f) {
      so = position + lnorm * 0.01f;
      shadow = true;
    }
  } else {
    position = {0.f, 0.f, 0.f};
    normal = {0.f, 0.f, 0.f};
  }
  float4* t = trace + 4 * size_t(id);
  t[0] = make_float4(position.x, position.y, position.z, __int_as_float(intersects));
  t[1] = make_float4(normal.x, normal.y, normal.z, __uint_as_float(id));
  t[2] = make_float4(uv.x, uv.y, __int_as_float(material), __uint_as_float(light_color));
  t[3] = make_float4(light_dir.x, light_dir.y, light_dir.z, light_strength);
  if (!shadow) return;
  if (shadow_q && s.sdf.n_drawables == 0) {
    // one atomic per group of converged lanes; entry: (so, dist_l), (dir_l, slot | light << 31)
    uint32_t const lanes = __activemask();
    uint32_t const lane = threadIdx.x & 31u;
    uint32_t const leader = uint32_t(__ffs(lanes)) - 1u;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(shadow_count, uint32_t(__popc(lanes)));
    base = __shfl_sync(lanes, base, int(leader));
    uint32_t const e = base + uint32_t(__popc(lanes & ((1u << lane) - 1u)));
    uint32_t const slot = fs.f * slots + id;
    shadow_q[2 * size_t(e)] = make_float4(so.x, so.y, so.z, dist_l);
    shadow_q[2 * size_t(e) + 1] = make_float4(dir_l.x, dir_l.y, dir_l.z, __uint_as_float(slot | (uint32_t(li) << 31)));
    return;
  }
  hit_rec hs;
  bool occluded = traverse<0, true, false>(s.nodes, s.tris, f3{so.x, so.y, so.z}, f3{dir_l.x, dir_l.y, dir_l.z},
      0.f, dist_l, hs, s.err, cn, ct);
  // any_hit's SDF loop (pt_trace.comp:319-327)
  for (int dsdf = 0; !occluded && dsdf < s.sdf.n_drawables; ++dsdf)
    occluded = sdfk::march(s.sdf, dsdf, so, dir_l, dist_l, true, &r).hits;
  if (occluded) return;
  v3 const col{c_lights[li].cx, c_lights[li].cy, c_lights[li].cz};
  light_strength = rs::length(col);
  light_color = rs::pack_unorm4x8(col.x / light_strength, col.y / light_strength, col.z / light_strength,
      0.f / light_strength);
  light_strength = light_strength * (2.f / dist_l);
  reinterpret_cast<float*>(t + 2)[3] = __uint_as_float(light_color);
  t[3] = make_float4(dir_l.x, dir_l.y, dir_l.z, light_strength);
}

// The NEE shadow rays k_trace_pass queued (meshes only): any_hit
// (pt_trace.comp:311-318) and, when unoccluded, the light term of the ray's
// trace record, as k_trace_pass computes it in place.
constexpr int kShadowBlock = 128;
__global__ void __launch_bounds__(kShadowBlock, 8) k_shadow_pass(scene_dev s, float4 const* __restrict__ q,
    uint32_t const* __restrict__ count, float4* __restrict__ trace) {
  uint32_t const i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= *count) return;
  float4 const a = q[2 * size_t(i)], b = q[2 * size_t(i) + 1];
  uint32_t const w = __float_as_uint(b.w);
  uint32_t const slot = w & 0x7fffffffu;
  int const li = int(w >> 31);
  float const dist_l = a.w;
  hit_rec hs;
  uint32_t cn = 0, ct = 0;
  if (traverse<0, true, false>(s.nodes, s.tris, f3{a.x, a.y, a.z}, f3{b.x, b.y, b.z}, 0.f, dist_l, hs, s.err, cn, ct))
    return;
  v3 const col{c_lights[li].cx, c_lights[li].cy, c_lights[li].cz};
  float light_strength = rs::length(col);
  uint32_t const light_color = rs::pack_unorm4x8(col.x / light_strength, col.y / light_strength,
      col.z / light_strength, 0.f / light_strength);
  light_strength = light_strength * (2.f / dist_l);
  float4* t = trace + 4 * size_t(slot);
  reinterpret_cast<float*>(t + 2)[3] = __uint_as_float(light_color);
  t[3] = make_float4(b.x, b.y, b.z, light_strength);
}

// ---- pt_color.comp ----------------------------------------------------------------
struct color_args {
  int2 const* mat_refs;
  int n_mats;
  float const* mat_data;
  float4* accum;
  float4* display;
  uint32_t W;
  uint32_t sample_index;
  int force;
  rs::tex2d const* textures;  // albedo textures by slot (material handle = slot + 1)
  int n_textures;
  rs::cubemap_dev cube;       // size <= 10: the sky gradient (pt_color.comp:190-199)
};

__device__ __forceinline__ bool naninf4(float4 v) {
  return isnan(v.x) || isnan(v.y) || isnan(v.z) || isnan(v.w) || isinf(v.x) || isinf(v.y) || isinf(v.z) ||
      isinf(v.w);
}

// pt_color.comp:77-101
__device__ __forceinline__ void accumulate(color_args const& a, float4 nc, int px, int py) {
  size_t const pi = size_t(py) * a.W + size_t(px);
  float4 last = a.accum[pi];
  if (naninf4(nc)) nc = last;
  float4 const actual_last = last;
  if (a.sample_index == 0) last = make_float4(nc.x, nc.y, nc.z, 1.f);
  else last = make_float4(last.x + nc.x, last.y + nc.y, last.z + nc.z, last.w + 1.f);
  if (naninf4(last)) last = actual_last;
  a.accum[pi] = last;
  a.display[pi] = make_float4(rs::gclamp(last.x / last.w, 0.f, 4.f), rs::gclamp(last.y / last.w, 0.f, 4.f),
      rs::gclamp(last.z / last.w, 0.f, 4.f), 1.f);
}

// A path that ends adds its colour to the accumulation (one frame in flight:
// fcol null) or leaves it in fcol[f * slots + pixel] for k_resolve_frames.
// block_sums[blockIdx.x]: the block's surviving rays.
__global__ void __launch_bounds__(kBlock, 4) k_color_pass(color_args a, pass_rand pr, float4* __restrict__ gen,
    float4* __restrict__ trace, uint32_t const* __restrict__ count, uint32_t* __restrict__ block_sums,
    float4* __restrict__ fcol, uint32_t slots, uint32_t nb) {
  frame_slot const fs = frame_of(nb);
  uint32_t const id = fs.id;
  float const* const tex = pr.tex + fs.f * pr.tex_stride;
  int const seed = pr.seed[fs.f];
  gen += 5 * size_t(fs.f) * slots;
  trace += 4 * size_t(fs.f) * slots;
  bool keep = false;
  if (id < count[fs.f]) {
    float4* gp = gen + 5 * size_t(id);
    float4* tp = trace + 4 * size_t(id);
    float4 const t0 = tp[0], t1 = tp[1], t2 = tp[2], t3 = tp[3];
    float4 g0 = gp[0], g1 = gp[1], g2 = gp[2], g3 = gp[3], g4 = gp[4];
    int const intersects = __float_as_int(t0.w);
    int const px = rs::f2i(g1.w), py = rs::f2i(g2.w);
    auto finish = [&](float4 nc) {
      if (fcol) fcol[size_t(fs.f) * slots + size_t(py) * a.W + size_t(px)] = nc;
      else accumulate(a, nc, px, py);
    };
    v3 const refl0 = xyz(g2);
    float const pdf0 = g4.x;
    if (intersects != 0) {
      if (intersects == 2) {
        reinterpret_cast<int*>(tp)[3] = 0;
        v3 const lc = rs::unpack_rgb(__float_as_uint(t2.w));
        v3 const c = lc * t3.w * refl0 / pdf0;
        finish(make_float4(c.x + g3.x, c.y + g3.y, c.z + g3.z, 1.f + g3.w));
      } else {
        v3 const normal = xyz(t1);
        rs::rng_t r;
        rs::random_init(r, tex, px, py, seed);
        uint32_t const uid = id;
        float const rvin = g0.w;
        rs::random_value(r, int(uint32_t(rs::f2i(56128966.f * rvin)) + 20945293u * uid));
        rs::random_value(r, int(uint32_t(rs::f2i(12233432.f * rvin)) + 74867839u * uid));
        rs::material_ctx mc;
        int const mi = __float_as_int(t2.z);
        bool const valid = mi >= 0 && mi < a.n_mats;
        int2 const ref = valid ? __ldg(a.mat_refs + mi) : make_int2(-1, 0);
        rs::mat_open(mc, ref.x, a.mat_data, ref.y);
        float const m0 = rs::random_next(r);
        float const m1 = rs::random_next(r);
        v3 const dir = xyz(g1);
        v3 const generated = rs::mat_bounce(mc, r, v2{m0, m1}, -dir, normal);
        v3 mrefl;
        float mpdf;
        v2 const uv{t2.x, t2.y};
        rs::mat_evaluate(mc, normal, generated, -dir, mrefl, mpdf, uv, a.textures, a.n_textures);
        float const rnd = rs::random_next(r);
        bool done = false;
        if (rnd > pdf0 * 1.f) {
          reinterpret_cast<int*>(tp)[3] = 0;
          v3 const c = refl0 / pdf0;
          finish(make_float4(g3.x + c.x, g3.y + c.y, g3.z + c.z, g3.w));
          done = true;
        } else if (a.force || pdf0 < 1e-5f || mpdf < 1e-6f || isnan(mpdf) || isinf(mpdf) || rs::nan3(mrefl) ||
                   rs::inf3(mrefl) || rs::nan3(generated) || rs::inf3(generated)) {
          reinterpret_cast<int*>(tp)[3] = 0;
          if (rs::nan3(mrefl) || rs::inf3(mrefl) || isnan(pdf0) || isinf(pdf0) || pdf0 < 1e-5f) {
            finish(g3);
          } else {
            v3 const c = refl0 / pdf0;
            finish(make_float4(g3.x + c.x, g3.y + c.y, g3.z + c.z, g3.w));
          }
          done = true;
        }
        if (!done) {
          if (t3.w > 0.f) {
            v3 lrefl{1.f, 1.f, 1.f};
            float lpdf = 1.f;
            rs::mat_evaluate(mc, normal, xyz(t3), -dir, lrefl, lpdf, uv, a.textures, a.n_textures);
            if (!rs::inf3(lrefl)) {
              v3 const lc = rs::unpack_rgb(__float_as_uint(t2.w));
              v3 const c = lc * t3.w * rs::clamp3(lrefl, 0.f, 1.f);
              g3 = make_float4(g3.x + c.x, g3.y + c.y, g3.z + c.z, g3.w);
            }
          }
          v3 const origin = xyz(t0) + 1e-4f * rs::faceforward(normal, -generated, normal);
          float const pdf1 = pdf0 * mpdf;
          v3 const refl1 = refl0 * mrefl;
          // the literal 2341335623 is an int with that bit pattern in GLSL: -1953631673
          float const rv1 = rs::random_value(r, int(uint32_t(rs::f2i(-1953631673.f * rvin)) + 357883444u * uid));
          gp[0] = make_float4(origin.x, origin.y, origin.z, rv1);
          gp[1] = make_float4(generated.x, generated.y, generated.z, g1.w);
          gp[2] = make_float4(refl1.x, refl1.y, refl1.z, g2.w);
          gp[3] = g3;
          gp[4] = make_float4(pdf1, g4.y, g4.z, g4.w);
          keep = true;
        }
      }
    } else {
      v3 const dir = xyz(g1);
      v3 env;
      if (a.cube.p && a.cube.size > 10) {
        env = rs::clamp3(refl0 * rs::cube_sample(a.cube, dir) / pdf0, 0.f, 16.f);
      } else {
        float const t = (dir.y + 1.f) / 2.f;
        v3 const sky = rs::mix3(v3{0.3f, 0.4f, 0.5f}, v3{1.f, 0.98f, 0.96f}, t);
        env = rs::clamp3(refl0 * sky / pdf0, 0.f, 16.f);
      }
      finish(make_float4(g3.x + env.x, g3.y + env.y, g3.z + env.z, g3.w));
    }
  }
  int const c = __syncthreads_count(keep);
  if (threadIdx.x == 0) block_sums[blockIdx.x] = uint32_t(c);
}

// ---- pt_ray_filter.comp (stable) ---------------------------------------------------
// Exclusive scan of one frame's per-block survivor counts (block f: frame f's
// nblocks sums), its total -> new_count[f].
__global__ void __launch_bounds__(1024) k_scan_blocks(uint32_t* __restrict__ sums, uint32_t nblocks,
    uint32_t* __restrict__ new_count) {
  sums += size_t(blockIdx.x) * nblocks;
  new_count += blockIdx.x;
  __shared__ uint32_t warp_tot[32];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  uint32_t const lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  for (uint32_t base = 0; base < nblocks; base += 1024) {
    uint32_t const i = base + threadIdx.x;
    uint32_t const v = i < nblocks ? sums[i] : 0u;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t const y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= uint32_t(o)) x += y;
    }
    if (lane == 31) warp_tot[warp] = x;
    __syncthreads();
    if (warp == 0) {
      uint32_t w = warp_tot[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t const y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= uint32_t(o)) w += y;
      }
      warp_tot[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    uint32_t const excl = carry + (warp ? warp_tot[warp - 1] : 0u) + x - v;
    if (i < nblocks) sums[i] = excl;
    __syncthreads();
    if (threadIdx.x == 0) carry += warp_tot[31];
    __syncthreads();
  }
  if (threadIdx.x == 0) *new_count = carry;
}

// Survivors of each frame's region, in order, to the front of the same region
// of gen_out (offsets: the scanned block sums).
__global__ void __launch_bounds__(kBlock) k_scatter(float4 const* __restrict__ gen_in, float4 const* __restrict__ trace,
    uint32_t const* __restrict__ count, uint32_t const* __restrict__ offsets, float4* __restrict__ gen_out,
    uint32_t slots, uint32_t nb) {
  __shared__ uint32_t warp_cnt[kBlock / 32];
  frame_slot const fs = frame_of(nb);
  uint32_t const id = fs.id;
  size_t const base = size_t(fs.f) * slots;
  gen_in += 5 * base;
  gen_out += 5 * base;
  trace += 4 * base;
  bool const keep = id < count[fs.f] && __float_as_int(trace[4 * size_t(id)].w) == 1;
  uint32_t const lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  uint32_t const ballot = __ballot_sync(0xffffffffu, keep);
  if (lane == 0) warp_cnt[warp] = __popc(ballot);
  __syncthreads();
  uint32_t before = 0;
  for (uint32_t w = 0; w < warp; ++w) before += warp_cnt[w];
  if (keep) {
    uint32_t const dst = offsets[blockIdx.x] + before + __popc(ballot & ((1u << lane) - 1u));
    uint32_t const src = __float_as_uint(trace[4 * size_t(id) + 1].w);  // generated_ray
#pragma unroll
    for (int k = 0; k < 5; ++k) gen_out[5 * size_t(dst) + k] = gen_in[5 * size_t(src) + k];
  }
}

// The frames in flight into the accumulation, in frame order, pixel by pixel
// (frame f restarts it when sample_index + f == 0).
__global__ void __launch_bounds__(kBlock) k_resolve_frames(color_args a, float4 const* __restrict__ fcol,
    uint32_t frames, uint32_t W, uint32_t H) {
  uint32_t const pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= W * H) return;
  uint32_t const s0 = a.sample_index;
  for (uint32_t f = 0; f < frames; ++f) {
    a.sample_index = s0 + f;
    accumulate(a, fcol[size_t(f) * W * H + pix], int(pix % W), int(pix / W));
  }
}

// ---- host side ----------------------------------------------------------------------
void free_ray_buffers(render_state& R) {
  for (void* p : {static_cast<void*>(R.gen[0]), static_cast<void*>(R.gen[1]), static_cast<void*>(R.trace),
           static_cast<void*>(R.counts), static_cast<void*>(R.block_sums), static_cast<void*>(R.fcol),
           static_cast<void*>(R.okeys[0]), static_cast<void*>(R.okeys[1]), static_cast<void*>(R.ovals[0]),
           static_cast<void*>(R.ovals[1]), R.otemp, static_cast<void*>(R.shadow_q)})
    cudaFree(p);
  R.gen[0] = R.gen[1] = nullptr;
  R.trace = R.fcol = nullptr;
  R.counts = R.block_sums = nullptr;
  R.okeys[0] = R.okeys[1] = R.ovals[0] = R.ovals[1] = nullptr;
  R.otemp = nullptr;
  R.otemp_bytes = 0;
  R.shadow_q = nullptr;
  R.frames_cap = 0;
}

// Ray buffers for `frames` frames in flight of a W x H render (grown, never shrunk).
int ensure_render_buffers(myrt_ctx* ctx, uint32_t W, uint32_t H, uint32_t frames) {
  int rc = ensure_images(ctx, W, H);
  render_state& R = ctx->render;
  if (rc || (R.gen[0] && R.frames_cap >= frames)) return rc;
  rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "ray buffers in use");
  if (rc) return rc;
  free_ray_buffers(R);
  size_t const n = size_t(W) * H * frames;
  size_t const nb = size_t(frames) * ((size_t(W) * H + kBlock - 1) / kBlock);
  auto alloc = [&](void** p, size_t bytes, char const* what) {
    if (!rc) rc = check_cuda(ctx, cudaMalloc(p, bytes), what);
  };
  alloc(reinterpret_cast<void**>(&R.gen[0]), n * 80, "ray state");
  alloc(reinterpret_cast<void**>(&R.gen[1]), n * 80, "ray state");
  alloc(reinterpret_cast<void**>(&R.trace), n * 64, "trace state");
  alloc(reinterpret_cast<void**>(&R.counts), (2 * kMaxFramesInFlight + 1) * sizeof(uint32_t), "ray counts");
  alloc(reinterpret_cast<void**>(&R.shadow_q), n * 32, "shadow rays");
  alloc(reinterpret_cast<void**>(&R.block_sums), std::max<size_t>(nb, 1) * sizeof(uint32_t), "block sums");
  if (frames > 1) alloc(reinterpret_cast<void**>(&R.fcol), n * 16, "frame colours");
  // visiting order of the trace passes: one key and slot per thread of a pass's grid
  size_t const threads = nb * kBlock;
  for (int k = 0; k < 2; ++k) {
    alloc(reinterpret_cast<void**>(&R.okeys[k]), threads * 4, "pass order keys");
    alloc(reinterpret_cast<void**>(&R.ovals[k]), threads * 4, "pass order slots");
  }
  if (!rc)
    rc = check_cuda(ctx, cub::DeviceRadixSort::SortPairs(nullptr, R.otemp_bytes, R.okeys[0], R.okeys[1], R.ovals[0],
                             R.ovals[1], int(threads), 0, kOrderKeyBits, ctx->stream), "pass order size");
  alloc(&R.otemp, std::max<size_t>(R.otemp_bytes, 16), "pass order temporary");
  if (rc) {
    free_ray_buffers(R);
    return rc;
  }
  R.frames_cap = frames;
  return MYRT_OK;
}

void mat_mul4(float const* a, float const* b, float* out) {
  for (int c = 0; c < 4; ++c)
    for (int r = 0; r < 4; ++r)
      out[c * 4 + r] = ((a[0 * 4 + r] * b[c * 4 + 0] + a[1 * 4 + r] * b[c * 4 + 1]) + a[2 * 4 + r] * b[c * 4 + 2]) +
          a[3 * 4 + r] * b[c * 4 + 3];
}

}  // namespace

// Releases the device buffers; the camera record and the sample counter stay.
void free_render(render_state& R) {
  free_ray_buffers(R);
  for (void* p : {static_cast<void*>(R.accum), static_cast<void*>(R.display), static_cast<void*>(R.pass_tex),
           static_cast<void*>(R.accum64)})
    cudaFree(p);
  R.accum = R.display = nullptr;
  R.pass_tex = nullptr;
  R.accum64 = nullptr;
  R.pass_tex_capacity = 0;
  R.width = R.height = 0;
}

// The accumulation and display images of a W x H render (both modes). A new
// size releases every render buffer and restarts accumulation.
int ensure_images(myrt_ctx* ctx, uint32_t W, uint32_t H) {
  render_state& R = ctx->render;
  if (R.width == W && R.height == H && R.accum) return MYRT_OK;
  free_render(R);
  size_t const n = size_t(W) * H;
  int rc = check_cuda(ctx, cudaMalloc(reinterpret_cast<void**>(&R.accum), n * 16), "accumulation image");
  if (!rc) rc = check_cuda(ctx, cudaMalloc(reinterpret_cast<void**>(&R.display), n * 16), "display image");
  if (!rc) rc = check_cuda(ctx, cudaMemsetAsync(R.accum, 0, n * 16, ctx->stream), "clear");
  if (!rc) rc = check_cuda(ctx, cudaMemsetAsync(R.display, 0, n * 16, ctx->stream), "clear");
  if (rc) {
    free_render(R);
    return rc;
  }
  R.width = W;
  R.height = H;
  R.sample_counter = 0;  // invalidate_texture -> invalidate_counter
  return MYRT_OK;
}

// Host random stream of sequential_pathtracer.cpp:282-498 for `frames` frames:
// pass_generate draws its int seed then the 1024 texture floats, pass_trace
// likewise, pass_color the floats first and then the int.
void draw_host_randomness(std::mt19937& rng, int frames, int bounces, std::vector<int>& seeds, std::vector<float>& tex) {
  int const passes = 2 * bounces + 3;
  seeds.resize(size_t(frames) * passes);
  tex.resize(size_t(frames) * passes * kTexSize);
  for (int f = 0; f < frames; ++f) {
    for (int p = 0; p < passes; ++p) {
      std::uniform_int_distribution<> dist;
      std::uniform_real_distribution<float> uni(0.f, 1.f);
      bool const is_color = p >= 1 && ((p - 1) % 2 == 1);
      int& s = seeds[size_t(f) * passes + p];
      float* t = tex.data() + (size_t(f) * passes + p) * kTexSize;
      if (!is_color) s = dist(rng);
      for (int k = 0; k < kTexSize; ++k) t[k] = uni(rng);
      if (is_color) s = dist(rng);
    }
  }
}

// Launch arguments of one reference-shading call: the camera (with depth of
// field and the bokeh mask), the scene and the colour pass (textures, cube
// map), shared by myrt_render and myrt_render_noalloc so both run the same
// frames.
struct frame_setup {
  camera_dev cd;
  scene_dev sd;
  color_args ca;
};

frame_setup make_frame_setup(myrt_ctx* ctx, myrt_camera const* cam, myrt_render_params const* p, float4* accum,
    float4* display, uint32_t sample_index) {
  device_scene const& S = ctx->scene;
  camera_dev cd{};
  mat_mul4(cam->inverse_view, cam->inverse_projection, cd.vp);
  cd.eye[0] = cam->inverse_view[12];
  cd.eye[1] = cam->inverse_view[13];
  cd.eye[2] = cam->inverse_view[14];
  cd.dof = p->dof_active ? 1 : 0;
  cd.lens[0] = p->lens_size[0];
  cd.lens[1] = p->lens_size[1];
  cd.focus = p->focus;
  if (p->bokeh_texture > 0 && size_t(p->bokeh_texture) <= ctx->textures.size()) {
    auto const& t = ctx->textures[size_t(p->bokeh_texture) - 1];
    cd.bokeh = rs::tex2d{t.data, t.w, t.h, t.wrap};
  }
  scene_dev sd{S.nodes, S.tris, S.tri_normals, S.tri_uvs, S.tri_material,
      reinterpret_cast<int2 const*>(S.materials), int(S.n_materials), S.material_data, ctx->d_err,
      make_sdf_dev(ctx, p->sdf_marching_steps, p->sdf_marching_epsilon)};
  color_args ca{reinterpret_cast<int2 const*>(S.materials), int(S.n_materials), S.material_data, accum, display,
      p->width, sample_index, 0, reinterpret_cast<rs::tex2d const*>(ctx->d_textures), int(ctx->textures.size()),
      rs::cubemap_dev{ctx->cubemap, ctx->cubemap_size}};
  return frame_setup{cd, sd, ca};
}

int render_reference_frames(myrt_ctx* ctx, myrt_camera const* cam, myrt_render_params const* p) {
  uint32_t const W = p->width, H = p->height;
  int const B = p->num_bounces;
  int const F = int(p->frames);
  int const passes = 2 * B + 3;
  size_t const n = size_t(W) * H;
  uint32_t const nb = uint32_t((n + kBlock - 1) / kBlock);
  // frames in flight: enough to fill about 16 Mi ray slots per launch (~5 GB of ray state; 4 Mi
  // left the late, sparse passes tail-bound: 0.52 against 0.42 ms per 512x512 frame)
  uint32_t K = ctx->tuning.ref_frames ? ctx->tuning.ref_frames : uint32_t(std::max<size_t>(1, (size_t(1) << 24) / n));
  K = std::min<uint32_t>({K, uint32_t(kMaxFramesInFlight), uint32_t(std::max(F, 1))});
  int rc = ensure_render_buffers(ctx, W, H, K);
  if (rc) return rc;
  render_state& R = ctx->render;
  std::vector<int> seeds;
  std::vector<float> tex;
  draw_host_randomness(ctx->host_rng, F, B, seeds, tex);
  if (R.pass_tex_capacity < tex.size()) {
    cudaFree(R.pass_tex);
    R.pass_tex = nullptr;
    R.pass_tex_capacity = 0;
    rc = check_cuda(ctx, cudaMalloc(&R.pass_tex, tex.size() * sizeof(float)), "pass randomness");
    if (rc) return rc;
    R.pass_tex_capacity = tex.size();
  }
  rc = check_cuda(ctx,
      cudaMemcpyAsync(R.pass_tex, tex.data(), tex.size() * sizeof(float), cudaMemcpyHostToDevice, ctx->stream),
      "pass randomness upload");
  if (rc) return rc;

  frame_setup const fs = make_frame_setup(ctx, cam, p, R.accum, R.display, R.sample_counter);
  camera_dev const& cd = fs.cd;
  scene_dev const& sd = fs.sd;
  color_args ca = fs.ca;
  cudaStream_t const st = ctx->stream;
  uint32_t* const cnt[2] = {R.counts, R.counts + kMaxFramesInFlight};
  // Visiting order of the trace passes (trace_order): sorted by origin / direction cell for the first
  // two passes, which hold most of the rays, once the frames in flight fill 1 Mi slots (0); never
  // (1); every pass (2). Results never depend on it.
  uint32_t const order = ctx->tuning.trace_order;
  // NEE shadow rays of mesh-only scenes walk in their own pass, every lane with a ray (a queue
  // entry names its slot in 31 bits)
  bool const split_shadow = sd.sdf.n_drawables == 0 && size_t(K) * n < (size_t(1) << 31);
  uint32_t* const shadow_count = R.counts + 2 * kMaxFramesInFlight;
  float3 klo, ksc;
  ray_key_grid(ctx->scene.bounds, klo, ksc);
  for (int f0 = 0; f0 < F; f0 += int(K)) {
    uint32_t const k = std::min<uint32_t>(K, uint32_t(F - f0));
    auto rand_of = [&](int pass) {
      pass_rand pr{};
      pr.tex = R.pass_tex + (size_t(f0) * passes + pass) * kTexSize;
      pr.tex_stride = uint32_t(passes * kTexSize);
      for (uint32_t j = 0; j < k; ++j) pr.seed[j] = seeds[(size_t(f0) + j) * passes + pass];
      return pr;
    };
    float4* const fcol = k > 1 ? R.fcol : nullptr;
    uint32_t const grid = k * nb;
    int cur = 0;
    ca.sample_index = R.sample_counter;
    k_generate<<<grid, kBlock, 0, st>>>(W, H, nb, rand_of(0), cd, R.gen[cur], cnt[cur]);
    int pass = 1;
    for (int i = 0; i <= B; ++i) {
      bool const last = i == B;
      bool const sorted = order == 2 || (order == 0 && i < 2 && size_t(k) * n >= (size_t(1) << 20));
      uint32_t const* perm = nullptr;
      if (sorted) {
        k_gen_keys<<<grid, kBlock, 0, st>>>(R.gen[cur], cnt[cur], uint32_t(n), nb, klo, ksc, R.okeys[0], R.ovals[0]);
        size_t tb = R.otemp_bytes;
        rc = check_cuda(ctx, cub::DeviceRadixSort::SortPairs(R.otemp, tb, R.okeys[0], R.okeys[1], R.ovals[0],
                                 R.ovals[1], int(size_t(grid) * kBlock), 0, kOrderKeyBits, st), "pass order sort");
        if (rc) return rc;
        perm = R.ovals[1];
      }
      if (split_shadow) {
        rc = check_cuda(ctx, cudaMemsetAsync(shadow_count, 0, sizeof(uint32_t), st), "shadow queue reset");
        if (rc) return rc;
      }
      k_trace_pass<<<grid, kBlock, 0, st>>>(sd, rand_of(pass), R.gen[cur], R.trace, cnt[cur], uint32_t(n), nb, perm,
          split_shadow ? R.shadow_q : nullptr, shadow_count);
      if (split_shadow)
        k_shadow_pass<<<uint32_t((size_t(k) * n + kShadowBlock - 1) / kShadowBlock), kShadowBlock, 0, st>>>(sd,
            R.shadow_q, shadow_count, R.trace);
      ++pass;
      ca.force = last ? 1 : 0;
      k_color_pass<<<grid, kBlock, 0, st>>>(ca, rand_of(pass), R.gen[cur], R.trace, cnt[cur], R.block_sums, fcol,
          uint32_t(n), nb);
      ++pass;
      if (!last) {
        k_scan_blocks<<<k, 1024, 0, st>>>(R.block_sums, nb, cnt[1 - cur]);
        k_scatter<<<grid, kBlock, 0, st>>>(R.gen[cur], R.trace, cnt[cur], R.block_sums, R.gen[1 - cur],
            uint32_t(n), nb);
        cur = 1 - cur;
      }
    }
    if (fcol) k_resolve_frames<<<nb, kBlock, 0, st>>>(ca, fcol, k, W, H);
    rc = check_cuda(ctx, cudaGetLastError(), "wavefront launch");
    if (rc) return rc;
    R.sample_counter += k;
  }
  return MYRT_OK;
}

// ---- render without device allocation -------------------------------------------
// Some callers cannot call cudaMalloc: hosts that hand all device memory to
// their own allocator or fixed budgets up front, and frame loops that must not
// pay cudaMalloc's implicit device synchronisation. For them the render can
// run with every scratch buffer (ray states, trace records, counts, block sums,
// the pass randomness) in one fixed array below; the caller passes the scene
// (through the context) and the two output images.
namespace {
constexpr size_t kNoAllocMaxPixels = 65536;  // width * height
constexpr size_t kNoAllocMaxPasses = 256;    // frames * (2 * num_bounces + 3)
constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kNaGen = align256(kNoAllocMaxPixels * 80);
constexpr size_t kNaTrace = align256(kNoAllocMaxPixels * 64);
constexpr size_t kNaCounts = 256;
constexpr size_t kNaSums = align256((kNoAllocMaxPixels / kBlock) * sizeof(uint32_t));
constexpr size_t kNaTex = align256(kNoAllocMaxPasses * kTexSize * sizeof(float));
constexpr size_t kNaBytes = 2 * kNaGen + kNaTrace + kNaCounts + kNaSums + kNaTex;  // 15.7 MB
}  // namespace

// Held by every device that loads the library, until exit. Every call shares it.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

namespace {
// Device address of g_noalloc_scratch on the context's device, resolved once per
// device with that device current (in host code the symbol is only a host-side
// stand-in). The caller has made ctx->device current.
int noalloc_scratch(myrt_ctx* ctx, unsigned char** out) {
  static std::mutex m;
  static void* addr[64] = {};
  if (ctx->device < 0 || ctx->device >= 64) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "device ordinal >= 64");
  std::lock_guard<std::mutex> lock(m);
  if (!addr[ctx->device]) {
    void* p = nullptr;
    int rc = check_cuda(ctx, cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(scratch)");
    if (rc) return rc;
    addr[ctx->device] = p;
  }
  *out = static_cast<unsigned char*>(addr[ctx->device]);
  return MYRT_OK;
}

// Restores the calling thread's current device when a call returns.
struct device_guard {
  int prev = -1;
  ~device_guard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};
}  // namespace

int render_reference_frames_noalloc(myrt_ctx* ctx, myrt_camera const* cam, myrt_render_params const* p,
    uint32_t sample_index, float4* accum, float4* display, cudaStream_t st) {
  uint32_t const W = p->width, H = p->height;
  int const B = p->num_bounces;
  int const F = int(p->frames);
  int const passes = 2 * B + 3;
  if (size_t(W) * H > kNoAllocMaxPixels)
    return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "myrt_render_noalloc: width * height exceeds 65536 pixels");
  if (size_t(F) * size_t(passes) > kNoAllocMaxPasses)
    return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT,
        "myrt_render_noalloc: frames * (2 * num_bounces + 3) exceeds 256 passes");
  device_guard guard;
  int rc = check_cuda(ctx, cudaGetDevice(&guard.prev), "cudaGetDevice");
  if (!rc && guard.prev != ctx->device) rc = check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  if (rc) return rc;
  unsigned char* base = nullptr;
  rc = noalloc_scratch(ctx, &base);
  if (rc) return rc;
  float4* gen[2] = {reinterpret_cast<float4*>(base), reinterpret_cast<float4*>(base + kNaGen)};
  float4* trace = reinterpret_cast<float4*>(base + 2 * kNaGen);
  uint32_t* counts = reinterpret_cast<uint32_t*>(base + 2 * kNaGen + kNaTrace);
  uint32_t* sums = reinterpret_cast<uint32_t*>(base + 2 * kNaGen + kNaTrace + kNaCounts);
  float* ptex = reinterpret_cast<float*>(base + 2 * kNaGen + kNaTrace + kNaCounts + kNaSums);

  // Work the context queued on its own stream (scene or transform updates, the
  // error word's reset) comes first when the caller passes another stream.
  if (st != ctx->stream) {
    rc = check_cuda(ctx, cudaEventRecord(ctx->order_event, ctx->stream), "cudaEventRecord");
    if (!rc) rc = check_cuda(ctx, cudaStreamWaitEvent(st, ctx->order_event, 0), "cudaStreamWaitEvent");
    if (rc) return rc;
  }

  // Host randomness in draw_host_randomness's order, staged through a stack
  // buffer of kNaTexChunk passes (no heap, no device allocation) and uploaded
  // with one copy per chunk.
  constexpr int kNaTexChunk = 16;
  int seeds[kNoAllocMaxPasses];
  float tbuf[kNaTexChunk * kTexSize];
  int const total = F * passes;
  for (int q0 = 0; q0 < total; q0 += kNaTexChunk) {
    int const qn = std::min(kNaTexChunk, total - q0);
    for (int j = 0; j < qn; ++j) {
      int const q = (q0 + j) % passes;
      std::uniform_int_distribution<> dist;
      std::uniform_real_distribution<float> uni(0.f, 1.f);
      bool const is_color = q >= 1 && ((q - 1) % 2 == 1);
      int& s = seeds[q0 + j];
      if (!is_color) s = dist(ctx->host_rng);
      for (int k = 0; k < kTexSize; ++k) tbuf[size_t(j) * kTexSize + k] = uni(ctx->host_rng);
      if (is_color) s = dist(ctx->host_rng);
    }
    rc = check_cuda(ctx,
        cudaMemcpyAsync(ptex + size_t(q0) * kTexSize, tbuf, size_t(qn) * kTexSize * sizeof(float),
            cudaMemcpyHostToDevice, st),
        "pass randomness upload");
    // A copy from pageable memory has read its source when the call returns, so
    // the buffer can be refilled at once.
    if (rc) return rc;
  }

  frame_setup const fs = make_frame_setup(ctx, cam, p, accum, display, sample_index);
  camera_dev const& cd = fs.cd;
  scene_dev const& sd = fs.sd;
  color_args ca = fs.ca;
  size_t const n = size_t(W) * H;
  uint32_t const nb = uint32_t((n + kBlock - 1) / kBlock);
  for (int f = 0; f < F; ++f) {  // one frame at a time: one region of ray slots
    auto rand_of = [&](int pass) {
      pass_rand pr{};
      pr.tex = ptex + (size_t(f) * passes + pass) * kTexSize;
      pr.tex_stride = 0;
      pr.seed[0] = seeds[f * passes + pass];
      return pr;
    };
    int cur = 0;
    ca.sample_index = sample_index + uint32_t(f);
    k_generate<<<nb, kBlock, 0, st>>>(W, H, nb, rand_of(0), cd, gen[cur], counts + cur);
    int pass = 1;
    for (int i = 0; i <= B; ++i) {
      bool const last = i == B;
      k_trace_pass<<<nb, kBlock, 0, st>>>(sd, rand_of(pass), gen[cur], trace, counts + cur, uint32_t(n), nb,
          nullptr, nullptr, nullptr);
      ++pass;
      ca.force = last ? 1 : 0;
      k_color_pass<<<nb, kBlock, 0, st>>>(ca, rand_of(pass), gen[cur], trace, counts + cur, sums, nullptr,
          uint32_t(n), nb);
      ++pass;
      if (!last) {
        k_scan_blocks<<<1, 1024, 0, st>>>(sums, nb, counts + (1 - cur));
        k_scatter<<<nb, kBlock, 0, st>>>(gen[cur], trace, counts + cur, sums, gen[1 - cur], uint32_t(n), nb);
        cur = 1 - cur;
      }
    }
    rc = check_cuda(ctx, cudaGetLastError(), "wavefront launch");
    if (rc) return rc;
  }
  return MYRT_OK;
}

// ---- SDF ray queries ------------------------------------------------------------
namespace {
// The SDF loops of nearest_hit / any_hit for one ray per thread. out: 8 floats
// per ray (hit, t, normal xyz, u, v, material bits).
__global__ void __launch_bounds__(128) k_trace_sdf(sdfk::sdf_dev s, float4 const* __restrict__ rays, uint32_t n,
    int any_hit, uint32_t const* __restrict__ rng_states, float4* __restrict__ out) {
  uint32_t const i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 const r0 = rays[2 * size_t(i)], r1 = rays[2 * size_t(i) + 1];
  v3 const ro = xyz(r0), rd = xyz(r1);
  float const maxd = r1.w;
  rs::rng_t rng;
  rng.state = rng_states ? rng_states[i] : 0u;
  rng.prime = 0;
  rng.tex = nullptr;
  bool hit = false;
  float t = maxd;
  v3 nrm{0.f, 0.f, 0.f};
  float u = 0.f, v = 0.f;
  int mat = -1;
  if (any_hit) {
    for (int d = 0; !hit && d < s.n_drawables; ++d) hit = sdfk::march(s, d, ro, rd, maxd, true, &rng).hits;
  } else {
    for (int d = 0; d < s.n_drawables; ++d) {
      sdfk::sdf_hit const h = sdfk::march(s, d, ro, rd, hit ? t : maxd, false, &rng);
      if (h.hits && h.t < t) {
        hit = true;
        t = h.t;
        nrm = h.normal;
        u = h.u;
        v = h.v;
        mat = h.material;
      }
    }
  }
  out[2 * size_t(i)] = make_float4(hit ? 1.f : 0.f, t, nrm.x, nrm.y);
  out[2 * size_t(i) + 1] = make_float4(nrm.z, u, v, __int_as_float(hit ? mat : -1));
}
}  // namespace

int trace_sdf_rays(myrt_ctx* ctx, myrt_ray const* rays, uint32_t n, int steps, float eps, int any_hit,
    uint32_t const* rng_states, float* out) {
  if (n == 0) return MYRT_OK;
  void* d_rays = nullptr;
  void* d_out = nullptr;
  void* d_rng = nullptr;
  int rc = check_cuda(ctx, cudaMalloc(&d_rays, size_t(n) * 32), "SDF query buffers");
  if (!rc) rc = check_cuda(ctx, cudaMalloc(&d_out, size_t(n) * 32), "SDF query buffers");
  if (!rc && rng_states) rc = check_cuda(ctx, cudaMalloc(&d_rng, size_t(n) * 4), "SDF query buffers");
  if (!rc)
    rc = check_cuda(ctx, cudaMemcpyAsync(d_rays, rays, size_t(n) * 32, cudaMemcpyHostToDevice, ctx->stream), "upload");
  if (!rc && rng_states)
    rc = check_cuda(ctx, cudaMemcpyAsync(d_rng, rng_states, size_t(n) * 4, cudaMemcpyHostToDevice, ctx->stream),
        "upload");
  if (!rc) {
    k_trace_sdf<<<(n + 127) / 128, 128, 0, ctx->stream>>>(make_sdf_dev(ctx, steps, eps),
        static_cast<float4 const*>(d_rays), n, any_hit, static_cast<uint32_t const*>(d_rng),
        static_cast<float4*>(d_out));
    rc = check_cuda(ctx, cudaGetLastError(), "SDF query launch");
  }
  if (!rc)
    rc = check_cuda(ctx, cudaMemcpyAsync(out, d_out, size_t(n) * 32, cudaMemcpyDeviceToHost, ctx->stream), "download");
  if (!rc) rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "SDF query");
  cudaFree(d_rays);
  cudaFree(d_out);
  cudaFree(d_rng);
  return rc;
}

}  // namespace myrt_b200

// ---- reference-mode textures and cube map ------------------------------------------------
namespace myrt_b200 {
namespace {
float host_half_rn(float f) {
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

int sync_texture_table(myrt_ctx* ctx) {
  cudaFree(ctx->d_textures);
  ctx->d_textures = nullptr;
  if (ctx->textures.empty()) return MYRT_OK;
  size_t const bytes = ctx->textures.size() * sizeof(myrt_ctx::texture_slot);
  int rc = check_cuda(ctx, cudaMalloc(reinterpret_cast<void**>(&ctx->d_textures), bytes), "texture table");
  if (!rc)
    rc = check_cuda(ctx, cudaMemcpyAsync(ctx->d_textures, ctx->textures.data(), bytes, cudaMemcpyHostToDevice,
                             ctx->stream), "texture table");
  if (!rc) rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "texture table");
  return rc;
}
}  // namespace

void free_textures(myrt_ctx* ctx) {
  for (auto& t : ctx->textures) cudaFree(t.data);
  ctx->textures.clear();
  cudaFree(ctx->d_textures);
  ctx->d_textures = nullptr;
  cudaFree(ctx->cubemap);
  ctx->cubemap = nullptr;
  ctx->cubemap_size = 0;
}

}  // namespace myrt_b200

using namespace myrt_b200;

extern "C" int myrt_texture_upload(myrt_ctx* ctx, uint32_t slot, float const* rgba, uint32_t width, uint32_t height,
    uint32_t wrap) {
  if (!ctx) return MYRT_ERR_INVALID_ARGUMENT;
  if (slot >= 256 || wrap > 2 || width > 16384 || height > 16384)
    return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "texture slot < 256, wrap 0..2, sides <= 16384");
  int rc = check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  if (rc) return rc;
  cudaStreamSynchronize(ctx->stream);
  if (ctx->textures.size() <= slot) ctx->textures.resize(size_t(slot) + 1);
  auto& t = ctx->textures[slot];
  cudaFree(t.data);
  t = myrt_ctx::texture_slot{};
  if (rgba && width && height) {
    size_t const bytes = size_t(width) * height * 16;
    rc = check_cuda(ctx, cudaMalloc(reinterpret_cast<void**>(&t.data), bytes), "texture");
    if (!rc) rc = check_cuda(ctx, cudaMemcpy(t.data, rgba, bytes, cudaMemcpyHostToDevice), "texture upload");
    if (rc) {
      cudaFree(t.data);
      t = myrt_ctx::texture_slot{};
      return rc;
    }
    t.w = int(width), t.h = int(height), t.wrap = int(wrap);
  }
  ctx->render.sample_counter = 0;
  return sync_texture_table(ctx);
}

extern "C" int myrt_cubemap_upload(myrt_ctx* ctx, float const* faces, uint32_t size) {
  if (!ctx) return MYRT_ERR_INVALID_ARGUMENT;
  if (size > 16384) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "cube map faces <= 16384 texels a side");
  int rc = check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  if (rc) return rc;
  cudaStreamSynchronize(ctx->stream);
  cudaFree(ctx->cubemap);
  ctx->cubemap = nullptr;
  ctx->cubemap_size = 0;
  ctx->render.sample_counter = 0;
  if (!faces || size == 0) return MYRT_OK;
  size_t const n = size_t(6) * size * size * 4;
  std::vector<float> h(n);
  for (size_t i = 0; i < n; ++i) h[i] = host_half_rn(faces[i]);  // RGB16F storage
  rc = check_cuda(ctx, cudaMalloc(reinterpret_cast<void**>(&ctx->cubemap), n * 4), "cube map");
  if (!rc) rc = check_cuda(ctx, cudaMemcpy(ctx->cubemap, h.data(), n * 4, cudaMemcpyHostToDevice), "cube map upload");
  if (rc) {
    cudaFree(ctx->cubemap);
    ctx->cubemap = nullptr;
    return rc;
  }
  ctx->cubemap_size = int(size);
  return MYRT_OK;
}
