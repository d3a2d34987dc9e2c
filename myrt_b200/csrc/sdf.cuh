// SDF drawables on the device: the reference's sphere tracing
// (src/pt/raymarch.glsl:84-171) over flat SDF programs.
//
// The reference generates a GLSL map() per scene from an instruction tree
// (src/pathtracer/sdf.cpp:122-407) using the per-type snippets of
// src/pathtracer/sdf.hpp:399-633. Here one evaluator runs a flat post-order
// program instead: modifiers move the position of the next primitive
// (innermost first), primitives push (distance, material), operators pop two
// and push one; each node starts from the caller's material, as the generated
// code does. Parameters use the reference's block layout (float, int as a
// float value, vec3 as three floats). Material choice in operators draws from
// the pass's random stream only while the material is being loaded (after the
// normal estimate), like raymarch.glsl's _mxm/_ldm.
//
// Compiled inside the -fmad=false translation unit (wavefront.cu): every + and
// * rounds separately; sqrt and division are IEEE; pow is CUDA's powf.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "refshade.cuh"

namespace myrt_b200 {
namespace sdfk {

using rs::v3;

constexpr int kStack = 24;  // program stack depth limit (checked at upload)

enum : int {
  OP_SPHERE = 1,
  OP_BOX = 2,
  OP_TORUS = 3,
  OP_CAPSULE = 4,
  OP_MENGER = 5,
  OP_UNION = 16,
  OP_SUBTRACTION = 17,
  OP_INTERSECTION = 18,
  OP_SMOOTH_UNION = 19,
  OP_TRANSLATE = 32,
  OP_MIRROR = 33,
};

struct sdf_dev {
  int2 const* instrs;    // (op, param offset)
  int2 const* programs;  // (first, count)
  float const* params;
  float const* drawables;  // 36 floats: transformation, inverse, sdf_index bits, pad
  int n_drawables;
  int steps;
  float eps;
  float4 const* skip_sphere;  // per instruction, or null (see map)
  int2 const* skip_next;
  // cell lists of union / smooth-union tree programs, or null (see map): 3
  // int4 per program ((lo.xyz, 1 / cell) bits; (nx, ny, nz, first cell), nx =
  // 0: none; escape sphere (C.xyz, radius) bits, see march), per cell the
  // first list entry, and the entries (instruction segment start | end << 16,
  // relative to the program)
  int4 const* cell_hdr;
  int const* cell_start;
  uint32_t const* cell_list;
  // per instruction: operators of its program up to and including it, or null
  // (material loads then evaluate everything)
  int const* op_count;
};

__device__ __forceinline__ v3 abs3(v3 a) { return {fabsf(a.x), fabsf(a.y), fabsf(a.z)}; }
__device__ __forceinline__ v3 max3s(v3 a, float s) { return {rs::gmax(a.x, s), rs::gmax(a.y, s), rs::gmax(a.z, s)}; }
__device__ __forceinline__ float len2(float x, float y) { return sqrtf(x * x + y * y); }

// sdf.hpp: menger_fractal
__device__ __forceinline__ float sd_menger(v3 p) {
#pragma unroll 1
  for (int n = 0; n < 4; n++) {
    p = abs3(p);
    if (p.x < p.y) {
      float const t = p.x;
      p.x = p.y;
      p.y = t;
    }
    if (p.x < p.z) {
      float const t = p.x;
      p.x = p.z;
      p.z = t;
    }
    if (p.y < p.z) {
      float const t = p.y;
      p.y = p.z;
      p.z = t;
    }
    p.z -= 1.f / 3.f;
    p.z = -fabsf(p.z);
    p.z += 1.f / 3.f;
    p = p * 3.f;
    p.x -= 2.f;
    p.y -= 2.f;
  }
  v3 const d = abs3(p) - v3{1.f, 1.f, 1.f};
  float dis = rs::gmin(rs::gmax(d.x, rs::gmax(d.y, d.z)), 0.f) + rs::length(max3s(d, 0.f));
  // pow(3, -4) == 1/81 exactly; the IEEE quotient is its correctly rounded
  // value, which is also what the host libm's powf returns for it.
  dis *= 1.f / 81.f;
  return dis;
}

// map(p) of program `prog`; load = g_do_load_materials (material draws from rng).
//
// Exact skipping (load == false only): a group "translations, primitive,
// union or smooth union (k)" combines the running value d0 with the
// primitive's distance d1. Its result is d0 itself, bit for bit, whenever
// d1 >= d0 + k: then (d1 - d0) / k rounds to at least 1, h clamps to 1,
// mix(d1, d0, 1) = d0 and k h (1 - h) = 0 (for a union, min(d0, d1) = d0).
// The primitive's distance is at least |p - c| - R for its bounding sphere
// (c, R), so the group is skipped when |p - c| >= d0 + k + R + margin, the
// margin covering the rounding of both sides. Material loads (load == true)
// skip the same way when the per-instruction operator counts are present: the
// operators left out still draw from the random stream, in program order.
//
// Cell lists (load == false, union / smooth-union trees): when p lies in the
// program's grid, only the instruction segments listed for p's cell run, in
// program order; every subtree left out, with its operator, would have left
// the other operand's value unchanged bit for bit at every point of the cell
// (sdf_skip.hpp sdf_cell_tables), so the result is the full evaluation's. The
// bounding-sphere test above still applies inside a segment, to groups whose
// operator runs in the same segment.
__device__ __forceinline__ float map(sdf_dev const& s, int prog, v3 p, bool load, rs::rng_t* rng, int& mat) {
  int2 const pr = __ldg(s.programs + prog);
  float dist[kStack];
  int mats[kStack];
  int sp = 0;
  v3 pos = p;
  float const* G = s.params;
  // material loads skip too when every left-out operator's draw can still be
  // made (op_count): a right operand left out never decides the material (t =
  // 0); a left operand left out decides it only on a draw of exactly 1, after
  // which the whole program runs again from the saved random state
  bool const counting = load && s.op_count != nullptr;
  bool const skipping = (!load || counting) && s.skip_next != nullptr;
  float const margin = 1e-4f + 1e-6f * ((fabsf(p.x) + fabsf(p.y)) + fabsf(p.z));
  int cell_li = 0, cell_le = 0;
  bool use_cells = false;
  if ((!load || counting) && s.cell_hdr != nullptr) {
    int4 const h1 = __ldg(s.cell_hdr + 3 * prog + 1);
    if (h1.x > 0) {
      int4 const h0 = __ldg(s.cell_hdr + 3 * prog);
      float const inv = __int_as_float(h0.w);
      float const fx = (p.x - __int_as_float(h0.x)) * inv, fy = (p.y - __int_as_float(h0.y)) * inv,
                  fz = (p.z - __int_as_float(h0.z)) * inv;
      if (fx >= 0.f && fy >= 0.f && fz >= 0.f && fx < float(h1.x) && fy < float(h1.y) && fz < float(h1.z)) {
        int const c = h1.w + (int(fz) * h1.y + int(fy)) * h1.x + int(fx);
        cell_li = __ldg(s.cell_start + c);
        cell_le = __ldg(s.cell_start + c + 1);
        use_cells = true;
      }
    }
  }
  rs::rng_t const saved = counting ? *rng : rs::rng_t{};
  bool redo = false;
  // the draws of the operators in instructions [a, b) that do not run
  auto draw_gap = [&](int a, int b) {
    if (b <= a) return;
    int const n = __ldg(s.op_count + pr.x + b - 1) - (a > 0 ? __ldg(s.op_count + pr.x + a - 1) : 0);
#pragma unroll 1
    for (int i = 0; i < n; ++i)
      if (rs::random_next(*rng) >= 1.f) redo = true;
  };
#pragma unroll 1
  for (int pass = 0;; ++pass) {
  bool const fast = pass == 0;
  int kend = fast && use_cells ? 0 : pr.y;  // cells: the first segment comes from the list
  int li = fast && use_cells ? cell_li : 0, le = fast && use_cells ? cell_le : 0;
  int drawn = 0;  // counting: the operators before this instruction have drawn
  sp = 0;
  pos = p;
#pragma unroll 1
  for (int k = 0;; ++k) {
    if (k >= kend) {
      if (li >= le) break;
      uint32_t const e = __ldg(s.cell_list + li++);
      k = int(e & 0xffffu);
      kend = int(e >> 16);
      if (counting) draw_gap(drawn, k);
    }
    if (skipping && fast) {
      int2 const nx = __ldg(s.skip_next + pr.x + k);
      // in a cell segment the group's operator must run in the same segment:
      // only then is the value below it on the stack its left operand
      if (nx.x > 0 && nx.x - pr.x <= kend) {
        float4 const b = __ldg(s.skip_sphere + pr.x + k);
        float const thr = ((dist[sp - 1] + __int_as_float(nx.y)) + b.w) + margin;
        float const qx = p.x - b.x, qy = p.y - b.y, qz = p.z - b.z;
        if (thr <= 0.f || (qx * qx + qy * qy) + qz * qz >= thr * thr) {
          if (counting) draw_gap(k, nx.x - pr.x);
          drawn = nx.x - pr.x;
          k = nx.x - pr.x - 1;  // continue after the group's operator
          continue;
        }
      }
    }
    drawn = k + 1;
    int2 const in = __ldg(s.instrs + pr.x + k);
    int const o = in.y;
    int m = mat;
    float d = 0.f;
    switch (in.x) {
      case OP_TRANSLATE:
        pos = pos - v3{__ldg(G + o), __ldg(G + o + 1), __ldg(G + o + 2)};
        continue;
      case OP_MIRROR: {
        int const ax = int(__ldg(G + o));
        if (ax == 0) pos.x = fabsf(pos.x);
        else if (ax == 1) pos.y = fabsf(pos.y);
        else pos.z = fabsf(pos.z);
        continue;
      }
      case OP_SPHERE:
        m = load ? int(__ldg(G + o + 1)) : -1;
        d = rs::length(pos) - __ldg(G + o);
        break;
      case OP_BOX: {
        m = load ? int(__ldg(G + o + 3)) : -1;
        v3 const q = abs3(pos) - v3{__ldg(G + o), __ldg(G + o + 1), __ldg(G + o + 2)};
        d = rs::length(max3s(q, 0.f)) + rs::gmin(rs::gmax(q.x, rs::gmax(q.y, q.z)), 0.f);
        break;
      }
      case OP_TORUS:
        m = load ? int(__ldg(G + o + 2)) : -1;
        d = len2(len2(pos.x, pos.z) - __ldg(G + o), pos.y) - __ldg(G + o + 1);
        break;
      case OP_CAPSULE: {
        m = load ? int(__ldg(G + o + 2)) : -1;
        v3 q = pos;
        q.y -= rs::gclamp(q.y, 0.f, __ldg(G + o));
        d = rs::length(q) - __ldg(G + o + 1);
        break;
      }
      case OP_MENGER:
        m = load ? int(__ldg(G + o)) : -1;
        d = sd_menger(pos);
        break;
      default: {
        float const d1 = dist[sp - 1], d0 = dist[sp - 2];
        int const m1 = mats[sp - 1], m0 = mats[sp - 2];
        sp -= 2;
        float t;
        if (in.x == OP_SMOOTH_UNION) {
          float const k = __ldg(G + o);
          float const h = rs::gclamp(0.5f + 0.5f * (d1 - d0) / k, 0.f, 1.f);
          t = 1.f - h;
          d = rs::mixf(d1, d0, h) - k * h * (1.f - h);
        } else {
          float const r = in.x == OP_UNION ? rs::gmin(d0, d1)
                                           : (in.x == OP_SUBTRACTION ? rs::gmax(-d0, d1) : rs::gmax(d0, d1));
          t = float(r == d1);
          d = r;
        }
        m = load ? (rs::random_next(*rng) < t ? m1 : m0) : -1;
        break;
      }
    }
    dist[sp] = d;
    mats[sp] = m;
    ++sp;
    pos = p;
  }
  if (counting && fast) draw_gap(drawn, pr.y);
  if (!redo) break;
  *rng = saved;  // a left-out left operand met a draw of 1: run everything
  redo = false;
  }
  mat = mats[sp - 1];
  return dist[sp - 1];
}

struct sdf_hit {
  bool hits;
  float t;
  v3 position, normal;
  float u, v;
  int material;
};

__device__ __forceinline__ v3 xform4(float const* m, v3 v, float w) {
  return {((__ldg(m + 0) * v.x + __ldg(m + 4) * v.y) + __ldg(m + 8) * v.z) + __ldg(m + 12) * w,
      ((__ldg(m + 1) * v.x + __ldg(m + 5) * v.y) + __ldg(m + 9) * v.z) + __ldg(m + 13) * w,
      ((__ldg(m + 2) * v.x + __ldg(m + 6) * v.y) + __ldg(m + 10) * v.z) + __ldg(m + 14) * w};
}

// raymarch.glsl:116-171 for drawable `cur`. Returns hits; fills the rest
// unless hits_only.
//
// Early exit (programs with cell lists and an escape sphere): once the march moves
// forward (si > 0), is outside the sphere (C, r) widened by eps and heads away
// from C, every later point keeps a value of at least eps (sdf_skip.hpp
// sdf_cells), so no hit can follow and the march ends as the reference's
// does without a hit, only sooner (a ray that misses everything otherwise
// steps until t overflows).
__device__ __forceinline__ sdf_hit march(
    sdf_dev const& s, int cur, v3 oro, v3 ord, float tmax, bool hits_only, rs::rng_t* rng) {
  sdf_hit hit;
  hit.hits = false;
  float const* dr = s.drawables + 36 * cur;
  float const* inv = dr + 16;
  int const prog = __float_as_int(__ldg(dr + 32));
  v3 const ro = xform4(inv, oro, 1.f), rd = xform4(inv, ord, 0.f);
  float const len = rs::length(rd);
  float res = -1.f;
  float t = 10.f * s.eps;
  int si = 0;
  float4 esc = make_float4(0.f, 0.f, 0.f, -1.f);
  if (s.cell_hdr != nullptr && __ldg(s.cell_hdr + 3 * prog + 1).x > 0) {
    int4 const e = __ldg(s.cell_hdr + 3 * prog + 2);
    esc = make_float4(__int_as_float(e.x), __int_as_float(e.y), __int_as_float(e.z), __int_as_float(e.w) + s.eps);
  }
#pragma unroll 1
  for (int i = 0; i < s.steps && t / len < tmax; i++) {
    int mdum = -1;
    v3 const q = ro + rd * t / len;
    float const m = map(s, prog, q, false, rng, mdum);
    if (si == 0) si = int(rs::signf(m));
    if (fabsf(m) < s.eps) {
      res = t;
      break;
    }
    if (si > 0 && esc.w > 0.f) {
      v3 const w{q.x - esc.x, q.y - esc.y, q.z - esc.z};
      if (rs::dot(w, rd) >= 0.f && rs::dot(w, w) >= esc.w * esc.w) break;
    }
    t += float(si) * m;
  }
  if (res < 0.f) return hit;
  hit.hits = true;
  if (hits_only) return hit;
  hit.t = res / len;
  hit.position = oro + res / len * ord;
  v3 const poas = ro + res * rd;
  v3 n{0.f, 0.f, 0.f};
#pragma unroll
  for (int i = 0; i < 4; i++) {
    v3 const e = 0.5773f * (2.f * v3{float(((i + 3) >> 1) & 1), float((i >> 1) & 1), float(i & 1)} - v3{1.f, 1.f, 1.f});
    int mdum = -1;
    n = n + e * map(s, prog, poas + 0.0005f * e / len, false, rng, mdum) * len;
  }
  v3 const gn = rs::normalize(n);
  int mat = -1;
  map(s, prog, poas, true, rng, mat);
  v3 const tn{((__ldg(inv + 0) * gn.x + __ldg(inv + 1) * gn.y) + __ldg(inv + 2) * gn.z) + __ldg(inv + 3) * 0.f,
      ((__ldg(inv + 4) * gn.x + __ldg(inv + 5) * gn.y) + __ldg(inv + 6) * gn.z) + __ldg(inv + 7) * 0.f,
      ((__ldg(inv + 8) * gn.x + __ldg(inv + 9) * gn.y) + __ldg(inv + 10) * gn.z) + __ldg(inv + 11) * 0.f};
  hit.normal = rs::normalize(tn);
  float const wx = powf(fabsf(hit.normal.x), 0.5f), wy = powf(fabsf(hit.normal.y), 0.5f),
              wz = powf(fabsf(hit.normal.z), 0.5f);
  float const sw = (wx + wy) + wz;
  hit.u = ((poas.y * wx + poas.z * wy) + poas.x * wz) / sw;
  hit.v = ((poas.z * wx + poas.x * wy) + poas.y * wz) / sw;
  hit.material = mat;
  return hit;
}

}  // namespace sdfk
}  // namespace myrt_b200
