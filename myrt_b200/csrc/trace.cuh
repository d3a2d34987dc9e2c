// Closest-hit / any-hit traversal of the 8-wide quantised BVH (bvh8.hpp).
//
// One thread per ray. A node is five 16-byte words fetched with 128-bit
// read-only loads; all eight child boxes are tested from registers; hit
// internal children form a "node group" (child_base, hit bits << 24 | imask)
// and hit leaf slots a "triangle group" (tri_base, 32-bit triangle mask).
// The stack holds node groups only; at most one per tree level, so its depth
// is bounded by the tree depth checked at upload (MYRT_STACK_MAX).
//
// Triangle tests are bit-exact restatements of the reference's
// Moller-Trumbore (src/pt/intersect.glsl:3-28) using explicitly rounded
// intrinsics (no FMA contraction, IEEE division), or the watertight test of
// Woop, Benthin and Wald (JCGT 2013). Closest hit keeps the smallest t, ties
// going to the smaller prim id, so the answer does not depend on the order in
// which the tree is walked (the reference keeps the first visited,
// src/pt/pt_trace.comp:267-269).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace myrt_b200 {

constexpr int MYRT_STACK_MAX = 32;

enum : uint32_t {
  ERR_STACK_OVERFLOW = 1u << 0,
};

// ---- exact-rounding vector helpers (no contraction) ----------------------
struct f3 {
  float x, y, z;
};
__device__ __forceinline__ f3 sub3(f3 a, f3 b) { return {__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)}; }
__device__ __forceinline__ float dot3(f3 a, f3 b) {
  return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ f3 cross3(f3 a, f3 b) {
  return {__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)), __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
      __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x))};
}

// src/pt/intersect.glsl:3-28, operation for operation.
__device__ __forceinline__ bool isect_reference(f3 o, f3 d, f3 v1, f3 v2, f3 v3, float& t, float& u, float& v) {
  const float float_epsilon = 1e-23f;
  const float border_epsilon = 1e-6f;
  f3 const e1 = sub3(v2, v1);
  f3 const e2 = sub3(v3, v1);
  f3 const P = cross3(d, e2);
  float const det = dot3(e1, P);
  if (det > -float_epsilon && det < float_epsilon) return false;
  float const inv_det = __fdiv_rn(1.0f, det);
  f3 const T = sub3(o, v1);
  u = __fmul_rn(dot3(T, P), inv_det);
  if (u < -border_epsilon || u > __fadd_rn(1.0f, border_epsilon)) return false;
  f3 const Q = cross3(T, e1);
  v = __fmul_rn(dot3(d, Q), inv_det);
  if (v < -border_epsilon || __fadd_rn(u, v) > __fadd_rn(1.0f, border_epsilon)) return false;
  float const tt = __fmul_rn(dot3(e2, Q), inv_det);
  if (tt > float_epsilon) {
    t = tt;
    return true;
  }
  return false;
}

// Watertight ray/triangle test (Woop, Benthin, Wald, JCGT 2(1), 2013),
// precomputed per ray: kx, ky, kz and the shear Sx, Sy, Sz.
struct wt_ray {
  int kx, ky, kz;
  float Sx, Sy, Sz;
};
__device__ __forceinline__ float comp(f3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }
__device__ __forceinline__ wt_ray wt_setup(f3 d) {
  wt_ray w;
  float const ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
  w.kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
  w.kx = w.kz + 1 == 3 ? 0 : w.kz + 1;
  w.ky = w.kx + 1 == 3 ? 0 : w.kx + 1;
  if (comp(d, w.kz) < 0.0f) {
    int const tmp = w.kx;
    w.kx = w.ky;
    w.ky = tmp;
  }
  float const dz = comp(d, w.kz);
  w.Sx = __fdiv_rn(comp(d, w.kx), dz);
  w.Sy = __fdiv_rn(comp(d, w.ky), dz);
  w.Sz = __fdiv_rn(1.0f, dz);
  return w;
}
__device__ __forceinline__ bool isect_watertight(
    wt_ray const& w, f3 o, f3 v0, f3 v1, f3 v2, float tmin, float& t, float& u, float& v) {
  f3 const A = sub3(v0, o), B = sub3(v1, o), C = sub3(v2, o);
  float const Az0 = comp(A, w.kz), Bz0 = comp(B, w.kz), Cz0 = comp(C, w.kz);
  float const Ax = __fsub_rn(comp(A, w.kx), __fmul_rn(w.Sx, Az0));
  float const Ay = __fsub_rn(comp(A, w.ky), __fmul_rn(w.Sy, Az0));
  float const Bx = __fsub_rn(comp(B, w.kx), __fmul_rn(w.Sx, Bz0));
  float const By = __fsub_rn(comp(B, w.ky), __fmul_rn(w.Sy, Bz0));
  float const Cx = __fsub_rn(comp(C, w.kx), __fmul_rn(w.Sx, Cz0));
  float const Cy = __fsub_rn(comp(C, w.ky), __fmul_rn(w.Sy, Cz0));
  float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
  float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
  float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
  if (U == 0.0f || V == 0.0f || W == 0.0f) {
    U = float(__dsub_rn(__dmul_rn(double(Cx), double(By)), __dmul_rn(double(Cy), double(Bx))));
    V = float(__dsub_rn(__dmul_rn(double(Ax), double(Cy)), __dmul_rn(double(Ay), double(Cx))));
    W = float(__dsub_rn(__dmul_rn(double(Bx), double(Ay)), __dmul_rn(double(By), double(Ax))));
  }
  if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
  float const det = __fadd_rn(__fadd_rn(U, V), W);
  if (det == 0.0f) return false;
  float const Az = __fmul_rn(w.Sz, Az0), Bz = __fmul_rn(w.Sz, Bz0), Cz = __fmul_rn(w.Sz, Cz0);
  float const T = __fadd_rn(__fadd_rn(__fmul_rn(U, Az), __fmul_rn(V, Bz)), __fmul_rn(W, Cz));
  float const rcp = __fdiv_rn(1.0f, det);
  float const tt = __fmul_rn(T, rcp);
  if (!(tt > 0.0f) || tt < tmin) return false;
  t = tt;
  u = __fmul_rn(V, rcp);
  v = __fmul_rn(W, rcp);
  return true;
}

// ---- traversal ------------------------------------------------------------
struct trace_args {
  const float4* rays;  // 2 float4 per ray: (o, tmin), (d, tmax)
  uint32_t n;
  const uint4* nodes;  // 5 uint4 per node
  const float4* tris;  // 3 float4 per triangle
  float4* hits;        // closest: (prim bits, t, u, v)
  uint8_t* occluded;   // any-hit output
  uint32_t* stat_nodes;
  uint32_t* stat_tris;
  uint32_t* err;
  int stack_cap;       // k_trace_smem: stack entries per thread
  uint32_t const* perm;  // visiting order (thread t takes ray perm[t]); null = input order
  // two-level (instanced) walk, k_trace_inst: `nodes` is the tree over the
  // instances, whose leaf slots index `inst` (4 float4 per instance record,
  // instances.hpp); the object-space trees of the geometries live in
  // blas_nodes / blas_tris
  const uint4* blas_nodes;
  const float4* blas_tris;
  const float4* inst;
  uint32_t* stat_inst;  // instances entered per ray (STATS)
};

// Byte (s & 3) of w as an exact float: one byte permute places it in the low
// mantissa bits of 2^23 (0x4B0000bb), one subtraction removes 2^23. This keeps
// the 48 plane conversions per node off the quarter-rate conversion pipe.
__device__ __forceinline__ float q8(uint32_t w, int s) {
  return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7440u | uint32_t(s & 3))) - 8388608.0f;
}

// Two lanes of packed FP32 (sm_100 add/fma .f32x2): each lane rounds exactly
// like the scalar __fadd_rn / fmaf, two planes per instruction.
__device__ __forceinline__ uint64_t pack2(uint32_t lo, uint32_t hi) {
  uint64_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "r"(lo), "r"(hi));
  return r;
}
__device__ __forceinline__ uint64_t pack2f(float lo, float hi) { return pack2(__float_as_uint(lo), __float_as_uint(hi)); }
__device__ __forceinline__ void unpack2(uint64_t v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
// Planes of slots s and s + 1 (s even) of word w, scaled: (q - 0) * sc + of per lane.
__device__ __forceinline__ void plane2(uint32_t w, int s, uint64_t sc2, uint64_t of2, float& t0, float& t1) {
  uint64_t q = pack2(__byte_perm(w, 0x4B000000u, 0x7440u | uint32_t(s & 3)),
      __byte_perm(w, 0x4B000000u, 0x7440u | uint32_t((s + 1) & 3)));
  uint64_t const m23 = 0xCB000000CB000000ull;  // (-2^23, -2^23)
  asm("add.rn.f32x2 %0, %0, %1;" : "+l"(q) : "l"(m23));
  uint64_t t;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(t) : "l"(q), "l"(sc2), "l"(of2));
  unpack2(t, t0, t1);
}
__device__ __forceinline__ float max3f(float a, float b, float c) {
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}
__device__ __forceinline__ float min3f(float a, float b, float c) {
  float r;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}

struct hit_rec {
  int32_t prim;   // -1 = none
  float t, u, v;
  uint32_t leaf;  // index of the hit triangle in the leaf-ordered array
};

// Per-ray traversal state of the 8-wide walk. step() performs one iteration
// (visit the next node of the current group, pushing the group if siblings
// remain, then test the triangles its leaf slots hit, then pop if the group is
// exhausted) and returns false once the ray is finished. The per-thread loop
// (traverse) and the persistent kernel (which refills finished lanes with new
// rays) both drive it, so they visit the same nodes in the same order.
// SS: distance between consecutive stack entries of one ray (1 for a
// per-thread array; the block size for a shared-memory stack laid out
// [entry][thread], which keeps every push and pop free of bank conflicts).
template <int ISECT, bool ANY, int SS = 1>
struct walker {
  f3 o, d;
  float tmin, tmax;
  float idx, idy, idz;  // box-test reciprocals, zero components nudged (no 0 * inf)
  uint32_t octinv;
  wt_ray wt;
  float tbest;
  int32_t best;
  float bu, bv;
  uint32_t bleaf;
  uint2 group;
  int sp;
  int cap;  // stack entries available
  bool occluded;

  __device__ __forceinline__ void init(f3 o_, f3 d_, float tmin_, float tmax_, int cap_ = MYRT_STACK_MAX) {
    cap = cap_;
    o = o_;
    d = d_;
    tmin = tmin_;
    tmax = tmax_;
    idx = 1.0f / (fabsf(d.x) > 1e-20f ? d.x : copysignf(1e-20f, d.x));
    idy = 1.0f / (fabsf(d.y) > 1e-20f ? d.y : copysignf(1e-20f, d.y));
    idz = 1.0f / (fabsf(d.z) > 1e-20f ? d.z : copysignf(1e-20f, d.z));
    uint32_t const oct = (d.x < 0.f ? 1u : 0u) | (d.y < 0.f ? 2u : 0u) | (d.z < 0.f ? 4u : 0u);
    octinv = oct ^ 7u;
    if (ISECT == 1) wt = wt_setup(d);
    tbest = tmax;
    best = -1;
    bu = bv = 0.f;
    bleaf = 0;
    occluded = false;
    sp = 0;
    group = make_uint2(0u, 0x80000000u);  // root: bit of slot 7 ^ octinv, imask 0 -> node 0
    tg = make_uint2(0u, 0u);
  }

  // Visits the next node of the current group: pushes the group if siblings
  // remain, replaces it by the node's hit internal children and returns the
  // hit leaf triangles in tgroup. False on a stack overflow (recorded in err).
  template <bool STATS>
  __device__ __forceinline__ bool visit(uint4 const* __restrict__ nodes, uint2* stack, uint32_t* err,
      uint32_t& n_nodes, uint2& tgroup) {
    {
      uint32_t const pos = 31u - __clz(group.y & 0xff000000u);
      group.y &= ~(1u << pos);
      uint32_t const slot = (pos - 24u) ^ octinv;
      uint32_t const node_idx = group.x + __popc(group.y & 0xffu & ((1u << slot) - 1u));
      if (group.y & 0xff000000u) {
        if (sp >= cap) {
          atomicOr(err, ERR_STACK_OVERFLOW);
          return false;
        }
        stack[SS * sp++] = group;
      }
      uint4 const* np = nodes + 5 * size_t(node_idx);
      uint4 const w0 = __ldg(np + 0);
      uint4 const w1 = __ldg(np + 1);
      uint4 const w2 = __ldg(np + 2);
      uint4 const w3 = __ldg(np + 3);
      uint4 const w4 = __ldg(np + 4);
      if (STATS) ++n_nodes;
      float const sx = __uint_as_float((w0.w & 0xffu) << 23) * idx;
      float const sy = __uint_as_float(((w0.w >> 8) & 0xffu) << 23) * idy;
      float const sz = __uint_as_float(((w0.w >> 16) & 0xffu) << 23) * idz;
      float const ox = (__uint_as_float(w0.x) - o.x) * idx;
      float const oy = (__uint_as_float(w0.y) - o.y) * idy;
      float const oz = (__uint_as_float(w0.z) - o.z) * idz;
      uint32_t const imask = w0.w >> 24;
      // near/far quantised planes per axis, swapped for negative directions
      uint32_t const nx0 = idx >= 0.f ? w2.x : w3.z, nx1 = idx >= 0.f ? w2.y : w3.w;
      uint32_t const fx0 = idx >= 0.f ? w3.z : w2.x, fx1 = idx >= 0.f ? w3.w : w2.y;
      uint32_t const ny0 = idy >= 0.f ? w2.z : w4.x, ny1 = idy >= 0.f ? w2.w : w4.y;
      uint32_t const fy0 = idy >= 0.f ? w4.x : w2.z, fy1 = idy >= 0.f ? w4.y : w2.w;
      uint32_t const nz0 = idz >= 0.f ? w3.x : w4.z, nz1 = idz >= 0.f ? w3.y : w4.w;
      uint32_t const fz0 = idz >= 0.f ? w4.z : w3.x, fz1 = idz >= 0.f ? w4.w : w3.y;
      uint32_t hit_internal = 0, hit_tris = 0;
      uint64_t const sx2 = pack2f(sx, sx), sy2 = pack2f(sy, sy), sz2 = pack2f(sz, sz);
      uint64_t const ox2 = pack2f(ox, ox), oy2 = pack2f(oy, oy), oz2 = pack2f(oz, oz);
#pragma unroll
      for (int s = 0; s < 8; s += 2) {
        uint32_t const nxw = s < 4 ? nx0 : nx1, fxw = s < 4 ? fx0 : fx1;
        uint32_t const nyw = s < 4 ? ny0 : ny1, fyw = s < 4 ? fy0 : fy1;
        uint32_t const nzw = s < 4 ? nz0 : nz1, fzw = s < 4 ? fz0 : fz1;
        float tnx[2], tfx[2], tny[2], tfy[2], tnz[2], tfz[2];
        plane2(nxw, s, sx2, ox2, tnx[0], tnx[1]);
        plane2(fxw, s, sx2, ox2, tfx[0], tfx[1]);
        plane2(nyw, s, sy2, oy2, tny[0], tny[1]);
        plane2(fyw, s, sy2, oy2, tfy[0], tfy[1]);
        plane2(nzw, s, sz2, oz2, tnz[0], tnz[1]);
        plane2(fzw, s, sz2, oz2, tfz[0], tfz[1]);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          int const c = s + h;
          float const tn = max3f(tnx[h], tny[h], fmaxf(tnz[h], tmin));
          float const tf = min3f(tfx[h], tfy[h], fminf(tfz[h], tbest));
          uint32_t const meta = ((c < 4 ? w1.z : w1.w) >> (8 * (c & 3))) & 0xffu;
          if (meta != 0u && tn <= tf * 1.00000024f) {
            if (imask & (1u << c)) {
              hit_internal |= 1u << ((c ^ octinv) + 24u);
            } else {
              uint32_t const cnt = meta >> 5, off = meta & 31u;
              hit_tris |= ((1u << cnt) - 1u) << off;
            }
          }
        }
      }
      group = make_uint2(w1.x, hit_internal | imask);
      tgroup = make_uint2(w1.y, hit_tris);
    }
    return true;
  }

  // Tests leaf triangle `leaf`. False when an any-hit query is answered.
  template <bool STATS>
  __device__ __forceinline__ bool test(float4 const* __restrict__ tris, uint32_t leaf, uint32_t& n_tris) {
    float4 const* tp = tris + 3 * size_t(leaf);
    float4 const p0 = __ldg(tp + 0);
    float4 const p1 = __ldg(tp + 1);
    float4 const p2 = __ldg(tp + 2);
    if (STATS) ++n_tris;
    float t, u, v;
    bool hit;
    if (ISECT == 0)
      hit = isect_reference(o, d, f3{p0.x, p0.y, p0.z}, f3{p1.x, p1.y, p1.z}, f3{p2.x, p2.y, p2.z}, t, u, v) &&
          t >= tmin;
    else
      hit = isect_watertight(wt, o, f3{p0.x, p0.y, p0.z}, f3{p1.x, p1.y, p1.z}, f3{p2.x, p2.y, p2.z}, tmin, t, u, v);
    if (!hit) return true;
    int32_t const prim = __float_as_int(p0.w);
    if (ANY) {
      if (t < tmax) {
        occluded = true;
        return false;
      }
    } else if (t < tbest || (t == tbest && best >= 0 && prim < best)) {
      tbest = t;
      best = prim;
      bu = u;
      bv = v;
      bleaf = leaf;
    }
    return true;
  }

  // One iteration: visit a node, test all the triangles it hit, pop if the
  // current group is exhausted.
  template <bool STATS>
  __device__ __forceinline__ bool step(uint4 const* __restrict__ nodes, float4 const* __restrict__ tris, uint2* stack,
      uint32_t* err, uint32_t& n_nodes, uint32_t& n_tris) {
    uint2 tgroup = make_uint2(0u, 0u);
    if (group.y & 0xff000000u) {
      if (!visit<STATS>(nodes, stack, err, n_nodes, tgroup)) return false;
    } else {
      group.y = 0;
    }
    while (tgroup.y) {
      uint32_t const b = __ffs(tgroup.y) - 1u;
      tgroup.y &= tgroup.y - 1u;
      if (!test<STATS>(tris, tgroup.x + b, n_tris)) return false;
    }
    if (!(group.y & 0xff000000u)) {
      if (sp == 0) return false;
      group = stack[SS * --sp];
    }
    return true;
  }

  // One unit of work per iteration: one triangle, one node or one pop, in the
  // same order as step(), so lanes of a warp stay busy with similar amounts of
  // work. Uses the member tg for triangles carried between iterations.
  uint2 tg;
  template <bool STATS>
  __device__ __forceinline__ bool step_unit(uint4 const* __restrict__ nodes, float4 const* __restrict__ tris,
      uint2* stack, uint32_t* err, uint32_t& n_nodes, uint32_t& n_tris) {
    if (tg.y) {
      uint32_t const b = __ffs(tg.y) - 1u;
      tg.y &= tg.y - 1u;
      return test<STATS>(tris, tg.x + b, n_tris);
    }
    if (group.y & 0xff000000u) return visit<STATS>(nodes, stack, err, n_nodes, tg);
    if (sp == 0) return false;
    group = stack[SS * --sp];
    return true;
  }

  __device__ __forceinline__ void result(hit_rec& h) const {
    h.prim = best;
    h.t = best >= 0 ? tbest : tmax;
    h.u = best >= 0 ? bu : 0.f;
    h.v = best >= 0 ? bv : 0.f;
    h.leaf = bleaf;
  }
};

// Walks the tree for one ray. Closest hit (ANY = false): fills h and returns
// whether a triangle was hit. Any hit (ANY = true): returns true at the first
// triangle with tmin <= t < tmax. n_nodes / n_tris count fetched nodes and
// tested triangles when STATS.
template <int ISECT, bool ANY, bool STATS, bool UNIT = false>
__device__ __forceinline__ bool traverse(uint4 const* __restrict__ nodes, float4 const* __restrict__ tris, f3 o, f3 d,
    float tmin, float tmax, hit_rec& h, uint32_t* err, uint32_t& n_nodes, uint32_t& n_tris) {
  uint2 stack[MYRT_STACK_MAX];
  walker<ISECT, ANY> w;
  w.init(o, d, tmin, tmax);
  if (UNIT) {
    while (w.template step_unit<STATS>(nodes, tris, stack, err, n_nodes, n_tris)) {
    }
  } else {
    while (w.template step<STATS>(nodes, tris, stack, err, n_nodes, n_tris)) {
    }
  }
  if (ANY) return w.occluded;
  w.result(h);
  return h.prim >= 0;
}

template <int ISECT, bool ANY, bool STATS>
__device__ __forceinline__ void store_result(trace_args const& a, uint32_t i, bool r, hit_rec const& h,
    uint32_t n_nodes, uint32_t n_tris) {
  if (ANY) {
    a.occluded[i] = r ? 1 : 0;
  } else {
    a.hits[i] = make_float4(__int_as_float(h.prim), h.t, h.u, h.v);
  }
  if (STATS) {
    a.stat_nodes[i] = n_nodes;
    a.stat_tris[i] = n_tris;
  }
}

// Two-level walk for instanced scenes: the reference's bvh_traverse_global
// with visit_object_aabb (src/pt/pt_trace.comp:98-116, 284-309). The tree over
// the instances is walked with the world ray; each instance leaf moves the ray
// into the instance's object space -- (inverse_transformation * vec4(o, 1)).xyz
// and (inverse_transformation * vec4(d, 0)).xyz, every product and sum rounded
// separately, left to right, the direction not renormalised -- and walks the
// geometry's object-space tree on the same stack with the same t scale.
// Triangles are tested in object space with the object-space ray, so t, u and v
// equal the reference's bit for bit; ties in t go to the smaller global prim id
// (the drawable's first prim id + the triangle's index in its geometry).
// Entering an instance saves the instance level's state on the stack (its node
// group, the instance leaves still pending and the world ray: 5 entries), so
// none of it occupies registers during the instance's walk.
constexpr int kInstanceSave = 5;

template <int ISECT, bool ANY>
__device__ __forceinline__ void set_walker_ray(walker<ISECT, ANY>& w, f3 o, f3 d) {
  w.o = o;
  w.d = d;
  w.idx = 1.0f / (fabsf(d.x) > 1e-20f ? d.x : copysignf(1e-20f, d.x));
  w.idy = 1.0f / (fabsf(d.y) > 1e-20f ? d.y : copysignf(1e-20f, d.y));
  w.idz = 1.0f / (fabsf(d.z) > 1e-20f ? d.z : copysignf(1e-20f, d.z));
  uint32_t const oct = (d.x < 0.f ? 1u : 0u) | (d.y < 0.f ? 2u : 0u) | (d.z < 0.f ? 4u : 0u);
  w.octinv = oct ^ 7u;
  if (ISECT == 1) w.wt = wt_setup(d);
}

// row . (x, y, z, w) summed left to right, each step rounded
__device__ __forceinline__ float row_dot(float4 r, f3 v, float vw) {
  return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(r.x, v.x), __fmul_rn(r.y, v.y)), __fmul_rn(r.z, v.z)),
      __fmul_rn(r.w, vw));
}

// Walks the two-level structure for one ray: as traverse(), n_inst counts the
// instances entered.
template <int ISECT, bool ANY, bool STATS>
__device__ __forceinline__ bool traverse_two_level(trace_args const& a, f3 o, f3 d, float tmin, float tmax,
    hit_rec& h, uint32_t& n_nodes, uint32_t& n_tris, uint32_t& n_inst) {
  uint2 stack[MYRT_STACK_MAX];
  walker<ISECT, ANY> w;
  w.init(o, d, tmin, tmax);
  uint2 pending = make_uint2(0u, 0u);  // instance leaves of the last top-level node
  bool answered = false;
  while (!answered) {
    while (pending.y) {
      uint32_t const b = __ffs(pending.y) - 1u;
      pending.y &= pending.y - 1u;
      int const save = w.sp;
      if (save + kInstanceSave > w.cap) {
        atomicOr(a.err, ERR_STACK_OVERFLOW);
        answered = true;
        break;
      }
      stack[save] = w.group;
      stack[save + 1] = pending;
      stack[save + 2] = make_uint2(__float_as_uint(w.o.x), __float_as_uint(w.o.y));
      stack[save + 3] = make_uint2(__float_as_uint(w.o.z), __float_as_uint(w.d.x));
      stack[save + 4] = make_uint2(__float_as_uint(w.d.y), __float_as_uint(w.d.z));
      w.sp = save + kInstanceSave;
      float4 const* r = a.inst + 4 * size_t(pending.x + b);
      float4 const r0 = __ldg(r + 0), r1 = __ldg(r + 1), r2 = __ldg(r + 2);
      int4 const meta = __ldg(reinterpret_cast<int4 const*>(r + 3));
      if (STATS) ++n_inst;
      f3 const oo{row_dot(r0, w.o, 1.0f), row_dot(r1, w.o, 1.0f), row_dot(r2, w.o, 1.0f)};
      f3 const od{row_dot(r0, w.d, 0.0f), row_dot(r1, w.d, 0.0f), row_dot(r2, w.d, 0.0f)};
      set_walker_ray(w, oo, od);
      w.group = make_uint2(uint32_t(meta.x), 0x80000000u);  // the geometry's root
      int32_t const prim_base = meta.y;
      // the instance's walk, on the stack above the saved state
      while (true) {
        uint2 tgroup = make_uint2(0u, 0u);
        if (w.group.y & 0xff000000u) {
          if (!w.template visit<STATS>(a.blas_nodes, stack, a.err, n_nodes, tgroup)) {
            answered = true;
            break;
          }
        } else {
          w.group.y = 0;
        }
        while (tgroup.y) {
          uint32_t const tb = __ffs(tgroup.y) - 1u;
          tgroup.y &= tgroup.y - 1u;
          float4 const* tp = a.blas_tris + 3 * size_t(tgroup.x + tb);
          float4 const p0 = __ldg(tp + 0);
          float4 const p1 = __ldg(tp + 1);
          float4 const p2 = __ldg(tp + 2);
          if (STATS) ++n_tris;
          float t, u, v;
          bool hit;
          if (ISECT == 0)
            hit = isect_reference(w.o, w.d, f3{p0.x, p0.y, p0.z}, f3{p1.x, p1.y, p1.z}, f3{p2.x, p2.y, p2.z}, t, u,
                      v) && t >= w.tmin;
          else
            hit = isect_watertight(w.wt, w.o, f3{p0.x, p0.y, p0.z}, f3{p1.x, p1.y, p1.z}, f3{p2.x, p2.y, p2.z},
                w.tmin, t, u, v);
          if (!hit) continue;
          int32_t const prim = prim_base + __float_as_int(p0.w);
          if (ANY) {
            if (t < w.tmax) {
              w.occluded = true;
              answered = true;
              break;
            }
          } else if (t < w.tbest || (t == w.tbest && w.best >= 0 && prim < w.best)) {
            w.tbest = t;
            w.best = prim;
            w.bu = u;
            w.bv = v;
          }
        }
        if (answered) break;
        if (!(w.group.y & 0xff000000u)) {
          if (w.sp == save + kInstanceSave) break;
          w.group = stack[--w.sp];
        }
      }
      if (answered) break;
      uint2 const s2 = stack[save + 2], s3 = stack[save + 3], s4 = stack[save + 4];
      w.group = stack[save];
      pending = stack[save + 1];
      w.sp = save;
      set_walker_ray(w, f3{__uint_as_float(s2.x), __uint_as_float(s2.y), __uint_as_float(s3.x)},
          f3{__uint_as_float(s3.y), __uint_as_float(s4.x), __uint_as_float(s4.y)});
    }
    if (answered) break;
    if (w.group.y & 0xff000000u) {
      if (!w.template visit<STATS>(a.nodes, stack, a.err, n_nodes, pending)) break;
      if (pending.y) continue;
    } else {
      w.group.y = 0;
    }
    if (!(w.group.y & 0xff000000u)) {
      if (w.sp == 0) break;
      w.group = stack[--w.sp];
    }
  }
  if (ANY) return w.occluded;
  h.prim = w.best;
  h.t = w.best >= 0 ? w.tbest : tmax;
  h.u = w.best >= 0 ? w.bu : 0.f;
  h.v = w.best >= 0 ? w.bv : 0.f;
  h.leaf = 0;
  return h.prim >= 0;
}

// The same walk as one loop whose every iteration visits one node of either
// level, so lanes of a warp in the instance tree and lanes inside instances
// run the same node-visit instructions together. The leaves of an instance-tree
// node become a tagged stack entry (first record | 1 << 31, leaf bits); popping
// one enters its lowest instance (the rest is pushed back), saving the world
// ray as three stack entries above which the instance's walk runs; popping
// back down to them leaves the instance. Stack use: instance depth x 2 +
// object depth + 3 (checked at upload).
constexpr int kInstanceRay = 3;

template <int ISECT, bool ANY, bool STATS>
__device__ __forceinline__ bool traverse_two_level_flat(trace_args const& a, f3 o, f3 d, float tmin, float tmax,
    hit_rec& h, uint32_t& n_nodes, uint32_t& n_tris, uint32_t& n_inst) {
  uint2 stack[MYRT_STACK_MAX];
  walker<ISECT, ANY> w;
  w.init(o, d, tmin, tmax);
  int base_sp = -1;  // stack depth at which the current instance's walk ends; -1 = instance level
  int32_t prim_base = 0;
  while (true) {
    if (w.group.y & 0xff000000u) {
      uint2 tg = make_uint2(0u, 0u);
      if (!w.template visit<STATS>(base_sp >= 0 ? a.blas_nodes : a.nodes, stack, a.err, n_nodes, tg)) break;
      if (tg.y) {
        if (base_sp < 0) {  // instance leaves: visited after the node's children
          if (w.sp >= w.cap) {
            atomicOr(a.err, ERR_STACK_OVERFLOW);
            break;
          }
          stack[w.sp++] = make_uint2(tg.x | 0x80000000u, tg.y);
        } else {
          bool answered = false;
          while (tg.y) {
            uint32_t const tb = __ffs(tg.y) - 1u;
            tg.y &= tg.y - 1u;
            float4 const* tp = a.blas_tris + 3 * size_t(tg.x + tb);
            float4 const p0 = __ldg(tp + 0);
            float4 const p1 = __ldg(tp + 1);
            float4 const p2 = __ldg(tp + 2);
            if (STATS) ++n_tris;
            float t, u, v;
            bool hit;
            if (ISECT == 0)
              hit = isect_reference(w.o, w.d, f3{p0.x, p0.y, p0.z}, f3{p1.x, p1.y, p1.z}, f3{p2.x, p2.y, p2.z}, t, u,
                        v) && t >= w.tmin;
            else
              hit = isect_watertight(w.wt, w.o, f3{p0.x, p0.y, p0.z}, f3{p1.x, p1.y, p1.z}, f3{p2.x, p2.y, p2.z},
                  w.tmin, t, u, v);
            if (!hit) continue;
            int32_t const prim = prim_base + __float_as_int(p0.w);
            if (ANY) {
              if (t < w.tmax) {
                w.occluded = true;
                answered = true;
                break;
              }
            } else if (t < w.tbest || (t == w.tbest && w.best >= 0 && prim < w.best)) {
              w.tbest = t;
              w.best = prim;
              w.bu = u;
              w.bv = v;
            }
          }
          if (answered) break;
        }
      }
      if (w.group.y & 0xff000000u) continue;
    }
    w.group.y = 0;
    if (base_sp >= 0 && w.sp == base_sp) {  // leave the instance: the world ray comes back
      uint2 const s0 = stack[w.sp - 3], s1 = stack[w.sp - 2], s2 = stack[w.sp - 1];
      w.sp -= kInstanceRay;
      set_walker_ray(w, f3{__uint_as_float(s0.x), __uint_as_float(s0.y), __uint_as_float(s1.x)},
          f3{__uint_as_float(s1.y), __uint_as_float(s2.x), __uint_as_float(s2.y)});
      base_sp = -1;
      continue;
    }
    if (w.sp == 0) break;
    uint2 const e = stack[--w.sp];
    if (!(e.x & 0x80000000u)) {
      w.group = e;
      continue;
    }
    // an instance leaf group: enter its lowest instance, keep the rest
    uint32_t const b = __ffs(e.y) - 1u;
    uint32_t const rest = e.y & (e.y - 1u);
    if (rest) stack[w.sp++] = make_uint2(e.x, rest);
    if (w.sp + kInstanceRay > w.cap) {
      atomicOr(a.err, ERR_STACK_OVERFLOW);
      break;
    }
    stack[w.sp] = make_uint2(__float_as_uint(w.o.x), __float_as_uint(w.o.y));
    stack[w.sp + 1] = make_uint2(__float_as_uint(w.o.z), __float_as_uint(w.d.x));
    stack[w.sp + 2] = make_uint2(__float_as_uint(w.d.y), __float_as_uint(w.d.z));
    w.sp += kInstanceRay;
    base_sp = w.sp;
    float4 const* r = a.inst + 4 * size_t((e.x & 0x7fffffffu) + b);
    float4 const r0 = __ldg(r + 0), r1 = __ldg(r + 1), r2 = __ldg(r + 2);
    int4 const meta = __ldg(reinterpret_cast<int4 const*>(r + 3));
    if (STATS) ++n_inst;
    f3 const oo{row_dot(r0, w.o, 1.0f), row_dot(r1, w.o, 1.0f), row_dot(r2, w.o, 1.0f)};
    f3 const od{row_dot(r0, w.d, 0.0f), row_dot(r1, w.d, 0.0f), row_dot(r2, w.d, 0.0f)};
    set_walker_ray(w, oo, od);
    w.group = make_uint2(uint32_t(meta.x), 0x80000000u);  // the geometry's root
    prim_base = meta.y;
  }
  if (ANY) return w.occluded;
  h.prim = w.best;
  h.t = w.best >= 0 ? w.tbest : tmax;
  h.u = w.best >= 0 ? w.bu : 0.f;
  h.v = w.best >= 0 ? w.bv : 0.f;
  h.leaf = 0;
  return h.prim >= 0;
}

// One thread per ray over the two-level structure.
template <int ISECT, bool ANY, bool STATS, bool FLAT = true>
__global__ void __launch_bounds__(128, 8) k_trace_inst(trace_args a) {
  uint32_t const t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n) return;
  uint32_t const i = a.perm ? __ldg(a.perm + t) : t;
  float4 const r0 = __ldg(a.rays + 2 * size_t(i));
  float4 const r1 = __ldg(a.rays + 2 * size_t(i) + 1);
  hit_rec h;
  uint32_t n_nodes = 0, n_tris = 0, n_inst = 0;
  bool const r = FLAT ? traverse_two_level_flat<ISECT, ANY, STATS>(a, f3{r0.x, r0.y, r0.z}, f3{r1.x, r1.y, r1.z},
                             r0.w, r1.w, h, n_nodes, n_tris, n_inst)
                       : traverse_two_level<ISECT, ANY, STATS>(a, f3{r0.x, r0.y, r0.z}, f3{r1.x, r1.y, r1.z}, r0.w,
                             r1.w, h, n_nodes, n_tris, n_inst);
  store_result<ISECT, ANY, STATS>(a, i, r, h, n_nodes, n_tris);
  if (STATS && a.stat_inst) a.stat_inst[i] = n_inst;
}

// One thread per ray, traversal stack in shared memory ([entry][thread],
// a.stack_cap entries per thread; dynamic shared memory of
// a.stack_cap * 128 * 8 bytes).
template <int ISECT, bool ANY, bool STATS>
__global__ void __launch_bounds__(128, 8) k_trace_smem(trace_args a) {
  extern __shared__ uint2 sstack[];
  uint32_t const t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n) return;
  uint32_t const i = a.perm ? __ldg(a.perm + t) : t;
  float4 const r0 = __ldg(a.rays + 2 * size_t(i));
  float4 const r1 = __ldg(a.rays + 2 * size_t(i) + 1);
  walker<ISECT, ANY, 128> w;
  w.init(f3{r0.x, r0.y, r0.z}, f3{r1.x, r1.y, r1.z}, r0.w, r1.w, a.stack_cap);
  uint32_t n_nodes = 0, n_tris = 0;
  uint2* stack = sstack + threadIdx.x;
  while (w.template step<STATS>(a.nodes, a.tris, stack, a.err, n_nodes, n_tris)) {
  }
  hit_rec h;
  if (!ANY) w.result(h);
  store_result<ISECT, ANY, STATS>(a, i, ANY ? w.occluded : h.prim >= 0, h, n_nodes, n_tris);
}

// One thread per ray. MINB = resident 128-thread blocks per SM the compiler
// must allow (8 leaves it 64 registers; more blocks cap the register count).
template <int ISECT, bool ANY, bool STATS, int MINB = 8, bool UNIT = false>
__global__ void __launch_bounds__(128, MINB) k_trace(trace_args a) {
  uint32_t const t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n) return;
  uint32_t const i = a.perm ? __ldg(a.perm + t) : t;
  float4 const r0 = __ldg(a.rays + 2 * size_t(i));
  float4 const r1 = __ldg(a.rays + 2 * size_t(i) + 1);
  hit_rec h;
  uint32_t n_nodes = 0, n_tris = 0;
  bool const r = traverse<ISECT, ANY, STATS, UNIT>(a.nodes, a.tris, f3{r0.x, r0.y, r0.z}, f3{r1.x, r1.y, r1.z}, r0.w,
      r1.w, h, a.err, n_nodes, n_tris);
  store_result<ISECT, ANY, STATS>(a, i, r, h, n_nodes, n_tris);
}

// Persistent variant: a fixed grid of warps; whenever at least `refill` lanes
// of a warp have finished their ray, those lanes take the next rays from a
// global counter (one atomic per warp), so warps stay full instead of waiting
// for their slowest ray (Aila and Laine, HPG 2009: persistent threads with
// dynamic fetch). *next must be 0 at launch.
template <int ISECT, bool ANY, bool STATS>
__global__ void __launch_bounds__(128) k_trace_persistent(trace_args a, uint32_t* __restrict__ next, uint32_t refill) {
  uint2 stack[MYRT_STACK_MAX];
  walker<ISECT, ANY> w;
  uint32_t const lane = threadIdx.x & 31u;
  uint32_t ray = 0;
  uint32_t n_nodes = 0, n_tris = 0;
  bool active = false;
  bool pool_left = true;  // warp-uniform
  while (true) {
    uint32_t const idle = __ballot_sync(0xffffffffu, !active);
    if (pool_left && __popc(idle) >= int(idle == 0xffffffffu ? 1u : refill)) {
      uint32_t const leader = __ffs(idle) - 1u;
      uint32_t base = 0;
      if (lane == leader) base = atomicAdd(next, uint32_t(__popc(idle)));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (base + uint32_t(__popc(idle)) >= a.n) pool_left = false;
      if (!active) {
        uint32_t const mine = base + __popc(idle & ((1u << lane) - 1u));
        if (mine < a.n) {
          uint32_t const ri = a.perm ? __ldg(a.perm + mine) : mine;
          float4 const r0 = __ldg(a.rays + 2 * size_t(ri));
          float4 const r1 = __ldg(a.rays + 2 * size_t(ri) + 1);
          w.init(f3{r0.x, r0.y, r0.z}, f3{r1.x, r1.y, r1.z}, r0.w, r1.w);
          ray = ri;
          n_nodes = n_tris = 0;
          active = true;
        }
      }
    }
    if (!__any_sync(0xffffffffu, active)) break;
    if (active && !w.template step<STATS>(a.nodes, a.tris, stack, a.err, n_nodes, n_tris)) {
      hit_rec h;
      if (!ANY) w.result(h);
      store_result<ISECT, ANY, STATS>(a, ray, ANY ? w.occluded : h.prim >= 0, h, n_nodes, n_tris);
      active = false;
    }
  }
}

}  // namespace myrt_b200
