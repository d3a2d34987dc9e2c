// Device BVH build: linear BVH (Morton order + radix tree) collapsed into the
// 80-byte 8-wide quantised nodes of bvh8.hpp, entirely on the GPU.
//
// The host builder (bvh8.cpp) makes better trees (binned SAH, SAH-optimal
// 8-wide collapse) but takes O(n log n) host time per upload; this builder
// rebuilds a 2 M-triangle scene in milliseconds, which is what dynamic scenes
// need (the reference rebuilds its TLAS on the host whenever an instance
// moves, src/pathtracer/scene.cpp:336-344). Answers of the ray queries do not
// depend on the tree (ties go to the smaller prim id), only their speed.
//
//   k_prim_boxes   padded triangle boxes (+1e-5, as generate_triangle_bounds,
//                  bvh.cpp:136-152) and the bounds of their centres
//   k_morton       63-bit Morton codes of the centres (21 bits per axis)
//   (CUB)          radix sort of (code, prim) pairs
//   k_radix_tree   binary radix tree over the sorted codes (Karras, "Maximizing
//                  parallelism in the construction of BVHs, octrees and k-d
//                  trees", HPG 2012); equal codes are ordered by position
//   k_boxes_up     internal boxes bottom-up, the second child to arrive at a
//                  node computes its box (atomic arrival counters)
//   k_collapse     one wide node per thread, level by level: expand the
//                  largest-area child with more than 4 triangles until 8
//                  children, then quantise, assign slots by octant and emit
//                  the node, its triangles and its internal children
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <vector>

#include "bvh8.hpp"
#include "bvh8_device.hpp"

namespace myrt_b200 {
namespace {

constexpr uint32_t kLeafBit = 0x80000000u;
constexpr uint32_t kNone = 0xffffffffu;
constexpr int kMaxLeaf = 4;

struct ibox {
  float4 lo, hi;  // w unused
};

__device__ __forceinline__ uint32_t f2ord(float f) {  // order-preserving float -> uint
  uint32_t const u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(uint32_t u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__global__ void k_prim_boxes(float const* __restrict__ pos, uint32_t n, float pad, ibox* __restrict__ boxes,
    uint32_t* __restrict__ cbounds) {
  uint32_t const i = blockIdx.x * blockDim.x + threadIdx.x;
  float c[3] = {0.f, 0.f, 0.f};
  bool const ok = i < n;
  if (ok) {
    float const* v = pos + 9 * size_t(i);
    float lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
      lo[a] = fminf(fminf(v[a], v[3 + a]), v[6 + a]) - pad;
      hi[a] = fmaxf(fmaxf(v[a], v[3 + a]), v[6 + a]) + pad;
      c[a] = 0.5f * (lo[a] + hi[a]);
    }
    boxes[i] = ibox{make_float4(lo[0], lo[1], lo[2], 0.f), make_float4(hi[0], hi[1], hi[2], 0.f)};
  }
  // block-wide min / max of the centres, then one atomic per block and bound
  __shared__ uint32_t s[6];
  if (threadIdx.x < 6) s[threadIdx.x] = threadIdx.x < 3 ? 0xffffffffu : 0u;
  __syncthreads();
  if (ok)
    for (int a = 0; a < 3; ++a) {
      atomicMin(&s[a], f2ord(c[a]));
      atomicMax(&s[3 + a], f2ord(c[a]));
    }
  __syncthreads();
  if (threadIdx.x < 3) atomicMin(&cbounds[threadIdx.x], s[threadIdx.x]);
  else if (threadIdx.x < 6) atomicMax(&cbounds[threadIdx.x], s[threadIdx.x]);
}

__device__ __forceinline__ uint64_t spread21(uint32_t v) {
  uint64_t x = v & 0x1fffffu;
  x = (x | (x << 32)) & 0x1f00000000ffffull;
  x = (x | (x << 16)) & 0x1f0000ff0000ffull;
  x = (x | (x << 8)) & 0x100f00f00f00f00full;
  x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
  x = (x | (x << 2)) & 0x1249249249249249ull;
  return x;
}

__global__ void k_morton(ibox const* __restrict__ boxes, uint32_t n, uint32_t const* __restrict__ cbounds,
    uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  uint32_t const i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  ibox const b = boxes[i];
  float const c[3] = {0.5f * (b.lo.x + b.hi.x), 0.5f * (b.lo.y + b.hi.y), 0.5f * (b.lo.z + b.hi.z)};
  uint64_t code = 0;
  for (int a = 0; a < 3; ++a) {
    float const lo = ord2f(cbounds[a]), hi = ord2f(cbounds[3 + a]);
    float const ext = hi - lo;
    float const t = ext > 0.f ? (c[a] - lo) / ext : 0.f;
    uint32_t const q = uint32_t(fminf(fmaxf(t * 2097152.f, 0.f), 2097151.f));
    code |= spread21(q) << a;
  }
  keys[i] = code;
  vals[i] = i;
}

__device__ __forceinline__ int delta(uint64_t const* k, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  uint64_t const a = k[i], b = k[j];
  if (a == b) return 64 + __clz(uint32_t(i) ^ uint32_t(j));
  return __clzll(a ^ b);
}

// internal node i: children (leaf bit | index), prim range, parents
__global__ void k_radix_tree(uint64_t const* __restrict__ keys, int n, uint2* __restrict__ child,
    uint2* __restrict__ range, uint32_t* __restrict__ parent_internal, uint32_t* __restrict__ parent_leaf) {
  int const i = int(blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= n - 1) return;
  int const d = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
  int const dmin = delta(keys, n, i, i - d);
  int lmax = 2;
  while (delta(keys, n, i, i + lmax * d) > dmin) lmax *= 2;
  int l = 0;
  for (int t = lmax / 2; t >= 1; t /= 2)
    if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
  int const j = i + l * d;
  int const dnode = delta(keys, n, i, j);
  int s = 0;
  int t = l;
  do {
    t = (t + 1) / 2;
    if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
  } while (t > 1);
  int const gamma = i + s * d + min(d, 0);
  int const first = min(i, j), last = max(i, j);
  uint32_t const left = first == gamma ? (kLeafBit | uint32_t(gamma)) : uint32_t(gamma);
  uint32_t const right = last == gamma + 1 ? (kLeafBit | uint32_t(gamma + 1)) : uint32_t(gamma + 1);
  child[i] = make_uint2(left, right);
  range[i] = make_uint2(uint32_t(first), uint32_t(last));
  if (left & kLeafBit) parent_leaf[gamma] = uint32_t(i);
  else parent_internal[gamma] = uint32_t(i);
  if (right & kLeafBit) parent_leaf[gamma + 1] = uint32_t(i);
  else parent_internal[gamma + 1] = uint32_t(i);
}

__device__ __forceinline__ ibox load_box(uint32_t ref, ibox const* leaf_boxes, uint32_t const* order,
    ibox const* inner) {
  if (ref & kLeafBit) return leaf_boxes[order[ref & ~kLeafBit]];
  ibox b;
  b.lo = __ldcg(&inner[ref].lo);
  b.hi = __ldcg(&inner[ref].hi);
  return b;
}
__device__ __forceinline__ ibox merge(ibox a, ibox b) {
  return ibox{make_float4(fminf(a.lo.x, b.lo.x), fminf(a.lo.y, b.lo.y), fminf(a.lo.z, b.lo.z), 0.f),
      make_float4(fmaxf(a.hi.x, b.hi.x), fmaxf(a.hi.y, b.hi.y), fmaxf(a.hi.z, b.hi.z), 0.f)};
}

__global__ void k_boxes_up(ibox const* __restrict__ leaf_boxes, uint32_t const* __restrict__ order, int n,
    uint2 const* __restrict__ child, uint32_t const* __restrict__ parent_internal,
    uint32_t const* __restrict__ parent_leaf, uint32_t* __restrict__ arrivals, ibox* __restrict__ inner) {
  int const l = int(blockIdx.x * blockDim.x + threadIdx.x);
  if (l >= n || n < 2) return;
  uint32_t node = parent_leaf[l];
  while (node != kNone) {
    __threadfence();
    if (atomicAdd(&arrivals[node], 1u) == 0u) return;  // the sibling is not done yet
    uint2 const c = child[node];
    ibox const b = merge(load_box(c.x, leaf_boxes, order, inner), load_box(c.y, leaf_boxes, order, inner));
    __stcg(&inner[node].lo, b.lo);
    __stcg(&inner[node].hi, b.hi);
    node = parent_internal[node];
  }
}

struct collapse_item {
  uint32_t ref;   // binary node (leaf bit | index)
  uint32_t wide;  // wide node index to write
  uint32_t depth;
};

struct collapse_args {
  ibox const* leaf_boxes;  // per prim (input order)
  uint32_t const* order;   // sorted position -> prim
  uint2 const* child;
  uint2 const* range;
  ibox const* inner;
  float const* pos;        // world triangles, 9 floats per prim
  bvh8_node* nodes;
  float4* tris;            // 3 per triangle
  uint32_t* counters;      // [0] wide nodes, [1] triangles, [2] / [5] queue lengths, [3] max depth, [4] leaf slots
  collapse_item const* in;
  uint32_t const* n_in;    // this level's queue length (device)
  collapse_item* out;
  uint32_t* n_out;         // the next level's (zeroed before the launch)
  int n;
};

__device__ __forceinline__ uint32_t prim_count(collapse_args const& a, uint32_t ref) {
  if (ref & kLeafBit) return 1u;
  uint2 const r = a.range[ref];
  return r.y - r.x + 1u;
}
__device__ __forceinline__ uint2 prim_range(collapse_args const& a, uint32_t ref) {
  if (ref & kLeafBit) return make_uint2(ref & ~kLeafBit, ref & ~kLeafBit);
  return a.range[ref];
}
__device__ __forceinline__ float area(ibox const& b) {
  float const dx = b.hi.x - b.lo.x, dy = b.hi.y - b.lo.y, dz = b.hi.z - b.lo.z;
  return ((dx + dy) * dz + dx * dy) * 2.f;
}

// Smallest e with extent / 2^e <= 255 (the host builder's biased_exponent_for).
__device__ __forceinline__ uint8_t biased_exponent(float extent) {
  if (!(extent > 0.f)) return uint8_t(127 - 100);
  int e;
  frexp(double(extent) / 255.0, &e);  // extent / 255 = m 2^e, m in [0.5, 1)
  while (e > -126 && ldexp(255.0, e - 1) >= double(extent)) --e;
  while (ldexp(255.0, e) < double(extent)) ++e;
  e = max(-126, min(127, e));
  return uint8_t(e + 127);
}

__global__ void k_collapse(collapse_args a) {
  uint32_t const it = blockIdx.x * blockDim.x + threadIdx.x;
  if (it >= *a.n_in) return;
  collapse_item const item = a.in[it];
  uint32_t kids[8];
  ibox kb[8];
  int nk = 0;
  if ((item.ref & kLeafBit) || prim_count(a, item.ref) <= uint32_t(kMaxLeaf)) {
    kids[0] = item.ref;  // the whole (small) tree is one leaf slot
    nk = 1;
  } else {
    uint2 const c = a.child[item.ref];
    kids[0] = c.x;
    kids[1] = c.y;
    nk = 2;
    while (nk < 8) {
      int best = -1;
      float ba = -1.f;
      for (int k = 0; k < nk; ++k) {
        if ((kids[k] & kLeafBit) || prim_count(a, kids[k]) <= uint32_t(kMaxLeaf)) continue;
        float const ar = area(load_box(kids[k], a.leaf_boxes, a.order, a.inner));
        if (ar > ba) {
          ba = ar;
          best = k;
        }
      }
      if (best < 0) break;
      uint2 const c2 = a.child[kids[best]];
      kids[best] = c2.x;
      kids[nk++] = c2.y;
    }
  }
  ibox nb = load_box(kids[0], a.leaf_boxes, a.order, a.inner);
  kb[0] = nb;
  for (int k = 1; k < nk; ++k) {
    kb[k] = load_box(kids[k], a.leaf_boxes, a.order, a.inner);
    nb = merge(nb, kb[k]);
  }
  float const cx = 0.5f * (nb.lo.x + nb.hi.x), cy = 0.5f * (nb.lo.y + nb.hi.y), cz = 0.5f * (nb.lo.z + nb.hi.z);
  // octant slot assignment (the host builder's rule): slot s faces (+-1, +-1,
  // +-1), bit a of s set meaning +; repeatedly the (child, slot) pair with the
  // largest projection takes the slot
  int slot_of[8];
  {
    bool kid_done[8] = {}, slot_done[8] = {};
    float cost[8][8];
    for (int k = 0; k < nk; ++k) {
      float const dx = 0.5f * (kb[k].lo.x + kb[k].hi.x) - cx;
      float const dy = 0.5f * (kb[k].lo.y + kb[k].hi.y) - cy;
      float const dz = 0.5f * (kb[k].lo.z + kb[k].hi.z) - cz;
      for (int s = 0; s < 8; ++s) cost[k][s] = ((s & 1) ? dx : -dx) + ((s & 2) ? dy : -dy) + ((s & 4) ? dz : -dz);
    }
    for (int r = 0; r < nk; ++r) {
      int bk = -1, bs = -1;
      float bc = -3.402823466e38f;
      for (int k = 0; k < nk; ++k) {
        if (kid_done[k]) continue;
        for (int s = 0; s < 8; ++s) {
          if (slot_done[s]) continue;
          if (cost[k][s] > bc) {
            bc = cost[k][s];
            bk = k;
            bs = s;
          }
        }
      }
      if (bk < 0) {  // NaN boxes: take the first free pair
        for (int k = 0; k < nk && bk < 0; ++k)
          if (!kid_done[k]) bk = k;
        for (int s = 0; s < 8 && bs < 0; ++s)
          if (!slot_done[s]) bs = s;
      }
      kid_done[bk] = slot_done[bs] = true;
      slot_of[bk] = bs;
    }
  }
  int slot_kid[8];
  for (int s = 0; s < 8; ++s) slot_kid[s] = -1;
  for (int k = 0; k < nk; ++k) slot_kid[slot_of[k]] = k;
  uint32_t n_int = 0, n_tri = 0;
  for (int k = 0; k < nk; ++k) {
    uint32_t const pc = prim_count(a, kids[k]);
    if (pc <= uint32_t(kMaxLeaf)) n_tri += pc;
    else ++n_int;
  }
  uint32_t const child_base = n_int ? atomicAdd(&a.counters[0], n_int) : 0u;
  uint32_t const tri_base = n_tri ? atomicAdd(&a.counters[1], n_tri) : 0u;
  uint32_t const out_base = n_int ? atomicAdd(a.n_out, n_int) : 0u;
  atomicMax(&a.counters[3], item.depth);

  bvh8_node node;
  node.px = nb.lo.x;
  node.py = nb.lo.y;
  node.pz = nb.lo.z;
  node.imask = 0;
  float const ext[3] = {nb.hi.x - nb.lo.x, nb.hi.y - nb.lo.y, nb.hi.z - nb.lo.z};
  double scale[3];
  for (int ax = 0; ax < 3; ++ax) {
    node.e[ax] = biased_exponent(ext[ax]);
    scale[ax] = ldexp(1.0, int(node.e[ax]) - 127);
  }
  float const p[3] = {node.px, node.py, node.pz};
  node.child_base = child_base;
  node.tri_base = tri_base;
  uint32_t tri_off = 0, rank = 0, slots = 0;
  for (int s = 0; s < 8; ++s) {
    int const k = slot_kid[s];
    if (k < 0) {
      for (int ax = 0; ax < 3; ++ax) {
        node.qlo[ax][s] = 1;
        node.qhi[ax][s] = 0;
      }
      node.meta[s] = 0;
      continue;
    }
    float const blo[3] = {kb[k].lo.x, kb[k].lo.y, kb[k].lo.z}, bhi[3] = {kb[k].hi.x, kb[k].hi.y, kb[k].hi.z};
    for (int ax = 0; ax < 3; ++ax) {
      double const lo = floor((double(blo[ax]) - double(p[ax])) / scale[ax]);
      double const hi = ceil((double(bhi[ax]) - double(p[ax])) / scale[ax]);
      node.qlo[ax][s] = uint8_t(fmin(fmax(lo, 0.0), 255.0));
      node.qhi[ax][s] = uint8_t(fmin(fmax(hi, 0.0), 255.0));
    }
    uint32_t const pc = prim_count(a, kids[k]);
    if (pc > uint32_t(kMaxLeaf)) {
      node.imask |= uint8_t(1u << s);
      node.meta[s] = uint8_t(0x20u | unsigned(s));
      a.out[out_base + rank] = collapse_item{kids[k], child_base + rank, item.depth + 1u};
      ++rank;
    } else {
      node.meta[s] = uint8_t(tri_off | (pc << 5));
      uint2 const r = prim_range(a, kids[k]);
      for (uint32_t q = r.x; q <= r.y; ++q) {
        uint32_t const prim = a.order[q];
        float const* v = a.pos + 9 * size_t(prim);
        float4* t = a.tris + 3 * size_t(tri_base + tri_off);
        t[0] = make_float4(v[0], v[1], v[2], __uint_as_float(prim));
        t[1] = make_float4(v[3], v[4], v[5], 0.f);
        t[2] = make_float4(v[6], v[7], v[8], 0.f);
        ++tri_off;
      }
      ++slots;
    }
  }
  if (slots) atomicAdd(&a.counters[4], slots);
  a.nodes[item.wide] = node;
}

template <typename T> int dalloc(T** p, size_t count, std::vector<void*>& owned) {
  cudaError_t const e = cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(count, 1) * sizeof(T));
  if (e != cudaSuccess) return int(e);
  owned.push_back(*p);
  return 0;
}

// Sub-allocation of the scratch block: 256-byte aligned slices.
struct carve {
  size_t total = 0;
  template <typename T> size_t take(size_t count) {
    size_t const at = total;
    total += (std::max<size_t>(count, 1) * sizeof(T) + 255) & ~size_t(255);
    return at;
  }
};

}  // namespace

int build_bvh8_device(float const* d_pos, size_t n_tris, cudaStream_t st, device_build_scratch& scratch,
    device_bvh8 const* reuse, device_bvh8& out, char const** what) {
  out = device_bvh8{};
  *what = nullptr;
  if (n_tris == 0) return 0;
  if (n_tris >= (size_t(1) << 30)) {
    *what = "too many triangles for the device builder";
    return -1;
  }
  auto const t0 = std::chrono::steady_clock::now();
  int const n = int(n_tris);
  int e = 0;
  size_t tb = 0;
  if ((e = int(cub::DeviceRadixSort::SortPairs(nullptr, tb, static_cast<uint64_t const*>(nullptr),
           static_cast<uint64_t*>(nullptr), static_cast<uint32_t const*>(nullptr), static_cast<uint32_t*>(nullptr), n,
           0, 63, st)))) {
    *what = "device BVH sort size";
    return e;
  }
  carve c;
  size_t const o_boxes = c.take<ibox>(n), o_cb = c.take<uint32_t>(6), o_k0 = c.take<uint64_t>(n),
               o_k1 = c.take<uint64_t>(n), o_v0 = c.take<uint32_t>(n), o_v1 = c.take<uint32_t>(n),
               o_child = c.take<uint2>(n), o_range = c.take<uint2>(n), o_par_i = c.take<uint32_t>(n),
               o_par_l = c.take<uint32_t>(n), o_arrivals = c.take<uint32_t>(n), o_counters = c.take<uint32_t>(8),
               o_inner = c.take<ibox>(n), o_q0 = c.take<collapse_item>(n), o_q1 = c.take<collapse_item>(n),
               o_temp = c.take<char>(tb);
  if (scratch.bytes < c.total) {
    scratch.release();
    if ((e = int(cudaMalloc(&scratch.base, c.total)))) {
      scratch.base = nullptr;
      *what = "device BVH scratch";
      return e;
    }
    scratch.bytes = c.total;
  }
  char* const B = static_cast<char*>(scratch.base);
  auto* const boxes = reinterpret_cast<ibox*>(B + o_boxes);
  auto* const cb = reinterpret_cast<uint32_t*>(B + o_cb);
  auto* const k0 = reinterpret_cast<uint64_t*>(B + o_k0);
  auto* const k1 = reinterpret_cast<uint64_t*>(B + o_k1);
  auto* const v0 = reinterpret_cast<uint32_t*>(B + o_v0);
  auto* const v1 = reinterpret_cast<uint32_t*>(B + o_v1);
  auto* const child = reinterpret_cast<uint2*>(B + o_child);
  auto* const range = reinterpret_cast<uint2*>(B + o_range);
  auto* const par_i = reinterpret_cast<uint32_t*>(B + o_par_i);
  auto* const par_l = reinterpret_cast<uint32_t*>(B + o_par_l);
  auto* const arrivals = reinterpret_cast<uint32_t*>(B + o_arrivals);
  auto* const counters = reinterpret_cast<uint32_t*>(B + o_counters);
  auto* const inner = reinterpret_cast<ibox*>(B + o_inner);
  collapse_item* const q[2] = {reinterpret_cast<collapse_item*>(B + o_q0), reinterpret_cast<collapse_item*>(B + o_q1)};
  void* const temp = B + o_temp;
  // wide nodes: at most one per 2 triangles (every wide node but the root holds > 4) + 1
  size_t const max_nodes = n_tris / 2 + 2;
  bvh8_node* nodes;
  float4* tris;
  bool const reused = reuse && reuse->nodes && reuse->tris && reuse->node_capacity >= max_nodes &&
                      reuse->tri_capacity >= 3 * n_tris;
  if (reused) {
    nodes = reuse->nodes;
    tris = reuse->tris;
  } else {
    std::vector<void*> keep;
    if ((e = dalloc(&nodes, max_nodes, keep)) || (e = dalloc(&tris, 3 * n_tris, keep))) {
      for (void* p : keep) cudaFree(p);
      *what = "device BVH output";
      return e;
    }
  }
  auto fail = [&](int err, char const* w) {
    if (!reused) {
      cudaFree(nodes);
      cudaFree(tris);
    }
    *what = w;
    return err;
  };
  // counters: [0] wide nodes (the root), [2] level-0 queue length (the root item)
  static uint32_t const init_cb[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
  static uint32_t const init_counters[8] = {1u, 0u, 1u, 0u, 0u, 0u, 0u, 0u};
  collapse_item const root{n >= 2 ? 0u : kLeafBit, 0u, 1u};
  cudaMemcpyAsync(cb, init_cb, sizeof init_cb, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(counters, init_counters, sizeof init_counters, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(q[0], &root, sizeof root, cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(par_i, 0xff, size_t(n) * 4, st);
  cudaMemsetAsync(par_l, 0xff, size_t(n) * 4, st);
  cudaMemsetAsync(arrivals, 0, size_t(n) * 4, st);
  uint32_t const blocks = uint32_t((n + 255) / 256);
  k_prim_boxes<<<blocks, 256, 0, st>>>(d_pos, uint32_t(n), 1e-5f, boxes, cb);
  k_morton<<<blocks, 256, 0, st>>>(boxes, uint32_t(n), cb, k0, v0);
  if ((e = int(cub::DeviceRadixSort::SortPairs(temp, tb, k0, k1, v0, v1, n, 0, 63, st))))
    return fail(e, "device BVH sort");
  if (n >= 2) {
    k_radix_tree<<<uint32_t((n - 1 + 255) / 256), 256, 0, st>>>(k1, n, child, range, par_i, par_l);
    k_boxes_up<<<blocks, 256, 0, st>>>(boxes, v1, n, child, par_i, par_l, arrivals, inner);
  }
  collapse_args ca{};
  ca.leaf_boxes = boxes;
  ca.order = v1;
  ca.child = child;
  ca.range = range;
  ca.inner = inner;
  ca.pos = d_pos;
  ca.nodes = nodes;
  ca.tris = tris;
  ca.counters = counters;
  ca.n = n;
  // Level l reads queue l & 1 (length in counters[2] or [5]) and appends to
  // the other. Levels are launched in batches without reading their lengths
  // back: a level holds at most 8^l items (and at most n), which sizes its
  // grid; threads past the device-side length return at once. One read-back
  // per batch finds the end.
  uint32_t hc[8];
  uint32_t bound = 1;
  for (int level = 0;;) {
    for (int b = 0; b < 8; ++b, ++level) {
      int const in = level & 1;
      uint32_t* const len_out = counters + (in ? 2 : 5);
      cudaMemsetAsync(len_out, 0, 4, st);
      ca.in = q[in];
      ca.n_in = counters + (in ? 5 : 2);
      ca.out = q[in ^ 1];
      ca.n_out = len_out;
      k_collapse<<<(bound + 127) / 128, 128, 0, st>>>(ca);
      bound = uint32_t(std::min<uint64_t>(uint64_t(bound) * 8u, uint64_t(n)));
    }
    cudaMemcpyAsync(hc, counters, sizeof hc, cudaMemcpyDeviceToHost, st);
    if ((e = int(cudaStreamSynchronize(st)))) return fail(e, "device BVH collapse");
    if (hc[(level & 1) ? 5 : 2] == 0) break;  // the next level's queue is empty
    if (level > 4096) return fail(-1, "device BVH collapse did not finish");
  }
  if ((e = int(cudaGetLastError()))) return fail(e, "device BVH launch");
  out.nodes = nodes;
  out.tris = tris;
  out.node_capacity = reused ? reuse->node_capacity : max_nodes;
  out.tri_capacity = reused ? reuse->tri_capacity : 3 * n_tris;
  out.n_nodes = hc[0];
  out.n_tris = hc[1];
  out.wide_depth = int(hc[3]);
  out.leaf_slots = hc[4];
  out.binary_nodes = n >= 2 ? size_t(2 * n - 1) : 1;
  out.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return 0;
}

}  // namespace myrt_b200
