// Forward (raster preview) renderer: forward_renderer::run
// (src/pathtracer/forward_renderer.cpp:13-58) without a graphics pipeline.
// fwd_generate.comp's multi-draw-indirect records have no counterpart: the
// triangles of all drawables are already baked to world space in draw order
// (prim id = drawable order, then index order), which is the order
// glMultiDrawElementsIndirect draws them in.
//
// One raster pass (the G-buffer pass of forward/vert.vert + frag.frag, and the
// shadow pass with FORWARD_ONLY_POSITION) is five launches:
//   k_fwd_setup     one thread per triangle: clip-space corners (proj * view *
//                   world position), the three edge functions of homogeneous
//                   rasterisation (Olano & Greer, "Triangle scan conversion
//                   using 2D homogeneous coordinates", 1997) over homogeneous
//                   window coordinates, the depth plane, the pixel bounding
//                   box (the whole viewport when a corner has w <= 0) and its
//                   pixel count
//   k_fwd_small     triangles whose box holds at most 64 pixels (the bulk of
//                   a fine mesh): 8 lanes per triangle walk its box
//   CUB inclusive sum of the larger triangles' 8-pixel row segments
//   k_fwd_pixels    one thread per (large triangle, row segment), found by
//                   binary search in the sums, so a triangle covering half
//                   the screen spreads over the whole grid
//   k_fwd_attributes  per pixel: the kept triangle's perspective-correct
//                   barycentrics from the same edge functions, the attributes
//                   vert.vert passes interpolated and written as frag.frag
//                   writes them (RGBA16F G-buffer layers, or RGBA32F shadow
//                   positions)
// (plus the clear of the depth keys). Per pixel, k_fwd_small and k_fwd_pixels
// test coverage at the centre with a top-left rule on exact ties, clip to
// -1 <= z_ndc <= 1, quantise depth to 24 bits and do a 64-bit atomicMin of
// (depth << 32 | triangle) into the pixel. The minimum is what GL_LESS in draw
// order keeps: the nearest depth, the first-drawn triangle among equal depths;
// it does not depend on which kernel or thread got there first.
// Edge functions of a shared edge are exact negations of each other (same
// products, operands swapped), so shared edges are watertight. This file is
// compiled with -fmad=false: every + and * rounds separately, which makes the
// visibility and G-buffer bit-reproducible by the CPU restatement.
//
// k_fwd_resolve is forward/resolve.frag:72-206 per pixel.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "../../include/myrt_cuda.h"
#include "ctx.hpp"
#include "refshade.cuh"

namespace myrt_b200 {

struct forward_state {
  uint32_t W = 0, H = 0, S = 0;
  float4* rec = nullptr;      // 4 per triangle: edge functions + depth plane, box
  uint64_t* count = nullptr;  // row segments per large triangle (0 for small ones)
  uint64_t* ends = nullptr;   // inclusive sums of count
  size_t tri_cap = 0;
  void* scan_temp = nullptr;
  size_t scan_bytes = 0;
  unsigned long long* vis = nullptr;   // W * H keys
  unsigned long long* svis = nullptr;  // S * S keys
  __half* gbuf = nullptr;              // 3 layers of W * H RGBA16F
  __half* result = nullptr;            // W * H RGBA16F
  float4* smap = nullptr;              // S * S RGBA32F
};

namespace {

using rs::v2;
using rs::v3;

constexpr unsigned long long kEmpty = ~0ull;
constexpr uint32_t kSmallBox = 64;  // box pixels handled by one 8-lane group
constexpr uint32_t kSegment = 8;    // pixels per work item of a large triangle

// 4x4 column-major helpers shared by the host-side matrix set-up
struct mat4 {
  float m[16];
};
mat4 mul(mat4 const& a, mat4 const& b) {
  mat4 c{};
  for (int col = 0; col < 4; ++col)
    for (int r = 0; r < 4; ++r) {
      float s = a.m[r] * b.m[col * 4];
      for (int k = 1; k < 4; ++k) s = s + a.m[k * 4 + r] * b.m[col * 4 + k];
      c.m[col * 4 + r] = s;
    }
  return c;
}
// general inverse by cofactors in double, rounded once to float
mat4 inverse(mat4 const& a) {
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
  mat4 r{};
  for (int i = 0; i < 16; ++i) r.m[i] = float(inv[i] / det);
  return r;
}

// the reference's light camera (forward_renderer.cpp:306-310) with rnu's
// conventions restated: quat(axis, angle) = (axis sin(angle/2), cos(angle/2)),
// rotation(q) its rotation matrix, orthographic(l, r, b, t, n, f) the glOrtho
// matrix
void default_shadow(mat4& view, mat4& proj) {
  double const a = -45.0 * 3.14159265358979323846 / 180.0;
  double const c = std::cos(a), s = std::sin(a);
  // rotation about x by a, then translation (0, 0, 15): M = R * T
  double M[16] = {1, 0, 0, 0, 0, c, s, 0, 0, -s, c, 0, 0, 0, 0, 1};
  M[12] = 0.0;
  M[13] = -s * 15.0;
  M[14] = c * 15.0;
  mat4 mf{};
  for (int i = 0; i < 16; ++i) mf.m[i] = float(M[i]);
  view = inverse(mf);
  double const l = -20, r = 20, b = 20, t = -20, n = 0.01, f = 1000.0;
  double P[16] = {};
  P[0] = 2.0 / (r - l);
  P[5] = 2.0 / (t - b);
  P[10] = -2.0 / (f - n);
  P[12] = -(r + l) / (r - l);
  P[13] = -(t + b) / (t - b);
  P[14] = -(f + n) / (f - n);
  P[15] = 1.0;
  for (int i = 0; i < 16; ++i) proj.m[i] = float(P[i]);
}

struct m4 {
  float m[16];
};
__device__ __forceinline__ float4 mulv(m4 const& a, float x, float y, float z, float w) {
  float4 r;
  float* o = &r.x;
#pragma unroll
  for (int i = 0; i < 4; ++i) o[i] = ((a.m[i] * x + a.m[4 + i] * y) + a.m[8 + i] * z) + a.m[12 + i] * w;
  return r;
}

// ---- raster pass ---------------------------------------------------------------------
struct setup_args {
  float const* pos;  // 9 floats per triangle
  uint32_t n;
  m4 pv;             // proj * view
  uint32_t W, H;
  float4* rec;
  uint64_t* count;
};

__global__ void k_fwd_setup(setup_args a) {
  uint32_t const t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n) return;
  float const* p = a.pos + size_t(t) * 9;
  float const hw = float(a.W) * 0.5f, hh = float(a.H) * 0.5f;
  float X[3], Y[3], Wc[3], Z[3];
  bool finite = true, front = true;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    float4 const c = mulv(a.pv, __ldg(p + 3 * k), __ldg(p + 3 * k + 1), __ldg(p + 3 * k + 2), 1.f);
    X[k] = (c.x + c.w) * hw;
    Y[k] = (c.y + c.w) * hh;
    Z[k] = c.z;
    Wc[k] = c.w;
    finite = finite && isfinite(X[k]) && isfinite(Y[k]) && isfinite(Z[k]) && isfinite(Wc[k]);
    front = front && Wc[k] > 0.f;
  }
  float e[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    int const j = (i + 1) % 3, k = (i + 2) % 3;
    e[i][0] = Y[j] * Wc[k] - Wc[j] * Y[k];
    e[i][1] = Wc[j] * X[k] - X[j] * Wc[k];
    e[i][2] = X[j] * Y[k] - Y[j] * X[k];
  }
  float const det = (e[0][0] * X[0] + e[0][1] * Y[0]) + e[0][2] * Wc[0];
  uint64_t cnt = 0;
  float4* r = a.rec + 4 * size_t(t);
  float4 box = make_float4(0.f, 0.f, 0.f, 0.f);  // bw = 0: nothing to draw
  if (finite && det != 0.f && isfinite(det)) {
    float const sg = det > 0.f ? 1.f : -1.f, ad = fabsf(det);
    uint32_t flags = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      float const ea = e[i][0] * sg, eb = e[i][1] * sg, ec = e[i][2] * sg;
      if (ea > 0.f || (ea == 0.f && eb > 0.f)) flags |= 1u << i;
      r[i] = make_float4(ea, eb, ec, Z[i] / ad);
    }
    int x0 = 0, y0 = 0, x1 = int(a.W) - 1, y1 = int(a.H) - 1;
    if (front) {
      float lx = INFINITY, ly = INFINITY, ux = -INFINITY, uy = -INFINITY;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        float const sx = X[k] / Wc[k], sy = Y[k] / Wc[k];
        lx = fminf(lx, sx), ux = fmaxf(ux, sx), ly = fminf(ly, sy), uy = fmaxf(uy, sy);
      }
      // centres x + 0.5 in [lx, ux], widened by a pixel against rounding
      x0 = int(fmaxf(floorf(lx) - 1.f, 0.f)), y0 = int(fmaxf(floorf(ly) - 1.f, 0.f));
      x1 = int(fminf(floorf(ux) + 1.f, float(a.W) - 1.f)), y1 = int(fminf(floorf(uy) + 1.f, float(a.H) - 1.f));
    }
    if (x1 >= x0 && y1 >= y0) {
      uint32_t const bw = uint32_t(x1 - x0 + 1), bh = uint32_t(y1 - y0 + 1);
      if (uint64_t(bw) * bh > kSmallBox) cnt = uint64_t(bh) * ((bw + kSegment - 1) / kSegment);
      box = make_float4(__int_as_float(x0), __int_as_float(y0), __uint_as_float(bw), __uint_as_float(flags | (bh << 4)));
    }
  }
  r[3] = box;
  a.count[t] = cnt;
}

struct cover {
  float e[3];
};
// edge functions at the centre of pixel (x, y); true when the centre is inside
__device__ __forceinline__ bool covered(float4 const* r, uint32_t flags, int x, int y, cover& cv) {
  float const X = float(x) + 0.5f, Y = float(y) + 0.5f;
  bool in = true;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    float4 const q = __ldg(r + i);
    cv.e[i] = (q.x * X + q.y * Y) + q.z;
    in = in && (cv.e[i] > 0.f || (cv.e[i] == 0.f && ((flags >> i) & 1u)));
  }
  return in;
}

// one fragment: coverage, clipping, depth, the keyed depth test
__device__ __forceinline__ void fragment(float4 const (&q)[3], uint32_t flags, uint32_t t, int x, int y, uint32_t W,
    unsigned long long* __restrict__ vis) {
  float const X = float(x) + 0.5f, Y = float(y) + 0.5f;
  float e[3];
  bool in = true;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    e[i] = (q[i].x * X + q[i].y * Y) + q[i].z;
    in = in && (e[i] > 0.f || (e[i] == 0.f && ((flags >> i) & 1u)));
  }
  if (!in) return;
  float const zn = (e[0] * q[0].w + e[1] * q[1].w) + e[2] * q[2].w;
  if (!(zn >= -1.f && zn <= 1.f)) return;
  uint32_t const d = __float2uint_rn((zn * 0.5f + 0.5f) * 16777215.f);
  if (d >= 0xffffffu) return;  // cannot pass GL_LESS against the cleared 1.0
  unsigned long long const key = (static_cast<unsigned long long>(d) << 32) | t;
  unsigned long long* dst = vis + size_t(y) * W + x;
  if (key < *reinterpret_cast<volatile unsigned long long*>(dst)) atomicMin(dst, key);
}

// triangles with at most kSmallBox box pixels: 8 lanes per triangle
__global__ void __launch_bounds__(256) k_fwd_small(float4 const* __restrict__ rec, uint32_t n, uint32_t W,
    unsigned long long* __restrict__ vis) {
  uint32_t const t = blockIdx.x * (blockDim.x / 8) + threadIdx.x / 8, lane = threadIdx.x % 8;
  if (t >= n) return;
  float4 const* r = rec + 4 * size_t(t);
  float4 const box = __ldg(r + 3);
  uint32_t const bw = __float_as_uint(box.z), fl = __float_as_uint(box.w), bh = fl >> 4;
  uint32_t const area = bw * bh;
  if (bw == 0 || area > kSmallBox) return;
  float4 const q[3] = {__ldg(r), __ldg(r + 1), __ldg(r + 2)};
  int const x0 = __float_as_int(box.x), y0 = __float_as_int(box.y);
  // k / bw as (k * ceil(2^16 / bw)) >> 16: exact while k * bw < 2^16 (k < 64, bw <= 64 here)
  uint32_t const inv = (65535u + bw) / bw;
  for (uint32_t k = lane; k < area; k += 8) {
    uint32_t const ky = (k * inv) >> 16;
    fragment(q, fl & 7u, t, x0 + int(k - ky * bw), y0 + int(ky), W, vis);
  }
}

// larger triangles: one thread per row segment of kSegment pixels
__global__ void __launch_bounds__(256) k_fwd_pixels(float4 const* __restrict__ rec,
    uint64_t const* __restrict__ ends, uint32_t n, uint32_t W, unsigned long long* __restrict__ vis) {
  if (n == 0) return;
  uint64_t const total = __ldg(ends + n - 1);
  uint64_t const stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += stride) {
    uint32_t lo = 0, hi = n - 1;  // first t with ends[t] > i
    while (lo < hi) {
      uint32_t const mid = (lo + hi) >> 1;
      if (__ldg(ends + mid) > i) hi = mid;
      else lo = mid + 1;
    }
    uint32_t const t = lo;
    uint64_t const local = i - (t ? __ldg(ends + t - 1) : 0ull);
    float4 const* r = rec + 4 * size_t(t);
    float4 const box = __ldg(r + 3);
    uint32_t const bw = __float_as_uint(box.z), fl = __float_as_uint(box.w);
    uint32_t const segs = (bw + kSegment - 1) / kSegment;
    float4 const q[3] = {__ldg(r), __ldg(r + 1), __ldg(r + 2)};
    int const y = __float_as_int(box.y) + int(local / segs);
    uint32_t const s0 = uint32_t(local % segs) * kSegment, s1 = min(s0 + kSegment, bw);
    int const x0 = __float_as_int(box.x);
    for (uint32_t k = s0; k < s1; ++k) fragment(q, fl & 7u, t, x0 + int(k), y, W, vis);
  }
}

__global__ void k_fill_keys(unsigned long long* p, size_t n) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    p[i] = kEmpty;
}

struct attr_args {
  float4 const* rec;
  unsigned long long const* vis;
  uint32_t W, H;
  float const* pos;
  float4 const* nrm;  // 3 per triangle, may be null
  float2 const* uv;   // 3 per triangle, may be null
  int32_t const* mat;
  __half* gbuf;       // G-buffer pass: 3 layers
  float4* smap;       // shadow pass: positions
};

__device__ __forceinline__ v3 ld3(float const* p) { return {__ldg(p), __ldg(p + 1), __ldg(p + 2)}; }
__device__ __forceinline__ void st_half4(__half* p, float x, float y, float z, float w) {
  __half2* q = reinterpret_cast<__half2*>(p);
  q[0] = __halves2half2(__float2half_rn(x), __float2half_rn(y));
  q[1] = __halves2half2(__float2half_rn(z), __float2half_rn(w));
}

__global__ void k_fwd_attributes(attr_args a) {
  uint32_t const x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= a.W || y >= a.H) return;
  size_t const px = size_t(y) * a.W + x, plane = size_t(a.W) * a.H;
  unsigned long long const key = a.vis[px];
  if (key == kEmpty) {  // glClearColor(0, 0, 0, 0)
    if (a.gbuf) {
      for (int l = 0; l < 3; ++l) st_half4(a.gbuf + 4 * (l * plane + px), 0.f, 0.f, 0.f, 0.f);
    } else {
      a.smap[px] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    return;
  }
  uint32_t const t = uint32_t(key & 0xffffffffu);
  float4 const* r = a.rec + 4 * size_t(t);
  cover cv;
  covered(r, 0u, int(x), int(y), cv);
  float const s = (cv.e[0] + cv.e[1]) + cv.e[2];
  float const l0 = cv.e[0] / s, l1 = cv.e[1] / s, l2 = cv.e[2] / s;
  float const* P = a.pos + size_t(t) * 9;
  v3 const p0 = ld3(P), p1 = ld3(P + 3), p2 = ld3(P + 6);
  v3 const pos = (l0 * p0 + l1 * p1) + l2 * p2;
  if (!a.gbuf) {
    a.smap[px] = make_float4(pos.x, pos.y, pos.z, 1.f);
    return;
  }
  v3 n;
  if (a.nrm) {
    float4 const* N = a.nrm + 3 * size_t(t);
    float4 const n0 = __ldg(N), n1 = __ldg(N + 1), n2 = __ldg(N + 2);
    n = rs::normalize((l0 * v3{n0.x, n0.y, n0.z} + l1 * v3{n1.x, n1.y, n1.z}) + l2 * v3{n2.x, n2.y, n2.z});
  } else {
    n = rs::normalize(rs::cross(rs::normalize(p1 - p0), rs::normalize(p2 - p0)));
  }
  float u = 0.f, v = 0.f;
  if (a.uv) {
    float2 const* U = a.uv + 3 * size_t(t);
    float2 const u0 = __ldg(U), u1 = __ldg(U + 1), u2 = __ldg(U + 2);
    u = (l0 * u0.x + l1 * u1.x) + l2 * u2.x;
    v = (l0 * u0.y + l1 * u1.y) + l2 * u2.y;
  }
  st_half4(a.gbuf + 4 * px, pos.x, pos.y, pos.z, 1.f);
  st_half4(a.gbuf + 4 * (plane + px), u, v, 0.f, 0.f);
  st_half4(a.gbuf + 4 * (2 * plane + px), n.x, n.y, n.z, float(__ldg(a.mat + t)));
}

// ---- resolve pass (forward/resolve.frag) ---------------------------------------------
struct resolve_args {
  __half const* gbuf;
  float4 const* smap;
  __half* out;
  uint32_t W, H, S;
  m4 pv;       // proj * view (the SSAO reprojection)
  m4 inv_vp;   // inverse(view) * inverse(proj) (background rays)
  m4 sview, sproj;
  float cam[3];    // inverse(view)[3].xyz
  float light[3];  // normalize((inverse(shadow_view) * (0, 0, 1, 0)).xyz)
  uint32_t seed;
  int2 const* mat_refs;
  int n_mats;
  float const* mat_data;
  rs::tex2d const* textures;
  int n_textures;
};

__device__ __forceinline__ float4 ld_half4(__half const* p) {
  __half2 const* q = reinterpret_cast<__half2 const*>(p);
  float2 const a = __half22float2(q[0]), b = __half22float2(q[1]);
  return make_float4(a.x, a.y, b.x, b.y);
}
// uint(f) as NVIDIA GPUs convert: truncation, saturated to [0, 2^32 - 1], NaN -> 0
__device__ __forceinline__ uint32_t f2u_sat(float f) {
  if (!(f > 0.f)) return 0u;
  if (f >= 4294967296.f) return 0xffffffffu;
  return uint32_t(f);
}
// int(f) for an index: truncation, NaN and out-of-range -> 0 (the caller clamps)
__device__ __forceinline__ int f2i_idx(float f) {
  return (f > -2147483648.f && f < 2147483648.f) ? int(f) : 0;
}
// random.glsl:52-60 (random_init_nt)
__device__ __forceinline__ void random_init_nt(rs::rng_t& r, int px, int py, int seed) {
  r.state = uint32_t(seed);
  r.prime = 0;
  r.tex = nullptr;
  int const a = rs::random_int(r, px ^ 0xba77fa);
  int const b = rs::random_int(r, py ^ 0xcca6df);
  int const c = rs::random_int(r, seed);
  int const seed_base = int(uint32_t(a) * 69019u + uint32_t(b) * 96013u + uint32_t(c));
  int const rem = seed_base % 12352345;
  rs::random_value(r, int(uint32_t(seed_base) + 16756614u * uint32_t(rem)));
}
__device__ __forceinline__ v2 rnd2(rs::rng_t& r) {
  float const a = rs::random_next(r);
  float const b = rs::random_next(r);
  return {a, b};
}

__global__ void __launch_bounds__(256) k_fwd_resolve(resolve_args a) {
  uint32_t const x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= a.W || y >= a.H) return;
  size_t const plane = size_t(a.W) * a.H, px = size_t(y) * a.W + x;
  float4 const g0 = ld_half4(a.gbuf + 4 * px);
  float4 const g1 = ld_half4(a.gbuf + 4 * (plane + px));
  float4 const g2 = ld_half4(a.gbuf + 4 * (2 * plane + px));
  float const fw = float(a.W), fh = float(a.H);
  if (g2.x == 0.f && g2.y == 0.f && g2.z == 0.f) {
    float const nx = (float(x) / fw) * 2.f - 1.f, ny = (float(y) / fh) * 2.f - 1.f;
    float4 const h = mulv(a.inv_vp, nx, ny, 1.f, 1.f);
    v3 const d = rs::normalize(v3{h.x, h.y, h.z});
    v3 const c = rs::mix3(v3{0.3f, 0.4f, 0.5f}, v3{1.0f, 0.98f, 0.96f}, (d.y + 1.f) / 2.f);
    st_half4(a.out + 4 * px, c.x, c.y, c.z, 1.f);
    return;
  }
  v3 const cam{a.cam[0], a.cam[1], a.cam[2]};
  v3 const position{g0.x, g0.y, g0.z};
  v3 const to_cam = rs::normalize(cam - position);
  v3 normal = rs::normalize(v3{g2.x, g2.y, g2.z});
  normal = rs::faceforward(normal, -to_cam, normal);
  v2 const uv{g1.x, g1.y};
  int const material = f2i_idx(g2.w);

  float4 const sp = mulv(a.sview, position.x, position.y, position.z, 1.f);
  float4 const spx = mulv(a.sproj, sp.x, sp.y, sp.z, sp.w);
  v3 const light{a.light[0], a.light[1], a.light[2]};
  float const su = ((spx.x / spx.w) + 1.f) / 2.f, sv = ((spx.y / spx.w) + 1.f) / 2.f;
  float const fs = float(a.S);

  rs::rng_t rng;
  uint32_t const sd = ((a.seed + 9897584u * f2u_sat(position.x)) ^ f2u_sat(position.y)) ^ f2u_sat(position.z);
  random_init_nt(rng, int(x), int(y), int(sd));

  float avg = 0.f;
  int const r = 9;
  for (int i = 0; i < r; ++i) {
    v2 const q = rnd2(rng);
    float const hx = 2.f * q.x - 1.f, hy = 2.f * q.y - 1.f;
    float const u = su + (2.5f * hx) / fs, v = sv + (2.5f * hy) / fs;
    if (u >= 1.f || v >= 1.f || u < 0.f || v < 0.f) {
      avg += 1.f;
      continue;
    }
    // texture() minifies here (the jitter moves the coordinate by texels from
    // pixel to pixel): GL_NEAREST_MIPMAP_LINEAR on the single level = nearest
    int const tx = int(uint32_t(f2i_idx(floorf(u * fs))) % a.S), ty = int(uint32_t(f2i_idx(floorf(v * fs))) % a.S);
    float4 const m = __ldg(a.smap + size_t(ty) * a.S + tx);
    v3 const check = position - 100.f * light;
    float const l1 = rs::length(check - v3{m.x, m.y, m.z});
    avg += (l1 - 100.f < 0.01f) ? 1.f : 0.f;
  }
  float const shadow = avg / float(r);

  rs::material_ctx mc;
  bool const valid = material >= 0 && material < a.n_mats;
  int2 const ref = valid ? __ldg(a.mat_refs + material) : make_int2(-1, 0);
  rs::mat_open(mc, ref.x, a.mat_data, ref.y);
  mc.ps.state = 2;  // s_diffuse
  v3 refl{0.f, 0.f, 0.f};
  float pdf = 1.f;
  rs::mat_evaluate(mc, normal, light, to_cam, refl, pdf, uv, a.textures, a.n_textures);
  v3 refgb{0.f, 0.f, 0.f};
  float refpdf = 1.f;
  mc.ps.state = 2;
  rs::mat_evaluate(mc, normal, normal, to_cam, refgb, refpdf, uv, a.textures, a.n_textures);

  float freeness = 0.f;
  float dist = 0.1f;
  for (int i = 0; i < 8; ++i) {
    do {
      v2 const q = rnd2(rng);
      v2 const hs{2.f * q.x - 1.f, 2.f * q.y - 1.f};
      v3 const world = rs::normalize(rs::transform_local_to_world(rs::sample_hemisphere(hs), normal));
      v3 const test = position + world * dist;
      float4 const hom = mulv(a.pv, test.x, test.y, test.z, 1.f);
      if (hom.w == 0.f) {
        freeness += 1.f;
        break;
      }
      float const qx = fminf(fmaxf((((hom.x / hom.w) + 1.f) / 2.f) * fw, 0.f), fw - 1.f);
      float const qy = fminf(fmaxf((((hom.y / hom.w) + 1.f) / 2.f) * fh, 0.f), fh - 1.f);
      size_t const o = size_t(f2i_idx(qy)) * a.W + size_t(f2i_idx(qx));
      float4 const on = ld_half4(a.gbuf + 4 * (2 * plane + o));
      if (on.x == 0.f && on.y == 0.f && on.z == 0.f) {
        freeness += 1.f;
        break;
      }
      float4 const op = ld_half4(a.gbuf + 4 * o);
      float const diff = rs::length(cam - v3{op.x, op.y, op.z}) - rs::length(cam - test);
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
  float const ndl = rs::gmax(0.f, rs::dot(normal, light));
  v3 const direct = (((lcol * refl) / pdf) * shadow) * ndl;
  v3 c = freeness * (refgb / refpdf + direct);
  float const k = 0.7f + 0.4f * rs::random_next(rng);
  c = c * k;
  st_half4(a.out + 4 * px, c.x, c.y, c.z, 1.f * 0.f);
}

template <typename T> int grow(myrt_ctx* ctx, T*& p, size_t& cap, size_t need, char const* what) {
  if (cap >= need) return MYRT_OK;
  cudaFree(p);
  p = nullptr;
  cap = 0;
  int const rc = check_cuda(ctx, cudaMalloc(reinterpret_cast<void**>(&p), need * sizeof(T)), what);
  if (!rc) cap = need;
  return rc;
}

m4 dev(mat4 const& m) {
  m4 r;
  std::memcpy(r.m, m.m, sizeof r.m);
  return r;
}

// one raster pass into keys (W x H) and then attributes
int raster_pass(myrt_ctx* ctx, forward_state& f, mat4 const& pv, uint32_t W, uint32_t H,
    unsigned long long* keys, __half* gbuf, float4* smap) {
  device_scene const& s = ctx->scene;
  cudaStream_t const st = ctx->stream;
  uint32_t const n = uint32_t(s.n_prims);
  k_fill_keys<<<std::max(1, ctx->sm_count) * 4, 256, 0, st>>>(keys, size_t(W) * H);
  if (n) {
    setup_args sa{s.world_pos, n, dev(pv), W, H, f.rec, f.count};
    k_fwd_setup<<<(n + 255) / 256, 256, 0, st>>>(sa);
    size_t tb = f.scan_bytes;
    int rc = check_cuda(ctx, cub::DeviceScan::InclusiveSum(f.scan_temp, tb, f.count, f.ends, int(n), st),
        "forward pixel-count scan");
    if (rc) return rc;
    k_fwd_small<<<(n + 31) / 32, 256, 0, st>>>(f.rec, n, W, keys);
    k_fwd_pixels<<<std::max(1, ctx->sm_count) * 8, 256, 0, st>>>(f.rec, f.ends, n, W, keys);
  }
  attr_args aa{f.rec, keys, W, H, s.world_pos, s.tri_normals, s.tri_uvs, s.tri_material, gbuf, smap};
  dim3 const blk(16, 16), grd((W + 15) / 16, (H + 15) / 16);
  k_fwd_attributes<<<grd, blk, 0, st>>>(aa);
  return check_cuda(ctx, cudaGetLastError(), "forward raster pass");
}

int ensure_forward(myrt_ctx* ctx, uint32_t W, uint32_t H, uint32_t S) {
  if (!ctx->forward) ctx->forward = new forward_state();
  forward_state& f = *ctx->forward;
  size_t const n = std::max<size_t>(1, ctx->scene.n_prims);
  int rc = MYRT_OK;
  if (f.tri_cap < n) {
    cudaFree(f.rec);
    cudaFree(f.count);
    cudaFree(f.ends);
    f.rec = nullptr, f.count = nullptr, f.ends = nullptr, f.tri_cap = 0;
    rc = check_cuda(ctx, cudaMalloc(reinterpret_cast<void**>(&f.rec), n * 4 * sizeof(float4)), "forward setup");
    if (!rc) rc = check_cuda(ctx, cudaMalloc(reinterpret_cast<void**>(&f.count), n * 8), "forward counts");
    if (!rc) rc = check_cuda(ctx, cudaMalloc(reinterpret_cast<void**>(&f.ends), n * 8), "forward counts");
    if (rc) return rc;
    f.tri_cap = n;
    size_t tb = 0;
    rc = check_cuda(ctx, cub::DeviceScan::InclusiveSum(nullptr, tb, f.count, f.ends, int(n), ctx->stream),
        "forward scan size");
    if (rc) return rc;
    cudaFree(f.scan_temp);
    f.scan_temp = nullptr;
    f.scan_bytes = 0;
    rc = check_cuda(ctx, cudaMalloc(&f.scan_temp, std::max<size_t>(tb, 16)), "forward scan storage");
    if (rc) return rc;
    f.scan_bytes = std::max<size_t>(tb, 16);
  }
  if (f.W != W || f.H != H) {
    cudaFree(f.vis);
    cudaFree(f.gbuf);
    cudaFree(f.result);
    f.vis = nullptr, f.gbuf = nullptr, f.result = nullptr, f.W = f.H = 0;
    size_t const px = size_t(W) * H;
    rc = check_cuda(ctx, cudaMalloc(reinterpret_cast<void**>(&f.vis), px * 8), "forward depth buffer");
    if (!rc) rc = check_cuda(ctx, cudaMalloc(reinterpret_cast<void**>(&f.gbuf), 3 * px * 8), "forward G-buffer");
    if (!rc) rc = check_cuda(ctx, cudaMalloc(reinterpret_cast<void**>(&f.result), px * 8), "forward result");
    if (rc) return rc;
    f.W = W, f.H = H;
  }
  if (f.S != S) {
    cudaFree(f.svis);
    cudaFree(f.smap);
    f.svis = nullptr, f.smap = nullptr, f.S = 0;
    size_t const px = size_t(S) * S;
    rc = check_cuda(ctx, cudaMalloc(reinterpret_cast<void**>(&f.svis), px * 8), "forward shadow depth");
    if (!rc) rc = check_cuda(ctx, cudaMalloc(reinterpret_cast<void**>(&f.smap), px * 16), "forward shadow map");
    if (rc) return rc;
    f.S = S;
  }
  return MYRT_OK;
}

int forward_run(myrt_ctx* ctx, myrt_forward_params const* p) {
  if (!p) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "null forward parameters");
  if (!ctx->scene.valid) return set_error(ctx, MYRT_ERR_NO_SCENE, "no scene uploaded");
  uint32_t const S = p->shadow_size ? p->shadow_size : 2048u;
  if (p->width == 0 || p->height == 0 || p->width > 16384 || p->height > 16384 || S > 16384)
    return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "forward image sizes must be 1..16384");
  if (ctx->scene.n_prims && !ctx->scene.world_pos)
    return set_error(ctx, MYRT_ERR_UNSUPPORTED, "scene has no world-space triangles");
  int rc = ensure_forward(ctx, p->width, p->height, S);
  if (rc) return rc;
  forward_state& f = *ctx->forward;
  mat4 view, proj, sview, sproj;
  std::memcpy(view.m, p->view, 64);
  std::memcpy(proj.m, p->projection, 64);
  if (p->custom_shadow) {
    std::memcpy(sview.m, p->shadow_view, 64);
    std::memcpy(sproj.m, p->shadow_projection, 64);
  } else {
    default_shadow(sview, sproj);
  }
  mat4 const pv = mul(proj, view), spv = mul(sproj, sview);
  mat4 const inv_view = inverse(view);
  mat4 const inv_vp = mul(inv_view, inverse(proj));
  mat4 const inv_sview = inverse(sview);
  // pass_render, then pass_shadow (forward_renderer.cpp:50-55)
  rc = raster_pass(ctx, f, pv, f.W, f.H, f.vis, f.gbuf, nullptr);
  if (!rc) rc = raster_pass(ctx, f, spv, S, S, f.svis, nullptr, f.smap);
  if (rc) return rc;
  resolve_args ra{};
  ra.gbuf = f.gbuf;
  ra.smap = f.smap;
  ra.out = f.result;
  ra.W = f.W, ra.H = f.H, ra.S = S;
  ra.pv = dev(pv);
  ra.inv_vp = dev(inv_vp);
  ra.sview = dev(sview);
  ra.sproj = dev(sproj);
  for (int k = 0; k < 3; ++k) ra.cam[k] = inv_view.m[12 + k];
  {
    // inverse(shadow_view) * (0, 0, 1, 0), normalised as resolve.frag:94-95
    float const lx = ((inv_sview.m[0] * 0.f + inv_sview.m[4] * 0.f) + inv_sview.m[8] * 1.f) + inv_sview.m[12] * 0.f;
    float const ly = ((inv_sview.m[1] * 0.f + inv_sview.m[5] * 0.f) + inv_sview.m[9] * 1.f) + inv_sview.m[13] * 0.f;
    float const lz =
        ((inv_sview.m[2] * 0.f + inv_sview.m[6] * 0.f) + inv_sview.m[10] * 1.f) + inv_sview.m[14] * 0.f;
    float const len = std::sqrt((lx * lx + ly * ly) + lz * lz);
    float const inv = 1.f / len;
    ra.light[0] = lx * inv, ra.light[1] = ly * inv, ra.light[2] = lz * inv;
  }
  ra.seed = p->random_seed;
  ra.mat_refs = reinterpret_cast<int2 const*>(ctx->scene.materials);
  ra.n_mats = int(ctx->scene.n_materials);
  ra.mat_data = ctx->scene.material_data;
  ra.textures = reinterpret_cast<rs::tex2d const*>(ctx->d_textures);
  ra.n_textures = int(ctx->textures.size());
  dim3 const blk(16, 16), grd((f.W + 15) / 16, (f.H + 15) / 16);
  k_fwd_resolve<<<grd, blk, 0, ctx->stream>>>(ra);
  return check_cuda(ctx, cudaGetLastError(), "forward resolve");
}

}  // namespace

void free_forward(myrt_ctx* ctx) {
  forward_state* f = ctx->forward;
  if (!f) return;
  cudaFree(f->rec);
  cudaFree(f->count);
  cudaFree(f->ends);
  cudaFree(f->scan_temp);
  cudaFree(f->vis);
  cudaFree(f->svis);
  cudaFree(f->gbuf);
  cudaFree(f->result);
  cudaFree(f->smap);
  delete f;
  ctx->forward = nullptr;
}

}  // namespace myrt_b200

using myrt_b200::check_cuda;
using myrt_b200::set_error;

extern "C" int myrt_forward_run(myrt_ctx* ctx, myrt_forward_params const* params) {
  if (!ctx) return MYRT_ERR_INVALID_ARGUMENT;
  int const rc = check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  if (rc) return rc;
  return myrt_b200::forward_run(ctx, params);
}

extern "C" int myrt_forward_read(myrt_ctx* ctx, uint32_t width, uint32_t height, uint32_t shadow_size,
    uint16_t* result, uint16_t* gbuffer, float* shadow_map, uint64_t* visibility) {
  if (!ctx) return MYRT_ERR_INVALID_ARGUMENT;
  myrt_b200::forward_state const* f = ctx->forward;
  if (!f || !f->W) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "no forward run yet");
  if (width != f->W || height != f->H || (shadow_size ? shadow_size : 2048u) != f->S)
    return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "read sizes differ from the last forward run");
  int rc = check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  size_t const px = size_t(f->W) * f->H, spx = size_t(f->S) * f->S;
  cudaStream_t const st = ctx->stream;
  if (!rc && result) rc = check_cuda(ctx, cudaMemcpyAsync(result, f->result, px * 8, cudaMemcpyDeviceToHost, st), "read");
  if (!rc && gbuffer)
    rc = check_cuda(ctx, cudaMemcpyAsync(gbuffer, f->gbuf, 3 * px * 8, cudaMemcpyDeviceToHost, st), "read");
  if (!rc && shadow_map)
    rc = check_cuda(ctx, cudaMemcpyAsync(shadow_map, f->smap, spx * 16, cudaMemcpyDeviceToHost, st), "read");
  if (!rc && visibility)
    rc = check_cuda(ctx, cudaMemcpyAsync(visibility, f->vis, px * 8, cudaMemcpyDeviceToHost, st), "read");
  if (!rc) rc = check_cuda(ctx, cudaStreamSynchronize(st), "forward read");
  return rc;
}

extern "C" int myrt_forward_buffers(myrt_ctx* ctx, void** result, void** gbuffer, void** shadow_map, void** visibility) {
  if (!ctx) return MYRT_ERR_INVALID_ARGUMENT;
  myrt_b200::forward_state const* f = ctx->forward;
  if (!f || !f->W) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "no forward run yet");
  if (result) *result = f->result;
  if (gbuffer) *gbuffer = f->gbuf;
  if (shadow_map) *shadow_map = f->smap;
  if (visibility) *visibility = f->vis;
  return MYRT_OK;
}

extern "C" int myrt_forward_default_shadow(float* view, float* projection) {
  myrt_b200::mat4 v, p;
  myrt_b200::default_shadow(v, p);
  if (view) std::memcpy(view, v.m, 64);
  if (projection) std::memcpy(projection, p.m, 64);
  return MYRT_OK;
}
