// Learned path guiding: a 4-layer, 64-wide MLP mapping frequency-encoded
// position, shading normal and view direction to a mixture of 8 von
// Mises-Fisher lobes, trained online from the renderer's own radiance samples.
//
// Kernels
//   k_guide_gather   queue slots -> raw shading points (position, normal,
//                    view, valid flag)
//   k_guide_forward  encoding + the MLP on tcgen05 (BF16 operands in
//                    shared memory, FP32 accumulator in TMEM) + the mixture
//                    parameters per point; persistent, 128 points per tile
//   k_guide_collect  training records of a finished wave -> samples
//                    (x, direction, weight = lum(L_i f cos) / pdf)
//   k_guide_train    forward + backward of 128-sample tiles on tcgen05: the
//                    data gradient dH = dZ W (W read MN-major) and the weight
//                    gradient dW += dZ^T H (both operands MN-major), dW kept
//                    in TMEM across a CTA's tiles, then stored as this CTA's
//                    partial gradient (no global atomics)
//   k_guide_adam     sum of the CTAs' partial gradients, Adam on the FP32
//                    master parameters, BF16 copy for the MLP
//
// Loss (per sample): -w log q(wi | x); its gradient is the KL-divergence
// gradient between the normalised target w * q_sample and q (Mueller et al.,
// "Neural Importance Sampling", 2019), with the target the product of the
// incident radiance estimate and the BSDF cosine.
//
// Layout: weights [4][64 out][64 in], biases [4][64]; 16,640 FP32 parameters.
// Feature vector (64): position normalised to the scene box (3), sin / cos of
// 2^f pi p for f = 0..5 (36), shading normal (3), view direction (3), 1, zeros.
// Output (64, 40 used): per lobe logit, kappa (softplus), mu (normalised).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "../../include/myrt_cuda.h"
#include "ctx.hpp"
#include "guide.cuh"
#include "tc.cuh"

namespace myrt_b200 {

enum : uint32_t {
  ERR_GUIDE_TIMEOUT = 1u << 5,  // a tensor-core wait ran out of polls
};

constexpr int kLayers = 4;
constexpr int kWidth = 64;
constexpr int kParams = kLayers * kWidth * kWidth + kLayers * kWidth;  // 16640
constexpr uint32_t kPollLimit = 1u << 22;

struct guide_state {
  float* params = nullptr;  // W then b
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  float* grads = nullptr;
  float* partials = nullptr;     // [kMaxParts][kParams] per-CTA gradients of one training launch
  uint32_t max_parts = 0;
  uint16_t* w_bf16 = nullptr;
  float* sums = nullptr;         // [0] loss sum, [1] weight sum
  uint32_t* counters = nullptr;  // [0] training samples collected
  float4* points = nullptr;      // 3 float4 per row
  float4* lobes = nullptr;       // 16 float4 per row
  size_t rows_cap = 0;
  float4* records = nullptr;
  size_t records_cap = 0;        // in records
  float4* samples = nullptr;     // 4 float4 per sample
  size_t samples_cap = 0;
  myrt_guide_params prm{0.5f, 1e-2f, 16u, 16384u, 1u, 1u, 1u, 10.f, 0u, 0u};
  uint32_t wave = 0;
  uint32_t tag = 0;
  uint64_t generation = ~uint64_t(0);
  uint64_t adam_t = 0;
  uint64_t steps = 0;
  uint64_t waves_trained = 0;
};

namespace {

struct mlp_args {
  uint16_t const* w;   // bf16 [4][64][64]
  float const* bias;   // [4][64]
  float center[3], inv_half[3];
  uint32_t* err;
  uint32_t poll_limit;  // polls of each CTA's first tensor-core wait (the others use kPollLimit)
  uint32_t stall;       // 1: that first wait watches a barrier nothing arrives at, so it runs out
                        // (exercises the timeout path; the MMA in flight is still drained)
};

// ---- encoding ------------------------------------------------------------------------
__device__ __forceinline__ void encode(mlp_args const& a, float4 p, float4 n, float4 wo, float (&f)[64]) {
  float pn[3] = {(p.x - a.center[0]) * a.inv_half[0], (p.y - a.center[1]) * a.inv_half[1],
      (p.z - a.center[2]) * a.inv_half[2]};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    pn[k] = fminf(fmaxf(pn[k], -1.f), 1.f);
    f[k] = pn[k];
  }
  // sin / cos of 2^f pi p: one sincospi per axis, then the double-angle
  // formulas (the features are rounded to BF16 before the first layer, far
  // above the recurrence's few-ulp drift)
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    float s, c;
    sincospif(pn[k], &s, &c);
#pragma unroll
    for (int fr = 0; fr < 6; ++fr) {
      f[3 + 6 * fr + 2 * k] = s;
      f[4 + 6 * fr + 2 * k] = c;
      float const s2 = 2.f * s * c;
      c = fmaf(-2.f * s, s, 1.f);
      s = s2;
    }
  }
  f[39] = n.x, f[40] = n.y, f[41] = n.z;
  f[42] = wo.x, f[43] = wo.y, f[44] = wo.z;
  f[45] = 1.f;
#pragma unroll
  for (int k = 46; k < 64; ++k) f[k] = 0.f;
}

// 64 floats -> one swizzled BF16 row of a tile
__device__ __forceinline__ void store_row(uint8_t* tile, uint32_t r, float const (&f)[64]) {
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    uint4 v;
    v.x = tc::pack_bf16(f[8 * c + 0], f[8 * c + 1]);
    v.y = tc::pack_bf16(f[8 * c + 2], f[8 * c + 3]);
    v.z = tc::pack_bf16(f[8 * c + 4], f[8 * c + 5]);
    v.w = tc::pack_bf16(f[8 * c + 6], f[8 * c + 7]);
    *reinterpret_cast<uint4*>(tile + tc::sw128_offset(r, uint32_t(c))) = v;
  }
}
__device__ __forceinline__ float bf16_lo(uint32_t u) { return __uint_as_float(u << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t u) { return __uint_as_float(u & 0xffff0000u); }
__device__ __forceinline__ void load_row(uint8_t const* tile, uint32_t r, float (&f)[64]) {
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    uint4 const v = *reinterpret_cast<uint4 const*>(tile + tc::sw128_offset(r, uint32_t(c)));
    f[8 * c + 0] = bf16_lo(v.x), f[8 * c + 1] = bf16_hi(v.x);
    f[8 * c + 2] = bf16_lo(v.y), f[8 * c + 3] = bf16_hi(v.y);
    f[8 * c + 4] = bf16_lo(v.z), f[8 * c + 5] = bf16_hi(v.z);
    f[8 * c + 6] = bf16_lo(v.w), f[8 * c + 7] = bf16_hi(v.w);
  }
}

// the accumulator row of this thread (64 columns starting at col) + bias
__device__ __forceinline__ void acc_row(uint32_t tmem, uint32_t col, float const* bias, float (&f)[64]) {
  uint32_t const warp = threadIdx.x >> 5;
  float lo[32], hi[32];
  tc::tmem_ld32(tmem + ((32u * warp) << 16) + col, lo);
  tc::tmem_ld32(tmem + ((32u * warp) << 16) + col + 32u, hi);
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    f[j] = lo[j] + (bias ? bias[j] : 0.f);
    f[32 + j] = hi[j] + (bias ? bias[32 + j] : 0.f);
  }
}

// weights (bf16 [4][64][64]) -> four swizzled 64 x 64 tiles; biases -> smem
__device__ __forceinline__ void load_weights(mlp_args const& a, uint8_t* wt, float* bias) {
  for (uint32_t i = threadIdx.x; i < kLayers * 64 * 8; i += blockDim.x) {
    uint32_t const l = i / 512, r = (i / 8) % 64, c = i % 8;
    uint4 const v = *reinterpret_cast<uint4 const*>(a.w + (size_t(l) * 64 + r) * 64 + c * 8);
    *reinterpret_cast<uint4*>(wt + l * 8192 + tc::sw128_offset(r, c)) = v;
  }
  for (uint32_t i = threadIdx.x; i < kLayers * 64; i += blockDim.x) bias[i] = a.bias[i];
}

// ---- mixture parameters -----------------------------------------------------------------
struct lobe_set {
  float w[kGuideLobes], kappa[kGuideLobes], mu[kGuideLobes][3], len[kGuideLobes], dk[kGuideLobes];
};
constexpr float kKappaMin = 0.01f, kKappaMax = 1000.f;

__device__ __forceinline__ void mixture(float const (&o)[64], lobe_set& L) {
  float mx = o[0];
#pragma unroll
  for (int k = 1; k < kGuideLobes; ++k) mx = fmaxf(mx, o[5 * k]);
  float sum = 0.f;
#pragma unroll
  for (int k = 0; k < kGuideLobes; ++k) {
    L.w[k] = __expf(o[5 * k] - mx);
    sum += L.w[k];
  }
#pragma unroll
  for (int k = 0; k < kGuideLobes; ++k) {
    L.w[k] = L.w[k] / sum;
    float const x = o[5 * k + 1];
    float const ex = __expf(-fabsf(x));  // softplus(x) = max(x, 0) + log(1 + e^-|x|)
    float const sp = fmaxf(x, 0.f) + log1pf(ex);
    float kap = sp + kKappaMin;
    float dk = x >= 0.f ? __frcp_rn(1.f + ex) : ex * __frcp_rn(1.f + ex);  // d softplus / dx
    if (kap > kKappaMax) {
      kap = kKappaMax;
      dk = 0.f;
    }
    L.kappa[k] = kap;
    L.dk[k] = dk;
    float const mx3 = o[5 * k + 2], my = o[5 * k + 3], mz = o[5 * k + 4];
    float const len = sqrtf(mx3 * mx3 + my * my + mz * mz);
    L.len[k] = len;
    if (len > 1e-6f) {
      L.mu[k][0] = mx3 / len, L.mu[k][1] = my / len, L.mu[k][2] = mz / len;
    } else {
      L.mu[k][0] = 0.f, L.mu[k][1] = 0.f, L.mu[k][2] = 1.f;
    }
  }
}
// kappa / (2 pi (1 - exp(-2 kappa)))
__device__ __forceinline__ float vmf_norm(float k) { return k / (-6.28318530717958648f * expm1f(-2.f * k)); }

// ---- k_guide_gather: queue slots -> points ---------------------------------------------
__global__ void __launch_bounds__(256) k_guide_gather(float4 const* __restrict__ queue, float4 const* __restrict__ hits,
    uint32_t const* __restrict__ count, float4* __restrict__ points) {
  uint32_t const n = *count;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float4 const h0 = hits[3 * size_t(i)], h1 = hits[3 * size_t(i) + 1], h2 = hits[3 * size_t(i) + 2];
    float4 const d = queue[3 * size_t(i) + 1];
    float wo[3] = {-d.x, -d.y, -d.z};
    float ng[3] = {h2.x, h2.y, h2.z}, ns[3] = {h1.x, h1.y, h1.z};
    float const gdo = (ng[0] * wo[0] + ng[1] * wo[1]) + ng[2] * wo[2];
    if (gdo < 0.f) ng[0] = -ng[0], ng[1] = -ng[1], ng[2] = -ng[2];
    if ((ns[0] * ng[0] + ns[1] * ng[1]) + ns[2] * ng[2] < 0.f) ns[0] = -ns[0], ns[1] = -ns[1], ns[2] = -ns[2];
    if (!((ns[0] * wo[0] + ns[1] * wo[1]) + ns[2] * wo[2] > 0.f)) ns[0] = ng[0], ns[1] = ng[1], ns[2] = ng[2];
    float const valid = __float_as_int(h0.w) >= 0 ? 1.f : 0.f;
    points[3 * size_t(i)] = make_float4(h0.x, h0.y, h0.z, valid);
    points[3 * size_t(i) + 1] = make_float4(ns[0], ns[1], ns[2], 0.f);
    points[3 * size_t(i) + 2] = make_float4(wo[0], wo[1], wo[2], 0.f);
  }
}

// ---- k_guide_forward --------------------------------------------------------------------
// Four warpgroups per CTA, each with its own 128-row tile, H tile, 64 TMEM
// columns and mbarrier; the four weight tiles are shared. A thread owns one row
// of its group's tile and keeps at most 32 accumulator columns in registers at a
// time (encoding, layer epilogues and the mixture head run in 8- or 32-column
// pieces), so 512 threads fit at 64 registers and two CTAs -- eight tiles in
// flight, 32 warps -- share an SM, one tile's MMAs overlapping the others'
// epilogues.
// Shared memory (from a 1024-aligned base): W tiles 4 x 8 KB, H tiles 4 x 16 KB,
// biases 1 KB, 4 mbarriers, 4 stall-test mbarriers, TMEM address.
constexpr uint32_t kFwdGroups = 4;
constexpr uint32_t kFwdW = 0, kFwdH = 32768, kFwdBias = 98304, kFwdBar = 99328, kFwdStall = 99360, kFwdTmem = 99392;
constexpr uint32_t kFwdSmem = 99400 + 1024;

__device__ __forceinline__ uint8_t* align1024(uint8_t* p) {
  uint32_t const s = tc::smem_u32(p);
  return p + ((1024u - (s & 1023u)) & 1023u);
}

// Encoding of one point (as encode()) written to row r of a swizzled tile in
// eight 16-byte chunks, each stored as soon as its 8 features exist.
__device__ __forceinline__ void encode_store(mlp_args const& a, float4 p, float4 n, float4 wo, uint8_t* tile,
    uint32_t r) {
  float pn[3] = {(p.x - a.center[0]) * a.inv_half[0], (p.y - a.center[1]) * a.inv_half[1],
      (p.z - a.center[2]) * a.inv_half[2]};
  float sn[3], cs[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    pn[k] = fminf(fmaxf(pn[k], -1.f), 1.f);
    sincospif(pn[k], &sn[k], &cs[k]);
  }
  float buf[8];
  auto put = [&](int i, float v) {
    buf[i & 7] = v;
    if ((i & 7) == 7) {
      uint4 q;
      q.x = tc::pack_bf16(buf[0], buf[1]);
      q.y = tc::pack_bf16(buf[2], buf[3]);
      q.z = tc::pack_bf16(buf[4], buf[5]);
      q.w = tc::pack_bf16(buf[6], buf[7]);
      *reinterpret_cast<uint4*>(tile + tc::sw128_offset(r, uint32_t(i >> 3))) = q;
    }
  };
  put(0, pn[0]);
  put(1, pn[1]);
  put(2, pn[2]);
#pragma unroll
  for (int fr = 0; fr < 6; ++fr) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      put(3 + 6 * fr + 2 * k, sn[k]);
      put(4 + 6 * fr + 2 * k, cs[k]);
      float const s2 = 2.f * sn[k] * cs[k];
      cs[k] = fmaf(-2.f * sn[k], sn[k], 1.f);
      sn[k] = s2;
    }
  }
  put(39, n.x);
  put(40, n.y);
  put(41, n.z);
  put(42, wo.x);
  put(43, wo.y);
  put(44, wo.z);
  put(45, 1.f);
#pragma unroll
  for (int k = 46; k < 64; ++k) put(k, 0.f);
}

// Hidden-layer epilogue of one row: accumulator + bias, ReLU, BF16, back into
// the group's H tile (the next layer's A operand), 32 columns at a time.
__device__ __forceinline__ void relu_to_tile(uint32_t tacc, float const* bias, uint8_t* tile, uint32_t r) {
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    float v[32];
    tc::tmem_ld32(tacc + 32u * h, v);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      float x[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) x[j] = v[8 * c + j] + bias[32 * h + 8 * c + j];
      uint4 q;  // ReLU inside the BF16 conversion
      q.x = tc::pack_bf16_relu(x[0], x[1]);
      q.y = tc::pack_bf16_relu(x[2], x[3]);
      q.z = tc::pack_bf16_relu(x[4], x[5]);
      q.w = tc::pack_bf16_relu(x[6], x[7]);
      *reinterpret_cast<uint4*>(tile + tc::sw128_offset(r, uint32_t(4 * h + c))) = q;
    }
  }
}

// Output layer of one row -> its mixture (as mixture()) as 16 float4:
// o[k] = (mu, kappa), o[8 + k] = (w, vmf normaliser, cdf, flag on k = 0).
// The first eight go to row r of the swizzled staging tile `st` (the group's H
// tile, free once the last layer's MMA is done), the other eight to the row's
// own 32 accumulator columns in TMEM (already read); the group copies them out
// as whole 128-byte segments, one half at a time. TMEM loads and stores are
// warp-wide.
__device__ __forceinline__ void head_to_stage(uint32_t tacc, float const* bias, float flag, uint8_t* st, uint32_t r) {
  float v[40];
  {
    float lo[32], hi[8];
    tc::tmem_ld32(tacc, lo);
    tc::tmem_ld8(tacc + 32u, hi);
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = lo[j] + bias[j];
#pragma unroll
    for (int j = 0; j < 8; ++j) v[32 + j] = hi[j] + bias[32 + j];
  }
  float mx = v[0];
#pragma unroll
  for (int k = 1; k < kGuideLobes; ++k) mx = fmaxf(mx, v[5 * k]);
  float sum = 0.f;
#pragma unroll
  for (int k = 0; k < kGuideLobes; ++k) {
    v[5 * k] = __expf(v[5 * k] - mx);
    sum += v[5 * k];
  }
  // fast intrinsics here: the lobes feed sampling and pdfs that always use the
  // stored values, so only their consistency matters, not their last bits
  float second[32];
  float cdf = 0.f;
  float const inv_sum = __frcp_rn(sum);
#pragma unroll
  for (int k = 0; k < kGuideLobes; ++k) {
    float const w = v[5 * k] * inv_sum;
    float const x = v[5 * k + 1];
    float const kap = fminf(fmaxf(x, 0.f) + __logf(1.f + __expf(-fabsf(x))) + kKappaMin, kKappaMax);
    cdf += w;
    float const mx3 = v[5 * k + 2], my = v[5 * k + 3], mz = v[5 * k + 4];
    float const l2 = mx3 * mx3 + my * my + mz * mz;
    float const il = rsqrtf(l2);
    float4 const mu = l2 > 1e-12f ? make_float4(mx3 * il, my * il, mz * il, kap) : make_float4(0.f, 0.f, 1.f, kap);
    *reinterpret_cast<float4*>(st + tc::sw128_offset(r, uint32_t(k))) = mu;
    second[4 * k + 0] = w;
    second[4 * k + 1] = __fdividef(kap, -6.28318530717958648f * (__expf(-2.f * kap) - 1.f));
    second[4 * k + 2] = k == kGuideLobes - 1 ? 1.f : cdf;
    second[4 * k + 3] = k == 0 ? flag : 0.f;
  }
  tc::tmem_st32(tacc, second);
}

// The second half back from TMEM into the staging tile.
__device__ __forceinline__ void second_to_stage(uint32_t tacc, uint8_t* st, uint32_t r) {
  float v[32];
  tc::tmem_ld32(tacc, v);
#pragma unroll
  for (int k = 0; k < kGuideLobes; ++k)
    *reinterpret_cast<float4*>(st + tc::sw128_offset(r, uint32_t(k))) =
        make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
}

// The group's staged 128 x 128-byte tile -> half `half` of the output rows
// (rows of 256 bytes); each warp store covers four whole 128-byte segments.
__device__ __forceinline__ void stage_out(uint8_t const* st, uint32_t tid, uint32_t first_row, uint32_t n, int half,
    float4* lobes) {
#pragma unroll
  for (uint32_t i = 0; i < 8; ++i) {
    uint32_t const idx = tid + 128u * i;
    uint32_t const r = idx >> 3, c = idx & 7u;
    if (first_row + r < n)
      lobes[size_t(first_row + r) * 2 * kGuideLobes + uint32_t(half) * kGuideLobes + c] =
          *reinterpret_cast<float4 const*>(st + tc::sw128_offset(r, c));
  }
}

__global__ void __launch_bounds__(128 * kFwdGroups, 2) k_guide_forward(mlp_args a, float4 const* __restrict__ points,
    uint32_t const* __restrict__ count_ptr, uint32_t n_fixed, float4* __restrict__ lobes) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* sm = align1024(smem_raw);
  uint8_t* wt = sm + kFwdW;
  float* bias = reinterpret_cast<float*>(sm + kFwdBias);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + kFwdTmem);
  uint32_t const warp = threadIdx.x >> 5;
  uint32_t const g = warp >> 2;                 // warpgroup: its tile, H buffer, TMEM columns, barrier
  uint32_t const q = warp & 3u;                 // TMEM lane quarter of this warp
  uint32_t const tid = threadIdx.x & 127u;      // row of the group's tile
  uint8_t* ht = sm + kFwdH + 16384u * g;
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kFwdBar) + g;
  uint64_t* stall_bar = reinterpret_cast<uint64_t*>(sm + kFwdStall) + g;
  uint32_t const bar_id = 1u + g;
  if (warp == 0) {
    tc::tmem_alloc(tmem_slot, 64 * kFwdGroups);
    tc::tmem_relinquish();
  }
  if (tid == 0) {
    tc::mbar_init(bar, 1);
    tc::mbar_init(stall_bar, 1);
  }
  load_weights(a, wt, bias);
  tc::fence_proxy_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  uint32_t const tmem = *tmem_slot + 64u * g;          // this group's accumulator columns
  uint32_t const tacc = tmem + ((32u * q) << 16);      // ... at this warp's lanes
  uint32_t const n = count_ptr ? *count_ptr : n_fixed;
  uint32_t phase = 0;
  bool failed = false;
  bool first_wait = true;
  constexpr uint32_t kIdF = tc::idesc_bf16_m128_n64(false, false);
  for (uint32_t tile = blockIdx.x * kFwdGroups + g; tile * 128u < n && !failed; tile += gridDim.x * kFwdGroups) {
    uint32_t const row = tile * 128u + tid;
    bool const valid = row < n;
    float4 p{0.f, 0.f, 0.f, 0.f}, nn{0.f, 0.f, 1.f, 0.f}, wo{0.f, 0.f, 1.f, 0.f};
    if (valid) {
      p = points[3 * size_t(row)];
      nn = points[3 * size_t(row) + 1];
      wo = points[3 * size_t(row) + 2];
    }
    encode_store(a, p, nn, wo, ht, tid);
    for (int l = 0; l < kLayers; ++l) {
      tc::fence_proxy_async();
      tc::fence_before_sync();
      tc::named_bar_sync(bar_id, 128);
      if (tid == 0) {
        tc::fence_after_sync();
        uint32_t const ha = tc::smem_u32(ht), wa = tc::smem_u32(wt + l * 8192);
#pragma unroll
        for (uint32_t k = 0; k < 4; ++k)
          tc::mma_bf16(tmem, tc::desc_sw128(ha + 32u * k, 16, 1024), tc::desc_sw128(wa + 32u * k, 16, 1024), kIdF,
              k > 0 ? 1u : 0u);
        tc::mma_commit(bar);
      }
      bool const ok = tc::mbar_wait_bounded(first_wait && a.stall ? stall_bar : bar, phase,
          first_wait ? a.poll_limit : kPollLimit);
      first_wait = false;
      phase ^= 1u;
      if (tc::named_bar_or(bar_id, 128, !ok)) {
        failed = true;
        break;
      }
      tc::fence_after_sync();
      if (l < kLayers - 1) {
        relu_to_tile(tacc, bias + 64 * l, ht, tid);
      } else {
        head_to_stage(tacc, bias + 64 * l, p.w, ht, tid);
        tc::named_bar_sync(bar_id, 128);
        stage_out(ht, tid, tile * 128u, n, 0, lobes);
        tc::named_bar_sync(bar_id, 128);
        second_to_stage(tacc, ht, tid);
        tc::named_bar_sync(bar_id, 128);
        stage_out(ht, tid, tile * 128u, n, 1, lobes);
        tc::named_bar_sync(bar_id, 128);  // the tile is rewritten next
      }
    }
  }
  if (failed) {
    if (tid == 0) atomicOr(a.err, ERR_GUIDE_TIMEOUT);
    tc::mbar_wait_bounded(bar, phase ^ 1u, kPollLimit);  // let the MMA in flight retire
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(*tmem_slot, 64 * kFwdGroups);
  }
}

// ---- k_guide_collect: records -> training samples ------------------------------------------
// records: [max_depth][stride] of kRecordWords float4; paths 0 .. n_paths-1 are live
__global__ void __launch_bounds__(256) k_guide_collect(float4 const* __restrict__ records, uint32_t stride,
    uint32_t n_paths, int max_depth, float tag, int radiance_only, float4 const* __restrict__ radiance,
    float4* __restrict__ samples, uint32_t capacity, uint32_t* __restrict__ count, float* __restrict__ sums) {
  size_t const total = size_t(n_paths) * size_t(max_depth);
  uint32_t const lane = threadIdx.x & 31u;
  float wsum = 0.f;
  // warp-uniform trip count; one atomic per warp and iteration reserves the slots
  for (size_t base = blockIdx.x * size_t(blockDim.x); base < total; base += size_t(gridDim.x) * blockDim.x) {
    size_t const i = base + threadIdx.x;
    bool keep = false;
    float w = 0.f;
    float4 r0, r1, r2, r3;
    if (i < total) {
      uint32_t const path = uint32_t(i % n_paths);
      size_t const v = i / n_paths;
      float4 const* r = records + (v * stride + path) * kRecordWords;
      r2 = r[2];
      if (r2.w == tag) {
        r0 = r[0], r1 = r[1], r3 = r[3];
        float4 const r4 = r[4], r5 = r[5];
        float4 const Lf = radiance[path];
        float const li_r = r4.x > 0.f ? (Lf.x - r5.x) / r4.x : 0.f;
        float const li_g = r4.y > 0.f ? (Lf.y - r5.y) / r4.y : 0.f;
        float const li_b = r4.z > 0.f ? (Lf.z - r5.z) / r4.z : 0.f;
        float const li = (0.2126f * li_r + 0.7152f * li_g) + 0.0722f * li_b;
        w = (radiance_only ? li : li * r1.w) / r0.w;
        keep = w > 0.f && isfinite(w);
      }
    }
    uint32_t const m = __ballot_sync(0xffffffffu, keep);
    uint32_t slot0 = 0;
    if (lane == 0 && m) slot0 = atomicAdd(count, uint32_t(__popc(m)));
    slot0 = __shfl_sync(0xffffffffu, slot0, 0);
    uint32_t const slot = slot0 + uint32_t(__popc(m & ((1u << lane) - 1u)));
    if (keep && slot < capacity) {
      wsum += w;
      float4* s = samples + size_t(slot) * 4;
      s[0] = make_float4(r0.x, r0.y, r0.z, w);
      s[1] = make_float4(r1.x, r1.y, r1.z, 0.f);
      s[2] = make_float4(r2.x, r2.y, r2.z, 0.f);
      s[3] = make_float4(r3.x, r3.y, r3.z, 0.f);
    }
  }
  for (int o = 16; o > 0; o >>= 1) wsum += __shfl_xor_sync(0xffffffffu, wsum, o);
  if (lane == 0 && wsum > 0.f) atomicAdd(sums + 1, wsum);
}

// ---- k_guide_train -----------------------------------------------------------------------------
// Shared memory: W 4 x 8 KB | H0..H3 4 x 16 KB | dZ 16 KB | zero 16 KB | bias 1 KB |
// dbias 1 KB | per-row (wi, weight) 2 KB | mbarrier | TMEM address | stall-test mbarrier.
constexpr uint32_t kTrW = 0, kTrH = 32768, kTrDZ = 98304, kTrZero = 114688, kTrBias = 131072, kTrDBias = 132096,
                   kTrRow = 133120, kTrBar = 135168, kTrTmem = 135176, kTrStall = 135184;
constexpr uint32_t kTrSmem = 135192 + 1024;
constexpr uint32_t kTmemCols = 512;  // accumulator (64) + dW for 4 layers (4 x 64)

struct train_args {
  mlp_args m;
  float4 const* samples;  // 4 float4 per sample
  uint32_t const* count;  // samples available (device), or null: n_fixed
  uint32_t n_fixed;
  uint32_t capacity;
  uint32_t batch;         // samples per step
  uint32_t step;          // which block of the sample buffer this step uses
  float const* sums;      // [1] = weight sum of the collected samples (null: no normalisation)
  float clamp;            // normalised weights above this are clamped (0: off)
  float* partials;        // [gridDim.x][kParams]: each CTA stores its gradient sum
  float* loss;            // loss sum (atomic)
};

__device__ __forceinline__ void warp_bias_sum(float const (&g)[64], float* dst) {
#pragma unroll
  for (int j = 0; j < 64; ++j) {
    float v = g[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(dst + j, v);
  }
}

__global__ void __launch_bounds__(128, 1) k_guide_train(train_args a) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* sm = align1024(smem_raw);
  uint8_t* wt = sm + kTrW;
  uint8_t* dz = sm + kTrDZ;
  uint8_t* zt = sm + kTrZero;
  float* bias = reinterpret_cast<float*>(sm + kTrBias);
  float* dbias = reinterpret_cast<float*>(sm + kTrDBias);
  float4* rowd = reinterpret_cast<float4*>(sm + kTrRow);
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kTrBar);
  uint64_t* stall_bar = reinterpret_cast<uint64_t*>(sm + kTrStall);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + kTrTmem);
  uint32_t const tid = threadIdx.x, warp = tid >> 5;
  auto H = [&](int l) { return sm + kTrH + uint32_t(l) * 16384u; };

  if (warp == 0) {
    tc::tmem_alloc(tmem_slot, kTmemCols);
    tc::tmem_relinquish();
  }
  if (tid == 0) {
    tc::mbar_init(bar, 1);
    tc::mbar_init(stall_bar, 1);
  }
  load_weights(a.m, wt, bias);
  for (uint32_t i = tid; i < 16384 / 16; i += blockDim.x) reinterpret_cast<uint4*>(zt)[i] = make_uint4(0, 0, 0, 0);
  for (uint32_t i = tid; i < kLayers * 64; i += blockDim.x) dbias[i] = 0.f;
  tc::fence_proxy_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  uint32_t const tmem = *tmem_slot;

  uint32_t const avail = a.count ? min(*a.count, a.capacity) : a.n_fixed;
  uint32_t n = min(avail, a.batch);
  uint32_t first = 0;
  if (avail > a.batch) first = uint32_t((uint64_t(a.step) * a.batch) % uint64_t(avail - a.batch + 1));
  float scale = 1.f, wmax = __builtin_huge_valf();
  if (a.sums && avail > 0) {
    float const mean = a.sums[1] / float(avail);
    scale = mean > 0.f ? 1.f / (mean * float(max(n, 1u))) : 0.f;
    if (a.clamp > 0.f) wmax = a.clamp / float(max(n, 1u));  // clamp * mean, after scaling
  }

  constexpr uint32_t kIdF = tc::idesc_bf16_m128_n64(false, false);
  constexpr uint32_t kIdDH = tc::idesc_bf16_m128_n64(false, true);
  constexpr uint32_t kIdDW = tc::idesc_bf16_m128_n64(true, true);
  uint32_t phase = 0;
  bool failed = false;
  bool first_wait = true;
  uint32_t tiles_done = 0;
  float loss_acc = 0.f;

  auto sync_for_mma = [&]() {
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
  };
  auto wait_mma = [&]() -> bool {
    bool const ok = tc::mbar_wait_bounded(first_wait && a.m.stall ? stall_bar : bar, phase,
        first_wait ? a.m.poll_limit : kPollLimit);
    first_wait = false;
    phase ^= 1u;
    bool const bad = __syncthreads_or(!ok);
    tc::fence_after_sync();
    return !bad;
  };

  for (uint32_t tile = blockIdx.x; tile * 128u < n && !failed; tile += gridDim.x) {
    uint32_t const row = tile * 128u + tid;
    bool const valid = row < n;
    float f[64];
    float4 s0{0.f, 0.f, 0.f, 0.f}, s1{0.f, 0.f, 1.f, 0.f}, s2{0.f, 0.f, 1.f, 0.f}, s3{0.f, 0.f, 1.f, 0.f};
    if (valid) {
      float4 const* s = a.samples + size_t(first + row) * 4;
      s0 = s[0], s1 = s[1], s2 = s[2], s3 = s[3];
    }
    rowd[tid] = make_float4(s3.x, s3.y, s3.z, valid ? fminf(s0.w * scale, wmax) : 0.f);
    encode(a.m, s0, s1, s2, f);
    store_row(H(0), tid, f);
    // forward
    for (int l = 0; l < kLayers && !failed; ++l) {
      sync_for_mma();
      if (tid == 0) {
        tc::fence_after_sync();
        uint32_t const ha = tc::smem_u32(H(l)), wa = tc::smem_u32(wt + l * 8192);
#pragma unroll
        for (uint32_t k = 0; k < 4; ++k)
          tc::mma_bf16(tmem, tc::desc_sw128(ha + 32u * k, 16, 1024), tc::desc_sw128(wa + 32u * k, 16, 1024), kIdF,
              k > 0 ? 1u : 0u);
        tc::mma_commit(bar);
      }
      if (!wait_mma()) {
        failed = true;
        break;
      }
      acc_row(tmem, 0, bias + 64 * l, f);
      if (l < kLayers - 1) {
#pragma unroll
        for (int j = 0; j < 64; ++j) f[j] = fmaxf(f[j], 0.f);
        store_row(H(l + 1), tid, f);
      }
    }
    if (failed) break;
    // loss gradient w.r.t. the 40 outputs
    {
      float4 const rd = rowd[tid];
      float const wgt = rd.w;
      lobe_set L;
      mixture(f, L);
      float fk[kGuideLobes], ck[kGuideLobes];
      float q = 0.f;
#pragma unroll
      for (int k = 0; k < kGuideLobes; ++k) {
        ck[k] = (L.mu[k][0] * rd.x + L.mu[k][1] * rd.y) + L.mu[k][2] * rd.z;
        fk[k] = vmf_norm(L.kappa[k]) * expf(L.kappa[k] * (ck[k] - 1.f));
        q += L.w[k] * fk[k];
      }
      float g[64];
#pragma unroll
      for (int j = 0; j < 64; ++j) g[j] = 0.f;
      if (wgt > 0.f && q > 1e-30f) {
        loss_acc += -wgt * logf(q);
        float const gq = -wgt / q;  // d loss / d q
#pragma unroll
        for (int k = 0; k < kGuideLobes; ++k) {
          float const kap = L.kappa[k];
          float const wf = L.w[k] * fk[k];
          g[5 * k] = gq * L.w[k] * (fk[k] - q);
          float const dlnc = 1.f / kap - 2.f / expm1f(2.f * kap);
          g[5 * k + 1] = gq * wf * (dlnc + (ck[k] - 1.f)) * L.dk[k];
          if (L.len[k] > 1e-6f) {
            float const gm = gq * wf * kap;  // d loss / d (mu . wi)
            float const dmu[3] = {gm * rd.x, gm * rd.y, gm * rd.z};
            float const proj = (dmu[0] * L.mu[k][0] + dmu[1] * L.mu[k][1]) + dmu[2] * L.mu[k][2];
#pragma unroll
            for (int c = 0; c < 3; ++c) g[5 * k + 2 + c] = (dmu[c] - proj * L.mu[k][c]) / L.len[k];
          }
        }
      }
      store_row(dz, tid, g);
      // bias gradient of the output layer from the BF16 values the MMAs see
      load_row(dz, tid, g);
      warp_bias_sum(g, dbias + 64 * 3);
    }
    // backward
    for (int l = kLayers - 1; l >= 0 && !failed; --l) {
      sync_for_mma();
      if (tid == 0) {
        tc::fence_after_sync();
        uint32_t const dza = tc::smem_u32(dz), ha = tc::smem_u32(H(l)), wa = tc::smem_u32(wt + l * 8192);
        // dW_l += dZ^T H_l over the 128 samples (K): A MN-major, its second 64-row
        // half read from the zero tile, B MN-major
        for (uint32_t k = 0; k < 8; ++k)
          tc::mma_bf16(tmem + 64u + 64u * uint32_t(l), tc::desc_sw128(dza + 2048u * k, kTrZero - kTrDZ, 1024),
              tc::desc_sw128(ha + 2048u * k, 16, 1024), kIdDW, (tiles_done > 0 || k > 0) ? 1u : 0u);
        if (l > 0) {
          // dH_l = dZ W_l: A K-major over the 64 outputs, B = W_l read MN-major
#pragma unroll
          for (uint32_t k = 0; k < 4; ++k)
            tc::mma_bf16(tmem, tc::desc_sw128(dza + 32u * k, 16, 1024), tc::desc_sw128(wa + 2048u * k, 16, 1024),
                kIdDH, k > 0 ? 1u : 0u);
        }
        tc::mma_commit(bar);
      }
      if (!wait_mma()) {
        failed = true;
        break;
      }
      if (l > 0) {
        float g[64], h[64];
        acc_row(tmem, 0, nullptr, g);
        load_row(H(l), tid, h);
#pragma unroll
        for (int j = 0; j < 64; ++j) g[j] = h[j] > 0.f ? g[j] : 0.f;
        store_row(dz, tid, g);
        load_row(dz, tid, g);
        warp_bias_sum(g, dbias + 64 * (l - 1));
      }
    }
    ++tiles_done;
  }
  if (failed) {
    if (tid == 0) atomicOr(a.m.err, ERR_GUIDE_TIMEOUT);
    tc::mbar_wait_bounded(bar, phase ^ 1u, kPollLimit);
  }
  // flush: this CTA's partial gradient, every entry written (zeros when it had
  // no tile): weight rows from TMEM (rows 0..63 live in warps 0 and 1), bias sums
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  bool const have = !failed && tiles_done > 0;
  float* part = a.partials + size_t(blockIdx.x) * kParams;
  if (warp < 2) {
    uint32_t const out = tid;  // row of dW = output index
    for (int l = 0; l < kLayers; ++l) {
      float g[64];
      if (have) acc_row(tmem, 64u + 64u * uint32_t(l), nullptr, g);
      else
#pragma unroll
        for (int j = 0; j < 64; ++j) g[j] = 0.f;
      float4* dst = reinterpret_cast<float4*>(part + (size_t(l) * 64 + out) * 64);
#pragma unroll
      for (int j = 0; j < 16; ++j) dst[j] = make_float4(g[4 * j], g[4 * j + 1], g[4 * j + 2], g[4 * j + 3]);
    }
  }
  for (uint32_t i = tid; i < kLayers * 64; i += blockDim.x) part[kLayers * 64 * 64 + i] = have ? dbias[i] : 0.f;
  for (int o = 16; o > 0; o >>= 1) loss_acc += __shfl_xor_sync(0xffffffffu, loss_acc, o);
  if ((tid & 31) == 0 && loss_acc != 0.f && a.loss) atomicAdd(a.loss, loss_acc);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, kTmemCols);
  }
}

// ---- gradient reduction, Adam + BF16 copy -------------------------------------------------------
// A block sums 32 parameters over the n_parts partial gradients: its 8 warps
// take every 8th part (a warp reads 128 contiguous bytes per part), then warp
// 0 adds the 8 sums in a fixed order, so the result does not depend on timing.
constexpr uint32_t kRedParams = 32;
__device__ __forceinline__ float reduce_parts(float const* __restrict__ parts, uint32_t n_parts, float* red) {
  uint32_t const lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  uint32_t const i = blockIdx.x * kRedParams + lane;
  float acc = 0.f;
  if (i < uint32_t(kParams))
    for (uint32_t q = warp; q < n_parts; q += 8u) acc += parts[size_t(q) * kParams + i];
  red[warp * 32u + lane] = acc;
  __syncthreads();
  float gi = 0.f;
  if (warp == 0)
#pragma unroll
    for (int w = 0; w < 8; ++w) gi += red[w * 32 + lane];
  return gi;
}

__global__ void __launch_bounds__(256) k_guide_reduce(float const* __restrict__ parts, uint32_t n_parts,
    float* __restrict__ g) {
  __shared__ float red[256];
  float const gi = reduce_parts(parts, n_parts, red);
  uint32_t const i = blockIdx.x * kRedParams + threadIdx.x;
  if (threadIdx.x < 32 && i < uint32_t(kParams)) g[i] = gi;
}

__global__ void __launch_bounds__(256) k_guide_adam(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
    float const* __restrict__ parts, uint32_t n_parts, uint16_t* __restrict__ wbf, float lr, float b1, float b2,
    float eps, float c1, float c2, uint32_t const* __restrict__ count) {
  __shared__ float red[256];
  if (count && *count == 0) return;  // nothing collected: no step
  float const gi = reduce_parts(parts, n_parts, red);
  uint32_t const i = blockIdx.x * kRedParams + threadIdx.x;
  if (threadIdx.x >= 32 || i >= uint32_t(kParams)) return;
  float const mi = b1 * m[i] + (1.f - b1) * gi;
  float const vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  float const pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  p[i] = pi;
  if (i < uint32_t(kLayers * 64 * 64)) wbf[i] = uint16_t(tc::pack_bf16(pi, 0.f) & 0xffffu);
}

__global__ void k_guide_to_bf16(float const* __restrict__ p, uint16_t* __restrict__ wbf) {
  uint32_t const i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < uint32_t(kLayers * 64 * 64)) wbf[i] = uint16_t(tc::pack_bf16(p[i], 0.f) & 0xffffu);
}

// ---- host helpers ----------------------------------------------------------------------------
template <typename T> int grow(myrt_ctx* ctx, T** p, size_t& cap, size_t want, size_t elem, char const* what) {
  if (cap >= want && *p) return MYRT_OK;
  cudaFree(*p);
  *p = nullptr;
  cap = 0;
  int rc = check_cuda(ctx, cudaMalloc(reinterpret_cast<void**>(p), want * elem), what);
  if (rc) return rc;
  cap = want;
  return MYRT_OK;
}

int init_params(myrt_ctx* ctx, guide_state& g) {
  std::vector<float> h(kParams, 0.f);
  std::mt19937 rng(g.prm.seed);
  float const lim = std::sqrt(6.f / 128.f);  // Glorot uniform, 64 + 64
  std::uniform_real_distribution<float> U(-lim, lim);
  for (int i = 0; i < kLayers * 64 * 64; ++i) h[i] = U(rng);
  // output layer: small weights, so the first mixtures are broad and even
  for (int i = 3 * 4096; i < 4 * 4096; ++i) h[i] *= 0.1f;
  cudaStream_t st = ctx->stream;
  int rc = check_cuda(ctx, cudaMemcpyAsync(g.params, h.data(), kParams * 4, cudaMemcpyHostToDevice, st), "guide init");
  if (!rc) rc = check_cuda(ctx, cudaMemsetAsync(g.adam_m, 0, kParams * 4, st), "guide init");
  if (!rc) rc = check_cuda(ctx, cudaMemsetAsync(g.adam_v, 0, kParams * 4, st), "guide init");
  if (!rc) rc = check_cuda(ctx, cudaMemsetAsync(g.grads, 0, kParams * 4, st), "guide init");
  if (!rc) {
    k_guide_to_bf16<<<(kLayers * 4096 + 255) / 256, 256, 0, st>>>(g.params, g.w_bf16);
    rc = check_cuda(ctx, cudaGetLastError(), "guide init");
  }
  if (!rc) rc = check_cuda(ctx, cudaStreamSynchronize(st), "guide init");
  // the host copy above must outlive the async copy: synchronised here
  g.adam_t = 0;
  g.steps = 0;
  g.wave = 0;
  g.waves_trained = 0;
  return rc;
}

int ensure_guide(myrt_ctx* ctx) {
  if (!ctx->guide) {
    ctx->guide = new guide_state();
    guide_state& g = *ctx->guide;
    int rc = MYRT_OK;
    auto alloc = [&](void** p, size_t bytes) {
      if (!rc) rc = check_cuda(ctx, cudaMalloc(p, bytes), "guide state");
    };
    alloc(reinterpret_cast<void**>(&g.params), kParams * 4);
    alloc(reinterpret_cast<void**>(&g.adam_m), kParams * 4);
    alloc(reinterpret_cast<void**>(&g.adam_v), kParams * 4);
    alloc(reinterpret_cast<void**>(&g.grads), kParams * 4);
    g.max_parts = uint32_t(std::max(ctx->sm_count, 1));
    alloc(reinterpret_cast<void**>(&g.partials), size_t(g.max_parts) * kParams * 4);
    alloc(reinterpret_cast<void**>(&g.w_bf16), kLayers * 4096 * 2);
    alloc(reinterpret_cast<void**>(&g.sums), 4 * 4);
    alloc(reinterpret_cast<void**>(&g.counters), 4 * 4);
    if (!rc) rc = check_cuda(ctx, cudaFuncSetAttribute(k_guide_forward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(kFwdSmem)), "guide kernel attributes");
    if (!rc) rc = check_cuda(ctx, cudaFuncSetAttribute(k_guide_train, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(kTrSmem)), "guide kernel attributes");
    if (!rc) rc = init_params(ctx, g);
    if (rc) {
      free_guide(ctx->guide);
      ctx->guide = nullptr;
      return rc;
    }
    g.generation = ctx->guide_generation;
  }
  if (ctx->guide->generation != ctx->guide_generation) {  // new scene: start learning afresh
    int rc = init_params(ctx, *ctx->guide);
    if (rc) return rc;
    ctx->guide->generation = ctx->guide_generation;
  }
  return MYRT_OK;
}

mlp_args make_mlp(myrt_ctx* ctx) {
  guide_state const& g = *ctx->guide;
  mlp_args a{};
  a.w = g.w_bf16;
  a.bias = g.params + kLayers * 4096;
  float const* b = ctx->scene.bounds;
  for (int k = 0; k < 3; ++k) {
    float const c = 0.5f * (b[k] + b[3 + k]);
    float const h = 0.5f * (b[3 + k] - b[k]);
    a.center[k] = c;
    a.inv_half[k] = h > 0.f ? 1.f / h : 1.f;
  }
  a.err = ctx->d_err;
  a.poll_limit = ctx->tuning.guide_poll_limit ? ctx->tuning.guide_poll_limit : kPollLimit;
  a.stall = ctx->tuning.guide_stall_test ? 1u : 0u;
  return a;
}

int launch_forward(myrt_ctx* ctx, mlp_args const& a, float4 const* points, uint32_t const* count, uint32_t n_fixed,
    size_t max_rows, float4* lobes, cudaStream_t st) {
  uint32_t const tiles = uint32_t((max_rows + 127) / 128);
  uint32_t const ctas = (tiles + kFwdGroups - 1) / kFwdGroups;
  uint32_t const grid = std::max(1u, std::min(ctas, uint32_t(std::max(ctx->sm_count, 1)) * 2u));
  k_guide_forward<<<grid, 128 * kFwdGroups, kFwdSmem, st>>>(a, points, count, n_fixed, lobes);
  return check_cuda(ctx, cudaGetLastError(), "guide forward launch");
}

// Launches one training pass; *parts = CTAs launched (partial gradients written).
int launch_train(myrt_ctx* ctx, train_args ta, uint32_t max_rows, cudaStream_t st, uint32_t* parts) {
  guide_state& g = *ctx->guide;
  uint32_t const tiles = (max_rows + 127) / 128;
  uint32_t const grid = std::max(1u, std::min(tiles, g.max_parts));
  ta.partials = g.partials;
  k_guide_train<<<grid, 128, kTrSmem, st>>>(ta);
  *parts = grid;
  return check_cuda(ctx, cudaGetLastError(), "guide train launch");
}

constexpr uint32_t kRedBlocks = (uint32_t(kParams) + kRedParams - 1) / kRedParams;

int adam_step(myrt_ctx* ctx, guide_state& g, uint32_t parts, uint32_t const* count, cudaStream_t st) {
  g.adam_t++;
  float const b1 = 0.9f, b2 = 0.99f;
  float const c1 = float(1.0 - std::pow(double(b1), double(g.adam_t)));
  float const c2 = float(1.0 - std::pow(double(b2), double(g.adam_t)));
  k_guide_adam<<<kRedBlocks, 256, 0, st>>>(g.params, g.adam_m, g.adam_v, g.partials, parts, g.w_bf16,
      g.prm.learning_rate, b1, b2, 1e-8f, c1, c2, count);
  g.steps++;
  return check_cuda(ctx, cudaGetLastError(), "guide adam launch");
}

}  // namespace

void free_guide(guide_state* g) {
  if (!g) return;
  for (void* p : {static_cast<void*>(g->params), static_cast<void*>(g->adam_m), static_cast<void*>(g->adam_v),
           static_cast<void*>(g->grads), static_cast<void*>(g->partials), static_cast<void*>(g->w_bf16),
           static_cast<void*>(g->sums),
           static_cast<void*>(g->counters), static_cast<void*>(g->points), static_cast<void*>(g->lobes),
           static_cast<void*>(g->records), static_cast<void*>(g->samples)})
    cudaFree(p);
  delete g;
}

// ---- wavefront hooks ----------------------------------------------------------------------------
int guide_prepare(myrt_ctx* ctx, size_t paths, myrt_render_params const* p, guide_dev& gd) {
  gd = guide_dev{};
  int rc = ensure_guide(ctx);
  if (rc) return rc;
  guide_state& g = *ctx->guide;
  int const depth = p->max_depth > 0 ? p->max_depth : 8;
  if (g.rows_cap < paths || !g.points || !g.lobes) {
    cudaFree(g.points);
    cudaFree(g.lobes);
    g.points = g.lobes = nullptr;
    g.rows_cap = 0;
    rc = check_cuda(ctx, cudaMalloc(reinterpret_cast<void**>(&g.points), paths * 48), "guide points");
    if (!rc) rc = check_cuda(ctx, cudaMalloc(reinterpret_cast<void**>(&g.lobes), paths * 256), "guide lobes");
    if (rc) return rc;
    g.rows_cap = paths;
  }
  size_t const nrec = paths * size_t(depth);
  if (!rc && (g.records_cap < nrec || !g.records)) {
    rc = grow(ctx, &g.records, g.records_cap, nrec, kRecordWords * sizeof(float4), "guide records");
    if (!rc) rc = check_cuda(ctx, cudaMemsetAsync(g.records, 0, nrec * kRecordWords * sizeof(float4), ctx->stream),
                      "clear");
    g.tag = 0;
  }
  if (!rc) rc = grow(ctx, &g.samples, g.samples_cap, std::max<size_t>(paths, 1u << 20), 4 * sizeof(float4),
                    "guide samples");
  if (rc) return rc;
  gd.paths = uint32_t(paths);
  gd.lobes = g.lobes;
  gd.records = g.prm.train ? g.records : nullptr;
  return MYRT_OK;
}

int guide_schedule(myrt_ctx* ctx, uint64_t* waves_trained, bool* training) {
  int rc = ensure_guide(ctx);
  if (rc) return rc;
  *waves_trained = ctx->guide->waves_trained;
  *training = ctx->guide->prm.train != 0;
  return MYRT_OK;
}

void guide_begin_wave(myrt_ctx* ctx, guide_dev& gd) {
  guide_state& g = *ctx->guide;
  g.tag = (g.tag + 1u) & 0xffffffu;
  if (g.tag == 0) g.tag = 1;
  gd.tag = float(g.tag);
  bool const warm = g.waves_trained >= g.prm.warmup_waves || !g.prm.train;
  gd.n_lobes = warm && g.prm.fraction > 0.f ? kGuideLobes : 0;
  gd.fraction = gd.n_lobes ? g.prm.fraction : 0.f;
  g.wave++;
}

int guide_infer(myrt_ctx* ctx, guide_dev const& gd, uint32_t, uint32_t, float4 const* queue, float4 const* hits,
    uint32_t const* count, cudaStream_t st) {
  if (gd.n_lobes == 0) return MYRT_OK;
  guide_state& g = *ctx->guide;
  uint32_t const grid = uint32_t(std::max(ctx->sm_count, 1)) * 4u;
  k_guide_gather<<<grid, 256, 0, st>>>(queue, hits, count, g.points);
  int rc = check_cuda(ctx, cudaGetLastError(), "guide gather launch");
  if (rc) return rc;
  return launch_forward(ctx, make_mlp(ctx), g.points, count, 0, gd.paths, g.lobes, st);
}

int guide_train(myrt_ctx* ctx, guide_dev const& gd, uint32_t paths, int max_depth, float4 const* radiance,
    cudaStream_t st) {
  guide_state& g = *ctx->guide;
  if (!gd.records || !g.prm.train) return MYRT_OK;
  int rc = check_cuda(ctx, cudaMemsetAsync(g.counters, 0, 16, st), "guide counters");
  if (!rc) rc = check_cuda(ctx, cudaMemsetAsync(g.sums, 0, 16, st), "guide sums");
  if (rc) return rc;
  uint32_t const grid = uint32_t(std::max(ctx->sm_count, 1)) * 8u;
  k_guide_collect<<<grid, 256, 0, st>>>(g.records, gd.paths, paths, max_depth, gd.tag, int(g.prm.target == 1),
      radiance, g.samples,
      uint32_t(g.samples_cap), g.counters, g.sums);
  rc = check_cuda(ctx, cudaGetLastError(), "guide collect launch");
  train_args ta{};
  ta.m = make_mlp(ctx);
  ta.samples = g.samples;
  ta.count = g.counters;
  ta.capacity = uint32_t(g.samples_cap);
  ta.batch = g.prm.batch;
  ta.sums = g.sums;
  ta.clamp = g.prm.weight_clamp;
  ta.loss = g.sums;
  for (uint32_t s = 0; !rc && s < g.prm.train_steps; ++s) {
    ta.step = uint32_t(g.steps);
    uint32_t parts = 0;
    rc = launch_train(ctx, ta, g.prm.batch, st, &parts);
    if (!rc) rc = adam_step(ctx, g, parts, g.counters, st);
  }
  g.waves_trained++;
  return rc;
}

// ---- C ABI helpers (api.cu) -----------------------------------------------------------------------
int guide_configure(myrt_ctx* ctx, myrt_guide_params const* p) {
  if (!(p->fraction >= 0.f && p->fraction <= 1.f) || !(p->learning_rate > 0.f) || p->batch < 128 ||
      p->batch % 128 != 0 || p->batch > (1u << 24) || p->train_steps > 1024 || !(p->weight_clamp >= 0.f) || p->target > 1)
    return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "guide parameters out of range");
  int rc = ensure_guide(ctx);
  if (rc) return rc;
  bool const reseed = p->seed != ctx->guide->prm.seed;
  ctx->guide->prm = *p;
  return reseed ? init_params(ctx, *ctx->guide) : MYRT_OK;
}

int guide_get_config(myrt_ctx* ctx, myrt_guide_params* p) {
  if (ctx->guide) *p = ctx->guide->prm;
  else *p = guide_state{}.prm;
  return MYRT_OK;
}

int guide_reset(myrt_ctx* ctx) {
  int rc = ensure_guide(ctx);
  if (rc) return rc;
  return init_params(ctx, *ctx->guide);
}

int guide_params_io(myrt_ctx* ctx, float* out, float const* in) {
  int rc = ensure_guide(ctx);
  if (rc) return rc;
  guide_state& g = *ctx->guide;
  cudaStream_t st = ctx->stream;
  if (in) {
    rc = check_cuda(ctx, cudaMemcpyAsync(g.params, in, kParams * 4, cudaMemcpyHostToDevice, st), "guide params");
    if (!rc) {
      k_guide_to_bf16<<<(kLayers * 4096 + 255) / 256, 256, 0, st>>>(g.params, g.w_bf16);
      rc = check_cuda(ctx, cudaGetLastError(), "guide params");
    }
  } else {
    rc = check_cuda(ctx, cudaMemcpyAsync(out, g.params, kParams * 4, cudaMemcpyDeviceToHost, st), "guide params");
  }
  if (!rc) rc = check_cuda(ctx, cudaStreamSynchronize(st), "guide params");
  return rc;
}

int guide_eval(myrt_ctx* ctx, float const* points, uint32_t n, float* lobes) {
  int rc = ensure_guide(ctx);
  if (rc || n == 0) return rc;
  cudaStream_t st = ctx->stream;
  void* d_pts = nullptr;
  void* d_lobes = nullptr;
  rc = check_cuda(ctx, cudaMalloc(&d_pts, size_t(n) * 48), "guide eval buffers");
  if (!rc) rc = check_cuda(ctx, cudaMalloc(&d_lobes, size_t(n) * 256), "guide eval buffers");
  if (!rc) rc = check_cuda(ctx, cudaMemcpyAsync(d_pts, points, size_t(n) * 48, cudaMemcpyHostToDevice, st), "upload");
  if (!rc)
    rc = launch_forward(ctx, make_mlp(ctx), static_cast<float4 const*>(d_pts), nullptr, n, n,
        static_cast<float4*>(d_lobes), st);
  if (!rc) rc = check_cuda(ctx, cudaMemcpyAsync(lobes, d_lobes, size_t(n) * 256, cudaMemcpyDeviceToHost, st), "read");
  if (!rc) rc = check_cuda(ctx, cudaStreamSynchronize(st), "guide eval");
  cudaFree(d_pts);
  cudaFree(d_lobes);
  return rc;
}

int guide_gradients(myrt_ctx* ctx, float const* samples, uint32_t n, float* grads, float* loss) {
  int rc = ensure_guide(ctx);
  if (rc) return rc;
  guide_state& g = *ctx->guide;
  cudaStream_t st = ctx->stream;
  void* d_s = nullptr;
  void* d_loss = nullptr;
  rc = check_cuda(ctx, cudaMalloc(&d_s, std::max<size_t>(n, 1) * 64), "guide gradient buffers");
  if (!rc) rc = check_cuda(ctx, cudaMalloc(&d_loss, 4), "guide gradient buffers");
  if (!rc && n) rc = check_cuda(ctx, cudaMemcpyAsync(d_s, samples, size_t(n) * 64, cudaMemcpyHostToDevice, st), "upload");
  if (!rc) rc = check_cuda(ctx, cudaMemsetAsync(g.grads, 0, kParams * 4, st), "clear");
  if (!rc) rc = check_cuda(ctx, cudaMemsetAsync(d_loss, 0, 4, st), "clear");
  if (!rc && n) {
    train_args ta{};
    ta.m = make_mlp(ctx);
    ta.samples = static_cast<float4 const*>(d_s);
    ta.count = nullptr;
    ta.n_fixed = n;
    ta.capacity = n;
    ta.batch = n;
    ta.step = 0;
    ta.sums = nullptr;
    ta.loss = static_cast<float*>(d_loss);
    uint32_t parts = 0;
    rc = launch_train(ctx, ta, n, st, &parts);
    if (!rc) {
      k_guide_reduce<<<kRedBlocks, 256, 0, st>>>(g.partials, parts, g.grads);
      rc = check_cuda(ctx, cudaGetLastError(), "guide reduce launch");
    }
  }
  if (!rc) rc = check_cuda(ctx, cudaMemcpyAsync(grads, g.grads, kParams * 4, cudaMemcpyDeviceToHost, st), "read");
  if (!rc && loss) rc = check_cuda(ctx, cudaMemcpyAsync(loss, d_loss, 4, cudaMemcpyDeviceToHost, st), "read");
  if (!rc) rc = check_cuda(ctx, cudaMemsetAsync(g.grads, 0, kParams * 4, st), "clear");
  if (!rc) rc = check_cuda(ctx, cudaStreamSynchronize(st), "guide gradients");
  cudaFree(d_s);
  cudaFree(d_loss);
  return rc;
}

int guide_train_samples(myrt_ctx* ctx, float const* samples, uint32_t n, uint32_t steps, float* loss_per_step) {
  int rc = ensure_guide(ctx);
  if (rc) return rc;
  guide_state& g = *ctx->guide;
  cudaStream_t st = ctx->stream;
  void* d_s = nullptr;
  void* d_loss = nullptr;
  rc = check_cuda(ctx, cudaMalloc(&d_s, std::max<size_t>(n, 1) * 64), "guide training buffers");
  if (!rc) rc = check_cuda(ctx, cudaMalloc(&d_loss, std::max<size_t>(steps, 1) * 4), "guide training buffers");
  if (!rc && n) rc = check_cuda(ctx, cudaMemcpyAsync(d_s, samples, size_t(n) * 64, cudaMemcpyHostToDevice, st), "upload");
  if (!rc) rc = check_cuda(ctx, cudaMemsetAsync(d_loss, 0, std::max<size_t>(steps, 1) * 4, st), "clear");
  uint32_t const batch = std::min(n, g.prm.batch);
  for (uint32_t s = 0; !rc && n && s < steps; ++s) {
    train_args ta{};
    ta.m = make_mlp(ctx);
    ta.samples = static_cast<float4 const*>(d_s);
    ta.count = nullptr;
    ta.n_fixed = n;
    ta.capacity = n;
    ta.batch = batch;
    ta.step = s;
    ta.sums = nullptr;
    ta.loss = static_cast<float*>(d_loss) + s;
    uint32_t parts = 0;
    rc = launch_train(ctx, ta, batch, st, &parts);
    if (!rc) rc = adam_step(ctx, g, parts, nullptr, st);
  }
  if (!rc && loss_per_step && steps)
    rc = check_cuda(ctx, cudaMemcpyAsync(loss_per_step, d_loss, size_t(steps) * 4, cudaMemcpyDeviceToHost, st), "read");
  if (!rc) rc = check_cuda(ctx, cudaStreamSynchronize(st), "guide training");
  cudaFree(d_s);
  cudaFree(d_loss);
  return rc;
}

int guide_stats(myrt_ctx* ctx, myrt_guide_stats* out) {
  std::memset(out, 0, sizeof(*out));
  if (!ctx->guide) return MYRT_OK;
  guide_state& g = *ctx->guide;
  out->adam_steps = g.steps;
  out->waves = g.wave;
  out->waves_trained = g.waves_trained;
  uint32_t c[4] = {0, 0, 0, 0};
  float s[4] = {0, 0, 0, 0};
  int rc = check_cuda(ctx, cudaMemcpyAsync(c, g.counters, 16, cudaMemcpyDeviceToHost, ctx->stream), "read");
  if (!rc) rc = check_cuda(ctx, cudaMemcpyAsync(s, g.sums, 16, cudaMemcpyDeviceToHost, ctx->stream), "read");
  if (!rc) rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "read");
  out->last_samples = c[0];
  out->last_loss = s[0];
  out->last_weight_sum = s[1];
  return rc;
}

}  // namespace myrt_b200
