// Learned path guiding: device-side view of the guide for the shade pass.
//
// The guide is a mixture of K von Mises-Fisher lobes per shading point,
// produced by a small MLP (guide.cu) from frequency-encoded position, the
// shading normal and the view direction. The shade pass draws the
// continuation from the guide with probability `fraction`, else from the
// BSDF, and weights it by the one-sample MIS mixture pdf
//   p(wi) = fraction * q(wi) + (1 - fraction) * p_bsdf(wi),
// so the estimator stays unbiased whatever the network outputs. Each sampled
// vertex leaves a training record; after the wave the incident radiance along
// its direction is (L_path - L_at_vertex) / throughput.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/myrt_cuda.h"
#include "refshade.cuh"

struct myrt_ctx;

namespace myrt_b200 {

constexpr int kGuideLobes = 8;
constexpr int kRecordWords = 6;  // float4 per training record

struct guide_dev {
  int n_lobes;          // 0: guiding off for this wave
  float fraction;       // probability of sampling the guide
  float4 const* lobes;  // per queue slot: 2 float4 per lobe (mu, kappa), (weight, norm, cdf, valid)
  float4* records;      // [max_depth][paths] records, kRecordWords float4 each
  uint32_t paths;       // record stride (paths per wave)
  float tag;            // record validity tag of this wave
};

struct guide_lobes {
  float4 a[kGuideLobes];  // mu xyz, kappa
  float4 b[kGuideLobes];  // weight, kappa / (2 pi (1 - exp(-2 kappa))), cdf, valid
};

__device__ __forceinline__ bool guide_load(guide_dev const& g, uint32_t slot, guide_lobes& gl) {
  if (!g.lobes) return false;
  float4 const* p = g.lobes + size_t(slot) * 2 * kGuideLobes;
#pragma unroll
  for (int k = 0; k < kGuideLobes; ++k) {
    gl.a[k] = p[k];
    gl.b[k] = p[kGuideLobes + k];
  }
  return gl.b[0].w > 0.f;
}

__device__ __forceinline__ float guide_pdf(guide_lobes const& gl, rs::v3 wi) {
  float q = 0.f;
#pragma unroll
  for (int k = 0; k < kGuideLobes; ++k) {
    float const c = (gl.a[k].x * wi.x + gl.a[k].y * wi.y) + gl.a[k].z * wi.z;
    q += gl.b[k].x * gl.b[k].y * __expf(gl.a[k].w * (c - 1.f));
  }
  return q;
}

__device__ __forceinline__ float guide_mix_pdf(guide_dev const& g, guide_lobes const& gl, rs::v3 wi, float pdf_bsdf) {
  return g.fraction * guide_pdf(gl, wi) + (1.f - g.fraction) * pdf_bsdf;
}

// Lobe by the weights' cdf, then a vMF direction (W. Jakob, "Numerically
// stable sampling of the von Mises Fisher distribution on S2", 2012).
__device__ __forceinline__ bool guide_sample(guide_lobes const& gl, float u_lobe, float u1, float u2, rs::v3& wi) {
  int k = 0;
#pragma unroll
  for (int j = 0; j < kGuideLobes - 1; ++j) k += u_lobe >= gl.b[j].z ? 1 : 0;
  float const kappa = gl.a[k].w;
  float const w = 1.f + __logf(u1 + (1.f - u1) * __expf(-2.f * kappa)) / kappa;
  float const r = sqrtf(fmaxf(0.f, 1.f - w * w));
  float s, c;
  __sincosf(6.28318530717958648f * u2, &s, &c);
  rs::v3 const mu{gl.a[k].x, gl.a[k].y, gl.a[k].z};
  float const sign = mu.z >= 0.f ? 1.f : -1.f;
  float const aa = -1.f / (sign + mu.z);
  float const bb = mu.x * mu.y * aa;
  rs::v3 const t{1.f + sign * mu.x * mu.x * aa, sign * bb, -sign * mu.x};
  rs::v3 const b{bb, sign + mu.y * mu.y * aa, -mu.y};
  wi = (t * (r * c) + b * (r * s)) + mu * w;
  return isfinite(wi.x) && isfinite(wi.y) && isfinite(wi.z);
}

// Training record of vertex v of `path`: position, pdf | shading normal,
// luminance of f cos | view direction, tag | sampled direction | throughput
// after the vertex | radiance of the path when the vertex was left (written
// by the next vertex's shade).
__device__ __forceinline__ float4* guide_record_at(guide_dev const& g, uint32_t path, int v) {
  return g.records + (size_t(v) * g.paths + path) * kRecordWords;
}

// Declared in guide.cu (host side).
int guide_prepare(myrt_ctx* ctx, size_t paths, myrt_render_params const* p, guide_dev& g);
// Training state for wave planning: waves trained so far (0 for a new network
// or a new scene) and whether this render trains.
int guide_schedule(myrt_ctx* ctx, uint64_t* waves_trained, bool* training);
void guide_begin_wave(myrt_ctx* ctx, guide_dev& g);
int guide_infer(myrt_ctx* ctx, guide_dev const& g, uint32_t WH, uint32_t sample_base, float4 const* queue,
    float4 const* hits, uint32_t const* count, cudaStream_t st);
int guide_train(myrt_ctx* ctx, guide_dev const& g, uint32_t paths, int max_depth, float4 const* radiance,
    cudaStream_t st);

}  // namespace myrt_b200
