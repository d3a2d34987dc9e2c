// Ray ordering for the closest-hit / any-hit queries: rays are visited in
// the order of a 24-bit key, the Morton code of the origin's cell in a 16^3
// grid over the scene box followed by the Morton code of the direction's cell
// in a 16^3 grid over [-1, 1]^3. Neighbouring lanes of a warp then walk
// similar paths through the tree (fewer divergent branches, node and triangle
// loads shared through L1). The order is a permutation of ray indices from a
// stable radix sort, so equal keys keep their input order (image rows of
// camera rays stay together); every result is still written at its ray's own
// index, so the order never changes any answer.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace myrt_b200 {

constexpr int kOrderKeyBits = 24;

// Spreads the low 4 bits of v to bits 0, 3, 6, 9.
__device__ __forceinline__ uint32_t spread4(uint32_t v) {
  v &= 15u;
  return (v & 1u) | ((v & 2u) << 2) | ((v & 4u) << 4) | ((v & 8u) << 6);
}
__device__ __forceinline__ uint32_t cell4(float x) {  // x in [0, 16) -> 0..15, clamped (NaN -> 0)
  return x >= 15.f ? 15u : (x > 0.f ? uint32_t(x) : 0u);
}

// The key of a ray with origin o and direction d (any length); lo and
// cell_scale map the scene box onto [0, 16)^3.
__device__ __forceinline__ uint32_t ray_key(float4 o, float4 d, float3 lo, float3 cell_scale) {
  uint32_t const ox = cell4((o.x - lo.x) * cell_scale.x);
  uint32_t const oy = cell4((o.y - lo.y) * cell_scale.y);
  uint32_t const oz = cell4((o.z - lo.z) * cell_scale.z);
  float const l2 = d.x * d.x + d.y * d.y + d.z * d.z;
  float const s = l2 > 0.f ? 8.f * rsqrtf(l2) : 0.f;  // unit direction in [-1, 1] -> [0, 16)
  uint32_t const dx = cell4(fmaf(d.x, s, 8.f)), dy = cell4(fmaf(d.y, s, 8.f)), dz = cell4(fmaf(d.z, s, 8.f));
  uint32_t const om = spread4(ox) | (spread4(oy) << 1) | (spread4(oz) << 2);
  uint32_t const dm = spread4(dx) | (spread4(dy) << 1) | (spread4(dz) << 2);
  return (om << 12) | dm;
}

// keys[i], vals[i] = i for rays given as (o, tmin), (d, tmax) float4 pairs.
static __global__ void __launch_bounds__(256) k_ray_keys(float4 const* __restrict__ rays, uint32_t n, float3 lo,
    float3 cell_scale, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  uint32_t const i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  keys[i] = ray_key(__ldg(rays + 2 * size_t(i)), __ldg(rays + 2 * size_t(i) + 1), lo, cell_scale);
  vals[i] = i;
}

// The scene box [b[0..2], b[3..5]] -> lo and cell_scale of ray_key.
inline void ray_key_grid(float const* b, float3& lo, float3& cell_scale) {
  float* plo = &lo.x;
  float* psc = &cell_scale.x;
  for (int k = 0; k < 3; ++k) {
    float const ext = b[3 + k] - b[k];
    plo[k] = b[k] - 1e-3f * ext;
    psc[k] = ext > 0.f ? 16.f / (ext * 1.002f) : 0.f;
  }
}

}  // namespace myrt_b200
