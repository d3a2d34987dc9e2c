// Device BVH build (bvh8_device.cu): the 8-wide node format of bvh8.hpp built
// on the GPU from world-space triangles already in device memory.
#pragma once
#include <cstddef>
#include <cuda_runtime.h>

#include "bvh8.hpp"

namespace myrt_b200 {

struct device_bvh8 {
  bvh8_node* nodes = nullptr;  // cudaMalloc'd, owned by the caller afterwards
  float4* tris = nullptr;      // 3 float4 per triangle (v0 | prim id bits, v1, v2), leaf order
  size_t n_nodes = 0, n_tris = 0, binary_nodes = 0, leaf_slots = 0;
  int wide_depth = 0;
  double seconds = 0.0;
};

// d_pos: 9 floats per triangle (v0, v1, v2), device memory. Returns 0 or a
// CUDA error code (with *what naming the step); synchronises `st`.
int build_bvh8_device(float const* d_pos, size_t n_tris, cudaStream_t st, device_bvh8& out, char const** what);

}  // namespace myrt_b200
