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
  size_t node_capacity = 0, tri_capacity = 0;  // allocated nodes / float4s
  int wide_depth = 0;
  double seconds = 0.0;
};

// The builder's temporary arrays (keys, radix tree, boxes, queues, sort
// temporary) in one device block that a context keeps between builds and
// grows on demand, so a rebuild allocates only its output.
struct device_build_scratch {
  void* base = nullptr;
  size_t bytes = 0;
  void release() {
    cudaFree(base);
    base = nullptr;
    bytes = 0;
  }
};

// d_pos: 9 floats per triangle (v0, v1, v2), device memory. Returns 0 or a
// CUDA error code (with *what naming the step); synchronises `st`. `reuse`
// (or null) offers output buffers: taken when both capacities suffice
// (out.nodes == reuse->nodes then), never freed by the builder; otherwise the
// output is allocated here.
int build_bvh8_device(float const* d_pos, size_t n_tris, cudaStream_t st, device_build_scratch& scratch,
    device_bvh8 const* reuse, device_bvh8& out, char const** what);

}  // namespace myrt_b200
