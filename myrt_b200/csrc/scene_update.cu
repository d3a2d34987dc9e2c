// Instance updates on the device: new drawable transforms (and material
// indices) re-bake the world-space triangles and shading normals from the
// object-space geometry kept since myrt_scene_upload, then the device builder
// (bvh8_device.cu) rebuilds the tree. The reference rebuilds its TLAS on the
// host whenever an instance hash changes (src/pathtracer/scene.cpp:336-344);
// here nothing but the drawables (160 bytes each) crosses PCIe.
//
// The bake repeats the host bake of myrt_scene_upload operation for operation
// (column-major mat4 times (v, 1) with left-to-right sums, normal matrix =
// mat3(transpose(inverse_transformation)), identity transforms copied), with
// every product and sum rounded separately, so an update gives the same world
// triangles as uploading the scene again with the new drawables.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/myrt_cuda.h"
#include "bvh8_device.hpp"
#include "ctx.hpp"
#include "trace.cuh"

namespace myrt_b200 {
namespace {

struct drawable_xf {
  float m[16];   // column-major transformation
  float nm[9];   // normal matrix, column-major 3x3
  int32_t ident;
  int32_t material;
  int32_t pad[1];
};

__device__ __forceinline__ float lin3(float a, float x, float b, float y, float c, float z) {
  return __fadd_rn(__fadd_rn(__fmul_rn(a, x), __fmul_rn(b, y)), __fmul_rn(c, z));
}

__global__ void k_bake(uint4 const* __restrict__ src, float4 const* __restrict__ verts,
    float4 const* __restrict__ nrms, drawable_xf const* __restrict__ dr, size_t n, float* __restrict__ pos,
    float4* __restrict__ tri_normals, int32_t* __restrict__ mat) {
  size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  uint4 const s = src[i];
  drawable_xf const& d = dr[s.w];
  uint32_t const vi[3] = {s.x, s.y, s.z};
  for (int k = 0; k < 3; ++k) {
    float4 const v = verts[vi[k]];
    float* out = pos + 9 * i + 3 * k;
    if (d.ident) {
      out[0] = v.x, out[1] = v.y, out[2] = v.z;
    } else {
      for (int r = 0; r < 3; ++r)
        out[r] = __fadd_rn(lin3(d.m[r], v.x, d.m[4 + r], v.y, d.m[8 + r], v.z), __fmul_rn(d.m[12 + r], 1.f));
    }
    if (tri_normals) {
      float4 const nv = nrms[vi[k]];
      float n3[3];
      if (d.ident) {
        n3[0] = nv.x, n3[1] = nv.y, n3[2] = nv.z;
      } else {
        for (int r = 0; r < 3; ++r) n3[r] = lin3(d.nm[r], nv.x, d.nm[3 + r], nv.y, d.nm[6 + r], nv.z);
      }
      tri_normals[3 * i + k] = make_float4(n3[0], n3[1], n3[2], 0.f);
    }
  }
  mat[i] = d.material;
}

__device__ __forceinline__ uint32_t f2ord(float f) {
  uint32_t const u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__global__ void k_bounds(float const* __restrict__ pos, size_t n_floats, uint32_t* __restrict__ out) {
  __shared__ uint32_t s[6];
  if (threadIdx.x < 6) s[threadIdx.x] = threadIdx.x < 3 ? 0xffffffffu : 0u;
  __syncthreads();
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n_floats; i += size_t(gridDim.x) * blockDim.x) {
    uint32_t const a = uint32_t(i % 3), o = f2ord(pos[i]);
    atomicMin(&s[a], o);
    atomicMax(&s[3 + a], o);
  }
  __syncthreads();
  if (threadIdx.x < 3) atomicMin(&out[threadIdx.x], s[threadIdx.x]);
  else if (threadIdx.x < 6) atomicMax(&out[threadIdx.x], s[threadIdx.x]);
}

float ord2f(uint32_t u) {
  uint32_t const b = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
  float f;
  std::memcpy(&f, &b, 4);
  return f;
}

bool same_geometry(myrt_drawable const& a, myrt_drawable const& b) {
  return a.indices_base_index == b.indices_base_index && a.points_base_index == b.points_base_index &&
      a.index_count == b.index_count;
}

}  // namespace

int scene_set_transforms(myrt_ctx* ctx, myrt_drawable const* drawables, size_t count) {
  device_scene& s = ctx->scene;
  if (!s.valid) return set_error(ctx, MYRT_ERR_NO_SCENE, "no scene uploaded");
  if (!s.prim_src || !s.raw_vertices)
    return set_error(ctx, MYRT_ERR_UNSUPPORTED, "scene has no object-space geometry to re-bake");
  if (!drawables || count != s.drawables.size())
    return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "the drawable count must match the uploaded scene");
  for (size_t i = 0; i < count; ++i)
    if (!same_geometry(drawables[i], s.drawables[i]))
      return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT,
          "only transforms and material indices may change; upload the scene again for new geometry");
  auto const t0 = std::chrono::steady_clock::now();
  std::vector<drawable_xf> xf(count);
  for (size_t i = 0; i < count; ++i) {
    myrt_drawable const& d = drawables[i];
    drawable_xf& x = xf[i];
    std::memcpy(x.m, d.transformation, sizeof x.m);
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) x.nm[c * 3 + r] = d.inverse_transformation[r * 4 + c];
    bool ident = true;
    for (int c = 0; c < 4; ++c)
      for (int r = 0; r < 4; ++r)
        if (d.transformation[c * 4 + r] != (c == r ? 1.f : 0.f)) ident = false;
    x.ident = ident ? 1 : 0;
    x.material = d.material_index;
  }
  cudaStream_t const st = ctx->stream;
  // staging (transforms, then the bounds words) and the corners: kept in the
  // scene between moves; the corners come from the spare set when there is one
  size_t const xf_bytes = (count * sizeof(drawable_xf) + 255) & ~size_t(255);
  int rc = MYRT_OK;
  if (s.move_stage_bytes < xf_bytes + 256) {
    cudaFree(s.move_stage);
    s.move_stage = nullptr;
    s.move_stage_bytes = 0;
    rc = check_cuda(ctx, cudaMalloc(&s.move_stage, xf_bytes + 256), "move staging");
    if (rc) return rc;
    s.move_stage_bytes = xf_bytes + 256;
  }
  auto* const d_xf = static_cast<drawable_xf*>(s.move_stage);
  auto* const d_b = reinterpret_cast<uint32_t*>(static_cast<char*>(s.move_stage) + xf_bytes);
  float* d_pos = s.spare_pos;
  bool const own_pos = d_pos == nullptr;
  if (own_pos) rc = check_cuda(ctx, cudaMalloc(reinterpret_cast<void**>(&d_pos), s.n_prims * 36), "world triangles");
  auto cleanup = [&]() {
    if (own_pos) cudaFree(d_pos);
  };
  // the spare set is the tree before the previous move: work that callers
  // queued on their own streams may still read it, so wait for the device
  // before overwriting it (freeing it, as a first move does, waits the same way)
  if (!rc && !own_pos) rc = check_cuda(ctx, cudaDeviceSynchronize(), "waiting for work on the previous tree");
  if (!rc)
    rc = check_cuda(ctx, cudaMemcpyAsync(d_xf, xf.data(), count * sizeof(drawable_xf), cudaMemcpyHostToDevice, st),
        "drawables");
  uint32_t const init_b[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
  if (!rc) rc = check_cuda(ctx, cudaMemcpyAsync(d_b, init_b, sizeof init_b, cudaMemcpyHostToDevice, st), "bounds");
  if (rc) {
    cleanup();
    return rc;
  }
  k_bake<<<uint32_t((s.n_prims + 255) / 256), 256, 0, st>>>(s.prim_src, s.raw_vertices, s.raw_normals, d_xf,
      s.n_prims, d_pos, s.raw_normals ? s.tri_normals : nullptr, s.tri_material);
  k_bounds<<<std::max(1, ctx->sm_count) * 4, 256, 0, st>>>(d_pos, 9 * s.n_prims, d_b);
  uint32_t hb[6];
  rc = check_cuda(ctx, cudaMemcpyAsync(hb, d_b, sizeof hb, cudaMemcpyDeviceToHost, st), "bounds");
  if (rc) {
    cleanup();
    return rc;
  }
  device_bvh8 spare;
  spare.nodes = reinterpret_cast<bvh8_node*>(s.spare_nodes);
  spare.tris = s.spare_tris;
  spare.node_capacity = s.spare_node_capacity;
  spare.tri_capacity = s.spare_tri_capacity;
  device_bvh8 dt;
  char const* what = nullptr;
  int const e = build_bvh8_device(d_pos, s.n_prims, st, ctx->build_scratch, &spare, dt, &what);
  if (e) {
    cleanup();
    return check_cuda(ctx, cudaError_t(e > 0 ? e : cudaErrorInvalidValue), what ? what : "device BVH build");
  }
  bool const took_spare = dt.nodes == spare.nodes;
  if (dt.wide_depth > MYRT_STACK_MAX) {
    if (!took_spare) {
      cudaFree(dt.nodes);
      cudaFree(dt.tris);
    }
    cleanup();
    return set_error(ctx, MYRT_ERR_UNSUPPORTED, "BVH deeper than the traversal stack");
  }
  // the re-baked corners become the rasteriser's; the previous corners and
  // tree become the spare set (a host-built tree has no reusable capacity)
  s.spare_pos = s.world_pos;
  s.world_pos = d_pos;
  if (!took_spare) {
    cudaFree(s.spare_nodes);
    cudaFree(s.spare_tris);
  }
  if (s.node_capacity > 0) {
    s.spare_nodes = s.nodes;
    s.spare_tris = s.tris;
    s.spare_node_capacity = s.node_capacity;
    s.spare_tri_capacity = s.tri_capacity;
  } else {
    cudaFree(s.nodes);
    cudaFree(s.tris);
    s.spare_nodes = nullptr;
    s.spare_tris = nullptr;
    s.spare_node_capacity = s.spare_tri_capacity = 0;
  }
  s.nodes = reinterpret_cast<uint4*>(dt.nodes);
  s.tris = dt.tris;
  s.node_capacity = dt.node_capacity;
  s.tri_capacity = dt.tri_capacity;
  s.n_nodes = dt.n_nodes;
  s.n_tris = dt.n_tris;
  s.stats = bvh8_stats{};
  s.stats.binary_nodes = dt.binary_nodes;
  s.stats.wide_nodes = dt.n_nodes;
  s.stats.leaf_slots = dt.leaf_slots;
  s.stats.triangles = dt.n_tris;
  s.stats.wide_depth = dt.wide_depth;
  s.stats.max_leaf_size = 4;
  for (int k = 0; k < 6; ++k) s.bounds[k] = ord2f(hb[k]);
  s.drawables.assign(drawables, drawables + count);
  if (s.instanced) {  // the instance level follows the new transforms (host build, small)
    int const e = upload_top_level(ctx, s.drawables);
    if (e) return e;
  }
  s.stats.build_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  ctx->render.sample_counter = 0;  // the image restarts, as after prepare() reported a change
  return MYRT_OK;
}

}  // namespace myrt_b200

extern "C" int myrt_scene_set_transforms(myrt_ctx* ctx, myrt_drawable const* drawables, size_t count) {
  if (!ctx) return MYRT_ERR_INVALID_ARGUMENT;
  int rc = myrt_b200::check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  if (rc) return rc;
  return myrt_b200::scene_set_transforms(ctx, drawables, count);
}
