// C ABI: context, scene upload and ray queries (include/myrt_cuda.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include <cub/device/device_radix_sort.cuh>

#include "../../include/myrt_cuda.h"
#include "bvh8.hpp"
#include "bvh8_device.hpp"
#include "ctx.hpp"
#include "rayorder.cuh"
#include "sdf_skip.hpp"
#include "trace.cuh"

namespace myrt_b200 {

int set_error(myrt_ctx* ctx, int code, std::string msg) {
  if (ctx) ctx->last_error = std::move(msg);
  return code;
}

int check_cuda(myrt_ctx* ctx, cudaError_t e, char const* what) {
  if (e == cudaSuccess) return MYRT_OK;
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  return set_error(ctx, e == cudaErrorMemoryAllocation ? MYRT_ERR_OUT_OF_MEMORY : MYRT_ERR_CUDA, m);
}

namespace {

void free_scene(device_scene& s) {
  cudaFree(s.raw_vertices);
  cudaFree(s.raw_normals);
  cudaFree(s.prim_src);
  cudaFree(s.world_pos);
  cudaFree(s.nodes);
  cudaFree(s.tris);
  cudaFree(s.tri_normals);
  cudaFree(s.tri_uvs);
  cudaFree(s.tri_material);
  cudaFree(s.materials);
  cudaFree(s.material_data);
  cudaFree(s.spare_nodes);
  cudaFree(s.spare_tris);
  cudaFree(s.spare_pos);
  cudaFree(s.move_stage);
  cudaFree(s.blas_nodes);
  cudaFree(s.blas_tris);
  cudaFree(s.tlas_nodes);
  cudaFree(s.inst_records);
  s = device_scene{};
}

bool is_identity(float const* m) {
  for (int c = 0; c < 4; ++c)
    for (int r = 0; r < 4; ++r)
      if (m[c * 4 + r] != (c == r ? 1.f : 0.f)) return false;
  return true;
}

// column-major mat4 * (x, y, z, w), left-to-right sums
void xform(float const* m, float const* v, float w, float* out) {
  for (int r = 0; r < 3; ++r) out[r] = ((m[r] * v[0] + m[4 + r] * v[1]) + m[8 + r] * v[2]) + m[12 + r] * w;
}

template <typename T> int upload(myrt_ctx* ctx, T** dst, T const* src, size_t count, char const* what) {
  if (count == 0) return MYRT_OK;
  int rc = check_cuda(ctx, cudaMalloc(reinterpret_cast<void**>(dst), count * sizeof(T)), what);
  if (rc) return rc;
  return check_cuda(ctx, cudaMemcpyAsync(*dst, src, count * sizeof(T), cudaMemcpyHostToDevice, ctx->stream), what);
}

int ensure_stage(myrt_ctx* ctx, size_t bytes) {
  if (ctx->stage_bytes >= bytes) return MYRT_OK;
  for (auto& p : ctx->stage) {
    cudaFree(p);
    p = nullptr;
  }
  ctx->stage_bytes = 0;
  for (auto& p : ctx->stage) {
    int rc = check_cuda(ctx, cudaMalloc(&p, bytes), "staging buffer");
    if (rc) return rc;
  }
  ctx->stage_bytes = bytes;
  return MYRT_OK;
}

constexpr uint32_t kChunkRays = 1u << 20;

constexpr uint32_t kCounterRing = 64;

template <int ISECT, bool ANY, bool STATS>
int launch_persistent(myrt_ctx* ctx, trace_args const& a, cudaStream_t s) {
  static int occ = 0;  // resident blocks per SM at 128 threads (per instantiation)
  if (!occ) {
    int rc = check_cuda(ctx,
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_trace_persistent<ISECT, ANY, STATS>, 128, 0),
        "occupancy query");
    if (rc) return rc;
    if (occ < 1) occ = 1;
  }
  uint32_t const bps = ctx->tuning.blocks_per_sm ? ctx->tuning.blocks_per_sm : uint32_t(occ);
  uint32_t grid = uint32_t(ctx->sm_count) * bps;
  grid = std::max(1u, std::min(grid, (a.n + 127) / 128));
  uint32_t* counter = ctx->d_next + (ctx->next_slot++ % kCounterRing);
  int rc = check_cuda(ctx, cudaMemsetAsync(counter, 0, sizeof(uint32_t), s), "ray counter");
  if (rc) return rc;
  uint32_t const refill = std::max(1u, std::min(32u, ctx->tuning.refill));
  k_trace_persistent<ISECT, ANY, STATS><<<grid, 128, 0, s>>>(a, counter, refill);
  return MYRT_OK;
}

constexpr uint32_t kOrderMin = 1u << 20;  // batches from this size on are sorted (trace_order 0)

void free_order(myrt_ctx::order_scratch& o) {
  for (int k = 0; k < 2; ++k) {
    cudaFree(o.keys[k]);
    cudaFree(o.vals[k]);
    o.keys[k] = o.vals[k] = nullptr;
  }
  cudaFree(o.temp);
  o.temp = nullptr;
  o.cap = o.temp_bytes = 0;
}

// Sorts the batch's ray indices by origin / direction cell (rayorder.cuh) into
// the lane's scratch and points a.perm at the order. The scratch of a lane is
// reused by later queries on any stream: each use waits for the previous one.
int order_rays(myrt_ctx* ctx, trace_args& a, int lane, cudaStream_t s) {
  auto& o = ctx->order[lane];
  if (!o.done) {
    int rc = check_cuda(ctx, cudaEventCreateWithFlags(&o.done, cudaEventDisableTiming), "ray order event");
    if (rc) return rc;
  }
  int rc = check_cuda(ctx, cudaStreamWaitEvent(s, o.done, 0), "ray order wait");
  if (rc) return rc;
  size_t need = 0;
  rc = check_cuda(ctx, cub::DeviceRadixSort::SortPairs(nullptr, need, o.keys[0], o.keys[1], o.vals[0], o.vals[1],
                           int(a.n), 0, kOrderKeyBits, s), "ray order size");
  if (rc) return rc;
  if (o.cap < a.n || o.temp_bytes < need) {
    rc = check_cuda(ctx, cudaStreamSynchronize(s), "ray order realloc");
    if (rc) return rc;
    free_order(o);
    size_t const cap = std::max<size_t>(a.n, o.cap);
    for (int k = 0; k < 2 && !rc; ++k) {
      rc = check_cuda(ctx, cudaMalloc(reinterpret_cast<void**>(&o.keys[k]), cap * 4), "ray order keys");
      if (!rc) rc = check_cuda(ctx, cudaMalloc(reinterpret_cast<void**>(&o.vals[k]), cap * 4), "ray order indices");
    }
    if (!rc) rc = check_cuda(ctx, cudaMalloc(&o.temp, need), "ray order temporary");
    if (rc) {
      free_order(o);
      return rc;
    }
    o.cap = cap;
    o.temp_bytes = need;
  }
  float3 lo, sc;
  ray_key_grid(ctx->scene.bounds, lo, sc);
  k_ray_keys<<<(a.n + 255) / 256, 256, 0, s>>>(a.rays, a.n, lo, sc, o.keys[0], o.vals[0]);
  rc = check_cuda(ctx, cudaGetLastError(), "ray key launch");
  if (rc) return rc;
  size_t tb = o.temp_bytes;
  rc = check_cuda(ctx, cub::DeviceRadixSort::SortPairs(o.temp, tb, o.keys[0], o.keys[1], o.vals[0], o.vals[1],
                           int(a.n), 0, kOrderKeyBits, s), "ray order sort");
  if (rc) return rc;
  a.perm = o.vals[1];
  return MYRT_OK;
}

int launch_trace_kernels(myrt_ctx* ctx, trace_args a, int intersector, bool any, bool stats, cudaStream_t s);

// lane: the ray-order scratch to use (0 = the context's stream, 1 = its
// second lane). host_chunk: a chunk of a host-memory query, sorted only when
// trace_order forces it.
int launch_trace(myrt_ctx* ctx, trace_args a, int intersector, bool any, bool stats, cudaStream_t s, int lane = 0,
    bool host_chunk = false) {
  if (a.n == 0) return MYRT_OK;
  uint32_t const mode = ctx->tuning.trace_order;
  bool const sorted = mode == 2 || (mode == 0 && !host_chunk && a.n >= kOrderMin);
  std::array<cudaEvent_t, 3> ev{};
  if (ctx->time_phases) {
    if (ctx->phase_pool.empty()) {
      for (auto& e : ev) {
        int rc = check_cuda(ctx, cudaEventCreate(&e), "phase timing event");
        if (rc) return rc;
      }
    } else {
      ev = ctx->phase_pool.back();
      ctx->phase_pool.pop_back();
    }
    cudaEventRecord(ev[0], s);
  }
  int rc = sorted ? order_rays(ctx, a, lane, s) : MYRT_OK;
  if (ctx->time_phases) cudaEventRecord(ev[1], s);
  if (!rc) rc = launch_trace_kernels(ctx, a, intersector, any, stats, s);
  if (ctx->time_phases) {
    cudaEventRecord(ev[2], s);
    ctx->phase_pending.push_back(ev);
  }
  if (!rc && sorted) rc = check_cuda(ctx, cudaEventRecord(ctx->order[lane].done, s), "ray order record");
  return rc;
}

int launch_trace_kernels(myrt_ctx* ctx, trace_args a, int intersector, bool any, bool stats, cudaStream_t s) {
  dim3 const block(128);
  dim3 const grid((a.n + 127) / 128);
  if (ctx->tuning.instancing) {
    a.nodes = ctx->scene.tlas_nodes;
    auto go_inst = [&](auto flat_tag) {
      constexpr bool FL = decltype(flat_tag)::value;
      if (intersector == MYRT_ISECT_REFERENCE) {
        if (stats) k_trace_inst<0, false, true, FL><<<grid, block, 0, s>>>(a);
        else if (any) k_trace_inst<0, true, false, FL><<<grid, block, 0, s>>>(a);
        else k_trace_inst<0, false, false, FL><<<grid, block, 0, s>>>(a);
      } else {
        if (stats) k_trace_inst<1, false, true, FL><<<grid, block, 0, s>>>(a);
        else if (any) k_trace_inst<1, true, false, FL><<<grid, block, 0, s>>>(a);
        else k_trace_inst<1, false, false, FL><<<grid, block, 0, s>>>(a);
      }
    };
    if (ctx->tuning.instancing == 2) go_inst(std::false_type{});
    else go_inst(std::true_type{});
    return check_cuda(ctx, cudaGetLastError(), "instanced trace launch");
  }
  if (ctx->tuning.trace_persistent) {
    int rc;
    if (intersector == MYRT_ISECT_REFERENCE) {
      if (any) rc = launch_persistent<0, true, false>(ctx, a, s);
      else if (stats) rc = launch_persistent<0, false, true>(ctx, a, s);
      else rc = launch_persistent<0, false, false>(ctx, a, s);
    } else {
      if (any) rc = launch_persistent<1, true, false>(ctx, a, s);
      else if (stats) rc = launch_persistent<1, false, true>(ctx, a, s);
      else rc = launch_persistent<1, false, false>(ctx, a, s);
    }
    if (rc) return rc;
    return check_cuda(ctx, cudaGetLastError(), "trace launch");
  }
  if (ctx->tuning.trace_smem_stack && !ctx->tuning.trace_unit_steps) {
    a.stack_cap = std::max(1, std::min(ctx->scene.stats.wide_depth + 1, MYRT_STACK_MAX));
    size_t const smem = size_t(a.stack_cap) * 128 * sizeof(uint2);
    auto go_smem = [&](auto kern) -> int {
      int rc = check_cuda(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
          "trace shared stack");
      if (rc) return rc;
      kern<<<grid, block, smem, s>>>(a);
      return MYRT_OK;
    };
    int rc;
    if (intersector == MYRT_ISECT_REFERENCE)
      rc = stats ? go_smem(k_trace_smem<0, false, true>) : any ? go_smem(k_trace_smem<0, true, false>)
                                                               : go_smem(k_trace_smem<0, false, false>);
    else
      rc = stats ? go_smem(k_trace_smem<1, false, true>) : any ? go_smem(k_trace_smem<1, true, false>)
                                                               : go_smem(k_trace_smem<1, false, false>);
    if (rc) return rc;
    return check_cuda(ctx, cudaGetLastError(), "trace launch");
  }
  // default: the 10-blocks register cap (48 registers, a few bytes of spills),
  // measured 1 % faster than 8 blocks (64 registers) on 27.9 M-ray batches
  uint32_t const mb = ctx->tuning.trace_min_blocks ? ctx->tuning.trace_min_blocks : 10u;
  bool const unit = ctx->tuning.trace_unit_steps != 0;
  auto go = [&](auto isect_tag) {
    constexpr int IS = decltype(isect_tag)::value;
    if (unit) {
      if (stats) k_trace<IS, false, true, 8, true><<<grid, block, 0, s>>>(a);
      else if (any) k_trace<IS, true, false, 8, true><<<grid, block, 0, s>>>(a);
      else k_trace<IS, false, false, 8, true><<<grid, block, 0, s>>>(a);
    } else if (stats) k_trace<IS, false, true><<<grid, block, 0, s>>>(a);
    else if (any) {
      if (mb >= 12) k_trace<IS, true, false, 12><<<grid, block, 0, s>>>(a);
      else if (mb >= 10) k_trace<IS, true, false, 10><<<grid, block, 0, s>>>(a);
      else k_trace<IS, true, false><<<grid, block, 0, s>>>(a);
    } else {
      if (mb >= 12) k_trace<IS, false, false, 12><<<grid, block, 0, s>>>(a);
      else if (mb >= 10) k_trace<IS, false, false, 10><<<grid, block, 0, s>>>(a);
      else k_trace<IS, false, false><<<grid, block, 0, s>>>(a);
    }
  };
  if (intersector == MYRT_ISECT_REFERENCE) go(std::integral_constant<int, 0>{});
  else go(std::integral_constant<int, 1>{});
  return check_cuda(ctx, cudaGetLastError(), "trace launch");
}

int validate_query(myrt_ctx* ctx, void const* rays, void const* out, int intersector) {
  if (!ctx) return MYRT_ERR_INVALID_ARGUMENT;
  if (!ctx->scene.valid) return set_error(ctx, MYRT_ERR_NO_SCENE, "no scene uploaded");
  if (!rays || !out) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "null ray or output pointer");
  if (intersector != MYRT_ISECT_REFERENCE && intersector != MYRT_ISECT_WATERTIGHT)
    return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "unknown intersector");
  if (ctx->tuning.instancing && !ctx->scene.instanced)
    return set_error(ctx, MYRT_ERR_UNSUPPORTED, "instancing = 1 needs a scene uploaded with instancing = 1");
  return MYRT_OK;
}

trace_args base_args(myrt_ctx* ctx) {
  trace_args a{};
  a.nodes = ctx->scene.nodes;
  a.tris = ctx->scene.tris;
  a.err = ctx->d_err;
  a.blas_nodes = ctx->scene.blas_nodes;
  a.blas_tris = ctx->scene.blas_tris;
  a.inst = ctx->scene.inst_records;
  return a;
}

// Host-memory query: chunks go round four streams, each running its chunks'
// upload, traversal and download in order, so the host-to-device copy engine
// always has the next chunk's upload queued while earlier chunks trace and
// download (with two streams it idled while a stream's download finished).
// Chunks are an eighth of the query (at least 64 Ki rays, at most kChunkRays),
// so that a query of 1 Mi rays pipelines too instead of running as one chunk.
int host_query(myrt_ctx* ctx, myrt_ray const* rays, uint32_t n, void* out, size_t out_stride, int intersector,
    bool any) {
  size_t const chunk_bytes = size_t(kChunkRays) * (sizeof(myrt_ray) + sizeof(myrt_hit));
  int rc = ensure_stage(ctx, chunk_bytes);
  if (rc) return rc;
  uint32_t const chunk = std::min<uint32_t>(kChunkRays, std::max<uint32_t>(1u << 16, ((n / 8) + 4095u) & ~4095u));
  cudaStream_t lanes[4] = {ctx->stream, ctx->aux_stream, ctx->copy_lanes[0], ctx->copy_lanes[1]};
  for (uint32_t c0 = 0, k = 0; c0 < n; c0 += chunk, ++k) {
    uint32_t const cn = std::min(chunk, n - c0);
    cudaStream_t const s = lanes[k & 3];
    char* base = static_cast<char*>(ctx->stage[k & 3]);
    auto* d_rays = reinterpret_cast<float4*>(base);
    char* d_out = base + size_t(kChunkRays) * sizeof(myrt_ray);
    rc = check_cuda(ctx, cudaMemcpyAsync(d_rays, rays + c0, size_t(cn) * sizeof(myrt_ray), cudaMemcpyHostToDevice, s),
        "ray upload");
    if (rc) return rc;
    trace_args a = base_args(ctx);
    a.rays = d_rays;
    a.n = cn;
    if (any) a.occluded = reinterpret_cast<uint8_t*>(d_out);
    else a.hits = reinterpret_cast<float4*>(d_out);
    // chunks stream through the copy engines, which bound this path: they are
    // traced in input order unless sorting is forced (trace_order 2)
    rc = launch_trace(ctx, a, intersector, any, false, s, int(k & 3), true);
    if (rc) return rc;
    rc = check_cuda(ctx,
        cudaMemcpyAsync(static_cast<char*>(out) + size_t(c0) * out_stride, d_out, size_t(cn) * out_stride,
            cudaMemcpyDeviceToHost, s),
        "result download");
    if (rc) return rc;
  }
  for (int l = 1; l < 4 && !rc; ++l) rc = check_cuda(ctx, cudaStreamSynchronize(lanes[l]), "sync");
  if (rc) return rc;
  return myrt_sync(ctx);
}

}  // namespace
}  // namespace myrt_b200

using namespace myrt_b200;

struct myrt_bvh8_host {
  myrt_b200::bvh8 tree;
};

namespace {
void fill_info(myrt_b200::bvh8_stats const& st, size_t n_nodes, size_t n_tris, myrt_bvh_info* info) {
  *info = myrt_bvh_info{};
  info->triangles = st.triangles;
  info->binary_nodes = st.binary_nodes;
  info->wide_nodes = st.wide_nodes;
  info->leaf_slots = st.leaf_slots;
  info->binary_depth = st.binary_depth;
  info->wide_depth = st.wide_depth;
  info->max_leaf_size = st.max_leaf_size;
  info->build_seconds = st.build_seconds;
  info->node_bytes = n_nodes * sizeof(myrt_b200::bvh8_node);
  info->triangle_bytes = n_tris * sizeof(myrt_b200::bvh8_triangle);
}
}  // namespace

extern "C" {

int myrt_bvh8_build(float const* positions, size_t n_tris, myrt_bvh8_host** out) {
  if (!out || (!positions && n_tris)) return MYRT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  auto* h = new (std::nothrow) myrt_bvh8_host;
  if (!h) return MYRT_ERR_OUT_OF_MEMORY;
  try {
    h->tree = build_bvh8(positions, n_tris, nullptr, bvh8_build_options{});
  } catch (...) {
    delete h;
    return MYRT_ERR_INVALID_ARGUMENT;
  }
  *out = h;
  return MYRT_OK;
}

int myrt_bvh8_get_info(myrt_bvh8_host const* h, myrt_bvh_info* info) {
  if (!h || !info) return MYRT_ERR_INVALID_ARGUMENT;
  fill_info(h->tree.stats, h->tree.nodes.size(), h->tree.triangles.size(), info);
  return MYRT_OK;
}

int myrt_bvh8_copy(myrt_bvh8_host const* h, void* nodes, void* triangles) {
  if (!h) return MYRT_ERR_INVALID_ARGUMENT;
  if (nodes) std::memcpy(nodes, h->tree.nodes.data(), h->tree.nodes.size() * sizeof(bvh8_node));
  if (triangles) std::memcpy(triangles, h->tree.triangles.data(), h->tree.triangles.size() * sizeof(bvh8_triangle));
  return MYRT_OK;
}

int myrt_bvh8_free(myrt_bvh8_host* h) {
  delete h;
  return MYRT_OK;
}

int myrt_ctx_create(myrt_device_opts const* opts, myrt_ctx** out) {
  if (!out) return MYRT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  auto* ctx = new (std::nothrow) myrt_ctx;
  if (!ctx) return MYRT_ERR_OUT_OF_MEMORY;
  ctx->device = opts ? opts->device : 0;
  int rc = check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  if (!rc) rc = check_cuda(ctx, cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "stream");
  if (!rc) rc = check_cuda(ctx, cudaStreamCreateWithFlags(&ctx->aux_stream, cudaStreamNonBlocking), "stream");
  for (auto& cs : ctx->copy_lanes)
    if (!rc) rc = check_cuda(ctx, cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "stream");
  if (!rc) rc = check_cuda(ctx, cudaEventCreateWithFlags(&ctx->order_event, cudaEventDisableTiming), "event");
  if (!rc) rc = check_cuda(ctx, cudaMalloc(&ctx->d_err, sizeof(uint32_t)), "error word");
  if (!rc) rc = check_cuda(ctx, cudaMemset(ctx->d_err, 0, sizeof(uint32_t)), "error word");
  if (!rc) rc = check_cuda(ctx, cudaMalloc(&ctx->d_next, kCounterRing * sizeof(uint32_t)), "ray counters");
  if (!rc)
    rc = check_cuda(ctx, cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, ctx->device),
        "SM count");
  if (rc) {
    myrt_ctx_destroy(ctx);
    return rc;
  }
  *out = ctx;
  return MYRT_OK;
}

int myrt_ctx_destroy(myrt_ctx* ctx) {
  if (!ctx) return MYRT_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->aux_stream) cudaStreamSynchronize(ctx->aux_stream);
  for (auto cs : ctx->copy_lanes)
    if (cs) cudaStreamSynchronize(cs);
  free_scene(ctx->scene);
  ctx->build_scratch.release();
  cudaFree(ctx->sdf.instrs);
  cudaFree(ctx->sdf.programs);
  cudaFree(ctx->sdf.params);
  cudaFree(ctx->sdf.drawables);
  cudaFree(ctx->sdf.skip_sphere);
  cudaFree(ctx->sdf.skip_next);
  cudaFree(ctx->sdf.cell_hdr);
  cudaFree(ctx->sdf.cell_start);
  cudaFree(ctx->sdf.cell_list);
  cudaFree(ctx->sdf.op_count);
  free_render(ctx->render);
  free_textures(ctx);
  free_forward(ctx);
  free_physical(ctx->physical);
  free_guide(ctx->guide);
  ctx->guide = nullptr;
  for (auto& p : ctx->stage) cudaFree(p);
  for (auto& o : ctx->order) {
    free_order(o);
    if (o.done) cudaEventDestroy(o.done);
  }
  for (auto* list : {&ctx->phase_pending, &ctx->phase_pool})
    for (auto& ev : *list)
      for (auto e : ev) cudaEventDestroy(e);
  cudaFree(ctx->d_err);
  cudaFree(ctx->d_next);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  if (ctx->aux_stream) cudaStreamDestroy(ctx->aux_stream);
  for (auto cs : ctx->copy_lanes)
    if (cs) cudaStreamDestroy(cs);
  if (ctx->order_event) cudaEventDestroy(ctx->order_event);
  delete ctx;
  return MYRT_OK;
}

int myrt_get_last_error(myrt_ctx* ctx, char* buf, size_t size) {
  if (!ctx || !buf || size == 0) return MYRT_ERR_INVALID_ARGUMENT;
  std::snprintf(buf, size, "%s", ctx->last_error.c_str());
  return MYRT_OK;
}

int myrt_set_tuning(myrt_ctx* ctx, myrt_tuning const* t) {
  if (!ctx || !t) return MYRT_ERR_INVALID_ARGUMENT;
  if (t->trace_persistent > 1 || t->refill < 1 || t->refill > 32 || t->blocks_per_sm > 64 || t->trace_min_blocks > 16 ||
      t->trace_unit_steps > 1 || (t->wave_paths != 0 && (t->wave_paths < 1024 || t->wave_paths > (1u << 28))) ||
      t->pt_blocks_per_sm > 16 || t->trace_smem_stack > 1 || t->trace_order > 2 || t->bvh_builder > 1 || t->sdf_cells > 128 ||
      t->guide_stall_test > 1 || t->instancing > 2 || t->pt_grid > 2 || t->ref_frames > 64)
    return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "tuning out of range");
  ctx->tuning = *t;
  return MYRT_OK;
}

int myrt_set_phase_timing(myrt_ctx* ctx, int enable) {
  if (!ctx) return MYRT_ERR_INVALID_ARGUMENT;
  ctx->time_phases = enable != 0;
  return MYRT_OK;
}

int myrt_get_phase_times(myrt_ctx* ctx, double* order_ms, double* traverse_ms, uint64_t* queries) {
  if (!ctx || !order_ms || !traverse_ms || !queries) return MYRT_ERR_INVALID_ARGUMENT;
  double o = 0.0, t = 0.0;
  int rc = MYRT_OK;
  for (auto& ev : ctx->phase_pending) {
    if (!rc) rc = check_cuda(ctx, cudaEventSynchronize(ev[2]), "phase timing");
    float a = 0.f, b = 0.f;
    if (!rc) rc = check_cuda(ctx, cudaEventElapsedTime(&a, ev[0], ev[1]), "phase timing");
    if (!rc) rc = check_cuda(ctx, cudaEventElapsedTime(&b, ev[1], ev[2]), "phase timing");
    o += a;
    t += b;
  }
  *queries = ctx->phase_pending.size();
  for (auto& ev : ctx->phase_pending) ctx->phase_pool.push_back(ev);
  ctx->phase_pending.clear();
  *order_ms = o;
  *traverse_ms = t;
  return rc;
}

int myrt_get_tuning(myrt_ctx* ctx, myrt_tuning* t) {
  if (!ctx || !t) return MYRT_ERR_INVALID_ARGUMENT;
  *t = ctx->tuning;
  return MYRT_OK;
}

int myrt_get_stream(myrt_ctx* ctx, void** stream) {
  if (!ctx || !stream) return MYRT_ERR_INVALID_ARGUMENT;
  *stream = ctx->stream;
  return MYRT_OK;
}

}  // extern "C"

namespace myrt_b200 {
// Uploads the tree over the drawables' world boxes and its instance records
// (rebuilt whenever transforms change).
int upload_top_level(myrt_ctx* ctx, std::vector<myrt_drawable> const& drawables) {
  device_scene& s = ctx->scene;
  two_level objects;
  objects.geometries = s.geometries;
  objects.drawable_geometry = s.drawable_geometry;
  objects.prim_base = s.drawable_prim_base;
  top_level top;
  try {
    top = build_top_level(objects, drawables.data(), drawables.size());
  } catch (std::exception const& e) {
    return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, std::string("instance tree build: ") + e.what());
  }
  if (top.nodes.empty()) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "instancing: no drawable has triangles");
  if (std::max(top.depth + s.blas_depth + kInstanceSave, 2 * top.depth + s.blas_depth + kInstanceRay) > MYRT_STACK_MAX)
    return set_error(ctx, MYRT_ERR_UNSUPPORTED, "instance tree + object tree deeper than the traversal stack");
  cudaFree(s.tlas_nodes);
  cudaFree(s.inst_records);
  s.tlas_nodes = nullptr;
  s.inst_records = nullptr;
  int rc = upload(ctx, reinterpret_cast<bvh8_node**>(&s.tlas_nodes), top.nodes.data(), top.nodes.size(),
      "instance tree upload");
  if (!rc)
    rc = upload(ctx, reinterpret_cast<instance_record**>(&s.inst_records), top.records.data(), top.records.size(),
        "instance record upload");
  s.n_tlas_nodes = top.nodes.size();
  s.n_inst_records = top.records.size();
  s.tlas_depth = top.depth;
  return rc;
}

// Object-space trees of the distinct geometries, then the instance level.
int upload_two_level(myrt_ctx* ctx, myrt_scene_view const* v, std::vector<myrt_drawable> const& drawables) {
  device_scene& s = ctx->scene;
  two_level objects;
  std::string err;
  if (!build_object_trees(v->vertices, v->vertex_count, v->indices, v->index_count, drawables.data(),
          drawables.size(), objects, err))
    return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, err);
  s.geometries = objects.geometries;
  s.drawable_geometry = objects.drawable_geometry;
  s.drawable_prim_base = objects.prim_base;
  s.blas_depth = objects.blas_depth;
  int rc = upload(ctx, reinterpret_cast<bvh8_node**>(&s.blas_nodes), objects.blas_nodes.data(),
      objects.blas_nodes.size(), "object tree upload");
  if (!rc)
    rc = upload(ctx, reinterpret_cast<bvh8_triangle**>(&s.blas_tris), objects.blas_tris.data(),
        objects.blas_tris.size(), "object triangle upload");
  s.n_blas_nodes = objects.blas_nodes.size();
  s.n_blas_tris = objects.blas_tris.size();
  if (!rc) rc = upload_top_level(ctx, drawables);
  if (!rc) s.instanced = true;
  return rc;
}
}  // namespace myrt_b200

extern "C" {

int myrt_scene_upload(myrt_ctx* ctx, myrt_scene_view const* v) {
  if (!ctx || !v) return MYRT_ERR_INVALID_ARGUMENT;
  if (!v->indices || !v->vertices || v->index_count == 0 || v->vertex_count == 0 || v->index_count % 3 != 0)
    return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "scene needs a non-empty index buffer (multiple of 3) and vertices");
  int rc = check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  if (rc) return rc;
  cudaStreamSynchronize(ctx->stream);
  free_scene(ctx->scene);

  std::vector<myrt_drawable> drawables;
  if (v->drawable_count == 0) {
    myrt_drawable d{};
    for (int k = 0; k < 4; ++k) d.transformation[k * 5] = d.inverse_transformation[k * 5] = 1.f;
    d.index_count = uint32_t(v->index_count);
    drawables.push_back(d);
  } else {
    if (!v->drawables) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "drawable_count > 0 but drawables is null");
    drawables.assign(v->drawables, v->drawables + v->drawable_count);
  }
  size_t n_prims = 0;
  for (auto const& d : drawables) {
    if (d.index_count % 3 != 0 || size_t(d.indices_base_index) + d.index_count > v->index_count)
      return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "drawable index range outside the index buffer");
    n_prims += d.index_count / 3;
  }
  if (n_prims >= (size_t(1) << 31)) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "too many triangles");

  std::vector<float> pos(9 * n_prims);
  std::vector<uint4> src(n_prims);
  std::vector<float4> nrm(v->normals ? 3 * n_prims : 0);
  std::vector<float2> uvs(v->uvs ? 3 * n_prims : 0);
  std::vector<int32_t> mat(n_prims);
  size_t p = 0;
  for (size_t di = 0; di < drawables.size(); ++di) {
    myrt_drawable const& d = drawables[di];
    bool const ident = is_identity(d.transformation);
    // normal matrix = mat3(transpose(inverse_transformation)) (pt_trace.comp:372)
    float nm[9];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) nm[c * 3 + r] = d.inverse_transformation[r * 4 + c];
    for (uint32_t t = 0; t < d.index_count / 3; ++t, ++p) {
      mat[p] = d.material_index;
      src[p].w = uint32_t(di);
      for (int k = 0; k < 3; ++k) {
        size_t const vi = size_t(d.points_base_index) + v->indices[d.indices_base_index + 3 * t + k];
        if (vi >= v->vertex_count) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "vertex index out of range");
        (&src[p].x)[k] = uint32_t(vi);
        float const* src = v->vertices + 4 * vi;
        float* dst = &pos[9 * p + 3 * k];
        if (ident) std::memcpy(dst, src, 12);
        else xform(d.transformation, src, 1.f, dst);
        if (v->normals) {
          float const* ns = v->normals + 4 * vi;
          float n3[3];
          if (ident) std::memcpy(n3, ns, 12);
          else
            for (int r = 0; r < 3; ++r) n3[r] = (nm[r] * ns[0] + nm[3 + r] * ns[1]) + nm[6 + r] * ns[2];
          nrm[3 * p + k] = make_float4(n3[0], n3[1], n3[2], 0.f);
        }
        if (v->uvs) uvs[3 * p + k] = make_float2(v->uvs[2 * vi], v->uvs[2 * vi + 1]);
      }
    }
  }

  bool const on_device = ctx->tuning.bvh_builder == 1;
  bvh8 tree;
  device_bvh8 dtree;
  if (on_device) {
    float* d_pos = nullptr;
    rc = upload(ctx, &d_pos, pos.data(), pos.size(), "triangle upload");
    if (rc) return rc;
    char const* what = nullptr;
    int const e = build_bvh8_device(d_pos, n_prims, ctx->stream, ctx->build_scratch, nullptr, dtree, &what);
    ctx->scene.world_pos = d_pos;
    if (e) return check_cuda(ctx, cudaError_t(e > 0 ? e : cudaErrorInvalidValue), what ? what : "device BVH build");
    if (dtree.wide_depth > MYRT_STACK_MAX) {
      cudaFree(dtree.nodes);
      cudaFree(dtree.tris);
      return set_error(ctx, MYRT_ERR_UNSUPPORTED, "BVH deeper than the traversal stack");
    }
  } else {
    try {
      tree = build_bvh8(pos.data(), n_prims, nullptr, bvh8_build_options{});
    } catch (std::exception const& e) {
      return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, std::string("bvh build: ") + e.what());
    }
    if (tree.stats.wide_depth > MYRT_STACK_MAX)
      return set_error(ctx, MYRT_ERR_UNSUPPORTED, "BVH deeper than the traversal stack");
  }

  device_scene& s = ctx->scene;
  if (on_device) {
    s.stats = bvh8_stats{};
    s.stats.binary_nodes = dtree.binary_nodes;
    s.stats.wide_nodes = dtree.n_nodes;
    s.stats.leaf_slots = dtree.leaf_slots;
    s.stats.triangles = dtree.n_tris;
    s.stats.wide_depth = dtree.wide_depth;
    s.stats.max_leaf_size = 4;
    s.stats.build_seconds = dtree.seconds;
  } else {
    s.stats = tree.stats;
  }
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (size_t i = 0; i < pos.size() / 3; ++i)
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], pos[3 * i + k]);
      hi[k] = std::max(hi[k], pos[3 * i + k]);
    }
  for (int k = 0; k < 3; ++k) {
    s.bounds[k] = lo[k];
    s.bounds[3 + k] = hi[k];
  }
  ctx->guide_generation++;  // a new scene invalidates what the guide learned
  s.n_prims = n_prims;
  if (on_device) {
    s.n_nodes = dtree.n_nodes;
    s.n_tris = dtree.n_tris;
    s.nodes = reinterpret_cast<uint4*>(dtree.nodes);
    s.tris = dtree.tris;
    s.node_capacity = dtree.node_capacity;
    s.tri_capacity = dtree.tri_capacity;
  } else {
    s.n_nodes = tree.nodes.size();
    s.n_tris = tree.triangles.size();
    rc = upload(ctx, reinterpret_cast<bvh8_node**>(&s.nodes), tree.nodes.data(), tree.nodes.size(), "node upload");
    if (!rc)
      rc = upload(ctx, reinterpret_cast<bvh8_triangle**>(&s.tris), tree.triangles.data(), tree.triangles.size(),
          "triangle upload");
  }
  if (!rc && !nrm.empty()) rc = upload(ctx, &s.tri_normals, nrm.data(), nrm.size(), "normal upload");
  if (!rc && !s.world_pos) rc = upload(ctx, &s.world_pos, pos.data(), pos.size(), "world triangle upload");
  // object-space geometry for transform updates
  if (!rc)
    rc = upload(ctx, &s.raw_vertices, reinterpret_cast<float4 const*>(v->vertices), v->vertex_count, "vertex upload");
  if (!rc && v->normals)
    rc = upload(ctx, &s.raw_normals, reinterpret_cast<float4 const*>(v->normals), v->vertex_count, "normal upload");
  if (!rc) rc = upload(ctx, &s.prim_src, src.data(), src.size(), "prim source upload");
  s.n_vertices = v->vertex_count;
  s.drawables = drawables;
  if (!rc && !uvs.empty()) rc = upload(ctx, &s.tri_uvs, uvs.data(), uvs.size(), "uv upload");
  if (!rc) rc = upload(ctx, &s.tri_material, mat.data(), mat.size(), "material index upload");
  if (!rc && v->material_count) {
    if (!v->materials) rc = set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "material_count > 0 but materials is null");
    else rc = upload(ctx, &s.materials, v->materials, v->material_count, "material upload");
    s.n_materials = v->material_count;
  }
  if (!rc && v->material_data_count) {
    if (!v->material_data) rc = set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "material_data is null");
    else rc = upload(ctx, &s.material_data, v->material_data, v->material_data_count, "material data upload");
    s.n_material_data = v->material_data_count;
  }
  if (!rc && ctx->tuning.instancing) rc = upload_two_level(ctx, v, drawables);
  if (!rc) rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "scene upload");
  if (rc) {
    free_scene(s);
    return rc;
  }
  s.valid = true;
  ctx->render.sample_counter = 0;  // prepare() reported a change -> invalidate_counter
  return MYRT_OK;
}


int myrt_sdf_upload(myrt_ctx* ctx, myrt_sdf_view const* v) {
  if (!ctx || !v) return MYRT_ERR_INVALID_ARGUMENT;
  int rc = check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  if (rc) return rc;
  cudaStreamSynchronize(ctx->stream);
  device_sdf& D = ctx->sdf;
  cudaFree(D.instrs);
  cudaFree(D.programs);
  cudaFree(D.params);
  cudaFree(D.drawables);
  cudaFree(D.skip_sphere);
  cudaFree(D.skip_next);
  cudaFree(D.cell_hdr);
  cudaFree(D.cell_start);
  cudaFree(D.cell_list);
  cudaFree(D.op_count);
  D = device_sdf{};
  ctx->render.sample_counter = 0;
  if (v->drawable_count == 0) return MYRT_OK;
  if (!v->instrs || !v->programs || !v->drawables || (v->param_count && !v->params))
    return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "null SDF array");
  // validate every program as the device evaluates it
  for (size_t p = 0; p < v->program_count; ++p) {
    myrt_sdf_program const pr = v->programs[p];
    if (pr.first < 0 || pr.count <= 0 || size_t(pr.first) + size_t(pr.count) > v->instr_count)
      return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "SDF program outside the instruction array");
    int depth = 0, max_depth = 0;
    bool pending_mod = false;
    for (int k = 0; k < pr.count; ++k) {
      myrt_sdf_instr const in = v->instrs[pr.first + k];
      int blocks = 0;
      switch (in.op) {
        case MYRT_SDF_SPHERE: blocks = 2; break;
        case MYRT_SDF_BOX: blocks = 4; break;
        case MYRT_SDF_TORUS: case MYRT_SDF_CAPSULE: blocks = 3; break;
        case MYRT_SDF_MENGER: blocks = 1; break;
        case MYRT_SDF_UNION: case MYRT_SDF_SUBTRACTION: case MYRT_SDF_INTERSECTION: blocks = 0; break;
        case MYRT_SDF_SMOOTH_UNION: blocks = 1; break;
        case MYRT_SDF_TRANSLATE: blocks = 3; break;
        case MYRT_SDF_MIRROR: blocks = 1; break;
        default: return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "unknown SDF opcode");
      }
      if (blocks && (in.param_offset < 0 || size_t(in.param_offset) + size_t(blocks) > v->param_count))
        return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "SDF parameter outside the parameter buffer");
      if (in.op == MYRT_SDF_MIRROR) {
        float const ax = v->params[in.param_offset];
        if (!(ax == 0.f || ax == 1.f || ax == 2.f)) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "mirror axis");
      }
      if (in.op >= MYRT_SDF_TRANSLATE) {
        pending_mod = true;
      } else if (in.op >= MYRT_SDF_UNION) {
        if (depth < 2 || pending_mod) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "SDF operator without two operands");
        --depth;
      } else {
        pending_mod = false;
        max_depth = std::max(max_depth, ++depth);
      }
    }
    if (depth != 1 || pending_mod) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "SDF program leaves no single result");
    if (max_depth > 24) return set_error(ctx, MYRT_ERR_UNSUPPORTED, "SDF program stack deeper than 24");
  }
  std::vector<float4> skip_sphere;
  std::vector<int2> skip_next;
  sdf_skip_tables(v, skip_sphere, skip_next);
  sdf_cells cells;
  std::vector<int> op_count;
  if (ctx->tuning.sdf_cells != 1) {
    sdf_cell_tables(v, ctx->tuning.sdf_cells ? int(ctx->tuning.sdf_cells) : 32, cells);
    if (!skip_next.empty() || !cells.list.empty()) sdf_op_counts(v, op_count);
  }
  std::vector<float> dr(v->drawable_count * 36);
  for (size_t d = 0; d < v->drawable_count; ++d) {
    myrt_sdf_drawable const& s = v->drawables[d];
    if (s.sdf_index < 0 || size_t(s.sdf_index) >= v->program_count)
      return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "SDF drawable references a missing program");
    std::memcpy(&dr[36 * d], &s, sizeof(myrt_sdf_drawable));
  }
  rc = upload(ctx, reinterpret_cast<myrt_sdf_instr**>(&D.instrs), v->instrs, v->instr_count, "SDF instructions");
  if (!rc)
    rc = upload(ctx, reinterpret_cast<myrt_sdf_program**>(&D.programs), v->programs, v->program_count, "SDF programs");
  if (!rc && v->param_count) rc = upload(ctx, &D.params, v->params, v->param_count, "SDF parameters");
  if (!rc) rc = upload(ctx, &D.drawables, dr.data(), dr.size(), "SDF drawables");
  if (!rc && !skip_next.empty()) {
    rc = upload(ctx, &D.skip_sphere, skip_sphere.data(), skip_sphere.size(), "SDF skip spheres");
    if (!rc) rc = upload(ctx, &D.skip_next, skip_next.data(), skip_next.size(), "SDF skip groups");
  }
  if (!rc && !cells.list.empty()) {
    rc = upload(ctx, &D.cell_hdr, cells.hdr.data(), cells.hdr.size(), "SDF cell headers");
    if (!rc) rc = upload(ctx, &D.cell_start, cells.start.data(), cells.start.size(), "SDF cell starts");
    if (!rc) rc = upload(ctx, &D.cell_list, cells.list.data(), cells.list.size(), "SDF cell lists");
  }
  if (!rc && !op_count.empty()) rc = upload(ctx, &D.op_count, op_count.data(), op_count.size(), "SDF operator counts");
  if (!rc) rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "SDF upload");
  if (rc) return rc;
  D.n_drawables = int(v->drawable_count);
  D.n_programs = int(v->program_count);
  return MYRT_OK;
}

int myrt_trace_sdf(myrt_ctx* ctx, myrt_ray const* rays, uint32_t n, int32_t steps, float eps, int any_hit,
    uint32_t const* rng_states, float* out) {
  if (!ctx) return MYRT_ERR_INVALID_ARGUMENT;
  if (!rays || !out) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "null ray or output pointer");
  if (steps < 0 || !(eps > 0.f)) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "steps >= 0 and eps > 0 required");
  return trace_sdf_rays(ctx, rays, n, steps, eps, any_hit, rng_states, out);
}

int myrt_scene_copy_bvh(myrt_ctx* ctx, void* nodes, void* triangles) {
  if (!ctx) return MYRT_ERR_INVALID_ARGUMENT;
  if (!ctx->scene.valid) return set_error(ctx, MYRT_ERR_NO_SCENE, "no scene uploaded");
  int rc = MYRT_OK;
  if (nodes)
    rc = check_cuda(ctx, cudaMemcpyAsync(nodes, ctx->scene.nodes, ctx->scene.n_nodes * sizeof(bvh8_node),
                             cudaMemcpyDeviceToHost, ctx->stream), "node read-back");
  if (!rc && triangles)
    rc = check_cuda(ctx, cudaMemcpyAsync(triangles, ctx->scene.tris, ctx->scene.n_tris * sizeof(bvh8_triangle),
                             cudaMemcpyDeviceToHost, ctx->stream), "triangle read-back");
  if (!rc) rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "BVH read-back");
  return rc;
}

int myrt_scene_bvh_info(myrt_ctx* ctx, myrt_bvh_info* info) {
  if (!ctx || !info) return MYRT_ERR_INVALID_ARGUMENT;
  if (!ctx->scene.valid) return set_error(ctx, MYRT_ERR_NO_SCENE, "no scene uploaded");
  fill_info(ctx->scene.stats, ctx->scene.n_nodes, ctx->scene.n_tris, info);
  return MYRT_OK;
}

int myrt_trace_closest(myrt_ctx* ctx, myrt_ray const* rays, uint32_t n, myrt_hit* hits, int intersector) {
  int rc = validate_query(ctx, rays, hits, intersector);
  if (rc) return rc;
  return host_query(ctx, rays, n, hits, sizeof(myrt_hit), intersector, false);
}

int myrt_trace_any(myrt_ctx* ctx, myrt_ray const* rays, uint32_t n, uint8_t* occluded, int intersector) {
  int rc = validate_query(ctx, rays, occluded, intersector);
  if (rc) return rc;
  return host_query(ctx, rays, n, occluded, sizeof(uint8_t), intersector, true);
}

int myrt_trace_closest_device(myrt_ctx* ctx, myrt_ray const* rays, uint32_t n, myrt_hit* hits, int intersector,
    void* stream) {
  int rc = validate_query(ctx, rays, hits, intersector);
  if (rc) return rc;
  trace_args a = base_args(ctx);
  a.rays = reinterpret_cast<float4 const*>(rays);
  a.n = n;
  a.hits = reinterpret_cast<float4*>(hits);
  return launch_trace(ctx, a, intersector, false, false, stream ? static_cast<cudaStream_t>(stream) : ctx->stream);
}

int myrt_trace_any_device(myrt_ctx* ctx, myrt_ray const* rays, uint32_t n, uint8_t* occluded, int intersector,
    void* stream) {
  int rc = validate_query(ctx, rays, occluded, intersector);
  if (rc) return rc;
  trace_args a = base_args(ctx);
  a.rays = reinterpret_cast<float4 const*>(rays);
  a.n = n;
  a.occluded = occluded;
  return launch_trace(ctx, a, intersector, true, false, stream ? static_cast<cudaStream_t>(stream) : ctx->stream);
}

int myrt_trace_closest_stats_device(myrt_ctx* ctx, myrt_ray const* rays, uint32_t n, myrt_hit* hits, uint32_t* nodes,
    uint32_t* tris, int intersector, void* stream) {
  int rc = validate_query(ctx, rays, hits, intersector);
  if (rc) return rc;
  if (!nodes || !tris) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "null counter pointer");
  trace_args a = base_args(ctx);
  a.rays = reinterpret_cast<float4 const*>(rays);
  a.n = n;
  a.hits = reinterpret_cast<float4*>(hits);
  a.stat_nodes = nodes;
  a.stat_tris = tris;
  return launch_trace(ctx, a, intersector, false, true, stream ? static_cast<cudaStream_t>(stream) : ctx->stream);
}

int myrt_render(myrt_ctx* ctx, myrt_camera const* camera, myrt_render_params const* p) {
  if (!ctx) return MYRT_ERR_INVALID_ARGUMENT;
  if (!camera || !p) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "null camera or params");
  if (!ctx->scene.valid) return set_error(ctx, MYRT_ERR_NO_SCENE, "no scene uploaded");
  if (p->width == 0 || p->height == 0 || uint64_t(p->width) * p->height > (uint64_t(1) << 30))
    return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "image size must be 1 .. 2^30 pixels");
  if (p->num_bounces < 0 || p->num_bounces > 1024)
    return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "num_bounces must be in [0, 1024]");
  if (p->shading != MYRT_SHADE_REFERENCE && p->shading != MYRT_SHADE_PHYSICAL && p->shading != MYRT_SHADE_GUIDED)
    return set_error(ctx, MYRT_ERR_UNSUPPORTED, "unknown shading mode");
  bool const physical = p->shading != MYRT_SHADE_REFERENCE;
  if (physical && (p->max_depth < 0 || p->max_depth > 64 || p->rr_start < 0 || p->accum_fp64 > 1))
    return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "max_depth must be in [0, 64], rr_start >= 0, accum_fp64 0 or 1");
  if (physical && p->frames > (1u << 24))
    return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "at most 2^24 samples per pixel per call");
  if (p->frames == 0) return MYRT_OK;
  // set_view_matrix / set_projection_matrix: a changed camera restarts accumulation;
  // so does a change of shading mode or accumulation precision
  render_state& R = ctx->render;
  if (!R.have_camera || std::memcmp(R.last_camera, camera, sizeof(R.last_camera)) != 0) {
    std::memcpy(R.last_camera, camera, sizeof(R.last_camera));
    R.have_camera = true;
    R.sample_counter = 0;
  }
  uint32_t const fp64 = physical ? p->accum_fp64 : 0u;
  if (R.mode != p->shading || R.fp64 != fp64) {
    R.mode = p->shading;
    R.fp64 = fp64;
    R.sample_counter = 0;
  }
  if (R.pending_first >= 0) {  // myrt_begin_samples
    R.sample_counter = physical ? uint32_t(R.pending_first) : 0u;
    R.restart = true;
    R.pending_first = -1;
  }
  int const rc = physical ? render_physical_frames(ctx, camera, p) : render_reference_frames(ctx, camera, p);
  R.restart = false;
  return rc;
}

int myrt_set_area_lights(myrt_ctx* ctx, myrt_area_light const* lights, uint32_t n) {
  if (!ctx) return MYRT_ERR_INVALID_ARGUMENT;
  return set_area_lights(ctx, lights, n);
}

int myrt_guide_configure(myrt_ctx* ctx, myrt_guide_params const* p) {
  if (!ctx || !p) return MYRT_ERR_INVALID_ARGUMENT;
  return guide_configure(ctx, p);
}
int myrt_guide_get_config(myrt_ctx* ctx, myrt_guide_params* p) {
  if (!ctx || !p) return MYRT_ERR_INVALID_ARGUMENT;
  return guide_get_config(ctx, p);
}
int myrt_guide_reset(myrt_ctx* ctx) {
  if (!ctx) return MYRT_ERR_INVALID_ARGUMENT;
  return guide_reset(ctx);
}
int myrt_guide_get_params(myrt_ctx* ctx, float* params) {
  if (!ctx || !params) return MYRT_ERR_INVALID_ARGUMENT;
  return guide_params_io(ctx, params, nullptr);
}
int myrt_guide_set_params(myrt_ctx* ctx, float const* params) {
  if (!ctx || !params) return MYRT_ERR_INVALID_ARGUMENT;
  return guide_params_io(ctx, nullptr, params);
}
int myrt_guide_eval(myrt_ctx* ctx, float const* points, uint32_t n, float* lobes) {
  if (!ctx || (n && (!points || !lobes))) return MYRT_ERR_INVALID_ARGUMENT;
  if (!ctx->scene.valid) return set_error(ctx, MYRT_ERR_NO_SCENE, "no scene uploaded (positions use its bounds)");
  return guide_eval(ctx, points, n, lobes);
}
int myrt_guide_gradients(myrt_ctx* ctx, float const* samples, uint32_t n, float* grads, float* loss) {
  if (!ctx || !grads || (n && !samples)) return MYRT_ERR_INVALID_ARGUMENT;
  if (!ctx->scene.valid) return set_error(ctx, MYRT_ERR_NO_SCENE, "no scene uploaded (positions use its bounds)");
  if (n > (1u << 24)) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "at most 2^24 samples");
  return guide_gradients(ctx, samples, n, grads, loss);
}
int myrt_guide_train(myrt_ctx* ctx, float const* samples, uint32_t n, uint32_t steps, float* loss_per_step) {
  if (!ctx || (n && !samples)) return MYRT_ERR_INVALID_ARGUMENT;
  if (!ctx->scene.valid) return set_error(ctx, MYRT_ERR_NO_SCENE, "no scene uploaded (positions use its bounds)");
  if (n > (1u << 24) || steps > 65536) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "too many samples or steps");
  return guide_train_samples(ctx, samples, n, steps, loss_per_step);
}
int myrt_guide_get_stats(myrt_ctx* ctx, myrt_guide_stats* out) {
  if (!ctx || !out) return MYRT_ERR_INVALID_ARGUMENT;
  return guide_stats(ctx, out);
}

int myrt_get_render_stats(myrt_ctx* ctx, myrt_render_stats* out) {
  if (!ctx || !out) return MYRT_ERR_INVALID_ARGUMENT;
  return get_render_stats(ctx, out);
}

int myrt_read_accumulation_f64(myrt_ctx* ctx, double* rgba_sum) {
  if (!ctx || !rgba_sum) return MYRT_ERR_INVALID_ARGUMENT;
  render_state const& R = ctx->render;
  if (!R.accum64 || !R.fp64) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "no FP64 accumulation in progress");
  size_t const bytes = size_t(R.width) * R.height * 32;
  int rc = check_cuda(ctx, cudaMemcpyAsync(rgba_sum, R.accum64, bytes, cudaMemcpyDeviceToHost, ctx->stream), "read");
  if (!rc) rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "read");
  return rc;
}

int myrt_render_noalloc(myrt_ctx* ctx, myrt_camera const* camera, myrt_render_params const* p, uint32_t sample_index,
    float* accum_rgba, float* display_rgba, void* stream) {
  if (!ctx) return MYRT_ERR_INVALID_ARGUMENT;
  if (!camera || !p || !accum_rgba || !display_rgba)
    return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "null camera, params or image pointer");
  if (!ctx->scene.valid) return set_error(ctx, MYRT_ERR_NO_SCENE, "no scene uploaded");
  if (p->width == 0 || p->height == 0) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "empty image");
  if (p->num_bounces < 0 || p->num_bounces > 1024)
    return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "num_bounces must be in [0, 1024]");
  if (p->shading != MYRT_SHADE_REFERENCE)
    return set_error(ctx, MYRT_ERR_UNSUPPORTED, "myrt_render_noalloc: only MYRT_SHADE_REFERENCE is supported");
  if (p->frames == 0) return MYRT_OK;
  return render_reference_frames_noalloc(ctx, camera, p, sample_index, reinterpret_cast<float4*>(accum_rgba),
      reinterpret_cast<float4*>(display_rgba), stream ? static_cast<cudaStream_t>(stream) : ctx->stream);
}

int myrt_render_size(myrt_ctx* ctx, uint32_t* width, uint32_t* height) {
  if (!ctx || !width || !height) return MYRT_ERR_INVALID_ARGUMENT;
  bool const any = ctx->render.accum != nullptr;
  *width = any ? ctx->render.width : 0u;
  *height = any ? ctx->render.height : 0u;
  return MYRT_OK;
}

int myrt_read_accumulation(myrt_ctx* ctx, float* rgba_sum, float* rgba_display) {
  if (!ctx) return MYRT_ERR_INVALID_ARGUMENT;
  render_state const& R = ctx->render;
  if (!R.accum) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "nothing rendered yet");
  size_t const bytes = size_t(R.width) * R.height * 16;
  int rc = MYRT_OK;
  if (rgba_sum)
    rc = check_cuda(ctx, cudaMemcpyAsync(rgba_sum, R.accum, bytes, cudaMemcpyDeviceToHost, ctx->stream), "read");
  if (!rc && rgba_display)
    rc = check_cuda(ctx, cudaMemcpyAsync(rgba_display, R.display, bytes, cudaMemcpyDeviceToHost, ctx->stream), "read");
  if (rc) return rc;
  return myrt_sync(ctx);
}

int myrt_render_buffers(myrt_ctx* ctx, void** accum, void** display) {
  if (!ctx) return MYRT_ERR_INVALID_ARGUMENT;
  if (accum) *accum = ctx->render.accum;
  if (display) *display = ctx->render.display;
  return MYRT_OK;
}

int myrt_reset_accumulation(myrt_ctx* ctx) {
  if (!ctx) return MYRT_ERR_INVALID_ARGUMENT;
  ctx->render.sample_counter = 0;
  ctx->render.pending_first = -1;
  return MYRT_OK;
}

int myrt_begin_samples(myrt_ctx* ctx, uint32_t first_sample) {
  if (!ctx) return MYRT_ERR_INVALID_ARGUMENT;
  if (first_sample > (1u << 30))
    return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "first sample index above 2^30");
  ctx->render.pending_first = first_sample;
  return MYRT_OK;
}

int myrt_render_buffer_f64(myrt_ctx* ctx, void** accum64) {
  if (!ctx || !accum64) return MYRT_ERR_INVALID_ARGUMENT;
  render_state const& R = ctx->render;
  if (!R.accum64 || !R.fp64) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "no FP64 accumulation in progress");
  *accum64 = R.accum64;
  return MYRT_OK;
}

int myrt_sample_count(myrt_ctx* ctx, uint32_t* count) {
  if (!ctx || !count) return MYRT_ERR_INVALID_ARGUMENT;
  *count = ctx->render.sample_counter;
  return MYRT_OK;
}

int myrt_set_seed(myrt_ctx* ctx, uint32_t seed) {
  if (!ctx) return MYRT_ERR_INVALID_ARGUMENT;
  ctx->host_rng.seed(seed);
  return MYRT_OK;
}

int myrt_sync(myrt_ctx* ctx) {
  if (!ctx) return MYRT_ERR_INVALID_ARGUMENT;
  int rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "stream sync");
  if (rc) return rc;
  rc = check_cuda(ctx, cudaDeviceSynchronize(), "device sync");
  if (rc) return rc;
  uint32_t err = 0;
  rc = check_cuda(ctx, cudaMemcpy(&err, ctx->d_err, sizeof(err), cudaMemcpyDeviceToHost), "error word");
  if (rc) return rc;
  if (err) {
    cudaMemset(ctx->d_err, 0, sizeof(uint32_t));
    char buf[96];
    std::snprintf(buf, sizeof buf, "device abort, error bits 0x%08x", err);
    return set_error(ctx, MYRT_ERR_DEVICE_ABORT, buf);
  }
  return MYRT_OK;
}

}  // extern "C"
