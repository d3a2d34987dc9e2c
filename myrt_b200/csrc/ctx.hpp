// Context state shared by the C-ABI translation units.
#pragma once
#include <cuda_runtime.h>

#include <array>

#include <cstdint>
#include <random>
#include <string>
#include <vector>

#include "../../include/myrt_cuda.h"
#include "bvh8.hpp"
#include "bvh8_device.hpp"
#include "instances.hpp"

namespace myrt_b200 {

struct guide_state;

// Device-resident scene: BVH, pre-gathered triangles and the shading buffers.
struct forward_state;  // raster.cu

struct device_scene {
  uint4* nodes = nullptr;      // 5 uint4 per wide node
  float4* tris = nullptr;      // 3 float4 per triangle reference (leaf order)
  // Shading attributes per baked triangle (prim id order): world-space
  // shading normals at the 3 corners, uvs, material index.
  float4* tri_normals = nullptr;  // 3 float4 per prim
  float2* tri_uvs = nullptr;      // 3 float2 per prim
  int32_t* tri_material = nullptr;
  myrt_material_ref* materials = nullptr;
  float* material_data = nullptr;
  size_t n_nodes = 0, n_tris = 0, n_prims = 0, n_materials = 0, n_material_data = 0;
  bvh8_stats stats{};
  float bounds[6] = {0, 0, 0, 0, 0, 0};  // world AABB of the triangles (min xyz, max xyz)
  bool valid = false;
  // object-space geometry kept for myrt_scene_set_transforms: vertices and
  // normals as uploaded, per prim its three vertex indices and its drawable
  float4* raw_vertices = nullptr;
  float4* raw_normals = nullptr;
  uint4* prim_src = nullptr;
  size_t n_vertices = 0;
  std::vector<myrt_drawable> drawables;
  // world-space corners per prim (9 floats, prim id = draw order) for the
  // forward renderer's rasteriser
  float* world_pos = nullptr;
  // capacities of nodes / tris when the device builder made them (0: host
  // tree, not reusable), and myrt_scene_set_transforms' second set of tree and
  // corner buffers: each move builds into the spare set and swaps, so repeated
  // moves allocate nothing
  size_t node_capacity = 0, tri_capacity = 0;
  uint4* spare_nodes = nullptr;
  float4* spare_tris = nullptr;
  float* spare_pos = nullptr;
  size_t spare_node_capacity = 0, spare_tri_capacity = 0;
  void* move_stage = nullptr;  // drawable transforms + bounds of a move
  size_t move_stage_bytes = 0;
  // two-level structure for instanced ray queries (tuning.instancing = 1,
  // instances.hpp): object-space trees of the distinct geometries, the tree over
  // the drawables' world boxes and its instance records (4 float4 each)
  uint4* blas_nodes = nullptr;
  float4* blas_tris = nullptr;
  uint4* tlas_nodes = nullptr;
  float4* inst_records = nullptr;
  size_t n_blas_nodes = 0, n_blas_tris = 0, n_tlas_nodes = 0, n_inst_records = 0;
  int blas_depth = 0, tlas_depth = 0;
  std::vector<geometry_tree> geometries;         // per distinct geometry
  std::vector<uint32_t> drawable_geometry;       // per drawable
  std::vector<uint32_t> drawable_prim_base;      // per drawable
  bool instanced = false;
};

// SDF drawables (uploaded separately; scene::prepare's sdf buffers).
struct device_sdf {
  int2* instrs = nullptr;
  int2* programs = nullptr;
  float* params = nullptr;
  float* drawables = nullptr;  // 36 floats each
  // per instruction: bounding sphere (centre, radius) of the group "modifiers,
  // primitive, union / smooth union" that starts there, and (index after the
  // group's operator, k bits); next 0 = not a skippable group start
  float4* skip_sphere = nullptr;
  int2* skip_next = nullptr;
  // cell lists of left-to-right chain programs (sdf_skip.hpp sdf_cells),
  // null when no program has them
  int4* cell_hdr = nullptr;
  int* cell_start = nullptr;
  uint32_t* cell_list = nullptr;
  int* op_count = nullptr;  // sdf_skip.hpp sdf_op_counts, null when not usable
  int n_drawables = 0;
  int n_programs = 0;
};

// Wavefront render state (sequential_pathtracer's buffers and counters).
struct render_state {
  uint32_t width = 0, height = 0;
  float4* gen[2] = {nullptr, nullptr};  // generate_output_t, 5 float4 per ray (ping-pong)
  float4* trace = nullptr;              // trace_output_t, 4 float4 per ray
  float4* accum = nullptr;              // debug_image: rgb sum, sample count in a
  float4* display = nullptr;            // output_image: clamp(sum / count, 0, 4)
  uint32_t* counts = nullptr;           // [2] active ray counts (ping-pong)
  uint32_t* block_sums = nullptr;       // per-block survivor counts, then offsets
  float* pass_tex = nullptr;            // frames * passes * 1024 random texture floats
  float4* fcol = nullptr;               // frames in flight: final colour per frame and pixel
  uint32_t frames_cap = 0;              // frames in flight the ray buffers hold
  uint32_t* okeys[2] = {nullptr, nullptr};  // visiting order of a trace pass: keys, slots
  uint32_t* ovals[2] = {nullptr, nullptr};
  void* otemp = nullptr;                // radix sort temporary
  float4* shadow_q = nullptr;           // NEE shadow rays of a trace pass, 2 float4 each
  size_t otemp_bytes = 0;
  size_t pass_tex_capacity = 0;         // in floats
  uint32_t sample_counter = 0;          // frames accumulated since the last reset
  int64_t pending_first = -1;           // myrt_begin_samples: first sample index of the next render
  bool restart = false;                 // the next physical render overwrites the images
  float last_camera[32] = {};
  bool have_camera = false;
  int mode = -1;                        // myrt_shading of the accumulation in progress
  uint32_t fp64 = 0;                    // physical modes: accumulation in accum64
  double4* accum64 = nullptr;           // physical modes, accum_fp64: rgb sum, count
};

// Physical / guided wavefront state: ray queues sized for one wave of paths.
struct physical_state {
  size_t capacity = 0;                  // paths per wave the buffers hold
  float4* queue[2] = {nullptr, nullptr};  // 3 float4 per ray: (o, path), (d, prev pdf), (throughput, -)
  float4* hits = nullptr;               // 3 float4 per queue slot: (p, kind), (ns, t), (ng, -)
  float4* shadow = nullptr;             // 3 float4 per shadow ray: (o, path), (d, tmax), (contribution, -)
  float4* radiance = nullptr;           // per path: rgb
  uint32_t* counts = nullptr;           // [0..1] ray queues, [2] shadow queue
  uint32_t* okeys[2] = {nullptr, nullptr};  // visiting order of an extension queue: keys, entries
  uint32_t* ovals[2] = {nullptr, nullptr};
  void* otemp = nullptr;                // radix sort temporary
  size_t otemp_bytes = 0;
  unsigned long long* stats = nullptr;  // paths, extension rays, shadow rays (cumulative)
  void* lights = nullptr;               // ps::area_light[n_lights]
  int n_lights = 0;
  void* tables = nullptr;               // scene + per-wave job tables of the last call
  size_t tables_cap = 0;
};

}  // namespace myrt_b200

struct myrt_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t aux_stream = nullptr;  // second lane for copy/compute overlap
  cudaStream_t copy_lanes[2] = {nullptr, nullptr};  // third and fourth lanes of the host-memory queries
  cudaEvent_t order_event = nullptr;  // orders a caller's stream after the context's stream
  std::string last_error;
  uint32_t* d_err = nullptr;          // device error word (atomicOr of ERR_* bits)
  myrt_b200::device_scene scene;
  myrt_b200::device_build_scratch build_scratch;  // device BVH builder temporaries, kept between builds
  myrt_b200::device_sdf sdf;
  myrt_b200::render_state render;
  myrt_b200::physical_state physical;
  myrt_b200::guide_state* guide = nullptr;  // learned proposal (guide.cu), created on first use
  uint64_t guide_generation = 0;            // bumped by scene uploads
  std::mt19937 host_rng{5489u};  // sequential_pathtracer::m_rng (default-constructed)
  myrt_tuning tuning{0u, 1u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
  int sm_count = 0;
  uint32_t* d_next = nullptr;    // ring of ray counters for the persistent traversal
  uint32_t next_slot = 0;
  // staging buffers of the host-memory entry points (one chunk slot per lane)
  void* stage[4] = {nullptr, nullptr, nullptr, nullptr};
  size_t stage_bytes = 0;
  // ray-order scratch per stream lane (keys and indices, double-buffered, and
  // the radix sort's temporary storage); `done` orders reuse across streams
  struct order_scratch {
    uint32_t* keys[2] = {nullptr, nullptr};
    uint32_t* vals[2] = {nullptr, nullptr};
    void* temp = nullptr;
    size_t cap = 0, temp_bytes = 0;
    cudaEvent_t done = nullptr;
  } order[4];
  // reference-mode textures (slots) and environment cube map; d_textures
  // mirrors `textures` as {float4*, w, h, wrap} records for the kernels
  struct texture_slot {
    float4* data = nullptr;
    int w = 0, h = 0, wrap = 0;
  };
  std::vector<texture_slot> textures;
  texture_slot* d_textures = nullptr;
  float4* cubemap = nullptr;
  int cubemap_size = 0;
  // forward (raster preview) renderer buffers, created on first use
  myrt_b200::forward_state* forward = nullptr;
  // phase timing of the ray queries: (before ordering, before traversal, after)
  bool time_phases = false;
  std::vector<std::array<cudaEvent_t, 3>> phase_pending, phase_pool;
};

namespace myrt_b200 {
int set_error(myrt_ctx* ctx, int code, std::string msg);
int check_cuda(myrt_ctx* ctx, cudaError_t e, char const* what);
void free_render(render_state& r);
void free_textures(myrt_ctx* ctx);
void free_forward(myrt_ctx* ctx);
void free_physical(physical_state& p);
int ensure_images(myrt_ctx* ctx, uint32_t W, uint32_t H);
int render_physical_frames(myrt_ctx* ctx, myrt_camera const* cam, myrt_render_params const* p);
int set_area_lights(myrt_ctx* ctx, myrt_area_light const* lights, uint32_t n);
int get_render_stats(myrt_ctx* ctx, myrt_render_stats* out);
void free_guide(guide_state* g);
int guide_configure(myrt_ctx* ctx, myrt_guide_params const* p);
int guide_reset(myrt_ctx* ctx);
int guide_params_io(myrt_ctx* ctx, float* out, float const* in);
int guide_eval(myrt_ctx* ctx, float const* points, uint32_t n, float* lobes);
int guide_gradients(myrt_ctx* ctx, float const* samples, uint32_t n, float* grads, float* loss);
int guide_train_samples(myrt_ctx* ctx, float const* samples, uint32_t n, uint32_t steps, float* loss_per_step);
int guide_stats(myrt_ctx* ctx, myrt_guide_stats* out);
int guide_get_config(myrt_ctx* ctx, myrt_guide_params* p);
int render_reference_frames(myrt_ctx* ctx, myrt_camera const* cam, myrt_render_params const* p);
int trace_sdf_rays(myrt_ctx* ctx, myrt_ray const* rays, uint32_t n, int steps, float eps, int any_hit,
    uint32_t const* rng_states, float* out);
int render_reference_frames_noalloc(myrt_ctx* ctx, myrt_camera const* cam, myrt_render_params const* p,
    uint32_t sample_index, float4* accum, float4* display, cudaStream_t st);
int upload_top_level(myrt_ctx* ctx, std::vector<myrt_drawable> const& drawables);
}  // namespace myrt_b200
