/*
 * myrt_cuda.h -- C ABI of the B200 wavefront path-tracing core.
 *
 * Plain C: pointers, sizes and POD structs only. Every function returns an
 * int status (MYRT_OK = 0, negative on error; see myrt_status) and never
 * throws. A context owns one CUDA device, one stream and all device memory;
 * it is not thread-safe (synchronise externally), different contexts may be
 * used from different threads. Host arrays passed in are read during the call
 * only.
 *
 * Each entry point names the reference interface it replaces
 * (johannes-braun/myrt, paths relative to that project).
 */
#ifndef MYRT_CUDA_H
#define MYRT_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MYRT_ABI_VERSION 1

typedef enum myrt_status {
  MYRT_OK = 0,
  MYRT_ERR_INVALID_ARGUMENT = -1,
  MYRT_ERR_CUDA = -2,
  MYRT_ERR_OUT_OF_MEMORY = -3,
  MYRT_ERR_NO_SCENE = -4,
  MYRT_ERR_UNSUPPORTED = -5,
  MYRT_ERR_DEVICE_ABORT = -6, /* a kernel hit an iteration or stack limit and stopped */
  MYRT_ERR_INTERNAL = -7
} myrt_status;

typedef struct myrt_ctx myrt_ctx;

typedef struct myrt_device_opts {
  int device;            /* CUDA ordinal */
  uint32_t flags;        /* reserved, 0 */
} myrt_device_opts;

/* 32-byte ray: origin, tmin, direction, tmax. Direction need not be unit. */
typedef struct myrt_ray {
  float o[3];
  float tmin;
  float d[3];
  float tmax;
} myrt_ray;

/* 16-byte hit: prim = triangle index in the uploaded index buffer order
 * (index_count / 3 numbering), -1 on miss; t and barycentrics u (weight of
 * the triangle's second vertex) and v (third vertex) as in
 * src/pt/intersect.glsl:3-28. On a miss t = ray tmax, u = v = 0. */
typedef struct myrt_hit {
  int32_t prim;
  float t;
  float u;
  float v;
} myrt_hit;

/* Instance record, byte-compatible with scene::drawable_geometry_t
 * (src/pathtracer/scene.hpp:97-104): 160 bytes. */
typedef struct myrt_drawable {
  float transformation[16];         /* column-major mat4 */
  float inverse_transformation[16]; /* column-major mat4 */
  uint32_t bvh_node_base_index;     /* ignored: the core builds its own BVH */
  uint32_t bvh_index_base_index;    /* ignored */
  uint32_t indices_base_index;
  uint32_t points_base_index;
  uint32_t index_count;
  int32_t material_index;
  int32_t geometry_index;
  int32_t pad;
} myrt_drawable;

/* scene::material_reference_t (src/pathtracer/scene.hpp:111-114). */
typedef struct myrt_material_ref {
  int32_t id;     /* material type id; 0 = the app's PBR type (7 floats) */
  int32_t offset; /* float offset into material_data */
} myrt_material_ref;

/* Host view of the scene arrays scene::prepare uploads
 * (src/pathtracer/scene.hpp:216-224, scene.cpp:330-409). vertices and
 * normals use the reference's 16-byte aligned_point_t stride (xyz + pad). If
 * drawable_count == 0 the whole index buffer is one drawable with an identity
 * transform and material 0. */
typedef struct myrt_scene_view {
  const uint32_t* indices;
  size_t index_count;
  const float* vertices; /* 4 floats per vertex */
  size_t vertex_count;
  const float* normals;  /* 4 floats per vertex, may be NULL */
  const float* uvs;      /* 2 floats per vertex, may be NULL */
  const myrt_drawable* drawables;
  size_t drawable_count;
  const myrt_material_ref* materials;
  size_t material_count;
  const float* material_data;
  size_t material_data_count;
} myrt_scene_view;

/* Build statistics of the uploaded scene's BVH. */
typedef struct myrt_bvh_info {
  uint64_t triangles;
  uint64_t binary_nodes;
  uint64_t wide_nodes;
  uint64_t leaf_slots;
  int32_t binary_depth;
  int32_t wide_depth;
  int32_t max_leaf_size;
  int32_t pad;
  double build_seconds;
  uint64_t node_bytes;
  uint64_t triangle_bytes;
} myrt_bvh_info;

/* Intersector selection. MYRT_ISECT_REFERENCE is Moller-Trumbore exactly as
 * src/pt/intersect.glsl:3-28 (det epsilon 1e-23, border slack 1e-6);
 * MYRT_ISECT_WATERTIGHT is Woop, Benthin and Wald (JCGT 2013). Both report
 * the closest hit with ties in t broken towards the smaller prim index. */
typedef enum myrt_intersector {
  MYRT_ISECT_REFERENCE = 0,
  MYRT_ISECT_WATERTIGHT = 1
} myrt_intersector;

/* ---- host-only BVH (no device needed) -------------------------------------- */

typedef struct myrt_bvh8_host myrt_bvh8_host;
/* Builds the 8-wide BVH on the host from world-space triangles (9 floats each:
 * v0, v1, v2). Replaces bvh::bvh + bvh::nodes() / reordered_indices()
 * (src/pathtracer/bvh.hpp:157-176) for callers that inspect the tree. */
int myrt_bvh8_build(const float* positions, size_t n_tris, myrt_bvh8_host** out);
int myrt_bvh8_get_info(const myrt_bvh8_host* bvh, myrt_bvh_info* info);
/* Copies the nodes (80 bytes each) and leaf-ordered triangles (48 bytes each). */
int myrt_bvh8_copy(const myrt_bvh8_host* bvh, void* nodes, void* triangles);
int myrt_bvh8_free(myrt_bvh8_host* bvh);

/* Launch configuration of the traversal kernels (set by hand or by the
 * autotuner, myrt_b200/autotune.py). */
typedef struct myrt_tuning {
  uint32_t trace_persistent; /* 0: one thread per ray; 1: persistent warps that refill finished lanes */
  uint32_t refill;           /* persistent: refill once at least this many lanes of a warp are idle (1..32) */
  uint32_t blocks_per_sm;    /* persistent: resident 128-thread blocks per SM (0 = occupancy maximum) */
  uint32_t trace_min_blocks; /* one-thread-per-ray: register cap as blocks per SM: 8 (64 regs), 10 (48 regs;
                                0 = 10), 12 */
  uint32_t trace_unit_steps; /* one-thread-per-ray: 0 = a node and all its triangles per iteration,
                                1 = one node, triangle or pop per iteration */
  uint32_t wave_paths;       /* physical / guided wavefront: paths in flight per wave (0 = 16 Mi; 4 Mi
                                while a guide trains and for batches, whose autotuner picks its own) */
  uint32_t pt_blocks_per_sm; /* physical / guided: resident 128-thread blocks per SM of the
                                grid-stride extend / shade / shadow kernels (0 = 8) */
  uint32_t trace_smem_stack; /* one-thread-per-ray: 1 = traversal stack in shared memory
                                (tree depth + 1 entries per ray), 0 = per-thread local memory */
  uint32_t bvh_builder;      /* myrt_scene_upload: 0 = host binned SAH + SAH-optimal 8-wide collapse,
                                1 = device linear BVH (Morton order, radix tree, 8-wide collapse on the
                                GPU): milliseconds for millions of triangles, slower traversal */
  uint32_t trace_order;      /* visiting order of closest / any-hit batches: 0 = device-memory queries
                                of at least 1 Mi rays sorted by origin and direction cell, host-memory
                                queries in input order; 1 = input order; 2 = always sorted. The
                                trace passes of reference shading likewise: 0 = the first two passes
                                sorted once the frames in flight hold 1 Mi rays, 1 = never, 2 = every
                                pass; and the extension queues of physical / guided waves: 0 = those
                                of vertices 1 and 2 in waves of at least 1 Mi paths, 1 = never, 2 =
                                every vertex after the camera's. Results never depend on it. */
  uint32_t sdf_cells;        /* myrt_sdf_upload: cells along the longest axis of the grid of
                                instruction segments built for each program that is a tree of
                                unions / smooth unions over translated spheres, boxes, tori and
                                capsules (0 = 32, 1 = no grid and no early exit, 2..128; programs
                                with thousands of primitives get coarser grids so that the upload
                                stays near a second). Results never depend on it. */
  uint32_t guide_poll_limit; /* guide tensor-core kernels: polls of each CTA's first mbarrier wait
                                (0 = 2^22, the bound of every other wait); a wait that runs out sets
                                the device error word (myrt_sync: MYRT_ERR_DEVICE_ABORT) after the
                                MMA in flight has retired and TMEM is freed */
  uint32_t guide_stall_test; /* 1: that first wait watches a barrier nothing arrives at, so it runs
                                out after guide_poll_limit polls: tests the timeout path without a
                                fault. 0 in normal use */
  uint32_t instancing;       /* ray queries (myrt_trace_closest / _any and their _device forms):
                                0 = one tree over the world-space (baked) triangles; 1 = the
                                reference's two-level walk (src/pt/pt_trace.comp:284-309): a tree
                                over the drawables' world boxes, each ray moved into the drawable's
                                object space by inverse_transformation and tested against the
                                untransformed geometry, so t, u and v equal the reference's bit for
                                bit (2 = the same walk as two nested loops, for comparison). 1 must
                                be set before myrt_scene_upload, which then also builds
                                one object-space tree per distinct geometry; renders always use the
                                baked tree. */
  uint32_t pt_grid;          /* physical / guided extend, shade and shadow kernels: 0 = default (2),
                                1 = grid-stride loops over pt_blocks_per_sm resident blocks per SM,
                                2 = one thread per queue entry (the grid covers the wave's paths;
                                blocks past the queue's count return at once; the mesh traversal
                                kernels then run under a 48-register cap unless pt_blocks_per_sm is
                                1..9, which gives them 64 registers).
                                Results never depend on it. */
  uint32_t ref_frames;       /* reference shading (myrt_render): frames of one call whose passes run
                                together, each in its own region of ray slots (0 = as many as fill
                                about 16 Mi rays, at most 64; 1 = one frame at a time, as the
                                reference; 2..64). Results never depend on it. */
} myrt_tuning;

/* ---- context ------------------------------------------------------------ */

/* Replaces the GL context + sequential_pathtracer construction
 * (src/main.cpp:228-231, src/pathtracer/sequential_pathtracer.hpp:22-59). */
int myrt_ctx_create(const myrt_device_opts* opts, myrt_ctx** out);
int myrt_ctx_destroy(myrt_ctx* ctx);
/* Copies the last error message (NUL-terminated, truncated to size). */
int myrt_get_last_error(myrt_ctx* ctx, char* buf, size_t size);
/* The context's CUDA stream (cudaStream_t) for callers that enqueue work. */
int myrt_get_stream(myrt_ctx* ctx, void** stream);
/* Traversal launch configuration (no counterpart in the reference, whose
 * dispatch sizes are fixed at 64 per group). */
int myrt_set_tuning(myrt_ctx* ctx, const myrt_tuning* tuning);
int myrt_get_tuning(myrt_ctx* ctx, myrt_tuning* tuning);

/* Device-time accounting of the closest / any-hit queries (no counterpart in
 * the reference): while enabled, each query records CUDA events around its
 * ordering phase (ray keys + radix sort) and its traversal kernel.
 * myrt_get_phase_times waits for the recorded queries, returns the summed
 * milliseconds and the number of traversal launches since the last call, and
 * clears them: one per device-memory query, one per chunk of a host-memory
 * query (chunks of an eighth of the query, 64 Ki to 1 Mi rays). */
int myrt_set_phase_timing(myrt_ctx* ctx, int enable);
int myrt_get_phase_times(myrt_ctx* ctx, double* order_ms, double* traverse_ms, uint64_t* queries);

/* ---- scene ---------------------------------------------------------------- */

/* Replaces scene::prepare's buffer uploads (src/pathtracer/scene.cpp:330-409)
 * and the per-geometry bvh build (scene.cpp:43-71): builds the 8-wide BVH over
 * all drawables (baked to world space) on the host, or on the device when
 * myrt_tuning.bvh_builder = 1, and keeps it in device memory. */
int myrt_scene_upload(myrt_ctx* ctx, const myrt_scene_view* scene);
int myrt_scene_bvh_info(myrt_ctx* ctx, myrt_bvh_info* info);
/* Moves instances (scene.cpp:336-344 rebuilds the reference's TLAS on the host
 * whenever an instance changes): new transformation, inverse_transformation
 * and material_index for every drawable of the uploaded scene (same count and
 * index ranges as uploaded). Re-bakes the world triangles and normals on the
 * device from the object-space geometry kept since the upload and rebuilds the
 * tree with the device builder; restarts accumulation. From the second move
 * on, the new tree is built into the buffers of the tree before the previous
 * move (no allocation), after a device-wide synchronisation, so work that
 * callers queued on their own streams against that older tree has finished. */
int myrt_scene_set_transforms(myrt_ctx* ctx, const myrt_drawable* drawables, size_t count);
/* Copies the scene's device tree to host memory: nodes (80 bytes each) and
 * leaf-ordered triangles (48 bytes each), as counted by myrt_scene_bvh_info;
 * either pointer may be null. Same layout as myrt_bvh8_copy. */
int myrt_scene_copy_bvh(myrt_ctx* ctx, void* nodes, void* triangles);

/* ---- ray queries ---------------------------------------------------------- */

/* Closest hit for n rays in HOST memory (pinned or pageable); results to host.
 * Replaces nearest_hit (src/pt/pt_trace.comp:331-386) for meshes and the CPU
 * pick path scene::pick (src/pathtracer/scene.cpp:273-314). Copies overlap the
 * kernels in chunks. */
int myrt_trace_closest(myrt_ctx* ctx, const myrt_ray* rays, uint32_t n, myrt_hit* hits, int intersector);
/* Same with DEVICE pointers, enqueued on `stream` (NULL = the ctx stream);
 * asynchronous: call myrt_sync to wait and collect device error status. */
int myrt_trace_closest_device(myrt_ctx* ctx, const myrt_ray* rays, uint32_t n, myrt_hit* hits, int intersector,
    void* stream);
/* Any hit (occlusion) for n host rays: occluded[i] = 1 if a triangle is hit
 * with tmin <= t < tmax. Replaces any_hit (src/pt/pt_trace.comp:311-329). */
int myrt_trace_any(myrt_ctx* ctx, const myrt_ray* rays, uint32_t n, uint8_t* occluded, int intersector);
int myrt_trace_any_device(myrt_ctx* ctx, const myrt_ray* rays, uint32_t n, uint8_t* occluded, int intersector,
    void* stream);
/* Per-ray traversal counters for the closest-hit kernel (device pointers):
 * nodes[i] = wide nodes fetched, tris[i] = triangles tested. Used to count the
 * algorithmic bytes per ray (80 B per node, 48 B per triangle). */
int myrt_trace_closest_stats_device(myrt_ctx* ctx, const myrt_ray* rays, uint32_t n, myrt_hit* hits,
    uint32_t* nodes, uint32_t* tris, int intersector, void* stream);

/* ---- SDF drawables ------------------------------------------------------------ */

/* Flat SDF program instructions. The reference compiles an instruction tree
 * (src/pathtracer/sdf.hpp:399-633) into GLSL (sdf.cpp:122-407); this core
 * evaluates the same tree as a post-order program: modifier instructions move
 * the position of the next primitive (innermost first), primitives push a
 * distance and a material, operators pop two and push one. param_offset indexes
 * the float parameter buffer, laid out per type as the reference's sdf_data
 * (float = 1 block, int = 1 block holding the value, vec3 = 3 blocks). */
typedef enum myrt_sdf_op {
  MYRT_SDF_SPHERE = 1,        /* radius, material */
  MYRT_SDF_BOX = 2,           /* size.xyz, material */
  MYRT_SDF_TORUS = 3,         /* radius_large, radius_small, material */
  MYRT_SDF_CAPSULE = 4,       /* vertical capsule: height, radius, material */
  MYRT_SDF_MENGER = 5,        /* material */
  MYRT_SDF_UNION = 16,
  MYRT_SDF_SUBTRACTION = 17,
  MYRT_SDF_INTERSECTION = 18,
  MYRT_SDF_SMOOTH_UNION = 19, /* factor */
  MYRT_SDF_TRANSLATE = 32,    /* offset.xyz */
  MYRT_SDF_MIRROR = 33        /* axis */
} myrt_sdf_op;

typedef struct myrt_sdf_instr {
  int32_t op;
  int32_t param_offset;
} myrt_sdf_instr;

typedef struct myrt_sdf_program {
  int32_t first; /* first instruction */
  int32_t count;
} myrt_sdf_program;

/* scene::drawable_sdf_t (src/pathtracer/scene.hpp:105-110): 144 bytes. */
typedef struct myrt_sdf_drawable {
  float transformation[16];         /* column-major */
  float inverse_transformation[16]; /* column-major */
  int32_t sdf_index;                /* program index */
  int32_t pad[3];
} myrt_sdf_drawable;

typedef struct myrt_sdf_view {
  const myrt_sdf_instr* instrs;
  size_t instr_count;
  const myrt_sdf_program* programs;
  size_t program_count;
  const float* params;
  size_t param_count;
  const myrt_sdf_drawable* drawables;
  size_t drawable_count;
} myrt_sdf_view;

/* Replaces the SDF half of scene::prepare (sdf data + drawable uploads,
 * src/pathtracer/scene.cpp:345-351, 399-401) and the GLSL assembly of
 * sdf_glsl_assembler (sdf.cpp:378-407). Programs are validated (opcodes,
 * parameter ranges, stack depth <= 24, one result). drawable_count == 0
 * removes all SDF drawables. Restarts accumulation. Programs that are trees
 * of unions / smooth unions also get, per cell of a grid (myrt_tuning.
 * sdf_cells), the instruction segments that can change their value there,
 * and a sphere outside which a march that moves away ends without a hit;
 * both leave every result bit-identical. */
int myrt_sdf_upload(myrt_ctx* ctx, const myrt_sdf_view* sdf);
/* SDF part of nearest_hit / any_hit (src/pt/pt_trace.comp:321-326, 342-352)
 * over all SDF drawables for n host rays (tmax = max distance), with
 * raymarch.glsl's marching (steps, eps). rng_states (may be NULL: all 0) start
 * each ray's random stream, which picks materials at operator blends. out: 8
 * floats per ray: hit (0/1), t, normal xyz, u, v, material (int bits). */
int myrt_trace_sdf(myrt_ctx* ctx, const myrt_ray* rays, uint32_t n, int32_t steps, float eps, int any_hit,
    const uint32_t* rng_states, float* out);

/* ---- wavefront rendering ---------------------------------------------------- */

/* The matrices sequential_pathtracer uploads to pt_generate.comp (column-major):
 * ray direction = normalize((inverse_view * inverse_projection * (ndc, 1, 1)).xyz),
 * origin = inverse_view column 3 (src/pt/pt_generate.comp:63-66). */
typedef struct myrt_camera {
  float inverse_view[16];
  float inverse_projection[16];
} myrt_camera;

typedef enum myrt_shading {
  /* The reference's passes and shading: 2 hard-coded sphere lights with NEE,
   * the PBR material's bounce/evaluate, Russian roulette on the path pdf, sky
   * gradient (src/pt/pt_trace.comp, pt_color.comp). */
  MYRT_SHADE_REFERENCE = 0,
  /* Physically based: GGX + Lambert BSDF over the same PBR record, next-event
   * estimation to the area lights (myrt_set_area_lights) with power-heuristic
   * MIS, Russian roulette on the throughput, constant environment radiance.
   * `frames` is the number of samples per pixel of the call. Results depend
   * only on (pixel, sample index, seed): wave size and batching do not change
   * them. */
  MYRT_SHADE_PHYSICAL = 1,
  /* MYRT_SHADE_PHYSICAL with a learned proposal mixed into BSDF sampling by
   * one-sample MIS (myrt_guide_*). */
  MYRT_SHADE_GUIDED = 2
} myrt_shading;

typedef struct myrt_render_params {
  uint32_t width, height;
  int32_t num_bounces; /* sequential_pathtracer::set_num_bounces (reference default 10) */
  uint32_t frames;     /* frames (one sample per pixel each) to accumulate in this call */
  int32_t shading;     /* myrt_shading */
  uint32_t flags;      /* reserved, 0 */
  int32_t sdf_marching_steps;  /* set_sdf_marching_steps (reference default 400) */
  float sdf_marching_epsilon;  /* set_sdf_marching_epsilon (reference default 1e-5) */
  /* physical and guided modes (ignored by MYRT_SHADE_REFERENCE) */
  int32_t max_depth;      /* surface vertices with NEE and a continuation ray (0: 8) */
  int32_t rr_start;       /* Russian roulette from this vertex index on */
  uint32_t seed;          /* key of the counter-based random stream */
  uint32_t accum_fp64;    /* 1: accumulate in FP64 (converged-oracle renders) */
  float env_radiance[3];  /* radiance of rays that leave the scene */
  uint32_t wave_paths;    /* paths in flight per wave (0: the context's tuning) */
  /* reference mode: depth of field (pt_generate.comp:35-48, bokeh.glsl;
   * sequential_pathtracer set_dof_enabled / set_lens_size / set_focus /
   * set_bokeh_mask) */
  int32_t dof_active;
  float lens_size[2];
  float focus;
  int32_t bokeh_texture;  /* texture slot + 1 of the bokeh mask (0: none, value 1 everywhere) */
} myrt_render_params;

/* Textures for the reference shading mode (the bindless albedo textures of
 * material_new.glsl:29-31 and the bokeh mask): slot < 256; rgba = width *
 * height * 4 floats (host memory), sampled as GL samples them at level 0
 * (GL_LINEAR; wrap 0 = GL_REPEAT, the reference's default, 1 = clamp to
 * edge, 2 = mirrored repeat). A PBR material's texture field (floats 5 and 6
 * of its 7) holds the handle as bits: (slot + 1, 0); (0, 0) = none. A null
 * rgba or zero size empties the slot. */
int myrt_texture_upload(myrt_ctx* ctx, uint32_t slot, const float* rgba, uint32_t width, uint32_t height,
    uint32_t wrap);
/* The environment cube map of pt_color.comp:190-199 (set_cubemap): 6 faces
 * (+x, -x, +y, -y, +z, -z), size * size * 4 floats each, stored at half
 * precision (the reference's RGB16F); size <= 10 (or 0) uses the sky
 * gradient, as the reference does for small or missing maps. */
int myrt_cubemap_upload(myrt_ctx* ctx, const float* faces_rgba, uint32_t size);

/* Parallelogram area light corner + a*edge_u + b*edge_v, a, b in [0, 1],
 * emitting `emission` (radiance) on the side of cross(edge_u, edge_v). Used by
 * the physical and guided modes; lights are not occluders for shadow rays.
 * Config "one 0.2 x 0.2 area light, emission 20" is one such record. */
typedef struct myrt_area_light {
  float corner[3];
  float edge_u[3];
  float edge_v[3];
  float emission[3];
} myrt_area_light;

/* Replaces the area lights (n <= 64; n = 0 removes them). Restarts
 * accumulation. NEE picks a light with probability proportional to
 * luminance(emission) * area. */
int myrt_set_area_lights(myrt_ctx* ctx, const myrt_area_light* lights, uint32_t n);

/* Renders `frames` frames, each the reference's generate -> {trace, color,
 * filter} x num_bounces -> trace, color sequence, accumulating into the
 * context's images. Replaces sequential_pathtracer::run
 * (src/pathtracer/sequential_pathtracer.cpp:10-69). A change of resolution or
 * camera, or a scene upload, restarts accumulation (invalidate_counter). The
 * host random stream is std::mt19937 (default seed 5489) drawn in the
 * reference's order; myrt_set_seed reseeds it. Asynchronous on the ctx stream
 * until myrt_read_accumulation or myrt_sync. */
int myrt_render(myrt_ctx* ctx, const myrt_camera* camera, const myrt_render_params* params);
/* Copies the accumulation image (debug_image: rgb sum, sample count in a) and
 * the display image (output_image: clamp(sum / count, 0, 4)), W*H*4 floats
 * each, row-major from pixel (0, 0); either pointer may be NULL. */
int myrt_read_accumulation(myrt_ctx* ctx, float* rgba_sum, float* rgba_display);
/* Rays traced by the physical / guided wavefront since the context was
 * created (cumulative; take differences around a call). */
typedef struct myrt_render_stats {
  uint64_t paths;           /* camera rays */
  uint64_t extension_rays;  /* closest-hit queries, camera rays included */
  uint64_t shadow_rays;     /* any-hit queries */
  uint64_t reserved;
} myrt_render_stats;
int myrt_get_render_stats(myrt_ctx* ctx, myrt_render_stats* out);

/* ---- batches: many views of many scenes in one CUDA graph ---------------------
 * A batch renders jobs (scene, camera, resolution, spp, seed) of the physical
 * mode over several scenes at once: waves pack whole sample rows of many jobs,
 * the whole frame (every wave of every job) is captured once as a CUDA graph
 * and each myrt_batch_render replays it. A job's image equals, bit for bit,
 * the same job rendered alone with myrt_render (MYRT_SHADE_PHYSICAL). No
 * counterpart in the reference (one view per sequential_pathtracer). */
typedef struct myrt_batch_job {
  uint32_t scene;          /* index into the batch's scene contexts */
  uint32_t width, height;
  uint32_t spp;            /* samples per pixel per myrt_batch_render */
  uint32_t seed;
  int32_t max_depth;       /* 0: 8 */
  int32_t rr_start;
  uint32_t accum_fp64;
  float env_radiance[3];
  int32_t sdf_marching_steps;
  float sdf_marching_epsilon;
  uint32_t pad;
  myrt_camera camera;
} myrt_batch_job;
typedef struct myrt_batch_info {
  uint32_t waves;           /* waves per frame */
  uint32_t max_wave_paths;  /* largest wave */
  uint64_t paths_per_frame;
  uint32_t graph_nodes;     /* nodes of the captured frame graph */
  uint32_t wave_paths;      /* tuning in force (0: the first scene context's) */
  uint32_t blocks_per_sm;
  uint32_t pad;
} myrt_batch_info;
typedef struct myrt_batch myrt_batch;
/* scenes: contexts holding the uploaded scenes (and their lights / SDF
 * drawables), all on one device; they must outlive the batch, and the batch
 * renders on scenes[0]'s stream. The batch owns its queues and images. */
int myrt_batch_create(myrt_ctx* const* scenes, uint32_t n_scenes, const myrt_batch_job* jobs, uint32_t n_jobs,
    myrt_batch** out);
/* Wave size (paths in flight) and resident blocks per SM of the grid-stride
 * kernels; 0 = the first scene context's tuning. Re-captures on next render. */
int myrt_batch_set_tuning(myrt_batch* batch, uint32_t wave_paths, uint32_t blocks_per_sm);
/* One graph launch: every job accumulates its spp samples. Asynchronous. */
int myrt_batch_render(myrt_batch* batch);
/* Job `job`'s accumulation (rgb sum, count): W*H*4 floats, and for FP64 jobs
 * W*H*4 doubles (either pointer may be NULL; an FP64 job's float image is
 * its display image sum / count). */
int myrt_batch_read(myrt_batch* batch, uint32_t job, float* rgba, double* rgba64);
int myrt_batch_reset(myrt_batch* batch);
int myrt_batch_get_info(myrt_batch* batch, myrt_batch_info* info);
/* Cumulative camera / extension / shadow ray counts of the batch's frames
 * (the batch's own wavefront; the scene contexts' counters are not touched). */
int myrt_batch_get_stats(myrt_batch* batch, myrt_render_stats* out);
int myrt_batch_destroy(myrt_batch* batch);

/* ---- learned path guiding (MYRT_SHADE_GUIDED) ----------------------------------
 * A 4-layer, 64-wide MLP (BF16 weights, FP32 accumulation on the tensor
 * cores) maps the shading point's frequency-encoded position, shading normal
 * and view direction to a mixture of 8 von Mises-Fisher lobes. The shade pass
 * samples it with probability `fraction` (one-sample MIS with the BSDF); after
 * every wave the network trains on that wave's radiance samples with Adam. No
 * counterpart in the reference. */
typedef struct myrt_guide_params {
  float fraction;         /* probability of sampling the guide (0.5) */
  float learning_rate;    /* Adam step size (1e-2) */
  uint32_t train_steps;   /* Adam steps after each wave (16) */
  uint32_t batch;         /* samples per step, multiple of 128 (16384) */
  uint32_t train;         /* 0: inference only, the network stays as it is */
  uint32_t warmup_waves;  /* waves sampled from the BSDF alone while the network learns (1) */
  uint32_t seed;          /* initialisation seed; a change re-initialises the network */
  float weight_clamp;     /* training weights are clamped to this multiple of their mean (10; 0: off) */
  uint32_t target;        /* 0: learn L_i * f * cos (product), 1: learn L_i (incident radiance) */
  uint32_t reserved;
} myrt_guide_params;
int myrt_guide_configure(myrt_ctx* ctx, const myrt_guide_params* params);
int myrt_guide_get_config(myrt_ctx* ctx, myrt_guide_params* params);
/* Re-initialises weights and Adam state (a scene upload does this too). */
int myrt_guide_reset(myrt_ctx* ctx);
/* FP32 master parameters: weights [4][64 out][64 in], then biases [4][64]
 * (16640 floats). Setting them also refreshes the BF16 copy. */
#define MYRT_GUIDE_PARAM_COUNT 16640
int myrt_guide_get_params(myrt_ctx* ctx, float* params);
int myrt_guide_set_params(myrt_ctx* ctx, const float* params);
/* Mixture for n host points (12 floats each: position, 1, shading normal, 0,
 * view direction, 0), positions normalised by the uploaded scene's bounds.
 * lobes: 64 floats per point: 8 x (mu xyz, kappa), then 8 x (weight,
 * kappa / (2 pi (1 - exp(-2 kappa))), cumulative weight, 1 for lobe 0). */
int myrt_guide_eval(myrt_ctx* ctx, const float* points, uint32_t n, float* lobes);
/* Gradient of sum_i -w_i log q(d_i | x_i) w.r.t. the parameters for n host
 * samples (16 floats each: position, w, shading normal, 0, view direction, 0,
 * d, 0), computed by the training kernel; loss (may be NULL) gets the sum. */
int myrt_guide_gradients(myrt_ctx* ctx, const float* samples, uint32_t n, float* grads, float* loss);
/* `steps` Adam steps on host samples (layout as above), batch = min(n, batch). */
int myrt_guide_train(myrt_ctx* ctx, const float* samples, uint32_t n, uint32_t steps, float* loss_per_step);
typedef struct myrt_guide_stats {
  uint64_t adam_steps;
  uint64_t waves;
  uint64_t waves_trained;
  uint32_t last_samples;  /* training samples the last wave produced */
  float last_loss;        /* loss sum of the last wave's steps */
  float last_weight_sum;
  uint32_t pad;
} myrt_guide_stats;
int myrt_guide_get_stats(myrt_ctx* ctx, myrt_guide_stats* out);

/* The FP64 accumulation (rgb sum, sample count) of a physical / guided render
 * made with accum_fp64 = 1, W*H*4 doubles. */
int myrt_read_accumulation_f64(myrt_ctx* ctx, double* rgba_sum);
/* Device pointers of the two images (valid until the next resolution change). */
int myrt_render_buffers(myrt_ctx* ctx, void** accum, void** display);
/* Size of the context's render images (0 x 0 before the first render): the
 * host arrays of myrt_read_accumulation(_f64) hold width * height * 4 values. */
int myrt_render_size(myrt_ctx* ctx, uint32_t* width, uint32_t* height);
/* Device pointer of the FP64 accumulation (W*H*4 doubles: rgb sum, sample
 * count) of a render made with accum_fp64 = 1. */
int myrt_render_buffer_f64(myrt_ctx* ctx, void** accum64);
/* Starts a new accumulation whose samples are numbered from first_sample: the
 * next myrt_render overwrites the images, and in the physical and guided modes
 * (whose results depend only on pixel, sample index and seed) renders sample
 * indices first_sample, first_sample + 1, ... No counterpart in the reference:
 * it lets N processes render disjoint slices of one image's samples and sum
 * their FP64 accumulations (myrt_b200/multigpu.py). In the reference mode the
 * accumulation restarts at sample 0. */
int myrt_begin_samples(myrt_ctx* ctx, uint32_t first_sample);
/* sequential_pathtracer::invalidate_counter / sample_count / the m_rng seed. */
int myrt_reset_accumulation(myrt_ctx* ctx);
int myrt_sample_count(myrt_ctx* ctx, uint32_t* count);
int myrt_set_seed(myrt_ctx* ctx, uint32_t seed);

/* Render without any device allocation. No counterpart in the reference: it
 * exists for callers that cannot call cudaMalloc -- hosts that give all device
 * memory to their own allocator or fixed budgets up front, and frame loops that
 * must not pay cudaMalloc's implicit device synchronisation. It runs the same
 * frames as myrt_render (same kernels, same host random stream of the context)
 * but keeps every scratch buffer in one static device array inside the library
 * (15.7 MB, held by every device that loads the library until the process
 * exits) and writes into CALLER-PROVIDED device images: accum_rgba (rgb sum,
 * count in a; read as well as written when sample_index > 0) and display_rgba,
 * width * height * 4 floats each. The caller tracks sample_index (0 starts a new
 * accumulation); the context's own images and sample counter are not touched.
 * Depth of field, the bokeh mask, albedo textures and the cube map apply as in
 * myrt_render; only MYRT_SHADE_REFERENCE is supported (else
 * MYRT_ERR_UNSUPPORTED). Limits: width * height <= 65536 and
 * frames * (2 * num_bounces + 3) <= 256, else MYRT_ERR_INVALID_ARGUMENT. The
 * first call on a device looks up the array's device address
 * (cudaGetSymbolAddress). The call must not be captured into a CUDA graph: each
 * call draws fresh pass randomness from the context's host stream and uploads
 * it with copies from a stack buffer, which a graph would replay frozen. All
 * calls share the array: calls that overlap on the GPU (other streams, other
 * threads) race and must be serialised by the caller. The call makes the
 * context's device current while it runs and then restores the caller's.
 * Asynchronous on `stream` (NULL = the ctx stream); a caller stream first waits
 * for the work already queued on the context's stream (scene and transform
 * updates). */
int myrt_render_noalloc(myrt_ctx* ctx, const myrt_camera* camera, const myrt_render_params* params,
    uint32_t sample_index, float* accum_rgba, float* display_rgba, void* stream);

/* The GLSL built-ins as the library computes them in the reference shading
 * (pt_generate / pt_color / pbr.glsl: sin, cos, atan, pow), the forward
 * preview's resolve and the post-processing passes (exp, pow). No counterpart
 * in the reference, whose GL driver supplies its own (GLSL leaves their
 * precision to the implementation). They are defined in
 * myrt_b200/csrc/glmath.hpp with IEEE-exact operations only, so a host build of
 * that header (-ffp-contract=off) gives the same bits; this call evaluates them
 * on the context's device: out[i] = fn(x[i]) or pow(x[i], y[i]). Host arrays
 * of n floats (y only for MYRT_GLSL_POW). Accuracy against the exact values:
 * sin / cos <= 2 ulp for |x| < 1e5, atan <= 2.5 ulp, exp <= 1 ulp,
 * pow <= 4.5 ulp. Synchronous. */
typedef enum myrt_glsl_fn {
  MYRT_GLSL_SIN = 0,
  MYRT_GLSL_COS = 1,
  MYRT_GLSL_ATAN = 2,
  MYRT_GLSL_EXP = 3,
  MYRT_GLSL_POW = 4
} myrt_glsl_fn;
int myrt_glsl_builtins(myrt_ctx* ctx, int fn, const float* x, const float* y, uint32_t n, float* out);

/* Waits for the context's work and returns MYRT_ERR_DEVICE_ABORT if a kernel
 * stopped at a limit since the last call (the error word is then cleared). */
int myrt_sync(myrt_ctx* ctx);

/* ---- post-processing (src/pathtracer/post_process.cpp, src/pt/pp_*.comp) ----
 * One pass over device images (float RGBA, row-major). Every pass rounds its
 * output to half precision, as the reference's RGBA16F targets do; texture
 * reads follow the reference sampler (bilinear, mirrored repeat). Bloom, blur2d
 * and the per-frame chain of main.cpp:840-875 are sequences of these passes
 * (myrt_b200/post.py). */
typedef enum myrt_pp_op {
  MYRT_PP_DENOISE = 0, /* pp_denoise.comp (denoise): p[0] exponent (spatial sigma), p[1] strength (range sigma) */
  MYRT_PP_BLUR = 1,    /* pp_blur.comp (blur): i[0] direction (0 = x, 1 = y), p[0] step */
  MYRT_PP_CUTOFF = 2,  /* pp_cutoff.comp (cutoff): p[0..3] value, i[0] leave_above */
  MYRT_PP_ADD = 3,     /* pp_add.comp (add): p[0] factor; the overlay image is sampled */
  MYRT_PP_TONEMAP = 4, /* pp_tonemap.comp / pp_tonemap_filmic.cl: filmic curve; i[0] = 1 sets alpha to 1 */
  MYRT_PP_FXAA = 5,    /* pp_fxaa.comp (fxaa) */
  MYRT_PP_SCALE = 6    /* linear_scale (post_process.cpp:112-127): bilinear resample to the output size */
} myrt_pp_op;
typedef struct myrt_pp_pass {
  int32_t op; /* myrt_pp_op */
  int32_t i[3];
  float p[4];
} myrt_pp_pass;
typedef struct myrt_image {
  float* rgba; /* device memory, width * height * 4 floats */
  uint32_t width, height;
} myrt_image;
/* Runs one pass on `stream` (null: the context's stream). The output must
 * have the input's size except for MYRT_PP_SCALE; `overlay` is used by
 * MYRT_PP_ADD only. Input and output must not overlap. */
int myrt_post_pass(myrt_ctx* ctx, const myrt_pp_pass* pass, const myrt_image* input, const myrt_image* overlay,
    const myrt_image* output, void* stream);

/* ---- forward (raster preview) renderer (src/pathtracer/forward_renderer.cpp,
 * src/pt/fwd_generate.comp, src/pt/forward/*) ----
 * forward_renderer::run on the uploaded scene: a G-buffer pass (world
 * position, uv, normal + material at RGBA16F), a shadow pass from a fixed
 * orthographic light (world positions at RGBA32F) and the resolve pass
 * (9-tap shadow test, the material's diffuse lobe towards the light and the
 * normal, 8-sample screen-space ambient occlusion, random brightness), into an
 * RGBA16F result. Rasterisation follows GL's rules: pixel centres at +0.5,
 * perspective-correct attributes, clipping to -w <= z <= w, a 24-bit depth
 * buffer with GL_LESS in draw order (triangles of drawable 0 first), no
 * culling. Rows are GL window rows (row 0 at the bottom). */
typedef struct myrt_forward_params {
  uint32_t width, height;
  float view[16];         /* set_view_matrix, column-major */
  float projection[16];   /* set_projection_matrix, column-major */
  uint32_t random_seed;   /* the resolve pass's random_seed uniform (run draws it from its generator) */
  uint32_t shadow_size;   /* shadow map edge in texels; 0 = 2048 (the reference's) */
  int32_t custom_shadow;  /* 0: the reference's light camera (forward_renderer.cpp:306-310); 1: the two below */
  float shadow_view[16];
  float shadow_projection[16];
} myrt_forward_params;
/* Runs the three passes on the context's stream. */
int myrt_forward_run(myrt_ctx* ctx, const myrt_forward_params* params);
/* Host copies of the last run (NULL skips one): result RGBA16F as half bits
 * (height * width * 4), G-buffer layers position / uv / normal + material as
 * half bits (3 * height * width * 4), shadow map RGBA32F (shadow_size^2 * 4),
 * visibility keys (height * width: 24-bit depth << 32 | triangle index; all
 * ones where nothing was drawn). width, height and shadow_size are the sizes
 * the host arrays were made for and must equal the last run's (shadow_size 0
 * = 2048), else MYRT_ERR_INVALID_ARGUMENT. Waits for the stream. */
int myrt_forward_read(myrt_ctx* ctx, uint32_t width, uint32_t height, uint32_t shadow_size, uint16_t* result,
    uint16_t* gbuffer, float* shadow_map, uint64_t* visibility);
/* Device pointers of the same four images (valid until the next run with
 * another size or context destruction). */
int myrt_forward_buffers(myrt_ctx* ctx, void** result, void** gbuffer, void** shadow_map, void** visibility);
/* The light camera the reference uses: view = inverse(rotation(axis (1,0,0),
 * -45 degrees) * translation(0, 0, 15)), projection = orthographic(-20, 20,
 * 20, -20, 0.01, 1000), column-major. */
int myrt_forward_default_shadow(float* view, float* projection);

#ifdef __cplusplus
}
#endif

#endif /* MYRT_CUDA_H */
