// C entry points around the reference's shader helper code, compiled as C++.
//
// TEST INFRASTRUCTURE ONLY. oracle/build_ref.py rewrites the reference's GLSL
// helper files mechanically (see its docstring) into oracle/_ref/glsl/ and this
// file includes them inside namespace glsl, on top of oracle/glsl_compat.hpp.
// What runs here is therefore the reference's own source for:
//   src/pt/random.glsl:14-85        (Wang hash, xorshift32, prime cycle)
//   src/pt/intersect.glsl:3-39      (Moller-Trumbore, ray/sphere)
//   src/pt/bvh.glsl:31-55           (slab test, node accessors)
//   src/pt/bvh.impl.glsl:8-72       (stackless bit-trail traversal)
//   src/pt/pt_trace.comp:229-309    (closest / any-hit triangle visitor and the
//                                    instance visitor visit_object_aabb)
//   src/pt/ggx.glsl, pbr.glsl, color.glsl, transform.glsl
//   src/pt/material_new.glsl        (after the same text substitution that
//                                    material_registry::push_type applies,
//                                    src/material.hpp:18-37)
#include "glsl_compat.hpp"

#include <cstdint>
#include <thread>
#include <vector>

#undef INT_MAX

namespace glsl {
#include "transform.glsl"
#include "random.glsl"
#include "intersect.glsl"
#include "pbr.glsl"

// Material record of the reference app's PBR type (src/main.cpp:447-464):
// albedo vec4unorm8 (1 float), ior, roughness, metallic, transmission, albedo
// texture uvec2 (2 floats) = 7 floats. The loader mirrors what
// generate_object_loaders emits for it (src/types.hpp:46-100; vec4unorm8 is
// loaded as unpackUnorm4x8(floatBitsToUint(x)), types.hpp:66).
struct color_t {
  vec4 value;
};
struct material {
  color_t albedo;
  float ior;
  float roughness;
  float metallic;
  float transmission;
  uvec2 albedo_texture;
};
struct sampler2D {
  explicit sampler2D(uvec2) {}
};
inline vec4 texture(sampler2D const&, vec2 const&) { return vec4(1.f); }

#include "material_new.glsl"

thread_local float const* g_material_data = nullptr;
inline material material_load_(uint buf) {
  material m;
  m.albedo.value = unpackUnorm4x8(floatBitsToUint(g_material_data[buf + 0]));
  m.ior = g_material_data[buf + 1];
  m.roughness = g_material_data[buf + 2];
  m.metallic = g_material_data[buf + 3];
  m.transmission = g_material_data[buf + 4];
  m.albedo_texture = uvec2(floatBitsToUint(g_material_data[buf + 5]), floatBitsToUint(g_material_data[buf + 6]));
  return m;
}
// material.hpp:26-27: "void {0}_load_mat_(uint buf) { {0}_instance_ = {0}_load_(buf); {0}_open_(); }"
inline void material_load_mat_(uint buf) {
  material_instance_ = material_load_(buf);
  material_open_();
}

// Mesh buffers of pt_trace.comp:82-90, bound per call (read-only, shared).
#define MYRT_POINT_TYPE vec3
#define MYRT_INDEX_TYPE uint
#define MYRT_BVH_NODE_PADDING_BYTES 3
#define MYRT_BVH_NODE_TYPE_SHIFT 31
#define MYRT_BVH_NODE_STRUCT bvh_node_t
#include "bvh.glsl"
static_assert(sizeof(bvh_node_t) == 48, "std430 node layout");

bvh_node_t const* bvh_nodes = nullptr;
uint const* bvh_indices = nullptr;
uint const* indices = nullptr;
vec4 const* points = nullptr;
// pt_trace.comp:34-47, :91-92: drawables and the tree over their world boxes
#include "pt_trace_geometry.glsl"
static_assert(sizeof(drawable_geometry_t) == 160, "std430 drawable layout");
drawable_geometry_t const* geometries = nullptr;
bvh_node_t const* global_bvh_nodes = nullptr;
uint const* global_bvh_indices = nullptr;

#define MYRT_BVH_NODES_BUFFER bvh_nodes
#define MYRT_BVH_INDICES_BUFFER bvh_indices
#define MYRT_BVH_TRAVERSE bvh_traverse
#define MYRT_BVH_VISIT_PRIMITIVE visit_triangle
#include "bvh.impl.glsl"
#undef MYRT_BVH_VISIT_PRIMITIVE
#undef MYRT_BVH_TRAVERSE
#undef MYRT_BVH_INDICES_BUFFER
#undef MYRT_BVH_NODES_BUFFER
#include "pt_trace_visitor.glsl"
// the second instantiation, as pt_trace.comp:108-116
#define MYRT_BVH_NODES_BUFFER global_bvh_nodes
#define MYRT_BVH_INDICES_BUFFER global_bvh_indices
#define MYRT_BVH_TRAVERSE bvh_traverse_global
#define MYRT_BVH_VISIT_PRIMITIVE visit_object_aabb
#include "bvh.impl.glsl"
#undef MYRT_BVH_VISIT_PRIMITIVE
#undef MYRT_BVH_TRAVERSE
#undef MYRT_BVH_INDICES_BUFFER
#undef MYRT_BVH_NODES_BUFFER

// ---- SDF: raymarch.glsl and the instruction snippets of sdf.hpp ---------------
// Records of pt_trace.comp:49-66.
struct drawable_sdf_t {
  mat4 transformation;
  mat4 inverse_transformation;
  int sdf_index;
  int pad[3];
};
struct hit_t {
  vec3 position;
  float t;
  vec3 normal;
  vec2 uv;
  bool hits;
  int material_index;
  int hits_light;
};
drawable_sdf_t const* sdf_drawables = nullptr;
float const* sdf_buffer = nullptr;
int sdf_marching_steps = 0;
#define MYRT_INJECT_SDF_MAP_CODE_HERE float map(vec3 p, _MT& _mt);
#include "raymarch.glsl"
#include "sdf_snippets.inc"

// The map() the reference's code generator would emit for a tree
// (sdf.cpp:122-345, map dispatch sdf.hpp:202 / sdf.cpp:400-407), written as an
// interpreter over this project's flat post-order program: modifier
// instructions transform the position of the next primitive (innermost
// first), primitives push (distance, material), operators pop two and push one;
// every node starts from the caller's material (`_MT _mt<node> = _mt`), the
// result is the last node's, scaled by the product of the modifiers'
// multipliers. Parameters are read from sdf_buffer exactly as the generated
// loaders do (float: the block, int: int(block), vec3: three blocks).
struct sdf_instr_ref {
  int op;
  int param;
};
struct sdf_program_ref {
  int first;
  int count;
};
sdf_instr_ref const* sdf_instrs = nullptr;
sdf_program_ref const* sdf_programs = nullptr;

float map(vec3 p, _MT& _mt) {
  sdf_program_ref const pr = sdf_programs[sdf_index_current];
  float dist[64];
  _MT mats[64];
  int sp = 0;
  vec3 pos = p;
  float mul = 1.f;
  for (int k = 0; k < pr.count; ++k) {
    sdf_instr_ref const in = sdf_instrs[pr.first + k];
    int const o = in.param;
    _MT m = _mt;
    switch (in.op) {
      case 32: {
        float jm = 1.f;
        pos = sdf_translate(pos, jm, vec3(_G(o), _G(o + 1), _G(o + 2)));
        mul = mul * jm;
        continue;
      }
      case 33: {
        float jm = 1.f;
        pos = sdf_mirror_axis(pos, jm, int(_G(o)));
        mul = mul * jm;
        continue;
      }
      case 1: dist[sp] = sdf_sphere(pos, m, _G(o), int(_G(o + 1))); break;
      case 2: dist[sp] = sdf_box(pos, m, vec3(_G(o), _G(o + 1), _G(o + 2)), int(_G(o + 3))); break;
      case 3: dist[sp] = sdf_torus(pos, m, _G(o), _G(o + 1), int(_G(o + 2))); break;
      case 4: dist[sp] = sdf_vertical_capsule(pos, m, _G(o), _G(o + 1), int(_G(o + 2))); break;
      case 5: dist[sp] = sdf_menger_fractal(pos, m, int(_G(o))); break;
      default: {
        float const b = dist[sp - 1], a = dist[sp - 2];
        _MT const mb = mats[sp - 1], ma = mats[sp - 2];
        sp -= 2;
        if (in.op == 16) dist[sp] = sdf_hard_union(a, b, ma, mb, m);
        else if (in.op == 17) dist[sp] = sdf_hard_subtraction(a, b, ma, mb, m);
        else if (in.op == 18) dist[sp] = sdf_hard_intersection(a, b, ma, mb, m);
        else dist[sp] = sdf_smooth_union(a, b, ma, mb, m, _G(o));
        break;
      }
    }
    mats[sp] = m;
    ++sp;
    pos = p;
  }
  _mt = mats[sp - 1];
  return mul * dist[sp - 1];
}
}  // namespace glsl

using namespace glsl;

extern "C" {

std::uint32_t ref_glsl_wang_hash(std::uint32_t a) { return random_wang_hash(a); }

// random_init(tex, pixel, seed) followed by n random_next() draws.
void ref_glsl_random_stream(float const* tex, int tex_size, int px, int py, int seed, int n, float* out,
    std::uint32_t* state_after_init) {
  sampler1D s{tex, tex_size};
  random_init(s, ivec2(px, py), seed);
  if (state_after_init) state_after_init[0] = random_state.rng_state;
  for (int i = 0; i < n; ++i) out[i] = random_next();
}

// random_value(seed[i]) from a given xorshift state.
void ref_glsl_random_values(std::uint32_t state, int const* seeds, int n, float* out, std::uint32_t* state_out) {
  random_state.rng_state = state;
  random_state.current_prime = 0;
  for (int i = 0; i < n; ++i) out[i] = random_value(seeds[i]);
  if (state_out) *state_out = random_state.rng_state;
}

int ref_glsl_intersect_triangle(float const* o, float const* d, float const* tri, float* t, float* bary) {
  float tt = 0.f;
  vec2 b(0.f, 0.f);
  bool const h =
      intersect_triangle(vec3(o[0], o[1], o[2]), vec3(d[0], d[1], d[2]), vec3(tri[0], tri[1], tri[2]),
          vec3(tri[3], tri[4], tri[5]), vec3(tri[6], tri[7], tri[8]), tt, b);
  *t = tt;
  bary[0] = b.x;
  bary[1] = b.y;
  return h ? 1 : 0;
}

float ref_glsl_intersect_sphere(float const* r0, float const* rd, float const* s0, float sr) {
  return intersect_sphere(vec3(r0[0], r0[1], r0[2]), vec3(rd[0], rd[1], rd[2]), vec3(s0[0], s0[1], s0[2]), sr);
}

void ref_glsl_transform_local_to_world(float const* v, float const* n, float* out) {
  vec3 const r = transform_local_to_world(vec3(v[0], v[1], v[2]), vec3(n[0], n[1], n[2]));
  out[0] = r.x;
  out[1] = r.y;
  out[2] = r.z;
}

std::uint32_t ref_glsl_pack_unorm4x8(float const* v) { return packUnorm4x8(vec4(v[0], v[1], v[2], v[3])); }

// pt_color.comp:137-143 for one surface hit: open the material, draw the two
// material randoms, bounce, evaluate. Runs from the given RNG state and
// returns the state afterwards, so a caller can continue the stream.
//   mat7   : the 7-float material record
//   io_rng : [rng_state, current_prime] in/out
//   out_gen: sampled direction; out_refl/out_pdf: evaluate() result;
//   out_lobe: pbr_state (0 reflect, 1 transmit, 2 diffuse); out_resample.
void ref_glsl_material_bounce_eval(float const* mat7, std::uint32_t* io_rng, float const* towards_viewer,
    float const* normal, float* out_gen, float* out_refl, float* out_pdf, int* out_lobe, float* out_resample) {
  random_state.rng_state = io_rng[0];
  random_state.current_prime = int(io_rng[1]);
  g_material_data = mat7;
  material_load_mat_(0);
  // pt_color.comp:139, drawn left to right as GLSL evaluates arguments
  float const r0 = random_next();
  float const r1 = random_next();
  vec2 const material_randoms = vec2(r0, r1);
  vec3 const tv(towards_viewer[0], towards_viewer[1], towards_viewer[2]);
  vec3 const n(normal[0], normal[1], normal[2]);
  vec3 const generated = material_bounce_(material_randoms, tv, n);
  vec3 refl;
  float pdf = 0.f;
  material_evaluate_(vec3(0.f), vec2(0.f, 0.f), n, generated, tv, refl, pdf);
  out_gen[0] = generated.x;
  out_gen[1] = generated.y;
  out_gen[2] = generated.z;
  out_refl[0] = refl.x;
  out_refl[1] = refl.y;
  out_refl[2] = refl.z;
  *out_pdf = pdf;
  *out_lobe = pbr_state;
  *out_resample = resample_factor;
  io_rng[0] = random_state.rng_state;
  io_rng[1] = std::uint32_t(random_state.current_prime);
}

// evaluate() for a given direction with the lobe state a previous bounce left
// behind (pt_color.comp:168-177 evaluates the NEE direction this way).
void ref_glsl_material_eval(float const* mat7, int lobe, float resample, float const* towards_light,
    float const* towards_viewer, float const* normal, float* out_refl, float* out_pdf) {
  g_material_data = mat7;
  material_load_mat_(0);
  pbr_state = lobe;
  resample_factor = resample;
  after_sample = false;
  vec3 refl;
  float pdf = 0.f;
  material_evaluate_(vec3(0.f), vec2(0.f, 0.f), vec3(normal[0], normal[1], normal[2]),
      vec3(towards_light[0], towards_light[1], towards_light[2]),
      vec3(towards_viewer[0], towards_viewer[1], towards_viewer[2]), refl, pdf);
  out_refl[0] = refl.x;
  out_refl[1] = refl.y;
  out_refl[2] = refl.z;
  *out_pdf = pdf;
}

// bvh.impl.glsl traversal with the pt_trace.comp visitor, for one drawable with
// an identity transform (what visit_object_aabb, pt_trace.comp:284-309, does
// for it). nodes: 48-byte reference records; any_hit selects any_hit()'s mode
// (pt_trace.comp:311-329). Outputs prim (-1 = miss), t, u, v.
void ref_glsl_traverse(void const* nodes, std::uint32_t const* node_indices, std::uint32_t const* tri_indices,
    float const* points_xyzw, float const* rays, std::size_t n, int any_hit, std::int32_t* prim, float* t_out,
    float* u_out, float* v_out, int nthreads) {
  bvh_nodes = static_cast<bvh_node_t const*>(nodes);
  bvh_indices = node_indices;
  indices = tri_indices;
  points = reinterpret_cast<vec4 const*>(points_xyzw);
  auto work = [=](std::size_t begin, std::size_t end) {
    for (std::size_t r = begin; r < end; ++r) {
      float const* q = rays + 8 * r;
      float const maxt = q[7];
      traversal_init();
      traversal.any_hit = any_hit != 0;
      traversal.t = maxt;
      traversal.global_t = maxt;
      bool const h = bvh_traverse(0, 0, vec3(q[0], q[1], q[2]), vec3(q[4], q[5], q[6]), maxt);
      prim[r] = h ? std::int32_t(traversal.hit_index) : -1;
      t_out[r] = h ? traversal.t : maxt;
      u_out[r] = h ? traversal.barycentric.x : 0.f;
      v_out[r] = h ? traversal.barycentric.y : 0.f;
    }
  };
  if (nthreads <= 1) {
    work(0, n);
    return;
  }
  std::vector<std::thread> pool;
  std::size_t const per = (n + std::size_t(nthreads) - 1) / std::size_t(nthreads);
  for (int i = 0; i < nthreads; ++i) {
    std::size_t const b = std::size_t(i) * per, e = std::min(n, b + per);
    if (b < e) pool.emplace_back(work, b, e);
  }
  for (auto& th : pool) th.join();
}

// The instanced query of nearest_hit / any_hit (pt_trace.comp:311-341, mesh
// part): bvh_traverse_global over the tree of the drawables' world boxes, whose
// visitor visit_object_aabb moves the ray into each drawable's object space and
// walks its geometry tree (node / index bases from the drawable record). Outputs
// per ray the drawable (hit_geometry), the triangle's index in its geometry
// (global_hit_index), t and the barycentrics; geometry -1 = miss.
void ref_glsl_traverse_instanced(void const* global_nodes, std::uint32_t const* global_indices,
    void const* object_nodes, std::uint32_t const* object_indices, std::uint32_t const* tri_indices,
    float const* points_xyzw, void const* drawables, float const* rays, std::size_t n, int any_hit,
    std::int32_t* geometry, std::int32_t* prim, float* t_out, float* u_out, float* v_out, int nthreads) {
  global_bvh_nodes = static_cast<bvh_node_t const*>(global_nodes);
  global_bvh_indices = global_indices;
  bvh_nodes = static_cast<bvh_node_t const*>(object_nodes);
  bvh_indices = object_indices;
  indices = tri_indices;
  points = reinterpret_cast<vec4 const*>(points_xyzw);
  geometries = static_cast<drawable_geometry_t const*>(drawables);
  auto work = [=](std::size_t begin, std::size_t end) {
    for (std::size_t r = begin; r < end; ++r) {
      float const* q = rays + 8 * r;
      float const maxt = q[7];
      traversal_init();
      traversal.any_hit = any_hit != 0;
      traversal.t = maxt;
      traversal.global_t = maxt;
      bool const h = bvh_traverse_global(0, 0, vec3(q[0], q[1], q[2]), vec3(q[4], q[5], q[6]), maxt);
      geometry[r] = h ? std::int32_t(traversal.hit_geometry) : -1;
      prim[r] = h ? std::int32_t(traversal.global_hit_index) : -1;
      t_out[r] = h ? traversal.global_t : maxt;
      u_out[r] = h ? traversal.global_barycentric.x : 0.f;
      v_out[r] = h ? traversal.global_barycentric.y : 0.f;
    }
  };
  if (nthreads <= 1) {
    work(0, n);
    return;
  }
  std::vector<std::thread> pool;
  std::size_t const per = (n + std::size_t(nthreads) - 1) / std::size_t(nthreads);
  for (int i = 0; i < nthreads; ++i) {
    std::size_t const b = std::size_t(i) * per, e = std::min(n, b + per);
    if (b < e) pool.emplace_back(work, b, e);
  }
  for (auto& th : pool) th.join();
}

// SDF program tables: instrs (op, param) pairs, programs (first, count) pairs,
// params the sdf_data floats, drawables 36 floats each (two column-major
// mat4, then sdf_index as an int bit pattern and 3 pad words).
static void bind_sdf(int const* instrs, int const* programs, float const* params, float const* drawables) {
  sdf_instrs = reinterpret_cast<sdf_instr_ref const*>(instrs);
  sdf_programs = reinterpret_cast<sdf_program_ref const*>(programs);
  sdf_buffer = params;
  sdf_drawables = reinterpret_cast<drawable_sdf_t const*>(drawables);
}

// map() of program `prog` at n points (xyz each); with load_materials the
// material draws consume the random stream started from rng_states[i].
void ref_sdf_map(int const* instrs, int const* programs, float const* params, int prog, float const* pts, size_t n,
    int load_materials, std::uint32_t const* rng_states, float* out_d, int* out_mat) {
  static_assert(sizeof(drawable_sdf_t) == 144, "drawable_sdf_t layout");
  bind_sdf(instrs, programs, params, nullptr);
  for (size_t i = 0; i < n; ++i) {
    sdf_index_current = prog;
    g_do_load_materials = load_materials != 0;
    random_state.rng_state = rng_states ? rng_states[i] : 0u;
    random_state.current_prime = 0;
    _MT m;
    m.index = -1;
    out_d[i] = map(vec3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]), m);
    out_mat[i] = m.index;
  }
}

// The SDF part of nearest_hit (pt_trace.comp:342-352) or of any_hit (:321-326)
// over all drawables, for n rays (8 floats: o, tmin, d, tmax; tmax is the
// max_distance). Each ray's random stream starts at rng_states[i] (it feeds
// the material choice of smooth/hard operators). Outputs: hits, t, normal
// (3), uv (2), material.
void ref_sdf_trace(int const* instrs, int const* programs, float const* params, float const* drawables,
    int n_drawables, float const* rays, size_t n, int steps, float eps, int any_hit,
    std::uint32_t const* rng_states, int* out_hit, float* out_t, float* out_n, float* out_uv, int* out_mat) {
  bind_sdf(instrs, programs, params, drawables);
  sdf_marching_steps = steps;
  for (size_t i = 0; i < n; ++i) {
    float const* q = rays + 8 * i;
    vec3 const ro(q[0], q[1], q[2]), rd(q[4], q[5], q[6]);
    float const max_distance = q[7];
    random_state.rng_state = rng_states ? rng_states[i] : 0u;
    random_state.current_prime = 0;
    hit_t hit;
    hit.hits = false;
    hit.t = max_distance;
    hit.material_index = -1;
    hit.normal = vec3(0.f);
    hit.uv = vec2(0.f, 0.f);
    if (any_hit) {
      for (int d = 0; d < n_drawables; ++d) {
        sdf_current = d;
        if (march_sdf(ro, rd, max_distance, true, steps, eps).hits) {
          hit.hits = true;
          break;
        }
      }
    } else {
      for (int d = 0; d < n_drawables; ++d) {
        sdf_current = d;
        hit_t h = march_sdf(ro, rd, hit.hits ? hit.t : max_distance, false, steps, eps);
        if (h.hits && h.t < hit.t) hit = h;
      }
    }
    out_hit[i] = hit.hits ? 1 : 0;
    out_t[i] = hit.hits ? hit.t : max_distance;
    out_n[3 * i] = hit.normal.x, out_n[3 * i + 1] = hit.normal.y, out_n[3 * i + 2] = hit.normal.z;
    out_uv[2 * i] = hit.uv.x, out_uv[2 * i + 1] = hit.uv.y;
    out_mat[i] = hit.hits ? hit.material_index : -1;
  }
}

}  // extern "C"

// ---- the forward renderer's resolve pass: src/pt/forward/resolve.frag ----------------------
// build_ref.py rewrites the shader (resolve_to_cpp) into forward_resolve.inc; it runs
// here once per fragment over host G-buffer and shadow-map images, with the
// material dispatch material_registry::generate_code emits for the one PBR type
// (src/material.hpp:39-65) and what a GL fragment invocation provides:
//   * gl_FragCoord = (x + 0.5, y + 0.5) (pixel centres; only .xy is read);
//   * cam_pos = inverse(view)[3].xyz, as forward/resolve.vert:17 passes it;
//   * texelFetch on the G-buffer array returns 0 outside the image;
//   * texture(shadow_map, uv) samples the nearest texel of level 0 (the
//     sampler's default GL_NEAREST_MIPMAP_LINEAR minifies here: the shadow taps
//     jitter by texels from fragment to fragment);
//   * dFdx / dFdy: the shader computes them but never uses the result, so they
//     return 0;
//   * every per-invocation global (pbr_state, after_sample, resample_factor,
//     the material type) starts at its initial value for each fragment.
namespace glsl {

// The dispatch material_registry::generate_code emits for the one PBR type
// (src/material.hpp:39-65): open / evaluate / bounce over the current type.
thread_local uint cmattype = ~0u;
void open(uint type, uint buf) {
  cmattype = type;
  switch (type) {
    case 0: material_load_mat_(buf); break;
  }
}
void evaluate(vec3 p, vec2 uv, vec3 n, vec3 tl, vec3 tv, vec3& ref, float& pdf) {
  ref = vec3(0, 0, 0);
  pdf = 1;
  if (cmattype == ~0u) return;
  switch (cmattype) {
    case 0: material_evaluate_(p, uv, n, tl, tv, ref, pdf); break;
  }
}
vec3 bounce(vec2 rnd, vec3 tv, vec3 n) {
  switch (cmattype) {
    case 0: return material_bounce_(rnd, tv, n); break;
  }
  return vec3(0);
}
// every per-invocation global at its initial value
void reset_invocation() {
  pbr_state = -1;
  after_sample = false;
  resample_factor = 1.f;
  cmattype = ~0u;
}

namespace fwd {

struct ivec3 {
  int x, y, z;
  ivec3(ivec2 v, int c) : x(v.x), y(v.y), z(c) {}
  ivec3(vec2 v, int c) : x(int(v.x)), y(int(v.y)), z(c) {}
};
struct ivec3_size {
  ivec2 xy;
  int z;
};
struct sampler2DArray {
  float const* data = nullptr;  // layer-major RGBA floats
  int w = 0, h = 0, layers = 0;
};
inline vec4 texelFetch(sampler2DArray const& s, ivec3 p, int) {
  if (p.x < 0 || p.y < 0 || p.z < 0 || p.x >= s.w || p.y >= s.h || p.z >= s.layers) return vec4(0.f);
  float const* q = s.data + 4 * ((size_t(p.z) * s.h + p.y) * s.w + p.x);
  return vec4(q[0], q[1], q[2], q[3]);
}
inline ivec3_size textureSize(sampler2DArray const& s, int) { return {ivec2(s.w, s.h), s.layers}; }
struct sampler2D {
  float const* data = nullptr;  // RGBA floats, size x size
  int size = 0;
};
inline ivec2 textureSize(sampler2D const& s, int) { return ivec2(s.size, s.size); }
inline int nearest_texel(float u, int size) {
  float const f = std::floor(u * float(size));
  int const i = (f > -2147483648.f && f < 2147483648.f) ? int(f) : 0;
  return int(uint(i) % uint(size));  // GL_REPEAT
}
inline vec4 texture(sampler2D const& s, vec2 uv) {
  float const* q = s.data + 4 * (size_t(nearest_texel(uv.y, s.size)) * s.size + nearest_texel(uv.x, s.size));
  return vec4(q[0], q[1], q[2], q[3]);
}
inline vec3 dFdx(vec3 const&) { return vec3(0.f); }
inline vec3 dFdy(vec3 const&) { return vec3(0.f); }
inline uint to_uint(float f) {
  if (!(f > 0.f)) return 0u;
  if (f >= 4294967296.f) return 0xffffffffu;
  return uint(f);
}
vec4 gl_FragCoord;

#include "forward_resolve.inc"

}  // namespace fwd
}  // namespace glsl

extern "C" void ref_forward_resolve(int width, int height, float const* gbuf, float const* smap, int shadow_size,
    float const* view, float const* proj, float const* shadow_view, float const* shadow_proj, std::uint32_t seed,
    std::int32_t const* refs, float const* mdata, float* out) {
  namespace f = glsl::fwd;
  auto m4 = [](float const* p) {
    glsl::mat4 m;
    for (int i = 0; i < 16; ++i) m.c[i / 4][i % 4] = p[i];
    return m;
  };
  f::view = m4(view);
  f::proj = m4(proj);
  f::shadow_view = m4(shadow_view);
  f::shadow_proj = m4(shadow_proj);
  f::random_seed = seed;
  f::gbuffer = f::sampler2DArray{gbuf, width, height, 3};
  f::shadow_map = f::sampler2D{smap, shadow_size};
  f::materials = reinterpret_cast<f::material_reference_t const*>(refs);
  f::materials_data = mdata;
  glsl::g_material_data = mdata;
  f::cam_pos = glsl::inverse(f::view)[3].xyz;
  for (int y = 0; y < height; ++y)
    for (int x = 0; x < width; ++x) {
      f::gl_FragCoord = glsl::vec4(float(x) + 0.5f, float(y) + 0.5f, 0.f, 1.f);
      glsl::reset_invocation();
      f::color = glsl::vec4(0.f);
      f::resolve_main();
      float* o = out + 4 * (size_t(y) * width + x);
      o[0] = f::color.x, o[1] = f::color.y, o[2] = f::color.z, o[3] = f::color.w;
    }
}

// ---- the path tracer's generate and color passes: src/pt/pt_generate.comp, pt_color.comp -----
// build_ref.py rewrites them (pass_to_cpp) into pt_generate.inc / pt_color.inc;
// they run here once per invocation over host buffers and images with what a
// GL compute dispatch provides: gl_GlobalInvocationID; imageLoad / imageStore on
// RGBA32F images (outside the image: load 0, store dropped); the random texture
// as a sampler1D; the bokeh mask sampled at level 0 with GL_LINEAR and its wrap
// mode (weights summed ((w00 t00 + w10 t10) + w01 t01) + w11 t11); no cube map
// bound (textureSize 0: the sky gradient). pt_generate is dispatched over the
// image's pixels only: its `pt.x > image_size.x` test would let a column
// x = width through whose store lands on the next row's first slot (a race
// between invocations in GL); the images the tests use are multiples of the 8x8
// work group, where no such invocation exists.
namespace glsl {
struct image2D {
  float* data = nullptr;  // RGBA32F, row-major
  int w = 0, h = 0;
};
inline vec4 imageLoad(image2D const& im, ivec2 p) {
  if (p.x < 0 || p.y < 0 || p.x >= im.w || p.y >= im.h) return vec4(0.f);
  float const* q = im.data + 4 * (size_t(p.y) * im.w + p.x);
  return vec4(q[0], q[1], q[2], q[3]);
}
inline void imageStore(image2D& im, ivec2 p, vec4 v) {
  if (p.x < 0 || p.y < 0 || p.x >= im.w || p.y >= im.h) return;
  float* q = im.data + 4 * (size_t(p.y) * im.w + p.x);
  q[0] = v.x, q[1] = v.y, q[2] = v.z, q[3] = v.w;
}
struct samplerCube {
  int size = 0;
};
inline ivec2 textureSize(samplerCube const& c, int) { return ivec2(c.size, c.size); }
inline vec4 textureLod(samplerCube const&, vec3 const&, int) { return vec4(0.f); }

namespace cpass {
struct gid_t {
  uint x = 0, y = 0, z = 0;
};
gid_t gl_GlobalInvocationID;
#include "pt_color.inc"
}  // namespace cpass

namespace gpass {
struct gid_t {
  uint x = 0, y = 0, z = 0;
  uvec2 xy;
};
gid_t gl_GlobalInvocationID;
struct sampler2D {
  float const* data = nullptr;  // RGBA floats
  int w = 0, h = 0, wrap = 0;   // wrap 0 repeat, 1 clamp to edge, 2 mirrored repeat
};
inline ivec2 textureSize(sampler2D const& s, int) { return ivec2(s.w, s.h); }
inline int wrap_texel(int i, int size, int mode) {
  if (mode == 1) return i < 0 ? 0 : (i >= size ? size - 1 : i);
  if (mode == 2) {
    int m = i % (2 * size);
    if (m < 0) m += 2 * size;
    int const a = m - size;
    return (size - 1) - (a >= 0 ? a : -(1 + a));
  }
  int m = i % size;
  return m < 0 ? m + size : m;
}
inline vec4 textureLod(sampler2D const& s, vec2 uv, int) {
  float const u = uv.x * float(s.w) - 0.5f, v = uv.y * float(s.h) - 0.5f;
  float const fu = std::floor(u), fv = std::floor(v);
  float const a = u - fu, b = v - fv;
  int const i0 = int(fu), j0 = int(fv);
  int const x0 = wrap_texel(i0, s.w, s.wrap), x1 = wrap_texel(i0 + 1, s.w, s.wrap);
  int const y0 = wrap_texel(j0, s.h, s.wrap), y1 = wrap_texel(j0 + 1, s.h, s.wrap);
  float const w00 = (1.f - a) * (1.f - b), w10 = a * (1.f - b), w01 = (1.f - a) * b, w11 = a * b;
  float const* t00 = s.data + 4 * (size_t(y0) * s.w + x0);
  float const* t10 = s.data + 4 * (size_t(y0) * s.w + x1);
  float const* t01 = s.data + 4 * (size_t(y1) * s.w + x0);
  float const* t11 = s.data + 4 * (size_t(y1) * s.w + x1);
  float r[4];
  for (int c = 0; c < 4; ++c) r[c] = ((w00 * t00[c] + w10 * t10[c]) + w01 * t01[c]) + w11 * t11[c];
  return vec4(r[0], r[1], r[2], r[3]);
}
#include "bokeh.inc"
#include "pt_generate.inc"
}  // namespace gpass
}  // namespace glsl

extern "C" {

// pt_color.comp over n rays: gen (80-byte generate_output_t) and trace (64-byte
// trace_output_t) are updated in place, accum / display are the debug and
// output images (W x H RGBA32F).
void ref_pass_color(int n, void* gen, void* trace, float* accum, float* display, int width, int height,
    std::uint32_t sample_index, int force_write_color, int random_sample, float const* random_tex, int tex_size,
    std::int32_t const* refs, float const* mdata) {
  namespace c = glsl::cpass;
  c::generate_output = static_cast<c::generate_output_t*>(gen);
  c::trace_output = static_cast<c::trace_output_t*>(trace);
  c::num_elements = uint(n);
  c::materials = reinterpret_cast<c::material_reference_t*>(const_cast<std::int32_t*>(refs));
  c::materials_data = const_cast<float*>(mdata);
  glsl::g_material_data = mdata;
  c::debug_image = glsl::image2D{accum, width, height};
  c::output_image = glsl::image2D{display, width, height};
  c::random_texture = glsl::sampler1D{random_tex, tex_size};
  c::cubemap = glsl::samplerCube{0};
  c::sample_index = sample_index;
  c::force_write_color = force_write_color != 0;
  c::random_sample = random_sample;
  for (int id = 0; id < n; ++id) {
    c::gl_GlobalInvocationID = c::gid_t{uint(id), 0u, 0u};
    glsl::reset_invocation();
    c::pass_main();
  }
}

// pt_generate.comp over a width x height image into gen (width * height records).
void ref_pass_generate(int width, int height, float const* inv_view, float const* inv_proj, int random_seed,
    float const* random_tex, int tex_size, int dof, float lens_x, float lens_y, float focus, float const* bokeh,
    int bokeh_w, int bokeh_h, int bokeh_wrap, void* gen) {
  namespace g = glsl::gpass;
  auto m4 = [](float const* p) {
    glsl::mat4 m;
    for (int i = 0; i < 16; ++i) m.c[i / 4][i % 4] = p[i];
    return m;
  };
  g::inverse_camera_view = m4(inv_view);
  g::inverse_camera_projection = m4(inv_proj);
  g::dof_active = dof != 0;
  g::image_size = glsl::uvec2(uint(width), uint(height));
  g::lens_size = glsl::vec2(lens_x, lens_y);
  g::focus = focus;
  g::random_seed = random_seed;
  g::random_texture = glsl::sampler1D{random_tex, tex_size};
  g::bokeh_shape = g::sampler2D{bokeh, bokeh ? bokeh_w : 0, bokeh ? bokeh_h : 0, bokeh_wrap};
  g::generate_output = static_cast<g::generate_output_t*>(gen);
  for (int y = 0; y < height; ++y)
    for (int x = 0; x < width; ++x) {
      g::gl_GlobalInvocationID = g::gid_t{uint(x), uint(y), 0u, glsl::uvec2(uint(x), uint(y))};
      glsl::reset_invocation();
      g::pass_main();
    }
}

}  // extern "C"
