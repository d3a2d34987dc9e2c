// C entry points around the reference's own BVH build and CPU traversal,
// compiled from the reference sources into oracle/_ref by oracle/build_ref.py.
//
// TEST INFRASTRUCTURE ONLY (golden-vector generation and the CPU baseline).
//
//   ref_bvh_build      -> myrt::generate_triangle_bounds + myrt::bvh
//                         (bvh.cpp:136-161, :356-512), split = dont_split or
//                         split_aabbs exactly as scene::push_geometry uses it
//                         (scene.cpp:60-62).
//   ref_bvh_aabb       -> bvh::aabb (bvh.cpp:554-556), the box scene::enqueue
//                         transforms for the tree over the drawables.
//   ref_bvh_build_instances -> scene::enqueue's world boxes (scene.cpp:255-271:
//                         the 8 corners of the geometry's box under the
//                         drawable's transformation) and scene::prepare's
//                         bvh(m_drawable_aabbs, dont_split) (scene.cpp:336-340).
//   ref_pick_closest   -> scene::pick (scene.cpp:273-314) for one drawable with
//                         an identity transform: the reference generator
//                         traversal bvh::traverse (bvh.cpp:237-346) feeding
//                         ray_t::intersect (bvh.cpp:514-538); first strictly
//                         closer hit wins. Rows are spread over the reference's
//                         myrt::thread_pool (thread_pool.hpp:135-162).
#include <cstdint>
#include <cstring>
#include <future>
#include <limits>
#include <memory>
#include <vector>

#include "bvh.hpp"
#include "thread_pool.hpp"

namespace {
struct ref_bvh_handle {
  std::unique_ptr<myrt::bvh> bvh;
  std::vector<std::uint32_t> indices;
  std::vector<rnu::vec3> points;
};
}  // namespace

extern "C" {

void* ref_bvh_build(std::uint32_t const* indices, std::size_t n_indices, float const* points_xyz,
    std::size_t n_points, int split_mode) {
  auto* h = new ref_bvh_handle;
  h->indices.assign(indices, indices + n_indices);
  h->points.resize(n_points);
  for (std::size_t i = 0; i < n_points; ++i)
    h->points[i] = rnu::vec3(points_xyz[3 * i + 0], points_xyz[3 * i + 1], points_xyz[3 * i + 2]);
  auto const aabbs = myrt::generate_triangle_bounds(
      std::span<std::uint32_t const>(h->indices), std::span<rnu::vec3 const>(h->points));
  h->bvh = std::make_unique<myrt::bvh>(aabbs, split_mode ? myrt::split_aabbs : myrt::dont_split);
  return h;
}

void ref_bvh_free(void* p) { delete static_cast<ref_bvh_handle*>(p); }

void ref_bvh_aabb(void* p, float* lo_hi) {
  myrt::aabb_t const b = static_cast<ref_bvh_handle*>(p)->bvh->aabb();
  for (int k = 0; k < 3; ++k) {
    lo_hi[k] = b.min[k];
    lo_hi[3 + k] = b.max[k];
  }
}

// boxes: per drawable its geometry's box (min xyz, max xyz); transforms: the
// drawables' column-major 4x4 transformation. The corner products are summed
// left to right (the reference multiplies with rnu, which is not vendored).
void* ref_bvh_build_instances(float const* boxes, float const* transforms, std::size_t n) {
  auto* h = new ref_bvh_handle;
  std::vector<myrt::aabb_t> aabbs(n);
  for (std::size_t d = 0; d < n; ++d) {
    float const* b = boxes + 6 * d;
    float const* m = transforms + 16 * d;
    myrt::aabb_t transformed;
    for (unsigned i = 0; i < 8; ++i) {
      float const p[3] = {b[(i & 1) ? 3 : 0], b[(i & 2) ? 4 : 1], b[(i & 4) ? 5 : 2]};
      rnu::vec3 q;
      for (int r = 0; r < 3; ++r) q[r] = ((m[r] * p[0] + m[4 + r] * p[1]) + m[8 + r] * p[2]) + m[12 + r] * 1.0f;
      transformed.enclose(q);
    }
    aabbs[d] = transformed;
  }
  h->bvh = std::make_unique<myrt::bvh>(std::span<myrt::aabb_t const>(aabbs), myrt::dont_split);
  return h;
}

std::size_t ref_bvh_node_count(void* p) { return static_cast<ref_bvh_handle*>(p)->bvh->nodes().size(); }

std::size_t ref_bvh_index_count(void* p) {
  return static_cast<ref_bvh_handle*>(p)->bvh->reordered_indices().size();
}

// 48-byte aligned_node_t records (bvh.hpp:98-139), byte for byte.
void ref_bvh_nodes(void* p, void* out) {
  auto const& n = static_cast<ref_bvh_handle*>(p)->bvh->nodes();
  static_assert(sizeof(myrt::aligned_node_t) == 48);
  std::memcpy(out, n.data(), n.size() * sizeof(myrt::aligned_node_t));
}

void ref_bvh_indices(void* p, std::uint32_t* out) {
  auto const& r = static_cast<ref_bvh_handle*>(p)->bvh->reordered_indices();
  std::memcpy(out, r.data(), r.size() * sizeof(std::uint32_t));
}

// rays: 8 floats each (ox, oy, oz, tmin, dx, dy, dz, tmax); tmin is ignored by
// the reference path (it accepts t > 1e-23).
void ref_pick_closest(void* p, float const* rays, std::size_t n, std::int32_t* prim, float* t_out, float* u_out,
    float* v_out, int nthreads) {
  auto* h = static_cast<ref_bvh_handle*>(p);
  auto work = [h, rays, prim, t_out, u_out, v_out](std::size_t begin, std::size_t end) {
    for (std::size_t r = begin; r < end; ++r) {
      float const* q = rays + 8 * r;
      myrt::ray_t ray;
      ray.origin = rnu::vec3(q[0], q[1], q[2]);
      ray.direction = rnu::vec3(q[4], q[5], q[6]);
      ray.length = q[7] * norm(ray.direction);
      bool have = false;
      float best_t = 0.f;
      rnu::vec2 best_bary;
      std::uint32_t best = 0;
      for (auto const& tri : h->bvh->traverse(ray)) {
        rnu::vec2 bary;
        auto const& v0 = h->points[h->indices[3 * tri + 0]];
        auto const& v1 = h->points[h->indices[3 * tri + 1]];
        auto const& v2 = h->points[h->indices[3 * tri + 2]];
        auto const hit = ray.intersect(v0, v1, v2, bary);
        if (hit && (!have || *hit < best_t)) {
          have = true;
          best_t = *hit;
          best_bary = bary;
          best = tri;
        }
      }
      prim[r] = have ? std::int32_t(best) : -1;
      t_out[r] = have ? best_t : std::numeric_limits<float>::infinity();
      u_out[r] = have ? best_bary.x : 0.f;
      v_out[r] = have ? best_bary.y : 0.f;
    }
  };
  if (nthreads <= 1) {
    work(0, n);
    return;
  }
  myrt::thread_pool pool{unsigned(nthreads)};
  std::vector<std::future<void>> jobs;
  std::size_t const block = 1024;
  for (std::size_t b = 0; b < n; b += block) {
    std::size_t const e = std::min(n, b + block);
    jobs.push_back(pool.run_async([&work, b, e] { work(b, e); }));
  }
  for (auto& j : jobs) j.get();
}

}  // extern "C"
