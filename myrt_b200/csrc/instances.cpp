// Host construction of the two-level (instanced) structure, instances.hpp.
#include "instances.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <stdexcept>
#include <tuple>

namespace myrt_b200 {

bool build_object_trees(float const* vertices, std::size_t vertex_count, std::uint32_t const* indices,
    std::size_t index_count, myrt_drawable const* drawables, std::size_t n_drawables, two_level& out,
    std::string& err) {
  auto const t0 = std::chrono::steady_clock::now();
  out = two_level{};
  std::map<std::tuple<std::uint32_t, std::uint32_t, std::uint32_t>, std::uint32_t> known;
  std::uint64_t prim = 0;
  for (std::size_t di = 0; di < n_drawables; ++di) {
    myrt_drawable const& d = drawables[di];
    if (d.index_count % 3 != 0 || std::size_t(d.indices_base_index) + d.index_count > index_count) {
      err = "drawable index range outside the index buffer";
      return false;
    }
    auto const key = std::make_tuple(d.indices_base_index, d.points_base_index, d.index_count);
    auto it = known.find(key);
    if (it == known.end()) {
      geometry_tree g;
      g.indices_base = d.indices_base_index;
      g.points_base = d.points_base_index;
      g.index_count = d.index_count;
      std::size_t const n = d.index_count / 3;
      if (n > 0) {
        std::vector<float> pos(9 * n);
        for (std::size_t t = 0; t < n; ++t)
          for (int k = 0; k < 3; ++k) {
            std::size_t const vi = std::size_t(d.points_base_index) + indices[d.indices_base_index + 3 * t + k];
            if (vi >= vertex_count) {
              err = "vertex index out of range";
              return false;
            }
            std::memcpy(&pos[9 * t + 3 * k], vertices + 4 * vi, 12);
          }
        bvh8 tree;
        try {
          tree = build_bvh8(pos.data(), n, nullptr, bvh8_build_options{});
        } catch (std::exception const& e) {
          err = std::string("bvh build: ") + e.what();
          return false;
        }
        auto const node_off = std::uint32_t(out.blas_nodes.size());
        auto const tri_off = std::uint32_t(out.blas_tris.size());
        for (bvh8_node nd : tree.nodes) {
          nd.child_base += node_off;
          nd.tri_base += tri_off;
          out.blas_nodes.push_back(nd);
        }
        out.blas_tris.insert(out.blas_tris.end(), tree.triangles.begin(), tree.triangles.end());
        g.root = node_off;
        for (int a = 0; a < 3; ++a) {
          g.lo[a] = tree.scene_lo[a];
          g.hi[a] = tree.scene_hi[a];
        }
        g.depth = tree.stats.wide_depth;
        g.empty = false;
        out.blas_depth = std::max(out.blas_depth, g.depth);
      }
      it = known.emplace(key, std::uint32_t(out.geometries.size())).first;
      out.geometries.push_back(g);
    }
    out.drawable_geometry.push_back(it->second);
    out.prim_base.push_back(std::uint32_t(prim));
    prim += d.index_count / 3;
  }
  if (prim >= (std::uint64_t(1) << 31)) {
    err = "too many triangles";
    return false;
  }
  out.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return true;
}

top_level build_top_level(two_level const& objects, myrt_drawable const* drawables, std::size_t n_drawables) {
  top_level out;
  // world boxes as (lo, hi, centre) "triangles": their box is the instance box
  // and their centroid its centre
  std::vector<float> boxes;
  std::vector<std::uint32_t> ids;
  boxes.reserve(9 * n_drawables);
  for (std::size_t di = 0; di < n_drawables; ++di) {
    geometry_tree const& g = objects.geometries[objects.drawable_geometry[di]];
    if (g.empty) continue;
    float const* m = drawables[di].transformation;  // column-major
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int c = 0; c < 8; ++c) {
      double const p[3] = {(c & 1) ? g.hi[0] : g.lo[0], (c & 2) ? g.hi[1] : g.lo[1], (c & 4) ? g.hi[2] : g.lo[2]};
      for (int r = 0; r < 3; ++r) {
        double const w = double(m[r]) * p[0] + double(m[4 + r]) * p[1] + double(m[8 + r]) * p[2] + double(m[12 + r]);
        lo[r] = std::min(lo[r], w);
        hi[r] = std::max(hi[r], w);
      }
    }
    // padding beyond the builder's 1e-5: the object-space ray of an instance
    // carries rounding relative to the coordinates' magnitude
    double mag = 0.0;
    for (int r = 0; r < 3; ++r) mag = std::max({mag, std::fabs(lo[r]), std::fabs(hi[r])});
    double const pad = 1e-5 + mag * 0x1p-18;
    float b[9];
    for (int r = 0; r < 3; ++r) {
      b[r] = std::nextafter(float(lo[r] - pad), -INFINITY);
      b[3 + r] = std::nextafter(float(hi[r] + pad), INFINITY);
      b[6 + r] = 0.5f * (b[r] + b[3 + r]);
    }
    boxes.insert(boxes.end(), b, b + 9);
    ids.push_back(std::uint32_t(di));
  }
  if (ids.empty()) return out;
  bvh8 tree = build_bvh8(boxes.data(), ids.size(), ids.data(), bvh8_build_options{});
  out.nodes = std::move(tree.nodes);
  out.depth = tree.stats.wide_depth;
  out.records.resize(tree.triangles.size());
  for (std::size_t k = 0; k < tree.triangles.size(); ++k) {
    std::uint32_t const di = tree.triangles[k].prim;
    myrt_drawable const& d = drawables[di];
    instance_record& rec = out.records[k];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 4; ++c) rec.row[r][c] = d.inverse_transformation[4 * c + r];
    rec.root = std::int32_t(objects.geometries[objects.drawable_geometry[di]].root);
    rec.prim_base = std::int32_t(objects.prim_base[di]);
    rec.drawable = std::int32_t(di);
    rec.pad = 0;
  }
  return out;
}

}  // namespace myrt_b200
