// Two-level (instanced) acceleration structure: the reference's scene layout
// (src/pathtracer/scene.cpp:43-71, 255-271, 336-344; src/pt/pt_trace.comp:284-309)
// rebuilt with the 8-wide nodes of bvh8.hpp.
//
// * One object-space tree per distinct geometry (a drawable's index range and
//   vertex base), built once at upload. Its triangle records keep the
//   triangle's index inside the geometry; every tree's nodes and triangles are
//   relocated into one node array and one triangle array.
// * One tree over the drawables' world boxes (the 8 corners of the geometry's
//   object box under `transformation`, as scene::enqueue computes them), rebuilt
//   whenever transforms change. Its leaf slots index 64-byte instance records
//   in leaf order: rows 0-2 of `inverse_transformation` (row r = the r-th
//   components of the four columns, so that row . (x, y, z, w) is GLSL's
//   (inverse_transformation * vec4).r), then (root node of the geometry's tree,
//   first prim id of the drawable, drawable index, 0) as integers.
//
// A ray entering an instance is moved into object space exactly as
// visit_object_aabb does (direction not renormalised, so t keeps its meaning
// across instances) and walks the geometry's tree; prim ids are the library's
// global numbering (drawables in order, triangles in index order).
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/myrt_cuda.h"
#include "bvh8.hpp"

namespace myrt_b200 {

struct geometry_tree {
  std::uint32_t indices_base = 0, points_base = 0, index_count = 0;
  std::uint32_t root = 0;    // node index in the object-space node array
  float lo[3] = {0, 0, 0};   // object box (padded triangle boxes)
  float hi[3] = {0, 0, 0};
  int depth = 0;
  bool empty = true;
};

struct instance_record {
  float row[3][4];
  std::int32_t root;
  std::int32_t prim_base;
  std::int32_t drawable;
  std::int32_t pad;
};
static_assert(sizeof(instance_record) == 64, "instance_record must be 64 bytes");

struct two_level {
  std::vector<bvh8_node> blas_nodes;
  std::vector<bvh8_triangle> blas_tris;
  std::vector<geometry_tree> geometries;
  std::vector<std::uint32_t> drawable_geometry;  // per drawable: index into geometries
  std::vector<std::uint32_t> prim_base;          // per drawable: first global prim id
  int blas_depth = 0;                            // deepest object-space tree
  double seconds = 0.0;
};

struct top_level {
  std::vector<bvh8_node> nodes;
  std::vector<instance_record> records;  // leaf order
  int depth = 0;
};

// Object-space trees of every distinct geometry of the drawables. vertices:
// xyzw per vertex (w ignored). Returns false with `err` set on bad input.
bool build_object_trees(float const* vertices, std::size_t vertex_count, std::uint32_t const* indices,
    std::size_t index_count, myrt_drawable const* drawables, std::size_t n_drawables, two_level& out,
    std::string& err);

// The tree over the drawables' world boxes and their instance records.
// Drawables of an empty geometry are left out.
top_level build_top_level(two_level const& objects, myrt_drawable const* drawables, std::size_t n_drawables);

}  // namespace myrt_b200
