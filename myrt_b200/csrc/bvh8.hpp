// Host BVH construction for the device traversal kernels.
//
// Stage 1: binned-SAH binary tree (16 bins, split cost 7 / intersection cost 2,
// as the reference's bvh::compute_split_axis, src/pathtracer/bvh.cpp:43-116),
// over triangle boxes padded by 1e-5 with the triangle centroid as split key
// (generate_triangle_bounds, bvh.cpp:136-152), split down to single
// triangles (`binary_leaf`). O(n log n): no spatial splits, so no mid-vector
// inserts or whole-tree index fix-ups (the reference's bvh.cpp:460-488 path).
//
// Stage 2: collapse into an 8-wide tree with quantised child boxes (emitted level
// by level, each level's nodes planned and written in parallel): one 80-byte
// node = five 16-byte words (compressed wide BVH in the manner of Ylitie,
// Karras and Laine, HPG 2017). Children are placed in slots by ray octant so
// that visiting slot bits from high to low is roughly front to back.
//
// Node layout (bvh8_node, little endian):
//   w0: float px, py, pz; u8 ex, ey, ez (biased float exponents of the
//       per-axis scale 2^e); u8 imask (bit s = slot s is an internal node)
//   w1: u32 child_base (index of the first internal child; internal children
//       are contiguous in slot order); u32 tri_base (first triangle of the
//       node's leaf slots; leaf triangles are contiguous); u8 meta[8]
//       (leaf slot: bits 0-4 = triangle offset from tri_base, bits 5-7 =
//       triangle count 1..4; internal slot: 0x20 | slot; empty: 0)
//   w2..w4: u8 qlo_x[8], qlo_y[8], qlo_z[8], qhi_x[8], qhi_y[8], qhi_z[8]
// Child box = p + q * 2^e, rounded outwards when quantised.
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

namespace myrt_b200 {

struct bvh8_node {
  float px, py, pz;
  std::uint8_t e[3];
  std::uint8_t imask;
  std::uint32_t child_base;
  std::uint32_t tri_base;
  std::uint8_t meta[8];
  std::uint8_t qlo[3][8];
  std::uint8_t qhi[3][8];
};
static_assert(sizeof(bvh8_node) == 80, "bvh8_node must be 80 bytes");

// One triangle reference in leaf order, pre-gathered for the device: three
// float4 with v0.xyz + prim id bits, v1.xyz, v2.xyz (48 bytes).
struct bvh8_triangle {
  float v0[3];
  std::uint32_t prim;
  float v1[3];
  std::uint32_t pad1;
  float v2[3];
  std::uint32_t pad2;
};
static_assert(sizeof(bvh8_triangle) == 48, "bvh8_triangle must be 48 bytes");

struct bvh8_build_options {
  int max_leaf = 4;        // triangles per wide-node leaf slot
  int binary_leaf = 1;     // triangles per leaf of the binary tree (1..max_leaf); the collapse regroups
                           // them into slots of up to max_leaf
  float collapse_prim_cost = 0.8f;  // collapse SAH: cost of a triangle test relative to a node visit
  int bins = 16;           // SAH bins per axis
  float cost_traverse = 7.f;
  float cost_intersect = 2.f;
  float box_padding = 1e-5f;
  int threads = 0;         // 0 = hardware concurrency
};

struct bvh8_stats {
  std::size_t binary_nodes = 0;
  std::size_t wide_nodes = 0;
  std::size_t leaf_slots = 0;
  std::size_t triangles = 0;
  int binary_depth = 0;
  int wide_depth = 0;
  int max_leaf_size = 0;
  double build_seconds = 0.0;
};

struct bvh8 {
  std::vector<bvh8_node> nodes;
  std::vector<bvh8_triangle> triangles;
  float scene_lo[3] = {0, 0, 0};
  float scene_hi[3] = {0, 0, 0};
  bvh8_stats stats;
};

// Builds from world-space triangles: `positions` holds 3 * n_tris float3
// vertices (v0, v1, v2 per triangle, 9 floats each); `prim_ids` (may be null)
// gives the id stored per triangle (default: its index). Returns an empty
// tree (no nodes) when n_tris == 0.
bvh8 build_bvh8(float const* positions, std::size_t n_tris, std::uint32_t const* prim_ids,
    bvh8_build_options const& opt);

}  // namespace myrt_b200
