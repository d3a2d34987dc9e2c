// Host BVH build: binned SAH -> 8-wide quantised tree. See bvh8.hpp.
#include "bvh8.hpp"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <future>
#include <limits>
#include <stdexcept>
#include <thread>

namespace myrt_b200 {
namespace {

struct box3 {
  float lo[3] = {std::numeric_limits<float>::max(), std::numeric_limits<float>::max(),
      std::numeric_limits<float>::max()};
  float hi[3] = {std::numeric_limits<float>::lowest(), std::numeric_limits<float>::lowest(),
      std::numeric_limits<float>::lowest()};
  void grow(box3 const& b) {
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], b.lo[a]);
      hi[a] = std::max(hi[a], b.hi[a]);
    }
  }
  void grow(float const* p) {
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], p[a]);
      hi[a] = std::max(hi[a], p[a]);
    }
  }
  bool valid() const { return lo[0] <= hi[0] && lo[1] <= hi[1] && lo[2] <= hi[2]; }
  // Same expression as aabb_t::surface_area (bvh.hpp:44-47).
  float area() const {
    if (!valid()) return 0.f;
    float const dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    return ((dx + dy) * dz + dx * dy) * 2.f;
  }
};

struct bnode {
  box3 box;
  std::int32_t left = -1;   // child pair: left, left + 1 (internal) ; -1 for leaves
  std::uint32_t begin = 0;  // leaf: prim range in `order`
  std::uint32_t count = 0;
};

struct builder {
  bvh8_build_options opt;
  std::vector<box3> prim_box;
  std::vector<float> prim_c;  // 3 per prim
  std::vector<std::uint32_t> order;
  std::vector<bnode> nodes;
  std::atomic<std::uint32_t> node_count{1};
  std::atomic<int> max_depth{0};
  std::atomic<int> max_leaf{0};

  void make_leaf(std::uint32_t ni, std::uint32_t b, std::uint32_t e, int depth) {
    nodes[ni].left = -1;
    nodes[ni].begin = b;
    nodes[ni].count = e - b;
    int d = max_depth.load();
    while (depth > d && !max_depth.compare_exchange_weak(d, depth)) {
    }
    int m = max_leaf.load();
    int const c = int(e - b);
    while (c > m && !max_leaf.compare_exchange_weak(m, c)) {
    }
  }

  // Builds the subtree for order[b, e) into node ni (its box already set).
  void build(std::uint32_t ni, std::uint32_t b, std::uint32_t e, int depth) {
    std::uint32_t const n = e - b;
    if (n <= 1) return make_leaf(ni, b, e, depth);

    box3 cb;
    for (std::uint32_t i = b; i < e; ++i) cb.grow(&prim_c[3 * order[i]]);

    int const bins = opt.bins;
    float best_cost = std::numeric_limits<float>::max();
    int best_axis = -1, best_bin = -1;
    float const parent_area = nodes[ni].box.area();
    std::vector<box3> bin_box(std::size_t(bins) * 3);
    std::vector<std::uint32_t> bin_cnt(std::size_t(bins) * 3, 0);
    float scale[3];
    for (int a = 0; a < 3; ++a) {
      float const ext = cb.hi[a] - cb.lo[a];
      scale[a] = ext > 0.f ? float(bins) / ext : 0.f;
    }
    for (std::uint32_t i = b; i < e; ++i) {
      std::uint32_t const p = order[i];
      for (int a = 0; a < 3; ++a) {
        if (scale[a] == 0.f) continue;
        int k = int((prim_c[3 * p + a] - cb.lo[a]) * scale[a]);
        k = std::clamp(k, 0, bins - 1);
        bin_box[std::size_t(a) * bins + k].grow(prim_box[p]);
        bin_cnt[std::size_t(a) * bins + k]++;
      }
    }
    std::vector<float> right_area(bins);
    std::vector<std::uint32_t> right_cnt(bins);
    for (int a = 0; a < 3; ++a) {
      if (scale[a] == 0.f) continue;
      box3 acc;
      std::uint32_t cnt = 0;
      for (int k = bins - 1; k > 0; --k) {
        acc.grow(bin_box[std::size_t(a) * bins + k]);
        cnt += bin_cnt[std::size_t(a) * bins + k];
        right_area[k] = acc.area();
        right_cnt[k] = cnt;
      }
      box3 lacc;
      std::uint32_t lcnt = 0;
      for (int k = 0; k < bins - 1; ++k) {
        lacc.grow(bin_box[std::size_t(a) * bins + k]);
        lcnt += bin_cnt[std::size_t(a) * bins + k];
        std::uint32_t const rcnt = right_cnt[k + 1];
        if (lcnt == 0 || rcnt == 0) continue;
        float const cost = opt.cost_traverse +
            opt.cost_intersect * (float(lcnt) * lacc.area() + float(rcnt) * right_area[k + 1]) /
                std::max(parent_area, 1e-30f);
        if (cost < best_cost) {
          best_cost = cost;
          best_axis = a;
          best_bin = k;
        }
      }
    }
    float const leaf_cost = opt.cost_intersect * float(n);
    if (n <= std::uint32_t(opt.binary_leaf) && (best_axis < 0 || best_cost >= leaf_cost))
      return make_leaf(ni, b, e, depth);

    std::uint32_t mid;
    if (best_axis < 0) {
      mid = b + n / 2;  // all centroids coincide: split the range in half
    } else {
      float const lo = cb.lo[best_axis], sc = scale[best_axis];
      auto it = std::partition(order.begin() + b, order.begin() + e, [&](std::uint32_t p) {
        int k = std::clamp(int((prim_c[3 * p + best_axis] - lo) * sc), 0, bins - 1);
        return k <= best_bin;
      });
      mid = std::uint32_t(it - order.begin());
      if (mid == b || mid == e) mid = b + n / 2;
    }

    std::uint32_t const l = node_count.fetch_add(2);
    nodes[ni].left = std::int32_t(l);
    nodes[ni].count = 0;
    box3 lb, rb;
    for (std::uint32_t i = b; i < mid; ++i) lb.grow(prim_box[order[i]]);
    for (std::uint32_t i = mid; i < e; ++i) rb.grow(prim_box[order[i]]);
    nodes[l].box = lb;
    nodes[l + 1].box = rb;
    if (n > 65536 && depth < 6) {
      auto fut = std::async(std::launch::async, [&] { build(l, b, mid, depth + 1); });
      build(l + 1, mid, e, depth + 1);
      fut.get();
    } else {
      build(l, b, mid, depth + 1);
      build(l + 1, mid, e, depth + 1);
    }
  }
};

std::uint8_t biased_exponent_for(float extent) {
  // Smallest e with extent / 2^e <= 255.
  if (!(extent > 0.f)) return std::uint8_t(127 - 100);
  int e = int(std::ceil(std::log2(double(extent) / 255.0)));
  while (std::ldexp(255.0, e) < double(extent)) ++e;
  e = std::clamp(e, -126, 127);
  return std::uint8_t(e + 127);
}

}  // namespace

bvh8 build_bvh8(float const* positions, std::size_t n_tris, std::uint32_t const* prim_ids,
    bvh8_build_options const& opt) {
  auto const t0 = std::chrono::steady_clock::now();
  bvh8 out;
  if (n_tris == 0) return out;
  if (n_tris >= (std::size_t(1) << 31)) throw std::runtime_error("too many triangles for one BVH");
  if (opt.max_leaf < 1 || opt.max_leaf > 4) throw std::runtime_error("max_leaf must be in [1, 4]");
  if (opt.binary_leaf < 1 || opt.binary_leaf > opt.max_leaf)
    throw std::runtime_error("binary_leaf must be in [1, max_leaf]");

  builder bld;
  bld.opt = opt;
  bld.prim_box.resize(n_tris);
  bld.prim_c.resize(3 * n_tris);
  bld.order.resize(n_tris);
  box3 scene;
  for (std::size_t i = 0; i < n_tris; ++i) {
    float const* v = positions + 9 * i;
    box3& bx = bld.prim_box[i];
    bx.grow(v);
    bx.grow(v + 3);
    bx.grow(v + 6);
    for (int a = 0; a < 3; ++a) {
      bx.lo[a] -= opt.box_padding;
      bx.hi[a] += opt.box_padding;
      bld.prim_c[3 * i + a] = (v[a] + v[3 + a] + v[6 + a]) / 3.0f;
    }
    scene.grow(bx);
    bld.order[i] = std::uint32_t(i);
  }
  bld.nodes.resize(2 * n_tris);
  bld.nodes[0].box = scene;
  bld.build(0, 0, std::uint32_t(n_tris), 0);
  std::uint32_t const nb = bld.node_count.load();
  for (int a = 0; a < 3; ++a) {
    out.scene_lo[a] = scene.lo[a];
    out.scene_hi[a] = scene.hi[a];
  }

  // ---- collapse to the 8-wide layout ----
  // SAH-optimal collapse by dynamic programming over the binary tree (Ylitie,
  // Karras, Laine, HPG 2017, sec. 3.1): cost[i-1] is the least SAH cost of
  // representing binary subtree n with at most i slots of its parent: one leaf
  // slot (subtrees of at most max_leaf triangles, merged), one internal slot
  // (a new wide node whose 8 slots are split between n's two children), or the
  // i slots split between the children directly.
  auto const& bn = bld.nodes;
  // A triangle test costs about 0.3 node visits in instructions, but the collapse is charged 0.8:
  // with binary leaves of one triangle this packs fewer triangles per slot and measured fastest
  // (3,400 -> 3,679 Mrays/s on the 655,872-triangle icosphere scene; 0.3: 3,562, 1.0-3.0: 3,669-3,672).
  float const kNodeCost = 1.0f, kPrimCost = opt.collapse_prim_cost;
  constexpr float kInf = std::numeric_limits<float>::infinity();
  struct dp_t {
    float cost[8];
    std::uint8_t dec[8];    // 0 leaf slot, 1 internal slot, 2 split between children, 3 use one slot fewer
    std::uint8_t split[8];  // left share for dec == 2
    std::uint8_t split8;    // left share of the 8 slots when n becomes a wide node
  };
  std::vector<dp_t> D(nb);
  std::vector<std::uint32_t> ntri(nb);
  for (std::int64_t i = std::int64_t(nb) - 1; i >= 0; --i) {
    bnode const& b = bn[std::size_t(i)];
    dp_t& d = D[std::size_t(i)];
    float const area = b.box.area();
    if (b.left < 0) {
      ntri[std::size_t(i)] = b.count;
      float const leaf = area * kPrimCost * float(b.count);
      for (int j = 0; j < 8; ++j) {
        d.cost[j] = leaf;
        d.dec[j] = j == 0 ? 0 : 3;
        d.split[j] = 0;
      }
      d.split8 = 0;
      continue;
    }
    std::size_t const L = std::size_t(b.left), R = L + 1;
    ntri[std::size_t(i)] = ntri[L] + ntri[R];
    float dist[9];
    std::uint8_t dsplit[9];
    for (int j = 2; j <= 8; ++j) {
      dist[j] = kInf;
      dsplit[j] = 1;
      for (int k = 1; k < j; ++k) {
        float const c = D[L].cost[k - 1] + D[R].cost[j - k - 1];
        if (c < dist[j]) {
          dist[j] = c;
          dsplit[j] = std::uint8_t(k);
        }
      }
    }
    float const leaf = ntri[std::size_t(i)] <= std::uint32_t(opt.max_leaf) ? area * kPrimCost * float(ntri[std::size_t(i)])
                                                                           : kInf;
    float const internal = area * kNodeCost + dist[8];
    d.split8 = dsplit[8];
    d.cost[0] = std::min(leaf, internal);
    d.dec[0] = leaf <= internal ? 0 : 1;
    d.split[0] = 0;
    for (int j = 2; j <= 8; ++j) {
      if (dist[j] < d.cost[j - 2]) {
        d.cost[j - 1] = dist[j];
        d.dec[j - 1] = 2;
        d.split[j - 1] = dsplit[j];
      } else {
        d.cost[j - 1] = d.cost[j - 2];
        d.dec[j - 1] = 3;
        d.split[j - 1] = 0;
      }
    }
  }
  // slots of the wide node made from binary node n, as (binary node, is_internal)
  struct slot_t {
    std::uint32_t bnode;
    bool internal;
  };
  auto gather = [&](auto&& self, std::uint32_t n, int i, std::vector<slot_t>& out_slots) -> void {
    dp_t const& d = D[n];
    switch (d.dec[i - 1]) {
      case 3: self(self, n, i - 1, out_slots); break;
      case 2:
        self(self, std::uint32_t(bn[n].left), d.split[i - 1], out_slots);
        self(self, std::uint32_t(bn[n].left + 1), i - d.split[i - 1], out_slots);
        break;
      case 0: out_slots.push_back({n, false}); break;
      default: out_slots.push_back({n, true}); break;
    }
  };
  // triangles of a leaf slot: every binary leaf under n, in order
  auto collect = [&](auto&& self, std::uint32_t n, std::vector<std::uint32_t>& prims) -> void {
    if (bn[n].left < 0) {
      for (std::uint32_t k = 0; k < bn[n].count; ++k) prims.push_back(bld.order[bn[n].begin + k]);
      return;
    }
    self(self, std::uint32_t(bn[n].left), prims);
    self(self, std::uint32_t(bn[n].left + 1), prims);
  };

  // Emission, level by level of the wide tree (nodes are numbered in breadth-first order, the
  // children of a node contiguous): plan every node of a level in parallel (its slots, boxes,
  // quantised planes, leaf meta, internal children and triangle count), turn the counts into
  // child and triangle bases by a prefix sum in level order, then write the nodes and their leaf
  // triangles in parallel. The result equals a sequential breadth-first emission.
  struct wide_plan {
    bvh8_node node;
    std::int32_t slot_kid[8];
    std::uint32_t kids[8];
    int n_kids;
    std::uint32_t n_tris;
    int n_leaf_slots;
  };
  auto plan = [&](std::uint32_t bnode_index, wide_plan& w, std::vector<slot_t>& slots,
                  std::vector<std::uint32_t>& prims) {
    slots.clear();
    if (bn[bnode_index].left < 0) {
      slots.push_back({bnode_index, false});  // a lone leaf (tiny scenes): one leaf slot
    } else {
      gather(gather, std::uint32_t(bn[bnode_index].left), D[bnode_index].split8, slots);
      gather(gather, std::uint32_t(bn[bnode_index].left + 1), 8 - D[bnode_index].split8, slots);
    }
    int const nk = int(slots.size());
    std::uint32_t kids[8];
    for (int k = 0; k < nk; ++k) kids[k] = slots[std::size_t(k)].bnode;

    box3 nbox;
    for (int k = 0; k < nk; ++k) nbox.grow(bn[kids[k]].box);
    float const cx = 0.5f * (nbox.lo[0] + nbox.hi[0]), cy = 0.5f * (nbox.lo[1] + nbox.hi[1]),
                cz = 0.5f * (nbox.lo[2] + nbox.hi[2]);

    // Octant slot assignment: slot s faces direction (+-1,+-1,+-1) with bit a of
    // s set meaning +; the child lying furthest that way takes the slot.
    int slot_of[8];
    {
      bool kid_done[8] = {}, slot_done[8] = {};
      float cost[8][8];
      for (int k = 0; k < nk; ++k) {
        float const dx = 0.5f * (bn[kids[k]].box.lo[0] + bn[kids[k]].box.hi[0]) - cx;
        float const dy = 0.5f * (bn[kids[k]].box.lo[1] + bn[kids[k]].box.hi[1]) - cy;
        float const dz = 0.5f * (bn[kids[k]].box.lo[2] + bn[kids[k]].box.hi[2]) - cz;
        for (int s = 0; s < 8; ++s)
          cost[k][s] = ((s & 1) ? dx : -dx) + ((s & 2) ? dy : -dy) + ((s & 4) ? dz : -dz);
      }
      for (int r = 0; r < nk; ++r) {
        int bk = -1, bs = -1;
        float bc = -std::numeric_limits<float>::max();
        for (int k = 0; k < nk; ++k) {
          if (kid_done[k]) continue;
          for (int s = 0; s < 8; ++s) {
            if (slot_done[s]) continue;
            if (cost[k][s] > bc) {
              bc = cost[k][s];
              bk = k;
              bs = s;
            }
          }
        }
        kid_done[bk] = slot_done[bs] = true;
        slot_of[bk] = bs;
      }
    }
    bool slot_internal[8];
    for (int s = 0; s < 8; ++s) {
      w.slot_kid[s] = -1;
      slot_internal[s] = false;
    }
    for (int k = 0; k < nk; ++k) {
      w.slot_kid[slot_of[k]] = std::int32_t(kids[k]);
      slot_internal[slot_of[k]] = slots[std::size_t(k)].internal;
    }

    bvh8_node& node = w.node;
    node = bvh8_node{};
    node.px = nbox.lo[0];
    node.py = nbox.lo[1];
    node.pz = nbox.lo[2];
    double scale[3];
    for (int a = 0; a < 3; ++a) {
      node.e[a] = biased_exponent_for(nbox.hi[a] - nbox.lo[a]);
      scale[a] = std::ldexp(1.0, int(node.e[a]) - 127);
    }
    float const p[3] = {node.px, node.py, node.pz};
    std::uint32_t tri_off = 0;
    w.n_kids = 0;
    w.n_leaf_slots = 0;
    for (int s = 0; s < 8; ++s) {
      if (w.slot_kid[s] < 0) {
        for (int a = 0; a < 3; ++a) {
          node.qlo[a][s] = 1;
          node.qhi[a][s] = 0;
        }
        node.meta[s] = 0;
        continue;
      }
      bnode const& c = bn[std::uint32_t(w.slot_kid[s])];
      for (int a = 0; a < 3; ++a) {
        double const lo = std::floor((double(c.box.lo[a]) - double(p[a])) / scale[a]);
        double const hi = std::ceil((double(c.box.hi[a]) - double(p[a])) / scale[a]);
        node.qlo[a][s] = std::uint8_t(std::clamp(lo, 0.0, 255.0));
        node.qhi[a][s] = std::uint8_t(std::clamp(hi, 0.0, 255.0));
      }
      if (slot_internal[s]) {
        node.imask |= std::uint8_t(1u << s);
        node.meta[s] = std::uint8_t(0x20u | unsigned(s));
        w.kids[w.n_kids++] = std::uint32_t(w.slot_kid[s]);
        w.slot_kid[s] = -1;  // only leaf slots keep their binary node for the triangle pass
      } else {
        prims.clear();
        collect(collect, std::uint32_t(w.slot_kid[s]), prims);
        std::uint32_t const cnt = std::uint32_t(prims.size());
        node.meta[s] = std::uint8_t(tri_off | (cnt << 5));
        tri_off += cnt;
        ++w.n_leaf_slots;
      }
    }
    w.n_tris = tri_off;
  };
  // parallel loop over [0, n) in contiguous chunks, fn(begin, end, worker scratch index)
  unsigned const workers = std::max(1u, opt.threads > 0 ? unsigned(opt.threads) : std::thread::hardware_concurrency());
  auto parallel_for = [&](std::size_t n, auto&& fn) {
    std::size_t const parts = std::min<std::size_t>(workers, (n + 1023) / 1024);
    if (parts <= 1) {
      fn(std::size_t(0), n, 0u);
      return;
    }
    std::vector<std::thread> pool;
    std::size_t const step = (n + parts - 1) / parts;
    for (std::size_t w = 0; w < parts; ++w) {
      std::size_t const b = w * step, e = std::min(n, b + step);
      if (b >= e) break;
      pool.emplace_back([&fn, b, e, w] { fn(b, e, unsigned(w)); });
    }
    for (auto& t : pool) t.join();
  };
  std::vector<std::vector<slot_t>> slot_scratch(workers);
  std::vector<std::vector<std::uint32_t>> prim_scratch(workers);

  out.triangles.resize(n_tris);
  std::vector<std::uint32_t> level{0}, next;  // binary nodes of the current level, in node order
  std::vector<wide_plan> plans;
  std::vector<std::uint32_t> child_base, tri_base;
  std::size_t level_base = 0, tris_done = 0, leaf_slots = 0;
  int wide_depth = 0;
  while (!level.empty()) {
    ++wide_depth;
    std::size_t const n_level = level.size();
    plans.resize(n_level);
    parallel_for(n_level, [&](std::size_t b, std::size_t e, unsigned w) {
      for (std::size_t i = b; i < e; ++i) plan(level[i], plans[i], slot_scratch[w], prim_scratch[w]);
    });
    child_base.resize(n_level);
    tri_base.resize(n_level);
    std::size_t next_base = level_base + n_level, kids_total = 0;
    for (std::size_t i = 0; i < n_level; ++i) {
      child_base[i] = std::uint32_t(next_base + kids_total);
      tri_base[i] = std::uint32_t(tris_done);
      kids_total += std::size_t(plans[i].n_kids);
      tris_done += plans[i].n_tris;
      leaf_slots += std::size_t(plans[i].n_leaf_slots);
    }
    out.nodes.resize(next_base + kids_total);
    next.resize(kids_total);
    parallel_for(n_level, [&](std::size_t b, std::size_t e, unsigned w) {
      std::vector<std::uint32_t>& pr = prim_scratch[w];
      for (std::size_t i = b; i < e; ++i) {
        wide_plan& wp = plans[i];
        wp.node.child_base = child_base[i];
        wp.node.tri_base = tri_base[i];
        out.nodes[level_base + i] = wp.node;
        for (int k = 0; k < wp.n_kids; ++k) next[child_base[i] - next_base + std::size_t(k)] = wp.kids[k];
        std::size_t t = tri_base[i];
        for (int s = 0; s < 8; ++s) {
          if (wp.slot_kid[s] < 0) continue;
          pr.clear();
          collect(collect, std::uint32_t(wp.slot_kid[s]), pr);
          for (std::uint32_t prim : pr) {
            float const* v = positions + 9 * std::size_t(prim);
            bvh8_triangle& tr = out.triangles[t++];
            tr = bvh8_triangle{};
            std::memcpy(tr.v0, v, 12);
            std::memcpy(tr.v1, v + 3, 12);
            std::memcpy(tr.v2, v + 6, 12);
            tr.prim = prim_ids ? prim_ids[prim] : prim;
          }
        }
      }
    });
    level_base = next_base;
    level.swap(next);
  }
  if (tris_done != n_tris) throw std::runtime_error("BVH emission lost triangles");

  auto const t1 = std::chrono::steady_clock::now();
  out.stats.binary_nodes = nb;
  out.stats.wide_nodes = out.nodes.size();
  out.stats.leaf_slots = leaf_slots;
  out.stats.triangles = out.triangles.size();
  out.stats.binary_depth = bld.max_depth.load();
  out.stats.wide_depth = wide_depth;
  out.stats.max_leaf_size = bld.max_leaf.load();
  out.stats.build_seconds = std::chrono::duration<double>(t1 - t0).count();
  return out;
}

}  // namespace myrt_b200
