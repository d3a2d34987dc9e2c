// Host analysis of flat SDF programs for the evaluator's exact skipping
// (sdf.cuh map): per instruction, the bounding sphere and extent of the group
// "translations, primitive, union / smooth union" that starts there; per
// left-to-right chain program, a grid of cell lists of the groups that can
// change the value inside each cell.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/myrt_cuda.h"

namespace myrt_b200 {

// Per instruction of valid programs: where a group "translations, primitive,
// union / smooth union" starts with a value already on the stack, the
// primitive's bounding sphere in the program's space (centre = summed
// translations + the primitive's own centre, radius R with distance >= |p - c|
// - R everywhere) and (absolute index after the operator, k bits). Primitives
// without such a bound (Menger sponge, degenerate parameters) and groups with a
// mirror are not skippable. Empty tables when nothing is skippable.
inline void sdf_skip_tables(myrt_sdf_view const* v, std::vector<float4>& sphere, std::vector<int2>& next) {
  sphere.assign(v->instr_count, make_float4(0.f, 0.f, 0.f, 0.f));
  next.assign(v->instr_count, make_int2(0, 0));
  std::vector<int> owner(v->instr_count, -1);
  bool any = false;
  float const* G = v->params;
  for (size_t p = 0; p < v->program_count; ++p) {
    myrt_sdf_program const pr = v->programs[p];
    int depth = 0;
    for (int g = 0; g < pr.count; ++g) {
      int const ag = pr.first + g;
      int j = g;
      double c[3] = {0.0, 0.0, 0.0};
      // a group starts at its first modifier (or at the primitive when it has
      // none): the evaluator tests the bound before applying any of them
      bool ok = depth >= 1 && (g == 0 || v->instrs[ag - 1].op < MYRT_SDF_TRANSLATE);
      while (ok && j < pr.count && v->instrs[pr.first + j].op >= MYRT_SDF_TRANSLATE) {
        myrt_sdf_instr const m = v->instrs[pr.first + j];
        if (m.op != MYRT_SDF_TRANSLATE) ok = false;
        else
          for (int a = 0; a < 3; ++a) c[a] += double(G[m.param_offset + a]);
        ++j;
      }
      double R = 0.0;
      bool bounded = false;  // only the primitives below have a bounding sphere
      if (ok && j + 1 < pr.count) {
        myrt_sdf_instr const prim = v->instrs[pr.first + j];
        myrt_sdf_instr const op = v->instrs[pr.first + j + 1];
        float const* q = G + prim.param_offset;
        switch (prim.op) {
          case MYRT_SDF_SPHERE:
            R = std::fabs(double(q[0]));
            bounded = true;
            break;
          case MYRT_SDF_BOX:
            if (q[0] >= 0.f && q[1] >= 0.f && q[2] >= 0.f) {
              R = std::sqrt(double(q[0]) * q[0] + double(q[1]) * q[1] + double(q[2]) * q[2]);
              bounded = true;
            }
            break;
          case MYRT_SDF_TORUS:
            R = std::fabs(double(q[0])) + double(q[1]);
            bounded = true;
            break;
          case MYRT_SDF_CAPSULE:
            if (q[0] >= 0.f) {
              c[1] += 0.5 * double(q[0]);
              R = 0.5 * double(q[0]) + double(q[1]);
              bounded = true;
            }
            break;
          default: break;  // operators, the Menger sponge: no bound
        }
        float k = -1.f;
        if (op.op == MYRT_SDF_UNION) k = 0.f;
        else if (op.op == MYRT_SDF_SMOOTH_UNION && G[op.param_offset] > 0.f) k = G[op.param_offset];
        bool const finite = std::isfinite(R) && std::isfinite(c[0]) && std::isfinite(c[1]) && std::isfinite(c[2]);
        if (k >= 0.f && finite && bounded) {
          // a negative R is a valid (tighter) bound too: distance >= |p - c| - R
          float4 const s = make_float4(float(c[0]), float(c[1]), float(c[2]), float(R) + 1e-6f * float(std::fabs(R)));
          int kbits;
          std::memcpy(&kbits, &k, sizeof kbits);
          int2 const n = make_int2(pr.first + j + 2, kbits);
          if (owner[ag] < 0) {
            owner[ag] = int(p);
            sphere[ag] = s;
            next[ag] = n;
            any = true;
          } else if (next[ag].x != n.x || next[ag].y != n.y || std::memcmp(&sphere[ag], &s, sizeof s) != 0) {
            next[ag] = make_int2(0, 0);  // instruction shared by programs with different groups
          }
        }
      }
      // stack depth after instruction g
      int const op = v->instrs[ag].op;
      if (op >= MYRT_SDF_TRANSLATE) {
      } else if (op >= MYRT_SDF_UNION) {
        --depth;
      } else {
        ++depth;
      }
    }
  }
  if (!any) {
    sphere.clear();
    next.clear();
  }
}

// Per instruction: the number of operator instructions of its program up to and
// including it, so that an evaluation that leaves out a range of instructions
// can still draw the random numbers those operators would have drawn (sdf.cuh
// map, material loads). Empty when programs share instructions at different
// offsets.
inline void sdf_op_counts(myrt_sdf_view const* v, std::vector<int>& out) {
  out.assign(v->instr_count, -1);
  for (size_t p = 0; p < v->program_count; ++p) {
    myrt_sdf_program const pr = v->programs[p];
    int n = 0;
    for (int k = 0; k < pr.count; ++k) {
      int const op = v->instrs[pr.first + k].op;
      if (op >= MYRT_SDF_UNION && op < MYRT_SDF_TRANSLATE) ++n;
      int& slot = out[pr.first + k];
      if (slot >= 0 && slot != n) {
        out.clear();
        return;
      }
      slot = n;
    }
  }
}

// Distance bounds of a primitive about a centre c (updated in place for the
// capsule, whose centre is its segment's midpoint):
//   |p - c| - R  <=  d(p)  <=  |p - c| + U   for every point p.
// Sphere (r): d = |p - c| - r. Box (b >= 0): the box lies within |b| of c and
// holds the ball of radius min(b). Torus (R1, r2): the ring is at |R1| from c.
// Capsule (h >= 0, r): the segment lies within h / 2 of its midpoint.
inline bool sdf_prim_bounds(int op, float const* q, double c[3], double& R, double& U) {
  switch (op) {
    case MYRT_SDF_SPHERE:
      R = std::fabs(double(q[0]));
      U = -double(q[0]);
      return true;
    case MYRT_SDF_BOX:
      if (!(q[0] >= 0.f && q[1] >= 0.f && q[2] >= 0.f)) return false;
      R = std::sqrt(double(q[0]) * q[0] + double(q[1]) * q[1] + double(q[2]) * q[2]);
      U = -double(std::fmin(q[0], std::fmin(q[1], q[2])));
      return true;
    case MYRT_SDF_TORUS:
      R = std::fabs(double(q[0])) + double(q[1]);
      U = std::fabs(double(q[0])) - double(q[1]);
      return true;
    case MYRT_SDF_CAPSULE:
      if (!(q[0] >= 0.f)) return false;
      c[1] += 0.5 * double(q[0]);
      R = 0.5 * double(q[0]) + double(q[1]);
      U = 0.5 * double(q[0]) - double(q[1]);
      return true;
    default: return false;
  }
}

// Per-program cell lists for the evaluator (sdf.cuh map).
//
// Programs that are trees of union / smooth-union operators over translated,
// bounded primitives (any shape: left or right folds, balanced trees) get a
// uniform grid over the primitives' bounding boxes. Two facts about an
// operator op(A, B) with factor k (k = 0 for a union), A the left operand:
//   * it returns A's value bit for bit where B >= A + k (h clamps to 1), and
//     B's where A >= B + k (h clamps to 0), up to the sign of a zero result;
//   * its value lies between min(A, B) - delta and min(A, B): a smooth union
//     never exceeds its smaller operand and falls below it by at most k / 4;
//     when one operand is a primitive it stays above min(lower bounds) -
//     max(delta of the other operand, k) (the blend lowers min(a, b) by
//     (k - |a - b|)^2 / 4k and never below the primitive minus k).
// Every node thus has a lower bound (its primitives' |p - c| - R minus its
// delta) and an upper bound (the smallest |p - c| + U of its primitives) over
// a cell. Walking the tree from the root, an operator whose right subtree's
// lower bound is at least the left's upper bound + k + a rounding margin
// drops the right subtree and itself, and the mirror case drops the left
// subtree and the operator, for every point of the cell. What remains of the
// program is stored as instruction segments in program order; the stack then
// holds the same values as the full evaluation at every step that runs.
// Points outside the grid evaluate the whole program.
//
// Escape sphere: the root's value is at least |p - C| - rho - delta_root with
// rho bounding every primitive's |c_i - C| + R_i, so a march that is outside
// the sphere (C, r_esc) and moving away from C never meets a value below eps
// again (sdf.cuh march).
struct sdf_cells {
  std::vector<int4> hdr;       // 3 per program: (lo.xyz, 1 / cell) bits; (nx, ny, nz, first cell);
                               // escape sphere (C.xyz, r_esc) bits
  std::vector<int> start;      // per program (cells + 1) offsets into list
  std::vector<uint32_t> list;  // segment (start | end << 16), relative to the program's first instruction
};

// cells_long: cells along the grid's longest axis (2..128).
inline void sdf_cell_tables(myrt_sdf_view const* v, int cells_long, sdf_cells& out) {
  out = sdf_cells{};
  out.hdr.assign(3 * v->program_count, make_int4(0, 0, 0, 0));
  float const* G = v->params;
  struct node {
    int first, end;  // instruction range (end exclusive); an operator's own index is end - 1
    int a = -1, b = -1;  // operand nodes (operators)
    double c[3] = {0.0, 0.0, 0.0}, R = 0.0, U = 0.0;  // primitives
    double k = 0.0, delta = 0.0;
  };
  bool any = false;
  size_t const max_entries = size_t(1) << 26;
  for (size_t p = 0; p < v->program_count; ++p) {
    myrt_sdf_program const pr = v->programs[p];
    if (pr.count >= 65536) continue;
    std::vector<node> ns;
    std::vector<int> st;
    int n_prims = 0;
    bool ok = true;
    for (int j = 0; ok && j < pr.count;) {
      myrt_sdf_instr const in = v->instrs[pr.first + j];
      if (in.op == MYRT_SDF_UNION || in.op == MYRT_SDF_SMOOTH_UNION) {
        if (st.size() < 2) { ok = false; break; }
        node n{};
        n.b = st.back();
        st.pop_back();
        n.a = st.back();
        st.pop_back();
        n.first = ns[n.a].first;
        n.end = j + 1;
        if (in.op == MYRT_SDF_SMOOTH_UNION) {
          if (!(G[in.param_offset] > 0.f)) { ok = false; break; }
          n.k = double(G[in.param_offset]);
        }
        bool const leaf_a = ns[n.a].a < 0, leaf_b = ns[n.b].a < 0;
        double const da = ns[n.a].delta, db = ns[n.b].delta;
        // both bounds hold; keep the smaller (two primitives: k / 4; a long
        // fold saturates at k)
        n.delta = std::fmax(da, db) + 0.25 * n.k;
        if (leaf_a || leaf_b) n.delta = std::fmin(n.delta, std::fmax(std::fmax(da, db), n.k));
        st.push_back(int(ns.size()));
        ns.push_back(n);
        ++j;
        continue;
      }
      node n{};
      n.first = j;
      while (j < pr.count && v->instrs[pr.first + j].op == MYRT_SDF_TRANSLATE) {
        float const* t = G + v->instrs[pr.first + j].param_offset;
        for (int a = 0; a < 3; ++a) n.c[a] += double(t[a]);
        ++j;
      }
      if (j >= pr.count) { ok = false; break; }
      myrt_sdf_instr const prim = v->instrs[pr.first + j];
      ok = sdf_prim_bounds(prim.op, G + prim.param_offset, n.c, n.R, n.U) && std::isfinite(n.R) &&
           std::isfinite(n.U) && std::isfinite(n.c[0]) && std::isfinite(n.c[1]) && std::isfinite(n.c[2]);
      ++j;
      n.end = j;
      st.push_back(int(ns.size()));
      ns.push_back(n);
      ++n_prims;
    }
    if (!ok || st.size() != 1 || n_prims < 8) continue;
    int const root = st[0];
    // grid over the primitives' bounding boxes, padded by the largest k
    double lo[3], hi[3], kmax = 0.0, scale = 1.0;
    bool first = true;
    for (node const& n : ns) {
      kmax = std::fmax(kmax, n.k);
      if (n.a >= 0) continue;
      double const r = std::fmax(std::fabs(n.R), std::fabs(n.U));
      for (int a = 0; a < 3; ++a) {
        lo[a] = first ? n.c[a] - r : std::fmin(lo[a], n.c[a] - r);
        hi[a] = first ? n.c[a] + r : std::fmax(hi[a], n.c[a] + r);
        scale = std::fmax(scale, std::fabs(n.c[a]) + r);
      }
      first = false;
    }
    double ext = 0.0;
    for (int a = 0; a < 3; ++a) {
      lo[a] -= kmax + 1e-3;
      hi[a] += kmax + 1e-3;
      ext = std::fmax(ext, hi[a] - lo[a]);
    }
    // host work is cells x nodes: coarser grids for very large programs keep
    // an upload within about 2^26 node bounds (about a second)
    int n_long = cells_long;
    while (n_long > 4 && double(n_long) * n_long * n_long * double(ns.size()) > double(1 << 26)) n_long = n_long * 3 / 4;
    float const inv_f = float(double(n_long) / ext);
    float lo_f[3];
    int dims[3];
    for (int a = 0; a < 3; ++a) {
      lo_f[a] = float(lo[a]);
      dims[a] = std::max(1, std::min(n_long, int(std::ceil((hi[a] - double(lo_f[a])) * double(inv_f)))));
    }
    size_t const ncell = size_t(dims[0]) * dims[1] * dims[2];
    double const cell = 1.0 / double(inv_f);
    // the device finds a point's cell by rounded float arithmetic: widen each
    // cell; the margin covers the rounding of every distance and of the
    // operators' values over the whole program
    double const widen = 1e-4 * cell + 1e-6 * scale;
    double const margin = 2e-3 + 4e-6 * double(n_prims) * scale;
    size_t const first_start = out.start.size();
    size_t const first_entry = out.list.size();
    // z-slabs of cells on host threads; each keeps its cells' segment counts
    // and segments, concatenated in cell order afterwards
    struct slab {
      std::vector<int> sizes;
      std::vector<uint32_t> segs;
    };
    int const n_threads = std::max(1, std::min<int>(dims[2], int(std::thread::hardware_concurrency())));
    std::vector<slab> slabs(n_threads);
    auto fill = [&](int t) {
      slab& out_t = slabs[t];
      std::vector<double> lb(ns.size()), ub(ns.size());
      std::vector<int> todo;
      uint32_t seg_s = 0, seg_e = 0;
      bool open = false;
      auto exec = [&](int s0, int e0) {  // append [s0, e0), merging with the open segment
        if (open && int(seg_e) == s0) {
          seg_e = uint32_t(e0);
          return;
        }
        if (open) out_t.segs.push_back(seg_s | (seg_e << 16));
        seg_s = uint32_t(s0);
        seg_e = uint32_t(e0);
        open = true;
      };
      int const z0 = int(int64_t(dims[2]) * t / n_threads), z1 = int(int64_t(dims[2]) * (t + 1) / n_threads);
      for (int z = z0; z < z1; ++z)
        for (int y = 0; y < dims[1]; ++y)
          for (int x = 0; x < dims[0]; ++x) {
            int const idx[3] = {x, y, z};
            double bmin[3], bmax[3];
            for (int a = 0; a < 3; ++a) {
              bmin[a] = double(lo_f[a]) + idx[a] * cell - widen;
              bmax[a] = double(lo_f[a]) + (idx[a] + 1) * cell + widen;
            }
            size_t const before = out_t.segs.size();
            for (size_t i = 0; i < ns.size(); ++i) {  // operands come before their operator
              node const& n = ns[i];
              if (n.a < 0) {
                double n2 = 0.0, f2 = 0.0;
                for (int a = 0; a < 3; ++a) {
                  double const o = std::fmax(0.0, std::fmax(bmin[a] - n.c[a], n.c[a] - bmax[a]));
                  double const f = std::fmax(std::fabs(n.c[a] - bmin[a]), std::fabs(n.c[a] - bmax[a]));
                  n2 += o * o;
                  f2 += f * f;
                }
                lb[i] = std::sqrt(n2) - n.R;
                ub[i] = std::sqrt(f2) + n.U;
              } else {
                // lb of an operator node is (its primitives' smallest bound -
                // its delta); lb + delta recovers the primitives' bound
                lb[i] = std::fmin(lb[n.a] + ns[n.a].delta, lb[n.b] + ns[n.b].delta) - n.delta;
                ub[i] = std::fmin(ub[n.a], ub[n.b]);
              }
            }
            open = false;
            todo.assign(1, root);
            while (!todo.empty()) {  // depth first, left operand first
              int const i = todo.back();
              todo.pop_back();
              if (i < 0) {  // an operator kept with both operands
                exec(-i - 1, -i);
                continue;
              }
              node const& n = ns[i];
              if (n.a < 0) {
                exec(n.first, n.end);
                continue;
              }
              if (lb[n.b] >= ub[n.a] + n.k + margin) {
                todo.push_back(n.a);  // the right operand and the operator drop out
              } else if (lb[n.a] >= ub[n.b] + n.k + margin) {
                todo.push_back(n.b);  // the left operand and the operator drop out
              } else {
                todo.push_back(-(n.end - 1) - 1);
                todo.push_back(n.b);
                todo.push_back(n.a);
              }
            }
            if (open) out_t.segs.push_back(seg_s | (seg_e << 16));
            out_t.sizes.push_back(int(out_t.segs.size() - before));
          }
    };
    {
      std::vector<std::thread> pool;
      for (int t = 1; t < n_threads; ++t) pool.emplace_back(fill, t);
      fill(0);
      for (std::thread& th : pool) th.join();
    }
    size_t total = out.list.size();
    for (slab const& sl : slabs) total += sl.segs.size();
    if (total > max_entries) continue;  // too large: no cells for this program
    out.start.reserve(first_start + ncell + 1);
    out.list.reserve(total);
    for (slab const& sl : slabs) {
      for (int n_seg : sl.sizes) {
        out.start.push_back(int(out.list.size()));
        out.list.resize(out.list.size() + size_t(n_seg));
      }
    }
    {  // copy the segments behind the offsets just laid out
      size_t at = first_entry;
      for (slab const& sl : slabs) {
        std::copy(sl.segs.begin(), sl.segs.end(), out.list.begin() + ptrdiff_t(at));
        at += sl.segs.size();
      }
    }
    out.start.push_back(int(out.list.size()));
    // escape sphere about the grid's centre; the radius carries a relative
    // margin for the rounding of values and positions far from the field
    float esc[4];
    double rho = 0.0;
    for (int a = 0; a < 3; ++a) esc[a] = float(0.5 * (lo[a] + hi[a]));
    for (node const& n : ns) {
      if (n.a >= 0) continue;
      double const dx = n.c[0] - esc[0], dy = n.c[1] - esc[1], dz = n.c[2] - esc[2];
      rho = std::fmax(rho, std::sqrt(dx * dx + dy * dy + dz * dz) + n.R);
    }
    esc[3] = float((rho + ns[root].delta + margin) * 1.001 + 1e-3);
    int lo_bits[3], inv_bits, esc_bits[4];
    std::memcpy(lo_bits, lo_f, sizeof lo_bits);
    std::memcpy(&inv_bits, &inv_f, sizeof inv_bits);
    std::memcpy(esc_bits, esc, sizeof esc_bits);
    out.hdr[3 * p + 0] = make_int4(lo_bits[0], lo_bits[1], lo_bits[2], inv_bits);
    out.hdr[3 * p + 1] = make_int4(dims[0], dims[1], dims[2], int(first_start));
    out.hdr[3 * p + 2] = make_int4(esc_bits[0], esc_bits[1], esc_bits[2], esc_bits[3]);
    any = true;
  }
  if (!any) out = sdf_cells{};
}

}  // namespace myrt_b200
