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
// A program that is a left-to-right chain "T* prim (T* prim op)*" of
// translations, bounded primitives and union / smooth-union operators keeps a
// running value d0 that is at most the smallest upper bound |p - c_i| + U_i
// of the groups before (a smooth union never exceeds the smaller operand). A
// group i returns d0 bit for bit wherever d_i >= d0 + k_i (see map). Over a
// cell of a uniform grid laid over the chain's bounding box, group i can be
// left out when its smallest lower bound is at least the running upper bound
// plus k_i plus a margin for rounding; the cell keeps the groups that remain,
// in program order. Points outside the grid evaluate the whole program.
//
// Escape sphere: the running value never falls more than k_max below the
// smallest primitive distance (a smooth union lowers min(d0, d1) by
// (k - |d1 - d0|)^2 / 4k, which keeps it above the newer operand minus k), so
// the chain's value is at least |p - C| - rho - k_max with rho bounding every
// group's |c_i - C| + R_i. A march that is outside the sphere (C, r_esc) and
// moving away from C never meets a value below eps again (sdf.cuh march).
struct sdf_cells {
  std::vector<int4> hdr;       // 4 per program: (lo.xyz, 1 / cell) bits; (nx, ny, nz, first cell);
                               // (head end, 0, 0, 0); escape sphere (C.xyz, r_esc) bits
  std::vector<int> start;      // per program (cells + 1) offsets into list
  std::vector<uint32_t> list;  // group (start | end << 16), relative to the program's first instruction
};

// cells_long: cells along the grid's longest axis (2..128).
inline void sdf_cell_tables(myrt_sdf_view const* v, int cells_long, sdf_cells& out) {
  out = sdf_cells{};
  out.hdr.assign(4 * v->program_count, make_int4(0, 0, 0, 0));
  float const* G = v->params;
  struct group {
    int first, end;
    double c[3], R, U, k;
  };
  bool any = false;
  size_t const max_entries = size_t(1) << 26;
  for (size_t p = 0; p < v->program_count; ++p) {
    myrt_sdf_program const pr = v->programs[p];
    if (pr.count >= 65536) continue;
    std::vector<group> gs;
    int j = 0;
    bool ok = true;
    while (ok && j < pr.count) {
      group g{};
      g.first = j;
      while (j < pr.count && v->instrs[pr.first + j].op == MYRT_SDF_TRANSLATE) {
        float const* t = G + v->instrs[pr.first + j].param_offset;
        for (int a = 0; a < 3; ++a) g.c[a] += double(t[a]);
        ++j;
      }
      if (j >= pr.count) { ok = false; break; }
      myrt_sdf_instr const prim = v->instrs[pr.first + j];
      ok = sdf_prim_bounds(prim.op, G + prim.param_offset, g.c, g.R, g.U);
      ++j;
      if (ok && !gs.empty()) {
        if (j >= pr.count) { ok = false; break; }
        myrt_sdf_instr const op = v->instrs[pr.first + j];
        if (op.op == MYRT_SDF_UNION) g.k = 0.0;
        else if (op.op == MYRT_SDF_SMOOTH_UNION && G[op.param_offset] > 0.f) g.k = double(G[op.param_offset]);
        else ok = false;
        ++j;
      }
      g.end = j;
      ok = ok && std::isfinite(g.R) && std::isfinite(g.U) && std::isfinite(g.c[0]) && std::isfinite(g.c[1]) &&
           std::isfinite(g.c[2]) && std::isfinite(g.k);
      if (ok) gs.push_back(g);
    }
    if (!ok || gs.size() < 8) continue;
    // grid over the groups' bounding boxes, padded by the largest k
    double lo[3], hi[3], kmax = 0.0, scale = 1.0;
    for (int a = 0; a < 3; ++a) lo[a] = hi[a] = gs[0].c[a];
    for (group const& g : gs) {
      double const r = std::fmax(std::fabs(g.R), std::fabs(g.U));
      kmax = std::fmax(kmax, g.k);
      for (int a = 0; a < 3; ++a) {
        lo[a] = std::fmin(lo[a], g.c[a] - r);
        hi[a] = std::fmax(hi[a], g.c[a] + r);
        scale = std::fmax(scale, std::fabs(g.c[a]) + r);
      }
    }
    double ext = 0.0;
    for (int a = 0; a < 3; ++a) {
      lo[a] -= kmax + 1e-3;
      hi[a] += kmax + 1e-3;
      ext = std::fmax(ext, hi[a] - lo[a]);
    }
    float const inv_f = float(double(cells_long) / ext);
    float lo_f[3];
    int dims[3];
    for (int a = 0; a < 3; ++a) {
      lo_f[a] = float(lo[a]);
      dims[a] = std::max(1, std::min(cells_long, int(std::ceil((hi[a] - double(lo_f[a])) * double(inv_f)))));
    }
    size_t const ncell = size_t(dims[0]) * dims[1] * dims[2];
    double const cell = 1.0 / double(inv_f);
    // the device finds a point's cell by rounded float arithmetic: widen each
    // cell; the margin covers the rounding of every distance and of the
    // running value over all the chain's groups
    double const widen = 1e-4 * cell + 1e-6 * scale;
    double const margin = 2e-3 + 4e-6 * double(gs.size()) * scale;
    size_t const first_start = out.start.size();
    size_t const first_entry = out.list.size();
    out.start.reserve(first_start + ncell + 1);
    std::vector<double> dmin(gs.size()), dmax(gs.size());
    for (int z = 0; z < dims[2]; ++z)
      for (int y = 0; y < dims[1]; ++y)
        for (int x = 0; x < dims[0]; ++x) {
          int const idx[3] = {x, y, z};
          double bmin[3], bmax[3];
          for (int a = 0; a < 3; ++a) {
            bmin[a] = double(lo_f[a]) + idx[a] * cell - widen;
            bmax[a] = double(lo_f[a]) + (idx[a] + 1) * cell + widen;
          }
          out.start.push_back(int(out.list.size()));
          double run = 0.0;
          for (size_t i = 0; i < gs.size(); ++i) {
            double n2 = 0.0, f2 = 0.0;
            for (int a = 0; a < 3; ++a) {
              double const c = gs[i].c[a];
              double const o = std::fmax(0.0, std::fmax(bmin[a] - c, c - bmax[a]));
              double const f = std::fmax(std::fabs(c - bmin[a]), std::fabs(c - bmax[a]));
              n2 += o * o;
              f2 += f * f;
            }
            double const lb = std::sqrt(n2) - gs[i].R, ub = std::sqrt(f2) + gs[i].U;
            if (i == 0) {
              run = ub;
              continue;
            }
            if (lb < run + gs[i].k + margin)
              out.list.push_back(uint32_t(gs[i].first) | (uint32_t(gs[i].end) << 16));
            run = std::fmin(run, ub);
          }
        }
    out.start.push_back(int(out.list.size()));
    if (out.list.size() > max_entries) {  // too large: no cells for this program
      out.start.resize(first_start);
      out.list.resize(first_entry);
      continue;
    }
    int lo_bits[3], inv_bits;
    std::memcpy(lo_bits, lo_f, sizeof lo_bits);
    std::memcpy(&inv_bits, &inv_f, sizeof inv_bits);
    out.hdr[4 * p + 0] = make_int4(lo_bits[0], lo_bits[1], lo_bits[2], inv_bits);
    out.hdr[4 * p + 1] = make_int4(dims[0], dims[1], dims[2], int(first_start));
    out.hdr[4 * p + 2] = make_int4(gs[0].end, 0, 0, 0);
    // escape sphere about the grid's centre; the radius carries a relative
    // margin for the rounding of values and positions far from the field
    float esc[4];
    double rho = 0.0;
    for (int a = 0; a < 3; ++a) esc[a] = float(0.5 * (lo[a] + hi[a]));
    for (group const& g : gs) {
      double const dx = g.c[0] - esc[0], dy = g.c[1] - esc[1], dz = g.c[2] - esc[2];
      rho = std::fmax(rho, std::sqrt(dx * dx + dy * dy + dz * dz) + g.R);
    }
    esc[3] = float((rho + kmax + margin) * 1.001 + 1e-3);
    int esc_bits[4];
    std::memcpy(esc_bits, esc, sizeof esc_bits);
    out.hdr[4 * p + 3] = make_int4(esc_bits[0], esc_bits[1], esc_bits[2], esc_bits[3]);
    any = true;
  }
  if (!any) out = sdf_cells{};
}

}  // namespace myrt_b200
