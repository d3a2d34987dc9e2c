// Host analysis of flat SDF programs for the evaluator's exact skipping
// (sdf.cuh map): per instruction, the bounding sphere and extent of the group
// "translations, primitive, union / smooth union" that starts there.
#pragma once
#include <cmath>
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

}  // namespace myrt_b200
