// Host check of the SDF cell tables (myrt_b200/csrc/sdf_skip.hpp): builds the
// tables the library uploads, then evaluates each program and sphere-traces
// seeded rays twice with the device evaluator's arithmetic restated on the host
// (sdf.cuh map / march, load == false, every + and * rounded separately):
// once in full and once as the device runs it (cell segments, the per-point
// bounding-sphere test and the escape sphere). It
// prints, per program, the grid, the number of points and marches whose
// results differ in any bit, and the instructions evaluated per march.
//
// Usage: sdf_cells_check <dir with instrs.bin programs.bin params.bin> <cells> <rays> <seed>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iterator>
#include <random>
#include <string>
#include <vector>

#include "../myrt_b200/csrc/sdf_skip.hpp"

using namespace myrt_b200;

namespace {

struct v3 {
  float x, y, z;
};
float gmin(float a, float b) { return b < a ? b : a; }
float gmax(float a, float b) { return a < b ? b : a; }
float gclamp(float v, float lo, float hi) { return gmin(gmax(v, lo), hi); }
float mixf(float a, float b, float t) { return a * (1.f - t) + b * t; }
float dot3(v3 a, v3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
float len3(v3 v) { return std::sqrt(dot3(v, v)); }
float len2(float x, float y) { return std::sqrt(x * x + y * y); }

template <class T> std::vector<T> read_all(std::string const& f) {
  std::ifstream s(f, std::ios::binary);
  std::vector<char> b((std::istreambuf_iterator<char>(s)), std::istreambuf_iterator<char>());
  std::vector<T> v(b.size() / sizeof(T));
  std::memcpy(v.data(), b.data(), v.size() * sizeof(T));
  return v;
}

std::vector<myrt_sdf_instr> I;
std::vector<myrt_sdf_program> P;
std::vector<float> G;
sdf_cells C;
std::vector<float4> skip_sphere;
std::vector<int2> skip_next;
long evaluated = 0;

float fbits(int b) {
  float f;
  std::memcpy(&f, &b, 4);
  return f;
}

float map(int prog, v3 p, bool cells) {
  myrt_sdf_program const pr = P[prog];
  float dist[64];
  int sp = 0;
  v3 pos = p;
  int kend = pr.count, li = 0, le = 0;
  bool const skipping = cells && !skip_next.empty();
  float const margin = 1e-4f + 1e-6f * ((std::fabs(p.x) + std::fabs(p.y)) + std::fabs(p.z));
  if (cells && !C.hdr.empty() && C.hdr[3 * prog + 1].x > 0) {
    int4 const h0 = C.hdr[3 * prog], h1 = C.hdr[3 * prog + 1];
    float const inv = fbits(h0.w);
    float const fx = (p.x - fbits(h0.x)) * inv, fy = (p.y - fbits(h0.y)) * inv, fz = (p.z - fbits(h0.z)) * inv;
    if (fx >= 0.f && fy >= 0.f && fz >= 0.f && fx < float(h1.x) && fy < float(h1.y) && fz < float(h1.z)) {
      int const c = h1.w + (int(fz) * h1.y + int(fy)) * h1.x + int(fx);
      li = C.start[c];
      le = C.start[c + 1];
      kend = 0;
    }
  }
  for (int k = 0;; ++k) {
    if (k >= kend) {
      if (li >= le) break;
      uint32_t const e = C.list[li++];
      k = int(e & 0xffffu);
      kend = int(e >> 16);
    }
    if (skipping) {  // the per-point bounding-sphere test, as the device runs it
      int2 const nx = skip_next[pr.first + k];
      if (nx.x > 0 && nx.x - pr.first <= kend) {
        float4 const b = skip_sphere[pr.first + k];
        float const thr = ((dist[sp - 1] + fbits(nx.y)) + b.w) + margin;
        float const qx = p.x - b.x, qy = p.y - b.y, qz = p.z - b.z;
        if (thr <= 0.f || (qx * qx + qy * qy) + qz * qz >= thr * thr) {
          k = nx.x - pr.first - 1;
          continue;
        }
      }
    }
    myrt_sdf_instr const in = I[pr.first + k];
    int const o = in.param_offset;
    float d = 0.f;
    ++evaluated;
    switch (in.op) {
      case MYRT_SDF_TRANSLATE:
        pos = {pos.x - G[o], pos.y - G[o + 1], pos.z - G[o + 2]};
        continue;
      case MYRT_SDF_SPHERE: d = len3(pos) - G[o]; break;
      case MYRT_SDF_BOX: {
        v3 const q{std::fabs(pos.x) - G[o], std::fabs(pos.y) - G[o + 1], std::fabs(pos.z) - G[o + 2]};
        d = len3({gmax(q.x, 0.f), gmax(q.y, 0.f), gmax(q.z, 0.f)}) + gmin(gmax(q.x, gmax(q.y, q.z)), 0.f);
        break;
      }
      case MYRT_SDF_TORUS: d = len2(len2(pos.x, pos.z) - G[o], pos.y) - G[o + 1]; break;
      case MYRT_SDF_CAPSULE: {
        v3 q = pos;
        q.y -= gclamp(q.y, 0.f, G[o]);
        d = len3(q) - G[o + 1];
        break;
      }
      case MYRT_SDF_UNION: case MYRT_SDF_SMOOTH_UNION: case MYRT_SDF_SUBTRACTION: case MYRT_SDF_INTERSECTION: {
        float const d1 = dist[sp - 1], d0 = dist[sp - 2];
        sp -= 2;
        if (in.op == MYRT_SDF_SMOOTH_UNION) {
          float const kk = G[o];
          float const h = gclamp(0.5f + 0.5f * (d1 - d0) / kk, 0.f, 1.f);
          d = mixf(d1, d0, h) - kk * h * (1.f - h);
        } else if (in.op == MYRT_SDF_UNION) {
          d = gmin(d0, d1);
        } else if (in.op == MYRT_SDF_SUBTRACTION) {
          d = gmax(-d0, d1);
        } else {
          d = gmax(d0, d1);
        }
        break;
      }
      default: std::fprintf(stderr, "opcode %d not restated here\n", in.op); std::exit(2);
    }
    dist[sp++] = d;
    pos = p;
  }
  return dist[sp - 1];
}

// raymarch.glsl:116-171 with the device's early exit when `cells`
bool march(int prog, v3 ro, v3 rd, float tmax, bool cells, float& t_hit) {
  float const len = len3(rd), eps = 1e-4f;
  float res = -1.f, t = 10.f * eps;
  int si = 0;
  float ex = 0.f, ey = 0.f, ez = 0.f, ew = -1.f;
  if (cells && !C.hdr.empty() && C.hdr[3 * prog + 1].x > 0) {
    int4 const e = C.hdr[3 * prog + 2];
    ex = fbits(e.x), ey = fbits(e.y), ez = fbits(e.z), ew = fbits(e.w) + eps;
  }
  for (int i = 0; i < 256 && t / len < tmax; i++) {
    v3 const q{ro.x + rd.x * t / len, ro.y + rd.y * t / len, ro.z + rd.z * t / len};
    float const m = map(prog, q, cells);
    if (si == 0) si = m > 0.f ? 1 : (m < 0.f ? -1 : 0);
    if (std::fabs(m) < eps) {
      res = t;
      break;
    }
    if (si > 0 && ew > 0.f) {
      v3 const w{q.x - ex, q.y - ey, q.z - ez};
      if (dot3(w, rd) >= 0.f && dot3(w, w) >= ew * ew) break;
    }
    t += float(si) * m;
  }
  t_hit = res;
  return res >= 0.f;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 5) return 2;
  std::string const dir = argv[1];
  I = read_all<myrt_sdf_instr>(dir + "/instrs.bin");
  P = read_all<myrt_sdf_program>(dir + "/programs.bin");
  G = read_all<float>(dir + "/params.bin");
  myrt_sdf_view v{};
  v.instrs = I.data();
  v.instr_count = I.size();
  v.programs = P.data();
  v.program_count = P.size();
  v.params = G.data();
  v.param_count = G.size();
  int const cells = std::atoi(argv[2]), n_rays = std::atoi(argv[3]);
  sdf_cell_tables(&v, cells, C);
  sdf_skip_tables(&v, skip_sphere, skip_next);
  std::mt19937 rng(unsigned(std::atoi(argv[4])));
  std::uniform_real_distribution<float> U(-2.5f, 2.5f), J(-0.3f, 0.3f);
  for (int prog = 0; prog < int(P.size()); ++prog) {
    int const grid = C.hdr.empty() ? 0 : C.hdr[3 * prog + 1].x;
    long bad_points = 0, points = 0, bad_marches = 0, hits = 0;
    long full_instr = 0, cell_instr = 0;
    for (int r = 0; r < n_rays; ++r) {
      v3 o{U(rng), U(rng), U(rng)}, d{U(rng), U(rng), U(rng)};
      if (r % 4 == 1) o = {0.4f * J(rng), 0.4f * J(rng), 0.4f * J(rng)};                 // inside the field
      if (r % 2 == 1) d = {-o.x + J(rng), -o.y + J(rng), -o.z + J(rng)};                  // aimed at it
      float const tmax = r % 3 == 0 ? 2.f : INFINITY;
      float ta, tb;
      long const e0 = evaluated;
      bool const a = march(prog, o, d, tmax, false, ta);
      long const e1 = evaluated;
      bool const b = march(prog, o, d, tmax, true, tb);
      full_instr += e1 - e0;
      cell_instr += evaluated - e1;
      hits += a;
      if (a != b || (a && std::memcmp(&ta, &tb, 4) != 0)) ++bad_marches;
      // the points of the full march, each evaluated both ways
      float const len = len3(d);
      float t = 1e-3f;
      for (int s = 0; s < 64 && t < 6.f; ++s) {
        v3 const q{o.x + d.x * t / len, o.y + d.y * t / len, o.z + d.z * t / len};
        float const fa = map(prog, q, false), fb = map(prog, q, true);
        ++points;
        if (std::memcmp(&fa, &fb, 4) != 0) ++bad_points;
        if (std::fabs(fa) < 1e-4f) break;
        t += std::fabs(fa);
      }
    }
    std::printf("%d %d %ld %ld %ld %ld %.1f %.1f\n", prog, grid, points, bad_points, hits, bad_marches,
        double(full_instr) / n_rays, double(cell_instr) / n_rays);
  }
  return 0;
}
