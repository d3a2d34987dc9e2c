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
std::vector<int> op_count;
long evaluated = 0, redos = 0;

// random.glsl's stream as the device restates it (refshade.cuh)
struct rng_t {
  uint32_t state;
  int prime;
};
uint32_t wang(uint32_t a) {
  a = (a ^ 61u) ^ (a >> 16);
  a = a + (a << 3);
  a = a ^ (a >> 4);
  a = a * 0x27d4eb2du;
  a = a ^ (a >> 15);
  return a;
}
float random_next(rng_t& r) {
  r.prime = r.prime == 5 ? 0 : r.prime + 1;
  r.state += wang(uint32_t(r.prime));
  r.state ^= (r.state << 13);
  r.state ^= (r.state >> 17);
  r.state ^= (r.state << 5);
  return gclamp(float(r.state) * (1.f / 4294967296.f), 0.f, 1.f);
}
// the state before random_next, given the state after it
rng_t random_prev(rng_t r) {
  uint32_t x = r.state;
  x ^= (x << 5) ^ (x << 10) ^ (x << 15) ^ (x << 20) ^ (x << 25) ^ (x << 30);
  x ^= (x >> 17);
  x ^= (x << 13) ^ (x << 26);
  x -= wang(uint32_t(r.prime));
  return rng_t{x, r.prime == 0 ? 5 : r.prime - 1};
}

float fbits(int b) {
  float f;
  std::memcpy(&f, &b, 4);
  return f;
}

float map(int prog, v3 p, bool cells, bool load = false, rng_t* rng = nullptr, int* mat = nullptr) {
  myrt_sdf_program const pr = P[prog];
  float dist[64];
  int mats[64];
  int sp = 0;
  v3 pos = p;
  int kend = pr.count, li = 0, le = 0;
  bool const counting = cells && load && !op_count.empty();
  bool const skipping = cells && (!load || counting) && !skip_next.empty();
  float const margin = 1e-4f + 1e-6f * ((std::fabs(p.x) + std::fabs(p.y)) + std::fabs(p.z));
  if (cells && (!load || counting) && !C.hdr.empty() && C.hdr[3 * prog + 1].x > 0) {
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
  rng_t const saved = counting ? *rng : rng_t{};
  bool redo = false;
  auto draw_gap = [&](int a, int b) {
    if (b <= a) return;
    int const n = op_count[pr.first + b - 1] - (a > 0 ? op_count[pr.first + a - 1] : 0);
    for (int i = 0; i < n; ++i)
      if (random_next(*rng) >= 1.f) redo = true;
  };
  int const cell_li = li, cell_le = le, cell_kend = kend;
  for (int pass = 0;; ++pass) {
  bool const fast = pass == 0;
  kend = fast ? cell_kend : pr.count;
  li = fast ? cell_li : 0;
  le = fast ? cell_le : 0;
  int drawn = 0;
  sp = 0;
  pos = p;
  for (int k = 0;; ++k) {
    if (k >= kend) {
      if (li >= le) break;
      uint32_t const e = C.list[li++];
      k = int(e & 0xffffu);
      kend = int(e >> 16);
      if (counting) draw_gap(drawn, k);
    }
    if (skipping && fast) {  // the per-point bounding-sphere test, as the device runs it
      int2 const nx = skip_next[pr.first + k];
      if (nx.x > 0 && nx.x - pr.first <= kend) {
        float4 const b = skip_sphere[pr.first + k];
        float const thr = ((dist[sp - 1] + fbits(nx.y)) + b.w) + margin;
        float const qx = p.x - b.x, qy = p.y - b.y, qz = p.z - b.z;
        if (thr <= 0.f || (qx * qx + qy * qy) + qz * qz >= thr * thr) {
          if (counting) draw_gap(k, nx.x - pr.first);
          drawn = nx.x - pr.first;
          k = nx.x - pr.first - 1;
          continue;
        }
      }
    }
    drawn = k + 1;
    myrt_sdf_instr const in = I[pr.first + k];
    int const o = in.param_offset;
    float d = 0.f;
    int m = -1;
    ++evaluated;
    switch (in.op) {
      case MYRT_SDF_TRANSLATE:
        pos = {pos.x - G[o], pos.y - G[o + 1], pos.z - G[o + 2]};
        continue;
      case MYRT_SDF_SPHERE: m = int(G[o + 1]); d = len3(pos) - G[o]; break;
      case MYRT_SDF_BOX: {
        m = int(G[o + 3]);
        v3 const q{std::fabs(pos.x) - G[o], std::fabs(pos.y) - G[o + 1], std::fabs(pos.z) - G[o + 2]};
        d = len3({gmax(q.x, 0.f), gmax(q.y, 0.f), gmax(q.z, 0.f)}) + gmin(gmax(q.x, gmax(q.y, q.z)), 0.f);
        break;
      }
      case MYRT_SDF_TORUS: m = int(G[o + 2]); d = len2(len2(pos.x, pos.z) - G[o], pos.y) - G[o + 1]; break;
      case MYRT_SDF_CAPSULE: {
        m = int(G[o + 2]);
        v3 q = pos;
        q.y -= gclamp(q.y, 0.f, G[o]);
        d = len3(q) - G[o + 1];
        break;
      }
      case MYRT_SDF_UNION: case MYRT_SDF_SMOOTH_UNION: case MYRT_SDF_SUBTRACTION: case MYRT_SDF_INTERSECTION: {
        float const d1 = dist[sp - 1], d0 = dist[sp - 2];
        int const m1 = mats[sp - 1], m0 = mats[sp - 2];
        sp -= 2;
        float t;
        if (in.op == MYRT_SDF_SMOOTH_UNION) {
          float const kk = G[o];
          float const h = gclamp(0.5f + 0.5f * (d1 - d0) / kk, 0.f, 1.f);
          t = 1.f - h;
          d = mixf(d1, d0, h) - kk * h * (1.f - h);
        } else {
          float const r = in.op == MYRT_SDF_UNION ? gmin(d0, d1)
                                                  : (in.op == MYRT_SDF_SUBTRACTION ? gmax(-d0, d1) : gmax(d0, d1));
          t = float(r == d1);
          d = r;
        }
        if (load) m = random_next(*rng) < t ? m1 : m0;
        break;
      }
      default: std::fprintf(stderr, "opcode %d not restated here\n", in.op); std::exit(2);
    }
    dist[sp] = d;
    mats[sp] = m;
    ++sp;
    pos = p;
  }
  if (counting && fast) draw_gap(drawn, pr.count);
  if (!redo) break;
  ++redos;
  *rng = saved;
  redo = false;
  }
  if (mat) *mat = mats[sp - 1];
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
  sdf_op_counts(&v, op_count);
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
    // material loads: distance, material and the random state after the call,
    // at points near the surfaces; then with a draw of exactly 1 planted at
    // each of the first 64 draw positions in turn
    long load_points = 0, bad_loads = 0, bad_forced = 0, redo_before = redos;
    for (int r = 0; r < n_rays / 4; ++r) {
      v3 o{U(rng), U(rng), U(rng)};
      v3 d{-o.x + J(rng), -o.y + J(rng), -o.z + J(rng)};
      float const len = len3(d);
      float t = 1e-3f, fa = 1.f;
      v3 q = o;
      for (int s = 0; s < 64 && t < 6.f; ++s) {  // march to near a surface
        q = {o.x + d.x * t / len, o.y + d.y * t / len, o.z + d.z * t / len};
        fa = map(prog, q, false);
        if (std::fabs(fa) < 1e-3f) break;
        t += std::fabs(fa);
      }
      rng_t const start{uint32_t(rng()), int(rng() % 6)};
      rng_t ra = start, rb = start;
      int ma = -7, mb = -7;
      float const la = map(prog, q, false, true, &ra, &ma), lb = map(prog, q, true, true, &rb, &mb);
      ++load_points;
      if (std::memcmp(&la, &lb, 4) != 0 || ma != mb || ra.state != rb.state || ra.prime != rb.prime) ++bad_loads;
      if (r % 8 == 0) {
        for (int j = 0; j < 64; ++j) {
          rng_t one{0xffffffc0u, int(rng() % 6)};  // random_next returns exactly 1 for this state
          rng_t s0 = one;
          for (int i = 0; i < j + 1; ++i) s0 = random_prev(s0);  // j draws before it
          rng_t fa2 = s0, fb2 = s0;
          int m1 = -7, m2 = -7;
          float const x1 = map(prog, q, false, true, &fa2, &m1), x2 = map(prog, q, true, true, &fb2, &m2);
          if (std::memcmp(&x1, &x2, 4) != 0 || m1 != m2 || fa2.state != fb2.state || fa2.prime != fb2.prime)
            ++bad_forced;
        }
      }
    }
    std::fprintf(stderr, "prog %d loads %ld bad %ld forced-one bad %ld redos %ld\n", prog, load_points, bad_loads,
        bad_forced, redos - redo_before);
    std::printf("%d %d %ld %ld %ld %ld %.1f %.1f %ld %ld %ld %ld\n", prog, grid, points, bad_points, hits, bad_marches,
        double(full_instr) / n_rays, double(cell_instr) / n_rays, load_points, bad_loads, bad_forced,
        redos - redo_before);
  }
  return 0;
}
