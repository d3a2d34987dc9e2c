// CPU oracle: restatement of the reference's ray-query algorithms.
//
// TEST INFRASTRUCTURE ONLY. Only tests/, the smoke check and bench.py's
// CPU-baseline leg load this library, as the checker. The product never
// calls it. Built with -ffp-contract=off -fwrapv (oracle/build.py).
//
// Pinning: these restatements are checked in tests/ against golden vectors
// produced by the reference's own code compiled in oracle/_ref (bvh.cpp,
// intersect.glsl, bvh.impl.glsl, pt_trace.comp's visitor), committed under
// tests/golden/.
//
// Contents (each cites what it follows):
//   orc_isect_reference   src/pt/intersect.glsl:3-28 (== bvh.cpp:514-538)
//   orc_isect_watertight  Woop, Benthin, Wald, JCGT 2(1) 2013 (same op order as
//                         the device kernel)
//   orc_refbvh_build      src/pathtracer/bvh.cpp:43-116, :136-161, :356-512 with
//                         dont_split (no primitive splitting)
//   orc_refbvh_traverse   src/pt/bvh.impl.glsl:8-72 + pt_trace.comp:259-282
//                         (first visited wins ties) and a canonical variant
//   orc_instanced_query   src/pt/pt_trace.comp:284-309 (visit_object_aabb): object-space
//                         walks of every drawable's geometry tree, canonical ties
//   orc_bvh8_traverse     the device traversal of the 8-wide tree, instrumented
//                         (nodes fetched, triangles tested per ray)
//   orc_brute_closest     all-triangle closest hit, canonical ties
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

namespace {

struct v3 {
  float x, y, z;
};
inline v3 sub(v3 a, v3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline float dot(v3 a, v3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline v3 cross(v3 a, v3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline float comp(v3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }

// intersect.glsl:3-28
bool isect_reference(v3 o, v3 d, v3 v1, v3 v2, v3 v3_, float& t, float& u, float& v) {
  float const float_epsilon = 1e-23f;
  float const border_epsilon = 1e-6f;
  v3 const e1 = sub(v2, v1);
  v3 const e2 = sub(v3_, v1);
  v3 const P = cross(d, e2);
  float const det = dot(e1, P);
  if (det > -float_epsilon && det < float_epsilon) return false;
  float const inv_det = 1.0f / det;
  v3 const T = sub(o, v1);
  u = dot(T, P) * inv_det;
  if (u < -border_epsilon || u > 1.0f + border_epsilon) return false;
  v3 const Q = cross(T, e1);
  v = dot(d, Q) * inv_det;
  if (v < -border_epsilon || u + v > 1.0f + border_epsilon) return false;
  float const tt = dot(e2, Q) * inv_det;
  if (tt > float_epsilon) {
    t = tt;
    return true;
  }
  return false;
}

struct wt_ray {
  int kx, ky, kz;
  float Sx, Sy, Sz;
};
wt_ray wt_setup(v3 d) {
  wt_ray w;
  float const ax = std::fabs(d.x), ay = std::fabs(d.y), az = std::fabs(d.z);
  w.kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
  w.kx = w.kz + 1 == 3 ? 0 : w.kz + 1;
  w.ky = w.kx + 1 == 3 ? 0 : w.kx + 1;
  if (comp(d, w.kz) < 0.0f) std::swap(w.kx, w.ky);
  float const dz = comp(d, w.kz);
  w.Sx = comp(d, w.kx) / dz;
  w.Sy = comp(d, w.ky) / dz;
  w.Sz = 1.0f / dz;
  return w;
}
bool isect_watertight(wt_ray const& w, v3 o, v3 v0, v3 v1, v3 v2, float tmin, float& t, float& u, float& v) {
  v3 const A = sub(v0, o), B = sub(v1, o), C = sub(v2, o);
  float const Az0 = comp(A, w.kz), Bz0 = comp(B, w.kz), Cz0 = comp(C, w.kz);
  float const Ax = comp(A, w.kx) - w.Sx * Az0, Ay = comp(A, w.ky) - w.Sy * Az0;
  float const Bx = comp(B, w.kx) - w.Sx * Bz0, By = comp(B, w.ky) - w.Sy * Bz0;
  float const Cx = comp(C, w.kx) - w.Sx * Cz0, Cy = comp(C, w.ky) - w.Sy * Cz0;
  float U = Cx * By - Cy * Bx;
  float V = Ax * Cy - Ay * Cx;
  float W = Bx * Ay - By * Ax;
  if (U == 0.0f || V == 0.0f || W == 0.0f) {
    U = float(double(Cx) * double(By) - double(Cy) * double(Bx));
    V = float(double(Ax) * double(Cy) - double(Ay) * double(Cx));
    W = float(double(Bx) * double(Ay) - double(By) * double(Ax));
  }
  if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
  float const det = (U + V) + W;
  if (det == 0.0f) return false;
  float const Az = w.Sz * Az0, Bz = w.Sz * Bz0, Cz = w.Sz * Cz0;
  float const T = (U * Az + V * Bz) + W * Cz;
  float const rcp = 1.0f / det;
  float const tt = T * rcp;
  if (!(tt > 0.0f) || tt < tmin) return false;
  t = tt;
  u = V * rcp;
  v = W * rcp;
  return true;
}

struct ray8 {
  v3 o;
  float tmin;
  v3 d;
  float tmax;
};
inline ray8 load_ray(float const* q) { return {{q[0], q[1], q[2]}, q[3], {q[4], q[5], q[6]}, q[7]}; }

// One triangle test with the acceptance rule of the device kernel.
inline bool test_tri(int isect, wt_ray const& wt, ray8 const& r, v3 p0, v3 p1, v3 p2, float& t, float& u, float& v) {
  if (isect == 0) return isect_reference(r.o, r.d, p0, p1, p2, t, u, v) && t >= r.tmin;
  return isect_watertight(wt, r.o, p0, p1, p2, r.tmin, t, u, v);
}
inline bool canonical_better(float t, std::int32_t prim, float tbest, std::int32_t best) {
  return t < tbest || (t == tbest && best >= 0 && prim < best);
}

template <typename F> void parallel_for(std::size_t n, int nthreads, F&& f) {
  if (nthreads <= 1 || n < 4096) {
    f(std::size_t(0), n);
    return;
  }
  std::vector<std::thread> th;
  std::size_t const per = (n + std::size_t(nthreads) - 1) / std::size_t(nthreads);
  for (int i = 0; i < nthreads; ++i) {
    std::size_t const b = std::size_t(i) * per, e = std::min(n, b + per);
    if (b < e) th.emplace_back([&f, b, e] { f(b, e); });
  }
  for (auto& x : th) x.join();
}

// ---- restated reference binary BVH (bvh.cpp) -------------------------------
struct aabb {
  v3 mn{std::numeric_limits<float>::max(), std::numeric_limits<float>::max(), std::numeric_limits<float>::max()};
  v3 mx{std::numeric_limits<float>::lowest(), std::numeric_limits<float>::lowest(),
      std::numeric_limits<float>::lowest()};
  v3 centroid{0, 0, 0};
  void enclose(v3 p) {
    mn = {std::min(mn.x, p.x), std::min(mn.y, p.y), std::min(mn.z, p.z)};
    mx = {std::max(mx.x, p.x), std::max(mx.y, p.y), std::max(mx.z, p.z)};
  }
  void enclose(aabb const& b) {
    mn = {std::min(mn.x, b.mn.x), std::min(mn.y, b.mn.y), std::min(mn.z, b.mn.z)};
    mx = {std::max(mx.x, b.mx.x), std::max(mx.y, b.mx.y), std::max(mx.z, b.mx.z)};
  }
  v3 dim() const { return sub(mx, mn); }
  float area() const {  // bvh.hpp:44-47
    v3 const d = dim();
    return ((d.x + d.y) * d.z + (d.x * d.y)) * 2.f;
  }
};

struct ref_node {  // bvh.hpp:98-139 layout
  float mn[3];
  std::uint32_t type_and_parent;
  float mx[3];
  std::uint32_t first, second;
  std::uint32_t pad[3];
};
static_assert(sizeof(ref_node) == 48);

// float -> int the way the x86 reference build truncates (cvttss2si: out of
// range or NaN gives INT_MIN).
inline int trunc_int(float f) {
  if (!(f > -2147483648.0f && f < 2147483648.0f)) return std::numeric_limits<int>::min();
  return int(f);
}

struct refbvh_builder {
  std::vector<aabb> aabbs;
  std::vector<std::uint32_t> idx;
  std::vector<ref_node> nodes;
  aabb full;

  // bvh.cpp:43-116 (including its prefix/suffix pairing as written)
  void split_axis(ref_node const& node, int& best_axis_out, float& plane, bool& should) {
    constexpr int B = 16;
    aabb sub_aabb;
    for (std::uint32_t i = node.first; i <= node.second; ++i) sub_aabb.enclose(aabbs[i].centroid);
    v3 const size = sub_aabb.dim();
    v3 const step{size.x / float(B), size.y / float(B), size.z / float(B)};
    std::array<std::array<aabb, B>, 3> bins{};
    std::array<std::array<int, B>, 3> counts{};
    for (std::uint32_t i = node.first; i <= node.second; ++i) {
      v3 const c = aabbs[i].centroid;
      v3 const rel = sub(c, sub_aabb.mn);
      int const id[3] = {std::clamp(trunc_int(rel.x / step.x), 0, B - 1), std::clamp(trunc_int(rel.y / step.y), 0, B - 1),
          std::clamp(trunc_int(rel.z / step.z), 0, B - 1)};
      for (int a = 0; a < 3; ++a) {
        bins[a][id[a]].enclose(aabbs[i]);
        counts[a][id[a]]++;
      }
    }
    std::array<std::array<aabb, B>, 3> acc{}, accr{};
    std::array<std::array<int, B>, 3> accc{};
    for (int a = 0; a < 3; ++a) {
      aabb run;
      for (int k = 0; k < B; ++k) {
        if (k == 0) run = bins[a][0];
        else run.enclose(bins[a][k]);
        acc[a][k] = run;
      }
      aabb runr;
      for (int k = B - 1; k >= 0; --k) {
        if (k == B - 1) runr = bins[a][B - 1];
        else runr.enclose(bins[a][k]);
        accr[a][k] = runr;
      }
      int c = 0;
      for (int k = 0; k < B; ++k) {
        c += counts[a][k];
        accc[a][k] = c;
      }
    }
    aabb nb;
    nb.mn = {node.mn[0], node.mn[1], node.mn[2]};
    nb.mx = {node.mx[0], node.mx[1], node.mx[2]};
    float const total_area = nb.area();
    float best_cost = std::numeric_limits<float>::max();
    int best_axis = 0, best_part = 0;
    for (int a = 0; a < 3; ++a) {
      for (int k = 0; k < B - 1; ++k) {
        int const cf = accc[a][k];
        int const cs = accc[a][B - 1 - k];
        float const af = acc[a][k].area();
        float const as = accr[a][k].area();
        float const cost = 7.f + 2.f * (float(cf) * (af / total_area) + float(cs) * (as / total_area));
        if (cost <= best_cost) {
          best_axis = a;
          best_part = k;
          best_cost = cost;
        }
      }
    }
    float const total_count = float(accc[best_axis][B - 1]);
    float const without = 2.f * total_count;
    plane = comp(sub_aabb.mn, best_axis) + comp(step, best_axis) * float(best_part + 1);
    best_axis_out = best_axis;
    should = best_cost < without;
  }

  // bvh.cpp:408-512 with dont_split (no primitive is ever duplicated)
  bool split(ref_node const& node, ref_node& l, ref_node& r) {
    if (node.second - node.first < 1) return false;
    int axis;
    float plane;
    bool should;
    split_axis(node, axis, plane, should);
    if (!should) return false;
    auto test = [&](std::uint32_t i) { return comp(aabbs[i].centroid, axis) < plane; };
    std::uint32_t first = node.first;
    std::uint32_t const last = node.second + 1;
    while (first != last && test(first)) first++;
    if (first != last) {
      for (std::uint32_t i = first; i != last; ++i) {
        if (test(i)) {
          std::swap(idx[i], idx[first]);
          std::swap(aabbs[i], aabbs[first]);
          ++first;
        }
      }
    }
    std::uint32_t const split_index = first == node.first ? first + 1 : first;
    l = ref_node{};
    r = ref_node{};
    l.first = node.first;
    l.second = split_index - 1;
    r.first = split_index;
    r.second = node.second;
    for (ref_node* c : {&l, &r}) {
      aabb b;
      for (std::uint32_t i = c->first; i <= c->second; ++i) b.enclose(aabbs[i]);
      c->mn[0] = b.mn.x, c->mn[1] = b.mn.y, c->mn[2] = b.mn.z;
      c->mx[0] = b.mx.x, c->mx[1] = b.mx.y, c->mx[2] = b.mx.z;
    }
    return true;
  }

  // bvh.cpp:356-407
  void create() {
    std::uint32_t const n = std::uint32_t(aabbs.size());
    idx.resize(n);
    for (std::uint32_t i = 0; i < n; ++i) idx[i] = i;
    nodes.reserve(2 * std::size_t(n));
    ref_node root{};
    root.mn[0] = full.mn.x, root.mn[1] = full.mn.y, root.mn[2] = full.mn.z;
    root.mx[0] = full.mx.x, root.mx[1] = full.mx.y, root.mx[2] = full.mx.z;
    root.type_and_parent = 0x80000000u;
    root.first = 0;
    root.second = n - 1;
    nodes.push_back(root);
    for (std::size_t cur = 0; cur < nodes.size(); ++cur) {
      ref_node l, r;
      ref_node const node = nodes[cur];
      if (split(node, l, r)) {
        nodes[cur].first = std::uint32_t(nodes.size());
        nodes[cur].second = std::uint32_t(nodes.size() + 1);
        nodes[cur].type_and_parent &= 0x7fffffffu;
        l.type_and_parent = 0x80000000u | std::uint32_t(cur);
        r.type_and_parent = 0x80000000u | std::uint32_t(cur);
        nodes.push_back(l);
        nodes.push_back(r);
      }
    }
  }
};

struct refbvh {
  std::vector<ref_node> nodes;
  std::vector<std::uint32_t> idx;
};

// bvh.glsl:31-45
inline bool slab(ref_node const& n, v3 o, v3 id, float mt, float& t) {
  v3 const t135{(n.mn[0] - o.x) * id.x, (n.mn[1] - o.y) * id.y, (n.mn[2] - o.z) * id.z};
  v3 const t246{(n.mx[0] - o.x) * id.x, (n.mx[1] - o.y) * id.y, (n.mx[2] - o.z) * id.z};
  // GLSL min/max: min(a, b) = b < a ? b : a
  auto mn = [](float a, float b) { return b < a ? b : a; };
  auto mx = [](float a, float b) { return a < b ? b : a; };
  v3 const minv{mn(t135.x, t246.x), mn(t135.y, t246.y), mn(t135.z, t246.z)};
  v3 const maxv{mx(t135.x, t246.x), mx(t135.y, t246.y), mx(t135.z, t246.z)};
  float const tmin = mx(mx(minv.x, minv.y), minv.z);
  float const tmax = mn(mn(maxv.x, maxv.y), maxv.z);
  if (tmax >= 0 && tmin <= tmax && tmin <= mt) {
    t = tmin;
    return true;
  }
  t = mt;
  return false;
}

}  // namespace

extern "C" {

// ---- intersectors -----------------------------------------------------------
int orc_isect_reference(float const* o, float const* d, float const* tri, float* t, float* uv) {
  float tt = 0, u = 0, v = 0;
  bool const h = isect_reference({o[0], o[1], o[2]}, {d[0], d[1], d[2]}, {tri[0], tri[1], tri[2]},
      {tri[3], tri[4], tri[5]}, {tri[6], tri[7], tri[8]}, tt, u, v);
  *t = tt;
  uv[0] = u;
  uv[1] = v;
  return h;
}

// ---- restated reference binary BVH ------------------------------------------
void* orc_refbvh_build(std::uint32_t const* indices, std::size_t n_indices, float const* points_xyz) {
  auto* out = new refbvh;
  refbvh_builder b;
  std::size_t const n = n_indices / 3;
  b.aabbs.resize(n);
  for (std::size_t i = 0; i < n; ++i) {  // bvh.cpp:136-152
    v3 p[3];
    for (int k = 0; k < 3; ++k) {
      float const* q = points_xyz + 3 * std::size_t(indices[3 * i + k]);
      p[k] = {q[0], q[1], q[2]};
    }
    aabb& a = b.aabbs[i];
    for (auto& q : p) a.enclose(q);
    a.mn = {a.mn.x - 1e-5f, a.mn.y - 1e-5f, a.mn.z - 1e-5f};
    a.mx = {a.mx.x + 1e-5f, a.mx.y + 1e-5f, a.mx.z + 1e-5f};
    v3 const s{(p[0].x + p[1].x) + p[2].x, (p[0].y + p[1].y) + p[2].y, (p[0].z + p[1].z) + p[2].z};
    a.centroid = {s.x / 3.0f, s.y / 3.0f, s.z / 3.0f};
    b.full.enclose(a);
  }
  if (n > 0) b.create();
  out->nodes = std::move(b.nodes);
  out->idx = std::move(b.idx);
  return out;
}
void orc_refbvh_free(void* h) { delete static_cast<refbvh*>(h); }
std::size_t orc_refbvh_node_count(void* h) { return static_cast<refbvh*>(h)->nodes.size(); }
void orc_refbvh_nodes(void* h, void* out) {
  auto const& n = static_cast<refbvh*>(h)->nodes;
  std::memcpy(out, n.data(), n.size() * sizeof(ref_node));
}
void orc_refbvh_indices(void* h, std::uint32_t* out) {
  auto const& r = static_cast<refbvh*>(h)->idx;
  std::memcpy(out, r.data(), r.size() * sizeof(std::uint32_t));
}

// bvh.impl.glsl:8-72 with the pt_trace.comp visitor. nodes: 48-byte records.
// canonical = 0: first visited wins ties (the reference); 1: smaller prim wins.
void orc_refbvh_query(void const* nodes_v, std::uint32_t const* bvh_idx, std::uint32_t const* indices,
    float const* points_xyzw, float const* rays, std::size_t n, int any_hit, int canonical, int isect,
    std::int32_t* prim, float* t_out, float* u_out, float* v_out, int nthreads);

void orc_refbvh_traverse(void const* nodes_v, std::uint32_t const* bvh_idx, std::uint32_t const* indices,
    float const* points_xyzw, float const* rays, std::size_t n, int any_hit, int canonical, std::int32_t* prim,
    float* t_out, float* u_out, float* v_out, int nthreads) {
  orc_refbvh_query(nodes_v, bvh_idx, indices, points_xyzw, rays, n, any_hit, canonical, -1, prim, t_out, u_out, v_out,
      nthreads);
}

}  // extern "C"

namespace {
struct query_hit {
  bool found;
  std::int32_t prim;
  float t, u, v;
};

// One ray through one reference tree (bvh.impl.glsl:8-72 + the pt_trace.comp
// visitor). Node child / parent indices and triangle indices are relative to
// the arrays passed in (the reference's node_base / primitive_base scheme).
query_hit refbvh_closest(ref_node const* nodes, std::uint32_t const* bvh_idx, std::uint32_t const* indices,
    float const* points_xyzw, ray8 const& ray, int any_hit, int canonical, int isect) {
  auto pt = [points_xyzw](std::uint32_t i) {
    return v3{points_xyzw[4 * i], points_xyzw[4 * i + 1], points_xyzw[4 * i + 2]};
  };
  v3 const ro = ray.o, rd = ray.d;
  wt_ray const wt = wt_setup(rd);
  v3 const inv{1.0f / rd.x, 1.0f / rd.y, 1.0f / rd.z};
  float maxt = ray.tmax;
  float best_t = ray.tmax, bu = 0, bv = 0;
  std::int32_t best = -1;
  bool found = false;
  std::uint32_t visited = 0, lr = 0, node_index = 0;
  float tmp;
  bool hits_any = slab(nodes[0], ro, inv, maxt, tmp);
  bool done = false;
  while (hits_any && !done) {
    ref_node current = nodes[node_index];
    while (!(current.type_and_parent & 0x80000000u)) {
      float tl, tr;
      ref_node const& fc = nodes[current.first];
      ref_node const& sc = nodes[current.second];
      bool const hl = slab(fc, ro, inv, maxt, tl);
      bool const hr = slab(sc, ro, inv, maxt, tr);
      if (!hl && !hr) break;
      bool const use_right = !hl || (hr && tl >= tr);
      lr = std::uint32_t(use_right) | (lr << 1);
      visited = std::uint32_t(hl && hr) | (visited << 1);
      node_index = use_right ? current.second : current.first;
      current = nodes[node_index];
    }
    if (current.type_and_parent & 0x80000000u) {
      for (std::uint32_t tri = current.first; tri <= current.second; ++tri) {
        std::uint32_t const pi = bvh_idx[tri];
        float t, u, v;
        bool h = isect < 0 ? isect_reference(ro, rd, pt(indices[3 * pi]), pt(indices[3 * pi + 1]),
                                 pt(indices[3 * pi + 2]), t, u, v)
                           : test_tri(isect, wt, ray, pt(indices[3 * pi]), pt(indices[3 * pi + 1]),
                                 pt(indices[3 * pi + 2]), t, u, v);
        h = h && t < maxt && (canonical ? canonical_better(t, std::int32_t(pi), best_t, best) : best_t > t);
        if (h) {
          best_t = t;
          bu = u;
          bv = v;
          best = std::int32_t(pi);
          found = true;
          maxt = canonical ? std::nextafter(t, std::numeric_limits<float>::infinity()) : t;
          if (any_hit) {
            done = true;
            break;
          }
        }
      }
      if (done) break;
    }
    while ((visited & 1u) != 1u) {
      if (visited == 0) {
        done = true;
        break;
      }
      node_index = nodes[node_index].type_and_parent & 0x7fffffffu;
      visited >>= 1;
      lr >>= 1;
    }
    if (done) break;
    std::uint32_t const parent = nodes[node_index].type_and_parent & 0x7fffffffu;
    node_index = (lr & 1u) ? nodes[parent].first : nodes[parent].second;
    visited ^= 1u;
  }
  return {found, found ? best : -1, found ? best_t : ray.tmax, found ? bu : 0.f, found ? bv : 0.f};
}

// GLSL's (m * vec4(v, w)).xyz for a column-major mat4: products and sums
// rounded one by one, left to right.
inline v3 mat4_apply(float const* m, v3 p, float w) {
  return {((m[0] * p.x + m[4] * p.y) + m[8] * p.z) + m[12] * w, ((m[1] * p.x + m[5] * p.y) + m[9] * p.z) + m[13] * w,
      ((m[2] * p.x + m[6] * p.y) + m[10] * p.z) + m[14] * w};
}
}  // namespace

extern "C" {

// isect -1: the reference's traversal as written (Moller-Trumbore, no tmin
// test); 0 / 1: Moller-Trumbore / watertight with the device kernels'
// acceptance rule (t >= tmin, t < tmax).
void orc_refbvh_query(void const* nodes_v, std::uint32_t const* bvh_idx, std::uint32_t const* indices,
    float const* points_xyzw, float const* rays, std::size_t n, int any_hit, int canonical, int isect,
    std::int32_t* prim, float* t_out, float* u_out, float* v_out, int nthreads) {
  auto const* nodes = static_cast<ref_node const*>(nodes_v);
  parallel_for(n, nthreads, [&](std::size_t b, std::size_t e) {
    for (std::size_t r = b; r < e; ++r) {
      query_hit const q =
          refbvh_closest(nodes, bvh_idx, indices, points_xyzw, load_ray(rays + 8 * r), any_hit, canonical, isect);
      prim[r] = q.prim;
      t_out[r] = q.t;
      u_out[r] = q.u;
      v_out[r] = q.v;
    }
  });
}

// Instanced scenes, src/pt/pt_trace.comp:284-309 (visit_object_aabb) under
// the two-level walk: for every drawable, the ray moved into object space by
// inverse_transformation (origin with w = 1, direction with w = 0, not
// renormalised) walks that drawable's geometry tree (node and index bases
// bvh_node_base_index / bvh_index_base_index of the drawable record, vertices
// at points_base_index, indices at indices_base_index, as the reference
// addresses them). Every drawable is visited (no tree over the instances: a
// tree only decides which instances are skipped, never the answer). Closest
// hit keeps the smallest t, ties to the smaller global prim id (drawable's
// first prim + the triangle's index in its geometry); any hit answers whether
// some t in [tmin, tmax) exists. drawables: 40 words each (myrt_drawable).
void orc_instanced_query(void const* nodes_v, std::uint32_t const* bvh_idx, std::uint32_t const* indices,
    float const* points_xyzw, void const* drawables_v, std::size_t n_drawables, float const* rays, std::size_t n,
    int any_hit, int isect, std::int32_t* prim, float* t_out, float* u_out, float* v_out, int nthreads) {
  auto const* nodes = static_cast<ref_node const*>(nodes_v);
  auto const* dw = static_cast<std::uint32_t const*>(drawables_v);
  std::vector<std::int32_t> prim_base(n_drawables);
  std::int64_t acc = 0;
  for (std::size_t i = 0; i < n_drawables; ++i) {
    prim_base[i] = std::int32_t(acc);
    acc += dw[40 * i + 36] / 3;
  }
  parallel_for(n, nthreads, [&](std::size_t b, std::size_t e) {
    for (std::size_t r = b; r < e; ++r) {
      ray8 const ray = load_ray(rays + 8 * r);
      query_hit best{false, -1, ray.tmax, 0.f, 0.f};
      for (std::size_t i = 0; i < n_drawables; ++i) {
        std::uint32_t const* d = dw + 40 * i;
        if (d[36] == 0) continue;
        float inv[16];
        std::memcpy(inv, d + 16, 64);
        ray8 const obj{mat4_apply(inv, ray.o, 1.0f), ray.tmin, mat4_apply(inv, ray.d, 0.0f), ray.tmax};
        query_hit const q = refbvh_closest(nodes + d[32], bvh_idx + d[33], indices + d[34], points_xyzw + 4 * size_t(d[35]),
            obj, any_hit, 1, isect);
        if (!q.found) continue;
        std::int32_t const gp = prim_base[i] + q.prim;
        if (any_hit) {
          best = {true, gp, q.t, q.u, q.v};
          break;
        }
        if (!best.found || canonical_better(q.t, gp, best.t, best.prim)) best = {true, gp, q.t, q.u, q.v};
      }
      prim[r] = best.found ? best.prim : -1;
      t_out[r] = best.found ? best.t : ray.tmax;
      u_out[r] = best.found ? best.u : 0.f;
      v_out[r] = best.found ? best.v : 0.f;
    }
  });
}

// ---- the device's 8-wide traversal, instrumented ----------------------------
// nodes: 20 uint32 per node; tris: 12 floats per triangle (v0, prim bits, v1, -, v2, -).
void orc_bvh8_traverse(std::uint32_t const* nodes, float const* tris, float const* rays, std::size_t n, int any_hit,
    int isect, std::int32_t* prim, float* t_out, float* u_out, float* v_out, std::uint32_t* n_nodes,
    std::uint32_t* n_tris, std::uint8_t* occluded, int nthreads) {
  parallel_for(n, nthreads, [&](std::size_t b, std::size_t e) {
    for (std::size_t r = b; r < e; ++r) {
      ray8 const ray = load_ray(rays + 8 * r);
      v3 const o = ray.o, d = ray.d;
      float const idx = 1.0f / (std::fabs(d.x) > 1e-20f ? d.x : std::copysign(1e-20f, d.x));
      float const idy = 1.0f / (std::fabs(d.y) > 1e-20f ? d.y : std::copysign(1e-20f, d.y));
      float const idz = 1.0f / (std::fabs(d.z) > 1e-20f ? d.z : std::copysign(1e-20f, d.z));
      std::uint32_t const oct = (d.x < 0.f ? 1u : 0u) | (d.y < 0.f ? 2u : 0u) | (d.z < 0.f ? 4u : 0u);
      std::uint32_t const octinv = oct ^ 7u;
      wt_ray const wt = wt_setup(d);
      float tbest = ray.tmax, bu = 0, bv = 0;
      std::int32_t best = -1;
      std::uint32_t cn = 0, ct = 0;
      bool occ = false;
      std::uint32_t stack_x[64], stack_y[64];
      int sp = 0;
      std::uint32_t gx = 0, gy = 0x80000000u;
      while (true) {
        std::uint32_t tx = 0, ty = 0;
        if (gy & 0xff000000u) {
          std::uint32_t const pos = 31u - std::uint32_t(__builtin_clz(gy & 0xff000000u));
          gy &= ~(1u << pos);
          std::uint32_t const slot = (pos - 24u) ^ octinv;
          std::uint32_t const node_idx = gx + std::uint32_t(__builtin_popcount(gy & 0xffu & ((1u << slot) - 1u)));
          if (gy & 0xff000000u) {
            stack_x[sp] = gx;
            stack_y[sp] = gy;
            ++sp;
          }
          std::uint32_t const* w = nodes + 20 * std::size_t(node_idx);
          ++cn;
          auto f = [](std::uint32_t u) {
            float x;
            std::memcpy(&x, &u, 4);
            return x;
          };
          float const sx = f((w[3] & 0xffu) << 23) * idx;
          float const sy = f(((w[3] >> 8) & 0xffu) << 23) * idy;
          float const sz = f(((w[3] >> 16) & 0xffu) << 23) * idz;
          float const ox = (f(w[0]) - o.x) * idx, oy = (f(w[1]) - o.y) * idy, oz = (f(w[2]) - o.z) * idz;
          std::uint32_t const imask = w[3] >> 24;
          auto const* q = reinterpret_cast<std::uint8_t const*>(w + 8);  // qlo[3][8], qhi[3][8]
          auto const* meta = reinterpret_cast<std::uint8_t const*>(w + 6);
          std::uint32_t hit_internal = 0, hit_tris = 0;
          for (int s = 0; s < 8; ++s) {
            float const lx = q[0 * 8 + s], ly = q[1 * 8 + s], lz = q[2 * 8 + s];
            float const hx = q[3 * 8 + s], hy = q[4 * 8 + s], hz = q[5 * 8 + s];
            float const nx = idx >= 0.f ? lx : hx, fx = idx >= 0.f ? hx : lx;
            float const ny = idy >= 0.f ? ly : hy, fy = idy >= 0.f ? hy : ly;
            float const nz = idz >= 0.f ? lz : hz, fz = idz >= 0.f ? hz : lz;
            float const tnx = std::fma(nx, sx, ox), tfx = std::fma(fx, sx, ox);
            float const tny = std::fma(ny, sy, oy), tfy = std::fma(fy, sy, oy);
            float const tnz = std::fma(nz, sz, oz), tfz = std::fma(fz, sz, oz);
            float const tn = std::fmax(std::fmax(tnx, tny), std::fmax(tnz, ray.tmin));
            float const tf = std::fmin(std::fmin(tfx, tfy), std::fmin(tfz, tbest));
            std::uint32_t const m = meta[s];
            if (m != 0u && tn <= tf * 1.00000024f) {
              if (imask & (1u << s)) hit_internal |= 1u << ((std::uint32_t(s) ^ octinv) + 24u);
              else hit_tris |= ((1u << (m >> 5)) - 1u) << (m & 31u);
            }
          }
          gx = w[4];
          gy = hit_internal | imask;
          tx = w[5];
          ty = hit_tris;
        } else {
          gy = 0;
        }
        while (ty) {
          std::uint32_t const bit = std::uint32_t(__builtin_ctz(ty));
          ty &= ty - 1u;
          float const* tp = tris + 12 * std::size_t(tx + bit);
          ++ct;
          float t, u, v;
          bool const h = test_tri(isect, wt, ray, {tp[0], tp[1], tp[2]}, {tp[4], tp[5], tp[6]},
              {tp[8], tp[9], tp[10]}, t, u, v);
          if (!h) continue;
          std::int32_t pid;
          std::memcpy(&pid, tp + 3, 4);
          if (any_hit) {
            if (t < ray.tmax) {
              occ = true;
              break;
            }
          } else if (canonical_better(t, pid, tbest, best)) {
            tbest = t;
            best = pid;
            bu = u;
            bv = v;
          }
        }
        if (any_hit && occ) break;
        if (!(gy & 0xff000000u)) {
          if (sp == 0) break;
          --sp;
          gx = stack_x[sp];
          gy = stack_y[sp];
        }
      }
      if (any_hit) {
        if (occluded) occluded[r] = occ ? 1 : 0;
      } else {
        prim[r] = best;
        t_out[r] = best >= 0 ? tbest : ray.tmax;
        u_out[r] = best >= 0 ? bu : 0.f;
        v_out[r] = best >= 0 ? bv : 0.f;
      }
      if (n_nodes) n_nodes[r] = cn;
      if (n_tris) n_tris[r] = ct;
    }
  });
}

// ---- brute force ---------------------------------------------------------
// tris9: 9 floats per triangle; prim id = triangle index.
void orc_brute_closest(float const* tris9, std::size_t n_tris, float const* rays, std::size_t n, int isect,
    std::int32_t* prim, float* t_out, float* u_out, float* v_out, int nthreads) {
  parallel_for(n, nthreads, [&](std::size_t b, std::size_t e) {
    for (std::size_t r = b; r < e; ++r) {
      ray8 const ray = load_ray(rays + 8 * r);
      wt_ray const wt = wt_setup(ray.d);
      float tbest = ray.tmax, bu = 0, bv = 0;
      std::int32_t best = -1;
      for (std::size_t i = 0; i < n_tris; ++i) {
        float const* p = tris9 + 9 * i;
        float t, u, v;
        if (!test_tri(isect, wt, ray, {p[0], p[1], p[2]}, {p[3], p[4], p[5]}, {p[6], p[7], p[8]}, t, u, v)) continue;
        if (canonical_better(t, std::int32_t(i), tbest, best)) {
          tbest = t;
          best = std::int32_t(i);
          bu = u;
          bv = v;
        }
      }
      prim[r] = best;
      t_out[r] = best >= 0 ? tbest : ray.tmax;
      u_out[r] = best >= 0 ? bu : 0.f;
      v_out[r] = best >= 0 ? bv : 0.f;
    }
  });
}

}  // extern "C"
