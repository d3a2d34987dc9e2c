// CPU restatement of the post-processing passes (TEST INFRASTRUCTURE ONLY:
// the checker of myrt_b200/csrc/postprocess.cu; loaded by tests/ only).
//
// Follows the reference's shaders operation for operation:
//   denoise  src/pt/pp_denoise.comp:15-62 (normpdf, normpdf3, 9 x 9 bilateral)
//   blur     src/pt/pp_blur.comp:7-52 (31 taps, textureLod at pixel corners)
//   cutoff   src/pt/pp_cutoff.comp:12-31
//   add      src/pt/pp_add.comp:11-23
//   tonemap  src/pt/pp_tonemap.comp:8-30, src/pt/pp_tonemap_filmic.cl:1-15
//   fxaa     src/pt/pp_fxaa.comp:8-105
//   scale    src/pathtracer/post_process.cpp:112-127 (glBlitNamedFramebuffer,
//            GL_LINEAR: restated as bilinear sampling at destination pixel
//            centres with clamp-to-edge)
// with the sampling rules of the reference's sampler object
// (post_process.cpp:41-55, OpenGL 4.6 section 8.14.2): bilinear at level 0,
// GL_MIRRORED_REPEAT, and every pass storing RGBA16F (round to nearest even).
// Compiled with -ffp-contract=off: every + and * rounds separately.
#include "oracle_glsl_math.hpp"
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>

namespace {

struct f4 {
  float x, y, z, w;
};
struct img {
  f4 const* p;
  int w, h;
};

float half_rn(float f) {
  uint32_t x;
  std::memcpy(&x, &f, 4);
  uint32_t const sign = x & 0x80000000u, ax = x & 0x7fffffffu;
  if (ax >= 0x7f800000u) return f;  // inf, nan
  uint32_t r;
  if (ax >= 0x477ff000u) {
    r = 0x7f800000u;  // rounds past 65504: infinity
  } else if (ax < 0x38800000u) {  // below 2^-14: half subnormals, quantum 2^-24
    float a;
    std::memcpy(&a, &ax, 4);
    float const q = std::nearbyint(a * 16777216.f) * (1.f / 16777216.f);
    std::memcpy(&r, &q, 4);
  } else {
    uint32_t const lsb = (ax >> 13) & 1u;
    r = (ax + 0x0fffu + lsb) & ~0x1fffu;
  }
  r |= sign;
  float out;
  std::memcpy(&out, &r, 4);
  return out;
}
f4 store16(f4 v) { return {half_rn(v.x), half_rn(v.y), half_rn(v.z), half_rn(v.w)}; }
f4 add(f4 a, f4 b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
f4 mul(float s, f4 a) { return {s * a.x, s * a.y, s * a.z, s * a.w}; }
f4 fetch(img const& t, int x, int y) {
  if (x < 0 || y < 0 || x >= t.w || y >= t.h) return {0.f, 0.f, 0.f, 0.f};
  return t.p[size_t(y) * t.w + x];
}
int mirror_repeat(int i, int size) {
  int m = i % (2 * size);
  if (m < 0) m += 2 * size;
  int const a = m - size;
  int const mi = a >= 0 ? a : -(1 + a);
  return (size - 1) - mi;
}
int clamp_edge(int i, int size) { return i < 0 ? 0 : (i >= size ? size - 1 : i); }
f4 bilinear(img const& t, float s, float tt, bool mirrored) {
  float const u = s * float(t.w) - 0.5f, v = tt * float(t.h) - 0.5f;
  float const fu = std::floor(u), fv = std::floor(v);
  float const a = u - fu, b = v - fv;
  int const i0 = int(fu), j0 = int(fv);
  int x0, x1, y0, y1;
  if (mirrored) {
    x0 = mirror_repeat(i0, t.w), x1 = mirror_repeat(i0 + 1, t.w);
    y0 = mirror_repeat(j0, t.h), y1 = mirror_repeat(j0 + 1, t.h);
  } else {
    x0 = clamp_edge(i0, t.w), x1 = clamp_edge(i0 + 1, t.w);
    y0 = clamp_edge(j0, t.h), y1 = clamp_edge(j0 + 1, t.h);
  }
  float const w00 = (1.f - a) * (1.f - b), w10 = a * (1.f - b), w01 = (1.f - a) * b, w11 = a * b;
  f4 const t00 = t.p[size_t(y0) * t.w + x0], t10 = t.p[size_t(y0) * t.w + x1];
  f4 const t01 = t.p[size_t(y1) * t.w + x0], t11 = t.p[size_t(y1) * t.w + x1];
  return add(add(add(mul(w00, t00), mul(w10, t10)), mul(w01, t01)), mul(w11, t11));
}

float normpdf(float x, float sigma) { return 0.39894f * orc_glsl::exp(((-0.5f * x) * x) / (sigma * sigma)) / sigma; }
float normpdf3(float vx, float vy, float vz, float sigma) {
  float const d = (vx * vx + vy * vy) + vz * vz;
  return 0.39894f * orc_glsl::exp((-0.5f * d) / (sigma * sigma)) / sigma;
}
float clamp01(float v) { return std::fmin(std::fmax(v, 0.f), 1.f); }

f4 denoise(img const& in, int x, int y, float sigma, float bsigma) {
  constexpr int kSize = 4;
  float kernel[2 * kSize + 1];
  for (int j = 0; j <= kSize; ++j) kernel[kSize + j] = kernel[kSize - j] = normpdf(float(j), sigma);
  f4 const c = fetch(in, x, y);
  float Z = 0.f, fx = 0.f, fy = 0.f, fz = 0.f;
  float const bZ = 1.f / normpdf(0.f, bsigma);
  for (int i = -kSize; i <= kSize; ++i)
    for (int j = -kSize; j <= kSize; ++j) {
      int const sx = std::min(std::max(x + i, 0), in.w - 1), sy = std::min(std::max(y + j, 0), in.h - 1);
      f4 const t = fetch(in, sx, sy);
      float const cx = clamp01(t.x), cy = clamp01(t.y), cz = clamp01(t.z);
      float const factor = ((normpdf3(cx - c.x, cy - c.y, cz - c.z, bsigma) * bZ) * kernel[kSize + j]) * kernel[kSize + i];
      Z += factor;
      fx += factor * cx, fy += factor * cy, fz += factor * cz;
    }
  return {fx / Z, fy / Z, fz / Z, 1.f};
}

float const kBlur[16] = {0.08756118061424645f, 0.08547984344465417f, 0.07952880794840879f, 0.0705164133185798f,
    0.05958841266910679f, 0.04798885898065629f, 0.03683205838316095f, 0.0269412473017388f, 0.018780823225920923f,
    0.012477173150624141f, 0.007899915153736418f, 0.004766876346593609f, 0.0027412691146821303f,
    0.001502371210393176f, 0.0007847156649807812f, 0.0003906237796399568f};

f4 blur(img const& in, int x, int y, int direction, float step) {
  float const ix = 1.f / float(in.w), iy = 1.f / float(in.h);
  float const px = float(x), py = float(y);
  f4 r = mul(kBlur[0], bilinear(in, px * ix, py * iy, true));
  int const dir = direction != 0 ? 1 : 0;
  float const sx = float(1 - dir) * step, sy = float(dir) * step;
  for (int i = 1; i < 16; ++i) {
    float const fi = float(i);
    f4 const s0 = bilinear(in, (px + fi * sx) * ix, (py + fi * sy) * iy, true);
    f4 const s1 = bilinear(in, (px - fi * sx) * ix, (py - fi * sy) * iy, true);
    r = add(r, mul(kBlur[i], add(s0, s1)));
  }
  return r;
}

f4 cutoff(img const& in, int x, int y, float const* value, int leave_above) {
  f4 c = fetch(in, x, y);
  float* cv = &c.x;
  for (int k = 0; k < 4; ++k) {
    bool const zero = leave_above ? cv[k] <= value[k] : cv[k] >= value[k];
    if (zero) cv[k] = 0.f;
  }
  return c;
}

float filmic(float x) {
  float const X = std::fmax(0.f, x - 0.004f);
  float const r = (X * (6.2f * X + 0.5f)) / (X * (6.2f * X + 1.7f) + 0.06f);
  return orc_glsl::pow(r, 1.3f);
}

float luma(f4 c) { return (c.x * 0.299f + c.y * 0.587f) + c.z * 0.114f; }

f4 fxaa(img const& in, int x, int y) {
  float const rx = float(in.w), ry = float(in.h);
  float const ivx = 1.f / rx, ivy = 1.f / ry;
  float const fx = float(x), fy = float(y);
  f4 const nw = bilinear(in, (fx + -1.f) * ivx, (fy + -1.f) * ivy, true);
  f4 const ne = bilinear(in, (fx + 1.f) * ivx, (fy + -1.f) * ivy, true);
  f4 const sw = bilinear(in, (fx + -1.f) * ivx, (fy + 1.f) * ivy, true);
  f4 const se = bilinear(in, (fx + 1.f) * ivx, (fy + 1.f) * ivy, true);
  f4 const m = bilinear(in, fx * ivx, fy * ivy, true);
  float const lNW = luma(nw), lNE = luma(ne), lSW = luma(sw), lSE = luma(se), lM = luma(m);
  float const lMin = std::fmin(lM, std::fmin(std::fmin(lNW, lNE), std::fmin(lSW, lSE)));
  float const lMax = std::fmax(lM, std::fmax(std::fmax(lNW, lNE), std::fmax(lSW, lSE)));
  float dx = -((lNW + lNE) - (lSW + lSE));
  float dy = (lNW + lSW) - (lNE + lSE);
  float const reduce = std::fmax((((lNW + lNE) + lSW) + lSE) * (0.25f * (1.f / 8.f)), 1.f / 128.f);
  float const rcp = 1.f / (std::fmin(std::fabs(dx), std::fabs(dy)) + reduce);
  dx = std::fmin(8.f, std::fmax(-8.f, dx * rcp)) * ivx;
  dy = std::fmin(8.f, std::fmax(-8.f, dy * rcp)) * ivy;
  float const bx = fx * ivx, by = fy * ivy;
  float const k1 = 1.f / 3.f - 0.5f, k2 = 2.f / 3.f - 0.5f;
  f4 const rgbA = mul(0.5f, add(bilinear(in, bx + dx * k1, by + dy * k1, true), bilinear(in, bx + dx * k2, by + dy * k2, true)));
  f4 const rgbB = add(mul(0.5f, rgbA),
      mul(0.25f, add(bilinear(in, bx + dx * -0.5f, by + dy * -0.5f, true), bilinear(in, bx + dx * 0.5f, by + dy * 0.5f, true))));
  float const lB = luma(rgbB);
  f4 const c = (lB < lMin || lB > lMax) ? rgbA : rgbB;
  return {c.x, c.y, c.z, 1.f};
}

}  // namespace

// op: 0 denoise, 1 blur, 2 cutoff, 3 add, 4 tonemap, 5 fxaa, 6 scale (the
// myrt_pp_op numbering). Images are float RGBA, row-major.
extern "C" int oracle_post_pass(int op, int const* iparam, float const* fparam, float const* in, int w, int h,
    float const* overlay, int ow_, int oh_, float* out, int out_w, int out_h) {
  img const I{reinterpret_cast<f4 const*>(in), w, h};
  img const O{reinterpret_cast<f4 const*>(overlay), ow_, oh_};
  f4* dst = reinterpret_cast<f4*>(out);
  for (int y = 0; y < out_h; ++y)
    for (int x = 0; x < out_w; ++x) {
      f4 v{};
      switch (op) {
        case 0: v = denoise(I, x, y, fparam[0], fparam[1]); break;
        case 1: v = blur(I, x, y, iparam[0], fparam[0]); break;
        case 2: v = cutoff(I, x, y, fparam, iparam[0]); break;
        case 3: v = add(fetch(I, x, y), mul(fparam[0], bilinear(O, float(x) / float(w), float(y) / float(h), true))); break;
        case 4: {
          f4 const c = fetch(I, x, y);
          v = {filmic(c.x), filmic(c.y), filmic(c.z), iparam[0] ? 1.f : c.w};
          break;
        }
        case 5: v = fxaa(I, x, y); break;
        case 6: v = bilinear(I, (float(x) + 0.5f) / float(out_w), (float(y) + 0.5f) / float(out_h), false); break;
        default: return -1;
      }
      dst[size_t(y) * out_w + x] = store16(v);
    }
  return 0;
}

extern "C" float oracle_half_rn(float f) { return half_rn(f); }
