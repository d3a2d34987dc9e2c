// Post-processing passes on device images: the reference's compute shaders
// src/pt/pp_denoise.comp, pp_blur.comp, pp_cutoff.comp, pp_add.comp,
// pp_tonemap.comp (= src/pt/pp_tonemap_filmic.cl), pp_fxaa.comp, and the
// linear_scale blit of src/pathtracer/post_process.cpp:112-127.
//
// Images are float4 (RGBA) in device memory, row-major. As in the reference,
// where every pass writes an RGBA16F image, each pass rounds its output to
// half precision (round to nearest even) and keeps it as float.
//
// Texture reads follow the OpenGL 4.6 sampling rules the reference's sampler
// sets up (post_process.cpp:41-55): texelFetch reads one texel (0 outside the
// image); texture / textureLod at level 0 filter bilinearly (GL_LINEAR: texel
// coordinates u = s W - 1/2, weights from the fractional parts) with
// GL_MIRRORED_REPEAT wrapping. The weighted sum is
// ((w00 t00 + w10 t10) + w01 t01) + w11 t11 with w00 = (1 - a)(1 - b),
// w10 = a (1 - b), w01 = (1 - a) b, w11 = a b. The linear_scale blit samples
// the source at the destination pixel centres with the same filter and
// clamp-to-edge wrapping. This unit is compiled without FMA contraction, and
// the exp / pow of denoise and tonemap are the library's GLSL built-ins
// (glmath.hpp), so a host restatement reproduces every pass bit for bit.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cmath>

#include "../../include/myrt_cuda.h"
#include "ctx.hpp"
#include "glmath.hpp"

namespace myrt_b200 {
namespace {

struct img_in {
  float4 const* p;
  int w, h;
};

__device__ __forceinline__ float half_rn(float x) { return __half2float(__float2half_rn(x)); }
__device__ __forceinline__ float4 store16(float4 v) {
  return make_float4(half_rn(v.x), half_rn(v.y), half_rn(v.z), half_rn(v.w));
}
__device__ __forceinline__ float4 fetch(img_in const& t, int x, int y) {
  if (x < 0 || y < 0 || x >= t.w || y >= t.h) return make_float4(0.f, 0.f, 0.f, 0.f);
  return t.p[size_t(y) * t.w + x];
}
__device__ __forceinline__ int mirror_repeat(int i, int size) {
  if (unsigned(i) < unsigned(size)) return i;  // in range: the mapping below gives i itself
  int m = i % (2 * size);
  if (m < 0) m += 2 * size;
  int const a = m - size;
  int const mi = a >= 0 ? a : -(1 + a);
  return (size - 1) - mi;
}
__device__ __forceinline__ int clamp_edge(int i, int size) { return i < 0 ? 0 : (i >= size ? size - 1 : i); }
__device__ __forceinline__ float4 f4add(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
__device__ __forceinline__ float4 f4mul(float s, float4 a) { return make_float4(s * a.x, s * a.y, s * a.z, s * a.w); }

// GL_LINEAR at level 0; mirrored = GL_MIRRORED_REPEAT, else clamp to edge
__device__ __forceinline__ float4 bilinear(img_in const& t, float s, float tt, bool mirrored) {
  float const u = s * float(t.w) - 0.5f, v = tt * float(t.h) - 0.5f;
  float const fu = floorf(u), fv = floorf(v);
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
  float4 const t00 = t.p[size_t(y0) * t.w + x0], t10 = t.p[size_t(y0) * t.w + x1];
  float4 const t01 = t.p[size_t(y1) * t.w + x0], t11 = t.p[size_t(y1) * t.w + x1];
  return f4add(f4add(f4add(f4mul(w00, t00), f4mul(w10, t10)), f4mul(w01, t01)), f4mul(w11, t11));
}

struct pass_args {
  img_in in, ov;
  float4* out;
  int ow, oh;
  int i0;
  float p[4];
};

// pp_denoise.comp: bilateral filter, 9 x 9 window (MSIZE 10), spatial sigma
// = exponent, range sigma = strength.
__device__ __forceinline__ float normpdf(float x, float sigma) {
  return 0.39894f * myrt_glmath::exp(((-0.5f * x) * x) / (sigma * sigma)) / sigma;
}
__device__ __forceinline__ float normpdf3(float3 v, float sigma) {
  float const d = (v.x * v.x + v.y * v.y) + v.z * v.z;
  return 0.39894f * myrt_glmath::exp((-0.5f * d) / (sigma * sigma)) / sigma;
}
__global__ void k_pp_denoise(pass_args a) {
  int const x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= a.ow || y >= a.oh) return;
  constexpr int kSize = 4;
  float kernel[2 * kSize + 1];
  for (int j = 0; j <= kSize; ++j) kernel[kSize + j] = kernel[kSize - j] = normpdf(float(j), a.p[0]);
  float4 const c4 = fetch(a.in, x, y);
  float3 const c{c4.x, c4.y, c4.z};
  float Z = 0.f;
  float3 fc{0.f, 0.f, 0.f};
  float const bZ = 1.f / normpdf(0.f, a.p[1]);
  for (int i = -kSize; i <= kSize; ++i)
    for (int j = -kSize; j <= kSize; ++j) {
      int const sx = min(max(x + i, 0), a.in.w - 1), sy = min(max(y + j, 0), a.in.h - 1);
      float4 const t = fetch(a.in, sx, sy);
      float3 const cc{fminf(fmaxf(t.x, 0.f), 1.f), fminf(fmaxf(t.y, 0.f), 1.f), fminf(fmaxf(t.z, 0.f), 1.f)};
      float const factor =
          ((normpdf3(float3{cc.x - c.x, cc.y - c.y, cc.z - c.z}, a.p[1]) * bZ) * kernel[kSize + j]) * kernel[kSize + i];
      Z += factor;
      fc.x += factor * cc.x, fc.y += factor * cc.y, fc.z += factor * cc.z;
    }
  a.out[size_t(y) * a.ow + x] = store16(make_float4(fc.x / Z, fc.y / Z, fc.z / Z, 1.f));
}

// pp_blur.comp: 31-tap Gaussian along x (direction 0) or y, taps `step` apart.
__constant__ float kBlur[16] = {0.08756118061424645f, 0.08547984344465417f, 0.07952880794840879f,
    0.0705164133185798f, 0.05958841266910679f, 0.04798885898065629f, 0.03683205838316095f, 0.0269412473017388f,
    0.018780823225920923f, 0.012477173150624141f, 0.007899915153736418f, 0.004766876346593609f,
    0.0027412691146821303f, 0.001502371210393176f, 0.0007847156649807812f, 0.0003906237796399568f};
__global__ void k_pp_blur(pass_args a) {
  int const x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= a.ow || y >= a.oh) return;
  float const ix = 1.f / float(a.in.w), iy = 1.f / float(a.in.h);
  float const px = float(x), py = float(y);
  float4 r = f4mul(kBlur[0], bilinear(a.in, px * ix, py * iy, true));
  int const dir = a.i0 != 0 ? 1 : 0;
  float const sx = float(1 - dir) * a.p[0], sy = float(dir) * a.p[0];
  for (int i = 1; i < 16; ++i) {
    float const fi = float(i);
    float4 const s0 = bilinear(a.in, (px + fi * sx) * ix, (py + fi * sy) * iy, true);
    float4 const s1 = bilinear(a.in, (px - fi * sx) * ix, (py - fi * sy) * iy, true);
    r = f4add(r, f4mul(kBlur[i], f4add(s0, s1)));
  }
  a.out[size_t(y) * a.ow + x] = store16(r);
}

// pp_cutoff.comp: zero every channel <= value (leave_above) or >= value.
__global__ void k_pp_cutoff(pass_args a) {
  int const x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= a.ow || y >= a.oh) return;
  float4 c = fetch(a.in, x, y);
  float* cv = &c.x;
  for (int k = 0; k < 4; ++k) {
    bool const zero = a.i0 ? cv[k] <= a.p[k] : cv[k] >= a.p[k];
    if (zero) cv[k] = 0.f;
  }
  a.out[size_t(y) * a.ow + x] = store16(c);
}

// pp_add.comp: color + factor * overlay sampled at pixel / size.
__global__ void k_pp_add(pass_args a) {
  int const x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= a.ow || y >= a.oh) return;
  float4 const c = fetch(a.in, x, y);
  float4 const o = bilinear(a.ov, float(x) / float(a.in.w), float(y) / float(a.in.h), true);
  a.out[size_t(y) * a.ow + x] = store16(f4add(c, f4mul(a.p[0], o)));
}

// pp_tonemap.comp / pp_tonemap_filmic.cl: filmic curve, pow 1.3; alpha kept
// (the GLSL pass) or set to 1 (the OpenCL kernel main.cpp runs): i0 = 1.
__device__ __forceinline__ float filmic(float x) {
  float const X = fmaxf(0.f, x - 0.004f);
  float const r = (X * (6.2f * X + 0.5f)) / (X * (6.2f * X + 1.7f) + 0.06f);
  return myrt_glmath::pow(r, 1.3f);
}
__global__ void k_pp_tonemap(pass_args a) {
  int const x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= a.ow || y >= a.oh) return;
  float4 const c = fetch(a.in, x, y);
  a.out[size_t(y) * a.ow + x] = store16(make_float4(filmic(c.x), filmic(c.y), filmic(c.z), a.i0 ? 1.f : c.w));
}

// pp_fxaa.comp: the "mobile" FXAA variant (reduce min 1/128, mul 1/8, span 8).
__device__ __forceinline__ float luma(float4 c) { return (c.x * 0.299f + c.y * 0.587f) + c.z * 0.114f; }
__global__ void k_pp_fxaa(pass_args a) {
  int const x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= a.ow || y >= a.oh) return;
  float const rx = float(a.in.w), ry = float(a.in.h);
  float const ivx = 1.f / rx, ivy = 1.f / ry;
  float const fx = float(x), fy = float(y);
  float4 const nw = bilinear(a.in, (fx + -1.f) * ivx, (fy + -1.f) * ivy, true);
  float4 const ne = bilinear(a.in, (fx + 1.f) * ivx, (fy + -1.f) * ivy, true);
  float4 const sw = bilinear(a.in, (fx + -1.f) * ivx, (fy + 1.f) * ivy, true);
  float4 const se = bilinear(a.in, (fx + 1.f) * ivx, (fy + 1.f) * ivy, true);
  float4 const m = bilinear(a.in, fx * ivx, fy * ivy, true);
  float const lNW = luma(nw), lNE = luma(ne), lSW = luma(sw), lSE = luma(se), lM = luma(m);
  float const lMin = fminf(lM, fminf(fminf(lNW, lNE), fminf(lSW, lSE)));
  float const lMax = fmaxf(lM, fmaxf(fmaxf(lNW, lNE), fmaxf(lSW, lSE)));
  float dx = -((lNW + lNE) - (lSW + lSE));
  float dy = (lNW + lSW) - (lNE + lSE);
  float const reduce = fmaxf((((lNW + lNE) + lSW) + lSE) * (0.25f * (1.f / 8.f)), 1.f / 128.f);
  float const rcp = 1.f / (fminf(fabsf(dx), fabsf(dy)) + reduce);
  dx = fminf(8.f, fmaxf(-8.f, dx * rcp)) * ivx;
  dy = fminf(8.f, fmaxf(-8.f, dy * rcp)) * ivy;
  float const bx = fx * ivx, by = fy * ivy;
  float const k1 = 1.f / 3.f - 0.5f, k2 = 2.f / 3.f - 0.5f;
  float4 const a1 = bilinear(a.in, bx + dx * k1, by + dy * k1, true);
  float4 const a2 = bilinear(a.in, bx + dx * k2, by + dy * k2, true);
  float4 const rgbA = f4mul(0.5f, f4add(a1, a2));
  float4 const b1 = bilinear(a.in, bx + dx * -0.5f, by + dy * -0.5f, true);
  float4 const b2 = bilinear(a.in, bx + dx * 0.5f, by + dy * 0.5f, true);
  float4 const rgbB = f4add(f4mul(0.5f, rgbA), f4mul(0.25f, f4add(b1, b2)));
  float const lB = luma(rgbB);
  float4 const c = (lB < lMin || lB > lMax) ? rgbA : rgbB;
  a.out[size_t(y) * a.ow + x] = store16(make_float4(c.x, c.y, c.z, 1.f));
}

// linear_scale: bilinear resample (clamp to edge) at destination pixel centres.
__global__ void k_pp_scale(pass_args a) {
  int const x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= a.ow || y >= a.oh) return;
  float const s = (float(x) + 0.5f) / float(a.ow), t = (float(y) + 0.5f) / float(a.oh);
  a.out[size_t(y) * a.ow + x] = store16(bilinear(a.in, s, t, false));
}

}  // namespace
}  // namespace myrt_b200

using namespace myrt_b200;

extern "C" int myrt_post_pass(myrt_ctx* ctx, myrt_pp_pass const* pass, myrt_image const* in, myrt_image const* overlay,
    myrt_image const* out, void* stream) {
  if (!ctx) return MYRT_ERR_INVALID_ARGUMENT;
  if (!pass || !in || !out || !in->rgba || !out->rgba || in->width == 0 || in->height == 0 || out->width == 0 ||
      out->height == 0)
    return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "post pass needs an input and an output image");
  if (in->width > 65536 || in->height > 65536 || out->width > 65536 || out->height > 65536)
    return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "post pass image larger than 65536 pixels a side");
  if (pass->op != MYRT_PP_SCALE && (out->width != in->width || out->height != in->height))
    return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "post pass output must have the input's size");
  if (pass->op == MYRT_PP_ADD && (!overlay || !overlay->rgba || overlay->width == 0 || overlay->height == 0))
    return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "add pass needs an overlay image");
  if (pass->op == MYRT_PP_DENOISE && !(pass->p[0] != 0.f && pass->p[1] != 0.f))
    return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "denoise sigmas must be non-zero");
  int rc = check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  if (rc) return rc;
  pass_args a{};
  a.in = img_in{reinterpret_cast<float4 const*>(in->rgba), int(in->width), int(in->height)};
  if (overlay && overlay->rgba)
    a.ov = img_in{reinterpret_cast<float4 const*>(overlay->rgba), int(overlay->width), int(overlay->height)};
  a.out = reinterpret_cast<float4*>(out->rgba);
  a.ow = int(out->width);
  a.oh = int(out->height);
  a.i0 = pass->i[0];
  for (int k = 0; k < 4; ++k) a.p[k] = pass->p[k];
  cudaStream_t const st = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
  dim3 const block(16, 16);
  dim3 const grid((out->width + 15) / 16, (out->height + 15) / 16);
  switch (pass->op) {
    case MYRT_PP_DENOISE: k_pp_denoise<<<grid, block, 0, st>>>(a); break;
    case MYRT_PP_BLUR: k_pp_blur<<<grid, block, 0, st>>>(a); break;
    case MYRT_PP_CUTOFF: k_pp_cutoff<<<grid, block, 0, st>>>(a); break;
    case MYRT_PP_ADD: k_pp_add<<<grid, block, 0, st>>>(a); break;
    case MYRT_PP_TONEMAP: k_pp_tonemap<<<grid, block, 0, st>>>(a); break;
    case MYRT_PP_FXAA: k_pp_fxaa<<<grid, block, 0, st>>>(a); break;
    case MYRT_PP_SCALE: k_pp_scale<<<grid, block, 0, st>>>(a); break;
    default: return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "unknown post pass");
  }
  return check_cuda(ctx, cudaGetLastError(), "post pass launch");
}
