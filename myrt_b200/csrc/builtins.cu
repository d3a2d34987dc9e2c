// myrt_glsl_builtins: the library's GLSL built-ins (glmath.hpp) evaluated on
// the device, so a caller -- or a test -- can check that a host build of the
// same header reproduces the shading's transcendentals bit for bit.
#include <cuda_runtime.h>

#include "../../include/myrt_cuda.h"
#include "ctx.hpp"
#include "glmath.hpp"

namespace myrt_b200 {
namespace {
__global__ void k_glsl_builtin(int fn, float const* __restrict__ x, float const* __restrict__ y, uint32_t n,
    float* __restrict__ out) {
  uint32_t const i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float const a = x[i];
  float r;
  switch (fn) {
    case MYRT_GLSL_SIN: r = myrt_glmath::sin(a); break;
    case MYRT_GLSL_COS: r = myrt_glmath::cos(a); break;
    case MYRT_GLSL_ATAN: r = myrt_glmath::atan(a); break;
    case MYRT_GLSL_EXP: r = myrt_glmath::exp(a); break;
    default: r = myrt_glmath::pow(a, y[i]); break;
  }
  out[i] = r;
}
}  // namespace
}  // namespace myrt_b200

extern "C" int myrt_glsl_builtins(myrt_ctx* ctx, int fn, const float* x, const float* y, uint32_t n, float* out) {
  using namespace myrt_b200;
  if (!ctx) return MYRT_ERR_INVALID_ARGUMENT;
  if (fn < MYRT_GLSL_SIN || fn > MYRT_GLSL_POW) return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "unknown built-in");
  if (n == 0) return MYRT_OK;
  if (!x || !out || (fn == MYRT_GLSL_POW && !y))
    return set_error(ctx, MYRT_ERR_INVALID_ARGUMENT, "null input or output");
  int rc = check_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  if (rc) return rc;
  size_t const bytes = size_t(n) * sizeof(float);
  float* d = nullptr;
  rc = check_cuda(ctx, cudaMalloc(&d, 3 * bytes), "built-in buffers");
  if (rc) return rc;
  cudaStream_t const s = ctx->stream;
  rc = check_cuda(ctx, cudaMemcpyAsync(d, x, bytes, cudaMemcpyHostToDevice, s), "upload");
  if (!rc && y) rc = check_cuda(ctx, cudaMemcpyAsync(d + n, y, bytes, cudaMemcpyHostToDevice, s), "upload");
  if (!rc) {
    k_glsl_builtin<<<(n + 255) / 256, 256, 0, s>>>(fn, d, d + n, n, d + 2 * size_t(n));
    rc = check_cuda(ctx, cudaGetLastError(), "built-in launch");
  }
  if (!rc) rc = check_cuda(ctx, cudaMemcpyAsync(out, d + 2 * size_t(n), bytes, cudaMemcpyDeviceToHost, s), "read");
  if (!rc) rc = check_cuda(ctx, cudaStreamSynchronize(s), "built-ins");
  cudaFree(d);
  return rc;
}
