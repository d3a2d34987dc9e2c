// Learned path guiding (host side and kernels): placeholder until the MLP lands.
#include "ctx.hpp"
#include "guide.cuh"

namespace myrt_b200 {

int guide_prepare(myrt_ctx* ctx, size_t, myrt_render_params const*, guide_dev& g) {
  g = guide_dev{};
  return set_error(ctx, MYRT_ERR_UNSUPPORTED, "guided shading is not available");
}
int guide_infer(myrt_ctx*, guide_dev const&, uint32_t, uint32_t, float4 const*, float4 const*, uint32_t const*,
    cudaStream_t) {
  return MYRT_OK;
}
int guide_train(myrt_ctx*, guide_dev const&, uint32_t, int, float4 const*, cudaStream_t) { return MYRT_OK; }

}  // namespace myrt_b200
