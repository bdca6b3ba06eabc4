// Tensor-core (tcgen05) forms of the separable Gaussian operator and the FP32
// operator dispatch.
#include "wdl_internal.cuh"

namespace wdl {

struct TcResources {
  int dummy = 0;
};

bool tc_supported(const wdl_ctx* ctx) { return false && ctx; }

int tc_init(wdl_ctx* ctx) {
  return set_error(ctx, WDL_ERR_UNSUPPORTED, "tensor-core operator not built yet");
}

void tc_free(wdl_ctx* ctx) {
  delete ctx->tc;
  ctx->tc = nullptr;
}

int conv_stack_f32(wdl_ctx* ctx, const float* in, float* out, float* tmp, size_t nimg,
                   cudaStream_t s) {
  if (ctx->precision == WDL_FP32) return conv_stack_simt_f32(ctx, in, out, tmp, nimg, s);
  return set_error(ctx, WDL_ERR_UNSUPPORTED, "tensor-core operator not available");
}

}  // namespace wdl
