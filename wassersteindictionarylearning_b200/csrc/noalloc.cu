// wdl_convolve_device_noalloc: the separable operator for callers that must not
// allocate device memory while they run — real-time or embedded hosts that
// reserve all memory up front, and processes running under a device-memory cap
// or a strict pool, where a cudaMalloc would fail, stall on a device-wide
// synchronisation, or break the caller's memory budget.
//
// The regular entry point (wdl_convolve_device) takes its scratch from the
// context's grow-only arena, which calls cudaMalloc the first time a size is
// seen.  This variant takes its scratch from the fixed array below instead and
// calls no allocating routine.  The caller still passes device pointers for
// the input and output.
//
// The array lives in the library's module, and CUDA loads a module on a
// device the first time something in it is used.  wdl_create therefore looks
// up the array's device address (noalloc_attach), which loads the module and
// reserves the kNoAllocScratchBytes on that device when the context is
// created, never inside a call of the entry point; the device keeps them until
// the process exits.  The address is kept per context, so a context created
// after the device's primary context was reset sees the array where the
// reloaded module put it.  All calls share the array, so calls that overlap on
// the GPU (different streams, or different host threads) race on it; serialise
// them.  Each call writes every scratch element it reads before reading it, so
// the array's previous contents never matter and nothing needs clearing.
#include "wdl_internal.cuh"

namespace wdl {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

template <typename T>
__global__ void k_noalloc_in(const double* __restrict__ in, T* __restrict__ out, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = (T)in[i];
}
template <typename T>
__global__ void k_noalloc_out(const T* __restrict__ in, double* __restrict__ out, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = (double)in[i];
}

inline size_t round256(size_t b) { return (b + 255) & ~size_t(255); }

template <typename T>
int convolve_noalloc_t(wdl_ctx* ctx, const double* u, double* out, int nv, cudaStream_t s) {
  const size_t n = (size_t)nv * ctx->N;
  const size_t part = round256(n * sizeof(T));
  if (3 * part > kNoAllocScratchBytes) {
    const size_t max_images = kNoAllocScratchBytes / (3 * round256(ctx->N * sizeof(T)));
    return set_error(ctx, WDL_ERR_INVALID_ARG,
                     "wdl_convolve_device_noalloc: " + std::to_string(nv) + " images need " +
                         std::to_string(3 * part) + " bytes of scratch; the fixed scratch holds " +
                         std::to_string(kNoAllocScratchBytes) + " bytes (at most " +
                         std::to_string(max_images) + " images of this grid)");
  }
  void* base = ctx->noalloc_scratch;
  if (!base) return set_error(ctx, WDL_ERR_CUDA, "no-allocation scratch array not attached");
  int rc;
  T* a = reinterpret_cast<T*>(base);
  T* b = reinterpret_cast<T*>(static_cast<char*>(base) + part);
  T* t = reinterpret_cast<T*>(static_cast<char*>(base) + 2 * part);
  const unsigned grid = grid_for(n, 256, ctx->sm_count);
  k_noalloc_in<T><<<grid, 256, 0, s>>>(u, a, n);
  WDL_LAUNCH_CHECK(ctx);
  if ((rc = conv_stack<T>(ctx, a, b, t, (size_t)nv, s))) return rc;
  k_noalloc_out<T><<<grid, 256, 0, s>>>(b, out, n);
  WDL_LAUNCH_CHECK(ctx);
  return WDL_OK;
}

}  // namespace

// In host code g_noalloc_scratch is only a host-side stand-in for the device
// symbol; its device address is looked up here, once per context, with the
// context's device current.
int noalloc_attach(wdl_ctx* ctx) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return cuda_error(ctx, e, "cudaGetSymbolAddress(g_noalloc_scratch)");
  ctx->noalloc_scratch = p;
  return WDL_OK;
}

}  // namespace wdl

extern "C" int wdl_convolve_device_noalloc(wdl_ctx* ctx, const double* u, double* out,
                                           int nvectors, void* stream) {
  if (!ctx) return WDL_ERR_INVALID_ARG;
  if (!u || !out || nvectors < 0)
    return wdl::set_error(ctx, WDL_ERR_INVALID_ARG, "bad arguments");
  if (nvectors == 0) return WDL_OK;
  if (cudaSetDevice(ctx->device) != cudaSuccess)
    return wdl::set_error(ctx, WDL_ERR_CUDA, "cudaSetDevice failed");
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
  return ctx->precision == WDL_FP64 ? wdl::convolve_noalloc_t<double>(ctx, u, out, nvectors, s)
                                    : wdl::convolve_noalloc_t<float>(ctx, u, out, nvectors, s);
}
