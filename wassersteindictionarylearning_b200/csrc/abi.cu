// extern "C" entry points of libwdl_b200 (declared in include/wdl.h): context
// life cycle, the KernelType operator on host pointers, and the host- and
// device-pointer forms of the hot path.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "wdl_internal.cuh"

namespace wdl {

static thread_local std::string g_create_error;

bool autotune_enabled() {
  static const bool on = [] {
    const char* v = std::getenv("WDL_AUTOTUNE");
    return !(v && v[0] == '0');
  }();
  return on;
}

int set_error(wdl_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->last_error = msg;
  else g_create_error = msg;
  return code;
}

int cuda_error(wdl_ctx* ctx, cudaError_t e, const char* where) {
  std::string m = std::string(where) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  return set_error(ctx, e == cudaErrorMemoryAllocation ? WDL_ERR_OUT_OF_MEMORY : WDL_ERR_CUDA, m);
}

int ensure_arena(wdl_ctx* ctx, size_t bytes) {
  if (bytes <= ctx->arena.bytes) return WDL_OK;
  WDL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (ctx->arena.ptr) WDL_CUDA_TRY(ctx, cudaFree(ctx->arena.ptr));
  ctx->arena.ptr = nullptr;
  ctx->arena.bytes = 0;
  WDL_CUDA_TRY(ctx, cudaMalloc(&ctx->arena.ptr, bytes));
  ctx->arena.bytes = bytes;
  return WDL_OK;
}

namespace {

using Io = Arena;

int ensure_io(wdl_ctx* ctx, Io& io, size_t bytes) {
  if (bytes <= io.bytes) return WDL_OK;
  WDL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (io.ptr) WDL_CUDA_TRY(ctx, cudaFree(io.ptr));
  io.ptr = nullptr;
  io.bytes = 0;
  WDL_CUDA_TRY(ctx, cudaMalloc(&io.ptr, bytes));
  io.bytes = bytes;
  return WDL_OK;
}

Io& io_of(wdl_ctx* ctx) { return ctx->io; }

// Carves consecutive 256-byte aligned device blocks out of the Io buffer.
struct Carver {
  char* p;
  template <typename T>
  T* take(size_t n) {
    T* r = reinterpret_cast<T*>(p);
    p += ((n * sizeof(T) + 255) / 256) * 256;
    return r;
  }
};
inline size_t rnd(size_t b) { return ((b + 255) / 256) * 256; }

int build_factors(wdl_ctx* ctx) {
  const int lens[3] = {ctx->W, ctx->H, ctx->D};
  const int naxes = ctx->ndim;
  for (int a = 0; a < naxes; ++a) {
    const int n = lens[a];
    ctx->axis_len[a] = n;
    std::vector<double> g64((size_t)n * n);
    std::vector<float> g32((size_t)n * n);
    // kernel1d[i] = max(EPSILON, exp(-i*i/gamma)) (cpp/kernels.h:637-640),
    // expanded to the dense symmetric factor G[i][j] = kernel1d[|i-j|].
    std::vector<double> k1d(n);
    for (int i = 0; i < n; ++i) k1d[i] = std::max(kEpsilon, std::exp(-(i * i) / ctx->gamma));
    ctx->axis_reach[a] = 0;
    for (int i = 0; i < n; ++i)
      if ((float)k1d[i] != 0.f) ctx->axis_reach[a] = i;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        g64[(size_t)i * n + j] = k1d[std::abs(i - j)];
        g32[(size_t)i * n + j] = (float)k1d[std::abs(i - j)];
      }
    WDL_CUDA_TRY(ctx, cudaMalloc(&ctx->G64[a], g64.size() * 8));
    WDL_CUDA_TRY(ctx, cudaMalloc(&ctx->G32[a], g32.size() * 4));
    WDL_CUDA_TRY(ctx, cudaMemcpy(ctx->G64[a], g64.data(), g64.size() * 8, cudaMemcpyHostToDevice));
    WDL_CUDA_TRY(ctx, cudaMemcpy(ctx->G32[a], g32.data(), g32.size() * 4, cudaMemcpyHostToDevice));
  }
  return WDL_OK;
}

template <typename T>
__global__ void k_to_t(const double* __restrict__ in, T* __restrict__ out, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = (T)in[i];
}
template <typename T>
__global__ void k_from_t(const T* __restrict__ in, double* __restrict__ out, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = (double)in[i];
}

// G (*) u for nvectors images given and returned as FP64 device arrays.
template <typename T>
int convolve_dev_t(wdl_ctx* ctx, const double* u, double* out, int nv, cudaStream_t s) {
  const size_t n = (size_t)nv * ctx->N;
  int rc;
  if ((rc = ensure_arena(ctx, 3 * rnd(n * sizeof(T)) + 256))) return rc;
  ctx->arena.reset();
  T* a = ctx->arena.take<T>(n);
  T* b = ctx->arena.take<T>(n);
  T* t = ctx->arena.take<T>(n);
  const unsigned G = grid_for(n, 256, ctx->sm_count);
  k_to_t<T><<<G, 256, 0, s>>>(u, a, n);
  WDL_LAUNCH_CHECK(ctx);
  if ((rc = conv_stack<T>(ctx, a, b, t, nv, s))) return rc;
  k_from_t<T><<<G, 256, 0, s>>>(b, out, n);
  WDL_LAUNCH_CHECK(ctx);
  return WDL_OK;
}

template <typename T>
int log_convolve_dev_t(wdl_ctx* ctx, const double* u, double* out, uint8_t* signs, int nv,
                       cudaStream_t s) {
  const size_t n = (size_t)nv * ctx->N;
  int rc;
  if ((rc = ensure_arena(ctx, 3 * rnd(n * sizeof(T)) + rnd(n) + 512))) return rc;
  ctx->arena.reset();
  T* a = ctx->arena.take<T>(n);
  T* b = ctx->arena.take<T>(n);
  T* t = ctx->arena.take<T>(n);
  uint8_t* ts = ctx->arena.take<uint8_t>(n);
  const unsigned G = grid_for(n, 256, ctx->sm_count);
  k_to_t<T><<<G, 256, 0, s>>>(u, a, n);
  WDL_LAUNCH_CHECK(ctx);
  if ((rc = log_conv_stack<T>(ctx, a, b, t, nv, signs, signs, signs ? ts : nullptr, s))) return rc;
  k_from_t<T><<<G, 256, 0, s>>>(b, out, n);
  WDL_LAUNCH_CHECK(ctx);
  return WDL_OK;
}

cudaStream_t pick(wdl_ctx* ctx, void* stream) {
  return stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
}

bool bad_sizes(int P, int K, int L) { return P < 1 || K < 1 || L < 1; }

}  // namespace
}  // namespace wdl

using namespace wdl;

extern "C" {

int wdl_abi_version(void) { return WDL_ABI_VERSION; }

const char* wdl_strerror(int status) {
  switch (status) {
    case WDL_OK: return "success";
    case WDL_ERR_INVALID_ARG: return "invalid argument";
    case WDL_ERR_CUDA: return "CUDA runtime error";
    case WDL_ERR_OUT_OF_MEMORY: return "out of device memory";
    case WDL_ERR_UNSUPPORTED: return "unsupported configuration";
    case WDL_ERR_NONFINITE: return "non-finite loss or gradient";
    case WDL_ERR_TIMEOUT: return "bounded wait timed out";
    case WDL_ERR_ADMISSION: return "request exceeds the memory budget";
    case WDL_ERR_NO_DEVICE: return "no usable sm_100 CUDA device";
    case WDL_ERR_BUSY: return "resource busy";
    default: return "unknown status";
  }
}

const char* wdl_last_error(const wdl_ctx* ctx) {
  return ctx ? ctx->last_error.c_str() : g_create_error.c_str();
}

int wdl_create(wdl_ctx** out, int device, int W, int H, int D, double gamma, int precision,
               int domain) {
  if (!out) return set_error(nullptr, WDL_ERR_INVALID_ARG, "ctx pointer is NULL");
  *out = nullptr;
  if (W < 1 || H < 1 || D < 1 || !(gamma > 0) || !std::isfinite(gamma))
    return set_error(nullptr, WDL_ERR_INVALID_ARG, "W, H, D must be >= 1 and gamma > 0");
  if (precision < WDL_FP32 || precision > WDL_FP64)
    return set_error(nullptr, WDL_ERR_INVALID_ARG, "unknown precision");
  if (domain != WDL_DOMAIN_KERNEL && domain != WDL_DOMAIN_LOG)
    return set_error(nullptr, WDL_ERR_INVALID_ARG, "unknown domain");
  if (domain == WDL_DOMAIN_LOG && D != 1)
    return set_error(nullptr, WDL_ERR_UNSUPPORTED, "the log domain is 2-D only (as the reference)");
  if (domain == WDL_DOMAIN_LOG && (precision == WDL_TF32 || precision == WDL_SPLIT_BF16))
    return set_error(nullptr, WDL_ERR_UNSUPPORTED,
                     "the log-sum-exp operator runs on CUDA cores: use WDL_FP32 or WDL_FP64");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return set_error(nullptr, WDL_ERR_NO_DEVICE, "no CUDA device visible");
  }
  if (device < 0 && cudaGetDevice(&device) != cudaSuccess)
    return set_error(nullptr, WDL_ERR_NO_DEVICE, "cudaGetDevice failed");
  if (device >= ndev) return set_error(nullptr, WDL_ERR_INVALID_ARG, "device index out of range");
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess)
    return set_error(nullptr, WDL_ERR_NO_DEVICE, "cudaGetDeviceProperties failed");
  if (prop.major != 10)
    return set_error(nullptr, WDL_ERR_NO_DEVICE,
                     "libwdl_b200 is built for sm_100a (B200) only; device is sm_" +
                         std::to_string(prop.major * 10 + prop.minor));
  if (cudaSetDevice(device) != cudaSuccess)
    return set_error(nullptr, WDL_ERR_NO_DEVICE, "cudaSetDevice failed");

  wdl_ctx* ctx = new (std::nothrow) wdl_ctx();
  if (!ctx) return set_error(nullptr, WDL_ERR_OUT_OF_MEMORY, "host allocation failed");
  ctx->device = device;
  ctx->W = W;
  ctx->H = H;
  ctx->D = D;
  ctx->ndim = D > 1 ? 3 : 2;
  ctx->N = (size_t)W * H * D;
  ctx->gamma = gamma;
  ctx->precision = precision;
  ctx->domain = domain;
  ctx->sm_count = prop.multiProcessorCount;
  int rc = WDL_OK;
  cudaError_t e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev_a);
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev_b);
  if (e != cudaSuccess) rc = cuda_error(ctx, e, "stream/event creation");
  if (rc == WDL_OK) rc = build_factors(ctx);
  if (rc == WDL_OK) rc = noalloc_attach(ctx);
  if (rc == WDL_OK && (precision == WDL_TF32 || precision == WDL_SPLIT_BF16)) {
    rc = tc_init(ctx);
  }
  if (rc != WDL_OK) {
    g_create_error = ctx->last_error;
    wdl_destroy(ctx);
    return rc;
  }
  *out = ctx;
  return WDL_OK;
}

int wdl_destroy(wdl_ctx* ctx) {
  if (!ctx) return WDL_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  tc_free(ctx);
  if (ctx->io.ptr) cudaFree(ctx->io.ptr);
  for (int a = 0; a < 3; ++a) {
    if (ctx->G64[a]) cudaFree(ctx->G64[a]);
    if (ctx->G32[a]) cudaFree(ctx->G32[a]);
  }
  if (ctx->arena.ptr) cudaFree(ctx->arena.ptr);
  if (ctx->lbfgs_arena.ptr) cudaFree(ctx->lbfgs_arena.ptr);
  if (ctx->d_trace) cudaFree(ctx->d_trace);
  if (ctx->d_taps) cudaFree(ctx->d_taps);
  for (auto& gr : ctx->graphs)
    if (gr.exec) cudaGraphExecDestroy(gr.exec);
  if (ctx->ev_a) cudaEventDestroy(ctx->ev_a);
  if (ctx->ev_b) cudaEventDestroy(ctx->ev_b);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return WDL_OK;
}

int wdl_synchronize(wdl_ctx* ctx) {
  if (!ctx) return WDL_ERR_INVALID_ARG;
  WDL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return tc_check_status(ctx);
}

size_t wdl_eval_bytes(const wdl_ctx* ctx, int P, int K, int L) {
  if (!ctx || bad_sizes(P, K, L)) return 0;
  return eval_bytes(ctx, P, K, L);
}

long long wdl_launch_count(const wdl_ctx* ctx) { return ctx ? ctx->launches : -1; }

int wdl_set_profiling(wdl_ctx* ctx, int on) {
  if (!ctx) return WDL_ERR_INVALID_ARG;
  ctx->profiling = on != 0;
  ctx->trace_level = on;
  ctx->conv_ms = 0;
  ctx->conv_launches = 0;
  ctx->conv_images = 0;
  ctx->log_exps = 0;
  return WDL_OK;
}

int wdl_phase_trace(wdl_ctx* ctx, double* out27) {
  if (!ctx || !out27) return WDL_ERR_INVALID_ARG;
  for (int i = 0; i < 27; ++i) out27[i] = 0;
  if (!ctx->d_trace) return WDL_OK;
  unsigned long long h[27];
  WDL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  WDL_CUDA_TRY(ctx, cudaMemcpy(h, ctx->d_trace, sizeof(h), cudaMemcpyDeviceToHost));
  for (int i = 0; i < 27; ++i) out27[i] = (double)h[i];
  return WDL_OK;
}

int wdl_set_autotune(wdl_ctx* ctx, int on) {
  if (!ctx) return WDL_ERR_INVALID_ARG;
  ctx->autotune = on != 0;
  return WDL_OK;
}

int wdl_set_wait_limit(wdl_ctx* ctx, double seconds) {
  if (!ctx) return WDL_ERR_INVALID_ARG;
  if (!(seconds >= 0) || seconds > 60)
    return set_error(ctx, WDL_ERR_INVALID_ARG, "wait limit must be in [0, 60] seconds (0: default)");
  ctx->wait_limit_s = seconds;
  return WDL_OK;
}

int wdl_inject_fault(wdl_ctx* ctx, int kind) {
  if (!ctx) return WDL_ERR_INVALID_ARG;
  if (kind != 0 && kind != WDL_FAULT_DROP_FIRST_ITERATION)
    return set_error(ctx, WDL_ERR_INVALID_ARG, "unknown fault kind");
  ctx->inject_fault = kind;
  return WDL_OK;
}

int wdl_autotune_count(const wdl_ctx* ctx) { return ctx ? (int)ctx->tuned.size() : WDL_ERR_INVALID_ARG; }

int wdl_autotune_entry(const wdl_ctx* ctx, int i, long long* key6, int* choice, float* ms) {
  if (!ctx || i < 0 || i >= (int)ctx->tuned.size()) return WDL_ERR_INVALID_ARG;
  const auto& e = ctx->tuned[i];
  if (key6) std::memcpy(key6, e.key, sizeof(e.key));
  if (choice) *choice = e.choice;
  if (ms) *ms = e.ms;
  return WDL_OK;
}

int wdl_exp_profile(const wdl_ctx* ctx, double* executed_exps) {
  if (!ctx || !executed_exps) return WDL_ERR_INVALID_ARG;
  *executed_exps = ctx->log_exps;
  return WDL_OK;
}

int wdl_conv_profile(const wdl_ctx* ctx, double* conv_ms, long long* conv_launches,
                     double* conv_images) {
  if (!ctx) return WDL_ERR_INVALID_ARG;
  if (conv_ms) *conv_ms = ctx->conv_ms;
  if (conv_launches) *conv_launches = ctx->conv_launches;
  if (conv_images) *conv_images = ctx->conv_images;
  return WDL_OK;
}

// ---- operator -----------------------------------------------------------------------
int wdl_convolve_device(wdl_ctx* ctx, const double* u, double* out, int nvectors, void* stream) {
  if (!ctx || !u || !out || nvectors < 0) return set_error(ctx, WDL_ERR_INVALID_ARG, "bad arguments");
  if (nvectors == 0) return WDL_OK;
  cudaSetDevice(ctx->device);
  cudaStream_t s = pick(ctx, stream);
  return ctx->precision == WDL_FP64 ? convolve_dev_t<double>(ctx, u, out, nvectors, s)
                                    : convolve_dev_t<float>(ctx, u, out, nvectors, s);
}

int wdl_convolve(wdl_ctx* ctx, const double* u, double* out, int nvectors) {
  if (!ctx || !u || !out || nvectors < 0) return set_error(ctx, WDL_ERR_INVALID_ARG, "bad arguments");
  if (nvectors == 0) return WDL_OK;
  cudaSetDevice(ctx->device);
  const size_t n = (size_t)nvectors * ctx->N;
  Io& io = io_of(ctx);
  int rc;
  if ((rc = ensure_io(ctx, io, 2 * rnd(n * 8)))) return rc;
  Carver c{static_cast<char*>(io.ptr)};
  double* du = c.take<double>(n);
  double* dout = c.take<double>(n);
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(du, u, n * 8, cudaMemcpyHostToDevice, ctx->stream));
  if ((rc = wdl_convolve_device(ctx, du, dout, nvectors, ctx->stream))) return rc;
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(out, dout, n * 8, cudaMemcpyDeviceToHost, ctx->stream));
  WDL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return tc_check_status(ctx);
}

static int log_convolve_common(wdl_ctx* ctx, const double* u, unsigned char* signs, double* out,
                               int nv) {
  if (!ctx || !u || !out || nv < 0) return set_error(ctx, WDL_ERR_INVALID_ARG, "bad arguments");
  if (ctx->ndim != 2)
    return set_error(ctx, WDL_ERR_UNSUPPORTED, "the log-domain operator is 2-D only");
  if (nv == 0) return WDL_OK;
  if (ctx->precision == WDL_TF32 || ctx->precision == WDL_SPLIT_BF16)
    return set_error(ctx, WDL_ERR_UNSUPPORTED, "log-sum-exp runs in WDL_FP32 or WDL_FP64");
  cudaSetDevice(ctx->device);
  const size_t n = (size_t)nv * ctx->N;
  Io& io = io_of(ctx);
  int rc;
  if ((rc = ensure_io(ctx, io, 2 * rnd(n * 8) + rnd(n)))) return rc;
  Carver c{static_cast<char*>(io.ptr)};
  double* du = c.take<double>(n);
  double* dout = c.take<double>(n);
  uint8_t* ds = c.take<uint8_t>(n);
  std::vector<uint8_t> bytes;
  if (signs) {  // bit i of byte i/8 (cpp/signArray.h:8-22) -> one byte per element
    bytes.resize(n);
    for (size_t i = 0; i < n; ++i) bytes[i] = (signs[i / 8] >> (i % 8)) & 1;
    WDL_CUDA_TRY(ctx, cudaMemcpyAsync(ds, bytes.data(), n, cudaMemcpyHostToDevice, ctx->stream));
  }
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(du, u, n * 8, cudaMemcpyHostToDevice, ctx->stream));
  rc = ctx->precision == WDL_FP64
           ? log_convolve_dev_t<double>(ctx, du, dout, signs ? ds : nullptr, nv, ctx->stream)
           : log_convolve_dev_t<float>(ctx, du, dout, signs ? ds : nullptr, nv, ctx->stream);
  if (rc) return rc;
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(out, dout, n * 8, cudaMemcpyDeviceToHost, ctx->stream));
  if (signs)
    WDL_CUDA_TRY(ctx, cudaMemcpyAsync(bytes.data(), ds, n, cudaMemcpyDeviceToHost, ctx->stream));
  WDL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (signs) {
    for (size_t i = 0; i < n; ++i) {
      if (bytes[i]) signs[i / 8] |= (unsigned char)(1u << (i % 8));
      else signs[i / 8] &= (unsigned char)~(1u << (i % 8));
    }
  }
  return WDL_OK;
}

int wdl_log_convolve(wdl_ctx* ctx, const double* log_u, double* out, int nvectors) {
  return log_convolve_common(ctx, log_u, nullptr, out, nvectors);
}

int wdl_log_convolve_signed(wdl_ctx* ctx, const double* log_u, unsigned char* signs, double* out,
                            int nvectors) {
  if (!signs) return set_error(ctx, WDL_ERR_INVALID_ARG, "signs is NULL");
  return log_convolve_common(ctx, log_u, signs, out, nvectors);
}

// ---- hot path -------------------------------------------------------------------------
int wdl_gradient_both_device(wdl_ctx* ctx, int P, int K, int L, int loss_type, const double* atoms,
                             const double* weights, const double* observed, const double* b_init,
                             double* result_la, double* result_dic, double* bary, double* loss,
                             double* b_last, void* stream) {
  if (!ctx) return WDL_ERR_INVALID_ARG;
  if (bad_sizes(P, K, L) || !atoms || !weights || !observed || !result_la)
    return set_error(ctx, WDL_ERR_INVALID_ARG, "bad sizes or NULL required pointer");
  if (loss_type < WDL_LOSS_TV || loss_type > WDL_LOSS_KL)
    return set_error(ctx, WDL_ERR_INVALID_ARG, "loss_type must be 1..4");
  cudaSetDevice(ctx->device);
  return gradient_both_dev(ctx, P, K, L, loss_type, atoms, weights, observed, b_init, result_la,
                           result_dic, bary, loss, b_last, pick(ctx, stream), true);
}

int wdl_gradient_both(wdl_ctx* ctx, int P, int K, int L, int loss_type, const double* atoms,
                      const double* weights, const double* observed, const double* b_init,
                      double* result_la, double* result_dic, double* bary, double* loss,
                      double* b_last) {
  if (!ctx) return WDL_ERR_INVALID_ARG;
  if (bad_sizes(P, K, L) || !atoms || !weights || !observed || !result_la)
    return set_error(ctx, WDL_ERR_INVALID_ARG, "bad sizes or NULL required pointer");
  cudaSetDevice(ctx->device);
  const size_t N = ctx->N, KN = (size_t)K * N, PK = (size_t)P * K, PN = (size_t)P * N,
               PKN = PK * N;
  Io& io = io_of(ctx);
  int rc;
  const size_t need = rnd(KN * 8) * 2 + rnd(PK * 8) * 2 + rnd(PN * 8) * 2 + rnd(PKN * 8) * 2 +
                      rnd(P * 8);
  if ((rc = ensure_io(ctx, io, need))) return rc;
  Carver c{static_cast<char*>(io.ptr)};
  double* d_atoms = c.take<double>(KN);
  double* d_w = c.take<double>(PK);
  double* d_obs = c.take<double>(PN);
  double* d_binit = b_init ? c.take<double>(PKN) : nullptr;
  double* d_la = c.take<double>(PK);
  double* d_dic = result_dic ? c.take<double>(KN) : nullptr;
  double* d_bary = bary ? c.take<double>(PN) : nullptr;
  double* d_loss = loss ? c.take<double>(P) : nullptr;
  double* d_blast = b_last ? c.take<double>(PKN) : nullptr;
  cudaStream_t s = ctx->stream;
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(d_atoms, atoms, KN * 8, cudaMemcpyHostToDevice, s));
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(d_w, weights, PK * 8, cudaMemcpyHostToDevice, s));
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(d_obs, observed, PN * 8, cudaMemcpyHostToDevice, s));
  if (b_init) WDL_CUDA_TRY(ctx, cudaMemcpyAsync(d_binit, b_init, PKN * 8, cudaMemcpyHostToDevice, s));
  if ((rc = wdl_gradient_both_device(ctx, P, K, L, loss_type, d_atoms, d_w, d_obs, d_binit, d_la,
                                     d_dic, d_bary, d_loss, d_blast, s)))
    return rc;
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(result_la, d_la, PK * 8, cudaMemcpyDeviceToHost, s));
  if (result_dic) WDL_CUDA_TRY(ctx, cudaMemcpyAsync(result_dic, d_dic, KN * 8, cudaMemcpyDeviceToHost, s));
  if (bary) WDL_CUDA_TRY(ctx, cudaMemcpyAsync(bary, d_bary, PN * 8, cudaMemcpyDeviceToHost, s));
  if (loss) WDL_CUDA_TRY(ctx, cudaMemcpyAsync(loss, d_loss, P * 8, cudaMemcpyDeviceToHost, s));
  if (b_last) WDL_CUDA_TRY(ctx, cudaMemcpyAsync(b_last, d_blast, PKN * 8, cudaMemcpyDeviceToHost, s));
  WDL_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  return tc_check_status(ctx);
}

int wdl_evaluate_both_device(wdl_ctx* ctx, int P, int K, int L, int loss_type, double scale_dic,
                             const double* x, double* g, int n, const double* observed, double* f,
                             const double* b_storage, double* b_last, double* bary, void* stream) {
  if (!ctx) return WDL_ERR_INVALID_ARG;
  if (bad_sizes(P, K, L) || !x || !g || !observed || !f || !(scale_dic != 0))
    return set_error(ctx, WDL_ERR_INVALID_ARG, "bad sizes, scale or NULL required pointer");
  if (loss_type < WDL_LOSS_TV || loss_type > WDL_LOSS_KL)
    return set_error(ctx, WDL_ERR_INVALID_ARG, "loss_type must be 1..4");
  cudaSetDevice(ctx->device);
  return evaluate_both_dev(ctx, P, K, L, loss_type, scale_dic, x, g, n, observed, f, b_storage,
                           b_last, bary, pick(ctx, stream));
}

static int regress_args(wdl_ctx* ctx, int P, int K, int L, int loss_type, double scale_dic,
                        const double* solution, const double* observed, int max_iterations) {
  if (bad_sizes(P, K, L) || !solution || !observed || !(scale_dic != 0) || !std::isfinite(scale_dic))
    return set_error(ctx, WDL_ERR_INVALID_ARG, "bad sizes, scale or NULL required pointer");
  if (loss_type < WDL_LOSS_TV || loss_type > WDL_LOSS_KL)
    return set_error(ctx, WDL_ERR_INVALID_ARG, "loss_type must be 1..4");
  if (max_iterations < 0) return set_error(ctx, WDL_ERR_INVALID_ARG, "max_iterations must be >= 0");
  return WDL_OK;
}

int wdl_regress_both_device(wdl_ctx* ctx, int P, int K, int L, int loss_type, double scale_dic,
                            double* solution, const double* observed, int max_iterations, double epsilon,
                            int warm_restart, int* status, double* f, int* evaluations, void* stream) {
  if (!ctx) return WDL_ERR_INVALID_ARG;
  int rc;
  if ((rc = regress_args(ctx, P, K, L, loss_type, scale_dic, solution, observed, max_iterations))) return rc;
  if (warm_restart && max_iterations < 10)
    return set_error(ctx, WDL_ERR_INVALID_ARG, "warm restart runs 10-iteration runs: max_iterations >= 10");
  cudaSetDevice(ctx->device);
  return regress_both_dev(ctx, P, K, L, loss_type, scale_dic, solution, observed, max_iterations, epsilon,
                          warm_restart, status, f, evaluations, pick(ctx, stream));
}

int wdl_regress_both(wdl_ctx* ctx, int P, int K, int L, int loss_type, double scale_dic, double* solution,
                     const double* observed, int max_iterations, double epsilon, int warm_restart,
                     int* status, double* f, int* evaluations) {
  if (!ctx) return WDL_ERR_INVALID_ARG;
  int rc;
  if ((rc = regress_args(ctx, P, K, L, loss_type, scale_dic, solution, observed, max_iterations))) return rc;
  if (warm_restart && max_iterations < 10)
    return set_error(ctx, WDL_ERR_INVALID_ARG, "warm restart runs 10-iteration runs: max_iterations >= 10");
  cudaSetDevice(ctx->device);
  const size_t N = ctx->N, n = (size_t)P * K + (size_t)K * N, PN = (size_t)P * N;
  Io& io = io_of(ctx);
  if ((rc = ensure_io(ctx, io, rnd(n * 8) + rnd(PN * 8) + 256))) return rc;
  Carver c{static_cast<char*>(io.ptr)};
  double* d_sol = c.take<double>(n);
  double* d_obs = c.take<double>(PN);
  cudaStream_t s = ctx->stream;
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(d_sol, solution, n * 8, cudaMemcpyHostToDevice, s));
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(d_obs, observed, PN * 8, cudaMemcpyHostToDevice, s));
  if ((rc = regress_both_dev(ctx, P, K, L, loss_type, scale_dic, d_sol, d_obs, max_iterations, epsilon,
                             warm_restart, status, f, evaluations, s)))
    return rc;
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(solution, d_sol, n * 8, cudaMemcpyDeviceToHost, s));
  WDL_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  return WDL_OK;
}

int wdl_evaluate_both(wdl_ctx* ctx, int P, int K, int L, int loss_type, double scale_dic,
                      const double* x, double* g, int n, const double* observed, double* f,
                      const double* b_storage, double* b_last, double* bary) {
  if (!ctx) return WDL_ERR_INVALID_ARG;
  if (bad_sizes(P, K, L) || !x || !g || !observed || !f)
    return set_error(ctx, WDL_ERR_INVALID_ARG, "bad sizes or NULL required pointer");
  cudaSetDevice(ctx->device);
  const size_t N = ctx->N, KN = (size_t)K * N, PK = (size_t)P * K, PN = (size_t)P * N,
               PKN = PK * N;
  if ((size_t)n != PK + KN) return set_error(ctx, WDL_ERR_INVALID_ARG, "n != P*K + K*N");
  Io& io = io_of(ctx);
  int rc;
  const size_t need = rnd((PK + KN) * 8) * 2 + rnd(PN * 8) * 2 + rnd(PKN * 8) * 2 + 256;
  if ((rc = ensure_io(ctx, io, need))) return rc;
  Carver c{static_cast<char*>(io.ptr)};
  double* d_x = c.take<double>(PK + KN);
  double* d_g = c.take<double>(PK + KN);
  double* d_obs = c.take<double>(PN);
  double* d_bary = bary ? c.take<double>(PN) : nullptr;
  double* d_bs = b_storage ? c.take<double>(PKN) : nullptr;
  double* d_bl = b_last ? c.take<double>(PKN) : nullptr;
  double* d_f = c.take<double>(1);
  cudaStream_t s = ctx->stream;
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(d_x, x, (PK + KN) * 8, cudaMemcpyHostToDevice, s));
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(d_obs, observed, PN * 8, cudaMemcpyHostToDevice, s));
  if (b_storage) WDL_CUDA_TRY(ctx, cudaMemcpyAsync(d_bs, b_storage, PKN * 8, cudaMemcpyHostToDevice, s));
  if ((rc = wdl_evaluate_both_device(ctx, P, K, L, loss_type, scale_dic, d_x, d_g, n, d_obs, d_f,
                                     d_bs, d_bl, d_bary, s)))
    return rc;
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(g, d_g, (PK + KN) * 8, cudaMemcpyDeviceToHost, s));
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(f, d_f, 8, cudaMemcpyDeviceToHost, s));
  if (bary) WDL_CUDA_TRY(ctx, cudaMemcpyAsync(bary, d_bary, PN * 8, cudaMemcpyDeviceToHost, s));
  if (b_last) WDL_CUDA_TRY(ctx, cudaMemcpyAsync(b_last, d_bl, PKN * 8, cudaMemcpyDeviceToHost, s));
  WDL_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  if ((rc = tc_check_status(ctx))) return rc;
  if (!std::isfinite(*f)) return set_error(ctx, WDL_ERR_NONFINITE, "objective is not finite");
  return WDL_OK;
}

int wdl_barycenter(wdl_ctx* ctx, int P, int K, int L, const double* atoms, const double* weights,
                   double* bary) {
  if (!ctx) return WDL_ERR_INVALID_ARG;
  if (bad_sizes(P, K, L) || !atoms || !weights || !bary)
    return set_error(ctx, WDL_ERR_INVALID_ARG, "bad sizes or NULL pointer");
  cudaSetDevice(ctx->device);
  const size_t N = ctx->N, KN = (size_t)K * N, PK = (size_t)P * K, PN = (size_t)P * N;
  Io& io = io_of(ctx);
  int rc;
  if ((rc = ensure_io(ctx, io, rnd(KN * 8) + rnd(PK * 8) + rnd(PN * 8)))) return rc;
  Carver c{static_cast<char*>(io.ptr)};
  double* d_atoms = c.take<double>(KN);
  double* d_w = c.take<double>(PK);
  double* d_bary = c.take<double>(PN);
  cudaStream_t s = ctx->stream;
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(d_atoms, atoms, KN * 8, cudaMemcpyHostToDevice, s));
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(d_w, weights, PK * 8, cudaMemcpyHostToDevice, s));
  if ((rc = barycenter_dev(ctx, P, K, L, d_atoms, d_w, d_bary, s))) return rc;
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(bary, d_bary, PN * 8, cudaMemcpyDeviceToHost, s));
  WDL_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  return tc_check_status(ctx);
}

}  // extern "C"
