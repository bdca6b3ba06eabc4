// wdl_batch_run: many independent problems — different grid sides (<= the
// context's), atom counts, iteration counts, histogram counts and modes — in
// ONE persistent launch of the fused tensor-core kernel (sinkhorn_tc.cu).
//
// The context's factor matrix serves every problem: the Gibbs factor of a side
// n is the leading n x n block of the factor of any larger side with the same
// gamma (G[i][j] = g(|i-j|)).  Inputs of all problems are staged in one upload,
// normalised (Problem::normalize_values, cpp/inverseWasserstein.h:53-74) by one
// table-driven kernel; the kernel's work items come from a host-built table
// ordered by round (iteration or reverse step) so that every problem's
// dependency chain advances in parallel; outputs are gathered into one region
// and copied back with one transfer.
#include <cstring>
#include <vector>

#include "wdl_internal.cuh"

namespace wdl {
namespace {

struct RowJob {          // normalise one row in FP64 and cast it to FP32
  const double* src;
  double* dst64;
  float* dst32;
  int len;
};

__global__ void k_rows(const RowJob* __restrict__ jobs, int njobs) {
  __shared__ double sh[32];
  for (int jb = blockIdx.x; jb < njobs; jb += gridDim.x) {
    const RowJob j = jobs[jb];
    double s = 0;
    for (int i = threadIdx.x; i < j.len; i += blockDim.x) s += j.src[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
      sh[31] = t;
    }
    __syncthreads();
    const double tot = sh[31];
    for (int i = threadIdx.x; i < j.len; i += blockDim.x) {
      const double v = j.src[i] / tot;
      if (j.dst64) j.dst64[i] = v;
      j.dst32[i] = (float)v;
    }
    __syncthreads();
  }
}

struct OutJob {  // gather an output: 0 = exp(acc), 1 = sum over P of gdic, 2 = copy (double)
  int kind, P;
  const float* src;
  const double* src64;
  double* dst;
  size_t len;     // elements of the output
};

__global__ void k_outputs(const OutJob* __restrict__ jobs, int njobs) {
  for (int jb = blockIdx.x; jb < njobs; jb += gridDim.x) {
    const OutJob j = jobs[jb];
    for (size_t i = threadIdx.x; i < j.len; i += blockDim.x) {
      if (j.kind == 0) {
        j.dst[i] = (double)expf(j.src[i]);
      } else if (j.kind == 1) {
        double s = 0;
        for (int p = 0; p < j.P; ++p) s += (double)j.src[(size_t)p * j.len + i];
        j.dst[i] = s;
      } else {
        j.dst[i] = j.src64[i];
      }
    }
  }
}

inline size_t r256(size_t b) { return (b + 255) & ~size_t(255); }

// Sequential 256-byte aligned layout: offsets are recorded, pointers formed
// against the real base only.
struct Carve {
  char* p;
  size_t off = 0;
  template <typename T>
  T* take(size_t n) {
    off = r256(off);
    T* r = p ? reinterpret_cast<T*>(p + off) : nullptr;
    off += n * sizeof(T);
    return r;
  }
  size_t mark() {
    off = r256(off);
    return off;
  }
};

}  // namespace

int batch_prepare(wdl_ctx* ctx, const wdl_problem* pb, int nprob, size_t extra_bytes, BatchPlan& bp,
                  cudaStream_t s) {
  if (!ctx || !pb || nprob < 1) return set_error(ctx, WDL_ERR_INVALID_ARG, "bad arguments");
  if (!tc_fused(ctx) || ctx->domain != WDL_DOMAIN_KERNEL)
    return set_error(ctx, WDL_ERR_UNSUPPORTED,
                     "many-problem launches need a kernel-domain WDL_TF32 or WDL_SPLIT_BF16 context "
                     "of a 2-D grid with sides <= 128");
  const bool split = ctx->precision == WDL_SPLIT_BF16;
  for (int q = 0; q < nprob; ++q) {
    const wdl_problem& w = pb[q];
    if (w.W < 1 || w.H < 1 || w.W > ctx->W || w.H > ctx->H || w.K < 1 || w.K > 64 || w.L < 1 ||
        w.P < 1 || !w.atoms || !w.weights || w.mode < WDL_MODE_WEIGHTS || w.mode > WDL_MODE_BARYCENTER)
      return set_error(ctx, WDL_ERR_INVALID_ARG, "problem " + std::to_string(q) + ": bad sizes or pointers");
    if (w.mode != WDL_MODE_BARYCENTER &&
        (!w.observed || w.loss_type < WDL_LOSS_TV || w.loss_type > WDL_LOSS_KL ||
         w.loss_type == WDL_LOSS_WASSERSTEIN))
      return set_error(ctx, WDL_ERR_INVALID_ARG,
                       "problem " + std::to_string(q) + ": needs observations and loss 1, 2 or 4");
  }
  bp.nprob = nprob;
  bp.buf.assign(nprob, BatchBuf{});
  bp.prs.assign(nprob, SkProblem{});
  // ---- layout: one arena region per problem, all in one allocation ----------------
  auto plan = [&](char* basep) {
    Carve c{basep};
    bp.probs = c.mark();
    c.take<SkProblem>(nprob);
    bp.gsync = c.mark();
    c.take<int>(2);
    bp.zero_b = c.mark();  // region that must start at zero
    for (int q = 0; q < nprob; ++q) {
      const wdl_problem& w = pb[q];
      const size_t N = (size_t)w.W * w.H, P = w.P, K = w.K, L = w.L;
      const bool fo = w.mode == WDL_MODE_BARYCENTER, dic = w.mode == WDL_MODE_BOTH;
      const size_t slots = fo ? 2 : L;
      BatchBuf& o = bp.buf[q];
      o.acc = c.take<float>(slots * P * N);
      o.dot = c.take<double>(P * K);
      o.nb = c.take<float>(dic ? 2 * P * N : 1);
      o.gwb = c.take<float>(fo ? 1 : 2 * P * N);
      o.v = c.take<float>(dic ? P * K * N : 1);
      o.r = c.take<float>(fo ? 1 : P * K * N);
      o.gdic = c.take<float>(dic ? P * K * N : 1);
    }
    bp.zero_e = c.mark();
    for (int q = 0; q < nprob; ++q) {
      const wdl_problem& w = pb[q];
      const size_t N = (size_t)w.W * w.H, P = w.P, K = w.K, L = w.L;
      const bool fo = w.mode == WDL_MODE_BARYCENTER;
      const size_t slots = fo ? 2 : L;
      BatchBuf& o = bp.buf[q];
      o.atoms64 = c.take<double>(K * N);
      o.lam64 = c.take<double>(P * K);
      o.loss = c.take<double>(P);
      o.atoms = c.take<float>(K * N);
      o.lam = c.take<float>(P * K);
      o.cb = c.take<float>(fo ? 1 : slots * P * K * N);
      o.phi = c.take<float>(slots * P * K * N);
      o.sync = c.take<int>(5 * P);
    }
    bp.in_b = c.mark();  // inputs: one upload
    for (int q = 0; q < nprob; ++q) {
      const wdl_problem& w = pb[q];
      const size_t N = (size_t)w.W * w.H;
      bp.buf[q].in_atoms = c.take<double>((size_t)w.K * N);
      bp.buf[q].in_w = c.take<double>((size_t)w.P * w.K);
      bp.buf[q].obs = w.mode == WDL_MODE_BARYCENTER ? nullptr : c.take<double>((size_t)w.P * N);
    }
    bp.in_e = c.mark();
    bp.out_b = bp.in_e;  // outputs: one download
    for (int q = 0; q < nprob; ++q) {
      const wdl_problem& w = pb[q];
      const size_t N = (size_t)w.W * w.H;
      const bool grad = w.mode != WDL_MODE_BARYCENTER;
      BatchBuf& o = bp.buf[q];
      o.out_la = (grad && w.result_la) ? c.take<double>((size_t)w.P * w.K) : nullptr;
      o.out_loss = (grad && w.loss) ? c.take<double>((size_t)w.P) : nullptr;
      o.out_bary = w.bary ? c.take<double>((size_t)w.P * N) : nullptr;
      o.out_dic = (w.mode == WDL_MODE_BOTH && w.result_dic) ? c.take<double>((size_t)w.K * N) : nullptr;
    }
    bp.out_e = c.mark();
    return c.off;
  };
  const size_t core = plan(nullptr);
  size_t n_rows = 0;
  bp.n_outjobs = 0;
  bp.n_items_all = 0;
  for (int q = 0; q < nprob; ++q) {
    const wdl_problem& w = pb[q];
    const bool grad = w.mode != WDL_MODE_BARYCENTER;
    n_rows += (size_t)w.K + w.P;
    bp.n_outjobs += (w.bary ? 1 : 0) + (w.mode == WDL_MODE_BOTH && w.result_dic ? 1 : 0) +
                    (grad && w.result_la ? 1 : 0) + (grad && w.loss ? 1 : 0);
    SkProblem tmp{};
    tmp.K = w.K;
    tmp.L = w.L;
    tmp.P = w.P;
    tmp.fwd_only = w.mode == WDL_MODE_BARYCENTER;
    tmp.need_dic = w.mode == WDL_MODE_BOTH;
    bp.n_items_all += sk_problem_items(tmp);
  }
  if (bp.n_items_all > 0x7fffffff) return set_error(ctx, WDL_ERR_INVALID_ARG, "too many work items");
  bp.rows_off = r256(core);
  bp.outj_off = r256(bp.rows_off + n_rows * sizeof(RowJob));
  bp.items_off = r256(bp.outj_off + bp.n_outjobs * sizeof(OutJob));
  bp.extra_off = r256(bp.items_off + bp.n_items_all * sizeof(int4));
  int rc;
  if ((rc = ensure_arena(ctx, bp.extra_off + extra_bytes + 256))) return rc;
  char* base = static_cast<char*>(ctx->arena.ptr);
  bp.base = base;
  plan(base);
  bp.sync = reinterpret_cast<int*>(base + bp.gsync);

  // ---- host tables ----------------------------------------------------------------
  std::vector<char> h_in(bp.in_e - bp.in_b);
  std::vector<RowJob> rows;
  rows.reserve(n_rows);
  std::vector<OutJob> outs;
  for (int q = 0; q < nprob; ++q) {
    const wdl_problem& w = pb[q];
    const size_t N = (size_t)w.W * w.H;
    BatchBuf& o = bp.buf[q];
    std::memcpy(h_in.data() + ((char*)o.in_atoms - base - bp.in_b), w.atoms, (size_t)w.K * N * 8);
    std::memcpy(h_in.data() + ((char*)o.in_w - base - bp.in_b), w.weights, (size_t)w.P * w.K * 8);
    if (o.obs) std::memcpy(h_in.data() + ((char*)o.obs - base - bp.in_b), w.observed, (size_t)w.P * N * 8);
    for (int k = 0; k < w.K; ++k) rows.push_back({o.in_atoms + k * N, o.atoms64 + k * N, o.atoms + k * N, (int)N});
    for (int p = 0; p < w.P; ++p) rows.push_back({o.in_w + (size_t)p * w.K, o.lam64 + (size_t)p * w.K, o.lam + (size_t)p * w.K, w.K});
    SkProblem& pr = bp.prs[q];
    pr = SkProblem{};
    sk_fill_geometry(pr, w.W, w.H, split);
    pr.K = w.K;
    pr.L = w.L;
    pr.P = w.P;
    pr.loss_type = w.mode == WDL_MODE_BARYCENTER ? WDL_LOSS_QUADRATIC : w.loss_type;
    pr.fwd_only = w.mode == WDL_MODE_BARYCENTER;
    pr.need_dic = w.mode == WDL_MODE_BOTH;
    pr.atoms = o.atoms;
    pr.lam = o.lam;
    pr.obs = o.obs;
    pr.b0 = nullptr;
    pr.cb = o.cb;
    pr.phi = o.phi;
    pr.acc = o.acc;
    pr.nb = o.nb;
    pr.gwb = o.gwb;
    pr.v = o.v;
    pr.r = o.r;
    pr.gdic = o.gdic;
    pr.dot = o.dot;
    pr.loss = o.loss;
    pr.sync = o.sync;
    if (o.out_bary)
      outs.push_back({0, w.P, o.acc + (size_t)(pr.fwd_only ? ((w.L - 1) & 1) : (w.L - 1)) * w.P * N,
                      nullptr, o.out_bary, (size_t)w.P * N});
    if (o.out_dic) outs.push_back({1, w.P, o.gdic, nullptr, o.out_dic, (size_t)w.K * N});
    if (o.out_la) outs.push_back({2, w.P, nullptr, o.dot, o.out_la, (size_t)w.P * w.K});
    if (o.out_loss) outs.push_back({2, w.P, nullptr, o.loss, o.out_loss, (size_t)w.P});
  }
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(base + bp.in_b, h_in.data(), h_in.size(), cudaMemcpyHostToDevice, s));
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(base + bp.rows_off, rows.data(), rows.size() * sizeof(RowJob), cudaMemcpyHostToDevice, s));
  if (!outs.empty())
    WDL_CUDA_TRY(ctx, cudaMemcpyAsync(base + bp.outj_off, outs.data(), outs.size() * sizeof(OutJob), cudaMemcpyHostToDevice, s));
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(base + bp.probs, bp.prs.data(), bp.prs.size() * sizeof(SkProblem), cudaMemcpyHostToDevice, s));
  k_rows<<<grid_for(rows.size(), 1, ctx->sm_count, 4), 256, 0, s>>>(reinterpret_cast<RowJob*>(base + bp.rows_off), (int)rows.size());
  WDL_LAUNCH_CHECK(ctx);
  // the error word is cleared here once; every launch clears only the counter
  WDL_CUDA_TRY(ctx, cudaMemsetAsync(bp.sync, 0, 2 * sizeof(int), s));
  // host copies must outlive the asynchronous uploads
  WDL_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  return WDL_OK;
}

void batch_items(const BatchPlan& bp, const std::vector<uint8_t>* active, std::vector<int4>& items) {
  items.clear();
  std::vector<size_t> first(bp.nprob + 1, 0);
  int rounds_max = 0;
  for (int q = 0; q < bp.nprob; ++q) {
    first[q + 1] = first[q] + bp.prs[q].P;
    const int rounds = bp.prs[q].fwd_only ? bp.prs[q].L : 2 * bp.prs[q].L;
    if (rounds > rounds_max) rounds_max = rounds;
  }
  for (int r = 0; r < rounds_max; ++r) {
    for (int q = 0; q < bp.nprob; ++q) {
      const SkProblem& pr = bp.prs[q];
      const int PK = pr.P * pr.K;
      if (r < pr.L) {
        for (int pk = 0; pk < PK; ++pk)
          if (!active || (*active)[first[q] + pk / pr.K]) items.push_back(make_int4(q, 0, r + 1, pk));
      } else if (!pr.fwd_only && r < 2 * pr.L) {
        const int sstep = 2 * pr.L - r;
        for (int pk = 0; pk < PK; ++pk) {
          if (active && !(*active)[first[q] + pk / pr.K]) continue;
          if (pr.need_dic) items.push_back(make_int4(q, 1, sstep, pk));
          items.push_back(make_int4(q, 2, sstep, pk));
        }
      }
    }
  }
}

int batch_launch(wdl_ctx* ctx, BatchPlan& bp, size_t n_items, cudaStream_t s) {
  char* base = bp.base;
  WDL_CUDA_TRY(ctx, cudaMemsetAsync(base + bp.zero_b, 0, bp.zero_e - bp.zero_b, s));
  SkArgs a{};
  a.G = ctx->G32[ctx->W >= ctx->H ? 0 : 1];
  a.Gn = ctx->W >= ctx->H ? ctx->W : ctx->H;
  a.nprobs = bp.nprob;
  a.probs = reinterpret_cast<SkProblem*>(base + bp.probs);
  a.items = reinterpret_cast<int4*>(base + bp.items_off);
  a.total = (long long)n_items;
  for (int q = 0; q < bp.nprob; ++q) a.apps += sk_problem_applications(bp.prs[q]);
  a.sync = bp.sync;
  return sinkhorn_tc_launch(ctx, a, s);
}

}  // namespace wdl

using namespace wdl;

extern "C" int wdl_batch_run(wdl_ctx* ctx, const wdl_problem* pb, int nprob) {
  if (!ctx) return WDL_ERR_INVALID_ARG;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return set_error(ctx, WDL_ERR_CUDA, "cudaSetDevice failed");
  cudaStream_t s = ctx->stream;
  BatchPlan bp;
  int rc;
  if ((rc = batch_prepare(ctx, pb, nprob, 0, bp, s))) return rc;
  std::vector<int4> items;
  batch_items(bp, nullptr, items);
  if (items.size() != bp.n_items_all) return set_error(ctx, WDL_ERR_INVALID_ARG, "internal: item count mismatch");
  if (ctx->inject_fault == WDL_FAULT_DROP_FIRST_ITERATION) {
    // host-side fault (wdl_inject_fault): no item of the first forward
    // iteration runs, so every other item waits on a flag nothing publishes
    std::vector<int4> kept;
    for (const int4& it : items)
      if (!(it.y == 0 && it.z == 1)) kept.push_back(it);
    items.swap(kept);
    ctx->inject_fault = 0;
  }
  char* base = bp.base;
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(base + bp.items_off, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice, s));
  if ((rc = batch_launch(ctx, bp, items.size(), s))) return rc;
  ctx->fused_sync = bp.sync;
  if (bp.n_outjobs) {
    k_outputs<<<grid_for(bp.n_outjobs, 1, ctx->sm_count, 4), 256, 0, s>>>(reinterpret_cast<OutJob*>(base + bp.outj_off), (int)bp.n_outjobs);
    WDL_LAUNCH_CHECK(ctx);
  }
  // ---- results: one download, scattered on the host --------------------------------
  std::vector<char> h_out(bp.out_e - bp.out_b);
  if (!h_out.empty())
    WDL_CUDA_TRY(ctx, cudaMemcpyAsync(h_out.data(), base + bp.out_b, h_out.size(), cudaMemcpyDeviceToHost, s));
  WDL_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  auto host_of = [&](const double* d) { return h_out.data() + ((const char*)d - base - bp.out_b); };
  for (int q = 0; q < nprob; ++q) {
    const wdl_problem& w = pb[q];
    const size_t N = (size_t)w.W * w.H;
    const BatchBuf& o = bp.buf[q];
    if (o.out_la) std::memcpy(w.result_la, host_of(o.out_la), (size_t)w.P * w.K * 8);
    if (o.out_loss) std::memcpy(w.loss, host_of(o.out_loss), (size_t)w.P * 8);
    if (o.out_bary) std::memcpy(w.bary, host_of(o.out_bary), (size_t)w.P * N * 8);
    if (o.out_dic) std::memcpy(w.result_dic, host_of(o.out_dic), (size_t)w.K * N * 8);
  }
  return tc_check_status(ctx);
}
