// Grouped block-sparse contraction: every (output block, block pair) GEMM of
// one qtensor::operator* (qtensor/qtensor.cpp:652-726) in a single launch.
//
// FP64 path: 64x64 CTA tiles, BK=16, 3-stage cp.async pipeline, four warps
// of 32x32 built from mma.sync m8n8k4 f64 (DMMA).  Operands are gathered
// through per-pair offset tables (row/column offsets of the strided tensor
// blocks), so any index permutation of the contraction is handled without a
// transpose pass; the tables are expanded on the device from the pair
// descriptors when the plan is built.
#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

#include "tt_internal.h"

namespace {

constexpr int BM = 64;
constexpr int BN = 64;
constexpr int BK = 16;
constexpr int STAGES = 3;
constexpr int THREADS = 128;
constexpr int SA = BM + 4;  // padded k-rows: conflict-free 8-byte fragment loads
constexpr int SB = BN + 4;
constexpr size_t SMEM_BYTES = sizeof(double) * STAGES * BK * (SA + SB);

struct PairDev {
  int64_t a_off, b_off;
  int32_t m, n, k;
  int32_t rowA, colA, rowB, colB;  // offsets of the tables in the table buffer
  int32_t a_mfast, b_kfast;        // unit stride along m (A) / along k (B)
};

struct TaskDev {
  int32_t out;
  int32_t m0, n0;
  int32_t p_begin, p_end;
};

struct OutDev {
  int64_t c_off;
  int32_t m, n, ldc;
};

struct TableJob {  // one of the four offset tables of a pair
  int32_t dst;     // offset in the table buffer
  int32_t len;
  int32_t nmodes;
  int32_t dims[TT_MAX_MODES];
  int64_t strides[TT_MAX_MODES];
};

__global__ void expand_tables(const TableJob* jobs, int njobs, int32_t* tab) {
  int j = blockIdx.x;
  if (j >= njobs) return;
  const TableJob& J = jobs[j];
  for (int i = threadIdx.x; i < J.len; i += blockDim.x) {
    int64_t off = 0;
    int r = i;
    for (int d = 0; d < J.nmodes; ++d) {
      int q = r / J.dims[d];
      off += (int64_t)(r - q * J.dims[d]) * J.strides[d];
      r = q;
    }
    tab[J.dst + i] = (int32_t)off;
  }
}

__device__ __forceinline__ void cp_async8(double* smem, const double* gmem, bool pred) {
  unsigned saddr = (unsigned)__cvta_generic_to_shared(smem);
  int src_bytes = pred ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(saddr), "l"(gmem),
               "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(c[0]), "+d"(c[1])
      : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(THREADS)
grouped_dgemm(const TaskDev* __restrict__ tasks, const OutDev* __restrict__ outs,
              const PairDev* __restrict__ pairs, const int32_t* __restrict__ tab,
              const double* __restrict__ A, const double* __restrict__ B,
              double* __restrict__ C, double alpha) {
  extern __shared__ double smem[];
  double* As = smem;                        // [STAGES][BK][SA]
  double* Bs = smem + STAGES * BK * SA;     // [STAGES][BK][SB]
  __shared__ int32_t rowA_s[BM];
  __shared__ int32_t colB_s[BN];

  const TaskDev task = tasks[blockIdx.x];
  const OutDev out = outs[task.out];
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int wm = (warp & 1) * 32;
  const int wn = (warp >> 1) * 32;
  const int g = lane >> 2;  // groupID
  const int t4 = lane & 3;  // thread in group

  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  for (int p = task.p_begin; p < task.p_end; ++p) {
    const PairDev P = pairs[p];
    __syncthreads();  // previous pair finished with rowA_s / colB_s / stages
    if (tid < BM) {
      int m = task.m0 + tid;
      rowA_s[tid] = m < P.m ? tab[P.rowA + m] : 0;
    } else {
      int n = task.n0 + tid - BM;
      colB_s[tid - BM] = n < P.n ? tab[P.colB + n] : 0;
    }
    __syncthreads();
    const double* Ab = A + P.a_off;
    const double* Bb = B + P.b_off;
    const int K = P.k;
    const int nchunks = (K + BK - 1) / BK;

    auto load_stage = [&](int chunk, int stage) {
      const int k0 = chunk * BK;
      double* as = As + stage * BK * SA;
      double* bs = Bs + stage * BK * SB;
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        int m, k;
        if (P.a_mfast) {
          m = tid & 63;
          k = (tid >> 6) + 2 * r;
        } else {
          k = tid & 15;
          m = (tid >> 4) + 8 * r;
        }
        int gk = k0 + k;
        bool ok = (task.m0 + m < P.m) && (gk < K);
        const double* src = ok ? Ab + rowA_s[m] + tab[P.colA + gk] : Ab;
        cp_async8(as + k * SA + m, src, ok);
      }
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        int n, k;
        if (P.b_kfast) {
          k = tid & 15;
          n = (tid >> 4) + 8 * r;
        } else {
          n = tid & 63;
          k = (tid >> 6) + 2 * r;
        }
        int gk = k0 + k;
        bool ok = (task.n0 + n < P.n) && (gk < K);
        const double* src = ok ? Bb + tab[P.rowB + gk] + colB_s[n] : Bb;
        cp_async8(bs + k * SB + n, src, ok);
      }
    };

#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
      if (s < nchunks) load_stage(s, s);
      cp_async_commit();
    }
    for (int c = 0; c < nchunks; ++c) {
      cp_async_wait<STAGES - 2>();
      __syncthreads();
      const int stage = c % STAGES;
      const double* as = As + stage * BK * SA;
      const double* bs = Bs + stage * BK * SB;
      const int ksteps = min(BK / 4, (K - c * BK + 3) >> 2);
      for (int kk = 0; kk < ksteps; ++kk) {
        double af[4], bf[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) af[i] = as[(kk * 4 + t4) * SA + wm + i * 8 + g];
#pragma unroll
        for (int j = 0; j < 4; ++j) bf[j] = bs[(kk * 4 + t4) * SB + wn + j * 8 + g];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) dmma(acc[i][j], af[i], bf[j]);
      }
      const int nxt = c + STAGES - 1;
      if (nxt < nchunks) load_stage(nxt, nxt % STAGES);
      cp_async_commit();
    }
    cp_async_wait<0>();
  }

  // epilogue: C tile = alpha * acc (blocks without pairs get zeros)
  double* Cb = C + out.c_off;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    int m = task.m0 + wm + i * 8 + g;
    if (m >= out.m) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        int n = task.n0 + wn + j * 8 + 2 * t4 + e;
        if (n < out.n) Cb[m + (int64_t)out.ldc * n] = alpha * acc[i][j][e];
      }
    }
  }
}

}  // namespace

struct tt_plan {
  int precision = TT_PREC_FP64;
  int n_tasks = 0;
  int n_pairs = 0;
  int n_out = 0;
  double flops = 0.0;
  TaskDev* d_tasks = nullptr;
  OutDev* d_outs = nullptr;
  PairDev* d_pairs = nullptr;
  int32_t* d_tab = nullptr;
};

extern "C" {

int tt_contract_plan(tt_ctx* ctx, const tt_out_block* outs, int n_out,
                     const tt_block_pair* pairs, int n_pairs, int precision,
                     tt_plan** plan_out) {
  TT_REQUIRE(ctx && plan_out, "tt_contract_plan: null argument");
  TT_REQUIRE(n_out >= 0 && n_pairs >= 0, "tt_contract_plan: negative count");
  TT_REQUIRE(precision == TT_PREC_FP64, "tt_contract_plan: unsupported precision");
  *plan_out = nullptr;
  // pairs grouped by output block (stable: keeps the reference's accumulation order)
  std::vector<int> order(n_pairs);
  std::iota(order.begin(), order.end(), 0);
  for (int i = 0; i < n_pairs; ++i)
    TT_REQUIRE(pairs[i].out_block >= 0 && pairs[i].out_block < n_out,
               "tt_contract_plan: pair references a missing output block");
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return pairs[a].out_block < pairs[b].out_block; });
  std::vector<PairDev> hp(n_pairs);
  std::vector<TableJob> jobs;
  jobs.reserve(4 * (size_t)n_pairs);
  int64_t tab_len = 0;
  double flops = 0.0;
  std::vector<int> first(n_out + 1, 0);
  std::vector<int64_t> work(n_out, 0);
  for (int ii = 0; ii < n_pairs; ++ii) {
    const tt_block_pair& q = pairs[order[ii]];
    TT_REQUIRE(q.n_m >= 0 && q.n_m <= TT_MAX_MODES && q.n_k >= 0 && q.n_k <= TT_MAX_MODES &&
                   q.n_n >= 0 && q.n_n <= TT_MAX_MODES,
               "tt_contract_plan: mode count out of range");
    int64_t m = 1, n = 1, k = 1;
    for (int i = 0; i < q.n_m; ++i) m *= q.m_dims[i];
    for (int i = 0; i < q.n_k; ++i) k *= q.k_dims[i];
    for (int i = 0; i < q.n_n; ++i) n *= q.n_dims[i];
    const tt_out_block& o = outs[q.out_block];
    TT_REQUIRE(m == o.m && n == o.n, "tt_contract_plan: pair shape does not match its output block");
    TT_REQUIRE(m < (1ll << 31) && n < (1ll << 31) && k < (1ll << 31), "tt_contract_plan: block too large");
    PairDev P;
    P.a_off = q.a_off;
    P.b_off = q.b_off;
    P.m = (int)m;
    P.n = (int)n;
    P.k = (int)k;
    auto add_job = [&](int len, int nmodes, const int32_t* dims, const int64_t* strides) {
      TableJob J;
      memset(&J, 0, sizeof(J));
      J.dst = (int32_t)tab_len;
      J.len = len;
      J.nmodes = nmodes;
      for (int i = 0; i < nmodes; ++i) {
        J.dims[i] = dims[i];
        J.strides[i] = strides[i];
      }
      jobs.push_back(J);
      tab_len += len;
      return J.dst;
    };
    P.rowA = add_job((int)m, q.n_m, q.m_dims, q.a_m_stride);
    P.colA = add_job((int)k, q.n_k, q.k_dims, q.a_k_stride);
    P.rowB = add_job((int)k, q.n_k, q.k_dims, q.b_k_stride);
    P.colB = add_job((int)n, q.n_n, q.n_dims, q.b_n_stride);
    // coalescing choice only: walk the operand along its unit-stride mode
    bool a_m_unit = q.n_m > 0 && q.a_m_stride[0] == 1;
    bool a_k_unit = q.n_k > 0 && q.a_k_stride[0] == 1;
    P.a_mfast = (a_m_unit || !a_k_unit) ? 1 : 0;
    bool b_k_unit = q.n_k > 0 && q.b_k_stride[0] == 1;
    P.b_kfast = b_k_unit ? 1 : 0;
    hp[ii] = P;
    first[q.out_block + 1]++;
    work[q.out_block] += k;
    flops += 2.0 * (double)m * (double)n * (double)k;
  }
  TT_REQUIRE(tab_len < (1ll << 31), "tt_contract_plan: offset tables too large");
  for (int o = 0; o < n_out; ++o) first[o + 1] += first[o];
  // tile tasks, longest first (LPT) so heavy blocks start early
  std::vector<TaskDev> tasks;
  std::vector<int64_t> tcost;
  for (int o = 0; o < n_out; ++o) {
    TT_REQUIRE(outs[o].m >= 0 && outs[o].n >= 0 && outs[o].ldc >= outs[o].m,
               "tt_contract_plan: bad output block");
    for (int m0 = 0; m0 < outs[o].m; m0 += BM)
      for (int n0 = 0; n0 < outs[o].n; n0 += BN) {
        TaskDev t{o, m0, n0, first[o], first[o + 1]};
        tasks.push_back(t);
        tcost.push_back(work[o] + 1);
      }
  }
  std::vector<int> torder(tasks.size());
  std::iota(torder.begin(), torder.end(), 0);
  std::stable_sort(torder.begin(), torder.end(), [&](int a, int b) { return tcost[a] > tcost[b]; });
  std::vector<TaskDev> tsorted(tasks.size());
  for (size_t i = 0; i < tasks.size(); ++i) tsorted[i] = tasks[torder[i]];
  std::vector<OutDev> ho(n_out);
  for (int o = 0; o < n_out; ++o) ho[o] = OutDev{outs[o].c_off, outs[o].m, outs[o].n, outs[o].ldc};

  tt_plan* plan = new tt_plan();
  plan->precision = precision;
  plan->n_tasks = (int)tsorted.size();
  plan->n_pairs = n_pairs;
  plan->n_out = n_out;
  plan->flops = flops;
  plan->d_tasks = tt::pool_alloc<TaskDev>(ctx, tsorted.size());
  plan->d_outs = tt::pool_alloc<OutDev>(ctx, ho.size());
  plan->d_pairs = tt::pool_alloc<PairDev>(ctx, hp.size());
  plan->d_tab = tt::pool_alloc<int32_t>(ctx, (size_t)tab_len);
  TableJob* d_jobs = tt::pool_alloc<TableJob>(ctx, jobs.size());
  if (!plan->d_tasks || !plan->d_outs || !plan->d_pairs || !plan->d_tab || !d_jobs) {
    tt_plan_destroy(ctx, plan);
    tt::pool_free(ctx, d_jobs);
    return tt::fail(TT_ERR_OOM, "tt_contract_plan: device allocation failed");
  }
  cudaStream_t s = ctx->stream;
  // staged copies: the host vectors may die at return without stalling the stream
  TT_CUDA(tt::h2d_async(ctx, plan->d_tasks, tsorted.data(), sizeof(TaskDev) * tsorted.size()));
  TT_CUDA(tt::h2d_async(ctx, plan->d_outs, ho.data(), sizeof(OutDev) * ho.size()));
  TT_CUDA(tt::h2d_async(ctx, plan->d_pairs, hp.data(), sizeof(PairDev) * hp.size()));
  TT_CUDA(tt::h2d_async(ctx, d_jobs, jobs.data(), sizeof(TableJob) * jobs.size()));
  if (!jobs.empty()) {
    expand_tables<<<(unsigned)jobs.size(), 128, 0, s>>>(d_jobs, (int)jobs.size(), plan->d_tab);
    TT_LAUNCH_CHECK(ctx);
  }
  tt::pool_free(ctx, d_jobs);  // stream-ordered: freed after expand_tables ran
  *plan_out = plan;
  return TT_OK;
}

int tt_contract_exec(tt_ctx* ctx, const tt_plan* plan, const double* A, const double* B,
                     double* C, double alpha) {
  TT_REQUIRE(ctx && plan, "tt_contract_exec: null argument");
  if (plan->n_tasks == 0) return TT_OK;
  static bool attr_set = false;
  if (!attr_set) {
    TT_CUDA(cudaFuncSetAttribute(grouped_dgemm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)SMEM_BYTES));
    attr_set = true;
  }
  grouped_dgemm<<<plan->n_tasks, THREADS, SMEM_BYTES, ctx->stream>>>(
      plan->d_tasks, plan->d_outs, plan->d_pairs, plan->d_tab, A, B, C, alpha);
  TT_LAUNCH_CHECK(ctx);
  return TT_OK;
}

int tt_plan_destroy(tt_ctx* ctx, tt_plan* plan) {
  if (!plan) return TT_OK;
  if (ctx) {
    tt::pool_free(ctx, plan->d_tasks);
    tt::pool_free(ctx, plan->d_outs);
    tt::pool_free(ctx, plan->d_pairs);
    tt::pool_free(ctx, plan->d_tab);
  }
  delete plan;
  return TT_OK;
}

int tt_plan_flops(const tt_plan* plan, double* flops) {
  TT_REQUIRE(plan && flops, "tt_plan_flops: null argument");
  *flops = plan->flops;
  return TT_OK;
}

}  // extern "C"
