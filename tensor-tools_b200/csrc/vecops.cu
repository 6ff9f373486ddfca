// Davidson vector kernels over flat block-sparse vectors (qtensor/qtensor.cpp
// :1031-1179,1606-1647): dot, multi-dot, norm, axpy, scale, linear
// combinations with device-side coefficients, masked random fill and the
// diagonal preconditioner.  All are HBM-bound streaming kernels: 16-byte
// vector loads, a fixed grid (a multiple of the SM count) and a deterministic
// reduction (same summation order on every run): per-block partials, summed in
// block order by the last block of the same launch.
#include <algorithm>
#include <cmath>
#include <atomic>
#include <mutex>
#include <vector>

#include "tt_internal.h"

namespace {

constexpr int RT = 256;       // threads per reduction block
constexpr int MAXVEC = 16;    // vectors per multi-dot / linear combination

inline int red_blocks(tt_ctx* ctx, int64_t n) {
  int64_t want = (n + RT * 4 - 1) / (RT * 4);
  int cap = ctx->num_sms * 4;
  if (want < 1) want = 1;
  return (int)(want < cap ? want : cap);
}

template <int NV>
__device__ __forceinline__ void block_reduce_store(double (&v)[NV], double* out, int stride) {
  __shared__ double sh[NV][RT / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    double x = v[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) sh[j][w] = x;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double s = 0.0;
    for (int i = 0; i < RT / 32; ++i) s += sh[threadIdx.x][i];
    out[threadIdx.x * stride + blockIdx.x] = s;
  }
}

// partial sums of sum_i xs[j][i]*y[i] for j < nv
struct PtrPack {
  const double* p[MAXVEC];
};

template <int NV>
__global__ void __launch_bounds__(RT) multidot_pass1(int64_t n, PtrPack xs,
                                                     const double* __restrict__ y,
                                                     double* part, int nv) {
  double acc[NV];
#pragma unroll
  for (int j = 0; j < NV; ++j) acc[j] = 0.0;
  const int64_t n2 = n / 2;
  const double2* y2 = reinterpret_cast<const double2*>(y);
  for (int64_t i = blockIdx.x * (int64_t)RT + threadIdx.x; i < n2; i += (int64_t)gridDim.x * RT) {
    double2 b = y2[i];
#pragma unroll
    for (int j = 0; j < NV; ++j) {
      if (j < nv) {
        double2 a = reinterpret_cast<const double2*>(xs.p[j])[i];
        acc[j] = fma(a.x, b.x, acc[j]);
        acc[j] = fma(a.y, b.y, acc[j]);
      }
    }
  }
  if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j)
      if (j < nv) acc[j] = fma(xs.p[j][n - 1], y[n - 1], acc[j]);
  }
  block_reduce_store<NV>(acc, part, gridDim.x);
}

// One launch for a whole multi-dot: pass 1 as above, then the last block to
// finish (a ticket counter, reset by that block) sums the per-block partials
// of every vector in the same order as reduce_pass2, so the result is
// bit-identical to the two-launch form.
template <int NV>
__global__ void __launch_bounds__(RT) multidot_fused(int64_t n, PtrPack xs, const double* __restrict__ y,
                                                     double* part, int nv, double* out, int do_sqrt,
                                                     unsigned int* ticket) {
  double acc[NV];
#pragma unroll
  for (int j = 0; j < NV; ++j) acc[j] = 0.0;
  const int64_t n2 = n / 2;
  const double2* y2 = reinterpret_cast<const double2*>(y);
  for (int64_t i = blockIdx.x * (int64_t)RT + threadIdx.x; i < n2; i += (int64_t)gridDim.x * RT) {
    double2 b = y2[i];
#pragma unroll
    for (int j = 0; j < NV; ++j) {
      if (j < nv) {
        double2 a = reinterpret_cast<const double2*>(xs.p[j])[i];
        acc[j] = fma(a.x, b.x, acc[j]);
        acc[j] = fma(a.y, b.y, acc[j]);
      }
    }
  }
  if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j)
      if (j < nv) acc[j] = fma(xs.p[j][n - 1], y[n - 1], acc[j]);
  }
  block_reduce_store<NV>(acc, part, gridDim.x);
  __shared__ bool last;
  __threadfence();  // this block's partials are visible before its ticket is taken
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int j = w; j < nv; j += RT / 32) {
    double s = 0.0;
    for (int i = lane; i < (int)gridDim.x; i += 32) s += __ldcg(part + j * gridDim.x + i);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) out[j] = do_sqrt ? sqrt(s) : s;
  }
  if (threadIdx.x == 0) *ticket = 0u;  // ready for the next reduction on this stream
}

// y -= sum_j coef[j] xs[j], then |y| -- the Gram-Schmidt projection and the
// norm of its result in one launch.  The grid, the pair-wise walk and the fma
// order are those of lincomb_kernel (per element) and of multidot_fused<1>
// (for the norm), so both results are bit-identical to the two launches.
__global__ void __launch_bounds__(RT) project_nrm2_kernel(int64_t n, int nv, PtrPack xs,
                                                          const double* __restrict__ coef, double* y,
                                                          double* part, double* out, unsigned int* ticket,
                                                          const int* cond) {
  if (cond && *cond == 0) return;  // conditional form: every block reads the same flag
  __shared__ double c[MAXVEC];
  if (threadIdx.x < nv) c[threadIdx.x] = -1.0 * coef[threadIdx.x];
  __syncthreads();
  double acc[1] = {0.0};
  const int64_t n2 = n / 2;
  double2* y2 = reinterpret_cast<double2*>(y);
  for (int64_t i = blockIdx.x * (int64_t)RT + threadIdx.x; i < n2; i += (int64_t)gridDim.x * RT) {
    double2 b = y2[i];
    for (int j = 0; j < nv; ++j) {
      const double2 a = reinterpret_cast<const double2*>(xs.p[j])[i];
      b.x = fma(c[j], a.x, b.x);
      b.y = fma(c[j], a.y, b.y);
    }
    y2[i] = b;
    acc[0] = fma(b.x, b.x, acc[0]);
    acc[0] = fma(b.y, b.y, acc[0]);
  }
  if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
    double t = y[n - 1];
    for (int j = 0; j < nv; ++j) t = fma(c[j], xs.p[j][n - 1], t);
    y[n - 1] = t;
    acc[0] = fma(t, t, acc[0]);
  }
  block_reduce_store<1>(acc, part, gridDim.x);
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    double s = 0.0;
    for (int i = lane; i < (int)gridDim.x; i += 32) s += __ldcg(part + i);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) out[0] = sqrt(s);
  }
  if (threadIdx.x == 0) *ticket = 0u;
}

__global__ void reduce_pass2(const double* part, int nblk, int nv, double* out, int do_sqrt) {
  // one warp per output, fixed order
  const int j = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (j >= nv) return;
  double s = 0.0;
  for (int i = lane; i < nblk; i += 32) s += part[j * nblk + i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) out[j] = do_sqrt ? sqrt(s) : s;
}

__global__ void axpy_kernel(int64_t n, double a, const double* __restrict__ x, double* __restrict__ y) {
  const int64_t n2 = n / 2;
  const double2* x2 = reinterpret_cast<const double2*>(x);
  double2* y2 = reinterpret_cast<double2*>(y);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n2; i += (int64_t)gridDim.x * blockDim.x) {
    double2 u = x2[i], v = y2[i];
    v.x = fma(a, u.x, v.x);
    v.y = fma(a, u.y, v.y);
    y2[i] = v;
  }
  if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) y[n - 1] = fma(a, x[n - 1], y[n - 1]);
}

struct ModeScale {
  double v[TT_SCALE_MODE_MAX];
};

// x[i + inner*(m + mid*o)] *= scale[m]: a diagonal operator on one mode of a
// column-major tensor (no alignment requirement: blocks of a qtensor arena
// start at arbitrary element offsets).
__global__ void scale_mode_kernel(int64_t inner, int mid, int64_t total, ModeScale s, double* __restrict__ x) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x)
    x[e] *= s.v[(int)((e / inner) % mid)];
}

__global__ void scal_kernel(int64_t n, double a, const double* d_nrm, double* __restrict__ x) {
  if (d_nrm) a = 1.0 / d_nrm[0];
  const int64_t n2 = n / 2;
  double2* x2 = reinterpret_cast<double2*>(x);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n2; i += (int64_t)gridDim.x * blockDim.x) {
    double2 v = x2[i];
    v.x *= a;
    v.y *= a;
    x2[i] = v;
  }
  if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) x[n - 1] *= a;
}

__global__ void lincomb_kernel(int64_t n, int nv, PtrPack xs, const double* __restrict__ coef,
                               double sign, int accumulate, double* __restrict__ y) {
  __shared__ double c[MAXVEC];
  if (threadIdx.x < nv) c[threadIdx.x] = sign * coef[threadIdx.x];
  __syncthreads();
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double s = accumulate ? y[i] : 0.0;
    for (int j = 0; j < nv; ++j) s = fma(c[j], xs.p[j][i], s);
    y[i] = s;
  }
}

// The Ritz vector and the residual of one Davidson iteration in one pass:
// x = sum_j cx[j] v_j, q = sum_j cq[j] va_j + cq[k] x, with the fma order of
// two lincomb_kernel launches (so the results are bit-identical to them).
__global__ void ritz_residual_kernel(int64_t n, int k, PtrPack vs, PtrPack vas, const double* __restrict__ cx,
                                     const double* __restrict__ cq, double* __restrict__ x, double* __restrict__ q) {
  __shared__ double a[MAXVEC], b[MAXVEC + 1];
  if (threadIdx.x < k) a[threadIdx.x] = cx[threadIdx.x];
  if (threadIdx.x <= k) b[threadIdx.x] = cq[threadIdx.x];
  __syncthreads();
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double xs = 0.0;
    for (int j = 0; j < k; ++j) xs = fma(a[j], vs.p[j][i], xs);
    double qs = 0.0;
    for (int j = 0; j < k; ++j) qs = fma(b[j], vas.p[j][i], qs);
    qs = fma(b[k], xs, qs);
    x[i] = xs;
    q[i] = qs;
  }
}

__device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__global__ void fill_random_kernel(int64_t n, double* x, int nranges, const int64_t* ranges, uint64_t seed) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    // binary search: is i inside one of the sorted [begin,end) ranges?
    int lo = 0, hi = nranges;
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if (ranges[2 * mid + 1] <= i) lo = mid + 1; else hi = mid;
    }
    bool in = lo < nranges && ranges[2 * lo] <= i;
    double v = 0.0;
    if (in) v = (double)(splitmix64(seed ^ (uint64_t)i * 0xD1B54A32D192ED03ull) >> 11) * 0x1.0p-53;
    x[i] = v;
  }
}

__global__ void precondition_kernel(int64_t n, double* __restrict__ x, const double* __restrict__ D, double theta) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double d = D[i];
    if (d != theta) x[i] = x[i] / (d - theta);
  }
}

inline int stream_blocks(tt_ctx* ctx, int64_t n) {
  int64_t want = (n + 511) / 512;
  int cap = ctx->num_sms * 8;
  if (want < 1) want = 1;
  return (int)(want < cap ? want : cap);
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

int launch_multidot(tt_ctx* ctx, int64_t n, int nv, const double* const* xs, const double* y,
                    double* d_out, int do_sqrt) {
  PtrPack pk;
  for (int j = 0; j < nv; ++j) {
    if (!aligned16(xs[j])) return tt::fail(TT_ERR_INVALID, "vectors must be 16-byte aligned");
    pk.p[j] = xs[j];
  }
  int nb = red_blocks(ctx, n);
  double* part = tt::partials(ctx, nb * nv);
  if (!part) return tt::fail(TT_ERR_OOM, "reduction scratch");
  if (nv <= 1)
    multidot_fused<1><<<nb, RT, 0, ctx->stream>>>(n, pk, y, part, nv, d_out, do_sqrt, ctx->d_ticket);
  else if (nv <= 4)
    multidot_fused<4><<<nb, RT, 0, ctx->stream>>>(n, pk, y, part, nv, d_out, do_sqrt, ctx->d_ticket);
  else
    multidot_fused<MAXVEC><<<nb, RT, 0, ctx->stream>>>(n, pk, y, part, nv, d_out, do_sqrt, ctx->d_ticket);
  TT_LAUNCH_CHECK(ctx);
  return TT_OK;
}

// ---- allocation-free multi-dot (tt_vec_multidot_noalloc) --------------------
// Some callers cannot allocate device memory: an application that reserves the
// whole device for its own pool and forbids further allocations, or a plugin
// host that only lends out buffers it owns.  Such a caller cannot create a
// tt_ctx (that allocates its stream, pool and scratch), so this variant keeps
// the reduction partials in a fixed array inside the library instead.
constexpr int NOALLOC_MAX_VEC = MAXVEC;      // at most 16 vectors per call
constexpr int NOALLOC_MAX_BLOCKS = 1024;     // partial sums per vector
// 16 x 1024 doubles = 128 KiB; every GPU that loads the library holds it until exit.
static __device__ __align__(256) double g_noalloc_partials[NOALLOC_MAX_VEC * NOALLOC_MAX_BLOCKS];

// Per-device set-up, cached only once it has succeeded: a failed attempt (for
// example a first call made while an earlier asynchronous error is pending,
// or during stream capture) leaves the slot unset, and the next call retries.
struct NoAllocDevice {
  std::mutex mu;
  std::atomic<bool> ready{false};
  double* partials = nullptr;   // device address of g_noalloc_partials on this device
  int num_sms = 0;
};
constexpr int NOALLOC_MAX_DEVICES = 64;
NoAllocDevice g_noalloc_dev[NOALLOC_MAX_DEVICES];

}  // namespace

extern "C" {

int tt_vec_multidot_noalloc(void* stream, int64_t n, int nvec, const double* const* xs, const double* y,
                            double* d_out) {
  TT_REQUIRE(xs && y && d_out, "tt_vec_multidot_noalloc: null argument");
  TT_REQUIRE(n >= 0, "tt_vec_multidot_noalloc: negative length");
  if (nvec < 1 || nvec > NOALLOC_MAX_VEC)
    return tt::fail(TT_ERR_INVALID, "tt_vec_multidot_noalloc: nvec must be 1..16 (fixed scratch of 16 x 1024 "
                                    "partial sums)");
  TT_REQUIRE(aligned16(y), "tt_vec_multidot_noalloc: vectors must be 16-byte aligned");
  int dev = 0;
  TT_CUDA(cudaGetDevice(&dev));
  TT_REQUIRE(dev >= 0 && dev < NOALLOC_MAX_DEVICES, "tt_vec_multidot_noalloc: device ordinal too large");
  NoAllocDevice& D = g_noalloc_dev[dev];
  // once per device, with that device current: the host needs the array's
  // device address (its host-side name is only a stand-in)
  if (!D.ready.load(std::memory_order_acquire)) {
    std::lock_guard<std::mutex> lock(D.mu);
    if (!D.ready.load(std::memory_order_relaxed)) {
      void* p = nullptr;
      int sms = 0;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
      if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      if (e != cudaSuccess) return tt::cuda_fail(e, "tt_vec_multidot_noalloc set-up", __FILE__, __LINE__);
      D.partials = static_cast<double*>(p);
      D.num_sms = sms;
      D.ready.store(true, std::memory_order_release);
    }
  }
  PtrPack pk;
  for (int j = 0; j < nvec; ++j) {
    TT_REQUIRE(xs[j] && aligned16(xs[j]), "tt_vec_multidot_noalloc: vectors must be 16-byte aligned");
    pk.p[j] = xs[j];
  }
  int64_t want = (n + RT * 4 - 1) / (RT * 4);
  int64_t cap = std::min<int64_t>(4 * (int64_t)D.num_sms, NOALLOC_MAX_BLOCKS);
  int nb = (int)std::max<int64_t>(1, std::min(want, cap));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // every partial that pass 2 reads is written by pass 1 first: nothing needs zeroing
  if (nvec <= 1)
    multidot_pass1<1><<<nb, RT, 0, s>>>(n, pk, y, D.partials, nvec);
  else if (nvec <= 4)
    multidot_pass1<4><<<nb, RT, 0, s>>>(n, pk, y, D.partials, nvec);
  else
    multidot_pass1<MAXVEC><<<nb, RT, 0, s>>>(n, pk, y, D.partials, nvec);
  TT_CUDA(cudaGetLastError());
  reduce_pass2<<<1, 32 * nvec, 0, s>>>(D.partials, nb, nvec, d_out, 0);
  TT_CUDA(cudaGetLastError());
  return TT_OK;
}

int tt_vec_multidot(tt_ctx* ctx, int64_t n, int nvec, const double* const* xs, const double* y,
                    double* d_out) {
  TT_REQUIRE(ctx && xs && y && d_out, "tt_vec_multidot: null argument");
  TT_REQUIRE(nvec >= 1 && nvec <= MAXVEC, "tt_vec_multidot: 1..16 vectors");
  TT_REQUIRE(aligned16(y), "tt_vec_multidot: vectors must be 16-byte aligned");
  return launch_multidot(ctx, n, nvec, xs, y, d_out, 0);
}

int tt_vec_dot(tt_ctx* ctx, int64_t n, const double* x, const double* y, double* d_out) {
  TT_REQUIRE(ctx && x && y && d_out, "tt_vec_dot: null argument");
  TT_REQUIRE(aligned16(y), "tt_vec_dot: vectors must be 16-byte aligned");
  const double* xs[1] = {x};
  return launch_multidot(ctx, n, 1, xs, y, d_out, 0);
}

int tt_vec_nrm2(tt_ctx* ctx, int64_t n, const double* x, double* d_out) {
  TT_REQUIRE(ctx && x && d_out, "tt_vec_nrm2: null argument");
  TT_REQUIRE(aligned16(x), "tt_vec_nrm2: vectors must be 16-byte aligned");
  const double* xs[1] = {x};
  return launch_multidot(ctx, n, 1, xs, x, d_out, 1);
}

int tt_vec_axpy(tt_ctx* ctx, int64_t n, double a, const double* x, double* y) {
  TT_REQUIRE(ctx && x && y, "tt_vec_axpy: null argument");
  TT_REQUIRE(aligned16(x) && aligned16(y), "tt_vec_axpy: vectors must be 16-byte aligned");
  if (n <= 0) return TT_OK;
  axpy_kernel<<<stream_blocks(ctx, n), 256, 0, ctx->stream>>>(n, a, x, y);
  TT_LAUNCH_CHECK(ctx);
  return TT_OK;
}

int tt_vec_scal(tt_ctx* ctx, int64_t n, double a, double* x) {
  TT_REQUIRE(ctx && x, "tt_vec_scal: null argument");
  TT_REQUIRE(aligned16(x), "tt_vec_scal: vectors must be 16-byte aligned");
  if (n <= 0) return TT_OK;
  scal_kernel<<<stream_blocks(ctx, n), 256, 0, ctx->stream>>>(n, a, nullptr, x);
  TT_LAUNCH_CHECK(ctx);
  return TT_OK;
}

int tt_vec_scale_mode(tt_ctx* ctx, int64_t inner, int mid, int64_t outer, const double* scale, double* x) {
  TT_REQUIRE(ctx && x && scale, "tt_vec_scale_mode: null argument");
  TT_REQUIRE(inner >= 0 && outer >= 0 && mid >= 1 && mid <= TT_SCALE_MODE_MAX, "tt_vec_scale_mode: bad extents");
  int64_t total = inner * mid * outer;
  if (total == 0) return TT_OK;
  ModeScale s{};
  for (int m = 0; m < mid; ++m) s.v[m] = scale[m];
  scale_mode_kernel<<<stream_blocks(ctx, total), 256, 0, ctx->stream>>>(inner, mid, total, s, x);
  TT_LAUNCH_CHECK(ctx);
  return TT_OK;
}

int tt_vec_scal_inv_dev(tt_ctx* ctx, int64_t n, const double* d_nrm, double* x) {
  TT_REQUIRE(ctx && x && d_nrm, "tt_vec_scal_inv_dev: null argument");
  TT_REQUIRE(aligned16(x), "tt_vec_scal_inv_dev: vectors must be 16-byte aligned");
  if (n <= 0) return TT_OK;
  scal_kernel<<<stream_blocks(ctx, n), 256, 0, ctx->stream>>>(n, 1.0, d_nrm, x);
  TT_LAUNCH_CHECK(ctx);
  return TT_OK;
}

int tt_vec_lincomb_dev(tt_ctx* ctx, int64_t n, int nvec, const double* const* xs,
                       const double* d_coef, double sign, int accumulate, double* y) {
  TT_REQUIRE(ctx && xs && d_coef && y, "tt_vec_lincomb_dev: null argument");
  TT_REQUIRE(nvec >= 0 && nvec <= MAXVEC, "tt_vec_lincomb_dev: 0..16 vectors");
  PtrPack pk;
  for (int j = 0; j < nvec; ++j) pk.p[j] = xs[j];
  if (n <= 0) return TT_OK;
  lincomb_kernel<<<stream_blocks(ctx, n), 256, 0, ctx->stream>>>(n, nvec, pk, d_coef, sign, accumulate, y);
  TT_LAUNCH_CHECK(ctx);
  return TT_OK;
}

int tt_vec_project_nrm2_dev_if(tt_ctx* ctx, int64_t n, int nvec, const double* const* xs, const double* d_coef,
                               double* y, double* d_norm, const int* d_cond) {
  TT_REQUIRE(ctx && xs && d_coef && y && d_norm, "tt_vec_project_nrm2_dev: null argument");
  TT_REQUIRE(nvec >= 0 && nvec <= MAXVEC, "tt_vec_project_nrm2_dev: 0..16 vectors");
  TT_REQUIRE(aligned16(y), "tt_vec_project_nrm2_dev: vectors must be 16-byte aligned");
  PtrPack pk;
  for (int j = 0; j < nvec; ++j) {
    if (!aligned16(xs[j])) return tt::fail(TT_ERR_INVALID, "tt_vec_project_nrm2_dev: vectors must be 16-byte aligned");
    pk.p[j] = xs[j];
  }
  const int nb = red_blocks(ctx, n);
  double* part = tt::partials(ctx, nb);
  if (!part) return tt::fail(TT_ERR_OOM, "reduction scratch");
  project_nrm2_kernel<<<nb, RT, 0, ctx->stream>>>(n, nvec, pk, d_coef, y, part, d_norm, ctx->d_ticket, d_cond);
  TT_LAUNCH_CHECK(ctx);
  return TT_OK;
}

int tt_vec_project_nrm2_dev(tt_ctx* ctx, int64_t n, int nvec, const double* const* xs, const double* d_coef,
                            double* y, double* d_norm) {
  return tt_vec_project_nrm2_dev_if(ctx, n, nvec, xs, d_coef, y, d_norm, nullptr);
}

int tt_vec_ritz_residual_dev(tt_ctx* ctx, int64_t n, int k, const double* const* vs, const double* const* vas,
                             const double* d_coef_x, const double* d_coef_q, double* x, double* q) {
  TT_REQUIRE(ctx && vs && vas && d_coef_x && d_coef_q && x && q, "tt_vec_ritz_residual_dev: null argument");
  TT_REQUIRE(k >= 1 && k < MAXVEC, "tt_vec_ritz_residual_dev: 1..15 vectors");
  PtrPack pv, pa;
  for (int j = 0; j < k; ++j) {
    pv.p[j] = vs[j];
    pa.p[j] = vas[j];
  }
  if (n <= 0) return TT_OK;
  ritz_residual_kernel<<<stream_blocks(ctx, n), 256, 0, ctx->stream>>>(n, k, pv, pa, d_coef_x, d_coef_q, x, q);
  TT_LAUNCH_CHECK(ctx);
  return TT_OK;
}

int tt_vec_fill_random(tt_ctx* ctx, int64_t n, double* x, int nranges, const int64_t* d_ranges,
                       uint64_t seed) {
  TT_REQUIRE(ctx && x && (nranges == 0 || d_ranges), "tt_vec_fill_random: null argument");
  if (n <= 0) return TT_OK;
  fill_random_kernel<<<stream_blocks(ctx, n), 256, 0, ctx->stream>>>(n, x, nranges, d_ranges, seed);
  TT_LAUNCH_CHECK(ctx);
  return TT_OK;
}

int tt_vec_precondition(tt_ctx* ctx, int64_t n, double* x, const double* D, double theta) {
  TT_REQUIRE(ctx && x && D, "tt_vec_precondition: null argument");
  if (n <= 0) return TT_OK;
  precondition_kernel<<<stream_blocks(ctx, n), 256, 0, ctx->stream>>>(n, x, D, theta);
  TT_LAUNCH_CHECK(ctx);
  return TT_OK;
}

}  // extern "C"
