// Device-resident control of tensor_davidsonIT (linalg/tensor_davidson.cpp:193-347).
//
// The host enqueues every iteration of the Davidson loop up front -- products,
// Gram-Schmidt, norms, linear combinations -- and these small control kernels
// carry the decisions that the host loop would otherwise make after reading
// scalars back: the Rayleigh-Ritz step (DIAG of the <= 16 x 16 projected
// matrix, the sign stabilisation, the Ritz coefficients), the convergence
// test, and the bookkeeping of the projected matrix M / Mnext.  Once the loop
// is done (converged, exhausted, or a Gram-Schmidt failure that the host
// handles with its own loop) later control kernels are no-ops, and the host
// reads the state once at the end.  One thread does the work (n <= 16).
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>

#include "tt_internal.h"

struct tt_dav_state {
  int done;      // 1 once the loop has ended
  int final_ii;  // iteration at which it ended (-2: Gram-Schmidt failure at fail_ii)
  int fail_ii;
  int iters;
  int refill;      // 1 while the current new vector is a random refill to orthogonalise
  int randomized;  // random refills in this call
  int cur;       // which of buf[0], buf[1] holds M (the other holds Mnext)
  double lambda, last_lambda, qnorm, gsnorm;
  double buf[2][TT_DAV_MAX * TT_DAV_MAX];
  double evals[TT_DAV_MAX];
  double coef_x[TT_DAV_MAX];      // Ritz vector:   x = sum_k coef_x[k] v[k]
  double coef_q[TT_DAV_MAX + 1];  // residual:      q = sum_k coef_q[k] va[k] + coef_q[ii+1] x
};

namespace {

// DIAG (linalg/lapack_wrapper.cpp:40-54, dsyev semantics) for one warp:
// parallel cyclic Jacobi with the round-robin ordering (every round rotates
// n/2 disjoint index pairs at once; Golub & Van Loan, "Matrix Computations",
// 4th ed., sec. 8.5.5), stopping when the off-diagonal mass falls below
// 1e-32 of the total, as the host DIAG does.  Eigenvalues ascending in ev,
// eigenvectors in the columns of M (column-major, n x n).  All 32 lanes call it.
__device__ void dav_diag_warp(int n, double* M, double* ev) {
  __shared__ double A[TT_DAV_MAX * TT_DAV_MAX], V[TT_DAV_MAX * TT_DAV_MAX];
  __shared__ double cs[TT_DAV_MAX / 2], sn[TT_DAV_MAX / 2];
  __shared__ int pp[TT_DAV_MAX / 2], qq[TT_DAV_MAX / 2];
  __shared__ int order[TT_DAV_MAX];
  const int lane = threadIdx.x & 31;
  for (int i = lane; i < n * n; i += 32) {
    A[i] = M[i];
    V[i] = (i % n == i / n) ? 1.0 : 0.0;
  }
  __syncwarp();
  const int N = n + (n & 1);  // even number of players; index n is a bye when n is odd
  const int npair = N / 2;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, fro = 0.0;
    for (int i = lane; i < n * n; i += 32) {
      const double a2 = A[i] * A[i];
      fro += a2;
      if (i % n != i / n) off += a2;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      off += __shfl_down_sync(0xffffffffu, off, o);
      fro += __shfl_down_sync(0xffffffffu, fro, o);
    }
    off = __shfl_sync(0xffffffffu, off, 0);  // lane 0's sums decide for the whole warp
    fro = __shfl_sync(0xffffffffu, fro, 0);
    if (off <= 1e-32 * fro || off == 0.0) break;
    for (int r = 0; r < N - 1; ++r) {
      if (lane < npair) {
        // round-robin: player 0 fixed, the others rotate by r
        auto player = [&](int i) { return i == 0 ? 0 : ((i - 1 + r) % (N - 1)) + 1; };
        int a = player(lane), b = player(N - 1 - lane);
        int p = a < b ? a : b, q = a < b ? b : a;
        double c = 1.0, sv = 0.0;
        if (q < n) {
          const double apq = A[p + n * q];
          if (apq != 0.0) {
            const double tau = (A[q + n * q] - A[p + n * p]) / (2.0 * apq);
            const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            c = 1.0 / sqrt(1.0 + t * t);
            sv = t * c;
          }
        } else {
          q = p;  // bye: identity rotation
        }
        pp[lane] = p;
        qq[lane] = q;
        cs[lane] = c;
        sn[lane] = sv;
      }
      __syncwarp();
      // A <- A J and V <- V J (columns p, q of every pair), then A <- J^T A (rows)
      for (int it = lane; it < npair * n; it += 32) {
        const int t = it / n, k = it % n;
        const int p = pp[t], q = qq[t];
        if (p == q || sn[t] == 0.0) continue;
        const double c = cs[t], sv = sn[t];
        const double akp = A[k + n * p], akq = A[k + n * q];
        A[k + n * p] = c * akp - sv * akq;
        A[k + n * q] = sv * akp + c * akq;
        const double vkp = V[k + n * p], vkq = V[k + n * q];
        V[k + n * p] = c * vkp - sv * vkq;
        V[k + n * q] = sv * vkp + c * vkq;
      }
      __syncwarp();
      for (int it = lane; it < npair * n; it += 32) {
        const int t = it / n, k = it % n;
        const int p = pp[t], q = qq[t];
        if (p == q || sn[t] == 0.0) continue;
        const double c = cs[t], sv = sn[t];
        const double apk = A[p + n * k], aqk = A[q + n * k];
        A[p + n * k] = c * apk - sv * aqk;
        A[q + n * k] = sv * apk + c * aqk;
      }
      __syncwarp();
      if (lane < npair && pp[lane] != qq[lane] && sn[lane] != 0.0) A[pp[lane] + n * qq[lane]] = A[qq[lane] + n * pp[lane]] = 0.0;
      __syncwarp();
    }
  }
  if (lane == 0) {  // stable insertion sort by eigenvalue
    for (int i = 0; i < n; ++i) order[i] = i;
    for (int i = 1; i < n; ++i) {
      const int o = order[i];
      int j = i - 1;
      while (j >= 0 && A[order[j] + n * order[j]] > A[o + n * o]) {
        order[j + 1] = order[j];
        --j;
      }
      order[j + 1] = o;
    }
  }
  __syncwarp();
  for (int j = lane; j < n; j += 32) ev[j] = A[order[j] + n * order[j]];
  for (int i = lane; i < n * n; i += 32) M[i] = V[(i % n) + n * order[i / n]];
  __syncwarp();
}

__global__ void dav_begin_kernel(tt_dav_state* st, const double* init_en) {
  if (threadIdx.x != 0) return;
  st->done = 0;
  st->final_ii = -1;
  st->fail_ii = -1;
  st->iters = 0;
  st->cur = 0;
  st->refill = 0;
  st->randomized = 0;
  st->last_lambda = 1000.0;
  const double lam = init_en[0];
  st->lambda = lam;
  st->buf[0][0] = lam;  // M[0] = Mnext[0] = lambda
  st->buf[1][0] = lam;
  st->coef_q[0] = 1.0;  // q = va[0] - lambda v[0]
  st->coef_q[1] = -lam;
}

__global__ void dav_ritz_kernel(tt_dav_state* st, int ii) {
  if (st->done) return;  // uniform: read before anything is written
  const int lane = threadIdx.x & 31;
  const int ni = ii + 1;
  double* M = st->buf[st->cur];
  double* Mn = st->buf[1 - st->cur];
  for (int e = lane; e < ni * ni; e += 32) {
    const int mi = e / ni, mj = e % ni;
    if (mj <= mi) {
      Mn[mj + mi * (ni + 1)] = M[mj + mi * ni];
      Mn[mi + mj * (ni + 1)] = M[mi + mj * ni];
    }
  }
  __syncwarp();
  dav_diag_warp(ni, M, st->evals);
  if (lane == 0) {
    const double lam = st->evals[0];
    st->lambda = lam;
    const double sgn = (M[0] < 0.0) ? -1.0 : 1.0;  // sign stabilisation (:265-268)
    for (int k = 0; k <= ii; ++k) {
      st->coef_x[k] = sgn * M[k];
      st->coef_q[k] = sgn * M[k];
    }
    st->coef_q[ii + 1] = -lam;
  }
}

__global__ void dav_conv_kernel(tt_dav_state* st, int ii, int maxiter, double tol, const double* qnorm) {
  if (threadIdx.x != 0 || st->done) return;
  const double qn = qnorm[0];
  const double lam = st->lambda;
  const bool converged = (qn < tol && fabs(lam - st->last_lambda) < tol) || qn < fmax(1e-12, tol * 1e-3);
  st->last_lambda = lam;
  st->qnorm = qn;
  st->iters = ii;
  if (qn < 1e-20 || (converged && ii >= 1) || ii == maxiter) {
    st->done = 1;
    st->final_ii = ii;
  }
}

__global__ void dav_row_kernel(tt_dav_state* st, int ii, const double* row, const double* gsnorm) {
  if (threadIdx.x != 0 || st->done) return;
  const double g = gsnorm[0];
  st->gsnorm = g;
  if (!(g >= 1e-10)) {
    // the random refill failed too (the space is exhausted): the loop ends
    // with the current Ritz vector, as the reference does after its retries
    st->done = 1;
    st->final_ii = ii;
    st->fail_ii = ii;
    return;
  }
  const int ni = ii + 1;
  st->cur = 1 - st->cur;  // swap(M, Mnext)
  double* M = st->buf[st->cur];
  const int l = ni;
  for (int k = 0; k < ni + 1; ++k) {
    M[l + k * (ni + 1)] = row[k];
    M[k + l * (ni + 1)] = row[k];
  }
}

// Gram-Schmidt failure inside the loop (linalg/tensor_davidson.cpp:298-316):
// when the projected new vector's norm is below 1e-10 the reference refills it
// with random numbers on the blocks of the previous vector and orthogonalises
// it again; when the vectors already span the problem (ni >= size) the loop
// ends instead.  One launch: every block reads the same norm and decides
// alike (all of them return when there is nothing to do); on a refill each
// thread draws its elements (the counter-based generator of
// tt_vec_fill_random), stores them and accumulates their overlaps with the
// earlier vectors, and the last block (ticket) sums the per-block partials in
// block order into dots and raises st->refill for the conditional
// projection that follows.
constexpr int RF_THREADS = 256;
struct RefillVecs {
  const double* p[TT_DAV_MAX];
};

__device__ __forceinline__ uint64_t rf_mix(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__global__ void __launch_bounds__(RF_THREADS)
dav_refill_kernel(tt_dav_state* st, int ii, int ni, int maxsize, int64_t n, RefillVecs xs, double* y, int nranges,
                  const int64_t* ranges, uint64_t seed, const double* gsnorm, double* part, double* dots,
                  unsigned int* ticket) {
  if (st->done || gsnorm[0] >= 1e-10) {
    if (blockIdx.x == 0 && threadIdx.x == 0) st->refill = 0;
    return;
  }
  if (ni >= maxsize) {  // nothing left to add: the loop ends with the current Ritz vector
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      st->refill = 0;
      st->done = 1;
      st->final_ii = ii;
      st->fail_ii = ii;
    }
    return;
  }
  double acc[TT_DAV_MAX];
  for (int j = 0; j < ni; ++j) acc[j] = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)RF_THREADS + threadIdx.x; i < n; i += (int64_t)gridDim.x * RF_THREADS) {
    int lo = 0, hi = nranges;  // is i inside one of the sorted [begin, end) ranges?
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (ranges[2 * mid + 1] <= i) lo = mid + 1; else hi = mid;
    }
    double v = 0.0;
    if (lo < nranges && ranges[2 * lo] <= i)
      v = (double)(rf_mix(seed ^ (uint64_t)i * 0xD1B54A32D192ED03ull) >> 11) * 0x1.0p-53;
    y[i] = v;
    for (int j = 0; j < ni; ++j) acc[j] = fma(xs.p[j][i], v, acc[j]);
  }
  __shared__ double red[RF_THREADS / 32][TT_DAV_MAX];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int j = 0; j < ni; ++j) {
    double x = acc[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) red[w][j] = x;
  }
  __syncthreads();
  if (threadIdx.x < ni) {
    double x = 0.0;
    for (int k = 0; k < RF_THREADS / 32; ++k) x += red[k][threadIdx.x];
    part[(int64_t)threadIdx.x * gridDim.x + blockIdx.x] = x;
  }
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (threadIdx.x < ni) {
    double x = 0.0;
    for (int b = 0; b < (int)gridDim.x; ++b) x += __ldcg(part + (int64_t)threadIdx.x * gridDim.x + b);
    dots[threadIdx.x] = x;
  }
  if (threadIdx.x == 0) {
    st->refill = 1;
    st->randomized++;
    *ticket = 0u;
  }
}

}  // namespace

extern "C" {

int tt_dav_state_create(tt_ctx* ctx, tt_dav_state** out) {
  TT_REQUIRE(ctx && out, "tt_dav_state_create: null argument");
  tt_dav_state* s = nullptr;
  TT_CUDA(cudaMalloc(&s, sizeof(tt_dav_state)));
  TT_CUDA(cudaMemsetAsync(s, 0, sizeof(tt_dav_state), ctx->stream));
  *out = s;
  return TT_OK;
}

int tt_dav_state_destroy(tt_ctx* ctx, tt_dav_state* st) {
  (void)ctx;
  if (st) cudaFree(st);
  return TT_OK;
}

int tt_dav_coefficients(tt_dav_state* st, double** coef_x, double** coef_q) {
  TT_REQUIRE(st && coef_x && coef_q, "tt_dav_coefficients: null argument");
  *coef_x = st->coef_x;
  *coef_q = st->coef_q;
  return TT_OK;
}

int tt_dav_begin(tt_ctx* ctx, tt_dav_state* st, const double* d_init_energy) {
  TT_REQUIRE(ctx && st && d_init_energy, "tt_dav_begin: null argument");
  dav_begin_kernel<<<1, 32, 0, ctx->stream>>>(st, d_init_energy);
  TT_LAUNCH_CHECK(ctx);
  return TT_OK;
}

int tt_dav_ritz(tt_ctx* ctx, tt_dav_state* st, int ii) {
  TT_REQUIRE(ctx && st && ii >= 1 && ii + 1 < TT_DAV_MAX, "tt_dav_ritz: bad argument");
  dav_ritz_kernel<<<1, 32, 0, ctx->stream>>>(st, ii);
  TT_LAUNCH_CHECK(ctx);
  return TT_OK;
}

int tt_dav_converged(tt_ctx* ctx, tt_dav_state* st, int ii, int maxiter, double tol, const double* d_qnorm) {
  TT_REQUIRE(ctx && st && d_qnorm && ii >= 0 && maxiter + 1 < TT_DAV_MAX, "tt_dav_converged: bad argument");
  dav_conv_kernel<<<1, 32, 0, ctx->stream>>>(st, ii, maxiter, tol, d_qnorm);
  TT_LAUNCH_CHECK(ctx);
  return TT_OK;
}

int tt_dav_add_row(tt_ctx* ctx, tt_dav_state* st, int ii, const double* d_row, const double* d_gsnorm) {
  TT_REQUIRE(ctx && st && d_row && d_gsnorm && ii >= 0 && ii + 2 < TT_DAV_MAX, "tt_dav_add_row: bad argument");
  dav_row_kernel<<<1, 32, 0, ctx->stream>>>(st, ii, d_row, d_gsnorm);
  TT_LAUNCH_CHECK(ctx);
  return TT_OK;
}

int tt_dav_gs_refill(tt_ctx* ctx, tt_dav_state* st, int ii, int ni, int maxsize, int64_t n,
                     const double* const* xs, double* y, int nranges, const int64_t* d_ranges, uint64_t seed,
                     const double* d_gsnorm, double* d_dots) {
  TT_REQUIRE(ctx && st && xs && y && d_gsnorm && d_dots && (nranges == 0 || d_ranges),
             "tt_dav_gs_refill: null argument");
  TT_REQUIRE(ni >= 1 && ni <= TT_DAV_MAX && ii >= 0 && n >= 0, "tt_dav_gs_refill: bad argument");
  RefillVecs v;
  for (int j = 0; j < ni; ++j) v.p[j] = xs[j];
  const int nb = (int)std::max<int64_t>(1, std::min<int64_t>((n + RF_THREADS - 1) / RF_THREADS,
                                                                  4 * (int64_t)ctx->num_sms));
  double* part = tt::partials(ctx, nb * ni);
  if (!part) return tt::fail(TT_ERR_OOM, "tt_dav_gs_refill: reduction scratch");
  dav_refill_kernel<<<nb, RF_THREADS, 0, ctx->stream>>>(st, ii, ni, maxsize, n, v, y, nranges, d_ranges, seed,
                                                        d_gsnorm, part, d_dots, ctx->d_ticket);
  TT_LAUNCH_CHECK(ctx);
  return TT_OK;
}

int tt_dav_refill_flag(tt_dav_state* st, const int** d_flag) {
  TT_REQUIRE(st && d_flag, "tt_dav_refill_flag: null argument");
  *d_flag = &st->refill;
  return TT_OK;
}

int tt_dav_read(tt_ctx* ctx, const tt_dav_state* st, tt_dav_result* out) {
  TT_REQUIRE(ctx && st && out, "tt_dav_read: null argument");
  // one synchronising read of the header: the flags and the Ritz value
  constexpr size_t kHead = offsetof(tt_dav_state, lambda) + sizeof(double);
  alignas(8) unsigned char h[kHead];
  int rc = tt_memcpy_d2h(ctx, h, st, kHead);
  if (rc != TT_OK) return rc;
  tt_dav_state head;
  std::memcpy(&head, h, kHead);
  out->done = head.done;
  out->final_ii = head.final_ii;
  out->fail_ii = head.fail_ii;
  out->iters = head.iters;
  out->randomized = head.randomized;
  out->lambda = head.lambda;
  return TT_OK;
}

}  // extern "C"
