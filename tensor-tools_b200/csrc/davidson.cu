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
#include <cmath>
#include <cstddef>
#include <cstring>

#include "tt_internal.h"

struct tt_dav_state {
  int done;      // 1 once the loop has ended
  int final_ii;  // iteration at which it ended (-2: Gram-Schmidt failure at fail_ii)
  int fail_ii;
  int iters;
  int cur;       // which of buf[0], buf[1] holds M (the other holds Mnext)
  double lambda, last_lambda, qnorm, gsnorm;
  double buf[2][TT_DAV_MAX * TT_DAV_MAX];
  double evals[TT_DAV_MAX];
  double coef_x[TT_DAV_MAX];      // Ritz vector:   x = sum_k coef_x[k] v[k]
  double coef_q[TT_DAV_MAX + 1];  // residual:      q = sum_k coef_q[k] va[k] + coef_q[ii+1] x
};

namespace {

// DIAG (linalg/lapack_wrapper.cpp:40-54, dsyev semantics): cyclic Jacobi on
// the n x n column-major A (overwritten), eigenvalues ascending in ev,
// eigenvectors in the columns of M.  Same rotation order and stopping rule as
// the host DIAG.
__device__ void dav_diag(int n, double* M, double* ev) {
  // working copies in shared memory (local arrays would live in slow local memory)
  __shared__ double A[TT_DAV_MAX * TT_DAV_MAX], V[TT_DAV_MAX * TT_DAV_MAX];
  for (int i = 0; i < n * n; ++i) {
    A[i] = M[i];
    V[i] = 0.0;
  }
  for (int i = 0; i < n; ++i) V[i + n * i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, fro = 0.0;
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        fro += A[i + n * j] * A[i + n * j];
        if (i != j) off += A[i + n * j] * A[i + n * j];
      }
    if (off <= 1e-32 * fro || off == 0.0) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = A[p + n * q];
        if (apq == 0.0) continue;
        const double tau = (A[q + n * q] - A[p + n * p]) / (2.0 * apq);
        const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
        const double c = 1.0 / sqrt(1.0 + t * t), s = t * c;
        for (int k = 0; k < n; ++k) {
          const double akp = A[k + n * p], akq = A[k + n * q];
          A[k + n * p] = c * akp - s * akq;
          A[k + n * q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          const double apk = A[p + n * k], aqk = A[q + n * k];
          A[p + n * k] = c * apk - s * aqk;
          A[q + n * k] = s * apk + c * aqk;
        }
        A[p + n * q] = A[q + n * p] = 0.0;
        for (int k = 0; k < n; ++k) {
          const double vkp = V[k + n * p], vkq = V[k + n * q];
          V[k + n * p] = c * vkp - s * vkq;
          V[k + n * q] = s * vkp + c * vkq;
        }
      }
  }
  int order[TT_DAV_MAX];
  for (int i = 0; i < n; ++i) order[i] = i;
  for (int i = 1; i < n; ++i) {  // stable insertion sort by eigenvalue
    const int o = order[i];
    int j = i - 1;
    while (j >= 0 && A[order[j] + n * order[j]] > A[o + n * o]) {
      order[j + 1] = order[j];
      --j;
    }
    order[j + 1] = o;
  }
  for (int j = 0; j < n; ++j) {
    ev[j] = A[order[j] + n * order[j]];
    for (int i = 0; i < n; ++i) M[i + n * j] = V[i + n * order[j]];
  }
}

__global__ void dav_begin_kernel(tt_dav_state* st, const double* init_en) {
  if (threadIdx.x != 0) return;
  st->done = 0;
  st->final_ii = -1;
  st->fail_ii = -1;
  st->iters = 0;
  st->cur = 0;
  st->last_lambda = 1000.0;
  const double lam = init_en[0];
  st->lambda = lam;
  st->buf[0][0] = lam;  // M[0] = Mnext[0] = lambda
  st->buf[1][0] = lam;
  st->coef_q[0] = 1.0;  // q = va[0] - lambda v[0]
  st->coef_q[1] = -lam;
}

__global__ void dav_ritz_kernel(tt_dav_state* st, int ii) {
  if (threadIdx.x != 0 || st->done) return;
  const int ni = ii + 1;
  double* M = st->buf[st->cur];
  double* Mn = st->buf[1 - st->cur];
  for (int mi = 0; mi < ni; ++mi)
    for (int mj = 0; mj <= mi; ++mj) {
      Mn[mj + mi * (ni + 1)] = M[mj + mi * ni];
      Mn[mi + mj * (ni + 1)] = M[mi + mj * ni];
    }
  dav_diag(ni, M, st->evals);
  const double lam = st->evals[0];
  st->lambda = lam;
  const double sgn = (M[0] < 0.0) ? -1.0 : 1.0;  // sign stabilisation (:265-268)
  for (int k = 0; k <= ii; ++k) {
    st->coef_x[k] = sgn * M[k];
    st->coef_q[k] = sgn * M[k];
  }
  st->coef_q[ii + 1] = -lam;
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
  if (!(g >= 1e-10)) {  // Gram-Schmidt failure: the host finishes with its own loop
    st->done = 1;
    st->final_ii = -2;
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
  out->lambda = head.lambda;
  return TT_OK;
}

}  // extern "C"
