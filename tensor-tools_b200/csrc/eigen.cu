// Batched symmetric eigensolver for the per-QN-sector density matrices of the
// block SVD (qtensor/qtensor_op.cpp:1229-1300), and the strided copy kernel
// that scatters sector matrices into U/V blocks (:1389-1436).
//
// Method: parallel cyclic two-sided Jacobi (Golub & Van Loan, "Matrix
// Computations", sec. 8.5: symmetric Schur 2x2 rotation, round-robin
// ordering of disjoint pairs).  One CTA per problem; every round rotates all
// n/2 disjoint pairs at once as independent 2x2 block updates
// A <- R_a^T A R_b, Z <- Z R_b.  The matrix and the eigenvectors sit in
// shared memory when n <= 104, otherwise in global memory (L2).
// Sweeps stop when the off-diagonal Frobenius norm falls below
// 1e-15 * ||A||_F (or after MAX_SWEEPS, reported as TT_ERR_NOCONV).
#include <cmath>
#include <vector>

#include "tt_internal.h"

namespace {

constexpr int ET = 512;          // threads per eigen CTA
constexpr int MAX_SWEEPS = 40;
constexpr int SMEM_N = 104;      // A and Z in shared memory: 2*104*104*8 B = 169 KB
constexpr int MAX_N = 2048;      // rotation tables in static shared memory: 33 KB

struct EigDev {
  int64_t g_off, w_off, a_off;
  int32_t n, flags;
};

__device__ double block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += red[i];
    red[32] = s;
  }
  __syncthreads();
  return red[32];
}

__global__ void __launch_bounds__(ET)
jacobi_eig(const EigDev* __restrict__ probs, double* G, double* Zg, double* W,
           const double* Amat, int* status) {
  extern __shared__ double sm[];
  __shared__ double red[33];
  __shared__ int perm[MAX_N + 2];
  __shared__ int pidx[MAX_N / 2 + 1], qidx[MAX_N / 2 + 1];
  __shared__ double cs[MAX_N / 2 + 1], sn[MAX_N / 2 + 1];

  const EigDev P = probs[blockIdx.x];
  const int n = P.n;
  double* Gp = G + P.g_off;
  double* Zp = Zg + P.g_off;
  double* Wp = W + P.w_off;
  const int tid = threadIdx.x;

  if (P.flags & TT_EIG_ROW_1X2) {
    if (tid == 0) {
      double a = Amat[P.a_off], b = Amat[P.a_off + 1];
      double d = sqrt(a * a + b * b);
      double z0, z1;
      if (d != 0.0) {
        double inv = 1.0 / d;
        z0 = a * inv;
        z1 = b * inv;
      } else {
        z0 = z1 = 1.0 / sqrt(2.0);
      }
      Wp[0] = d * d;
      Wp[1] = 0.0;
      Zp[0] = z0;
      Zp[1] = z1;
      Zp[2] = -z1;
      Zp[3] = z0;
    }
    return;
  }
  if (n <= 0) return;
  const bool in_smem = n <= SMEM_N;
  double* A = in_smem ? sm : Gp;
  double* Z = in_smem ? sm + SMEM_N * SMEM_N : Zp;
  const int lda = in_smem ? SMEM_N : n;
  for (int e = tid; e < n * n; e += blockDim.x) {
    int i = e % n, j = e / n;
    if (in_smem) A[i + lda * j] = Gp[e];
    Z[i + lda * j] = (i == j) ? 1.0 : 0.0;
  }
  const int m = n + (n & 1);  // even number of slots; slot n is a dummy when n is odd
  const int half = m / 2;
  for (int i = tid; i < m; i += blockDim.x) perm[i] = i;
  __syncthreads();

  // ||A||_F for the stopping rule
  double loc = 0.0;
  for (int e = tid; e < n * n; e += blockDim.x) {
    double v = A[(e % n) + lda * (e / n)];
    loc += v * v;
  }
  const double fro2 = block_sum(loc, red);
  const double tol2 = fro2 * 1e-30;
  __syncthreads();

  int sweep = 0;
  for (; sweep < MAX_SWEEPS; ++sweep) {
    // off-diagonal norm
    loc = 0.0;
    for (int e = tid; e < n * n; e += blockDim.x) {
      int i = e % n, j = e / n;
      if (i != j) {
        double v = A[i + lda * j];
        loc += v * v;
      }
    }
    double off = block_sum(loc, red);
    if (off <= tol2 || fro2 == 0.0) break;
    for (int round = 0; round < m - 1; ++round) {
      // rotations of this round
      for (int t = tid; t < half; t += blockDim.x) {
        int p = perm[t], q = perm[m - 1 - t];
        if (p > q) { int x = p; p = q; q = x; }
        double c = 1.0, s = 0.0;
        if (q < n) {
          double apq = A[p + lda * q];
          if (apq != 0.0) {
            double app = A[p + lda * p], aqq = A[q + lda * q];
            double tau = (aqq - app) / (2.0 * apq);
            double tt = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            c = 1.0 / sqrt(1.0 + tt * tt);
            s = tt * c;
          }
        }
        pidx[t] = p;
        qidx[t] = q;
        cs[t] = c;
        sn[t] = s;
      }
      __syncthreads();
      // A <- R_a^T A R_b on all 2x2 blocks (a, b)
      for (int e = tid; e < half * half; e += blockDim.x) {
        int a = e % half, b = e / half;
        int pa = pidx[a], qa = qidx[a], pb = pidx[b], qb = qidx[b];
        double ca = cs[a], sa = sn[a], cb = cs[b], sb = sn[b];
        bool qa_ok = qa < n, qb_ok = qb < n;
        double x00 = A[pa + lda * pb];
        double x01 = qb_ok ? A[pa + lda * qb] : 0.0;
        double x10 = qa_ok ? A[qa + lda * pb] : 0.0;
        double x11 = (qa_ok && qb_ok) ? A[qa + lda * qb] : 0.0;
        double y00 = cb * x00 - sb * x01, y01 = sb * x00 + cb * x01;
        double y10 = cb * x10 - sb * x11, y11 = sb * x10 + cb * x11;
        double z00 = ca * y00 - sa * y10, z01 = ca * y01 - sa * y11;
        double z10 = sa * y00 + ca * y10, z11 = sa * y01 + ca * y11;
        if (a == b) { z01 = 0.0; z10 = 0.0; }
        A[pa + lda * pb] = z00;
        if (qb_ok) A[pa + lda * qb] = z01;
        if (qa_ok) A[qa + lda * pb] = z10;
        if (qa_ok && qb_ok) A[qa + lda * qb] = z11;
      }
      // Z <- Z R_b
      for (int e = tid; e < n * half; e += blockDim.x) {
        int i = e % n, b = e / n;
        int pb = pidx[b], qb = qidx[b];
        if (qb >= n) continue;
        double cb = cs[b], sb = sn[b];
        double z0 = Z[i + lda * pb], z1 = Z[i + lda * qb];
        Z[i + lda * pb] = cb * z0 - sb * z1;
        Z[i + lda * qb] = sb * z0 + cb * z1;
      }
      __syncthreads();
      // round-robin: slot 0 fixed, slots 1..m-1 rotate
      if (tid == 0) {
        int last = perm[m - 1];
        for (int i = m - 1; i > 1; --i) perm[i] = perm[i - 1];
        perm[1] = last;
      }
      __syncthreads();
    }
  }
  if (sweep == MAX_SWEEPS && tid == 0) atomicExch(status, 1);
  __syncthreads();
  // sort eigenpairs descending (ties by index); stage the sorted vectors in G
  for (int i = tid; i < n; i += blockDim.x) {
    double li = A[i + lda * i];
    int rank = 0;
    for (int j = 0; j < n; ++j) {
      double lj = A[j + lda * j];
      rank += (lj > li) || (lj == li && j < i);
    }
    Wp[rank] = li;
    perm[i] = rank;
  }
  __syncthreads();
  if (in_smem) {
    for (int e = tid; e < n * n; e += blockDim.x) {
      int i = e % n, j = e / n;
      Zp[i + n * perm[j]] = Z[i + lda * j];
    }
  } else {
    for (int e = tid; e < n * n; e += blockDim.x) {
      int i = e % n, j = e / n;
      Gp[i + n * perm[j]] = Z[i + lda * j];
    }
    __syncthreads();
    for (int e = tid; e < n * n; e += blockDim.x) Zp[e] = Gp[e];
  }
}

__global__ void strided_copy(const tt_copy_desc* __restrict__ d, const double* __restrict__ src,
                             double* __restrict__ dst) {
  const tt_copy_desc D = d[blockIdx.y];
  int64_t total = 1;
  for (int i = 0; i < D.n_modes; ++i) total *= D.dims[i];
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = e, so = D.src_off, dof = D.dst_off;
    for (int i = 0; i < D.n_modes; ++i) {
      int64_t q = r / D.dims[i];
      int64_t j = r - q * D.dims[i];
      so += j * D.src_stride[i];
      dof += j * D.dst_stride[i];
      r = q;
    }
    dst[dof] = src[so];
  }
}

}  // namespace

extern "C" {

int tt_sym_eig_batched(tt_ctx* ctx, const tt_eig_problem* probs, int n_probs, double* G,
                       double* Z, double* w, const double* A) {
  TT_REQUIRE(ctx && (n_probs == 0 || (probs && G && Z && w)), "tt_sym_eig_batched: null argument");
  if (n_probs == 0) return TT_OK;
  std::vector<EigDev> hp(n_probs);
  for (int i = 0; i < n_probs; ++i) {
    TT_REQUIRE(probs[i].n >= 0 && probs[i].n <= MAX_N, "tt_sym_eig_batched: size out of range");
    if (probs[i].flags & TT_EIG_ROW_1X2)
      TT_REQUIRE(probs[i].n == 2 && A != nullptr, "tt_sym_eig_batched: 1x2 case needs n == 2 and A");
    hp[i] = EigDev{probs[i].g_off, probs[i].w_off, probs[i].a_off, probs[i].n, probs[i].flags};
  }
  EigDev* dp = tt::pool_alloc<EigDev>(ctx, n_probs);
  int* dstatus = tt::pool_alloc<int>(ctx, 1);
  if (!dp || !dstatus) return tt::fail(TT_ERR_OOM, "tt_sym_eig_batched: allocation failed");
  TT_CUDA(cudaMemcpyAsync(dp, hp.data(), sizeof(EigDev) * n_probs, cudaMemcpyHostToDevice, ctx->stream));
  TT_CUDA(cudaMemsetAsync(dstatus, 0, sizeof(int), ctx->stream));
  const size_t smem = sizeof(double) * 2 * SMEM_N * SMEM_N;
  static thread_local uint64_t attr = 0;  // per host thread and device
  if (tt::first_on_device(attr, ctx->device))
    TT_CUDA(cudaFuncSetAttribute(jacobi_eig, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  jacobi_eig<<<n_probs, ET, smem, ctx->stream>>>(dp, G, Z, w, A, dstatus);
  TT_LAUNCH_CHECK(ctx);
  int hstatus = 0;
  TT_CUDA(cudaMemcpyAsync(&hstatus, dstatus, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  TT_CUDA(cudaStreamSynchronize(ctx->stream));
  tt::pool_free(ctx, dp);
  tt::pool_free(ctx, dstatus);
  if (hstatus) return tt::fail(TT_ERR_NOCONV, "tt_sym_eig_batched: Jacobi sweep limit reached");
  return TT_OK;
}

int tt_strided_copy_batched(tt_ctx* ctx, const tt_copy_desc* descs, int n, const double* src,
                            double* dst) {
  TT_REQUIRE(ctx && (n == 0 || (descs && src && dst)), "tt_strided_copy_batched: null argument");
  if (n == 0) return TT_OK;
  int64_t maxe = 1;
  for (int i = 0; i < n; ++i) {
    TT_REQUIRE(descs[i].n_modes >= 0 && descs[i].n_modes <= TT_MAX_MODES, "tt_strided_copy_batched: modes");
    int64_t t = 1;
    for (int j = 0; j < descs[i].n_modes; ++j) t *= descs[i].dims[j];
    if (t > maxe) maxe = t;
  }
  TT_REQUIRE(n <= 65535, "tt_strided_copy_batched: too many descriptors");
  tt_copy_desc* dd = tt::pool_alloc<tt_copy_desc>(ctx, n);
  if (!dd) return tt::fail(TT_ERR_OOM, "tt_strided_copy_batched: allocation failed");
  TT_CUDA(tt::h2d_async(ctx, dd, descs, sizeof(tt_copy_desc) * n));  // staged: descs may be reused
  int gx = (int)((maxe + 255) / 256);
  if (gx > 64) gx = 64;
  dim3 grid(gx, n);
  strided_copy<<<grid, 256, 0, ctx->stream>>>(dd, src, dst);
  TT_LAUNCH_CHECK(ctx);
  tt::pool_free(ctx, dd);
  return TT_OK;
}

}  // extern "C"
