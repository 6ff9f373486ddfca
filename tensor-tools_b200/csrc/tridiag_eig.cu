// Two-phase symmetric eigensolver for the per-QN-sector density matrices of
// the block SVD (qtensor/qtensor_op.cpp:1229-1300): all eigenvalues first (so
// the host can apply the truncation rule of :1290-1300), then eigenvectors
// only for the states that are kept.
//
// Phase 1 (tt_sym_eigvals_batched), one CTA per sector:
//   Householder reduction to tridiagonal form T = Q^T G Q (Golub & Van Loan,
//   "Matrix Computations", 4th ed., alg. 8.3.1), reflectors kept below the
//   subdiagonal of G; then every eigenvalue of T by bisection on Sturm
//   sequence counts (ibid. sec. 8.4.1), one thread per eigenvalue.
// Phase 2 (tt_sym_eigvecs_batched), one CTA per sector:
//   inverse iteration on T - lambda I (tridiagonal LU with partial pivoting,
//   tiny pivots replaced by eps*||T||), one thread per wanted eigenvector;
//   classical Gram-Schmidt applied twice inside clusters of close eigenvalues
//   (gap <= 1e-3 ||T||, the clustering rule of LAPACK's inverse iteration);
//   back-transformation z = Q y with the stored reflectors.
// The matrix sits in shared memory when n <= 160, otherwise in global memory.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

#include "tt_internal.h"

namespace {

constexpr int TT = 512;          // threads per CTA
constexpr int SM_N = 160;        // full n x n FP64 matrix in shared memory up to this size
constexpr int MAX_N = 2048;
constexpr int INV_ITERS = 3;

struct EigDev {
  int64_t g_off, w_off, a_off;
  int32_t n, flags, nvec, pad;
};

__device__ double block_reduce(double v, double* red, bool is_max) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    double u = __shfl_down_sync(0xffffffffu, v, o);
    v = is_max ? fmax(v, u) : v + u;
  }
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = red[0];
    for (int i = 1; i < (int)(blockDim.x >> 5); ++i) s = is_max ? fmax(s, red[i]) : s + red[i];
    red[32] = s;
  }
  __syncthreads();
  return red[32];
}

// number of eigenvalues of T (diag d, squared offdiag e2) that are < x
__device__ int sturm_count(const double* d, const double* e2, int n, double x, double pivmin) {
  double q = d[0] - x;
  if (fabs(q) <= pivmin) q = -pivmin;
  int c = q <= 0.0;
  for (int i = 1; i < n; ++i) {
    q = d[i] - x - e2[i - 1] / q;
    if (fabs(q) <= pivmin) q = -pivmin;
    c += q <= 0.0;
  }
  return c;
}

__global__ void __launch_bounds__(TT)
tridiag_eigvals(const EigDev* __restrict__ probs, double* G, double* Tg, double* W, const double* Amat) {
  extern __shared__ double sm[];
  __shared__ double red[33];
  __shared__ double s_beta, s_tau, s_scale;
  const EigDev P = probs[blockIdx.x];
  const int n = P.n;
  const int tid = threadIdx.x;
  double* Wp = W + P.w_off;
  double* dg = Tg + 3 * P.w_off;  // d[n], e[n], tau[n]
  double* eg = dg + n;
  double* tg = eg + n;
  if (n <= 0) return;
  if (P.flags & TT_EIG_ROW_1X2) {
    if (tid == 0) {
      double a = Amat[P.a_off], b = Amat[P.a_off + 1];
      Wp[0] = a * a + b * b;
      Wp[1] = 0.0;
    }
    return;
  }
  const bool in_smem = n <= SM_N;
  double* Gp = G + P.g_off;
  double* A = in_smem ? sm : Gp;
  double* v = in_smem ? sm + SM_N * SM_N : sm;
  double* p = v + n;
  double* d = p + n;    // diag
  double* e2 = d + n;   // offdiag squared
  const int lda = n;
  if (in_smem)
    for (int i = tid; i < n * n; i += blockDim.x) A[i] = Gp[i];
  __syncthreads();

  for (int k = 0; k + 2 < n; ++k) {
    const int m = n - k - 1;  // length of x = A[k+1:n, k]
    double loc = 0.0;
    for (int i = 1 + tid; i < m; i += blockDim.x) {
      double t = A[(k + 1 + i) + lda * k];
      loc += t * t;
    }
    const double sigma = block_reduce(loc, red, false);
    if (tid == 0) {
      double alpha = A[(k + 1) + lda * k];
      if (sigma == 0.0) {
        s_tau = 0.0;
        s_beta = alpha;
        s_scale = 0.0;
      } else {
        double mu = sqrt(alpha * alpha + sigma);
        double beta = alpha <= 0.0 ? mu : -mu;
        s_tau = (beta - alpha) / beta;
        s_scale = 1.0 / (alpha - beta);
        s_beta = beta;
      }
      tg[k] = s_tau;
      eg[k] = s_beta;
    }
    __syncthreads();
    const double tau = s_tau;
    if (tau == 0.0) continue;  // column already reduced
    // v = [1, x[1:] * scale]; keep v[1:] below the subdiagonal for phase 2
    for (int i = tid; i < m; i += blockDim.x) {
      double vi = (i == 0) ? 1.0 : A[(k + 1 + i) + lda * k] * s_scale;
      v[i] = vi;
      if (i > 0) A[(k + 1 + i) + lda * k] = vi;
    }
    __syncthreads();
    // p = tau * A22 v, one warp per row (A22 symmetric: read the column)
    const int warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
    for (int r = warp; r < m; r += nw) {
      const double* col = A + (k + 1) + lda * (k + 1 + r);
      double s = 0.0;
      for (int c = lane; c < m; c += 32) s += col[c] * v[c];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
      if (lane == 0) p[r] = tau * s;
    }
    __syncthreads();
    loc = 0.0;
    for (int i = tid; i < m; i += blockDim.x) loc += v[i] * p[i];
    const double K = 0.5 * tau * block_reduce(loc, red, false);
    for (int i = tid; i < m; i += blockDim.x) p[i] -= K * v[i];  // w
    __syncthreads();
    // A22 -= v w^T + w v^T
    for (int e = tid; e < m * m; e += blockDim.x) {
      int r = e % m, c = e / m;
      A[(k + 1 + r) + lda * (k + 1 + c)] -= v[r] * p[c] + p[r] * v[c];
    }
    __syncthreads();
  }
  // T: diagonal, offdiagonal (the last one is A[n-1,n-2])
  for (int i = tid; i < n; i += blockDim.x) {
    double di = A[i + lda * i];
    d[i] = di;
    dg[i] = di;
  }
  if (tid == 0) {
    if (n >= 2) eg[n - 2] = A[(n - 1) + lda * (n - 2)];
    eg[n - 1] = 0.0;
    tg[n - 1] = 0.0;
    if (n >= 2) tg[n - 2] = 0.0;
  }
  __syncthreads();
  for (int i = tid; i < n - 1; i += blockDim.x) e2[i] = eg[i] * eg[i];
  if (in_smem) {  // phase 2 reads the reflectors from G
    for (int i = tid; i < n * n; i += blockDim.x) Gp[i] = A[i];
  }
  __syncthreads();
  // Gershgorin bounds and the pivot floor of the Sturm recurrence
  double lo_loc = DBL_MAX, hi_loc = -DBL_MAX, e2max = 0.0;
  for (int i = tid; i < n; i += blockDim.x) {
    double r = (i > 0 ? fabs(eg[i - 1]) : 0.0) + (i < n - 1 ? fabs(eg[i]) : 0.0);
    lo_loc = fmin(lo_loc, d[i] - r);
    hi_loc = fmax(hi_loc, d[i] + r);
    if (i < n - 1) e2max = fmax(e2max, e2[i]);
  }
  const double gu = block_reduce(hi_loc, red, true);
  const double gl = -block_reduce(-lo_loc, red, true);
  const double emax = block_reduce(e2max, red, true);
  const double bnorm = fmax(fabs(gl), fabs(gu));
  const double pivmin = DBL_MIN * fmax(1.0, emax);
  const double atol = 4.0 * DBL_EPSILON * bnorm + 2.0 * pivmin;
  if (bnorm == 0.0) {  // T == 0: every eigenvalue is exactly zero
    for (int j = tid; j < n; j += blockDim.x) Wp[j] = 0.0;
    return;
  }
  // Bisection for the j-th smallest eigenvalue, two levels per round: three
  // lanes of a group evaluate the Sturm count at the midpoint and at the
  // midpoints of both halves, so a round takes the same two steps (same
  // points, same tests) as two rounds of plain bisection.
  auto open_interval = [&](double lo, double hi) {
    return hi - lo > fmax(atol, 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)));
  };
  const int lane = tid & 31, wid = tid >> 5, nwarp = blockDim.x >> 5;
  const int grp = lane < 30 ? lane / 3 : 0, sub = lane % 3;
  for (int base = wid * 10; base < n; base += nwarp * 10) {
    const int j = base + grp;
    const bool active = lane < 30 && j < n;
    double lo = gl - atol, hi = gu + atol;
    int it = 0;
    bool work = active && open_interval(lo, hi);
    while (__any_sync(0xffffffffu, work)) {
      const double mid = 0.5 * (lo + hi), lm = 0.5 * (lo + mid), rm = 0.5 * (mid + hi);
      const double x = sub == 0 ? mid : (sub == 1 ? lm : rm);
      const int c = work ? sturm_count(d, e2, n, x, pivmin) : 0;
      const int cm = __shfl_sync(0xffffffffu, c, 3 * grp);
      const int cl = __shfl_sync(0xffffffffu, c, 3 * grp + 1);
      const int cr = __shfl_sync(0xffffffffu, c, 3 * grp + 2);
      if (work) {
        const bool left = cm > j;
        if (left) hi = mid; else lo = mid;
        ++it;
        if (it < 128 && open_interval(lo, hi)) {
          const double x2 = left ? lm : rm;
          if ((left ? cl : cr) > j) hi = x2; else lo = x2;
          ++it;
        }
        work = it < 128 && open_interval(lo, hi);
      }
    }
    if (active && sub == 0) Wp[n - 1 - j] = 0.5 * (lo + hi);  // descending order
  }
}

// solve (T - lambda I) y = b in place (y holds b on entry); U holds 3n scratch
__device__ void tri_solve(const double* d, const double* e, int n, double lambda, double tiny, double* y,
                          double* U, int ystride) {
  double* u0 = U;
  double* u1 = U + n;
  double* u2 = U + 2 * n;
  // forward elimination with partial pivoting, transforming b on the fly
  double di = d[0] - lambda, si = n > 1 ? e[0] : 0.0, ti = 0.0;
  double bi = y[0];
  for (int i = 0; i + 1 < n; ++i) {
    double ci = e[i];
    double an = d[i + 1] - lambda;
    double bn = (i + 2 < n) ? e[i + 1] : 0.0;
    double bnext = y[(int64_t)(i + 1) * ystride];
    if (fabs(di) >= fabs(ci)) {
      if (di == 0.0) di = tiny;
      double mlt = ci / di;
      u0[i] = di;
      u1[i] = si;
      u2[i] = ti;
      y[(int64_t)i * ystride] = bi;
      bi = bnext - mlt * bi;
      double nd = an - mlt * si, ns = bn - mlt * ti;
      di = nd;
      si = ns;
      ti = 0.0;
    } else {
      double mlt = di / ci;
      u0[i] = ci;
      u1[i] = an;
      u2[i] = bn;
      y[(int64_t)i * ystride] = bnext;
      bi = bi - mlt * bnext;
      double nd = si - mlt * an, ns = ti - mlt * bn;
      di = nd;
      si = ns;
      ti = 0.0;
    }
  }
  if (fabs(di) < tiny) di = di < 0.0 ? -tiny : tiny;
  u0[n - 1] = di;
  y[(int64_t)(n - 1) * ystride] = bi;
  // back substitution
  for (int i = n - 1; i >= 0; --i) {
    double s = y[(int64_t)i * ystride];
    if (i + 1 < n) s -= u1[i] * y[(int64_t)(i + 1) * ystride];
    if (i + 2 < n) s -= u2[i] * y[(int64_t)(i + 2) * ystride];
    double piv = u0[i];
    if (fabs(piv) < tiny) piv = piv < 0.0 ? -tiny : tiny;
    y[(int64_t)i * ystride] = s / piv;
  }
}

__device__ __forceinline__ double hash_unit(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (double)(z >> 11) * 0x1.0p-53 * 2.0 - 1.0;
}

__global__ void __launch_bounds__(TT)
tridiag_eigvecs(const EigDev* __restrict__ probs, const double* G, const double* Tg, const double* W, double* Zg,
                double* work, const double* Amat, int smem_cap) {
  extern __shared__ double zsm[];  // n*nvec eigenvector block + n reflector, when they fit
  __shared__ double red[33];
  __shared__ double coef[MAX_N / 2];
  __shared__ int cstart[MAX_N / 2];
  const EigDev P = probs[blockIdx.x];
  const int n = P.n, nvec = P.nvec;
  const int tid = threadIdx.x;
  if (n <= 0 || nvec <= 0) return;
  double* Zout = Zg + P.g_off;  // n x nvec, leading dimension n
  // the iterations run on a shared-memory copy when it fits
  const bool in_smem = (int64_t)n * nvec + n <= (int64_t)smem_cap;
  double* Z = in_smem ? zsm : Zout;
  double* vk = in_smem ? zsm + (int64_t)n * nvec : nullptr;
  if (P.flags & TT_EIG_ROW_1X2) {
    Z = Zout;
    if (tid == 0) {
      double a = Amat[P.a_off], b = Amat[P.a_off + 1];
      double dd = sqrt(a * a + b * b), z0, z1;
      if (dd != 0.0) {
        double inv = 1.0 / dd;
        z0 = a * inv;
        z1 = b * inv;
      } else {
        z0 = z1 = 1.0 / sqrt(2.0);
      }
      Z[0] = z0;
      Z[1] = z1;
      if (nvec > 1) {
        Z[2] = -z1;
        Z[3] = z0;
      }
    }
    return;
  }
  const double* d = Tg + 3 * P.w_off;
  const double* e = d + n;
  const double* tau = e + n;
  const double* lam = W + P.w_off;  // descending
  const double* Gp = G + P.g_off;
  // 3n scratch per eigenvector (3 n*n per problem in global memory), in shared
  // memory after the eigenvectors and the reflector when it fits
  const bool u_smem = in_smem && 4 * (int64_t)n * nvec + n <= (int64_t)smem_cap;
  double* U = u_smem ? zsm + (int64_t)n * nvec + n : work + 3 * P.g_off;
  // ||T||_1 for the pivot floor and the cluster tolerance
  double loc = 0.0;
  for (int i = tid; i < n; i += blockDim.x)
    loc = fmax(loc, fabs(d[i]) + (i > 0 ? fabs(e[i - 1]) : 0.0) + (i + 1 < n ? fabs(e[i]) : 0.0));
  const double tnorm = block_reduce(loc, red, true);
  // pivot floor; a (numerically) zero T takes 1 so that b / tiny cannot overflow
  const double tiny = tnorm > 1e-250 ? fmax(DBL_EPSILON * tnorm, DBL_MIN) : 1.0;
  const double ortol = 1e-3 * tnorm;
  // (a) inverse iteration, one thread per eigenvector
  for (int j = tid; j < nvec; j += blockDim.x) {
    double* y = Z + (int64_t)n * j;
    for (int i = 0; i < n; ++i) y[i] = hash_unit(((uint64_t)P.g_off << 20) ^ ((uint64_t)j << 32) ^ (uint64_t)i);
    for (int it = 0; it < INV_ITERS; ++it) {
      tri_solve(d, e, n, lam[j], tiny, y, U + (int64_t)3 * n * j, 1);
      double s = 0.0;
      for (int i = 0; i < n; ++i) s += y[i] * y[i];
      double inv = 1.0 / sqrt(s);
      for (int i = 0; i < n; ++i) y[i] *= inv;
    }
  }
  // cluster starts: j begins a new cluster when lam[j-1] - lam[j] > ortol
  if (tid == 0) {
    int c = 0;
    for (int j = 0; j < nvec; ++j) {
      if (j == 0 || lam[j - 1] - lam[j] > ortol) c = j;
      cstart[j < MAX_N / 2 ? j : MAX_N / 2 - 1] = c;
    }
  }
  __syncthreads();
  // (b) Gram-Schmidt twice against the earlier members of the cluster
  for (int j = 1; j < nvec && j < MAX_N / 2; ++j) {
    const int c0 = cstart[j];
    if (c0 == j) continue;
    double* y = Z + (int64_t)n * j;
    for (int pass = 0; pass < 6; ++pass) {
      for (int r = 0; r < 2; ++r) {
        const int nk = j - c0;
        const int warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
        for (int k = warp; k < nk; k += nw) {
          const double* yk = Z + (int64_t)n * (c0 + k);
          double s = 0.0;
          for (int i = lane; i < n; i += 32) s += yk[i] * y[i];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
          if (lane == 0) coef[k] = s;
        }
        __syncthreads();
        for (int i = tid; i < n; i += blockDim.x) {
          double s = y[i];
          for (int k = 0; k < nk; ++k) s -= coef[k] * Z[(int64_t)n * (c0 + k) + i];
          y[i] = s;
        }
        __syncthreads();
      }
      loc = 0.0;
      for (int i = tid; i < n; i += blockDim.x) loc += y[i] * y[i];
      double nrm = sqrt(block_reduce(loc, red, false));
      if (nrm > 0.5 || pass == 5) {
        double inv = nrm > 0.0 ? 1.0 / nrm : 0.0;
        for (int i = tid; i < n; i += blockDim.x) y[i] *= inv;
        __syncthreads();
        break;
      }
      // the iterate had collapsed onto earlier vectors: one more inverse
      // iteration from the orthogonal remainder, then orthogonalise again
      if (tid == 0) {
        double inv = nrm > 0.0 ? 1.0 / nrm : 1.0;
        for (int i = 0; i < n; ++i) y[i] = nrm > 0.0 ? y[i] * inv : hash_unit((uint64_t)(j * 7919 + i + pass));
        tri_solve(d, e, n, lam[j], tiny, y, U + (int64_t)3 * n * j, 1);
      }
      __syncthreads();
    }
  }
  __syncthreads();
  // (c) back-transformation z = H_0 H_1 ... H_{n-3} y, last reflector first
  for (int k = n - 3; k >= 0; --k) {
    const double tk = tau[k];
    if (tk == 0.0) continue;
    const int m = n - k - 1;
    const int warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
    const double* refl = Gp + (k + 1) + (int64_t)n * k;  // v[1:] = refl[1:], v[0] = 1
    if (vk) {
      for (int i = tid; i < m; i += blockDim.x) vk[i] = (i == 0) ? 1.0 : refl[i];
      __syncthreads();
      refl = vk;
    }
    for (int j = warp; j < nvec; j += nw) {
      const double* y = Z + (int64_t)n * j + (k + 1);
      double s = (lane == 0) ? y[0] : 0.0;  // v_0 = 1
      for (int i = 1 + lane; i < m; i += 32) s += refl[i] * y[i];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
      if (lane == 0) coef[j] = tk * s;
    }
    __syncthreads();
    for (int el = tid; el < m * nvec; el += blockDim.x) {
      int i = el % m, j = el / m;
      double vi = (i == 0) ? 1.0 : refl[i];
      Z[(int64_t)n * j + k + 1 + i] -= vi * coef[j];
    }
    __syncthreads();
  }
  // deterministic gauge: the largest-magnitude entry of each vector is positive
  for (int j = tid; j < nvec; j += blockDim.x) {
    double* y = Z + (int64_t)n * j;
    int imax = 0;
    for (int i = 1; i < n; ++i)
      if (fabs(y[i]) > fabs(y[imax])) imax = i;
    if (y[imax] < 0.0)
      for (int i = 0; i < n; ++i) y[i] = -y[i];
  }
  if (in_smem) {
    __syncthreads();
    for (int64_t i = tid; i < (int64_t)n * nvec; i += blockDim.x) Zout[i] = Z[i];
  }
}

std::vector<EigDev> to_dev(const tt_eig_problem* probs, int n_probs, const int* nvec) {
  std::vector<EigDev> hp(n_probs);
  for (int i = 0; i < n_probs; ++i)
    hp[i] = EigDev{probs[i].g_off, probs[i].w_off, probs[i].a_off, probs[i].n, probs[i].flags,
                   nvec ? nvec[i] : 0, 0};
  return hp;
}

size_t vals_smem() { return sizeof(double) * ((size_t)SM_N * SM_N + 4 * (size_t)SM_N); }
constexpr int64_t kVecsSmemCap = 25 * 1024;  // doubles (200 KB) of eigenvectors + reflector in shared memory

}  // namespace

extern "C" {

int tt_sym_eigvals_batched(tt_ctx* ctx, const tt_eig_problem* probs, int n_probs, double* G, double* T,
                           double* w, const double* A) {
  TT_REQUIRE(ctx && (n_probs == 0 || (probs && G && T && w)), "tt_sym_eigvals_batched: null argument");
  if (n_probs == 0) return TT_OK;
  for (int i = 0; i < n_probs; ++i) {
    TT_REQUIRE(probs[i].n >= 0 && probs[i].n <= MAX_N, "tt_sym_eigvals_batched: n must be 0..2048");
    if (probs[i].flags & TT_EIG_ROW_1X2)
      TT_REQUIRE(probs[i].n == 2 && A, "tt_sym_eigvals_batched: 1x2 case needs n == 2 and A");
  }
  std::vector<EigDev> hp = to_dev(probs, n_probs, nullptr);
  EigDev* dp = tt::pool_alloc<EigDev>(ctx, n_probs);
  if (!dp) return tt::fail(TT_ERR_OOM, "tt_sym_eigvals_batched: allocation failed");
  TT_CUDA(tt::h2d_async(ctx, dp, hp.data(), sizeof(EigDev) * n_probs));
  static thread_local bool attr = false;  // per host thread: each may drive its own device
  if (!attr) {
    TT_CUDA(cudaFuncSetAttribute(tridiag_eigvals, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vals_smem()));
    attr = true;
  }
  tridiag_eigvals<<<n_probs, TT, vals_smem(), ctx->stream>>>(dp, G, T, w, A);
  TT_LAUNCH_CHECK(ctx);
  tt::pool_free(ctx, dp);
  return TT_OK;
}

int tt_sym_eigvecs_batched(tt_ctx* ctx, const tt_eig_problem* probs, int n_probs, const int* nvec,
                           const double* G, const double* T, const double* w, double* Z, double* work,
                           const double* A) {
  TT_REQUIRE(ctx && (n_probs == 0 || (probs && nvec && G && T && w && Z && work)),
             "tt_sym_eigvecs_batched: null argument");
  if (n_probs == 0) return TT_OK;
  for (int i = 0; i < n_probs; ++i) {
    TT_REQUIRE(probs[i].n >= 0 && probs[i].n <= MAX_N, "tt_sym_eigvecs_batched: n must be 0..2048");
    TT_REQUIRE(nvec[i] >= 0 && nvec[i] <= probs[i].n && nvec[i] <= MAX_N / 2,
               "tt_sym_eigvecs_batched: nvec must be 0..min(n, 1024)");
    if (probs[i].flags & TT_EIG_ROW_1X2) TT_REQUIRE(A, "tt_sym_eigvecs_batched: 1x2 case needs A");
  }
  std::vector<EigDev> hp = to_dev(probs, n_probs, nvec);
  EigDev* dp = tt::pool_alloc<EigDev>(ctx, n_probs);
  if (!dp) return tt::fail(TT_ERR_OOM, "tt_sym_eigvecs_batched: allocation failed");
  TT_CUDA(tt::h2d_async(ctx, dp, hp.data(), sizeof(EigDev) * n_probs));
  // shared memory for the largest problem that fits (the others iterate in global memory)
  int64_t need = 0;
  for (int i = 0; i < n_probs; ++i) {
    const int64_t with_u = 4 * (int64_t)probs[i].n * nvec[i] + probs[i].n;  // Z, reflector and LU scratch
    const int64_t z_only = (int64_t)probs[i].n * nvec[i] + probs[i].n;
    if (with_u <= kVecsSmemCap) need = std::max(need, with_u);
    else if (z_only <= kVecsSmemCap) need = std::max(need, z_only);
  }
  static thread_local bool attr = false;  // per host thread: each may drive its own device
  if (!attr) {
    TT_CUDA(cudaFuncSetAttribute(tridiag_eigvecs, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(sizeof(double) * kVecsSmemCap)));
    attr = true;
  }
  tridiag_eigvecs<<<n_probs, TT, sizeof(double) * (size_t)need, ctx->stream>>>(dp, G, T, w, Z, work, A, (int)need);
  TT_LAUNCH_CHECK(ctx);
  tt::pool_free(ctx, dp);
  return TT_OK;
}

}  // extern "C"
