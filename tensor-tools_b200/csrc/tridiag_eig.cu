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
#include <cooperative_groups.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

#include "tt_internal.h"

namespace {

constexpr int TT = 512;          // threads per CTA
constexpr int SM_N = 160;        // full n x n FP64 matrix in shared memory up to this size
constexpr int MAX_N = 4096;
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

// ---------------------------------------------------------------------------
// Sectors with n > SM_N: one thread-block cluster (CL CTAs, distributed shared
// memory) per sector, so a large density matrix is reduced by CL SMs at once
// instead of one SM streaming it from L2.
//
// Phase 1: the columns of G are dealt out cyclically (column c to CTA c % CL)
// and held in each CTA's shared memory when they fit (global otherwise).  For
// column k the owner builds the reflector v and publishes it; every CTA forms
// p = tau A22 v on its own columns and the partial p.v; after a second
// cluster barrier every CTA gathers p and the partial dots (fixed order, so
// every CTA holds the same w = p - (tau/2)(p.v) v) and applies the rank-2
// update to its own columns.  Two cluster barriers per column; the published
// buffers alternate by the parity of k, so no third barrier is needed.
// Bisection then runs over all warps of the cluster.
//
// Phase 2: CTA r owns eigenvectors [r q, r q + q), q = ceil(nvec / CL).
// Inverse iteration runs one thread per vector.  Gram-Schmidt (twice, inside
// the clusters of close eigenvalues as in the one-CTA kernel) takes vectors
// in order: each CTA projects the current vector y on its own earlier cluster
// members and publishes the partial sum of projections; after a cluster
// barrier every CTA subtracts all partial sums in CTA order.  Every CTA thus
// holds the same iterate, decides collapse/retry identically, and one barrier
// per projection round suffices (partial sums alternate between two buffers).
// The back-transformation needs no communication: every CTA applies all
// reflectors to its own vectors, staged a few at a time in shared memory.
// Every loop bound here is the same in all CTAs of a cluster, so every CTA
// reaches every cluster barrier.
namespace cgx = cooperative_groups;

constexpr int CL_STAGE = 4;  // reflectors staged per round of the back-transformation
constexpr int CL_MAX = 16;   // largest cluster the kernels are launched with

// doubles of shared memory the phase-1 cluster kernel needs besides the column slab
constexpr int CL_WARPS = TT / 32;  // warps per CTA
__host__ __device__ inline int64_t cluster_vals_extra(int n) { return 5 * (int64_t)n + 2 * CL_MAX * CL_WARPS; }

__device__ __forceinline__ int first_owned(int from, int rank, int CL) {
  // smallest l with rank + CL * l >= from
  return from <= rank ? 0 : (from - rank + CL - 1) / CL;
}

__global__ void __launch_bounds__(TT)
tridiag_eigvals_cluster(const EigDev* __restrict__ probs, double* G, double* Tg, double* W, int cap) {
  extern __shared__ double sm[];
  __shared__ double red[33];
  __shared__ double s_tau;
  cgx::cluster_group cluster = cgx::this_cluster();
  const int CL = (int)cluster.num_blocks();
  const int rank = (int)cluster.block_rank();
  const EigDev P = probs[blockIdx.x / CL];
  const int n = P.n;
  const int tid = threadIdx.x;
  if (n <= 0) return;  // the same problem for the whole cluster
  double* Gp = G + P.g_off;
  double* Wp = W + P.w_off;
  double* dg = Tg + 3 * P.w_off;
  double* eg = dg + n;
  double* tg = eg + n;
  const int lcols = (n + CL - 1) / CL;
  const int64_t extra = cluster_vals_extra(n);
  const bool in_smem = (int64_t)lcols * n + extra <= cap;
  double* rest = in_smem ? sm + (int64_t)lcols * n : sm;
  double* vbuf = rest;            // [2][n]: reflector published by the column's owner, tau in the last slot
  double* vloc = vbuf + 2 * n;    // this CTA's copy of v
  double* pfull = vloc + n;       // [2][n]: p, pushed here by the owners of its columns
  double* pdots = pfull + 2 * n;  // [2][CL_MAX * CL_WARPS]: partial p.v of every warp of the cluster
  auto col = [&](int l) -> double* {  // l-th owned column (global column rank + CL l)
    return in_smem ? sm + (int64_t)l * n : Gp + (int64_t)(rank + CL * l) * n;
  };
  if (in_smem)
    for (int l = 0; l < lcols && rank + CL * l < n; ++l)
      for (int i = tid; i < n; i += blockDim.x) sm[(int64_t)l * n + i] = Gp[(int64_t)(rank + CL * l) * n + i];
  __syncthreads();
  const int warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
  const int nslot = CL * nw;  // partial dots per column
  int lend = 0;               // owned columns that exist
  while (lend < lcols && rank + CL * lend < n) ++lend;
  double* const abase = col(0);
  const int64_t lstride = in_smem ? (int64_t)n : (int64_t)CL * n;  // between owned columns
  for (int k = 0; k + 2 < n; ++k) {
    const int m = n - k - 1;  // m <= n - 1: the last slot of vbuf is free for tau
    const int par = k & 1;
    const int owner = k % CL;
    if (rank == owner && warp == 0) {  // the reflector, by one warp of the owner
      const double* a = col(k / CL);
      double l0s = 0.0, l1s = 0.0;
      int i = 1 + lane;
      for (; i + 32 < m; i += 64) {
        l0s += a[k + 1 + i] * a[k + 1 + i];
        l1s += a[k + 33 + i] * a[k + 33 + i];
      }
      for (; i < m; i += 32) l0s += a[k + 1 + i] * a[k + 1 + i];
      double loc = l0s + l1s;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) loc += __shfl_xor_sync(0xffffffffu, loc, o);
      const double alpha = a[k + 1];
      double tau = 0.0, beta = alpha, scale = 0.0;
      if (loc != 0.0) {
        const double mu = sqrt(alpha * alpha + loc);
        beta = alpha <= 0.0 ? mu : -mu;
        tau = (beta - alpha) / beta;
        scale = 1.0 / (alpha - beta);
      }
      if (lane == 0) {
        tg[k] = tau;
        eg[k] = beta;
        vbuf[par * n + n - 1] = tau;
      }
      if (tau != 0.0)
        for (int j = lane; j < m; j += 32) {
          const double vi = (j == 0) ? 1.0 : a[k + 1 + j] * scale;
          vbuf[par * n + j] = vi;
          if (j > 0) Gp[(k + 1 + j) + (int64_t)n * k] = vi;  // reflector kept for phase 2
        }
    }
    cluster.sync();
    // one parallel pull of v and tau from the owner
    const double* ov = cluster.map_shared_rank(vbuf + par * n, owner);
    if (tid == 0) s_tau = ov[n - 1];
    for (int i = tid; i < m; i += blockDim.x) vloc[i] = ov[i];
    __syncthreads();
    const double tau = s_tau;
    if (tau == 0.0) continue;  // column already reduced (same decision in every CTA)
    // p = tau A22 v on the owned columns (A22 symmetric: column dot v), one
    // warp per column with four independent chains; lanes 0..CL-1 push p_c
    // into every CTA's pfull, and every warp pushes its share of p.v into
    // every CTA's pdots
    const int l0 = first_owned(k + 1, rank, CL);
    double wpart = 0.0;
    for (int l = l0 + warp; l < lend; l += nw) {
      const int c = rank + CL * l;
      const double* __restrict__ a = col(l) + k + 1;
      double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
      int i = lane;
      for (; i + 96 < m; i += 128) {
        s0 += a[i] * vloc[i];
        s1 += a[i + 32] * vloc[i + 32];
        s2 += a[i + 64] * vloc[i + 64];
        s3 += a[i + 96] * vloc[i + 96];
      }
      for (; i < m; i += 32) s0 += a[i] * vloc[i];
      double s = (s0 + s1) + (s2 + s3);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      const double pc = tau * s;
      if (lane < CL) *cluster.map_shared_rank(pfull + par * n + (c - k - 1), lane) = pc;
      wpart += pc * vloc[c - k - 1];
    }
    if (lane < CL) *cluster.map_shared_rank(pdots + par * CL_MAX * CL_WARPS + rank * nw + warp, lane) = wpart;
    cluster.sync();
    // p.v: every warp sums the same partials in the same order, so every
    // warp of every CTA holds the same K
    double x = 0.0;
    for (int j = lane; j < nslot; j += 32) x += pdots[par * CL_MAX * CL_WARPS + j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    const double K = 0.5 * tau * x;
    const double* pf = pfull + par * n;
    // A22 -= v w^T + w v^T on the owned columns, w = p - K v formed on the
    // fly: rows outer (v_i, w_i in registers), owned columns inner, four at a
    // time so their loads and stores overlap
    for (int i = tid; i < m; i += blockDim.x) {
      const double vi = vloc[i], wi = pf[i] - K * vi;
      double* __restrict__ ai = abase + (k + 1 + i);
      int l = l0;
      for (; l + 3 < lend; l += 4) {
        const int c0 = rank + CL * l - k - 1;
        const double v0 = vloc[c0], v1 = vloc[c0 + CL], v2 = vloc[c0 + 2 * CL], v3 = vloc[c0 + 3 * CL];
        const double w0 = pf[c0] - K * v0, w1 = pf[c0 + CL] - K * v1, w2 = pf[c0 + 2 * CL] - K * v2,
                     w3 = pf[c0 + 3 * CL] - K * v3;
        const double a0 = ai[l * lstride], a1 = ai[(l + 1) * lstride], a2 = ai[(l + 2) * lstride],
                     a3 = ai[(l + 3) * lstride];
        ai[l * lstride] = a0 - (vi * w0 + wi * v0);
        ai[(l + 1) * lstride] = a1 - (vi * w1 + wi * v1);
        ai[(l + 2) * lstride] = a2 - (vi * w2 + wi * v2);
        ai[(l + 3) * lstride] = a3 - (vi * w3 + wi * v3);
      }
      for (; l < lend; ++l) {
        const int cc = rank + CL * l - k - 1;
        const double vc = vloc[cc], wc = pf[cc] - K * vc;
        ai[l * lstride] -= vi * wc + wi * vc;
      }
    }
    __syncthreads();
  }
  // T: diagonal from the owners, the last off-diagonal A[n-1, n-2]
  for (int l = 0; l < lcols; ++l) {
    const int c = rank + CL * l;
    if (c >= n) break;
    if (tid == 0) dg[c] = col(l)[c];
    if (c == n - 2 && tid == 0) eg[n - 2] = col(l)[n - 1];
  }
  if (rank == 0 && tid == 0) {
    eg[n - 1] = 0.0;
    tg[n - 1] = 0.0;
    if (n >= 2) tg[n - 2] = 0.0;
  }
  __threadfence();
  cluster.sync();  // also the last access of another CTA's shared memory
  double* d = vloc;
  double* e2 = pfull;
  for (int i = tid; i < n; i += blockDim.x) {
    d[i] = dg[i];
    e2[i] = i < n - 1 ? eg[i] * eg[i] : 0.0;
  }
  __syncthreads();
  double lo_loc = DBL_MAX, hi_loc = -DBL_MAX, e2max = 0.0;
  for (int i = tid; i < n; i += blockDim.x) {
    const double r = (i > 0 ? fabs(eg[i - 1]) : 0.0) + (i < n - 1 ? fabs(eg[i]) : 0.0);
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
  if (bnorm == 0.0) {
    for (int j = rank * (int)blockDim.x + tid; j < n; j += CL * (int)blockDim.x) Wp[j] = 0.0;
    return;
  }
  // bisection as in tridiag_eigvals, over every warp of the cluster
  auto open_interval = [&](double lo, double hi) {
    return hi - lo > fmax(atol, 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)));
  };
  const int grp = lane < 30 ? lane / 3 : 0, sub = lane % 3;
  for (int base = (rank * nw + warp) * 10; base < n; base += CL * nw * 10) {
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
    if (active && sub == 0) Wp[n - 1 - j] = 0.5 * (lo + hi);
  }
}

__global__ void __launch_bounds__(TT)
tridiag_eigvecs_cluster(const EigDev* __restrict__ probs, const double* G, const double* Tg, const double* W,
                        double* Zg, double* work, int cap) {
  extern __shared__ double zsm[];
  __shared__ double red[33];
  __shared__ double coef[MAX_N / 2];
  __shared__ int cstart[MAX_N / 2];
  cgx::cluster_group cluster = cgx::this_cluster();
  const int CL = (int)cluster.num_blocks();
  const int rank = (int)cluster.block_rank();
  const EigDev P = probs[blockIdx.x / CL];
  const int n = P.n, nvec = P.nvec;
  const int tid = threadIdx.x;
  if (n <= 0 || nvec <= 0) return;  // the same problem for the whole cluster
  double* Zout = Zg + P.g_off;
  const int q = (nvec + CL - 1) / CL;
  const int j0 = rank * q, j1 = min(nvec, j0 + q), nown = max(0, j1 - j0);
  const bool in_smem = (int64_t)q * n + 6 * (int64_t)n <= cap;
  double* Z = in_smem ? zsm : Zout + (int64_t)n * j0;  // own vector t at Z + n t
  double* ybuf = in_smem ? zsm + (int64_t)q * n : zsm;  // the current Gram-Schmidt iterate
  double* ubuf = ybuf + n;                              // [2][n] published partial projections
  double* scr = ubuf + 2 * n;                           // 3n LU scratch
  const double* d = Tg + 3 * P.w_off;
  const double* e = d + n;
  const double* tau = e + n;
  const double* lam = W + P.w_off;  // descending
  const double* Gp = G + P.g_off;
  const int warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
  double loc = 0.0;
  for (int i = tid; i < n; i += blockDim.x)
    loc = fmax(loc, fabs(d[i]) + (i > 0 ? fabs(e[i - 1]) : 0.0) + (i + 1 < n ? fabs(e[i]) : 0.0));
  const double tnorm = block_reduce(loc, red, true);
  const double tiny = tnorm > 1e-250 ? fmax(DBL_EPSILON * tnorm, DBL_MIN) : 1.0;
  const double ortol = 1e-3 * tnorm;
  // (a) inverse iteration on the own vectors, one thread each (same start vectors as the one-CTA kernel)
  for (int t = tid; t < nown; t += blockDim.x) {
    const int j = j0 + t;
    double* y = Z + (int64_t)n * t;
    for (int i = 0; i < n; ++i) y[i] = hash_unit(((uint64_t)P.g_off << 20) ^ ((uint64_t)j << 32) ^ (uint64_t)i);
    for (int it = 0; it < INV_ITERS; ++it) {
      tri_solve(d, e, n, lam[j], tiny, y, work + 3 * P.g_off + (int64_t)3 * n * j, 1);
      double s = 0.0;
      for (int i = 0; i < n; ++i) s += y[i] * y[i];
      const double inv = 1.0 / sqrt(s);
      for (int i = 0; i < n; ++i) y[i] *= inv;
    }
  }
  if (tid == 0) {
    int c = 0;
    for (int j = 0; j < nvec && j < MAX_N / 2; ++j) {
      if (j == 0 || lam[j - 1] - lam[j] > ortol) c = j;
      cstart[j] = c;
    }
  }
  __syncthreads();
  cluster.sync();  // every start vector is in place
  // (b) Gram-Schmidt, vector by vector.  Which CTAs hold members of the
  // cluster [c0, j) follows from c0, j and q alone, so no flags are exchanged;
  // every CTA holds the same iterate y and forms its norm in the same order.
  int g = 0;
  for (int j = 1; j < nvec && j < MAX_N / 2; ++j) {
    const int c0 = cstart[j];
    if (c0 == j) continue;
    const int owner = j / q;
    const double* yj = in_smem ? cluster.map_shared_rank(zsm + (int64_t)n * (j - owner * q), owner)
                               : Zout + (int64_t)n * j;
    __syncthreads();  // every read of the previous iterate is done
    for (int i = tid; i < n; i += blockDim.x) ybuf[i] = yj[i];
    __syncthreads();
    const int ka = max(c0, j0), kb = min(j, j1);  // own members of the cluster before j
    const int o_lo = c0 / q, o_hi = (j - 1) / q;  // CTAs that own members
    for (int pass = 0; pass < 6; ++pass) {
      double n0 = 0.0;  // |y|^2 before the projections, every warp alike
      for (int i = lane; i < n; i += 32) n0 += ybuf[i] * ybuf[i];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) n0 += __shfl_xor_sync(0xffffffffu, n0, o);
      for (int r = 0; r < 2; ++r) {
        const int par = g & 1;
        double* u = ubuf + par * n;
        for (int k = ka + warp; k < kb; k += nw) {
          const double* __restrict__ zk = Z + (int64_t)n * (k - j0);
          double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;  // independent chains
          int i = lane;
          for (; i + 96 < n; i += 128) {
            s0 += zk[i] * ybuf[i];
            s1 += zk[i + 32] * ybuf[i + 32];
            s2 += zk[i + 64] * ybuf[i + 64];
            s3 += zk[i + 96] * ybuf[i + 96];
          }
          for (; i < n; i += 32) s0 += zk[i] * ybuf[i];
          double s = (s0 + s1) + (s2 + s3);
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
          if (lane == 0) coef[k - ka] = s;
        }
        __syncthreads();
        if (kb > ka)
          for (int i = tid; i < n; i += blockDim.x) {
            const double* __restrict__ zi = Z + (int64_t)n * (ka - j0) + i;
            double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
            int k = 0;
            const int nk = kb - ka;
            for (; k + 3 < nk; k += 4) {
              s0 += coef[k] * zi[(int64_t)n * k];
              s1 += coef[k + 1] * zi[(int64_t)n * (k + 1)];
              s2 += coef[k + 2] * zi[(int64_t)n * (k + 2)];
              s3 += coef[k + 3] * zi[(int64_t)n * (k + 3)];
            }
            for (; k < nk; ++k) s0 += coef[k] * zi[(int64_t)n * k];
            u[i] = (s0 + s1) + (s2 + s3);
          }
        cluster.sync();
        for (int i = tid; i < n; i += blockDim.x) {
          double rr[CL_MAX];  // every remote load in flight at once, then the sum in CTA order
#pragma unroll
          for (int o = 0; o < CL_MAX; ++o)
            rr[o] = (o >= o_lo && o <= o_hi && o < CL) ? *cluster.map_shared_rank(u + i, o) : 0.0;
          double s = ybuf[i];
#pragma unroll
          for (int o = 0; o < CL_MAX; ++o) s -= rr[o];
          ybuf[i] = s;
        }
        __syncthreads();
        ++g;
        if (r == 0) {
          // "twice is enough" (Kahan, Parlett): a second projection only when
          // the first removed more than half of |y|^2; every CTA and warp holds
          // the same y and takes the same decision
          double n1 = 0.0;
          for (int i = lane; i < n; i += 32) n1 += ybuf[i] * ybuf[i];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) n1 += __shfl_xor_sync(0xffffffffu, n1, o);
          if (n1 > 0.5 * n0) break;
        }
      }
      double nl = 0.0;  // every warp: the whole norm, same order
      for (int i = lane; i < n; i += 32) nl += ybuf[i] * ybuf[i];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) nl += __shfl_xor_sync(0xffffffffu, nl, o);
      const double nrm = sqrt(nl);
      if (nrm > 0.5 || pass == 5) {
        const double inv = nrm > 0.0 ? 1.0 / nrm : 0.0;
        if (rank == owner)
          for (int i = tid; i < n; i += blockDim.x) Z[(int64_t)n * (j - j0) + i] = ybuf[i] * inv;
        break;
      }
      // collapsed onto earlier vectors: one more inverse iteration from the
      // orthogonal remainder (every CTA alike), then orthogonalise again
      __syncthreads();
      if (tid == 0) {
        const double inv = nrm > 0.0 ? 1.0 / nrm : 1.0;
        for (int i = 0; i < n; ++i) ybuf[i] = nrm > 0.0 ? ybuf[i] * inv : hash_unit((uint64_t)(j * 7919 + i + pass));
        tri_solve(d, e, n, lam[j], tiny, ybuf, scr, 1);
      }
      __syncthreads();
    }
  }
  cluster.sync();  // no CTA reads another's shared memory after this point
  // (c) back-transformation z = H_0 H_1 ... H_{n-3} y, last reflector first
  double* stg = ubuf;  // CL_STAGE staged reflectors (5n doubles available)
  for (int kb = n - 3; kb >= 0; kb -= CL_STAGE) {
    __syncthreads();
    for (int s = 0; s < CL_STAGE && kb - s >= 0; ++s) {
      const int k = kb - s, m = n - k - 1;
      for (int i = tid; i < m; i += blockDim.x) stg[(int64_t)s * n + i] = (i == 0) ? 1.0 : Gp[(k + 1 + i) + (int64_t)n * k];
    }
    __syncthreads();
    for (int t = warp; t < nown; t += nw) {
      double* y = Z + (int64_t)n * t;
      for (int s = 0; s < CL_STAGE && kb - s >= 0; ++s) {
        const int k = kb - s, m = n - k - 1;
        const double tk = tau[k];
        if (tk == 0.0) continue;
        const double* __restrict__ v = stg + (int64_t)s * n;
        const double* __restrict__ yk = y + k + 1;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;  // independent chains
        int i = lane;
        for (; i + 96 < m; i += 128) {
          a0 += v[i] * yk[i];
          a1 += v[i + 32] * yk[i + 32];
          a2 += v[i + 64] * yk[i + 64];
          a3 += v[i + 96] * yk[i + 96];
        }
        for (; i < m; i += 32) a0 += v[i] * yk[i];
        double acc = (a0 + a1) + (a2 + a3);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        const double c = tk * acc;
        for (int i = lane; i < m; i += 32) y[k + 1 + i] -= v[i] * c;
        __syncwarp();
      }
    }
  }
  __syncthreads();
  // (d) deterministic gauge: the largest-magnitude entry (first on ties) is positive
  for (int t = warp; t < nown; t += nw) {
    double* y = Z + (int64_t)n * t;
    double best = -1.0;
    int bi = n;
    for (int i = lane; i < n; i += 32) {
      const double a = fabs(y[i]);
      if (a > best) { best = a; bi = i; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
    }
    const bool flip = bi < n && y[bi] < 0.0;
    __syncwarp();
    if (flip)
      for (int i = lane; i < n; i += 32) y[i] = -y[i];
  }
  if (in_smem) {
    __syncthreads();
    for (int64_t i = tid; i < (int64_t)n * nown; i += blockDim.x) Zout[(int64_t)n * j0 + i] = Z[i];
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

// Sectors above the shared-memory size of the one-CTA kernels go to the cluster kernels.
bool is_big(const EigDev& e) { return e.n > SM_N && !(e.flags & TT_EIG_ROW_1X2); }

// Cluster size and shared-memory caps of the cluster kernels on this thread's
// device: 16 CTAs per cluster when the device can co-schedule that many with
// the full shared-memory carve-out, else 8, else none (the one-CTA kernels
// take every problem).
struct ClusterPlan {
  int device = -1;
  int cl = 0;
  int64_t vals_cap = 0, vecs_cap = 0;  // doubles of dynamic shared memory per CTA
};

const ClusterPlan& cluster_plan(tt_ctx* ctx) {
  static thread_local ClusterPlan cp;
  if (cp.device == ctx->device) return cp;
  cp = ClusterPlan();
  cp.device = ctx->device;
  int optin = 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device) != cudaSuccess) {
    cudaGetLastError();
    return cp;
  }
  cudaFuncAttributes fa, fb;
  if (cudaFuncGetAttributes(&fa, tridiag_eigvals_cluster) != cudaSuccess ||
      cudaFuncGetAttributes(&fb, tridiag_eigvecs_cluster) != cudaSuccess) {
    cudaGetLastError();
    return cp;
  }
  const int64_t va = ((int64_t)optin - (int64_t)fa.sharedSizeBytes - 1024) / 8;
  const int64_t vb = ((int64_t)optin - (int64_t)fb.sharedSizeBytes - 1024) / 8;
  if (va < cluster_vals_extra(MAX_N) || vb < 6 * MAX_N) return cp;
  const void* kernels[2] = {(const void*)tridiag_eigvals_cluster, (const void*)tridiag_eigvecs_cluster};
  const int64_t caps[2] = {va, vb};
  for (int k = 0; k < 2; ++k) {
    if (cudaFuncSetAttribute(kernels[k], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(caps[k] * 8)) !=
            cudaSuccess ||
        cudaFuncSetAttribute(kernels[k], cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
      cudaGetLastError();
      return cp;
    }
  }
  for (int cl : {CL_MAX, 8}) {
    bool ok = true;
    for (int k = 0; k < 2 && ok; ++k) {
      cudaLaunchConfig_t cfg = {};
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = cl;
      at[0].val.clusterDim.y = 1;
      at[0].val.clusterDim.z = 1;
      cfg.gridDim = dim3(cl);
      cfg.blockDim = dim3(TT);
      cfg.dynamicSmemBytes = (size_t)(caps[k] * 8);
      cfg.attrs = at;
      cfg.numAttrs = 1;
      int nc = 0;
      if (cudaOccupancyMaxActiveClusters(&nc, kernels[k], &cfg) != cudaSuccess) {
        cudaGetLastError();
        nc = 0;
      }
      ok = nc >= 1;
    }
    if (ok) {
      cp.cl = cl;
      break;
    }
  }
  cp.vals_cap = va;
  cp.vecs_cap = vb;
  return cp;
}

// One cluster of `cl` CTAs per problem; `need` doubles of dynamic shared memory.
template <class... Args>
cudaError_t launch_cluster(tt_ctx* ctx, int cl, int n_probs, int64_t need, const void* kernel, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = cl;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3((unsigned)(cl * n_probs));
  cfg.blockDim = dim3(TT);
  cfg.dynamicSmemBytes = (size_t)(need * 8);
  cfg.stream = ctx->stream;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  void* argv[] = {(void*)&args...};
  const cudaError_t e = cudaLaunchKernelExC(&cfg, kernel, argv);
  tt::count_launch(ctx);
  return e;
}

}  // namespace

extern "C" {

int tt_sym_eigvals_batched(tt_ctx* ctx, const tt_eig_problem* probs, int n_probs, double* G, double* T,
                           double* w, const double* A) {
  TT_REQUIRE(ctx && (n_probs == 0 || (probs && G && T && w)), "tt_sym_eigvals_batched: null argument");
  if (n_probs == 0) return TT_OK;
  for (int i = 0; i < n_probs; ++i) {
    TT_REQUIRE(probs[i].n >= 0 && probs[i].n <= MAX_N, "tt_sym_eigvals_batched: n must be 0..4096");
    if (probs[i].flags & TT_EIG_ROW_1X2)
      TT_REQUIRE(probs[i].n == 2 && A, "tt_sym_eigvals_batched: 1x2 case needs n == 2 and A");
  }
  std::vector<EigDev> all = to_dev(probs, n_probs, nullptr);
  const ClusterPlan& cp = cluster_plan(ctx);
  std::vector<EigDev> small, big;
  for (const EigDev& e : all) (cp.cl > 0 && is_big(e) ? big : small).push_back(e);
  EigDev* dp = tt::pool_alloc<EigDev>(ctx, all.size());
  if (!dp) return tt::fail(TT_ERR_OOM, "tt_sym_eigvals_batched: allocation failed");
  small.insert(small.end(), big.begin(), big.end());  // small problems first, then the cluster ones
  TT_CUDA(tt::h2d_async(ctx, dp, small.data(), sizeof(EigDev) * small.size()));
  const int n_small = (int)(small.size() - big.size());
  static thread_local uint64_t attr = 0;  // per host thread and device
  if (tt::first_on_device(attr, ctx->device))
    TT_CUDA(cudaFuncSetAttribute(tridiag_eigvals, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vals_smem()));
  if (n_small > 0) {
    tridiag_eigvals<<<n_small, TT, vals_smem(), ctx->stream>>>(dp, G, T, w, A);
    TT_LAUNCH_CHECK(ctx);
  }
  if (!big.empty()) {
    int64_t need = 0;  // doubles: the column slab in shared memory when it fits under the cap
    for (const EigDev& e : big) {
      const int64_t lcols = (e.n + cp.cl - 1) / cp.cl;
      const int64_t extra = cluster_vals_extra(e.n);
      const int64_t full = lcols * e.n + extra;
      need = std::max(need, full <= cp.vals_cap ? full : extra);
    }
    TT_CUDA(launch_cluster(ctx, cp.cl, (int)big.size(), need, (const void*)tridiag_eigvals_cluster,
                           dp + n_small, G, T, w, (int)need));
  }
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
    TT_REQUIRE(probs[i].n >= 0 && probs[i].n <= MAX_N, "tt_sym_eigvecs_batched: n must be 0..4096");
    TT_REQUIRE(nvec[i] >= 0 && nvec[i] <= probs[i].n && nvec[i] <= MAX_N / 2,
               "tt_sym_eigvecs_batched: nvec must be 0..min(n, 2048)");
    if (probs[i].flags & TT_EIG_ROW_1X2) TT_REQUIRE(A, "tt_sym_eigvecs_batched: 1x2 case needs A");
  }
  std::vector<EigDev> all = to_dev(probs, n_probs, nvec);
  const ClusterPlan& cp = cluster_plan(ctx);
  std::vector<EigDev> small, big;
  for (const EigDev& e : all) (cp.cl > 0 && is_big(e) ? big : small).push_back(e);
  EigDev* dp = tt::pool_alloc<EigDev>(ctx, all.size());
  if (!dp) return tt::fail(TT_ERR_OOM, "tt_sym_eigvecs_batched: allocation failed");
  const int n_small = (int)small.size();
  small.insert(small.end(), big.begin(), big.end());
  TT_CUDA(tt::h2d_async(ctx, dp, small.data(), sizeof(EigDev) * small.size()));
  // shared memory for the largest problem that fits (the others iterate in global memory)
  int64_t need = 0;
  for (int i = 0; i < n_small; ++i) {
    const EigDev& e = small[i];
    const int64_t with_u = 4 * (int64_t)e.n * e.nvec + e.n;  // Z, reflector and LU scratch
    const int64_t z_only = (int64_t)e.n * e.nvec + e.n;
    if (with_u <= kVecsSmemCap) need = std::max(need, with_u);
    else if (z_only <= kVecsSmemCap) need = std::max(need, z_only);
  }
  static thread_local uint64_t attr = 0;  // per host thread and device
  if (tt::first_on_device(attr, ctx->device))
    TT_CUDA(cudaFuncSetAttribute(tridiag_eigvecs, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(sizeof(double) * kVecsSmemCap)));
  if (n_small > 0) {
    tridiag_eigvecs<<<n_small, TT, sizeof(double) * (size_t)need, ctx->stream>>>(dp, G, T, w, Z, work, A,
                                                                                  (int)need);
    TT_LAUNCH_CHECK(ctx);
  }
  if (!big.empty()) {
    int64_t needc = 0;  // doubles: own eigenvectors in shared memory when they fit, plus 6n of buffers
    for (const EigDev& e : big) {
      const int64_t q = (e.nvec + cp.cl - 1) / cp.cl;
      const int64_t extra = 6 * (int64_t)e.n;
      const int64_t full = q * e.n + extra;
      needc = std::max(needc, full <= cp.vecs_cap ? full : extra);
    }
    TT_CUDA(launch_cluster(ctx, cp.cl, (int)big.size(), needc, (const void*)tridiag_eigvecs_cluster,
                           dp + n_small, G, T, w, Z, work, (int)needc));
  }
  tt::pool_free(ctx, dp);
  return TT_OK;
}

}  // extern "C"
