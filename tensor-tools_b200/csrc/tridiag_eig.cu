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
  int32_t n, flags, nvec, nb;  // nb: panel width of the blocked cluster reduction
  int64_t s_off;               // its n x 2nb panel scratch (blocked cluster reduction)
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

// number of eigenvalues of T (diag d, squared offdiag e2) that are < x: the
// sign changes of the Sturm sequence p_i = (d_i - x) p_{i-1} - e2_{i-1} p_{i-2}
// of leading principal minors (Golub & Van Loan, "Matrix Computations", 4th
// ed., sec. 8.4.1), counted as LAPACK's dlaebz counts the non-positive pivots
// q_i = p_i / p_{i-1} of T - x I -- without its division per step: a pivot
// with |q_i| <= pivmin is replaced by a tiny negative one (here p_i = -p_{i-1}
// 2^-200, which steers the next step as q = -pivmin does), and the pair
// (p_{i-1}, p_i) is rescaled by a power of two when p_i leaves [2^-400, 2^400]
__device__ int sturm_count(const double* d, const double* e2, int n, double x, double pivmin) {
  double pm = 1.0;
  double p = d[0] - x;
  if (fabs(p) <= pivmin) p = -pivmin;
  int c = p <= 0.0;
  for (int i = 1; i < n; ++i) {
    double pn = fma(d[i] - x, p, -e2[i - 1] * pm);
    if (fabs(pn) <= pivmin * fabs(p)) pn = -p * 0x1p-200;
    c += (pn < 0.0) != (p < 0.0);
    const double a = fabs(pn);
    if (a > 0x1p400 || a < 0x1p-400) {
      int ex;
      frexp(pn, &ex);
      const double sc = ldexp(1.0, -ex);
      pn *= sc;
      p *= sc;
    }
    pm = p;
    p = pn;
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
// The LU factors go to u0, u1, u2, entry i at [i * ustride] (ustride > 1
// interleaves the factors of neighbouring threads, so that their accesses
// coalesce); y's entry i is at [i * ystride].
__device__ void tri_solve(const double* d, const double* e, int n, double lambda, double tiny, double* y,
                          double* u0, double* u1, double* u2, int ystride, int ustride) {
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
      u0[(int64_t)i * ustride] = di;
      u1[(int64_t)i * ustride] = si;
      u2[(int64_t)i * ustride] = ti;
      y[(int64_t)i * ystride] = bi;
      bi = bnext - mlt * bi;
      double nd = an - mlt * si, ns = bn - mlt * ti;
      di = nd;
      si = ns;
      ti = 0.0;
    } else {
      double mlt = di / ci;
      u0[(int64_t)i * ustride] = ci;
      u1[(int64_t)i * ustride] = an;
      u2[(int64_t)i * ustride] = bn;
      y[(int64_t)i * ystride] = bnext;
      bi = bi - mlt * bnext;
      double nd = si - mlt * an, ns = ti - mlt * bn;
      di = nd;
      si = ns;
      ti = 0.0;
    }
  }
  if (fabs(di) < tiny) di = di < 0.0 ? -tiny : tiny;
  u0[(int64_t)(n - 1) * ustride] = di;
  y[(int64_t)(n - 1) * ystride] = bi;
  // back substitution
  for (int i = n - 1; i >= 0; --i) {
    double s = y[(int64_t)i * ystride];
    if (i + 1 < n) s -= u1[(int64_t)i * ustride] * y[(int64_t)(i + 1) * ystride];
    if (i + 2 < n) s -= u2[(int64_t)i * ustride] * y[(int64_t)(i + 2) * ystride];
    double piv = u0[(int64_t)i * ustride];
    if (fabs(piv) < tiny) piv = piv < 0.0 ? -tiny : tiny;
    y[(int64_t)i * ystride] = s / piv;
  }
}

// tri_solve for a thread's column of an interleaved batch (y, u0, u1, u2 all
// with stride st), with the global loads issued PF steps ahead: the values of
// the next PF steps are fetched while the current PF are computed (the
// threads of a CTA walk the same rows in lockstep, so the batch's accesses
// coalesce and the latency of one step is the arithmetic's, not memory's).
// The same elimination with partial pivoting as tri_solve, but each step
// takes one reciprocal: u0 keeps 1 / pivot (the pivot clamped to +-tiny as
// the back substitution of tri_solve clamps it), used for the multiplier
// and again in the back substitution.  The right-hand side is y * scale
// (the previous iterate's normalisation, applied as it is read), and the
// return value is the squared norm of the solution, summed as it is solved.
constexpr int PF = 8;
__device__ __forceinline__ double clamped_rcp(double piv, double tiny) {
  return 1.0 / (fabs(piv) < tiny ? (piv < 0.0 ? -tiny : tiny) : piv);
}
__device__ double tri_solve_il(const double* d, const double* e, int n, double lambda, double tiny, double scale,
                               double* y, double* u0, double* u1, double* u2, int64_t st) {
  // forward elimination; step i reads y[i + 1]
  double di = d[0] - lambda, si = n > 1 ? e[0] : 0.0, ti = 0.0;
  double bi = y[0] * scale;
  double cur[PF], nxt[PF];
#pragma unroll
  for (int k = 0; k < PF; ++k) cur[k] = 1 + k < n ? y[(int64_t)(1 + k) * st] * scale : 0.0;
  for (int i0 = 0; i0 + 1 < n; i0 += PF) {
#pragma unroll
    for (int k = 0; k < PF; ++k) {
      const int r = i0 + PF + 1 + k;
      nxt[k] = r < n ? y[(int64_t)r * st] * scale : 0.0;
    }
#pragma unroll
    for (int k = 0; k < PF; ++k) {
      const int i = i0 + k;
      if (i + 1 < n) {
        double ci = e[i];
        double an = d[i + 1] - lambda;
        double bn = (i + 2 < n) ? e[i + 1] : 0.0;
        double bnext = cur[k];
        if (fabs(di) >= fabs(ci)) {
          if (di == 0.0) di = tiny;
          const double r = 1.0 / di;
          const double mlt = ci * r;
          u0[(int64_t)i * st] = fabs(di) < tiny ? clamped_rcp(di, tiny) : r;
          u1[(int64_t)i * st] = si;
          u2[(int64_t)i * st] = ti;
          y[(int64_t)i * st] = bi;
          bi = bnext - mlt * bi;
          double nd = an - mlt * si, ns = bn - mlt * ti;
          di = nd;
          si = ns;
          ti = 0.0;
        } else {
          const double r = 1.0 / ci;
          const double mlt = di * r;
          u0[(int64_t)i * st] = fabs(ci) < tiny ? clamped_rcp(ci, tiny) : r;
          u1[(int64_t)i * st] = an;
          u2[(int64_t)i * st] = bn;
          y[(int64_t)i * st] = bnext;
          bi = bi - mlt * bnext;
          double nd = si - mlt * an, ns = ti - mlt * bn;
          di = nd;
          si = ns;
          ti = 0.0;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < PF; ++k) cur[k] = nxt[k];
  }
  u0[(int64_t)(n - 1) * st] = clamped_rcp(di, tiny);
  y[(int64_t)(n - 1) * st] = bi;
  // back substitution, i = n - 1 down to 0; step i reads y[i], u0[i], u1[i], u2[i]
  double x1 = 0.0, x2 = 0.0;  // y[i + 1], y[i + 2] as solved
  double ss = 0.0;
  double cy[PF], c0[PF], c1[PF], c2[PF], ny[PF], n0[PF], n1[PF], n2[PF];
#pragma unroll
  for (int k = 0; k < PF; ++k) {
    const int i = n - 1 - k;
    cy[k] = i >= 0 ? y[(int64_t)i * st] : 0.0;
    c0[k] = i >= 0 ? u0[(int64_t)i * st] : 1.0;
    c1[k] = i >= 0 ? u1[(int64_t)i * st] : 0.0;
    c2[k] = i >= 0 ? u2[(int64_t)i * st] : 0.0;
  }
  for (int b0 = n - 1; b0 >= 0; b0 -= PF) {
#pragma unroll
    for (int k = 0; k < PF; ++k) {
      const int i = b0 - PF - k;
      ny[k] = i >= 0 ? y[(int64_t)i * st] : 0.0;
      n0[k] = i >= 0 ? u0[(int64_t)i * st] : 1.0;
      n1[k] = i >= 0 ? u1[(int64_t)i * st] : 0.0;
      n2[k] = i >= 0 ? u2[(int64_t)i * st] : 0.0;
    }
#pragma unroll
    for (int k = 0; k < PF; ++k) {
      const int i = b0 - k;
      if (i >= 0) {
        double s = cy[k];
        if (i + 1 < n) s -= c1[k] * x1;
        if (i + 2 < n) s -= c2[k] * x2;
        const double xi = s * c0[k];
        y[(int64_t)i * st] = xi;
        ss = fma(xi, xi, ss);
        x2 = x1;
        x1 = xi;
      }
    }
#pragma unroll
    for (int k = 0; k < PF; ++k) {
      cy[k] = ny[k];
      c0[k] = n0[k];
      c1[k] = n1[k];
      c2[k] = n2[k];
    }
  }
  return ss;
}

// U holds the three factor rows back to back (3 n doubles)
__device__ void tri_solve(const double* d, const double* e, int n, double lambda, double tiny, double* y,
                          double* U, int ystride) {
  tri_solve(d, e, n, lambda, tiny, y, U, U + n, U + 2 * n, ystride, 1);
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
// Phase 1 is the blocked Householder tridiagonalisation of LAPACK's dsytrd /
// dlatrd (Golub & Van Loan, "Matrix Computations", 4th ed., sec. 8.3.1 with
// the panel form of sec. 5.1.7): the reflectors of a panel of nb columns are
// formed one by one against the matrix as it stood at the start of the
// panel, corrected on the fly by the panel's V and W (A22 v - V W^T v -
// W V^T v), and the trailing matrix receives the rank-2nb update
// A -= V W^T + W V^T once per panel.  Only the lower triangle is read or
// updated.  Index c (row or column) belongs to CTA c % CL.  Per column j,
// two cluster barriers:
//   1. the owners of rows >= j bring column j up to date and push it to
//      every CTA (barrier A);
//   2. every CTA forms the same reflector from the whole column (same data,
//      same reduction order), keeps v, and pushes its partial V^T v, W^T v;
//   3. every CTA runs A22 v over the lower triangle of its own columns: one
//      warp per block of 64 rows, each lane two rows, columns 16 at a time;
//      an element A[i,c] (i >= c) adds A[i,c] v_i to the dot of column c and,
//      below the diagonal, A[i,c] v_c to row i.  The column dots are summed
//      across the lanes by a butterfly reduce-scatter (lane k ends with
//      column k % 16), the row sums go to the row's owner (a slot per
//      sender), and the CTA's share of v^T A22 v to every CTA (barrier B);
//   4. every CTA completes p = A22 v on its own rows (own dot + the pushed row
//      sums, in CTA order), w' = tau (p - V W^T v - W V^T v) and
//      w = w' - (tau/2)(w'.v) v with w'.v = tau (v^T A22 v - 2 (V^T v).(W^T v));
//      the panel's rows, which every CTA needs, have their row sums and
//      column dots pushed to every CTA.
// Every CTA sums pushed partials in CTA order, so every decision and scalar
// is the same in every CTA.  The trailing update goes through a global
// n x 2nb scratch (two barriers per panel): m8n8k4 FP64 tensor-core (DMMA)
// products of 32 rows x 16 own columns per warp, the rows' [V W] read from
// the scratch and the columns' from shared memory.  The eigenvalues follow by
// bisection in a separate, GPU-wide launch (bisect_sectors).
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
constexpr int PNB_MAX = 32;  // widest panel of the blocked reduction
constexpr int NWARP = TT / 32;
struct VecTaskB {
  int32_t prob, j0;  // problem (index into the problem array) and first eigenvalue
};

// doubles of dynamic shared memory of the blocked cluster reduction
__host__ __device__ inline int64_t blocked_smem(int n, int nb, int CL) {
  const int64_t nloc = (n + CL - 1) / CL;
  return 2 * (int64_t)nb * nloc        // V, W of the panel on the own rows
         + 2 * nloc                    // the own rows of the current and the next column
         + (int64_t)CL * nloc          // the pushed column, then v, owner-major
         + (int64_t)CL * nloc          // this CTA's row sums of A22 v, owner-major
         + (int64_t)CL * nloc          // pushed row sums of A22 v on the own rows, per sender
         + (int64_t)NWARP * nloc       // per-warp column dots
         + CL_MAX * 2 * (int64_t)nb    // pushed V^T v, W^T v partials
         + CL_MAX                      // pushed v^T A22 v partials
         + CL_MAX * (int64_t)nb        // pushed row sums on the panel's rows
         + nb                          // pushed column dots of the panel's rows
         + 2 * (int64_t)nb * nb        // V, W on the panel's rows
         + 2 * (int64_t)nb;            // V^T v, W^T v
}

// D += A B for one m8n8k4 FP64 tile (DMMA): A 8x4 row fragment (lane L holds
// A[L/4][L%4]), B 4x8 column fragment (B[L%4][L/4]), D 8x8 (D[L/4][2(L%4)+e])
__device__ __forceinline__ void dmma_tr(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

__device__ __forceinline__ int first_owned(int from, int rank, int CL) {
  // smallest l with rank + CL * l >= from
  return from <= rank ? 0 : (from - rank + CL - 1) / CL;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// acc[k] (k < 16) summed over the 32 lanes of the warp, lane L receiving the
// sum of index L % 16: a butterfly sum across the half-warps, then a
// reduce-scatter (31 shuffles for 16 sums)
__device__ __forceinline__ double warp_reduce_scatter16(double (&acc)[16], int lane) {
#pragma unroll
  for (int k = 0; k < 16; ++k) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], 16);
#pragma unroll
  for (int s = 8; s >= 1; s >>= 1) {
    const bool up = (lane & s) != 0;
#pragma unroll
    for (int k = 0; k < s; ++k) {
      const double send = up ? acc[k] : acc[k + s];
      const double keep = up ? acc[k + s] : acc[k];
      acc[k] = keep + __shfl_xor_sync(0xffffffffu, send, s);
    }
  }
  return acc[0];
}

__global__ void __launch_bounds__(TT)
tridiag_eigvals_cluster(const EigDev* __restrict__ probs, double* G, double* Tg, double* W, double* VWg) {
  extern __shared__ double sm[];
  __shared__ double red[33];
  __shared__ double s_K;
  __shared__ double vw_part[NWARP * 2 * PNB_MAX];  // per-warp V^T v, W^T v sums

  cgx::cluster_group cluster = cgx::this_cluster();
  const int CL = (int)cluster.num_blocks();
  const int rank = (int)cluster.block_rank();
  const EigDev P = probs[blockIdx.x / CL];
  const int n = P.n;
  const int tid = threadIdx.x;
  if (n <= 0) return;  // the same problem for the whole cluster
  const int nb = P.nb;
  double* Gp = G + P.g_off;
  double* Wp = W + P.w_off;
  double* dg = Tg + 3 * P.w_off;
  double* eg = dg + n;
  double* tg = eg + n;
  double* VW = VWg + P.s_off;  // n x 2nb, row-major: [i][t] = V(i, t), [i][nb + t] = W(i, t)
  const int warp = tid >> 5, lane = tid & 31;
  const int nloc = (n + CL - 1) / CL;
  int lown = 0;  // own indices c = rank + CL l, l < lown
  while (lown < nloc && rank + CL * lown < n) ++lown;
  double* Vl = sm;                            // [nb][nloc]
  double* Wl = Vl + (int64_t)nb * nloc;       // [nb][nloc]
  double* xc = Wl + (int64_t)nb * nloc;       // [2][nloc]: own rows of a column, by parity of jj
  // Vectors over all rows are kept owner-major: row i = r + CL l at [r nloc + l],
  // so what one CTA pushes to another is contiguous on both sides
  const int lg = __ffs(CL) - 1;  // CL is a power of two
  auto om = [&](int i) { return ((i & (CL - 1)) * nloc) + (i >> lg); };
  double* xo = xc + 2 * nloc;                 // [CL][nloc]: column j as pushed, then v
  double* yl = xo + (int64_t)CL * nloc;       // [CL][nloc]: this CTA's row sums of A22 v
  double* yb = yl + (int64_t)CL * nloc;       // [CL][nloc]: row sums of A22 v on the own rows, by sender
  double* dw = yb + (int64_t)CL * nloc;       // [NWARP][nloc]: column dots by warp
  double* r2 = dw + (int64_t)NWARP * nloc;    // [CL_MAX][2nb]: V^T v, W^T v partials by sender
  double* r3 = r2 + CL_MAX * 2 * nb;          // [CL_MAX]: v^T A22 v partials by sender
  double* yp = r3 + CL_MAX;                   // [CL_MAX][nb]: row sums on the panel's rows by sender
  double* dp = yp + CL_MAX * nb;              // [nb]: column dots of the panel's rows
  double* Vp = dp + nb;                       // [nb][nb]: Vp[t nb + s] = v_t[k0 + s]
  double* Wq = Vp + nb * nb;                  // [nb][nb]: Wq[t nb + s] = w_t[k0 + s]
  double* cvt = Wq + nb * nb;                 // [nb]: V^T v
  double* cwt = cvt + nb;                     // [nb]: W^T v
  for (int k0 = 0; k0 + 2 < n; k0 += nb) {
    const int nbe = min(nb, n - 2 - k0);  // reflector columns k0 .. k0 + nbe - 1
    for (int jj = 0; jj < nbe; ++jj) {
      const int j = k0 + jj;
      double* xcur = xc + (jj & 1) * nloc;
      // ---- 1: column j on the own rows >= j, pushed to every CTA ----
      const int l1 = first_owned(j, rank, CL);
      {
        // four threads per row, each summing a quarter of the panel's terms
        // (the loop bound is the same for the whole warp: the shuffles need it)
        const int sub = tid & 3;
        for (int base = l1 + (warp << 3); base < lown; base += blockDim.x >> 2) {
          const int l = base + (lane >> 2);
          const bool act = l < lown;
          double corr = 0.0;
          if (act)
#pragma unroll 1
            for (int t = sub; t < jj; t += 4)
              corr += Vl[t * nloc + l] * Wq[t * nb + jj] + Wl[t * nloc + l] * Vp[t * nb + jj];
          corr += __shfl_xor_sync(0xffffffffu, corr, 1);
          corr += __shfl_xor_sync(0xffffffffu, corr, 2);
          if (act && sub == 0) xcur[l] = (jj == 0 ? Gp[(rank + CL * l) + (int64_t)n * j] : xcur[l]) - corr;
        }
      }
      __syncthreads();
      for (int e = tid; e < (lown - l1) * CL; e += blockDim.x) {
        const int q = e / (lown - l1), l = l1 + e % (lown - l1);
        *cluster.map_shared_rank(xo + rank * nloc + l, q) = xcur[l];
      }
      cluster.sync();  // A
      // ---- 2: the reflector (same in every CTA), v kept, V^T v and W^T v partials ----
      const double alpha = xo[om(j + 1)];  // read before the reduction's barriers, overwritten below
      double part = 0.0;
      for (int i = j + 2 + tid; i < n; i += blockDim.x) part += xo[om(i)] * xo[om(i)];
      const double sigma = block_reduce(part, red, false);
      double tau = 0.0, beta = alpha, scale = 0.0;
      if (sigma != 0.0) {
        const double mu = sqrt(alpha * alpha + sigma);
        beta = alpha <= 0.0 ? mu : -mu;
        tau = (beta - alpha) / beta;
        scale = 1.0 / (alpha - beta);
      }
      if (rank == j % CL && tid == 0) {
        dg[j] = xo[om(j)];
        tg[j] = tau;
        eg[j] = beta;
      }
      for (int i = j + 1 + tid; i < n; i += blockDim.x) xo[om(i)] = i == j + 1 ? 1.0 : xo[om(i)] * scale;
      __syncthreads();
      for (int l = tid; l < lown; l += blockDim.x) {
        const int i = rank + CL * l;
        const double vi = i >= j + 1 ? xo[rank * nloc + l] : 0.0;
        Vl[jj * nloc + l] = vi;
        Wl[jj * nloc + l] = 0.0;
        if (i >= j + 2) Gp[i + (int64_t)n * j] = vi;  // reflector kept below the subdiagonal for phase 2
      }
      for (int s = tid; s < nb; s += blockDim.x) {
        const int row = k0 + s;
        Vp[jj * nb + s] = row >= j + 1 && row < n ? xo[om(row)] : 0.0;
      }
      __syncthreads();
      const int lf = first_owned(j + 1, rank, CL);
      // V^T v and W^T v partials over the own rows >= j + 1: lane t of each
      // warp sums column t over every NWARP-th row, the warps' sums are added
      // in warp order and pushed to every CTA
      if (jj > 0) {
        double sv = 0.0, sw = 0.0;
        if (lane < jj)
          for (int l = lf + warp; l < lown; l += NWARP) {
            const double v = Vl[jj * nloc + l];
            sv += Vl[lane * nloc + l] * v;
            sw += Wl[lane * nloc + l] * v;
          }
        vw_part[warp * 2 * PNB_MAX + lane] = sv;
        vw_part[warp * 2 * PNB_MAX + PNB_MAX + lane] = sw;
        __syncthreads();
        if (tid < 2 * PNB_MAX) {
          const int t = tid & (PNB_MAX - 1);
          if (t < jj) {
            double a = 0.0;
            for (int w = 0; w < NWARP; ++w) a += vw_part[w * 2 * PNB_MAX + tid];
            const int slot = rank * 2 * nb + (tid < PNB_MAX ? t : nb + t);
            for (int q = 0; q < CL; ++q) *cluster.map_shared_rank(r2 + slot, q) = a;
          }
        }
      }
      // ---- 3: p = A22 v from the lower triangle of the own columns ----
      if (jj + 1 < nbe)  // the next column's own rows: unchanged until its step 1
        for (int l = lf + tid; l < lown; l += blockDim.x)
          xc[((jj + 1) & 1) * nloc + l] = Gp[(rank + CL * l) + (int64_t)n * (j + 1)];
      double kp = 0.0;  // this thread's share of v^T A22 v
      if (tau != 0.0) {
        for (int l = lf + lane; l < lown; l += 32) dw[warp * nloc + l] = 0.0;
        __syncwarp();
        // blocks of 64 rows from row j + 1, two rows per lane (i0 = rb + lane,
        // i1 = i0 + 32); the longest (last) blocks are dealt first and back and
        // forth, so the warps' shares come out even
        const int nrb = (n - j - 1 + 63) / 64;
        const int64_t cstep = (int64_t)n * CL;  // from one own column to the next
        for (int round = 0; round * NWARP < nrb; ++round) {
          const int o = round * NWARP + ((round & 1) ? NWARP - 1 - warp : warp);
          if (o >= nrb) continue;
          const int rb = j + 1 + 64 * (nrb - 1 - o);
          const int i0 = rb + lane, i1 = i0 + 32;
          const double v0 = i0 < n ? xo[om(i0)] : 0.0, v1 = i1 < n ? xo[om(i1)] : 0.0;
          // rows past the end read row n - 1 (weighted by v = 0, sums discarded)
          const double* g0 = Gp + min(i0, n - 1) + (int64_t)n * rank;
          const double* g1 = Gp + min(i1, n - 1) + (int64_t)n * rank;
          const int le = first_owned(min(n, rb + 64), rank, CL);  // own columns c < the block's end
          const int lfull = min(le, first_owned(rb, rank, CL));   // own columns c < rb: no masking
          double y0 = 0.0, y1 = 0.0;
          int lt = lf;
          for (; lt + 16 <= lfull; lt += 16) {
            double acc[16];
#pragma unroll
            for (int h = 0; h < 16; h += 8) {  // eight columns' loads in flight at a time
              double a0[8], a1[8];
#pragma unroll
              for (int k = 0; k < 8; ++k) {
                a0[k] = g0[(lt + h + k) * cstep];
                a1[k] = g1[(lt + h + k) * cstep];
              }
#pragma unroll
              for (int k = 0; k < 8; ++k) {
                const double vc = xo[rank * nloc + lt + h + k];
                y0 = fma(a0[k], vc, y0);
                y1 = fma(a1[k], vc, y1);
                acc[h + k] = fma(a1[k], v1, a0[k] * v0);
              }
            }
            const double d = warp_reduce_scatter16(acc, lane);
            if (lane < 16) dw[warp * nloc + lt + lane] += d;
          }
          for (; lt < le; lt += 16) {  // the rest, masked: the block's diagonal part and a short tail
            double acc[16];
#pragma unroll
            for (int h = 0; h < 16; h += 8) {
              double a0[8], a1[8];
#pragma unroll
              for (int k = 0; k < 8; ++k) {
                const int c = rank + CL * (lt + h + k);
                const bool cv = lt + h + k < le;
                a0[k] = cv && i0 >= c ? g0[(lt + h + k) * cstep] : 0.0;
                a1[k] = cv && i1 >= c ? g1[(lt + h + k) * cstep] : 0.0;
              }
#pragma unroll
              for (int k = 0; k < 8; ++k) {
                const int c = rank + CL * (lt + h + k);
                const double vc = lt + h + k < le ? xo[rank * nloc + lt + h + k] : 0.0;
                y0 = fma(i0 > c ? a0[k] : 0.0, vc, y0);
                y1 = fma(i1 > c ? a1[k] : 0.0, vc, y1);
                acc[h + k] = fma(a1[k], v1, a0[k] * v0);
              }
            }
            const double d = warp_reduce_scatter16(acc, lane);
            if (lane < 16 && lt + lane < le) dw[warp * nloc + lt + lane] += d;
          }
          if (i0 < n) {
            yl[om(i0)] = y0;
            kp += v0 * y0;
          }
          if (i1 < n) {
            yl[om(i1)] = y1;
            kp += v1 * y1;
          }
        }
      }
      __syncthreads();
      if (tau != 0.0) {
        // the row sums to their owners (rows below j + 1 and beyond n ride
        // along unread), those of the panel's rows to every CTA
        const int lmin = (j + 1) >> lg, cnt = nloc - lmin;
        for (int e = tid; e < CL * cnt; e += blockDim.x) {
          const int d = e / cnt, l = lmin + e % cnt;
          *cluster.map_shared_rank(yb + rank * nloc + l, d) = yl[d * nloc + l];
        }
        for (int e = tid; e < CL * nb; e += blockDim.x) {
          const int q = e / nb, s = e % nb, row = k0 + s;
          if (row >= j + 1 && row < n) *cluster.map_shared_rank(yp + rank * nb + s, q) = yl[om(row)];
        }
      }
      if (tau != 0.0)
        for (int l = lf + tid; l < lown; l += blockDim.x) {
          double d = 0.0;
          for (int w = 0; w < NWARP; ++w) d += dw[w * nloc + l];
          dw[l] = d;  // the column's dot, kept in warp 0's row
          const int c = rank + CL * l;
          kp += xo[rank * nloc + l] * d;
          if (c < k0 + nb)
            for (int q = 0; q < CL; ++q) *cluster.map_shared_rank(dp + (c - k0), q) = d;
        }
      const double vav_part = block_reduce(kp, red, false);
      if (tid < CL) *cluster.map_shared_rank(r3 + rank, tid) = vav_part;
      cluster.sync();  // B
      // ---- 4: w on the own rows and on the panel's rows ----
      if (warp == 0) {  // V^T v, W^T v and the scalar K = (tau/2) w'.v, one lane per panel column
        double a = 0.0, b = 0.0;
        if (lane < jj)
          for (int q = 0; q < CL; ++q) {
            a += r2[q * 2 * nb + lane];
            b += r2[q * 2 * nb + nb + lane];
          }
        if (lane < jj) {
          cvt[lane] = a;
          cwt[lane] = b;
        }
        const double cc = warp_sum(a * b);
        if (lane == 0) {
          double vav = 0.0;
          for (int q = 0; q < CL; ++q) vav += r3[q];
          s_K = 0.5 * tau * tau * (vav - 2.0 * cc);
        }
      }
      __syncthreads();
      if (tau != 0.0) {
        const double K = s_K;
        // own rows: four threads per row, each summing a quarter of the terms
        // (the loop bound is the same for the whole warp: the shuffles need it)
        const int sub = tid & 3;
        for (int base = lf + (warp << 3); base < lown; base += blockDim.x >> 2) {
          const int l = base + (lane >> 2);
          const bool act = l < lown;
          double p = 0.0, corr = 0.0;
          if (act) {
#pragma unroll 1
            for (int q = sub; q < CL; q += 4) p += yb[q * nloc + l];
#pragma unroll 1
            for (int t = sub; t < jj; t += 4) corr += Vl[t * nloc + l] * cwt[t] + Wl[t * nloc + l] * cvt[t];
          }
          p += __shfl_xor_sync(0xffffffffu, p, 1);
          p += __shfl_xor_sync(0xffffffffu, p, 2);
          corr += __shfl_xor_sync(0xffffffffu, corr, 1);
          corr += __shfl_xor_sync(0xffffffffu, corr, 2);
          if (act && sub == 0) Wl[jj * nloc + l] = tau * (dw[l] + p - corr) - K * Vl[jj * nloc + l];
        }
        // the panel's rows: sixteen threads per row
        const int s = tid >> 4, sub16 = tid & 15;
        if (s < nb) {
          const int row = k0 + s;
          const bool live = row >= j + 1 && row < n;
          double p = 0.0, corr = 0.0;
          if (live) {
            for (int q = sub16; q < CL; q += 16) p += yp[q * nb + s];
            for (int t = sub16; t < jj; t += 16) corr += Vp[t * nb + s] * cwt[t] + Wq[t * nb + s] * cvt[t];
          }
#pragma unroll
          for (int o = 1; o < 16; o <<= 1) {
            p += __shfl_xor_sync(0xffffffffu, p, o);
            corr += __shfl_xor_sync(0xffffffffu, corr, o);
          }
          if (sub16 == 0) Wq[jj * nb + s] = live ? tau * (dp[s] + p - corr) - K * Vp[jj * nb + s] : 0.0;
        }
      } else {
        for (int s = tid; s < nb; s += blockDim.x) Wq[jj * nb + s] = 0.0;
      }
      __syncthreads();
    }
    // ---- trailing update A[k1:, k1:] -= V W^T + W V^T (lower triangle) through the global scratch ----
    const int k1 = k0 + nbe;
    for (int e = tid; e < lown * 2 * nbe; e += blockDim.x) {
      const int l = e / (2 * nbe), t2 = e - l * 2 * nbe;
      const int i = rank + CL * l;
      if (i < k1) continue;
      const int t = t2 < nbe ? t2 : t2 - nbe;
      VW[(int64_t)i * 2 * nb + (t2 < nbe ? t : nb + t)] = (t2 < nbe ? Vl : Wl)[t * nloc + l];
    }
    __threadfence();
    cluster.sync();
    // DMMA (m8n8k4 f64) tiles: a warp takes 32 rows x 16 own columns and runs
    // P = V W^T + W V^T over the panel's k, the rows' [V W] fragments read
    // straight from the scratch (no shared staging, no barrier per tile); the
    // lower triangle of its block then receives A -= P
    const int lf = first_owned(k1, rank, CL);
    const int nbe4 = (nbe + 3) & ~3;
    const int gr = lane >> 2, gk = lane & 3;
    const int nrt = (n - k1 + 31) >> 5;                 // 32-row tiles
    const int ncb = (first_owned(n, rank, CL) - lf + 15) >> 4;  // 16-column blocks
    for (int task = warp; task < nrt * ncb; task += NWARP) {
      const int i0 = k1 + 32 * (task / ncb), lb = lf + 16 * (task % ncb);
      if (rank + CL * lb > i0 + 31) continue;  // the block lies above the diagonal
      const int le = min(first_owned(min(n, i0 + 32), rank, CL), lb + 16);
      double acc[4][2][2];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
#pragma unroll
      for (int part = 0; part < 2; ++part) {
        // part 0: V (rows) x W (columns); part 1: W x V
        const int xo0 = part ? nb : 0;
        const double* Y = part ? Vl : Wl;
#pragma unroll 1
        for (int t = 0; t < nbe4; t += 4) {
          const int k = t + gk;
          const bool kv = k < nbe;
          double af[4], bf[2];
#pragma unroll
          for (int a = 0; a < 4; ++a) {
            const int i = i0 + 8 * a + gr;
            af[a] = kv && i < n ? VW[(int64_t)i * 2 * nb + xo0 + k] : 0.0;
          }
#pragma unroll
          for (int b = 0; b < 2; ++b) {
            const int l = lb + 8 * b + gr;
            bf[b] = kv && l < le ? Y[k * nloc + l] : 0.0;
          }
#pragma unroll
          for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) dmma_tr(acc[a][b], af[a], bf[b]);
        }
      }
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        const int i = i0 + 8 * a + gr;
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const int l = lb + 8 * b + 2 * gk + e;
            const int c = rank + CL * l;
            if (i < n && l < le && i >= c) Gp[(int64_t)n * c + i] -= acc[a][b][e];
          }
      }
    }
    __threadfence();
    cluster.sync();
  }
  // T: the last two diagonal entries and the last off-diagonal A[n-1, n-2]
  if (tid == 0) {
    if (rank == (n - 2) % CL) {
      dg[n - 2] = Gp[(n - 2) + (int64_t)n * (n - 2)];
      eg[n - 2] = Gp[(n - 1) + (int64_t)n * (n - 2)];
    }
    if (rank == (n - 1) % CL) dg[n - 1] = Gp[(n - 1) + (int64_t)n * (n - 1)];
    if (rank == 0) {
      eg[n - 1] = 0.0;
      tg[n - 1] = 0.0;
      tg[n - 2] = 0.0;
    }
  }
  __threadfence();
  cluster.sync();  // also the last access of another CTA's shared memory
}

// Bisection for the cluster-sized sectors after their tridiagonalisation,
// spread over the GPU: a CTA of BS_THREADS threads takes BS_PER eigenvalues
// of one problem, with the problem's d and e^2 in shared memory.  Sixteen
// lanes serve one eigenvalue: in a round they count at the 15 points that
// four successive halvings of the current interval can probe (the nodes of a
// four-level bisection tree, each computed by the same chain of midpoints
// that plain bisection would compute), then every lane of the group walks
// the tree with the shared counts.  The intervals, the stopping rule and so
// the eigenvalues are bit for bit those of plain bisection; a round advances
// four halvings instead of one, so an eigenvalue takes about 13 rounds of
// Sturm chains instead of 50.
constexpr int BS_THREADS = 128;
constexpr int BS_LANES = 16;  // lanes per eigenvalue: 15 probes, one idle
constexpr int BS_LEVELS = 4;  // halvings per round
constexpr int BS_PER = BS_THREADS / BS_LANES;

__global__ void __launch_bounds__(BS_THREADS)
bisect_sectors(const EigDev* __restrict__ probs, const VecTaskB* __restrict__ tasks, const double* Tg, double* W) {
  extern __shared__ double bs_sm[];
  __shared__ double red[33];
  const VecTaskB tk = tasks[blockIdx.x];
  const EigDev P = probs[tk.prob];
  const int n = P.n;
  const double* dg = Tg + 3 * P.w_off;
  const double* eg = dg + n;
  double* Wp = W + P.w_off;
  const int tid = threadIdx.x, lane = tid & 31;
  double* d = bs_sm;
  double* e2 = bs_sm + n;
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
    for (int j = tk.j0 + tid; j < min(n, tk.j0 + BS_PER); j += blockDim.x) Wp[n - 1 - j] = 0.0;
    return;
  }
  auto open_interval = [&](double lo, double hi) {
    return hi - lo > fmax(atol, 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)));
  };
  const int sub = lane & (BS_LANES - 1);          // this lane's tree node: in-order position sub + 1
  const int base = lane & ~(BS_LANES - 1);        // first lane of the group
  const int j = tk.j0 + tid / BS_LANES;
  const bool active = j < n;
  constexpr int ROOT = 1 << (BS_LEVELS - 1);      // in-order position of the root (8)
  double lo = gl - atol, hi = gu + atol;
  int it = 0;
  bool work = active && open_interval(lo, hi);
  while (__any_sync(0xffffffffu, work)) {
    int c = 0;
    if (work && sub < 2 * ROOT - 1) {
      // descend from the round's interval to node sub + 1 by midpoints
      const int p = sub + 1;
      double a = lo, b = hi;
      int pos = ROOT, half = ROOT >> 1;
      while (pos != p) {
        const double m = 0.5 * (a + b);
        if (p < pos) { b = m; pos -= half; } else { a = m; pos += half; }
        half >>= 1;
      }
      c = sturm_count(d, e2, n, 0.5 * (a + b), pivmin);
    }
    // every lane of the group walks the same path with the group's counts
    int pos = ROOT, half = ROOT >> 1;
    bool go = work;
#pragma unroll
    for (int lev = 0; lev < BS_LEVELS; ++lev) {
      const int cp = __shfl_sync(0xffffffffu, c, base + pos - 1);
      go = go && it < 128 && open_interval(lo, hi);
      if (go) {
        const double mid = 0.5 * (lo + hi);
        if (cp > j) { hi = mid; pos -= half; } else { lo = mid; pos += half; }
        half >>= 1;
        ++it;
      }
    }
    if (work) work = it < 128 && open_interval(lo, hi);
  }
  if (active && sub == 0) Wp[n - 1 - j] = 0.5 * (lo + hi);
}

__global__ void __launch_bounds__(TT)
tridiag_eigvecs_cluster(const EigDev* __restrict__ probs, const double* G, const double* Tg, const double* W,
                        double* Zg, double* work, int cap, const int* __restrict__ only_flagged) {
  extern __shared__ double zsm[];
  __shared__ double red[33];
  __shared__ double coef[MAX_N / 2];
  __shared__ int cstart[MAX_N / 2];
  cgx::cluster_group cluster = cgx::this_cluster();
  const int CL = (int)cluster.num_blocks();
  const int rank = (int)cluster.block_rank();
  // as the fallback of the blocked path: only the problems it flagged (the
  // whole cluster returns alike, before any barrier)
  if (only_flagged && only_flagged[blockIdx.x / CL] == 0) return;
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

// ---------------------------------------------------------------------------
// Eigenvectors of the cluster-sized sectors, across the whole GPU.
//
// (1) inverse iteration, one thread per wanted vector (same start vectors and
//     solves as the kernels above);
// (2) CholeskyQR2 (Fukaya et al., "CholeskyQR2: a simple and communication-
//     avoiding algorithm", 2014): G = Z^T Z, G = L L^T, Z <- Z L^-T, twice.
//     In exact arithmetic this is Gram-Schmidt in column (descending
//     eigenvalue) order, i.e. what the kernels above do inside clusters of
//     close eigenvalues; against the other vectors it only removes components
//     of the size of their orthogonality error.  A pivot L_jj below 1e-4 in
//     the first pass means vector j had collapsed onto earlier ones (its
//     orthonormalised form would carry a residual of eps ||T|| / L_jj): the
//     problem is flagged and the cluster kernel above, which re-iterates such
//     vectors, redoes it from the start;
// (3) back-transformation z = Q y with the reflectors grouped 32 at a time in
//     the compact WY form Q_p = I - V T V^T (LAPACK dlarft, forward and
//     columnwise), then the deterministic gauge.
// Every launch is batched over the problems; (1)-(3) use as many CTAs as
// there are vectors, rows or tiles.
constexpr int IV_THREADS = 128;   // vectors per CTA of the inverse iteration
constexpr int GT = 64;            // Gram tile
constexpr int CH_PB = 32;         // Cholesky panel
constexpr int TS_ROWS = 32;       // rows per CTA of the triangular solve
constexpr int BT_NB = 32;         // reflectors per compact-WY panel
constexpr int BT_VB = 16;         // vectors per CTA of the back-transformation
constexpr int BT_ROWS = 64;       // row chunk of the back-transformation
constexpr double COLLAPSE_PIVOT2 = 1e-8;  // L_jj^2 below this: collapsed vector
__device__ unsigned long long g_eig_redo;  // problems whose vectors the cluster kernel redid (device-wide)

struct VecTask {
  int32_t prob, j0;  // problem (index into the problem array) and first item
};
struct TileTask {
  int32_t prob, a, b;  // problem and tile / panel coordinates
};

__device__ double tnorm1(const double* d, const double* e, int n, double* red) {
  double loc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    loc = fmax(loc, fabs(d[i]) + (i > 0 ? fabs(e[i - 1]) : 0.0) + (i + 1 < n ? fabs(e[i]) : 0.0));
  return block_reduce(loc, red, true);
}

// (1) inverse iteration: thread t of task (p, j0) computes vector j0 + t
__global__ void __launch_bounds__(IV_THREADS)
inv_iter_batched(const EigDev* __restrict__ probs, const VecTask* __restrict__ tasks, const double* Tg,
                 const double* W, double* Zg, double* work) {
  __shared__ double red[33];
  const VecTask tk = tasks[blockIdx.x];
  const EigDev P = probs[tk.prob];
  const int n = P.n;
  const double* d = Tg + 3 * P.w_off;
  const double* e = d + n;
  const double* lam = W + P.w_off;
  const double tnorm = tnorm1(d, e, n, red);
  const double tiny = tnorm > 1e-250 ? fmax(DBL_EPSILON * tnorm, DBL_MIN) : 1.0;
  const int t = threadIdx.x, j = tk.j0 + t;
  const int cnt = min(IV_THREADS, P.nvec - tk.j0);  // vectors of this CTA
  const bool active = t < cnt;  // no early return: the barrier below needs every thread
  // the CTA's iterates and LU factors interleaved (element i of its vector t
  // at [i cnt + t]), so that the threads' accesses coalesce: the iterates and
  // two factor rows in the problem's work area (3 n cnt doubles from
  // work + 3 g_off + 3 n j0), the third factor row in the CTA's own columns
  // of Z (n cnt doubles), which receive the vectors at the end
  double* wb = work + 3 * P.g_off + (int64_t)3 * n * tk.j0;
  double* zb = Zg + P.g_off + (int64_t)n * tk.j0;
  double* y = wb + t;
  const int64_t nc = (int64_t)n * cnt;
  // each iterate's normalisation is applied as the next solve (or the final
  // copy) reads it; its norm is summed in the solve's back substitution
  double inv = 1.0;
  if (active) {
    for (int i = 0; i < n; ++i)
      y[(int64_t)i * cnt] = hash_unit(((uint64_t)P.g_off << 20) ^ ((uint64_t)j << 32) ^ (uint64_t)i);
    for (int it = 0; it < INV_ITERS; ++it) {
      const double s = tri_solve_il(d, e, n, lam[j], tiny, inv, y, wb + nc + t, wb + 2 * nc + t, zb + t, cnt);
      inv = 1.0 / sqrt(s);
    }
  }
  __syncthreads();  // every thread's third factor row in Z is dead
  if (active) {
    double* z = zb + (int64_t)n * t;
    int i = 0;
    for (; i + PF <= n; i += PF) {
      double v[PF];
#pragma unroll
      for (int k = 0; k < PF; ++k) v[k] = y[(int64_t)(i + k) * cnt];
#pragma unroll
      for (int k = 0; k < PF; ++k) z[i + k] = v[k] * inv;
    }
    for (; i < n; ++i) z[i] = y[(int64_t)i * cnt] * inv;
  }
}

// (2a) Gram matrix, lower 64 x 64 tiles (a >= b): G[r + m c] = sum_i Z[i, r] Z[i, c],
// G at work + 3 g_off, leading dimension m = nvec; 256 threads, 4 x 4 outputs each
__global__ void __launch_bounds__(256)
gram_tiles(const EigDev* __restrict__ probs, const TileTask* __restrict__ tasks, const double* Zg, double* work,
           const int* __restrict__ flags) {
  __shared__ double sa[16][GT + 2], sb[16][GT + 2];
  const TileTask tk = tasks[blockIdx.x];
  if (flags[tk.prob]) return;
  const EigDev P = probs[tk.prob];
  const int n = P.n, m = P.nvec;
  const double* Z = Zg + P.g_off;
  double* Gm = work + 3 * P.g_off;
  const int r0 = tk.a * GT, c0 = tk.b * GT;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[4][4] = {};
  for (int i0 = 0; i0 < n; i0 += 16) {
    __syncthreads();
    for (int e2 = threadIdx.x; e2 < 16 * GT; e2 += blockDim.x) {
      const int rr = e2 & 15, cc = e2 >> 4;
      const int i = i0 + rr;
      sa[rr][cc] = (i < n && r0 + cc < m) ? Z[i + (int64_t)n * (r0 + cc)] : 0.0;
      sb[rr][cc] = (i < n && c0 + cc < m) ? Z[i + (int64_t)n * (c0 + cc)] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      double av[4], bv[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        av[u] = sa[k][tx * 4 + u];
        bv[u] = sb[k][ty * 4 + u];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int w = 0; w < 4; ++w) acc[u][w] += av[u] * bv[w];
    }
  }
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int w = 0; w < 4; ++w) {
      const int r = r0 + tx * 4 + u, c = c0 + ty * 4 + w;
      if (r < m && c < m && r >= c) Gm[r + (int64_t)m * c] = acc[u][w];
    }
}

// (2b) Cholesky G = L L^T of the lower triangle in place, right-looking with
// 32-column panels, one cluster per problem: CTA 0 factors the diagonal
// block, every CTA solves its share of the panel's rows, the trailing tiles
// are dealt out to the CTAs.  Pivots below COLLAPSE_PIVOT2 (first pass)
// flag the problem; a flagged or non-positive pivot is replaced by 1 so the
// arithmetic stays finite (the problem is redone by the fallback).
__global__ void __launch_bounds__(TT)
chol_cluster(const EigDev* __restrict__ probs, double* work, int* flags, int check) {
  __shared__ double Ld[CH_PB][CH_PB + 1];
  __shared__ double tl[2][GT][CH_PB + 1];
  __shared__ int s_flag;
  cgx::cluster_group cluster = cgx::this_cluster();
  const int CL = (int)cluster.num_blocks();
  const int rank = (int)cluster.block_rank();
  const int pi = blockIdx.x / CL;
  if (flags[pi]) return;  // the whole cluster alike
  const EigDev P = probs[pi];
  const int m = P.nvec;
  double* A = work + 3 * P.g_off;
  const int tid = threadIdx.x;
  for (int p0 = 0; p0 < m; p0 += CH_PB) {
    const int pb = min(CH_PB, m - p0);
    // (i) the diagonal block, every CTA (identical arithmetic; only CTA 0 writes)
    for (int e2 = tid; e2 < pb * pb; e2 += blockDim.x) {
      const int r = e2 % pb, c = e2 / pb;
      Ld[r][c] = r >= c ? A[(p0 + r) + (int64_t)m * (p0 + c)] : 0.0;
    }
    if (tid == 0) s_flag = 0;
    __syncthreads();
    for (int k = 0; k < pb; ++k) {
      if (tid == 0) {
        double dk = Ld[k][k];
        if (!(dk > (check ? COLLAPSE_PIVOT2 : 0.0))) {
          s_flag = 1;
          dk = 1.0;
        }
        Ld[k][k] = sqrt(dk);
      }
      __syncthreads();
      const double piv = Ld[k][k];
      for (int r = k + 1 + tid; r < pb; r += blockDim.x) Ld[r][k] /= piv;
      __syncthreads();
      for (int e2 = tid; e2 < pb * pb; e2 += blockDim.x) {
        const int r = e2 % pb, c = e2 / pb;
        if (c > k && r >= c) Ld[r][c] -= Ld[r][k] * Ld[c][k];
      }
      __syncthreads();
    }
    if (rank == 0) {
      for (int e2 = tid; e2 < pb * pb; e2 += blockDim.x) {
        const int r = e2 % pb, c = e2 / pb;
        if (r >= c) A[(p0 + r) + (int64_t)m * (p0 + c)] = Ld[r][c];
      }
      if (tid == 0 && s_flag && atomicExch(&flags[pi], 1) == 0) atomicAdd(&g_eig_redo, 1ull);
    }
    // (ii) rows below the block: L[i, p0:p0+pb] = A[i, p0:p0+pb] L_pp^-T
    const int rbeg = p0 + pb;
    for (int i = rbeg + rank * (int)blockDim.x + tid; i < m; i += CL * (int)blockDim.x) {
      double x[CH_PB];
#pragma unroll
      for (int k = 0; k < CH_PB; ++k) x[k] = k < pb ? A[i + (int64_t)m * (p0 + k)] : 0.0;  // all loads in flight
#pragma unroll
      for (int k = 0; k < CH_PB; ++k) {
        if (k < pb) {
          double v = x[k];
          for (int t = 0; t < k; ++t) v -= x[t] * Ld[k][t];
          x[k] = v / Ld[k][k];
          A[i + (int64_t)m * (p0 + k)] = x[k];
        }
      }
    }
    __threadfence();
    cluster.sync();
    // (iii) trailing update of the lower tiles (a >= b) of A[rbeg:, rbeg:]
    const int nt = (m - rbeg + GT - 1) / GT;
    const int ntiles = nt * (nt + 1) / 2;
    for (int t = rank; t < ntiles; t += CL) {
      int ta = 0;
      while ((ta + 1) * (ta + 2) / 2 <= t) ++ta;
      const int tb = t - ta * (ta + 1) / 2;
      const int ra = rbeg + ta * GT, rb = rbeg + tb * GT;
      __syncthreads();
      for (int e2 = tid; e2 < GT * pb; e2 += blockDim.x) {
        const int r = e2 % GT, k = e2 / GT;
        tl[0][r][k] = ra + r < m ? A[(ra + r) + (int64_t)m * (p0 + k)] : 0.0;
        tl[1][r][k] = rb + r < m ? A[(rb + r) + (int64_t)m * (p0 + k)] : 0.0;
      }
      __syncthreads();
      for (int e2 = tid; e2 < GT * GT; e2 += blockDim.x) {
        const int r = e2 % GT, c = e2 / GT;
        const int gi = ra + r, gj = rb + c;
        if (gi < m && gj < m && gi >= gj) {
          double acc = 0.0;
          for (int k = 0; k < pb; ++k) acc += tl[0][r][k] * tl[1][c][k];
          A[gi + (int64_t)m * gj] -= acc;
        }
      }
    }
    __threadfence();
    cluster.sync();
  }
}

// (2c) Z <- Z L^-T, row by row (rows are independent): TS_ROWS rows per CTA,
// columns in 32-wide panels: the solved part enters through a small GEMM,
// the panel's own triangle by substitution
__global__ void __launch_bounds__(256)
trsm_rows(const EigDev* __restrict__ probs, const VecTask* __restrict__ tasks, double* Zg, const double* work,
          const int* __restrict__ flags) {
  __shared__ double sx[TS_ROWS][CH_PB + 1];   // solved values, one 32-column chunk
  __shared__ double sl[CH_PB][CH_PB + 1];     // L rows of the panel, one 32-column chunk
  __shared__ double acc_s[TS_ROWS][CH_PB + 1];
  const VecTask tk = tasks[blockIdx.x];
  if (flags[tk.prob]) return;
  const EigDev P = probs[tk.prob];
  const int n = P.n, m = P.nvec;
  double* Z = Zg + P.g_off;
  const double* L = work + 3 * P.g_off;
  const int i0 = tk.j0;
  const int tid = threadIdx.x;
  const int r = tid & 31, cg = tid >> 5;  // row in the block, column group of 4
  // the chunks of Z (TS_ROWS x CH_PB) and L (CH_PB x CH_PB) are staged
  // through registers one chunk ahead of the one in shared memory
  constexpr int PER = TS_ROWS * CH_PB / 256;
  static_assert(PER * 256 == TS_ROWS * CH_PB && TS_ROWS == CH_PB, "chunk split");
  auto load = [&](int p0, int pb, int k0, double (&rx)[PER], double (&rl)[PER]) {
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const int e2 = tid + 256 * q, rr = e2 % TS_ROWS, kk = e2 / TS_ROWS;
      rx[q] = i0 + rr < n ? Z[(i0 + rr) + (int64_t)n * (k0 + kk)] : 0.0;
      rl[q] = rr < pb ? L[(p0 + rr) + (int64_t)m * (k0 + kk)] : 0.0;
    }
  };
  for (int p0 = 0; p0 < m; p0 += CH_PB) {
    const int pb = min(CH_PB, m - p0);
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    double rx[PER], rl[PER];
    if (p0 > 0) load(p0, pb, 0, rx, rl);
    for (int k0 = 0; k0 < p0; k0 += CH_PB) {
      __syncthreads();
#pragma unroll
      for (int q = 0; q < PER; ++q) {
        const int e2 = tid + 256 * q, rr = e2 % TS_ROWS, kk = e2 / TS_ROWS;
        sx[rr][kk] = rx[q];
        sl[rr][kk] = rl[q];
      }
      if (k0 + CH_PB < p0) load(p0, pb, k0 + CH_PB, rx, rl);
      __syncthreads();
#pragma unroll 8
      for (int kk = 0; kk < CH_PB; ++kk) {
        const double xv = sx[r][kk];
#pragma unroll
        for (int u = 0; u < 4; ++u) acc[u] += xv * sl[cg * 4 + u][kk];
      }
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < 4; ++u) acc_s[r][cg * 4 + u] = acc[u];
    for (int e2 = tid; e2 < CH_PB * CH_PB; e2 += blockDim.x) {
      const int lr = e2 % CH_PB, lk = e2 / CH_PB;
      sl[lr][lk] = (lr < pb && lk <= lr) ? L[(p0 + lr) + (int64_t)m * (p0 + lk)] : 0.0;
    }
    __syncthreads();
    if (tid < TS_ROWS && i0 + tid < n) {
      double x[CH_PB];
      double* zr = Z + (i0 + tid);
#pragma unroll
      for (int c = 0; c < CH_PB; ++c) {
        if (c < pb) {
          double v = zr[(int64_t)n * (p0 + c)] - acc_s[tid][c];
          for (int t = 0; t < c; ++t) v -= x[t] * sl[c][t];
          x[c] = v / sl[c][c];
          zr[(int64_t)n * (p0 + c)] = x[c];
        }
      }
    }
  }
}

// (3a) compact-WY factor T of the reflectors [32 b, 32 b + 32) of a problem:
// S = V^T V (v_k(k+1) = 1, v_k(i) = G(i, k) for i >= k + 2), then the dlarft
// recurrence T(0:c, c) = -tau_c T(0:c, 0:c) S(0:c, c), T(c, c) = tau_c
__global__ void __launch_bounds__(256)
wy_factors(const EigDev* __restrict__ probs, const TileTask* __restrict__ tasks, const double* G, const double* Tg,
           double* work, const int* __restrict__ flags) {
  __shared__ double S[BT_NB][BT_NB + 1];
  __shared__ double T[BT_NB][BT_NB + 1];
  const TileTask tk = tasks[blockIdx.x];
  if (flags[tk.prob]) return;
  const EigDev P = probs[tk.prob];
  const int n = P.n;
  const double* Gp = G + P.g_off;
  const double* tau = Tg + 3 * P.w_off + 2 * n;
  const int k0 = tk.a * BT_NB, mm = min(BT_NB, n - 2 - k0);
  double* Tout = work + 3 * P.g_off + (int64_t)P.nvec * P.nvec + (int64_t)tk.a * BT_NB * BT_NB;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  // S(a, c), a < c: v_a . v_c over rows >= k0 + c + 1 (v_c vanishes above)
  for (int pr = warp; pr < mm * mm; pr += nw) {
    const int a = pr % mm, c = pr / mm;
    if (a >= c) continue;
    const int ka = k0 + a, kc = k0 + c;
    double acc = 0.0;
    for (int i = kc + 1 + lane; i < n; i += 32) {
      const double va = (i == ka + 1) ? 1.0 : Gp[i + (int64_t)n * ka];
      const double vc = (i == kc + 1) ? 1.0 : Gp[i + (int64_t)n * kc];
      acc += va * vc;
    }
    acc = warp_sum(acc);
    if (lane == 0) S[a][c] = acc;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    for (int c = 0; c < mm; ++c) {
      const double tc = tau[k0 + c];
      // T(a, c) = -tc * sum_{b in [a, c)} T(a, b) S(b, c), lanes over a
      double x = 0.0;
      if (lane < c) {
        for (int b = lane; b < c; ++b) x += T[lane][b] * S[b][c];
        T[lane][c] = -tc * x;
      }
      if (lane == 0) T[c][c] = tc;
      __syncwarp();
    }
  }
  __syncthreads();
  for (int e2 = threadIdx.x; e2 < BT_NB * BT_NB; e2 += blockDim.x) {
    const int a = e2 % BT_NB, c = e2 / BT_NB;
    Tout[e2] = (a < mm && c < mm && a <= c) ? T[a][c] : 0.0;
  }
}

// (3b) z = Q y for the vectors [j0, j0 + BT_VB) of a problem: panels last to
// first, Y <- Y - V (T (V^T Y)) over rows >= k0 + 1; then the gauge (largest
// magnitude entry positive, first on ties)
__global__ void __launch_bounds__(512)
wy_apply(const EigDev* __restrict__ probs, const VecTask* __restrict__ tasks, const double* G, double* Zg,
         const double* work, const int* __restrict__ flags) {
  __shared__ double sv[BT_ROWS][BT_NB + 1];
  __shared__ double sy[BT_ROWS][BT_VB + 1];
  __shared__ double X[BT_NB][BT_VB + 1];
  __shared__ double X2[BT_NB][BT_VB + 1];
  __shared__ double Tm[BT_NB][BT_NB + 1];
  const VecTask tk = tasks[blockIdx.x];
  if (flags[tk.prob]) return;
  const EigDev P = probs[tk.prob];
  const int n = P.n, nv = min(BT_VB, P.nvec - tk.j0);
  const double* Gp = G + P.g_off;
  double* Y = Zg + P.g_off + (int64_t)n * tk.j0;
  const double* Tst = work + 3 * P.g_off + (int64_t)P.nvec * P.nvec;
  const int tid = threadIdx.x;
  const int npan = (n - 2 + BT_NB - 1) / BT_NB;
  const int xa = tid / BT_VB, xc = tid % BT_VB;  // the (reflector, vector) entry of X this thread sums
  // Row chunks of V (BT_ROWS x BT_NB) and Y (BT_ROWS x BT_VB) are staged through
  // registers one chunk ahead of the one in shared memory, so the global loads
  // of chunk c + 1 are in flight while chunk c is being used.
  constexpr int NV_PER = BT_ROWS * BT_NB / 512, NY_PER = BT_ROWS * BT_VB / 512;
  static_assert(NV_PER * 512 == BT_ROWS * BT_NB && NY_PER * 512 == BT_ROWS * BT_VB, "chunk split");
  auto load_v = [&](int k0, int mm, int i0, double (&rv)[NV_PER]) {
#pragma unroll
    for (int q = 0; q < NV_PER; ++q) {
      const int e2 = tid + 512 * q, rr = e2 % BT_ROWS, a = e2 / BT_ROWS;
      const int i = i0 + rr, ka = k0 + a;
      rv[q] = (a < mm && i < n && i >= ka + 1) ? ((i == ka + 1) ? 1.0 : Gp[i + (int64_t)n * ka]) : 0.0;
    }
  };
  auto load_y = [&](int i0, double (&ry)[NY_PER]) {
#pragma unroll
    for (int q = 0; q < NY_PER; ++q) {
      const int e2 = tid + 512 * q, rr = e2 % BT_ROWS, c = e2 / BT_ROWS;
      ry[q] = (i0 + rr < n && c < nv) ? Y[(i0 + rr) + (int64_t)n * c] : 0.0;
    }
  };
  for (int pnl = npan - 1; pnl >= 0; --pnl) {
    const int k0 = pnl * BT_NB, mm = min(BT_NB, n - 2 - k0);
    __syncthreads();
    for (int e2 = tid; e2 < BT_NB * BT_NB; e2 += blockDim.x) Tm[e2 % BT_NB][e2 / BT_NB] = Tst[(int64_t)pnl * BT_NB * BT_NB + e2];
    double xs = 0.0;
    double rv[NV_PER], ry[NY_PER];
    // X = V^T Y over rows >= k0 + 1
    load_v(k0, mm, k0 + 1, rv);
    load_y(k0 + 1, ry);
    for (int i0 = k0 + 1; i0 < n; i0 += BT_ROWS) {
      __syncthreads();
#pragma unroll
      for (int q = 0; q < NV_PER; ++q) sv[(tid + 512 * q) % BT_ROWS][(tid + 512 * q) / BT_ROWS] = rv[q];
#pragma unroll
      for (int q = 0; q < NY_PER; ++q) sy[(tid + 512 * q) % BT_ROWS][(tid + 512 * q) / BT_ROWS] = ry[q];
      if (i0 + BT_ROWS < n) {
        load_v(k0, mm, i0 + BT_ROWS, rv);
        load_y(i0 + BT_ROWS, ry);
      }
      __syncthreads();
#pragma unroll 8
      for (int rr = 0; rr < BT_ROWS; ++rr) xs += sv[rr][xa] * sy[rr][xc];
    }
    X[xa][xc] = xs;
    __syncthreads();
    // X2 = T X (T upper triangular)
    {
      double t2 = 0.0;
      for (int b = xa; b < BT_NB; ++b) t2 += Tm[xa][b] * X[b][xc];
      X2[xa][xc] = t2;
    }
    // Y -= V X2, each thread NY_PER entries of the chunk
    load_v(k0, mm, k0 + 1, rv);
    load_y(k0 + 1, ry);
    for (int i0 = k0 + 1; i0 < n; i0 += BT_ROWS) {
      __syncthreads();
#pragma unroll
      for (int q = 0; q < NV_PER; ++q) sv[(tid + 512 * q) % BT_ROWS][(tid + 512 * q) / BT_ROWS] = rv[q];
      double yc[NY_PER];
#pragma unroll
      for (int q = 0; q < NY_PER; ++q) yc[q] = ry[q];
      if (i0 + BT_ROWS < n) {
        load_v(k0, mm, i0 + BT_ROWS, rv);
        load_y(i0 + BT_ROWS, ry);
      }
      __syncthreads();
#pragma unroll
      for (int q = 0; q < NY_PER; ++q) {
        const int e2 = tid + 512 * q, rr = e2 % BT_ROWS, c = e2 / BT_ROWS;
        const int i = i0 + rr;
        if (i < n && c < nv) {
          double u = 0.0;
#pragma unroll 8
          for (int a = 0; a < BT_NB; ++a) u += sv[rr][a] * X2[a][c];
          Y[i + (int64_t)n * c] = yc[q] - u;
        }
      }
    }
  }
  __syncthreads();
  // gauge, one warp per vector
  const int lane = tid & 31, warp = tid >> 5;
  if (warp < nv) {
    double* y = Y + (int64_t)n * warp;
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
}

std::vector<EigDev> to_dev(const tt_eig_problem* probs, int n_probs, const int* nvec) {
  std::vector<EigDev> hp(n_probs);
  for (int i = 0; i < n_probs; ++i)
    hp[i] = EigDev{probs[i].g_off, probs[i].w_off, probs[i].a_off, probs[i].n, probs[i].flags,
                   nvec ? nvec[i] : 0, 0, 0};
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
  if (vb < 6 * MAX_N) return cp;
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
  if (cudaFuncSetAttribute(chol_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
    cudaGetLastError();
    return cp;
  }
  for (int cl : {CL_MAX, 8}) {
    bool ok = blocked_smem(MAX_N, 8, cl) <= va;  // the largest sector fits at the narrowest panel
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
  double* vw = nullptr;
  if (!big.empty()) {
    // panel width per problem: the widest whose shared memory fits; the
    // panel scratch (n x 2nb per problem) lives in the pool
    int64_t need = 0, scratch = 0;
    for (EigDev& e : big) {
      e.nb = PNB_MAX;
      while (e.nb > 8 && blocked_smem(e.n, e.nb, cp.cl) > cp.vals_cap) e.nb /= 2;
      need = std::max(need, blocked_smem(e.n, e.nb, cp.cl));
      e.s_off = scratch;
      scratch += (int64_t)e.n * 2 * e.nb;
    }
    TT_REQUIRE(need <= cp.vals_cap, "tt_sym_eigvals_batched: sector too large for the cluster eigensolver");
    vw = tt::pool_alloc<double>(ctx, (size_t)scratch);
    if (!vw) return tt::fail(TT_ERR_OOM, "tt_sym_eigvals_batched: allocation failed");
    TT_CUDA(tt::h2d_async(ctx, dp + n_small, big.data(), sizeof(EigDev) * big.size()));
    TT_CUDA(launch_cluster(ctx, cp.cl, (int)big.size(), need, (const void*)tridiag_eigvals_cluster,
                           dp + n_small, G, T, w, vw));
    // their eigenvalues, BS_PER per CTA over the whole GPU
    std::vector<VecTaskB> bt;
    int nmax = 0;
    for (size_t b = 0; b < big.size(); ++b) {
      nmax = std::max(nmax, big[b].n);
      for (int j0 = 0; j0 < big[b].n; j0 += BS_PER) bt.push_back(VecTaskB{n_small + (int32_t)b, j0});
    }
    VecTaskB* d_bt = tt::pool_alloc<VecTaskB>(ctx, bt.size());
    if (!d_bt) return tt::fail(TT_ERR_OOM, "tt_sym_eigvals_batched: allocation failed");
    TT_CUDA(tt::h2d_async(ctx, d_bt, bt.data(), sizeof(VecTaskB) * bt.size()));
    const size_t bs_smem = sizeof(double) * 2 * (size_t)nmax;
    static thread_local uint64_t bs_attr = 0;
    if (tt::first_on_device(bs_attr, ctx->device))
      TT_CUDA(cudaFuncSetAttribute(bisect_sectors, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)(sizeof(double) * 2 * MAX_N)));
    bisect_sectors<<<(unsigned)bt.size(), BS_THREADS, bs_smem, ctx->stream>>>(dp, d_bt, T, w);
    TT_LAUNCH_CHECK(ctx);
    tt::pool_free(ctx, d_bt);
  }
  tt::pool_free(ctx, vw);
  tt::pool_free(ctx, dp);
  return TT_OK;
}

int tt_eig_redo_count(tt_ctx* ctx, int64_t* count) {
  TT_REQUIRE(ctx && count, "tt_eig_redo_count: null argument");
  unsigned long long* h = reinterpret_cast<unsigned long long*>(ctx->h_scalars);
  TT_CUDA(cudaMemcpyFromSymbolAsync(h, g_eig_redo, sizeof(unsigned long long), 0, cudaMemcpyDeviceToHost,
                                    ctx->stream));
  TT_CUDA(cudaStreamSynchronize(ctx->stream));
  *count = (int64_t)*h;
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
    // the GPU-wide path: inverse iteration, CholeskyQR2, compact-WY
    // back-transformation; problems it flags are redone by the cluster kernel
    const int nbig = (int)big.size();
    std::vector<VecTask> iv, ts, ap;
    std::vector<TileTask> gm, wy;
    for (int p = 0; p < nbig; ++p) {
      const EigDev& e = big[p];
      for (int j = 0; j < e.nvec; j += IV_THREADS) iv.push_back(VecTask{p, j});
      const int nt = (e.nvec + GT - 1) / GT;
      for (int a = 0; a < nt; ++a)
        for (int b = 0; b <= a; ++b) gm.push_back(TileTask{p, a, b});
      if (e.nvec > 0) {
        for (int i = 0; i < e.n; i += TS_ROWS) ts.push_back(VecTask{p, i});
        for (int k = 0; k * BT_NB < e.n - 2; ++k) wy.push_back(TileTask{p, k, 0});
        for (int j = 0; j < e.nvec; j += BT_VB) ap.push_back(VecTask{p, j});
      }
    }
    const size_t bytes = sizeof(int) * nbig + sizeof(VecTask) * (iv.size() + ts.size() + ap.size()) +
                         sizeof(TileTask) * (gm.size() + wy.size()) + 64;
    char* buf = tt::pool_alloc<char>(ctx, bytes);
    if (!buf) return tt::fail(TT_ERR_OOM, "tt_sym_eigvecs_batched: allocation failed");
    int* flags = reinterpret_cast<int*>(buf);
    VecTask* d_iv = reinterpret_cast<VecTask*>(buf + ((sizeof(int) * nbig + 15) & ~(size_t)15));
    VecTask* d_ts = d_iv + iv.size();
    VecTask* d_ap = d_ts + ts.size();
    TileTask* d_gm = reinterpret_cast<TileTask*>(d_ap + ap.size());
    TileTask* d_wy = d_gm + gm.size();
    TT_CUDA(cudaMemsetAsync(flags, 0, sizeof(int) * nbig, ctx->stream));
    TT_CUDA(tt::h2d_async(ctx, d_iv, iv.data(), sizeof(VecTask) * iv.size()));
    TT_CUDA(tt::h2d_async(ctx, d_ts, ts.data(), sizeof(VecTask) * ts.size()));
    TT_CUDA(tt::h2d_async(ctx, d_ap, ap.data(), sizeof(VecTask) * ap.size()));
    TT_CUDA(tt::h2d_async(ctx, d_gm, gm.data(), sizeof(TileTask) * gm.size()));
    TT_CUDA(tt::h2d_async(ctx, d_wy, wy.data(), sizeof(TileTask) * wy.size()));
    const EigDev* db = dp + n_small;
    if (!iv.empty()) {
      inv_iter_batched<<<(unsigned)iv.size(), IV_THREADS, 0, ctx->stream>>>(db, d_iv, T, w, Z, work);
      TT_LAUNCH_CHECK(ctx);
    }
    for (int pass = 0; pass < 2 && !gm.empty(); ++pass) {
      gram_tiles<<<(unsigned)gm.size(), 256, 0, ctx->stream>>>(db, d_gm, Z, work, flags);
      TT_LAUNCH_CHECK(ctx);
      TT_CUDA(launch_cluster(ctx, cp.cl, nbig, 0, (const void*)chol_cluster, db, work, flags, pass == 0 ? 1 : 0));
      trsm_rows<<<(unsigned)ts.size(), 256, 0, ctx->stream>>>(db, d_ts, Z, work, flags);
      TT_LAUNCH_CHECK(ctx);
    }
    if (!wy.empty()) {
      wy_factors<<<(unsigned)wy.size(), 256, 0, ctx->stream>>>(db, d_wy, G, T, work, flags);
      TT_LAUNCH_CHECK(ctx);
      wy_apply<<<(unsigned)ap.size(), 512, 0, ctx->stream>>>(db, d_ap, G, Z, work, flags);
      TT_LAUNCH_CHECK(ctx);
    }
    int64_t needc = 0;  // fallback: own eigenvectors in shared memory when they fit, plus 6n of buffers
    for (const EigDev& e : big) {
      const int64_t q = (e.nvec + cp.cl - 1) / cp.cl;
      const int64_t extra = 6 * (int64_t)e.n;
      const int64_t full = q * e.n + extra;
      needc = std::max(needc, full <= cp.vecs_cap ? full : extra);
    }
    TT_CUDA(launch_cluster(ctx, cp.cl, nbig, needc, (const void*)tridiag_eigvecs_cluster, db, G, T, w, Z, work,
                           (int)needc, (const int*)flags));
    tt::pool_free(ctx, buf);
  }
  tt::pool_free(ctx, dp);
  return TT_OK;
}

}  // extern "C"
