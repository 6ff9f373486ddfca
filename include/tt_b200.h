/*
 * tt_b200.h -- C ABI of the B200 two-site DMRG inner loop.
 *
 * This is the boundary between the C++ host classes that mirror
 * tensor-tools' qtensor / big_qtensor / svd_bond / Davidson / dmrg interface
 * and the sm_100a kernels.  Every entry point is extern "C", takes plain
 * pointers and sizes, returns an int status (TT_OK == 0) and never throws;
 * the message of the last failure on the calling thread is returned by
 * tt_get_last_error().
 *
 * Reference interfaces replaced (paths relative to the tensor-tools tree):
 *   tt_contract_plan/exec    qtensor<T>::operator*      qtensor/qtensor.cpp:523-734
 *                            dtensor<T>::operator*      dtensor/dtensor.cpp:300-368
 *   tt_vec_*                 qtensor<T>::inner_product / add / contract / norm /
 *                            normalize / operator*=     qtensor/qtensor.cpp:1031-1179,1606-1647
 *                            dtensor<T>::add / inner_product / norm
 *                                                       dtensor/dtensor.cpp:792-849
 *   tt_vec_fill_random       qtensor<T>::setRandom      qtensor/qtensor.cpp:381-388
 *   tt_vec_precondition      elemWiseDivide             linalg/tensor_davidson.cpp:25-36
 *   tt_dav_*                 tensor_davidsonIT control  linalg/tensor_davidson.cpp:193-347,
 *                            DIAG                       linalg/lapack_wrapper.cpp:40-54
 *   tt_sym_eig_batched       CTF Matrix::svd per QN sector (ScaLAPACK pdgesvd)
 *                                                       qtensor/qtensor_op.cpp:1269,
 *                                                       dtensor/dtensor_op.cpp:175
 *                            DIAG (dsyev)               linalg/lapack_wrapper.cpp:40-54
 *   tt_copy2d_batched        CTF slice of sector matrices into U/V blocks
 *                                                       qtensor/qtensor_op.cpp:1229-1246,1389-1436
 *   tt_strided_copy          dtensor<T>::diagonal / qtensor permute
 *                                                       dtensor/dtensor.cpp:511-571
 *
 * The object-level API that big_qtensor / dmrg callers bind (qtensor
 * handles, svd_bond, the DMRG drivers) is declared in tt_dmrg.h.
 */
#ifndef TT_B200_H
#define TT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define TT_OK              0
#define TT_ERR_INVALID     1  /* bad argument, plan or descriptor            */
#define TT_ERR_OOM         2  /* device or host allocation failed            */
#define TT_ERR_CUDA        3  /* CUDA runtime or launch error                */
#define TT_ERR_TIMEOUT     4  /* a bounded device wait gave up               */
#define TT_ERR_NOCONV      5  /* an iterative kernel did not converge        */
#define TT_ERR_NO_DEVICE   6  /* no usable sm_100 device                     */

/* ---- precision of the block contractions -------------------------------- */
#define TT_PREC_FP64       0  /* DMMA f64 tensor-core tiles                  */
#define TT_PREC_TF32       1  /* tcgen05 kind::tf32, FP32 accumulator in TMEM */
#define TT_PREC_TF32X3     2  /* tcgen05 kind::tf32 on hi/lo splits of the FP64
                                 operands (hi*hi + hi*lo + lo*hi), FP32 accumulator */
/* Per contraction, TF32 / 3xTF32 where the plan's cost model (padded tile
 * work, DRAM bytes including the operand packing, launches) predicts the
 * tensor-core form to be faster than FP64 DMMA, FP64 elsewhere -- e.g. the
 * bandwidth-bound contractions over a small MPO link.  Never less accurate
 * than the forced kind. */
#define TT_PREC_TF32_AUTO   3
#define TT_PREC_TF32X3_AUTO 4

#define TT_MAX_MODES       6  /* tensor modes per GEMM dimension of a pair   */
#define TT_DAV_MAX        16  /* Krylov vectors of the device-resident Davidson */

typedef struct tt_ctx tt_ctx;
typedef struct tt_plan tt_plan;

/* ---- context, memory ---------------------------------------------------- */
/* One context per device and host thread: a CUDA stream, a stream-ordered
 * memory pool and the plan cache.  A context is not thread-safe. */
int tt_ctx_create(int device, tt_ctx** out);
int tt_ctx_destroy(tt_ctx* ctx);
int tt_ctx_synchronize(tt_ctx* ctx);
/* cudaStream_t of the context, as an opaque pointer (for event timing). */
int tt_ctx_stream(tt_ctx* ctx, void** stream);
/* Host wall seconds spent blocked in synchronisations of this context's
 * stream (device-to-host reads, tt_ctx_synchronize) and how many there were. */
int tt_ctx_wait_stats(tt_ctx* ctx, double* seconds, int64_t* count);
/* Pool allocations that failed once, trimmed the pool to its use and
 * succeeded or failed on the retry (each trim synchronises the stream). */
int tt_ctx_pool_trims(tt_ctx* ctx, int64_t* count);
/* Host wall seconds inside the context's device allocate and free calls:
 * totals, the largest single call since the last reset, the number of
 * allocations, how many were served from the block cache, and the bytes the
 * cache holds now.  reset_max != 0 zeroes the two maxima after reading. */
int tt_ctx_alloc_stats(tt_ctx* ctx, double* alloc_s, double* alloc_max_s, double* free_s, double* free_max_s,
                       int64_t* allocs, int64_t* cache_hits, int64_t* cached_bytes, int reset_max);
/* Block cache: allocations of 32 MB or more are rounded up to a size class
 * (at most 25% above the request) and, when freed, kept by the context (up
 * to `bytes` in total, the blocks freed longest ago evicted first; default
 * 32 GiB) for the next allocation on its stream that fits in one (a block at
 * most 1.5x the request's class), instead of going back to the device pool,
 * which can stall the host for seconds assembling a multi-gigabyte block.  Cached
 * blocks count as used in tt_ctx_memory; an allocation that fails returns
 * them to the pool and retries.  0 turns the cache off and releases it. */
int tt_ctx_set_block_cache(tt_ctx* ctx, int64_t bytes);
/* Sticky device status of the context: TT_OK, or TT_ERR_TIMEOUT once a bounded
 * wait inside a tensor-core contraction has given up (that contraction's output
 * is incomplete).  Every synchronisation of the context -- tt_ctx_synchronize
 * and tt_memcpy_d2h, hence every Davidson call and block SVD -- returns
 * TT_ERR_TIMEOUT while it is set, so a run with skipped tiles cannot report a
 * result.  tt_ctx_device_status synchronises and reads it;
 * tt_ctx_clear_device_status synchronises and resets it.  No counterpart in the
 * reference (which has no device waits). */
int tt_ctx_device_status(tt_ctx* ctx, int* status);
int tt_ctx_clear_device_status(tt_ctx* ctx);
/* Test hook: polls of the main-loop mbarrier waits of the tensor-core kernels
 * launched from now on before they give up (default 2^26; polls < 0 restores
 * it, 0 makes the first wait give up).  The drain that lets issued copies and
 * MMAs land before shared and tensor memory are released keeps the default. */
int tt_ctx_set_wait_limit(tt_ctx* ctx, int64_t polls);
/* Bytes of the context's stream-ordered pool: in use now, the high-water mark
 * of use (reset to the current use when reset_high is non-zero) and reserved
 * from the device (freed blocks stay cached in the pool). */
int tt_ctx_memory(tt_ctx* ctx, int64_t* used, int64_t* used_high, int64_t* reserved, int reset_high);
const char* tt_get_last_error(void);

int tt_device_alloc(tt_ctx* ctx, size_t bytes, void** dptr);
int tt_device_free(tt_ctx* ctx, void* dptr);
int tt_memcpy_h2d(tt_ctx* ctx, void* dst, const void* src, size_t bytes);
int tt_memcpy_d2h(tt_ctx* ctx, void* dst, const void* src, size_t bytes);
int tt_memcpy_d2d(tt_ctx* ctx, void* dst, const void* src, size_t bytes);
int tt_memset_zero(tt_ctx* ctx, void* dst, size_t bytes);
/* Counts kernel launches issued through this context (all tt_* kernels). */
int tt_ctx_launch_count(tt_ctx* ctx, int64_t* count);
/* CUDA events on the context's stream, for device-side timing. */
int tt_event_create(tt_ctx* ctx, void** ev);
int tt_event_record(tt_ctx* ctx, void* ev);
int tt_event_elapsed_ms(void* ev_start, void* ev_stop, float* ms);  /* waits for ev_stop */
int tt_event_destroy(void* ev);

/* ---- grouped block contraction ------------------------------------------
 * One launch computes, for every output block o,
 *     C_o = alpha * sum_{pairs p of o} A_p (M x K) * B_p (K x N)
 * where C_o is stored column-major at C + c_off with leading dimension ldc,
 * and the GEMM views of A_p and B_p are arbitrary strided tensor blocks:
 *     A_p(m,k) = A[a_off + sum_i m_i*a_m_stride[i] + sum_j k_j*a_k_stride[j]]
 *     B_p(k,n) = B[b_off + sum_j k_j*b_k_stride[j] + sum_i n_i*b_n_stride[i]]
 * with m, k, n decomposed mixed-radix over m_dims, k_dims, n_dims (first mode
 * fastest).  Output blocks without pairs are written with zeros.  This is
 * qtensor::operator*'s inner loop "C[indC] += A_L*B_R" over all block pairs
 * of one contraction (qtensor/qtensor.cpp:652-726), flattened into one launch.
 */
typedef struct {
  int64_t c_off;
  int32_t m, n;
  int32_t ldc;
} tt_out_block;

typedef struct {
  int32_t out_block;             /* index into the tt_out_block list        */
  int32_t n_m, n_k, n_n;         /* number of modes in each GEMM dimension   */
  int64_t a_off, b_off;
  int32_t m_dims[TT_MAX_MODES];
  int32_t k_dims[TT_MAX_MODES];
  int32_t n_dims[TT_MAX_MODES];
  int64_t a_m_stride[TT_MAX_MODES];
  int64_t a_k_stride[TT_MAX_MODES];
  int64_t b_k_stride[TT_MAX_MODES];
  int64_t b_n_stride[TT_MAX_MODES];
} tt_block_pair;

int tt_contract_plan(tt_ctx* ctx, const tt_out_block* outs, int n_out,
                     const tt_block_pair* pairs, int n_pairs, int precision,
                     tt_plan** plan);
/* As tt_contract_plan, with a hint for the *_AUTO choice: keep bit 0 (A) /
 * bit 1 (B) marks an operand that the caller will keep packed across several
 * execs (tt_contract_exec_keep), so its packing is charged once for several
 * of them.  The hint changes only the precision chosen, never the results of
 * a given precision. */
int tt_contract_plan_keep(tt_ctx* ctx, const tt_out_block* outs, int n_out,
                          const tt_block_pair* pairs, int n_pairs, int precision, int keep,
                          tt_plan** plan);
int tt_contract_exec(tt_ctx* ctx, const tt_plan* plan, const double* A,
                     const double* B, double* C, double alpha);
/* tt_contract_exec that keeps packed operands: bit 0 of keep keeps A's
 * tensor-core packing (TF32 hi/lo tiles) in the plan after the exec and reuses
 * it in later execs given the same A pointer, bit 1 the same for B -- for an
 * operand that stays fixed over many execs, such as the environments of one
 * Davidson call.  The caller vouches that the data behind a kept pointer has
 * not changed, and releases the packings (tt_plan_release_packed, or the plan's
 * destruction) before it does.  Bit 2 (A) / bit 3 (B) keep only the packing
 * buffer of an operand that is packed afresh in every exec, so that a run of
 * execs allocates it once (released with the kept packings).  FP64 plans
 * ignore keep. */
int tt_contract_exec_keep(tt_ctx* ctx, const tt_plan* plan, const double* A, const double* B, double* C,
                          double alpha, int keep);
int tt_plan_release_packed(tt_ctx* ctx, const tt_plan* plan);
int tt_plan_destroy(tt_ctx* ctx, tt_plan* plan);
/* Algorithmic work of one exec: sum over pairs of 2*m*n*k. */
/* Device bytes a plan holds (offset tables, tasks, packing jobs). */
/* Host seconds this thread's planner spent in its stages since the thread
 * started (diagnostic): [0] pair offset tables, [1] the precision choice of
 * the automatic modes, [2] tile tasks and row-stationary chunks, [3]
 * tensor-core packing jobs, [4] device tables, uploads and the rest.  The
 * first min(n, 5) are written. */
int tt_contract_plan_timers(double* seconds, int n);
int tt_plan_device_bytes(const tt_plan* plan, int64_t* bytes);
int tt_plan_flops(const tt_plan* plan, double* flops);
/* The precision the plan runs in (TT_PREC_FP64 / TF32 / TF32X3): an *_AUTO
 * request resolves to one of them when the plan is built. */
int tt_plan_precision(const tt_plan* plan, int* precision);
/* The cost model behind the *_AUTO precisions, without a device: the
 * predicted microseconds of one exec of the contraction (described as for
 * tt_contract_plan) in FP64 and in the tensor-core kind, and the precision
 * tt_contract_plan would choose on a device with num_sms SMs. */
int tt_contract_predict(const tt_out_block* outs, int n_out, const tt_block_pair* pairs,
                        int n_pairs, int precision, int num_sms, double* us_fp64,
                        double* us_tc, int* choice);
/* Device status of the plan's tensor-core launches since the plan was built:
 * TT_OK, or TT_ERR_TIMEOUT when a bounded wait on the MMA completion barrier
 * gave up (the tile was then skipped).  Synchronises the context's stream. */
int tt_plan_device_status(tt_ctx* ctx, const tt_plan* plan, int* status);

/* ---- Davidson vector kernels (flat, deterministic reductions) -----------
 * Vectors are contiguous FP64 arrays of n elements (all blocks of a
 * block-sparse tensor laid out back to back).  Scalars that feed the host
 * (dots, norms) are written to device memory; read them with
 * tt_memcpy_d2h.  Coefficient arrays may live on the device so that no host
 * round trip is needed between dependent kernels. */
int tt_vec_dot(tt_ctx* ctx, int64_t n, const double* x, const double* y, double* d_out);
/* d_out[j] = <xs[j], y> for j < nvec (1..16), reading y once.  xs is a
 * HOST array of nvec device pointers. */
int tt_vec_multidot(tt_ctx* ctx, int64_t n, int nvec, const double* const* xs,
                    const double* y, double* d_out);
/* Allocation-free tt_vec_multidot (no counterpart in the reference).  For
 * callers that cannot allocate device memory -- and therefore cannot create a
 * tt_ctx -- such as an application that reserves the whole GPU for its own
 * memory pool, or a plugin host that only lends out buffers it owns.  The
 * caller passes the inputs, the output (d_out, nvec doubles on the device) and
 * a CUDA stream (cudaStream_t as void*, 0 for the legacy default stream) on
 * the current device; nothing is allocated.  Partial sums live in a fixed
 * 16 x 1024-double (128 KiB) array inside the library that every GPU loading
 * it holds until the process exits, so nvec is limited to 1..16 (larger is
 * rejected with TT_ERR_INVALID); n is not limited.  The first call on a device
 * looks up that array's device address (cudaGetSymbolAddress) and should come
 * before any stream capture; only a successful look-up is kept, so a first
 * call that fails (an earlier asynchronous error still pending, say) is retried
 * by the next call.  All calls share the array: calls that overlap
 * on the GPU (different streams, or host threads without ordering) race. */
int tt_vec_multidot_noalloc(void* stream, int64_t n, int nvec, const double* const* xs,
                            const double* y, double* d_out);
int tt_vec_nrm2(tt_ctx* ctx, int64_t n, const double* x, double* d_out);
int tt_vec_axpy(tt_ctx* ctx, int64_t n, double a, const double* x, double* y);
int tt_vec_scal(tt_ctx* ctx, int64_t n, double a, double* x);
/* x *= 1/ *d_nrm, with the norm read on the device. */
int tt_vec_scal_inv_dev(tt_ctx* ctx, int64_t n, const double* d_nrm, double* x);
/* x[i + inner*(m + mid*o)] *= scale[m] (scale: mid <= TT_SCALE_MODE_MAX host
 * values): a diagonal one-site operator such as Sz applied to one mode of a
 * column-major block; no alignment requirement */
#define TT_SCALE_MODE_MAX 8
int tt_vec_scale_mode(tt_ctx* ctx, int64_t inner, int mid, int64_t outer, const double* scale, double* x);
/* y = sum_j sign * coef[j] * xs[j] (+ y if accumulate), coefficients on the
 * device: the Gram-Schmidt projection and Ritz-vector build in one pass.
 * xs is a HOST array of nvec (0..16) device pointers. */
int tt_vec_lincomb_dev(tt_ctx* ctx, int64_t n, int nvec, const double* const* xs,
                       const double* d_coef, double sign, int accumulate, double* y);
/* The Gram-Schmidt projection and its norm in one launch: y -= sum_j
 * coef[j] xs[j] (coefficients on the device), then *d_norm = |y|;
 * bit-identical to tt_vec_lincomb_dev(..., -1.0, 1, y) followed by
 * tt_vec_nrm2.  xs is a HOST array of nvec (0..16) device pointers. */
int tt_vec_project_nrm2_dev(tt_ctx* ctx, int64_t n, int nvec, const double* const* xs,
                            const double* d_coef, double* y, double* d_norm);
/* The same, enqueued unconditionally but a no-op unless *d_cond (a device int)
 * is non-zero when it runs. */
int tt_vec_project_nrm2_dev_if(tt_ctx* ctx, int64_t n, int nvec, const double* const* xs,
                               const double* d_coef, double* y, double* d_norm, const int* d_cond);
/* The Ritz vector and residual of a Davidson iteration in one pass
 * (linalg/tensor_davidson.cpp:255-269): x = sum_{j<k} coef_x[j] vs[j] and
 * q = sum_{j<k} coef_q[j] vas[j] + coef_q[k] x, coefficients on the device;
 * bit-identical to two tt_vec_lincomb_dev calls.  vs and vas are HOST arrays
 * of k (1..15) device pointers. */
int tt_vec_ritz_residual_dev(tt_ctx* ctx, int64_t n, int k, const double* const* vs,
                             const double* const* vas, const double* d_coef_x,
                             const double* d_coef_q, double* x, double* q);
/* x[r] = uniform(0,1) for every element inside the given [begin,end) element
 * ranges (blocks present in the tensor), 0 elsewhere; counter-based RNG. */
int tt_vec_fill_random(tt_ctx* ctx, int64_t n, double* x, int nranges,
                       const int64_t* d_ranges, uint64_t seed);
/* x[i] = x[i] / (D[i] - theta) where D[i] != theta. */
int tt_vec_precondition(tt_ctx* ctx, int64_t n, double* x, const double* D, double theta);

/* ---- device-resident Davidson control (tensor_davidsonIT) -----------------
 * The decisions of the Davidson loop (linalg/tensor_davidson.cpp:193-347) run
 * on the device so that a caller can enqueue every iteration without reading
 * scalars back: tt_dav_begin takes the initial Rayleigh quotient, tt_dav_ritz
 * diagonalises the projected matrix (DIAG: dsyev semantics, <= TT_DAV_MAX) and
 * writes the Ritz coefficients (tt_dav_coefficients gives their device
 * addresses, for tt_vec_lincomb_dev), tt_dav_converged applies the
 * convergence test to the residual norm, tt_dav_add_row adds the new row of
 * the projected matrix unless Gram-Schmidt failed (norm < 1e-10).  After the
 * loop has ended every control call is a no-op; tt_dav_read synchronises and
 * returns where it ended (final_ii, or -2 with fail_ii for a Gram-Schmidt
 * failure that the caller finishes on the host). */
typedef struct tt_dav_state tt_dav_state;
typedef struct {
  int done, final_ii, fail_ii, iters, randomized;
  double lambda;
} tt_dav_result;
int tt_dav_state_create(tt_ctx* ctx, tt_dav_state** st);
int tt_dav_state_destroy(tt_ctx* ctx, tt_dav_state* st);
int tt_dav_coefficients(tt_dav_state* st, double** coef_x, double** coef_q);
int tt_dav_begin(tt_ctx* ctx, tt_dav_state* st, const double* d_init_energy);
int tt_dav_ritz(tt_ctx* ctx, tt_dav_state* st, int ii);
int tt_dav_converged(tt_ctx* ctx, tt_dav_state* st, int ii, int maxiter, double tol, const double* d_qnorm);
int tt_dav_add_row(tt_ctx* ctx, tt_dav_state* st, int ii, const double* d_row, const double* d_gsnorm);
int tt_dav_read(tt_ctx* ctx, const tt_dav_state* st, tt_dav_result* out);
/* Gram-Schmidt failure on the device (linalg/tensor_davidson.cpp:298-316):
 * enqueued after every projection of a new vector y = v[ni]; a no-op unless
 * the norm at d_gsnorm is below 1e-10.  Then, when ni < maxsize, y is
 * refilled with random numbers on the [begin, end) element ranges d_ranges
 * (the blocks of the previous vector, sorted), its overlaps with xs[0..ni-1]
 * go to d_dots and the flag at tt_dav_refill_flag is raised for a following
 * tt_vec_project_nrm2_dev_if; when ni >= maxsize the loop ends with the
 * current Ritz vector.  A refill that fails again ends the loop the same way
 * (tt_dav_add_row).  tt_dav_result.randomized counts the refills. */
int tt_dav_gs_refill(tt_ctx* ctx, tt_dav_state* st, int ii, int ni, int maxsize, int64_t n,
                     const double* const* xs, double* y, int nranges, const int64_t* d_ranges, uint64_t seed,
                     const double* d_gsnorm, double* d_dots);
int tt_dav_refill_flag(tt_dav_state* st, const int** d_flag);

/* ---- strided copies ------------------------------------------------------
 * dst[dst_off + sum_i j_i*dst_stride[i]] = src[src_off + sum_i j_i*src_stride[i]]
 * over all j in dims (up to TT_MAX_MODES modes). */
typedef struct {
  int32_t n_modes;
  int32_t dims[TT_MAX_MODES];
  int64_t src_off, dst_off;
  int64_t src_stride[TT_MAX_MODES];
  int64_t dst_stride[TT_MAX_MODES];
} tt_copy_desc;
int tt_strided_copy_batched(tt_ctx* ctx, const tt_copy_desc* descs, int n,
                            const double* src, double* dst);

/* ---- symmetric eigensolver (density matrices of the block SVD) ----------
 * For each problem p: G_p is n x n symmetric, column-major with leading
 * dimension n, at G + g_off[p].  On return the eigenvalues are in
 * w[w_off[p] ...] in DESCENDING order and the matching orthonormal
 * eigenvectors are the columns of Z_p at Z + g_off[p] (same layout).  G is
 * destroyed.  Cyclic Jacobi with a bounded sweep count; status
 * TT_ERR_NOCONV if a problem did not reach the off-diagonal tolerance. */
#define TT_EIG_ROW_1X2  1  /* problem is the 2x2 Gram of a 1x2 sector matrix */
typedef struct {
  int64_t g_off;
  int64_t w_off;
  int64_t a_off;        /* TT_EIG_ROW_1X2: the 1x2 matrix (a, b) at A + a_off */
  int32_t n;
  int32_t flags;
} tt_eig_problem;
/* TT_EIG_ROW_1X2 reproduces the reference's 1x2 workaround for ScaLAPACK
 * (qtensor/qtensor_op.cpp:1247-1267): the leading eigenvector is (a,b)/d,
 * d = |(a,b)|, or (1,1)/sqrt(2) when d == 0; eigenvalues d*d and 0. */
int tt_sym_eig_batched(tt_ctx* ctx, const tt_eig_problem* probs, int n_probs,
                       double* G, double* Z, double* w, const double* A);

/* Two-phase eigensolver used by the block SVD (n <= 4096 and nvec <= 2048 per problem).
 * Phase 1: Householder tridiagonalisation of each G_p in place (reflectors
 * below the subdiagonal), d/e/tau of T_p in T[3*w_off .. 3*w_off + 3n), and
 * every eigenvalue in DESCENDING order in w[w_off ..] (bisection).  Phase 2:
 * the eigenvectors of the nvec[p] largest eigenvalues as the first nvec[p]
 * columns of Z + g_off (leading dimension n), by inverse iteration on T_p,
 * Gram-Schmidt inside clusters of close eigenvalues, and back-transformation
 * with the reflectors left in G; work holds 3*n*n doubles per problem at
 * 3*g_off.  TT_EIG_ROW_1X2 problems follow the 1x2 rule described above. */
int tt_sym_eigvals_batched(tt_ctx* ctx, const tt_eig_problem* probs, int n_probs, double* G,
                           double* T, double* w, const double* A);
int tt_sym_eigvecs_batched(tt_ctx* ctx, const tt_eig_problem* probs, int n_probs, const int* nvec,
                           const double* G, const double* T, const double* w, double* Z,
                           double* work, const double* A);
/* Problems (since the process started, all contexts on the device) whose
 * CholeskyQR2 found an inverse-iteration vector collapsed onto earlier ones,
 * so that the cluster kernel recomputed their eigenvectors; synchronises the
 * context's stream. */
int tt_eig_redo_count(tt_ctx* ctx, int64_t* count);

#ifdef __cplusplus
}
#endif
#endif /* TT_B200_H */
