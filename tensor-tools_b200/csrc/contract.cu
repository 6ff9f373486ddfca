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
#include <chrono>
#include <cstring>
#include <functional>
#include <map>
#include <numeric>
#include <unordered_map>
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

// ---------------------------------------------------------------------------
// Skinny FP64 path: contractions whose output blocks have at most SK_N
// columns and whose pairs contract at most SK_K elements -- the middle
// contraction of H_eff*x and of the environment update, (a' b) x (w s1 s2)
// times (w s1 s2) x (s1' s2' w'), with rows a' b in the hundreds of
// thousands and k, n the MPO link sector widths.  A 64 x 64 DMMA tile wastes
// most of its work there, and the contraction is bound by reading T1 and
// writing T2.  Here a CTA takes SK_ROWS rows of one output block; each
// thread keeps its row's n outputs in registers across all pairs of the
// block, with the pair's B (k x n, tiny) staged in shared memory, and reads
// its A row through the offset tables (coalesced along a unit-stride row
// mode).  Pairs are summed in the plan's order, as in grouped_dgemm.  The
// kernel is instantiated for NC = 4, 8, 16, 32 output columns (the plan's
// widest block rounded up), so a narrow contraction issues no work for
// columns it does not have and keeps few registers (more CTAs per SM).
constexpr int SK_N = 32;
constexpr int SK_K = 64;
constexpr int SK_ROWS = 256;
constexpr int64_t SK_STAGE_BYTES = 64 * 1024;  // dynamic shared memory for a task's staged pairs

template <int NC>
__global__ void __launch_bounds__(SK_ROWS)
skinny_dgemm(const TaskDev* __restrict__ tasks, const OutDev* __restrict__ outs,
             const PairDev* __restrict__ pairs, const int32_t* __restrict__ tab,
             const double* __restrict__ A, const double* __restrict__ B, double* __restrict__ C,
             double alpha, int staged) {
  // staged != 0: every pair's B (k x NC, zero past n) and A column offsets are
  // staged once for the task (dynamic shared memory sized by the plan), so the
  // pairs run without barriers; else one pair at a time through sB / sColA
  extern __shared__ double sk_dyn[];
  __shared__ double sB[SK_K][NC];
  __shared__ int32_t sColA[SK_K];
  const TaskDev task = tasks[blockIdx.x];
  const OutDev out = outs[task.out];
  const int r = task.m0 + threadIdx.x;
  double acc[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) acc[c] = 0.0;
  if (staged) {
    double* bst = sk_dyn;
    int ktot = 0;
    for (int p = task.p_begin; p < task.p_end; ++p) ktot += pairs[p].k;
    int32_t* cst = reinterpret_cast<int32_t*>(sk_dyn + (int64_t)ktot * NC);
    int k0 = 0;
    for (int p = task.p_begin; p < task.p_end; ++p) {
      const PairDev P = pairs[p];
      for (int e = threadIdx.x; e < P.k * NC; e += blockDim.x) {
        const int kk = e / NC, c = e % NC;
        bst[(k0 + kk) * NC + c] = c < P.n ? B[P.b_off + tab[P.rowB + kk] + tab[P.colB + c]] : 0.0;
      }
      for (int kk = threadIdx.x; kk < P.k; kk += blockDim.x) cst[k0 + kk] = tab[P.colA + kk];
      k0 += P.k;
    }
    __syncthreads();
    k0 = 0;
    for (int p = task.p_begin; p < task.p_end; ++p) {
      const PairDev P = pairs[p];
      if (r < P.m) {
        const double* __restrict__ arow = A + P.a_off + tab[P.rowA + r];
        for (int kk = 0; kk < P.k; ++kk) {
          const double a = arow[cst[k0 + kk]];
#pragma unroll
          for (int c = 0; c < NC; ++c) acc[c] = fma(a, bst[(k0 + kk) * NC + c], acc[c]);
        }
      }
      k0 += P.k;
    }
  } else {
    for (int p = task.p_begin; p < task.p_end; ++p) {
      const PairDev P = pairs[p];
      __syncthreads();  // the previous pair's B is no longer read
      for (int e = threadIdx.x; e < P.k * NC; e += blockDim.x) {
        const int kk = e / NC, c = e % NC;
        sB[kk][c] = c < P.n ? B[P.b_off + tab[P.rowB + kk] + tab[P.colB + c]] : 0.0;  // zero past n
      }
      for (int kk = threadIdx.x; kk < P.k; kk += blockDim.x) sColA[kk] = tab[P.colA + kk];
      __syncthreads();
      if (r < P.m) {
        const double* __restrict__ arow = A + P.a_off + tab[P.rowA + r];
        for (int kk = 0; kk < P.k; ++kk) {
          const double a = arow[sColA[kk]];
#pragma unroll
          for (int c = 0; c < NC; ++c) acc[c] = fma(a, sB[kk][c], acc[c]);
        }
      }
    }
  }
  if (r < out.m) {
    double* Cb = C + out.c_off + r;
#pragma unroll
    for (int c = 0; c < NC; ++c)
      if (c < out.n) Cb[(int64_t)out.ldc * c] = alpha * acc[c];
  }
}

// Row-stationary form of the skinny path.  Output blocks that read the same
// A blocks (the same rows, other column sectors: for the middle contraction
// the (s1' s2' w') sectors fed by one T1 block) are gathered into chunks of
// at most RS_COLS columns; a task is one chunk's SK_ROWS-row tile.  Each distinct
// A block of the chunk is read once per row and multiplied into a combined B
// (k x NC: every pair's B block at its output's columns, zeros elsewhere), so
// T1 crosses HBM once instead of once per output sector.
// combined columns per chunk: 16 keeps the accumulators of a 256-row task at
// about 70 registers a thread (three CTAs per SM); 32 halved the occupancy and
// ran slower than reading a shared A block twice
constexpr int RS_COLS = 16;
struct RsChunk {
  int32_t a_begin, a_end;  // its distinct A blocks in rs_a
  int32_t o_begin, o_end;  // its output blocks in rs_o
  int32_t m;               // rows (shared by the chunk's outputs)
  int32_t ktot;            // sum of k over its A blocks
};
struct RsA {
  int32_t pair;            // a pair reading this A block (its rowA / colA tables, a_off, k)
  int32_t e_begin, e_end;  // the pairs of the chunk reading it, in rs_e
};
struct RsE {
  int32_t pair, col;  // a pair and the first combined column of its output
};
struct RsO {
  int32_t out, col;  // an output block and its first combined column
};

template <int NC>
__global__ void __launch_bounds__(SK_ROWS)
skinny_rs(const TaskDev* __restrict__ tasks, const RsChunk* __restrict__ chunks, const RsA* __restrict__ ra,
          const RsE* __restrict__ re, const RsO* __restrict__ ro, const OutDev* __restrict__ outs,
          const PairDev* __restrict__ pairs, const int32_t* __restrict__ tab, const double* __restrict__ A,
          const double* __restrict__ B, double* __restrict__ C, double alpha) {
  extern __shared__ double rs_dyn[];  // ktot x NC combined B, then ktot A column offsets
  const TaskDev task = tasks[blockIdx.x];
  const RsChunk ch = chunks[task.out];
  const int r = task.m0 + threadIdx.x;
  double* bst = rs_dyn;
  int32_t* cst = reinterpret_cast<int32_t*>(rs_dyn + (int64_t)ch.ktot * NC);
  for (int e = threadIdx.x; e < ch.ktot * NC; e += blockDim.x) bst[e] = 0.0;
  __syncthreads();
  int k0 = 0;
  for (int a = ch.a_begin; a < ch.a_end; ++a) {
    const RsA X = ra[a];
    const PairDev PA = pairs[X.pair];
    for (int kk = threadIdx.x; kk < PA.k; kk += blockDim.x) cst[k0 + kk] = tab[PA.colA + kk];
    for (int q = X.e_begin; q < X.e_end; ++q) {
      const RsE E = re[q];
      const PairDev P = pairs[E.pair];
      for (int e = threadIdx.x; e < P.k * P.n; e += blockDim.x) {
        const int kk = e / P.n, c = e % P.n;
        bst[(k0 + kk) * NC + E.col + c] = B[P.b_off + tab[P.rowB + kk] + tab[P.colB + c]];
      }
    }
    k0 += PA.k;
  }
  __syncthreads();
  double acc[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) acc[c] = 0.0;
  if (r < ch.m) {
    k0 = 0;
    for (int a = ch.a_begin; a < ch.a_end; ++a) {
      const PairDev PA = pairs[ra[a].pair];
      const double* __restrict__ arow = A + PA.a_off + tab[PA.rowA + r];
      for (int kk = 0; kk < PA.k; ++kk) {
        const double x = arow[cst[k0 + kk]];
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[c] = fma(x, bst[(k0 + kk) * NC + c], acc[c]);
      }
      k0 += PA.k;
    }
    for (int o = ch.o_begin; o < ch.o_end; ++o) {
      const RsO O = ro[o];
      const OutDev out = outs[O.out];
      double* Cb = C + out.c_off + r;
#pragma unroll
      for (int c = 0; c < NC; ++c)
        if (c >= O.col && c < O.col + out.n) Cb[(int64_t)out.ldc * (c - O.col)] = alpha * acc[c];
    }
  }
}

// ---------------------------------------------------------------------------
// Mixed-precision path: tcgen05 (5th-generation tensor cores), kind::tf32.
//
// Two launches per contraction.  pack_tf32_ab converts every operand block
// once into TF32 hi/lo tiles (x = hi + lo, both rounded to nearest) stored in
// the exact K-major 128-byte-swizzled layout of a shared-memory MMA operand
// tile; grouped_tc_persist then feeds the tensor cores from those tiles with
// bulk copies and accumulates 128 x 128 output tiles in tensor memory (FP32).
// The split form issues hi*hi + hi*lo + lo*hi per k-step.
constexpr int TC_BM = 128;
constexpr int TC_BN = 128;
constexpr int TC_BK = 32;                        // fp32 elements = one 128-byte swizzle row
constexpr uint32_t TC_WAIT_LIMIT = 1u << 26;
static_assert(TC_BN == TC_BM, "packed tiles are 128 rows for both operands");

// Instruction descriptor: D f32, A/B tf32, both K-major, N = TC_BN, M = TC_BM.
constexpr uint32_t TC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_BN >> 3) << 17) |
                              ((uint32_t)(TC_BM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor, K-major with 128-byte swizzle: rows of 128
// bytes, 8-row groups 1024 bytes apart (stride byte offset), version 1.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1 << 16;              // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;    // stride byte offset
  d |= (uint64_t)1 << 46;              // descriptor version
  d |= (uint64_t)2 << 61;              // SWIZZLE_128B
  return d;
}

// Byte offset of element (row r, k) in a K-major 128B-swizzled tile.
__device__ __forceinline__ uint32_t sw128_off(int r, int k) {
  return (uint32_t)((r >> 3) * 1024 + (r & 7) * 128 + ((((k >> 2) ^ (r & 7))) << 4) + (k & 3) * 4);
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void mbar_init(uint32_t addr, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(addr), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t addr, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(addr), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait for the phase with the given parity; false on timeout
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t addr, uint32_t parity, uint32_t limit = TC_WAIT_LIMIT) {
  for (uint32_t it = 0; it < limit; ++it)
    if (mbar_try_wait(addr, parity)) return true;
  return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %3, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %4, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(accumulate), "r"(TC_IDESC)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

// ---- operand packing: FP64 blocks -> TF32 hi/lo tiles, pre-swizzled --------
// A packed tile holds 128 rows x 32 k of one operand block as TF32 hi
// (16 KB) followed by TF32 lo (16 KB), each laid out exactly as the K-major
// 128-byte-swizzled shared-memory tile the MMA reads, so one bulk copy moves
// it into shared memory unchanged.  Edges are zero-padded.  Tile (rt, kt) of
// a block sits at base + (rt * kt_count + kt) * 32 KB.
struct PackJob {
  int64_t x_off;             // block offset in the operand (elements)
  int64_t dst;               // packed block base (bytes)
  int32_t rows, K;           // logical rows (m or n) and k
  int32_t row_tab, k_tab;    // offset tables: element = X[x_off + tab[row_tab + r] + tab[k_tab + k]]
  int32_t kt_count;
  int32_t row_unit;          // rows have unit stride: walk them fastest
};
struct PackTile {
  int32_t job, rt, kt;
};
constexpr int TC_TILE_BYTES = 2 * TC_BM * TC_BK * 4;  // hi + lo = 32 KB

// ---- grouped tcgen05 GEMM over packed tiles ---------------------------------
// A block pair in packed form: the bases of its A and B packed blocks and its
// number of 32-wide k-chunks.  The GEMM kernel (grouped_tc_persist below)
// streams each chunk's A and B tiles into a TC_RING-stage ring of
// TC_RING_STAGE bytes with plain bulk copies.
struct PairTC {
  int64_t a_base, b_base;  // packed block bases (bytes)
  int32_t kt;              // k tiles of the pair
  int32_t pad;
};
constexpr int TC_RING = 3;
constexpr int TC_RING_STAGE = 4 * TC_BM * TC_BK * 4;  // A hi, A lo, B hi, B lo: 64 KB
constexpr size_t TC_BULK_SMEM = (size_t)TC_RING * TC_RING_STAGE + 1024;

__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(mbar)
               : "memory");
}

// ---- persistent form --------------------------------------------------------
// One CTA per SM walks the tiles blockIdx.x, blockIdx.x + gridDim.x, ...
// (longest first) with specialised warps: warp 0 (one thread) streams the
// packed tiles of every k-chunk of every tile into the TC_RING-stage ring,
// running ahead across tile boundaries; warp 1 (one thread) issues the MMAs
// into one of two 128-column TMEM accumulators, alternating per tile, and
// commits each stage to its empty barrier and each finished tile to the
// accumulator's full barrier; warps 2-5 drain a finished accumulator
// (tcgen05.ld, alpha * acc as FP64) while the MMAs of the next tile fill the
// other one, then release it through the accumulator's empty barrier (four
// arrivals).  A warp may read only its quarter of the 128 TMEM lanes (warp
// index mod 4), so warps 2, 3, 4, 5 cover lanes 64, 96, 0, 32.  Every wait is
// bounded; on timeout the CTA records TT_ERR_TIMEOUT, stops issuing, lets
// what it issued land (bounded) and frees TMEM.
constexpr int TC_P_THREADS = 192;
constexpr uint32_t TC_P_COLS = 2 * TC_BN;

__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}

template <bool SPLIT>
__global__ void __launch_bounds__(TC_P_THREADS, 1)
grouped_tc_persist(const TaskDev* __restrict__ tasks, int n_tasks, const OutDev* __restrict__ outs,
                   const PairTC* __restrict__ pairs, const uint8_t* __restrict__ packA,
                   const uint8_t* __restrict__ packB, double* __restrict__ C, double alpha, int* __restrict__ status,
                   int* __restrict__ ctx_status, uint32_t wait_limit) {
  extern __shared__ uint8_t tc_smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[TC_RING], empty_bar[TC_RING], accf_bar[2], acce_bar[2];
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int flag;
  __shared__ int issued, consumed, committed_tiles;

  const uint32_t sbase = (smem_u32(tc_smem_raw) + 1023u) & ~1023u;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t half = SPLIT ? (uint32_t)TC_TILE_BYTES : (uint32_t)(TC_TILE_BYTES / 2);  // bytes per operand tile

  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(TC_P_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int i = 0; i < TC_RING; ++i) {
      mbar_init(smem_u32(&full_bar[i]), 1);
      mbar_init(smem_u32(&empty_bar[i]), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(smem_u32(&accf_bar[b]), 1);
      mbar_init(smem_u32(&acce_bar[b]), 4);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    flag = 0;
    issued = 0;
    consumed = 0;
    committed_tiles = 0;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;

  if (warp == 0) {
    if (lane == 0) {  // producer
      int g = 0;
      for (int t = blockIdx.x; t < n_tasks && !flag; t += gridDim.x) {
        const TaskDev task = tasks[t];
        const int rt = task.m0 / TC_BM, nt = task.n0 / TC_BN;
        for (int p = task.p_begin; p < task.p_end && !flag; ++p) {
          const PairTC q = pairs[p];
          for (int kt = 0; kt < q.kt; ++kt, ++g) {
            const int s = g % TC_RING;
            if (g >= TC_RING &&
                !mbar_wait_bounded(smem_u32(&empty_bar[s]), (uint32_t)((g / TC_RING - 1) & 1), wait_limit)) {
              flag = 1;
              break;
            }
            const uint32_t st = sbase + s * TC_RING_STAGE;
            mbar_expect_tx(smem_u32(&full_bar[s]), 2 * half);
            bulk_g2s(st, packA + q.a_base + (int64_t)(rt * q.kt + kt) * TC_TILE_BYTES, half, smem_u32(&full_bar[s]));
            bulk_g2s(st + TC_TILE_BYTES, packB + q.b_base + (int64_t)(nt * q.kt + kt) * TC_TILE_BYTES, half,
                     smem_u32(&full_bar[s]));
            issued = g + 1;
          }
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      int g = 0, i = 0;
      for (int t = blockIdx.x; t < n_tasks && !flag; t += gridDim.x, ++i) {
        const TaskDev task = tasks[t];
        int nch = 0;
        for (int p = task.p_begin; p < task.p_end; ++p) nch += pairs[p].kt;
        const int b = i & 1;
        if (i >= 2 && !mbar_wait_bounded(smem_u32(&acce_bar[b]), (uint32_t)(((i >> 1) - 1) & 1), wait_limit)) {
          flag = 1;
          break;
        }
        tc_fence_after();
        const uint32_t acc_tm = tmem + (uint32_t)(b * TC_BN);
        for (int c = 0; c < nch; ++c, ++g) {
          const int s = g % TC_RING;
          if (!mbar_wait_bounded(smem_u32(&full_bar[s]), (uint32_t)((g / TC_RING) & 1), wait_limit)) {
            flag = 1;
            break;
          }
          tc_fence_after();
          const uint32_t ah = sbase + s * TC_RING_STAGE, al = ah + TC_TILE_BYTES / 2;
          const uint32_t bh = ah + TC_TILE_BYTES, bl = bh + TC_TILE_BYTES / 2;
#pragma unroll
          for (int kk = 0; kk < TC_BK / 8; ++kk) {
            const uint32_t adv = 32u * kk;
            const uint32_t acc = (c > 0 || kk > 0) ? 1u : 0u;
            if (SPLIT) {
              mma_tf32(acc_tm, sw128_desc(al + adv), sw128_desc(bh + adv), acc);
              mma_tf32(acc_tm, sw128_desc(ah + adv), sw128_desc(bl + adv), 1u);
              mma_tf32(acc_tm, sw128_desc(ah + adv), sw128_desc(bh + adv), 1u);
            } else {
              mma_tf32(acc_tm, sw128_desc(ah + adv), sw128_desc(bh + adv), acc);
            }
          }
          mma_commit(smem_u32(&empty_bar[s]));
          consumed = g + 1;
        }
        if (flag) break;
        if (nch > 0) mma_commit(smem_u32(&accf_bar[b]));
        else mbar_arrive(smem_u32(&accf_bar[b]));
        committed_tiles = i + 1;
      }
    }
  } else {  // epilogue, warps 2..5
    const int q4 = warp & 3;
    int i = 0;
    for (int t = blockIdx.x; t < n_tasks; t += gridDim.x, ++i) {
      // decisions are warp-uniform: the TMEM loads below are .sync.aligned
      if (__any_sync(0xffffffffu, flag != 0)) break;
      const TaskDev task = tasks[t];
      const OutDev out = outs[task.out];
      int nch = 0;
      for (int p = task.p_begin; p < task.p_end; ++p) nch += pairs[p].kt;
      const int b = i & 1;
      const bool ok = mbar_wait_bounded(smem_u32(&accf_bar[b]), (uint32_t)((i >> 1) & 1), wait_limit);
      if (!__all_sync(0xffffffffu, ok)) {
        if (lane == 0) flag = 1;
        break;
      }
      tc_fence_after();
      double* Cb = C + out.c_off;
      const int m = task.m0 + q4 * 32 + lane;
#pragma unroll
      for (int c16 = 0; c16 < TC_BN / 16; ++c16) {
        float v[16];
        if (nch > 0) {
          tmem_ld16(tmem + ((uint32_t)(q4 * 32) << 16) + (uint32_t)(b * TC_BN + c16 * 16), v);
        } else {
#pragma unroll
          for (int j = 0; j < 16; ++j) v[j] = 0.f;
        }
        if (m < out.m) {
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int n = task.n0 + c16 * 16 + j;
            if (n < out.n) Cb[m + (int64_t)out.ldc * n] = alpha * (double)v[j];
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&acce_bar[b]));
    }
  }
  __syncwarp();
  __syncthreads();
  if (tid == 0 && flag) {
    // let the copies that were issued but not consumed land and the last
    // committed MMAs finish before shared and tensor memory are released
    for (int g = consumed; g < issued; ++g)
      mbar_wait_bounded(smem_u32(&full_bar[g % TC_RING]), (uint32_t)((g / TC_RING) & 1));
    if (consumed > 0)
      mbar_wait_bounded(smem_u32(&empty_bar[(consumed - 1) % TC_RING]), (uint32_t)(((consumed - 1) / TC_RING) & 1));
    if (committed_tiles > 0) {  // the last tile commit's arrival
      const int il = committed_tiles - 1;
      mbar_wait_bounded(smem_u32(&accf_bar[il & 1]), (uint32_t)((il >> 1) & 1));
    }
    atomicExch(status, TT_ERR_TIMEOUT);
    atomicExch_system(ctx_status, TT_ERR_TIMEOUT);  // the context's mapped status word
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_P_COLS) : "memory");
}

// Both operands' packing in one launch: tiles [0, n_a) of A, then those of B.
template <bool SPLIT>
__global__ void __launch_bounds__(128)
pack_tf32_ab(const PackJob* __restrict__ jobsA, const PackTile* __restrict__ tilesA, int n_a,
             const PackJob* __restrict__ jobsB, const PackTile* __restrict__ tilesB, const int32_t* __restrict__ tab,
             const double* __restrict__ A, const double* __restrict__ B, uint8_t* __restrict__ pa,
             uint8_t* __restrict__ pb) {
  // the tile is assembled in shared memory at its swizzled offsets, then
  // written out with consecutive 16-byte stores (a thread's 16 bytes of a
  // row would otherwise land in a different 128-byte line per lane)
  __shared__ __align__(128) uint8_t st[TC_TILE_BYTES];
  const bool is_a = (int)blockIdx.x < n_a;
  const PackTile t = is_a ? tilesA[blockIdx.x] : tilesB[blockIdx.x - n_a];
  const PackJob J = is_a ? jobsA[t.job] : jobsB[t.job];
  const double* X = is_a ? A : B;
  const int tid = threadIdx.x;
  uint8_t* dst = (is_a ? pa : pb) + J.dst + (int64_t)(t.rt * J.kt_count + t.kt) * TC_TILE_BYTES;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int r = J.row_unit ? tid : (tid >> 3) + 16 * i;
    const int q = J.row_unit ? i : (tid & 7);
    const int gr = t.rt * TC_BM + r;
    double x[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int gk = t.kt * TC_BK + 4 * q + e;
      x[e] = (gr < J.rows && gk < J.K) ? X[J.x_off + tab[J.row_tab + gr] + tab[J.k_tab + gk]] : 0.0;
    }
    uint32_t h[4], l[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      h[e] = to_tf32(__double2float_rn(x[e]));
      l[e] = SPLIT ? to_tf32(__double2float_rn(x[e] - (double)__uint_as_float(h[e]))) : 0u;
    }
    const uint32_t o = sw128_off(r, 4 * q);
    *reinterpret_cast<uint4*>(st + o) = make_uint4(h[0], h[1], h[2], h[3]);
    if (SPLIT) *reinterpret_cast<uint4*>(st + TC_TILE_BYTES / 2 + o) = make_uint4(l[0], l[1], l[2], l[3]);
  }
  __syncthreads();
  constexpr int NV = (SPLIT ? TC_TILE_BYTES : TC_TILE_BYTES / 2) / 16;
#pragma unroll 4
  for (int v = tid; v < NV; v += blockDim.x)
    reinterpret_cast<uint4*>(dst)[v] = reinterpret_cast<const uint4*>(st)[v];
}

// Cost model of the *_AUTO precisions: predicted device time (microseconds)
// of one exec of a contraction in `prec` (FP64 DMMA, or a tcgen05 kind with
// its two packing launches).  Work is counted on padded tiles (an output tile
// runs every pair of its block over k rounded up to the k-step); the grid is
// bound by the total at the full-chip rate, by its longest tile at one SM's
// rate, and by its DRAM bytes.  The tensor-core form moves each operand
// element three more times (read by the packer, written packed, read packed),
// so a contraction with a small k -- the bandwidth-bound middle contraction
// of H_eff*x and of the environment update -- stays in FP64, which is exact
// to more digits and faster there (measured at bond dimension 1024 on the
// J1-J2 cylinder: 354 us FP64 against 685 us packed tensor-core form, while
// L*x and *R take 141 and 161 us on the tensor cores against 301 and 473 us
// in FP64).  Rates are the measured single-block throughputs of the two
// kernels on B200 (4096^3: DMMA 26 TFLOP/s, tcgen05 690 TFLOP/s of TF32
// products).
double predict_us(const tt_out_block* outs, int n_out, const std::vector<PairDev>& hp,
                  const std::vector<int>& first, int prec, int num_sms, int keep = 0) {
  constexpr double kDmmaRate = 27e12, kTcRate = 650e12, kHbm = 6.0e12, kLaunchUs = 2.5;
  const bool tc = prec != TT_PREC_FP64;
  // the DMMA kernel stops at k rounded up to its k-step of 4; the tcgen05
  // kernel runs whole 32-wide k-chunks
  const int tm = tc ? TC_BM : BM, tn = tc ? TC_BN : BN, tk = tc ? TC_BK : 4;
  const double rate = tc ? (prec == TT_PREC_TF32X3 ? kTcRate / 3.0 : kTcRate) : kDmmaRate;
  auto up = [](int x, int t) { return (double)((x + t - 1) / t) * t; };
  double total = 0.0, longest = 0.0, bytes = 0.0;
  std::map<int64_t, std::pair<double, double>> ua, ub;  // distinct operand blocks: (elements, padded elements)
  for (int o = 0; o < n_out; ++o) {
    double kpad = 0.0;
    for (int i = first[o]; i < first[o + 1]; ++i) {
      const PairDev& P = hp[i];
      kpad += up(P.k, tk);
      ua.emplace(P.a_off, std::make_pair((double)P.m * P.k, up(P.m, tm) * up(P.k, tk)));
      ub.emplace(P.b_off, std::make_pair((double)P.n * P.k, up(P.n, tn) * up(P.k, tk)));
    }
    const double tiles = up(outs[o].m, tm) / tm * (up(outs[o].n, tn) / tn);
    const double task = 2.0 * tm * tn * kpad;
    total += tiles * task;
    if (tiles > 0) longest = std::max(longest, task);
    bytes += 8.0 * outs[o].m * outs[o].n;  // C
  }
  // FP64 reads every operand element once from DRAM; the tensor-core form
  // also writes the packed tiles (hi + lo: 8 bytes per padded element, TF32:
  // 4) and reads them back
  const double packed = prec == TT_PREC_TF32X3 ? 8.0 : 4.0;
  // an operand kept packed across execs (keep bit 0: A, bit 1: B) is packed
  // once for kKeptUses of them
  constexpr double kKeptUses = 4.0;
  for (int w = 0; w < 2; ++w) {
    const double share = ((keep >> w) & 1) ? 1.0 / kKeptUses : 1.0;
    for (const auto& kv : (w == 0 ? ua : ub))
      bytes += 8.0 * kv.second.first + (tc ? 2.0 * packed * kv.second.second * share : 0.0);
  }
  const double t = std::max({total / rate, longest / (rate / std::max(1, num_sms)), bytes / kHbm});
  return t * 1e6 + (tc ? 3 : 1) * kLaunchUs;
}

}  // namespace

struct tt_plan {
  int precision = TT_PREC_FP64;
  bool skinny = false;      // FP64 plan run by skinny_dgemm (row tasks of SK_ROWS)
  int skinny_nc = SK_N;     // its widest output block (the kernel instance covers it)
  int64_t skinny_ktot = 0;  // the largest sum of k over one output block's pairs
  // row-stationary form of a skinny plan (skinny_rs), when its chunks are valid
  bool rs = false;
  int rs_n_tasks = 0, rs_nc = SK_N;
  int64_t rs_ktot = 0;
  TaskDev* d_rs_tasks = nullptr;
  RsChunk* d_rs_chunks = nullptr;
  RsA* d_rs_a = nullptr;
  RsE* d_rs_e = nullptr;
  RsO* d_rs_o = nullptr;
  int* d_status = nullptr;  // tensor-core path: TT_OK or TT_ERR_TIMEOUT
  // tensor-core path: packing jobs and tiles of the unique A / B blocks, the
  // pairs in packed form, and the packed sizes (buffers are taken from the
  // stream-ordered pool for each exec)
  PackJob* d_jobsA = nullptr;
  PackJob* d_jobsB = nullptr;
  PackTile* d_tilesA = nullptr;
  PackTile* d_tilesB = nullptr;
  PairTC* d_pairtc = nullptr;
  int n_tilesA = 0, n_tilesB = 0;
  int64_t bytesA = 0, bytesB = 0;
  int n_tasks = 0;
  int n_pairs = 0;
  int n_out = 0;
  double flops = 0.0;
  int64_t dev_bytes = 0;  // device memory the plan holds (tables, tasks, packing jobs)
  // tensor-core path: packed operands kept between execs (tt_contract_exec_keep)
  // and the operand each was packed from; released by tt_plan_release_packed
  mutable uint8_t* kept[2] = {nullptr, nullptr};
  mutable const double* kept_src[2] = {nullptr, nullptr};
  // packing buffers reused across execs for operands packed afresh each time
  // (keep bits 2 and 3), so that a run of execs allocates them once
  mutable uint8_t* scratch[2] = {nullptr, nullptr};
  TaskDev* d_tasks = nullptr;
  OutDev* d_outs = nullptr;
  PairDev* d_pairs = nullptr;
  int32_t* d_tab = nullptr;
};

extern "C" {

// Host seconds of the planner's stages on this thread (tt_contract_plan_timers):
// pair tables, precision choice, tile tasks and the row-stationary chunks,
// tensor-core packing jobs, device tables and uploads.
static thread_local double g_plan_stage_s[5];
struct PlanLap {
  std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
  int stage = 0;
  void operator()(int k) {
    const auto now = std::chrono::steady_clock::now();
    g_plan_stage_s[k] += std::chrono::duration<double>(now - t).count();
    t = now;
    stage = k + 1;
  }
  ~PlanLap() {
    if (stage < 5) (*this)(4);
  }
};

int tt_contract_plan(tt_ctx* ctx, const tt_out_block* outs, int n_out,
                     const tt_block_pair* pairs, int n_pairs, int precision,
                     tt_plan** plan_out) {
  return tt_contract_plan_keep(ctx, outs, n_out, pairs, n_pairs, precision, 0, plan_out);
}

int tt_contract_plan_keep(tt_ctx* ctx, const tt_out_block* outs, int n_out, const tt_block_pair* pairs,
                          int n_pairs, int precision, int keep, tt_plan** plan_out) {
  PlanLap lap;
  TT_REQUIRE(ctx && plan_out, "tt_contract_plan: null argument");
  TT_REQUIRE(n_out >= 0 && n_pairs >= 0, "tt_contract_plan: negative count");
  TT_REQUIRE(precision >= TT_PREC_FP64 && precision <= TT_PREC_TF32X3_AUTO,
             "tt_contract_plan: unsupported precision");
  const bool automatic = precision == TT_PREC_TF32_AUTO || precision == TT_PREC_TF32X3_AUTO;
  if (automatic) precision = precision == TT_PREC_TF32_AUTO ? TT_PREC_TF32 : TT_PREC_TF32X3;
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
  std::map<std::vector<int64_t>, int32_t> tab_of;  // table contents -> its offset
  std::vector<int64_t> tab_key;
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
    // an offset table is a function of (length, dims, strides) alone: pairs
    // that address the same rows or columns of a block share one table
    auto add_job = [&](int len, int nmodes, const int32_t* dims, const int64_t* strides) {
      tab_key.assign({(int64_t)len, (int64_t)nmodes});
      for (int i = 0; i < nmodes; ++i) {
        tab_key.push_back(dims[i]);
        tab_key.push_back(strides[i]);
      }
      auto hit = tab_of.find(tab_key);
      if (hit != tab_of.end()) return hit->second;
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
      tab_of.emplace(tab_key, J.dst);
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
  lap(0);
  for (int o = 0; o < n_out; ++o) first[o + 1] += first[o];
  // FP64 unless the tensor-core form is predicted clearly (20 %) faster: the
  // model is coarse, and FP64 is the more accurate of the two
  if (automatic && predict_us(outs, n_out, hp, first, precision, ctx->num_sms, keep) >
                       0.8 * predict_us(outs, n_out, hp, first, TT_PREC_FP64, ctx->num_sms))
    precision = TT_PREC_FP64;
  lap(1);
  const bool tc = precision != TT_PREC_FP64;
  // FP64 plans whose output blocks are at most SK_N wide and whose pairs
  // contract at most SK_K elements run on the skinny kernel
  bool skinny = !tc && n_pairs > 0;
  for (int o = 0; o < n_out && skinny; ++o) skinny = outs[o].n <= SK_N;
  for (int i = 0; i < n_pairs && skinny; ++i) skinny = hp[i].k <= SK_K && hp[i].n <= SK_N;
  const int tile_m = tc ? TC_BM : (skinny ? SK_ROWS : BM), tile_n = tc ? TC_BN : (skinny ? SK_N : BN);
  // tile tasks, longest first (LPT) so heavy blocks start early
  std::vector<TaskDev> tasks;
  std::vector<int64_t> tcost;
  for (int o = 0; o < n_out; ++o) {
    TT_REQUIRE(outs[o].m >= 0 && outs[o].n >= 0 && outs[o].ldc >= outs[o].m,
               "tt_contract_plan: bad output block");
    for (int m0 = 0; m0 < outs[o].m; m0 += tile_m)
      for (int n0 = 0; n0 < outs[o].n; n0 += tile_n) {
        TaskDev t{o, m0, n0, first[o], first[o + 1]};
        tasks.push_back(t);
        tcost.push_back(work[o] + 1);
      }
  }
  std::vector<int> torder(tasks.size());
  std::iota(torder.begin(), torder.end(), 0);
  bool rs_ok = false;
  std::vector<RsChunk> rs_chunks;
  std::vector<RsA> rs_a;
  std::vector<RsE> rs_e;
  std::vector<RsO> rs_o;
  std::vector<TaskDev> rs_tasks;
  int64_t rs_ktot = 0;
  if (skinny) {
    // The skinny kernel is bound by reading A, and every output block that
    // shares A's blocks (the same rows, other column sectors) reads them
    // again.  Tasks of such output blocks are interleaved by row tile, so the
    // CTAs that run together read the same A rows and all but the first read
    // hit L2.  Groups: output blocks linked through a shared A block
    // (union-find on the pairs' A offsets), heaviest group first.
    std::vector<int> parent(n_out);
    std::iota(parent.begin(), parent.end(), 0);
    auto root = [&](int o) {
      int r = o;
      while (parent[r] != r) r = parent[r];
      while (parent[o] != r) {  // path compression
        const int up = parent[o];
        parent[o] = r;
        o = up;
      }
      return r;
    };
    std::unordered_map<int64_t, int> owner;
    for (int o = 0; o < n_out; ++o)
      for (int i = first[o]; i < first[o + 1]; ++i) {
        auto it = owner.emplace(hp[i].a_off, o).first;
        const int ra = root(it->second), rb = root(o);
        if (ra != rb) parent[rb] = ra;
      }
    std::vector<int> groot(n_out);
    for (int o = 0; o < n_out; ++o) groot[o] = root(o);
    std::vector<int64_t> gcost(n_out, 0);
    for (int o = 0; o < n_out; ++o) gcost[groot[o]] += work[o] + 1;
    // row-stationary chunks (skinny_rs): a group's outputs in order, at most
    // SK_N combined columns each; valid when the group's outputs share their
    // rows and every A block is read through the same tables by all its pairs
    rs_ok = true;
    std::unordered_map<int64_t, int> a_first;  // a_off -> first pair reading it
    for (int i = 0; i < n_pairs && rs_ok; ++i) {
      auto it = a_first.emplace(hp[i].a_off, i).first;
      const tt_block_pair& x = pairs[order[it->second]];
      const tt_block_pair& y = pairs[order[i]];
      rs_ok = hp[i].m == hp[it->second].m && hp[i].k == hp[it->second].k && x.n_m == y.n_m && x.n_k == y.n_k;
      for (int d = 0; d < x.n_m && rs_ok; ++d)
        rs_ok = x.m_dims[d] == y.m_dims[d] && x.a_m_stride[d] == y.a_m_stride[d];
      for (int d = 0; d < x.n_k && rs_ok; ++d)
        rs_ok = x.k_dims[d] == y.k_dims[d] && x.a_k_stride[d] == y.a_k_stride[d];
    }
    std::vector<std::vector<int>> members(n_out);
    for (int o = 0; o < n_out; ++o) members[groot[o]].push_back(o);
    for (int g = 0; g < n_out && rs_ok; ++g)
      for (int o : members[g]) rs_ok = rs_ok && outs[o].m == outs[members[g][0]].m;
    std::vector<int> gorder;
    for (int g = 0; g < n_out; ++g)
      if (!members[g].empty()) gorder.push_back(g);
    std::stable_sort(gorder.begin(), gorder.end(), [&](int a, int b) { return gcost[a] > gcost[b]; });
    for (int g : gorder) {
      if (!rs_ok) break;
      size_t c0 = rs_chunks.size();
      auto open_chunk = [&]() {
        RsChunk c{(int32_t)rs_a.size(), (int32_t)rs_a.size(), (int32_t)rs_o.size(), (int32_t)rs_o.size(),
                  (int32_t)outs[members[g][0]].m, 0};
        rs_chunks.push_back(c);
      };
      open_chunk();
      int cols = 0;
      std::unordered_map<int64_t, int> a_slot;  // a_off -> index in rs_a within the chunk
      std::vector<std::vector<RsE>> ents;       // per rs_a entry of the chunk
      auto close_chunk = [&]() {
        RsChunk& c = rs_chunks.back();
        for (size_t i = 0; i < ents.size(); ++i) {
          rs_a[c.a_begin + i].e_begin = (int32_t)rs_e.size();
          rs_e.insert(rs_e.end(), ents[i].begin(), ents[i].end());
          rs_a[c.a_begin + i].e_end = (int32_t)rs_e.size();
          c.ktot += hp[rs_a[c.a_begin + i].pair].k;
        }
        c.a_end = (int32_t)rs_a.size();
        c.o_end = (int32_t)rs_o.size();
        ents.clear();
        a_slot.clear();
      };
      for (int o : members[g]) {
        if (cols + outs[o].n > RS_COLS && cols > 0) {
          close_chunk();
          open_chunk();
          cols = 0;
        }
        rs_o.push_back(RsO{o, cols});
        for (int i = first[o]; i < first[o + 1]; ++i) {
          auto it = a_slot.find(hp[i].a_off);
          if (it == a_slot.end()) {
            it = a_slot.emplace(hp[i].a_off, (int)ents.size()).first;
            rs_a.push_back(RsA{i, 0, 0});
            ents.emplace_back();
          }
          ents[it->second].push_back(RsE{i, cols});
        }
        cols += outs[o].n;
      }
      close_chunk();
      // tasks: the group's row tiles, its chunks interleaved within a tile
      const int m = outs[members[g][0]].m;
      for (int m0 = 0; m0 < m; m0 += SK_ROWS)
        for (size_t c = c0; c < rs_chunks.size(); ++c) rs_tasks.push_back(TaskDev{(int32_t)c, m0, 0, 0, 0});
    }
    for (const RsChunk& c : rs_chunks) rs_ktot = std::max<int64_t>(rs_ktot, c.ktot);
    for (const RsO& x : rs_o) rs_ok = rs_ok && outs[x.out].n <= RS_COLS;  // every chunk fits its instance
    if (rs_ok) rs_ok = rs_ktot * (int64_t)(RS_COLS * sizeof(double) + sizeof(int32_t)) <= SK_STAGE_BYTES;
    // the per-pair skinny kernel (no row-stationary chunks): tasks of a group
    // interleaved by row tile, heaviest group first; with the chunks, the
    // tile tasks are not run and stay in their plain order
    if (!rs_ok)
      std::stable_sort(torder.begin(), torder.end(), [&](int a, int b) {
        const int ga = groot[tasks[a].out], gb = groot[tasks[b].out];
        if (ga != gb) return gcost[ga] != gcost[gb] ? gcost[ga] > gcost[gb] : ga < gb;
        if (tasks[a].m0 != tasks[b].m0) return tasks[a].m0 < tasks[b].m0;
        return tasks[a].out < tasks[b].out;
      });
  } else {
    std::stable_sort(torder.begin(), torder.end(), [&](int a, int b) { return tcost[a] > tcost[b]; });
  }
  std::vector<TaskDev> tsorted(tasks.size());
  for (size_t i = 0; i < tasks.size(); ++i) tsorted[i] = tasks[torder[i]];
  std::vector<OutDev> ho(n_out);
  for (int o = 0; o < n_out; ++o) ho[o] = OutDev{outs[o].c_off, outs[o].m, outs[o].n, outs[o].ldc};

  lap(2);
  // tensor-core path: one packing job per distinct operand block
  std::vector<PackJob> ja, jb;
  std::vector<PackTile> ta, tb;
  std::vector<PairTC> ptc;
  int64_t bytesA = 0, bytesB = 0;
  if (tc) {
    std::map<int64_t, int> ua, ub;
    ptc.resize(n_pairs);
    for (int ii = 0; ii < n_pairs; ++ii) {
      const PairDev& P = hp[ii];
      const int kt = (P.k + TC_BK - 1) / TC_BK;
      auto ia = ua.find(P.a_off);
      if (ia == ua.end()) {
        const int rt = (P.m + TC_BM - 1) / TC_BM;
        ja.push_back(PackJob{P.a_off, bytesA, P.m, P.k, P.rowA, P.colA, kt, P.a_mfast});
        for (int r = 0; r < rt; ++r)
          for (int k = 0; k < kt; ++k) ta.push_back(PackTile{(int32_t)ja.size() - 1, r, k});
        bytesA += (int64_t)rt * kt * TC_TILE_BYTES;
        ia = ua.emplace(P.a_off, (int)ja.size() - 1).first;
      }
      auto ib = ub.find(P.b_off);
      if (ib == ub.end()) {
        const int rt = (P.n + TC_BN - 1) / TC_BN;
        jb.push_back(PackJob{P.b_off, bytesB, P.n, P.k, P.colB, P.rowB, kt, P.b_kfast ? 0 : 1});
        for (int r = 0; r < rt; ++r)
          for (int k = 0; k < kt; ++k) tb.push_back(PackTile{(int32_t)jb.size() - 1, r, k});
        bytesB += (int64_t)rt * kt * TC_TILE_BYTES;
        ib = ub.emplace(P.b_off, (int)jb.size() - 1).first;
      }
      ptc[ii] = PairTC{ja[ia->second].dst, jb[ib->second].dst, kt, 0};
    }
    TT_REQUIRE(ta.size() < (1u << 31) && tb.size() < (1u << 31), "tt_contract_plan: too many packed tiles");
  }

  tt_plan* plan = new tt_plan();
  plan->precision = precision;
  plan->skinny = skinny;
  if (skinny) {
    int wmax = 1;
    for (int o = 0; o < n_out; ++o) wmax = std::max(wmax, outs[o].n);
    plan->skinny_nc = wmax;
    for (int o = 0; o < n_out; ++o) {
      int64_t kt = 0;
      for (int i = first[o]; i < first[o + 1]; ++i) kt += hp[i].k;
      plan->skinny_ktot = std::max(plan->skinny_ktot, kt);
    }
  }
  plan->n_tilesA = (int)ta.size();
  plan->n_tilesB = (int)tb.size();
  plan->bytesA = bytesA;
  plan->bytesB = bytesB;
  plan->n_tasks = (int)tsorted.size();
  plan->n_pairs = n_pairs;
  plan->n_out = n_out;
  plan->flops = flops;
  plan->dev_bytes = (int64_t)(sizeof(TaskDev) * tsorted.size() + sizeof(OutDev) * ho.size() +
                              sizeof(PairDev) * hp.size() + sizeof(int32_t) * (size_t)tab_len +
                              sizeof(PackJob) * (ja.size() + jb.size()) + sizeof(PackTile) * (ta.size() + tb.size()) +
                              sizeof(PairTC) * ptc.size());
  plan->d_tasks = tt::pool_alloc<TaskDev>(ctx, tsorted.size());
  plan->d_outs = tt::pool_alloc<OutDev>(ctx, ho.size());
  plan->d_pairs = tt::pool_alloc<PairDev>(ctx, hp.size());
  plan->d_tab = tt::pool_alloc<int32_t>(ctx, (size_t)tab_len);
  plan->d_status = tt::pool_alloc<int>(ctx, 1);
  TableJob* d_jobs = tt::pool_alloc<TableJob>(ctx, jobs.size());
  bool tc_ok = true;
  if (tc) {
    plan->d_jobsA = tt::pool_alloc<PackJob>(ctx, ja.size());
    plan->d_jobsB = tt::pool_alloc<PackJob>(ctx, jb.size());
    plan->d_tilesA = tt::pool_alloc<PackTile>(ctx, ta.size());
    plan->d_tilesB = tt::pool_alloc<PackTile>(ctx, tb.size());
    plan->d_pairtc = tt::pool_alloc<PairTC>(ctx, ptc.size());
    tc_ok = (ja.empty() || plan->d_jobsA) && (jb.empty() || plan->d_jobsB) && (ta.empty() || plan->d_tilesA) &&
            (tb.empty() || plan->d_tilesB) && (ptc.empty() || plan->d_pairtc);
  }
  if (!plan->d_tasks || !plan->d_outs || !plan->d_pairs || !plan->d_tab || !plan->d_status || !d_jobs || !tc_ok) {
    tt_plan_destroy(ctx, plan);
    tt::pool_free(ctx, d_jobs);
    return tt::fail(TT_ERR_OOM, "tt_contract_plan: device allocation failed");
  }
  cudaStream_t s = ctx->stream;
  TT_CUDA(cudaMemsetAsync(plan->d_status, 0, sizeof(int), s));
  lap(3);
  // staged copies: the host vectors may die at return without stalling the stream
  TT_CUDA(tt::h2d_async(ctx, plan->d_tasks, tsorted.data(), sizeof(TaskDev) * tsorted.size()));
  TT_CUDA(tt::h2d_async(ctx, plan->d_outs, ho.data(), sizeof(OutDev) * ho.size()));
  TT_CUDA(tt::h2d_async(ctx, plan->d_pairs, hp.data(), sizeof(PairDev) * hp.size()));
  TT_CUDA(tt::h2d_async(ctx, d_jobs, jobs.data(), sizeof(TableJob) * jobs.size()));
  if (tc) {
    TT_CUDA(tt::h2d_async(ctx, plan->d_jobsA, ja.data(), sizeof(PackJob) * ja.size()));
    TT_CUDA(tt::h2d_async(ctx, plan->d_jobsB, jb.data(), sizeof(PackJob) * jb.size()));
    TT_CUDA(tt::h2d_async(ctx, plan->d_tilesA, ta.data(), sizeof(PackTile) * ta.size()));
    TT_CUDA(tt::h2d_async(ctx, plan->d_tilesB, tb.data(), sizeof(PackTile) * tb.size()));
    TT_CUDA(tt::h2d_async(ctx, plan->d_pairtc, ptc.data(), sizeof(PairTC) * ptc.size()));
  }
  if (!jobs.empty()) {
    expand_tables<<<(unsigned)jobs.size(), 128, 0, s>>>(d_jobs, (int)jobs.size(), plan->d_tab);
    TT_LAUNCH_CHECK(ctx);
  }
  tt::pool_free(ctx, d_jobs);  // stream-ordered: freed after expand_tables ran
  if (rs_ok && !rs_tasks.empty()) {
    plan->d_rs_tasks = tt::pool_alloc<TaskDev>(ctx, rs_tasks.size());
    plan->d_rs_chunks = tt::pool_alloc<RsChunk>(ctx, rs_chunks.size());
    plan->d_rs_a = tt::pool_alloc<RsA>(ctx, rs_a.size());
    plan->d_rs_e = tt::pool_alloc<RsE>(ctx, rs_e.size());
    plan->d_rs_o = tt::pool_alloc<RsO>(ctx, rs_o.size());
    if (plan->d_rs_tasks && plan->d_rs_chunks && plan->d_rs_a && plan->d_rs_e && plan->d_rs_o) {
      TT_CUDA(tt::h2d_async(ctx, plan->d_rs_tasks, rs_tasks.data(), sizeof(TaskDev) * rs_tasks.size()));
      TT_CUDA(tt::h2d_async(ctx, plan->d_rs_chunks, rs_chunks.data(), sizeof(RsChunk) * rs_chunks.size()));
      TT_CUDA(tt::h2d_async(ctx, plan->d_rs_a, rs_a.data(), sizeof(RsA) * rs_a.size()));
      TT_CUDA(tt::h2d_async(ctx, plan->d_rs_e, rs_e.data(), sizeof(RsE) * rs_e.size()));
      TT_CUDA(tt::h2d_async(ctx, plan->d_rs_o, rs_o.data(), sizeof(RsO) * rs_o.size()));
      plan->rs = true;
      plan->rs_n_tasks = (int)rs_tasks.size();
      plan->rs_ktot = rs_ktot;
      int wmax = 1;
      for (const RsChunk& c : rs_chunks) {
        int w = 0;
        for (int o = c.o_begin; o < c.o_end; ++o) w += outs[rs_o[o].out].n;
        wmax = std::max(wmax, w);
      }
      plan->rs_nc = wmax;
      plan->dev_bytes += (int64_t)(sizeof(TaskDev) * rs_tasks.size() + sizeof(RsChunk) * rs_chunks.size() +
                                   sizeof(RsA) * rs_a.size() + sizeof(RsE) * rs_e.size() + sizeof(RsO) * rs_o.size());
    }
  }
  *plan_out = plan;
  return TT_OK;
}

int tt_contract_exec(tt_ctx* ctx, const tt_plan* plan, const double* A, const double* B,
                     double* C, double alpha) {
  return tt_contract_exec_keep(ctx, plan, A, B, C, alpha, 0);
}

int tt_plan_release_packed(tt_ctx* ctx, const tt_plan* plan) {
  TT_REQUIRE(ctx && plan, "tt_plan_release_packed: null argument");
  for (int w = 0; w < 2; ++w) {
    tt::pool_free(ctx, plan->kept[w]);
    plan->kept[w] = nullptr;
    plan->kept_src[w] = nullptr;
    tt::pool_free(ctx, plan->scratch[w]);
    plan->scratch[w] = nullptr;
  }
  return TT_OK;
}

int tt_contract_exec_keep(tt_ctx* ctx, const tt_plan* plan, const double* A, const double* B, double* C,
                          double alpha, int keep) {
  TT_REQUIRE(ctx && plan, "tt_contract_exec: null argument");
  if (plan->n_tasks == 0) return TT_OK;
  static thread_local uint64_t attr_set = 0;  // per host thread and device
  if (tt::first_on_device(attr_set, ctx->device)) {
    TT_CUDA(cudaFuncSetAttribute(grouped_dgemm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)SMEM_BYTES));
    TT_CUDA(cudaFuncSetAttribute(grouped_tc_persist<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)TC_BULK_SMEM));
    TT_CUDA(cudaFuncSetAttribute(grouped_tc_persist<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)TC_BULK_SMEM));
  }
  if (plan->precision == TT_PREC_FP64) {
    if (plan->rs) {
      const int nc = plan->rs_nc <= 4 ? 4 : plan->rs_nc <= 8 ? 8 : plan->rs_nc <= 16 ? 16 : 32;
      const size_t dyn = (size_t)(plan->rs_ktot * (int64_t)(nc * sizeof(double) + sizeof(int32_t)));
      using RsFn = void (*)(const TaskDev*, const RsChunk*, const RsA*, const RsE*, const RsO*, const OutDev*,
                            const PairDev*, const int32_t*, const double*, const double*, double*, double);
      const int which = nc == 4 ? 0 : nc == 8 ? 1 : nc == 16 ? 2 : 3;
      const RsFn fns[4] = {skinny_rs<4>, skinny_rs<8>, skinny_rs<16>, skinny_rs<32>};
      static thread_local uint64_t rs_attr[4] = {0, 0, 0, 0};  // per instance, per host thread and device
      if (tt::first_on_device(rs_attr[which], ctx->device))
        TT_CUDA(cudaFuncSetAttribute(fns[which], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SK_STAGE_BYTES));
      fns[which]<<<plan->rs_n_tasks, SK_ROWS, dyn, ctx->stream>>>(
          plan->d_rs_tasks, plan->d_rs_chunks, plan->d_rs_a, plan->d_rs_e, plan->d_rs_o, plan->d_outs,
          plan->d_pairs, plan->d_tab, A, B, C, alpha);
    } else if (plan->skinny) {
      const int nc = plan->skinny_nc <= 4 ? 4 : plan->skinny_nc <= 8 ? 8 : plan->skinny_nc <= 16 ? 16 : 32;
      // every pair of a task staged at once when the widest task fits
      const int64_t need = plan->skinny_ktot * (int64_t)(nc * sizeof(double) + sizeof(int32_t));
      const bool staged = need <= SK_STAGE_BYTES;
      const size_t dyn = staged ? (size_t)need : 0;
      using SkinnyFn = void (*)(const TaskDev*, const OutDev*, const PairDev*, const int32_t*, const double*,
                                const double*, double*, double, int);
      const int which = nc == 4 ? 0 : nc == 8 ? 1 : nc == 16 ? 2 : 3;
      const SkinnyFn fns[4] = {skinny_dgemm<4>, skinny_dgemm<8>, skinny_dgemm<16>, skinny_dgemm<32>};
      static thread_local uint64_t attr[4] = {0, 0, 0, 0};  // per instance, per host thread and device
      if (tt::first_on_device(attr[which], ctx->device))
        TT_CUDA(cudaFuncSetAttribute(fns[which], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SK_STAGE_BYTES));
      fns[which]<<<plan->n_tasks, SK_ROWS, dyn, ctx->stream>>>(plan->d_tasks, plan->d_outs, plan->d_pairs,
                                                              plan->d_tab, A, B, C, alpha, staged ? 1 : 0);
    } else
      grouped_dgemm<<<plan->n_tasks, THREADS, SMEM_BYTES, ctx->stream>>>(
          plan->d_tasks, plan->d_outs, plan->d_pairs, plan->d_tab, A, B, C, alpha);
    TT_LAUNCH_CHECK(ctx);
    return TT_OK;
  }
  // pack the operands into tensor-core tiles (pool buffers, released in
  // stream order); an operand kept from an earlier exec of this plan, packed
  // from the same source, is reused as it is
  const bool split = plan->precision == TT_PREC_TF32X3;
  const double* src[2] = {A, B};
  const int64_t bytes[2] = {plan->bytesA, plan->bytesB};
  uint8_t* pk[2] = {nullptr, nullptr};
  bool fresh[2] = {false, false};
  bool from_scratch[2] = {false, false};
  for (int w = 0; w < 2; ++w) {
    const bool k = (keep >> w) & 1;
    if (k && plan->kept[w] && plan->kept_src[w] == src[w]) {
      pk[w] = plan->kept[w];
      continue;
    }
    if (k && plan->kept[w]) {  // kept from another source: stale
      tt::pool_free(ctx, plan->kept[w]);
      plan->kept[w] = nullptr;
      plan->kept_src[w] = nullptr;
    }
    fresh[w] = true;
    if (!k && ((keep >> (2 + w)) & 1)) {  // repacked every exec into a buffer the plan keeps
      if (!plan->scratch[w]) plan->scratch[w] = tt::pool_alloc<uint8_t>(ctx, (size_t)std::max<int64_t>(bytes[w], 16));
      pk[w] = plan->scratch[w];
      from_scratch[w] = true;
      continue;
    }
    pk[w] = tt::pool_alloc<uint8_t>(ctx, (size_t)std::max<int64_t>(bytes[w], 16));
  }
  uint8_t* pa = pk[0];
  uint8_t* pb = pk[1];
  if (!pa || !pb) {
    if (fresh[0] && !from_scratch[0]) tt::pool_free(ctx, pa);
    if (fresh[1] && !from_scratch[1]) tt::pool_free(ctx, pb);
    return tt::fail(TT_ERR_OOM, "tt_contract_exec: packed operand allocation failed");
  }
  {
    // one launch for the operands that need packing: tiles [0, na) of A, then those of B
    const int na = fresh[0] ? plan->n_tilesA : 0, nb = fresh[1] ? plan->n_tilesB : 0;
    if (na + nb > 0) {
      const unsigned nt = (unsigned)(na + nb);
      if (split)
        pack_tf32_ab<true><<<nt, 128, 0, ctx->stream>>>(plan->d_jobsA, plan->d_tilesA, na, plan->d_jobsB,
                                                         plan->d_tilesB, plan->d_tab, A, B, pa, pb);
      else
        pack_tf32_ab<false><<<nt, 128, 0, ctx->stream>>>(plan->d_jobsA, plan->d_tilesA, na, plan->d_jobsB,
                                                          plan->d_tilesB, plan->d_tab, A, B, pa, pb);
      TT_LAUNCH_CHECK(ctx);
    }
  }
  const unsigned grid = (unsigned)std::min(plan->n_tasks, std::max(1, ctx->num_sms));
  if (split)
    grouped_tc_persist<true><<<grid, TC_P_THREADS, TC_BULK_SMEM, ctx->stream>>>(
        plan->d_tasks, plan->n_tasks, plan->d_outs, plan->d_pairtc, pa, pb, C, alpha, plan->d_status,
        ctx->d_dev_status, ctx->wait_limit);
  else
    grouped_tc_persist<false><<<grid, TC_P_THREADS, TC_BULK_SMEM, ctx->stream>>>(
        plan->d_tasks, plan->n_tasks, plan->d_outs, plan->d_pairtc, pa, pb, C, alpha, plan->d_status,
        ctx->d_dev_status, ctx->wait_limit);
  cudaError_t le = cudaGetLastError();
  for (int w = 0; w < 2; ++w) {
    if (!fresh[w] || from_scratch[w]) continue;
    if ((keep >> w) & 1) {
      plan->kept[w] = pk[w];
      plan->kept_src[w] = src[w];
    } else {
      tt::pool_free(ctx, pk[w]);
    }
  }
  if (le != cudaSuccess) return tt::cuda_fail(le, "tt_contract_exec: tensor-core launch", __FILE__, __LINE__);
  tt::count_launch(ctx);
  return TT_OK;
}

int tt_plan_destroy(tt_ctx* ctx, tt_plan* plan) {
  if (!plan) return TT_OK;
  if (ctx) {
    tt_plan_release_packed(ctx, plan);
    tt::pool_free(ctx, plan->d_tasks);
    tt::pool_free(ctx, plan->d_outs);
    tt::pool_free(ctx, plan->d_pairs);
    tt::pool_free(ctx, plan->d_tab);
    tt::pool_free(ctx, plan->d_status);
    tt::pool_free(ctx, plan->d_jobsA);
    tt::pool_free(ctx, plan->d_jobsB);
    tt::pool_free(ctx, plan->d_tilesA);
    tt::pool_free(ctx, plan->d_tilesB);
    tt::pool_free(ctx, plan->d_pairtc);
    tt::pool_free(ctx, plan->d_rs_tasks);
    tt::pool_free(ctx, plan->d_rs_chunks);
    tt::pool_free(ctx, plan->d_rs_a);
    tt::pool_free(ctx, plan->d_rs_e);
    tt::pool_free(ctx, plan->d_rs_o);
  }
  delete plan;
  return TT_OK;
}

int tt_plan_device_status(tt_ctx* ctx, const tt_plan* plan, int* status) {
  TT_REQUIRE(ctx && plan && status, "tt_plan_device_status: null argument");
  int h = 0;
  TT_CUDA(cudaMemcpyAsync(&h, plan->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  TT_CUDA(cudaStreamSynchronize(ctx->stream));
  *status = h;
  return TT_OK;
}

int tt_contract_predict(const tt_out_block* outs, int n_out, const tt_block_pair* pairs, int n_pairs,
                        int precision, int num_sms, double* us_fp64, double* us_tc, int* choice) {
  TT_REQUIRE(outs && (n_pairs == 0 || pairs) && us_fp64 && us_tc && choice, "tt_contract_predict: null argument");
  TT_REQUIRE(n_out >= 0 && n_pairs >= 0 && num_sms >= 1, "tt_contract_predict: bad counts");
  TT_REQUIRE(precision == TT_PREC_TF32_AUTO || precision == TT_PREC_TF32X3_AUTO,
             "tt_contract_predict: precision must be TT_PREC_TF32_AUTO or TT_PREC_TF32X3_AUTO");
  const int kind = precision == TT_PREC_TF32_AUTO ? TT_PREC_TF32 : TT_PREC_TF32X3;
  // the pairs grouped by output block, as tt_contract_plan groups them
  std::vector<int> order(n_pairs);
  std::iota(order.begin(), order.end(), 0);
  for (int i = 0; i < n_pairs; ++i)
    TT_REQUIRE(pairs[i].out_block >= 0 && pairs[i].out_block < n_out,
               "tt_contract_predict: pair references a missing output block");
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return pairs[a].out_block < pairs[b].out_block; });
  std::vector<PairDev> hp(n_pairs);
  std::vector<int> first(n_out + 1, 0);
  for (int ii = 0; ii < n_pairs; ++ii) {
    const tt_block_pair& q = pairs[order[ii]];
    TT_REQUIRE(q.n_m >= 0 && q.n_m <= TT_MAX_MODES && q.n_k >= 0 && q.n_k <= TT_MAX_MODES && q.n_n >= 0 &&
                   q.n_n <= TT_MAX_MODES,
               "tt_contract_predict: mode count out of range");
    int64_t m = 1, n = 1, k = 1;
    for (int i = 0; i < q.n_m; ++i) m *= q.m_dims[i];
    for (int i = 0; i < q.n_k; ++i) k *= q.k_dims[i];
    for (int i = 0; i < q.n_n; ++i) n *= q.n_dims[i];
    PairDev P;
    memset(&P, 0, sizeof(P));
    P.a_off = q.a_off;
    P.b_off = q.b_off;
    P.m = (int)m;
    P.n = (int)n;
    P.k = (int)k;
    hp[ii] = P;
    first[q.out_block + 1]++;
  }
  for (int o = 0; o < n_out; ++o) first[o + 1] += first[o];
  *us_fp64 = predict_us(outs, n_out, hp, first, TT_PREC_FP64, num_sms);
  *us_tc = predict_us(outs, n_out, hp, first, kind, num_sms);
  *choice = *us_tc > 0.8 * *us_fp64 ? TT_PREC_FP64 : kind;  // the rule tt_contract_plan applies
  return TT_OK;
}

int tt_plan_precision(const tt_plan* plan, int* precision) {
  TT_REQUIRE(plan && precision, "tt_plan_precision: null argument");
  *precision = plan->precision;
  return TT_OK;
}

int tt_contract_plan_timers(double* seconds, int n) {
  TT_REQUIRE(seconds && n >= 0, "tt_contract_plan_timers: null argument");
  for (int i = 0; i < n && i < 5; ++i) seconds[i] = g_plan_stage_s[i];
  return TT_OK;
}

int tt_plan_device_bytes(const tt_plan* plan, int64_t* bytes) {
  TT_REQUIRE(plan && bytes, "tt_plan_device_bytes: null argument");
  *bytes = plan->dev_bytes;
  return TT_OK;
}

int tt_plan_flops(const tt_plan* plan, double* flops) {
  TT_REQUIRE(plan && flops, "tt_plan_flops: null argument");
  *flops = plan->flops;
  return TT_OK;
}

}  // extern "C"
