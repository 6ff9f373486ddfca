// Internal runtime shared by the sm_100a kernels and the C ABI entry points.
#pragma once

#include <chrono>
#include <cuda_runtime.h>

#include <cstdint>
#include <unordered_map>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/tt_b200.h"

struct tt_ctx {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  cudaMemPool_t pool = nullptr;
  int64_t launches = 0;
  // small pinned staging buffer for scalar reads
  double* h_scalars = nullptr;
  // device scratch for the reductions: per-block partial sums, and the
  // ticket counter with which the last block of a reduction finds itself
  // (zero between reductions; the last block resets it)
  double* d_partials = nullptr;
  int partials_cap = 0;
  unsigned int* d_ticket = nullptr;
  // pinned staging ring for host->device copies that must not stall the stream
  char* stage = nullptr;
  size_t stage_cap = 0;
  size_t stage_head = 0;
  // host wall time spent blocked in stream synchronisations, and their count
  double wait_seconds = 0.0;
  int64_t pool_trims = 0;  // allocations that failed once, trimmed the pool and retried
  int64_t waits = 0;
  // host wall time inside the pool's allocate and free calls (total, largest
  // single call since the last tt_ctx_alloc_stats reset) and their counts
  double alloc_seconds = 0.0, alloc_max_seconds = 0.0;
  double free_seconds = 0.0, free_max_seconds = 0.0;
  int64_t allocs = 0;
  // Blocks of at least kLargeBlockBytes are allocated in size classes (a
  // quarter of a power of two apart) and kept by the context when freed, up
  // to block_cache_cap bytes (the oldest evicted first), for the next
  // allocation on this stream that fits in one (at most 1.5x its class).  The device pool can stall the host for seconds when a
  // multi-gigabyte request has to be assembled from freed memory; a steady
  // sweep asks for the same classes step after step and is served from here.
  struct CachedBlock {
    void* p;
    size_t bytes;    // its class
    uint64_t stamp;  // when it was freed (the oldest is evicted first)
  };
  std::unordered_map<void*, size_t> large_class_of;   // every live or cached large block
  std::vector<CachedBlock> large_free;                // cached blocks (tens at most)
  uint64_t large_clock = 0;
  size_t large_cached = 0;
  size_t block_cache_cap = (size_t)32 << 30;
  int64_t large_hits = 0;
  // sticky status of the bounded device waits (mapped pinned memory, so a
  // kernel that gives up writes TT_ERR_TIMEOUT straight into host memory);
  // every synchronisation of the context checks it
  int* h_dev_status = nullptr;
  int* d_dev_status = nullptr;
  // polls of the main-loop waits of the tensor-core kernels before they give
  // up (tt_ctx_set_wait_limit lowers it to test the timeout path)
  uint32_t wait_limit = 1u << 26;
};

namespace tt {

void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what, const char* file, int line);

// Launch bookkeeping: every kernel launch goes through this so the context
// can report how many of its kernels ran.
inline void count_launch(tt_ctx* ctx) { ctx->launches++; }

// Stream-ordered allocation from the context's pool.  Freed blocks stay
// reserved in the pool (release threshold unlimited), which can leave the
// device without a free range large enough for a big request although the
// pool holds enough in total: on failure the stream is drained, the pool's
// unused reserve is returned to the device and the request is retried once.
cudaError_t pool_malloc(tt_ctx* ctx, void** p, size_t bytes);

template <class T>
inline T* pool_alloc(tt_ctx* ctx, size_t n) {
  void* p = nullptr;
  if (n == 0) n = 1;
  if (pool_malloc(ctx, &p, n * sizeof(T)) != cudaSuccess) return nullptr;
  return static_cast<T*>(p);
}
cudaError_t pool_free(tt_ctx* ctx, void* p);
// Returns every cached large block to the device pool.
cudaError_t release_block_cache(tt_ctx* ctx);
constexpr size_t kLargeBlockBytes = (size_t)32 << 20;

// Per-thread, per-device "done once" flags for cudaFuncSetAttribute, which
// acts on the current device only: bit d of a thread_local mask.  Returns
// true the first time it is called for (mask, device).
inline bool first_on_device(uint64_t& mask, int device) {
  const uint64_t bit = (uint64_t)1 << (device & 63);
  if (mask & bit) return false;
  mask |= bit;
  return true;
}

// TT_ERR_TIMEOUT once a bounded device wait of this context has given up
// (read after a synchronisation), else TT_OK.
int device_status(tt_ctx* ctx);

// Reduction scratch of at least n doubles (grown on demand).
double* partials(tt_ctx* ctx, int n);

// Asynchronous host->device copy on the context's stream.  The source is
// first copied into the pinned staging ring, so the caller may release it on
// return and the stream is not serialised (pageable sources would be).  When
// the ring wraps, the stream is synchronised once so no staged bytes still in
// flight are overwritten.  Copies larger than the ring fall back to a plain
// (pageable) cudaMemcpyAsync.
cudaError_t h2d_async(tt_ctx* ctx, void* dst, const void* src, size_t bytes);

}  // namespace tt

#define TT_CUDA(expr)                                                   \
  do {                                                                  \
    cudaError_t _e = (expr);                                            \
    if (_e != cudaSuccess) return tt::cuda_fail(_e, #expr, __FILE__, __LINE__); \
  } while (0)

#define TT_LAUNCH_CHECK(ctx)                                             \
  do {                                                                   \
    tt::count_launch(ctx);                                               \
    cudaError_t _e = cudaGetLastError();                                 \
    if (_e != cudaSuccess) return tt::cuda_fail(_e, "kernel launch", __FILE__, __LINE__); \
  } while (0)

#define TT_REQUIRE(cond, msg)                                            \
  do {                                                                   \
    if (!(cond)) return tt::fail(TT_ERR_INVALID, msg);                   \
  } while (0)
