// Context, stream-ordered device memory and error reporting of the C ABI.
#include <cstring>
#include <string>

#include <chrono>

#include "tt_internal.h"

namespace tt {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* what, const char* file, int line) {
  char buf[512];
  snprintf(buf, sizeof(buf), "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
  g_last_error = buf;
  return e == cudaErrorMemoryAllocation ? TT_ERR_OOM : TT_ERR_CUDA;
}

double* partials(tt_ctx* ctx, int n) {
  if (n > ctx->partials_cap) {
    if (ctx->d_partials) cudaFree(ctx->d_partials);
    ctx->d_partials = nullptr;
    int cap = n < 4096 ? 4096 : n;
    if (cudaMalloc(&ctx->d_partials, sizeof(double) * cap) != cudaSuccess) {
      ctx->partials_cap = 0;
      return nullptr;
    }
    ctx->partials_cap = cap;
  }
  return ctx->d_partials;
}

int device_status(tt_ctx* ctx) {
  if (ctx->h_dev_status && *(volatile int*)ctx->h_dev_status != TT_OK)
    return fail(TT_ERR_TIMEOUT,
                "a bounded wait of a tensor-core contraction gave up: its output is incomplete "
                "(tt_ctx_clear_device_status resets the context's status)");
  return TT_OK;
}

static cudaError_t pool_malloc_impl(tt_ctx* ctx, void** p, size_t bytes) {
  cudaError_t e = cudaMallocAsync(p, bytes, ctx->stream);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    ctx->pool_trims++;
    // the cached large blocks go back first, then the pool returns what it
    // holds unused to the device
    if (release_block_cache(ctx) == cudaSuccess && cudaStreamSynchronize(ctx->stream) == cudaSuccess &&
        cudaMemPoolTrimTo(ctx->pool, 0) == cudaSuccess)
      e = cudaMallocAsync(p, bytes, ctx->stream);
    if (e != cudaSuccess) cudaGetLastError();
  }
  return e;
}

// Size class of a large block: 2^k + j * 2^(k-2) for the smallest such value
// >= bytes (j = 1..4), so a class is at most 25% above the request.  With
// bytes >= 32 MB every class is a multiple of 8 MB.
static size_t large_class(size_t bytes) {
  int k = 63 - __builtin_clzll((unsigned long long)bytes);
  const size_t base = (size_t)1 << k, step = base >> 2;
  if (bytes == base) return base;
  return base + (bytes - base + step - 1) / step * step;
}

cudaError_t pool_malloc(tt_ctx* ctx, void** p, size_t bytes) {
  auto t0 = std::chrono::steady_clock::now();
  cudaError_t e = cudaSuccess;
  if (bytes >= kLargeBlockBytes && ctx->block_cache_cap > 0) {
    const size_t cls = large_class(bytes);
    // the smallest cached block of this class or up to 1.5x it
    size_t best = SIZE_MAX, at = 0;
    for (size_t i = 0; i < ctx->large_free.size(); ++i) {
      const size_t b = ctx->large_free[i].bytes;
      if (b >= cls && b <= cls + cls / 2 && b < best) { best = b; at = i; }
    }
    if (best != SIZE_MAX) {
      *p = ctx->large_free[at].p;  // freed earlier on this stream: stream order makes it free now
      ctx->large_free[at] = ctx->large_free.back();
      ctx->large_free.pop_back();
      ctx->large_cached -= best;
      ctx->large_hits++;
    } else {
      e = pool_malloc_impl(ctx, p, cls);
      if (e == cudaSuccess) ctx->large_class_of[*p] = cls;
    }
  } else {
    e = pool_malloc_impl(ctx, p, bytes);
  }
  const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  ctx->alloc_seconds += dt;
  if (dt > ctx->alloc_max_seconds) ctx->alloc_max_seconds = dt;
  ctx->allocs++;
  return e;
}

cudaError_t pool_free(tt_ctx* ctx, void* p) {
  if (!p) return cudaSuccess;
  auto t0 = std::chrono::steady_clock::now();
  cudaError_t e = cudaSuccess;
  auto it = ctx->large_class_of.find(p);
  bool cached = false;
  if (it != ctx->large_class_of.end()) {
    const size_t cls = it->second;
    if (cls <= ctx->block_cache_cap) {
      // room for it: the blocks freed longest ago go back to the pool
      while (ctx->large_cached + cls > ctx->block_cache_cap && !ctx->large_free.empty()) {
        size_t old = 0;
        for (size_t i = 1; i < ctx->large_free.size(); ++i)
          if (ctx->large_free[i].stamp < ctx->large_free[old].stamp) old = i;
        const tt_ctx::CachedBlock victim = ctx->large_free[old];
        ctx->large_free[old] = ctx->large_free.back();
        ctx->large_free.pop_back();
        ctx->large_cached -= victim.bytes;
        ctx->large_class_of.erase(victim.p);
        cudaError_t ev = cudaFreeAsync(victim.p, ctx->stream);
        if (ev != cudaSuccess && e == cudaSuccess) e = ev;
      }
      ctx->large_free.push_back({p, cls, ++ctx->large_clock});
      ctx->large_cached += cls;
      cached = true;
    } else {
      ctx->large_class_of.erase(it);
    }
  }
  if (!cached) {
    cudaError_t ef = cudaFreeAsync(p, ctx->stream);
    if (e == cudaSuccess) e = ef;
  }
  const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  ctx->free_seconds += dt;
  if (dt > ctx->free_max_seconds) ctx->free_max_seconds = dt;
  return e;
}

cudaError_t release_block_cache(tt_ctx* ctx) {
  cudaError_t first = cudaSuccess;
  for (const auto& b : ctx->large_free) {
    ctx->large_class_of.erase(b.p);
    cudaError_t e = cudaFreeAsync(b.p, ctx->stream);
    if (e != cudaSuccess && first == cudaSuccess) first = e;
  }
  ctx->large_free.clear();
  ctx->large_cached = 0;
  return first;
}

cudaError_t h2d_async(tt_ctx* ctx, void* dst, const void* src, size_t bytes) {
  if (bytes == 0) return cudaSuccess;
  const size_t need = (bytes + 255) & ~(size_t)255;
  if (!ctx->stage || need > ctx->stage_cap)
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream);
  if (ctx->stage_head + need > ctx->stage_cap) {
    auto t0 = std::chrono::steady_clock::now();
    cudaError_t e = cudaStreamSynchronize(ctx->stream);  // every staged copy has landed
    ctx->wait_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    ctx->waits++;
    if (e != cudaSuccess) return e;
    ctx->stage_head = 0;
  }
  char* p = ctx->stage + ctx->stage_head;
  std::memcpy(p, src, bytes);
  ctx->stage_head += need;
  return cudaMemcpyAsync(dst, p, bytes, cudaMemcpyHostToDevice, ctx->stream);
}

}  // namespace tt

namespace {
constexpr size_t kBounceBytes = (size_t)1 << 20;  // pinned bounce buffer for small reads

cudaError_t timed_sync(tt_ctx* ctx) {
  auto t0 = std::chrono::steady_clock::now();
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  ctx->wait_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  ctx->waits++;
  return e;
}
}  // namespace

extern "C" {

const char* tt_get_last_error(void) { return tt::g_last_error.c_str(); }

int tt_ctx_create(int device, tt_ctx** out) {
  TT_REQUIRE(out != nullptr, "tt_ctx_create: null output");
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
    return tt::fail(TT_ERR_NO_DEVICE, "tt_ctx_create: no CUDA device");
  TT_REQUIRE(device >= 0 && device < n, "tt_ctx_create: device ordinal out of range");
  TT_CUDA(cudaSetDevice(device));
  cudaDeviceProp prop;
  TT_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10)
    return tt::fail(TT_ERR_NO_DEVICE, "tt_ctx_create: kernels are built for sm_100a only");
  tt_ctx* ctx = new tt_ctx();
  ctx->device = device;
  ctx->num_sms = prop.multiProcessorCount;
  TT_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
  TT_CUDA(cudaDeviceGetDefaultMemPool(&ctx->pool, device));
  uint64_t thresh = UINT64_MAX;  // keep freed blocks cached in the pool
  TT_CUDA(cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &thresh));
  TT_CUDA(cudaMallocHost(&ctx->h_scalars, kBounceBytes));
  TT_CUDA(cudaHostAlloc((void**)&ctx->h_dev_status, sizeof(int), cudaHostAllocMapped));
  *ctx->h_dev_status = TT_OK;
  TT_CUDA(cudaHostGetDevicePointer((void**)&ctx->d_dev_status, ctx->h_dev_status, 0));
  ctx->stage_cap = (size_t)64 << 20;
  TT_CUDA(cudaMallocHost(&ctx->stage, ctx->stage_cap));
  if (!tt::partials(ctx, 16 * 4 * ctx->num_sms + 64) ||
      cudaMalloc(&ctx->d_ticket, sizeof(unsigned int)) != cudaSuccess ||
      cudaMemset(ctx->d_ticket, 0, sizeof(unsigned int)) != cudaSuccess) {
    if (ctx->d_partials) cudaFree(ctx->d_partials);
    if (ctx->d_ticket) cudaFree(ctx->d_ticket);
    delete ctx;
    return tt::fail(TT_ERR_OOM, "tt_ctx_create: scratch allocation failed");
  }
  *out = ctx;
  return TT_OK;
}

int tt_ctx_destroy(tt_ctx* ctx) {
  if (!ctx) return TT_OK;
  cudaSetDevice(ctx->device);
  tt::release_block_cache(ctx);
  cudaStreamSynchronize(ctx->stream);
  if (ctx->d_partials) cudaFree(ctx->d_partials);
  if (ctx->d_ticket) cudaFree(ctx->d_ticket);
  if (ctx->h_scalars) cudaFreeHost(ctx->h_scalars);
  if (ctx->h_dev_status) cudaFreeHost(ctx->h_dev_status);
  if (ctx->stage) cudaFreeHost(ctx->stage);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
  return TT_OK;
}


int tt_ctx_synchronize(tt_ctx* ctx) {
  TT_REQUIRE(ctx, "null context");
  TT_CUDA(timed_sync(ctx));
  return tt::device_status(ctx);
}

int tt_ctx_device_status(tt_ctx* ctx, int* status) {
  TT_REQUIRE(ctx && status, "null argument");
  TT_CUDA(timed_sync(ctx));
  *status = *(volatile int*)ctx->h_dev_status;
  return TT_OK;
}

int tt_ctx_clear_device_status(tt_ctx* ctx) {
  TT_REQUIRE(ctx, "null context");
  TT_CUDA(timed_sync(ctx));
  *(volatile int*)ctx->h_dev_status = TT_OK;
  return TT_OK;
}

int tt_ctx_memory(tt_ctx* ctx, int64_t* used, int64_t* used_high, int64_t* reserved, int reset_high) {
  TT_REQUIRE(ctx, "null context");
  uint64_t u = 0, h = 0, r = 0;
  TT_CUDA(cudaMemPoolGetAttribute(ctx->pool, cudaMemPoolAttrUsedMemCurrent, &u));
  TT_CUDA(cudaMemPoolGetAttribute(ctx->pool, cudaMemPoolAttrUsedMemHigh, &h));
  TT_CUDA(cudaMemPoolGetAttribute(ctx->pool, cudaMemPoolAttrReservedMemCurrent, &r));
  if (used) *used = (int64_t)u;
  if (used_high) *used_high = (int64_t)h;
  if (reserved) *reserved = (int64_t)r;
  if (reset_high) {
    uint64_t zero = 0;
    TT_CUDA(cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrUsedMemHigh, &zero));
  }
  return TT_OK;
}

int tt_ctx_set_wait_limit(tt_ctx* ctx, int64_t polls) {
  TT_REQUIRE(ctx, "null context");
  TT_REQUIRE(polls < ((int64_t)1 << 32), "tt_ctx_set_wait_limit: polls out of range");
  ctx->wait_limit = polls < 0 ? (1u << 26) : (uint32_t)polls;
  return TT_OK;
}

int tt_ctx_wait_stats(tt_ctx* ctx, double* seconds, int64_t* count) {
  TT_REQUIRE(ctx, "null context");
  if (seconds) *seconds = ctx->wait_seconds;
  if (count) *count = ctx->waits;
  return TT_OK;
}

int tt_ctx_pool_trims(tt_ctx* ctx, int64_t* count) {
  TT_REQUIRE(ctx && count, "tt_ctx_pool_trims: null argument");
  *count = ctx->pool_trims;
  return TT_OK;
}

int tt_ctx_stream(tt_ctx* ctx, void** stream) {
  TT_REQUIRE(ctx && stream, "null argument");
  *stream = (void*)ctx->stream;
  return TT_OK;
}

int tt_ctx_launch_count(tt_ctx* ctx, int64_t* count) {
  TT_REQUIRE(ctx && count, "null argument");
  *count = ctx->launches;
  return TT_OK;
}

int tt_event_create(tt_ctx* ctx, void** ev) {
  TT_REQUIRE(ctx && ev, "null argument");
  cudaEvent_t e;
  TT_CUDA(cudaEventCreate(&e));
  *ev = (void*)e;
  return TT_OK;
}

int tt_event_record(tt_ctx* ctx, void* ev) {
  TT_REQUIRE(ctx && ev, "null argument");
  TT_CUDA(cudaEventRecord((cudaEvent_t)ev, ctx->stream));
  return TT_OK;
}

int tt_event_elapsed_ms(void* a, void* b, float* ms) {
  TT_REQUIRE(a && b && ms, "null argument");
  TT_CUDA(cudaEventSynchronize((cudaEvent_t)b));
  TT_CUDA(cudaEventElapsedTime(ms, (cudaEvent_t)a, (cudaEvent_t)b));
  return TT_OK;
}

int tt_event_destroy(void* ev) {
  if (ev) cudaEventDestroy((cudaEvent_t)ev);
  return TT_OK;
}

int tt_device_alloc(tt_ctx* ctx, size_t bytes, void** dptr) {
  TT_REQUIRE(ctx && dptr, "null argument");
  *dptr = nullptr;
  if (bytes == 0) bytes = 16;
  TT_CUDA(tt::pool_malloc(ctx, dptr, bytes));
  return TT_OK;
}

int tt_device_free(tt_ctx* ctx, void* dptr) {
  TT_REQUIRE(ctx, "null context");
  TT_CUDA(tt::pool_free(ctx, dptr));
  return TT_OK;
}

int tt_ctx_alloc_stats(tt_ctx* ctx, double* alloc_s, double* alloc_max_s, double* free_s, double* free_max_s,
                       int64_t* allocs, int64_t* cache_hits, int64_t* cached_bytes, int reset_max) {
  TT_REQUIRE(ctx, "tt_ctx_alloc_stats: null context");
  if (alloc_s) *alloc_s = ctx->alloc_seconds;
  if (alloc_max_s) *alloc_max_s = ctx->alloc_max_seconds;
  if (free_s) *free_s = ctx->free_seconds;
  if (free_max_s) *free_max_s = ctx->free_max_seconds;
  if (allocs) *allocs = ctx->allocs;
  if (cache_hits) *cache_hits = ctx->large_hits;
  if (cached_bytes) *cached_bytes = (int64_t)ctx->large_cached;
  if (reset_max) ctx->alloc_max_seconds = ctx->free_max_seconds = 0.0;
  return TT_OK;
}

int tt_ctx_set_block_cache(tt_ctx* ctx, int64_t bytes) {
  TT_REQUIRE(ctx, "tt_ctx_set_block_cache: null context");
  TT_REQUIRE(bytes >= 0, "tt_ctx_set_block_cache: negative size");
  ctx->block_cache_cap = (size_t)bytes;
  if (ctx->large_cached > ctx->block_cache_cap) TT_CUDA(tt::release_block_cache(ctx));
  return TT_OK;
}

int tt_memcpy_h2d(tt_ctx* ctx, void* dst, const void* src, size_t bytes) {
  TT_REQUIRE(ctx, "null context");
  if (bytes == 0) return TT_OK;
  if (bytes < ((size_t)1 << 20)) {
    TT_CUDA(tt::h2d_async(ctx, dst, src, bytes));  // staged: the source may be reused at once
  } else {
    // bulk data straight from the caller's buffer (pin it for full bandwidth;
    // a pinned source must stay untouched until the stream is synchronised)
    TT_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
  }
  return TT_OK;
}

int tt_memcpy_d2h(tt_ctx* ctx, void* dst, const void* src, size_t bytes) {
  TT_REQUIRE(ctx, "null context");
  if (bytes == 0) return TT_OK;
  if (bytes <= kBounceBytes) {
    // small reads (Davidson scalars, SVD spectra) bounce through pinned memory:
    // a copy into pageable memory is staged by the driver at a much higher cost
    TT_CUDA(cudaMemcpyAsync(ctx->h_scalars, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    TT_CUDA(timed_sync(ctx));
    std::memcpy(dst, ctx->h_scalars, bytes);
    return tt::device_status(ctx);
  }
  auto t0 = std::chrono::steady_clock::now();
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream);  // blocks if pageable
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  ctx->wait_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  ctx->waits++;
  TT_CUDA(e);
  return tt::device_status(ctx);
}

int tt_memcpy_d2d(tt_ctx* ctx, void* dst, const void* src, size_t bytes) {
  TT_REQUIRE(ctx, "null context");
  if (bytes == 0) return TT_OK;
  TT_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
  return TT_OK;
}

int tt_memset_zero(tt_ctx* ctx, void* dst, size_t bytes) {
  TT_REQUIRE(ctx, "null context");
  if (bytes == 0) return TT_OK;
  TT_CUDA(cudaMemsetAsync(dst, 0, bytes, ctx->stream));
  return TT_OK;
}

}  // extern "C"
