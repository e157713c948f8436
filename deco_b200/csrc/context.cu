// context.cu — error state, context lifecycle and the device exclusive scan
// used by every count/compact step (filters, pattern extraction, transposes).
#include <map>
#include <mutex>
#include <chrono>
#include <atomic>
#include <cstdlib>

#include "common.cuh"

namespace deco {

static thread_local std::string g_last_error;
void set_last_error(const std::string& msg) { g_last_error = msg; }

static std::atomic<long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

// programmatic dependent launch inside solves (common.cuh)
static thread_local bool t_pdl = false;
static bool pdl_allowed() {
  static const bool on = [] {
    const char* e = std::getenv("DECO_PDL");
    return !(e && std::atoi(e) == 0);
  }();
  return on;
}
bool pdl_active() { return t_pdl; }
PdlScope::PdlScope(bool on) : prev(t_pdl) { t_pdl = on && pdl_allowed(); }
PdlScope::~PdlScope() { t_pdl = prev; }

// ------------------------------------------------------------ block cache
namespace {
std::mutex g_cache_mu;
std::map<cudaStream_t, std::multimap<size_t, void*>> g_cache;  // stream -> (capacity -> block)
std::map<cudaStream_t, int> g_live;                            // streams of live contexts
constexpr size_t kCacheMin = size_t(1) << 20;

bool cache_on() {
  static const bool on = [] {
    const char* e = std::getenv("DECO_CACHE");
    return !(e && std::atoi(e) == 0);
  }();
  return on;
}
}  // namespace

std::atomic<long long> g_alloc_requests{0};

void* dev_alloc(size_t bytes, cudaStream_t s, size_t* capacity) {
  g_alloc_requests.fetch_add(1, std::memory_order_relaxed);
  if (cache_on() && bytes >= kCacheMin) {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    auto it = g_cache.find(s);
    if (it != g_cache.end()) {
      auto& mm = it->second;
      auto b = mm.lower_bound(bytes);
      if (b != mm.end() && b->first <= bytes + bytes / 4 + kCacheMin) {
        void* p = b->second;
        *capacity = b->first;
        mm.erase(b);
        return p;
      }
    }
  }
  void* p = nullptr;
  const double t0 = trace_clock_ms();
  cudaError_t e = cudaMallocAsync(&p, bytes, s);
  trace_slow_call("cudaMallocAsync", bytes, t0);
  if (e != cudaSuccess) {  // give this stream's cached blocks back to the pool and try once more
    cudaGetLastError();
    cache_trim_stream(s);
    e = cudaMallocAsync(&p, bytes, s);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw Error(DECO_ERR_ALLOC, "device allocation of " + std::to_string(bytes) +
                                    " bytes failed: " + cudaGetErrorString(e));
  }
  *capacity = bytes;
  return p;
}

void dev_free(void* p, size_t capacity, cudaStream_t s) {
  if (!p) return;
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    const bool live = g_live.count(s) != 0;
    if (cache_on() && live && capacity >= kCacheMin) {
      g_cache[s].emplace(capacity, p);
      return;
    }
    if (!live) {  // the owning context (and maybe its stream) is gone
      cudaFree(p);
      return;
    }
  }
  cudaFreeAsync(p, s);
}

void cache_attach_stream(cudaStream_t s) {
  std::lock_guard<std::mutex> lk(g_cache_mu);
  ++g_live[s];
}

void cache_trim_stream(cudaStream_t s) {
  std::lock_guard<std::mutex> lk(g_cache_mu);
  auto it = g_cache.find(s);
  if (it == g_cache.end()) return;
  for (auto& kv : it->second) cudaFreeAsync(kv.second, s);
  g_cache.erase(it);
}

void cache_detach_stream(cudaStream_t s) {
  cache_trim_stream(s);
  std::lock_guard<std::mutex> lk(g_cache_mu);
  auto it = g_live.find(s);
  if (it != g_live.end() && --it->second <= 0) g_live.erase(it);
}

static bool trace_env() {
  static const bool on = [] {
    const char* e = std::getenv("DECO_TRACE");
    return e && std::atoi(e) != 0;
  }();
  return on;
}

double trace_clock_ms() {
  if (!trace_env()) return 0.0;
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void trace_slow_call(const char* what, size_t bytes, double t0_ms) {
  if (!trace_env()) return;
  const double dt = trace_clock_ms() - t0_ms;
  if (dt > 5.0) std::fprintf(stderr, "[deco-trace] slow %s of %.1f MB: %.1f ms\n", what, bytes / 1e6, dt);
}

void trace_mark(deco_ctx_s* ctx, const char* label) {
  if (!ctx->trace) return;
  cudaStreamSynchronize(ctx->stream);
  const double t =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
  if (label) {
    size_t reserved = 0, used = 0;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, ctx->device) == cudaSuccess) {
      cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
      cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used);
    }
    std::fprintf(stderr, "[deco-trace] %-28s %9.3f ms  pool %.2f/%.2f GB\n", label, t - ctx->trace_t, used / 1e9,
                 reserved / 1e9);
  }
  ctx->trace_t = t;
}

namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kTile = kScanThreads * kScanItems;

__device__ __forceinline__ long long block_exclusive_scan(long long v, long long* smem, long long* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  long long x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    long long y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) smem[wid] = x;
  __syncthreads();
  if (wid == 0) {
    long long w = lane < (blockDim.x >> 5) ? smem[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      long long y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    smem[lane] = w;  // inclusive warp totals
  }
  __syncthreads();
  long long warp_off = wid > 0 ? smem[wid - 1] : 0;
  if (total) *total = smem[(blockDim.x >> 5) - 1];
  return warp_off + x - v;
}

__global__ void __launch_bounds__(kScanThreads) tile_sums(const int* __restrict__ in, long long n,
                                                          long long* __restrict__ sums) {
  __shared__ long long sm[32];
  long long base = (long long)blockIdx.x * kTile;
  long long s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    long long i = base + (long long)threadIdx.x * kScanItems + k;
    if (i < n) s += in[i];
  }
  long long tot;
  block_exclusive_scan(s, sm, &tot);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kScanThreads) scan_sums(long long* __restrict__ sums, long long nt,
                                                          long long* __restrict__ total) {
  __shared__ long long sm[32];
  long long carry = 0;
  for (long long b = 0; b < nt; b += kScanThreads) {
    long long i = b + threadIdx.x;
    long long v = i < nt ? sums[i] : 0;
    long long tot;
    long long ex = block_exclusive_scan(v, sm, &tot);
    if (i < nt) sums[i] = carry + ex;
    carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(kScanThreads) tile_scan(const int* __restrict__ in, long long n,
                                                          const long long* __restrict__ offs,
                                                          const long long* __restrict__ total,
                                                          int* __restrict__ out) {
  __shared__ long long sm[32];
  long long base = (long long)blockIdx.x * kTile + (long long)threadIdx.x * kScanItems;
  long long loc[kScanItems];
  long long s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    loc[k] = (base + k < n) ? in[base + k] : 0;
    s += loc[k];
  }
  long long ex = block_exclusive_scan(s, sm, nullptr) + offs[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) out[base + k] = (int)ex;
    ex += loc[k];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = (int)*total;
}

}  // namespace

long long exclusive_scan_int(deco_ctx_s* ctx, const int* counts, int* out, long long n) {
  long long nt = cdiv(n, kTile);
  if (nt < 1) nt = 1;
  DevBuf<long long> sums(nt + 1, ctx->stream);
  long long* total = sums.get() + nt;
  tile_sums<<<(int)nt, kScanThreads, 0, ctx->stream>>>(counts, n, sums.get());
  DECO_CHECK_LAUNCH();
  scan_sums<<<1, kScanThreads, 0, ctx->stream>>>(sums.get(), nt, total);
  DECO_CHECK_LAUNCH();
  tile_scan<<<(int)nt, kScanThreads, 0, ctx->stream>>>(counts, n, sums.get(), total, out);
  DECO_CHECK_LAUNCH();
  long long h_total = 0;
  DECO_CUDA(cudaMemcpyAsync(&h_total, total, sizeof(long long), cudaMemcpyDeviceToHost, ctx->stream));
  DECO_CUDA(cudaStreamSynchronize(ctx->stream));
  DECO_REQUIRE(h_total <= 2147483647LL, DECO_ERR_ARG, "row pointer total exceeds int32");
  return h_total;
}

}  // namespace deco

using namespace deco;

extern "C" {

const char* deco_last_error(void) { return g_last_error.c_str(); }
const char* deco_version(void) { return "deco_b200 0.1 (sm_100a)"; }
long long deco_launch_count(void) { return g_launches.load(); }
long long deco_alloc_count(void) { return g_alloc_requests.load(); }

int deco_ctx_create(int device, void* stream, deco_ctx* out) {
  return guard([&] {
    DECO_REQUIRE(out, DECO_ERR_ARG, "out is NULL");
    int ndev = 0;
    DECO_CUDA(cudaGetDeviceCount(&ndev));
    DECO_REQUIRE(device >= 0 && device < ndev, DECO_ERR_ARG, "device index out of range");
    DECO_CUDA(cudaSetDevice(device));
    auto* c = new deco_ctx_s();
    c->device = device;
    if (stream) {
      c->stream = static_cast<cudaStream_t>(stream);
    } else {
      DECO_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
      c->own_stream = true;
    }
    cudaDeviceProp prop;
    DECO_CUDA(cudaGetDeviceProperties(&prop, device));
    c->num_sms = prop.multiProcessorCount;
    // DECO_AUTOTUNE=0 keeps the heuristic SpMV widths (profiler runs distort timings)
    if (const char* e = std::getenv("DECO_AUTOTUNE")) c->autotune = std::atoi(e) != 0;
    if (const char* e = std::getenv("DECO_BSR")) c->bsr = std::atoi(e) != 0;
    if (const char* e = std::getenv("DECO_PADDED")) c->padded = std::atoi(e) != 0;
    if (const char* e = std::getenv("DECO_SLOT_CODES")) c->slot_codes = std::atoi(e) != 0;
    if (const char* e = std::getenv("DECO_TRACE")) c->trace = std::atoi(e) != 0;
    // keep freed device memory in the stream-ordered pool instead of returning it
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      unsigned long long threshold = ~0ULL;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
    }
    cache_attach_stream(c->stream);
    DECO_CUDA(cudaEventCreate(&c->ev0));
    DECO_CUDA(cudaEventCreate(&c->ev1));
    DECO_CUDA(cudaMallocHost(&c->host_scalars, 1024 * sizeof(double)));
    c->red.alloc(64 * 1024, c->stream);
    c->counter.alloc(64, c->stream);
    c->counter.zero(c->stream);
    *out = c;
  });
}

int deco_ctx_destroy(deco_ctx ctx) {
  return guard([&] {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    ctx->red.release();
    ctx->counter.release();
    if (ctx->host_scalars) cudaFreeHost(ctx->host_scalars);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    cache_detach_stream(ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
  });
}

int deco_ctx_sync(deco_ctx ctx) {
  return guard([&] {
    DECO_REQUIRE(ctx, DECO_ERR_ARG, "ctx is NULL");
    DECO_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int deco_ctx_stream(deco_ctx ctx, void** stream) {
  return guard([&] {
    DECO_REQUIRE(ctx && stream, DECO_ERR_ARG, "NULL argument");
    *stream = ctx->stream;
  });
}

int deco_ctx_trim(deco_ctx ctx) {
  return guard([&] {
    DECO_REQUIRE(ctx, DECO_ERR_ARG, "ctx is NULL");
    cache_trim_stream(ctx->stream);
  });
}

int deco_ctx_set_autotune(deco_ctx ctx, int autotune) {
  return guard([&] {
    DECO_REQUIRE(ctx, DECO_ERR_ARG, "ctx is NULL");
    ctx->autotune = autotune;
  });
}

}  // extern "C"
