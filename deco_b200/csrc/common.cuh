// common.cuh — shared infrastructure of libdeco_b200: error handling across the
// C ABI, padded device buffers, the context (device + stream + scratch), and
// warp/block reduction helpers.  Every entry point of the C ABI returns an int
// status (0 = ok) and never exits; deco_last_error() describes the failure.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "deco_b200.h"

namespace deco {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string& msg);

#define DECO_CUDA(call)                                                                           \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess)                                                                        \
      throw ::deco::Error(DECO_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_) +     \
                                             " (" + __FILE__ + ":" + std::to_string(__LINE__) + ")"); \
  } while (0)

// every kernel launch site is followed by DECO_CHECK_LAUNCH(), which also counts
// the launch (deco_launch_count)
void count_launch();
#define DECO_CHECK_LAUNCH()                 \
  do {                                      \
    ::deco::count_launch();                 \
    DECO_CUDA(cudaGetLastError());          \
  } while (0)

#define DECO_REQUIRE(cond, code, msg)                          \
  do {                                                         \
    if (!(cond)) throw ::deco::Error((code), std::string(msg)); \
  } while (0)

// Wraps a C-ABI body: converts exceptions into status codes.
template <typename F>
int guard(F&& f) {
  try {
    f();
    return DECO_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    set_last_error("host allocation failed");
    return DECO_ERR_ALLOC;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return DECO_ERR_INTERNAL;
  }
}

// DECO_TRACE=1 diagnostics for host calls that take unusually long
double trace_clock_ms();
void trace_slow_call(const char* what, size_t bytes, double t0_ms);

// Elements of slack after every device array: vectorised loads (16 bytes) may
// touch up to 3 elements past the last valid one; the slack is zero-filled.
constexpr size_t kPad = 16;

// Device memory of the library.  Large blocks (>= 1 MiB) freed on a stream are
// kept in a per-stream cache and handed to later requests on the SAME stream
// (stream order makes the reuse safe), because the stream-ordered pool's
// cudaMallocAsync occasionally stalls for hundreds of milliseconds on large
// requests even when its reserved memory could serve them; a solve that
// rebuilds its setup every step then allocates nothing after the first step.
// Smaller blocks go straight to the pool.  DECO_CACHE=0 disables the cache;
// deco_ctx_trim returns a stream's cached blocks to the pool.
void* dev_alloc(size_t bytes, cudaStream_t s, size_t* capacity);
void dev_free(void* p, size_t capacity, cudaStream_t s);
void cache_attach_stream(cudaStream_t s);
void cache_detach_stream(cudaStream_t s);  // frees the stream's cached blocks
void cache_trim_stream(cudaStream_t s);

// Owning device buffer with zeroed padding; moves, does not copy.
template <typename T>
class DevBuf {
 public:
  DevBuf() = default;
  explicit DevBuf(size_t n, cudaStream_t s = 0) { alloc(n, s); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p_(o.p_), n_(o.n_), cap_(o.cap_), s_(o.s_) { o.p_ = nullptr; o.n_ = 0; o.cap_ = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      p_ = o.p_; n_ = o.n_; cap_ = o.cap_; s_ = o.s_;
      o.p_ = nullptr; o.n_ = 0; o.cap_ = 0;
    }
    return *this;
  }
  ~DevBuf() { release(); }

  // Stream-ordered allocation (dev_alloc): no device-wide synchronisation.
  void alloc(size_t n, cudaStream_t s = 0) {
    release();
    n_ = n;
    s_ = s;
    p_ = static_cast<T*>(dev_alloc((n + kPad) * sizeof(T), s, &cap_));
    DECO_CUDA(cudaMemsetAsync(p_ + n, 0, kPad * sizeof(T), s));
  }
  void zero(cudaStream_t s) {
    if (p_) DECO_CUDA(cudaMemsetAsync(p_, 0, (n_ + kPad) * sizeof(T), s));
  }
  void release() {
    if (p_) dev_free(p_, cap_, s_);
    p_ = nullptr;
    n_ = 0;
    cap_ = 0;
  }
  T* get() const { return p_; }
  size_t size() const { return n_; }
  explicit operator bool() const { return p_ != nullptr; }

 private:
  T* p_ = nullptr;
  size_t n_ = 0;
  size_t cap_ = 0;
  cudaStream_t s_ = 0;
};

}  // namespace deco

// ----------------------------------------------------------------- handles

struct deco_ctx_s {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int num_sms = 148;
  int autotune = 1;
  int bsr = 1;        // cell-block copies for CPR systems (DECO_BSR=0 disables)
  int padded = 1;     // slot-padded copies of short-row 2x2-block matrices (DECO_PADDED=0 disables)
  int slot_codes = 1; // offset-coded slot columns of the padded copies (DECO_SLOT_CODES=0 disables)
  int trace = 0;      // DECO_TRACE=1: host wall time of setup sub-steps on stderr
  double trace_t = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // small pinned host buffer for scalar read-backs
  double* host_scalars = nullptr;
  // reusable device scratch for reductions (partials + counters)
  deco::DevBuf<double> red;
  deco::DevBuf<unsigned int> counter;
};

namespace deco {

// ------------------------------------------------------------ device helpers

template <typename T>
__device__ __forceinline__ T warp_sum(T v, unsigned mask = 0xffffffffu) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
  return v;
}

template <int W, typename T>
__device__ __forceinline__ T subwarp_sum(T v) {
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__host__ __device__ __forceinline__ long long cdiv(long long a, long long b) { return (a + b - 1) / b; }

// exclusive scan of int counts[0..n) into out[0..n] (out[n] = total);
// returns the total.  64-bit accumulation; throws if the total exceeds int32.
long long exclusive_scan_int(deco_ctx_s* ctx, const int* counts, int* out, long long n);

// DECO_TRACE=1: synchronises the stream and prints the wall time since the last
// mark (setup diagnostics; no effect otherwise)
void trace_mark(deco_ctx_s* ctx, const char* label);

// grid size for a grid-stride kernel: a multiple of the SM count
inline int grid_for(const deco_ctx_s* ctx, long long work, int block, int per_sm = 8) {
  long long g = cdiv(work, block);
  long long cap = (long long)ctx->num_sms * per_sm;
  if (g > cap) g = cap;
  return int(g < 1 ? 1 : g);
}

// ------------------------------------------- programmatic dependent launch
// Inside a GMRES solve (and only there: the matrices are constant while it
// runs) the kernels of an iteration are launched with programmatic stream
// serialisation: a kernel's blocks may be scheduled while its predecessor's
// last wave still runs.  Every kernel launched that way follows one protocol:
//   * before pdl_wait() it reads only data written two or more kernels earlier
//     (the matrices, older basis columns) and writes nothing;
//   * pdl_wait() returns once the predecessor has completed and its writes are
//     visible; pdl_trigger() comes after it, so when a kernel is launched the
//     kernel two places before it has completed.
// The slot-padded products load their matrix slots before the wait, so the
// first blocks of a product stream the matrix during the tail of the kernel
// before it.  A kernel launched without the attribute runs in plain stream
// order and the two instructions are no-ops for it.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

// true while the calling thread runs a solve with programmatic launches
// (PdlScope; DECO_PDL=0 turns them off)
bool pdl_active();
struct PdlScope {
  bool prev;
  explicit PdlScope(bool on);
  ~PdlScope();
};

// Launches kernel k (a kernel that follows the protocol above) with the
// programmatic-serialisation attribute when pdl_active(), else as <<<...>>>.
template <typename... KP, typename... Args>
void launch_k(void (*k)(KP...), dim3 grid, dim3 block, size_t shm, cudaStream_t s, Args&&... args) {
  if (pdl_active()) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = shm;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    DECO_CUDA(cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...));
  } else {
    k<<<grid, block, shm, s>>>(std::forward<Args>(args)...);
  }
}

}  // namespace deco
