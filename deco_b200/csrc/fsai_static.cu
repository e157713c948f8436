// fsai_static.cu — an FSAI apply that performs no device allocation at all.
//
// deco_fsai_apply keeps its intermediate vector (FL x) inside the FSAI handle.
// Some callers cannot allocate device memory while they run: an application
// that hands all device memory to its own pool at start-up and forbids raw
// cudaMalloc afterwards, or a time-stepping loop that must not allocate once it
// has started (allocation can stall or fail under memory pressure).  This entry
// point keeps the intermediate in one file-scope device array of fixed size
// instead, so the call itself allocates nothing, and many FSAI handles applied
// one after another share that one intermediate.
//
// Limits and behaviour:
//   * at most kStaticRows (2^20) rows; larger factors are rejected with an error;
//   * the array lives as long as the library is loaded, on every device that
//     loads it (8 MiB each);
//   * the first call on a device resolves the array's device address with
//     cudaGetSymbolAddress (with that device current) and caches it; make that
//     first call before any stream capture;
//   * all calls share the array and it keeps the last call's contents; nothing
//     needs clearing, since the first product writes every entry before the
//     second reads it;
//   * calls that overlap on the GPU (two streams at once) race on the array.
#include <map>
#include <mutex>

#include "fsai.cuh"

namespace deco {
namespace {

constexpr int kStaticRows = 1 << 20;
// one intermediate of up to kStaticRows float64 values (or float32 values for a
// float32 factor); device code could name it directly, host code may not
__device__ __align__(256) double g_fsai_scratch[kStaticRows + kPad];

std::mutex g_addr_mu;
std::map<int, void*> g_addr;  // device ordinal -> device address of g_fsai_scratch

// Device address of the scratch array on `device`, resolved once per device.
void* scratch_address(int device) {
  std::lock_guard<std::mutex> lk(g_addr_mu);
  auto it = g_addr.find(device);
  if (it != g_addr.end()) return it->second;
  int prev = -1;
  DECO_CUDA(cudaGetDevice(&prev));
  if (prev != device) DECO_CUDA(cudaSetDevice(device));
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_fsai_scratch);
  if (prev != device) cudaSetDevice(prev);
  if (e != cudaSuccess)
    throw Error(DECO_ERR_CUDA, std::string("cudaGetSymbolAddress of the static FSAI scratch failed: ") +
                                   cudaGetErrorString(e));
  g_addr[device] = p;
  return p;
}

// the matrix's chosen sub-warp width, or the heuristic one: never the timing
// autotuner, which allocates
int width_no_alloc(const deco_csr_s* A, bool f32) {
  const int sw = f32 ? A->sw32 : A->sw64;
  return sw ? sw : heuristic_subwarp(A->avg_row, f32 ? 4 : 2);
}

}  // namespace
}  // namespace deco

using namespace deco;

extern "C" int deco_fsai_apply_static(deco_ctx ctx, deco_fsai F, const double* x, double* y) {
  return guard([&] {
    DECO_REQUIRE(ctx && F && x && y, DECO_ERR_ARG, "NULL argument");
    DECO_REQUIRE(F->n <= kStaticRows, DECO_ERR_ARG,
                 "deco_fsai_apply_static: the factor has more rows than the static scratch holds (" +
                     std::to_string(F->n) + " > " + std::to_string(kStaticRows) + "); use deco_fsai_apply");
    void* tmp = scratch_address(ctx->device);
    const int n = F->n;
    if (F->precision == 32) {
      float* t = static_cast<float*>(tmp);
      launch_spmv_sw<float, double>(ctx->stream, width_no_alloc(&F->FL, true), n, 1, F->FL.r.get(), F->FL.c.get(),
                                    F->FL.v32.get(), x, EpiStore<float>{t});
      launch_spmv_sw<float, float>(ctx->stream, width_no_alloc(&F->FUt, true), n, 1, F->FUt.r.get(), F->FUt.c.get(),
                                   F->FUt.v32.get(), t, EpiStore<double>{y});
    } else {
      double* t = static_cast<double*>(tmp);
      launch_spmv_sw<double, double>(ctx->stream, width_no_alloc(&F->FL, false), n, 1, F->FL.r.get(), F->FL.c.get(),
                                     F->FL.v.get(), x, EpiStore<double>{t});
      launch_spmv_sw<double, double>(ctx->stream, width_no_alloc(&F->FUt, false), n, 1, F->FUt.r.get(),
                                     F->FUt.c.get(), F->FUt.v.get(), t, EpiStore<double>{y});
    }
  });
}
