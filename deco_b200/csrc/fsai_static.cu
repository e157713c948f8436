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
//     cudaGetSymbolAddress (with that device current) and caches it for the
//     life of the process; make that first call before any stream capture.
//     The cached address does not survive cudaDeviceReset (or any other
//     destruction of the device's primary context): a process that resets a
//     device must not call this entry point on it again;
//   * all calls share the array and it keeps the last call's contents; nothing
//     needs clearing, since the first product writes every entry before the
//     second reads it;
//   * calls that overlap on the GPU (two streams at once) race on the array;
//   * the two products take the product deco_fsai_apply takes (the autotuner's
//     choice, or the layout rules): with the slot-padded copies the results are
//     identical to its results; the cell-block and CSR kernels run at their
//     heuristic widths here (no timing, no shared state), which may sum in
//     another order than deco_fsai_apply's tuned widths: equal to rounding.
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

// the heuristic sub-warp width: never the timing autotuner, which allocates, nor
// the width it caches on the matrix, which another thread's deco_fsai_apply may
// be writing at the same time
int width_no_alloc(const deco_csr_s* A, bool f32) { return heuristic_subwarp(A->avg_row, f32 ? 4 : 2); }

// One factor product with the kernel deco_fsai_apply would pick when that needs no
// allocation: the slot-padded copies (scalar rows, or 2x2 cell blocks with x
// aligned for pair loads), else the CSR kernel at the width chosen above.
template <typename VT, typename XT, class Epi>
void product_no_alloc(deco_ctx_s* ctx, deco_csr_s* A, const XT* x, Epi epi) {
  const bool f32 = sizeof(VT) == 4;
  const int plan = f32 ? A->plan32 : A->plan64;  // the product autotuner's choice (0: the layout rules)
  if (plan == 2 && A->bbs > 1 && (!f32 || A->bv32) &&
      reinterpret_cast<uintptr_t>(x) % (A->bbs == 2 ? 2 * sizeof(XT) : sizeof(XT)) == 0) {
    int sw = 1;  // the cell-block kernel's heuristic lanes per cell (no shared state)
    while (sw < 16 && sw < A->avg_blk / (A->bbs == 2 ? 4.0 : 2.0)) sw <<= 1;
    launch_bsr<VT, XT, Epi>(ctx->stream, A, sw, false, x, epi);
    return;
  }
  if (plan != 3 && A->ew && (!f32 || A->ev32)) {
    if (!A->bbs) {
      launch_ell1<VT, XT, Epi>(ctx->stream, A, x, epi);
      return;
    }
    if (A->bbs == 2 && reinterpret_cast<uintptr_t>(x) % (2 * sizeof(XT)) == 0) {
      launch_ell2<VT, XT, Epi>(ctx->stream, A, false, x, epi);
      return;
    }
    if (A->bbs == 3) {
      launch_ell3<VT, XT, Epi>(ctx->stream, A, false, x, epi);
      return;
    }
  }
  const VT* v;
  if constexpr (sizeof(VT) == 4) v = A->v32.get(); else v = A->v.get();
  launch_spmv_sw<VT, XT>(ctx->stream, width_no_alloc(A, f32), A->n, 1, A->r.get(), A->c.get(), v, x, epi);
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
    if (F->precision == 32) {
      float* t = static_cast<float*>(tmp);
      product_no_alloc<float, double>(ctx, &F->FL, x, EpiStore<float>{t});
      product_no_alloc<float, float>(ctx, &F->FUt, t, EpiStore<double>{y});
    } else {
      double* t = static_cast<double*>(tmp);
      product_no_alloc<double, double>(ctx, &F->FL, x, EpiStore<double>{t});
      product_no_alloc<double, double>(ctx, &F->FUt, t, EpiStore<double>{y});
    }
  });
}
