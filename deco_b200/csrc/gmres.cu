// gmres.cu — restarted right / left preconditioned GMRES(m) on the device
// (solver/rgmres.tpp:8-139, solver/lgmres.tpp:1-134; Givens :141-160).
//
// Arnoldi step: classical Gram-Schmidt with reorthogonalisation (CGS2) in two
// passes over the basis, the second projection taken from the Gram matrix
// instead of a second dot pass:
//   pass A   one read of V computes  h = V^T w  and the new Gram row  V^T v_j.
//            The block that finishes last forms G (the Gram matrix of the
//            stored basis), the reorthogonalisation h2 = V^T (w - V h) =
//            h - G h, and the coefficients c = h + h2, which leave (I - G)^2 of
//            the orthogonality defect, as CGS2 does.
//   pass B   w'' = w - V c, written as the next basis column, and ||w''||^2.
//            The last block sets H(:,j) = c, H(j+1,j) = ||w''|| and applies the
//            Givens rotations (the reference's formulas) on the device.
// Normalisation is lazy: column k is stored unnormalised with a scale s_k that
// the next SpMV epilogue, the coefficients and the combination absorb, so no
// pass is spent on scaling.  Per iteration the basis is read twice (the
// reference's modified Gram-Schmidt, rgmres.tpp:72-75, reads it 2(j+1) times and
// w 3(j+1) times).  |g_{j+1}| returns to the host one iteration behind: the next
// iteration is already queued when the host checks convergence, so the device
// does not wait on the host.
//
// Precision 32: V, w, z in float32 with float64 accumulation; H, G, g and the
// rotations in float64; every restart recomputes the true residual b - A x and
// the solution update in float64 (iterative refinement).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <mutex>
#include <type_traits>
#include <vector>

#include "cpr.cuh"

namespace deco {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
// Largest restart length m.  The basis costs (m + 1) n words of HBM; the
// kernels' per-column scratch (coefficients, one Hessenberg column, rotations)
// lives in dynamic shared memory sized by the launch; the bound keeps the float32
// dot pass's stages (64 KB) plus one column of coefficients (8 (m+1) bytes) well
// inside a block's shared memory.
constexpr int kMaxRestart = 1000;
constexpr int kColsD = kWarps * 8;  // columns one block row of the dot pass takes (8 per warp)
// back substitution with the triangle of H in shared memory up to this order
// (j (j + 1) / 2 + j + 1 doubles, under the 227 KB opt-in limit); past it the
// same arithmetic reads H from global memory
constexpr int kBacksolveShm = 200;
// host read-back of |g_{j+1}|: a ring of kRing pinned slots (values from kSlot0,
// tags from kTag0) that the update pass writes; the host runs up to `lookahead`
// Arnoldi steps ahead (<= kRing - 2)
constexpr int kRing = 8;
constexpr int kSlot0 = 4;
constexpr int kTag0 = 24;  // the ring's tags (8-byte words of the context's pinned buffer)
// step tags, unique in the process, so a slot never matches an earlier solve's post
std::atomic<unsigned long long> g_step_tag{0};
constexpr double kEps = 2.220446049250312e-16;

// device state (float64): H (m+1)*m | G (m+1)^2 | g | cs | sn | s | c | sums 2(m+2) | sc
struct State {
  double* H; double* G; double* g; double* cs; double* sn; double* s; double* c; double* sums; double* sc;
  int m;
  __host__ __device__ double& h(int i, int j) const { return H[i + (size_t)j * (m + 1)]; }
  __host__ __device__ double& gm(int i, int j) const { return G[i + (size_t)j * (m + 1)]; }
  static size_t doubles(int m) {
    return (size_t)(m + 1) * m + (size_t)(m + 1) * (m + 1) + 5 * (size_t)(m + 1) + 2 * (size_t)(m + 2) + 16;
  }
  void bind(double* b, int m_) {
    m = m_;
    H = b;
    G = H + (size_t)(m + 1) * m;
    g = G + (size_t)(m + 1) * (m + 1);
    cs = g + (m + 1);
    sn = cs + (m + 1);
    s = sn + (m + 1);
    c = s + (m + 1);
    sums = c + (m + 1);
    sc = sums + 2 * (m + 2);
  }
};
enum { SC_RES = 0, SC_BREAK = 1, SC_BETA = 2 };

// |g_{j+1}| of Arnoldi step j posted straight into pinned host memory by the
// update pass (no copy or event in the stream between the step's last kernel
// and the next step's first, so those launch back to back): the value, a
// system-scope fence, then a tag unique to the step.  The host polls the tag.
struct HostSlot {
  double* val = nullptr;              // device view of the pinned ring of values
  unsigned long long* tag = nullptr;  // device view of the pinned ring of tags
  unsigned long long t = 0;           // this step's tag
  __device__ void post(double v) const {
    if (!val) return;
    *val = v;
    __threadfence_system();
    *reinterpret_cast<volatile unsigned long long*>(tag) = t;
  }
};


// deterministic last-block reduction of red[i*nb + b] over b for i < ncols.
// Warp w owns columns w, w + 8, ...; it works on four of them at once so four
// independent loads per lane are in flight (this runs in one block while the
// rest of the GPU waits); each column's summation order is the lane-strided one.
__device__ void finalize_partials(const double* red, int nb, int ncols, double* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i0 = warp; i0 < ncols; i0 += 4 * kWarps) {
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    const double* p[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) p[u] = red + (size_t)min(i0 + u * kWarps, ncols - 1) * nb;
#pragma unroll 4
    for (int b = lane; b < nb; b += 32)
#pragma unroll
      for (int u = 0; u < 4; ++u) s[u] += __ldcg(p[u] + b);
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const double t = warp_sum(s[u]);
      if (lane == 0 && i0 + u * kWarps < ncols) out[i0 + u * kWarps] = t;
    }
  }
}

// The same reduction for nb <= 32 MAXB partials per column, with every load of
// four columns issued before the sums (up to 4 MAXB loads in flight per lane
// instead of 16); each column sums in the same lane-strided order, so the result
// is identical.  For the last block of the dot pass, which holds up the next
// kernel while it runs.
template <int MAXB>
__device__ void finalize_partials_wide(const double* red, int nb, int ncols, double* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i0 = warp; i0 < ncols; i0 += 4 * kWarps) {
    double v[4][MAXB];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const double* p = red + (size_t)min(i0 + u * kWarps, ncols - 1) * nb;
#pragma unroll
      for (int t = 0; t < MAXB; ++t) {
        const int b = lane + 32 * t;
        v[u][t] = b < nb ? __ldcg(p + b) : 0.0;
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      double s = 0.0;
#pragma unroll
      for (int t = 0; t < MAXB; ++t)
        if (lane + 32 * t < nb) s += v[u][t];
      const double tot = warp_sum(s);
      if (lane == 0 && i0 + u * kWarps < ncols) out[i0 + u * kWarps] = tot;
    }
  }
}

// true in the block that finishes last (no waiting: an atomic ticket)
__device__ __forceinline__ bool last_block(unsigned* counter) {
  __shared__ bool amlast;
  __threadfence();
  __syncthreads();
  const unsigned nblk = gridDim.x * gridDim.y;  // the ticket wraps to 0 for the next launch
  if (threadIdx.x == 0) amlast = atomicInc(counter, nblk - 1) == nblk - 1;
  __syncthreads();
  return amlast;
}

__device__ void block_sum_to(double v, double* red_slot) {
  __shared__ double part[kWarps];
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
#pragma unroll
    for (int k = 0; k < kWarps; ++k) t += part[k];
    *red_slot = t;
  }
}

__device__ void givens_make(double x, double y, double& c, double& s) {
  if (fabs(y) < kEps) { c = 1.0; s = 0.0; }
  else if (fabs(y) > fabs(x)) { double nu = x / y; s = 1.0 / sqrt(1.0 + nu * nu); c = nu * s; }
  else { double nu = y / x; c = 1.0 / sqrt(1.0 + nu * nu); s = nu * c; }
}
__device__ void givens_apply(double c, double s, double& dx, double& dy) {
  double t = c * dx + s * dy;
  dy = -s * dx + c * dy;
  dx = t;
}

// 128-bit vectors of the basis precision: 4 floats or 2 doubles per load
template <typename T> struct Vec4;
template <> struct Vec4<float> {
  using t = float4;
  static constexpr int N = 4;
  __device__ static double dot(const float4& a, const float4& b) {
    return (double)a.x * b.x + (double)a.y * b.y + (double)a.z * b.z + (double)a.w * b.w;
  }
  __device__ static float4 zero() { return make_float4(0.f, 0.f, 0.f, 0.f); }
  __device__ static double get(const float4& a, int e) { return e == 0 ? a.x : e == 1 ? a.y : e == 2 ? a.z : a.w; }
};
template <> struct Vec4<double> {
  using t = double2;
  static constexpr int N = 2;
  __device__ static double dot(const double2& a, const double2& b) { return a.x * b.x + a.y * b.y; }
  __device__ static double2 zero() { return make_double2(0.0, 0.0); }
  __device__ static double get(const double2& a, int e) { return e == 0 ? a.x : a.y; }
};

// last block of pass A: h, the new Gram row, c = h + (h - G h) and H(:,j);
// hs: ncols doubles of shared memory
__device__ void dots_finish(int ncols, int j, const double* __restrict__ red, State st, double* hs) {
  if (gridDim.x <= 32 * 10) finalize_partials_wide<10>(red, gridDim.x, 2 * ncols, st.sums);
  else finalize_partials(red, gridDim.x, 2 * ncols, st.sums);
  __syncthreads();
  // h_i = s_i (u_i . w);  G(i,j) = s_i s_j (u_i . u_j)
  const double sj = st.s[j];
  for (int i = threadIdx.x; i < ncols; i += kThreads) {
    hs[i] = st.sums[i] * st.s[i];
    const double gij = st.s[i] * sj * st.sums[ncols + i];
    st.gm(i, j) = gij;
    st.gm(j, i) = gij;
  }
  __syncthreads();
  // c = h + (h - G h): the second Gram-Schmidt projection from the Gram matrix
  // (one thread per row of G; the loads of a row are independent, so several
  // are in flight while the sum runs in order)
  for (int i = threadIdx.x; i < ncols; i += kThreads) {
    double gh = 0.0;
#pragma unroll 32
    for (int k = 0; k < ncols; ++k) gh += st.gm(i, k) * hs[k];
    const double ci = hs[i] + (hs[i] - gh);
    st.h(i, j) = ci;
    st.c[i] = ci * st.s[i];  // coefficient on the stored (unnormalised) column
  }
}


// 16-byte copy global -> shared that does not pass through registers (cp.async,
// completion tracked per thread by commit / wait groups)
__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// partial dot of one float4 pair, returned in float64: the four products are
// summed in float32 (about one rounding per product, the size of the rounding the
// stored basis itself carries) and converted once, so a float32 element costs a
// quarter of a conversion instead of two
__device__ __forceinline__ double vdot(const float4& a, const float4& b) {
  return (double)fmaf(a.w, b.w, fmaf(a.z, b.z, fmaf(a.y, b.y, a.x * b.x)));
}

// ---- pass A: raw dots u_c . w and u_c . u_j for c < ncols (u = stored columns).
// Blocks own contiguous ranges of 128-bit vectors, walked in chunks of
// kChunk = 32 * kVecPerLane vectors (kVecPerLane per lane).  Warp w streams
// columns w, w+8, ... (CPW of them: the smallest power of two with 8*CPW >= ncols,
// at most 8; past 64 columns further blocks per row range, blockIdx.y = 1, 2, ...,
// take columns 64..127, ...) against w and u_j, keeping per-column partial sums
// in registers.  The column chunks reach the warp through a private ring of
// kStages shared-memory stages filled by cp.async kStages - 1 chunks ahead, so
// the loads in flight hold no registers and no block barrier paces the warps;
// each lane reads back only the vectors it copied itself.  w and u_j, which every
// warp of the block needs, are read per chunk through L1.  Rows past the last full
// vector are summed by the last block.  (Measured on B200, float32 basis, 8M rows,
// restart 50, every step of a cycle: 0.160 ms per step against 0.170 ms with
// double-buffered w/u_j tiles and registers for the column loads; an update pass
// of the same bytes runs at 0.135 ms.)
constexpr int kVecPerLane = 4;
constexpr int kChunk = 32 * kVecPerLane;
constexpr int kStages = 4;
constexpr size_t kDotsStageBytes = (size_t)kWarps * kStages * kChunk * 16;  // 64 KB per block
template <typename T, int CPW>  // T = float
__global__ void __launch_bounds__(kThreads) arnoldi_dots(long long n, long long ld, int ncols, int j,
                                                         const T* __restrict__ V, const T* __restrict__ w,
                                                         double* __restrict__ red, unsigned* counter, State st) {
  static_assert(std::is_same<T, float>::value, "the staged dot pass is the float32-basis form");
  extern __shared__ __align__(16) unsigned char dots_smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float4* stg = reinterpret_cast<float4*>(dots_smem) + (size_t)warp * kStages * kChunk;
  double* hs = reinterpret_cast<double*>(dots_smem + kDotsStageBytes);  // ncols doubles for dots_finish
  const int cbase = blockIdx.y * (kWarps * CPW);
  int nk = 0;  // columns of this warp (uniform over its lanes)
#pragma unroll
  for (int k = 0; k < CPW; ++k) nk += (cbase + warp + k * kWarps < ncols) ? 1 : 0;
  const long long nvec = n / 4;
  const long long per = (nvec + gridDim.x - 1) / gridDim.x;
  const long long v0 = min(nvec, per * blockIdx.x), v1 = min(nvec, v0 + per);
  const float4* __restrict__ wv4 = reinterpret_cast<const float4*>(w);
  const float4* __restrict__ uv4 = reinterpret_cast<const float4*>(V + (size_t)j * ld);
  // a block's row range is a few dozen chunks: 32-bit bookkeeping, advanced
  // incrementally (no division per unit)
  const int nch = (int)((v1 - v0 + kChunk - 1) / kChunk);
  // the producer cursor: next (chunk, column) unit to copy and its stage; one
  // commit group per unit (empty past the end) keeps the wait_group count uniform
  int pch = 0, pk = 0, pst = 0;
  auto issue = [&]() {
    if (pch < nch) {
      const float4* __restrict__ vc = reinterpret_cast<const float4*>(V + (size_t)(cbase + warp + pk * kWarps) * ld);
      float4* dst = stg + pst * kChunk;
      const long long c0 = v0 + (long long)pch * kChunk + lane;
#pragma unroll
      for (int q = 0; q < kVecPerLane; ++q)
        if (c0 + q * 32 < v1) cp_async16(dst + q * 32 + lane, vc + c0 + q * 32);
      if (++pk == nk) { pk = 0; ++pch; }
      if (++pst == kStages) pst = 0;
    }
    cp_async_commit();
  };
  double pw[CPW], pu[CPW];
#pragma unroll
  for (int k = 0; k < CPW; ++k) { pw[k] = 0.0; pu[k] = 0.0; }
  if (nk > 0) {
#pragma unroll
    for (int i = 0; i < kStages - 1; ++i) issue();
  }
  // the copies above read basis columns only (written two or more kernels
  // back); w is the predecessor's output
  pdl_wait();
  pdl_trigger();
  int cst = 0;  // the consumer's stage
  for (int ch = 0; ch < nch && nk > 0; ++ch) {
    const long long c0 = v0 + (long long)ch * kChunk + lane;
    float4 wv[kVecPerLane], uv[kVecPerLane];
#pragma unroll
    for (int q = 0; q < kVecPerLane; ++q) {
      const bool in = c0 + q * 32 < v1;
      wv[q] = in ? __ldg(wv4 + c0 + q * 32) : make_float4(0.f, 0.f, 0.f, 0.f);
      uv[q] = in ? __ldg(uv4 + c0 + q * 32) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
#pragma unroll
    for (int k = 0; k < CPW; ++k) {
      if (k < nk) {
        issue();
        cp_async_wait<kStages - 1>();  // this lane's copies of the unit (ch, k) have landed
        const float4* src = stg + cst * kChunk;
        if (++cst == kStages) cst = 0;
#pragma unroll
        for (int q = 0; q < kVecPerLane; ++q) {
          const float4 v = c0 + q * 32 < v1 ? src[q * 32 + lane] : make_float4(0.f, 0.f, 0.f, 0.f);
          pw[k] += vdot(v, wv[q]);
          pu[k] += vdot(v, uv[q]);
        }
      }
    }
  }
  cp_async_wait<0>();
  if (blockIdx.x == gridDim.x - 1 && lane == 0) {  // rows past the last full vector
    const T* __restrict__ uj = V + (size_t)j * ld;
    for (long long r = nvec * 4; r < n; ++r)
#pragma unroll
      for (int k = 0; k < CPW; ++k) {
        const int c = cbase + warp + k * kWarps;
        if (c < ncols) {
          const double v = (double)V[(size_t)c * ld + r];
          pw[k] += v * (double)w[r];
          pu[k] += v * (double)uj[r];
        }
      }
  }
#pragma unroll
  for (int k = 0; k < CPW; ++k) {
    const int c = cbase + warp + k * kWarps;
    const double a = warp_sum(pw[k]), b = warp_sum(pu[k]);
    if (lane == 0 && c < ncols) {
      red[(size_t)c * gridDim.x + blockIdx.x] = a;
      red[(size_t)(ncols + c) * gridDim.x + blockIdx.x] = b;
    }
  }
  if (!last_block(counter)) return;
  dots_finish(ncols, j, red, st, hs);
}

// ---- pass A, float32 basis, through the bulk-copy (TMA) engine.
// The same units, stages and sums as arnoldi_dots, but each unit (one chunk of
// one column, up to 2 KB) is ONE cp.async.bulk issued by lane 0 of the warp,
// completing on an mbarrier of its stage (transaction bytes); the lanes wait on
// that barrier and read back the whole chunk.  The per-lane copy instructions
// and their address arithmetic go away, which is what bounded the per-lane form
// (an issue-rate limit at 16 warps per SM).  Each lane sums its vectors in the
// same order as arnoldi_dots, so the dots are bit-identical.  Every wait on a
// barrier is bounded: past kSpinLimit polls the kernel records SC_TIMEOUT,
// stops issuing copies, and before returning waits (bounded again) for the
// copies it has in flight.
constexpr size_t kDotsBarBytes = (size_t)kWarps * kStages * sizeof(unsigned long long);
constexpr unsigned kSpinLimit = 1u << 24;
enum { SC_TIMEOUT = 3 };

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// true once the barrier's phase `parity` has completed, false after kSpinLimit polls
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* b, unsigned parity) {
  for (unsigned it = 0; it < kSpinLimit; ++it)
    if (mbar_try_wait(b, parity)) return true;
  return false;
}
__device__ __forceinline__ unsigned long long policy_evict_first() {
  unsigned long long p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;\n" : "=l"(p));
  return p;
}
// global -> shared bulk copy (16-byte aligned addresses, size a multiple of 16)
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* b,
                                         unsigned long long policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;\n" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(b)), "l"(policy)
      : "memory");
}

template <int CPW>
__global__ void __launch_bounds__(kThreads) arnoldi_dots_bulk(long long n, long long ld, int ncols, int j,
                                                              const float* __restrict__ V, const float* __restrict__ w,
                                                              double* __restrict__ red, unsigned* counter, State st) {
  extern __shared__ __align__(128) unsigned char dots_smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float4* stg = reinterpret_cast<float4*>(dots_smem) + (size_t)warp * kStages * kChunk;
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(dots_smem + kDotsStageBytes) + warp * kStages;
  double* hs = reinterpret_cast<double*>(dots_smem + kDotsStageBytes + kDotsBarBytes);  // ncols doubles
  const int cbase = blockIdx.y * (kWarps * CPW);
  int nk = 0;  // columns of this warp (uniform over its lanes)
#pragma unroll
  for (int k = 0; k < CPW; ++k) nk += (cbase + warp + k * kWarps < ncols) ? 1 : 0;
  const long long nvec = n / 4;
  const long long per = (nvec + gridDim.x - 1) / gridDim.x;
  const long long v0 = min(nvec, per * blockIdx.x), v1 = min(nvec, v0 + per);
  const int nvb = (int)(v1 - v0);  // 16-byte vectors of this block's row range
  const int nch = (nvb + kChunk - 1) / kChunk;
  const int nunits = nch * nk;
  if (lane == 0) {
#pragma unroll
    for (int s = 0; s < kStages; ++s) mbar_init(bar + s, 1);
    fence_async_shared();
  }
  __syncwarp();
  const unsigned long long pol = policy_evict_first();
  const float4* __restrict__ Vv = reinterpret_cast<const float4*>(V);
  const long long ldv = ld / 4;
  // producer cursor (kept by every lane, used by lane 0): next unit, its chunk,
  // its column slot and its stage
  int pu = 0, pch = 0, pk = 0, pst = 0;
  bool dead = false;  // a barrier wait ran out: no further copies
  auto issue = [&]() {
    if (pu < nunits && !dead) {
      if (lane == 0) {
        const int off = pch * kChunk;
        const unsigned bytes = (unsigned)min(kChunk, nvb - off) * 16u;
        const float4* src = Vv + (size_t)(cbase + warp + pk * kWarps) * ldv + v0 + off;
        fence_async_shared();  // the lanes' reads of this stage (ordered by __syncwarp) before the copy's writes
        mbar_expect_tx(bar + pst, bytes);
        bulk_g2s(stg + pst * kChunk, src, bytes, bar + pst, pol);
      }
      ++pu;
      if (++pk == nk) { pk = 0; ++pch; }
      if (++pst == kStages) pst = 0;
    }
  };
#pragma unroll
  for (int i = 0; i < kStages - 1; ++i) issue();
  // the copies above read basis columns only (written two or more kernels
  // back); w is the predecessor's output
  pdl_wait();
  pdl_trigger();
  const float4* __restrict__ wv4 = reinterpret_cast<const float4*>(w);
  const float4* __restrict__ uv4 = Vv + (size_t)j * ldv;
  double pw[CPW], pq[CPW];
#pragma unroll
  for (int k = 0; k < CPW; ++k) { pw[k] = 0.0; pq[k] = 0.0; }
  int cu = 0, cst = 0;  // the consumer's unit and stage
  unsigned cph = 0;     // parity of the stage's current phase (flips when cst wraps)
  for (int ch = 0; ch < nch && nk > 0 && !dead; ++ch) {
    const int cnt = min(kChunk, nvb - ch * kChunk);
    const long long c0 = v0 + (long long)ch * kChunk + lane;
    float4 wv[kVecPerLane], uv[kVecPerLane];
#pragma unroll
    for (int q = 0; q < kVecPerLane; ++q) {
      const bool in = lane + q * 32 < cnt;
      wv[q] = in ? __ldg(wv4 + c0 + q * 32) : make_float4(0.f, 0.f, 0.f, 0.f);
      uv[q] = in ? __ldg(uv4 + c0 + q * 32) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
#pragma unroll
    for (int k = 0; k < CPW; ++k) {
      if (k < nk && !dead) {
        issue();  // unit cu + kStages - 1 into the stage unit cu - 1 used
        // the outcome is made warp-uniform, so the lanes stay converged
        if (!__all_sync(0xffffffffu, mbar_wait_bounded(bar + cst, cph))) {
          dead = true;
          if (lane == 0) st.sc[SC_TIMEOUT] = 1.0;
          break;
        }
        const float4* src = stg + cst * kChunk;
#pragma unroll
        for (int q = 0; q < kVecPerLane; ++q) {
          if (lane + q * 32 < cnt) {
            const float4 v = src[q * 32 + lane];
            pw[k] += vdot(v, wv[q]);
            pq[k] += vdot(v, uv[q]);
          }
        }
        __syncwarp();
        ++cu;
        if (++cst == kStages) { cst = 0; cph ^= 1u; }
      }
    }
  }
  if (dead) {  // let the copies in flight land before the block's shared memory goes away
    for (; cu < pu; ++cu) {
      mbar_wait_bounded(bar + cst, cph);
      if (++cst == kStages) { cst = 0; cph ^= 1u; }
    }
  }
  if (blockIdx.x == gridDim.x - 1 && lane == 0) {  // rows past the last full vector
    const float* __restrict__ uj = V + (size_t)j * ld;
    for (long long r = nvec * 4; r < n; ++r)
#pragma unroll
      for (int k = 0; k < CPW; ++k) {
        const int c = cbase + warp + k * kWarps;
        if (c < ncols) {
          const double v = (double)V[(size_t)c * ld + r];
          pw[k] += v * (double)w[r];
          pq[k] += v * (double)uj[r];
        }
      }
  }
#pragma unroll
  for (int k = 0; k < CPW; ++k) {
    const int c = cbase + warp + k * kWarps;
    const double a = warp_sum(pw[k]), b = warp_sum(pq[k]);
    if (lane == 0 && c < ncols) {
      red[(size_t)c * gridDim.x + blockIdx.x] = a;
      red[(size_t)(ncols + c) * gridDim.x + blockIdx.x] = b;
    }
  }
  if (!last_block(counter)) return;
  dots_finish(ncols, j, red, st, hs);
}

// ---- pass A for the float64 basis: the same dots with w and u_j held in
// registers: warp w owns columns w, w+8, ...; each lane loads its 128-bit vectors
// of w and u_j once per step and streams its columns against them (no barriers;
// the block's warps share w and u_j through L1).  Measured on B200 at restart 50
// on the 8M-row system: 0.62 ms per iteration for the whole orthogonalisation,
// against 0.83 ms with the shared-memory tiles of the float32 form.
template <typename T>
__global__ void __launch_bounds__(kThreads) arnoldi_dots_reg(long long n, long long ld, int ncols, int j,
                                                             const T* __restrict__ V, const T* __restrict__ w,
                                                             double* __restrict__ red, unsigned* counter, State st) {
  using VT = typename Vec4<T>::t;
  constexpr int N = Vec4<T>::N;
  pdl_wait();
  pdl_trigger();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int cbase = blockIdx.y * kColsD;  // block row y of the grid takes columns 64y .. 64y + 63
  const long long nvec = n / N;
  const long long per = (nvec + gridDim.x - 1) / gridDim.x;
  const long long v0 = per * blockIdx.x, v1 = min(nvec, v0 + per);
  const VT* __restrict__ wv4 = reinterpret_cast<const VT*>(w);
  const VT* __restrict__ uv4 = reinterpret_cast<const VT*>(V + (size_t)j * ld);
  double pw[8], pu[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) { pw[k] = 0.0; pu[k] = 0.0; }
  for (long long base = v0; base < v1; base += 32 * kVecPerLane) {
    VT wv[kVecPerLane], uv[kVecPerLane];
#pragma unroll
    for (int q = 0; q < kVecPerLane; ++q) {
      const long long vi = base + lane + 32 * q;
      wv[q] = vi < v1 ? wv4[vi] : Vec4<T>::zero();
      uv[q] = vi < v1 ? uv4[vi] : Vec4<T>::zero();
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int c = cbase + warp + k * kWarps;
      if (c < ncols) {
        const VT* __restrict__ vc = reinterpret_cast<const VT*>(V + (size_t)c * ld);
        VT v[kVecPerLane];
#pragma unroll
        for (int q = 0; q < kVecPerLane; ++q) {
          const long long vi = base + lane + 32 * q;
          v[q] = vi < v1 ? __ldcs(vc + vi) : Vec4<T>::zero();
        }
#pragma unroll
        for (int q = 0; q < kVecPerLane; ++q) {
          pw[k] += Vec4<T>::dot(v[q], wv[q]);
          pu[k] += Vec4<T>::dot(v[q], uv[q]);
        }
      }
    }
  }
  if (blockIdx.x == gridDim.x - 1 && lane == 0) {  // rows past the last full vector
    const T* __restrict__ uj = V + (size_t)j * ld;
    for (long long r = nvec * N; r < n; ++r)
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int c = cbase + warp + k * kWarps;
        if (c < ncols) {
          const double v = (double)V[(size_t)c * ld + r];
          pw[k] += v * (double)w[r];
          pu[k] += v * (double)uj[r];
        }
      }
  }
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int c = cbase + warp + k * kWarps;
    const double a = warp_sum(pw[k]), b = warp_sum(pu[k]);
    if (lane == 0 && c < ncols) {
      red[(size_t)c * gridDim.x + blockIdx.x] = a;
      red[(size_t)(ncols + c) * gridDim.x + blockIdx.x] = b;
    }
  }
  if (!last_block(counter)) return;
  extern __shared__ double dyn_hs[];
  dots_finish(ncols, j, red, st, dyn_hs);
}

// Dynamic shared memory that lets at most `blocks` blocks of a kernel share an
// SM (and still lets `blocks` fit): the single-wave grid-stride passes size
// their grids as `blocks` per SM, and under programmatic launch their blocks
// are placed while the previous kernel still holds part of the GPU; if an SM
// could take more, the early SMs fill up and the grid's equal shares pile on
// fewer SMs.  (Measured on the 1.5M-row system: the float32 dot pass with room
// for three blocks per SM took 0.330 ms per iteration against 0.259 ms capped.)
size_t smem_for_blocks(int blocks, size_t need) {
  static std::mutex mu;
  static std::vector<std::pair<int, int>> per_dev;  // (shared memory per SM, reserved per block)
  int dev = 0;
  DECO_CUDA(cudaGetDevice(&dev));
  std::pair<int, int> a;
  {
    std::lock_guard<std::mutex> lk(mu);
    if ((int)per_dev.size() <= dev) per_dev.resize(dev + 1, {0, 0});
    if (!per_dev[dev].first) {
      DECO_CUDA(cudaDeviceGetAttribute(&per_dev[dev].first, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
      DECO_CUDA(cudaDeviceGetAttribute(&per_dev[dev].second, cudaDevAttrReservedSharedMemoryPerBlock, dev));
    }
    a = per_dev[dev];
  }
  const size_t sm = (size_t)a.first, res = (size_t)a.second;
  // blocks + 1 blocks would need more than the SM has, whatever the kernel's
  // static shared memory and the allocation rounding; `blocks` still fit with
  // up to 1 KB of static shared memory each
  const size_t cap = (sm / (blocks + 1) + 15) / 16 * 16;
  if (need >= cap || (size_t)blocks * (cap + res + 1024) > sm) return need;
  return cap;
}

constexpr size_t kDotsShmMax = 96 * 1024;  // the dot passes' dynamic shared memory limit

// the staged float32 dot passes need more than the 48 KB of shared memory a
// block gets by default: raise the limit once per (instantiation, device)
template <int CPW>
void allow_dots_smem() {
  static std::mutex mu;
  static std::vector<int> done;
  int dev = 0;
  DECO_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if ((int)done.size() <= dev) done.resize(dev + 1, 0);
  if (done[dev]) return;
  static_assert(kDotsStageBytes + kDotsBarBytes + sizeof(double) * (kMaxRestart + 1) <= kDotsShmMax, "dot pass smem");
  DECO_CUDA(cudaFuncSetAttribute(arnoldi_dots<float, CPW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kDotsShmMax));
  DECO_CUDA(cudaFuncSetAttribute(arnoldi_dots_bulk<CPW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kDotsShmMax));
  done[dev] = 1;
}

// The float32 dot pass at two blocks per SM: the per-lane cp.async form for up
// to 16 columns, the bulk-copy form from 17 (measured per launch on the 4M-row
// system: 33.5 / 50.8 us per-lane against 36.4 / 52.2 us bulk at 1 and 2
// columns per warp, 86.9 against 77.8 us at 4).
template <int CPW>
void launch_dots_f32(cudaStream_t s, dim3 grid, size_t shm, long long n, long long ld, int nc, int j, const float* V,
                     const float* w, double* red, unsigned* counter, State st) {
  allow_dots_smem<CPW>();
  if (CPW >= 4)
    launch_k(arnoldi_dots_bulk<CPW>, grid, kThreads, smem_for_blocks(2, kDotsStageBytes + kDotsBarBytes + shm), s, n,
             ld, nc, j, V, w, red, counter, st);
  else
    launch_k(arnoldi_dots<float, CPW>, grid, kThreads, smem_for_blocks(2, kDotsStageBytes + shm), s, n, ld, nc, j, V, w,
             red, counter, st);
}

template <typename T>
void launch_arnoldi_dots(cudaStream_t s, int nb, long long n, long long ld, int nc, int j, const T* V, const T* w,
                         double* red, unsigned* counter, State st) {
  const size_t shm = sizeof(double) * (size_t)nc;  // h for the last block (dots_finish)
  if constexpr (std::is_same<T, double>::value) {
    launch_k(arnoldi_dots_reg<T>, dim3(nb, (nc + kColsD - 1) / kColsD), kThreads, shm, s, n, ld, nc, j, V, w, red,
             counter, st);
  } else {
    // two blocks per SM of 64 KB stages each (measured at restart 50 on 8M rows:
    // 0.160 ms per step against 0.170 with three blocks per SM)
    const int nbd = nb / 2;
    if (nc <= kWarps) launch_dots_f32<1>(s, nbd, shm, n, ld, nc, j, V, w, red, counter, st);
    else if (nc <= 2 * kWarps) launch_dots_f32<2>(s, nbd, shm, n, ld, nc, j, V, w, red, counter, st);
    else if (nc <= 4 * kWarps) launch_dots_f32<4>(s, nbd, shm, n, ld, nc, j, V, w, red, counter, st);
    else  // 8 columns per warp; past 64 columns further block rows, 64 columns each
      launch_dots_f32<8>(s, dim3(nbd, (nc + kColsD - 1) / kColsD), shm, n, ld, nc, j, V, w, red, counter, st);
  }
}

// ---- pass B: w'' = w - sum_c coef_c u_c, stored as column j+1; ||w''||^2.
// One thread per 128-bit vector of rows; the columns go in batches of U whose
// loads are all issued before their products, so U independent 16-byte loads
// per thread are in flight (U = 16 float32 / 8 float64; each element still
// subtracts the columns in order).  Measured on B200, float32 basis, 8M rows,
// restart 50: 0.135 ms per step against 0.152 ms with the column loop unrolled by 4.
// Dynamic shared memory: 4 (ncols + 1) doubles (the coefficients, then column j
// of H and the earlier rotations for the last block).
template <typename T>
__global__ void __launch_bounds__(kThreads) arnoldi_update(long long n, long long ld, int ncols, int j,
                                                           const T* __restrict__ V, const T* __restrict__ w,
                                                           T* __restrict__ out, double* __restrict__ red,
                                                           unsigned* counter, State st, HostSlot hs) {
  using VT = typename Vec4<T>::t;
  constexpr int N = Vec4<T>::N;
  constexpr int U = N == 4 ? 16 : 8;
  extern __shared__ double dyn_u[];
  const long long nvec = n / N;
  // Before the dependency wait: L2 prefetches of this thread's first vector of w
  // and of up to U basis columns (written two or more kernels back; only the
  // coefficients come from the dot pass), so that DRAM traffic overlaps the dot
  // pass's last block forming the coefficients.  No registers are held.
  {
    const long long v0 = (long long)blockIdx.x * kThreads + threadIdx.x;
    if (v0 < nvec) {
      asm volatile("prefetch.global.L2 [%0];\n" ::"l"(reinterpret_cast<const VT*>(w) + v0));
      const int np = ncols < U ? ncols : U;
      for (int u = 0; u < np; ++u)
        asm volatile("prefetch.global.L2 [%0];\n" ::"l"(reinterpret_cast<const VT*>(V + (size_t)u * ld) + v0));
    }
  }
  pdl_wait();
  pdl_trigger();
  double* cs_ = dyn_u;
  for (int i = threadIdx.x; i < ncols; i += kThreads) cs_[i] = st.c[i];
  __syncthreads();
  double ss = 0.0;
  for (long long vi = (long long)blockIdx.x * kThreads + threadIdx.x; vi < nvec;
       vi += (long long)gridDim.x * kThreads) {
    const VT wv = reinterpret_cast<const VT*>(w)[vi];
    double x[N];
#pragma unroll
    for (int e = 0; e < N; ++e) x[e] = Vec4<T>::get(wv, e);
    int i = 0;
    for (; i + U <= ncols; i += U) {
      VT v[U];
#pragma unroll
      for (int u = 0; u < U; ++u) v[u] = __ldcs(reinterpret_cast<const VT*>(V + (size_t)(i + u) * ld) + vi);
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const double ci = cs_[i + u];
#pragma unroll
        for (int e = 0; e < N; ++e) x[e] -= ci * Vec4<T>::get(v[u], e);
      }
    }
    for (; i < ncols; ++i) {
      const VT v = __ldcs(reinterpret_cast<const VT*>(V + (size_t)i * ld) + vi);
      const double ci = cs_[i];
#pragma unroll
      for (int e = 0; e < N; ++e) x[e] -= ci * Vec4<T>::get(v, e);
    }
    T o[N];
#pragma unroll
    for (int e = 0; e < N; ++e) {
      o[e] = (T)x[e];
      ss += (double)o[e] * (double)o[e];
    }
    VT ov;
    if constexpr (N == 4) ov = make_float4(o[0], o[1], o[2], o[3]);
    else ov = make_double2(o[0], o[1]);
    reinterpret_cast<VT*>(out)[vi] = ov;
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) {  // rows past the last full vector
    for (long long r = nvec * N; r < n; ++r) {
      double x = (double)w[r];
      for (int i = 0; i < ncols; ++i) x -= cs_[i] * (double)V[(size_t)i * ld + r];
      const T xq = (T)x;
      out[r] = xq;
      ss += (double)xq * (double)xq;
    }
  }
  block_sum_to(ss, red + blockIdx.x);
  if (!last_block(counter)) return;
  finalize_partials(red, gridDim.x, 1, st.sc + SC_BETA);
  // the rotations run on a shared-memory copy of column j and of the earlier
  // rotations (one thread, a chain of j dependent updates)
  double* hc = dyn_u + (ncols + 1);  // j + 2 entries
  double* rc = hc + (ncols + 1);     // j entries
  double* rs = rc + (ncols + 1);
  for (int i = threadIdx.x; i <= j; i += kThreads) hc[i] = st.h(i, j);
  for (int i = threadIdx.x; i < j; i += kThreads) { rc[i] = st.cs[i]; rs[i] = st.sn[i]; }
  __syncthreads();
  if (threadIdx.x == 0) {
    const double beta = sqrt(st.sc[SC_BETA]);
    hc[j + 1] = beta;
    st.s[j + 1] = beta != 0.0 ? 1.0 / beta : 0.0;
    for (int i = 0; i <= j - 1; ++i) givens_apply(rc[i], rs[i], hc[i], hc[i + 1]);
    givens_make(hc[j], hc[j + 1], st.cs[j], st.sn[j]);
    givens_apply(st.cs[j], st.sn[j], hc[j], hc[j + 1]);
    givens_apply(st.cs[j], st.sn[j], st.g[j], st.g[j + 1]);
    st.sc[SC_RES] = fabs(st.g[j + 1]);
    hs.post(st.sc[SC_RES]);
  }
  __syncthreads();
  for (int i = threadIdx.x; i <= j + 1; i += kThreads) st.h(i, j) = hc[i];
}

// ---- column 0: u_0 = r, s_0 = 1/||r||, g_0 = ||r|| (rgmres.tpp:54-55); out[0] = ||r||
template <typename T>
__global__ void __launch_bounds__(kThreads) start_cycle(long long n, const double* __restrict__ r, T* __restrict__ u0,
                                                        double* __restrict__ red, unsigned* counter, State st,
                                                        double* __restrict__ out) {
  double ss = 0.0, sq = 0.0;
  for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kThreads) {
    const double v = r[i];
    const T vq = (T)v;
    u0[i] = vq;
    ss += v * v;
    sq += (double)vq * (double)vq;
  }
  block_sum_to(ss, red + blockIdx.x);
  block_sum_to(sq, red + gridDim.x + blockIdx.x);
  if (!last_block(counter)) return;
  finalize_partials(red, gridDim.x, 2, out);
  __syncthreads();
  if (threadIdx.x == 0) {
    const double nrm = sqrt(out[0]), nq = sqrt(out[1]);
    out[0] = nrm;
    st.g[0] = nrm;
    st.s[0] = nq != 0.0 ? 1.0 / nq : 0.0;  // scale of the stored column
  }
}

// ---- ||x||_2 in float64, deterministic
template <typename X>
__global__ void __launch_bounds__(kThreads) norm2_kernel(long long n, const X* __restrict__ x, double* __restrict__ red,
                                                         unsigned* counter, double* __restrict__ out) {
  double ss = 0.0;
  for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kThreads) {
    const double v = (double)x[i];
    ss += v * v;
  }
  block_sum_to(ss, red + blockIdx.x);
  if (!last_block(counter)) return;
  finalize_partials(red, gridDim.x, 1, out);
  __syncthreads();
  if (threadIdx.x == 0) out[0] = sqrt(out[0]);
}

// back substitution g(1:j) = H(1:j,1:j) \ g(1:j)  (rgmres.tpp:95-104), then the
// coefficients on the stored columns c_i = y_i s_i
// One block: the upper triangle of H's first j columns (packed by columns,
// H(k,i) at i (i + 1) / 2 + k) and g are staged in dynamic shared memory when
// SHM, then column by column g_i /= H(i,i) and, in parallel over k < i,
// g_k -= H(k,i) g_i (every element sees the same operations in the same order as
// the sequential column-oriented substitution).  Without SHM the same
// arithmetic reads H from global memory (orders past kBacksolveShm).
template <bool SHM>
__global__ void __launch_bounds__(kThreads) backsolve(State st, int j) {
  extern __shared__ double dyn_b[];
  double* g = dyn_b;       // j + 1 doubles
  double* hs = g + j + 1;  // j (j + 1) / 2 doubles (SHM)
  auto H = [&](int k, int i) -> double { return SHM ? hs[(size_t)i * (i + 1) / 2 + k] : st.h(k, i); };
  if (SHM)
    for (int i = 0; i < j; ++i)
      for (int k = threadIdx.x; k <= i; k += kThreads) hs[(size_t)i * (i + 1) / 2 + k] = st.h(k, i);
  for (int k = threadIdx.x; k <= j; k += kThreads) g[k] = st.g[k];
  __syncthreads();
  for (int i = j - 1; i >= 0; --i) {
    const double hii = H(i, i);
    if (hii == 0.0) {  // the same value in every thread: the whole block leaves
      if (threadIdx.x == 0) st.sc[SC_BREAK] = 1.0;
      return;
    }
    if (threadIdx.x == 0) g[i] /= hii;
    __syncthreads();
    const double gi = g[i];
    for (int k = threadIdx.x; k < i; k += kThreads) g[k] -= H(k, i) * gi;
    __syncthreads();
  }
  if (threadIdx.x == 0) st.sc[SC_BREAK] = 0.0;
  for (int k = threadIdx.x; k <= j; k += kThreads) st.g[k] = g[k];
  const int nc = j > 0 ? j : 1;
  for (int i = threadIdx.x; i < nc; i += kThreads) st.c[i] = g[i] * st.s[i];
}

void launch_backsolve(cudaStream_t s, State st, int j) {
  if (j <= kBacksolveShm) {
    const size_t shm = sizeof(double) * ((size_t)j + 1 + (size_t)j * (j + 1) / 2);
    if (shm > 48 * 1024) {
      static_assert(sizeof(double) * (kBacksolveShm + 1 + kBacksolveShm * (kBacksolveShm + 1) / 2) <= 227 * 1024,
                    "back-substitution triangle must fit the opt-in shared memory");
      DECO_CUDA(cudaFuncSetAttribute(backsolve<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
    }
    backsolve<true><<<1, kThreads, shm, s>>>(st, j);
  } else {
    backsolve<false><<<1, kThreads, sizeof(double) * ((size_t)j + 1), s>>>(st, j);
  }
}

// out = sum_{i < ncols} c_i u_i  (rgmres.tpp:106-109: w = g_0 v_0, then w += g_i v_i)
template <typename T, typename Y>
__global__ void __launch_bounds__(kThreads) combine(long long n, long long ld, int ncols, const T* __restrict__ V,
                                                    const double* __restrict__ c, Y* __restrict__ out) {
  // one thread per 128-bit vector of rows, coefficients in shared memory, the
  // column loop unrolled so several vector loads are in flight (each element
  // sums in the same order as a row-by-row loop)
  using VT = typename Vec4<T>::t;
  constexpr int N = Vec4<T>::N;
  extern __shared__ double cs[];  // ncols doubles
  for (int i = threadIdx.x; i < ncols; i += kThreads) cs[i] = c[i];
  __syncthreads();
  const long long nvec = n / N;
  for (long long vi = (long long)blockIdx.x * kThreads + threadIdx.x; vi < nvec;
       vi += (long long)gridDim.x * kThreads) {
    double s[N];
    {
      const VT v = __ldcs(reinterpret_cast<const VT*>(V) + vi);
#pragma unroll
      for (int e = 0; e < N; ++e) s[e] = cs[0] * Vec4<T>::get(v, e);
    }
#pragma unroll 4
    for (int i = 1; i < ncols; ++i) {
      const VT v = __ldcs(reinterpret_cast<const VT*>(V + (size_t)i * ld) + vi);
      const double ci = cs[i];
#pragma unroll
      for (int e = 0; e < N; ++e) s[e] += ci * Vec4<T>::get(v, e);
    }
#pragma unroll
    for (int e = 0; e < N; ++e) out[vi * N + e] = (Y)s[e];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) {  // rows past the last full vector
    for (long long r = nvec * N; r < n; ++r) {
      double s = cs[0] * (double)V[r];
      for (int i = 1; i < ncols; ++i) s += cs[i] * (double)V[(size_t)i * ld + r];
      out[r] = (Y)s;
    }
  }
}

template <typename X>
__global__ void axpy_into(long long n, const X* __restrict__ z, double* __restrict__ x) {
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x)
    x[r] += (double)z[r];
}

template <typename S, typename D>
__global__ void scale_convert(long long n, const S* __restrict__ a, const double* __restrict__ s, D* __restrict__ b) {
  const double f = s ? __ldg(s) : 1.0;
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x)
    b[r] = (D)(f * (double)a[r]);
}

// ------------------------------------------------------------------ driver

template <typename T>
struct Solver {
  deco_ctx_s* ctx;
  deco_csr_s* A;
  deco_cpr_s* P;
  const deco_sol_params& prm;
  long long n, ld;
  int m, nb;
  DevBuf<T> V, w, z;
  DevBuf<double> st_buf, xtmp, r64, norm;
  State st{};
  // DECO_PROFILE=1: events around the phases of every Arnoldi step of a cycle
  bool profile = false;
  int lookahead = 3;  // Arnoldi steps queued beyond the one whose |g| the host is waiting for
  double step_timeout_ms = 600e3;
  std::vector<cudaEvent_t> pev;
  double t_phase[4] = {0, 0, 0, 0};  // precond, matvec, dot pass, update pass
  // the |g| ring: host views, device views, and the tag each slot waits for
  volatile double* hval = nullptr;
  volatile unsigned long long* htag = nullptr;
  double* dval = nullptr;
  unsigned long long* dtag = nullptr;
  unsigned long long tags[kRing] = {};
  ~Solver() {
    for (auto e : pev) cudaEventDestroy(e);
  }

  Solver(deco_ctx_s* c, deco_csr_s* a, deco_cpr_s* p, const deco_sol_params& pr) : ctx(c), A(a), P(p), prm(pr) {
    trace_mark(ctx, "gmres: enter");
    n = A->n;
    ld = (n + 31) / 32 * 32;
    m = prm.restart;
    nb = 4 * ctx->num_sms;
    cudaStream_t s = ctx->stream;
    V.alloc((size_t)ld * (m + 1), s);
    w.alloc(n, s);
    z.alloc(n, s);
    st_buf.alloc(State::doubles(m), s);
    st.bind(st_buf.get(), m);
    xtmp.alloc(n, s);
    r64.alloc(n, s);
    norm.alloc(4, s);
    const size_t need = (size_t)(2 * (m + 2)) * nb;
    if (ctx->red.size() < need) ctx->red.alloc(need, s);
    if (const char* e = std::getenv("DECO_PROFILE")) profile = std::atoi(e) != 0;
    if (const char* e = std::getenv("DECO_LOOKAHEAD")) lookahead = std::max(0, std::min(kRing - 2, std::atoi(e)));
    if (const char* e = std::getenv("DECO_STEP_TIMEOUT")) step_timeout_ms = std::max(1.0, std::atof(e)) * 1e3;
    if (profile) {
      pev.resize(5 * (size_t)(m + 1));
      for (auto& e : pev) DECO_CUDA(cudaEventCreate(&e));
    }
    trace_mark(ctx, "gmres: allocate");
  }

  // adds the phase times of steps [0, steps) of the cycle that just finished
  void collect(int steps) {
    if (!profile) return;
    for (int j = 0; j < steps; ++j) {
      float t[4] = {0, 0, 0, 0};
      for (int q = 0; q < 4; ++q) DECO_CUDA(cudaEventElapsedTime(&t[q], pev[5 * j + q], pev[5 * j + q + 1]));
      for (int q = 0; q < 4; ++q) t_phase[q] += t[q];
    }
  }

  T* col(int i) { return V.get() + (size_t)i * ld; }

  // y = M^{-1} x
  template <typename X, typename Y>
  void precond(const X* x, Y* y) {
    if (!P) {
      scale_convert<X, Y><<<nb, kThreads, 0, ctx->stream>>>(n, x, nullptr, y);
      DECO_CHECK_LAUNCH();
      return;
    }
    if (P->prm.precision == 32) {
      if constexpr (std::is_same<X, double>::value && std::is_same<Y, double>::value) cpr_apply32<double, double>(ctx, P, x, y);
      else if constexpr (std::is_same<X, double>::value && std::is_same<Y, float>::value) cpr_apply32<double, float>(ctx, P, x, y);
      else if constexpr (std::is_same<X, float>::value && std::is_same<Y, float>::value) cpr_apply32<float, float>(ctx, P, x, y);
      else throw Error(DECO_ERR_INTERNAL, "unsupported precision combination");
    } else {
      if constexpr (std::is_same<X, double>::value && std::is_same<Y, double>::value) cpr_apply64(ctx, P, x, y);
      else throw Error(DECO_ERR_UNSUPPORTED, "precision-32 solve needs a CPR built with precision 32");
    }
  }

  // y = s * (A x) in the basis precision, s on the device
  template <typename X>
  void matvec_scaled(const X* x, T* y, const double* s) {
    if constexpr (std::is_same<T, float>::value) spmv<float, X>(ctx, A, x, EpiStoreScaled<float>{y, s});
    else spmv<double, X>(ctx, A, x, EpiStoreScaled<double>{y, s});
  }

  double norm2(const double* x) {
    norm2_kernel<double><<<nb, kThreads, 0, ctx->stream>>>(n, x, ctx->red.get(), ctx->counter.get(), norm.get());
    DECO_CHECK_LAUNCH();
    double h = 0;
    DECO_CUDA(cudaMemcpyAsync(&h, norm.get(), sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    DECO_CUDA(cudaStreamSynchronize(ctx->stream));
    return h;
  }

  // Arnoldi step j: writes column j of H/G, g_{j+1}, rotation j and basis column
  // j+1; the update pass posts |g_{j+1}| into host slot j % kRing with tag tags[j % kRing].
  void arnoldi_step(int j, bool left) {
    cudaStream_t s = ctx->stream;
    const double* sj = st.s + j;
    // phase order per step: [pev0] precond [pev1] matvec [pev2] dot pass [pev3] update
    // pass [pev4] (left GMRES runs the matvec first; its phases are recorded accordingly)
    if (profile) DECO_CUDA(cudaEventRecord(pev[5 * j], s));
    if (!left) {
      precond<T, T>(col(j), z.get());
      if (profile) DECO_CUDA(cudaEventRecord(pev[5 * j + 1], s));
      matvec_scaled<T>(z.get(), w.get(), sj);
    } else {
      matvec_scaled<T>(col(j), z.get(), sj);
      if (profile) DECO_CUDA(cudaEventRecord(pev[5 * j + 1], s));
      precond<T, T>(z.get(), w.get());
    }
    if (profile) DECO_CUDA(cudaEventRecord(pev[5 * j + 2], s));
    const int nc = j + 1;
    launch_arnoldi_dots<T>(s, nb, n, ld, nc, j, V.get(), w.get(), ctx->red.get(), ctx->counter.get(), st);
    DECO_CHECK_LAUNCH();
    if (profile) DECO_CUDA(cudaEventRecord(pev[5 * j + 3], s));
    HostSlot hs;
    hs.val = dval + j % kRing;
    hs.tag = dtag + j % kRing;
    hs.t = tags[j % kRing] = g_step_tag.fetch_add(1, std::memory_order_relaxed) + 1;
    // nb = 4 blocks per SM (smem_for_blocks: no fifth block on an SM)
    launch_k(arnoldi_update<T>, nb, kThreads, smem_for_blocks(4, sizeof(double) * 4 * (nc + 1)), s, n, ld, nc, j,
             V.get(), w.get(), col(j + 1), ctx->red.get(), ctx->counter.get(), st, hs);
    DECO_CHECK_LAUNCH();
    if (profile) DECO_CUDA(cudaEventRecord(pev[5 * j + 4], s));
  }

  // |g_{j+1}| of step j, once the update pass has posted it.  The host polls
  // the tag; every 1024 polls it asks the stream whether it failed or drained,
  // and gives up (DECO_ERR_CUDA) when the step has not finished after
  // DECO_STEP_TIMEOUT seconds (default 600).
  double step_result(int j) {
    const int slot = j % kRing;
    volatile unsigned long long* tp = htag + slot;
    double t0 = -1.0;
    for (unsigned long long spin = 1; *tp != tags[slot]; ++spin) {
      if ((spin & 1023) == 0) {
        const cudaError_t e = cudaStreamQuery(ctx->stream);
        if (e == cudaSuccess) {
          if (*tp == tags[slot]) break;
          throw Error(DECO_ERR_INTERNAL, "gmres: an Arnoldi step finished without posting its residual");
        }
        if (e != cudaErrorNotReady) DECO_CUDA(e);
        const double now =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
        if (t0 < 0.0) t0 = now;
        else if (now - t0 > step_timeout_ms)
          throw Error(DECO_ERR_CUDA, "gmres: an Arnoldi step did not finish within DECO_STEP_TIMEOUT seconds");
      }
    }
    std::atomic_thread_fence(std::memory_order_acquire);
    return hval[slot];
  }

  void run(const double* b, double* x, deco_sol_result* res, double* resvec) {
    cudaStream_t s = ctx->stream;
    // the iteration's products and Arnoldi passes launch programmatically
    // (common.cuh): A and the preconditioner stay constant from here on
    PdlScope pdl(true);
    const bool left = prm.type == 1;
    const int itmax = prm.itmax;
    double* r = r64.get();
    DECO_CUDA(cudaEventRecord(ctx->ev0, s));
    if (!prm.use_x0) {
      DECO_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, s));
      if (left) precond<double, double>(b, r);
      else DECO_CUDA(cudaMemcpyAsync(r, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    } else {
      spmv<double, double>(ctx, A, x, EpiResid<double, double>{b, left ? xtmp.get() : r});
      if (left) precond<double, double>(xtmp.get(), r);
    }
    const double bnorm = left ? norm2(r) : norm2(b);
    const double abstol = prm.reltol * bnorm;
    int flag = 1, iter = 0, restarts = 0;
    double rnorm = 0.0;
    volatile double* hsc = ctx->host_scalars;
    // the ring of posted |g| values and their tags in the context's pinned buffer
    hval = hsc + kSlot0;
    htag = reinterpret_cast<volatile unsigned long long*>(ctx->host_scalars + kTag0);
    {
      void* d = nullptr;
      DECO_CUDA(cudaHostGetDevicePointer(&d, ctx->host_scalars, 0));
      dval = static_cast<double*>(d) + kSlot0;
      dtag = reinterpret_cast<unsigned long long*>(static_cast<double*>(d) + kTag0);
    }
    while (iter < itmax) {
      DECO_CUDA(cudaMemsetAsync(st_buf.get(), 0, sizeof(double) * State::doubles(m), s));
      start_cycle<T><<<nb, kThreads, 0, s>>>(n, r, col(0), ctx->red.get(), ctx->counter.get(), st, norm.get());
      DECO_CHECK_LAUNCH();
      DECO_CUDA(cudaMemcpyAsync(const_cast<double*>(hsc) + 2, norm.get(), sizeof(double), cudaMemcpyDeviceToHost, s));
      DECO_CUDA(cudaStreamSynchronize(s));
      // The reference's loop (rgmres.tpp:58-66) checks |g_j| before Arnoldi step j.
      // Here the host keeps up to `lookahead` steps queued past the |g_j| it is
      // checking, so a late host thread does not leave the GPU idle.  When |g_j|
      // meets the tolerance, steps j.. are dropped: step k wrote only column k of
      // H/G, g_{k+1}, rotation k and basis column k+1, which the back substitution
      // over j columns never reads.
      const int base = iter;
      int j = 0, launched = 0;
      for (;;) {
        if (!(j < m && base + j < itmax)) break;
        double gj = hsc[2];  // |g_0|; step 0 is launched only after it is checked
        if (j > 0) gj = step_result(j - 1);
        rnorm = fabs(gj);
        if (resvec) resvec[base + j] = rnorm / bnorm;
        if (rnorm < abstol) { flag = 0; break; }
        while (launched < m && base + launched < itmax && launched <= j + lookahead) {
          arnoldi_step(launched, left);
          ++launched;
        }
        ++j;
      }
      iter = base + j;
      launch_backsolve(s, st, j);
      DECO_CHECK_LAUNCH();
      // sc[SC_BREAK .. SC_TIMEOUT] -> hsc[16 ..]
      DECO_CUDA(cudaMemcpyAsync(const_cast<double*>(hsc) + 16, st.sc + SC_BREAK,
                                sizeof(double) * (SC_TIMEOUT - SC_BREAK + 1), cudaMemcpyDeviceToHost, s));
      DECO_CUDA(cudaStreamSynchronize(s));
      if (hsc[16 + SC_TIMEOUT - SC_BREAK] != 0.0)
        throw Error(DECO_ERR_CUDA, "Arnoldi dot pass: a bulk copy into shared memory did not complete");
      if (hsc[16] != 0.0)
        throw Error(DECO_ERR_BREAKDOWN, "Error in rgmres: Zero diagonal element in upper triangular matrix.");
      collect(launched);
      combine<T, double><<<nb, kThreads, sizeof(double) * (j > 0 ? j : 1), s>>>(n, ld, j > 0 ? j : 1, V.get(), st.c,
                                                                                 xtmp.get());
      DECO_CHECK_LAUNCH();
      if (!left) {
        precond<double, double>(xtmp.get(), r);  // r is scratch for z here
        axpy_into<double><<<nb, kThreads, 0, s>>>(n, r, x);
        DECO_CHECK_LAUNCH();
        spmv<double, double>(ctx, A, x, EpiResid<double, double>{b, r});
      } else {
        axpy_into<double><<<nb, kThreads, 0, s>>>(n, xtmp.get(), x);
        DECO_CHECK_LAUNCH();
        spmv<double, double>(ctx, A, x, EpiResid<double, double>{b, xtmp.get()});
        precond<double, double>(xtmp.get(), r);
      }
      ++restarts;
      rnorm = norm2(r);
      if (rnorm < abstol) { flag = 0; break; }
    }
    DECO_CUDA(cudaEventRecord(ctx->ev1, s));
    DECO_CUDA(cudaEventSynchronize(ctx->ev1));
    float ms = 0.f;
    DECO_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    trace_mark(ctx, "gmres: solve");
    res->iter = iter;
    res->flag = flag;
    res->res_abs = rnorm;
    res->res_rel = rnorm / bnorm;
    res->t_solve_ms = ms;
    res->restarts = restarts;
    res->t_precond_ms = t_phase[0];
    res->t_matvec_ms = t_phase[1];
    res->t_ortho_ms = t_phase[2] + t_phase[3];
    res->t_dots_ms = t_phase[2];
    // the residual of the original (not decoupled) system: b - A x on the
    // decoupled system, mapped back through the inverse of the CPR's decoupling
    spmv<double, double>(ctx, A, x, EpiResid<double, double>{b, xtmp.get()});
    res->res_rel_orig = P ? cpr_original_relres(ctx, P, xtmp.get(), b) : norm2(xtmp.get()) / norm2(b);
    if (prm.verbosity > 0) {
      std::printf("\n--------------------------------\n");
      std::printf("Profile of %s:\n", left ? "lGMRES" : "rGMRES");
      std::printf("iteration count =  %d\n", iter);
      std::printf("residual = %.2e\n", rnorm / bnorm);
    }
  }
};

}  // namespace

}  // namespace deco

using namespace deco;

extern "C" {

int deco_gmres_solve(deco_ctx ctx, deco_csr A, deco_cpr P, const double* b, double* x, const deco_sol_params* prm,
                     deco_sol_result* res, double* resvec) {
  return guard([&] {
    DECO_REQUIRE(ctx && A && b && x && prm && res, DECO_ERR_ARG, "NULL argument");
    DECO_REQUIRE(prm->type == 0 || prm->type == 1, DECO_ERR_ARG, "type must be 0 (rgmres) or 1 (lgmres)");
    DECO_REQUIRE(prm->restart >= 1, DECO_ERR_ARG, "restart must be >= 1");
    DECO_REQUIRE(prm->restart <= kMaxRestart, DECO_ERR_UNSUPPORTED,
                 "restart must be <= " + std::to_string(kMaxRestart) + " on this path");
    DECO_REQUIRE(prm->itmax >= 0, DECO_ERR_ARG, "itmax must be >= 0");
    DECO_REQUIRE(prm->precision == 64 || prm->precision == 32, DECO_ERR_ARG, "precision must be 64 or 32");
    DECO_REQUIRE(A->n == A->m, DECO_ERR_ARG, "A must be square");
    if (P) DECO_REQUIRE(P->n == A->n, DECO_ERR_ARG, "preconditioner size does not match A");
    if (prm->precision == 32) {
      DECO_REQUIRE(!P || P->prm.precision == 32, DECO_ERR_ARG, "precision-32 solve needs a CPR built with precision 32");
      if (!A->v32) make_f32_values(ctx, A);
      Solver<float> S(ctx, A, P, *prm);
      S.run(b, x, res, resvec);
    } else {
      Solver<double> S(ctx, A, P, *prm);
      S.run(b, x, res, resvec);
    }
  });
}

}  // extern "C"
