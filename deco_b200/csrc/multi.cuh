// multi.cuh — products with K right-hand sides at once, for the batched solve.
//
// Multi-vectors are row-interleaved: X[row * K + k], so the K values a matrix
// entry multiplies sit in one 32-byte (float) or 64-byte (double) segment and
// every entry of the matrix is read once for all K columns.  The kernel is the
// cell-block product of spmv.cuh widened to K columns: a sub-warp of SW lanes
// owns a block row (BS matrix rows), lanes take whole blocks, and the BS x K
// sums of the block row stay in registers until the sub-warp reduction; then
// the lanes share the NR x K epilogue writes.  A scalar CSR matrix is the BS = 1
// case (one column index per entry, one value plane).
#pragma once
#include "spmv.cuh"

namespace deco {

// K values of one multi-vector row from / to doubles with 16-byte accesses
// (scalar ones when K does not fill them)
template <int K, typename T>
__device__ __forceinline__ void row_load(const T* __restrict__ p, double* v) {
  if (reinterpret_cast<uintptr_t>(p) % 16 != 0) {  // a caller's vector that is not 16-byte aligned
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = (double)p[k];
    return;
  }
  if constexpr (sizeof(T) == 4 && K % 4 == 0) {
#pragma unroll
    for (int q = 0; q < K / 4; ++q) {
      const float4 t = reinterpret_cast<const float4*>(p)[q];
      v[4 * q] = t.x; v[4 * q + 1] = t.y; v[4 * q + 2] = t.z; v[4 * q + 3] = t.w;
    }
  } else if constexpr (sizeof(T) == 8 && K % 2 == 0) {
#pragma unroll
    for (int q = 0; q < K / 2; ++q) {
      const double2 t = reinterpret_cast<const double2*>(p)[q];
      v[2 * q] = t.x; v[2 * q + 1] = t.y;
    }
  } else {
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = (double)p[k];
  }
}
template <int K, typename T>
__device__ __forceinline__ void row_store(T* p, const double* v) {
  if (reinterpret_cast<uintptr_t>(p) % 16 != 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) p[k] = (T)v[k];
    return;
  }
  if constexpr (sizeof(T) == 4 && K % 4 == 0) {
#pragma unroll
    for (int q = 0; q < K / 4; ++q)
      reinterpret_cast<float4*>(p)[q] =
          make_float4((float)v[4 * q], (float)v[4 * q + 1], (float)v[4 * q + 2], (float)v[4 * q + 3]);
  } else if constexpr (sizeof(T) == 8 && K % 2 == 0) {
#pragma unroll
    for (int q = 0; q < K / 2; ++q) reinterpret_cast<double2*>(p)[q] = make_double2(v[2 * q], v[2 * q + 1]);
  } else {
#pragma unroll
    for (int k = 0; k < K; ++k) p[k] = (T)v[k];
  }
}

// ------------------------------------------------------------ epilogues
// epi.row(row, v): all K values of one output row at once (16-byte accesses;
// the same per-element arithmetic as epi(row, k, v[k]))
// epi(row, k, value): value = (A X)[row][k] (row = cell for a restricted product)
template <int K, typename YT> struct MStore {
  YT* y;
  __device__ void operator()(int row, int k, double v) const { y[(long long)row * K + k] = (YT)v; }
  __device__ void row(int row, const double* v) const { row_store<K>(y + (long long)row * K, v); }
};
template <int K, typename YT> struct MAdd {
  YT* y;
  __device__ void operator()(int row, int k, double v) const {
    const long long o = (long long)row * K + k;
    y[o] = (YT)((double)y[o] + v);
  }
  __device__ void row(int row, const double* v) const {
    double o[K];
    row_load<K>(y + (long long)row * K, o);
#pragma unroll
    for (int k = 0; k < K; ++k) o[k] = o[k] + v[k];
    row_store<K>(y + (long long)row * K, o);
  }
};
template <int K, typename ZT, typename YT> struct MResid {  // y = z - A x
  const ZT* z; YT* y;
  __device__ void operator()(int row, int k, double v) const {
    const long long o = (long long)row * K + k;
    y[o] = (YT)((double)z[o] - v);
  }
  __device__ void row(int row, const double* v) const {
    double o[K];
    row_load<K>(z + (long long)row * K, o);
#pragma unroll
    for (int k = 0; k < K; ++k) o[k] = o[k] - v[k];
    row_store<K>(y + (long long)row * K, o);
  }
};
template <int K, typename ZT, typename YT> struct MRestrict {  // y[s] = r[s*bs+p] - (A x)[s*bs]
  const ZT* r; YT* y; int bs, p;
  __device__ void operator()(int s, int k, double v) const {
    y[(long long)s * K + k] = (YT)((double)r[((long long)s * bs + p) * K + k] - v);
  }
  __device__ void row(int s, const double* v) const {
    double o[K];
    row_load<K>(r + ((long long)s * bs + p) * K, o);
#pragma unroll
    for (int k = 0; k < K; ++k) o[k] = o[k] - v[k];
    row_store<K>(y + (long long)s * K, o);
  }
};
template <int K, typename YT> struct MProlong {  // x[s*bs+p] += (F t)[s]
  YT* x; int bs, p;
  __device__ void operator()(int s, int k, double v) const {
    const long long o = ((long long)s * bs + p) * K + k;
    x[o] = (YT)((double)x[o] + v);
  }
  __device__ void row(int s, const double* v) const {
    YT* px = x + ((long long)s * bs + p) * K;
    double o[K];
    row_load<K>(px, o);
#pragma unroll
    for (int k = 0; k < K; ++k) o[k] = o[k] + v[k];
    row_store<K>(px, o);
  }
};
// y = scale[q] * (A x) with q = system(row) * K + k: the per-instance scale of the
// lazily normalised basis column (scale[q * stride]); cell_sys maps a cell
// (bs rows) to its system
template <int K, typename YT> struct MStoreScaled {
  YT* y; const double* scale; long long stride; const int* cell_sys; int bs;
  __device__ void operator()(int row, int k, double v) const {
    const int sys = __ldg(cell_sys + row / bs);
    y[(long long)row * K + k] = (YT)(__ldg(scale + (long long)(sys * K + k) * stride) * v);
  }
  __device__ void row(int row, const double* v) const {
    const int sys = __ldg(cell_sys + row / bs);
    double o[K];
#pragma unroll
    for (int k = 0; k < K; ++k) o[k] = __ldg(scale + (long long)(sys * K + k) * stride) * v[k];
    row_store<K>(y + (long long)row * K, o);
  }
};

// K consecutive values from x + o (o a multiple of K) as doubles, with 16-byte loads
template <int K, typename XT>
__device__ __forceinline__ void load_k(const XT* __restrict__ x, long long o, double* out) {
  if constexpr (sizeof(XT) == 4 && K % 4 == 0) {
#pragma unroll
    for (int q = 0; q < K / 4; ++q) {
      const float4 t = __ldg(reinterpret_cast<const float4*>(x + o) + q);
      out[4 * q] = t.x; out[4 * q + 1] = t.y; out[4 * q + 2] = t.z; out[4 * q + 3] = t.w;
    }
  } else if constexpr (sizeof(XT) == 8 && K % 2 == 0) {
#pragma unroll
    for (int q = 0; q < K / 2; ++q) {
      const double2 t = __ldg(reinterpret_cast<const double2*>(x + o) + q);
      out[2 * q] = t.x; out[2 * q + 1] = t.y;
    }
  } else {
#pragma unroll
    for (int q = 0; q < K; ++q) out[q] = (double)__ldg(x + o + q);
  }
}

// K consecutive float32 values from x + o (o a multiple of K), as float32
template <int K>
__device__ __forceinline__ void load_k_f32(const float* __restrict__ x, long long o, float* out) {
  if constexpr (K % 4 == 0) {
#pragma unroll
    for (int q = 0; q < K / 4; ++q) {
      const float4 t = __ldg(reinterpret_cast<const float4*>(x + o) + q);
      out[4 * q] = t.x; out[4 * q + 1] = t.y; out[4 * q + 2] = t.z; out[4 * q + 3] = t.w;
    }
  } else {
#pragma unroll
    for (int q = 0; q < K; ++q) out[q] = __ldg(x + o + q);
  }
}

// Optional skip of finished systems: block row s is left out (its outputs are
// not written) when active[cell_sys[s / div]] == 0.
struct MMGate {
  const int* cell_sys = nullptr;
  const int* active = nullptr;
  int ncell = 0;  // cells of the system the map covers
  int div = 1;    // block rows per cell of the matrix at hand (set by spmm)
};

// ------------------------------------------------------------ the kernel
// Register cap: three resident blocks per SM for 1x1 and 2x2 blocks (80
// registers; the K = 8 float32 runs otherwise take 82 and fall to two blocks,
// 38 % slower), two for 3x3 blocks (whose K = 8 sums need more).
template <int SW, int BS, int K, bool ROW0, typename VT, typename XT, class Epi>
__global__ void __launch_bounds__(256, BS > 2 ? 2 : 3) bsr_mm_kernel(int nbr, const int* __restrict__ br, const int* __restrict__ bc,
                                                     const VT* __restrict__ bv, long long plane,
                                                     const XT* __restrict__ x, Epi epi, MMGate gate) {
  constexpr int NR = ROW0 ? 1 : BS;
  const int lane = threadIdx.x & (SW - 1);
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int s = int(gid / SW);
  const bool valid = s < nbr && (!gate.active || __ldg(gate.active + __ldg(gate.cell_sys + s / gate.div)) != 0);
  double acc[NR][K];
#pragma unroll
  for (int q = 0; q < NR; ++q)
#pragma unroll
    for (int k = 0; k < K; ++k) acc[q][k] = 0.0;
  if (valid) {
    const int a = __ldg(br + s), e = __ldg(br + s + 1);
    for (int blk = a + lane; blk < e; blk += SW) {
      const long long col0 = (long long)__ldcs(bc + blk) * BS;
      if constexpr (BS > 1 && kRunF32<VT, XT>) {
        // float32 runs over the BS entries of each block row (as the
        // single-vector cell-block product), accumulated in float64
        float xv[BS][K];
#pragma unroll
        for (int t = 0; t < BS; ++t) load_k_f32<K>(x, (col0 + t) * K, xv[t]);
#pragma unroll
        for (int q = 0; q < NR; ++q) {
          float w[BS];
#pragma unroll
          for (int t = 0; t < BS; ++t) w[t] = __ldcs(bv + q * plane + (long long)blk * BS + t);
#pragma unroll
          for (int k = 0; k < K; ++k) {
            float run = w[0] * xv[0][k];
#pragma unroll
            for (int t = 1; t < BS; ++t) run = fmaf(w[t], xv[t][k], run);
            acc[q][k] += (double)run;
          }
        }
      } else {
#pragma unroll
        for (int t = 0; t < BS; ++t) {
          double xv[K];
          load_k<K, XT>(x, (col0 + t) * K, xv);
#pragma unroll
          for (int q = 0; q < NR; ++q) {
            const double w = (double)__ldcs(bv + q * plane + (long long)blk * BS + t);
#pragma unroll
            for (int k = 0; k < K; ++k) acc[q][k] += w * xv[k];
          }
        }
      }
    }
  }
  if (SW > 1) {
#pragma unroll
    for (int q = 0; q < NR; ++q)
#pragma unroll
      for (int k = 0; k < K; ++k) acc[q][k] = subwarp_sum<SW>(acc[q][k]);
  }
  if (!valid) return;
#pragma unroll
  for (int q = 0; q < NR; ++q)
#pragma unroll
    for (int k = 0; k < K; ++k)
      if ((q * K + k) % SW == lane) epi(ROW0 ? s : s * BS + q, k, acc[q][k]);
}

// K-column product of a 2x2-block matrix with a slot-padded copy (see
// ell2_kernel): one thread per cell holds the cell's 2 x K sums, walks its W
// slots (column, two values per plane, the K values of the two x rows it
// multiplies) and writes its outputs; no row pointer, no sub-warp reduction.
// The block rows sum in slot order as in the single-vector padded product.
template <int W, int K, bool ROW0, typename VT, typename XT, class Epi>
__global__ void __launch_bounds__(256, 3) ell2_mm_kernel(int nbr, const int* __restrict__ ec,
                                                         const VT* __restrict__ ev, const XT* __restrict__ x, Epi epi,
                                                         MMGate gate) {
  constexpr int NR = ROW0 ? 1 : 2;
  using V2 = typename Pair<VT>::V;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nbr) return;
  if (gate.active && __ldg(gate.active + __ldg(gate.cell_sys + s / gate.div)) == 0) return;
  const V2* __restrict__ e2 = reinterpret_cast<const V2*>(ev);
  double acc[NR][K];
#pragma unroll
  for (int q = 0; q < NR; ++q)
#pragma unroll
    for (int k = 0; k < K; ++k) acc[q][k] = 0.0;
#pragma unroll 2
  for (int j = 0; j < W; ++j) {
    const long long o = (long long)__ldcs(ec + (long long)j * nbr + s) * 2 * K;  // x rows 2c, 2c+1
    const V2 a = __ldcs(e2 + (long long)j * nbr + s);
    V2 b = a;
    if (!ROW0) b = __ldcs(e2 + (long long)(W + j) * nbr + s);
    if constexpr (kRunF32<VT, XT>) {
      float x0[K], x1[K];
      load_k_f32<K>(x, o, x0);
      load_k_f32<K>(x, o + K, x1);
#pragma unroll
      for (int k = 0; k < K; ++k) {
        acc[0][k] += (double)fmaf(a.y, x1[k], a.x * x0[k]);
        if (!ROW0) acc[NR - 1][k] += (double)fmaf(b.y, x1[k], b.x * x0[k]);
      }
    } else {
      double x0[K], x1[K];
      load_k<K, XT>(x, o, x0);
      load_k<K, XT>(x, o + K, x1);
#pragma unroll
      for (int k = 0; k < K; ++k) {
        acc[0][k] += (double)a.x * x0[k];
        acc[0][k] += (double)a.y * x1[k];
        if (!ROW0) {
          acc[NR - 1][k] += (double)b.x * x0[k];
          acc[NR - 1][k] += (double)b.y * x1[k];
        }
      }
    }
  }
#pragma unroll
  for (int q = 0; q < NR; ++q) epi.row(ROW0 ? s : 2 * s + q, acc[q]);
}

// K-column product of a scalar matrix with a slot-padded copy (see ell1_kernel):
// one thread per row holds the row's K sums; float32 values times float32 x sum
// each group of four slots in float32 per column, as the single-vector kernel.
template <int W, int K, typename VT, typename XT, class Epi>
__global__ void __launch_bounds__(256, 3) ell1_mm_kernel(int n, const int* __restrict__ ec, const VT* __restrict__ ev,
                                                         const XT* __restrict__ x, Epi epi, MMGate gate) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (gate.active && __ldg(gate.active + __ldg(gate.cell_sys + i / gate.div)) == 0) return;
  double acc[K];
#pragma unroll
  for (int k = 0; k < K; ++k) acc[k] = 0.0;
#pragma unroll
  for (int g = 0; g < W; g += 4) {
    if constexpr (kRunF32<VT, XT>) {
      float run[K];
#pragma unroll
      for (int k = 0; k < K; ++k) run[k] = 0.f;
#pragma unroll
      for (int j = g; j < g + 4; ++j) {
        const long long o = (long long)__ldcs(ec + (long long)j * n + i) * K;
        const float v = __ldcs(ev + (long long)j * n + i);
        float xv[K];
        load_k_f32<K>(x, o, xv);
#pragma unroll
        for (int k = 0; k < K; ++k) run[k] = fmaf(v, xv[k], run[k]);
      }
#pragma unroll
      for (int k = 0; k < K; ++k) acc[k] += (double)run[k];
    } else {
#pragma unroll
      for (int j = g; j < g + 4; ++j) {
        const long long o = (long long)__ldcs(ec + (long long)j * n + i) * K;
        const double v = (double)__ldcs(ev + (long long)j * n + i);
        double xv[K];
        load_k<K, XT>(x, o, xv);
#pragma unroll
        for (int k = 0; k < K; ++k) acc[k] += v * xv[k];
      }
    }
  }
  epi.row(i, acc);
}

template <int K, typename VT, typename XT, class Epi>
void launch_ell1_mm(cudaStream_t st, const deco_csr_s* A, const VT* ev, const XT* x, Epi epi, MMGate gate) {
  if (A->n <= 0) return;
  const unsigned grid = (unsigned)cdiv(A->n, 256);
  if (A->ew == 4) ell1_mm_kernel<4, K, VT, XT, Epi><<<grid, 256, 0, st>>>(A->n, A->ec.get(), ev, x, epi, gate);
  else ell1_mm_kernel<8, K, VT, XT, Epi><<<grid, 256, 0, st>>>(A->n, A->ec.get(), ev, x, epi, gate);
  DECO_CHECK_LAUNCH();
}

template <int K, typename VT, typename XT, class Epi>
void launch_ell2_mm(cudaStream_t st, const deco_csr_s* A, const VT* ev, bool row0, const XT* x, Epi epi,
                    MMGate gate) {
  const int nbr = A->n / 2;
  if (nbr <= 0) return;
  const unsigned grid = (unsigned)cdiv(nbr, 256);
  if (A->ew == 4) {
    if (row0) ell2_mm_kernel<4, K, true, VT, XT, Epi><<<grid, 256, 0, st>>>(nbr, A->ec.get(), ev, x, epi, gate);
    else ell2_mm_kernel<4, K, false, VT, XT, Epi><<<grid, 256, 0, st>>>(nbr, A->ec.get(), ev, x, epi, gate);
  } else if (A->ew == 7) {
    if (row0) ell2_mm_kernel<7, K, true, VT, XT, Epi><<<grid, 256, 0, st>>>(nbr, A->ec.get(), ev, x, epi, gate);
    else ell2_mm_kernel<7, K, false, VT, XT, Epi><<<grid, 256, 0, st>>>(nbr, A->ec.get(), ev, x, epi, gate);
  } else {
    if (row0) ell2_mm_kernel<8, K, true, VT, XT, Epi><<<grid, 256, 0, st>>>(nbr, A->ec.get(), ev, x, epi, gate);
    else ell2_mm_kernel<8, K, false, VT, XT, Epi><<<grid, 256, 0, st>>>(nbr, A->ec.get(), ev, x, epi, gate);
  }
  DECO_CHECK_LAUNCH();
}

// A matrix for the K-column product: its cell-block copy when it has one
// (BS = bbs), else the CSR arrays as BS = 1 blocks.
struct MMView {
  int bs, nbr;
  const int* br;
  const int* bc;
  long long plane;
  const double* v64;
  const float* v32;
  int sw;
};

inline MMView mm_view(const deco_csr_s* A) {
  MMView m{};
  if (A->bbs > 1) {
    m.bs = A->bbs; m.nbr = A->n / A->bbs; m.br = A->br.get(); m.bc = A->bc.get();
    m.plane = A->bplane; m.v64 = A->bv.get(); m.v32 = A->bv32.get();
    m.sw = 1;
    while (m.sw < 16 && m.sw < A->avg_blk / 2.0) m.sw <<= 1;
  } else {
    m.bs = 1; m.nbr = A->n; m.br = A->r.get(); m.bc = A->c.get(); m.plane = A->nz;
    m.v64 = A->v.get(); m.v32 = A->v32.get();
    m.sw = 1;
    while (m.sw < 16 && m.sw < A->avg_row / 2.0) m.sw <<= 1;
  }
  return m;
}

template <int SW, int BS, int K, bool ROW0, typename VT, typename XT, class Epi>
void launch_mm_sw(cudaStream_t st, const MMView& M, const VT* v, const XT* x, Epi epi, MMGate gate) {
  const unsigned grid = (unsigned)cdiv((long long)M.nbr * SW, 256);
  bsr_mm_kernel<SW, BS, K, ROW0, VT, XT, Epi><<<grid, 256, 0, st>>>(M.nbr, M.br, M.bc, v, M.plane, x, epi, gate);
  DECO_CHECK_LAUNCH();
}

template <int BS, int K, bool ROW0, typename VT, typename XT, class Epi>
void launch_mm_bs(cudaStream_t st, const MMView& M, const VT* v, const XT* x, Epi epi, MMGate gate) {
  switch (M.sw) {
    case 1: launch_mm_sw<1, BS, K, ROW0>(st, M, v, x, epi, gate); break;
    case 2: launch_mm_sw<2, BS, K, ROW0>(st, M, v, x, epi, gate); break;
    case 4: launch_mm_sw<4, BS, K, ROW0>(st, M, v, x, epi, gate); break;
    case 8: launch_mm_sw<8, BS, K, ROW0>(st, M, v, x, epi, gate); break;
    default: launch_mm_sw<16, BS, K, ROW0>(st, M, v, x, epi, gate); break;
  }
}

// Y = op(A X) with K columns; row0: the restricted product over row 0 of every
// cell of size `bs` (A must then have a cell-block copy of that size, or bs = 1).
template <int K, typename VT, typename XT, class Epi>
void spmm(deco_ctx_s* ctx, const deco_csr_s* A, const XT* x, Epi epi, bool row0 = false, MMGate gate = MMGate{},
          int sw = 0) {
  MMView M = mm_view(A);
  if (sw) M.sw = sw;
  const VT* v;
  if constexpr (sizeof(VT) == 4) v = M.v32; else v = M.v64;
  DECO_REQUIRE(v != nullptr, DECO_ERR_INTERNAL, "matrix values of the requested precision are missing");
  DECO_REQUIRE(!row0 || M.bs > 1, DECO_ERR_INTERNAL, "restricted K-column product needs a cell-block copy");
  if (gate.active) {  // block rows per cell: 1 for cell blocks and the pressure system, bs for scalar rows
    if (gate.ncell > 0 && M.nbr % gate.ncell == 0) gate.div = M.nbr / gate.ncell;
    else gate = MMGate{};
  }
  cudaStream_t st = ctx->stream;
  if (A->ew && !A->nov && (M.bs == 2 || (M.bs == 1 && !A->bbs && !row0))) {  // (no overflow lists here)
    const VT* ev;
    if constexpr (sizeof(VT) == 4) ev = A->ev32.get(); else ev = A->ev.get();
    if (ev) {
      if (M.bs == 2) launch_ell2_mm<K, VT, XT, Epi>(st, A, ev, row0, x, epi, gate);
      else launch_ell1_mm<K, VT, XT, Epi>(st, A, ev, x, epi, gate);
      return;
    }
  }
  if (M.bs == 1) launch_mm_bs<1, K, false, VT, XT, Epi>(st, M, v, x, epi, gate);
  else if (M.bs == 2) {
    if (row0) launch_mm_bs<2, K, true, VT, XT, Epi>(st, M, v, x, epi, gate);
    else launch_mm_bs<2, K, false, VT, XT, Epi>(st, M, v, x, epi, gate);
  } else {
    if (row0) launch_mm_bs<3, K, true, VT, XT, Epi>(st, M, v, x, epi, gate);
    else launch_mm_bs<3, K, false, VT, XT, Epi>(st, M, v, x, epi, gate);
  }
}

}  // namespace deco
