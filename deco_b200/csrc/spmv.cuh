// spmv.cuh — CSR sparse matrix-vector product for sm_100a, and the device
// CSR handle.
//
// Algorithm (the reference's alg::spmv, core/alg.hpp:50-64, computes the same
// sums row by row in column order):
//   * a sub-warp of SW lanes (1..32, chosen per matrix by the autotuner) owns a
//     row; lanes stride over the row with 128-bit loads of values (double2 /
//     float4) and the matching 64/128-bit loads of column indices, starting
//     from the row start rounded down to the vector width and masking entries
//     outside the row, so every load is aligned and coalesced across the
//     sub-warps of a warp;
//   * values and columns stream through with evict-first loads, x is read
//     through the read-only path (L1/L2 keep the 7-point stencil's x tiles);
//   * sums accumulate in float64 (float32 values times float32 x: short runs
//     of products summed in float32 first) and are reduced with warp shuffles;
//   * the epilogue fuses the vector operation that follows the product in the
//     CPR and GMRES sequences (store, accumulate, residual, pressure
//     restriction, pressure prolongation), so those never cost a pass of
//     their own.
#pragma once
#include <type_traits>

#include "common.cuh"

struct deco_csr_s {
  int n = 0, m = 0, nz = 0;
  deco::DevBuf<int> r, c;
  deco::DevBuf<double> v;
  deco::DevBuf<float> v32;
  int sw64 = 0, sw32 = 0;   // sub-warp width per value precision (0 = not chosen yet)
  int max_row = 0;
  double avg_row = 0;
  // Cell-block copy for matrices of bs x bs cell blocks (reservoir systems):
  // one column index per block instead of per entry, entries the CSR pattern
  // lacks stored as zeros, and the values kept as bs row planes (plane q holds
  // in-block row q of every block) so a product over row 0 of each cell reads
  // one plane only.  bbs == 0: no block copy.
  int bbs = 0, nblk = 0;
  long long bplane = 0;       // plane stride in values: nblk * bbs rounded up to 4 (16-byte aligned planes)
  deco::DevBuf<int> br, bc;   // block-row pointers (n / bbs + 1), block columns
  deco::DevBuf<double> bv;    // bbs planes of bplane values
  deco::DevBuf<float> bv32;
  int bsw64 = 0, bsw32 = 0;
  double avg_blk = 0;
  // Slot-padded copy (bbs == 2 or 3: of the cell blocks; bbs == 0: of the scalar
  // rows, ec[k * n + i] / ev[k * n + i] holding row i's entry k).  ew = 4, 7 or 8
  // slots per cell (4 or 8 per scalar row; 0: none), slot-major (slot k of all
  // cells contiguous), unused slots repeating one of the cell's columns (or
  // column 0) with zero values.  2x2 cells (at most ew blocks each):
  // ec[k * ncell + s] is the block column, value plane q (in-block row q), slot k
  // the block row's two values at pair index (q * ew + k) * ncell + s.
  int ew = 0;
  deco::DevBuf<int> ec;
  deco::DevBuf<double> ev;
  deco::DevBuf<float> ev32;
  // 3x3 cell blocks (bbs == 3): ew slots per cell hold the cell's first blocks;
  // a cell with more than ew blocks keeps ew - 1 in slots and marks the last
  // slot with column -1, whose value planes 0 and 1 carry (as int bits) the
  // start and count of its remaining blocks in the overflow list (oc: block
  // columns; ov / ov32: the 9 values of each block, row-major).  Value plane
  // 3 q + t of slot k (in-block row q, column t): ev[((3 q + t) ew + k) ncell + s].
  int nov = 0;
  deco::DevBuf<int> eo;  // per cell: start of its overflow blocks (the float32 refill reuses it)
  deco::DevBuf<int> oc;
  deco::DevBuf<double> ov;
  deco::DevBuf<float> ov32;
  // Offset-coded slot columns: when the slots' column offsets (block column
  // minus the cell's own index, or column minus the row for scalar rows) take at
  // most 256 (eb = 1) or 65536 (eb = 2) distinct values, eoff holds them sorted
  // and ecode[k * nrow + s] (eb bytes each) the position of slot k's offset, so
  // the products read 1 or 2 bytes per slot instead of a 4-byte column.  eb = 0:
  // the products read ec.
  int eb = 0, noff = 0;
  deco::DevBuf<unsigned char> ecode;
  deco::DevBuf<int> eoff;
  // The product the autotuner chose per value precision (tune_product_plan):
  // 0 = not chosen (the layout rules: slot-padded copy, else cell blocks, else
  // CSR), 1 = slot-padded copy, 2 = cell-block kernel, 3 = CSR kernel.
  int plan64 = 0, plan32 = 0;
};

namespace deco {

template <typename VT> struct Vec;
template <> struct Vec<double> { using V = double2; using I = int2; static constexpr int W = 2; };
template <> struct Vec<float> { using V = float4; using I = int4; static constexpr int W = 4; };

__device__ __forceinline__ double2 ld_stream(const double2* p) { return __ldcs(p); }
__device__ __forceinline__ float4 ld_stream(const float4* p) { return __ldcs(p); }
__device__ __forceinline__ int2 ld_stream(const int2* p) { return __ldcs(p); }
__device__ __forceinline__ int4 ld_stream(const int4* p) { return __ldcs(p); }

__device__ __forceinline__ double elem(const double2& v, int q) { return q == 0 ? v.x : v.y; }
__device__ __forceinline__ double elem(const float4& v, int q) {
  return q == 0 ? v.x : (q == 1 ? v.y : (q == 2 ? v.z : v.w));
}
__device__ __forceinline__ int elem(const int2& v, int q) { return q == 0 ? v.x : v.y; }
__device__ __forceinline__ int elem(const int4& v, int q) {
  return q == 0 ? v.x : (q == 1 ? v.y : (q == 2 ? v.z : v.w));
}

// Float32 values times float32 x: the products of one short run (the entries of
// one 128-bit value load in CSR, one row of one cell block) are summed in float32
// and converted once; the runs accumulate in float64.  On B200 a float32 ->
// float64 conversion issues at about 16 per clock per SM, a quarter of the float64
// FMA rate, and widening every operand (six conversions per 2x2 block) bounded the
// float32 product below the HBM roofline: 145 us against 135 us for the 8M-row
// 2x2-block matrix (67 % against 71 % of the copy bandwidth).  Summing whole rows
// in float32 (129 us) moved the mixed-precision iteration counts.
template <typename VT, typename XT>
constexpr bool kRunF32 = std::is_same<VT, float>::value && std::is_same<XT, float>::value;

// ----------------------------------------------------------------- epilogues
template <typename YT> struct EpiStore {
  YT* y;
  __device__ void operator()(int o, double s) const { y[o] = (YT)s; }
};
template <typename YT> struct EpiAdd {
  YT* y;
  __device__ void operator()(int o, double s) const { y[o] = (YT)((double)y[o] + s); }
};
template <typename YT> struct EpiStoreScaled {  // y = s * (A x), s read from device memory
  YT* y; const double* s;
  __device__ void operator()(int o, double v) const { y[o] = (YT)(__ldg(s) * v); }
};
template <typename ZT, typename YT> struct EpiResid {  // y = z - A x
  const ZT* z; YT* y;
  __device__ void operator()(int o, double s) const { y[o] = (YT)((double)z[o] - s); }
};
template <typename ZT, typename YT> struct EpiRestrict {  // y[s] = r[s*bs+p] - (A x)[s*bs]
  const ZT* r; YT* y; int bs, p;
  __device__ void operator()(int o, double s) const { y[o] = (YT)((double)r[(long long)o * bs + p] - s); }
};
template <typename YT> struct EpiProlong {  // x[s*bs+p] += (F t)[s]
  YT* x; int bs, p;
  __device__ void operator()(int o, double s) const {
    long long i = (long long)o * bs + p;
    x[i] = (YT)((double)x[i] + s);
  }
};

// ---------------------------------------------------------------- the kernel
template <int SW, typename VT, typename XT, class Epi>
__global__ void __launch_bounds__(256) spmv_kernel(int nrows_out, int row_stride, const int* __restrict__ rp,
                                                   const int* __restrict__ ci, const VT* __restrict__ vv,
                                                   const XT* __restrict__ x, Epi epi) {
  using VV = typename Vec<VT>::V;
  using VI = typename Vec<VT>::I;
  constexpr int W = Vec<VT>::W;
  pdl_wait();
  pdl_trigger();
  const int lane = threadIdx.x & (SW - 1);
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int orow = int(gid / SW);
  const bool valid = orow < nrows_out;
  double sum = 0.0;
  if (valid) {
    const long long row = (long long)orow * row_stride;
    const int a = __ldg(rp + row), e = __ldg(rp + row + 1);
    for (int k = (a & ~(W - 1)) + lane * W; k < e; k += SW * W) {
      const VV v4 = ld_stream(reinterpret_cast<const VV*>(vv + k));
      const VI c4 = ld_stream(reinterpret_cast<const VI*>(ci + k));
      const VT* vs = reinterpret_cast<const VT*>(&v4);
      if constexpr (kRunF32<VT, XT>) {
        float run = 0.f;
#pragma unroll
        for (int q = 0; q < W; ++q) {
          const int idx = k + q;
          if (idx >= a && idx < e) run = fmaf(vs[q], __ldg(x + elem(c4, q)), run);
        }
        sum += (double)run;
      } else {
#pragma unroll
        for (int q = 0; q < W; ++q) {
          const int idx = k + q;
          if (idx >= a && idx < e) sum += (double)vs[q] * (double)__ldg(x + elem(c4, q));
        }
      }
    }
  }
  if (SW > 1) sum = subwarp_sum<SW>(sum);
  if (valid && lane == 0) epi(orow, sum);
}

template <typename VT, typename XT, class Epi>
void launch_spmv_sw(cudaStream_t st, int sw, int nrows_out, int row_stride, const int* r, const int* c,
                    const VT* v, const XT* x, Epi epi) {
  if (nrows_out <= 0) return;
  const int block = 256;
  const long long threads = (long long)nrows_out * sw;
  const unsigned grid = (unsigned)cdiv(threads, block);
  switch (sw) {
    case 1: launch_k(spmv_kernel<1, VT, XT, Epi>, grid, block, 0, st, nrows_out, row_stride, r, c, v, x, epi); break;
    case 2: launch_k(spmv_kernel<2, VT, XT, Epi>, grid, block, 0, st, nrows_out, row_stride, r, c, v, x, epi); break;
    case 4: launch_k(spmv_kernel<4, VT, XT, Epi>, grid, block, 0, st, nrows_out, row_stride, r, c, v, x, epi); break;
    case 8: launch_k(spmv_kernel<8, VT, XT, Epi>, grid, block, 0, st, nrows_out, row_stride, r, c, v, x, epi); break;
    case 16: launch_k(spmv_kernel<16, VT, XT, Epi>, grid, block, 0, st, nrows_out, row_stride, r, c, v, x, epi); break;
    default: launch_k(spmv_kernel<32, VT, XT, Epi>, grid, block, 0, st, nrows_out, row_stride, r, c, v, x, epi); break;
  }
  DECO_CHECK_LAUNCH();
}

// ------------------------------------------------------- cell-block kernel
// A sub-warp of SW lanes owns a block row (one cell: BS matrix rows); each lane
// takes whole blocks: one 4-byte block column, the BS x values of that cell (a
// single 8/16-byte pair load for BS == 2) and BS values per computed row.  ROW0
// computes only in-block row 0 of every cell (the restricted product of
// alg::spmv with bs > 1) and reads only that value plane.
template <typename T> struct Pair;
template <> struct Pair<double> { using V = double2; };
template <> struct Pair<float> { using V = float2; };

template <int SW, int BS, bool ROW0, typename VT, typename XT, class Epi>
__global__ void __launch_bounds__(256) bsr_kernel(int nbr, const int* __restrict__ br, const int* __restrict__ bc,
                                                  const VT* __restrict__ bv, long long plane,
                                                  const XT* __restrict__ x, Epi epi) {
  constexpr int NR = ROW0 ? 1 : BS;
  pdl_wait();
  pdl_trigger();
  const int lane = threadIdx.x & (SW - 1);
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int s = int(gid / SW);
  const bool valid = s < nbr;
  double sum[NR];
#pragma unroll
  for (int q = 0; q < NR; ++q) sum[q] = 0.0;
  using XA = typename std::conditional<kRunF32<VT, XT>, float, double>::type;  // x and run type
  if (valid) {
    const int a = __ldg(br + s), e = __ldg(br + s + 1);
    for (int k = a + lane; k < e; k += SW) {
      const long long j = (long long)__ldcs(bc + k) * BS;
      XA xv[BS];
      if constexpr (BS == 2) {
        const typename Pair<XT>::V p = __ldg(reinterpret_cast<const typename Pair<XT>::V*>(x + j));
        xv[0] = (XA)p.x;
        xv[1] = (XA)p.y;
      } else {
#pragma unroll
        for (int t = 0; t < BS; ++t) xv[t] = (XA)__ldg(x + j + t);
      }
#pragma unroll
      for (int q = 0; q < NR; ++q) {
        const VT* vp = bv + q * plane + (long long)k * BS;
        XA wv[BS];
        if constexpr (BS == 2) {
          const typename Pair<VT>::V w = __ldcs(reinterpret_cast<const typename Pair<VT>::V*>(vp));
          wv[0] = (XA)w.x;
          wv[1] = (XA)w.y;
        } else {
#pragma unroll
          for (int t = 0; t < BS; ++t) wv[t] = (XA)__ldcs(vp + t);
        }
        if constexpr (kRunF32<VT, XT>) {
          float run = wv[0] * xv[0];
#pragma unroll
          for (int t = 1; t < BS; ++t) run = fmaf(wv[t], xv[t], run);
          sum[q] += (double)run;
        } else {
#pragma unroll
          for (int t = 0; t < BS; ++t) sum[q] += wv[t] * xv[t];
        }
      }
    }
  }
  if (SW > 1) {
#pragma unroll
    for (int q = 0; q < NR; ++q) sum[q] = subwarp_sum<SW>(sum[q]);
  }
  if (valid && lane == 0) {
    if (ROW0) {
      epi(s, sum[0]);
    } else {
#pragma unroll
      for (int q = 0; q < NR; ++q) epi(s * BS + q, sum[q]);
    }
  }
}

// 2 x 2 cells: each lane takes a PAIR of consecutive blocks per step, from the
// pair-aligned start of the block row, with one 8-byte load of their two columns
// and one 16-byte (float) or two 16-byte (double) loads of their values per
// plane; blocks outside the row are masked (their loads stay inside the padded
// arrays: the planes are 16-byte aligned and the index array has slack).
// One pair of blocks as loaded: their two columns and the values of both planes.
template <typename VT> struct PairLoad;
template <> struct PairLoad<float> {
  int2 c;
  float4 w0, w1;
  template <bool ROW0>
  __device__ void load(const int* bc, const float* bv, long long plane, int k) {
    c = __ldcs(reinterpret_cast<const int2*>(bc + k));
    w0 = __ldcs(reinterpret_cast<const float4*>(bv + 2LL * k));
    if (!ROW0) w1 = __ldcs(reinterpret_cast<const float4*>(bv + plane + 2LL * k));
  }
};
template <> struct PairLoad<double> {
  int2 c;
  double2 w0a, w0b, w1a, w1b;
  template <bool ROW0>
  __device__ void load(const int* bc, const double* bv, long long plane, int k) {
    c = __ldcs(reinterpret_cast<const int2*>(bc + k));
    w0a = __ldcs(reinterpret_cast<const double2*>(bv + 2LL * k));
    w0b = __ldcs(reinterpret_cast<const double2*>(bv + 2LL * k) + 1);
    if (!ROW0) {
      w1a = __ldcs(reinterpret_cast<const double2*>(bv + plane + 2LL * k));
      w1b = __ldcs(reinterpret_cast<const double2*>(bv + plane + 2LL * k) + 1);
    }
  }
};

// Adds block h (0 or 1) of a loaded pair times x to the two row sums.
template <bool ROW0, typename VT, typename XT>
__device__ __forceinline__ void pair_accumulate(const PairLoad<VT>& L, int h, const XT* __restrict__ x, double& s0,
                                                double& s1) {
  const int col = h == 0 ? L.c.x : L.c.y;
  const typename Pair<XT>::V p = __ldg(reinterpret_cast<const typename Pair<XT>::V*>(x + 2LL * col));
  if constexpr (kRunF32<VT, XT>) {
    const float a0 = h == 0 ? L.w0.x : L.w0.z, a1 = h == 0 ? L.w0.y : L.w0.w;
    s0 += (double)fmaf(a1, p.y, a0 * p.x);
    if (!ROW0) {
      const float b0 = h == 0 ? L.w1.x : L.w1.z, b1 = h == 0 ? L.w1.y : L.w1.w;
      s1 += (double)fmaf(b1, p.y, b0 * p.x);
    }
  } else if constexpr (std::is_same<VT, float>::value) {
    const float a0 = h == 0 ? L.w0.x : L.w0.z, a1 = h == 0 ? L.w0.y : L.w0.w;
    s0 += (double)a0 * (double)p.x;
    s0 += (double)a1 * (double)p.y;
    if (!ROW0) {
      const float b0 = h == 0 ? L.w1.x : L.w1.z, b1 = h == 0 ? L.w1.y : L.w1.w;
      s1 += (double)b0 * (double)p.x;
      s1 += (double)b1 * (double)p.y;
    }
  } else {
    const double2 a = h == 0 ? L.w0a : L.w0b;
    s0 += a.x * (double)p.x;
    s0 += a.y * (double)p.y;
    if (!ROW0) {
      const double2 b = h == 0 ? L.w1a : L.w1b;
      s1 += b.x * (double)p.x;
      s1 += b.y * (double)p.y;
    }
  }
}

// Each lane handles two pairs per loop step (k and k + 2 SW): both pairs' index
// and value loads are issued before either pair's x gathers, so a lane keeps
// twice the bytes in flight through the index -> x dependence.  The sums run in
// the same order as a one-pair-per-step loop.  (Measured on B200, float32 values,
// L2 flushed: 8M-row system matrix 135 -> 127 us, its lower FSAI factor with four
// blocks per cell 90 -> 86 us.)
template <int SW, bool ROW0, typename VT, typename XT, class Epi>
__global__ void __launch_bounds__(256) bsr2_pair_kernel(int nbr, const int* __restrict__ br, const int* __restrict__ bc,
                                                        const VT* __restrict__ bv, long long plane,
                                                        const XT* __restrict__ x, Epi epi) {
  pdl_wait();
  pdl_trigger();
  const int lane = threadIdx.x & (SW - 1);
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int s = int(gid / SW);
  const bool valid = s < nbr;
  double s0 = 0.0, s1 = 0.0;
  if (valid) {
    const int a = __ldg(br + s), e = __ldg(br + s + 1);
    for (int k = (a & ~1) + 2 * lane; k < e; k += 4 * SW) {
      const int kb = k + 2 * SW;
      PairLoad<VT> P, Q;
      P.template load<ROW0>(bc, bv, plane, k);
      if (kb < e) Q.template load<ROW0>(bc, bv, plane, kb);
      if (k >= a) pair_accumulate<ROW0, VT, XT>(P, 0, x, s0, s1);
      if (k + 1 < e) pair_accumulate<ROW0, VT, XT>(P, 1, x, s0, s1);
      if (kb < e) {
        pair_accumulate<ROW0, VT, XT>(Q, 0, x, s0, s1);
        if (kb + 1 < e) pair_accumulate<ROW0, VT, XT>(Q, 1, x, s0, s1);
      }
    }
  }
  if (SW > 1) {
    s0 = subwarp_sum<SW>(s0);
    if (!ROW0) s1 = subwarp_sum<SW>(s1);
  }
  if (valid && lane == 0) {
    if (ROW0) {
      epi(s, s0);
    } else {
      epi(2 * s, s0);
      epi(2 * s + 1, s1);
    }
  }
}

// Slot-padded 2x2 product: one thread per cell, W independent slots, every load
// a coalesced 8- or 16-byte load of a slot-major array and no row pointer in the
// dependence chain (column and values -> x gather -> sum).  The block rows sum in
// slot order, i.e. the cell's block order.  (Measured on B200 for the lower FSAI
// factor of the 8M-row system, four blocks per cell, L2 flushed: 65 us float32 and
// 111 us float64, against 89 us and 152 us with the pair kernel.)
// Column of slot entry idx of the padded copy whose own row (or cell) is `base`:
// the stored column (EB = 0), or base + the offset the 1- or 2-byte code selects.
template <int EB>
__device__ __forceinline__ int slot_col(const int* __restrict__ ec, const unsigned char* __restrict__ code,
                                        const int* __restrict__ off, long long idx, int base) {
  if constexpr (EB == 0) return __ldcs(ec + idx);
  else if constexpr (EB == 1) return base + __ldg(off + __ldcs(code + idx));
  else return base + __ldg(off + __ldcs(reinterpret_cast<const unsigned short*>(code) + idx));
}

template <int W, bool ROW0, typename VT, typename XT, class Epi, int EB = 0>
__global__ void __launch_bounds__(256) ell2_kernel(int nbr, const int* __restrict__ ec, const VT* __restrict__ ev,
                                                   const XT* __restrict__ x, Epi epi,
                                                   const unsigned char* __restrict__ code = nullptr,
                                                   const int* __restrict__ off = nullptr) {
  using V2 = typename Pair<VT>::V;
  using X2 = typename Pair<XT>::V;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nbr) return;
  const V2* __restrict__ e2 = reinterpret_cast<const V2*>(ev);
  int cc[W];
  V2 a[W], b[W];
#pragma unroll
  for (int k = 0; k < W; ++k) {
    cc[k] = slot_col<EB>(ec, code, off, (long long)k * nbr + s, s);
    a[k] = __ldcs(e2 + (long long)k * nbr + s);
    if (!ROW0) b[k] = __ldcs(e2 + (long long)(W + k) * nbr + s);
  }
  // the matrix slots above are constant during a solve; x and the epilogue's
  // vectors may be the predecessor's output
  pdl_wait();
  pdl_trigger();
  double s0 = 0.0, s1 = 0.0;
#pragma unroll
  for (int k = 0; k < W; ++k) {
    const X2 p = __ldg(reinterpret_cast<const X2*>(x) + cc[k]);
    if constexpr (kRunF32<VT, XT>) {
      s0 += (double)fmaf(a[k].y, p.y, a[k].x * p.x);
      if (!ROW0) s1 += (double)fmaf(b[k].y, p.y, b[k].x * p.x);
    } else {
      s0 += (double)a[k].x * (double)p.x;
      s0 += (double)a[k].y * (double)p.y;
      if (!ROW0) {
        s1 += (double)b[k].x * (double)p.x;
        s1 += (double)b[k].y * (double)p.y;
      }
    }
  }
  if (ROW0) {
    epi(s, s0);
  } else {
    epi(2 * s, s0);
    epi(2 * s + 1, s1);
  }
}

// Slot-padded 3x3 product: one thread per cell, W slots, every value load a
// coalesced 4- or 8-byte load of one of the 9 (3 for ROW0) slot-major value
// planes; the block rows sum in slot order, which is the cell's block order
// (as the cell-block kernel with one lane per cell sums them).  A slot with
// column -1 (only the last) sends the thread to the cell's overflow blocks.
template <typename VT> __device__ __forceinline__ int slot_bits(VT v);
template <> __device__ __forceinline__ int slot_bits<double>(double v) { return (int)__double_as_longlong(v); }
template <> __device__ __forceinline__ int slot_bits<float>(float v) { return __float_as_int(v); }

template <bool ROW0, typename VT, typename XT>
__device__ __forceinline__ void block3_accumulate(const VT (&w)[9], const XT* __restrict__ x, int col, double* sum) {
  constexpr int NR = ROW0 ? 1 : 3;
  using XA = typename std::conditional<kRunF32<VT, XT>, float, double>::type;
  const long long j = 3LL * col;
  XA xv[3];
#pragma unroll
  for (int t = 0; t < 3; ++t) xv[t] = (XA)__ldg(x + j + t);
#pragma unroll
  for (int q = 0; q < NR; ++q) {
    if constexpr (kRunF32<VT, XT>) {
      float run = w[3 * q] * xv[0];
      run = fmaf(w[3 * q + 1], xv[1], run);
      run = fmaf(w[3 * q + 2], xv[2], run);
      sum[q] += (double)run;
    } else {
#pragma unroll
      for (int t = 0; t < 3; ++t) sum[q] += (XA)w[3 * q + t] * xv[t];
    }
  }
}

template <int W, bool ROW0, typename VT, typename XT, class Epi>
__global__ void __launch_bounds__(256) ell3_kernel(int nbr, const int* __restrict__ ec, const VT* __restrict__ ev,
                                                   const int* __restrict__ oc, const VT* __restrict__ ov,
                                                   const XT* __restrict__ x, Epi epi) {
  constexpr int NR = ROW0 ? 1 : 3;
  // float32 values: every slot's values are loaded up front (W x 3 NR registers),
  // so a thread has all its matrix bytes in flight at once; float64 values are
  // loaded slot by slot
  constexpr bool kAll = sizeof(VT) == 4;
  constexpr int WP = kAll ? W : 1;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nbr) return;
  int cc[W];
  VT wa[WP][3 * NR];
#pragma unroll
  for (int k = 0; k < W; ++k) {
    cc[k] = __ldcs(ec + (long long)k * nbr + s);
    if constexpr (kAll) {
#pragma unroll
      for (int p = 0; p < 3 * NR; ++p) wa[k][p] = __ldcs(ev + ((long long)p * W + k) * nbr + s);
    }
  }
  // the slots above are constant during a solve; x and the epilogue's vectors
  // may be the predecessor's output
  pdl_wait();
  pdl_trigger();
  double sum[NR];
#pragma unroll
  for (int q = 0; q < NR; ++q) sum[q] = 0.0;
#pragma unroll
  for (int k = 0; k < W; ++k) {
    VT w[9];
#pragma unroll
    for (int p = 0; p < 3 * NR; ++p) {
      if constexpr (kAll) w[p] = wa[k][p];
      else w[p] = __ldcs(ev + ((long long)p * W + k) * nbr + s);
    }
    if (k == W - 1 && cc[k] < 0) {  // the cell's remaining blocks, from the overflow list
      const int o0 = slot_bits<VT>(w[0]), no = slot_bits<VT>(w[1]);
      for (int o = o0; o < o0 + no; ++o) {
        VT u[9];
#pragma unroll
        for (int p = 0; p < 9; ++p) u[p] = ov[9LL * o + p];
        block3_accumulate<ROW0, VT, XT>(u, x, oc[o], sum);
      }
    } else {
      block3_accumulate<ROW0, VT, XT>(w, x, cc[k], sum);
    }
  }
  if (ROW0) {
    epi(s, sum[0]);
  } else {
#pragma unroll
    for (int q = 0; q < NR; ++q) epi(3 * s + q, sum[q]);
  }
}

// Slot-padded scalar product (a CSR matrix with at most W entries per row: the
// FSAI factors of a pressure system): one thread per row, slot-major coalesced
// loads.  Float32 values times float32 x: each group of four slots is summed in
// float32 and converted once, as the CSR kernel sums one 128-bit value load.
template <int W, typename VT, typename XT, class Epi, int EB = 0>
__global__ void __launch_bounds__(256) ell1_kernel(int n, const int* __restrict__ ec, const VT* __restrict__ ev,
                                                   const XT* __restrict__ x, Epi epi,
                                                   const unsigned char* __restrict__ code = nullptr,
                                                   const int* __restrict__ off = nullptr,
                                                   const int* __restrict__ eo = nullptr,
                                                   const int* __restrict__ oc = nullptr,
                                                   const VT* __restrict__ ov = nullptr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int cc[W];
  VT vv[W];
#pragma unroll
  for (int k = 0; k < W; ++k) {
    cc[k] = slot_col<EB>(ec, code, off, (long long)k * n + i, i);
    vv[k] = __ldcs(ev + (long long)k * n + i);
  }
  pdl_wait();
  pdl_trigger();
  // a row longer than the slots marks its last slot with column -1 (value 0) and
  // keeps the rest of its entries in the overflow list, added after the slots
  const bool over = EB == 0 && cc[W - 1] < 0;
  if (over) cc[W - 1] = 0;
  double sum = 0.0;
  if constexpr (kRunF32<VT, XT>) {
#pragma unroll
    for (int g = 0; g < W; g += 4) {
      float run = 0.f;
#pragma unroll
      for (int k = g; k < g + 4; ++k) run = fmaf(vv[k], __ldg(x + cc[k]), run);
      sum += (double)run;
    }
  } else {
#pragma unroll
    for (int k = 0; k < W; ++k) sum += (double)vv[k] * (double)__ldg(x + cc[k]);
  }
  if (over) {
    const int o0 = eo[i], o1 = eo[i + 1];
    for (int o = o0; o < o1; ++o) {
      if constexpr (kRunF32<VT, XT>) sum += (double)(ov[o] * __ldg(x + oc[o]));
      else sum += (double)ov[o] * (double)__ldg(x + oc[o]);
    }
  }
  epi(i, sum);
}

template <typename VT, typename XT, class Epi>
void launch_ell1(cudaStream_t st, const deco_csr_s* A, const XT* x, Epi epi) {
  if (A->n <= 0) return;
  const VT* ev;
  const VT* ov;
  if constexpr (sizeof(VT) == 4) { ev = A->ev32.get(); ov = A->ov32.get(); } else { ev = A->ev.get(); ov = A->ov.get(); }
  const unsigned grid = (unsigned)cdiv(A->n, 256);
  const unsigned char* cd = A->ecode.get();
  const int* of = A->eoff.get();
  auto go = [&](auto eb) {
    constexpr int EB = decltype(eb)::value;
    if (A->ew == 4)
      launch_k(ell1_kernel<4, VT, XT, Epi, EB>, grid, 256, 0, st, A->n, A->ec.get(), ev, x, epi, cd, of, A->eo.get(),
               A->oc.get(), ov);
    else
      launch_k(ell1_kernel<8, VT, XT, Epi, EB>, grid, 256, 0, st, A->n, A->ec.get(), ev, x, epi, cd, of, A->eo.get(),
               A->oc.get(), ov);
  };
  if (A->eb == 1) go(std::integral_constant<int, 1>{});
  else if (A->eb == 2) go(std::integral_constant<int, 2>{});
  else go(std::integral_constant<int, 0>{});
  DECO_CHECK_LAUNCH();
}

template <typename VT, typename XT, class Epi>
void launch_ell2(cudaStream_t st, const deco_csr_s* A, bool row0, const XT* x, Epi epi) {
  const int nbr = A->n / 2;
  if (nbr <= 0) return;
  const VT* ev;
  if constexpr (sizeof(VT) == 4) ev = A->ev32.get(); else ev = A->ev.get();
  const unsigned grid = (unsigned)cdiv(nbr, 256);
  const unsigned char* cd = A->ecode.get();
  const int* of = A->eoff.get();
  auto go = [&](auto eb) {
    constexpr int EB = decltype(eb)::value;
    if (A->ew == 4) {
      if (row0) launch_k(ell2_kernel<4, true, VT, XT, Epi, EB>, grid, 256, 0, st, nbr, A->ec.get(), ev, x, epi, cd, of);
      else launch_k(ell2_kernel<4, false, VT, XT, Epi, EB>, grid, 256, 0, st, nbr, A->ec.get(), ev, x, epi, cd, of);
    } else if (A->ew == 7) {
      if (row0) launch_k(ell2_kernel<7, true, VT, XT, Epi, EB>, grid, 256, 0, st, nbr, A->ec.get(), ev, x, epi, cd, of);
      else launch_k(ell2_kernel<7, false, VT, XT, Epi, EB>, grid, 256, 0, st, nbr, A->ec.get(), ev, x, epi, cd, of);
    } else {
      if (row0) launch_k(ell2_kernel<8, true, VT, XT, Epi, EB>, grid, 256, 0, st, nbr, A->ec.get(), ev, x, epi, cd, of);
      else launch_k(ell2_kernel<8, false, VT, XT, Epi, EB>, grid, 256, 0, st, nbr, A->ec.get(), ev, x, epi, cd, of);
    }
  };
  if (A->eb == 1) go(std::integral_constant<int, 1>{});
  else if (A->eb == 2) go(std::integral_constant<int, 2>{});
  else go(std::integral_constant<int, 0>{});
  DECO_CHECK_LAUNCH();
}

template <typename VT, typename XT, class Epi>
void launch_ell3(cudaStream_t st, const deco_csr_s* A, bool row0, const XT* x, Epi epi) {
  const int nbr = A->n / 3;
  if (nbr <= 0) return;
  const VT* ev;
  const VT* ov;
  if constexpr (sizeof(VT) == 4) { ev = A->ev32.get(); ov = A->ov32.get(); } else { ev = A->ev.get(); ov = A->ov.get(); }
  const unsigned grid = (unsigned)cdiv(nbr, 256);
  auto go = [&](auto wc) {
    constexpr int W = decltype(wc)::value;
    if (row0) launch_k(ell3_kernel<W, true, VT, XT, Epi>, grid, 256, 0, st, nbr, A->ec.get(), ev, A->oc.get(), ov, x, epi);
    else launch_k(ell3_kernel<W, false, VT, XT, Epi>, grid, 256, 0, st, nbr, A->ec.get(), ev, A->oc.get(), ov, x, epi);
  };
  if (A->ew == 4) go(std::integral_constant<int, 4>{});
  else if (A->ew == 7) go(std::integral_constant<int, 7>{});
  else go(std::integral_constant<int, 8>{});
  DECO_CHECK_LAUNCH();
}

// the slot-padded product of a cell-block matrix (2x2 or 3x3 cells)
template <typename VT, typename XT, class Epi>
void launch_ell_cells(cudaStream_t st, const deco_csr_s* A, bool row0, const XT* x, Epi epi) {
  if (A->bbs == 3) launch_ell3<VT, XT, Epi>(st, A, row0, x, epi);
  else launch_ell2<VT, XT, Epi>(st, A, row0, x, epi);
}

template <int BS, bool ROW0, typename VT, typename XT, class Epi>
void launch_bsr_bs(cudaStream_t st, int sw, int nbr, const int* br, const int* bc, const VT* bv, long long plane,
                   const XT* x, Epi epi) {
  if constexpr (BS == 2) {
    const unsigned grid = (unsigned)cdiv((long long)nbr * sw, 256);
    switch (sw) {
      case 1: launch_k(bsr2_pair_kernel<1, ROW0, VT, XT, Epi>, grid, 256, 0, st, nbr, br, bc, bv, plane, x, epi); break;
      case 2: launch_k(bsr2_pair_kernel<2, ROW0, VT, XT, Epi>, grid, 256, 0, st, nbr, br, bc, bv, plane, x, epi); break;
      case 4: launch_k(bsr2_pair_kernel<4, ROW0, VT, XT, Epi>, grid, 256, 0, st, nbr, br, bc, bv, plane, x, epi); break;
      default: launch_k(bsr2_pair_kernel<8, ROW0, VT, XT, Epi>, grid, 256, 0, st, nbr, br, bc, bv, plane, x, epi); break;
    }
    DECO_CHECK_LAUNCH();
    return;
  }
  const int block = 256;
  const unsigned grid = (unsigned)cdiv((long long)nbr * sw, block);
  switch (sw) {
    case 1: launch_k(bsr_kernel<1, BS, ROW0, VT, XT, Epi>, grid, block, 0, st, nbr, br, bc, bv, plane, x, epi); break;
    case 2: launch_k(bsr_kernel<2, BS, ROW0, VT, XT, Epi>, grid, block, 0, st, nbr, br, bc, bv, plane, x, epi); break;
    case 4: launch_k(bsr_kernel<4, BS, ROW0, VT, XT, Epi>, grid, block, 0, st, nbr, br, bc, bv, plane, x, epi); break;
    case 8: launch_k(bsr_kernel<8, BS, ROW0, VT, XT, Epi>, grid, block, 0, st, nbr, br, bc, bv, plane, x, epi); break;
    default: launch_k(bsr_kernel<16, BS, ROW0, VT, XT, Epi>, grid, block, 0, st, nbr, br, bc, bv, plane, x, epi); break;
  }
  DECO_CHECK_LAUNCH();
}

// y = op(A x) from the cell-block copy: all rows (row0 = false) or row 0 of
// every cell (row0 = true, output index = cell).
template <typename VT, typename XT, class Epi>
void launch_bsr(cudaStream_t st, const deco_csr_s* A, int sw, bool row0, const XT* x, Epi epi) {
  const int nbr = A->n / A->bbs;
  if (nbr <= 0) return;
  const VT* bv;
  if constexpr (sizeof(VT) == 4) bv = A->bv32.get(); else bv = A->bv.get();
  const long long plane = A->bplane;
  if (A->bbs == 2) {
    if (row0) launch_bsr_bs<2, true, VT, XT, Epi>(st, sw, nbr, A->br.get(), A->bc.get(), bv, plane, x, epi);
    else launch_bsr_bs<2, false, VT, XT, Epi>(st, sw, nbr, A->br.get(), A->bc.get(), bv, plane, x, epi);
  } else {
    if (row0) launch_bsr_bs<3, true, VT, XT, Epi>(st, sw, nbr, A->br.get(), A->bc.get(), bv, plane, x, epi);
    else launch_bsr_bs<3, false, VT, XT, Epi>(st, sw, nbr, A->br.get(), A->bc.get(), bv, plane, x, epi);
  }
}

// heuristic width: about two vector loads per lane per row, the best width
// measured on B200 for 7- and 14-entry rows in float64 (W = 2) and float32 (W = 4)
inline int heuristic_subwarp(double avg_row, int W) {
  const double half_loads = avg_row / (2.0 * W);
  int sw = 1;
  while (sw < 32 && sw < half_loads) sw <<= 1;
  return sw;
}

// Chooses (and caches) the sub-warp width of A for float64 (f32 = false) or
// float32 values: heuristic, refined by timing candidates when ctx->autotune.
int tuned_subwarp(deco_ctx_s* ctx, deco_csr_s* A, bool f32);

// Width for the cell-block kernel: about two blocks per lane, refined like
// tuned_subwarp.
int tuned_bsr_subwarp(deco_ctx_s* ctx, deco_csr_s* A, bool f32);

// The product autotuner: times every product A has a layout for -- the
// slot-padded copy (a thread per cell or per row: rows grouped per thread), the
// cell-block kernel at its tuned lanes per cell, the CSR kernel at its tuned
// lanes per row -- once per matrix shape and value precision (cached across
// setups), and records the fastest in A->plan64 / plan32, keeping the layout
// rules' choice unless another is at least 5 % faster.  No-op without
// ctx->autotune, below 4096 rows, or inside a stream capture.
void tune_product_plan(deco_ctx_s* ctx, deco_csr_s* A, bool f32);

// Builds (or rebuilds) the cell-block copy of A for bs x bs cells when the
// zero padding stays within max_fill x nz stored values; otherwise A keeps no
// block copy.  Float32 planes are made when A has float32 values.
void make_bsr(deco_ctx_s* ctx, deco_csr_s* A, int bs, double max_fill = 1.25);
// Builds the slot-padded copy of a 2x2-block matrix (4 slots when no cell has
// more than 4 blocks, else 7 or 8, the fewest that hold the widest cell, when the
// padding stays within 25 %; otherwise none), float32 values too when the block
// copy has them.  3x3-block matrices get 4, 7 or 8 slots, the fewest that hold
// all but at most 2 % of the cells within 25 % padding, the rest of the wider
// cells' blocks going to the overflow list.
// make_bsr and make_f32_values call it.
void make_padded(deco_ctx_s* ctx, deco_csr_s* A);
// The scalar slot-padded copy of a CSR matrix without cell blocks (4 slots when no
// row has more than 4 entries, 8 when none has more than 8 and the padding stays
// within 25 %), float32 values too when A has them; make_f32_values refreshes it.
void make_padded_scalar(deco_ctx_s* ctx, deco_csr_s* A);
// Offset codes of the slot columns of A's padded copy (nrow = cells for 2x2
// blocks, rows for scalar rows): 1-byte codes when at most 256 distinct column
// offsets occur, 2-byte codes up to 65536, none otherwise (and none when
// ctx->slot_codes is off).  make_padded and make_padded_scalar call it.
void make_slot_codes(deco_ctx_s* ctx, deco_csr_s* A, int nrow);
void drop_bsr(deco_csr_s* A);

// y = op(A x) over rows 0, bs, 2bs, ... (nrows_out = n / bs rows).  Uses the
// cell-block copy when A has one, the product is over all rows or row 0 of
// every cell, and x is aligned for the pair loads.
template <typename VT, typename XT, class Epi>
void spmv(deco_ctx_s* ctx, deco_csr_s* A, const XT* x, Epi epi, int bs = 1) {
  const bool f32 = sizeof(VT) == 4;
  const int plan = f32 ? A->plan32 : A->plan64;  // 0: the layout rules below
  if (plan != 3 && A->bbs > 1 && (bs == 1 || bs == A->bbs) && (!f32 || A->bv32) &&
      (reinterpret_cast<uintptr_t>(x) % (A->bbs == 2 ? 2 * sizeof(XT) : sizeof(XT))) == 0) {
    if (plan != 2 && A->ew && (!f32 || A->ev32)) {
      launch_ell_cells<VT, XT, Epi>(ctx->stream, A, bs != 1, x, epi);
      return;
    }
    launch_bsr<VT, XT, Epi>(ctx->stream, A, tuned_bsr_subwarp(ctx, A, f32), bs != 1, x, epi);
    return;
  }
  if (plan != 3 && !A->bbs && A->ew && bs == 1 && (!f32 || A->ev32)) {
    launch_ell1<VT, XT, Epi>(ctx->stream, A, x, epi);
    return;
  }
  const int sw = tuned_subwarp(ctx, A, f32);
  const VT* v;
  if constexpr (sizeof(VT) == 4) v = A->v32.get(); else v = A->v.get();
  launch_spmv_sw<VT, XT, Epi>(ctx->stream, sw, (A->n + bs - 1) / bs, bs, A->r.get(), A->c.get(), v, x, epi);
}

}  // namespace deco
