// fsai.cu — FSAI preconditioner on the device: filters, lower pattern, batched
// per-row dense LU grouped by order, D-scaling, transpose, apply.
//
// Per row i the reference (precond/FSAI/numeric.tpp:59-133, gather.cpp:14-88,
// LU_main.cpp:14-48) gathers M = A[P,P]^T for the row's pattern P (the row of
// lower(A) minus its last entry d), factors M with partial pivoting (dgetrf)
// and solves  M^T fU = -A[P,d]  and  M fL = -A[d,P]^T  (dgetrs 'T' / 'N').
// Here the same steps run with the dense arithmetic written as separately
// rounded multiplies and adds (no FMA contraction), in the operation order of a
// textbook LU with partial pivoting, so the factor values match the CPU
// restatement bit for bit and the reference's LAPACK to rounding.
//
// Rows are grouped by order k into classes and processed in ONE launch:
//   class 1 (k <= 7): one thread per row, M held per thread (registers and
//            its local frame);
//   classes 2-3 (k <= 16, <= 32): a group of S = 16 or 32 lanes per row, lane
//            c holding column c of M in registers; the pivot row's multipliers
//            travel by shuffles;
//   class 4 (32 < k <= 64): one warp per row, M in shared memory (32 KB).
#include <algorithm>

#include <climits>

#include "fsai.cuh"

namespace deco {

namespace {

constexpr int kLuBlock = 128;
// class 4: 64x64 system + rhs + pivots = 34048 B for the block's first warp
constexpr int kSmemBytes = 36 * 1024;

__device__ __forceinline__ int bsearch_le(const int* __restrict__ a, int lo, int hi, int target) {
  int mn = lo, mx = hi, mid = (lo + hi) >> 1;
  while (mx - mn > 1) {
    if (__ldg(a + mid) > target) mx = mid; else mn = mid;
    mid = (mn + mx) >> 1;
  }
  return mid;
}

// a - b*c and a + b*c with two roundings (the CPU oracle is built without contraction)
__device__ __forceinline__ double msub(double a, double b, double c) { return __dsub_rn(a, __dmul_rn(b, c)); }
__device__ __forceinline__ double madd(double a, double b, double c) { return __dadd_rn(a, __dmul_rn(b, c)); }

// ------------------------------------------------------------------ filters
__device__ __forceinline__ bool keep_entry(int i, int col, double v, double D, double tol_rel, double tol_abs) {
  if (col == i) return true;
  const double a = fabs(v);
  return (tol_rel == 0.0 || a > D) && (tol_abs == 0.0 || a > tol_abs);
}

// Half a warp per row: each lane takes every 16th entry, a ballot gives the kept
// entries' positions, so the row's reads and the compacted writes are coalesced
// (one thread per row walked its row alone: 2.4 ms for the 111M entries of the
// 8M-row system).  The kept entries keep their order.
__device__ __forceinline__ double filter_diag_tol(int i, int a, int e, const int* __restrict__ c,
                                                  const double* __restrict__ v, double tol_rel, unsigned hmask) {
  double D = 0.0;
  if (tol_rel != 0.0 && (threadIdx.x & 15) == 0) D = fabs(__dmul_rn(v[bsearch_le(c, a, e, i)], tol_rel));
  return __shfl_sync(hmask, D, 0, 16);
}

__global__ void filter_count(int n, const int* __restrict__ r, const int* __restrict__ c,
                             const double* __restrict__ v, double tol_rel, double tol_abs, int* __restrict__ cnt) {
  const int lane = threadIdx.x & 15;
  const unsigned hmask = 0xFFFFu << (threadIdx.x & 16);
  const long long step = ((long long)gridDim.x * blockDim.x) >> 4;
  for (long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 4; i < n; i += step) {
    const int a = r[i], e = r[i + 1];
    const double D = filter_diag_tol((int)i, a, e, c, v, tol_rel, hmask);
    int k = 0;
    for (int j0 = a; j0 < e; j0 += 16) {
      const int j = j0 + lane;
      const bool keep = j < e && keep_entry((int)i, c[j], v[j], D, tol_rel, tol_abs);
      k += __popc(__ballot_sync(hmask, keep) & hmask);
    }
    if (lane == 0) cnt[i] = k;
  }
}

__global__ void filter_copy(int n, const int* __restrict__ r, const int* __restrict__ c, const double* __restrict__ v,
                            double tol_rel, double tol_abs, const int* __restrict__ ro, int* __restrict__ co,
                            double* __restrict__ vo) {
  const int lane = threadIdx.x & 15;
  const unsigned hmask = 0xFFFFu << (threadIdx.x & 16);
  const unsigned below = hmask & ((1u << (threadIdx.x & 31)) - 1u);  // this half's lanes before this one
  const long long step = ((long long)gridDim.x * blockDim.x) >> 4;
  for (long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 4; i < n; i += step) {
    const int a = r[i], e = r[i + 1];
    const double D = filter_diag_tol((int)i, a, e, c, v, tol_rel, hmask);
    int o = ro[i];
    for (int j0 = a; j0 < e; j0 += 16) {
      const int j = j0 + lane;
      int cj = 0;
      double vj = 0.0;
      bool keep = false;
      if (j < e) {
        cj = c[j];
        vj = v[j];
        keep = keep_entry((int)i, cj, vj, D, tol_rel, tol_abs);
      }
      const unsigned bal = __ballot_sync(hmask, keep);
      if (keep) {
        const int pos = o + __popc(bal & below);
        co[pos] = cj;
        vo[pos] = vj;
      }
      o += __popc(bal & hmask);
    }
  }
}

// ---------------------------------------------------------- lower(A) pattern
// precond/FSAI/symbolic.tpp:104-148: the leading run of columns <= i
__global__ void lower_count(int n, const int* __restrict__ r, const int* __restrict__ c, int* __restrict__ cnt) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int k = 0;
    for (int j = r[i]; j < r[i + 1] && c[j] <= i; ++j) ++k;
    cnt[i] = k;
  }
}

__global__ void lower_copy(int n, const int* __restrict__ r, const int* __restrict__ c, const int* __restrict__ fr,
                           int* __restrict__ fc) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int o = fr[i];
    for (int j = r[i]; j < r[i + 1] && c[j] <= i; ++j) fc[o++] = c[j];
  }
}

// ---------------------------------------------------------- lower(A·A) pattern
// precond/FSAI/symbolic.tpp:149-172 (power 2): row i of the pattern is the set
// of columns c <= i of the rows k of A that row i of A references, sorted.
// One warp per row: the candidates gather into the warp's shared-memory buffer
// (ballot-compacted), a bitonic sort orders them, and the distinct values are
// counted (mode 0) or written (mode 1).  A row with more than kSqCap candidates
// raises *overflow and is left out (the caller reports it).
constexpr int kSqCap = 2048;
constexpr int kSqWarps = 4;

__global__ void __launch_bounds__(kSqWarps * 32) lower_square(int n, const int* __restrict__ r,
                                                             const int* __restrict__ c, int mode,
                                                             int* __restrict__ cnt, const int* __restrict__ fr,
                                                             int* __restrict__ fc, int* __restrict__ overflow) {
  extern __shared__ int sqbuf[];
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  int* buf = sqbuf + wl * kSqCap;
  const unsigned lt = (1u << lane) - 1u;
  for (int i = blockIdx.x * kSqWarps + wl; i < n; i += gridDim.x * kSqWarps) {
    int m = 0;
    bool over = false;
    for (int e = r[i]; e < r[i + 1] && !over; ++e) {
      const int k = c[e];
      const int kb = r[k], ke = r[k + 1];
      for (int t0 = kb; t0 < ke; t0 += 32) {
        const int t = t0 + lane;
        const int col = t < ke ? c[t] : INT_MAX;
        const bool take = col <= i;
        const unsigned mask = __ballot_sync(0xffffffffu, take);
        if (m + __popc(mask) > kSqCap) { over = true; break; }
        if (take) buf[m + __popc(mask & lt)] = col;
        m += __popc(mask);
        // row k is sorted: once a lane sees a column > i, the rest of the row is too
        if (__any_sync(0xffffffffu, t < ke && col > i)) break;
      }
    }
    if (over) {
      if (lane == 0) atomicExch(overflow, 1);
      if (mode == 0 && lane == 0) cnt[i] = 0;
      continue;
    }
    int np2 = 1;
    while (np2 < m) np2 <<= 1;
    for (int t = m + lane; t < np2; t += 32) buf[t] = INT_MAX;
    __syncwarp();
    for (int size = 2; size <= np2; size <<= 1)
      for (int stride = size >> 1; stride > 0; stride >>= 1) {
        for (int t = lane; t < np2 / 2; t += 32) {
          const int lo = 2 * stride * (t / stride) + (t % stride), hi = lo + stride;
          const bool up = (lo & size) == 0;
          const int a = buf[lo], b2 = buf[hi];
          if ((a > b2) == up) { buf[lo] = b2; buf[hi] = a; }
        }
        __syncwarp();
      }
    // distinct values, in order
    int total = 0;
    for (int t0 = 0; t0 < m; t0 += 32) {
      const int t = t0 + lane;
      const bool first = t < m && (t == 0 || buf[t] != buf[t - 1]);
      const unsigned mask = __ballot_sync(0xffffffffu, first);
      if (mode == 1 && first) fc[fr[i] + total + __popc(mask & lt)] = buf[t];
      total += __popc(mask);
    }
    if (mode == 0 && lane == 0) cnt[i] = total;
    __syncwarp();
  }
}

// ------------------------------------------------------------- row classes
__device__ __forceinline__ int order_class(int k) {
  return k <= 0 ? 0 : (k <= 7 ? 1 : (k <= 16 ? 2 : (k <= 32 ? 3 : (k <= 64 ? 4 : 5))));
}

__global__ void class_hist(int n, const int* __restrict__ fr, int* __restrict__ hist, int* __restrict__ kmax) {
  __shared__ int h[6];
  if (threadIdx.x < 6) h[threadIdx.x] = 0;
  __syncthreads();
  int m = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int k = fr[i + 1] - fr[i] - 1;
    atomicAdd(&h[order_class(k)], 1);
    m = max(m, k);
  }
  m = __reduce_max_sync(0xffffffffu, m);
  if ((threadIdx.x & 31) == 0) atomicMax(kmax, m);
  __syncthreads();
  if (threadIdx.x < 6 && h[threadIdx.x]) atomicAdd(&hist[threadIdx.x], h[threadIdx.x]);
}

// warp-aggregated: lanes of one class share a single atomic on the class cursor
__global__ void class_scatter(int n, const int* __restrict__ fr, int* __restrict__ cursor, int* __restrict__ perm) {
  const int lane = threadIdx.x & 31;
  for (int base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31; base < n; base += gridDim.x * blockDim.x) {
    const int i = base + lane;
    const int cl = i < n ? order_class(fr[i + 1] - fr[i] - 1) : 0;
    const unsigned same = __match_any_sync(0xffffffffu, cl);
    const int leader = __ffs(same) - 1;
    int pos = 0;
    if (lane == leader && cl >= 1 && cl <= 4) pos = atomicAdd(&cursor[cl], __popc(same));
    pos = __shfl_sync(0xffffffffu, pos, leader) + __popc(same & ((1u << lane) - 1));
    if (i < n && cl >= 1 && cl <= 4) perm[pos] = i;
  }
}

// ------------------------------------------------- class 1: thread per row
// M(i,j) of the column-major k x k system lives in m[i][j]; every index is a
// compile-time constant after unrolling, rows/columns >= k are predicated off.
template <int K>
__device__ void solve_row_reg(int i, const int* __restrict__ Ar, const int* __restrict__ Ac,
                              const double* __restrict__ Av, const int* __restrict__ Fr, const int* __restrict__ Fc,
                              double* __restrict__ FLv, double* __restrict__ FUv) {
  const int a = Fr[i], e = Fr[i + 1] - 1, k = e - a;
  const int d = Fc[e];
  int P[K];
#pragma unroll
  for (int t = 0; t < K; ++t) P[t] = t < k ? Fc[a + t] : 0x7fffffff;
  double m[K][K], rl[K], ru[K];
#pragma unroll
  for (int x = 0; x < K; ++x) {
    rl[x] = 0.0; ru[x] = 0.0;
#pragma unroll
    for (int y = 0; y < K; ++y) m[x][y] = 0.0;
  }
  // gather: M(col,row) = A(P[row], P[col]);  ru[row] = -A(P[row], d)
#pragma unroll
  for (int row = 0; row < K; ++row) {
    if (row < k) {
      const int g = P[row];
      const int ga = Ar[g], gb = Ar[g + 1];
      int q = 0;  // merge pointer into P
      for (int s = ga; s < gb; ++s) {
        const int col = Ac[s];
        while (q < k && __ldg(Fc + a + q) < col) ++q;  // pattern sorted ascending
        if (q < k && __ldg(Fc + a + q) == col) {
          const double val = Av[s];
#pragma unroll
          for (int t = 0; t < K; ++t)
            if (t == q) m[t][row] = val;
        }
      }
      const int j = bsearch_le(Ac, ga, gb, d);
      if (Ac[j] == d) ru[row] = -Av[j];
    }
  }
  {  // rl[col] = -A(d, P[col])
    const int da = Ar[d], db = Ar[d + 1];
    int q = 0;
    for (int s = da; s < db; ++s) {
      const int col = Ac[s];
      while (q < k && __ldg(Fc + a + q) < col) ++q;
      if (q < k && __ldg(Fc + a + q) == col) {
        const double val = -Av[s];
#pragma unroll
        for (int t = 0; t < K; ++t)
          if (t == q) rl[t] = val;
      }
    }
  }
  // LU with partial pivoting (first index of the largest |entry|)
  int piv[K];
#pragma unroll
  for (int j = 0; j < K; ++j) {
    piv[j] = j;
    if (j < k) {
      int p = j;
      double best = fabs(m[j][j]);
#pragma unroll
      for (int x = j + 1; x < K; ++x)
        if (x < k && fabs(m[x][j]) > best) { best = fabs(m[x][j]); p = x; }
      piv[j] = p;
#pragma unroll
      for (int x = j + 1; x < K; ++x)
        if (x == p) {
#pragma unroll
          for (int t = 0; t < K; ++t) { double s = m[j][t]; m[j][t] = m[x][t]; m[x][t] = s; }
        }
      const double dg = m[j][j];
      if (dg != 0.0) {
        const double inv = __ddiv_rn(1.0, dg);
#pragma unroll
        for (int x = j + 1; x < K; ++x)
          if (x < k) m[x][j] = __dmul_rn(m[x][j], inv);
      }
#pragma unroll
      for (int t = j + 1; t < K; ++t)
        if (t < k) {
          const double u = m[j][t];
#pragma unroll
          for (int x = j + 1; x < K; ++x)
            if (x < k) m[x][t] = msub(m[x][t], m[x][j], u);
        }
    }
  }
  // M^T fU = ru : U^T, unit L^T, then P^T
#pragma unroll
  for (int j = 0; j < K; ++j)
    if (j < k) {
      double s = ru[j];
#pragma unroll
      for (int x = 0; x < j; ++x) s = msub(s, m[x][j], ru[x]);
      ru[j] = __ddiv_rn(s, m[j][j]);
    }
#pragma unroll
  for (int j = K - 1; j >= 0; --j)
    if (j < k) {
      double s = ru[j];
#pragma unroll
      for (int x = j + 1; x < K; ++x)
        if (x < k) s = msub(s, m[x][j], ru[x]);
      ru[j] = s;
    }
#pragma unroll
  for (int j = K - 1; j >= 0; --j)
    if (j < k && piv[j] != j) {
#pragma unroll
      for (int x = j + 1; x < K; ++x)
        if (x == piv[j]) { double s = ru[j]; ru[j] = ru[x]; ru[x] = s; }
    }
  // M fL = rl : P, unit L, U
#pragma unroll
  for (int j = 0; j < K; ++j)
    if (j < k && piv[j] != j) {
#pragma unroll
      for (int x = j + 1; x < K; ++x)
        if (x == piv[j]) { double s = rl[j]; rl[j] = rl[x]; rl[x] = s; }
    }
#pragma unroll
  for (int j = 0; j < K; ++j)
    if (j < k) {
#pragma unroll
      for (int x = j + 1; x < K; ++x)
        if (x < k) rl[x] = msub(rl[x], m[x][j], rl[j]);
    }
#pragma unroll
  for (int j = K - 1; j >= 0; --j)
    if (j < k) {
      rl[j] = __ddiv_rn(rl[j], m[j][j]);
#pragma unroll
      for (int x = 0; x < j; ++x) rl[x] = msub(rl[x], m[x][j], rl[j]);
    }
#pragma unroll
  for (int t = 0; t < K; ++t)
    if (t < k) { FLv[a + t] = rl[t]; FUv[a + t] = ru[t]; }
}

// --------------------------------------- classes 2-3: a lane group per row
// S lanes (16 or 32; k <= S) solve one row's system.  Lane c holds column c
// of M in registers (col[t] = M(t, c)), ru_c and, as the factorisation moves
// rows, the entry of rl at its current row position (rl is carried along with
// the row swaps and eliminated step by step, which is the forward substitution
// P M = L U needs).  Every element sees the separately rounded operations of the
// textbook order the thread-per-row form used:
//   step j: pivot = first index of the largest |M(x, j)|, x >= j (lane j scans
//   its column); rows j and p swapped in every column; lane j scales its
//   multipliers by 1 / M(j, j); the multipliers reach every lane by shuffles and
//   column t subtracts M(x, j) M(j, t) from M(x, t); row x of rl subtracts
//   M(x, j) rl_j;
// then U^T a = ru (right-looking, lane j accumulating in ascending x), the
// unit L^T sweep from the bottom (each b_j sums its terms in ascending x, so it
// runs serially, lane j after lane j + 1), the pivots undone on b, and U on rl
// from the bottom.  Loops run to S with predicates on k, so the two or four
// groups of a warp stay converged for the full-warp shuffles.
// Shared memory per group: the pattern (S ints), b (S doubles), pivots (S ints).
template <int S>
__device__ void solve_row_group(int i, int* __restrict__ sP, double* __restrict__ sb, int* __restrict__ spv,
                                const int* __restrict__ Ar, const int* __restrict__ Ac, const double* __restrict__ Av,
                                const int* __restrict__ Fr, const int* __restrict__ Fc, double* __restrict__ FLv,
                                double* __restrict__ FUv) {
  constexpr unsigned kAll = 0xffffffffu;
  const int g = threadIdx.x & (S - 1);
  int a = 0, k = 0, d = 0;
  if (i >= 0) {
    a = Fr[i];
    const int e = Fr[i + 1] - 1;
    k = e - a;
    d = Fc[e];
  }
  if (g < k) sP[g] = Fc[a + g];
  __syncwarp();
  // gather: col[t] = M(t, g) = A(P[g], P[t]);  ru = -A(P[g], d);  rl = -A(d, P[g])
  double col[S];
#pragma unroll
  for (int t = 0; t < S; ++t) col[t] = 0.0;
  double ru = 0.0, rl = 0.0;
  if (g < k) {
    const int pg = sP[g];
    const int ga = Ar[pg], gb = Ar[pg + 1];
    int q = 0;  // merge pointer into the (ascending) pattern
    for (int s2 = ga; s2 < gb; ++s2) {
      const int cc = Ac[s2];
      while (q < k && sP[q] < cc) ++q;
      if (q < k && sP[q] == cc) {
        const double val = Av[s2];
#pragma unroll
        for (int t = 0; t < S; ++t)
          if (t == q) col[t] = val;
      }
      if (cc == d) ru = -Av[s2];
    }
    const int da = Ar[d], db = Ar[d + 1];
    const int jx = bsearch_le(Ac, da, db, pg);
    if (Ac[jx] == pg) rl = -Av[jx];
  }
  // LU with partial pivoting, rl carried along (forward substitution with unit L)
#pragma unroll
  for (int j = 0; j < S; ++j) {
    int p = j;
    if (g == j) {
      double best = fabs(col[j]);
#pragma unroll
      for (int x = 0; x < S; ++x)
        if (x > j && x < k && fabs(col[x]) > best) { best = fabs(col[x]); p = x; }
    }
    p = __shfl_sync(kAll, p, j, S);
    if (g == 0) spv[j] = p;
    if (p != j) {  // uniform over the group
#pragma unroll
      for (int x = 0; x < S; ++x)
        if (x > j && x == p) { const double t = col[j]; col[j] = col[x]; col[x] = t; }
    }
    {
      const double rj = __shfl_sync(kAll, rl, j, S), rp = __shfl_sync(kAll, rl, p, S);
      if (g == j) rl = rp;
      else if (g == p) rl = rj;
    }
    if (g == j && j < k && col[j] != 0.0) {
      const double inv = __ddiv_rn(1.0, col[j]);
#pragma unroll
      for (int x = 0; x < S; ++x)
        if (x > j && x < k) col[x] = __dmul_rn(col[x], inv);
    }
    const double rlj = __shfl_sync(kAll, rl, j, S);
#pragma unroll
    for (int x = 0; x < S; ++x) {
      if (x <= j) continue;  // (constant bounds: every loop here unrolls to static register indices)
      const double mx = __shfl_sync(kAll, col[x], j, S);  // M(x, j), the multiplier
      if (x < k) {
        if (g > j && g < k) col[x] = msub(col[x], mx, col[j]);
        if (g == x) rl = msub(rl, mx, rlj);
      }
    }
  }
  // U^T a = ru: lane g holds s_g; a_x = s_x / U(x, x), then s_g -= U(x, g) a_x for g > x
#pragma unroll
  for (int x = 0; x < S; ++x) {
    if (g == x && x < k) ru = __ddiv_rn(ru, col[x]);
    const double ax = __shfl_sync(kAll, ru, x, S);
    if (g > x && g < k && x < k) ru = msub(ru, col[x], ax);
  }
  // unit L^T b = a from the bottom: b_j = a_j - sum_{x > j} L(x, j) b_x, x ascending
#pragma unroll
  for (int j = S - 1; j >= 0; --j) {
    if (g == j && j < k) {
      double s2 = ru;
#pragma unroll
      for (int x = 0; x < S; ++x)
        if (x > j && x < k) s2 = msub(s2, col[x], sb[x]);
      sb[j] = s2;
    }
    __syncwarp();
  }
  // fU = P^T b
  if (g == 0)
    for (int j = k - 1; j >= 0; --j) {
      const int pj = spv[j];
      if (pj != j) { const double t = sb[j]; sb[j] = sb[pj]; sb[pj] = t; }
    }
  __syncwarp();
  if (g < k) FUv[a + g] = sb[g];
  // U fL = (L^-1 P rl) from the bottom: rl_j /= U(j, j), then rl_x -= U(x, j) rl_j for x < j
#pragma unroll
  for (int j = S - 1; j >= 0; --j) {
    if (g == j && j < k) rl = __ddiv_rn(rl, col[j]);
    const double rj = __shfl_sync(kAll, rl, j, S);
#pragma unroll
    for (int x = 0; x < S; ++x) {
      if (x >= j) continue;
      const double ux = __shfl_sync(kAll, col[x], j, S);  // U(x, j) from lane j
      if (g == x && j < k) rl = msub(rl, ux, rj);
    }
  }
  if (g < k) FLv[a + g] = rl;
  __syncwarp();
}

// --------------------------------------------------- class 4: warp per row
// M column-major in shared memory: M(i,j) = sm[i + j*k].
__device__ int find_in_pattern(const int* __restrict__ P, int k, int key) {
  int lo = 0, hi = k - 1;
  while (lo <= hi) {
    int mid = (lo + hi) >> 1;
    int v = P[mid];
    if (v == key) return mid;
    if (v < key) lo = mid + 1; else hi = mid - 1;
  }
  return -1;
}

__device__ void solve_row_warp(int i, double* __restrict__ sm, double* __restrict__ rl, double* __restrict__ ru,
                               int* __restrict__ piv, const int* __restrict__ Ar, const int* __restrict__ Ac,
                               const double* __restrict__ Av, const int* __restrict__ Fr,
                               const int* __restrict__ Fc, double* __restrict__ FLv, double* __restrict__ FUv) {
  const int lane = threadIdx.x & 31;
  const int a = Fr[i], e = Fr[i + 1] - 1, k = e - a;
  const int d = Fc[e];
  const int* P = Fc + a;
  for (int t = lane; t < k * k; t += 32) sm[t] = 0.0;
  for (int t = lane; t < k; t += 32) { rl[t] = 0.0; ru[t] = 0.0; }
  __syncwarp();
  for (int row = 0; row < k; ++row) {
    const int g = P[row];
    const int ga = Ar[g], gb = Ar[g + 1];
    for (int s = ga + lane; s < gb; s += 32) {
      const int col = Ac[s];
      const int q = find_in_pattern(P, k, col);
      if (q >= 0) sm[q + row * k] = Av[s];
      if (col == d) ru[row] = -Av[s];
    }
  }
  {
    const int da = Ar[d], db = Ar[d + 1];
    for (int s = da + lane; s < db; s += 32) {
      const int q = find_in_pattern(P, k, Ac[s]);
      if (q >= 0) rl[q] = -Av[s];
    }
  }
  __syncwarp();
  // LU with partial pivoting
  for (int j = 0; j < k; ++j) {
    double best = -1.0;
    int p = 0x7fffffff;
    for (int x = j + lane; x < k; x += 32) {
      double v = fabs(sm[x + j * k]);
      if (v > best) { best = v; p = x; }  // rows visited in increasing order per lane
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      double ob = __shfl_xor_sync(0xffffffffu, best, o);
      int op = __shfl_xor_sync(0xffffffffu, p, o);
      if (ob > best || (ob == best && op < p)) { best = ob; p = op; }
    }
    // first index of the maximum, as a sequential scan with strict '>' finds
    if (lane == 0) piv[j] = p;
    if (p != j)
      for (int t = lane; t < k; t += 32) {
        double s = sm[j + t * k];
        sm[j + t * k] = sm[p + t * k];
        sm[p + t * k] = s;
      }
    __syncwarp();
    const double dg = sm[j + j * k];
    if (dg != 0.0) {
      const double inv = __ddiv_rn(1.0, dg);
      for (int x = j + 1 + lane; x < k; x += 32) sm[x + j * k] = __dmul_rn(sm[x + j * k], inv);
    }
    __syncwarp();
    for (int t = j + 1; t < k; ++t) {
      const double u = sm[j + t * k];
      for (int x = j + 1 + lane; x < k; x += 32) sm[x + t * k] = msub(sm[x + t * k], sm[x + j * k], u);
    }
    __syncwarp();
  }
  // M^T fU = ru (lane 0 runs the short recurrences; k <= 64)
  if (lane == 0) {
    for (int j = 0; j < k; ++j) {
      double s = ru[j];
      for (int x = 0; x < j; ++x) s = msub(s, sm[x + j * k], ru[x]);
      ru[j] = __ddiv_rn(s, sm[j + j * k]);
    }
    for (int j = k - 1; j >= 0; --j) {
      double s = ru[j];
      for (int x = j + 1; x < k; ++x) s = msub(s, sm[x + j * k], ru[x]);
      ru[j] = s;
    }
    for (int j = k - 1; j >= 0; --j)
      if (piv[j] != j) { double s = ru[j]; ru[j] = ru[piv[j]]; ru[piv[j]] = s; }
    for (int j = 0; j < k; ++j)
      if (piv[j] != j) { double s = rl[j]; rl[j] = rl[piv[j]]; rl[piv[j]] = s; }
  }
  __syncwarp();
  // M fL = rl: forward with unit L, backward with U (lanes over rows)
  for (int j = 0; j < k; ++j) {
    const double bj = rl[j];
    for (int x = j + 1 + lane; x < k; x += 32) rl[x] = msub(rl[x], sm[x + j * k], bj);
    __syncwarp();
  }
  for (int j = k - 1; j >= 0; --j) {
    if (lane == 0) rl[j] = __ddiv_rn(rl[j], sm[j + j * k]);
    __syncwarp();
    const double bj = rl[j];
    for (int x = lane; x < j; x += 32) rl[x] = msub(rl[x], sm[x + j * k], bj);
    __syncwarp();
  }
  for (int t = lane; t < k; t += 32) { FLv[a + t] = rl[t]; FUv[a + t] = ru[t]; }
  __syncwarp();
}

// one launch: blocks [0,b1) class 1 (a row per thread), [b1,b2) class 2 (8 per
// block), [b2,b3) class 3 (4 per block), then class 4 (one per block); perm holds
// the rows class by class, from offsets o[0..3]
template <int S>
__device__ __forceinline__ void group_row(int q, int nq, const int* __restrict__ rows, int* gP, double* gB, int* gPv,
                                          const int* __restrict__ Ar, const int* __restrict__ Ac,
                                          const double* __restrict__ Av, const int* __restrict__ Fr,
                                          const int* __restrict__ Fc, double* __restrict__ FLv,
                                          double* __restrict__ FUv) {
  const int g0 = threadIdx.x & ~(S - 1);  // the group's first thread: its slice of the shared arrays
  solve_row_group<S>(q < nq ? rows[q] : -1, gP + g0, gB + g0, gPv + g0, Ar, Ac, Av, Fr, Fc, FLv, FUv);
}

// KR: the order of class 1's per-thread system (4 when no row is wider, else 7);
// WIDE: whether classes 2-4 occur.  The narrow instantiations carry only the
// class-1 code, so they need far fewer registers (more rows in flight per SM);
// the launch still covers every row of the factor.
template <int KR, bool WIDE>
__global__ void __launch_bounds__(kLuBlock) fsai_local_systems(
    const int* __restrict__ perm, int4 cnt, int4 off, int b1, int b2, int b3, const int* __restrict__ Ar,
    const int* __restrict__ Ac, const double* __restrict__ Av, const int* __restrict__ Fr,
    const int* __restrict__ Fc, double* __restrict__ FLv, double* __restrict__ FUv) {
  extern __shared__ double smem[];
  __shared__ int gP[WIDE ? kLuBlock : 1];
  __shared__ double gB[WIDE ? kLuBlock : 1];
  __shared__ int gPv[WIDE ? kLuBlock : 1];
  const int b = blockIdx.x;
  if (b < b1) {
    const int q = b * kLuBlock + threadIdx.x;
    if (q < cnt.x) solve_row_reg<KR>(perm[off.x + q], Ar, Ac, Av, Fr, Fc, FLv, FUv);
    return;
  }
  if constexpr (WIDE) {
  if (b < b2) {
    group_row<16>((b - b1) * (kLuBlock / 16) + threadIdx.x / 16, cnt.y, perm + off.y, gP, gB, gPv, Ar, Ac, Av, Fr,
                  Fc, FLv, FUv);
    return;
  }
  if (b < b3) {
    group_row<32>((b - b2) * (kLuBlock / 32) + threadIdx.x / 32, cnt.z, perm + off.z, gP, gB, gPv, Ar, Ac, Av, Fr,
                  Fc, FLv, FUv);
    return;
  }
  const int q = b - b3;
  if ((threadIdx.x >> 5) != 0 || q >= cnt.w) return;
  double* base = smem;  // 64x64 system (32 KB), then rhs and pivots
  double* rl = smem + 64 * 64;
  solve_row_warp(perm[off.w + q], base, rl, rl + 64, reinterpret_cast<int*>(rl + 128), Ar, Ac, Av, Fr, Fc, FLv, FUv);
  }
}

// ------------------------------------------------- D-scaling (diagonal.cpp)
// Row i only reads its own FL/FU rows and rows of A, so the diagonal reset, D_i
// and the scaling of row i fuse into one thread.
__global__ void fsai_scale(int n, const int* __restrict__ Ar, const int* __restrict__ Ac,
                           const double* __restrict__ Av, const int* __restrict__ Fr, const int* __restrict__ Fc,
                           double* __restrict__ FLv, double* __restrict__ FUv) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int aF = Fr[i], bF = Fr[i + 1];
    if (bF == aF) continue;  // an empty pattern row has no diagonal to set
    FLv[bF - 1] = 1.0;
    FUv[bF - 1] = 1.0;
    double sum = 0.0;
    for (int j = aF; j < bF; ++j) {
      const double fl = FLv[j];
      if (fl != 0.0) {
        const int colF = Fc[j];
        int pa = Ar[colF], pb = Ar[colF + 1], pu = aF;
        double s = 0.0;
        while (pa < pb && pu < bF) {
          const int ca = Ac[pa], cu = Fc[pu];
          if (ca == cu) { s = madd(s, Av[pa], FUv[pu]); ++pa; ++pu; }
          else if (ca < cu) ++pa;
          else ++pu;
        }
        sum = madd(sum, fl, s);
      }
    }
    const double D = (sum < 0.0) ? -__ddiv_rn(1.0, __dsqrt_rn(fabs(sum))) : __ddiv_rn(1.0, __dsqrt_rn(sum));
    const double Da = fabs(D);
    for (int j = aF; j < bF; ++j) {
      FLv[j] = __dmul_rn(FLv[j], D);
      FUv[j] = __dmul_rn(FUv[j], Da);
    }
  }
}

// ------------------------------------------------------- transpose (CSR.hpp)
__global__ void col_count(long long nz, const int* __restrict__ c, int* __restrict__ cnt) {
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < nz; j += (long long)gridDim.x * blockDim.x)
    atomicAdd(&cnt[c[j]], 1);
}

__global__ void col_scatter(int n, const int* __restrict__ r, const int* __restrict__ c, const double* __restrict__ v,
                            int* __restrict__ cursor, int* __restrict__ tc, double* __restrict__ tv) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    for (int j = r[i]; j < r[i + 1]; ++j) {
      const int pos = atomicAdd(&cursor[c[j]], 1);
      tc[pos] = i;
      tv[pos] = v[j];
    }
}

// rows of the transpose get their entries in ascending source-row order, the
// order the reference's sequential scatter produces (CSR.hpp:193-206)
// (rows of up to kSortReg entries are sorted in registers: loaded once, an
// unrolled insertion sort on compile-time indices, stored once)
constexpr int kSortReg = 12;
__global__ void sort_rows(int n, const int* __restrict__ r, int* __restrict__ c, double* __restrict__ v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int a = r[i], e = r[i + 1];
    if (e - a <= kSortReg) {
      int kc[kSortReg];
      double kv[kSortReg];
#pragma unroll
      for (int t = 0; t < kSortReg; ++t) {
        kc[t] = a + t < e ? c[a + t] : INT_MAX;
        kv[t] = a + t < e ? v[a + t] : 0.0;
      }
      // insertion sort: the columns are distinct, so the order is the ascending one
#pragma unroll
      for (int t = 1; t < kSortReg; ++t)
#pragma unroll
        for (int u = t; u > 0; --u)
          if (kc[u - 1] > kc[u]) {
            const int tc = kc[u]; kc[u] = kc[u - 1]; kc[u - 1] = tc;
            const double tv = kv[u]; kv[u] = kv[u - 1]; kv[u - 1] = tv;
          }
#pragma unroll
      for (int t = 0; t < kSortReg; ++t)
        if (a + t < e) { c[a + t] = kc[t]; v[a + t] = kv[t]; }
      continue;
    }
    for (int j = a + 1; j < e; ++j) {
      const int key = c[j];
      const double val = v[j];
      int t = j - 1;
      while (t >= a && c[t] > key) { c[t + 1] = c[t]; v[t + 1] = v[t]; --t; }
      c[t + 1] = key;
      v[t + 1] = val;
    }
  }
}

}  // namespace

void csr_filter(deco_ctx_s* ctx, const deco_csr_s* A, double tol_rel, double tol_abs, deco_csr_s* out) {
  cudaStream_t st = ctx->stream;
  const int n = A->n;
  DevBuf<int> cnt(n + 1, st);
  const int g = grid_for(ctx, n, 256);
  trace_mark(ctx, "filter: count buffer");
  filter_count<<<g, 256, 0, st>>>(n, A->r.get(), A->c.get(), A->v.get(), tol_rel, tol_abs, cnt.get());
  DECO_CHECK_LAUNCH();
  trace_mark(ctx, "filter: count");
  out->n = n;
  out->m = A->m;
  out->r.alloc(n + 1, st);
  out->nz = (int)exclusive_scan_int(ctx, cnt.get(), out->r.get(), n);
  trace_mark(ctx, "filter: scan");
  out->c.alloc(out->nz, st);
  out->v.alloc(out->nz, st);
  trace_mark(ctx, "filter: allocate");
  filter_copy<<<g, 256, 0, st>>>(n, A->r.get(), A->c.get(), A->v.get(), tol_rel, tol_abs, out->r.get(),
                                 out->c.get(), out->v.get());
  DECO_CHECK_LAUNCH();
  trace_mark(ctx, "filter: copy");
  refresh_stats(ctx, out);
}

void csr_filter_inplace(deco_ctx_s* ctx, deco_csr_s* A, double tol_rel, double tol_abs) {
  deco_csr_s B;
  csr_filter(ctx, A, tol_rel, tol_abs, &B);
  drop_bsr(A);
  A->nz = B.nz;
  A->r = std::move(B.r);
  A->c = std::move(B.c);
  A->v = std::move(B.v);
  if (A->v32) make_f32_values(ctx, A);
  refresh_stats(ctx, A);
}

void csr_transpose(deco_ctx_s* ctx, int n, int m, int nz, const int* r, const int* c, const double* v,
                   deco_csr_s* T) {
  cudaStream_t st = ctx->stream;
  T->n = m;
  T->m = n;
  T->nz = nz;
  DevBuf<int> ccount(m + 1, st);
  ccount.zero(st);
  if (nz) {
    col_count<<<grid_for(ctx, nz, 256), 256, 0, st>>>(nz, c, ccount.get());
    DECO_CHECK_LAUNCH();
  }
  T->r.alloc(m + 1, st);
  exclusive_scan_int(ctx, ccount.get(), T->r.get(), m);
  T->c.alloc(nz, st);
  T->v.alloc(nz, st);
  if (nz) {
    DECO_CUDA(cudaMemcpyAsync(ccount.get(), T->r.get(), sizeof(int) * m, cudaMemcpyDeviceToDevice, st));
    col_scatter<<<grid_for(ctx, n, 256), 256, 0, st>>>(n, r, c, v, ccount.get(), T->c.get(), T->v.get());
    DECO_CHECK_LAUNCH();
    sort_rows<<<grid_for(ctx, m, 256), 256, 0, st>>>(m, T->r.get(), T->c.get(), T->v.get());
    DECO_CHECK_LAUNCH();
  }
  refresh_stats(ctx, T);
}

void fsai_build(deco_ctx_s* ctx, const deco_csr_s* A0, double tol_rel, double tol_abs, int power, int precision,
                deco_fsai_s* F, int bs) {
  cudaStream_t st = ctx->stream;
  DECO_REQUIRE(A0->n == A0->m, DECO_ERR_ARG, "FSAI needs a square matrix");
  DECO_REQUIRE(power == 1 || power == 2, DECO_ERR_UNSUPPORTED,
               "FSAI power " + std::to_string(power) + " is not implemented (symbolic.tpp:173-176 supports 1 and 2)");
  DECO_REQUIRE(precision == 64 || precision == 32, DECO_ERR_ARG, "precision must be 64 or 32");
  const int n = A0->n;
  trace_mark(ctx, nullptr);
  F->n = n;
  F->precision = precision;
  // 1. filtered copy (FSAI.hpp:22-28)
  deco_csr_s Af;
  const deco_csr_s* A = A0;
  if (tol_rel != 0.0 || tol_abs != 0.0) {
    csr_filter(ctx, A0, tol_rel, tol_abs, &Af);
    A = &Af;
  }
  const int g = grid_for(ctx, n, 256);
  trace_mark(ctx, "fsai filter");
  // 2. symbolic: lower(A) (power 1) or lower(A A) (power 2)
  DevBuf<int> cnt(n + 1, st);
  deco_csr_s& FL = F->FL;
  FL.n = FL.m = n;
  FL.r.alloc(n + 1, st);
  if (power == 1) {
    lower_count<<<g, 256, 0, st>>>(n, A->r.get(), A->c.get(), cnt.get());
    DECO_CHECK_LAUNCH();
    FL.nz = (int)exclusive_scan_int(ctx, cnt.get(), FL.r.get(), n);
    FL.c.alloc(FL.nz, st);
    lower_copy<<<g, 256, 0, st>>>(n, A->r.get(), A->c.get(), FL.r.get(), FL.c.get());
    DECO_CHECK_LAUNCH();
  } else {
    const size_t smem = sizeof(int) * kSqCap * kSqWarps;
    DECO_CUDA(cudaFuncSetAttribute(lower_square, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    DevBuf<int> over(1, st);
    over.zero(st);
    const int gs = grid_for(ctx, cdiv(n, kSqWarps), 1, 16);
    lower_square<<<gs, kSqWarps * 32, smem, st>>>(n, A->r.get(), A->c.get(), 0, cnt.get(), nullptr, nullptr,
                                                  over.get());
    DECO_CHECK_LAUNCH();
    FL.nz = (int)exclusive_scan_int(ctx, cnt.get(), FL.r.get(), n);
    int ho = 0;
    DECO_CUDA(cudaMemcpyAsync(&ho, over.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    DECO_CUDA(cudaStreamSynchronize(st));
    DECO_REQUIRE(ho == 0, DECO_ERR_UNSUPPORTED,
                 "FSAI power 2: a row of A A has more than " + std::to_string(kSqCap) + " candidate columns");
    FL.c.alloc(FL.nz, st);
    lower_square<<<gs, kSqWarps * 32, smem, st>>>(n, A->r.get(), A->c.get(), 1, nullptr, FL.r.get(), FL.c.get(),
                                                  over.get());
    DECO_CHECK_LAUNCH();
  }
  FL.v.alloc(FL.nz, st);
  FL.v.zero(st);
  F->nz = FL.nz;
  DevBuf<double> fu(FL.nz, st);  // FU values in FL's (lower) layout before the transpose
  fu.zero(st);
  trace_mark(ctx, "fsai symbolic");
  // 3. group rows by order and solve the local systems in one launch
  DevBuf<int> hist(16, st);
  hist.zero(st);
  class_hist<<<g, 256, 0, st>>>(n, FL.r.get(), hist.get(), hist.get() + 8);
  DECO_CHECK_LAUNCH();
  int h[16];
  DECO_CUDA(cudaMemcpyAsync(h, hist.get(), sizeof(h), cudaMemcpyDeviceToHost, st));
  DECO_CUDA(cudaStreamSynchronize(st));
  F->max_order = h[8];
  DECO_REQUIRE(h[5] == 0, DECO_ERR_UNSUPPORTED,
               "FSAI local system of order " + std::to_string(h[8]) + " exceeds the supported maximum of 64");
  const int n1 = h[1], n2 = h[2], n3 = h[3], n4 = h[4];
  const int nsolve = n1 + n2 + n3 + n4;
  if (nsolve > 0) {
    DevBuf<int> perm(nsolve, st);
    int cur[5] = {0, 0, n1, n1 + n2, n1 + n2 + n3};
    DevBuf<int> cursor(5, st);
    DECO_CUDA(cudaMemcpyAsync(cursor.get(), cur, sizeof(cur), cudaMemcpyHostToDevice, st));
    class_scatter<<<g, 256, 0, st>>>(n, FL.r.get(), cursor.get(), perm.get());
    DECO_CHECK_LAUNCH();
    const int b1 = (int)cdiv(n1, kLuBlock);
    const int b2 = b1 + (int)cdiv(n2, kLuBlock / 16);
    const int b3 = b2 + (int)cdiv(n3, kLuBlock / 32);
    const int nblk = b3 + n4;
    const size_t smem = n4 > 0 ? kSmemBytes : 0;
    const int4 cnt4 = make_int4(n1, n2, n3, n4), off4 = make_int4(0, n1, n1 + n2, n1 + n2 + n3);
    if (n2 + n3 + n4 > 0) {
      if (smem) DECO_CUDA(cudaFuncSetAttribute(fsai_local_systems<7, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               kSmemBytes));
      fsai_local_systems<7, true><<<nblk, kLuBlock, smem, st>>>(perm.get(), cnt4, off4, b1, b2, b3, A->r.get(),
                                                                A->c.get(), A->v.get(), FL.r.get(), FL.c.get(),
                                                                FL.v.get(), fu.get());
    } else if (h[8] <= 4) {
      fsai_local_systems<4, false><<<nblk, kLuBlock, 0, st>>>(perm.get(), cnt4, off4, b1, b2, b3, A->r.get(),
                                                              A->c.get(), A->v.get(), FL.r.get(), FL.c.get(),
                                                              FL.v.get(), fu.get());
    } else {  // orders up to 7 (the 2x2 cells of a 7-point stencil)
      fsai_local_systems<7, false><<<nblk, kLuBlock, 0, st>>>(perm.get(), cnt4, off4, b1, b2, b3, A->r.get(),
                                                              A->c.get(), A->v.get(), FL.r.get(), FL.c.get(),
                                                              FL.v.get(), fu.get());
    }
    DECO_CHECK_LAUNCH();
  }
  trace_mark(ctx, "fsai local systems");
  // 4. D = diag(FL A FU^T); FL *= D, FU *= |D|  (diagonal.cpp:6-73)
  fsai_scale<<<g, 256, 0, st>>>(n, A->r.get(), A->c.get(), A->v.get(), FL.r.get(), FL.c.get(), FL.v.get(), fu.get());
  DECO_CHECK_LAUNCH();
  trace_mark(ctx, "fsai scaling");
  // 5. FU^T (trans_mat_full)
  deco_csr_s& U = F->FUt;
  csr_transpose(ctx, n, n, FL.nz, FL.r.get(), FL.c.get(), fu.get(), &U);
  refresh_stats(ctx, &FL);
  trace_mark(ctx, "fsai transpose");
  if (bs > 1) {
    make_bsr(ctx, &FL, bs);
    make_bsr(ctx, &U, bs);
  } else {  // (csr_transpose refreshed U's row statistics)
    make_padded_scalar(ctx, &FL);
    make_padded_scalar(ctx, &U);
  }
  trace_mark(ctx, "fsai block copies");
  F->tmp.alloc(n, st);
  if (precision == 32) {
    make_f32_values(ctx, &FL);
    make_f32_values(ctx, &U);
    F->tmp32.alloc(n, st);
  }
  DECO_CUDA(cudaStreamSynchronize(st));
  trace_mark(ctx, "fsai f32 copies");
}

}  // namespace deco

using namespace deco;

extern "C" {

int deco_fsai_create(deco_ctx ctx, deco_csr A, double tol_rel, double tol_abs, int power, int precision,
                     deco_fsai* out) {
  return guard([&] {
    DECO_REQUIRE(ctx && A && out, DECO_ERR_ARG, "NULL argument");
    auto* F = new deco_fsai_s();
    try {
      fsai_build(ctx, A, tol_rel, tol_abs, power, precision, F);
    } catch (...) {
      delete F;
      throw;
    }
    *out = F;
  });
}

int deco_fsai_destroy(deco_fsai F) {
  return guard([&] { delete F; });
}

int deco_fsai_info(deco_fsai F, int* n, int* nz, int* max_order) {
  return guard([&] {
    DECO_REQUIRE(F, DECO_ERR_ARG, "F is NULL");
    if (n) *n = F->n;
    if (nz) *nz = F->nz;
    if (max_order) *max_order = F->max_order;
  });
}

int deco_fsai_blocks(deco_fsai F, int* bs, int* nblk_lower, int* nblk_upper) {
  return guard([&] {
    DECO_REQUIRE(F, DECO_ERR_ARG, "F is NULL");
    if (bs) *bs = F->FL.bbs;
    if (nblk_lower) *nblk_lower = F->FL.nblk;
    if (nblk_upper) *nblk_upper = F->FUt.nblk;
  });
}

int deco_fsai_padded(deco_fsai F, int* slots_lower, int* slots_upper) {
  return guard([&] {
    DECO_REQUIRE(F, DECO_ERR_ARG, "F is NULL");
    if (slots_lower) *slots_lower = F->FL.ew;
    if (slots_upper) *slots_upper = F->FUt.ew;
  });
}

int deco_fsai_slot_codes(deco_fsai F, int* bytes_lower, int* bytes_upper) {
  return guard([&] {
    DECO_REQUIRE(F, DECO_ERR_ARG, "F is NULL");
    if (bytes_lower) *bytes_lower = !F->FL.ew ? 0 : (F->FL.eb ? F->FL.eb : 4);
    if (bytes_upper) *bytes_upper = !F->FUt.ew ? 0 : (F->FUt.eb ? F->FUt.eb : 4);
  });
}

int deco_fsai_download(deco_ctx ctx, deco_fsai F, int* Lr, int* Lc, double* Lv, int* Ur, int* Uc, double* Uv) {
  int rc = deco_csr_download(ctx, &F->FL, Lr, Lc, Lv);
  if (rc) return rc;
  return deco_csr_download(ctx, &F->FUt, Ur, Uc, Uv);
}

int deco_fsai_apply(deco_ctx ctx, deco_fsai F, const double* x, double* y) {
  return guard([&] {
    DECO_REQUIRE(ctx && F && x && y, DECO_ERR_ARG, "NULL argument");
    if (F->precision == 32) {
      spmv<float, double>(ctx, &F->FL, x, EpiStore<float>{F->tmp32.get()});
      spmv<float, float>(ctx, &F->FUt, F->tmp32.get(), EpiStore<double>{y});
    } else {
      fsai_apply_t<double, double, double>(ctx, F, x, F->tmp.get(), EpiStore<double>{y});
    }
  });
}

int deco_fsai_apply_f32(deco_ctx ctx, deco_fsai F, const float* x, float* y) {
  return guard([&] {
    DECO_REQUIRE(ctx && F && x && y, DECO_ERR_ARG, "NULL argument");
    DECO_REQUIRE(F->precision == 32, DECO_ERR_ARG, "deco_fsai_apply_f32 needs a factor made with precision 32");
    fsai_apply_t<float, float, float>(ctx, F, x, F->tmp32.get(), EpiStore<float>{y});
  });
}

}  // extern "C"
