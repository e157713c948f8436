// cpr.cu — CPR two-stage preconditioner on the device.
//
// Setup (precond/CPR.hpp:42-172).  Every decoupling step of the reference —
// fix_diag (:753-840), the quasi-IMPES(-GE) weights (:322-447), row scaling
// (core/alg.hpp:152-177), DRS (:518-600), IMPES (:450-516) and CPD (:603-750)
// — reads and writes only the rows of one cell, so they fuse into a single
// kernel with one thread per cell that applies them in the reference's order.
// The arithmetic is written as separately rounded operations in that order,
// so the decoupled matrix and right-hand side are bit-identical to the CPU
// oracle's.  Then: optional zero filter, A_pp extraction (core/CSR.hpp:338-420)
// and its relative filter, the global and local FSAI setups, and fix_diag undone.
//
// Apply (apply_seq3, :235-274) as 8 SpMV launches whose epilogues carry the
// vector work: restriction r[s*bs+p] - (A x)[s*bs], prolongation
// x[s*bs+p] += xp, residual r - A x, and the final x += FSAI(rt) accumulate
// straight into x, so rt is never written back.
#include <cmath>
#include <vector>

#include "cpr.cuh"

namespace deco {

namespace {

__device__ __forceinline__ int bsearch_le(const int* __restrict__ a, int lo, int hi, int target) {
  int mn = lo, mx = hi, mid = (lo + hi) >> 1;
  while (mx - mn > 1) {
    if (a[mid] > target) mx = mid; else mn = mid;
    mid = (mn + mx) >> 1;
  }
  return mid;
}

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double madd(double a, double b, double c) { return dadd(a, dmul(b, c)); }
__device__ __forceinline__ double msub(double a, double b, double c) { return dsub(a, dmul(b, c)); }

enum : int { ERR_NONE = 0, ERR_SINGULAR = 1, ERR_PATTERN = 2, ERR_BS = 3 };

struct DecoupleArgs {
  int sn, bs, pid, weights, use_drs, cpd;
  double e_dd, e_ps;
  const int* r;
  const int* c;
  double* v;
  double* b;
  double* w;
  double* w0;              // quasi-IMPES weights as computed (before the DRS reset)
  unsigned char* ops;      // per cell: bits 0-2 rows kept by DRS, bit 3 rows 1 and 2 swapped
  double* J;
  char* chk;
  int* err;
  int* nfixed;
};

// bs x bs LU with partial pivoting + solve of M w = rhs (column-major M):
// the dgesv of quasi_IMPES (CPR.hpp:364) as the CPU oracle restates it.
__device__ void small_lu_solve(int k, double* M, double* b) {
  int piv[3];
  for (int j = 0; j < k; ++j) {
    int p = j;
    double best = fabs(M[j + j * k]);
    for (int i = j + 1; i < k; ++i)
      if (fabs(M[i + j * k]) > best) { best = fabs(M[i + j * k]); p = i; }
    piv[j] = p;
    if (p != j)
      for (int t = 0; t < k; ++t) { double s = M[j + t * k]; M[j + t * k] = M[p + t * k]; M[p + t * k] = s; }
    double d = M[j + j * k];
    if (d != 0.0) {
      double inv = ddiv(1.0, d);
      for (int i = j + 1; i < k; ++i) M[i + j * k] = dmul(M[i + j * k], inv);
    }
    for (int t = j + 1; t < k; ++t) {
      double u = M[j + t * k];
      for (int i = j + 1; i < k; ++i) M[i + t * k] = msub(M[i + t * k], M[i + j * k], u);
    }
  }
  for (int j = 0; j < k; ++j)
    if (piv[j] != j) { double s = b[j]; b[j] = b[piv[j]]; b[piv[j]] = s; }
  for (int j = 0; j < k; ++j)
    for (int i = j + 1; i < k; ++i) b[i] = msub(b[i], M[i + j * k], b[j]);
  for (int j = k - 1; j >= 0; --j) {
    b[j] = ddiv(b[j], M[j + j * k]);
    for (int i = 0; i < j; ++i) b[i] = msub(b[i], M[i + j * k], b[j]);
  }
}

// Per-cell scratch arrays are written at positions that come from the data
// (column % bs); store_at spells such a write as an unrolled compare-and-select
// so that, with the block size a template constant, every array stays in
// registers (with a run-time bs they spilled to a 432-byte stack frame).
template <int N>
__device__ __forceinline__ void store_at(double* arr, int idx, double val) {
#pragma unroll
  for (int t = 0; t < N; ++t)
    if (t == idx) arr[t] = val;
}

// One cell of the decoupling: fix_diag -> weights -> row scaling -> DRS -> IMPES
// -> CPD in the reference's order.  r, c and v are the matrix's row pointers,
// columns and values, or a block's staged copy of its cells' rows (row pointers
// rebased to the copy); b and the per-cell outputs are always global.
template <int BS>
__device__ __forceinline__ void decouple_cell(const DecoupleArgs& a, int s, const int* __restrict__ r,
                                              const int* __restrict__ c, double* __restrict__ v) {
  const int bs = BS > 0 ? BS : a.bs;
  double* __restrict__ b = a.b;
  const int i0 = s * bs;
  // rows of a cell must share one pattern (IMPES/CPD work position by position)
  const int len = r[i0 + 1] - r[i0];
  for (int p = 1; p < bs; ++p)
    if (r[i0 + p + 1] - r[i0 + p] != len) { atomicExch(a.err, ERR_PATTERN); return; }

  // ---- fix_diag (CPR.hpp:753-840), small_tol = big_tol = 1e-20
  const double tol = 1e-20;
  unsigned char op = 0;
  {
    int j0 = bsearch_le(c, r[i0], r[i0 + 1], i0);
    if (fabs(v[j0]) < tol) { v[j0] = (v[j0] > 0) ? tol : -tol; a.chk[i0] = 1; atomicAdd(a.nfixed, 1); }
    if (bs == 3) {
      int j1 = bsearch_le(c, r[i0 + 1], r[i0 + 2], i0 + 1);
      int j2 = bsearch_le(c, r[i0 + 2], r[i0 + 3], i0 + 2);
      if (fabs(v[j1]) < tol || fabs(v[j2]) < tol) {
        if (fabs(v[j1 + 1]) > tol || fabs(v[j2 - 1]) > tol) {
          const int ia1 = r[i0 + 1], ib1 = r[i0 + 2];
          for (int t = 0; t < ib1 - ia1; ++t) { double x = v[ia1 + t]; v[ia1 + t] = v[ib1 + t]; v[ib1 + t] = x; }
          double x = b[i0 + 1]; b[i0 + 1] = b[i0 + 2]; b[i0 + 2] = x;
          op |= 8;
        } else {
          if (fabs(v[j1]) < tol) { v[j1] = (v[j1] > 0) ? tol : -tol; a.chk[i0 + 1] = 1; atomicAdd(a.nfixed, 1); }
          if (fabs(v[j2]) < tol) { v[j2] = (v[j2] > 0) ? tol : -tol; a.chk[i0 + 2] = 1; atomicAdd(a.nfixed, 1); }
        }
      }
    } else if (bs == 2) {
      int j1 = bsearch_le(c, r[i0 + 1], r[i0 + 2], i0 + 1);
      if (fabs(v[j1]) < tol) { v[j1] = (v[j1] > 0) ? tol : -tol; a.chk[i0 + 1] = 1; atomicAdd(a.nfixed, 1); }
    }
  }

  // ---- weights
  double w[3] = {1.0, 0.0, 0.0};
  if (a.weights == 2) {  // quasi_IMPES_GE (CPR.hpp:372-447), pressure id 0
    double Apb[4] = {0, 0, 0, 0}, bp[2] = {0, 0};
    for (int p = 0; p < bs; ++p) {
      const int i = i0 + p;
      const int j = bsearch_le(c, r[i], r[i + 1], i);
      for (int k = 1; k < bs; ++k) {
        if (p == 0) bp[k - 1] = -v[j + k - p];
        else store_at<4>(Apb, (p - 1) * (bs - 1) + c[j + k - p] % bs - 1, v[j + k - p]);
      }
    }
    if (bs == 3) {
      const double det = dsub(dmul(Apb[0], Apb[3]), dmul(Apb[1], Apb[2]));
      if (det == 0.0) { atomicExch(a.err, ERR_SINGULAR); return; }
      const double inv = ddiv(1.0, det);
      const double q0 = dmul(Apb[3], inv), q1 = dmul(-Apb[1], inv), q2 = dmul(-Apb[2], inv), q3 = dmul(Apb[0], inv);
      w[1] = dadd(dmul(q0, bp[0]), dmul(q2, bp[1]));
      w[2] = dadd(dmul(q1, bp[0]), dmul(q3, bp[1]));
    } else if (bs == 2) {
      if (Apb[0] == 0.0) { atomicExch(a.err, ERR_SINGULAR); return; }
      w[1] = ddiv(bp[0], Apb[0]);
    } else {
      atomicExch(a.err, ERR_BS);
      return;
    }
  } else if (a.weights == 1) {  // quasi_IMPES (CPR.hpp:322-369): B^T w = e_0
    double B[9];
    for (int t = 0; t < 9; ++t) B[t] = 0.0;
    for (int p = 0; p < bs; ++p) {
      const int i = i0 + p, ia = r[i], ib = r[i + 1];
      const int j = bsearch_le(c, ia, ib, i);
      if (c[j] != i) continue;
      for (int k = 0; k < bs; ++k) {
        const int q = j + k - p;
        if (q < ia || q >= ib) continue;
        if (c[q] / bs == s) store_at<9>(B, p * bs + c[q] % bs, v[q]);
      }
    }
    w[0] = 0.0; w[1] = 0.0; w[2] = 0.0;
    w[a.pid] = 1.0;
    small_lu_solve(bs, B, w);
  }
  for (int p = 0; p < bs; ++p) a.w0[i0 + p] = w[p];
  if (a.weights != 0) {
    for (int p = 0; p < bs; ++p) {
      const int i = i0 + p;
      for (int j = r[i]; j < r[i + 1]; ++j) v[j] = dmul(v[j], w[p]);
      b[i] = dmul(b[i], w[p]);
    }
  }

  // ---- DRS (CPR.hpp:518-600)
  bool wd[3] = {true, true, true};
  if (a.use_drs) {
    for (int p = 0; p < bs; ++p) {
      const int i = i0 + p, ia = r[i], ib = r[i + 1];
      const double diag = v[bsearch_le(c, ia, ib, i - p)];
      double off = -fabs(diag);
      for (int j = ia; j < ib; ++j) off = dadd(off, (c[j] % bs == 0) ? fabs(v[j]) : 0.0);
      wd[p] = !(diag < dmul(a.e_dd, off));
    }
    if (a.e_ps != 0.0) {
      const int ia = r[i0], ib = r[i0 + 1];
      const int jd = bsearch_le(c, ia, ib, i0);
      const double diag = fabs(v[jd]);
      double off[3] = {0.0, 0.0, 0.0};
      for (int j = ia; j < ib; ++j) {
        if (j == jd) continue;
        const int q = c[j] % bs;
#pragma unroll
        for (int t = 0; t < 3; ++t)
          if (t == q) off[t] = dadd(off[t], fabs(v[j]));
      }
      for (int p = 0; p < bs; ++p) wd[p] = wd[p] && !(off[p] < dmul(a.e_ps, diag));
    }
    wd[0] = true;
    if (a.weights != 0)
      for (int p = 0; p < bs; ++p)
        if (!wd[p]) {
          const int i = i0 + p;
          const double d = w[p];
          for (int j = r[i]; j < r[i + 1]; ++j) v[j] = ddiv(v[j], d);
          b[i] = ddiv(b[i], d);
          w[p] = 1.0;
        }
  }
  for (int p = 0; p < bs; ++p) a.w[i0 + p] = w[p];
  for (int p = 0; p < bs; ++p) op |= wd[p] ? (1 << p) : 0;
  a.ops[s] = op;

  // ---- IMPES (CPR.hpp:450-516): pressure row (offset 0) accumulates the others
  {
    const int ia0 = r[i0];
    for (int k = 0; k < bs; ++k) {
      const int ia = r[i0 + k], ib = r[i0 + k + 1];
      if (!a.use_drs) {
        if (k == 0) continue;
        for (int j = ia; j < ib; ++j) v[ia0 + (j - ia)] = dadd(v[ia0 + (j - ia)], v[j]);
      } else {
        const double ww = wd[k] ? 1.0 : 0.0;
        if (k == 0) {
          for (int j = ia; j < ib; ++j) v[j] = dmul(v[j], ww);
        } else {
          for (int j = ia; j < ib; ++j) v[ia0 + (j - ia)] = madd(v[ia0 + (j - ia)], ww, v[j]);
        }
      }
    }
    double sum = 0.0;
    for (int j = 0; j < bs; ++j) sum = madd(sum, a.use_drs ? (wd[j] ? 1.0 : 0.0) : 1.0, b[i0 + j]);
    b[i0] = sum;
  }

  // ---- CPD (CPR.hpp:603-750): J = diag(D) B^{-1}; rows and b of the cell <- J (.)
  if (a.cpd) {
    double B[9], Dp[3], o[9];
    for (int p = 0; p < bs; ++p) {
      const int i = i0 + p;
      const int j = bsearch_le(c, r[i], r[i + 1], i);
      Dp[p] = v[j];
      for (int k = 0; k < bs; ++k) store_at<9>(B, p * bs + c[j + k - p] % bs, v[j + k - p]);
    }
    if (bs == 3) {
      const double c0 = dsub(dmul(B[4], B[8]), dmul(B[5], B[7]));
      const double c1 = dsub(dmul(B[1], B[8]), dmul(B[2], B[7]));
      const double c2 = dsub(dmul(B[1], B[5]), dmul(B[2], B[4]));
      const double det = dadd(dsub(dmul(B[0], c0), dmul(B[3], c1)), dmul(B[6], c2));
      if (det == 0.0) { atomicExch(a.err, ERR_SINGULAR); return; }
      const double inv = ddiv(1.0, det);
      o[0] = dmul(dmul(c0, inv), Dp[0]);
      o[1] = dmul(dmul(-c1, inv), Dp[0]);
      o[2] = dmul(dmul(c2, inv), Dp[0]);
      o[3] = dmul(dmul(-dsub(dmul(B[3], B[8]), dmul(B[5], B[6])), inv), Dp[1]);
      o[4] = dmul(dmul(dsub(dmul(B[0], B[8]), dmul(B[2], B[6])), inv), Dp[1]);
      o[5] = dmul(dmul(-dsub(dmul(B[0], B[5]), dmul(B[2], B[3])), inv), Dp[1]);
      o[6] = dmul(dmul(dsub(dmul(B[3], B[7]), dmul(B[4], B[6])), inv), Dp[2]);
      o[7] = dmul(dmul(-dsub(dmul(B[0], B[7]), dmul(B[1], B[6])), inv), Dp[2]);
      o[8] = dmul(dmul(dsub(dmul(B[0], B[4]), dmul(B[1], B[3])), inv), Dp[2]);
    } else if (bs == 2) {
      const double det = dsub(dmul(B[0], B[3]), dmul(B[1], B[2]));
      if (det == 0.0) { atomicExch(a.err, ERR_SINGULAR); return; }
      const double inv = ddiv(1.0, det);
      o[0] = dmul(dmul(B[3], inv), Dp[0]);
      o[1] = dmul(dmul(-B[1], inv), Dp[0]);
      o[2] = dmul(dmul(-B[2], inv), Dp[1]);
      o[3] = dmul(dmul(B[0], inv), Dp[1]);
    } else {
      atomicExch(a.err, ERR_BS);
      return;
    }
    for (int t = 0; t < bs * bs; ++t) a.J[(long long)s * bs * bs + t] = o[t];
    // position by position: new row p = J[p,p] * row p + sum_{k != p} J[p,k] * row k
    for (int t = 0; t < len; ++t) {
      double old[3];
      for (int k = 0; k < bs; ++k) old[k] = v[r[i0 + k] + t];
      for (int p = 0; p < bs; ++p) {
        double nv = dmul(old[p], o[p * bs + p]);
        for (int k = 0; k < bs; ++k)
          if (k != p) nv = madd(nv, old[k], o[p * bs + k]);
        v[r[i0 + p] + t] = nv;
      }
    }
    double xb[3], sum[3];
    for (int k = 0; k < bs; ++k) xb[k] = b[i0 + k];
    for (int p = 0; p < bs; ++p) {
      sum[p] = 0.0;
      for (int j = 0; j < bs; ++j) sum[p] = madd(sum[p], o[p * bs + j], xb[j]);
    }
    for (int p = 0; p < bs; ++p) b[i0 + p] = sum[p];
  }
}

// Cells in groups of blockDim.x: each group's rows (row pointers, columns,
// values) are first staged in shared memory with coalesced loads, the cells run
// on the staged copy (their searches and row walks hit shared memory instead of
// dependent global loads), and the values go back with coalesced stores.  A group
// whose rows do not fit the staging space runs on global memory.
template <int BS>  // 2 or 3; 0: the block size from a.bs (at most 3)
__global__ void cpr_decouple(DecoupleArgs a, int stage_entries) {
  const int bs = BS > 0 ? BS : a.bs;
  extern __shared__ __align__(16) unsigned char dsm[];
  const int nb = blockDim.x;
  double* vs = reinterpret_cast<double*>(dsm);                 // stage_entries values
  int* cs = reinterpret_cast<int*>(vs + stage_entries);        // stage_entries columns
  int* rs = cs + stage_entries;                                 // nb * bs + 1 row pointers
  for (int base = blockIdx.x * nb; base < a.sn; base += gridDim.x * nb) {
    const int s = base + threadIdx.x;
    const int cend = min(base + nb, a.sn);
    const int row0 = base * bs, row1 = cend * bs;
    const int e0 = a.r[row0], ne = a.r[row1] - e0;
    const bool staged = ne <= stage_entries;  // the same for every thread of the block
    if (staged) {
      for (int t = threadIdx.x; t <= row1 - row0; t += nb) rs[t] = a.r[row0 + t] - e0;
      for (int t = threadIdx.x; t < ne; t += nb) {
        cs[t] = a.c[e0 + t];
        vs[t] = a.v[e0 + t];
      }
      __syncthreads();
      // row i of the group at rs[i - row0]; its entries at [rs[..], rs[.. + 1]) of cs / vs
      if (s < a.sn) decouple_cell<BS>(a, s, rs - row0, cs, vs);
      __syncthreads();
      for (int t = threadIdx.x; t < ne; t += nb) a.v[e0 + t] = vs[t];
      __syncthreads();  // the copy is read before the next group overwrites it
    } else if (s < a.sn) {
      decouple_cell<BS>(a, s, a.r, a.c, a.v);
    }
  }
}

// The right-hand-side half of cpr_decouple for a new vector: the same row
// operations of every cell (row swap, weights, DRS undo, IMPES sum, CPD), with
// the same separately rounded arithmetic in the same order, so a vector
// replayed here is bit-identical to one decoupled together with A.
__global__ void cpr_decouple_rhs(int sn, int bs, int weights, int use_drs, int cpd, const double* __restrict__ w0,
                                 const unsigned char* __restrict__ ops, const double* __restrict__ J,
                                 double* __restrict__ b) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < sn; s += gridDim.x * blockDim.x) {
    const long long i0 = (long long)s * bs;
    const unsigned op = ops[s];
    double x[3];
    for (int p = 0; p < bs; ++p) x[p] = b[i0 + p];
    if (op & 8) { double t = x[1]; x[1] = x[2]; x[2] = t; }
    if (weights != 0) {
      for (int p = 0; p < bs; ++p) x[p] = dmul(x[p], w0[i0 + p]);
      if (use_drs)
        for (int p = 0; p < bs; ++p)
          if (!(op & (1u << p))) x[p] = ddiv(x[p], w0[i0 + p]);
    }
    double sum = 0.0;
    for (int j = 0; j < bs; ++j) sum = madd(sum, use_drs ? ((op & (1u << j)) ? 1.0 : 0.0) : 1.0, x[j]);
    x[0] = sum;
    if (cpd) {
      const double* o = J + (long long)s * bs * bs;
      double y[3];
      for (int p = 0; p < bs; ++p) {
        y[p] = 0.0;
        for (int j = 0; j < bs; ++j) y[p] = madd(y[p], o[p * bs + j], x[j]);
      }
      for (int p = 0; p < bs; ++p) x[p] = y[p];
    }
    for (int p = 0; p < bs; ++p) b[i0 + p] = x[p];
  }
}

// e_k: 1 in row k of every cell, 0 elsewhere (column k of I, per cell)
__global__ void cpr_unit_column(long long n, int bs, int k, double* __restrict__ e) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    e[i] = (i % bs == k) ? 1.0 : 0.0;
}

// Per cell: T (column k = T e_k, from Tk), y = T^-1 r and z = T^-1 b by Gaussian
// elimination with partial pivoting; per-block sums of |y|^2 and |z|^2 in a fixed
// order (part[blockIdx.x], part[gridDim.x + blockIdx.x]).
__global__ void cpr_undecoupled_norms(int sn, int bs, const double* __restrict__ T0, const double* __restrict__ T1,
                                      const double* __restrict__ T2, const double* __restrict__ r,
                                      const double* __restrict__ b, double* __restrict__ part) {
  double sr = 0.0, sb = 0.0;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < sn; s += gridDim.x * blockDim.x) {
    const long long i0 = (long long)s * bs;
    double M[3][5];
    const double* Tk[3] = {T0, T1, T2};
    for (int i = 0; i < bs; ++i) {
      for (int k = 0; k < bs; ++k) M[i][k] = Tk[k][i0 + i];
      M[i][bs] = r[i0 + i];
      M[i][bs + 1] = b[i0 + i];
    }
    bool singular = false;
    for (int c = 0; c < bs; ++c) {
      int piv = c;
      for (int i = c + 1; i < bs; ++i)
        if (fabs(M[i][c]) > fabs(M[piv][c])) piv = i;
      if (M[piv][c] == 0.0) { singular = true; break; }
      if (piv != c)
        for (int k = 0; k < bs + 2; ++k) { const double t = M[c][k]; M[c][k] = M[piv][k]; M[piv][k] = t; }
      for (int i = 0; i < bs; ++i) {
        if (i == c) continue;
        const double f = M[i][c] / M[c][c];
        for (int k = c; k < bs + 2; ++k) M[i][k] -= f * M[c][k];
      }
    }
    if (singular) { sr = NAN; continue; }
    for (int i = 0; i < bs; ++i) {
      const double y = M[i][bs] / M[i][i], z = M[i][bs + 1] / M[i][i];
      sr += y * y;
      sb += z * z;
    }
  }
  __shared__ double ps[2][32];
  sr = warp_sum(sr);
  sb = warp_sum(sb);
  if ((threadIdx.x & 31) == 0) { ps[0][threadIdx.x >> 5] = sr; ps[1][threadIdx.x >> 5] = sb; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, c = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { a += ps[0][w]; c += ps[1][w]; }
    part[blockIdx.x] = a;
    part[gridDim.x + blockIdx.x] = c;
  }
}

__global__ void unfix_diag(int n, const int* __restrict__ r, const int* __restrict__ c, double* __restrict__ v,
                           const char* __restrict__ chk) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (chk[i]) v[bsearch_le(c, r[i], r[i + 1], i)] = 0.0;
}

// A_pp (core/CSR.hpp:338-420, weights == nullptr)
__global__ void local_count(int sn, int bs, int p, const int* __restrict__ r, const int* __restrict__ c,
                            int* __restrict__ cnt) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < sn; i += gridDim.x * blockDim.x) {
    int k = 0;
    for (int j = r[bs * i + p]; j < r[bs * i + p + 1]; ++j) k += (c[j] % bs == p);
    cnt[i] = k;
  }
}

__global__ void local_copy(int sn, int bs, int p, const int* __restrict__ r, const int* __restrict__ c,
                           const double* __restrict__ v, const int* __restrict__ lr, int* __restrict__ lc,
                           double* __restrict__ lv) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < sn; i += gridDim.x * blockDim.x) {
    int o = lr[i];
    for (int j = r[bs * i + p]; j < r[bs * i + p + 1]; ++j)
      if (c[j] % bs == p) { lc[o] = c[j] / bs; lv[o] = v[j]; ++o; }
  }
}

// seq1 helpers: rts[i] = r[i*bs+p];  x = 0 except x[i*bs+p] = xp[i];  x[i*bs+p] += xp[i]
template <typename RT, typename YT>
__global__ void gather_pressure(int sn, int bs, int p, const RT* __restrict__ r, YT* __restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < sn; i += gridDim.x * blockDim.x) y[i] = (YT)r[(long long)i * bs + p];
}
template <typename XT, typename PT>
__global__ void scatter_pressure(int n, int bs, int p, const PT* __restrict__ xp, XT* __restrict__ x, int add) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int q = i % bs;
    if (add) {
      if (q == p) x[i] = (XT)((double)x[i] + (double)xp[i / bs]);
    } else {
      x[i] = q == p ? (XT)xp[i / bs] : (XT)0;
    }
  }
}

struct Ev {
  deco_ctx_s* ctx;
  cudaEvent_t a, b;
  explicit Ev(deco_ctx_s* c) : ctx(c) {
    DECO_CUDA(cudaEventCreate(&a));
    DECO_CUDA(cudaEventCreate(&b));
    DECO_CUDA(cudaEventRecord(a, ctx->stream));
  }
  double stop() {
    DECO_CUDA(cudaEventRecord(b, ctx->stream));
    DECO_CUDA(cudaEventSynchronize(b));
    float ms = 0;
    DECO_CUDA(cudaEventElapsedTime(&ms, a, b));
    DECO_CUDA(cudaEventRecord(a, ctx->stream));
    return ms;
  }
  ~Ev() { cudaEventDestroy(a); cudaEventDestroy(b); }
};

}  // namespace

static void cpr_build(deco_ctx_s* ctx, deco_csr_s* A, double* d_b, const deco_cpr_params& prm, deco_cpr_s* P) {
  cudaStream_t st = ctx->stream;
  const int bs = prm.block_size;
  DECO_REQUIRE(bs == 2 || bs == 3, DECO_ERR_UNSUPPORTED, "block_size must be 2 or 3");
  DECO_REQUIRE(A->n == A->m, DECO_ERR_ARG, "CPR needs a square matrix");
  DECO_REQUIRE(A->n % bs == 0, DECO_ERR_ARG,
               "n is not divisible by bs, n = " + std::to_string(A->n) + ", bs = " + std::to_string(bs));
  DECO_REQUIRE(prm.pressure_id >= 0 && prm.pressure_id < bs, DECO_ERR_ARG, "pressure_id out of range");
  // quasi_IMPES_GE (CPR.hpp:372-447) fills its (bs-1)x(bs-1) system at index
  // (p - 1)(bs - 1) + column % bs - 1 for every row p != p_id and writes the
  // weights to rows 1..bs-1 of the cell: with p_id != 0 row 0 lands at a negative
  // index and the weight of row p_id is overwritten, so only p_id = 0 has a
  // defined result to reproduce
  DECO_REQUIRE(prm.weights != 2 || prm.pressure_id == 0, DECO_ERR_UNSUPPORTED,
               "quasiimpes_GE weights need pressure_id 0 (the reference's quasi_IMPES_GE indexes from row 0)");
  DECO_REQUIRE(prm.seq >= 0 && prm.seq <= 3, DECO_ERR_ARG, "seq must be 0, 1, 2 or 3");
  DECO_REQUIRE((prm.glo_type == 0 || prm.glo_type == 1) && (prm.loc_type == 0 || prm.loc_type == 1),
               DECO_ERR_UNSUPPORTED, "prec_glo / prec_loc type must be FSAI or Jacobi on the GPU path");
  DECO_REQUIRE(prm.weights >= 0 && prm.weights <= 2, DECO_ERR_ARG, "weights must be 0, 1 or 2");
  DECO_REQUIRE(prm.precision == 64 || prm.precision == 32, DECO_ERR_ARG, "precision must be 64 or 32");
  P->prm = prm;
  P->A = A;
  P->n = A->n;
  P->bs = bs;
  P->p = prm.pressure_id;
  P->sn = A->n / bs;
  Ev ev(ctx);
  P->J.alloc((size_t)P->sn * bs * bs, st);
  P->w.alloc(P->n, st);
  P->w0.alloc(P->n, st);
  P->ops.alloc(P->sn, st);
  P->check_diag.alloc(P->n, st);
  P->check_diag.zero(st);
  DevBuf<int> flags(2, st);
  flags.zero(st);
  DecoupleArgs a;
  a.sn = P->sn; a.bs = bs; a.pid = P->p; a.weights = prm.weights; a.use_drs = prm.use_drs; a.cpd = prm.cpd;
  a.e_dd = prm.drs_e_dd; a.e_ps = prm.drs_e_ps;
  a.r = A->r.get(); a.c = A->c.get(); a.v = A->v.get(); a.b = d_b;
  a.w = P->w.get(); a.w0 = P->w0.get(); a.ops = P->ops.get(); a.J = P->J.get(); a.chk = P->check_diag.get(); a.err = flags.get(); a.nfixed = flags.get() + 1;
  // groups of 128 cells (64 for bs 3) staged in 64 KB of shared memory: 3.6k
  // entries for a 7-point bs-2 group, about 4.6k for bs 3, room for 5.3k
  const int nbk = bs == 3 ? 64 : 128;
  const size_t dsmem = 64 * 1024;
  const int stage_entries = (int)((dsmem - sizeof(int) * ((size_t)nbk * bs + 1)) / (sizeof(double) + sizeof(int)));
  auto go = [&](auto kern) {
    DECO_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsmem));
    kern<<<grid_for(ctx, P->sn, nbk, 16), nbk, dsmem, st>>>(a, stage_entries);
  };
  if (bs == 2) go(cpr_decouple<2>);
  else if (bs == 3) go(cpr_decouple<3>);
  else go(cpr_decouple<0>);
  DECO_CHECK_LAUNCH();
  int hf[2];
  DECO_CUDA(cudaMemcpyAsync(hf, flags.get(), sizeof(hf), cudaMemcpyDeviceToHost, st));
  DECO_CUDA(cudaStreamSynchronize(st));
  DECO_REQUIRE(hf[0] != ERR_SINGULAR, DECO_ERR_SINGULAR, "determinant is zero in CPD decoupling");
  DECO_REQUIRE(hf[0] != ERR_PATTERN, DECO_ERR_PATTERN, "rows of a cell do not share one column pattern");
  DECO_REQUIRE(hf[0] == ERR_NONE, DECO_ERR_UNSUPPORTED, "unknown block size CPD decoupling");
  P->fixed = hf[1];
  if (prm.tol_zero != 0.0) csr_filter_inplace(ctx, A, 0.0, prm.tol_zero);
  P->t_ms[0] = ev.stop();
  // A_pp
  {
    DevBuf<int> cnt(P->sn + 1, st);
    const int g = grid_for(ctx, P->sn, 256);
    local_count<<<g, 256, 0, st>>>(P->sn, bs, P->p, A->r.get(), A->c.get(), cnt.get());
    DECO_CHECK_LAUNCH();
    P->Ap.n = P->Ap.m = P->sn;
    P->Ap.r.alloc(P->sn + 1, st);
    P->Ap.nz = (int)exclusive_scan_int(ctx, cnt.get(), P->Ap.r.get(), P->sn);
    P->Ap.c.alloc(P->Ap.nz, st);
    P->Ap.v.alloc(P->Ap.nz, st);
    local_copy<<<g, 256, 0, st>>>(P->sn, bs, P->p, A->r.get(), A->c.get(), A->v.get(), P->Ap.r.get(), P->Ap.c.get(),
                                  P->Ap.v.get());
    DECO_CHECK_LAUNCH();
    refresh_stats(ctx, &P->Ap);
    if (prm.loc_tol_rel > 1e-20) csr_filter_inplace(ctx, &P->Ap, prm.loc_tol_rel, 0.0);
  }
  P->t_ms[1] = ev.stop();
  const int jbs = prm.glo_block_size > 0 ? prm.glo_block_size : bs;
  if (prm.glo_type == 1) jacobi_build(ctx, A, jbs, prm.precision, &P->jac);
  else fsai_build(ctx, A, prm.glo_tol_rel, prm.glo_tol_abs, prm.glo_power, prm.precision, &P->glo, bs);
  P->t_ms[2] = ev.stop();
  if (prm.loc_type == 1)
    jacobi_build(ctx, &P->Ap, prm.loc_block_size > 0 ? prm.loc_block_size : 1, prm.precision, &P->jloc);
  else fsai_build(ctx, &P->Ap, prm.loc_tol_rel, prm.loc_tol_abs, prm.loc_power, prm.precision, &P->loc);
  P->t_ms[3] = ev.stop();
  // seq 2 with an FSAI global stage also builds the Jacobi of prec_glo (CPR.hpp:154-162)
  if (prm.seq == 2 && prm.glo_type == 0) jacobi_build(ctx, A, jbs, prm.precision, &P->jac);
  P->t_ms[0] += ev.stop();
  if (P->fixed)
    unfix_diag<<<grid_for(ctx, P->n, 256), 256, 0, st>>>(P->n, A->r.get(), A->c.get(), A->v.get(),
                                                         P->check_diag.get());
  DECO_CHECK_LAUNCH();
  P->rt.alloc(P->n, st);
  P->rts.alloc(P->sn, st);
  make_bsr(ctx, A, bs);
  if (prm.precision == 32) {
    make_f32_values(ctx, A);
    P->rt32.alloc(P->n, st);
    P->rts32.alloc(P->sn, st);
  }
  // choose SpMV widths now, outside any later graph capture
  tuned_subwarp(ctx, A, false);
  if (prm.precision == 32) tuned_subwarp(ctx, A, true);
  for (deco_csr_s* M : {&P->glo.FL, &P->glo.FUt, &P->loc.FL, &P->loc.FUt})
    if (M->n) tuned_subwarp(ctx, M, prm.precision == 32);
  for (deco_csr_s* M : {A, &P->glo.FL, &P->glo.FUt})
    if (M->bbs) {
      tuned_bsr_subwarp(ctx, M, false);
      if (prm.precision == 32) tuned_bsr_subwarp(ctx, M, true);
    }
  // then which product each matrix takes (slot-padded, cell blocks or CSR)
  for (deco_csr_s* M : {A, &P->glo.FL, &P->glo.FUt, &P->loc.FL, &P->loc.FUt})
    if (M->n) {
      tune_product_plan(ctx, M, false);
      if (prm.precision == 32) tune_product_plan(ctx, M, true);
    }
  DECO_CUDA(cudaStreamSynchronize(st));
  P->t_ms[4] = P->t_ms[0] + P->t_ms[1] + P->t_ms[2] + P->t_ms[3] + ev.stop();
}

// The global stage (FSAI, or Jacobi with prec_glo.type Jacobi) and the local
// stage (FSAI or Jacobi on A_pp): epi(row, value) with value = (M in)[row].
// alias: the reference calls this stage in place (precond_glo(rt, rt)).
template <typename VT, typename XT, typename TT, class Epi>
void glo_stage(deco_ctx_s* ctx, deco_cpr_s* P, const XT* in, TT* tmp, Epi epi, bool alias = false) {
  if (P->prm.glo_type == 1) jacobi_apply<VT, XT>(ctx, &P->jac, in, epi, alias);
  else fsai_apply_t<VT, XT, TT>(ctx, &P->glo, in, tmp, epi);
}
template <typename VT, typename XT, typename TT, class Epi>
void loc_stage(deco_ctx_s* ctx, deco_cpr_s* P, const XT* in, TT* tmp, Epi epi) {
  if (P->prm.loc_type == 1) jacobi_apply<VT, XT>(ctx, &P->jloc, in, epi);
  else fsai_apply_t<VT, XT, TT>(ctx, &P->loc, in, tmp, epi);
}

void cpr_apply64(deco_ctx_s* ctx, deco_cpr_s* P, const double* r, double* x) {
  deco_csr_s* A = P->A;
  const int bs = P->bs, p = P->p;
  if (P->prm.seq == 1) {
    cudaStream_t st = ctx->stream;
    gather_pressure<double, double><<<grid_for(ctx, P->sn, 256), 256, 0, st>>>(P->sn, bs, p, r, P->rts.get());
    DECO_CHECK_LAUNCH();
    loc_stage<double, double, double>(ctx, P, P->rts.get(), P->loc.tmp.get(), EpiStore<double>{P->rts.get()});
    scatter_pressure<double, double><<<grid_for(ctx, P->n, 256), 256, 0, st>>>(P->n, bs, p, P->rts.get(), x, 0);
    DECO_CHECK_LAUNCH();
    spmv<double, double>(ctx, A, x, EpiResid<double, double>{r, P->rt.get()});
    glo_stage<double, double, double>(ctx, P, P->rt.get(), P->glo.tmp.get(), EpiStore<double>{x});
    scatter_pressure<double, double><<<grid_for(ctx, P->n, 256), 256, 0, st>>>(P->n, bs, p, P->rts.get(), x, 1);
    DECO_CHECK_LAUNCH();
    return;
  }
  // seq 3 (and its first half, seq 0); seq 2 starts with the Jacobi stage
  if (P->prm.seq == 2) jacobi_apply<double, double>(ctx, &P->jac, r, EpiStore<double>{x});
  else glo_stage<double, double, double>(ctx, P, r, P->glo.tmp.get(), EpiStore<double>{x});
  spmv<double, double>(ctx, A, x, EpiRestrict<double, double>{r, P->rts.get(), bs, p}, bs);
  loc_stage<double, double, double>(ctx, P, P->rts.get(), P->loc.tmp.get(), EpiProlong<double>{x, bs, p});
  if (P->prm.seq == 0) return;
  spmv<double, double>(ctx, A, x, EpiResid<double, double>{r, P->rt.get()});
  glo_stage<double, double, double>(ctx, P, P->rt.get(), P->glo.tmp.get(), EpiAdd<double>{x}, true);
}

template <typename RT, typename XT>
void cpr_apply32(deco_ctx_s* ctx, deco_cpr_s* P, const RT* r, XT* x) {
  deco_csr_s* A = P->A;
  const int bs = P->bs, p = P->p;
  float* tg = P->glo.tmp32.get();
  float* tl = P->loc.tmp32.get();
  if (P->prm.seq == 1) {
    cudaStream_t st = ctx->stream;
    gather_pressure<RT, float><<<grid_for(ctx, P->sn, 256), 256, 0, st>>>(P->sn, bs, p, r, P->rts32.get());
    DECO_CHECK_LAUNCH();
    loc_stage<float, float, float>(ctx, P, P->rts32.get(), tl, EpiStore<float>{P->rts32.get()});
    scatter_pressure<XT, float><<<grid_for(ctx, P->n, 256), 256, 0, st>>>(P->n, bs, p, P->rts32.get(), x, 0);
    DECO_CHECK_LAUNCH();
    spmv<float, XT>(ctx, A, x, EpiResid<RT, float>{r, P->rt32.get()});
    glo_stage<float, float, float>(ctx, P, P->rt32.get(), tg, EpiStore<XT>{x});
    scatter_pressure<XT, float><<<grid_for(ctx, P->n, 256), 256, 0, st>>>(P->n, bs, p, P->rts32.get(), x, 1);
    DECO_CHECK_LAUNCH();
    return;
  }
  if (P->prm.seq == 2) jacobi_apply<float, RT>(ctx, &P->jac, r, EpiStore<XT>{x});
  else glo_stage<float, RT, float>(ctx, P, r, tg, EpiStore<XT>{x});
  spmv<float, XT>(ctx, A, x, EpiRestrict<RT, float>{r, P->rts32.get(), bs, p}, bs);
  loc_stage<float, float, float>(ctx, P, P->rts32.get(), tl, EpiProlong<XT>{x, bs, p});
  if (P->prm.seq == 0) return;
  spmv<float, XT>(ctx, A, x, EpiResid<RT, float>{r, P->rt32.get()});
  glo_stage<float, float, float>(ctx, P, P->rt32.get(), tg, EpiAdd<XT>{x}, true);
}

double cpr_original_relres(deco_ctx_s* ctx, deco_cpr_s* P, const double* r, const double* b) {
  cudaStream_t st = ctx->stream;
  const int bs = P->bs;
  const long long n = P->n;
  const deco_cpr_params& m = P->prm;
  DevBuf<double> Tk[3];
  for (int k = 0; k < bs; ++k) {
    Tk[k].alloc(n, st);
    cpr_unit_column<<<grid_for(ctx, n, 256), 256, 0, st>>>(n, bs, k, Tk[k].get());
    DECO_CHECK_LAUNCH();
    cpr_decouple_rhs<<<grid_for(ctx, P->sn, 256), 256, 0, st>>>(P->sn, bs, m.weights, m.use_drs, m.cpd, P->w0.get(),
                                                                P->ops.get(), P->J.get(), Tk[k].get());
    DECO_CHECK_LAUNCH();
  }
  const int grid = grid_for(ctx, P->sn, 256);
  DevBuf<double> part(2 * (size_t)grid, st);
  cpr_undecoupled_norms<<<grid, 256, 0, st>>>(P->sn, bs, Tk[0].get(), bs > 1 ? Tk[1].get() : nullptr,
                                              bs > 2 ? Tk[2].get() : nullptr, r, b, part.get());
  DECO_CHECK_LAUNCH();
  std::vector<double> h(2 * (size_t)grid);
  DECO_CUDA(cudaMemcpyAsync(h.data(), part.get(), sizeof(double) * h.size(), cudaMemcpyDeviceToHost, st));
  DECO_CUDA(cudaStreamSynchronize(st));
  double sr = 0.0, sb = 0.0;
  for (int i = 0; i < grid; ++i) { sr += h[i]; sb += h[grid + i]; }
  return std::sqrt(sr) / std::sqrt(sb);
}

template void cpr_apply32<double, double>(deco_ctx_s*, deco_cpr_s*, const double*, double*);
template void cpr_apply32<double, float>(deco_ctx_s*, deco_cpr_s*, const double*, float*);
template void cpr_apply32<float, float>(deco_ctx_s*, deco_cpr_s*, const float*, float*);

}  // namespace deco

using namespace deco;

extern "C" {

int deco_cpr_create(deco_ctx ctx, deco_csr A, double* d_b, const deco_cpr_params* prm, deco_cpr* out) {
  return guard([&] {
    DECO_REQUIRE(ctx && A && d_b && prm && out, DECO_ERR_ARG, "NULL argument");
    auto* P = new deco_cpr_s();
    try {
      cpr_build(ctx, A, d_b, *prm, P);
    } catch (...) {
      delete P;
      throw;
    }
    *out = P;
  });
}

int deco_cpr_destroy(deco_cpr P) {
  return guard([&] { delete P; });
}

int deco_cpr_apply(deco_ctx ctx, deco_cpr P, const double* r, double* x) {
  return guard([&] {
    DECO_REQUIRE(ctx && P && r && x, DECO_ERR_ARG, "NULL argument");
    DECO_REQUIRE(r != x, DECO_ERR_ARG, "r and x must not alias");
    if (P->prm.precision == 32) cpr_apply32<double, double>(ctx, P, r, x);
    else cpr_apply64(ctx, P, r, x);
  });
}

int deco_cpr_pressure(deco_cpr P, deco_csr* Ap) {
  return guard([&] {
    DECO_REQUIRE(P && Ap, DECO_ERR_ARG, "NULL argument");
    *Ap = &P->Ap;
  });
}

int deco_cpr_fsai(deco_cpr P, int which, deco_fsai* F) {
  return guard([&] {
    DECO_REQUIRE(P && F && (which == 0 || which == 1), DECO_ERR_ARG, "bad argument");
    DECO_REQUIRE((which == 0 ? P->prm.glo_type : P->prm.loc_type) == 0, DECO_ERR_ARG,
                 "that stage is a Jacobi preconditioner, not an FSAI");
    *F = which == 0 ? &P->glo : &P->loc;
  });
}

int deco_cpr_timings(deco_cpr P, double* ms5) {
  return guard([&] {
    DECO_REQUIRE(P && ms5, DECO_ERR_ARG, "NULL argument");
    for (int i = 0; i < 5; ++i) ms5[i] = P->t_ms[i];
  });
}

int deco_cpr_decouple_rhs(deco_ctx ctx, deco_cpr P, double* d_b) {
  return guard([&] {
    DECO_REQUIRE(ctx && P && d_b, DECO_ERR_ARG, "NULL argument");
    const deco_cpr_params& m = P->prm;
    cpr_decouple_rhs<<<grid_for(ctx, P->sn, 256), 256, 0, ctx->stream>>>(
        P->sn, P->bs, m.weights, m.use_drs, m.cpd, P->w0.get(), P->ops.get(), P->J.get(), d_b);
    DECO_CHECK_LAUNCH();
  });
}

int deco_cpr_fixed_diagonals(deco_cpr P, int* count) {
  return guard([&] {
    DECO_REQUIRE(P && count, DECO_ERR_ARG, "NULL argument");
    *count = P->fixed;
  });
}

}  // extern "C"
