/* deco_oracle.c — plain-C restatement of the reference's CPR-Krylov hot path.
 * TEST INFRASTRUCTURE ONLY (see deco_oracle.h).  Scalar, single-threaded,
 * written for clarity: every function names the reference lines it follows. */
#include "deco_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ALLOC(T, n) ((T*)calloc((size_t)((n) > 0 ? (n) : 1), sizeof(T)))

void orc_csr_free(orc_csr* A) {
  free(A->r); free(A->c); free(A->v);
  A->r = NULL; A->c = NULL; A->v = NULL;
}

static orc_csr csr_copy(const orc_csr* A) {
  orc_csr B = *A;
  B.r = ALLOC(int, A->n + 1); B.c = ALLOC(int, A->nz); B.v = ALLOC(double, A->nz);
  memcpy(B.r, A->r, sizeof(int) * (A->n + 1));
  memcpy(B.c, A->c, sizeof(int) * A->nz);
  memcpy(B.v, A->v, sizeof(double) * A->nz);
  return B;
}

/* core/alg.hpp:16-25 (core::binarysearch): index of the last element <= target in
 * [lo, hi) by bisection; returns lo when every element is larger. */
static int bsearch_le(const int* a, int lo, int hi, int target) {
  int mn = lo, mx = hi, mid = (lo + hi) >> 1;
  while (mx - mn > 1) {
    if (a[mid] > target) mx = mid; else mn = mid;
    mid = (mn + mx) >> 1;
  }
  return mid;
}

/* core/alg.hpp:50-64: b[i/bs] = sum_j v[j] x[c[j]] for rows i = 0, bs, 2bs, ... */
void orc_spmv(int n, const int* r, const int* c, const double* v, const double* x, double* y, int bs) {
  for (int i = 0; i < n; i += bs) {
    double s = 0.0;
    for (int j = r[i]; j < r[i + 1]; ++j) s += v[j] * x[c[j]];
    y[i / bs] = s;
  }
}

/* core/CSR.hpp:423-473 (filter: keep |v| > tol) and :476-525 (filter_proper: keep
 * |v| > |a_ii * tol|); the diagonal (col == row + shift) is always kept. */
int orc_filter(orc_csr* A, double tol, int relative, int shift) {
  int* rp = ALLOC(int, A->n + 1);
  int* cp = ALLOC(int, A->nz);
  double* vp = ALLOC(double, A->nz);
  int nz = 0;
  rp[0] = 0;
  for (int i = 0; i < A->n; ++i) {
    double D = tol;
    if (relative) D = fabs(A->v[bsearch_le(A->c, A->r[i], A->r[i + 1], i + shift)] * tol);
    for (int j = A->r[i]; j < A->r[i + 1]; ++j)
      if (fabs(A->v[j]) > D || A->c[j] == i + shift) { cp[nz] = A->c[j]; vp[nz] = A->v[j]; ++nz; }
    rp[i + 1] = nz;
  }
  free(A->r); free(A->c); free(A->v);
  A->r = rp; A->c = cp; A->v = vp; A->nz = nz;
  return 0;
}

static int cmp_int(const void* a, const void* b) {
  int x = *(const int*)a, y = *(const int*)b;
  return (x > y) - (x < y);
}

/* precond/FSAI/symbolic.tpp:101-176.  Power 1: lower(A) including the diagonal,
 * scanning each sorted row up to the first column > i.  Power 2: lower(A*A) as a
 * sorted set of columns (the reference builds it with a hash table and a radix
 * sort, which yields the same sorted unique set). */
static int fsai_symbolic(const orc_csr* A, int power, orc_csr* F) {
  const int n = A->n;
  F->n = n; F->m = A->m;
  F->r = ALLOC(int, n + 1);
  if (power == 1) {
    for (int i = 0; i < n; ++i) {
      int k = 0;
      for (int j = A->r[i]; j < A->r[i + 1] && A->c[j] <= i; ++j) ++k;
      F->r[i + 1] = F->r[i] + k;
    }
    F->nz = F->r[n];
    F->c = ALLOC(int, F->nz);
    for (int i = 0; i < n; ++i) {
      int o = F->r[i];
      for (int j = A->r[i]; j < A->r[i + 1] && A->c[j] <= i; ++j) F->c[o++] = A->c[j];
    }
  } else if (power == 2) {
    int cap = 64, *buf = ALLOC(int, cap);
    int** rows = ALLOC(int*, n);
    for (int i = 0; i < n; ++i) {
      int m = 0;
      for (int j = A->r[i]; j < A->r[i + 1]; ++j) {
        int cA = A->c[j];
        for (int k = A->r[cA]; k < A->r[cA + 1]; ++k) {
          int key = A->c[k];
          if (key > i) break;
          if (m == cap) { cap *= 2; buf = (int*)realloc(buf, sizeof(int) * cap); }
          buf[m++] = key;
        }
      }
      qsort(buf, m, sizeof(int), cmp_int);
      int u = 0;
      for (int t = 0; t < m; ++t)
        if (u == 0 || buf[t] != buf[u - 1]) buf[u++] = buf[t];
      rows[i] = ALLOC(int, u + 1);
      rows[i][0] = u;
      memcpy(rows[i] + 1, buf, sizeof(int) * u);
      F->r[i + 1] = F->r[i] + u;
    }
    F->nz = F->r[n];
    F->c = ALLOC(int, F->nz);
    for (int i = 0; i < n; ++i) {
      memcpy(F->c + F->r[i], rows[i] + 1, sizeof(int) * rows[i][0]);
      free(rows[i]);
    }
    free(rows); free(buf);
  } else {
    return -1;
  }
  F->v = ALLOC(double, F->nz);
  return 0;
}

/* LU with partial pivoting of a column-major k x k matrix M (Golub & Van Loan,
 * Algorithm 3.4.1, outer-product form): the factorisation LAPACK dgetrf returns,
 * pivot = first index of the largest |entry| in the column. */
static void lu_factor(int k, double* M, int* piv) {
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
      double inv = 1.0 / d;
      for (int i = j + 1; i < k; ++i) M[i + j * k] *= inv;
    }
    for (int t = j + 1; t < k; ++t) {
      double u = M[j + t * k];
      for (int i = j + 1; i < k; ++i) M[i + t * k] -= M[i + j * k] * u;
    }
  }
}

/* Solve M x = b ('N') from the factors (dgetrs 'N'): P, then L (unit), then U. */
static void lu_solve_n(int k, const double* M, const int* piv, double* b) {
  for (int j = 0; j < k; ++j)
    if (piv[j] != j) { double s = b[j]; b[j] = b[piv[j]]; b[piv[j]] = s; }
  for (int j = 0; j < k; ++j)
    for (int i = j + 1; i < k; ++i) b[i] -= M[i + j * k] * b[j];
  for (int j = k - 1; j >= 0; --j) {
    b[j] /= M[j + j * k];
    for (int i = 0; i < j; ++i) b[i] -= M[i + j * k] * b[j];
  }
}

/* Solve M^T x = b ('T') from the factors (dgetrs 'T'): U^T, then unit L^T, then P^T. */
static void lu_solve_t(int k, const double* M, const int* piv, double* b) {
  for (int j = 0; j < k; ++j) {
    double s = b[j];
    for (int i = 0; i < j; ++i) s -= M[i + j * k] * b[i];
    b[j] = s / M[j + j * k];
  }
  for (int j = k - 1; j >= 0; --j) {
    double s = b[j];
    for (int i = j + 1; i < k; ++i) s -= M[i + j * k] * b[i];
    b[j] = s;
  }
  for (int j = k - 1; j >= 0; --j)
    if (piv[j] != j) { double s = b[j]; b[j] = b[piv[j]]; b[piv[j]] = s; }
}

/* position of `key` in the sorted pattern P[0..k), or -1 */
static int find_pos(const int* P, int k, int key) {
  int lo = 0, hi = k - 1;
  while (lo <= hi) {
    int mid = (lo + hi) >> 1;
    if (P[mid] == key) return mid;
    if (P[mid] < key) lo = mid + 1; else hi = mid - 1;
  }
  return -1;
}

/* precond/FSAI/numeric.tpp:59-133 with gather.cpp:14-88, LU_main.cpp:14-48,
 * scatter numeric.tpp:33-54, MxM_diag diagonal.cpp:6-52, Jacobi_scale
 * diagonal.cpp:57-73.  Row i with pattern P (the row minus its last entry d, the
 * diagonal) and order k = |P|:
 *   M = A[P,P]^T (the reference stores A[P,P] row-major and LAPACK reads it as
 *   column-major), LU(M);  fU: M^T fU = -A[P,d];  fL: M fL = -A[d,P]^T.
 * Rows are independent, so the reference's descending-size processing order
 * (sorting.hpp:214-239) does not change any value. */
static void fsai_numeric(const orc_csr* A, orc_csr* FL, orc_csr* FU) {
  const int n = A->n;
  int kmax = 0;
  for (int i = 0; i < n; ++i) { int k = FL->r[i + 1] - FL->r[i] - 1; if (k > kmax) kmax = k; }
  double* M = ALLOC(double, kmax * kmax);
  double* rl = ALLOC(double, kmax);
  double* ru = ALLOC(double, kmax);
  int* piv = ALLOC(int, kmax);
  for (int i = 0; i < n; ++i) {
    const int a = FL->r[i], e = FL->r[i + 1] - 1, k = e - a;
    if (k <= 0) continue;
    const int* P = FL->c + a;
    const int d = FL->c[e];
    memset(M, 0, sizeof(double) * k * k);
    memset(rl, 0, sizeof(double) * k);
    memset(ru, 0, sizeof(double) * k);
    for (int row = 0; row < k; ++row) {
      const int g = P[row];
      for (int s = A->r[g]; s < A->r[g + 1]; ++s) {
        int col = find_pos(P, k, A->c[s]);
        if (col >= 0) M[col + row * k] = A->v[s];  /* M(col,row) = A(P[row],P[col]) */
      }
      int j = bsearch_le(A->c, A->r[g], A->r[g + 1], d);
      if (A->c[j] == d) ru[row] = -A->v[j];
    }
    for (int s = A->r[d]; s < A->r[d + 1]; ++s) {
      int col = find_pos(P, k, A->c[s]);
      if (col >= 0) rl[col] = -A->v[s];
    }
    lu_factor(k, M, piv);
    lu_solve_t(k, M, piv, ru);
    lu_solve_n(k, M, piv, rl);
    for (int t = 0; t < k; ++t) { FL->v[a + t] = rl[t]; FU->v[a + t] = ru[t]; }
  }
  free(M); free(rl); free(ru); free(piv);

  double* D = ALLOC(double, n);
  for (int i = 0; i < n; ++i) { FL->v[FL->r[i + 1] - 1] = 1.0; FU->v[FL->r[i + 1] - 1] = 1.0; }
  for (int i = 0; i < n; ++i) {
    const int aF = FL->r[i], bF = FL->r[i + 1];
    double sum = 0.0;
    for (int j = aF; j < bF; ++j) {
      double fl = FL->v[j];
      if (fl != 0.0) {
        int colF = FL->c[j], pa = A->r[colF], pb = A->r[colF + 1], pu = aF;
        double s = 0.0;
        while (pa < pb && pu < bF) {
          if (A->c[pa] == FL->c[pu]) { s += A->v[pa] * FU->v[pu]; ++pa; ++pu; }
          else if (A->c[pa] < FL->c[pu]) ++pa;
          else ++pu;
        }
        sum += fl * s;
      }
    }
    D[i] = (sum < 0.0) ? (-1.0 / sqrt(fabs(sum))) : (1.0 / sqrt(sum));
  }
  for (int i = 0; i < n; ++i) {
    double dd = D[i], da = fabs(dd);
    for (int j = FL->r[i]; j < FL->r[i + 1]; ++j) { FL->v[j] *= dd; FU->v[j] *= da; }
  }
  free(D);
}

/* core/CSR.hpp:151-211 (trans_mat_full): counting-sort transpose; within each
 * output row the entries keep ascending source-row order. */
static void csr_transpose(orc_csr* F) {
  const int n = F->n;
  int* rt = ALLOC(int, n + 1);
  int* ct = ALLOC(int, F->nz);
  double* vt = ALLOC(double, F->nz);
  for (int j = 0; j < F->nz; ++j) rt[F->c[j] + 1]++;
  for (int i = 0; i < n; ++i) rt[i + 1] += rt[i];
  int* pos = ALLOC(int, n);
  memcpy(pos, rt, sizeof(int) * n);
  for (int i = 0; i < n; ++i)
    for (int j = F->r[i]; j < F->r[i + 1]; ++j) {
      int k = pos[F->c[j]]++;
      ct[k] = i; vt[k] = F->v[j];
    }
  free(pos);
  free(F->r); free(F->c); free(F->v);
  F->r = rt; F->c = ct; F->v = vt;
}

/* precond/FSAI/FSAI.hpp:14-37 + FSAI.tpp:10-32: optional filtered copy
 * (filter_proper(tol_rel) then filter(tol_abs)), symbolic, numeric, then FU is
 * transposed into an upper CSR. */
int orc_fsai_setup(const orc_csr* A0, double tol_rel, double tol_abs, int power, orc_fsai* F) {
  orc_csr A = csr_copy(A0);
  if (tol_rel != 0.0) orc_filter(&A, tol_rel, 1, 0);
  if (tol_abs != 0.0) orc_filter(&A, tol_abs, 0, 0);
  memset(F, 0, sizeof(*F));
  int rc = fsai_symbolic(&A, power, &F->FL);
  if (rc) { orc_csr_free(&A); return rc; }
  F->FU = F->FL;
  F->FU.r = ALLOC(int, A.n + 1); F->FU.c = ALLOC(int, F->FL.nz); F->FU.v = ALLOC(double, F->FL.nz);
  memcpy(F->FU.r, F->FL.r, sizeof(int) * (A.n + 1));
  memcpy(F->FU.c, F->FL.c, sizeof(int) * F->FL.nz);
  fsai_numeric(&A, &F->FL, &F->FU);
  csr_transpose(&F->FU);
  orc_csr_free(&A);
  return 0;
}

/* precond/FSAI/FSAI.hpp:40-47: temp = FL x; y = FU^T temp (x may alias y). */
void orc_fsai_apply(const orc_fsai* F, const double* x, double* tmp, double* y) {
  orc_spmv(F->FL.n, F->FL.r, F->FL.c, F->FL.v, x, tmp, 1);
  orc_spmv(F->FU.n, F->FU.r, F->FU.c, F->FU.v, tmp, y, 1);
}

void orc_fsai_free(orc_fsai* F) { orc_csr_free(&F->FL); orc_csr_free(&F->FU); }

/* ---------------------------------------------------------------- CPR setup */

/* precond/CPR.hpp:753-840 (fix_diag) with small_tol = big_tol = 1e-20 (:76). */
static char* fix_diag(orc_csr* A, double* b, int bs, double small_tol, double big_tol) {
  char* chk = ALLOC(char, A->n);
  const int sn = A->n / bs;
  int *Ar = A->r, *Ac = A->c;
  double* Av = A->v;
  for (int s = 0; s < sn; ++s) {
    int i = s * bs;
    int j0 = bsearch_le(Ac, Ar[i], Ar[i + 1], i);
    if (fabs(Av[j0]) < small_tol) { Av[j0] = (Av[j0] > 0) ? small_tol : -small_tol; chk[i] = 1; }
    if (bs == 3) {
      int j1 = bsearch_le(Ac, Ar[i + 1], Ar[i + 2], i + 1);
      int j2 = bsearch_le(Ac, Ar[i + 2], Ar[i + 3], i + 2);
      if (fabs(Av[j1]) < small_tol || fabs(Av[j2]) < small_tol) {
        if (fabs(Av[j1 + 1]) > small_tol || fabs(Av[j2 - 1]) > small_tol) {
          /* swap the values of rows i+1 and i+2 (same pattern) and of b */
          int ia1 = Ar[i + 1], ib1 = Ar[i + 2];
          for (int t = 0; t < ib1 - ia1; ++t) { double x = Av[ia1 + t]; Av[ia1 + t] = Av[ib1 + t]; Av[ib1 + t] = x; }
          double x = b[i + 1]; b[i + 1] = b[i + 2]; b[i + 2] = x;
        } else {
          if (fabs(Av[j1]) < small_tol) { Av[j1] = (Av[j1] > 0) ? big_tol : -big_tol; chk[i + 1] = 1; }
          if (fabs(Av[j2]) < small_tol) { Av[j2] = (Av[j2] > 0) ? big_tol : -big_tol; chk[i + 2] = 1; }
        }
      }
    } else if (bs == 2) {
      int j1 = bsearch_le(Ac, Ar[i + 1], Ar[i + 2], i + 1);
      if (fabs(Av[j1]) < small_tol) { Av[j1] = (Av[j1] > 0) ? big_tol : -big_tol; chk[i + 1] = 1; }
    }
  }
  return chk;
}

/* precond/CPR.hpp:842-855: entries fixed above are set back to zero */
static void unfix_diag(orc_csr* A, const char* chk) {
  for (int i = 0; i < A->n; ++i)
    if (chk[i]) A->v[bsearch_le(A->c, A->r[i], A->r[i + 1], i)] = 0.0;
}

/* precond/CPR.hpp:372-447 (quasi_IMPES_GE), pressure id 0: w_p = 1 and
 * w_s = A_ss^{-T} (-A_ps^T) from the cell's diagonal block. */
static int quasi_impes_ge(const orc_csr* A, int bs, double* w) {
  const int sn = A->n / bs, bs1 = bs - 1;
  for (int s = 0; s < sn; ++s) {
    double Ap[4] = {0, 0, 0, 0}, bp[2] = {0, 0};
    for (int p = 0; p < bs; ++p) {
      int i = s * bs + p;
      int j = bsearch_le(A->c, A->r[i], A->r[i + 1], i);
      for (int k = 1; k < bs; ++k) {
        if (p == 0) bp[k - 1] = -A->v[j + k - p];
        else Ap[(p - 1) * bs1 + (A->c[j + k - p]) % bs - 1] = A->v[j + k - p];
      }
    }
    w[s * bs] = 1.0;
    if (bs1 == 2) {
      double det = Ap[0] * Ap[3] - Ap[1] * Ap[2];
      if (det == 0.0) return -10;
      double inv = 1.0 / det;
      double i0 = Ap[3] * inv, i1 = -Ap[1] * inv, i2 = -Ap[2] * inv, i3 = Ap[0] * inv;
      w[s * bs + 1] = i0 * bp[0] + i2 * bp[1];
      w[s * bs + 2] = i1 * bp[0] + i3 * bp[1];
    } else if (bs1 == 1) {
      if (Ap[0] == 0.0) return -10;
      w[s * bs + 1] = bp[0] / Ap[0];
    } else {
      return -11;
    }
  }
  return 0;
}

/* precond/CPR.hpp:322-369 (quasi_IMPES): w = B^{-T} e_p per cell, B the diagonal block. */
static int quasi_impes(const orc_csr* A, int bs, int pid, double* w) {
  const int sn = A->n / bs;
  double B[9];
  int piv[3];
  memset(w, 0, sizeof(double) * A->n);
  for (int s = 0; s < sn; ++s) {
    memset(B, 0, sizeof(B));
    for (int p = 0; p < bs; ++p) {
      int i = s * bs + p, ia = A->r[i], ib = A->r[i + 1];
      int j = bsearch_le(A->c, ia, ib, i);
      if (A->c[j] != i) continue;
      for (int k = 0; k < bs; ++k) {
        int q = j + k - p;
        if (q < ia || q >= ib) continue;
        if (A->c[q] / bs == s) B[p * bs + A->c[q] % bs] = A->v[q];
      }
    }
    /* LAPACK reads the row-major B as column-major, i.e. solves B^T w = e_p */
    double* ws = w + s * bs;
    ws[pid] = 1.0;
    lu_factor(bs, B, piv);
    lu_solve_n(bs, B, piv, ws);
  }
  return 0;
}

/* precond/CPR.hpp:518-584 (drs_weights) */
static char* drs_weights(const orc_csr* A, int bs, double e_dd, double e_ps) {
  const int sn = A->n / bs;
  char* w = ALLOC(char, A->n);
  for (int s = 0; s < sn; ++s)
    for (int p = 0; p < bs; ++p) {
      int i = s * bs + p, ia = A->r[i], ib = A->r[i + 1];
      double diag = A->v[bsearch_le(A->c, ia, ib, i - p)];
      double off = -fabs(diag);
      for (int j = ia; j < ib; ++j) off += (A->c[j] % bs == 0) ? fabs(A->v[j]) : 0.0;
      w[i] = (diag < e_dd * off) ? 0 : 1;
    }
  if (e_ps != 0.0) {
    double off[3];
    for (int s = 0; s < sn; ++s) {
      int i = s * bs, ia = A->r[i], ib = A->r[i + 1];
      int jd = bsearch_le(A->c, ia, ib, i);
      double diag = fabs(A->v[jd]);
      for (int p = 0; p < bs; ++p) off[p] = 0.0;
      for (int j = ia; j < ib; ++j) {
        if (j == jd) continue;
        off[A->c[j] % bs] += fabs(A->v[j]);
      }
      for (int p = 0; p < bs; ++p) w[i + p] &= (off[p] < e_ps * diag) ? 0 : 1;
    }
  }
  for (int s = 0; s < sn; ++s) w[s * bs] = 1;
  return w;
}

/* precond/CPR.hpp:603-685 (CPD_build): J = diag(D) B^{-1} per cell */
static int cpd_build(const orc_csr* A, int bs, double* vj) {
  const int sn = A->n / bs;
  for (int s = 0; s < sn; ++s) {
    double B[9], Dp[3];
    for (int p = 0; p < bs; ++p) {
      int i = s * bs + p;
      int j = bsearch_le(A->c, A->r[i], A->r[i + 1], i);
      Dp[p] = A->v[j];
      for (int k = 0; k < bs; ++k) B[p * bs + A->c[j + k - p] % bs] = A->v[j + k - p];
    }
    double* o = vj + (size_t)s * bs * bs;
    if (bs == 3) {
      double det = B[0] * (B[4] * B[8] - B[5] * B[7]) - B[3] * (B[1] * B[8] - B[2] * B[7]) +
                   B[6] * (B[1] * B[5] - B[2] * B[4]);
      if (det == 0.0) return -10;
      double inv = 1.0 / det;
      o[0] = (B[4] * B[8] - B[5] * B[7]) * inv * Dp[0];
      o[1] = -(B[1] * B[8] - B[2] * B[7]) * inv * Dp[0];
      o[2] = (B[1] * B[5] - B[2] * B[4]) * inv * Dp[0];
      o[3] = -(B[3] * B[8] - B[5] * B[6]) * inv * Dp[1];
      o[4] = (B[0] * B[8] - B[2] * B[6]) * inv * Dp[1];
      o[5] = -(B[0] * B[5] - B[2] * B[3]) * inv * Dp[1];
      o[6] = (B[3] * B[7] - B[4] * B[6]) * inv * Dp[2];
      o[7] = -(B[0] * B[7] - B[1] * B[6]) * inv * Dp[2];
      o[8] = (B[0] * B[4] - B[1] * B[3]) * inv * Dp[2];
    } else if (bs == 2) {
      double det = B[0] * B[3] - B[1] * B[2];
      if (det == 0.0) return -10;
      double inv = 1.0 / det;
      o[0] = B[3] * inv * Dp[0];
      o[1] = -B[1] * inv * Dp[0];
      o[2] = -B[2] * inv * Dp[1];
      o[3] = B[0] * inv * Dp[1];
    } else {
      return -11;
    }
  }
  return 0;
}

/* precond/CPR.hpp:688-726 (CPD_apply on the matrix): row p of each cell becomes
 * sum_k J[p,k] * (old row k), position by position (the rows share a pattern). */
static void cpd_apply_mat(const double* vj, orc_csr* A, int bs) {
  const int sn = A->n / bs;
  double* scr = ALLOC(double, A->nz);
  memcpy(scr, A->v, sizeof(double) * A->nz);
  for (int s = 0; s < sn; ++s)
    for (int p = 0; p < bs; ++p) {
      int i = s * bs + p;
      const double* J = vj + (size_t)s * bs * bs + p * bs;
      int ia = A->r[i], ib = A->r[i + 1];
      double* table = A->v + ia;
      for (int j = ia; j < ib; ++j) A->v[j] *= J[p];
      for (int k = 0; k < bs; ++k) {
        if (k == p) continue;
        int r0 = A->r[s * bs + k], r1 = A->r[s * bs + k + 1];
        for (int j = r0; j < r1; ++j) table[j - r0] += scr[j] * J[k];
      }
    }
  free(scr);
}

/* precond/CPR.hpp:730-750 (CPD_apply on a vector) */
static void cpd_apply_vec(const double* vj, double* x, int n, int bs) {
  double sum[3];
  for (int s = 0; s < n / bs; ++s) {
    for (int p = 0; p < bs; ++p) {
      sum[p] = 0.0;
      for (int j = 0; j < bs; ++j) sum[p] += vj[(size_t)(s * bs + p) * bs + j] * x[s * bs + j];
    }
    for (int p = 0; p < bs; ++p) x[s * bs + p] = sum[p];
  }
}

/* precond/CPR.hpp:450-471 and :475-516 (IMPES): the pressure row (offset 0, the
 * default argument at both call sites :104-105) accumulates the other rows of its
 * cell, optionally weighted by the DRS mask. */
static void impes_mat(orc_csr* A, int bs, const char* wd) {
  const int sn = A->n / bs;
  for (int s = 0; s < sn; ++s) {
    double* table = A->v + A->r[s * bs];
    for (int k = 0; k < bs; ++k) {
      int i = s * bs + k, ia = A->r[i], ib = A->r[i + 1];
      if (!wd) {
        if (k == 0) continue;
        for (int j = ia; j < ib; ++j) table[j - ia] += A->v[j];
      } else {
        double w = wd[i] ? 1.0 : 0.0;
        if (k == 0) { for (int j = ia; j < ib; ++j) A->v[j] *= w; }
        else { for (int j = ia; j < ib; ++j) table[j - ia] += w * A->v[j]; }
      }
    }
  }
}

static void impes_vec(double* x, int n, int bs, const char* wd) {
  for (int s = 0; s < n / bs; ++s) {
    double sum = 0.0;
    for (int j = 0; j < bs; ++j) sum += (wd ? (wd[s * bs + j] ? 1.0 : 0.0) : 1.0) * x[s * bs + j];
    x[s * bs] = sum;
  }
}

/* core/CSR.hpp:338-420 (local_matrix, no unscaling): rows s*bs+p, columns with
 * c % bs == p, mapped to c / bs. */
static orc_csr local_matrix(const orc_csr* A, int bs, int p) {
  orc_csr L;
  L.n = A->n / bs; L.m = A->m / bs;
  L.r = ALLOC(int, L.n + 1);
  for (int i = 0; i < L.n; ++i) {
    int k = 0;
    for (int j = A->r[bs * i + p]; j < A->r[bs * i + p + 1]; ++j) k += (A->c[j] % bs == p);
    L.r[i + 1] = L.r[i] + k;
  }
  L.nz = L.r[L.n];
  L.c = ALLOC(int, L.nz); L.v = ALLOC(double, L.nz);
  for (int i = 0; i < L.n; ++i) {
    int o = L.r[i];
    for (int j = A->r[bs * i + p]; j < A->r[bs * i + p + 1]; ++j)
      if (A->c[j] % bs == p) { L.c[o] = A->c[j] / bs; L.v[o] = A->v[j]; ++o; }
  }
  return L;
}

/* precond/CPR.hpp:42-172 (the CPR constructor), in its order. */
int orc_cpr_setup(const orc_cpr_params* prm, int n, const int* r, const int* c, const double* v,
                  const double* b, orc_cpr** out) {
  const int bs = prm->bs;
  if (bs < 1 || n % bs) return -1;
  orc_cpr* P = ALLOC(orc_cpr, 1);
  P->prm = *prm;
  P->n = n; P->sn = n / bs;
  orc_csr A0 = {n, n, r[n], (int*)r, (int*)c, (double*)v};
  P->A = csr_copy(&A0);
  P->b = ALLOC(double, n);
  memcpy(P->b, b, sizeof(double) * n);
  orc_csr* A = &P->A;
  int rc = 0;

  P->check_diag = fix_diag(A, P->b, bs, 1e-20, 1e-20);
  P->w = ALLOC(double, n);
  if (prm->weights == 2) rc = quasi_impes_ge(A, bs, P->w);
  else if (prm->weights == 1) rc = quasi_impes(A, bs, prm->p, P->w);
  if (rc) { orc_cpr_free(P); return rc; }
  if (prm->weights != 0) {
    for (int i = 0; i < n; ++i)
      for (int j = A->r[i]; j < A->r[i + 1]; ++j) A->v[j] *= P->w[i];
    for (int i = 0; i < n; ++i) P->b[i] *= P->w[i];
  }
  char* wd = NULL;
  if (prm->use_drs) {
    wd = drs_weights(A, bs, prm->e_dd, prm->e_ps);
    if (prm->weights != 0)
      for (int i = 0; i < n; ++i)
        if (!wd[i]) {
          double d = P->w[i];
          for (int j = A->r[i]; j < A->r[i + 1]; ++j) A->v[j] /= d;
          P->b[i] /= d;
          P->w[i] = 1.0;
        }
  }
  impes_mat(A, bs, wd);
  impes_vec(P->b, n, bs, wd);
  free(wd);
  if (prm->cpd) {
    P->J = ALLOC(double, (size_t)P->sn * bs * bs);
    rc = cpd_build(A, bs, P->J);
    if (rc) { orc_cpr_free(P); return rc; }
    cpd_apply_mat(P->J, A, bs);
    cpd_apply_vec(P->J, P->b, n, bs);
  }
  if (prm->tol_zero != 0.0) orc_filter(A, prm->tol_zero, 0, 0);
  P->Ap = local_matrix(A, bs, prm->p);
  if (prm->loc_tol_rel > 1e-20) orc_filter(&P->Ap, prm->loc_tol_rel, 1, 0);
  rc = orc_fsai_setup(A, prm->glo_tol_rel, prm->glo_tol_abs, prm->glo_power, &P->glo);
  if (!rc) rc = orc_fsai_setup(&P->Ap, prm->loc_tol_rel, prm->loc_tol_abs, prm->loc_power, &P->loc);
  if (rc) { orc_cpr_free(P); return rc; }
  unfix_diag(A, P->check_diag);
  P->xp = ALLOC(double, P->sn);
  P->rt = ALLOC(double, n);
  P->tmp_g = ALLOC(double, n);
  P->tmp_l = ALLOC(double, P->sn);
  *out = P;
  return 0;
}

/* precond/CPR.hpp:176-299: the apply sequences (seq 2 needs block Jacobi and is
 * not restated). */
void orc_cpr_apply(orc_cpr* P, const double* r, double* x) {
  const int n = P->n, sn = P->sn, bs = P->prm.bs, p = P->prm.p;
  orc_csr* A = &P->A;
  double *rt = P->rt, *xp = P->xp;
  switch (P->prm.seq) {
    case 1:
      for (int i = 0; i < sn; ++i) rt[i] = r[i * bs + p];
      orc_fsai_apply(&P->loc, rt, P->tmp_l, xp);
      memset(x, 0, sizeof(double) * n);
      for (int i = 0; i < sn; ++i) x[i * bs + p] = xp[i];
      orc_spmv(n, A->r, A->c, A->v, x, rt, 1);
      for (int i = 0; i < n; ++i) rt[i] = r[i] - rt[i];
      orc_fsai_apply(&P->glo, rt, P->tmp_g, x);
      for (int i = 0; i < sn; ++i) x[i * bs + p] += xp[i];
      return;
    case 0:
    case 3:
    default:
      orc_fsai_apply(&P->glo, r, P->tmp_g, x);
      orc_spmv(n, A->r, A->c, A->v, x, rt, bs);
      for (int i = 0; i < sn; ++i) rt[i] = r[i * bs + p] - rt[i];
      orc_fsai_apply(&P->loc, rt, P->tmp_l, xp);
      for (int i = 0; i < sn; ++i) x[i * bs + p] += xp[i];
      if (P->prm.seq == 0) return;
      orc_spmv(n, A->r, A->c, A->v, x, rt, 1);
      for (int i = 0; i < n; ++i) rt[i] = r[i] - rt[i];
      orc_fsai_apply(&P->glo, rt, P->tmp_g, rt);
      for (int i = 0; i < n; ++i) x[i] += rt[i];
      return;
  }
}

void orc_cpr_free(orc_cpr* P) {
  if (!P) return;
  orc_csr_free(&P->A); orc_csr_free(&P->Ap);
  orc_fsai_free(&P->glo); orc_fsai_free(&P->loc);
  free(P->b); free(P->w); free(P->J); free(P->xp); free(P->rt); free(P->tmp_g); free(P->tmp_l);
  free(P->check_diag);
  free(P);
}

/* ------------------------------------------------------------------- GMRES */

static double dot(int n, const double* a, const double* b) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

/* solver/rgmres.tpp:141-154 */
static void givens_make(double x, double y, double* c, double* s) {
  if (fabs(y) < 2.220446049250312e-16) { *c = 1.0; *s = 0.0; }
  else if (fabs(y) > fabs(x)) { double nu = x / y; *s = 1.0 / sqrt(1.0 + nu * nu); *c = nu * *s; }
  else { double nu = y / x; *c = 1.0 / sqrt(1.0 + nu * nu); *s = nu * *c; }
}
/* solver/rgmres.tpp:156-160 */
static void givens_apply(double c, double s, double* dx, double* dy) {
  double t = c * *dx + s * *dy;
  *dy = -s * *dx + c * *dy;
  *dx = t;
}

/* solver/rgmres.tpp:8-139 (left = 0) and solver/lgmres.tpp:1-134 (left = 1):
 * restarted GMRES(m) with modified Gram-Schmidt, Givens rotations, back
 * substitution and a true (or preconditioned) residual at every restart.
 * `itmax` counts inner iterations; x starts at zero. */
int orc_gmres(orc_cpr* P, int left, double tol, int m, int itmax, double* x, int* iter_out,
              double* res_abs, double* res_rel, int* flag_out, double* resvec) {
  const int n = P->n;
  orc_csr* A = &P->A;
  const double* b = P->b;
  double* r = ALLOC(double, n);
  double* z = ALLOC(double, n);
  double* w = ALLOC(double, n);
  double* V = ALLOC(double, (size_t)n * (m + 1));
  double* H = ALLOC(double, (size_t)(m + 1) * m);
  double* g = ALLOC(double, m + 1);
  double* cs = ALLOC(double, m + 1);
  double* sn = ALLOC(double, m + 1);
#define HH(i, j) H[(i) + (size_t)(j) * (m + 1)]
  int flag = 1, iter = 0;
  memset(x, 0, sizeof(double) * n);
  double bnorm, rnorm = 0.0;
  if (!left) {
    bnorm = sqrt(dot(n, b, b));
    memcpy(r, b, sizeof(double) * n);
  } else {
    orc_cpr_apply(P, b, r);
    bnorm = sqrt(dot(n, r, r));
  }
  const double abstol = tol * bnorm;
  while (iter < itmax) {
    memset(H, 0, sizeof(double) * (m + 1) * m);
    memset(g, 0, sizeof(double) * (m + 1));
    memset(cs, 0, sizeof(double) * (m + 1));
    memset(sn, 0, sizeof(double) * (m + 1));
    g[0] = sqrt(dot(n, r, r));
    for (int i = 0; i < n; ++i) V[i] = (1.0 / g[0]) * r[i];
    int j = 0;
    while (j < m && iter < itmax) {
      rnorm = fabs(g[j]);
      if (resvec) resvec[iter] = rnorm / bnorm;
      if (rnorm < abstol) { flag = 0; break; }
      double* vj = V + (size_t)j * n;
      if (!left) {
        orc_cpr_apply(P, vj, z);
        orc_spmv(n, A->r, A->c, A->v, z, w, 1);
      } else {
        orc_spmv(n, A->r, A->c, A->v, vj, z, 1);
        orc_cpr_apply(P, z, w);
      }
      for (int i = 0; i <= j; ++i) {
        double h = dot(n, V + (size_t)i * n, w);
        HH(i, j) = h;
        const double* vi = V + (size_t)i * n;
        for (int t = 0; t < n; ++t) w[t] = 1.0 * w[t] + (-h) * vi[t];
      }
      HH(j + 1, j) = sqrt(dot(n, w, w));
      double* vn = V + (size_t)(j + 1) * n;
      for (int t = 0; t < n; ++t) vn[t] = (1.0 / HH(j + 1, j)) * w[t];
      for (int i = 0; i <= j - 1; ++i) givens_apply(cs[i], sn[i], &HH(i, j), &HH(i + 1, j));
      givens_make(HH(j, j), HH(j + 1, j), &cs[j], &sn[j]);
      givens_apply(cs[j], sn[j], &HH(j, j), &HH(j + 1, j));
      givens_apply(cs[j], sn[j], &g[j], &g[j + 1]);
      ++j; ++iter;
    }
    for (int i = j - 1; i >= 0; --i) {
      if (HH(i, i) == 0.0) { flag = -2; goto done; }
      g[i] /= HH(i, i);
      for (int k = 0; k < i; ++k) g[k] -= HH(k, i) * g[i];
    }
    for (int t = 0; t < n; ++t) w[t] = g[0] * V[t];
    for (int i = 1; i < j; ++i) {
      const double* vi = V + (size_t)i * n;
      for (int t = 0; t < n; ++t) w[t] = 1.0 * w[t] + g[i] * vi[t];
    }
    if (!left) {
      orc_cpr_apply(P, w, z);
      for (int t = 0; t < n; ++t) x[t] += z[t];
      orc_spmv(n, A->r, A->c, A->v, x, r, 1);
      for (int t = 0; t < n; ++t) r[t] = b[t] - r[t];
    } else {
      for (int t = 0; t < n; ++t) x[t] += w[t];
      orc_spmv(n, A->r, A->c, A->v, x, z, 1);
      for (int t = 0; t < n; ++t) z[t] = b[t] - z[t];
      orc_cpr_apply(P, z, r);
    }
    rnorm = sqrt(dot(n, r, r));
    if (rnorm < abstol) { flag = 0; break; }
  }
done:
  *res_abs = rnorm;
  *res_rel = rnorm / bnorm;
  *iter_out = iter;
  *flag_out = flag;
  free(r); free(z); free(w); free(V); free(H); free(g); free(cs); free(sn);
#undef HH
  return 0;
}

int orc_cpr_sizes(const orc_cpr* P, long long* o) {
  o[0] = P->A.nz; o[1] = P->Ap.n; o[2] = P->Ap.nz; o[3] = P->glo.FL.nz; o[4] = P->loc.FL.nz;
  return 0;
}

/* which: 0 = decoupled A, 1 = A_pp, 2 = global FSAI (FL, FU^T), 3 = pressure FSAI */
void orc_cpr_get(const orc_cpr* P, int which, int* r, int* c, double* v, int* r2, int* c2, double* v2) {
  const orc_csr *X = NULL, *Y = NULL;
  if (which == 0) X = &P->A;
  else if (which == 1) X = &P->Ap;
  else if (which == 2) { X = &P->glo.FL; Y = &P->glo.FU; }
  else { X = &P->loc.FL; Y = &P->loc.FU; }
  memcpy(r, X->r, sizeof(int) * (X->n + 1));
  memcpy(c, X->c, sizeof(int) * X->nz);
  memcpy(v, X->v, sizeof(double) * X->nz);
  if (Y && r2) {
    memcpy(r2, Y->r, sizeof(int) * (Y->n + 1));
    memcpy(c2, Y->c, sizeof(int) * Y->nz);
    memcpy(v2, Y->v, sizeof(double) * Y->nz);
  }
}

void orc_cpr_get_b(const orc_cpr* P, double* b) { memcpy(b, P->b, sizeof(double) * P->n); }
