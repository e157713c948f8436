// fsai.cuh — FSAI factor handle and the CSR utilities shared with the CPR setup.
#pragma once
#include "spmv.cuh"

struct deco_fsai_s {
  int n = 0, nz = 0, max_order = 0, precision = 64;
  deco_csr_s FL;    // lower factor, diagonal last in each row
  deco_csr_s FUt;   // FU stored transposed: upper CSR, rows ascending
  deco::DevBuf<double> tmp;   // intermediate FL x (float64 apply)
  deco::DevBuf<float> tmp32;  // intermediate FL x (float32 apply)
};

namespace deco {

// Filtered copy of A (core/CSR.hpp:423-525 applied as the FSAI constructor does,
// FSAI.hpp:22-28): keep |v| > |a_ii tol_rel| (if tol_rel != 0) and |v| > tol_abs
// (if tol_abs != 0); the diagonal always stays.  Writes a new matrix into out.
void csr_filter(deco_ctx_s* ctx, const deco_csr_s* A, double tol_rel, double tol_abs, deco_csr_s* out);

// In-place variant used by CPR (A->filter(tol_zero), Ap->filter_proper(tol)).
void csr_filter_inplace(deco_ctx_s* ctx, deco_csr_s* A, double tol_rel, double tol_abs);

// FSAI setup on a device matrix (the setup always runs in float64).
// bs > 1: the factors also get cell-block copies (make_bsr) for their products.
void fsai_build(deco_ctx_s* ctx, const deco_csr_s* A, double tol_rel, double tol_abs, int power, int precision,
                deco_fsai_s* F, int bs = 1);

// y = FU^T (FL x) with fused epilogue on the second product.
template <typename VT, typename XT, typename TT, class Epi>
void fsai_apply_t(deco_ctx_s* ctx, deco_fsai_s* F, const XT* x, TT* tmp, Epi epi) {
  spmv<VT, XT>(ctx, &F->FL, x, EpiStore<TT>{tmp});
  spmv<VT, TT>(ctx, &F->FUt, tmp, epi);
}

// T = A^T for the n x m CSR (r, c, v): atomic column scatter, then every row of
// T sorted by source row, so the result does not depend on scheduling.
void csr_transpose(deco_ctx_s* ctx, int n, int m, int nz, const int* r, const int* c, const double* v,
                   deco_csr_s* T);

void refresh_stats(deco_ctx_s* ctx, deco_csr_s* A);
void make_f32_values(deco_ctx_s* ctx, deco_csr_s* A);

}  // namespace deco
