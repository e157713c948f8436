// jacobi.cuh — point and block Jacobi (precond/Jacobi/Jacobi.hpp, Jacobi.tpp):
// the global stage of a CPR built with prec_glo.type "Jacobi", the first stage
// of apply_seq2 (CPR.hpp:202-233), and a local stage with prec_loc.type "Jacobi".
//
// Setup, one thread per cell: gather the bs x bs diagonal block exactly as
// Jacobi::blocked (Jacobi.tpp:26-69) and invert it with Gauss-Jordan elimination
// and partial pivoting (the reference calls LAPACK dgetrf + dgetri, so the
// inverses agree to rounding, not bit for bit); bs = 1 stores 1 / a_ii
// (Jacobi::classic, bit-exact).  Apply, one thread per cell: b = J x with the
// reference's summation order.  When the reference calls the apply in place
// (precond_glo(rt, rt) in apply_seq2/3), its row loop reads the already
// overwritten entries of the cell; ALIAS reproduces that.
#pragma once
#include "spmv.cuh"

struct deco_jacobi_s {
  int bs = 0, sn = 0, n = 0;
  deco::DevBuf<double> J;   // sn blocks of bs x bs, row-major B^{-1}
  deco::DevBuf<float> J32;
};

namespace deco {

// Builds J from the diagonal blocks of A; throws DECO_ERR_SINGULAR for a
// singular block.
void jacobi_build(deco_ctx_s* ctx, const deco_csr_s* A, int bs, int precision, deco_jacobi_s* J);

template <int BS, bool ALIAS, typename VT, typename XT, class Epi>
__global__ void jacobi_apply_kernel(int sn, const VT* __restrict__ J, const XT* x, Epi epi) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < sn; s += gridDim.x * blockDim.x) {
    const long long o = (long long)s * BS;
    double xv[BS];
#pragma unroll
    for (int k = 0; k < BS; ++k) xv[k] = (double)x[o + k];
    const VT* Jp = J + (long long)s * BS * BS;
#pragma unroll
    for (int p = 0; p < BS; ++p) {
      double sum = (double)Jp[p * BS] * xv[0];
#pragma unroll
      for (int k = 1; k < BS; ++k) sum += (double)Jp[p * BS + k] * xv[k];
      if (ALIAS) xv[p] = (double)(XT)sum;  // the in-place loop reads this row's new value next
      epi((int)(o + p), sum);
    }
  }
}

// epi(row, value) for every row: value = (J x)[row]; alias = true reproduces an
// in-place call of the reference.
template <typename VT, typename XT, class Epi>
void jacobi_apply(deco_ctx_s* ctx, const deco_jacobi_s* J, const XT* x, Epi epi, bool alias = false) {
  const VT* Jv;
  if constexpr (sizeof(VT) == 4) Jv = J->J32.get(); else Jv = J->J.get();
  const int g = grid_for(ctx, J->sn, 256);
  cudaStream_t st = ctx->stream;
#define DECO_JAC(BS)                                                                                          \
  do {                                                                                                        \
    if (alias) jacobi_apply_kernel<BS, true, VT, XT, Epi><<<g, 256, 0, st>>>(J->sn, Jv, x, epi);              \
    else jacobi_apply_kernel<BS, false, VT, XT, Epi><<<g, 256, 0, st>>>(J->sn, Jv, x, epi);                   \
  } while (0)
  switch (J->bs) {
    case 1: DECO_JAC(1); break;
    case 2: DECO_JAC(2); break;
    default: DECO_JAC(3); break;
  }
#undef DECO_JAC
  DECO_CHECK_LAUNCH();
}

}  // namespace deco
