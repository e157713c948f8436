// adjoint.cu — differentiation of the CPR-GMRES solve x = A^{-1} b.
//
// No counterpart in the reference, which only solves forward.  For a loss L(x)
// with g = dL/dx:
//   A^T lambda = g,   dL/db = lambda,   dL/dA_ij = -lambda_i x_j  (on A's pattern).
// The adjoint system is the transpose of the ORIGINAL matrix, decoupled per cell
// by its own CPR setup (transpose first, then decouple): the transpose of a
// decoupled matrix has singular cell blocks for the decoupling, while A^T keeps
// the block structure of a reservoir matrix with its cell blocks transposed.
// Because CPR decouples by left-multiplying with a block-diagonal matrix T,
// the GMRES solve of T A^T lambda = T g returns the adjoint lambda itself.
// Every right-hand side g is decoupled by replaying the recorded row operations
// (deco_cpr_decouple_rhs), so one setup serves any number of adjoint solves.
//
// The gradient kernel is a streaming pass over A's pattern: per stored entry it
// reads a 4-byte column index, gathers x (the stencil keeps it in L2) and
// writes one 8-byte value; lambda_i is loaded once per row.
#include "cpr.cuh"

struct deco_adjoint_s {
  deco_csr_s At;                  // A^T, decoupled in place by P
  deco_cpr_s* P = nullptr;        // CPR of the transposed system
  deco::DevBuf<double> rhs;       // decoupled right-hand side of the current solve
  ~deco_adjoint_s() { deco_cpr_destroy(P); }
};

namespace deco {

namespace {

// A sub-warp of SW lanes per row; lanes stride over the row's entries.
template <int SW>
__global__ void grad_pattern(int n, const int* __restrict__ r, const int* __restrict__ c,
                             const double* __restrict__ lam, const double* __restrict__ x, double alpha,
                             double* __restrict__ grad) {
  const int lane = threadIdx.x % SW;
  const long long groups = (long long)gridDim.x * (blockDim.x / SW);
  for (long long i = (long long)blockIdx.x * (blockDim.x / SW) + threadIdx.x / SW; i < n; i += groups) {
    const double a = alpha;
    const double li = lam[i];
    const int e = r[i + 1];
    for (int j = r[i] + lane; j < e; j += SW) __stcs(grad + j, a * (li * __ldg(x + __ldcs(c + j))));
  }
}

}  // namespace

}  // namespace deco

using namespace deco;

extern "C" {

int deco_csr_transpose(deco_ctx ctx, deco_csr A, deco_csr* At) {
  return guard([&] {
    DECO_REQUIRE(ctx && A && At, DECO_ERR_ARG, "NULL argument");
    auto* T = new deco_csr_s();
    try {
      csr_transpose(ctx, A->n, A->m, A->nz, A->r.get(), A->c.get(), A->v.get(), T);
    } catch (...) {
      delete T;
      throw;
    }
    *At = T;
  });
}

int deco_grad_A_pattern(deco_ctx ctx, deco_csr A, const double* d_lambda, const double* d_x, double alpha,
                        double* d_grad) {
  return guard([&] {
    DECO_REQUIRE(ctx && A && d_lambda && d_x && d_grad, DECO_ERR_ARG, "NULL argument");
    if (A->n == 0) return;
    const int block = 256;
    if (A->avg_row > 12.0) {
      grad_pattern<16><<<grid_for(ctx, (long long)A->n * 16, block), block, 0, ctx->stream>>>(
          A->n, A->r.get(), A->c.get(), d_lambda, d_x, alpha, d_grad);
    } else {
      grad_pattern<8><<<grid_for(ctx, (long long)A->n * 8, block), block, 0, ctx->stream>>>(
          A->n, A->r.get(), A->c.get(), d_lambda, d_x, alpha, d_grad);
    }
    DECO_CHECK_LAUNCH();
  });
}

int deco_adjoint_create(deco_ctx ctx, deco_csr A, const deco_cpr_params* prm, deco_adjoint* out) {
  return guard([&] {
    DECO_REQUIRE(ctx && A && prm && out, DECO_ERR_ARG, "NULL argument");
    DECO_REQUIRE(A->n == A->m, DECO_ERR_ARG, "the adjoint needs a square matrix");
    auto* J = new deco_adjoint_s();
    try {
      csr_transpose(ctx, A->n, A->m, A->nz, A->r.get(), A->c.get(), A->v.get(), &J->At);
      J->rhs.alloc(A->n, ctx->stream);
      J->rhs.zero(ctx->stream);
      int rc = deco_cpr_create(ctx, &J->At, J->rhs.get(), prm, &J->P);
      if (rc != DECO_OK) throw Error(rc, std::string("CPR of the transposed system: ") + deco_last_error());
    } catch (...) {
      delete J;
      throw;
    }
    *out = J;
  });
}

int deco_adjoint_destroy(deco_adjoint J) {
  return guard([&] { delete J; });
}

int deco_adjoint_solve(deco_ctx ctx, deco_adjoint J, const double* d_g, double* d_lambda,
                       const deco_sol_params* prm, deco_sol_result* res, double* h_resvec) {
  return guard([&] {
    DECO_REQUIRE(ctx && J && d_g && d_lambda && prm, DECO_ERR_ARG, "NULL argument");
    const int n = J->At.n;
    DECO_CUDA(cudaMemcpyAsync(J->rhs.get(), d_g, sizeof(double) * (size_t)n, cudaMemcpyDefault, ctx->stream));
    int rc = deco_cpr_decouple_rhs(ctx, J->P, J->rhs.get());
    if (rc != DECO_OK) throw Error(rc, deco_last_error());
    rc = deco_gmres_solve(ctx, &J->At, J->P, J->rhs.get(), d_lambda, prm, res, h_resvec);
    if (rc != DECO_OK) throw Error(rc, deco_last_error());
  });
}

int deco_adjoint_parts(deco_adjoint J, deco_csr* At, deco_cpr* P) {
  return guard([&] {
    DECO_REQUIRE(J, DECO_ERR_ARG, "NULL argument");
    if (At) *At = &J->At;
    if (P) *P = J->P;
  });
}

}  // extern "C"
