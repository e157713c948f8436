// cpr.cuh — CPR preconditioner handle and the templated apply used by GMRES.
#pragma once
#include "fsai.cuh"
#include "jacobi.cuh"

struct deco_cpr_s {
  deco_cpr_params prm{};
  int n = 0, sn = 0, bs = 1, p = 0;
  deco_csr_s* A = nullptr;        // the decoupled system (borrowed, mutated in place)
  deco_csr_s Ap;                  // pressure matrix A_pp
  deco_fsai_s glo, loc;           // global FSAI on A, local FSAI on A_pp (when their type is FSAI)
  deco_jacobi_s jac;              // Jacobi on A: the global stage (type Jacobi) or seq 2's first stage
  deco_jacobi_s jloc;             // Jacobi on A_pp (local type Jacobi)
  deco::DevBuf<double> J, w;      // CPD blocks, IMPES weights
  deco::DevBuf<double> w0;        // weights before the DRS reset (right-hand-side replay)
  deco::DevBuf<unsigned char> ops;  // per-cell DRS row flags and row swap (right-hand-side replay)
  deco::DevBuf<char> check_diag;  // rows whose diagonal fix_diag replaced
  deco::DevBuf<double> rt, rts;   // residual (n) and restricted residual (sn)
  deco::DevBuf<float> rt32, rts32;
  int fixed = 0;
  double t_ms[5] = {0, 0, 0, 0, 0};
};

namespace deco {

// x = M^{-1} r, float64 preconditioner (apply_seq0/1/3, precond/CPR.hpp:176-299).
void cpr_apply64(deco_ctx_s* ctx, deco_cpr_s* P, const double* r, double* x);

// ||T^-1 r|| / ||T^-1 b|| for the block-diagonal decoupling T that the CPR setup
// applied to the system (row swaps, weights, DRS, IMPES sum, CPD), r and b given
// in the decoupled form: the relative residual of the original system.  T's
// blocks are recovered by replaying the decoupling on unit vectors; NaN if a
// block is singular.  Synchronises the context's stream.
double cpr_original_relres(deco_ctx_s* ctx, deco_cpr_s* P, const double* r, const double* b);

// x = M^{-1} r with float32 factors, float32 A copy and float32 internal vectors;
// r and x may be float64 or float32.
template <typename RT, typename XT>
void cpr_apply32(deco_ctx_s* ctx, deco_cpr_s* P, const RT* r, XT* x);

}  // namespace deco
