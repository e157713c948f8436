// Oracle library built from the reference's own, unmodified headers
// (CPR<int,int,double,FSAI,FSAI> + SOL), exported through a small C ABI so the
// tests can run the reference on the very inputs the GPU path sees.
//
// TEST INFRASTRUCTURE ONLY: this file is compiled by oracle/ref/Makefile into
// oracle/_ref/libdeco_ref.so.  Nothing in the product loads it.
//
// The include list follows the reference's precompiled header core/pch.h:1-51,
// minus hypre (core/pch.h:33-36, not on this path); MPI, boost::property_tree
// and LAPACKE come from the shims in oracle/ref/shim.
#include <limits.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <functional>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <memory>
#include <stack>
#include <string>
#include <unordered_map>
#include <vector>

#include <mpi.h>
#include <omp.h>
MPI_Comm deco_comm = MPI_COMM_WORLD;

#include <boost/property_tree/json_parser.hpp>
#include <boost/property_tree/ptree.hpp>

#include <cblas.h>
#include <lapacke.h>

#include "core/header.h"
#include "core/profiler.hpp"
#include "core/alg.hpp"
#include "core/CSR.hpp"
#include "precond/FSAI/core.tpp"
#include "core/MxM.cpp"
#include "IO/cpp_read.hpp"
#include "IO/ptree.hpp"
#include "adapter/csr2coo.cpp"
#include "precond/FSAI/FSAI.hpp"
#include "precond/Jacobi/Jacobi.hpp"
#include "precond/CPR.hpp"
#include "solver/SOL.hpp"

#include <cstring>

using Mat = CSR<int, int, double>;
using CPRff = CPR<int, int, double, FSAI, FSAI>;
using CPRjf = CPR<int, int, double, Jacobi, FSAI>;
using CPRfj = CPR<int, int, double, FSAI, Jacobi>;
using CPRjj = CPR<int, int, double, Jacobi, Jacobi>;

namespace {

double now() { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }

std::shared_ptr<Mat> make_matrix(int n, const int* r, const int* c, const double* v) {
  int nz = r[n];
  auto A = std::make_shared<Mat>(n, n, nz);
  std::memcpy(A->r, r, sizeof(int) * (n + 1));
  std::memcpy(A->c, c, sizeof(int) * nz);
  std::memcpy(A->v, v, sizeof(double) * nz);
  // single-rank metadata exactly as IO::distribute_csr_matrix fills it (IO/cpp_read.hpp:473-500)
  return IO::distribute_csr_matrix(A, 0, 1, 1);
}

void copy_out(const Mat& M, int* r, int* c, double* v) {
  if (r) std::memcpy(r, M.r, sizeof(int) * (M.n + 1));
  if (c) std::memcpy(c, M.c, sizeof(int) * M.nz);
  if (v) std::memcpy(v, M.v, sizeof(double) * M.nz);
}

struct FsaiHandle {
  boost::property_tree::ptree pt;
  std::shared_ptr<Mat> A;
  std::unique_ptr<FSAI<int, int, double>> F;
  double t_setup = 0;
};

struct CprHandle {
  boost::property_tree::ptree pt;  // whole parameter tree; CPR keeps references into it
  std::shared_ptr<Mat> A;
  double* b = nullptr;
  std::shared_ptr<CPRBase<double>> P;
  std::shared_ptr<Mat> Ap;
  FSAI<int, int, double>* Fglo = nullptr;
  FSAI<int, int, double>* Floc = nullptr;
  double t_setup = 0;
  int n = 0;
};

}  // namespace

extern "C" {

void ref_spmv(int n, const int* r, const int* c, const double* v, const double* x, double* y, int bs) {
  alg::spmv(n, r, c, v, x, y, bs);
}

void ref_filter(int n, const int* r, const int* c, const double* v, double tol, int relative, int* nz_out,
                int* ro, int* co, double* vo) {
  auto A = make_matrix(n, r, c, v);
  if (relative) A->filter_proper(tol);
  else A->filter(tol);
  *nz_out = A->nz;
  copy_out(*A, ro, co, vo);
}

void* ref_fsai_create(int n, const int* r, const int* c, const double* v, double tol_rel, double tol_abs,
                      int power) {
  auto* h = new FsaiHandle();
  h->pt.put("tol_rel", tol_rel);
  h->pt.put("tol_abs", tol_abs);
  h->pt.put("power", power);
  h->A = make_matrix(n, r, c, v);
  double t0 = now();
  h->F.reset(new FSAI<int, int, double>(h->pt, h->A));
  h->t_setup = now() - t0;
  return h;
}

int ref_fsai_nnz(void* hv) { return static_cast<FsaiHandle*>(hv)->F->FL->nz; }
double ref_fsai_setup_time(void* hv) { return static_cast<FsaiHandle*>(hv)->t_setup; }

void ref_fsai_get(void* hv, int* Lr, int* Lc, double* Lv, int* Ur, int* Uc, double* Uv) {
  auto* h = static_cast<FsaiHandle*>(hv);
  copy_out(*h->F->FL, Lr, Lc, Lv);
  copy_out(*h->F->FU, Ur, Uc, Uv);
}

void ref_fsai_apply(void* hv, const double* x, double* y) {
  auto* h = static_cast<FsaiHandle*>(hv);
  h->F->apply(x, y);
}

void ref_fsai_destroy(void* hv) { delete static_cast<FsaiHandle*>(hv); }

// params_json: a full parameter file (keys "prec" and optionally "sol"), comments allowed.
void* ref_cpr_create(const char* params_json, int n, const int* r, const int* c, const double* v, const double* b) {
  auto* h = new CprHandle();
  h->pt = deco::read_json_string(params_json);
  h->A = make_matrix(n, r, c, v);
  h->n = n;
  h->b = memres<double>(n);
  std::memcpy(h->b, b, sizeof(double) * n);
  const auto& prec = h->pt.get_child("prec");
  std::string glo = prec.get<std::string>("prec_glo.type");
  std::string loc = prec.get<std::string>("prec_loc.type");
  double t0 = now();
  if (glo == "Jacobi" && loc == "Jacobi") {
    auto P = std::make_shared<CPRjj>(prec, h->A, h->b);
    h->Ap = P->Ap;
    h->P = P;
  } else if (loc == "Jacobi") {
    auto P = std::make_shared<CPRfj>(prec, h->A, h->b);
    h->Ap = P->Ap;
    h->Fglo = P->Fglo.get();
    h->P = P;
  } else if (glo == "Jacobi") {
    auto P = std::make_shared<CPRjf>(prec, h->A, h->b);
    h->Ap = P->Ap;
    h->Floc = P->Floc.get();
    h->P = P;
  } else {
    auto P = std::make_shared<CPRff>(prec, h->A, h->b);
    h->Ap = P->Ap;
    h->Fglo = P->Fglo.get();
    h->Floc = P->Floc.get();
    h->P = P;
  }
  h->t_setup = now() - t0;
  return h;
}

double ref_cpr_setup_time(void* hv) { return static_cast<CprHandle*>(hv)->t_setup; }

// sizes: [nnz(A), n(Ap), nnz(Ap), nnz(F_glo), nnz(F_loc)]
void ref_cpr_sizes(void* hv, long long* out) {
  auto* h = static_cast<CprHandle*>(hv);
  out[0] = h->A->nz;
  out[1] = h->Ap->n;
  out[2] = h->Ap->nz;
  out[3] = h->Fglo ? h->Fglo->FL->nz : 0;
  out[4] = h->Floc ? h->Floc->FL->nz : 0;
}

void ref_cpr_get_A(void* hv, int* r, int* c, double* v, double* b) {
  auto* h = static_cast<CprHandle*>(hv);
  copy_out(*h->A, r, c, v);
  if (b) std::memcpy(b, h->b, sizeof(double) * h->n);
}

void ref_cpr_get_Ap(void* hv, int* r, int* c, double* v) {
  auto* h = static_cast<CprHandle*>(hv);
  copy_out(*h->Ap, r, c, v);
}

// which: 0 = global FSAI (on A), 1 = local/pressure FSAI (on Ap)
int ref_cpr_get_fsai(void* hv, int which, int* Lr, int* Lc, double* Lv, int* Ur, int* Uc, double* Uv) {
  auto* h = static_cast<CprHandle*>(hv);
  auto* F = which == 0 ? h->Fglo : h->Floc;
  if (!F) return -1;
  copy_out(*F->FL, Lr, Lc, Lv);
  copy_out(*F->FU, Ur, Uc, Uv);
  return 0;
}

void ref_cpr_apply(void* hv, const double* r, double* x) {
  auto* h = static_cast<CprHandle*>(hv);
  std::vector<double> rr(r, r + h->n);  // apply takes a mutable input
  h->P->apply(rr.data(), x);
}

// Runs SOL on the decoupled system held by the handle.  sol_json: the "sol"
// object (keys type, reltol, restart, itmax, verbosity).
int ref_solve(void* hv, const char* sol_json, double* x_out, int* iter, double* res_abs, double* res_rel,
              int* flag, double* t_solve) {
  auto* h = static_cast<CprHandle*>(hv);
  boost::property_tree::ptree sol = deco::read_json_string(sol_json);
  double* b = memres<double>(h->n);  // SOL takes ownership of b and x (solver/SOL.hpp:46-49)
  std::memcpy(b, h->b, sizeof(double) * h->n);
  double t0 = now();
  auto S = std::make_shared<SOL<int, int, double>>(sol, h->A, h->P->apply, b, nullptr);
  *t_solve = now() - t0;
  std::memcpy(x_out, S->get_result(), sizeof(double) * h->n);
  *iter = S->iter;
  *res_abs = S->res_abs;
  *res_rel = S->res_rel;
  *flag = S->flag;
  return 0;
}

void ref_cpr_destroy(void* hv) {
  auto* h = static_cast<CprHandle*>(hv);
  h->P.reset();
  free(h->b);
  delete h;
}

int ref_num_threads() { return omp_get_max_threads(); }

}  // extern "C"
