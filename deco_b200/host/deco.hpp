// deco.hpp — C++ host classes with the reference's interfaces, running on the GPU
// through the C ABI of include/deco_b200.h.
//
//   CSR<R,C,V>                         core/CSR.hpp:4-13      (device-resident copy)
//   FSAI<R,C,V>(ptree, A)              precond/FSAI/FSAI.hpp:14-47
//   CPR<R,C,V,Mglobal,Mlocal>(ptree, A, b)   precond/CPR.hpp:42-172
//   SOL<R,C,V>(ptree, A, precond, b, x)      solver/SOL.hpp:19-49
//   ADJ<R,C,V>(ptree prec, A)                adjoint solve + dL/dA (no reference counterpart)
//
// A drop-in for the reference's call sequence (cpr.cpp:60-79):
//   auto P = std::make_shared<CPR<int,int,double,FSAI,FSAI>>(param.get_child("prec"), A, b);
//   auto S = std::make_shared<SOL<int,int,double>>(param.get_child("sol"), A, P->apply, b, x);
// Differences that follow from the device: the vectors the preconditioners and
// solvers take (b, x, and the arguments of apply) are DEVICE pointers (float64);
// CSR keeps its host arrays r, c, v (the reference's public members) and a
// device copy that CPR modifies in place — download() refreshes the host arrays.
// Errors raise deco::gpu_error (the reference calls exit()).
#pragma once
#include <cuda_runtime.h>

#include <functional>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "deco_b200.h"
#include "ptree.hpp"

namespace deco {

struct gpu_error : std::runtime_error {
  int code;
  gpu_error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc, const char* what) {
  if (rc != DECO_OK) throw gpu_error(rc, std::string(what) + ": " + deco_last_error());
}

// One process-wide context per device (the reference's global deco_comm analogue).
inline deco_ctx context(int device = 0) {
  static std::map<int, deco_ctx> ctxs;
  auto it = ctxs.find(device);
  if (it != ctxs.end()) return it->second;
  deco_ctx c = nullptr;
  check(deco_ctx_create(device, nullptr, &c), "deco_ctx_create");
  ctxs[device] = c;
  return c;
}

inline void sync() { check(deco_ctx_sync(context()), "deco_ctx_sync"); }

// Device vector helper (owning).
template <typename V>
struct DeviceVector {
  V* p = nullptr;
  size_t n = 0;
  explicit DeviceVector(size_t n_) : n(n_) {
    if (cudaMalloc(&p, sizeof(V) * (n ? n : 1)) != cudaSuccess) throw gpu_error(DECO_ERR_ALLOC, "cudaMalloc");
  }
  DeviceVector(const V* host, size_t n_) : DeviceVector(n_) { upload(host); }
  ~DeviceVector() { cudaFree(p); }
  DeviceVector(const DeviceVector&) = delete;
  DeviceVector& operator=(const DeviceVector&) = delete;
  void upload(const V* host) {
    void* s = nullptr;
    check(deco_ctx_stream(context(), &s), "stream");
    if (cudaMemcpyAsync(p, host, sizeof(V) * n, cudaMemcpyHostToDevice, (cudaStream_t)s) != cudaSuccess)
      throw gpu_error(DECO_ERR_CUDA, "upload");
    sync();
  }
  void download(V* host) const {
    void* s = nullptr;
    check(deco_ctx_stream(context(), &s), "stream");
    if (cudaMemcpyAsync(host, p, sizeof(V) * n, cudaMemcpyDeviceToHost, (cudaStream_t)s) != cudaSuccess)
      throw gpu_error(DECO_ERR_CUDA, "download");
    sync();
  }
};

template <typename R = int, typename C = int, typename V = double>
class CSR {
  static_assert(sizeof(R) == 4 && sizeof(C) == 4 && sizeof(V) == 8, "the GPU path is CSR<int,int,double>");

 public:
  C n = 0, m = 0;
  R nz = 0;
  std::vector<R> r;
  std::vector<C> c;
  std::vector<V> v;
  deco_csr dev = nullptr;

  CSR() = default;
  CSR(C n_, C m_, R nz_, const R* r_, const C* c_, const V* v_) : n(n_), m(m_), nz(nz_) {
    r.assign(r_, r_ + n + 1);
    c.assign(c_, c_ + nz);
    v.assign(v_, v_ + nz);
    check(deco_csr_create(context(), n, m, nz, r.data(), c.data(), v.data(), 0, &dev), "deco_csr_create");
  }
  ~CSR() {
    if (dev && owns) deco_csr_destroy(dev);
  }
  CSR(const CSR&) = delete;
  CSR& operator=(const CSR&) = delete;

  static std::shared_ptr<CSR> borrow(deco_csr h) {
    auto A = std::make_shared<CSR>();
    A->dev = h;
    A->owns = false;
    check(deco_csr_info(h, &A->n, &A->m, &A->nz), "deco_csr_info");
    return A;
  }

  // b = A x, or the restricted product for bs > 1 (core/alg.hpp:50-64); device pointers
  void apply(const V* x, V*& b, const int bs = 1) { check(deco_spmv(context(), dev, x, b, bs), "deco_spmv"); }

  // refresh the host arrays from the (possibly decoupled) device matrix
  void download() {
    check(deco_csr_info(dev, &n, &m, &nz), "deco_csr_info");
    r.resize(n + 1);
    c.resize(nz);
    v.resize(nz);
    check(deco_csr_download(context(), dev, r.data(), c.data(), v.data()), "deco_csr_download");
  }

 private:
  bool owns = true;
};

template <typename R = int, typename C = int, typename V = double>
class FSAI {
 public:
  std::string name = "FSAI";
  deco_fsai dev = nullptr;
  const ptree& param;
  std::function<void(const V*, V*&)> apply;

  FSAI(const ptree& pt, std::shared_ptr<CSR<R, C, V>> A, int precision = 64) : param(pt) {
    check(deco_fsai_create(context(), A->dev, pt.get<double>("tol_rel"), pt.get<double>("tol_abs"),
                           pt.get<int>("power"), precision, &dev),
          "deco_fsai_create");
    owns = true;
    bind();
  }
  FSAI(const ptree& pt, deco_fsai borrowed) : dev(borrowed), param(pt) { bind(); }
  ~FSAI() {
    if (owns && dev) deco_fsai_destroy(dev);
  }

 private:
  bool owns = false;
  void bind() {
    apply = [this](const V* x, V*& b) { check(deco_fsai_apply(context(), dev, x, b), "deco_fsai_apply"); };
  }
};

template <typename V>
class CPRBase {
 public:
  virtual ~CPRBase() { registry().erase(&apply); }
  std::function<void(V*, V*&)> apply;
  deco_cpr dev = nullptr;
  // SOL receives `P->apply` (cpr.cpp:76); this lets it find the native handle.
  static std::map<const void*, deco_cpr>& registry() {
    static std::map<const void*, deco_cpr> m;
    return m;
  }
};

namespace detail {
inline int weights_id(const std::string& w) {
  if (w == "none") return 0;
  if (w == "quasiimpes") return 1;
  if (w == "quasiimpes_GE") return 2;
  throw std::invalid_argument("Unknown weights type " + w);
}
// the `prec` object of a parameter file (precond/CPR.hpp:49-65,118,130)
inline deco_cpr_params cpr_params(const ptree& pt, int precision) {
  deco_cpr_params prm{};
  prm.block_size = pt.get<int>("block_size");
  prm.pressure_id = pt.get<int>("pressure_id");
  prm.seq = pt.get<int>("seq");
  prm.weights = weights_id(pt.get<std::string>("weights"));
  prm.use_drs = pt.get<int>("use_drs");
  prm.drs_e_dd = pt.get<double>("drs.e_dd");
  prm.drs_e_ps = pt.get<double>("drs.e_ps");
  prm.cpd = pt.get<int>("CPD");
  prm.tol_zero = pt.get<double>("tol_zero");
  const std::string glo = pt.get<std::string>("prec_glo.type"), loc = pt.get<std::string>("prec_loc.type");
  auto stage = [](const std::string& t) {
    if (t == "FSAI") return 0;
    if (t == "Jacobi") return 1;
    throw gpu_error(DECO_ERR_UNSUPPORTED, "the GPU path builds FSAI or Jacobi stages (got " + t +
                                              "); hypre AMG stays on the CPU build");
  };
  prm.glo_type = stage(glo);
  prm.loc_type = stage(loc);
  prm.glo_block_size = pt.get<int>("prec_glo.block_size", prm.block_size);
  prm.loc_block_size = pt.get<int>("prec_loc.block_size", 1);
  prm.glo_tol_rel = pt.get<double>("prec_glo.tol_rel", 0.0);
  prm.glo_tol_abs = pt.get<double>("prec_glo.tol_abs", 0.0);
  prm.glo_power = pt.get<int>("prec_glo.power", 1);
  prm.loc_tol_rel = pt.get<double>("prec_loc.tol_rel");
  prm.loc_tol_abs = pt.get<double>("prec_loc.tol_abs", 0.0);
  prm.loc_power = pt.get<int>("prec_loc.power", 1);
  prm.precision = pt.get<int>("precision", precision);
  return prm;
}

// the `sol` object of a parameter file (solver/SOL.hpp:19-39, rgmres.tpp:13-16)
inline deco_sol_params sol_params(const ptree& pt, int precision, bool use_x0) {
  deco_sol_params sp{};
  const std::string type = pt.get<std::string>("type");
  if (type == "rgmres") sp.type = 0;
  else if (type == "lgmres") sp.type = 1;
  else throw std::invalid_argument("Invalid solver type: " + type);
  sp.reltol = pt.get<double>("reltol");
  sp.restart = pt.get<int>("restart");
  sp.itmax = pt.get<int>("itmax");
  sp.verbosity = pt.get<int>("verbosity", 0);
  sp.precision = pt.get<int>("precision", precision);
  sp.use_x0 = use_x0 ? 1 : 0;
  return sp;
}
}  // namespace detail

template <typename R = int, typename C = int, typename V = double,
          template <typename, typename, typename> class Mglobal = FSAI,
          template <typename, typename, typename> class Mlocal = FSAI>
class CPR : public CPRBase<V> {
 public:
  std::shared_ptr<CSR<R, C, V>> A, Ap;
  std::shared_ptr<FSAI<R, C, V>> Fglo, Floc;
  const ptree& param;
  int bs, p;

  // precision: 64, or 32 for the float32 preconditioner (ptree key "precision" overrides)
  CPR(const ptree& pt, std::shared_ptr<CSR<R, C, V>> A_, V*& b, int precision = 64) : A(A_), param(pt) {
    deco_cpr_params prm = detail::cpr_params(pt, precision);
    bs = prm.block_size;
    p = prm.pressure_id;
    check(deco_cpr_create(context(), A->dev, b, &prm, &this->dev), "deco_cpr_create");
    deco_csr hp = nullptr;
    check(deco_cpr_pressure(this->dev, &hp), "deco_cpr_pressure");
    Ap = CSR<R, C, V>::borrow(hp);
    deco_fsai fg = nullptr, fl = nullptr;
    check(deco_cpr_fsai(this->dev, 0, &fg), "deco_cpr_fsai");
    check(deco_cpr_fsai(this->dev, 1, &fl), "deco_cpr_fsai");
    Fglo = std::make_shared<FSAI<R, C, V>>(pt.get_child("prec_glo"), fg);
    Floc = std::make_shared<FSAI<R, C, V>>(pt.get_child("prec_loc"), fl);
    deco_cpr h = this->dev;
    this->apply = [h](V* r, V*& x) { check(deco_cpr_apply(context(), h, r, x), "deco_cpr_apply"); };
    CPRBase<V>::registry()[&this->apply] = h;
  }
  ~CPR() override {
    Fglo.reset();
    Floc.reset();
    Ap.reset();
    if (this->dev) deco_cpr_destroy(this->dev);
  }

  // setup phases in ms: decoupling, get local matrix, Global precond, Local  precond, Prec
  std::vector<double> timings() const {
    std::vector<double> t(5);
    check(deco_cpr_timings(this->dev, t.data()), "deco_cpr_timings");
    return t;
  }
};

template <typename R = int, typename C = int, typename V = double>
class SOL {
 public:
  const ptree& param;
  std::shared_ptr<CSR<R, C, V>> A;
  V* b;
  V* x;
  int iter = 0;
  double res_abs = 0, res_rel = 0;
  double res_rel_orig = 0;  // original (not decoupled) system; res_rel is on the decoupled one
  int flag = 1;
  double time_ms = 0;
  std::vector<double> resvec;

  // solver/SOL.hpp:19-39: the solve runs in the constructor.  b and x are device
  // pointers; x == nullptr starts from zero into an owned buffer (get_result()).
  SOL(const ptree& pt, std::shared_ptr<CSR<R, C, V>> A_, const std::function<void(V*, V*&)>& precond, V* b_,
      V* x_ = nullptr, int precision = 64)
      : param(pt), A(A_), b(b_), x(x_) {
    auto& reg = CPRBase<V>::registry();
    auto it = reg.find(&precond);
    if (it == reg.end())
      throw gpu_error(DECO_ERR_ARG, "SOL on the GPU needs the apply of a CPR built on the GPU");
    run(it->second, precision);
  }

  V* get_result() const { return x; }
  ~SOL() {
    if (owned_x) cudaFree(owned_x);
  }

 private:
  V* owned_x = nullptr;
  void run(deco_cpr P, int precision) {
    deco_sol_params sp = detail::sol_params(param, precision, x != nullptr);
    if (!x) {
      if (cudaMalloc(&owned_x, sizeof(V) * A->n) != cudaSuccess) throw gpu_error(DECO_ERR_ALLOC, "cudaMalloc x");
      x = owned_x;
    }
    resvec.assign((size_t)sp.itmax + 1, 0.0);
    deco_sol_result res{};
    check(deco_gmres_solve(context(), A->dev, P, b, x, &sp, &res, resvec.data()), "deco_gmres_solve");
    iter = res.iter;
    flag = res.flag;
    res_abs = res.res_abs;
    res_rel = res.res_rel;
    res_rel_orig = res.res_rel_orig;
    time_ms = res.t_solve_ms;
    resvec.resize(iter);
  }
};

// Adjoint of the solve x = A^{-1} b (no counterpart in the reference).  For a
// loss L(x) with g = dL/dx:  A^T lambda = g,  dL/db = lambda,
// dL/dA_ij = -lambda_i x_j on A's pattern.  Built from A with its ORIGINAL
// values (before a forward CPR decouples it in place): A^T is transposed on the
// device and decoupled by its own CPR.  solve() takes any number of right-hand
// sides; the forward x is the only state the gradient needs.
template <typename R = int, typename C = int, typename V = double>
class ADJ {
 public:
  const ptree& param;
  deco_adjoint dev = nullptr;
  C n = 0;
  int iter = 0, flag = 1;
  double res_abs = 0, res_rel = 0, time_ms = 0;
  std::vector<double> resvec;

  ADJ(const ptree& prec, std::shared_ptr<CSR<R, C, V>> A, int precision = 64) : param(prec), n(A->n) {
    deco_cpr_params prm = detail::cpr_params(prec, precision);
    precision_ = prm.precision;
    check(deco_adjoint_create(context(), A->dev, &prm, &dev), "deco_adjoint_create");
  }
  ~ADJ() {
    if (dev) deco_adjoint_destroy(dev);
  }
  ADJ(const ADJ&) = delete;
  ADJ& operator=(const ADJ&) = delete;

  // lambda = A^{-T} g (device pointers); lambda is the initial guess if use_x0
  void solve(const ptree& sol, const V* g, V* lambda, bool use_x0 = false) {
    deco_sol_params sp = detail::sol_params(sol, precision_, use_x0);
    resvec.assign((size_t)sp.itmax + 1, 0.0);
    deco_sol_result res{};
    check(deco_adjoint_solve(context(), dev, g, lambda, &sp, &res, resvec.data()), "deco_adjoint_solve");
    iter = res.iter;
    flag = res.flag;
    res_abs = res.res_abs;
    res_rel = res.res_rel;
    time_ms = res.t_solve_ms;
    resvec.resize(iter);
  }

  // grad[e] = alpha * lambda_i * x_j over A's stored entries (dL/dA for alpha = -1)
  static void grad_A(const CSR<R, C, V>& A, const V* lambda, const V* x, V* grad, V alpha = -1) {
    check(deco_grad_A_pattern(context(), A.dev, lambda, x, alpha, grad), "deco_grad_A_pattern");
  }

 private:
  int precision_ = 64;
};

}  // namespace deco
