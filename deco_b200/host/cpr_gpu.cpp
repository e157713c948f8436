// cpr_gpu — the reference's `cpr` driver (cpr.cpp:8-91) on the GPU path.
//
//   deco_cpr_gpu param.json [--precision 64|32]
//
// Reads the same JSON parameter files (comments allowed, IO/ptree.hpp:27-119),
// the same binary CSR / rhs files (IO/cpp_read.hpp:331-442: int n, m, nz;
// r[n+1]; c[nz]; v[nz] and int n; b[n]; rhs "ones" = A*1), builds
// CPR<int,int,double,FSAI,FSAI> and SOL on the GPU and prints the reference's
// solver summary (rgmres.tpp:130-135) and its profiler node names.
// prec.row_order / prec.col_order other than 12(3) reorder every cell's unknowns
// first, as the reference's driver does (cpr.cpp:41, adapter/csr2coo.cpp).
// `"parallel": {"hardware": "GPU"}` selects this path; the reference never reads
// that key (cpr.cpp:19-21).  IO.format "synthetic" (IO.preset, IO.seed) runs a
// generated system instead of files.
//
// An optional "adjoint" object ({"observations": N, "seed": S, "wfile_lambda":
// path}) differentiates L = sum_k w_k p(cell_k) over N seeded cells with seeded
// weights w_k in [0,1): after the forward solve it solves A^T lambda = dL/dx
// with CPR on A^T (ADJ), forms dL/dA = -lambda_i x_j on A's pattern and prints
// the adjoint summary.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <vector>

#include "deco.hpp"
#include "deco_gen.h"

using namespace deco;
using Mat = CSR<int, int, double>;

static double now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

static bool read_matrix(const std::string& fn, int& n, int& m, int& nz, std::vector<int>& r, std::vector<int>& c,
                        std::vector<double>& v) {
  std::ifstream f(fn, std::ios::binary);
  if (!f) return false;
  f.read((char*)&n, 4);
  f.read((char*)&m, 4);
  f.read((char*)&nz, 4);
  r.resize(n + 1);
  c.resize(nz);
  v.resize(nz);
  f.read((char*)r.data(), 4LL * (n + 1));
  f.read((char*)c.data(), 4LL * nz);
  f.read((char*)v.data(), 8LL * nz);
  return (bool)f;
}

static bool read_rhs(const std::string& fn, int n, const std::vector<int>& r, const std::vector<int>& c,
                     const std::vector<double>& v, std::vector<double>& b) {
  b.assign(n, 0.0);
  if (fn == "unity" || fn == "unitary" || fn == "uno" || fn == "one" || fn == "ones") {
    for (int i = 0; i < n; ++i)
      for (int j = r[i]; j < r[i + 1]; ++j) b[i] += v[j];
    return true;
  }
  if (fn == "zero") return true;
  std::ifstream f(fn, std::ios::binary);
  if (!f) return false;
  int nn = 0;
  f.read((char*)&nn, 4);
  if (nn != n) return false;
  f.read((char*)b.data(), 8LL * n);
  return (bool)f;
}

// AD::block_reorder (adapter/csr2coo.cpp:18-86): the unknowns of every cell are
// permuted so the pressure equation and variable come first.  row_order /
// col_order list, for each new position, the old 1-based position in the cell.
// New row s*bs + p is old row s*bs + (row_order[p] - 1); each column moves
// within its cell the same way by col_order; rows end up sorted by column (the
// reference sorts the coordinate list by row, then column) and b follows the rows.
static void block_reorder(int n, std::vector<int>& r, std::vector<int>& c, std::vector<double>& v,
                          std::vector<double>& b, int bs, const std::string& row_order, const std::string& col_order) {
  if ((int)row_order.size() != bs || (int)col_order.size() != bs)
    throw std::invalid_argument("prec.row_order / prec.col_order must list the " + std::to_string(bs) +
                                " positions of a cell");
  std::vector<int> ord_row(bs), reord_col(bs);
  for (int i = 0; i < bs; ++i) {
    const int ro = row_order[i] - '1', co = col_order[i] - '1';
    if (ro < 0 || ro >= bs || co < 0 || co >= bs) throw std::invalid_argument("bad prec.row_order / prec.col_order");
    ord_row[i] = ro;
    reord_col[co] = i;
  }
  std::vector<int> nr(n + 1, 0), nc(c.size());
  std::vector<double> nv(v.size()), nb(b.size());
  for (int i = 0; i < n; ++i) {
    const int old = i - i % bs + ord_row[i % bs];
    nr[i + 1] = nr[i] + (r[old + 1] - r[old]);
  }
  std::vector<std::pair<int, double>> row;
  for (int i = 0; i < n; ++i) {
    const int old = i - i % bs + ord_row[i % bs];
    row.clear();
    for (int j = r[old]; j < r[old + 1]; ++j) row.emplace_back(c[j] - c[j] % bs + reord_col[c[j] % bs], v[j]);
    std::sort(row.begin(), row.end(), [](const std::pair<int, double>& a, const std::pair<int, double>& b) {
      return a.first < b.first;
    });
    for (size_t k = 0; k < row.size(); ++k) {
      nc[nr[i] + k] = row[k].first;
      nv[nr[i] + k] = row[k].second;
    }
    nb[i] = b[old];
  }
  r.swap(nr);
  c.swap(nc);
  v.swap(nv);
  b.swap(nb);
}

int main(int argc, char** argv) {
  if (argc < 2) {
    std::cerr << "Usage: " << argv[0] << " param.json [--precision 64|32]" << std::endl;
    return 2;
  }
  int precision = 64;
  for (int i = 2; i + 1 < argc; ++i)
    if (!std::strcmp(argv[i], "--precision")) precision = std::atoi(argv[i + 1]);
  try {
    ptree param = read_json_file(argv[1]);
    const std::string hw = param.get<std::string>("parallel.hardware", "GPU");
    if (hw != "GPU" && hw != "gpu")
      std::cerr << "note: parallel.hardware = " << hw << "; this binary runs the GPU path" << std::endl;
    int n = 0, m = 0, nz = 0;
    std::vector<int> r, c;
    std::vector<double> v, b;
    const std::string format = param.get<std::string>("IO.format");
    double t0 = now();
    if (format == "synthetic") {
      deco_gen_params gp;
      if (deco_gen_preset(param.get<int>("IO.preset", 1), param.get<unsigned long long>("IO.seed", 1234ULL), &gp))
        throw std::invalid_argument("unknown IO.preset");
      long long nnz = 0;
      if (deco_gen_size(&gp, &n, &nnz)) throw std::runtime_error("deco_gen_size failed");
      m = n;
      nz = (int)nnz;
      r.resize(n + 1);
      c.resize(nz);
      v.resize(nz);
      b.resize(n);
      if (deco_gen_fill(&gp, r.data(), c.data(), v.data(), b.data(), nullptr)) throw std::runtime_error("gen failed");
    } else if (format == "bin" || format == "binary") {
      if (!read_matrix(param.get<std::string>("IO.file_A"), n, m, nz, r, c, v))
        throw std::runtime_error("Could not read " + param.get<std::string>("IO.file_A"));
      if (!read_rhs(param.get<std::string>("IO.file_b"), n, r, c, v, b))
        throw std::runtime_error("Could not read " + param.get<std::string>("IO.file_b"));
    } else {
      throw std::invalid_argument("Unknown global IO::format: " + format);
    }
    const int bs = param.get<int>("prec.block_size");
    {
      std::string id;
      for (int k = 1; k <= bs; ++k) id += char('0' + k);
      const std::string ro = param.get<std::string>("prec.row_order", id), co = param.get<std::string>("prec.col_order", id);
      if (ro != id || co != id) block_reorder(n, r, c, v, b, bs, ro, co);
    }
    std::printf("matrix size:\tn = %d, m = %d, nz = %d  (IO %.3f s)\n", n, m, nz, now() - t0);

    auto A = std::make_shared<Mat>(n, m, nz, r.data(), c.data(), v.data());
    DeviceVector<double> bd(b.data(), b.size());
    double* bp = bd.p;
    sync();
    double t_prec = now();
    auto P = std::make_shared<CPR<int, int, double, FSAI, FSAI>>(param.get_child("prec"), A, bp, precision);
    sync();
    t_prec = now() - t_prec;
    double t_sol = now();
    auto S = std::make_shared<SOL<int, int, double>>(param.get_child("sol"), A, P->apply, bp, nullptr, precision);
    sync();
    t_sol = now() - t_sol;
    // the solver summary of rgmres.tpp:130-135 (printed here whatever sol.verbosity says)
    std::printf("\n--------------------------------\n");
    std::printf("Profile of %s:\n", param.get<std::string>("sol.type") == "lgmres" ? "lGMRES" : "rGMRES");
    std::printf("iteration count =  %d\n", S->iter);
    std::printf("residual = %.2e\n", S->res_rel);
    std::printf("residual of the original system = %.2e\n", S->res_rel_orig);
    auto t = P->timings();
    std::printf("\nprofile (s)\n");
    std::printf("  setup & solve       %10.5f\n", t_prec + t_sol);
    std::printf("    Prec              %10.5f\n", t_prec);
    std::printf("      decoupling      %10.5f\n", (t[0] + t[1]) / 1e3);
    std::printf("      Global precond  %10.5f\n", t[2] / 1e3);
    std::printf("      Local  precond  %10.5f\n", t[3] / 1e3);
    std::printf("    Solve             %10.5f\n", t_sol);
    std::printf("flag = %d  precision = %d\n", S->flag, precision);
    const std::string wfile = param.get<std::string>("IO.wfile_x", "");
    if (!wfile.empty() && wfile != "null") {
      std::vector<double> x(n);
      cudaMemcpy(x.data(), S->get_result(), sizeof(double) * n, cudaMemcpyDeviceToHost);
      std::ofstream f(wfile, std::ios::binary);
      f.write((const char*)&n, 4);
      f.write((const char*)x.data(), 8LL * n);
    }
    int adj_flag = 0;
    if (param.find("adjoint")) {
      // A was decoupled in place by the forward CPR: the adjoint starts from the original values
      const int nobs = param.get<int>("adjoint.observations", 20);
      const unsigned long long seed = param.get<unsigned long long>("adjoint.seed", 2024ULL);
      const int ncell = n / bs;
      if (nobs < 1 || nobs > ncell) throw std::invalid_argument("adjoint.observations out of range");
      std::vector<double> u(2LL * nobs), g(n, 0.0);
      deco_gen_uniform(seed, 77, 2LL * nobs, u.data());
      for (int k = 0; k < nobs; ++k) g[(long long)std::min(ncell - 1, (int)(u[2 * k] * ncell)) * bs] += u[2 * k + 1];
      double t_adj = now();
      auto A0 = std::make_shared<Mat>(n, m, nz, r.data(), c.data(), v.data());
      ADJ<int, int, double> J(param.get_child("prec"), A0, precision);
      DeviceVector<double> gd(g.data(), n), lam(n), grad((size_t)nz);
      J.solve(param.get_child("sol"), gd.p, lam.p);
      ADJ<int, int, double>::grad_A(*A0, lam.p, S->get_result(), grad.p);
      sync();
      t_adj = now() - t_adj;
      std::vector<double> hl(n), hg((size_t)nz);
      lam.download(hl.data());
      grad.download(hg.data());
      double nl = 0, ng = 0;
      for (double e : hl) nl += e * e;
      for (double e : hg) ng += e * e;
      std::printf("\nadjoint iteration count =  %d\n", J.iter);
      std::printf("adjoint residual = %.2e\n", J.res_rel);
      std::printf("|dL/db| = %.6e  |dL/dA| = %.6e  (%d observations, %.5f s)\n", std::sqrt(nl), std::sqrt(ng), nobs,
                  t_adj);
      const std::string wl = param.get<std::string>("adjoint.wfile_lambda", "");
      if (!wl.empty() && wl != "null") {
        std::ofstream f(wl, std::ios::binary);
        f.write((const char*)&n, 4);
        f.write((const char*)hl.data(), 8LL * n);
      }
      adj_flag = J.flag;
    }
    return (S->flag == 0 && adj_flag == 0) ? 0 : 1;
  } catch (const std::exception& e) {
    std::cerr << "error: " << e.what() << std::endl;
    return 3;
  }
}
