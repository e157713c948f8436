// gmres.cu — restarted right / left preconditioned GMRES(m) on the device
// (solver/rgmres.tpp:8-139, solver/lgmres.tpp:1-134; Givens :141-160).
//
// Arnoldi step: classical Gram-Schmidt with one reorthogonalisation (CGS2) in
// three fused passes over the basis V (column-major, one column per vector):
//   pass A   h  = V^T w                                  (dots)
//   pass B   w' = w - V h;  h2 = V^T w';  s = ||w'||^2   (update + dots; the
//            second read of each V tile hits L2)
//            the block that finishes last reduces the partial sums, forms
//            H(:,j) = h + h2, beta = sqrt(s - ||h2||^2) (w'' = w' - V h2 is
//            orthogonal to V, so Pythagoras gives its norm without a pass),
//            and applies the Givens rotations to H(:,j) and g — on the device;
//   pass C   v_{j+1} = (w' - V h2) / beta.
// Only |g_{j+1}| (8 bytes) returns to the host per iteration.  The reference
// uses modified Gram-Schmidt (rgmres.tpp:72-75): 5(j+1) vector passes per
// step against 3(j+1)+5 here.
//
// Precision 32: V, w, z in float32 with float64 dot accumulation; H, g and the
// rotations in float64; every restart recomputes the true residual b - A x and
// the solution update in float64 (iterative refinement).
#include <cmath>
#include <vector>

#include "cpr.cuh"

namespace deco {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kColsPerWarp = 8;
constexpr int kMaxCols = kWarps * kColsPerWarp;  // basis columns the CGS kernels handle (restart <= 63)
constexpr double kEps = 2.220446049250312e-16;

// st layout (float64): H (m+1)*m | g | cs | sn | hA | hB (m+1 each) | sc[16]
struct State {
  double* H; double* g; double* cs; double* sn; double* hA; double* hB; double* sc;
  int m;
  __host__ __device__ double& h(int i, int j) const { return H[i + (size_t)j * (m + 1)]; }
};
enum { SC_SS = 0, SC_BETA = 1, SC_INVB = 2, SC_RES = 3, SC_BREAK = 4, SC_NORM = 5, SC_INVN = 6 };

__device__ __forceinline__ double ldv(const double* p) { return __ldcs(p); }
__device__ __forceinline__ double ldv(const float* p) { return (double)__ldcs(p); }

// deterministic last-block reduction of red[i*nb + b] over b for i < ncols
__device__ void finalize_partials(const double* red, int nb, int ncols, double* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = warp; i < ncols; i += kWarps) {
    double s = 0.0;
    for (int b = lane; b < nb; b += 32) s += __ldcg(red + (size_t)i * nb + b);
    s = warp_sum(s);
    if (lane == 0) out[i] = s;
  }
}

__device__ __forceinline__ bool last_block(unsigned* counter) {
  __shared__ bool amlast;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) amlast = atomicInc(counter, gridDim.x - 1) == gridDim.x - 1;
  __syncthreads();
  return amlast;
}

// warp-reduce v and add it to acc[i*kWarps + warp]
__device__ __forceinline__ void acc_add(double* acc, int i, double v) {
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) acc[i * kWarps + (threadIdx.x >> 5)] += v;
}

__device__ void flush_acc(double* acc, int ncols, double* red) {
  __syncthreads();
  for (int i = threadIdx.x; i < ncols; i += kThreads) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) s += acc[i * kWarps + w];
    red[(size_t)i * gridDim.x + blockIdx.x] = s;
  }
}

// ---- pass A: hA[i] = V_i . w, i < ncols.  Warp w owns columns w, w+8, ...;
// its lanes stride over rows and keep one partial sum per owned column in
// registers for the whole kernel, so every column is reduced once per block.
// The block's tile of w is staged in shared memory and shared by the warps.
template <typename T, int KPW>
__global__ void __launch_bounds__(kThreads) cgs_pass_a(long long n, long long ld, int ncols, const T* __restrict__ V,
                                                       const T* __restrict__ w, double* __restrict__ red,
                                                       unsigned* counter, double* __restrict__ hA) {
  __shared__ double ws[kThreads];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double p[KPW];
#pragma unroll
  for (int k = 0; k < KPW; ++k) p[k] = 0.0;
  for (long long base = (long long)blockIdx.x * kThreads; base < n; base += (long long)gridDim.x * kThreads) {
    const long long r = base + threadIdx.x;
    ws[threadIdx.x] = r < n ? (double)w[r] : 0.0;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < KPW; ++k) {
      const int c = warp + k * kWarps;
      if (c < ncols) {
        const T* vc = V + (size_t)c * ld + base;
#pragma unroll
        for (int q = 0; q < kThreads / 32; ++q) {
          const int t = lane + 32 * q;
          if (base + t < n) p[k] += ldv(vc + t) * ws[t];
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int k = 0; k < KPW; ++k) {
    const int c = warp + k * kWarps;
    const double t = warp_sum(p[k]);
    if (lane == 0 && c < ncols) red[(size_t)c * gridDim.x + blockIdx.x] = t;
  }
  if (last_block(counter)) finalize_partials(red, gridDim.x, ncols, hA);
}

__device__ void givens_make(double x, double y, double& c, double& s) {
  if (fabs(y) < kEps) { c = 1.0; s = 0.0; }
  else if (fabs(y) > fabs(x)) { double nu = x / y; s = 1.0 / sqrt(1.0 + nu * nu); c = nu * s; }
  else { double nu = y / x; c = 1.0 / sqrt(1.0 + nu * nu); s = nu * c; }
}
__device__ void givens_apply(double c, double s, double& dx, double& dy) {
  double t = c * dx + s * dy;
  dy = -s * dx + c * dy;
  dx = t;
}

// ---- pass B: w' = w - V hA (in place), hB = V^T w', ss = ||w'||^2.  Each
// block tile of kThreads rows x ncols columns is read once from HBM into
// shared memory while the update runs; the second dot product then reads the
// tile from shared memory, warp w owning columns w, w+8, ... with per-lane
// partials in registers.  The last block finalises column j of H and the
// Givens rotations.
template <typename T, int KPW>
__global__ void __launch_bounds__(kThreads) cgs_pass_b(long long n, long long ld, int ncols, const T* __restrict__ V,
                                                       T* __restrict__ w, double* __restrict__ red, unsigned* counter,
                                                       State st, int j) {
  extern __shared__ unsigned char smraw[];
  double* hs = reinterpret_cast<double*>(smraw);            // ncols coefficients
  double* ws = hs + kMaxCols;                                // kThreads updated w'
  T* Vs = reinterpret_cast<T*>(ws + kThreads);               // ncols x kThreads tile
  __shared__ double ssw[kWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < ncols; i += kThreads) hs[i] = st.hA[i];
  __syncthreads();
  double p[KPW];
#pragma unroll
  for (int k = 0; k < KPW; ++k) p[k] = 0.0;
  double ss = 0.0;
  for (long long base = (long long)blockIdx.x * kThreads; base < n; base += (long long)gridDim.x * kThreads) {
    const long long r = base + threadIdx.x;
    if (r < n) {
      double x = (double)w[r];
#pragma unroll 8
      for (int i = 0; i < ncols; ++i) {
        const T v = __ldcs(V + (size_t)i * ld + r);
        Vs[i * kThreads + threadIdx.x] = v;
        x -= hs[i] * (double)v;
      }
      const T xq = (T)x;
      w[r] = xq;
      ws[threadIdx.x] = (double)xq;
      ss += (double)xq * (double)xq;
    } else {
      for (int i = 0; i < ncols; ++i) Vs[i * kThreads + threadIdx.x] = (T)0;
      ws[threadIdx.x] = 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < KPW; ++k) {
      const int c = warp + k * kWarps;
      if (c < ncols) {
        const T* vc = Vs + c * kThreads;
#pragma unroll
        for (int q = 0; q < kThreads / 32; ++q) p[k] += (double)vc[lane + 32 * q] * ws[lane + 32 * q];
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int k = 0; k < KPW; ++k) {
    const int c = warp + k * kWarps;
    const double t = warp_sum(p[k]);
    if (lane == 0 && c < ncols) red[(size_t)c * gridDim.x + blockIdx.x] = t;
  }
  ss = warp_sum(ss);
  if (lane == 0) ssw[warp] = ss;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
#pragma unroll
    for (int k = 0; k < kWarps; ++k) t += ssw[k];
    red[(size_t)ncols * gridDim.x + blockIdx.x] = t;
  }
  if (!last_block(counter)) return;
  finalize_partials(red, gridDim.x, ncols + 1, st.hB);
  __syncthreads();
  if (threadIdx.x == 0) {
    double ssum = st.hB[ncols], h2n = 0.0;
    for (int i = 0; i < ncols; ++i) {
      st.h(i, j) = st.hA[i] + st.hB[i];
      h2n += st.hB[i] * st.hB[i];
    }
    double b2 = ssum - h2n;
    double beta = b2 > 0.0 ? sqrt(b2) : 0.0;
    st.h(j + 1, j) = beta;
    st.sc[SC_BETA] = beta;
    st.sc[SC_INVB] = beta != 0.0 ? 1.0 / beta : 0.0;
    for (int i = 0; i <= j - 1; ++i) givens_apply(st.cs[i], st.sn[i], st.h(i, j), st.h(i + 1, j));
    givens_make(st.h(j, j), st.h(j + 1, j), st.cs[j], st.sn[j]);
    givens_apply(st.cs[j], st.sn[j], st.h(j, j), st.h(j + 1, j));
    givens_apply(st.cs[j], st.sn[j], st.g[j], st.g[j + 1]);
    st.sc[SC_RES] = fabs(st.g[j + 1]);
  }
}

template <typename T>
size_t pass_b_smem(int ncols) { return (size_t)(kMaxCols + kThreads) * sizeof(double) + (size_t)ncols * kThreads * sizeof(T); }

// ---- pass C: v_{j+1} = (w' - V hB) / beta
template <typename T>
__global__ void __launch_bounds__(kThreads) cgs_pass_c(long long n, long long ld, int ncols, const T* __restrict__ V,
                                                       const T* __restrict__ w, State st, T* __restrict__ vout) {
  const double inv = st.sc[SC_INVB];
  for (long long r = (long long)blockIdx.x * kThreads + threadIdx.x; r < n; r += (long long)gridDim.x * kThreads) {
    double x = (double)w[r];
    for (int i = 0; i < ncols; ++i) x -= st.hB[i] * (double)__ldcs(V + (size_t)i * ld + r);
    vout[r] = (T)(x * inv);
  }
}

// ---- norms, scaling, combination
template <typename T>
__global__ void __launch_bounds__(kThreads) sumsq(long long n, const T* __restrict__ x, double* __restrict__ red,
                                                  unsigned* counter, double* __restrict__ out) {
  extern __shared__ double acc[];
  for (int t = threadIdx.x; t < kWarps; t += kThreads) acc[t] = 0.0;
  __syncthreads();
  double s = 0.0;
  for (long long r = (long long)blockIdx.x * kThreads + threadIdx.x; r < n; r += (long long)gridDim.x * kThreads) {
    double v = (double)x[r];
    s += v * v;
  }
  acc_add(acc, 0, s);
  flush_acc(acc, 1, red);
  if (last_block(counter)) {
    finalize_partials(red, gridDim.x, 1, out);
    __syncthreads();
    if (threadIdx.x == 0) {
      out[0] = sqrt(out[0]);
      out[1] = 1.0 / out[0];  // reference: axpby(n, 1/g[0], r, v0)
    }
  }
}

template <typename S, typename T>
__global__ void scale_into(long long n, const S* __restrict__ x, const double* __restrict__ factor, T* __restrict__ y) {
  const double f = *factor;
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x)
    y[r] = (T)(f * (double)x[r]);
}

template <typename T, typename Y>
__global__ void combine(long long n, long long ld, int ncols, const T* __restrict__ V, const double* __restrict__ y,
                        Y* __restrict__ out) {
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x) {
    double s = y[0] * (double)V[r];
    for (int i = 1; i < ncols; ++i) s = 1.0 * s + y[i] * (double)V[(size_t)i * ld + r];
    out[r] = (Y)s;
  }
}

template <typename X>
__global__ void axpy_into(long long n, const X* __restrict__ z, double* __restrict__ x) {
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x)
    x[r] += (double)z[r];
}

// back substitution g(1:j) = H(1:j,1:j) \ g(1:j)  (rgmres.tpp:95-104)
__global__ void backsolve(State st, int j) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  st.sc[SC_BREAK] = 0.0;
  for (int i = j - 1; i >= 0; --i) {
    if (st.h(i, i) == 0.0) { st.sc[SC_BREAK] = 1.0; return; }
    st.g[i] /= st.h(i, i);
    for (int k = 0; k < i; ++k) st.g[k] -= st.h(k, i) * st.g[i];
  }
}

__global__ void set_g0(State st, const double* norm) { st.g[0] = norm[0]; }

template <typename S, typename D>
__global__ void convert(long long n, const S* __restrict__ a, D* __restrict__ b) {
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x)
    b[r] = (D)a[r];
}

// ------------------------------------------------------------------ driver

template <typename T>
struct Solver {
  deco_ctx_s* ctx;
  deco_csr_s* A;
  deco_cpr_s* P;
  const deco_sol_params& prm;
  long long n, ld;
  int m, nb;
  DevBuf<T> V, w, z;
  DevBuf<double> st_buf, xtmp, r64, norm;
  State st{};

  Solver(deco_ctx_s* c, deco_csr_s* a, deco_cpr_s* p, const deco_sol_params& pr) : ctx(c), A(a), P(p), prm(pr) {
    n = A->n;
    ld = (n + 31) / 32 * 32;
    m = prm.restart;
    nb = 2 * ctx->num_sms;
    cudaStream_t s = ctx->stream;
    V.alloc((size_t)ld * (m + 1), s);
    w.alloc(n, s);
    z.alloc(n, s);
    st_buf.alloc((size_t)(m + 1) * m + 5 * (m + 1) + 16, s);
    xtmp.alloc(n, s);
    r64.alloc(n, s);
    norm.alloc(4, s);
    double* b = st_buf.get();
    st.m = m;
    st.H = b;
    st.g = b + (size_t)(m + 1) * m;
    st.cs = st.g + (m + 1);
    st.sn = st.cs + (m + 1);
    st.hA = st.sn + (m + 1);
    st.hB = st.hA + (m + 1);
    st.sc = st.hB + (m + 1);
    size_t need = (size_t)(m + 2) * nb;
    if (ctx->red.size() < need) ctx->red.alloc(need, s);
    DECO_CUDA(cudaFuncSetAttribute(cgs_pass_b<T, kColsPerWarp>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)pass_b_smem<T>(kMaxCols)));
  }

  int grid() const { return nb; }

  // y = M^{-1} x
  template <typename X, typename Y>
  void precond(const X* x, Y* y) {
    if (!P) {
      convert<X, Y><<<grid(), kThreads, 0, ctx->stream>>>(n, x, y);
      DECO_CHECK_LAUNCH();
      return;
    }
    if (P->prm.precision == 32) {
      if constexpr (std::is_same<X, double>::value && std::is_same<Y, double>::value) cpr_apply32<double, double>(ctx, P, x, y);
      else if constexpr (std::is_same<X, double>::value && std::is_same<Y, float>::value) cpr_apply32<double, float>(ctx, P, x, y);
      else if constexpr (std::is_same<X, float>::value && std::is_same<Y, float>::value) cpr_apply32<float, float>(ctx, P, x, y);
      else throw Error(DECO_ERR_INTERNAL, "unsupported precision combination");
    } else {
      if constexpr (std::is_same<X, double>::value && std::is_same<Y, double>::value) cpr_apply64(ctx, P, x, y);
      else throw Error(DECO_ERR_UNSUPPORTED, "precision-32 solve needs a CPR built with precision 32");
    }
  }

  // y = A x in the basis precision
  template <typename X>
  void matvec(const X* x, T* y) {
    if constexpr (std::is_same<T, float>::value) spmv<float, X>(ctx, A, x, EpiStore<float>{y});
    else spmv<double, X>(ctx, A, x, EpiStore<double>{y});
  }

  template <typename X>
  double norm2(const X* x) {
    size_t sm = kWarps * sizeof(double);
    sumsq<X><<<grid(), kThreads, sm, ctx->stream>>>(n, x, ctx->red.get(), ctx->counter.get(), norm.get());
    DECO_CHECK_LAUNCH();
    double h = 0;
    DECO_CUDA(cudaMemcpyAsync(&h, norm.get(), sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    DECO_CUDA(cudaStreamSynchronize(ctx->stream));
    return h;
  }

  T* col(int i) { return V.get() + (size_t)i * ld; }

  void run(const double* b, double* x, deco_sol_result* res, double* resvec) {
    cudaStream_t s = ctx->stream;
    const bool left = prm.type == 1;
    const int itmax = prm.itmax;
    const int g = grid();
    double* r = r64.get();
    DECO_CUDA(cudaEventRecord(ctx->ev0, s));
    // initial residual
    if (!prm.use_x0) {
      DECO_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, s));
      if (left) precond<double, double>(b, r);
      else DECO_CUDA(cudaMemcpyAsync(r, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    } else {
      spmv<double, double>(ctx, A, x, EpiResid<double, double>{b, left ? xtmp.get() : r});
      if (left) precond<double, double>(xtmp.get(), r);
    }
    const double bnorm = left ? norm2(r) : norm2(b);
    const double abstol = prm.reltol * bnorm;
    int flag = 1, iter = 0, restarts = 0;
    double rnorm = 0.0;
    double* hsc = ctx->host_scalars;
    while (iter < itmax) {
      DECO_CUDA(cudaMemsetAsync(st_buf.get(), 0, sizeof(double) * ((size_t)(m + 1) * m + 5 * (m + 1) + 16), s));
      double g0 = norm2(r);
      set_g0<<<1, 1, 0, s>>>(st, norm.get());
      scale_into<double, T><<<g, kThreads, 0, s>>>(n, r, norm.get() + 1, col(0));
      DECO_CHECK_LAUNCH();
      int j = 0;
      double gj = g0;
      while (j < m && iter < itmax) {
        rnorm = fabs(gj);
        if (resvec) resvec[iter] = rnorm / bnorm;
        if (rnorm < abstol) { flag = 0; break; }
        if (!left) {
          precond<T, T>(col(j), z.get());
          matvec<T>(z.get(), w.get());
        } else {
          matvec<T>(col(j), z.get());
          precond<T, T>(z.get(), w.get());
        }
        const int nc = j + 1;
        cgs_pass_a<T, kColsPerWarp><<<g, kThreads, 0, s>>>(n, ld, nc, V.get(), w.get(), ctx->red.get(),
                                                           ctx->counter.get(), st.hA);
        DECO_CHECK_LAUNCH();
        cgs_pass_b<T, kColsPerWarp><<<g, kThreads, pass_b_smem<T>(nc), s>>>(n, ld, nc, V.get(), w.get(),
                                                                           ctx->red.get(), ctx->counter.get(), st, j);
        DECO_CHECK_LAUNCH();
        cgs_pass_c<T><<<g * 4, kThreads, 0, s>>>(n, ld, nc, V.get(), w.get(), st, col(j + 1));
        DECO_CHECK_LAUNCH();
        DECO_CUDA(cudaMemcpyAsync(hsc, st.sc + SC_RES, sizeof(double), cudaMemcpyDeviceToHost, s));
        DECO_CUDA(cudaStreamSynchronize(s));
        gj = hsc[0];
        ++j;
        ++iter;
      }
      backsolve<<<1, 1, 0, s>>>(st, j);
      DECO_CHECK_LAUNCH();
      DECO_CUDA(cudaMemcpyAsync(hsc, st.sc + SC_BREAK, sizeof(double), cudaMemcpyDeviceToHost, s));
      DECO_CUDA(cudaStreamSynchronize(s));
      if (hsc[0] != 0.0)
        throw Error(DECO_ERR_BREAKDOWN, "Error in rgmres: Zero diagonal element in upper triangular matrix.");
      combine<T, double><<<g * 4, kThreads, 0, s>>>(n, ld, j > 0 ? j : 1, V.get(), st.g, xtmp.get());
      DECO_CHECK_LAUNCH();
      if (!left) {
        precond<double, double>(xtmp.get(), r);  // r used as scratch for z
        axpy_into<double><<<g * 4, kThreads, 0, s>>>(n, r, x);
        DECO_CHECK_LAUNCH();
        spmv<double, double>(ctx, A, x, EpiResid<double, double>{b, r});
      } else {
        axpy_into<double><<<g * 4, kThreads, 0, s>>>(n, xtmp.get(), x);
        DECO_CHECK_LAUNCH();
        spmv<double, double>(ctx, A, x, EpiResid<double, double>{b, xtmp.get()});
        precond<double, double>(xtmp.get(), r);
      }
      ++restarts;
      rnorm = norm2(r);
      if (rnorm < abstol) { flag = 0; break; }
    }
    DECO_CUDA(cudaEventRecord(ctx->ev1, s));
    DECO_CUDA(cudaEventSynchronize(ctx->ev1));
    float ms = 0.f;
    DECO_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    res->iter = iter;
    res->flag = flag;
    res->res_abs = rnorm;
    res->res_rel = rnorm / bnorm;
    res->t_solve_ms = ms;
    res->restarts = restarts;
    if (prm.verbosity > 0) {
      std::printf("\n--------------------------------\n");
      std::printf("Profile of %s:\n", left ? "lGMRES" : "rGMRES");
      std::printf("iteration count =  %d\n", iter);
      std::printf("residual = %.2e\n", rnorm / bnorm);
    }
  }
};

}  // namespace

}  // namespace deco

using namespace deco;

extern "C" {

int deco_gmres_solve(deco_ctx ctx, deco_csr A, deco_cpr P, const double* b, double* x, const deco_sol_params* prm,
                     deco_sol_result* res, double* resvec) {
  return guard([&] {
    DECO_REQUIRE(ctx && A && b && x && prm && res, DECO_ERR_ARG, "NULL argument");
    DECO_REQUIRE(prm->type == 0 || prm->type == 1, DECO_ERR_ARG, "type must be 0 (rgmres) or 1 (lgmres)");
    DECO_REQUIRE(prm->restart >= 1, DECO_ERR_ARG, "restart must be >= 1");
    DECO_REQUIRE(prm->restart < kMaxCols, DECO_ERR_UNSUPPORTED,
                 "restart must be < " + std::to_string(kMaxCols) + " on this path");
    DECO_REQUIRE(prm->itmax >= 0, DECO_ERR_ARG, "itmax must be >= 0");
    DECO_REQUIRE(prm->precision == 64 || prm->precision == 32, DECO_ERR_ARG, "precision must be 64 or 32");
    DECO_REQUIRE(A->n == A->m, DECO_ERR_ARG, "A must be square");
    if (P) DECO_REQUIRE(P->n == A->n, DECO_ERR_ARG, "preconditioner size does not match A");
    if (prm->precision == 32) {
      DECO_REQUIRE(!P || P->prm.precision == 32, DECO_ERR_ARG, "precision-32 solve needs a CPR built with precision 32");
      if (!A->v32) make_f32_values(ctx, A);
      Solver<float> S(ctx, A, P, *prm);
      S.run(b, x, res, resvec);
    } else {
      Solver<double> S(ctx, A, P, *prm);
      S.run(b, x, res, resvec);
    }
  });
}

}  // extern "C"
