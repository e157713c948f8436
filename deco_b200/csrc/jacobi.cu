// jacobi.cu — setup of the point / block Jacobi preconditioner (Jacobi.tpp).
#include "jacobi.cuh"

namespace deco {

namespace {

__device__ __forceinline__ int find_diag(const int* __restrict__ c, int lo, int hi, int target) {
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (c[mid] > target) hi = mid; else lo = mid;
  }
  return lo;
}

// one thread per cell: gather the diagonal block as Jacobi::blocked does
// (Jacobi.tpp:49-60: entries around the diagonal position that fall in the
// cell's columns, row-major), then invert it by Gauss-Jordan with partial
// pivoting.  bs == 1: 1 / a_ii (Jacobi::classic, Jacobi.tpp:3-21).
template <int BS>
__global__ void jacobi_setup(int sn, const int* __restrict__ r, const int* __restrict__ c,
                             const double* __restrict__ v, double* __restrict__ J, int* __restrict__ err) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < sn; s += gridDim.x * blockDim.x) {
    double B[BS][BS], X[BS][BS];
    for (int p = 0; p < BS; ++p)
      for (int k = 0; k < BS; ++k) { B[p][k] = 0.0; X[p][k] = p == k ? 1.0 : 0.0; }
    for (int p = 0; p < BS; ++p) {
      const int i = s * BS + p, ia = r[i], ib = r[i + 1];
      if (ib <= ia) continue;
      const int j = find_diag(c, ia, ib, i);
      if constexpr (BS == 1) {
        B[0][0] = v[j];
      } else {
        for (int k = 0; k < BS; ++k) {
          const int q = j + k - p;
          if (q < ia || q >= ib) continue;
          if (c[q] / BS == s) B[p][c[q] % BS] = v[q];
        }
      }
    }
    double* out = J + (long long)s * BS * BS;
    if constexpr (BS == 1) {  // no check, as Jacobi::classic: a zero diagonal gives inf
      out[0] = 1.0 / B[0][0];
      continue;
    }
    bool singular = false;
    for (int col = 0; col < BS; ++col) {
      int piv = col;
      for (int q = col + 1; q < BS; ++q)
        if (fabs(B[q][col]) > fabs(B[piv][col])) piv = q;
      if (B[piv][col] == 0.0) { singular = true; break; }
      if (piv != col)
        for (int k = 0; k < BS; ++k) {
          double t = B[col][k]; B[col][k] = B[piv][k]; B[piv][k] = t;
          t = X[col][k]; X[col][k] = X[piv][k]; X[piv][k] = t;
        }
      const double inv = 1.0 / B[col][col];
      for (int k = 0; k < BS; ++k) { B[col][k] *= inv; X[col][k] *= inv; }
      for (int q = 0; q < BS; ++q) {
        if (q == col) continue;
        const double f = B[q][col];
        if (f == 0.0) continue;
        for (int k = 0; k < BS; ++k) { B[q][k] -= f * B[col][k]; X[q][k] -= f * X[col][k]; }
      }
    }
    if (singular) atomicExch(err, 1);
    for (int p = 0; p < BS; ++p)
      for (int k = 0; k < BS; ++k) out[p * BS + k] = X[p][k];
  }
}

__global__ void jacobi_to_f32(const double* __restrict__ a, float* __restrict__ b, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

}  // namespace

void jacobi_build(deco_ctx_s* ctx, const deco_csr_s* A, int bs, int precision, deco_jacobi_s* J) {
  DECO_REQUIRE(bs >= 1 && bs <= 3, DECO_ERR_UNSUPPORTED, "Jacobi block_size must be 1, 2 or 3");
  DECO_REQUIRE(A->n == A->m, DECO_ERR_ARG, "Jacobi needs a square matrix");
  DECO_REQUIRE(A->n % bs == 0, DECO_ERR_ARG, "n is not divisible by the Jacobi block_size");
  cudaStream_t st = ctx->stream;
  J->bs = bs;
  J->n = A->n;
  J->sn = A->n / bs;
  const long long nv = (long long)J->sn * bs * bs;
  J->J.alloc(nv, st);
  DevBuf<int> err(1, st);
  err.zero(st);
  const int g = grid_for(ctx, J->sn, 128, 16);
  switch (bs) {
    case 1: jacobi_setup<1><<<g, 128, 0, st>>>(J->sn, A->r.get(), A->c.get(), A->v.get(), J->J.get(), err.get()); break;
    case 2: jacobi_setup<2><<<g, 128, 0, st>>>(J->sn, A->r.get(), A->c.get(), A->v.get(), J->J.get(), err.get()); break;
    default: jacobi_setup<3><<<g, 128, 0, st>>>(J->sn, A->r.get(), A->c.get(), A->v.get(), J->J.get(), err.get()); break;
  }
  DECO_CHECK_LAUNCH();
  if (precision == 32) {
    J->J32.alloc(nv, st);
    jacobi_to_f32<<<grid_for(ctx, nv, 256), 256, 0, st>>>(J->J.get(), J->J32.get(), nv);
    DECO_CHECK_LAUNCH();
  }
  int h = 0;
  DECO_CUDA(cudaMemcpyAsync(&h, err.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
  DECO_CUDA(cudaStreamSynchronize(st));
  DECO_REQUIRE(h == 0, DECO_ERR_SINGULAR, "singular diagonal block in Jacobi setup");
}

}  // namespace deco
