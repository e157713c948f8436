// batch.cu — many independent systems, each with K right-hand sides, solved
// together (no counterpart in the reference, which solves one system).
//
// Layout.  The systems are one block-diagonal matrix (system q owns rows
// [row_off[q], row_off[q+1]) and only references its own columns), so ONE CPR
// setup on it is the per-system setups at once: every decoupling, extraction
// and FSAI step is row- or cell-local, and the FSAI local systems of all
// systems are solved in the same launch grouped by order.  Right-hand sides
// and iterates are row-interleaved multi-vectors X[row * K + k] (multi.cuh),
// so each product reads the matrix once for all K columns.
//
// Solve.  One right-preconditioned GMRES(m) per (system, column) instance,
// advanced in lockstep: the products and preconditioner applies run on all
// instances at once; the Arnoldi dots are segmented by system (row chunks never
// straddle two systems) and reduced per instance in a fixed order, so results do
// not depend on scheduling.  Each instance follows the single-system algorithm of
// gmres.cu — CGS2 with the second projection from the Gram matrix, lazy
// normalisation, the reference's Givens formulas (rgmres.tpp:141-160), its inner
// and outer convergence checks and its iteration limit — and stops contributing
// once converged.  A whole restart cycle (m Arnoldi steps, the back
// substitution, the solution update and the true residual) is captured once in a
// CUDA graph that runs inside a device-side while loop (a conditional graph
// node), so the whole solve is one graph launch.  Systems whose instances have
// all finished are skipped by the products, dots and updates of the inner steps.
#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <type_traits>
#include <vector>

#include "cpr.cuh"
#include "multi.cuh"

namespace deco {

namespace {

constexpr int kT = 256;            // threads per block of the batch kernels
constexpr int kChunkRows = 4096;   // rows per dot chunk (chunks never cross systems)
// blocks of the update pass per chunk (one per chunk left the 512-instance batch
// with five and a fraction waves of long blocks, and small batches with a part of
// the GPU; measured on 8 systems of 30k-100k cells: 211 blocks, 35 % of the DRAM
// peak)
constexpr int kUpdSub = 4;
constexpr double kEpsB = 2.220446049250312e-16;
// largest restart length: the kernels keep one coefficient per (basis column,
// right-hand side) in dynamic shared memory, K (m + 1) doubles (32 KB at m = 512
// and K = 8, under the 48 KB a block gets without opting in)
constexpr int kMaxRestartB = 512;

// per-instance state, `stride` doubles each: H (m+1)m | G (m+1)^2 | g | cs | sn | s | c | misc
struct BState {
  double* base;
  long long stride;
  int m;
  __host__ __device__ static long long doubles(int m) {
    return (long long)(m + 1) * m + (long long)(m + 1) * (m + 1) + 5LL * (m + 1) + 16;
  }
  __device__ double* q(int i) const { return base + (long long)i * stride; }
  __device__ double& H(int qi, int i, int j) const { return q(qi)[i + (long long)j * (m + 1)]; }
  __device__ double& G(int qi, int i, int j) const { return q(qi)[(long long)(m + 1) * m + i + (long long)j * (m + 1)]; }
  __device__ double* g(int qi) const { return q(qi) + (long long)(m + 1) * m + (long long)(m + 1) * (m + 1); }
  __device__ double* cs(int qi) const { return g(qi) + (m + 1); }
  __device__ double* sn(int qi) const { return cs(qi) + (m + 1); }
  __device__ double* s(int qi) const { return sn(qi) + (m + 1); }
  __device__ double* c(int qi) const { return s(qi) + (m + 1); }
  // misc: [0] |g| of the last step, [1] steps taken this cycle, [2] converged-at step (-1 none),
  // [3] basis columns the solution update combines
  __device__ double* misc(int qi) const { return c(qi) + (m + 1); }
  // host-side offset of s (for the scaled-product epilogue)
  __host__ static long long s_offset(int m) { return (long long)(m + 1) * m + (long long)(m + 1) * (m + 1) + 3LL * (m + 1); }
};

// per-instance integer status
struct Inst {
  int* active;     // 1 while the instance runs Arnoldi steps in this cycle
  int* done;       // 1 once the outer check passed or the iteration limit was hit
  int* iters;      // inner iterations so far
  int* flag;       // 0 converged, 1 not
  double* bnorm;   // ||b|| of the decoupled right-hand side
  double* res;     // last true residual norm
  int* sys_active; // per system: any instance still active in this cycle
  int* remaining;  // [0] number of unfinished instances
};

// ---- chunk helpers: chunk c covers rows [crow[c], crow[c+1]) of system csys[c]
__device__ __forceinline__ bool chunk_live(const int* csys, const int* sys_active, int c) {
  return sys_active[csys[c]] != 0;
}

// sum over rows of a chunk for each k: threads are (row-in-tile, k) pairs
template <int K>
__device__ __forceinline__ void reduce_k(double v, double* smem_k, double* out_k) {
  // lanes with the same k: xor over the row bits of the lane (K divides 32)
#pragma unroll
  for (int o = 16; o >= K; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane < K) smem_k[warp * K + lane] = v;
  __syncthreads();
  if (threadIdx.x < K) {
    double t = 0.0;
    for (int w = 0; w < kT / 32; ++w) t += smem_k[w * K + threadIdx.x];
    *out_k = t;
  }
  __syncthreads();
}

// ---- cycle start: u0 = r (basis precision), partial ||r||^2 and ||u0||^2 per (chunk, k)
template <int K, typename T>
__global__ void __launch_bounds__(kT) b_start(const int* crow, const int* csys, Inst in, const double* __restrict__ r,
                                              T* __restrict__ u0, double* __restrict__ red, int nchunk) {
  __shared__ double sm[(kT / 32) * K];
  const int c = blockIdx.x;
  if (!chunk_live(csys, in.sys_active, c)) {
    if (threadIdx.x < K) { red[(long long)threadIdx.x * nchunk + c] = 0.0; red[(long long)(K + threadIdx.x) * nchunk + c] = 0.0; }
    return;
  }
  const long long e0 = (long long)crow[c] * K, e1 = (long long)crow[c + 1] * K;
  double ss = 0.0, sq = 0.0;
  for (long long e = e0 + threadIdx.x; e < e1; e += kT) {
    const double v = r[e];
    const T t = (T)v;
    u0[e] = t;
    ss += v * v;
    sq += (double)t * (double)t;
  }
  const int k = threadIdx.x % K;
  double o1, o2;
  reduce_k<K>(ss, sm, &o1);
  if (threadIdx.x < K) red[(long long)k * nchunk + c] = o1;
  reduce_k<K>(sq, sm, &o2);
  if (threadIdx.x < K) red[(long long)(K + k) * nchunk + c] = o2;
}

// one thread per instance: g0, s0, and the inner check at j = 0 (rgmres.tpp:58-63)
template <int K>
__global__ void b_start_fin(int Q, const int* sch, BState st, Inst in, const double* __restrict__ red, int nchunk,
                            double reltol, int itmax) {
  const int qi = blockIdx.x * blockDim.x + threadIdx.x;
  if (qi >= Q) return;
  const int sys = qi / K, k = qi % K;
  double* g = st.g(qi);
  double* misc = st.misc(qi);
  misc[1] = 0.0;
  misc[2] = -1.0;
  // the rotations read g_{j+1} before writing it (rgmres.tpp:86): it starts at zero every cycle
  for (int i = 1; i <= st.m; ++i) g[i] = 0.0;
  if (in.done[qi]) { in.active[qi] = 0; return; }
  double ss = 0.0, sq = 0.0;
  for (int c = sch[sys]; c < sch[sys + 1]; ++c) {
    ss += red[(long long)k * nchunk + c];
    sq += red[(long long)(K + k) * nchunk + c];
  }
  const double nrm = sqrt(ss), nq = sqrt(sq);
  g[0] = nrm;
  st.s(qi)[0] = nq != 0.0 ? 1.0 / nq : 0.0;
  misc[0] = nrm;
  const bool run = in.iters[qi] < itmax;
  if (!(nrm < reltol * in.bnorm[qi]) && run) {
    in.active[qi] = 1;
  } else {
    in.active[qi] = 0;
    if (run) { misc[2] = 0.0; in.flag[qi] = 0; }  // converged before step 0 of this cycle
  }
}

__global__ void b_sys_all(int nsys, int* sys_active) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nsys) sys_active[i] = 1;
}

__global__ void fill_cell_sys(int nsys, const int* __restrict__ cell_off, int* __restrict__ cell_sys) {
  for (int q = blockIdx.x; q < nsys; q += gridDim.x)
    for (int c = cell_off[q] + threadIdx.x; c < cell_off[q + 1]; c += blockDim.x) cell_sys[c] = q;
}

// per system: any instance active?
template <int K>
__global__ void b_sys_active(int nsys, Inst in) {
  const int sys = blockIdx.x * blockDim.x + threadIdx.x;
  if (sys >= nsys) return;
  int a = 0;
  for (int k = 0; k < K; ++k) a |= in.active[sys * K + k];
  in.sys_active[sys] = a;
}

// ---- vector access for the dot and update passes: a thread moves Ev consecutive
// elements of a multi-vector per load (16 bytes when K allows: float4 / double2),
// all of one row, so they belong to instances Ev*p .. Ev*p + Ev - 1 where the
// phase p = (element / Ev) % (K / Ev) is fixed for a thread over its whole sweep.
template <typename T, int E> struct VecN;
template <> struct VecN<float, 4> { using t = float4; };
template <> struct VecN<float, 2> { using t = float2; };
template <> struct VecN<float, 1> { using t = float; };
template <> struct VecN<double, 2> { using t = double2; };
template <> struct VecN<double, 1> { using t = double; };

template <typename T, int E>
__device__ __forceinline__ void vload(const T* __restrict__ p, double* o, bool stream) {
  using V = typename VecN<T, E>::t;
  const V v = stream ? __ldcs(reinterpret_cast<const V*>(p)) : __ldg(reinterpret_cast<const V*>(p));
  if constexpr (E == 1) {
    o[0] = (double)v;
  } else {
    const T* e = reinterpret_cast<const T*>(&v);
#pragma unroll
    for (int q = 0; q < E; ++q) o[q] = (double)e[q];
  }
}
template <int E>
__device__ __forceinline__ void vload_f32(const float* __restrict__ p, float* o, bool stream) {
  using V = typename VecN<float, E>::t;
  const V v = stream ? __ldcs(reinterpret_cast<const V*>(p)) : __ldg(reinterpret_cast<const V*>(p));
  if constexpr (E == 1) {
    o[0] = v;
  } else {
    const float* e = reinterpret_cast<const float*>(&v);
#pragma unroll
    for (int q = 0; q < E; ++q) o[q] = e[q];
  }
}
template <typename T, int E>
__device__ __forceinline__ void vstore(T* p, const T* o) {
  using V = typename VecN<T, E>::t;
  *reinterpret_cast<V*>(p) = *reinterpret_cast<const V*>(o);
}

template <int K, typename T> struct VShape {
  static constexpr int E = (16 / (int)sizeof(T)) < K ? (16 / (int)sizeof(T)) : K;  // elements per load
  static constexpr int P = K / E;                                                  // phases
  static constexpr int G = 16 / E;                                                 // columns per dot block
};

// Sums acc[s] (s < NS slots) over the block's threads of equal phase, in a fixed
// order; returns in `out` (shared, [P][NS]) the totals per (phase, slot).
template <int P, int NS>
__device__ __forceinline__ void reduce_phase(const double* acc, double* part /* [kT/32][P][NS] */, int phase0,
                                             double* out /* [P][NS] */) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int s2 = 0; s2 < NS; ++s2) {
    double v = acc[s2];
#pragma unroll
    for (int o = 16; o >= P; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane < P) part[(warp * P + (phase0 + lane) % P) * NS + s2] = v;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < P * NS; t += blockDim.x) {
    double sum = 0.0;
    for (int w = 0; w < kT / 32; ++w) sum += part[w * P * NS + t];
    out[t] = sum;
  }
  __syncthreads();
}

// ---- pass A (vectorised): raw dots u_i . w and u_i . u_j for the block's group of
// G columns, per (chunk, instance)
template <int K, typename T, int G>
__global__ void __launch_bounds__(kT) b_dots_v(const int* crow, const int* csys, Inst in, long long ld, int j,
                                               const T* __restrict__ V, const T* __restrict__ w,
                                               double* __restrict__ red, int nchunk) {
  using S = VShape<K, T>;
  constexpr int E = S::E, P = S::P, NS = 2 * E * G;
  __shared__ double part[(kT / 32) * P * NS];
  __shared__ double tot[P * NS];
  // the column groups of a chunk are adjacent in launch order, so the chunk's w
  // and u_j, which every group reads, are still in L2 for the later groups
  const int c = blockIdx.y, i0 = blockIdx.x * G;
  const int ni = min(G, j + 1 - i0);
  const bool live = chunk_live(csys, in.sys_active, c);
  const long long f0 = (long long)crow[c] * K / E, f1 = (long long)crow[c + 1] * K / E;
  double acc[NS];
#pragma unroll
  for (int t = 0; t < NS; ++t) acc[t] = 0.0;
  if (live) {
    const T* __restrict__ uj = V + (long long)j * ld;
    if constexpr (std::is_same<T, float>::value) {
      // float32 basis: a thread's vectors f and f + kT hold the same instances
      // (kT is a multiple of the phase count), so each instance's two products
      // are summed in float32 and converted once (no widening of w and u_j, a
      // quarter of the conversions, two rows' loads in flight per thread)
      for (long long f = f0 + threadIdx.x; f < f1; f += 2 * kT) {
        const long long g = f + kT;
        const bool two = g < f1;
        float wa[E], ua[E], wb[E], ub[E];
        vload_f32<E>(w + f * E, wa, false);
        vload_f32<E>(uj + f * E, ua, false);
        if (two) {
          vload_f32<E>(w + g * E, wb, false);
          vload_f32<E>(uj + g * E, ub, false);
        } else {
#pragma unroll
          for (int q = 0; q < E; ++q) { wb[q] = 0.f; ub[q] = 0.f; }
        }
#pragma unroll
        for (int t = 0; t < G; ++t) {
          if (t < ni) {  // uniform over the block
            const float* col = V + (long long)(i0 + t) * ld;
            float va[E], vb[E];
            vload_f32<E>(col + f * E, va, true);
            if (two) vload_f32<E>(col + g * E, vb, true);
            else {
#pragma unroll
              for (int q = 0; q < E; ++q) vb[q] = 0.f;
            }
#pragma unroll
            for (int q = 0; q < E; ++q) {
              acc[t * E + q] += (double)fmaf(vb[q], wb[q], va[q] * wa[q]);
              acc[(G + t) * E + q] += (double)fmaf(vb[q], ub[q], va[q] * ua[q]);
            }
          }
        }
      }
    } else {
      for (long long f = f0 + threadIdx.x; f < f1; f += kT) {
        double wv[E], uv[E];
        vload<T, E>(w + f * E, wv, false);
        vload<T, E>(uj + f * E, uv, false);
#pragma unroll
        for (int t = 0; t < G; ++t) {
          if (t < ni) {  // uniform over the block
            double v[E];
            vload<T, E>(V + (long long)(i0 + t) * ld + f * E, v, true);
#pragma unroll
            for (int q = 0; q < E; ++q) {
              acc[t * E + q] += v[q] * wv[q];
              acc[(G + t) * E + q] += v[q] * uv[q];
            }
          }
        }
      }
    }
  }
  reduce_phase<P, NS>(acc, part, (int)(f0 % P), tot);
  const int nc = j + 1;
  for (int t2 = threadIdx.x; t2 < P * NS; t2 += kT) {
    const int ph = t2 / NS, sl = t2 % NS;
    const int gram = sl / (G * E), t = (sl / E) % G, q = sl % E;
    if (t >= ni) continue;
    const int k = E * ph + q;
    const int col = (gram ? nc : 0) + i0 + t;
    red[((long long)col * K + k) * nchunk + c] = live ? tot[t2] : 0.0;
  }
}

// ---- pass B (vectorised): u_{j+1} = w - sum_i c_i u_i; partial ||u_{j+1}||^2 per instance
template <int K, typename T>
__global__ void __launch_bounds__(kT) b_update_v(const int* crow, const int* csys, BState st, Inst in, long long ld,
                                                 int j, const T* __restrict__ V, const T* __restrict__ w,
                                                 T* __restrict__ out, double* __restrict__ red, int nchunk) {
  using S = VShape<K, T>;
  constexpr int E = S::E, P = S::P;
  extern __shared__ double cf_u[];  // [nc][K] coefficients
  __shared__ double part[(kT / 32) * P * E];
  __shared__ double tot[P * E];
  // blockIdx.y = sub-block: kUpdSub blocks share a chunk (interleaved vectors), so
  // the grid has enough blocks to even out across the SMs; each writes its own
  // partials, the finishing kernel sums them in a fixed order
  const int c = blockIdx.x, sub = blockIdx.y, sys = csys[c], nc = j + 1;
  double* __restrict__ redp = red + (long long)sub * K * nchunk;
  if (!in.sys_active[sys]) {
    if (threadIdx.x < K) redp[(long long)threadIdx.x * nchunk + c] = 0.0;
    return;
  }
  for (int t = threadIdx.x; t < K * nc; t += kT) {
    const int i = t / K, kk = t % K, qi = sys * K + kk;
    cf_u[i * K + kk] = in.active[qi] ? st.c(qi)[i] : 0.0;
  }
  __syncthreads();
  const long long f0 = (long long)crow[c] * K / E, f1 = (long long)crow[c + 1] * K / E;
  const long long fs = f0 + (long long)sub * kT;  // this sub-block's first vector
  const int ph = (int)((fs + threadIdx.x) % P);
  double ss[E];
#pragma unroll
  for (int q = 0; q < E; ++q) ss[q] = 0.0;
  // the columns go in batches of UB whose loads are all issued before their
  // products (UB independent loads per thread in flight; each element still
  // subtracts the columns in order)
  constexpr int UB = sizeof(T) == 4 ? 16 : 8;
  for (long long f = fs + threadIdx.x; f < f1; f += (long long)kUpdSub * kT) {
    double x[E];
    vload<T, E>(w + f * E, x, false);
    int i = 0;
    for (; i + UB <= nc; i += UB) {
      double v[UB][E];
#pragma unroll
      for (int u = 0; u < UB; ++u) vload<T, E>(V + (long long)(i + u) * ld + f * E, v[u], true);
#pragma unroll
      for (int u = 0; u < UB; ++u)
#pragma unroll
        for (int q = 0; q < E; ++q) x[q] -= cf_u[(i + u) * K + E * ph + q] * v[u][q];
    }
    for (; i < nc; ++i) {
      double v[E];
      vload<T, E>(V + (long long)i * ld + f * E, v, true);
#pragma unroll
      for (int q = 0; q < E; ++q) x[q] -= cf_u[i * K + E * ph + q] * v[q];
    }
    T o[E];
#pragma unroll
    for (int q = 0; q < E; ++q) {
      o[q] = (T)x[q];
      ss[q] += (double)o[q] * (double)o[q];
    }
    vstore<T, E>(out + f * E, o);
  }
  reduce_phase<P, E>(ss, part, (int)(fs % P), tot);
  for (int t2 = threadIdx.x; t2 < P * E; t2 += kT) redp[(long long)t2 * nchunk + c] = tot[t2];
}

// one warp per instance: h, the Gram row of u_j, c = h + (h - G h), H(:,j), coefficients
// (dynamic shared memory: (kT / 32) (j + 1) doubles, h of each warp's instance)
template <int K>
__global__ void b_dots_fin(int Q, const int* sch, BState st, Inst in, int j, const double* __restrict__ red,
                           int nchunk) {
  extern __shared__ double hs_f[];
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  double* hw = hs_f + (size_t)wl * (j + 1);
  const int qi = blockIdx.x * (kT / 32) + wl;
  if (qi >= Q || !in.active[qi]) return;
  const int sys = qi / K, k = qi % K, nc = j + 1;
  const double* s = st.s(qi);
  const double sj = s[j];
  for (int i = lane; i < nc; i += 32) {
    double a = 0.0, b = 0.0;
    for (int c = sch[sys]; c < sch[sys + 1]; ++c) {
      a += red[((long long)i * K + k) * nchunk + c];
      b += red[((long long)(nc + i) * K + k) * nchunk + c];
    }
    hw[i] = a * s[i];
    const double gij = s[i] * sj * b;
    st.G(qi, i, j) = gij;
    st.G(qi, j, i) = gij;
  }
  __syncwarp();
  for (int i = lane; i < nc; i += 32) {
    double gh = 0.0;
    for (int t = 0; t < nc; ++t) gh += st.G(qi, i, t) * hw[t];
    const double ci = hw[i] + (hw[i] - gh);
    st.H(qi, i, j) = ci;
    st.c(qi)[i] = ci * s[i];
  }
}

__device__ void b_givens_make(double x, double y, double& c, double& s) {
  if (fabs(y) < kEpsB) { c = 1.0; s = 0.0; }
  else if (fabs(y) > fabs(x)) { double nu = x / y; s = 1.0 / sqrt(1.0 + nu * nu); c = nu * s; }
  else { double nu = y / x; c = 1.0 / sqrt(1.0 + nu * nu); s = nu * c; }
}
__device__ void b_givens_apply(double c, double s, double& dx, double& dy) {
  double t = c * dx + s * dy;
  dy = -s * dx + c * dy;
  dx = t;
}

// one thread per instance: H(j+1,j), s_{j+1}, the rotations, |g_{j+1}|, the inner check
template <int K>
__global__ void b_update_fin(int Q, const int* sch, BState st, Inst in, int j, const double* __restrict__ red,
                             int nchunk, double reltol, int itmax) {
  const int qi = blockIdx.x * blockDim.x + threadIdx.x;
  if (qi >= Q || !in.active[qi]) return;
  const int sys = qi / K, k = qi % K;
  double ss = 0.0;
  for (int c = sch[sys]; c < sch[sys + 1]; ++c)
#pragma unroll
    for (int sub = 0; sub < kUpdSub; ++sub) ss += red[((long long)sub * K + k) * nchunk + c];
  const double beta = sqrt(ss);
  st.H(qi, j + 1, j) = beta;
  st.s(qi)[j + 1] = beta != 0.0 ? 1.0 / beta : 0.0;
  double* cs = st.cs(qi);
  double* sn = st.sn(qi);
  double* g = st.g(qi);
  for (int i = 0; i <= j - 1; ++i) b_givens_apply(cs[i], sn[i], st.H(qi, i, j), st.H(qi, i + 1, j));
  b_givens_make(st.H(qi, j, j), st.H(qi, j + 1, j), cs[j], sn[j]);
  b_givens_apply(cs[j], sn[j], st.H(qi, j, j), st.H(qi, j + 1, j));
  b_givens_apply(cs[j], sn[j], g[j], g[j + 1]);
  double* misc = st.misc(qi);
  misc[0] = fabs(g[j + 1]);
  misc[1] = j + 1;
  in.iters[qi] += 1;
  // the reference checks |g_{j+1}| at the top of the next step, if there is one
  // (rgmres.tpp:58-66): inside the cycle and below the iteration limit
  if (j + 1 < st.m && in.iters[qi] < itmax) {
    if (fabs(g[j + 1]) < reltol * in.bnorm[qi]) {
      misc[2] = j + 1;
      in.flag[qi] = 0;
      in.active[qi] = 0;
    }
  } else {
    in.active[qi] = 0;  // cycle full or limit reached: the restart decides
  }
}

// ---- cycle end: back substitution (rgmres.tpp:95-104) and coefficients c_i = y_i s_i;
// instances that took no part in the cycle get zero coefficients.
template <int K>
__global__ void b_backsolve(int Q, BState st, Inst in, int* breakdown) {
  const int qi = blockIdx.x * blockDim.x + threadIdx.x;
  if (qi >= Q) return;
  double* c = st.c(qi);
  const int m = st.m;
  for (int i = 0; i <= m; ++i) c[i] = 0.0;
  double* misc = st.misc(qi);
  misc[3] = 0.0;  // columns the combination reads for this instance
  if (in.done[qi]) return;
  const int j = misc[2] >= 0.0 ? (int)misc[2] : (int)misc[1];
  double* g = st.g(qi);
  for (int i = j - 1; i >= 0; --i) {
    if (st.H(qi, i, i) == 0.0) { atomicExch(breakdown, 1); return; }
    g[i] /= st.H(qi, i, i);
    for (int t = 0; t < i; ++t) g[t] -= st.H(qi, t, i) * g[i];
  }
  const int nc = j > 0 ? j : 1;  // j = 0: the reference still adds M^{-1}(g_0 v_0)
  for (int i = 0; i < nc; ++i) c[i] = g[i] * st.s(qi)[i];
  misc[3] = nc;
}

// xtmp = sum_i c_i u_i per instance (rgmres.tpp:106-109), over the columns that
// instance computed in this cycle (misc[3], set by b_backsolve; 0 = no update):
// columns past them were never written for it
template <int K, typename T>
__global__ void __launch_bounds__(kT) b_combine(const int* crow, const int* csys, BState st, long long ld, int ncols,
                                                const T* __restrict__ V, double* __restrict__ out) {
  extern __shared__ double cf_c[];  // [K][ncols] coefficients
  __shared__ int ncq[K];
  const int c = blockIdx.x, sys = csys[c];
  for (int t = threadIdx.x; t < K * ncols; t += kT) {
    const int kk = t / ncols, i = t % ncols;
    cf_c[kk * ncols + i] = st.c(sys * K + kk)[i];
  }
  if (threadIdx.x < K) ncq[threadIdx.x] = (int)st.misc(sys * K + threadIdx.x)[3];
  __syncthreads();
  const int k = threadIdx.x % K;
  const int nck = ncq[k];
  const long long e0 = (long long)crow[c] * K, e1 = (long long)crow[c + 1] * K;
  for (long long e = e0 + threadIdx.x; e < e1; e += kT) {
    double s = 0.0;
    if (nck > 0) {
      s = cf_c[k * ncols] * (double)V[e];
      for (int i = 1; i < nck; ++i) s += cf_c[k * ncols + i] * (double)V[(long long)i * ld + e];
    }
    out[e] = s;
  }
}

__global__ void b_axpy(long long n, const double* __restrict__ z, double* __restrict__ x) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    x[i] += z[i];
}

// partial ||v||^2 per (chunk, k) of a float64 multi-vector
template <int K>
__global__ void __launch_bounds__(kT) b_norm_part(const int* crow, const double* __restrict__ v,
                                                  double* __restrict__ red, int nchunk) {
  __shared__ double sm[(kT / 32) * K];
  const int c = blockIdx.x, k = threadIdx.x % K;
  const long long e0 = (long long)crow[c] * K, e1 = (long long)crow[c + 1] * K;
  double ss = 0.0;
  for (long long e = e0 + threadIdx.x; e < e1; e += kT) ss += v[e] * v[e];
  double o;
  reduce_k<K>(ss, sm, &o);
  if (threadIdx.x < K) red[(long long)k * nchunk + c] = o;
}

// ||b|| per instance at the start of the solve
template <int K>
__global__ void b_bnorm(int Q, const int* sch, Inst in, const double* __restrict__ red, int nchunk) {
  const int qi = blockIdx.x * blockDim.x + threadIdx.x;
  if (qi >= Q) return;
  const int sys = qi / K, k = qi % K;
  double ss = 0.0;
  for (int c = sch[sys]; c < sch[sys + 1]; ++c) ss += red[(long long)k * nchunk + c];
  in.bnorm[qi] = sqrt(ss);
  in.res[qi] = in.bnorm[qi];
  in.done[qi] = 0;
  in.iters[qi] = 0;
  in.flag[qi] = 1;
  in.active[qi] = 0;
  if (qi == 0) in.remaining[0] = Q;
}

// outer check (rgmres.tpp:118-123) and the count of unfinished instances
template <int K>
__global__ void b_outer(int Q, const int* sch, Inst in, const double* __restrict__ red, int nchunk, double reltol,
                        int itmax) {
  __shared__ int cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  for (int qi = threadIdx.x; qi < Q; qi += blockDim.x) {
    if (in.done[qi]) continue;
    const int sys = qi / K, k = qi % K;
    double ss = 0.0;
    for (int c = sch[sys]; c < sch[sys + 1]; ++c) ss += red[(long long)k * nchunk + c];
    const double rn = sqrt(ss);
    in.res[qi] = rn;
    if (rn < reltol * in.bnorm[qi]) { in.flag[qi] = 0; in.done[qi] = 1; }
    else if (in.iters[qi] >= itmax) in.done[qi] = 1;
    if (!in.done[qi]) atomicAdd(&cnt, 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) in.remaining[0] = cnt;
}

// the last kernel of a cycle inside the device-side loop: count the cycle and
// keep looping while instances are unfinished and the cycle bound is not reached
__global__ void b_continue(cudaGraphConditionalHandle h, const int* __restrict__ remaining, int* __restrict__ cycles,
                           int max_cycles) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int c = ++cycles[0];
  cudaGraphSetConditional(h, (remaining[0] > 0 && c < max_cycles) ? 1u : 0u);
}

// right-hand-side replay of the decoupling on a K-column multi-vector (cpr.cu)
template <int K>
__global__ void b_decouple_rhs(int sn, int bs, int weights, int use_drs, int cpd, const double* __restrict__ w0,
                               const unsigned char* __restrict__ ops, const double* __restrict__ J,
                               double* __restrict__ b) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < (long long)sn * K;
       t += (long long)gridDim.x * blockDim.x) {
    const int s = int(t / K), k = int(t % K);
    const long long i0 = (long long)s * bs;
    const unsigned op = ops[s];
    double x[3];
    for (int p = 0; p < bs; ++p) x[p] = b[(i0 + p) * K + k];
    if (op & 8) { double u = x[1]; x[1] = x[2]; x[2] = u; }
    if (weights != 0) {
      for (int p = 0; p < bs; ++p) x[p] = __dmul_rn(x[p], w0[i0 + p]);
      if (use_drs)
        for (int p = 0; p < bs; ++p)
          if (!(op & (1u << p))) x[p] = __ddiv_rn(x[p], w0[i0 + p]);
    }
    double sum = 0.0;
    for (int j = 0; j < bs; ++j) sum = __dadd_rn(sum, __dmul_rn(use_drs ? ((op & (1u << j)) ? 1.0 : 0.0) : 1.0, x[j]));
    x[0] = sum;
    if (cpd) {
      const double* o = J + (long long)s * bs * bs;
      double y[3];
      for (int p = 0; p < bs; ++p) {
        y[p] = 0.0;
        for (int j = 0; j < bs; ++j) y[p] = __dadd_rn(y[p], __dmul_rn(o[p * bs + j], x[j]));
      }
      for (int p = 0; p < bs; ++p) x[p] = y[p];
    }
    for (int p = 0; p < bs; ++p) b[(i0 + p) * K + k] = x[p];
  }
}

}  // namespace

}  // namespace deco

using namespace deco;

struct deco_batch_s {
  deco_csr_s* A = nullptr;   // borrowed: the caller's block-diagonal matrix, decoupled in place
  deco_cpr_s* P = nullptr;   // owned
  int nsys = 0, K = 0, bs = 0, n = 0, ncell = 0, nchunk = 0;
  std::vector<int> h_row_off;
  std::vector<int> widths;   // chosen product widths per system
  deco::DevBuf<int> cell_sys, crow, csys, sch;
  deco::DevBuf<double> zero_b;
  ~deco_batch_s() { deco_cpr_destroy(P); }
};

namespace deco {
namespace {

// Scratch and state of one batched solve.
template <int K, typename T>
struct BatchSolver {
  deco_ctx_s* ctx;
  deco_batch_s* B;
  deco_sol_params prm;
  int m, Q;
  long long n, ld, nk;
  DevBuf<T> V, w, z;
  DevBuf<double> r, xtmp, z64, bdec, stbuf, red;
  DevBuf<int> ints, brk, cyc;
  DevBuf<double> dres;
  BState st{};
  Inst in{};
  // CPR scratch for K columns
  DevBuf<T> tg, tl, rt, rts;
  DevBuf<double> tg64, tl64, rt64, rts64;

  BatchSolver(deco_ctx_s* c, deco_batch_s* b, const deco_sol_params& p) : ctx(c), B(b), prm(p) {
    cudaStream_t s = ctx->stream;
    m = prm.restart;
    Q = B->nsys * K;
    n = B->n;
    nk = n * K;
    ld = (nk + 31) / 32 * 32;
    V.alloc((size_t)ld * (m + 1), s);
    w.alloc(nk, s);
    z.alloc(nk, s);
    r.alloc(nk, s);
    xtmp.alloc(nk, s);
    z64.alloc(nk, s);
    bdec.alloc(nk, s);
    const long long sd = BState::doubles(m);
    stbuf.alloc((size_t)sd * Q, s);
    stbuf.zero(s);
    st.base = stbuf.get();
    st.stride = sd;
    st.m = m;
    red.alloc((size_t)2 * (m + 1) * K * B->nchunk + 16, s);
    ints.alloc((size_t)5 * Q + B->nsys + 8, s);
    ints.zero(s);
    dres.alloc((size_t)2 * Q, s);
    brk.alloc(1, s);
    brk.zero(s);
    cyc.alloc(1, s);
    in.active = ints.get();
    in.done = in.active + Q;
    in.iters = in.done + Q;
    in.flag = in.iters + Q;
    in.sys_active = in.flag + Q;
    in.remaining = in.sys_active + B->nsys;
    in.bnorm = dres.get();
    in.res = dres.get() + Q;
    const long long ncell = B->ncell;
    tg.alloc(nk, s); rt.alloc(nk, s); tl.alloc(ncell * K, s); rts.alloc(ncell * K, s);
    tg64.alloc(nk, s); rt64.alloc(nk, s); tl64.alloc(ncell * K, s); rts64.alloc(ncell * K, s);
  }

  T* col(int i) { return V.get() + (size_t)i * ld; }

  // x = M^{-1} r on K columns (apply_seq3 / apply_seq0 of CPR.hpp:235-274, 300-325);
  // VT: value precision of the preconditioner; R/X: vector types
  // gate: leave out the cells of systems with no running instance (inner steps
  // only; the restart update must cover every system with a coefficient)
  template <typename VT, typename R, typename X, typename S>
  void precond(const R* rin, X* x, S* tg_, S* tl_, S* rt_, S* rts_, MMGate gate = MMGate{}) {
    deco_cpr_s* P = B->P;
    const int bs = P->bs, p = P->p;
    deco_csr_s* A = P->A;
    spmm<K, VT, R>(ctx, &P->glo.FL, rin, MStore<K, S>{tg_}, false, gate);
    spmm<K, VT, S>(ctx, &P->glo.FUt, tg_, MStore<K, X>{x}, false, gate);
    spmm<K, VT, X>(ctx, A, x, MRestrict<K, R, S>{rin, rts_, bs, p}, true, gate);
    spmm<K, VT, S>(ctx, &P->loc.FL, rts_, MStore<K, S>{tl_}, false, gate);
    spmm<K, VT, S>(ctx, &P->loc.FUt, tl_, MProlong<K, X>{x, bs, p}, false, gate);
    if (P->prm.seq == 0) return;
    spmm<K, VT, X>(ctx, A, x, MResid<K, R, S>{rin, rt_}, false, gate);
    spmm<K, VT, S>(ctx, &P->glo.FL, rt_, MStore<K, S>{tg_}, false, gate);
    spmm<K, VT, S>(ctx, &P->glo.FUt, tg_, MAdd<K, X>{x}, false, gate);
  }

  MMGate inner_gate() const { return MMGate{B->cell_sys.get(), in.sys_active, B->ncell, 1}; }

  template <typename R, typename X>
  void apply_inner(const R* rin, X* x) {
    if constexpr (sizeof(T) == 4) precond<float>(rin, x, tg.get(), tl.get(), rt.get(), rts.get(), inner_gate());
    else precond<double>(rin, x, tg.get(), tl.get(), rt.get(), rts.get(), inner_gate());
  }

  void apply_outer(const double* rin, double* x) {
    if constexpr (sizeof(T) == 4) precond<float>(rin, x, tg.get(), tl.get(), rt.get(), rts.get());
    else precond<double>(rin, x, tg64.get(), tl64.get(), rt64.get(), rts64.get());
  }

  // one restart cycle: start, m Arnoldi steps, back substitution, update, true residual
  void cycle(double* x) {
    cudaStream_t s = ctx->stream;
    const int nch = B->nchunk;
    const int* crow = B->crow.get();
    const int* csys = B->csys.get();
    const int* sch = B->sch.get();
    const int qb = (int)cdiv(Q, 128);
    // all systems live for the start kernel (finished instances are masked by b_start_fin)
    b_sys_all<<<(int)cdiv(B->nsys, 128), 128, 0, s>>>(B->nsys, in.sys_active);
    DECO_CHECK_LAUNCH();
    b_start<K, T><<<nch, kT, 0, s>>>(crow, csys, in, r.get(), col(0), red.get(), nch);
    DECO_CHECK_LAUNCH();
    b_start_fin<K><<<qb, 128, 0, s>>>(Q, sch, st, in, red.get(), nch, prm.reltol, prm.itmax);
    DECO_CHECK_LAUNCH();
    b_sys_active<K><<<(int)cdiv(B->nsys, 128), 128, 0, s>>>(B->nsys, in);
    DECO_CHECK_LAUNCH();
    const long long soff = BState::s_offset(m);
    for (int j = 0; j < m; ++j) {
      apply_inner<T, T>(col(j), z.get());
      if constexpr (sizeof(T) == 4)
        spmm<K, float, T>(ctx, B->A, z.get(), MStoreScaled<K, T>{w.get(), st.base + soff + j, st.stride,
                                                                  B->cell_sys.get(), B->bs}, false, inner_gate());
      else
        spmm<K, double, T>(ctx, B->A, z.get(), MStoreScaled<K, T>{w.get(), st.base + soff + j, st.stride,
                                                                   B->cell_sys.get(), B->bs}, false, inner_gate());
      // two basis columns per block: 80 registers and three resident blocks per SM
      // instead of 126 and two for 16 bytes' worth of columns, which the L2 reuse
      // of w and u_j across a chunk's groups makes the faster choice (measured on
      // the 64-system batch: 5.7 s against 6.3 s mixed, 8.2 s against 10.2 s float64)
      constexpr int G = VShape<K, T>::G > 2 ? 2 : VShape<K, T>::G;
      b_dots_v<K, T, G><<<dim3((j + G) / G, nch), kT, 0, s>>>(crow, csys, in, ld, j, V.get(), w.get(), red.get(), nch);
      DECO_CHECK_LAUNCH();
      b_dots_fin<K><<<(int)cdiv(Q, kT / 32), kT, sizeof(double) * (kT / 32) * (j + 1), s>>>(Q, sch, st, in, j,
                                                                                            red.get(), nch);
      DECO_CHECK_LAUNCH();
      b_update_v<K, T><<<dim3(nch, kUpdSub), kT, sizeof(double) * K * (j + 1), s>>>(crow, csys, st, in, ld, j, V.get(),
                                                                                     w.get(), col(j + 1), red.get(), nch);
      DECO_CHECK_LAUNCH();
      b_update_fin<K><<<qb, 128, 0, s>>>(Q, sch, st, in, j, red.get(), nch, prm.reltol, prm.itmax);
      DECO_CHECK_LAUNCH();
      b_sys_active<K><<<(int)cdiv(B->nsys, 128), 128, 0, s>>>(B->nsys, in);
      DECO_CHECK_LAUNCH();
    }
    b_backsolve<K><<<qb, 128, 0, s>>>(Q, st, in, brk.get());
    DECO_CHECK_LAUNCH();
    b_combine<K, T><<<nch, kT, sizeof(double) * K * m, s>>>(crow, csys, st, ld, m, V.get(), xtmp.get());
    DECO_CHECK_LAUNCH();
    apply_outer(xtmp.get(), z64.get());
    b_axpy<<<grid_for(ctx, nk, 256), 256, 0, s>>>(nk, z64.get(), x);
    DECO_CHECK_LAUNCH();
    spmm<K, double, double>(ctx, B->A, x, MResid<K, double, double>{bdec.get(), r.get()});
    b_norm_part<K><<<nch, kT, 0, s>>>(crow, r.get(), red.get(), nch);
    DECO_CHECK_LAUNCH();
    b_outer<K><<<1, 1024, 0, s>>>(Q, sch, in, red.get(), nch, prm.reltol, prm.itmax);
    DECO_CHECK_LAUNCH();
  }

  void run(const double* b_in, double* x, int* h_iters, double* h_res, int* h_flags, deco_batch_result* res) {
    cudaStream_t s = ctx->stream;
    deco_cpr_s* P = B->P;
    const int nch = B->nchunk;
    DECO_CUDA(cudaEventRecord(ctx->ev0, s));
    DECO_CUDA(cudaMemcpyAsync(bdec.get(), b_in, sizeof(double) * (size_t)nk, cudaMemcpyDefault, s));
    b_decouple_rhs<K><<<grid_for(ctx, (long long)P->sn * K, 256), 256, 0, s>>>(
        P->sn, P->bs, P->prm.weights, P->prm.use_drs, P->prm.cpd, P->w0.get(), P->ops.get(), P->J.get(), bdec.get());
    DECO_CHECK_LAUNCH();
    b_norm_part<K><<<nch, kT, 0, s>>>(B->crow.get(), bdec.get(), red.get(), nch);
    DECO_CHECK_LAUNCH();
    b_bnorm<K><<<(int)cdiv(Q, 128), 128, 0, s>>>(Q, B->sch.get(), in, red.get(), nch);
    DECO_CHECK_LAUNCH();
    DECO_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * (size_t)nk, s));
    DECO_CUDA(cudaMemcpyAsync(r.get(), bdec.get(), sizeof(double) * (size_t)nk, cudaMemcpyDeviceToDevice, s));
    // Cycle launch mode (DECO_BATCH_GRAPH): 2 (default) the whole solve is ONE
    // graph launch, the cycle graph inside a device-side while loop (a conditional
    // graph node whose condition the last kernel of the cycle sets from the count
    // of unfinished instances and a cycle counter bounded by itmax / m + 2);
    // 1: the cycle graph relaunched by the host, which reads the count after each
    // cycle; 0: the same kernels launched directly.
    int mode = 2;
    if (const char* e = std::getenv("DECO_BATCH_GRAPH")) mode = std::max(0, std::min(2, std::atoi(e)));
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    struct GraphGuard {
      cudaGraph_t* g; cudaGraphExec_t* e;
      ~GraphGuard() { if (*e) cudaGraphExecDestroy(*e); if (*g) cudaGraphDestroy(*g); }
    } gg{&graph, &exec};
    const int max_cycles = prm.itmax / std::max(1, m) + 2;
    DECO_CUDA(cudaMemsetAsync(cyc.get(), 0, sizeof(int), s));
    auto capture = [&](cudaGraph_t into, bool loop_tail, cudaGraphConditionalHandle h) {
      if (into) DECO_CUDA(cudaStreamBeginCaptureToGraph(s, into, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
      else DECO_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      try {
        cycle(x);
        if (loop_tail) {
          b_continue<<<1, 1, 0, s>>>(h, in.remaining, cyc.get(), max_cycles);
          DECO_CHECK_LAUNCH();
        }
      } catch (...) {
        cudaGraph_t tmp = nullptr;
        cudaStreamEndCapture(s, &tmp);
        if (tmp && !into) cudaGraphDestroy(tmp);
        throw;
      }
      cudaGraph_t out = nullptr;
      DECO_CUDA(cudaStreamEndCapture(s, &out));
      if (!into) graph = out;
    };
    if (mode == 2) {
      DECO_CUDA(cudaGraphCreate(&graph, 0));
      cudaGraphConditionalHandle h;
      DECO_CUDA(cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault));
      cudaGraphNodeParams cp = {};
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = h;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      cudaGraphNode_t node;
      DECO_CUDA(cudaGraphAddNode(&node, graph, nullptr, 0, &cp));
      capture(cp.conditional.phGraph_out[0], true, h);
      DECO_CUDA(cudaGraphInstantiate(&exec, graph, 0));
    } else if (mode == 1) {
      capture(nullptr, false, 0);
      DECO_CUDA(cudaGraphInstantiate(&exec, graph, 0));
    }
    volatile int* hrem = reinterpret_cast<volatile int*>(ctx->host_scalars + 64);
    int cycles = 0;
    if (mode == 2) {
      DECO_CUDA(cudaGraphLaunch(exec, s));
      DECO_CUDA(cudaMemcpyAsync(const_cast<int*>(hrem), cyc.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
      DECO_CUDA(cudaStreamSynchronize(s));
      cycles = *hrem;
    } else {
      for (; cycles < max_cycles; ++cycles) {
        if (mode == 1) DECO_CUDA(cudaGraphLaunch(exec, s));
        else cycle(x);
        DECO_CUDA(cudaMemcpyAsync(const_cast<int*>(hrem), in.remaining, sizeof(int), cudaMemcpyDeviceToHost, s));
        DECO_CUDA(cudaStreamSynchronize(s));
        if (*hrem == 0) { ++cycles; break; }
      }
    }
    int hb = 0;
    DECO_CUDA(cudaMemcpyAsync(&hb, brk.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    DECO_CUDA(cudaEventRecord(ctx->ev1, s));
    DECO_CUDA(cudaEventSynchronize(ctx->ev1));
    float ms = 0.f;
    DECO_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    DECO_REQUIRE(hb == 0, DECO_ERR_BREAKDOWN, "Error in rgmres: Zero diagonal element in upper triangular matrix.");
    std::vector<int> hi((size_t)Q), hf((size_t)Q);
    std::vector<double> hr((size_t)Q), hbn((size_t)Q);
    DECO_CUDA(cudaMemcpy(hi.data(), in.iters, sizeof(int) * Q, cudaMemcpyDeviceToHost));
    DECO_CUDA(cudaMemcpy(hf.data(), in.flag, sizeof(int) * Q, cudaMemcpyDeviceToHost));
    DECO_CUDA(cudaMemcpy(hr.data(), in.res, sizeof(double) * Q, cudaMemcpyDeviceToHost));
    DECO_CUDA(cudaMemcpy(hbn.data(), in.bnorm, sizeof(double) * Q, cudaMemcpyDeviceToHost));
    int maxit = 0, nconv = 0;
    for (int q = 0; q < Q; ++q) {
      if (h_iters) h_iters[q] = hi[q];
      if (h_flags) h_flags[q] = hf[q];
      if (h_res) h_res[q] = hbn[q] > 0 ? hr[q] / hbn[q] : hr[q];
      maxit = std::max(maxit, hi[q]);
      nconv += hf[q] == 0;
    }
    res->max_iter = maxit;
    res->converged = nconv;
    res->cycles = cycles;
    res->t_solve_ms = ms;
    res->graph = mode;
  }
};

}  // namespace
}  // namespace deco

extern "C" {

int deco_batch_create(deco_ctx ctx, deco_csr A, int nsys, const int* h_row_off, int nrhs, const deco_cpr_params* prm,
                      deco_batch* out) {
  return guard([&] {
    DECO_REQUIRE(ctx && A && h_row_off && prm && out, DECO_ERR_ARG, "NULL argument");
    DECO_REQUIRE(nsys >= 1, DECO_ERR_ARG, "nsys must be >= 1");
    DECO_REQUIRE(nrhs == 1 || nrhs == 2 || nrhs == 4 || nrhs == 8, DECO_ERR_UNSUPPORTED,
                 "nrhs must be 1, 2, 4 or 8 on this path");
    DECO_REQUIRE(prm->glo_type == 0 && prm->loc_type == 0 && (prm->seq == 0 || prm->seq == 3), DECO_ERR_UNSUPPORTED,
                 "the batched solve runs CPR seq 0 or 3 with FSAI stages");
    const int bs = prm->block_size;
    DECO_REQUIRE(h_row_off[0] == 0 && h_row_off[nsys] == A->n, DECO_ERR_ARG, "row offsets must span the matrix");
    for (int q = 0; q < nsys; ++q)
      DECO_REQUIRE(h_row_off[q + 1] > h_row_off[q] && h_row_off[q] % bs == 0, DECO_ERR_ARG,
                   "every system needs rows, starting at a cell boundary");
    auto* Bt = new deco_batch_s();
    try {
      cudaStream_t st = ctx->stream;
      Bt->A = A;
      Bt->nsys = nsys;
      Bt->K = nrhs;
      Bt->bs = bs;
      Bt->n = A->n;
      Bt->ncell = A->n / bs;
      Bt->h_row_off.assign(h_row_off, h_row_off + nsys + 1);
      Bt->zero_b.alloc(A->n, st);
      Bt->zero_b.zero(st);
      int rc = deco_cpr_create(ctx, A, Bt->zero_b.get(), prm, &Bt->P);
      if (rc != DECO_OK) throw Error(rc, deco_last_error());
      DECO_REQUIRE(A->bbs == bs && Bt->P->glo.FL.n == A->n, DECO_ERR_UNSUPPORTED,
                   "the batched solve needs systems of dense bs x bs cell blocks");
      // chunks of at most kChunkRows rows inside each system
      std::vector<int> crow, csys, sch, cell_off;
      for (int q = 0; q < nsys; ++q) {
        sch.push_back((int)csys.size());
        cell_off.push_back(h_row_off[q] / bs);
        for (int r0 = h_row_off[q]; r0 < h_row_off[q + 1]; r0 += kChunkRows) {
          crow.push_back(r0);
          csys.push_back(q);
        }
      }
      sch.push_back((int)csys.size());
      cell_off.push_back(A->n / bs);
      crow.push_back(A->n);
      Bt->nchunk = (int)csys.size();
      // the dot pass runs the chunks along the grid's y dimension
      DECO_REQUIRE(Bt->nchunk <= 65535, DECO_ERR_UNSUPPORTED,
                   "the batch has more than 65535 row chunks of 4096 rows; split it into several batches");
      Bt->crow.alloc(crow.size(), st);
      Bt->csys.alloc(csys.size(), st);
      Bt->sch.alloc(sch.size(), st);
      DevBuf<int> coff(cell_off.size(), st);
      DECO_CUDA(cudaMemcpyAsync(Bt->crow.get(), crow.data(), sizeof(int) * crow.size(), cudaMemcpyHostToDevice, st));
      DECO_CUDA(cudaMemcpyAsync(Bt->csys.get(), csys.data(), sizeof(int) * csys.size(), cudaMemcpyHostToDevice, st));
      DECO_CUDA(cudaMemcpyAsync(Bt->sch.get(), sch.data(), sizeof(int) * sch.size(), cudaMemcpyHostToDevice, st));
      DECO_CUDA(cudaMemcpyAsync(coff.get(), cell_off.data(), sizeof(int) * cell_off.size(), cudaMemcpyHostToDevice, st));
      Bt->cell_sys.alloc(Bt->ncell, st);
      fill_cell_sys<<<std::min(nsys, 65535), 256, 0, st>>>(nsys, coff.get(), Bt->cell_sys.get());
      DECO_CHECK_LAUNCH();
      // product width per system: about two blocks per lane of that system's block rows
      std::vector<int> hbr(Bt->ncell + 1);
      DECO_CUDA(cudaMemcpyAsync(hbr.data(), A->br.get(), sizeof(int) * hbr.size(), cudaMemcpyDeviceToHost, st));
      DECO_CUDA(cudaStreamSynchronize(st));
      for (int q = 0; q < nsys; ++q) {
        const int c0 = cell_off[q], c1 = cell_off[q + 1];
        const double avg = double(hbr[c1] - hbr[c0]) / std::max(1, c1 - c0);
        int sw = 1;
        while (sw < 16 && sw < avg / 2.0) sw <<= 1;
        Bt->widths.push_back(sw);
      }
    } catch (...) {
      delete Bt;
      throw;
    }
    *out = Bt;
  });
}

int deco_batch_destroy(deco_batch Bt) {
  return guard([&] { delete Bt; });
}

int deco_batch_info(deco_batch Bt, int* nsys, int* nrhs, int* nchunk, int* h_widths) {
  return guard([&] {
    DECO_REQUIRE(Bt, DECO_ERR_ARG, "NULL argument");
    if (nsys) *nsys = Bt->nsys;
    if (nrhs) *nrhs = Bt->K;
    if (nchunk) *nchunk = Bt->nchunk;
    if (h_widths) std::copy(Bt->widths.begin(), Bt->widths.end(), h_widths);
  });
}

int deco_batch_cpr(deco_batch Bt, deco_cpr* P) {
  return guard([&] {
    DECO_REQUIRE(Bt && P, DECO_ERR_ARG, "NULL argument");
    *P = Bt->P;
  });
}

int deco_batch_apply(deco_ctx ctx, deco_batch Bt, const double* d_R, double* d_X) {
  return guard([&] {
    DECO_REQUIRE(ctx && Bt && d_R && d_X && d_R != d_X, DECO_ERR_ARG, "NULL or aliased argument");
    deco_sol_params sp{};
    sp.restart = 1;
    sp.precision = Bt->P->prm.precision;
    auto go = [&](auto kc, auto tc) {
      constexpr int K = decltype(kc)::value;
      using T = typename decltype(tc)::type;
      BatchSolver<K, T> S(ctx, Bt, sp);
      S.apply_outer(d_R, d_X);
      DECO_CUDA(cudaStreamSynchronize(ctx->stream));
    };
    struct F32 { using type = float; };
    struct F64 { using type = double; };
    const bool f32 = sp.precision == 32;
    switch (Bt->K) {
      case 1: f32 ? go(std::integral_constant<int, 1>{}, F32{}) : go(std::integral_constant<int, 1>{}, F64{}); break;
      case 2: f32 ? go(std::integral_constant<int, 2>{}, F32{}) : go(std::integral_constant<int, 2>{}, F64{}); break;
      case 4: f32 ? go(std::integral_constant<int, 4>{}, F32{}) : go(std::integral_constant<int, 4>{}, F64{}); break;
      default: f32 ? go(std::integral_constant<int, 8>{}, F32{}) : go(std::integral_constant<int, 8>{}, F64{}); break;
    }
  });
}

int deco_batch_solve(deco_ctx ctx, deco_batch Bt, const double* d_B, double* d_X, const deco_sol_params* prm,
                     int* h_iters, double* h_res_rel, int* h_flags, deco_batch_result* res) {
  return guard([&] {
    DECO_REQUIRE(ctx && Bt && d_B && d_X && prm && res, DECO_ERR_ARG, "NULL argument");
    DECO_REQUIRE(prm->type == 0, DECO_ERR_UNSUPPORTED, "the batched solve runs rgmres");
    DECO_REQUIRE(prm->restart >= 1 && prm->restart <= kMaxRestartB, DECO_ERR_UNSUPPORTED,
                 "restart must be in [1, " + std::to_string(kMaxRestartB) + "]");
    DECO_REQUIRE(prm->itmax >= 0, DECO_ERR_ARG, "itmax must be >= 0");
    DECO_REQUIRE(prm->precision == Bt->P->prm.precision, DECO_ERR_ARG,
                 "solve precision must match the precision of the batch's CPR");
    DECO_REQUIRE(!prm->use_x0, DECO_ERR_UNSUPPORTED, "the batched solve starts from zero");
    auto go = [&](auto kc, auto tc) {
      constexpr int K = decltype(kc)::value;
      using T = typename decltype(tc)::type;
      BatchSolver<K, T> S(ctx, Bt, *prm);
      S.run(d_B, d_X, h_iters, h_res_rel, h_flags, res);
    };
    struct F32 { using type = float; };
    struct F64 { using type = double; };
    const bool f32 = prm->precision == 32;
    switch (Bt->K) {
      case 1: f32 ? go(std::integral_constant<int, 1>{}, F32{}) : go(std::integral_constant<int, 1>{}, F64{}); break;
      case 2: f32 ? go(std::integral_constant<int, 2>{}, F32{}) : go(std::integral_constant<int, 2>{}, F64{}); break;
      case 4: f32 ? go(std::integral_constant<int, 4>{}, F32{}) : go(std::integral_constant<int, 4>{}, F64{}); break;
      default: f32 ? go(std::integral_constant<int, 8>{}, F32{}) : go(std::integral_constant<int, 8>{}, F64{}); break;
    }
  });
}

}  // extern "C"
