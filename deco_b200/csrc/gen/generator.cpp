// Seeded synthetic fully-implicit reservoir Jacobians (see include/deco_gen.h).
//
// Equations per cell s (rows s*bs + a):
//   a = 0      total / pressure equation: sum_t T_st (p_s - p_t) + compressibility
//   a = 1..bs-1 phase equations: upwinded fractional flow f_a(S_up) * T (p_s - p_t)
//              + accumulation phi V / dt on the phase's own saturation.
// Saturation derivatives of the face fluxes are upwinded along a seeded flow
// potential: the upstream cell gets +c on its diagonal block, the downstream cell
// -c on the off-diagonal block, and the non-upwind side keeps a tiny entry so that
// every coupling block is dense.
// Wells are vertical columns that add a productivity index to the pressure
// diagonal (and f_a * PI to the phase rows), which anchors the elliptic block.
#include "../../../include/deco_gen.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <utility>
#include <vector>

namespace {

inline uint64_t mix64(uint64_t z) {  // splitmix64 finaliser
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
inline uint64_t hsh(uint64_t seed, uint64_t stream, uint64_t idx) {
  return mix64(mix64(seed * 0x2545F4914F6CDD1Dull + stream) ^ (idx * 0x9E3779B97F4A7C15ull));
}
inline double u01(uint64_t h) { return double(h >> 11) * (1.0 / 9007199254740992.0); }
inline double uni(uint64_t seed, uint64_t stream, uint64_t idx) { return u01(hsh(seed, stream, idx)); }
inline double logu(double lo, double hi, double u) { return std::exp(std::log(lo) + u * (std::log(hi) - std::log(lo))); }
inline double gauss(uint64_t seed, uint64_t stream, uint64_t idx) {
  double u1 = uni(seed, stream, 2 * idx), u2 = uni(seed, stream, 2 * idx + 1);
  if (u1 < 1e-300) u1 = 1e-300;
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

enum Stream : uint64_t {
  S_LOGK = 1, S_LAYER = 2, S_FACE = 3, S_FACE_G = 4, S_ACC = 5, S_FRAC = 6, S_WELL = 7,
  S_FAULT = 8, S_CHAN = 9, S_XTRA = 10, S_RHS = 11
};

struct Sys {
  const deco_gen_params* p;
  int nx, ny, nz, bs;
  long long nc;
  std::vector<std::pair<int, int>> faults;  // sorted unique (a<b)
  std::vector<long long> xr;                // per-cell fault adjacency (CSR)
  std::vector<int> xc;
  std::vector<double> logk;
  std::vector<char> well;
};

int validate(const deco_gen_params* p) {
  if (!p) return -1;
  if (p->nx < 1 || p->ny < 1 || p->nz < 1) return -2;
  if (p->bs != 2 && p->bs != 3) return -3;
  if (p->acc_lo <= 0 || p->acc_hi < p->acc_lo || p->cpl_lo <= 0 || p->cpl_hi < p->cpl_lo) return -4;
  return 0;
}

bool stencil_neighbor(const Sys& s, int a, int b) {
  long long d = (long long)b - a;
  if (d < 0) d = -d;
  long long nxy = (long long)s.nx * s.ny;
  if (d == 1) return (std::min(a, b) % s.nx) != s.nx - 1;  // same x-row
  if (d == s.nx) return ((std::min(a, b) / s.nx) % s.ny) != s.ny - 1;
  if (d == nxy) return true;
  return false;
}

void build_faults(Sys& s) {
  const deco_gen_params* p = s.p;
  long long nf = (long long)std::llround(p->fault_frac * (double)s.nc);
  s.faults.clear();
  s.faults.reserve(nf);
  for (long long f = 0; f < nf && s.nc > 2; ++f) {
    int a = int(hsh(p->seed, S_FAULT, 2 * f) % (uint64_t)s.nc);
    int b = int(hsh(p->seed, S_FAULT, 2 * f + 1) % (uint64_t)s.nc);
    if (a == b) continue;
    if (a > b) std::swap(a, b);
    if (stencil_neighbor(s, a, b)) continue;
    s.faults.emplace_back(a, b);
  }
  std::sort(s.faults.begin(), s.faults.end());
  s.faults.erase(std::unique(s.faults.begin(), s.faults.end()), s.faults.end());
  s.xr.assign(s.nc + 1, 0);
  for (auto& e : s.faults) { s.xr[e.first + 1]++; s.xr[e.second + 1]++; }
  for (long long i = 0; i < s.nc; ++i) s.xr[i + 1] += s.xr[i];
  s.xc.assign(s.xr[s.nc], 0);
  std::vector<long long> pos(s.xr.begin(), s.xr.end() - 1);
  for (auto& e : s.faults) { s.xc[pos[e.first]++] = e.second; s.xc[pos[e.second]++] = e.first; }
  for (long long i = 0; i < s.nc; ++i) std::sort(s.xc.begin() + s.xr[i], s.xc.begin() + s.xr[i + 1]);
}

void box_smooth(std::vector<double>& f, int nx, int ny, int nz, bool vertical) {
  std::vector<double> g(f.size());
  auto idx = [&](int x, int y, int z) { return (long long)x + (long long)nx * (y + (long long)ny * z); };
  // x
#pragma omp parallel for collapse(2)
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        double a = f[idx(x, y, z)], l = x > 0 ? f[idx(x - 1, y, z)] : a, r = x < nx - 1 ? f[idx(x + 1, y, z)] : a;
        g[idx(x, y, z)] = (l + a + r) / 3.0;
      }
#pragma omp parallel for collapse(2)
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        double a = g[idx(x, y, z)], l = y > 0 ? g[idx(x, y - 1, z)] : a, r = y < ny - 1 ? g[idx(x, y + 1, z)] : a;
        f[idx(x, y, z)] = (l + a + r) / 3.0;
      }
  if (!vertical) return;
#pragma omp parallel for collapse(2)
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        double a = f[idx(x, y, z)], l = z > 0 ? f[idx(x, y, z - 1)] : a, r = z < nz - 1 ? f[idx(x, y, z + 1)] : a;
        g[idx(x, y, z)] = (l + a + r) / 3.0;
      }
  f.swap(g);
}

void standardize(std::vector<double>& f, double sigma) {
  // fixed chunks summed in order: the result does not depend on the thread count
  const long long n = (long long)f.size();
  const int nch = 1024;
  std::vector<double> p1(nch, 0.0), p2(nch, 0.0);
#pragma omp parallel for
  for (int ch = 0; ch < nch; ++ch) {
    const long long a = n * ch / nch, b = n * (ch + 1) / nch;
    double t1 = 0, t2 = 0;
    for (long long i = a; i < b; ++i) { t1 += f[i]; t2 += f[i] * f[i]; }
    p1[ch] = t1;
    p2[ch] = t2;
  }
  double s1 = 0, s2 = 0;
  for (int ch = 0; ch < nch; ++ch) { s1 += p1[ch]; s2 += p2[ch]; }
  double mean = s1 / n, var = s2 / n - mean * mean, sd = var > 0 ? std::sqrt(var) : 1.0;
#pragma omp parallel for
  for (long long i = 0; i < n; ++i) f[i] = (f[i] - mean) / sd * sigma;
}

void build_logk(Sys& s) {
  const deco_gen_params* p = s.p;
  s.logk.assign(s.nc, 0.0);
  long long nc = s.nc;
#pragma omp parallel for
  for (long long i = 0; i < nc; ++i) s.logk[i] = gauss(p->seed, S_LOGK, i);
  for (int k = 0; k < p->smooth; ++k) box_smooth(s.logk, s.nx, s.ny, s.nz, !p->layered);
  if (p->layered) {
    standardize(s.logk, 0.45 * p->sigma);
    const long long nxy = (long long)s.nx * s.ny;
#pragma omp parallel for
    for (long long i = 0; i < nc; ++i) s.logk[i] += 0.9 * p->sigma * gauss(p->seed, S_LAYER, i / nxy);
  } else {
    standardize(s.logk, p->sigma);
  }
  // channels: sinusoidal high-k bodies in x-y, a few layers thick
  const double lc = std::log(std::max(p->channel_contrast, 1.0));
  std::vector<char> in_channel(p->n_channels > 0 ? nc : 0, 0);
  for (int ch = 0; ch < p->n_channels; ++ch) {
    double y0 = uni(p->seed, S_CHAN, 8 * ch + 0) * s.ny;
    double amp = (0.05 + 0.15 * uni(p->seed, S_CHAN, 8 * ch + 1)) * s.ny;
    double lam = (0.3 + 0.7 * uni(p->seed, S_CHAN, 8 * ch + 2)) * s.nx;
    double ph = 6.283185307179586 * uni(p->seed, S_CHAN, 8 * ch + 3);
    int th = std::max(1, s.nz / 10);
    int z0 = int(uni(p->seed, S_CHAN, 8 * ch + 4) * std::max(1, s.nz - th + 1));
    double hw = std::max(1.0, s.ny / 40.0);
#pragma omp parallel for collapse(2)
    for (int z = z0; z < std::min(s.nz, z0 + th); ++z)
      for (int x = 0; x < s.nx; ++x) {
        double yc = y0 + amp * std::sin(6.283185307179586 * x / lam + ph);
        for (int y = 0; y < s.ny; ++y)
          if (std::fabs(y - yc) <= hw) in_channel[(long long)x + (long long)s.nx * (y + (long long)s.ny * z)] = 1;
      }
  }
  // channel cells carry permeability contrast x the background median (ln k = 0):
  // the contrast is between channel and matrix, not on top of the matrix's tail
  if (p->n_channels > 0) {
#pragma omp parallel for
    for (long long i = 0; i < nc; ++i)
      if (in_channel[i]) s.logk[i] = lc + 0.1 * p->sigma * gauss(p->seed, S_CHAN + 100, (uint64_t)i);
  }
}

void build_wells(Sys& s) {
  const deco_gen_params* p = s.p;
  s.well.assign(s.nc, 0);
  for (int w = 0; w < p->n_wells; ++w) {
    int x = int(uni(p->seed, S_WELL, 2 * w) * s.nx), y = int(uni(p->seed, S_WELL, 2 * w + 1) * s.ny);
    for (int z = 0; z < s.nz; ++z) s.well[(long long)x + (long long)s.nx * (y + (long long)s.ny * z)] = 1;
  }
}

// neighbour cells of s in ascending order, including s itself
int neighbours(const Sys& s, int c, int* out) {
  const int nx = s.nx, ny = s.ny;
  const long long nxy = (long long)nx * ny;
  int x = c % nx, y = (c / nx) % ny, z = int(c / nxy);
  int st[7], k = 0;
  if (z > 0) st[k++] = int(c - nxy);
  if (y > 0) st[k++] = c - nx;
  if (x > 0) st[k++] = c - 1;
  st[k++] = c;
  if (x < nx - 1) st[k++] = c + 1;
  if (y < ny - 1) st[k++] = c + nx;
  if (z < s.nz - 1) st[k++] = int(c + nxy);
  // merge with fault partners (sorted, disjoint from stencil)
  long long a = s.xr[c], b = s.xr[c + 1];
  int i = 0, m = 0;
  while (i < k || a < b) {
    if (a >= b || (i < k && st[i] < s.xc[a])) out[m++] = st[i++];
    else out[m++] = s.xc[a++];
  }
  return m;
}

// axis multiplier of the face (a,b): 1 for x/y, kz_kx for z, 0.5 for faults
double face_mult(const Sys& s, int a, int b) {
  long long d = std::llabs((long long)b - a);
  if (stencil_neighbor(s, a, b)) return d == (long long)s.nx * s.ny ? s.p->kz_kx : 1.0;
  return 0.5;
}

// flow potential: a regional gradient (mostly +x) plus a small per-cell jitter;
// the upstream cell of every face is the one with the higher potential, so the
// upwinded saturation couplings never form a cycle
inline double potential(const Sys& s, int c) {
  const int x = c % s.nx, y = (c / s.nx) % s.ny;
  const long long z = (long long)c / ((long long)s.nx * s.ny);
  return -(x + 0.37 * y + 0.13 * (double)z) + 0.3 * uni(s.p->seed, S_FACE, (uint64_t)c);
}

struct CellData {
  double acc, fr[3];
};

inline CellData cell_data(const Sys& s, int c) {
  const deco_gen_params* p = s.p;
  CellData d;
  d.acc = logu(p->acc_lo, p->acc_hi, uni(p->seed, S_ACC, c));
  d.fr[0] = 1.0;
  if (s.bs == 2) {
    d.fr[1] = 0.05 + 0.9 * uni(p->seed, S_FRAC, 2 * (uint64_t)c);
  } else {
    d.fr[1] = 0.05 + 0.55 * uni(p->seed, S_FRAC, 2 * (uint64_t)c);
    d.fr[2] = 0.05 + 0.30 * uni(p->seed, S_FRAC, 2 * (uint64_t)c + 1);
  }
  return d;
}

}  // namespace

extern "C" {

int deco_gen_preset(int config, unsigned long long seed, deco_gen_params* p) {
  if (!p) return -1;
  std::memset(p, 0, sizeof(*p));
  p->seed = seed;
  p->kz_kx = 1.0;
  p->acc_lo = 1e3; p->acc_hi = 1e5;
  p->cpl_lo = 1e-2; p->cpl_hi = 1.0;
  p->n_wells = 4;
  p->comp = 1e-3;
  p->smooth = 2;
  p->channel_contrast = 1.0;
  switch (config) {
    case 1: p->nx = 40; p->ny = 40; p->nz = 20; p->bs = 2; p->sigma = 1.5; break;
    case 2: p->nx = 100; p->ny = 100; p->nz = 50; p->bs = 3; p->sigma = 2.0; p->layered = 1;
            p->kz_kx = 0.1; p->fault_frac = 0.01; break;
    case 3: p->nx = 200; p->ny = 200; p->nz = 100; p->bs = 2; p->sigma = 2.5; p->n_channels = 6;
            p->channel_contrast = 1e4; p->comp = 1.0; break;
    case 5: p->nx = 64; p->ny = 64; p->nz = 32; p->bs = 2; p->sigma = 1.5; break;
    default: return -1;
  }
  return 0;
}

int deco_gen_size(const deco_gen_params* p, int* n, long long* nnz) {
  int e = validate(p);
  if (e) return e;
  Sys s;
  s.p = p; s.nx = p->nx; s.ny = p->ny; s.nz = p->nz; s.bs = p->bs;
  s.nc = (long long)p->nx * p->ny * p->nz;
  if (s.nc * p->bs > 2147483647LL) return -5;
  build_faults(s);
  long long blocks = s.nc + 2 * (long long)s.faults.size();
  blocks += 2LL * ((long long)(p->nx - 1) * p->ny * p->nz + (long long)p->nx * (p->ny - 1) * p->nz +
                   (long long)p->nx * p->ny * (p->nz - 1));
  long long z = blocks * p->bs * p->bs;
  if (z > 2147483647LL) return -5;
  if (n) *n = int(s.nc * p->bs);
  if (nnz) *nnz = z;
  return 0;
}

}  // extern "C"

namespace {

// Assembly of the whole system, in one of two modes:
//   fill      (dLdA == nullptr): writes r, c, v (and b, logk_out when non-null);
//   gradient  (dLdA != nullptr): accumulates dL/d ln k[cell] from dL/dA on the
//             pattern into dLdlogk, using that every entry that depends on a
//             face transmissibility T is T times a coefficient independent of k,
//             and dT/d ln k_a = T k_b / (k_a + k_b) for T = 2 k_a k_b/(k_a+k_b) * mult.
// logk_in == nullptr generates the seeded field; otherwise it is used as given.
int assemble(const deco_gen_params* p, const double* logk_in, int* r, int* c, double* v, double* b,
             double* logk_out, const double* dLdA, double* dLdlogk) {
  int e = validate(p);
  if (e) return e;
  int n;
  long long nnz;
  if ((e = deco_gen_size(p, &n, &nnz))) return e;
  Sys s;
  s.p = p; s.nx = p->nx; s.ny = p->ny; s.nz = p->nz; s.bs = p->bs;
  s.nc = (long long)p->nx * p->ny * p->nz;
  build_faults(s);
  if (logk_in) s.logk.assign(logk_in, logk_in + s.nc);
  else build_logk(s);
  build_wells(s);
  const int bs = s.bs;
  const long long nc = s.nc;
  const bool grad = dLdA != nullptr;

  // row pointers: every row of a cell has bs * |neighbours| entries
  std::vector<long long> cstart(nc + 1, 0);
#pragma omp parallel for
  for (long long i = 0; i < nc; ++i) {
    int nb[64];
    cstart[i + 1] = neighbours(s, int(i), nb);
  }
  for (long long i = 0; i < nc; ++i) cstart[i + 1] += cstart[i];
  if (cstart[nc] * bs * bs != nnz) return -6;
  // gradient mode: the neighbour side of each face, written per (cell, slot), summed after
  std::vector<double> nbpart(grad ? cstart[nc] : 0, 0.0);
  if (grad)
    for (long long i = 0; i < nc; ++i) dLdlogk[i] = 0.0;

#pragma omp parallel for schedule(static, 256)
  for (long long ci = 0; ci < nc; ++ci) {
    const int cs = int(ci);
    int nb[64];
    const int m = neighbours(s, cs, nb);
    const long long rowlen = (long long)m * bs;
    const long long base = cstart[ci] * bs * bs;  // first entry of row cs*bs
    if (!grad) {
      for (int a = 0; a < bs; ++a) r[(long long)cs * bs + a] = int(base + a * rowlen);
      if (ci == nc - 1) r[n] = int(base + bs * rowlen);
    }
    int self = -1;
    for (int q = 0; q < m; ++q)
      if (nb[q] == cs) self = q;

    double D[3][3] = {{0}};
    double O[64][3][3];
    const CellData me = cell_data(s, cs);
    const double ks = std::exp(s.logk[ci]);
    double gself = 0.0;
    for (int q = 0; q < m; ++q) {
      const int t = nb[q];
      if (t == cs) continue;
      const int fa = std::min(cs, t), fb = std::max(cs, t);
      const uint64_t fid = (uint64_t)fa * 2654435761ull ^ ((uint64_t)fb << 20) ^ (uint64_t)fb;
      const double kt = std::exp(s.logk[t]);
      const double T = 2.0 * ks * kt / (ks + kt) * face_mult(s, fa, fb);
      // upwind side from a seeded flow potential (acyclic, as a real flux field is)
      const int up = potential(s, fa) > potential(s, fb) ? fa : fb;
      const double g = logu(p->cpl_lo, p->cpl_hi, uni(p->seed, S_FACE_G, fid));
      const CellData ud = (up == cs) ? me : cell_data(s, up);
      if (!grad) {
        double (*Ob)[3] = O[q];
        // pressure columns
        Ob[0][0] = -T;
        D[0][0] += T;
        for (int a = 1; a < bs; ++a) { Ob[a][0] = -T * ud.fr[a]; D[a][0] += T * ud.fr[a]; }
        // saturation columns (upwinded)
        for (int a = 0; a < bs; ++a)
          for (int bb = 1; bb < bs; ++bb) {
            double cab = (a == 0) ? 0.1 * T * g : (a == bb ? T * g : -0.3 * T * g);
            if (up == cs) {
              D[a][bb] += cab;
              Ob[a][bb] = 1e-3 * cab;  // the non-upwind side keeps a tiny entry
            } else {
              Ob[a][bb] = -cab;
            }
          }
        continue;
      }
      // gradient: the same entries divided by T (off-diagonal block kO, diagonal-block part kD)
      double kO[3][3] = {{0}}, kD[3][3] = {{0}};
      kO[0][0] = -1.0;
      kD[0][0] = 1.0;
      for (int a = 1; a < bs; ++a) { kO[a][0] = -ud.fr[a]; kD[a][0] = ud.fr[a]; }
      for (int a = 0; a < bs; ++a)
        for (int bb = 1; bb < bs; ++bb) {
          const double kab = (a == 0) ? 0.1 * g : (a == bb ? g : -0.3 * g);
          if (up == cs) {
            kD[a][bb] = kab;
            kO[a][bb] = 1e-3 * kab;
          } else {
            kO[a][bb] = -kab;
          }
        }
      double G = 0.0;  // dL/dT of this face through row block cs
      for (int a = 0; a < bs; ++a) {
        const double* row = dLdA + base + a * rowlen;
        for (int bb = 0; bb < bs; ++bb) G += row[q * bs + bb] * kO[a][bb] + row[self * bs + bb] * kD[a][bb];
      }
      gself += G * T * kt / (ks + kt);
      nbpart[cstart[ci] + q] = G * T * ks / (ks + kt);
    }
    if (grad) {
      dLdlogk[ci] += gself;
      continue;
    }
    // accumulation, compressibility, wells (independent of k)
    D[0][0] += p->comp;
    for (int a = 1; a < bs; ++a) {
      D[a][a] += me.acc;
      D[0][a] += 0.02 * me.acc * (0.5 + 0.5 * uni(p->seed, S_XTRA, 4 * (uint64_t)cs + a));
      D[a][0] += p->comp * me.fr[a];
      for (int bb = 1; bb < bs; ++bb)
        if (bb != a) D[a][bb] += 0.05 * me.acc * uni(p->seed, S_XTRA, 4 * (uint64_t)cs + 3);
    }
    if (s.well[ci]) {
      const double PI = 100.0;
      D[0][0] += PI;
      for (int a = 1; a < bs; ++a) D[a][0] += PI * me.fr[a];
    }
    // scatter rows
    for (int a = 0; a < bs; ++a) {
      long long o = base + a * rowlen;
      for (int q = 0; q < m; ++q) {
        const double (*B)[3] = (q == self) ? D : O[q];
        for (int bb = 0; bb < bs; ++bb) {
          c[o] = nb[q] * bs + bb;
          v[o] = B[a][bb];
          ++o;
        }
      }
    }
  }
  if (grad) {  // the neighbour halves, in cell order (deterministic)
    for (long long ci = 0; ci < nc; ++ci) {
      int nb[64];
      const int m = neighbours(s, int(ci), nb);
      for (int q = 0; q < m; ++q)
        if (nb[q] != ci) dLdlogk[nb[q]] += nbpart[cstart[ci] + q];
    }
    return 0;
  }
  if (b) deco_gen_uniform(p->seed, S_RHS, n, b);
  if (logk_out) std::memcpy(logk_out, s.logk.data(), sizeof(double) * nc);
  return 0;
}

}  // namespace

extern "C" {

int deco_gen_fill(const deco_gen_params* p, int* r, int* c, double* v, double* b, double* logk) {
  return assemble(p, nullptr, r, c, v, b, logk, nullptr, nullptr);
}

int deco_gen_fill_logk(const deco_gen_params* p, const double* logk, int* r, int* c, double* v, double* b) {
  if (!logk) return -1;
  return assemble(p, logk, r, c, v, b, nullptr, nullptr, nullptr);
}

int deco_gen_grad_logk(const deco_gen_params* p, const double* logk, const double* dLdA, double* dLdlogk) {
  if (!dLdA || !dLdlogk) return -1;
  return assemble(p, logk, nullptr, nullptr, nullptr, nullptr, nullptr, dLdA, dLdlogk);
}

void deco_gen_uniform(unsigned long long seed, unsigned long long stream, long long n, double* out) {
#pragma omp parallel for
  for (long long i = 0; i < n; ++i) out[i] = uni(seed, 1000 + stream, (uint64_t)i);
}

}  // extern "C"
