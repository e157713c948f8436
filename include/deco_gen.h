/*
 * deco_gen.h — seeded synthetic reservoir systems (host only, no CUDA).
 *
 * The reference ships its sample systems (Norne, SPE11C, Sleipner) only as
 * Git-LFS pointers (ABC/*.bin, .gitattributes:1-2), so every workload in this
 * project is generated here: a fully-implicit two-phase (bs=2: p, Sw) or
 * three-phase (bs=3: p, Sw, Sg) Jacobian on an nx*ny*nz grid with 7-point
 * TPFA couplings, harmonic-mean transmissibilities and optional long-range
 * fault connections.
 *
 * Layout produced (what the reference's block arithmetic requires,
 * precond/CPR.hpp:355-358,404-409,626-631):
 *   - cell-major interleaved unknowns, pressure first (row s*bs+0);
 *   - sorted column indices inside every row;
 *   - a dense bs x bs block for every cell-cell coupling, so the bs rows of a
 *     cell share one column pattern (precond/CPR.hpp:484-492);
 *   - CSR with int32 row pointers and columns and float64 values, i.e. the
 *     reference's CSR<int,int,double> (core/CSR.hpp:4-13) and its binary file
 *     layout (IO/cpp_read.hpp:331-349).
 *
 * Every random draw is a counter-based hash of (seed, stream, index), so the
 * output is identical for any thread count and on any machine.
 */
#ifndef DECO_GEN_H
#define DECO_GEN_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct deco_gen_params {
  int nx, ny, nz;            /* grid cells per axis                              */
  int bs;                    /* unknowns per cell: 2 or 3                        */
  double sigma;              /* std-dev of ln(k)                                 */
  double kz_kx;              /* vertical anisotropy: k_z = kz_kx * k            */
  int layered;               /* 1: ln(k) = per-layer mean + lateral variation    */
  int n_channels;            /* high-permeability channels                       */
  double channel_contrast;   /* k multiplier inside a channel                    */
  double fault_frac;         /* long-range connections per cell (fraction)       */
  int n_wells;               /* wells: strong pressure-diagonal source terms     */
  double acc_lo, acc_hi;     /* saturation accumulation, log-uniform range       */
  double cpl_lo, cpl_hi;     /* coupling-block scale, log-uniform range          */
  double comp;               /* pressure accumulation / mean transmissibility    */
  int smooth;                /* box-filter passes on ln(k) (spatial correlation) */
  unsigned long long seed;
} deco_gen_params;

/* Preset for the named workloads: 1 = 40x40x20x2, 2 = 100x100x50x3 + 1% faults,
 * 3 = 200x200x100x2 with 1e4-contrast channels, 5 = 64x64x32x2 (adjoint).
 * Returns 0, or -1 for an unknown id. */
int deco_gen_preset(int config, unsigned long long seed, deco_gen_params* p);

/* Rows and nonzeros of the system that deco_gen_fill() will produce. */
int deco_gen_size(const deco_gen_params* p, int* n, long long* nnz);

/* Fill r[n+1], c[nnz], v[nnz]; b[n] (uniform [0,1)) and logk[nx*ny*nz] may be
 * NULL.  Returns 0, or a negative code on invalid parameters / int32 overflow. */
int deco_gen_fill(const deco_gen_params* p, int* r, int* c, double* v, double* b,
                  double* logk);

/* The same system assembled from a caller-given ln(k) field (nx*ny*nz values)
 * instead of the seeded one; b is the seeded right-hand side as before. */
int deco_gen_fill_logk(const deco_gen_params* p, const double* logk, int* r, int* c, double* v, double* b);

/* Chain rule from the matrix to the permeability: given dL/dA on the pattern
 * (nnz values, in the order deco_gen_fill writes them), writes dL/d ln k for
 * every cell.  Every transmissibility-dependent entry is T times a coefficient
 * independent of k, with T = 2 k_a k_b / (k_a + k_b) * mult per face; wells and
 * accumulation terms do not depend on k.  logk == NULL uses the seeded field. */
int deco_gen_grad_logk(const deco_gen_params* p, const double* logk, const double* dLdA, double* dLdlogk);

/* Uniform [0,1) vector from the same counter-based generator (stream id lets
 * callers draw independent right-hand sides). */
void deco_gen_uniform(unsigned long long seed, unsigned long long stream, long long n,
                      double* out);

#ifdef __cplusplus
}
#endif
#endif
