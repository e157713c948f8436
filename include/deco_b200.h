/*
 * deco_b200.h — C ABI of the B200 CPR-Krylov path (libdeco_b200.so).
 *
 * This is the drop-in boundary for the reference's hot path (amavliut/deco):
 * the reference's C++ classes CSR, FSAI, CPR and SOL (header-only templates,
 * core/CSR.hpp, precond/FSAI/FSAI.hpp, precond/CPR.hpp, solver/SOL.hpp) are
 * re-expressed on the host side as thin C++ classes (deco_b200/host/deco.hpp)
 * that forward to the functions below.  Signatures use plain pointers and
 * sizes only.
 *
 * Conventions
 *   - Matrices are CSR<int,int,double> exactly as in the reference
 *     (core/CSR.hpp:6-13): int32 row pointers r[n+1], int32 sorted columns
 *     c[nz], float64 values v[nz]; cell-major unknowns, pressure id p.
 *   - Every call returns DECO_OK (0) or a negative DECO_ERR_* code; the
 *     message is in deco_last_error() (per host thread).  Nothing exits the
 *     process (the reference calls exit() on zero pivots: precond/CPR.hpp:416,
 *     643, 665; solver/rgmres.tpp:96-99 — here those are DECO_ERR_SINGULAR /
 *     DECO_ERR_BREAKDOWN statuses).
 *   - Vector arguments named d_* are device pointers (float64 unless stated);
 *     h_* are host pointers.  Calls are ordered on the context's stream;
 *     functions returning host data synchronise that stream.
 *   - Handles are not thread-safe; one host thread per context.
 */
#ifndef DECO_B200_H
#define DECO_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status codes */
#define DECO_OK 0
#define DECO_ERR_ARG (-1)        /* invalid argument                         */
#define DECO_ERR_CUDA (-2)       /* CUDA runtime error                       */
#define DECO_ERR_ALLOC (-3)      /* device or host allocation failed         */
#define DECO_ERR_SINGULAR (-4)   /* zero determinant / pivot in a cell block */
#define DECO_ERR_BREAKDOWN (-5)  /* zero Hessenberg diagonal in GMRES        */
#define DECO_ERR_UNSUPPORTED (-6)/* option not implemented on this path      */
#define DECO_ERR_PATTERN (-7)    /* matrix layout assumption violated        */
#define DECO_ERR_INTERNAL (-8)

typedef struct deco_ctx_s* deco_ctx;
typedef struct deco_csr_s* deco_csr;
typedef struct deco_fsai_s* deco_fsai;
typedef struct deco_cpr_s* deco_cpr;

/* Last error message of the calling host thread ("" if none). */
const char* deco_last_error(void);
/* Library version string. */
const char* deco_version(void);
/* Kernels this library has launched in this process (all contexts). */
long long deco_launch_count(void);
/* Device-memory requests this library has made in this process (every request
 * of its stream-ordered allocator, whether served from its block cache or by
 * cudaMallocAsync).  No counterpart in the reference: a diagnostic, e.g. to
 * check that deco_fsai_apply_static allocates nothing. */
long long deco_alloc_count(void);

/* ------------------------------------------------------------------ context
 * Replaces the reference's process-global state (MPI_Comm deco_comm,
 * core/pch.h:23; OpenMP thread pool).  stream == NULL creates a private
 * non-blocking stream. */
int deco_ctx_create(int device, void* stream, deco_ctx* out);
int deco_ctx_destroy(deco_ctx ctx);
int deco_ctx_sync(deco_ctx ctx);
int deco_ctx_stream(deco_ctx ctx, void** stream);
/* autotune != 0: SpMV sub-warp width is chosen per matrix by timing (default 1). */
int deco_ctx_set_autotune(deco_ctx ctx, int autotune);
/* Returns the device blocks the context keeps for reuse to the device's memory
 * pool.  Blocks of 1 MiB and more that the library frees stay cached per
 * stream and serve later requests on that stream (no counterpart in the
 * reference, which allocates host memory with malloc). */
int deco_ctx_trim(deco_ctx ctx);

/* --------------------------------------------------------------- matrices
 * Replaces CSR<int,int,double> construction and its raw arrays
 * (core/CSR.hpp:45-70) on the device.  where = 0: arrays are host memory;
 * where = 1: arrays are device memory (copied).  The matrix keeps float64
 * values; deco_csr_make_f32() adds a float32 copy used by mixed precision. */
int deco_csr_create(deco_ctx ctx, int n, int m, int nz, const int* r, const int* c, const double* v,
                    int where, deco_csr* out);
int deco_csr_destroy(deco_csr A);
int deco_csr_info(deco_csr A, int* n, int* m, int* nz);
/* Copies the current (possibly CPR-modified) arrays to host buffers. */
int deco_csr_download(deco_ctx ctx, deco_csr A, int* h_r, int* h_c, double* h_v);
/* Overwrite values (same pattern) from host (where=0) or device (where=1). */
int deco_csr_set_values(deco_ctx ctx, deco_csr A, const double* v, int where);
int deco_csr_make_f32(deco_ctx ctx, deco_csr A);
/* SpMV sub-warp width in use (1..32) and the one the autotuner picked. */
int deco_csr_subwarp(deco_csr A, int* sw);
int deco_csr_set_subwarp(deco_csr A, int sw);
/* Cell-block copy for matrices made of bs x bs cell blocks (bs 2 or 3): one
 * column index per block, entries the pattern lacks stored as zeros, values in
 * row planes.  Every later product with A reads it (all rows, or row 0 of each
 * cell for a restricted product with the same bs).  CPR setup adds it to its
 * system and to the global FSAI factors.  Not built (status OK, *nblk = 0 from
 * deco_csr_blocks) when padding would exceed a quarter of the stored entries;
 * bs = 0 removes it.  No counterpart in the reference (core/CSR.hpp stores CSR
 * only). */
int deco_csr_set_blocks(deco_ctx ctx, deco_csr A, int bs);
int deco_csr_blocks(deco_csr A, int* bs, int* nblk);
/* Slots per cell of the padded copy that products of a 2x2-block matrix use
 * when every cell has at most 4 blocks (4 slots) or at most 7 or 8 blocks with
 * at most 25 % padding (7 or 8 slots); of a 3x3-block matrix, the fewest of 4, 7
 * or 8 slots that leave at most 2 % of the cells wider (their further blocks
 * go to an overflow list) within 25 % padding; or slots per row of the scalar
 * padded copy that an FSAI factor without cell blocks gets (4, or 8 with at
 * most 25 % padding); 0 without one.  The block forms are
 * made with the block copy; DECO_PADDED=0 in the environment at context
 * creation turns them off.  No counterpart in the reference. */
int deco_csr_padded(deco_csr A, int* slots);
/* The product a full y = A x of this matrix takes for float64 (precision 64) or
 * float32 (32) values: kind 1 = the slot-padded copy (one thread per cell of
 * 2x2 or 3x3 blocks, or per scalar row: rows grouped per thread), 2 = the cell-block
 * kernel with `lanes` lanes per cell, 3 = the CSR kernel with `lanes` lanes per
 * row.  A CPR setup times the products each of its matrices has a layout for
 * and keeps the fastest (the layout rules' choice unless another is at least
 * 5 % faster; DECO_AUTOTUNE=0 keeps the rules).  No counterpart in the
 * reference. */
int deco_csr_product_plan(deco_csr A, int precision, int* kind, int* lanes);
/* Bytes per slot column the padded products read: 1 or 2 when the slots'
 * column offsets (column minus the slot's own row or cell) take at most 256 or
 * 65536 distinct values and the copy stores a code per slot and the offsets
 * once (`noffsets` of them), 4 when it stores the columns themselves, 0 without
 * a padded copy.  Copies of fewer than 2^22 slots keep 4-byte columns (their
 * products are bound by launch and tail, not bytes), and so does every copy
 * after DECO_SLOT_CODES=0 at context creation.
 * No counterpart in the reference. */
int deco_csr_slot_codes(deco_csr A, int* bytes, int* noffsets);

/* y = A x (bs == 1), or the restricted product of alg::spmv with bs > 1:
 * y[i/bs] = (A x)[i] for rows i = 0, bs, 2bs, ...   (core/alg.hpp:50-64,
 * CSR::apply core/CSR.hpp:132-136).  d_x and d_y must not alias. */
int deco_spmv(deco_ctx ctx, deco_csr A, const double* d_x, double* d_y, int bs);
/* float32 values + float32 vectors (requires deco_csr_make_f32). */
int deco_spmv_f32(deco_ctx ctx, deco_csr A, const float* d_x, float* d_y, int bs);
/* d_r = d_b - A d_x (the residual the solvers form, solver/rgmres.tpp:43-47). */
int deco_residual(deco_ctx ctx, deco_csr A, const double* d_b, const double* d_x, double* d_r);

/* ------------------------------------------------------------------- FSAI
 * FSAI(const ptree&, shared_ptr<CSR>) of precond/FSAI/FSAI.hpp:14-37:
 * optional filtered copy (filter_proper(tol_rel), then filter(tol_abs),
 * core/CSR.hpp:423-525), pattern = lower(A) (power 1) or lower(A^2)
 * (power 2) (precond/FSAI/symbolic.tpp:101-176), one dense LU per row
 * (numeric.tpp:59-133), D-scaling (diagonal.cpp:6-73), FU stored transposed
 * (core/CSR.hpp:151-211).  precision: 64 or 32 (float32 factor values for
 * the apply; the setup always computes in float64). */
int deco_fsai_create(deco_ctx ctx, deco_csr A, double tol_rel, double tol_abs, int power, int precision,
                     deco_fsai* out);
int deco_fsai_destroy(deco_fsai F);
int deco_fsai_info(deco_fsai F, int* n, int* nz, int* max_order);
/* Cell-block copies of the two factors (deco_csr_set_blocks): block size (0
 * without) and stored blocks of FL and of FU^T. */
int deco_fsai_blocks(deco_fsai F, int* bs, int* nblk_lower, int* nblk_upper);
/* Padded slots of FL and FU^T (deco_csr_padded): per cell of their 2x2- or
 * 3x3-block copies, or per row for factors without cell blocks (the pressure
 * FSAI); 4 for power-1 factors of 7-point systems, 0 without.  No counterpart in the
 * reference. */
int deco_fsai_padded(deco_fsai F, int* slots_lower, int* slots_upper);
/* Bytes per slot column of FL's and FU^T's padded copies (deco_csr_slot_codes).
 * No counterpart in the reference. */
int deco_fsai_slot_codes(deco_fsai F, int* bytes_lower, int* bytes_upper);
/* FL (lower, diagonal last) and FU^T (upper) in the reference's layout. */
int deco_fsai_download(deco_ctx ctx, deco_fsai F, int* h_Lr, int* h_Lc, double* h_Lv, int* h_Ur, int* h_Uc,
                       double* h_Uv);
/* y = FU^T (FL x)  (FSAI::precond, FSAI.hpp:40-47).  d_x may equal d_y. */
int deco_fsai_apply(deco_ctx ctx, deco_fsai F, const double* d_x, double* d_y);
/* Same product as deco_fsai_apply, for callers that must not allocate device
 * memory while they run (an application whose own pool owns all device memory
 * after start-up, or a time-stepping loop that may not allocate once started).
 * This call allocates nothing: the intermediate FL x lives in one fixed 8 MiB
 * device array inside the library, shared by every call and every handle, so F
 * may have at most 2^20 rows (larger factors return DECO_ERR_ARG).  The first
 * call on a device looks up that array's address; make it before any stream
 * capture.  Calls that overlap on the GPU (several streams at once) race on the
 * array.  Has no counterpart in the reference. */
int deco_fsai_apply_static(deco_ctx ctx, deco_fsai F, const double* d_x, double* d_y);
/* y = FU^T (FL x) with float32 vectors, for a factor made with precision 32:
 * the product a mixed-precision CPR applies inside its own preconditioner
 * (float32 values, float32 intermediate).  d_x may equal d_y.  A precision-64
 * factor returns DECO_ERR_ARG.  Has no counterpart in the reference (its FSAI
 * works in double only). */
int deco_fsai_apply_f32(deco_ctx ctx, deco_fsai F, const float* d_x, float* d_y);

/* -------------------------------------------------------------------- CPR
 * CPR<int,int,double,Mglobal,Mlocal>(const ptree& prec, shared_ptr<CSR> A, V*& b)
 * of precond/CPR.hpp:42-172.  Mutates A and d_b in place exactly as the
 * reference (fix_diag, weights, row scaling, optional DRS, IMPES, CPD,
 * optional zero filter, A_pp extraction and filter, FSAI setups, fix_diag
 * undone).  The fields mirror the JSON keys read there. */
typedef struct deco_cpr_params {
  int block_size;        /* prec.block_size (2 or 3)                         */
  int pressure_id;       /* prec.pressure_id                                 */
  int seq;               /* prec.seq: 0, 1, 2 or 3                           */
  int weights;           /* prec.weights: 0 none, 1 quasiimpes, 2 quasiimpes_GE */
  int use_drs;           /* prec.use_drs                                     */
  double drs_e_dd;       /* prec.drs.e_dd                                    */
  double drs_e_ps;       /* prec.drs.e_ps                                    */
  int cpd;               /* prec.CPD                                         */
  double tol_zero;       /* prec.tol_zero                                    */
  double glo_tol_rel, glo_tol_abs; int glo_power;  /* prec.prec_glo.{tol_rel,tol_abs,power} */
  double loc_tol_rel, loc_tol_abs; int loc_power;  /* prec.prec_loc.{tol_rel,tol_abs,power} */
  int precision;         /* 64: float64 preconditioner; 32: float32 factors,
                            float32 A copy and float32 vectors inside the apply */
  int glo_type;          /* prec.prec_glo.type: 0 FSAI, 1 Jacobi (CPR<...,Jacobi,...>) */
  int loc_type;          /* prec.prec_loc.type: 0 FSAI, 1 Jacobi                */
  int glo_block_size;    /* prec.prec_glo.block_size: block size of the Jacobi of
                            seq 2 or of a Jacobi global stage (1: point Jacobi) */
  int loc_block_size;    /* prec.prec_loc.block_size (Jacobi local stage)       */
} deco_cpr_params;

int deco_cpr_create(deco_ctx ctx, deco_csr A, double* d_b, const deco_cpr_params* prm, deco_cpr* out);
int deco_cpr_destroy(deco_cpr P);
/* x = M^{-1} r with the configured sequence (apply_seq0/1/2/3, CPR.hpp:176-299). */
int deco_cpr_apply(deco_ctx ctx, deco_cpr P, const double* d_r, double* d_x);
/* Borrowed handles of the pressure matrix and the two FSAI factors
 * (which = 0 global on A, 1 local on A_pp).  Valid while P lives. */
int deco_cpr_pressure(deco_cpr P, deco_csr* Ap);
int deco_cpr_fsai(deco_cpr P, int which, deco_fsai* F);
/* Setup timings in milliseconds: [decoupling, A_pp extraction, FSAI global,
 * FSAI local, total] (the reference's profiler nodes "decoupling",
 * "get local matrix", "Global precond", "Local  precond", "Prec"). */
int deco_cpr_timings(deco_cpr P, double* h_ms5);
/* Number of diagonal entries fix_diag replaced (CPR.hpp:753-840). */
int deco_cpr_fixed_diagonals(deco_cpr P, int* count);
/* Decouples another right-hand side d_b (n doubles, in place) with the row
 * operations deco_cpr_create applied to A and its b: the same per-cell row
 * swap, weights, DRS reset, IMPES sum and CPD product, rounded identically,
 * so the result is bit-identical to a vector decoupled by deco_cpr_create.
 * The reference decouples only the b it is constructed with
 * (precond/CPR.hpp:42-172); this serves several right-hand sides per setup. */
int deco_cpr_decouple_rhs(deco_ctx ctx, deco_cpr P, double* d_b);

/* ------------------------------------------------------------------ solve
 * SOL<R,C,V>(ptree sol, A, precond, b, x) of solver/SOL.hpp:19-39 with
 * type rgmres (solver/rgmres.tpp) or lgmres (solver/lgmres.tpp).  The
 * Arnoldi step is classical Gram-Schmidt with one reorthogonalisation
 * (CGS2) instead of the reference's modified Gram-Schmidt.
 * precision 64: float64 everywhere.  precision 32: float32 Krylov basis and
 * inner SpMV with float64 dot accumulation, float64 Hessenberg/Givens and a
 * float64 true residual and solution update at every restart (iterative
 * refinement); requires a CPR built with precision 32. */
typedef struct deco_sol_params {
  int type;              /* 0 rgmres, 1 lgmres                               */
  double reltol;         /* sol.reltol                                       */
  int restart;           /* sol.restart, 1..1000 (the reference allows any)  */
  int itmax;             /* sol.itmax (total inner iterations)               */
  int verbosity;         /* sol.verbosity                                    */
  int precision;         /* 64 or 32                                         */
  int use_x0;            /* 1: d_x holds the initial guess; 0: start at zero */
} deco_sol_params;

typedef struct deco_sol_result {
  int iter;              /* inner iterations (SOL::iter)                     */
  int flag;              /* 0 converged, 1 not converged (SOL::flag)          */
  double res_abs;        /* final residual norm (SOL::res_abs)               */
  double res_rel;        /* res_abs / ||b|| (SOL::res_rel)                   */
  double t_solve_ms;     /* device time of the solve                         */
  int restarts;          /* completed restart cycles                         */
  /* with the environment variable DECO_PROFILE=1: device time summed over the
   * Arnoldi steps spent in the preconditioner, in the SpMV with A, and in the
   * orthogonalisation (0 otherwise) */
  double t_precond_ms, t_matvec_ms, t_ortho_ms;
  /* ||b0 - A0 x|| / ||b0|| for the ORIGINAL system A0 x = b0, before the CPR
   * decoupling rewrote A and b (res_rel is on the decoupled system, as the
   * reference reports it).  Equals the true relative residual when P is NULL. */
  double res_rel_orig;
  /* with DECO_PROFILE=1: the part of t_ortho_ms spent in the dot pass (the rest
   * is the update pass) */
  double t_dots_ms;
} deco_sol_result;

/* Solves A x = b with preconditioner P (NULL: identity).  A and d_b are the
 * (decoupled) system.  h_resvec (optional, host, itmax+1 doubles) receives
 * the residual history |g_j|/||b|| that the reference computes
 * (rgmres.tpp:61) but discards. */
int deco_gmres_solve(deco_ctx ctx, deco_csr A, deco_cpr P, const double* d_b, double* d_x,
                     const deco_sol_params* prm, deco_sol_result* res, double* h_resvec);

/* ---------------------------------------------------------------- adjoint
 * Differentiation of x = A^{-1} b (no counterpart in the reference).  For a
 * loss L(x) with g = dL/dx the adjoint solve is A^T lambda = g; then
 * dL/db = lambda and dL/dA_ij = -lambda_i x_j on A's sparsity pattern.  The
 * adjoint system is A^T transposed first and then decoupled per cell by the
 * same CPR setup as the forward system (decoupling the transpose of an
 * already decoupled matrix leaves singular cell blocks), so lambda solves
 * the original A^T lambda = g, with no back-transformation.  Only x from the
 * forward solve is kept; no Krylov basis is stored. */

/* At = A^T on the device: rows of At list their entries in ascending column
 * order (the order of core/CSR.hpp:193-206's sequential scatter). */
int deco_csr_transpose(deco_ctx ctx, deco_csr A, deco_csr* At);

/* d_grad[e] = alpha * (d_lambda[i] * d_x[j]) for every stored entry e = (i, j)
 * of A, in A's CSR order; alpha = -1 gives dL/dA. */
int deco_grad_A_pattern(deco_ctx ctx, deco_csr A, const double* d_lambda, const double* d_x, double alpha,
                        double* d_grad);

typedef struct deco_adjoint_s* deco_adjoint;

/* Builds A^T from A (its current values: pass the matrix before any forward
 * decoupling) and the CPR preconditioner of the transposed system.  A is not
 * modified and may be destroyed afterwards. */
int deco_adjoint_create(deco_ctx ctx, deco_csr A, const deco_cpr_params* prm, deco_adjoint* out);
int deco_adjoint_destroy(deco_adjoint J);
/* Solves A^T d_lambda = d_g (d_g is not modified); prm, res, h_resvec as in
 * deco_gmres_solve.  Any number of right-hand sides may be solved with one
 * deco_adjoint. */
int deco_adjoint_solve(deco_ctx ctx, deco_adjoint J, const double* d_g, double* d_lambda,
                       const deco_sol_params* prm, deco_sol_result* res, double* h_resvec);
/* The transposed matrix (decoupled in place by the adjoint's CPR) and its
 * preconditioner, owned by J. */
int deco_adjoint_parts(deco_adjoint J, deco_csr* At, deco_cpr* P);

/* ------------------------------------------------------------ batched solve
 * Many independent systems, each with nrhs right-hand sides, solved together
 * (no counterpart in the reference).  The systems are one block-diagonal
 * matrix A: system q owns rows [h_row_off[q], h_row_off[q+1]) (cell-aligned)
 * and references only its own columns.  deco_batch_create builds ONE CPR on A
 * (decoupling A in place, as deco_cpr_create), which is every system's CPR at
 * once.  Right-hand sides and solutions are row-interleaved multi-vectors:
 * B[row * nrhs + k].  Every (system, column) pair is an rgmres(m) instance with
 * its own Hessenberg matrix, rotations, convergence checks (inner and outer,
 * rgmres.tpp:58-66,118-123) and iteration limit; all instances advance in
 * lockstep through products that read the matrix once for all columns, and a
 * restart cycle runs as one CUDA graph. */
typedef struct deco_batch_s* deco_batch;

typedef struct deco_batch_result {
  int max_iter;          /* largest inner iteration count over the instances  */
  int converged;         /* instances with flag 0                             */
  int cycles;            /* restart cycles run                                */
  int graph;             /* 2: one graph launch with a device-side cycle loop;
                            1: the cycle graph relaunched per cycle; 0: direct */
  double t_solve_ms;     /* device time of the solve                          */
} deco_batch_result;

/* nrhs: 1, 2, 4 or 8.  prm: CPR seq 0 or 3 with FSAI stages; the systems must
 * consist of dense bs x bs cell blocks (their products use cell-block copies). */
int deco_batch_create(deco_ctx ctx, deco_csr A, int nsys, const int* h_row_off, int nrhs,
                      const deco_cpr_params* prm, deco_batch* out);
int deco_batch_destroy(deco_batch B);
/* h_widths (optional, nsys ints): the product width chosen for each system. */
int deco_batch_info(deco_batch B, int* nsys, int* nrhs, int* nchunk, int* h_widths);
int deco_batch_cpr(deco_batch B, deco_cpr* P);
/* X = M^{-1} R for every system and column with the batch's CPR (float64 in and
 * out; precision 32 runs the float32 preconditioner, as at a GMRES restart). */
int deco_batch_apply(deco_ctx ctx, deco_batch B, const double* d_R, double* d_X);
/* Solves every instance from x = 0.  d_B: the ORIGINAL right-hand sides (not
 * decoupled; they are decoupled into scratch by the recorded row operations).
 * prm.type must be rgmres and prm.precision the CPR's.  Optional host outputs,
 * nsys * nrhs each in (system, column) order: iterations, final true relative
 * residual of the decoupled system, flag. */
int deco_batch_solve(deco_ctx ctx, deco_batch B, const double* d_B, double* d_X, const deco_sol_params* prm,
                     int* h_iters, double* h_res_rel, int* h_flags, deco_batch_result* res);

#ifdef __cplusplus
}
#endif
#endif
