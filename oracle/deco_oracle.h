/* deco_oracle.h — plain-C restatement of the reference's CPR-Krylov hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the CPU checker the GPU path is compared
 * against; it is itself pinned against the reference compiled from its own
 * sources (oracle/_ref/libdeco_ref.so) by tests/test_oracle.py and by the
 * golden fixtures in tests/golden/.  Nothing in the product links it.
 *
 * Conventions follow the reference: CSR with int32 row pointers / columns and
 * float64 values (core/CSR.hpp:4-13), sorted columns, cell-major unknowns with
 * the pressure at offset p of each block of bs rows.
 */
#ifndef DECO_ORACLE_H
#define DECO_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_csr {
  int n, m, nz;
  int *r, *c;
  double *v;
} orc_csr;

typedef struct orc_fsai {
  orc_csr FL;  /* lower, diagonal last in each row            */
  orc_csr FU;  /* transposed: upper CSR, rows ascending        */
} orc_fsai;

typedef struct orc_cpr_params {
  int bs, p, seq;
  int weights;           /* 0 none, 1 quasiimpes, 2 quasiimpes_GE          */
  int use_drs;
  double e_dd, e_ps;
  int cpd;
  double tol_zero;
  double loc_tol_rel;    /* prec_loc.tol_rel: filter of A_pp in CPR          */
  double glo_tol_rel, glo_tol_abs; int glo_power;
  double loc_tol_abs;    int loc_power;
} orc_cpr_params;

typedef struct orc_cpr {
  orc_cpr_params prm;
  orc_csr A;             /* decoupled system (mutated copy)                */
  double* b;             /* decoupled rhs                                  */
  orc_csr Ap;            /* pressure matrix                                */
  orc_fsai glo, loc;
  double *w, *J, *xp, *rt, *tmp_g, *tmp_l;
  char* check_diag;
  int n, sn;
} orc_cpr;

void orc_csr_free(orc_csr* A);

void orc_spmv(int n, const int* r, const int* c, const double* v, const double* x, double* y, int bs);
int orc_filter(orc_csr* A, double tol, int relative, int shift);
int orc_fsai_setup(const orc_csr* A, double tol_rel, double tol_abs, int power, orc_fsai* F);
void orc_fsai_apply(const orc_fsai* F, const double* x, double* tmp, double* y);
void orc_fsai_free(orc_fsai* F);

int orc_cpr_setup(const orc_cpr_params* prm, int n, const int* r, const int* c, const double* v,
                  const double* b, orc_cpr** out);
void orc_cpr_apply(orc_cpr* P, const double* r, double* x);
void orc_cpr_free(orc_cpr* P);

/* left = 0: right-preconditioned rgmres (solver/rgmres.tpp); 1: lgmres */
int orc_gmres(orc_cpr* P, int left, double reltol, int restart, int itmax, double* x, int* iter,
              double* res_abs, double* res_rel, int* flag, double* resvec);

/* Accessors for bindings */
int orc_cpr_sizes(const orc_cpr* P, long long* out5);
void orc_cpr_get(const orc_cpr* P, int which, int* r, int* c, double* v, int* r2, int* c2, double* v2);
void orc_cpr_get_b(const orc_cpr* P, double* b);

#ifdef __cplusplus
}
#endif
#endif
