/*
 * CPU oracle: a plain-C restatement of the reference's pressure-Poisson
 * path (PSI-BOIL Src/Field/Scalar, Src/Solver/Linear/Krylov,
 * Src/Solver/Preconditioner, Src/Solver/Additive, Src/Domain coarsening).
 *
 * TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load it, and only as the checker. The
 * engine never calls it.
 *
 * Layout: interior cells only, index = (i*ny + j)*nz + k (k fastest), i.e.
 * the reference's val[i][j][k] block without its BW=3 halo. Halo values in
 * the reference are zero on the non-periodic faces of these problems and
 * the boundary coefficients are zero after the boundary correction, so every
 * out-of-domain neighbour term is taken as the product with a zero value,
 * in the reference's operation order. On a periodic axis the halo holds the
 * cell at the other end (Scalar::exchange, scalar_exchange.cpp:47-58), so
 * the neighbour across that face is that cell.
 */
#ifndef PSIBOIL_ORACLE_H
#define PSIBOIL_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int nx, ny, nz;
  double *c, *w, *e, *s, *n, *b, *t;
  int per;   /* periodic axes: bit 0 i, 1 j, 2 k (the reference's periodic
                halo, scalar_exchange.cpp:47-58, zero jump value) */
} orc_mat;

typedef struct {
  int converged;   /* the solver's boolean result                         */
  int iterations;  /* iterations actually performed                       */
  int printed;     /* the count the reference prints ("iterations = i+1") */
  double res0, res;
  int status;      /* 0 ok, 1 max-iter, 2 stale, 3 breakdown, 4 initial  */
} orc_stats;

/* y = A x, operation order of Scalar::operator=(const A_x&)
 * (Src/Field/Scalar/scalar_operators.cpp:49-72). */
void orc_spmv(const orc_mat *A, const double *x, double *y);
/* r = b - A x, order of Scalar::operator=(const y_m_A_x&) (:22-46). */
void orc_resid(const orc_mat *A, const double *x, const double *b, double *r);
/* Scalar::dot (scalar.h:296-298), sequential i,j,k order. */
double orc_dot(size_t n, const double *x, const double *y);
/* Scalar::dot_voldiv_avg (scalar.h:317-326) with a uniform cell volume. */
double orc_dot_voldiv_avg(size_t n, const double *x, const double *y, double dV);
/* Scalar::max_abs_voldiv (scalar_minmax.cpp:155-165). */
double orc_max_abs_voldiv(size_t n, const double *x, double dV);

/* CG with the diagonal preconditioner, CG::solve (cg.cpp:10-182) with
 * Diagonal::form/solve (preconditioner_form.cpp:4-13,
 * preconditioner_solve.cpp:4-11). x is updated in place. `hist`, if not
 * NULL, receives res after each iteration (up to maxit entries). */
int orc_cg(const orc_mat *A, double *x, const double *b, int mini, int maxit,
           double res_rat, double res_tol, double scale, int stalecount,
           double dV, orc_stats *st, double *hist);
/* the same with a preconditioner: prec 0 Diagonal, 1/2/3 IncompleteCholesky0/2/3 */
int orc_cg_prec(const orc_mat *A, double *x, const double *b, int mini, int maxit,
                double res_rat, double res_tol, double scale, int stalecount,
                double dV, orc_stats *st, double *hist, int prec);

/* BiCGStab with the diagonal preconditioner, BiCGS::solve (bicgs.cpp:9-229). */
int orc_bicgs(const orc_mat *A, double *x, const double *b, int mini, int maxit,
              double res_rat, double res_tol, double scale, int stalecount,
              double dV, orc_stats *st, double *hist);
/* the same with a preconditioner (prec as for orc_cg_prec) */
int orc_bicgs_prec(const orc_mat *A, double *x, const double *b, int mini, int maxit,
                   double res_rat, double res_tol, double scale, int stalecount,
                   double dV, orc_stats *st, double *hist, int prec);
/* Conjugate gradient squared, CGS::solve (cgs.cpp:8-210). */
int orc_cgs_prec(const orc_mat *A, double *x, const double *b, int mini, int maxit,
                 double res_rat, double res_tol, double scale, int stalecount,
                 double dV, orc_stats *st, double *hist, int prec);

/* Jacobi::solve (Src/Solver/Linear/Iterative/jacobi.cpp:10-75) with the
 * matrix's stored inverse central coefficient ci; st->res0/res are sqrt(r.r). */
int orc_jacobi(const orc_mat *A, const double *ci, double *x, const double *b, int mini,
               int maxit, double res_rat, double res_tol, orc_stats *st, double *hist);
/* GaussSeidel::solve (gaussseidel.cpp:10-117), lexicographic in-place sweeps. */
int orc_gauss_seidel(const orc_mat *A, const double *ci, double *x, const double *b, int mini,
                     int maxit, double res_rat, double res_tol, double scale, int stalecount,
                     double dV, orc_stats *st, double *hist);

/* Additive-correction multigrid (Src/Solver/Additive) around the levels'
 * solver (CG unless orc_ac_set_smoother names another). */
typedef struct orc_ac orc_ac;

/* Builds the level hierarchy with Domain::coarsen's rule
 * (domain_coarsen.cpp:6-112, factor from domain_factor.cpp:4-21) and the
 * OR-coarsened active flags (additive_coarsen_flag.cpp:4-41). aflag: 1 =
 * active. h: fine spacing (uniform). is2d: z is a dummy direction. */
orc_ac *orc_ac_create(const orc_mat *A, const uint8_t *aflag, double h);
void orc_ac_destroy(orc_ac *ac);
/* The solver of every level (default CG): 0 CG, 1 BiCGS, 2 CGS (with the
 * Prec code prec), 3 Jacobi, 4 Gauss-Seidel (level 0 with ci0, the stored
 * A.ci, kept by the caller; coarse levels with 1/c). */
void orc_ac_set_smoother(orc_ac *ac, int kind, int prec, const double *ci0);
/* AC::resrat / AC::restol (the level solvers' ResRat and ResTol, atto by
 * default, additive.h:105-110), AC::use_linf_error (additive.h:141) and AC's
 * own solver (AC(cen, sol): sol_kind -1 = the levels' solver, else 0 CG,
 * 1 BiCGS, 2 CGS, 3 Jacobi, 4 Gauss-Seidel, with sol_prec), which
 * call_solver uses for post-smoothing and the coarsest level
 * (additive_cycle_functions.cpp:100-107). */
void orc_ac_set_params(orc_ac *ac, double resrat_val, double restol_val, int use_linf,
                       int sol_kind, int sol_prec);
/* 1 when the last flex cycle stopped at its visit bound (see oracle.c),
 * and the bound itself (smoother calls per flex cycle, 10^6 by default) */
int orc_ac_flex_capped(const orc_ac *ac);
void orc_ac_set_flex_cap(orc_ac *ac, long long cap);
int orc_ac_nlevels(const orc_ac *ac);
void orc_ac_level_dims(const orc_ac *ac, int l, int *dims /* 3 */);
/* Coarse operators of all levels (AC::coarsen_system,
 * additive_coarsen_system.cpp:4-140). Called by orc_ac_cycle too. */
void orc_ac_coarsen_all(orc_ac *ac);
/* Copies level l's 7 coefficient arrays (c,w,e,s,n,b,t) out. */
void orc_ac_level_matrix(const orc_ac *ac, int l, double *out7);

/* AC::cycle (additive_cycle.cpp:4-99, additive_cycle_functions.cpp,
 * additive_recursive.cpp). init/loop: -1 none, 1 V, 2 F, 4 W, 5 flex; a
 * loop of none is the reference's "just solve" branch.
 * toler: ResTol, factor: ResRat (negative disables), mv/ms as in the
 * reference, max_cyc/min_cyc/stop_if_div/priority_min_cyc as the setters.
 * res_hist receives [initial res, res after cycle 1, ...] (max_cyc+2). */
int orc_ac_cycle(orc_ac *ac, double *x, const double *b, int init, int loop,
                 double toler, double factor, const int mv[3], const int ms[3],
                 int max_cyc, int min_cyc, int stop_if_div, int priority_min_cyc,
                 int *ncyc, double *res_hist, int *nhist);

#ifdef __cplusplus
}
#endif
#endif
