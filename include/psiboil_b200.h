/*
 * psiboil_b200: B200-native pressure-Poisson engine — C ABI.
 *
 * Plain pointers and sizes only; every function returns an int status
 * (PBG_OK or a negative PBG_ERR_*) and never aborts. pbg_last_error()
 * returns the message of the calling thread's last failure.
 *
 * The reference (PSI-BOIL) has no C ABI or plugin interface; its swap
 * points are C++ virtuals. Each entry point below names the reference
 * interface it stands in for:
 *   - Linear::solve / Krylov::solve        Src/Solver/Linear/linear.h:46-56,
 *                                          Src/Solver/Linear/Krylov/krylov.h:20-30
 *   - CG::solve, BiCGS::solve, CGS::solve  Src/Solver/Linear/Krylov/cg.cpp:10-182,
 *                                          bicgs.cpp:9-229, cgs.cpp:8-210
 *   - Jacobi::solve, GaussSeidel::solve    Src/Solver/Linear/Iterative/jacobi.cpp:10-75,
 *                                          gaussseidel.cpp:10-117
 *   - AC::AC, AC::cycle and the vcycle/fcycle/wcycle/fullcycle overloads and
 *     setters                             Src/Solver/Additive/additive.h:26-142
 *   - Matrix (c, w, e, s, n, b, t, ci)     Src/Matrix/matrix.h:23-54
 *   - Pressure::discretize                 Src/Equation/Centered/Pressure/pressure_discretize.cpp:11-151
 *     (with a cut Body: Src/Body/body_interface.cpp fV, fSw..fSt)
 *   - Pressure::update_rhs                 pressure_update_rhs.cpp:16-139
 *   - Momentum::project                    Src/Equation/Staggered/Momentum/momentum_project.cpp:11-80
 *   - Scalar::operator=(A_x), (y_m_A_x)    Src/Field/Scalar/scalar_operators.cpp:22-72
 *   - Scalar::dot, dot_voldiv_avg          Src/Field/Scalar/scalar.h:296-326
 *
 * Array layout. Compact arrays hold interior cells only, index
 * (i*ny + j)*nz + k with k fastest. Strided entry points take the
 * reference's contiguous val[0][0] block directly: element (i,j,k) of the
 * interior lives at base[offset + i*si + j*sj + k*sk]; for a PSI-BOIL
 * Scalar with BW = 3 that is si = (nj+6)*(nk+6), sj = nk+6, sk = 1,
 * offset = 3*(si+sj+sk).
 *
 * `where` says whether caller pointers are host (PBG_HOST) or device
 * (PBG_DEVICE, on the session's device) memory. A session works on its own
 * non-blocking stream (pbg_session_stream), which other streams' work is
 * not ordered against: device inputs must be complete before the call
 * (make the session's stream wait on an event of the stream that wrote
 * them, or synchronise that stream). A call returns with its results
 * complete.
 */
#ifndef PSIBOIL_B200_H
#define PSIBOIL_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PBG_API_VERSION 1

typedef struct pbg_session pbg_session;

/* call status */
enum {
  PBG_OK = 0,
  PBG_ERR_ARG = -1,
  PBG_ERR_CUDA = -2,
  PBG_ERR_STATE = -3,
  PBG_ERR_NOMEM = -4,
  PBG_ERR_UNSUPPORTED = -5,
  PBG_ERR_ADMISSION = -6
};

/* solve status (pbg_result.status) */
enum {
  PBG_CONVERGED = 0,
  PBG_MAXITER = 1,
  PBG_STALE = 2,
  PBG_BREAKDOWN = 3,
  PBG_INITIAL = 4,   /* converged before the first iteration */
  PBG_NAN = 5,
  PBG_DIVERGED = 6   /* AC divergence guard, or an engine refinement sweep that did not
                        reduce the residual: the last good iterate restored */
};

enum { PBG_HOST = 0, PBG_DEVICE = 1 };
enum { PBG_BC_NEUMANN_ = 0, PBG_BC_DIRICHLET_ = 1, PBG_BC_PERIODIC_ = 2 };

/* solvers */
enum {
  PBG_SOLVER_CG = 0,      /* CG with diagonal preconditioner (reference parity)   */
  PBG_SOLVER_BICGS = 1,   /* BiCGStab with diagonal preconditioner (parity)       */
  PBG_SOLVER_AC = 2,      /* additive-correction multigrid, level solver from
                             ac_smoother (parity)                               */
  PBG_SOLVER_ENGINE = 3,  /* flexible CG + AC K-cycle (the engine's fast solver)  */
  PBG_SOLVER_CGS = 4,     /* conjugate gradient squared, CGS::solve (parity)       */
  PBG_SOLVER_JACOBI = 5,  /* Jacobi::solve (Src/Solver/Linear/Iterative, parity)   */
  PBG_SOLVER_GAUSS_SEIDEL = 6  /* GaussSeidel::solve, lexicographic (parity)       */
};
enum { PBG_FP64 = 0, PBG_MIXED = 1 };
enum { PBG_CYCLE_NONE = -1, PBG_CYCLE_V = 1, PBG_CYCLE_F = 2, PBG_CYCLE_W = 4, PBG_CYCLE_FLEX = 5 };

typedef struct {
  int solver;
  int precision;          /* PBG_FP64 or PBG_MIXED (engine only)                */
  /* Linear::solve(A, x, b, MinIter, MaxIter, name, ResRat, ResTol, scale,
   * stalecount, precform) */
  int min_iter;
  int max_iter;
  double res_rat;         /* ResRat (default 0.01); < 0 disables              */
  double res_tol;         /* ResTol (default 1e-15)                            */
  double scale;
  int stalecount;         /* <= 0: off; at most 64                              */
  /* AC::cycle(init, loop, ResTol, ResRat, mv, ms, &ncyc) and setters */
  int init_cycle;         /* PBG_CYCLE_NONE | V | F | W | FLEX (a full cycle first) */
  int loop_cycle;         /* PBG_CYCLE_V | F | W | FLEX, or PBG_CYCLE_NONE: the
                             reference's "just solve" branch (additive_cycle.cpp:
                             66-71): one call of AC's solver on level 0 (MaxIter 40,
                             ResRat 0.001, ResTol 1e-15), then not converged with
                             cycles = max_cycles                                */
  double toler;           /* ResTol of the cycle loop (< 0 disables)            */
  double factor;          /* ResRat of the cycle loop (< 0 disables)            */
  int max_cycles, min_cycles, stop_if_div, priority_min_cyc;
  int mv[3], ms[3];
  /* engine */
  double tol;             /* target |b - A x| / |b| (FP64 true residual)        */
  double inner_tol;       /* mixed: FP32 inner solve reduction per sweep         */
  int max_sweeps;         /* mixed: refinement sweeps at most                    */
  /* reference-parity solvers: 1 = every global sum rounded as the
   * reference's sequential i,j,k loop rounds it (bit-for-bit reference
   * results; computed in parallel, see pbg_seq_sum, about 15x the time of
   * a tree sum); 0 = deterministic tree sums */
  int exact_sums;
  /* engine: cells of the dense coarsest level (0: 512). Larger (4096) saves
   * launches in repeated solves with one matrix and costs a longer set-up
   * after every matrix change (a dense inverse, O(cells^3)). */
  int coarse_max;
  /* Krylov preconditioner (CG, BiCGS, CGS), the reference's Prec codes
   * (preconditioner.h:15-29): 0 diagonal (Prec::di, default), 1 IC0, 2 IC2,
   * 3 IC3 (incomplete Cholesky, preconditioner_form.cpp:16-144 /
   * preconditioner_solve.cpp:14-110; bit for bit with exact_sums). The IC
   * factor reads the lower couplings w, s, b, as the reference's does, also
   * for a non-symmetric matrix. */
  int prec;
  /* 1: start from x = 0 whatever x holds (x is then output only, and with
   * PBG_HOST it is not copied to the device); 0: x is the initial guess,
   * as in the reference's Linear::solve. */
  int x0_zero;
  /* PBG_SOLVER_AC: the solver that smooths every level and solves the
   * coarsest one, the Linear the reference's Centered object holds
   * (additive_cycle_functions.cpp:90-107): PBG_SOLVER_CG (default),
   * PBG_SOLVER_BICGS, PBG_SOLVER_CGS (each with `prec`), PBG_SOLVER_JACOBI
   * or PBG_SOLVER_GAUSS_SEIDEL (level 0 with the uploaded A.ci, coarse levels
   * with ci = 1/c, as additive_coarsen_system.cpp forms it). */
  int ac_smoother;
  /* PBG_SOLVER_AC: AC's own solver, AC(cen, sol) (additive.cpp:41-45), which
   * call_solver uses for post-smoothing and the coarsest level
   * (additive_cycle_functions.cpp:100-107): -1 (default) the same as
   * ac_smoother, else a solver code as for ac_smoother with ac_solver_prec. */
  int ac_solver, ac_solver_prec;
  /* PBG_SOLVER_AC: AC::resrat / AC::restol, the ResRat and ResTol of the
   * level solvers (additive.h:105-110; default 1e-18, boil::atto). */
  double ac_resrat, ac_restol;
  /* PBG_SOLVER_AC: AC::use_linf_error (additive.h:141): 1 drives the cycle's
   * tests with max |r/dV| instead of the volume-averaged 2-norm. */
  int use_linf;
  /* PBG_SOLVER_AC with PBG_CYCLE_FLEX: smoother calls per flex cycle at most
   * (0: 10^6). The reference's flex cycle returns only when level 0's
   * smoother reaches AC::resrat, and runs forever when it never does; at this
   * bound the cycle ends and the solve reports PBG_MAXITER. */
  int flex_visits;
  /* PBG_SOLVER_AC: the time step dt that scales AC's residual measure
   * (additive_residual.cpp:19-27, L[0]->time->dt(); default 1). The level
   * solvers get `scale` as their scale (the reference passes dti * scale,
   * additive_cycle_functions.cpp:90-107). */
  double ac_dt;
} pbg_params;

typedef struct {
  int status;             /* PBG_CONVERGED ...                                   */
  int converged;          /* the reference's bool return value                    */
  int iterations;         /* Krylov iterations performed (engine: all sweeps)    */
  int cycles;             /* AC cycles (the reference's *ncyc)                    */
  int sweeps;             /* refinement sweeps (engine)                           */
  int levels;             /* multigrid levels                                     */
  double res0, res;       /* reference residual measure at start / end            */
  double relres;          /* engine: FP64 |b - A x| / |b| at return               */
  double seconds;         /* wall time of the call                                */
} pbg_result;

const char *pbg_last_error(void);
int pbg_version(void);
int pbg_device_count(int *count);

/* Defaults of the reference: MinIter(1), MaxIter(20), ResRat(0.01),
 * ResTol(1e-15), scale 1, stalecount -1 (linear.h:46-56, resrat.h,
 * restol.h, maxiter.h); AC defaults of additive.cpp:11-19 (max_cyc 20,
 * min_cyc 0, stop_if_div true, priority_min_cyc true, mv {20,20,20},
 * ms {-1,-1,-1}); engine tol 1e-8, inner_tol 1e-3, max_sweeps 8. */
void pbg_params_default(pbg_params *p, int solver);

/* A session owns one grid (nx, ny, nz interior cells, nz == 1 for 2-D, uniform
 * spacing h), its matrix, the multigrid hierarchies and all scratch on one
 * device. bc: imin, imax, jmin, jmax, kmin, kmax (PBG_BC_NEUMANN_ |
 * PBG_BC_DIRICHLET_ | PBG_BC_PERIODIC_), used by pbg_assemble_pressure.
 * PBG_BC_PERIODIC_ goes on both faces of an axis: the matrix's couplings
 * on that axis's outer faces then join the cells at the two ends, as the
 * reference's periodic halo does (Scalar::exchange,
 * scalar_exchange.cpp:47-58, with a zero jump value). The reference-parity
 * solvers (CG, BiCGS, CGS, Jacobi, Gauss-Seidel, IC preconditioners, AC)
 * take periodic matrices; the on-device assembly, the pressure step and the
 * engine solver return PBG_ERR_UNSUPPORTED on a periodic session. Stands in
 * for the Centered/Pressure object plus its Linear solver
 * (centered.h:62-200). */
int pbg_session_create(int nx, int ny, int nz, double h, const int bc[6], int device,
                       pbg_session **out);
int pbg_session_destroy(pbg_session *s);
int pbg_session_info(const pbg_session *s, long long *ncell, int *symmetric,
                     long long *device_bytes);
/* Cell volume used by the reference-parity residual measure
 * sqrt(dot_voldiv_avg(r, r))/scale (scalar.h:317-326); default h*h*h.
 * Domain::dV of the level (domain_surfaces_volumes.cpp:60-61). */
int pbg_session_set_cell_volume(pbg_session *s, double dV);

/* Upload the seven coefficient arrays of the reference's Matrix
 * (matrix.h:23-54; sign convention A x = c x_P - sum a_nb x_nb), strided
 * as described above. A matrix whose e/n/t equal the next cell's w/s/b bit
 * for bit is stored in the symmetric four-array form. */
int pbg_matrix_upload(pbg_session *s, const double *c, const double *w, const double *e,
                      const double *sv, const double *n, const double *b, const double *t,
                      long long si, long long sj, long long sk, long long offset, int where);
/* Download the matrix in compact layout (any pointer may be NULL). */
int pbg_matrix_download(pbg_session *s, double *c, double *w, double *e, double *sv, double *n,
                        double *b, double *t, int where);
/* Active-cell flags (the reference's ScalarInt aflag, centered.h:196; 1 =
 * active), strided like the matrix. Default: all active. */
int pbg_active_upload(pbg_session *s, const int *aflag, long long si, long long sj, long long sk,
                      long long offset, int where);
/* The matrix's stored inverse central coefficient A.ci (matrix.h:23-54),
 * strided like the matrix, for PBG_SOLVER_JACOBI and PBG_SOLVER_GAUSS_SEIDEL,
 * which divide by it (jacobi.cpp:43, gaussseidel.cpp:51). The reference
 * forms ci before it scales the central coefficient of cells inside a body
 * by 1e-12 (pressure_discretize.cpp:127-138), so there ci is not 1/c. Until
 * it is uploaded, and after every change of the matrix, those solvers use
 * 1/c. */
int pbg_ci_upload(pbg_session *s, const double *ci, long long si, long long sj, long long sk,
                  long long offset, int where);

/* On-device assembly of the pressure matrix from cell densities and a solid
 * mask (1 = solid), Pressure::discretize with a harmonic face density:
 * A.w = dS/dx/rho_face, c = sum, faces touching solid cells zeroed, boundary
 * correction (Neumann c -= a_bnd; Dirichlet a_bnd = 0), solid cells c *= 1e-12
 * (pressure_discretize.cpp:24-148, centered_system_bnd.cpp). Also sets the
 * active flags to !solid. Compact arrays. */
int pbg_assemble_pressure(pbg_session *s, const double *rho, const uint8_t *solid, int where);

/* The pressure-correction step around the solve (compact layouts; faces:
 * u (nx+1) x ny x nz, v nx x (ny+1) x nz, w nx x ny x (nz+1), k fastest,
 * face f of u between cells f-1 and f; w may be NULL in 2-D). Bit for bit
 * the reference on a uniform grid whose coordinates are exact multiples of
 * h (n a power of two).
 *
 * pbg_assemble_mix: Pressure::discretize (pressure_discretize.cpp:24-148)
 * for a two-phase Matter (matter.cpp:78): cell density PropertyMix
 * rho_a*col + rho_b*(1-col) with col clamped to [0,1]
 * (property_value.cpp:52-70), face density the arithmetic mean of the two
 * cells (:73-85; a boundary face takes the boundary cell's), dS/dx with
 * dx = h/2 from a boundary cell's centre to the wall, then
 * Centered::create_system_bnd (Neumann c -= a_bnd; Dirichlet a_bnd = 0).
 * col NULL: one fluid of density rho_a. solid (1 = solid, may be NULL):
 * faces to solid cells cut, solid cells c *= 1e-12. Replaces the host
 * assembly of Pressure(...)/discretize(). Sets the active flags. */
int pbg_assemble_mix(pbg_session *s, const double *col, double rho_a, double rho_b,
                     const uint8_t *solid, int where);
/* Pressure::update_rhs (pressure_update_rhs.cpp:16-139): rhs = dS/dt *
 * (u_w - u_e + v_s - v_n + w_b - w_t) per cell. solid (may be NULL): a
 * voxel body, the immersed-body branch (:65-101): faces to solid
 * neighbours are left out and solid cells get 0. */
int pbg_divergence(pbg_session *s, const double *u, const double *v, const double *w,
                   const uint8_t *solid, double dt, double *rhs, int where);
/* Momentum::project (momentum_project.cpp:11-80): every interior face
 * u += (p[i-1] - p[i]) / rho_face * dt / h (rho_face as in
 * pbg_assemble_mix); with a solid mask the immersed-body branch (:47-73):
 * only faces between two fluid cells, u += (p[i-1] - p[i]) * dt /
 * rho_face / h. The normal faces on the domain boundary keep the caller's
 * values (the boundary condition; walls are 0), w is not touched in 2-D.
 * u, v, w updated in place. */
int pbg_project(pbg_session *s, const double *p, const double *col, double rho_a, double rho_b,
                const uint8_t *solid, double dt, double *u, double *v, double *w, int where);
/* One pressure-correction step on the device: pbg_assemble_mix,
 * pbg_divergence, pbg_solve of p (p in: initial guess; solver scale
 * params->scale / dt as Centered::solve passes, centered_solve.cpp:25-31)
 * and pbg_project. u, v, w and p updated in place; with PBG_HOST each
 * input crosses to the device once and each output back once. */
int pbg_pressure_step(pbg_session *s, const double *col, double rho_a, double rho_b,
                      const uint8_t *solid, double dt, double *u, double *v, double *w,
                      double *p, int where, const pbg_params *params, pbg_result *res);
/* An immersed body with cut cells for the four functions above (the
 * reference's Body after Domain(gx, gy, gz, &body) has cut it): fV the
 * fluid volume fraction of every cell (Body::fV(i,j,k); 0 inside the body,
 * between 0 and 1 in a cut cell), fS the face fractions of every cell as
 * Body::fSw..fSt(i,j,k) return them, six planes of ncell in the order
 * w e s n b t (only the cut cells' are read). The body's cut-cell list is
 * its cut cells (0 < fV < 1). With a body those functions take solid =
 * NULL and follow the reference's body branches: discretize's cut-cell
 * fractions and off-cell decoupling (pressure_discretize.cpp:72-119; the
 * matrix is then stored in the seven-array form, as the two cells of a
 * face carry their own fractions), update_rhs's face fractions (:34-43)
 * and project's fluid-only faces. Cells on the domain boundary must not be
 * cut (PBG_ERR_UNSUPPORTED). fV = NULL removes the body. PBG_SOLVER_ENGINE
 * solves such a matrix by FP64 refinement around its symmetric part; a
 * sweep that does not reduce the residual is undone and ends the solve with
 * PBG_DIVERGED (strongly non-symmetric matrices: use BiCGS or CGS). */
int pbg_body_upload(pbg_session *s, const double *fV, const double *fS, int where);

/* Solve A x = b with x as initial guess and result (x updated in place,
 * b read only), compact layout. The reference-parity solvers follow
 * Linear::solve / AC::cycle semantics (x0 as given, residual measure
 * sqrt(dot_voldiv_avg(r))/scale, stopping tests, return value). */
int pbg_solve(pbg_session *s, double *x, const double *b, int where, const pbg_params *p,
              pbg_result *r);
/* Same with strided x and b (the reference's Scalar blocks). */
int pbg_solve_strided(pbg_session *s, double *x, const double *b, long long si, long long sj,
                      long long sk, long long offset, int where, const pbg_params *p,
                      pbg_result *r);
/* Residual history of the last solve: per iteration (Krylov), per cycle
 * including the initial residual (AC), or per FCG iteration (engine). */
int pbg_history(const pbg_session *s, double *out, int cap, int *count);

/* Operators, compact layout: y = A x (scalar_operators.cpp:49-72),
 * r = b - A x (:22-46), dots (scalar.h:296-326): out[0] = x.y,
 * out[1] = sum x*y/dV/dV / N / N. */
int pbg_spmv(pbg_session *s, const double *x, double *y, int where);
int pbg_residual(pbg_session *s, const double *x, const double *b, double *r, int where);
int pbg_dot(pbg_session *s, const double *x, const double *y, int where, double out[2]);
/* Sequential sum in index order, rounded after every addition: out[0] for
 * a, out[1] for b (0 when b is NULL), n terms. It reproduces the
 * reference's `real sum = 0; for_ijk sum += ...` loops (scalar.h:296-326,
 * the reductions behind CG::solve and AC::residual) bit for bit, computed
 * in parallel; the reference-parity solvers use the same reduction when
 * pbg_params.exact_sums is set. */
int pbg_seq_sum(pbg_session *s, const double *a, const double *b, long long n, int where,
                double out[2]);

/* Multigrid hierarchy sizes: count and per-level dims (3 ints per level).
 * kind 0: the reference AC hierarchy (Domain::coarsen rule), kind 1: the
 * engine's aggregation hierarchy. */
int pbg_levels(pbg_session *s, int kind, int *count, int *dims, int cap);
/* Coarse matrix of the reference AC hierarchy, level l (7 compact arrays
 * c,w,e,s,n,b,t concatenated, AC::coarsen_system). */
int pbg_ac_level_matrix(pbg_session *s, int level, double *out7, int where);

/* Seeded workload generator (the same code the oracle uses): kind 0 single
 * bubble n^3, 1 bubbles + solid cylinder, 2 member of the uneven batch.
 * params: n, nb, rmin, rmax, rc, ratio, index, n2d, s2lo, s2hi, s3lo, s3hi,
 * stream. With rho == NULL only dims/h are returned. */
int pbg_generate(int kind, const double *params, uint64_t seed, int dims[3], double *h,
                 double *rho, uint8_t *solid, double *b);
/* Flow state of one pressure-correction step of the same workload: the
 * liquid colour col (cells), a predicted velocity u, v, w (face layouts of
 * pbg_assemble_mix; walls 0) drawn from stream params[12], and the phase
 * densities rho[0] liquid, rho[1] vapour. */
int pbg_generate_flow(int kind, const double *params, uint64_t seed, double *col, double *u,
                      double *v, double *w, double rho[2]);

/* Instrumentation (no reference counterpart): kernels launched by this
 * library so far in the process; the session's CUDA stream (for events);
 * the average device time of one launch of a hot kernel timed alone with
 * CUDA events (which 0: the engine's fine-level smoothing sweep, precision
 * PBG_FP64 | PBG_MIXED for FP32; which 1: the reference-order FP64 SpMV)
 * and its algorithmic bytes per launch. */
unsigned long long pbg_launch_count(void);
int pbg_session_stream(pbg_session *s, void **stream);
int pbg_bench_kernel(pbg_session *s, int which, int precision, int reps, double *ms,
                     double *bytes_per_launch);

/* ---------------------------------------------------------------------------
 * Batched solves (no counterpart in the reference, which solves one pressure
 * system per Pressure object and MPI rank): many independent problems of
 * uneven 2-D / 3-D sizes solved together by the engine's solver (flexible CG
 * + AC K-cycle; mixed FP32 inner / FP64 refinement, or plain FP64). Every
 * problem keeps its matrix, hierarchy and solution resident on the device
 * until removed; a solve starts from the stored solution (warm start) unless
 * it is reset. Results do not depend on which problems share a solve.
 * ------------------------------------------------------------------------- */
typedef struct pbg_batch pbg_batch;

typedef struct {
  int precision;    /* PBG_MIXED or PBG_FP64                                  */
  int slots;        /* problems in flight at once                             */
  int threads;      /* launch shape: threads per CTA (multiple of 32, 64..512) */
  int tile_cells;   /* cells per tile (>= threads)                            */
  int grid;         /* CTAs per tile kernel                                    */
  int kc_max;       /* levels 1..kc_max run a K-cycle, deeper levels one visit */
  int tail_cells;   /* a problem's coarse levels of at most this many cells run
                       their whole K-cycle in one CTA (0: none)                */
} pbg_batch_config;

void pbg_batch_config_default(pbg_batch_config *c);
int pbg_batch_create(const pbg_batch_config *c, int device, pbg_batch **out);
int pbg_batch_destroy(pbg_batch *b);
/* Device bytes one problem of these dimensions takes (admission control). */
int pbg_batch_problem_bytes(pbg_batch *b, int nx, int ny, int nz, long long *bytes);
/* Add a problem (nx*ny*nz > 64 cells; nz == 1 for 2-D); its id. bc as for
 * pbg_session_create; NULL: Neumann walls with a Dirichlet top (kmax in 3-D,
 * jmax in 2-D). */
int pbg_batch_add(pbg_batch *b, int nx, int ny, int nz, double h, const int bc[6], int *id);
int pbg_batch_remove(pbg_batch *b, int id);
/* Inputs as for a session: cell densities and solid mask (assembled on the
 * device, pbg_assemble_pressure), right-hand side, initial guess (NULL:
 * zero). */
int pbg_batch_set_fields(pbg_batch *b, int id, const double *rho, const uint8_t *solid, int where);
int pbg_batch_set_rhs(pbg_batch *b, int id, const double *rhs, int where);
int pbg_batch_set_x(pbg_batch *b, int id, const double *x, int where);
int pbg_batch_get_x(pbg_batch *b, int id, double *x, int where);
/* Solve problems ids[0..n-1] to p->tol (FP64 |b - A x| / |b|; p->inner_tol,
 * p->max_sweeps, p->max_iter as for the engine). Largest problems are
 * started first; a problem enters as soon as a slot is free. res[i]
 * (optional) gets the outcome; res[i].seconds is the time from the start of
 * the call until problem i finished. */
int pbg_batch_solve(pbg_batch *b, const int *ids, int n, const pbg_params *p, pbg_result *res);
/* Pick the launch shape for this batch: time the solve of ids under each
 * candidate shape and keep the fastest. With cache_path, the choice is read
 * from / written to that JSON file (keyed by device and batch signature).
 * best (optional) receives it; the batch keeps it. */
int pbg_batch_autotune(pbg_batch *b, const int *ids, int n, const pbg_params *p,
                       const char *cache_path, pbg_batch_config *best);

/* ---------------------------------------------------------------------------
 * Serving (no counterpart in the reference): a request loop on one GPU. A
 * session is one grid whose matrix, hierarchy and last solution stay on the
 * device (the next request starts from that solution); sessions are admitted
 * while their device bytes fit the HBM budget. Requests from any thread
 * are queued; a worker thread admits them into the running batch as slots
 * free up (continuous batching: requests that arrive while others are on
 * the GPU join at the next outer iteration) and records each latency from
 * submission to completion. One request per session is in flight at a
 * time; a session's later requests wait for it in order. A result does not
 * depend on the other requests in flight.
 * ------------------------------------------------------------------------- */
typedef struct pbg_server pbg_server;

typedef struct {
  int precision;          /* PBG_MIXED or PBG_FP64                             */
  int slots;              /* requests in flight at once                        */
  long long hbm_budget;   /* device bytes the sessions may take (0: 150 GB)    */
  int iters_per_poll;     /* outer iterations between completion checks        */
  int threads, tile_cells, grid, kc_max, tail_cells;  /* as pbg_batch_config  */
  double tol, inner_tol;  /* as pbg_params                                     */
  int max_sweeps, max_iter;
} pbg_server_config;

typedef struct {
  long long submitted, completed, queued, in_flight;
  long long sessions, device_bytes;   /* admitted sessions and their bytes       */
  unsigned long long kernel_launches;
} pbg_server_stats;

void pbg_server_config_default(pbg_server_config *c);
int pbg_server_create(const pbg_server_config *c, int device, pbg_server **out);
/* Stops the worker after the requests in flight (queued ones are dropped). */
int pbg_server_destroy(pbg_server *s);
/* PBG_ERR_ADMISSION if the session's device bytes do not fit the budget. */
int pbg_server_open_session(pbg_server *s, int nx, int ny, int nz, double h, const int bc[6],
                            int *sid);
/* Waits for the session's requests, then frees its device memory. */
int pbg_server_close_session(pbg_server *s, int sid);
/* Queue a solve on session sid: new cell densities and solid mask (both
 * NULL: matrix unchanged), right-hand side. Host inputs are copied at
 * submission; device inputs are read when the request starts, so they must
 * stay valid until pbg_server_wait returns for it. */
int pbg_server_submit(pbg_server *s, int sid, const double *rho, const uint8_t *solid,
                      const double *rhs, int where, long long *rid);
/* Queue a solve whose inputs are made on the device when it starts: one
 * bubble (centre in cell units, radius in cells, density 1 inside and
 * `ratio` outside) and a uniform right-hand side in [-1, 1] from
 * rhs_seed, made zero-mean over the cells and scaled by 1/h^2. */
int pbg_server_submit_bubble(pbg_server *s, int sid, const double center[3], double radius,
                             double ratio, unsigned long long rhs_seed, long long *rid);
/* Wait for a request (timeout_s < 0: no limit); PBG_ERR_STATE on timeout.
 * latency_s: submission to completion. A request's record is released by
 * the first wait that returns it. */
int pbg_server_wait(pbg_server *s, long long rid, double timeout_s, pbg_result *res,
                    double *latency_s);
/* The session's current solution (waits until it has no request in flight). */
int pbg_server_get_x(pbg_server *s, int sid, double *x, int where);
int pbg_server_stats_get(pbg_server *s, pbg_server_stats *st);

/* ---------------------------------------------------------------------------
 * Checkpoints in the reference's .bck format (Scalar::save / Scalar::load,
 * Src/Field/Scalar/scalar_save.cpp:20-32, scalar_load.cpp:26-37; a Centered
 * checkpoint is phi then cold, centered_save.cpp:4-23): per field three ints
 * (block extents with the BW = 3 halo) and the block's doubles, k fastest.
 * Reading checks the extents (the reference's load does not).
 * ------------------------------------------------------------------------- */
/* name_file(base, ".bck", step, cpu) (Src/Global/global_name_file.cpp:4-33) */
int pbg_bck_name(const char *base, int step, int cpu, char *out, int cap);
/* nfields full blocks of ni x nj x nk doubles */
int pbg_bck_write(const char *path, int nfields, const double *const *fields, int ni, int nj, int nk,
                  int where);
int pbg_bck_read(const char *path, int nfields, double *const *fields, int ni, int nj, int nk, int where);
/* compact interior fields of an nx x ny x nz grid (halo written as zero) */
int pbg_bck_write_compact(const char *path, int nfields, const double *const *fields, int nx, int ny,
                          int nz, int where);
int pbg_bck_read_compact(const char *path, int nfields, double *const *fields, int nx, int ny, int nz,
                         int where);

/* Dot products without allocating (no counterpart in the reference).
 * For callers that cannot call cudaMalloc where they need a dot product: a
 * host code that hands the whole device memory to its own pool at start-up
 * (a further cudaMalloc fails or takes memory the pool counted on), or a
 * time-step loop that must not take an allocation's latency, device-wide
 * synchronisation or failure path in mid-step. Same results as pbg_dot:
 * out[0] = x.y, out[1] = sum x*y/dV/dV / n / n, written to `out` (two
 * doubles in device memory); x and y are device arrays of n doubles, on
 * `stream` (a cudaStream_t, NULL for the default stream) of the current
 * device. No session is needed and nothing is allocated: the scratch is a
 * fixed array of about 19 KB in the library's device memory, held on every
 * GPU that loads the library until the process exits; n must not exceed
 * 2^31 - 1 (larger n is rejected with PBG_ERR_ARG). Every call on a device
 * shares that array and it keeps the last call's contents; calls that
 * overlap on the GPU race and must be serialised. The first call on a
 * device looks the array up for that device (make that call before any
 * stream capture); a failed look-up is retried by the next call. */
int pbg_dot_noalloc(const double *x, const double *y, long long n, double dV, double *out,
                    void *stream);

#ifdef __cplusplus
}
#endif
#endif
