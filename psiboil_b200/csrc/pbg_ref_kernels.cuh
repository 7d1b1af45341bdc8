// Reference-parity solvers: host drivers and the kernels the C-ABI calls
// directly. See pbg_ref_kernels.cu.
#pragma once

#include <vector>

#include "pbg_common.cuh"
#include "pbg_session.h"

namespace pbg {

// Incomplete Cholesky factor (compact arrays; kind 1 = IC0, 2 = IC2, 3 =
// IC3) and the hyperplane weights h = wa i + wb j + k of its schedule.
struct IcFactor {
  double *c, *w, *s, *b, *tw, *ts, *nw;
  int kind, wa, wb;
};

struct KrylovParams {
  int prec = 0;            // Prec code: 0 diagonal, 1 IC0, 2 IC2, 3 IC3
  int mini, maxit, stalecount, hist_cap;
  double res_rat, res_tol, scale, dV;
  double *seq = nullptr;   // exact-order reduction terms (2 x ncell), null: tree
  const double *ci = nullptr;  // Jacobi / Gauss-Seidel: the matrix's stored 1/c (null: 1/c here)
};

// solver codes of the drivers below: 0 CG, 1 BiCGS, 2 CGS, 3 Jacobi,
// 4 Gauss-Seidel
struct RefKrylovWork {
  DBuf<double> r, q, pA, pB, rt, ph, v, s, sh, t, u;
  DBuf<double> mcd;                               // 1 / c (the diagonal preconditioner)
  DBuf<double> xold;                              // Gauss-Seidel: x before the sweep (periodic)
  const double *rhs = nullptr, *ci = nullptr;     // Jacobi / Gauss-Seidel operands of a solve
  DBuf<double> z, mc, mw, ms, mb, mtw, mts, mnw;  // IC preconditioner
  void ensure(size_t n, int solver);
  IcFactor ic(int kind, size_t n);
};

struct RefKrylovResult {
  int converged, status, iterations;
  double res0, res;
};

__global__ void k_spmv_ref(MatView<double> A, const double *__restrict__ x, double *__restrict__ y);
__global__ void k_resid_ref(MatView<double> A, const double *__restrict__ x,
                            const double *__restrict__ b, double *__restrict__ r);
__global__ void k_seq_sum(long long N, const double *__restrict__ a, const double *__restrict__ b,
                          double *seq, unsigned *count, double *out);
// Lays out an exact-order reduction scratch of exact_scratch_doubles(ncell)
// doubles at base (header, records, zeroed flags and counters).
void exact_scratch_init(double *base, long long ncell, cudaStream_t s);
__global__ void k_dot2(long long N, const double *__restrict__ x, const double *__restrict__ y,
                       double dV, double *part, unsigned *count, double *out);

void enqueue_ref_setup(const MatView<double> &A, double *x, const double *b, const KrylovParams &pr,
                       int solver, RefKrylovWork &w, const RedPool &red, KrylovState *st,
                       cudaStream_t s);
void enqueue_ref_iters(const MatView<double> &A, double *x, int solver, int count,
                       RefKrylovWork &w, const RedPool &red, KrylovState *st, double *hist,
                       cudaStream_t s, bool exact, int prec);
RefKrylovResult ref_krylov_solve(const MatView<double> &A, double *x, const double *b,
                                 const KrylovParams &pr, int solver, RefKrylovWork &w,
                                 const RedPool &red, KrylovState *st, KrylovState *hst,
                                 double *hist, cudaStream_t s);

struct RefACLevel {
  int nx = 0, ny = 0, nz = 0, CI = 1, CJ = 1, CK = 1;
  double dV = 0;
  Mat64 A;                 // coarse levels: general storage
  DBuf<double> phi, fnew;
  DBuf<uint8_t> aflag;
};

struct RefACParams {
  int init, loop;          // -1 none, 1 V, 2 F, 4 W, 5 flex (loop -1: "just solve")
  double toler, factor;
  int max_cyc, min_cyc, stop_if_div, priority_min_cyc;
  int mv[3], ms[3];
  double resrat_val, restol_val;
  bool use_linf = false;
  long long flex_visits = 1000000;
};

struct RefACResult {
  int converged, cycles, diverged, nhist;
  double res0, res;
  int visits;              // smoother calls of the last flex cycle
  int flex_capped;         // a flex cycle stopped at its visit bound
};

struct RefACCtx {
  cudaStream_t s;
  RefKrylovWork *w;
  RedPool *red;
  KrylovState *st;
  KrylovState *hst = nullptr;   // pinned host copy of st (flex: the smoother's converged flag)
  long long flex_visits = 1000000;
  double *dscal, *dmean, *hbuf;
  unsigned long long *dlinf;
  int mv[3], ms[3];
  double resrat_val, restol_val;
};

class RefAC {
 public:
  std::vector<RefACLevel> L;
  DBuf<double> fold;
  double *seq = nullptr;   // exact-order reduction terms, or null
  MatView<double> A0v{};
  // the smoother of every level (the Centered object's Linear): solver code
  // of the drivers above, its Prec code, and level 0's stored ci (or null)
  int sm_kind = 0, sm_prec = 0;
  const double *sm_ci0 = nullptr;
  // AC's own solver for call_solver (post-smoothing, coarsest level):
  // sol_kind -1 = the levels' smoother
  int sol_kind = -1, sol_prec = 0;
  // the level solvers' scale (dti * scale) and the dt of AC's residual measure
  double sm_scale = 1.0, res_dt = 1.0;

  void build(const MatView<double> &A0, const uint8_t *aflag0, double h, cudaStream_t s);
  MatView<double> view(int l) const;
  void coarsen_all(cudaStream_t s);
  RefACResult cycle(double *x, const double *b, const RefACParams &pa, RefACCtx &cx,
                    double *res_hist, int hist_cap);
  int nlevels() const { return (int)L.size(); }

 private:
  double residual(RedPool &red, double *dscal, unsigned long long *dlinf, double *hbuf,
                  cudaStream_t s, double *linf);
  void smooth(int l, int mi, double res_rat, double res_tol, int ms, RefKrylovWork &w,
              RedPool &red, KrylovState *st, cudaStream_t s, bool as_solver = false);
  void solve_l(int l, int mi, double res_rat, double res_tol, int ms, RefACCtx &cx);
  bool smooth_converged(int l, int mi, double res_rat, double res_tol, int ms, RefACCtx &cx);
  void restrict_to(int l, RedPool &red, double *dmean, cudaStream_t s);
  void interp_from(int l, cudaStream_t s);
  void run(int kind, int l, RefACCtx &cx);
  void v_cycle(int l, RefACCtx &cx);
  void fw_cycle(int l, RefACCtx &cx, bool w);
  void flex_cycle(int l, RefACCtx &cx);
  void full_cycle(int l, int kind, RefACCtx &cx);
  long long flex_calls_ = 0;
  bool flex_capped_ = false;
};

}  // namespace pbg
