// Reference-side binding: PSI-BOIL's Krylov solvers backed by the B200
// engine through its C ABI (psiboil_b200.h).
//
// Include after "Include/psi-boil.h" inside a PSI-BOIL build and link with
// -lpsiboil_b200 -lcudart. Then
//
//     Krylov * solver = new pbg_psiboil::GpuCG(d, Prec::di());   // was: new CG(d, Prec::di())
//     Pressure pr(p, f, uvw, time, solver, &mixed);
//     AC multigrid(&pr);                  // the reference AC now smooths on the GPU
//     multigrid.vcycle(ResRat(1e-2));
//
// keeps every call site of Linear::solve (Src/Solver/Linear/linear.h:46-56):
// Centered::solve (centered_solve.cpp:31) and AC::call_smoother /
// call_solver (additive_cycle_functions.cpp:90-107) reach the GPU without
// change. Arguments keep their meaning (MinIter, MaxIter, ResRat, ResTol,
// scale, stalecount), x is updated in place, the return value is the
// converged flag, and a non-NULL name prints the reference's log line
// (cg.cpp:175-179). The Scalar blocks are passed as they are: their
// interior starts at (si, sj, sk) of the contiguous val[0][0] block
// (global_malloc.cpp:35-56) with strides (nj*nk, nk, 1).
//
// GpuJacobi(d) and GpuGaussSeidel(d) (below) replace Jacobi(d) and
// GaussSeidel(d) (Src/Solver/Linear/Iterative) the same way.
//
// One engine session is kept per grid size (AC's coarse levels have their
// own), and the matrix is uploaded on every call because the reference
// rebuilds coarse operators in every cycle (additive_cycle_functions.cpp:25-26).
// The session's cell volume is the grid's first cell's; a stretched grid
// (spacings or volumes varying by more than 1e-10 relative) is refused with
// std::runtime_error, since the solvers' residual measure sums x*y/dV/dV
// with one dV.
//
// GpuAC (at the end) replaces AC itself: `pbg_psiboil::GpuAC multigrid(&pr);`
// for `AC multigrid(&pr);`, with AC's constructor, cycle/vcycle/fcycle/
// wcycle/fullcycle/flexcycle overloads and setters (additive.h:28-142). The
// whole cycle runs on the GPU: the hierarchy, every level's smoother and
// AC's own solver stay on the device for the call; one upload of the
// fine matrix, flags, right-hand side and guess per call.
#pragma once

#include <array>
#include <cmath>
#include <cstdio>
#include <map>
#include <stdexcept>
#include <tuple>
#include <vector>

#include "psiboil_b200.h"

namespace pbg_psiboil {

// The session's cell volume and spacing of a grid (its first cell's), or an
// error for a stretched grid. The reference's spacings come from its node
// coordinates, so a uniform grid's cells differ in their last bits; cells
// within 1e-10 relative of the first count as uniform.
inline void uniform_grid(const Scalar &x, double &h, double &dV) {
  h = x.dxc(x.si());
  dV = x.dV(x.si(), x.sj(), x.sk());
  auto same = [](double a, double b) { return std::fabs(a - b) <= 1.0e-10 * std::fabs(b); };
  for (int i = x.si(); i <= x.ei(); ++i)
    if (!same(x.dxc(i), h)) throw std::runtime_error("psiboil_b200: stretched grid (dxc varies)");
  for (int j = x.sj(); j <= x.ej(); ++j)
    if (!same(x.dyc(j), x.dyc(x.sj()))) throw std::runtime_error("psiboil_b200: stretched grid (dyc varies)");
  for (int k = x.sk(); k <= x.ek(); ++k)
    if (!same(x.dzc(k), x.dzc(x.sk()))) throw std::runtime_error("psiboil_b200: stretched grid (dzc varies)");
  for (int i = x.si(); i <= x.ei(); ++i)
    for (int j = x.sj(); j <= x.ej(); ++j)
      for (int k = x.sk(); k <= x.ek(); ++k)
        if (!same(x.dV(i, j, k), dV)) throw std::runtime_error("psiboil_b200: cell volumes vary");
}

class SessionCache {
 public:
  ~SessionCache() {
    for (auto &kv : m_) pbg_session_destroy(kv.second);
  }
  // the session of x's grid (created on first use, cell volume set); a
  // periodic axis of x (BndType::periodic on both faces) makes it periodic
  pbg_session *get(const Scalar &x) {
    const int nx = x.ei() - x.si() + 1, ny = x.ej() - x.sj() + 1, nz = x.ek() - x.sk() + 1;
    int bc[6] = {0, 0, 0, 0, 0, 0};
    const Dir dirs[6] = {Dir::imin(), Dir::imax(), Dir::jmin(), Dir::jmax(), Dir::kmin(), Dir::kmax()};
    for (int f = 0; f < 6; ++f)
      if (x.bc().type(dirs[f], BndType::periodic())) bc[f] = PBG_BC_PERIODIC_;
    for (int ax = 0; ax < 3; ++ax)
      if (bc[2 * ax] != bc[2 * ax + 1]) bc[2 * ax] = bc[2 * ax + 1] = 0;
    auto key = std::make_tuple(nx, ny, nz, bc[0] + 2 * bc[2] + 4 * bc[4]);
    auto it = m_.find(key);
    if (it != m_.end()) return it->second;
    double h, dV;
    uniform_grid(x, h, dV);
    pbg_session *s = nullptr;
    if (pbg_session_create(nx, ny, nz, h, bc, 0, &s) != PBG_OK)
      throw std::runtime_error(pbg_last_error());
    if (pbg_session_set_cell_volume(s, dV) != PBG_OK) throw std::runtime_error(pbg_last_error());
    m_[key] = s;
    return s;
  }

 private:
  std::map<std::tuple<int, int, int, int>, pbg_session *> m_;
};

inline void strides_of(const Scalar &x, long long &si, long long &sj, long long &sk,
                       long long &off) {
  si = (long long)x.nj() * x.nk();
  sj = x.nk();
  sk = 1;
  off = x.si() * si + x.sj() * sj + x.sk();
}

class GpuKrylov : public Krylov {
 public:
  GpuKrylov(const Domain &d, int solver, const Prec &pc, bool exact_sums)
      : Krylov(d, Prec::di()), solver_(solver), prec_(int(pc)), exact_(exact_sums) {}
  int solver_code() const { return solver_; }
  int prec_code() const { return prec_; }

  bool solve(Matrix &A, Scalar &x, Scalar &b, const MinIter &mini, const MaxIter &mi,
             const char *name = NULL, const ResRat &rr = ResRat(), const ResTol &rt = ResTol(),
             const real scale = 1.0, const int stalecount = -1,
             const bool precform = true) override {
    (void)precform;  // the preconditioner is formed on every call
    pbg_session *s = cache_.get(x);
    long long si, sj, sk, off;
    strides_of(x, si, sj, sk, off);
    check(pbg_matrix_upload(s, &A.c[0][0][0], &A.w[0][0][0], &A.e[0][0][0], &A.s[0][0][0],
                            &A.n[0][0][0], &A.b[0][0][0], &A.t[0][0][0], si, sj, sk, off,
                            PBG_HOST));
    pbg_params p;
    pbg_params_default(&p, solver_);
    p.min_iter = int(mini);
    p.max_iter = int(mi);
    p.res_rat = real(rr);
    p.res_tol = real(rt);
    p.scale = scale;
    p.stalecount = stalecount;
    p.exact_sums = exact_ ? 1 : 0;
    p.prec = prec_;
    pbg_result r;
    check(pbg_solve_strided(s, &x[0][0][0], &b[0][0][0], si, sj, sk, off, PBG_HOST, &p, &r));
    x.exchange();
    if (name != NULL)
      boil::oout << name << ", residual = " << r.res << ", ratio = " << r.res / r.res0
                 << ", iterations = " << r.iterations + (r.status == PBG_MAXITER ? 1 : 0)
                 << boil::endl;
    return r.converged != 0;
  }

 private:
  static void check(int rc) {
    if (rc != PBG_OK) throw std::runtime_error(pbg_last_error());
  }
  int solver_;
  int prec_;
  bool exact_;
  SessionCache cache_;
};

// CG(d, Prec::di() | ic0() | ic2() | ic3()) on the GPU (Src/Solver/Linear/Krylov/cg.h)
class GpuCG : public GpuKrylov {
 public:
  explicit GpuCG(const Domain &d, const Prec &pc = Prec::di(), bool exact_sums = false)
      : GpuKrylov(d, PBG_SOLVER_CG, pc, exact_sums) {}
};

// BiCGS(d, pc) on the GPU (Src/Solver/Linear/Krylov/bicgs.h)
class GpuBiCGS : public GpuKrylov {
 public:
  explicit GpuBiCGS(const Domain &d, const Prec &pc = Prec::di(), bool exact_sums = false)
      : GpuKrylov(d, PBG_SOLVER_BICGS, pc, exact_sums) {}
};

// CGS(d, pc) on the GPU (Src/Solver/Linear/Krylov/cgs.h)
class GpuCGS : public GpuKrylov {
 public:
  explicit GpuCGS(const Domain &d, const Prec &pc = Prec::di(), bool exact_sums = false)
      : GpuKrylov(d, PBG_SOLVER_CGS, pc, exact_sums) {}
};

// Jacobi(d) and GaussSeidel(d) on the GPU (Src/Solver/Linear/Iterative).
// Both divide by the matrix's stored A.ci, which is uploaded with the
// matrix on every call. Gauss-Seidel's lexicographic sweep runs as one
// launch per hyperplane i + j + k, which gives the sequential sweep's
// values; its log line is the reference's (gaussseidel.cpp:109-113).
// Jacobi's log prints sqrt(r.r) where the reference prints it divided by
// |A x| (jacobi.cpp:65-71).
class GpuIterative : public Iterative {
 public:
  GpuIterative(const Domain &d, int solver, bool exact_sums)
      : Iterative(d), solver_(solver), exact_(exact_sums) {}
  int solver_code() const { return solver_; }

  bool solve(Matrix &A, Scalar &x, Scalar &b, const MinIter &mini, const MaxIter &mi,
             const char *name = NULL, const ResRat &rr = ResRat(), const ResTol &rt = ResTol(),
             const real scale = 1.0, const int stalecount = -1,
             const bool precform = true) override {
    (void)precform;
    pbg_session *s = cache_.get(x);
    long long si, sj, sk, off;
    strides_of(x, si, sj, sk, off);
    check(pbg_matrix_upload(s, &A.c[0][0][0], &A.w[0][0][0], &A.e[0][0][0], &A.s[0][0][0],
                            &A.n[0][0][0], &A.b[0][0][0], &A.t[0][0][0], si, sj, sk, off,
                            PBG_HOST));
    check(pbg_ci_upload(s, &A.ci[0][0][0], si, sj, sk, off, PBG_HOST));
    pbg_params p;
    pbg_params_default(&p, solver_);
    p.min_iter = int(mini);
    p.max_iter = int(mi);
    p.res_rat = real(rr);
    p.res_tol = real(rt);
    p.scale = scale;
    p.stalecount = stalecount;
    p.exact_sums = exact_ ? 1 : 0;
    pbg_result r;
    check(pbg_solve_strided(s, &x[0][0][0], &b[0][0][0], si, sj, sk, off, PBG_HOST, &p, &r));
    x.exchange();
    if (name != NULL)
      boil::oout << name << ", residual = " << r.res << ", ratio = " << r.res / r.res0
                 << ", iterations = " << r.iterations + (r.status == PBG_MAXITER ? 1 : 0)
                 << boil::endl;
    return r.converged != 0;
  }

 private:
  static void check(int rc) {
    if (rc != PBG_OK) throw std::runtime_error(pbg_last_error());
  }
  int solver_;
  bool exact_;
  SessionCache cache_;
};

class GpuJacobi : public GpuIterative {
 public:
  explicit GpuJacobi(const Domain &d, bool exact_sums = false)
      : GpuIterative(d, PBG_SOLVER_JACOBI, exact_sums) {}
};

class GpuGaussSeidel : public GpuIterative {
 public:
  explicit GpuGaussSeidel(const Domain &d, bool exact_sums = false)
      : GpuIterative(d, PBG_SOLVER_GAUSS_SEIDEL, exact_sums) {}
};

// The PSI-BOIL solver behind a Linear*: its engine solver code and Prec
// code (the reference's classes and the Gpu* classes above).
inline void solver_code_of(Linear *l, int &code, int &prec) {
  prec = 0;
  if (auto *g = dynamic_cast<GpuKrylov *>(l)) { code = g->solver_code(); prec = g->prec_code(); return; }
  if (auto *g = dynamic_cast<GpuIterative *>(l)) { code = g->solver_code(); return; }
  if (dynamic_cast<CG *>(l)) code = PBG_SOLVER_CG;
  else if (dynamic_cast<BiCGS *>(l)) code = PBG_SOLVER_BICGS;
  else if (dynamic_cast<CGS *>(l)) code = PBG_SOLVER_CGS;
  else if (dynamic_cast<Jacobi *>(l)) code = PBG_SOLVER_JACOBI;
  else if (dynamic_cast<GaussSeidel *>(l)) code = PBG_SOLVER_GAUSS_SEIDEL;
  else throw std::runtime_error("psiboil_b200: AC with a solver that is not CG, BiCGS, CGS, Jacobi or GaussSeidel");
  if (code <= PBG_SOLVER_BICGS || code == PBG_SOLVER_CGS) {
    if (dynamic_cast<IncompleteCholesky0 *>(l->prec)) prec = 1;
    else if (dynamic_cast<IncompleteCholesky2 *>(l->prec)) prec = 2;
    else if (dynamic_cast<IncompleteCholesky3 *>(l->prec)) prec = 3;
  }
}

// Read access to the Centered members AC reads (A, phi, fnew, aflag, time),
// which are protected: member pointers formed inside a class derived from
// Centered. Nothing is constructed.
struct CenteredAccess : public Centered {
  static Matrix Centered::*A_of() { return &CenteredAccess::A; }
  static Scalar Centered::*phi_of() { return &CenteredAccess::phi; }
  static Scalar Centered::*fnew_of() { return &CenteredAccess::fnew; }
  static ScalarInt Centered::*aflag_of() { return &CenteredAccess::aflag; }
  static const Times *Equation::*time_of() { return &CenteredAccess::time; }
};

// AC (Src/Solver/Additive/additive.h:28-142) on the GPU. Same constructor,
// cycle(init, loop, ResTol, ResRat, mv, ms, &ncyc) and its overloads, and
// setters. Each cycle call, like the reference's, updates the right-hand
// side (Centered::update_rhs), rebuilds the coarse operators from the
// current matrix and runs the cycle; here every level lives on the device
// for the whole call. The levels are smoothed by the Centered object's
// Linear (CG, BiCGS, CGS with its Prec, Jacobi or GaussSeidel, or their Gpu*
// counterparts) and call_solver uses `sol` when one is given, as the
// reference's AC does. exact_sums: every global sum in the reference's
// sequential order (results bit for bit equal to the reference's).
//
// The log lines are the reference's (additive_cycle_functions.cpp:33-65)
// without the max-norm column. use_engine(precision) instead solves each
// cycle() call with the engine's flexible CG preconditioned by the AC
// K-cycle to the cycle's ResRat / ResTol (FP64 or mixed precision); ncyc
// then receives its iteration count.
class GpuAC {
 public:
  explicit GpuAC(Centered *cen, Linear *sol = NULL, bool exact_sums = false)
      : cen_(cen), exact_(exact_sums) {
    solver_code_of(cen->solver, sm_, sm_prec_);
    if (sol) solver_code_of(sol, sol_, sol_prec_);
  }

  bool cycle(const Cycle &init, const Cycle &loop, const ResTol &toler, const ResRat &factor,
             const std::array<MaxIter, 3> &mv, const std::array<MaxIter, 3> &ms, int *ncyc = NULL) {
    Matrix &A = cen_->*CenteredAccess::A_of();
    Scalar &phi = cen_->*CenteredAccess::phi_of();
    Scalar &fnew = cen_->*CenteredAccess::fnew_of();
    ScalarInt &aflag = cen_->*CenteredAccess::aflag_of();
    const Times *time = cen_->*CenteredAccess::time_of();
    cen_->update_rhs();  // init_cycles (additive_cycle_functions.cpp:15-18)
    pbg_session *s = cache_.get(phi);
    long long si, sj, sk, off;
    strides_of(phi, si, sj, sk, off);
    check(pbg_matrix_upload(s, &A.c[0][0][0], &A.w[0][0][0], &A.e[0][0][0], &A.s[0][0][0],
                            &A.n[0][0][0], &A.b[0][0][0], &A.t[0][0][0], si, sj, sk, off, PBG_HOST));
    check(pbg_active_upload(s, &aflag[0][0][0], si, sj, sk, off, PBG_HOST));
    check(pbg_ci_upload(s, &A.ci[0][0][0], si, sj, sk, off, PBG_HOST));
    pbg_params p;
    pbg_result r;
    if (engine_ >= 0) {
      pbg_params_default(&p, PBG_SOLVER_ENGINE);
      p.precision = engine_;
      p.tol = real(factor) > 0.0 ? real(factor) : 1.0e-8;
      p.max_iter = 500;
      check(pbg_solve_strided(s, &phi[0][0][0], &fnew[0][0][0], si, sj, sk, off, PBG_HOST, &p, &r));
      phi.exchange();
      boil::oout << "Engine: relative residual = " << r.relres << ", iterations = " << r.iterations
                 << boil::endl;
      if (ncyc) *ncyc = r.iterations;
      return r.converged != 0;
    }
    pbg_params_default(&p, PBG_SOLVER_AC);
    p.init_cycle = cycle_code(init);
    p.loop_cycle = cycle_code(loop);
    p.toler = real(toler);
    p.factor = real(factor);
    p.max_cycles = max_cyc_;
    p.min_cycles = min_cyc_;
    p.stop_if_div = stop_if_div_ ? 1 : 0;
    p.priority_min_cyc = prio_ ? 1 : 0;
    for (int q = 0; q < 3; ++q) { p.mv[q] = int(mv[q]); p.ms[q] = int(ms[q]); }
    p.exact_sums = exact_ ? 1 : 0;
    p.ac_smoother = sm_;
    p.prec = sm_prec_;
    p.ac_solver = sol_;
    p.ac_solver_prec = sol_prec_;
    p.ac_resrat = real(resrat_);
    p.ac_restol = real(restol_);
    p.use_linf = use_linf_ ? 1 : 0;
    p.scale = time->dti() * cen_->get_scale();
    p.ac_dt = time->dt();
    check(pbg_solve_strided(s, &phi[0][0][0], &fnew[0][0][0], si, sj, sk, off, PBG_HOST, &p, &r));
    phi.exchange();
    // the reference's log lines, from the cycle's residual history
    int nh = 0;
    check(pbg_history(s, NULL, 0, &nh));
    std::vector<double> h(nh > 0 ? nh : 1);
    check(pbg_history(s, h.data(), nh, &nh));
    if (nh > 0) boil::oout << "Initial res = " << h[0] << boil::endl;
    if (r.cycles == 0 && r.converged) {
      boil::oout << "Converged in 0 cycles!" << boil::endl;
    } else {
      const int first = p.init_cycle != PBG_CYCLE_NONE ? 0 : 1;
      for (int q = 1; q < nh; ++q) boil::oout << "Cycle " << (first + q - 1) << "; res = " << h[q] << boil::endl;
      if (r.converged)
        boil::oout << "Converged in " << r.cycles << (r.cycles > 1 ? " cycles!" : " cycle!") << boil::endl;
      else if (r.status == PBG_DIVERGED)
        boil::oout << "Failed to conv. " << r.cycles << " cycles!" << boil::endl;
    }
    if (ncyc) *ncyc = r.cycles;
    return r.converged != 0;
  }

  // additive.h:40-95
  bool vcycle(const ResTol &t, const ResRat &f, int *n = NULL) { return cycle(Cycle::none(), Cycle::V(), t, f, mv_, ms_, n); }
  bool fcycle(const ResTol &t, const ResRat &f, int *n = NULL) { return cycle(Cycle::none(), Cycle::F(), t, f, mv_, ms_, n); }
  bool wcycle(const ResTol &t, const ResRat &f, int *n = NULL) { return cycle(Cycle::none(), Cycle::W(), t, f, mv_, ms_, n); }
  bool fullcycle(const Cycle &l, const ResTol &t, const ResRat &f, int *n = NULL) { return cycle(Cycle::V(), l, t, f, mv_, ms_, n); }
  bool flexcycle(const ResTol &t, const ResRat &f, int *n = NULL) { return cycle(Cycle::none(), Cycle::flex(), t, f, mv_, ms_, n); }
  bool vcycle(const ResRat &f, int *n = NULL) { return vcycle(ResTol(-1.0), f, n); }
  bool fcycle(const ResRat &f, int *n = NULL) { return fcycle(ResTol(-1.0), f, n); }
  bool wcycle(const ResRat &f, int *n = NULL) { return wcycle(ResTol(-1.0), f, n); }
  bool fullcycle(const Cycle &l, const ResRat &f, int *n = NULL) { return fullcycle(l, ResTol(-1.0), f, n); }
  bool flexcycle(const ResRat &f, int *n = NULL) { return flexcycle(ResTol(-1.0), f, n); }
  bool vcycle(const ResTol &t, int *n = NULL) { return vcycle(t, ResRat(-1.0), n); }
  bool fcycle(const ResTol &t, int *n = NULL) { return fcycle(t, ResRat(-1.0), n); }
  bool wcycle(const ResTol &t, int *n = NULL) { return wcycle(t, ResRat(-1.0), n); }
  bool fullcycle(const Cycle &l, const ResTol &t, int *n = NULL) { return fullcycle(l, t, ResRat(-1.0), n); }
  bool flexcycle(const ResTol &t, int *n = NULL) { return flexcycle(t, ResRat(-1.0), n); }

  // setters and getters (additive.h:97-142)
  void max_cycles(const int mc) { max_cyc_ = mc; }
  int max_cycles() const { return max_cyc_; }
  void min_cycles(const int mc) { min_cyc_ = mc; }
  int min_cycles() const { return min_cyc_; }
  void restol(const ResTol &rt) { restol_ = rt; }
  ResTol restol() const { return restol_; }
  void resrat(const ResRat &rr) { resrat_ = rr; }
  ResRat resrat() const { return resrat_; }
  void stale_iter_array(const std::array<MaxIter, 3> &mn) { ms_ = mn; }
  std::array<MaxIter, 3> stale_iter_array() const { return ms_; }
  void max_iter_array(const std::array<MaxIter, 3> &mn) { mv_ = mn; }
  std::array<MaxIter, 3> max_iter_array() const { return mv_; }
  void stop_if_diverging(const bool &s) { stop_if_div_ = s; }
  bool stop_if_diverging() const { return stop_if_div_; }
  void priority_min_cycle(const bool &s) { prio_ = s; }
  bool priority_min_cycle() { return prio_; }
  void use_linf_error(const bool &s) { use_linf_ = s; }
  bool use_linf_error() const { return use_linf_; }

  // solve every cycle() call with the engine (PBG_FP64 or PBG_MIXED); -1:
  // the reference's cycles again
  void use_engine(int precision) { engine_ = precision; }

 private:
  static void check(int rc) {
    if (rc != PBG_OK) throw std::runtime_error(pbg_last_error());
  }
  static int cycle_code(const Cycle &c) {
    if (c == Cycle::V()) return PBG_CYCLE_V;
    if (c == Cycle::F()) return PBG_CYCLE_F;
    if (c == Cycle::W()) return PBG_CYCLE_W;
    if (c == Cycle::flex()) return PBG_CYCLE_FLEX;
    return PBG_CYCLE_NONE;
  }
  Centered *cen_;
  bool exact_;
  int sm_ = PBG_SOLVER_CG, sm_prec_ = 0, sol_ = -1, sol_prec_ = 0;
  int max_cyc_ = 20, min_cyc_ = 0, engine_ = -1;
  bool stop_if_div_ = true, prio_ = true, use_linf_ = false;
  ResTol restol_ = ResTol(boil::atto);
  ResRat resrat_ = ResRat(boil::atto);
  std::array<MaxIter, 3> mv_ = {MaxIter(20), MaxIter(20), MaxIter(20)};
  std::array<MaxIter, 3> ms_ = {MaxIter(-1), MaxIter(-1), MaxIter(-1)};
  SessionCache cache_;
};

}  // namespace pbg_psiboil
