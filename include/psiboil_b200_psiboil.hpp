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
#pragma once

#include <cstdio>
#include <map>
#include <stdexcept>
#include <tuple>

#include "psiboil_b200.h"

namespace pbg_psiboil {

class SessionCache {
 public:
  ~SessionCache() {
    for (auto &kv : m_) pbg_session_destroy(kv.second);
  }
  pbg_session *get(const Scalar &x) {
    const int nx = x.ei() - x.si() + 1, ny = x.ej() - x.sj() + 1, nz = x.ek() - x.sk() + 1;
    auto key = std::make_tuple(nx, ny, nz);
    auto it = m_.find(key);
    if (it != m_.end()) return it->second;
    pbg_session *s = nullptr;
    const int bc[6] = {0, 0, 0, 0, 0, 0};
    if (pbg_session_create(nx, ny, nz, x.dxc(x.si()), bc, 0, &s) != PBG_OK)
      throw std::runtime_error(pbg_last_error());
    m_[key] = s;
    return s;
  }

 private:
  std::map<std::tuple<int, int, int>, pbg_session *> m_;
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
    check(pbg_session_set_cell_volume(s, x.dV(x.si(), x.sj(), x.sk())));
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
    check(pbg_session_set_cell_volume(s, x.dV(x.si(), x.sj(), x.sk())));
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

}  // namespace pbg_psiboil
