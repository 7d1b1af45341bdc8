/*
 * Fixture harness around the UNMODIFIED PSI-BOIL reference library.
 *
 * Test infrastructure only: it is the parity checker and the timed CPU
 * baseline, never part of the product. It is linked against the reference
 * built from its own sources by oracle/build_ref.py.
 *
 * What it does, with reference code doing the solving:
 *  - builds a uniform Domain and a Pressure equation exactly as the
 *    reference's application mains do (Tests/Bubble3d/main-bubble-3d.cpp:
 *    Grid1D/Domain/Times, `new CG(d, Prec::di())`, `Pressure pr(...)`,
 *    `AC multigrid(&pr)`);
 *  - the `Fixture` subclass overrides `Pressure::discretize` with the
 *    workload's harmonic-density face coefficients and voxel solid mask
 *    (the face stage of psiboil_b200/csrc/problem_gen.h), then calls the
 *    reference's own `Centered::create_system_bnd()` for the boundary
 *    correction, sets `ci = 1/c`, scales solid cells by pico
 *    (pressure_discretize.cpp:125-148) and clears `aflag` on solid cells;
 *  - overrides `update_rhs` to load the seeded right-hand side;
 *  - runs one of:
 *      cg     `Centered::solve` -> `CG::solve` (Src/Solver/Linear/Krylov/cg.cpp)
 *      bicgs  `Centered::solve` -> `BiCGS::solve` (bicgs.cpp)
 *      ac     `AC::vcycle(ResRat)` (Src/Solver/Additive/additive_cycle.cpp)
 *    with x0 = 0 and dt = 1, and writes the matrix, rhs, solution and a
 *    text summary (iterations, cycles, residual history parsed from the
 *    reference's own log lines, wall time of the solve call alone).
 *
 * Usage:
 *   ref_harness --kind single|cyl|batch --n N [--nb NB --rmin R --rmax R
 *               --rc R --ratio Q] [--index I --n2d M --s2 LO HI --s3 LO HI]
 *               --seed S --solver cg|bicgs|cgs|jacobi|gs|ac [--acsm SOLVER] --resrat RR --maxit M
 *               [--maxcyc C --guard 0|1 --cycle V|F|W|flex|none --init none|V|F|W
 *                --mincyc C --linf 0|1 --acsolver SOLVER --acresrat RR] [--prec di|ic0|ic2|ic3] [--save NAME]
 *               [--step 1 --dt DT] [--convect F] [--periodic MASK] --out PREFIX
 *
 * --solver cgs runs `CGS::solve` (cgs.cpp), --solver jacobi `Jacobi::solve`
 * and --solver gs `GaussSeidel::solve` (Src/Solver/Linear/Iterative);
 * --convect F adds the upwind
 * convection of pbg_gen_convect to the fixture after the boundary
 * correction (a non-symmetric matrix, for BiCGS and CGS).
 *
 * With --solver ac: --cycle flex runs AC's flex cycle and --cycle none its
 * "just solve" branch (AC::cycle with Cycle::none() as the loop, through
 * AC::cycle(init, loop, ResTol(-1), ResRat, mv, ms)); --init V|F|W starts
 * with a full cycle of that kind; --linf 1 sets use_linf_error(true);
 * --acsolver names a distinct solver for AC(cen, sol); --acresrat sets
 * AC::resrat, the ResRat of the level solvers (atto by default). In the
 * engine-linked build (ref_harness_gpu), --gpu 1 swaps the Pressure's solver
 * for the drop-in Gpu* class and --gpu 2 also swaps AC for GpuAC.
 *
 * --periodic MASK makes the axes of MASK (bit 0 i, 1 j, 2 k) periodic: the
 * grids are built with Periodic::yes(), the pressure (and velocity) get
 * BndType::periodic() on both faces, and the fixture's boundary faces on
 * those axes couple to the cell at the other end.
 *
 * --step 1 runs one pressure-correction step with the reference's own
 * classes and no override: a two-phase Matter (liquid and vapour densities
 * of the workload mixed by the colour function of pbg_gen_flow,
 * matter.cpp:78 -> PropertyMix), `Pressure pr(...)` whose constructor runs
 * Pressure::discretize, `pr.solve(...)` (Pressure::update_rhs from the
 * predicted velocity u*, then the Krylov solver with scale dti), and
 * `Momentum::project(p)` (momentum_project.cpp:11-80). It writes the
 * matrix, the right-hand side, the pressure and the projected faces
 * (PREFIX.u/.v/.w, the layouts of pbg_gen_flow).
 */
#include "Include/psi-boil.h"
#include "problem_gen.h"
#ifdef PBG_WITH_ENGINE
#include "psiboil_b200_psiboil.hpp"
#endif

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace {

struct Args {
  std::string kind = "single", solver = "cg", out = "ref", cycle = "V", save, prec = "di", acsm = "cg";
  int n = 16, nb = 0, index = 0, n2d = 0, s2lo = 64, s2hi = 512, s3lo = 32, s3hi = 96;
  double rmin = 4, rmax = 16, rc = 0, ratio = 1000;
  unsigned long long seed = 1;
  double resrat = 1e-8;
  int maxit = 20000, maxcyc = 20, guard = 1, dump = 1, repeat = 1, gpu = 0, exact = 1;
  int step = 0;
  double dt = 1.0, convect = 0.0, body = 0.0;
  int periodic = 0;   // periodic axes: bit 0 i, 1 j, 2 k
  std::string init = "none", acsolver;  // AC: full-cycle init, distinct solver
  int linf = 0, mincyc = 0;
  double acresrat = -1.0;   // AC::resrat (the level solvers' ResRat), default atto
};

Args parse(int argc, char **argv) {
  Args a;
  for (int q = 1; q < argc; ++q) {
    std::string k = argv[q];
    auto nxt = [&]() -> const char * {
      if (q + 1 >= argc) { std::fprintf(stderr, "missing value for %s\n", k.c_str()); std::exit(2); }
      return argv[++q];
    };
    if (k == "--kind") a.kind = nxt();
    else if (k == "--n") a.n = std::atoi(nxt());
    else if (k == "--nb") a.nb = std::atoi(nxt());
    else if (k == "--rmin") a.rmin = std::atof(nxt());
    else if (k == "--rmax") a.rmax = std::atof(nxt());
    else if (k == "--rc") a.rc = std::atof(nxt());
    else if (k == "--ratio") a.ratio = std::atof(nxt());
    else if (k == "--index") a.index = std::atoi(nxt());
    else if (k == "--n2d") a.n2d = std::atoi(nxt());
    else if (k == "--s2") { a.s2lo = std::atoi(nxt()); a.s2hi = std::atoi(nxt()); }
    else if (k == "--s3") { a.s3lo = std::atoi(nxt()); a.s3hi = std::atoi(nxt()); }
    else if (k == "--seed") a.seed = std::strtoull(nxt(), nullptr, 10);
    else if (k == "--solver") a.solver = nxt();
    else if (k == "--body") a.body = std::atof(nxt());
    else if (k == "--acsm") a.acsm = nxt();
    else if (k == "--resrat") a.resrat = std::atof(nxt());
    else if (k == "--maxit") a.maxit = std::atoi(nxt());
    else if (k == "--maxcyc") a.maxcyc = std::atoi(nxt());
    else if (k == "--guard") a.guard = std::atoi(nxt());
    else if (k == "--cycle") a.cycle = nxt();
    else if (k == "--dump") a.dump = std::atoi(nxt());
    else if (k == "--repeat") a.repeat = std::atoi(nxt());
    else if (k == "--gpu") a.gpu = std::atoi(nxt());
    else if (k == "--exact") a.exact = std::atoi(nxt());
    else if (k == "--out") a.out = nxt();
    else if (k == "--save") a.save = nxt();
    else if (k == "--prec") a.prec = nxt();
    else if (k == "--step") a.step = std::atoi(nxt());
    else if (k == "--dt") a.dt = std::atof(nxt());
    else if (k == "--convect") a.convect = std::atof(nxt());
    else if (k == "--periodic") a.periodic = std::atoi(nxt());
    else if (k == "--init") a.init = nxt();
    else if (k == "--acsolver") a.acsolver = nxt();
    else if (k == "--linf") a.linf = std::atoi(nxt());
    else if (k == "--mincyc") a.mincyc = std::atoi(nxt());
    else if (k == "--acresrat") a.acresrat = std::atof(nxt());
    else { std::fprintf(stderr, "unknown argument %s\n", k.c_str()); std::exit(2); }
  }
  return a;
}

/* Pressure equation whose matrix and rhs come from the seeded fixture. */
class Fixture : public Pressure {
 public:
  Fixture(const Scalar &p, const Scalar &f, const Vector &u, Times &t,
          Linear *sm, Matter *m, const pbg_problem_desc &d,
          const std::vector<double> &rho, const std::vector<uint8_t> &solid,
          const std::vector<double> &rhs, double convect)
      : Pressure(p, f, u, t, sm, m), D(d), RHO(rho), SOLID(solid), RHS(rhs), CONV(convect) {
    ready = true;
    discretize();
    for (int i = 0; i < D.nx; ++i)
      for (int j = 0; j < D.ny; ++j)
        for (int k = 0; k < D.nz; ++k)
          aflag[i + boil::BW][j + boil::BW][k + boil::BW] = SOLID[at(i, j, k)] ? 0 : 1;
  }

  size_t at(int i, int j, int k) const { return ((size_t)i * D.ny + j) * D.nz + k; }

  void discretize(const Scalar *diff_eddy = NULL) override {
    if (!ready) { Pressure::discretize(diff_eddy); return; }
    const size_t N = pbg_ncells(&D);
    std::vector<double> c(N), w(N), e(N), s(N), n(N), b(N), t(N);
    pbg_gen_faces_per(D.nx, D.ny, D.nz, D.h, pbg_periodic_mask(D.bc), RHO.data(), SOLID.data(),
                      c.data(), w.data(), e.data(), s.data(), n.data(), b.data(), t.data());
    const int B = boil::BW;
    for (int i = 0; i < D.nx; ++i)
      for (int j = 0; j < D.ny; ++j)
        for (int k = 0; k < D.nz; ++k) {
          size_t p = at(i, j, k);
          A.c[i + B][j + B][k + B] = c[p];
          A.w[i + B][j + B][k + B] = w[p]; A.e[i + B][j + B][k + B] = e[p];
          A.s[i + B][j + B][k + B] = s[p]; A.n[i + B][j + B][k + B] = n[p];
          A.b[i + B][j + B][k + B] = b[p]; A.t[i + B][j + B][k + B] = t[p];
        }
    /* the reference's own boundary correction */
    Centered::create_system_bnd();
    /* non-symmetric variant: upwind convection along +x (pbg_gen_convect) */
    if (CONV != 0.0)
      for (int i = 1; i < D.nx; ++i)
        for (int j = 0; j < D.ny; ++j)
          for (int k = 0; k < D.nz; ++k) {
            if (SOLID[at(i, j, k)] || SOLID[at(i - 1, j, k)]) continue;
            A.w[i + B][j + B][k + B] += CONV;
            A.c[i + B][j + B][k + B] += CONV;
          }
    for (int i = 0; i < D.nx; ++i)
      for (int j = 0; j < D.ny; ++j)
        for (int k = 0; k < D.nz; ++k) {
          A.ci[i + B][j + B][k + B] = 1.0 / A.c[i + B][j + B][k + B];
          if (SOLID[at(i, j, k)]) {
            A.c[i + B][j + B][k + B] *= boil::pico;
            A.w[i + B][j + B][k + B] = 0.0; A.e[i + B][j + B][k + B] = 0.0;
            A.s[i + B][j + B][k + B] = 0.0; A.n[i + B][j + B][k + B] = 0.0;
            A.b[i + B][j + B][k + B] = 0.0; A.t[i + B][j + B][k + B] = 0.0;
          }
        }
  }

  real update_rhs() override {
    const int B = boil::BW;
    for (int i = 0; i < D.nx; ++i)
      for (int j = 0; j < D.ny; ++j)
        for (int k = 0; k < D.nz; ++k)
          fnew[i + B][j + B][k + B] = RHS[at(i, j, k)];
    return 0.0;
  }

  /* interior dump of one reference array into the engine's layout */
  void dump(const Scalar &s, std::vector<double> &out) const {
    const int B = boil::BW;
    out.resize(pbg_ncells(&D));
    for (int i = 0; i < D.nx; ++i)
      for (int j = 0; j < D.ny; ++j)
        for (int k = 0; k < D.nz; ++k)
          out[at(i, j, k)] = s[i + B][j + B][k + B];
  }
  void dump_matrix(std::ofstream &f) const {
    std::vector<double> v;
    const Scalar *arr[8] = {&A.c, &A.w, &A.e, &A.s, &A.n, &A.b, &A.t, &A.ci};
    for (auto *s : arr) { dump(*s, v); f.write((const char *)v.data(), v.size() * sizeof(double)); }
  }
  void dump_phi(std::vector<double> &v) const { dump(phi, v); }
  void dump_fnew(std::vector<double> &v) const { dump(fnew, v); }

 private:
  pbg_problem_desc D;
  std::vector<double> RHO;
  std::vector<uint8_t> SOLID;
  std::vector<double> RHS;
  double CONV = 0.0;
  bool ready = false;
};

/* The reference's own Pressure (no override), with read access to the
 * matrix and the right-hand side it assembled. */
class Probe : public Pressure {
 public:
  Probe(const Scalar &p, const Scalar &f, const Vector &u, Times &t, Linear *sm, Matter *m)
      : Pressure(p, f, u, t, sm, m) {}
  void dump_matrix(const pbg_problem_desc &D, std::ofstream &f) const {
    const Scalar *arr[8] = {&A.c, &A.w, &A.e, &A.s, &A.n, &A.b, &A.t, &A.ci};
    for (auto *s : arr) dump_cells(*s, D, f);
  }
  void dump_rhs(const pbg_problem_desc &D, std::ofstream &f) const { dump_cells(fnew, D, f); }
  /* the immersed body as the pressure equation sees it: fV of every cell,
   * the six face fractions fSw..fSt(i,j,k) of every cell (the accessors'
   * values, planes w e s n b t), and 1.0 for the cells of the cut-cell list
   * (Body::ijk(cc), cc < nccells()) */
  void dump_body(const pbg_problem_desc &D, std::ofstream &f) const {
    const int B = boil::BW;
    const size_t N = pbg_ncells(&D);
    std::vector<double> out(8 * N, 0.0);
    const Body &bd = dom->ibody();
    auto at = [&](int i, int j, int k) { return ((size_t)i * D.ny + j) * D.nz + k; };
    for (int i = 0; i < D.nx; ++i)
      for (int j = 0; j < D.ny; ++j)
        for (int k = 0; k < D.nz; ++k) {
          const int I = i + B, J = j + B, K = k + B;
          const size_t p = at(i, j, k);
          out[p] = bd.fV(I, J, K);
          out[1 * N + p] = bd.fSw(I, J, K); out[2 * N + p] = bd.fSe(I, J, K);
          out[3 * N + p] = bd.fSs(I, J, K); out[4 * N + p] = bd.fSn(I, J, K);
          out[5 * N + p] = bd.fSb(I, J, K); out[6 * N + p] = bd.fSt(I, J, K);
        }
    for (int cc = 0; cc < bd.nccells(); ++cc) {
      int i, j, k;
      bd.ijk(cc, &i, &j, &k);
      if (i >= B && i < D.nx + B && j >= B && j < D.ny + B && k >= B && k < D.nz + B)
        out[7 * N + at(i - B, j - B, k - B)] = 1.0;
    }
    f.write((const char *)out.data(), out.size() * sizeof(double));
  }

  static void dump_cells(const Scalar &s, const pbg_problem_desc &D, std::ofstream &f) {
    const int B = boil::BW;
    std::vector<double> out(pbg_ncells(&D));
    for (int i = 0; i < D.nx; ++i)
      for (int j = 0; j < D.ny; ++j)
        for (int k = 0; k < D.nz; ++k) out[((size_t)i * D.ny + j) * D.nz + k] = s[i + B][j + B][k + B];
    f.write((const char *)out.data(), out.size() * sizeof(double));
  }
};

/* A closed sphere as an ASCII STL: latitude/longitude quads split in two
 * triangles, vertices counter-clockwise seen from outside (the pole rows
 * give one triangle each). */
void write_sphere_stl(const std::string &path, double cx, double cy, double cz, double r) {
  const int nt = 24, np = 48;
  const double pi = 3.14159265358979323846;
  auto pt = [&](int it, int ip, double *v) {
    const double th = pi * it / nt, ph = 2.0 * pi * ip / np;
    v[0] = cx + r * std::sin(th) * std::cos(ph);
    v[1] = cy + r * std::sin(th) * std::sin(ph);
    v[2] = cz + r * std::cos(th);
  };
  std::ofstream f(path);
  f.precision(17);
  f << "solid sphere\n";
  auto tri = [&](const double *a, const double *b, const double *c) {
    double u[3], w[3], n[3];
    for (int q = 0; q < 3; ++q) { u[q] = b[q] - a[q]; w[q] = c[q] - a[q]; }
    n[0] = u[1] * w[2] - u[2] * w[1];
    n[1] = u[2] * w[0] - u[0] * w[2];
    n[2] = u[0] * w[1] - u[1] * w[0];
    const double l = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    f << " facet normal " << n[0] / l << " " << n[1] / l << " " << n[2] / l << "\n  outer loop\n";
    f << "   vertex " << a[0] << " " << a[1] << " " << a[2] << "\n";
    f << "   vertex " << b[0] << " " << b[1] << " " << b[2] << "\n";
    f << "   vertex " << c[0] << " " << c[1] << " " << c[2] << "\n";
    f << "  endloop\n endfacet\n";
  };
  for (int it = 0; it < nt; ++it)
    for (int ip = 0; ip < np; ++ip) {
      double a[3], b[3], c[3], d[3];
      pt(it, ip, a); pt(it + 1, ip, b); pt(it + 1, ip + 1, c); pt(it, ip + 1, d);
      if (it > 0) tri(a, b, d);        /* (t0,p0) (t1,p0) (t0,p1) */
      if (it < nt - 1) tri(d, b, c);   /* (t0,p1) (t1,p0) (t1,p1) */
    }
  f << "endsolid sphere\n";
}

/* Face extents of one component in the layouts of pbg_gen_flow. */
void face_dims(const pbg_problem_desc &D, int m, int &ex, int &ey, int &ez) {
  ex = D.nx + (m == 0);
  ey = D.ny + (m == 1);
  ez = D.nz + (m == 2);
}

void put_faces(Vector &uvw, int m, const pbg_problem_desc &D, const std::vector<double> &src) {
  const Comp comps[3] = {Comp::u(), Comp::v(), Comp::w()};
  const int B = boil::BW;
  int ex, ey, ez;
  face_dims(D, m, ex, ey, ez);
  for (int i = 0; i < ex; ++i)
    for (int j = 0; j < ey; ++j)
      for (int k = 0; k < ez; ++k) uvw[comps[m]][i + B][j + B][k + B] = src[((size_t)i * ey + j) * ez + k];
}

void write_faces(const Vector &uvw, int m, const pbg_problem_desc &D, const std::string &path) {
  const Comp comps[3] = {Comp::u(), Comp::v(), Comp::w()};
  const int B = boil::BW;
  int ex, ey, ez;
  face_dims(D, m, ex, ey, ez);
  std::vector<double> out((size_t)ex * ey * ez);
  for (int i = 0; i < ex; ++i)
    for (int j = 0; j < ey; ++j)
      for (int k = 0; k < ez; ++k) out[((size_t)i * ey + j) * ez + k] = uvw[comps[m]][i + B][j + B][k + B];
  std::ofstream f(path, std::ios::binary);
  f.write((const char *)out.data(), out.size() * sizeof(double));
}

/* --step 1: one pressure-correction step through the reference's classes. */
int run_step(const Args &a, const pbg_problem_desc &D) {
  const size_t N = pbg_ncells(&D);
  std::vector<double> col(N), fu(pbg_nfaces(&D, 0)), fv(pbg_nfaces(&D, 1)), fw(pbg_nfaces(&D, 2));
  pbg_gen_flow(&D, 0, col.data(), fu.data(), fv.data(), fw.data());

  std::ostringstream log;
  std::streambuf *saved = std::cout.rdbuf(log.rdbuf());
  std::cout.precision(17);

  const double h = D.h;
  auto pd = [&](int ax) { return (a.periodic & (1 << ax)) ? Periodic::yes() : Periodic::no(); };
  Grid1D gx(Range<real>(0.0, D.nx * h), Range<real>(h, h), D.nx, pd(0));
  Grid1D gy(Range<real>(0.0, D.ny * h), Range<real>(h, h), D.ny, pd(1));
  Grid1D *gz = (D.nz > 1) ? new Grid1D(Range<real>(0.0, D.nz * h), Range<real>(h, h), D.nz, pd(2))
                          : new Grid1D(h);
  /* --body R: a sphere of radius R cells inside the domain, written as an
   * ASCII STL and cut by the reference's own Body (Body::Body(name),
   * Domain(gx, gy, gz, &body)) */
  Body *body = nullptr;
  if (a.body > 0.0) {
    const std::string stl = a.out + ".stl";
    write_sphere_stl(stl, 0.5 * D.nx * h + 0.37 * h, 0.5 * D.ny * h + 0.21 * h,
                     0.5 * D.nz * h + 0.13 * h, a.body * h);
    body = new Body(stl);
  }
  Domain *dp = body ? new Domain(gx, gy, *gz, body) : new Domain(gx, gy, *gz);
  Domain &d = *dp;
  Times time(1, a.dt);
  const Prec pc = a.prec == "ic0" ? Prec::ic0() : a.prec == "ic2" ? Prec::ic2()
                 : a.prec == "ic3" ? Prec::ic3() : Prec::di();
  Linear *solver = nullptr;
  if (a.solver == "bicgs") solver = new BiCGS(d, pc);
  else solver = new CG(d, pc);

  const Dir dirs[6] = {Dir::imin(), Dir::imax(), Dir::jmin(), Dir::jmax(), Dir::kmin(), Dir::kmax()};
  Scalar p(d), f(d), c(d);
  for (int q = 0; q < 6; ++q) {
    const bool pseudo = D.nz == 1 && q >= 4;
    if (pseudo) p.bc().add(BndCnd(dirs[q], BndType::pseudo()));
    else if (D.bc[q] == PBG_BC_DIRICHLET) p.bc().add(BndCnd(dirs[q], BndType::dirichlet(), 0.0));
    else p.bc().add(BndCnd(dirs[q], BndType::neumann()));
    c.bc().add(BndCnd(dirs[q], pseudo ? BndType::pseudo() : BndType::neumann()));
  }
  Vector uvw(d), xyz(d);
  const Comp comps[3] = {Comp::u(), Comp::v(), Comp::w()};
  for (int m = 0; m < 3; ++m)
    for (int q = 0; q < 6; ++q) {
      const BndType t = (D.nz == 1 && q >= 4) ? BndType::pseudo() : BndType::wall();
      uvw.bc(comps[m]).add(BndCnd(dirs[q], t));
      xyz.bc(comps[m]).add(BndCnd(dirs[q], t));
    }
  const int B = boil::BW;
  for (int i = 0; i < D.nx; ++i)
    for (int j = 0; j < D.ny; ++j)
      for (int k = 0; k < D.nz; ++k) c[i + B][j + B][k + B] = col[((size_t)i * D.ny + j) * D.nz + k];
  c.bnd_update();
  c.exchange_all();
  put_faces(uvw, 0, D, fu);
  put_faces(uvw, 1, D, fv);
  put_faces(uvw, 2, D, fw);

  Matter liquid(d), vapour(d);
  liquid.rho(D.rho_liquid);
  vapour.rho(D.rho_vapour);
  Matter mix(liquid, vapour, &c);

  Probe pr(p, f, uvw, time, solver, &mix);
  p = 0.0;
  auto t0 = std::chrono::steady_clock::now();
  pr.solve(ResTol(boil::atto), ResRat(a.resrat), "refsolve", a.maxit);
  Momentum ns(uvw, xyz, time, solver, &mix);
  ns.project(p);
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  std::cout.rdbuf(saved);

  int iters = -1;
  double res_final = -1, ratio_final = -1;
  std::istringstream in(log.str());
  std::string line;
  while (std::getline(in, line)) {
    size_t q;
    if ((q = line.find("refsolve, residual = ")) != std::string::npos)
      std::sscanf(line.c_str() + q, "refsolve, residual = %lf, ratio = %lf, iterations = %d", &res_final,
                  &ratio_final, &iters);
  }
  {
    std::ofstream fa(a.out + ".A", std::ios::binary);
    pr.dump_matrix(D, fa);
    if (body) {
      std::ofstream fbd(a.out + ".body", std::ios::binary);
      pr.dump_body(D, fbd);
    }
    std::ofstream fb(a.out + ".b", std::ios::binary);
    pr.dump_rhs(D, fb);
    std::ofstream fx(a.out + ".x", std::ios::binary);
    Probe::dump_cells(p, D, fx);
  }
  write_faces(uvw, 0, D, a.out + ".u");
  write_faces(uvw, 1, D, a.out + ".v");
  write_faces(uvw, 2, D, a.out + ".w");
  std::ofstream fm(a.out + ".txt");
  fm.precision(17);
  fm << "nx " << D.nx << "\nny " << D.ny << "\nnz " << D.nz << "\n";
  fm << "solver " << a.solver << "\niterations " << iters << "\nresidual " << res_final
     << "\nratio " << ratio_final << "\nseconds " << secs << "\n";
  std::printf("{\"step\": 1, \"solver\": \"%s\", \"iterations\": %d, \"ratio\": %.17g, "
              "\"seconds\": %.6f, \"cells\": %zu}\n", a.solver.c_str(), iters, ratio_final, secs, N);
  return 0;
}

/* The AC run of --solver ac with the harness's settings, for the
 * reference's AC and for the drop-in GpuAC alike. */
template <typename ACT>
bool run_ac(ACT &mg, const Args &a, int *ncyc) {
  mg.max_cycles(a.maxcyc);
  mg.min_cycles(a.mincyc);
  mg.stop_if_diverging(a.guard != 0);
  mg.use_linf_error(a.linf != 0);
  if (a.acresrat > 0.0) mg.resrat(ResRat(a.acresrat));
  struct C {
    static Cycle of(const std::string &c) {
      return c == "V" ? Cycle::V() : c == "F" ? Cycle::F() : c == "W" ? Cycle::W()
             : c == "flex" ? Cycle::flex() : Cycle::none();
    }
  };
  const std::array<MaxIter, 3> mv = {{MaxIter(20), MaxIter(20), MaxIter(20)}};
  const std::array<MaxIter, 3> ms = {{MaxIter(-1), MaxIter(-1), MaxIter(-1)}};
  if (a.init != "none" || a.cycle == "flex" || a.cycle == "none")
    return mg.cycle(C::of(a.init), C::of(a.cycle), ResTol(-1.0), ResRat(a.resrat), mv, ms, ncyc);
  if (a.cycle == "F") return mg.fcycle(ResRat(a.resrat), ncyc);
  if (a.cycle == "W") return mg.wcycle(ResRat(a.resrat), ncyc);
  return mg.vcycle(ResRat(a.resrat), ncyc);
}

pbg_problem_desc make_desc(const Args &a) {
  pbg_problem_desc d;
  if (a.kind == "single") pbg_desc_single_bubble(&d, a.n, a.seed);
  else if (a.kind == "cyl") pbg_desc_bubbles_cylinder(&d, a.n, a.nb, a.rmin, a.rmax, a.rc, a.ratio, a.seed);
  else if (a.kind == "batch") pbg_desc_batch_member(&d, a.seed, a.index, a.n2d, a.s2lo, a.s2hi, a.s3lo, a.s3hi);
  else { std::fprintf(stderr, "unknown kind\n"); std::exit(2); }
  return d;
}

}  // namespace

int main(int argc, char **argv) {
  Args a = parse(argc, argv);
  pbg_problem_desc D = make_desc(a);
  for (int ax = 0; ax < 3; ++ax)
    if (a.periodic & (1 << ax)) D.bc[2 * ax] = D.bc[2 * ax + 1] = PBG_BC_PERIODIC;
  if (a.step && a.periodic) { std::fprintf(stderr, "--step takes walls only\n"); return 2; }
  if (a.step) return run_step(a, D);
  const size_t N = pbg_ncells(&D);
  std::vector<double> rho(N), rhs(N);
  std::vector<uint8_t> solid(N);
  pbg_gen_fields(&D, rho.data(), solid.data());
  pbg_gen_rhs(&D, 0, solid.data(), rhs.data());

  std::ostringstream log;
  std::streambuf *saved = std::cout.rdbuf(log.rdbuf());
  std::cout.precision(17);

  const double h = D.h;
  auto pd = [&](int ax) { return (a.periodic & (1 << ax)) ? Periodic::yes() : Periodic::no(); };
  Grid1D gx(Range<real>(0.0, D.nx * h), Range<real>(h, h), D.nx, pd(0));
  Grid1D gy(Range<real>(0.0, D.ny * h), Range<real>(h, h), D.ny, pd(1));
  Grid1D *gz = (D.nz > 1) ? new Grid1D(Range<real>(0.0, D.nz * h), Range<real>(h, h), D.nz, pd(2))
                          : new Grid1D(h);
  Domain d(gx, gy, *gz);
  Times time(1, 1.0);

  Linear *solver = nullptr;
  const Prec pc = a.prec == "ic0" ? Prec::ic0() : a.prec == "ic2" ? Prec::ic2()
                 : a.prec == "ic3" ? Prec::ic3() : Prec::di();
  /* with --solver ac, --acsm names the Pressure's own solver, which AC uses
     on every level (additive_cycle_functions.cpp:90-107) */
  const std::string lin = a.solver == "ac" ? a.acsm : a.solver;
#ifdef PBG_WITH_ENGINE
  /* the drop-in: the engine's Krylov classes behind the reference's virtual */
  if (a.gpu && lin == "bicgs") solver = new pbg_psiboil::GpuBiCGS(d, pc, a.exact != 0);
  else if (a.gpu && lin == "cgs") solver = new pbg_psiboil::GpuCGS(d, pc, a.exact != 0);
  else if (a.gpu && lin == "jacobi") solver = new pbg_psiboil::GpuJacobi(d, a.exact != 0);
  else if (a.gpu && lin == "gs") solver = new pbg_psiboil::GpuGaussSeidel(d, a.exact != 0);
  else if (a.gpu) solver = new pbg_psiboil::GpuCG(d, pc, a.exact != 0);
  else
#endif
  if (lin == "bicgs") solver = new BiCGS(d, pc);
  else if (lin == "cgs") solver = new CGS(d, pc);
  else if (lin == "jacobi") solver = new Jacobi(d);
  else if (lin == "gs") solver = new GaussSeidel(d);
  else solver = new CG(d, pc);

  Vector uvw(d);
  Scalar p(d), f(d);
  const Dir dirs[6] = {Dir::imin(), Dir::imax(), Dir::jmin(), Dir::jmax(), Dir::kmin(), Dir::kmax()};
  for (int q = 0; q < 6; ++q) {
    if (D.nz == 1 && q >= 4) p.bc().add(BndCnd(dirs[q], BndType::pseudo()));
    else if (D.bc[q] == PBG_BC_PERIODIC) p.bc().add(BndCnd(dirs[q], BndType::periodic()));
    else if (D.bc[q] == PBG_BC_DIRICHLET) p.bc().add(BndCnd(dirs[q], BndType::dirichlet(), 0.0));
    else p.bc().add(BndCnd(dirs[q], BndType::neumann()));
  }
  const Comp comps[3] = {Comp::u(), Comp::v(), Comp::w()};
  for (int m = 0; m < 3; ++m)
    for (int q = 0; q < 6; ++q) {
      if (D.nz == 1 && q >= 4) uvw.bc(comps[m]).add(BndCnd(dirs[q], BndType::pseudo()));
      else if (D.bc[q] == PBG_BC_PERIODIC) uvw.bc(comps[m]).add(BndCnd(dirs[q], BndType::periodic()));
      else uvw.bc(comps[m]).add(BndCnd(dirs[q], BndType::wall()));
    }
  Matter fluid(d);
  fluid.rho(1.0);

  Fixture pr(p, f, uvw, time, solver, &fluid, D, rho, solid, rhs, a.convect);

  p = 0.0;
  bool conv = false;
  int ncyc = -1;
  double secs = 0.0;
  std::vector<double> rep_secs;
  if (a.solver == "ac") {
    /* --acsolver: AC's own solver (AC(cen, sol), additive.cpp:8-48), used by
       call_solver (post-smoothing, coarsest level); the levels keep the
       Pressure's solver for call_smoother */
    Linear *acsol = nullptr;
    if (a.acsolver == "cg") acsol = new CG(d, pc);
    else if (a.acsolver == "bicgs") acsol = new BiCGS(d, pc);
    else if (a.acsolver == "cgs") acsol = new CGS(d, pc);
    else if (a.acsolver == "jacobi") acsol = new Jacobi(d);
    else if (a.acsolver == "gs") acsol = new GaussSeidel(d);
    p = 0.0;
    auto t0 = std::chrono::steady_clock::now();
#ifdef PBG_WITH_ENGINE
    /* --gpu 2: the reference's AC replaced by the engine's GpuAC */
    if (a.gpu == 2) {
      pbg_psiboil::GpuAC mg(&pr, acsol, a.exact != 0);
      conv = run_ac(mg, a, &ncyc);
    } else
#endif
    {
      AC mg(&pr, acsol);
      conv = run_ac(mg, a, &ncyc);
    }
    secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  } else {
    /* `repeat` timed solves from x0 = 0 (the first one's log is parsed) */
    for (int rep = 0; rep < a.repeat; ++rep) {
      p = 0.0;
      auto t0 = std::chrono::steady_clock::now();
      pr.solve(ResTol(boil::atto), ResRat(a.resrat), rep == 0 ? "refsolve" : NULL, a.maxit);
      double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      rep_secs.push_back(dt);
      if (rep == 0) secs = dt;
    }
  }
  /* the reference's own checkpoint of the result (phi, cold) */
  if (!a.save.empty()) pr.save(a.save.c_str(), 0);
  std::cout.rdbuf(saved);

  /* parse the reference's own log lines */
  int iters = -1;
  double res_final = -1, ratio_final = -1;
  std::vector<double> cycle_res;
  double res0_ac = -1;
  std::istringstream in(log.str());
  std::string line;
  while (std::getline(in, line)) {
    size_t q;
    if ((q = line.find("refsolve, residual = ")) != std::string::npos) {
      std::sscanf(line.c_str() + q, "refsolve, residual = %lf, ratio = %lf, iterations = %d",
                  &res_final, &ratio_final, &iters);
    } else if (line.rfind("Initial res = ", 0) == 0) {
      std::sscanf(line.c_str(), "Initial res = %lf", &res0_ac);
    } else if (line.rfind("Cycle ", 0) == 0) {
      int c;
      double r;
      if (std::sscanf(line.c_str(), "Cycle %d; res = %lf", &c, &r) == 2) cycle_res.push_back(r);
    }
  }
  if (a.solver != "ac") conv = (ratio_final >= 0 && ratio_final < a.resrat);

  if (a.dump) {
    std::ofstream fa(a.out + ".A", std::ios::binary);
    pr.dump_matrix(fa);
    std::vector<double> v;
    pr.dump_fnew(v);
    std::ofstream fb(a.out + ".b", std::ios::binary);
    fb.write((const char *)v.data(), v.size() * sizeof(double));
    pr.dump_phi(v);
    std::ofstream fx(a.out + ".x", std::ios::binary);
    fx.write((const char *)v.data(), v.size() * sizeof(double));
  }
  std::ofstream fm(a.out + ".txt");
  fm.precision(17);
  fm << "nx " << D.nx << "\nny " << D.ny << "\nnz " << D.nz << "\n";
  fm << "solver " << a.solver << "\nconverged " << (conv ? 1 : 0) << "\n";
  fm << "iterations " << iters << "\nresidual " << res_final << "\nratio " << ratio_final << "\n";
  fm << "cycles " << ncyc << "\nres0 " << res0_ac << "\n";
  fm << "cycle_res";
  for (double r : cycle_res) fm << " " << r;
  fm << "\nseconds " << secs << "\n";
  fm << "repeat_seconds";
  for (double r : rep_secs) fm << " " << r;
  fm << "\n";
  fm.close();
  std::printf("{\"solver\": \"%s\", \"converged\": %d, \"iterations\": %d, \"cycles\": %d, "
              "\"ratio\": %.17g, \"seconds\": %.6f, \"cells\": %zu, \"repeat_seconds\": [",
              a.solver.c_str(), conv ? 1 : 0, iters, ncyc, ratio_final, secs, N);
  for (size_t q = 0; q < rep_secs.size(); ++q) std::printf("%s%.6f", q ? ", " : "", rep_secs[q]);
  std::printf("]}\n");
  return 0;
}
