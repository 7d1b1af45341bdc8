// Pressure-matrix assembly of one cell (shared by the session and batch
// paths): the fixture discretisation of the reference harness, bit-identical
// to pbg_gen_assemble (problem_gen.h, which cites the reference lines each
// step follows): harmonic face density, faces between solid and fluid cells
// cut, Neumann sides folded into the diagonal before Dirichlet sides are
// dropped, solid cells scaled by 1e-12 with no couplings
// (Src/Equation/Centered/Pressure/pressure_discretize.cpp:24-148,
// Src/Equation/Centered/centered_system_bnd.cpp:17-62,143-185).
#pragma once
#include <cstdint>

#include "../../include/psiboil_b200.h"
#include "pbg_common.cuh"
#include "problem_gen.h"

namespace pbg {

__device__ __forceinline__ double harm_d(double a, double b) {
  return __ddiv_rn(__dmul_rn(__dmul_rn(a, b), 2.0), __dadd_rn(a, b));
}

// Writes the symmetric storage of cell p at position q: c (diagonal) and
// the w, s, b couplings to the previous cell in i, j, k.
__device__ __forceinline__ void assemble_cell(int nx, int ny, int nz, double h, const int (&bc)[6],
                                              const double *__restrict__ rho,
                                              const uint8_t *__restrict__ solid, long long p, Pos q,
                                              double &C, double &W, double &S, double &B) {
  const long long SI = (long long)ny * nz, SJ = nz;
  const double hx = __ddiv_rn(__dmul_rn(h, h), h);
  const double rp = rho[p];
  const uint8_t sp = solid[p];
  double a[6];
  a[0] = __ddiv_rn(hx, q.i > 0 ? harm_d(rho[p - SI], rp) : rp);
  a[1] = __ddiv_rn(hx, q.i < nx - 1 ? harm_d(rp, rho[p + SI]) : rp);
  a[2] = __ddiv_rn(hx, q.j > 0 ? harm_d(rho[p - SJ], rp) : rp);
  a[3] = __ddiv_rn(hx, q.j < ny - 1 ? harm_d(rp, rho[p + SJ]) : rp);
  if (nz > 1) {
    a[4] = __ddiv_rn(hx, q.k > 0 ? harm_d(rho[p - 1], rp) : rp);
    a[5] = __ddiv_rn(hx, q.k < nz - 1 ? harm_d(rp, rho[p + 1]) : rp);
  } else {
    a[4] = 0.0;
    a[5] = 0.0;
  }
  double c = a[0];
  for (int f = 1; f < 6; ++f) c = __dadd_rn(c, a[f]);
  if (q.i > 0 && solid[p - SI] != sp) a[0] = 0.0;
  if (q.i < nx - 1 && solid[p + SI] != sp) a[1] = 0.0;
  if (q.j > 0 && solid[p - SJ] != sp) a[2] = 0.0;
  if (q.j < ny - 1 && solid[p + SJ] != sp) a[3] = 0.0;
  if (q.k > 0 && solid[p - 1] != sp) a[4] = 0.0;
  if (q.k < nz - 1 && solid[p + 1] != sp) a[5] = 0.0;
  if (!sp) {
    c = a[0];
    for (int f = 1; f < 6; ++f) c = __dadd_rn(c, a[f]);
  }
  const bool onb[6] = {q.i == 0, q.i == nx - 1, q.j == 0, q.j == ny - 1, q.k == 0, q.k == nz - 1};
  for (int f = 0; f < 6; ++f) {  // Neumann sides first, in face order
    if (bc[f] != PBG_BC_NEUMANN || (nz == 1 && f >= 4) || !onb[f]) continue;
    c = __dsub_rn(c, a[f]);
    a[f] = 0.0;
  }
  for (int f = 0; f < 6; ++f)
    if (bc[f] == PBG_BC_DIRICHLET && onb[f]) a[f] = 0.0;
  if (sp) {
    c = __dmul_rn(c, 1.0e-12);
    for (int f = 0; f < 6; ++f) a[f] = 0.0;
  }
  C = c;
  W = a[0];
  S = a[2];
  B = a[4];
}

}  // namespace pbg
