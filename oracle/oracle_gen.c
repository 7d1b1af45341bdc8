/*
 * Oracle-side entry to the shared seeded workload generator
 * (psiboil_b200/csrc/problem_gen.h). TEST INFRASTRUCTURE ONLY.
 *
 * kind 0: single bubble n^3; 1: bubbles + solid cylinder; 2: batch member.
 * params: n, nb, rmin, rmax, rc, ratio, index, n2d, s2lo, s2hi, s3lo, s3hi,
 *         rhs stream, periodic axes.
 * With solid == NULL only dims and hb (h, density ratio) are written;
 * otherwise out receives rho, rhs, c, w, e, s, n, b, t, ci (N each).
 */
#include <stdlib.h>
#include "problem_gen.h"

/* params[13]: periodic axes (bit 0 i, 1 j, 2 k): both faces of each set
 * axis become PBG_BC_PERIODIC */
static void make_desc(int kind, const double *params, uint64_t seed, pbg_problem_desc *dd) {
  pbg_problem_desc d;
  int n = (int)params[0];
  if (kind == 0) pbg_desc_single_bubble(&d, n, seed);
  else if (kind == 1)
    pbg_desc_bubbles_cylinder(&d, n, (int)params[1], params[2], params[3], params[4],
                              params[5], seed);
  else
    pbg_desc_batch_member(&d, seed, (int)params[6], (int)params[7], (int)params[8],
                          (int)params[9], (int)params[10], (int)params[11]);
  const int per = (int)params[13];
  for (int ax = 0; ax < 3; ++ax)
    if (per & (1 << ax)) d.bc[2 * ax] = d.bc[2 * ax + 1] = PBG_BC_PERIODIC;
  *dd = d;
}

int orc_gen_problem(int kind, const double *params, uint64_t seed, int *dims,
                    uint8_t *solid, double *hb, double *out) {
  pbg_problem_desc d;
  make_desc(kind, params, seed, &d);
  dims[0] = d.nx; dims[1] = d.ny; dims[2] = d.nz;
  hb[0] = d.h;
  hb[1] = d.rho_liquid / d.rho_vapour;
  if (!solid) return 0;
  size_t N = pbg_ncells(&d);
  double *rho = out, *b = out + N;
  pbg_gen_fields(&d, rho, solid);
  pbg_gen_rhs(&d, (uint64_t)params[12], solid, b);
  double *m = out + 2 * N;
  pbg_gen_assemble(d.nx, d.ny, d.nz, d.h, d.bc, rho, solid, m, m + N, m + 2 * N, m + 3 * N,
                   m + 4 * N, m + 5 * N, m + 6 * N, m + 7 * N);
  return 0;
}

/* Flow state of a pressure-correction step (pbg_gen_flow): colour and the
 * face velocities u, v, w, plus the two phase densities in rho2 (liquid,
 * vapour) and the pressure boundary types in bc (imin..kmax). `stream` is
 * params[12]. */
int orc_gen_flow(int kind, const double *params, uint64_t seed, double *col, double *u,
                 double *v, double *w, double *rho2, int *bc) {
  pbg_problem_desc d;
  make_desc(kind, params, seed, &d);
  for (int f = 0; f < 6; ++f) bc[f] = d.bc[f];
  rho2[0] = d.rho_liquid;
  rho2[1] = d.rho_vapour;
  pbg_gen_flow(&d, (uint64_t)params[12], col, u, v, w);
  return 0;
}

/* Non-symmetric variant of a fixture matrix (pbg_gen_convect), in place. */
int orc_convect(int nx, int ny, int nz, double F, const uint8_t *solid, double *c, double *w,
                double *ci) {
  pbg_gen_convect(nx, ny, nz, F, solid, c, w, ci);
  return 0;
}
