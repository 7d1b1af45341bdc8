/*
 * Seeded workload generator for pressure-Poisson problems.
 *
 * One header shared (bit-for-bit) by the engine library, the CPU oracle and
 * the reference fixture harness, so that every party solves exactly the same
 * system. Plain C99 (static inline), usable from C, C++ and CUDA host code.
 *
 * Cell layout: interior cells only, index = (i*ny + j)*nz + k, k fastest.
 * This is the interior of the reference's `val[i][j][k]` block
 * (Src/Global/global_malloc.cpp:35-56, k fastest) without the BW=3 halo.
 * A 2-D problem has nz == 1.
 *
 * Random numbers: the 64-bit Mersenne Twister (Matsumoto & Nishimura 2000,
 * the `std::mt19937_64` engine of the C++ standard), restated here so that C
 * code produces the same stream; u01 = (draw >> 11) * 2^-53.
 *
 * Pressure assembly (pbg_gen_assemble) is the fixture discretisation: it
 * follows Src/Equation/Centered/Pressure/pressure_discretize.cpp:24-148
 * (face coefficient dS/dx/rho_face, c = sum of the six, faces touching
 * solid cells zeroed on both sides, c of fluid cells recomputed, boundary
 * correction, ci = 1/c, solid cells c *= pico and faces zeroed) and
 * Src/Equation/Centered/centered_system_bnd.cpp:17-62,143-185 (Neumann:
 * c -= a_bnd, a_bnd = 0; Dirichlet p = 0: a_bnd = 0), with a HARMONIC face
 * density instead of the reference's arithmetic PropertyMix
 * (Src/Matter/property_value.cpp:73-85), as the workload specifies.
 */
#ifndef PSIBOIL_B200_PROBLEM_GEN_H
#define PSIBOIL_B200_PROBLEM_GEN_H

#include <stdint.h>
#include <stddef.h>
#include <math.h>
#include <string.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* 64-bit Mersenne Twister                                             */
/* ------------------------------------------------------------------ */
typedef struct { uint64_t mt[312]; int idx; } pbg_mt64;

static inline void pbg_mt64_seed(pbg_mt64 *g, uint64_t seed) {
  g->mt[0] = seed;
  for (int i = 1; i < 312; ++i)
    g->mt[i] = 6364136223846793005ULL * (g->mt[i - 1] ^ (g->mt[i - 1] >> 62)) + (uint64_t)i;
  g->idx = 312;
}

static inline uint64_t pbg_mt64_next(pbg_mt64 *g) {
  if (g->idx >= 312) {
    const uint64_t UM = 0xFFFFFFFF80000000ULL, LM = 0x7FFFFFFFULL;
    for (int i = 0; i < 312; ++i) {
      uint64_t x = (g->mt[i] & UM) | (g->mt[(i + 1) % 312] & LM);
      uint64_t xa = x >> 1;
      if (x & 1ULL) xa ^= 0xB5026F5AA96619E9ULL;
      g->mt[i] = g->mt[(i + 156) % 312] ^ xa;
    }
    g->idx = 0;
  }
  uint64_t y = g->mt[g->idx++];
  y ^= (y >> 29) & 0x5555555555555555ULL;
  y ^= (y << 17) & 0x71D67FFFEDA60000ULL;
  y ^= (y << 37) & 0xFFF7EEE000000000ULL;
  y ^= (y >> 43);
  return y;
}

static inline double pbg_u01(pbg_mt64 *g) {
  return (double)(pbg_mt64_next(g) >> 11) * (1.0 / 9007199254740992.0);
}

/* ------------------------------------------------------------------ */
/* Problem description                                                 */
/* ------------------------------------------------------------------ */
enum { PBG_BC_NEUMANN = 0, PBG_BC_DIRICHLET = 1, PBG_BC_PERIODIC = 2 };
enum { PBG_MAX_BUBBLES = 64 };

typedef struct {
  int nx, ny, nz;            /* interior cells; nz == 1 is a 2-D problem   */
  double h;                  /* uniform spacing (unit-cube side / cells)   */
  double rho_liquid;         /* density outside bubbles                    */
  double rho_vapour;         /* density inside bubbles                     */
  int nbub;
  double bub[PBG_MAX_BUBBLES][4]; /* centre x,y,z and radius, cell units   */
  int has_cyl;               /* solid cylinder along z                     */
  double cyl[3];             /* axis x, axis y, radius (cell units)        */
  int bc[6];                 /* imin, imax, jmin, jmax, kmin, kmax         */
  uint64_t seed;             /* seed of the right-hand side                */
} pbg_problem_desc;

static inline size_t pbg_ncells(const pbg_problem_desc *d) {
  return (size_t)d->nx * (size_t)d->ny * (size_t)d->nz;
}

static inline void pbg_default_bc(pbg_problem_desc *d) {
  for (int f = 0; f < 6; ++f) d->bc[f] = PBG_BC_NEUMANN;
  if (d->nz > 1) d->bc[5] = PBG_BC_DIRICHLET; /* top (kmax) */
  else d->bc[3] = PBG_BC_DIRICHLET;           /* 2-D: top is jmax */
}

/* One bubble of radius 0.2 centred at (0.5, 0.5, 0.4) of an n^3 unit cube. */
static inline void pbg_desc_single_bubble(pbg_problem_desc *d, int n, uint64_t seed) {
  memset(d, 0, sizeof(*d));
  d->nx = d->ny = d->nz = n;
  d->h = 1.0 / (double)n;
  d->rho_liquid = 1000.0;
  d->rho_vapour = 1.0;
  d->nbub = 1;
  d->bub[0][0] = 0.5 * n; d->bub[0][1] = 0.5 * n; d->bub[0][2] = 0.4 * n;
  d->bub[0][3] = 0.2 * n;
  pbg_default_bc(d);
  d->seed = seed;
}

/* n^3 cube, nb non-overlapping bubbles with radii U[rmin, rmax] cells at
 * rejection-sampled centres, a solid cylinder along z of radius rc cells on
 * the axis (n/2, n/2), density ratio `ratio`. Bubbles stay clear of each
 * other (gap >= 1 cell), of the cylinder and of the walls. */
static inline void pbg_desc_bubbles_cylinder(pbg_problem_desc *d, int n, int nb,
                                             double rmin, double rmax,
                                             double rc, double ratio,
                                             uint64_t seed) {
  memset(d, 0, sizeof(*d));
  d->nx = d->ny = d->nz = n;
  d->h = 1.0 / (double)n;
  d->rho_liquid = ratio;
  d->rho_vapour = 1.0;
  d->has_cyl = rc > 0.0;
  d->cyl[0] = 0.5 * n; d->cyl[1] = 0.5 * n; d->cyl[2] = rc;
  pbg_default_bc(d);
  d->seed = seed;
  pbg_mt64 g;
  pbg_mt64_seed(&g, seed * 2654435761ULL + 17ULL);
  if (nb > PBG_MAX_BUBBLES) nb = PBG_MAX_BUBBLES;
  int placed = 0;
  for (int tries = 0; placed < nb && tries < 1000000; ++tries) {
    double r = rmin + (rmax - rmin) * pbg_u01(&g);
    double cx = r + (n - 2.0 * r) * pbg_u01(&g);
    double cy = r + (n - 2.0 * r) * pbg_u01(&g);
    double cz = r + (n - 2.0 * r) * pbg_u01(&g);
    int ok = 1;
    if (d->has_cyl) {
      double dxy = sqrt((cx - d->cyl[0]) * (cx - d->cyl[0]) + (cy - d->cyl[1]) * (cy - d->cyl[1]));
      if (dxy < d->cyl[2] + r + 1.0) ok = 0;
    }
    for (int q = 0; ok && q < placed; ++q) {
      double ddx = cx - d->bub[q][0], ddy = cy - d->bub[q][1], ddz = cz - d->bub[q][2];
      if (sqrt(ddx * ddx + ddy * ddy + ddz * ddz) < r + d->bub[q][3] + 1.0) ok = 0;
    }
    if (!ok) continue;
    d->bub[placed][0] = cx; d->bub[placed][1] = cy; d->bub[placed][2] = cz;
    d->bub[placed][3] = r;
    ++placed;
  }
  d->nbub = placed;
}

/* Member `index` of a batch of uneven problems: the first `n2d` members are
 * 2-D squares with side log-uniform in [s2lo, s2hi], the rest 3-D cubes with
 * side log-uniform in [s3lo, s3hi]; 1-8 bubbles of radius U[0.05, 0.2] of
 * the side; density ratio log-uniform in [10, 1000]. */
static inline void pbg_desc_batch_member(pbg_problem_desc *d, uint64_t seed, int index,
                                         int n2d, int s2lo, int s2hi, int s3lo, int s3hi) {
  memset(d, 0, sizeof(*d));
  pbg_mt64 g;
  pbg_mt64_seed(&g, seed * 1000003ULL + (uint64_t)index * 7919ULL + 1ULL);
  int is2d = index < n2d;
  double lo = is2d ? s2lo : s3lo, hi = is2d ? s2hi : s3hi;
  int side = (int)floor(exp(log(lo) + (log(hi) - log(lo)) * pbg_u01(&g)));
  if (side < 2) side = 2;
  d->nx = d->ny = side;
  d->nz = is2d ? 1 : side;
  d->h = 1.0 / (double)side;
  double ratio = exp(log(10.0) + (log(1000.0) - log(10.0)) * pbg_u01(&g));
  d->rho_liquid = ratio;
  d->rho_vapour = 1.0;
  int nb = 1 + (int)(8.0 * pbg_u01(&g));
  if (nb > 8) nb = 8;
  for (int q = 0; q < nb; ++q) {
    double r = (0.05 + 0.15 * pbg_u01(&g)) * side;
    d->bub[q][0] = r + (side - 2.0 * r) * pbg_u01(&g);
    d->bub[q][1] = r + (side - 2.0 * r) * pbg_u01(&g);
    d->bub[q][2] = is2d ? 0.5 : r + (side - 2.0 * r) * pbg_u01(&g);
    d->bub[q][3] = r;
  }
  d->nbub = nb;
  pbg_default_bc(d);
  d->seed = seed * 31ULL + (uint64_t)index;
}

/* ------------------------------------------------------------------ */
/* Fields                                                              */
/* ------------------------------------------------------------------ */
static inline int pbg_in_bubble(const pbg_problem_desc *d, int i, int j, int k) {
  double x = i + 0.5, y = j + 0.5, z = (d->nz > 1) ? k + 0.5 : 0.5;
  for (int q = 0; q < d->nbub; ++q) {
    double ddx = x - d->bub[q][0], ddy = y - d->bub[q][1], ddz = z - d->bub[q][2];
    if (d->nz == 1) ddz = 0.0;
    if (ddx * ddx + ddy * ddy + ddz * ddz < d->bub[q][3] * d->bub[q][3]) return 1;
  }
  return 0;
}

static inline int pbg_in_solid(const pbg_problem_desc *d, int i, int j, int k) {
  (void)k;
  if (!d->has_cyl) return 0;
  double x = i + 0.5 - d->cyl[0], y = j + 0.5 - d->cyl[1];
  return x * x + y * y < d->cyl[2] * d->cyl[2];
}

/* Cell density (sharp colour function) and solid mask (1 = solid). */
static inline void pbg_gen_fields(const pbg_problem_desc *d, double *rho, uint8_t *solid) {
  for (int i = 0; i < d->nx; ++i)
    for (int j = 0; j < d->ny; ++j)
      for (int k = 0; k < d->nz; ++k) {
        size_t c = ((size_t)i * d->ny + j) * d->nz + k;
        rho[c] = pbg_in_bubble(d, i, j, k) ? d->rho_vapour : d->rho_liquid;
        solid[c] = (uint8_t)pbg_in_solid(d, i, j, k);
      }
}

/* Right-hand side: U[-1,1] per cell (drawn for every cell, in index
 * order), zero on solid cells, minus the mean over fluid cells, times
 * 1/h^2. `stream` selects an independent request (0 for the first). */
static inline void pbg_gen_rhs(const pbg_problem_desc *d, uint64_t stream,
                               const uint8_t *solid, double *b) {
  pbg_mt64 g;
  pbg_mt64_seed(&g, d->seed ^ (0x9E3779B97F4A7C15ULL * (stream + 1ULL)));
  size_t n = pbg_ncells(d);
  double sum = 0.0;
  size_t nf = 0;
  for (size_t c = 0; c < n; ++c) {
    double u = 2.0 * pbg_u01(&g) - 1.0;
    b[c] = solid[c] ? 0.0 : u;
    if (!solid[c]) { sum += b[c]; ++nf; }
  }
  double mean = nf ? sum / (double)nf : 0.0;
  double s = 1.0 / (d->h * d->h);
  for (size_t c = 0; c < n; ++c)
    b[c] = solid[c] ? 0.0 : (b[c] - mean) * s;
}

/* ------------------------------------------------------------------ */
/* Flow state of a pressure-correction step                           */
/* ------------------------------------------------------------------ */
/* Face layouts (interior faces of the staggered Vector, boundary faces
 * included): u (nx+1) x ny x nz, v nx x (ny+1) x nz, w nx x ny x (nz+1),
 * each k fastest. Face f of u lies between cells f-1 and f. */
static inline size_t pbg_nfaces(const pbg_problem_desc *d, int comp) {
  return (size_t)(d->nx + (comp == 0)) * (size_t)(d->ny + (comp == 1)) *
         (size_t)(d->nz + (comp == 2));
}

/* Liquid colour of a cell (1 liquid, 0 vapour): a linear ramp over three
 * cells across each bubble's surface, the minimum over the bubbles. */
static inline double pbg_color_at(const pbg_problem_desc *d, int i, int j, int k) {
  double x = i + 0.5, y = j + 0.5, z = (d->nz > 1) ? k + 0.5 : 0.5;
  double c = 1.0;
  for (int q = 0; q < d->nbub; ++q) {
    double ddx = x - d->bub[q][0], ddy = y - d->bub[q][1], ddz = z - d->bub[q][2];
    if (d->nz == 1) ddz = 0.0;
    double s = (sqrt(ddx * ddx + ddy * ddy + ddz * ddz) - d->bub[q][3]) / 3.0 + 0.5;
    if (s < 0.0) s = 0.0;
    if (s > 1.0) s = 1.0;
    if (s < c) c = s;
  }
  return c;
}

/* Colour field and a predicted velocity u* for one step: face velocities
 * U[-0.5, 0.5) drawn over u, then v, then w faces in index order; the
 * normal faces on the domain boundary are walls (0), and w is 0 in 2-D.
 * `stream` selects an independent draw. */
static inline void pbg_gen_flow(const pbg_problem_desc *d, uint64_t stream, double *col,
                                double *u, double *v, double *w) {
  const int nx = d->nx, ny = d->ny, nz = d->nz;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) col[((size_t)i * ny + j) * nz + k] = pbg_color_at(d, i, j, k);
  pbg_mt64 g;
  pbg_mt64_seed(&g, d->seed ^ (0xD1B54A32D192ED03ULL * (stream + 1ULL)));
  for (int i = 0; i <= nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        double r = pbg_u01(&g) - 0.5;
        u[((size_t)i * ny + j) * nz + k] = (i == 0 || i == nx) ? 0.0 : r;
      }
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j <= ny; ++j)
      for (int k = 0; k < nz; ++k) {
        double r = pbg_u01(&g) - 0.5;
        v[((size_t)i * (ny + 1) + j) * nz + k] = (j == 0 || j == ny) ? 0.0 : r;
      }
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k <= nz; ++k) {
        double r = nz > 1 ? pbg_u01(&g) - 0.5 : 0.0;
        w[((size_t)i * ny + j) * (nz + 1) + k] = (k == 0 || k == nz) ? 0.0 : r;
      }
}

/* Harmonic mean of two face-adjacent densities; symmetric bit-for-bit. */
static inline double pbg_harm(double a, double b) {
  return (a * b) * 2.0 / (a + b);
}

/* Periodic axes of a boundary-type list: bit d set when both faces of axis
 * d (0 i, 1 j, 2 k) are periodic. */
static inline int pbg_periodic_mask(const int bc[6]) {
  int m = 0;
  for (int d = 0; d < 3; ++d)
    if (bc[2 * d] == PBG_BC_PERIODIC && bc[2 * d + 1] == PBG_BC_PERIODIC) m |= 1 << d;
  return m;
}

/* Fixture assembly, stage 1: face coefficients dS/dx/rho_face from the
 * cell densities (pressure_discretize.cpp:24-57), c = sum of the six
 * (:65-67), faces between fluid and solid cells zeroed on both sides and c
 * of fluid cells recomputed (:72-119 for a voxel body: every fluid/solid
 * face pair is a "touch"). Boundary faces use the boundary cell's density;
 * on a periodic axis (bit d of per) the boundary face couples to the cell
 * at the other end, as the reference's periodic halo does
 * (scalar_exchange.cpp:47-58), with the same harmonic density both ways. */
static inline void pbg_gen_faces_per(int nx, int ny, int nz, double h, int per,
                                     const double *rho, const uint8_t *solid,
                                     double *c, double *w, double *e, double *s,
                                     double *n, double *b, double *t) {
  const size_t SI = (size_t)ny * nz, SJ = (size_t)nz;
  const double hx = (h * h) / h; /* dS / dx for a uniform cube */
  const int pi = per & 1, pj = (per >> 1) & 1, pk = (per >> 2) & 1;
  /* neighbour index across each face, or -1 outside a non-periodic face */
#define PBG_WEST(i) ((i) > 0 ? (long long)(p - SI) : (pi ? (long long)(p + (size_t)(nx - 1) * SI) : -1LL))
#define PBG_EAST(i) ((i) < nx - 1 ? (long long)(p + SI) : (pi ? (long long)(p - (size_t)(nx - 1) * SI) : -1LL))
#define PBG_SOUTH(j) ((j) > 0 ? (long long)(p - SJ) : (pj ? (long long)(p + (size_t)(ny - 1) * SJ) : -1LL))
#define PBG_NORTH(j) ((j) < ny - 1 ? (long long)(p + SJ) : (pj ? (long long)(p - (size_t)(ny - 1) * SJ) : -1LL))
#define PBG_BOT(k) ((k) > 0 ? (long long)(p - 1) : (pk ? (long long)(p + (size_t)(nz - 1)) : -1LL))
#define PBG_TOP(k) ((k) < nz - 1 ? (long long)(p + 1) : (pk ? (long long)(p - (size_t)(nz - 1)) : -1LL))
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        size_t p = (size_t)i * SI + (size_t)j * SJ + k;
        double rp = rho[p];
        long long qw = PBG_WEST(i), qe = PBG_EAST(i), qs = PBG_SOUTH(j), qn = PBG_NORTH(j);
        long long qb = PBG_BOT(k), qt = PBG_TOP(k);
        double rw = qw >= 0 ? pbg_harm(rho[qw], rp) : rp;
        double re = qe >= 0 ? pbg_harm(rp, rho[qe]) : rp;
        double rs = qs >= 0 ? pbg_harm(rho[qs], rp) : rp;
        double rn = qn >= 0 ? pbg_harm(rp, rho[qn]) : rp;
        double rb = qb >= 0 ? pbg_harm(rho[qb], rp) : rp;
        double rt = qt >= 0 ? pbg_harm(rp, rho[qt]) : rp;
        w[p] = hx / rw; e[p] = hx / re;
        s[p] = hx / rs; n[p] = hx / rn;
        if (nz > 1) { b[p] = hx / rb; t[p] = hx / rt; }
        else { b[p] = 0.0; t[p] = 0.0; }
        c[p] = w[p] + e[p] + s[p] + n[p] + b[p] + t[p];
      }
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        size_t p = (size_t)i * SI + (size_t)j * SJ + k;
        int sp = solid[p];
        long long qw = PBG_WEST(i), qe = PBG_EAST(i), qs = PBG_SOUTH(j), qn = PBG_NORTH(j);
        long long qb = PBG_BOT(k), qt = PBG_TOP(k);
        if (qw >= 0 && solid[qw] != sp) w[p] = 0.0;
        if (qe >= 0 && solid[qe] != sp) e[p] = 0.0;
        if (qs >= 0 && solid[qs] != sp) s[p] = 0.0;
        if (qn >= 0 && solid[qn] != sp) n[p] = 0.0;
        if (nz > 1 && qb >= 0 && solid[qb] != sp) b[p] = 0.0;
        if (nz > 1 && qt >= 0 && solid[qt] != sp) t[p] = 0.0;
      }
#undef PBG_WEST
#undef PBG_EAST
#undef PBG_SOUTH
#undef PBG_NORTH
#undef PBG_BOT
#undef PBG_TOP
  for (size_t p = 0; p < (size_t)nx * SI; ++p)
    if (!solid[p]) c[p] = w[p] + e[p] + s[p] + n[p] + b[p] + t[p];
}

static inline void pbg_gen_faces(int nx, int ny, int nz, double h,
                                 const double *rho, const uint8_t *solid,
                                 double *c, double *w, double *e, double *s,
                                 double *n, double *b, double *t) {
  pbg_gen_faces_per(nx, ny, nz, h, 0, rho, solid, c, w, e, s, n, b, t);
}

/* Fixture assembly, stage 2: boundary correction restated from
 * centered_system_bnd.cpp:17-62 (Neumann sides in the order imin, imax,
 * jmin, jmax, kmin, kmax: c -= a_bnd, a_bnd = 0) and :143-185 (Dirichlet
 * p = 0: a_bnd = 0, c keeps it); periodic faces keep their couplings; then
 * ci = 1/c (pressure_discretize.cpp:127)
 * and solid cells c *= pico with all faces zeroed (:132-148). 2-D problems
 * (nz == 1) have no k faces. */
static inline void pbg_gen_bc_finalize(int nx, int ny, int nz, const int bc[6],
                                       const uint8_t *solid,
                                       double *c, double *w, double *e, double *s,
                                       double *n, double *b, double *t, double *ci) {
  const size_t SI = (size_t)ny * nz, SJ = (size_t)nz;
  const double pico = 1.0e-12;
  for (int pass = 0; pass < 2; ++pass)
    for (int f = 0; f < 6; ++f) {
      if (bc[f] != (pass == 0 ? PBG_BC_NEUMANN : PBG_BC_DIRICHLET)) continue;
      if (nz == 1 && f >= 4) continue;
      for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
          for (int k = 0; k < nz; ++k) {
            size_t p = (size_t)i * SI + (size_t)j * SJ + k;
            double *a = NULL;
            if (f == 0 && i == 0) a = &w[p];
            if (f == 1 && i == nx - 1) a = &e[p];
            if (f == 2 && j == 0) a = &s[p];
            if (f == 3 && j == ny - 1) a = &n[p];
            if (f == 4 && k == 0) a = &b[p];
            if (f == 5 && k == nz - 1) a = &t[p];
            if (a) {
              if (pass == 0) c[p] -= *a;
              *a = 0.0;
            }
          }
    }
  for (size_t p = 0; p < (size_t)nx * SI; ++p) {
    ci[p] = 1.0 / c[p];
    if (solid[p]) {
      c[p] *= pico;
      w[p] = e[p] = s[p] = n[p] = b[p] = t[p] = 0.0;
    }
  }
}

/* Non-symmetric variant of the fixture, the shape of the reference's other
 * Centered equations (convection-diffusion): first-order upwind convection
 * with a mass flux F > 0 along +x between fluid cells adds F to the west
 * coupling and to the diagonal of the downstream cell. Applied after the
 * boundary correction; ci = 1/c is recomputed for the cells it changes. */
static inline void pbg_gen_convect(int nx, int ny, int nz, double F, const uint8_t *solid,
                                   double *c, double *w, double *ci) {
  const size_t SI = (size_t)ny * nz;
  for (int i = 1; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        size_t p = (size_t)i * SI + (size_t)j * nz + k;
        if (solid[p] || solid[p - SI]) continue;
        w[p] += F;
        c[p] += F;
        if (ci) ci[p] = 1.0 / c[p];
      }
}

/* Full fixture assembly (stage 1 + stage 2). Outputs the seven coefficient
 * arrays with the reference sign convention  A x = c x_P - sum a_nb x_nb,
 * and ci = 1/c taken before the solid-cell scaling. */
static inline void pbg_gen_assemble(int nx, int ny, int nz, double h, const int bc[6],
                                    const double *rho, const uint8_t *solid,
                                    double *c, double *w, double *e, double *s,
                                    double *n, double *b, double *t, double *ci) {
  pbg_gen_faces_per(nx, ny, nz, h, pbg_periodic_mask(bc), rho, solid, c, w, e, s, n, b, t);
  pbg_gen_bc_finalize(nx, ny, nz, bc, solid, c, w, e, s, n, b, t, ci);
}

#ifdef __cplusplus
}
#endif
#endif
