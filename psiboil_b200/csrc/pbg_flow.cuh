// The pressure-correction step around the solve, on the device: the
// pressure matrix of a two-phase mixture (Pressure::discretize with the
// reference's PropertyMix density), the right-hand side from the predicted
// velocity (Pressure::update_rhs) and the velocity projection
// (Momentum::project). One thread per cell, IEEE operations in the
// reference's order (no contraction), so that every output is bit for bit
// the reference's on a uniform grid whose coordinates are exact multiples
// of h (n a power of two).
//
// Cells: index (i*ny + j)*nz + k. Faces: u (nx+1) x ny x nz, v nx x (ny+1)
// x nz, w nx x ny x (nz+1), k fastest; face f of u lies between cells f-1
// and f, so the west face of cell (i,j,k) is u[(i*ny + j)*nz + k].
#pragma once
#include <cstdint>

#include "../../include/psiboil_b200.h"
#include "pbg_common.cuh"

namespace pbg {

// Cell position: 32-bit multiply-shift division (Geo) below 2^31 cells,
// 64-bit division above.
__device__ __forceinline__ Pos flow_pos(const Geo &g, long long p, int ny, int nz) {
  if (g.n != 0u) return g.pos((uint32_t)p);
  return pos_of(p, ny, nz);
}

// Cell density of the mixture, PropertyMix::value(i,j,k)
// (Src/Matter/property_value.cpp:52-70): col clamped to [0, 1], then
// rho_a * col + rho_b * (1 - col).
__device__ __forceinline__ double mix_cell(const double *__restrict__ col, double ra, double rb,
                                           long long p) {
  double c = col[p];
  if (c > 1.0) c = 1.0;
  if (c < 0.0) c = 0.0;
  return __dadd_rn(__dmul_rn(ra, c), __dmul_rn(rb, __dsub_rn(1.0, c)));
}

// Density at the face between cell p and its lower neighbour pm,
// PropertyMix::value(Comp,i,j,k) (:73-85): 0.5 * (value(p) + value(pm)).
// A boundary face passes pm == p (the reference's ghost cell holds the
// boundary cell's colour). col == nullptr: a single fluid of density ra
// (a constant Property returns its value, :18-21).
__device__ __forceinline__ double mix_face(const double *__restrict__ col, double ra, double rb,
                                           long long p, long long pm) {
  if (!col) return ra;
  return __dmul_rn(0.5, __dadd_rn(mix_cell(col, ra, rb, p), mix_cell(col, ra, rb, pm)));
}

// Pressure::discretize (Src/Equation/Centered/Pressure/
// pressure_discretize.cpp:24-67,91-148) with Centered::create_system_bnd
// (Src/Equation/Centered/centered_system_bnd.cpp:17-62,142-184), written in
// the symmetric storage c, w, s, b of cell p:
//  * a_f = dS / dx / rho_face with dS = h*h; dx = h between two cell
//    centres and h/2 between a boundary cell's centre and the wall (the
//    reference's zero-width ghost cells, grid1d_correct_boundaries.cpp);
//    the dummy k direction of a 2-D grid keeps h on both sides
//  * c = w + e + s + n + b + t; faces between fluid and solid cells
//    zeroed on both sides and c of fluid cells recomputed
//  * Neumann sides, and the pseudo k sides of a 2-D grid, in the order
//    imin..kmax: c -= a_bnd, a_bnd = 0; Dirichlet sides: a_bnd = 0
//  * solid cells: c *= 1e-12, no couplings.
// With a cut body (bidx != nullptr; solid then holds its off cells, fV = 0,
// and bidx the index of each cut cell, 0 < fV < 1, in bfs, six face
// fractions w e s n b t per cut cell) the body branch of :72-119 instead:
// the reference visits the cells of the body's cut-cell list, which are its
// cut cells. A coupling of a cut cell to a cut neighbour is multiplied by
// the cell's own face fraction; a coupling between a listed cell and an
// off cell, in either direction, is zeroed; c of every cell that is not
// off is recomputed. The two cells of a face carry their own fractions,
// so the matrix is not symmetric. Cells on the domain boundary must not
// be cut (their neighbours beyond it count as fluid).
__device__ __forceinline__ void assemble_mix_cell(int nx, int ny, int nz, double h, const int (&bc)[6],
                                                  const double *__restrict__ col, double ra, double rb,
                                                  const uint8_t *__restrict__ solid,
                                                  const int *__restrict__ bidx,
                                                  const double *__restrict__ bfs, long long p, Pos q,
                                                  double (&a)[6], double &C) {
  const long long SI = (long long)ny * nz, SJ = nz;
  const double hh = __dmul_rn(h, h);
  const double hx = __ddiv_rn(hh, h);
  const double hxb = __ddiv_rn(hh, __dmul_rn(0.5, h));
  a[0] = __ddiv_rn(q.i == 0 ? hxb : hx, mix_face(col, ra, rb, p, q.i > 0 ? p - SI : p));
  a[1] = __ddiv_rn(q.i == nx - 1 ? hxb : hx, mix_face(col, ra, rb, q.i < nx - 1 ? p + SI : p, p));
  a[2] = __ddiv_rn(q.j == 0 ? hxb : hx, mix_face(col, ra, rb, p, q.j > 0 ? p - SJ : p));
  a[3] = __ddiv_rn(q.j == ny - 1 ? hxb : hx, mix_face(col, ra, rb, q.j < ny - 1 ? p + SJ : p, p));
  if (nz > 1) {
    a[4] = __ddiv_rn(q.k == 0 ? hxb : hx, mix_face(col, ra, rb, p, q.k > 0 ? p - 1 : p));
    a[5] = __ddiv_rn(q.k == nz - 1 ? hxb : hx, mix_face(col, ra, rb, q.k < nz - 1 ? p + 1 : p, p));
  } else {
    a[4] = __ddiv_rn(hx, mix_face(col, ra, rb, p, p));
    a[5] = a[4];
  }
  double c = a[0];
  for (int f = 1; f < 6; ++f) c = __dadd_rn(c, a[f]);
  const uint8_t sp = solid ? solid[p] : 0;
  if (bidx) {
    const long long nbp[6] = {p - SI, p + SI, p - SJ, p + SJ, p - 1, p + 1};
    const bool inb[6] = {q.i > 0, q.i < nx - 1, q.j > 0, q.j < ny - 1, q.k > 0, q.k < nz - 1};
    const int me = bidx[p];
    for (int f = 0; f < 6; ++f) {
      if (!inb[f]) continue;
      const int nb = bidx[nbp[f]];
      if (me >= 0 && nb >= 0) a[f] = __dmul_rn(a[f], bfs[6ll * me + f]);
      if ((me >= 0 || nb >= 0) && (sp || solid[nbp[f]])) a[f] = 0.0;
    }
    if (!sp) {
      c = a[0];
      for (int f = 1; f < 6; ++f) c = __dadd_rn(c, a[f]);
    }
  } else if (solid) {
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
  }
  const bool onb[6] = {q.i == 0, q.i == nx - 1, q.j == 0, q.j == ny - 1, q.k == 0, q.k == nz - 1};
  for (int f = 0; f < 6; ++f) {
    const bool pseudo = nz == 1 && f >= 4;
    if (!onb[f] || !(pseudo || bc[f] == PBG_BC_NEUMANN_)) continue;
    c = __dsub_rn(c, a[f]);
    a[f] = 0.0;
  }
  for (int f = 0; f < 6; ++f)
    if (onb[f] && !(nz == 1 && f >= 4) && bc[f] == PBG_BC_DIRICHLET_) a[f] = 0.0;
  if (sp) {
    c = __dmul_rn(c, 1.0e-12);
    for (int f = 0; f < 6; ++f) a[f] = 0.0;
  }
  C = c;
}

// Writes c, w, s, b (and e, n, t when E is not null: the seven-array form
// of a cut body's matrix).
__global__ void k_assemble_mix(Geo G, int nx, int ny, int nz, double h, int4 bc03, int2 bc45,
                               const double *__restrict__ col, double ra, double rb,
                               const uint8_t *__restrict__ solid, const int *__restrict__ bidx,
                               const double *__restrict__ bfs, double *__restrict__ C,
                               double *__restrict__ W, double *__restrict__ S, double *__restrict__ B,
                               double *__restrict__ E, double *__restrict__ Nn, double *__restrict__ T,
                               uint8_t *__restrict__ aflag) {
  const long long N = (long long)nx * ny * nz;
  const int bc[6] = {bc03.x, bc03.y, bc03.z, bc03.w, bc45.x, bc45.y};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    Pos q = flow_pos(G, p, ny, nz);
    double a[6], c;
    assemble_mix_cell(nx, ny, nz, h, bc, col, ra, rb, solid, bidx, bfs, p, q, a, c);
    C[p] = c;
    W[p] = a[0];
    S[p] = a[2];
    B[p] = a[4];
    if (E) {
      E[p] = a[1];
      Nn[p] = a[3];
      T[p] = a[5];
    }
    aflag[p] = (solid && solid[p]) ? 0 : 1;
  }
}

// Pressure::update_rhs (pressure_update_rhs.cpp:16-139): fnew = 0;
// += a u_w; -= a u_e; += a v_s; -= a v_n; += a w_b; -= a w_t with
// a = dS * dti (the caller passes a); then += fext + fbnd, which are zero
// for homogeneous boundary values. With a solid mask (a voxel body: every
// fluid cell uncut, face fractions 1) the immersed-body branch (:65-101): a
// face counts only if the neighbour across it is fluid (cells beyond the
// domain count as fluid), and solid cells get 0. With a cut body (bidx, bfs
// as for the assembly) the face areas of a cut cell are first multiplied by
// its face fractions (:34-43; an uncut fluid cell's fractions are 1). w may
// be nullptr in 2-D (its faces then count as zero).
__global__ void k_divergence(Geo G, int nx, int ny, int nz, double a, const double *__restrict__ u,
                             const double *__restrict__ v, const double *__restrict__ w,
                             const uint8_t *__restrict__ solid, const int *__restrict__ bidx,
                             const double *__restrict__ bfs, double *__restrict__ rhs) {
  const long long N = (long long)nx * ny * nz;
  const long long SI = (long long)ny * nz, SJ = nz;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    Pos q = flow_pos(G, p, ny, nz);
    const long long iu = p;  // west face of the cell
    const long long iv = ((long long)q.i * (ny + 1) + q.j) * nz + q.k;
    const long long iw = ((long long)q.i * ny + q.j) * (nz + 1) + q.k;
    bool open[6] = {true, true, true, true, true, true};
    if (solid) {
      open[0] = q.i == 0 || !solid[p - SI];
      open[1] = q.i == nx - 1 || !solid[p + SI];
      open[2] = q.j == 0 || !solid[p - SJ];
      open[3] = q.j == ny - 1 || !solid[p + SJ];
      open[4] = q.k == 0 || !solid[p - 1];
      open[5] = q.k == nz - 1 || !solid[p + 1];
    }
    double ad[6] = {a, a, a, a, a, a};
    if (bidx && bidx[p] >= 0)
      for (int d = 0; d < 6; ++d) ad[d] = __dmul_rn(a, bfs[6ll * bidx[p] + d]);
    double f = 0.0;
    if (open[0]) f = __dadd_rn(f, __dmul_rn(ad[0], u[iu]));
    if (open[1]) f = __dsub_rn(f, __dmul_rn(ad[1], u[iu + SI]));
    if (open[2]) f = __dadd_rn(f, __dmul_rn(ad[2], v[iv]));
    if (open[3]) f = __dsub_rn(f, __dmul_rn(ad[3], v[iv + nz]));
    if (open[4]) f = __dadd_rn(f, __dmul_rn(ad[4], w ? w[iw] : 0.0));
    if (open[5]) f = __dsub_rn(f, __dmul_rn(ad[5], w ? w[iw + 1] : 0.0));
    if (solid && solid[p]) f = 0.0;
    rhs[p] = __dadd_rn(f, 0.0);
  }
}

// Momentum::project (Src/Equation/Staggered/Momentum/momentum_project.cpp:
// 11-80) on every interior face: without a body (:26-45)
// u += (p[i-1] - p[i]) / rho_face * dt / dxc; with a solid mask, the
// immersed-body branch (:47-73): only faces between two fluid cells, as
// u += (p[i-1] - p[i]) * dt / rho_face / dxc. dxc = h. Thread p owns the
// west, south and bottom faces of its cell; the faces on the domain
// boundary are not touched (they hold the walls' values, which
// bnd_update_nooutlet restores in the reference), nor is w in 2-D.
__device__ __forceinline__ double project_increment(double pm, double pp, double rho, double dt, double h,
                                                    bool body) {
  const double dp = __dsub_rn(pm, pp);
  if (body) return __ddiv_rn(__ddiv_rn(__dmul_rn(dp, dt), rho), h);
  return __ddiv_rn(__dmul_rn(__ddiv_rn(dp, rho), dt), h);
}

__global__ void k_project(Geo G, int nx, int ny, int nz, double h, double dt, const double *__restrict__ pr,
                          const double *__restrict__ col, double ra, double rb,
                          const uint8_t *__restrict__ solid, double *__restrict__ u, double *__restrict__ v,
                          double *__restrict__ w) {
  const long long N = (long long)nx * ny * nz;
  const long long SI = (long long)ny * nz, SJ = nz;
  const bool body = solid != nullptr;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    Pos q = flow_pos(G, p, ny, nz);
    const bool sp = body && solid[p];
    const double pp = pr[p];
    if (q.i > 0 && !(body && (sp || solid[p - SI])))
      u[p] = __dadd_rn(u[p], project_increment(pr[p - SI], pp, mix_face(col, ra, rb, p, p - SI), dt, h, body));
    if (q.j > 0 && !(body && (sp || solid[p - SJ]))) {
      const long long iv = ((long long)q.i * (ny + 1) + q.j) * nz + q.k;
      v[iv] = __dadd_rn(v[iv], project_increment(pr[p - SJ], pp, mix_face(col, ra, rb, p, p - SJ), dt, h, body));
    }
    if (nz > 1 && q.k > 0 && !(body && (sp || solid[p - 1]))) {
      const long long iw = ((long long)q.i * ny + q.j) * (nz + 1) + q.k;
      w[iw] = __dadd_rn(w[iw], project_increment(pr[p - 1], pp, mix_face(col, ra, rb, p, p - 1), dt, h, body));
    }
  }
}

}  // namespace pbg
