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
__device__ __forceinline__ void assemble_mix_cell(int nx, int ny, int nz, double h, const int (&bc)[6],
                                                  const double *__restrict__ col, double ra, double rb,
                                                  const uint8_t *__restrict__ solid, long long p, Pos q,
                                                  double &C, double &W, double &S, double &B) {
  const long long SI = (long long)ny * nz, SJ = nz;
  const double hh = __dmul_rn(h, h);
  const double hx = __ddiv_rn(hh, h);
  const double hxb = __ddiv_rn(hh, __dmul_rn(0.5, h));
  double a[6];
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
  if (solid) {
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
  W = a[0];
  S = a[2];
  B = a[4];
}

__global__ void k_assemble_mix(Geo G, int nx, int ny, int nz, double h, int4 bc03, int2 bc45,
                               const double *__restrict__ col, double ra, double rb,
                               const uint8_t *__restrict__ solid, double *__restrict__ C,
                               double *__restrict__ W, double *__restrict__ S, double *__restrict__ B,
                               uint8_t *__restrict__ aflag) {
  const long long N = (long long)nx * ny * nz;
  const int bc[6] = {bc03.x, bc03.y, bc03.z, bc03.w, bc45.x, bc45.y};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    Pos q = flow_pos(G, p, ny, nz);
    double c, w, sv, b;
    assemble_mix_cell(nx, ny, nz, h, bc, col, ra, rb, solid, p, q, c, w, sv, b);
    C[p] = c;
    W[p] = w;
    S[p] = sv;
    B[p] = b;
    aflag[p] = (solid && solid[p]) ? 0 : 1;
  }
}

// Pressure::update_rhs (pressure_update_rhs.cpp:16-139): fnew = 0;
// += a u_w; -= a u_e; += a v_s; -= a v_n; += a w_b; -= a w_t with
// a = dS * dti (the caller passes a); then += fext + fbnd, which are zero
// for homogeneous boundary values. With a solid mask (a voxel body: every
// fluid cell uncut, face fractions 1) the immersed-body branch (:65-101): a
// face counts only if the neighbour across it is fluid (cells beyond the
// domain count as fluid), and solid cells get 0. w may be nullptr in 2-D
// (its faces then count as zero).
__global__ void k_divergence(Geo G, int nx, int ny, int nz, double a, const double *__restrict__ u,
                             const double *__restrict__ v, const double *__restrict__ w,
                             const uint8_t *__restrict__ solid, double *__restrict__ rhs) {
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
    double f = 0.0;
    if (open[0]) f = __dadd_rn(f, __dmul_rn(a, u[iu]));
    if (open[1]) f = __dsub_rn(f, __dmul_rn(a, u[iu + SI]));
    if (open[2]) f = __dadd_rn(f, __dmul_rn(a, v[iv]));
    if (open[3]) f = __dsub_rn(f, __dmul_rn(a, v[iv + nz]));
    if (open[4]) f = __dadd_rn(f, __dmul_rn(a, w ? w[iw] : 0.0));
    if (open[5]) f = __dsub_rn(f, __dmul_rn(a, w ? w[iw + 1] : 0.0));
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
