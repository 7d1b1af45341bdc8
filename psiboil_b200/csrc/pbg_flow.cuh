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

// ---------------------------------------------------------------------------
// Row-vector forms of the three flow kernels: a thread owns 4 consecutive
// cells of a k-row (nz % 4 == 0, no cut body, fewer than 2^31 cells), reads
// every row with 16-byte loads and shares what neighbouring cells of the row
// have in common: the mixture density of each cell is formed once, the face
// density and coefficient between two cells of the row once (the top face
// of a cell is the bottom face of the next). Every value is computed by the
// same operations in the same order as the one-cell kernels above, so the
// outputs are bit for bit theirs.
// ---------------------------------------------------------------------------
constexpr int kFlowV = 4;

__device__ __forceinline__ void ld4d(const double *__restrict__ a, uint32_t p, double (&o)[4]) {
  const double2 u = *reinterpret_cast<const double2 *>(a + p);
  const double2 v = *reinterpret_cast<const double2 *>(a + p + 2);
  o[0] = u.x; o[1] = u.y; o[2] = v.x; o[3] = v.y;
}
__device__ __forceinline__ void st4d(double *__restrict__ a, uint32_t p, const double (&o)[4]) {
  *reinterpret_cast<double2 *>(a + p) = make_double2(o[0], o[1]);
  *reinterpret_cast<double2 *>(a + p + 2) = make_double2(o[2], o[3]);
}
__device__ __forceinline__ uchar4 ld4b(const uint8_t *__restrict__ a, uint32_t p) {
  return *reinterpret_cast<const uchar4 *>(a + p);
}
__device__ __forceinline__ uint8_t byte_of(uchar4 v, int m) {
  return m == 0 ? v.x : m == 1 ? v.y : m == 2 ? v.z : v.w;
}
// mixture densities of 4 cells of a row (mix_cell), or ra without colour
__device__ __forceinline__ void mix4(const double *__restrict__ col, double ra, double rb, uint32_t p,
                                     double (&o)[4]) {
  if (!col) { o[0] = o[1] = o[2] = o[3] = ra; return; }
  double c[4];
  ld4d(col, p, c);
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    double v = c[m];
    if (v > 1.0) v = 1.0;
    if (v < 0.0) v = 0.0;
    o[m] = __dadd_rn(__dmul_rn(ra, v), __dmul_rn(rb, __dsub_rn(1.0, v)));
  }
}
__device__ __forceinline__ double mix1(const double *__restrict__ col, double ra, double rb, long long p) {
  return col ? mix_cell(col, ra, rb, p) : ra;
}
// 0.5 * (value(first) + value(second)), mix_face's order; a constant
// density without colour
__device__ __forceinline__ double face_of(bool col, double ra, double m1, double m2) {
  return col ? __dmul_rn(0.5, __dadd_rn(m1, m2)) : ra;
}

__global__ void __launch_bounds__(kThreads)
    kv_assemble_mix(Geo G, int nx, int ny, int nz, double h, int4 bc03, int2 bc45,
                    const double *__restrict__ col, double ra, double rb, const uint8_t *__restrict__ solid,
                    double *__restrict__ C, double *__restrict__ W, double *__restrict__ S,
                    double *__restrict__ B, uint8_t *__restrict__ aflag) {
  const int bc[6] = {bc03.x, bc03.y, bc03.z, bc03.w, bc45.x, bc45.y};
  const uint32_t SI = G.nynz, SJ = (uint32_t)nz;
  const double hh = __dmul_rn(h, h);
  const double hx = __ddiv_rn(hh, h);
  const double hxb = __ddiv_rn(hh, __dmul_rn(0.5, h));
  const bool hc = col != nullptr;
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < G.n / kFlowV; g += gridDim.x * blockDim.x) {
    const uint32_t p = g * kFlowV;
    const Pos q = G.pos(p);
    double mc[4], mw[4], me[4], ms[4], mn[4];
    mix4(col, ra, rb, p, mc);
    if (q.i > 0) mix4(col, ra, rb, p - SI, mw);
    if (q.i < nx - 1) mix4(col, ra, rb, p + SI, me);
    if (q.j > 0) mix4(col, ra, rb, p - SJ, ms);
    if (q.j < ny - 1) mix4(col, ra, rb, p + SJ, mn);
    const double mkm = q.k > 0 ? mix1(col, ra, rb, (long long)p - 1) : 0.0;
    const double mkp = q.k + kFlowV < nz ? mix1(col, ra, rb, (long long)p + kFlowV) : 0.0;
    // bottom faces of the row's cells and the top face of its last cell
    double bf[5];
    bf[0] = q.k == 0 ? __ddiv_rn(hxb, face_of(hc, ra, mc[0], mc[0])) : __ddiv_rn(hx, face_of(hc, ra, mc[0], mkm));
#pragma unroll
    for (int m = 1; m < 4; ++m) bf[m] = __ddiv_rn(hx, face_of(hc, ra, mc[m], mc[m - 1]));
    bf[4] = q.k + kFlowV == nz ? __ddiv_rn(hxb, face_of(hc, ra, mc[3], mc[3]))
                               : __ddiv_rn(hx, face_of(hc, ra, mkp, mc[3]));
    uchar4 sc = make_uchar4(0, 0, 0, 0), sw = sc, se = sc, ss = sc, sn = sc;
    uint8_t skm = 0, skp = 0;
    if (solid) {
      sc = ld4b(solid, p);
      if (q.i > 0) sw = ld4b(solid, p - SI);
      if (q.i < nx - 1) se = ld4b(solid, p + SI);
      if (q.j > 0) ss = ld4b(solid, p - SJ);
      if (q.j < ny - 1) sn = ld4b(solid, p + SJ);
      if (q.k > 0) skm = solid[p - 1];
      if (q.k + kFlowV < nz) skp = solid[p + kFlowV];
    }
    double oc[4], ow[4], os[4], ob[4];
    uchar4 af;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      double a[6];
      a[0] = __ddiv_rn(q.i == 0 ? hxb : hx, q.i > 0 ? face_of(hc, ra, mc[m], mw[m]) : face_of(hc, ra, mc[m], mc[m]));
      a[1] = __ddiv_rn(q.i == nx - 1 ? hxb : hx,
                       q.i < nx - 1 ? face_of(hc, ra, me[m], mc[m]) : face_of(hc, ra, mc[m], mc[m]));
      a[2] = __ddiv_rn(q.j == 0 ? hxb : hx, q.j > 0 ? face_of(hc, ra, mc[m], ms[m]) : face_of(hc, ra, mc[m], mc[m]));
      a[3] = __ddiv_rn(q.j == ny - 1 ? hxb : hx,
                       q.j < ny - 1 ? face_of(hc, ra, mn[m], mc[m]) : face_of(hc, ra, mc[m], mc[m]));
      a[4] = bf[m];
      a[5] = bf[m + 1];
      const int kk = q.k + m;
      double c = a[0];
#pragma unroll
      for (int f = 1; f < 6; ++f) c = __dadd_rn(c, a[f]);
      const uint8_t sp = byte_of(sc, m);
      if (solid) {
        const uint8_t sbm = m > 0 ? byte_of(sc, m - 1) : skm, stp = m < 3 ? byte_of(sc, m + 1) : skp;
        if (q.i > 0 && byte_of(sw, m) != sp) a[0] = 0.0;
        if (q.i < nx - 1 && byte_of(se, m) != sp) a[1] = 0.0;
        if (q.j > 0 && byte_of(ss, m) != sp) a[2] = 0.0;
        if (q.j < ny - 1 && byte_of(sn, m) != sp) a[3] = 0.0;
        if (kk > 0 && sbm != sp) a[4] = 0.0;
        if (kk < nz - 1 && stp != sp) a[5] = 0.0;
        if (!sp) {
          c = a[0];
#pragma unroll
          for (int f = 1; f < 6; ++f) c = __dadd_rn(c, a[f]);
        }
      }
      const bool onb[6] = {q.i == 0, q.i == nx - 1, q.j == 0, q.j == ny - 1, kk == 0, kk == nz - 1};
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        if (!onb[f] || bc[f] != PBG_BC_NEUMANN_) continue;
        c = __dsub_rn(c, a[f]);
        a[f] = 0.0;
      }
#pragma unroll
      for (int f = 0; f < 6; ++f)
        if (onb[f] && bc[f] == PBG_BC_DIRICHLET_) a[f] = 0.0;
      if (sp) {
        c = __dmul_rn(c, 1.0e-12);
#pragma unroll
        for (int f = 0; f < 6; ++f) a[f] = 0.0;
      }
      oc[m] = c; ow[m] = a[0]; os[m] = a[2]; ob[m] = a[4];
      const uint8_t fl = sp ? 0 : 1;
      if (m == 0) af.x = fl; else if (m == 1) af.y = fl; else if (m == 2) af.z = fl; else af.w = fl;
    }
    st4d(C, p, oc);
    st4d(W, p, ow);
    st4d(S, p, os);
    st4d(B, p, ob);
    *reinterpret_cast<uchar4 *>(aflag + p) = af;
  }
}

// update_rhs for 4 cells of a row, the voxel-body branch of k_divergence.
__global__ void __launch_bounds__(kThreads)
    kv_divergence(Geo G, int nx, int ny, int nz, double a, const double *__restrict__ u,
                  const double *__restrict__ v, const double *__restrict__ w,
                  const uint8_t *__restrict__ solid, double *__restrict__ rhs) {
  const uint32_t SI = G.nynz, SJ = (uint32_t)nz;
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < G.n / kFlowV; g += gridDim.x * blockDim.x) {
    const uint32_t p = g * kFlowV;
    const Pos q = G.pos(p);
    const uint32_t iv = ((uint32_t)q.i * (ny + 1) + q.j) * nz + q.k;
    const long long iw = ((long long)q.i * ny + q.j) * (nz + 1) + q.k;
    double uw[4], ue[4], vs[4], vn[4], wz[5];
    ld4d(u, p, uw);
    ld4d(u, p + SI, ue);
    ld4d(v, iv, vs);
    ld4d(v, iv + nz, vn);
#pragma unroll
    for (int m = 0; m < 5; ++m) wz[m] = w[iw + m];
    uchar4 sc = make_uchar4(0, 0, 0, 0), sw = sc, se = sc, ss = sc, sn = sc;
    uint8_t skm = 0, skp = 0;
    if (solid) {
      sc = ld4b(solid, p);
      if (q.i > 0) sw = ld4b(solid, p - SI);
      if (q.i < nx - 1) se = ld4b(solid, p + SI);
      if (q.j > 0) ss = ld4b(solid, p - SJ);
      if (q.j < ny - 1) sn = ld4b(solid, p + SJ);
      if (q.k > 0) skm = solid[p - 1];
      if (q.k + kFlowV < nz) skp = solid[p + kFlowV];
    }
    double o[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      const int kk = q.k + m;
      bool open[6] = {true, true, true, true, true, true};
      if (solid) {
        const uint8_t sbm = m > 0 ? byte_of(sc, m - 1) : skm, stp = m < 3 ? byte_of(sc, m + 1) : skp;
        open[0] = q.i == 0 || !byte_of(sw, m);
        open[1] = q.i == nx - 1 || !byte_of(se, m);
        open[2] = q.j == 0 || !byte_of(ss, m);
        open[3] = q.j == ny - 1 || !byte_of(sn, m);
        open[4] = kk == 0 || !sbm;
        open[5] = kk == nz - 1 || !stp;
      }
      double f = 0.0;
      if (open[0]) f = __dadd_rn(f, __dmul_rn(a, uw[m]));
      if (open[1]) f = __dsub_rn(f, __dmul_rn(a, ue[m]));
      if (open[2]) f = __dadd_rn(f, __dmul_rn(a, vs[m]));
      if (open[3]) f = __dsub_rn(f, __dmul_rn(a, vn[m]));
      if (open[4]) f = __dadd_rn(f, __dmul_rn(a, wz[m]));
      if (open[5]) f = __dsub_rn(f, __dmul_rn(a, wz[m + 1]));
      if (solid && byte_of(sc, m)) f = 0.0;
      o[m] = __dadd_rn(f, 0.0);
    }
    st4d(rhs, p, o);
  }
}

// Momentum::project for 4 cells of a row (the faces k_project's threads own).
__global__ void __launch_bounds__(kThreads)
    kv_project(Geo G, int nx, int ny, int nz, double h, double dt, const double *__restrict__ pr,
               const double *__restrict__ col, double ra, double rb, const uint8_t *__restrict__ solid,
               double *__restrict__ u, double *__restrict__ v, double *__restrict__ w) {
  const uint32_t SI = G.nynz, SJ = (uint32_t)nz;
  const bool body = solid != nullptr;
  const bool hc = col != nullptr;
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < G.n / kFlowV; g += gridDim.x * blockDim.x) {
    const uint32_t p = g * kFlowV;
    const Pos q = G.pos(p);
    double pc[4], mc[4];
    ld4d(pr, p, pc);
    mix4(col, ra, rb, p, mc);
    uchar4 sc = make_uchar4(0, 0, 0, 0), sw = sc, ss = sc;
    uint8_t skm = 0;
    if (body) {
      sc = ld4b(solid, p);
      if (q.i > 0) sw = ld4b(solid, p - SI);
      if (q.j > 0) ss = ld4b(solid, p - SJ);
      if (q.k > 0) skm = solid[p - 1];
    }
    if (q.i > 0) {
      double pw[4], mw[4], uo[4];
      ld4d(pr, p - SI, pw);
      mix4(col, ra, rb, p - SI, mw);
      ld4d(u, p, uo);
#pragma unroll
      for (int m = 0; m < 4; ++m)
        if (!(body && (byte_of(sc, m) || byte_of(sw, m))))
          uo[m] = __dadd_rn(uo[m], project_increment(pw[m], pc[m], face_of(hc, ra, mc[m], mw[m]), dt, h, body));
      st4d(u, p, uo);
    }
    if (q.j > 0) {
      const uint32_t iv = ((uint32_t)q.i * (ny + 1) + q.j) * nz + q.k;
      double ps[4], mS[4], vo[4];
      ld4d(pr, p - SJ, ps);
      mix4(col, ra, rb, p - SJ, mS);
      ld4d(v, iv, vo);
#pragma unroll
      for (int m = 0; m < 4; ++m)
        if (!(body && (byte_of(sc, m) || byte_of(ss, m))))
          vo[m] = __dadd_rn(vo[m], project_increment(ps[m], pc[m], face_of(hc, ra, mc[m], mS[m]), dt, h, body));
      st4d(v, iv, vo);
    }
    if (nz > 1) {
      const long long iw = ((long long)q.i * ny + q.j) * (nz + 1) + q.k;
      const double pkm = q.k > 0 ? pr[p - 1] : 0.0;
      const double mkm = q.k > 0 ? mix1(col, ra, rb, (long long)p - 1) : 0.0;
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const int kk = q.k + m;
        if (kk == 0) continue;
        const uint8_t sbm = m > 0 ? byte_of(sc, m - 1) : skm;
        if (body && (byte_of(sc, m) || sbm)) continue;
        const double pb = m > 0 ? pc[m - 1] : pkm;
        const double mb = m > 0 ? mc[m - 1] : mkm;
        w[iw + m] = __dadd_rn(w[iw + m], project_increment(pb, pc[m], face_of(hc, ra, mc[m], mb), dt, h, body));
      }
    }
  }
}

}  // namespace pbg
