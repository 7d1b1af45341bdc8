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
#include <cstring>

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

// Correctly rounded IEEE double operations on the host and the device, for
// constants that the host forms once per launch (the host's double
// arithmetic is IEEE binary64 with round to nearest, as __ddiv_rn is).
__host__ __device__ __forceinline__ double div_rn(double a, double b) {
#ifdef __CUDA_ARCH__
  return __ddiv_rn(a, b);
#else
  return a / b;
#endif
}
__host__ __device__ __forceinline__ double mul_rn(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}
__host__ __device__ __forceinline__ double quiet_nan() {
#ifdef __CUDA_ARCH__
  return __longlong_as_double(0x7ff8000000000000LL);
#else
  const unsigned long long u = 0x7ff8000000000000ULL;
  double d;
  memcpy(&d, &u, sizeof d);
  return d;
#endif
}


// Momentum::project (Src/Equation/Staggered/Momentum/momentum_project.cpp:
// 11-80) on every interior face: without a body (:26-45)
// u += (p[i-1] - p[i]) / rho_face * dt / dxc; with a solid mask, the
// immersed-body branch (:47-73): only faces between two fluid cells, as
// u += (p[i-1] - p[i]) * dt / rho_face / dxc. dxc = h. Thread p owns the
// west, south and bottom faces of its cell; the faces on the domain
// boundary are not touched (they hold the walls' values, which
// bnd_update_nooutlet restores in the reference), nor is w in 2-D.
// Division by a divisor b known in advance (the spacing h, the density of a
// pure phase), rounded to nearest like a / b itself: with y = RN(1/b) formed
// once, q0 = RN(a y) lies within one ulp of a/b, the remainder r = a - b q0
// is exact in one FMA, and RN(q0 + r y) = RN(a/b) (Markstein's theorem:
// P. Markstein, IBM J. Res. Develop. 34(1), 1990; its use for a divisor
// known in advance: N. Brisebarre, J.-M. Muller and S. K. Raina, IEEE Trans.
// Comput. 53(8), 2004). The theorem needs every intermediate normal, so b
// is restricted to [2^-60, 2^60] and |a| to (2^-900, 2^900); zero, infinite
// and NaN dividends, and everything outside those ranges, take the division
// itself.
struct KnownDiv {
  double b, y;
  bool ok;
  KnownDiv() = default;
  __host__ __device__ __forceinline__ explicit KnownDiv(double b_) : b(b_) {
    y = div_rn(1.0, b_);
    const double m = fabs(b_);
    ok = m >= 0x1p-60 && m <= 0x1p60;
  }
  // a / b (a zero dividend: a b, the signed zero a / b is)
  __device__ __forceinline__ double operator()(double a) const {
    const double m = fabs(a);
    if (ok && m > 0x1p-900 && m < 0x1p900) {
      const double q0 = __dmul_rn(a, y);
      return __fma_rn(__fma_rn(-q0, b, a), y, q0);
    }
    if (ok && m == 0.0) return __dmul_rn(a, b);
    return __ddiv_rn(a, b);
  }
  // a / d for any d: the corrected product when d is b (b nonzero, so d == b
  // means the same bits), else the division (a zero dividend over a finite
  // nonzero d: a d, the same signed zero)
  __device__ __forceinline__ double by(double a, double d) const {
    if (d == b && ok) return (*this)(a);
    if (a == 0.0 && d != 0.0 && isfinite(d)) return __dmul_rn(a, d);
    return __ddiv_rn(a, d);
  }
};

// Face densities of the two pure phases (colour 1 and 0) and the spacing:
// the divisors the projection meets on every face away from an interface.
struct PhaseDiv {
  KnownDiv a, b, h;
  PhaseDiv() = default;
  __host__ __device__ __forceinline__ PhaseDiv(double ra, double rb, double h_) : a(ra), b(rb), h(h_) {}
  __device__ __forceinline__ double by_rho(double x, double rho) const {
    if (rho == a.b && a.ok) return a(x);
    return b.by(x, rho);
  }
};

// project_increment with the divisions by a pure-phase density and by h
// done by KnownDiv: the same bits
__device__ __forceinline__ double project_increment_k(double pm, double pp, double rho, double dt,
                                                      const PhaseDiv &D, bool body) {
  const double dp = __dsub_rn(pm, pp);
  if (body) return D.h(D.by_rho(__dmul_rn(dp, dt), rho));
  return D.h(__dmul_rn(D.by_rho(dp, rho), dt));
}

// project_increment for the fast groups of the marching projection: both
// divisions by Markstein's correction with no fallback (exact for +0 too;
// -0 would come out +0); a face density that is not a pure phase's, a
// dividend outside the range where the correction is exact (+0 included,
// -0 not), or a divisor outside [2^-60, 2^60] sets miss, and the group is
// redone by the general code.
struct ProjFast {
  double ka, kb, ra, rb, ya, yb, h, yh;
  bool hok;
  ProjFast() = default;
  __host__ __device__ __forceinline__ explicit ProjFast(const PhaseDiv &D) {
    const double nan = quiet_nan();
    ka = D.a.ok ? D.a.b : nan;
    kb = D.b.ok ? D.b.b : nan;
    ra = D.a.b; rb = D.b.b; ya = D.a.y; yb = D.b.y;
    h = D.h.b; yh = D.h.y; hok = D.h.ok;
  }
  __device__ __forceinline__ static double corr(double a, double b, double y, bool &miss) {
    const double m = fabs(a);
    miss |= !((m > 0x1p-900 && m < 0x1p900) || __double_as_longlong(a) == 0);
    const double q0 = __dmul_rn(a, y);
    return __fma_rn(__fma_rn(-q0, b, a), y, q0);
  }
  __device__ __forceinline__ double inc(double pm, double pp, double rho, double dt, bool body,
                                        bool &miss) const {
    const double dp = __dsub_rn(pm, pp);
    const bool isa = rho == ka;
    miss |= !(isa || rho == kb) || !hok;
    const double bb = isa ? ra : rb, yy = isa ? ya : yb;
    if (body) return corr(corr(__dmul_rn(dp, dt), bb, yy, miss), h, yh, miss);
    return corr(__dmul_rn(corr(dp, bb, yy, miss), dt), h, yh, miss);
  }
};

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
// Several cells of a k-row per thread (nz % 4 == 0, no cut body, fewer than
// 2^31 cells): rows are read with 16-byte loads, and what neighbouring cells
// of the row have in common is formed once (the mixture density of a cell,
// the face between two cells of the row: the top face of a cell is the
// bottom face of the next). The row helpers, the divergence in this form,
// and the marching assembly and projection below. Every value is computed
// by the same operations in the same order as the one-cell kernels above,
// so the outputs are bit for bit theirs.
// ---------------------------------------------------------------------------
constexpr int kFlowV = 4;  // cells a thread of the divergence; nz % kFlowV == 0

__device__ __forceinline__ double mix1(const double *__restrict__ col, double ra, double rb, long long p) {
  return col ? mix_cell(col, ra, rb, p) : ra;
}
// V cells of a row (V = 2 or 4): doubles in 16-byte pairs, solid flags as
// one V-byte word (byte m is cell m's)
template <int V>
__device__ __forceinline__ void ldvd(const double *__restrict__ a, uint32_t p, double (&o)[V]) {
#pragma unroll
  for (int q = 0; q < V; q += 2) {
    const double2 t = *reinterpret_cast<const double2 *>(a + p + q);
    o[q] = t.x;
    o[q + 1] = t.y;
  }
}
template <int V>
__device__ __forceinline__ void stvd(double *__restrict__ a, uint32_t p, const double (&o)[V]) {
#pragma unroll
  for (int q = 0; q < V; q += 2) *reinterpret_cast<double2 *>(a + p + q) = make_double2(o[q], o[q + 1]);
}
template <int V>
__device__ __forceinline__ uint32_t ldvb(const uint8_t *__restrict__ a, uint32_t p) {
  if constexpr (V == 4) return *reinterpret_cast<const uint32_t *>(a + p);
  else return *reinterpret_cast<const uint16_t *>(a + p);
}
template <int V>
__device__ __forceinline__ void stvb(uint8_t *__restrict__ a, uint32_t p, uint32_t f) {
  if constexpr (V == 4) *reinterpret_cast<uint32_t *>(a + p) = f;
  else *reinterpret_cast<uint16_t *>(a + p) = (uint16_t)f;
}
// every byte of a V-byte word set to b
template <int V>
__device__ __forceinline__ uint32_t bytes_all(uint32_t b) { return b * (V == 4 ? 0x01010101u : 0x0101u); }
__device__ __forceinline__ uint32_t byte_at(uint32_t x, int m) { return (x >> (8 * m)) & 0xffu; }
// mixture densities of V cells of a row (mix_cell), or ra without colour
template <int V>
__device__ __forceinline__ void mixv(const double *__restrict__ col, double ra, double rb, uint32_t p,
                                     double (&o)[V]) {
  if (!col) {
#pragma unroll
    for (int m = 0; m < V; ++m) o[m] = ra;
    return;
  }
  double c[V];
  ldvd<V>(col, p, c);
#pragma unroll
  for (int m = 0; m < V; ++m) {
    double v = c[m];
    if (v > 1.0) v = 1.0;
    if (v < 0.0) v = 0.0;
    o[m] = __dadd_rn(__dmul_rn(ra, v), __dmul_rn(rb, __dsub_rn(1.0, v)));
  }
}
// 0.5 * (value(first) + value(second)), mix_face's order; a constant
// density without colour
__device__ __forceinline__ double face_of(bool col, double ra, double m1, double m2) {
  return col ? __dmul_rn(0.5, __dadd_rn(m1, m2)) : ra;
}

// update_rhs for V cells of a row (V = kFlowV = 4), the voxel-body branch of
// k_divergence; the solid flags of the V cells are one V-byte word. Bounded
// for one block an SM, the compiler gives it 77 registers a thread (three
// blocks fit an SM): 6% faster at 512^3 than the 64-register form at four
// blocks, 3% slower at 256^3.
template <int V>
__global__ void __launch_bounds__(kThreads, 1)
    kv_divergence(Geo G, int nx, int ny, int nz, double a, const double *__restrict__ u,
                  const double *__restrict__ v, const double *__restrict__ w,
                  const uint8_t *__restrict__ solid, double *__restrict__ rhs) {
  const uint32_t SI = G.nynz, SJ = (uint32_t)nz;
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < G.n / V; g += gridDim.x * blockDim.x) {
    const uint32_t p = g * V;
    const Pos q = G.pos(p);
    const uint32_t iv = ((uint32_t)q.i * (ny + 1) + q.j) * nz + q.k;
    const long long iw = ((long long)q.i * ny + q.j) * (nz + 1) + q.k;
    double uw[V], ue[V], vs[V], vn[V], wz[V + 1];
    ldvd<V>(u, p, uw);
    ldvd<V>(u, p + SI, ue);
    ldvd<V>(v, iv, vs);
    ldvd<V>(v, iv + nz, vn);
#pragma unroll
    for (int m = 0; m < V + 1; ++m) wz[m] = w[iw + m];
    uint32_t sc = 0u, sw = 0u, se = 0u, ss = 0u, sn = 0u, skm = 0u, skp = 0u;
    if (solid) {
      sc = ldvb<V>(solid, p);
      if (q.i > 0) sw = ldvb<V>(solid, p - SI);
      if (q.i < nx - 1) se = ldvb<V>(solid, p + SI);
      if (q.j > 0) ss = ldvb<V>(solid, p - SJ);
      if (q.j < ny - 1) sn = ldvb<V>(solid, p + SJ);
      if (q.k > 0) skm = solid[p - 1];
      if (q.k + V < nz) skp = solid[p + V];
    }
    double o[V];
#pragma unroll
    for (int m = 0; m < V; ++m) {
      const int kk = q.k + m;
      bool open[6] = {true, true, true, true, true, true};
      if (solid) {
        const uint32_t sbm = m > 0 ? byte_at(sc, m - 1) : skm, stp = m < V - 1 ? byte_at(sc, m + 1) : skp;
        open[0] = q.i == 0 || !byte_at(sw, m);
        open[1] = q.i == nx - 1 || !byte_at(se, m);
        open[2] = q.j == 0 || !byte_at(ss, m);
        open[3] = q.j == ny - 1 || !byte_at(sn, m);
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
      if (solid && byte_at(sc, m)) f = 0.0;
      o[m] = __dadd_rn(f, 0.0);
    }
    stvd<V>(rhs, p, o);
  }
}

// ---------------------------------------------------------------------------
// Marching forms of the assembly and the projection (nz % 4 == 0, no cut
// body, fewer than 2^31 cells). A thread owns a group of V consecutive
// cells of a row (V = 2 in both kernels: at 64 registers a thread four
// blocks share an SM, against two at V = 4). A block of 256 threads owns a
// tile of the (j, k) plane, TJ rows of V KQ cells (KQ threads a row,
// TJ = 256 / KQ), and walks it through LEN consecutive i planes, the
// previous plane in registers, without shared memory or barriers: the rows
// beside a thread's own (other threads' own rows) are read directly, from
// L1/L2, and the k neighbours come from the lanes around it. The
// assembly's coefficient of the face between planes i and i+1 is formed
// once, as the east face of i and the west face of i+1. Every value is the
// same operations in the same order as the one-cell kernels, so the outputs
// are bit for bit theirs.
// ---------------------------------------------------------------------------
constexpr int kMarchI = 8;  // planes a walk, at most
constexpr int kAsmV = 2;    // cells a thread, assembly
constexpr int kProjV = 2;   // cells a thread, projection

// threads a row: the smallest power of two with v KQ >= nz, at most 256 / v
inline int march_kq(int nz, int v) {
  int q = 1;
  while (q < kThreads / v && v * q < nz) q *= 2;
  return q;
}
// planes a walk: kMarchI, halved (down to 2) while the grid would hold
// fewer than four blocks an SM of a 148-SM GPU
inline int march_len(int nx, int ny, int nz, int v) {
  const int kq = march_kq(nz, v), tj = kThreads / kq;
  const long long tiles = (long long)((nz + v * kq - 1) / (v * kq)) * ((ny + tj - 1) / tj);
  int len = kMarchI;
  while (len > 2 && tiles * ((nx + len - 1) / len) < 4 * 148) len /= 2;
  return len;
}
inline dim3 march_grid(int nx, int ny, int nz, int v) {
  const int kq = march_kq(nz, v), tj = kThreads / kq, len = march_len(nx, ny, nz, v);
  return dim3((unsigned)((nz + v * kq - 1) / (v * kq)), (unsigned)((ny + tj - 1) / tj),
              (unsigned)((nx + len - 1) / len));
}
inline bool march_fits(int nx, int ny, int nz) {
  for (int v : {kAsmV, kProjV}) {
    const dim3 g = march_grid(nx, ny, nz, v);
    if (g.y > 65535u || g.z > 65535u) return false;
  }
  return true;
}

// hx / f for a face density f, with hx / ra and hx / rb formed once: away
// from an interface every interior face coefficient is one of the two (a
// division is deterministic, so the cached quotient is the same bits). A
// zero density never takes the cached quotient (-0 == +0 would pick the
// wrong sign of infinity).
struct QuotCache {
  double hx, ra, rb, qa, qb;
  QuotCache() = default;
  __host__ __device__ __forceinline__ QuotCache(double hx_, double ra_, double rb_) : hx(hx_), ra(ra_), rb(rb_) {
    qa = div_rn(hx_, ra_);
    qb = div_rn(hx_, rb_);
  }
  __device__ __forceinline__ double operator()(double f) const {
    if (f != 0.0) {
      if (f == ra) return qa;
      if (f == rb) return qb;
    }
    return __ddiv_rn(hx, f);
  }
};

// Cache-only quotients for the fast groups of the marching assembly: hx and
// hxb (the wall faces' numerator) over either pure-phase density. A face
// density that is neither (an interface face), or a zero density, sets
// miss and returns a placeholder.
struct QuotOnly {
  double ka, kb, qa, qb, qba, qbb;
  QuotOnly() = default;
  __host__ __device__ __forceinline__ QuotOnly(double hx, double hxb, double ra, double rb) {
    const double nan = quiet_nan();
    ka = ra != 0.0 ? ra : nan;
    kb = rb != 0.0 ? rb : nan;
    qa = div_rn(hx, ra);
    qb = div_rn(hx, rb);
    qba = div_rn(hxb, ra);
    qbb = div_rn(hxb, rb);
  }
  __device__ __forceinline__ double in(double f, bool &miss) const {
    const bool isa = f == ka;
    miss |= !(isa || f == kb);
    return isa ? qa : qb;
  }
  __device__ __forceinline__ double bnd(double f, bool &miss) const {
    const bool isa = f == ka;
    miss |= !(isa || f == kb);
    return isa ? qba : qbb;
  }
};

// Per-launch constants of the marching kernels, formed on the host with the
// same correctly rounded operations the one-cell kernels use (hx = h^2 / h;
// hxb = h^2 / (h / 2), the wall faces' numerator; the cached quotients and
// reciprocals). Passed as __grid_constant__ parameters, they are read from
// the constant bank rather than held in every thread's registers.
struct AsmConst {
  double hx, hxb;
  QuotCache Q;
  QuotOnly QC;
};
inline AsmConst asm_const(double h, double ra, double rb) {
  AsmConst K;
  const double hh = mul_rn(h, h);
  K.hx = div_rn(hh, h);
  K.hxb = div_rn(hh, mul_rn(0.5, h));
  K.Q = QuotCache(K.hx, ra, rb);
  K.QC = QuotOnly(K.hx, K.hxb, ra, rb);
  return K;
}
struct ProjConst {
  PhaseDiv D;
  ProjFast PF;
};
inline ProjConst proj_const(double ra, double rb, double h) {
  ProjConst K;
  K.D = PhaseDiv(ra, rb, h);
  K.PF = ProjFast(K.D);
  return K;
}

template <int V>
__global__ void __launch_bounds__(kThreads, V == 2 ? 4 : 2)
    km_assemble_mix(int nx, int ny, int nz, int KQ, int LEN, const __grid_constant__ AsmConst K, int4 bc03,
                    int2 bc45,
                    const double *__restrict__ col, double ra, double rb, const uint8_t *__restrict__ solid,
                    double *__restrict__ C, double *__restrict__ W, double *__restrict__ S,
                    double *__restrict__ B, uint8_t *__restrict__ aflag) {
  const int bc[6] = {bc03.x, bc03.y, bc03.z, bc03.w, bc45.x, bc45.y};
  const int TJ = kThreads / KQ;
  const int tx = (int)threadIdx.x % KQ, ty = (int)threadIdx.x / KQ;
  const int k = (int)blockIdx.x * V * KQ + V * tx, j = (int)blockIdx.y * TJ + ty;
  const int i0 = (int)blockIdx.z * LEN, i1 = min(nx, i0 + LEN);
  const bool own = j < ny && k < nz;
  const uint32_t SI = (uint32_t)ny * nz, SJ = (uint32_t)nz;
  const double &hxb = K.hxb;
  const bool hc = col != nullptr;
  const QuotCache &Q = K.Q;
  const QuotOnly &QC = K.QC;
  // the lanes before and after hold the row's previous and next groups
  const int lane = (int)threadIdx.x & 31;
  const bool kdn = lane > 0 && tx > 0, kup = lane < 31 && tx < KQ - 1;
  // the thread's own group of plane ip: mixture densities and solid flags
  auto stage = [&](int ip, double (&mq)[V], uint32_t &sq) {
    if (own) {
      const uint32_t p = (uint32_t)ip * SI + (uint32_t)j * SJ + (uint32_t)k;
      mixv<V>(col, ra, rb, p, mq);
      sq = solid ? ldvb<V>(solid, p) : 0u;
    }
  };
  double mC[V] = {}, mN[V] = {}, aW[V] = {};
  uint32_t sP = 0u, sC = 0u, sN = 0u;
  stage(i0, mC, sC);
  if (own && i0 > 0) {
    double mP[V];
    const uint32_t p = (uint32_t)(i0 - 1) * SI + (uint32_t)j * SJ + (uint32_t)k;
    mixv<V>(col, ra, rb, p, mP);
    sP = solid ? ldvb<V>(solid, p) : 0u;
#pragma unroll
    for (int m = 0; m < V; ++m) aW[m] = Q(face_of(hc, ra, mC[m], mP[m]));
  }
  for (int i = i0; i < i1; ++i) {
    if (i + 1 < nx) stage(i + 1, mN, sN);
    // the row's k neighbours from the lanes around, else read; the south
    // and north rows read directly
    double mkm = __shfl_up_sync(0xffffffffu, mC[V - 1], 1), mkp = __shfl_down_sync(0xffffffffu, mC[0], 1);
    unsigned skm_ = __shfl_up_sync(0xffffffffu, byte_at(sC, V - 1), 1), skp_ = __shfl_down_sync(0xffffffffu, byte_at(sC, 0), 1);
    if (own) {
      const uint32_t p = (uint32_t)i * SI + (uint32_t)j * SJ + (uint32_t)k;
      if (!kdn) { mkm = k > 0 ? mix1(col, ra, rb, (long long)p - 1) : 0.0; skm_ = (k > 0 && solid) ? solid[p - 1] : 0u; }
      if (!kup) { mkp = k + V < nz ? mix1(col, ra, rb, (long long)p + V) : 0.0; skp_ = (k + V < nz && solid) ? solid[p + V] : 0u; }
      if (k == 0) { mkm = 0.0; skm_ = 0u; }
      if (k + V >= nz) { mkp = 0.0; skp_ = 0u; }
      const uint8_t skm = (uint8_t)skm_, skp = (uint8_t)skp_;
      double mS[V] = {}, mNo[V] = {};
      uint32_t sS = 0u, sNo = 0u;
      if (j > 0) { mixv<V>(col, ra, rb, p - SJ, mS); if (solid) sS = ldvb<V>(solid, p - SJ); }
      if (j < ny - 1) { mixv<V>(col, ra, rb, p + SJ, mNo); if (solid) sNo = ldvb<V>(solid, p + SJ); }
      // A group away from the i and j walls whose cells and neighbours all
      // carry the same solid flag needs none of the wall and body rules but
      // the k walls' (a solid group only scales c by 1e-12 and drops its
      // couplings): the same values in far fewer instructions. Rows run
      // along k, so a warp's groups mostly agree on the branch.
      bool fast = i > 0 && i < nx - 1 && j > 0 && j < ny - 1;
      const uint32_t sp0 = byte_at(sC, 0);
      if (solid && fast) {
        const uint32_t wv = bytes_all<V>(sp0);
        bool same = sC == wv && sP == wv && sN == wv && sS == wv && sNo == wv && (k == 0 || skm == sp0) &&
                    (k + V == nz || skp == sp0);
        fast = same;
      }
      if (fast) {
        // the group with quotients from qin (interior faces) and qbnd (the k
        // walls' faces)
        double e[V], oc[V], ow[V], os[V], ob[V];
        auto group = [&](auto &&qin, auto &&qbnd) {
          double bfx[V + 1];
          bfx[0] = k == 0 ? qbnd(face_of(hc, ra, mC[0], mC[0])) : qin(face_of(hc, ra, mC[0], mkm));
#pragma unroll
          for (int m = 1; m < V; ++m) bfx[m] = qin(face_of(hc, ra, mC[m], mC[m - 1]));
          bfx[V] = k + V == nz ? qbnd(face_of(hc, ra, mC[V - 1], mC[V - 1])) : qin(face_of(hc, ra, mkp, mC[V - 1]));
#pragma unroll
          for (int m = 0; m < V; ++m) {
            const double a0 = aW[m];
            const double a1 = qin(face_of(hc, ra, mN[m], mC[m]));
            const double a2 = qin(face_of(hc, ra, mC[m], mS[m]));
            const double a3 = qin(face_of(hc, ra, mNo[m], mC[m]));
            double a4 = bfx[m];
            const double a5 = bfx[m + 1];
            double c = __dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(a0, a1), a2), a3), a4), a5);
            if (m == 0 && k == 0) {
              if (bc[4] == PBG_BC_NEUMANN_) { c = __dsub_rn(c, a4); a4 = 0.0; }
              else if (bc[4] == PBG_BC_DIRICHLET_) a4 = 0.0;
            }
            if (m == V - 1 && k + V == nz && bc[5] == PBG_BC_NEUMANN_) c = __dsub_rn(c, a5);
            e[m] = a1;
            if (sp0) {
              c = __dmul_rn(c, 1.0e-12);
              a4 = 0.0;
            }
            oc[m] = c; ow[m] = sp0 ? 0.0 : a0; os[m] = sp0 ? 0.0 : a2; ob[m] = a4;
          }
        };
        bool miss = false;
        group([&](double f) { return QC.in(f, miss); }, [&](double f) { return QC.bnd(f, miss); });
        // an interface face: the group again, dividing where the cache misses
        if (miss) group([&](double f) { return Q(f); }, [&](double f) { return __ddiv_rn(hxb, f); });
#pragma unroll
        for (int m = 0; m < V; ++m) aW[m] = e[m];
        stvd<V>(C, p, oc);
        stvd<V>(W, p, ow);
        stvd<V>(S, p, os);
        stvd<V>(B, p, ob);
        stvb<V>(aflag, p, bytes_all<V>(sp0 ? 0u : 1u));
      } else {
        double bf[V + 1];
        bf[0] = k == 0 ? __ddiv_rn(hxb, face_of(hc, ra, mC[0], mC[0])) : Q(face_of(hc, ra, mC[0], mkm));
#pragma unroll
        for (int m = 1; m < V; ++m) bf[m] = Q(face_of(hc, ra, mC[m], mC[m - 1]));
        bf[V] = k + V == nz ? __ddiv_rn(hxb, face_of(hc, ra, mC[V - 1], mC[V - 1])) : Q(face_of(hc, ra, mkp, mC[V - 1]));
        uint32_t af = 0u;
#pragma unroll
        for (int m = 0; m < V; ++m) {
          const int kk = k + m;
          const double ms_ = mS[m], mn_ = mNo[m];
          double a[6];
          a[0] = i > 0 ? aW[m] : __ddiv_rn(hxb, face_of(hc, ra, mC[m], mC[m]));
          a[1] = i < nx - 1 ? Q(face_of(hc, ra, mN[m], mC[m])) : __ddiv_rn(hxb, face_of(hc, ra, mC[m], mC[m]));
          aW[m] = a[1];  // the west face of the next plane's cell
          a[2] = j > 0 ? Q(face_of(hc, ra, mC[m], ms_)) : __ddiv_rn(hxb, face_of(hc, ra, mC[m], mC[m]));
          a[3] = j < ny - 1 ? Q(face_of(hc, ra, mn_, mC[m])) : __ddiv_rn(hxb, face_of(hc, ra, mC[m], mC[m]));
          a[4] = bf[m];
          a[5] = bf[m + 1];
          double c = a[0];
#pragma unroll
          for (int f = 1; f < 6; ++f) c = __dadd_rn(c, a[f]);
          const uint32_t sp = byte_at(sC, m);
          if (solid) {
            const uint32_t sbm = m > 0 ? byte_at(sC, m - 1) : skm, stp = m < V - 1 ? byte_at(sC, m + 1) : skp;
            if (i > 0 && byte_at(sP, m) != sp) a[0] = 0.0;
            if (i < nx - 1 && byte_at(sN, m) != sp) a[1] = 0.0;
            if (j > 0 && byte_at(sS, m) != sp) a[2] = 0.0;
            if (j < ny - 1 && byte_at(sNo, m) != sp) a[3] = 0.0;
            if (kk > 0 && sbm != sp) a[4] = 0.0;
            if (kk < nz - 1 && stp != sp) a[5] = 0.0;
            if (!sp) {
              c = a[0];
#pragma unroll
              for (int f = 1; f < 6; ++f) c = __dadd_rn(c, a[f]);
            }
          }
          const bool onb[6] = {i == 0, i == nx - 1, j == 0, j == ny - 1, kk == 0, kk == nz - 1};
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
          // one cell at a time (8-byte stores; a thread's cells fill whole
          // 16-byte pairs together) keeps the outputs out of registers
          C[p + m] = c;
          W[p + m] = a[0];
          S[p + m] = a[2];
          B[p + m] = a[4];
          af |= (sp ? 0u : 1u) << (8 * m);
        }
        stvb<V>(aflag, p, af);
      }
    }
    sP = sC;
    sC = sN;
#pragma unroll
    for (int m = 0; m < V; ++m) mC[m] = mN[m];
  }
}

// The projection's walk, without shared memory or barriers: the previous
// plane in registers, the south row (j - 1) read directly (from L1/L2: it is
// another thread's own row), the k - 1 neighbour from the previous lane when
// that lane holds the row's previous group, else read. Faces follow the
// one-cell kernel's rules and arithmetic:
//  * a group of solid cells updates no face at all;
//  * a group with all three lower neighbours inside the domain and no solid
//    cell in it or below it on any axis updates every face, both divisions
//    by Markstein's correction when every face density is a pure phase's;
//  * any other group (or one whose correction misses) takes the general
//    per-face rules with KnownDiv's divisions.
template <int V>
__global__ void __launch_bounds__(kThreads, V == 2 ? 4 : 2)
    km_project(int nx, int ny, int nz, int KQ, int LEN, const __grid_constant__ ProjConst K, double dt,
               const double *__restrict__ pr,
               const double *__restrict__ col, double ra, double rb, const uint8_t *__restrict__ solid,
               double *__restrict__ u, double *__restrict__ v, double *__restrict__ w) {
  const int TJ = kThreads / KQ;
  const int tx = (int)threadIdx.x % KQ, ty = (int)threadIdx.x / KQ, lane = (int)threadIdx.x & 31;
  const int k = (int)blockIdx.x * V * KQ + V * tx, j = (int)blockIdx.y * TJ + ty;
  const int i0 = (int)blockIdx.z * LEN, i1 = min(nx, i0 + LEN);
  const bool own = j < ny && k < nz;
  const uint32_t SI = (uint32_t)ny * nz, SJ = (uint32_t)nz;
  const bool body = solid != nullptr;
  const bool hc = col != nullptr;
  const PhaseDiv &D = K.D;
  const ProjFast &PF = K.PF;
  const bool kshfl = lane > 0 && tx > 0;  // the previous lane holds the group before
  double pP[V] = {}, mP[V] = {};
  uint32_t sP = 0u;
  if (own && i0 > 0) {
    const uint32_t p = (uint32_t)(i0 - 1) * SI + (uint32_t)j * SJ + (uint32_t)k;
    ldvd<V>(pr, p, pP);
    mixv<V>(col, ra, rb, p, mP);
    sP = body ? ldvb<V>(solid, p) : 0u;
  }
  for (int i = i0; i < i1; ++i) {
    const uint32_t p = (uint32_t)i * SI + (uint32_t)j * SJ + (uint32_t)k;
    double pC[V] = {}, mC[V] = {};
    double pS[V] = {}, mS[V] = {};
    uint32_t sC = 0u, sS = 0u;
    if (own) {
      ldvd<V>(pr, p, pC);
      mixv<V>(col, ra, rb, p, mC);
      if (body) sC = ldvb<V>(solid, p);
      if (j > 0) {
        ldvd<V>(pr, p - SJ, pS);
        mixv<V>(col, ra, rb, p - SJ, mS);
        if (body) sS = ldvb<V>(solid, p - SJ);
      }
    }
    double pk = __shfl_up_sync(0xffffffffu, pC[V - 1], 1);
    double mk = __shfl_up_sync(0xffffffffu, mC[V - 1], 1);
    unsigned sk = __shfl_up_sync(0xffffffffu, byte_at(sC, V - 1), 1);
    if (!kshfl && own && k > 0) {
      pk = pr[p - 1];
      mk = mix1(col, ra, rb, (long long)p - 1);
      sk = body ? solid[p - 1] : 0u;
    }
    bool fast = own && i > 0 && j > 0 && k > 0;
    bool skip = false;
    if (body && own) {
      skip = true;
#pragma unroll
      for (int m = 0; m < V; ++m) skip = skip && byte_at(sC, m) != 0u;
      if (fast) {
        const uint32_t any = sC | sP | sS | sk;
        fast = any == 0;
      }
    }
    if (skip) {
    } else if (fast) {
      const uint32_t iv = ((uint32_t)i * (ny + 1) + j) * nz + k;
      const long long iw = ((long long)i * ny + j) * (nz + 1) + k;
      bool miss = false;
      double uo[V], vo[V], wo[V];
      ldvd<V>(u, p, uo);
      ldvd<V>(v, iv, vo);
#pragma unroll
      for (int m = 0; m < V; ++m) wo[m] = w[iw + m];
#pragma unroll
      for (int m = 0; m < V; ++m) {
        uo[m] = __dadd_rn(uo[m], PF.inc(pP[m], pC[m], face_of(hc, ra, mC[m], mP[m]), dt, body, miss));
        vo[m] = __dadd_rn(vo[m], PF.inc(pS[m], pC[m], face_of(hc, ra, mC[m], mS[m]), dt, body, miss));
        const double pb = m > 0 ? pC[m - 1] : pk;
        const double mb = m > 0 ? mC[m - 1] : mk;
        wo[m] = __dadd_rn(wo[m], PF.inc(pb, pC[m], face_of(hc, ra, mC[m], mb), dt, body, miss));
      }
      if (!miss) {
        stvd<V>(u, p, uo);
        stvd<V>(v, iv, vo);
#pragma unroll
        for (int m = 0; m < V; ++m) w[iw + m] = wo[m];
      }
      fast = !miss;
    }
    if (!skip && !fast && own) {
      if (i > 0) {
        double uo[V];
        ldvd<V>(u, p, uo);
#pragma unroll
        for (int m = 0; m < V; ++m)
          if (!(body && (byte_at(sC, m) || byte_at(sP, m))))
            uo[m] = __dadd_rn(uo[m], project_increment_k(pP[m], pC[m], face_of(hc, ra, mC[m], mP[m]), dt, D, body));
        stvd<V>(u, p, uo);
      }
      if (j > 0) {
        const uint32_t iv = ((uint32_t)i * (ny + 1) + j) * nz + k;
        double vo[V];
        ldvd<V>(v, iv, vo);
#pragma unroll
        for (int m = 0; m < V; ++m)
          if (!(body && (byte_at(sC, m) || byte_at(sS, m))))
            vo[m] = __dadd_rn(vo[m], project_increment_k(pS[m], pC[m], face_of(hc, ra, mC[m], mS[m]), dt, D, body));
        stvd<V>(v, iv, vo);
      }
      if (nz > 1) {
        const long long iw = ((long long)i * ny + j) * (nz + 1) + k;
#pragma unroll
        for (int m = 0; m < V; ++m) {
          const int kk = k + m;
          if (kk == 0) continue;
          const unsigned sbm = m > 0 ? byte_at(sC, m - 1) : sk;
          if (body && (byte_at(sC, m) || sbm)) continue;
          const double pb = m > 0 ? pC[m - 1] : pk;
          const double mb = m > 0 ? mC[m - 1] : mk;
          w[iw + m] = __dadd_rn(w[iw + m], project_increment_k(pb, pC[m], face_of(hc, ra, mC[m], mb), dt, D, body));
        }
      }
    }
#pragma unroll
    for (int m = 0; m < V; ++m) {
      pP[m] = pC[m];
      mP[m] = mC[m];
    }
    sP = sC;
  }
}

}  // namespace pbg
