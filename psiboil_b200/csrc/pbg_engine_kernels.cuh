// Engine kernels: flexible CG preconditioned by an additive-correction
// (piecewise-constant aggregation, Galerkin coarse operator) K-cycle.
// Templated on the storage/arithmetic type T (double for the plain FP64
// path, float inside the mixed-precision refinement); every global sum is
// accumulated in double.
//
// Matrices are symmetric 7-point operators stored as c, w, s, b; the east,
// north and top coefficients of cell p are w, s, b of the next cell in that
// direction (zero on the last plane).
#pragma once
#include "pbg_engine.cuh"

namespace pbg {

// Off-diagonal part sum_nb a_nb x_nb of cell p (x given by a functor).
template <typename T, typename XF>
__device__ __forceinline__ T offdiag(const EMat<T> &A, uint32_t p, Pos q, XF x) {
  const uint32_t SI = A.g.nynz, SJ = (uint32_t)A.nz;
  T v = 0;
  if (q.i > 0) v += A.w[p] * x(p - SI);
  if (q.i < A.nx - 1) v += A.w[p + SI] * x(p + SI);
  if (q.j > 0) v += A.s[p] * x(p - SJ);
  if (q.j < A.ny - 1) v += A.s[p + SJ] * x(p + SJ);
  if (q.k > 0) v += A.b[p] * x(p - 1);
  if (q.k < A.nz - 1) v += A.b[p + 1] * x(p + 1);
  return v;
}

// Storage of the diagonal. FP64 operators keep c: (A x)_p = c x_p -
// sum_nb a_nb x_nb. FP32 operators keep the diagonal excess d = c - sum_nb
// a_nb (rounded once from FP64) and apply the edge form
//   (A x)_p = d x_p + sum_nb a_nb (x_p - x_nb).
// Rounding the couplings of the edge form to FP32 perturbs A by a relative
// 2^-24 in the energy norm, whatever its condition number; rounding c does
// not (its small row sums are lost), which would limit every FP32 inner
// solve of the mixed refinement to a reduction of about 2^-24 x cond(A).
template <typename T>
constexpr bool kEdgeForm = sizeof(T) == 4;

// (A x)_p with x given by a functor
template <typename T, typename XF>
__device__ __forceinline__ T ax_f(const EMat<T> &A, uint32_t p, Pos q, XF x) {
  if constexpr (kEdgeForm<T>) {
    const T xp = x(p);
    return A.c[p] * xp + offdiag(A, p, q, [&](uint32_t s) { return xp - x(s); });
  } else {
    return A.c[p] * x(p) - offdiag(A, p, q, x);
  }
}

template <typename T>
__device__ __forceinline__ T ax_at(const EMat<T> &A, uint32_t p, Pos q, const T *__restrict__ x) {
  return ax_f(A, p, q, [&](uint32_t s) { return x[s]; });
}

#define GRID_LOOP(p, N)                                                       \
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < (uint32_t)(N); \
       p += gridDim.x * blockDim.x)

// ---------------------------------------------------------------- smoothers
// Damped Jacobi with the stored inverse diagonal:
//   x' = x + w (D^-1 (r + sum_nb a_nb x_nb) - x)   (= x + w D^-1 (r - A x))

// x = w D^-1 r   (first sweep from a zero guess)
template <typename T>
__global__ void __launch_bounds__(kThreads, 8) k_jac0(EMat<T> A, const T *__restrict__ r, T *__restrict__ x, T omega,
                       const int *stop) {
  PBG_PDL_ENTRY();
  if (stop && *stop) return;
  GRID_LOOP(p, A.g.n) x[p] = omega * r[p] * A.dinv[p];
}

template <typename T>
__global__ void __launch_bounds__(kThreads, 8) k_jac(EMat<T> A, const T *__restrict__ r, const T *__restrict__ xi,
                      T *__restrict__ xo, T omega, const int *stop) {
  PBG_PDL_ENTRY();
  if (stop && *stop) return;
  GRID_LOOP(p, A.g.n) {
    Pos q = A.g.pos(p);
    T on = offdiag(A, p, q, [&](uint32_t s) { return xi[s]; });
    T xp = xi[p];
    xo[p] = xp + omega * ((r[p] + on) * A.dinv[p] - xp);
  }
}

// Two damped-Jacobi sweeps from a zero guess in one pass:
//   x1 = w D^-1 r;  x2 = x1 + w (D^-1 (r + sum_nb a_nb x1_nb) - x1)
// with x1 at the neighbours formed from r and D^-1 there. When ks is set the
// right-hand side is the K-cycle residual r = b2 - a1 q2, formed on the fly
// and stored to r_out for the later passes of the same cycle.
template <typename T>
__global__ void __launch_bounds__(kThreads, 8)
    k_jac2(EMat<T> A, const T *__restrict__ r, const T *__restrict__ b2, const T *__restrict__ q2,
           const KScal *ks, T *__restrict__ r_out, T *__restrict__ xo, T omega, const int *stop) {
  PBG_PDL_ENTRY();
  if (stop && *stop) return;
  const T a1 = ks ? (T)ks->a1 : T(0);
  auto rv = [&](uint32_t s) -> T { return ks ? b2[s] - a1 * q2[s] : r[s]; };
  auto x1 = [&](uint32_t s) -> T { return omega * rv(s) * A.dinv[s]; };
  GRID_LOOP(p, A.g.n) {
    Pos q = A.g.pos(p);
    const T rp = rv(p);
    if (ks) r_out[p] = rp;
    const T d = A.dinv[p];
    const T xp = omega * rp * d;
    const T on = offdiag(A, p, q, x1);
    xo[p] = xp + omega * ((rp + on) * d - xp);
  }
}

// Restriction by the transpose of piecewise-constant prolongation: the
// coarse rhs is the block sum of the fine residual r - A x. Eight lanes per
// coarse cell, one per child (a, b, c) of its 2x2x2 block; absent children
// (unit extents, odd edges) add zero; the eight are summed by shuffles in a
// fixed order. t = 8 * coarse cell + child.
template <typename T>
__device__ __forceinline__ T restrict_child(const EMat<T> &A, const T *r, const T *x, const Geo &H, uint32_t t) {
  const int fx = A.nx > 1 ? 2 : 1, fy = A.ny > 1 ? 2 : 1, fz = A.nz > 1 ? 2 : 1;
  const uint32_t c = t & 7u;
  const int a = (int)(c >> 2), bb = (int)((c >> 1) & 1u), cc = (int)(c & 1u);
  if (a >= fx || bb >= fy || cc >= fz) return T(0);
  const Pos Q = H.pos(t >> 3);
  const int i = Q.i * fx + a, j = Q.j * fy + bb, k = Q.k * fz + cc;
  if (i >= A.nx || j >= A.ny || k >= A.nz) return T(0);
  const uint32_t p = ((uint32_t)i * A.ny + j) * A.nz + k;
  return r[p] - ax_at(A, p, Pos{i, j, k}, x);
}

// Sum over the eight lanes of a coarse cell (every lane of the warp must
// take part); lane (t & 7) == 0 holds the result.
template <typename T>
__device__ __forceinline__ T sum8(T v) {
  v += __shfl_xor_sync(0xffffffffu, v, 1);
  v += __shfl_xor_sync(0xffffffffu, v, 2);
  v += __shfl_xor_sync(0xffffffffu, v, 4);
  return v;
}

// One thread per coarse cell, children summed in (a, b, c) order. On large
// levels this reads better (consecutive threads take fine cells two apart
// in k) than eight lanes per coarse cell, which spread one warp's load over
// eight rows; the eight-lane form is for small levels, where one thread per
// coarse cell would leave most of the GPU idle.
constexpr uint32_t kRestrictSerialMin = 32768;  // coarse cells

template <typename T>
__device__ __forceinline__ T restrict_cell(const EMat<T> &A, const T *r, const T *x, const Geo &H, uint32_t P) {
  const int fx = A.nx > 1 ? 2 : 1, fy = A.ny > 1 ? 2 : 1, fz = A.nz > 1 ? 2 : 1;
  const Pos Q = H.pos(P);
  T sum = 0;
  for (int a = 0; a < fx; ++a) {
    const int i = Q.i * fx + a;
    if (i >= A.nx) break;
    for (int bb = 0; bb < fy; ++bb) {
      const int j = Q.j * fy + bb;
      if (j >= A.ny) break;
      for (int cc = 0; cc < fz; ++cc) {
        const int k = Q.k * fz + cc;
        if (k >= A.nz) break;
        const uint32_t p = ((uint32_t)i * A.ny + j) * A.nz + k;
        sum += r[p] - ax_at(A, p, Pos{i, j, k}, x);
      }
    }
  }
  return sum;
}

template <typename T>
__global__ void __launch_bounds__(kThreads, 8) k_resid_restrict(EMat<T> A, const T *__restrict__ r, const T *__restrict__ x,
                                 Geo H, T *__restrict__ rH, const int *stop) {
  PBG_PDL_ENTRY();
  if (stop && *stop) return;
  if (H.n >= kRestrictSerialMin) {
    GRID_LOOP(P, H.n) rH[P] = restrict_cell(A, r, x, H, P);
    return;
  }
  const uint32_t total = H.n * 8u;
  // warp-uniform trip count: every lane reaches the shuffles
  for (uint32_t base = blockIdx.x * blockDim.x; base < total; base += gridDim.x * blockDim.x) {
    const uint32_t t = base + threadIdx.x;
    const bool valid = t < total;
    T v = valid ? restrict_child(A, r, x, H, t) : T(0);
    v = sum8(v);
    if (valid && (t & 7u) == 0u) rH[t >> 3] = v;
  }
}

// x' = xi + P e (prolongation of the coarse correction), then one sweep.
// e is the coarse array eH, or — after a K-cycle — e = c1 z1H + c2 z2H with
// c1 = a1 - a2 beta, c2 = a2 from the coarse level's scalars ksH.
template <typename T>
__global__ void __launch_bounds__(kThreads, 8)
    k_prolong_jac(EMat<T> A, const T *__restrict__ r, const T *__restrict__ xi, int Hny, int Hnz,
                  const T *__restrict__ eH, const T *__restrict__ z2H, const KScal *ksH,
                  T *__restrict__ xo, T omega, const int *stop) {
  PBG_PDL_ENTRY();
  if (stop && *stop) return;
  const int sx = A.nx > 1 ? 1 : 0, sy = A.ny > 1 ? 1 : 0, sz = A.nz > 1 ? 1 : 0;
  const uint32_t HnYZ = (uint32_t)Hny * Hnz;
  T c1 = 1, c2 = 0;
  if (ksH) { c1 = (T)(ksH->a1 - ksH->a2 * ksH->beta); c2 = (T)ksH->a2; }
  auto e = [&](int i, int j, int k) -> T {
    const uint32_t P = (uint32_t)(i >> sx) * HnYZ + (uint32_t)(j >> sy) * Hnz + (uint32_t)(k >> sz);
    return ksH ? c1 * eH[P] + c2 * z2H[P] : eH[P];
  };
  GRID_LOOP(p, A.g.n) {
    Pos q = A.g.pos(p);
    const uint32_t SI = A.g.nynz, SJ = (uint32_t)A.nz;
    T on = 0;
    if (q.i > 0) on += A.w[p] * (xi[p - SI] + e(q.i - 1, q.j, q.k));
    if (q.i < A.nx - 1) on += A.w[p + SI] * (xi[p + SI] + e(q.i + 1, q.j, q.k));
    if (q.j > 0) on += A.s[p] * (xi[p - SJ] + e(q.i, q.j - 1, q.k));
    if (q.j < A.ny - 1) on += A.s[p + SJ] * (xi[p + SJ] + e(q.i, q.j + 1, q.k));
    if (q.k > 0) on += A.b[p] * (xi[p - 1] + e(q.i, q.j, q.k - 1));
    if (q.k < A.nz - 1) on += A.b[p + 1] * (xi[p + 1] + e(q.i, q.j, q.k + 1));
    T xp = xi[p] + e(q.i, q.j, q.k);
    xo[p] = xp + omega * ((r[p] + on) * A.dinv[p] - xp);
  }
}

// Last post-smoothing sweep of a preconditioner application with fused dot
// products for the Krylov step that consumes z:  d0 = z.r, d1 = z.u
template <typename T>
__global__ void __launch_bounds__(kThreads, 8) k_jac_dots(EMat<T> A, const T *__restrict__ r, const T *__restrict__ xi,
                           T *__restrict__ z, T omega, const T *__restrict__ u, double *out2,
                           double *part, unsigned *count, const int *stop) {
  PBG_PDL_ENTRY();
  if (stop && *stop) return;
  double v[2] = {0.0, 0.0};
  GRID_LOOP(p, A.g.n) {
    Pos q = A.g.pos(p);
    T on = offdiag(A, p, q, [&](uint32_t s) { return xi[s]; });
    T xp = xi[p];
    T zz = xp + omega * ((r[p] + on) * A.dinv[p] - xp);
    z[p] = zz;
    v[0] += (double)zz * (double)r[p];
    if (u) v[1] += (double)zz * (double)u[p];
  }
  double o[2];
  if (grid_reduce<2>(v, part, count, o)) { out2[0] = o[0]; out2[1] = o[1]; }
}

// ---------------------------------------------------------------- K-cycle
// Two flexible-CG steps on a coarse level (Notay's K-cycle), with the
// level's own cycle as the preconditioner:
//   z1 = M b; q1 = A z1; a1 = z1.b / z1.q1; r1 = b - a1 q1
//   z2 = M r1; v = A z2; beta = z2.q1 / z1.q1; p2 = z2 - beta z1
//   a2 = p2.r1 / p2.q2;  x = a1 z1 + a2 p2
// p2.q2 = z2.v - 2 beta z2.q1 + beta^2 z1.q1 and z1.r1 = z1.b - a1 z1.q1
// use the symmetry of A, so that q2 is never formed.
template <typename T>
__global__ void __launch_bounds__(kThreads, 8) k_kc_q1(EMat<T> A, const T *__restrict__ z1, const T *__restrict__ b,
                        T *__restrict__ q1, KScal *ks, double *part, unsigned *count,
                        const int *stop) {
  PBG_PDL_ENTRY();
  if (stop && *stop) return;
  double v[2] = {0.0, 0.0};
  GRID_LOOP(p, A.g.n) {
    Pos q = A.g.pos(p);
    T qq = ax_at(A, p, q, z1);
    q1[p] = qq;
    v[0] += (double)z1[p] * (double)b[p];
    v[1] += (double)z1[p] * (double)qq;
  }
  double o[2];
  if (grid_reduce<2>(v, part, count, o)) {
    ks->zb = o[0];
    ks->zq = o[1];
    ks->a1 = (o[1] > 0.0 && o[1] == o[1]) ? o[0] / o[1] : 0.0;
  }
}

template <typename T>
__global__ void __launch_bounds__(kThreads, 8) k_kc_r1(long long N, const T *__restrict__ b, const T *__restrict__ q1,
                        T *__restrict__ r1, const KScal *ks, const int *stop) {
  PBG_PDL_ENTRY();
  if (stop && *stop) return;
  const T a1 = (T)ks->a1;
  GRID_LOOP(p, N) r1[p] = b[p] - a1 * q1[p];
}

template <typename T>
__global__ void __launch_bounds__(kThreads, 8) k_kc_q2(EMat<T> A, const T *__restrict__ z2, const T *__restrict__ q1,
                        const T *__restrict__ r1, T *__restrict__ vv, KScal *ks, double *part,
                        unsigned *count, const int *stop) {
  PBG_PDL_ENTRY();
  if (stop && *stop) return;
  double v[3] = {0.0, 0.0, 0.0};
  GRID_LOOP(p, A.g.n) {
    Pos q = A.g.pos(p);
    T av = ax_at(A, p, q, z2);
    vv[p] = av;
    double zz = (double)z2[p];
    v[0] += zz * (double)q1[p];
    v[1] += zz * (double)r1[p];
    v[2] += zz * (double)av;
  }
  double o[3];
  if (grid_reduce<3>(v, part, count, o)) {
    const double zq = ks->zq;
    double beta = zq > 0.0 ? o[0] / zq : 0.0;
    double z1r1 = ks->zb - ks->a1 * zq;
    double pr = o[1] - beta * z1r1;
    double pq = o[2] - 2.0 * beta * o[0] + beta * beta * zq;
    double a2 = (pq > 0.0 && pq == pq && pr == pr) ? pr / pq : 0.0;
    ks->beta = beta;
    ks->a2 = a2;
  }
}

template <typename T>
__global__ void __launch_bounds__(kThreads, 8) k_kc_x(long long N, const T *__restrict__ z1, const T *__restrict__ z2,
                       T *__restrict__ x, const KScal *ks, const int *stop) {
  PBG_PDL_ENTRY();
  if (stop && *stop) return;
  const T c1 = (T)(ks->a1 - ks->a2 * ks->beta), c2 = (T)ks->a2;
  GRID_LOOP(p, N) x[p] = c1 * z1[p] + c2 * z2[p];
}

// Coarsest level: z = Ainv r with the dense inverse (FP64, or its FP32
// copy in the mixed path), one warp per row, FP64 sums.
template <typename T, typename AT>
__global__ void k_dense_solve(int n, const AT *__restrict__ Ainv, const T *__restrict__ r,
                              T *__restrict__ z, const int *stop) {
  PBG_PDL_ENTRY();
  if (stop && *stop) return;
  const int lane = threadIdx.x & 31;
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (row >= n) return;
  double acc = 0.0;
  for (int c = lane; c < n; c += 32) acc += (double)Ainv[(long long)row * n + c] * (double)r[c];
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
  if (lane == 0) z[row] = (T)acc;
}

// ---------------------------------------------------------------- outer FCG
// Flexible CG with one-vector orthogonalisation (FCG(1)):
//   beta = z.q_old / p_old.q_old;  p = z - beta p_old;  q = A p
//   alpha = p.r / p.q;  x += alpha p;  r -= alpha q
// p.r = z.r - beta p_old.r, with z.r and z.q_old from the last smoothing
// sweep (k_jac_dots) and p_old.r from the previous update (k_fcg_xr).
// p is double-buffered by iteration parity; each thread forms p at its
// neighbours from z and p_old.
template <typename T>
__global__ void __launch_bounds__(kThreads, 8) k_fcg_pq(EMat<T> A, const T *__restrict__ z, T *pA, T *pB, T *__restrict__ qv,
                         FcgScal *fs, double *part, unsigned *count) {
  PBG_PDL_ENTRY();
  if (fs->done) return;
  const int it = fs->iter;
  const T *pold = (it & 1) ? pB : pA;
  T *pnew = (it & 1) ? pA : pB;
  const double betad = (it == 0 || !(fs->pq > 0.0)) ? 0.0 : fs->zq / fs->pq;
  const T beta = (T)betad;
  auto pv = [&](uint32_t s) -> T { return it == 0 ? z[s] : z[s] - beta * pold[s]; };
  double v[1] = {0.0};
  GRID_LOOP(p, A.g.n) {
    Pos q = A.g.pos(p);
    T pp = pv(p);
    T qq = ax_f(A, p, q, pv);
    pnew[p] = pp;
    qv[p] = qq;
    v[0] += (double)pp * (double)qq;
  }
  double o[1];
  if (grid_reduce<1>(v, part, count, o)) {
    double pr = fs->zr - betad * (it == 0 ? 0.0 : fs->pr);
    fs->beta = betad;
    fs->pq = o[0];
    fs->alpha = (o[0] > 0.0 && o[0] == o[0]) ? pr / o[0] : 0.0;
    if (!(o[0] > 0.0) || !(o[0] == o[0])) { fs->done = 1; fs->status = ST_BREAKDOWN; }
  }
}

template <typename T>
__global__ void __launch_bounds__(kThreads, 8) k_fcg_xr(long long N, T *__restrict__ x, T *__restrict__ r, const T *pA,
                         const T *pB, const T *__restrict__ qv, FcgScal *fs,
                         double *part, unsigned *count) {
  PBG_PDL_ENTRY();
  if (fs->done) return;
  const int it = fs->iter;
  const T *pp = (it & 1) ? pA : pB;
  const T alpha = (T)fs->alpha;
  double v[2] = {0.0, 0.0};
  GRID_LOOP(p, N) {
    T pv = pp[p];
    x[p] += alpha * pv;
    T rv = r[p] - alpha * qv[p];
    r[p] = rv;
    v[0] += (double)rv * (double)rv;
    v[1] += (double)pv * (double)rv;
  }
  double o[2];
  if (grid_reduce<2>(v, part, count, o)) {
    fs->rr = o[0];
    fs->pr = o[1];
    double rel = sqrt(o[0] / fs->rr0);
    if (fs->hist && it < kHistMax) fs->hist[it] = rel;
    fs->iter = it + 1;
    if (rel <= fs->tol) { fs->done = 1; fs->converged = 1; fs->status = ST_CONVERGED; }
    else if (!(rel == rel)) { fs->done = 1; fs->status = ST_NAN; }
    else if (it + 1 >= fs->maxit) { fs->done = 1; fs->status = ST_MAXITER; }
  }
}

// r = b, x = 0 (T), rr0 = |b|^2; fs set up for a new solve
template <typename T>
__global__ void __launch_bounds__(kThreads, 8) k_fcg_init(long long N, const T *__restrict__ b, T *__restrict__ x,
                           T *__restrict__ r, FcgScal *fs, double tol, int maxit, double *hist,
                           double *part, unsigned *count) {
  PBG_PDL_ENTRY();
  double v[1] = {0.0};
  GRID_LOOP(p, N) {
    T bv = b[p];
    r[p] = bv;
    x[p] = 0;
    v[0] += (double)bv * (double)bv;
  }
  double o[1];
  if (grid_reduce<1>(v, part, count, o)) {
    fs->rr0 = o[0];
    fs->rr = o[0];
    fs->hist = hist;
    fs->tol = tol;
    fs->maxit = maxit;
    fs->iter = 0;
    fs->loops = 0;
    fs->pq = 0.0;
    fs->pr = 0.0;
    fs->zq = 0.0;
    fs->zr = 0.0;
    fs->converged = 0;
    if (!(o[0] > 0.0)) { fs->done = 1; fs->converged = 1; fs->status = ST_INITIAL; }
    else if (maxit <= 0) { fs->done = 1; fs->status = ST_MAXITER; }
    else { fs->done = 0; fs->status = ST_RUNNING; }
  }
}

// ---------------------------------------------------------------- refinement
// x64 += e (T), elementwise
template <typename T>
__global__ void __launch_bounds__(kThreads, 8) k_add_corr(long long N, double *__restrict__ x, const T *__restrict__ e) {
  PBG_PDL_ENTRY();
  GRID_LOOP(p, N) x[p] += (double)e[p];
}

// r = b - A x in FP64, r32 = (T) r, out[0] = |r|^2, out[1] = |b|^2
template <typename T>
__global__ void __launch_bounds__(kThreads, 8) k_true_resid(EMat<double> A, const double *__restrict__ x, const double *__restrict__ b,
                             double *__restrict__ r, T *__restrict__ rT, double *out, double *part,
                             unsigned *count) {
  PBG_PDL_ENTRY();
  double v[2] = {0.0, 0.0};
  GRID_LOOP(p, A.g.n) {
    Pos q = A.g.pos(p);
    double rv = b[p] - ax_at(A, p, q, x);
    if (r) r[p] = rv;
    if (rT) rT[p] = (T)rv;
    v[0] += rv * rv;
    v[1] += b[p] * b[p];
  }
  double o[2];
  if (grid_reduce<2>(v, part, count, o)) { out[0] = o[0]; out[1] = o[1]; }
}

// The same for a non-symmetric operator in the seven-array form (a cut
// body's pressure matrix), which the engine solves by refinement around
// its symmetric part: r = b - (c x - sum a_nb x_nb).
template <typename T>
__global__ void __launch_bounds__(kThreads, 8) k_true_resid_ns(MatView<double> A, Geo G, const double *__restrict__ x,
                                const double *__restrict__ b, double *__restrict__ r,
                                T *__restrict__ rT, double *out, double *part, unsigned *count) {
  PBG_PDL_ENTRY();
  const uint32_t SI = G.nynz, SJ = (uint32_t)A.nz;
  double v[2] = {0.0, 0.0};
  GRID_LOOP(p, G.n) {
    const Pos q = G.pos(p);
    const Nb<double> a = coeffs(A, p, q);
    double nb = 0.0;
    if (q.i > 0) nb += a.w * x[p - SI];
    if (q.i < A.nx - 1) nb += a.e * x[p + SI];
    if (q.j > 0) nb += a.s * x[p - SJ];
    if (q.j < A.ny - 1) nb += a.n * x[p + SJ];
    if (q.k > 0) nb += a.b * x[p - 1];
    if (q.k < A.nz - 1) nb += a.t * x[p + 1];
    const double rv = b[p] - (A.c[p] * x[p] - nb);
    if (r) r[p] = rv;
    if (rT) rT[p] = (T)rv;
    v[0] += rv * rv;
    v[1] += b[p] * b[p];
  }
  double o[2];
  if (grid_reduce<2>(v, part, count, o)) { out[0] = o[0]; out[1] = o[1]; }
}

// ---------------------------------------------------------------- hierarchy
// Galerkin coarse operator P^T A P for piecewise-constant aggregation by 2
// in every direction with more than one cell (last block partial on odd
// sizes): c_H = sum c - 2 sum(internal couplings), w_H / s_H / b_H = sum of
// the couplings across the block's west / south / bottom face.
}  // namespace pbg
