// Vectorised fine-level kernels: each thread owns V consecutive cells of one
// k-row (V = 4 in FP32 with float4 loads, V = 2 in FP64 with double2), so
// every array is read with 16-byte loads, the cell position is computed once
// per V cells and the k-neighbours come from the same vector (plus one
// scalar at each end). Used when nz % V == 0 (16-byte alignment of every
// row start follows from cudaMalloc's 256-byte alignment); the scalar
// kernels cover every other shape. Per-cell arithmetic equals the scalar
// kernels' (same formulas, same operation order).
#pragma once

#include "pbg_engine_kernels.cuh"

namespace pbg {

template <typename T> struct VecTraits;
template <> struct VecTraits<float> { static constexpr int V = 4; using W = float4; };
template <> struct VecTraits<double> { static constexpr int V = 2; using W = double2; };

template <typename T>
struct Vec {
  T v[VecTraits<T>::V];
};

template <typename T>
__device__ __forceinline__ Vec<T> ldv(const T *__restrict__ a, uint32_t p) {
  using W = typename VecTraits<T>::W;
  W w = *reinterpret_cast<const W *>(a + p);
  Vec<T> r;
  if constexpr (VecTraits<T>::V == 4) { r.v[0] = w.x; r.v[1] = w.y; r.v[2] = w.z; r.v[3] = w.w; }
  else { r.v[0] = w.x; r.v[1] = w.y; }
  return r;
}

template <typename T>
__device__ __forceinline__ void stv(T *__restrict__ a, uint32_t p, const Vec<T> &r) {
  using W = typename VecTraits<T>::W;
  W w;
  if constexpr (VecTraits<T>::V == 4) { w.x = r.v[0]; w.y = r.v[1]; w.z = r.v[2]; w.w = r.v[3]; }
  else { w.x = r.v[0]; w.y = r.v[1]; }
  *reinterpret_cast<W *>(a + p) = w;
}

template <typename T>
__device__ __forceinline__ Vec<T> zerov() {
  Vec<T> r;
#pragma unroll
  for (int m = 0; m < VecTraits<T>::V; ++m) r.v[m] = T(0);
  return r;
}

// Coefficients around V cells starting at p (row position q).
template <typename T>
struct CoefV {
  Vec<T> w, we, s, sn, b;
  T bk;   // b of the cell after the group (its coupling to the group's last cell)
};

template <typename T>
__device__ __forceinline__ CoefV<T> load_coef(const EMat<T> &A, uint32_t p, Pos q) {
  constexpr int V = VecTraits<T>::V;
  const uint32_t SI = A.g.nynz, SJ = (uint32_t)A.nz;
  CoefV<T> C;
  C.w = ldv(A.w, p);
  C.we = q.i < A.nx - 1 ? ldv(A.w, p + SI) : zerov<T>();
  C.s = ldv(A.s, p);
  C.sn = q.j < A.ny - 1 ? ldv(A.s, p + SJ) : zerov<T>();
  C.b = ldv(A.b, p);
  C.bk = q.k + V < A.nz ? A.b[p + V] : T(0);
  return C;
}

// A field around V cells: centre vector, the four lateral vectors and the
// scalars before/after the group along k (zero outside the domain). F is a
// functor with vec(p) -> Vec<T> (aligned) and one(p) -> T.
template <typename T>
struct HoodV {
  Vec<T> c, w, e, s, n;
  T km, kp;
};

template <typename T, typename F>
__device__ __forceinline__ HoodV<T> load_hood(const EMat<T> &A, uint32_t p, Pos q, F f) {
  constexpr int V = VecTraits<T>::V;
  const uint32_t SI = A.g.nynz, SJ = (uint32_t)A.nz;
  HoodV<T> H;
  H.c = f.vec(p);
  H.w = q.i > 0 ? f.vec(p - SI) : zerov<T>();
  H.e = q.i < A.nx - 1 ? f.vec(p + SI) : zerov<T>();
  H.s = q.j > 0 ? f.vec(p - SJ) : zerov<T>();
  H.n = q.j < A.ny - 1 ? f.vec(p + SJ) : zerov<T>();
  H.km = q.k > 0 ? f.one(p - 1) : T(0);
  H.kp = q.k + V < A.nz ? f.one(p + V) : T(0);
  return H;
}

// sum_nb a_nb x_nb of lane m, in the scalar kernels' order (w, e, s, n, b, t)
template <typename T>
__device__ __forceinline__ T offd(const CoefV<T> &C, const HoodV<T> &X, int m) {
  constexpr int V = VecTraits<T>::V;
  const T xl = m > 0 ? X.c.v[m - 1] : X.km;
  const T xr = m < V - 1 ? X.c.v[m + 1] : X.kp;
  const T bt = m < V - 1 ? C.b.v[m + 1] : C.bk;
  T v = 0;
  v += C.w.v[m] * X.w.v[m];
  v += C.we.v[m] * X.e.v[m];
  v += C.s.v[m] * X.s.v[m];
  v += C.sn.v[m] * X.n.v[m];
  v += C.b.v[m] * xl;
  v += bt * xr;
  return v;
}

// field accessors
template <typename T>
struct FArr {
  const T *a;
  __device__ Vec<T> vec(uint32_t p) const { return ldv(a, p); }
  __device__ T one(uint32_t p) const { return a[p]; }
};
// w * r * dinv (the first Jacobi sweep from zero)
template <typename T>
struct FJac0 {
  const T *r, *d;
  T om;
  __device__ Vec<T> vec(uint32_t p) const {
    Vec<T> a = ldv(r, p), b = ldv(d, p);
#pragma unroll
    for (int m = 0; m < VecTraits<T>::V; ++m) a.v[m] = om * a.v[m] * b.v[m];
    return a;
  }
  __device__ T one(uint32_t p) const { return om * r[p] * d[p]; }
};
// b2 - a1 q2 (the K-cycle's second right-hand side)
template <typename T>
struct FKc {
  const T *b, *q;
  T a1;
  __device__ Vec<T> vec(uint32_t p) const {
    Vec<T> x = ldv(b, p), y = ldv(q, p);
#pragma unroll
    for (int m = 0; m < VecTraits<T>::V; ++m) x.v[m] = x.v[m] - a1 * y.v[m];
    return x;
  }
  __device__ T one(uint32_t p) const { return b[p] - a1 * q[p]; }
};
template <typename T>
struct FJac0Kc {
  FKc<T> r;
  const T *d;
  T om;
  __device__ Vec<T> vec(uint32_t p) const {
    Vec<T> a = r.vec(p), b = ldv(d, p);
#pragma unroll
    for (int m = 0; m < VecTraits<T>::V; ++m) a.v[m] = om * a.v[m] * b.v[m];
    return a;
  }
  __device__ T one(uint32_t p) const { return om * r.one(p) * d[p]; }
};

// one wave of the 64-register vector kernels: 4 blocks of 256 per SM
constexpr int kVecBlocks = 148 * 4;
// blocks an SM of the two-sweep and FCG direction kernels: their float4
// neighbourhoods (FP32) need up to 80 registers a thread, which at four
// blocks an SM (64) would spill to local memory, so FP32 runs three; FP64
// (double2) keeps four
template <typename T> constexpr int kVecWideSm = sizeof(T) == 4 ? 3 : 4;
template <typename T> constexpr int kVecWideBlocks = 148 * kVecWideSm<T>;

#define VGRID_LOOP(g, NG)                                                       \
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < (uint32_t)(NG); \
       g += gridDim.x * blockDim.x)

// two sweeps from zero (k_jac2)
template <typename T>
__global__ void __launch_bounds__(kThreads, kVecWideSm<T>)
    kv_jac2(EMat<T> A, const T *__restrict__ r, const T *__restrict__ b2, const T *__restrict__ q2,
            const KScal *ks, T *__restrict__ r_out, T *__restrict__ xo, T omega, const int *stop) {
  PBG_PDL_ENTRY();
  if (stop && *stop) return;
  constexpr int V = VecTraits<T>::V;
  const T a1 = ks ? (T)ks->a1 : T(0);
  VGRID_LOOP(gi, A.g.n / V) {
    const uint32_t p = gi * V;
    const Pos q = A.g.pos(p);
    const CoefV<T> C = load_coef(A, p, q);
    const Vec<T> d = ldv(A.dinv, p);
    HoodV<T> X;
    Vec<T> rp;
    if (ks) {
      FKc<T> fr{b2, q2, a1};
      rp = fr.vec(p);
      X = load_hood(A, p, q, FJac0Kc<T>{fr, A.dinv, omega});
      stv(r_out, p, rp);
    } else {
      rp = ldv(r, p);
      X = load_hood(A, p, q, FJac0<T>{r, A.dinv, omega});
    }
    Vec<T> o;
#pragma unroll
    for (int m = 0; m < V; ++m) {
      const T xp = X.c.v[m];
      o.v[m] = xp + omega * ((rp.v[m] + offd(C, X, m)) * d.v[m] - xp);
    }
    stv(xo, p, o);
  }
}

// one sweep: xo = xi + w (D^-1 (r + sum a x) - xi), optional dots z.r, z.u
// With usel set, u is the q of the previous FCG iteration: uB when the
// current iteration number is odd, uA when it is even.
template <typename T, bool DOTS>
__global__ void __launch_bounds__(kThreads, 4)
    kv_jac(EMat<T> A, const T *__restrict__ r, const T *__restrict__ xi, T *__restrict__ xo, T omega,
           const T *uA, const T *uB, const FcgScal *usel, double *out2, double *part,
           unsigned *count, const int *stop) {
  PBG_PDL_ENTRY();
  if (stop && *stop) return;
  constexpr int V = VecTraits<T>::V;
  const T *u = (usel && (usel->iter & 1)) ? uB : uA;
  double acc[2] = {0.0, 0.0};
  VGRID_LOOP(gi, A.g.n / V) {
    const uint32_t p = gi * V;
    const Pos q = A.g.pos(p);
    const CoefV<T> C = load_coef(A, p, q);
    const Vec<T> d = ldv(A.dinv, p), rp = ldv(r, p);
    const HoodV<T> X = load_hood(A, p, q, FArr<T>{xi});
    Vec<T> o;
#pragma unroll
    for (int m = 0; m < V; ++m) {
      const T xp = X.c.v[m];
      o.v[m] = xp + omega * ((rp.v[m] + offd(C, X, m)) * d.v[m] - xp);
    }
    stv(xo, p, o);
    if constexpr (DOTS) {
      const Vec<T> uu = u ? ldv(u, p) : zerov<T>();
#pragma unroll
      for (int m = 0; m < V; ++m) {
        acc[0] += (double)o.v[m] * (double)rp.v[m];
        acc[1] += (double)o.v[m] * (double)uu.v[m];
      }
    }
  }
  if constexpr (DOTS) {
    double o2[2];
    if (grid_reduce<2>(acc, part, count, o2)) { out2[0] = o2[0]; out2[1] = o2[1]; }
  }
}

// prolongation of the coarse correction + one sweep. The coarse index of
// lanes m is ((i>>sx), (j>>sy), (k+m)>>sz); with sz = 1 and V even the
// group's parents are V/2 consecutive coarse cells.
template <typename T>
__global__ void __launch_bounds__(kThreads, 4)
    kv_prolong_jac(EMat<T> A, const T *__restrict__ r, const T *__restrict__ xi, int Hny, int Hnz,
                   const T *__restrict__ eH, const T *__restrict__ z2H, const KScal *ksH,
                   T *__restrict__ xo, T omega, const int *stop) {
  PBG_PDL_ENTRY();
  if (stop && *stop) return;
  constexpr int V = VecTraits<T>::V;
  const int sx = A.nx > 1 ? 1 : 0, sy = A.ny > 1 ? 1 : 0;
  const uint32_t HnYZ = (uint32_t)Hny * Hnz;
  T c1 = 1, c2 = 0;
  if (ksH) { c1 = (T)(ksH->a1 - ksH->a2 * ksH->beta); c2 = (T)ksH->a2; }
  auto e = [&](uint32_t P) -> T { return ksH ? c1 * eH[P] + c2 * z2H[P] : eH[P]; };
  // x + P e around the group: lane m's parent along k is (k+m)>>1 (nz > 1 here)
  VGRID_LOOP(gi, A.g.n / V) {
    const uint32_t p = gi * V;
    const Pos q = A.g.pos(p);
    auto parent = [&](int i, int j, int k) -> uint32_t {
      return (uint32_t)(i >> sx) * HnYZ + (uint32_t)(j >> sy) * Hnz + (uint32_t)(k >> 1);
    };
    auto rowv = [&](uint32_t pp, int i, int j) -> Vec<T> {
      Vec<T> x = ldv(xi, pp);
#pragma unroll
      for (int m = 0; m < V; ++m) x.v[m] += e(parent(i, j, q.k + m));
      return x;
    };
    const uint32_t SI = A.g.nynz, SJ = (uint32_t)A.nz;
    HoodV<T> X;
    X.c = rowv(p, q.i, q.j);
    X.w = q.i > 0 ? rowv(p - SI, q.i - 1, q.j) : zerov<T>();
    X.e = q.i < A.nx - 1 ? rowv(p + SI, q.i + 1, q.j) : zerov<T>();
    X.s = q.j > 0 ? rowv(p - SJ, q.i, q.j - 1) : zerov<T>();
    X.n = q.j < A.ny - 1 ? rowv(p + SJ, q.i, q.j + 1) : zerov<T>();
    X.km = q.k > 0 ? xi[p - 1] + e(parent(q.i, q.j, q.k - 1)) : T(0);
    X.kp = q.k + V < A.nz ? xi[p + V] + e(parent(q.i, q.j, q.k + V)) : T(0);
    const CoefV<T> C = load_coef(A, p, q);
    const Vec<T> d = ldv(A.dinv, p), rp = ldv(r, p);
    Vec<T> o;
#pragma unroll
    for (int m = 0; m < V; ++m) {
      const T xp = X.c.v[m];
      o.v[m] = xp + omega * ((rp.v[m] + offd(C, X, m)) * d.v[m] - xp);
    }
    stv(xo, p, o);
  }
}

// (A x)_m of lane m
template <typename T>
__device__ __forceinline__ T axv(const T c, const CoefV<T> &C, const HoodV<T> &X, int m) {
  if constexpr (kEdgeForm<T>) {  // c holds the diagonal excess (ax_f)
    constexpr int V = VecTraits<T>::V;
    const T xp = X.c.v[m];
    const T xl = m > 0 ? X.c.v[m - 1] : X.km;
    const T xr = m < V - 1 ? X.c.v[m + 1] : X.kp;
    const T bt = m < V - 1 ? C.b.v[m + 1] : C.bk;
    T v = 0;
    v += C.w.v[m] * (xp - X.w.v[m]);
    v += C.we.v[m] * (xp - X.e.v[m]);
    v += C.s.v[m] * (xp - X.s.v[m]);
    v += C.sn.v[m] * (xp - X.n.v[m]);
    v += C.b.v[m] * (xp - xl);
    v += bt * (xp - xr);
    return c * xp + v;
  } else {
    return c * X.c.v[m] - offd(C, X, m);
  }
}

// FCG direction: p = z - beta p_old, q = A z - beta q_old (A p = A z - beta
// A p_old), p.q. Reads z at the stencil, p_old and q_old once per cell.
template <typename T>
__global__ void __launch_bounds__(kThreads, kVecWideSm<T>)
    kv_fcg_pq(EMat<T> A, const T *__restrict__ z, T *pA, T *pB, T *qA, T *qB, FcgScal *fs,
              double *part, unsigned *count) {
  PBG_PDL_ENTRY();
  if (fs->done) return;
  constexpr int V = VecTraits<T>::V;
  const int it = fs->iter;
  const T *pold = (it & 1) ? pB : pA;
  T *pnew = (it & 1) ? pA : pB;
  const T *qold = (it & 1) ? qB : qA;
  T *qnew = (it & 1) ? qA : qB;
  const double betad = (it == 0 || !(fs->pq > 0.0)) ? 0.0 : fs->zq / fs->pq;
  const T beta = (T)betad;
  double acc[1] = {0.0};
  VGRID_LOOP(gi, A.g.n / V) {
    const uint32_t p = gi * V;
    const Pos q = A.g.pos(p);
    const CoefV<T> C = load_coef(A, p, q);
    const Vec<T> c = ldv(A.c, p);
    const HoodV<T> Z = load_hood(A, p, q, FArr<T>{z});
    Vec<T> pv, qv;
    if (it == 0) {
#pragma unroll
      for (int m = 0; m < V; ++m) { pv.v[m] = Z.c.v[m]; qv.v[m] = axv(c.v[m], C, Z, m); }
    } else {
      const Vec<T> po = ldv(pold, p), qo = ldv(qold, p);
#pragma unroll
      for (int m = 0; m < V; ++m) {
        pv.v[m] = Z.c.v[m] - beta * po.v[m];
        qv.v[m] = axv(c.v[m], C, Z, m) - beta * qo.v[m];
      }
    }
    stv(pnew, p, pv);
    stv(qnew, p, qv);
#pragma unroll
    for (int m = 0; m < V; ++m) acc[0] += (double)pv.v[m] * (double)qv.v[m];
  }
  double o[1];
  if (grid_reduce<1>(acc, part, count, o)) {
    double pr = fs->zr - betad * (it == 0 ? 0.0 : fs->pr);
    fs->beta = betad;
    fs->pq = o[0];
    fs->alpha = (o[0] > 0.0 && o[0] == o[0]) ? pr / o[0] : 0.0;
    if (!(o[0] > 0.0) || !(o[0] == o[0])) { fs->done = 1; fs->status = ST_BREAKDOWN; }
  }
}

// x += alpha p, r -= alpha q, |r|^2, p.r (p, q: the buffers kv_fcg_pq wrote)
template <typename T>
__global__ void __launch_bounds__(kThreads, 4)
    kv_fcg_xr(long long N, T *__restrict__ x, T *__restrict__ r, const T *pA, const T *pB,
              const T *qA, const T *qB, FcgScal *fs, double *part, unsigned *count) {
  PBG_PDL_ENTRY();
  if (fs->done) return;
  constexpr int V = VecTraits<T>::V;
  const int it = fs->iter;
  const T *pp = (it & 1) ? pA : pB;
  const T *qq = (it & 1) ? qA : qB;
  const T alpha = (T)fs->alpha;
  double acc[2] = {0.0, 0.0};
  VGRID_LOOP(gi, (uint32_t)(N / V)) {
    const uint32_t p = gi * V;
    Vec<T> xv = ldv(x, p), rv = ldv(r, p);
    const Vec<T> pv = ldv(pp, p), qv = ldv(qq, p);
#pragma unroll
    for (int m = 0; m < V; ++m) {
      xv.v[m] += alpha * pv.v[m];
      rv.v[m] = rv.v[m] - alpha * qv.v[m];
      acc[0] += (double)rv.v[m] * (double)rv.v[m];
      acc[1] += (double)pv.v[m] * (double)rv.v[m];
    }
    stv(x, p, xv);
    stv(r, p, rv);
  }
  double o[2];
  if (grid_reduce<2>(acc, part, count, o)) {
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

}  // namespace pbg
