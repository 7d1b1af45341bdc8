// Bottom of the engine's K-cycle in one thread block, in shared memory.
//
// The coarse levels of the hierarchy are latency-bound: one K-cycle call at
// a level of a few thousand cells is ~40 dependent passes over tiny arrays.
// As separate kernel launches, or as passes over global memory, each pass
// costs about a microsecond of latency. k_bottom runs a whole kcycle(first)
// — its recursion down to the coarsest level and the dense coarsest solve —
// inside one 1024-thread block with every work vector (and every matrix
// below the first level, and the coarsest inverse) in shared memory, so a
// pass costs a shared-memory access plus __syncthreads(). The first level's
// right-hand side is read from global memory and its result is left in
// global memory as (z1, z2, a1, a2, beta), which the finer level's
// prolongation reads as e = (a1 - a2 beta) z1 + a2 z2. The arithmetic per
// cell is the same as the grid kernels'.
#pragma once

#include "pbg_engine_kernels.cuh"

namespace pbg {

constexpr int kBotThreads = 1024;
constexpr int kBotMaxLevels = 8;
constexpr size_t kBotSmemMax = 200 * 1024;   // dynamic shared memory budget
// Largest first level: one block keeps up with the launched kernels only on
// levels of a few hundred cells (a 4096-cell K-cycle call is ~10M thread
// instructions, about 150 us on one SM).
constexpr long long kBotMaxCells = 512;

template <typename T>
struct BotLevel {
  EMat<T> A;             // global arrays (copied to shared for levels > first)
  KScal *ks;             // global
  T *gb, *gz1, *gz2;     // global b / z1 / z2 (first level only)
  uint32_t off;          // byte offset of this level's shared block
  int smem_matrix;       // matrix copied to shared memory
};

template <typename T>
struct BotCtx {
  int first, last;
  BotLevel<T> L[kBotMaxLevels];
  const double *Ainv;    // dense inverse of the coarsest level (global)
  int ncoarse;
  uint32_t ainv_off;     // its shared copy
  size_t smem_bytes;
  T omega;
};

// shared bytes of one level: 7 vectors (+ 5 matrix arrays when copied)
template <typename T>
__host__ __device__ inline size_t bot_level_bytes(long long n, bool matrix) {
  size_t b = (size_t)n * sizeof(T) * (7 + (matrix ? 5 : 0));
  return (b + 15) & ~(size_t)15;
}

// sums of NV values over the block, returned to every thread
template <int NV>
__device__ __forceinline__ void bot_sum(double (&v)[NV]) {
  __shared__ double red[NV][kBotThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  warp_sum<NV>(v);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NV; ++q) red[q][wid] = v[q];
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += red[q][w];
    v[q] = s;
  }
}

#define BOT_LOOP(p, N) for (uint32_t p = threadIdx.x; p < (uint32_t)(N); p += blockDim.x)

// Work vectors of one level in shared memory.
template <typename T>
struct BotVec {
  T *b, *z1, *z2, *q1, *r1, *xa, *xb;
};

// Depth D = level - first is a template parameter: precond<D> calls
// kcycle<D+1>, so the call chain is bounded at compile time (no run-time
// recursion, a statically known stack).
template <typename T>
struct Bottom {
  const BotCtx<T> &C;
  char *sm;
  EMat<T> *A;      // per-level views, in shared memory (one copy per block)
  BotVec<T> *V;
  const double *Ainv;

  __device__ Bottom(const BotCtx<T> &c, char *smem, EMat<T> *a, BotVec<T> *v)
      : C(c), sm(smem), A(a), V(v) {
    Ainv = (const double *)(sm + C.ainv_off);
    if (threadIdx.x != 0) return;
    const int nl = C.last - C.first + 1;
    for (int d = 0; d < nl; ++d) {
      const BotLevel<T> &L = C.L[d];
      const size_t n = (size_t)L.A.g.n;
      T *base = (T *)(sm + L.off);
      V[d] = {base, base + n, base + 2 * n, base + 3 * n, base + 4 * n, base + 5 * n, base + 6 * n};
      A[d] = L.A;
      if (L.smem_matrix) {
        T *m = base + 7 * n;
        A[d].c = m; A[d].w = m + n; A[d].s = m + 2 * n; A[d].b = m + 3 * n; A[d].dinv = m + 4 * n;
      }
    }
  }

  // copy matrices, the coarsest inverse and the first level's rhs in
  __device__ void load() {
    const int nl = C.last - C.first + 1;
    for (int d = 0; d < nl; ++d) {
      const BotLevel<T> &L = C.L[d];
      if (!L.smem_matrix) continue;
      const uint32_t n = L.A.g.n;
      T *c = (T *)A[d].c, *w = (T *)A[d].w, *s = (T *)A[d].s, *b = (T *)A[d].b, *di = (T *)A[d].dinv;
      BOT_LOOP(p, n) {
        c[p] = L.A.c[p]; w[p] = L.A.w[p]; s[p] = L.A.s[p]; b[p] = L.A.b[p]; di[p] = L.A.dinv[p];
      }
    }
    double *ai = (double *)Ainv;
    BOT_LOOP(p, (uint32_t)(C.ncoarse * C.ncoarse)) ai[p] = C.Ainv[p];
    BOT_LOOP(p, C.L[0].A.g.n) V[0].b[p] = C.L[0].gb[p];
    __syncthreads();
  }

  __device__ void store() {
    BOT_LOOP(p, C.L[0].A.g.n) {
      C.L[0].gz1[p] = V[0].z1[p];
      C.L[0].gz2[p] = V[0].z2[p];
    }
  }

  // z = Ainv r on the coarsest level (FP64 inverse)
  __device__ void dense(const T *r, T *z) {
    const int n = C.ncoarse;
    for (int row = threadIdx.x; row < n; row += blockDim.x) {
      double acc = 0.0;
      for (int c = 0; c < n; ++c) acc += Ainv[row * n + c] * (double)r[c];
      z[row] = (T)acc;
    }
    __syncthreads();
  }

  // the level preconditioner M r -> z (kc: r = b - a1 q1, stored to r1)
  template <int D>
  __device__ __noinline__ void precond(const T *r, T *z, bool kc) {
    const int l = C.first + D;
    if (l == C.last) { dense(r, z); return; }
    const EMat<T> &M = A[D];
    const BotVec<T> &v = V[D];
    const T om = C.omega;
    const T a1 = kc ? (T)C.L[D].ks->a1 : T(0);
    const T *rr = kc ? v.r1 : r;
    // two sweeps from zero
    BOT_LOOP(p, M.g.n) {
      Pos q = M.g.pos(p);
      auto rv = [&](uint32_t s) -> T { return kc ? v.b[s] - a1 * v.q1[s] : r[s]; };
      auto x1 = [&](uint32_t s) -> T { return om * rv(s) * M.dinv[s]; };
      const T rp = rv(p), d = M.dinv[p], xp = om * rp * d;
      if (kc) v.r1[p] = rp;
      v.xb[p] = xp + om * ((rp + offdiag(M, p, q, x1)) * d - xp);
    }
    __syncthreads();
    // restriction of r - A x to the next level
    const EMat<T> &H = A[D + 1];
    const BotVec<T> &vh = V[D + 1];
    const int fx = M.nx > 1 ? 2 : 1, fy = M.ny > 1 ? 2 : 1, fz = M.nz > 1 ? 2 : 1;
    BOT_LOOP(P, H.g.n) {
      Pos Q = H.g.pos(P);
      T sum = 0;
      for (int a = 0; a < fx; ++a) {
        int i = Q.i * fx + a;
        if (i >= M.nx) break;
        for (int bb = 0; bb < fy; ++bb) {
          int j = Q.j * fy + bb;
          if (j >= M.ny) break;
          for (int cc = 0; cc < fz; ++cc) {
            int k = Q.k * fz + cc;
            if (k >= M.nz) break;
            uint32_t p = ((uint32_t)i * M.ny + j) * M.nz + k;
            sum += rr[p] - ax_at(M, p, Pos{i, j, k}, v.xb);
          }
        }
      }
      vh.b[P] = sum;
    }
    __syncthreads();
    const bool dense_next = (l + 1 == C.last);
    if (dense_next) dense(vh.b, vh.xa);
    else if constexpr (D + 1 < kBotMaxLevels - 1) kcycle<D + 1>();
    // prolongation + one sweep
    const int sx = M.nx > 1 ? 1 : 0, sy = M.ny > 1 ? 1 : 0, sz = M.nz > 1 ? 1 : 0;
    const uint32_t HnYZ = (uint32_t)H.ny * H.nz;
    T c1 = 1, c2 = 0;
    if (!dense_next) {
      const KScal *kh = C.L[D + 1].ks;
      c1 = (T)(kh->a1 - kh->a2 * kh->beta);
      c2 = (T)kh->a2;
    }
    auto e = [&](int i, int j, int k) -> T {
      const uint32_t P = (uint32_t)(i >> sx) * HnYZ + (uint32_t)(j >> sy) * H.nz + (uint32_t)(k >> sz);
      return dense_next ? vh.xa[P] : c1 * vh.z1[P] + c2 * vh.z2[P];
    };
    BOT_LOOP(p, M.g.n) {
      Pos q = M.g.pos(p);
      const uint32_t SI = M.g.nynz, SJ = (uint32_t)M.nz;
      T on = 0;
      if (q.i > 0) on += M.w[p] * (v.xb[p - SI] + e(q.i - 1, q.j, q.k));
      if (q.i < M.nx - 1) on += M.w[p + SI] * (v.xb[p + SI] + e(q.i + 1, q.j, q.k));
      if (q.j > 0) on += M.s[p] * (v.xb[p - SJ] + e(q.i, q.j - 1, q.k));
      if (q.j < M.ny - 1) on += M.s[p + SJ] * (v.xb[p + SJ] + e(q.i, q.j + 1, q.k));
      if (q.k > 0) on += M.b[p] * (v.xb[p - 1] + e(q.i, q.j, q.k - 1));
      if (q.k < M.nz - 1) on += M.b[p + 1] * (v.xb[p + 1] + e(q.i, q.j, q.k + 1));
      T xp = v.xb[p] + e(q.i, q.j, q.k);
      v.xa[p] = xp + om * ((rr[p] + on) * M.dinv[p] - xp);
    }
    __syncthreads();
    // last sweep
    BOT_LOOP(p, M.g.n) {
      Pos q = M.g.pos(p);
      const T on = offdiag(M, p, q, [&](uint32_t s) { return v.xa[s]; });
      const T xp = v.xa[p];
      z[p] = xp + om * ((rr[p] + on) * M.dinv[p] - xp);
    }
    __syncthreads();
  }

  // two flexible-CG steps on a level (same formulas as k_kc_q1 / k_kc_q2)
  template <int D>
  __device__ __noinline__ void kcycle() {
    const EMat<T> &M = A[D];
    const BotVec<T> &v = V[D];
    KScal *ks = C.L[D].ks;
    precond<D>(v.b, v.z1, false);
    double v2[2] = {0.0, 0.0};
    BOT_LOOP(p, M.g.n) {
      Pos q = M.g.pos(p);
      const T qq = ax_at(M, p, q, v.z1);
      v.q1[p] = qq;
      v2[0] += (double)v.z1[p] * (double)v.b[p];
      v2[1] += (double)v.z1[p] * (double)qq;
    }
    bot_sum<2>(v2);
    if (threadIdx.x == 0) {
      ks->zb = v2[0];
      ks->zq = v2[1];
      ks->a1 = (v2[1] > 0.0 && v2[1] == v2[1]) ? v2[0] / v2[1] : 0.0;
    }
    __syncthreads();
    precond<D>(nullptr, v.z2, true);
    double v3[3] = {0.0, 0.0, 0.0};
    BOT_LOOP(p, M.g.n) {
      Pos q = M.g.pos(p);
      const T av = ax_at(M, p, q, v.z2);
      const double zz = (double)v.z2[p];
      v3[0] += zz * (double)v.q1[p];
      v3[1] += zz * (double)v.r1[p];
      v3[2] += zz * (double)av;
    }
    bot_sum<3>(v3);
    if (threadIdx.x == 0) {
      const double zq = ks->zq;
      const double beta = zq > 0.0 ? v3[0] / zq : 0.0;
      const double z1r1 = ks->zb - ks->a1 * zq;
      const double pr = v3[1] - beta * z1r1;
      const double pq = v3[2] - 2.0 * beta * v3[0] + beta * beta * zq;
      ks->beta = beta;
      ks->a2 = (pq > 0.0 && pq == pq && pr == pr) ? pr / pq : 0.0;
    }
    __syncthreads();
  }
};

// The level table lives in device memory (written once per work set).
template <typename T>
__global__ void __launch_bounds__(kBotThreads, 1) k_bottom(const BotCtx<T> *__restrict__ ctx,
                                                           const int *stop) {
  extern __shared__ __align__(16) char bot_smem[];
  // raw storage (the view types have constructors, which shared variables
  // do not run; thread 0 fills them)
  __shared__ __align__(16) char views_raw[sizeof(EMat<T>) * kBotMaxLevels];
  __shared__ __align__(16) char vecs_raw[sizeof(BotVec<T>) * kBotMaxLevels];
  if (stop && *stop) return;
  Bottom<T> B(*ctx, bot_smem, reinterpret_cast<EMat<T> *>(views_raw),
              reinterpret_cast<BotVec<T> *>(vecs_raw));
  __syncthreads();
  B.load();
  B.template kcycle<0>();
  B.store();
}

}  // namespace pbg
