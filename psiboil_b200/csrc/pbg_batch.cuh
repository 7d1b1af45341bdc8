// Batched engine, device side: many independent pressure problems of
// uneven sizes (2-D and 3-D) solved together, each in a "slot".
//
// Work layout: every level of every occupied slot is cut into tiles of a
// fixed number of cells; the tiles of all slots for level l form one flat
// list (a contiguous range of the tile array). Every kernel below runs a
// fixed grid that strides over the tile list of one level and processes the
// cells of each tile, so one launch does the same phase for every problem,
// whatever its size. The launch sequence of one outer iteration (captured
// once as a CUDA graph) is that of the deepest hierarchy in the batch;
// problems whose hierarchy ends earlier take their dense solve where it
// ends and skip the deeper launches (per-slot filters at the top of each
// tile).
//
// Per-problem state lives on the device (BState): an outer FP64 refinement
// state machine (INIT -> RUN -> DONE) around the inner flexible CG in T.
// Every decision of a slot is taken by the last tile of that slot to finish
// a reduction, after all of the slot's tiles in that launch are done, so a
// tile never sees its slot's state change during a launch.
//
// Reductions are per slot and deterministic: each tile writes a block
// partial to its own entry, and the slot's last-arriving tile sums the
// slot's partials in a fixed order (b_reduce). A problem's tiles, and so
// every bit of its result, do not depend on which other problems share the
// batch.
//
// Algorithm (per problem) = the engine's (pbg_engine_kernels.cuh): FCG(1)
// on the finest level, preconditioned by the AC K-cycle (piecewise-constant
// aggregation by 2, Galerkin coarse operators, damped Jacobi with two fused
// pre-sweeps and two post-sweeps, two FCG steps per coarse level up to
// kc_max, one visit below), dense inverse on the coarsest level; FP64 true
// residual and correction in the outer loop.
#pragma once
#include <cstdint>

#include "pbg_assemble.cuh"
#include "pbg_engine.cuh"
#include "pbg_engine_kernels.cuh"
#include "pbg_vec.cuh"

namespace pbg {

constexpr int kBMaxLev = 12;    // levels per problem
constexpr int kBDenseMax = 64;  // cells of the coarsest level (dense inverse in shared memory)
constexpr int kBThreadsMax = 512;

enum BPhase { BP_IDLE = 0, BP_INIT = 1, BP_RUN = 2, BP_DONE = 3 };

// One level of a problem.
template <typename T>
struct BLev {
  EMat<T> A;                              // operator in T (c, w, s, b, dinv)
  double *c64, *w64, *s64, *b64;          // FP64 operator (level 0: the assembled matrix)
  T *b, *x, *z1, *z2, *q1, *r1, *xa, *xb;
};

// Level 0 of a mixed-precision (FP32) batch keeps its inner-solve arrays in
// padded rows: the fast axis (k in 3-D; j in 2-D, whose rows are relabelled
// (nx, 1, ny)) is rounded up to a multiple of 4 cells, so that every group
// of four cells is one 16-byte vector and the row neighbours are aligned
// vectors too. Pad cells hold zero coefficients, zero inverse diagonal and
// zero vectors, and every kernel leaves them zero; the FP64 arrays of level
// 0 (matrix, solution, right-hand side, fields) stay compact.
template <typename T>
constexpr bool kBPad = sizeof(T) == 4;

// Device descriptor of the problem in a slot (written by the host).
template <typename T>
struct BProb {
  int nlev, ncoarse;
  int tail;                 // first level run by the CTA-local tail (kBMaxLev: none)
  int nx, ny, nz;
  int F, nzp, rel2d;        // padded level 0: fast-axis extent, padded extent, 2-D relabelled
  Geo g0;                   // compact level-0 geometry (the FP64 arrays)
  int bc[6];
  double h;
  const double *rho;        // assembly inputs (device) or null: level-0 FP64 matrix given
  const uint8_t *solid;
  double *x;                // FP64 solution (in: initial guess, out: result)
  const double *b;          // FP64 right-hand side
  double *Ainv;             // ncoarse x ncoarse
  T *x0, *r0, *z0, *pA, *pB, *q0;
  BLev<T> L[kBMaxLev];
};

// Per-slot solver state (device). Read back by the host after a solve.
struct BState {
  int phase, setup;         // BPhase; setup: hierarchy (re)computation requested
  int sweeps, iters, status, converged;
  int max_sweeps, maxit, inner_maxit, mixed;
  double tol, inner_tol, bb, rel, rel0;
  FcgScal f;                // inner flexible CG (f.done: inner solve finished)
  KScal ks[kBMaxLev];
};

struct BTile {
  int slot;
  uint32_t p0, n;           // cells [p0, p0 + n) of the slot's level
};

// Everything a batch kernel needs (device pointers), passed by value.
template <typename T>
struct BCtx {
  const BProb<T> *prob;     // [S]
  BState *st;               // [S]
  const BTile *tiles;       // all levels
  const int *lbeg;          // [kBMaxLev + 1]: tiles of level l are [lbeg[l], lbeg[l+1])
  const int *tbeg, *tcnt;   // [kBMaxLev * S]: first tile and tile count of (level, slot)
  double *part;             // [tiles * 4] per-tile partial sums
  unsigned *cnt;            // [kBMaxLev * S] arrival counters (zero between launches)
  int S;
  int kc_max;               // levels 1..kc_max run a K-cycle, deeper ones one visit
  T omega;
};

// Tiles of level l, grid-strided, with the next tile's record loaded one
// iteration ahead: a CTA's chain of dependent descriptor loads (tile ->
// slot state and problem -> arrays) then starts from a record already in
// registers. `continue` in the body moves to the next tile.
#define BTILE_FOR(C, l, t, tl)                                                                     \
  for (int t = (C).lbeg[l] + (int)blockIdx.x, e_##t = (C).lbeg[(l) + 1]; t < e_##t; t = e_##t)   \
    for (BTile tl = (C).tiles[t], n_##t = tl; t < e_##t; t += (int)gridDim.x, tl = n_##t)          \
      if (n_##t = t + (int)gridDim.x < e_##t ? (C).tiles[t + (int)gridDim.x] : tl, true)
#define BCELL_LOOP(T_, p) for (uint32_t p = (T_).p0 + threadIdx.x; p < (T_).p0 + (T_).n; p += blockDim.x)

// Is slot s running its inner solve (this launch's work applies)?
__device__ __forceinline__ bool b_running(const BState &S) { return S.phase == BP_RUN && !S.f.done; }

// Padded level-0 index -> compact index of the FP64 arrays; false for a pad
// cell. Without padding the index is the same.
template <typename T>
__device__ __forceinline__ bool b_compact(const BProb<T> &P, uint32_t pp, uint32_t &p) {
  if constexpr (!kBPad<T>) {
    p = pp;
    return true;
  } else {
    const uint32_t row = P.L[0].A.g.dnz.div(pp), k = pp - row * (uint32_t)P.nzp;
    if (k >= (uint32_t)P.F) return false;
    p = row * (uint32_t)P.F + k;
    return true;
  }
}

// Kernels with a padded level-0 path: at most 64 registers, so that 512-thread
// CTAs keep two per SM (the vector path would otherwise take up to 90).
#define BPAD_BOUNDS __launch_bounds__(kBThreadsMax, 2)

// Groups of four cells of a padded level-0 tile (tiles start at multiples of
// four and hold a multiple of four cells).
#define BGROUP_LOOP(T_, p)                                                          \
  for (uint32_t g_ = threadIdx.x, p = (T_).p0 + 4u * threadIdx.x; g_ < (T_).n / 4u; \
       g_ += blockDim.x, p = (T_).p0 + 4u * g_)

// Block sum of v[0..K-1] in a fixed order (warp shuffles, then warps in
// index order); the result is valid on thread 0. Ends with the CTA
// synchronised, so sm can be reused at once.
template <int K>
__device__ __forceinline__ void b_block_sum(double (&v)[K], double (*sm)[kBThreadsMax / 32]) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  warp_sum<K>(v);
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < K; ++q) sm[q][wid] = v[q];
  __syncthreads();
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < K; ++q) {
      double s = 0.0;
      for (int w = 0; w < nw; ++w) s += sm[q][w];
      v[q] = s;
    }
  __syncthreads();
}

// Per-slot segmented reduction of K values. Every tile of the slot writes
// its block sum; the slot's last-arriving tile then sums the slot's tile
// partials with the whole CTA (thread t takes tiles t, t + blockDim, ... in
// order, then the fixed block order). The grouping depends only on the
// slot's own tile count, so the bits do not depend on the other slots.
// Returns true on thread 0 of that last tile, with out = the slot's sums.
// Called by every thread of the CTA (it synchronises the CTA).
template <int K, typename T>
__device__ bool b_reduce(const BCtx<T> &C, int l, int t, int slot, double (&v)[K], double (&out)[K]) {
  __shared__ double sm[K][kBThreadsMax / 32];
  __shared__ int last;
  b_block_sum<K>(v, sm);
  const int key = l * C.S + slot;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < K; ++q) C.part[(size_t)t * 4 + q] = v[q];
    __threadfence();
    const unsigned prev = atomicAdd(&C.cnt[key], 1u);
    last = prev == (unsigned)C.tcnt[key] - 1u;
  }
  __syncthreads();
  const int is_last = last;
  __syncthreads();  // `last` may be rewritten by this CTA's next tile
  if (!is_last) return false;
  __threadfence();
  const int tb = C.tbeg[key], tn = C.tcnt[key];
  double acc[K];
#pragma unroll
  for (int q = 0; q < K; ++q) acc[q] = 0.0;
  for (int e = threadIdx.x; e < tn; e += blockDim.x)
#pragma unroll
    for (int q = 0; q < K; ++q) acc[q] += __ldcg(&C.part[(size_t)(tb + e) * 4 + q]);
  b_block_sum<K>(acc, sm);
  if (threadIdx.x != 0) return false;
#pragma unroll
  for (int q = 0; q < K; ++q) out[q] = acc[q];
  C.cnt[key] = 0u;
  return true;
}

// ---------------------------------------------------------------- set-up
// Level 0 of flagged slots: assemble the FP64 matrix from the fields (or
// keep the uploaded one).
template <typename T>
__global__ void kb_assemble(BCtx<T> C) {
  BTILE_FOR(C, 0, t, tl) {
    if (!C.st[tl.slot].setup) continue;
    const BProb<T> &P = C.prob[tl.slot];
    if (!P.rho) continue;
    const BLev<T> &V = P.L[0];
    BCELL_LOOP(tl, pp) {
      uint32_t p;
      if (!b_compact(P, pp, p)) continue;
      double c, w, s, b;
      const Pos q = P.g0.pos(p);
      assemble_cell(P.nx, P.ny, P.nz, P.h, P.bc, P.rho, P.solid, (long long)p, q, c, w, s, b);
      V.c64[p] = c; V.w64[p] = w; V.s64[p] = s; V.b64[p] = b;
    }
  }
}

// Level l >= 1 of flagged slots: Galerkin operator from level l-1 (as
// k_galerkin), FP64.
template <typename T>
__global__ void kb_galerkin(BCtx<T> C, int l) {
  BTILE_FOR(C, l, t, tl) {
    if (!C.st[tl.slot].setup) continue;
    const BProb<T> &P = C.prob[tl.slot];
    const BLev<T> &F = P.L[l - 1], &V = P.L[l];
    // the fine FP64 arrays: level 0's are compact even when its T arrays are padded
    const Geo Fg = l == 1 ? P.g0 : F.A.g;
    const int fx = Fg.nx > 1 ? 2 : 1, fy = Fg.ny > 1 ? 2 : 1, fz = Fg.nz > 1 ? 2 : 1;
    BCELL_LOOP(tl, P_) {
      Pos Q = V.A.g.pos(P_);
      double c = 0.0, w = 0.0, s = 0.0, b = 0.0;
      const int i0 = Q.i * fx, j0 = Q.j * fy, k0 = Q.k * fz;
      for (int a = 0; a < fx && i0 + a < Fg.nx; ++a)
        for (int bb = 0; bb < fy && j0 + bb < Fg.ny; ++bb)
          for (int cc = 0; cc < fz && k0 + cc < Fg.nz; ++cc) {
            const uint32_t p = ((uint32_t)(i0 + a) * Fg.ny + (j0 + bb)) * Fg.nz + (k0 + cc);
            c += F.c64[p];
            if (a == 0) w += F.w64[p]; else c -= 2.0 * F.w64[p];
            if (bb == 0) s += F.s64[p]; else c -= 2.0 * F.s64[p];
            if (cc == 0) b += F.b64[p]; else c -= 2.0 * F.b64[p];
          }
      V.c64[P_] = c; V.w64[P_] = w; V.s64[P_] = s; V.b64[P_] = b;
    }
  }
}

// Level l of flagged slots: inverse diagonal, and the operator in T (FP32:
// edge form with the diagonal excess, see kEdgeForm; FP64: the level's own
// arrays).
template <typename T>
__global__ void kb_finish(BCtx<T> C, int l) {
  if constexpr (kBPad<T>) {
    if (l == 0) {
      // padded level 0: compact FP64 in, padded T out (2-D: the j coupling
      // goes to the fast axis, b); pad cells keep their zeros
      BTILE_FOR(C, 0, t, tl) {
        if (!C.st[tl.slot].setup) continue;
        const BProb<T> &P = C.prob[tl.slot];
        const BLev<T> &V = P.L[0];
        const Geo &G = P.g0;
        const uint32_t SI = G.nynz, SJ = (uint32_t)G.nz;
        BCELL_LOOP(tl, pp) {
          uint32_t p;
          if (!b_compact(P, pp, p)) continue;
          const double c = V.c64[p];
          const Pos q = G.pos(p);
          double sum = 0.0;
          if (q.i > 0) sum += V.w64[p];
          if (q.i < G.nx - 1) sum += V.w64[p + SI];
          if (q.j > 0) sum += V.s64[p];
          if (q.j < G.ny - 1) sum += V.s64[p + SJ];
          if (q.k > 0) sum += V.b64[p];
          if (q.k < G.nz - 1) sum += V.b64[p + 1];
          const_cast<T *>(V.A.dinv)[pp] = (T)(1.0 / c);
          const_cast<T *>(V.A.c)[pp] = (T)(c - sum);
          const_cast<T *>(V.A.w)[pp] = (T)V.w64[p];
          const_cast<T *>(V.A.s)[pp] = P.rel2d ? T(0) : (T)V.s64[p];
          const_cast<T *>(V.A.b)[pp] = P.rel2d ? (T)V.s64[p] : (T)V.b64[p];
        }
      }
      return;
    }
  }
  BTILE_FOR(C, l, t, tl) {
    if (!C.st[tl.slot].setup) continue;
    const BLev<T> &V = C.prob[tl.slot].L[l];
    const EMat<T> &A = V.A;
    const uint32_t SI = A.g.nynz, SJ = (uint32_t)A.nz;
    T *dinv = const_cast<T *>(A.dinv);
    BCELL_LOOP(tl, p) {
      const double c = V.c64[p];
      dinv[p] = (T)(1.0 / c);
      if constexpr (kEdgeForm<T>) {
        const Pos q = A.g.pos(p);
        double sum = 0.0;
        if (q.i > 0) sum += V.w64[p];
        if (q.i < A.nx - 1) sum += V.w64[p + SI];
        if (q.j > 0) sum += V.s64[p];
        if (q.j < A.ny - 1) sum += V.s64[p + SJ];
        if (q.k > 0) sum += V.b64[p];
        if (q.k < A.nz - 1) sum += V.b64[p + 1];
        const_cast<T *>(A.c)[p] = (T)(c - sum);
        const_cast<T *>(A.w)[p] = (T)V.w64[p];
        const_cast<T *>(A.s)[p] = (T)V.s64[p];
        const_cast<T *>(A.b)[p] = (T)V.b64[p];
      }
    }
  }
}

// Dense inverse of every flagged slot's coarsest operator: one CTA per
// slot, Gauss-Jordan in shared memory (the same exchange steps and pivot
// skip as k_gj_block), then the setup flag is cleared.
template <typename T>
__global__ void kb_dense_inverse(BCtx<T> C, double rel_tol) {
  __shared__ double D[kBDenseMax][kBDenseMax + 1];
  __shared__ double rowk[kBDenseMax], colk[kBDenseMax];
  __shared__ double dmax;
  for (int slot = blockIdx.x; slot < C.S; slot += gridDim.x) {
    BState &S = C.st[slot];
    if (!S.setup) continue;
    const BProb<T> &P = C.prob[slot];
    const BLev<T> &V = P.L[P.nlev - 1];
    const int n = P.ncoarse;
    for (int e = threadIdx.x; e < kBDenseMax * kBDenseMax; e += blockDim.x) D[e / kBDenseMax][e % kBDenseMax] = 0.0;
    __syncthreads();
    const uint32_t SI = V.A.g.nynz, SJ = (uint32_t)V.A.nz;
    for (int p = threadIdx.x; p < n; p += blockDim.x) {
      Pos q = V.A.g.pos((uint32_t)p);
      D[p][p] = V.c64[p];
      if (q.i > 0) { D[p][p - SI] = -V.w64[p]; D[p - SI][p] = -V.w64[p]; }
      if (q.j > 0) { D[p][p - SJ] = -V.s64[p]; D[p - SJ][p] = -V.s64[p]; }
      if (q.k > 0) { D[p][p - 1] = -V.b64[p]; D[p - 1][p] = -V.b64[p]; }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double m = 0.0;
      for (int i = 0; i < n; ++i) m = fmax(m, D[i][i]);
      dmax = m;
    }
    __syncthreads();
    const double thr = rel_tol * dmax;
    for (int k = 0; k < n; ++k) {
      if (threadIdx.x < n) { rowk[threadIdx.x] = D[k][threadIdx.x]; colk[threadIdx.x] = D[threadIdx.x][k]; }
      __syncthreads();
      const double akk = rowk[k];
      const bool sk = !(akk > thr);
      const double piv = sk ? 0.0 : 1.0 / akk;
      for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int i = e / n, j = e - i * n;
        double v;
        if (sk) v = (i == k || j == k) ? 0.0 : D[i][j];
        else if (i == k && j == k) v = piv;
        else if (i == k) v = rowk[j] * piv;
        else if (j == k) v = -colk[i] * piv;
        else v = D[i][j] - colk[i] * rowk[j] * piv;
        D[i][j] = v;
      }
      __syncthreads();
    }
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) P.Ainv[e] = D[e / n][e % n];
    __syncthreads();
    if (threadIdx.x == 0) S.setup = 0;
  }
}

// ---------------------------------------------------------------- outer loop
// x += e for slots whose inner solve just finished.
template <typename T>
__global__ void kb_outer_corr(BCtx<T> C) {
  BTILE_FOR(C, 0, t, tl) {
    const BState &S = C.st[tl.slot];
    if (!(S.phase == BP_RUN && S.f.done)) continue;
    const BProb<T> &P = C.prob[tl.slot];
    BCELL_LOOP(tl, pp) {
      uint32_t p;
      if (b_compact(P, pp, p)) P.x[p] += (double)P.x0[pp];
    }
  }
}

// FP64 true residual r = b - A x for new slots and for slots whose inner
// solve just finished; r0 = (T) r starts the next inner solve. The slot's
// last tile runs the refinement decisions (as Engine::solve_mixed /
// solve_fp64).
template <typename T>
__global__ void kb_outer_resid(BCtx<T> C) {
  BTILE_FOR(C, 0, t, tl) {
    BState &S = C.st[tl.slot];
    if (!(S.phase == BP_INIT || (S.phase == BP_RUN && S.f.done))) continue;
    const BProb<T> &P = C.prob[tl.slot];
    const Geo &G = P.g0;
    const BLev<T> &V = P.L[0];
    double v[3] = {0.0, 0.0, 0.0};
    BCELL_LOOP(tl, pp) {
      uint32_t p;
      if (!b_compact(P, pp, p)) continue;
      Pos q = G.pos(p);
      const uint32_t SI = G.nynz, SJ = (uint32_t)G.nz;
      const double *x = P.x;
      double on = 0.0;
      if (q.i > 0) on += V.w64[p] * x[p - SI];
      if (q.i < G.nx - 1) on += V.w64[p + SI] * x[p + SI];
      if (q.j > 0) on += V.s64[p] * x[p - SJ];
      if (q.j < G.ny - 1) on += V.s64[p + SJ] * x[p + SJ];
      if (q.k > 0) on += V.b64[p] * x[p - 1];
      if (q.k < G.nz - 1) on += V.b64[p + 1] * x[p + 1];
      const double bp = P.b[p];
      const double r = bp - (V.c64[p] * x[p] - on);
      const T rt = (T)r;
      P.r0[pp] = rt;
      P.x0[pp] = T(0);
      P.q0[pp] = T(0);
      v[0] += r * r;
      v[1] += bp * bp;
      v[2] += (double)rt * (double)rt;
    }
    double o[3];
    if (b_reduce<3>(C, 0, t, tl.slot, v, o)) {
      const bool fresh = S.phase == BP_INIT;
      if (fresh) {
        S.bb = o[1];
        S.sweeps = 0;
        S.iters = 0;
        S.converged = 0;
        S.status = ST_RUNNING;
        if (!(o[1] > 0.0)) {
          S.rel = 0.0; S.rel0 = 0.0; S.converged = 1; S.status = ST_INITIAL; S.phase = BP_DONE;
          continue;
        }
        S.rel = sqrt(o[0] / o[1]);
        S.rel0 = S.rel;
      } else {
        const double nrel = sqrt(o[0] / S.bb);
        S.iters += S.f.iter;
        S.sweeps += 1;
        if (!(nrel == nrel)) { S.rel = nrel; S.status = ST_NAN; S.phase = BP_DONE; continue; }
        if (S.f.status == ST_BREAKDOWN && nrel >= S.rel) {
          S.rel = nrel; S.status = ST_BREAKDOWN; S.phase = BP_DONE; continue;
        }
        S.rel = nrel;
      }
      if (S.rel <= S.tol) { S.converged = 1; S.status = ST_CONVERGED; S.phase = BP_DONE; continue; }
      const int left = S.maxit - S.iters;
      if (S.sweeps >= S.max_sweeps || left <= 0 || !(o[2] > 0.0)) {
        S.status = ST_MAXITER; S.phase = BP_DONE; continue;
      }
      // next inner solve
      const double itol = S.mixed ? fmax(S.inner_tol, 0.9 * S.tol / S.rel) : fmin(0.9 * S.tol / S.rel, 0.5);
      FcgScal &f = S.f;
      f.rr0 = o[2]; f.rr = o[2]; f.tol = itol;
      f.maxit = left < S.inner_maxit ? left : S.inner_maxit;
      f.iter = 0; f.pq = 0.0; f.pr = 0.0; f.zq = 0.0; f.zr = 0.0; f.beta = 0.0; f.alpha = 0.0;
      f.converged = 0; f.status = ST_RUNNING; f.hist = nullptr;
      f.done = 0;
      S.phase = BP_RUN;
    }
  }
}

// ---------------------------------------------------------------- K-cycle: cell arithmetic
// One cell of each K-cycle phase, shared by the tile kernels and the
// CTA-local tail (kb_tail), so both compute the same bits.

// Right-hand side of the preconditioner application on level l: the FCG
// residual on level 0, the restricted b on coarse levels, or (kc) the
// K-cycle residual r1.
template <typename T>
__device__ __forceinline__ const T *b_rhs(const BProb<T> &P, int l, bool kc) {
  return l == 0 ? P.r0 : (kc ? P.L[l].r1 : P.L[l].b);
}

// Two damped-Jacobi sweeps from zero (k_jac2) into xb; kc: rhs b - a1 q1,
// formed on the fly and stored to r1.
template <typename T>
__device__ __forceinline__ void cell_jac2(const BLev<T> &V, const T *r, uint32_t p, T a1, bool kc, T om) {
  const EMat<T> &A = V.A;
  auto rv = [&](uint32_t s) -> T { return kc ? V.b[s] - a1 * V.q1[s] : r[s]; };
  auto x1 = [&](uint32_t s) -> T { return om * rv(s) * A.dinv[s]; };
  const Pos q = A.g.pos(p);
  const T rp = rv(p);
  if (kc) V.r1[p] = rp;
  const T d = A.dinv[p];
  const T xp = om * rp * d;
  const T on = offdiag(A, p, q, x1);
  V.xb[p] = xp + om * ((rp + on) * d - xp);
}

// Row of the dense coarsest solve: one warp, FP64 sums (lane 0 writes).
template <typename T>
__device__ __forceinline__ void warp_dense_row(const double *Ainv, int n, const T *b, T *x, int row) {
  const int lane = threadIdx.x & 31;
  double acc = 0.0;
  for (int col = lane; col < n; col += 32) acc += Ainv[row * n + col] * (double)b[col];
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
  if (lane == 0) x[row] = (T)acc;
}

// xa = xb + P e, then one sweep (k_prolong_jac); e from level l+1: eH
// (dense solution or single visit) or c1 z1 + c2 z2 (two).
template <typename T>
__device__ __forceinline__ void cell_prolong_jac(const BLev<T> &V, const BLev<T> &Hl, const T *r, const T *eH,
                                                 bool two, T c1, T c2, T om, uint32_t p) {
  const EMat<T> &A = V.A;
  const Geo &H = Hl.A.g;
  const T *z2H = Hl.z2;
  const int sx = A.nx > 1 ? 1 : 0, sy = A.ny > 1 ? 1 : 0, sz = A.nz > 1 ? 1 : 0;
  auto e = [&](int i, int j, int k) -> T {
    const uint32_t Pc = (uint32_t)(i >> sx) * H.nynz + (uint32_t)(j >> sy) * (uint32_t)H.nz + (uint32_t)(k >> sz);
    return two ? c1 * eH[Pc] + c2 * z2H[Pc] : eH[Pc];
  };
  const T *xi = V.xb;
  const Pos q = A.g.pos(p);
  const uint32_t SI = A.g.nynz, SJ = (uint32_t)A.nz;
  T on = 0;
  if (q.i > 0) on += A.w[p] * (xi[p - SI] + e(q.i - 1, q.j, q.k));
  if (q.i < A.nx - 1) on += A.w[p + SI] * (xi[p + SI] + e(q.i + 1, q.j, q.k));
  if (q.j > 0) on += A.s[p] * (xi[p - SJ] + e(q.i, q.j - 1, q.k));
  if (q.j < A.ny - 1) on += A.s[p + SJ] * (xi[p + SJ] + e(q.i, q.j + 1, q.k));
  if (q.k > 0) on += A.b[p] * (xi[p - 1] + e(q.i, q.j, q.k - 1));
  if (q.k < A.nz - 1) on += A.b[p + 1] * (xi[p + 1] + e(q.i, q.j, q.k + 1));
  const T xp = xi[p] + e(q.i, q.j, q.k);
  V.xa[p] = xp + om * ((r[p] + on) * A.dinv[p] - xp);
}

// z = xa + w D^-1 (rhs - A xa); returns z
template <typename T>
__device__ __forceinline__ T cell_jac(const BLev<T> &V, const T *r, T *z, T om, uint32_t p) {
  const EMat<T> &A = V.A;
  const Pos q = A.g.pos(p);
  const T on = offdiag(A, p, q, [&](uint32_t s) { return V.xa[s]; });
  const T xp = V.xa[p];
  const T zz = xp + om * ((r[p] + on) * A.dinv[p] - xp);
  z[p] = zz;
  return zz;
}

// q1 = A z1; v += (z1.b, z1.q1)
template <typename T>
__device__ __forceinline__ void cell_q1(const BLev<T> &V, uint32_t p, double (&v)[2]) {
  const Pos q = V.A.g.pos(p);
  const T qq = ax_at(V.A, p, q, V.z1);
  V.q1[p] = qq;
  v[0] += (double)V.z1[p] * (double)V.b[p];
  v[1] += (double)V.z1[p] * (double)qq;
}

// v += (z2.q1, z2.r1, z2.A z2)
template <typename T>
__device__ __forceinline__ void cell_q2(const BLev<T> &V, uint32_t p, double (&v)[3]) {
  const Pos q = V.A.g.pos(p);
  const T av = ax_at(V.A, p, q, V.z2);
  const double zz = (double)V.z2[p];
  v[0] += zz * (double)V.q1[p];
  v[1] += zz * (double)V.r1[p];
  v[2] += zz * (double)av;
}

// K-cycle scalars from the two steps' sums (k_kc_q1 / k_kc_q2)
__device__ __forceinline__ void kc_after_q1(KScal &k, const double (&o)[2]) {
  k.zb = o[0];
  k.zq = o[1];
  k.a1 = (o[1] > 0.0 && o[1] == o[1]) ? o[0] / o[1] : 0.0;
}
__device__ __forceinline__ void kc_after_q2(KScal &k, const double (&o)[3]) {
  const double zq = k.zq;
  const double beta = zq > 0.0 ? o[0] / zq : 0.0;
  const double z1r1 = k.zb - k.a1 * zq;
  const double pr = o[1] - beta * z1r1;
  const double pq = o[2] - 2.0 * beta * o[0] + beta * beta * zq;
  k.beta = beta;
  k.a2 = (pq > 0.0 && pq == pq && pr == pr) ? pr / pq : 0.0;
}

// Does the tile-kernel K-cycle on level l apply to this slot? (Level l
// exists, is not the coarsest, and is above the slot's CTA-local tail.)
template <typename T>
__device__ __forceinline__ bool b_tile_level(const BState &S, const BProb<T> &P, int l) {
  return b_running(S) && l < P.nlev - 1 && l < P.tail;
}

// Coarse correction read by the prolongation on level l (from level l+1)
template <typename T>
__device__ __forceinline__ void b_coarse(const BProb<T> &P, const BState &S, int l, int kc_max,
                                         const T *&eH, bool &two, T &c1, T &c2) {
  const BLev<T> &Hl = P.L[l + 1];
  const bool hdense = P.nlev - 1 == l + 1;
  two = !hdense && (l + 1) <= kc_max;
  eH = hdense ? Hl.x : Hl.z1;
  c1 = 1;
  c2 = 0;
  if (two) {
    const KScal &k = S.ks[l + 1];
    c1 = (T)(k.a1 - k.a2 * k.beta);
    c2 = (T)k.a2;
  }
}

// ---------------------------------------------------------------- padded level 0: groups of four
// The level-0 phases on a padded tile, four cells per thread with 16-byte
// loads (the helpers of the single-problem vector kernels; the same
// formulas as the cell functions above).

// two damped-Jacobi sweeps from zero into xb (level 0 has no K-cycle rhs)
template <typename T>
__device__ __forceinline__ void vgroup_jac2(const BLev<T> &V, const T *r, T om, uint32_t p) {
  constexpr int W = VecTraits<T>::V;
  const EMat<T> &A = V.A;
  const Pos q = A.g.pos(p);
  const CoefV<T> Cf = load_coef(A, p, q);
  const Vec<T> d = ldv(A.dinv, p), rp = ldv(r, p);
  const HoodV<T> X = load_hood(A, p, q, FJac0<T>{r, A.dinv, om});
  Vec<T> o;
#pragma unroll
  for (int m = 0; m < W; ++m) {
    const T xp = X.c.v[m];
    o.v[m] = xp + om * ((rp.v[m] + offd(Cf, X, m)) * d.v[m] - xp);
  }
  stv(V.xb, p, o);
}

// residual rhs - A xb of a group, into xa (free until the prolongation):
// the restriction onto level 1 then only sums children
template <typename T>
__device__ __forceinline__ void vgroup_resid(const BLev<T> &V, const T *r, uint32_t p) {
  constexpr int W = VecTraits<T>::V;
  const EMat<T> &A = V.A;
  const Pos q = A.g.pos(p);
  const CoefV<T> Cf = load_coef(A, p, q);
  const Vec<T> c = ldv(A.c, p), rp = ldv(r, p);
  const HoodV<T> X = load_hood(A, p, q, FArr<T>{V.xb});
  Vec<T> o;
#pragma unroll
  for (int m = 0; m < W; ++m) o.v[m] = rp.v[m] - axv(c.v[m], Cf, X, m);
  stv(V.xa, p, o);
}

// coarse cell Pc of level 1 = the sum of its children's residuals (in xa),
// in restrict_cell's (a, b, c) order
template <typename T>
__device__ __forceinline__ T restrict_sum_pad(const BProb<T> &P, const EMat<T> &A, const T *res, const Geo &H,
                                              uint32_t Pc) {
  const Pos Q = H.pos(Pc);
  const int fx = A.nx > 1 ? 2 : 1, fy = A.ny > 1 ? 2 : 1, fz = P.F > 1 ? 2 : 1;
  const int qj = P.rel2d ? 0 : Q.j, qk = P.rel2d ? Q.j : Q.k;
  T sum = 0;
  for (int a = 0; a < fx; ++a) {
    const int i = Q.i * fx + a;
    if (i >= A.nx) break;
    for (int bb = 0; bb < fy; ++bb) {
      const int j = qj * fy + bb;
      if (j >= A.ny) break;
      for (int cc = 0; cc < fz; ++cc) {
        const int k = qk * fz + cc;
        if (k >= P.F) break;
        sum += res[((uint32_t)i * A.ny + j) * A.nz + k];
      }
    }
  }
  return sum;
}

// xa = xb + P e, then one sweep; pad lanes (k >= F) take no correction
template <typename T>
__device__ __forceinline__ void vgroup_prolong_jac(const BProb<T> &P, const BLev<T> &V, const BLev<T> &Hl,
                                                   const T *r, const T *eH, bool two, T c1, T c2, T om,
                                                   uint32_t p) {
  constexpr int W = VecTraits<T>::V;
  const EMat<T> &A = V.A;
  const Geo &H = Hl.A.g;
  const T *z2H = Hl.z2;
  const int sx = A.nx > 1 ? 1 : 0, sy = A.ny > 1 ? 1 : 0, sz = P.F > 1 ? 1 : 0;
  const int F = P.F;
  auto e = [&](int i, int j, int k) -> T {
    if (k >= F) return T(0);
    const uint32_t Pc = (uint32_t)(i >> sx) * H.nynz + (uint32_t)(j >> sy) * (uint32_t)H.nz + (uint32_t)(k >> sz);
    return two ? c1 * eH[Pc] + c2 * z2H[Pc] : eH[Pc];
  };
  const T *xi = V.xb;
  const Pos q = A.g.pos(p);
  auto rowv = [&](uint32_t pr, int i, int j) -> Vec<T> {
    Vec<T> x = ldv(xi, pr);
#pragma unroll
    for (int m = 0; m < W; ++m) x.v[m] += e(i, j, q.k + m);
    return x;
  };
  const uint32_t SI = A.g.nynz, SJ = (uint32_t)A.nz;
  HoodV<T> X;
  X.c = rowv(p, q.i, q.j);
  X.w = q.i > 0 ? rowv(p - SI, q.i - 1, q.j) : zerov<T>();
  X.e = q.i < A.nx - 1 ? rowv(p + SI, q.i + 1, q.j) : zerov<T>();
  X.s = q.j > 0 ? rowv(p - SJ, q.i, q.j - 1) : zerov<T>();
  X.n = q.j < A.ny - 1 ? rowv(p + SJ, q.i, q.j + 1) : zerov<T>();
  X.km = q.k > 0 ? xi[p - 1] + e(q.i, q.j, q.k - 1) : T(0);
  X.kp = q.k + W < A.nz ? xi[p + W] + e(q.i, q.j, q.k + W) : T(0);
  const CoefV<T> Cf = load_coef(A, p, q);
  const Vec<T> d = ldv(A.dinv, p), rp = ldv(r, p);
  Vec<T> o;
#pragma unroll
  for (int m = 0; m < W; ++m) {
    const T xp = X.c.v[m];
    o.v[m] = xp + om * ((rp.v[m] + offd(Cf, X, m)) * d.v[m] - xp);
  }
  stv(V.xa, p, o);
}

// z = xa + w D^-1 (r - A xa); v += (z.r, z.q0)
template <typename T>
__device__ __forceinline__ void vgroup_jac(const BProb<T> &P, const BLev<T> &V, const T *r, T om, uint32_t p,
                                           double (&v)[2]) {
  constexpr int W = VecTraits<T>::V;
  const EMat<T> &A = V.A;
  const Pos q = A.g.pos(p);
  const CoefV<T> Cf = load_coef(A, p, q);
  const Vec<T> d = ldv(A.dinv, p), rp = ldv(r, p), qo = ldv(P.q0, p);
  const HoodV<T> X = load_hood(A, p, q, FArr<T>{V.xa});
  Vec<T> o;
#pragma unroll
  for (int m = 0; m < W; ++m) {
    const T xp = X.c.v[m];
    o.v[m] = xp + om * ((rp.v[m] + offd(Cf, X, m)) * d.v[m] - xp);
    v[0] += (double)o.v[m] * (double)rp.v[m];
    v[1] += (double)o.v[m] * (double)qo.v[m];
  }
  stv(P.z0, p, o);
}

// ---------------------------------------------------------------- K-cycle: tile kernels
template <typename T>
__global__ void BPAD_BOUNDS kb_jac2(BCtx<T> C, int l, int kc) {
  BTILE_FOR(C, l, t, tl) {
    const BState &S = C.st[tl.slot];
    const BProb<T> &P = C.prob[tl.slot];
    if (!b_tile_level(S, P, l)) continue;
    const T a1 = kc ? (T)S.ks[l].a1 : T(0);
    const T *r = l == 0 ? P.r0 : P.L[l].b;
    if (kBPad<T> && l == 0) {
      BGROUP_LOOP(tl, p) vgroup_jac2(P.L[0], r, C.omega, p);
      continue;
    }
    BCELL_LOOP(tl, p) cell_jac2(P.L[l], r, p, a1, kc != 0, C.omega);
  }
}

// b on level l+1 = block sums of (rhs - A xb) on level l, one thread per
// coarse cell (restrict_cell): the problems of the batch already fill the
// GPU, so the eight-lane form is kept for the single-CTA tail.
template <typename T>
__global__ void kb_restrict(BCtx<T> C, int l, int kc) {
  BTILE_FOR(C, l + 1, t, tl) {
    const BState &S = C.st[tl.slot];
    const BProb<T> &P = C.prob[tl.slot];
    if (!b_tile_level(S, P, l)) continue;
    const T *r = b_rhs(P, l, kc != 0);
    const BLev<T> &V = P.L[l], &H = P.L[l + 1];
    if (kBPad<T> && l == 0) {  // the residuals are in xa (kb_resid0)
      BCELL_LOOP(tl, Pc) H.b[Pc] = restrict_sum_pad(P, V.A, V.xa, H.A.g, Pc);
      continue;
    }
    BCELL_LOOP(tl, Pc) H.b[Pc] = restrict_cell(V.A, r, V.xb, H.A.g, Pc);
  }
}

// padded level 0: residuals of the two sweeps into xa, for kb_restrict
template <typename T>
__global__ void BPAD_BOUNDS kb_resid0(BCtx<T> C) {
  if constexpr (kBPad<T>) {
    BTILE_FOR(C, 0, t, tl) {
      const BState &S = C.st[tl.slot];
      const BProb<T> &P = C.prob[tl.slot];
      if (!b_tile_level(S, P, 0)) continue;
      BGROUP_LOOP(tl, p) vgroup_resid(P.L[0], P.r0, p);
    }
  }
}

// x = Ainv b on level L for slots whose coarsest level is L and not inside
// their tail (one CTA per slot, one warp per row).
template <typename T>
__global__ void kb_dense(BCtx<T> C, int L) {
  const int wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int slot = blockIdx.x; slot < C.S; slot += gridDim.x) {
    const BState &S = C.st[slot];
    const BProb<T> &P = C.prob[slot];
    if (!b_running(S) || P.nlev - 1 != L || P.tail <= L) continue;
    const BLev<T> &V = P.L[L];
    for (int row = wid; row < P.ncoarse; row += nw) warp_dense_row(P.Ainv, P.ncoarse, V.b, V.x, row);
  }
}

template <typename T>
__global__ void BPAD_BOUNDS kb_prolong_jac(BCtx<T> C, int l, int kc) {
  BTILE_FOR(C, l, t, tl) {
    const BState &S = C.st[tl.slot];
    const BProb<T> &P = C.prob[tl.slot];
    if (!b_tile_level(S, P, l)) continue;
    const T *eH;
    bool two;
    T c1, c2;
    b_coarse(P, S, l, C.kc_max, eH, two, c1, c2);
    const T *r = b_rhs(P, l, kc != 0);
    if (kBPad<T> && l == 0) {
      BGROUP_LOOP(tl, p) vgroup_prolong_jac(P, P.L[0], P.L[1], r, eH, two, c1, c2, C.omega, p);
      continue;
    }
    BCELL_LOOP(tl, p) cell_prolong_jac(P.L[l], P.L[l + 1], r, eH, two, c1, c2, C.omega, p);
  }
}

// Last sweep; level 0 writes z0 and reduces z.r0 and z.q0 (q of the
// previous FCG iteration) into the slot's FCG scalars.
template <typename T>
__global__ void BPAD_BOUNDS kb_jac(BCtx<T> C, int l, int kc) {
  BTILE_FOR(C, l, t, tl) {
    BState &S = C.st[tl.slot];
    const BProb<T> &P = C.prob[tl.slot];
    if (!b_tile_level(S, P, l)) continue;
    const BLev<T> &V = P.L[l];
    const T *r = b_rhs(P, l, kc != 0);
    T *z = l == 0 ? P.z0 : (kc ? V.z2 : V.z1);
    double v[2] = {0.0, 0.0};
    if (kBPad<T> && l == 0) {
      BGROUP_LOOP(tl, p) vgroup_jac(P, V, r, C.omega, p, v);
      double o[2];
      if (b_reduce<2>(C, 0, t, tl.slot, v, o)) { S.f.zr = o[0]; S.f.zq = o[1]; }
      continue;
    }
    BCELL_LOOP(tl, p) {
      const T zz = cell_jac(V, r, z, C.omega, p);
      if (l == 0) {
        v[0] += (double)zz * (double)r[p];
        v[1] += (double)zz * (double)P.q0[p];
      }
    }
    if (l == 0) {
      double o[2];
      if (b_reduce<2>(C, 0, t, tl.slot, v, o)) { S.f.zr = o[0]; S.f.zq = o[1]; }
    }
  }
}

template <typename T>
__global__ void kb_kc_q1(BCtx<T> C, int l) {
  BTILE_FOR(C, l, t, tl) {
    BState &S = C.st[tl.slot];
    const BProb<T> &P = C.prob[tl.slot];
    if (!b_tile_level(S, P, l)) continue;
    double v[2] = {0.0, 0.0};
    BCELL_LOOP(tl, p) cell_q1(P.L[l], p, v);
    double o[2];
    if (b_reduce<2>(C, l, t, tl.slot, v, o)) kc_after_q1(S.ks[l], o);
  }
}

template <typename T>
__global__ void kb_kc_q2(BCtx<T> C, int l) {
  BTILE_FOR(C, l, t, tl) {
    BState &S = C.st[tl.slot];
    const BProb<T> &P = C.prob[tl.slot];
    if (!b_tile_level(S, P, l)) continue;
    double v[3] = {0.0, 0.0, 0.0};
    BCELL_LOOP(tl, p) cell_q2(P.L[l], p, v);
    double o[3];
    if (b_reduce<3>(C, l, t, tl.slot, v, o)) kc_after_q2(S.ks[l], o);
  }
}

// ---------------------------------------------------------------- K-cycle: CTA-local tail
// Block sum of K values, broadcast to every thread (fixed order).
template <int K>
__device__ __forceinline__ void t_allreduce(double (&v)[K], double (*sm)[kBThreadsMax / 32], double (&bc)[4]) {
  b_block_sum<K>(v, sm);
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < K; ++q) bc[q] = v[q];
  __syncthreads();
#pragma unroll
  for (int q = 0; q < K; ++q) v[q] = bc[q];
  __syncthreads();
}

#define TCELL_LOOP(p, N) for (uint32_t p = threadIdx.x; p < (uint32_t)(N); p += blockDim.x)

// The whole K-cycle of level `top` of one slot, by one CTA (every level
// from `top` down lies in one tile, so a CTA barrier separates the phases).
// The same program as the tile-kernel sequence, with the recursion as a
// loop and a program counter per level: 0 / 2 start the first / second
// preconditioner application, 1 / 3 finish it. Leaves z1 (and z2) on level
// top and its scalars in S.ks[top] as a1 = c1, a2 = c2, beta = 0.
template <typename T>
__device__ void t_kcycle(const BProb<T> &P, BState &S, int top, int kc_max, T om) {
  __shared__ double sm[3][kBThreadsMax / 32];
  __shared__ double bc[4];
  const int last = P.nlev - 1;
  const int nw = blockDim.x >> 5, wid = threadIdx.x >> 5;
  int step[kBMaxLev];
  double c1v[kBMaxLev], c2v[kBMaxLev];
  KScal ks[kBMaxLev];
  int l = top;
  step[l] = 0;
  for (int guard = 0; guard < (1 << 24); ++guard) {
    const BLev<T> &V = P.L[l];
    const uint32_t n = V.A.g.n;
    const int s = step[l];
    const bool second = s >= 2;
    const T *rr = second ? V.r1 : V.b;
    if (s == 0 || s == 2) {
      const T a1 = second ? (T)ks[l].a1 : T(0);
      TCELL_LOOP(p, n) cell_jac2(V, V.b, p, a1, second, om);
      __syncthreads();
      const BLev<T> &H = P.L[l + 1];
      for (uint32_t base = 0; base < H.A.g.n * 8u; base += blockDim.x) {
        const uint32_t u = base + threadIdx.x;
        const bool valid = u < H.A.g.n * 8u;
        T v = valid ? restrict_child(V.A, rr, V.xb, H.A.g, u) : T(0);
        v = sum8(v);
        if (valid && (u & 7u) == 0u) H.b[u >> 3] = v;
      }
      __syncthreads();
      step[l] = s + 1;
      if (l + 1 == last) {
        for (int row = wid; row < P.ncoarse; row += nw) warp_dense_row(P.Ainv, P.ncoarse, H.b, H.x, row);
        __syncthreads();
      } else {
        l = l + 1;
        step[l] = 0;
      }
      continue;
    }
    {
      const BLev<T> &H = P.L[l + 1];
      const bool hdense = l + 1 == last;
      const bool two = !hdense && (l + 1) <= kc_max;
      const T *eH = hdense ? H.x : H.z1;
      const T c1 = hdense ? T(1) : (T)c1v[l + 1], c2 = hdense ? T(0) : (T)c2v[l + 1];
      TCELL_LOOP(p, n) cell_prolong_jac(V, H, rr, eH, two, c1, c2, om, p);
      __syncthreads();
      TCELL_LOOP(p, n) cell_jac(V, rr, second ? V.z2 : V.z1, om, p);
      __syncthreads();
    }
    if (!second) {
      if (l > kc_max) {
        c1v[l] = 1.0;
        c2v[l] = 0.0;
      } else {
        double v[2] = {0.0, 0.0};
        TCELL_LOOP(p, n) cell_q1(V, p, v);
        t_allreduce<2>(v, sm, bc);
        kc_after_q1(ks[l], v);
        step[l] = 2;
        continue;
      }
    } else {
      double v[3] = {0.0, 0.0, 0.0};
      TCELL_LOOP(p, n) cell_q2(V, p, v);
      t_allreduce<3>(v, sm, bc);
      kc_after_q2(ks[l], v);
      c1v[l] = ks[l].a1 - ks[l].a2 * ks[l].beta;
      c2v[l] = ks[l].a2;
    }
    if (l == top) break;
    l = l - 1;
  }
  if (threadIdx.x == 0) {
    S.ks[top].a1 = c1v[top];
    S.ks[top].a2 = c2v[top];
    S.ks[top].beta = 0.0;
  }
  __syncthreads();
}

// K-cycles of level l for every slot whose tail starts there.
template <typename T>
__global__ void __launch_bounds__(kBThreadsMax) kb_tail(BCtx<T> C, int l) {
  for (int slot = blockIdx.x; slot < C.S; slot += gridDim.x) {
    BState &S = C.st[slot];
    const BProb<T> &P = C.prob[slot];
    if (!b_running(S) || P.tail != l) continue;
    t_kcycle(P, S, l, C.kc_max, C.omega);
  }
}

// ---------------------------------------------------------------- outer FCG (level 0)
// p = z - beta p_old, q = A p, alpha = p.r / p.q (k_fcg_pq)
template <typename T>
__global__ void BPAD_BOUNDS kb_fcg_pq(BCtx<T> C) {
  BTILE_FOR(C, 0, t, tl) {
    BState &S = C.st[tl.slot];
    if (!b_running(S)) continue;
    const BProb<T> &P = C.prob[tl.slot];
    const EMat<T> &A = P.L[0].A;
    FcgScal &f = S.f;
    const int it = f.iter;
    const T *pold = (it & 1) ? P.pB : P.pA;
    T *pnew = (it & 1) ? P.pA : P.pB;
    const double betad = (it == 0 || !(f.pq > 0.0)) ? 0.0 : f.zq / f.pq;
    const T beta = (T)betad;
    const T *z = P.z0;
    auto pv = [&](uint32_t s) -> T { return it == 0 ? z[s] : z[s] - beta * pold[s]; };
    double v[1] = {0.0};
    if constexpr (kBPad<T>) {
      // q = A z - beta q_old (= A p, with q_old = A p_old kept in q0), so
      // only z is read around the group (as kv_fcg_pq)
      constexpr int W = VecTraits<T>::V;
      BGROUP_LOOP(tl, p) {
        const Pos q = A.g.pos(p);
        const CoefV<T> Cf = load_coef(A, p, q);
        const Vec<T> c = ldv(A.c, p);
        const HoodV<T> Z = load_hood(A, p, q, FArr<T>{z});
        Vec<T> pv, qv;
        if (it == 0) {
#pragma unroll
          for (int m = 0; m < W; ++m) { pv.v[m] = Z.c.v[m]; qv.v[m] = axv(c.v[m], Cf, Z, m); }
        } else {
          const Vec<T> po = ldv(pold, p), qo = ldv(P.q0, p);
#pragma unroll
          for (int m = 0; m < W; ++m) {
            pv.v[m] = Z.c.v[m] - beta * po.v[m];
            qv.v[m] = axv(c.v[m], Cf, Z, m) - beta * qo.v[m];
          }
        }
#pragma unroll
        for (int m = 0; m < W; ++m) v[0] += (double)pv.v[m] * (double)qv.v[m];
        stv(pnew, p, pv);
        stv(P.q0, p, qv);
      }
    } else {
      BCELL_LOOP(tl, p) {
        Pos q = A.g.pos(p);
        const T pp = pv(p);
        const T qq = ax_f(A, p, q, pv);
        pnew[p] = pp;
        P.q0[p] = qq;
        v[0] += (double)pp * (double)qq;
      }
    }
    double o[1];
    if (b_reduce<1>(C, 0, t, tl.slot, v, o)) {
      const double pr = f.zr - betad * (it == 0 ? 0.0 : f.pr);
      f.beta = betad;
      f.pq = o[0];
      f.alpha = (o[0] > 0.0 && o[0] == o[0]) ? pr / o[0] : 0.0;
      if (!(o[0] > 0.0) || !(o[0] == o[0])) { f.done = 1; f.status = ST_BREAKDOWN; }
    }
  }
}

// x += alpha p, r -= alpha q; inner convergence (k_fcg_xr)
template <typename T>
__global__ void BPAD_BOUNDS kb_fcg_xr(BCtx<T> C) {
  BTILE_FOR(C, 0, t, tl) {
    BState &S = C.st[tl.slot];
    if (!b_running(S)) continue;
    const BProb<T> &P = C.prob[tl.slot];
    FcgScal &f = S.f;
    const int it = f.iter;
    const T *pp = (it & 1) ? P.pA : P.pB;
    const T alpha = (T)f.alpha;
    double v[2] = {0.0, 0.0};
    if constexpr (kBPad<T>) {
      constexpr int W = VecTraits<T>::V;
      BGROUP_LOOP(tl, p) {
        const Vec<T> pv = ldv(pp, p), qv = ldv(P.q0, p);
        Vec<T> xv = ldv(P.x0, p), rv = ldv(P.r0, p);
#pragma unroll
        for (int m = 0; m < W; ++m) {
          xv.v[m] += alpha * pv.v[m];
          rv.v[m] = rv.v[m] - alpha * qv.v[m];
          v[0] += (double)rv.v[m] * (double)rv.v[m];
          v[1] += (double)pv.v[m] * (double)rv.v[m];
        }
        stv(P.x0, p, xv);
        stv(P.r0, p, rv);
      }
    } else {
      BCELL_LOOP(tl, p) {
        const T pv = pp[p];
        P.x0[p] += alpha * pv;
        const T rv = P.r0[p] - alpha * P.q0[p];
        P.r0[p] = rv;
        v[0] += (double)rv * (double)rv;
        v[1] += (double)pv * (double)rv;
      }
    }
    double o[2];
    if (b_reduce<2>(C, 0, t, tl.slot, v, o)) {
      f.rr = o[0];
      f.pr = o[1];
      const double rel = sqrt(o[0] / f.rr0);
      f.iter = it + 1;
      if (rel <= f.tol) { f.done = 1; f.converged = 1; f.status = ST_CONVERGED; }
      else if (!(rel == rel)) { f.done = 1; f.status = ST_NAN; }
      else if (it + 1 >= f.maxit) { f.done = 1; f.status = ST_MAXITER; }
    }
  }
}

}  // namespace pbg
