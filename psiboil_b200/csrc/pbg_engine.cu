// Host side of the engine solver (hierarchy set-up, K-cycle recursion,
// flexible CG and the mixed-precision refinement loop).
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <vector>

#include "pbg_engine.cuh"
#include "pbg_engine_kernels.cuh"
#include "pbg_vec.cuh"

namespace pbg {

// ---------------------------------------------------------------- hierarchy set-up kernels
// Output arrays of one level's numeric set-up: the FP64 operator, its
// inverse diagonal and, in the mixed path (c32 != nullptr), the FP32
// operator in edge form (c32 = diagonal excess, see kEdgeForm).
struct LevelOut {
  double *c, *w, *s, *b, *d;
  float *c32, *w32, *s32, *b32, *d32;
};

// Inverse diagonal and FP32 copies of a level whose FP64 operator is set.
__global__ void k_level_finish(EMat<double> A, LevelOut o) {
  GRID_LOOP(p, A.g.n) {
    const double c = A.c[p];
    o.d[p] = 1.0 / c;
    if (o.c32) {
      const Pos q = A.g.pos(p);
      const double sum = offdiag(A, p, q, [](uint32_t) { return 1.0; });
      o.c32[p] = (float)(c - sum);
      o.w32[p] = (float)A.w[p]; o.s32[p] = (float)A.s[p]; o.b32[p] = (float)A.b[p];
      o.d32[p] = (float)(1.0 / c);
    }
  }
}

// Galerkin coarse operator P^T A P for piecewise-constant aggregation by 2
// per direction (the sum over a block of every entry of A; each internal
// coupling enters the block's diagonal twice), FP64.
__global__ void k_galerkin(EMat<double> A, Geo H, LevelOut o) {
  const int fx = A.nx > 1 ? 2 : 1, fy = A.ny > 1 ? 2 : 1, fz = A.nz > 1 ? 2 : 1;
  GRID_LOOP(P, H.n) {
    Pos Q = H.pos(P);
    double c = 0.0, w = 0.0, s = 0.0, b = 0.0;
    const int i0 = Q.i * fx, j0 = Q.j * fy, k0 = Q.k * fz;
    for (int a = 0; a < fx && i0 + a < A.nx; ++a)
      for (int bb = 0; bb < fy && j0 + bb < A.ny; ++bb)
        for (int cc = 0; cc < fz && k0 + cc < A.nz; ++cc) {
          const uint32_t p = ((uint32_t)(i0 + a) * A.ny + (j0 + bb)) * A.nz + (k0 + cc);
          c += A.c[p];
          if (a == 0) w += A.w[p]; else c -= 2.0 * A.w[p];
          if (bb == 0) s += A.s[p]; else c -= 2.0 * A.s[p];
          if (cc == 0) b += A.b[p]; else c -= 2.0 * A.b[p];
        }
    o.c[P] = c; o.w[P] = w; o.s[P] = s; o.b[P] = b;
  }
}

// ---------------------------------------------------------------- dense coarsest
// Dense n x n matrix of the coarsest symmetric 7-point operator (D zeroed
// beforehand).
__global__ void k_dense_fill(EMat<double> A, double *__restrict__ D) {
  const uint32_t n = A.g.n, SI = A.g.nynz, SJ = (uint32_t)A.nz;
  GRID_LOOP(p, n) {
    Pos q = A.g.pos(p);
    D[(size_t)p * n + p] = A.c[p];
    if (q.i > 0) { D[(size_t)p * n + p - SI] = -A.w[p]; D[(size_t)(p - SI) * n + p] = -A.w[p]; }
    if (q.j > 0) { D[(size_t)p * n + p - SJ] = -A.s[p]; D[(size_t)(p - SJ) * n + p] = -A.s[p]; }
    if (q.k > 0) { D[(size_t)p * n + p - 1] = -A.b[p]; D[(size_t)(p - 1) * n + p] = -A.b[p]; }
  }
}

// Largest diagonal entry, for the pivot threshold (one block of 1024).
__global__ void k_dense_dmax(int n, const double *__restrict__ D, double *dmax) {
  double m = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, D[(size_t)i * n + i]);
  for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, off));
  __shared__ double wm[32];
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < (int)(blockDim.x >> 5); ++q) m = fmax(m, wm[q]);
    *dmax = fmax(m, wm[0]);
  }
}

constexpr int kGjB = 32;     // pivots per block step
constexpr int kGjRows = 32;  // rows per CTA (each reuses the pivot rows from L2)

// One blocked Gauss-Jordan exchange on the pivots k0 .. k0+kb-1 (out of
// place, A -> B). With A11 the pivot block, G = A11^-1 (by scalar
// Gauss-Jordan in shared memory, every CTA redundantly):
//   B11 = G, B12 = G A12, B21 = -A21 G, B22 = A22 - A21 G A12.
// After the last block B = A^-1. A pivot not above rel_tol * dmax (a
// solid-only aggregate, or the constant mode of an all-Neumann problem)
// is skipped: its row and column become zero, i.e. that unknown is held at
// zero, which gives a generalised inverse of a consistent singular system
// (in a positive semi-definite matrix a zero Schur pivot has a zero row
// and column, so nothing else changes).
__global__ void __launch_bounds__(256) k_gj_block(int n, int k0, const double *__restrict__ A,
                                                  double *__restrict__ B, const double *dmax,
                                                  double rel_tol) {
  __shared__ double G[kGjB][kGjB + 1];
  __shared__ double U[kGjRows][kGjB + 1];
  __shared__ double S[kGjRows][kGjB + 1];
  __shared__ double rowk[kGjB], colk[kGjB];
  const int kb = min(kGjB, n - k0);
  const double thr = rel_tol * (*dmax);
  for (int e = threadIdx.x; e < kGjB * kGjB; e += blockDim.x) {
    const int r = e / kGjB, c = e % kGjB;
    G[r][c] = (r < kb && c < kb) ? A[(size_t)(k0 + r) * n + k0 + c] : 0.0;
  }
  __syncthreads();
  for (int k = 0; k < kb; ++k) {
    if (threadIdx.x < kb) { rowk[threadIdx.x] = G[k][threadIdx.x]; colk[threadIdx.x] = G[threadIdx.x][k]; }
    __syncthreads();
    const double akk = rowk[k];
    const bool sk = !(akk > thr);
    const double piv = sk ? 0.0 : 1.0 / akk;
    for (int e = threadIdx.x; e < kb * kb; e += blockDim.x) {
      const int i = e / kb, j = e - i * kb;
      double v;
      if (sk) v = (i == k || j == k) ? 0.0 : G[i][j];
      else if (i == k && j == k) v = piv;
      else if (i == k) v = rowk[j] * piv;
      else if (j == k) v = -colk[i] * piv;
      else v = G[i][j] - colk[i] * rowk[j] * piv;
      G[i][j] = v;
    }
    __syncthreads();
  }
  const int ntile = (n + kGjRows - 1) / kGjRows;
  for (int t = blockIdx.x; t < ntile; t += gridDim.x) {
    const int i0 = t * kGjRows;
    // U: the row coefficients on the pivot rows; S: the rows' pivot-column entries
    for (int e = threadIdx.x; e < kGjRows * kGjB; e += blockDim.x) {
      const int ii = e / kGjB, l = e % kGjB, i = i0 + ii;
      S[ii][l] = (i < n && l < kb) ? A[(size_t)i * n + k0 + l] : 0.0;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < kGjRows * kGjB; e += blockDim.x) {
      const int ii = e / kGjB, l = e % kGjB, i = i0 + ii;
      double u = 0.0;
      if (i < n && l < kb) {
        if (i >= k0 && i < k0 + kb) u = G[i - k0][l];
        else
          for (int m = 0; m < kb; ++m) u += S[ii][m] * G[m][l];
      }
      U[ii][l] = u;
    }
    __syncthreads();
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
      const bool jin = j >= k0 && j < k0 + kb;
      double a[kGjB];
#pragma unroll
      for (int l = 0; l < kGjB; ++l) a[l] = (!jin && l < kb) ? A[(size_t)(k0 + l) * n + j] : 0.0;
      for (int ii = 0; ii < kGjRows; ++ii) {
        const int i = i0 + ii;
        if (i >= n) break;
        const bool iin = i >= k0 && i < k0 + kb;
        double v;
        if (jin) v = iin ? U[ii][j - k0] : -U[ii][j - k0];
        else {
          double acc = 0.0;
#pragma unroll
          for (int l = 0; l < kGjB; ++l) acc += U[ii][l] * a[l];
          v = iin ? acc : A[(size_t)i * n + j] - acc;
        }
        B[(size_t)i * n + j] = v;
      }
    }
    __syncthreads();
  }
}


template <typename T>
void EWork<T>::ensure(const std::vector<ELevel> &lv) {
  if (L.size() == lv.size() && x0.n == (size_t)lv[0].ncell()) return;
  drop_graph();
  L.clear();
  L.resize(lv.size());
  for (size_t l = 0; l < lv.size(); ++l) {
    size_t n = (size_t)lv[l].ncell();
    Lv &v = L[l];
    v.b.alloc(n); v.x.alloc(n); v.xa.alloc(n); v.xb.alloc(n);
    if (l > 0) { v.z1.alloc(n); v.z2.alloc(n); v.q1.alloc(n); v.r1.alloc(n); v.v.alloc(n); }
  }
  size_t n0 = (size_t)lv[0].ncell();
  x0.alloc(n0); r0.alloc(n0); z0.alloc(n0); pA.alloc(n0); pB.alloc(n0); q0.alloc(n0);
  q0b.alloc(n0);
  ks.alloc(lv.size());
  fs.alloc(1);
  PBG_CUDA(cudaMemset(fs.p, 0, sizeof(FcgScal)));
}

template <typename T>
void EWork<T>::drop_graph() {
  if (iter_graph) cudaGraphExecDestroy(iter_graph);
  if (loop_graph) cudaGraphExecDestroy(loop_graph);
  iter_graph = nullptr;
  loop_graph = nullptr;
  iter_nodes = 0;
}

// Programmatic dependent launch measured no gain inside the captured
// iteration (20.0 against 20.2 ms at 256^3), so it is off unless PBG_PDL=1.
bool pdl_enabled() {
  static const bool on = [] {
    const char *e = getenv("PBG_PDL");
    return e && atoi(e) == 1;
  }();
  return on;
}

// End of one FCG iteration in the device-side loop (a conditional WHILE
// node of a CUDA graph): continue while the solve is running, and never
// more than maxit times, whatever the flags say.
__global__ void k_fcg_continue(cudaGraphConditionalHandle h, FcgScal *fs) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int n = ++fs->loops;
  cudaGraphSetConditional(h, (!fs->done && n < fs->maxit) ? 1u : 0u);
}

// Start of the device-side loop: enter it only if the solve has not
// converged at the start (k_fcg_init sets done when |r0| is already below
// the tolerance). With this gate in front of the WHILE node, no kernel of
// the loop body runs once the solve is done, so the body's kernels are
// captured without the done flag and do not load it before their work.
__global__ void k_fcg_gate(cudaGraphConditionalHandle h, const FcgScal *fs) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  cudaGraphSetConditional(h, (!fs->done && fs->loops < fs->maxit) ? 1u : 0u);
}

// The FCG iterations of a refinement sweep run as a device-side loop (a
// conditional WHILE graph node) unless PBG_GRAPH_LOOP=0, which replays the
// one-iteration graph in host-polled chunks instead.
static bool graph_loop_enabled() {
  static const bool on = [] {
    const char *e = getenv("PBG_GRAPH_LOOP");
    return !(e && atoi(e) == 0);
  }();
  return on;
}

// Tuning knobs (environment): PBG_COARSE_MAX sets the size of the dense
// coarsest level, PBG_KC_MAX the deepest level that runs a K-cycle,
// PBG_OMEGA the damped-Jacobi weight (0 < omega < 1).
EngineOpts::EngineOpts() {
  const char *c = getenv("PBG_COARSE_MAX");
  if (c && atoi(c) > 0) coarse_max = atoi(c);
  const char *k = getenv("PBG_KC_MAX");
  if (k && atoi(k) > 0) kc_max = atoi(k);
  const char *o = getenv("PBG_OMEGA");
  if (o && atof(o) > 0.0 && atof(o) < 1.0) omega = atof(o);
}

template struct EWork<double>;
template struct EWork<float>;

Engine::~Engine() {
  if (hsc) cudaFreeHost(hsc);
}

template <> EMat<double> Engine::mat<double>(int l) const { return L[l].m64; }
template <> EMat<float> Engine::mat<float>(int l) const { return L[l].m32; }
template <> const void *Engine::ainv<double>() const { return Ainv.p; }
template <> const void *Engine::ainv<float>() const { return Ainv32.p; }

// Row-scaled FP16 copy of the dense inverse: row i is stored as a / s_i with
// s_i = max_j |a_ij|, so every entry lies in [-1, 1] (one warp per row).
__global__ void k_to_half_rows(int n, const double *__restrict__ a, __half *__restrict__ o,
                               float *__restrict__ sc) {
  const int lane = threadIdx.x & 31;
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (row >= n) return;
  const double *ar = a + (long long)row * n;
  double m = 0.0;
  for (int c = lane; c < n; c += 32) m = fmax(m, fabs(ar[c]));
  for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, off));
  const double inv = m > 0.0 ? 1.0 / m : 0.0;
  for (int c = lane; c < n; c += 32) o[(long long)row * n + c] = __double2half(ar[c] * inv);
  if (lane == 0) sc[row] = (float)m;
}

// z = Ainv r from the row-scaled FP16 copy: 16-byte loads of eight entries,
// FP32 sums, one warp per row (n a multiple of 8)
__global__ void k_dense_solve_h(int n, const __half *__restrict__ Ah, const float *__restrict__ sc,
                                const float *__restrict__ r, float *__restrict__ z, const int *stop) {
  PBG_PDL_ENTRY();
  if (stop && *stop) return;
  const int lane = threadIdx.x & 31;
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (row >= n) return;
  const uint4 *ar = reinterpret_cast<const uint4 *>(Ah + (long long)row * n);
  float acc = 0.0f;
  for (int c8 = lane; c8 < n / 8; c8 += 32) {
    const uint4 u = ar[c8];
    const __half2 *h = reinterpret_cast<const __half2 *>(&u);
    const float4 r0 = *reinterpret_cast<const float4 *>(r + c8 * 8);
    const float4 r1 = *reinterpret_cast<const float4 *>(r + c8 * 8 + 4);
    const float2 a0 = __half22float2(h[0]), a1 = __half22float2(h[1]);
    const float2 a2 = __half22float2(h[2]), a3 = __half22float2(h[3]);
    acc += a0.x * r0.x + a0.y * r0.y + a1.x * r0.z + a1.y * r0.w;
    acc += a2.x * r1.x + a2.y * r1.y + a3.x * r1.z + a3.y * r1.w;
  }
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
  if (lane == 0) z[row] = acc * sc[row];
}

// Large coarsest levels in the mixed path apply the FP16 copy (half the
// bytes of the FP32 one) unless PBG_DENSE_HALF=0.
static bool dense_half_enabled() {
  static const bool on = [] {
    const char *e = getenv("PBG_DENSE_HALF");
    return !(e && atoi(e) == 0);
  }();
  return on;
}
constexpr int kDenseHalfMin = 2048;  // coarsest cells from which the FP16 copy is used

__global__ void k_to_float(long long N, const double *__restrict__ a, float *__restrict__ o) {
  GRID_LOOP(p, N) o[p] = (float)a[p];
}

// z = Ainv r on the coarsest level (the FP32 inverse for T = float)
template <typename T>
void Engine::dense_solve(const T *r, T *z, const int *stop, cudaStream_t s) {
  using AT = typename std::conditional<sizeof(T) == 4, float, double>::type;
  const int blocks = (int)(((long long)ncoarse * 32 + kThreads - 1) / kThreads);
  if constexpr (sizeof(T) == 4) {
    if (Ainv16.n) {
      launch_pdl(k_dense_solve_h, blocks, kThreads, s, ncoarse, (const __half *)Ainv16.p,
                 (const float *)Ainv16s.p, (const float *)r, (float *)z, stop);
      return;
    }
  }
  launch_pdl(k_dense_solve<T, AT>, blocks, kThreads, s, ncoarse, (const AT *)ainv<T>(), r, z, stop);
}

void Engine::build(const EMat<double> &A0, cudaStream_t s, bool mixed) {
  w64.drop_graph();
  w32.drop_graph();
  w64.L.clear();
  w32.L.clear();
  L.clear();
  L.emplace_back();
  {
    ELevel &l0 = L[0];
    l0.nx = A0.nx; l0.ny = A0.ny; l0.nz = A0.nz;
    l0.d64.alloc(l0.ncell());
    l0.m64 = make_emat<double>(A0.nx, A0.ny, A0.nz, A0.c, A0.w, A0.s, A0.b, l0.d64.p);
  }
  while (L.back().ncell() > opt.coarse_max &&
         (L.back().nx > 1 || L.back().ny > 1 || L.back().nz > 1)) {
    const ELevel &f = L.back();
    ELevel c;
    c.nx = f.nx > 1 ? (f.nx + 1) / 2 : 1;
    c.ny = f.ny > 1 ? (f.ny + 1) / 2 : 1;
    c.nz = f.nz > 1 ? (f.nz + 1) / 2 : 1;
    long long n = c.ncell();
    c.c64.alloc(n); c.w64.alloc(n); c.s64.alloc(n); c.b64.alloc(n); c.d64.alloc(n);
    c.m64 = make_emat<double>(c.nx, c.ny, c.nz, c.c64.p, c.w64.p, c.s64.p, c.b64.p, c.d64.p);
    L.push_back(std::move(c));
  }
  ncoarse = (int)L.back().ncell();
  Ainv.alloc((size_t)ncoarse * ncoarse);
  if (mixed) Ainv32.alloc((size_t)ncoarse * ncoarse);
  Ainv16.release();
  Ainv16s.release();
  if (mixed && dense_half_enabled() && ncoarse >= kDenseHalfMin && ncoarse % 8 == 0) {
    Ainv16.alloc((size_t)ncoarse * ncoarse);
    Ainv16s.alloc((size_t)ncoarse);
  }
  Dtmp.alloc((size_t)ncoarse * ncoarse);
  have32 = false;
  if (mixed) {
    for (auto &lv : L) {
      long long m = lv.ncell();
      lv.c32.alloc(m); lv.w32.alloc(m); lv.s32.alloc(m); lv.b32.alloc(m); lv.d32.alloc(m);
      lv.m32 = make_emat<float>(lv.nx, lv.ny, lv.nz, lv.c32.p, lv.w32.p, lv.s32.p, lv.b32.p, lv.d32.p);
    }
    have32 = true;
  }
  if (!hsc) PBG_CUDA(cudaMallocHost((void **)&hsc, 64 * sizeof(double)));
  if (dsc.n < 8) dsc.alloc(8);
  compute(s);
  PBG_CUDA(cudaStreamSynchronize(s));
}

// Numeric set-up on the allocated hierarchy, all on the device: inverse
// diagonals, Galerkin coarse operators, FP32 copies and the dense inverse of
// the coarsest level. Used by build() and again after the fine matrix
// changed in place: buffers, and so the captured iteration graphs, stay
// valid. Enqueued on s, no host synchronisation.
void Engine::compute(cudaStream_t s) {
  auto out = [&](ELevel &lv) {
    LevelOut o{const_cast<double *>(lv.m64.c),
               const_cast<double *>(lv.m64.w), const_cast<double *>(lv.m64.s),
               const_cast<double *>(lv.m64.b), lv.d64.p,
               nullptr, nullptr, nullptr, nullptr, nullptr};
    if (have32) { o.c32 = lv.c32.p; o.w32 = lv.w32.p; o.s32 = lv.s32.p; o.b32 = lv.b32.p; o.d32 = lv.d32.p; }
    return o;
  };
  k_level_finish<<<grid_for(L[0].ncell()), kThreads, 0, s>>>(L[0].m64, out(L[0])); note_launch();
  for (size_t l = 1; l < L.size(); ++l) {
    ELevel &c = L[l];
    k_galerkin<<<grid_for(c.ncell()), kThreads, 0, s>>>(L[l - 1].m64, Geo(c.nx, c.ny, c.nz), out(c));
    k_level_finish<<<grid_for(c.ncell()), kThreads, 0, s>>>(c.m64, out(c));
    note_launch(); note_launch();
  }
  // dense inverse of the coarsest operator: blocked Gauss-Jordan, out of place
  const int n = ncoarse;
  const size_t nn = (size_t)n * n;
  PBG_CUDA(cudaMemsetAsync(Dtmp.p, 0, nn * sizeof(double), s));
  k_dense_fill<<<grid_for(n), kThreads, 0, s>>>(L.back().m64, Dtmp.p); note_launch();
  k_dense_dmax<<<1, 1024, 0, s>>>(n, Dtmp.p, dsc.p + 7); note_launch();
  double *src = Dtmp.p, *dst = Ainv.p;
  const int tiles = (n + kGjRows - 1) / kGjRows;
  for (int k0 = 0; k0 < n; k0 += kGjB) {
    k_gj_block<<<tiles, 256, 0, s>>>(n, k0, src, dst, dsc.p + 7, 1e-10); note_launch();
    std::swap(src, dst);
  }
  if (src != Ainv.p)
    PBG_CUDA(cudaMemcpyAsync(Ainv.p, src, nn * sizeof(double), cudaMemcpyDeviceToDevice, s));
  if (have32) {
    k_to_float<<<grid_for((long long)nn), kThreads, 0, s>>>((long long)nn, Ainv.p, Ainv32.p); note_launch();
    if (Ainv16.n) {
      const int blocks = (int)(((long long)ncoarse * 32 + kThreads - 1) / kThreads);
      k_to_half_rows<<<blocks, kThreads, 0, s>>>(ncoarse, Ainv.p, Ainv16.p, Ainv16s.p); note_launch();
    }
  }
  PBG_CUDA(cudaGetLastError());
}

// Numeric refresh for a changed fine matrix of the same shape at the same
// addresses; false if the hierarchy has to be built anew.
bool Engine::refresh(const EMat<double> &A0, bool mixed, cudaStream_t s) {
  if (L.empty() || (mixed && !have32) || L[0].nx != A0.nx || L[0].ny != A0.ny || L[0].nz != A0.nz ||
      L[0].m64.c != A0.c || L[0].m64.w != A0.w || L[0].m64.s != A0.s || L[0].m64.b != A0.b)
    return false;
  compute(s);
  return true;
}

// Preconditioner M r -> z on level l. kc: the K-cycle's second application,
// whose right-hand side r1 = b - a1 q1 is formed (and stored) by k_jac2.
template <typename T>
void Engine::precond(int l, const T *r, T *z, bool dots, const T *u, double *out2, EWork<T> &w,
                     RedPool &red, const int *stop, cudaStream_t s, bool kc) {
  const int last = (int)L.size() - 1;
  const T om = (T)opt.omega;
  auto &v = w.L[l];
  if (l == last) {
    dense_solve<T>(r, z, stop, s);
    if (dots) {  // a level-0 problem small enough to be the coarsest
      EMat<T> A = mat<T>(l);
      PBG_CUDA(cudaMemcpyAsync(v.xa.p, z, sizeof(T) * A.ncell(), cudaMemcpyDeviceToDevice, s));
      // omega = 0 keeps z and computes the dot products
      launch_pdl(k_jac_dots<T>, grid_for(A.ncell()), kThreads, s, A, r, (const T *)v.xa.p, z, T(0), u, out2,
                 red.slot_part(0), red.slot_count(0), stop);
    }
    return;
  }
  EMat<T> A = mat<T>(l);
  const int g = grid_for(A.ncell());
  const ELevel &H = L[l + 1];
  auto &vh = w.L[l + 1];
  const T *rr = kc ? v.r1.p : r;
  const bool vec = A.nz % VecTraits<T>::V == 0;
  const int gv = grid_for(A.ncell() / VecTraits<T>::V, kThreads, kVecBlocks);
  const KScal *ksl = kc ? w.ks.p + l : nullptr;
  const int gw = grid_for(A.ncell() / VecTraits<T>::V, kThreads, kVecWideBlocks<T>);
  launch_pdl(vec ? kv_jac2<T> : k_jac2<T>, vec ? gw : g, kThreads, s, A, r, (const T *)v.b.p,
             (const T *)v.q1.p, ksl, v.r1.p, v.xb.p, om, stop);
  const long long rthreads = H.ncell() >= kRestrictSerialMin ? H.ncell() : H.ncell() * 8;
  launch_pdl(k_resid_restrict<T>, grid_for(rthreads), kThreads, s, A, rr, (const T *)v.xb.p,
             Geo(H.nx, H.ny, H.nz), vh.b.p, stop);
  const T *eH, *z2H = nullptr;
  const KScal *ksH = nullptr;
  if (l + 1 == last) {
    dense_solve<T>(vh.b.p, vh.x.p, stop, s);
    eH = vh.x.p;
  } else {
    if (l + 1 <= opt.kc_max) {
      kcycle<T>(l + 1, w, red, stop, s);
      eH = vh.z1.p; z2H = vh.z2.p; ksH = w.ks.p + l + 1;
    } else {  // one visit: e = M b on level l+1
      precond<T>(l + 1, vh.b.p, vh.z1.p, false, nullptr, nullptr, w, red, stop, s, false);
      eH = vh.z1.p;
    }
  }
  launch_pdl(vec ? kv_prolong_jac<T> : k_prolong_jac<T>, vec ? gv : g, kThreads, s, A, rr,
             (const T *)v.xb.p, H.ny, H.nz, eH, z2H, ksH, v.xa.p, om, stop);
  if (dots && vec && l == 0) {
    // u is the q of the previous FCG iteration, picked by parity on the device
    launch_pdl(kv_jac<T, true>, gv, kThreads, s, A, rr, (const T *)v.xa.p, z, om, (const T *)w.q0.p,
               (const T *)w.q0b.p, (const FcgScal *)w.fs.p, out2, red.slot_part(0), red.slot_count(0), stop);
  } else if (dots) {
    launch_pdl(k_jac_dots<T>, g, kThreads, s, A, rr, (const T *)v.xa.p, z, om, u, out2, red.slot_part(0),
               red.slot_count(0), stop);
  } else if (vec) {
    launch_pdl(kv_jac<T, false>, gv, kThreads, s, A, rr, (const T *)v.xa.p, z, om, (const T *)nullptr,
               (const T *)nullptr, (const FcgScal *)nullptr, (double *)nullptr, (double *)nullptr,
               (unsigned *)nullptr, stop);
  } else {
    launch_pdl(k_jac<T>, g, kThreads, s, A, rr, (const T *)v.xa.p, z, om, stop);
  }
}

template <typename T>
void Engine::kcycle(int l, EWork<T> &w, RedPool &red, const int *stop, cudaStream_t s) {
  EMat<T> A = mat<T>(l);
  const int g = grid_for(A.ncell());
  auto &v = w.L[l];
  KScal *ks = w.ks.p + l;
  precond<T>(l, v.b.p, v.z1.p, false, nullptr, nullptr, w, red, stop, s, false);
  launch_pdl(k_kc_q1<T>, g, kThreads, s, A, (const T *)v.z1.p, (const T *)v.b.p, v.q1.p, ks,
             red.slot_part(0), red.slot_count(0), stop);
  precond<T>(l, nullptr, v.z2.p, false, nullptr, nullptr, w, red, stop, s, true);
  launch_pdl(k_kc_q2<T>, g, kThreads, s, A, (const T *)v.z2.p, (const T *)v.q1.p, (const T *)v.r1.p, v.v.p,
             ks, red.slot_part(0), red.slot_count(0), stop);
}

// Flexible CG on level 0 for A e = b (e starts at zero); returns iterations.
// One iteration (the preconditioner's K-cycle over all levels plus the two
// FCG kernels) is captured once into a CUDA graph and replayed; every kernel
// in it returns at once when the device-side done flag is set.
template <typename T>
int Engine::fcg(EWork<T> &w, const T *b, double tol, int maxit, RedPool &red, cudaStream_t s,
                double *hist, FcgScal *hfs) {
  EMat<T> A = mat<T>(0);
  const long long N = A.ncell();
  const int g = grid_for(N);
  FcgScal *fs = w.fs.p;
  // one FCG iteration: the preconditioner's K-cycle over all levels plus
  // the two FCG kernels; every kernel returns at once when *stop is set
  // (stop == nullptr: no check)
  auto iteration = [&](const int *stop) {
    precond<T>(0, w.r0.p, w.z0.p, true, w.q0.p, &fs->zr, w, red, stop, s, false);
    if (A.nz % VecTraits<T>::V == 0 && (int)L.size() > 1) {
      const int gv = grid_for(N / VecTraits<T>::V, kThreads, kVecBlocks);
      const int gw = grid_for(N / VecTraits<T>::V, kThreads, kVecWideBlocks<T>);
      launch_pdl(kv_fcg_pq<T>, gw, kThreads, s, A, (const T *)w.z0.p, w.pA.p, w.pB.p, w.q0.p, w.q0b.p, fs,
                 red.slot_part(0), red.slot_count(0));
      launch_pdl(kv_fcg_xr<T>, gv, kThreads, s, N, w.x0.p, w.r0.p, (const T *)w.pA.p, (const T *)w.pB.p,
                 (const T *)w.q0.p, (const T *)w.q0b.p, fs, red.slot_part(0), red.slot_count(0));
    } else {
      launch_pdl(k_fcg_pq<T>, g, kThreads, s, A, (const T *)w.z0.p, w.pA.p, w.pB.p, w.q0.p, fs,
                 red.slot_part(0), red.slot_count(0));
      launch_pdl(k_fcg_xr<T>, g, kThreads, s, N, w.x0.p, w.r0.p, (const T *)w.pA.p, (const T *)w.pB.p,
                 (const T *)w.q0.p, fs, red.slot_part(0), red.slot_count(0));
    }
  };
  if (!w.iter_graph) {
    cudaGraph_t graph = nullptr;
    const unsigned long long before = g_launch_count;
    PBG_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    try {
      iteration(&fs->done);
    } catch (...) {
      cudaStreamEndCapture(s, &graph);  // leave the stream usable
      if (graph) cudaGraphDestroy(graph);
      throw;
    }
    PBG_CUDA(cudaStreamEndCapture(s, &graph));
    w.iter_nodes = (size_t)(g_launch_count - before);
    __atomic_sub_fetch(&g_launch_count, (unsigned long long)w.iter_nodes, __ATOMIC_RELAXED);
    PBG_CUDA(cudaGraphInstantiate(&w.iter_graph, graph, 0));
    cudaGraphDestroy(graph);
    if (graph_loop_enabled()) {
      // the same iteration as the body of a WHILE node: a gate kernel sets
      // its condition before the first pass, the last kernel of the body
      // after each pass
      cudaGraph_t lg = nullptr;
      PBG_CUDA(cudaGraphCreate(&lg, 0));
      try {
        cudaGraphConditionalHandle h;
        PBG_CUDA(cudaGraphConditionalHandleCreate(&h, lg, 0, cudaGraphCondAssignDefault));
        cudaKernelNodeParams kp = {};
        const FcgScal *cfs = fs;
        void *kargs[] = {(void *)&h, (void *)&cfs};
        kp.func = (void *)k_fcg_gate;
        kp.gridDim = dim3(1);
        kp.blockDim = dim3(32);
        kp.sharedMemBytes = 0;
        kp.kernelParams = kargs;
        kp.extra = nullptr;
        cudaGraphNode_t gate;
        PBG_CUDA(cudaGraphAddKernelNode(&gate, lg, nullptr, 0, &kp));
        cudaGraphNodeParams np = {};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t node;
        PBG_CUDA(cudaGraphAddNode(&node, lg, &gate, 1, &np));
        cudaGraph_t body = np.conditional.phGraph_out[0];
        PBG_CUDA(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        try {
          iteration(nullptr);
          k_fcg_continue<<<1, 32, 0, s>>>(h, fs);
        } catch (...) {
          cudaStreamEndCapture(s, &body);
          throw;
        }
        PBG_CUDA(cudaStreamEndCapture(s, &body));
        __atomic_sub_fetch(&g_launch_count, (unsigned long long)w.iter_nodes, __ATOMIC_RELAXED);
        PBG_CUDA(cudaGraphInstantiate(&w.loop_graph, lg, 0));
      } catch (...) {
        cudaGraphDestroy(lg);
        throw;
      }
      cudaGraphDestroy(lg);
    }
  }
  PBG_CUDA(cudaMemsetAsync(w.q0.p, 0, sizeof(T) * N, s));
  PBG_CUDA(cudaMemsetAsync(w.q0b.p, 0, sizeof(T) * N, s));
  k_fcg_init<T><<<g, kThreads, 0, s>>>(N, b, w.x0.p, w.r0.p, fs, tol, maxit, hist,
                                       red.slot_part(0), red.slot_count(0)); note_launch();
  PBG_CUDA(cudaGetLastError());
  if (w.loop_graph) {
    PBG_CUDA(cudaGraphLaunch(w.loop_graph, s));
    PBG_CUDA(cudaMemcpyAsync(hfs, fs, sizeof(FcgScal), cudaMemcpyDeviceToHost, s));
    PBG_CUDA(cudaStreamSynchronize(s));
    __atomic_add_fetch(&g_launch_count, (unsigned long long)hfs->loops * (w.iter_nodes + 1) + 1, __ATOMIC_RELAXED);
    return hfs->iter;
  }
  int enq = 0, chunk = 4;
  for (;;) {
    PBG_CUDA(cudaMemcpyAsync(hfs, fs, sizeof(FcgScal), cudaMemcpyDeviceToHost, s));
    PBG_CUDA(cudaStreamSynchronize(s));
    if (hfs->done || enq >= maxit) break;
    int cnt = chunk;
    if (enq + cnt > maxit) cnt = maxit - enq;
    for (int c = 0; c < cnt; ++c) PBG_CUDA(cudaGraphLaunch(w.iter_graph, s));
    __atomic_add_fetch(&g_launch_count, (unsigned long long)(cnt * w.iter_nodes), __ATOMIC_RELAXED);
    enq += cnt;
    if (chunk < 16) chunk *= 2;
  }
  return hfs->iter;
}

// Symmetric approximation of a seven-array operator in the engine's
// storage: each coupling the mean of the two cells' own values (w of a cell
// and e of its west neighbour, and so on), c unchanged; a coupling that only
// one side keeps drops out. That one-sided case is a cell inside a body
// (c = 1e-12 c0, its couplings zeroed) next to a fluid cell off the cut
// list: half the coupling against that tiny diagonal would make the
// approximation indefinite, while in the matrix itself the inside cell's
// value is decoupled. On the reference's cut sphere the refinement around
// it reduces the residual by 1e-2 to 3e-2 per sweep past the first; the
// smaller of the two sides instead (always diagonally dominant) gave 2e-2
// to 4e-2 there but lost the upwind part of a convected matrix, where the
// mean keeps it as a skew term.
__device__ __forceinline__ double sym_coupling(double x, double y) {
  return (x != 0.0 && y != 0.0) ? 0.5 * (x + y) : 0.0;
}

__global__ void k_symmetrize(MatView<double> A, Geo G, double *__restrict__ C, double *__restrict__ W,
                             double *__restrict__ S, double *__restrict__ B) {
  const uint32_t SI = G.nynz, SJ = (uint32_t)A.nz;
  GRID_LOOP(p, G.n) {
    const Pos q = G.pos(p);
    const Nb<double> a = coeffs(A, p, q);
    C[p] = A.c[p];
    W[p] = q.i > 0 ? sym_coupling(a.w, A.e[p - SI]) : 0.0;
    S[p] = q.j > 0 ? sym_coupling(a.s, A.n[p - SJ]) : 0.0;
    B[p] = q.k > 0 ? sym_coupling(a.b, A.t[p - 1]) : 0.0;
  }
}

void symmetrize(const MatView<double> &A, double *c, double *w, double *s, double *b, cudaStream_t st) {
  k_symmetrize<<<grid_for(A.ncell()), kThreads, 0, st>>>(A, Geo(A.nx, A.ny, A.nz), c, w, s, b);
  note_launch();
  PBG_CUDA(cudaGetLastError());
}

// r = b - A x with the operator the solve is for (the symmetric level 0,
// or the seven-array one whose symmetric part the hierarchy holds), its
// rounding into rT, and |r|^2, |b|^2 into dsc[0..1].
template <typename T>
void Engine::true_resid(const double *x, const double *b, T *rT, RedPool &red, cudaStream_t s) {
  const EMat<double> A = L[0].m64;
  const int g = grid_for(A.ncell());
  if (nonsym)
    k_true_resid_ns<T><<<g, kThreads, 0, s>>>(top, A.g, x, b, nullptr, rT, dsc.p, red.slot_part(0),
                                              red.slot_count(0));
  else
    k_true_resid<T><<<g, kThreads, 0, s>>>(A, x, b, nullptr, rT, dsc.p, red.slot_part(0), red.slot_count(0));
  note_launch();
}

// A non-symmetric operator is solved by refinement around its symmetric
// part, which converges only while the asymmetry is mild (a cut body's face
// fractions); with a strong one (convection) a sweep can raise the
// residual. The iterate before each correction is kept, and a sweep that
// does not reduce the residual is undone and ends the solve (ST_DIVERGED).
void Engine::keep_iterate(const double *x, long long N, cudaStream_t s) {
  if (!nonsym) return;
  if (xtmp.n < (size_t)N) xtmp.alloc(N);
  PBG_CUDA(cudaMemcpyAsync(xtmp.p, x, N * sizeof(double), cudaMemcpyDeviceToDevice, s));
}

void Engine::restore_iterate(double *x, long long N, cudaStream_t s) {
  PBG_CUDA(cudaMemcpyAsync(x, xtmp.p, N * sizeof(double), cudaMemcpyDeviceToDevice, s));
  PBG_CUDA(cudaStreamSynchronize(s));
}

EngineResult Engine::solve_fp64(double *x, const double *b, double tol, int maxit, RedPool &red,
                                cudaStream_t s, double *hist) {
  w64.ensure(L);
  const EMat<double> A = L[0].m64;
  const long long N = A.ncell();
  const int g = grid_for(N);
  FcgScal *hfs = (FcgScal *)hsc;
  double *rhs = w64.L[0].b.p;
  EngineResult res{ST_RUNNING, 0, 0, 0, 0.0};
  true_resid<double>(x, b, rhs, red, s);
  PBG_CUDA(cudaMemcpyAsync(hsc + 32, dsc.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
  PBG_CUDA(cudaStreamSynchronize(s));
  double rr = hsc[32], bb = hsc[33];
  if (!(bb > 0.0)) { res.status = ST_INITIAL; res.converged = 1; return res; }
  double rel = std::sqrt(rr / bb);
  // a non-symmetric operator converges by the refinement around its
  // symmetric part: more sweeps
  const int sweeps = nonsym ? 16 : 4;
  for (int sweep = 0; sweep < sweeps && rel > tol; ++sweep) {
    double itol = std::fmin(0.9 * tol / rel, 0.5);
    int its = fcg<double>(w64, rhs, itol, maxit - res.iterations, red, s, hist, hfs);
    res.iterations += its;
    res.sweeps++;
    keep_iterate(x, N, s);
    k_add_corr<double><<<g, kThreads, 0, s>>>(N, x, w64.x0.p); note_launch();
    true_resid<double>(x, b, rhs, red, s);
    PBG_CUDA(cudaMemcpyAsync(hsc + 32, dsc.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    PBG_CUDA(cudaStreamSynchronize(s));
    const double nrel = std::sqrt(hsc[32] / bb);
    if (nonsym && !(nrel < rel)) { restore_iterate(x, N, s); res.status = ST_DIVERGED; break; }
    rel = nrel;
    if (hfs->status == ST_NAN || hfs->status == ST_BREAKDOWN) { res.status = hfs->status; break; }
    if (res.iterations >= maxit) break;
  }
  res.relres = rel;
  if (rel <= tol) { res.converged = 1; res.status = ST_CONVERGED; }
  else if (res.status == ST_RUNNING) res.status = (rel == rel) ? ST_MAXITER : ST_NAN;
  return res;
}

EngineResult Engine::solve_mixed(double *x, const double *b, double tol, double inner_tol,
                                 int max_sweeps, int inner_maxit, RedPool &red, cudaStream_t s,
                                 double *hist) {
  w32.ensure(L);
  const EMat<double> A = L[0].m64;
  const long long N = A.ncell();
  const int g = grid_for(N);
  FcgScal *hfs = (FcgScal *)hsc;
  float *rhs = w32.L[0].b.p;
  EngineResult res{ST_RUNNING, 0, 0, 0, 0.0};
  true_resid<float>(x, b, rhs, red, s);
  PBG_CUDA(cudaMemcpyAsync(hsc + 32, dsc.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
  PBG_CUDA(cudaStreamSynchronize(s));
  double rr = hsc[32], bb = hsc[33];
  if (!(bb > 0.0)) { res.status = ST_INITIAL; res.converged = 1; return res; }
  double rel = std::sqrt(rr / bb);
  for (int sweep = 0; sweep < max_sweeps && rel > tol; ++sweep) {
    // solve no further than the outer target needs in the last sweep
    double itol = std::fmax(inner_tol, 0.9 * tol / rel);
    // history slots this sweep may fill: it < kHistMax in k_fcg_xr, so the
    // offset pointer is passed only while offset + kHistMax stays in bounds
    double *h = (hist && res.iterations == 0) ? hist : nullptr;
    int its = fcg<float>(w32, rhs, itol, inner_maxit, red, s, h, hfs);
    res.iterations += its;
    res.sweeps++;
    keep_iterate(x, N, s);
    k_add_corr<float><<<g, kThreads, 0, s>>>(N, x, w32.x0.p); note_launch();
    true_resid<float>(x, b, rhs, red, s);
    PBG_CUDA(cudaMemcpyAsync(hsc + 32, dsc.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    PBG_CUDA(cudaStreamSynchronize(s));
    double nrel = std::sqrt(hsc[32] / bb);
    if (nonsym && !(nrel < rel)) { restore_iterate(x, N, s); res.status = ST_DIVERGED; break; }
    if (!(nrel == nrel)) { rel = nrel; res.status = ST_NAN; break; }
    if (hfs->status == ST_BREAKDOWN && nrel >= rel) { rel = nrel; res.status = ST_BREAKDOWN; break; }
    rel = nrel;
  }
  res.relres = rel;
  if (rel <= tol) { res.converged = 1; res.status = ST_CONVERGED; }
  else if (res.status == ST_RUNNING) res.status = ST_MAXITER;
  return res;
}

// Times the fine-level smoothing sweep the solver launches: the vectorised
// kv_jac when the rows allow it, else the scalar k_jac.
template <typename T>
static double time_sweeps(const EMat<T> &A, const T *r, T *xa, T *xb, T om, int reps, cudaStream_t s) {
  cudaEvent_t e0, e1;
  PBG_CUDA(cudaEventCreate(&e0));
  PBG_CUDA(cudaEventCreate(&e1));
  const bool vec = A.nz % VecTraits<T>::V == 0;
  const int g = grid_for(A.ncell());
  const int gv = grid_for(A.ncell() / VecTraits<T>::V, kThreads, kVecBlocks);
  auto sweep = [&](const T *xi, T *xo) {
    if (vec)
      kv_jac<T, false><<<gv, kThreads, 0, s>>>(A, r, xi, xo, om, nullptr, nullptr, nullptr, nullptr,
                                               nullptr, nullptr, nullptr);
    else
      k_jac<T><<<g, kThreads, 0, s>>>(A, r, xi, xo, om, nullptr);
    note_launch();
  };
  sweep(xa, xb);
  PBG_CUDA(cudaEventRecord(e0, s));
  for (int q = 0; q < reps; ++q) sweep((q & 1) ? xb : xa, (q & 1) ? xa : xb);
  PBG_CUDA(cudaEventRecord(e1, s));
  PBG_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  PBG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return (double)ms / reps;
}

double Engine::bench_sweep(int precision, int reps, cudaStream_t s) {
  if (precision == 0) {
    w64.ensure(L);
    PBG_CUDA(cudaMemsetAsync(w64.r0.p, 0, sizeof(double) * L[0].ncell(), s));
    PBG_CUDA(cudaMemsetAsync(w64.L[0].xa.p, 0, sizeof(double) * L[0].ncell(), s));
    return time_sweeps<double>(L[0].m64, w64.r0.p, w64.L[0].xa.p, w64.L[0].xb.p, 0.8, reps, s);
  }
  w32.ensure(L);
  PBG_CUDA(cudaMemsetAsync(w32.r0.p, 0, sizeof(float) * L[0].ncell(), s));
  PBG_CUDA(cudaMemsetAsync(w32.L[0].xa.p, 0, sizeof(float) * L[0].ncell(), s));
  return time_sweeps<float>(L[0].m32, w32.r0.p, w32.L[0].xa.p, w32.L[0].xb.p, 0.8f, reps, s);
}

}  // namespace pbg
