// Common device/host definitions of the B200 pressure-Poisson engine.
//
// Cell layout on the device: interior cells only, index = (i*ny + j)*nz + k
// (k fastest), the interior of the reference's val[i][j][k] block
// (PSI-BOIL Src/Global/global_malloc.cpp:35-56). Out-of-domain neighbours
// contribute nothing: their coefficients are zero after the boundary
// correction (Src/Equation/Centered/centered_system_bnd.cpp), which is what
// the reference's zero-valued halo multiplies.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <stdexcept>
#include <string>
#include <utility>

#include "pbg_exact_sum.cuh"

namespace pbg {

constexpr int kThreads = 256;          // threads per block of the streaming kernels
constexpr int kMaxBlocks = 148 * 8;    // grid cap: 8 blocks of 256 per SM on 148 SMs
constexpr int kStaleMax = 64;          // longest Krylov staleness window kept on device
constexpr int kHistMax = 4096;         // residual history entries kept on device

struct CudaError : std::runtime_error {
  explicit CudaError(const std::string &s) : std::runtime_error(s) {}
};

#define PBG_CUDA(call)                                                              \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess)                                                          \
      throw ::pbg::CudaError(std::string(#call) + ": " + cudaGetErrorString(e_));   \
  } while (0)

// Kernel launches issued by this library (a process-wide counter, read
// through pbg_launch_count); used to report the launches of a timed region.
extern unsigned long long g_launch_count;
inline void note_launch() { __atomic_add_fetch(&g_launch_count, 1ULL, __ATOMIC_RELAXED); }

// Grid of an exact-order reduction: one thread per element.
inline int grid_exact(long long n, int threads = kThreads) {
  long long b = (n + threads - 1) / threads;
  return (int)(b < 1 ? 1 : b);
}

inline int grid_for(long long n, int threads = kThreads, int cap = kMaxBlocks) {
  long long b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return (int)b;
}

// ---------------------------------------------------------------------------
// Programmatic dependent launch. A kernel launched with launch_pdl may be
// scheduled while its predecessor in the stream (or the graph captured from
// it) drains, so that the launch latency of the many small coarse-level
// kernels overlaps the tail of the previous one. Every such kernel starts
// with PBG_PDL_ENTRY: it waits for the predecessor grid to complete and its
// memory to be visible (griddepcontrol.wait, a hardware dependency, not a
// spin) before touching anything, then lets its own successor be scheduled.
// Without the launch attribute both instructions return at once.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
#define PBG_PDL_ENTRY() \
  do {                   \
    ::pbg::pdl_wait();   \
    ::pbg::pdl_trigger(); \
  } while (0)

// PBG_PDL=0 in the environment launches these kernels the ordinary way.
bool pdl_enabled();

template <typename... K, typename... A>
inline void launch_pdl(void (*kern)(K...), int grid, int block, cudaStream_t s, A &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  PBG_CUDA(cudaLaunchKernelEx(&cfg, kern, std::forward<A>(args)...));
  note_launch();
}

// ---------------------------------------------------------------------------
// Matrix views. General storage keeps all seven arrays (the reference's
// Matrix, Src/Matrix/matrix.h:23-54). Symmetric storage keeps c, w, s, b and
// reads e(i) = w(i+1), n(j) = s(j+1), t(k) = b(k+1); it is chosen only when
// the uploaded arrays satisfy those identities bit for bit, so the stencil
// value is unchanged.
// ---------------------------------------------------------------------------
template <typename T>
struct MatView {
  int nx, ny, nz;
  const T *c, *w, *e, *s, *n, *b, *t;   // e, n, t == nullptr: symmetric storage
  int per;   // periodic axes: bit 0 i, bit 1 j, bit 2 k (0 in aggregate initialisers)
  __host__ __device__ long long ncell() const { return (long long)nx * ny * nz; }
};

// Unsigned division by a run-time constant with a multiply-high and a shift
// (Granlund & Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994): for d >= 1 take s = ceil(log2 d) and
// m = floor(2^32 (2^s - d) / d) + 1; then n / d = (umulhi(n, m) + n) >> s
// for every n < 2^31 (the sum stays below 2^32). Cell counts are capped
// at 2^31 per session.
struct FastDiv {
  uint32_t d, m, s;
  FastDiv() : d(1), m(1), s(0) {}
  explicit FastDiv(uint32_t dv) : d(dv) {
    s = 0;
    while ((1ull << s) < dv) ++s;
    m = (uint32_t)((((1ull << 32) * ((1ull << s) - dv)) / dv) + 1);
  }
  __host__ __device__ __forceinline__ uint32_t div(uint32_t n) const {
#ifdef __CUDA_ARCH__
    return (__umulhi(n, m) + n) >> s;
#else
    return (uint32_t)((((uint64_t)n * m) >> 32) + n) >> s;
#endif
  }
};

// Position of a cell from its linear index.
struct Pos { int i, j, k; };
__device__ __forceinline__ Pos pos_of(long long p, int ny, int nz) {
  long long nynz = (long long)ny * nz;
  int i = (int)(p / nynz);
  long long rem = p - (long long)i * nynz;
  int j = (int)(rem / nz);
  int k = (int)(rem - (long long)j * nz);
  return {i, j, k};
}

// Grid geometry with precomputed divisors (cells < 2^31).
struct Geo {
  int nx, ny, nz;
  uint32_t n, nynz;
  FastDiv dnynz, dnz;
  Geo() = default;
  Geo(int x, int y, int z)
      : nx(x), ny(y), nz(z), n((uint32_t)x * y * z), nynz((uint32_t)y * z), dnynz((uint32_t)y * z),
        dnz((uint32_t)z) {}
  __device__ __forceinline__ Pos pos(uint32_t p) const {
    uint32_t i = dnynz.div(p);
    uint32_t rem = p - i * nynz;
    uint32_t j = dnz.div(rem);
    return {(int)i, (int)j, (int)(rem - j * (uint32_t)nz)};
  }
};

// The six neighbour coefficients of cell p (zero outside the domain).
template <typename T>
struct Nb { T w, e, s, n, b, t; };

// Indices of the six neighbours of cell p: -1 across a non-periodic
// boundary face; across a periodic one the cell at the other end, which is
// where the reference's periodic halo copy takes its value from
// (Src/Field/Scalar/scalar_exchange.cpp:47-58).
struct NbIdx { long long w, e, s, n, b, t; };

template <typename T>
__device__ __forceinline__ NbIdx nb_index(const MatView<T> &A, long long p, Pos q) {
  const long long SI = (long long)A.ny * A.nz, SJ = A.nz;
  NbIdx o;
  o.w = q.i > 0 ? p - SI : -1;
  o.e = q.i < A.nx - 1 ? p + SI : -1;
  o.s = q.j > 0 ? p - SJ : -1;
  o.n = q.j < A.ny - 1 ? p + SJ : -1;
  o.b = q.k > 0 ? p - 1 : -1;
  o.t = q.k < A.nz - 1 ? p + 1 : -1;
  if (A.per) {  // uniform: the wrap only for a periodic matrix
    if ((A.per & 1) && q.i == 0) o.w = p + (long long)(A.nx - 1) * SI;
    if ((A.per & 1) && q.i == A.nx - 1) o.e = p - (long long)(A.nx - 1) * SI;
    if ((A.per & 2) && q.j == 0) o.s = p + (long long)(A.ny - 1) * SJ;
    if ((A.per & 2) && q.j == A.ny - 1) o.n = p - (long long)(A.ny - 1) * SJ;
    if ((A.per & 4) && q.k == 0) o.b = p + (long long)(A.nz - 1);
    if ((A.per & 4) && q.k == A.nz - 1) o.t = p - (long long)(A.nz - 1);
  }
  return o;
}

template <typename T>
__device__ __forceinline__ Nb<T> coeffs(const MatView<T> &A, long long p, Pos q) {
  Nb<T> o;
  o.w = A.w[p];
  o.s = A.s[p];
  o.b = A.b[p];
  if (A.e) {
    o.e = A.e[p];
    o.n = A.n[p];
    o.t = A.t[p];
  } else if (!A.per) {
    const long long SI = (long long)A.ny * A.nz, SJ = A.nz;
    o.e = q.i < A.nx - 1 ? A.w[p + SI] : T(0);
    o.n = q.j < A.ny - 1 ? A.s[p + SJ] : T(0);
    o.t = q.k < A.nz - 1 ? A.b[p + 1] : T(0);
  } else {
    const NbIdx m = nb_index(A, p, q);
    o.e = m.e >= 0 ? A.w[m.e] : T(0);
    o.n = m.n >= 0 ? A.s[m.n] : T(0);
    o.t = m.t >= 0 ? A.b[m.t] : T(0);
  }
  return o;
}

// ---------------------------------------------------------------------------
// Deterministic grid reduction: each block reduces its values (fixed warp
// order), writes one partial per value, and the last block to arrive sums
// the partials in block order and runs the finalize step. No spin waits: the
// "last block" is found with one atomic counter that the last block resets.
// ---------------------------------------------------------------------------
struct RedScratch {
  double *part;        // [kRedSlots][kMaxBlocks] partial sums
  unsigned *count;     // [kRedSlots] arrival counters (zero between uses)
};
constexpr int kRedVals = 4;   // values reduced by one kernel at most

template <int NV>
__device__ __forceinline__ void warp_sum(double (&v)[NV]) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1)
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] += __shfl_down_sync(0xffffffffu, v[q], off);
}

// Returns true in thread 0 of the last block; out[] then holds the totals.
//
// Exact-order mode (seq != nullptr, a scratch laid out by
// exact_scratch_doubles): the launch has one thread per element (thread p
// holds element p's term in v) and the result is the reference's sequential
// i,j,k summation (Src/Field/Scalar/scalar.h:296-326) reproduced to the bit,
// computed in parallel by exact_reduce (pbg_exact_sum.cuh). Used by the
// reference-parity solvers on request.
template <int NV>
__device__ bool grid_reduce(double (&v)[NV], double *part, unsigned *count, double (&out)[NV],
                            double *seq = nullptr, long long n = 0) {
  __shared__ double sm[NV][kThreads / 32];
  __shared__ bool last;
  if constexpr (NV <= kExactVals) {
    if (seq && blockDim.x == kExactChunkThreads) return exact_reduce<NV>(v, seq, n, count, out);
  }
  if (seq) {  // other launch shapes: the last block adds every term in order
    const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (p < n)
#pragma unroll
      for (int q = 0; q < NV; ++q) seq[q * n + p] = v[q];
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned prev = atomicAdd(count, 1u);
      last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return false;
    __threadfence();
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double s = 0.0;
      for (long long e = 0; e < n; ++e) s = __dadd_rn(s, __ldcg(&seq[q * n + e]));
      out[q] = s;
    }
    *count = 0u;
    return true;
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  warp_sum<NV>(v);
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NV; ++q) sm[q][wid] = v[q];
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double s = 0.0;
      for (int w = 0; w < nw; ++w) s += sm[q][w];
      part[q * kMaxBlocks + blockIdx.x] = s;
    }
    __threadfence();
    unsigned prev = atomicAdd(count, 1u);
    last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  double acc[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) acc[q] = 0.0;
  for (int bl = threadIdx.x; bl < (int)gridDim.x; bl += blockDim.x)
#pragma unroll
    for (int q = 0; q < NV; ++q) acc[q] += __ldcg(&part[q * kMaxBlocks + bl]);
  warp_sum<NV>(acc);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NV; ++q) sm[q][wid] = acc[q];
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double s = 0.0;
      for (int w = 0; w < nw; ++w) s += sm[q][w];
      out[q] = s;
    }
    *count = 0u;
    return true;
  }
  return false;
}

// Status words shared by all solvers (also the C-ABI result codes).
enum SolveStatus : int {
  ST_RUNNING = -1,
  ST_CONVERGED = 0,
  ST_MAXITER = 1,
  ST_STALE = 2,
  ST_BREAKDOWN = 3,
  ST_INITIAL = 4,     // converged before the first iteration
  ST_NAN = 5,
  ST_DIVERGED = 6,
};

}  // namespace pbg
