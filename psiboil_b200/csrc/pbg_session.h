// Internal host-side structures of the engine (not part of the C-ABI).
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <vector>

#include "pbg_common.cuh"

namespace pbg {

// Owning device allocation.
template <typename T>
struct DBuf {
  T *p = nullptr;
  size_t n = 0;
  DBuf() = default;
  explicit DBuf(size_t count) { alloc(count); }
  DBuf(const DBuf &) = delete;
  DBuf &operator=(const DBuf &) = delete;
  DBuf(DBuf &&o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  DBuf &operator=(DBuf &&o) noexcept {
    if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
    return *this;
  }
  ~DBuf() { release(); }
  void alloc(size_t count) {
    release();
    n = count;
    if (count) PBG_CUDA(cudaMalloc((void **)&p, sizeof(T) * (count ? count : 1)));
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  size_t bytes() const { return n * sizeof(T); }
};

// Device-resident scalar state of one Krylov solve (CG / BiCGS / FCG).
struct KrylovState {
  // parameters
  double res_rat, res_tol, scale, dV, ncell;
  int mini, maxit, stalecount, hist_cap;
  // running values
  double rho, rho_old, alfa, beta, omega, pq, res, res0, rr0, aux0, aux1;
  int iter, done, converged, status, iterations, pending_x, pad0, pad1;
  double *seq;   // exact-order reduction terms (null: tree reduction)
  double stale[kStaleMax];
};

// Reduction scratch: partial sums and arrival counters, one slot per
// concurrently pending reduction.
constexpr int kRedSlots = 8;
struct RedPool {
  DBuf<double> part;     // kRedSlots * kRedVals * kMaxBlocks
  DBuf<unsigned> count;  // kRedSlots
  void init() {
    part.alloc((size_t)kRedSlots * kRedVals * kMaxBlocks);
    count.alloc(kRedSlots);
    PBG_CUDA(cudaMemset(count.p, 0, count.bytes()));
  }
  double *slot_part(int s) const { return part.p + (size_t)s * kRedVals * kMaxBlocks; }
  unsigned *slot_count(int s) const { return count.p + s; }
};

// Full seven-array FP64 matrix on the device (general storage), or the
// four-array symmetric form when the upload passes the symmetry check.
struct Mat64 {
  int nx = 0, ny = 0, nz = 0;
  bool sym = false;
  int per = 0;   // periodic axes (bit 0 i, 1 j, 2 k)
  DBuf<double> c, w, e, s, n, b, t;
  MatView<double> view() const {
    return {nx, ny, nz, c.p, w.p, sym ? nullptr : e.p, s.p, sym ? nullptr : n.p, b.p,
            sym ? nullptr : t.p, per};
  }
  long long ncell() const { return (long long)nx * ny * nz; }
};

}  // namespace pbg
