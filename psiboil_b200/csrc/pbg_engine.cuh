// Engine solver: flexible CG + additive-correction K-cycle, FP64 and mixed.
#pragma once
#include <cuda_fp16.h>

#include <vector>

#include "pbg_common.cuh"
#include "pbg_session.h"

namespace pbg {

// Symmetric 7-point operator: c, w, s, b (east/north/top from the next cell)
// and the inverse diagonal dinv = 1/c used by the smoother.
template <typename T>
struct EMat {
  int nx, ny, nz;
  Geo g;
  const T *c, *w, *s, *b, *dinv;
  __host__ __device__ long long ncell() const { return (long long)nx * ny * nz; }
};

template <typename T>
inline EMat<T> make_emat(int nx, int ny, int nz, const T *c, const T *w, const T *s, const T *b,
                         const T *dinv) {
  EMat<T> m;
  m.nx = nx; m.ny = ny; m.nz = nz;
  m.g = Geo(nx, ny, nz);
  m.c = c; m.w = w; m.s = s; m.b = b; m.dinv = dinv;
  return m;
}

// Scalars of one K-cycle visit on a coarse level.
struct KScal {
  double zb, zq, a1, beta, a2, pad[3];
};

// Scalars of one flexible-CG solve.
struct FcgScal {
  double zr, zq;          // written together by k_jac_dots (z.r, z.q_old)
  double pr, pq, beta, alpha, rr, rr0, tol;
  int iter, maxit, done, converged, status;
  int loops;              // iterations run by the device-side loop (bounds it)
  double *hist;           // per-iteration |r|/|r0| (kHistMax entries) or null
};

// One aggregation level of the engine hierarchy.
struct ELevel {
  int nx = 0, ny = 0, nz = 0;
  DBuf<double> c64, w64, s64, b64;     // level >= 1 (level 0 borrows the session's)
  DBuf<double> d64;                    // inverse diagonal (every level)
  DBuf<float> c32, w32, s32, b32, d32; // mixed precision copies
  EMat<double> m64{};
  EMat<float> m32{};
  long long ncell() const { return (long long)nx * ny * nz; }
};

// Per-precision work vectors of every level.
template <typename T>
struct EWork {
  struct Lv {
    DBuf<T> b, x, z1, z2, q1, r1, v, xa, xb;
  };
  std::vector<Lv> L;
  DBuf<T> x0, r0, z0, pA, pB, q0, q0b; // outer FCG on level 0 (q0/q0b: q by parity)
  DBuf<KScal> ks;                      // one per level
  DBuf<FcgScal> fs;
  cudaGraphExec_t iter_graph = nullptr;  // one captured FCG iteration
  cudaGraphExec_t loop_graph = nullptr;  // the same iteration in a device-side while loop
  size_t iter_nodes = 0;
  void ensure(const std::vector<ELevel> &lv);
  void drop_graph();
  ~EWork() { drop_graph(); }
};

struct EngineOpts {
  double omega = 0.8;        // damped-Jacobi weight
  int coarse_max = 512;      // coarsest level size (dense direct solve)
  int kc_max = 99;           // levels 1..kc_max run a K-cycle, deeper levels one visit
  EngineOpts();
};

struct EngineResult {
  int status, converged, iterations, sweeps;
  double relres;             // FP64 true residual |b - A x| / |b|
};

class Engine {
 public:
  std::vector<ELevel> L;
  DBuf<double> Ainv;           // dense inverse of the coarsest operator
  DBuf<float> Ainv32;          // its FP32 copy (mixed path)
  DBuf<__half> Ainv16;         // row-scaled FP16 copy (mixed path, large coarsest levels)
  DBuf<float> Ainv16s;         // the row scales
  DBuf<double> Dtmp;           // its Gauss-Jordan work copy
  int ncoarse = 0;
  bool have32 = false;
  EngineOpts opt;
  EWork<double> w64;
  EWork<float> w32;
  DBuf<double> r64, xtmp, dsc; // FP64 refinement residual, scratch, scalars
  double *hsc = nullptr;       // pinned host scalars
  // a non-symmetric operator (seven arrays): the hierarchy is built from its
  // symmetric part, and the refinement's true residual uses this one
  MatView<double> top{};
  bool nonsym = false;

  ~Engine();
  void build(const EMat<double> &A0, cudaStream_t s, bool mixed);
  void compute(cudaStream_t s);
  bool refresh(const EMat<double> &A0, bool mixed, cudaStream_t s);
  // Plain FP64: FCG + FP64 K-cycle to |r|/|b| <= tol.
  EngineResult solve_fp64(double *x, const double *b, double tol, int maxit, RedPool &red,
                          cudaStream_t s, double *hist);
  // Mixed: FP32 FCG + FP32 K-cycle to inner_tol inside FP64 refinement.
  EngineResult solve_mixed(double *x, const double *b, double tol, double inner_tol,
                           int max_sweeps, int inner_maxit, RedPool &red, cudaStream_t s,
                           double *hist);
  int nlevels() const { return (int)L.size(); }
  template <typename T> EMat<T> mat(int l) const;
  template <typename T> const void *ainv() const;
  template <typename T> void dense_solve(const T *r, T *z, const int *stop, cudaStream_t s);
  // Average duration (ms) of the fine-level smoothing sweep, `reps` launches
  // back to back between CUDA events on stream s; precision 0 FP64, 1 FP32.
  double bench_sweep(int precision, int reps, cudaStream_t s);

 private:
  template <typename T> void precond(int l, const T *r, T *z, bool dots, const T *u, double *out2,
                                     EWork<T> &w, RedPool &red, const int *stop, cudaStream_t s,
                                     bool kc);
  template <typename T> void kcycle(int l, EWork<T> &w, RedPool &red, const int *stop, cudaStream_t s);
  template <typename T> int fcg(EWork<T> &w, const T *b, double tol, int maxit, RedPool &red,
                                cudaStream_t s, double *hist, FcgScal *hfs);
  template <typename T> void true_resid(const double *x, const double *b, T *rT, RedPool &red,
                                        cudaStream_t s);
  void keep_iterate(const double *x, long long N, cudaStream_t s);
  void restore_iterate(double *x, long long N, cudaStream_t s);
};

// The symmetric part of a seven-array operator in the engine's storage
// c, w, s, b (k_symmetrize), enqueued on st.
void symmetrize(const MatView<double> &A, double *c, double *w, double *s, double *b, cudaStream_t st);

}  // namespace pbg
