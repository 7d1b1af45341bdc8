// Batched engine, host interface (implementation: pbg_batch.cu).
//
// A BatchEngine holds problems (each with its own device arena: FP64
// matrix, hierarchy, inner-precision copies, vectors, right-hand side and
// solution, all resident until the problem is destroyed) and a fixed number
// of slots. A problem attached to a slot is solved by the batch iteration
// together with every other attached problem; a finished problem leaves its
// slot (collect) and keeps its solution on the device, so that the next
// request on it starts from it (warm start). Problems can be attached while
// others are running: new slots start at the next outer iteration.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <memory>
#include <utility>
#include <vector>

namespace pbg {

// Launch shape of the batch kernels (picked by the autotuner).
struct BatchShape {
  int threads = 256;      // threads per CTA
  int tile_cells = 1024;  // cells per tile
  int grid = 148 * 4;     // CTAs of every tile kernel
  int kc_max = 99;        // levels 1..kc_max run a K-cycle, deeper levels one visit
  int tail_cells = 1024;  // levels of at most this many cells run in one CTA per problem (0: none)
};

struct BatchSolveParams {
  double tol = 1e-8;        // FP64 |b - A x| / |b|
  double inner_tol = 1e-3;  // mixed: inner reduction per refinement sweep
  int max_sweeps = 8;       // refinement sweeps at most (plain FP64: 4)
  int max_iter = 500;       // inner iterations at most, all sweeps together
  int inner_max_iter = 500; // inner iterations per sweep
};

struct BatchOutcome {
  int status, converged, iterations, sweeps;
  double relres, relres0;   // FP64 true residual at return / at start
};

class BatchEngineBase {
 public:
  virtual ~BatchEngineBase() {}
  // A new problem (throws on bad sizes or allocation failure); its id.
  virtual int create_problem(int nx, int ny, int nz, double h, const int bc[6]) = 0;
  virtual void destroy_problem(int id) = 0;
  // Device bytes a problem of this size takes (admission control).
  virtual size_t problem_bytes(int nx, int ny, int nz) const = 0;
  virtual int levels(int id) const = 0;
  // Inputs (where: 0 host, 1 device). set_fields / set_matrix mark the
  // hierarchy for recomputation at the next step.
  virtual void set_fields(int id, const double *rho, const uint8_t *solid, int where) = 0;
  virtual void set_matrix(int id, const double *c, const double *w, const double *s,
                          const double *b, int where) = 0;
  virtual void set_rhs(int id, const double *b, int where) = 0;
  virtual void set_x(int id, const double *x, int where) = 0;
  virtual void zero_x(int id) = 0;
  virtual void get_x(int id, double *x, int where) = 0;
  virtual double *device_x(int id) = 0;
  virtual double *device_rhs(int id) = 0;
  // The problem's own field buffers (for inputs made on the device); after
  // writing them, fields_changed marks the matrix for re-assembly.
  virtual double *device_rho(int id) = 0;
  virtual uint8_t *device_solid(int id) = 0;
  virtual void fields_changed(int id) = 0;
  // Attach a problem to a free slot for one solve; the slot, or -1 if none.
  virtual int attach(int id, const BatchSolveParams &p) = 0;
  virtual int free_slots() const = 0;
  virtual int active() const = 0;
  // Set-up of newly attached problems, then `iterations` outer iterations.
  virtual void step(int iterations) = 0;
  // Problems that finished (they leave their slots).
  virtual std::vector<std::pair<int, BatchOutcome>> collect() = 0;
  virtual void set_shape(const BatchShape &s) = 0;
  virtual BatchShape shape() const = 0;
  virtual unsigned long long kernel_launches() const = 0;
  cudaStream_t stream = nullptr;
};

// precision: 1 mixed (FP32 inner), 0 plain FP64.
std::unique_ptr<BatchEngineBase> make_batch_engine(int precision, int slots, const BatchShape &shape);

}  // namespace pbg
