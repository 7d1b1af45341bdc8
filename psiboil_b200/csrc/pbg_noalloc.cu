// pbg_dot_noalloc: the dot-product entry point for callers that cannot
// allocate GPU memory.
//
// pbg_dot (pbg_capi.cu) reduces through per-block partial sums and an
// arrival counter that live in the session's scratch, which the session
// allocates with cudaMalloc. Some callers cannot allocate at the point where
// they need a dot product: a host code that hands the whole device memory to
// its own pool when it starts (a further cudaMalloc fails, or takes memory
// the pool counted on), or a time-step loop that must not take an
// allocation's latency, its device-wide synchronisation or its failure path
// in the middle of a step. This variant takes device inputs and a device
// output and keeps its scratch in a fixed file-scope __device__ array
// instead, so it calls no cudaMalloc, cudaFree or allocating library routine.
//
// Limits and sharing: the scratch holds one partial sum per block for two
// values (kMaxBlocks blocks), so any n up to 2^31 - 1 elements fits; larger
// n is rejected. Every GPU that loads the library holds the array (about
// 19 KB) until the process exits. Every call on a device shares it and it
// keeps the last call's contents: the arrival counter, which must start at
// zero, is cleared at the start of each call; calls that overlap on the GPU
// (on different streams, or from different host threads) race on the
// array and give wrong results — serialise them.
//
// Set-up: the first call on a device, with that device current, looks up
// the array's device address with cudaGetSymbolAddress (a host-side name of
// a __device__ variable is not a device address) and keeps it for later
// calls; a look-up that fails is retried by the next call. Make the first
// call on each device before any stream capture.
#include <mutex>

#include "../../include/psiboil_b200.h"
#include "pbg_common.cuh"

namespace pbg {

// partial sums (2 values x kMaxBlocks blocks) and the arrival counter
static __device__ __align__(256) double g_noalloc_part[2 * kMaxBlocks];
static __device__ __align__(256) unsigned g_noalloc_count[4];

// Same arithmetic as k_dot2 (reference-parity dot products,
// Src/Field/Scalar/scalar.h:296-326): out[0] = sum x*y,
// out[1] = sum x*y/dV/dV / n / n.
__global__ void __launch_bounds__(kThreads, 8)
    k_dot2_noalloc(long long N, const double *__restrict__ x, const double *__restrict__ y,
                   double dV, double *part, unsigned *count, double *out) {
  double v[2] = {0.0, 0.0};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    v[0] += __dmul_rn(x[p], y[p]);
    v[1] += __ddiv_rn(__ddiv_rn(__dmul_rn(x[p], y[p]), dV), dV);
  }
  double o[2];
  if (grid_reduce<2>(v, part, count, o)) {
    const double n = (double)N;
    out[0] = o[0];
    out[1] = o[1] / n / n;
  }
}

// the C ABI's per-thread error message (pbg_last_error), pbg_capi.cu
void set_last_error(const char *msg);

namespace {

constexpr int kMaxDevices = 64;
double *g_part_addr[kMaxDevices];
unsigned *g_count_addr[kMaxDevices];
bool g_ready[kMaxDevices];
std::mutex g_setup_mutex;

int err(int code, const char *m) {
  set_last_error(m);
  return code;
}

}  // namespace
}  // namespace pbg

extern "C" int pbg_dot_noalloc(const double *x, const double *y, long long n, double dV,
                               double *out, void *stream) {
  using namespace pbg;
  if (!x || !y || !out) return err(PBG_ERR_ARG, "pbg_dot_noalloc: NULL argument");
  if (n < 1 || n > 2147483647LL)
    return err(PBG_ERR_ARG, "pbg_dot_noalloc: n must be in [1, 2^31 - 1] (fixed scratch and 32-bit grid)");
  if (!(dV > 0.0)) return err(PBG_ERR_ARG, "pbg_dot_noalloc: dV must be > 0");
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return err(PBG_ERR_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return err(PBG_ERR_UNSUPPORTED, "pbg_dot_noalloc: device index too large");
  // once per device, with that device current: the array's device address
  // (marked ready only after both look-ups succeed, so a failure is retried)
  {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_ready[dev]) {
      double *pa = nullptr;
      unsigned *ca = nullptr;
      e = cudaGetSymbolAddress((void **)&pa, g_noalloc_part);
      if (e == cudaSuccess) e = cudaGetSymbolAddress((void **)&ca, g_noalloc_count);
      if (e != cudaSuccess) {
        cudaGetLastError();
        return err(PBG_ERR_CUDA, cudaGetErrorString(e));
      }
      g_part_addr[dev] = pa;
      g_count_addr[dev] = ca;
      g_ready[dev] = true;
    }
  }
  cudaStream_t s = (cudaStream_t)stream;
  // the arrival counter must start at zero
  e = cudaMemsetAsync(g_count_addr[dev], 0, sizeof(unsigned), s);
  if (e != cudaSuccess) return err(PBG_ERR_CUDA, cudaGetErrorString(e));
  k_dot2_noalloc<<<grid_for(n), kThreads, 0, s>>>(n, x, y, dV, g_part_addr[dev], g_count_addr[dev], out);
  e = cudaGetLastError();
  if (e != cudaSuccess) return err(PBG_ERR_CUDA, cudaGetErrorString(e));
  return PBG_OK;
}
