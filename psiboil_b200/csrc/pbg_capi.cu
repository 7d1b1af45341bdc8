// C ABI of the engine: sessions, uploads, on-device pressure assembly and
// the solver entry points. No torch types; plain pointers and sizes.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/psiboil_b200.h"
#include "pbg_assemble.cuh"
#include "pbg_engine.cuh"
#include "pbg_flow.cuh"
#include "pbg_ref_kernels.cuh"
#include "problem_gen.h"

using namespace pbg;

static thread_local std::string g_err;
namespace pbg {
unsigned long long g_launch_count = 0;
void set_last_error(const char *msg) { g_err = msg; }
}

struct pbg_session {
  int device = 0;
  cudaStream_t stream = nullptr;
  int nx = 0, ny = 0, nz = 0;
  double h = 0.0, dV = 0.0;
  int bc[6] = {0, 0, 0, 0, 0, 0};
  int per = 0;                     // periodic axes (bit 0 i, 1 j, 2 k)
  Mat64 A;
  bool have_matrix = false;
  DBuf<uint8_t> aflag;
  RedPool red;
  DBuf<KrylovState> kst;
  KrylovState *hkst = nullptr;
  RefKrylovWork rkw;
  std::unique_ptr<RefAC> refac;
  bool refac_dirty = true;
  std::unique_ptr<Engine> eng;
  bool eng_dirty = true, eng_mixed = false;
  DBuf<double> dx, db, dscal, hist, seq;
  DBuf<double> frhs;               // pressure-step right-hand side (ncell)
  DBuf<double> ci;                 // uploaded A.ci (Jacobi, Gauss-Seidel)
  // immersed body with cut cells (pbg_body_upload): off cells, the index of
  // each cut cell in bfs (-1: not cut) and six face fractions per cut cell
  DBuf<uint8_t> boff;
  DBuf<int> bidx;
  DBuf<double> bfs;
  long long ncut = 0;
  // symmetric part of a non-symmetric matrix, the engine's hierarchy input
  DBuf<double> symc, symw, syms, symb;
  unsigned long long mat_gen = 0, ci_gen = ~0ull;  // ci is valid while ci_gen == mat_gen
  DBuf<unsigned long long> dlinf;
  double *hbuf = nullptr;          // pinned: 64 doubles
  double *px = nullptr, *pb = nullptr;  // pinned staging (ncell each)
  std::vector<double> hhist;
  int nhist = 0;
  long long ncell() const { return (long long)nx * ny * nz; }
};

namespace {

// Geometry with 32-bit division for the flow kernels (n = 0 above 2^31
// cells selects their 64-bit path).
Geo flow_geo(const pbg_session *s) {
  if (s->ncell() >= (1ll << 31)) {
    Geo g;
    g.n = 0;
    return g;
  }
  return Geo(s->nx, s->ny, s->nz);
}

// The flow kernels that own 4 cells of a k-row per thread (the divergence's
// row form and the marching assembly and projection) take grids with
// nz % 4 == 0 below 2^31 cells, no cut body and a marching grid within the
// launch limits; PBG_FLOW_SCALAR=1 selects the one-cell kernels (the same
// bits).
bool flow_vec(const pbg_session *s, bool cut) {
  static const bool scalar = [] {
    const char *e = std::getenv("PBG_FLOW_SCALAR");
    return e && e[0] == '1';
  }();
  return !scalar && !cut && s->nz % kFlowV == 0 && s->ncell() < (1ll << 31) &&
         march_fits(s->nx, s->ny, s->nz);
}

int fail(int code, const std::string &m) {
  g_err = m;
  return code;
}

// The solid mask and cut-cell data a flow kernel gets: the caller's voxel
// mask, or the session's body when it has cut cells (a body without cut
// cells changes nothing in the reference: every body branch is guarded by
// nccells() > 0).
struct BodyArgs {
  const uint8_t *off = nullptr;
  const int *idx = nullptr;
  const double *fs = nullptr;
};
int body_args(const pbg_session *s, const uint8_t *solid_dev, BodyArgs &b) {
  b.off = solid_dev;
  if (s->ncut == 0) return PBG_OK;
  if (solid_dev) return fail(PBG_ERR_ARG, "the session holds a body: pass solid = NULL");
  b.off = s->boff.p;
  b.idx = s->bidx.p;
  b.fs = s->bfs.p;
  return PBG_OK;
}


template <typename F>
int guard(pbg_session *s, F &&f) {
  try {
    if (s) PBG_CUDA(cudaSetDevice(s->device));
    return f();
  } catch (const CudaError &e) {
    return fail(PBG_ERR_CUDA, e.what());
  } catch (const std::bad_alloc &) {
    return fail(PBG_ERR_NOMEM, "host allocation failed");
  } catch (const std::exception &e) {
    return fail(PBG_ERR_STATE, e.what());
  }
}

// (i,j,k) interior of a strided array -> compact
template <typename T, typename U>
void gather(const T *src, U *dst, int nx, int ny, int nz, long long si, long long sj, long long sk,
            long long off) {
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k)
        dst[((size_t)i * ny + j) * nz + k] = (U)src[off + i * si + j * sj + k * sk];
}

__global__ void k_gather(const double *__restrict__ src, double *__restrict__ dst, int nx, int ny,
                         int nz, long long si, long long sj, long long sk, long long off) {
  const long long N = (long long)nx * ny * nz;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    Pos q = pos_of(p, ny, nz);
    dst[p] = src[off + q.i * si + q.j * sj + q.k * sk];
  }
}
__global__ void k_scatter(const double *__restrict__ src, double *__restrict__ dst, int nx, int ny,
                          int nz, long long si, long long sj, long long sk, long long off) {
  const long long N = (long long)nx * ny * nz;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    Pos q = pos_of(p, ny, nz);
    dst[off + q.i * si + q.j * sj + q.k * sk] = src[p];
  }
}

// On-device fixture assembly (one thread per cell, assemble_cell).
__global__ void k_assemble(int nx, int ny, int nz, double h, int4 bc03, int2 bc45,
                           const double *__restrict__ rho, const uint8_t *__restrict__ solid,
                           double *__restrict__ C, double *__restrict__ W, double *__restrict__ S,
                           double *__restrict__ B, uint8_t *__restrict__ aflag) {
  const long long N = (long long)nx * ny * nz;
  const int bc[6] = {bc03.x, bc03.y, bc03.z, bc03.w, bc45.x, bc45.y};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    Pos q = pos_of(p, ny, nz);
    double c, w, sv, b;
    assemble_cell(nx, ny, nz, h, bc, rho, solid, p, q, c, w, sv, b);
    C[p] = c;
    W[p] = w;
    S[p] = sv;
    B[p] = b;
    aflag[p] = solid[p] ? 0 : 1;
  }
}

// Host buffers: pinned ones (cudaMallocHost, cudaHostRegister, torch's
// pin_memory) are copied by DMA directly; pageable ones go through the
// session's pinned staging in chunks, the host copy of chunk k+1 (split over
// a few threads) overlapping the DMA of chunk k.
bool is_pinned(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

constexpr size_t kStageChunk = 16u << 20;

void par_memcpy(void *dst, const void *src, size_t n) {
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t parts = std::min<size_t>({8, hw, n / (2u << 20)});
  if (parts <= 1) {
    std::memcpy(dst, src, n);
    return;
  }
  const size_t step = (n / parts + 63) & ~size_t(63);
  std::vector<std::thread> th;
  for (size_t q = 1; q < parts; ++q) {
    const size_t off = q * step;
    if (off >= n) break;
    th.emplace_back([=] { std::memcpy((char *)dst + off, (const char *)src + off, std::min(step, n - off)); });
  }
  std::memcpy(dst, src, std::min(step, n));
  for (auto &t : th) t.join();
}

// host -> device of n bytes; stage: pinned scratch of at least n bytes
void h2d(pbg_session *s, void *dev, const void *host, size_t n, void *stage) {
  if (is_pinned(host)) {
    PBG_CUDA(cudaMemcpyAsync(dev, host, n, cudaMemcpyHostToDevice, s->stream));
    return;
  }
  for (size_t off = 0; off < n; off += kStageChunk) {
    const size_t len = std::min(kStageChunk, n - off);
    par_memcpy((char *)stage + off, (const char *)host + off, len);
    PBG_CUDA(cudaMemcpyAsync((char *)dev + off, (char *)stage + off, len, cudaMemcpyHostToDevice, s->stream));
  }
}

// device -> host of n bytes (returns with the data on the host)
void d2h(pbg_session *s, void *host, const void *dev, size_t n, void *stage) {
  if (is_pinned(host)) {
    PBG_CUDA(cudaMemcpyAsync(host, dev, n, cudaMemcpyDeviceToHost, s->stream));
    PBG_CUDA(cudaStreamSynchronize(s->stream));
    return;
  }
  std::vector<cudaEvent_t> ev;
  for (size_t off = 0; off < n; off += kStageChunk) {
    const size_t len = std::min(kStageChunk, n - off);
    PBG_CUDA(cudaMemcpyAsync((char *)stage + off, (const char *)dev + off, len, cudaMemcpyDeviceToHost, s->stream));
    cudaEvent_t e;
    PBG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    PBG_CUDA(cudaEventRecord(e, s->stream));
    ev.push_back(e);
  }
  size_t k = 0;
  cudaError_t err = cudaSuccess;
  for (size_t off = 0; off < n; off += kStageChunk, ++k) {
    if (err == cudaSuccess) err = cudaEventSynchronize(ev[k]);
    if (err == cudaSuccess) par_memcpy((char *)host + off, (char *)stage + off, std::min(kStageChunk, n - off));
  }
  for (cudaEvent_t e : ev) cudaEventDestroy(e);
  PBG_CUDA(err);
}

void ensure_staging(pbg_session *s) {
  if (!s->px) {
    PBG_CUDA(cudaMallocHost((void **)&s->px, sizeof(double) * s->ncell()));
    PBG_CUDA(cudaMallocHost((void **)&s->pb, sizeof(double) * s->ncell()));
  }
  if (s->dx.n == 0) { s->dx.alloc(s->ncell()); s->db.alloc(s->ncell()); }
}

void invalidate(pbg_session *s) {
  s->refac_dirty = true;
  s->eng_dirty = true;
}

}  // namespace

extern "C" {

const char *pbg_last_error(void) { return g_err.c_str(); }
int pbg_version(void) { return PBG_API_VERSION; }

int pbg_device_count(int *count) {
  if (!count) return fail(PBG_ERR_ARG, "count is NULL");
  cudaError_t e = cudaGetDeviceCount(count);
  if (e != cudaSuccess) { *count = 0; return fail(PBG_ERR_CUDA, cudaGetErrorString(e)); }
  return PBG_OK;
}

void pbg_params_default(pbg_params *p, int solver) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->solver = solver;
  p->precision = PBG_FP64;
  p->min_iter = 1;
  p->max_iter = 20;
  p->res_rat = 0.01;
  p->res_tol = 1.0e-15;
  p->scale = 1.0;
  p->stalecount = -1;
  p->init_cycle = PBG_CYCLE_NONE;
  p->loop_cycle = PBG_CYCLE_V;
  p->toler = -1.0;
  p->factor = 0.01;
  p->max_cycles = 20;
  p->min_cycles = 0;
  p->stop_if_div = 1;
  p->priority_min_cyc = 1;
  for (int q = 0; q < 3; ++q) { p->mv[q] = 20; p->ms[q] = -1; }
  p->tol = 1.0e-8;
  p->inner_tol = 1.0e-3;
  p->max_sweeps = 8;
  p->ac_smoother = PBG_SOLVER_CG;
  p->ac_solver = -1;
  p->ac_resrat = 1.0e-18;
  p->ac_restol = 1.0e-18;
  p->flex_visits = 1000000;
  p->ac_dt = 1.0;
  if (solver == PBG_SOLVER_ENGINE) p->max_iter = 500;
}

int pbg_session_create(int nx, int ny, int nz, double h, const int bc[6], int device,
                       pbg_session **out) {
  if (!out) return fail(PBG_ERR_ARG, "out is NULL");
  *out = nullptr;
  if (nx < 1 || ny < 1 || nz < 1 || !(h > 0.0))
    return fail(PBG_ERR_ARG, "grid dimensions must be >= 1 and h > 0");
  if ((long long)nx * ny * nz > (1LL << 31))
    return fail(PBG_ERR_ARG, "more than 2^31 cells in one session");
  auto s = std::make_unique<pbg_session>();
  s->device = device;
  s->nx = nx; s->ny = ny; s->nz = nz; s->h = h;
  s->dV = (h * h) * h;
  if (bc) for (int f = 0; f < 6; ++f) s->bc[f] = bc[f];
  for (int f = 0; f < 6; ++f)
    if (s->bc[f] != PBG_BC_NEUMANN_ && s->bc[f] != PBG_BC_DIRICHLET_ && s->bc[f] != PBG_BC_PERIODIC_)
      return fail(PBG_ERR_ARG, "boundary types are PBG_BC_NEUMANN_, PBG_BC_DIRICHLET_ or PBG_BC_PERIODIC_");
  for (int d = 0; d < 3; ++d) {
    const bool a = s->bc[2 * d] == PBG_BC_PERIODIC_, b2 = s->bc[2 * d + 1] == PBG_BC_PERIODIC_;
    if (a != b2) return fail(PBG_ERR_ARG, "a periodic axis needs PBG_BC_PERIODIC_ on both of its faces");
    if (a) s->per |= 1 << d;
  }
  int rc = guard(s.get(), [&]() -> int {
    PBG_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    s->red.init();
    s->kst.alloc(1);
    PBG_CUDA(cudaMallocHost((void **)&s->hkst, sizeof(KrylovState)));
    PBG_CUDA(cudaMallocHost((void **)&s->hbuf, 64 * sizeof(double)));
    s->aflag.alloc(s->ncell());
    PBG_CUDA(cudaMemset(s->aflag.p, 1, s->ncell()));
    s->dscal.alloc(8);
    s->dlinf.alloc(1);
    s->hist.alloc(kHistMax);
    return PBG_OK;
  });
  if (rc != PBG_OK) return rc;
  *out = s.release();
  return PBG_OK;
}

int pbg_session_destroy(pbg_session *s) {
  if (!s) return PBG_OK;
  int rc = guard(s, [&]() -> int {
    if (s->stream) cudaStreamSynchronize(s->stream);
    s->eng.reset();
    s->refac.reset();
    if (s->hkst) cudaFreeHost(s->hkst);
    if (s->hbuf) cudaFreeHost(s->hbuf);
    if (s->px) cudaFreeHost(s->px);
    if (s->pb) cudaFreeHost(s->pb);
    s->hkst = nullptr; s->hbuf = s->px = s->pb = nullptr;
    return PBG_OK;
  });
  cudaStream_t st = s->stream;
  delete s;
  if (st) cudaStreamDestroy(st);
  return rc;
}

}  // extern "C"

extern "C" {

int pbg_session_info(const pbg_session *s, long long *ncell, int *symmetric, long long *device_bytes) {
  if (!s) return fail(PBG_ERR_ARG, "session is NULL");
  if (ncell) *ncell = s->ncell();
  if (symmetric) *symmetric = s->A.sym ? 1 : 0;
  if (device_bytes) {
    size_t b = s->A.c.bytes() + s->A.w.bytes() + s->A.e.bytes() + s->A.s.bytes() + s->A.n.bytes() +
               s->A.b.bytes() + s->A.t.bytes() + s->aflag.bytes() + s->dx.bytes() + s->db.bytes() +
               s->ci.bytes() + s->boff.bytes() + s->bidx.bytes() + s->bfs.bytes() + s->symc.bytes() +
               s->symw.bytes() + s->syms.bytes() + s->symb.bytes();
    *device_bytes = (long long)b;
  }
  return PBG_OK;
}

int pbg_session_set_cell_volume(pbg_session *s, double dV) {
  if (!s || !(dV > 0.0)) return fail(PBG_ERR_ARG, "bad cell volume");
  s->dV = dV;
  return PBG_OK;
}

// Checks of an uploaded seven-array matrix, one thread per cell: bit 0 of
// *flags when the symmetric form does not hold (e(i) == w(i+1), n(j) ==
// s(j+1), t(k) == b(k+1) bit for bit, across a periodic face with the cell
// at the other end, and zero on a non-periodic outer face), bit 1 when a
// coupling across a non-periodic outer face is non-zero.
__global__ void k_mat_check(MatView<double> A, unsigned *flags) {
  const long long N = A.ncell();
  unsigned f = 0;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    const Pos q = pos_of(p, A.ny, A.nz);
    const NbIdx m = nb_index(A, p, q);
    const double ee = m.e >= 0 ? A.w[m.e] : 0.0;
    const double nn = m.n >= 0 ? A.s[m.n] : 0.0;
    const double tt = m.t >= 0 ? A.b[m.t] : 0.0;
    if (__double_as_longlong(ee) != __double_as_longlong(A.e[p]) ||
        __double_as_longlong(nn) != __double_as_longlong(A.n[p]) ||
        __double_as_longlong(tt) != __double_as_longlong(A.t[p]))
      f |= 1u;
    if ((m.w < 0 && A.w[p] != 0.0) || (m.e < 0 && A.e[p] != 0.0) || (m.s < 0 && A.s[p] != 0.0) ||
        (m.n < 0 && A.n[p] != 0.0) || (m.b < 0 && A.b[p] != 0.0) || (m.t < 0 && A.t[p] != 0.0))
      f |= 2u;
  }
  for (int off = 16; off > 0; off >>= 1) f |= __shfl_down_sync(0xffffffffu, f, off);
  if ((threadIdx.x & 31) == 0 && f) atomicOr(flags, f);
}

// One compact device array from a caller array: a straight copy for the
// compact layout, else a gather (host arrays through a staging vector).
static void upload_compact(pbg_session *s, const double *src, double *dst, long long si, long long sj,
                           long long sk, long long offset, int where) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  const long long N = s->ncell();
  const bool compact = si == (long long)ny * nz && sj == nz && sk == 1;
  if (where == PBG_HOST) {
    if (compact) {
      PBG_CUDA(cudaMemcpyAsync(dst, src + offset, N * 8, cudaMemcpyHostToDevice, s->stream));
    } else {
      std::vector<double> h(N);
      gather(src, h.data(), nx, ny, nz, si, sj, sk, offset);
      PBG_CUDA(cudaMemcpyAsync(dst, h.data(), N * 8, cudaMemcpyHostToDevice, s->stream));
      PBG_CUDA(cudaStreamSynchronize(s->stream));
    }
  } else if (compact) {
    PBG_CUDA(cudaMemcpyAsync(dst, src + offset, N * 8, cudaMemcpyDeviceToDevice, s->stream));
  } else {
    k_gather<<<grid_for(N), kThreads, 0, s->stream>>>(src, dst, nx, ny, nz, si, sj, sk, offset); note_launch();
  }
}

int pbg_matrix_upload(pbg_session *s, const double *c, const double *w, const double *e,
                      const double *sv, const double *n, const double *b, const double *t,
                      long long si, long long sj, long long sk, long long offset, int where) {
  if (!s || !c || !w || !e || !sv || !n || !b || !t) return fail(PBG_ERR_ARG, "NULL argument");
  return guard(s, [&]() -> int {
    const long long N = s->ncell();
    Mat64 &A = s->A;
    A.nx = s->nx; A.ny = s->ny; A.nz = s->nz;
    A.per = s->per;
    // same-size uploads keep the buffers (the engine then refreshes in place)
    if (A.c.n != (size_t)N) { A.c.alloc(N); A.w.alloc(N); A.s.alloc(N); A.b.alloc(N); }
    if (A.e.n != (size_t)N) { A.e.alloc(N); A.n.alloc(N); A.t.alloc(N); }
    const double *src[7] = {c, w, e, sv, n, b, t};
    DBuf<double> *dst[7] = {&A.c, &A.w, &A.e, &A.s, &A.n, &A.b, &A.t};
    for (int q = 0; q < 7; ++q) upload_compact(s, src[q], dst[q]->p, si, sj, sk, offset, where);
    // symmetry and outer faces, checked on the device
    PBG_CUDA(cudaMemsetAsync(s->dlinf.p, 0, sizeof(unsigned long long), s->stream));
    A.sym = false;
    k_mat_check<<<grid_for(N), kThreads, 0, s->stream>>>(A.view(), (unsigned *)s->dlinf.p); note_launch();
    PBG_CUDA(cudaMemcpyAsync(s->hbuf, s->dlinf.p, 8, cudaMemcpyDeviceToHost, s->stream));
    PBG_CUDA(cudaStreamSynchronize(s->stream));
    unsigned flags = 0;
    std::memcpy(&flags, s->hbuf, sizeof(flags));
    if (flags & 2u) {
      s->have_matrix = false;
      return fail(PBG_ERR_UNSUPPORTED,
                  "the matrix couples a cell across a non-periodic outer face (apply the boundary "
                  "correction first, or create the session with periodic boundaries on that axis)");
    }
    A.sym = !(flags & 1u);
    if (A.sym) { A.e.release(); A.n.release(); A.t.release(); }
    s->have_matrix = true;
    ++s->mat_gen;
    invalidate(s);
    return PBG_OK;
  });
}

int pbg_matrix_download(pbg_session *s, double *c, double *w, double *e, double *sv, double *n,
                        double *b, double *t, int where) {
  if (!s) return fail(PBG_ERR_ARG, "session is NULL");
  if (!s->have_matrix) return fail(PBG_ERR_STATE, "no matrix");
  return guard(s, [&]() -> int {
    const long long N = s->ncell();
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const long long SI = (long long)ny * nz, SJ = nz;
    std::vector<double> h(7 * N, 0.0);
    const Mat64 &A = s->A;
    const double *src[7] = {A.c.p, A.w.p, A.e.p, A.s.p, A.n.p, A.b.p, A.t.p};
    for (int q = 0; q < 7; ++q)
      if (src[q]) PBG_CUDA(cudaMemcpyAsync(&h[q * N], src[q], N * 8, cudaMemcpyDeviceToHost, s->stream));
    PBG_CUDA(cudaStreamSynchronize(s->stream));
    const int per = A.per;
    if (A.sym)
      for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
          for (int k = 0; k < nz; ++k) {
            long long p = ((long long)i * ny + j) * nz + k;
            h[2 * N + p] = i < nx - 1 ? h[1 * N + p + SI] : ((per & 1) ? h[1 * N + p - (nx - 1) * SI] : 0.0);
            h[4 * N + p] = j < ny - 1 ? h[3 * N + p + SJ] : ((per & 2) ? h[3 * N + p - (ny - 1) * SJ] : 0.0);
            h[6 * N + p] = k < nz - 1 ? h[5 * N + p + 1] : ((per & 4) ? h[5 * N + p - (nz - 1)] : 0.0);
          }
    double *dst[7] = {c, w, e, sv, n, b, t};
    for (int q = 0; q < 7; ++q) {
      if (!dst[q]) continue;
      if (where == PBG_HOST) std::memcpy(dst[q], &h[q * N], N * 8);
      else PBG_CUDA(cudaMemcpyAsync(dst[q], &h[q * N], N * 8, cudaMemcpyHostToDevice, s->stream));
    }
    PBG_CUDA(cudaStreamSynchronize(s->stream));
    return PBG_OK;
  });
}

int pbg_active_upload(pbg_session *s, const int *aflag, long long si, long long sj, long long sk,
                      long long offset, int where) {
  if (!s || !aflag) return fail(PBG_ERR_ARG, "NULL argument");
  if (where != PBG_HOST) return fail(PBG_ERR_UNSUPPORTED, "active flags are uploaded from host memory");
  return guard(s, [&]() -> int {
    std::vector<uint8_t> h(s->ncell());
    for (int i = 0; i < s->nx; ++i)
      for (int j = 0; j < s->ny; ++j)
        for (int k = 0; k < s->nz; ++k)
          h[((size_t)i * s->ny + j) * s->nz + k] = aflag[offset + i * si + j * sj + k * sk] ? 1 : 0;
    PBG_CUDA(cudaMemcpy(s->aflag.p, h.data(), h.size(), cudaMemcpyHostToDevice));
    invalidate(s);
    return PBG_OK;
  });
}

int pbg_ci_upload(pbg_session *s, const double *ci, long long si, long long sj, long long sk,
                  long long offset, int where) {
  if (!s || !ci) return fail(PBG_ERR_ARG, "NULL argument");
  if (!s->have_matrix) return fail(PBG_ERR_STATE, "no matrix uploaded or assembled");
  return guard(s, [&]() -> int {
    const long long N = s->ncell();
    if (s->ci.n != (size_t)N) s->ci.alloc(N);
    if (where == PBG_HOST) {
      std::vector<double> h(N);
      gather(ci, h.data(), s->nx, s->ny, s->nz, si, sj, sk, offset);
      PBG_CUDA(cudaMemcpyAsync(s->ci.p, h.data(), N * 8, cudaMemcpyHostToDevice, s->stream));
      PBG_CUDA(cudaStreamSynchronize(s->stream));
    } else {
      k_gather<<<grid_for(N), kThreads, 0, s->stream>>>(ci, s->ci.p, s->nx, s->ny, s->nz, si, sj, sk,
                                                         offset); note_launch();
      PBG_CUDA(cudaGetLastError());
    }
    s->ci_gen = s->mat_gen;
    return PBG_OK;
  });
}

int pbg_body_upload(pbg_session *s, const double *fV, const double *fS, int where) {
  if (!s) return fail(PBG_ERR_ARG, "session is NULL");
  if (!fV) {  // no body
    s->boff.release(); s->bidx.release(); s->bfs.release();
    s->ncut = 0;
    return PBG_OK;
  }
  if (!fS) return fail(PBG_ERR_ARG, "fS is NULL");
  return guard(s, [&]() -> int {
    const long long N = s->ncell();
    std::vector<double> v(N), f(6 * N);
    if (where == PBG_HOST) {
      std::memcpy(v.data(), fV, N * 8);
      std::memcpy(f.data(), fS, 6 * N * 8);
    } else {
      PBG_CUDA(cudaMemcpy(v.data(), fV, N * 8, cudaMemcpyDeviceToHost));
      PBG_CUDA(cudaMemcpy(f.data(), fS, 6 * N * 8, cudaMemcpyDeviceToHost));
    }
    std::vector<uint8_t> off(N);
    std::vector<int> idx(N, -1);
    std::vector<double> fs;
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    for (long long p = 0; p < N; ++p) {
      off[p] = v[p] == 0.0 ? 1 : 0;          // Body::off_p (body_interface.cpp:131-137)
      if (!(v[p] > 0.0 && v[p] < 1.0)) continue;  // Body::cut_p (:56-61)
      const int i = (int)(p / ((long long)ny * nz)), j = (int)(p / nz % ny), k = (int)(p % nz);
      if (i == 0 || i == nx - 1 || j == 0 || j == ny - 1 || (nz > 1 && (k == 0 || k == nz - 1)))
        return fail(PBG_ERR_UNSUPPORTED, "a cut cell on the domain boundary");
      idx[p] = (int)(fs.size() / 6);
      for (int d = 0; d < 6; ++d) fs.push_back(f[(size_t)d * N + p]);
    }
    s->ncut = (long long)(fs.size() / 6);
    s->boff.alloc(N);
    s->bidx.alloc(N);
    s->bfs.alloc(fs.empty() ? 6 : fs.size());
    PBG_CUDA(cudaMemcpy(s->boff.p, off.data(), N, cudaMemcpyHostToDevice));
    PBG_CUDA(cudaMemcpy(s->bidx.p, idx.data(), N * sizeof(int), cudaMemcpyHostToDevice));
    if (!fs.empty()) PBG_CUDA(cudaMemcpy(s->bfs.p, fs.data(), fs.size() * 8, cudaMemcpyHostToDevice));
    return PBG_OK;
  });
}

int pbg_assemble_pressure(pbg_session *s, const double *rho, const uint8_t *solid, int where) {
  if (!s || !rho || !solid) return fail(PBG_ERR_ARG, "NULL argument");
  if (s->per) return fail(PBG_ERR_UNSUPPORTED, "periodic boundaries: the on-device assembly and the flow functions take walls only (upload the matrix)");
  return guard(s, [&]() -> int {
    const long long N = s->ncell();
    DBuf<double> drho;
    DBuf<uint8_t> dsol;
    const double *r = rho;
    const uint8_t *so = solid;
    if (where == PBG_HOST) {
      drho.alloc(N); dsol.alloc(N);
      PBG_CUDA(cudaMemcpyAsync(drho.p, rho, N * 8, cudaMemcpyHostToDevice, s->stream));
      PBG_CUDA(cudaMemcpyAsync(dsol.p, solid, N, cudaMemcpyHostToDevice, s->stream));
      r = drho.p; so = dsol.p;
    }
    Mat64 &A = s->A;
    A.nx = s->nx; A.ny = s->ny; A.nz = s->nz; A.sym = true;
    if (A.c.n != (size_t)N) { A.c.alloc(N); A.w.alloc(N); A.s.alloc(N); A.b.alloc(N); }
    A.e.release(); A.n.release(); A.t.release();
    k_assemble<<<grid_for(N), kThreads, 0, s->stream>>>(
        s->nx, s->ny, s->nz, s->h, make_int4(s->bc[0], s->bc[1], s->bc[2], s->bc[3]),
        make_int2(s->bc[4], s->bc[5]), r, so, A.c.p, A.w.p, A.s.p, A.b.p, s->aflag.p); note_launch();
    PBG_CUDA(cudaGetLastError());
    PBG_CUDA(cudaStreamSynchronize(s->stream));
    s->have_matrix = true;
    ++s->mat_gen;
    invalidate(s);
    return PBG_OK;
  });
}

int pbg_assemble_mix(pbg_session *s, const double *col, double rho_a, double rho_b, const uint8_t *solid,
                     int where) {
  if (!s) return fail(PBG_ERR_ARG, "session is NULL");
  if (s->per) return fail(PBG_ERR_UNSUPPORTED, "periodic boundaries: the on-device assembly and the flow functions take walls only (upload the matrix)");
  if (!(rho_a > 0.0) || (col && !(rho_b > 0.0))) return fail(PBG_ERR_ARG, "densities must be positive");
  return guard(s, [&]() -> int {
    const long long N = s->ncell();
    DBuf<double> dcol;
    DBuf<uint8_t> dsol;
    const double *cp = col;
    const uint8_t *sp = solid;
    if (where == PBG_HOST) {
      if (col) {
        dcol.alloc(N);
        PBG_CUDA(cudaMemcpyAsync(dcol.p, col, N * 8, cudaMemcpyHostToDevice, s->stream));
        cp = dcol.p;
      }
      if (solid) {
        dsol.alloc(N);
        PBG_CUDA(cudaMemcpyAsync(dsol.p, solid, N, cudaMemcpyHostToDevice, s->stream));
        sp = dsol.p;
      }
    }
    BodyArgs bd;
    if (int rc = body_args(s, sp, bd)) return rc;
    Mat64 &A = s->A;
    // a cut body's face fractions differ between the two cells of a face:
    // the seven-array form
    const bool sym = bd.idx == nullptr;
    A.nx = s->nx; A.ny = s->ny; A.nz = s->nz; A.sym = sym;
    if (A.c.n != (size_t)N) { A.c.alloc(N); A.w.alloc(N); A.s.alloc(N); A.b.alloc(N); }
    if (sym) { A.e.release(); A.n.release(); A.t.release(); }
    else if (A.e.n != (size_t)N) { A.e.alloc(N); A.n.alloc(N); A.t.alloc(N); }
    if (flow_vec(s, bd.idx != nullptr)) {
      km_assemble_mix<kAsmV><<<march_grid(s->nx, s->ny, s->nz, kAsmV), kThreads, 0, s->stream>>>(
          s->nx, s->ny, s->nz, march_kq(s->nz, kAsmV), march_len(s->nx, s->ny, s->nz, kAsmV),
          asm_const(s->h, rho_a, rho_b), make_int4(s->bc[0], s->bc[1], s->bc[2], s->bc[3]),
          make_int2(s->bc[4], s->bc[5]), cp, rho_a, rho_b, bd.off, A.c.p, A.w.p, A.s.p, A.b.p, s->aflag.p);
    } else {
      k_assemble_mix<<<grid_for(N), kThreads, 0, s->stream>>>(
          flow_geo(s), s->nx, s->ny, s->nz, s->h, make_int4(s->bc[0], s->bc[1], s->bc[2], s->bc[3]),
          make_int2(s->bc[4], s->bc[5]), cp, rho_a, rho_b, bd.off, bd.idx, bd.fs, A.c.p, A.w.p, A.s.p, A.b.p,
          A.e.p, A.n.p, A.t.p, s->aflag.p);
    }
    note_launch();
    PBG_CUDA(cudaGetLastError());
    PBG_CUDA(cudaStreamSynchronize(s->stream));
    s->have_matrix = true;
    ++s->mat_gen;
    invalidate(s);
    return PBG_OK;
  });
}

}  // extern "C"

namespace {

// Face counts of the three velocity components.
long long nfaces(const pbg_session *s, int m) {
  return (long long)(s->nx + (m == 0)) * (s->ny + (m == 1)) * (s->nz + (m == 2));
}

// Device copies of host face arrays (where == PBG_HOST) or the caller's
// device pointers. w may be NULL in 2-D.
struct FaceArgs {
  DBuf<double> buf[3];
  double *d[3] = {nullptr, nullptr, nullptr};
  void in(pbg_session *s, double *const f[3], int where, bool copy) {
    for (int m = 0; m < 3; ++m) {
      if (!f[m]) continue;
      if (where == PBG_HOST) {
        buf[m].alloc(nfaces(s, m));
        if (copy)
          PBG_CUDA(cudaMemcpyAsync(buf[m].p, f[m], nfaces(s, m) * 8, cudaMemcpyHostToDevice, s->stream));
        d[m] = buf[m].p;
      } else {
        d[m] = f[m];
      }
    }
  }
  void out(pbg_session *s, double *const f[3], int where) {
    if (where != PBG_HOST) return;
    for (int m = 0; m < 3; ++m)
      if (f[m]) PBG_CUDA(cudaMemcpyAsync(f[m], d[m], nfaces(s, m) * 8, cudaMemcpyDeviceToHost, s->stream));
  }
};

int check_faces(const pbg_session *s, const double *u, const double *v, const double *w) {
  if (!u || !v) return fail(PBG_ERR_ARG, "u and v are required");
  if (!w && s->nz > 1) return fail(PBG_ERR_ARG, "w is required in 3-D");
  return PBG_OK;
}

}  // namespace

extern "C" {

int pbg_divergence(pbg_session *s, const double *u, const double *v, const double *w, const uint8_t *solid,
                   double dt, double *rhs, int where) {
  if (!s || !rhs) return fail(PBG_ERR_ARG, "NULL argument");
  if (s->per) return fail(PBG_ERR_UNSUPPORTED, "periodic boundaries: the on-device assembly and the flow functions take walls only (upload the matrix)");
  if (int rc = check_faces(s, u, v, w)) return rc;
  if (!(dt > 0.0)) return fail(PBG_ERR_ARG, "dt must be positive");
  return guard(s, [&]() -> int {
    const long long N = s->ncell();
    FaceArgs fa;
    double *f[3] = {const_cast<double *>(u), const_cast<double *>(v), const_cast<double *>(w)};
    fa.in(s, f, where, true);
    DBuf<double> drhs;
    DBuf<uint8_t> dsol;
    double *r = rhs;
    const uint8_t *sp = solid;
    if (where == PBG_HOST) {
      drhs.alloc(N);
      r = drhs.p;
      if (solid) {
        dsol.alloc(N);
        PBG_CUDA(cudaMemcpyAsync(dsol.p, solid, N, cudaMemcpyHostToDevice, s->stream));
        sp = dsol.p;
      }
    }
    BodyArgs bd;
    if (int rc = body_args(s, sp, bd)) return rc;
    const double dti = 1.0 / dt;
    const double a = (s->h * s->h) * dti;
    if (flow_vec(s, bd.idx != nullptr))
      kv_divergence<kFlowV><<<grid_for(N / kFlowV), kThreads, 0, s->stream>>>(
          flow_geo(s), s->nx, s->ny, s->nz, a, fa.d[0], fa.d[1], fa.d[2], bd.off, r);
    else
      k_divergence<<<grid_for(N), kThreads, 0, s->stream>>>(flow_geo(s), s->nx, s->ny, s->nz, a, fa.d[0], fa.d[1],
                                                            fa.d[2], bd.off, bd.idx, bd.fs, r);
    note_launch();
    PBG_CUDA(cudaGetLastError());
    if (where == PBG_HOST) PBG_CUDA(cudaMemcpyAsync(rhs, r, N * 8, cudaMemcpyDeviceToHost, s->stream));
    PBG_CUDA(cudaStreamSynchronize(s->stream));
    return PBG_OK;
  });
}

int pbg_project(pbg_session *s, const double *p, const double *col, double rho_a, double rho_b,
                const uint8_t *solid, double dt, double *u, double *v, double *w, int where) {
  if (!s || !p) return fail(PBG_ERR_ARG, "NULL argument");
  if (s->per) return fail(PBG_ERR_UNSUPPORTED, "periodic boundaries: the on-device assembly and the flow functions take walls only (upload the matrix)");
  if (int rc = check_faces(s, u, v, w)) return rc;
  if (!(dt > 0.0)) return fail(PBG_ERR_ARG, "dt must be positive");
  if (!(rho_a > 0.0) || (col && !(rho_b > 0.0))) return fail(PBG_ERR_ARG, "densities must be positive");
  return guard(s, [&]() -> int {
    const long long N = s->ncell();
    FaceArgs fa;
    double *f[3] = {u, v, w};
    fa.in(s, f, where, true);
    DBuf<double> dp, dcol;
    DBuf<uint8_t> dsol;
    const double *pp = p, *cp = col;
    const uint8_t *sp = solid;
    if (where == PBG_HOST) {
      dp.alloc(N);
      PBG_CUDA(cudaMemcpyAsync(dp.p, p, N * 8, cudaMemcpyHostToDevice, s->stream));
      pp = dp.p;
      if (col) {
        dcol.alloc(N);
        PBG_CUDA(cudaMemcpyAsync(dcol.p, col, N * 8, cudaMemcpyHostToDevice, s->stream));
        cp = dcol.p;
      }
      if (solid) {
        dsol.alloc(N);
        PBG_CUDA(cudaMemcpyAsync(dsol.p, solid, N, cudaMemcpyHostToDevice, s->stream));
        sp = dsol.p;
      }
    }
    BodyArgs bd;
    if (int rc = body_args(s, sp, bd)) return rc;
    if (flow_vec(s, false))
      km_project<kProjV><<<march_grid(s->nx, s->ny, s->nz, kProjV), kThreads, 0, s->stream>>>(
          s->nx, s->ny, s->nz, march_kq(s->nz, kProjV), march_len(s->nx, s->ny, s->nz, kProjV),
          proj_const(rho_a, rho_b, s->h), dt, pp, cp, rho_a, rho_b, bd.off, fa.d[0], fa.d[1], fa.d[2]);
    else
      k_project<<<grid_for(N), kThreads, 0, s->stream>>>(flow_geo(s), s->nx, s->ny, s->nz, s->h, dt, pp, cp, rho_a,
                                                         rho_b, bd.off, fa.d[0], fa.d[1], fa.d[2]);
    note_launch();
    PBG_CUDA(cudaGetLastError());
    fa.out(s, f, where);
    PBG_CUDA(cudaStreamSynchronize(s->stream));
    return PBG_OK;
  });
}

int pbg_pressure_step(pbg_session *s, const double *col, double rho_a, double rho_b, const uint8_t *solid,
                      double dt, double *u, double *v, double *w, double *p, int where, const pbg_params *prm,
                      pbg_result *res) {
  if (!s || !p || !prm) return fail(PBG_ERR_ARG, "NULL argument");
  if (s->per) return fail(PBG_ERR_UNSUPPORTED, "periodic boundaries: the on-device assembly and the flow functions take walls only (upload the matrix)");
  if (int rc = check_faces(s, u, v, w)) return rc;
  if (!(dt > 0.0)) return fail(PBG_ERR_ARG, "dt must be positive");
  return guard(s, [&]() -> int {
    const long long N = s->ncell();
    // inputs on the device once; every stage then runs on device pointers
    FaceArgs fa;
    double *f[3] = {u, v, w};
    fa.in(s, f, where, true);
    DBuf<double> dcol, dp;
    DBuf<uint8_t> dsol;
    const double *cp = col;
    const uint8_t *sp = solid;
    double *pp = p;
    if (s->frhs.n != (size_t)N) s->frhs.alloc(N);
    if (where == PBG_HOST) {
      if (col) {
        dcol.alloc(N);
        PBG_CUDA(cudaMemcpyAsync(dcol.p, col, N * 8, cudaMemcpyHostToDevice, s->stream));
        cp = dcol.p;
      }
      if (solid) {
        dsol.alloc(N);
        PBG_CUDA(cudaMemcpyAsync(dsol.p, solid, N, cudaMemcpyHostToDevice, s->stream));
        sp = dsol.p;
      }
      dp.alloc(N);
      PBG_CUDA(cudaMemcpyAsync(dp.p, p, N * 8, cudaMemcpyHostToDevice, s->stream));
      pp = dp.p;
    }
    int rc = pbg_assemble_mix(s, cp, rho_a, rho_b, sp, PBG_DEVICE);
    if (rc != PBG_OK) return rc;
    rc = pbg_divergence(s, fa.d[0], fa.d[1], fa.d[2], sp, dt, s->frhs.p, PBG_DEVICE);
    if (rc != PBG_OK) return rc;
    // Centered::solve hands the solver scale * dti (centered_solve.cpp:31)
    pbg_params q = *prm;
    q.scale = prm->scale * (1.0 / dt);
    pbg_result local;
    rc = pbg_solve(s, pp, s->frhs.p, PBG_DEVICE, &q, res ? res : &local);
    if (rc != PBG_OK) return rc;
    rc = pbg_project(s, pp, cp, rho_a, rho_b, sp, dt, fa.d[0], fa.d[1], fa.d[2], PBG_DEVICE);
    if (rc != PBG_OK) return rc;
    fa.out(s, f, where);
    if (where == PBG_HOST) PBG_CUDA(cudaMemcpyAsync(p, pp, N * 8, cudaMemcpyDeviceToHost, s->stream));
    PBG_CUDA(cudaStreamSynchronize(s->stream));
    return PBG_OK;
  });
}

}  // extern "C"

namespace {

void ensure_refac(pbg_session *s) {
  if (!s->refac) s->refac = std::make_unique<RefAC>();
  if (s->refac_dirty) {
    s->refac->build(s->A.view(), s->aflag.p, s->h, s->stream);
    PBG_CUDA(cudaStreamSynchronize(s->stream));
    s->refac_dirty = false;
  }
}

void ensure_engine(pbg_session *s, bool mixed, int coarse_max) {
  if (!s->eng) s->eng = std::make_unique<Engine>();
  if (coarse_max > 0 && coarse_max != s->eng->opt.coarse_max) {
    s->eng->opt.coarse_max = coarse_max;  // a different hierarchy: build anew
    s->eng->L.clear();
    s->eng_dirty = true;
  }
  if (s->eng_dirty || (mixed && !s->eng->have32)) {
    const Mat64 &A = s->A;
    EMat<double> m = make_emat<double>(A.nx, A.ny, A.nz, A.c.p, A.w.p, A.s.p, A.b.p, nullptr);
    s->eng->nonsym = !A.sym;
    if (!A.sym) {
      // a cut body's matrix: the hierarchy from its symmetric part, the
      // refinement against the matrix itself
      const long long N = s->ncell();
      if (s->symc.n != (size_t)N) { s->symc.alloc(N); s->symw.alloc(N); s->syms.alloc(N); s->symb.alloc(N); }
      symmetrize(A.view(), s->symc.p, s->symw.p, s->syms.p, s->symb.p, s->stream);
      m = make_emat<double>(A.nx, A.ny, A.nz, s->symc.p, s->symw.p, s->syms.p, s->symb.p, nullptr);
      s->eng->top = A.view();
    }
    // same shape and buffers (a re-assembled matrix): numeric refresh only
    if (s->eng->refresh(m, mixed, s->stream)) {
      s->eng_dirty = false;
      return;
    }
    s->eng->build(m, s->stream, mixed || s->eng_mixed);
    s->eng_mixed = s->eng_mixed || mixed;
    s->eng_dirty = false;
  }
}

// Scratch of the exact-order reductions (2 terms per cell, the chunk and
// group records and the look-back flags), when requested.
double *exact_terms(pbg_session *s, const pbg_params *p) {
  if (!p->exact_sums) return nullptr;
  const size_t need = exact_scratch_doubles(s->ncell());
  if (s->seq.n < need) {
    s->seq.alloc(need);
    exact_scratch_init(s->seq.p, s->ncell(), s->stream);
  }
  return exact_seq(s->seq.p);
}

int solve_device(pbg_session *s, double *xd, const double *bd, const pbg_params *p, pbg_result *r) {
  pbg_result out;
  std::memset(&out, 0, sizeof(out));
  const double dV = s->dV;
  s->nhist = 0;
  if (p->solver == PBG_SOLVER_CG || p->solver == PBG_SOLVER_BICGS || p->solver == PBG_SOLVER_CGS ||
      p->solver == PBG_SOLVER_JACOBI || p->solver == PBG_SOLVER_GAUSS_SEIDEL) {
    KrylovParams pr;
    pr.mini = p->min_iter; pr.maxit = p->max_iter;
    pr.stalecount = p->stalecount > kStaleMax ? kStaleMax : p->stalecount;
    pr.hist_cap = kHistMax;
    pr.res_rat = p->res_rat; pr.res_tol = p->res_tol; pr.scale = p->scale; pr.dV = dV;
    pr.seq = exact_terms(s, p);
    if (p->prec < 0 || p->prec > 3) return fail(PBG_ERR_ARG, "prec must be 0 (diagonal), 1 (IC0), 2 (IC2) or 3 (IC3)");
    pr.prec = p->prec;
    const int kind = p->solver == PBG_SOLVER_CG ? 0 : p->solver == PBG_SOLVER_BICGS ? 1
                     : p->solver == PBG_SOLVER_CGS ? 2 : p->solver == PBG_SOLVER_JACOBI ? 3 : 4;
    if (kind >= 3) {  // no preconditioner (iterative.h:15-31); A.ci if uploaded
      pr.prec = 0;
      pr.ci = s->ci_gen == s->mat_gen ? s->ci.p : nullptr;
    }
    RefKrylovResult rr = ref_krylov_solve(s->A.view(), xd, bd, pr, kind,
                                          s->rkw, s->red, s->kst.p, s->hkst, s->hist.p, s->stream);
    out.status = rr.status;
    out.converged = rr.converged;
    out.iterations = rr.iterations;
    out.res0 = rr.res0;
    out.res = rr.res;
    out.levels = 1;
    int nh = rr.iterations < kHistMax ? rr.iterations : kHistMax;
    s->hhist.resize(nh);
    if (nh) PBG_CUDA(cudaMemcpy(s->hhist.data(), s->hist.p, nh * 8, cudaMemcpyDeviceToHost));
    s->nhist = nh;
  } else if (p->solver == PBG_SOLVER_AC) {
    ensure_refac(s);
    RefACParams pa;
    pa.init = p->init_cycle; pa.loop = p->loop_cycle;
    pa.toler = p->toler; pa.factor = p->factor;
    pa.max_cyc = p->max_cycles; pa.min_cyc = p->min_cycles;
    pa.stop_if_div = p->stop_if_div; pa.priority_min_cyc = p->priority_min_cyc;
    for (int q = 0; q < 3; ++q) { pa.mv[q] = p->mv[q]; pa.ms[q] = p->ms[q] > kStaleMax ? kStaleMax : p->ms[q]; }
    pa.resrat_val = p->ac_resrat;  // AC::resrat / restol (additive.cpp:17-18 default atto)
    pa.restol_val = p->ac_restol;
    pa.use_linf = p->use_linf != 0;
    s->refac->sm_scale = p->scale;
    s->refac->res_dt = p->ac_dt;
    pa.flex_visits = p->flex_visits > 0 ? p->flex_visits : 1000000;
    auto cyc_ok = [](int c, bool none_ok) {
      return c == PBG_CYCLE_V || c == PBG_CYCLE_F || c == PBG_CYCLE_W || c == PBG_CYCLE_FLEX ||
             (none_ok && c == PBG_CYCLE_NONE);
    };
    if (!cyc_ok(p->loop_cycle, true) || !cyc_ok(p->init_cycle, true))
      return fail(PBG_ERR_ARG, "cycles are PBG_CYCLE_NONE, V, F, W or FLEX");
    RefACCtx cx;
    cx.s = s->stream; cx.w = &s->rkw; cx.red = &s->red; cx.st = s->kst.p;
    cx.dscal = s->dscal.p; cx.dmean = s->dscal.p + 4; cx.hbuf = s->hbuf; cx.dlinf = s->dlinf.p;
    for (int q = 0; q < 3; ++q) { cx.mv[q] = pa.mv[q]; cx.ms[q] = pa.ms[q]; }
    cx.resrat_val = pa.resrat_val; cx.restol_val = pa.restol_val;
    cx.hst = s->hkst;
    s->refac->seq = exact_terms(s, p);
    auto kind_of = [](int sv) {
      return sv == PBG_SOLVER_CG ? 0 : sv == PBG_SOLVER_BICGS ? 1 : sv == PBG_SOLVER_CGS ? 2
             : sv == PBG_SOLVER_JACOBI ? 3 : sv == PBG_SOLVER_GAUSS_SEIDEL ? 4 : -1;
    };
    const int sm = p->ac_smoother;
    if (kind_of(sm) < 0)
      return fail(PBG_ERR_ARG, "ac_smoother must be CG, BiCGS, CGS, Jacobi or Gauss-Seidel");
    if (p->ac_solver != -1 && kind_of(p->ac_solver) < 0)
      return fail(PBG_ERR_ARG, "ac_solver must be -1 (the smoother), CG, BiCGS, CGS, Jacobi or Gauss-Seidel");
    if (p->prec < 0 || p->prec > 3 || p->ac_solver_prec < 0 || p->ac_solver_prec > 3)
      return fail(PBG_ERR_ARG, "prec must be 0 (diagonal), 1 (IC0), 2 (IC2) or 3 (IC3)");
    s->refac->sm_kind = kind_of(sm);
    s->refac->sm_prec = s->refac->sm_kind <= 2 ? p->prec : 0;
    s->refac->sol_kind = p->ac_solver == -1 ? -1 : kind_of(p->ac_solver);
    s->refac->sol_prec = s->refac->sol_kind >= 0 && s->refac->sol_kind <= 2 ? p->ac_solver_prec : 0;
    s->refac->sm_ci0 = s->ci_gen == s->mat_gen ? s->ci.p : nullptr;
    s->hhist.assign(p->max_cycles + 3, 0.0);  // initial, cycle 0 (a full-cycle start), cycles
    RefACResult ar = s->refac->cycle(xd, bd, pa, cx, s->hhist.data(), (int)s->hhist.size());
    s->nhist = ar.nhist < (int)s->hhist.size() ? ar.nhist : (int)s->hhist.size();
    out.converged = ar.converged;
    out.cycles = ar.cycles;
    out.status = ar.converged ? PBG_CONVERGED : (ar.diverged ? PBG_DIVERGED : PBG_MAXITER);
    out.iterations = ar.visits;  // flex cycles: smoother calls of the last one
    out.res0 = ar.res0;
    out.res = ar.res;
    out.levels = s->refac->nlevels();
  } else if (p->solver == PBG_SOLVER_ENGINE) {
    if (s->A.per)
      return fail(PBG_ERR_UNSUPPORTED, "periodic boundaries: the engine solver takes walls only "
                                       "(use CG, BiCGS, CGS or AC)");
    const bool mixed = p->precision == PBG_MIXED;
    if (p->coarse_max < 0) return fail(PBG_ERR_ARG, "coarse_max must be >= 0");
    ensure_engine(s, mixed, p->coarse_max);
    EngineResult er = mixed ? s->eng->solve_mixed(xd, bd, p->tol, p->inner_tol, p->max_sweeps,
                                                  p->max_iter, s->red, s->stream, s->hist.p)
                            : s->eng->solve_fp64(xd, bd, p->tol, p->max_iter, s->red, s->stream,
                                                 s->hist.p);
    out.status = er.status;
    out.converged = er.converged;
    out.iterations = er.iterations;
    out.sweeps = er.sweeps;
    out.relres = er.relres;
    out.res = er.relres;
    out.levels = s->eng->nlevels();
    int nh = er.iterations < kHistMax ? er.iterations : kHistMax;
    s->hhist.resize(nh);
    if (nh) PBG_CUDA(cudaMemcpy(s->hhist.data(), s->hist.p, nh * 8, cudaMemcpyDeviceToHost));
    s->nhist = nh;
  } else {
    return fail(PBG_ERR_ARG, "unknown solver");
  }
  if (r) *r = out;
  return PBG_OK;
}

}  // namespace

extern "C" {

int pbg_solve_strided(pbg_session *s, double *x, const double *b, long long si, long long sj,
                      long long sk, long long offset, int where, const pbg_params *p,
                      pbg_result *r) {
  if (!s || !x || !b || !p) return fail(PBG_ERR_ARG, "NULL argument");
  if (!s->have_matrix) return fail(PBG_ERR_STATE, "no matrix uploaded or assembled");
  if (p->solver == PBG_SOLVER_ENGINE && !(p->tol > 0.0))
    return fail(PBG_ERR_ARG, "engine tolerance must be > 0");
  return guard(s, [&]() -> int {
    auto t0 = std::chrono::steady_clock::now();
    const long long N = s->ncell();
    const bool compact = (si == (long long)s->ny * s->nz && sj == s->nz && sk == 1 && offset == 0);
    int rc;
    const bool zero = p->x0_zero != 0;
    if (where == PBG_DEVICE && compact) {
      if (zero) PBG_CUDA(cudaMemsetAsync(x, 0, N * 8, s->stream));
      rc = solve_device(s, x, b, p, r);
    } else {
      ensure_staging(s);
      if (zero) PBG_CUDA(cudaMemsetAsync(s->dx.p, 0, N * 8, s->stream));
      if (where == PBG_HOST) {
        if (compact) {
          if (!zero) h2d(s, s->dx.p, x, N * 8, s->px);
          h2d(s, s->db.p, b, N * 8, s->pb);
        } else {
          if (!zero) gather(x, s->px, s->nx, s->ny, s->nz, si, sj, sk, offset);
          gather(b, s->pb, s->nx, s->ny, s->nz, si, sj, sk, offset);
          if (!zero) PBG_CUDA(cudaMemcpyAsync(s->dx.p, s->px, N * 8, cudaMemcpyHostToDevice, s->stream));
          PBG_CUDA(cudaMemcpyAsync(s->db.p, s->pb, N * 8, cudaMemcpyHostToDevice, s->stream));
        }
      } else {
        if (!zero) {
          k_gather<<<grid_for(N), kThreads, 0, s->stream>>>(x, s->dx.p, s->nx, s->ny, s->nz, si, sj, sk, offset);
          note_launch();
        }
        k_gather<<<grid_for(N), kThreads, 0, s->stream>>>(b, s->db.p, s->nx, s->ny, s->nz, si, sj, sk, offset); note_launch();
      }
      rc = solve_device(s, s->dx.p, s->db.p, p, r);
      if (rc == PBG_OK) {
        if (where == PBG_HOST && compact) {
          d2h(s, x, s->dx.p, N * 8, s->px);
        } else if (where == PBG_HOST) {
          PBG_CUDA(cudaMemcpyAsync(s->px, s->dx.p, N * 8, cudaMemcpyDeviceToHost, s->stream));
          PBG_CUDA(cudaStreamSynchronize(s->stream));
          for (int i = 0; i < s->nx; ++i)
            for (int j = 0; j < s->ny; ++j)
              for (int k = 0; k < s->nz; ++k)
                x[offset + i * si + j * sj + k * sk] = s->px[((size_t)i * s->ny + j) * s->nz + k];
        } else {
          k_scatter<<<grid_for(N), kThreads, 0, s->stream>>>(s->dx.p, x, s->nx, s->ny, s->nz, si, sj, sk, offset); note_launch();
        }
      }
    }
    PBG_CUDA(cudaStreamSynchronize(s->stream));
    if (r) r->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return rc;
  });
}

int pbg_solve(pbg_session *s, double *x, const double *b, int where, const pbg_params *p,
              pbg_result *r) {
  if (!s) return fail(PBG_ERR_ARG, "session is NULL");
  return pbg_solve_strided(s, x, b, (long long)s->ny * s->nz, s->nz, 1, 0, where, p, r);
}

int pbg_history(const pbg_session *s, double *out, int cap, int *count) {
  if (!s) return fail(PBG_ERR_ARG, "session is NULL");
  int n = s->nhist < cap ? s->nhist : cap;
  if (out && n > 0) std::memcpy(out, s->hhist.data(), n * 8);
  if (count) *count = s->nhist;
  return PBG_OK;
}

static int op_run(pbg_session *s, int op, const double *x, const double *b, double *y, int where,
                  double *out2) {
  if (!s) return fail(PBG_ERR_ARG, "session is NULL");
  if (op != 2 && !s->have_matrix) return fail(PBG_ERR_STATE, "no matrix");
  return guard(s, [&]() -> int {
    const long long N = s->ncell();
    const double *dxp = x, *dbp = b;
    double *dyp = y;
    DBuf<double> t1, t2, t3;
    if (where == PBG_HOST) {
      t1.alloc(N);
      PBG_CUDA(cudaMemcpyAsync(t1.p, x, N * 8, cudaMemcpyHostToDevice, s->stream));
      dxp = t1.p;
      if (b) { t2.alloc(N); PBG_CUDA(cudaMemcpyAsync(t2.p, b, N * 8, cudaMemcpyHostToDevice, s->stream)); dbp = t2.p; }
      if (y) { t3.alloc(N); dyp = t3.p; }
    }
    const int g = grid_for(N);
    if (op == 0) { k_spmv_ref<<<g, kThreads, 0, s->stream>>>(s->A.view(), dxp, dyp); note_launch(); }
    else if (op == 1) { k_resid_ref<<<g, kThreads, 0, s->stream>>>(s->A.view(), dxp, dbp, dyp); note_launch(); }
    else {
      k_dot2<<<g, kThreads, 0, s->stream>>>(N, dxp, dbp, (s->h * s->h) * s->h, s->red.slot_part(0),
                                           s->red.slot_count(0), s->dscal.p); note_launch();
      PBG_CUDA(cudaMemcpyAsync(s->hbuf, s->dscal.p, 16, cudaMemcpyDeviceToHost, s->stream));
    }
    PBG_CUDA(cudaGetLastError());
    if (where == PBG_HOST && y) PBG_CUDA(cudaMemcpyAsync(y, dyp, N * 8, cudaMemcpyDeviceToHost, s->stream));
    PBG_CUDA(cudaStreamSynchronize(s->stream));
    if (op == 2) {
      double n = (double)N;
      out2[0] = s->hbuf[0];
      out2[1] = s->hbuf[1] / n / n;
    }
    return PBG_OK;
  });
}

int pbg_seq_sum(pbg_session *s, const double *a, const double *b, long long n, int where, double out[2]) {
  if (!s || !a || !out) return fail(PBG_ERR_ARG, "NULL argument");
  if (n < 1 || n > (1LL << 31) - 1) return fail(PBG_ERR_ARG, "n must be in 1 .. 2^31-1");
  return guard(s, [&]() -> int {
    const double *da = a, *db = b;
    DBuf<double> t1, t2, scratch(exact_scratch_doubles(n)), res(2);
    if (where == PBG_HOST) {
      t1.alloc(n);
      PBG_CUDA(cudaMemcpyAsync(t1.p, a, n * 8, cudaMemcpyHostToDevice, s->stream));
      da = t1.p;
      if (b) {
        t2.alloc(n);
        PBG_CUDA(cudaMemcpyAsync(t2.p, b, n * 8, cudaMemcpyHostToDevice, s->stream));
        db = t2.p;
      }
    }
    exact_scratch_init(scratch.p, n, s->stream);
    k_seq_sum<<<grid_exact(n), kThreads, 0, s->stream>>>(n, da, db, exact_seq(scratch.p),
                                                          s->red.slot_count(0), res.p); note_launch();
    PBG_CUDA(cudaGetLastError());
    PBG_CUDA(cudaMemcpyAsync(s->hbuf, res.p, 16, cudaMemcpyDeviceToHost, s->stream));
    PBG_CUDA(cudaStreamSynchronize(s->stream));
    out[0] = s->hbuf[0];
    out[1] = s->hbuf[1];
    return PBG_OK;
  });
}

int pbg_spmv(pbg_session *s, const double *x, double *y, int where) {
  if (!x || !y) return fail(PBG_ERR_ARG, "NULL argument");
  return op_run(s, 0, x, nullptr, y, where, nullptr);
}
int pbg_residual(pbg_session *s, const double *x, const double *b, double *r, int where) {
  if (!x || !b || !r) return fail(PBG_ERR_ARG, "NULL argument");
  return op_run(s, 1, x, b, r, where, nullptr);
}
int pbg_dot(pbg_session *s, const double *x, const double *y, int where, double out[2]) {
  if (!x || !y || !out) return fail(PBG_ERR_ARG, "NULL argument");
  return op_run(s, 2, x, y, nullptr, where, out);
}

int pbg_levels(pbg_session *s, int kind, int *count, int *dims, int cap) {
  if (!s || !count) return fail(PBG_ERR_ARG, "NULL argument");
  if (!s->have_matrix) return fail(PBG_ERR_STATE, "no matrix");
  return guard(s, [&]() -> int {
    std::vector<int> d;
    if (kind == 0) {
      ensure_refac(s);
      for (auto &l : s->refac->L) { d.push_back(l.nx); d.push_back(l.ny); d.push_back(l.nz); }
    } else {
      ensure_engine(s, false, 0);
      for (auto &l : s->eng->L) { d.push_back(l.nx); d.push_back(l.ny); d.push_back(l.nz); }
    }
    *count = (int)d.size() / 3;
    if (dims) for (int q = 0; q < (int)d.size() && q < 3 * cap; ++q) dims[q] = d[q];
    return PBG_OK;
  });
}

int pbg_ac_level_matrix(pbg_session *s, int level, double *out7, int where) {
  if (!s || !out7) return fail(PBG_ERR_ARG, "NULL argument");
  if (!s->have_matrix) return fail(PBG_ERR_STATE, "no matrix");
  return guard(s, [&]() -> int {
    ensure_refac(s);
    if (level < 1 || level >= s->refac->nlevels()) return fail(PBG_ERR_ARG, "level out of range");
    s->refac->coarsen_all(s->stream);
    const RefACLevel &L = s->refac->L[level];
    const long long n = (long long)L.nx * L.ny * L.nz;
    const double *src[7] = {L.A.c.p, L.A.w.p, L.A.e.p, L.A.s.p, L.A.n.p, L.A.b.p, L.A.t.p};
    for (int q = 0; q < 7; ++q)
      PBG_CUDA(cudaMemcpyAsync(out7 + q * n, src[q], n * 8,
                               where == PBG_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                               s->stream));
    PBG_CUDA(cudaStreamSynchronize(s->stream));
    return PBG_OK;
  });
}

int pbg_generate(int kind, const double *params, uint64_t seed, int dims[3], double *h,
                 double *rho, uint8_t *solid, double *b) {
  if (!params || !dims || !h) return fail(PBG_ERR_ARG, "NULL argument");
  pbg_problem_desc d;
  int n = (int)params[0];
  if (kind == 0) pbg_desc_single_bubble(&d, n, seed);
  else if (kind == 1)
    pbg_desc_bubbles_cylinder(&d, n, (int)params[1], params[2], params[3], params[4], params[5], seed);
  else if (kind == 2)
    pbg_desc_batch_member(&d, seed, (int)params[6], (int)params[7], (int)params[8], (int)params[9],
                          (int)params[10], (int)params[11]);
  else return fail(PBG_ERR_ARG, "unknown kind");
  dims[0] = d.nx; dims[1] = d.ny; dims[2] = d.nz;
  *h = d.h;
  if (!rho) return PBG_OK;
  if (!solid || !b) return fail(PBG_ERR_ARG, "rho, solid and b go together");
  pbg_gen_fields(&d, rho, solid);
  pbg_gen_rhs(&d, (uint64_t)params[12], solid, b);
  return PBG_OK;
}

int pbg_generate_flow(int kind, const double *params, uint64_t seed, double *col, double *u, double *v,
                      double *w, double rho[2]) {
  if (!params || !col || !u || !v || !w || !rho) return fail(PBG_ERR_ARG, "NULL argument");
  pbg_problem_desc d;
  int n = (int)params[0];
  if (kind == 0) pbg_desc_single_bubble(&d, n, seed);
  else if (kind == 1)
    pbg_desc_bubbles_cylinder(&d, n, (int)params[1], params[2], params[3], params[4], params[5], seed);
  else if (kind == 2)
    pbg_desc_batch_member(&d, seed, (int)params[6], (int)params[7], (int)params[8], (int)params[9],
                          (int)params[10], (int)params[11]);
  else return fail(PBG_ERR_ARG, "unknown kind");
  rho[0] = d.rho_liquid;
  rho[1] = d.rho_vapour;
  pbg_gen_flow(&d, (uint64_t)params[12], col, u, v, w);
  return PBG_OK;
}

}  // extern "C"

extern "C" {

unsigned long long pbg_launch_count(void) { return __atomic_load_n(&pbg::g_launch_count, __ATOMIC_RELAXED); }

int pbg_session_stream(pbg_session *s, void **stream) {
  if (!s || !stream) return fail(PBG_ERR_ARG, "NULL argument");
  *stream = (void *)s->stream;
  return PBG_OK;
}

int pbg_bench_kernel(pbg_session *s, int which, int precision, int reps, double *ms,
                     double *bytes_per_launch) {
  if (!s || !ms || reps < 1) return fail(PBG_ERR_ARG, "bad argument");
  if (!s->have_matrix) return fail(PBG_ERR_STATE, "no matrix");
  return guard(s, [&]() -> int {
    const long long N = s->ncell();
    if (which == 0) {
      if (!s->A.sym) return fail(PBG_ERR_UNSUPPORTED, "engine needs a symmetric matrix");
      ensure_engine(s, precision == 1, 0);
      *ms = s->eng->bench_sweep(precision, reps, s->stream);
      if (bytes_per_launch) *bytes_per_launch = (double)N * (precision == 1 ? 28.0 : 56.0);
      return PBG_OK;
    }
    if (which == 1) {
      ensure_staging(s);
      PBG_CUDA(cudaMemsetAsync(s->dx.p, 0, N * 8, s->stream));
      cudaEvent_t e0, e1;
      PBG_CUDA(cudaEventCreate(&e0));
      PBG_CUDA(cudaEventCreate(&e1));
      const int g = grid_for(N);
      k_spmv_ref<<<g, kThreads, 0, s->stream>>>(s->A.view(), s->dx.p, s->db.p); note_launch();
      PBG_CUDA(cudaEventRecord(e0, s->stream));
      for (int q = 0; q < reps; ++q) {
        k_spmv_ref<<<g, kThreads, 0, s->stream>>>(s->A.view(), (q & 1) ? s->db.p : s->dx.p,
                                                  (q & 1) ? s->dx.p : s->db.p); note_launch();
      }
      PBG_CUDA(cudaEventRecord(e1, s->stream));
      PBG_CUDA(cudaEventSynchronize(e1));
      float t = 0.f;
      PBG_CUDA(cudaEventElapsedTime(&t, e0, e1));
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      *ms = (double)t / reps;
      if (bytes_per_launch) *bytes_per_launch = (double)N * (s->A.sym ? 48.0 : 72.0);
      return PBG_OK;
    }
    return fail(PBG_ERR_ARG, "unknown kernel id");
  });
}

}  // extern "C"
