// Serving loop (pbg_server_*): sessions resident on the device, a request
// queue fed from any thread, and one worker thread that runs the batched
// engine continuously — admitting queued requests into free slots at every
// outer iteration, stepping the batch, and retiring finished requests.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/psiboil_b200.h"
#include "pbg_batch_engine.h"
#include "pbg_common.cuh"
#include "pbg_session.h"

namespace pbg {
void set_last_error(const char *msg);  // pbg_capi.cu

namespace {

using Clock = std::chrono::steady_clock;

// ---------------------------------------------------------------- request inputs made on the device
// One bubble: density 1 inside the sphere (cell centres, cell units), ratio
// outside; no solid cells.
__global__ void k_bubble_fields(int nx, int ny, int nz, double cx, double cy, double cz, double r,
                                double ratio, double *__restrict__ rho, uint8_t *__restrict__ solid) {
  const long long N = (long long)nx * ny * nz;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    const Pos q = pos_of(p, ny, nz);
    const double dx = q.i + 0.5 - cx, dy = q.j + 0.5 - cy, dz = nz > 1 ? q.k + 0.5 - cz : 0.0;
    rho[p] = (dx * dx + dy * dy + dz * dz <= r * r) ? 1.0 : ratio;
    solid[p] = 0;
  }
}

// A counter-based uniform in [-1, 1) per cell (splitmix64 of seed and index).
__device__ __forceinline__ double cell_uniform(unsigned long long seed, long long p) {
  unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(p + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

constexpr int kRhsBlocks = 296;

// b = uniform draws; per-block sums (fixed grid, so the sum order is fixed)
__global__ void k_rhs_draw(long long N, unsigned long long seed, double *__restrict__ b,
                           double *__restrict__ part) {
  __shared__ double sm[kThreads / 32];
  double v = 0.0;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    const double u = cell_uniform(seed, p);
    b[p] = u;
    v += u;
  }
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sm[w];
    part[blockIdx.x] = s;
  }
}

// b = (b - mean) * scale
__global__ void k_rhs_center(long long N, const double *__restrict__ part, int nparts, double scale,
                             double *__restrict__ b) {
  __shared__ double mean;
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int k = 0; k < nparts; ++k) s += part[k];
    mean = s / (double)N;
  }
  __syncthreads();
  const double m = mean;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x)
    b[p] = (b[p] - m) * scale;
}

}  // namespace
}  // namespace pbg

struct pbg_server {
  struct Session {
    int pid = -1;
    int nx = 0, ny = 0, nz = 0;
    double h = 0.0;
    long long bytes = 0;
    bool busy = false;
    std::deque<long long> queue;  // later requests of this session, in order
  };
  enum Kind { HOST = 0, DEVICE = 1, BUBBLE = 2 };
  struct Request {
    int sid = -1;
    int kind = HOST;
    bool fields = false;
    std::vector<double> rho, rhs;
    std::vector<uint8_t> solid;
    const double *drho = nullptr, *drhs = nullptr;
    const uint8_t *dsolid = nullptr;
    double center[3] = {0, 0, 0}, radius = 0, ratio = 1;
    unsigned long long seed = 0;
    pbg::Clock::time_point t_submit, t_done;
    bool done = false;
    pbg_result res;
  };

  int device = 0;
  pbg_server_config cfg;
  std::unique_ptr<pbg::BatchEngineBase> eng;
  pbg::DBuf<double> part;  // right-hand side generation scratch (worker only)

  std::mutex mu;                       // everything below
  std::condition_variable cv_work, cv_done;
  std::map<int, Session> sessions;
  int next_sid = 0;
  long long next_rid = 0;
  std::map<long long, Request> reqs;
  std::deque<long long> ready;         // requests whose session is idle, in arrival order
  std::map<int, long long> running;    // problem id -> request id
  long long bytes_used = 0, submitted = 0, completed = 0;
  bool stop = false;
  std::string worker_error;
  std::mutex eng_mu;                   // the engine (worker loop, session open/close)
  std::thread worker;

  void run();
  void start_request(long long rid, Request &r, Session &s);
};

namespace {

int sfail(int code, const std::string &m) {
  pbg::set_last_error(m.c_str());
  return code;
}

template <typename F>
int sguard(pbg_server *s, F &&f) {
  try {
    if (s) PBG_CUDA(cudaSetDevice(s->device));
    return f();
  } catch (const pbg::CudaError &e) {
    return sfail(PBG_ERR_CUDA, e.what());
  } catch (const std::invalid_argument &e) {
    return sfail(PBG_ERR_ARG, e.what());
  } catch (const std::bad_alloc &) {
    return sfail(PBG_ERR_NOMEM, "host allocation failed");
  } catch (const std::exception &e) {
    return sfail(PBG_ERR_STATE, e.what());
  }
}

}  // namespace

// Stage a request's inputs into its session's buffers and attach it
// (worker thread, engine and state locks held).
void pbg_server::start_request(long long rid, Request &r, Session &s) {
  const long long N = (long long)s.nx * s.ny * s.nz;
  if (r.kind == HOST) {
    if (r.fields) eng->set_fields(s.pid, r.rho.data(), r.solid.data(), PBG_HOST);
    eng->set_rhs(s.pid, r.rhs.data(), PBG_HOST);
  } else if (r.kind == DEVICE) {
    if (r.fields) eng->set_fields(s.pid, r.drho, r.dsolid, PBG_DEVICE);
    eng->set_rhs(s.pid, r.drhs, PBG_DEVICE);
  } else {
    const int g = pbg::grid_for(N);
    pbg::k_bubble_fields<<<g, pbg::kThreads, 0, eng->stream>>>(s.nx, s.ny, s.nz, r.center[0], r.center[1],
                                                               r.center[2], r.radius, r.ratio,
                                                               eng->device_rho(s.pid), eng->device_solid(s.pid));
    pbg::k_rhs_draw<<<pbg::kRhsBlocks, pbg::kThreads, 0, eng->stream>>>(N, r.seed, eng->device_rhs(s.pid), part.p);
    pbg::k_rhs_center<<<pbg::kRhsBlocks, pbg::kThreads, 0, eng->stream>>>(N, part.p, pbg::kRhsBlocks,
                                                                          1.0 / (s.h * s.h), eng->device_rhs(s.pid));
    PBG_CUDA(cudaGetLastError());
    for (int k = 0; k < 3; ++k) pbg::note_launch();
    eng->fields_changed(s.pid);
  }
  // host copies are no longer needed
  std::vector<double>().swap(r.rho);
  std::vector<double>().swap(r.rhs);
  std::vector<uint8_t>().swap(r.solid);
  pbg::BatchSolveParams p;
  p.tol = cfg.tol;
  p.inner_tol = cfg.inner_tol;
  p.max_sweeps = cfg.precision == PBG_FP64 ? std::min(cfg.max_sweeps, 4) : cfg.max_sweeps;
  p.max_iter = cfg.max_iter;
  p.inner_max_iter = cfg.max_iter;
  if (eng->attach(s.pid, p) < 0) throw std::runtime_error("server: no free slot");
  s.busy = true;
  running[s.pid] = rid;
}

void pbg_server::run() {
  try {
    PBG_CUDA(cudaSetDevice(device));
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu);
        std::lock_guard<std::mutex> ek(eng_mu);
        if (stop) break;
        while (!ready.empty() && eng->free_slots() > 0) {
          const long long rid = ready.front();
          ready.pop_front();
          Request &r = reqs.at(rid);
          start_request(rid, r, sessions.at(r.sid));
        }
        if (eng->active() == 0) {
          eng_mu.unlock();
          cv_work.wait_for(lk, std::chrono::milliseconds(50), [&] { return stop || !ready.empty(); });
          eng_mu.lock();
          continue;
        }
      }
      std::vector<std::pair<int, pbg::BatchOutcome>> done;
      std::vector<int> nlev;
      {
        std::lock_guard<std::mutex> ek(eng_mu);
        eng->step(cfg.iters_per_poll);
        done = eng->collect();
        for (auto &d : done) nlev.push_back(eng->levels(d.first));
      }
      if (done.empty()) continue;
      const auto now = pbg::Clock::now();
      std::lock_guard<std::mutex> lk(mu);
      for (size_t k = 0; k < done.size(); ++k) {
        const auto &d = done[k];
        const long long rid = running.at(d.first);
        running.erase(d.first);
        Request &r = reqs.at(rid);
        std::memset(&r.res, 0, sizeof(r.res));
        r.res.status = d.second.status;
        r.res.converged = d.second.converged;
        r.res.iterations = d.second.iterations;
        r.res.sweeps = d.second.sweeps;
        r.res.levels = nlev[k];
        r.res.res0 = d.second.relres0;
        r.res.res = d.second.relres;
        r.res.relres = d.second.relres;
        r.t_done = now;
        r.res.seconds = std::chrono::duration<double>(now - r.t_submit).count();
        r.done = true;
        ++completed;
        Session &s = sessions.at(r.sid);
        s.busy = false;
        if (!s.queue.empty()) {
          ready.push_back(s.queue.front());
          s.queue.pop_front();
        }
      }
      cv_done.notify_all();
    }
  } catch (const std::exception &e) {
    std::lock_guard<std::mutex> lk(mu);
    worker_error = e.what();
    stop = true;
    cv_done.notify_all();
  }
}

extern "C" {

void pbg_server_config_default(pbg_server_config *c) {
  if (!c) return;
  pbg_batch_config b;
  pbg_batch_config_default(&b);
  c->precision = PBG_MIXED;
  c->slots = 64;
  c->hbm_budget = 150ll * 1000 * 1000 * 1000;
  c->iters_per_poll = 1;
  c->threads = b.threads;
  c->tile_cells = b.tile_cells;
  c->grid = b.grid;
  c->kc_max = b.kc_max;
  c->tail_cells = b.tail_cells;
  c->tol = 1e-8;
  c->inner_tol = 1e-3;
  c->max_sweeps = 8;
  c->max_iter = 500;
}

int pbg_server_create(const pbg_server_config *c, int device, pbg_server **out) {
  if (!out) return sfail(PBG_ERR_ARG, "out is NULL");
  *out = nullptr;
  auto s = std::make_unique<pbg_server>();
  s->device = device;
  if (c) s->cfg = *c;
  else pbg_server_config_default(&s->cfg);
  pbg_server_config &k = s->cfg;
  if (k.precision != PBG_MIXED && k.precision != PBG_FP64) return sfail(PBG_ERR_ARG, "server: bad precision");
  if (k.slots < 1 || k.iters_per_poll < 1 || !(k.tol > 0.0) || k.max_sweeps < 1 || k.max_iter < 1)
    return sfail(PBG_ERR_ARG, "server: bad configuration");
  if (k.hbm_budget <= 0) k.hbm_budget = 150ll * 1000 * 1000 * 1000;
  int rc = sguard(s.get(), [&]() -> int {
    pbg::BatchShape sh;
    sh.threads = k.threads;
    sh.tile_cells = k.tile_cells;
    sh.grid = k.grid;
    sh.kc_max = k.kc_max;
    sh.tail_cells = k.tail_cells;
    s->eng = pbg::make_batch_engine(k.precision == PBG_MIXED ? 1 : 0, k.slots, sh);
    s->part.alloc(pbg::kRhsBlocks);
    return PBG_OK;
  });
  if (rc != PBG_OK) return rc;
  pbg_server *raw = s.get();
  s->worker = std::thread([raw] { raw->run(); });
  *out = s.release();
  return PBG_OK;
}

int pbg_server_destroy(pbg_server *s) {
  if (!s) return PBG_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  int rc = sguard(s, [&]() -> int {
    s->eng.reset();
    return PBG_OK;
  });
  delete s;
  return rc;
}

int pbg_server_open_session(pbg_server *s, int nx, int ny, int nz, double h, const int bc[6], int *sid) {
  if (!s || !sid) return sfail(PBG_ERR_ARG, "NULL argument");
  if (!(h > 0.0)) return sfail(PBG_ERR_ARG, "h must be > 0");
  return sguard(s, [&]() -> int {
    // problem_bytes only computes the layout (no device or shared state)
    const long long bytes = (long long)s->eng->problem_bytes(nx, ny, nz);
    {
      std::lock_guard<std::mutex> lk(s->mu);
      if (s->bytes_used + bytes > s->cfg.hbm_budget)
        return sfail(PBG_ERR_ADMISSION, "server: session does not fit the HBM budget");
      s->bytes_used += bytes;  // reserved until the session exists
    }
    int pid = -1;
    try {
      std::lock_guard<std::mutex> ek(s->eng_mu);
      pid = s->eng->create_problem(nx, ny, nz, h, bc);
    } catch (...) {
      std::lock_guard<std::mutex> lk(s->mu);
      s->bytes_used -= bytes;
      throw;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    pbg_server::Session ses;
    ses.pid = pid;
    ses.nx = nx; ses.ny = ny; ses.nz = nz; ses.h = h;
    ses.bytes = bytes;
    const int id = s->next_sid++;
    s->sessions[id] = ses;
    *sid = id;
    return PBG_OK;
  });
}

// Wait until the session has nothing queued or running (state lock held);
// false if the session is gone or the worker stopped.
static bool wait_idle(pbg_server *s, std::unique_lock<std::mutex> &lk, int sid) {
  auto idle = [&] {
    auto it = s->sessions.find(sid);
    if (s->stop || it == s->sessions.end()) return true;
    if (it->second.busy || !it->second.queue.empty()) return false;
    for (long long r : s->ready)
      if (s->reqs.at(r).sid == sid) return false;
    return true;
  };
  s->cv_done.wait(lk, idle);
  return s->sessions.count(sid) && !s->stop;
}

int pbg_server_close_session(pbg_server *s, int sid) {
  if (!s) return sfail(PBG_ERR_ARG, "NULL argument");
  return sguard(s, [&]() -> int {
    int pid;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      if (!s->sessions.count(sid)) return sfail(PBG_ERR_ARG, "server: unknown session");
      if (!wait_idle(s, lk, sid)) return sfail(PBG_ERR_STATE, "server: worker stopped: " + s->worker_error);
      pid = s->sessions.at(sid).pid;
      s->bytes_used -= s->sessions.at(sid).bytes;
      s->sessions.erase(sid);
    }
    std::lock_guard<std::mutex> ek(s->eng_mu);
    s->eng->destroy_problem(pid);
    return PBG_OK;
  });
}

static int enqueue(pbg_server *s, int sid, pbg_server::Request &&r, long long *rid) {
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) return sfail(PBG_ERR_STATE, "server: stopped: " + s->worker_error);
  auto it = s->sessions.find(sid);
  if (it == s->sessions.end()) return sfail(PBG_ERR_ARG, "server: unknown session");
  r.sid = sid;
  r.t_submit = pbg::Clock::now();
  const long long id = s->next_rid++;
  s->reqs.emplace(id, std::move(r));
  pbg_server::Session &ses = it->second;
  bool waiting = ses.busy;
  for (long long q : s->ready)
    if (s->reqs.at(q).sid == sid) waiting = true;
  if (waiting) ses.queue.push_back(id);
  else s->ready.push_back(id);
  ++s->submitted;
  *rid = id;
  s->cv_work.notify_one();
  return PBG_OK;
}

int pbg_server_submit(pbg_server *s, int sid, const double *rho, const uint8_t *solid, const double *rhs,
                      int where, long long *rid) {
  if (!s || !rhs || !rid || (!rho) != (!solid)) return sfail(PBG_ERR_ARG, "bad arguments");
  return sguard(s, [&]() -> int {
    long long N;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      auto it = s->sessions.find(sid);
      if (it == s->sessions.end()) return sfail(PBG_ERR_ARG, "server: unknown session");
      N = (long long)it->second.nx * it->second.ny * it->second.nz;
    }
    pbg_server::Request r;
    r.fields = rho != nullptr;
    if (where == PBG_HOST) {
      r.kind = pbg_server::HOST;
      r.rhs.assign(rhs, rhs + N);
      if (r.fields) {
        r.rho.assign(rho, rho + N);
        r.solid.assign(solid, solid + N);
      }
    } else {
      r.kind = pbg_server::DEVICE;
      r.drhs = rhs;
      r.drho = rho;
      r.dsolid = solid;
    }
    return enqueue(s, sid, std::move(r), rid);
  });
}

int pbg_server_submit_bubble(pbg_server *s, int sid, const double center[3], double radius, double ratio,
                             unsigned long long rhs_seed, long long *rid) {
  if (!s || !center || !rid || !(radius >= 0.0) || !(ratio > 0.0)) return sfail(PBG_ERR_ARG, "bad arguments");
  return sguard(s, [&]() -> int {
    pbg_server::Request r;
    r.kind = pbg_server::BUBBLE;
    r.fields = true;
    for (int k = 0; k < 3; ++k) r.center[k] = center[k];
    r.radius = radius;
    r.ratio = ratio;
    r.seed = rhs_seed;
    return enqueue(s, sid, std::move(r), rid);
  });
}

int pbg_server_wait(pbg_server *s, long long rid, double timeout_s, pbg_result *res, double *latency_s) {
  if (!s) return sfail(PBG_ERR_ARG, "NULL argument");
  return sguard(s, [&]() -> int {
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(rid);
    if (it == s->reqs.end()) return sfail(PBG_ERR_ARG, "server: unknown request");
    auto ready_fn = [&] { return s->stop || s->reqs.at(rid).done; };
    if (timeout_s < 0) s->cv_done.wait(lk, ready_fn);
    else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready_fn))
      return sfail(PBG_ERR_STATE, "server: wait timed out");
    pbg_server::Request &r = s->reqs.at(rid);
    if (!r.done) return sfail(PBG_ERR_STATE, "server: worker stopped: " + s->worker_error);
    if (res) *res = r.res;
    if (latency_s) *latency_s = r.res.seconds;
    s->reqs.erase(rid);
    return PBG_OK;
  });
}

int pbg_server_get_x(pbg_server *s, int sid, double *x, int where) {
  if (!s || !x) return sfail(PBG_ERR_ARG, "NULL argument");
  return sguard(s, [&]() -> int {
    int pid;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      if (!s->sessions.count(sid)) return sfail(PBG_ERR_ARG, "server: unknown session");
      if (!wait_idle(s, lk, sid)) return sfail(PBG_ERR_STATE, "server: worker stopped: " + s->worker_error);
      pid = s->sessions.at(sid).pid;
    }
    std::lock_guard<std::mutex> ek(s->eng_mu);
    s->eng->get_x(pid, x, where);
    return PBG_OK;
  });
}

int pbg_server_stats_get(pbg_server *s, pbg_server_stats *st) {
  if (!s || !st) return sfail(PBG_ERR_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  st->submitted = s->submitted;
  st->completed = s->completed;
  st->in_flight = (long long)s->running.size();
  st->queued = s->submitted - s->completed - st->in_flight;
  st->sessions = (long long)s->sessions.size();
  st->device_bytes = s->bytes_used;
  st->kernel_launches = s->eng ? s->eng->kernel_launches() : 0;
  return PBG_OK;
}

}  // extern "C"
