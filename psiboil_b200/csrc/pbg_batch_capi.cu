// C ABI of the batched engine (pbg_batch_*) and its autotuner.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <new>
#include <numeric>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/psiboil_b200.h"
#include "pbg_batch_engine.h"
#include "pbg_common.cuh"

namespace pbg {
void set_last_error(const char *msg);  // pbg_capi.cu
}

struct pbg_batch {
  int device = 0;
  pbg_batch_config cfg;
  std::unique_ptr<pbg::BatchEngineBase> eng;
  std::vector<long long> cells;  // per problem id (0: removed)
};

namespace {

using pbg::BatchShape;
using pbg::BatchSolveParams;

int bfail(int code, const std::string &m) {
  pbg::set_last_error(m.c_str());
  return code;
}

template <typename F>
int bguard(pbg_batch *b, F &&f) {
  try {
    if (b) PBG_CUDA(cudaSetDevice(b->device));
    return f();
  } catch (const pbg::CudaError &e) {
    return bfail(PBG_ERR_CUDA, e.what());
  } catch (const std::invalid_argument &e) {
    return bfail(PBG_ERR_ARG, e.what());
  } catch (const std::bad_alloc &) {
    return bfail(PBG_ERR_NOMEM, "host allocation failed");
  } catch (const std::exception &e) {
    return bfail(PBG_ERR_STATE, e.what());
  }
}

BatchShape shape_of(const pbg_batch_config &c) {
  BatchShape s;
  s.threads = c.threads;
  s.tile_cells = c.tile_cells;
  s.grid = c.grid;
  s.kc_max = c.kc_max;
  s.tail_cells = c.tail_cells;
  return s;
}

BatchSolveParams solve_params(const pbg_params *p, int precision) {
  BatchSolveParams q;
  if (p) {
    q.tol = p->tol;
    q.inner_tol = p->inner_tol;
    q.max_sweeps = p->max_sweeps;
    q.max_iter = p->max_iter;
    q.inner_max_iter = p->max_iter;
  }
  if (precision == PBG_FP64 && q.max_sweeps > 4) q.max_sweeps = 4;  // as the engine's FP64 path
  if (!(q.tol > 0.0) || q.max_sweeps < 1 || q.max_iter < 1)
    throw std::invalid_argument("batch: tol must be > 0, max_sweeps and max_iter >= 1");
  return q;
}

// Solve ids to completion: largest first, each entering as soon as a slot
// is free. Fills res (may be null). Returns the wall seconds.
double run_solve(pbg_batch *b, const int *ids, int n, const pbg_params *p, pbg_result *res) {
  const BatchSolveParams prm = solve_params(p, b->cfg.precision);
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  for (int i = 0; i < n; ++i)
    if (ids[i] < 0 || ids[i] >= (int)b->cells.size() || b->cells[ids[i]] == 0)
      throw std::invalid_argument("batch: unknown problem id");
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int c) { return b->cells[ids[a]] > b->cells[ids[c]]; });
  std::vector<int> index_of(b->cells.size(), -1);
  for (int i = 0; i < n; ++i) {
    if (index_of[ids[i]] >= 0) throw std::invalid_argument("batch: a problem id appears twice");
    index_of[ids[i]] = i;
  }
  if (res) std::memset(res, 0, sizeof(pbg_result) * n);
  const auto t0 = std::chrono::steady_clock::now();
  int next = 0, finished = 0, chunk = 2;
  long long stepped = 0;
  const long long limit = (long long)prm.max_iter * prm.max_sweeps + 64ll * prm.max_sweeps + 64;
  long long since_admit = 0;
  while (finished < n) {
    while (next < n && b->eng->free_slots() > 0) {
      if (b->eng->attach(ids[order[next]], prm) < 0) break;
      ++next;
      since_admit = 0;
    }
    b->eng->step(chunk);
    stepped += chunk;
    since_admit += chunk;
    auto done = b->eng->collect();
    const double now = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    for (auto &d : done) {
      ++finished;
      if (!res) continue;
      pbg_result &r = res[index_of[d.first]];
      r.status = d.second.status;
      r.converged = d.second.converged;
      r.iterations = d.second.iterations;
      r.sweeps = d.second.sweeps;
      r.levels = b->eng->levels(d.first);
      r.res0 = d.second.relres0;
      r.res = d.second.relres;
      r.relres = d.second.relres;
      r.seconds = now;
    }
    chunk = done.empty() ? std::min(chunk * 2, 16) : 2;
    // every attached problem finishes within `limit` outer iterations
    if (since_admit > limit) throw std::runtime_error("batch: solve did not finish (iteration bound exceeded)");
  }
  (void)stepped;
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

std::string device_name(int dev) {
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return "unknown";
  return prop.name;
}

// Key of an autotuning result: device, precision and the batch's sizes.
std::string tune_key(pbg_batch *b, const int *ids, int n) {
  unsigned long long h = 1469598103934665603ull;  // FNV-1a over the cell counts
  long long total = 0;
  for (int i = 0; i < n; ++i) {
    const long long c = b->cells[ids[i]];
    total += c;
    for (int k = 0; k < 8; ++k) { h ^= (unsigned long long)((c >> (8 * k)) & 0xff); h *= 1099511628211ull; }
  }
  std::ostringstream os;
  os << device_name(b->device) << "|p" << b->cfg.precision << "|n" << n << "|c" << total << "|h" << std::hex << h;
  std::string s = os.str();
  for (char &ch : s)
    if (ch == '"' || ch == '\\') ch = '_';
  return s;
}

bool tune_read(const std::string &path, const std::string &key, pbg_batch_config &c) {
  std::ifstream f(path);
  if (!f) return false;
  std::string line, want = "\"" + key + "\"";
  while (std::getline(f, line)) {
    const size_t at = line.find(want);
    if (at == std::string::npos) continue;
    int th, tc, g, kc, tl;
    const char *q = line.c_str() + at + want.size();
    if (std::sscanf(q, ": {\"threads\": %d, \"tile_cells\": %d, \"grid\": %d, \"kc_max\": %d, \"tail_cells\": %d",
                    &th, &tc, &g, &kc, &tl) == 5) {
      c.threads = th; c.tile_cells = tc; c.grid = g; c.kc_max = kc; c.tail_cells = tl;
      return true;
    }
  }
  return false;
}

// The cache file is a JSON object with one entry per line.
void tune_write(const std::string &path, const std::string &key, const pbg_batch_config &c, double ms) {
  std::vector<std::string> entries;
  {
    std::ifstream f(path);
    std::string line, want = "\"" + key + "\"";
    while (f && std::getline(f, line)) {
      if (line.find("\": {\"threads\"") == std::string::npos || line.find(want) != std::string::npos) continue;
      while (!line.empty() && (line.back() == ',' || line.back() == ' ')) line.pop_back();
      entries.push_back(line);
    }
  }
  char buf[512];
  std::snprintf(buf, sizeof(buf),
                "  \"%s\": {\"threads\": %d, \"tile_cells\": %d, \"grid\": %d, \"kc_max\": %d, \"tail_cells\": %d, \"ms\": %.3f}",
                key.c_str(), c.threads, c.tile_cells, c.grid, c.kc_max, c.tail_cells, ms);
  entries.push_back(buf);
  std::ofstream o(path);
  o << "{\n";
  for (size_t i = 0; i < entries.size(); ++i) o << entries[i] << (i + 1 < entries.size() ? ",\n" : "\n");
  o << "}\n";
}

}  // namespace

extern "C" {

void pbg_batch_config_default(pbg_batch_config *c) {
  if (!c) return;
  BatchShape s;
  c->precision = PBG_MIXED;
  c->slots = 64;
  c->threads = s.threads;
  c->tile_cells = s.tile_cells;
  c->grid = s.grid;
  c->kc_max = s.kc_max;
  c->tail_cells = s.tail_cells;
}

int pbg_batch_create(const pbg_batch_config *c, int device, pbg_batch **out) {
  if (!out) return bfail(PBG_ERR_ARG, "out is NULL");
  *out = nullptr;
  auto b = std::make_unique<pbg_batch>();
  b->device = device;
  if (c) b->cfg = *c;
  else pbg_batch_config_default(&b->cfg);
  if (b->cfg.precision != PBG_MIXED && b->cfg.precision != PBG_FP64)
    return bfail(PBG_ERR_ARG, "batch: precision must be PBG_MIXED or PBG_FP64");
  int rc = bguard(b.get(), [&]() -> int {
    b->eng = pbg::make_batch_engine(b->cfg.precision == PBG_MIXED ? 1 : 0, b->cfg.slots, shape_of(b->cfg));
    return PBG_OK;
  });
  if (rc == PBG_OK) *out = b.release();
  return rc;
}

int pbg_batch_destroy(pbg_batch *b) {
  if (!b) return PBG_OK;
  int rc = bguard(b, [&]() -> int {
    b->eng.reset();
    return PBG_OK;
  });
  delete b;
  return rc;
}

int pbg_batch_problem_bytes(pbg_batch *b, int nx, int ny, int nz, long long *bytes) {
  if (!b || !bytes) return bfail(PBG_ERR_ARG, "NULL argument");
  return bguard(b, [&]() -> int {
    *bytes = (long long)b->eng->problem_bytes(nx, ny, nz);
    return PBG_OK;
  });
}

int pbg_batch_add(pbg_batch *b, int nx, int ny, int nz, double h, const int bc[6], int *id) {
  if (!b || !id) return bfail(PBG_ERR_ARG, "NULL argument");
  if (!(h > 0.0)) return bfail(PBG_ERR_ARG, "h must be > 0");
  return bguard(b, [&]() -> int {
    const int k = b->eng->create_problem(nx, ny, nz, h, bc);
    if (k >= (int)b->cells.size()) b->cells.resize(k + 1, 0);
    b->cells[k] = (long long)nx * ny * nz;
    *id = k;
    return PBG_OK;
  });
}

int pbg_batch_remove(pbg_batch *b, int id) {
  if (!b) return bfail(PBG_ERR_ARG, "NULL argument");
  return bguard(b, [&]() -> int {
    b->eng->destroy_problem(id);
    b->cells[id] = 0;
    return PBG_OK;
  });
}

int pbg_batch_set_fields(pbg_batch *b, int id, const double *rho, const uint8_t *solid, int where) {
  if (!b || !rho || !solid) return bfail(PBG_ERR_ARG, "NULL argument");
  return bguard(b, [&]() -> int {
    b->eng->set_fields(id, rho, solid, where);
    return PBG_OK;
  });
}

int pbg_batch_set_rhs(pbg_batch *b, int id, const double *rhs, int where) {
  if (!b || !rhs) return bfail(PBG_ERR_ARG, "NULL argument");
  return bguard(b, [&]() -> int {
    b->eng->set_rhs(id, rhs, where);
    return PBG_OK;
  });
}

int pbg_batch_set_x(pbg_batch *b, int id, const double *x, int where) {
  if (!b) return bfail(PBG_ERR_ARG, "NULL argument");
  return bguard(b, [&]() -> int {
    if (x) b->eng->set_x(id, x, where);
    else b->eng->zero_x(id);
    return PBG_OK;
  });
}

int pbg_batch_get_x(pbg_batch *b, int id, double *x, int where) {
  if (!b || !x) return bfail(PBG_ERR_ARG, "NULL argument");
  return bguard(b, [&]() -> int {
    b->eng->get_x(id, x, where);
    return PBG_OK;
  });
}

int pbg_batch_solve(pbg_batch *b, const int *ids, int n, const pbg_params *p, pbg_result *res) {
  if (!b || (n > 0 && !ids) || n < 0) return bfail(PBG_ERR_ARG, "bad arguments");
  return bguard(b, [&]() -> int {
    run_solve(b, ids, n, p, res);
    return PBG_OK;
  });
}

int pbg_batch_autotune(pbg_batch *b, const int *ids, int n, const pbg_params *p,
                       const char *cache_path, pbg_batch_config *best) {
  if (!b || !ids || n < 1) return bfail(PBG_ERR_ARG, "bad arguments");
  return bguard(b, [&]() -> int {
    const std::string key = tune_key(b, ids, n);
    pbg_batch_config cfg = b->cfg;
    if (cache_path && tune_read(cache_path, key, cfg)) {
      b->eng->set_shape(shape_of(cfg));
      b->cfg = cfg;
      if (best) *best = cfg;
      return PBG_OK;
    }
    auto timed = [&](const pbg_batch_config &c) {
      b->eng->set_shape(shape_of(c));
      for (int i = 0; i < n; ++i) b->eng->zero_x(ids[i]);
      return run_solve(b, ids, n, p, nullptr);
    };
    // warm-up (hierarchy set-up, graph capture), then coordinate descent
    timed(cfg);
    double best_s = timed(cfg);
    pbg_batch_config bc = cfg;
    auto consider = [&](pbg_batch_config c) {
      if (c.tile_cells < c.threads) return;
      timed(c);  // capture
      const double s = timed(c);
      if (s < best_s) { best_s = s; bc = c; }
    };
    for (int th : {128, 256, 512})
      for (int mult : {2, 4, 8, 16, 32}) {
        pbg_batch_config c = bc;
        c.threads = th;
        c.tile_cells = th * mult;
        if (c.threads == cfg.threads && c.tile_cells == cfg.tile_cells) continue;
        consider(c);
      }
    const pbg_batch_config after_tiles = bc;
    for (int g : {148 * 2, 148 * 4, 148 * 8, 148 * 16}) {
      pbg_batch_config c = after_tiles;
      c.grid = g;
      if (g == after_tiles.grid) continue;
      consider(c);
    }
    const pbg_batch_config after_grid = bc;
    for (int kc : {1, 2, 3, 4, 99}) {
      pbg_batch_config c = after_grid;
      c.kc_max = kc;
      if (kc == after_grid.kc_max) continue;
      consider(c);
    }
    const pbg_batch_config after_kc = bc;
    for (int tl : {0, 512, 1024, 4096, 16384}) {
      pbg_batch_config c = after_kc;
      c.tail_cells = tl;
      if (tl == after_kc.tail_cells) continue;
      consider(c);
    }
    b->eng->set_shape(shape_of(bc));
    for (int i = 0; i < n; ++i) b->eng->zero_x(ids[i]);
    b->cfg = bc;
    if (cache_path) tune_write(cache_path, key, bc, best_s * 1e3);
    if (best) *best = bc;
    return PBG_OK;
  });
}

}  // extern "C"
