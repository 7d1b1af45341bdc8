// Batched engine, host side: problem arenas, slots, flat tile lists, the
// captured iteration graph per hierarchy depth, and the continuous
// attach / step / collect loop (pbg_batch_engine.h).
#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "pbg_batch.cuh"
#include "pbg_batch_engine.h"

namespace pbg {

namespace {

constexpr size_t kAlign = 256;

size_t align_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

// Level sizes of the aggregation hierarchy: halve (rounding up) every
// direction longer than 1 until at most kBDenseMax cells remain.
int level_dims(int nx, int ny, int nz, int (*d)[3]) {
  int l = 0;
  d[0][0] = nx; d[0][1] = ny; d[0][2] = nz;
  while ((long long)d[l][0] * d[l][1] * d[l][2] > kBDenseMax) {
    if (l + 1 >= kBMaxLev) return -1;
    for (int a = 0; a < 3; ++a) d[l + 1][a] = d[l][a] > 1 ? (d[l][a] + 1) / 2 : 1;
    ++l;
  }
  return l + 1;
}

}  // namespace

template <typename T>
class BatchEngine : public BatchEngineBase {
  static constexpr bool kMixed = sizeof(T) == 4;

  struct Prob {
    int nx, ny, nz, nlev;
    double h;
    int bc[6];
    int dims[kBMaxLev][3];
    DBuf<char> arena;
    size_t bytes = 0;
    BProb<T> d;              // device pointers into the arena
    double *rho = nullptr;   // assembly inputs in the arena
    uint8_t *solid = nullptr;
    bool assemble = false;   // rho/solid given (else the level-0 FP64 matrix)
    bool need_setup = true;
    bool have_matrix = false;
    int slot = -1;
  };

  std::vector<std::unique_ptr<Prob>> probs_;
  int S_;
  BatchShape shape_;
  std::vector<int> slot_pid_;
  int active_ = 0;
  bool tiles_dirty_ = true, setup_pending_ = false;
  int dmax_ = 0;
  unsigned long long sig_ = 0;  // launch-sequence signature of the attached slots

  DBuf<BProb<T>> dprob_;
  DBuf<BState> dst_;
  DBuf<BTile> dtiles_;
  size_t tile_cap_ = 0;
  DBuf<int> dlbeg_, dtbeg_, dtcnt_;
  DBuf<double> dpart_;
  DBuf<unsigned> dcnt_;
  // pinned host staging
  BProb<T> *hprob_ = nullptr;
  BState *hst_ = nullptr, *hout_ = nullptr;
  int *hphase_ = nullptr;
  char *htile_ = nullptr;
  size_t htile_cap_ = 0;

  struct Graph {
    cudaGraphExec_t exec = nullptr;
    size_t nodes = 0;
  };
  // graphs by (launch-sequence signature, per-level grid code)
  std::map<std::pair<unsigned long long, unsigned long long>, Graph> graphs_;
  int lgrid_[kBMaxLev] = {};     // tile-kernel grid per level: min(grid, tiles rounded up to 2^k)
  unsigned long long gcode_ = 0; // the lgrid_ values, 5 bits of log2 each
  unsigned long long launches_ = 0;

 public:
  BatchEngine(int slots, const BatchShape &shape) : S_(slots), shape_(shape), slot_pid_(slots, -1) {
    if (slots < 1) throw std::invalid_argument("batch: slots must be >= 1");
    check_shape(shape_);
    PBG_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    dprob_.alloc(S_);
    dst_.alloc(S_);
    dtbeg_.alloc((size_t)kBMaxLev * S_);
    dtcnt_.alloc((size_t)kBMaxLev * S_);
    dlbeg_.alloc(kBMaxLev + 1);
    dcnt_.alloc((size_t)kBMaxLev * S_);
    PBG_CUDA(cudaMemset(dst_.p, 0, sizeof(BState) * S_));
    PBG_CUDA(cudaMemset(dcnt_.p, 0, sizeof(unsigned) * kBMaxLev * S_));
    PBG_CUDA(cudaMemset(dlbeg_.p, 0, sizeof(int) * (kBMaxLev + 1)));
    PBG_CUDA(cudaMallocHost((void **)&hprob_, sizeof(BProb<T>) * S_));
    PBG_CUDA(cudaMallocHost((void **)&hst_, sizeof(BState) * S_));
    PBG_CUDA(cudaMallocHost((void **)&hout_, sizeof(BState) * S_));
    PBG_CUDA(cudaMallocHost((void **)&hphase_, sizeof(int) * S_));
  }

  ~BatchEngine() override {
    if (stream) cudaStreamSynchronize(stream);
    drop_graphs();
    if (hprob_) cudaFreeHost(hprob_);
    if (hst_) cudaFreeHost(hst_);
    if (hout_) cudaFreeHost(hout_);
    if (hphase_) cudaFreeHost(hphase_);
    if (htile_) cudaFreeHost(htile_);
    probs_.clear();
    if (stream) cudaStreamDestroy(stream);
  }

  static void check_shape(const BatchShape &s) {
    if (s.threads < 64 || s.threads > kBThreadsMax || s.threads % 32)
      throw std::invalid_argument("batch: threads must be a multiple of 32 in [64, 512]");
    if (s.tile_cells < s.threads || s.tile_cells > (1 << 20) || s.tile_cells % 4)
      throw std::invalid_argument("batch: tile_cells must be a multiple of 4 in [threads, 2^20]");
    if (s.grid < 1 || s.grid > 65535) throw std::invalid_argument("batch: grid must be in [1, 65535]");
    if (s.kc_max < 0) throw std::invalid_argument("batch: kc_max must be >= 0");
    if (s.tail_cells < 0 || s.tail_cells > (1 << 20)) throw std::invalid_argument("batch: tail_cells must be in [0, 2^20]");
  }

  // ------------------------------------------------------------ problems
  // Padded level-0 geometry of the inner solve (kBPad): (nx, ny0, nzp) with
  // true fast extent F; otherwise the compact one.
  static void level0_pad(int nx, int ny, int nz, int &ny0, int &F, int &nzp) {
    (void)nx;
    if (!kBPad<T>) { ny0 = ny; F = nz; nzp = nz; return; }
    if (nz == 1) { ny0 = 1; F = ny; }
    else { ny0 = ny; F = nz; }
    nzp = (F + 3) / 4 * 4;
  }

  static size_t level_cells(const Prob &P, int l) {
    if (l == 0 && kBPad<T>) return (size_t)P.nx * P.d.L[0].A.ny * P.d.L[0].A.nz;
    return (size_t)P.dims[l][0] * P.dims[l][1] * P.dims[l][2];
  }

  size_t layout(int nx, int ny, int nz, Prob *P) const {
    int dims[kBMaxLev][3];
    const int nlev = level_dims(nx, ny, nz, dims);
    int ny0, F, nzp;
    level0_pad(nx, ny, nz, ny0, F, nzp);
    const size_t n0p = (size_t)nx * ny0 * nzp;
    if (nlev < 2) throw std::invalid_argument("batch: a problem needs more than 64 cells and at most 12 levels");
    size_t off = 0;
    // every array ends with 256 bytes of slack: the vectorised kernels' last
    // group and their shifted pairs of 16-byte loads may read past the end
    auto take = [&](size_t bytes) {
      const size_t o = off;
      off += align_up(bytes + 256);
      return o;
    };
    struct Off { size_t c64, w64, s64, b64, c, w, s, b, d, vb, vx, z1, z2, q1, r1, xa, xb; };
    Off lo[kBMaxLev];
    for (int l = 0; l < nlev; ++l) {
      const size_t n = (size_t)dims[l][0] * dims[l][1] * dims[l][2];
      const size_t nt = l == 0 ? n0p : n;  // cells of the level's T arrays
      Off &o = lo[l];
      o.c64 = take(8 * n); o.w64 = take(8 * n); o.s64 = take(8 * n); o.b64 = take(8 * n);
      if (kMixed) { o.c = take(4 * nt); o.w = take(4 * nt); o.s = take(4 * nt); o.b = take(4 * nt); }
      o.d = take(sizeof(T) * nt);
      if (l > 0) {
        o.vb = take(sizeof(T) * n); o.vx = take(sizeof(T) * n); o.z1 = take(sizeof(T) * n);
        o.z2 = take(sizeof(T) * n); o.q1 = take(sizeof(T) * n); o.r1 = take(sizeof(T) * n);
      }
      o.xa = take(sizeof(T) * nt); o.xb = take(sizeof(T) * nt);
    }
    const size_t n0 = (size_t)nx * ny * nz;
    const size_t ox0 = take(sizeof(T) * n0p), or0 = take(sizeof(T) * n0p), oz0 = take(sizeof(T) * n0p),
                 opA = take(sizeof(T) * n0p), opB = take(sizeof(T) * n0p), oq0 = take(sizeof(T) * n0p);
    const size_t ox = take(8 * n0), ob = take(8 * n0), orho = take(8 * n0), osol = take(n0);
    const int nc = dims[nlev - 1][0] * dims[nlev - 1][1] * dims[nlev - 1][2];
    const size_t oai = take(8 * (size_t)nc * nc);
    if (!P) return off;
    // assign pointers
    P->nlev = nlev;
    std::memcpy(P->dims, dims, sizeof(dims));
    P->arena.alloc(off);
    P->bytes = off;
    char *base = P->arena.p;
    auto at = [&](size_t o) { return (void *)(base + o); };
    BProb<T> &d = P->d;
    std::memset(&d, 0, sizeof(d));
    d.nlev = nlev;
    d.ncoarse = nc;
    d.nx = nx; d.ny = ny; d.nz = nz;
    d.F = F; d.nzp = nzp; d.rel2d = (kBPad<T> && nz == 1) ? 1 : 0;
    d.g0 = Geo(nx, ny, nz);
    for (int l = 0; l < nlev; ++l) {
      const Off &o = lo[l];
      BLev<T> &V = d.L[l];
      V.c64 = (double *)at(o.c64); V.w64 = (double *)at(o.w64); V.s64 = (double *)at(o.s64); V.b64 = (double *)at(o.b64);
      const T *c, *w, *s, *b;
      if (kMixed) { c = (T *)at(o.c); w = (T *)at(o.w); s = (T *)at(o.s); b = (T *)at(o.b); }
      else { c = (T *)V.c64; w = (T *)V.w64; s = (T *)V.s64; b = (T *)V.b64; }
      if (l == 0 && kBPad<T>) V.A = make_emat<T>(nx, ny0, nzp, c, w, s, b, (T *)at(o.d));
      else V.A = make_emat<T>(dims[l][0], dims[l][1], dims[l][2], c, w, s, b, (T *)at(o.d));
      if (l > 0) {
        V.b = (T *)at(o.vb); V.x = (T *)at(o.vx); V.z1 = (T *)at(o.z1); V.z2 = (T *)at(o.z2);
        V.q1 = (T *)at(o.q1); V.r1 = (T *)at(o.r1);
      }
      V.xa = (T *)at(o.xa); V.xb = (T *)at(o.xb);
    }
    d.x0 = (T *)at(ox0); d.r0 = (T *)at(or0); d.z0 = (T *)at(oz0);
    d.pA = (T *)at(opA); d.pB = (T *)at(opB); d.q0 = (T *)at(oq0);
    d.x = (double *)at(ox);
    d.b = (const double *)at(ob);
    P->rho = (double *)at(orho);
    P->solid = (uint8_t *)at(osol);
    d.Ainv = (double *)at(oai);
    return off;
  }

  size_t problem_bytes(int nx, int ny, int nz) const override { return layout(nx, ny, nz, nullptr); }

  int create_problem(int nx, int ny, int nz, double h, const int bc[6]) override {
    if (nx < 1 || ny < 1 || nz < 1 || (long long)nx * ny * nz >= (1ll << 31))
      throw std::invalid_argument("batch: bad dimensions");
    auto P = std::make_unique<Prob>();
    P->nx = nx; P->ny = ny; P->nz = nz; P->h = h;
    // default: Neumann walls, Dirichlet top (kmax in 3-D, jmax in 2-D)
    const int top = nz > 1 ? 5 : 3;
    for (int f = 0; f < 6; ++f) P->bc[f] = bc ? bc[f] : (f == top ? PBG_BC_DIRICHLET : PBG_BC_NEUMANN);
    layout(nx, ny, nz, P.get());
    // pad cells (and everything else) start at zero; kernels keep pads zero
    PBG_CUDA(cudaMemsetAsync(P->arena.p, 0, P->bytes, stream));
    P->d.h = h;
    for (int f = 0; f < 6; ++f) P->d.bc[f] = P->bc[f];
    PBG_CUDA(cudaMemsetAsync(P->d.x, 0, 8 * (size_t)nx * ny * nz, stream));
    PBG_CUDA(cudaMemsetAsync((void *)P->d.b, 0, 8 * (size_t)nx * ny * nz, stream));
    for (size_t i = 0; i < probs_.size(); ++i)
      if (!probs_[i]) { probs_[i] = std::move(P); return (int)i; }
    probs_.push_back(std::move(P));
    return (int)probs_.size() - 1;
  }

  Prob &get(int id) const {
    if (id < 0 || id >= (int)probs_.size() || !probs_[id]) throw std::invalid_argument("batch: unknown problem id");
    return *probs_[id];
  }

  void destroy_problem(int id) override {
    Prob &P = get(id);
    if (P.slot >= 0) throw std::runtime_error("batch: problem is being solved");
    PBG_CUDA(cudaStreamSynchronize(stream));
    probs_[id].reset();
  }

  int levels(int id) const override { return get(id).nlev; }

  static cudaMemcpyKind kind(int where) { return where == 1 ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice; }

  void set_fields(int id, const double *rho, const uint8_t *solid, int where) override {
    Prob &P = get(id);
    if (P.slot >= 0) throw std::runtime_error("batch: problem is being solved");
    const size_t n = (size_t)P.nx * P.ny * P.nz;
    PBG_CUDA(cudaMemcpyAsync(P.rho, rho, 8 * n, kind(where), stream));
    PBG_CUDA(cudaMemcpyAsync(P.solid, solid, n, kind(where), stream));
    P.assemble = true;
    P.have_matrix = true;
    P.need_setup = true;
  }

  void set_matrix(int id, const double *c, const double *w, const double *s, const double *b, int where) override {
    Prob &P = get(id);
    if (P.slot >= 0) throw std::runtime_error("batch: problem is being solved");
    const size_t n = (size_t)P.nx * P.ny * P.nz;
    const BLev<T> &V = P.d.L[0];
    PBG_CUDA(cudaMemcpyAsync(V.c64, c, 8 * n, kind(where), stream));
    PBG_CUDA(cudaMemcpyAsync(V.w64, w, 8 * n, kind(where), stream));
    PBG_CUDA(cudaMemcpyAsync(V.s64, s, 8 * n, kind(where), stream));
    PBG_CUDA(cudaMemcpyAsync(V.b64, b, 8 * n, kind(where), stream));
    P.assemble = false;
    P.have_matrix = true;
    P.need_setup = true;
  }

  void set_rhs(int id, const double *b, int where) override {
    Prob &P = get(id);
    if (P.slot >= 0) throw std::runtime_error("batch: problem is being solved");
    PBG_CUDA(cudaMemcpyAsync((void *)P.d.b, b, 8 * (size_t)P.nx * P.ny * P.nz, kind(where), stream));
  }

  void set_x(int id, const double *x, int where) override {
    Prob &P = get(id);
    if (P.slot >= 0) throw std::runtime_error("batch: problem is being solved");
    PBG_CUDA(cudaMemcpyAsync(P.d.x, x, 8 * (size_t)P.nx * P.ny * P.nz, kind(where), stream));
  }

  void zero_x(int id) override {
    Prob &P = get(id);
    if (P.slot >= 0) throw std::runtime_error("batch: problem is being solved");
    PBG_CUDA(cudaMemsetAsync(P.d.x, 0, 8 * (size_t)P.nx * P.ny * P.nz, stream));
  }

  void get_x(int id, double *x, int where) override {
    Prob &P = get(id);
    if (P.slot >= 0) throw std::runtime_error("batch: problem is being solved");
    PBG_CUDA(cudaMemcpyAsync(x, P.d.x, 8 * (size_t)P.nx * P.ny * P.nz,
                             where == 1 ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, stream));
    PBG_CUDA(cudaStreamSynchronize(stream));
  }

  double *device_x(int id) override { return get(id).d.x; }
  double *device_rhs(int id) override { return const_cast<double *>(get(id).d.b); }
  double *device_rho(int id) override { return get(id).rho; }
  uint8_t *device_solid(int id) override { return get(id).solid; }
  void fields_changed(int id) override {
    Prob &P = get(id);
    if (P.slot >= 0) throw std::runtime_error("batch: problem is being solved");
    P.assemble = true;
    P.have_matrix = true;
    P.need_setup = true;
  }

  // ------------------------------------------------------------ slots
  int free_slots() const override { return S_ - active_; }
  int active() const override { return active_; }

  int attach(int id, const BatchSolveParams &prm) override {
    Prob &P = get(id);
    if (P.slot >= 0) throw std::runtime_error("batch: problem already attached");
    if (!P.have_matrix) throw std::runtime_error("batch: problem has no matrix");
    int s = -1;
    for (int q = 0; q < S_; ++q)
      if (slot_pid_[q] < 0) { s = q; break; }
    if (s < 0) return -1;
    // the staging entries of this slot may still feed an earlier copy
    PBG_CUDA(cudaStreamSynchronize(stream));
    BProb<T> &d = hprob_[s];
    d = P.d;
    d.tail = tail_level(P);
    d.rho = P.assemble ? P.rho : nullptr;
    d.solid = P.assemble ? P.solid : nullptr;
    BState &st = hst_[s];
    std::memset(&st, 0, sizeof(st));
    st.phase = BP_INIT;
    st.setup = P.need_setup ? 1 : 0;
    st.status = ST_RUNNING;
    st.tol = prm.tol;
    st.inner_tol = prm.inner_tol;
    st.max_sweeps = prm.max_sweeps;
    st.maxit = prm.max_iter;
    st.inner_maxit = prm.inner_max_iter;
    st.mixed = kMixed ? 1 : 0;
    st.f.done = 1;
    PBG_CUDA(cudaMemcpyAsync(dprob_.p + s, &d, sizeof(d), cudaMemcpyHostToDevice, stream));
    PBG_CUDA(cudaMemcpyAsync(dst_.p + s, &st, sizeof(st), cudaMemcpyHostToDevice, stream));
    if (P.need_setup) setup_pending_ = true;
    P.need_setup = false;
    P.slot = s;
    slot_pid_[s] = id;
    ++active_;
    tiles_dirty_ = true;
    return s;
  }

  // First level (>= 1, not the coarsest) with at most tail_cells cells:
  // its K-cycle and everything below runs in one CTA; kBMaxLev if none.
  int tail_level(const Prob &P) const {
    if (shape_.tail_cells <= 0) return kBMaxLev;
    for (int l = 1; l < P.nlev - 1; ++l)
      if ((long long)P.dims[l][0] * P.dims[l][1] * P.dims[l][2] <= shape_.tail_cells) return l;
    return kBMaxLev;
  }

  // ------------------------------------------------------------ tiles
  void rebuild_tiles() {
    std::vector<BTile> tiles;
    std::vector<int> lbeg(kBMaxLev + 1, 0), tbeg((size_t)kBMaxLev * S_, 0), tcnt((size_t)kBMaxLev * S_, 0);
    dmax_ = 0;
    int dtile = 0;
    unsigned dense_mask = 0, tail_mask = 0;
    for (int s = 0; s < S_; ++s) {
      if (slot_pid_[s] < 0) continue;
      const Prob &P = get(slot_pid_[s]);
      const int tl = tail_level(P);
      dmax_ = std::max(dmax_, P.nlev);
      dtile = std::max(dtile, std::min(P.nlev - 1, tl));
      if (tl < kBMaxLev) tail_mask |= 1u << tl;
      else dense_mask |= 1u << (P.nlev - 1);
    }
    sig_ = (unsigned long long)dtile | ((unsigned long long)dense_mask << 8) |
           ((unsigned long long)tail_mask << 24) | ((unsigned long long)dmax_ << 40);
    const uint32_t tc = (uint32_t)shape_.tile_cells;
    for (int l = 0; l < kBMaxLev; ++l) {
      lbeg[l] = (int)tiles.size();
      for (int s = 0; s < S_; ++s) {
        if (slot_pid_[s] < 0) continue;
        const Prob &P = get(slot_pid_[s]);
        if (P.nlev <= l) continue;
        const uint32_t n = (uint32_t)level_cells(P, l);
        tbeg[(size_t)l * S_ + s] = (int)tiles.size();
        int k = 0;
        for (uint32_t p0 = 0; p0 < n; p0 += tc, ++k) tiles.push_back({s, p0, std::min(tc, n - p0)});
        tcnt[(size_t)l * S_ + s] = k;
      }
    }
    lbeg[kBMaxLev] = (int)tiles.size();
    // small levels launch only as many CTAs as they have tiles (rounded up
    // to a power of two so that the graphs stay few); the grid-stride tile
    // loops are correct for any grid
    gcode_ = 0;
    for (int l = 0; l < kBMaxLev; ++l) {
      const int nt = std::max(1, lbeg[l + 1] - lbeg[l]);
      int g = 1, lg = 0;
      while (g < nt && g < shape_.grid) { g <<= 1; ++lg; }
      lgrid_[l] = std::min(g, shape_.grid);
      gcode_ |= (unsigned long long)lg << (5 * l);
    }
    const size_t nt = std::max<size_t>(tiles.size(), 1);
    if (nt > tile_cap_) {
      PBG_CUDA(cudaStreamSynchronize(stream));
      drop_graphs();  // kernel arguments point at the old arrays
      tile_cap_ = nt + nt / 2;
      dtiles_.alloc(tile_cap_);
      dpart_.alloc(tile_cap_ * 4);
    }
    const size_t bytes = sizeof(BTile) * tiles.size() + sizeof(int) * (lbeg.size() + 2 * tbeg.size());
    PBG_CUDA(cudaStreamSynchronize(stream));  // the staging buffer may feed an earlier copy
    if (bytes > htile_cap_) {
      if (htile_) cudaFreeHost(htile_);
      htile_ = nullptr;
      htile_cap_ = bytes + bytes / 2;
      PBG_CUDA(cudaMallocHost((void **)&htile_, htile_cap_));
    }
    char *h = htile_;
    std::memcpy(h, tiles.data(), sizeof(BTile) * tiles.size());
    PBG_CUDA(cudaMemcpyAsync(dtiles_.p, h, sizeof(BTile) * tiles.size(), cudaMemcpyHostToDevice, stream));
    h += sizeof(BTile) * tiles.size();
    std::memcpy(h, lbeg.data(), sizeof(int) * lbeg.size());
    PBG_CUDA(cudaMemcpyAsync(dlbeg_.p, h, sizeof(int) * lbeg.size(), cudaMemcpyHostToDevice, stream));
    h += sizeof(int) * lbeg.size();
    std::memcpy(h, tbeg.data(), sizeof(int) * tbeg.size());
    PBG_CUDA(cudaMemcpyAsync(dtbeg_.p, h, sizeof(int) * tbeg.size(), cudaMemcpyHostToDevice, stream));
    h += sizeof(int) * tbeg.size();
    std::memcpy(h, tcnt.data(), sizeof(int) * tcnt.size());
    PBG_CUDA(cudaMemcpyAsync(dtcnt_.p, h, sizeof(int) * tcnt.size(), cudaMemcpyHostToDevice, stream));
    tiles_dirty_ = false;
  }

  BCtx<T> ctx() const {
    BCtx<T> C;
    C.prob = dprob_.p;
    C.st = dst_.p;
    C.tiles = dtiles_.p;
    C.lbeg = dlbeg_.p;
    C.tbeg = dtbeg_.p;
    C.tcnt = dtcnt_.p;
    C.part = dpart_.p;
    C.cnt = dcnt_.p;
    C.S = S_;
    C.kc_max = shape_.kc_max;
    C.omega = (T)0.8;
    return C;
  }

  // ------------------------------------------------------------ launches
  int slot_grid() const { return std::min(S_, shape_.grid); }

  void setup_launches(int D) {
    const BCtx<T> C = ctx();
    const int G = shape_.grid, NT = shape_.threads;
    kb_assemble<T><<<G, NT, 0, stream>>>(C);
    for (int l = 1; l < D; ++l) kb_galerkin<T><<<G, NT, 0, stream>>>(C, l);
    for (int l = 0; l < D; ++l) kb_finish<T><<<G, NT, 0, stream>>>(C, l);
    kb_dense_inverse<T><<<slot_grid(), 256, 0, stream>>>(C, 1e-10);
    PBG_CUDA(cudaGetLastError());
    count(2 * D + 1);
  }

  // Launch sequence of one preconditioner application on level l (tile
  // kernels), with the dense solves and CTA-local tails of level l+1 and
  // the tile K-cycle of level l+1 where some slot needs them; counts the
  // launches.
  void seq_precond(const BCtx<T> &C, int l, int kc, size_t &n) {
    const int G = lgrid_[l], GH = lgrid_[l + 1 < kBMaxLev ? l + 1 : l], NT = shape_.threads;
    const int dtile = (int)(sig_ & 0xff);
    const unsigned dense_mask = (unsigned)((sig_ >> 8) & 0xffff), tail_mask = (unsigned)((sig_ >> 24) & 0xffff);
    kb_jac2<T><<<G, NT, 0, stream>>>(C, l, kc); ++n;
    if (kBPad<T> && l == 0) { kb_resid0<T><<<G, NT, 0, stream>>>(C); ++n; }
    kb_restrict<T><<<GH, NT, 0, stream>>>(C, l, kc); ++n;
    if (dense_mask & (1u << (l + 1))) { kb_dense<T><<<slot_grid(), NT, 0, stream>>>(C, l + 1); ++n; }
    if (tail_mask & (1u << (l + 1))) { kb_tail<T><<<slot_grid(), NT, 0, stream>>>(C, l + 1); ++n; }
    if (l + 1 < dtile) seq_kcycle(C, l + 1, n);
    kb_prolong_jac<T><<<G, NT, 0, stream>>>(C, l, kc); ++n;
    kb_jac<T><<<G, NT, 0, stream>>>(C, l, kc); ++n;
  }

  void seq_kcycle(const BCtx<T> &C, int l, size_t &n) {
    const int G = lgrid_[l], NT = shape_.threads;
    seq_precond(C, l, 0, n);
    if (l <= shape_.kc_max) {
      kb_kc_q1<T><<<G, NT, 0, stream>>>(C, l); ++n;
      seq_precond(C, l, 1, n);
      kb_kc_q2<T><<<G, NT, 0, stream>>>(C, l); ++n;
    }
  }

  Graph &graph(unsigned long long sig) {
    const std::pair<unsigned long long, unsigned long long> key(sig, gcode_);
    auto it = graphs_.find(key);
    if (it != graphs_.end()) return it->second;
    const BCtx<T> C = ctx();
    const int G = lgrid_[0], NT = shape_.threads;
    cudaGraph_t g = nullptr;
    size_t n = 0;
    PBG_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    try {
      kb_outer_corr<T><<<G, NT, 0, stream>>>(C); ++n;
      kb_outer_resid<T><<<G, NT, 0, stream>>>(C); ++n;
      seq_precond(C, 0, 0, n);
      kb_fcg_pq<T><<<G, NT, 0, stream>>>(C); ++n;
      kb_fcg_xr<T><<<G, NT, 0, stream>>>(C); ++n;
      PBG_CUDA(cudaGetLastError());
    } catch (...) {
      cudaStreamEndCapture(stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    PBG_CUDA(cudaStreamEndCapture(stream, &g));
    Graph gr;
    gr.nodes = n;
    cudaError_t e = cudaGraphInstantiate(&gr.exec, g, 0);
    cudaGraphDestroy(g);
    PBG_CUDA(e);
    return graphs_[key] = gr;
  }

  void count(unsigned long long n) {
    launches_ += n;
    __atomic_add_fetch(&g_launch_count, n, __ATOMIC_RELAXED);
  }

  void drop_graphs() {
    for (auto &kv : graphs_)
      if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    graphs_.clear();
  }

  void step(int iterations) override {
    if (active_ == 0) return;
    if (tiles_dirty_) rebuild_tiles();
    if (setup_pending_) {
      setup_launches(dmax_);
      setup_pending_ = false;
    }
    Graph &g = graph(sig_);
    for (int k = 0; k < iterations; ++k) PBG_CUDA(cudaGraphLaunch(g.exec, stream));
    count((unsigned long long)iterations * g.nodes);
  }

  std::vector<std::pair<int, BatchOutcome>> collect() override {
    std::vector<std::pair<int, BatchOutcome>> out;
    if (active_ == 0) return out;
    PBG_CUDA(cudaMemcpy2DAsync(hphase_, sizeof(int), &dst_.p[0].phase, sizeof(BState), sizeof(int), S_,
                               cudaMemcpyDeviceToHost, stream));
    PBG_CUDA(cudaStreamSynchronize(stream));
    std::vector<int> done;
    for (int s = 0; s < S_; ++s)
      if (slot_pid_[s] >= 0 && hphase_[s] == BP_DONE) {
        PBG_CUDA(cudaMemcpyAsync(hout_ + s, dst_.p + s, sizeof(BState), cudaMemcpyDeviceToHost, stream));
        done.push_back(s);
      }
    if (done.empty()) return out;
    PBG_CUDA(cudaStreamSynchronize(stream));
    for (int s : done) {
      const BState &st = hout_[s];
      BatchOutcome o;
      o.status = st.status;
      o.converged = st.converged;
      o.iterations = st.iters;
      o.sweeps = st.sweeps;
      o.relres = st.rel;
      o.relres0 = st.rel0;
      const int id = slot_pid_[s];
      out.push_back({id, o});
      get(id).slot = -1;
      slot_pid_[s] = -1;
      --active_;
      tiles_dirty_ = true;
    }
    return out;
  }

  void set_shape(const BatchShape &s) override {
    check_shape(s);
    if (active_) throw std::runtime_error("batch: shape change while problems are attached");
    PBG_CUDA(cudaStreamSynchronize(stream));
    drop_graphs();
    shape_ = s;
    tiles_dirty_ = true;
  }
  BatchShape shape() const override { return shape_; }
  unsigned long long kernel_launches() const override { return launches_; }
};

std::unique_ptr<BatchEngineBase> make_batch_engine(int precision, int slots, const BatchShape &shape) {
  if (precision == 1) return std::make_unique<BatchEngine<float>>(slots, shape);
  return std::make_unique<BatchEngine<double>>(slots, shape);
}

}  // namespace pbg
