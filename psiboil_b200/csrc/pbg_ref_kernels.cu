// Reference-parity kernels: the reference's per-element arithmetic, in the
// reference's operation order, with explicit round-to-nearest intrinsics so
// that the compiler cannot contract a multiply and an add into one FMA.
// Only the order of the global sums differs from the reference (a tree
// instead of a sequential i,j,k sum).
#include <cstring>

#include "pbg_ref_kernels.cuh"

namespace pbg {

// ---------------------------------------------------------------------------
// Stencil helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ double ld0(const double *x, long long p, bool ok) {
  return ok ? x[p] : 0.0;
}

// y = A x at cell p, order of Scalar::operator=(const A_x&)
// (Src/Field/Scalar/scalar_operators.cpp:49-72):
//   y = c x;  y -= (w xw + e xe);  y -= (s xs + n xn);  y -= (b xb + t xt)
template <typename XF>
__device__ __forceinline__ double ref_ax(const MatView<double> &A, long long p, Pos q, XF xv) {
  Nb<double> a = coeffs(A, p, q);
  double xw, xe, xs, xn, xb, xt;
  if (!A.per) {  // uniform: the plain neighbour form unless the matrix is periodic
    const long long SI = (long long)A.ny * A.nz, SJ = A.nz;
    xw = q.i > 0 ? xv(p - SI) : 0.0; xe = q.i < A.nx - 1 ? xv(p + SI) : 0.0;
    xs = q.j > 0 ? xv(p - SJ) : 0.0; xn = q.j < A.ny - 1 ? xv(p + SJ) : 0.0;
    xb = q.k > 0 ? xv(p - 1) : 0.0; xt = q.k < A.nz - 1 ? xv(p + 1) : 0.0;
  } else {
    const NbIdx m = nb_index(A, p, q);
    xw = m.w >= 0 ? xv(m.w) : 0.0; xe = m.e >= 0 ? xv(m.e) : 0.0;
    xs = m.s >= 0 ? xv(m.s) : 0.0; xn = m.n >= 0 ? xv(m.n) : 0.0;
    xb = m.b >= 0 ? xv(m.b) : 0.0; xt = m.t >= 0 ? xv(m.t) : 0.0;
  }
  double v = __dmul_rn(A.c[p], xv(p));
  v = __dsub_rn(v, __dadd_rn(__dmul_rn(a.w, xw), __dmul_rn(a.e, xe)));
  v = __dsub_rn(v, __dadd_rn(__dmul_rn(a.s, xs), __dmul_rn(a.n, xn)));
  v = __dsub_rn(v, __dadd_rn(__dmul_rn(a.b, xb), __dmul_rn(a.t, xt)));
  return v;
}

// r = b - A x at cell p, order of Scalar::operator=(const y_m_A_x&)
// (scalar_operators.cpp:22-46):
//   r = b - c x;  r += w xw + e xe;  r += s xs + n xn;  r += b xb + t xt
__device__ __forceinline__ double ref_bmax(const MatView<double> &A, long long p, Pos q,
                                           const double *x, double bp) {
  Nb<double> a = coeffs(A, p, q);
  double xw, xe, xs, xn, xb, xt;
  if (!A.per) {
    const long long SI = (long long)A.ny * A.nz, SJ = A.nz;
    xw = ld0(x, p - SI, q.i > 0); xe = ld0(x, p + SI, q.i < A.nx - 1);
    xs = ld0(x, p - SJ, q.j > 0); xn = ld0(x, p + SJ, q.j < A.ny - 1);
    xb = ld0(x, p - 1, q.k > 0); xt = ld0(x, p + 1, q.k < A.nz - 1);
  } else {
    const NbIdx m = nb_index(A, p, q);
    xw = ld0(x, m.w, m.w >= 0); xe = ld0(x, m.e, m.e >= 0);
    xs = ld0(x, m.s, m.s >= 0); xn = ld0(x, m.n, m.n >= 0);
    xb = ld0(x, m.b, m.b >= 0); xt = ld0(x, m.t, m.t >= 0);
  }
  double v = __dsub_rn(bp, __dmul_rn(A.c[p], x[p]));
  v = __dadd_rn(v, __dadd_rn(__dmul_rn(a.w, xw), __dmul_rn(a.e, xe)));
  v = __dadd_rn(v, __dadd_rn(__dmul_rn(a.s, xs), __dmul_rn(a.n, xn)));
  v = __dadd_rn(v, __dadd_rn(__dmul_rn(a.b, xb), __dmul_rn(a.t, xt)));
  return v;
}

// element of Scalar::dot_voldiv_avg: x*y/dV/dV (scalar.h:317-326)
__device__ __forceinline__ double voldiv(double x, double y, double dV) {
  return __ddiv_rn(__ddiv_rn(__dmul_rn(x, y), dV), dV);
}

// res = sqrt(d/N/N)/scale (cg.cpp:68 and :115)
__device__ __forceinline__ double res_of(double d, const KrylovState *st) {
  return __ddiv_rn(__dsqrt_rn(__ddiv_rn(__ddiv_rn(d, st->ncell), st->ncell)), st->scale);
}

// ---------------------------------------------------------------------------
// Plain operators (parity tests and building blocks)
// ---------------------------------------------------------------------------
__global__ void k_spmv_ref(MatView<double> A, const double *__restrict__ x, double *__restrict__ y) {
  const long long N = A.ncell();
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    Pos q = pos_of(p, A.ny, A.nz);
    y[p] = ref_ax(A, p, q, [&](long long r) { return x[r]; });
  }
}

__global__ void k_resid_ref(MatView<double> A, const double *__restrict__ x,
                            const double *__restrict__ b, double *__restrict__ r) {
  const long long N = A.ncell();
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    Pos q = pos_of(p, A.ny, A.nz);
    r[p] = ref_bmax(A, p, q, x, b[p]);
  }
}

// out[0] = sum x*y, out[1] = sum x*y/dV/dV (deterministic tree order)
__global__ void k_dot2(long long N, const double *__restrict__ x, const double *__restrict__ y,
                       double dV, double *part, unsigned *count, double *out) {
  double v[2] = {0.0, 0.0};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    v[0] += __dmul_rn(x[p], y[p]);
    v[1] += voldiv(x[p], y[p], dV);
  }
  double o[2];
  if (grid_reduce<2>(v, part, count, o)) { out[0] = o[0]; out[1] = o[1]; }
}

// Sequential sum of n terms: out[0] = (..((0 + a0) + a1) + ..) + a_{n-1}, the
// reference's `for_ijk sum += ...` order, and out[1] the same for b (when
// given). One thread per term, exact-order reduction.
__global__ void k_seq_sum(long long N, const double *__restrict__ a, const double *__restrict__ b,
                          double *seq, unsigned *count, double *out) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double v[2] = {p < N ? a[p] : 0.0, (p < N && b) ? b[p] : 0.0};
  double o[2];
  if (grid_reduce<2>(v, nullptr, count, o, seq, N)) { out[0] = o[0]; out[1] = o[1]; }
}

void exact_scratch_init(double *base, long long ncell, cudaStream_t s) {
  const long long ch = (ncell + kExactChunkThreads - 1) / kExactChunkThreads + 1;
  const long long gr = (ch + kExactGroup - 1) / kExactGroup + 1;
  char *q = reinterpret_cast<char *>(base) + kExactHdrBytes + sizeof(double) * (size_t)kExactVals * ncell;
  ExactHdr h;
  std::memset(&h, 0, sizeof(h));
  h.wrec = reinterpret_cast<ExactRec *>(q); q += sizeof(ExactRec) * kExactVals * (size_t)ch * kExactWarps;
  h.crec = reinterpret_cast<ExactRec *>(q); q += sizeof(ExactRec) * kExactVals * (size_t)ch;
  h.grec = reinterpret_cast<ExactRec *>(q); q += sizeof(ExactRec) * kExactVals * (size_t)gr;
  h.agg = reinterpret_cast<double *>(q); q += sizeof(double) * kExactVals * (size_t)ch;
  h.incl = reinterpret_cast<double *>(q); q += sizeof(double) * kExactVals * (size_t)ch;
  h.flag = reinterpret_cast<unsigned *>(q); q += sizeof(unsigned) * (size_t)ch;
  h.gcount = reinterpret_cast<unsigned *>(q); q += sizeof(unsigned) * (size_t)gr;
  h.cap_chunks = ch;
  h.cap_groups = gr;
  h.gen = 1;
  if ((size_t)(q - reinterpret_cast<char *>(base)) > exact_scratch_doubles(ncell) * sizeof(double))
    throw CudaError("exact-sum scratch layout exceeds its allocation");
  PBG_CUDA(cudaMemsetAsync(h.flag, 0, sizeof(unsigned) * (size_t)(ch + gr), s));
  PBG_CUDA(cudaMemcpyAsync(base, &h, sizeof(h), cudaMemcpyHostToDevice, s));
  PBG_CUDA(cudaStreamSynchronize(s));
}

// ---------------------------------------------------------------------------
// CG with the diagonal preconditioner, CG::solve (cg.cpp:10-182),
// Diagonal::form/solve (preconditioner_form.cpp:4-13,
// preconditioner_solve.cpp:4-11): Mc = 1/c, z = r*Mc.
//
// Per iteration two kernels:
//   k_cg_pq : p = z + beta p (p = z at i = 0), q = A p, pq = p.q, alfa
//   k_cg_xr : x += alfa p, r -= alfa q, res, convergence, next rho = r.z
// p is double-buffered (read p_old, write p_new) so that each thread can
// form p at its six neighbours from z and p_old without a grid barrier.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double mc_of(const double *c, long long p) { return __ddiv_rn(1.0, c[p]); }

// Mc = 1 / c once per solve (Diagonal::form, preconditioner_form.cpp:4-13);
// the kernels below read it instead of dividing at every use
__global__ void k_recip(long long N, const double *__restrict__ c, double *__restrict__ mc) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x)
    mc[p] = mc_of(c, p);
}

__device__ void stale_init_dev(KrylovState *st, double res0) {
  int n = st->stalecount > kStaleMax ? kStaleMax : st->stalecount;
  for (int q = 0; q < n; ++q) st->stale[q] = 1.0e24;  // boil::unreal
  if (n > 0) st->stale[n - 1] = res0;
}

// true when stale (cg.cpp:138-160); otherwise rotates the window
__device__ bool stale_step_dev(KrylovState *st, double res) {
  int n = st->stalecount > kStaleMax ? kStaleMax : st->stalecount;
  if (n <= 0) return false;
  bool stale = true;
  for (int q = 0; q < n; ++q)
    if (res < st->stale[q]) { stale = false; break; }
  if (stale) return true;
  for (int q = 0; q < n - 1; ++q) st->stale[q] = st->stale[q + 1];
  st->stale[n - 1] = res;
  return false;
}

__global__ void k_cg_init(MatView<double> A, const double *__restrict__ x,
                          const double *__restrict__ b, double *__restrict__ r,
                          KrylovState *st, double *part, unsigned *count, const double *__restrict__ mc) {
  const long long N = A.ncell();
  const double dV = st->dV;
  double v[2] = {0.0, 0.0};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    Pos q = pos_of(p, A.ny, A.nz);
    double rv = ref_bmax(A, p, q, x, b[p]);
    r[p] = rv;
    v[0] += voldiv(rv, rv, dV);
    v[1] += __dmul_rn(rv, __dmul_rn(rv, mc[p]));
  }
  double o[2];
  if (grid_reduce<2>(v, part, count, o, st->seq, N)) {
    double res = res_of(o[0], st);
    st->res0 = res;
    st->res = res;
    st->rho = o[1];
    st->iter = 0;
    st->iterations = 0;
    st->converged = 0;
    st->pending_x = 0;
    stale_init_dev(st, res);
    if (res < st->res_tol) {  // cg.cpp:83
      st->done = 1;
      st->converged = 1;
      st->status = ST_INITIAL;
    } else if (st->maxit <= 0) {
      st->done = 1;
      st->status = ST_MAXITER;
    } else {
      st->done = 0;
      st->status = ST_RUNNING;
    }
  }
}

__global__ void __launch_bounds__(kThreads, 3) k_cg_pq(MatView<double> A, const double *__restrict__ r, double *pA, double *pB,
                        double *__restrict__ qv, KrylovState *st, double *part, unsigned *count,
                        const double *__restrict__ zarr, const double *__restrict__ mc) {
  if (st->done) return;
  const int it = st->iter;
  const double *pold = (it & 1) ? pB : pA;
  double *pnew = (it & 1) ? pA : pB;
  const double beta = it == 0 ? 0.0 : __ddiv_rn(st->rho, st->rho_old);
  const long long N = A.ncell();
  // z = r * Mc (diagonal) or the preconditioner's output zarr
  auto pv = [&](long long s) {
    double z = zarr ? zarr[s] : __dmul_rn(r[s], mc[s]);
    return it == 0 ? z : __dadd_rn(z, __dmul_rn(beta, pold[s]));
  };
  double v[1] = {0.0};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    Pos q = pos_of(p, A.ny, A.nz);
    double pp = pv(p);
    double qq = ref_ax(A, p, q, pv);
    pnew[p] = pp;
    qv[p] = qq;
    v[0] += __dmul_rn(pp, qq);
  }
  double o[1];
  if (grid_reduce<1>(v, part, count, o, st->seq, N)) {
    st->beta = beta;
    st->pq = o[0];
    st->alfa = __ddiv_rn(st->rho, o[0]);
  }
}

// Seq = false: tree-order sums only (the split path), without the
// exact-order reduction's code and shared memory
template <bool Seq>
__global__ void __launch_bounds__(kThreads, 3) k_cg_xr(long long N, const double *__restrict__ mc, double *__restrict__ x,
                        double *__restrict__ r, const double *pA, const double *pB,
                        const double *__restrict__ qv, KrylovState *st, double *hist,
                        double *part, unsigned *count, int ic) {
  if (st->done) return;
  const int it = st->iter;
  const double *p_ = (it & 1) ? pA : pB;  // the buffer k_cg_pq wrote
  const double alfa = st->alfa, dV = st->dV;
  double v[2] = {0.0, 0.0};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    x[p] = __dadd_rn(x[p], __dmul_rn(alfa, p_[p]));
    double rv = __dsub_rn(r[p], __dmul_rn(alfa, qv[p]));
    r[p] = rv;
    v[0] += voldiv(rv, rv, dV);
    v[1] += __dmul_rn(rv, __dmul_rn(rv, mc[p]));
  }
  double o[2];
  if (grid_reduce<2>(v, part, count, o, Seq ? st->seq : nullptr, N)) {
    double res = res_of(o[0], st);
    st->res = res;
    if (hist && it < st->hist_cap) hist[it] = res;
    const bool minok = it >= st->mini - 1;
    if ((res < st->res_tol && minok) || (res < st->res0 * st->res_rat && minok)) {
      st->done = 1; st->converged = 1; st->status = ST_CONVERGED; st->iterations = it + 1;
    } else if (stale_step_dev(st, res)) {
      st->done = 1; st->status = ST_STALE; st->iterations = it + 1;
    } else if (!(res == res)) {
      st->done = 1; st->status = ST_NAN; st->iterations = it + 1;
    } else {
      if (!ic) {  // with an IC preconditioner k_cg_rho forms rho after the solve
        st->rho_old = st->rho;
        st->rho = o[1];
      }
      st->iter = it + 1;
      st->iterations = it + 1;
      if (it + 1 >= st->maxit) { st->done = 1; st->status = ST_MAXITER; }
    }
  }
}

// ---------------------------------------------------------------------------
// CG with the diagonal preconditioner and tree-order sums, split for
// 16-byte access (nz even): k_cg_p forms p = z + beta p_old in place
// (z = r Mc), k_cg_q forms q = A p with the dot p.q, and k_cg_xr follows as
// in the fused path (given the one p buffer twice). Every element gets the
// arithmetic of k_cg_pq / ref_ax in the same order, so the iterates equal
// the fused path's up to the order of the global sums.
// ---------------------------------------------------------------------------
__global__ void k_cg_p(long long N, const double *__restrict__ r, const double *__restrict__ mc,
                       double *__restrict__ p, KrylovState *st) {
  if (st->done) return;
  const int it = st->iter;
  const double beta = it == 0 ? 0.0 : __ddiv_rn(st->rho, st->rho_old);
  const long long NP = N / 2;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < NP;
       g += (long long)gridDim.x * blockDim.x) {
    const double2 rv = reinterpret_cast<const double2 *>(r)[g];
    const double2 mv = reinterpret_cast<const double2 *>(mc)[g];
    double2 z = make_double2(__dmul_rn(rv.x, mv.x), __dmul_rn(rv.y, mv.y));
    if (it > 0) {
      const double2 po = reinterpret_cast<const double2 *>(p)[g];
      z.x = __dadd_rn(z.x, __dmul_rn(beta, po.x));
      z.y = __dadd_rn(z.y, __dmul_rn(beta, po.y));
    }
    reinterpret_cast<double2 *>(p)[g] = z;
  }
  if ((N & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
    const long long e = N - 1;
    double z = __dmul_rn(r[e], mc[e]);
    if (it > 0) z = __dadd_rn(z, __dmul_rn(beta, p[e]));
    p[e] = z;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) st->beta = beta;
}

// q = A p for two cells of one k-row (nz even), in ref_ax's order
__global__ void __launch_bounds__(kThreads, 4) k_cg_q(MatView<double> A, Geo G, const double *__restrict__ p, double *__restrict__ qv,
                       KrylovState *st, double *part, unsigned *count) {
  if (st->done) return;
  const long long SI = (long long)A.ny * A.nz, SJ = A.nz;
  const long long NP = A.ncell() / 2;
  double v[1] = {0.0};
  auto ld2 = [&](const double *a, long long e) { return reinterpret_cast<const double2 *>(a + e)[0]; };
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < NP;
       g += (long long)gridDim.x * blockDim.x) {
    const long long e = 2 * g;
    const Pos q = G.pos((uint32_t)e);
    const double2 x = ld2(p, e), c = ld2(A.c, e), w = ld2(A.w, e), s = ld2(A.s, e), b = ld2(A.b, e);
    const double2 z2 = make_double2(0.0, 0.0);
    const double2 xw = q.i > 0 ? ld2(p, e - SI) : z2, xe = q.i < A.nx - 1 ? ld2(p, e + SI) : z2;
    const double2 xs = q.j > 0 ? ld2(p, e - SJ) : z2, xn = q.j < A.ny - 1 ? ld2(p, e + SJ) : z2;
    const double xb0 = q.k > 0 ? p[e - 1] : 0.0, xt1 = q.k + 2 < A.nz ? p[e + 2] : 0.0;
    double2 ec, nc, tc;
    if (A.e) {
      ec = ld2(A.e, e); nc = ld2(A.n, e); tc = ld2(A.t, e);
    } else {
      ec = q.i < A.nx - 1 ? ld2(A.w, e + SI) : z2;
      nc = q.j < A.ny - 1 ? ld2(A.s, e + SJ) : z2;
      tc = make_double2(b.y, q.k + 2 < A.nz ? A.b[e + 2] : 0.0);
    }
    // lane 0: k, lane 1: k + 1 (its b neighbour is lane 0, lane 0's t neighbour is lane 1)
    double y0 = __dmul_rn(c.x, x.x);
    y0 = __dsub_rn(y0, __dadd_rn(__dmul_rn(w.x, xw.x), __dmul_rn(ec.x, xe.x)));
    y0 = __dsub_rn(y0, __dadd_rn(__dmul_rn(s.x, xs.x), __dmul_rn(nc.x, xn.x)));
    y0 = __dsub_rn(y0, __dadd_rn(__dmul_rn(b.x, xb0), __dmul_rn(tc.x, x.y)));
    double y1 = __dmul_rn(c.y, x.y);
    y1 = __dsub_rn(y1, __dadd_rn(__dmul_rn(w.y, xw.y), __dmul_rn(ec.y, xe.y)));
    y1 = __dsub_rn(y1, __dadd_rn(__dmul_rn(s.y, xs.y), __dmul_rn(nc.y, xn.y)));
    y1 = __dsub_rn(y1, __dadd_rn(__dmul_rn(b.y, x.x), __dmul_rn(tc.y, xt1)));
    reinterpret_cast<double2 *>(qv + e)[0] = make_double2(y0, y1);
    v[0] += __dmul_rn(x.x, y0);
    v[0] += __dmul_rn(x.y, y1);
  }
  double o[1];
  if (grid_reduce<1>(v, part, count, o)) {
    st->pq = o[0];
    st->alfa = __ddiv_rn(st->rho, o[0]);
  }
}

// ---------------------------------------------------------------------------
// Incomplete Cholesky preconditioners (Prec::ic0/ic2/ic3):
// IncompleteCholesky0/2/3::form (preconditioner_form.cpp:16-144) and ::solve
// (preconditioner_solve.cpp:14-110). The reference runs factor and sweeps in
// lexicographic i, j, k order. Every value a cell reads was written by a cell
// with a smaller index h = a i + b j + k (a = b = 2 for IC0/IC2; a = 5, b = 2
// for IC3, whose Mnw term reaches (i-1, j+2, k)), so one launch per
// hyperplane h processes independent cells, each with the reference's
// arithmetic in the reference's order (__dmul_rn/__dsub_rn/__ddiv_rn/
// __dsqrt_rn, no contraction): the results are the reference's bit for bit.
// The arrays are compact and start at zero; the factor's writes outside the
// domain (the reference's halo, which no interior cell reads) are skipped,
// and so are the sweeps' terms with a neighbour outside (the reference
// multiplies them by its zero halo).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double msub(double s, double a, double b) { return __dsub_rn(s, __dmul_rn(a, b)); }

// cell (i, j, k) of hyperplane h for thread index t over the (i, j) plane
__device__ __forceinline__ bool ic_cell(const MatView<double> &A, int h, int wa, int wb, long long t, int &i,
                                        int &j, int &k) {
  i = (int)(t / A.ny);
  j = (int)(t - (long long)i * A.ny);
  k = h - wa * i - wb * j;
  return k >= 0 && k < A.nz;
}

__global__ void k_ic_form(MatView<double> A, IcFactor M, int h) {
  const long long SI = (long long)A.ny * A.nz, SJ = A.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)A.nx * A.ny;
       t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    if (!ic_cell(A, h, M.wa, M.wb, t, i, j, k)) continue;
    const long long p = ((long long)i * A.ny + j) * A.nz + k;
    const bool xp = i + 1 < A.nx, yp = j + 1 < A.ny, zp = k + 1 < A.nz, zm = k > 0, ym = j > 0;
    double sum = A.c[p];
    sum = msub(sum, M.w[p], M.w[p]);
    if (M.kind >= 2) sum = msub(sum, M.tw[p], M.tw[p]);
    if (M.kind == 3) sum = msub(sum, M.nw[p], M.nw[p]);
    sum = msub(sum, M.s[p], M.s[p]);
    if (M.kind >= 2) sum = msub(sum, M.ts[p], M.ts[p]);
    sum = msub(sum, M.b[p], M.b[p]);
    sum = __dsqrt_rn(sum);
    M.c[p] = sum;
    if (M.kind == 1) {
      if (xp) M.w[p + SI] = __ddiv_rn(-A.w[p + SI], sum);
      if (yp) M.s[p + SJ] = __ddiv_rn(-A.s[p + SJ], sum);
      if (zp) M.b[p + 1] = __ddiv_rn(-A.b[p + 1], sum);
      continue;
    }
    if (xp) M.w[p + SI] = __ddiv_rn(-A.w[p + SI], sum);
    if (xp && zm) M.tw[p + SI - 1] = __ddiv_rn(__dmul_rn(-M.w[p + SI - 1], M.b[p]), sum);
    if (M.kind == 3 && xp && ym)
      M.nw[p + SI - SJ] = __ddiv_rn(__dsub_rn(__dmul_rn(-M.w[p + SI - SJ], M.s[p]),
                                              __dmul_rn(M.tw[p + SI - SJ], M.ts[p])), sum);
    if (yp) {
      if (M.kind == 2) M.s[p + SJ] = __ddiv_rn(-A.s[p + SJ], sum);
      else M.s[p + SJ] = __ddiv_rn(msub(msub(-A.s[p + SJ], M.w[p + SJ], M.nw[p]), M.nw[p + SJ], M.s[p]), sum);
    }
    if (yp && zm) {
      if (M.kind == 2) M.ts[p + SJ - 1] = __ddiv_rn(__dmul_rn(-M.s[p + SJ - 1], M.b[p]), sum);
      else
        M.ts[p + SJ - 1] = __ddiv_rn(__dsub_rn(__dmul_rn(-M.s[p + SJ - 1], M.b[p]),
                                               __dmul_rn(M.tw[p + SJ - 1], M.nw[p])), sum);
    }
    if (zp) M.b[p + 1] = __ddiv_rn(msub(msub(-A.b[p + 1], M.w[p + 1], M.tw[p]), M.s[p + 1], M.ts[p]), sum);
  }
}

// forward sweep on hyperplane h: z = (r - lower terms) / Mc
__global__ void k_ic_fwd(MatView<double> A, IcFactor M, int h, const double *__restrict__ r, double *z,
                         const KrylovState *st) {
  if (st->done) return;
  const long long SI = (long long)A.ny * A.nz, SJ = A.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)A.nx * A.ny;
       t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    if (!ic_cell(A, h, M.wa, M.wb, t, i, j, k)) continue;
    const long long p = ((long long)i * A.ny + j) * A.nz + k;
    double sum = r[p];
    if (i > 0) sum = msub(sum, M.w[p], z[p - SI]);
    if (M.kind >= 2 && i > 0 && k + 1 < A.nz) sum = msub(sum, M.tw[p], z[p - SI + 1]);
    if (M.kind == 3 && i > 0 && j + 1 < A.ny) sum = msub(sum, M.nw[p], z[p - SI + SJ]);
    if (j > 0) sum = msub(sum, M.s[p], z[p - SJ]);
    if (M.kind >= 2 && j > 0 && k + 1 < A.nz) sum = msub(sum, M.ts[p], z[p - SJ + 1]);
    if (k > 0) sum = msub(sum, M.b[p], z[p - 1]);
    z[p] = __ddiv_rn(sum, M.c[p]);
  }
}

// backward sweep on hyperplane h: z = (z - upper terms) / Mc
__global__ void k_ic_bwd(MatView<double> A, IcFactor M, int h, double *z, const KrylovState *st) {
  if (st->done) return;
  const long long SI = (long long)A.ny * A.nz, SJ = A.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)A.nx * A.ny;
       t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    if (!ic_cell(A, h, M.wa, M.wb, t, i, j, k)) continue;
    const long long p = ((long long)i * A.ny + j) * A.nz + k;
    const bool xp = i + 1 < A.nx, yp = j + 1 < A.ny, zp = k + 1 < A.nz, zm = k > 0, ym = j > 0;
    double sum = z[p];
    if (xp) sum = msub(sum, M.w[p + SI], z[p + SI]);
    if (M.kind >= 2 && xp && zm) sum = msub(sum, M.tw[p + SI - 1], z[p + SI - 1]);
    if (M.kind == 3 && xp && ym) sum = msub(sum, M.nw[p + SI - SJ], z[p + SI - SJ]);
    if (yp) sum = msub(sum, M.s[p + SJ], z[p + SJ]);
    if (M.kind >= 2 && yp && zm) sum = msub(sum, M.ts[p + SJ - 1], z[p + SJ - 1]);
    if (zp) sum = msub(sum, M.b[p + 1], z[p + 1]);
    z[p] = __ddiv_rn(sum, M.c[p]);
  }
}

// rho = r.z (Scalar::dot, scalar.h:296-298) for the next CG step
__global__ void k_cg_rho(long long N, const double *__restrict__ r, const double *__restrict__ z,
                         KrylovState *st, double *part, unsigned *count) {
  if (st->done) return;
  double v[1] = {0.0};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x)
    v[0] += __dmul_rn(r[p], z[p]);
  double o[1];
  if (grid_reduce<1>(v, part, count, o, st->seq, N)) {
    st->rho_old = st->rho;
    st->rho = o[0];
  }
}


// ---------------------------------------------------------------------------
// BiCGStab, BiCGS::solve (bicgs.cpp:9-229). One iteration:
//   k_bi_rho   rho = r~.r; breakdown test; beta                     (:91-99)
//   k_bi_p     p = r (i=0) | p = r + beta p; p -= (beta omega) v; p^ = p Mc
//   k_bi_v     v = A p^; r~.v; alfa                                 (:124-133)
//   k_bi_s     s = r - alfa v; s.s; early exit test; s^ = s Mc      (:137-159)
//   k_bi_t     t = A s^; t.s, t.t; omega                           (:163-175)
//   k_bi_xr    x += alfa p^; x += omega s^; r = s - omega t; res; tests
// The early exit of :146-150 (x += alfa p^, break) is carried by
// pending_x, which k_bi_xr applies and clears. With an incomplete Cholesky
// preconditioner (diag == 0) the IC sweeps form p^ and s^ instead.
// ---------------------------------------------------------------------------
__global__ void k_bi_init(MatView<double> A, const double *__restrict__ x, const double *__restrict__ b,
                          double *__restrict__ r, double *__restrict__ rt, KrylovState *st,
                          double *part, unsigned *count) {
  const long long N = A.ncell();
  const double dV = st->dV;
  double v[1] = {0.0};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    Pos q = pos_of(p, A.ny, A.nz);
    double rv = ref_bmax(A, p, q, x, b[p]);
    r[p] = rv;
    rt[p] = rv;
    v[0] += voldiv(rv, rv, dV);
  }
  double o[1];
  if (grid_reduce<1>(v, part, count, o, st->seq, N)) {
    double res = res_of(o[0], st);
    st->res0 = res;
    st->res = res;
    st->iter = 0;
    st->iterations = 0;
    st->converged = 0;
    st->pending_x = 0;
    stale_init_dev(st, res);
    if (res < st->res_tol) {
      st->done = 1; st->converged = 1; st->status = ST_INITIAL;
    } else if (st->maxit <= 0) {
      st->done = 1; st->status = ST_MAXITER;
    } else {
      st->done = 0; st->status = ST_RUNNING;
    }
  }
}

__global__ void k_bi_rho(long long N, const double *__restrict__ rt, const double *__restrict__ r,
                         KrylovState *st, double *part, unsigned *count) {
  if (st->done) return;
  double v[1] = {0.0};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x)
    v[0] += __dmul_rn(rt[p], r[p]);
  double o[1];
  if (grid_reduce<1>(v, part, count, o, st->seq, N)) {
    const int it = st->iter;
    st->rho = o[0];
    if (__dsqrt_rn(fabs(o[0])) < st->res_tol) {
      st->done = 1; st->status = ST_BREAKDOWN; st->iterations = it + 1;
    } else if (it > 0) {
      st->beta = __dmul_rn(__ddiv_rn(o[0], st->rho_old), __ddiv_rn(st->alfa, st->omega));
    }
  }
}

__global__ void k_bi_p(long long N, const double *__restrict__ c, const double *__restrict__ r,
                       double *__restrict__ pv, const double *__restrict__ v, double *__restrict__ ph,
                       const KrylovState *st, int diag) {
  if (st->done) return;
  const int it = st->iter;
  const double beta = st->beta, bo = __dmul_rn(st->beta, st->omega);
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    double pp;
    if (it == 0) pp = r[p];
    else {
      pp = __dadd_rn(r[p], __dmul_rn(beta, pv[p]));
      pp = __dsub_rn(pp, __dmul_rn(bo, v[p]));
    }
    pv[p] = pp;
    if (diag) ph[p] = __dmul_rn(pp, c[p]);
  }
}

// y = A x and up to two dots with y: mode 0 -> rt.y (alfa), mode 1 -> y.s, y.y (omega)
__global__ void k_bi_spmv(MatView<double> A, const double *__restrict__ x, double *__restrict__ y,
                          const double *__restrict__ o1, int mode, KrylovState *st,
                          double *part, unsigned *count) {
  if (st->done) return;
  const long long N = A.ncell();
  double v[2] = {0.0, 0.0};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    Pos q = pos_of(p, A.ny, A.nz);
    double yv = ref_ax(A, p, q, [&](long long s) { return x[s]; });
    y[p] = yv;
    if (mode == 0) v[0] += __dmul_rn(o1[p], yv);
    else { v[0] += __dmul_rn(yv, o1[p]); v[1] += __dmul_rn(yv, yv); }
  }
  double o[2];
  if (grid_reduce<2>(v, part, count, o, st->seq, N)) {
    if (mode == 0) st->alfa = __ddiv_rn(st->rho, o[0]);
    else { st->aux0 = o[0]; st->aux1 = o[1]; st->omega = __ddiv_rn(o[0], o[1]); }
  }
}

__global__ void k_bi_s(long long N, const double *__restrict__ c, const double *__restrict__ r,
                       const double *__restrict__ v, double *__restrict__ s, double *__restrict__ sh,
                       KrylovState *st, double *part, unsigned *count, int diag) {
  if (st->done) return;
  const double alfa = st->alfa;
  double a[1] = {0.0};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    double sv = __dsub_rn(r[p], __dmul_rn(alfa, v[p]));
    s[p] = sv;
    if (diag) sh[p] = __dmul_rn(sv, c[p]);
    a[0] += __dmul_rn(sv, sv);
  }
  double o[1];
  if (grid_reduce<1>(a, part, count, o, st->seq, N)) {
    if (__dsqrt_rn(o[0]) < st->res_tol) {
      st->pending_x = 1;  // x += alfa p^, then stop (bicgs.cpp:146-150)
      st->done = 1; st->status = ST_BREAKDOWN; st->iterations = st->iter + 1;
    }
  }
}

__global__ void k_bi_xr(long long N, double *__restrict__ x, double *__restrict__ r,
                        const double *__restrict__ ph, const double *__restrict__ sh,
                        const double *__restrict__ s, const double *__restrict__ t,
                        KrylovState *st, double *hist, double *part, unsigned *count) {
  const int pend = st->pending_x;
  if (st->done && !pend) return;
  const double alfa = st->alfa, omega = st->omega, dV = st->dV;
  double v[1] = {0.0};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    double xv = __dadd_rn(x[p], __dmul_rn(alfa, ph[p]));
    if (pend) { x[p] = xv; continue; }
    x[p] = __dadd_rn(xv, __dmul_rn(omega, sh[p]));
    double rv = __dsub_rn(s[p], __dmul_rn(omega, t[p]));
    r[p] = rv;
    v[0] += voldiv(rv, rv, dV);
  }
  double o[1];
  if (grid_reduce<1>(v, part, count, o, st->seq, N)) {
    if (pend) { st->pending_x = 0; return; }
    const int it = st->iter;
    double res = res_of(o[0], st);
    st->res = res;
    if (hist && it < st->hist_cap) hist[it] = res;
    const bool minok = it >= st->mini - 1;
    if ((res < st->res_tol && minok) || (res < st->res0 * st->res_rat && minok)) {
      st->done = 1; st->converged = 1; st->status = ST_CONVERGED; st->iterations = it + 1;
    } else if (omega >= -st->res_tol && omega <= st->res_tol) {  // bicgs.cpp:189
      st->done = 1; st->status = ST_BREAKDOWN; st->iterations = it + 1;
    } else if (stale_step_dev(st, res)) {
      st->done = 1; st->status = ST_STALE; st->iterations = it + 1;
    } else if (!(res == res)) {
      st->done = 1; st->status = ST_NAN; st->iterations = it + 1;
    } else {
      st->rho_old = st->rho;
      st->iter = it + 1;
      st->iterations = it + 1;
      if (it + 1 >= st->maxit) { st->done = 1; st->status = ST_MAXITER; }
    }
  }
}


// ---------------------------------------------------------------------------
// Conjugate gradient squared, CGS::solve (cgs.cpp:8-210). One iteration:
//   k_cgs_rho  rho = r~.r; breakdown test; beta = rho / rho_old      (:83-104)
//   k_cgs_up   u = r + beta q; p = u + beta^2 p; p += beta q (u = p = r at
//              i = 0); p^ = p Mc                                      (:90-115)
//   k_bi_spmv  v^ = A p^; r~.v^; alfa                                (:120-126)
//   k_cgs_qs   q = u - alfa v^; s = u + q; u^ = s Mc                  (:131-139)
//   k_cgs_xr   x += alfa u^; r -= alfa A u^; res; tests               (:144-196)
// The initialisation (r = b - A x, r~ = r, res0) is k_bi_init's. With an
// incomplete Cholesky preconditioner (diag == 0) the IC sweeps form p^
// and u^ instead.
// ---------------------------------------------------------------------------
__global__ void k_cgs_rho(long long N, const double *__restrict__ rt, const double *__restrict__ r,
                          KrylovState *st, double *part, unsigned *count) {
  if (st->done) return;
  double v[1] = {0.0};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x)
    v[0] += __dmul_rn(rt[p], r[p]);
  double o[1];
  if (grid_reduce<1>(v, part, count, o, st->seq, N)) {
    const int it = st->iter;
    st->rho = o[0];
    if (__dsqrt_rn(fabs(o[0])) < st->res_tol) {
      st->done = 1; st->status = ST_BREAKDOWN; st->iterations = it + 1;
    } else if (it > 0) {
      st->beta = __ddiv_rn(o[0], st->rho_old);
    }
  }
}

__global__ void k_cgs_up(long long N, const double *__restrict__ c, const double *__restrict__ r,
                         const double *__restrict__ q, double *__restrict__ u, double *__restrict__ pv,
                         double *__restrict__ ph, const KrylovState *st, int diag) {
  if (st->done) return;
  const int it = st->iter;
  const double beta = st->beta, bb = __dmul_rn(st->beta, st->beta);
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    double uu, pp;
    if (it == 0) {
      uu = r[p];
      pp = uu;
    } else {
      uu = __dadd_rn(r[p], __dmul_rn(beta, q[p]));
      pp = __dadd_rn(uu, __dmul_rn(bb, pv[p]));
      pp = __dadd_rn(pp, __dmul_rn(beta, q[p]));
    }
    u[p] = uu;
    pv[p] = pp;
    if (diag) ph[p] = __dmul_rn(pp, c[p]);
  }
}

__global__ void k_cgs_qs(long long N, const double *__restrict__ c, const double *__restrict__ u,
                         const double *__restrict__ v, double *__restrict__ q, double *__restrict__ s,
                         double *__restrict__ sh, const KrylovState *st, int diag) {
  if (st->done) return;
  const double alfa = st->alfa;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    const double qq = __dsub_rn(u[p], __dmul_rn(alfa, v[p]));
    const double ss = __dadd_rn(u[p], qq);
    q[p] = qq;
    s[p] = ss;
    if (diag) sh[p] = __dmul_rn(ss, c[p]);
  }
}

__global__ void k_cgs_xr(MatView<double> A, double *__restrict__ x, double *__restrict__ r,
                         const double *__restrict__ sh, KrylovState *st, double *hist, double *part,
                         unsigned *count) {
  if (st->done) return;
  const long long N = A.ncell();
  const double alfa = st->alfa, dV = st->dV;
  double v[1] = {0.0};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    Pos q = pos_of(p, A.ny, A.nz);
    x[p] = __dadd_rn(x[p], __dmul_rn(alfa, sh[p]));
    const double qq = ref_ax(A, p, q, [&](long long t) { return sh[t]; });
    const double rv = __dsub_rn(r[p], __dmul_rn(alfa, qq));
    r[p] = rv;
    v[0] += voldiv(rv, rv, dV);
  }
  double o[1];
  if (grid_reduce<1>(v, part, count, o, st->seq, N)) {
    const int it = st->iter;
    double res = res_of(o[0], st);
    st->res = res;
    if (hist && it < st->hist_cap) hist[it] = res;
    const bool minok = it >= st->mini - 1;
    if ((res < st->res_tol && minok) || (res < st->res0 * st->res_rat && minok)) {
      st->done = 1; st->converged = 1; st->status = ST_CONVERGED; st->iterations = it + 1;
    } else if (stale_step_dev(st, res)) {
      st->done = 1; st->status = ST_STALE; st->iterations = it + 1;
    } else if (!(res == res)) {
      st->done = 1; st->status = ST_NAN; st->iterations = it + 1;
    } else {
      st->rho_old = st->rho;
      st->iter = it + 1;
      st->iterations = it + 1;
      if (it + 1 >= st->maxit) { st->done = 1; st->status = ST_MAXITER; }
    }
  }
}


// ---------------------------------------------------------------------------
// Additive-correction multigrid, reference form (Src/Solver/Additive).
// Coarse cell (I,J,K) covers fine cells I*CI..I*CI+CI-1 (likewise J, K),
// the index map of additive_coarsen_system.cpp:30-36.
// ---------------------------------------------------------------------------
struct FineCell {
  const MatView<double> &A;
  __device__ FineCell(const MatView<double> &a) : A(a) {}
  __device__ long long at(int i, int j, int k) const {
    return ((long long)i * A.ny + j) * A.nz + k;
  }
  __device__ double c(int i, int j, int k) const { return A.c[at(i, j, k)]; }
  __device__ double w(int i, int j, int k) const { return A.w[at(i, j, k)]; }
  __device__ double s(int i, int j, int k) const { return A.s[at(i, j, k)]; }
  __device__ double b(int i, int j, int k) const { return A.b[at(i, j, k)]; }
  __device__ double e(int i, int j, int k) const {
    return A.e ? A.e[at(i, j, k)]
               : (i < A.nx - 1 ? A.w[at(i + 1, j, k)] : ((A.per & 1) ? A.w[at(0, j, k)] : 0.0));
  }
  __device__ double n(int i, int j, int k) const {
    return A.n ? A.n[at(i, j, k)]
               : (j < A.ny - 1 ? A.s[at(i, j + 1, k)] : ((A.per & 2) ? A.s[at(i, 0, k)] : 0.0));
  }
  __device__ double t(int i, int j, int k) const {
    return A.t ? A.t[at(i, j, k)]
               : (k < A.nz - 1 ? A.b[at(i, j, k + 1)] : ((A.per & 4) ? A.b[at(i, j, 0)] : 0.0));
  }
  // a neighbour's value of a level field: the zero halo outside a
  // non-periodic face, the other end's cell across a periodic one
  __device__ double nbv(const double *x, int i, int j, int k) const {
    if (i < 0 || i >= A.nx) { if (!(A.per & 1)) return 0.0; i = i < 0 ? i + A.nx : i - A.nx; }
    if (j < 0 || j >= A.ny) { if (!(A.per & 2)) return 0.0; j = j < 0 ? j + A.ny : j - A.ny; }
    if (k < 0 || k >= A.nz) { if (!(A.per & 4)) return 0.0; k = k < 0 ? k + A.nz : k - A.nz; }
    return x[at(i, j, k)];
  }
};

struct CoarseOut { int nx, ny, nz; double *c, *w, *e, *s, *n, *b, *t; };

// AC::coarsen_system (additive_coarsen_system.cpp:4-140), one thread per
// coarse cell, the reference's summation order.
__global__ void k_ac_coarsen(MatView<double> A, CoarseOut H, int CI, int CJ, int CK) {
  FineCell f(A);
  const long long NH = (long long)H.nx * H.ny * H.nz;
  for (long long P = blockIdx.x * (long long)blockDim.x + threadIdx.x; P < NH;
       P += (long long)gridDim.x * blockDim.x) {
    Pos Q = pos_of(P, H.ny, H.nz);
    const int i0 = Q.i * CI, j0 = Q.j * CJ, k0 = Q.k * CK;
    double c = 0.0;
    for (int i = 0; i < CI; ++i)
      for (int j = 0; j < CJ; ++j)
        for (int k = 0; k < CK; ++k) c = __dadd_rn(c, f.c(i0 + i, j0 + j, k0 + k));
    for (int j = 0; j < CJ; ++j)
      for (int k = 0; k < CK; ++k) {
        for (int i = 0; i < CI - 1; ++i) c = __dsub_rn(c, f.e(i0 + i, j0 + j, k0 + k));
        for (int i = 1; i < CI; ++i) c = __dsub_rn(c, f.w(i0 + i, j0 + j, k0 + k));
      }
    double e = 0.0, w = 0.0;
    for (int j = 0; j < CJ; ++j)
      for (int k = 0; k < CK; ++k) {
        e = __dadd_rn(e, f.e(i0 + CI - 1, j0 + j, k0 + k));
        w = __dadd_rn(w, f.w(i0, j0 + j, k0 + k));
      }
    for (int i = 0; i < CI; ++i)
      for (int k = 0; k < CK; ++k) {
        for (int j = 0; j < CJ - 1; ++j) c = __dsub_rn(c, f.n(i0 + i, j0 + j, k0 + k));
        for (int j = 1; j < CJ; ++j) c = __dsub_rn(c, f.s(i0 + i, j0 + j, k0 + k));
      }
    double n = 0.0, s = 0.0;
    for (int i = 0; i < CI; ++i)
      for (int k = 0; k < CK; ++k) {
        n = __dadd_rn(n, f.n(i0 + i, j0 + CJ - 1, k0 + k));
        s = __dadd_rn(s, f.s(i0 + i, j0, k0 + k));
      }
    for (int i = 0; i < CI; ++i)
      for (int j = 0; j < CJ; ++j) {
        for (int k = 0; k < CK - 1; ++k) c = __dsub_rn(c, f.t(i0 + i, j0 + j, k0 + k));
        for (int k = 1; k < CK; ++k) c = __dsub_rn(c, f.b(i0 + i, j0 + j, k0 + k));
      }
    double t = 0.0, b = 0.0;
    for (int i = 0; i < CI; ++i)
      for (int j = 0; j < CJ; ++j) {
        t = __dadd_rn(t, f.t(i0 + i, j0 + j, k0 + CK - 1));
        b = __dadd_rn(b, f.b(i0 + i, j0 + j, k0));
      }
    H.c[P] = c; H.w[P] = w; H.e[P] = e; H.s[P] = s; H.n[P] = n; H.b[P] = b; H.t[P] = t;
  }
}

// AC::coarsen_flag (additive_coarsen_flag.cpp:4-41): OR over the block
__global__ void k_ac_flag(int fny, int fnz, const uint8_t *__restrict__ af, int Hnx, int Hny, int Hnz,
                          uint8_t *__restrict__ aH, int CI, int CJ, int CK) {
  const long long NH = (long long)Hnx * Hny * Hnz;
  for (long long P = blockIdx.x * (long long)blockDim.x + threadIdx.x; P < NH;
       P += (long long)gridDim.x * blockDim.x) {
    Pos Q = pos_of(P, Hny, Hnz);
    uint8_t v = 0;
    for (int i = 0; i < CI; ++i)
      for (int j = 0; j < CJ; ++j)
        for (int k = 0; k < CK; ++k)
          v |= af[((long long)(Q.i * CI + i) * fny + (Q.j * CJ + j)) * fnz + (Q.k * CK + k)];
    aH[P] = v;
  }
}

// AC::restriction (additive_restriction.cpp:12-177): coarse rhs = block sum
// of the fine residual in the reference's order (D = c minus the block's
// internal couplings, taken e, w, n, s, t, b), zero on inactive coarse cells;
// the block also sums the active values and counts them for the zero-mean
// step (:151-174), finished by k_ac_submean.
__global__ void k_ac_restrict(MatView<double> A, const double *__restrict__ phi,
                              const double *__restrict__ fnew, int Hnx, int Hny, int Hnz,
                              double *__restrict__ fH, const uint8_t *__restrict__ aH,
                              int CI, int CJ, int CK, double *mean_out, double *part,
                              unsigned *count, double *seq) {
  FineCell f(A);
  auto ph = [&](int i, int j, int k) -> double { return f.nbv(phi, i, j, k); };
  const long long NH = (long long)Hnx * Hny * Hnz;
  double v[2] = {0.0, 0.0};
  for (long long P = blockIdx.x * (long long)blockDim.x + threadIdx.x; P < NH;
       P += (long long)gridDim.x * blockDim.x) {
    Pos Q = pos_of(P, Hny, Hnz);
    const int i0 = Q.i * CI, j0 = Q.j * CJ, k0 = Q.k * CK;
    double F = 0.0;
    for (int i = 0; i < CI; ++i)
      for (int j = 0; j < CJ; ++j)
        for (int k = 0; k < CK; ++k) F = __dadd_rn(F, fnew[f.at(i0 + i, j0 + j, k0 + k)]);
    for (int j = 0; j < CJ; ++j)
      for (int k = 0; k < CK; ++k) {
        F = __dadd_rn(F, __dmul_rn(f.e(i0 + CI - 1, j0 + j, k0 + k), ph(i0 + CI, j0 + j, k0 + k)));
        F = __dadd_rn(F, __dmul_rn(f.w(i0, j0 + j, k0 + k), ph(i0 - 1, j0 + j, k0 + k)));
      }
    for (int i = 0; i < CI; ++i)
      for (int k = 0; k < CK; ++k) {
        F = __dadd_rn(F, __dmul_rn(f.n(i0 + i, j0 + CJ - 1, k0 + k), ph(i0 + i, j0 + CJ, k0 + k)));
        F = __dadd_rn(F, __dmul_rn(f.s(i0 + i, j0, k0 + k), ph(i0 + i, j0 - 1, k0 + k)));
      }
    for (int i = 0; i < CI; ++i)
      for (int j = 0; j < CJ; ++j) {
        F = __dadd_rn(F, __dmul_rn(f.t(i0 + i, j0 + j, k0 + CK - 1), ph(i0 + i, j0 + j, k0 + CK)));
        F = __dadd_rn(F, __dmul_rn(f.b(i0 + i, j0 + j, k0), ph(i0 + i, j0 + j, k0 - 1)));
      }
    for (int i = 0; i < CI; ++i)
      for (int j = 0; j < CJ; ++j)
        for (int k = 0; k < CK; ++k) {
          const int a = i0 + i, bb = j0 + j, cc = k0 + k;
          double D = f.c(a, bb, cc);
          if (i < CI - 1) D = __dsub_rn(D, f.e(a, bb, cc));
          if (i > 0) D = __dsub_rn(D, f.w(a, bb, cc));
          if (j < CJ - 1) D = __dsub_rn(D, f.n(a, bb, cc));
          if (j > 0) D = __dsub_rn(D, f.s(a, bb, cc));
          if (k < CK - 1) D = __dsub_rn(D, f.t(a, bb, cc));
          if (k > 0) D = __dsub_rn(D, f.b(a, bb, cc));
          F = __dsub_rn(F, __dmul_rn(D, phi[f.at(a, bb, cc)]));
        }
    if (!aH[P]) F = 0.0;
    fH[P] = F;
    if (aH[P]) { v[0] += F; v[1] += 1.0; }
  }
  double o[2];
  if (grid_reduce<2>(v, part, count, o, seq, NH)) *mean_out = __ddiv_rn(o[0], o[1]);
}

__global__ void k_ac_submean(long long NH, double *__restrict__ fH, const uint8_t *__restrict__ aH,
                             const double *mean) {
  const double m = *mean;
  for (long long P = blockIdx.x * (long long)blockDim.x + threadIdx.x; P < NH;
       P += (long long)gridDim.x * blockDim.x)
    if (aH[P]) fH[P] = __dsub_rn(fH[P], m);
}

// AC::interpolation (additive_interpolation.cpp:12-64): h.phi += H.phi
__global__ void k_ac_interp(int nx, int ny, int nz, double *__restrict__ phi, int Hny, int Hnz,
                            const double *__restrict__ phiH, int CI, int CJ, int CK) {
  const long long N = (long long)nx * ny * nz;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    Pos q = pos_of(p, ny, nz);
    long long P = ((long long)(q.i / CI) * Hny + q.j / CJ) * Hnz + q.k / CK;
    phi[p] = __dadd_rn(phi[p], phiH[P]);
  }
}

// AC::residual (additive_residual.cpp:4-30) with dt = 1: res = b - A phi,
// out[0] = sqrt(dot_voldiv_avg(res,res)), linf via an order-free max of
// |res/dV| (non-negative doubles order like their bit patterns).
__global__ void k_ac_resnorm(MatView<double> A, const double *__restrict__ phi,
                             const double *__restrict__ fnew, double dV, double *out,
                             unsigned long long *linf_bits, double *part, unsigned *count,
                             double *seq) {
  const long long N = A.ncell();
  double v[1] = {0.0};
  double mx = 0.0;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    Pos q = pos_of(p, A.ny, A.nz);
    double rv = ref_bmax(A, p, q, phi, fnew[p]);
    v[0] += voldiv(rv, rv, dV);
    mx = fmax(mx, fabs(__ddiv_rn(rv, dV)));
  }
  for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, off));
  if ((threadIdx.x & 31) == 0) atomicMax(linf_bits, (unsigned long long)__double_as_longlong(mx));
  double o[1];
  if (grid_reduce<1>(v, part, count, o, seq, N)) {
    double n = (double)N;
    out[0] = __dsqrt_rn(__ddiv_rn(__ddiv_rn(o[0], n), n));
  }
}

// ---------------------------------------------------------------------------
// Jacobi::solve (Src/Solver/Linear/Iterative/jacobi.cpp:10-75) and
// GaussSeidel::solve (gaussseidel.cpp:10-117). Both update x in place with
// the matrix's stored inverse central coefficient ci and form r = b - A x
// after every sweep. Jacobi measures sqrt(r.r) (jacobi.cpp:24,52,59-61);
// Gauss-Seidel measures sqrt(dot_voldiv_avg(r, r)) / scale and keeps a stale
// window (gaussseidel.cpp:24,68,85-105).
//
// Gauss-Seidel's sweep runs i, then j, then k (for_vijk) and reads the new
// values of the cells before the current one and the old values of the
// cells after it. Every neighbour of (i, j, k) lies on the hyperplane
// i + j + k - 1 (those before it) or i + j + k + 1 (those after it), so one
// launch per hyperplane h = i + j + k, in increasing h, computes every cell
// from exactly the values the sequential sweep uses.
// ---------------------------------------------------------------------------
// all entries unreal (gaussseidel.cpp:28-33; CG also seeds the last with res0)
__device__ void stale_fill_dev(KrylovState *st) {
  int n = st->stalecount > kStaleMax ? kStaleMax : st->stalecount;
  for (int q = 0; q < n; ++q) st->stale[q] = 1.0e24;  // boil::unreal
}

// the residual measure of the two solvers from the sum over cells
__device__ __forceinline__ double it_res(double d, const KrylovState *st, int gs) {
  return gs ? res_of(d, st) : __dsqrt_rn(d);
}

__global__ void k_it_init(MatView<double> A, const double *__restrict__ x,
                          const double *__restrict__ b, double *__restrict__ r, KrylovState *st,
                          double *part, unsigned *count, int gs) {
  const long long N = A.ncell();
  const double dV = st->dV;
  double v[1] = {0.0};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    Pos q = pos_of(p, A.ny, A.nz);
    double rv = ref_bmax(A, p, q, x, b[p]);
    r[p] = rv;
    v[0] += gs ? voldiv(rv, rv, dV) : __dmul_rn(rv, rv);
  }
  double o[1];
  if (grid_reduce<1>(v, part, count, o, st->seq, N)) {
    const double res = it_res(o[0], st, gs);
    st->res0 = res;
    st->res = res;
    st->iter = 0;
    st->iterations = 0;
    st->converged = 0;
    st->pending_x = 0;
    if (gs) stale_fill_dev(st);
    if (res < st->res_tol) {  // jacobi.cpp:35, gaussseidel.cpp:43
      st->done = 1;
      st->converged = 1;
      st->status = ST_INITIAL;
    } else if (st->maxit <= 0) {
      st->done = 1;
      st->status = ST_MAXITER;
    } else {
      st->done = 0;
      st->status = ST_RUNNING;
    }
  }
}

// x = ci (r + c x) with the r of the previous sweep (jacobi.cpp:42-44)
__global__ void k_jacobi_x(long long N, const double *__restrict__ c, const double *__restrict__ ci,
                           const double *__restrict__ r, double *__restrict__ x,
                           const KrylovState *st) {
  if (st->done) return;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x)
    x[p] = __dmul_rn(ci[p], __dadd_rn(r[p], __dmul_rn(c[p], x[p])));
}

// the cells of hyperplane h: x = ci (b + w xw + e xe + s xs + n xn + b xb
// + t xt), summed left to right (gaussseidel.cpp:50-60). One thread per
// (i, j) column; k = h - i - j. Across a periodic face the reference reads
// its halo, filled by the exchange before the sweep: xold, a copy of x
// taken before the sweep (only read when the matrix has periodic axes).
__global__ void k_gs_plane(MatView<double> A, const double *__restrict__ ci,
                           const double *__restrict__ b, double *x, int h, const KrylovState *st,
                           const double *__restrict__ xold) {
  if (st->done) return;
  const long long nij = (long long)A.nx * A.ny;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nij;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / A.ny), j = (int)(t - (long long)i * A.ny);
    const int k = h - i - j;
    if (k < 0 || k >= A.nz) continue;
    const long long p = ((long long)i * A.ny + j) * A.nz + k;
    const Pos q{i, j, k};
    Nb<double> a = coeffs(A, p, q);
    const NbIdx m = nb_index(A, p, q);
    // interior neighbours from x (this sweep's values where they come
    // first), wrapped ones from the pre-sweep copy
    auto nv = [&](long long idx, bool inside) {
      return idx < 0 ? 0.0 : (inside ? x[idx] : xold[idx]);
    };
    double v = b[p];
    v = __dadd_rn(v, __dmul_rn(a.w, nv(m.w, i > 0)));
    v = __dadd_rn(v, __dmul_rn(a.e, nv(m.e, i < A.nx - 1)));
    v = __dadd_rn(v, __dmul_rn(a.s, nv(m.s, j > 0)));
    v = __dadd_rn(v, __dmul_rn(a.n, nv(m.n, j < A.ny - 1)));
    v = __dadd_rn(v, __dmul_rn(a.b, nv(m.b, k > 0)));
    v = __dadd_rn(v, __dmul_rn(a.t, nv(m.t, k < A.nz - 1)));
    x[p] = __dmul_rn(ci[p], v);
  }
}

// r = b - A x after a sweep, the residual measure and the exits
// (jacobi.cpp:47-61, gaussseidel.cpp:63-105)
__global__ void k_it_resid(MatView<double> A, const double *__restrict__ x,
                           const double *__restrict__ b, double *__restrict__ r, KrylovState *st,
                           double *hist, double *part, unsigned *count, int gs) {
  if (st->done) return;
  const int it = st->iter;
  const long long N = A.ncell();
  const double dV = st->dV;
  double v[1] = {0.0};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    Pos q = pos_of(p, A.ny, A.nz);
    double rv = ref_bmax(A, p, q, x, b[p]);
    r[p] = rv;
    v[0] += gs ? voldiv(rv, rv, dV) : __dmul_rn(rv, rv);
  }
  double o[1];
  if (grid_reduce<1>(v, part, count, o, st->seq, N)) {
    const double res = it_res(o[0], st, gs);
    st->res = res;
    if (hist && it < st->hist_cap) hist[it] = res;
    const bool minok = it >= st->mini - 1;
    if ((res < st->res_tol && minok) || (res < st->res0 * st->res_rat && minok)) {
      st->done = 1; st->converged = 1; st->status = ST_CONVERGED; st->iterations = it + 1;
    } else if (gs && stale_step_dev(st, res)) {
      st->done = 1; st->status = ST_STALE; st->iterations = it + 1;
    } else if (!(res == res)) {
      st->done = 1; st->status = ST_NAN; st->iterations = it + 1;
    } else {
      st->iter = it + 1;
      st->iterations = it + 1;
      if (it + 1 >= st->maxit) { st->done = 1; st->status = ST_MAXITER; }
    }
  }
}

// ---------------------------------------------------------------------------
// Host drivers
// ---------------------------------------------------------------------------
__global__ void k_krylov_setup(KrylovState *st, KrylovParams pr, long long ncell) {
  st->res_rat = pr.res_rat;
  st->res_tol = pr.res_tol;
  st->scale = pr.scale;
  st->dV = pr.dV;
  st->ncell = (double)ncell;
  st->mini = pr.mini;
  st->maxit = pr.maxit;
  st->stalecount = pr.stalecount;
  st->hist_cap = pr.hist_cap;
  st->seq = pr.seq;
  st->done = 0;
  st->converged = 0;
  st->status = ST_RUNNING;
  st->iter = 0;
  st->iterations = 0;
  st->pending_x = 0;
  st->rho = st->rho_old = st->alfa = st->beta = st->omega = st->pq = 0.0;
}

void RefKrylovWork::ensure(size_t n, int solver) {
  auto fit = [n](DBuf<double> &b) { if (b.n < n) b.alloc(n); };
  fit(r); fit(mcd);
  if (solver >= 3) return;  // Jacobi, Gauss-Seidel: r and 1/c only
  fit(q); fit(pA); fit(pB);
  if (solver >= 1) { fit(rt); fit(ph); fit(v); fit(s); fit(sh); fit(t); }
  if (solver == 2) fit(u);
}

IcFactor RefKrylovWork::ic(int kind, size_t n) {
  auto fit = [n](DBuf<double> &b) { if (b.n < n) b.alloc(n); };
  fit(z); fit(mc); fit(mw); fit(ms); fit(mb);
  if (kind >= 2) { fit(mtw); fit(mts); }
  if (kind == 3) fit(mnw);
  IcFactor M;
  M.c = mc.p; M.w = mw.p; M.s = ms.p; M.b = mb.p;
  M.tw = kind >= 2 ? mtw.p : nullptr;
  M.ts = kind >= 2 ? mts.p : nullptr;
  M.nw = kind == 3 ? mnw.p : nullptr;
  M.kind = kind;
  M.wa = kind == 3 ? 5 : 2;
  M.wb = 2;
  return M;
}

// hyperplanes of the IC schedule (h = wa i + wb j + k over the grid)
static int ic_planes(const MatView<double> &A, const IcFactor &M) {
  return M.wa * (A.nx - 1) + M.wb * (A.ny - 1) + (A.nz - 1) + 1;
}

void enqueue_ref_setup(const MatView<double> &A, double *x, const double *b, const KrylovParams &pr,
                       int solver, RefKrylovWork &w, const RedPool &red, KrylovState *st,
                       cudaStream_t s) {
  const long long N = A.ncell();
  const int g = pr.seq ? grid_exact(N) : grid_for(N);
  w.ensure((size_t)N, solver);
  k_krylov_setup<<<1, 1, 0, s>>>(st, pr, N); note_launch();
  if (solver >= 3) {  // Jacobi, Gauss-Seidel: ci as stored with the matrix, else 1/c
    w.rhs = b;
    w.ci = pr.ci;
    if (!w.ci) {
      k_recip<<<grid_for(N), kThreads, 0, s>>>(N, A.c, w.mcd.p); note_launch();
      w.ci = w.mcd.p;
    }
    k_it_init<<<g, kThreads, 0, s>>>(A, x, b, w.r.p, st, red.slot_part(0), red.slot_count(0),
                                     solver == 4 ? 1 : 0); note_launch();
    PBG_CUDA(cudaGetLastError());
    return;
  }
  PBG_CUDA(cudaMemsetAsync(w.pA.p, 0, sizeof(double) * N, s));
  if (solver >= 1) {
    PBG_CUDA(cudaMemsetAsync(w.v.p, 0, sizeof(double) * N, s));
    PBG_CUDA(cudaMemsetAsync(w.q.p, 0, sizeof(double) * N, s));
  }
  if (pr.prec > 0) {  // IncompleteCholesky*::form on every solve (precform)
    const IcFactor M = w.ic(pr.prec, (size_t)N);
    DBuf<double> *arr[8] = {&w.z, &w.mc, &w.mw, &w.ms, &w.mb, &w.mtw, &w.mts, &w.mnw};
    for (DBuf<double> *a : arr)
      if (a->p) PBG_CUDA(cudaMemsetAsync(a->p, 0, sizeof(double) * N, s));
    const int H = ic_planes(A, M), gp = grid_for((long long)A.nx * A.ny);
    for (int h = 0; h < H; ++h) { k_ic_form<<<gp, kThreads, 0, s>>>(A, M, h); note_launch(); }
  }
  k_recip<<<grid_for(N), kThreads, 0, s>>>(N, A.c, w.mcd.p); note_launch();
  if (solver == 0)
    k_cg_init<<<g, kThreads, 0, s>>>(A, x, b, w.r.p, st, red.slot_part(0), red.slot_count(0), w.mcd.p);
  else
    k_bi_init<<<g, kThreads, 0, s>>>(A, x, b, w.r.p, w.rt.p, st, red.slot_part(0), red.slot_count(0));
  note_launch();
  PBG_CUDA(cudaGetLastError());
}

// z = M^-1 r with the IC factor: forward then backward hyperplane sweeps
static void ic_apply(const MatView<double> &A, const IcFactor &M, const double *r, double *z,
                     const KrylovState *st, cudaStream_t s) {
  const int H = ic_planes(A, M), gp = grid_for((long long)A.nx * A.ny);
  for (int h = 0; h < H; ++h) { k_ic_fwd<<<gp, kThreads, 0, s>>>(A, M, h, r, z, st); note_launch(); }
  for (int h = H - 1; h >= 0; --h) { k_ic_bwd<<<gp, kThreads, 0, s>>>(A, M, h, z, st); note_launch(); }
}

void enqueue_ref_iters(const MatView<double> &A, double *x, int solver, int count,
                       RefKrylovWork &w, const RedPool &red, KrylovState *st, double *hist,
                       cudaStream_t s, bool exact, int prec) {
  const long long N = A.ncell();
  const int g = exact ? grid_exact(N) : grid_for(N);
  double *P0 = red.slot_part(0), *P1 = red.slot_part(1);
  unsigned *C0 = red.slot_count(0), *C1 = red.slot_count(1);
  const int diag = prec > 0 ? 0 : 1;
  if (solver >= 3) {  // Jacobi, Gauss-Seidel
    const int gs = solver == 4 ? 1 : 0;
    const int H = A.nx + A.ny + A.nz - 2, gp = grid_for((long long)A.nx * A.ny);
    for (int it = 0; it < count; ++it) {
      if (gs) {
        if (A.per) {  // the halo the exchange fills before each sweep
          if (w.xold.n < (size_t)N) w.xold.alloc(N);
          PBG_CUDA(cudaMemcpyAsync(w.xold.p, x, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
        }
        for (int h = 0; h < H; ++h) {
          k_gs_plane<<<gp, kThreads, 0, s>>>(A, w.ci, w.rhs, x, h, st, w.xold.p); note_launch();
        }
      } else {
        k_jacobi_x<<<grid_for(N), kThreads, 0, s>>>(N, A.c, w.ci, w.r.p, x, st); note_launch();
      }
      k_it_resid<<<g, kThreads, 0, s>>>(A, x, w.rhs, w.r.p, st, hist, P0, C0, gs); note_launch();
    }
    PBG_CUDA(cudaGetLastError());
    return;
  }
  IcFactor M{};
  if (prec > 0) M = w.ic(prec, (size_t)N);
  for (int it = 0; it < count; ++it) {
    if (solver == 0 && prec > 0) {
      // z = M^-1 r (forward and backward sweeps), rho = r.z, then the CG step
      ic_apply(A, M, w.r.p, w.z.p, st, s);
      k_cg_rho<<<g, kThreads, 0, s>>>(N, w.r.p, w.z.p, st, P0, C0); note_launch();
      k_cg_pq<<<g, kThreads, 0, s>>>(A, w.r.p, w.pA.p, w.pB.p, w.q.p, st, P0, C0, w.z.p, w.mcd.p); note_launch();
      k_cg_xr<true><<<g, kThreads, 0, s>>>(N, w.mcd.p, x, w.r.p, w.pA.p, w.pB.p, w.q.p, st, hist, P1, C1, 1); note_launch();
    } else if (solver == 0 && !exact && A.nz % 2 == 0 && !A.per) {
      const int gq = grid_for(N / 2);
      k_cg_p<<<gq, kThreads, 0, s>>>(N, w.r.p, w.mcd.p, w.pA.p, st); note_launch();
      k_cg_q<<<gq, kThreads, 0, s>>>(A, Geo(A.nx, A.ny, A.nz), w.pA.p, w.q.p, st, P0, C0); note_launch();
      k_cg_xr<false><<<g, kThreads, 0, s>>>(N, w.mcd.p, x, w.r.p, w.pA.p, w.pA.p, w.q.p, st, hist, P1, C1, 0); note_launch();
    } else if (solver == 0) {
      k_cg_pq<<<g, kThreads, 0, s>>>(A, w.r.p, w.pA.p, w.pB.p, w.q.p, st, P0, C0, nullptr, w.mcd.p); note_launch();
      k_cg_xr<true><<<g, kThreads, 0, s>>>(N, w.mcd.p, x, w.r.p, w.pA.p, w.pB.p, w.q.p, st, hist, P1, C1, 0); note_launch();
    } else if (solver == 1) {
      k_bi_rho<<<g, kThreads, 0, s>>>(N, w.rt.p, w.r.p, st, P0, C0); note_launch();
      k_bi_p<<<g, kThreads, 0, s>>>(N, w.mcd.p, w.r.p, w.pA.p, w.v.p, w.ph.p, st, diag); note_launch();
      if (!diag) ic_apply(A, M, w.pA.p, w.ph.p, st, s);
      k_bi_spmv<<<g, kThreads, 0, s>>>(A, w.ph.p, w.v.p, w.rt.p, 0, st, P1, C1); note_launch();
      k_bi_s<<<g, kThreads, 0, s>>>(N, w.mcd.p, w.r.p, w.v.p, w.s.p, w.sh.p, st, P0, C0, diag); note_launch();
      if (!diag) ic_apply(A, M, w.s.p, w.sh.p, st, s);
      k_bi_spmv<<<g, kThreads, 0, s>>>(A, w.sh.p, w.t.p, w.s.p, 1, st, P1, C1); note_launch();
      k_bi_xr<<<g, kThreads, 0, s>>>(N, x, w.r.p, w.ph.p, w.sh.p, w.s.p, w.t.p, st, hist, P0, C0); note_launch();
    } else {
      k_cgs_rho<<<g, kThreads, 0, s>>>(N, w.rt.p, w.r.p, st, P0, C0); note_launch();
      k_cgs_up<<<g, kThreads, 0, s>>>(N, w.mcd.p, w.r.p, w.q.p, w.u.p, w.pA.p, w.ph.p, st, diag); note_launch();
      if (!diag) ic_apply(A, M, w.pA.p, w.ph.p, st, s);
      k_bi_spmv<<<g, kThreads, 0, s>>>(A, w.ph.p, w.v.p, w.rt.p, 0, st, P1, C1); note_launch();
      k_cgs_qs<<<g, kThreads, 0, s>>>(N, w.mcd.p, w.u.p, w.v.p, w.q.p, w.s.p, w.sh.p, st, diag); note_launch();
      if (!diag) ic_apply(A, M, w.s.p, w.sh.p, st, s);
      k_cgs_xr<<<g, kThreads, 0, s>>>(A, x, w.r.p, w.sh.p, st, hist, P0, C0); note_launch();
    }
  }
  PBG_CUDA(cudaGetLastError());
}

// Full solve with host polling of the device status every chunk.
RefKrylovResult ref_krylov_solve(const MatView<double> &A, double *x, const double *b,
                                 const KrylovParams &pr, int solver, RefKrylovWork &w,
                                 const RedPool &red, KrylovState *st, KrylovState *hst,
                                 double *hist, cudaStream_t s) {
  enqueue_ref_setup(A, x, b, pr, solver, w, red, st, s);
  int enq = 0, chunk = 8;
  for (;;) {
    PBG_CUDA(cudaMemcpyAsync(hst, st, sizeof(KrylovState), cudaMemcpyDeviceToHost, s));
    PBG_CUDA(cudaStreamSynchronize(s));
    if (hst->done || enq >= pr.maxit) break;
    int cnt = chunk;
    if (enq + cnt > pr.maxit) cnt = pr.maxit - enq;
    enqueue_ref_iters(A, x, solver, cnt, w, red, st, hist, s, pr.seq != nullptr, pr.prec);
    enq += cnt;
    if (chunk < 256) chunk *= 2;
  }
  RefKrylovResult r;
  r.converged = hst->converged;
  r.status = hst->status;
  r.iterations = hst->iterations;
  r.res0 = hst->res0;
  r.res = hst->res;
  return r;
}

// ----------------------------- reference AC ---------------------------------
static int first_factor(int n) {  // Domain::factor (domain_factor.cpp:4-21)
  int m = n - 1;
  for (;;) {
    if (m <= 0) return n;
    if (n % m == 0) return n / m;
    m--;
    if (m == 0 || m == 1) return n;
  }
}

void RefAC::build(const MatView<double> &A0, const uint8_t *aflag0, double h, cudaStream_t s) {
  L.clear();
  L.emplace_back();
  RefACLevel &l0 = L.back();
  l0.nx = A0.nx; l0.ny = A0.ny; l0.nz = A0.nz;
  l0.CI = l0.CJ = l0.CK = 1;
  double hx = h, hy = h, hz = h;
  l0.dV = hx * hy * hz;
  const long long N0 = A0.ncell();
  l0.phi.alloc(N0); l0.fnew.alloc(N0); l0.aflag.alloc(N0);
  PBG_CUDA(cudaMemcpyAsync(l0.aflag.p, aflag0, N0, cudaMemcpyDeviceToDevice, s));
  fold.alloc(N0);
  A0v = A0;
  // Domain::coarsen (domain_coarsen.cpp:6-112): factor = smallest prime
  // factor, coarsen a direction while interior % factor == 0, interior > 4
  // and interior != factor; stop when no direction coarsens.
  for (int lev = 1; lev < 64; ++lev) {
    const RefACLevel &f = L.back();
    int n[3] = {f.nx, f.ny, f.nz}, fac[3], ok[3];
    for (int d = 0; d < 3; ++d) {
      fac[d] = (d == 2 && A0.nz == 1) ? 2 : first_factor(n[d]);
      ok[d] = !((n[d] % fac[d]) != 0 || (n[d] + 6) <= 10 || n[d] == fac[d]);
    }
    if (!ok[0] && !ok[1] && !ok[2]) break;
    RefACLevel c;
    c.CI = ok[0] ? fac[0] : 1; c.CJ = ok[1] ? fac[1] : 1; c.CK = ok[2] ? fac[2] : 1;
    c.nx = n[0] / c.CI; c.ny = n[1] / c.CJ; c.nz = n[2] / c.CK;
    hx *= c.CI; hy *= c.CJ; hz *= c.CK;
    c.dV = hx * hy * hz;
    const long long NH = (long long)c.nx * c.ny * c.nz;
    c.A.nx = c.nx; c.A.ny = c.ny; c.A.nz = c.nz; c.A.sym = false;
    c.A.per = A0.per;  // coarse levels keep the fine level's periodic axes
    DBuf<double> *arr[7] = {&c.A.c, &c.A.w, &c.A.e, &c.A.s, &c.A.n, &c.A.b, &c.A.t};
    for (auto *a : arr) a->alloc(NH);
    c.phi.alloc(NH); c.fnew.alloc(NH); c.aflag.alloc(NH);
    k_ac_flag<<<grid_for(NH), kThreads, 0, s>>>(f.ny, f.nz, f.aflag.p, c.nx, c.ny, c.nz, c.aflag.p,
                                                 c.CI, c.CJ, c.CK); note_launch();
    L.push_back(std::move(c));
  }
  PBG_CUDA(cudaGetLastError());
}

MatView<double> RefAC::view(int l) const { return l == 0 ? A0v : L[l].A.view(); }

void RefAC::coarsen_all(cudaStream_t s) {
  for (size_t l = 1; l < L.size(); ++l) {
    RefACLevel &c = L[l];
    CoarseOut H{c.nx, c.ny, c.nz, c.A.c.p, c.A.w.p, c.A.e.p, c.A.s.p, c.A.n.p, c.A.b.p, c.A.t.p};
    long long NH = (long long)c.nx * c.ny * c.nz;
    k_ac_coarsen<<<grid_for(NH), kThreads, 0, s>>>(view((int)l - 1), H, c.CI, c.CJ, c.CK); note_launch();
  }
  PBG_CUDA(cudaGetLastError());
}

double RefAC::residual(RedPool &red, double *dscal, unsigned long long *dlinf, double *hbuf,
                       cudaStream_t s, double *linf) {
  const RefACLevel &l0 = L[0];
  PBG_CUDA(cudaMemsetAsync(dlinf, 0, sizeof(unsigned long long), s));
  const int g = seq ? grid_exact(A0v.ncell()) : grid_for(A0v.ncell());
  k_ac_resnorm<<<g, kThreads, 0, s>>>(A0v, l0.phi.p, l0.fnew.p, l0.dV, dscal, dlinf,
                                      red.slot_part(2), red.slot_count(2), seq); note_launch();
  PBG_CUDA(cudaGetLastError());
  PBG_CUDA(cudaMemcpyAsync(hbuf, dscal, sizeof(double), cudaMemcpyDeviceToHost, s));
  PBG_CUDA(cudaMemcpyAsync(hbuf + 1, dlinf, sizeof(double), cudaMemcpyDeviceToHost, s));
  PBG_CUDA(cudaStreamSynchronize(s));
  // sqrt(dot_voldiv_avg) * dt and max_abs_voldiv * dt (additive_residual.cpp:19-27)
  if (linf) *linf = hbuf[1] * res_dt;
  return hbuf[0] * res_dt;
}

// call_smoother (the level's Linear) or, with as_solver, call_solver (AC's
// own solver when one is set), additive_cycle_functions.cpp:90-107
void RefAC::smooth(int l, int mi, double res_rat, double res_tol, int ms, RefKrylovWork &w,
                   RedPool &red, KrylovState *st, cudaStream_t s, bool as_solver) {
  const bool own = as_solver && sol_kind >= 0;
  const int kind = own ? sol_kind : sm_kind;
  KrylovParams pr;
  pr.mini = 1; pr.maxit = mi; pr.stalecount = ms;
  pr.res_rat = res_rat; pr.res_tol = res_tol; pr.scale = sm_scale; pr.dV = L[l].dV; pr.hist_cap = 0;
  pr.seq = seq;
  pr.prec = own ? sol_prec : sm_prec;
  pr.ci = l == 0 ? sm_ci0 : nullptr;  // coarse levels: ci = 1/c (additive_coarsen_system.cpp)
  MatView<double> A = view(l);
  enqueue_ref_setup(A, L[l].phi.p, L[l].fnew.p, pr, kind, w, red, st, s);
  enqueue_ref_iters(A, L[l].phi.p, kind, mi, w, red, st, nullptr, s, seq != nullptr, pr.prec);
}

void RefAC::solve_l(int l, int mi, double res_rat, double res_tol, int ms, RefACCtx &cx) {
  smooth(l, mi, res_rat, res_tol, ms, *cx.w, *cx.red, cx.st, cx.s, true);
}

// call_smoother's return value, the solver's converged flag (a host round trip)
bool RefAC::smooth_converged(int l, int mi, double res_rat, double res_tol, int ms, RefACCtx &cx) {
  smooth(l, mi, res_rat, res_tol, ms, *cx.w, *cx.red, cx.st, cx.s, false);
  PBG_CUDA(cudaMemcpyAsync(cx.hst, cx.st, sizeof(KrylovState), cudaMemcpyDeviceToHost, cx.s));
  PBG_CUDA(cudaStreamSynchronize(cx.s));
  return cx.hst->converged != 0;
}

void RefAC::restrict_to(int l, RedPool &red, double *dmean, cudaStream_t s) {
  RefACLevel &f = L[l], &c = L[l + 1];
  long long NH = (long long)c.nx * c.ny * c.nz;
  int g = seq ? grid_exact(NH) : grid_for(NH);
  k_ac_restrict<<<g, kThreads, 0, s>>>(view(l), f.phi.p, f.fnew.p, c.nx, c.ny, c.nz, c.fnew.p,
                                        c.aflag.p, c.CI, c.CJ, c.CK, dmean, red.slot_part(3),
                                        red.slot_count(3), seq); note_launch();
  k_ac_submean<<<g, kThreads, 0, s>>>(NH, c.fnew.p, c.aflag.p, dmean); note_launch();
  PBG_CUDA(cudaGetLastError());
}

void RefAC::interp_from(int l, cudaStream_t s) {
  RefACLevel &c = L[l], &f = L[l - 1];
  long long N = (long long)f.nx * f.ny * f.nz;
  k_ac_interp<<<grid_for(N), kThreads, 0, s>>>(f.nx, f.ny, f.nz, f.phi.p, c.ny, c.nz, c.phi.p, c.CI,
                                               c.CJ, c.CK); note_launch();
  PBG_CUDA(cudaGetLastError());
}


// AC::cycle and its recursions (additive_cycle.cpp:4-99,
// additive_cycle_functions.cpp:12-107, additive_recursive.cpp:4-197).
void RefAC::run(int kind, int l, RefACCtx &cx) {
  if (kind == 1) v_cycle(l, cx);
  else if (kind == 2 || kind == 4) fw_cycle(l, cx, kind == 4);
  else if (kind == 5) flex_cycle(l, cx);
  else throw CudaError("AC: unknown cycle kind");
}

void RefAC::v_cycle(int l, RefACCtx &cx) {
  const int last = (int)L.size() - 1;
  if (l != last) {
    smooth(l, cx.mv[0], cx.resrat_val, cx.restol_val, cx.ms[0], *cx.w, *cx.red, cx.st, cx.s);
    restrict_to(l, *cx.red, cx.dmean, cx.s);
    v_cycle(l + 1, cx);
    solve_l(l, cx.mv[2], cx.resrat_val, cx.restol_val, cx.ms[2], cx);
    if (l > 0) interp_from(l, cx.s);
  } else {
    solve_l(l, 100, -1.0, cx.restol_val, -1, cx);
    if (l > 0) interp_from(l, cx.s);
  }
}

void RefAC::fw_cycle(int l, RefACCtx &cx, bool w) {
  const int last = (int)L.size() - 1;
  if (l != last) {
    smooth(l, cx.mv[0], cx.resrat_val, cx.restol_val, cx.ms[0], *cx.w, *cx.red, cx.st, cx.s);
    restrict_to(l, *cx.red, cx.dmean, cx.s);
    fw_cycle(l + 1, cx, w);
    smooth(l, cx.mv[1], cx.resrat_val, cx.restol_val, cx.ms[1], *cx.w, *cx.red, cx.st, cx.s);
    restrict_to(l, *cx.red, cx.dmean, cx.s);
    if (w) fw_cycle(l + 1, cx, w);
    else v_cycle(l + 1, cx);
    solve_l(l, cx.mv[2], cx.resrat_val, cx.restol_val, cx.ms[2], cx);
    if (l > 0) interp_from(l, cx.s);
  } else {
    solve_l(l, 100, -1.0, cx.restol_val, -1, cx);
    if (l > 0) interp_from(l, cx.s);
  }
}

// AC::flex_cycle (additive_recursive.cpp:161-197). The reference recurses
// on (level, sign) in tail position; here the same walk is a loop. A level
// whose smoother converges (to AC::resrat) hands its correction up and the
// finer level smooths with mv[2], ms[2] (Sign::pos); one that does not
// restricts down, where the next level smooths with mv[0], ms[0]
// (Sign::neg); the coarsest level is solved and interpolated up with
// Sign::neg. It starts at level l and ends when level 0's smoother
// converges. That needs the smoother's converged flag on the host: one
// round trip per smoother call. The reference never returns when level 0
// never converges; here the walk stops after cx.flex_visits smoother calls.
void RefAC::flex_cycle(int l, RefACCtx &cx) {
  const int last = (int)L.size() - 1;
  bool pos = false;
  flex_calls_ = 0;
  for (;;) {
    if (l != last) {
      const int idx = pos ? 2 : 0;
      if (++flex_calls_ > cx.flex_visits) { flex_capped_ = true; return; }
      if (smooth_converged(l, cx.mv[idx], cx.resrat_val, cx.restol_val, cx.ms[idx], cx)) {
        if (l == 0) return;
        interp_from(l, cx.s);
        l -= 1;
        pos = true;
      } else {
        restrict_to(l, *cx.red, cx.dmean, cx.s);
        l += 1;
        pos = false;
      }
    } else {
      solve_l(l, 100, -1.0, cx.restol_val, -1, cx);
      if (l == 0) return;
      interp_from(l, cx.s);
      l -= 1;
      pos = false;
    }
  }
}

void RefAC::full_cycle(int l, int kind, RefACCtx &cx) {
  const int last = (int)L.size() - 1;
  if (l != last) {
    restrict_to(l, *cx.red, cx.dmean, cx.s);
    full_cycle(l + 1, kind, cx);
    if (kind == 1 || kind == 2 || kind == 4 || kind == 5) run(kind, l, cx);
    else solve_l(l, 100, -1.0, cx.restol_val, -1, cx);  // the reference's "shouldn't happen" branch
  } else {
    solve_l(l, 100, -1.0, cx.restol_val, -1, cx);
    if (l > 0) interp_from(l, cx.s);
  }
}

RefACResult RefAC::cycle(double *x, const double *b, const RefACParams &pa, RefACCtx &cx,
                         double *res_hist, int hist_cap) {
  RefACLevel &l0 = L[0];
  const long long N0 = A0v.ncell();
  cudaStream_t s = cx.s;
  cx.flex_visits = pa.flex_visits;
  flex_capped_ = false;
  flex_calls_ = 0;
  PBG_CUDA(cudaMemcpyAsync(l0.phi.p, x, sizeof(double) * N0, cudaMemcpyDeviceToDevice, s));
  PBG_CUDA(cudaMemcpyAsync(l0.fnew.p, b, sizeof(double) * N0, cudaMemcpyDeviceToDevice, s));
  coarsen_all(s);  // rebuilt on every call (additive_cycle_functions.cpp:25-26)
  RefACResult out{};
  int nh = 0;
  auto record = [&](double r) {
    if (res_hist && nh < hist_cap) res_hist[nh] = r;
    nh++;
  };
  auto restore = [&]() {
    PBG_CUDA(cudaMemcpyAsync(l0.phi.p, fold.p, sizeof(double) * N0, cudaMemcpyDeviceToDevice, s));
  };
  // init_cycles (additive_cycle_functions.cpp:12-44); with use_linf the
  // tests read max |r/dV| (additive_cycle_functions.cpp:58-60)
  double linf_0;
  const double res_0 = residual(*cx.red, cx.dscal, cx.dlinf, cx.hbuf, s, &linf_0);
  record(res_0);
  PBG_CUDA(cudaMemcpyAsync(fold.p, l0.phi.p, sizeof(double) * N0, cudaMemcpyDeviceToDevice, s));
  out.res0 = res_0;
  const double res_0_control = pa.use_linf ? linf_0 : res_0;
  if ((res_0_control < pa.toler && pa.min_cyc == 0) || res_0 == 0.0) {
    out.converged = 1; out.cycles = 0; out.res = res_0;
  } else {
    for (size_t l = 1; l < L.size(); ++l) {
      long long n = (long long)L[l].nx * L[l].ny * L[l].nz;
      PBG_CUDA(cudaMemsetAsync(L[l].phi.p, 0, sizeof(double) * n, s));
      PBG_CUDA(cudaMemsetAsync(L[l].fnew.p, 0, sizeof(double) * n, s));
    }
    double linf_m1 = 0.0;
    double res_m1;
    if (pa.init != -1) {
      full_cycle(0, pa.init, cx);
      res_m1 = residual(*cx.red, cx.dscal, cx.dlinf, cx.hbuf, s, &linf_m1);
      record(res_m1);  // the reference logs it as cycle 0
      // converged(..., cycle 0, ...) (additive_cycle.cpp:39-43): its return
      // value is dropped, but its divergence branch compares the residual
      // with itself, so unless cycle 0 meets the tolerance stop_if_div
      // restores phi = fold, the initial guess
      const double rc = pa.use_linf ? linf_m1 : res_m1;
      const double rb = pa.use_linf ? linf_0 : res_0;
      if (!(0 >= pa.min_cyc && (rc / rb < pa.factor || rc < pa.toler))) {
        bool check = pa.stop_if_div != 0;
        if (pa.priority_min_cyc && 0 < pa.min_cyc) check = false;
        if (check) restore();
      }
    } else {
      res_m1 = residual(*cx.red, cx.dscal, cx.dlinf, cx.hbuf, s, &linf_m1);
    }
    out.cycles = pa.max_cyc;
    out.converged = 0;
    out.res = res_m1;
    for (int c = 1; c <= pa.max_cyc; ++c) {
      if (pa.loop != 1 && pa.loop != 2 && pa.loop != 4 && pa.loop != 5) {
        // just solve (additive_cycle.cpp:66-71): AC's solver on level 0
        solve_l(0, 40, 0.001, 1.0e-15, -1, cx);
        out.res = residual(*cx.red, cx.dscal, cx.dlinf, cx.hbuf, s, nullptr);
        break;
      }
      run(pa.loop, 0, cx);
      if (flex_capped_) {  // the flex walk hit its bound: stop, not converged
        out.res = residual(*cx.red, cx.dscal, cx.dlinf, cx.hbuf, s, nullptr);
        out.cycles = c;
        out.flex_capped = 1;
        break;
      }
      double linf1;
      const double res1 = residual(*cx.red, cx.dscal, cx.dlinf, cx.hbuf, s, &linf1);
      record(res1);
      out.res = res1;
      const double rc = pa.use_linf ? linf1 : res1;
      const double r0 = pa.use_linf ? linf_m1 : res_m1;   // linf_m1 is never refreshed (:78)
      const double rb = pa.use_linf ? linf_0 : res_0;
      int con;
      if (c >= pa.min_cyc && (rc / rb < pa.factor || rc < pa.toler)) {
        con = 0;
      } else {
        bool check = pa.stop_if_div != 0;
        if (pa.priority_min_cyc && c < pa.min_cyc) check = false;
        if (check && rc >= r0) {
          restore();
          con = 1;
        } else {
          con = 2;
        }
      }
      res_m1 = res1;
      if (con == 0) { out.converged = 1; out.cycles = c; break; }
      if (con == 1) { out.converged = 0; out.cycles = c; out.diverged = 1; break; }
      PBG_CUDA(cudaMemcpyAsync(fold.p, l0.phi.p, sizeof(double) * N0, cudaMemcpyDeviceToDevice, s));
    }
  }
  PBG_CUDA(cudaMemcpyAsync(x, l0.phi.p, sizeof(double) * N0, cudaMemcpyDeviceToDevice, s));
  PBG_CUDA(cudaStreamSynchronize(s));
  out.nhist = nh;
  out.visits = (int)flex_calls_;
  return out;
}

}  // namespace pbg
