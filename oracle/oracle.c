/*
 * CPU oracle: plain-C restatement of the reference pressure-Poisson path.
 * TEST INFRASTRUCTURE ONLY (the parity checker); see oracle.h.
 *
 * Every function states the reference file:line it follows. Operation
 * order is kept where it decides the rounding (SpMV pair sums, residual
 * accumulation, sequential dot products, coarse-operator sums).
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define IDX(i, j, k) (((size_t)(i) * ny + (size_t)(j)) * nz + (size_t)(k))

/* ------------------------------------------------------------------ */
/* Scalar operators                                                    */
/* ------------------------------------------------------------------ */

/* The value of field x at (i, j, k), which may lie one cell outside the
 * grid: the reference's halo, zero on a non-periodic face and the cell at
 * the other end on a periodic one (scalar_exchange.cpp:47-58). */
static double halo(const orc_mat *A, const double *x, int i, int j, int k) {
  const int nx = A->nx, ny = A->ny, nz = A->nz;
  if (i < 0 || i >= nx) { if (!(A->per & 1)) return 0.0; i = i < 0 ? i + nx : i - nx; }
  if (j < 0 || j >= ny) { if (!(A->per & 2)) return 0.0; j = j < 0 ? j + ny : j - ny; }
  if (k < 0 || k >= nz) { if (!(A->per & 4)) return 0.0; k = k < 0 ? k + nz : k - nz; }
  return x[IDX(i, j, k)];
}

/* scalar_operators.cpp:49-72: four passes; each pair sum is formed first
 * and then subtracted. Out-of-domain neighbours are the halo. */
void orc_spmv(const orc_mat *A, const double *x, double *y) {
  const int nx = A->nx, ny = A->ny, nz = A->nz;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        size_t p = IDX(i, j, k);
        double xw = halo(A, x, i - 1, j, k), xe = halo(A, x, i + 1, j, k);
        double xs = halo(A, x, i, j - 1, k), xn = halo(A, x, i, j + 1, k);
        double xb = halo(A, x, i, j, k - 1), xt = halo(A, x, i, j, k + 1);
        double v = A->c[p] * x[p];
        v -= (A->w[p] * xw + A->e[p] * xe);
        v -= (A->s[p] * xs + A->n[p] * xn);
        v -= (A->b[p] * xb + A->t[p] * xt);
        y[p] = v;
      }
}

/* scalar_operators.cpp:22-46 */
void orc_resid(const orc_mat *A, const double *x, const double *b, double *r) {
  const int nx = A->nx, ny = A->ny, nz = A->nz;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        size_t p = IDX(i, j, k);
        double xw = halo(A, x, i - 1, j, k), xe = halo(A, x, i + 1, j, k);
        double xs = halo(A, x, i, j - 1, k), xn = halo(A, x, i, j + 1, k);
        double xb = halo(A, x, i, j, k - 1), xt = halo(A, x, i, j, k + 1);
        double v = b[p] - A->c[p] * x[p];
        v += A->w[p] * xw + A->e[p] * xe;
        v += A->s[p] * xs + A->n[p] * xn;
        v += A->b[p] * xb + A->t[p] * xt;
        r[p] = v;
      }
}

/* scalar.h:296-298 */
double orc_dot(size_t n, const double *x, const double *y) {
  double d = 0.0;
  for (size_t p = 0; p < n; ++p) d += x[p] * y[p];
  return d;
}

/* scalar.h:317-326: d += x*y/dV/dV, then d/N/N */
double orc_dot_voldiv_avg(size_t n, const double *x, const double *y, double dV) {
  double d = 0.0;
  for (size_t p = 0; p < n; ++p) d += x[p] * y[p] / dV / dV;
  return d / (double)n / (double)n;
}

/* scalar_minmax.cpp:155-165 */
double orc_max_abs_voldiv(size_t n, const double *x, double dV) {
  double v = fabs(x[0] / dV);
  for (size_t p = 0; p < n; ++p)
    if (fabs(x[p] / dV) > v) v = fabs(x[p] / dV);
  return v;
}

/* ------------------------------------------------------------------ */
/* Krylov solvers                                                      */
/* ------------------------------------------------------------------ */

/* staleness window of cg.cpp:39-45,138-160 / bicgs.cpp:58-64,195-217 */
typedef struct { double *v; int n; } stale_win;

static void stale_init(stale_win *w, int n, double res0) {
  w->n = n > 0 ? n : 0;
  w->v = NULL;
  if (w->n) {
    w->v = (double *)malloc(sizeof(double) * w->n);
    for (int q = 0; q < w->n; ++q) w->v[q] = 1.0e24; /* boil::unreal */
    w->v[w->n - 1] = res0;
  }
}
/* returns 1 when stale (breaks), else rotates the window */
static int stale_step(stale_win *w, double res) {
  if (!w->n) return 0;
  int stale = 1;
  for (int q = 0; q < w->n; ++q)
    if (res < w->v[q]) { stale = 0; break; }
  if (stale) return 1;
  memmove(w->v, w->v + 1, sizeof(double) * (w->n - 1));
  w->v[w->n - 1] = res;
  return 0;
}

/* cg.cpp:10-182 with Diagonal (preconditioner_form.cpp:4-13,
 * preconditioner_solve.cpp:4-11) */
/* Incomplete Cholesky IC0 / IC2 / IC3: IncompleteCholesky0/2/3::form
 * (preconditioner_form.cpp:16-144) and ::solve (preconditioner_solve.cpp:
 * 14-110), in the reference's lexicographic order and operation order, on
 * compact arrays. Entries outside the domain (the reference's halo) are not
 * stored: the factor writes them but no interior cell reads them, and the
 * sweeps multiply them by the zero halo of z, so those terms are skipped. */
typedef struct {
  int kind;
  double *c, *w, *s, *b, *tw, *ts, *nw;
} orc_ic;

static void ic_form(const orc_mat *A, orc_ic *M) {
  const int nx = A->nx, ny = A->ny, nz = A->nz;
  const size_t SI = (size_t)ny * nz, SJ = nz;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        const size_t p = ((size_t)i * ny + j) * nz + k;
        const int xp = i + 1 < nx, yp = j + 1 < ny, zp = k + 1 < nz, zm = k > 0, ym = j > 0;
        double sum = A->c[p];
        sum = sum - M->w[p] * M->w[p];
        if (M->kind >= 2) sum = sum - M->tw[p] * M->tw[p];
        if (M->kind == 3) sum = sum - M->nw[p] * M->nw[p];
        sum = sum - M->s[p] * M->s[p];
        if (M->kind >= 2) sum = sum - M->ts[p] * M->ts[p];
        sum = sum - M->b[p] * M->b[p];
        sum = sqrt(sum);
        M->c[p] = sum;
        if (M->kind == 1) { /* IC0 (:16-38) */
          if (xp) M->w[p + SI] = -A->w[p + SI] / sum;
          if (yp) M->s[p + SJ] = -A->s[p + SJ] / sum;
          if (zp) M->b[p + 1] = -A->b[p + 1] / sum;
          continue;
        }
        /* IC2 (:42-84), IC3 (:88-144) */
        if (xp) M->w[p + SI] = -A->w[p + SI] / sum;
        if (xp && zm) M->tw[p + SI - 1] = -M->w[p + SI - 1] * M->b[p] / sum;
        if (M->kind == 3 && xp && ym)
          M->nw[p + SI - SJ] = (-M->w[p + SI - SJ] * M->s[p] - M->tw[p + SI - SJ] * M->ts[p]) / sum;
        if (yp) {
          if (M->kind == 2) M->s[p + SJ] = -A->s[p + SJ] / sum;
          else M->s[p + SJ] = (-A->s[p + SJ] - M->w[p + SJ] * M->nw[p] - M->nw[p + SJ] * M->s[p]) / sum;
        }
        if (yp && zm) {
          if (M->kind == 2) M->ts[p + SJ - 1] = -M->s[p + SJ - 1] * M->b[p] / sum;
          else M->ts[p + SJ - 1] = (-M->s[p + SJ - 1] * M->b[p] - M->tw[p + SJ - 1] * M->nw[p]) / sum;
        }
        if (zp) M->b[p + 1] = (-A->b[p + 1] - M->w[p + 1] * M->tw[p] - M->s[p + 1] * M->ts[p]) / sum;
      }
}

static void ic_solve(const orc_mat *A, const orc_ic *M, double *z, const double *r) {
  const int nx = A->nx, ny = A->ny, nz = A->nz;
  const size_t SI = (size_t)ny * nz, SJ = nz;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        const size_t p = ((size_t)i * ny + j) * nz + k;
        double sum = r[p];
        if (i > 0) sum = sum - M->w[p] * z[p - SI];
        if (M->kind >= 2 && i > 0 && k + 1 < nz) sum = sum - M->tw[p] * z[p - SI + 1];
        if (M->kind == 3 && i > 0 && j + 1 < ny) sum = sum - M->nw[p] * z[p - SI + SJ];
        if (j > 0) sum = sum - M->s[p] * z[p - SJ];
        if (M->kind >= 2 && j > 0 && k + 1 < nz) sum = sum - M->ts[p] * z[p - SJ + 1];
        if (k > 0) sum = sum - M->b[p] * z[p - 1];
        z[p] = sum / M->c[p];
      }
  for (int i = nx - 1; i >= 0; --i)
    for (int j = ny - 1; j >= 0; --j)
      for (int k = nz - 1; k >= 0; --k) {
        const size_t p = ((size_t)i * ny + j) * nz + k;
        const int xp = i + 1 < nx, yp = j + 1 < ny, zp = k + 1 < nz, zm = k > 0, ym = j > 0;
        double sum = z[p];
        if (xp) sum = sum - M->w[p + SI] * z[p + SI];
        if (M->kind >= 2 && xp && zm) sum = sum - M->tw[p + SI - 1] * z[p + SI - 1];
        if (M->kind == 3 && xp && ym) sum = sum - M->nw[p + SI - SJ] * z[p + SI - SJ];
        if (yp) sum = sum - M->s[p + SJ] * z[p + SJ];
        if (M->kind >= 2 && yp && zm) sum = sum - M->ts[p + SJ - 1] * z[p + SJ - 1];
        if (zp) sum = sum - M->b[p + 1] * z[p + 1];
        z[p] = sum / M->c[p];
      }
}

/* cg.cpp:10-182 with Prec::di (prec 0) or Prec::ic0/ic2/ic3 (1, 2, 3) */
int orc_cg_prec(const orc_mat *A, double *x, const double *b, int mini, int maxit,
                double res_rat, double res_tol, double scale, int stalecount,
                double dV, orc_stats *st, double *hist, int prec);

int orc_cg(const orc_mat *A, double *x, const double *b, int mini, int maxit,
           double res_rat, double res_tol, double scale, int stalecount,
           double dV, orc_stats *st, double *hist) {
  return orc_cg_prec(A, x, b, mini, maxit, res_rat, res_tol, scale, stalecount, dV, st, hist, 0);
}

int orc_cg_prec(const orc_mat *A, double *x, const double *b, int mini, int maxit,
                double res_rat, double res_tol, double scale, int stalecount,
                double dV, orc_stats *st, double *hist, int prec) {
  const size_t N = (size_t)A->nx * A->ny * A->nz;
  double *p = calloc(N, sizeof(double)), *q = calloc(N, sizeof(double));
  double *r = calloc(N, sizeof(double)), *z = calloc(N, sizeof(double));
  double *Mc = calloc(N, sizeof(double));
  orc_ic M = {prec, NULL, NULL, NULL, NULL, NULL, NULL, NULL};
  if (prec > 0) {
    M.c = calloc(N, sizeof(double)); M.w = calloc(N, sizeof(double));
    M.s = calloc(N, sizeof(double)); M.b = calloc(N, sizeof(double));
    if (prec >= 2) { M.tw = calloc(N, sizeof(double)); M.ts = calloc(N, sizeof(double)); }
    if (prec == 3) M.nw = calloc(N, sizeof(double));
    ic_form(A, &M);
  }
  for (size_t c = 0; c < N; ++c) Mc[c] = 1.0 / A->c[c];
  orc_resid(A, x, b, r);
  double res = sqrt(orc_dot_voldiv_avg(N, r, r, dV)) / scale;
  double res0 = res;
  stale_win win;
  stale_init(&win, stalecount, res);
  orc_stats s = {0, 0, 0, res0, res, 0};
  if (res < res_tol) {
    s.converged = 1; s.status = 4;
    free(p); free(q); free(r); free(z); free(Mc); free(win.v);
    free(M.c); free(M.w); free(M.s); free(M.b); free(M.tw); free(M.ts); free(M.nw);
    if (st) *st = s;
    return 1;
  }
  double rho = 0, rho_old = 0, alfa, beta, pq;
  int converged = 0, i, broke = 0;
  s.status = 1;
  for (i = 0; i < maxit; ++i) {
    if (prec > 0) ic_solve(A, &M, z, r);
    else
      for (size_t c = 0; c < N; ++c) z[c] = r[c] * Mc[c];
    rho = orc_dot(N, r, z);
    if (i == 0) {
      memcpy(p, z, N * sizeof(double));
    } else {
      beta = rho / rho_old;
      for (size_t c = 0; c < N; ++c) p[c] = z[c] + beta * p[c];
    }
    orc_spmv(A, p, q);
    pq = orc_dot(N, p, q);
    alfa = rho / pq;
    for (size_t c = 0; c < N; ++c) x[c] += alfa * p[c];
    for (size_t c = 0; c < N; ++c) r[c] -= alfa * q[c];
    res = sqrt(orc_dot_voldiv_avg(N, r, r, dV)) / scale;
    if (hist) hist[i] = res;
    if (res < res_tol && i >= mini - 1) { converged = 1; broke = 1; s.status = 0; break; }
    if (res < res0 * res_rat && i >= mini - 1) { converged = 1; broke = 1; s.status = 0; break; }
    if (stale_step(&win, res)) { broke = 1; s.status = 2; break; }
    rho_old = rho;
  }
  s.converged = converged;
  s.iterations = broke ? i + 1 : maxit;
  s.printed = i + 1;
  s.res = res;
  if (st) *st = s;
  free(p); free(q); free(r); free(z); free(Mc); free(win.v);
  free(M.c); free(M.w); free(M.s); free(M.b); free(M.tw); free(M.ts); free(M.nw);
  return converged;
}

/* The preconditioner of a Krylov solve: Prec::di (prec 0, Mc = 1/c, z = r
 * Mc) or Prec::ic0/ic2/ic3 (1, 2, 3), formed once per solve as
 * Krylov::solve does with precform (bicgs.cpp:37-39, cgs.cpp:38-39). */
typedef struct {
  int prec;
  double *Mc;
  orc_ic M;
} orc_prec;

static void prec_form(const orc_mat *A, int prec, orc_prec *P) {
  const size_t N = (size_t)A->nx * A->ny * A->nz;
  P->prec = prec;
  P->Mc = calloc(N, sizeof(double));
  for (size_t c = 0; c < N; ++c) P->Mc[c] = 1.0 / A->c[c];
  orc_ic M = {prec, NULL, NULL, NULL, NULL, NULL, NULL, NULL};
  if (prec > 0) {
    M.c = calloc(N, sizeof(double)); M.w = calloc(N, sizeof(double));
    M.s = calloc(N, sizeof(double)); M.b = calloc(N, sizeof(double));
    if (prec >= 2) { M.tw = calloc(N, sizeof(double)); M.ts = calloc(N, sizeof(double)); }
    if (prec == 3) M.nw = calloc(N, sizeof(double));
    ic_form(A, &M);
  }
  P->M = M;
}

/* M z = r (Diagonal::solve, preconditioner_solve.cpp:4-11, or the IC sweeps) */
static void prec_solve(const orc_mat *A, const orc_prec *P, double *z, const double *r) {
  const size_t N = (size_t)A->nx * A->ny * A->nz;
  if (P->prec > 0) ic_solve(A, &P->M, z, r);
  else
    for (size_t c = 0; c < N; ++c) z[c] = r[c] * P->Mc[c];
}

static void prec_free(orc_prec *P) {
  free(P->Mc);
  free(P->M.c); free(P->M.w); free(P->M.s); free(P->M.b); free(P->M.tw); free(P->M.ts); free(P->M.nw);
}

/* bicgs.cpp:9-229 with Prec::di (prec 0) or Prec::ic0/ic2/ic3 */
int orc_bicgs_prec(const orc_mat *A, double *x, const double *b, int mini, int maxit,
                   double res_rat, double res_tol, double scale, int stalecount,
                   double dV, orc_stats *st, double *hist, int prec) {
  const size_t N = (size_t)A->nx * A->ny * A->nz;
  double *p = calloc(N, sizeof(double)), *r = calloc(N, sizeof(double));
  double *s = calloc(N, sizeof(double)), *t = calloc(N, sizeof(double));
  double *v = calloc(N, sizeof(double)), *p_ = calloc(N, sizeof(double));
  double *r_ = calloc(N, sizeof(double)), *s_ = calloc(N, sizeof(double));
  orc_prec P;
  prec_form(A, prec, &P);
  orc_resid(A, x, b, r);
  double res = sqrt(orc_dot_voldiv_avg(N, r, r, dV)) / scale;
  double res0 = res;
  stale_win win;
  stale_init(&win, stalecount, res);
  orc_stats so = {0, 0, 0, res0, res, 0};
  int converged = 0, i, broke = 0;
  if (res < res_tol) {
    so.converged = 1; so.status = 4;
    goto done_early;
  }
  memcpy(r_, r, N * sizeof(double));
  double alfa = 0, beta, omega = 0, rho = 0, rho_old = 0, r_v, ss, ts, tt;
  so.status = 1;
  for (i = 0; i < maxit; ++i) {
    rho = orc_dot(N, r_, r);
    if (sqrt(fabs(rho)) < res_tol) { broke = 1; so.status = 3; break; }
    if (i == 0) {
      memcpy(p, r, N * sizeof(double));
    } else {
      beta = (rho / rho_old) * (alfa / omega);
      for (size_t c = 0; c < N; ++c) p[c] = r[c] + beta * p[c];
      double bo = beta * omega;
      for (size_t c = 0; c < N; ++c) p[c] -= bo * v[c];
    }
    prec_solve(A, &P, p_, p);
    orc_spmv(A, p_, v);
    r_v = orc_dot(N, r_, v);
    alfa = rho / r_v;
    for (size_t c = 0; c < N; ++c) s[c] = r[c] - alfa * v[c];
    ss = orc_dot(N, s, s);
    if (sqrt(ss) < res_tol) {
      for (size_t c = 0; c < N; ++c) x[c] += alfa * p_[c];
      broke = 1; so.status = 3;
      break;
    }
    prec_solve(A, &P, s_, s);
    orc_spmv(A, s_, t);
    ts = orc_dot(N, t, s);
    tt = orc_dot(N, t, t);
    omega = ts / tt;
    for (size_t c = 0; c < N; ++c) x[c] += alfa * p_[c];
    for (size_t c = 0; c < N; ++c) x[c] += omega * s_[c];
    for (size_t c = 0; c < N; ++c) r[c] = s[c] - omega * t[c];
    res = sqrt(orc_dot_voldiv_avg(N, r, r, dV)) / scale;
    if (hist) hist[i] = res;
    if (res < res_tol && i >= mini - 1) { converged = 1; broke = 1; so.status = 0; break; }
    if (res < res0 * res_rat && i >= mini - 1) { converged = 1; broke = 1; so.status = 0; break; }
    if (omega >= -res_tol && omega <= res_tol) { broke = 1; so.status = 3; break; }
    if (stale_step(&win, res)) { broke = 1; so.status = 2; break; }
    rho_old = rho;
  }
  so.converged = converged;
  so.iterations = broke ? i + 1 : maxit;
  so.printed = i + 1;
  so.res = res;
done_early:
  if (st) *st = so;
  free(p); free(r); free(s); free(t); free(v); free(p_); free(r_); free(s_);
  prec_free(&P);
  free(win.v);
  return converged || so.status == 4;
}

int orc_bicgs(const orc_mat *A, double *x, const double *b, int mini, int maxit,
              double res_rat, double res_tol, double scale, int stalecount,
              double dV, orc_stats *st, double *hist) {
  return orc_bicgs_prec(A, x, b, mini, maxit, res_rat, res_tol, scale, stalecount, dV, st, hist, 0);
}

/* cgs.cpp:8-210 (conjugate gradient squared) with Prec::di or Prec::ic* */
int orc_cgs_prec(const orc_mat *A, double *x, const double *b, int mini, int maxit,
                 double res_rat, double res_tol, double scale, int stalecount,
                 double dV, orc_stats *st, double *hist, int prec) {
  const size_t N = (size_t)A->nx * A->ny * A->nz;
  double *p = calloc(N, sizeof(double)), *q = calloc(N, sizeof(double));
  double *r = calloc(N, sizeof(double)), *s = calloc(N, sizeof(double));
  double *u = calloc(N, sizeof(double)), *p_ = calloc(N, sizeof(double));
  double *q_ = calloc(N, sizeof(double)), *r_ = calloc(N, sizeof(double));
  double *u_ = calloc(N, sizeof(double)), *v_ = calloc(N, sizeof(double));
  orc_prec P;
  prec_form(A, prec, &P);
  orc_resid(A, x, b, r);
  double res = sqrt(orc_dot_voldiv_avg(N, r, r, dV)) / scale;
  double res0 = res;
  stale_win win;
  stale_init(&win, stalecount, res);
  orc_stats so = {0, 0, 0, res0, res, 0};
  int converged = 0, i, broke = 0;
  if (res < res_tol) { /* cgs.cpp:69: returns true */
    so.converged = 1; so.status = 4;
    goto done_early;
  }
  memcpy(r_, r, N * sizeof(double));
  double alfa, beta, rho = 0, rho_old = 0, r_v_;
  so.status = 1;
  for (i = 0; i < maxit; ++i) {
    rho = orc_dot(N, r_, r);
    if (sqrt(fabs(rho)) < res_tol) { broke = 1; so.status = 3; break; }
    if (i == 0) {
      memcpy(u, r, N * sizeof(double));
      memcpy(p, u, N * sizeof(double));
    } else {
      beta = rho / rho_old;
      const double bb = beta * beta;
      for (size_t c = 0; c < N; ++c) u[c] = r[c] + beta * q[c];
      for (size_t c = 0; c < N; ++c) p[c] = u[c] + bb * p[c];
      for (size_t c = 0; c < N; ++c) p[c] += beta * q[c];
    }
    prec_solve(A, &P, p_, p);
    orc_spmv(A, p_, v_);
    r_v_ = orc_dot(N, r_, v_);
    alfa = rho / r_v_;
    for (size_t c = 0; c < N; ++c) q[c] = u[c] - alfa * v_[c];
    for (size_t c = 0; c < N; ++c) s[c] = u[c] + q[c];
    prec_solve(A, &P, u_, s);
    for (size_t c = 0; c < N; ++c) x[c] += alfa * u_[c];
    orc_spmv(A, u_, q_);
    for (size_t c = 0; c < N; ++c) r[c] -= alfa * q_[c];
    res = sqrt(orc_dot_voldiv_avg(N, r, r, dV)) / scale;
    if (hist) hist[i] = res;
    if (res < res_tol && i >= mini - 1) { converged = 1; broke = 1; so.status = 0; break; }
    if (res < res0 * res_rat && i >= mini - 1) { converged = 1; broke = 1; so.status = 0; break; }
    if (stale_step(&win, res)) { broke = 1; so.status = 2; break; }
    rho_old = rho;
  }
  so.converged = converged;
  so.iterations = broke ? i + 1 : maxit;
  so.printed = i + 1;
  so.res = res;
done_early:
  if (st) *st = so;
  free(p); free(q); free(r); free(s); free(u); free(p_); free(q_); free(r_); free(u_); free(v_);
  prec_free(&P);
  free(win.v);
  return converged || so.status == 4;
}

/* ------------------------------------------------------------------ */
/* Stationary iterations (Src/Solver/Linear/Iterative)                 */
/* ------------------------------------------------------------------ */

/* Jacobi::solve (jacobi.cpp:10-75): x = ci (r + c x) with the residual of
 * the previous sweep, then r = b - A x; the measure is sqrt(r.r) (res and
 * res0 in st are square roots). */
int orc_jacobi(const orc_mat *A, const double *ci, double *x, const double *b, int mini,
               int maxit, double res_rat, double res_tol, orc_stats *st, double *hist) {
  const size_t N = (size_t)A->nx * A->ny * A->nz;
  double *r = calloc(N, sizeof(double));
  orc_resid(A, x, b, r);
  double res = orc_dot(N, r, r);
  const double res0 = res;
  orc_stats so = {0, 0, 0, sqrt(res0), sqrt(res), 0};
  if (sqrt(res) < res_tol) {
    so.converged = 1; so.status = 4;
    if (st) *st = so;
    free(r);
    return 1;
  }
  int converged = 0, i, broke = 0;
  so.status = 1;
  for (i = 0; i < maxit; ++i) {
    for (size_t c = 0; c < N; ++c) x[c] = ci[c] * (r[c] + A->c[c] * x[c]);
    orc_resid(A, x, b, r);
    res = orc_dot(N, r, r);
    if (hist) hist[i] = sqrt(res);
    if (sqrt(res) < res_tol && i >= mini - 1) { converged = 1; broke = 1; so.status = 0; break; }
    if (sqrt(res) < sqrt(res0) * res_rat && i >= mini - 1) {
      converged = 1; broke = 1; so.status = 0; break;
    }
  }
  so.converged = converged;
  so.iterations = broke ? i + 1 : maxit;
  so.printed = i + 1;
  so.res = sqrt(res);
  if (st) *st = so;
  free(r);
  return converged;
}

/* GaussSeidel::solve (gaussseidel.cpp:10-117): in-place sweeps in i, j, k
 * order, x = ci (b + w xw + e xe + s xs + n xn + b xb + t xt) summed left to
 * right, then r = b - A x; the measure is sqrt(dot_voldiv_avg(r, r)) / scale
 * and the stale window starts with every entry unreal (:28-33). */
int orc_gauss_seidel(const orc_mat *A, const double *ci, double *x, const double *b, int mini,
                     int maxit, double res_rat, double res_tol, double scale, int stalecount,
                     double dV, orc_stats *st, double *hist) {
  const int nx = A->nx, ny = A->ny, nz = A->nz;
  const size_t N = (size_t)nx * ny * nz, SI = (size_t)ny * nz, SJ = (size_t)nz;
  double *r = calloc(N, sizeof(double));
  orc_resid(A, x, b, r);
  double res = sqrt(orc_dot_voldiv_avg(N, r, r, dV)) / scale;
  const double res0 = res;
  stale_win win;
  stale_init(&win, stalecount, res);
  for (int q = 0; q < win.n; ++q) win.v[q] = 1.0e24; /* boil::unreal, no res0 */
  orc_stats so = {0, 0, 0, res0, res, 0};
  if (res < res_tol) {
    so.converged = 1; so.status = 4;
    if (st) *st = so;
    free(r); free(win.v);
    return 1;
  }
  int converged = 0, it, broke = 0;
  so.status = 1;
  /* the halo is filled by the exchange before each sweep (:12, :53): on a
   * periodic face it holds the other end's value from before the sweep */
  double *xh = calloc(N, sizeof(double));
  for (it = 0; it < maxit; ++it) {
    memcpy(xh, x, N * sizeof(double));
    for (int i = 0; i < nx; ++i)
      for (int j = 0; j < ny; ++j)
        for (int k = 0; k < nz; ++k) {
          const size_t p = ((size_t)i * ny + j) * nz + k;
          double v = b[p];
          v += A->w[p] * (i > 0 ? x[p - SI] : halo(A, xh, i - 1, j, k));
          v += A->e[p] * (i < nx - 1 ? x[p + SI] : halo(A, xh, i + 1, j, k));
          v += A->s[p] * (j > 0 ? x[p - SJ] : halo(A, xh, i, j - 1, k));
          v += A->n[p] * (j < ny - 1 ? x[p + SJ] : halo(A, xh, i, j + 1, k));
          v += A->b[p] * (k > 0 ? x[p - 1] : halo(A, xh, i, j, k - 1));
          v += A->t[p] * (k < nz - 1 ? x[p + 1] : halo(A, xh, i, j, k + 1));
          x[p] = ci[p] * v;
        }
    orc_resid(A, x, b, r);
    res = sqrt(orc_dot_voldiv_avg(N, r, r, dV)) / scale;
    if (hist) hist[it] = res;
    if (res < res_tol && it >= mini - 1) { converged = 1; broke = 1; so.status = 0; break; }
    if (res < res0 * res_rat && it >= mini - 1) { converged = 1; broke = 1; so.status = 0; break; }
    if (stale_step(&win, res)) { broke = 1; so.status = 2; break; }
  }
  so.converged = converged;
  so.iterations = broke ? it + 1 : maxit;
  so.printed = it + 1;
  so.res = res;
  if (st) *st = so;
  free(r); free(win.v); free(xh);
  return converged;
}

/* ------------------------------------------------------------------ */
/* Additive-correction multigrid                                       */
/* ------------------------------------------------------------------ */

typedef struct {
  int nx, ny, nz;     /* interior cells of this level                 */
  int CI, CJ, CK;     /* ratio to the finer level (level 0: 1,1,1)    */
  double dV;          /* cell volume (uniform)                        */
  orc_mat A;
  double *phi, *fnew; /* level unknown and rhs                        */
  uint8_t *aflag;
} orc_level;

struct orc_ac {
  int nlevels;
  orc_level L[64];
  double *fold;       /* last "good" fine solution                    */
  double *res;        /* fine residual scratch                        */
  /* cycle parameters (additive.cpp:11-19) */
  double resrat_val, restol_val;
  /* the smoother of every level (the Centered object's Linear): 0 CG,
   * 1 BiCGS, 2 CGS (with prec), 3 Jacobi, 4 Gauss-Seidel; ci0 level 0's
   * stored ci (coarse levels: 1/c) */
  int sm_kind, sm_prec;
  const double *ci0;
  /* AC's own solver (AC(cen, sol), additive.cpp:41-45) for call_solver:
   * sol_kind -1 = the levels' solver */
  int sol_kind, sol_prec;
  int use_linf;       /* AC::use_linf_error (additive.h:141) */
  int flex_capped;    /* the last flex cycle hit its visit bound */
  long long flex_cap; /* smoother calls per flex cycle at most */
};

/* Domain::factor (domain_factor.cpp:4-21): first factor = smallest prime */
static int first_factor(int n) {
  int m = n - 1;
  for (;;) {
    if (m <= 0) return n;
    if (n % m == 0) return n / m;
    m--;
    if (m == 0) return n;
    if (m == 1) return n;
  }
}

static void alloc_level(orc_level *lv) {
  size_t N = (size_t)lv->nx * lv->ny * lv->nz;
  double **arr[7] = {&lv->A.c, &lv->A.w, &lv->A.e, &lv->A.s, &lv->A.n, &lv->A.b, &lv->A.t};
  for (int q = 0; q < 7; ++q) *arr[q] = calloc(N, sizeof(double));
  lv->phi = calloc(N, sizeof(double));
  lv->fnew = calloc(N, sizeof(double));
  lv->aflag = calloc(N, 1);
  lv->A.nx = lv->nx; lv->A.ny = lv->ny; lv->A.nz = lv->nz;
  lv->A.per = 0;
}

/* additive.cpp:8-48 + domain_coarsen.cpp:6-112 + additive_coarsen_flag.cpp */
orc_ac *orc_ac_create(const orc_mat *A, const uint8_t *aflag, double h) {
  orc_ac *ac = calloc(1, sizeof(orc_ac));
  ac->resrat_val = 1.0e-18; /* boil::atto */
  ac->restol_val = 1.0e-18;
  ac->sol_kind = -1;
  ac->flex_cap = 1000000;
  orc_level *L0 = &ac->L[0];
  L0->nx = A->nx; L0->ny = A->ny; L0->nz = A->nz;
  L0->CI = L0->CJ = L0->CK = 1;
  alloc_level(L0);
  L0->A.per = A->per;
  size_t N0 = (size_t)A->nx * A->ny * A->nz;
  memcpy(L0->A.c, A->c, N0 * 8); memcpy(L0->A.w, A->w, N0 * 8);
  memcpy(L0->A.e, A->e, N0 * 8); memcpy(L0->A.s, A->s, N0 * 8);
  memcpy(L0->A.n, A->n, N0 * 8); memcpy(L0->A.b, A->b, N0 * 8);
  memcpy(L0->A.t, A->t, N0 * 8);
  memcpy(L0->aflag, aflag, N0);
  const int dummy_z = (A->nz == 1);
  double hx = h, hy = h, hz = h;
  L0->dV = hx * hy * hz;
  ac->fold = calloc(N0, sizeof(double));
  ac->res = calloc(N0, sizeof(double));
  int l = 1;
  for (; l < 64; ++l) {
    orc_level *f = &ac->L[l - 1];
    int n[3] = {f->nx, f->ny, f->nz};
    int fac[3] = {2, 2, 2}, ok[3];
    for (int d = 0; d < 3; ++d) {
      if (!(d == 2 && dummy_z)) fac[d] = first_factor(n[d]);
      ok[d] = !((n[d] % fac[d]) != 0 || (n[d] + 6) <= 10 || n[d] == fac[d]);
    }
    if (!ok[0] && !ok[1] && !ok[2]) break;
    orc_level *c = &ac->L[l];
    c->CI = ok[0] ? fac[0] : 1; c->CJ = ok[1] ? fac[1] : 1; c->CK = ok[2] ? fac[2] : 1;
    c->nx = n[0] / c->CI; c->ny = n[1] / c->CJ; c->nz = n[2] / c->CK;
    hx *= c->CI; hy *= c->CJ; hz *= c->CK;
    c->dV = hx * hy * hz;
    alloc_level(c);
    c->A.per = A->per; /* coarse Scalars keep the boundary conditions */
    /* OR of the fine active flags (additive_coarsen_flag.cpp:20-38) */
    const int nyf = f->ny, nzf = f->nz;
    for (int I = 0; I < c->nx; ++I)
      for (int J = 0; J < c->ny; ++J)
        for (int K = 0; K < c->nz; ++K) {
          uint8_t v = 0;
          for (int i = 0; i < c->CI; ++i)
            for (int j = 0; j < c->CJ; ++j)
              for (int k = 0; k < c->CK; ++k)
                v |= f->aflag[((size_t)(I * c->CI + i) * nyf + (J * c->CJ + j)) * nzf + (K * c->CK + k)];
          c->aflag[((size_t)I * c->ny + J) * c->nz + K] = v;
        }
  }
  ac->nlevels = l;
  return ac;
}

void orc_ac_destroy(orc_ac *ac) {
  if (!ac) return;
  for (int l = 0; l < ac->nlevels; ++l) {
    orc_level *lv = &ac->L[l];
    free(lv->A.c); free(lv->A.w); free(lv->A.e); free(lv->A.s);
    free(lv->A.n); free(lv->A.b); free(lv->A.t);
    free(lv->phi); free(lv->fnew); free(lv->aflag);
  }
  free(ac->fold); free(ac->res);
  free(ac);
}

int orc_ac_nlevels(const orc_ac *ac) { return ac->nlevels; }

void orc_ac_level_dims(const orc_ac *ac, int l, int *dims) {
  dims[0] = ac->L[l].nx; dims[1] = ac->L[l].ny; dims[2] = ac->L[l].nz;
}

void orc_ac_level_matrix(const orc_ac *ac, int l, double *out7) {
  const orc_level *lv = &ac->L[l];
  size_t N = (size_t)lv->nx * lv->ny * lv->nz;
  const double *arr[7] = {lv->A.c, lv->A.w, lv->A.e, lv->A.s, lv->A.n, lv->A.b, lv->A.t};
  for (int q = 0; q < 7; ++q) memcpy(out7 + q * N, arr[q], N * 8);
}

/* additive_coarsen_system.cpp:4-140 (h fine, H coarse) */
static void coarsen_system(const orc_level *h, orc_level *H) {
  const int CI = H->CI, CJ = H->CJ, CK = H->CK;
  const int nyf = h->ny, nzf = h->nz;
#define F(arr, i, j, k) h->A.arr[((size_t)(i) * nyf + (size_t)(j)) * nzf + (size_t)(k)]
  for (int I = 0; I < H->nx; ++I)
    for (int J = 0; J < H->ny; ++J)
      for (int K = 0; K < H->nz; ++K) {
        size_t P = ((size_t)I * H->ny + J) * H->nz + K;
        int i0 = I * CI, j0 = J * CJ, k0 = K * CK;
        double c = 0.0;
        for (int i = 0; i < CI; ++i)
          for (int j = 0; j < CJ; ++j)
            for (int k = 0; k < CK; ++k) c += F(c, i0 + i, j0 + j, k0 + k);
        for (int j = 0; j < CJ; ++j)
          for (int k = 0; k < CK; ++k) {
            for (int i = 0; i < CI - 1; ++i) c -= F(e, i0 + i, j0 + j, k0 + k);
            for (int i = 1; i < CI; ++i) c -= F(w, i0 + i, j0 + j, k0 + k);
          }
        double e = 0.0, w = 0.0;
        for (int j = 0; j < CJ; ++j)
          for (int k = 0; k < CK; ++k) {
            e += F(e, i0 + CI - 1, j0 + j, k0 + k);
            w += F(w, i0, j0 + j, k0 + k);
          }
        for (int i = 0; i < CI; ++i)
          for (int k = 0; k < CK; ++k) {
            for (int j = 0; j < CJ - 1; ++j) c -= F(n, i0 + i, j0 + j, k0 + k);
            for (int j = 1; j < CJ; ++j) c -= F(s, i0 + i, j0 + j, k0 + k);
          }
        double n = 0.0, s = 0.0;
        for (int i = 0; i < CI; ++i)
          for (int k = 0; k < CK; ++k) {
            n += F(n, i0 + i, j0 + CJ - 1, k0 + k);
            s += F(s, i0 + i, j0, k0 + k);
          }
        for (int i = 0; i < CI; ++i)
          for (int j = 0; j < CJ; ++j) {
            for (int k = 0; k < CK - 1; ++k) c -= F(t, i0 + i, j0 + j, k0 + k);
            for (int k = 1; k < CK; ++k) c -= F(b, i0 + i, j0 + j, k0 + k);
          }
        double t = 0.0, b = 0.0;
        for (int i = 0; i < CI; ++i)
          for (int j = 0; j < CJ; ++j) {
            t += F(t, i0 + i, j0 + j, k0 + CK - 1);
            b += F(b, i0 + i, j0 + j, k0);
          }
        H->A.c[P] = c; H->A.e[P] = e; H->A.w[P] = w; H->A.n[P] = n;
        H->A.s[P] = s; H->A.t[P] = t; H->A.b[P] = b;
      }
#undef F
}

void orc_ac_coarsen_all(orc_ac *ac) {
  for (int l = 1; l < ac->nlevels; ++l) coarsen_system(&ac->L[l - 1], &ac->L[l]);
}

/* additive_restriction.cpp:12-177 */
static void restriction(const orc_level *h, orc_level *H) {
  const int CI = H->CI, CJ = H->CJ, CK = H->CK;
  const int nxf = h->nx, nyf = h->ny, nzf = h->nz;
  double *D = malloc(sizeof(double) * CI * CJ * CK);
#define FI(i, j, k) (((size_t)(i) * nyf + (size_t)(j)) * nzf + (size_t)(k))
#define PHI(i, j, k) halo(&h->A, h->phi, (i), (j), (k))
#define DD(i, j, k) D[((i) * CJ + (j)) * CK + (k)]
  for (int I = 0; I < H->nx; ++I)
    for (int J = 0; J < H->ny; ++J)
      for (int K = 0; K < H->nz; ++K) {
        size_t P = ((size_t)I * H->ny + J) * H->nz + K;
        int i0 = I * CI, j0 = J * CJ, k0 = K * CK;
        double f = 0.0;
        for (int i = 0; i < CI; ++i)
          for (int j = 0; j < CJ; ++j)
            for (int k = 0; k < CK; ++k) {
              DD(i, j, k) = h->A.c[FI(i0 + i, j0 + j, k0 + k)];
              f += h->fnew[FI(i0 + i, j0 + j, k0 + k)];
            }
        for (int j = 0; j < CJ; ++j)
          for (int k = 0; k < CK; ++k) {
            f += h->A.e[FI(i0 + CI - 1, j0 + j, k0 + k)] * PHI(i0 + CI, j0 + j, k0 + k);
            f += h->A.w[FI(i0, j0 + j, k0 + k)] * PHI(i0 - 1, j0 + j, k0 + k);
            for (int i = 0; i < CI - 1; ++i) DD(i, j, k) -= h->A.e[FI(i0 + i, j0 + j, k0 + k)];
            for (int i = CI - 1; i > 0; --i) DD(i, j, k) -= h->A.w[FI(i0 + i, j0 + j, k0 + k)];
          }
        for (int i = 0; i < CI; ++i)
          for (int k = 0; k < CK; ++k) {
            f += h->A.n[FI(i0 + i, j0 + CJ - 1, k0 + k)] * PHI(i0 + i, j0 + CJ, k0 + k);
            f += h->A.s[FI(i0 + i, j0, k0 + k)] * PHI(i0 + i, j0 - 1, k0 + k);
            for (int j = 0; j < CJ - 1; ++j) DD(i, j, k) -= h->A.n[FI(i0 + i, j0 + j, k0 + k)];
            for (int j = CJ - 1; j > 0; --j) DD(i, j, k) -= h->A.s[FI(i0 + i, j0 + j, k0 + k)];
          }
        for (int i = 0; i < CI; ++i)
          for (int j = 0; j < CJ; ++j) {
            f += h->A.t[FI(i0 + i, j0 + j, k0 + CK - 1)] * PHI(i0 + i, j0 + j, k0 + CK);
            f += h->A.b[FI(i0 + i, j0 + j, k0)] * PHI(i0 + i, j0 + j, k0 - 1);
            for (int k = 0; k < CK - 1; ++k) DD(i, j, k) -= h->A.t[FI(i0 + i, j0 + j, k0 + k)];
            for (int k = CK - 1; k > 0; --k) DD(i, j, k) -= h->A.b[FI(i0 + i, j0 + j, k0 + k)];
          }
        for (int i = 0; i < CI; ++i)
          for (int j = 0; j < CJ; ++j)
            for (int k = 0; k < CK; ++k) f -= DD(i, j, k) * h->phi[FI(i0 + i, j0 + j, k0 + k)];
        H->fnew[P] = f;
      }
#undef FI
#undef PHI
#undef DD
  free(D);
  const size_t NH = (size_t)H->nx * H->ny * H->nz;
  for (size_t P = 0; P < NH; ++P)
    if (!H->aflag[P]) H->fnew[P] = 0.0;
  /* zero-mean normalisation over active coarse cells (:151-174) */
  double sum = 0.0;
  int ncell = 0;
  for (size_t P = 0; P < NH; ++P)
    if (H->aflag[P]) { sum += H->fnew[P]; ncell++; }
  sum /= (double)ncell;
  for (size_t P = 0; P < NH; ++P)
    if (H->aflag[P]) H->fnew[P] -= sum;
}

/* additive_interpolation.cpp:12-64 (H coarse -> h fine) */
static void interpolation(const orc_level *H, orc_level *h) {
  const int CI = H->CI, CJ = H->CJ, CK = H->CK;
  const int nyf = h->ny, nzf = h->nz;
  for (int I = 0; I < H->nx; ++I)
    for (int J = 0; J < H->ny; ++J)
      for (int K = 0; K < H->nz; ++K) {
        double v = H->phi[((size_t)I * H->ny + J) * H->nz + K];
        for (int i = 0; i < CI; ++i)
          for (int j = 0; j < CJ; ++j)
            for (int k = 0; k < CK; ++k)
              h->phi[((size_t)(I * CI + i) * nyf + (J * CJ + j)) * nzf + (K * CK + k)] += v;
      }
}

/* additive_residual.cpp:4-30 with dt = 1 */
static double residual(orc_ac *ac, double *linf) {
  orc_level *h = &ac->L[0];
  size_t N = (size_t)h->nx * h->ny * h->nz;
  orc_resid(&h->A, h->phi, h->fnew, ac->res);
  double r2 = sqrt(orc_dot_voldiv_avg(N, ac->res, ac->res, h->dV)) * 1.0;
  if (linf) *linf = orc_max_abs_voldiv(N, ac->res, h->dV) * 1.0;
  return r2;
}

/* call_smoother / call_solver (additive_cycle_functions.cpp:90-107): the
 * level's Linear solver (CG unless set) with scale dti*scale = 1 */
/* call_smoother (as_solver 0, the level's Linear) and call_solver
 * (as_solver 1, AC's own solver); returns the solver's converged flag */
static int smooth_as(orc_ac *ac, int l, int mi, double res_rat, double res_tol, int ms, int as_solver) {
  orc_level *lv = &ac->L[l];
  const int use_sol = as_solver && ac->sol_kind >= 0;
  const int k = use_sol ? ac->sol_kind : ac->sm_kind;
  const int prec = use_sol ? ac->sol_prec : ac->sm_prec;
  int ok;
  if (k == 1) {
    ok = orc_bicgs_prec(&lv->A, lv->phi, lv->fnew, 1, mi, res_rat, res_tol, 1.0, ms, lv->dV, NULL, NULL,
                        prec);
  } else if (k == 2) {
    ok = orc_cgs_prec(&lv->A, lv->phi, lv->fnew, 1, mi, res_rat, res_tol, 1.0, ms, lv->dV, NULL, NULL,
                      prec);
  } else if (k == 3 || k == 4) {
    /* coarse levels: ci = 1/c (additive_coarsen_system.cpp) */
    const size_t N = (size_t)lv->A.nx * lv->A.ny * lv->A.nz;
    double *ci = NULL;
    if (l > 0 || !ac->ci0) {
      ci = malloc(N * sizeof(double));
      for (size_t c = 0; c < N; ++c) ci[c] = 1.0 / lv->A.c[c];
    }
    const double *cv = ci ? ci : ac->ci0;
    if (k == 3) ok = orc_jacobi(&lv->A, cv, lv->phi, lv->fnew, 1, mi, res_rat, res_tol, NULL, NULL);
    else ok = orc_gauss_seidel(&lv->A, cv, lv->phi, lv->fnew, 1, mi, res_rat, res_tol, 1.0, ms, lv->dV,
                               NULL, NULL);
    free(ci);
  } else {
    ok = orc_cg_prec(&lv->A, lv->phi, lv->fnew, 1, mi, res_rat, res_tol, 1.0, ms, lv->dV, NULL, NULL,
                     prec);
  }
  return ok;
}

static void smooth(orc_ac *ac, int l, int mi, double res_rat, double res_tol, int ms) {
  smooth_as(ac, l, mi, res_rat, res_tol, ms, 0);
}

/* call_solver */
static void solve_l(orc_ac *ac, int l, int mi, double res_rat, double res_tol, int ms) {
  smooth_as(ac, l, mi, res_rat, res_tol, ms, 1);
}

void orc_ac_set_smoother(orc_ac *ac, int kind, int prec, const double *ci0) {
  ac->sm_kind = kind;
  ac->sm_prec = prec;
  ac->ci0 = ci0;
}

int orc_ac_flex_capped(const orc_ac *ac) { return ac->flex_capped; }
void orc_ac_set_flex_cap(orc_ac *ac, long long cap) { ac->flex_cap = cap; }

void orc_ac_set_params(orc_ac *ac, double resrat_val, double restol_val, int use_linf,
                       int sol_kind, int sol_prec) {
  ac->resrat_val = resrat_val;
  ac->restol_val = restol_val;
  ac->use_linf = use_linf;
  ac->sol_kind = sol_kind;
  ac->sol_prec = sol_prec;
}

static void v_cycle(orc_ac *ac, int l, const int mv[3], const int ms[3]);

/* additive_recursive.cpp:4-34 */
static void v_cycle(orc_ac *ac, int l, const int mv[3], const int ms[3]) {
  if (l != ac->nlevels - 1) {
    smooth(ac, l, mv[0], ac->resrat_val, ac->restol_val, ms[0]);
    restriction(&ac->L[l], &ac->L[l + 1]);
    v_cycle(ac, l + 1, mv, ms);
    solve_l(ac, l, mv[2], ac->resrat_val, ac->restol_val, ms[2]);
    if (l > 0) interpolation(&ac->L[l], &ac->L[l - 1]);
  } else {
    solve_l(ac, l, 100, -1.0, ac->restol_val, -1);
    if (l > 0) interpolation(&ac->L[l], &ac->L[l - 1]);
  }
}

/* additive_recursive.cpp:37-76 (f) and 79-118 (w) */
static void fw_cycle(orc_ac *ac, int l, const int mv[3], const int ms[3], int w) {
  if (l != ac->nlevels - 1) {
    smooth(ac, l, mv[0], ac->resrat_val, ac->restol_val, ms[0]);
    restriction(&ac->L[l], &ac->L[l + 1]);
    fw_cycle(ac, l + 1, mv, ms, w);
    smooth(ac, l, mv[1], ac->resrat_val, ac->restol_val, ms[1]);
    restriction(&ac->L[l], &ac->L[l + 1]);
    if (w) fw_cycle(ac, l + 1, mv, ms, w);
    else v_cycle(ac, l + 1, mv, ms);
    solve_l(ac, l, mv[2], ac->resrat_val, ac->restol_val, ms[2]);
    if (l > 0) interpolation(&ac->L[l], &ac->L[l - 1]);
  } else {
    solve_l(ac, l, 100, -1.0, ac->restol_val, -1);
    if (l > 0) interpolation(&ac->L[l], &ac->L[l - 1]);
  }
}

/* additive_recursive.cpp:161-197, the recursion unrolled into a loop over
 * (level, sign): a level whose smoother converges hands its correction up
 * (Sign::pos on the finer level: mv[2], ms[2]); one that does not restricts
 * down (Sign::neg: mv[0], ms[0]); the coarsest level is solved and
 * interpolated up with Sign::neg. It starts at level l and ends when level
 * 0's smoother converges.
 * The reference recurses without a bound and never returns when level 0
 * never converges (AC::resrat at its default atto, for instance); here at
 * most flex_cap smoother calls (10^6 unless set) are made, after which the
 * cycle ends and flex_capped is set. */
static void flex_cycle(orc_ac *ac, int l, const int mv[3], const int ms[3]) {
  const int last = ac->nlevels - 1;
  long long visits = 0, cap = ac->flex_cap;
  int pos = 0;
  ac->flex_capped = 0;
  for (;;) {
    if (l != last) {
      const int idx = pos ? 2 : 0;
      if (++visits > cap) { ac->flex_capped = 1; return; }
      if (smooth_as(ac, l, mv[idx], ac->resrat_val, ac->restol_val, ms[idx], 0)) {
        if (l == 0) return;
        interpolation(&ac->L[l], &ac->L[l - 1]);
        l -= 1;
        pos = 1;
      } else {
        restriction(&ac->L[l], &ac->L[l + 1]);
        l += 1;
        pos = 0;
      }
    } else {
      solve_l(ac, l, 100, -1.0, ac->restol_val, -1);
      if (l == 0) return;
      interpolation(&ac->L[l], &ac->L[l - 1]);
      l -= 1;
      pos = 0;
    }
  }
}

static void run_cycle(orc_ac *ac, int kind, int l, const int mv[3], const int ms[3]) {
  if (kind == 1) v_cycle(ac, l, mv, ms);
  else if (kind == 2) fw_cycle(ac, l, mv, ms, 0);
  else if (kind == 4) fw_cycle(ac, l, mv, ms, 1);
  else if (kind == 5) flex_cycle(ac, l, mv, ms);
  else solve_l(ac, l, 100, -1.0, ac->restol_val, -1); /* full_cycle's "shouldn't happen" branch */
}

/* additive_recursive.cpp:121-158 */
static void full_cycle(orc_ac *ac, int l, int kind, const int mv[3], const int ms[3]) {
  if (l != ac->nlevels - 1) {
    restriction(&ac->L[l], &ac->L[l + 1]);
    full_cycle(ac, l + 1, kind, mv, ms);
    run_cycle(ac, kind, l, mv, ms);
  } else {
    solve_l(ac, l, 100, -1.0, ac->restol_val, -1);
    if (l > 0) interpolation(&ac->L[l], &ac->L[l - 1]);
  }
}

/* AC::cycle (additive_cycle.cpp:4-99), init_cycles and converged
 * (additive_cycle_functions.cpp:12-87). loop 1 V, 2 F, 4 W, 5 flex; any
 * other loop value is the "just solve" branch (:66-71): one call of AC's
 * solver on level 0 (MaxIter 40, ResRat 0.001, ResTol femto), then the
 * loop ends and the cycle reports max_cyc cycles, not converged. With
 * use_linf the tests read the max-norm residual instead: against the
 * initial one for the ratio, and for the divergence check against the
 * value before the loop, which the reference never refreshes (its
 * `reslinf_m1 = reslinf_m1`, additive_cycle.cpp:78). */
int orc_ac_cycle(orc_ac *ac, double *x, const double *b, int init, int loop,
                 double toler, double factor, const int mv[3], const int ms[3],
                 int max_cyc, int min_cyc, int stop_if_div, int priority_min_cyc,
                 int *ncyc, double *res_hist, int *nhist) {
  orc_level *L0 = &ac->L[0];
  const size_t N0 = (size_t)L0->nx * L0->ny * L0->nz;
  int nh = 0;
  memcpy(L0->phi, x, N0 * 8);
  memcpy(L0->fnew, b, N0 * 8);
  orc_ac_coarsen_all(ac);
  double linf_0;
  double res_0 = residual(ac, &linf_0);
  if (res_hist) res_hist[nh] = res_0;
  nh++;
  memcpy(ac->fold, L0->phi, N0 * 8);
  int ret = 0, nc = 0;
  const double res_0_control = ac->use_linf ? linf_0 : res_0;
  if ((res_0_control < toler && min_cyc == 0) || res_0 == 0.0) {
    ret = 1; nc = 0;
    goto out;
  }
  for (int l = 1; l < ac->nlevels; ++l) {
    size_t N = (size_t)ac->L[l].nx * ac->L[l].ny * ac->L[l].nz;
    memset(ac->L[l].phi, 0, N * 8);
    memset(ac->L[l].fnew, 0, N * 8);
  }
  double res_m1, linf_m1;
  if (init != -1) {
    full_cycle(ac, 0, init, mv, ms);
    res_m1 = residual(ac, &linf_m1);
    if (res_hist) res_hist[nh] = res_m1;  /* the reference logs "Cycle 0" */
    nh++;
    /* converged(..., cycle 0, ...) (:39-43): its return value is dropped,
     * but its divergence branch runs. It compares the residual with itself
     * (res0 is res_m1, the same state), so unless cycle 0 already meets the
     * tolerance, stop_if_div restores phi = fold, the initial guess
     * (additive_cycle_functions.cpp:67-83). */
    const double rc = ac->use_linf ? linf_m1 : res_m1;
    const double rbc = ac->use_linf ? linf_0 : res_0;
    if (!(0 >= min_cyc && (rc / rbc < factor || rc < toler))) {
      int check = stop_if_div;
      if (priority_min_cyc && 0 < min_cyc) check = 0;
      if (check) memcpy(L0->phi, ac->fold, N0 * 8);
    }
  } else {
    res_m1 = residual(ac, &linf_m1);
  }
  nc = max_cyc;
  for (int c = 1; c <= max_cyc; ++c) {
    if (loop != 1 && loop != 2 && loop != 4 && loop != 5) {
      /* just solve */
      solve_l(ac, 0, 40, 0.001, 1.0e-15, -1);
      break;
    }
    run_cycle(ac, loop, 0, mv, ms);
    double linf1;
    double res1 = residual(ac, &linf1);
    if (res_hist) res_hist[nh] = res1;
    nh++;
    const double rc = ac->use_linf ? linf1 : res1;
    const double r0c = ac->use_linf ? linf_m1 : res_m1;
    const double rbc = ac->use_linf ? linf_0 : res_0;
    int con;
    if (c >= min_cyc && (rc / rbc < factor || rc < toler)) {
      con = 0;
    } else {
      int check = stop_if_div;
      if (priority_min_cyc && c < min_cyc) check = 0;
      if (check && rc >= r0c) {
        memcpy(L0->phi, ac->fold, N0 * 8);
        con = 1;
      } else {
        con = 2;
      }
    }
    res_m1 = res1;  /* linf_m1 stays (the reference's self-assignment) */
    if (con == 0) { ret = 1; nc = c; goto out; }
    if (con == 1) { ret = 0; nc = c; goto out; }
    memcpy(ac->fold, L0->phi, N0 * 8);
  }
  ret = 0;
out:
  memcpy(x, L0->phi, N0 * 8);
  if (ncyc) *ncyc = nc;
  if (nhist) *nhist = nh;
  return ret;
}
