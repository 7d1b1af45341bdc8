// Exact-order FP64 summation in parallel.
//
// The reference adds a dot product's terms one after another in i,j,k order
// with round-to-nearest after every addition (`for_ijk sum += ...`,
// Src/Field/Scalar/scalar.h:296-326). The reference-parity solvers reproduce
// that sum to the bit. A single thread adding 16.7 M terms takes tens of
// milliseconds per dot product, so the sum is computed like this instead.
//
// Binade argument. Let s be the running sum, 2^e <= |s| < 2^(e+1), and
// u = 2^(e-52) its ulp. While the running sum stays inside that binade every
// partial sum is an integer multiple of u, and
//     fl(s + a) = s + u * rint(a / u)       (round half to even),
// unless a/u is exactly half-way between two integers (a tie, whose
// direction depends on the parity of s/u). So over a stretch of terms that
// keeps the sum in one binade and holds no tie, the sequential sum is s plus
// u times an integer sum, which any order computes exactly.
//
// Per chunk of kThreads terms (one block of the reducing kernel):
//   1. the terms are stored (for the chunks that need a sequential pass);
//   2. an approximate prefix of all earlier terms comes from a decoupled
//      look-back over the chunks' published sums (bounded polling: a block
//      that gives up only loses its hint);
//   3. for the three exponents around the hint, e0..e0+2, the block computes
//      K = sum of rint(a/u) and the minimum and maximum of its running
//      integer prefix, and whether every term was tie-free and finite;
//   4. the last chunk of each group of kExactGroup chunks to arrive composes
//      the group's records for the exponents of the group's last chunk;
//   5. the last block of the launch walks the groups in order with the exact
//      running sum: a group (or chunk) whose record holds the current
//      exponent and keeps s/u + prefix inside [2^52 + 1, 2^53 - 1] is
//      applied as s += u K; anything else is added term by term.
// Every step of the walk is either the sequential rounding itself or an
// integer sum proven equal to it, so the result is the sequential sum bit
// for bit whatever the hints were; bad hints only cost time.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace pbg {

constexpr int kExactChunkThreads = 256;  // terms per chunk (the reducing block)
constexpr int kExactGroup = 64;          // chunks per group record
constexpr int kExactVals = 2;            // sums per reducing kernel at most
constexpr int kExactPoll = 4096;         // look-back polls before a block gives up its hint

// Record of one chunk or group for the exponents e0, e0+1, e0+2.
struct ExactRec {
  long long K[3], mn[3], mx[3];
  int e0;   // exponent of candidate 0
  int ok;   // bit c: candidate c usable
};

// Header stored kExactHdrBytes before the terms (the `seq` pointer).
struct ExactHdr {
  ExactRec *crec;      // [kExactVals][cap_chunks]
  ExactRec *grec;      // [kExactVals][cap_groups]
  double *agg;         // [kExactVals][cap_chunks] chunk sums (hints)
  double *incl;        // [kExactVals][cap_chunks] inclusive prefixes (hints)
  unsigned *flag;      // [cap_chunks] (gen << 2) | 1 sums published, 2 prefix published
  unsigned *gcount;    // [cap_groups] chunk arrivals per group, zero between uses
  long long cap_chunks, cap_groups;
  unsigned gen;        // launch generation of the look-back flags
  unsigned pad;
};
constexpr size_t kExactHdrBytes = 256;
static_assert(sizeof(ExactHdr) <= kExactHdrBytes, "exact-sum header");

// Doubles of a scratch buffer for terms of ncell cells (header and records
// included); the `seq` pointer handed to the kernels is exact_seq(base).
inline size_t exact_scratch_doubles(long long ncell) {
  const long long ch = (ncell + kExactChunkThreads - 1) / kExactChunkThreads + 1;
  const long long gr = (ch + kExactGroup - 1) / kExactGroup + 1;
  size_t bytes = kExactHdrBytes + sizeof(double) * (size_t)kExactVals * ncell;
  bytes += sizeof(ExactRec) * kExactVals * (size_t)(ch + gr);
  bytes += sizeof(double) * 2 * kExactVals * (size_t)ch;
  bytes += sizeof(unsigned) * (size_t)(ch + gr) + 1024;
  return (bytes + 7) / 8;
}
inline double *exact_seq(double *base) { return base + kExactHdrBytes / 8; }

__device__ __forceinline__ const ExactHdr *exact_hdr(const double *seq) {
  return reinterpret_cast<const ExactHdr *>(reinterpret_cast<const char *>(seq) - kExactHdrBytes);
}

__device__ __forceinline__ unsigned ld_volatile_u32(const unsigned *p) {
  return *reinterpret_cast<const volatile unsigned *>(p);
}

// Record load through L2 (records written by other blocks of the launch).
__device__ __forceinline__ void exact_load(ExactRec &d, const ExactRec *s) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    d.K[c] = __ldcg(&s->K[c]);
    d.mn[c] = __ldcg(&s->mn[c]);
    d.mx[c] = __ldcg(&s->mx[c]);
  }
  d.e0 = __ldcg(&s->e0);
  d.ok = __ldcg(&s->ok);
}

// Applies a record to the running sum s when it is provably the sequential
// result; returns false (s unchanged) otherwise.
__device__ __forceinline__ bool exact_apply(double &s, const ExactRec &R) {
  if (!(s != 0.0) || !isfinite(s)) return false;
  const int e = ilogb(s);
  if (e < -960 || e > 1000) return false;
  const int c = e - R.e0;
  if (c < 0 || c > 2 || !((R.ok >> c) & 1)) return false;
  const long long LO = (1LL << 52) + 1, HI = (1LL << 53) - 1;
  long long S = (long long)ldexp(fabs(s), 52 - e);  // exact, in [2^52, 2^53)
  if (s < 0.0) S = -S;
  const long long lo = S + R.mn[c], hi = S + R.mx[c];
  if (s > 0.0) {
    if (lo < LO || hi > HI) return false;
  } else {
    if (hi > -LO || lo < -HI) return false;
  }
  S += R.K[c];
  s = ldexp((double)S, e - 52);
  return true;
}

// Block-wide inclusive scan of three 64-bit integers (kExactChunkThreads
// threads); returns the block totals in tot.
__device__ __forceinline__ void exact_scan3(long long (&x)[3], long long (&tot)[3],
                                            long long (*sm)[kExactChunkThreads / 32]) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  constexpr int NW = kExactChunkThreads / 32;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      long long y = __shfl_up_sync(0xffffffffu, x[c], off);
      if (lane >= off) x[c] += y;
    }
  if (lane == 31)
#pragma unroll
    for (int c = 0; c < 3; ++c) sm[c][wid] = x[c];
  __syncthreads();
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    long long base = 0;
    for (int w = 0; w < wid; ++w) base += sm[c][w];
    long long t = 0;
    for (int w = 0; w < NW; ++w) t += sm[c][w];
    x[c] += base;
    tot[c] = t;
  }
  __syncthreads();
}

// Block-wide min and max of three 64-bit integers.
__device__ __forceinline__ void exact_minmax3(long long (&mn)[3], long long (&mx)[3],
                                              long long (*smn)[kExactChunkThreads / 32],
                                              long long (*smx)[kExactChunkThreads / 32]) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  constexpr int NW = kExactChunkThreads / 32;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      long long a = __shfl_down_sync(0xffffffffu, mn[c], off);
      long long b = __shfl_down_sync(0xffffffffu, mx[c], off);
      mn[c] = a < mn[c] ? a : mn[c];
      mx[c] = b > mx[c] ? b : mx[c];
    }
  if (lane == 0)
#pragma unroll
    for (int c = 0; c < 3; ++c) { smn[c][wid] = mn[c]; smx[c][wid] = mx[c]; }
  __syncthreads();
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    long long a = smn[c][0], b = smx[c][0];
    for (int w = 1; w < NW; ++w) {
      a = smn[c][w] < a ? smn[c][w] : a;
      b = smx[c][w] > b ? smx[c][w] : b;
    }
    mn[c] = a;
    mx[c] = b;
  }
  __syncthreads();
}

// The exact-order reduction. Launch shape: one thread per term, blocks of
// kExactChunkThreads, every thread of every block calls it. Returns true in
// thread 0 of the last block to finish, with out[q] the sequential sum of
// the v[q] in thread order.
template <int NV>
__device__ bool exact_reduce(const double (&v)[NV], double *seq, long long n, unsigned *count,
                             double (&out)[NV]) {
  static_assert(NV <= kExactVals, "exact_reduce: too many sums");
  constexpr int NW = kExactChunkThreads / 32;
  const ExactHdr *H = exact_hdr(seq);
  const long long cap = H->cap_chunks, capg = H->cap_groups;
  const unsigned gen = ld_volatile_u32(&H->gen) & 0x3fffffffu;
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  const long long b = blockIdx.x;
  const long long nch = gridDim.x;
  const long long p = b * kExactChunkThreads + t;

  __shared__ double s_agg[NV][NW];
  __shared__ double s_hint[NV];
  __shared__ long long s_a[3][NW], s_b[3][NW];
  __shared__ ExactRec s_rec;
  __shared__ bool s_last;
  __shared__ int s_cmd;
  __shared__ long long s_arg;
  __shared__ ExactRec s_buf[kExactGroup];
  __shared__ double s_terms[kExactChunkThreads];

  // 1. the terms
  double a[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    a[q] = p < n ? v[q] : 0.0;
    if (p < n) seq[q * n + p] = v[q];
  }

  // 2. chunk sums and the look-back hint
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double x = a[q];
    for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
    if (lane == 0) s_agg[q][wid] = x;
  }
  __syncthreads();
  if (wid == 0) {
    double my[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double x = 0.0;
      for (int w = 0; w < NW; ++w) x += s_agg[q][w];
      my[q] = x;
    }
    if (lane == 0) {
#pragma unroll
      for (int q = 0; q < NV; ++q) H->agg[q * cap + b] = my[q];
      __threadfence();
      atomicExch(&H->flag[b], (gen << 2) | 1u);
    }
    __syncwarp();
    double pre[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) pre[q] = 0.0;
    bool okh = true;
    long long top = b - 1;
    int polls = 0;
    while (top >= 0) {
      const long long j = top - lane;
      int st = 2;  // before the first chunk: an inclusive prefix of zero
      if (j >= 0) {
        unsigned f = ld_volatile_u32(&H->flag[j]);
        st = ((f >> 2) == gen) ? (int)(f & 3u) : 0;
      }
      const unsigned incl = __ballot_sync(0xffffffffu, st == 2);
      const unsigned notr = __ballot_sync(0xffffffffu, st == 0);
      const int fi = incl ? __ffs(incl) - 1 : 32;
      const unsigned need = fi == 32 ? 0xffffffffu : ((2u << fi) - 1u);
      if (notr & need) {
        if (++polls > kExactPoll) { okh = false; break; }
        __nanosleep(32);
        continue;
      }
      __threadfence();
#pragma unroll
      for (int q = 0; q < NV; ++q) {
        double x = 0.0;
        if (j >= 0 && lane < fi) x = __ldcg(&H->agg[q * cap + j]);
        else if (j >= 0 && lane == fi) x = __ldcg(&H->incl[q * cap + j]);
        for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
        pre[q] += __shfl_sync(0xffffffffu, x, 0);
      }
      if (fi < 32) break;
      top -= 32;
    }
    if (lane == 0) {
#pragma unroll
      for (int q = 0; q < NV; ++q) s_hint[q] = okh ? pre[q] : __longlong_as_double(0x7ff8000000000000LL);
      if (okh) {
#pragma unroll
        for (int q = 0; q < NV; ++q) H->incl[q * cap + b] = pre[q] + my[q];
        __threadfence();
        atomicExch(&H->flag[b], (gen << 2) | 2u);
      }
    }
  }
  __syncthreads();

  // 3. chunk records for the exponents around the hint
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    const double hint = s_hint[q];
    int e0 = 0;
    bool have = isfinite(hint) && hint != 0.0;
    if (have) {
      e0 = ilogb(hint) - 1;
      have = e0 >= -960 && e0 + 2 <= 1000;
    }
    if (!have) {
      if (t == 0) {
        ExactRec R;
        for (int c = 0; c < 3; ++c) R.K[c] = R.mn[c] = R.mx[c] = 0;
        R.e0 = 0;
        R.ok = 0;
        H->crec[q * cap + b] = R;
      }
      continue;  // uniform across the block
    }
    long long k[3];
    int okb = 0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double y = a[q] * ldexp(1.0, 52 - (e0 + c));
      // finite, |y| <= 2^53 and not half-way between two integers
      const bool good = isfinite(y) && fabs(y) <= 9007199254740992.0 && fabs(y - trunc(y)) != 0.5;
      k[c] = good ? __double2ll_rn(y) : 0;
      if (__syncthreads_and(good)) okb |= 1 << c;
    }
    long long tot[3];
    exact_scan3(k, tot, s_a);
    long long mn[3] = {k[0], k[1], k[2]}, mx[3] = {k[0], k[1], k[2]};
    exact_minmax3(mn, mx, s_a, s_b);
    if (t == 0) {
      ExactRec R;
      R.e0 = e0;
      R.ok = okb;
      for (int c = 0; c < 3; ++c) {
        R.K[c] = tot[c];
        R.mn[c] = mn[c];
        R.mx[c] = mx[c];
        const long long L = 1LL << 53;
        if (mn[c] <= -L || mx[c] >= L || tot[c] <= -L || tot[c] >= L) R.ok &= ~(1 << c);
      }
      H->crec[q * cap + b] = R;
    }
  }

  // 4. group records
  const long long g = b / kExactGroup;
  const long long g0 = g * kExactGroup;
  const int gsize = (int)((nch - g0) < kExactGroup ? (nch - g0) : kExactGroup);
  if (t == 0) {
    __threadfence();
    unsigned prev = atomicAdd(&H->gcount[g], 1u);
    s_last = (prev == (unsigned)gsize - 1);
  }
  __syncthreads();
  if (s_last && wid == 0) {
    __threadfence();
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      const int E0 = __ldcg(&H->crec[q * cap + g0 + gsize - 1].e0);
      long long K[3], mn[3], mx[3];
      int okm = 7;
#pragma unroll
      for (int c = 0; c < 3; ++c) { K[c] = 0; mn[c] = 0x7fffffffffffffffLL; mx[c] = -0x7fffffffffffffffLL; }
      // two chunks per lane, in order
      for (int h = 0; h < 2; ++h) {
        const int jj = 2 * lane + h;
        if (jj >= gsize) continue;
        const ExactRec *R = &H->crec[q * cap + g0 + jj];
        const int e0 = __ldcg(&R->e0), ok = __ldcg(&R->ok);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const int cc = E0 + c - e0;
          if (cc < 0 || cc > 2 || !((ok >> cc) & 1)) { okm &= ~(1 << c); continue; }
          const long long rk = __ldcg(&R->K[cc]), rn = __ldcg(&R->mn[cc]), rx = __ldcg(&R->mx[cc]);
          const long long lo = K[c] + rn, hi = K[c] + rx;
          mn[c] = lo < mn[c] ? lo : mn[c];
          mx[c] = hi > mx[c] ? hi : mx[c];
          K[c] += rk;
        }
      }
      // invalid candidates carry zeros so that the sums below stay bounded
#pragma unroll
      for (int c = 0; c < 3; ++c)
        if (!((okm >> c) & 1)) { K[c] = 0; mn[c] = 0; mx[c] = 0; }
      // exclusive scan of K over the lanes, then min/max of excl + lane range
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        long long incl = K[c];
        for (int off = 1; off < 32; off <<= 1) {
          long long y = __shfl_up_sync(0xffffffffu, incl, off);
          if (lane >= off) incl += y;
        }
        const long long excl = incl - K[c];
        long long lo = 2 * lane < gsize ? excl + mn[c] : 0x7fffffffffffffffLL;
        long long hi = 2 * lane < gsize ? excl + mx[c] : -0x7fffffffffffffffLL;
        for (int off = 16; off > 0; off >>= 1) {
          long long a2 = __shfl_down_sync(0xffffffffu, lo, off), b2 = __shfl_down_sync(0xffffffffu, hi, off);
          lo = a2 < lo ? a2 : lo;
          hi = b2 > hi ? b2 : hi;
        }
        const long long total = __shfl_sync(0xffffffffu, incl, 31);
        const bool allok = __all_sync(0xffffffffu, (2 * lane >= gsize) || ((okm >> c) & 1));
        if (lane == 0) {
          s_rec.K[c] = total;
          s_rec.mn[c] = lo;
          s_rec.mx[c] = hi;
          const long long L = 1LL << 53;
          bool good = allok && lo > -L && hi < L && total > -L && total < L;
          if (c == 0) s_rec.ok = 0;
          if (good) s_rec.ok |= 1 << c;
        }
      }
      if (lane == 0) {
        s_rec.e0 = E0;
        H->grec[q * capg + g] = s_rec;
      }
      __syncwarp();
    }
    if (lane == 0) H->gcount[g] = 0u;
  }

  // 5. the last block walks the groups
  if (t == 0) {
    __threadfence();
    unsigned prev = atomicAdd(count, 1u);
    s_last = (prev == (unsigned)nch - 1);
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
  const long long ng = (nch + kExactGroup - 1) / kExactGroup;
  double res[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double s = 0.0;   // meaningful in thread 0
    long long gi = 0;
    while (gi < ng) {
      // a batch of group records
      const int nb = (int)((ng - gi) < kExactGroup ? (ng - gi) : kExactGroup);
      if (t < nb) exact_load(s_buf[t], &H->grec[q * capg + gi + t]);
      __syncthreads();
      if (t == 0) {
        int k = 0;
        while (k < nb && exact_apply(s, s_buf[k])) ++k;
        s_cmd = k;
      }
      __syncthreads();
      const int k = s_cmd;
      __syncthreads();
      gi += k;
      if (k == nb) continue;
      // group gi needs its chunk records
      const long long c0 = gi * kExactGroup;
      const int cs = (int)((nch - c0) < kExactGroup ? (nch - c0) : kExactGroup);
      if (t < cs) exact_load(s_buf[t], &H->crec[q * cap + c0 + t]);
      __syncthreads();
      int ci = 0;
      while (ci < cs) {
        if (t == 0) {
          int m = ci;
          while (m < cs && exact_apply(s, s_buf[m])) ++m;
          s_cmd = m;
        }
        __syncthreads();
        const int m = s_cmd;
        __syncthreads();
        ci = m;
        if (ci >= cs) break;
        // chunk c0 + ci term by term
        const long long e0 = (c0 + ci) * kExactChunkThreads;
        const int len = (int)((n - e0) < kExactChunkThreads ? (n - e0) : kExactChunkThreads);
        if (t < len) s_terms[t] = __ldcg(&seq[q * n + e0 + t]);
        __syncthreads();
        if (t == 0)
          for (int e = 0; e < len; ++e) s = __dadd_rn(s, s_terms[e]);
        __syncthreads();
        ++ci;
      }
      ++gi;
    }
    res[q] = s;
  }
  if (t != 0) return false;
#pragma unroll
  for (int q = 0; q < NV; ++q) out[q] = res[q];
  ExactHdr *Hw = const_cast<ExactHdr *>(H);
  const unsigned nxt = (gen + 1u) & 0x3fffffffu;
  Hw->gen = nxt ? nxt : 1u;  // generation 0 is the zeroed flags' value
  *count = 0u;
  __threadfence();
  return true;
}

}  // namespace pbg
