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
//   3. for the three exponents around the hint, e0..e0+2, each warp computes
//      K = sum of rint(a/u) over its 32 terms, the minimum and maximum of its
//      running integer prefix, and whether every term was tie-free and
//      finite; the chunk's record composes its warps' records;
//   4. the last chunk of each group of kExactGroup chunks to arrive composes
//      the group's records for the exponents of the group's last chunk;
//   5. the last block of the launch walks the groups in order with the exact
//      running sum (one warp per sum): a group, chunk or warp record that
//      holds the current exponent and keeps s/u + prefix inside
//      [2^52 + 1, 2^53 - 1] is applied as s += u K; a warp segment whose
//      record does not is added term by term.
// Every step of the walk is either the sequential rounding itself or an
// integer sum proven equal to it, so the result is the sequential sum bit
// for bit whatever the hints were; bad hints only cost time.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace pbg {

constexpr int kExactChunkThreads = 256;  // terms per chunk (the reducing block)
constexpr int kExactWarps = kExactChunkThreads / 32;  // warp records per chunk
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
  ExactRec *wrec;      // [kExactVals][cap_chunks][kExactWarps] (32 terms each)
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
  bytes += sizeof(ExactRec) * kExactVals * (size_t)(ch * (kExactWarps + 1) + gr);
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

// Running sum of the walk. While `in` holds, s = S * 2^(e-52) with |S| in
// [2^52, 2^53): the record applications keep it there, so s is formed only
// when a chunk is added term by term, or at the end.
struct ExactWalk {
  double s;
  long long S;
  int e;
  bool in;
};

__device__ __forceinline__ bool exact_walk_apply(ExactWalk &w, const ExactRec &R) {
  if (!w.in) {
    if (!(w.s != 0.0) || !isfinite(w.s)) return false;
    const int e = ilogb(w.s);
    if (e < -960 || e > 1000) return false;
    long long S = (long long)ldexp(fabs(w.s), 52 - e);  // exact
    w.S = w.s < 0.0 ? -S : S;
    w.e = e;
    w.in = true;
  }
  const int c = w.e - R.e0;
  if (c < 0 || c > 2 || !((R.ok >> c) & 1)) return false;
  const long long LO = (1LL << 52) + 1, HI = (1LL << 53) - 1;
  const long long lo = w.S + R.mn[c], hi = w.S + R.mx[c];
  if (w.S > 0) {
    if (lo < LO || hi > HI) return false;
  } else {
    if (hi > -LO || lo < -HI) return false;
  }
  w.S += R.K[c];
  return true;
}

__device__ __forceinline__ void exact_walk_flush(ExactWalk &w) {
  if (w.in) {
    w.s = ldexp((double)w.S, w.e - 52);
    w.in = false;
  }
}

// The walk of sum q by one warp: lane 0 carries the running sum through the
// group records, descending into a group's chunk records, a chunk's warp
// records and a warp segment's 32 terms only where a record does not apply.
// The lanes load the records and terms (rec: 32 records, wrec: a chunk's
// warp records, term: one chunk's terms). Returns the sum on lane 0.
static __device__ __noinline__ double exact_walk(const ExactHdr *H, const double *seq, long long n, long long nch,
                                          int q, long long cap, long long capg, ExactRec *rec, ExactRec *wrec,
                                          double *term) {
  const int lane = threadIdx.x & 31;
  const long long ng = (nch + kExactGroup - 1) / kExactGroup;
  ExactWalk w{0.0, 0, 0, false};
  long long gi = 0;
  while (gi < ng) {
    const int nb = (int)((ng - gi) < 32 ? (ng - gi) : 32);
    if (lane < nb) exact_load(rec[lane], &H->grec[q * capg + gi + lane]);
    __syncwarp();
    int k = 0;
    if (lane == 0)
      while (k < nb && exact_walk_apply(w, rec[k])) ++k;
    k = __shfl_sync(0xffffffffu, k, 0);
    __syncwarp();
    gi += k;
    if (k == nb) continue;
    // group gi: its chunk records, 32 at a time
    const long long c0 = gi * kExactGroup;
    const int cs = (int)((nch - c0) < kExactGroup ? (nch - c0) : kExactGroup);
    for (int h0 = 0; h0 < cs; h0 += 32) {
      const int hb = (cs - h0) < 32 ? (cs - h0) : 32;
      if (lane < hb) exact_load(rec[lane], &H->crec[q * cap + c0 + h0 + lane]);
      __syncwarp();
      int ci = 0;
      while (ci < hb) {
        int m = ci;
        if (lane == 0)
          while (m < hb && exact_walk_apply(w, rec[m])) ++m;
        m = __shfl_sync(0xffffffffu, m, 0);
        if (m >= hb) break;
        // chunk c0 + h0 + m: its warp records, then the terms of a warp
        // segment where one does not apply
        const long long ch = c0 + h0 + m;
        const long long e0 = ch * kExactChunkThreads;
        const int len = (int)((n - e0) < kExactChunkThreads ? (n - e0) : kExactChunkThreads);
        if (lane < kExactWarps) exact_load(wrec[lane], &H->wrec[(q * cap + ch) * kExactWarps + lane]);
        for (int e = lane; e < len; e += 32) term[e] = __ldcg(&seq[q * n + e0 + e]);
        __syncwarp();
        if (lane == 0) {
          for (int ww = 0; ww < kExactWarps && 32 * ww < len; ++ww) {
            if (exact_walk_apply(w, wrec[ww])) continue;
            exact_walk_flush(w);
            double sv = w.s;
            const int e1 = (32 * ww + 32) < len ? (32 * ww + 32) : len;
#pragma unroll 8
            for (int e = 32 * ww; e < e1; ++e) sv = __dadd_rn(sv, term[e]);
            w.s = sv;
          }
        }
        __syncwarp();
        ci = m + 1;
      }
      __syncwarp();
    }
    ++gi;
  }
  exact_walk_flush(w);
  return w.s;
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
  __shared__ ExactRec s_wr[NV][kExactWarps];
  __shared__ ExactRec s_rec;
  __shared__ bool s_last;
  __shared__ ExactRec s_wrec[kExactVals][32];
  __shared__ double s_wterm[kExactVals][kExactChunkThreads];
  __shared__ double s_res[kExactVals];

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

  // 3. records for the exponents around the hint: one per warp (32 terms,
  // warp scans only), composed by thread 0 into the chunk's record
  constexpr long long L53 = 1LL << 53;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    const double hint = s_hint[q];
    int e0 = 0;
    bool have = isfinite(hint) && hint != 0.0;
    if (have) {
      e0 = ilogb(hint) - 1;
      have = e0 >= -960 && e0 + 2 <= 1000;
    }
    ExactRec W;
    W.e0 = e0;
    W.ok = 0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      long long k = 0;
      bool good = false;
      if (have) {
        const double y = a[q] * ldexp(1.0, 52 - (e0 + c));
        // finite, |y| <= 2^53 and not half-way between two integers
        good = isfinite(y) && fabs(y) <= 9007199254740992.0 && fabs(y - trunc(y)) != 0.5;
        k = good ? __double2ll_rn(y) : 0;
      }
      // inclusive prefix over the warp, its total and range
      for (int off = 1; off < 32; off <<= 1) {
        const long long v = __shfl_up_sync(0xffffffffu, k, off);
        if (lane >= off) k += v;
      }
      long long mn = k, mx = k;
      for (int off = 16; off > 0; off >>= 1) {
        const long long a2 = __shfl_xor_sync(0xffffffffu, mn, off), b2 = __shfl_xor_sync(0xffffffffu, mx, off);
        mn = a2 < mn ? a2 : mn;
        mx = b2 > mx ? b2 : mx;
      }
      W.K[c] = __shfl_sync(0xffffffffu, k, 31);
      W.mn[c] = mn;
      W.mx[c] = mx;
      if (__all_sync(0xffffffffu, good) && mn > -L53 && mx < L53) W.ok |= 1 << c;
    }
    if (lane == 0) {
      s_wr[q][wid] = W;
      H->wrec[(q * cap + b) * kExactWarps + wid] = W;
    }
  }
  __syncthreads();
  if (t < NV) {  // thread q composes sum q's chunk record from its warp records
    const int q = t;
    ExactRec R;
    R.e0 = s_wr[q][0].e0;
    R.ok = 7;
    for (int c = 0; c < 3; ++c) {
      long long K = 0, mn = 0x7fffffffffffffffLL, mx = -0x7fffffffffffffffLL;
      for (int w = 0; w < kExactWarps; ++w) {
        const ExactRec &Wr = s_wr[q][w];
        if (!((Wr.ok >> c) & 1)) { R.ok &= ~(1 << c); break; }
        const long long lo = K + Wr.mn[c], hi = K + Wr.mx[c];
        mn = lo < mn ? lo : mn;
        mx = hi > mx ? hi : mx;
        K += Wr.K[c];
      }
      if (!((R.ok >> c) & 1) || mn <= -L53 || mx >= L53 || K <= -L53 || K >= L53) {
        R.ok &= ~(1 << c);
        K = mn = mx = 0;
      }
      R.K[c] = K;
      R.mn[c] = mn;
      R.mx[c] = mx;
    }
    if (!(isfinite(s_hint[q]) && s_hint[q] != 0.0)) R.ok = 0;
    H->crec[q * cap + b] = R;
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

  // 5. the last block walks the groups; warp q walks sum q
  if (t == 0) {
    __threadfence();
    unsigned prev = atomicAdd(count, 1u);
    s_last = (prev == (unsigned)nch - 1);
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
  if (wid < NV) {
    const double r = exact_walk(H, seq, n, nch, wid, cap, capg, s_wrec[wid], s_wr[wid], s_wterm[wid]);
    if (lane == 0) s_res[wid] = r;
  }
  __syncthreads();
  if (t != 0) return false;
#pragma unroll
  for (int q = 0; q < NV; ++q) out[q] = s_res[q];
  ExactHdr *Hw = const_cast<ExactHdr *>(H);
  const unsigned nxt = (gen + 1u) & 0x3fffffffu;
  Hw->gen = nxt ? nxt : 1u;  // generation 0 is the zeroed flags' value
  *count = 0u;
  __threadfence();
  return true;
}

}  // namespace pbg
