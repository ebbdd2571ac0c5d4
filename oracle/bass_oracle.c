/*
 * bass_oracle.c -- CPU oracle for the BASS sparse-state hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is a plain-C restatement of the
 * reference's Numba kernels (Skill0issue/BASS-Basis-Adapative-Sparse-Simulations-).
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
 * arm may load it, and only as the checker or the timed CPU baseline.  The
 * product (the CUDA library and its Python host) never calls into it.
 *
 * Conventions shared with the reference:
 *   - a key is a uint64 bitstring, qubit q is bit q (LSB = qubit 0)
 *     (src/simulation/exact_simulator.py:116-119, bass_simulator.py:616-620);
 *   - amplitudes are complex128, stored interleaved (re, im);
 *   - a 2-qubit matrix index is (bit_q1 << 1) | bit_q2 (sparse_state.py:96-98).
 *
 * Deliberate, documented deviations (all are tie-break / summation-order
 * choices; none changes a surviving key set on inputs without exact ties):
 *   - top-k selection orders candidates by (|a|^2 descending, key ascending)
 *     instead of np.argpartition's unspecified tie order, and keeps the
 *     survivors in their input order (a stable filter);
 *   - |a|^2 is re*re + im*im everywhere (the reference's BASS driver uses
 *     np.abs(a)**2, i.e. hypot(re, im)**2, which can differ by one ulp);
 *   - every reduction (sums of |a|^2, |a|^4 and the RDM moments) is exact and
 *     order independent: each term is truncated toward zero to a multiple of
 *     2^-96 and added in signed 128-bit integer arithmetic, and the total is
 *     rounded once to double (round to nearest even).  numpy's np.sum is a
 *     pairwise sum whose rounding depends on the array order, which after a
 *     top-k truncation is np.argpartition's order;
 *   - a 2-qubit output amplitude sums its contributions in ascending input
 *     index (b_q1 b_q2) order instead of the input array order.
 * The CUDA library computes the same quantities by the same rules, so the two
 * agree bit for bit.  Compiled with -ffp-contract=off (no fused multiply-add).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

typedef struct { double re, im; } cd;

static inline cd cd_mul(cd a, cd b) {
  cd r;
  r.re = a.re * b.re - a.im * b.im;
  r.im = a.re * b.im + a.im * b.re;
  return r;
}
static inline cd cd_add(cd a, cd b) { cd r; r.re = a.re + b.re; r.im = a.im + b.im; return r; }
static inline int cd_nz(cd a) { return a.re != 0.0 || a.im != 0.0; }
static inline double cd_p(cd a) { return a.re * a.re + a.im * a.im; }

/* murmur3 fmix64 finaliser (published constants), used for hashing and for
   order-independent key-set fingerprints. */
static inline uint64_t fmix64(uint64_t z) {
  z ^= z >> 33; z *= 0xff51afd7ed558ccdULL;
  z ^= z >> 33; z *= 0xc4ceb9fe1a85ec53ULL;
  z ^= z >> 33; return z;
}

/* ------------------------------------------------------------------ */
/* exact, order-independent accumulation                                */
/* ------------------------------------------------------------------ */
typedef __int128 i128;
typedef unsigned __int128 u128;
#define FX_FRAC 96

/* trunc(v * 2^96) toward zero, for finite |v| < 2^31 */
static inline i128 fx_from(double v) {
  uint64_t b;
  memcpy(&b, &v, sizeof b);
  int e = (int)((b >> 52) & 0x7FF);
  if (e == 0) return 0;                       /* zero or subnormal: below 2^-96 */
  uint64_t m = (b & 0xFFFFFFFFFFFFFULL) | 0x10000000000000ULL;   /* v = m * 2^(e-1075) */
  int sh = e - 1075 + FX_FRAC;
  i128 r;
  if (sh >= 0) r = (i128)((u128)m << sh);
  else if (sh > -64) r = (i128)(m >> (-sh));
  else r = 0;
  return (b >> 63) ? -r : r;
}

/* round-to-nearest-even of s * 2^-96 */
static inline double fx_to(i128 s) {
  if (s == 0) return 0.0;
  int neg = s < 0;
  u128 u = neg ? (u128)0 - (u128)s : (u128)s;
  uint64_t hi = (uint64_t)(u >> 64), lo = (uint64_t)u;
  int msb = hi ? 127 - __builtin_clzll(hi) : 63 - __builtin_clzll(lo);
  double r;
  if (msb <= 52) {
    r = ldexp((double)lo, -FX_FRAC);
  } else {
    int sh = msb - 52;
    u128 mant = u >> sh;
    u128 rem = u & (((u128)1 << sh) - 1);
    u128 half = (u128)1 << (sh - 1);
    if (rem > half || (rem == half && (mant & 1))) mant += 1;
    r = ldexp((double)(uint64_t)mant, sh - FX_FRAC);
  }
  return neg ? -r : r;
}

/* ------------------------------------------------------------------ */
/* open-addressing key -> index table (the reference uses an identity   */
/* hash with linear probing, bass_simulator.py:100-153; the result of  */
/* every caller is independent of the hash function).                   */
/* ------------------------------------------------------------------ */
typedef struct { uint64_t* k; int64_t* v; uint64_t mask; } oht;
#define OHT_EMPTY 0xFFFFFFFFFFFFFFFFULL

static int oht_init(oht* h, int64_t n) {
  uint64_t cap = 16;
  while (cap < (uint64_t)(2 * n + 16)) cap <<= 1;
  h->k = (uint64_t*)malloc(cap * sizeof(uint64_t));
  h->v = (int64_t*)malloc(cap * sizeof(int64_t));
  if (!h->k || !h->v) { free(h->k); free(h->v); return -1; }
  memset(h->k, 0xFF, cap * sizeof(uint64_t));
  h->mask = cap - 1;
  return 0;
}
static void oht_free(oht* h) { free(h->k); free(h->v); }
static inline int64_t oht_find(const oht* h, uint64_t key) {
  uint64_t s = fmix64(key) & h->mask;
  while (h->k[s] != OHT_EMPTY) {
    if (h->k[s] == key) return h->v[s];
    s = (s + 1) & h->mask;
  }
  return -1;
}
static inline void oht_put(oht* h, uint64_t key, int64_t val) {
  uint64_t s = fmix64(key) & h->mask;
  while (h->k[s] != OHT_EMPTY) {
    if (h->k[s] == key) { h->v[s] = val; return; }
    s = (s + 1) & h->mask;
  }
  h->k[s] = key; h->v[s] = val;
}

/* ------------------------------------------------------------------ */
/* parallel building blocks.  With -fopenmp the heavy kernels below run */
/* on every host thread; their results do not depend on the thread     */
/* count (work is split into contiguous ranges, sorts are stable, every */
/* sum is exact), so they equal the single-threaded ones bit for bit.   */
/* ------------------------------------------------------------------ */
#ifdef _OPENMP
#include <omp.h>
static int par_tid(void) { return omp_get_thread_num(); }
static int par_avail(void) { return omp_get_max_threads(); }
#else
static int par_tid(void) { return 0; }
static int par_avail(void) { return 1; }
#endif
static int g_threads = 1;  /* threads the kernels may use (orc_set_threads) */
static int par_max(void) { return g_threads; }

/* threads for n items: at most one per 32768 items */
static int par_threads_for(int64_t n) {
  int t = par_max();
  if ((int64_t)t > n / 32768) t = (int)(n / 32768);
  return t < 1 ? 1 : t;
}
/* start of range t of T contiguous ranges over [0, n) */
static inline int64_t par_lo(int64_t n, int T, int t) { return (int64_t)(((i128)n * t) / T); }

/* Threads the kernels may use: n > 0 that many (at most the OpenMP maximum),
   n <= 0 every host thread OpenMP offers.  The default is one.  Returns the
   number set. */
int orc_set_threads(int n) {
  const int avail = par_avail();
  g_threads = (n <= 0 || n > avail) ? avail : n;
  return g_threads;
}
int orc_threads(void) { return par_max(); }

/* Stable LSD radix sort of keys[0..n) carrying a payload of psize (8 or 16)
   bytes per item, 11-bit digits; a digit that is the same for every item is
   skipped (a stable pass over it changes nothing).  Items are spread over
   threads in contiguous ranges and placed by (digit, thread) offsets, so the
   order is that of a sequential stable sort. */
static int par_radix_sort(uint64_t* keys, void* pay, size_t psize, int64_t n) {
  if (n <= 1) return 0;
  enum { RB = 11, NB = 1 << RB };
  const int T = par_threads_for(n);
  uint64_t* tk = (uint64_t*)malloc((size_t)n * sizeof(uint64_t));
  char* tp = (char*)malloc((size_t)n * psize);
  int64_t* cnt = (int64_t*)malloc((size_t)T * NB * sizeof(int64_t));
  if (!tk || !tp || !cnt) { free(tk); free(tp); free(cnt); return -1; }
  uint64_t *ks = keys, *kd = tk;
  char *ps = (char*)pay, *pd = tp;
  for (int shift = 0; shift < 64; shift += RB) {
    memset(cnt, 0, (size_t)T * NB * sizeof(int64_t));
#pragma omp parallel num_threads(T)
    {
      const int t = par_tid();
      int64_t* c = cnt + (size_t)t * NB;
      for (int64_t i = par_lo(n, T, t); i < par_lo(n, T, t + 1); ++i) c[(ks[i] >> shift) & (NB - 1)]++;
    }
    int single = 0;
    for (int d = 0; d < NB && !single; ++d) {
      int64_t tot = 0;
      for (int t = 0; t < T; ++t) tot += cnt[(size_t)t * NB + d];
      if (tot == n) single = 1;
    }
    if (single) continue;
    int64_t run = 0;
    for (int d = 0; d < NB; ++d)
      for (int t = 0; t < T; ++t) {
        const int64_t c = cnt[(size_t)t * NB + d];
        cnt[(size_t)t * NB + d] = run;
        run += c;
      }
#pragma omp parallel num_threads(T)
    {
      const int t = par_tid();
      int64_t* c = cnt + (size_t)t * NB;
      for (int64_t i = par_lo(n, T, t); i < par_lo(n, T, t + 1); ++i) {
        const int64_t d = c[(ks[i] >> shift) & (NB - 1)]++;
        kd[d] = ks[i];
        if (psize == 16) memcpy(pd + (size_t)d * 16, ps + (size_t)i * 16, 16);
        else memcpy(pd + (size_t)d * 8, ps + (size_t)i * 8, 8);
      }
    }
    uint64_t* tku = ks; ks = kd; kd = tku;
    char* tpc = ps; ps = pd; pd = tpc;
  }
  if (ks != keys) {
    memcpy(keys, ks, (size_t)n * sizeof(uint64_t));
    memcpy(pay, ps, (size_t)n * psize);
  }
  free(tk); free(tp); free(cnt);
  return 0;
}

/* exact sum of |a|^2 (sq = 0) or |a|^4 (sq = 1) over a[0..n) */
static i128 par_sum_p(const cd* a, int64_t n, int sq) {
  const int T = par_threads_for(n);
  i128 part[256];
  const int TT = T > 256 ? 256 : T;
#pragma omp parallel num_threads(TT)
  {
    const int t = par_tid();
    i128 s = 0;
    for (int64_t i = par_lo(n, TT, t); i < par_lo(n, TT, t + 1); ++i) {
      const double p = cd_p(a[i]);
      s += fx_from(sq ? p * p : p);
    }
    part[t] = s;
  }
  i128 s = 0;
  for (int t = 0; t < TT; ++t) s += part[t];
  return s;
}

/* ------------------------------------------------------------------ */
/* sparse_state.py:15-67  apply_1qubit_gate_kernel_opt                */
/* ------------------------------------------------------------------ */
static int64_t expand_1q_range(const uint64_t* x_in, const cd* a_in, int64_t lo, int64_t hi,
                               uint64_t* x_out, cd* a_out, const cd* G, int q, int write) {
  int64_t n = 0;
  uint64_t m = 1ULL << q;
  cd g00 = G[0], g01 = G[1], g10 = G[2], g11 = G[3];
  for (int64_t i = lo; i < hi; ++i) {
    uint64_t x = x_in[i];
    cd a = a_in[i];
    uint64_t base = x & ~m;
    cd o0, o1;
    if (((x >> q) & 1ULL) == 0) { o0 = cd_mul(g00, a); o1 = cd_mul(g10, a); }
    else { o0 = cd_mul(g01, a); o1 = cd_mul(g11, a); }
    if (cd_nz(o0)) { if (write) { x_out[n] = base; a_out[n] = o0; } ++n; }
    if (cd_nz(o1)) { if (write) { x_out[n] = base | m; a_out[n] = o1; } ++n; }
  }
  return n;
}
int64_t orc_expand_1q(const uint64_t* x_in, const cd* a_in, int64_t nnz_in,
                      uint64_t* x_out, cd* a_out, const cd* G, int q) {
  const int T = par_threads_for(nnz_in);
  if (T == 1) return expand_1q_range(x_in, a_in, 0, nnz_in, x_out, a_out, G, q, 1);
  int64_t* off = (int64_t*)calloc((size_t)T + 1, sizeof(int64_t));
  if (!off) return -2;
#pragma omp parallel num_threads(T)
  {
    const int t = par_tid();
    off[t + 1] = expand_1q_range(x_in, a_in, par_lo(nnz_in, T, t), par_lo(nnz_in, T, t + 1), 0, 0, G, q, 0);
  }
  for (int t = 0; t < T; ++t) off[t + 1] += off[t];
#pragma omp parallel num_threads(T)
  {
    const int t = par_tid();
    expand_1q_range(x_in, a_in, par_lo(nnz_in, T, t), par_lo(nnz_in, T, t + 1), x_out + off[t], a_out + off[t],
                    G, q, 1);
  }
  const int64_t n = off[T];
  free(off);
  return n;
}

/* sparse_state.py:70-124  apply_2qubit_gate_kernel_opt (expansion only) */
int64_t orc_expand_2q(const uint64_t* x_in, const cd* a_in, int64_t nnz_in,
                      uint64_t* x_out, cd* a_out, int64_t cap_out,
                      const cd* G, int q1, int q2) {
  int64_t n = 0;
  uint64_t m1 = 1ULL << q1, m2 = 1ULL << q2;
  for (int64_t i = 0; i < nnz_in; ++i) {
    uint64_t x = x_in[i];
    cd a = a_in[i];
    int in_idx = (int)((((x >> q1) & 1ULL) << 1) | ((x >> q2) & 1ULL));
    uint64_t base = x & ~(m1 | m2);
    for (int o = 0; o < 4; ++o) {
      cd amp = cd_mul(G[o * 4 + in_idx], a);
      if (cd_nz(amp)) {
        uint64_t xn = base;
        if ((o >> 1) & 1) xn |= m1;
        if (o & 1) xn |= m2;
        if (n >= cap_out) return -1;
        x_out[n] = xn; a_out[n] = amp; ++n;
      }
    }
  }
  return n;
}

/* sparse_state.py:150-172  radix_sort_uint64: stable LSD sort, 4 x 16 bits.
   A pass whose digit is constant over the input is a no-op for a stable
   sort, so it is skipped (the result is identical). */
int orc_radix_sort(uint64_t* keys, cd* vals, int64_t n) {
  return par_radix_sort(keys, vals, sizeof(cd), n);
}

/* sparse_state.py:127-147  merge_sorted_kernel: sum adjacent equal keys in
   place (left to right); sums that cancel to zero are kept. */
int64_t orc_merge_sorted(uint64_t* x, cd* a, int64_t nnz) {
  if (nnz == 0) return 0;
  const int T = par_threads_for(nnz);
  if (T == 1) {
    int64_t w = 0;
    for (int64_t r = 1; r < nnz; ++r) {
      if (x[r] == x[w]) a[w] = cd_add(a[w], a[r]);
      else { ++w; x[w] = x[r]; a[w] = a[r]; }
    }
    return w + 1;
  }
  /* runs of equal keys, each summed left to right by the thread whose range
     holds the run's first item, written to a copy at the run's rank */
  int64_t* off = (int64_t*)calloc((size_t)T + 1, sizeof(int64_t));
  uint64_t* tx = (uint64_t*)malloc((size_t)nnz * sizeof(uint64_t));
  cd* ta = (cd*)malloc((size_t)nnz * sizeof(cd));
  if (!off || !tx || !ta) { free(off); free(tx); free(ta); return -2; }
#pragma omp parallel num_threads(T)
  {
    const int t = par_tid();
    int64_t c = 0;
    for (int64_t i = par_lo(nnz, T, t); i < par_lo(nnz, T, t + 1); ++i) c += (i == 0 || x[i] != x[i - 1]);
    off[t + 1] = c;
  }
  for (int t = 0; t < T; ++t) off[t + 1] += off[t];
#pragma omp parallel num_threads(T)
  {
    const int t = par_tid();
    int64_t w = off[t];
    for (int64_t i = par_lo(nnz, T, t); i < par_lo(nnz, T, t + 1); ++i) {
      if (!(i == 0 || x[i] != x[i - 1])) continue;
      cd acc = a[i];
      for (int64_t r = i + 1; r < nnz && x[r] == x[i]; ++r) acc = cd_add(acc, a[r]);
      tx[w] = x[i]; ta[w] = acc; ++w;
    }
  }
  const int64_t n = off[T];
  memcpy(x, tx, (size_t)n * sizeof(uint64_t));
  memcpy(a, ta, (size_t)n * sizeof(cd));
  free(off); free(tx); free(ta);
  return n;
}

/* SparseState.apply_single_qubit_gate (sparse_state.py:268-296) without the
   trailing truncation: expand, stable sort, merge.  Output is key-sorted. */
int64_t orc_apply_1q(const uint64_t* x_in, const cd* a_in, int64_t nnz_in,
                     uint64_t* x_out, cd* a_out, const cd* G, int q) {
  int64_t n = orc_expand_1q(x_in, a_in, nnz_in, x_out, a_out, G, q);
  if (orc_radix_sort(x_out, a_out, n)) return -2;
  return orc_merge_sorted(x_out, a_out, n);
}

/* bass_simulator.py:292-354  apply_2qubit_gate_ht: <=4 children per entry;
   an output exists if at least one of its contributions G[o,in]*a is non-zero;
   the output set and its first-occurrence order follow the reference.  The
   non-zero contributions are summed in ascending in_idx order (see header).
   x_out/a_out need 4*nnz_in entries. */
int64_t orc_apply_2q_ht(const uint64_t* x_in, const cd* a_in, int64_t nnz_in,
                        uint64_t* x_out, cd* a_out, const cd* G, int q1, int q2) {
  uint64_t m1 = 1ULL << q1, m2 = 1ULL << q2;
  oht grp;                       /* base key -> group id */
  if (oht_init(&grp, nnz_in)) return -2;
  int64_t* mem = (int64_t*)malloc((size_t)(nnz_in > 0 ? nnz_in : 1) * 4 * sizeof(int64_t));
  if (!mem) { oht_free(&grp); return -2; }
  int64_t ng = 0;
  int64_t* gid = (int64_t*)malloc((size_t)(nnz_in > 0 ? nnz_in : 1) * sizeof(int64_t));
  if (!gid) { free(mem); oht_free(&grp); return -2; }
  for (int64_t i = 0; i < nnz_in; ++i) {
    uint64_t base = x_in[i] & ~(m1 | m2);
    int64_t g = oht_find(&grp, base);
    if (g < 0) { g = ng++; oht_put(&grp, base, g); for (int t = 0; t < 4; ++t) mem[4 * g + t] = -1; }
    int in_idx = (int)((((x_in[i] >> q1) & 1ULL) << 1) | ((x_in[i] >> q2) & 1ULL));
    mem[4 * g + in_idx] = i;
    gid[i] = g;
  }
  oht out;                       /* output key -> output slot */
  if (oht_init(&out, 4 * nnz_in)) { free(mem); free(gid); oht_free(&grp); return -2; }
  int64_t n = 0;
  for (int64_t i = 0; i < nnz_in; ++i) {
    uint64_t xi = x_in[i];
    cd a = a_in[i];
    int in_idx = (int)((((xi >> q1) & 1ULL) << 1) | ((xi >> q2) & 1ULL));
    uint64_t base = xi & ~(m1 | m2);
    for (int o = 0; o < 4; ++o) {
      if (!cd_nz(cd_mul(G[o * 4 + in_idx], a))) continue;
      uint64_t xn = base;
      if ((o >> 1) & 1) xn |= m1;
      if (o & 1) xn |= m2;
      if (oht_find(&out, xn) >= 0) continue;     /* already emitted */
      const int64_t* mm = mem + 4 * gid[i];
      int have = 0;
      cd acc = {0.0, 0.0};
      for (int t = 0; t < 4; ++t) {
        if (mm[t] < 0) continue;
        cd c = cd_mul(G[o * 4 + t], a_in[mm[t]]);
        if (!cd_nz(c)) continue;
        acc = have ? cd_add(acc, c) : c;
        have = 1;
      }
      x_out[n] = xn; a_out[n] = acc; oht_put(&out, xn, n); ++n;
    }
  }
  oht_free(&out); oht_free(&grp); free(mem); free(gid);
  return n;
}

/* SparseState.apply_two_qubit_gate (sparse_state.py:303-370) without the
   trailing truncation.  The reference expands, sorts and merges; the merged
   output is the same set of keys and (up to summation order) the same sums as
   the hash version, so the oracle computes the hash version (in_idx order
   sums) and sorts it by key.  x_out/a_out need 4*nnz_in entries. */
int64_t orc_apply_2q_sorted(const uint64_t* x_in, const cd* a_in, int64_t nnz_in,
                            uint64_t* x_out, cd* a_out, int64_t cap_out,
                            const cd* G, int q1, int q2) {
  if (cap_out < 4 * nnz_in) return -1;
  int64_t n = orc_apply_2q_ht(x_in, a_in, nnz_in, x_out, a_out, G, q1, q2);
  if (n < 0) return n;
  if (orc_radix_sort(x_out, a_out, n)) return -2;
  return n;
}

/* sparse_state.py:178-190  apply_2qubit_diagonal_kernel (in place) */
void orc_phase_2q(const uint64_t* x, cd* a, int64_t nnz, int q1, int q2, const cd* diag) {
#pragma omp parallel for num_threads(par_threads_for(nnz)) schedule(static)
  for (int64_t i = 0; i < nnz; ++i) {
    int b1 = (int)((x[i] >> q1) & 1ULL), b2 = (int)((x[i] >> q2) & 1ULL);
    a[i] = cd_mul(a[i], diag[(b1 << 1) | b2]);
  }
}

/* ------------------------------------------------------------------ */
/* top-k selection by (p descending, key ascending)                    */
/* ------------------------------------------------------------------ */
/* Keep the k best entries of (x, a)[0..n) in their input order.  Returns the
   new count; *kept = sum of kept |a|^2, *total = sum of all |a|^2 (both
   exact).  If n <= k nothing is removed.  The threshold is the entry of rank
   k - 1 by (|a|^2 descending, key ascending): found by a radix select on the
   bit patterns of |a|^2 (non-negative doubles order as their bits), then, for
   the entries whose |a|^2 equals the threshold, by their keys. */
static int u64_cmp(const void* A, const void* B) {
  const uint64_t a = *(const uint64_t*)A, b = *(const uint64_t*)B;
  return (a > b) - (a < b);
}
int64_t orc_select_topk(uint64_t* x, cd* a, int64_t n, int64_t k, double* kept, double* total) {
  const double tot = fx_to(par_sum_p(a, n, 0));
  if (total) *total = tot;
  if (n <= k) { if (kept) *kept = tot; return n; }
  if (k <= 0) { if (kept) *kept = 0.0; return 0; }
  const int T = par_threads_for(n);
  enum { RB = 11, NB = 1 << RB };
  uint64_t* pb = (uint64_t*)malloc((size_t)n * sizeof(uint64_t));
  int64_t* cnt = (int64_t*)malloc((size_t)T * NB * sizeof(int64_t));
  if (!pb || !cnt) { free(pb); free(cnt); return -2; }
#pragma omp parallel for num_threads(T) schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const double p = cd_p(a[i]);
    memcpy(&pb[i], &p, sizeof p);
  }
  /* digits from the top: bits [53, 64), [42, 53), ..., [9, 20), [0, 9) */
  uint64_t pre = 0;   /* the fixed high bits of the threshold pattern */
  int64_t need = k;   /* rank, among the entries matching pre, still to place */
  int fixed = 64;     /* bits >= fixed are fixed in pre */
  while (fixed > 0) {
    const int shift = fixed >= RB ? fixed - RB : 0;
    const int width = fixed - shift;
    const uint64_t dmask = (1ULL << width) - 1;
    memset(cnt, 0, (size_t)T * NB * sizeof(int64_t));
#pragma omp parallel num_threads(T)
    {
      const int t = par_tid();
      int64_t* c = cnt + (size_t)t * NB;
      for (int64_t i = par_lo(n, T, t); i < par_lo(n, T, t + 1); ++i)
        if (fixed == 64 || (pb[i] >> fixed) == (pre >> fixed)) c[(pb[i] >> shift) & dmask]++;
    }
    int64_t above = 0;
    int d = (int)dmask;
    for (; d > 0; --d) {
      int64_t c = 0;
      for (int t = 0; t < T; ++t) c += cnt[(size_t)t * NB + d];
      if (above + c >= need) break;
      above += c;
    }
    need -= above;
    pre |= (uint64_t)d << shift;
    fixed = shift;
  }
  /* the entries at the threshold pattern: the need-th smallest key */
  int64_t m = 0;
  for (int64_t i = 0; i < n; ++i) m += (pb[i] == pre);
  uint64_t* tk = (uint64_t*)malloc((size_t)(m > 0 ? m : 1) * sizeof(uint64_t));
  if (!tk) { free(pb); free(cnt); return -2; }
  m = 0;
  for (int64_t i = 0; i < n; ++i) if (pb[i] == pre) tk[m++] = x[i];
  qsort(tk, (size_t)m, sizeof(uint64_t), u64_cmp);
  const uint64_t key_t = tk[need - 1];
  free(tk);
  /* the survivors, in input order: counts per range, then the copies */
  int64_t* off = (int64_t*)calloc((size_t)T + 1, sizeof(int64_t));
  i128* ks = (i128*)calloc((size_t)T, sizeof(i128));
  uint64_t* tx = (uint64_t*)malloc((size_t)n * sizeof(uint64_t));
  cd* ta = (cd*)malloc((size_t)n * sizeof(cd));
  if (!off || !ks || !tx || !ta) { free(off); free(ks); free(tx); free(ta); free(pb); free(cnt); return -2; }
#pragma omp parallel num_threads(T)
  {
    const int t = par_tid();
    int64_t c = 0;
    for (int64_t i = par_lo(n, T, t); i < par_lo(n, T, t + 1); ++i)
      c += pb[i] > pre || (pb[i] == pre && x[i] <= key_t);
    off[t + 1] = c;
  }
  for (int t = 0; t < T; ++t) off[t + 1] += off[t];
#pragma omp parallel num_threads(T)
  {
    const int t = par_tid();
    int64_t w = off[t];
    i128 acc = 0;
    for (int64_t i = par_lo(n, T, t); i < par_lo(n, T, t + 1); ++i) {
      if (!(pb[i] > pre || (pb[i] == pre && x[i] <= key_t))) continue;
      double p;
      memcpy(&p, &pb[i], sizeof p);
      acc += fx_from(p);
      tx[w] = x[i]; ta[w] = a[i]; ++w;
    }
    ks[t] = acc;
  }
  const int64_t w = off[T];
  i128 kacc = 0;
  for (int t = 0; t < T; ++t) kacc += ks[t];
  memcpy(x, tx, (size_t)w * sizeof(uint64_t));
  memcpy(a, ta, (size_t)w * sizeof(cd));
  if (kept) *kept = fx_to(kacc);
  free(off); free(ks); free(tx); free(ta); free(pb); free(cnt);
  return w;
}

/* truncation.py:68-113  top_k_truncate_kernel_opt: returns (nnz', gamma_sq)
   where gamma_sq is the kept |a|^2 mass (the whole mass if nnz <= k). */
int64_t orc_topk_truncate(uint64_t* x, cd* a, int64_t nnz, int64_t k, double* gamma_sq) {
  double kept = 0.0, total = 0.0;
  int64_t r = orc_select_topk(x, a, nnz, k, &kept, &total);
  *gamma_sq = kept;
  return r;
}

/* truncation.py:116-159  random_k_truncate_kernel_opt: LCG partial
   Fisher-Yates; survivors in permutation order. */
int64_t orc_randomk_truncate(uint64_t* x, cd* a, int64_t nnz, int64_t k, int64_t seed, double* gamma_sq) {
  if (nnz <= k) {
    i128 g = 0;
    for (int64_t i = 0; i < nnz; ++i) g += fx_from(cd_p(a[i]));
    *gamma_sq = fx_to(g);
    return nnz;
  }
  int64_t* perm = (int64_t*)malloc((size_t)nnz * sizeof(int64_t));
  uint64_t* tx = (uint64_t*)malloc((size_t)k * sizeof(uint64_t));
  cd* ta = (cd*)malloc((size_t)k * sizeof(cd));
  if (!perm || !tx || !ta) { free(perm); free(tx); free(ta); return -2; }
  for (int64_t i = 0; i < nnz; ++i) perm[i] = i;
  int64_t rng = seed;
  for (int64_t i = 0; i < k; ++i) {
    rng = (1103515245LL * rng + 12345LL) & 0x7FFFFFFFLL;
    int64_t r = i + (rng % (nnz - i));
    int64_t t = perm[i]; perm[i] = perm[r]; perm[r] = t;
  }
  i128 g = 0;
  for (int64_t j = 0; j < k; ++j) {
    int64_t id = perm[j];
    tx[j] = x[id]; ta[j] = a[id];
    g += fx_from(cd_p(a[id]));
  }
  memcpy(x, tx, (size_t)k * sizeof(uint64_t));
  memcpy(a, ta, (size_t)k * sizeof(cd));
  free(perm); free(tx); free(ta);
  *gamma_sq = fx_to(g);
  return k;
}

/* bass_simulator.py:441-470 (with ht_build :108-123)  compute_all_1qubit_rdms.
   rho is N x 2 x 2 complex, row-major.  Per qubit q: rho00 = sum of |a|^2 over
   keys with bit q clear, rho11 over keys with it set, rho01 = sum over pairs
   (x, x | 2^q) of a_x * conj(a_partner), rho10 = conj(rho01) (term by term,
   exactly as the reference's separate accumulation).  Exact sums. */
int orc_rdm_all(const uint64_t* x, const cd* a, int64_t nnz, int N, cd* rho) {
  memset(rho, 0, (size_t)N * 4 * sizeof(cd));
  i128* acc = (i128*)calloc((size_t)N * 4, sizeof(i128));
  oht h;
  if (!acc || oht_init(&h, nnz)) { free(acc); return -2; }
  for (int64_t i = 0; i < nnz; ++i) oht_put(&h, x[i], i);
  const int T = par_threads_for(nnz);
  i128* tacc = (i128*)calloc((size_t)T * N * 4, sizeof(i128));
  if (!tacc) { oht_free(&h); free(acc); return -2; }
#pragma omp parallel num_threads(T)
  {
    const int th = par_tid();
    i128* my = tacc + (size_t)th * N * 4;
    for (int64_t i = par_lo(nnz, T, th); i < par_lo(nnz, T, th + 1); ++i) {
      uint64_t xi = x[i];
      cd ai = a[i];
      i128 prob = fx_from(ai.re * ai.re + ai.im * ai.im);
      for (int q = 0; q < N; ++q) {
        int bit = (int)((xi >> q) & 1ULL);
        i128* r = my + (size_t)q * 4;
        r[bit] += prob;
        if (bit == 0) {
          int64_t p = oht_find(&h, xi | (1ULL << q));
          if (p >= 0) {
            cd caj = {a[p].re, -a[p].im};
            cd t = cd_mul(ai, caj);
            r[2] += fx_from(t.re);
            r[3] += fx_from(t.im);
          }
        }
      }
    }
  }
  for (int th = 0; th < T; ++th)
    for (int v = 0; v < N * 4; ++v) acc[v] += tacc[(size_t)th * N * 4 + v];
  free(tacc);
  for (int q = 0; q < N; ++q) {
    cd* r = rho + (size_t)q * 4;
    i128* c = acc + (size_t)q * 4;
    r[0].re = fx_to(c[0]);
    r[3].re = fx_to(c[1]);
    r[1].re = fx_to(c[2]); r[1].im = fx_to(c[3]);
    r[2].re = fx_to(c[2]); r[2].im = -fx_to(c[3]);
  }
  oht_free(&h); free(acc);
  return 0;
}

/* bass_simulator.py:386-437  eigh_2x2: descending eigenvalues, eigenvectors
   as columns of V (row-major 2x2 complex). */
void orc_eigh_2x2(const cd* rho, double* evals, cd* V) {
  double a = rho[0].re, d = rho[3].re;
  cd b = rho[1];
  double b_sq = b.re * b.re + b.im * b.im;
  double tau = (d - a) * 0.5;
  double disc = sqrt(tau * tau + b_sq);
  evals[0] = (a + d) * 0.5 + disc;
  evals[1] = (a + d) * 0.5 - disc;
  memset(V, 0, 4 * sizeof(cd));
  if (b_sq < 1e-28) {
    if (a >= d) { V[0].re = 1.0; V[3].re = 1.0; }
    else { V[1].re = 1.0; V[2].re = 1.0; }
  } else {
    double tdp = tau + disc, tdm = tau - disc;
    double n0 = sqrt(b_sq + tdp * tdp), n1 = sqrt(b_sq + tdm * tdm);
    V[0].re = b.re / n0; V[0].im = b.im / n0;
    V[2].re = tdp / n0;
    V[1].re = b.re / n1; V[1].im = b.im / n1;
    V[3].re = tdm / n1;
  }
}

/* bass_simulator.py:156-199  apply_1qubit_rotation_sparse: group by
   x & ~m (ascending), pair-combine by U, drop |a'| <= 1e-30.  Output is
   written to x_out/a_out (capacity 2*nnz) and is key-sorted. */
typedef struct { uint64_t r; int64_t i; } ri;
static int ri_cmp(const void* A, const void* B) {
  const ri* a = (const ri*)A; const ri* b = (const ri*)B;
  if (a->r < b->r) return -1;
  if (a->r > b->r) return 1;
  return (a->i < b->i) ? -1 : (a->i > b->i);
}
/* the outputs of the groups that start in [lo, hi) of the grouped order
   (r ascending, then input index), written when write != 0 */
static int64_t rotate_1q_range(const uint64_t* x, const cd* a, const uint64_t* r, const int64_t* idx,
                               int64_t nnz, int64_t lo, int64_t hi, int qubit, const cd* U, uint64_t* x_out,
                               cd* a_out, int write) {
  const uint64_t m = 1ULL << qubit;
  int64_t n = 0, i = lo;
  while (i < hi) {
    const uint64_t rr = r[i];
    int64_t j = i + 1;
    while (j < nnz && r[j] == rr) ++j;
    cd a0 = {0.0, 0.0}, a1 = {0.0, 0.0};
    for (int64_t t = i; t < j; ++t) {
      const int64_t oi = idx[t];
      if (((x[oi] >> qubit) & 1ULL) == 0) a0 = a[oi]; else a1 = a[oi];
    }
    cd n0 = cd_add(cd_mul(U[0], a0), cd_mul(U[1], a1));
    cd n1 = cd_add(cd_mul(U[2], a0), cd_mul(U[3], a1));
    if (hypot(n0.re, n0.im) > 1e-30) { if (write) { x_out[n] = rr; a_out[n] = n0; } ++n; }
    if (hypot(n1.re, n1.im) > 1e-30) { if (write) { x_out[n] = rr | m; a_out[n] = n1; } ++n; }
    i = j;
  }
  return n;
}
int64_t orc_rotate_1q(const uint64_t* x, const cd* a, int64_t nnz, int qubit, const cd* U,
                      uint64_t* x_out, cd* a_out) {
  const uint64_t m = 1ULL << qubit;
  uint64_t* r = (uint64_t*)malloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(uint64_t));
  int64_t* idx = (int64_t*)malloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(int64_t));
  const int T = par_threads_for(nnz);
  int64_t* st = (int64_t*)calloc((size_t)T + 1, sizeof(int64_t));
  int64_t* off = (int64_t*)calloc((size_t)T + 1, sizeof(int64_t));
  if (!r || !idx || !st || !off) { free(r); free(idx); free(st); free(off); return -2; }
#pragma omp parallel for num_threads(T) schedule(static)
  for (int64_t i = 0; i < nnz; ++i) { r[i] = x[i] & ~m; idx[i] = i; }
  /* group by x & ~m ascending; within a group, input order (a stable sort) */
  if (par_radix_sort(r, idx, sizeof(int64_t), nnz)) { free(r); free(idx); free(st); free(off); return -2; }
  /* ranges of whole groups: each range start moved forward to a group start */
  for (int t = 0; t <= T; ++t) {
    int64_t lo = par_lo(nnz, T, t);
    while (lo > 0 && lo < nnz && r[lo] == r[lo - 1]) ++lo;
    st[t] = lo;
  }
#pragma omp parallel num_threads(T)
  {
    const int t = par_tid();
    off[t + 1] = rotate_1q_range(x, a, r, idx, nnz, st[t], st[t + 1], qubit, U, 0, 0, 0);
  }
  for (int t = 0; t < T; ++t) off[t + 1] += off[t];
#pragma omp parallel num_threads(T)
  {
    const int t = par_tid();
    rotate_1q_range(x, a, r, idx, nnz, st[t], st[t + 1], qubit, U, x_out + off[t], a_out + off[t], 1);
  }
  const int64_t n = off[T];
  free(r); free(idx); free(st); free(off);
  return n;
}

/* Groups of entries that agree on every bit except q1 and q2, ascending by
   the remaining bits: g[4 * t + idx] = entry index or -1, idx = (bit_q1 << 1)
   | bit_q2.  Returns the number of groups (or -2), bases in base_out. */
static int64_t groups_2q(const uint64_t* x, int64_t nnz, int q1, int q2, int64_t** g_out,
                         uint64_t** base_out) {
  uint64_t m12 = (1ULL << q1) | (1ULL << q2);
  ri* v = (ri*)malloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(ri));
  int64_t* g = (int64_t*)malloc((size_t)(nnz > 0 ? nnz : 1) * 4 * sizeof(int64_t));
  uint64_t* b = (uint64_t*)malloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(uint64_t));
  if (!v || !g || !b) { free(v); free(g); free(b); return -2; }
  for (int64_t i = 0; i < nnz; ++i) { v[i].r = x[i] & ~m12; v[i].i = i; }
  qsort(v, (size_t)nnz, sizeof(ri), ri_cmp);
  int64_t ng = 0, i = 0;
  while (i < nnz) {
    uint64_t r = v[i].r;
    for (int t = 0; t < 4; ++t) g[4 * ng + t] = -1;
    while (i < nnz && v[i].r == r) {
      int64_t oi = v[i].i;
      int idx = (int)((((x[oi] >> q1) & 1ULL) << 1) | ((x[oi] >> q2) & 1ULL));
      g[4 * ng + idx] = oi;
      ++i;
    }
    b[ng++] = r;
  }
  free(v);
  *g_out = g;
  *base_out = b;
  return ng;
}

/* bass_simulator.py:200-231  compute_2qubit_rdm: 4x4 rho (row-major), index
   (bit_q1 << 1) | bit_q2; over the groups of entries that share every other
   bit, rho[p][q] += a_p * conj(a_q).  Exact sums (the reference sums in
   group order in floating point). */
int orc_rdm_2q(const uint64_t* x, const cd* a, int64_t nnz, int q1, int q2, cd* rho) {
  int64_t* g;
  uint64_t* b;
  int64_t ng = groups_2q(x, nnz, q1, q2, &g, &b);
  if (ng < 0) return -2;
  i128 acc[16][2];
  memset(acc, 0, sizeof(acc));
  const cd zero = {0.0, 0.0};
  for (int64_t t = 0; t < ng; ++t) {
    cd v[4];
    for (int k = 0; k < 4; ++k) v[k] = g[4 * t + k] >= 0 ? a[g[4 * t + k]] : zero;
    for (int p = 0; p < 4; ++p)
      for (int q = 0; q < 4; ++q) {
        cd cq = {v[q].re, -v[q].im};
        cd c = cd_mul(v[p], cq);
        acc[4 * p + q][0] += fx_from(c.re);
        acc[4 * p + q][1] += fx_from(c.im);
      }
  }
  for (int k = 0; k < 16; ++k) { rho[k].re = fx_to(acc[k][0]); rho[k].im = fx_to(acc[k][1]); }
  free(g); free(b);
  return 0;
}

/* bass_simulator.py:237-289  apply_2qubit_rotation_sparse: per group,
   a_out[o] = sum over the present inputs of U4[o][idx] * a_in[idx] (ascending
   idx, exact-zero products skipped as in the 2-qubit gate), children with
   |a_out| <= 1e-30 dropped.  Output key-sorted; x_out/a_out hold 4*nnz. */
int64_t orc_rotate_2q(const uint64_t* x, const cd* a, int64_t nnz, int q1, int q2, const cd* U4,
                      uint64_t* x_out, cd* a_out) {
  int64_t* g;
  uint64_t* b;
  int64_t ng = groups_2q(x, nnz, q1, q2, &g, &b);
  if (ng < 0) return -2;
  uint64_t m1 = 1ULL << q1, m2 = 1ULL << q2;
  int64_t n = 0;
  for (int64_t t = 0; t < ng; ++t) {
    for (int o = 0; o < 4; ++o) {
      int have = 0;
      cd acc = {0.0, 0.0};
      for (int k = 0; k < 4; ++k) {
        if (g[4 * t + k] < 0) continue;
        cd c = cd_mul(U4[o * 4 + k], a[g[4 * t + k]]);
        if (!cd_nz(c)) continue;
        acc = have ? cd_add(acc, c) : c;
        have = 1;
      }
      if (hypot(acc.re, acc.im) > 1e-30) {
        uint64_t xn = b[t];
        if ((o >> 1) & 1) xn |= m1;
        if (o & 1) xn |= m2;
        x_out[n] = xn; a_out[n] = acc; ++n;
      }
    }
  }
  free(g); free(b);
  if (orc_radix_sort(x_out, a_out, n)) return -2;
  return n;
}

/* ------------------------------------------------------------------ */
/* reductions and fingerprints                                          */
/* ------------------------------------------------------------------ */
double orc_sum_p(const cd* a, int64_t n) { return fx_to(par_sum_p(a, n, 0)); }
double orc_sum_p2(const cd* a, int64_t n) { return fx_to(par_sum_p(a, n, 1)); }
/* exposes the accumulator for tests: exact sum of v[0..n) */
double orc_exact_sum(const double* v, int64_t n) {
  i128 s = 0;
  for (int64_t i = 0; i < n; ++i) s += fx_from(v[i]);
  return fx_to(s);
}
/* Order-independent fingerprint of a key set: (count, sum of fmix64(k) mod
   2^64, xor of fmix64(k ^ c)).  With a != NULL only keys whose |a|^2 exceeds
   pmin are included.  Same definition in the CUDA library. */
void orc_fingerprint(const uint64_t* x, const cd* a, int64_t n, double pmin, uint64_t* out3) {
  uint64_t c = 0, s = 0, z = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (a && !(cd_p(a[i]) > pmin)) continue;
    ++c;
    s += fmix64(x[i]);
    z ^= fmix64(x[i] ^ 0x5851F42D4C957F2DULL);
  }
  out3[0] = c; out3[1] = s; out3[2] = z;
}
