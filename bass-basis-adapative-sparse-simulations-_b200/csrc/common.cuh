// common.cuh -- shared device code of libbass_b200 (sm_100a).
//
// Arithmetic rules (shared with the CPU oracle, so that both agree bit for bit):
//   * complex products and sums are evaluated with explicit round-to-nearest
//     intrinsics, never fused into FMA;
//   * |a|^2 = re*re + im*im;
//   * every reduction is exact and order independent: a term is truncated
//     toward zero to a multiple of 2^-96, summed in signed 128-bit integers,
//     and the total is rounded once to double (round to nearest even).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/bass_b200.h"

namespace bass {

typedef __int128 i128;
typedef unsigned __int128 u128;

constexpr int kTile = 2048;          // entries a tile CTA holds (kThreads x kPerThread)
constexpr int kThreads = 256;        // threads per tile CTA
constexpr int kPerThread = kTile / kThreads;
// Merge tiles start every kStep Z positions; backing a boundary off to the
// start of its group (at most 4 entries for 2-qubit groups) can grow a tile to
// kStep + 4 <= kTile entries, so every entry has a thread.
constexpr int kStep = kTile - 8;
constexpr int kTilePad = kTile + 8;
constexpr int kHistBins = 8192;      // 13-bit radix-select digits
constexpr int kGroupBins = 128;      // bins per coarse group of a selection histogram
constexpr int kHistGroups = kHistBins / kGroupBins;  // coarse counts stored after the bins
constexpr int kCandSmem = 4096;      // candidates sorted in shared memory
constexpr int kRankMax = 1024;       // candidates ranked by direct counting (one per thread of a selection block)
constexpr int kMaxSets = 64;         // partition sets (one per qubit for RDMs)
// RDM moments of the qubits at physical bits 0 .. kRdmLowBits - 1 come from
// one pass over plain tiles plus a halo of kRdmHalo entries (k_rdm_low)
constexpr int kRdmLowBits = 10;
constexpr int kRdmHalo = 1 << (kRdmLowBits - 1);
constexpr int kFxFrac = 96;
constexpr long long kSpinLimit = 1LL << 22;  // a few seconds at most

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
__device__ __forceinline__ void set_error(bass_ctrl* c, int code) {
  atomicOr(&c->error, 1 << code);
}

// Spins a bounded wait makes before it gives up (bass_ctrl.wait_limit: 0 the
// default kSpinLimit, > 0 that many, < 0 none).
__device__ __forceinline__ long long wait_limit(const bass_ctrl* c) {
  const int w = *(volatile const int*)&c->wait_limit;
  return w == 0 ? kSpinLimit : (w < 0 ? 0 : (long long)w);
}

// ---------------------------------------------------------------------------
// bulk asynchronous copies (TMA, untiled) into this CTA's shared memory
// ---------------------------------------------------------------------------
// Global source and shared destination 16-byte aligned, sizes multiples of
// 16 bytes; the source is always this GPU's own memory and every copy lands
// in the issuing CTA's shared memory only.  Completion is counted in bytes
// on an mbarrier of the CTA.
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned arrivals) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n\tfence.mbarrier_init.release.cluster;" ::"r"(
                   smem_addr(bar)),
               "r"(arrivals)
               : "memory");
}
// One arrival that also expects `bytes` of copies on the current phase.
__device__ __forceinline__ void mbar_arrive_expect(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
// true once the phase of the given parity has completed (the thread may be
// suspended for up to about a microsecond before it returns false)
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity), "r"(1000)
      : "memory");
  return ok != 0;
}
// Orders this CTA's earlier generic-proxy accesses of shared memory (after a
// barrier: every thread's) before the bulk copies issued next.
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}
// A hint: bring [src, src + bytes) into L2 (no completion to wait for).
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

// ---------------------------------------------------------------------------
// exact accumulation
// ---------------------------------------------------------------------------
// fx_from(v) = trunc(|v| * 2^96) with the sign of v (terms below 2^-96 vanish).
__host__ __device__ __forceinline__ i128 fx_from_bits(double v) {
  uint64_t b;
#ifdef __CUDA_ARCH__
  b = (uint64_t)__double_as_longlong(v);
#else
  memcpy(&b, &v, sizeof b);
#endif
  int e = (int)((b >> 52) & 0x7FF);
  if (e == 0) return 0;
  uint64_t m = (b & 0xFFFFFFFFFFFFFULL) | 0x10000000000000ULL;
  int sh = e - 1075 + kFxFrac;
  i128 r;
  if (sh >= 0) r = (i128)((u128)m << sh);
  else if (sh > -64) r = (i128)(m >> (-sh));
  else r = 0;
  return (b >> 63) ? -r : r;
}

// fx_from of a non-negative finite double given by its bit pattern (a
// probability), with integer operations only.
__device__ __forceinline__ i128 fx_from_pbits(unsigned long long b) {
  const int e = (int)(b >> 52);
  const unsigned long long m = (b & 0xFFFFFFFFFFFFFULL) | 0x10000000000000ULL;
  const int sh = e - 1075 + kFxFrac;  // value * 2^96 = m * 2^sh
  if (e == 0 || sh <= -64) return 0;
  if (sh < 0) return (i128)(m >> (-sh));
  return (i128)((u128)m << sh);
}

// On the device, for |v| < 2^31 (every probability and moment summed here),
// the same integer is formed in exact floating-point steps: hi =
// floor(|v| * 2^32) and lo = floor(frac(|v| * 2^32) * 2^64); both scalings are
// by powers of two and x - floor(x) is exact, so nothing is rounded.
__host__ __device__ __forceinline__ i128 fx_from(double v) {
#ifdef __CUDA_ARCH__
  const double x = __dmul_rn(fabs(v), 4294967296.0);
  if (!(x < 9223372036854775808.0)) return fx_from_bits(v);
  const unsigned long long hi = __double2ull_rz(x);
  const double r = __dsub_rn(x, __ull2double_rn(hi));
  const unsigned long long lo = __double2ull_rz(__dmul_rn(r, 18446744073709551616.0));
  const i128 m = (i128)(((u128)hi << 64) | (u128)lo);
  return v < 0.0 ? -m : m;
#else
  return fx_from_bits(v);
#endif
}

// floor(v * 2^96) for 0 <= v < 4 as h * 2^48 + l, with h and l integers
// below 2^50 and 2^48 held exactly in doubles: x = v * 2^96 and the scalings
// by 2^-48 and 2^48 are exact (powers of two), x - h * 2^48 is exact (both are
// multiples of ulp(x), the difference is below 2^48), and truncation to an
// integer rounds nothing else.  Eight such h (or l) add exactly in a double
// (every partial sum is an integer below 2^53), so a run of terms is summed in
// floating point and joined into the 128-bit sum once (fx_join96).
__device__ __forceinline__ void fx_split96(double v, double* h, double* l) {
  const double x = __dmul_rn(v, 0x1p96);
  const double hi = trunc(__dmul_rn(x, 0x1p-48));
  *h = hi;
  *l = trunc(__dsub_rn(x, __dmul_rn(hi, 0x1p48)));
}
__device__ __forceinline__ i128 fx_join96(double h, double l) {
  return (i128)(((u128)__double2ull_rz(h) << 48) + (u128)__double2ull_rz(l));
}
// Signed form: fx_from(v) for |v| < 2 goes to the split accumulators (h, l)
// (fx_split96 of |v|, negated for v < 0; at most eight terms before
// fx_join96s), larger values straight to the 128-bit sum w.
__device__ __forceinline__ void fx_acc96(double v, double& h, double& l, i128& w) {
  const double a = fabs(v);
  if (a < 2.0) {
    double hh, ll;
    fx_split96(a, &hh, &ll);
    if (v < 0.0) {
      hh = -hh;
      ll = -ll;
    }
    h = __dadd_rn(h, hh);
    l = __dadd_rn(l, ll);
  } else {
    w += fx_from(v);
  }
}
__device__ __forceinline__ i128 fx_join96s(double h, double l) {
  return (i128)__double2ll_rz(h) * (i128)281474976710656LL + (i128)__double2ll_rz(l);
}

__device__ __forceinline__ int clz128(u128 u) {
  uint64_t hi = (uint64_t)(u >> 64), lo = (uint64_t)u;
  return hi ? __clzll((long long)hi) : 64 + __clzll((long long)lo);
}

__device__ __forceinline__ double fx_to(i128 s) {
  if (s == 0) return 0.0;
  bool neg = s < 0;
  u128 u = neg ? (u128)0 - (u128)s : (u128)s;
  int msb = 127 - clz128(u);
  double r;
  if (msb <= 52) {
    r = ldexp((double)(uint64_t)u, -kFxFrac);
  } else {
    int sh = msb - 52;
    u128 mant = u >> sh;
    u128 rem = u & (((u128)1 << sh) - 1);
    u128 half = (u128)1 << (sh - 1);
    if (rem > half || (rem == half && (mant & 1))) mant += 1;
    r = ldexp((double)(uint64_t)mant, sh - kFxFrac);
  }
  return neg ? -r : r;
}

__device__ __forceinline__ i128 shfl_down_i128(i128 v, int off) {
  uint64_t lo = (uint64_t)v, hi = (uint64_t)((u128)v >> 64);
  lo = __shfl_down_sync(0xffffffffu, lo, off);
  hi = __shfl_down_sync(0xffffffffu, hi, off);
  return (i128)(((u128)hi << 64) | lo);
}

__device__ __forceinline__ i128 warp_sum_i128(i128 v) {
  for (int off = 16; off > 0; off >>= 1) v += shfl_down_i128(v, off);
  return v;  // valid in lane 0
}

// Block-wide sum of NV 128-bit values; the result is valid in thread 0.
// scratch: NV * (blockDim/32) i128 in shared memory.
template <int NV>
__device__ __forceinline__ void block_sum_i128(i128 (&v)[NV], i128* scratch) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = warp_sum_i128(v[k]);
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) scratch[k * nw + w] = v[k];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      i128 s = 0;
      for (int i = 0; i < nw; ++i) s += scratch[k * nw + i];
      v[k] = s;
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// complex arithmetic without fused multiply-add
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                      __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) {
  return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y));
}
__device__ __forceinline__ double prob(double2 a) {
  return __dadd_rn(__dmul_rn(a.x, a.x), __dmul_rn(a.y, a.y));
}
__device__ __forceinline__ bool cnz(double2 a) { return a.x != 0.0 || a.y != 0.0; }
// the stored amplitude times the pending renormalisation factors
__device__ __forceinline__ double2 scale_load(double2 a, double r0, double r1) {
  a = make_double2(__dmul_rn(a.x, r0), __dmul_rn(a.y, r0));
  return make_double2(__dmul_rn(a.x, r1), __dmul_rn(a.y, r1));
}

// ---------------------------------------------------------------------------
// amplitude storage (bass_state.amp_type)
// ---------------------------------------------------------------------------
// A complex64 entry is read as the double2 of its float parts (exact).  Its
// value with a pending renormalisation is the scaled value rounded back to
// complex64, so every reader sees what the materialised state would hold.
__device__ __forceinline__ double2 f2d(float2 v) { return make_double2((double)v.x, (double)v.y); }
__device__ __forceinline__ float2 d2f(double2 v) {
  return make_float2(__double2float_rn(v.x), __double2float_rn(v.y));
}
__device__ __forceinline__ double2 amp_raw(const double* amps, long long i, int c64) {
  return c64 ? f2d(reinterpret_cast<const float2*>(amps)[i]) : reinterpret_cast<const double2*>(amps)[i];
}
__device__ __forceinline__ double2 amp_scale(double2 raw, int c64, double r0, double r1) {
  const double2 v = scale_load(raw, r0, r1);
  return c64 ? f2d(d2f(v)) : v;
}
__device__ __forceinline__ double2 amp_get(const double* amps, long long i, int c64, double r0, double r1) {
  return amp_scale(amp_raw(amps, i, c64), c64, r0, r1);
}
// stores v (a complex64 state rounds it to float parts)
__device__ __forceinline__ void amp_put(double* amps, long long i, double2 v, int c64) {
  if (c64) reinterpret_cast<float2*>(amps)[i] = d2f(v);
  else reinterpret_cast<double2*>(amps)[i] = v;
}

// FP32 gate arithmetic of complex64 states: the compensated dot product Dot2
// of Ogita, Rump and Oishi ("Accurate sum and dot product", SIAM J. Sci.
// Comput. 26(6), 2005), built from Knuth's TwoSum and the fused-multiply-add
// TwoProduct.  Every product's rounding error and every addition's rounding
// error are carried in a second float and added back once, so a sum of
// complex products is as accurate as if evaluated in twice the precision and
// then rounded to float.
struct Dot2f {
  float s, c;
};
__device__ __forceinline__ void dot2_add(Dot2f& d, float x, float y) {
  const float p = __fmul_rn(x, y);
  const float pe = __fmaf_rn(x, y, -p);  // x*y - p, exactly
  const float t = __fadd_rn(d.s, p);
  const float z = __fsub_rn(t, d.s);
  const float se = __fadd_rn(__fsub_rn(d.s, __fsub_rn(t, z)), __fsub_rn(p, z));  // s + p - t, exactly
  d.s = t;
  d.c = __fadd_rn(d.c, __fadd_rn(pe, se));
}
__device__ __forceinline__ float dot2_get(const Dot2f& d) { return __fadd_rn(d.s, d.c); }
// (re, im) += g * a
__device__ __forceinline__ void cdot2_add(Dot2f& re, Dot2f& im, float2 g, float2 a) {
  dot2_add(re, g.x, a.x);
  dot2_add(re, -g.y, a.y);
  dot2_add(im, g.x, a.y);
  dot2_add(im, g.y, a.x);
}
// g * a of float-valued complex numbers, rounded once to complex64 (as double2)
__device__ __forceinline__ double2 cmul_c64(double2 g, double2 a) {
  Dot2f re{0.f, 0.f}, im{0.f, 0.f};
  cdot2_add(re, im, d2f(g), d2f(a));
  return make_double2((double)dot2_get(re), (double)dot2_get(im));
}

// ---------------------------------------------------------------------------
// keys
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint64_t fmix64(uint64_t z) {
  z ^= z >> 33; z *= 0xff51afd7ed558ccdULL;
  z ^= z >> 33; z *= 0xc4ceb9fe1a85ec53ULL;
  z ^= z >> 33; return z;
}
constexpr uint64_t kFpSalt = 0x5851F42D4C957F2DULL;

// physical key -> true key, given qat[p] = qubit at physical bit p
__device__ __forceinline__ uint64_t true_key(uint64_t y, const int8_t* qat, int nq) {
  uint64_t x = 0;
  while (y) {
    int p = __ffsll((long long)y) - 1;
    x |= 1ULL << qat[p];
    y &= y - 1;
  }
  (void)nq;
  return x;
}

// Move physical bit t down to bit position gb (bits gb..t-1 shift up by one).
// For gb = 0 this is "target to the lowest bit"; for gb = 1 bit 0 stays.
__device__ __forceinline__ uint64_t zmove(uint64_t y, int t, int gb) {
  uint64_t lomask = (1ULL << gb) - 1;
  uint64_t bt = (y >> t) & 1ULL;
  uint64_t hi = (t >= 63) ? 0 : (y >> (t + 1)) << (t + 1);
  uint64_t midm = ((1ULL << t) - 1) & ~lomask;  // bits gb..t-1
  uint64_t mid = y & midm;
  return hi | (mid << 1) | (bt << gb) | (y & lomask);
}

// ---------------------------------------------------------------------------
// warp-cooperative searches (32 probes per step)
// ---------------------------------------------------------------------------
// first index in [lo, hi) where the monotone (true...false) predicate is false
template <class Pred>
__device__ __forceinline__ long long warp_first_false(long long lo, long long hi, Pred pred) {
  const int lane = threadIdx.x & 31;
  while (hi - lo > 32) {
    long long span = hi - lo;
    long long p = lo + (span * (lane + 1)) / 33;
    bool t = pred(p);
    unsigned m = __ballot_sync(0xffffffffu, t);
    int c = __popc(m);
    long long nlo = (c == 0) ? lo : lo + (span * c) / 33 + 1;
    long long nhi = (c == 32) ? hi : lo + (span * (c + 1)) / 33;
    lo = nlo;
    hi = nhi;
  }
  long long p = lo + lane;
  bool t = (p < hi) && pred(p);
  unsigned m = __ballot_sync(0xffffffffu, t);
  return lo + __popc(m);
}

// Three lower bounds on one sorted array in lockstep: lo[k] becomes the first
// index in [lo[k], hi[k]) with keys[i] >= thr[k] (hi[k] if none).  Every round
// each lane probes one position of every unfinished search, so the three
// chains of dependent loads overlap.  Called by all 32 lanes of a warp.
__device__ __forceinline__ void warp_lower_bound3(const uint64_t* keys, long long (&lo)[3], long long (&hi)[3],
                                                  const uint64_t (&thr)[3]) {
  const int lane = threadIdx.x & 31;
  while (hi[0] - lo[0] > 32 || hi[1] - lo[1] > 32 || hi[2] - lo[2] > 32) {
    bool tk[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const long long span = hi[k] - lo[k];
      tk[k] = span > 32 && keys[lo[k] + (span * (lane + 1)) / 33] < thr[k];
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const long long span = hi[k] - lo[k];
      const unsigned m = __ballot_sync(0xffffffffu, tk[k]);
      if (span > 32) {
        const int c = __popc(m);
        const long long nlo = (c == 0) ? lo[k] : lo[k] + (span * c) / 33 + 1;
        const long long nhi = (c == 32) ? hi[k] : lo[k] + (span * (c + 1)) / 33;
        lo[k] = nlo;
        hi[k] = nhi;
      }
    }
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const long long p = lo[k] + lane;
    const bool t = p < hi[k] && keys[p] < thr[k];
    lo[k] += __popc(__ballot_sync(0xffffffffu, t));
  }
}

// Programmatic dependent launch (launch_pdl): wait until the previous
// kernel of the stream has completed and its memory is visible; signal that
// this block's part of the grid no longer needs its SM to itself, so the next
// kernel may be scheduled.  Both are no-ops for a kernel launched normally.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
// Nanosecond wall clock of the GPU (profiling of phases inside one launch).
__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// One galloping round before warp_lower_bound3, for three searches whose
// answers lie near a known position P: lanes 10k .. 10k + 9 probe P -/+ 4^l
// (l = 0..9) for search k, backwards when back[k] (the answer is at or before
// P) and forwards otherwise (the answer is after P), and [lo[k], hi[k]) shrinks
// to the bracket between the nearest probe on the far side of the answer and
// the one before it.  Probes outside [lo[k], hi[k]) count as far side and
// load nothing.  Called by all 32 lanes of a warp.
__device__ __forceinline__ void warp_bracket3(const uint64_t* keys, long long P, long long (&lo)[3],
                                              long long (&hi)[3], const uint64_t (&thr)[3],
                                              const bool (&back)[3]) {
  const int lane = threadIdx.x & 31;
  const int k = lane / 10, l = lane - 10 * k;
  bool far = false;
#pragma unroll
  for (int kk = 0; kk < 3; ++kk) {
    if (k == kk) {
      const long long d = 1LL << (2 * l);
      if (back[kk]) {
        const long long pos = P - d;
        far = pos < lo[kk] || keys[pos] < thr[kk];
      } else {
        const long long pos = P + d;
        far = pos >= hi[kk] || keys[pos] >= thr[kk];
      }
    }
  }
  const unsigned m = __ballot_sync(0xffffffffu, far);
#pragma unroll
  for (int kk = 0; kk < 3; ++kk) {
    const unsigned mk = (m >> (10 * kk)) & 0x3FFu;
    long long nlo, nhi;
    if (mk) {
      const int l0 = __ffs(mk) - 1;
      const long long dfar = 1LL << (2 * l0), dnear = l0 ? 1LL << (2 * (l0 - 1)) : 0;
      if (back[kk]) {
        nlo = P - dfar + 1;
        nhi = P - dnear + 1;
      } else {
        nlo = P + dnear + 1;
        nhi = P + dfar + 1;
      }
    } else if (back[kk]) {
      nlo = lo[kk];
      nhi = P - (1LL << 18) + 1;
    } else {
      nlo = P + (1LL << 18) + 1;
      nhi = hi[kk];
    }
    if (nlo > lo[kk]) lo[kk] = nlo;
    if (nhi < hi[kk]) hi[kk] = nhi;
    if (lo[kk] > hi[kk]) lo[kk] = hi[kk];
  }
}

// ---------------------------------------------------------------------------
// decoupled look-back (exclusive prefix of per-tile counts)
// status word: bits 62-63 flag (1 aggregate, 2 inclusive), bits 0-61 value
// ---------------------------------------------------------------------------
constexpr unsigned long long kFlagAgg = 1ULL << 62;
constexpr unsigned long long kFlagInc = 2ULL << 62;
constexpr unsigned long long kValMask = (1ULL << 62) - 1;

__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
// Atomic add with release semantics at GPU scope, no value returned.
__device__ __forceinline__ void red_release_add(unsigned long long* p, unsigned long long v) {
  asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void st_release(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Called by one thread.  Returns the exclusive prefix of tile `tile`.
__device__ __forceinline__ long long lookback(unsigned long long* status, long long tile,
                                              long long agg, bass_ctrl* ctrl) {
  if (tile == 0) {
    st_release(&status[0], kFlagInc | (unsigned long long)agg);
    return 0;
  }
  st_release(&status[tile], kFlagAgg | (unsigned long long)agg);
  long long excl = 0;
  long long k = tile - 1;
  long long spins = 0;
  const long long lim = wait_limit(ctrl);
  while (true) {
    unsigned long long s = ld_acquire(&status[k]);
    if ((s >> 62) == 0) {
      if (++spins > lim) {
        set_error(ctrl, BASS_ERR_WAIT);
        break;
      }
      continue;
    }
    excl += (long long)(s & kValMask);
    if ((s >> 62) == 2) break;
    if (k == 0) break;
    --k;
  }
  st_release(&status[tile], kFlagInc | (unsigned long long)(excl + agg));
  return excl;
}

// Called by all 32 lanes of one warp; returns the exclusive prefix of `tile`
// in every lane.  Each step reads the status words of the 32 nearest
// predecessors at once, sums their aggregates up to the nearest inclusive one
// and stops there, so a tile walks back 32 tiles per dependent load.
__device__ __forceinline__ long long lookback_warp(unsigned long long* status, long long tile,
                                                   long long agg, bass_ctrl* ctrl) {
  const int lane = threadIdx.x & 31;
  if (tile == 0) {
    if (lane == 0) st_release(&status[0], kFlagInc | (unsigned long long)agg);
    return 0;
  }
  if (lane == 0) st_release(&status[tile], kFlagAgg | (unsigned long long)agg);
  long long excl = 0;
  long long base = tile - 1;
  long long spins = 0;
  bool gave_up = false;
  const long long lim = wait_limit(ctrl);
  while (true) {
    const long long k = base - lane;
    unsigned long long s;
    do {
      s = (k >= 0 && !gave_up) ? ld_acquire(&status[k]) : kFlagInc;
      if (++spins > lim) gave_up = true;
    } while (__any_sync(0xffffffffu, (s >> 62) == 0));
    const unsigned inc = __ballot_sync(0xffffffffu, (s >> 62) == 2);
    const int stop = inc ? __ffs(inc) - 1 : 32;
    long long v = (lane <= stop) ? (long long)(s & kValMask) : 0;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    excl += __shfl_sync(0xffffffffu, v, 0);
    if (inc) break;
    base -= 32;
  }
  if (gave_up && lane == 0) set_error(ctrl, BASS_ERR_WAIT);
  if (lane == 0) st_release(&status[tile], kFlagInc | (unsigned long long)(excl + agg));
  return excl;
}


// ---------------------------------------------------------------------------
// workspace
// ---------------------------------------------------------------------------
// tiles of an op: merge kinds step by kStep, the plain (K_IDENT) kind by kTile
__host__ __device__ __forceinline__ long long merge_tiles(long long n) { return (n + kStep - 1) / kStep; }
__host__ __device__ __forceinline__ long long plain_tiles(long long n) { return (n + kTile - 1) / kTile; }

struct Partial {
  i128 s[4];
  long long c[2];
  long long pad[2];
};

struct SelState {
  long long n_out;       // children produced by the op (after drop rules)
  long long k_keep;
  long long n_cand;      // children of the level-2 boundary bin (slot indices in ws.cand_bits)
  unsigned long long t_bits;
  unsigned long long t_key;  // ~0: every child at t_bits kept; else the largest kept true key there
  int do_trunc;
  int stage;             // 0 keep all, 3 threshold resolved
  int pad;               // K_IDENT guard: a zero amplitude was produced
  double total;          // exact sum of |a|^2 over the op's output (truncating ops only)
  long long n_written;
  double kept;           // exact sum of |a|^2 over the kept children
  double kept_p2;        // ... of |a|^4 (rotation steps)
  int skip_write;        // the write pass has nothing to do (rejected rotation)
  int accept;            // rotation step: the candidate lowers PR
  double pr_new;         // rotation step: PR of the candidate
  int8_t qat[64];        // output qubit order, for the key tie-break at t_bits
};

struct WsView {
  long long* part;               // kMaxSets x (max_tiles + 1) x 6
  unsigned long long* status;    // max_tiles
  unsigned int* hist1;           // kHistBins bins, then kHistGroups coarse counts
  unsigned int* hist2;           // kHistBins bins, then kHistGroups coarse counts
  Partial* partials;             // kMaxSets x max_tiles
  unsigned long long* cand_bits; // max_n: slot indices (boundary-bin candidates of a selection)
  unsigned long long* cand_key;  // max_n
  SelState* sel;
  unsigned int* counters;        // 64 tile counters
  uint64_t* tmp_keys;            // max_n; gate ops: the slot array (|a|^2 bits per child)
  double2* tmp_amps;             // max_n; gate ops: the staged children's amplitudes
  uint64_t* stage_keys;          // max_n; gate ops: the staged children's keys
  uint8_t* kmask;                // max_n / 8 + 64: one bit per slot, kept by the selection (bit
                                 // i & 7 of byte i >> 3; the count pass, then the boundary settle)
  unsigned int* sort_hist;       // radix-sort tile histograms (256 x max_tiles)
  i128* red;                     // 1024 per-CTA reduction partials
  unsigned long long* fp;        // 8 fingerprint accumulators
  long long max_n;
  long long max_tiles;
  long long sort_tiles;
};

}  // namespace bass
