// merge.cu -- the pairing pipeline of libbass_b200.
//
// A state is sorted by physical key.  An op acting on qubit q (physical bit t)
// reads the state in "Z order": the order of zmove(key, t, gb), which brings
// bit t down to bit gb so that the entries a gate combines (keys that differ
// only in the gate's bits) become adjacent.  Within a block of keys sharing the
// bits above t, Z order is the merge of the block's bit-t-clear run and its
// bit-t-set run, so one merge pass pairs every entry with its partners:
//
//   k_partition   one warp per tile boundary: finds the block of the boundary
//                 and the merge-path split inside it (warp-cooperative
//                 32-ary searches), then backs the boundary off to the start of
//                 its group so that no group straddles two tiles;
//   k_tile        loads a tile's (at most five) contiguous input segments,
//                 splits them by bit t and merges them in shared memory, then
//                 evaluates every group (gate / rotation / permutation / RDM
//                 moments); the evaluation pass stages every child (|a|^2 bit
//                 pattern, key, amplitude) at its slot index;
//   k_select_coop one-launch selection (grid barriers): radix select of the top-k threshold
//                 on the IEEE bits of |a|^2 (13-bit digits, then an exact
//                 (|a|^2 desc, key asc) ordering of the boundary candidates),
//                 survivors per tile, exact sums, rotation decision, tile scan;
//   k_compact     copies the surviving staged children to their tile's offset;
//   finalize_op   (last CTA of the write step) output descriptor (count, new
//                 bit order, pending renormalisation) and the gamma /
//                 truncation bookkeeping.
//
// The output is again sorted by its (new) physical key: children of a group
// are emitted in child-index order, groups in Z order.
#include <math.h>

#include <atomic>

#include "internal.h"

namespace bass {

struct Hdr {
  const uint64_t* keys;
  const double2* amps;
  long long n;
  long long ntiles;
  double r0, r1;
  int t;
  int nq;
  int c64;  // the state stores complex64 amplitudes
  int8_t qat_out[64];
};

// The blocks of a launch that work on one op.  A plain launch is one group
// (blockIdx.x of gridDim.x); a segmented launch (one op on each of many
// states) splits its grid into one group per state, see seg_enter.
struct Grp {
  int bid;   // block index within the group
  int nblk;  // blocks in the group
};
__device__ __forceinline__ Grp whole_grid() { return Grp{(int)blockIdx.x, (int)gridDim.x}; }

// The op's output qubit order: the input's, with the target qubit's
// position t = pos[q] moved down to gb (positions gb..t-1 move up by one) for
// the kinds that bring a target to the low bits.  One position per thread
// (threads 0-63 of the block); the caller synchronises before reading it.
__device__ __forceinline__ void out_order_par(const bass_state* in, int kind, int q, int gb, int8_t* qat_out) {
  const int p = threadIdx.x;
  if (p < 64) {
    int src = p;
    if (kind == K_GATE1 || kind == K_ROT1 || kind == K_GATE2 || kind == K_PERM) {
      const int t = in->pos[q];
      if (p > gb && p <= t) src = p - 1;
      if (p == gb) src = t;
    }
    qat_out[p] = in->qat[src];
  }
}

// ---------------------------------------------------------------------------
// partition
// ---------------------------------------------------------------------------
// record per boundary: P' (adjusted Z position), s, mid, e (block bounds), i, j
// zero: also clear the op's small workspace region (what zero_small clears);
// nothing here reads it, and the kernels after the partition find it zeroed.
// The op's small workspace region (tile counters, histograms, selection
// state, look-back status words: what zero_small clears), zeroed by a group.
__device__ __forceinline__ void zero_op_region(const OpArgs& a, Grp g) {
  unsigned long long* zp = reinterpret_cast<unsigned long long*>(a.ws.counters);
  const long long nw =
      (long long)((reinterpret_cast<const char*>(a.ws.status + a.ws.max_tiles) - reinterpret_cast<const char*>(zp)) / 8);
  for (long long i = (long long)g.bid * blockDim.x + threadIdx.x; i < nw; i += (long long)g.nblk * blockDim.x)
    zp[i] = 0ULL;
}

__device__ __forceinline__ void partition_body(const OpArgs& a, int kind, int zero, int set, Grp g) {
  if (zero && set == 0) zero_op_region(a, g);
  const bass_state* in = a.in;
  const long long n = in->nnz;
  const int q = (kind == K_RDM) ? set : a.q;
  const int t = in->pos[q];
  if (kind == K_RDM && a.rdm_low && t < kRdmLowBits) return;  // paired by k_rdm_low
  const int gb = a.gb;
  const int sh = gb + 1;
  const uint64_t* keys = in->keys;
  const long long ntiles = merge_tiles(n);
  long long* recs = a.ws.part + (long long)set * (a.ws.max_tiles + 1) * 6;
  const int lane = threadIdx.x & 31;
  const long long warp = ((long long)g.bid * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)g.nblk * blockDim.x) >> 5;
  if (ntiles + 1 > a.ws.max_tiles + 1) {
    if (warp == 0 && lane == 0) set_error(a.ctrl, BASS_ERR_WORKSPACE);
    return;
  }
  for (long long b = warp; b <= ntiles; b += nwarps) {
    const long long P = b * kStep;
    long long r0, r1, r2, r3, r4, r5;
    if (P >= n) {
      r0 = n; r1 = n; r2 = n; r3 = n; r4 = 0; r5 = 0;
    } else {
      const uint64_t y = keys[P];
      const uint64_t lo_key = (y >> (t + 1)) << (t + 1);
      const uint64_t mid_key = lo_key | (1ULL << t);
      const uint64_t hi_key = lo_key + (2ULL << t);
      const bool hi_ovf = hi_key <= lo_key;
      // block start, run split and block end in one lockstep search
      long long lo3[3] = {0, ((y >> t) & 1ULL) ? 0 : P + 1, hi_ovf ? n : P + 1};
      long long hi3[3] = {P + 1, ((y >> t) & 1ULL) ? P + 1 : n, n};
      const uint64_t thr3[3] = {lo_key, mid_key, hi_key};
      const bool back3[3] = {true, ((y >> t) & 1ULL) != 0, false};
      warp_bracket3(keys, P, lo3, hi3, thr3, back3);
      warp_lower_bound3(keys, lo3, hi3, thr3);
      const long long s = lo3[0], mid = lo3[1], e = lo3[2];
      const long long d = P - s, len0 = mid - s, len1 = e - mid;
      long long lo = d - len1 > 0 ? d - len1 : 0;
      long long hi = d < len0 ? d : len0;
      long long i = warp_first_false(lo, hi, [&](long long m) {
        return zmove(keys[s + m], t, gb) < zmove(keys[mid + d - 1 - m], t, gb);
      });
      long long j = d - i;
      if (kind != K_PERM) {
        // back the boundary off to the start of its group: the two entries
        // at the split and the two before it in each run, fetched at once
        long long idx = -1;
        if (lane == 0 && i < len0) idx = s + i;
        if (lane == 1 && j < len1) idx = mid + j;
        if (lane == 2 && i >= 1) idx = s + i - 1;
        if (lane == 3 && i >= 2) idx = s + i - 2;
        if (lane == 4 && j >= 1) idx = mid + j - 1;
        if (lane == 5 && j >= 2) idx = mid + j - 2;
        const uint64_t zv = (idx >= 0) ? zmove(keys[idx], t, gb) : ~0ULL;
        const uint64_t z0 = __shfl_sync(0xffffffffu, zv, 0), z1 = __shfl_sync(0xffffffffu, zv, 1);
        const uint64_t a1 = __shfl_sync(0xffffffffu, zv, 2), a2 = __shfl_sync(0xffffffffu, zv, 3);
        const uint64_t c1 = __shfl_sync(0xffffffffu, zv, 4), c2 = __shfl_sync(0xffffffffu, zv, 5);
        const uint64_t gid = (z0 < z1 ? z0 : z1) >> sh;
        int b0 = 0, b1 = 0;
        if (i >= 1 && (a1 >> sh) == gid) b0 = (i >= 2 && (a2 >> sh) == gid) ? 2 : 1;
        if (j >= 1 && (c1 >> sh) == gid) b1 = (j >= 2 && (c2 >> sh) == gid) ? 2 : 1;
        i -= b0;
        j -= b1;
      }
      r0 = s + i + j; r1 = s; r2 = mid; r3 = e; r4 = i; r5 = j;
    }
    if (lane == 0) {
      long long* r = recs + b * 6;
      r[0] = r0; r[1] = r1; r[2] = r2; r[3] = r3; r[4] = r4; r[5] = r5;
    }
  }
  pdl_trigger();
}

__global__ void k_partition(const __grid_constant__ OpArgs a, int kind, int zero) {
  pdl_wait();
  partition_body(a, kind, zero, blockIdx.y, whole_grid());
}

// ---------------------------------------------------------------------------
// block scan
// ---------------------------------------------------------------------------
__device__ __forceinline__ int block_excl_scan(int v, int* sWarp, int* total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int x = v;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, off);
    if (lane >= off) x += y;
  }
  if (lane == 31) sWarp[w] = x;
  __syncthreads();
  if (w == 0) {
    int s = (lane < nw) ? sWarp[lane] : 0;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, s, off);
      if (lane >= off) s += y;
    }
    if (lane < nw) sWarp[lane] = s;
  }
  __syncthreads();
  int excl = x - v + (w > 0 ? sWarp[w - 1] : 0);
  *total = sWarp[nw - 1];
  __syncthreads();
  return excl;
}

// ---------------------------------------------------------------------------
// groups -> children
// ---------------------------------------------------------------------------
// entries per group / children per group of each kind
template <int KIND>
struct KindTraits {
  static constexpr int kMaxChildren = (KIND == K_GATE2) ? 4 : (KIND == K_GATE1 || KIND == K_ROT1) ? 2 : 1;
};

// Children of the group whose first Z-ordered entry is at position p of the
// Z-ordered tile.  Returns the mask of children that exist (0 if p does not
// start a group); child o has the new physical key base | o and amplitude
// ca[o].  Within a group, entries are in ascending local index, so the sums
// run over the local index in ascending order.
// The rotation's drop rule hypot(re, im) > 1e-30 (bass_simulator.py:156-199),
// decided without calling hypot outside a narrow band: hypot lies between
// max(|re|, |im|) and sqrt(2) max(|re|, |im|) (within its last-place error),
// so the answer is known unless max is within [7e-31, 1e-30].
__device__ __forceinline__ bool above_drop(double2 c) {
  if (c.x != c.x || c.y != c.y) return hypot(c.x, c.y) > 1e-30;  // NaN: as hypot decides
  const double m = fmax(fabs(c.x), fabs(c.y));
  if (m > 1e-30) return true;
  if (m < 7e-31) return false;
  return hypot(c.x, c.y) > 1e-30;
}

// The tile's amplitudes as the evaluation sees them: stored in load order,
// read at Z position p through the merge's permutation (identity when there
// is none), with the state's pending renormalisation applied.
struct AmpView {
  const double2* sA;   // complex128 amplitudes in load order, or
  const float2* sAf;   // complex64 amplitudes (c64)
  const uint16_t* sP;  // Z position -> load position, or nullptr
  double r0, r1;
  bool scaled;
  bool c64;
  __device__ __forceinline__ double2 operator()(int p) const {
    const int q = sP ? (int)sP[p] : p;
    const double2 v = c64 ? f2d(sAf[q]) : sA[q];
    return scaled ? amp_scale(v, c64 ? 1 : 0, r0, r1) : v;
  }
};

// The children of the group that starts at Z position p (0 if p does not
// start one).  G is the op's gate matrix, read from the kernel's parameter
// block (k_tile takes its arguments as a __grid_constant__), so every lane
// loads the same constant-bank words.
template <int KIND, bool F32>
__device__ __forceinline__ unsigned group_children(int p, int E, const uint64_t* sZ, const AmpView& sA, int gb,
                                                   const double2* G, int drop_zero, uint64_t* base,
                                                   double2* ca) {
  constexpr int NC = KindTraits<KIND>::kMaxChildren;
  const uint64_t z = sZ[p];
  if (KIND == K_PERM || KIND == K_IDENT) {
    const double2 v = sA(p);
    if (KIND == K_IDENT && drop_zero && !cnz(v)) return 0u;
    *base = z;
    ca[0] = v;
    return 1u;
  }
  const int sh = gb + 1;
  const uint64_t gid = z >> sh;
  if (p > 0 && (sZ[p - 1] >> sh) == gid) return 0u;
  *base = gid << sh;
  double2 ar[NC];
  int lr[NC];
#pragma unroll
  for (int r = 0; r < NC; ++r) {
    const uint64_t zr = (p + r < E) ? sZ[p + r] : ~0ULL;
    const bool in = (p + r < E) && (zr >> sh) == gid;
    lr[r] = in ? (int)(zr & ((1u << sh) - 1)) : -1;
    ar[r] = in ? sA(p + r) : make_double2(0.0, 0.0);
  }
  unsigned mask = 0;
  if (F32) {
    // complex64: float gate entries and amplitudes, compensated FP32 sums
    // (Dot2); a contribution counts when neither factor is zero
    if (KIND == K_GATE1 || KIND == K_GATE2) {
#pragma unroll
      for (int o = 0; o < NC; ++o) {
        Dot2f re{0.f, 0.f}, im{0.f, 0.f};
        bool have = false;
#pragma unroll
        for (int r = 0; r < NC; ++r) {
          if (lr[r] < 0) continue;
          const float2 g = d2f(G[o * NC + lr[r]]), x = d2f(ar[r]);
          if (!((g.x != 0.f || g.y != 0.f) && (x.x != 0.f || x.y != 0.f))) continue;
          cdot2_add(re, im, g, x);
          have = true;
        }
        const double2 acc = make_double2((double)dot2_get(re), (double)dot2_get(im));
        ca[o] = acc;
        if (drop_zero == 2 ? above_drop(acc) : have) mask |= 1u << o;
      }
    } else if (KIND == K_ROT1) {
      const float2 zero = make_float2(0.f, 0.f);
      const float2 a0 = (lr[0] == 0) ? d2f(ar[0]) : zero;
      const float2 a1 = (lr[0] == 1) ? d2f(ar[0]) : (lr[1] == 1 ? d2f(ar[1]) : zero);
#pragma unroll
      for (int o = 0; o < 2; ++o) {
        Dot2f re{0.f, 0.f}, im{0.f, 0.f};
        cdot2_add(re, im, d2f(G[o * 2]), a0);
        cdot2_add(re, im, d2f(G[o * 2 + 1]), a1);
        const double2 c = make_double2((double)dot2_get(re), (double)dot2_get(im));
        ca[o] = c;
        if (above_drop(c)) mask |= 1u << o;
      }
    }
    return mask;
  }
  if (KIND == K_GATE1 || KIND == K_GATE2) {
#pragma unroll
    for (int o = 0; o < NC; ++o) {
      double2 acc = make_double2(0.0, 0.0);
      bool have = false;
#pragma unroll
      for (int r = 0; r < NC; ++r) {
        if (lr[r] < 0) continue;
        const double2 pr = cmul(G[o * NC + lr[r]], ar[r]);
        if (!cnz(pr)) continue;
        acc = have ? cadd(acc, pr) : pr;
        have = true;
      }
      ca[o] = acc;
      // drop_zero 2 (a 2-qubit rotation): the rotation's rule |a| > 1e-30
      // (bass_simulator.py:275) instead of "some product was non-zero"
      if (drop_zero == 2 ? above_drop(acc) : have) mask |= 1u << o;
    }
  } else if (KIND == K_ROT1) {
    const double2 zero = make_double2(0.0, 0.0);
    const double2 a0 = (lr[0] == 0) ? ar[0] : zero;
    const double2 a1 = (lr[0] == 1) ? ar[0] : (lr[1] == 1 ? ar[1] : zero);
#pragma unroll
    for (int o = 0; o < 2; ++o) {
      const double2 c = cadd(cmul(G[o * 2], a0), cmul(G[o * 2 + 1], a1));
      ca[o] = c;
      if (above_drop(c)) mask |= 1u << o;
    }
  }
  return mask;
}

// group_children for the state's amplitude type
template <int KIND>
__device__ __forceinline__ unsigned group_children_t(bool c64, int p, int E, const uint64_t* sZ, const AmpView& sA,
                                                     int gb, const double2* G, int drop_zero, uint64_t* base,
                                                     double2* ca) {
  return c64 ? group_children<KIND, true>(p, E, sZ, sA, gb, G, drop_zero, base, ca)
             : group_children<KIND, false>(p, E, sZ, sA, gb, G, drop_zero, base, ca);
}

__device__ __forceinline__ bool keep_child(uint64_t bits, uint64_t key, const SelState& S,
                                           const int8_t* qat) {
  if (!S.do_trunc) return true;
  if (bits > S.t_bits) return true;
  if (bits < S.t_bits) return false;
  return S.t_key == ~0ULL || true_key(key, qat, 64) <= S.t_key;
}

// Does the child with this slot survive the selection?  (T, incl) = (t_bits,
// t_key == ~0) when truncating, (0, true) otherwise.  With incl false the
// children at exactly T are settled by true key (keep_child, and k_compact's
// check against t_key).
__device__ __forceinline__ bool slot_kept(unsigned long long bits, unsigned long long T, bool incl) {
  return bits != ~0ULL && (bits > T || (incl && bits == T));
}

__host__ __device__ constexpr int slots_per_entry(int kind) {
  return kind == K_GATE2 ? 4 : (kind == K_GATE1 || kind == K_ROT1) ? 2 : 1;
}

// ---------------------------------------------------------------------------
// finalisation
// ---------------------------------------------------------------------------
// mode 0: plain op; mode 1: basis-rotation step (always renormalises, keeps
// the retained mass in sel->kept for the decision)
// The kept mass comes from the selection's final phase (set when the op
// truncates or is a rotation step, the only cases that use it).
// One thread.  Runs in the last CTA of the write pass to finish, so the
// selection's results (written by the previous kernel) and n_written (written
// by the CTA of the last tile, before its fence) are read through volatile.
// The output's qubit order is written by write_done.
__device__ void finalize_op(const OpArgs& a, const bass_trunc& tr, int mode, int kind) {
  volatile SelState* sel = a.ws.sel;
  const bass_state* in = a.in;
  bass_state* out = a.out;
  bass_ctrl* c = a.ctrl;
  const double kept = sel->kept;
  const long long n_in = in->nnz;
  long long nw = sel->n_written;
  if (nw > out->cap) {  // the write pass skipped the tiles that did not fit
    set_error(c, BASS_ERR_CAPACITY);
    nw = 0;
  }
  out->nq = in->nq;
  out->amp_type = in->amp_type;
  out->nnz = nw;
  out->rscale[0] = 1.0;
  out->rscale[1] = 1.0;
  if (kind == K_PERM) return;  // first pass of a 2-qubit gate: no bookkeeping
  // an amplitude update is an input entry of a gate or a rotation step; a
  // plain truncation (K_IDENT) transforms nothing
  if (kind != K_IDENT) c->amp_updates += n_in;
  c->n_ops += 1;
  const int trunc = sel->do_trunc;
  if (mode == 1) {
    const double nrm = sqrt(kept);
    if (nrm > 1e-30) out->rscale[0] = 1.0 / nrm;
    return;
  }
  c->last_truncated = trunc;
  if (!trunc) return;
  const double total = sel->total;
  c->last_kept = kept;
  c->last_total = total;
  c->n_trunc += 1;
  if (tr.gamma_mode == 1) c->gamma_running *= (total > 1e-30 ? kept / total : 0.0);
  else if (tr.gamma_mode == 2) c->state_gamma *= (total > 1e-30 ? sqrt(kept / total) : 0.0);
  else if (tr.gamma_mode == 3) c->state_gamma *= sqrt(kept);
  if (tr.renorm == 1) {
    const double nrm = sqrt(kept);
    if (nrm > 1e-30) out->rscale[0] = 1.0 / nrm;
  } else if (tr.renorm == 2) {
    out->rscale[0] = 1.0 / sqrt(kept);
  }
  if (tr.mark_active) {
    c->truncation_active = 1;
    c->gates_since_trunc = 0;
  }
}

// Block-wide, at the end of a write pass: the last CTA to arrive writes the
// output descriptor (its qubit order one position per thread, the rest by
// finalize_op).
__device__ void write_done(const OpArgs& a, int kind, Grp g) {
  __shared__ int sLastW;
  __shared__ int8_t sQo[64];
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned long long d = atomicAdd(&reinterpret_cast<unsigned long long*>(a.ws.counters)[59], 1ULL);
    sLastW = (d == (unsigned long long)g.nblk - 1);
  }
  __syncthreads();
  if (!sLastW) return;
  __threadfence();
  out_order_par(a.in, kind, a.q, a.gb, sQo);
  __syncthreads();
  if (threadIdx.x == 0) finalize_op(a, a.tr, a.fin_mode, kind);
  if (threadIdx.x < 64) {
    a.out->qat[threadIdx.x] = sQo[threadIdx.x];
    a.out->pos[sQo[threadIdx.x]] = (int8_t)threadIdx.x;
  }
  if (!a.commit) return;
  // rotation step without a trace: k_commit's work, here.  An accepted
  // candidate (a.out) becomes the state (a.in): the two descriptors are
  // swapped one 8-byte word per thread.
  __syncthreads();
  const volatile SelState* sel = a.ws.sel;
  if (!sel->accept) return;
  constexpr int kWords = (int)(sizeof(bass_state) / 8);
  static_assert(sizeof(bass_state) % 8 == 0, "descriptor words");
  unsigned long long* pc = reinterpret_cast<unsigned long long*>(const_cast<bass_state*>(a.in));
  unsigned long long* pt = reinterpret_cast<unsigned long long*>(a.out);
  unsigned long long wc = 0, wt = 0;
  if (threadIdx.x < kWords) {
    wc = pc[threadIdx.x];
    wt = pt[threadIdx.x];
  }
  __syncthreads();
  if (threadIdx.x < kWords) {
    pc[threadIdx.x] = wt;
    pt[threadIdx.x] = wc;
  }
  if (threadIdx.x == 0) {
    bass_ctrl* c = a.ctrl;
    c->pr_cur = sel->pr_new;
    const double frac = c->frac[a.j];
    c->gamma_running *= sqrt(frac > 1e-30 ? frac : 0.0);
  }
}

// The selection state into shared memory, one 8-byte word per thread (the
// caller synchronises before reading it).
__device__ __forceinline__ void load_sel(SelState* dst, const SelState* src) {
  constexpr int kWords = (int)(sizeof(SelState) / 8);
  static_assert(sizeof(SelState) % 8 == 0, "selection state words");
  if ((int)threadIdx.x < kWords)
    reinterpret_cast<unsigned long long*>(dst)[threadIdx.x] =
        __ldcg(reinterpret_cast<const unsigned long long*>(src) + threadIdx.x);
}

// ---------------------------------------------------------------------------
// the tile kernel
// ---------------------------------------------------------------------------
// Passes: P_HIST (evaluate every child once: its |a|^2 bits go to the slot
// array, its key and amplitude to the staging arrays at the same index, plus
// the child count), P_WRITE (the first pass of a 2-qubit gate, one child per
// entry, and the compaction after a diagonal 1-qubit gate), P_RDM (per-qubit
// moments).
template <int KIND, int PASS, bool C64>
__device__ __forceinline__ void tile_body(const OpArgs& a, Grp g) {
  extern __shared__ __align__(16) unsigned char smem[];
  double2* sA = reinterpret_cast<double2*>(smem);
  uint64_t* sZ = reinterpret_cast<uint64_t*>(sA + kTilePad);
  uint16_t* sIdx = reinterpret_cast<uint16_t*>(sZ + kTilePad);
  uint16_t* sPerm = sIdx;  // after the merge: Z position -> load position
  // write pass only: per-position offsets and kept masks
  uint16_t* sOff = sIdx + kTilePad;
  uint8_t* sMask = reinterpret_cast<uint8_t*>(sOff + kTilePad);
  __shared__ Hdr H;
  __shared__ SelState S;
  __shared__ long long sItem, sBase, sZstart;
  __shared__ long long sSegLo[5], sSegOff[6];
  __shared__ int sSegPos[5], sGap[5];
  __shared__ uint64_t sBar;  // completion of the tile's bulk copies
  __shared__ int sWarp[32];
  __shared__ i128 sRed[4 * (kThreads / 32)];

  const int tid = threadIdx.x;
  load_sel(&S, a.ws.sel);
  __syncthreads();
  if (KIND == K_IDENT && a.guard && S.pad == 0) return;
  // a rejected rotation candidate is not written (the descriptor still is)
  const bool skip = PASS == P_WRITE && S.skip_write;

  if (tid == 0) {
    const bass_state* in = a.in;
    H.keys = in->keys;
    H.amps = reinterpret_cast<const double2*>(in->amps);
    H.n = in->nnz;
    H.r0 = in->rscale[0];
    H.r1 = in->rscale[1];
    H.nq = in->nq;
    H.c64 = in->amp_type == BASS_AMP_C64;
    if (H.c64 != (int)C64) set_error(a.ctrl, BASS_ERR_ARG);  // launched for the other amplitude type
    H.t = (KIND == K_IDENT || KIND == K_RDM) ? 0 : in->pos[a.q];
    H.ntiles = (KIND == K_IDENT) ? plain_tiles(H.n) : merge_tiles(H.n);
    mbar_init(&sBar, 1);
  }
  out_order_par(a.in, KIND, a.q, a.gb, H.qat_out);
  __syncthreads();
  // bulk copies need 16-byte aligned arrays (every allocation of this library
  // is; a caller's arrays at an 8-byte offset take the per-entry copies)
  const bool tma = ((reinterpret_cast<uintptr_t>(H.keys) | reinterpret_cast<uintptr_t>(H.amps)) & 15) == 0;
  constexpr unsigned kAmpBytes = C64 ? 8u : 16u;
  unsigned phase = 0;  // parity of sBar's current phase

  const int gb = a.gb;
  const long long ntiles = H.ntiles;
  constexpr int NS = slots_per_entry(KIND);
  const bool bad = ntiles > a.ws.max_tiles || (PASS == P_HIST && (long long)NS * H.n > a.ws.max_n) ||
                   H.c64 != (int)C64;
  if (bad && g.bid == 0 && tid == 0) set_error(a.ctrl, BASS_ERR_WORKSPACE);
  if (bad && PASS != P_WRITE) return;
  const bool scaled = !(H.r0 == 1.0 && H.r1 == 1.0);
  // P_RDM: items are (set, tile); K_RDM sets are qubits, the 4x4 moments of
  // a qubit pair (K_GATE2) split into a.nsets = 4 sets of four values that
  // share one partition
  // P_RDM of K_RDM with rdm_low: the items cover only the sets whose qubit
  // sits at physical bit kRdmLowBits or above (sHigh, the same list in every
  // CTA); k_rdm_low does the others
  __shared__ int8_t sHigh[64];
  __shared__ int sNHigh;
  if (PASS == P_RDM && tid == 0) {
    int nh = 0;
    for (int s2 = 0; s2 < a.nsets && s2 < 64; ++s2)
      if (!(KIND == K_RDM && a.rdm_low && a.in->pos[a.q + s2] < kRdmLowBits)) sHigh[nh++] = (int8_t)s2;
    sNHigh = nh;
  }
  __syncthreads();
  const long long nitems = (bad || skip) ? 0 : (PASS == P_RDM) ? ntiles * sNHigh : ntiles;
  long long cnt = 0;
  const int base_e = tid * kPerThread;

  for (;;) {
    if (tid == 0) sItem = (long long)atomicAdd(&reinterpret_cast<unsigned long long*>(a.ws.counters)[a.counter], 1ULL);
    __syncthreads();
    const long long item = sItem;
    if (item >= nitems) break;
    const int set = (PASS == P_RDM) ? (int)sHigh[item / ntiles] : 0;
    const long long tile = (PASS == P_RDM) ? item % ntiles : item;
    const int t = (KIND == K_RDM) ? a.in->pos[a.q + set] : H.t;
    const int pset = (KIND == K_RDM) ? set : 0;  // the partition records this item reads

    // ---- segments ---------------------------------------------------------
    if (tid == 0) {
      long long lo[5] = {0, 0, 0, 0, 0}, len[5] = {0, 0, 0, 0, 0};
      long long zs;
      if (KIND == K_IDENT) {
        lo[0] = tile * kTile;
        len[0] = (H.n - lo[0] < kTile) ? H.n - lo[0] : kTile;
        zs = lo[0];
      } else {
        const long long* rc = a.ws.part + ((long long)pset * (a.ws.max_tiles + 1) + tile) * 6;
        const long long* rn = rc + 6;
        zs = rc[0];
        if (rc[1] == rn[1]) {
          lo[0] = rc[1] + rc[4]; len[0] = rn[4] - rc[4];
          lo[1] = rc[2] + rc[5]; len[1] = rn[5] - rc[5];
        } else {
          lo[0] = rc[1] + rc[4]; len[0] = rc[2] - lo[0];
          lo[1] = rc[2] + rc[5]; len[1] = rc[3] - lo[1];
          lo[2] = rc[3];         len[2] = rn[1] - rc[3];
          lo[3] = rn[1];         len[3] = rn[4];
          lo[4] = rn[2];         len[4] = rn[5];
        }
      }
      long long o = 0;
      bool bad = false;
      for (int k = 0; k < 5; ++k) {
        if (len[k] < 0 || lo[k] < 0 || lo[k] + len[k] > H.n) { len[k] = 0; bad = true; }
        sSegLo[k] = lo[k];
        sSegOff[k] = o;
        o += len[k];
      }
      if (o > kTile || bad || zs < 0 || zs + o > H.n) {  // inconsistent partition: skip the tile, report
        set_error(a.ctrl, BASS_ERR_ARG);
        for (int k = 0; k < 5; ++k) sSegOff[k] = 0;
        o = 0;
      }
      sSegOff[5] = o;
      sZstart = zs;
      // shared positions: segment k starts at its packed offset, or one
      // position later, so that its positions have the parity of its source
      // entries (both ends of a bulk copy of 8-byte data 16-byte aligned); at
      // most five gaps, inside kTilePad.  A plain tile has one segment from
      // an even entry (tile * kTile) and no gap.
      int gap = 0;
      for (int k = 0; k < 5; ++k) {
        const long long ln = sSegOff[k + 1] - sSegOff[k];
        if (tma && ln > 0 && ((sSegOff[k] + gap - sSegLo[k]) & 1)) ++gap;
        sGap[k] = gap;
        sSegPos[k] = (int)sSegOff[k] + gap;
      }
      if (tma) {
        // the bulk copies of every segment's 16-byte aligned body [f, l):
        // one arrival that expects all their bytes, then the copies
        unsigned bytes = 0;
        for (int k = 0; k < 5; ++k) {
          const long long l0 = sSegLo[k], ln = sSegOff[k + 1] - sSegOff[k];
          if (ln > 0) bytes += (unsigned)(((l0 + ln) & ~1LL) - ((l0 + 1) & ~1LL)) * (8u + kAmpBytes);
        }
        fence_proxy_async_smem();  // the previous tile's shared accesses (all threads: barrier above)
        mbar_arrive_expect(&sBar, bytes);
        for (int k = 0; k < 5; ++k) {
          const long long l0 = sSegLo[k], ln = sSegOff[k + 1] - sSegOff[k];
          if (ln <= 0) continue;
          const long long f = (l0 + 1) & ~1LL, l = (l0 + ln) & ~1LL;
          if (l <= f) continue;
          const int p = sSegPos[k] + (int)(f - l0);
          const unsigned nb = (unsigned)(l - f);
          bulk_load(sZ + p, H.keys + f, 8u * nb, &sBar);
          if (C64)
            bulk_load(reinterpret_cast<float2*>(sA) + p, reinterpret_cast<const float2*>(H.amps) + f, 8u * nb, &sBar);
          else
            bulk_load(sA + p, H.amps + f, 16u * nb, &sBar);
        }
      }
      if (a.prof) atomicAdd(reinterpret_cast<unsigned long long*>(&a.ctrl->prof_in[KIND * 5 + PASS]),
                            (unsigned long long)o);
    }
    __syncthreads();
    const int E = (int)sSegOff[5];

    // ---- load: bulk copies straight into shared memory ------------------------
    // (issued by thread 0 above); warp 0 fetches the at most two ragged
    // entries of each segment (an odd first entry, an even last one) with
    // plain loads, then every thread waits for the copies' bytes on sBar.  The
    // wait is bounded (the copies complete unless the byte count is wrong);
    // giving up records BASS_ERR_WAIT and ends the pass.
    if (tma) {
      if (tid < 10) {
        const int k = tid >> 1;
        const long long l0 = sSegLo[k], ln = sSegOff[k + 1] - sSegOff[k];
        if (ln > 0) {
          const long long f = (l0 + 1) & ~1LL, l = (l0 + ln) & ~1LL;
          const bool last = tid & 1;
          if (last ? l < l0 + ln : l0 < f) {
            const long long i = last ? l : l0;
            const int p = sSegPos[k] + (int)(i - l0);
            sZ[p] = H.keys[i];
            if (C64) reinterpret_cast<float2*>(sA)[p] = reinterpret_cast<const float2*>(H.amps)[i];
            else sA[p] = H.amps[i];
          }
        }
      }
      bool done = false;
      for (long long sp = 0; sp < kSpinLimit && !done; ++sp) done = mbar_try_wait(&sBar, phase);
      phase ^= 1u;
      if (__syncthreads_or(!done)) {
        if (tid == 0) set_error(a.ctrl, BASS_ERR_WAIT);
        break;
      }
    } else {
      // 8-byte aligned arrays: asynchronous per-entry copies (no gaps)
      const int o1 = (int)sSegOff[1], o2 = (int)sSegOff[2], o3 = (int)sSegOff[3], o4 = (int)sSegOff[4];
      const unsigned zb = (unsigned)__cvta_generic_to_shared(sZ);
      const unsigned ab = (unsigned)__cvta_generic_to_shared(sA);
      constexpr bool c64 = C64;
#pragma unroll
      for (int k = 0; k < kPerThread; ++k) {
        const int e = k * kThreads + tid;
        if (e < E) {
          const int sg = (e >= o1) + (e >= o2) + (e >= o3) + (e >= o4);
          const long long src = sSegLo[sg] + (e - sSegOff[sg]);
          asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(zb + 8u * e), "l"(H.keys + src) : "memory");
          if (c64)
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(ab + 8u * e),
                         "l"(reinterpret_cast<const float2*>(H.amps) + src)
                         : "memory");
          else
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(ab + 16u * e), "l"(H.amps + src)
                         : "memory");
        }
      }
      asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
      __syncthreads();
    }

    // ---- Z order: stable split by the target bit, merge, write back --------
    // The split rewrites the Z keys (zmove of the loaded keys) in place, bit-
    // clear run first, with their load positions in sIdx; the merge reads the
    // two runs and leaves the Z-ordered keys in sZ and, in sIdx, the load
    // position of each Z position (the amplitudes are not moved).
    if (KIND != K_IDENT) {
      const int lane = tid & 31, w = tid >> 5;
      const unsigned lt = (1u << lane) - 1;
      unsigned m0[kPerThread];
      uint64_t zk[kPerThread];
      int pe[kPerThread];  // shared position of load position e
      int c0 = 0;
      const int o1 = (int)sSegOff[1], o2 = (int)sSegOff[2], o3 = (int)sSegOff[3], o4 = (int)sSegOff[4];
#pragma unroll
      for (int k = 0; k < kPerThread; ++k) {
        const int e = w * 256 + k * 32 + lane;
        pe[k] = e + sGap[(e >= o1) + (e >= o2) + (e >= o3) + (e >= o4)];
        zk[k] = e < E ? zmove(sZ[pe[k]], t, gb) : ~0ULL;
        const bool is0 = e < E && !((zk[k] >> gb) & 1ULL);
        m0[k] = __ballot_sync(0xffffffffu, is0);
        c0 += __popc(m0[k]);
      }
      if (lane == 0) sWarp[w] = c0;
      __syncthreads();
      int wb0 = 0, n0 = 0;
#pragma unroll
      for (int i = 0; i < kThreads / 32; ++i) {
        const int v = sWarp[i];
        if (i < w) wb0 += v;
        n0 += v;
      }
      const int wstart = w * 256 < E ? w * 256 : E;
      int r0 = wb0, r1 = wstart - wb0;
#pragma unroll
      for (int k = 0; k < kPerThread; ++k) {
        const int e = w * 256 + k * 32 + lane;
        const unsigned ones = __ballot_sync(0xffffffffu, e < E) & ~m0[k];
        if (e < E) {
          const int dst = ((m0[k] >> lane) & 1u) ? r0 + __popc(m0[k] & lt) : n0 + r1 + __popc(ones & lt);
          sZ[dst] = zk[k];  // in place: every thread read its keys before the barrier above
          sIdx[dst] = (uint16_t)pe[k];
        }
        r0 += __popc(m0[k]);
        r1 += __popc(ones);
      }
      __syncthreads();
      const int n1 = E - n0;
      const uint64_t* K0 = sZ;
      const uint64_t* K1 = sZ + n0;
      const int d = base_e < E ? base_e : E;
      int lo = d - n1 > 0 ? d - n1 : 0, hi = d < n0 ? d : n0;
      while (lo < hi) {
        const int m = (lo + hi) >> 1;
        if (K0[m] < K1[d - 1 - m]) lo = m + 1;
        else hi = m;
      }
      int i = lo, j = d - lo;
      uint64_t rz[kPerThread];
      int rs[kPerThread];
      uint64_t z0 = (i < n0) ? K0[i] : ~0ULL;
      uint64_t z1 = (j < n1) ? K1[j] : ~0ULL;
#pragma unroll
      for (int k = 0; k < kPerThread; ++k) {
        const bool take0 = z0 < z1;
        rz[k] = take0 ? z0 : z1;
        rs[k] = take0 ? i : n0 + j;
        if (take0) {
          ++i;
          z0 = (i < n0) ? K0[i] : ~0ULL;
        } else {
          ++j;
          z1 = (j < n1) ? K1[j] : ~0ULL;
        }
      }
      uint16_t rp[kPerThread];
#pragma unroll
      for (int k = 0; k < kPerThread; ++k) rp[k] = (d + k < E) ? sIdx[rs[k]] : 0;
      // Each thread writes its kPerThread consecutive positions in a skewed
      // order, starting at element sk = (lane / 2) mod 8: the 16 lanes of a
      // half-warp then hit 16 different bank pairs with their 8-byte stores
      // (in plain order they hit two).  The registers are rotated by sk
      // first (a fixed network of selects, no dynamic register indexing).
      static_assert(kPerThread == 8, "skewed write-back of eight positions");
      const int sk = (lane >> 1) & 7;
#pragma unroll
      for (int b = 1; b < kPerThread; b <<= 1) {
        uint64_t tz[kPerThread];
        uint16_t tp[kPerThread];
#pragma unroll
        for (int k = 0; k < kPerThread; ++k) {
          tz[k] = (sk & b) ? rz[(k + b) & 7] : rz[k];
          tp[k] = (sk & b) ? rp[(k + b) & 7] : rp[k];
        }
#pragma unroll
        for (int k = 0; k < kPerThread; ++k) {
          rz[k] = tz[k];
          rp[k] = tp[k];
        }
      }
      __syncthreads();
#pragma unroll
      for (int k = 0; k < kPerThread; ++k) {
        const int pos = d + ((k + sk) & 7);   // rz[k] now holds position d + (k + sk) mod 8
        if (pos < E) {
          sZ[pos] = rz[k];
          sPerm[pos] = rp[k];  // the amplitudes stay where they were loaded (sIdx was read above)
        }
      }
      __syncthreads();
    }

    constexpr bool c64 = C64;
    const AmpView amp{sA, reinterpret_cast<const float2*>(sA), KIND == K_IDENT ? nullptr : sPerm, H.r0, H.r1,
                      scaled, c64};

    // ---- evaluate ------------------------------------------------------------
    // Round r gives position r * kThreads + tid to thread tid, so neighbouring
    // threads handle neighbouring groups and write neighbouring outputs.
    if (PASS == P_RDM && KIND == K_GATE2) {
      // 4x4 moments of the pair (q1 at bit 1, q2 at bit 0 after the first
      // pass): per group of up to four entries a_i (i = (b_q1 << 1) | b_q2),
      // set 0: |a_0|^2 .. |a_3|^2; set 1: Re/Im a_0 conj(a_1), a_0 conj(a_2);
      // set 2: a_0 conj(a_3), a_1 conj(a_2); set 3: a_1 conj(a_3), a_2 conj(a_3)
      // (bass_simulator.py:200-231, rho[p][q] += a_p conj(a_q)).
      i128 v[4] = {0, 0, 0, 0};
      double dh[4] = {0.0, 0.0, 0.0, 0.0}, dl[4] = {0.0, 0.0, 0.0, 0.0};
      for (int p = tid; p < E; p += kThreads) {
        const uint64_t gid = sZ[p] >> 2;
        if (p > 0 && (sZ[p - 1] >> 2) == gid) continue;
        const double2 zero = make_double2(0.0, 0.0);
        double2 g0 = zero, g1 = zero, g2 = zero, g3 = zero;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          if (p + r < E) {
            const uint64_t zr = sZ[p + r];
            if ((zr >> 2) == gid) {
              const double2 v2 = amp(p + r);
              const unsigned i = (unsigned)(zr & 3);
              if (i == 0) g0 = v2;
              else if (i == 1) g1 = v2;
              else if (i == 2) g2 = v2;
              else g3 = v2;
            }
          }
        }
        double m[4];
        if (set == 0) {
          m[0] = prob(g0); m[1] = prob(g1); m[2] = prob(g2); m[3] = prob(g3);
        } else {
          // the set's two pairs (i, j), i < j: a_i conj(a_j)
          const double2 ai = set == 3 ? g1 : g0, aj = set == 1 ? g1 : g3;
          const double2 bi = set == 1 ? g0 : set == 2 ? g1 : g2, bj = set == 3 ? g3 : g2;
          const double2 c0 = cmul(ai, make_double2(aj.x, -aj.y));
          const double2 c1 = cmul(bi, make_double2(bj.x, -bj.y));
          m[0] = c0.x; m[1] = c0.y; m[2] = c1.x; m[3] = c1.y;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) fx_acc96(m[k], dh[k], dl[k], v[k]);
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) v[k] += fx_join96s(dh[k], dl[k]);
      block_sum_i128<4>(v, sRed);
      if (tid == 0) {
        Partial* pt = a.ws.partials + (long long)set * a.ws.max_tiles + tile;
        pt->s[0] = v[0]; pt->s[1] = v[1]; pt->s[2] = v[2]; pt->s[3] = v[3];
      }
    } else if (PASS == P_RDM) {
      // at most kPerThread positions per thread, so at most eight terms per
      // split accumulator (fx_acc96) before they are joined
      i128 v[4] = {0, 0, 0, 0};
      double dh[4] = {0.0, 0.0, 0.0, 0.0}, dl[4] = {0.0, 0.0, 0.0, 0.0};
      for (int p = tid; p < E; p += kThreads) {
        const uint64_t z = sZ[p];
        const uint64_t gid = z >> 1;
        if (p > 0 && (sZ[p - 1] >> 1) == gid) continue;
        const double2 x0 = amp(p);
        if ((z & 1ULL) == 0) {
          fx_acc96(prob(x0), dh[0], dl[0], v[0]);
          if (p + 1 < E && (sZ[p + 1] >> 1) == gid) {
            const double2 x1 = amp(p + 1);
            fx_acc96(prob(x1), dh[1], dl[1], v[1]);
            const double2 c = cmul(x0, make_double2(x1.x, -x1.y));
            fx_acc96(c.x, dh[2], dl[2], v[2]);
            fx_acc96(c.y, dh[3], dl[3], v[3]);
          }
        } else {
          fx_acc96(prob(x0), dh[1], dl[1], v[1]);
        }
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) v[k] += fx_join96s(dh[k], dl[k]);
      block_sum_i128<4>(v, sRed);
      if (tid == 0) {
        Partial* pt = a.ws.partials + (long long)set * a.ws.max_tiles + tile;
        pt->s[0] = v[0]; pt->s[1] = v[1]; pt->s[2] = v[2]; pt->s[3] = v[3];
      }
    } else if (PASS == P_WRITE) {
      // write_mode 2: one child per entry (a 2-qubit gate's first pass),
      //   base = the tile's Z start; 0: the drop rule decides (diagonal
      //   1-qubit gate compaction), base by decoupled look-back.  Gates,
      //   rotations and truncations write through k_compact instead.
      constexpr int MC = KindTraits<KIND>::kMaxChildren;
      uint64_t kb;
      double2 ca[MC];

      const int wmode = a.write_mode;
      // (a) kept-children mask per position
      for (int p = tid; p < E; p += kThreads) {
        unsigned mk = 0;
        if (wmode == 2) {
          mk = 1u;
        } else {
          const unsigned cm = group_children_t<KIND>(c64, p, E, sZ, amp, gb, a.G, a.drop_zero, &kb, ca);
          if ((cm & 1u) && keep_child((uint64_t)__double_as_longlong(prob(ca[0])), kb, S, H.qat_out)) mk = 1u;
        }
        sMask[p] = (uint8_t)mk;
        sOff[p] = (uint16_t)__popc(mk);
      }
      __syncthreads();
      // (b) counts -> exclusive offsets in place (position order)
      int run = 0;
#pragma unroll
      for (int k = 0; k < kPerThread; ++k)
        if (base_e + k < E) run += sOff[base_e + k];
      int tile_total;
      int ex = block_excl_scan(run, sWarp, &tile_total);
#pragma unroll
      for (int k = 0; k < kPerThread; ++k) {
        const int p = base_e + k;
        if (p < E) {
          const int c = sOff[p];
          sOff[p] = (uint16_t)ex;
          ex += c;
        }
      }
      // (c) the tile's base in the output
      if (wmode == 0) {
        if (tid < 32) {
          const long long b = lookback_warp(a.ws.status, tile, tile_total, a.ctrl);
          if (tid == 0) sBase = b;
        }
      } else if (tid == 0) {
        sBase = sZstart;
      }
      __syncthreads();
      if (tid == 0) {
        const long long b = sBase;
        if (tile == ntiles - 1) a.ws.sel->n_written = b + tile_total;
        if (b + tile_total > a.out->cap) set_error(a.ctrl, BASS_ERR_CAPACITY);
        if (a.prof) atomicAdd(reinterpret_cast<unsigned long long*>(&a.ctrl->prof_out[KIND * 5 + PASS]),
                              (unsigned long long)tile_total);
      }
      // (d) write the kept children
      if (sBase + tile_total <= a.out->cap) {
        uint64_t* ok = a.out->keys;
        double* oa = a.out->amps;
        for (int p = tid; p < E; p += kThreads) {
          const unsigned mk = sMask[p];
          if (!mk) continue;
          long long o = sBase + sOff[p];
          group_children_t<KIND>(c64, p, E, sZ, amp, gb, a.G, a.drop_zero, &kb, ca);
#pragma unroll
          for (int c = 0; c < MC; ++c) {
            if ((mk >> c) & 1u) {
              ok[o] = kb | (uint64_t)c;
              amp_put(oa, o, ca[c], c64);
              ++o;
            }
          }
        }
      }
    } else if (PASS == P_HIST) {
      // every child is staged at its slot index: |a|^2 bits in the slot
      // array, key and amplitude in the staging arrays (the write step
      // compacts the survivors from there)
      uint64_t kb;
      double2 ca[NS];
      unsigned long long* slots = reinterpret_cast<unsigned long long*>(a.ws.tmp_keys) + NS * sZstart;
      uint64_t* skeys = a.ws.stage_keys + sZstart;  // one base key per Z position (staged_key)
      double2* samps = a.ws.tmp_amps + NS * sZstart;
      float2* sampf = reinterpret_cast<float2*>(a.ws.tmp_amps) + NS * sZstart;
      for (int p = tid; p < E; p += kThreads) {
        const unsigned cm = group_children_t<KIND>(c64, p, E, sZ, amp, gb, a.G, a.drop_zero, &kb, ca);
        unsigned long long sb[NS];
#pragma unroll
        for (int c = 0; c < NS; ++c) {
          if ((cm >> c) & 1u) {
            sb[c] = (unsigned long long)__double_as_longlong(prob(ca[c]));
            ++cnt;
          } else {
            sb[c] = ~0ULL;
          }
        }
        if (cm) {  // every slot of the group is written (a missing child's slot holds ~0 bits)
          skeys[p] = kb;
          if (NS == 1) {
            if (c64) sampf[p] = d2f(ca[0]);
            else samps[p] = ca[0];
          } else {
            if (c64) {
#pragma unroll
              for (int c = 0; c < NS; c += 2) {
                const float2 f0 = d2f(ca[c]), f1 = d2f(ca[c + 1]);
                *reinterpret_cast<float4*>(sampf + (long long)NS * p + c) = make_float4(f0.x, f0.y, f1.x, f1.y);
              }
            } else {
#pragma unroll
              for (int c = 0; c < NS; ++c) samps[(long long)NS * p + c] = ca[c];
            }
          }
        }
        if (NS == 1) {
          slots[p] = sb[0];
        } else {
#pragma unroll
          for (int c = 0; c < NS; c += 2)
            *reinterpret_cast<ulonglong2*>(slots + (long long)NS * p + c) = make_ulonglong2(sb[c], sb[c + 1]);
        }
      }
    }
    __syncthreads();
  }

  pdl_trigger();
  // ---- write pass: the last CTA to finish writes the output descriptor ------
  if (PASS == P_WRITE && a.fin) write_done(a, KIND, g);

  // ---- flush: the CTA's child count ----------------------------------------
  if (PASS == P_HIST) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, off);
    if ((tid & 31) == 0) reinterpret_cast<long long*>(sRed)[tid >> 5] = cnt;
    __syncthreads();
    if (tid == 0) {
      long long c = 0;
      for (int w = 0; w < kThreads / 32; ++w) c += reinterpret_cast<long long*>(sRed)[w];
      a.ws.partials[g.bid].c[0] = c;
    }
  }
}

// The tile pass of one op on a state of complex64 (C64) or complex128 amplitudes.
template <int KIND, int PASS, bool C64>
__global__ void __launch_bounds__(kThreads, 4) k_tile(const __grid_constant__ OpArgs a) {
  pdl_wait();
  tile_body<KIND, PASS, C64>(a, whole_grid());
}

// ---------------------------------------------------------------------------
// selection: one launch per op, every block resident (grid barriers)
// ---------------------------------------------------------------------------
// After the evaluation pass has written every child's |a|^2 bit pattern to the
// slot array (NS words per Z position, ~0 where a group has fewer children),
// k_select_coop finds the top-k threshold and prepares the write pass:
//   1. the child count (from the evaluation pass's per-CTA partials) decides
//      whether the op truncates;
//   2. radix select on the bit patterns: a 13-bit histogram of bits 50-62,
//      then of bits 37-49 inside the boundary bin; every block reads the
//      histograms and finds the boundary bins itself, so each level costs
//      one grid barrier;
//   3. per tile, the number of survivors (into ws.status) and per CTA the
//      exact kept mass, total mass and, for a rotation step, sum of |a|^4.
//      When the threshold lies inside the level-2 bin, this pass keeps what
//      lies above the bin and collects the bin's children (slot, true key);
//      after a barrier every block settles them (the k-th best by bits, then
//      smallest true key: settle_small, or settle_radix in block 0 for more
//      than kCandSmem) and adds the kept ones to the tile counts and sums;
//   4. the last block to finish step 3: the exact sums, the rotation
//      decision, and an exclusive scan of the tile counts (each tile of the
//      write step then knows its base).
// Children tied at the threshold pattern t_bits are kept up to the largest
// kept true key t_key; the write step applies the same rule.  The grid
// barrier is a counter and a generation word in the
// workspace with a bounded spin (BASS_ERR_WAIT, then every block returns).
constexpr int kSelThreads = 1024;
// dynamic shared memory of the selection: the histograms (kHistBins words),
// later the boundary candidates (bits, true key, slot index)
constexpr size_t kSelSmem = (size_t)kCandSmem * 24;

// Grid-wide barrier of the selection's grid (every block resident, see
// launch_select_t).  An arrival counter that only grows within the kernel
// (the op's workspace clear zeroes it): the b-th barrier of a block adds one
// (release) and waits until the counter reaches b x blocks (acquire), so no
// arrival waits for an atomic's result and no last block has to publish a
// release.  Every block passes the same barriers in the same order; gen is
// the block's count of barriers passed (shared memory, zero at the start of
// the kernel).  Returns false (error recorded) if the wait gave up.
__device__ bool grid_sync(const OpArgs& a, Grp gr, unsigned long long& gen) {
  __shared__ int sOk;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long* cnt = reinterpret_cast<unsigned long long*>(a.ws.counters) + 60;
    const unsigned long long target = (gen + 1) * (unsigned long long)gr.nblk;
    __threadfence();
    red_release_add(cnt, 1ULL);
    int ok = 1;
    long long spins = 0;
    const long long lim = wait_limit(a.ctrl);
    while (ld_acquire(cnt) < target) {
      if (++spins > lim) {
        set_error(a.ctrl, BASS_ERR_WAIT);
        ok = 0;
        break;
      }
      __nanosleep(32);
    }
    __threadfence();
    gen += 1;
    sOk = ok;
  }
  __syncthreads();
  return sOk != 0;
}

// Block-wide (warp 0 works): the bin b of an 8192-bin histogram in global
// memory (written by other blocks, with coarse counts of its 64 groups of 128
// bins after the bins) with count(bins > b) < k <= count(bins >= b);
// *c_gt = count(bins > b), *c_b = count(b).  Needs 1 <= k <= total.  Reads the
// 64 coarse counts and the 128 bins of one group.
__device__ int find_bin(const unsigned int* hist, long long k, long long* c_gt, long long* c_b) {
  __shared__ int sRes;
  __shared__ long long sAbove, sCnt;
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    // coarse: lane holds groups 2 lane and 2 lane + 1
    const long long g0 = __ldcg(hist + kHistBins + 2 * lane);
    const long long g1 = __ldcg(hist + kHistBins + 2 * lane + 1);
    const long long v = g0 + g1;
    long long suf = v;  // groups >= 2 lane
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const long long y = __shfl_down_sync(0xffffffffu, suf, off);
      if (lane + off < 32) suf += y;
    }
    const unsigned m = __ballot_sync(0xffffffffu, suf >= k);
    const int L = m ? 31 - __clz(m) : 0;
    long long above = __shfl_sync(0xffffffffu, suf - v, L);  // groups > 2 L + 1
    const long long c1 = __shfl_sync(0xffffffffu, g1, L);
    int G = 2 * L + 1;
    if (above + c1 < k) {
      above += c1;
      G = 2 * L;
    }
    // fine: lane holds bins 128 G + 4 lane .. + 3
    const unsigned* hb = hist + G * kGroupBins + 4 * lane;
    long long f[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) f[q] = __ldcg(hb + q);
    const long long w = f[0] + f[1] + f[2] + f[3];
    long long suf2 = w;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const long long y = __shfl_down_sync(0xffffffffu, suf2, off);
      if (lane + off < 32) suf2 += y;
    }
    const unsigned m2 = __ballot_sync(0xffffffffu, above + suf2 >= k);
    const int L2 = m2 ? 31 - __clz(m2) : 0;
    if (lane == L2) {
      long long ab = above + suf2 - w;  // bins above this lane's four
      int q = 3;
      for (; q > 0; --q) {
        if (ab + f[q] >= k) break;
        ab += f[q];
      }
      sRes = G * kGroupBins + 4 * lane + q;
      sAbove = ab;
      sCnt = f[q];
    }
  }
  __syncthreads();
  *c_gt = sAbove;
  *c_b = sCnt;
  return sRes;
}

// Adds the block's shared histogram h into the global histogram gh and its
// coarse counts of 64 groups of 128 bins (gh[kHistBins + g]), for find_bin.
__device__ void flush_hist(const unsigned int* h, unsigned int* gh) {
  for (int i = threadIdx.x; i < kHistBins; i += blockDim.x)
    if (h[i]) atomicAdd(&gh[i], h[i]);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int g = w; g < kHistGroups; g += nw) {
    const unsigned* hg = h + g * kGroupBins;
    unsigned c = 0;
#pragma unroll
    for (int q = 0; q < kGroupBins / 32; ++q) c += hg[32 * q + lane];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) c += __shfl_down_sync(0xffffffffu, c, off);
    if (lane == 0 && c) atomicAdd(&gh[kHistBins + g], c);
  }
}

// Block-wide histogram of the slots (LEVEL 1: bits >> 50; LEVEL 2: bits
// 37-49 of the slots whose bits >> 50 equal pre), added into gh.
template <int LEVEL>
__device__ void slot_hist_phase(const unsigned long long* slots, long long nslots, unsigned long long pre,
                                unsigned int* h, unsigned int* gh, Grp g) {
  for (int i = threadIdx.x; i < kHistBins; i += blockDim.x) h[i] = 0;
  __syncthreads();
  // eight slots per thread and round, plain shared atomics (measured faster
  // here than warp aggregation with __match_any_sync)
  const ulonglong2* v = reinterpret_cast<const ulonglong2*>(slots);
  const long long n2 = nslots >> 1;
  const long long stride = (long long)g.nblk * blockDim.x;
  for (long long b = (long long)g.bid * blockDim.x; b < n2; b += 4 * stride) {
    unsigned key[8];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const long long i = b + u * stride + threadIdx.x;
      const ulonglong2 x = (i < n2) ? v[i] : make_ulonglong2(~0ULL, ~0ULL);
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const unsigned long long bits = c ? x.y : x.x;
        const bool valid = bits != ~0ULL && (LEVEL == 1 || (bits >> 50) == pre);
        const unsigned bin =
            LEVEL == 1 ? (unsigned)(bits >> 50) : (unsigned)((bits >> 37) & (kHistBins - 1));
        key[2 * u + c] = valid ? bin : 0xFFFFFFFFu;
      }
    }
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (key[u] != 0xFFFFFFFFu) atomicAdd(&h[key[u]], 1u);
  }
  if ((nslots & 1) && g.bid == 0 && threadIdx.x == 0) {
    const unsigned long long bits = slots[nslots - 1];
    const bool valid = bits != ~0ULL && (LEVEL == 1 || (bits >> 50) == pre);
    const unsigned bin = LEVEL == 1 ? (unsigned)(bits >> 50) : (unsigned)((bits >> 37) & (kHistBins - 1));
    if (valid) atomicAdd(&h[bin], 1u);
  }
  __syncthreads();
  flush_hist(h, gh);
}

// better(a, b): a ranks strictly above b
__device__ __forceinline__ bool better(unsigned long long ab, unsigned long long ak,
                                       unsigned long long bb, unsigned long long bk) {
  return ab > bb || (ab == bb && ak < bk);
}

// Sorts sb / sk [0, m) (m <= kCandSmem) by (bits desc, key asc), moving si
// along: bitonic, padded to a power of two with pairs that rank below every
// candidate.
__device__ void sort_pairs(unsigned long long* sb, unsigned long long* sk, unsigned long long* si, long long m) {
  const int tid = threadIdx.x;
  int P = 1;
  while (P < m) P <<= 1;
  for (int i = tid + (int)m; i < P; i += blockDim.x) {
    sb[i] = 0;
    sk[i] = ~0ULL;
    si[i] = 0;
  }
  __syncthreads();
  for (int size = 2; size <= P; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = tid; i < P; i += blockDim.x) {
        const int jx = i ^ stride;
        if (jx > i) {
          const bool up = (i & size) == 0;
          const bool sw = up ? better(sb[jx], sk[jx], sb[i], sk[i]) : better(sb[i], sk[i], sb[jx], sk[jx]);
          if (sw) {
            unsigned long long tb = sb[i], tk = sk[i], ti = si[i];
            sb[i] = sb[jx]; sk[i] = sk[jx]; si[i] = si[jx]; sb[jx] = tb; sk[jx] = tk; si[jx] = ti;
          }
        }
      }
      __syncthreads();
    }
  }
}

// The physical key of the child staged at slot i: the evaluation pass stages
// one key per Z position, its group's base key (low lns bits clear), and
// child c of the group sits at slot (position << lns) | c.
__device__ __forceinline__ uint64_t staged_key(const uint64_t* sk, unsigned long long i, int lns, bool streaming) {
  const unsigned long long p = i >> lns;
  const uint64_t base = streaming ? __ldcs(sk + p) : __ldcg(sk + p);
  return base | (uint64_t)(i & ((1ULL << lns) - 1));
}

// The true key of the child staged at slot i (qat: the op's output order,
// lns: log2 of the slots per entry).
__device__ __forceinline__ unsigned long long cand_true_key(const OpArgs& a, unsigned long long i, int lns,
                                                            const int8_t* qat) {
  return true_key(staged_key(a.ws.stage_keys, i, lns, false), qat, 64);
}

// The threshold of the level-2 boundary bin's m candidates (slot indices in
// ws.cand_bits; m <= kCandSmem), one block: the need-th best child by (bits
// desc, true key asc) gives (t_bits, t_key); t_key is ~0 when every candidate
// at t_bits is kept.  The candidates stay in shared memory (bits, true key,
// slot index: three arrays of kCandSmem words, in some order) for the caller.
__device__ void settle_small(const OpArgs& a, unsigned char* smem, long long m, long long need, int lns,
                             const int8_t* qat, unsigned long long* tb_out, unsigned long long* tk_out) {
  unsigned long long* sb = reinterpret_cast<unsigned long long*>(smem);
  unsigned long long* sk = sb + kCandSmem;
  unsigned long long* ssi = sk + kCandSmem;
  const unsigned long long* slots = reinterpret_cast<const unsigned long long*>(a.ws.tmp_keys);
  const int tid = threadIdx.x;
  for (long long i = tid; i < m; i += blockDim.x) {
    const unsigned long long si = __ldcg(a.ws.cand_bits + i);
    ssi[i] = si;
    sb[i] = __ldcg(slots + si);
    sk[i] = cand_true_key(a, si, lns, qat);
  }
  __syncthreads();
  const long long r = need < 1 ? 0 : (need > m ? m - 1 : need - 1);
  __shared__ int sSel, sCut;
  if (tid == 0) { sSel = 0; sCut = 0; }
  __syncthreads();
  if (m <= kRankMax) {
    // few: the rank of each candidate is the number that rank above it
    for (long long i = tid; i < m; i += blockDim.x) {
      long long rank = 0;
      for (long long jx = 0; jx < m; ++jx) rank += better(sb[jx], sk[jx], sb[i], sk[i]);
      if (rank == r) sSel = (int)i;
    }
  } else {
    sort_pairs(sb, sk, ssi, m);
    if (tid == 0) sSel = (int)r;
  }
  __syncthreads();
  const unsigned long long tb = sb[sSel], tk = sk[sSel];
  for (long long i = tid; i < m; i += blockDim.x)
    if (sb[i] == tb && sk[i] > tk) sCut = 1;
  __syncthreads();
  *tb_out = tb;
  *tk_out = sCut ? tk : ~0ULL;
  __syncthreads();
}

// The same threshold for m > kCandSmem (one block): radix select on the
// low 37 bits of the bit pattern (the 26-bit prefix pre is shared), then, if
// the cut falls inside a run of equal patterns, on the true keys of that run.
__device__ void settle_radix(const OpArgs& a, unsigned char* smem, long long m, long long need,
                             unsigned long long pre, int lns, const int8_t* qat, unsigned long long* tb_out,
                             unsigned long long* tk_out) {
  unsigned int* h = reinterpret_cast<unsigned int*>(smem);
  const unsigned long long* slots = reinterpret_cast<const unsigned long long*>(a.ws.tmp_keys);
  const int tid = threadIdx.x;
  __shared__ unsigned long long sLow, sKeyPre;
  __shared__ long long sNeed;
  __shared__ unsigned int sLastCount;
  if (tid == 0) { sLow = 0; sNeed = need; sKeyPre = 0; }
  __syncthreads();
  const unsigned long long m37 = (1ULL << 37) - 1;
  for (int shift = 32; shift >= 0; shift -= 8) {
    for (int i = tid; i < 256; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const unsigned long long p = sLow;
    for (long long i = tid; i < m; i += blockDim.x) {
      const unsigned long long lb = __ldcg(slots + __ldcg(a.ws.cand_bits + i)) & m37;
      if (shift == 32 || (lb >> (shift + 8)) == p) atomicAdd(&h[(unsigned)(lb >> shift) & 255u], 1u);
    }
    __syncthreads();
    if (tid == 0) {
      long long above = 0;
      int b = 255;
      for (; b > 0; --b) {
        if (above + h[b] >= sNeed) break;
        above += h[b];
      }
      sNeed -= above;
      sLow = (p << 8) | (unsigned long long)b;
      sLastCount = h[b];
    }
    __syncthreads();
  }
  const unsigned long long tb = (pre << 37) | sLow;
  const long long take = sNeed;  // children at tb that are kept
  if (take >= (long long)sLastCount) {
    *tb_out = tb;
    *tk_out = ~0ULL;
    __syncthreads();
    return;
  }
  // the take smallest true keys among the children at tb
  for (int shift = 56; shift >= 0; shift -= 8) {
    for (int i = tid; i < 256; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const unsigned long long p = sKeyPre;
    for (long long i = tid; i < m; i += blockDim.x) {
      const unsigned long long si = __ldcg(a.ws.cand_bits + i);
      if (__ldcg(slots + si) != tb) continue;
      const unsigned long long k = cand_true_key(a, si, lns, qat);
      if (shift == 56 || (k >> (shift + 8)) == p) atomicAdd(&h[(unsigned)(k >> shift) & 255u], 1u);
    }
    __syncthreads();
    if (tid == 0) {
      long long below = 0;
      int b = 0;
      for (; b < 255; ++b) {
        if (below + h[b] >= sNeed) break;
        below += h[b];
      }
      sNeed -= below;
      sKeyPre = (p << 8) | (unsigned long long)b;
    }
    __syncthreads();
  }
  *tb_out = tb;
  *tk_out = sKeyPre;
  __syncthreads();
}

// The tile holding Z position z (tiles start at the partition's adjusted
// positions P'_b <= b * kStep; plain tiles every kTile positions).
// positions fit 32 bits (every op's count is below 2^31), so the divisions
// are 32-bit divisions by constants
__device__ __forceinline__ long long tile_of(long long z, int kind, const long long* part) {
  const unsigned zu = (unsigned)z;
  if (kind == K_IDENT) return (long long)(zu / (unsigned)kTile);
  const long long b0 = (long long)(zu / (unsigned)kStep);
  return (z >= part[(b0 + 1) * 6]) ? b0 + 1 : b0;
}

// A grid-stride stream over the slot array, eight consecutive slots per
// thread: the survivors per tile (atomically added into ws.status[tile],
// which the op cleared; one atomic per warp when its 256 slots lie in one
// tile), the kept mask (the thread's eight kept bits as one byte of
// ws.kmask), and, per CTA in partials s[0..2], the exact mass of the survivors,
// their sum of |a|^4 (P2) and the exact mass of all children (when
// truncating).  cand: the children of the level-2 boundary bin (bits >> 37 ==
// cpre, all below T) are listed as well (slot indices in ws.cand_bits,
// counted in sel->n_cand), for settle_boundary.
template <bool P2>
__device__ void count_phase(const OpArgs& a, int ns, int kind, unsigned long long T, bool incl, bool trunc,
                            i128* sRed, bool cand, unsigned long long cpre, Grp g) {
  const long long n = a.in->nnz;
  const long long nslots = (long long)ns * n;
  const bool sums = P2 || trunc;
  const bool want_total = trunc && !P2;  // gamma bookkeeping of plain truncations only
  const int lns = ns == 4 ? 2 : ns == 2 ? 1 : 0;  // slots per entry: 1, 2 or 4
  const int lane = threadIdx.x & 31;
  const unsigned long long* slots = reinterpret_cast<const unsigned long long*>(a.ws.tmp_keys);
  const long long* part = a.ws.part;
  i128 v[3] = {0, 0, 0};
  const long long nchunk = (nslots + 7) >> 3;
  const long long stride = (long long)g.nblk * blockDim.x;
  // the thread's chunk of slots [8c, 8c + 8)
  auto load_chunk = [&](long long c, unsigned long long* x) {
    const long long s0 = c << 3;
    if (s0 + 8 <= nslots) {
      const ulonglong2* q = reinterpret_cast<const ulonglong2*>(slots + s0);
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const ulonglong2 y = q[u];
        x[2 * u] = y.x;
        x[2 * u + 1] = y.y;
      }
    } else {
#pragma unroll
      for (int u = 0; u < 8; ++u) x[u] = (s0 + u < nslots) ? slots[s0 + u] : ~0ULL;
    }
  };
  for (long long cb = (long long)g.bid * blockDim.x + (threadIdx.x & ~31); cb < nchunk; cb += stride) {
    const long long c = cb + lane;  // this thread's chunk: slots [8c, 8c + 8)
    const long long s0 = c << 3;
    unsigned long long x[8];
    load_chunk(c, x);
    if (cand) {
      // the boundary bin's children: slot indices appended to the list, one
      // atomic per warp
      unsigned cm = 0;
#pragma unroll
      for (int u = 0; u < 8; ++u) cm |= (unsigned)(x[u] != ~0ULL && (x[u] >> 37) == cpre) << u;
      if (__any_sync(0xffffffffu, cm != 0)) {
        const int cc = __popc(cm);
        int inc = cc;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, inc, off);
          if (lane >= off) inc += y;
        }
        unsigned long long base = 0;
        if (lane == 31)
          base = atomicAdd(reinterpret_cast<unsigned long long*>(&a.ws.sel->n_cand), (unsigned long long)inc);
        base = __shfl_sync(0xffffffffu, base, 31);
        long long k = (long long)base + inc - cc;
        for (int u = 0; u < 8; ++u) {
          if (!((cm >> u) & 1u)) continue;
          if (k < a.ws.max_n) a.ws.cand_bits[k] = (unsigned long long)(s0 + u);
          ++k;
        }
      }
    }
    unsigned km = 0;
    // the chunk's sums as exact integer-valued doubles (fx_split96), folded
    // into v after the chunk; values of 2 and above take the integer path
    double dh[3] = {0.0, 0.0, 0.0}, dl[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const bool kept = slot_kept(x[u], T, incl);
      km |= (unsigned)kept << u;
      if (sums) {
        if (x[u] < 0x4000000000000000ULL) {  // 0 <= p < 2
          const double p = __longlong_as_double((long long)x[u]);
          double h, l;
          fx_split96(p, &h, &l);
          if (want_total) {
            dh[2] = __dadd_rn(dh[2], h);
            dl[2] = __dadd_rn(dl[2], l);
          }
          dh[0] = __dadd_rn(dh[0], kept ? h : 0.0);
          dl[0] = __dadd_rn(dl[0], kept ? l : 0.0);
          if (P2) {
            fx_split96(kept ? __dmul_rn(p, p) : 0.0, &h, &l);
            dh[1] = __dadd_rn(dh[1], h);
            dl[1] = __dadd_rn(dl[1], l);
          }
        } else if (x[u] != ~0ULL) {
          const i128 f = fx_from_pbits(x[u]);
          if (want_total) v[2] += f;
          if (kept) {
            v[0] += f;
            if (P2) {
              const double p = __longlong_as_double((long long)x[u]);
              v[1] += fx_from_pbits((unsigned long long)__double_as_longlong(__dmul_rn(p, p)));
            }
          }
        }
      }
    }
    if (sums) {
#pragma unroll
      for (int k = 0; k < 3; ++k) v[k] += fx_join96(dh[k], dl[k]);
    }
    // the kept bits of the chunk for the write step (a warp stores 32
    // consecutive bytes)
    const bool live = c < nchunk;
    if (live) a.ws.kmask[c] = (uint8_t)km;
    // survivors per tile
    const long long last = (s0 + 7 < nslots ? s0 + 7 : nslots - 1);
    const long long t0 = live ? tile_of(s0 >> lns, kind, part) : -1;
    const long long t1 = live ? tile_of(last >> lns, kind, part) : -1;
    const long long w0 = __shfl_sync(0xffffffffu, t0, 0);
    const bool uniform = __all_sync(0xffffffffu, !live || (t0 == w0 && t1 == w0));
    if (uniform) {
      int cnt = __popc(km);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, off);
      if (lane == 0 && cnt) atomicAdd(reinterpret_cast<unsigned long long*>(a.ws.status + w0), (unsigned long long)cnt);
    } else if (live) {
      for (int u = 0; u < 8; ++u) {
        if (!((km >> u) & 1u)) continue;
        const long long tb = (u == 0) ? t0 : tile_of((s0 + u) >> lns, kind, part);
        atomicAdd(reinterpret_cast<unsigned long long*>(a.ws.status + tb), 1ULL);
      }
    }
  }
  block_sum_i128<3>(v, sRed);
  if (threadIdx.x == 0) {
    Partial* pt = a.ws.partials + g.bid;
    pt->s[0] = v[0];
    pt->s[1] = v[1];
    pt->s[2] = v[2];
  }
}

// The boundary bin of a selection whose threshold lies inside its level-2
// bin (late): its m children (slot indices in ws.cand_bits, collected by
// the count pass) are below every kept child of the other bins.  Run by one
// block (the last to finish): the need-th best of them by (bits desc, true
// key asc) gives (t_bits, t_key); the kept ones are added to their tiles'
// counts, to the kept mask and to this thread's share of the kept mass
// (vk[0]) and sum of |a|^4 (vk[1]).  qat: the op's output order (for the
// true keys).
template <bool P2>
__device__ void settle_boundary(const OpArgs& a, int ns, int kind, unsigned long long lpre, long long lneed,
                                const int8_t* qat, i128* vk) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ long long sM;
  SelState* sel = a.ws.sel;
  const int tid = threadIdx.x;
  if (tid == 0) sM = *(volatile long long*)&sel->n_cand;
  __syncthreads();
  long long m = sM;
  if (m > a.ws.max_n) {
    if (tid == 0) set_error(a.ctrl, BASS_ERR_WORKSPACE);
    m = a.ws.max_n;
  }
  const int lns = ns == 4 ? 2 : ns == 2 ? 1 : 0;
  unsigned long long tb, tk;
  if (m <= kCandSmem) settle_small(a, smem, m, lneed, lns, qat, &tb, &tk);
  else settle_radix(a, smem, m, lneed, lpre, lns, qat, &tb, &tk);
  if (tid == 0) {
    sel->t_bits = tb;
    sel->t_key = tk;
  }
  const unsigned long long* slots = reinterpret_cast<const unsigned long long*>(a.ws.tmp_keys);
  const bool in_smem = m <= kCandSmem;  // settle_small left (bits, key, slot) there
  const unsigned long long* sb = reinterpret_cast<const unsigned long long*>(smem);
  for (long long k = tid; k < m; k += blockDim.x) {
    const unsigned long long i = in_smem ? sb[2 * kCandSmem + k] : __ldcg(a.ws.cand_bits + k);
    const unsigned long long bits = in_smem ? sb[k] : __ldcg(slots + i);
    if (bits > tb || (bits == tb && (in_smem ? sb[kCandSmem + k] : cand_true_key(a, i, lns, qat)) <= tk)) {
      atomicAdd(reinterpret_cast<unsigned long long*>(a.ws.status + tile_of((long long)(i >> lns), kind, a.ws.part)),
                1ULL);
      atomicOr(reinterpret_cast<unsigned int*>(a.ws.kmask) + (i >> 5), 1u << (i & 31));
      vk[0] += fx_from_pbits(bits);
      if (P2) {
        const double p = __longlong_as_double((long long)bits);
        vk[1] += fx_from_pbits((unsigned long long)__double_as_longlong(__dmul_rn(p, p)));
      }
    }
  }
  __threadfence();
  __syncthreads();
}

// The last block after the counts: exact kept / total mass (tied children added
// back: vk, this thread's share of the settled boundary bin), the rotation
// decision (mode 1, the rule of bass_simulator.py:795-814: the candidate's PR
// = kept^2 / sum |a|^4 against ctrl->pr_cur; a rejected candidate is not
// written unless a trace is kept), and the exclusive scan of the tile counts
// in ws.status.
__device__ void final_phase(const OpArgs& a, int nblk, int kind, int mode, int j, int trace, i128* sRed,
                            const i128* vk) {
  volatile SelState* sel = a.ws.sel;  // written by other blocks of this kernel
  i128 v[3] = {vk[0], vk[1], 0};
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
    const Partial* p = a.ws.partials + b;
    v[0] += (i128)(((u128)__ldcg((const unsigned long long*)&p->s[0] + 1) << 64) |
                   __ldcg((const unsigned long long*)&p->s[0]));
    v[1] += (i128)(((u128)__ldcg((const unsigned long long*)&p->s[1] + 1) << 64) |
                   __ldcg((const unsigned long long*)&p->s[1]));
    v[2] += (i128)(((u128)__ldcg((const unsigned long long*)&p->s[2] + 1) << 64) |
                   __ldcg((const unsigned long long*)&p->s[2]));
  }
  block_sum_i128<3>(v, sRed);
  if (threadIdx.x == 0) {
    const int trunc = sel->do_trunc;
    const double kept = fx_to(v[0]);
    const double p2 = fx_to(v[1]);
    sel->kept = kept;
    sel->kept_p2 = p2;
    if (trunc) sel->total = fx_to(v[2]);
    if (mode == 1) {
      const long long n_kept = trunc ? (sel->k_keep > 0 ? sel->k_keep : 0) : sel->n_out;
      bass_ctrl* c = a.ctrl;
      const double pr_new = (n_kept == 0 || !(p2 > 0.0)) ? INFINITY : __ddiv_rn(__dmul_rn(kept, kept), p2);
      const bool reject = pr_new >= c->pr_cur * (1.0 - c->pr_tie_tol);
      c->frac[j] = kept;
      c->accept[j] = reject ? 0 : 1;
      sel->accept = reject ? 0 : 1;
      sel->pr_new = pr_new;
      sel->skip_write = (reject && !trace) ? 1 : 0;
    }
  }
  // exclusive scan of the per-tile counts: every thread owns a contiguous run
  // of C tiles (all its loads issued at once), one block scan of the run sums
  __shared__ long long sW[32];
  __shared__ long long sCarry;
  const long long n = a.in->nnz;
  const long long ntiles = (kind == K_IDENT) ? plain_tiles(n) : merge_tiles(n);
  const int t = threadIdx.x, lane = t & 31, w = t >> 5, nw = blockDim.x >> 5;
  const long long C = (ntiles + blockDim.x - 1) / blockDim.x;
  const long long lo = (long long)t * C;
  const long long hi = lo + C < ntiles ? lo + C : ntiles;
  constexpr int kRun = 8;
  long long cr[kRun];
  long long run = 0;
  if (C <= kRun) {
#pragma unroll
    for (int q = 0; q < kRun; ++q) {
      cr[q] = (lo + q < hi) ? (long long)__ldcg(a.ws.status + lo + q) : 0;
      run += cr[q];
    }
  } else {
    for (long long b = lo; b < hi; ++b) run += (long long)__ldcg(a.ws.status + b);
  }
  long long x = run;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const long long y = __shfl_up_sync(0xffffffffu, x, off);
    if (lane >= off) x += y;
  }
  if (lane == 31) sW[w] = x;
  __syncthreads();
  if (w == 0) {
    long long y = (lane < nw) ? sW[lane] : 0;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const long long z = __shfl_up_sync(0xffffffffu, y, off);
      if (lane >= off) y += z;
    }
    if (lane < nw) sW[lane] = y;
    if (lane == nw - 1) sCarry = y;
  }
  __syncthreads();
  long long ex = x - run + (w > 0 ? sW[w - 1] : 0);
  if (C <= kRun) {
#pragma unroll
    for (int q = 0; q < kRun; ++q) {
      if (lo + q < hi) a.ws.status[lo + q] = (unsigned long long)ex;
      ex += cr[q];
    }
  } else {
    for (long long b = lo; b < hi; ++b) {
      const long long c = (long long)__ldcg(a.ws.status + b);
      a.ws.status[b] = (unsigned long long)ex;
      ex += c;
    }
  }
  if (t == 0) {
    sel->n_written = sCarry;
    if (sCarry > a.out->cap) set_error(a.ctrl, BASS_ERR_CAPACITY);
  }
}

// After count_phase: the last block to finish settles the boundary bin (if
// late) and runs final_phase (the others exit), which needs every block's
// partial sums and tile counts.
template <bool P2>
__device__ void finish_by_last_block(const OpArgs& a, int ns, int kind, int mode, int j, int trace, i128* sRed,
                                     Grp g, bool late, unsigned long long lpre, long long lneed, const int8_t* qat) {
  __shared__ int sLast;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned long long d = atomicAdd(&reinterpret_cast<unsigned long long*>(a.ws.counters)[58], 1ULL);
    sLast = (d == (unsigned long long)g.nblk - 1);
    __threadfence();
  }
  __syncthreads();
  if (!sLast) return;
  const unsigned long long t0 = a.prof ? gtimer() : 0ULL;
  i128 vk[2] = {0, 0};
  if (late) settle_boundary<P2>(a, ns, kind, lpre, lneed, qat, vk);
  final_phase(a, g.nblk, kind, mode, j, trace, sRed, vk);
  if (a.prof && threadIdx.x == 0 && a.ws.sel->do_trunc) {
    unsigned long long* pin = reinterpret_cast<unsigned long long*>(a.ctrl->prof_in);
    unsigned long long* pout = reinterpret_cast<unsigned long long*>(a.ctrl->prof_out);
    atomicAdd(pin + S_SLOT_KEPT, gtimer() - t0);
    atomicAdd(pout + S_SLOT_KEPT, 1ULL);
  }
}

template <bool P2>
__device__ __forceinline__ void select_body(const OpArgs& a, Grp g, int ns, int kind, int nblk_hist, int mode, int j,
                                            int trace) {
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned int* h = reinterpret_cast<unsigned int*>(smem);
  __shared__ long long sS[kSelThreads / 32];
  __shared__ i128 sRed[3 * (kSelThreads / 32)];
  __shared__ long long sNout;
  __shared__ unsigned long long sBarGen;  // grid barriers passed by this block
  __shared__ int8_t sQat[64];
  SelState* sel = a.ws.sel;
  const int tid = threadIdx.x;
  const long long n = a.in->nnz;
  const long long nslots = (long long)ns * n;
  const long long ntiles = (kind == K_IDENT) ? plain_tiles(n) : merge_tiles(n);
  if (nslots > a.ws.max_n || ntiles > a.ws.max_tiles || n >= (1LL << 31)) {  // uniform: every block returns
    if (g.bid == 0 && tid == 0) set_error(a.ctrl, BASS_ERR_WORKSPACE);
    return;
  }
  const unsigned long long* slots = reinterpret_cast<const unsigned long long*>(a.ws.tmp_keys);
  // profiling: block 0 times its phases (level 1, level 2, count pass),
  // barrier waits included; the last block times the boundary settle and the
  // final phase
  const bool ptime = a.prof && g.bid == 0 && tid == 0;
  unsigned long long tp[4] = {0, 0, 0, 0};
  if (ptime) tp[0] = gtimer();
  // 1. the child count
  long long cn = 0;
  for (int b = tid; b < nblk_hist; b += blockDim.x) cn += __ldcg(&a.ws.partials[b].c[0]);
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) cn += __shfl_down_sync(0xffffffffu, cn, off);
  if ((tid & 31) == 0) sS[tid >> 5] = cn;
  __syncthreads();
  if (tid == 0) {
    long long s = 0;
    for (int w = 0; w < kSelThreads / 32; ++w) s += sS[w];
    sNout = s;
    sBarGen = 0ULL;
  }
  __syncthreads();
  const long long n_out = sNout;
  const bool trunc = !(a.k_cond < 0 || n_out <= a.k_cond || a.k_keep >= n_out);
  unsigned long long T = 0ULL, tkey = ~0ULL;
  bool incl = true;
  bool late = false;  // the threshold lies inside the level-2 bin lpre: settled by the last block
  unsigned long long lpre = 0;
  long long lneed = 0;
  int two = 0;        // a level-2 pass was needed
  if (trunc && a.k_keep <= 0) {
    T = ~0ULL;
    tkey = 0ULL;
    incl = false;
  } else if (trunc) {
    // 2. radix select on the bit patterns
    slot_hist_phase<1>(slots, nslots, 0, h, a.ws.hist1, g);
    if (!grid_sync(a, g, sBarGen)) return;
    long long c_gt, c_b1;
    const int b1 = find_bin(a.ws.hist1, a.k_keep, &c_gt, &c_b1);
    const long long need = a.k_keep - c_gt;
    if (ptime) tp[1] = gtimer();
    if (c_b1 == need) {
      T = (unsigned long long)b1 << 50;
    } else {
      two = 1;
      slot_hist_phase<2>(slots, nslots, (unsigned long long)b1, h, a.ws.hist2, g);
      if (!grid_sync(a, g, sBarGen)) return;
      long long c_gt2, c_b2;
      const int b2 = find_bin(a.ws.hist2, need, &c_gt2, &c_b2);
      const long long need2 = need - c_gt2;
      const unsigned long long pre = ((unsigned long long)b1 << 13) | (unsigned long long)b2;
      if (c_b2 == need2) {
        T = pre << 37;
      } else {
        // the bin's children are settled after the count pass, which keeps
        // everything above the bin and lists the bin itself
        late = true;
        lpre = pre;
        lneed = need2;
        T = (pre + 1) << 37;
      }
    }
  }
  if (g.bid == 0 && tid == 0) {
    sel->n_out = n_out;
    sel->k_keep = a.k_keep;
    sel->do_trunc = trunc ? 1 : 0;
    sel->stage = trunc ? 3 : 0;
    sel->t_bits = T;
    sel->t_key = tkey;
  }
  if (late) {
    out_order_par(a.in, kind, a.q, a.gb, sQat);
    __syncthreads();
    if (g.bid == 0 && tid < 64) sel->qat[tid] = sQat[tid];
  }
  // 3. survivors per tile and exact sums
  if (ptime) tp[2] = gtimer();
  count_phase<P2>(a, ns, kind, trunc ? T : 0ULL, incl, trunc, sRed, late, lpre, g);
  if (ptime && trunc) {
    tp[3] = gtimer();
    if (!tp[1]) tp[1] = tp[0];
    unsigned long long* pin = reinterpret_cast<unsigned long long*>(a.ctrl->prof_in);
    unsigned long long* pout = reinterpret_cast<unsigned long long*>(a.ctrl->prof_out);
    for (int q = 0; q < 3; ++q) {
      atomicAdd(pin + S_SLOT_HIST1 + q, tp[q + 1] - tp[q]);
      atomicAdd(pout + S_SLOT_HIST1 + q, 1ULL);
    }
    atomicAdd(pin + S_SLOT_KEPT + 1, (unsigned long long)two);
    atomicAdd(pout + S_SLOT_KEPT + 1, 1ULL);
  }
  // 4. boundary bin, sums, decision, tile offsets
  pdl_trigger();
  finish_by_last_block<P2>(a, ns, kind, mode, j, trace, sRed, g, late, lpre, lneed, sQat);
}

// nblk_hist: CTAs of the evaluation pass (per-CTA child counts in partials c[0]).
template <bool P2>
__global__ void __launch_bounds__(kSelThreads) k_select_coop(const __grid_constant__ OpArgs a, int ns, int kind,
                                                              int nblk_hist, int mode, int j, int trace) {
  pdl_wait();
  select_body<P2>(a, whole_grid(), ns, kind, nblk_hist, mode, j, trace);
}

// ---------------------------------------------------------------------------
// the write step of a gate / rotation / truncation: compaction
// ---------------------------------------------------------------------------
// One CTA per tile (block-strided).  The tile's children sit at its slot
// range [NS * P'_b, NS * P'_{b+1}) of the staging arrays, in output order; the
// survivors are written from the tile's base (the selection's scan of the
// tile counts) on.  Which children survive is read from the selection's kept
// mask (one bit per slot: its count pass and boundary settle).  The range is
// taken in chunks of kChunk slots: thread 0 copies the chunk's staged
// amplitudes, staged keys and mask words into shared memory with TMA bulk
// copies (their 16-byte aligned bodies; warp 0 fetches the at most two ragged
// 8-byte end entries of each array with plain loads); then the survivors are
// ranked and written from shared memory.
// The last CTA to finish writes the output descriptor.  A rejected rotation
// candidate is not written.
constexpr int kChunk = 8 * kThreads;  // slots per chunk (one round of eight per thread)
constexpr int kChunkPad = kChunk + 2;  // an odd first entry sits one position in
constexpr int kMaskWords = kChunk / 32 + 8;  // the chunk's kept-mask words, from a 16-byte boundary
// dynamic shared memory of the compaction: amplitudes (16 B), keys, mask words
constexpr size_t kCompactSmem = (size_t)kChunkPad * (16 + 8) + 4 * kMaskWords;

// Bulk copy of entries [lo, hi) of an array of `esz`-byte entries (esz 8 or
// 16) into shared memory at position (index - (lo & ~1)), so that both ends
// are 16-byte aligned (body_bytes: the bytes it copies).  For 8-byte entries
// the ragged entries lo (odd) and hi - 1 (even) are left to copy_ragged.
__device__ __forceinline__ unsigned body_bytes(long long lo, long long hi, unsigned esz) {
  const long long f = esz == 16 ? lo : (lo + 1) & ~1LL;
  const long long l = esz == 16 ? hi : hi & ~1LL;
  return (hi <= lo || l <= f) ? 0u : (unsigned)(esz * (l - f));
}
__device__ __forceinline__ void copy_body(void* dst, const void* src, long long lo, long long hi, unsigned esz,
                                          uint64_t* bar) {
  const unsigned nb = body_bytes(lo, hi, esz);
  if (nb == 0) return;
  const long long f = esz == 16 ? lo : (lo + 1) & ~1LL;
  const long long e0 = lo & ~1LL;
  bulk_load(static_cast<unsigned char*>(dst) + esz * (f - e0), static_cast<const unsigned char*>(src) + esz * f, nb,
            bar);
}
// The entry of [lo, hi) that copy_body leaves out at its start (last = false)
// or end (last = true), if any, by a plain load.
template <typename E>
__device__ __forceinline__ void copy_ragged(E* dst, const E* src, long long lo, long long hi, bool last) {
  if (sizeof(E) == 16 || hi <= lo) return;
  const long long f = (lo + 1) & ~1LL, l = hi & ~1LL, e0 = lo & ~1LL;
  if (last ? l < hi : lo < f) {
    const long long i = last ? l : lo;
    dst[i - e0] = src[i];
  }
}

template <bool C64>
__device__ __forceinline__ void compact_body(const OpArgs& a, Grp g, int ns, int kind) {
  extern __shared__ __align__(16) unsigned char smem[];
  double2* cA = reinterpret_cast<double2*>(smem);                                  // amplitudes
  float2* cAf = reinterpret_cast<float2*>(cA);
  uint64_t* cK = reinterpret_cast<uint64_t*>(cA + kChunkPad);                      // staged keys
  unsigned int* cM = reinterpret_cast<unsigned int*>(cK + kChunkPad);              // kept-mask words
  __shared__ SelState S;
  __shared__ int sCnt[8][kThreads / 32];  // survivors per (round u, warp)
  __shared__ uint64_t sBar;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  load_sel(&S, a.ws.sel);
  if (tid == 0) mbar_init(&sBar, 1);
  __syncthreads();
  const long long n = a.in->nnz;
  const long long ntiles = (kind == K_IDENT) ? plain_tiles(n) : merge_tiles(n);
  const unsigned int* kmw = reinterpret_cast<const unsigned int*>(a.ws.kmask);  // 32 slots per word
  const bool aligned = ((reinterpret_cast<uintptr_t>(a.ws.tmp_amps) | reinterpret_cast<uintptr_t>(a.ws.stage_keys) |
                         reinterpret_cast<uintptr_t>(kmw)) & 15) == 0;
  const bool ok = ntiles <= a.ws.max_tiles && (long long)ns * n <= a.ws.max_n && aligned;
  if (!ok && g.bid == 0 && tid == 0) set_error(a.ctrl, BASS_ERR_WORKSPACE);
  uint64_t* okeys = a.out->keys;
  double2* oamps = reinterpret_cast<double2*>(a.out->amps);
  float2* oampf = reinterpret_cast<float2*>(a.out->amps);
  const float2* stf = reinterpret_cast<const float2*>(a.ws.tmp_amps);
  constexpr bool c64 = C64;
  constexpr unsigned kAmpBytes = C64 ? 8u : 16u;
  const long long cap = a.out->cap;
  const int lns = ns == 4 ? 2 : ns == 2 ? 1 : 0;
  const unsigned lt = (1u << lane) - 1;
  long long written = 0;
  unsigned phase = 0;
  bool stop = !ok || S.skip_write;
  for (long long b = g.bid; !stop && b < ntiles; b += g.nblk) {
    long long z0, z1;
    if (kind == K_IDENT) {
      z0 = b * kTile;
      z1 = (z0 + kTile < n) ? z0 + kTile : n;
    } else {
      z0 = a.ws.part[b * 6];
      z1 = a.ws.part[(b + 1) * 6];
    }
    const long long s1 = ns * z1;
    long long base = (long long)a.ws.status[b];
    // chunks of 8 x 256 slots; slot (u, tid) = i0 + 256 u + tid, so every
    // warp's shared reads and global stores cover consecutive slots
    for (long long i0 = ns * z0; i0 < s1; i0 += kChunk) {
      const long long i1 = (i0 + kChunk < s1) ? i0 + kChunk : s1;
      const long long q0 = i0 >> lns, q1 = ((i1 - 1) >> lns) + 1;  // staged keys of the chunk
      const long long e0 = i0 & ~1LL, k0 = q0 & ~1LL;
      // mask words [m0, m1): every word of the chunk's slots and the one after
      // (the funnel shift's high word), widened to 16-byte boundaries; inside
      // the mask's nslots / 8 + 64 bytes
      const long long m0 = (i0 >> 5) & ~3LL, m1 = ((((i1 - 1) >> 5) + 2) + 3) & ~3LL;
      if (tid == 0) {
        fence_proxy_async_smem();  // the previous chunk's shared accesses (barrier at its end)
        // the expected bytes first (one arrival), then the copies
        mbar_arrive_expect(&sBar, body_bytes(i0, i1, kAmpBytes) + body_bytes(q0, q1, 8) + 4u * (unsigned)(m1 - m0));
        bulk_load(cM, kmw + m0, 4u * (unsigned)(m1 - m0), &sBar);
        if (C64) copy_body(cAf, stf, i0, i1, 8, &sBar);
        else copy_body(cA, a.ws.tmp_amps, i0, i1, 16, &sBar);
        copy_body(cK, a.ws.stage_keys, q0, q1, 8, &sBar);
      }
      if (tid < 4) {
        const bool last = tid & 1;
        if (tid < 2) {
          if (C64) copy_ragged(cAf, stf, i0, i1, last);
        } else {
          copy_ragged(cK, a.ws.stage_keys, q0, q1, last);
        }
      }
      bool done = false;
      for (long long sp = 0; sp < kSpinLimit && !done; ++sp) done = mbar_try_wait(&sBar, phase);
      phase ^= 1u;
      if (__syncthreads_or(!done)) {
        if (tid == 0) set_error(a.ctrl, BASS_ERR_WAIT);
        stop = true;
        break;
      }
      // the kept bits of the warp's 32 slots of each round u (slots i0 + 256 u
      // + 32 w .. + 31; two mask words, shifted to the warp's first slot, the
      // slots past the chunk cleared)
      unsigned bal[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const long long p0 = i0 + u * kThreads + 32 * w;
        const long long nv = i1 - p0;  // slots of the chunk among the 32
        unsigned bits = 0;
        if (nv > 0) {
          const int mw = (int)((p0 >> 5) - m0);
          bits = __funnelshift_r(cM[mw], cM[mw + 1], (unsigned)(p0 & 31));
        }
        bal[u] = nv >= 32 ? bits : (nv <= 0 ? 0u : bits & ((1u << nv) - 1u));
      }
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (lane == 0) sCnt[u][w] = __popc(bal[u]);
      __syncthreads();
      // the 64 survivor counts in slot order (round major, warp minor): every
      // warp scans them itself, lane l holding entries 2l and 2l + 1
      static_assert(8 * (kThreads / 32) == 64, "two counts per lane");
      const int* fc = &sCnt[0][0];
      const int c0 = fc[2 * lane], c1 = fc[2 * lane + 1];
      int inc = c0 + c1;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, inc, off);
        if (lane >= off) inc += y;
      }
      const int tot = __shfl_sync(0xffffffffu, inc, 31);  // survivors of the chunk
      const int mine = (w & 1) ? inc - c1 : inc - c0 - c1;  // offset of entry 2l + (w & 1)
      if (base + tot <= cap) {
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int ahead = __shfl_sync(0xffffffffu, mine, u * 4 + (w >> 1));  // entry 8u + w
          if ((bal[u] >> lane) & 1u) {
            const long long i = i0 + u * kThreads + tid;
            const long long o = base + ahead + __popc(bal[u] & lt);
            okeys[o] = cK[(i >> lns) - k0] | (uint64_t)(i & ((1LL << lns) - 1));
            if (c64) oampf[o] = cAf[i - e0];
            else oamps[o] = cA[i - e0];
          }
        }
      } else if (tid == 0) {
        set_error(a.ctrl, BASS_ERR_CAPACITY);
      }
      base += tot;
      written += tot;
      __syncthreads();  // sCnt and the chunk buffers are reused by the next chunk
    }
  }
  if (tid == 0 && a.prof && written)
    atomicAdd(reinterpret_cast<unsigned long long*>(&a.ctrl->prof_out[kind * 5 + P_WRITE]),
              (unsigned long long)written);
  // the last CTA to finish writes the output descriptor
  pdl_trigger();
  write_done(a, kind, g);
}

template <bool C64>
__global__ void __launch_bounds__(256) k_compact(const __grid_constant__ OpArgs a, int ns, int kind) {
  pdl_wait();
  compact_body<C64>(a, whole_grid(), ns, kind);
}

// ---------------------------------------------------------------------------
// RDM moments of the qubits at low physical bits: one pass
// ---------------------------------------------------------------------------
// bass_simulator.py:441-470 for every qubit whose physical bit t is below
// kRdmLowBits, without a merge pass per qubit: the state is read in plain
// tiles of kTile entries (key order) plus the next kRdmHalo entries, which
// hold the partner x | 2^t of every tile entry x with bit t clear (the keys
// between x and x + 2^t are distinct integers, so at most 2^t - 1 of them
// come first); a binary search over at most 2^t positions finds it.  The four
// moments of each such qubit (|a|^2 of its bit-0 and bit-1 entries, re and im
// of a_x conj(a_{x | 2^t})) are the sums of k_tile's P_RDM pass, exact:
// each warp adds its lanes' sums into its own shared accumulators, and at the
// end every CTA writes one partial per qubit (slot blockIdx.x of the qubit's
// set; the grid, at most ws.max_tiles, goes to counter 6 for k_rdm_final).
constexpr int kRdmSpan = kTile + kRdmHalo;
constexpr int kRdmSpanPad = kRdmSpan + 2;
constexpr size_t kRdmLowSmem = (size_t)kRdmSpanPad * (16 + 8);  // amplitudes, keys

template <bool C64>
__global__ void __launch_bounds__(kThreads) k_rdm_low(const __grid_constant__ OpArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  double2* sA = reinterpret_cast<double2*>(smem);
  float2* sAf = reinterpret_cast<float2*>(sA);
  uint64_t* sK = reinterpret_cast<uint64_t*>(sA + kRdmSpanPad);
  __shared__ uint64_t sBar;
  __shared__ long long sItem;
  __shared__ i128 sAcc[kThreads / 32][kRdmLowBits][4];  // per warp, qubit and moment
  __shared__ int sSet[kRdmLowBits];  // the set of the qubit at physical bit t, or -1
  pdl_wait();
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  for (int i = lane; i < kRdmLowBits * 4; i += 32) sAcc[w][i >> 2][i & 3] = 0;
  const bass_state* in = a.in;
  const long long n = in->nnz;
  const long long ntiles = plain_tiles(n);
  if (tid == 0) mbar_init(&sBar, 1);
  if (tid < kRdmLowBits) {
    int set = -1;
    if (tid < in->nq) {
      const int q = in->qat[tid] - a.q;
      if (q >= 0 && q < a.nsets) set = q;
    }
    sSet[tid] = set;
  }
  const double r0 = in->rscale[0], r1 = in->rscale[1];
  const bool scaled = !(r0 == 1.0 && r1 == 1.0);
  const uint64_t* keys = in->keys;
  const double2* amps = reinterpret_cast<const double2*>(in->amps);
  const float2* ampf = reinterpret_cast<const float2*>(in->amps);
  // bulk copies need both arrays 16-byte aligned; keys at an 8-byte offset
  // take plain loads
  const bool bulk = ((reinterpret_cast<uintptr_t>(keys) | reinterpret_cast<uintptr_t>(amps)) & 15) == 0;
  const bool bad = ntiles > a.ws.max_tiles || (in->amp_type == BASS_AMP_C64) != C64;
  if (bad && blockIdx.x == 0 && tid == 0) set_error(a.ctrl, BASS_ERR_WORKSPACE);
  auto amp = [&](int p) {
    const double2 v = C64 ? f2d(sAf[p]) : sA[p];
    return scaled ? amp_scale(v, C64 ? 1 : 0, r0, r1) : v;
  };
  __syncthreads();
  unsigned phase = 0;
  unsigned long long* item_ctr = &reinterpret_cast<unsigned long long*>(a.ws.counters)[a.counter];
  for (;;) {
    if (tid == 0) sItem = bad ? ntiles : (long long)atomicAdd(item_ctr, 1ULL);
    __syncthreads();
    const long long b = sItem;
    if (b >= ntiles) break;
    const long long lo = b * kTile;  // even: both arrays start on 16-byte words
    const long long own_end = (lo + kTile < n) ? lo + kTile : n;
    const long long hi = (own_end + kRdmHalo < n) ? own_end + kRdmHalo : n;
    const int own = (int)(own_end - lo), E = (int)(hi - lo);
    if (bulk) {
      if (tid == 0) {
        fence_proxy_async_smem();  // the previous tile's shared accesses (barrier above)
        mbar_arrive_expect(&sBar, body_bytes(lo, hi, 8) + body_bytes(lo, hi, C64 ? 8u : 16u));
        copy_body(sK, keys, lo, hi, 8, &sBar);
        if (C64) copy_body(sAf, ampf, lo, hi, 8, &sBar);
        else copy_body(sA, amps, lo, hi, 16, &sBar);
      }
      // an odd last entry of the 8-byte arrays (lo is even: no odd first one)
      if (tid == 0) copy_ragged(sK, keys, lo, hi, true);
      if (C64 && tid == 1) copy_ragged(sAf, ampf, lo, hi, true);
      bool done = false;
      for (long long sp = 0; sp < kSpinLimit && !done; ++sp) done = mbar_try_wait(&sBar, phase);
      phase ^= 1u;
      if (__syncthreads_or(!done)) {
        if (tid == 0) set_error(a.ctrl, BASS_ERR_WAIT);
        break;
      }
    } else {
      for (int i = tid; i < E; i += kThreads) {
        sK[i] = keys[lo + i];
        if (C64) sAf[i] = ampf[lo + i];
        else sA[i] = amps[lo + i];
      }
      __syncthreads();
    }
    if (a.prof && tid == 0)
      atomicAdd(reinterpret_cast<unsigned long long*>(&a.ctrl->prof_in[K_RDM * 5 + P_HIST]), (unsigned long long)E);
    for (int t = 0; t < kRdmLowBits; ++t) {
      const int set = sSet[t];
      if (set < 0) continue;  // the same for every thread
      const uint64_t bit = 1ULL << t;
      const int reach = 1 << t;  // the partner lies at most this many positions on
      // at most kPerThread positions per thread: at most eight terms per
      // split accumulator (fx_acc96) before they are joined
      i128 v[4] = {0, 0, 0, 0};
      double dh[4] = {0.0, 0.0, 0.0, 0.0}, dl[4] = {0.0, 0.0, 0.0, 0.0};
      for (int e = tid; e < own; e += kThreads) {
        const uint64_t x = sK[e];
        const double2 ax = amp(e);
        if (x & bit) {
          fx_acc96(prob(ax), dh[1], dl[1], v[1]);
          continue;
        }
        fx_acc96(prob(ax), dh[0], dl[0], v[0]);
        const uint64_t y = x | bit;
        int L = e + 1;
        const int R0 = (e + reach < E - 1 ? e + reach : E - 1) + 1;  // search [e + 1, R0)
        int R = R0;
        while (L < R) {
          const int m = (L + R) >> 1;
          if (sK[m] < y) L = m + 1;
          else R = m;
        }
        if (L < R0 && sK[L] == y) {
          const double2 ay = amp(L);
          const double2 c = cmul(ax, make_double2(ay.x, -ay.y));
          fx_acc96(c.x, dh[2], dl[2], v[2]);
          fx_acc96(c.y, dh[3], dl[3], v[3]);
        }
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        v[k] += fx_join96s(dh[k], dl[k]);
        v[k] = warp_sum_i128(v[k]);
      }
      if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 4; ++k) sAcc[w][t][k] += v[k];
      }
    }
    __syncthreads();  // the buffers are reused by the next tile
  }
  // the CTA's sums: thread (t, k) adds the warps' accumulators
  __syncthreads();
  if (tid < kRdmLowBits * 4) {
    const int t = tid >> 2, k = tid & 3, set = sSet[t];
    if (set >= 0 && !bad) {
      i128 sum = 0;
#pragma unroll
      for (int ww = 0; ww < kThreads / 32; ++ww) sum += sAcc[ww][t][k];
      a.ws.partials[(long long)set * a.ws.max_tiles + blockIdx.x].s[k] = sum;
    }
  }
  if (blockIdx.x == 0 && tid == 0)
    reinterpret_cast<unsigned long long*>(a.ws.counters)[6] = gridDim.x;
}

// Rotation step, after the write pass: keep the candidate if accepted.
__global__ void k_commit(bass_state* cur, bass_state* tmp, WsView ws, bass_ctrl* c, int j, int trace) {
  const SelState* sel = ws.sel;
  if (!sel->accept) return;
  bass_state t = *cur;
  *cur = *tmp;
  *tmp = t;
  c->pr_cur = sel->pr_new;
  const double frac = c->frac[j];
  c->gamma_running *= sqrt(frac > 1e-30 ? frac : 0.0);
  if (trace && c->trace) {
    const long long i = c->trace_len;
    if (i >= c->trace_cap) {
      set_error(c, BASS_ERR_CAPACITY);
      return;
    }
    uint64_t* e = c->trace + i * BASS_TRACE_WORDS;
    e[0] = 1;
    e[1] = (uint64_t)j;
    for (int k = 2; k < BASS_TRACE_WORDS; ++k) e[k] = 0;
    c->trace_len = i + 1;
  }
}

// low: the sets of qubits at physical bits below kRdmLowBits hold k_rdm_low's
// partials (one per CTA of its grid, counter 6), the others the merge pass's
// (one per merge tile)
__global__ void k_rdm_final(const bass_state* st, double* rho, WsView ws, int first, int low) {
  __shared__ i128 sRed[4 * 8];
  const int set = blockIdx.x;
  const long long n = st->nnz;
  const long long ntiles = (low && st->pos[first + set] < kRdmLowBits)
                               ? (long long)reinterpret_cast<const unsigned long long*>(ws.counters)[6]
                               : merge_tiles(n);
  i128 v[4] = {0, 0, 0, 0};
  for (long long t = threadIdx.x; t < ntiles; t += blockDim.x) {
    const Partial& p = ws.partials[(long long)set * ws.max_tiles + t];
    v[0] += p.s[0]; v[1] += p.s[1]; v[2] += p.s[2]; v[3] += p.s[3];
  }
  block_sum_i128<4>(v, sRed);
  if (threadIdx.x == 0) {
    double* r = rho + 4 * (first + set);
    r[0] = fx_to(v[0]);
    r[1] = fx_to(v[1]);
    r[2] = fx_to(v[2]);
    r[3] = fx_to(v[3]);
  }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
// Dynamic shared memory of a tile pass and its persistent grid (every CTA
// that fits at once, at most 1024), set up on first use.
template <int KIND, int PASS, bool C64>
static cudaError_t tile_grid(size_t* smem_out, int* grid_out) {
  const size_t smem = (size_t)kTilePad * (16 + 8 + 2 + (PASS == P_WRITE ? 3 : 0));
  static PerDevice cache;
  *smem_out = smem;
  return per_device(cache, grid_out, [smem](int* grid) {
    cudaError_t e = cudaFuncSetAttribute(k_tile<KIND, PASS, C64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int occ = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_tile<KIND, PASS, C64>, kThreads, smem);
    if (e != cudaSuccess) return e;
    *grid = device().sms * (occ > 0 ? occ : 1);
    if (*grid > 1024) *grid = 1024;
    return cudaSuccess;
  });
}

template <int KIND, int PASS, bool C64>
static cudaError_t launch_tile_t(OpArgs a, int counter, cudaStream_t s, int* grid_out) {
  size_t smem = 0;
  int grid = 0;
  cudaError_t e = tile_grid<KIND, PASS, C64>(&smem, &grid);
  if (e != cudaSuccess) return e;
  a.counter = counter;
  a.prof = prof_on() ? 1 : 0;
  KLAUNCH(KIND * 5 + PASS, s, launch_pdl(k_tile<KIND, PASS, C64>, dim3(grid), dim3(kThreads), smem, s, a));
  if (grid_out) *grid_out = grid;
  return cudaGetLastError();
}

// the tile pass for the op's amplitude type (a.c64, from the host's record of the state)
template <int KIND, int PASS>
static cudaError_t launch_tile(OpArgs a, int counter, cudaStream_t s, int* grid_out) {
  return a.c64 ? launch_tile_t<KIND, PASS, true>(a, counter, s, grid_out)
               : launch_tile_t<KIND, PASS, false>(a, counter, s, grid_out);
}

cudaError_t zero_small(const WsView& ws, cudaStream_t s) {
  // counters, hist1, hist2, sel and the look-back status words are contiguous
  const size_t bytes = (size_t)((char*)(ws.status + ws.max_tiles) - (char*)ws.counters);
  return cudaMemsetAsync(ws.counters, 0, bytes, s);
}

// A cooperative launch (the runtime guarantees that every block of the grid
// is resident at once, or refuses the launch), as a programmatic dependent
// launch where the runtime accepts both attributes together; otherwise a
// plain cooperative launch.  The choice is made on the first launch and kept.
template <typename... K, typename... A>
static cudaError_t launch_coop(void (*kern)(K...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                               A&&... args) {
  static std::atomic<int> with_pdl{1};
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[2];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  if (with_pdl.load(std::memory_order_relaxed)) {
    cfg.numAttrs = 2;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, kern, args...);
    if (e == cudaSuccess) return e;
    cudaGetLastError();  // refused before launch: clear it and launch without PDL
    with_pdl.store(0, std::memory_order_relaxed);
  }
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, std::forward<A>(args)...);
}

// Launch of the selection; grid = every block that fits on the GPU at once
// (its grid barriers need them all resident), launched cooperatively so that
// the runtime guarantees that residency.  Where it is also a programmatic
// dependent launch, each block waits until the evaluation pass has completed.
template <bool P2>
static cudaError_t launch_select_t(OpArgs a, int ns, int kind, int gh, int mode, int j, int trace,
                                   cudaStream_t s) {
  const size_t smem = kSelSmem;
  static PerDevice cache;
  int grid = 0;
  cudaError_t e = per_device(cache, &grid, [smem](int* g) {
    const void* f = (const void*)k_select_coop<P2>;
    cudaError_t e2 = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e2 != cudaSuccess) return e2;
    int occ = 0;
    e2 = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, f, kSelThreads, smem);
    if (e2 != cudaSuccess) return e2;
    if (occ < 1) return cudaErrorInvalidConfiguration;
    *g = device().sms * occ;
    if (*g > 1024) *g = 1024;  // per-CTA partials
    return cudaSuccess;
  });
  if (e != cudaSuccess) return e;
  a.prof = prof_on() ? 1 : 0;
  dim3 grd(grid), blk(kSelThreads);
  KLAUNCH(S_SELECT1, s, e = launch_coop(k_select_coop<P2>, grd, blk, smem, s, a, ns, kind, gh, mode, j, trace));
  return e;
}

static cudaError_t launch_select(OpArgs a, int ns, int kind, int gh, int mode, int j, int trace, cudaStream_t s) {
  return mode == 1 ? launch_select_t<true>(a, ns, kind, gh, mode, j, trace, s)
                   : launch_select_t<false>(a, ns, kind, gh, mode, j, trace, s);
}

// Opts a kernel of kThreads threads in to `smem` bytes of dynamic shared
// memory and returns its resident grid (once per device).
template <typename K>
static cudaError_t smem_grid(PerDevice& cache, K kern, size_t smem, int* grid) {
  return per_device(cache, grid, [kern, smem](int* v) {
    cudaError_t e = cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int occ = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kThreads, smem);
    if (e != cudaSuccess) return e;
    *v = device().sms * (occ > 0 ? occ : 1);
    return cudaSuccess;
  });
}

template <int KIND>
static cudaError_t merge_op(OpArgs a, const bass_trunc& tr, int fin_mode, int j, cudaStream_t s) {
  cudaError_t e = cudaSuccess;
  a.k_cond = tr.k_cond;
  a.k_keep = tr.k_keep;
  a.nsets = 1;
  if constexpr (KIND != K_IDENT) {
    // the partition also clears the small workspace region
    KLAUNCH(S_PARTITION, s, launch_pdl(k_partition, dim3(device().grid_small, 1), dim3(256), 0, s, a, (int)KIND, 1));
  } else {
    if ((e = zero_small(a.ws, s)) != cudaSuccess) return e;
  }
  if constexpr (KIND != K_PERM) {
    constexpr int ns = slots_per_entry(KIND);
    int gh = 0;
    if ((e = launch_tile<KIND, P_HIST>(a, 0, s, &gh)) != cudaSuccess) return e;
    if ((e = launch_select(a, ns, KIND, gh, fin_mode, j, tr.trace, s)) != cudaSuccess) return e;
  }
  a.fin = 1;
  a.fin_mode = fin_mode;
  a.tr = tr;
  a.j = j;
  if constexpr (KIND == K_PERM) {
    a.write_mode = 2;
    return launch_tile<KIND, P_WRITE>(a, 3, s, nullptr);
  } else {
    a.prof = prof_on() ? 1 : 0;
    static PerDevice grid_c64, grid_c128;
    int gc = 0;
    if ((e = a.c64 ? smem_grid(grid_c64, k_compact<true>, kCompactSmem, &gc)
                   : smem_grid(grid_c128, k_compact<false>, kCompactSmem, &gc)) != cudaSuccess)
      return e;
    if (a.c64)
      KLAUNCH(KIND * 5 + P_WRITE, s,
              launch_pdl(k_compact<true>, dim3(gc), dim3(kThreads), kCompactSmem, s, a,
                         (int)slots_per_entry(KIND), (int)KIND));
    else
      KLAUNCH(KIND * 5 + P_WRITE, s,
              launch_pdl(k_compact<false>, dim3(gc), dim3(kThreads), kCompactSmem, s, a,
                         (int)slots_per_entry(KIND), (int)KIND));
    return cudaGetLastError();
  }
}

cudaError_t run_merge_op(int kind, OpArgs a, const bass_trunc& tr, int finalize_mode, int j,
                         cudaStream_t s) {
  switch (kind) {
    case K_GATE1: return merge_op<K_GATE1>(a, tr, finalize_mode, j, s);
    case K_ROT1: return merge_op<K_ROT1>(a, tr, finalize_mode, j, s);
    case K_GATE2: return merge_op<K_GATE2>(a, tr, finalize_mode, j, s);
    case K_PERM: return merge_op<K_PERM>(a, tr, finalize_mode, j, s);
    case K_IDENT: return merge_op<K_IDENT>(a, tr, finalize_mode, j, s);
  }
  return cudaErrorInvalidValue;
}

cudaError_t run_commit(bass_state* cur, bass_state* tmp, bass_ctrl* ctrl, const WsView& ws, int j, int trace,
                       cudaStream_t s) {
  KLAUNCH(S_REDUCE, s, k_commit<<<1, 1, 0, s>>>(cur, tmp, ws, ctrl, j, trace));
  return cudaGetLastError();
}

// write pass only (keep everything the drop rule keeps); used by the guarded
// compaction after a 1-qubit diagonal gate.  The caller zeroed the small region.
cudaError_t run_ident_write(OpArgs a, cudaStream_t s) {
  a.write_mode = 0;
  return launch_tile<K_IDENT, P_WRITE>(a, 3, s, nullptr);
}

cudaError_t run_rdm(const bass_state* st, int nq, double* rho, bass_ctrl* ctrl, const WsView& ws,
                    cudaStream_t s, int c64) {
  cudaError_t e = cudaSuccess;
  OpArgs a{};
  a.c64 = c64;
  a.in = st;
  a.out = nullptr;
  a.ctrl = ctrl;
  a.ws = ws;
  a.q = 0;
  a.gb = 0;
  a.nsets = nq;
  a.rdm_low = 1;
  // the partition also clears the small workspace region; the qubits at
  // physical bits below kRdmLowBits take one pass of k_rdm_low instead of a
  // partition and a merge pass each
  KLAUNCH(S_PARTITION, s, launch_pdl(k_partition, dim3(device().grid_small, nq), dim3(256), 0, s, a, (int)K_RDM, 1));
  if ((e = launch_tile<K_RDM, P_RDM>(a, 0, s, nullptr)) != cudaSuccess) return e;
  {
    static PerDevice grid_c64, grid_c128;
    int gl = 0;
    if ((e = c64 ? smem_grid(grid_c64, k_rdm_low<true>, kRdmLowSmem, &gl)
                 : smem_grid(grid_c128, k_rdm_low<false>, kRdmLowSmem, &gl)) != cudaSuccess)
      return e;
    if (gl > ws.max_tiles) gl = (int)ws.max_tiles;  // one partial slot per CTA
    a.counter = 5;
    a.prof = prof_on() ? 1 : 0;
    if (c64)
      KLAUNCH(K_RDM * 5 + P_HIST, s, launch_pdl(k_rdm_low<true>, dim3(gl), dim3(kThreads), kRdmLowSmem, s, a));
    else
      KLAUNCH(K_RDM * 5 + P_HIST, s, launch_pdl(k_rdm_low<false>, dim3(gl), dim3(kThreads), kRdmLowSmem, s, a));
  }
  KLAUNCH(S_RDM_FINAL, s, k_rdm_final<<<nq, 256, 0, s>>>(st, rho, ws, 0, 1));
  return cudaGetLastError();
}

// 4x4 moments of the qubit pair (q1, q2): the first pass of a 2-qubit gate
// brings q2 to bit 0 (st -> tmp), then one moment pass over tmp groups the
// entries by every other bit with q1 at bit 1.  rho: 16 doubles, see k_tile's
// P_RDM pass for K_GATE2 (set s writes rho[4 s .. 4 s + 3]).
cudaError_t run_rdm_2q(const bass_state* st, bass_state* tmp, int q1, int q2, double* rho, bass_ctrl* ctrl,
                       const WsView& ws, cudaStream_t s, int c64) {
  OpArgs a{};
  a.c64 = c64;
  a.in = st; a.out = tmp; a.ctrl = ctrl; a.ws = ws; a.q = q2; a.gb = 0;
  bass_trunc none{};
  none.k_cond = -1;
  cudaError_t e = run_merge_op(K_PERM, a, none, 0, 0, s);
  if (e != cudaSuccess) return e;
  OpArgs b{};
  b.in = tmp; b.out = nullptr; b.ctrl = ctrl; b.ws = ws; b.q = q1; b.gb = 1; b.nsets = 4; b.c64 = c64;
  // the partition also clears the small workspace region
  KLAUNCH(S_PARTITION, s, launch_pdl(k_partition, dim3(device().grid_small, 1), dim3(256), 0, s, b, (int)K_GATE2, 1));
  if ((e = launch_tile<K_GATE2, P_RDM>(b, 0, s, nullptr)) != cudaSuccess) return e;
  KLAUNCH(S_RDM_FINAL, s, k_rdm_final<<<4, 256, 0, s>>>(tmp, rho, ws, 0, 0));
  return cudaGetLastError();
}

// RDM moments with a caller-prepared workspace view: the same kernels as
// run_rdm, without clearing any workspace region (the caller clears the tile
// counters) and with a final reduction that refuses states whose tile count
// exceeds the view's capacity.  Used by the no-allocation entry point.
__global__ void k_rdm_final_bounded(const bass_state* st, double* rho, WsView ws, bass_ctrl* c) {
  __shared__ i128 sRed[4 * 8];
  const int set = blockIdx.x;
  const long long ntiles = merge_tiles(st->nnz);
  if (ntiles > ws.max_tiles) {
    if (threadIdx.x == 0) {
      set_error(c, BASS_ERR_WORKSPACE);
      for (int k = 0; k < 4; ++k) rho[4 * set + k] = NAN;
    }
    return;
  }
  i128 v[4] = {0, 0, 0, 0};
  for (long long t = threadIdx.x; t < ntiles; t += blockDim.x) {
    const Partial& p = ws.partials[(long long)set * ws.max_tiles + t];
    v[0] += p.s[0]; v[1] += p.s[1]; v[2] += p.s[2]; v[3] += p.s[3];
  }
  block_sum_i128<4>(v, sRed);
  if (threadIdx.x == 0) {
    double* r = rho + 4 * set;
    r[0] = fx_to(v[0]);
    r[1] = fx_to(v[1]);
    r[2] = fx_to(v[2]);
    r[3] = fx_to(v[3]);
  }
}

cudaError_t run_rdm_prepared(const bass_state* st, int nq, double* rho, bass_ctrl* ctrl, const WsView& ws,
                             cudaStream_t s, int c64) {
  OpArgs a{};
  a.c64 = c64;
  a.in = st;
  a.out = nullptr;
  a.ctrl = ctrl;
  a.ws = ws;
  a.q = 0;
  a.gb = 0;
  a.nsets = nq;
  KLAUNCH(S_PARTITION, s, k_partition<<<dim3(device().grid_small, nq), 256, 0, s>>>(a, K_RDM, 0));
  cudaError_t e = launch_tile<K_RDM, P_RDM>(a, 0, s, nullptr);
  if (e != cudaSuccess) return e;
  KLAUNCH(S_RDM_FINAL, s, k_rdm_final_bounded<<<nq, 256, 0, s>>>(st, rho, ws, ctrl));
  return cudaGetLastError();
}


// ---------------------------------------------------------------------------
// segmented launches: one op on each of many states per launch
// ---------------------------------------------------------------------------
// Group g of a grid of N blocks over S states starts at
// start(s) = s + (N - S) * wp[s] / W, W = wp[S]: every state gets at least
// one block and the rest are shared in proportion to the work weights.
__device__ __forceinline__ long long seg_start(const SegPlan* plan, int s, long long N) {
  const int S = plan->nseg;
  const long long W = plan->wp[S] > 0 ? plan->wp[S] : 1;
  return (long long)s + ((N - S) * plan->wp[s]) / W;
}

// Blocks of state s's group in a grid of N blocks.
__device__ __forceinline__ int seg_size(const SegPlan* plan, int s, long long N) {
  return (int)(seg_start(plan, s + 1, N) - seg_start(plan, s, N));
}

// This block's state (the last s with start(s) <= blockIdx.x) and group; the
// state's op is copied into *sa.  Called by the whole block.
__device__ Grp seg_enter(const OpArgs* ops, const SegPlan* plan, OpArgs* sa, int* seg_out) {
  __shared__ int sSeg, sBid, sN;
  if (threadIdx.x == 0) {
    const long long N = gridDim.x, b = blockIdx.x;
    int lo = 0, hi = plan->nseg - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (seg_start(plan, mid, N) <= b) lo = mid;
      else hi = mid - 1;
    }
    sSeg = lo;
    sBid = (int)(b - seg_start(plan, lo, N));
    sN = seg_size(plan, lo, N);
  }
  __syncthreads();
  constexpr int kWords = (int)(sizeof(OpArgs) / 8);
  static_assert(sizeof(OpArgs) % 8 == 0, "op words");
  const unsigned long long* src = reinterpret_cast<const unsigned long long*>(ops + sSeg);
  unsigned long long* dst = reinterpret_cast<unsigned long long*>(sa);
  for (int i = threadIdx.x; i < kWords; i += blockDim.x) dst[i] = src[i];
  __syncthreads();
  if (seg_out) *seg_out = sSeg;
  return Grp{sBid, sN};
}

// The block groups of an op: work weight of state s = its input entries plus
// one tile (times its qubits for an RDM).  One block.
__global__ void k_seg_plan(const OpArgs* ops, int nseg, int kind, SegPlan* plan) {
  __shared__ long long sW[kMaxSeg];
  for (int s = threadIdx.x; s < nseg; s += blockDim.x) {
    const long long n = ops[s].in->nnz;
    sW[s] = (n + kStep) * (kind == K_RDM ? (long long)ops[s].nsets : 1LL);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    long long run = 0;
    for (int s = 0; s < nseg; ++s) {
      plan->wp[s] = run;
      run += sW[s];
    }
    plan->wp[nseg] = run;
    plan->nseg = nseg;
    plan->kind = kind;
  }
}

__global__ void k_partition_seg(const OpArgs* ops, const SegPlan* plan, int kind, int zero) {
  __shared__ OpArgs sa;
  const Grp g = seg_enter(ops, plan, &sa, nullptr);
  if (kind == K_IDENT) {  // no merge: only the op's workspace region is cleared
    if (zero && blockIdx.y == 0) zero_op_region(sa, g);
    return;
  }
  if (kind == K_RDM && (int)blockIdx.y >= sa.nsets) return;  // qubits this state does not have
  partition_body(sa, kind, zero, blockIdx.y, g);
}

template <int KIND, int PASS, bool C64>
__global__ void __launch_bounds__(kThreads, 4) k_tile_seg(const OpArgs* ops, const SegPlan* plan) {
  __shared__ OpArgs sa;
  const Grp g = seg_enter(ops, plan, &sa, nullptr);
  tile_body<KIND, PASS, C64>(sa, g);
}

// nblk_hist: grid of the evaluation pass; this state's evaluation group wrote
// its per-CTA child counts to partials[0 .. its group size).
template <bool P2>
__global__ void __launch_bounds__(kSelThreads) k_select_seg(const OpArgs* ops, const SegPlan* plan, int ns, int kind,
                                                             int nblk_hist, int mode, int trace) {
  __shared__ OpArgs sa;
  int seg = 0;
  const Grp g = seg_enter(ops, plan, &sa, &seg);
  select_body<P2>(sa, g, ns, kind, seg_size(plan, seg, nblk_hist), mode, sa.j, trace);
}

template <bool C64>
__global__ void __launch_bounds__(256) k_compact_seg(const OpArgs* ops, const SegPlan* plan, int ns, int kind) {
  __shared__ OpArgs sa;
  const Grp g = seg_enter(ops, plan, &sa, nullptr);
  compact_body<C64>(sa, g, ns, kind);
}

// per state, the moments of each of its qubits (grid: qubit x state)
__global__ void k_rdm_final_seg(const OpArgs* ops) {
  __shared__ i128 sRed[4 * 8];
  const OpArgs& a = ops[blockIdx.y];
  const int set = blockIdx.x;
  if (set >= a.nsets) return;
  const long long ntiles = merge_tiles(a.in->nnz);
  if (ntiles > a.ws.max_tiles) {
    if (threadIdx.x == 0) set_error(a.ctrl, BASS_ERR_WORKSPACE);
    return;
  }
  i128 v[4] = {0, 0, 0, 0};
  for (long long t = threadIdx.x; t < ntiles; t += blockDim.x) {
    const Partial& p = a.ws.partials[(long long)set * a.ws.max_tiles + t];
    v[0] += p.s[0]; v[1] += p.s[1]; v[2] += p.s[2]; v[3] += p.s[3];
  }
  block_sum_i128<4>(v, sRed);
  if (threadIdx.x == 0) {
    double* r = a.rho + 4 * set;
    r[0] = fx_to(v[0]);
    r[1] = fx_to(v[1]);
    r[2] = fx_to(v[2]);
    r[3] = fx_to(v[3]);
  }
}


// Grid of a segmented kernel: every block of it that fits at once, and at
// least one block per state.
template <typename F>
static int seg_grid(F kern, int threads, size_t smem, int nseg) {
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, threads, smem) != cudaSuccess || occ < 1) occ = 1;
  const int g = device().sms * occ;
  return g > nseg ? g : nseg;
}

// The resident grid of the segmented selection on the current device (one
// block group per segment, so a launch takes at most this many segments).
template <bool P2>
static cudaError_t seg_select_grid(int* out) {
  static PerDevice cache;
  return per_device(cache, out, [](int* g) {
    const size_t ssmem = kSelSmem;
    cudaError_t e = cudaFuncSetAttribute(k_select_seg<P2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ssmem);
    if (e != cudaSuccess) return e;
    *g = seg_grid(k_select_seg<P2>, kSelThreads, ssmem, 1);
    if (*g > 1024) *g = 1024;
    return cudaSuccess;
  });
}

cudaError_t seg_max_segments(int* out) {
  int a = 0, b = 0;
  cudaError_t e = seg_select_grid<true>(&a);
  if (e == cudaSuccess) e = seg_select_grid<false>(&b);
  if (e != cudaSuccess) return e;
  *out = a < b ? a : b;
  return cudaSuccess;
}

template <int KIND, bool C64>
static cudaError_t merge_op_seg(const OpArgs* ops, int nseg, int fin_mode, int trace, SegPlan* plan,
                                cudaStream_t s) {
  KLAUNCH(S_SMALL, s, k_seg_plan<<<1, 1024, 0, s>>>(ops, nseg, KIND, plan));
  const int np = device().grid_small > nseg ? device().grid_small : nseg;
  KLAUNCH(S_PARTITION, s, k_partition_seg<<<dim3(np, 1), 256, 0, s>>>(ops, plan, KIND, 1));
  constexpr int PASS = KIND == K_PERM ? P_WRITE : P_HIST;
  const size_t smem = (size_t)kTilePad * (16 + 8 + 2 + (PASS == P_WRITE ? 3 : 0));
  static int nt = 0;
  if (nt == 0) {
    cudaError_t e = cudaFuncSetAttribute(k_tile_seg<KIND, PASS, C64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    nt = seg_grid(k_tile_seg<KIND, PASS, C64>, kThreads, smem, 1);
  }
  const int gt = nt > nseg ? nt : nseg;
  KLAUNCH(KIND * 5 + PASS, s, k_tile_seg<KIND, PASS, C64><<<gt, kThreads, smem, s>>>(ops, plan));
  if (KIND == K_PERM) return cudaGetLastError();
  constexpr int ns = slots_per_entry(KIND);
  const size_t ssmem = kSelSmem;
  cudaError_t e = cudaSuccess;
  if (fin_mode == 1) {
    int gs1 = 0;
    if ((e = seg_select_grid<true>(&gs1)) != cudaSuccess) return e;
    if (nseg > gs1) return cudaErrorInvalidValue;  // the groups' barriers need every block resident
    KLAUNCH(S_SELECT1, s, e = launch_coop(k_select_seg<true>, dim3(gs1), dim3(kSelThreads), ssmem, s, ops, plan, ns,
                                          (int)KIND, gt, fin_mode, trace));
  } else {
    int gs0 = 0;
    if ((e = seg_select_grid<false>(&gs0)) != cudaSuccess) return e;
    if (nseg > gs0) return cudaErrorInvalidValue;
    KLAUNCH(S_SELECT1, s, e = launch_coop(k_select_seg<false>, dim3(gs0), dim3(kSelThreads), ssmem, s, ops, plan, ns,
                                          (int)KIND, gt, fin_mode, trace));
  }
  if (e != cudaSuccess) return e;
  static PerDevice grid_seg;
  int gc = 0;
  if ((e = smem_grid(grid_seg, k_compact_seg<C64>, kCompactSmem, &gc)) != cudaSuccess) return e;
  if (gc < nseg) gc = nseg;
  KLAUNCH(KIND * 5 + P_WRITE, s, k_compact_seg<C64><<<gc, kThreads, kCompactSmem, s>>>(ops, plan, ns, (int)KIND));
  return cudaGetLastError();
}

template <int KIND>
static cudaError_t merge_op_seg_t(const OpArgs* ops, int nseg, int c64, int fin_mode, int trace, SegPlan* plan,
                                  cudaStream_t s) {
  return c64 ? merge_op_seg<KIND, true>(ops, nseg, fin_mode, trace, plan, s)
             : merge_op_seg<KIND, false>(ops, nseg, fin_mode, trace, plan, s);
}

cudaError_t run_merge_op_seg(int kind, const OpArgs* ops, int nseg, int c64, int fin_mode, int trace,
                             SegPlan* plan, cudaStream_t s) {
  if (nseg < 1 || nseg > kMaxSeg) return cudaErrorInvalidValue;
  switch (kind) {
    case K_GATE1: return merge_op_seg_t<K_GATE1>(ops, nseg, c64, fin_mode, trace, plan, s);
    case K_ROT1: return merge_op_seg_t<K_ROT1>(ops, nseg, c64, fin_mode, trace, plan, s);
    case K_GATE2: return merge_op_seg_t<K_GATE2>(ops, nseg, c64, fin_mode, trace, plan, s);
    case K_PERM: return merge_op_seg_t<K_PERM>(ops, nseg, c64, fin_mode, trace, plan, s);
    case K_IDENT: return merge_op_seg_t<K_IDENT>(ops, nseg, c64, fin_mode, trace, plan, s);
  }
  return cudaErrorInvalidValue;
}

template <bool C64>
static cudaError_t rdm_seg(const OpArgs* ops, int nseg, int max_nq, SegPlan* plan, cudaStream_t s) {
  KLAUNCH(S_SMALL, s, k_seg_plan<<<1, 1024, 0, s>>>(ops, nseg, K_RDM, plan));
  const int np = device().grid_small > nseg ? device().grid_small : nseg;
  KLAUNCH(S_PARTITION, s, k_partition_seg<<<dim3(np, max_nq), 256, 0, s>>>(ops, plan, K_RDM, 1));
  const size_t smem = (size_t)kTilePad * (16 + 8 + 2);
  static int nt = 0;
  if (nt == 0) {
    cudaError_t e = cudaFuncSetAttribute(k_tile_seg<K_RDM, P_RDM, C64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    nt = seg_grid(k_tile_seg<K_RDM, P_RDM, C64>, kThreads, smem, 1);
  }
  const int gt = nt > nseg ? nt : nseg;
  KLAUNCH(K_RDM * 5 + P_RDM, s, k_tile_seg<K_RDM, P_RDM, C64><<<gt, kThreads, smem, s>>>(ops, plan));
  KLAUNCH(S_RDM_FINAL, s, k_rdm_final_seg<<<dim3(max_nq, nseg), 256, 0, s>>>(ops));
  return cudaGetLastError();
}

cudaError_t run_rdm_seg(const OpArgs* ops, int nseg, int max_nq, int c64, SegPlan* plan, cudaStream_t s) {
  if (nseg < 1 || nseg > kMaxSeg || max_nq < 1 || max_nq > kMaxSets) return cudaErrorInvalidValue;
  return c64 ? rdm_seg<true>(ops, nseg, max_nq, plan, s) : rdm_seg<false>(ops, nseg, max_nq, plan, s);
}

}  // namespace bass
