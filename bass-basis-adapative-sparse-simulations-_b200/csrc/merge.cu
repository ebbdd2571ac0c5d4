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
//                 moments) and, depending on the pass, histograms the
//                 children's |a|^2, gathers top-k boundary candidates, or
//                 writes the surviving children in order (decoupled look-back);
//   k_select*     radix select of the top-k threshold (13-bit digits on the
//                 IEEE bits of |a|^2, then an exact (|a|^2 desc, key asc)
//                 ordering of the boundary candidates);
//   k_finalize    output descriptor (count, new bit order, pending
//                 renormalisation) and the gamma / truncation bookkeeping.
//
// The output is again sorted by its (new) physical key: children of a group
// are emitted in child-index order, groups in Z order.
#include <math.h>

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
  int8_t qat_out[64];
};

__device__ __forceinline__ void out_order(const bass_state* in, int kind, int t, int gb, int8_t* qat_out) {
  for (int p = 0; p < 64; ++p) qat_out[p] = in->qat[p];
  if (kind == K_GATE1 || kind == K_ROT1 || kind == K_GATE2 || kind == K_PERM) {
    int8_t qt = in->qat[t];
    for (int p = t; p > gb; --p) qat_out[p] = in->qat[p - 1];
    qat_out[gb] = qt;
  }
}

// ---------------------------------------------------------------------------
// partition
// ---------------------------------------------------------------------------
// record per boundary: P' (adjusted Z position), s, mid, e (block bounds), i, j
__global__ void k_partition(OpArgs a, int kind) {
  const int set = blockIdx.y;
  const bass_state* in = a.in;
  const long long n = in->nnz;
  const int q = (kind == K_RDM) ? set : a.q;
  const int t = in->pos[q];
  const int gb = a.gb;
  const int sh = gb + 1;
  const uint64_t* keys = in->keys;
  const long long ntiles = merge_tiles(n);
  long long* recs = a.ws.part + (long long)set * (a.ws.max_tiles + 1) * 6;
  const int lane = threadIdx.x & 31;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
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
      long long s = warp_first_false(0, P + 1, [&](long long i) { return keys[i] < lo_key; });
      long long mid = warp_first_false(s, n, [&](long long i) { return keys[i] < mid_key; });
      long long e = hi_ovf ? n : warp_first_false(P, n, [&](long long i) { return keys[i] < hi_key; });
      const long long d = P - s, len0 = mid - s, len1 = e - mid;
      long long lo = d - len1 > 0 ? d - len1 : 0;
      long long hi = d < len0 ? d : len0;
      long long i = warp_first_false(lo, hi, [&](long long m) {
        return zmove(keys[s + m], t, gb) < zmove(keys[mid + d - 1 - m], t, gb);
      });
      long long j = d - i;
      if (kind != K_PERM) {
        uint64_t z0 = (i < len0) ? zmove(keys[s + i], t, gb) : ~0ULL;
        uint64_t z1 = (j < len1) ? zmove(keys[mid + j], t, gb) : ~0ULL;
        uint64_t gid = (z0 < z1 ? z0 : z1) >> sh;
        int b0 = 0, b1 = 0;
        while (b0 < 2 && i - b0 - 1 >= 0 && (zmove(keys[s + i - b0 - 1], t, gb) >> sh) == gid) ++b0;
        while (b1 < 2 && j - b1 - 1 >= 0 && (zmove(keys[mid + j - b1 - 1], t, gb) >> sh) == gid) ++b1;
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
// Children of the group whose first Z-ordered entry is at merged position p
// (0 if p does not start a group).  Keys are the new physical keys.
template <int KIND>
__device__ __forceinline__ int group_children(int p, int E, const uint64_t* sZ, const double2* sA,
                                              const uint16_t* sM, int gb, const double2* G,
                                              int drop_zero, uint64_t* ck, double2* ca) {
  const uint64_t z = sZ[sM[p]];
  if (KIND == K_PERM || KIND == K_IDENT) {
    const double2 v = sA[sM[p]];
    if (KIND == K_IDENT && drop_zero && !cnz(v)) return 0;
    ck[0] = z;
    ca[0] = v;
    return 1;
  }
  const int sh = gb + 1;
  const uint64_t gid = z >> sh;
  if (p > 0 && (sZ[sM[p - 1]] >> sh) == gid) return 0;
  double2 av[4];
  int present = 0;
  for (int r = p; r < E; ++r) {
    const uint64_t zr = sZ[sM[r]];
    if ((zr >> sh) != gid) break;
    const int li = (int)(zr & ((1u << sh) - 1));
    av[li] = sA[sM[r]];
    present |= 1 << li;
  }
  int m = 0;
  if (KIND == K_GATE1 || KIND == K_GATE2) {
    const int nc = 1 << sh;
    for (int o = 0; o < nc; ++o) {
      double2 acc = make_double2(0.0, 0.0);
      bool have = false;
      for (int li = 0; li < nc; ++li) {
        if (!((present >> li) & 1)) continue;
        const double2 pr = cmul(G[o * nc + li], av[li]);
        if (!cnz(pr)) continue;
        acc = have ? cadd(acc, pr) : pr;
        have = true;
      }
      if (have) {
        ck[m] = (gid << sh) | (uint64_t)o;
        ca[m] = acc;
        ++m;
      }
    }
  } else if (KIND == K_ROT1) {
    const double2 a0 = (present & 1) ? av[0] : make_double2(0.0, 0.0);
    const double2 a1 = (present & 2) ? av[1] : make_double2(0.0, 0.0);
#pragma unroll
    for (int o = 0; o < 2; ++o) {
      const double2 c = cadd(cmul(G[o * 2], a0), cmul(G[o * 2 + 1], a1));
      if (hypot(c.x, c.y) > 1e-30) {
        ck[m] = (gid << 1) | (uint64_t)o;
        ca[m] = c;
        ++m;
      }
    }
  }
  return m;
}

__device__ __forceinline__ bool keep_child(uint64_t bits, uint64_t key, const SelState& S,
                                           const int8_t* qat) {
  if (!S.do_trunc) return true;
  if (bits > S.t_bits) return true;
  if (bits < S.t_bits) return false;
  return S.t_key == ~0ULL || true_key(key, qat, 64) <= S.t_key;
}

// ---------------------------------------------------------------------------
// the tile kernel
// ---------------------------------------------------------------------------
template <int KIND, int PASS>
__global__ void __launch_bounds__(kThreads) k_tile(OpArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  uint64_t* sZ = reinterpret_cast<uint64_t*>(smem);
  double2* sA = reinterpret_cast<double2*>(sZ + kTilePad);
  uint16_t* sIdx = reinterpret_cast<uint16_t*>(sA + kTilePad);
  uint16_t* sM = sIdx + kTilePad;
  unsigned int* sHist = reinterpret_cast<unsigned int*>(sM + kTilePad);
  __shared__ Hdr H;
  __shared__ SelState S;
  __shared__ long long sItem, sBase;
  __shared__ long long sSegLo[5], sSegOff[6];
  __shared__ int sWarp[32];
  __shared__ i128 sRed[4 * (kThreads / 32)];

  const int tid = threadIdx.x;
  if (tid == 0) S = *a.ws.sel;
  __syncthreads();
  if (PASS == P_HIST2 && S.stage != 1) return;
  if (PASS == P_GATHER && S.stage != 2) return;
  if (KIND == K_IDENT && a.guard && S.pad == 0) return;

  if (tid == 0) {
    const bass_state* in = a.in;
    H.keys = in->keys;
    H.amps = reinterpret_cast<const double2*>(in->amps);
    H.n = in->nnz;
    H.r0 = in->rscale[0];
    H.r1 = in->rscale[1];
    H.nq = in->nq;
    H.t = (KIND == K_IDENT || KIND == K_RDM) ? 0 : in->pos[a.q];
    H.ntiles = (KIND == K_IDENT) ? plain_tiles(H.n) : merge_tiles(H.n);
    out_order(in, KIND, H.t, a.gb, H.qat_out);
  }
  if (PASS == P_HIST || PASS == P_HIST2)
    for (int i = tid; i < kHistBins; i += kThreads) sHist[i] = 0;
  __syncthreads();

  const int gb = a.gb;
  const long long ntiles = H.ntiles;
  if (ntiles > a.ws.max_tiles) {  // the workspace is too small for this state
    if (blockIdx.x == 0 && tid == 0) set_error(a.ctrl, BASS_ERR_WORKSPACE);
    return;
  }
  const long long nitems = (KIND == K_RDM) ? ntiles * a.nsets : ntiles;
  i128 acc[4] = {0, 0, 0, 0};
  long long cnt = 0;
  const int base_e = tid * kPerThread;

  for (;;) {
    if (tid == 0) sItem = (long long)atomicAdd(&reinterpret_cast<unsigned long long*>(a.ws.counters)[a.counter], 1ULL);
    __syncthreads();
    const long long item = sItem;
    if (item >= nitems) break;
    const int set = (KIND == K_RDM) ? (int)(item / ntiles) : 0;
    const long long tile = (KIND == K_RDM) ? item % ntiles : item;
    const int t = (KIND == K_RDM) ? a.in->pos[a.q + set] : H.t;

    // ---- segments ---------------------------------------------------------
    if (tid == 0) {
      long long lo[5] = {0, 0, 0, 0, 0}, len[5] = {0, 0, 0, 0, 0};
      if (KIND == K_IDENT) {
        lo[0] = tile * kTile;
        len[0] = (H.n - lo[0] < kTile) ? H.n - lo[0] : kTile;
      } else {
        const long long* rc = a.ws.part + ((long long)set * (a.ws.max_tiles + 1) + tile) * 6;
        const long long* rn = rc + 6;
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
      if (o > kTile || bad) {  // inconsistent partition: skip the tile, report
        set_error(a.ctrl, BASS_ERR_ARG);
        for (int k = 0; k < 5; ++k) sSegOff[k] = 0;
        o = 0;
      }
      sSegOff[5] = o;
      if (a.prof) atomicAdd(reinterpret_cast<unsigned long long*>(&a.ctrl->prof_in[KIND * 5 + PASS]),
                            (unsigned long long)o);
    }
    __syncthreads();
    const int E = (int)sSegOff[5];

    // ---- load (Z keys, scaled amplitudes) ---------------------------------
    for (int e = tid; e < E; e += kThreads) {
      int k = 0;
      while (k < 4 && e >= sSegOff[k + 1]) ++k;
      const long long g = sSegLo[k] + (e - sSegOff[k]);
      const uint64_t y = H.keys[g];
      sZ[e] = (KIND == K_IDENT) ? y : zmove(y, t, gb);
      sA[e] = scale_load(H.amps[g], H.r0, H.r1);
    }
    __syncthreads();

    // ---- Z order: split by the target bit, merge ---------------------------
    if (KIND != K_IDENT) {
      int c0 = 0;
#pragma unroll
      for (int k = 0; k < kPerThread; ++k) {
        const int e = base_e + k;
        if (e < E && !((sZ[e] >> gb) & 1ULL)) ++c0;
      }
      int n0;
      const int ex0 = block_excl_scan(c0, sWarp, &n0);
      int w0 = ex0, w1 = (base_e < E ? base_e : E) - ex0;
#pragma unroll
      for (int k = 0; k < kPerThread; ++k) {
        const int e = base_e + k;
        if (e >= E) break;
        if (!((sZ[e] >> gb) & 1ULL)) sIdx[w0++] = (uint16_t)e;
        else sIdx[n0 + w1++] = (uint16_t)e;
      }
      __syncthreads();
      const int n1 = E - n0;
      const uint16_t* S0 = sIdx;
      const uint16_t* S1 = sIdx + n0;
      const int d = base_e < E ? base_e : E;
      int lo = d - n1 > 0 ? d - n1 : 0, hi = d < n0 ? d : n0;
      while (lo < hi) {
        const int m = (lo + hi) >> 1;
        if (sZ[S0[m]] < sZ[S1[d - 1 - m]]) lo = m + 1;
        else hi = m;
      }
      int i = lo, j = d - lo;
#pragma unroll
      for (int k = 0; k < kPerThread; ++k) {
        const int p = d + k;
        if (p >= E) break;
        const bool take0 = i < n0 && (j >= n1 || sZ[S0[i]] < sZ[S1[j]]);
        sM[p] = take0 ? S0[i++] : S1[j++];
      }
    } else {
      for (int e = tid; e < E; e += kThreads) sM[e] = (uint16_t)e;
    }
    __syncthreads();

    // ---- evaluate ------------------------------------------------------------
    const int pend = (base_e + kPerThread < E) ? base_e + kPerThread : E;
    if (PASS == P_RDM) {
      i128 v[4] = {0, 0, 0, 0};
      for (int p = base_e; p < pend; ++p) {
        const uint64_t z = sZ[sM[p]];
        const uint64_t gid = z >> 1;
        if (p > 0 && (sZ[sM[p - 1]] >> 1) == gid) continue;
        const double2 x0 = sA[sM[p]];
        if ((z & 1ULL) == 0) {
          v[0] += fx_from(prob(x0));
          if (p + 1 < E && (sZ[sM[p + 1]] >> 1) == gid) {
            const double2 x1 = sA[sM[p + 1]];
            v[1] += fx_from(prob(x1));
            const double2 c = cmul(x0, make_double2(x1.x, -x1.y));
            v[2] += fx_from(c.x);
            v[3] += fx_from(c.y);
          }
        } else {
          v[1] += fx_from(prob(x0));
        }
      }
      block_sum_i128<4>(v, sRed);
      if (tid == 0) {
        Partial* pt = a.ws.partials + (long long)set * a.ws.max_tiles + tile;
        pt->s[0] = v[0]; pt->s[1] = v[1]; pt->s[2] = v[2]; pt->s[3] = v[3];
      }
    } else if (PASS == P_WRITE) {
      uint64_t ck[4];
      double2 ca[4];
      int kc = 0;
      for (int p = base_e; p < pend; ++p) {
        const int m = group_children<KIND>(p, E, sZ, sA, sM, gb, a.G, a.drop_zero, ck, ca);
        for (int c = 0; c < m; ++c)
          if (keep_child((uint64_t)__double_as_longlong(prob(ca[c])), ck[c], S, H.qat_out)) ++kc;
      }
      int tile_total;
      const int ex = block_excl_scan(kc, sWarp, &tile_total);
      if (tid == 0) {
        const long long b = lookback(a.ws.status, tile, tile_total, a.ctrl);
        sBase = b;
        if (tile == ntiles - 1) a.ws.sel->n_written = b + tile_total;
        if (b + tile_total > a.out->cap) set_error(a.ctrl, BASS_ERR_CAPACITY);
        if (a.prof) atomicAdd(reinterpret_cast<unsigned long long*>(&a.ctrl->prof_out[KIND * 5 + PASS]),
                              (unsigned long long)tile_total);
      }
      __syncthreads();
      long long o = sBase + ex;
      if (sBase + tile_total <= a.out->cap) {
        uint64_t* ok = a.out->keys;
        double2* oa = reinterpret_cast<double2*>(a.out->amps);
        for (int p = base_e; p < pend; ++p) {
          const int m = group_children<KIND>(p, E, sZ, sA, sM, gb, a.G, a.drop_zero, ck, ca);
          for (int c = 0; c < m; ++c) {
            const double pv = prob(ca[c]);
            if (keep_child((uint64_t)__double_as_longlong(pv), ck[c], S, H.qat_out)) {
              ok[o] = ck[c];
              oa[o] = ca[c];
              ++o;
              acc[0] += fx_from(pv);
              ++cnt;
            }
          }
        }
      }
    } else {
      uint64_t ck[4];
      double2 ca[4];
      for (int p = base_e; p < pend; ++p) {
        const int m = group_children<KIND>(p, E, sZ, sA, sM, gb, a.G, a.drop_zero, ck, ca);
        for (int c = 0; c < m; ++c) {
          const double pv = prob(ca[c]);
          const uint64_t bits = (uint64_t)__double_as_longlong(pv);
          if (PASS == P_HIST) {
            atomicAdd(&sHist[bits >> 50], 1u);
            acc[0] += fx_from(pv);
            ++cnt;
          } else if (PASS == P_HIST2) {
            if ((bits >> 50) == S.prefix) atomicAdd(&sHist[(bits >> 37) & (kHistBins - 1)], 1u);
          } else if (PASS == P_GATHER) {
            if ((bits >> 37) == S.prefix) {
              const unsigned long long slot =
                  atomicAdd(reinterpret_cast<unsigned long long*>(&a.ws.sel->n_cand), 1ULL);
              if ((long long)slot < a.ws.max_n) {
                a.ws.cand_bits[slot] = bits;
                a.ws.cand_key[slot] = true_key(ck[c], H.qat_out, 64);
              } else {
                a.ws.sel->cand_overflow = 1;
              }
            }
          }
        }
      }
    }
    __syncthreads();
  }

  // ---- flush ---------------------------------------------------------------
  if (PASS == P_HIST || PASS == P_HIST2) {
    unsigned int* gh = (PASS == P_HIST) ? a.ws.hist1 : a.ws.hist2;
    for (int i = tid; i < kHistBins; i += kThreads)
      if (sHist[i]) atomicAdd(&gh[i], sHist[i]);
  }
  if (PASS == P_HIST || PASS == P_WRITE) {
    i128 v[2] = {acc[0], (i128)cnt};
    block_sum_i128<2>(v, sRed);
    if (tid == 0) {
      Partial* pt = a.ws.partials + blockIdx.x;
      pt->s[0] = v[0];
      pt->c[0] = (long long)v[1];
    }
  }
}

// ---------------------------------------------------------------------------
// selection
// ---------------------------------------------------------------------------
// Block of 1024 threads.  Returns the bin b with count(bins > b) < k <=
// count(bins >= b); *c_gt = count(bins > b).  Needs 1 <= k <= total.
__device__ int find_bin(const unsigned int* hist, long long k, long long* c_gt, long long* sS) {
  __shared__ int sRes;
  __shared__ long long sAbove;
  const int t = threadIdx.x;
  long long s = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) s += hist[8 * t + i];
  sS[t] = s;
  __syncthreads();
  if (t < 32) {
    long long ls = 0;
    for (int i = 0; i < 32; ++i) ls += sS[32 * t + i];
    long long suf = ls;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      long long v = __shfl_down_sync(0xffffffffu, suf, off);
      if (t + off < 32) suf += v;
    }
    const unsigned m = __ballot_sync(0xffffffffu, suf >= k);
    const int L = m ? 31 - __clz(m) : 0;
    if (t == L) {
      long long above = suf - ls;
      int tt = 32 * L + 31;
      for (; tt > 32 * L; --tt) {
        if (above + sS[tt] >= k) break;
        above += sS[tt];
      }
      int b = 8 * tt + 7;
      for (; b > 8 * tt; --b) {
        const long long h = hist[b];
        if (above + h >= k) break;
        above += h;
      }
      sRes = b;
      sAbove = above;
    }
  }
  __syncthreads();
  *c_gt = sAbove;
  return sRes;
}

__global__ void __launch_bounds__(1024) k_select1(OpArgs a, int nblk) {
  __shared__ long long sS[1024];
  __shared__ i128 sRed[2 * 32];
  SelState* sel = a.ws.sel;
  i128 v[2] = {0, 0};
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
    v[0] += a.ws.partials[b].s[0];
    v[1] += (i128)a.ws.partials[b].c[0];
  }
  block_sum_i128<2>(v, sRed);
  __shared__ int sGo;
  if (threadIdx.x == 0) {
    const long long n_out = (long long)v[1];
    sel->n_out = n_out;
    sel->total = fx_to(v[0]);
    sel->k_keep = a.k_keep;
    sGo = 0;
    if (a.k_cond < 0 || n_out <= a.k_cond || a.k_keep >= n_out) {
      sel->do_trunc = 0;
      sel->stage = 0;
    } else if (a.k_keep <= 0) {
      sel->do_trunc = 1;
      sel->stage = 3;
      sel->t_bits = ~0ULL;
      sel->t_key = 0;
    } else {
      sel->do_trunc = 1;
      sGo = 1;
    }
  }
  __syncthreads();
  if (!sGo) return;
  long long c_gt;
  const int b1 = find_bin(a.ws.hist1, a.k_keep, &c_gt, sS);
  if (threadIdx.x == 0) {
    const long long need = a.k_keep - c_gt;
    if ((long long)a.ws.hist1[b1] == need) {
      sel->stage = 3;
      sel->t_bits = (unsigned long long)b1 << 50;
      sel->t_key = ~0ULL;
    } else {
      sel->stage = 1;
      sel->prefix = (unsigned long long)b1;
      sel->need = need;
    }
  }
}

__global__ void __launch_bounds__(1024) k_select2(OpArgs a) {
  __shared__ long long sS[1024];
  SelState* sel = a.ws.sel;
  if (sel->stage != 1) return;
  long long c_gt;
  const long long need = sel->need;
  const int b2 = find_bin(a.ws.hist2, need, &c_gt, sS);
  if (threadIdx.x == 0) {
    const long long need2 = need - c_gt;
    const unsigned long long pre = (sel->prefix << 13) | (unsigned long long)b2;
    if ((long long)a.ws.hist2[b2] == need2) {
      sel->stage = 3;
      sel->t_bits = pre << 37;
      sel->t_key = ~0ULL;
    } else {
      sel->stage = 2;
      sel->prefix = pre;
      sel->need = need2;
    }
  }
}

// better(a, b): a ranks strictly above b
__device__ __forceinline__ bool better(unsigned long long ab, unsigned long long ak,
                                       unsigned long long bb, unsigned long long bk) {
  return ab > bb || (ab == bb && ak < bk);
}

__global__ void __launch_bounds__(1024) k_select_exact(OpArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned long long* sb = reinterpret_cast<unsigned long long*>(smem);
  unsigned long long* sk = sb + kCandSmem;
  SelState* sel = a.ws.sel;
  if (sel->stage != 2) return;
  long long m = sel->n_cand;
  if (sel->cand_overflow || m > a.ws.max_n) {
    if (threadIdx.x == 0) set_error(a.ctrl, BASS_ERR_WORKSPACE);
    m = a.ws.max_n;
  }
  const long long need = sel->need;
  const int tid = threadIdx.x;
  if (m <= kCandSmem) {
    int P = 1;
    while (P < m) P <<= 1;
    for (int i = tid; i < P; i += blockDim.x) {
      if (i < m) { sb[i] = a.ws.cand_bits[i]; sk[i] = a.ws.cand_key[i]; }
      else { sb[i] = 0; sk[i] = ~0ULL; }
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
              unsigned long long tb = sb[i], tk = sk[i];
              sb[i] = sb[jx]; sk[i] = sk[jx]; sb[jx] = tb; sk[jx] = tk;
            }
          }
        }
        __syncthreads();
      }
    }
    if (tid == 0) {
      const long long r = (need >= 1 && need <= m) ? need - 1 : 0;
      sel->t_bits = sb[r];
      sel->t_key = sk[r];
      sel->stage = 3;
    }
    return;
  }
  // many candidates (ties): radix select on (low 37 bits of |a|^2, ~key), 8-bit digits
  unsigned int* h = reinterpret_cast<unsigned int*>(smem);
  __shared__ u128 sPrefix;
  __shared__ long long sNeed;
  if (tid == 0) { sPrefix = 0; sNeed = need; }
  __syncthreads();
  const unsigned long long m37 = (1ULL << 37) - 1;
  for (int shift = 96; shift >= 0; shift -= 8) {
    for (int i = tid; i < 256; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const u128 pre = sPrefix;
    for (long long i = tid; i < m; i += blockDim.x) {
      const u128 comp = ((u128)(a.ws.cand_bits[i] & m37) << 64) | (u128)(~a.ws.cand_key[i]);
      if ((comp >> (shift + 8)) == pre) atomicAdd(&h[(unsigned)(comp >> shift) & 255u], 1u);
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
      sPrefix = (pre << 8) | (u128)b;
    }
    __syncthreads();
  }
  if (tid == 0) {
    const u128 comp = sPrefix;
    sel->t_bits = (sel->prefix << 37) | (uint64_t)((comp >> 64) & m37);
    sel->t_key = ~(uint64_t)comp;
    sel->stage = 3;
  }
}

// ---------------------------------------------------------------------------
// finalisation
// ---------------------------------------------------------------------------
// mode 0: plain op; mode 1: basis-rotation step (always renormalises, keeps
// the retained mass in sel->kept for the decision)
__global__ void k_finalize(OpArgs a, bass_trunc tr, int mode, int kind, int nblk) {
  __shared__ i128 sRed[8];
  SelState* sel = a.ws.sel;
  i128 v[1] = {0};
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) v[0] += a.ws.partials[b].s[0];
  block_sum_i128<1>(v, sRed);
  if (threadIdx.x != 0) return;
  const bass_state* in = a.in;
  bass_state* out = a.out;
  bass_ctrl* c = a.ctrl;
  const double kept = fx_to(v[0]);
  const long long n_in = in->nnz;
  long long nw = sel->n_written;
  if (nw > out->cap) {  // the write pass skipped the tiles that did not fit
    set_error(c, BASS_ERR_CAPACITY);
    nw = 0;
  }
  const int t = (kind == K_IDENT) ? 0 : in->pos[a.q];
  int8_t qat[64];
  out_order(in, kind, t, a.gb, qat);
  for (int p = 0; p < 64; ++p) {
    out->qat[p] = qat[p];
    out->pos[qat[p]] = (int8_t)p;
  }
  out->nq = in->nq;
  out->nnz = nw;
  out->rscale[0] = 1.0;
  out->rscale[1] = 1.0;
  sel->kept = kept;
  if (kind == K_PERM) return;  // first pass of a 2-qubit gate: no bookkeeping
  c->amp_updates += n_in;
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

__global__ void k_rdm_final(const bass_state* st, double* rho, WsView ws, int first) {
  __shared__ i128 sRed[4 * 8];
  const int set = blockIdx.x;
  const long long n = st->nnz;
  const long long ntiles = merge_tiles(n);
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
template <int KIND, int PASS>
static cudaError_t launch_tile(OpArgs a, int counter, cudaStream_t s, int* grid_out) {
  const size_t smem = (size_t)kTilePad * 28 + ((PASS == P_HIST || PASS == P_HIST2) ? kHistBins * 4 : 0);
  static int grid = 0;
  if (grid == 0) {
    cudaError_t e = cudaFuncSetAttribute(k_tile<KIND, PASS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int occ = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_tile<KIND, PASS>, kThreads, smem);
    if (e != cudaSuccess) return e;
    grid = device().sms * (occ > 0 ? occ : 1);
    if (grid > 1024) grid = 1024;
  }
  a.counter = counter;
  a.prof = prof_on() ? 1 : 0;
  KLAUNCH(KIND * 5 + PASS, s, k_tile<KIND, PASS><<<grid, kThreads, smem, s>>>(a));
  if (grid_out) *grid_out = grid;
  return cudaGetLastError();
}

cudaError_t zero_small(const WsView& ws, cudaStream_t s) {
  // counters, hist1, hist2, sel and the look-back status words are contiguous
  const size_t bytes = (size_t)((char*)(ws.status + ws.max_tiles) - (char*)ws.counters);
  return cudaMemsetAsync(ws.counters, 0, bytes, s);
}

template <int KIND>
static cudaError_t merge_op(OpArgs a, const bass_trunc& tr, int fin_mode, cudaStream_t s) {
  cudaError_t e = zero_small(a.ws, s);
  if (e != cudaSuccess) return e;
  a.k_cond = tr.k_cond;
  a.k_keep = tr.k_keep;
  a.nsets = 1;
  if constexpr (KIND != K_IDENT) {
    KLAUNCH(S_PARTITION, s, k_partition<<<dim3(device().grid_small, 1), 256, 0, s>>>(a, KIND));
  }
  if constexpr (KIND != K_PERM) {
    int gh = 0;
    if ((e = launch_tile<KIND, P_HIST>(a, 0, s, &gh)) != cudaSuccess) return e;
    KLAUNCH(S_SELECT1, s, k_select1<<<1, 1024, 0, s>>>(a, gh));
    if ((e = launch_tile<KIND, P_HIST2>(a, 1, s, nullptr)) != cudaSuccess) return e;
    KLAUNCH(S_SELECT2, s, k_select2<<<1, 1024, 0, s>>>(a));
    if ((e = launch_tile<KIND, P_GATHER>(a, 2, s, nullptr)) != cudaSuccess) return e;
    static bool attr = false;
    if (!attr) {
      cudaFuncSetAttribute(k_select_exact, cudaFuncAttributeMaxDynamicSharedMemorySize, kCandSmem * 16);
      attr = true;
    }
    KLAUNCH(S_SELECT_EXACT, s, k_select_exact<<<1, 1024, kCandSmem * 16, s>>>(a));
  }
  int gw = 0;
  if ((e = launch_tile<KIND, P_WRITE>(a, 3, s, &gw)) != cudaSuccess) return e;
  KLAUNCH(S_FINALIZE, s, k_finalize<<<1, 256, 0, s>>>(a, tr, fin_mode, KIND, gw));
  return cudaGetLastError();
}

cudaError_t run_merge_op(int kind, OpArgs a, const bass_trunc& tr, int finalize_mode, int j,
                         cudaStream_t s) {
  (void)j;
  switch (kind) {
    case K_GATE1: return merge_op<K_GATE1>(a, tr, finalize_mode, s);
    case K_ROT1: return merge_op<K_ROT1>(a, tr, finalize_mode, s);
    case K_GATE2: return merge_op<K_GATE2>(a, tr, finalize_mode, s);
    case K_PERM: return merge_op<K_PERM>(a, tr, finalize_mode, s);
    case K_IDENT: return merge_op<K_IDENT>(a, tr, finalize_mode, s);
  }
  return cudaErrorInvalidValue;
}

// write pass only (keep everything the drop rule keeps); used by the guarded
// compaction after a 1-qubit diagonal gate.  The caller zeroed the small region.
cudaError_t run_ident_write(OpArgs a, cudaStream_t s) {
  return launch_tile<K_IDENT, P_WRITE>(a, 3, s, nullptr);
}

cudaError_t run_rdm(const bass_state* st, int nq, double* rho, bass_ctrl* ctrl, const WsView& ws,
                    cudaStream_t s) {
  cudaError_t e = zero_small(ws, s);
  if (e != cudaSuccess) return e;
  OpArgs a{};
  a.in = st;
  a.out = nullptr;
  a.ctrl = ctrl;
  a.ws = ws;
  a.q = 0;
  a.gb = 0;
  a.nsets = nq;
  KLAUNCH(S_PARTITION, s, k_partition<<<dim3(device().grid_small, nq), 256, 0, s>>>(a, K_RDM));
  if ((e = launch_tile<K_RDM, P_RDM>(a, 0, s, nullptr)) != cudaSuccess) return e;
  KLAUNCH(S_RDM_FINAL, s, k_rdm_final<<<nq, 256, 0, s>>>(st, rho, ws, 0));
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
                             cudaStream_t s) {
  OpArgs a{};
  a.in = st;
  a.out = nullptr;
  a.ctrl = ctrl;
  a.ws = ws;
  a.q = 0;
  a.gb = 0;
  a.nsets = nq;
  KLAUNCH(S_PARTITION, s, k_partition<<<dim3(device().grid_small, nq), 256, 0, s>>>(a, K_RDM));
  cudaError_t e = launch_tile<K_RDM, P_RDM>(a, 0, s, nullptr);
  if (e != cudaSuccess) return e;
  KLAUNCH(S_RDM_FINAL, s, k_rdm_final_bounded<<<nq, 256, 0, s>>>(st, rho, ws, ctrl));
  return cudaGetLastError();
}

}  // namespace bass
