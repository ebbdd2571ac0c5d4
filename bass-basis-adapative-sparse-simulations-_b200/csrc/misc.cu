// misc.cu -- streaming kernels of libbass_b200: reductions, fingerprints,
// diagonal gates, state set-up / import / export, the LSD radix sort and the
// merge of sorted duplicates, gathers, and the basis-rotation decision.
#include <math.h>

#include "internal.h"

namespace bass {

enum RedMode { R_NORM2 = 0, R_P2 = 1 };

// ---------------------------------------------------------------------------
// reductions over a state (exact): per-CTA partials in ws.red
// ---------------------------------------------------------------------------
template <int MODE, bool C64>
__device__ __forceinline__ void reduce_body(const bass_state* st, const WsView& ws, int bid, int nblk) {
  __shared__ i128 sRed[8];
  const long long n = st->nnz;
  const double r0 = st->rscale[0], r1 = st->rscale[1];
  constexpr int c64 = C64;
  const double* amps = st->amps;
  i128 v[1] = {0};
  // eight entries per thread and round, summed exactly in the split
  // accumulators (fx_acc96) and joined once per round
  const long long stride = (long long)nblk * blockDim.x;
  for (long long i0 = (long long)bid * blockDim.x + threadIdx.x; i0 < n; i0 += 8 * stride) {
    double2 x[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const long long i = i0 + u * stride;
      x[u] = i < n ? amp_raw(amps, i, c64) : make_double2(0.0, 0.0);
    }
    double h = 0.0, l = 0.0;
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const double p = prob(amp_scale(x[u], c64, r0, r1));
      fx_acc96(MODE == R_NORM2 ? p : __dmul_rn(p, p), h, l, v[0]);
    }
    v[0] += fx_join96s(h, l);
  }
  block_sum_i128<1>(v, sRed);
  if (threadIdx.x == 0) ws.red[bid] = v[0];
}

template <int MODE, bool C64>
__global__ void __launch_bounds__(256) k_reduce_state(const bass_state* st, WsView ws) {
  reduce_body<MODE, C64>(st, ws, blockIdx.x, gridDim.x);
}

// segmented: state blockIdx.y of the ops, gridDim.x blocks each
template <int MODE, bool C64>
__global__ void __launch_bounds__(256) k_reduce_state_seg(const OpArgs* ops) {
  const OpArgs& a = ops[blockIdx.y];
  reduce_body<MODE, C64>(a.in, a.ws, blockIdx.x, gridDim.x);
}

__device__ __forceinline__ double reduce_red(const WsView& ws, int nblk, i128* sRed) {
  i128 v[1] = {0};
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) v[0] += ws.red[b];
  block_sum_i128<1>(v, sRed);
  return fx_to(v[0]);  // valid in thread 0
}

// dest = reduced value (mode NORM2: sum |a|^2)
__global__ void k_red_store(WsView ws, int nblk, double* dest) {
  __shared__ i128 sRed[8];
  const double s = reduce_red(ws, nblk, sRed);
  if (threadIdx.x == 0) *dest = s;
}

// bass_simulator.py:574-578 _pr
__device__ __forceinline__ void pr_final_body(const bass_state* st, const WsView& ws, int nblk, bass_ctrl* c) {
  __shared__ i128 sRed[8];
  const double S = reduce_red(ws, nblk, sRed);
  if (threadIdx.x == 0) {
    const double pr = (st->nnz == 0) ? INFINITY : (S > 1e-60 ? 1.0 / S : INFINITY);
    c->pr_last = pr;
    c->pr_cur = pr;
  }
}
__global__ void k_pr_final(const bass_state* st, WsView ws, int nblk, bass_ctrl* c) { pr_final_body(st, ws, nblk, c); }
__global__ void k_pr_final_seg(const OpArgs* ops, int nblk) {
  const OpArgs& a = ops[blockIdx.x];
  pr_final_body(a.in, a.ws, nblk, a.ctrl);
}

// bass_simulator.py:551-554 _renorm: norm = sqrt(sum |a|^2); if norm > 1e-30 the
// amplitudes become a * (1/norm).  The factor goes to a free rscale slot; if
// both are taken the array is rewritten first (k_materialize).
__device__ __forceinline__ void renorm_apply_body(bass_state* st, const WsView& ws, int nblk) {
  __shared__ i128 sRed[8];
  const double S = reduce_red(ws, nblk, sRed);
  if (threadIdx.x != 0) return;
  const double nrm = sqrt(S);
  ws.sel->pad = 0;
  if (!(nrm > 1e-30)) return;
  const double r = 1.0 / nrm;
  if (st->rscale[0] == 1.0 && st->rscale[1] == 1.0) st->rscale[0] = r;
  else if (st->rscale[1] == 1.0) st->rscale[1] = r;
  else {
    ws.sel->pad = 3;
    ws.sel->kept = r;
  }
}
__global__ void k_renorm_apply(bass_state* st, WsView ws, int nblk) { renorm_apply_body(st, ws, nblk); }
__global__ void k_renorm_apply_seg(const OpArgs* ops, int nblk) {
  const OpArgs& a = ops[blockIdx.x];
  renorm_apply_body(const_cast<bass_state*>(a.in), a.ws, nblk);
}

__device__ __forceinline__ void materialize_body(bass_state* st, const WsView& ws, bass_ctrl* c, int bid, int nblk) {
  if (ws.sel->pad != 3) return;
  const long long n = st->nnz;
  const double r0 = st->rscale[0], r1 = st->rscale[1];
  const int c64 = st->amp_type == BASS_AMP_C64;
  for (long long i = (long long)bid * blockDim.x + threadIdx.x; i < n; i += (long long)nblk * blockDim.x)
    amp_put(st->amps, i, amp_get(st->amps, i, c64, r0, r1), c64);
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned done = atomicAdd(&c->sync_counter, 1u);
    if (done == (unsigned)nblk - 1) {
      st->rscale[0] = ws.sel->kept;
      st->rscale[1] = 1.0;
      c->sync_counter = 0;
    }
  }
}
__global__ void k_materialize(bass_state* st, WsView ws, bass_ctrl* c) {
  materialize_body(st, ws, c, blockIdx.x, gridDim.x);
}
__global__ void k_materialize_seg(const OpArgs* ops) {
  const OpArgs& a = ops[blockIdx.y];
  materialize_body(const_cast<bass_state*>(a.in), a.ws, a.ctrl, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------------------
// fingerprints (order independent: wrapping sums, xors, counts)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_fingerprint(const bass_state* st, double pmin, WsView ws) {
  __shared__ int8_t qat[64];
  if (threadIdx.x < 64) qat[threadIdx.x] = st->qat[threadIdx.x];
  __syncthreads();
  const long long n = st->nnz;
  const double r0 = st->rscale[0], r1 = st->rscale[1];
  const int c64 = st->amp_type == BASS_AMP_C64;
  unsigned long long c = 0, s = 0, x = 0, c2 = 0, s2 = 0, x2 = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const uint64_t tk = true_key(st->keys[i], qat, 64);
    const uint64_t f1 = fmix64(tk), f2 = fmix64(tk ^ kFpSalt);
    ++c; s += f1; x ^= f2;
    if (prob(amp_get(st->amps, i, c64, r0, r1)) > pmin) { ++c2; s2 += f1; x2 ^= f2; }
  }
  for (int off = 16; off > 0; off >>= 1) {
    c += __shfl_down_sync(0xffffffffu, c, off);
    s += __shfl_down_sync(0xffffffffu, s, off);
    x ^= __shfl_down_sync(0xffffffffu, x, off);
    c2 += __shfl_down_sync(0xffffffffu, c2, off);
    s2 += __shfl_down_sync(0xffffffffu, s2, off);
    x2 ^= __shfl_down_sync(0xffffffffu, x2, off);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&ws.fp[0], c); atomicAdd(&ws.fp[1], s); atomicXor(&ws.fp[2], x);
    atomicAdd(&ws.fp[3], c2); atomicAdd(&ws.fp[4], s2); atomicXor(&ws.fp[5], x2);
  }
}

// copy the fingerprint out and/or append a renorm event to the trace
__global__ void k_fp_out(WsView ws, uint64_t* out6, bass_ctrl* c, int append, int only_if_trunc) {
  if (out6)
    for (int k = 0; k < 6; ++k) out6[k] = ws.fp[k];
  if (!append || !c->trace) return;
  if (only_if_trunc && !c->last_truncated) return;
  const long long i = c->trace_len;
  if (i >= c->trace_cap) { set_error(c, BASS_ERR_CAPACITY); return; }
  uint64_t* e = c->trace + i * BASS_TRACE_WORDS;
  e[0] = 0; e[1] = ws.fp[0]; e[2] = ws.fp[1]; e[3] = ws.fp[2];
  e[4] = ws.fp[3]; e[5] = ws.fp[4]; e[6] = ws.fp[5];
  c->trace_len = i + 1;
}

// ---------------------------------------------------------------------------
// diagonal gates
// ---------------------------------------------------------------------------
// sparse_state.py:178-190: a *= diag[(b_q1 << 1) | b_q2], in place
template <bool C64>
__device__ __forceinline__ void phase2q_body(bass_state* st, double2 d0, double2 d1, double2 d2, double2 d3, int q1,
                                             int q2, bass_ctrl* c, int bid, int nblk) {
  const long long n = st->nnz;
  const int t1 = st->pos[q1], t2 = st->pos[q2];
  const double r0 = st->rscale[0], r1 = st->rscale[1];
  constexpr int c64 = C64;
  double* amps = st->amps;
  const uint64_t* keys = st->keys;
  for (long long i = (long long)bid * blockDim.x + threadIdx.x; i < n; i += (long long)nblk * blockDim.x) {
    const uint64_t y = keys[i];
    const int idx = (int)((((y >> t1) & 1ULL) << 1) | ((y >> t2) & 1ULL));
    const double2 d = idx == 0 ? d0 : idx == 1 ? d1 : idx == 2 ? d2 : d3;
    const double2 v = amp_get(amps, i, c64, r0, r1);
    amp_put(amps, i, c64 ? cmul_c64(v, d) : cmul(v, d), c64);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned done = atomicAdd(&c->sync_counter, 1u);
    if (done == (unsigned)nblk - 1) {
      st->rscale[0] = 1.0;
      st->rscale[1] = 1.0;
      c->amp_updates += n;
      c->n_ops += 1;
      c->prof_in[S_PHASE2Q] += n;
      c->prof_out[S_PHASE2Q] += n;
      c->sync_counter = 0;
    }
  }
}

template <bool C64>
__global__ void k_phase2q(bass_state* st, double2 d0, double2 d1, double2 d2, double2 d3, int q1, int q2,
                          bass_ctrl* c) {
  phase2q_body<C64>(st, d0, d1, d2, d3, q1, q2, c, blockIdx.x, gridDim.x);
}

// segmented: state blockIdx.y, diagonal G[0..3], qubits (q, j)
template <bool C64>
__global__ void k_phase2q_seg(const OpArgs* ops) {
  const OpArgs& a = ops[blockIdx.y];
  phase2q_body<C64>(const_cast<bass_state*>(a.in), a.G[0], a.G[1], a.G[2], a.G[3], a.q, a.j, a.ctrl, blockIdx.x,
                    gridDim.x);
}

// 1-qubit diagonal gate: a = g_bb * a; children that are exactly zero are
// dropped by the reference's kernel, so a zero result raises the compaction flag
template <bool C64>
__global__ void k_phase1q(bass_state* st, double2 g0, double2 g1, int q, bass_ctrl* c, WsView ws) {
  const long long n = st->nnz;
  const int t = st->pos[q];
  const double r0 = st->rscale[0], r1 = st->rscale[1];
  constexpr int c64 = C64;
  double* amps = st->amps;
  const uint64_t* keys = st->keys;
  bool zero = false;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double2 g = ((keys[i] >> t) & 1ULL) ? g1 : g0;
    const double2 a = amp_get(amps, i, c64, r0, r1);
    const double2 v = c64 ? cmul_c64(g, a) : cmul(g, a);
    amp_put(amps, i, v, c64);
    zero |= !cnz(v);
  }
  if (__any_sync(0xffffffffu, zero) && (threadIdx.x & 31) == 0) ws.sel->pad = 1;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned done = atomicAdd(&c->sync_counter, 1u);
    if (done == gridDim.x - 1) {
      st->rscale[0] = 1.0;
      st->rscale[1] = 1.0;
      c->amp_updates += n;
      c->n_ops += 1;
      c->prof_in[S_PHASE1Q] += n;
      c->prof_out[S_PHASE1Q] += n;
      c->sync_counter = 0;
    }
  }
}

__global__ void k_phase1q_fin(bass_state* st, bass_state* tmp, WsView ws) {
  if (ws.sel->pad != 1) return;
  bass_state t = *tmp;
  t.nnz = ws.sel->n_written;
  t.rscale[0] = 1.0;
  t.rscale[1] = 1.0;
  t.nq = st->nq;
  for (int p = 0; p < 64; ++p) { t.pos[p] = st->pos[p]; t.qat[p] = st->qat[p]; }
  *tmp = *st;
  *st = t;
}

// ---------------------------------------------------------------------------
// state set-up, copies, gathers
// ---------------------------------------------------------------------------
__global__ void k_state_init(bass_state* st, uint64_t* keys, double* amps, long long cap, int nq,
                             uint64_t init_key, int amp_type) {
  st->keys = keys;
  st->amps = amps;
  st->nnz = 1;
  st->cap = cap;
  st->rscale[0] = 1.0;
  st->rscale[1] = 1.0;
  st->nq = nq;
  st->amp_type = amp_type;
  for (int p = 0; p < 64; ++p) { st->pos[p] = (int8_t)p; st->qat[p] = (int8_t)p; }
  keys[0] = init_key;
  amp_put(amps, 0, make_double2(1.0, 0.0), amp_type == BASS_AMP_C64);
}

__global__ void k_state_adopt(bass_state* st, uint64_t* keys, double* amps, long long cap, int nq,
                              long long n, int amp_type) {
  st->keys = keys;
  st->amps = amps;
  st->nnz = n;
  st->cap = cap;
  st->rscale[0] = 1.0;
  st->rscale[1] = 1.0;
  st->nq = nq;
  st->amp_type = amp_type;
  for (int p = 0; p < 64; ++p) { st->pos[p] = (int8_t)p; st->qat[p] = (int8_t)p; }
}

__global__ void k_copy_desc(bass_state* dst, const bass_state* src) { *dst = *src; }

// deep copy of entries; dst keeps its own buffers
__global__ void k_clone(bass_state* dst, const bass_state* src, bass_ctrl* c) {
  const long long n = src->nnz;
  if (n > dst->cap || dst->amp_type != src->amp_type) {
    if (blockIdx.x == 0 && threadIdx.x == 0) set_error(c, n > dst->cap ? BASS_ERR_CAPACITY : BASS_ERR_ARG);
    return;
  }
  const int c64 = src->amp_type == BASS_AMP_C64;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    dst->keys[i] = src->keys[i];
    amp_put(dst->amps, i, amp_raw(src->amps, i, c64), c64);
  }
}
__global__ void k_clone_desc(bass_state* dst, const bass_state* src) {
  if (src->nnz > dst->cap || dst->amp_type != src->amp_type) return;
  dst->nnz = src->nnz;
  dst->rscale[0] = src->rscale[0];
  dst->rscale[1] = src->rscale[1];
  dst->nq = src->nq;
  for (int p = 0; p < 64; ++p) { dst->pos[p] = src->pos[p]; dst->qat[p] = src->qat[p]; }
}

__global__ void k_gather(const bass_state* in, bass_state* out, const int64_t* idx, long long n,
                         bass_ctrl* c) {
  if (n > out->cap) {
    if (blockIdx.x == 0 && threadIdx.x == 0) set_error(c, BASS_ERR_CAPACITY);
    return;
  }
  const long long nin = in->nnz;
  const int c64 = in->amp_type == BASS_AMP_C64;
  if (out->amp_type != in->amp_type) {
    if (blockIdx.x == 0 && threadIdx.x == 0) set_error(c, BASS_ERR_ARG);
    return;
  }
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long k = idx[i];
    if (k < 0 || k >= nin) { set_error(c, BASS_ERR_ARG); continue; }
    out->keys[i] = in->keys[k];
    amp_put(out->amps, i, amp_raw(in->amps, k, c64), c64);
  }
}
__global__ void k_gather_desc(const bass_state* in, bass_state* out, long long n) {
  if (n > out->cap || out->amp_type != in->amp_type) return;
  out->nnz = n;
  out->rscale[0] = in->rscale[0];
  out->rscale[1] = in->rscale[1];
  out->nq = in->nq;
  for (int p = 0; p < 64; ++p) { out->pos[p] = in->pos[p]; out->qat[p] = in->qat[p]; }
}

// export: true keys and scaled amplitudes (sorted afterwards)
// (output amplitudes of the state's type; amp_type is what the caller expects)
__global__ void k_export(const bass_state* st, uint64_t* ok, double* oa, long long max_n, int amp_type,
                         bass_ctrl* c) {
  __shared__ int8_t qat[64];
  if (threadIdx.x < 64) qat[threadIdx.x] = st->qat[threadIdx.x];
  __syncthreads();
  const long long n = st->nnz;
  if (n > max_n) return;
  if (st->amp_type != amp_type) {
    if (blockIdx.x == 0 && threadIdx.x == 0) set_error(c, BASS_ERR_ARG);
    return;
  }
  const double r0 = st->rscale[0], r1 = st->rscale[1];
  const int c64 = amp_type == BASS_AMP_C64;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    ok[i] = true_key(st->keys[i], qat, 64);
    amp_put(oa, i, amp_get(st->amps, i, c64, r0, r1), c64);
  }
}

// ---------------------------------------------------------------------------
// LSD radix sort, 8-bit digits, stable (sparse_state.py:150-172 sorts 16-bit
// digits; any stable LSD order gives the same result)
// ---------------------------------------------------------------------------
constexpr int kSortTile = 2048;

__global__ void __launch_bounds__(256) k_rs_hist(const uint64_t* keys, const long long* n_dev,
                                                 long long n_host, int shift, WsView ws) {
  __shared__ unsigned int h[256];
  const long long n = n_dev ? *n_dev : n_host;
  const long long ntiles = (n + kSortTile - 1) / kSortTile;
  if (ntiles > ws.sort_tiles || n > ws.max_n) return;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    h[threadIdx.x] = 0;
    __syncthreads();
    const long long lo = tile * kSortTile;
    const long long hi = lo + kSortTile < n ? lo + kSortTile : n;
    for (long long i = lo + threadIdx.x; i < hi; i += blockDim.x)
      atomicAdd(&h[(unsigned)(keys[i] >> shift) & 255u], 1u);
    __syncthreads();
    ws.sort_hist[(long long)threadIdx.x * ws.sort_tiles + tile] = h[threadIdx.x];
    __syncthreads();
  }
}

// exclusive scan of the digit-major histogram (256 x ntiles), one CTA
__global__ void __launch_bounds__(1024) k_rs_scan(const long long* n_dev, long long n_host, WsView ws) {
  __shared__ unsigned long long sPart[1024];
  const long long n = n_dev ? *n_dev : n_host;
  const long long ntiles = (n + kSortTile - 1) / kSortTile;
  if (ntiles > ws.sort_tiles || n > ws.max_n) return;
  const long long total = 256 * ntiles;
  const long long per = (total + blockDim.x - 1) / blockDim.x;
  const long long lo = threadIdx.x * per;
  const long long hi = lo + per < total ? lo + per : total;
  auto at = [&](long long k) -> unsigned int& {
    const long long d = k / ntiles, t = k % ntiles;
    return ws.sort_hist[d * ws.sort_tiles + t];
  };
  unsigned long long s = 0;
  for (long long k = lo; k < hi; ++k) s += at(k);
  sPart[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long run = 0;
    for (int i = 0; i < (int)blockDim.x; ++i) {
      const unsigned long long v = sPart[i];
      sPart[i] = run;
      run += v;
    }
  }
  __syncthreads();
  unsigned long long run = sPart[threadIdx.x];
  for (long long k = lo; k < hi; ++k) {
    const unsigned int v = at(k);
    at(k) = (unsigned int)run;
    run += v;
  }
}

// P: the amplitude payload moved with each key (16 B complex128, 8 B complex64)
template <typename P>
__global__ void __launch_bounds__(256) k_rs_scatter(const uint64_t* ik, const P* ia, uint64_t* ok,
                                                    P* oa, const long long* n_dev, long long n_host,
                                                    int shift, WsView ws) {
  __shared__ unsigned int cntw[8][257];
  __shared__ unsigned int run[256];
  __shared__ unsigned int base[256];
  const long long n = n_dev ? *n_dev : n_host;
  const long long ntiles = (n + kSortTile - 1) / kSortTile;
  if (ntiles > ws.sort_tiles || n > ws.max_n) return;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    base[threadIdx.x] = ws.sort_hist[(long long)threadIdx.x * ws.sort_tiles + tile];
    run[threadIdx.x] = 0;
    const long long lo = tile * kSortTile;
    for (int r = 0; r < kSortTile / 256; ++r) {
      for (int d = threadIdx.x; d < 8 * 257; d += 256) (&cntw[0][0])[d] = 0;
      __syncthreads();
      const long long i = lo + r * 256 + threadIdx.x;
      const bool valid = i < n;
      uint64_t key = 0;
      P amp{};
      unsigned dig = 256;
      if (valid) {
        key = ik[i];
        amp = ia[i];
        dig = (unsigned)(key >> shift) & 255u;
      }
      const unsigned peers = __match_any_sync(0xffffffffu, dig);
      const unsigned rank = __popc(peers & ((1u << lane) - 1));
      if (rank == 0) cntw[w][dig] = __popc(peers);
      __syncthreads();
      if (valid) {
        unsigned off = base[dig] + run[dig] + rank;
        for (int ww = 0; ww < w; ++ww) off += cntw[ww][dig];
        ok[off] = key;
        oa[off] = amp;
      }
      __syncthreads();
      {
        unsigned add = 0;
        for (int ww = 0; ww < 8; ++ww) add += cntw[ww][threadIdx.x];
        run[threadIdx.x] += add;
      }
      __syncthreads();
    }
  }
}

template <typename P>
__global__ void k_copy_entries(const uint64_t* ik, const P* ia, uint64_t* ok, P* oa,
                               const long long* n_dev, long long n_host) {
  const long long n = n_dev ? *n_dev : n_host;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    ok[i] = ik[i];
    oa[i] = ia[i];
  }
}

template <typename P>
static cudaError_t radix_sort_t(uint64_t* keys, P* amps, long long n_host, const long long* n_dev, int key_bits,
                                const WsView& ws, cudaStream_t s) {
  const int grid = device().grid_small;
  uint64_t* ks = keys;
  P* as = amps;
  uint64_t* kd = ws.tmp_keys;
  P* ad = reinterpret_cast<P*>(ws.tmp_amps);
  int passes = 0;
  for (int shift = 0; shift < key_bits; shift += 8) {
    KLAUNCH(S_SORT, s, k_rs_hist<<<grid, 256, 0, s>>>(ks, n_dev, n_host, shift, ws));
    KLAUNCH(S_SORT, s, k_rs_scan<<<1, 1024, 0, s>>>(n_dev, n_host, ws));
    KLAUNCH(S_SORT, s, k_rs_scatter<P><<<grid, 256, 0, s>>>(ks, as, kd, ad, n_dev, n_host, shift, ws));
    uint64_t* tk = ks; ks = kd; kd = tk;
    P* ta = as; as = ad; ad = ta;
    ++passes;
  }
  if (passes & 1) KLAUNCH(S_SORT, s, k_copy_entries<P><<<grid, 256, 0, s>>>(ks, as, keys, amps, n_dev, n_host));
  return cudaGetLastError();
}

// amps: complex128 pairs, or complex64 pairs when c64
cudaError_t run_radix_sort(uint64_t* keys, double* amps, long long n_host, const long long* n_dev, int key_bits,
                           const WsView& ws, bass_ctrl* ctrl, cudaStream_t s, int c64) {
  (void)ctrl;
  if (c64)
    return radix_sort_t(keys, reinterpret_cast<unsigned long long*>(amps), n_host, n_dev, key_bits, ws, s);
  return radix_sort_t(keys, reinterpret_cast<ulonglong2*>(amps), n_host, n_dev, key_bits, ws, s);
}

// ---------------------------------------------------------------------------
// sparse_state.py:127-147 merge_sorted_kernel: sum runs of equal keys (left to
// right), one output per run, order kept (decoupled look-back on run heads)
// ---------------------------------------------------------------------------
// complex64 runs are summed in FP32 with the compensated (TwoSum) sum
__global__ void __launch_bounds__(256) k_merge_runs(const uint64_t* keys, const double* amps,
                                                    const long long* n_dev, long long n_host, WsView ws,
                                                    bass_ctrl* c, int c64) {
  __shared__ long long sItem, sBase;
  __shared__ int sWarp[32];
  const long long n = n_dev ? *n_dev : n_host;
  const long long ntiles = (n + kTile - 1) / kTile;
  if (ntiles > ws.max_tiles || n > ws.max_n) {
    if (blockIdx.x == 0 && threadIdx.x == 0) set_error(c, BASS_ERR_WORKSPACE);
    return;
  }
  for (;;) {
    if (threadIdx.x == 0) sItem = (long long)atomicAdd(&reinterpret_cast<unsigned long long*>(ws.counters)[5], 1ULL);
    __syncthreads();
    const long long tile = sItem;
    if (tile >= ntiles) break;
    const long long lo = tile * kTile + threadIdx.x * kPerThread;
    int heads = 0;
    for (int k = 0; k < kPerThread; ++k) {
      const long long i = lo + k;
      if (i < n && (i == 0 || keys[i] != keys[i - 1])) ++heads;
    }
    int total;
    // block scan (inline to keep this file independent of merge.cu)
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = heads;
    for (int off = 1; off < 32; off <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, x, off);
      if (lane >= off) x += y;
    }
    if (lane == 31) sWarp[w] = x;
    __syncthreads();
    if (w == 0) {
      int sv = (lane < 8) ? sWarp[lane] : 0;
      for (int off = 1; off < 32; off <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, sv, off);
        if (lane >= off) sv += y;
      }
      if (lane < 8) sWarp[lane] = sv;
    }
    __syncthreads();
    const int ex = x - heads + (w > 0 ? sWarp[w - 1] : 0);
    total = sWarp[7];
    if (threadIdx.x == 0) {
      const long long b = lookback(ws.status, tile, total, c);
      sBase = b;
      if (tile == ntiles - 1) ws.sel->n_written = b + total;
    }
    __syncthreads();
    long long o = sBase + ex;
    for (int k = 0; k < kPerThread; ++k) {
      const long long i = lo + k;
      if (i < n && (i == 0 || keys[i] != keys[i - 1])) {
        double2 acc = amp_raw(amps, i, c64);
        if (c64) {
          Dot2f re{(float)acc.x, 0.f}, im{(float)acc.y, 0.f};
          for (long long r = i + 1; r < n && keys[r] == keys[i]; ++r) {
            const double2 v = amp_raw(amps, r, 1);
            dot2_add(re, (float)v.x, 1.f);
            dot2_add(im, (float)v.y, 1.f);
          }
          acc = make_double2((double)dot2_get(re), (double)dot2_get(im));
        } else {
          for (long long r = i + 1; r < n && keys[r] == keys[i]; ++r) acc = cadd(acc, amp_raw(amps, r, 0));
        }
        ws.tmp_keys[o] = keys[i];
        amp_put(reinterpret_cast<double*>(ws.tmp_amps), o, acc, c64);
        ++o;
      }
    }
    __syncthreads();
  }
}

__global__ void k_merge_out(uint64_t* keys, double* amps, WsView ws, long long* n_out, bass_state* st, int c64) {
  const long long n = ws.sel->n_written;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    keys[i] = ws.tmp_keys[i];
    amp_put(amps, i, amp_raw(reinterpret_cast<const double*>(ws.tmp_amps), i, c64), c64);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (n_out) *n_out = n;
    if (st) st->nnz = n;
  }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// dense vectors (bass_simulator.py:608-621 to_statevector; fidelity.py:48-68
// compute_fidelity, runner.py:620-626 np.vdot), for n <= 30 qubits
// ---------------------------------------------------------------------------
// psi[true key] = a (pending scale applied); psi was zeroed.  A key with a
// bit at or above nq (a state of more qubits than psi holds) is refused.
__global__ void k_dense_scatter(const bass_state* st, double2* psi, int nq, bass_ctrl* c) {
  __shared__ int8_t qat[64];
  if (threadIdx.x < 64) qat[threadIdx.x] = st->qat[threadIdx.x];
  __syncthreads();
  const long long n = st->nnz;
  const double r0 = st->rscale[0], r1 = st->rscale[1];
  const int c64 = st->amp_type == BASS_AMP_C64;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
  {
    const uint64_t tk = true_key(st->keys[i], qat, 64);
    if (tk >> nq) {
      set_error(c, BASS_ERR_ARG);
      continue;
    }
    psi[tk] = amp_get(st->amps, i, c64, r0, r1);
  }
}

// U applied to qubit j of a dense vector of 2 half entries: each pair
// (bit j clear, bit j set) becomes (u00 a0 + u01 a1, u10 a0 + u11 a1).
__global__ void k_dense_1q(double2* psi, long long half, int j, double2 u00, double2 u01, double2 u10,
                           double2 u11) {
  const long long lowmask = (1LL << j) - 1;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < half;
       p += (long long)gridDim.x * blockDim.x) {
    const long long i0 = ((p & ~lowmask) << 1) | (p & lowmask), i1 = i0 | (1LL << j);
    const double2 a0 = psi[i0], a1 = psi[i1];
    psi[i0] = cadd(cmul(u00, a0), cmul(u01, a1));
    psi[i1] = cadd(cmul(u10, a0), cmul(u11, a1));
  }
}

// A 4x4 gate G (index (b_q1 << 1) | b_q2, row-major) applied to qubits
// (q1, q2) of a dense vector of 4 quarter entries: each group of four
// amplitudes is read, multiplied and written back by one thread, the sum over
// input indices in ascending order (exact_simulator.py:121-144).
__global__ void k_dense_2q(double2* psi, long long quarter, int q1, int q2, const __grid_constant__ DenseG4 g) {
  const int lo = q1 < q2 ? q1 : q2, hi = q1 < q2 ? q2 : q1;
  // p has nq - 2 bits: a zero is inserted at bit lo, then (in the nq - 1 bit
  // result) at bit hi
  const long long mlo = (1LL << lo) - 1, mhi = (1LL << hi) - 1;
  const long long b1 = 1LL << q1, b2 = 1LL << q2;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < quarter;
       p += (long long)gridDim.x * blockDim.x) {
    long long i = ((p & ~mlo) << 1) | (p & mlo);
    i = ((i & ~mhi) << 1) | (i & mhi);
    const long long idx[4] = {i, i | b2, i | b1, i | b1 | b2};
    double2 a[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) a[r] = psi[idx[r]];
#pragma unroll
    for (int o = 0; o < 4; ++o) {
      double2 acc = cmul(g.m[o * 4], a[0]);
#pragma unroll
      for (int r = 1; r < 4; ++r) acc = cadd(acc, cmul(g.m[o * 4 + r], a[r]));
      psi[idx[o]] = acc;
    }
  }
}

// Per-CTA exact partial sums of conj(u_i) v_i (re, im) into ws.red[2 b ..];
// sparse: u is psi at the state's true keys and v its amplitudes.
template <bool SPARSE>
__global__ void __launch_bounds__(256) k_dot(const double2* u, const double2* v, long long n,
                                             const bass_state* st, int nq, WsView ws, bass_ctrl* ctl) {
  __shared__ i128 sRed[2 * 8];
  __shared__ int8_t qat[64];
  long long nn = n;
  double r0 = 1.0, r1 = 1.0;
  int c64 = 0;
  if (SPARSE) {
    if (threadIdx.x < 64) qat[threadIdx.x] = st->qat[threadIdx.x];
    __syncthreads();
    nn = st->nnz;
    r0 = st->rscale[0];
    r1 = st->rscale[1];
    c64 = st->amp_type == BASS_AMP_C64;
  }
  i128 acc[2] = {0, 0};
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i0 = (long long)blockIdx.x * blockDim.x + threadIdx.x; i0 < nn; i0 += 8 * stride) {
    double h[2] = {0.0, 0.0}, l[2] = {0.0, 0.0};
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const long long i = i0 + k * stride;
      if (i >= nn) break;
      double2 a, b;
      if (SPARSE) {
        const uint64_t tk = true_key(st->keys[i], qat, 64);
        if (tk >> nq) {  // refused as in k_dense_scatter
          set_error(ctl, BASS_ERR_ARG);
          continue;
        }
        a = u[tk];
        b = amp_get(st->amps, i, c64, r0, r1);
      } else {
        a = u[i];
        b = v[i];
      }
      const double2 c = cmul(make_double2(a.x, -a.y), b);
      fx_acc96(c.x, h[0], l[0], acc[0]);
      fx_acc96(c.y, h[1], l[1], acc[1]);
    }
    acc[0] += fx_join96s(h[0], l[0]);
    acc[1] += fx_join96s(h[1], l[1]);
  }
  block_sum_i128<2>(acc, sRed);
  if (threadIdx.x == 0) {
    ws.red[2 * blockIdx.x] = acc[0];
    ws.red[2 * blockIdx.x + 1] = acc[1];
  }
}

__global__ void k_dot_final(WsView ws, int nblk, double* out) {
  __shared__ i128 sRed[2 * 8];
  i128 acc[2] = {0, 0};
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
    acc[0] += ws.red[2 * b];
    acc[1] += ws.red[2 * b + 1];
  }
  block_sum_i128<2>(acc, sRed);
  if (threadIdx.x == 0) {
    out[0] = fx_to(acc[0]);
    out[1] = fx_to(acc[1]);
  }
}

cudaError_t run_to_dense(const bass_state* st, const double* host_U, int nq, double* psi, bass_ctrl* ctrl,
                         cudaStream_t s) {
  const long long n = 1LL << nq;
  cudaError_t e = cudaMemsetAsync(psi, 0, (size_t)n * 16, s);
  if (e != cudaSuccess) return e;
  double2* p = reinterpret_cast<double2*>(psi);
  KLAUNCH(S_SMALL, s, k_dense_scatter<<<device().grid_small, 256, 0, s>>>(st, p, nq, ctrl));
  if (host_U) {
    const int grid = device().sms * 8;
    for (int j = 0; j < nq; ++j) {
      const double* u = host_U + 8 * j;
      KLAUNCH(S_SMALL, s,
              k_dense_1q<<<grid, 256, 0, s>>>(p, n / 2, j, make_double2(u[0], u[1]), make_double2(u[2], u[3]),
                                               make_double2(u[4], u[5]), make_double2(u[6], u[7])));
    }
  }
  return cudaGetLastError();
}

cudaError_t run_dense_gate(double* psi, int nq, const double* host_G, int nqg, int q1, int q2, cudaStream_t s) {
  double2* p = reinterpret_cast<double2*>(psi);
  const int grid = device().sms * 8;
  const double* u = host_G;
  if (nqg == 1) {
    KLAUNCH(S_SMALL, s,
            k_dense_1q<<<grid, 256, 0, s>>>(p, (1LL << nq) / 2, q1, make_double2(u[0], u[1]),
                                             make_double2(u[2], u[3]), make_double2(u[4], u[5]),
                                             make_double2(u[6], u[7])));
  } else {
    DenseG4 g;
    for (int i = 0; i < 16; ++i) g.m[i] = make_double2(u[2 * i], u[2 * i + 1]);
    KLAUNCH(S_SMALL, s, k_dense_2q<<<grid, 256, 0, s>>>(p, (1LL << nq) / 4, q1, q2, g));
  }
  return cudaGetLastError();
}

cudaError_t run_dot(const double* u, const double* v, long long n, const bass_state* st, int nq, double* out,
                    bass_ctrl* ctrl, const WsView& ws, cudaStream_t s) {
  const int grid = 512;  // ws.red holds 1024 partials: two per CTA
  const double2* a = reinterpret_cast<const double2*>(u);
  const double2* b = reinterpret_cast<const double2*>(v);
  if (st) KLAUNCH(S_REDUCE, s, k_dot<true><<<grid, 256, 0, s>>>(a, b, 0, st, nq, ws, ctrl));
  else KLAUNCH(S_REDUCE, s, k_dot<false><<<grid, 256, 0, s>>>(a, b, n, nullptr, 64, ws, ctrl));
  KLAUNCH(S_REDUCE, s, k_dot_final<<<1, 256, 0, s>>>(ws, grid, out));
  return cudaGetLastError();
}

cudaError_t run_reduce(const bass_state* st, int mode, double* dest, bass_ctrl* ctrl,
                       const WsView& ws, cudaStream_t s) {
  const int grid = device().grid_small > 1024 ? 1024 : device().grid_small;
  const bool c64 = state_c64(st);
  if (mode == R_NORM2) {
    if (c64) KLAUNCH(S_REDUCE, s, k_reduce_state<R_NORM2, true><<<grid, 256, 0, s>>>(st, ws));
    else KLAUNCH(S_REDUCE, s, k_reduce_state<R_NORM2, false><<<grid, 256, 0, s>>>(st, ws));
  } else {
    if (c64) KLAUNCH(S_REDUCE, s, k_reduce_state<R_P2, true><<<grid, 256, 0, s>>>(st, ws));
    else KLAUNCH(S_REDUCE, s, k_reduce_state<R_P2, false><<<grid, 256, 0, s>>>(st, ws));
  }
  if (dest) KLAUNCH(S_REDUCE, s, k_red_store<<<1, 256, 0, s>>>(ws, grid, dest));
  else KLAUNCH(S_REDUCE, s, k_pr_final<<<1, 256, 0, s>>>(st, ws, grid, ctrl));
  return cudaGetLastError();
}

cudaError_t run_fingerprint(const bass_state* st, double pmin, uint64_t* out6, const WsView& ws,
                            cudaStream_t s, bass_ctrl* ctrl, int append_event, int only_if_trunc) {
  cudaError_t e = cudaMemsetAsync(ws.fp, 0, 8 * sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  KLAUNCH(S_FINGERPRINT, s, k_fingerprint<<<device().grid_small, 256, 0, s>>>(st, pmin, ws));
  KLAUNCH(S_FINGERPRINT, s, k_fp_out<<<1, 1, 0, s>>>(ws, out6, ctrl, append_event, only_if_trunc));
  return cudaGetLastError();
}

cudaError_t run_renorm(bass_state* st, bass_ctrl* ctrl, const WsView& ws, cudaStream_t s) {
  const int grid = device().grid_small > 1024 ? 1024 : device().grid_small;
  if (state_c64(st)) KLAUNCH(S_REDUCE, s, k_reduce_state<R_NORM2, true><<<grid, 256, 0, s>>>(st, ws));
  else KLAUNCH(S_REDUCE, s, k_reduce_state<R_NORM2, false><<<grid, 256, 0, s>>>(st, ws));
  KLAUNCH(S_REDUCE, s, k_renorm_apply<<<1, 256, 0, s>>>(st, ws, grid));
  KLAUNCH(S_SMALL, s, k_materialize<<<device().sms * 4, 256, 0, s>>>(st, ws, ctrl));
  return cudaGetLastError();
}

cudaError_t run_phase2q_seg(const OpArgs* ops, int nseg, int c64, cudaStream_t s) {
  const dim3 grid(device().sms, nseg);
  if (c64) KLAUNCH(S_PHASE2Q, s, k_phase2q_seg<true><<<grid, 256, 0, s>>>(ops));
  else KLAUNCH(S_PHASE2Q, s, k_phase2q_seg<false><<<grid, 256, 0, s>>>(ops));
  return cudaGetLastError();
}

// mode 1: PR of every state (ctrl->pr_last); mode 0: renormalise every state
cudaError_t run_reduce_seg(const OpArgs* ops, int nseg, int mode, int c64, cudaStream_t s) {
  const int gx = 64;  // partials per state (ws.red holds 1024)
  const dim3 grid(gx, nseg);
  if (mode == 1) {
    if (c64) KLAUNCH(S_REDUCE, s, k_reduce_state_seg<R_P2, true><<<grid, 256, 0, s>>>(ops));
    else KLAUNCH(S_REDUCE, s, k_reduce_state_seg<R_P2, false><<<grid, 256, 0, s>>>(ops));
    KLAUNCH(S_REDUCE, s, k_pr_final_seg<<<nseg, 256, 0, s>>>(ops, gx));
  } else {
    if (c64) KLAUNCH(S_REDUCE, s, k_reduce_state_seg<R_NORM2, true><<<grid, 256, 0, s>>>(ops));
    else KLAUNCH(S_REDUCE, s, k_reduce_state_seg<R_NORM2, false><<<grid, 256, 0, s>>>(ops));
    KLAUNCH(S_REDUCE, s, k_renorm_apply_seg<<<nseg, 256, 0, s>>>(ops, gx));
    KLAUNCH(S_SMALL, s, k_materialize_seg<<<dim3(device().sms, nseg), 256, 0, s>>>(ops));
  }
  return cudaGetLastError();
}

cudaError_t run_phase2q(bass_state* st, const double* d, int q1, int q2, bass_ctrl* ctrl, cudaStream_t s) {
  const double2 d0 = make_double2(d[0], d[1]), d1 = make_double2(d[2], d[3]);
  const double2 d2 = make_double2(d[4], d[5]), d3 = make_double2(d[6], d[7]);
  if (state_c64(st))
    KLAUNCH(S_PHASE2Q, s, k_phase2q<true><<<device().sms * 4, 256, 0, s>>>(st, d0, d1, d2, d3, q1, q2, ctrl));
  else
    KLAUNCH(S_PHASE2Q, s, k_phase2q<false><<<device().sms * 4, 256, 0, s>>>(st, d0, d1, d2, d3, q1, q2, ctrl));
  return cudaGetLastError();
}

cudaError_t run_phase1q(bass_state* st, bass_state* tmp, const double* g, int q, bass_ctrl* ctrl,
                        const WsView& ws, cudaStream_t s, int c64) {
  cudaError_t e = zero_small(ws, s);
  if (e != cudaSuccess) return e;
  if (c64)
    KLAUNCH(S_PHASE1Q, s, k_phase1q<true><<<device().sms * 4, 256, 0, s>>>(st, make_double2(g[0], g[1]),
                                                                           make_double2(g[2], g[3]), q, ctrl, ws));
  else
    KLAUNCH(S_PHASE1Q, s, k_phase1q<false><<<device().sms * 4, 256, 0, s>>>(st, make_double2(g[0], g[1]),
                                                                            make_double2(g[2], g[3]), q, ctrl, ws));
  OpArgs a{};
  a.in = st;
  a.out = tmp;
  a.ctrl = ctrl;
  a.ws = ws;
  a.drop_zero = 1;
  a.guard = 1;
  a.nsets = 1;
  a.k_cond = -1;
  a.c64 = c64;
  e = run_ident_write(a, s);
  if (e != cudaSuccess) return e;
  KLAUNCH(S_PHASE1Q, s, k_phase1q_fin<<<1, 1, 0, s>>>(st, tmp, ws));
  return cudaGetLastError();
}

cudaError_t run_state_init(bass_state* st, uint64_t* keys, double* amps, long long cap, int nq,
                           uint64_t key, int amp_type, cudaStream_t s) {
  KLAUNCH(S_SMALL, s, k_state_init<<<1, 1, 0, s>>>(st, keys, amps, cap, nq, key, amp_type));
  return cudaGetLastError();
}

cudaError_t run_import(bass_state* st, const uint64_t* keys, const double* amps, long long n, int nq,
                       const WsView& ws, bass_ctrl* ctrl, cudaStream_t s, uint64_t* st_keys,
                       double* st_amps, long long cap, int amp_type) {
  const int c64 = amp_type == BASS_AMP_C64;
  cudaError_t e = cudaMemcpyAsync(st_keys, keys, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s);
  if (e != cudaSuccess) return e;
  e = cudaMemcpyAsync(st_amps, amps, n * (c64 ? 2 * sizeof(float) : 2 * sizeof(double)), cudaMemcpyDeviceToDevice, s);
  if (e != cudaSuccess) return e;
  KLAUNCH(S_SMALL, s, k_state_adopt<<<1, 1, 0, s>>>(st, st_keys, st_amps, cap, nq, n, amp_type));
  e = run_radix_sort(st_keys, st_amps, n, nullptr, nq > 0 ? nq : 1, ws, ctrl, s, c64);
  if (e != cudaSuccess) return e;
  if ((e = zero_small(ws, s)) != cudaSuccess) return e;
  KLAUNCH(S_MERGE_RUNS, s, k_merge_runs<<<device().grid_small, 256, 0, s>>>(st_keys, st_amps, nullptr, n, ws, ctrl, c64));
  KLAUNCH(S_MERGE_RUNS, s, k_merge_out<<<device().grid_small, 256, 0, s>>>(st_keys, st_amps, ws, nullptr, st, c64));
  return cudaGetLastError();
}

cudaError_t run_export(const bass_state* st, uint64_t* ok, double* oa, int key_bits, const WsView& ws,
                       bass_ctrl* ctrl, cudaStream_t s, int amp_type) {
  KLAUNCH(S_SORT, s, k_export<<<device().grid_small, 256, 0, s>>>(st, ok, oa, ws.max_n, amp_type, ctrl));
  return run_radix_sort(ok, oa, 0, reinterpret_cast<const long long*>(&st->nnz), key_bits, ws, ctrl, s,
                        amp_type == BASS_AMP_C64);
}

cudaError_t run_merge_sorted(uint64_t* keys, double* amps, long long n, long long* n_out,
                             const WsView& ws, bass_ctrl* ctrl, cudaStream_t s) {
  cudaError_t e = zero_small(ws, s);
  if (e != cudaSuccess) return e;
  KLAUNCH(S_MERGE_RUNS, s, k_merge_runs<<<device().grid_small, 256, 0, s>>>(keys, amps, nullptr, n, ws, ctrl, 0));
  KLAUNCH(S_MERGE_RUNS, s, k_merge_out<<<device().grid_small, 256, 0, s>>>(keys, amps, ws, n_out, nullptr, 0));
  return cudaGetLastError();
}

cudaError_t run_clone(bass_state* dst, const bass_state* src, bass_ctrl* ctrl, cudaStream_t s) {
  KLAUNCH(S_SMALL, s, k_clone<<<device().sms * 4, 256, 0, s>>>(dst, src, ctrl));
  KLAUNCH(S_SMALL, s, k_clone_desc<<<1, 1, 0, s>>>(dst, src));
  return cudaGetLastError();
}

cudaError_t run_copy_desc(bass_state* dst, const bass_state* src, cudaStream_t s) {
  KLAUNCH(S_SMALL, s, k_copy_desc<<<1, 1, 0, s>>>(dst, src));
  return cudaGetLastError();
}

__global__ void k_ctrl_init(bass_ctrl* c, uint64_t* trace, long long cap, double tol) {
  bass_ctrl z;
  memset(&z, 0, sizeof z);
  z.gamma_running = 1.0;
  z.state_gamma = 1.0;
  z.trace = trace;
  z.trace_cap = cap;
  z.pr_tie_tol = tol;
  *c = z;
}

cudaError_t run_ctrl_init(bass_ctrl* c, uint64_t* trace, long long cap, double tol, cudaStream_t s) {
  KLAUNCH(S_SMALL, s, k_ctrl_init<<<1, 1, 0, s>>>(c, trace, cap, tol));
  return cudaGetLastError();
}

cudaError_t run_gather(const bass_state* in, bass_state* out, const int64_t* idx, long long n,
                       bass_ctrl* ctrl, cudaStream_t s) {
  KLAUNCH(S_SMALL, s, k_gather<<<device().sms * 4, 256, 0, s>>>(in, out, idx, n, ctrl));
  KLAUNCH(S_SMALL, s, k_gather_desc<<<1, 1, 0, s>>>(in, out, n));
  return cudaGetLastError();
}

}  // namespace bass
