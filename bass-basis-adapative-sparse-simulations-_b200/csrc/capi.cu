// capi.cu -- the extern "C" entry points of libbass_b200.so (include/bass_b200.h).
#include <stdlib.h>
#include <string.h>

#include <atomic>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "internal.h"

namespace bass {

// ---------------------------------------------------------------------------
// instrumentation
// ---------------------------------------------------------------------------
struct ProfRec {
  int slot;
  cudaEvent_t a, b;
};
static std::atomic<long long> g_launches{0};
static std::atomic<bool> g_prof{false};
static std::mutex g_prof_mu;
static std::vector<ProfRec> g_recs;
static std::vector<cudaEvent_t> g_pool;

static cudaEvent_t pool_event() {
  if (!g_pool.empty()) {
    cudaEvent_t e = g_pool.back();
    g_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

bool prof_on() { return g_prof.load(std::memory_order_relaxed); }

ProfScope::ProfScope(int s, cudaStream_t st) : slot(s), stream(st), start(nullptr), on(prof_on()) {
  if (on) {
    std::lock_guard<std::mutex> lk(g_prof_mu);
    start = pool_event();
    cudaEventRecord(start, stream);
  }
}

ProfScope::~ProfScope() {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (on && start) {
    std::lock_guard<std::mutex> lk(g_prof_mu);
    cudaEvent_t stop = pool_event();
    cudaEventRecord(stop, stream);
    g_recs.push_back(ProfRec{slot, start, stop});
  }
}

const Device& device() {
  static Device d[kMaxDevices + 1];
  static std::once_flag once[kMaxDevices + 1];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) dev = kMaxDevices;
  std::call_once(once[dev], [dev] {
    Device x{};
    int sms = 0;
    if (dev < kMaxDevices) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    x.sms = sms > 0 ? sms : 1;
    x.grid_small = x.sms * 8;
    x.grid_tile = x.sms * 2;
    x.grid_tile_h = x.sms;
    d[dev] = x;
  });
  return d[dev];
}

// ---------------------------------------------------------------------------
// workspace layout: a pure function of its size, so that every call can carve
// it without extra arguments.  max_n bounds every op's input and output count.
// ---------------------------------------------------------------------------
static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

struct Layout {
  size_t counters, hist1, hist2, sel, status, fp, red, part, partials, cand_bits, cand_key, tmp_keys,
      tmp_amps, stage_keys, kmask, sort_hist, total;
  long long max_tiles, sort_tiles;
};

static Layout layout_for(long long max_n) {
  Layout L{};
  L.max_tiles = max_n / kStep + 2;
  L.sort_tiles = max_n / 2048 + 2;
  size_t o = 0;
  L.counters = o; o += align256(64 * 8);
  L.hist1 = o; o += align256((kHistBins + kHistGroups) * 4);
  L.hist2 = o; o += align256((kHistBins + kHistGroups) * 4);
  L.sel = o; o += align256(sizeof(SelState));
  L.status = o; o += align256((size_t)L.max_tiles * 8);
  L.fp = o; o += align256(8 * 8);
  L.red = o; o += align256(1024 * sizeof(i128));
  L.part = o; o += align256((size_t)kMaxSets * (L.max_tiles + 1) * 6 * 8);
  const long long np = (long long)kMaxSets * L.max_tiles > 1024 ? (long long)kMaxSets * L.max_tiles : 1024;
  L.partials = o; o += align256((size_t)np * sizeof(Partial));
  L.cand_bits = o; o += align256((size_t)max_n * 8);
  L.cand_key = o; o += align256((size_t)max_n * 8);
  L.tmp_keys = o; o += align256((size_t)max_n * 8);
  L.tmp_amps = o; o += align256((size_t)max_n * 16);
  L.stage_keys = o; o += align256((size_t)max_n * 8);
  L.kmask = o; o += align256((size_t)max_n / 8 + 64);
  L.sort_hist = o; o += align256((size_t)256 * L.sort_tiles * 4);
  L.total = o;
  return L;
}

size_t ws_bytes_for(long long max_n) { return layout_for(max_n < 1 ? 1 : max_n).total; }

bool carve(void* ws, size_t ws_bytes, WsView* v) {
  if (!ws || ((uintptr_t)ws & 255)) return false;
  if (ws_bytes < ws_bytes_for(1)) return false;
  long long lo = 1, hi = 1LL << 40;
  while (lo < hi) {  // largest max_n whose layout fits
    const long long mid = lo + (hi - lo + 1) / 2;
    if (ws_bytes_for(mid) <= ws_bytes) lo = mid;
    else hi = mid - 1;
  }
  const Layout L = layout_for(lo);
  char* b = static_cast<char*>(ws);
  v->counters = reinterpret_cast<unsigned int*>(b + L.counters);
  v->hist1 = reinterpret_cast<unsigned int*>(b + L.hist1);
  v->hist2 = reinterpret_cast<unsigned int*>(b + L.hist2);
  v->sel = reinterpret_cast<SelState*>(b + L.sel);
  v->status = reinterpret_cast<unsigned long long*>(b + L.status);
  v->fp = reinterpret_cast<unsigned long long*>(b + L.fp);
  v->red = reinterpret_cast<i128*>(b + L.red);
  v->part = reinterpret_cast<long long*>(b + L.part);
  v->partials = reinterpret_cast<Partial*>(b + L.partials);
  v->cand_bits = reinterpret_cast<unsigned long long*>(b + L.cand_bits);
  v->cand_key = reinterpret_cast<unsigned long long*>(b + L.cand_key);
  v->tmp_keys = reinterpret_cast<uint64_t*>(b + L.tmp_keys);
  v->tmp_amps = reinterpret_cast<double2*>(b + L.tmp_amps);
  v->stage_keys = reinterpret_cast<uint64_t*>(b + L.stage_keys);
  v->kmask = reinterpret_cast<uint8_t*>(b + L.kmask);
  v->sort_hist = reinterpret_cast<unsigned int*>(b + L.sort_hist);
  v->max_n = lo;
  v->max_tiles = L.max_tiles;
  v->sort_tiles = L.sort_tiles;
  return true;
}

static int status_of(cudaError_t e) { return e == cudaSuccess ? BASS_OK : BASS_ERR_CUDA; }

// The amplitude type of every descriptor set up through this library, keyed
// by its device address (unique across devices under unified addressing).
// Launches pick the kernels for that type from here; the kernels compare it
// with the descriptor's own amp_type and refuse a mismatch (BASS_ERR_ARG).
// A descriptor never set up here counts as complex128.
static std::mutex g_type_mu;
static std::unordered_map<const void*, int> g_types;

static void remember_type(const bass_state* st, int amp_type) {
  std::lock_guard<std::mutex> lk(g_type_mu);
  if (amp_type == BASS_AMP_C128) g_types.erase(st);
  else g_types[st] = amp_type;
}

int state_c64(const bass_state* st) {
  std::lock_guard<std::mutex> lk(g_type_mu);
  const auto it = g_types.find(st);
  return it != g_types.end() && it->second == BASS_AMP_C64;
}

static void load_G(OpArgs& a, const double* g, int n) {
  for (int i = 0; i < n; ++i) a.G[i] = make_double2(g[2 * i], g[2 * i + 1]);
}

}  // namespace bass

using namespace bass;

#define CHECK_WS(ws, bytes, v) \
  WsView v;                    \
  if (!carve(ws, bytes, &v)) return BASS_ERR_WORKSPACE;

extern "C" {

const char* bass_version(void) { return "bass_b200 1.0 (sm_100a)"; }

size_t bass_state_bytes(void) { return sizeof(bass_state); }
size_t bass_ctrl_bytes(void) { return sizeof(bass_ctrl); }
size_t bass_workspace_bytes(int64_t max_in, int64_t max_out, int num_qubits) {
  (void)num_qubits;
  // the evaluation pass of a 2-qubit gate keeps four |a|^2 slots per input entry
  const long long m = 4 * max_in > max_out ? 4 * max_in : max_out;
  return ws_bytes_for(m);
}

static bool amp_type_ok(int t) { return t == BASS_AMP_C128 || t == BASS_AMP_C64; }
// Key arrays are read as 8-byte words, amplitude arrays as 16-byte
// (complex128) or 8-byte (complex64) vectors.
static bool arrays_aligned(const void* keys, const void* amps, int amp_type) {
  const uintptr_t ka = reinterpret_cast<uintptr_t>(keys), aa = reinterpret_cast<uintptr_t>(amps);
  return (ka & 7) == 0 && (aa & (amp_type == BASS_AMP_C64 ? 7 : 15)) == 0;
}

int bass_state_init_typed(bass_state* st, uint64_t* keys, double* amps, int64_t cap, int num_qubits,
                          uint64_t init_key, int amp_type, void* stream) {
  if (!st || !keys || !amps || cap < 1 || num_qubits < 1 || num_qubits > BASS_MAX_QUBITS || !amp_type_ok(amp_type))
    return BASS_ERR_ARG;
  if (num_qubits < 64 && (init_key >> num_qubits) != 0) return BASS_ERR_ARG;
  if (!arrays_aligned(keys, amps, amp_type)) return BASS_ERR_ARG;
  remember_type(st, amp_type);
  return status_of(run_state_init(st, keys, amps, cap, num_qubits, init_key, amp_type, (cudaStream_t)stream));
}

int bass_state_init(bass_state* st, uint64_t* keys, double* amps, int64_t cap, int num_qubits,
                    uint64_t init_key, void* stream) {
  return bass_state_init_typed(st, keys, amps, cap, num_qubits, init_key, BASS_AMP_C128, stream);
}

int bass_state_import_typed(bass_state* st, uint64_t* st_keys, double* st_amps, int64_t cap,
                            const uint64_t* keys, const double* amps, int64_t n, int num_qubits, int amp_type,
                            void* ws, size_t ws_bytes, bass_ctrl* ctrl, void* stream) {
  if (!st || !st_keys || !st_amps || (n > 0 && (!keys || !amps)) || n < 0 || n > cap || num_qubits < 1 ||
      num_qubits > BASS_MAX_QUBITS || !ctrl || !amp_type_ok(amp_type))
    return BASS_ERR_ARG;
  if (!arrays_aligned(st_keys, st_amps, amp_type) || (n > 0 && !arrays_aligned(keys, amps, amp_type)))
    return BASS_ERR_ARG;
  CHECK_WS(ws, ws_bytes, v);
  if (n > v.max_n) return BASS_ERR_WORKSPACE;
  remember_type(st, amp_type);
  return status_of(run_import(st, keys, amps, n, num_qubits, v, ctrl, (cudaStream_t)stream, st_keys,
                              st_amps, cap, amp_type));
}

int bass_state_import_into(bass_state* st, uint64_t* st_keys, double* st_amps, int64_t cap,
                           const uint64_t* keys, const double* amps, int64_t n, int num_qubits,
                           void* ws, size_t ws_bytes, bass_ctrl* ctrl, void* stream) {
  return bass_state_import_typed(st, st_keys, st_amps, cap, keys, amps, n, num_qubits, BASS_AMP_C128, ws,
                                 ws_bytes, ctrl, stream);
}

int bass_state_export_typed(const bass_state* st, uint64_t* out_keys, double* out_amps, int key_bits,
                            int amp_type, void* ws, size_t ws_bytes, bass_ctrl* ctrl, void* stream) {
  if (!st || !out_keys || !out_amps || !ctrl || key_bits < 1 || key_bits > 64 || !amp_type_ok(amp_type))
    return BASS_ERR_ARG;
  if (!arrays_aligned(out_keys, out_amps, amp_type)) return BASS_ERR_ARG;
  CHECK_WS(ws, ws_bytes, v);
  return status_of(run_export(st, out_keys, out_amps, key_bits, v, ctrl, (cudaStream_t)stream, amp_type));
}

int bass_state_export(const bass_state* st, uint64_t* out_keys, double* out_amps, void* ws,
                      size_t ws_bytes, bass_ctrl* ctrl, void* stream) {
  return bass_state_export_typed(st, out_keys, out_amps, 64, BASS_AMP_C128, ws, ws_bytes, ctrl, stream);
}

int bass_state_export_bits(const bass_state* st, uint64_t* out_keys, double* out_amps, int key_bits,
                           void* ws, size_t ws_bytes, bass_ctrl* ctrl, void* stream) {
  return bass_state_export_typed(st, out_keys, out_amps, key_bits, BASS_AMP_C128, ws, ws_bytes, ctrl, stream);
}

int bass_state_copy_desc(bass_state* dst, const bass_state* src, void* stream) {
  if (!dst || !src) return BASS_ERR_ARG;
  remember_type(dst, state_c64(src) ? BASS_AMP_C64 : BASS_AMP_C128);
  return status_of(run_copy_desc(dst, src, (cudaStream_t)stream));
}

int bass_state_clone(bass_state* dst, const bass_state* src, bass_ctrl* ctrl, void* stream) {
  if (!dst || !src || !ctrl) return BASS_ERR_ARG;
  return status_of(run_clone(dst, src, ctrl, (cudaStream_t)stream));
}

int bass_ctrl_init(bass_ctrl* ctrl, uint64_t* trace, int64_t trace_cap, double pr_tie_tol, void* stream) {
  if (!ctrl || trace_cap < 0 || (trace_cap > 0 && !trace) || !(pr_tie_tol >= 0.0)) return BASS_ERR_ARG;
  return status_of(run_ctrl_init(ctrl, trace, trace_cap, pr_tie_tol, (cudaStream_t)stream));
}

int bass_gate_1q(const bass_state* in, bass_state* out, const double* host_G, int q, bass_trunc tr,
                 bass_ctrl* ctrl, void* ws, size_t ws_bytes, void* stream) {
  if (!in || !out || in == out || !host_G || q < 0 || q >= BASS_MAX_QUBITS || !ctrl) return BASS_ERR_ARG;
  CHECK_WS(ws, ws_bytes, v);
  cudaStream_t s = (cudaStream_t)stream;
  OpArgs a{};
  a.in = in; a.out = out; a.ctrl = ctrl; a.ws = v; a.q = q; a.gb = 0; a.c64 = state_c64(in);
  load_G(a, host_G, 4);
  cudaError_t e = run_merge_op(K_GATE1, a, tr, 0, 0, s);
  if (e == cudaSuccess && tr.trace) e = run_fingerprint(out, kSigPmin, nullptr, v, s, ctrl, 1, 1);
  return status_of(e);
}

int bass_gate_2q(const bass_state* in, bass_state* tmp, bass_state* out, const double* host_G, int q1,
                 int q2, bass_trunc tr, bass_ctrl* ctrl, void* ws, size_t ws_bytes, void* stream) {
  if (!in || !tmp || !out || in == tmp || tmp == out || in == out || !host_G || q1 < 0 || q2 < 0 ||
      q1 >= BASS_MAX_QUBITS || q2 >= BASS_MAX_QUBITS || q1 == q2 || !ctrl)
    return BASS_ERR_ARG;
  CHECK_WS(ws, ws_bytes, v);
  cudaStream_t s = (cudaStream_t)stream;
  // pass 1: bring q2 to the lowest physical bit (a pure reorder)
  OpArgs a{};
  a.in = in; a.out = tmp; a.ctrl = ctrl; a.ws = v; a.q = q2; a.gb = 0; a.c64 = state_c64(in);
  bass_trunc none{};
  none.k_cond = -1;
  cudaError_t e = run_merge_op(K_PERM, a, none, 0, 0, s);
  if (e != cudaSuccess) return status_of(e);
  // pass 2: merge on q1 above it; groups of four are (b_q1, b_q2) in input-index order
  OpArgs b{};
  b.in = tmp; b.out = out; b.ctrl = ctrl; b.ws = v; b.q = q1; b.gb = 1; b.c64 = a.c64;
  load_G(b, host_G, 16);
  e = run_merge_op(K_GATE2, b, tr, 0, 0, s);
  if (e == cudaSuccess && tr.trace) e = run_fingerprint(out, kSigPmin, nullptr, v, s, ctrl, 1, 1);
  return status_of(e);
}

int bass_rotate_2q(const bass_state* in, bass_state* tmp, bass_state* out, const double* host_U4, int q1,
                   int q2, bass_trunc tr, bass_ctrl* ctrl, void* ws, size_t ws_bytes, void* stream) {
  if (!in || !tmp || !out || in == tmp || tmp == out || in == out || !host_U4 || q1 < 0 || q2 < 0 ||
      q1 >= BASS_MAX_QUBITS || q2 >= BASS_MAX_QUBITS || q1 == q2 || !ctrl)
    return BASS_ERR_ARG;
  CHECK_WS(ws, ws_bytes, v);
  cudaStream_t s = (cudaStream_t)stream;
  // pass 1: bring q2 to the lowest physical bit (a pure reorder)
  OpArgs a{};
  a.in = in; a.out = tmp; a.ctrl = ctrl; a.ws = v; a.q = q2; a.gb = 0; a.c64 = state_c64(in);
  bass_trunc none{};
  none.k_cond = -1;
  cudaError_t e = run_merge_op(K_PERM, a, none, 0, 0, s);
  if (e != cudaSuccess) return status_of(e);
  // pass 2: groups of four (b_q1, b_q2), the rotation's drop rule
  OpArgs b{};
  b.in = tmp; b.out = out; b.ctrl = ctrl; b.ws = v; b.q = q1; b.gb = 1; b.drop_zero = 2; b.c64 = a.c64;
  load_G(b, host_U4, 16);
  e = run_merge_op(K_GATE2, b, tr, 0, 0, s);
  if (e == cudaSuccess && tr.trace) e = run_fingerprint(out, kSigPmin, nullptr, v, s, ctrl, 1, 1);
  return status_of(e);
}

int bass_rdm_2q(const bass_state* st, bass_state* tmp, int q1, int q2, double* rho, bass_ctrl* ctrl, void* ws,
                size_t ws_bytes, void* stream) {
  if (!st || !tmp || st == tmp || !rho || !ctrl || q1 < 0 || q2 < 0 || q1 >= BASS_MAX_QUBITS ||
      q2 >= BASS_MAX_QUBITS || q1 == q2)
    return BASS_ERR_ARG;
  CHECK_WS(ws, ws_bytes, v);
  return status_of(run_rdm_2q(st, tmp, q1, q2, rho, ctrl, v, (cudaStream_t)stream, state_c64(st)));
}

int bass_to_dense(const bass_state* st, const double* host_U, int nq, double* psi, bass_ctrl* ctrl, void* stream) {
  if (!st || !psi || !ctrl || nq < 1 || nq > 30) return BASS_ERR_ARG;
  return status_of(run_to_dense(st, host_U, nq, psi, ctrl, (cudaStream_t)stream));
}

int bass_dense_gate(double* psi, int nq, const double* host_G, int gate_qubits, int q1, int q2, void* stream) {
  if (!psi || !host_G || nq < 1 || nq > 34 || (gate_qubits != 1 && gate_qubits != 2) || q1 < 0 || q1 >= nq)
    return BASS_ERR_ARG;
  if (gate_qubits == 2 && (nq < 2 || q2 < 0 || q2 >= nq || q2 == q1)) return BASS_ERR_ARG;
  return status_of(run_dense_gate(psi, nq, host_G, gate_qubits, q1, q2, (cudaStream_t)stream));
}

int bass_dense_dot(const double* u, const double* v, int64_t n, double* out, bass_ctrl* ctrl, void* ws,
                   size_t ws_bytes, void* stream) {
  if (!u || !v || !out || !ctrl || n < 0) return BASS_ERR_ARG;
  CHECK_WS(ws, ws_bytes, w);
  return status_of(run_dot(u, v, n, nullptr, 64, out, ctrl, w, (cudaStream_t)stream));
}

int bass_sparse_dot(const bass_state* st, const double* psi, int nq, double* out, bass_ctrl* ctrl, void* ws,
                    size_t ws_bytes, void* stream) {
  if (!st || !psi || !out || !ctrl || nq < 1 || nq > 30) return BASS_ERR_ARG;
  CHECK_WS(ws, ws_bytes, w);
  return status_of(run_dot(psi, nullptr, 0, st, nq, out, ctrl, w, (cudaStream_t)stream));
}

int bass_phase_1q(bass_state* st, bass_state* tmp, const double* host_diag2, int q, bass_ctrl* ctrl,
                  void* ws, size_t ws_bytes, void* stream) {
  if (!st || !tmp || st == tmp || !host_diag2 || q < 0 || q >= BASS_MAX_QUBITS || !ctrl) return BASS_ERR_ARG;
  CHECK_WS(ws, ws_bytes, v);
  return status_of(run_phase1q(st, tmp, host_diag2, q, ctrl, v, (cudaStream_t)stream, state_c64(st)));
}

int bass_phase_2q(bass_state* st, const double* host_diag4, int q1, int q2, bass_ctrl* ctrl, void* stream) {
  if (!st || !host_diag4 || q1 < 0 || q2 < 0 || q1 >= BASS_MAX_QUBITS || q2 >= BASS_MAX_QUBITS || q1 == q2 ||
      !ctrl)
    return BASS_ERR_ARG;
  return status_of(run_phase2q(st, host_diag4, q1, q2, ctrl, (cudaStream_t)stream));
}

int bass_topk(const bass_state* in, bass_state* out, bass_trunc tr, bass_ctrl* ctrl, void* ws,
              size_t ws_bytes, void* stream) {
  if (!in || !out || in == out || !ctrl) return BASS_ERR_ARG;
  CHECK_WS(ws, ws_bytes, v);
  cudaStream_t s = (cudaStream_t)stream;
  OpArgs a{};
  a.in = in; a.out = out; a.ctrl = ctrl; a.ws = v; a.q = 0; a.gb = 0; a.c64 = state_c64(in);
  cudaError_t e = run_merge_op(K_IDENT, a, tr, 0, 0, s);
  if (e == cudaSuccess && tr.trace) e = run_fingerprint(out, kSigPmin, nullptr, v, s, ctrl, 1, 1);
  return status_of(e);
}

int bass_gather(const bass_state* in, bass_state* out, const int64_t* idx, int64_t n, bass_ctrl* ctrl,
                void* stream) {
  if (!in || !out || in == out || (n > 0 && !idx) || n < 0 || !ctrl) return BASS_ERR_ARG;
  return status_of(run_gather(in, out, idx, n, ctrl, (cudaStream_t)stream));
}

int bass_lcg_choose(int64_t nnz, int64_t k, int64_t seed, int64_t* host_idx) {
  if (nnz < 0 || k < 0 || k > nnz || (k > 0 && !host_idx)) return BASS_ERR_ARG;
  std::vector<int64_t> perm((size_t)nnz);
  for (int64_t i = 0; i < nnz; ++i) perm[(size_t)i] = i;
  int64_t rng = seed;
  for (int64_t i = 0; i < k; ++i) {
    rng = (1103515245LL * rng + 12345LL) & 0x7FFFFFFFLL;
    const int64_t r = i + (rng % (nnz - i));
    const int64_t t = perm[(size_t)i];
    perm[(size_t)i] = perm[(size_t)r];
    perm[(size_t)r] = t;
  }
  memcpy(host_idx, perm.data(), (size_t)k * sizeof(int64_t));
  return BASS_OK;
}

int bass_renorm(bass_state* st, int trace, bass_ctrl* ctrl, void* ws, size_t ws_bytes, void* stream) {
  if (!st || !ctrl) return BASS_ERR_ARG;
  CHECK_WS(ws, ws_bytes, v);
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = zero_small(v, s);
  if (e == cudaSuccess) e = run_renorm(st, ctrl, v, s);
  if (e == cudaSuccess && trace) e = run_fingerprint(st, kSigPmin, nullptr, v, s, ctrl, 1, 0);
  return status_of(e);
}

int bass_pr(const bass_state* st, bass_ctrl* ctrl, void* ws, size_t ws_bytes, void* stream) {
  if (!st || !ctrl) return BASS_ERR_ARG;
  CHECK_WS(ws, ws_bytes, v);
  return status_of(run_reduce(st, 1, nullptr, ctrl, v, (cudaStream_t)stream));
}

int bass_norm2(const bass_state* st, double* out, void* ws, size_t ws_bytes, void* stream) {
  if (!st || !out) return BASS_ERR_ARG;
  CHECK_WS(ws, ws_bytes, v);
  return status_of(run_reduce(st, 0, out, nullptr, v, (cudaStream_t)stream));
}

int bass_rdm_1q(const bass_state* st, int num_qubits, double* rho, bass_ctrl* ctrl, void* ws,
                size_t ws_bytes, void* stream) {
  if (!st || !rho || !ctrl || num_qubits < 1 || num_qubits > BASS_MAX_QUBITS) return BASS_ERR_ARG;
  CHECK_WS(ws, ws_bytes, v);
  return status_of(run_rdm(st, num_qubits, rho, ctrl, v, (cudaStream_t)stream, state_c64(st)));
}

int bass_rotate_step(bass_state* cur, bass_state* tmp, const double* host_U, int j, int64_t k, int trace,
                     bass_ctrl* ctrl, void* ws, size_t ws_bytes, void* stream) {
  if (!cur || !tmp || cur == tmp || !host_U || j < 0 || j >= 64 || k < 0 || !ctrl) return BASS_ERR_ARG;
  CHECK_WS(ws, ws_bytes, v);
  cudaStream_t s = (cudaStream_t)stream;
  OpArgs a{};
  a.in = cur; a.out = tmp; a.ctrl = ctrl; a.ws = v; a.q = j; a.gb = 0; a.c64 = state_c64(cur);
  load_G(a, host_U, 4);
  bass_trunc tr{};
  tr.k_cond = k;
  tr.k_keep = k;
  tr.trace = trace;
  // without a trace the write pass commits; with one, the candidate's
  // fingerprint comes first and k_commit follows it
  a.commit = trace ? 0 : 1;
  cudaError_t e = run_merge_op(K_ROT1, a, tr, 1, j, s);
  if (e == cudaSuccess && trace) e = run_fingerprint(tmp, kSigPmin, nullptr, v, s, ctrl, 1, 0);
  if (e == cudaSuccess && trace) e = run_commit(cur, tmp, ctrl, v, j, trace, s);
  return status_of(e);
}

int bass_fingerprint(const bass_state* st, double pmin, uint64_t* out6, void* ws, size_t ws_bytes,
                     void* stream) {
  if (!st || !out6) return BASS_ERR_ARG;
  CHECK_WS(ws, ws_bytes, v);
  return status_of(run_fingerprint(st, pmin, out6, v, (cudaStream_t)stream, nullptr, 0, 0));
}

int bass_radix_sort_u64(uint64_t* keys, double* amps, int64_t n, int key_bits, void* ws, size_t ws_bytes,
                        bass_ctrl* ctrl, void* stream) {
  if ((n > 0 && (!keys || !amps)) || n < 0 || key_bits < 1 || key_bits > 64) return BASS_ERR_ARG;
  CHECK_WS(ws, ws_bytes, v);
  if (n > v.max_n) return BASS_ERR_WORKSPACE;
  return status_of(run_radix_sort(keys, amps, n, nullptr, key_bits, v, ctrl, (cudaStream_t)stream, 0));
}

int bass_merge_sorted(uint64_t* keys, double* amps, int64_t n, int64_t* n_out, void* ws, size_t ws_bytes,
                      bass_ctrl* ctrl, void* stream) {
  if ((n > 0 && (!keys || !amps)) || n < 0 || !n_out || !ctrl) return BASS_ERR_ARG;
  CHECK_WS(ws, ws_bytes, v);
  if (n > v.max_n) return BASS_ERR_WORKSPACE;
  return status_of(run_merge_sorted(keys, amps, n, reinterpret_cast<long long*>(n_out), v, ctrl,
                                    (cudaStream_t)stream));
}

int64_t bass_launch_count(void) { return (int64_t)g_launches.load(); }

void bass_profile_enable(int on) { g_prof.store(on != 0); }

int bass_profile_collect(double* host_ms, int64_t* host_launches, int nslots) {
  if (nslots < 0 || (nslots > 0 && (!host_ms || !host_launches))) return BASS_ERR_ARG;
  for (int i = 0; i < nslots; ++i) { host_ms[i] = 0.0; host_launches[i] = 0; }
  std::lock_guard<std::mutex> lk(g_prof_mu);
  for (const ProfRec& r : g_recs) {
    if (cudaEventSynchronize(r.b) != cudaSuccess) return BASS_ERR_CUDA;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, r.a, r.b);
    if (r.slot >= 0 && r.slot < nslots) {
      host_ms[r.slot] += ms;
      host_launches[r.slot] += 1;
    }
    g_pool.push_back(r.a);
    g_pool.push_back(r.b);
  }
  g_recs.clear();
  return BASS_OK;
}

int bass_error(bass_ctrl* ctrl, void* stream) {
  if (!ctrl) return -1;
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaStreamSynchronize(s) != cudaSuccess) return 1 << BASS_ERR_CUDA;
  int32_t err = 0;
  if (cudaMemcpy(&err, &ctrl->error, sizeof err, cudaMemcpyDeviceToHost) != cudaSuccess) return 1 << BASS_ERR_CUDA;
  if (err) {
    const int32_t zero = 0;
    cudaMemcpy(&ctrl->error, &zero, sizeof zero, cudaMemcpyHostToDevice);
  }
  return err;
}

}  // extern "C"

// ---- batched (segmented) ops ---------------------------------------------------
namespace bass {
static size_t batch_ops_bytes(int max_ops) { return align256((size_t)max_ops * sizeof(OpArgs)); }

struct BatchView {
  SegPlan* plan;
  OpArgs* ops_a;
  OpArgs* ops_b;
};

static bool carve_batch(void* ws, size_t bytes, int n, BatchView* v) {
  if (!ws || ((uintptr_t)ws & 255) || n < 1 || n > kMaxSeg) return false;
  const size_t need = align256(sizeof(SegPlan)) + 2 * batch_ops_bytes(n);
  if (bytes < need) return false;
  char* b = static_cast<char*>(ws);
  v->plan = reinterpret_cast<SegPlan*>(b);
  v->ops_a = reinterpret_cast<OpArgs*>(b + align256(sizeof(SegPlan)));
  v->ops_b = reinterpret_cast<OpArgs*>(b + align256(sizeof(SegPlan)) + batch_ops_bytes(n));
  return true;
}

// The single-state op of one segment (the fields every kind shares); returns
// false if the segment's arguments are invalid.
static bool seg_common(const bass_seg_op& o, OpArgs* a) {
  *a = OpArgs{};
  if (!o.in || !o.ctrl || !carve(o.ws, o.ws_bytes, &a->ws)) return false;
  a->in = o.in;
  a->out = o.out;
  a->ctrl = o.ctrl;
  a->nsets = 1;
  a->fin = 1;
  a->k_cond = o.tr.k_cond;
  a->k_keep = o.tr.k_keep;
  a->tr = o.tr;
  a->tr.trace = 0;
  a->prof = prof_on() ? 1 : 0;
  a->c64 = state_c64(o.in);
  return true;
}

// Copies n ops to the device (the host array is pageable, so the copy is
// staged before this returns and the array may be reused at once).
static cudaError_t upload(OpArgs* dev, const std::vector<OpArgs>& host, cudaStream_t s) {
  return cudaMemcpyAsync(dev, host.data(), host.size() * sizeof(OpArgs), cudaMemcpyHostToDevice, s);
}

static int same_type(const std::vector<OpArgs>& v) {
  for (const OpArgs& a : v)
    if (a.c64 != v[0].c64) return 0;
  return 1;
}
}  // namespace bass

extern "C" {

int bass_batch_max_segments(void) {
  int n = 0;
  if (seg_max_segments(&n) != cudaSuccess) return 0;
  return n < kMaxSeg ? n : kMaxSeg;
}

size_t bass_batch_ws_bytes(int max_ops) {
  if (max_ops < 1) max_ops = 1;
  return align256(sizeof(SegPlan)) + 2 * batch_ops_bytes(max_ops);
}

#define BATCH_PROLOGUE()                                          \
  if (!ops || n < 1 || n > kMaxSeg) return BASS_ERR_ARG;          \
  BatchView bv;                                                   \
  if (!carve_batch(batch_ws, batch_ws_bytes, n, &bv)) return BASS_ERR_WORKSPACE; \
  cudaStream_t s = (cudaStream_t)stream;                          \
  std::vector<OpArgs> A((size_t)n);

int bass_gate_1q_batch(const bass_seg_op* ops, int n, void* batch_ws, size_t batch_ws_bytes, void* stream) {
  BATCH_PROLOGUE();
  for (int i = 0; i < n; ++i) {
    const bass_seg_op& o = ops[i];
    if (!seg_common(o, &A[i]) || !o.out || o.out == o.in || o.q1 < 0 || o.q1 >= BASS_MAX_QUBITS) return BASS_ERR_ARG;
    A[i].q = o.q1;
    load_G(A[i], o.G, 4);
  }
  if (!same_type(A)) return BASS_ERR_ARG;
  cudaError_t e = upload(bv.ops_a, A, s);
  if (e == cudaSuccess) e = run_merge_op_seg(K_GATE1, bv.ops_a, n, A[0].c64, 0, 0, bv.plan, s);
  return status_of(e);
}

int bass_gate_2q_batch(const bass_seg_op* ops, int n, void* batch_ws, size_t batch_ws_bytes, void* stream) {
  BATCH_PROLOGUE();
  std::vector<OpArgs> B((size_t)n);
  for (int i = 0; i < n; ++i) {
    const bass_seg_op& o = ops[i];
    if (!seg_common(o, &A[i]) || !o.tmp || !o.out || o.in == o.tmp || o.tmp == o.out || o.in == o.out ||
        o.q1 < 0 || o.q2 < 0 || o.q1 >= BASS_MAX_QUBITS || o.q2 >= BASS_MAX_QUBITS || o.q1 == o.q2)
      return BASS_ERR_ARG;
    B[i] = A[i];
    // pass 1: q2 to the lowest physical bit (a reorder, into tmp)
    A[i].out = o.tmp;
    A[i].q = o.q2;
    A[i].write_mode = 2;
    A[i].counter = 3;
    A[i].k_cond = -1;
    A[i].tr = bass_trunc{};
    A[i].tr.k_cond = -1;
    // pass 2: groups of four on q1 above it, from tmp
    B[i].in = o.tmp;
    B[i].q = o.q1;
    B[i].gb = 1;
    load_G(B[i], o.G, 16);
  }
  if (!same_type(A)) return BASS_ERR_ARG;
  cudaError_t e = upload(bv.ops_a, A, s);
  if (e == cudaSuccess) e = upload(bv.ops_b, B, s);
  if (e == cudaSuccess) e = run_merge_op_seg(K_PERM, bv.ops_a, n, A[0].c64, 0, 0, bv.plan, s);
  if (e == cudaSuccess) e = run_merge_op_seg(K_GATE2, bv.ops_b, n, A[0].c64, 0, 0, bv.plan, s);
  return status_of(e);
}

int bass_phase_2q_batch(const bass_seg_op* ops, int n, void* batch_ws, size_t batch_ws_bytes, void* stream) {
  BATCH_PROLOGUE();
  for (int i = 0; i < n; ++i) {
    const bass_seg_op& o = ops[i];
    if (!seg_common(o, &A[i]) || o.q1 < 0 || o.q2 < 0 || o.q1 >= BASS_MAX_QUBITS || o.q2 >= BASS_MAX_QUBITS ||
        o.q1 == o.q2)
      return BASS_ERR_ARG;
    A[i].q = o.q1;
    A[i].j = o.q2;
    load_G(A[i], o.G, 4);
  }
  if (!same_type(A)) return BASS_ERR_ARG;
  cudaError_t e = upload(bv.ops_a, A, s);
  if (e == cudaSuccess) e = run_phase2q_seg(bv.ops_a, n, A[0].c64, s);
  return status_of(e);
}

int bass_topk_batch(const bass_seg_op* ops, int n, void* batch_ws, size_t batch_ws_bytes, void* stream) {
  BATCH_PROLOGUE();
  for (int i = 0; i < n; ++i) {
    const bass_seg_op& o = ops[i];
    if (!seg_common(o, &A[i]) || !o.out || o.out == o.in) return BASS_ERR_ARG;
  }
  if (!same_type(A)) return BASS_ERR_ARG;
  cudaError_t e = upload(bv.ops_a, A, s);
  if (e == cudaSuccess) e = run_merge_op_seg(K_IDENT, bv.ops_a, n, A[0].c64, 0, 0, bv.plan, s);
  return status_of(e);
}

int bass_rotate_step_batch(const bass_seg_op* ops, int n, void* batch_ws, size_t batch_ws_bytes, void* stream) {
  BATCH_PROLOGUE();
  for (int i = 0; i < n; ++i) {
    const bass_seg_op& o = ops[i];
    if (!seg_common(o, &A[i]) || !o.tmp || o.tmp == o.in || o.q1 < 0 || o.q1 >= 64 || o.tr.k_keep < 0)
      return BASS_ERR_ARG;
    A[i].out = o.tmp;
    A[i].q = o.q1;
    A[i].j = o.q1;
    A[i].k_cond = o.tr.k_keep;
    A[i].k_keep = o.tr.k_keep;
    A[i].fin_mode = 1;
    A[i].commit = 1;
    load_G(A[i], o.G, 4);
  }
  if (!same_type(A)) return BASS_ERR_ARG;
  cudaError_t e = upload(bv.ops_a, A, s);
  if (e == cudaSuccess) e = run_merge_op_seg(K_ROT1, bv.ops_a, n, A[0].c64, 1, 0, bv.plan, s);
  return status_of(e);
}

int bass_rdm_1q_batch(const bass_seg_op* ops, int n, void* batch_ws, size_t batch_ws_bytes, void* stream) {
  BATCH_PROLOGUE();
  int max_nq = 1;
  for (int i = 0; i < n; ++i) {
    const bass_seg_op& o = ops[i];
    if (!seg_common(o, &A[i]) || !o.rho || o.num_qubits < 1 || o.num_qubits > BASS_MAX_QUBITS) return BASS_ERR_ARG;
    A[i].nsets = o.num_qubits;
    A[i].rho = o.rho;
    A[i].fin = 0;
    if (o.num_qubits > max_nq) max_nq = o.num_qubits;
  }
  if (!same_type(A)) return BASS_ERR_ARG;
  cudaError_t e = upload(bv.ops_a, A, s);
  if (e == cudaSuccess) e = run_rdm_seg(bv.ops_a, n, max_nq, A[0].c64, bv.plan, s);
  return status_of(e);
}

int bass_pr_batch(const bass_seg_op* ops, int n, int mode, void* batch_ws, size_t batch_ws_bytes, void* stream) {
  BATCH_PROLOGUE();
  if (mode != 0 && mode != 1) return BASS_ERR_ARG;
  for (int i = 0; i < n; ++i)
    if (!seg_common(ops[i], &A[i])) return BASS_ERR_ARG;
  if (!same_type(A)) return BASS_ERR_ARG;
  cudaError_t e = upload(bv.ops_a, A, s);
  if (e == cudaSuccess) e = run_reduce_seg(bv.ops_a, n, mode, A[0].c64, s);
  return status_of(e);
}

}  // extern "C"
