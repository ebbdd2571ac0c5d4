// internal.h -- host-side launchers shared by the .cu files of libbass_b200.
#pragma once

#include <atomic>
#include <mutex>
#include <utility>
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace bass {

enum Kind { K_GATE1 = 0, K_ROT1 = 1, K_GATE2 = 2, K_PERM = 3, K_IDENT = 4, K_RDM = 5 };
enum Pass { P_HIST = 0, P_HIST2 = 1, P_GATHER = 2, P_WRITE = 3, P_RDM = 4 };

// Op description passed by value to every tile kernel.
struct OpArgs {
  const bass_state* in;
  bass_state* out;
  bass_ctrl* ctrl;
  WsView ws;
  double2 G[16];
  int q;          // qubit whose physical bit is the merge target (K_RDM: first set)
  int gb;         // pregrouped low bits (0, or 1 for the second pass of a 2-qubit gate)
  int nsets;      // K_RDM: number of qubits; otherwise 1
  int counter;    // tile-counter slot
  int drop_zero;  // K_IDENT: drop entries whose amplitude is exactly zero
  int guard;      // K_IDENT: run only if ws.sel->pad (zero flag) is set
  int prof;       // count entries into ctrl->prof_in / prof_out
  int write_mode; // P_WRITE: 0 look-back + drop rule, 2 one child per entry
  int fin;        // P_WRITE: the last CTA to finish writes the output descriptor (finalize_op)
  int fin_mode;   // finalize_op: 0 gate / truncation, 1 rotation step
  int commit;     // rotation step: the last CTA of the write pass also commits (swaps in an accepted candidate)
  int j;          // rotation step: the rotated qubit
  long long k_cond, k_keep;
  bass_trunc tr;  // finalize_op: gamma / renormalisation rules
  int c64;        // the input state stores complex64 amplitudes (selects the kernels)
  int rdm_low;    // K_RDM: the qubits at physical bits below kRdmLowBits are left to k_rdm_low
  double* rho;    // RDM moments of a segmented RDM (4 per qubit)
};

// Segmented launches: one op on each of up to kMaxSeg states in one launch.
// The grid is split into one block group per state, sized by the state's
// share of the op's work (every state gets at least one block).
constexpr int kMaxSeg = 1024;
struct SegPlan {
  int nseg;
  int kind;
  long long wp[kMaxSeg + 1];  // exclusive prefix of the states' work weights
};

enum Slot {
  S_PARTITION = 30, S_SELECT1 = 31, S_SELECT2 = 32, S_SELECT_EXACT = 33, S_FINALIZE = 34, S_REDUCE = 35,
  S_FINGERPRINT = 36, S_PHASE2Q = 37, S_PHASE1Q = 38, S_RDM_FINAL = 39, S_SORT = 40, S_MERGE_RUNS = 41,
  S_SMALL = 42, S_SLOT_HIST1 = 43, S_SLOT_HIST2 = 44, S_SLOT_GATHER = 45, S_SLOT_KEPT = 46
};

// Brackets one kernel launch: counts it and, when profiling is on, records
// CUDA events around it on its stream.
struct ProfScope {
  ProfScope(int slot, cudaStream_t s);
  ~ProfScope();
  int slot;
  cudaStream_t stream;
  cudaEvent_t start;
  bool on;
};
bool prof_on();
#define KLAUNCH(slot, stream, ...)        \
  do {                                    \
    ::bass::ProfScope _ps((slot), (stream)); \
    __VA_ARGS__;                          \
  } while (0)

// Launch with programmatic dependent launch: the grid may be scheduled while
// the previous kernel of the stream finishes (after every block of that
// kernel has called pdl_trigger or exited).  The kernel must call pdl_wait
// before it touches any memory, so only the launch itself overlaps.
template <typename... K, typename... A>
inline cudaError_t launch_pdl(void (*kern)(K...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              A&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, std::forward<A>(args)...);
}

struct Device {
  int sms;
  int grid_tile;    // persistent grid of the tile kernels
  int grid_tile_h;  // ... of the histogram passes (more shared memory)
  int grid_small;
};
// The current device's properties (looked up once per device).
const Device& device();

// A launch-configuration value (a kernel's resident grid) worked out once per
// device: it depends only on the device, so racing first computations store
// the same value.
constexpr int kMaxDevices = 64;
struct PerDevice {
  std::atomic<int> v[kMaxDevices];
};
template <typename F>
inline cudaError_t per_device(PerDevice& c, int* out, F compute) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return compute(out);
  int x = c.v[dev].load(std::memory_order_acquire);
  if (x == 0) {
    if ((e = compute(&x)) != cudaSuccess) return e;
    c.v[dev].store(x, std::memory_order_release);
  }
  *out = x;
  return cudaSuccess;
}

bool carve(void* ws, size_t ws_bytes, WsView* v);
// 1 if the state was set up (bass_state_init_typed / import / copy_desc) with
// complex64 amplitudes: the host's record of each descriptor's type, which
// selects the kernels to launch (the kernels check the descriptor's own field)
int state_c64(const bass_state* st);
size_t ws_bytes_for(long long max_n);

// merge.cu
cudaError_t run_merge_op(int kind, OpArgs a, const bass_trunc& tr, int finalize_mode, int j,
                         cudaStream_t s);
cudaError_t run_rdm(const bass_state* st, int nq, double* rho, bass_ctrl* ctrl, const WsView& ws,
                    cudaStream_t s, int c64);
cudaError_t zero_small(const WsView& ws, cudaStream_t s);
cudaError_t run_to_dense(const bass_state* st, const double* host_U, int nq, double* psi, bass_ctrl* ctrl,
                         cudaStream_t s);
cudaError_t run_dot(const double* u, const double* v, long long n, const bass_state* st, int nq, double* out,
                    bass_ctrl* ctrl, const WsView& ws, cudaStream_t s);
cudaError_t run_rdm_2q(const bass_state* st, bass_state* tmp, int q1, int q2, double* rho, bass_ctrl* ctrl,
                       const WsView& ws, cudaStream_t s, int c64);
cudaError_t run_rdm_prepared(const bass_state* st, int nq, double* rho, bass_ctrl* ctrl, const WsView& ws,
                             cudaStream_t s, int c64);
cudaError_t run_ident_write(OpArgs a, cudaStream_t s);
// rotation step: keep the candidate in *tmp if the decision accepted it
cudaError_t run_commit(bass_state* cur, bass_state* tmp, bass_ctrl* ctrl, const WsView& ws, int j, int trace,
                       cudaStream_t s);

// merge.cu, segmented: ops_dev holds nseg OpArgs (all of one amplitude type),
// plan_dev is scratch for the block groups
cudaError_t run_merge_op_seg(int kind, const OpArgs* ops_dev, int nseg, int c64, int fin_mode, int trace,
                             SegPlan* plan_dev, cudaStream_t s);
cudaError_t run_rdm_seg(const OpArgs* ops_dev, int nseg, int max_nq, int c64, SegPlan* plan_dev, cudaStream_t s);
// the most segments one segmented launch takes on the current device
cudaError_t seg_max_segments(int* out);
// misc.cu, segmented: diagonal 2-qubit phases; PR (mode 1) or renormalisation (mode 0)
cudaError_t run_phase2q_seg(const OpArgs* ops_dev, int nseg, int c64, cudaStream_t s);
cudaError_t run_reduce_seg(const OpArgs* ops_dev, int nseg, int mode, int c64, cudaStream_t s);

// misc.cu
struct DenseG4 {
  double2 m[16];
};
cudaError_t run_dense_gate(double* psi, int nq, const double* host_G, int nqg, int q1, int q2, cudaStream_t s);
cudaError_t run_reduce(const bass_state* st, int mode, double* dest, bass_ctrl* ctrl,
                       const WsView& ws, cudaStream_t s);
cudaError_t run_fingerprint(const bass_state* st, double pmin, uint64_t* out6, const WsView& ws,
                            cudaStream_t s, bass_ctrl* ctrl, int append_event, int only_if_trunc);
cudaError_t run_radix_sort(uint64_t* keys, double* amps, long long n, const long long* n_dev,
                           int key_bits, const WsView& ws, bass_ctrl* ctrl, cudaStream_t s, int c64);
cudaError_t run_renorm(bass_state* st, bass_ctrl* ctrl, const WsView& ws, cudaStream_t s);
cudaError_t run_phase2q(bass_state* st, const double* d, int q1, int q2, bass_ctrl* ctrl, cudaStream_t s);
cudaError_t run_phase1q(bass_state* st, bass_state* tmp, const double* g, int q, bass_ctrl* ctrl,
                        const WsView& ws, cudaStream_t s, int c64);
cudaError_t run_state_init(bass_state* st, uint64_t* keys, double* amps, long long cap, int nq,
                           uint64_t key, int amp_type, cudaStream_t s);
cudaError_t run_import(bass_state* st, const uint64_t* keys, const double* amps, long long n, int nq,
                       const WsView& ws, bass_ctrl* ctrl, cudaStream_t s, uint64_t* st_keys,
                       double* st_amps, long long cap, int amp_type);
cudaError_t run_export(const bass_state* st, uint64_t* ok, double* oa, int key_bits, const WsView& ws,
                       bass_ctrl* ctrl, cudaStream_t s, int amp_type);
cudaError_t run_merge_sorted(uint64_t* keys, double* amps, long long n, long long* n_out,
                             const WsView& ws, bass_ctrl* ctrl, cudaStream_t s);
cudaError_t run_clone(bass_state* dst, const bass_state* src, bass_ctrl* ctrl, cudaStream_t s);
cudaError_t run_copy_desc(bass_state* dst, const bass_state* src, cudaStream_t s);
cudaError_t run_gather(const bass_state* in, bass_state* out, const int64_t* idx, long long n,
                       bass_ctrl* ctrl, cudaStream_t s);
cudaError_t run_ctrl_init(bass_ctrl* c, uint64_t* trace, long long cap, double tol, cudaStream_t s);

constexpr double kSigPmin = 1e-24;  // |a|^2 threshold of the significant-key fingerprint

constexpr int kSmallWords = 64 /*counters*/ + 2 * kHistBins;  // zeroed at the start of every op

}  // namespace bass
