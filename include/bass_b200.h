/*
 * bass_b200.h -- C ABI of libbass_b200.so, the B200 (sm_100a) kernels of the
 * BASS sparse-state simulation hot path.
 *
 * The reference (Skill0issue/BASS-Basis-Adapative-Sparse-Simulations-) has no
 * FFI: its boundary is the Python API of SparseState / BASS /
 * FixedBasisSimulator over Numba kernels that take caller-owned numpy arrays
 * and return counts.  Every entry point below replaces one of those kernels
 * (or one step of the Python driver around them) and names it.  Conventions:
 *
 *   - all pointers are device pointers unless the name says host_;
 *   - nothing here allocates: buffers, the workspace and the state / control
 *     descriptors are allocated by the caller (bass_*_bytes give the sizes);
 *   - every call is asynchronous on the given CUDA stream (cudaStream_t passed
 *     as void*; NULL = legacy default stream) and returns a status code; device
 *     side failures (capacity, a bounded wait that gave up) are recorded in
 *     bass_ctrl.error and read back with bass_error();
 *   - calls that share a workspace or a control block must be ordered (same
 *     stream); the library is otherwise reentrant.
 *
 * State representation.  A state is a bass_state descriptor in device memory
 * pointing at two caller-owned arrays of capacity cap: keys (uint64) and amps
 * (complex128, interleaved re/im).  Keys are stored in a permuted bit order:
 * physical bit p holds qubit qat[p] (pos[] is the inverse), and the array is
 * sorted ascending by physical key with no duplicates.  A state stores
 * complex128 or complex64 amplitudes (amp_type); every entry point reads the
 * type from the descriptor, except the few whose host arrays must have it
 * (the _typed set-up, import and export calls).  Every pairing kernel
 * moves the qubits it acts on to the lowest physical bits, so a gate's
 * partners always meet in one merge pass.  A stored amplitude is multiplied
 * by rscale[0] and then by rscale[1] on every read: a renormalisation is
 * recorded there instead of rewriting the array (numpy's a /= norm computes
 * a * (1/norm), which this reproduces exactly).
 */
#ifndef BASS_B200_H
#define BASS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define BASS_OK 0
#define BASS_ERR_CAPACITY 1  /* an output did not fit its buffer            */
#define BASS_ERR_WAIT 2      /* a bounded device wait gave up                */
#define BASS_ERR_ARG 3       /* invalid argument                             */
#define BASS_ERR_CUDA 4      /* a CUDA runtime call failed                   */
#define BASS_ERR_WORKSPACE 5 /* workspace too small for the request          */

#define BASS_MAX_QUBITS 63

/* amplitude storage of a state (bass_state.amp_type) */
#define BASS_AMP_C128 0 /* complex128: interleaved double re, im                 */
#define BASS_AMP_C64 1  /* complex64: interleaved float re, im (amps points at
                           floats); gate arithmetic in FP32 with compensated
                           (error-free) products and sums, while |a|^2, every
                           sum, the top-k threshold and the RDM moments stay in
                           FP64 */

/* ---- device-resident descriptors (layout is part of the ABI) ------------- */
typedef struct bass_state {
  uint64_t* keys;     /* physical keys, sorted ascending, unique            */
  double* amps;       /* interleaved complex128                              */
  int64_t nnz;        /* number of valid entries                             */
  int64_t cap;        /* capacity of keys/amps                               */
  double rscale[2];   /* pending renormalisation factors (1.0 = none)        */
  int32_t nq;         /* number of qubits                                    */
  int32_t amp_type;   /* BASS_AMP_C128 or BASS_AMP_C64 (storage of amps)     */
  int8_t pos[64];     /* pos[q]: physical bit of qubit q                     */
  int8_t qat[64];     /* qat[p]: qubit stored at physical bit p              */
} bass_state;

#define BASS_TRACE_WORDS 7 /* u64 per trace event, see bass_ctrl.trace */
/* Kernel slots of the profiler: 0..29 are the tile kernels (kind * 5 + pass,
   kind: 0 gate1, 1 rot1, 2 gate2, 3 perm, 4 plain, 5 rdm; pass: 0 evaluation,
   3 write (the compaction for gate, rotation and truncation kinds), 4 moments;
   passes 1 and 2 are unused), then 30 partition, 31 selection (one launch),
   35 reductions (norm, PR, dot products, the traced rotation commit),
   36 fingerprint, 37 phase2q, 38 phase1q, 39 rdm_final, 40 radix sort,
   41 merge runs, 42 small bookkeeping kernels (dense statevectors among
   them).  Slots 32-34 and 43-47 are unused and keep the numbering stable. */
#define BASS_PROF_SLOTS 48

typedef struct bass_ctrl {
  double gamma_running;   /* BASS._gamma_running                              */
  double state_gamma;     /* SparseState.gamma                                */
  double pr_cur;          /* running PR of the current optimisation pass       */
  double pr_last;         /* last PR computed by bass_pr                       */
  double last_kept;       /* kept |a|^2 mass of the last truncation            */
  double last_total;      /* total |a|^2 mass seen by the last truncation      */
  int32_t truncation_active;
  int32_t gates_since_trunc;
  int32_t error;          /* sticky BASS_ERR_* bits (1 << code)                */
  int32_t last_truncated; /* 1 if the last op truncated                        */
  int64_t amp_updates;    /* sum of input entries over all applied ops         */
  int64_t n_trunc;        /* truncations performed                             */
  int64_t n_ops;
  int32_t accept[64];     /* per-qubit decision of the current pass            */
  double frac[64];        /* retained mass of each attempted rotation          */
  uint64_t* trace;        /* optional event log (BASS_TRACE_WORDS per event)   */
  int64_t trace_cap;
  int64_t trace_len;
  double pr_tie_tol;      /* a rotation must lower PR by more than this (rel.) */
  uint32_t sync_counter;  /* last-block bookkeeping of in-place kernels        */
  int32_t wait_limit;     /* spins of a bounded device wait before it gives up:
                             0 the default (2^22), > 0 that many, < 0 none (a
                             wait that is not already satisfied gives up at once;
                             for tests of the give-up path)                      */
  int64_t prof_in[BASS_PROF_SLOTS];   /* entries read per kernel slot (profiling on) */
  int64_t prof_out[BASS_PROF_SLOTS];  /* entries written per kernel slot            */
} bass_ctrl;

/* Truncation request attached to an op (passed by value).  The op truncates
   when its output count exceeds k_cond (k_cond < 0: never), keeping the k_keep
   entries of largest |a|^2, ties broken by smaller (true) key. */
typedef struct bass_trunc {
  int64_t k_cond;
  int64_t k_keep;
  int32_t gamma_mode;   /* 0 none; 1 gamma_running *= kept/total (BASS.simulate);
                           2 state_gamma *= sqrt(kept/total) (FixedBasisSimulator);
                           3 state_gamma *= sqrt(kept) (SparseState.truncate_top_k) */
  int32_t renorm;       /* 0 none; 1 renormalise if norm > 1e-30; 2 unconditionally */
  int32_t mark_active;  /* set truncation_active, reset gates_since_trunc      */
  int32_t trace;        /* append a renorm event to the trace when truncating  */
} bass_trunc;

/* ---- sizes --------------------------------------------------------------- */
size_t bass_state_bytes(void);
size_t bass_ctrl_bytes(void);
/* workspace for ops whose inputs hold at most max_in entries and whose
   outputs at most max_out entries (before truncation); it is sized for
   max(4 * max_in, max_out) entries, since the evaluation pass of a 2-qubit
   gate keeps four 8-byte |a|^2 slots per input entry */
size_t bass_workspace_bytes(int64_t max_in, int64_t max_out, int num_qubits);

/* ---- state management ----------------------------------------------------- */
/* Every key array is 8-byte aligned and every amplitude array 16-byte
   (complex128) or 8-byte (complex64) aligned, as every cudaMalloc'd or torch
   buffer is; init, import and export refuse other arrays with BASS_ERR_ARG
   before touching the GPU.  Tile loads take TMA bulk copies where both arrays
   of a state are 16-byte aligned, per-entry copies otherwise. */
/* SparseState.__init__ (sparse_state.py:202-219): |init_key>, amplitude 1. */
int bass_state_init(bass_state* st, uint64_t* keys, double* amps, int64_t cap, int num_qubits,
                    uint64_t init_key, void* stream);
/* bass_state_init for a state of the given amplitude storage (BASS_AMP_*);
   amps then holds cap complex values of that type. */
int bass_state_init_typed(bass_state* st, uint64_t* keys, double* amps, int64_t cap, int num_qubits,
                          uint64_t init_key, int amp_type, void* stream);
/* Build a state in the buffers (st_keys, st_amps, capacity cap) from n
   entries (true keys, amps) in any order: radix sort by key, then duplicates
   are merged as sparse_state.py:127-147 does; identity bit order. */
int bass_state_import_into(bass_state* st, uint64_t* st_keys, double* st_amps, int64_t cap,
                           const uint64_t* keys, const double* amps, int64_t n, int num_qubits,
                           void* ws, size_t ws_bytes, bass_ctrl* ctrl, void* stream);
/* bass_state_import_into for a state of the given amplitude storage: amps
   and st_amps hold values of that type; duplicates of complex64 states are
   summed in FP32 with the compensated (TwoSum) sum. */
int bass_state_import_typed(bass_state* st, uint64_t* st_keys, double* st_amps, int64_t cap,
                            const uint64_t* keys, const double* amps, int64_t n, int num_qubits, int amp_type,
                            void* ws, size_t ws_bytes, bass_ctrl* ctrl, void* stream);
/* Write the state as true keys sorted ascending and amplitudes with the
   pending renormalisation applied (SparseState.x / .alpha); st->nnz entries.
   _bits sorts on the low key_bits bits only (keys < 2^num_qubits). */
int bass_state_export(const bass_state* st, uint64_t* out_keys, double* out_amps, void* ws,
                      size_t ws_bytes, bass_ctrl* ctrl, void* stream);
int bass_state_export_bits(const bass_state* st, uint64_t* out_keys, double* out_amps, int key_bits,
                           void* ws, size_t ws_bytes, bass_ctrl* ctrl, void* stream);
/* bass_state_export_bits for a state of the given amplitude storage (out_amps
   holds values of that type); a state of another type is refused on the
   device (BASS_ERR_ARG in ctrl, nothing written). */
int bass_state_export_typed(const bass_state* st, uint64_t* out_keys, double* out_amps, int key_bits,
                            int amp_type, void* ws, size_t ws_bytes, bass_ctrl* ctrl, void* stream);
/* Copy descriptor contents (pointers included) from src to dst. */
int bass_state_copy_desc(bass_state* dst, const bass_state* src, void* stream);
/* Deep copy of entries into dst's own buffers (SparseState.copy). */
int bass_state_clone(bass_state* dst, const bass_state* src, bass_ctrl* ctrl, void* stream);
int bass_ctrl_init(bass_ctrl* ctrl, uint64_t* trace, int64_t trace_cap, double pr_tie_tol, void* stream);

/* ---- gates ------------------------------------------------------------------ */
/* Non-diagonal 1-qubit gate: sparse_state.py:15-67 (expansion, exact-zero
   children dropped) + :150-172 / :127-147 (sort + merge of duplicates) +
   optional truncation.  G: 2x2 complex128 row-major, host pointer. */
int bass_gate_1q(const bass_state* in, bass_state* out, const double* host_G, int q,
                 bass_trunc tr, bass_ctrl* ctrl, void* ws, size_t ws_bytes, void* stream);
/* Non-diagonal 2-qubit gate: bass_simulator.py:292-354 apply_2qubit_gate_ht
   (also SparseState.apply_two_qubit_gate, sparse_state.py:303-377) + optional
   truncation.  Uses tmp as scratch state.  G: 4x4 complex128, index
   (bit_q1 << 1) | bit_q2, host pointer. */
int bass_gate_2q(const bass_state* in, bass_state* tmp, bass_state* out, const double* host_G,
                 int q1, int q2, bass_trunc tr, bass_ctrl* ctrl, void* ws, size_t ws_bytes,
                 void* stream);
/* 2-qubit basis rotation: bass_simulator.py:237-289
   apply_2qubit_rotation_sparse (used by the brick-wall pair passes,
   :679-728) + optional truncation.  As bass_gate_2q, but a child is kept when
   |a| > 1e-30 (the rotation's drop rule).  U4: 4x4 complex128, index
   (bit_q1 << 1) | bit_q2, host pointer.  Output key-sorted. */
int bass_rotate_2q(const bass_state* in, bass_state* tmp, bass_state* out, const double* host_U4,
                   int q1, int q2, bass_trunc tr, bass_ctrl* ctrl, void* ws, size_t ws_bytes,
                   void* stream);
/* Diagonal 1-qubit gate in place (g01 = g10 = 0): children of the reference's
   1-qubit kernel that are exactly zero are dropped (compacts only if one is). */
int bass_phase_1q(bass_state* st, bass_state* tmp, const double* host_diag2, int q, bass_ctrl* ctrl,
                  void* ws, size_t ws_bytes, void* stream);
/* sparse_state.py:178-190 apply_2qubit_diagonal_kernel, in place. */
int bass_phase_2q(bass_state* st, const double* host_diag4, int q1, int q2, bass_ctrl* ctrl,
                  void* stream);

/* ---- truncation -------------------------------------------------------------- */
/* truncation.py:68-113 top_k_truncate_kernel_opt, bass_simulator.py:899-916
   (simulate-level), :565-572 (_truncate_state), simulator.py:170-201. */
int bass_topk(const bass_state* in, bass_state* out, bass_trunc tr, bass_ctrl* ctrl, void* ws,
              size_t ws_bytes, void* stream);
/* Keep the entries at the given (device) indices, which must be ascending so
   that the output stays sorted (truncation.py:116-159 random_k and the
   np.random.choice path of simulator.py:178-186 choose the indices). */
int bass_gather(const bass_state* in, bass_state* out, const int64_t* idx, int64_t n,
                bass_ctrl* ctrl, void* stream);
/* truncation.py:116-159: the LCG partial Fisher-Yates of random_k_truncate,
   run on the host; writes the k chosen indices (permutation order) to
   host_idx.  Needs O(nnz) host memory. */
int bass_lcg_choose(int64_t nnz, int64_t k, int64_t seed, int64_t* host_idx);

/* ---- statistics ------------------------------------------------------------ */
/* bass_simulator.py:551-554 _renorm: records 1/sqrt(sum |a|^2) if > 1e-30. */
int bass_renorm(bass_state* st, int trace, bass_ctrl* ctrl, void* ws, size_t ws_bytes, void* stream);
/* bass_simulator.py:574-578 _pr: ctrl->pr_last = 1 / sum |a|^4 (inf if empty). */
int bass_pr(const bass_state* st, bass_ctrl* ctrl, void* ws, size_t ws_bytes, void* stream);
/* sum |a|^2 into *out (device double). */
int bass_norm2(const bass_state* st, double* out, void* ws, size_t ws_bytes, void* stream);
/* bass_simulator.py:441-470 compute_all_1qubit_rdms: rho[4q..4q+3] =
   (rho00, rho11, Re rho01, Im rho01), device doubles. */
int bass_rdm_1q(const bass_state* st, int num_qubits, double* rho, bass_ctrl* ctrl, void* ws,
                size_t ws_bytes, void* stream);
/* bass_simulator.py:200-231 compute_2qubit_rdm for the qubit pair (q1, q2),
   index (bit_q1 << 1) | bit_q2, rho[p][q] = sum over groups of a_p conj(a_q),
   exact sums.  rho: 16 device doubles, (rho00, rho11, rho22, rho33,
   Re/Im rho01, Re/Im rho02, Re/Im rho03, Re/Im rho12, Re/Im rho13,
   Re/Im rho23); the lower triangle is the conjugate.  tmp is scratch. */
int bass_rdm_2q(const bass_state* st, bass_state* tmp, int q1, int q2, double* rho, bass_ctrl* ctrl,
                void* ws, size_t ws_bytes, void* stream);
/* bass_simulator.py:608-621 to_statevector on the device: psi (2^nq
   complex128, device) = the state at its true keys (pending scale applied),
   then each frame U_j applied to logical qubit j in order (host_U: nq 2x2
   complex128 row-major; NULL for no frames).  nq <= 30; a key of more
   qubits than nq sets BASS_ERR_ARG and is skipped. */
int bass_to_dense(const bass_state* st, const double* host_U, int nq, double* psi, bass_ctrl* ctrl,
                  void* stream);
/* exact_simulator.py:114-144 ExactSimulator._apply_1qubit_dense /
   _apply_2qubit_dense: a gate applied in place to a dense statevector psi
   (2^nq complex128, device, nq <= 34).  gate_qubits 1: host_G is 2x2 on qubit
   q1 (q2 ignored); 2: host_G is 4x4, index (bit_q1 << 1) | bit_q2.  Each
   output is a sum over input indices in ascending order, without FMA. */
int bass_dense_gate(double* psi, int nq, const double* host_G, int gate_qubits, int q1, int q2, void* stream);
/* runner.py:620-626 np.vdot(u, v) of two device complex128 vectors of n
   entries: out[0..1] = sum conj(u_i) v_i, exact sums (device doubles). */
int bass_dense_dot(const double* u, const double* v, int64_t n, double* out, bass_ctrl* ctrl, void* ws,
                   size_t ws_bytes, void* stream);
/* fidelity.py:48-68 compute_fidelity's overlap: out[0..1] = sum over the
   state's entries of conj(psi[x]) a_x (psi: dense 2^nq complex128, device). */
int bass_sparse_dot(const bass_state* st, const double* psi, int nq, double* out, bass_ctrl* ctrl, void* ws,
                    size_t ws_bytes, void* stream);
/* bass_rdm_1q for callers that cannot allocate device memory (a host runtime
   that owns all device memory, a plugin or embedding that may only pass the
   buffers it was given, code that may not call cudaMalloc at that point).  No counterpart in
   the reference.  The scratch is a static array inside the library (about
   4.8 MB, held on every GPU that loads the library until exit); the state may
   hold at most 2^20 entries (max_entries is the caller's bound on st->nnz;
   larger values return BASS_ERR_WORKSPACE).  A state that does not fit the
   scratch although max_entries said it would (more than 516 merge tiles,
   about 1,052,640 entries) is refused on the device: the call returns
   BASS_OK, ctrl->error gets BASS_ERR_WORKSPACE and rho gets NaN.  All calls
   share the array, so calls that may overlap on the GPU race and must be
   serialised.  The first call on a device looks up the array's address (a
   runtime query, cudaGetSymbolAddress); the address is kept for the life of
   the process: it does not survive cudaDeviceReset.  Allocates nothing. */
int bass_rdm_1q_noalloc(const bass_state* st, int64_t max_entries, int num_qubits, double* rho,
                        bass_ctrl* ctrl, void* stream);
/* One coordinate-descent step of bass_simulator.py:755-814: rotate qubit j of
   *cur by host_U (2x2) into *tmp (bass_simulator.py:156-199), keep the top k
   (:565-572), renormalise (:551-554), compare PR with ctrl->pr_cur and keep the
   rotated state (swapping the contents of *cur and *tmp) only if it lowers PR
   by more than ctrl->pr_tie_tol.  Records ctrl->accept[j], ctrl->frac[j].
   The candidate's PR is frac^2 / sum |a|^4 over the kept children (exact
   sums), decided before the candidate is written: a rejected candidate is
   written to *tmp only when trace != 0 (its fingerprint goes to the trace). */
int bass_rotate_step(bass_state* cur, bass_state* tmp, const double* host_U, int j, int64_t k,
                     int trace, bass_ctrl* ctrl, void* ws, size_t ws_bytes, void* stream);
/* Order-independent key-set fingerprints of a state: out[0..2] over all keys,
   out[3..5] over keys with |a|^2 > pmin (count, sum fmix64, xor fmix64). */
int bass_fingerprint(const bass_state* st, double pmin, uint64_t* out6, void* ws, size_t ws_bytes,
                     void* stream);

/* ---- array-level kernels (the reference's Numba kernels on plain arrays) --- */
/* sparse_state.py:150-172 radix_sort_uint64: stable sort of n (key, amp) pairs
   on the low key_bits bits; in place (uses the workspace). */
int bass_radix_sort_u64(uint64_t* keys, double* amps, int64_t n, int key_bits, void* ws,
                        size_t ws_bytes, bass_ctrl* ctrl, void* stream);
/* sparse_state.py:127-147 merge_sorted_kernel: merge adjacent equal keys of a
   sorted array in place; the new count is written to *n_out (device). */
int bass_merge_sorted(uint64_t* keys, double* amps, int64_t n, int64_t* n_out, void* ws,
                      size_t ws_bytes, bass_ctrl* ctrl, void* stream);

/* ---- batched (segmented) ops ------------------------------------------------------ */
/* One op on each of n independent states in one set of launches: every
   kernel's grid is split into one block group per state, sized by the
   state's share of the work (each state gets at least one block), and each
   group runs the single-state algorithm on its state (own descriptor,
   control block and workspace).  This is the "segment offset" form of the
   calls above: the host array describes the segments, the library copies it
   into the batch workspace (bass_batch_ws_bytes) and launches once per pass
   for all of them.  All states of one call must have the same amplitude type;
   n <= 256 for ops that truncate or rotate (their selection keeps every block
   of the grid resident).  No counterpart in the reference, whose simulators
   run one state at a time. */
typedef struct bass_seg_op {
  bass_state* in;    /* input state (rotation step: the current state)         */
  bass_state* tmp;   /* scratch state of 2-qubit ops; a rotation's candidate   */
  bass_state* out;   /* output state                                          */
  bass_ctrl* ctrl;   /* this state's control block                            */
  void* ws;          /* this state's workspace                                */
  size_t ws_bytes;
  double G[32];      /* 2x2 (first 8 doubles) or 4x4 complex128, row-major     */
  int32_t q1, q2;    /* gate qubits; a rotation step's qubit j is q1           */
  bass_trunc tr;     /* truncation (rotation step: k = tr.k_keep)              */
  double* rho;       /* RDM: 4 device doubles per qubit                        */
  int32_t num_qubits;/* RDM: qubits of this state                              */
  int32_t pad;
} bass_seg_op;
size_t bass_batch_ws_bytes(int max_ops);
/* The most states one segmented call takes on the current device (a call's
   selection keeps one block group per state resident; no counterpart in the
   reference, which has no batched path).  0 if no device. */
int bass_batch_max_segments(void);
/* bass_gate_1q on every segment (sparse_state.py:15-67 + truncation) */
int bass_gate_1q_batch(const bass_seg_op* host_ops, int n, void* batch_ws, size_t batch_ws_bytes, void* stream);
/* bass_gate_2q on every segment (bass_simulator.py:292-354 + truncation) */
int bass_gate_2q_batch(const bass_seg_op* host_ops, int n, void* batch_ws, size_t batch_ws_bytes, void* stream);
/* bass_phase_2q on every segment (sparse_state.py:178-190); diag = G[0..7] */
int bass_phase_2q_batch(const bass_seg_op* host_ops, int n, void* batch_ws, size_t batch_ws_bytes, void* stream);
/* bass_topk on every segment (truncation.py:68-113) */
int bass_topk_batch(const bass_seg_op* host_ops, int n, void* batch_ws, size_t batch_ws_bytes, void* stream);
/* bass_rotate_step on every segment (bass_simulator.py:755-814), no trace */
int bass_rotate_step_batch(const bass_seg_op* host_ops, int n, void* batch_ws, size_t batch_ws_bytes,
                           void* stream);
/* bass_rdm_1q on every segment (bass_simulator.py:441-470) */
int bass_rdm_1q_batch(const bass_seg_op* host_ops, int n, void* batch_ws, size_t batch_ws_bytes, void* stream);
/* bass_pr (mode 1) or bass_renorm (mode 0) on every segment (bass_simulator.py:574-578, 551-554) */
int bass_pr_batch(const bass_seg_op* host_ops, int n, int mode, void* batch_ws, size_t batch_ws_bytes,
                  void* stream);

/* ---- instrumentation ------------------------------------------------------------ */
/* Number of kernels this library has launched (process-wide). */
int64_t bass_launch_count(void);
/* Profiling on/off (process-wide).  When on, every kernel launch is bracketed by
   CUDA events on its stream and the tile kernels count the entries they read and
   write into ctrl->prof_in / prof_out. */
void bass_profile_enable(int on);
/* Synchronises, then writes per slot the summed event time (ms) and the number
   of launches since the last collect, and forgets them. */
int bass_profile_collect(double* host_ms, int64_t* host_launches, int nslots);

/* ---- errors ----------------------------------------------------------------- */
/* Synchronises `stream`, returns the sticky device error bits and clears them. */
int bass_error(bass_ctrl* ctrl, void* stream);
const char* bass_version(void);

#ifdef __cplusplus
}
#endif
#endif /* BASS_B200_H */
