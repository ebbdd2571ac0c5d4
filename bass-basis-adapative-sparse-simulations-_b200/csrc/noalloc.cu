// noalloc.cu -- per-qubit RDM moments for callers that cannot allocate device
// memory.
//
// bass_rdm_1q needs a caller-allocated workspace.  Some callers cannot make
// that allocation: host runtimes whose device memory is owned by another
// allocator that hands out no scratch, plugins and embeddings that may only
// pass the buffers they were given, and code running at a point where it may
// not call cudaMalloc (which synchronises the device).  bass_rdm_1q_noalloc computes the same
// moments with its scratch in the file-scope array below instead.
//
// Limits and rules:
//   * the state may hold at most kNoAllocMaxEntries (2^20) entries; larger
//     requests are refused with BASS_ERR_WORKSPACE before any work is queued;
//     a state that does not fit the scratch although max_entries said it
//     would is refused by the kernels themselves (BASS_ERR_WORKSPACE in ctrl,
//     NaN in rho);
//   * the array (about 4.8 MB) is part of the library image: every GPU that
//     loads the library holds it until the process exits;
//   * all calls share the one array: calls that may overlap on the GPU (other
//     streams, other host threads) race and must be serialised by the caller;
//     the tile counters are cleared at the start of every call, everything else
//     is fully rewritten by each call;
//   * the first call on a device resolves the array's device address
//     (cudaGetSymbolAddress, with that device current).  The address is
//     cached for the life of the process; it is not valid after
//     cudaDeviceReset.
#include <stddef.h>

#include <mutex>

#include "internal.h"

namespace bass {

constexpr long long kNoAllocMaxEntries = 1LL << 20;
constexpr long long kNoAllocTiles = kNoAllocMaxEntries / kStep + 2;

struct NoAllocScratch {
  unsigned long long counters[64];
  SelState sel;
  long long part[(long long)kMaxSets * (kNoAllocTiles + 1) * 6];
  Partial partials[(long long)kMaxSets * kNoAllocTiles];
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

static std::mutex g_noalloc_mu;
static NoAllocScratch* g_noalloc_addr[256];

// Device address of g_noalloc_scratch on the current device (resolved once).
static cudaError_t noalloc_scratch(NoAllocScratch** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 256) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_addr[dev] = static_cast<NoAllocScratch*>(p);
  }
  *out = g_noalloc_addr[dev];
  return cudaSuccess;
}

}  // namespace bass

using namespace bass;

extern "C" int bass_rdm_1q_noalloc(const bass_state* st, int64_t max_entries, int num_qubits, double* rho,
                                   bass_ctrl* ctrl, void* stream) {
  if (!st || !rho || !ctrl || num_qubits < 1 || num_qubits > BASS_MAX_QUBITS || max_entries < 0)
    return BASS_ERR_ARG;
  if (max_entries > kNoAllocMaxEntries) return BASS_ERR_WORKSPACE;
  NoAllocScratch* sc = nullptr;
  if (noalloc_scratch(&sc) != cudaSuccess) return BASS_ERR_CUDA;
  cudaStream_t s = (cudaStream_t)stream;
  // the tile counters and the selection state must start at zero
  cudaError_t e = cudaMemsetAsync(sc, 0, offsetof(NoAllocScratch, part), s);
  if (e != cudaSuccess) return BASS_ERR_CUDA;
  WsView v{};
  v.counters = reinterpret_cast<unsigned int*>(sc->counters);
  v.sel = &sc->sel;
  v.part = sc->part;
  v.partials = sc->partials;
  v.max_n = kNoAllocMaxEntries;
  v.max_tiles = kNoAllocTiles;
  return run_rdm_prepared(st, num_qubits, rho, ctrl, v, s, state_c64(st)) == cudaSuccess ? BASS_OK : BASS_ERR_CUDA;
}
