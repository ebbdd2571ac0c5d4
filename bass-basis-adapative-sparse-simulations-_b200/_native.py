"""ctypes binding of libbass_b200.so and the device objects built on it.

Everything per-entry runs in the CUDA library; this module owns the device
buffers (torch CUDA tensors), passes raw pointers and sizes through the C ABI
(include/bass_b200.h) and reads back the few scalars the host driver needs.
There is no CPU fallback: ``lib()`` raises if the library or a GPU is missing.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbass_b200.so")
_lib = None

TRACE_WORDS = 7
SIG_PMIN = 1e-24
AMP_C128, AMP_C64 = 0, 1   # bass_state.amp_type


def amp_type_of(dtype) -> int:
    """BASS_AMP_* of a numpy complex dtype (complex128 or complex64)."""
    dt = np.dtype(dtype)
    if dt == np.complex128:
        return AMP_C128
    if dt == np.complex64:
        return AMP_C64
    raise ValueError(f"amplitudes must be complex128 or complex64, not {dt}")

# status codes / error bits
OK, ERR_CAPACITY, ERR_WAIT, ERR_ARG, ERR_CUDA, ERR_WORKSPACE = 0, 1, 2, 3, 4, 5
_ERR_NAMES = {ERR_CAPACITY: "capacity overflow", ERR_WAIT: "bounded device wait gave up",
              ERR_ARG: "invalid argument", ERR_CUDA: "CUDA runtime error",
              ERR_WORKSPACE: "workspace too small"}

# numpy mirrors of the device descriptors (C layout, natural alignment)
STATE_DTYPE = np.dtype([("keys", "<u8"), ("amps", "<u8"), ("nnz", "<i8"), ("cap", "<i8"),
                        ("rscale", "<f8", (2,)), ("nq", "<i4"), ("amp_type", "<i4"),
                        ("pos", "i1", (64,)), ("qat", "i1", (64,))], align=True)
CTRL_DTYPE = np.dtype([("gamma_running", "<f8"), ("state_gamma", "<f8"), ("pr_cur", "<f8"),
                       ("pr_last", "<f8"), ("last_kept", "<f8"), ("last_total", "<f8"),
                       ("truncation_active", "<i4"), ("gates_since_trunc", "<i4"), ("error", "<i4"),
                       ("last_truncated", "<i4"), ("amp_updates", "<i8"), ("n_trunc", "<i8"),
                       ("n_ops", "<i8"), ("accept", "<i4", (64,)), ("frac", "<f8", (64,)),
                       ("trace", "<u8"), ("trace_cap", "<i8"), ("trace_len", "<i8"),
                       ("pr_tie_tol", "<f8"), ("sync_counter", "<u4"), ("wait_limit", "<i4"),
                       ("prof_in", "<i8", (48,)), ("prof_out", "<i8", (48,))], align=True)
PROF_SLOTS = 48
KINDS = ["gate1", "rot1", "gate2", "perm", "plain", "rdm"]
PASSES = ["hist", "hist2", "gather", "write", "rdm"]
SLOT_NAMES = [f"k_tile<{k},{p}>" for k in KINDS for p in PASSES] + [
    "k_partition", "k_select_coop", "k_select2", "k_tie_coop", "k_finalize", "reductions", "k_fingerprint",
    "k_phase2q", "k_phase1q", "k_rdm_final", "radix_sort", "merge_runs", "bookkeeping", "select:level1",
    "select:level2", "select:count", "select:settle+final", "select:two_level"]
# select:* slots hold nanoseconds of k_select_coop's phases (block 0's clock,
# barrier waits included; the last block's for settle+final) in prof_in and the
# number of timed launches in prof_out; two_level counts (in prof_in) the
# selections whose threshold needed the level-2 histogram, out of all
# truncating selections (prof_out)
SELECT_PHASE_SLOTS = (43, 44, 45, 46)
SELECT_SPEC_SLOT = 47
# the write step of gates, rotations and truncations is k_compact, counted in the write slot
SLOT_NAMES[0 * 5 + 3] = "k_compact<gate1>"
SLOT_NAMES[1 * 5 + 3] = "k_compact<rot1>"
SLOT_NAMES[2 * 5 + 3] = "k_compact<gate2>"
SLOT_NAMES[4 * 5 + 3] = "k_compact<plain>"
# the RDM qubits at low physical bits: one pass of k_rdm_low (the RDM kind's evaluation slot)
SLOT_NAMES[5 * 5 + 0] = "k_rdm_low"


class Trunc(ctypes.Structure):
    """bass_trunc (passed by value)."""
    _fields_ = [("k_cond", ctypes.c_int64), ("k_keep", ctypes.c_int64), ("gamma_mode", ctypes.c_int32),
                ("renorm", ctypes.c_int32), ("mark_active", ctypes.c_int32), ("trace", ctypes.c_int32)]


NO_TRUNC = Trunc(-1, 0, 0, 0, 0, 0)

# bass_seg_op (include/bass_b200.h), one segment of a batched op
SEG_OP_DTYPE = np.dtype([("in", "<u8"), ("tmp", "<u8"), ("out", "<u8"), ("ctrl", "<u8"), ("ws", "<u8"),
                         ("ws_bytes", "<u8"), ("G", "<f8", (32,)), ("q1", "<i4"), ("q2", "<i4"),
                         ("k_cond", "<i8"), ("k_keep", "<i8"), ("gamma_mode", "<i4"), ("renorm", "<i4"),
                         ("mark_active", "<i4"), ("trace", "<i4"), ("rho", "<u8"), ("num_qubits", "<i4"),
                         ("pad", "<i4")], align=True)


class BassError(RuntimeError):
    pass


def build(force=False):
    import importlib.util
    spec = importlib.util.spec_from_file_location("_bass_build", os.path.join(_HERE, "build.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m.build(force=force)


def load_library():
    """Load libbass_b200.so (no GPU needed); raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise BassError(f"{LIB_PATH} is missing: build it with build.py (nvcc, sm_100a)")
    L = ctypes.CDLL(LIB_PATH)
    P, I32, I64, D, SZ = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_double, ctypes.c_size_t
    sig = {
        "bass_version": (ctypes.c_char_p, []),
        "bass_state_bytes": (SZ, []),
        "bass_batch_max_segments": (I32, []),
        "bass_ctrl_bytes": (SZ, []),
        "bass_workspace_bytes": (SZ, [I64, I64, I32]),
        "bass_state_init": (I32, [P, P, P, I64, I32, ctypes.c_uint64, P]),
        "bass_state_init_typed": (I32, [P, P, P, I64, I32, ctypes.c_uint64, I32, P]),
        "bass_state_import_typed": (I32, [P, P, P, I64, P, P, I64, I32, I32, P, SZ, P, P]),
        "bass_state_export_typed": (I32, [P, P, P, I32, I32, P, SZ, P, P]),
        "bass_state_import_into": (I32, [P, P, P, I64, P, P, I64, I32, P, SZ, P, P]),
        "bass_state_export": (I32, [P, P, P, P, SZ, P, P]),
        "bass_state_export_bits": (I32, [P, P, P, I32, P, SZ, P, P]),
        "bass_state_copy_desc": (I32, [P, P, P]),
        "bass_state_clone": (I32, [P, P, P, P]),
        "bass_ctrl_init": (I32, [P, P, I64, D, P]),
        "bass_gate_1q": (I32, [P, P, P, I32, Trunc, P, P, SZ, P]),
        "bass_gate_2q": (I32, [P, P, P, P, I32, I32, Trunc, P, P, SZ, P]),
        "bass_rotate_2q": (I32, [P, P, P, P, I32, I32, Trunc, P, P, SZ, P]),
        "bass_phase_1q": (I32, [P, P, P, I32, P, P, SZ, P]),
        "bass_phase_2q": (I32, [P, P, I32, I32, P, P]),
        "bass_topk": (I32, [P, P, Trunc, P, P, SZ, P]),
        "bass_gather": (I32, [P, P, P, I64, P, P]),
        "bass_lcg_choose": (I32, [I64, I64, I64, P]),
        "bass_renorm": (I32, [P, I32, P, P, SZ, P]),
        "bass_pr": (I32, [P, P, P, SZ, P]),
        "bass_norm2": (I32, [P, P, P, SZ, P]),
        "bass_rdm_1q": (I32, [P, I32, P, P, P, SZ, P]),
        "bass_rdm_2q": (I32, [P, P, I32, I32, P, P, P, SZ, P]),
        "bass_to_dense": (I32, [P, P, I32, P, P, P]),
        "bass_dense_dot": (I32, [P, P, I64, P, P, P, SZ, P]),
        "bass_dense_gate": (I32, [P, I32, P, I32, I32, I32, P]),
        "bass_sparse_dot": (I32, [P, P, I32, P, P, P, SZ, P]),
        "bass_rotate_step": (I32, [P, P, P, I32, I64, I32, P, P, SZ, P]),
        "bass_fingerprint": (I32, [P, D, P, P, SZ, P]),
        "bass_radix_sort_u64": (I32, [P, P, I64, I32, P, SZ, P, P]),
        "bass_merge_sorted": (I32, [P, P, I64, P, P, SZ, P, P]),
        "bass_error": (I32, [P, P]),
        "bass_batch_ws_bytes": (SZ, [I32]),
        "bass_gate_1q_batch": (I32, [P, I32, P, SZ, P]),
        "bass_gate_2q_batch": (I32, [P, I32, P, SZ, P]),
        "bass_phase_2q_batch": (I32, [P, I32, P, SZ, P]),
        "bass_topk_batch": (I32, [P, I32, P, SZ, P]),
        "bass_rotate_step_batch": (I32, [P, I32, P, SZ, P]),
        "bass_rdm_1q_batch": (I32, [P, I32, P, SZ, P]),
        "bass_pr_batch": (I32, [P, I32, I32, P, SZ, P]),
        "bass_launch_count": (I64, []),
        "bass_profile_enable": (None, [I32]),
        "bass_profile_collect": (I32, [P, P, I32]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    assert L.bass_state_bytes() == STATE_DTYPE.itemsize, "bass_state layout mismatch"
    assert L.bass_ctrl_bytes() == CTRL_DTYPE.itemsize, "bass_ctrl layout mismatch"
    _lib = L
    return L


def lib():
    """The library, on a machine with a CUDA device (raises otherwise)."""
    import torch
    if not torch.cuda.is_available():
        raise BassError("bass_b200 needs a CUDA device (no CPU fallback)")
    return load_library()


def check(status, what):
    if status != OK:
        raise BassError(f"{what} failed: {_ERR_NAMES.get(status, status)}")


def _ptr(t) -> int:
    return int(t.data_ptr())


def _host(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data)


class Engine:
    """Per-stream device context: control block, workspace, optional trace."""

    def __init__(self, max_n: int, num_qubits: int, trace_cap: int = 0, pr_tie_tol: float = 1e-12,
                 device=None, ctrl=None, rho=None):
        import torch
        self.L = lib()
        self.torch = torch
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.max_n = int(max(max_n, 16))
        self.nq = int(num_qubits)
        self.ws_bytes = int(self.L.bass_workspace_bytes(self.max_n // 4, self.max_n, self.nq))
        self.ws = torch.empty(self.ws_bytes, dtype=torch.uint8, device=self.device)
        # ctrl / rho: optional views into larger device tensors (a batch keeps
        # every state's control block and moments contiguous, to read them at once)
        self.ctrl = ctrl if ctrl is not None else torch.zeros(self.L.bass_ctrl_bytes(), dtype=torch.uint8,
                                                               device=self.device)
        self.trace_cap = int(trace_cap)
        self.trace = (torch.zeros(max(trace_cap, 1) * TRACE_WORDS, dtype=torch.int64, device=self.device)
                      if trace_cap else None)
        self.rho = rho if rho is not None else torch.zeros(4 * 64, dtype=torch.float64, device=self.device)
        self.scratch_f64 = torch.zeros(8, dtype=torch.float64, device=self.device)
        self.scratch_u64 = torch.zeros(8, dtype=torch.int64, device=self.device)
        self.pr_tie_tol = float(pr_tie_tol)
        self.reset()

    # -- plumbing ---------------------------------------------------------------
    @property
    def stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    @property
    def ctrl_ptr(self):
        return ctypes.c_void_p(_ptr(self.ctrl))

    @property
    def ws_ptr(self):
        return ctypes.c_void_p(_ptr(self.ws))

    def reset(self):
        tp = ctypes.c_void_p(_ptr(self.trace)) if self.trace is not None else None
        check(self.L.bass_ctrl_init(self.ctrl_ptr, tp, self.trace_cap, self.pr_tie_tol, self.stream),
              "bass_ctrl_init")

    def read_ctrl(self):
        """Synchronising read of the control block (numpy record), through a
        pinned host buffer."""
        torch = self.torch
        if getattr(self, "_ctrl_host", None) is None:
            self._ctrl_host = torch.empty(self.ctrl.numel(), dtype=torch.uint8, pin_memory=True)
        self._ctrl_host.copy_(self.ctrl, non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()
        return np.frombuffer(self._ctrl_host.numpy().tobytes(), dtype=CTRL_DTYPE)[0]

    def ctrl_field(self, name, np_dtype):
        off = CTRL_DTYPE.fields[name][1]
        size = np.dtype(np_dtype).itemsize
        return self.ctrl[off:off + size]

    def set_ctrl(self, name, value):
        """Asynchronous write of one scalar control field: a fill of the field
        on the stream (no host synchronisation)."""
        torch = self.torch
        dt = CTRL_DTYPE.fields[name][0]
        off = CTRL_DTYPE.fields[name][1]
        view = {np.dtype("<f8"): torch.float64, np.dtype("<i8"): torch.int64, np.dtype("<u8"): torch.int64,
                np.dtype("<i4"): torch.int32, np.dtype("<u4"): torch.int32}.get(np.dtype(dt))
        if view is None:
            raise TypeError(f"control field {name} is not a scalar")
        if np.dtype(dt).kind == "u":   # same bits through the signed view
            value = int(np.array([value], dtype=dt).view(np.dtype(dt).str.replace("u", "i"))[0])
        self.ctrl[off:off + np.dtype(dt).itemsize].view(view).fill_(value)

    def check_errors(self):
        """Synchronising read of the control block; raises on a device error."""
        c = self.read_ctrl()
        if int(c["error"]):
            self.raise_on_error()
        return c

    def raise_on_error(self):
        err = self.L.bass_error(self.ctrl_ptr, self.stream)
        if err:
            names = [v for k, v in _ERR_NAMES.items() if err & (1 << k)]
            raise BassError("device error: " + ", ".join(names or [str(err)]))

    def trace_events(self):
        """The device trace as an (n, 7) uint64 array (synchronising)."""
        if self.trace is None:
            return np.zeros((0, TRACE_WORDS), np.uint64)
        c = self.read_ctrl()
        n = int(c["trace_len"])
        return self.trace[: n * TRACE_WORDS].cpu().numpy().view(np.uint64).reshape(n, TRACE_WORDS)

    def append_trace(self, row):
        """Host-side event (e.g. "optimisation passed its PR gate"), appended in
        stream order after a synchronising read of the trace length."""
        if self.trace is None:
            return
        c = self.read_ctrl()
        n = int(c["trace_len"])
        if n >= self.trace_cap:
            raise BassError("trace capacity exceeded")
        r = np.array(row, dtype=np.uint64).view(np.int64)
        self.trace[n * TRACE_WORDS:(n + 1) * TRACE_WORDS].copy_(self.torch.from_numpy(r.copy()))
        self.set_ctrl("trace_len", n + 1)


class DevState:
    """One device descriptor plus its key / amplitude buffers (complex128, or
    complex64 with ``amp_type=AMP_C64``)."""

    def __init__(self, eng: Engine, cap: int, init_key: int = 0, amp_type: int = AMP_C128):
        torch = eng.torch
        self.eng = eng
        self.cap = int(max(cap, 1))
        self.amp_type = int(amp_type)
        self.desc = torch.zeros(eng.L.bass_state_bytes(), dtype=torch.uint8, device=eng.device)
        self.keys = torch.zeros(self.cap, dtype=torch.int64, device=eng.device)
        ft = torch.float32 if self.amp_type == AMP_C64 else torch.float64
        self.amps = torch.zeros(2 * self.cap, dtype=ft, device=eng.device)
        self.init(init_key)

    @property
    def np_dtype(self):
        return np.complex64 if self.amp_type == AMP_C64 else np.complex128

    @property
    def ptr(self):
        return ctypes.c_void_p(_ptr(self.desc))

    def init(self, key: int = 0):
        check(self.eng.L.bass_state_init_typed(self.ptr, ctypes.c_void_p(_ptr(self.keys)),
                                               ctypes.c_void_p(_ptr(self.amps)), self.cap, self.eng.nq,
                                               ctypes.c_uint64(int(key)), self.amp_type, self.eng.stream),
              "bass_state_init")

    def read_desc(self):
        return np.frombuffer(self.desc.cpu().numpy().tobytes(), dtype=STATE_DTYPE)[0]

    def nnz_view(self):
        off = STATE_DTYPE.fields["nnz"][1]
        return self.desc[off:off + 8].view(self.eng.torch.int64)

    def export(self, key_bits=None):
        """(true keys sorted ascending, amplitudes) as numpy arrays (synchronising)."""
        eng = self.eng
        n = int(self.read_desc()["nnz"])
        torch = eng.torch
        ok = torch.empty(max(n, 1), dtype=torch.int64, device=eng.device)
        oa = torch.empty(2 * max(n, 1), dtype=self.amps.dtype, device=eng.device)
        bits = eng.nq if key_bits is None else key_bits
        check(eng.L.bass_state_export_typed(self.ptr, ctypes.c_void_p(_ptr(ok)), ctypes.c_void_p(_ptr(oa)),
                                            int(bits), self.amp_type, eng.ws_ptr, eng.ws_bytes, eng.ctrl_ptr,
                                            eng.stream), "bass_state_export")
        # both copies into pinned host memory (torch's caching host allocator),
        # queued back to back, one synchronisation; the arrays view the pinned
        # buffers, which stay alive with them
        hk = torch.empty(max(n, 1), dtype=torch.int64, pin_memory=True)
        ha = torch.empty(2 * max(n, 1), dtype=oa.dtype, pin_memory=True)
        hk.copy_(ok, non_blocking=True)
        ha.copy_(oa, non_blocking=True)
        torch.cuda.current_stream(eng.device).synchronize()
        x = hk.numpy()[:n].view(np.uint64)
        a = ha.numpy()[:2 * n].view(self.np_dtype)
        return x, a

    def load(self, x, a):
        """Replace the contents by (true keys, amplitudes) given in any order."""
        eng = self.eng
        torch = eng.torch
        x = np.ascontiguousarray(x, dtype=np.uint64)
        a = np.ascontiguousarray(a, dtype=self.np_dtype)
        n = len(x)
        if n > self.cap:
            raise BassError("state capacity exceeded")
        real = np.float32 if self.amp_type == AMP_C64 else np.float64
        kx = torch.from_numpy(x.view(np.int64).copy()).to(eng.device) if n else self.keys
        ka = torch.from_numpy(a.view(real).copy()).to(eng.device) if n else self.amps
        check(eng.L.bass_state_import_typed(self.ptr, ctypes.c_void_p(_ptr(self.keys)),
                                            ctypes.c_void_p(_ptr(self.amps)), self.cap,
                                            ctypes.c_void_p(_ptr(kx)), ctypes.c_void_p(_ptr(ka)), n, eng.nq,
                                            self.amp_type, eng.ws_ptr, eng.ws_bytes, eng.ctrl_ptr, eng.stream),
              "bass_state_import_into")
        eng.torch.cuda.current_stream(eng.device).synchronize()  # kx / ka are temporaries

    def fingerprint(self, pmin=SIG_PMIN):
        eng = self.eng
        check(eng.L.bass_fingerprint(self.ptr, float(pmin), ctypes.c_void_p(_ptr(eng.scratch_u64)),
                                     eng.ws_ptr, eng.ws_bytes, eng.stream), "bass_fingerprint")
        return tuple(int(v) for v in eng.scratch_u64[:6].cpu().numpy().view(np.uint64))


def swap(a: DevState, b: DevState):
    """Swap two host handles (the device descriptors stay where they are)."""
    a.desc, b.desc = b.desc, a.desc
    a.keys, b.keys = b.keys, a.keys
    a.amps, b.amps = b.amps, a.amps
    a.cap, b.cap = b.cap, a.cap


def trunc(k_cond, k_keep, gamma_mode=0, renorm=0, mark_active=0, trace=0):
    return Trunc(int(k_cond), int(k_keep), int(gamma_mode), int(renorm), int(mark_active), int(trace))


def host_c128(m) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(m, dtype=np.complex128)).view(np.float64).copy()
