"""CPU oracle for the BASS sparse-state hot path -- TEST INFRASTRUCTURE ONLY.

A restatement of the reference's algorithm (Skill0issue/BASS-Basis-Adapative-
Sparse-Simulations-): the per-entry kernels are plain C (``bass_oracle.c``,
compiled by :func:`build`), the per-gate drivers below follow

  * ``SparseState``            src/core/sparse_state.py:193-415
  * ``BASS``                   src/simulation/bass_simulator.py:478-929
  * ``FixedBasisSimulator``    src/simulation/simulator.py:61-253

line by line.  Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``
(its cpu_baseline leg and its ``--impl reference`` arm) may import this module,
and only as the checker or as the timed CPU baseline; the product never does.

Deliberate deviations from the reference (see the header of bass_oracle.c):
top-k ties are broken by key (ascending) and survivors keep their input order;
|a|^2 is re*re+im*im; every reduction is exact (order independent); a basis
rotation is kept only if it lowers the participation ratio by more than
``pr_tie_tol`` (1e-12 relative; the reference keeps it on any decrease, so a
rotation that leaves PR unchanged up to summation noise, such as a pure bit
relabel, is decided by that noise there).  The oracle is pinned against the
reference's own outputs, with the same two tie rules patched into it, by the
golden fixtures under tests/golden/.

Every driver can record a trace: one event per renormalisation point of the
reference (the simulate-level truncation, every attempted basis rotation, the
end of a basis optimisation), carrying the nnz and an order-independent
fingerprint of the surviving key set, plus every accepted rotation.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SRC = os.path.join(_HERE, "bass_oracle.c")
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

U64 = np.uint64
C128 = np.complex128


def build(force: bool = False) -> str:
    """Compile bass_oracle.c into oracle/_build/liboracle.so (gcc, -O2, no FMA,
    OpenMP).  The heavy kernels run on ``set_threads(n)`` host threads (one by
    default); their results do not depend on the thread count."""
    os.makedirs(os.path.dirname(_LIB_PATH), exist_ok=True)
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(_SRC):
        cmd = ["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared",
               "-o", _LIB_PATH, _SRC, "-lm"]
        subprocess.check_call(cmd)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P, I64, I = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int
        D, DP = ctypes.c_double, ctypes.POINTER(ctypes.c_double)
        sig = {
            "orc_expand_1q": (I64, [P, P, I64, P, P, P, I]),
            "orc_expand_2q": (I64, [P, P, I64, P, P, I64, P, I, I]),
            "orc_radix_sort": (I, [P, P, I64]),
            "orc_merge_sorted": (I64, [P, P, I64]),
            "orc_apply_1q": (I64, [P, P, I64, P, P, P, I]),
            "orc_apply_2q_sorted": (I64, [P, P, I64, P, P, I64, P, I, I]),
            "orc_apply_2q_ht": (I64, [P, P, I64, P, P, P, I, I]),
            "orc_phase_2q": (None, [P, P, I64, I, I, P]),
            "orc_select_topk": (I64, [P, P, I64, I64, DP, DP]),
            "orc_topk_truncate": (I64, [P, P, I64, I64, DP]),
            "orc_randomk_truncate": (I64, [P, P, I64, I64, I64, DP]),
            "orc_rdm_all": (I, [P, P, I64, I, P]),
            "orc_eigh_2x2": (None, [P, P, P]),
            "orc_rotate_1q": (I64, [P, P, I64, I, P, P, P]),
            "orc_rdm_2q": (I, [P, P, I64, I, I, P]),
            "orc_rotate_2q": (I64, [P, P, I64, I, I, P, P, P]),
            "orc_sum_p": (D, [P, I64]),
            "orc_sum_p2": (D, [P, I64]),
            "orc_fingerprint": (None, [P, P, I64, D, P]),
            "orc_exact_sum": (D, [P, I64]),
            "orc_threads": (I, []),
            "orc_set_threads": (I, [I]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def set_threads(n: int) -> int:
    """Host threads for the oracle's kernels (n <= 0: every thread OpenMP
    offers); returns the number in effect."""
    return int(lib().orc_set_threads(int(n)))


def _p(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data)


def _c(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=C128)


# ----------------------------------------------------------------------------
# kernel-level wrappers (each mirrors one reference kernel)
# ----------------------------------------------------------------------------
def expand_1q(x, a, G, q):
    """sparse_state.py:15-67 apply_1qubit_gate_kernel_opt."""
    x = np.ascontiguousarray(x, dtype=U64); a = _c(a); G = _c(G)
    xo = np.empty(2 * len(x) + 1, U64); ao = np.empty(2 * len(x) + 1, C128)
    n = lib().orc_expand_1q(_p(x), _p(a), len(x), _p(xo), _p(ao), _p(G), int(q))
    return xo[:n].copy(), ao[:n].copy()


def radix_sort(keys, vals):
    """sparse_state.py:150-172 radix_sort_uint64 (stable), returns sorted copies."""
    k = np.array(keys, dtype=U64, copy=True); v = np.array(vals, dtype=C128, copy=True)
    if lib().orc_radix_sort(_p(k), _p(v), len(k)):
        raise MemoryError
    return k, v


def merge_sorted(keys, vals):
    """sparse_state.py:127-147 merge_sorted_kernel, returns merged copies."""
    k = np.array(keys, dtype=U64, copy=True); v = np.array(vals, dtype=C128, copy=True)
    n = lib().orc_merge_sorted(_p(k), _p(v), len(k))
    return k[:n], v[:n]


def apply_1q(x, a, G, q):
    """SparseState.apply_single_qubit_gate without truncation: expand, sort, merge."""
    x = np.ascontiguousarray(x, dtype=U64); a = _c(a); G = _c(G)
    xo = np.empty(2 * len(x) + 1, U64); ao = np.empty(2 * len(x) + 1, C128)
    n = lib().orc_apply_1q(_p(x), _p(a), len(x), _p(xo), _p(ao), _p(G), int(q))
    if n < 0:
        raise MemoryError
    return xo[:n].copy(), ao[:n].copy()


def apply_2q_sorted(x, a, G, q1, q2):
    """SparseState.apply_two_qubit_gate without truncation: expand, sort, merge."""
    x = np.ascontiguousarray(x, dtype=U64); a = _c(a); G = _c(G)
    cap = 4 * len(x) + 1
    xo = np.empty(cap, U64); ao = np.empty(cap, C128)
    n = lib().orc_apply_2q_sorted(_p(x), _p(a), len(x), _p(xo), _p(ao), cap, _p(G), int(q1), int(q2))
    if n < 0:
        raise RuntimeError("Temporary buffer overflow")
    return xo[:n].copy(), ao[:n].copy()


def apply_2q_ht(x, a, G, q1, q2):
    """bass_simulator.py:292-354 apply_2qubit_gate_ht (first-occurrence order)."""
    x = np.ascontiguousarray(x, dtype=U64); a = _c(a); G = _c(G)
    xo = np.empty(4 * len(x) + 1, U64); ao = np.empty(4 * len(x) + 1, C128)
    n = lib().orc_apply_2q_ht(_p(x), _p(a), len(x), _p(xo), _p(ao), _p(G), int(q1), int(q2))
    if n < 0:
        raise MemoryError
    return xo[:n].copy(), ao[:n].copy()


def phase_2q(x, a, q1, q2, diag):
    """sparse_state.py:178-190 apply_2qubit_diagonal_kernel, returns a new amp array."""
    x = np.ascontiguousarray(x, dtype=U64); a = np.array(a, dtype=C128, copy=True)
    d = _c(diag)
    lib().orc_phase_2q(_p(x), _p(a), len(x), int(q1), int(q2), _p(d))
    return a


def select_topk(x, a, k):
    """Top-k by (|a|^2 desc, key asc), survivors in input order.
    Returns (x', a', kept_mass, total_mass)."""
    x = np.array(x, dtype=U64, copy=True); a = np.array(a, dtype=C128, copy=True)
    kept = ctypes.c_double(); tot = ctypes.c_double()
    n = lib().orc_select_topk(_p(x), _p(a), len(x), int(k), ctypes.byref(kept), ctypes.byref(tot))
    if n < 0:
        raise MemoryError
    return x[:n], a[:n], kept.value, tot.value


def topk_truncate(x, a, k):
    """truncation.py:68-113 top_k_truncate_kernel_opt -> (x', a', gamma_sq)."""
    x = np.array(x, dtype=U64, copy=True); a = np.array(a, dtype=C128, copy=True)
    g = ctypes.c_double()
    n = lib().orc_topk_truncate(_p(x), _p(a), len(x), int(k), ctypes.byref(g))
    return x[:n], a[:n], g.value


def randomk_truncate(x, a, k, seed):
    """truncation.py:116-159 random_k_truncate_kernel_opt -> (x', a', gamma_sq)."""
    x = np.array(x, dtype=U64, copy=True); a = np.array(a, dtype=C128, copy=True)
    g = ctypes.c_double()
    n = lib().orc_randomk_truncate(_p(x), _p(a), len(x), int(k), int(seed), ctypes.byref(g))
    return x[:n], a[:n], g.value


def rdm_all(x, a, N):
    """bass_simulator.py:441-470 compute_all_1qubit_rdms -> complex (N, 2, 2)."""
    x = np.ascontiguousarray(x, dtype=U64); a = _c(a)
    rho = np.zeros((N, 2, 2), C128)
    if lib().orc_rdm_all(_p(x), _p(a), len(x), int(N), _p(rho)):
        raise MemoryError
    return rho


def eigh_2x2(rho):
    """bass_simulator.py:386-437 eigh_2x2 -> (evals[2], V (2,2))."""
    rho = _c(rho)
    ev = np.zeros(2); V = np.zeros((2, 2), C128)
    lib().orc_eigh_2x2(_p(rho), _p(ev), _p(V))
    return ev, V


def rotate_1q(x, a, qubit, U):
    """bass_simulator.py:156-199 apply_1qubit_rotation_sparse (returns new arrays)."""
    x = np.ascontiguousarray(x, dtype=U64); a = _c(a); U = _c(U)
    xo = np.empty(2 * len(x) + 1, U64); ao = np.empty(2 * len(x) + 1, C128)
    n = lib().orc_rotate_1q(_p(x), _p(a), len(x), int(qubit), _p(U), _p(xo), _p(ao))
    if n < 0:
        raise MemoryError
    return xo[:n].copy(), ao[:n].copy()


def rdm_2q(x, a, q1, q2):
    """bass_simulator.py:200-231 compute_2qubit_rdm -> complex (4, 4), index
    (bit_q1 << 1) | bit_q2; exact sums."""
    x = np.ascontiguousarray(x, dtype=U64); a = _c(a)
    rho = np.zeros((4, 4), C128)
    if lib().orc_rdm_2q(_p(x), _p(a), len(x), int(q1), int(q2), _p(rho)):
        raise MemoryError
    return rho


def rotate_2q(x, a, q1, q2, U4):
    """bass_simulator.py:237-289 apply_2qubit_rotation_sparse (returns new,
    key-sorted arrays)."""
    x = np.ascontiguousarray(x, dtype=U64); a = _c(a); U4 = _c(U4)
    xo = np.empty(4 * len(x) + 1, U64); ao = np.empty(4 * len(x) + 1, C128)
    n = lib().orc_rotate_2q(_p(x), _p(a), len(x), int(q1), int(q2), _p(U4), _p(xo), _p(ao))
    if n < 0:
        raise MemoryError
    return xo[:n].copy(), ao[:n].copy()


SIG_PMIN = 1e-24   # |a|^2 threshold of the "significant keys" fingerprint


def fingerprint(x, a=None, pmin=0.0) -> tuple[int, int, int]:
    """Order-independent fingerprint (count, sum, xor) of a key set; with ``a``
    only keys whose |a|^2 exceeds ``pmin`` count.  Same definition as the CUDA
    library's ``bass_fingerprint``."""
    x = np.ascontiguousarray(x, dtype=U64)
    out = np.zeros(3, U64)
    if a is None:
        lib().orc_fingerprint(_p(x), None, len(x), 0.0, _p(out))
    else:
        a = _c(a)
        lib().orc_fingerprint(_p(x), _p(a), len(x), float(pmin), _p(out))
    return int(out[0]), int(out[1]), int(out[2])


def exact_sum(v) -> float:
    """The exact, order-independent sum used for every reduction."""
    v = np.ascontiguousarray(v, dtype=np.float64)
    return float(lib().orc_exact_sum(_p(v), len(v)))


def sum_p(a) -> float:
    a = _c(a)
    return float(lib().orc_sum_p(_p(a), len(a)))


def sum_p2(a) -> float:
    a = _c(a)
    return float(lib().orc_sum_p2(_p(a), len(a)))


# ----------------------------------------------------------------------------
# drivers
# ----------------------------------------------------------------------------
class Trace:
    """Event log shared by the oracle drivers (and mirrored by the CUDA host).

    ``events`` is a list of 7-tuples of ints (the golden fixtures store the same
    rows as a uint64 array):
      (0, nnz, fp_sum, fp_xor, sig_count, sig_sum, sig_xor)
          a renormalisation point of the reference (after a simulate-level
          truncation, after each attempted basis rotation, at the end of
          _optimize_basis); fp_* fingerprint every key, sig_* only the keys
          with |a|^2 > SIG_PMIN after the renormalisation;
      (1, j, 0, 0, 0, 0, 0)      a basis rotation of qubit j was kept;
      (2, gate, 0, 0, 0, 0, 0)   _optimize_basis passed its PR gate.
    """

    def __init__(self):
        self.events = []

    def renorm(self, x, a):
        c, s, z = fingerprint(x)
        c2, s2, z2 = fingerprint(x, a, SIG_PMIN)
        self.events.append((0, c, s, z, c2, s2, z2))

    def accept(self, j):
        self.events.append((1, int(j), 0, 0, 0, 0, 0))

    def opt(self, i):
        self.events.append((2, int(i), 0, 0, 0, 0, 0))

    def array(self):
        return np.array(self.events, dtype=np.uint64).reshape(-1, 7)


class OracleSparseState:
    """sparse_state.py:193-415 (state as two exact-length arrays)."""

    def __init__(self, num_qubits, k, init_state=None):
        self.N = num_qubits
        self.k = k
        self.x = np.array([0 if init_state is None else init_state], dtype=U64)
        self.alpha = np.array([1.0 + 0.0j], dtype=C128)
        self.gamma = 1.0

    @property
    def nnz(self):
        return len(self.x)

    def apply_gate(self, gate, method="top-k", seed="None"):
        # sparse_state.py:379-385
        if gate.n_qubits == 1:
            self.x, self.alpha = apply_1q(self.x, self.alpha, gate.matrix, gate.qubits[0])
        elif gate.n_qubits == 2:
            self.x, self.alpha = apply_2q_sorted(self.x, self.alpha, gate.matrix, *gate.qubits)
        else:
            raise NotImplementedError("Only 1- and 2-qubit gates supported")
        if self.nnz > self.k:
            if method == "top-k":
                self.truncate_top_k()
            else:
                self.truncate_random_k(seed)

    def truncate_top_k(self):
        # sparse_state.py:388-400
        if self.nnz <= self.k:
            return
        self.x, self.alpha, gsq = topk_truncate(self.x, self.alpha, self.k)
        gl = np.sqrt(gsq)
        self.alpha /= gl
        self.gamma *= gl

    def truncate_random_k(self, seed):
        # sparse_state.py:402-415
        if self.nnz <= self.k:
            return
        if seed is None:
            seed = int(np.random.randint(0, 2**31))
        self.x, self.alpha, gsq = randomk_truncate(self.x, self.alpha, self.k, seed)
        gl = np.sqrt(gsq)
        self.alpha /= gl
        self.gamma *= gl


def _is_gate_diagonal(G, tol=1e-12):
    # bass_simulator.py:473-475
    return np.max(np.abs(G - np.diag(np.diag(G)))) < tol


def _kron_2x2(A, B):
    # bass_simulator.py:357-383 (block assembly, element by element)
    C = np.empty((4, 4), dtype=C128)
    for i in range(2):
        for j in range(2):
            C[2 * i:2 * i + 2, 2 * j:2 * j + 2] = A[i, j] * B
    return C


def eigh_2x2_py(rho):
    """bass_simulator.py:386-437 in Python scalar arithmetic (IEEE double)."""
    from math import sqrt
    a = float(rho[0, 0].real); d = float(rho[1, 1].real); b = complex(rho[0, 1])
    b_sq = b.real ** 2 + b.imag ** 2
    tau = (d - a) * 0.5
    disc = sqrt(tau * tau + b_sq)
    V = np.zeros((2, 2), dtype=C128)
    if b_sq < 1e-28:
        if a >= d:
            V[0, 0] = 1.0; V[1, 1] = 1.0
        else:
            V[0, 1] = 1.0; V[1, 0] = 1.0
    else:
        tdp = tau + disc; tdm = tau - disc
        n0 = sqrt(b_sq + tdp * tdp); n1 = sqrt(b_sq + tdm * tdm)
        V[0, 0] = complex(b.real / n0, b.imag / n0)
        V[1, 0] = tdp / n0
        V[0, 1] = complex(b.real / n1, b.imag / n1)
        V[1, 1] = tdm / n1
    return np.array([(a + d) * 0.5 + disc, (a + d) * 0.5 - disc]), V


class OracleBASS:
    """bass_simulator.py:478-929: 1-qubit coordinate descent and, with
    use_2qubit_rotations, the brick-wall 2-qubit passes (:679-728, :819-824)."""

    def __init__(self, num_qubits, k, optimize_every=5, buffer_factor=2, truncate_every=1,
                 max_nnz_factor=8, use_2qubit_rotations=False, verbose=False, use_fast_eigh=True,
                 use_diag_gate=True, use_kron_cache=True, pr_opt_threshold=0.90, trace=None,
                 pr_tie_tol=1e-12):
        self.use_2qubit_rotations = use_2qubit_rotations
        self.N = num_qubits
        self.k = k
        self.optimize_every = optimize_every
        self.buffer_factor = buffer_factor
        self.truncate_every = truncate_every
        self.max_nnz_factor = max_nnz_factor
        self.use_fast_eigh = use_fast_eigh
        self.use_diag_gate = use_diag_gate
        self.use_kron_cache = use_kron_cache
        self.pr_opt_threshold = pr_opt_threshold
        self.pr_tie_tol = pr_tie_tol
        self.trace = trace
        self.U = None
        self._kron_cache = {}
        self._gamma_running = 1.0
        self._pr_at_last_opt = 0.0
        self.stats = {"gates": 0, "amp_updates": 0, "rotations": 0, "accepted": 0, "opt_calls": 0}

    # bass_simulator.py:551-554
    def _renorm(self, st):
        norm = np.sqrt(sum_p(st.alpha))
        if norm > 1e-30:
            st.alpha /= norm
        if self.trace is not None:
            self.trace.renorm(st.x, st.alpha)

    # bass_simulator.py:565-572
    def _truncate_state(self, st):
        if st.nnz <= self.k:
            return
        st.x, st.alpha, _, _ = select_topk(st.x, st.alpha, self.k)

    # bass_simulator.py:574-578
    def _pr(self, st):
        if st.nnz == 0:
            return float("inf")
        denom = sum_p2(st.alpha)
        return 1.0 / denom if denom > 1e-60 else float("inf")

    def _get_kron(self, q1, q2):
        if not self.use_kron_cache:
            return _kron_2x2(self.U[q1], self.U[q2])
        key = (q1, q2)
        if key not in self._kron_cache:
            self._kron_cache[key] = _kron_2x2(self.U[q1], self.U[q2])
        return self._kron_cache[key]

    def _invalidate_kron(self, qubit):
        for key in [kk for kk in self._kron_cache if qubit in kk]:
            del self._kron_cache[key]

    # bass_simulator.py:730-827 (1-qubit passes)
    def _descent_pass(self, st, qubits=None):
        """One pass of the 1-qubit coordinate descent (bass_simulator.py:739-816):
        the RDMs of the state, then a rotation step for every qubit in turn
        (``qubits``: only those, for a bounded timing sample); returns whether
        some rotation was kept."""
        all_rho = rdm_all(st.x, st.alpha, self.N)
        pr = self._pr(st)
        improved = False
        for j in (range(self.N) if qubits is None else qubits):
            if self.use_fast_eigh:
                _, V = eigh_2x2_py(all_rho[j])
            else:
                evals, V = np.linalg.eigh(all_rho[j])
                V = V[:, np.argsort(-evals)]
                if np.linalg.det(V).real < 0:
                    V[:, 1] *= -1
            if abs(V[0, 1]) + abs(V[1, 0]) < 1e-10:
                continue
            x_save, a_save, U_save = st.x, st.alpha, self.U[j].copy()
            self.stats["rotations"] += 1
            self.stats["amp_updates"] += st.nnz
            st.x, st.alpha = rotate_1q(st.x, st.alpha, j, V.conj().T)
            self._truncate_state(st)
            frac = sum_p(st.alpha)
            p2 = sum_p2(st.alpha)
            self._renorm(st)
            # PR of the renormalised candidate, from the exact sums of the
            # unnormalised one: frac^2 / sum |a|^4 (the reference evaluates
            # 1 / sum |a/sqrt(frac)|^4; the two differ by rounding only)
            pr_new = (frac * frac) / p2 if (st.nnz > 0 and p2 > 0) else float("inf")
            # the reference's rule is `pr_new >= pr`; a rotation must lower
            # PR by more than pr_tie_tol (relative) to count (0 restores it)
            if pr_new >= pr * (1.0 - self.pr_tie_tol):
                st.x, st.alpha = x_save, a_save
                self.U[j] = U_save
            else:
                self.U[j] = self.U[j] @ V
                pr = pr_new
                self._gamma_running *= np.sqrt(frac if frac > 1e-30 else 0)
                self._invalidate_kron(j)
                improved = True
                self.stats["accepted"] += 1
                if self.trace is not None:
                    self.trace.accept(j)
        return improved

    def _optimize_basis(self, st, gate_index=-1):
        if self._pr(st) < self.k / 4:
            return
        self.stats["opt_calls"] += 1
        if self.trace is not None:
            self.trace.opt(gate_index)
        for _pass in range(3):
            if not self._descent_pass(st):
                break
        if self.use_2qubit_rotations and self.N >= 2:
            self._optimize_2q_pass(st, [(i, i + 1) for i in range(0, self.N - 1, 2)])
            self._optimize_2q_pass(st, [(i, i + 1) for i in range(1, self.N - 1, 2)])
        self._truncate_state(st)
        self._renorm(st)

    # bass_simulator.py:679-728
    def _optimize_2q_pass(self, st, pairs):
        for q1, q2 in pairs:
            rho = rdm_2q(st.x, st.alpha, q1, q2)
            evals, evecs = np.linalg.eigh(rho)
            V = evecs[:, np.argsort(-evals)]
            V_rot = V.conj().T
            x_save, a_save = st.x, st.alpha
            pr_before = self._pr(st)
            st.x, st.alpha = rotate_2q(st.x, st.alpha, q1, q2, V_rot)
            self._truncate_state(st)
            frac1 = sum_p(st.alpha)
            self._renorm(st)
            st.x, st.alpha = rotate_2q(st.x, st.alpha, q1, q2, V)
            self._truncate_state(st)
            frac2 = sum_p(st.alpha)
            self._renorm(st)
            pr_after = self._pr(st)
            # the reference restores when `pr_after > pr_before`; here PR must
            # drop by more than pr_tie_tol (relative), as for the 1-qubit steps
            if pr_after > pr_before * (1.0 - self.pr_tie_tol):
                st.x, st.alpha = x_save, a_save
            else:
                self._gamma_running *= np.sqrt(frac1 * frac2)

    # bass_simulator.py:829-845
    def optimize_trigger(self, st):
        if self.pr_opt_threshold >= 1.0:
            return True
        return self._pr(st) > self._pr_at_last_opt / self.pr_opt_threshold

    # bass_simulator.py:847-929
    def simulate(self, circuit, initial_state=0):
        self.U = [np.eye(2, dtype=C128) for _ in range(self.N)]
        self._kron_cache = {}
        self._pr_at_last_opt = 0.0
        hard_cap = min(self.max_nnz_factor * self.k, 2 ** self.N)
        internal_k = min(max(max(self.buffer_factor, 2) * self.k, hard_cap), 2 ** self.N)
        st = OracleSparseState(self.N, internal_k, initial_state)
        M = len(circuit)
        self._gamma_running = 1.0
        truncation_active = False
        gates_since_trunc = 0
        for i, gate in enumerate(circuit):
            self.stats["gates"] += 1
            if gate.n_qubits == 1:
                q = gate.qubits[0]
                G = self.U[q].conj().T @ gate.matrix @ self.U[q]
                self.stats["amp_updates"] += st.nnz
                st.x, st.alpha = apply_1q(st.x, st.alpha, G, q)
                if st.nnz > st.k:
                    st.truncate_top_k()
                gates_since_trunc += 1
            elif gate.n_qubits == 2:
                q1, q2 = gate.qubits
                Ut = self._get_kron(q1, q2)
                G = Ut.conj().T @ gate.matrix @ Ut
                self.stats["amp_updates"] += st.nnz
                if self.use_diag_gate and _is_gate_diagonal(G):
                    st.alpha = phase_2q(st.x, st.alpha, q1, q2, np.diag(G).astype(C128))
                    if self.optimize_every > 0 and (i + 1) % self.optimize_every == 0 and i + 1 < M:
                        if truncation_active and self.optimize_trigger(st):
                            self._optimize_basis(st, i)
                            self._pr_at_last_opt = self._pr(st)
                        truncation_active = False
                    continue
                st.x, st.alpha = apply_2q_ht(st.x, st.alpha, G, q1, q2)
                gates_since_trunc += 1
            else:
                raise ValueError(f"{gate.n_qubits}-qubit gates unsupported")

            over_hard = st.nnz > hard_cap
            over_budget = st.nnz > self.k
            if over_hard or (over_budget and gates_since_trunc >= self.truncate_every):
                truncation_active = True
                st.x, st.alpha, kept, total = select_topk(st.x, st.alpha, self.k)
                self._gamma_running *= kept / total if total > 1e-30 else 0
                self._renorm(st)
                gates_since_trunc = 0

            if self.optimize_every > 0 and (i + 1) % self.optimize_every == 0 and i + 1 < M:
                if truncation_active and self.optimize_trigger(st):
                    self._optimize_basis(st, i)
                    self._pr_at_last_opt = self._pr(st)
                truncation_active = False

        st.gamma = np.sqrt(max(self._gamma_running, 0))
        return st

    # bass_simulator.py:608-621
    def to_statevector(self, st):
        if self.N > 24:
            raise ValueError(f"N={self.N} too large for statevector")
        psi = np.zeros(2 ** self.N, dtype=C128)
        psi[st.x.astype(np.int64)] = st.alpha
        for j in range(self.N):
            psi3d = psi.reshape(-1, 2, 1 << j)
            psi = np.einsum("ij,kjl->kil", self.U[j], psi3d).reshape(-1)
        return psi


class OracleFixedBasis:
    """simulator.py:61-253 (top-k and the LCG-seeded paths)."""

    def __init__(self, num_qubits, k, truncation="top-k", verbose=False, log_every=1, max_nnz_factor=8):
        if truncation not in ("top-k", "random-k"):
            raise ValueError("Unknown truncation")
        self.N = num_qubits
        self.k = k
        self._truncate_name = truncation

    def simulate(self, circuit, initial_state=None, seed=None):
        st = OracleSparseState(self.N, self.k, initial_state)
        L = len(circuit)
        gamma_hist = np.empty(L + 1); nnz_hist = np.empty(L + 1)
        gamma_hist[0] = 1.0; nnz_hist[0] = st.nnz
        if seed is None:
            seed = int(np.random.randint(0, 2**31))
        cur = seed
        for i, gate in enumerate(circuit):
            cur = (1103515245 * cur + 12345) & 0x7FFFFFFF
            if gate.n_qubits == 2:
                q1, q2 = gate.qubits
                st.x, st.alpha = apply_2q_ht(st.x, st.alpha, gate.matrix, q1, q2)
                if st.nnz > self.k:
                    if self._truncate_name == "top-k":
                        st.x, st.alpha, kept, total = select_topk(st.x, st.alpha, self.k)
                    else:
                        probs = np.abs(st.alpha) ** 2
                        total = np.sum(probs)
                        np.random.seed(cur)
                        pn = probs / total if total > 1e-30 else np.ones(st.nnz) / st.nnz
                        idx = np.random.choice(st.nnz, size=self.k, replace=False, p=pn)
                        kept = np.sum(probs[idx])
                        st.x, st.alpha = st.x[idx].copy(), st.alpha[idx].copy()
                    st.gamma *= np.sqrt(kept / total) if total > 1e-30 else 0
                    norm = np.sqrt(sum_p(st.alpha))
                    if norm > 1e-30:
                        st.alpha /= norm
            else:
                st.apply_gate(gate, self._truncate_name, cur)
            gamma_hist[i + 1] = st.gamma
            nnz_hist[i + 1] = st.nnz
        self.gamma_history = gamma_hist
        self.nnz_history = nnz_hist
        return st
