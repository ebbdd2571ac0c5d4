"""SparseState on the GPU -- drop-in for src/core/sparse_state.py:193-415.

The state lives in device memory as a sorted array of (physical key,
complex128 amplitude) plus a descriptor (include/bass_b200.h, bass_state).
``x`` and ``alpha`` are read-only host copies of the nnz entries (the
reference keeps capacity-length arrays whose first nnz entries are valid, so
``x[:nnz]`` works on both), in the reference's entry order: ascending true
key after every gate (sparse_state.py:268-301 sorts), and the order of the
drawn entries after a random-k truncation (truncation.py:116-159), and the
hash-table gate's order in FixedBasisSimulator.  The device keeps
the entries sorted by physical key; that order is tracked on the host, as the
true keys in order, only while it differs from key order.  Reading ``x``,
``alpha``, ``nnz`` or ``gamma`` synchronises the stream.
"""
from __future__ import annotations

import numpy as np

from . import _native as nat
from .linalg import is_gate_diagonal  # noqa: F401  (re-exported for callers)


class SparseState:
    """|phi> = sum_i alpha_i |x_i>, at most ``k`` entries after a truncation."""

    def __init__(self, num_qubits, k, init_state=None, *, dtype=np.complex128, _capacity=None, _engine=None,
                 _trace_cap=0):
        self.N = int(num_qubits)
        self.k = int(k)
        self.dtype = np.dtype(dtype)
        at = nat.amp_type_of(self.dtype)
        self.RADIX_THRESHOLD = 2000  # kept for interface parity; the GPU path always merges
        # like the reference's 4k temporary buffers: a gate whose truncation is
        # decided afterwards (random-k) first writes up to 4k entries
        cap = int(_capacity) if _capacity is not None else 4 * self.k + 16
        self._eng = _engine if _engine is not None else nat.Engine(
            max_n=4 * cap + 64, num_qubits=self.N, trace_cap=_trace_cap)
        key = 0 if init_state is None else int(init_state)
        self._cur = nat.DevState(self._eng, cap, key, at)
        self._tmp = nat.DevState(self._eng, cap, 0, at)
        self._tmp2 = nat.DevState(self._eng, cap, 0, at)
        self._version = 0
        self._export = None
        self._order = None   # the reference's entry order (true keys) when not ascending

    # ---- host views -----------------------------------------------------------
    def __repr__(self):
        return f"SparseState(N={self.N}, k={self.k}, nnz={self.nnz}, γ²={self.gamma ** 2:.6f})"

    @property
    def nnz(self) -> int:
        n = int(self._cur.read_desc()["nnz"])
        self._eng.check_errors()
        return n

    @property
    def gamma(self) -> float:
        return float(self._eng.check_errors()["state_gamma"])

    @gamma.setter
    def gamma(self, v):
        self._eng.set_ctrl("state_gamma", float(v))

    def _exported(self):
        """The entries in ascending true-key order (host copies)."""
        if self._export is None or self._export[0] != self._version:
            self._eng.check_errors()
            x, a = self._cur.export()
            self._export = (self._version, x, a, None)
        return self._export[1], self._export[2]

    def _in_order(self):
        """The entries in the reference's order (see the module docstring)."""
        x, a = self._exported()
        if self._order is None:
            return x, a
        if self._export[3] is None:
            pos = np.searchsorted(x, self._order)
            if len(self._order) != len(x) or not np.array_equal(x[np.minimum(pos, len(x) - 1)], self._order):
                raise RuntimeError("entry order out of step with the device state")
            self._export = self._export[:3] + ((self._order, a[pos]),)
        return self._export[3]

    @property
    def x(self) -> np.ndarray:
        return self._in_order()[0]

    @property
    def alpha(self) -> np.ndarray:
        return self._in_order()[1]

    def _touch(self):
        self._version += 1

    def _rekeyed(self):
        """After an op whose result the reference holds in key order."""
        self._touch()
        self._order = None

    def _set_order(self, keys):
        """Record the reference's entry order (true keys, a permutation of
        the state's keys); None or ascending keys mean key order."""
        if keys is None:
            self._order = None
            return
        keys = np.asarray(keys, dtype=np.uint64)
        self._order = None if (len(keys) < 2 or bool(np.all(keys[1:] > keys[:-1]))) else keys.copy()
        self._export = None if self._export is None else self._export[:3] + (None,)

    def load(self, x, alpha):
        """Replace the entries (any order; duplicate keys are summed); they
        read back in ascending key order."""
        self._cur.load(x, alpha)
        self._rekeyed()

    def _load_in_order(self, x, alpha):
        """load() of distinct keys that then read back in the given order (the
        reference's arrays after a random-k draw)."""
        x = np.asarray(x, dtype=np.uint64)
        self._cur.load(x, alpha)
        self._touch()
        self._set_order(x)

    def copy(self):
        new = SparseState(self.N, self.k, dtype=self.dtype, _capacity=self._cur.cap)
        x, a = self._in_order()
        new._load_in_order(x, a)
        new.gamma = self.gamma
        return new

    def to_dense(self):
        if self.N > 20:
            raise ValueError("Dense conversion only allowed for N <= 20")
        x, a = self._exported()
        dense = np.zeros(2 ** self.N, dtype=self.dtype)
        dense[x.astype(np.int64)] = a
        return dense

    def to_dense_device(self, U=None):
        """The dense statevector on the device (torch complex128, 2^N entries,
        N <= 30): the entries at their true keys, then each frame U[j] applied
        to qubit j (bass_simulator.py:608-621 with U = the BASS frames)."""
        eng = self._eng
        if self.N > 30:
            raise ValueError(f"N={self.N} too large for a dense statevector")
        torch = eng.torch
        psi = torch.empty(2 ** self.N, dtype=torch.complex128, device=eng.device)
        hu = None
        if U is not None:
            hu = nat.host_c128(np.stack([np.asarray(u, dtype=np.complex128) for u in U]))
        nat.check(eng.L.bass_to_dense(self._cur.ptr, None if hu is None else nat._host(hu), int(self.N),
                                      nat.ctypes.c_void_p(psi.data_ptr()), eng.ctrl_ptr, eng.stream),
                  "bass_to_dense")
        eng.check_errors()
        return psi

    def probability_distribution(self):
        return np.abs(self.alpha) ** 2 / (self.gamma ** 2)

    def sample(self, num_samples=1):
        probs = self.probability_distribution()
        probs /= probs.sum()
        idx = np.random.choice(self.nnz, size=num_samples, p=probs)
        return self.x[idx]

    # ---- device ops -------------------------------------------------------------
    def _apply_1q(self, G, q, tr):
        eng = self._eng
        G = np.asarray(G, dtype=np.complex128)
        if G[0, 1] == 0 and G[1, 0] == 0:
            # every off-diagonal child is exactly zero: an in-place phase
            d = nat.host_c128([G[0, 0], G[1, 1]])
            nat.check(eng.L.bass_phase_1q(self._cur.ptr, self._tmp.ptr, nat._host(d), int(q), eng.ctrl_ptr,
                                          eng.ws_ptr, eng.ws_bytes, eng.stream), "bass_phase_1q")
        else:
            g = nat.host_c128(G)
            nat.check(eng.L.bass_gate_1q(self._cur.ptr, self._tmp.ptr, nat._host(g), int(q), tr, eng.ctrl_ptr,
                                         eng.ws_ptr, eng.ws_bytes, eng.stream), "bass_gate_1q")
            nat.swap(self._cur, self._tmp)
        self._rekeyed()

    def _apply_2q(self, G, q1, q2, tr):
        eng = self._eng
        g = nat.host_c128(G)
        nat.check(eng.L.bass_gate_2q(self._cur.ptr, self._tmp.ptr, self._tmp2.ptr, nat._host(g), int(q1),
                                     int(q2), tr, eng.ctrl_ptr, eng.ws_ptr, eng.ws_bytes, eng.stream),
                  "bass_gate_2q")
        nat.swap(self._cur, self._tmp2)
        self._rekeyed()

    def _rotate_2q(self, U4, q1, q2, tr):
        """bass_simulator.py:237-289 apply_2qubit_rotation_sparse with the
        truncation tr fused; the previous state is left in _tmp2."""
        eng = self._eng
        u = nat.host_c128(U4)
        nat.check(eng.L.bass_rotate_2q(self._cur.ptr, self._tmp.ptr, self._tmp2.ptr, nat._host(u), int(q1),
                                       int(q2), tr, eng.ctrl_ptr, eng.ws_ptr, eng.ws_bytes, eng.stream),
                  "bass_rotate_2q")
        nat.swap(self._cur, self._tmp2)
        self._rekeyed()

    def _rdm_2q(self, q1, q2) -> np.ndarray:
        """bass_simulator.py:200-231 compute_2qubit_rdm: 4x4 complex, index
        (bit_q1 << 1) | bit_q2 (synchronising)."""
        eng = self._eng
        nat.check(eng.L.bass_rdm_2q(self._cur.ptr, self._tmp.ptr, int(q1), int(q2),
                                    nat.ctypes.c_void_p(nat._ptr(eng.rho)), eng.ctrl_ptr, eng.ws_ptr,
                                    eng.ws_bytes, eng.stream), "bass_rdm_2q")
        r = eng.rho[:16].cpu().numpy()
        rho = np.zeros((4, 4), dtype=np.complex128)
        for i in range(4):
            rho[i, i] = r[i]
        for n, (i, j) in enumerate([(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]):
            rho[i, j] = complex(r[4 + 2 * n], r[5 + 2 * n])
            rho[j, i] = np.conj(rho[i, j])
        return rho

    def _spare(self):
        """A fourth device buffer (the 2-qubit passes park the saved state there)."""
        if getattr(self, "_tmp3", None) is None:
            self._tmp3 = nat.DevState(self._eng, self._cur.cap, 0, self._cur.amp_type)
        return self._tmp3

    def _phase_2q(self, diag, q1, q2):
        eng = self._eng
        d = nat.host_c128(diag)
        nat.check(eng.L.bass_phase_2q(self._cur.ptr, nat._host(d), int(q1), int(q2), eng.ctrl_ptr, eng.stream),
                  "bass_phase_2q")
        self._touch()

    def _topk(self, tr):
        eng = self._eng
        nat.check(eng.L.bass_topk(self._cur.ptr, self._tmp.ptr, tr, eng.ctrl_ptr, eng.ws_ptr, eng.ws_bytes,
                                  eng.stream), "bass_topk")
        nat.swap(self._cur, self._tmp)
        self._rekeyed()

    def _renorm(self, trace=0):
        eng = self._eng
        nat.check(eng.L.bass_renorm(self._cur.ptr, int(trace), eng.ctrl_ptr, eng.ws_ptr, eng.ws_bytes,
                                    eng.stream), "bass_renorm")
        self._touch()

    def _norm2(self) -> float:
        eng = self._eng
        nat.check(eng.L.bass_norm2(self._cur.ptr, nat.ctypes.c_void_p(nat._ptr(eng.scratch_f64)), eng.ws_ptr,
                                   eng.ws_bytes, eng.stream), "bass_norm2")
        return float(eng.scratch_f64[0].item())

    def _pr(self) -> float:
        """bass_simulator.py:574-578 (synchronising)."""
        eng = self._eng
        nat.check(eng.L.bass_pr(self._cur.ptr, eng.ctrl_ptr, eng.ws_ptr, eng.ws_bytes, eng.stream), "bass_pr")
        return float(eng.read_ctrl()["pr_last"])

    def _gather_sorted(self, idx):
        eng = self._eng
        torch = eng.torch
        idx = np.sort(np.asarray(idx, dtype=np.int64))
        t = torch.from_numpy(idx).to(eng.device)
        nat.check(eng.L.bass_gather(self._cur.ptr, self._tmp.ptr, nat.ctypes.c_void_p(nat._ptr(t)), len(idx),
                                    eng.ctrl_ptr, eng.stream), "bass_gather")
        torch.cuda.current_stream(eng.device).synchronize()
        nat.swap(self._cur, self._tmp)
        self._rekeyed()

    # ---- reference API ------------------------------------------------------------
    def apply_gate(self, gate, method="top-k", seed="None"):
        """sparse_state.py:379-385: expand, merge duplicates, then truncate to k
        (top-k: gamma *= sqrt(kept), alpha /= sqrt(kept); random-k: LCG)."""
        tr = nat.trunc(self.k, self.k, 3, 2) if method == "top-k" else nat.NO_TRUNC
        if gate.n_qubits == 1:
            # a diagonal gate cannot grow the state, so the phase path needs no truncation
            self._apply_1q(gate.matrix, gate.qubits[0], tr)
        elif gate.n_qubits == 2:
            self._apply_2q(gate.matrix, gate.qubits[0], gate.qubits[1], tr)
        else:
            raise NotImplementedError("Only 1- and 2-qubit gates supported")
        if method != "top-k" and self.nnz > self.k:
            self.truncate_random_k(seed)

    def apply_single_qubit_gate(self, gate, method, seed):
        self.apply_gate(gate, method, seed)

    def apply_two_qubit_gate(self, gate, method, seed):
        self.apply_gate(gate, method, seed)

    def truncate_top_k(self):
        """sparse_state.py:388-400 / truncation.py:68-113."""
        self._topk(nat.trunc(self.k, self.k, 3, 2))

    def truncate_random_k(self, seed):
        """sparse_state.py:402-415 / truncation.py:116-159: the LCG partial
        Fisher-Yates picks k entries by their index in the array, in the
        reference's entry order (key order after a gate, the drawn order after
        an earlier random-k truncation); the drawn entries keep the order of
        the draw.  Host-driven: export, choose, re-import."""
        n = self.nnz
        if n <= self.k:
            return
        if seed is None:
            seed = int(np.random.randint(0, 2 ** 31))
        x, a = self._in_order()
        idx = np.empty(self.k, dtype=np.int64)
        nat.check(self._eng.L.bass_lcg_choose(n, self.k, int(seed), nat._host(idx)), "bass_lcg_choose")
        self._load_in_order(x[idx], a[idx])
        gsq = self._norm2()
        gl = float(np.sqrt(gsq))
        self._renorm()
        self.gamma = self.gamma * gl
