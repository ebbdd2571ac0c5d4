"""BASS on the GPU -- drop-in for src/simulation/bass_simulator.py:478-929.

The per-gate driver stays on the host and follows ``BASS.simulate``
(bass_simulator.py:847-929) step by step: frames U_j and the conjugated gate
matrices are numpy (bit-identical to the reference's), every per-entry step
is a CUDA kernel.  The host synchronises only where the reference's control
flow reads a state-dependent value: at each optimisation point (is a
truncation pending, has PR grown), once per optimisation pass (the RDMs for
the 2x2 eigen-solves; the accept flags of the pass), and, when
``truncate_every > 1``, after every non-diagonal gate (the truncation rule then
depends on nnz).  With the default ``truncate_every=1`` the simulate-level
truncation (keep the top k, gamma_running *= kept/total, renormalise) is
fused into the gate's kernels and decided on the device.

Precision form: ``dtype=np.complex64`` stores the amplitudes as complex64
(16-byte entries instead of 24).  Gate and rotation arithmetic is then FP32
with compensated products and sums (each output rounded once), while |a|^2,
the norm, the top-k threshold, the discarded weight, the PR and the RDM
moments behind the rotation-angle solve stay FP64 (exact sums on the device,
the 2x2 eigen-solve and the frames on the host).  ``record_truncations=True``
keeps, per simulate-level truncation, (gate index, kept mass, total mass) in
``self.truncations`` (one synchronising read per gate, for reports).

One deliberate difference: a basis rotation is kept only if it lowers the
participation ratio by more than ``pr_tie_tol`` (relative, default 1e-12).
The reference keeps it on any decrease, so rotations that leave PR unchanged
up to rounding (a pure relabel of a qubit, for instance) are decided there by
the summation order of np.sum; with pr_tie_tol=0 the rule is the reference's.
"""
from __future__ import annotations

import numpy as np

from . import _native as nat
from .linalg import eigh_2x2, eigh_numpy, is_gate_diagonal, kron_2x2
from .state import SparseState


class BASS:
    def __init__(self, num_qubits, k, optimize_every=5, buffer_factor=2, truncate_every=1, max_nnz_factor=8,
                 use_2qubit_rotations=False, verbose=False, use_fast_eigh=True, use_diag_gate=True,
                 use_kron_cache=True, pr_opt_threshold=0.90, *, pr_tie_tol=1e-12, trace=False,
                 trace_cap=None, dtype=np.complex128, record_truncations=False):
        self.N = num_qubits
        self.k = k
        self.optimize_every = optimize_every
        self.buffer_factor = buffer_factor
        self.verbose = verbose
        self.use_fast_eigh = use_fast_eigh
        self.use_diag_gate = use_diag_gate
        self.use_kron_cache = use_kron_cache
        self.truncate_every = truncate_every
        self.max_nnz_factor = max_nnz_factor
        self.use_2qubit_rotations = use_2qubit_rotations
        self.pr_opt_threshold = pr_opt_threshold
        self.pr_tie_tol = pr_tie_tol
        self.trace = bool(trace)
        self.trace_cap = trace_cap
        self.dtype = np.dtype(dtype)
        nat.amp_type_of(self.dtype)
        self.record_truncations = bool(record_truncations)
        self.truncations = []
        self._kron_cache = {}
        self.U = None
        self._gamma_running = 1.0
        self._pr_at_last_opt = 0.0
        self.stats = {}
        self.last_state = None

    # bass_simulator.py:580-593
    def _get_kron(self, q1, q2):
        if not self.use_kron_cache:
            return kron_2x2(self.U[q1], self.U[q2])
        key = (q1, q2)
        if key not in self._kron_cache:
            self._kron_cache[key] = kron_2x2(self.U[q1], self.U[q2])
        return self._kron_cache[key]

    def _invalidate_kron(self, qubit):
        for key in [kk for kk in self._kron_cache if qubit in kk]:
            del self._kron_cache[key]

    # bass_simulator.py:829-845
    def optimize_trigger(self, state):
        if self.pr_opt_threshold >= 1.0:
            return True
        return state._pr() > self._pr_at_last_opt / self.pr_opt_threshold

    # bass_simulator.py:730-827 (1-qubit coordinate descent)
    def _optimize_basis(self, state, gate_index=-1, pr=None):
        """pr: the state's PR when the caller has just computed it."""
        eng = state._eng
        if (state._pr() if pr is None else pr) < self.k / 4:
            return
        self.stats["opt_calls"] += 1
        if self.trace:
            eng.append_trace((2, gate_index, 0, 0, 0, 0, 0))
        N = self.N
        for _pass in range(3):
            nat.check(eng.L.bass_rdm_1q(state._cur.ptr, N, nat.ctypes.c_void_p(nat._ptr(eng.rho)), eng.ctrl_ptr,
                                        eng.ws_ptr, eng.ws_bytes, eng.stream), "bass_rdm_1q")
            nat.check(eng.L.bass_pr(state._cur.ptr, eng.ctrl_ptr, eng.ws_ptr, eng.ws_bytes, eng.stream), "bass_pr")
            r = eng.rho[:4 * N].cpu().numpy().reshape(N, 4)
            tried = {}
            for j in range(N):
                c01 = complex(r[j, 2], r[j, 3])
                rho = np.array([[r[j, 0], c01], [c01.conjugate(), r[j, 1]]], dtype=np.complex128)
                _, V = eigh_2x2(rho) if self.use_fast_eigh else eigh_numpy(rho)
                if abs(V[0, 1]) + abs(V[1, 0]) < 1e-10:
                    continue
                tried[j] = V
                u = nat.host_c128(V.conj().T)
                nat.check(eng.L.bass_rotate_step(state._cur.ptr, state._tmp.ptr, nat._host(u), j, self.k,
                                                 int(self.trace), eng.ctrl_ptr, eng.ws_ptr, eng.ws_bytes,
                                                 eng.stream), "bass_rotate_step")
            state._touch()
            improved = False
            if tried:
                c = eng.read_ctrl()
                for j, V in tried.items():
                    self.stats["rotations"] += 1
                    if c["accept"][j]:
                        self.U[j] = self.U[j] @ V
                        self._invalidate_kron(j)
                        improved = True
                        self.stats["accepted"] += 1
            if not improved:
                break
        if self.use_2qubit_rotations and self.N >= 2:     # bass_simulator.py:819-824
            self._optimize_2q_pass(state, [(i, i + 1) for i in range(0, self.N - 1, 2)])
            self._optimize_2q_pass(state, [(i, i + 1) for i in range(1, self.N - 1, 2)])
        state._topk(nat.trunc(self.k, self.k))   # _truncate_state
        state._renorm(int(self.trace))           # _renorm

    # bass_simulator.py:679-728
    def _optimize_2q_pass(self, state, pairs):
        """Brick-wall 2-qubit truncation alignment: per pair, rotate into the
        eigenbasis of its 4x4 RDM, truncate, rotate back, truncate; keep the
        result if PR drops by more than pr_tie_tol (relative; the reference
        keeps it unless PR rose), with gamma *= sqrt(frac1 * frac2)."""
        eng = state._eng
        tr = nat.trunc(self.k, self.k)             # _truncate_state, fused into each rotation
        for q1, q2 in pairs:
            rho = state._rdm_2q(q1, q2)
            evals, evecs = np.linalg.eigh(rho)
            V = evecs[:, np.argsort(-evals)]
            pr_before = state._pr()
            state._rotate_2q(V.conj().T, q1, q2, tr)
            spare = state._spare()
            nat.swap(state._tmp2, spare)           # the saved state, until the decision
            frac1 = state._norm2()
            state._renorm(int(self.trace))
            state._rotate_2q(V, q1, q2, tr)
            frac2 = state._norm2()
            state._renorm(int(self.trace))
            pr_after = state._pr()
            if pr_after > pr_before * (1.0 - self.pr_tie_tol):
                nat.swap(state._cur, spare)        # restore
                state._touch()
            else:
                g = float(eng.read_ctrl()["gamma_running"])
                eng.set_ctrl("gamma_running", g * np.sqrt(frac1 * frac2))

    def _general_truncation(self, state, hard_cap, gates_since):
        """The simulate-level truncation rule when truncate_every > 1 (host decides)."""
        n = state.nnz
        over_hard = n > hard_cap
        over_budget = n > self.k
        if over_hard or (over_budget and gates_since >= self.truncate_every):
            state._topk(nat.trunc(self.k, self.k, 1, 1, 1, int(self.trace)))
            return 0
        return gates_since

    # bass_simulator.py:847-929
    def simulate(self, circuit, initial_state=0):
        N, k = self.N, self.k
        self.U = [np.eye(2, dtype=np.complex128) for _ in range(N)]
        self._kron_cache = {}
        self._pr_at_last_opt = 0.0
        self.stats = {"gates": 0, "rotations": 0, "accepted": 0, "opt_calls": 0}
        hard_cap = min(self.max_nnz_factor * k, 2 ** N)
        internal_k = min(max(max(self.buffer_factor, 2) * k, hard_cap), 2 ** N)
        fast = self.truncate_every == 1
        cap = (min(k, 2 ** N) + 16) if fast else 4 * hard_cap + 16
        tcap = self.trace_cap if self.trace_cap is not None else (4 * len(circuit) * (N + 4) + 1024 if self.trace else 0)
        state = SparseState(N, internal_k, initial_state, dtype=self.dtype, _capacity=cap, _trace_cap=tcap)
        eng = state._eng
        M = len(circuit)
        gates_since = 0
        tr_flag = int(self.trace)
        fused = nat.trunc(k, k, 1, 1, 1, tr_flag)
        internal = nat.trunc(internal_k, internal_k, 3, 2, 0, 0)
        self.truncations = []
        n_trunc_seen = 0
        for i, gate in enumerate(circuit):
            if self.record_truncations and i > 0:
                n_trunc_seen = self._record(eng, i - 1, n_trunc_seen)
            self.stats["gates"] += 1
            if gate.n_qubits == 1:
                q = gate.qubits[0]
                G = self.U[q].conj().T @ gate.matrix @ self.U[q]
                if fast:
                    state._apply_1q(G, q, fused)
                else:
                    state._apply_1q(G, q, internal)
                    gates_since += 1
                    gates_since = self._general_truncation(state, hard_cap, gates_since)
            elif gate.n_qubits == 2:
                q1, q2 = gate.qubits
                Ut = self._get_kron(q1, q2)
                G = Ut.conj().T @ gate.matrix @ Ut
                if self.use_diag_gate and is_gate_diagonal(G):
                    state._phase_2q(np.diag(G).astype(np.complex128), q1, q2)
                    self._maybe_optimize(state, i, M)
                    continue
                if fast:
                    state._apply_2q(G, q1, q2, fused)
                else:
                    state._apply_2q(G, q1, q2, nat.NO_TRUNC)
                    gates_since += 1
                    gates_since = self._general_truncation(state, hard_cap, gates_since)
            else:
                raise ValueError(f"{gate.n_qubits}-qubit gates unsupported")
            self._maybe_optimize(state, i, M)
        if self.record_truncations and M:
            self._record(eng, M - 1, n_trunc_seen)
        c = eng.read_ctrl()
        eng.raise_on_error()
        self._gamma_running = float(c["gamma_running"])
        state.gamma = np.sqrt(max(self._gamma_running, 0))
        self.stats["amp_updates"] = int(c["amp_updates"])
        self.stats["truncations"] = int(c["n_trunc"])
        self.last_state = state
        return state

    def _record(self, eng, i, seen):
        """Append gate i's simulate-level truncation, if it made one."""
        c = eng.read_ctrl()
        n = int(c["n_trunc"])
        if n > seen and int(c["last_truncated"]):
            self.truncations.append((i, float(c["last_kept"]), float(c["last_total"])))
        return n

    def _maybe_optimize(self, state, i, M):
        """bass_simulator.py:917-925: every optimize_every gates, if a
        truncation happened since the last check and PR has grown past the
        trigger (optimize_trigger), optimise the basis.  The PR reduction is
        launched before the one synchronising read of the control block, so
        the flag and the PR arrive together."""
        if self.optimize_every > 0 and (i + 1) % self.optimize_every == 0 and i + 1 < M:
            eng = state._eng
            nat.check(eng.L.bass_pr(state._cur.ptr, eng.ctrl_ptr, eng.ws_ptr, eng.ws_bytes, eng.stream), "bass_pr")
            c = eng.read_ctrl()
            if int(c["truncation_active"]):
                pr = float(c["pr_last"])
                if self.pr_opt_threshold >= 1.0 or pr > self._pr_at_last_opt / self.pr_opt_threshold:
                    self._optimize_basis(state, i, pr=pr)
                    self._pr_at_last_opt = state._pr()
            eng.set_ctrl("truncation_active", 0)

    # bass_simulator.py:608-621
    def to_statevector(self, state):
        if self.N > 24:
            raise ValueError(f"N={self.N} too large for statevector")
        psi = np.zeros(2 ** self.N, dtype=np.complex128)
        x, a = state.x, state.alpha
        psi[x.astype(np.int64)] = a
        for j in range(self.N):
            psi3d = psi.reshape(-1, 2, 1 << j)
            psi = np.einsum("ij,kjl->kil", self.U[j], psi3d).reshape(-1)
        return psi

    def to_statevector_device(self, state):
        """to_statevector on the device (torch complex128), for N <= 30."""
        return state.to_dense_device(U=self.U)

    def trace_events(self):
        """The device trace of the last simulate() call (trace=True)."""
        if self.last_state is None:
            return np.zeros((0, nat.TRACE_WORDS), np.uint64)
        return self.last_state._eng.trace_events()
