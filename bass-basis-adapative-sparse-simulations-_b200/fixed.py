"""FixedBasisSimulator on the GPU -- drop-in for src/simulation/simulator.py:61-253.

No basis frame: 2-qubit gates go through the hash-merge gate followed by the
simulate-level truncation (top-k: gamma *= sqrt(kept/total), renormalise;
random-k: numpy's seeded weighted choice), 1-qubit gates through
SparseState.apply_gate.  The per-gate seed follows the same LCG
(simulator.py:158).  gamma and nnz histories are recorded on the device and
read once at the end; per-gate runtimes come from CUDA events.

Random-k draws entries by their index, so the entry order matters there.  The
reference's hash-table gate (bass_simulator.py:292-354) emits its output in
first-occurrence order over the input entries (input order, then output
index 0-3), and the weighted choice keeps the drawn order.  The device state
is key-sorted, so in random-k mode that order is tracked on the host
(``ht_order`` below, ``SparseState._set_order``) and the choice runs over the
entries in it.
"""
from __future__ import annotations

import numpy as np

from . import _native as nat
from .state import SparseState


def ht_order(x, a, G, q1, q2):
    """The output keys of apply_2qubit_gate_ht (bass_simulator.py:292-354) in
    the order it emits them: input entries in their order, for each the
    output indices 0-3 whose product G[out, in] * a is not exactly zero; a
    key's position is that of its first occurrence."""
    x = np.asarray(x, dtype=np.uint64)
    a = np.asarray(a, dtype=np.complex128)
    G = np.asarray(G, dtype=np.complex128)
    if len(x) == 0:
        return x.copy()
    s1, s2 = np.uint64(q1), np.uint64(q2)
    m1, m2 = np.uint64(1) << s1, np.uint64(1) << s2
    one = np.uint64(1)
    in_idx = (((x >> s1) & one) << one | ((x >> s2) & one)).astype(np.int64)
    base = x & ~(m1 | m2)
    keys = np.empty((len(x), 4), dtype=np.uint64)
    live = np.empty((len(x), 4), dtype=bool)
    for o in range(4):
        keys[:, o] = base | (m1 if o >> 1 else np.uint64(0)) | (m2 if o & 1 else np.uint64(0))
        prod = G[o, in_idx] * a
        live[:, o] = (prod.real != 0.0) | (prod.imag != 0.0)
    flat = keys[live]   # row-major: input order, then output index
    u, first = np.unique(flat, return_index=True)
    return u[np.argsort(first, kind="stable")]


class FixedBasisSimulator:
    def __init__(self, num_qubits, k, truncation="top-k", verbose=True, log_every=1, max_nnz_factor=8):
        self.N = num_qubits
        self.k = k
        self.verbose = verbose
        self.log_every = log_every
        if truncation not in ["top-k", "random-k"]:
            raise ValueError("Unknown truncation")
        self._truncate_name = truncation
        self.max_nnz_factor = max_nnz_factor

    def _random_k_2q(self, state, cur_seed):
        """simulator.py:177-196, over the entries in the reference's order."""
        x, a = state._in_order()
        probs = np.abs(a) ** 2
        total = np.sum(probs)
        np.random.seed(cur_seed)
        pn = probs / total if total > 1e-30 else np.ones(len(a)) / len(a)
        idx = np.random.choice(len(a), size=self.k, replace=False, p=pn)
        kept = np.sum(probs[idx])
        state._load_in_order(x[idx], a[idx])
        state.gamma = state.gamma * (np.sqrt(kept / total) if total > 1e-30 else 0)
        state._renorm()

    def simulate(self, circuit, initial_state=None, seed=None):
        import torch
        state = SparseState(self.N, self.k, initial_state)
        eng = state._eng
        L = len(circuit)
        dev = eng.device
        gamma_hist = torch.empty(L + 1, dtype=torch.float64, device=dev)
        nnz_hist = torch.empty(L + 1, dtype=torch.int64, device=dev)
        gamma_hist[0] = 1.0
        nnz_hist[0] = 1
        g_view = eng.ctrl_field("state_gamma", np.float64).view(torch.float64)
        events = [torch.cuda.Event(enable_timing=True) for _ in range(L + 1)]
        events[0].record()
        if seed is None:
            seed = int(np.random.randint(0, 2 ** 31))
        cur = seed
        topk = self._truncate_name == "top-k"
        for i, gate in enumerate(circuit):
            cur = (1103515245 * cur + 12345) & 0x7FFFFFFF
            if gate.n_qubits == 2:
                q1, q2 = gate.qubits
                if topk:
                    state._apply_2q(gate.matrix, q1, q2, nat.trunc(self.k, self.k, 2, 1))
                else:
                    xin, ain = state._in_order()
                    order = ht_order(xin, ain, gate.matrix, q1, q2)
                    state._apply_2q(gate.matrix, q1, q2, nat.NO_TRUNC)
                    state._set_order(order)
                    if state.nnz > self.k:
                        self._random_k_2q(state, cur)
            else:
                state.apply_gate(gate, self._truncate_name, cur)
            gamma_hist[i + 1].copy_(g_view[0])
            nnz_hist[i + 1].copy_(state._cur.nnz_view()[0])
            events[i + 1].record()
            if self.verbose and (i % self.log_every == 0):
                print(f"[Gate {i + 1}/{L}] type={gate.n_qubits}q | nnz: {int(nnz_hist[i + 1])} | "
                      f"γ²={float(gamma_hist[i + 1]) ** 2:.6e}")
        torch.cuda.synchronize(dev)
        eng.raise_on_error()
        self.runtime_per_gate = np.array([events[i].elapsed_time(events[i + 1]) / 1e3 for i in range(L)])
        self.gamma_history = gamma_hist.cpu().numpy()
        self.nnz_history = nnz_hist.cpu().numpy().astype(np.float64)
        return state

    def get_metrics(self):
        return {
            "runtime_per_gate": self.runtime_per_gate,
            "gamma_squared": self.gamma_history ** 2,
            "nnz": self.nnz_history,
            "total_runtime": self.runtime_per_gate.sum(),
            "avg_runtime_per_gate": self.runtime_per_gate.mean(),
        }
