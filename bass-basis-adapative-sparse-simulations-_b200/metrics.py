"""Fidelity and sparsity metrics (src/benchmarking/fidelity.py:48-102 and
src/experimentation/runner.py:620-626), on the device for device vectors.

Each function takes the same arguments as the reference's.  An exact state
given as a device tensor (torch, on the state's GPU) is read there: the
overlaps are exact sums on the device (bass_sparse_dot / bass_dense_dot).  A
host numpy array takes the reference's own numpy formula.
"""
from __future__ import annotations

import numpy as np

from . import _native as nat


def _is_device(v) -> bool:
    return hasattr(v, "is_cuda") and v.is_cuda


def _out2(eng):
    v = eng.scratch_f64[:2].cpu().numpy()
    return complex(v[0], v[1])


def sparse_overlap(sparse_state, exact_state) -> complex:
    """sum over the state's entries of conj(exact[x]) a_x."""
    if _is_device(exact_state):
        eng = sparse_state._eng
        psi = exact_state.contiguous()
        nat.check(eng.L.bass_sparse_dot(sparse_state._cur.ptr, nat.ctypes.c_void_p(psi.data_ptr()),
                                        int(sparse_state.N), nat.ctypes.c_void_p(nat._ptr(eng.scratch_f64)),
                                        eng.ctrl_ptr, eng.ws_ptr, eng.ws_bytes, eng.stream), "bass_sparse_dot")
        out = _out2(eng)
        eng.check_errors()
        return out
    xs = sparse_state.x[: sparse_state.nnz]
    alphas = sparse_state.alpha[: sparse_state.nnz]
    return complex(np.dot(np.asarray(exact_state)[xs.astype(np.int64)].conj(), alphas))


def dense_overlap(u, v, eng=None) -> complex:
    """np.vdot(u, v); exact on the device when both are device tensors."""
    if _is_device(u) and _is_device(v):
        if eng is None:
            raise ValueError("dense_overlap of device tensors needs the state's engine")
        if u.numel() != v.numel():
            raise ValueError("length mismatch")
        u, v = u.contiguous(), v.contiguous()
        nat.check(eng.L.bass_dense_dot(nat.ctypes.c_void_p(u.data_ptr()), nat.ctypes.c_void_p(v.data_ptr()),
                                       int(u.numel()), nat.ctypes.c_void_p(nat._ptr(eng.scratch_f64)),
                                       eng.ctrl_ptr, eng.ws_ptr, eng.ws_bytes, eng.stream), "bass_dense_dot")
        return _out2(eng)
    return complex(np.vdot(np.asarray(u), np.asarray(v)))


# fidelity.py:48-68
def compute_fidelity(sparse_state, exact_state) -> float:
    return float(abs(sparse_overlap(sparse_state, exact_state)) ** 2)


# fidelity.py:71-79
def compute_fidelity_bounds(sparse_state):
    return sparse_state.gamma ** 2, 1.0


# fidelity.py:82-92
def compute_participation_ratio(sparse_state) -> float:
    if sparse_state.nnz == 0:
        return float("inf")
    return float(sparse_state._pr())


# fidelity.py:95-102
def estimate_cross_entropy_fidelity(sparse_state, exact_state, num_samples=1000) -> float:
    samples = sparse_state.sample(num_samples)
    if _is_device(exact_state):
        torch = sparse_state._eng.torch
        idx = torch.as_tensor(samples.astype(np.int64), device=exact_state.device)
        probs = (exact_state[idx].abs() ** 2).cpu().numpy()
    else:
        probs = np.abs(np.asarray(exact_state)[samples.astype(np.int64)]) ** 2
    return float(2 ** sparse_state.N * np.mean(probs) - 1)


# runner.py:620-626 fidelity_bass, with the statevector built on the device;
# like the reference it reports 0.0 above 24 qubits (no exact state there)
def fidelity_bass(sim, state, exact_sv) -> float:
    if sim.N > 24:
        return 0.0
    psi = sim.to_statevector_device(state)
    if not _is_device(exact_sv):
        exact_sv = psi.new_tensor(np.asarray(exact_sv))
    return float(abs(dense_overlap(exact_sv, psi, state._eng)) ** 2)
