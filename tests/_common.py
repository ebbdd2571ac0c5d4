"""Helpers shared by the test modules (golden fixture loading, event comparison)."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

BASS_CASES = ["bass_tfim_n10_k32", "bass_brick_n12_k64", "bass_brick_n16_k256_opt1",
              "bass_haar2q_n12_k128", "bass_brick_n20_k512_trunc2"]
LARGE_CASES = ["config1_tfim_n24_k65536", "config2_brick_n40_d30_k1024", "config2_brick_n40_d12_k4096"]
BASS2Q_CASES = ["bass2q_brick_n10_k32", "bass2q_tfim_n10_k48"]   # use_2qubit_rotations=True


class Gate:
    """A gate rebuilt from a fixture row (duck-types the reference's gates)."""

    def __init__(self, meta, mat):
        self.n_qubits = int(meta[0])
        self.qubits = (int(meta[1]),) if self.n_qubits == 1 else (int(meta[1]), int(meta[2]))
        d = 2 ** self.n_qubits
        self.matrix = np.ascontiguousarray(mat[:d, :d])


def load_case(name):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    circ = [Gate(m, g) for m, g in zip(z["gate_meta"], z["gate_mats"])]
    kw = eval(str(z["kwargs"])) if "kwargs" in z else {}
    return z, circ, kw


def sig_events(ev):
    """Comparable view of a trace: renorm events by their significant-key
    fingerprint, accept/opt events by (type, index)."""
    ev = np.asarray(ev, dtype=np.uint64).reshape(-1, 7)
    out = []
    for e in ev:
        if int(e[0]) == 0:
            out.append((0, int(e[4]), int(e[5]), int(e[6])))
        else:
            out.append((int(e[0]), int(e[1])))
    return out


def first_mismatch(a, b):
    for i in range(min(len(a), len(b))):
        if a[i] != b[i]:
            return i
    return None if len(a) == len(b) else min(len(a), len(b))


def sorted_state(x, a):
    x = np.asarray(x, dtype=np.uint64)
    o = np.argsort(x, kind="stable")
    return x[o], np.asarray(a)[o]
