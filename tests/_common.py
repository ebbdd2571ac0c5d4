"""Helpers shared by the test modules (golden fixture loading, event comparison)."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

BASS_CASES = ["bass_tfim_n10_k32", "bass_brick_n12_k64", "bass_brick_n16_k256_opt1",
              "bass_haar2q_n12_k128", "bass_brick_n20_k512_trunc2"]
LARGE_CASES = ["config1_tfim_n24_k65536", "config2_brick_n40_d30_k1024", "config2_brick_n40_d12_k4096",
               "config2_brick_n40_d10_k16384"]
# fixtures whose every event matches in full: the fingerprint of all keys too,
# not only of the keys with |a|^2 > 1e-24.  In the others a few events differ
# in entries below that threshold, which the reference's |a|^2 (hypot squared)
# and ours (re^2 + im^2) round differently.
FULL_MATCH_CASES = ["bass_tfim_n10_k32", "bass_haar2q_n12_k128", "bass_brick_n20_k512_trunc2",
                    "config1_tfim_n24_k65536", "config2_brick_n40_d12_k4096", "config2_brick_n40_d10_k16384",
                    "bass2q_tfim_n10_k48"]
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


_M1 = np.uint64(0xff51afd7ed558ccd)
_M2 = np.uint64(0xc4ceb9fe1a85ec53)


def fmix64(z):
    """murmur3's 64-bit finaliser on a uint64 array (wrapping arithmetic)."""
    z = np.asarray(z, dtype=np.uint64).copy()
    with np.errstate(over="ignore"):
        z ^= z >> np.uint64(33)
        z *= _M1
        z ^= z >> np.uint64(33)
        z *= _M2
        z ^= z >> np.uint64(33)
    return z


def pair_fingerprint(x, a):
    """Order-independent fingerprint of a state's (key, amplitude) pairs:
    (count, sum, xor) over entries of fmix64(key ^ fmix64(re bits ^
    fmix64(im bits))).  Equal fingerprints mean equal key sets with
    bit-identical amplitudes, up to a 64-bit hash collision."""
    x = np.ascontiguousarray(x, dtype=np.uint64)
    a = np.ascontiguousarray(a, dtype=np.complex128)
    bits = a.view(np.uint64).reshape(-1, 2)
    h = fmix64(x ^ fmix64(bits[:, 0] ^ fmix64(bits[:, 1])))
    with np.errstate(over="ignore"):
        s = int(np.sum(h, dtype=np.uint64)) if len(h) else 0
    z = int(np.bitwise_xor.reduce(h)) if len(h) else 0
    return len(x), s, z


def full_events(ev):
    """A trace as a list of 7-tuples (every column compared)."""
    return [tuple(int(v) for v in e) for e in np.asarray(ev, dtype=np.uint64).reshape(-1, 7)]


def agreeing_prefix(a, b):
    """Length of the common prefix of two event lists."""
    m = first_mismatch(a, b)
    return min(len(a), len(b)) if m is None else m
