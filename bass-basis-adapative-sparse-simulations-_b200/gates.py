"""Gate objects with the reference's interface and angle conventions.

Mirrors src/core/gates.py of the reference: a gate is ``qubits`` (a tuple, not
sorted), ``matrix`` (complex128, 2^n x 2^n) and ``n_qubits``.  The 2-qubit
matrix index is ``(bit_q1 << 1) | bit_q2`` (src/core/sparse_state.py:96-98).
The named rotations keep the reference's conventions, which differ from the
usual half-angle ones:

  RXGate(theta)  = exp(+i theta X)             (gates.py:106-111)
  RZZGate(theta) = exp(+i theta Z (x) Z)       (gates.py:115-120)
  RZGate(theta)  = exp(-i theta Z / 2)         (gates.py:124-128)
  RYGate(theta)  = exp(-i theta Y / 2)         (gates.py:133-137)

Matrices are built with the same numpy expressions as the reference so that a
given angle yields bit-identical complex128 entries.  Any object exposing
``qubits``, ``matrix`` and ``n_qubits`` (the reference's own gate objects
included) is accepted by the simulators.
"""
from __future__ import annotations

import numpy as np


class QuantumGate:
    """Base class: ``QuantumGate(qubits, matrix)`` (gates.py:6-23)."""

    def __init__(self, qubits, matrix):
        self.qubits = tuple(qubits)
        self.matrix = np.array(matrix, dtype=np.complex128)
        self.n_qubits = len(qubits)
        dim = 2 ** self.n_qubits
        assert self.matrix.shape == (dim, dim), "Matrix dimension mismatch"

    def __repr__(self):
        return f"{self.__class__.__name__}(qubits={self.qubits})"


class SingleQubitGate(QuantumGate):
    def __init__(self, qubit, matrix):
        super().__init__((qubit,), matrix)


class TwoQubitGate(QuantumGate):
    def __init__(self, qubit1, qubit2, matrix):
        super().__init__((qubit1, qubit2), matrix)


class HGate(SingleQubitGate):
    def __init__(self, qubit):
        super().__init__(qubit, np.array([[1, 1], [1, -1]]) / np.sqrt(2))


class XGate(SingleQubitGate):
    def __init__(self, qubit):
        super().__init__(qubit, np.array([[0, 1], [1, 0]]))


class YGate(SingleQubitGate):
    def __init__(self, qubit):
        super().__init__(qubit, np.array([[0, -1j], [1j, 0]]))


class ZGate(SingleQubitGate):
    def __init__(self, qubit):
        super().__init__(qubit, np.array([[1, 0], [0, -1]]))


class SGate(SingleQubitGate):
    def __init__(self, qubit):
        super().__init__(qubit, np.array([[1, 0], [0, 1j]]))


class TGate(SingleQubitGate):
    def __init__(self, qubit):
        super().__init__(qubit, np.array([[1, 0], [0, np.exp(1j * np.pi / 4)]]))


class CNOTGate(TwoQubitGate):
    def __init__(self, control, target):
        super().__init__(control, target,
                         np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0]]))


class CZGate(TwoQubitGate):
    def __init__(self, qubit1, qubit2):
        super().__init__(qubit1, qubit2, np.diag([1, 1, 1, -1]))


class RXGate(SingleQubitGate):
    """exp(+i theta X)."""

    def __init__(self, qubit, theta):
        c, s = np.cos(theta), np.sin(theta)
        super().__init__(qubit, np.array([[c, 1j * s], [1j * s, c]], dtype=np.complex128))


class RZZGate(TwoQubitGate):
    """exp(+i theta Z (x) Z), diagonal."""

    def __init__(self, qubit1, qubit2, theta):
        p, m = np.exp(1j * theta), np.exp(-1j * theta)
        super().__init__(qubit1, qubit2, np.diag([p, m, m, p]).astype(np.complex128))


class RZGate(SingleQubitGate):
    """exp(-i theta Z / 2)."""

    def __init__(self, qubit, theta):
        p, m = np.exp(-1j * theta / 2), np.exp(1j * theta / 2)
        super().__init__(qubit, np.array([[p, 0], [0, m]], dtype=np.complex128))


class RYGate(SingleQubitGate):
    """exp(-i theta Y / 2)."""

    def __init__(self, qubit, theta):
        c, s = np.cos(theta / 2), np.sin(theta / 2)
        super().__init__(qubit, np.array([[c, -s], [s, c]], dtype=np.complex128))


def haar_random_unitary(dimension, seed=None):
    """Haar-random U(dimension); seeds the global numpy RNG like the reference
    (gates.py:152-164) and draws with scipy.stats.unitary_group."""
    from scipy.stats import unitary_group
    if seed is not None:
        np.random.seed(seed)
    return unitary_group.rvs(dimension)


class RandomTwoQubitGate(TwoQubitGate):
    """Haar-random 2-qubit gate (gates.py:142-149)."""

    def __init__(self, qubit1, qubit2, seed=None):
        super().__init__(qubit1, qubit2, haar_random_unitary(4, seed))
