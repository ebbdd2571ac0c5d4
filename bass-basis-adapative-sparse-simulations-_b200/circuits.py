"""Seeded circuit generators for the benchmark workloads.

``tfim_circuit`` draws exactly like the reference's ``generate_tfim_circuit``
(src/utils/random_circuits.py:100-165): per Trotter layer one
``rng.uniform(J-dJ, J+dJ, N-1)`` draw for the couplings, then one
``rng.uniform(h-dh, h+dh, N)`` draw for the fields, then RZZ on (i, i+1) and
RX on every qubit.  The same ``numpy.random.Generator`` therefore yields the
same gate list as the reference.

``brickwork_circuit`` is the 1D brickwork workload (the reference has no
generator for it): per layer a Haar-random SU(2) on every qubit (a complex
Gaussian 2x2, QR, columns phase-fixed by diag(R)/|diag(R)|, divided by
sqrt(det)), then CZ on the pairs (i, i+1) with i = layer (mod 2), each pair
skipped with probability 1/2.  All draws come from one generator, in that
order.
"""
from __future__ import annotations

import numpy as np

from .gates import CZGate, RXGate, RZZGate, SingleQubitGate


def tfim_circuit(num_qubits, num_layers, J=1.0, h=3.0, dt=0.3, rng=None,
                 disorder_strength_J=0.0, disorder_strength_h=0.0):
    if rng is None:
        rng = np.random.default_rng(0)
    circuit = []
    for _ in range(num_layers):
        J_vals = rng.uniform(J - disorder_strength_J, J + disorder_strength_J, size=num_qubits - 1)
        h_vals = rng.uniform(h - disorder_strength_h, h + disorder_strength_h, size=num_qubits)
        for i in range(num_qubits - 1):
            circuit.append(RZZGate(i, i + 1, J_vals[i] * dt))
        for i in range(num_qubits):
            circuit.append(RXGate(i, h_vals[i] * dt))
    return circuit


def haar_su2(rng) -> np.ndarray:
    """Haar-random SU(2) from one seeded generator (QR of a complex Gaussian)."""
    z = (rng.standard_normal((2, 2)) + 1j * rng.standard_normal((2, 2))) / np.sqrt(2.0)
    q, r = np.linalg.qr(z)
    d = np.diag(r)
    q = q * (d / np.abs(d))
    return q / np.sqrt(np.linalg.det(q))


def brickwork_circuit(num_qubits, depth, rng=None, p_skip=0.5):
    if rng is None:
        rng = np.random.default_rng(0)
    circuit = []
    for layer in range(depth):
        for q in range(num_qubits):
            circuit.append(SingleQubitGate(q, haar_su2(rng)))
        for i in range(layer % 2, num_qubits - 1, 2):
            if rng.random() < p_skip:
                continue
            circuit.append(CZGate(i, i + 1))
    return circuit


def config1_circuit(seed=0, num_qubits=24, num_layers=20):
    """TFIM Trotter workload: J=1, h_i ~ U[0.5, 1.5] per layer and site, dt=0.1."""
    return tfim_circuit(num_qubits, num_layers, J=1.0, h=1.0, dt=0.1,
                        rng=np.random.default_rng(seed), disorder_strength_h=0.5)


def config2_circuit(seed=0, num_qubits=40, depth=30):
    """Brickwork workload: Haar SU(2) layers, CZ pairs skipped with p=1/2."""
    return brickwork_circuit(num_qubits, depth, rng=np.random.default_rng(seed))


def config4_batch(seed=0, count=256, n_range=(16, 48), layer_range=(10, 60), h_range=(0.3, 2.0),
                  m_range=(10, 20), dt=0.05, disorder_h=0.0):
    """The batched workload: ``count`` TFIM Trotter circuits (J = 1) with the
    qubit count, layer count, field h (one per circuit) and budget K = 2^m
    drawn uniformly per circuit from one seeded generator.  Returns
    (specs, circuits) with specs[i] = (n, K).  ``disorder_h`` > 0 draws every
    site's field from [h - disorder_h, h + disorder_h] instead (a uniform
    field makes many |a|^2 exactly equal, so top-k ties are common)."""
    rng = np.random.default_rng(seed)
    specs, circuits = [], []
    for _ in range(count):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        layers = int(rng.integers(layer_range[0], layer_range[1] + 1))
        h = float(rng.uniform(h_range[0], h_range[1]))
        m = int(rng.integers(m_range[0], m_range[1] + 1))
        circuits.append(tfim_circuit(n, layers, J=1.0, h=h, dt=dt, rng=rng, disorder_strength_h=disorder_h))
        specs.append((n, 2 ** m))
    return specs, circuits


class Config5Stream:
    """The served workload as a lazily built sequence of requests (circuit, n,
    K).  Request i is drawn from its own seeded generator (seed, i): with
    probability 1/2 from the batched workload's TFIM distribution
    (``config4_batch`` arguments in ``tfim``), otherwise a brickwork circuit
    with n, depth and K = 2^m uniform in the given ranges.  ``spec(i)`` gives
    (n, K) without building the circuit; circuits are built on first access."""

    def __init__(self, seed=0, count=100, tfim=None, brick_n=(20, 44), brick_depth=(10, 30), brick_m=(12, 22)):
        self.seed = int(seed)
        self.count = int(count)
        self.tfim = dict(tfim or {})
        self.brick = (brick_n, brick_depth, brick_m)
        self._cache = {}

    def __len__(self):
        return self.count

    def _draw(self, i):
        rng = np.random.default_rng([self.seed, int(i)])
        if rng.random() < 0.5:
            t = self.tfim
            n_range, layer_range = t.get("n_range", (16, 48)), t.get("layer_range", (10, 60))
            h_range, m_range = t.get("h_range", (0.3, 2.0)), t.get("m_range", (10, 20))
            n = int(rng.integers(n_range[0], n_range[1] + 1))
            layers = int(rng.integers(layer_range[0], layer_range[1] + 1))
            h = float(rng.uniform(h_range[0], h_range[1]))
            m = int(rng.integers(m_range[0], m_range[1] + 1))
            return rng, ("tfim", n, layers, h, m)
        brick_n, brick_depth, brick_m = self.brick
        n = int(rng.integers(brick_n[0], brick_n[1] + 1))
        depth = int(rng.integers(brick_depth[0], brick_depth[1] + 1))
        m = int(rng.integers(brick_m[0], brick_m[1] + 1))
        return rng, ("brick", n, depth, 0.0, m)

    def spec(self, i):
        _, (_, n, _, _, m) = self._draw(i)
        return n, 2 ** m

    def __getitem__(self, i):
        if i < 0 or i >= self.count:
            raise IndexError(i)
        if i not in self._cache:
            rng, (kind, n, d, h, m) = self._draw(i)
            if kind == "tfim":
                t = self.tfim
                circ = tfim_circuit(n, d, J=1.0, h=h, dt=t.get("dt", 0.05), rng=rng,
                                    disorder_strength_h=t.get("disorder_h", 0.0))
            else:
                circ = brickwork_circuit(n, d, rng=rng)
            self._cache[i] = (circ, n, 2 ** m)
        return self._cache[i]

    def release(self, i):
        """Drop request i's circuit from the cache (after it was served)."""
        self._cache.pop(i, None)


def config5_requests(seed=0, count=100, tfim=None, brick_n=(20, 44), brick_depth=(10, 30), brick_m=(12, 22)):
    """The served workload: ``count`` requests (circuit, n, K), built at once
    (see ``Config5Stream`` for the distribution and a lazy form)."""
    st = Config5Stream(seed, count, tfim, brick_n, brick_depth, brick_m)
    return [st[i] for i in range(count)]
