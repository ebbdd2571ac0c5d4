"""The hash-table gate's entry order (FixedBasisSimulator, random-k mode).

ht_order restates, on the host, the order in which the reference's
apply_2qubit_gate_ht (bass_simulator.py:292-354) emits output keys; the
oracle's orc_apply_2q_ht emits in that order too.  Checked here on CPU on
seeded inputs, including gates with zero entries (children skipped) and
inputs in an arbitrary (non-sorted) order."""
import numpy as np
import pytest


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_ht_order_matches_oracle(pkg, orc, seed):
    from bass_b200.fixed import ht_order
    rng = np.random.default_rng(seed)
    N = 10
    x = rng.permutation(np.unique(rng.integers(0, 2 ** N, size=300, dtype=np.uint64)))
    a = rng.standard_normal(len(x)) + 1j * rng.standard_normal(len(x))
    a[::7] = 0.0
    G = rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4))
    if seed % 2:
        G[1, :] = 0.0      # output index 1 never emitted
        G[:, 2] = 0.0      # inputs with in_idx 2 emit nothing
    q1, q2 = int(rng.integers(0, N)), int((rng.integers(1, N) + seed) % N)
    if q1 == q2:
        q2 = (q1 + 1) % N
    xo, _ = orc.apply_2q_ht(x, a, G, q1, q2)
    assert np.array_equal(ht_order(x, a, G, q1, q2), xo)


def test_ht_order_empty(pkg):
    from bass_b200.fixed import ht_order
    out = ht_order(np.zeros(0, np.uint64), np.zeros(0, np.complex128), np.eye(4), 0, 1)
    assert out.dtype == np.uint64 and len(out) == 0
