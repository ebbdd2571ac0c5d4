"""metrics.py's host path (numpy exact states) against the reference's
fidelity.py formulas, on a stand-in state object (no GPU needed)."""
import numpy as np


class FakeState:
    def __init__(self, N, x, a, gamma):
        self.N, self.x, self.alpha, self.gamma = N, x, a, gamma
        self.nnz = len(x)

    def sample(self, num_samples=1):                       # sparse_state.py:261-265
        p = np.abs(self.alpha) ** 2 / self.gamma ** 2
        p /= p.sum()
        return self.x[np.random.choice(self.nnz, size=num_samples, p=p)]

    def _pr(self):
        return 1.0 / np.sum(np.abs(self.alpha) ** 4)


def test_host_formulas(pkg):
    from bass_b200 import metrics
    rng = np.random.default_rng(3)
    N = 10
    exact = rng.standard_normal(2 ** N) + 1j * rng.standard_normal(2 ** N)
    exact /= np.linalg.norm(exact)
    x = np.sort(rng.choice(2 ** N, size=200, replace=False)).astype(np.uint64)
    a = exact[x.astype(np.int64)] * (1 + 0.01 * rng.standard_normal(200))
    a /= np.linalg.norm(a)
    st = FakeState(N, x, a, 0.8)
    # fidelity.py:48-68
    ref_f = float(np.abs(np.dot(exact[x].conj(), a)) ** 2)
    assert metrics.compute_fidelity(st, exact) == ref_f
    # fidelity.py:71-79
    assert metrics.compute_fidelity_bounds(st) == (0.8 ** 2, 1.0)
    # fidelity.py:95-102
    np.random.seed(9)
    s = st.sample(300)
    ref_x = 2 ** N * np.mean(np.abs(exact[s]) ** 2) - 1
    np.random.seed(9)
    assert metrics.estimate_cross_entropy_fidelity(st, exact, 300) == ref_x
    # runner.py:620-626 (the vdot part)
    assert metrics.dense_overlap(exact, exact) == complex(np.vdot(exact, exact))


def test_fidelity_bass_above_24_qubits_is_zero(pkg):
    # runner.py:620-626 returns 0.0 for N > 24 without building a statevector
    from bass_b200 import metrics

    class FakeSim:
        def __init__(self, N):
            self.N = N

        def to_statevector_device(self, state):
            raise AssertionError("no statevector above 24 qubits")

    for N in (25, 30, 40):
        assert metrics.fidelity_bass(FakeSim(N), None, None) == 0.0
