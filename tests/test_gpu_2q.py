"""The 2-qubit rotation path on the GPU against the oracle and the reference.

bass_rdm_2q / bass_rotate_2q restate compute_2qubit_rdm and
apply_2qubit_rotation_sparse (bass_simulator.py:200-289); BASS with
use_2qubit_rotations=True runs the brick-wall pair passes (:679-728).
Exact sums on both sides, so the comparisons with the oracle are bit for bit.
"""
import numpy as np
import pytest

from _common import BASS2Q_CASES, first_mismatch, load_case, sig_events, sorted_state

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def B(pkg):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from bass_b200 import _native
    _native.build()
    _native.lib()
    return pkg


def rand_state(rng, N, n):
    x = np.unique(rng.integers(0, 2 ** N, size=3 * n, dtype=np.uint64))[:n]
    rng.shuffle(x)
    a = rng.standard_normal(len(x)) + 1j * rng.standard_normal(len(x))
    return x, a / np.linalg.norm(a)


def gpu_state(N, x, a, cap=None):
    from bass_b200.state import SparseState
    st = SparseState(N, 10 ** 9, _capacity=cap or 4 * len(x) + 16)
    st.load(x, a)
    return st


CASES = [(12, 300, (0, 1)), (12, 300, (3, 7)), (12, 300, (11, 4)), (20, 40000, (5, 17)), (20, 40000, (19, 0))]


@pytest.mark.parametrize("N,n,qq", CASES)
def test_rdm_2q_exact(B, orc, N, n, qq):
    rng = np.random.default_rng(N + n + qq[0])
    x, a = rand_state(rng, N, n)
    st = gpu_state(N, x, a)
    rho = st._rdm_2q(*qq)
    assert np.array_equal(rho, orc.rdm_2q(x, a, *qq))


@pytest.mark.parametrize("N,n,qq", CASES)
def test_rotate_2q_exact(B, orc, N, n, qq):
    from bass_b200 import _native
    rng = np.random.default_rng(7 + N + n + qq[1])
    x, a = rand_state(rng, N, n)
    a[: len(a) // 7] *= 1e-40          # groups of these alone give children under the 1e-30 drop rule
    a /= np.linalg.norm(a)
    evals, evecs = np.linalg.eigh(orc.rdm_2q(x, a, *qq))
    V = evecs[:, np.argsort(-evals)]
    for U4 in (V.conj().T, V):
        st = gpu_state(N, x, a)
        st._rotate_2q(U4, qq[0], qq[1], _native.NO_TRUNC)
        xo, ao = orc.rotate_2q(x, a, qq[0], qq[1], U4)
        assert np.array_equal(st.x, xo)
        assert np.array_equal(st.alpha, ao)
    # with the fused top-k
    k = max(1, n // 3)
    st = gpu_state(N, x, a)
    st._rotate_2q(V.conj().T, qq[0], qq[1], _native.trunc(k, k))
    xo, ao = orc.rotate_2q(x, a, qq[0], qq[1], V.conj().T)
    xk, ak, _, _ = orc.select_topk(xo, ao, k)
    xs, as_ = sorted_state(xk, ak)
    assert np.array_equal(st.x, xs)
    assert np.array_equal(st.alpha, as_)


def _gpu_bass(z, circ, kw, trace=True):
    from bass_b200.bass import BASS
    b = BASS(int(z["N"]), int(z["k"]), trace=trace, **kw)
    return b, b.simulate(circ)


@pytest.mark.parametrize("name", BASS2Q_CASES)
def test_bass_2q_matches_oracle_exactly(B, orc, name):
    z, circ, kw = load_case(name)
    b, st = _gpu_bass(z, circ, kw)
    tr = orc.Trace()
    ob = orc.OracleBASS(int(z["N"]), int(z["k"]), trace=tr, **kw)
    ost = ob.simulate(circ)
    mine = [tuple(int(v) for v in e) for e in b.trace_events()]
    ref = [tuple(int(v) for v in e) for e in tr.array()]
    assert first_mismatch(mine, ref) is None, f"first divergent event {first_mismatch(mine, ref)}"
    xs, as_ = sorted_state(ost.x, ost.alpha)
    assert np.array_equal(st.x, xs) and np.array_equal(st.alpha, as_)
    assert st.gamma == ost.gamma
    for j in range(int(z["N"])):
        assert np.array_equal(b.U[j], ob.U[j])


@pytest.mark.parametrize("name", BASS2Q_CASES)
def test_bass_2q_matches_reference_goldens(B, name):
    z, circ, kw = load_case(name)
    b, st = _gpu_bass(z, circ, kw)
    mine, ref = sig_events(b.trace_events()), sig_events(z["events"])
    assert first_mismatch(mine, ref) is None, f"first divergent event {first_mismatch(mine, ref)}"
    assert np.array_equal(st.x, z["x"])
    assert abs(np.vdot(z["a"], st.alpha)) ** 2 >= 1 - 1e-10
    assert abs(st.gamma - float(z["gamma"])) <= 1e-9 * float(z["gamma"])
