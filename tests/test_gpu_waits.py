"""Bounded device waits: a wait that gives up records BASS_ERR_WAIT, every
kernel returns, and the context stays usable.

The selection's grid barriers are bounded spins (bass_ctrl.wait_limit).  With
wait_limit < 0 a barrier that is not already open gives up at once, so the
first block to arrive at the first barrier of a truncating op gives up
deterministically; the op's result is then undefined (it is written inside
the output's bounds only) and the error bit reports it.  Nothing here faults
or hangs the GPU: every wait ends after at most one poll.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env(pkg):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from bass_b200 import _native
    _native.build()
    return pkg


def _state(seed, N, n):
    from bass_b200.state import SparseState
    rng = np.random.default_rng(seed)
    x = np.unique(rng.integers(0, 2 ** N, size=n + 100, dtype=np.uint64))[:n]
    a = rng.standard_normal(len(x)) + 1j * rng.standard_normal(len(x))
    a /= np.linalg.norm(a)
    st = SparseState(N, n, _capacity=2 * n + 16)
    st.load(x, a)
    return st, x, a


def test_selection_barrier_gives_up_and_recovers(env, orc):
    from bass_b200 import _native as nat
    from bass_b200.gates import haar_random_unitary
    N, n, k = 30, 300_000, 200_000
    st, x, a = _state(11, N, n)
    eng = st._eng
    G = haar_random_unitary(2, seed=3)
    eng.set_ctrl("wait_limit", -1)
    st._apply_1q(G, 7, nat.trunc(k, k, 3, 2))
    with pytest.raises(nat.BassError, match="wait gave up"):
        eng.raise_on_error()
    # the error was read and cleared; with the default limit the same op on
    # the same input is exact again
    eng.set_ctrl("wait_limit", 0)
    assert int(eng.read_ctrl()["error"]) == 0
    st.load(x, a)
    st._apply_1q(G, 7, nat.trunc(k, k, 0, 0))
    got_x, got_a = st.x, st.alpha
    ox, oa = orc.apply_1q(x, a, G, 7)
    ox, oa, _, _ = orc.select_topk(ox, oa, k)
    o = np.argsort(ox)
    assert np.array_equal(got_x, ox[o]) and np.array_equal(got_a, oa[o])
