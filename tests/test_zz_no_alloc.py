"""bass_rdm_1q_noalloc: the RDM moments for callers that cannot allocate.

Some callers of this library cannot allocate device memory when they need the
moments: host runtimes that own all device memory and only hand out the
state's buffers, and plugins or embeddings that may only pass the buffers they
were given.  The entry point under test keeps its scratch in a static
array inside the library and must give exactly the same moments as
bass_rdm_1q (same kernels, exact order-independent sums).  The file name makes
pytest collect it last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_ENTRIES = 1 << 20


@pytest.fixture(scope="module")
def lib(pkg):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from bass_b200 import _native
    _native.build()
    L = _native.lib()
    L.bass_rdm_1q_noalloc.restype = ctypes.c_int
    L.bass_rdm_1q_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_void_p]
    return L


def make_state(seed, N, n):
    from bass_b200 import _native, gates
    from bass_b200.state import SparseState
    rng = np.random.default_rng(seed)
    x = np.unique(rng.integers(0, 2 ** N, size=3 * n, dtype=np.uint64))[:n]
    a = rng.standard_normal(len(x)) + 1j * rng.standard_normal(len(x))
    st = SparseState(N, len(x), _capacity=4 * len(x) + 16)
    st.load(x, a)
    # a few gates so that the stored bit order is no longer the identity
    st._apply_1q(gates.HGate(0).matrix, 3, _native.NO_TRUNC)
    st._apply_2q(gates.CNOTGate(0, 1).matrix, 1, N - 1, _native.NO_TRUNC)
    return st


def rdm_with_workspace(st, N):
    from bass_b200 import _native
    eng = st._eng
    _native.check(eng.L.bass_rdm_1q(st._cur.ptr, N, ctypes.c_void_p(_native._ptr(eng.rho)), eng.ctrl_ptr,
                                    eng.ws_ptr, eng.ws_bytes, eng.stream), "bass_rdm_1q")
    return eng.rho[:4 * N].cpu().numpy().copy()


def rdm_noalloc(L, st, N):
    import torch
    from bass_b200 import _native
    eng = st._eng
    out = torch.full((4 * N,), float("nan"), dtype=torch.float64, device=eng.device)
    rc = L.bass_rdm_1q_noalloc(st._cur.ptr, st._cur.cap, N, ctypes.c_void_p(_native._ptr(out)),
                               eng.ctrl_ptr, eng.stream)
    assert rc == 0
    r = out.cpu().numpy().copy()
    eng.raise_on_error()
    return r


def test_noalloc_matches_workspace_rdm_twice(lib):
    # two calls in a row on different states: the shared static scratch keeps
    # the first call's contents, which must not leak into the second
    for seed, N, n in [(1, 40, 200000), (2, 24, 30000)]:
        st = make_state(seed, N, n)
        want = rdm_with_workspace(st, N)
        got = rdm_noalloc(lib, st, N)
        assert np.array_equal(got, want)            # same kernels, exact sums: identical
    st = make_state(3, 40, 200000)
    first = rdm_noalloc(lib, st, 40)
    second = rdm_noalloc(lib, st, 40)
    assert np.array_equal(first, second)
    assert np.array_equal(second, rdm_with_workspace(st, 40))


def test_noalloc_refuses_large_states(lib):
    import torch
    from bass_b200 import _native
    st = make_state(4, 20, 1000)
    eng = st._eng
    out = torch.zeros(4 * 20, dtype=torch.float64, device=eng.device)
    rc = lib.bass_rdm_1q_noalloc(st._cur.ptr, MAX_ENTRIES + 1, 20, ctypes.c_void_p(_native._ptr(out)),
                                 eng.ctrl_ptr, eng.stream)
    assert rc == _native.ERR_WORKSPACE


def test_noalloc_refuses_oversized_state_on_device(lib):
    # max_entries understates the state: the host check passes and the
    # kernels' own tile-count guards refuse the state (no scratch is touched
    # beyond its bounds): error bit in ctrl, NaN moments, status still OK
    import torch
    from bass_b200 import _native
    from bass_b200.state import SparseState
    N, n = 40, 1_100_000
    rng = np.random.default_rng(5)
    x = np.unique(rng.integers(0, 2 ** N, size=n + 1000, dtype=np.uint64))[:n]
    a = rng.standard_normal(len(x)) + 1j * rng.standard_normal(len(x))
    st = SparseState(N, len(x), _capacity=len(x) + 16)
    st.load(x, a)
    assert st.nnz == n
    eng = st._eng
    out = torch.zeros(4 * N, dtype=torch.float64, device=eng.device)
    rc = lib.bass_rdm_1q_noalloc(st._cur.ptr, MAX_ENTRIES, N, ctypes.c_void_p(_native._ptr(out)),
                                 eng.ctrl_ptr, eng.stream)
    assert rc == 0
    with pytest.raises(_native.BassError, match="workspace"):
        eng.raise_on_error()
    assert np.isnan(out.cpu().numpy()).all()
    # the library is still usable afterwards: a state that fits gives the
    # workspace entry point's moments
    st2 = make_state(6, 24, 30000)
    assert np.array_equal(rdm_noalloc(lib, st2, 24), rdm_with_workspace(st2, 24))
