"""Tile loads of a state whose key array starts 8 bytes into its buffer (the
C ABI allows 8-byte aligned keys): the evaluation pass then copies entry by
entry instead of by bulk copies, and every result is the same bit for bit as
from a 16-byte aligned state (and, for complex128, as the oracle's)."""
import ctypes

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
    _native.lib()
    return pkg


def _state(N, x, a, dtype):
    from bass_b200.state import SparseState
    st = SparseState(N, 10 ** 9, dtype=dtype, _capacity=4 * len(x) + 16)
    st.load(x, a)
    return st


def _offset_keys(st, x, a):
    """Re-import (x, a) into the state's current descriptor with its keys 8
    bytes into a fresh buffer; returns the device buffers, which the caller
    keeps alive while the descriptor points into them."""
    eng, cur = st._eng, st._cur
    torch = eng.torch
    kb = torch.zeros(cur.cap + 1, dtype=torch.int64, device=eng.device)
    ab = torch.zeros_like(cur.amps)
    kx = torch.from_numpy(np.ascontiguousarray(x, dtype=np.uint64).view(np.int64).copy()).to(eng.device)
    real = np.float32 if cur.amp_type == 1 else np.float64
    ka = torch.from_numpy(np.ascontiguousarray(a, dtype=cur.np_dtype).view(real).copy()).to(eng.device)
    assert kb.data_ptr() % 16 == 0
    rc = eng.L.bass_state_import_typed(cur.ptr, ctypes.c_void_p(kb.data_ptr() + 8), ctypes.c_void_p(ab.data_ptr()),
                                       cur.cap, ctypes.c_void_p(kx.data_ptr()), ctypes.c_void_p(ka.data_ptr()),
                                       len(x), eng.nq, cur.amp_type, eng.ws_ptr, eng.ws_bytes, eng.ctrl_ptr,
                                       eng.stream)
    assert rc == 0
    torch.cuda.current_stream(eng.device).synchronize()
    st._rekeyed()
    return kb, ab, kx, ka


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_offset_keys_gate_1q_truncated(env, orc, dtype):
    from bass_b200 import _native as nat
    from bass_b200.gates import haar_random_unitary
    rng = np.random.default_rng(21)
    N, n, k = 30, 40_000, 50_000
    x = np.unique(rng.integers(0, 2 ** N, size=n + 100, dtype=np.uint64))[:n]
    a = (rng.standard_normal(len(x)) + 1j * rng.standard_normal(len(x))).astype(dtype)
    G = haar_random_unitary(2, seed=5)
    ref = _state(N, x, a, dtype)
    ref._apply_1q(G, 7, nat.trunc(k, k))
    st = _state(N, x, a, dtype)
    keep = _offset_keys(st, x, a)
    st._apply_1q(G, 7, nat.trunc(k, k))
    st._eng.raise_on_error()
    assert np.array_equal(st.x, ref.x) and np.array_equal(st.alpha, ref.alpha)
    if dtype == np.complex128:
        ox, oa = orc.apply_1q(x, a, G, 7)
        ox, oa, _, _ = orc.select_topk(ox, oa, k)
        o = np.argsort(ox)
        assert np.array_equal(st.x, ox[o]) and np.array_equal(st.alpha, oa[o])
    del keep


def test_offset_keys_gate_2q(env, orc):
    from bass_b200 import _native as nat
    from bass_b200.gates import haar_random_unitary
    rng = np.random.default_rng(22)
    N, n = 24, 30_000
    x = np.unique(rng.integers(0, 2 ** N, size=n + 100, dtype=np.uint64))[:n]
    a = rng.standard_normal(len(x)) + 1j * rng.standard_normal(len(x))
    G = haar_random_unitary(4, seed=9)
    st = _state(N, x, a, np.complex128)
    keep = _offset_keys(st, x, a)
    st._apply_2q(G, 3, 17, nat.NO_TRUNC)
    st._eng.raise_on_error()
    ox, oa = orc.apply_2q_sorted(x, a, G, 3, 17)
    assert np.array_equal(st.x, ox) and np.array_equal(st.alpha, oa)
    del keep
