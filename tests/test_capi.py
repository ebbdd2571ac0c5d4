"""CPU checks of the C ABI: the library loads without a GPU, exports every
symbol that include/bass_b200.h declares, and its descriptor layouts match
the numpy mirrors used by the host driver."""
import os
import re

import pytest

from conftest import PKG_DIR, ROOT

HEADER = os.path.join(ROOT, "include", "bass_b200.h")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(bass_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def native(pkg):
    from bass_b200 import _native
    _native.build()
    return _native


def test_header_symbols_exported(native):
    L = native.load_library()
    syms = declared_symbols()
    assert len(syms) >= 25
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_layouts(native):
    L = native.load_library()
    assert L.bass_state_bytes() == native.STATE_DTYPE.itemsize == 184
    assert L.bass_ctrl_bytes() == native.CTRL_DTYPE.itemsize
    assert L.bass_version().startswith(b"bass_b200")


def test_workspace_sizes_monotone(native):
    L = native.load_library()
    sizes = [L.bass_workspace_bytes(n, 4 * n, 40) for n in (1, 1000, 1 << 16, 1 << 22)]
    assert sizes == sorted(sizes)
    assert sizes[-1] < 64 * (4 << 22) + (64 << 20)   # about 45 bytes per output entry
    assert L.bass_workspace_bytes(1000, 1000, 40) == L.bass_workspace_bytes(1000, 4000, 40)


def test_lcg_choose_matches_reference_rule(native, orc):
    """bass_lcg_choose (host code) is the partial Fisher-Yates of truncation.py:116-159."""
    import numpy as np
    L = native.load_library()
    for nnz, k, seed in [(10, 3, 1), (300, 150, 12345 + 150), (1000, 1, 7)]:
        idx = np.empty(k, np.int64)
        assert L.bass_lcg_choose(nnz, k, seed, native._host(idx)) == 0
        x = np.arange(nnz, dtype=np.uint64)
        a = np.ones(nnz, np.complex128)
        xo, _, _ = orc.randomk_truncate(x, a, k, seed)
        assert np.array_equal(idx.astype(np.uint64), xo)


def test_state_arrays_must_be_aligned(native):
    """Keys 8-byte, complex128 amplitudes 16-byte, complex64 amplitudes
    8-byte aligned: other arrays are refused with BASS_ERR_ARG before any
    CUDA call (the addresses below are never dereferenced)."""
    import ctypes
    L = native.load_library()
    ERR_ARG, C128, C64 = 3, 0, 1
    desc = ctypes.create_string_buffer(L.bass_state_bytes())
    p = ctypes.c_void_p
    st, ctrl, ws = p(ctypes.addressof(desc)), p(0x7000), p(0x9000)
    base = 0x100000
    # init: 8-byte-offset complex128 amplitudes, 4-byte-offset keys
    assert L.bass_state_init_typed(st, p(base), p(base + 8), 16, 10, 0, C128, None) == ERR_ARG
    assert L.bass_state_init_typed(st, p(base + 4), p(base + 16), 16, 10, 0, C128, None) == ERR_ARG
    assert L.bass_state_init_typed(st, p(base + 4), p(base + 8), 16, 10, 0, C64, None) == ERR_ARG
    assert L.bass_state_init_typed(st, p(base), p(base + 4), 16, 10, 0, C64, None) == ERR_ARG
    # import: the state's arrays and the input arrays
    assert L.bass_state_import_typed(st, p(base), p(base + 8), 16, p(base), p(base + 16), 4, 10, C128,
                                     ws, 1 << 20, ctrl, None) == ERR_ARG
    assert L.bass_state_import_typed(st, p(base), p(base + 16), 16, p(base + 4), p(base + 16), 4, 10, C128,
                                     ws, 1 << 20, ctrl, None) == ERR_ARG
    # export
    assert L.bass_state_export_typed(st, p(base), p(base + 8), 64, C128, ws, 1 << 20, ctrl, None) == ERR_ARG


def test_library_refuses_without_gpu(native):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(native.BassError):
        native.lib()


def test_package_has_no_oracle_import():
    """The product never imports the oracle."""
    for root, _, files in os.walk(PKG_DIR):
        for f in files:
            if f.endswith(".py"):
                src = open(os.path.join(root, f)).read()
                assert not re.search(r"^\s*(from|import)\s+oracle", src, flags=re.M), f
                assert "liboracle" not in src, f
