"""The precision form: complex64 amplitudes (dtype=np.complex64).

Gate and rotation arithmetic is FP32 with compensated products and sums; |a|^2,
the norm, the top-k threshold, the discarded weight and the RDM moments stay
FP64.  Checked against the complex128 path (itself bit-exact against the
oracle) and against FP64 references: the reference's own final config-1 state
and the dense FP64 statevector of the reference's ExactSimulator.

Tolerances, written here once: amplitudes of single ops agree with the
complex128 result to 2^-22 relative (a few float ulps); whole-run states agree
to fidelity >= 1 - 1e-6; per-layer discarded weight to 1e-6 absolute.
"""
import os

import numpy as np
import pytest

from _common import GOLDEN, load_case

pytestmark = pytest.mark.gpu

OP_RTOL = 2.0 ** -22
FID_TOL = 1e-6
DISCARD_TOL = 1e-6


@pytest.fixture(scope="module")
def env(pkg):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from bass_b200 import _native
    _native.build()
    return pkg


def _pair(N, x, a, cap=None):
    from bass_b200.state import SparseState
    n = len(x)
    cap = cap or 4 * n + 16
    s128 = SparseState(N, n, _capacity=cap)
    s64 = SparseState(N, n, dtype=np.complex64, _capacity=cap)
    s128.load(x, a)
    s64.load(x, a.astype(np.complex64))
    return s128, s64


def _rand(seed, N, n):
    rng = np.random.default_rng(seed)
    x = np.unique(rng.integers(0, 2 ** N, size=n + 64, dtype=np.uint64))[:n]
    a = rng.standard_normal(len(x)) + 1j * rng.standard_normal(len(x))
    return x, a / np.linalg.norm(a)


def _close(s64, s128, rtol=OP_RTOL):
    assert s64.alpha.dtype == np.complex64
    assert np.array_equal(s64.x, s128.x)
    ref = s128.alpha
    err = np.abs(s64.alpha.astype(np.complex128) - ref)
    assert np.all(err <= rtol * np.maximum(np.abs(ref), np.max(np.abs(ref)) * 1e-6))


def test_c64_import_export_roundtrip(env):
    x, a = _rand(1, 30, 5000)
    _, s64 = _pair(30, x, a)
    o = np.argsort(x)
    assert np.array_equal(s64.x, x[o])
    assert np.array_equal(s64.alpha, a.astype(np.complex64)[o])


def test_c64_gates_track_c128(env):
    from bass_b200 import _native as nat
    from bass_b200.gates import CNOTGate, haar_random_unitary
    N = 28
    x, a = _rand(2, N, 5000)
    s128, s64 = _pair(N, x, a, cap=64 * 5000)
    U = haar_random_unitary(2, seed=5)
    U4 = haar_random_unitary(4, seed=6)
    for st in (s128, s64):
        st._apply_1q(U, 3, nat.NO_TRUNC)
        st._apply_1q(U.conj().T, N - 1, nat.NO_TRUNC)
        st._apply_2q(U4, 5, 17, nat.NO_TRUNC)
        st._apply_2q(CNOTGate(0, 1).matrix, 2, 9, nat.NO_TRUNC)
        st._phase_2q(np.exp(1j * np.arange(4) * 0.3), 4, 11)
    # entries that cancel to exactly zero in one precision and not the other
    # would change the key set; with generic amplitudes they do not
    _close(s64, s128, rtol=4 * OP_RTOL)
    for st in (s128, s64):
        st._topk(nat.trunc(30000, 30000, 3, 2))
    assert s128.nnz == 30000
    assert np.array_equal(s64.x, s128.x)
    assert abs(s64.gamma - s128.gamma) <= 1e-6 * s128.gamma   # kept mass of float-rounded inputs
    f = abs(np.vdot(s128.alpha, s64.alpha.astype(np.complex128))) ** 2
    # rounding the renormalised amplitudes to float moves the norm by ~1e-10
    assert f >= 1 - 1e-8


def test_c64_norm_pr_rdm_are_fp64(env):
    from bass_b200 import _native as nat
    N = 24
    x, a = _rand(3, N, 10000)
    a64 = a.astype(np.complex64)
    _, s64 = _pair(N, x, a)
    # FP64 sums of the complex64 values, exactly as the device forms them
    ad = a64.astype(np.complex128)
    p = ad.real * ad.real + ad.imag * ad.imag
    assert abs(s64._norm2() - np.sum(p)) <= 1e-14
    assert abs(s64._pr() - 1.0 / np.sum(p * p)) <= 1e-10 * (1.0 / np.sum(p * p))
    eng = s64._eng
    nat.check(eng.L.bass_rdm_1q(s64._cur.ptr, N, nat.ctypes.c_void_p(nat._ptr(eng.rho)), eng.ctrl_ptr,
                                eng.ws_ptr, eng.ws_bytes, eng.stream), "bass_rdm_1q")
    rho = eng.rho[:4 * N].cpu().numpy().reshape(N, 4)
    for q in (0, 7, N - 1):
        bit = (x >> np.uint64(q)) & np.uint64(1)
        assert abs(rho[q, 1] - np.sum(p[bit == 1])) <= 1e-14


def _layer_discards(b, gates_per_layer, layers):
    """Discarded weight per layer: 1 - prod(kept / total) over its truncations."""
    keep = np.ones(layers)
    for i, kept, total in b.truncations:
        keep[i // gates_per_layer] *= kept / total
    return 1.0 - keep


def test_config3_precision_form(env):
    """Config 3: config 1's circuit and K in complex64, against the complex128
    run, the reference's own complex128 final state, and the FP64 dense state."""
    from bass_b200 import metrics
    from bass_b200.bass import BASS
    from bass_b200.dense import ExactSimulator
    z, circ, kw = load_case("config1_tfim_n24_k65536")
    N, K = 24, 2 ** 16
    b128 = BASS(N, K, record_truncations=True, **kw)
    s128 = b128.simulate(circ)
    b64 = BASS(N, K, dtype=np.complex64, record_truncations=True, **kw)
    s64 = b64.simulate(circ)
    assert s64.alpha.dtype == np.complex64
    # against the complex128 run
    a128 = dict(zip(s128.x.tolist(), s128.alpha))
    ov = sum(np.conj(a128.get(k, 0.0)) * complex(v) for k, v in zip(s64.x.tolist(), s64.alpha))
    f_c128 = abs(ov) ** 2
    assert f_c128 >= 1 - FID_TOL, f_c128
    # against the reference's own complex128 run (tie-patched golden)
    aref = dict(zip(z["x"].tolist(), z["a"]))
    ov = sum(np.conj(aref.get(k, 0.0)) * complex(v) for k, v in zip(s64.x.tolist(), s64.alpha))
    assert abs(ov) ** 2 >= 1 - FID_TOL
    # per-layer discarded weight (20 TFIM layers of 2N - 1 gates)
    d128 = _layer_discards(b128, 2 * N - 1, 20)
    d64 = _layer_discards(b64, 2 * N - 1, 20)
    assert np.max(np.abs(d64 - d128)) <= DISCARD_TOL, np.max(np.abs(d64 - d128))
    assert abs(s64.gamma ** 2 - s128.gamma ** 2) <= DISCARD_TOL
    # against the FP64 dense statevector
    psi = ExactSimulator(N, verbose=False).simulate_device(circ)
    f64, f128 = metrics.compute_fidelity(s64, psi), metrics.compute_fidelity(s128, psi)
    assert abs(f64 - f128) <= FID_TOL
    print(f"config 3: F(c64, c128) = 1 - {1 - f_c128:.3e}; F vs exact {f64:.9f} (c128 {f128:.9f}); "
          f"max per-layer discard difference {np.max(np.abs(d64 - d128)):.3e}")
