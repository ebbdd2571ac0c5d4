"""Dense FP64 statevectors on the GPU against the reference's ExactSimulator
(exact_simulator.py:66-144), and config 1 (TFIM n=24, K=2^16) scored against
the exact state the way the reference scores it (fidelity.py:48-65).

The fixture ``dense_exact.npz`` was written by make_golden.py --only-dense
from the reference's own ExactSimulator: three small circuits in full, and at
n=24 the exact amplitudes at the keys of the config-1 BASS fixture plus the
reference's compute_fidelity of that fixture's state.
"""
import os

import numpy as np
import pytest

from _common import GOLDEN, Gate, load_case

pytestmark = pytest.mark.gpu

TOL = 1e-12   # per amplitude: dense gates round differently from numpy's einsum


@pytest.fixture(scope="module")
def env(pkg):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from bass_b200 import _native
    _native.build()
    return np.load(os.path.join(GOLDEN, "dense_exact.npz"))


@pytest.mark.parametrize("name", ["brick_n12", "tfim_n14", "haar2q_n10"])
def test_dense_matches_reference_exact(env, name):
    from bass_b200.dense import ExactSimulator
    z = env
    N = int(z[f"{name}_N"])
    circ = [Gate(m, g) for m, g in zip(z[f"{name}_gate_meta"], z[f"{name}_gate_mats"])]
    psi = ExactSimulator(N, verbose=False).simulate(circ)
    ref = z[f"{name}_psi"]
    assert np.max(np.abs(psi - ref)) < TOL
    assert abs(np.vdot(psi, psi).real - 1.0) < 1e-12


def test_config1_fidelity_against_exact(env, pkg):
    from bass_b200 import metrics
    from bass_b200.bass import BASS
    from bass_b200.dense import ExactSimulator
    z = env
    fx, circ, kw = load_case("config1_tfim_n24_k65536")
    psi = ExactSimulator(24, verbose=False).simulate_device(circ)
    # the device's exact state at the fixture's keys and at the reference's
    # 256 largest amplitudes
    x = z["config1_x"].astype(np.int64)
    import torch
    at_x = psi[torch.as_tensor(x, device=psi.device)].cpu().numpy()
    assert np.max(np.abs(at_x - z["config1_psi_at_x"])) < TOL
    top = psi[torch.as_tensor(z["config1_top_idx"], device=psi.device)].cpu().numpy()
    assert np.max(np.abs(top - z["config1_top_psi"])) < TOL
    # BASS config 1 on the device, scored on the device against the device's
    # exact state: the reference's fidelity of its own run, and gamma^2
    b = BASS(24, 2 ** 16, **kw)
    st = b.simulate(circ)
    f = metrics.compute_fidelity(st, psi)
    f_ref = float(z["config1_fidelity"])
    assert abs(f - f_ref) < 1e-9, (f, f_ref)
    g2, g2_ref = st.gamma ** 2, float(fx["gamma"]) ** 2
    assert abs(g2 - g2_ref) <= 1e-10 * g2_ref
    # the retained-mass bound of fidelity.py:68-76 holds as it does for the reference
    assert (f >= g2) == (f_ref >= g2_ref)
    print(f"config 1: fidelity {f:.12f} (reference {f_ref:.12f}), gamma^2 {g2:.12f}")
