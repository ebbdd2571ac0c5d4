"""The oracle's 2-qubit rotation path against the reference's own outputs.

tests/golden/kernels2q.npz and bass2q_*.npz come from
``make_golden.py --only-2q``: the reference's compute_2qubit_rdm and
apply_2qubit_rotation_sparse (bass_simulator.py:200-289) on seeded vectors,
and tie-patched BASS runs with use_2qubit_rotations=True (the pair passes of
bass_simulator.py:679-728, 819-824).
"""
import os

import numpy as np
import pytest

from _common import BASS2Q_CASES, GOLDEN, first_mismatch, load_case, sig_events, sorted_state


@pytest.fixture(scope="module")
def kv2():
    return np.load(os.path.join(GOLDEN, "kernels2q.npz"))


PAIRS = [(0, 1), (3, 7), (11, 4)]


@pytest.mark.parametrize("qq", PAIRS)
def test_rdm_2q(orc, kv2, qq):
    q1, q2 = qq
    rho = orc.rdm_2q(kv2["x"], kv2["a"], q1, q2)
    ref = kv2[f"rdm2q_{q1}_{q2}"]
    # the reference sums in group order, the oracle exactly
    assert np.max(np.abs(rho - ref)) <= 1e-15
    assert np.array_equal(rho, rho.conj().T)   # the lower triangle is the conjugate term by term


@pytest.mark.parametrize("qq", PAIRS)
def test_rotate_2q(orc, kv2, qq):
    q1, q2 = qq
    xo, ao = orc.rotate_2q(kv2["x"], kv2["a"], q1, q2, kv2[f"rot2q_{q1}_{q2}_U"])
    assert np.array_equal(xo, kv2[f"rot2q_{q1}_{q2}_x"])
    assert np.array_equal(ao, kv2[f"rot2q_{q1}_{q2}_a"])   # same products and order, bit for bit


@pytest.mark.parametrize("name", BASS2Q_CASES)
def test_bass_2q_trace_matches_tie_patched_reference(orc, name):
    z, circ, kw = load_case(name)
    tr = orc.Trace()
    b = orc.OracleBASS(int(z["N"]), int(z["k"]), trace=tr, **kw)
    st = b.simulate(circ)
    mine, ref = sig_events(tr.array()), sig_events(z["events"])
    assert first_mismatch(mine, ref) is None, f"first divergent event {first_mismatch(mine, ref)}"
    xs, as_ = sorted_state(st.x, st.alpha)
    assert np.array_equal(xs, z["x"])
    assert abs(np.vdot(z["a"], as_)) ** 2 >= 1 - 1e-12
    assert abs(st.gamma - float(z["gamma"])) <= 1e-9 * float(z["gamma"])
    for j in range(int(z["N"])):
        assert np.allclose(b.U[j], z["U"][j], rtol=0, atol=1e-8)
