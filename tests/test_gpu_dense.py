"""Device statevectors and metrics against the host formulas of the reference
(bass_simulator.py:608-621 to_statevector, fidelity.py:48-102,
runner.py:620-626)."""
import numpy as np
import pytest

from _common import load_case

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


def dense_run(N, circ):
    """Plain dense simulation (bit q of the index is qubit q)."""
    psi = np.zeros(2 ** N, np.complex128)
    psi[0] = 1.0
    for g in circ:
        m = np.asarray(g.matrix, np.complex128)
        if g.n_qubits == 1:
            q = g.qubits[0]
            v = psi.reshape(-1, 2, 2 ** q)
            psi = np.einsum("ij,kjl->kil", m, v).reshape(-1)
        else:
            q1, q2 = g.qubits
            v = psi.reshape([2] * N)                      # axis N-1-q is qubit q
            v = np.moveaxis(v, [N - 1 - q1, N - 1 - q2], [0, 1]).reshape(4, -1)
            v = (m @ v).reshape([2, 2] + [2] * (N - 2))
            psi = np.moveaxis(v, [0, 1], [N - 1 - q1, N - 1 - q2]).reshape(-1)
    return psi


def test_to_statevector_device_matches_host(B):
    from bass_b200.bass import BASS
    z, circ, kw = load_case("bass_brick_n12_k64")
    b = BASS(int(z["N"]), int(z["k"]), **kw)
    st = b.simulate(circ)
    host = b.to_statevector(st)
    dev = b.to_statevector_device(st).cpu().numpy()
    assert np.max(np.abs(dev - host)) <= 1e-14
    assert np.array_equal(st.to_dense_device().cpu().numpy(), st.to_dense())   # no frames: a scatter


def test_metrics_device_equal_host(B):
    import torch
    from bass_b200 import metrics
    from bass_b200.bass import BASS
    from bass_b200.fixed import FixedBasisSimulator
    z, circ, _ = load_case("bass_brick_n12_k64")
    N = int(z["N"])
    exact = dense_run(N, circ)
    exact_d = torch.as_tensor(exact, device="cuda")
    f = FixedBasisSimulator(N, 64, verbose=False)
    fs = f.simulate(circ)
    h = metrics.compute_fidelity(fs, exact)
    d = metrics.compute_fidelity(fs, exact_d)
    assert abs(h - d) <= 1e-13 and 0.0 < d <= 1.0 + 1e-12
    b = BASS(N, 64)
    bs = b.simulate(circ)
    fh = abs(np.vdot(exact, b.to_statevector(bs))) ** 2            # runner.py:620-626
    fd = metrics.fidelity_bass(b, bs, exact_d)
    assert abs(fh - fd) <= 1e-12 and 0.0 < fd <= 1.0 + 1e-12
    assert metrics.compute_fidelity_bounds(bs)[0] == bs.gamma ** 2
    pr = metrics.compute_participation_ratio(bs)
    assert abs(pr - 1.0 / np.sum(np.abs(bs.alpha) ** 4)) <= 1e-10 * pr
    np.random.seed(5)
    xh = metrics.estimate_cross_entropy_fidelity(fs, exact, 500)
    np.random.seed(5)
    xd = metrics.estimate_cross_entropy_fidelity(fs, exact_d, 500)
    assert abs(xh - xd) <= 1e-12 * max(1.0, abs(xh))


def test_dense_guard_refuses_wider_state(B):
    """A state with keys beyond the requested qubit count: the kernel's own
    bound check records BASS_ERR_ARG and writes nothing out of range."""
    import torch
    from bass_b200 import _native
    from bass_b200.state import SparseState
    x = np.array([1, 5, 700, 1023], np.uint64)
    st = SparseState(10, 64)
    st.load(x, np.ones(4, np.complex128) / 2)
    eng = st._eng
    psi = torch.zeros(2 ** 8, dtype=torch.complex128, device="cuda")
    _native.check(eng.L.bass_to_dense(st._cur.ptr, None, 8, _native.ctypes.c_void_p(psi.data_ptr()),
                                      eng.ctrl_ptr, eng.stream), "bass_to_dense")
    c = eng.read_ctrl()
    eng.set_ctrl("error", 0)
    assert int(c["error"]) != 0
    assert psi[1].item() == 0.5 and psi[5].item() == 0.5
    assert abs(psi).sum().item() == 1.0
