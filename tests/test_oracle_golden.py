"""The CPU oracle against the reference's own outputs (tests/golden/*.npz).

The fixtures were produced by tests/golden/make_golden.py, which runs the
reference (src/core/sparse_state.py, src/core/truncation.py,
src/simulation/bass_simulator.py, src/simulation/simulator.py).  Keys, output
order and key sets must match exactly; amplitudes may differ by a few ulps
(the reference's Numba kernels are compiled with fastmath and sum in array
order; the oracle sums exactly); the BASS traces must match event for event
against the tie-patched reference (see make_golden.py).
"""
import numpy as np
import pytest

from _common import (BASS_CASES, BASS2Q_CASES, FULL_MATCH_CASES, LARGE_CASES, first_mismatch, full_events,
                     load_case, sig_events, sorted_state)

RTOL = 1e-13   # relative amplitude tolerance for per-kernel comparisons


@pytest.fixture(scope="module")
def kv():
    import os
    from _common import GOLDEN
    return np.load(os.path.join(GOLDEN, "kernels.npz"))


def close(a, b, rtol=RTOL):
    a = np.asarray(a); b = np.asarray(b)
    assert a.shape == b.shape
    scale = max(1e-300, float(np.max(np.abs(b))) if b.size else 1.0)
    assert np.max(np.abs(a - b), initial=0.0) <= rtol * scale


def test_fingerprint_definition(orc):
    x = np.random.default_rng(1).integers(0, 2**63, size=1000, dtype=np.uint64)

    def fmix(z):
        z = z.copy()
        with np.errstate(over="ignore"):
            z ^= z >> np.uint64(33); z *= np.uint64(0xff51afd7ed558ccd)
            z ^= z >> np.uint64(33); z *= np.uint64(0xc4ceb9fe1a85ec53)
            z ^= z >> np.uint64(33)
        return z

    s = int(np.sum(fmix(x), dtype=np.uint64))
    z = int(np.bitwise_xor.reduce(fmix(x ^ np.uint64(0x5851F42D4C957F2D))))
    assert orc.fingerprint(x) == (1000, s, z)
    assert orc.fingerprint(x[::-1]) == (1000, s, z)


def test_exact_sum_is_order_independent(orc):
    from fractions import Fraction
    rng = np.random.default_rng(2)
    v = rng.standard_normal(20000) * np.exp(rng.uniform(-30, 0, 20000))
    s = orc.exact_sum(v)
    for _ in range(3):
        assert orc.exact_sum(rng.permutation(v)) == s
    exact = float(sum(Fraction(t) for t in v))
    assert abs(s - exact) <= 1e-15 * abs(exact) + 1e-28


@pytest.mark.parametrize("name", ["rx", "h", "x", "rz", "haar"])
@pytest.mark.parametrize("q", [0, 5, 11])
def test_expand_and_apply_1q(orc, kv, name, q):
    x, a, g = kv["x"], kv["a"], kv[f"g_{name}"]
    xo, ao = orc.expand_1q(x, a, g, q)
    assert np.array_equal(xo, kv[f"exp1q_{name}_{q}_x"])
    close(ao, kv[f"exp1q_{name}_{q}_a"])
    xo, ao = orc.apply_1q(x, a, g, q)
    assert np.array_equal(xo, kv[f"app1q_{name}_{q}_x"])
    close(ao, kv[f"app1q_{name}_{q}_a"])


@pytest.mark.parametrize("name", ["u4", "cz", "cnot"])
@pytest.mark.parametrize("qq", [(0, 1), (7, 2), (11, 4)])
def test_2q_gates(orc, kv, name, qq):
    q1, q2 = qq
    x, a, g = kv["x"], kv["a"], kv[f"g2_{name}"]
    xo, ao = orc.apply_2q_ht(x, a, g, q1, q2)
    assert np.array_equal(xo, kv[f"ht2q_{name}_{q1}_{q2}_x"])      # first-occurrence order
    close(ao, kv[f"ht2q_{name}_{q1}_{q2}_a"])
    xo, ao = orc.apply_2q_sorted(x, a, g, q1, q2)
    assert np.array_equal(xo, kv[f"app2q_{name}_{q1}_{q2}_x"])     # key-sorted
    close(ao, kv[f"app2q_{name}_{q1}_{q2}_a"])
    ad = orc.phase_2q(x, a, q1, q2, np.diag(g))
    close(ad, kv[f"diag2q_{name}_{q1}_{q2}_a"])


def test_radix_sort_and_merge(orc, kv):
    k, v = orc.radix_sort(kv["sort_in_k"], kv["sort_in_v"])
    assert np.array_equal(k, kv["sort_out_k"])
    assert np.array_equal(v, kv["sort_out_v"])           # a stable sort moves values exactly
    k, v = orc.merge_sorted(k, v)
    assert np.array_equal(k, kv["merge_out_k"])
    close(v, kv["merge_out_v"])


@pytest.mark.parametrize("k", [1, 37, 150])
def test_truncations(orc, kv, k):
    x, a = kv["x"], kv["a"]
    xo, ao, g = orc.topk_truncate(x, a, k)
    assert np.array_equal(np.sort(xo), np.sort(kv[f"topk_{k}_x"]))
    assert abs(g - float(kv[f"topk_{k}_gsq"])) <= 1e-13 * g
    xo, ao, g = orc.randomk_truncate(x, a, k, 12345 + k)
    assert np.array_equal(xo, kv[f"randk_{k}_x"])          # permutation order, exactly
    assert np.array_equal(ao, kv[f"randk_{k}_a"])
    assert abs(g - float(kv[f"randk_{k}_gsq"])) <= 1e-13 * g


def test_rdm_eigh_rotation(orc, kv):
    x, a = kv["x"], kv["a"]
    rho = orc.rdm_all(x, a, 12)
    close(rho, kv["rdm"], 1e-13)
    for r, ev, V in zip(kv["eigh_in"], kv["eigh_ev"], kv["eigh_V"]):
        e2, V2 = orc.eigh_2x2(r)
        assert np.array_equal(e2, ev) and np.array_equal(V2, V)      # same formula, bit for bit
        e3, V3 = orc.eigh_2x2_py(r)
        assert np.array_equal(e3, ev) and np.array_equal(V3, V)
    for q in (0, 6, 11):
        xo, ao = orc.rotate_1q(x, a, q, kv[f"rot_{q}_U"])
        assert np.array_equal(xo, kv[f"rot_{q}_x"])
        close(ao, kv[f"rot_{q}_a"])


def test_circuit_generator_pins(pkg):
    """The package's TFIM generator reproduces the reference's draws bit for bit."""
    z, circ, _ = load_case("config1_tfim_n24_k65536")
    mine = pkg.circuits.config1_circuit(seed=0)
    assert len(mine) == len(circ)
    for g, h in zip(mine, circ):
        assert g.qubits == h.qubits
        assert np.array_equal(g.matrix.view(np.uint64), h.matrix.view(np.uint64))


def _run_oracle_bass(orc, name):
    z, circ, kw = load_case(name)
    tr = orc.Trace()
    b = orc.OracleBASS(int(z["N"]), int(z["k"]), trace=tr, **kw)
    st = b.simulate(circ)
    return z, tr, b, st


@pytest.mark.parametrize("name", BASS_CASES + LARGE_CASES)
def test_bass_trace_matches_tie_patched_reference(orc, name):
    z, tr, b, st = _run_oracle_bass(orc, name)
    mine, ref = sig_events(tr.array()), sig_events(z["events"])
    assert first_mismatch(mine, ref) is None, f"first divergent event {first_mismatch(mine, ref)}"
    xs, as_ = sorted_state(st.x, st.alpha)
    assert np.array_equal(xs, z["x"])
    fid = abs(np.vdot(z["a"], as_)) ** 2
    assert fid >= 1 - 1e-12
    assert abs(st.gamma - float(z["gamma"])) <= 1e-9 * float(z["gamma"])
    for j in range(int(z["N"])):
        assert np.allclose(b.U[j], z["U"][j], rtol=0, atol=1e-8)   # frames accumulate rounding


def test_config1_matches_unpatched_reference(orc):
    """Without basis rotations (TFIM never passes the PR gate) the unpatched
    reference and the oracle agree on every truncated key set."""
    z, tr, b, st = _run_oracle_bass(orc, "config1_tfim_n24_k65536")
    assert first_mismatch(sig_events(tr.array()), sig_events(z["raw_events"])) is None
    assert abs(st.gamma - float(z["raw_gamma"])) <= 1e-12


@pytest.mark.parametrize("name", ["fixed_topk_n12_k64", "fixed_randk_n12_k64"])
def test_fixed_basis(orc, name):
    z, circ, _ = load_case(name)
    f = orc.OracleFixedBasis(12, 64, truncation="top-k" if "topk" in name else "random-k")
    st = f.simulate(circ, seed=4242)
    xs, as_ = sorted_state(st.x, st.alpha)
    assert np.array_equal(xs, z["x"])
    close(as_, z["a"], 1e-10)
    assert np.array_equal(f.nnz_history, z["nnz_hist"])
    assert np.allclose(f.gamma_history ** 2, z["gamma_sq_hist"], rtol=1e-10, atol=0)


@pytest.mark.parametrize("name", FULL_MATCH_CASES)
def test_bass_full_key_sets_match_reference(orc, name):
    """Every event, including the fingerprint of all keys (not only the
    significant ones), equals the reference's."""
    z, circ, kw = load_case(name)
    tr = orc.Trace()
    orc.OracleBASS(int(z["N"]), int(z["k"]), trace=tr, **kw).simulate(circ)
    assert first_mismatch(full_events(tr.array()), full_events(z["events"])) is None
