"""GPU parity: every CUDA op through the C ABI against the CPU oracle, then
whole simulations against the oracle's traces and the reference's goldens.

The CUDA path and the oracle share their arithmetic rules (no fused
multiply-add, |a|^2 = re^2 + im^2, exact order-independent reductions), so the
comparisons are exact: keys, amplitudes, gamma, accept decisions and every
key-set fingerprint must be identical.
"""
import numpy as np
import pytest

from _common import (BASS_CASES, FULL_MATCH_CASES, LARGE_CASES, agreeing_prefix, first_mismatch, full_events,
                     load_case, sig_events, sorted_state)

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


def rand_state(rng, N, n, zero_at=None):
    x = np.unique(rng.integers(0, 2 ** N, size=3 * n, dtype=np.uint64))[:n]
    rng.shuffle(x)
    a = rng.standard_normal(len(x)) + 1j * rng.standard_normal(len(x))
    if zero_at is not None:
        a[zero_at] = 0.0
    return x, a


def gpu_state(B, N, x, a, cap=None):
    from bass_b200.state import SparseState
    cap = cap or 4 * len(x) + 16
    st = SparseState(N, 10 ** 9, _capacity=cap)
    st.load(x, a)
    return st


def same(x1, a1, x2, a2):
    assert np.array_equal(x1, x2), (len(x1), len(x2))
    assert np.array_equal(a1, a2), np.max(np.abs(a1 - a2))


def gates_1q(rng):
    from bass_b200 import gates
    z = (rng.standard_normal((2, 2)) + 1j * rng.standard_normal((2, 2)))
    q, _ = np.linalg.qr(z)
    return {"rx": gates.RXGate(0, 0.37).matrix, "h": gates.HGate(0).matrix, "x": gates.XGate(0).matrix,
            "haar": q, "rz": gates.RZGate(0, 0.61).matrix, "y": gates.YGate(0).matrix}


def test_import_export_roundtrip(B):
    from bass_b200 import _native
    rng = np.random.default_rng(0)
    for N, n in [(12, 1), (12, 300), (40, 5000), (63, 20000)]:
        x, a = rand_state(rng, N, n)
        st = gpu_state(B, N, x, a)
        xs, as_ = sorted_state(x, a)
        same(st.x, st.alpha, xs, as_)
        st._eng.raise_on_error()
    # duplicates are merged (summed left to right after a stable sort)
    x = np.array([5, 3, 5, 9, 3, 5], np.uint64)
    a = np.arange(6) + 1j * np.arange(6)
    st = gpu_state(B, 8, x, a)
    assert list(st.x) == [3, 5, 9]
    assert np.allclose(st.alpha, [1 + 4 + 1j * 5, 0 + 2 + 5 + 1j * 7, 3 + 3j])
    assert _native is not None


@pytest.mark.parametrize("N,n", [(12, 300), (24, 5000), (40, 30000)])
def test_gate_1q_exact(B, orc, N, n):
    rng = np.random.default_rng(N)
    x, a = rand_state(rng, N, n, zero_at=3)
    for name, G in gates_1q(rng).items():
        for q in sorted({0, 1, N // 2, N - 1}):
            st = gpu_state(B, N, x, a)
            from bass_b200 import _native
            st._apply_1q(G, q, _native.NO_TRUNC)
            xo, ao = orc.apply_1q(x, a, G, q)
            same(st.x, st.alpha, xo, ao)
            st._eng.raise_on_error()


@pytest.mark.parametrize("N,n", [(12, 300), (30, 20000)])
def test_gate_2q_exact(B, orc, N, n):
    from bass_b200 import _native, gates
    rng = np.random.default_rng(7 + N)
    x, a = rand_state(rng, N, n, zero_at=1)
    mats = {"u4": gates.haar_random_unitary(4, seed=3), "cz": gates.CZGate(0, 1).matrix,
            "cnot": gates.CNOTGate(0, 1).matrix}
    for name, G in mats.items():
        for (q1, q2) in [(0, 1), (1, 0), (N - 1, 2), (3, N - 1), (N // 2, N // 2 + 1)]:
            st = gpu_state(B, N, x, a)
            st._apply_2q(G, q1, q2, _native.NO_TRUNC)
            xo, ao = orc.apply_2q_sorted(x, a, G, q1, q2)
            same(st.x, st.alpha, xo, ao)
            st._eng.raise_on_error()


def test_gate_sequences_exact(B, orc):
    """Many gates in a row exercise every physical bit order."""
    from bass_b200 import _native
    rng = np.random.default_rng(11)
    N = 20
    x, a = rand_state(rng, N, 4000)
    st = gpu_state(B, N, x, a, cap=1 << 18)
    xo, ao = x, a
    for step in range(40):
        if rng.random() < 0.7:
            q = int(rng.integers(N))
            G = gates_1q(rng)["haar"]
            st._apply_1q(G, q, _native.NO_TRUNC)
            xo, ao = orc.apply_1q(xo, ao, G, q)
        else:
            q1, q2 = (int(v) for v in rng.choice(N, 2, replace=False))
            from bass_b200 import gates
            G = gates.haar_random_unitary(4, seed=step)
            st._apply_2q(G, q1, q2, _native.NO_TRUNC)
            xo, ao = orc.apply_2q_sorted(xo, ao, G, q1, q2)
        if len(xo) > 30000:
            st._topk(_native.trunc(20000, 20000))
            xo, ao, _, _ = orc.select_topk(xo, ao, 20000)
            xo, ao = sorted_state(xo, ao)
    same(st.x, st.alpha, *sorted_state(xo, ao))


@pytest.mark.parametrize("k", [1, 37, 150, 299])
def test_topk_exact(B, orc, k):
    from bass_b200 import _native
    rng = np.random.default_rng(k)
    x, a = rand_state(rng, 16, 300)
    a[10] = a[20] = a[30] = 0.5 + 0.5j           # exact ties
    a[40] = a[50] = (0.5 + 0.5j) * 1j
    st = gpu_state(B, 16, x, a)
    st._topk(_native.trunc(k, k, 3, 2))           # SparseState.truncate_top_k semantics
    xo, ao, kept, total = orc.select_topk(x, a, k)
    xs, as_ = sorted_state(xo, ao)
    as_ = as_ / np.sqrt(kept)
    assert np.array_equal(st.x, xs)
    assert np.array_equal(st.alpha, as_ * 1.0) or np.max(np.abs(st.alpha - as_)) < 1e-15
    assert abs(st.gamma - np.sqrt(kept)) <= 1e-15


def test_topk_large_ties(B, orc):
    """All candidates equal: the exact selection falls back to the radix path."""
    from bass_b200 import _native
    N, n, k = 20, 20000, 7000
    x = np.unique(np.random.default_rng(5).integers(0, 2 ** N, size=3 * n, dtype=np.uint64))[:n]
    a = np.full(len(x), 0.25 + 0.0j)
    st = gpu_state(B, N, x, a)
    st._topk(_native.trunc(k, k))
    xo, ao, _, _ = orc.select_topk(x, a, k)
    assert np.array_equal(st.x, np.sort(xo))


@pytest.mark.parametrize("n_tied", [7, 100, 2000, 6000])
def test_topk_ties_at_threshold(B, orc, n_tied):
    """A run of equal |a|^2 straddling rank k: the survivors among them are the
    smallest keys, and the kept mass counts them exactly.  Tie sizes cover the
    counting (<= 256), sorting (<= 4096) and radix paths of the boundary
    bin's settle step."""
    from bass_b200 import _native
    rng = np.random.default_rng(9 + n_tied)
    N, n = 24, max(30000, 12 * n_tied)
    x = np.unique(rng.integers(0, 2 ** N, size=2 * n, dtype=np.uint64))[:n]
    rng.shuffle(x)
    a = (rng.uniform(0.5, 1.0, n) + 1j * rng.uniform(-0.5, 0.5, n)) / 100.0
    tied = np.full(n_tied, 0.0065 + 0.0j)
    big = np.abs(a) ** 2 > np.abs(tied[0]) ** 2
    k = int(big.sum()) + n_tied // 2          # the cut falls inside the tied run
    idx = np.flatnonzero(~big)[:n_tied]
    a[idx] = tied
    st = gpu_state(B, N, x, a)
    st._topk(_native.trunc(k, k, 3, 2))           # SparseState.truncate_top_k semantics
    xo, ao, kept, _ = orc.select_topk(x, a, k)
    assert st.nnz == k
    xs, as_ = sorted_state(xo, ao)
    assert np.array_equal(st.x, xs)
    assert abs(st.gamma - np.sqrt(kept)) <= 1e-15
    assert np.max(np.abs(st.alpha - as_ / np.sqrt(kept))) < 1e-15


def test_rdm_exact(B, orc):
    rng = np.random.default_rng(3)
    for N, n in [(12, 300), (40, 50000)]:
        x, a = rand_state(rng, N, n)
        st = gpu_state(B, N, x, a)
        eng = st._eng
        from bass_b200 import _native
        _native.check(eng.L.bass_rdm_1q(st._cur.ptr, N, _native.ctypes.c_void_p(_native._ptr(eng.rho)),
                                        eng.ctrl_ptr, eng.ws_ptr, eng.ws_bytes, eng.stream), "rdm")
        r = eng.rho[:4 * N].cpu().numpy().reshape(N, 4)
        ro = orc.rdm_all(x, a, N)
        assert np.array_equal(r[:, 0], ro[:, 0, 0].real)
        assert np.array_equal(r[:, 1], ro[:, 1, 1].real)
        assert np.array_equal(r[:, 2], ro[:, 0, 1].real)
        assert np.array_equal(r[:, 3], ro[:, 0, 1].imag)


def test_norm_pr_exact(B, orc):
    rng = np.random.default_rng(4)
    x, a = rand_state(rng, 30, 70000)
    st = gpu_state(B, 30, x, a)
    assert st._norm2() == orc.sum_p(a)
    assert st._pr() == 1.0 / orc.sum_p2(a)


def test_fingerprint(B, orc):
    rng = np.random.default_rng(8)
    x, a = rand_state(rng, 40, 10000)
    a[::7] *= 1e-14
    st = gpu_state(B, 40, x, a)
    fp = st._cur.fingerprint(1e-24)
    assert fp[:3] == orc.fingerprint(x)
    assert fp[3:] == orc.fingerprint(x, a, 1e-24)


def test_radix_sort_and_merge_vs_reference(B, kv=None):
    import os
    import torch
    from _common import GOLDEN
    from bass_b200 import _native
    z = np.load(os.path.join(GOLDEN, "kernels.npz"))
    eng = _native.Engine(max_n=4096, num_qubits=40)
    k = torch.from_numpy(z["sort_in_k"].view(np.int64).copy()).cuda()
    v = torch.from_numpy(z["sort_in_v"].view(np.float64).copy()).cuda()
    n = len(z["sort_in_k"])
    P = _native.ctypes.c_void_p
    _native.check(eng.L.bass_radix_sort_u64(P(_native._ptr(k)), P(_native._ptr(v)), n, 64, eng.ws_ptr,
                                            eng.ws_bytes, eng.ctrl_ptr, eng.stream), "sort")
    assert np.array_equal(k.cpu().numpy().view(np.uint64), z["sort_out_k"])
    assert np.array_equal(v.cpu().numpy().view(np.complex128), z["sort_out_v"])
    nout = torch.zeros(1, dtype=torch.int64, device="cuda")
    _native.check(eng.L.bass_merge_sorted(P(_native._ptr(k)), P(_native._ptr(v)), n, P(_native._ptr(nout)),
                                          eng.ws_ptr, eng.ws_bytes, eng.ctrl_ptr, eng.stream), "merge")
    m = int(nout.item())
    assert np.array_equal(k[:m].cpu().numpy().view(np.uint64), z["merge_out_k"])
    assert np.allclose(v[:2 * m].cpu().numpy().view(np.complex128), z["merge_out_v"], rtol=1e-14, atol=0)


def test_rotation_step_matches_oracle(B, orc):
    """One coordinate-descent step: rotate, truncate, renormalise, decide."""
    from bass_b200 import _native
    from bass_b200.linalg import eigh_2x2
    rng = np.random.default_rng(21)
    N, n, k = 16, 3000, 2500
    x, a = rand_state(rng, N, n)
    a /= np.sqrt(orc.sum_p(a))
    st = gpu_state(B, N, x, a)
    eng = st._eng
    rho = orc.rdm_all(x, a, N)
    for j in (0, 5, 15):
        _, V = eigh_2x2(rho[j])
        nat = _native
        nat.check(eng.L.bass_pr(st._cur.ptr, eng.ctrl_ptr, eng.ws_ptr, eng.ws_bytes, eng.stream), "pr")
        u = nat.host_c128(V.conj().T)
        nat.check(eng.L.bass_rotate_step(st._cur.ptr, st._tmp.ptr, nat._host(u), j, k, 0, eng.ctrl_ptr,
                                         eng.ws_ptr, eng.ws_bytes, eng.stream), "rot")
        st._touch()
        c = eng.read_ctrl()
        xr, ar = orc.rotate_1q(x, a, j, V.conj().T)
        xt, at, _, _ = orc.select_topk(xr, ar, k)
        frac = orc.sum_p(at)
        pr_new = frac * frac / orc.sum_p2(at)
        at = at / np.sqrt(frac)
        pr = 1.0 / orc.sum_p2(a)
        acc = not (pr_new >= pr * (1.0 - 1e-12))
        assert int(c["accept"][j]) == int(acc)
        assert c["frac"][j] == frac
        if acc:
            x, a = xt, at
        same(st.x, st.alpha, *sorted_state(x, a))


def _gpu_bass(B, z, circ, kw, trace=True):
    from bass_b200.bass import BASS
    b = BASS(int(z["N"]), int(z["k"]), trace=trace, **kw)
    st = b.simulate(circ)
    return b, st


@pytest.mark.parametrize("name", BASS_CASES)
def test_bass_matches_oracle_exactly(B, orc, name):
    z, circ, kw = load_case(name)
    b, st = _gpu_bass(B, z, circ, kw)
    tr = orc.Trace()
    ob = orc.OracleBASS(int(z["N"]), int(z["k"]), trace=tr, **kw)
    ost = ob.simulate(circ)
    mine = [tuple(int(v) for v in e) for e in b.trace_events()]
    ref = [tuple(int(v) for v in e) for e in tr.array()]
    assert first_mismatch(mine, ref) is None, f"first divergent event {first_mismatch(mine, ref)}"
    same(st.x, st.alpha, *sorted_state(ost.x, ost.alpha))
    assert st.gamma == ost.gamma
    for j in range(int(z["N"])):
        assert np.array_equal(b.U[j], ob.U[j])
    assert b.stats["amp_updates"] == ob.stats["amp_updates"]
    assert b.stats["rotations"] == ob.stats["rotations"] and b.stats["accepted"] == ob.stats["accepted"]


@pytest.mark.parametrize("name", BASS_CASES + LARGE_CASES)
def test_bass_matches_reference_goldens(B, name):
    z, circ, kw = load_case(name)
    b, st = _gpu_bass(B, z, circ, kw)
    mine, ref = sig_events(b.trace_events()), sig_events(z["events"])
    assert first_mismatch(mine, ref) is None, f"first divergent event {first_mismatch(mine, ref)}"
    assert np.array_equal(st.x, z["x"])
    fid = abs(np.vdot(z["a"], st.alpha)) ** 2
    assert fid >= 1 - 1e-10
    assert abs(st.gamma - float(z["gamma"])) <= 1e-9 * float(z["gamma"])


@pytest.mark.parametrize("name", FULL_MATCH_CASES)
def test_bass_full_key_sets_match_reference(B, name):
    """Every event in full (the fingerprint of all keys, the nnz, accept and
    optimisation events) equals the tie-patched reference's."""
    z, circ, kw = load_case(name)
    b, st = _gpu_bass(B, z, circ, kw)
    assert first_mismatch(full_events(b.trace_events()), full_events(z["events"])) is None


@pytest.mark.parametrize("name", BASS_CASES + LARGE_CASES)
def test_bass_matches_unpatched_reference(B, name):
    """Against the unmodified reference (np.argpartition, `pr_new >= pr`):
    identical significant key sets at every event up to the first event at
    which the unmodified and the tie-patched reference themselves part (a
    rotation whose PR change is rounding noise, or a tie at the top-k
    boundary); for config 1 and the other runs where they never part, the
    whole trace."""
    z, circ, kw = load_case(name)
    b, _ = _gpu_bass(B, z, circ, kw)
    mine = sig_events(b.trace_events())
    raw, patched = sig_events(z["raw_events"]), sig_events(z["events"])
    n = agreeing_prefix(raw, patched)
    assert n > 0
    assert mine[:n] == raw[:n]
    if raw == patched:
        assert mine == raw


@pytest.mark.parametrize("name", ["fixed_topk_n12_k64"])
def test_fixed_basis_vs_reference(B, name):
    from bass_b200.fixed import FixedBasisSimulator
    z, circ, _ = load_case(name)
    f = FixedBasisSimulator(12, 64, truncation="top-k", verbose=False)
    st = f.simulate(circ, seed=4242)
    assert np.array_equal(st.x, z["x"])
    assert np.max(np.abs(st.alpha - z["a"])) < 1e-10
    m = f.get_metrics()
    assert np.array_equal(m["nnz"], z["nnz_hist"])
    assert np.allclose(m["gamma_squared"], z["gamma_sq_hist"], rtol=1e-10, atol=0)


def test_fixed_basis_random_k_vs_reference(B):
    """simulator.py:177-196: random-k after a 2-qubit gate draws over the hash
    table's first-occurrence order and keeps the drawn order; 1-qubit gates
    draw with the LCG over the key-sorted array.  Same draws as the reference
    run recorded in the fixture: the same key sets, histories and gammas."""
    from bass_b200.fixed import FixedBasisSimulator
    z, circ, _ = load_case("fixed_randk_n12_k64")
    f = FixedBasisSimulator(12, 64, truncation="random-k", verbose=False)
    st = f.simulate(circ, seed=4242)
    xs, as_ = sorted_state(st.x, st.alpha)
    assert np.array_equal(xs, z["x"])
    assert np.max(np.abs(as_ - z["a"])) < 1e-10
    m = f.get_metrics()
    assert np.array_equal(m["nnz"], z["nnz_hist"])
    assert np.allclose(m["gamma_squared"], z["gamma_sq_hist"], rtol=1e-10, atol=0)


def test_random_k_keeps_drawn_order(B, orc):
    """Two random-k truncations in a row: the second draws over the order the
    first left (truncation.py:116-159), as the oracle's arrays do."""
    from bass_b200 import gates
    from bass_b200.state import SparseState
    st = SparseState(10, 200)
    ost = orc.OracleSparseState(10, 200)
    for g in [gates.HGate(q) for q in range(9)] + [gates.RXGate(9, 0.7)]:
        st.apply_gate(g)
        ost.apply_gate(g)
    for k, seed in [(120, 11), (50, 12)]:
        st.k = ost.k = k
        st.truncate_random_k(seed)
        ost.truncate_random_k(seed)
        assert np.array_equal(st.x, ost.x)                  # same entries, same order
        assert np.max(np.abs(st.alpha - ost.alpha)) < 1e-12
        assert abs(st.gamma - ost.gamma) < 1e-12


def test_sparse_state_api(B, orc):
    """apply_gate / truncate_top_k / truncate_random_k / to_dense / copy."""
    from bass_b200 import gates
    from bass_b200.state import SparseState
    st = SparseState(10, 16)
    ost = orc.OracleSparseState(10, 16)
    circ = [gates.HGate(q) for q in range(6)] + [gates.RXGate(q, 0.3 + 0.1 * q) for q in range(10)] + \
        [gates.CNOTGate(0, 3), gates.CZGate(2, 7), gates.RZZGate(1, 2, 0.4), gates.TGate(4), gates.SGate(5)]
    for g in circ:
        st.apply_gate(g)
        ost.apply_gate(g)
    same(st.x, st.alpha, *sorted_state(ost.x, ost.alpha))
    assert st.gamma == ost.gamma
    d = st.to_dense()
    assert d.shape == (1024,) and abs(np.vdot(d, d) - 1) < 1e-12
    c = st.copy()
    same(c.x, c.alpha, st.x, st.alpha)
    # random-k on a key-sorted state (1-qubit gates only): the reference's own order
    st2 = SparseState(10, 40)
    ost2 = orc.OracleSparseState(10, 40)
    for q in range(8):
        g = gates.RXGate(q, 0.5 + 0.05 * q)
        st2.apply_gate(g, method="random-k", seed=99 + q)
        ost2.apply_gate(g, method="random-k", seed=99 + q)
    same(st2.x, st2.alpha, ost2.x, ost2.alpha)   # the drawn order of the last truncation too


def test_edge_cases(B, orc):
    from bass_b200 import _native, gates
    from bass_b200.bass import BASS
    # k >= 2^N: nothing is ever truncated
    circ = [gates.HGate(q) for q in range(5)] + [gates.CNOTGate(0, 1)]
    st = BASS(5, 64).simulate(circ)
    assert st.nnz == 32
    # k = 1
    st = BASS(6, 1).simulate([gates.HGate(0), gates.HGate(1), gates.CNOTGate(0, 2)])
    assert st.nnz == 1
    # an X gate drops nothing but moves every key; applying it twice restores the state
    rng = np.random.default_rng(2)
    x, a = rand_state(rng, 14, 500)
    s = gpu_state(B, 14, x, a)
    s._apply_1q(gates.XGate(0).matrix, 3, _native.NO_TRUNC)
    s._apply_1q(gates.XGate(0).matrix, 3, _native.NO_TRUNC)
    same(s.x, s.alpha, *sorted_state(x, a))
    # a diagonal gate with a zero entry drops the entries it zeroes
    s = gpu_state(B, 14, x, a)
    s._apply_1q(np.diag([1.0, 0.0]).astype(complex), 4, _native.NO_TRUNC)
    xo, ao = orc.apply_1q(x, a, np.diag([1.0, 0.0]).astype(complex), 4)
    same(s.x, s.alpha, xo, ao)
    # an empty state stays empty
    s = gpu_state(B, 14, x[:0], a[:0])
    s._apply_1q(gates.HGate(0).matrix, 2, _native.NO_TRUNC)
    assert s.nnz == 0
    s._eng.raise_on_error()
