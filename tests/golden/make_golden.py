"""Generate the golden fixtures in this directory by running the reference.

Usage:  python tests/golden/make_golden.py --reference /path/to/reference [mode]

The reference checkout is given by ``--reference`` or the ``BASS_REFERENCE``
environment variable.  Modes: (none) the kernel vectors and the BASS /
FixedBasisSimulator runs; ``--only-2q`` the 2-qubit rotation fixtures;
``--only-k14`` the brickwork run at n=40, depth 10, K=2^14;
``--only-dense`` the reference's dense statevectors (ExactSimulator).

The reference (Skill0issue/BASS-Basis-Adapative-Sparse-Simulations-, pure
Python + Numba) is copied to a temporary directory (Numba's ``cache=True``
writes next to the sources), its packages get ``__init__.py`` files as its
README instructs, and its own classes and kernels are run on seeded inputs.
Nothing here is needed at test time: the tests read only the .npz files.

Recorded per BASS run (the reference object is instrumented, not modified):
  * every call of ``BASS._renorm`` (after a simulate-level truncation, after
    each attempted basis rotation, at the end of ``_optimize_basis``): nnz and
    an order-independent fingerprint of the surviving key set;
  * every accepted rotation (``_invalidate_kron(j)``) and every
    ``_optimize_basis`` call that passes its PR gate (with the gate index);
  * the relative gap between the k-th and (k+1)-th |a|^2 at every
    ``np.argpartition`` (to show the top-k boundary has no ties);
  * the final state (keys sorted, amplitudes), gamma and the frames U.
"""
from __future__ import annotations

import argparse
import importlib.util
import inspect
import os
import shutil
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402  (fingerprint definition)


def load_pkg():
    d = os.path.join(ROOT, "bass-basis-adapative-sparse-simulations-_b200")
    spec = importlib.util.spec_from_file_location("bass_b200", os.path.join(d, "__init__.py"),
                                                  submodule_search_locations=[d])
    m = importlib.util.module_from_spec(spec)
    sys.modules["bass_b200"] = m
    spec.loader.exec_module(m)
    return m


def import_reference(ref_dir):
    tmp = tempfile.mkdtemp(prefix="bassref_")
    dst = os.path.join(tmp, "ref")
    shutil.copytree(ref_dir, dst, ignore=shutil.ignore_patterns(".git", "tests", "*.png"))
    for sub in ["src", "src/core", "src/simulation", "src/benchmarking", "src/experimentation",
                "src/utils", "src/visualization"]:
        open(os.path.join(dst, sub, "__init__.py"), "a").close()
    sys.path.insert(0, dst)
    import src.core.sparse_state as ss
    import src.core.truncation as tr
    import src.core.gates as gates
    import src.simulation.bass_simulator as bs
    import src.simulation.simulator as fs
    import src.utils.random_circuits as rc
    import src.simulation.exact_simulator as ex
    import src.benchmarking.fidelity as fid
    return dict(ss=ss, tr=tr, gates=gates, bs=bs, fs=fs, rc=rc, ex=ex, fid=fid)


class GapRecorder:
    """Wraps numpy.argpartition; records the top-k boundary gap of every call.

    Numba resolves the module-global ``np`` when it compiles, so the module
    object itself cannot be replaced; only the Python-level callers of
    ``np.argpartition`` (the BASS driver) see the wrapper.
    """

    def __init__(self, gaps):
        self._gaps = gaps
        self._orig = np.argpartition

    def gap(self, a, k):
        s = np.sort(np.asarray(a))[::-1]
        if len(s) > k and s[k - 1] > 0:
            self._gaps.append(float((s[k - 1] - s[k]) / s[k - 1]))

    def __call__(self, a, kth, *args, **kw):
        if isinstance(kth, (int, np.integer)) and kth < 0:
            self.gap(a, -int(kth))
        return self._orig(a, kth, *args, **kw)


def instrument(b, events):
    orig_renorm, orig_inv, orig_opt = b._renorm, b._invalidate_kron, b._optimize_basis

    def _renorm(state):
        orig_renorm(state)
        c, s, z = oracle.fingerprint(state.x[:state.nnz])
        c2, s2, z2 = oracle.fingerprint(state.x[:state.nnz], state.alpha[:state.nnz], oracle.SIG_PMIN)
        events.append((0, c, s, z, c2, s2, z2))

    def _inv(j):
        events.append((1, int(j), 0, 0, 0, 0, 0))
        orig_inv(j)

    def _opt(state):
        if b._pr(state) >= b.k / 4:
            i = inspect.currentframe().f_back.f_locals.get("i", -1)
            events.append((2, int(i), 0, 0, 0, 0, 0))
        orig_opt(state)

    b._renorm, b._invalidate_kron, b._optimize_basis = _renorm, _inv, _opt


PR_TIE_TOL = 1e-12


_ACTIVE_RECORDER = []


def _topk_tiebreak(probs, keys, k):
    """Indices of the k largest probs, ties broken by smaller key."""
    if _ACTIVE_RECORDER:
        _ACTIVE_RECORDER[-1].gap(probs, k)
    return np.lexsort((np.asarray(keys), -np.asarray(probs)))[:k]


def tie_patched_bass(R):
    """The reference's BASS class with its two tie rules made deterministic.

    The reference's own method sources are patched textually at run time
    (nothing of them is stored here):
      * ``np.argpartition(probs, -self.k)[-self.k :]`` (simulate, _truncate_state)
        becomes a selection by (|a|^2 descending, key ascending);
      * ``if pr_new >= pr:`` (_optimize_basis) becomes
        ``if pr_new >= pr * (1.0 - PR_TIE_TOL):``, and the 2-qubit pass's
        ``if pr_after > pr_before:`` becomes
        ``if pr_after > pr_before * (1.0 - PR_TIE_TOL):``.
    """
    import textwrap
    bs = R["bs"]
    ns = dict(bs.__dict__)
    ns["_topk_tiebreak"] = _topk_tiebreak
    ns["PR_TIE_TOL"] = PR_TIE_TOL
    methods = {}
    subs = {
        "simulate": [("np.argpartition(probs, -self.k)[-self.k :]", "_topk_tiebreak(probs, state.x[: state.nnz], self.k)")],
        "_truncate_state": [("np.argpartition(probs, -self.k)[-self.k :]", "_topk_tiebreak(probs, state.x[: state.nnz], self.k)")],
        "_optimize_basis": [("if pr_new >= pr:", "if pr_new >= pr * (1.0 - PR_TIE_TOL):")],
        "_optimize_2q_pass": [("if pr_after > pr_before:", "if pr_after > pr_before * (1.0 - PR_TIE_TOL):")],
    }
    for name, reps in subs.items():
        src = textwrap.dedent(inspect.getsource(getattr(bs.BASS, name)))
        for old, new in reps:
            assert old in src, (name, old)
            src = src.replace(old, new)
        exec(compile(src, f"<tie-patched {name}>", "exec"), ns)
        methods[name] = ns[name]
    return type("TiePatchedBASS", (bs.BASS,), methods)


def run_bass(R, N, k, circuit, patched=True, **kw):
    events, gaps = [], []
    rec = GapRecorder(gaps)
    np.argpartition = rec
    _ACTIVE_RECORDER.append(rec)
    try:
        cls = tie_patched_bass(R) if patched else R["bs"].BASS
        b = cls(N, k, **kw)
        instrument(b, events)
        t0 = time.perf_counter()
        st = b.simulate(circuit)
        dt = time.perf_counter() - t0
    finally:
        np.argpartition = rec._orig
        _ACTIVE_RECORDER.pop()
    x = st.x[:st.nnz].copy(); a = st.alpha[:st.nnz].copy()
    o = np.argsort(x)
    return dict(events=np.array(events, dtype=np.uint64).reshape(-1, 7), x=x[o], a=a[o],
                gamma=np.float64(st.gamma), U=np.array(b.U), min_gap=np.float64(min(gaps) if gaps else 1.0),
                n_trunc=np.int64(len(gaps)), seconds=np.float64(dt))


def gate_arrays(circuit):
    """Serialise a gate list: (nq, q1, q2) per gate and 4x4 matrices (1q in the top-left)."""
    meta = np.zeros((len(circuit), 3), np.int64)
    mats = np.zeros((len(circuit), 4, 4), np.complex128)
    for i, g in enumerate(circuit):
        meta[i, 0] = g.n_qubits
        meta[i, 1] = g.qubits[0]
        meta[i, 2] = g.qubits[1] if g.n_qubits == 2 else -1
        d = 2 ** g.n_qubits
        mats[i, :d, :d] = g.matrix
    return meta, mats


def kernel_vectors(R, rng):
    """Small known-answer vectors for every reference kernel on the path."""
    ss, tr, bs = R["ss"], R["tr"], R["bs"]
    out = {}
    N = 12
    n = 300
    x = np.unique(rng.integers(0, 2 ** N, size=2 * n).astype(np.uint64))[:n]
    rng.shuffle(x)
    a = rng.standard_normal(len(x)) + 1j * rng.standard_normal(len(x))
    a[5] = 0.0  # an exact-zero amplitude (kept by merges, dropped by expansion)
    out["x"] = x; out["a"] = a
    G = np.array(R["gates"].RXGate(0, 0.37).matrix)
    Gh = np.array(R["gates"].HGate(0).matrix)
    Gx = np.array(R["gates"].XGate(0).matrix)
    Gd = np.array(R["gates"].RZGate(0, 0.61).matrix)
    Ghaar = oracle_free_haar(rng)
    for name, g in [("rx", G), ("h", Gh), ("x", Gx), ("rz", Gd), ("haar", Ghaar)]:
        for q in (0, 5, 11):
            xo = np.zeros(2 * len(x), np.uint64); ao = np.zeros(2 * len(x), np.complex128)
            m = ss.apply_1qubit_gate_kernel_opt(x, a, len(x), xo, ao, np.ascontiguousarray(g), q)
            out[f"exp1q_{name}_{q}_x"] = xo[:m].copy(); out[f"exp1q_{name}_{q}_a"] = ao[:m].copy()
            st = ss.SparseState(N, 10 ** 6)
            st.x = x.copy(); st.alpha = a.copy(); st.nnz = len(x)
            st._temp_x = np.zeros(4 * len(x), np.uint64); st._temp_alpha = np.zeros(4 * len(x), np.complex128)
            st.apply_gate(R["gates"].SingleQubitGate(q, g))
            out[f"app1q_{name}_{q}_x"] = st.x[:st.nnz].copy(); out[f"app1q_{name}_{q}_a"] = st.alpha[:st.nnz].copy()
            out[f"g_{name}"] = g
    U4 = R["gates"].haar_random_unitary(4, seed=7)
    CZ = np.array(R["gates"].CZGate(0, 1).matrix)
    CN = np.array(R["gates"].CNOTGate(0, 1).matrix)
    for name, g in [("u4", U4), ("cz", CZ), ("cnot", CN)]:
        out[f"g2_{name}"] = g
        for (q1, q2) in ((0, 1), (7, 2), (11, 4)):
            cap = 4 * len(x)
            hk = np.full(1 << 14, np.iinfo(np.uint64).max, np.uint64); hv = np.zeros(1 << 14, np.int32)
            xo = np.zeros(cap, np.uint64); ao = np.zeros(cap, np.complex128)
            m = bs.apply_2qubit_gate_ht(x, a, len(x), xo, ao, np.ascontiguousarray(g), q1, q2, hk, hv)
            out[f"ht2q_{name}_{q1}_{q2}_x"] = xo[:m].copy(); out[f"ht2q_{name}_{q1}_{q2}_a"] = ao[:m].copy()
            st = ss.SparseState(N, 10 ** 6)
            st.x = x.copy(); st.alpha = a.copy(); st.nnz = len(x)
            st.apply_gate(R["gates"].TwoQubitGate(q1, q2, g))
            out[f"app2q_{name}_{q1}_{q2}_x"] = st.x[:st.nnz].copy(); out[f"app2q_{name}_{q1}_{q2}_a"] = st.alpha[:st.nnz].copy()
            diag = np.diag(g).astype(np.complex128)
            ad = a.copy()
            ss.apply_2qubit_diagonal_kernel(x, ad, len(x), q1, q2, diag)
            out[f"diag2q_{name}_{q1}_{q2}_a"] = ad
    # radix sort + merge on keys with duplicates
    kd = rng.integers(0, 2 ** 40, size=700).astype(np.uint64)
    kd = np.concatenate([kd, kd[:200], kd[:50]]); rng.shuffle(kd)
    vd = rng.standard_normal(len(kd)) + 1j * rng.standard_normal(len(kd))
    k2, v2 = kd.copy(), vd.copy()
    ss.radix_sort_uint64(k2, v2, len(k2))
    out["sort_in_k"] = kd; out["sort_in_v"] = vd; out["sort_out_k"] = k2.copy(); out["sort_out_v"] = v2.copy()
    m = ss.merge_sorted_kernel(k2, v2, len(k2))
    out["merge_out_k"] = k2[:m].copy(); out["merge_out_v"] = v2[:m].copy()
    # truncations
    for kk in (1, 37, 150):
        x2, a2 = x.copy(), a.copy()
        m, g = tr.top_k_truncate_kernel_opt(x2, a2, len(x2), kk)
        out[f"topk_{kk}_x"] = x2[:m].copy(); out[f"topk_{kk}_gsq"] = np.float64(g)
        x2, a2 = x.copy(), a.copy()
        m, g = tr.random_k_truncate_kernel_opt(x2, a2, len(x2), kk, 12345 + kk)
        out[f"randk_{kk}_x"] = x2[:m].copy(); out[f"randk_{kk}_a"] = a2[:m].copy(); out[f"randk_{kk}_gsq"] = np.float64(g)
    # RDMs, eigensolver, rotation
    hk = np.full(1 << 12, np.iinfo(np.uint64).max, np.uint64); hv = np.zeros(1 << 12, np.int32)
    bs.ht_build(x, len(x), hk, hv)
    out["rdm"] = bs.compute_all_1qubit_rdms(x, a, len(x), N, hk, hv)
    rhos = []
    for i in range(64):
        h = rng.standard_normal((2, 2)) + 1j * rng.standard_normal((2, 2))
        h = h @ h.conj().T
        if i % 8 == 0:
            h = np.diag(np.diag(h)).astype(np.complex128)
        rhos.append(h)
    rhos.append(np.array([[0.3, 0], [0, 0.7]], np.complex128))
    rhos.append(np.array([[0.7, 1e-15], [1e-15, 0.3]], np.complex128))
    rhos = np.array(rhos)
    out["eigh_in"] = rhos
    ev, V = zip(*[bs.eigh_2x2(r) for r in rhos])
    out["eigh_ev"] = np.array(ev); out["eigh_V"] = np.array(V)
    for q in (0, 6, 11):
        _, Vq = bs.eigh_2x2(out["rdm"][q])
        x2 = np.concatenate([x, np.zeros(len(x), np.uint64)]); a2 = np.concatenate([a, np.zeros(len(x), np.complex128)])
        m = bs.apply_1qubit_rotation_sparse(x2, a2, len(x), q, np.ascontiguousarray(Vq.conj().T))
        out[f"rot_{q}_U"] = Vq.conj().T; out[f"rot_{q}_x"] = x2[:m].copy(); out[f"rot_{q}_a"] = a2[:m].copy()
    return out


def kernel_vectors_2q(R, rng):
    """Known-answer vectors of the 2-qubit RDM and 2-qubit rotation kernels."""
    bs = R["bs"]
    out = {}
    N, n = 12, 300
    x = np.unique(rng.integers(0, 2 ** N, size=2 * n).astype(np.uint64))[:n]
    rng.shuffle(x)
    a = rng.standard_normal(len(x)) + 1j * rng.standard_normal(len(x))
    a /= np.linalg.norm(a)
    out["x"] = x; out["a"] = a
    for (q1, q2) in ((0, 1), (3, 7), (11, 4)):
        rho = bs.compute_2qubit_rdm(x, a, len(x), q1, q2)
        evals, evecs = np.linalg.eigh(rho)
        V = evecs[:, np.argsort(-evals)]
        U4 = np.ascontiguousarray(V.conj().T)
        x2 = np.concatenate([x, np.zeros(3 * len(x), np.uint64)])
        a2 = np.concatenate([a, np.zeros(3 * len(x), np.complex128)])
        m = bs.apply_2qubit_rotation_sparse(x2, a2, len(x), q1, q2, U4)
        o = np.argsort(x2[:m])
        out[f"rdm2q_{q1}_{q2}"] = rho
        out[f"rot2q_{q1}_{q2}_U"] = U4
        out[f"rot2q_{q1}_{q2}_x"] = x2[:m][o].copy(); out[f"rot2q_{q1}_{q2}_a"] = a2[:m][o].copy()
    return out


def main_2q(R, pkg):
    """The 2-qubit rotation fixtures only (kernels2q.npz and the bass2q runs)."""
    rng = np.random.default_rng(20261204)
    kv = kernel_vectors_2q(R, rng)
    np.savez_compressed(os.path.join(HERE, "kernels2q.npz"), **kv)
    print("kernels2q.npz", len(kv))
    cases = [
        ("bass2q_brick_n10_k32", 10, 32, pkg.circuits.brickwork_circuit(10, 8, rng=np.random.default_rng(21)),
         {"use_2qubit_rotations": True}),
        ("bass2q_tfim_n10_k48", 10, 48, pkg.circuits.tfim_circuit(
            10, 10, J=1.0, h=1.0, dt=0.3, rng=np.random.default_rng(22), disorder_strength_h=0.5),
         {"use_2qubit_rotations": True}),
    ]
    for name, N, k, circ, kw in cases:
        r = run_bass(R, N, k, circ, patched=True, **kw)
        meta, mats = gate_arrays(circ)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), N=np.int64(N), k=np.int64(k),
                            kwargs=np.array(repr(kw)), gate_meta=meta, gate_mats=mats,
                            pr_tie_tol=np.float64(PR_TIE_TOL), **r)
        print(name, "events", len(r["events"]), "nnz", len(r["x"]), "gamma", float(r["gamma"]),
              "min_gap", float(r["min_gap"]), f"{float(r['seconds']):.2f}s")


def write_bass_cases(R, cases):
    """Run each case on the tie-patched and on the unmodified reference and
    store both traces (the unmodified one as raw_*)."""
    for name, N, k, circ, kw in cases:
        r = run_bass(R, N, k, circ, patched=True, **kw)
        raw = run_bass(R, N, k, circ, patched=False, **kw)
        meta, mats = gate_arrays(circ)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), N=np.int64(N), k=np.int64(k),
                            kwargs=np.array(repr(kw)), gate_meta=meta, gate_mats=mats,
                            pr_tie_tol=np.float64(PR_TIE_TOL), **r,
                            **{f"raw_{key}": raw[key] for key in ("events", "gamma", "min_gap", "n_trunc")})
        print(name, "events", len(r["events"]), "nnz", len(r["x"]), "gamma", float(r["gamma"]),
              "raw gamma", float(raw["gamma"]), "min_gap", float(r["min_gap"]), "n_trunc",
              int(r["n_trunc"]), f"{float(r['seconds']):.2f}s", flush=True)


def main_dense(R, pkg):
    """The reference's dense FP64 statevectors (ExactSimulator,
    exact_simulator.py:66-144): two small circuits in full, and config 1
    (TFIM n=24, 20 layers) at the keys of the config-1 BASS fixture, with the
    reference's compute_fidelity (fidelity.py:48-65) of that fixture's state."""
    ex = R["ex"].ExactSimulator
    out = {}
    small = [("brick_n12", 12, pkg.circuits.brickwork_circuit(12, 10, rng=np.random.default_rng(4))),
             ("tfim_n14", 14, pkg.circuits.tfim_circuit(14, 6, J=1.0, h=1.0, dt=0.3, rng=np.random.default_rng(9),
                                                        disorder_strength_h=0.5))]
    np.random.seed(17)
    small.append(("haar2q_n10", 10, R["rc"].generate_random_circuit(10, 8)))
    for name, N, circ in small:
        meta, mats = gate_arrays(circ)
        out[f"{name}_N"] = np.int64(N)
        out[f"{name}_gate_meta"] = meta
        out[f"{name}_gate_mats"] = mats
        out[f"{name}_psi"] = ex(N, verbose=False).simulate(circ)
        print(name, "done", flush=True)
    z = np.load(os.path.join(HERE, "config1_tfim_n24_k65536.npz"))
    circ = pkg.circuits.config1_circuit(seed=0)
    t0 = time.perf_counter()
    psi = ex(24, verbose=False).simulate(circ)
    dt = time.perf_counter() - t0
    x = z["x"]
    st = R["ss"].SparseState(24, len(x))
    st.x = x.copy(); st.alpha = z["a"].copy(); st.nnz = len(x); st.gamma = float(z["gamma"])
    out["config1_x"] = x
    out["config1_psi_at_x"] = psi[x.astype(np.int64)]
    out["config1_fidelity"] = np.float64(R["fid"].compute_fidelity(st, psi))
    top = np.argsort(-np.abs(psi))[:256]
    out["config1_top_idx"] = top.astype(np.int64)
    out["config1_top_psi"] = psi[top]
    out["config1_norm2"] = np.float64(np.vdot(psi, psi).real)
    out["config1_seconds"] = np.float64(dt)
    np.savez_compressed(os.path.join(HERE, "dense_exact.npz"), **out)
    print("dense_exact.npz: config-1 fidelity", float(out["config1_fidelity"]), "gamma^2",
          float(z["gamma"]) ** 2, f"{dt:.1f}s", flush=True)


def oracle_free_haar(rng):
    z = (rng.standard_normal((2, 2)) + 1j * rng.standard_normal((2, 2))) / np.sqrt(2.0)
    q, r = np.linalg.qr(z)
    d = np.diag(r)
    return q * (d / np.abs(d))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("BASS_REFERENCE"),
                    help="the reference checkout (default: $BASS_REFERENCE)")
    ap.add_argument("--skip-large", action="store_true")
    ap.add_argument("--only-2q", action="store_true", help="write only the 2-qubit rotation fixtures")
    ap.add_argument("--only-k14", action="store_true", help="write only the n=40 depth-10 K=2^14 run")
    ap.add_argument("--only-dense", action="store_true", help="write only the dense statevector fixtures")
    args = ap.parse_args()
    if not args.reference:
        ap.error("give the reference checkout with --reference or $BASS_REFERENCE")
    oracle.build()
    R = import_reference(args.reference)
    pkg = load_pkg()
    if args.only_2q:
        main_2q(R, pkg)
        return
    if args.only_k14:
        write_bass_cases(R, [("config2_brick_n40_d10_k16384", 40, 2 ** 14,
                              pkg.circuits.config2_circuit(seed=0, depth=10), {})])
        return
    if args.only_dense:
        main_dense(R, pkg)
        return
    rng = np.random.default_rng(20261203)

    # kernel-level known-answer vectors
    kv = kernel_vectors(R, rng)
    np.savez_compressed(os.path.join(HERE, "kernels.npz"), **kv)
    print("kernels.npz", len(kv))

    # the circuit generators must reproduce the reference's draws
    c_ref = R["rc"].generate_tfim_circuit(24, 20, J=1.0, h=1.0, dt=0.1, rng=np.random.default_rng(0),
                                          disorder_strength_h=0.5)
    c_pkg = pkg.circuits.config1_circuit(seed=0)
    m_ref, g_ref = gate_arrays(c_ref)
    m_pkg, g_pkg = gate_arrays(c_pkg)
    assert np.array_equal(m_ref, m_pkg) and np.array_equal(g_ref.view(np.uint64), g_pkg.view(np.uint64))

    cases = []
    # small BASS cases that exercise every branch (rotations accepted/rejected,
    # non-diagonal 2q gates through the hash path, diagonal fast path)
    cases.append(("bass_tfim_n10_k32", 10, 32, pkg.circuits.tfim_circuit(
        10, 12, J=1.0, h=1.0, dt=0.3, rng=np.random.default_rng(3), disorder_strength_h=0.5), {}))
    cases.append(("bass_brick_n12_k64", 12, 64, pkg.circuits.brickwork_circuit(
        12, 10, rng=np.random.default_rng(4)), {}))
    cases.append(("bass_brick_n16_k256_opt1", 16, 256, pkg.circuits.brickwork_circuit(
        16, 12, rng=np.random.default_rng(5)), {"optimize_every": 1, "buffer_factor": 1}))
    np.random.seed(11)
    rnd = R["rc"].generate_random_circuit(12, 6)
    cases.append(("bass_haar2q_n12_k128", 12, 128, rnd, {}))
    cases.append(("bass_brick_n20_k512_trunc2", 20, 512, pkg.circuits.brickwork_circuit(
        20, 8, rng=np.random.default_rng(6)), {"truncate_every": 2}))
    if not args.skip_large:
        cases.append(("config1_tfim_n24_k65536", 24, 2 ** 16, c_pkg, {}))
        cases.append(("config2_brick_n40_d30_k1024", 40, 2 ** 10, pkg.circuits.config2_circuit(seed=0), {}))
        cases.append(("config2_brick_n40_d12_k4096", 40, 2 ** 12, pkg.circuits.config2_circuit(seed=1, depth=12), {}))
    write_bass_cases(R, cases)

    # FixedBasisSimulator: top-k and random-k (seeded)
    for name, trunc in [("fixed_topk_n12_k64", "top-k"), ("fixed_randk_n12_k64", "random-k")]:
        circ = pkg.circuits.tfim_circuit(12, 8, J=1.0, h=1.0, dt=0.3, rng=np.random.default_rng(8),
                                         disorder_strength_h=0.5)
        np.random.seed(13)
        circ = circ + R["rc"].generate_random_circuit(12, 2)
        f = R["fs"].FixedBasisSimulator(12, 64, truncation=trunc, verbose=False)
        st = f.simulate(circ, seed=4242)
        met = f.get_metrics()
        meta, mats = gate_arrays(circ)
        x = st.x[:st.nnz].copy(); a = st.alpha[:st.nnz].copy(); o = np.argsort(x)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), N=np.int64(12), k=np.int64(64),
                            gate_meta=meta, gate_mats=mats, x=x[o], a=a[o], gamma=np.float64(st.gamma),
                            gamma_sq_hist=met["gamma_squared"], nnz_hist=met["nnz"])
        print(name, "nnz", st.nnz, "gamma", st.gamma)


if __name__ == "__main__":
    main()
