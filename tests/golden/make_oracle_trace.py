"""Record the CPU oracle's trace of a large BASS run as a golden fixture.

Usage:
  python tests/golden/make_oracle_trace.py [--n 40] [--depth 30] [--k 4194304] [--seed 0]

The default is the benchmark workload itself: ``BASS(40, 2**22)`` with default
settings on the seeded brickwork circuit of 40 qubits and depth 30.  The
reference (Python + Numba) would need days for it, so the fixture comes from
the oracle (``oracle/``: plain-C kernels driven like the reference's
``BASS.simulate``), which is pinned to the reference's own outputs at smaller
sizes by the other fixtures in this directory.  A single-threaded run takes
one to two hours.

Recorded (the state itself, 100 MB, is not stored):
  * the trace: every renormalisation point (nnz and the order-independent
    fingerprints of all keys and of the keys with |a|^2 > 1e-24), every
    accepted rotation, every optimisation that passed its PR gate;
  * the final state's fingerprints: all keys, significant keys, and the
    (key, amplitude-bits) pair fingerprint of ``tests/_common.py``;
  * gamma, the frames U, the update / rotation counters and the run time.
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle import oracle  # noqa: E402
from _common import pair_fingerprint  # noqa: E402


def load_pkg():
    import importlib.util
    d = os.path.join(ROOT, "bass-basis-adapative-sparse-simulations-_b200")
    spec = importlib.util.spec_from_file_location("bass_b200", os.path.join(d, "__init__.py"),
                                                  submodule_search_locations=[d])
    m = importlib.util.module_from_spec(spec)
    sys.modules["bass_b200"] = m
    spec.loader.exec_module(m)
    return m


def fixture_name(n, depth, k, seed):
    tag = f"config2_brick_n{n}_d{depth}_k{k}"
    return tag + ("_oracle" if seed == 0 else f"_s{seed}_oracle")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=40)
    ap.add_argument("--depth", type=int, default=30)
    ap.add_argument("--k", type=int, default=2 ** 22)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    oracle.build()
    pkg = load_pkg()
    circ = pkg.circuits.config2_circuit(seed=args.seed, num_qubits=args.n, depth=args.depth)
    tr = oracle.Trace()
    b = oracle.OracleBASS(args.n, args.k, trace=tr)
    t0 = time.perf_counter()
    st = b.simulate(circ)
    dt = time.perf_counter() - t0
    fp_all = oracle.fingerprint(st.x)
    fp_sig = oracle.fingerprint(st.x, st.alpha, oracle.SIG_PMIN)
    fp_pair = pair_fingerprint(st.x, st.alpha)
    stats = b.stats
    out = args.out or os.path.join(HERE, fixture_name(args.n, args.depth, args.k, args.seed) + ".npz")
    np.savez_compressed(
        out, N=np.int64(args.n), k=np.int64(args.k), depth=np.int64(args.depth), seed=np.int64(args.seed),
        events=tr.array(), gamma=np.float64(st.gamma), U=np.array(b.U),
        fp_all=np.array(fp_all, dtype=np.uint64), fp_sig=np.array(fp_sig, dtype=np.uint64),
        fp_pair=np.array(fp_pair, dtype=np.uint64), nnz=np.int64(st.nnz),
        amp_updates=np.int64(stats["amp_updates"]), rotations=np.int64(stats["rotations"]),
        accepted=np.int64(stats["accepted"]), opt_calls=np.int64(stats["opt_calls"]),
        seconds=np.float64(dt), pr_tie_tol=np.float64(b.pr_tie_tol))
    print(f"{out}: {len(tr.events)} events, nnz={st.nnz}, gamma={st.gamma:.12e}, "
          f"updates={stats['amp_updates']}, rotations={stats['rotations']}, accepted={stats['accepted']}, "
          f"{dt:.1f} s", flush=True)


if __name__ == "__main__":
    main()
