"""Parity at the benchmark's own size: BASS(40, 2**22) on the seeded brickwork
circuit of 40 qubits and depth 30 (the workload bench.py times), against the
CPU oracle's run of the same circuit recorded in
tests/golden/config2_brick_n40_d30_k4194304_oracle.npz (made by
tests/golden/make_oracle_trace.py; the oracle is pinned to the reference's
own outputs by the smaller fixtures).

Compared: every trace event (each renormalisation point with nnz and the
fingerprints of all keys and of the significant keys, every accepted
rotation, every optimisation that passed its PR gate), the final key set and
(key, amplitude bits) fingerprints, gamma bit for bit, the frames U, and the
update / rotation counters.  The GPU and the oracle use the same arithmetic
(no FMA, exact sums), so the comparison is exact."""
import os

import numpy as np
import pytest

from _common import GOLDEN, first_mismatch, pair_fingerprint

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(GOLDEN, "config2_brick_n40_d30_k4194304_oracle.npz")


@pytest.mark.skipif(not os.path.exists(FIXTURE), reason="oracle trace of the headline run not recorded")
def test_headline_run_matches_oracle_trace(pkg):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from bass_b200 import _native
    from bass_b200.bass import BASS
    _native.build()
    z = np.load(FIXTURE)
    n, k, depth, seed = int(z["N"]), int(z["k"]), int(z["depth"]), int(z["seed"])
    circ = pkg.circuits.config2_circuit(seed=seed, num_qubits=n, depth=depth)
    b = BASS(n, k, trace=True)
    st = b.simulate(circ)
    mine = [tuple(int(v) for v in e) for e in b.trace_events()]
    ref = [tuple(int(v) for v in e) for e in z["events"]]
    assert first_mismatch(mine, ref) is None, f"first divergent event {first_mismatch(mine, ref)}"
    assert len(mine) == len(ref)
    assert st.nnz == int(z["nnz"])
    x, a = st.x, st.alpha
    assert np.array_equal(np.array(pair_fingerprint(x, a), dtype=np.uint64), z["fp_pair"])
    fp = st._cur.fingerprint(_native.SIG_PMIN)
    assert np.array_equal(np.array(fp[:3], dtype=np.uint64), z["fp_all"])
    assert np.array_equal(np.array(fp[3:6], dtype=np.uint64), z["fp_sig"])
    assert st.gamma == float(z["gamma"])
    for j in range(n):
        assert np.array_equal(b.U[j], z["U"][j])
    assert b.stats["amp_updates"] == int(z["amp_updates"])
    assert b.stats["rotations"] == int(z["rotations"]) and b.stats["accepted"] == int(z["accepted"])
    assert b.stats["opt_calls"] == int(z["opt_calls"])
