"""The served form: an open-loop Poisson request stream through BassServer.

Checked: every request completes; admission keeps the resident footprint under
the budget (which is set small here so that requests wait for memory); each
result is bit-identical to the same request run alone, and, where the plain
complex128 run keeps no basis rotation, matches it to fidelity >= 1 - 1e-6
(site-disordered fields: no top-k ties; see test_gpu_batch.py on rotations).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env(pkg):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from bass_b200 import _native
    _native.build()
    return pkg


def _requests(pkg, count=24):
    tfim = dict(n_range=(10, 20), layer_range=(3, 10), m_range=(6, 11), dt=0.3, disorder_h=0.25)
    return pkg.circuits.config5_requests(seed=5, count=count, tfim=tfim, brick_n=(10, 18), brick_depth=(4, 10),
                                         brick_m=(6, 10))


def _fid(x1, a1, x2, a2):
    d = dict(zip(x1.tolist(), a1.astype(np.complex128)))
    ov = sum(np.conj(d.get(k, 0.0)) * complex(v) for k, v in zip(x2.tolist(), a2))
    return abs(ov) ** 2 / (np.vdot(a1, a1).real * np.vdot(a2, a2).real)


def test_served_stream(env):
    from bass_b200.batch import BatchedBASS, state_bytes
    from bass_b200.bass import BASS
    from bass_b200.served import BassServer, poisson_arrivals
    reqs = _requests(env)
    arrivals = poisson_arrivals(400.0, 10.0, np.random.default_rng(1))[:len(reqs)]
    assert len(arrivals) == len(reqs)
    budget = 3 * max(state_bytes(n, k) for _, n, k in reqs)
    srv = BassServer(budget_bytes=budget)
    res = srv.serve(reqs, arrivals)
    assert sorted(r.index for r in res) == list(range(len(reqs))) and not srv.unfinished
    assert srv.peak_bytes <= budget
    s = srv.summary(res)
    assert s["completed"] == len(reqs) and s["p99_s"] >= s["p50_s"] > 0
    for r in res[:: max(1, len(res) // 8)]:
        circ, n, k = reqs[r.index]
        alone = BatchedBASS([(n, k)]).simulate([circ])[0]
        assert np.array_equal(alone.x, r.x) and np.array_equal(alone.alpha, r.alpha)
        assert alone.gamma == r.gamma
        b = BASS(n, k)
        plain = b.simulate(circ)
        # without basis rotations (on either side) the runs are comparable entry by entry
        if not b.stats["accepted"] and all(np.array_equal(u, np.eye(2)) for u in alone.U):
            assert _fid(plain.x, plain.alpha, r.x, r.alpha) >= 1 - 1e-6
