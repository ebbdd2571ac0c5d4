"""The oracle's kernels on several host threads give the single-threaded
results bit for bit (the CPU baseline of bench.py runs them on every host
thread; the parity tests run them on one).  Sizes above the per-thread
minimum of 32768 items, so the parallel paths run."""
import numpy as np
import pytest


@pytest.fixture()
def threads(orc):
    yield orc
    orc.set_threads(1)


def _state(rng, N, n):
    x = np.unique(rng.integers(0, 2 ** N, size=n + n // 4, dtype=np.uint64))[:n]
    x = rng.permutation(x)
    a = rng.standard_normal(len(x)) + 1j * rng.standard_normal(len(x))
    a[::97] = 0.0
    return x, a


def _run_all(orc, x, a, N):
    rng = np.random.default_rng(11)
    G = np.linalg.qr(rng.standard_normal((2, 2)) + 1j * rng.standard_normal((2, 2)))[0]
    out = {}
    out["apply_1q"] = orc.apply_1q(x, a, G, 5)
    xs, as_ = np.sort(x), a[np.argsort(x)]
    out["rotate_1q"] = orc.rotate_1q(x, a, 7, G)
    out["rotate_1q_sorted"] = orc.rotate_1q(xs, as_, N - 1, G)
    out["select_topk"] = orc.select_topk(x, a, len(x) // 3)
    ties = np.round(a, 1)   # many exactly equal |a|^2: the key tie-break decides
    out["select_ties"] = orc.select_topk(x, ties, len(x) // 2)
    out["rdm"] = orc.rdm_all(xs, as_, N)
    out["sums"] = (orc.sum_p(a), orc.sum_p2(a))
    kk = np.concatenate([xs, xs[::3]])
    aa = np.concatenate([as_, as_[::3]])
    o = np.argsort(kk, kind="stable")
    out["merge"] = orc.merge_sorted(kk[o], aa[o])
    return out


def _same(u, v):
    if isinstance(u, tuple):
        return len(u) == len(v) and all(_same(p, q) for p, q in zip(u, v))
    u, v = np.atleast_1d(np.asarray(u)), np.atleast_1d(np.asarray(v))
    return u.shape == v.shape and np.array_equal(u.view(np.uint8), v.view(np.uint8))


def test_threads_bit_identical(threads):
    orc = threads
    rng = np.random.default_rng(3)
    N = 30
    x, a = _state(rng, N, 200_000)
    orc.set_threads(1)
    one = _run_all(orc, x, a, N)
    n = orc.set_threads(4)
    assert n >= 1
    many = _run_all(orc, x, a, N)
    for k in one:
        assert _same(one[k], many[k]), k
