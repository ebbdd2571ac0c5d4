"""bench.py's multi-rank logic on CPU: two gloo ranks (replicas only, the
process group carries the barrier and the timing reduction and nothing else)."""
import importlib.util
import os
import socket

import pytest

from conftest import ROOT


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        b = _bench()
        dist.barrier()
        t, u = b.over_ranks(dist, torch.device("cpu"), 1.0 + rank, 10.0 * (rank + 1))
        q.put((rank, t, u))
    finally:
        dist.destroy_process_group()


def test_over_ranks_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, t, u in got:
        assert t == 2.0 and u == 30.0          # time: max over ranks; units: sum


def test_single_process_is_identity():
    b = _bench()
    assert b.over_ranks(None, None, 3.5, 7.0) == (3.5, 7.0)


def test_reference_arm_other_ranks_print_nothing(capsys):
    b = _bench()
    a = b.args_parser().parse_args(["--impl", "reference", "--steps", "1", "--warmup", "0"])
    b.run_reference(a, rank=1, world=2)
    assert capsys.readouterr().out == ""
