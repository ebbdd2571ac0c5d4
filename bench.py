#!/usr/bin/env python
"""Benchmark of the BASS sparse-state hot path on B200.

Workload (one step): ``BASS(40, 2**22).simulate(circuit)`` with default
BASS settings on the 1D brickwork circuit of 40 qubits and depth 30 (a
Haar-random SU(2) on every qubit each layer, CZ on alternating neighbour
pairs each skipped with probability 1/2; seeded synthetic circuit), complex128
amplitudes, uint64 keys, top-k budget K = 2^22.  Metric: amplitude updates per
second (one amplitude update = one input entry transformed by one gate or one
basis-rotation step; counted on the device).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs one process per GPU (torchrun), each an independent replica of the
workload (the path does not shard); value = sum of all ranks' updates / the
slowest rank's time.  ``--impl reference`` times the CPU oracle (a plain-C
restatement of the reference's Numba kernels driven like the reference) on a
bounded sample of the same workload: the first 28 gates at K = 2^22.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "bass-basis-adapative-sparse-simulations-_b200")
CPU_SAMPLE_GATES = 28


def load_pkg():
    if "bass_b200" in sys.modules:
        return sys.modules["bass_b200"]
    spec = importlib.util.spec_from_file_location("bass_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    m = importlib.util.module_from_spec(spec)
    sys.modules["bass_b200"] = m
    spec.loader.exec_module(m)
    return m


def args_parser():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=40)
    ap.add_argument("--depth", type=int, default=30)
    ap.add_argument("--k", type=int, default=2 ** 22)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-profile", action="store_true")
    ap.add_argument("--op", default=None, choices=["gate1", "rot1", "gate2", "rdm"],
                    help="time one op kind on a seeded random state of K entries instead of the "
                         "workload (a per-kernel microbenchmark; also the small case for ncu)")
    ap.add_argument("--dtype", default="complex128", choices=["complex128", "complex64"])
    return ap


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(self.rows)}


# ---------------------------------------------------------------------------
# CPU baseline (oracle port of the reference's algorithm)
# ---------------------------------------------------------------------------
def cpu_sample(circuit, n, k):
    sys.path.insert(0, ROOT)
    from oracle import oracle
    oracle.build()
    b = oracle.OracleBASS(n, k)
    t0 = time.perf_counter()
    b.simulate(circuit[:CPU_SAMPLE_GATES])
    dt = time.perf_counter() - t0
    return b.stats["amp_updates"], dt


def run_reference(a, rank, world):
    if rank != 0:
        return
    pkg = load_pkg()
    circ = pkg.circuits.config2_circuit(seed=a.seed, num_qubits=a.n, depth=a.depth)
    for _ in range(a.warmup):
        cpu_sample(circ, a.n, a.k)
    ups, secs = [], []
    for _ in range(a.steps):
        u, dt = cpu_sample(circ, a.n, a.k)
        ups.append(u)
        secs.append(dt)
    value = sum(ups) / sum(secs)
    sample = f"first {CPU_SAMPLE_GATES} gates of the workload circuit at K={a.k}, per step"
    line = {
        "impl": "reference", "metric": "amp_updates_per_s", "value": value, "unit": "amp-updates/s",
        "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * sum(secs) / len(secs),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "complex128",
        "data": "synthetic (seeded brickwork circuit)",
        "config": workload_config(a),
        "cpu_baseline": {"value": value, "unit": "amp-updates/s", "cores": 1, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "amp-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def workload_config(a):
    return {"workload": f"BASS brickwork n={a.n} depth={a.depth} K=2^{a.k.bit_length() - 1} complex128",
            "n_qubits": a.n, "depth": a.depth, "K": a.k, "optimize_every": 5, "buffer_factor": 2,
            "parallelism": f"replicas x{a.gpus}", "l2": "flushed between steps (512 MB write)"}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(a, rank, world, dist):
    import numpy as np
    import torch
    pkg = load_pkg()
    from bass_b200 import _native
    from bass_b200.bass import BASS
    _native.build()
    L = _native.lib()
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    circ = pkg.circuits.config2_circuit(seed=a.seed, num_qubits=a.n, depth=a.depth)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)

    def barrier():
        if dist is not None:
            dist.barrier()

    def step():
        b = BASS(a.n, a.k)
        st = b.simulate(circ)
        return b, st

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()

    sampler = ClockSampler(dev.index)
    sampler.start()
    launches0 = L.bass_launch_count()
    times, ups = [], []
    for _ in range(a.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        b, st = step()
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
        ups.append(b.stats["amp_updates"])
    launches = (L.bass_launch_count() - launches0) // max(a.steps, 1)
    clocks = sampler.stop()
    t_total, u_total = over_ranks(dist, dev, sum(times), float(sum(ups)))
    value = u_total / t_total

    # end to end through the public API: host circuit in, host state (x, alpha) out
    e2e_t, e2e_u, h2d, d2h = [], [], 0, 0
    for _ in range(a.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        b = BASS(a.n, a.k)
        st = b.simulate(circ)
        x, al = st.x, st.alpha
        t1 = time.perf_counter()
        e2e_t.append(t1 - t0)
        e2e_u.append(b.stats["amp_updates"])
        h2d = sum(g.matrix.nbytes for g in circ)
        d2h = x.nbytes + al.nbytes
    e2e_total, e2e_units = over_ranks(dist, dev, sum(e2e_t), float(sum(e2e_u)))
    e2e_value = e2e_units / e2e_total

    roofline = None
    kernels = None
    if not a.no_profile:
        roofline, kernels = profile_step(a, circ, L, _native, BASS, torch, 1e3 * t_total / a.steps)

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        u, dt = cpu_sample(circ, a.n, a.k)
        cpu = {"value": u / dt, "unit": "amp-updates/s", "cores": 1, "kind": "port",
               "sample": f"first {CPU_SAMPLE_GATES} gates of the workload circuit at K={a.k} "
                         f"({dt:.1f} s, {u} updates)"}

    if rank == 0:
        line = {
            "metric": "amp_updates_per_s", "value": value, "unit": "amp-updates/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * t_total / a.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "complex128",
            "data": "synthetic (seeded brickwork circuit)", "config": workload_config(a),
            "e2e": {"value": e2e_value, "unit": "amp-updates/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": int(launches), "clocks": clocks, "roofline": roofline, "cpu_baseline": cpu,
            "amp_updates_per_step": int(statistics.mean(ups)), "kernels": kernels,
            "bass_stats": {k: int(v) for k, v in b.stats.items()},
        }
        print(json.dumps(line), flush=True)


def profile_step(a, circ, L, nat, BASS, torch, step_ms):
    """One extra step with per-launch CUDA events and per-kernel entry counters."""
    import numpy as np
    L.bass_profile_enable(1)
    ms = np.zeros(nat.PROF_SLOTS)
    cnt = np.zeros(nat.PROF_SLOTS, dtype=np.int64)
    L.bass_profile_collect(nat._host(ms), nat._host(cnt), nat.PROF_SLOTS)
    b = BASS(a.n, a.k)
    st = b.simulate(circ)
    torch.cuda.synchronize()
    c = st._eng.read_ctrl()
    L.bass_profile_collect(nat._host(ms), nat._host(cnt), nat.PROF_SLOTS)
    L.bass_profile_enable(0)
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    kernels = []
    for s in np.argsort(-ms):
        if ms[s] <= 0:
            break
        nbytes = 24 * (int(c["prof_in"][s]) + int(c["prof_out"][s]))
        kernels.append({"kernel": nat.SLOT_NAMES[s], "ms": round(float(ms[s]), 3), "launches": int(cnt[s]),
                        "share": round(float(ms[s] / ms.sum()), 4),
                        "gbs": round(nbytes / (ms[s] * 1e-3) / 1e9, 1) if nbytes else None})
    phases = select_phases(c, nat)
    tile_slots = [s for s in range(30) if ms[s] > 0]
    dom = max(tile_slots, key=lambda s: ms[s])
    per_launch_bytes = 24 * (int(c["prof_in"][dom]) + int(c["prof_out"][dom])) / cnt[dom]
    avg_s = ms[dom] * 1e-3 / cnt[dom]
    achieved = per_launch_bytes / avg_s / 1e9
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic_per_entry.json")
    if os.path.exists(tfile):
        tj = json.load(open(tfile))
        if nat.SLOT_NAMES[dom] in tj:
            traffic = tj[nat.SLOT_NAMES[dom]] * per_launch_bytes / 24
    # the whole simulate call: every gate / rotation / truncation reads its
    # input once and writes its output once (24 B per entry each way), over
    # the timed step's duration (RDMs, selection, partitions all included)
    kinds = (0, 1, 2, 4)  # gate1, rot1, gate2, plain; the 2-qubit gate's first pass is overhead
    step_bytes = 24 * (sum(int(c["prof_in"][k * 5 + 0]) for k in kinds) +
                       sum(int(c["prof_out"][k * 5 + 3]) for k in kinds))
    step_gbs = step_bytes / (step_ms * 1e-3) / 1e9
    top = int(np.argmax(ms))  # the longest kernel overall (the selection has no algorithmic bytes of its own)
    roof = {"bound": "hbm", "kernel": nat.SLOT_NAMES[dom], "achieved": round(achieved, 1), "peak": peak,
            "peak_source": peak_src, "unit": "GB/s", "frac": round(achieved / peak, 4),
            "traffic": traffic, "bytes_per_launch": per_launch_bytes,
            "whole_step": {"achieved": round(step_gbs, 1), "frac": round(step_gbs / peak, 4),
                           "bytes_per_step": step_bytes,
                           "note": "24 B per entry read + 24 B per entry written by every gate, rotation step "
                                   "and truncation, over the timed step"},
            "longest_kernel": {"kernel": nat.SLOT_NAMES[top], "share": round(float(ms[top] / ms.sum()), 4),
                               "note": "share of the profiled step; the roofline above is that of the "
                                       "longest tile pass, the kernels that move the state's own bytes"},
            "note": "algorithmic bytes = 24 B per entry read + 24 B per entry written; timing from a "
                    "profiled step (CUDA events around each launch on its stream)"}
    kernels = kernels[:12]
    if phases:
        kernels.append({"kernel": "k_select_coop phases (us per launch)", **phases})
    return roof, kernels


def run_op(a):
    """One op kind, repeated on a state of K entries: a seeded random state
    (40-bit keys, Gaussian amplitudes, so |a|^2 is exponentially distributed
    as in a scrambled circuit).  gate1 / gate2: a Haar-random gate with the
    simulate-level top-K truncation fused (the state stays at K entries);
    rot1: a basis-rotation step (rotate, keep the top K, accept if PR drops);
    rdm: the 1-qubit RDMs of all qubits.  Targets cycle over the qubits.
    Prints one JSON line: ms per op and the per-kernel table (CUDA events
    around each launch)."""
    import numpy as np
    import torch
    import ctypes
    pkg = load_pkg()
    from bass_b200 import _native as nat
    from bass_b200.state import SparseState
    nat.build()
    L = nat.lib()
    torch.cuda.set_device(0)
    rng = np.random.default_rng(a.seed)
    n, K = a.n, a.k
    x = np.unique(rng.integers(0, 2 ** n, size=K + K // 8 + 64, dtype=np.uint64))[:K]
    amp = rng.standard_normal(len(x)) + 1j * rng.standard_normal(len(x))
    amp /= np.sqrt(np.vdot(amp, amp).real)
    dt = np.dtype(a.dtype)
    st = SparseState(n, K, dtype=dt, _capacity=K + 16)
    st.load(x, amp.astype(dt))
    eng = st._eng
    tr = nat.trunc(K, K, 1, 1, 1, 0)
    eng.set_ctrl("pr_cur", 1e300)

    def haar(d):
        z = (rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))) / np.sqrt(2)
        qm, r = np.linalg.qr(z)
        return qm * (np.diag(r) / np.abs(np.diag(r)))

    def one(i):
        q = (7 * i) % n
        if a.op == "gate1":
            st._apply_1q(haar(2), q, tr)
        elif a.op == "gate2":
            q2 = (q + 1) % n
            st._apply_2q(haar(4), q, q2, tr)
        elif a.op == "rot1":
            th = 0.3 + 0.1 * (i % 5)
            U = np.array([[np.cos(th), -np.sin(th)], [np.sin(th), np.cos(th)]], dtype=np.complex128)
            nat.check(L.bass_rotate_step(st._cur.ptr, st._tmp.ptr, nat._host(nat.host_c128(U)), q, K, 0,
                                         eng.ctrl_ptr, eng.ws_ptr, eng.ws_bytes, eng.stream), "bass_rotate_step")
            eng.set_ctrl("pr_cur", 1e300)   # every candidate is accepted: the state keeps changing
        else:
            nat.check(L.bass_rdm_1q(st._cur.ptr, n, ctypes.c_void_p(nat._ptr(eng.rho)), eng.ctrl_ptr,
                                    eng.ws_ptr, eng.ws_bytes, eng.stream), "bass_rdm_1q")

    for i in range(a.warmup):
        one(i)
    torch.cuda.synchronize()
    L.bass_profile_enable(1)
    ms = np.zeros(nat.PROF_SLOTS)
    cnt = np.zeros(nat.PROF_SLOTS, dtype=np.int64)
    L.bass_profile_collect(nat._host(ms), nat._host(cnt), nat.PROF_SLOTS)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for i in range(a.steps):
        one(a.warmup + i)
    e1.record()
    torch.cuda.synchronize()
    L.bass_profile_collect(nat._host(ms), nat._host(cnt), nat.PROF_SLOTS)
    L.bass_profile_enable(0)
    eng.raise_on_error()
    c = eng.read_ctrl()
    kern = []
    B = 24 if dt == np.complex128 else 16
    for sl in np.argsort(-ms):
        if ms[sl] <= 0:
            break
        nb = B * (int(c["prof_in"][sl]) + int(c["prof_out"][sl]))
        kern.append({"kernel": nat.SLOT_NAMES[sl], "us_per_launch": round(1e3 * ms[sl] / max(cnt[sl], 1), 2),
                     "launches": int(cnt[sl]), "share": round(float(ms[sl] / ms.sum()), 4),
                     "gbs": round(nb / (ms[sl] * 1e-3) / 1e9, 1) if nb else None})
    phases = select_phases(c, nat)
    print(json.dumps({"op": a.op, "K": K, "n_qubits": n, "dtype": a.dtype, "nnz": st.nnz,
                      "select_phases_us": phases,
                      "us_per_op": round(1e3 * e0.elapsed_time(e1) / a.steps, 2),
                      "us_per_op_profiled": round(1e3 * ms.sum() / a.steps, 2), "kernels": kern}), flush=True)


def select_phases(c, nat):
    """Mean microseconds per selection launch of each of its phases."""
    out = {}
    for sl in nat.SELECT_PHASE_SLOTS:
        nl = int(c["prof_out"][sl])
        if nl:
            out[nat.SLOT_NAMES[sl]] = round(int(c["prof_in"][sl]) / nl / 1e3, 2)
    nl = int(c["prof_out"][nat.SELECT_SPEC_SLOT])
    if nl:
        out["two_level_frac"] = round(int(c["prof_in"][nat.SELECT_SPEC_SLOT]) / nl, 3)
    return out


def over_ranks(dist, dev, seconds, units):
    """The job's time (max over ranks) and units (sum over ranks); replicas
    share nothing else."""
    if dist is None:
        return float(seconds), float(units)
    import torch
    tt = torch.tensor([float(seconds)], dtype=torch.float64, device=dev)
    uu = torch.tensor([float(units)], dtype=torch.float64, device=dev)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    dist.all_reduce(uu, op=dist.ReduceOp.SUM)
    return float(tt.item()), float(uu.item())


def main():
    a = args_parser().parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    dist = None
    if a.impl == "reference":
        run_reference(a, rank, world)
        return
    if a.op is not None:
        run_op(a)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist
    try:
        run_ours(a, rank, world, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
