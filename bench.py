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
CPU_SAMPLE_GATES = 26   # the CPU sample: these gates, then a coordinate-descent pass ...
CPU_SAMPLE_QUBITS = 12  # ... over these first qubits


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
    ap.add_argument("--op", default=None,
                    help="comma-separated op kinds (gate1, rot1, gate2, rdm): time each on a seeded random "
                         "state of K entries instead of the workload (a per-kernel microbenchmark; also "
                         "the small case for ncu)")
    ap.add_argument("--dtype", default="complex128", choices=["complex128", "complex64"])
    ap.add_argument("--form", default=None, choices=["precision", "batched", "served"],
                    help="measure one of the other forms instead of the plain workload: precision "
                         "(complex64 TFIM n=24 K=2^16 against complex128), batched (256 TFIM circuits "
                         "of uneven size in segmented launches, against the plain path), served "
                         "(Poisson request stream through BassServer)")
    ap.add_argument("--count", type=int, default=256, help="batched form: circuits")
    ap.add_argument("--plain-every", type=int, default=8,
                    help="batched form: the plain path is timed on every this-many-th circuit")
    ap.add_argument("--rates", default="50,200,800", help="served form: arrival rates (circuits/s)")
    ap.add_argument("--seconds", type=float, default=60.0, help="served form: arrival window per rate")
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
def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_sample(circuit, n, k):
    """The CPU oracle (the reference's algorithm restated in C, driven like
    BASS.simulate) on every host thread: the workload's first CPU_SAMPLE_GATES
    gates (the state grows to K and truncation starts), then one pass of the
    basis optimisation over the first CPU_SAMPLE_QUBITS qubits (the RDMs, then
    for each qubit a rotation step with top-K and the PR decision).  Returns (amp-updates, seconds,
    rotation steps, threads); updates are counted as on the GPU (one input
    entry of a gate or rotation step)."""
    sys.path.insert(0, ROOT)
    from oracle import oracle
    oracle.build()
    threads = oracle.set_threads(0)
    b = oracle.OracleBASS(n, k)
    t0 = time.perf_counter()
    st = b.simulate(circuit[:CPU_SAMPLE_GATES])
    b._descent_pass(st, range(min(n, CPU_SAMPLE_QUBITS)))
    dt = time.perf_counter() - t0
    return b.stats["amp_updates"], dt, b.stats["rotations"], threads


def cpu_sample_text(k, dt, u, rot, threads):
    return (f"first {CPU_SAMPLE_GATES} gates of the workload circuit at K={k}, then one basis-optimisation pass "
            f"over qubits 0-{CPU_SAMPLE_QUBITS - 1} ({rot} rotation steps with top-K, one RDM), {threads} threads on {cpu_model()} "
            f"({dt:.1f} s, {u} updates)")


def run_reference(a, rank, world):
    if rank != 0:
        return
    pkg = load_pkg()
    circ = pkg.circuits.config2_circuit(seed=a.seed, num_qubits=a.n, depth=a.depth)
    for _ in range(a.warmup):   # loads and warms the oracle (a small budget: seconds, not minutes)
        cpu_sample(circ, a.n, 2 ** 10)
    ups, secs = [], []
    for _ in range(a.steps):
        u, dt, rot, threads = cpu_sample(circ, a.n, a.k)
        ups.append(u)
        secs.append(dt)
    value = sum(ups) / sum(secs)
    sample = "per step: " + cpu_sample_text(a.k, sum(secs) / len(secs), ups[0], rot, threads)
    line = {
        "impl": "reference", "metric": "amp_updates_per_s", "value": value, "unit": "amp-updates/s",
        "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * sum(secs) / len(secs),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "complex128",
        "data": "synthetic (seeded brickwork circuit)",
        "config": workload_config(a),
        "cpu_baseline": {"value": value, "unit": "amp-updates/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "amp-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def workload_config(a):
    return {"workload": f"BASS brickwork n={a.n} depth={a.depth} K=2^{a.k.bit_length() - 1} {a.dtype}",
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

    dt = np.dtype(a.dtype)

    def step():
        b = BASS(a.n, a.k, dtype=dt)
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
        b = BASS(a.n, a.k, dtype=dt)
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
        u, dt, rot, threads = cpu_sample(circ, a.n, a.k)
        cpu = {"value": u / dt, "unit": "amp-updates/s", "cores": threads, "kind": "port",
               "sample": cpu_sample_text(a.k, dt, u, rot, threads)}

    if rank == 0:
        line = {
            "metric": "amp_updates_per_s", "value": value, "unit": "amp-updates/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * t_total / a.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": a.dtype,
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
    b = BASS(a.n, a.k, dtype=np.dtype(a.dtype))
    st = b.simulate(circ)
    be = 24 if np.dtype(a.dtype) == np.complex128 else 16   # bytes per entry
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
        nbytes = be * (int(c["prof_in"][s]) + int(c["prof_out"][s]))
        kernels.append({"kernel": nat.SLOT_NAMES[s], "ms": round(float(ms[s]), 3), "launches": int(cnt[s]),
                        "share": round(float(ms[s] / ms.sum()), 4),
                        "gbs": round(nbytes / (ms[s] * 1e-3) / 1e9, 1) if nbytes else None})
    phases = select_phases(c, nat)
    tile_slots = [s for s in range(30) if ms[s] > 0]
    dom = max(tile_slots, key=lambda s: ms[s])
    per_launch_bytes = be * (int(c["prof_in"][dom]) + int(c["prof_out"][dom])) / cnt[dom]
    avg_s = ms[dom] * 1e-3 / cnt[dom]
    achieved = per_launch_bytes / avg_s / 1e9
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic_per_entry.json")
    if os.path.exists(tfile):
        tj = json.load(open(tfile))
        if nat.SLOT_NAMES[dom] in tj:
            traffic = tj[nat.SLOT_NAMES[dom]] * per_launch_bytes / be if be == 24 else None
    # the whole simulate call: every gate / rotation / truncation reads its
    # input once and writes its output once (24 B per entry each way), over
    # the timed step's duration (RDMs, selection, partitions all included)
    kinds = (0, 1, 2, 4)  # gate1, rot1, gate2, plain; the 2-qubit gate's first pass is overhead
    step_bytes = be * (sum(int(c["prof_in"][k * 5 + 0]) for k in kinds) +
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


def overlap_fidelity(x1, a1, x2, a2):
    """|<1|2>|^2 / (<1|1><2|2>) of two sparse states given as key / amplitude arrays."""
    import numpy as np
    a1 = np.asarray(a1, dtype=np.complex128)
    a2 = np.asarray(a2, dtype=np.complex128)
    o1 = np.argsort(x1)
    xs, as1 = np.asarray(x1)[o1], a1[o1]
    pos = np.searchsorted(xs, x2)
    pos = np.minimum(pos, max(len(xs) - 1, 0))
    hit = (len(xs) > 0) & (xs[pos] == x2) if len(xs) else np.zeros(len(x2), bool)
    ov = np.sum(np.conj(as1[pos[hit]]) * a2[hit]) if len(xs) else 0.0
    n1 = np.vdot(a1, a1).real
    n2 = np.vdot(a2, a2).real
    return float(abs(ov) ** 2 / (n1 * n2)) if n1 > 0 and n2 > 0 else 0.0


def perturbed_fidelity(pkg, spec, circ, ref_state, eps):
    """Fidelity between ref_state (BASS complex128 on circ) and BASS complex128
    on circ with its first 1-qubit gate preceded by an X rotation of eps rad."""
    import numpy as np
    from bass_b200.bass import BASS
    c2 = list(circ)
    j = next(t for t, g in enumerate(c2) if g.n_qubits == 1)
    R = np.array([[np.cos(eps), -1j * np.sin(eps)], [-1j * np.sin(eps), np.cos(eps)]])
    c2[j] = pkg.gates.QuantumGate(c2[j].qubits, R @ c2[j].matrix)
    st = BASS(*spec).simulate(c2)
    return overlap_fidelity(ref_state.x, ref_state.alpha, st.x, st.alpha)


def identity_frames(U):
    """Every frame of a finished batched / served state is the identity."""
    import numpy as np
    return all(np.array_equal(np.asarray(u), np.eye(2)) for u in U)


def timed(fn):
    """fn() timed with CUDA events on the current stream (synchronised)."""
    import torch
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    out = fn()
    e1.record()
    torch.cuda.synchronize()
    return out, e0.elapsed_time(e1) / 1e3


def form_precision(a, pkg):
    """Config 3: the config-1 TFIM circuit (n=24, 20 layers, K=2^16) with
    complex64 amplitudes against the complex128 run: throughput of both,
    fidelity, and the discarded weight of every simulate-level truncation."""
    import numpy as np
    from bass_b200.bass import BASS
    circ = pkg.circuits.config1_circuit(seed=a.seed)
    n, K = 24, 2 ** 16
    res = {}
    for name, dt in [("complex128", np.complex128), ("complex64", np.complex64)]:
        for _ in range(a.warmup):
            BASS(n, K, dtype=dt).simulate(circ)
        ts, ups = [], []
        for _ in range(a.steps):
            b = BASS(n, K, dtype=dt)
            st, t = timed(lambda: b.simulate(circ))
            ts.append(t)
            ups.append(b.stats["amp_updates"])
        rec = BASS(n, K, dtype=dt, record_truncations=True)
        rst = rec.simulate(circ)
        res[name] = {"amp_updates_per_s": sum(ups) / sum(ts), "ms_per_circuit": 1e3 * sum(ts) / len(ts),
                     "state": (rst.x, rst.alpha, rst.gamma, [np.array(u) for u in rec.U]),
                     "trunc": rec.truncations, "accepted": rec.stats["accepted"]}
    x1, a1, g1, U1 = res["complex128"]["state"]
    x2, a2, g2, U2 = res["complex64"]["state"]
    same_frames = all(np.array_equal(u, v) for u, v in zip(U1, U2))
    d128 = {i: 1.0 - kept / tot for i, kept, tot in res["complex128"]["trunc"]}
    d64 = {i: 1.0 - kept / tot for i, kept, tot in res["complex64"]["trunc"]}
    gates_per_layer = len(circ) // 20
    per_layer = {}
    for i in sorted(set(d128) | set(d64)):
        L = i // gates_per_layer
        per_layer.setdefault(L, [0.0, 0.0])
        per_layer[L][0] += d128.get(i, 0.0)
        per_layer[L][1] += d64.get(i, 0.0)
    out = {"form": "precision", "workload": "TFIM n=24 20 layers dt=0.1 h~U[0.5,1.5] K=2^16 (config 3)",
           "complex128": {k: v for k, v in res["complex128"].items() if k in ("amp_updates_per_s", "ms_per_circuit")},
           "complex64": {k: v for k, v in res["complex64"].items() if k in ("amp_updates_per_s", "ms_per_circuit")},
           "speedup_c64": res["complex64"]["amp_updates_per_s"] / res["complex128"]["amp_updates_per_s"],
           "fidelity_c64_vs_c128": overlap_fidelity(x1, a1, x2, a2) if same_frames else None,
           "same_frames": same_frames, "gamma_sq": {"complex128": g1 ** 2, "complex64": g2 ** 2},
           "discarded_weight_per_layer": {str(L): {"complex128": v[0], "complex64": v[1]}
                                          for L, v in sorted(per_layer.items())},
           "max_layer_discarded_diff": max((abs(v[0] - v[1]) for v in per_layer.values()), default=0.0)}
    return out


def form_batched(a, pkg):
    """Config 4: ``count`` TFIM circuits of uneven n, depth and K through
    BatchedBASS (complex64, segmented launches) against the plain complex128
    path (BASS.simulate one circuit at a time), timed on every
    ``plain_every``-th circuit; fidelity of the batched result to the plain
    one on those circuits."""
    import numpy as np
    from bass_b200.bass import BASS
    from bass_b200.batch import BatchedBASS
    specs, circs = pkg.circuits.config4_batch(seed=a.seed, count=a.count)
    BatchedBASS(specs[:4], dtype=np.complex64).simulate(circs[:4])   # warm-up: kernels loaded, pools built
    bb = BatchedBASS(specs, dtype=np.complex64)
    got, t_batch = timed(lambda: bb.simulate(circs))
    sample = list(range(0, len(specs), max(1, a.plain_every)))
    BASS(*specs[sample[0]]).simulate(circs[sample[0]])
    t_plain, fids, ups_plain = 0.0, [], 0
    for i in sample:
        b = BASS(*specs[i])
        st, t = timed(lambda: b.simulate(circs[i]))
        t_plain += t
        ups_plain += b.stats["amp_updates"]
        fids.append(overlap_fidelity(st.x, st.alpha, got[i].x, got[i].alpha)
                    if not b.stats["accepted"] and identity_frames(got[i].U) else None)
    comparable = [f for f in fids if f is not None]
    plain_cps = len(sample) / t_plain
    batch_cps = len(specs) / t_batch
    # precision on tie-free inputs: the same distribution with site-disordered
    # fields (a uniform field on the open chain makes mirror-image amplitudes
    # exactly equal, and complex64 rounding then breaks top-k ties differently)
    nd = min(64, len(specs))
    specs_d, circs_d = pkg.circuits.config4_batch(seed=a.seed + 1, count=nd, disorder_h=0.25)
    got_d = BatchedBASS(specs_d, dtype=np.complex64).simulate(circs_d)
    fd, split, low = [], 0, []
    for i in range(nd):
        b = BASS(*specs_d[i])
        st = b.simulate(circs_d[i])
        same = not b.stats["accepted"] and identity_frames(got_d[i].U)
        split += (not b.stats["accepted"]) != identity_frames(got_d[i].U)
        if same:
            fd.append(overlap_fidelity(st.x, st.alpha, got_d[i].x, got_d[i].alpha))
            if fd[-1] < 1 - 1e-6:
                rec = {"n": specs_d[i][0], "K": specs_d[i][1], "gates": len(circs_d[i]),
                       "truncations": int(b.stats["truncations"]), "fidelity": fd[-1]}
                if len(low) < 8:
                    # the same complex128 run with the first 1-qubit gate turned by a further
                    # 1e-7 rad about X: how far the truncated evolution carries a perturbation
                    # of the size of complex64 rounding
                    rec["complex128_perturbed_1e-7"] = perturbed_fidelity(pkg, specs_d[i], circs_d[i], st, 1e-7)
                low.append(rec)
    return {"form": "batched", "workload": f"{len(specs)} TFIM circuits, n~U[16,48], layers~U[10,60], "
                                           "h~U[0.3,2], dt=0.05, K=2^U[10,20] (config 4)",
            "batched_complex64": {"circuits_per_s": batch_cps, "seconds": t_batch,
                                  "amp_updates_per_s": bb.stats["amp_updates"] / t_batch},
            "plain_complex128": {"circuits_per_s": plain_cps, "circuits_timed": len(sample), "seconds": t_plain,
                                 "amp_updates_per_s": ups_plain / t_plain},
            "speedup_circuits_per_s": batch_cps / plain_cps,
            "fidelity_min": min(comparable) if comparable else None, "fidelity_compared": len(comparable),
            "fidelity_below_1e-6": sum(1 for f in comparable if f < 1 - 1e-6),
            "tie_free": {"circuits": nd, "compared": len(fd), "fidelity_min": min(fd) if fd else None,
                         "fidelity_below_1e-6": sum(1 for f in fd if f < 1 - 1e-6),
                         "rotation_decisions_differ": split, "below": low[:12],
                         "note": "config-4 distribution with site fields h_i ~ U[h - 0.25, h + 0.25]"},
            "fidelity_note": "compared entry by entry where neither run kept a basis rotation (both in the "
                             "computational basis); a run that kept one holds its state in another frame, and "
                             "a near-tie PR decision can go either way under complex64 rounding"}


def form_served(a, pkg):
    """Config 5: open-loop Poisson request streams (one per rate) through
    BassServer: circuits/s, p50 / p99 latency; the plain path's circuits/s on
    the same request mix for comparison (every plain_every-th request)."""
    import numpy as np
    from bass_b200.bass import BASS
    from bass_b200.served import BassServer, poisson_arrivals
    out = {"form": "served", "workload": "requests 50/50 TFIM (config 4 distribution) or brickwork n~U[20,44], "
                                         "depth~U[10,30], K=2^U[12,22]; 150 GB state budget (config 5)",
           "seconds_per_rate": a.seconds, "rates": {}}
    for r, rate in enumerate(float(x) for x in a.rates.split(",")):
        rng = np.random.default_rng(a.seed + 17 * r)
        arr = poisson_arrivals(rate, a.seconds, rng)
        reqs = pkg.circuits.Config5Stream(seed=a.seed + r, count=len(arr))
        srv = BassServer(budget_bytes=150e9)
        res = srv.serve(reqs, arr, stop_after=a.seconds + 30.0)
        summ = srv.summary(res)
        out["rates"][str(int(rate))] = {k: summ[k] for k in ("completed", "unfinished", "circuits_per_s", "p50_s",
                                                            "p99_s", "elapsed_s", "peak_state_bytes")}
        out["rates"][str(int(rate))]["offered"] = len(arr)
    reqs = pkg.circuits.config5_requests(seed=a.seed, count=max(8, 4 * a.plain_every))
    sample = reqs[::max(1, a.plain_every // 2)]
    t_plain = 0.0
    for circ, n, k in sample:
        b = BASS(n, k)
        _, t = timed(lambda: b.simulate(circ))
        t_plain += t
    out["plain_complex128_circuits_per_s"] = len(sample) / t_plain
    return out


def run_form(a):
    import torch
    pkg = load_pkg()
    from bass_b200 import _native
    _native.build()
    torch.cuda.set_device(0)
    fn = {"precision": form_precision, "batched": form_batched, "served": form_served}[a.form]
    print(json.dumps(fn(a, pkg)), flush=True)


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
        import copy
        for op in a.op.split(","):
            if op not in ("gate1", "rot1", "gate2", "rdm"):
                raise SystemExit(f"unknown op {op}")
            b = copy.copy(a)
            b.op = op
            run_op(b)
        return
    if a.form is not None:
        run_form(a)
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
