"""Serving BASS simulations: continuous batching of circuit requests on one GPU.

``BassServer.serve(requests, arrivals)`` replays an open-loop request stream
(request i becomes visible ``arrivals[i]`` seconds after the start).  Arrived
requests wait in a FIFO queue and are admitted while their device footprint
(``batch.state_bytes``: state buffers and workspace for min(K, 2^n) entries)
fits the state budget and a batch slot is free.  Every admitted request stays
resident on the device until it finishes; each stage advances every resident
request by one gate through the segmented launches of ``batch.StatePool``, so
requests that arrive while others run join the next stage and their work
shares the same launches.  A finished request's state is read back to the host
(keys, amplitudes, gamma) and its memory returns to the budget.

Latency of a request = the time its result is on the host minus its arrival
time (queueing included).  ``summary`` reports completed circuits per second
and the p50 / p99 latency.  A request's result does not depend on the other
requests it shared stages with (the kernels' results do not depend on their
block grouping; see tests/test_gpu_served.py).
"""
from __future__ import annotations

import time
from collections import deque

import numpy as np

from .batch import MAX_SEG, StatePool, state_bytes


def poisson_arrivals(rate, duration, rng):
    """Arrival times of a Poisson process of the given rate (per second) in [0, duration)."""
    t, out = 0.0, []
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t >= duration:
            return np.array(out)
        out.append(t)


class Result:
    __slots__ = ("index", "arrival", "start", "finish", "x", "alpha", "gamma", "amp_updates")

    @property
    def latency(self):
        return self.finish - self.arrival


class BassServer:
    def __init__(self, budget_bytes=150e9, dtype=np.complex64, max_live=MAX_SEG, **bass_kw):
        self.budget = float(budget_bytes)
        self.dtype = np.dtype(dtype)
        self.max_live = int(max_live)
        self.bass_kw = bass_kw
        self.pool = None

    def footprint(self, num_qubits, k):
        return state_bytes(num_qubits, k, self.dtype)

    def serve(self, requests, arrivals, stop_after=None, clock=time.perf_counter):
        """requests[i] = (circuit, num_qubits, k); a sequence with a
        ``spec(i)`` method giving (num_qubits, k) is read lazily (a request's
        circuit is fetched when it is admitted).  Runs until every request has
        finished, or until ``stop_after`` seconds (requests still queued or
        running then are abandoned and listed in ``self.unfinished``).
        Returns the finished requests' Results in completion order."""
        import torch
        order = np.argsort(np.asarray(arrivals, dtype=np.float64), kind="stable")
        arrivals = np.asarray(arrivals, dtype=np.float64)
        spec = requests.spec if hasattr(requests, "spec") else (lambda i: tuple(requests[i][1:3]))
        fps = {}

        def fp(i):
            if i not in fps:
                fps[i] = self.footprint(*spec(i))
                if fps[i] > self.budget:
                    raise ValueError(f"request {i} does not fit the state budget on its own")
            return fps[i]
        pool = self.pool = StatePool(max_slots=min(self.max_live, MAX_SEG), dtype=self.dtype, **self.bass_kw)
        incoming = deque(int(i) for i in order)
        waiting = deque()
        meta = {}
        used = 0.0
        done = []
        self.peak_bytes = 0.0
        self.stages = 0
        t0 = clock()
        while incoming or waiting or pool.busy.any():
            now = clock() - t0
            if stop_after is not None and now >= stop_after:
                break
            while incoming and arrivals[incoming[0]] <= now:
                waiting.append(incoming.popleft())
            # admission: FIFO while the footprint fits and a slot is free, on
            # stages that keep every resident request's optimisation points
            # on the same stages (their rotation steps then share launches)
            while waiting and pool.free_slots() and pool.in_phase() and used + fp(waiting[0]) <= self.budget:
                i = waiting.popleft()
                c = pool.add(*requests[i])
                meta[c] = (i, now)
                used += fp(i)
            self.peak_bytes = max(self.peak_bytes, used)
            if not pool.busy.any():
                if incoming:   # idle until the next arrival
                    time.sleep(max(0.0, min(arrivals[incoming[0]] - (clock() - t0), 0.01)))
                continue
            finished = pool.step()
            self.stages += 1
            finished = np.concatenate([finished, np.nonzero(pool.busy & (pool.pos >= pool.length))[0]])
            for c in np.unique(finished).astype(int):
                st = pool.take(c)
                r = Result()
                r.index, r.start = meta.pop(c)
                r.x, r.alpha, r.gamma, r.amp_updates = st.x, st.alpha, st.gamma, st.amp_updates
                torch.cuda.current_stream().synchronize()
                r.finish = clock() - t0
                r.arrival = float(arrivals[r.index])
                used -= fp(r.index)
                done.append(r)
                if hasattr(requests, "release"):
                    requests.release(r.index)
        self.elapsed = clock() - t0
        self.unfinished = [i for i, _ in meta.values()] + list(waiting) + list(incoming)
        self.stats = dict(pool.stats)
        return done

    def summary(self, results, elapsed=None):
        elapsed = self.elapsed if elapsed is None else elapsed
        lat = np.array([r.latency for r in results]) if results else np.zeros(0)
        return {
            "completed": len(results), "unfinished": len(getattr(self, "unfinished", [])),
            "circuits_per_s": len(results) / elapsed if elapsed > 0 else 0.0,
            "p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
            "elapsed_s": elapsed, "stages": self.stages, "peak_state_bytes": self.peak_bytes,
            "amp_updates": int(sum(r.amp_updates for r in results)),
        }
