"""Batched BASS: many independent circuits advanced together on one GPU.

``BatchedBASS(specs).simulate(circuits)`` runs ``BASS(num_qubits, k).simulate``
(bass_simulator.py:847-929, default settings) for every circuit, with the
circuits of uneven qubit count, depth and budget k advancing together, one
gate each per stage.  At each stage the ops of all live circuits go to the GPU
as segmented launches (include/bass_b200.h, ``bass_*_batch``): one set of
launches per op kind for all circuits, each kernel's grid split into one block
group per state in proportion to its size.  The optimisation points are
batched the same way: one device-to-host read of every circuit's control
block decides which circuits optimise, their RDMs come from one segmented
launch, the 2x2 eigen-solves run vectorised on the host, and coordinate step j
rotates qubit j of every optimising circuit in one segmented launch.

``StatePool`` is the machinery: slots that circuits enter (``add``) and leave
(``take``) between stages, so a server can admit requests while others run
(``served.py``).  A circuit's stages do not depend on which other circuits
share them.

Default amplitudes are complex64 (the precision form: FP32 gate arithmetic
with compensated sums, FP64 norms, threshold, discarded weight and moments).
Frames that are not the identity are applied with the same numpy
expressions as ``BASS.simulate``, and every kernel's result is independent of
the block group that computes it, so a complex128 batch reproduces the plain
path bit for bit; a complex64 batch is checked against it by fidelity.
"""
from __future__ import annotations

import numpy as np

from . import _native as nat
from .linalg import eigh_2x2_many, kron_2x2
from .state import SparseState

MAX_SEG = 256   # resident circuits of a pool (a launch takes bass_batch_max_segments() of them)


def gate_arrays(circuit):
    """A circuit's gate kinds, qubits and 4x4 matrices (1-qubit in the top-left
    2x2), stacked so that a stage gathers them with numpy."""
    n = len(circuit)
    kind = np.zeros(n, np.int8)
    q1 = np.zeros(n, np.int32)
    q2 = np.zeros(n, np.int32)
    mat = np.zeros((n, 4, 4), np.complex128)
    for t, g in enumerate(circuit):
        if g.n_qubits not in (1, 2):
            raise ValueError(f"{g.n_qubits}-qubit gates unsupported")
        kind[t] = g.n_qubits
        q1[t] = g.qubits[0]
        if g.n_qubits == 2:
            q2[t] = g.qubits[1]
        d = 2 ** g.n_qubits
        mat[t, :d, :d] = g.matrix
    return kind, q1, q2, mat


def state_bytes(num_qubits, k, dtype=np.complex64):
    """Device bytes one circuit holds while it runs: three state buffers of
    capacity min(k, 2^n) + 16 (keys and amplitudes) and the workspace sized for
    that capacity (bass_workspace_bytes)."""
    L = nat.load_library()
    cap = min(int(k), 2 ** int(num_qubits)) + 16
    max_n = 4 * cap + 64
    entry = 8 + np.dtype(dtype).itemsize
    return int(3 * cap * entry + L.bass_workspace_bytes(max_n // 4, max_n, int(num_qubits)))


class StatePool:
    """Up to ``max_slots`` BASS simulations that advance one gate per stage."""

    def __init__(self, max_slots=MAX_SEG, dtype=np.complex64, optimize_every=5, pr_opt_threshold=0.90,
                 pr_tie_tol=1e-12, max_nnz_factor=8, buffer_factor=2):
        import torch
        self.torch = torch
        self.L = nat.lib()
        self.dtype = np.dtype(dtype)
        nat.amp_type_of(self.dtype)
        self.optimize_every = optimize_every
        self.pr_opt_threshold = pr_opt_threshold
        self.pr_tie_tol = pr_tie_tol
        self.max_nnz_factor = max_nnz_factor
        self.buffer_factor = buffer_factor
        S = self.max_slots = int(max_slots)
        self.device = torch.device("cuda", torch.cuda.current_device())
        cb = self.L.bass_ctrl_bytes()
        # every slot's control block and RDM moments are contiguous: one read covers them all
        self.ctrl_all = torch.zeros((S, cb), dtype=torch.uint8, device=self.device)
        self.rho_all = torch.zeros((S, 4 * 64), dtype=torch.float64, device=self.device)
        # a segmented selection keeps one block group per state resident: a
        # launch takes at most this many states (one selection block per SM)
        self.seg_chunk = max(1, min(MAX_SEG, int(self.L.bass_batch_max_segments())))
        self.bws_bytes = int(self.L.bass_batch_ws_bytes(self.seg_chunk))
        self.bws = torch.empty(self.bws_bytes, dtype=torch.uint8, device=self.device)
        self.stream = nat.ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        self.states = [None] * S
        self.gates = [None] * S
        self.kron = [dict() for _ in range(S)]
        self.pcur, self.ptmp, self.ptmp2, self.pctrl, self.pws, self.wsb, self.prho = (
            np.zeros(S, np.uint64) for _ in range(7))
        self.nq = np.zeros(S, np.int32)
        self.kk = np.zeros(S, np.int64)
        self.pos = np.zeros(S, np.int64)
        self.length = np.zeros(S, np.int64)
        self.busy = np.zeros(S, bool)
        self.pr_last_opt = np.zeros(S)
        self.Uarr = np.zeros((S, 64, 2, 2), np.complex128)
        self.ident = np.ones((S, 64), bool)
        self.stats = {"stages": 0, "launch_calls": 0, "opt_calls": 0, "rotations": 0, "accepted": 0}
        self.phase0 = 0

    # ---- slots -------------------------------------------------------------------------
    def free_slots(self):
        return int((~self.busy).sum())

    def in_phase(self):
        """Whether a circuit added now reaches its optimisation points (after
        every optimize_every gates of its own) on the same stages as the
        circuits already running: then the rotation steps of all of them go
        to the GPU in the same segmented launches.  True on every
        optimize_every-th stage since the pool last became non-empty, and
        whenever it is empty."""
        if self.optimize_every <= 0 or not self.busy.any():
            self.phase0 = self.stats["stages"]
            return True
        return (self.stats["stages"] - self.phase0) % self.optimize_every == 0

    def live(self):
        """Slots with gates left."""
        return np.nonzero(self.busy & (self.pos < self.length))[0]

    def add(self, circuit, num_qubits, k):
        """Start a circuit in a free slot (returns the slot)."""
        free = np.nonzero(~self.busy)[0]
        if not len(free):
            raise RuntimeError("no free slot")
        c = int(free[0])
        N, k = int(num_qubits), int(k)
        hard_cap = min(self.max_nnz_factor * k, 2 ** N)
        internal_k = min(max(max(self.buffer_factor, 2) * k, hard_cap), 2 ** N)
        cap = min(k, 2 ** N) + 16
        eng = nat.Engine(max_n=4 * cap + 64, num_qubits=N, pr_tie_tol=self.pr_tie_tol,
                         ctrl=self.ctrl_all[c], rho=self.rho_all[c])
        st = SparseState(N, internal_k, 0, dtype=self.dtype, _capacity=cap, _engine=eng)
        self.states[c] = st
        self.gates[c] = gate_arrays(circuit)
        self.kron[c] = {}
        ptr = nat._ptr
        self.pcur[c], self.ptmp[c], self.ptmp2[c] = ptr(st._cur.desc), ptr(st._tmp.desc), ptr(st._tmp2.desc)
        self.pctrl[c], self.pws[c], self.wsb[c], self.prho[c] = ptr(eng.ctrl), ptr(eng.ws), eng.ws_bytes, ptr(eng.rho)
        self.nq[c], self.kk[c] = N, k
        self.pos[c], self.length[c] = 0, len(circuit)
        self.pr_last_opt[c] = 0.0
        self.Uarr[c] = np.eye(2)
        self.ident[c] = True
        self.busy[c] = True
        return c

    def take(self, c):
        """The finished state of slot c, with gamma set as BASS.simulate sets it
        (and the frames in ``U``); the slot becomes free."""
        self._sync_handles([c])
        st = self.states[c]
        ctl = st._eng.read_ctrl()
        st.gamma = np.sqrt(max(float(ctl["gamma_running"]), 0.0))
        st._eng.raise_on_error()
        st.U = [self.Uarr[c, j].copy() for j in range(int(self.nq[c]))]
        st.amp_updates = int(ctl["amp_updates"])
        # the slot's control block and moments are reused: the state keeps copies
        st._eng.ctrl = st._eng.ctrl.clone()
        st._eng.rho = st._eng.rho.clone()
        self.states[c] = None
        self.gates[c] = None
        self.busy[c] = False
        return st

    # ---- plumbing ------------------------------------------------------------------------
    def _ops(self, idx):
        """bass_seg_op rows for the slots idx (an int array)."""
        o = np.zeros(len(idx), dtype=nat.SEG_OP_DTYPE)
        o["in"] = self.pcur[idx]
        o["tmp"] = self.ptmp[idx]
        o["out"] = self.ptmp2[idx]
        o["ctrl"] = self.pctrl[idx]
        o["ws"] = self.pws[idx]
        o["ws_bytes"] = self.wsb[idx]
        o["rho"] = self.prho[idx]
        o["num_qubits"] = self.nq[idx]
        o["k_cond"] = -1
        return o

    @staticmethod
    def _swap(a, b, idx):
        a[idx], b[idx] = b[idx].copy(), a[idx].copy()

    def _call(self, name, o, *extra):
        f = getattr(self.L, name)
        for part in range(0, len(o), self.seg_chunk):
            chunk = np.ascontiguousarray(o[part:part + self.seg_chunk])
            nat.check(f(nat.ctypes.c_void_p(chunk.ctypes.data), len(chunk), *extra,
                        nat.ctypes.c_void_p(nat._ptr(self.bws)), self.bws_bytes, self.stream), name)
        self.stats["launch_calls"] += 1

    def _ctrl(self):
        """Every slot's control block (one synchronising read)."""
        return np.frombuffer(self.ctrl_all.cpu().numpy().tobytes(), dtype=nat.CTRL_DTYPE)

    def _set_ctrl_field(self, idx, name, value):
        off = nat.CTRL_DTYPE.fields[name][1]
        b = np.array([value], dtype=nat.CTRL_DTYPE.fields[name][0]).view(np.uint8)
        t = self.torch.from_numpy(b.copy()).to(self.device)
        ii = self.torch.as_tensor(np.asarray(idx, dtype=np.int64), device=self.device)
        self.ctrl_all[ii, off:off + len(b)] = t

    def _sync_handles(self, idx):
        """Point each state's host handles at the descriptors the arrays say are current."""
        for c in idx:
            st = self.states[c]
            by = {nat._ptr(d.desc): d for d in (st._cur, st._tmp, st._tmp2)}
            st._cur, st._tmp, st._tmp2 = by[int(self.pcur[c])], by[int(self.ptmp[c])], by[int(self.ptmp2[c])]
            st._touch()

    def _kron(self, c, q1, q2):
        """kron(U[q1], U[q2]) of slot c, cached until either frame changes (bass_simulator.py:580-593)."""
        d = self.kron[c]
        key = (q1, q2)
        if key not in d:
            d[key] = kron_2x2(self.Uarr[c, q1], self.Uarr[c, q2])
        return d[key]

    # ---- ops -------------------------------------------------------------------------------
    def _fused(self, o, idx):
        """The simulate-level truncation fused into a gate (k, gamma *= kept/total, renormalise)."""
        o["k_cond"] = self.kk[idx]
        o["k_keep"] = self.kk[idx]
        o["gamma_mode"] = 1
        o["renorm"] = 1
        o["mark_active"] = 1

    def _gate1(self, idx, q, G):
        o = self._ops(idx)
        o["q1"] = q
        o["G"][:, :8] = np.ascontiguousarray(G).view(np.float64).reshape(len(idx), 8)
        self._fused(o, idx)
        self._call("bass_gate_1q_batch", o)
        self._swap(self.pcur, self.ptmp2, idx)   # the op wrote its "out" descriptor

    def _gate2(self, idx, qa, qb, G):
        o = self._ops(idx)
        o["q1"] = qa
        o["q2"] = qb
        o["G"][:, :32] = np.ascontiguousarray(G).view(np.float64).reshape(len(idx), 32)
        self._fused(o, idx)
        self._call("bass_gate_2q_batch", o)
        self._swap(self.pcur, self.ptmp2, idx)

    def _phase2(self, idx, qa, qb, d):
        o = self._ops(idx)
        o["q1"] = qa
        o["q2"] = qb
        o["G"][:, :8] = np.ascontiguousarray(d).view(np.float64).reshape(len(idx), 8)
        self._call("bass_phase_2q_batch", o)

    def _phase1(self, c, G, q):
        """A frame made a 1-qubit gate diagonal: the single-state call (rare)."""
        self._sync_handles([c])
        self.states[c]._apply_1q(G, q, nat.NO_TRUNC)
        self.pcur[c] = nat._ptr(self.states[c]._cur.desc)
        self.ptmp[c] = nat._ptr(self.states[c]._tmp.desc)
        self.ptmp2[c] = nat._ptr(self.states[c]._tmp2.desc)
        self.stats["launch_calls"] += 1

    # ---- one stage -----------------------------------------------------------------------
    def step(self):
        """Every live slot applies its next gate (BASS.simulate's loop body for
        gate pos, bass_simulator.py:860-926); returns the slots that finished."""
        live = self.live()
        if not len(live):
            return live
        self.stats["stages"] += 1
        pos = self.pos[live]
        kind = np.array([self.gates[c][0][p] for c, p in zip(live, pos)])
        q1 = np.array([self.gates[c][1][p] for c, p in zip(live, pos)])
        q2 = np.array([self.gates[c][2][p] for c, p in zip(live, pos)])
        mat = np.stack([self.gates[c][3][p] for c, p in zip(live, pos)])
        one, two = kind == 1, kind == 2
        if one.any():
            c1, qa = live[one], q1[one]
            G = mat[one][:, :2, :2]
            for r in np.nonzero(~self.ident[c1, qa])[0]:   # rotated frames: as BASS.simulate computes them
                U = self.Uarr[c1[r], qa[r]]
                G[r] = U.conj().T @ G[r] @ U
            diag = (G[:, 0, 1] == 0) & (G[:, 1, 0] == 0)
            if (~diag).any():
                self._gate1(c1[~diag], qa[~diag], G[~diag])
            for c, g, q in zip(c1[diag], G[diag], qa[diag]):
                self._phase1(int(c), g, int(q))
        if two.any():
            c2, qa, qb = live[two], q1[two], q2[two]
            G = mat[two]
            for r in np.nonzero(~(self.ident[c2, qa] & self.ident[c2, qb]))[0]:
                Ut = self._kron(int(c2[r]), int(qa[r]), int(qb[r]))
                G[r] = Ut.conj().T @ G[r] @ Ut
            off = np.abs(G - np.einsum("nii->ni", G)[:, :, None] * np.eye(4)).max(axis=(1, 2))
            diag = off < 1e-12
            if diag.any():
                self._phase2(c2[diag], qa[diag], qb[diag], np.einsum("nii->ni", G[diag]))
            if (~diag).any():
                self._gate2(c2[~diag], qa[~diag], qb[~diag], G[~diag])
        self.pos[live] += 1
        if self.optimize_every > 0:
            p1 = self.pos[live]   # i + 1 of BASS.simulate
            chk = live[(p1 % self.optimize_every == 0) & (p1 < self.length[live])]
            if len(chk):
                self._maybe_optimize(chk)
        return live[self.pos[live] >= self.length[live]]

    # ---- optimisation points (bass_simulator.py:730-845) ------------------------------
    def _pr(self, idx):
        """PR of the states idx (one segmented launch, one read)."""
        self._call("bass_pr_batch", self._ops(idx), 1)
        return self._ctrl()["pr_last"][idx].astype(np.float64)

    def _maybe_optimize(self, chk):
        c = self._ctrl()
        act = chk[c["truncation_active"][chk] != 0]
        if len(act):
            pr = self._pr(act)
            if self.pr_opt_threshold >= 1.0:
                trig = np.ones(len(act), bool)
            else:
                trig = pr > self.pr_last_opt[act] / self.pr_opt_threshold
            T, prT = act[trig], pr[trig]
            if len(T):
                opt = T[prT >= self.kk[T] / 4]
                if len(opt):
                    self._optimize(opt)
                    self.pr_last_opt[T] = self._pr(T)
                else:
                    self.pr_last_opt[T] = prT
        self._set_ctrl_field(chk, "truncation_active", 0)

    def _optimize(self, T):
        st = self.stats
        st["opt_calls"] += len(T)
        active = T
        for _pass in range(3):
            o = self._ops(active)
            self._call("bass_rdm_1q_batch", o)
            self._call("bass_pr_batch", o, 1)          # pr_cur of each state's pass
            rho = self.rho_all[self.torch.as_tensor(active, device=self.device)].cpu().numpy()
            nq = self.nq[active]
            Vall = eigh_2x2_many(np.concatenate([rho[r, :4 * n].reshape(n, 4) for r, n in enumerate(nq)]))
            starts = np.concatenate([[0], np.cumsum(nq)])
            tried = np.zeros((len(active), 64), bool)
            Vs = np.zeros((len(active), 64, 2, 2), np.complex128)
            for r, n in enumerate(nq):
                V = Vall[starts[r]:starts[r + 1]]
                Vs[r, :n] = V
                tried[r, :n] = (np.abs(V[:, 0, 1]) + np.abs(V[:, 1, 0])) >= 1e-10
            for jq in range(int(nq.max())):
                rr = np.nonzero(tried[:, jq])[0]
                if not len(rr):
                    continue
                idx = active[rr]
                oj = self._ops(idx)
                oj["q1"] = jq
                Uh = np.ascontiguousarray(np.conj(np.swapaxes(Vs[rr, jq], 1, 2)))
                oj["G"][:, :8] = Uh.view(np.float64).reshape(len(rr), 8)
                oj["k_keep"] = self.kk[idx]
                oj["k_cond"] = self.kk[idx]
                self._call("bass_rotate_step_batch", oj)
            c = self._ctrl()
            improved = np.zeros(len(active), bool)
            for r, cc in enumerate(active):
                js = np.nonzero(tried[r])[0]
                st["rotations"] += len(js)
                acc = js[c["accept"][cc][js] != 0]
                for jq in acc:
                    self.Uarr[cc, jq] = self.Uarr[cc, jq] @ Vs[r, jq]
                    self.ident[cc, jq] = False
                    for key in [kk for kk in self.kron[cc] if jq in kk]:
                        del self.kron[cc][key]
                st["accepted"] += len(acc)
                improved[r] = len(acc) > 0
            active = active[improved]
            if not len(active):
                break
        o = self._ops(T)
        o["k_cond"] = self.kk[T]
        o["k_keep"] = self.kk[T]
        self._call("bass_topk_batch", o)                 # _truncate_state
        self._swap(self.pcur, self.ptmp2, T)
        self._call("bass_pr_batch", self._ops(T), 0)    # _renorm


class BatchedBASS:
    """BASS on many circuits at once.  ``specs``: (num_qubits, k) per circuit."""

    def __init__(self, specs, dtype=np.complex64, **kw):
        self.specs = [(int(n), int(k)) for n, k in specs]
        self.dtype = np.dtype(dtype)
        self.kw = kw
        self.stats = {}

    def simulate(self, circuits):
        """Run circuits[i] on specs[i]; returns the final states in order."""
        if len(circuits) != len(self.specs):
            raise ValueError("one circuit per spec")
        out = [None] * len(circuits)
        pool = StatePool(max_slots=max(1, min(MAX_SEG, len(circuits))), dtype=self.dtype, **self.kw)
        todo = list(range(len(circuits)))[::-1]
        slot_of = {}
        while todo or len(pool.live()) or pool.busy.any():
            while todo and pool.free_slots() and pool.in_phase():
                i = todo.pop()
                slot_of[pool.add(circuits[i], *self.specs[i])] = i
            for c in np.nonzero(pool.busy & (pool.pos >= pool.length))[0]:
                out[slot_of.pop(int(c))] = pool.take(int(c))
            pool.step()
        self.stats = dict(pool.stats)
        self.stats["amp_updates"] = int(sum(s.amp_updates for s in out))
        return out
