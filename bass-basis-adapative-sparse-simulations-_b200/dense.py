"""Dense FP64 statevector simulation on the GPU -- drop-in for
src/simulation/exact_simulator.py:66-144 (``ExactSimulator``).

The reference uses its dense simulator as the exact answer that sparse states
are scored against (``runner.py:615-617``, ``fidelity.py:48-65``).  This one
keeps the 2^N complex128 amplitudes on the device and applies every gate in
place with ``bass_dense_gate`` (one thread per pair or group of four
amplitudes).  ``simulate`` returns a host numpy array like the reference's;
``simulate_device`` returns the device tensor, which ``metrics`` reads on
the device.  N <= 24 as in the reference (``exact_simulator.py:72``), or up to
34 through ``max_qubits``.
"""
from __future__ import annotations

import numpy as np

from . import _native as nat


class ExactSimulator:
    def __init__(self, num_qubits, verbose=True, *, max_qubits=24, device=None):
        if num_qubits > max_qubits:
            raise ValueError(f"N={num_qubits} too large for exact simulation")
        self.N = int(num_qubits)
        self.verbose = verbose
        self._device = device

    def simulate_device(self, circuit, initial_state=None):
        import torch
        L = nat.lib()
        dev = torch.device("cuda", torch.cuda.current_device() if self._device is None else self._device)
        psi = torch.zeros(2 ** self.N, dtype=torch.complex128, device=dev)
        psi[0 if initial_state is None else int(initial_state)] = 1.0
        stream = nat.ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
        ptr = nat.ctypes.c_void_p(psi.data_ptr())
        for gate in circuit:
            n = gate.n_qubits
            if n not in (1, 2):
                raise NotImplementedError()
            g = nat.host_c128(gate.matrix)
            q1 = int(gate.qubits[0])
            q2 = int(gate.qubits[1]) if n == 2 else 0
            nat.check(L.bass_dense_gate(ptr, self.N, nat._host(g), n, q1, q2, stream), "bass_dense_gate")
        return psi

    def simulate(self, circuit, initial_state=None):
        return self.simulate_device(circuit, initial_state).cpu().numpy()

    def apply_gate_exact(self, state, gate):
        """One gate on a host statevector (returns a new host array)."""
        import torch
        psi = torch.as_tensor(np.asarray(state, dtype=np.complex128)).cuda(self._device)
        L = nat.lib()
        stream = nat.ctypes.c_void_p(torch.cuda.current_stream(psi.device).cuda_stream)
        g = nat.host_c128(gate.matrix)
        q1 = int(gate.qubits[0])
        q2 = int(gate.qubits[1]) if gate.n_qubits == 2 else 0
        nat.check(L.bass_dense_gate(nat.ctypes.c_void_p(psi.data_ptr()), self.N, nat._host(g), gate.n_qubits,
                                    q1, q2, stream), "bass_dense_gate")
        return psi.cpu().numpy()
