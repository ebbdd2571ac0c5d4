"""bass_b200 -- B200-native sparse-state simulation hot path of BASS.

Drop-in for the reference's ``BASS``, ``SparseState`` and
``FixedBasisSimulator`` (src/simulation/bass_simulator.py,
src/core/sparse_state.py, src/simulation/simulator.py).  Host code is Python;
device buffers are torch CUDA tensors; every per-entry operation runs in the
hand-written sm_100a kernels of ``libbass_b200.so`` (``csrc/``), reached
through the C ABI declared in ``include/bass_b200.h``.  There is no CPU
fallback: constructing a simulator without the CUDA library or without a GPU
raises.

The directory name is not a Python identifier, so the package is imported
under the name ``bass_b200`` by a file-location import of this directory's
``__init__.py`` (as ``load_pkg()`` in bench.py and tests/conftest.py do).
"""
from . import gates, circuits  # noqa: F401
from .gates import (  # noqa: F401
    QuantumGate, SingleQubitGate, TwoQubitGate, HGate, XGate, YGate, ZGate, SGate, TGate,
    CNOTGate, CZGate, RXGate, RZZGate, RZGate, RYGate, RandomTwoQubitGate, haar_random_unitary,
)


def __getattr__(name):
    # The GPU classes load libbass_b200.so on first use.
    if name in ("SparseState",):
        from .state import SparseState
        return SparseState
    if name in ("BASS",):
        from .bass import BASS
        return BASS
    if name in ("FixedBasisSimulator",):
        from .fixed import FixedBasisSimulator
        return FixedBasisSimulator
    raise AttributeError(name)
