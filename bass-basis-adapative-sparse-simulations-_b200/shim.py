"""Run code written against the reference on this package, unchanged.

The reference's modules are imported by dotted path
(``src.simulation.bass_simulator`` and so on, see its
``src/experimentation/runner.py:90-108``).  ``install()`` registers this
package's modules under those names, so the reference's experiment runner and
notebooks construct the GPU classes (``BASS``, ``SparseState``,
``FixedBasisSimulator`` and the gate classes) without edits.  Its other
modules (the dense ``ExactSimulator``, the fidelity metrics, the random-circuit
generators) stay its own and work on these classes as they are: the states
expose ``x``, ``alpha``, ``nnz``, ``gamma``, ``N`` and ``sample`` like the
reference's.

    from bass_b200 import shim
    shim.install()
    from src.experimentation.runner import run_trial_timed   # reference code, GPU classes
"""
from __future__ import annotations

import importlib
import sys

# reference module path -> this package's module
ALIASES = {
    "src.simulation.bass_simulator": "bass",    # BASS (bass_simulator.py:478-929)
    "src.core.sparse_state": "state",           # SparseState (sparse_state.py:193-400)
    "src.simulation.simulator": "fixed",        # FixedBasisSimulator (simulator.py:61-253)
    "src.core.gates": "gates",                  # gate classes (gates.py)
}

_saved: dict = {}


def install() -> dict:
    """Point the reference's module names at this package; returns the map."""
    pkg = __name__.rsplit(".", 1)[0]
    done = {}
    for ref_name, ours in ALIASES.items():
        mod = importlib.import_module(f"{pkg}.{ours}")
        if ref_name not in _saved:
            _saved[ref_name] = sys.modules.get(ref_name)
        sys.modules[ref_name] = mod
        done[ref_name] = mod
    return done


def uninstall() -> None:
    """Restore whatever those names pointed at before install()."""
    for ref_name, prev in list(_saved.items()):
        if prev is None:
            sys.modules.pop(ref_name, None)
        else:
            sys.modules[ref_name] = prev
        del _saved[ref_name]
