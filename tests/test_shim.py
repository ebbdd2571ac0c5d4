"""The module-alias shim: the reference's own experiment runner, imported
after shim.install(), builds this package's classes (runner.py:90-108)."""
import importlib.util
import os
import sys

import pytest

from conftest import ROOT

REF = os.environ.get("BASS_REFERENCE", "")


def _make_golden():
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(ROOT, "tests", "golden",
                                                                             "make_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


@pytest.mark.skipif(not REF or not os.path.isdir(REF), reason="set BASS_REFERENCE to a reference checkout")
@pytest.mark.filterwarnings("ignore::SyntaxWarning")   # a docstring escape in the reference's runner
def test_reference_runner_uses_gpu_classes(pkg):
    mg = _make_golden()
    before = {k: v for k, v in sys.modules.items() if k == "src" or k.startswith("src.")}
    try:
        mg.import_reference(REF)            # the reference's packages, importable by path
        from bass_b200 import bass, fixed, gates, shim, state
        shim.install()
        sys.modules.pop("src.experimentation.runner", None)
        runner = importlib.import_module("src.experimentation.runner")
        assert runner.BASS is bass.BASS
        assert runner.FixedBasisSimulator is fixed.FixedBasisSimulator
        assert runner.HGate is gates.HGate and runner.RandomTwoQubitGate is gates.RandomTwoQubitGate
        assert sys.modules["src.core.sparse_state"].SparseState is state.SparseState
        import numpy as np
        circ = runner.make_brickwork(6, 3, np.random.default_rng(0))
        assert circ and all(isinstance(g, gates.QuantumGate) for g in circ)
        shim.uninstall()
        assert sys.modules.get("src.simulation.bass_simulator") is not bass
    finally:
        for k in [k for k in sys.modules if k == "src" or k.startswith("src.")]:
            if k not in before:
                del sys.modules[k]
        sys.modules.update(before)
