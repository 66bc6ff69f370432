"""The engine as a drop-in: oracle/_ref/adapter_driver runs it through the
reference's own Algorithm / TimedAlgorithm interface (the C++ adapter in
stencil-optimalizations_b200/host/gol_b200_algorithm.hpp), two rounds on one
instance as ExperimentManager does, and validates the grid with the
reference's own GoLCpuNaive<char> and Grid::equals."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "adapter_driver")


@pytest.mark.skipif(not os.path.exists(DRIVER), reason="adapter driver not built (needs reference sources)")
@pytest.mark.parametrize("args", [["256", "128", "100", "42"],
                                  ["512", "320", "77", "7", "4"],
                                  ["1024", "96", "64", "3", "8", "local"],
                                  ["128", "64", "0", "5"],
                                  ["512", "200", "33", "9", "1", "k1"],
                                  ["2048", "64", "20", "4", "6", "k1"],
                                  ["1024", "500", "100", "11", "6", "resident"]])
def test_engine_behind_reference_algorithm_interface(args):
    r = subprocess.run([DRIVER, *args], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "valid (equals GoLCpuNaive)" in r.stdout
    if "k1" in args:
        assert "engine depth: 1 generation per pass" in r.stdout
