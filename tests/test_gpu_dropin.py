"""The reference-style C++ driver with the dg::b200 classes swapped in.

oracle/dropin_test.cpp builds the reference's Mesh2D, QuadratureRule, operators,
ode::RungeKutta4 and WaveHoltz, and the drop-ins of include/wdg_b200.hpp with the
same arguments, and exits non-zero if any answer differs beyond its tolerance
(1e-12 per operator, 1e-11 after ten RK4 steps).  The binary is built by
`make -C oracle ref` where the reference sources are present.
"""
import os
import subprocess

import pytest

from conftest import require_reference_build

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "..", "oracle", "_ref", "dropin_test")


@pytest.mark.gpu
def test_reference_driver_with_dropins():
    require_reference_build(BIN)
    out = subprocess.run([BIN], capture_output=True, text=True, timeout=300)
    print(out.stdout)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "drop-in ok" in out.stdout
