"""The reference-style C++ driver (tests/drivers/tgv_driver.cu, built against
include/lbm3/) runs on the GPU and gives the same kinetic-energy history as
the same case built through the Python mirror of the C ABI."""
import subprocess

import pytest

import lbm3_b200 as L
from test_hooks import build_driver

pytestmark = pytest.mark.gpu


def test_cpp_driver_matches_the_python_api(tmp_path):
    exe = build_driver(tmp_path)
    out = subprocess.run([str(exe), "20"], check=True, capture_output=True, text=True).stdout.split("\n")
    assert out[0].startswith("fluid_updates")
    e0 = float(out[1].split()[1])
    steps, e20 = out[2].split()
    assert int(steps) == 20
    s = L.taylor_green(32)
    with L.build_grids(s.case) as g:
        assert g.kinetic_energy(s.u_initial_phys, s.domain_length) == pytest.approx(e0, rel=1e-12)
        g.update_all_grids(20)
        assert g.kinetic_energy(s.u_initial_phys, s.domain_length) == pytest.approx(float(e20), rel=1e-9)


def test_cpp_driver_with_a_refined_level(tmp_path):
    """The same driver with GRID_LEVEL_COUNT = 2 and the reference's
    getRefinementModifier (central cube): the C++ hook path builds the same
    two-level grid and history as the refinement box of the Python mirror."""
    exe = build_driver(tmp_path, levels=2)
    out = subprocess.run([str(exe), "10"], check=True, capture_output=True, text=True).stdout.split("\n")
    e0 = float(out[1].split()[1])
    steps, e10 = out[2].split()
    assert int(steps) == 10
    s = L.taylor_green_refined(32)
    with L.build_grids(s.case) as g:
        assert g.level_count() == 2
        assert g.kinetic_energy(s.u_initial_phys, s.domain_length) == pytest.approx(e0, rel=1e-12)
        g.update_all_grids(10)
        assert g.kinetic_energy(s.u_initial_phys, s.domain_length) == pytest.approx(float(e10), rel=1e-9)
