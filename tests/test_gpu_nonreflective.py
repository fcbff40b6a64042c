"""The reference's non-reflective boundary study on the GPU: a 20 mm pipe at
Re 1000 started from rest, with a plain (Dirichlet) velocity inlet, the
characteristic non-reflective inlet and the impedance inlet at three density
tolerances.  The area-averaged inlet velocity and pressure after every step
are compared with the histories the reference stored for the same case
(tests/golden/nonreflective_*.txt, made by make_nonreflective_golden.py):
the deviation, scaled by the largest magnitude of the stored series, must
stay under the bound of each run over the first 5,000 steps.  The bounds grow
with the impedance scheme's sensitivity: at a tolerance of 2e-7 the inlet
velocity creeps up by the clamp's width each step, so rounding differences
of the streamed state move it most."""
from pathlib import Path

import numpy as np
import pytest

import lbm3_b200 as L
from lbm3_b200 import cases as CS

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"

RUNS = [  # fixture, scheme, tolerance, bound on |ours - stored| / max|stored| (velocity, pressure)
    ("dirichlet", "dirichlet", 0.0, (1e-6, 1e-4)),
    ("characteristic", "characteristic", 0.0, (1e-5, 1e-4)),
    ("impedance2e-5", "impedance", 2e-5, (1e-4, 2e-4)),
    ("impedance2e-6", "impedance", 2e-6, (5e-4, 2e-3)),
    ("impedance2e-7", "impedance", 2e-7, (1e-2, 1e-2)),
]


@pytest.mark.parametrize("name,scheme,tol,bounds", RUNS)
def test_inlet_history_matches_the_reference(name, scheme, tol, bounds):
    pin = np.loadtxt(GOLDEN / f"nonreflective_{name}.txt", delimiter=";", comments="#")
    steps = int(pin[-1, 0])
    s = CS.non_reflective_pipe(scheme, tol)
    ours = np.empty((steps, 2))
    with L.build_grids(s.case) as g:
        for it in range(steps):
            g.update_all_grids(1)
            fl = g.open_boundary_flow(0, reset=True)   # tracker period 1
            ours[it] = fl["normal_velocity"], fl["pressure"]
    rows = pin[:, 0].astype(int) - 1
    for col, bound in zip((0, 1), bounds):
        got, ref = ours[rows, col], pin[:, col + 1]
        dev = np.abs(got - ref).max() / np.abs(ref).max()
        assert dev < bound, (name, col, dev)
    # the first step to FP32 rounding
    assert ours[0, 0] == pytest.approx(pin[0, 1], rel=1e-6)
