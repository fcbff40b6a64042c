"""Taylor-Couette torque on the GPU in SI units against the analytic value
(cases/torqueTest/torqueTestMain.cu:45-54)."""
import numpy as np
import pytest

import lbm3_b200 as L
from lbm3_b200 import _abi as A
from test_walls import couette_case, couette_torque_lattice

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("storage", [A.LBM_STORE_F32, A.LBM_STORE_F16])
def test_couette_torque_matches_theory(storage):
    c = couette_case(storage=storage)
    with L.build_grids(c) as g:
        g.update_all_grids(3000)
        g.wall_force(0, reset=True)
        g.update_all_grids(500)
        t_in = g.wall_force(0)[5]
        t_out = g.wall_force(1, reset=True)[5]
        info = g.info()
    # analytic torque in SI: lattice torque x rho (res/1000)^4 / dt^2 x 1e-3 (N mm -> N m)
    res_m = info.res / 1000.0
    t = couette_torque_lattice() * c.rho_phys * res_m ** 4 / info.dt_phys ** 2 * 1e-3
    tol = 0.01 if storage == A.LBM_STORE_F32 else 0.03
    assert t_in == pytest.approx(t, rel=tol)
    assert t_out == pytest.approx(-t, rel=tol)
