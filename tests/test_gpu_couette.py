"""Taylor-Couette torque on the GPU in SI units against the analytic value
(cases/torqueTest/torqueTestMain.cu:45-54), and the storage-precision study
on it: FP16 and BF16 shifted populations against FP32."""
import pytest

import lbm3_b200 as L
from lbm3_b200 import _abi as A
from test_walls import couette_case, couette_torque_lattice

pytestmark = pytest.mark.gpu


def steady_torques(storage):
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
    return t_in, t_out, t


def test_couette_torque_matches_theory_in_every_storage():
    t32_in, t32_out, t = steady_torques(A.LBM_STORE_F32)
    assert t32_in == pytest.approx(t, rel=0.01)
    assert t32_out == pytest.approx(-t, rel=0.01)
    # shifted 16-bit storage: FP16 keeps the torque within 1e-3 of FP32;
    # BF16, with its 8-bit mantissa, within 3e-3
    for st, tol in ((A.LBM_STORE_F16, 1e-3), (A.LBM_STORE_BF16, 3e-3)):
        t_in, t_out, _ = steady_torques(st)
        assert t_in == pytest.approx(t32_in, rel=tol), st
        assert t_out == pytest.approx(t32_out, rel=tol), st
