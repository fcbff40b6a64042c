"""GPU interpolated bounceback against the oracle, and the analytic channel."""
import numpy as np
import pytest

import lbm3_b200 as L
from lbm3_b200 import _abi as A
from lbm3_b200 import geometry as G
import oracle as O
from helpers import FIELD_REL_L2, field_errors, plan_ijk, rel_l2
from test_walls import channel_case

pytestmark = pytest.mark.gpu


def sphere_case(storage=A.LBM_STORE_F32):
    c = L.periodic_box(32, 24, 24, nu_lattice=0.02, ux=0.02, storage=storage)
    G.set_bodies(c, [G.icosphere(3, 6.0, (0.3, 0.2, 0.1))])
    c.track_wall_force = 1
    return c


@pytest.mark.parametrize("steps", [1, 30])
def test_sphere_ibb_matches_oracle(steps):
    c = sphere_case()
    p = L.Plan(c)
    o = O.OracleGrid(c)
    with L.build_grids(c) as g:
        info = g.info()
        assert info.wall_adjacent_count == p.info().wall_adjacent_count > 0
        g.update_all_grids(steps)
        o.step(steps)
        wm = p.array("wall_map")
        fl = wm != -3
        gm, om = g.macro(), o.macro()
        e_rho, e_u = field_errors(gm[:, fl], om[:, fl])
        assert e_rho < FIELD_REL_L2 and e_u < FIELD_REL_L2, (e_rho, e_u)
        # momentum-exchange force accumulated per wall-adjacent cell
        fg = g.wall_force_raw()
        fo = np.ctypeslib.as_array(o.g.wallForce, shape=(3 * info.wall_adjacent_count,)).reshape(3, -1)
        assert rel_l2(fg, fo) < 1e-4
        # FP64 reduction of the total force (lattice units) matches the oracle's
        ro = o.wall_force(0)
        rg = g.wall_force(0)
        res = info.res / 1000.0
        conv = c.rho_phys * res ** 4 / (info.dt_phys ** 2)
        assert np.allclose(rg[:3], ro[:3] / steps * conv, rtol=1e-4, atol=1e-12)
    o.close()


def test_channel_profile_on_gpu():
    nu, gx, h = 0.1, 1e-6, 10.2
    c = channel_case(nu=nu, gx=gx)
    p = L.Plan(c)
    with L.build_grids(c) as g:
        g.update_all_grids(3000)
        m = g.macro()
    _, _, kz = plan_ijk(p)
    info = p.info()
    z = info.oz + kz * info.res
    fluid = p.array("wall_map") != -3
    ua = gx * (h * h - z[fluid] ** 2) / (2 * nu)
    err = np.max(np.abs(m[1][fluid] - ua)) / ua.max()
    assert err < 0.01, err


def test_channel_wall_force_balances_body_force():
    """At steady state the walls take the whole body force: sum of the wall
    forces on the fluid = -g * (number of fluid cells)."""
    nu, gx = 0.1, 1e-6
    c = channel_case(nu=nu, gx=gx)
    with L.build_grids(c) as g:
        g.update_all_grids(4000)
        g.wall_force(0, reset=True)
        g.update_all_grids(100)
        f0 = g.wall_force(0)
        f1 = g.wall_force(1)
        info = g.info()
    res = info.res / 1000.0
    conv = c.rho_phys * res ** 4 / (info.dt_phys ** 2)
    fluid_cells = info.cell_count - info.wall_cell_count
    total = (f0[0] + f1[0]) / conv
    # periodic ghost cells are not tracked: compare with the active cells
    active = (info.cell_count_x - 2) * (info.cell_count_y - 2) * (fluid_cells // (info.cell_count_x * info.cell_count_y))
    assert abs(total + gx * active) / (gx * active) < 0.02, (total, -gx * active)
