"""GPU forcing rotors against the oracle."""
import numpy as np
import pytest

import lbm3_b200 as L
from lbm3_b200 import _abi as A
from lbm3_b200 import geometry as G
import oracle as O
from helpers import FIELD_REL_L2, density_velocity_errors, rel_l2

pytestmark = pytest.mark.gpu


def rotor_case(storage=A.LBM_STORE_F32, omega=2.0, bodies=False):
    c = L.periodic_box(40, 40, 30, nu_lattice=0.02, storage=storage)
    tris = G.rotor(hub_radius=3, tip_radius=12, chord=5, thickness=1.5, hub_length=6)
    G.set_rotors(c, [(tris, dict(axis=2, origin=(0.0, 0.0, 0.0), radians_per_second=omega))])
    c.track_rotor_force = 1
    if bodies:
        G.set_bodies(c, [G.box((-18.0, -18.0, 9.0), (18.0, 18.0, 12.0))])
        c.track_wall_force = 1
        c.collision_limiter = 0.0
    return c


@pytest.mark.parametrize("steps", [1, 30])
@pytest.mark.parametrize("bodies", [False, True])
def test_rotor_matches_oracle(steps, bodies):
    c = rotor_case(bodies=bodies)
    p = L.Plan(c)
    o = O.OracleGrid(c)
    with L.build_grids(c) as g:
        g.update_all_grids(steps)
        o.step(steps)
        fl = p.array("wall_map") != -3
        e_rho, e_u, d_rho = density_velocity_errors(g.macro()[:, fl], o.macro()[:, fl])
        assert e_rho < FIELD_REL_L2 and e_u < FIELD_REL_L2 and d_rho < 1e-6, (e_rho, e_u, d_rho)
        # force bins: totals per component agree; individual bins may differ
        # by a cell whose position rounds across a bin edge
        bg, bo = g.rotor_bins(0), o.rotor_bins(0)
        assert np.allclose(bg.sum(axis=1), bo.sum(axis=1), rtol=1e-4, atol=1e-6)
        assert rel_l2(bg, bo) < 1e-3
        ri = g.rotor_info(0)
        assert ri.radians_elapsed == pytest.approx((steps * g.info().dt_phys * 2.0) % (2 * np.pi), rel=1e-9)
    o.close()


def test_rotor_force_and_speed_control():
    c = rotor_case()
    with L.build_grids(c) as g:
        g.update_all_grids(20)
        f = g.rotor_force(0, reset=True)
        # the rotor drives the fluid about +z: its torque on the fluid is positive
        assert f[5] > 0
        g.set_rotor_speed(0, 0.0)
        a0 = g.rotor_info(0).radians_elapsed
        g.update_all_grids(5)
        assert g.rotor_info(0).radians_elapsed == a0
        # a stopped rotor brakes the spinning fluid: negative torque
        assert g.rotor_force(0)[5] < 0


def test_rotor_low_precision_storage():
    a_case, b_case = rotor_case(), rotor_case(storage=A.LBM_STORE_F16)
    with L.build_grids(a_case) as a, L.build_grids(b_case) as b:
        a.update_all_grids(50)
        b.update_all_grids(50)
        ma, mb = a.macro(), b.macro()
    assert rel_l2(mb[1:4].reshape(-1), ma[1:4].reshape(-1)) < 5e-3
