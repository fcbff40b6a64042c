"""GPU open boundaries (velocity inlet, non-reflective pressure outlet,
velocity or periodic sides, with and without a body) against the oracle."""
import numpy as np
import pytest

import lbm3_b200 as L
from lbm3_b200 import _abi as A
from lbm3_b200 import geometry as G
import oracle as O
from helpers import FIELD_REL_L2, density_velocity_errors, rel_l2

pytestmark = pytest.mark.gpu


def _perturbed(c, seed=7):
    """Plan, oracle and GPU grids of a case whose state is the equilibrium
    plus seeded noise, so every branch of the boundary closure sees non-trivial
    input."""
    p = L.Plan(c)
    o = O.OracleGrid(c)
    g = L.build_grids(c)
    f = o.populations()
    rng = np.random.default_rng(seed)
    f = (f + 2e-4 * rng.standard_normal(f.shape) * np.abs(f).max()).astype(np.float32)
    o.set_populations(f)
    g.set_populations(f)
    return p, o, g


@pytest.mark.parametrize("sides", ["velocity", "periodic"])
@pytest.mark.parametrize("steps", [1, 40])
def test_open_channel_matches_oracle(sides, steps):
    """Fields to the FP32 bar (density as rho = 1 + dRho: the noise keeps dRho
    near 1e-5, where its own relative error measures contraction rounding
    only), reference values and tracked sums of every open cell."""
    c = L.open_channel(32, 16, 12, u_in=0.04, nu_lattice=0.02, sides=sides)
    p, o, g = _perturbed(c)
    with g:
        g.update_all_grids(steps)
        o.step(steps)
        e_rho, e_u, d_rho = density_velocity_errors(g.macro(), o.macro())
        assert e_rho < FIELD_REL_L2 and e_u < FIELD_REL_L2 and d_rho < 1e-6, (e_rho, e_u, d_rho)
        np.testing.assert_array_equal(g.array("open_index"), o.open_index())
        ref_g, ref_o = g.open_reference(), o.open_reference()
        assert rel_l2(ref_g[1], ref_o[1]) < FIELD_REL_L2
        assert np.abs(ref_g[0] - ref_o[0]).max() < 1e-6
        cum_g, cum_o = g.open_cumulative(), o.open_cumulative()
        assert rel_l2(cum_g[1], cum_o[1]) < FIELD_REL_L2
        assert np.abs(cum_g[0] - cum_o[0]).max() < 1e-6 * steps
    o.close()


def test_sphere_in_open_channel_matches_oracle():
    c = L.open_channel(48, 24, 24, u_in=0.04, nu_lattice=0.02)
    G.set_bodies(c, [G.icosphere(3, 4.0, (16.0, 12.0, 12.0))])
    c.track_wall_force = 1
    p = L.Plan(c)
    o = O.OracleGrid(c)
    steps = 60
    with L.build_grids(c) as g:
        g.update_all_grids(steps)
        o.step(steps)
        fl = p.array("wall_map") != -3
        e_rho, e_u, d_rho = density_velocity_errors(g.macro()[:, fl], o.macro()[:, fl])
        assert e_rho < FIELD_REL_L2 and e_u < FIELD_REL_L2 and d_rho < 1e-6, (e_rho, e_u, d_rho)
        info = g.info()
        fo = np.ctypeslib.as_array(o.g.wallForce, shape=(3 * info.wall_adjacent_count,)).reshape(3, -1)
        assert rel_l2(g.wall_force_raw(), fo) < 1e-4
        # the tracked momentum exchange is the force on the fluid: the stream
        # is decelerated, drag = -Fx (cases/flowAroundSphere/flowAroundSphereMain.cu:212)
        assert g.wall_force(0)[0] < 0
    o.close()


def test_uniform_flow_rates():
    """Uniform stream: the inlet carries rho u A in, the outlet the same out."""
    u = 0.04
    c = L.open_channel(24, 12, 12, u_in=u, nu_lattice=0.02)
    with L.build_grids(c) as g:
        g.update_all_grids(50)
        inlet = g.open_boundary_flow(0)
        outlet = g.open_boundary_flow(1, reset=True)
        # inlet face without edges: 10 x 10 cells of 1 mm^2; u_in is 1 m/s
        assert inlet["area"] == pytest.approx(100e-6)
        assert inlet["normal_velocity"] == pytest.approx(-1.0, rel=1e-4)
        assert outlet["normal_velocity"] == pytest.approx(1.0, rel=1e-4)
        assert outlet["mass_flow"] == pytest.approx(1.0 * 100e-6, rel=1e-4)
        assert abs(outlet["pressure"]) < 1e-3
        # the reset zeroed the sums
        assert np.abs(g.open_cumulative()).max() == 0.0


@pytest.mark.parametrize("storage", [A.LBM_STORE_F16, A.LBM_STORE_BF16])
def test_open_channel_low_precision_storage(storage):
    c32 = L.open_channel(32, 16, 12, u_in=0.04, nu_lattice=0.02)
    c16 = L.open_channel(32, 16, 12, u_in=0.04, nu_lattice=0.02, storage=storage)
    G.set_bodies(c32, [G.icosphere(2, 3.0, (12.0, 8.0, 6.0))])
    G.set_bodies(c16, [G.icosphere(2, 3.0, (12.0, 8.0, 6.0))])
    with L.build_grids(c32) as a, L.build_grids(c16) as b:
        a.update_all_grids(100)
        b.update_all_grids(100)
        ma, mb = a.macro(), b.macro()
    tol = 2e-3 if storage == A.LBM_STORE_F16 else 2e-2
    assert rel_l2(mb[1:4].reshape(-1), ma[1:4].reshape(-1)) < tol


@pytest.mark.parametrize("tolerance", [2e-5, 2e-3])
@pytest.mark.parametrize("steps", [1, 30])
def test_impedance_scheme_matches_oracle(tolerance, steps):
    """The impedance open-boundary scheme (non-reflective velocity inlet and
    pressure outlet clamped to within the density tolerance of the
    non-reflecting state): fields, and the reference arrays, which under this
    scheme hold the previous completed boundary state."""
    c = L.open_channel(32, 16, 12, u_in=0.04, nu_lattice=0.02, inlet_non_reflective=True)
    c.open_bc_scheme = A.LBM_OPEN_IMPEDANCE
    c.rho_reflection_tolerance = tolerance
    p, o, g = _perturbed(c, seed=11)
    with g:
        g.update_all_grids(steps)
        o.step(steps)
        e_rho, e_u, d_rho = density_velocity_errors(g.macro(), o.macro())
        assert e_rho < FIELD_REL_L2 and e_u < FIELD_REL_L2 and d_rho < 1e-6, (e_rho, e_u, d_rho)
        ref_g, ref_o = g.open_reference(), o.open_reference()
        assert np.abs(ref_g[0] - ref_o[0]).max() < 1e-6
        assert rel_l2(ref_g[1], ref_o[1]) < FIELD_REL_L2
    o.close()
