"""Parity at the configurations' own sizes: the flow-around-sphere grid
(256x128x128, icosphere of 20,480 triangles, velocity inlet, non-reflective
outlet) and the plain-method Taylor-Green vortex (64^3, 1000 steps), GPU
against the oracle built from the same case (every table its own)."""
import numpy as np
import pytest

import lbm3_b200 as L
import oracle as O
from helpers import FIELD_REL_L2, density_velocity_errors, field_errors, rel_l2

pytestmark = pytest.mark.gpu


def test_sphere_configuration_fields_and_drag():
    """100 steps of the sphere configuration: fields to the FP32 bar, and the
    drag force of the body to 1e-4 against the oracle's momentum exchange."""
    s = L.flow_around_sphere(256, 128, 128)
    o = O.OracleGrid(s.case)
    steps = 100
    with L.build_grids(s.case) as g:
        g.update_all_grids(steps)
        o.step(steps)
        fl = o.int_array("wallMap") != -3
        e_rho, e_u, d_rho = density_velocity_errors(g.macro()[:, fl], o.macro()[:, fl])
        assert e_rho < FIELD_REL_L2 and e_u < FIELD_REL_L2 and d_rho < 1e-6, (e_rho, e_u, d_rho)
        # drag: FP64 sum of the per-cell momentum-exchange force, averaged
        # over the steps; the oracle's sum is in lattice units, summed over steps
        info = g.info()
        dx = info.res / 1000.0
        to_si = s.case.rho_phys * dx ** 4 / info.dt_phys ** 2
        drag_gpu = g.wall_force(0)[0]
        drag_oracle = o.wall_force(0)[0] / steps * to_si
        assert drag_gpu == pytest.approx(drag_oracle, rel=1e-4), (drag_gpu, drag_oracle)
    o.close()


def test_tgv64_plain_method_full_run():
    """The plain-method configuration for its 1000 steps: fields to the FP32
    bar, and the kinetic-energy history to twice that bar (the energy is
    quadratic in the velocity, so a relative velocity error e moves it by at
    most about 2e; the GPU contracts multiply-adds and the oracle does not, so
    the two drift apart by rounding)."""
    s = L.tgv_plain_method()
    o = O.OracleGrid(s.case)
    with L.build_grids(s.case) as g:
        eg, eo = [], []
        for _ in range(10):
            g.update_all_grids(100)
            o.step(100)
            eg.append(g.kinetic_energy(s.u_initial_phys, s.domain_length))
            eo.append(o.kinetic_energy(s.u_initial_phys, s.domain_length))
        e_rho, e_u = field_errors(g.macro(), o.macro())
        assert e_rho < FIELD_REL_L2 and e_u < FIELD_REL_L2, (e_rho, e_u)
        assert g.info().iterations_finished == 1000
    eg, eo = np.array(eg), np.array(eo)
    assert np.max(np.abs(eg - eo) / eo) < 2 * FIELD_REL_L2
    # the vortex decays
    assert eg[-1] < eg[0]
    o.close()
