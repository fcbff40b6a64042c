"""FP64 global accumulators (lbm_global_sums): mass and momentum over the
fluid cells against the oracle's FP64 sums of the same state, and mass
conservation of a closed periodic domain."""
import numpy as np
import pytest

import lbm3_b200 as L
from lbm3_b200 import geometry as G
import oracle as O

pytestmark = pytest.mark.gpu


def test_sums_match_the_oracle_with_walls_and_open_boundaries():
    c = L.open_channel(48, 24, 24, u_in=0.04, nu_lattice=0.02)
    G.set_bodies(c, [G.icosphere(3, 4.0, (16.0, 12.0, 12.0))])
    o = O.OracleGrid(c)
    with L.build_grids(c) as g:
        g.update_all_grids(40)
        o.step(40)
        s = g.global_sums()
        ref = o.global_sums()
        assert s["cells"] == ref[5]
        assert s["sum_rho"] == pytest.approx(ref[0], rel=1e-7)
        assert s["sum_drho"] == pytest.approx(ref[1], rel=1e-4, abs=1e-6 * ref[5])
        info = g.info()
        dx = info.res / 1000.0
        scale = c.rho_phys * dx ** 3 * dx / info.dt_phys
        assert s["momentum_x"] / scale == pytest.approx(ref[2], rel=1e-5)
        assert s["mass"] == pytest.approx(c.rho_phys * dx ** 3 * ref[0], rel=1e-7)
    o.close()


def test_closed_periodic_domain_conserves_mass():
    """A periodic box with a turning rotor: momentum appears, mass stays."""
    c = L.periodic_box(40, 40, 30, nu_lattice=0.02)
    tris = G.rotor(hub_radius=3, tip_radius=12, chord=5, thickness=1.5, hub_length=6)
    G.set_rotors(c, [(tris, dict(axis=2, origin=(0.0, 0.0, 0.0), radians_per_second=2.0))])
    with L.build_grids(c) as g:
        s0 = g.global_sums()
        g.update_all_grids(200)
        s1 = g.global_sums()
    assert s1["cells"] == s0["cells"]
    # FP32 populations: drift per cell of the order of FP32 rounding per step
    assert abs(s1["sum_drho"] - s0["sum_drho"]) / s0["cells"] < 1e-5
    assert abs(s1["momentum_x"]) + abs(s1["momentum_y"]) > 0.0
