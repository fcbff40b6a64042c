"""Section-plane flow reports (getFlowReportXY/ZY/ZX) on the GPU against the
oracle's sums, and their physics on a uniform stream."""
import numpy as np
import pytest

import lbm3_b200 as L
from lbm3_b200 import _abi as A
from lbm3_b200 import geometry as G
import oracle as O

pytestmark = pytest.mark.gpu


def converted(t, info, rho_phys=1.0):
    """The unit conversion of include/flowReportFunctions.h:322-351 on raw sums."""
    px = info.res / 1000.0
    area, vs = px * px, px / info.dt_phys
    ps = rho_phys * vs * vs / 3.0
    mfs = rho_phys * area * vs
    return np.array([t[0] / t[5] * vs, (t[0] + t[1]) * mfs, t[2] * mfs * vs, t[3] / t[5] * ps,
                     t[1] * area * ps * vs, t[4] * mfs * vs * vs, t[5] * info.res * info.res])


def case():
    c = L.open_channel(48, 24, 24, u_in=0.04, nu_lattice=0.02)
    G.set_bodies(c, [G.icosphere(2, 4.0, (20.0, 12.0, 12.0))])
    G.set_rotors(c, [(G.rotor(hub_radius=2, tip_radius=6, chord=3, thickness=1.0, hub_length=4,
                              center=(34.0, 12.0, 12.0)),
                      dict(axis=0, origin=(34.0, 12.0, 12.0), radians_per_second=3.0))])
    return c


@pytest.mark.parametrize("plane,cut", [(A.PLANE_ZY, 20.5), (A.PLANE_ZY, 34.5), (A.PLANE_XY, 12.5),
                                       (A.PLANE_ZX, 11.5)])
def test_flow_report_matches_oracle(plane, cut):
    c = case()
    p = L.Plan(c)
    o = O.OracleGrid(c)
    with L.build_grids(c) as g:
        g.update_all_grids(40)
        o.step(40)
        info = g.info()
        rep = g.flow_report(plane, cut)
        n = (info.cell_count_x, info.cell_count_y, info.cell_count_z)
        o_ = (info.ox, info.oy, info.oz)
        axis = {A.PLANE_XY: 2, A.PLANE_ZY: 0, A.PLANE_ZX: 1}[plane]
        layer = int(np.float32((cut - o_[axis]) / info.res + 0.5))
        ha, va = (0 if plane == A.PLANE_XY else 2), (0 if plane == A.PLANE_ZX else 1)
        t = o.flow_sums(plane, layer, 0, n[ha], 0, n[va])
        want = converted(t, info)
        got = np.array(list(rep.values()))
        assert got[6] == want[6]  # same fluid pixels
        # planes along the stream carry sums that nearly cancel, so the bar is
        # relative to what a 1 m/s unit stream through the same area gives
        area = got[6] * 1e-6
        ps = (info.res / 1000.0 / info.dt_phys) ** 2 / 3.0
        unit = np.array([1.0, area, area, ps, area * ps, area])
        assert np.all(np.abs(got[:6] - want[:6]) <= 1e-4 * np.abs(want[:6]) + 1e-6 * unit), (got, want)
    o.close()


def test_uniform_stream_through_a_cropped_plane():
    c = L.open_channel(32, 16, 16, u_in=0.04, nu_lattice=0.02)
    with L.build_grids(c) as g:
        g.update_all_grids(10)
        # interior crop of 10 x 10 cells (faces at 3 and 13 mm, bounds given
        # with margin) at x = 16 mm: u_in is 1 m/s
        rep = g.flow_report(A.PLANE_ZY, 16.5, bounds=(0, 2.8, 2.8, 0, 13.2, 13.2))
        assert rep["area_mm2"] == pytest.approx(100.0)
        assert rep["normal_velocity"] == pytest.approx(1.0, rel=1e-4)
        assert rep["mass_flow"] == pytest.approx(1.0 * 100e-6, rel=1e-4)
        with pytest.raises(A.LbmError):
            g.flow_report(A.PLANE_ZY, 500.0)


@pytest.mark.parametrize("plane,frac", [(A.PLANE_XY, 0.013), (A.PLANE_ZY, -0.31), (A.PLANE_ZX, 0.07)])
def test_flow_report_on_two_levels_matches_oracle(plane, frac):
    """A refined Taylor-Green domain: the section image at the finest level,
    filled by both levels (the coarse level's layers bracket the cut and are
    blended), against the oracle's restatement of the same image."""
    s = L.taylor_green(32)
    c = s.case
    c.grid_level_count = 2
    q = float(s.domain_length)
    c.refine_box[0][:] = (-0.2 * q, -0.25 * q, -0.2 * q, 0.22 * q, 0.25 * q, 0.2 * q)
    d = O.OracleDomain(c)
    cut = frac * q
    with L.build_grids(c) as g:
        g.update_all_grids(3)
        d.step(3)
        rep = g.flow_report(plane, cut)
        t, level = d.flow_image(plane, cut)
        info = g.info(level)
        want = converted(t, info)
        got = np.array(list(rep.values()))
        assert got[6] == pytest.approx(want[6])  # same fluid pixels, areas of the image level
        area = got[6] * 1e-6
        ps = (info.res / 1000.0 / info.dt_phys) ** 2 / 3.0
        unit = np.array([1.0, area, area, ps, area * ps, area])
        assert np.all(np.abs(got[:6] - want[:6]) <= 1e-4 * np.abs(want[:6]) + 1e-6 * unit), (got, want)
