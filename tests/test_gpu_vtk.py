"""VTK export (exportVTK, include/exportVTK.h:17-158): the written file holds
every cell with its centre, wall flag, physical velocity and pressure, grid
id, resolution and interface-overlap flag, consistent with the device state
read back through the ABI."""
import numpy as np
import pytest

import lbm3_b200 as L
from lbm3_b200 import geometry as G
from helpers import plan_ijk

pytestmark = pytest.mark.gpu


def read_vtk(path):
    lines = open(path).read().split("\n")
    assert lines[0] == "# vtk DataFile Version 3.0"
    assert lines[2] == "ASCII" and lines[3] == "DATASET POLYDATA"
    n = int(lines[4].split()[1])
    pts = np.array([[float(v) for v in l.split()] for l in lines[5:5 + n]], np.float32)
    q = 5 + n
    assert lines[q] == f"VERTICES {n} {2 * n}"
    q += 1 + n
    sections = {}
    assert lines[q] == f"POINT_DATA {n}"
    q += 1
    while q < len(lines) and lines[q]:
        head = lines[q].split()
        if head[0] == "SCALARS":
            vals = np.array([float(v) for v in lines[q + 2:q + 2 + n]])
            sections[head[1]] = vals
            q += 2 + n
        else:  # VECTORS
            vals = np.array([[float(v) for v in l.split()] for l in lines[q + 1:q + 1 + n]])
            sections[head[1]] = vals
            q += 1 + n
    return pts, sections


def test_vtk_export_matches_the_state(tmp_path):
    c = L.open_channel(24, 12, 12, u_in=0.04, nu_lattice=0.02)
    G.set_bodies(c, [G.icosphere(2, 3.0, (8.0, 6.0, 6.0))])
    p = L.Plan(c)
    with L.build_grids(c) as g:
        g.update_all_grids(20)
        path = tmp_path / "snap.vtk"
        g.export_vtk(path)
        m = g.macro()
        info = g.info()
        wm = g.array("wall_map")
    pts, sec = read_vtk(path)
    i, j, k = plan_ijk(p)
    np.testing.assert_array_equal(pts[:, 0], (i * np.float32(info.res) + np.float32(info.ox)).astype(np.float32))
    np.testing.assert_array_equal(pts[:, 2], (k * np.float32(info.res) + np.float32(info.oz)).astype(np.float32))
    np.testing.assert_array_equal(sec["wall"], (wm == -3).astype(float))
    fluid = wm != -3
    scale = np.float32(info.res / 1000.0) / np.float32(info.dt_phys)
    np.testing.assert_allclose(sec["velocity_m_s"][fluid, 0], m[1][fluid] * scale, rtol=1e-6, atol=1e-12)
    assert np.all(sec["velocity_m_s"][~fluid] == 0)
    cs = 0.57735026918962576 * (info.res / 1000.0) / info.dt_phys
    np.testing.assert_allclose(sec["pressure_Pa"][fluid], m[0][fluid] * c.rho_phys * cs * cs, rtol=1e-5,
                               atol=1e-9)
    assert np.all(sec["grid_id"] == 0)
    np.testing.assert_allclose(sec["grid_resolution_mm"], info.res)
    np.testing.assert_array_equal(sec["interface_overlap"], np.zeros(len(wm)))
    p.close()
