"""Setup parity: every table the product's host builder produces for bodies,
open boundaries and rotors is bit-identical to the oracle's own restatement
of the reference's setup chain (readSTL bounds, sortSTLToBins, voxelizeSTL /
sumRayMaps, markKeepCells, deleteExcessCells, buildWallMarkers,
buildLinkExistenceMarkerArray, buildLinkLengthArray, packWallData,
buildRotors; include/voxelizerFunctions.h, include/markerFunctions.h,
include/gridBuilderFunctions.h:402-1564,
include/boundaryConditions/interpolatedBouncebackFunctions.h:181-695,
include/rotorFunctions.h:315-470)."""
import numpy as np
import pytest

import lbm3_b200 as L
import oracle as O
from lbm3_b200 import geometry as G
from lbm3_b200 import serving as S

from test_rotor import rotor_case
from test_walls import channel_case, couette_case

ROW_ARRAYS = [("shifter", "shifter"), ("row_i", "rowI"), ("row_j", "rowJ"), ("row_k", "rowK"),
              ("row_jplus", "rowJP"), ("row_kplus", "rowKP"), ("row_jkplus", "rowJKP"), ("wall_map", "wallMap"),
              ("periodic_index", "perIndex"), ("periodic_source", "perSource")]


def assert_same_tables(case):
    p = L.Plan(case)
    o = O.OracleGrid(case)
    try:
        info = p.info()
        assert info.cell_count == o.g.cellCount
        assert p.fluid_updates_per_iteration == o.g.fluidUpdates
        for mine, theirs in ROW_ARRAYS:
            np.testing.assert_array_equal(p.array(mine), o.int_array(theirs), err_msg=mine)
        w = o.wall_arrays()
        np.testing.assert_array_equal(p.array("wall_index"), w["index"])
        np.testing.assert_array_equal(p.uint_array("wall_data"), w["wall_data"])
        np.testing.assert_array_equal(p.uint_array("link_length").reshape(7, -1), w["link_length"])
        np.testing.assert_array_equal(p.wall_velocity().reshape(3, -1), w["wall_velocity"])
        np.testing.assert_array_equal(p.array("open_index"), o.open_index())
        assert p.rotor_count() == o.g.rotorCount
        for r in range(p.rotor_count()):
            ri, ot = p.rotor_info(r), o.rotor_tables(r)
            assert ri.res == ot["res"]
            np.testing.assert_array_equal(np.array(ri.bounds[:], np.float32), ot["bounds"])
            np.testing.assert_array_equal(np.array(ri.cell_count[:]), ot["cell_count"])
            np.testing.assert_array_equal(p.rotor_array(r, "map"), ot["map"])
            np.testing.assert_array_equal(p.rotor_array(r, "interpolation"), ot["interpolation"])
        return info
    finally:
        o.close()
        p.close()


def test_sphere_in_channel_tables():
    c = L.open_channel(32, 16, 16, u_in=0.04, nu_lattice=0.02)
    G.set_bodies(c, [G.icosphere(2, 3.0, (12.0, 8.0, 8.0))])
    info = assert_same_tables(c)
    assert info.wall_adjacent_count > 0 and info.wall_cell_count > 0


def test_sphere_configuration_tables():
    """The flow-around-sphere configuration at full size: 256x128x128 with an
    icosphere of 20,480 triangles (voxelizer, markers, links, open lists)."""
    s = L.flow_around_sphere(256, 128, 128)
    info = assert_same_tables(s.case)
    assert info.cell_count > 4_000_000


def test_rotating_walls_tables():
    """Taylor-Couette meshes with a turning inner wall: wallIDs, link
    lengths of curved walls and rigid-rotation wall velocities."""
    assert_same_tables(couette_case())


def test_slab_channel_tables():
    assert_same_tables(channel_case())


@pytest.mark.parametrize("seed", [7, 11])
def test_serving_request_tables(seed):
    """Seeded serving channels (ellipsoid or icosphere obstacle)."""
    rng = np.random.default_rng(seed)
    for q in range(3):
        r = S.channel_request(q, int(rng.choice([32, 48])), rng, 100)
        assert_same_tables(r.case)


def test_rotor_tables():
    assert_same_tables(rotor_case(G.rotor(hub_radius=3, tip_radius=12, chord=5, thickness=1.5, hub_length=6)))
    lo = (3.3, 4.1, 5.2)
    assert_same_tables(rotor_case(G.box(lo, (lo[0] + 7.7, lo[1] + 5.3, lo[2] + 6.1))))


def test_two_bodies_last_wins_and_union():
    """Overlapping bodies: the union of solid intervals (sumRayMaps) and the
    wallID priority of the last body (buildWallMarkers)."""
    c = L.open_channel(48, 24, 24, u_in=0.03, nu_lattice=0.02)
    G.set_bodies(c, [G.icosphere(2, 4.0, (16.0, 12.0, 12.0)), G.box((17.0, 9.0, 9.0), (25.0, 15.0, 15.0))])
    assert_same_tables(c)
