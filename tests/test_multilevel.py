"""Multilevel grids on the host: the product's builder against the oracle's
own restatement of the reference's multilevel setup (initializeGridInfo,
markRefinementCells with getRefinementModifier, buildFinerGridBuilder,
deleteExcessCells, buildWallMarkers with parent inheritance, the interface
lists of gridBuilderToGrid; include/gridBuilderFunctions.h:9-1231,
include/markerFunctions.h:222-450), table for table and bit for bit; and the
interface fit (include/updateInterface.h:262-306, :443-545) reproducing
every velocity field of its quadratic family exactly."""
import numpy as np
import pytest

import lbm3_b200 as L
import oracle as O
from lbm3_b200 import geometry as G

from test_setup_parity import ROW_ARRAYS

INTERFACE_ARRAYS = ["f2c_index", "f2c_child", "c2f_index", "c2f_child", "leftover_index", "leftover_parent",
                    "leftover_nbr"]


def assert_same_levels(case):
    p = L.Plan(case)
    d = O.OracleDomain(case)
    try:
        assert p.level_count() == d.level_count == case.grid_level_count
        total = 0
        for l in range(p.level_count()):
            info, o = p.info(l), d.level(l)
            assert info.cell_count == o.g.cellCount, l
            assert (info.res, info.ox, info.oy, info.oz, info.nu, info.dt_phys) == \
                (o.g.res, o.g.ox, o.g.oy, o.g.oz, o.g.nu, o.g.dtPhys), l
            total += o.g.fluidUpdates << l
            for mine, theirs in ROW_ARRAYS:
                np.testing.assert_array_equal(p.array(mine, l), o.int_array(theirs), err_msg=f"{mine} level {l}")
            w = o.wall_arrays()
            np.testing.assert_array_equal(p.array("wall_index", l), w["index"])
            np.testing.assert_array_equal(p.uint_array("wall_data", l), w["wall_data"])
            np.testing.assert_array_equal(p.uint_array("link_length", l).reshape(7, -1), w["link_length"])
            np.testing.assert_array_equal(p.wall_velocity(l).reshape(3, -1), w["wall_velocity"])
            np.testing.assert_array_equal(p.array("open_index", l), o.open_index())
            if l + 1 < p.level_count():
                theirs = d.interface(l)
                for name in INTERFACE_ARRAYS:
                    np.testing.assert_array_equal(p.array(name, l), theirs[name], err_msg=f"{name} level {l}")
        assert p.fluid_updates_per_iteration == total
        return [p.info(l) for l in range(p.level_count())]
    finally:
        d.close()
        p.close()


def test_refined_taylor_green_tables():
    """The reference's refined Taylor-Green grid (central cube on level 1)."""
    infos = assert_same_levels(L.taylor_green_refined(32).case)
    assert infos[0].f2c_count > 0 and infos[0].c2f_count > 0
    # the fine cube and the coarse cells under it: every level-1 cell has a parent
    assert infos[1].cell_count > 0 and infos[1].periodic_count == 0


def test_three_level_box_with_hook_tables():
    """Three levels from a refinement hook (getRefinementModifier) on a
    periodic box, off-centre so that the fine boxes are ragged against the
    coarse rows, with leftover fine cells."""
    c = L.periodic_box(30, 22, 18, nu_lattice=0.02)
    c.grid_level_count = 3

    def refine(i, j, k, mark, info):
        x, y, z = i * info.res + info.ox, j * info.res + info.oy, k * info.res + info.oz
        if info.grid_id == 0:
            return mark or (-8.7 < x < 5.6 and -7.8 < y < 3.1 and -4.5 < z < 3.9)
        return mark or (-5.9 < x < 1.2 and -4.6 < y < 0.8 and -2.3 < z < 1.3)
    L.set_hooks(c, refinement=refine)
    infos = assert_same_levels(c)
    assert [i.cell_count > 0 for i in infos] == [True, True, True]
    assert infos[0].c2f_count > 0 and infos[1].c2f_count > 0


def test_refined_sphere_channel_tables():
    """Two levels with a body: wall refinement around the sphere
    (markAllFinerWalls + WALL_REFINEMENT_COUNT), walls and wallIDs inherited
    from the parent, links through the interface at length 1/2, open
    boundaries on level 0."""
    c = L.open_channel(48, 24, 24, u_in=0.04, nu_lattice=0.02)
    G.set_bodies(c, [G.icosphere(2, 4.0, (16.0, 12.0, 12.0))])
    c.grid_level_count = 2
    c.wall_refinement_count = 2
    infos = assert_same_levels(c)
    assert infos[1].wall_adjacent_count > 0 and infos[0].f2c_count > 0


def slab_channel_refined():
    """A plane channel whose refined block (from a refinement hook that
    overrides the wall marks, as the reference's Taylor-Green hook does)
    ends across the walls: coarse stencils there hold wall cells, so the
    band has leftover fine cells, some next to a wall."""
    from test_walls import channel_case
    c = channel_case(n_xy=24, half_height=6.2, nz=18)
    c.grid_level_count = 2

    def refine(i, j, k, mark, info):
        x, y = i * info.res + info.ox, j * info.res + info.oy
        return -5.1 < x < 4.3 and -3.7 < y < 5.2
    L.set_hooks(c, refinement=refine)
    return c


def test_refined_slab_channel_leftover_tables():
    infos = assert_same_levels(slab_channel_refined())
    assert infos[0].leftover_count > 0 and infos[1].wall_cell_count > 0


def test_refinement_box_and_hook_agree():
    """A refinement box is the same refinement as the equivalent hook."""
    a = L.taylor_green_refined(32).case
    b = L.taylor_green(32).case
    b.grid_level_count = 2
    half = np.float32(0.25) * np.float32(L.taylor_green(32).domain_length)

    def refine(i, j, k, mark, info):
        if info.grid_id != 0:
            return False
        x = np.float32(i * np.float32(info.res) + np.float32(info.ox))
        y = np.float32(j * np.float32(info.res) + np.float32(info.oy))
        z = np.float32(k * np.float32(info.res) + np.float32(info.oz))
        return bool(-half < x < half and -half < y < half and -half < z < half)
    L.set_hooks(b, refinement=refine)
    pa, pb = L.Plan(a), L.Plan(b)
    for l in range(2):
        np.testing.assert_array_equal(pa.array("shifter", l), pb.array("shifter", l))
        np.testing.assert_array_equal(pa.array("c2f_index", 0), pb.array("c2f_index", 0))
    pa.close()
    pb.close()


def _corner_records(rng):
    """8 corner records of a random velocity field of the fit's family, with
    the strain estimates the populations would carry."""
    keys = ["0", "x", "y", "z", "xy", "xz", "yz", "xyz", "xx", "yy", "zz"]
    C = [{k: rng.normal() for k in keys} for _ in range(3)]
    D = {k: rng.normal() * 1e-2 for k in ["0", "x", "y", "z", "xy", "xz", "yz", "xyz"]}

    def u(r):
        x, y, z = r
        return np.array([c["0"] + c["x"] * x + c["y"] * y + c["z"] * z + c["xy"] * x * y + c["xz"] * x * z +
                         c["yz"] * y * z + c["xyz"] * x * y * z + c["xx"] * x * x + c["yy"] * y * y +
                         c["zz"] * z * z for c in C])

    def grad(r):
        x, y, z = r
        G = np.zeros((3, 3))
        for a, c in enumerate(C):
            G[a] = [c["x"] + c["xy"] * y + c["xz"] * z + c["xyz"] * y * z + 2 * c["xx"] * x,
                    c["y"] + c["xy"] * x + c["yz"] * z + c["xyz"] * x * z + 2 * c["yy"] * y,
                    c["z"] + c["xz"] * x + c["yz"] * y + c["xyz"] * x * y + 2 * c["zz"] * z]
        return G

    def rho(r):
        x, y, z = r
        return (D["0"] + D["x"] * x + D["y"] * y + D["z"] * z + D["xy"] * x * y + D["xz"] * x * z +
                D["yz"] * y * z + D["xyz"] * x * y * z)

    rec = np.zeros((8, 9))
    for q in range(8):
        r = np.array([(q & 1) - 0.5, ((q >> 1) & 1) - 0.5, ((q >> 2) & 1) - 0.5])
        g = grad(r)
        rec[q] = [rho(r), *u(r), g[0, 1] + g[1, 0], g[1, 2] + g[2, 1], g[0, 2] + g[2, 0],
                  g[0, 0] - g[1, 1], g[0, 0] - g[2, 2]]
    return rec, u, grad, rho


@pytest.mark.parametrize("seed", range(4))
def test_interface_fit_reproduces_its_family(seed):
    """Density trilinear and velocity quadratic per axis with cross terms:
    the fit of the 8 corner records returns value and gradient exactly (to
    FP32 rounding) at the centre (fine-to-coarse) and at the 8 fine-cell
    offsets (coarse-to-fine)."""
    rng = np.random.default_rng(seed)
    rec, u, grad, rho = _corner_records(rng)
    for r in [(0.0, 0.0, 0.0)] + [(sx * 0.25, sy * 0.25, sz * 0.25) for sx in (-1, 1) for sy in (-1, 1)
                                   for sz in (-1, 1)]:
        out = O.fit_check(rec, *r)
        np.testing.assert_allclose(out[0], rho(r), atol=2e-7)
        np.testing.assert_allclose(out[1:4], u(r), rtol=1e-5, atol=1e-5)
        np.testing.assert_allclose(out[4:].reshape(3, 3), grad(r), rtol=1e-5, atol=2e-5)
