"""Static bodies: voxelizer known answers, IBB link lengths, and an analytic
Poiseuille pin for the interpolated bounceback of the oracle."""
import numpy as np
import pytest

import lbm3_b200 as L
from lbm3_b200 import _abi as A
from lbm3_b200 import geometry as G
import oracle as O
from helpers import plan_ijk


def channel_case(n_xy=8, half_height=10.2, nz=32, nu=0.1, gx=1e-6, track=True):
    """Plane channel: periodic in x and y, two slabs bounding |z| < half_height,
    driven by the body force gx (lattice units).  Cell centres sit at
    half-integer coordinates, so the walls cut the links at fraction 0.7."""
    c = L.periodic_box(n_xy, n_xy, nz, nu_lattice=nu)
    big = 100.0
    lower = G.box((-big, -big, -big), (big, big, -half_height))
    upper = G.box((-big, -big, half_height), (big, big, big))
    G.set_bodies(c, [lower, upper])
    c.gx = gx
    c.track_wall_force = int(track)
    # AllOne collision, as the reference's channel drivers select for walls
    # (cases/poiseuilleFlow/poiseuilleFlowMain.cu:84); K17 with the default
    # limiter is not stable at this high viscosity (omega1 = 1.25)
    c.collision_limiter = 0.0
    return c


def test_box_slabs_voxelize_to_exact_cells():
    c = channel_case()
    p = L.Plan(c)
    info = p.info()
    wm = p.array("wall_map")
    # cell centres z = -16.5 ... 16.5 (34 cells); fluid where |z| < 10.2
    nx, ny, nz = info.cell_count_x, info.cell_count_y, info.cell_count_z
    z = np.arange(nz) + info.oz
    fluid_k = (np.abs(z) < 10.2).sum()
    assert (wm != -3).sum() == nx * ny * fluid_k
    # one wall layer kept on each side, deeper cells deleted
    assert info.wall_cell_count == 2 * nx * ny
    assert info.cell_count == nx * ny * (fluid_k + 2)


def test_plane_link_lengths_have_the_analytic_code():
    p = L.Plan(channel_case())
    info = p.info()
    wd = p.uint_array("wall_data")
    ll = p.uint_array("link_length").reshape(7, -1)
    nw = info.wall_adjacent_count
    assert nw > 0
    expected = int(0.7 * 254 + 0.5)  # wall 0.7 cells beyond the outermost fluid centre
    idx = p.array("wall_index")
    nx, ny = info.cell_count_x, info.cell_count_y
    i, j = idx % nx, (idx // nx) % ny
    interior = (i > 0) & (i < nx - 1) & (j > 0) & (j < ny - 1)
    assert interior.sum() == 2 * (nx - 2) * (ny - 2)
    for w in np.nonzero(interior)[0]:
        links = bin(int(wd[w]) & 0x7FFFFFE).count("1")
        assert links == 9  # the 9 directions with a z component towards the wall
        codes = [(int(ll[q // 4, w]) >> (8 * (q % 4))) & 255 for q in range(links)]
        assert codes == [expected] * links


def test_icosphere_solid_volume():
    c = L.periodic_box(48, 48, 48)
    G.set_bodies(c, [G.icosphere(4, 12.0, (0.31, 0.17, -0.23))])
    p = L.Plan(c)
    info = p.info()
    n_all = info.cell_count_x * info.cell_count_y * info.cell_count_z
    solid = info.wall_cell_count + (n_all - info.cell_count)
    vol = 4.0 / 3.0 * np.pi * 12.0 ** 3
    assert abs(solid - vol) / vol < 0.02
    # every wall-adjacent cell has at least one link
    wd = p.uint_array("wall_data")
    assert np.all((wd & 0x7FFFFFE) != 0)


def test_rotating_body_gets_rigid_rotation_velocity():
    c = L.periodic_box(16, 16, 16)
    c.dt_phys_global = 1e-3
    tris = G.icosphere(3, 4.0)
    G.set_bodies(c, [(tris, {"motion": A.LBM_WALL_ROTATING, "axis": 2, "origin": (0, 0, 0),
                             "radians_per_second": 2.0})])
    p = L.Plan(c)
    v = p.wall_velocity()
    idx = p.array("wall_index")
    info = p.info()
    # recover cell centres of the wall-adjacent cells from the dense ordering
    nx, ny = info.cell_count_x, info.cell_count_y
    # the box has no deleted cells outside the sphere: rows are full i-lines
    assert v.shape == (3, len(idx))
    s = 2.0 * 1e-3 / info.res
    assert np.all(np.abs(v[2]) == 0)
    speed = np.hypot(v[0], v[1])
    assert speed.max() > 0 and speed.max() < s * 6.0


def test_invalid_bodies_are_rejected():
    c = L.periodic_box(8, 8, 8)
    G.set_bodies(c, [G.box((-1, -1, -1), (1, 1, 1))])
    c.body[0].motion = 7
    with pytest.raises(A.LbmError):
        L.Plan(c)
    c.body[0].motion = A.LBM_WALL_STATIC
    c.body[0].triangle_count = 0
    with pytest.raises(A.LbmError):
        L.Plan(c)


def test_oracle_poiseuille_matches_the_analytic_profile():
    """Force-driven channel between IBB walls at |z| = 10.2: the steady
    velocity profile is u(z) = g (h^2 - z^2) / (2 nu)."""
    nu, g, h = 0.1, 1e-6, 10.2
    c = channel_case(nu=nu, gx=g)
    p = L.Plan(c)
    o = O.OracleGrid(c)
    o.step(3000)
    m = o.macro()
    info = p.info()
    wm = p.array("wall_map")
    _, _, kz = plan_ijk(p)
    z = info.oz + kz * info.res
    fluid = wm != -3
    ux = m[1][fluid]
    ua = g * (h * h - z[fluid] ** 2) / (2 * nu)
    err = np.max(np.abs(ux - ua)) / ua.max()
    assert err < 0.01, err
    o.close()


def couette_case(nu=0.1, u_wall=0.01, r1=10.0, r2=16.0, nz=4, storage=A.LBM_STORE_F32):
    """Periodic Taylor-Couette annulus (cases/torqueTest/torqueTestMain.cu:1-60):
    a voxelized inner cylinder turning about z inside a fixed bore, both
    extending past the periodic z range; 1 mm cells, dt = 1 ms."""
    c = L.periodic_box(36, 36, nz, nu_lattice=nu, storage=storage)
    c.collision_limiter = 0.0
    omega = u_wall / r1 / 1e-3  # rad/s so that the wall moves u_wall cells per step
    G.set_bodies(c, [(G.cylinder(r1, -10, 10), dict(motion=A.LBM_WALL_ROTATING, axis=2, origin=(0, 0, 0),
                                                     radians_per_second=omega)),
                     G.bored_block(19.5, r2, -10, 10)])
    c.track_wall_force = 1
    return c


def couette_torque_lattice(nu=0.1, u_wall=0.01, r1=10.0, r2=16.0, nz=4):
    """Analytic torque on an annulus of length nz (torqueTestMain.cu:45-54), lattice units."""
    om = u_wall / r1
    return 4 * np.pi * nu * om * r1 ** 2 * r2 ** 2 / (r2 ** 2 - r1 ** 2) * nz


def test_oracle_taylor_couette_torque():
    """Steady torque of the inner and outer walls against the analytic value
    (moving-wall interpolated bounceback and the momentum-exchange tracker)."""
    c = couette_case()
    o = O.OracleGrid(c)
    o.step(3000)
    a0, a1 = o.wall_force(0)[5], o.wall_force(1)[5]
    o.step(500)
    t_in = (o.wall_force(0)[5] - a0) / 500
    t_out = (o.wall_force(1)[5] - a1) / 500
    t = couette_torque_lattice()
    assert t_in == pytest.approx(t, rel=0.01)
    assert t_out == pytest.approx(-t, rel=0.01)
    o.close()
