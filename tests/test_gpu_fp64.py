"""The FP64 build of the kernels (LBM_STORE_F64: FP64 populations and FP64
arithmetic), the reference of the storage-precision study.  It is checked
against the FP32 oracle (the two differ only by FP32 rounding over a few
steps) and against the GPU's FP32 path, on every kernel of the step:
collide-stream with interpolated bounceback, the open boundary, periodic
ghosts and the rotor forcing."""
import numpy as np
import pytest

import lbm3_b200 as L
from lbm3_b200 import _abi as A
from lbm3_b200 import geometry as G
import oracle as O
from helpers import FIELD_REL_L2, density_velocity_errors

pytestmark = pytest.mark.gpu


def sphere_channel(storage):
    c = L.open_channel(48, 24, 24, u_in=0.04, nu_lattice=0.02, storage=storage)
    G.set_bodies(c, [G.icosphere(3, 4.0, (16.0, 12.0, 12.0))])
    c.track_wall_force = 1
    c.track_open_boundaries = 1
    return c


@pytest.mark.parametrize("steps", [1, 50])
def test_fp64_build_matches_the_oracle(steps):
    c = sphere_channel(A.LBM_STORE_F64)
    o = O.OracleGrid(c)
    with L.build_grids(c) as g:
        assert g.info().storage == A.LBM_STORE_F64
        g.update_all_grids(steps)
        o.step(steps)
        fl = o.int_array("wallMap") != -3
        e_rho, e_u, d_rho = density_velocity_errors(g.macro()[:, fl], o.macro()[:, fl])
        assert e_rho < FIELD_REL_L2 and e_u < FIELD_REL_L2 and d_rho < 1e-6, (e_rho, e_u, d_rho)
    o.close()


def test_fp64_and_fp32_agree_to_fp32_rounding():
    out = {}
    for st in (A.LBM_STORE_F32, A.LBM_STORE_F64):
        with L.build_grids(sphere_channel(st)) as g:
            g.update_all_grids(100)
            out[st] = (g.macro(), g.wall_force(0))
    e_rho, e_u, _ = density_velocity_errors(out[A.LBM_STORE_F32][0], out[A.LBM_STORE_F64][0])
    assert e_rho < FIELD_REL_L2 and e_u < FIELD_REL_L2, (e_rho, e_u)
    f32, f64 = out[A.LBM_STORE_F32][1], out[A.LBM_STORE_F64][1]
    assert abs(f32[0] - f64[0]) <= 1e-4 * abs(f64[0]), (f32, f64)


def test_fp64_periodic_rotor_box():
    """Periodic ghosts and rotor forcing in FP64 against the FP32 oracle."""
    c = L.periodic_box(40, 40, 30, nu_lattice=0.02, storage=A.LBM_STORE_F64)
    tris = G.rotor(hub_radius=3, tip_radius=12, chord=5, thickness=1.5, hub_length=6)
    G.set_rotors(c, [(tris, dict(axis=2, origin=(0.0, 0.0, 0.0), radians_per_second=2.0))])
    o = O.OracleGrid(c)
    with L.build_grids(c) as g:
        g.update_all_grids(30)
        o.step(30)
        e_rho, e_u, d_rho = density_velocity_errors(g.macro(), o.macro())
        assert e_u < FIELD_REL_L2 and d_rho < 1e-6, (e_rho, e_u, d_rho)
    o.close()
