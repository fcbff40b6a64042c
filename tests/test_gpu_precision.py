"""Storage-precision study against the FP64 build of the kernels
(LBM_STORE_F64: FP64 populations and arithmetic), on converged cases:
drag of a sphere in a channel at steady state, the Taylor-Couette torque of
a turning wall (moving-wall interpolated bounceback), the velocity field, and
the mass drift of a closed periodic box stirred by a forcing rotor.  FP32,
FP16-shifted and BF16-shifted populations (FP32 arithmetic) are compared
with FP64; the printed table is the study's result."""
import numpy as np
import pytest

import lbm3_b200 as L
from lbm3_b200 import _abi as A
from lbm3_b200 import geometry as G
from helpers import rel_l2
from test_walls import couette_case

pytestmark = pytest.mark.gpu

STORAGES = [("f64", A.LBM_STORE_F64), ("f32", A.LBM_STORE_F32), ("f16", A.LBM_STORE_F16),
            ("bf16", A.LBM_STORE_BF16)]


def steady_sphere(storage, steps=6000, window=500):
    """Sphere D = 8 in a 64x32x32 channel at u = 0.04, nu = 0.04 (Re 8):
    the drag averaged over the last `window` steps of a converged run."""
    c = L.open_channel(64, 32, 32, u_in=0.04, nu_lattice=0.04, collision_limiter=0.0, storage=storage)
    G.set_bodies(c, [G.icosphere(3, 4.0, (20.0, 16.0, 16.0))])
    c.track_wall_force = 1
    with L.build_grids(c) as g:
        g.update_all_grids(steps - window)
        g.wall_force(0, reset=True)
        g.update_all_grids(window)
        drag = g.wall_force(0)[0]
        macro = g.macro()
        fluid = g.array("wall_map") != -3
    return drag, macro[:, fluid]


def couette(storage):
    c = couette_case(storage=storage)
    with L.build_grids(c) as g:
        g.update_all_grids(3000)
        g.wall_force(0, reset=True)
        g.update_all_grids(500)
        return g.wall_force(0)[5]


def rotor_box_mass(storage, steps=2000):
    """Relative change of the total mass of a closed periodic box stirred by a
    forcing rotor over `steps` steps (FP64 accumulators on the device)."""
    c = L.periodic_box(40, 40, 30, nu_lattice=0.02, storage=storage)
    tris = G.rotor(hub_radius=3, tip_radius=12, chord=5, thickness=1.5, hub_length=6)
    G.set_rotors(c, [(tris, dict(axis=2, origin=(0.0, 0.0, 0.0), radians_per_second=2.0))])
    with L.build_grids(c) as g:
        m0 = g.global_sums()["sum_rho"]
        g.update_all_grids(steps)
        m1 = g.global_sums()["sum_rho"]
        return (m1 - m0) / m0


def test_storage_precision_against_fp64():
    drag, fields, torque, drift = {}, {}, {}, {}
    for name, st in STORAGES:
        drag[name], fields[name] = steady_sphere(st)
        torque[name] = couette(st)
        drift[name] = rotor_box_mass(st)
    print("\nstorage  drag rel.err   torque rel.err   velocity rel.L2   mass drift (2000 steps)")
    for name, _ in STORAGES:
        e_d = abs(drag[name] - drag["f64"]) / abs(drag["f64"])
        e_t = abs(torque[name] - torque["f64"]) / abs(torque["f64"])
        e_u = rel_l2(fields[name][1:4].reshape(-1), fields["f64"][1:4].reshape(-1))
        print(f"{name:6s}   {e_d:.3e}      {e_t:.3e}        {e_u:.3e}         {drift[name]:+.3e}")
    for name in ("f32", "f16"):
        # the north star's bar: 16-bit shifted storage within 1e-3 of FP64
        assert abs(drag[name] - drag["f64"]) <= 1e-3 * abs(drag["f64"]), (name, drag)
        assert abs(torque[name] - torque["f64"]) <= 1e-3 * abs(torque["f64"]), (name, torque)
    assert abs(drag["bf16"] - drag["f64"]) <= 1e-2 * abs(drag["f64"]), drag
    assert abs(drift["f64"]) < 1e-12
