"""Device footprint: grid_memory_bytes, which the serving loop admits
requests by, counts every array a build allocates.  Checked against the
device's free-memory drop across a build of a case with walls, open
boundaries and a rotor."""
import numpy as np
import pytest
import torch

import lbm3_b200 as L
from lbm3_b200 import geometry as G

pytestmark = pytest.mark.gpu

MIB = 1 << 20


def busy_case():
    c = L.open_channel(96, 48, 48, u_in=0.04, nu_lattice=0.02)
    G.set_bodies(c, [G.icosphere(3, 6.0, (30.0, 24.0, 24.0)), G.box((60.0, 10.0, 10.0), (70.0, 20.0, 38.0))])
    tris = G.rotor(hub_radius=3, tip_radius=10, chord=4, thickness=1.5, hub_length=6)
    tris = (tris.reshape(-1, 3, 3) + np.array([45.0, 24.0, 24.0], np.float32)).reshape(-1, 9)
    G.set_rotors(c, [(tris, dict(axis=0, origin=(45.0, 24.0, 24.0), radians_per_second=1.0))])
    c.track_rotor_force = 1
    c.track_wall_force = 1
    c.track_open_boundaries = 1
    return c


def test_footprint_counts_every_allocation():
    torch.cuda.set_device(0)
    c = busy_case()
    p = L.Plan(c)
    planned = int(p.info().grid_memory_bytes)
    p.close()
    # a first build loads the library's device code and warms the allocator
    L.build_grids(c).close()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    g = L.build_grids(c)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    built = int(g.info().grid_memory_bytes)
    g.close()
    used = free0 - free1
    assert built == planned
    # the driver hands out memory in pages: the drop is the footprint rounded
    # up, never less than what was counted minus one page
    assert planned <= used + 2 * MIB, (planned, used)
    assert used <= planned + 64 * MIB, (planned, used)
