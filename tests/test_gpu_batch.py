"""Many-domain batch stepping: each domain of a batch ends where it ends
when stepped alone."""
import numpy as np
import pytest
import torch

import lbm3_b200 as L
from lbm3_b200 import _abi as A
from lbm3_b200 import geometry as G

pytestmark = pytest.mark.gpu


def cases():
    c1 = L.tgv_plain_method().case
    c2 = L.open_channel(32, 16, 16, u_in=0.04, nu_lattice=0.02)
    G.set_bodies(c2, [G.icosphere(2, 3.0, (12.0, 8.0, 8.0))])
    c3 = L.periodic_box(24, 24, 24, nu_lattice=0.02, storage=A.LBM_STORE_F16)
    G.set_rotors(c3, [(G.rotor(hub_radius=2, tip_radius=7, chord=3, thickness=1.0, hub_length=4),
                       dict(axis=2, origin=(0, 0, 0), radians_per_second=2.0))])
    return [c1, c2, c3]


def test_batch_matches_domains_stepped_alone():
    alone = []
    for c in cases():
        with L.build_grids(c) as g:
            g.update_all_grids(25)
            alone.append(g.macro())
    grids = [L.build_grids(c) for c in cases()]
    streams = [torch.cuda.Stream() for _ in grids]
    try:
        for g, s in zip(grids, streams):
            g.set_stream(s.cuda_stream)
        L.update_batch(grids, 10)
        L.update_batch(grids, 15)
        for g, ref in zip(grids, alone):
            g.synchronize()
            np.testing.assert_array_equal(g.macro(), ref)
    finally:
        for g in grids:
            g.close()


def test_batch_rejects_null_entries():
    import ctypes as C
    arr = (C.c_void_p * 2)(None, None)
    assert A.lib().lbm_update_batch(arr, 2, 1) == A.LBM_ERR_INVALID
