"""Many-domain batch stepping: each domain of a batch ends where it ends
when stepped alone."""
import numpy as np
import pytest
import torch

import lbm3_b200 as L
from lbm3_b200 import _abi as A
from lbm3_b200 import geometry as G
from helpers import FIELD_REL_L2, rel_l2

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


def packed_cases(storage):
    """Three single-level domains of one storage type: Taylor-Green 32^3 with
    periodic ghosts, a channel around a sphere (open boundaries, walls) and a
    stirred periodic box with a body force."""
    c1 = L.taylor_green(32, storage=storage).case
    c2 = L.open_channel(40, 20, 18, u_in=0.04, nu_lattice=0.02, storage=storage)
    G.set_bodies(c2, [G.icosphere(2, 3.5, (14.0, 10.0, 9.0))])
    c2.track_wall_force = 1
    c3 = L.periodic_box(20, 28, 24, nu_lattice=0.03, storage=storage)
    c3.gx = 1e-5
    return [c1, c2, c3]


def _run_packed(cases, plan):
    """Populations and wall forces after the step plan: batch updates with
    member steps in between (("batch", n) or ("member", n))."""
    grids = [L.build_grids(c) for c in cases]
    try:
        with L.PackedBatch(grids) as b:
            for kind, n in plan:
                if kind == "batch":
                    b.update(n)
                else:
                    for g in grids:
                        g.update_all_grids(n)
        out = []
        for g, c in zip(grids, cases):
            g.synchronize()
            out.append((g.populations(), g.wall_force(0) if c.track_wall_force else None))
        return out
    finally:
        for g in grids:
            g.close()


PLAN = [("batch", 4), ("batch", 5), ("member", 2), ("batch", 2)]   # 13 steps


@pytest.mark.parametrize("storage", [A.LBM_STORE_F32, A.LBM_STORE_F16, A.LBM_STORE_BF16])
def test_packed_batch_matches_domains_stepped_alone(storage):
    """One packed launch set for all members.  Each member ends bit for bit
    where it ends as a batch of its own (the same kernel; graph pairs, a
    trailing odd step and member steps in between), and within the FP32 field
    bar of the member stepped by lbm_update_all_grids, whose paired kernel
    takes the descriptor as a kernel parameter and may contract differently."""
    cases = packed_cases(storage)
    together = _run_packed(cases, PLAN)
    for c, (f, force) in zip(cases, together):
        (fa, forcea), = _run_packed([c], PLAN)
        np.testing.assert_array_equal(f, fa)
        if force is not None:
            np.testing.assert_allclose(force, forcea, rtol=1e-12, atol=1e-12 * np.abs(force).max())
        with L.build_grids(c) as g:
            g.update_all_grids(13)
            ref = g.populations()
            tol = FIELD_REL_L2 if storage == A.LBM_STORE_F32 else 1e-3
            assert rel_l2(f, ref) < tol
            if force is not None:
                fr = g.wall_force(0)
                assert np.abs(force - fr).max() <= 1e-4 * np.abs(fr).max()
    info_grids = [L.build_grids(c) for c in cases]
    with L.PackedBatch(info_grids) as b:
        info = b.info()
        assert info.domain_count == 3 and info.launches_per_step == 3
        assert info.cells == sum(g.info(0).cell_count for g in info_grids)
    for g in info_grids:
        g.close()


def test_packed_batch_requires_one_parity_and_plain_members():
    c = packed_cases(A.LBM_STORE_F32)
    grids = [L.build_grids(c[0]), L.build_grids(c[2])]
    try:
        grids[1].update_all_grids(1)
        with L.PackedBatch(grids) as b:
            with pytest.raises(A.LbmError):
                b.update(2)
            grids[0].update_all_grids(1)
            b.update(2)
        f16 = L.build_grids(packed_cases(A.LBM_STORE_F16)[2])
        with pytest.raises(A.LbmError):
            L.PackedBatch([grids[0], f16])
        f16.close()
        r = L.periodic_box(24, 24, 24, nu_lattice=0.02)
        G.set_rotors(r, [(G.rotor(hub_radius=2, tip_radius=7, chord=3, thickness=1.0, hub_length=4),
                          dict(axis=2, origin=(0, 0, 0), radians_per_second=2.0))])
        with L.build_grids(r) as rg:
            with pytest.raises(A.LbmError):
                L.PackedBatch([grids[0], rg])
        with pytest.raises(A.LbmError):
            L.PackedBatch([grids[0], grids[0]])
    finally:
        for g in grids:
            g.close()
