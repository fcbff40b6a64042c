"""Checkpoint and resume: a run resumed from a saved state, in the same or in
freshly built grids, continues exactly as the uninterrupted run."""
import numpy as np
import pytest

import lbm3_b200 as L
from lbm3_b200 import _abi as A
from lbm3_b200 import geometry as G

pytestmark = pytest.mark.gpu


def full_case(storage=A.LBM_STORE_F32):
    c = L.open_channel(48, 24, 24, u_in=0.04, nu_lattice=0.02, storage=storage)
    G.set_bodies(c, [G.icosphere(2, 3.0, (30.0, 12.0, 12.0))])
    c.track_wall_force = 1
    G.set_rotors(c, [(G.rotor(hub_radius=2, tip_radius=6, chord=3, thickness=1.0, hub_length=4,
                              center=(14.0, 12.0, 12.0)),
                      dict(axis=2, origin=(14.0, 12.0, 12.0), radians_per_second=3.0))])
    c.track_rotor_force = 1
    return c


def snapshot(g):
    return dict(macro=g.macro(), wall=g.wall_force_raw(), ref=g.open_reference(), cum=g.open_cumulative(),
                bins=g.rotor_bins(0), angle=g.rotor_info(0).radians_elapsed, it=g.info().iterations_finished)


def check_same(a, b):
    for k in ("macro", "wall", "ref", "cum"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    assert np.allclose(a["bins"], b["bins"], rtol=1e-5, atol=1e-7)
    assert a["angle"] == b["angle"] and a["it"] == b["it"]


@pytest.mark.parametrize("storage", [A.LBM_STORE_F32, A.LBM_STORE_F16])
def test_resume_matches_uninterrupted_run(storage):
    c = full_case(storage)
    with L.build_grids(c) as g:
        g.update_all_grids(10)
        state = g.save_state()
        g.update_all_grids(15)
        ref = snapshot(g)
        # rewind the same grids
        g.load_state(state)
        g.update_all_grids(15)
        check_same(ref, snapshot(g))
    # resume in grids built afresh from the same case
    with L.build_grids(full_case(storage)) as h:
        h.update_all_grids(3)  # state that the load replaces
        h.load_state(state)
        h.update_all_grids(15)
        check_same(ref, snapshot(h))


def test_state_of_another_case_is_rejected():
    with L.build_grids(full_case()) as g:
        state = g.save_state()
    other = L.open_channel(40, 24, 24)
    with L.build_grids(other) as h:
        with pytest.raises(A.LbmError):
            h.load_state(state)
        with pytest.raises(A.LbmError):
            h.load_state(b"\0" * 64)
