"""The kinetic energy without device allocation, for callers that cannot
allocate (a serving loop whose HBM is committed by footprint admission),
checked through the C ABI against the allocating path.  Collected last so a
run that stops at the first failure has already run every other test."""
import ctypes as C

import pytest

import lbm3_b200 as L
from lbm3_b200 import _abi as A

pytestmark = pytest.mark.gpu

# relative tolerance of the kinetic-energy tests
ENERGY_REL = 1e-6


def _energies(g, setup):
    lib = A.lib()
    ref, new = C.c_double(), C.c_double()
    A.check(lib.lbm_kinetic_energy(g.handle, setup.u_initial_phys, setup.domain_length, C.byref(ref)))
    A.check(lib.lbm_kinetic_energy_noalloc(g.handle, setup.u_initial_phys, setup.domain_length, C.byref(new)))
    return ref.value, new.value


@pytest.mark.parametrize("storage", [A.LBM_STORE_F32, A.LBM_STORE_F16])
def test_noalloc_energy_matches_allocating_path(storage):
    s = L.tgv_plain_method(storage=storage)
    with L.build_grids(s.case) as g:
        g.update_all_grids(5)
        # two calls in a row on the same state, then one more after further steps
        for _ in range(2):
            ref, new = _energies(g, s)
            assert ref > 0
            assert abs(new - ref) <= ENERGY_REL * ref, (new, ref)
        g.update_all_grids(5)
        ref, new = _energies(g, s)
        assert abs(new - ref) <= ENERGY_REL * ref, (new, ref)


def test_noalloc_energy_rejects_grids_beyond_its_scratch():
    # 4,194,304 cells is the limit; 254 x 126 x 128 active cells plus ghost
    # layers (256 x 128 x 130 = 4,259,840) exceed it
    c = L.periodic_box(254, 126, 128, nu_lattice=0.01, ux=0.01)
    with L.build_grids(c) as g:
        assert g.info().cell_count > 4194304
        out = C.c_double()
        rc = A.lib().lbm_kinetic_energy_noalloc(g.handle, 1.0, 1000.0, C.byref(out))
        assert rc == A.LBM_ERR_INVALID
        assert b"static scratch" in A.lib().lbm_last_error()
