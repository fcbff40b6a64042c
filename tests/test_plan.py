"""Host grid construction of the product vs the oracle: tables must match bit for bit."""
import numpy as np
import pytest

import lbm3_b200 as L
from lbm3_b200 import _abi as A
import oracle as O

PAIRS = [
    ("shifter", "shifter"), ("row_i", "rowI"), ("row_j", "rowJ"), ("row_k", "rowK"),
    ("row_jplus", "rowJP"), ("row_kplus", "rowKP"), ("row_jkplus", "rowJKP"),
    ("wall_map", "wallMap"), ("periodic_index", "perIndex"), ("periodic_source", "perSource"),
]


def _cases():
    yield "tgv64", L.tgv_plain_method().case
    yield "box10x8x6", L.periodic_box(10, 8, 6)
    yield "box2x2x2", L.periodic_box(2, 2, 2)


@pytest.mark.parametrize("name,case", list(_cases()))
def test_plan_tables_match_oracle(name, case):
    p = L.Plan(case)
    g = O.OracleGrid(case)
    info = p.info()
    assert info.cell_count == g.cell_count
    assert (info.cell_count_x, info.cell_count_y, info.cell_count_z) == (g.g.nx, g.g.ny, g.g.nz)
    assert info.row_count == g.g.rowCount
    assert np.float32(info.nu) == np.float32(g.g.nu)
    assert np.float32(info.ox) == np.float32(g.g.ox)
    for ours, theirs in PAIRS:
        a, b = p.array(ours), g.int_array(theirs)
        assert a.shape == b.shape, ours
        assert np.array_equal(a, b), ours
    assert p.fluid_updates_per_iteration == g.g.fluidUpdates
    g.close()
    p.close()


def test_plan_counts_for_a_periodic_box():
    p = L.Plan(L.periodic_box(10, 8, 6))
    i = p.info()
    nx, ny, nz = 12, 10, 8
    assert i.cell_count == nx * ny * nz
    assert i.periodic_count == nx * ny * nz - (nx - 2) * (ny - 2) * (nz - 2)
    assert i.row_count == ny * nz          # one compressed row per i-line
    assert i.wall_cell_count == 0
    wm = p.array("wall_map")
    assert (wm == -2).sum() == i.periodic_count and (wm == -1).sum() == (nx - 2) * (ny - 2) * (nz - 2)
    # every periodic source is an interior cell
    src = p.array("periodic_source")
    assert np.all(wm[src] == -1)


def test_plan_reports_storage_footprint():
    c32 = L.tgv_plain_method().case
    c16 = L.tgv_plain_method(storage=A.LBM_STORE_F16).case
    b32 = L.Plan(c32).info().grid_memory_bytes
    b16 = L.Plan(c16).info().grid_memory_bytes
    n = L.Plan(c32).info().cell_count
    # population planes are padded to an odd number of 128-byte lines
    extra = (b32 - b16) - 27 * n * 2
    assert abs(extra) <= 27 * 256, extra


@pytest.mark.parametrize("mutate,code", [
    (lambda c: setattr(c, "grid_level_count", 5), A.LBM_ERR_BUILD),
    (lambda c: setattr(c, "grid_level_count", 0), A.LBM_ERR_BUILD),
    (lambda c: setattr(c, "wall_refinement_count", -1), A.LBM_ERR_BUILD),
    (lambda c: c.bounds.__setitem__(3, c.bounds[0] - 1.0), A.LBM_ERR_BUILD),
    (lambda c: setattr(c.face[0], "kind", 7), A.LBM_ERR_BUILD),
    (lambda c: setattr(c, "res_global", 0.0), A.LBM_ERR_BUILD),
    (lambda c: setattr(c, "storage", 9), A.LBM_ERR_BUILD),
    (lambda c: setattr(c, "open_bc_scheme", 2), A.LBM_ERR_BUILD),
    (lambda c: (setattr(c, "open_bc_scheme", A.LBM_OPEN_IMPEDANCE),
                setattr(c, "rho_reflection_tolerance", -1e-5)), A.LBM_ERR_BUILD),
])
def test_plan_rejects_invalid_cases(mutate, code):
    c = L.tgv_plain_method().case
    mutate(c)
    with pytest.raises(A.LbmError) as e:
        L.Plan(c)
    assert e.value.code == code
    assert str(e.value)
