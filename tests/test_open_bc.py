"""Moment-based open boundaries on the CPU: the oracle's closure against the
reference's generated code (golden vectors), the product plan's open lists
against the oracle's own construction, and the oracle's channel flow."""
import json
from pathlib import Path

import numpy as np
import pytest

import lbm3_b200 as L
from lbm3_b200 import _abi as A
from lbm3_b200 import geometry as G
import oracle as O
from helpers import plan_ijk

GOLDEN = Path(__file__).resolve().parent / "golden" / "mbbc_vectors.json"
CX = [0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, 0, 0, -1, 1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1]
CY = [0, 0, 0, 0, 0, -1, 1, 0, 0, 0, 0, -1, 1, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1, -1, 1]
CZ = [0, 0, 0, -1, 1, 0, 0, -1, 1, 1, -1, 0, 0, -1, 1, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, -1, 1]


def _cases():
    return json.loads(GOLDEN.read_text())["cases"]


def test_golden_covers_every_outer_normal():
    codes = {c["code"] for c in _cases()}
    want = {(nx + 5) * 100 + (ny + 5) * 10 + (nz + 5)
            for nx in (-1, 0, 1) for ny in (-1, 0, 1) for nz in (-1, 0, 1) if (nx, ny, nz) != (0, 0, 0)}
    assert codes == want


def test_mbbc_apply_bit_exact():
    """applyMBBC (include/boundaryConditions/applyMBBC.h) for all 26 normals."""
    for c in _cases():
        f = np.array(c["f"], dtype=np.float32)
        got = O.mbbc_apply(c["code"], c["rho"], c["u"], f)
        np.testing.assert_array_equal(got, np.array(c["f_out"], dtype=np.float32), err_msg=str(c["code"]))


def test_mbbc_restore_bit_exact():
    """restoreRho / restoreUxUyUz (include/boundaryConditions/restoreRho.h, restoreUxUyUz.h)."""
    for c in _cases():
        f = np.array(c["f"], dtype=np.float32)
        assert O.mbbc_restore_rho(c["code"], c["u"], f) == np.float32(c["rho_out"]), c["code"]
        np.testing.assert_array_equal(O.mbbc_restore_u(c["code"], c["rho"], f),
                                      np.array(c["u_out"], dtype=np.float32), err_msg=str(c["code"]))


def test_mbbc_reproduces_equilibrium():
    """Closing the unknowns of an equilibrium state with its own moments
    returns the equilibrium populations (every normal).  Restoring rho and u
    is exact on faces; on edges and corners the relations keep only the
    constant and linear parts of the equilibrium moments, so they are exact
    to O(|u|^2)."""
    rho, u = 1.01, (0.03, -0.02, 0.01)
    feq = O.feq(rho - 1.0, *u) + np.array([8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8, np.float32)
    for nx in (-1, 0, 1):
        for ny in (-1, 0, 1):
            for nz in (-1, 0, 1):
                if (nx, ny, nz) == (0, 0, 0):
                    continue
                code = (nx + 5) * 100 + (ny + 5) * 10 + (nz + 5)
                unknown = [d for d in range(27) if nx * CX[d] < 0 or ny * CY[d] < 0 or nz * CZ[d] < 0]
                f = feq.copy()
                f[unknown] = 0.0
                out = O.mbbc_apply(code, rho, u, f)
                np.testing.assert_allclose(out, feq, rtol=0, atol=2e-6, err_msg=str(code))
                tol = 1e-5 if abs(nx) + abs(ny) + abs(nz) == 1 else 2.0 * float(np.dot(u, u))
                assert abs(O.mbbc_restore_rho(code, u, f) - rho) < tol, code
                np.testing.assert_allclose(O.mbbc_restore_u(code, rho, f), u, atol=tol, err_msg=str(code))


def test_unknown_normal_code_rejected():
    with pytest.raises(ValueError):
        O.mbbc_apply(555, 1.0, (0, 0, 0), np.zeros(27, np.float32))


@pytest.mark.parametrize("sides", ["velocity", "periodic"])
def test_open_lists_match_oracle(sides):
    c = L.open_channel(32, 16, 12, sides=sides)
    p = L.Plan(c)
    info = p.info()
    idx = p.array("open_index")
    assert info.open_bc_count == len(idx) > 0
    o = O.OracleGrid(c)
    np.testing.assert_array_equal(o.open_index(), idx)
    o.close()
    # every open cell is a boundary cell with a valid interior source
    i, j, k = plan_ijk(p)
    on_face = (i[idx] == 0) | (i[idx] == 31) | (j[idx] == 0) | (j[idx] == 15) | (k[idx] == 0) | (k[idx] == 11)
    assert on_face.all()
    src = p.array("open_source")
    assert ((i[src] > 0) & (i[src] < 31) & (j[src] > 0) & (j[src] < 15) & (k[src] > 0) & (k[src] < 11)).all()


def test_open_lists_with_body_match_oracle():
    c = L.open_channel(40, 20, 20)
    G.set_bodies(c, [G.icosphere(2, 4.0, (14.0, 10.0, 10.0))])
    p = L.Plan(c)
    o = O.OracleGrid(c)
    np.testing.assert_array_equal(o.open_index(), p.array("open_index"))
    o.close()


def test_open_list_counts():
    # velocity sides own all edges and corners: every boundary cell is open
    c = L.open_channel(32, 16, 12)
    info = L.Plan(c).info()
    assert info.open_bc_count == 32 * 16 * 12 - 30 * 14 * 10
    assert info.periodic_count == 0
    # periodic sides of lower priority: the x faces own their rims and are
    # open entirely; the remaining side cells are periodic ghosts
    c = L.open_channel(32, 16, 12, sides="periodic")
    info = L.Plan(c).info()
    assert info.open_bc_count == 2 * 16 * 12
    assert info.periodic_count == 30 * (16 * 12 - 14 * 10)


def test_oracle_uniform_channel_flow_is_steady():
    """A uniform stream through velocity inlet, pressure outlet and velocity
    sides stays uniform (all populations at equilibrium)."""
    c = L.open_channel(24, 12, 12, u_in=0.04, nu_lattice=0.02)
    o = O.OracleGrid(c)
    o.step(100)
    m = o.macro()
    assert np.abs(m[1] - 0.04).max() < 5e-6
    assert np.abs(m[2:]).max() < 5e-6
    assert np.abs(m[0]).max() < 5e-6
    # reference values follow the state: inlet uNormal = -u_in, outlet +u_in
    ref = o.open_reference()
    idx = o.open_index()
    i = o.int_array("I")[idx]
    j = o.int_array("J")[idx]
    k = o.int_array("K")[idx]
    face = (j > 0) & (j < 11) & (k > 0) & (k < 11)
    assert np.allclose(ref[1][face & (i == 0)], -0.04, atol=1e-5)
    assert np.allclose(ref[1][face & (i == 23)], 0.04, atol=1e-5)
    # cumulative uNormal: 100 steps of the tracked normal velocity
    cum = o.open_cumulative()
    assert np.allclose(cum[1][face & (i == 23)], 4.0, rtol=1e-4)
    o.close()


def test_oracle_outlet_pressure_wave_leaves():
    """A density pulse reaches the non-reflective outlet and leaves; with a
    reflecting (strict) outlet more of it stays in the channel."""
    def residual(non_reflective):
        c = L.open_channel(48, 8, 8, u_in=0.02, nu_lattice=0.02, sides="periodic",
                           outlet_non_reflective=non_reflective)
        o = O.OracleGrid(c)
        f = o.populations()
        i = o.int_array("I")
        pulse = (i >= 30) & (i <= 34)
        w = np.array([8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8, np.float32)
        f[:, pulse] += 0.002 * w[:, None]  # slot order is irrelevant for an isotropic bump
        o.set_populations(f)
        o.step(120)
        m = o.macro()
        inner = (i > 2) & (i < 45)
        out = float(np.sqrt(np.mean(m[0][inner] ** 2)))
        o.close()
        return out
    assert residual(True) < residual(False)
