"""Per-cell driver hooks (getOpenBC, getInitialCondition, getLocalBC as
lbm_case callbacks): a hook that restates the face table builds the same
tables; a spatially varying hook is honoured identically by the product's
builder and the oracle; the reference-style C++ driver headers compile."""
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

import lbm3_b200 as L
import oracle as O
from lbm3_b200 import _abi as A
from lbm3_b200 import geometry as G

from test_setup_parity import assert_same_tables
from test_walls import couette_case

ROOT = Path(__file__).resolve().parents[1]


def face_hook_for(case):
    """A getOpenBC hook restating a case's face table."""
    faces = [case.face[f] for f in range(6)]

    def hook(bc, i, j, k, info):
        touch = [i == 0, i == info.cell_count_x - 1, j == 0, j == info.cell_count_y - 1,
                 k == 0, k == info.cell_count_z - 1]
        best = -1
        for f in range(6):
            if touch[f] and (best < 0 or faces[f].priority > faces[best].priority):
                best = f
        if best < 0:
            return
        fb = faces[best]
        bc.openBCID = fb.open_bc_id
        bc.nonReflective = fb.non_reflective
        bc.nonReflectiveBeta = fb.non_reflective_beta
        if fb.kind == A.LBM_BC_PERIODIC:
            bc.periodic = 1
        elif fb.kind == A.LBM_BC_VELOCITY:
            bc.dirichletU = 1
            bc.ux, bc.uy, bc.uz = fb.ux, fb.uy, fb.uz
        else:
            bc.dirichletRho = 1
            bc.dRho = fb.dRho
    return hook


def test_default_bc_is_the_reference_default():
    bc = A.LbmBC()
    A.lib().lbm_default_bc(bc)
    assert bc.wallID == -1 and bc.useIBB == 1 and bc.nonReflective == 1
    assert bc.nonReflectiveBeta == 7.0 and bc.nuMultiplier == 1.0
    assert bc.collisionLimiter == pytest.approx(0.05)


def test_open_bc_hook_restating_the_faces_builds_the_same_grid():
    c = L.open_channel(32, 16, 16, u_in=0.04, nu_lattice=0.02)
    G.set_bodies(c, [G.icosphere(2, 3.0, (12.0, 8.0, 8.0))])
    ref = L.Plan(c)
    hooked = L.open_channel(32, 16, 16, u_in=0.04, nu_lattice=0.02)
    G.set_bodies(hooked, [G.icosphere(2, 3.0, (12.0, 8.0, 8.0))])
    L.set_hooks(hooked, open_bc=face_hook_for(c))
    p = L.Plan(hooked)
    for name in ("shifter", "wall_map", "open_index", "periodic_index"):
        np.testing.assert_array_equal(p.array(name), ref.array(name))
    p.close()
    ref.close()
    assert_same_tables(hooked)


def test_varying_inlet_and_wall_velocity_hooks_match_the_oracle():
    """A parabolic inlet profile from getOpenBC and a rotating wall from
    getLocalBC: product builder and oracle agree table for table."""
    c = couette_case()

    def local(bc, i, j, k, info):
        if bc.wallID == 0:
            x = i * info.res + info.ox
            y = j * info.res + info.oy
            s = 10.0 * info.dt_phys / info.res
            bc.ux, bc.uy = -s * y, s * x

    L.set_hooks(c, local_bc=local)
    p = L.Plan(c)
    wv = p.wall_velocity().reshape(3, -1)
    assert np.abs(wv).max() > 0
    p.close()
    assert_same_tables(c)

    ch = L.open_channel(32, 16, 16, u_in=0.04, nu_lattice=0.02)
    base = face_hook_for(ch)

    def inlet(bc, i, j, k, info):
        base(bc, i, j, k, info)
        if bc.dirichletU and i == 0:
            yy = (j + 0.5) / info.cell_count_y
            zz = (k + 0.5) / info.cell_count_z
            bc.ux = 0.04 * 16.0 * yy * (1 - yy) * zz * (1 - zz)

    L.set_hooks(ch, open_bc=inlet)
    assert_same_tables(ch)


def test_initial_condition_hook_equals_the_built_in_taylor_green():
    s = L.tgv_plain_method()
    ref = O.OracleGrid(s.case)
    c = L.tgv_plain_method().case
    u0, length = c.tgv_u0, c.tgv_length
    c.ic_kind = A.LBM_IC_UNIFORM
    f32 = np.float32

    def ic(bc, i, j, k, info):
        x = f32(f32(i) * f32(info.res) + f32(info.ox))
        y = f32(f32(j) * f32(info.res) + f32(info.oy))
        z = f32(f32(k) * f32(info.res) + f32(info.oz))
        X, Y, Z = f32(x / f32(length)), f32(y / f32(length)), f32(z / f32(length))
        u = f32(u0)
        bc.ux = f32(f32(f32(u * np.sin(X)) * np.cos(Y)) * np.cos(Z))
        bc.uy = f32(f32(f32(-u * np.cos(X)) * np.sin(Y)) * np.cos(Z))
        bc.uz = 0.0
        bc.dRho = f32(f32(f32(f32(3.0) * u * u / f32(16.0)) * f32(np.cos(f32(2) * X) + np.cos(f32(2) * Y)))
                      * f32(f32(2.0) + np.cos(f32(2) * Z)))

    L.set_hooks(c, initial_condition=ic)
    hooked = O.OracleGrid(c)
    # float32 numpy sin/cos may differ from the C library in the last bit
    assert np.abs(hooked.populations() - ref.populations()).max() < 1e-8
    hooked.close()
    ref.close()


def nvcc():
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    cand = Path(cuda) / "bin" / "nvcc"
    return str(cand) if cand.exists() else "nvcc"


def build_driver(out: Path, levels: int = 1) -> Path:
    lib = ROOT / "lbm3_b200" / "_lib"
    exe = out / f"tgv_driver_{levels}"
    subprocess.run([nvcc(), "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", f"-DTGV_LEVELS={levels}",
                    "-I", str(ROOT / "include"), str(ROOT / "tests" / "drivers" / "tgv_driver.cu"),
                    "-L", str(lib), "-llbm3_b200", "-Xlinker", "-rpath", "-Xlinker", str(lib), "-o", str(exe)],
                   check=True)
    return exe


@pytest.mark.parametrize("levels", [1, 2])
def test_reference_style_driver_compiles(tmp_path, levels):
    exe = build_driver(tmp_path, levels)
    assert exe.exists()
