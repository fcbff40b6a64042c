"""The C-ABI library loads and exports every entry point include/lbm3_b200.h declares."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

from lbm3_b200 import _abi as A

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "lbm3_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*[A-Za-z_][\w\s\*]*?\b(lbm_\w+)\s*\(", text, flags=re.M)))


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 15
    lib = A.lib()
    for n in names:
        assert hasattr(lib, n), n
    assert {s[0] for s in A.SIGNATURES} == set(names)


def test_struct_layouts_match_the_header(tmp_path):
    src = tmp_path / "sizes.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "lbm3_b200.h"\n'
                   'int main(void){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(lbm_case), sizeof(lbm_face_bc),'
                   ' sizeof(lbm_grid_info), offsetof(lbm_case, storage), offsetof(lbm_grid_info, grid_memory_bytes),'
                   ' offsetof(lbm_case, track_rotor_force), sizeof(lbm_rotor), sizeof(lbm_rotor_info),'
                   ' sizeof(lbm_batch_info), offsetof(lbm_batch_info, collide_items));'
                   'return 0;}\n')
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    assert int(out[0]) == C.sizeof(A.LbmCase)
    assert int(out[1]) == C.sizeof(A.LbmFaceBC)
    assert int(out[2]) == C.sizeof(A.LbmGridInfo)
    assert int(out[3]) == A.LbmCase.storage.offset
    assert int(out[4]) == A.LbmGridInfo.grid_memory_bytes.offset
    assert int(out[5]) == A.LbmCase.track_rotor_force.offset
    assert int(out[6]) == C.sizeof(A.LbmRotor)
    assert int(out[7]) == C.sizeof(A.LbmRotorInfo)
    assert int(out[8]) == C.sizeof(A.LbmBatchInfo)
    assert int(out[9]) == A.LbmBatchInfo.collide_items.offset


def test_null_arguments_are_rejected_without_a_device():
    lib = A.lib()
    assert lib.lbm_plan_grids(None, None, None) == A.LBM_ERR_INVALID
    assert b"null" in lib.lbm_last_error()
    assert lib.lbm_update_all_grids(None, 1) == A.LBM_ERR_INVALID
    assert lib.lbm_read_array(None, 0, 0, None, 0) == A.LBM_ERR_INVALID
    assert lib.lbm_update_batch(None, 1, 1) == A.LBM_ERR_INVALID
    out = (C.c_double * 7)()
    assert lib.lbm_flow_report(None, 0, 0.0, None, out) == A.LBM_ERR_INVALID
    assert lib.lbm_rotor_force(None, 0, 0, out) == A.LBM_ERR_INVALID
    assert lib.lbm_set_rotor_speed(None, 0, 1.0) == A.LBM_ERR_INVALID
    assert lib.lbm_open_boundary_flow(None, 0, 0, out) == A.LBM_ERR_INVALID
    n = C.c_size_t()
    assert lib.lbm_state_bytes(None, C.byref(n)) == A.LBM_ERR_INVALID
    assert lib.lbm_save_state(None, None, 0) == A.LBM_ERR_INVALID
    assert lib.lbm_load_state(None, None, 0) == A.LBM_ERR_INVALID
    assert lib.lbm_kinetic_energy_noalloc(None, 1.0, 1.0, out) == A.LBM_ERR_INVALID
    h = C.c_void_p()
    assert lib.lbm_batch_create(None, 1, C.byref(h)) == A.LBM_ERR_INVALID
    arr = (C.c_void_p * 2)(None, None)
    assert lib.lbm_batch_create(arr, 2, C.byref(h)) == A.LBM_ERR_INVALID and not h.value
    assert lib.lbm_batch_update(None, 1) == A.LBM_ERR_INVALID
    ms = C.c_float()
    assert lib.lbm_batch_time_steps(None, 1, C.byref(ms)) == A.LBM_ERR_INVALID
    info = A.LbmBatchInfo()
    assert lib.lbm_batch_get_info(None, C.byref(info)) == A.LBM_ERR_INVALID
    lib.lbm_batch_free(None)


def test_plan_rotor_queries_on_the_host():
    import lbm3_b200 as L
    from lbm3_b200 import geometry as G
    c = L.periodic_box(24, 24, 16, nu_lattice=0.02)
    G.set_rotors(c, [(G.rotor(hub_radius=2, tip_radius=7, chord=3, thickness=1.0, hub_length=4),
                      dict(axis=2, origin=(0.0, 0.0, 0.0), radians_per_second=2.0))])
    p = L.Plan(c)
    assert p.rotor_count() == 1
    info = A.LbmRotorInfo()
    assert A.lib().lbm_plan_rotor_info(p._h, 0, 1, C.byref(info)) == A.LBM_ERR_INVALID
    # the force bins live on the device only
    buf = (C.c_uint * 4)()
    assert A.lib().lbm_plan_read_array(p._h, 0, A.ARRAY_ROTOR_BASE + 3, buf, 16) == A.LBM_ERR_INVALID


def test_build_without_device_fails_loudly():
    lib = A.lib()
    if lib.lbm_device_count() > 0:
        pytest.skip("a CUDA device is visible")
    import lbm3_b200 as L
    with pytest.raises(A.LbmError) as e:
        L.build_grids(L.tgv_plain_method().case)
    assert e.value.code == A.LBM_ERR_NO_DEVICE
