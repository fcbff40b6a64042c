"""Bulk segments of the collide-stream kernels, checked on the host: a
segment may run across consecutive rows of a dense block, but each lane must
keep the per-cell neighbours, no lane may need the wrapped +1 neighbour, and
every non-solid cell is collided exactly once."""
import ctypes as C
import subprocess
from pathlib import Path

import pytest

import lbm3_b200 as L
from lbm3_b200 import build as B
from lbm3_b200 import geometry as G

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    B.build()
    out = tmp_path_factory.mktemp("seg") / "segment_check.so"
    objs = [str(B.OBJ_DIR / "builder.o"), str(B.OBJ_DIR / "geometry.o")]
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I/usr/local/cuda/include",
                    str(ROOT / "tests" / "drivers" / "segment_check.cpp"), *objs, "-o", str(out)], check=True)
    lib = C.CDLL(str(out))
    lib.lbm_segment_check.argtypes = [C.c_void_p, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
    return lib


def _cases():
    yield "box26x18x12", L.periodic_box(24, 16, 10, nu_lattice=0.004, ux=0.04), 128
    yield "tgv66", L.tgv_plain_method().case, 128
    yield "channel", L.open_channel(32, 16, 12), 128
    sphere = L.open_channel(48, 24, 24)
    G.set_bodies(sphere, [G.icosphere(3, 4.0, (16.0, 12.0, 12.0))])
    yield "sphere", sphere, None
    yield "refined", L.taylor_green_refined(32).case, None


@pytest.mark.parametrize("name,case,longest", list(_cases()))
def test_segments_keep_neighbours_and_cover_every_cell(checker, name, case, longest):
    segs, top = C.c_longlong(), C.c_longlong()
    assert checker.lbm_segment_check(C.byref(case), C.byref(segs), C.byref(top)) == 0
    assert segs.value > 0
    if longest is not None:  # dense blocks of short rows fill whole tiles
        assert top.value == longest
