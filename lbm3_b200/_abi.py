"""ctypes view of the C ABI declared in ``include/lbm3_b200.h``.

The shared library is built in-tree (``lbm3_b200/_lib/liblbm3_b200.so``) by
``lbm3_b200.build``.  Loading fails loudly when it is missing: there is no
CPU or Python fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "liblbm3_b200.so"

# status codes
LBM_OK = 0
LBM_ERR_INVALID = -1
LBM_ERR_CUDA = -2
LBM_ERR_OOM = -3
LBM_ERR_BUILD = -4
LBM_ERR_UNSUPPORTED = -5
LBM_ERR_NO_DEVICE = -6

# boundary kinds
LBM_BC_PERIODIC = 0
LBM_BC_VELOCITY = 1
LBM_BC_PRESSURE = 2

# faces
FACE_XMIN, FACE_XMAX, FACE_YMIN, FACE_YMAX, FACE_ZMIN, FACE_ZMAX = range(6)

# initial conditions
LBM_IC_UNIFORM = 0
LBM_IC_TAYLOR_GREEN = 1

# storage
LBM_STORE_F32 = 0
LBM_STORE_F16 = 1
LBM_STORE_BF16 = 2
LBM_STORE_F64 = 3
LBM_OPEN_CHARACTERISTIC = 0
LBM_OPEN_IMPEDANCE = 1
STORAGE_NAMES = {LBM_STORE_F32: "f32", LBM_STORE_F16: "f16", LBM_STORE_BF16: "bf16", LBM_STORE_F64: "f64"}

# arrays
ARRAY_F = 0
ARRAY_SHIFTER = 1
ARRAY_ROW_I = 2
ARRAY_ROW_J = 3
ARRAY_ROW_K = 4
ARRAY_ROW_JPLUS = 5
ARRAY_ROW_KPLUS = 6
ARRAY_ROW_JKPLUS = 7
ARRAY_WALL_MAP = 8
ARRAY_PERIODIC_INDEX = 9
ARRAY_PERIODIC_SOURCE = 10
ARRAY_MACRO = 11


class LbmFaceBC(C.Structure):
    _fields_ = [
        ("kind", C.c_int), ("open_bc_id", C.c_int), ("priority", C.c_int),
        ("non_reflective", C.c_int), ("non_reflective_beta", C.c_float),
        ("dRho", C.c_float), ("ux", C.c_float), ("uy", C.c_float), ("uz", C.c_float),
    ]


LBM_WALL_STATIC = 0
LBM_WALL_ROTATING = 1
LBM_MAX_BODIES = 16
ARRAY_WALL_INDEX = 12
ARRAY_WALL_DATA = 13
ARRAY_LINK_LENGTH = 14
ARRAY_WALL_FORCE = 15
ARRAY_WALL_VELOCITY = 16
ARRAY_OPEN_INDEX = 17
ARRAY_OPEN_SOURCE = 18
ARRAY_OPEN_REFERENCE = 19
ARRAY_OPEN_CUMULATIVE = 20
ARRAY_F2C_INDEX = 21
ARRAY_F2C_CHILD = 22
ARRAY_C2F_INDEX = 23
ARRAY_C2F_CHILD = 24
ARRAY_LEFTOVER_INDEX = 25
ARRAY_LEFTOVER_PARENT = 26
ARRAY_LEFTOVER_NBR = 27
LBM_MAX_LEVELS = 4
LBM_ERR_DEVICE_WAIT = -7


class LbmBody(C.Structure):
    _fields_ = [
        ("triangles", C.POINTER(C.c_float)), ("triangle_count", C.c_int), ("motion", C.c_int),
        ("axis", C.c_int), ("origin", C.c_float * 3), ("radians_per_second", C.c_float),
    ]


LBM_MAX_ROTORS = 4
ARRAY_ROTOR_BASE = 32
PLANE_XY, PLANE_ZY, PLANE_ZX = 0, 1, 2


class LbmRotor(C.Structure):
    _fields_ = [
        ("triangles", C.POINTER(C.c_float)), ("triangle_count", C.c_int), ("axis", C.c_int),
        ("origin", C.c_float * 3), ("radians_per_second", C.c_float),
    ]


class LbmRotorInfo(C.Structure):
    _fields_ = [
        ("res", C.c_float), ("bounds", C.c_float * 6), ("cell_count", C.c_int * 3), ("block_count", C.c_int),
        ("nonzero_block_count", C.c_int), ("axis", C.c_int), ("origin", C.c_float * 3),
        ("radians_per_second", C.c_float), ("radians_elapsed", C.c_double),
    ]


class LbmCase(C.Structure):
    _fields_ = [
        ("grid_level_count", C.c_int), ("wall_refinement_count", C.c_int),
        ("res_global", C.c_float), ("nu_phys", C.c_float), ("rho_phys", C.c_float),
        ("dt_phys_global", C.c_float), ("bounds", C.c_float * 6),
        ("track_wall_force", C.c_int), ("track_open_boundaries", C.c_int),
        ("face", LbmFaceBC * 6),
        ("ic_kind", C.c_int), ("ic_dRho", C.c_float), ("ic_ux", C.c_float),
        ("ic_uy", C.c_float), ("ic_uz", C.c_float),
        ("tgv_u0", C.c_float), ("tgv_length", C.c_float),
        ("collision_limiter", C.c_float), ("nu_multiplier", C.c_float),
        ("gx", C.c_float), ("gy", C.c_float), ("gz", C.c_float), ("use_ibb", C.c_int),
        ("body_count", C.c_int), ("body", LbmBody * LBM_MAX_BODIES),
        ("storage", C.c_int),
        ("rotor_count", C.c_int), ("rotor", LbmRotor * LBM_MAX_ROTORS), ("track_rotor_force", C.c_int),
        ("open_bc_hook", C.c_void_p), ("initial_condition_hook", C.c_void_p), ("local_bc_hook", C.c_void_p),
        ("hook_user", C.c_void_p),
        ("refine_box", (C.c_float * 6) * LBM_MAX_LEVELS), ("refinement_hook", C.c_void_p),
        ("open_bc_scheme", C.c_int), ("rho_reflection_tolerance", C.c_float),
    ]


class LbmBatchInfo(C.Structure):
    _fields_ = [
        ("domain_count", C.c_int), ("cells", C.c_longlong), ("collide_items", C.c_int),
        ("open_chunks", C.c_int), ("periodic_cells", C.c_int), ("launches_per_step", C.c_int),
    ]


class LbmBC(C.Structure):
    """lbm_bc: BCStruct as a per-cell hook fills it."""
    _fields_ = [
        ("dRho", C.c_float), ("ux", C.c_float), ("uy", C.c_float), ("uz", C.c_float),
        ("gx", C.c_float), ("gy", C.c_float), ("gz", C.c_float),
        ("wallID", C.c_int), ("openBCID", C.c_int),
        ("useIBB", C.c_int), ("dirichletU", C.c_int), ("dirichletRho", C.c_int),
        ("periodic", C.c_int), ("nonReflective", C.c_int),
        ("nonReflectiveBeta", C.c_float), ("collisionLimiter", C.c_float), ("nuMultiplier", C.c_float),
    ]


class LbmGridInfo(C.Structure):
    _fields_ = [
        ("grid_id", C.c_int), ("cell_count", C.c_int), ("cell_count_x", C.c_int),
        ("cell_count_y", C.c_int), ("cell_count_z", C.c_int), ("row_count", C.c_int),
        ("wall_cell_count", C.c_int), ("wall_adjacent_count", C.c_int),
        ("periodic_count", C.c_int), ("open_bc_count", C.c_int),
        ("esotwist_flipper", C.c_int), ("iterations_finished", C.c_int), ("storage", C.c_int),
        ("res", C.c_float), ("ox", C.c_float), ("oy", C.c_float), ("oz", C.c_float),
        ("nu", C.c_float), ("dt_phys", C.c_float), ("grid_memory_bytes", C.c_ulonglong),
        ("f2c_count", C.c_int), ("c2f_count", C.c_int), ("leftover_count", C.c_int),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


# lbm_cell_hook: void (*)(void* user, lbm_bc* bc, int i, int j, int k, const lbm_grid_info* info)
CELL_HOOK = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(LbmBC), C.c_int, C.c_int, C.c_int, C.POINTER(LbmGridInfo))
# lbm_refinement_hook: void (*)(void* user, int i, int j, int k, int* mark, const lbm_grid_info* info)
REFINEMENT_HOOK = C.CFUNCTYPE(None, C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int),
                              C.POINTER(LbmGridInfo))

# (name, restype, argtypes) of every exported function
_P = C.c_void_p
SIGNATURES = [
    ("lbm_last_error", C.c_char_p, []),
    ("lbm_device_count", C.c_int, []),
    ("lbm_default_bc", None, [C.POINTER(LbmBC)]),
    ("lbm_plan_grids", C.c_int, [C.POINTER(LbmCase), C.POINTER(_P), C.POINTER(C.c_longlong)]),
    ("lbm_free_plan", None, [_P]),
    ("lbm_plan_level_count", C.c_int, [_P]),
    ("lbm_plan_info", C.c_int, [_P, C.c_int, C.POINTER(LbmGridInfo)]),
    ("lbm_plan_read_array", C.c_int, [_P, C.c_int, C.c_int, _P, C.c_size_t]),
    ("lbm_build_grids", C.c_int, [C.POINTER(LbmCase), C.POINTER(_P), C.POINTER(C.c_longlong)]),
    ("lbm_free_grids", None, [_P]),
    ("lbm_set_stream", C.c_int, [_P, _P]),
    ("lbm_update_all_grids", C.c_int, [_P, C.c_int]),
    ("lbm_update_batch", C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.c_int]),
    ("lbm_batch_create", C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.POINTER(_P)]),
    ("lbm_batch_update", C.c_int, [_P, C.c_int]),
    ("lbm_batch_time_steps", C.c_int, [_P, C.c_int, C.POINTER(C.c_float)]),
    ("lbm_batch_get_info", C.c_int, [_P, C.POINTER(LbmBatchInfo)]),
    ("lbm_batch_free", None, [_P]),
    ("lbm_synchronize", C.c_int, [_P]),
    ("lbm_set_graphs", C.c_int, [_P, C.c_int]),
    ("lbm_time_steps_graph", C.c_int, [_P, C.c_int, C.POINTER(C.c_float)]),
    ("lbm_time_steps", C.c_int, [_P, C.c_int, C.POINTER(C.c_float)]),
    ("lbm_last_kernel_time", C.c_int, [_P, C.POINTER(C.c_float), C.POINTER(C.c_int)]),
    ("lbm_last_launch_count", C.c_int, [_P, C.POINTER(C.c_longlong)]),
    ("lbm_level_count", C.c_int, [_P]),
    ("lbm_get_grid_info", C.c_int, [_P, C.c_int, C.POINTER(LbmGridInfo)]),
    ("lbm_read_array", C.c_int, [_P, C.c_int, C.c_int, _P, C.c_size_t]),
    ("lbm_write_f", C.c_int, [_P, C.c_int, _P, C.c_size_t]),
    ("lbm_kinetic_energy", C.c_int, [_P, C.c_float, C.c_float, C.POINTER(C.c_double)]),
    ("lbm_kinetic_energy_noalloc", C.c_int, [_P, C.c_float, C.c_float, C.POINTER(C.c_double)]),
    ("lbm_global_sums", C.c_int, [_P, C.POINTER(C.c_double)]),
    ("lbm_wall_force", C.c_int, [_P, C.c_int, C.c_int, C.POINTER(C.c_double)]),
    ("lbm_open_boundary_flow", C.c_int, [_P, C.c_int, C.c_int, C.POINTER(C.c_double)]),
    ("lbm_plan_rotor_info", C.c_int, [_P, C.c_int, C.c_int, C.c_void_p]),
    ("lbm_get_rotor_info", C.c_int, [_P, C.c_int, C.c_int, C.c_void_p]),
    ("lbm_set_rotor_speed", C.c_int, [_P, C.c_int, C.c_float]),
    ("lbm_rotor_force", C.c_int, [_P, C.c_int, C.c_int, C.POINTER(C.c_double)]),
    ("lbm_flow_report", C.c_int, [_P, C.c_int, C.c_float, C.c_void_p, C.POINTER(C.c_double)]),
    ("lbm_export_vtk", C.c_int, [_P, C.c_char_p]),
    ("lbm_state_bytes", C.c_int, [_P, C.POINTER(C.c_size_t)]),
    ("lbm_save_state", C.c_int, [_P, C.c_void_p, C.c_size_t]),
    ("lbm_load_state", C.c_int, [_P, C.c_void_p, C.c_size_t]),
    ("lbm_apply_collision_batch", C.c_int,
     [_P, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, _P]),
]


class LbmError(RuntimeError):
    """A C-ABI call returned a negative status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code


_lib = None


def lib() -> C.CDLL:
    """Load the in-tree CUDA library (no fallback)."""
    global _lib
    if _lib is None:
        path = Path(os.environ.get("LBM3_B200_LIB", LIB_PATH))
        if not path.exists():
            raise ImportError(
                f"{path} is missing; build it with `python -m lbm3_b200.build` "
                "(the CUDA library is required, there is no fallback)")
        handle = C.CDLL(str(path))
        for name, res, args in SIGNATURES:
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def check(code: int) -> int:
    if code < 0:
        msg = lib().lbm_last_error()
        raise LbmError(code, msg.decode() if msg else "")
    return code
