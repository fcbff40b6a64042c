"""Host-side mirror of the reference driver API over the C ABI.

``build_grids`` / ``Grids.update_all_grids`` correspond to the reference's
``buildGrids`` and ``updateAllGrids`` (include/gridBuilderFunctions.h:1577,
include/updateGrid.h:388); ``Plan`` exposes the host-only construction used
for footprint admission and table parity.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi as A

_INT_ARRAYS = {
    "shifter": A.ARRAY_SHIFTER, "row_i": A.ARRAY_ROW_I, "row_j": A.ARRAY_ROW_J,
    "row_k": A.ARRAY_ROW_K, "row_jplus": A.ARRAY_ROW_JPLUS, "row_kplus": A.ARRAY_ROW_KPLUS,
    "row_jkplus": A.ARRAY_ROW_JKPLUS, "wall_map": A.ARRAY_WALL_MAP,
    "periodic_index": A.ARRAY_PERIODIC_INDEX, "periodic_source": A.ARRAY_PERIODIC_SOURCE,
    "wall_index": A.ARRAY_WALL_INDEX, "open_index": A.ARRAY_OPEN_INDEX, "open_source": A.ARRAY_OPEN_SOURCE,
    # interfaces towards the next finer level, read on the coarse level
    "f2c_index": A.ARRAY_F2C_INDEX, "f2c_child": A.ARRAY_F2C_CHILD, "c2f_index": A.ARRAY_C2F_INDEX,
    "c2f_child": A.ARRAY_C2F_CHILD, "leftover_index": A.ARRAY_LEFTOVER_INDEX,
    "leftover_parent": A.ARRAY_LEFTOVER_PARENT, "leftover_nbr": A.ARRAY_LEFTOVER_NBR,
}
_UINT_ARRAYS = {"wall_data": A.ARRAY_WALL_DATA, "link_length": A.ARRAY_LINK_LENGTH}


def _int_len(info: A.LbmGridInfo, which: int) -> int:
    if which in (A.ARRAY_SHIFTER, A.ARRAY_WALL_MAP):
        return info.cell_count
    if which in (A.ARRAY_PERIODIC_INDEX, A.ARRAY_PERIODIC_SOURCE):
        return info.periodic_count
    if which in (A.ARRAY_WALL_INDEX, A.ARRAY_WALL_DATA):
        return info.wall_adjacent_count
    if which == A.ARRAY_LINK_LENGTH:
        return 7 * info.wall_adjacent_count
    if which in (A.ARRAY_OPEN_INDEX, A.ARRAY_OPEN_SOURCE):
        return info.open_bc_count
    if which in (A.ARRAY_F2C_INDEX, A.ARRAY_F2C_CHILD):
        return info.f2c_count
    if which in (A.ARRAY_C2F_INDEX, A.ARRAY_C2F_CHILD):
        return info.c2f_count
    if which in (A.ARRAY_LEFTOVER_INDEX, A.ARRAY_LEFTOVER_PARENT):
        return info.leftover_count
    if which == A.ARRAY_LEFTOVER_NBR:
        return 3 * info.leftover_count
    return info.row_count


class Plan:
    """Host-only grid construction (no GPU needed)."""

    def __init__(self, case: A.LbmCase):
        lib = A.lib()
        self._h = C.c_void_p()
        fu = C.c_longlong()
        A.check(lib.lbm_plan_grids(C.byref(case), C.byref(self._h), C.byref(fu)))
        self.fluid_updates_per_iteration = fu.value
        self.case = case

    def uint_array(self, name: str, level: int = 0) -> np.ndarray:
        which = _UINT_ARRAYS[name]
        n = _int_len(self.info(level), which)
        out = np.empty(n, dtype=np.uint32)
        A.check(A.lib().lbm_plan_read_array(self._h, level, which, out.ctypes.data_as(C.c_void_p), out.nbytes))
        return out

    def rotor_count(self, level: int = 0) -> int:
        n = 0
        while n < A.LBM_MAX_ROTORS:
            info = A.LbmRotorInfo()
            if A.lib().lbm_plan_rotor_info(self._h, level, n, C.byref(info)) != 0:
                break
            n += 1
        return n

    def rotor_info(self, r: int, level: int = 0) -> A.LbmRotorInfo:
        info = A.LbmRotorInfo()
        A.check(A.lib().lbm_plan_rotor_info(self._h, level, r, C.byref(info)))
        return info

    def rotor_array(self, r: int, part: str, level: int = 0) -> np.ndarray:
        """Rotor tables: part 'map' (int32 [blocks]), 'index' (int32 [nonzero]),
        'interpolation' (uint32 [64 * nonzero])."""
        info = self.rotor_info(r, level)
        which, n, dt = {"map": (0, info.block_count, np.int32), "index": (1, info.nonzero_block_count, np.int32),
                        "interpolation": (2, 64 * info.nonzero_block_count, np.uint32)}[part]
        out = np.empty(n, dtype=dt)
        A.check(A.lib().lbm_plan_read_array(self._h, level, A.ARRAY_ROTOR_BASE + 4 * r + which,
                                            out.ctypes.data_as(C.c_void_p), out.nbytes))
        return out

    def wall_velocity(self, level: int = 0) -> np.ndarray:
        """[3][wallCount] wall velocity of every wall-adjacent cell (lattice units)."""
        n = self.info(level).wall_adjacent_count
        out = np.empty((3, n), dtype=np.float32)
        A.check(A.lib().lbm_plan_read_array(self._h, level, A.ARRAY_WALL_VELOCITY,
                                            out.ctypes.data_as(C.c_void_p), out.nbytes))
        return out

    def close(self):
        if self._h:
            A.lib().lbm_free_plan(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def level_count(self) -> int:
        return A.check(A.lib().lbm_plan_level_count(self._h))

    def info(self, level: int = 0) -> A.LbmGridInfo:
        out = A.LbmGridInfo()
        A.check(A.lib().lbm_plan_info(self._h, level, C.byref(out)))
        return out

    def array(self, name: str, level: int = 0) -> np.ndarray:
        which = _INT_ARRAYS[name]
        n = _int_len(self.info(level), which)
        out = np.empty(n, dtype=np.int32)
        A.check(A.lib().lbm_plan_read_array(self._h, level, which,
                                            out.ctypes.data_as(C.c_void_p), out.nbytes))
        return out


class Grids:
    """All levels of one domain resident on the current CUDA device."""

    def __init__(self, case: A.LbmCase):
        lib = A.lib()
        self._h = C.c_void_p()
        fu = C.c_longlong()
        A.check(lib.lbm_build_grids(C.byref(case), C.byref(self._h), C.byref(fu)))
        self.fluid_updates_per_iteration = fu.value
        self.case = case

    # lifetime
    def close(self):
        if self._h:
            A.lib().lbm_free_grids(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    # stepping
    def set_stream(self, stream_ptr: int | None):
        A.check(A.lib().lbm_set_stream(self._h, C.c_void_p(stream_ptr or 0)))

    def update_all_grids(self, coarse_steps: int = 1):
        A.check(A.lib().lbm_update_all_grids(self._h, int(coarse_steps)))

    def synchronize(self):
        A.check(A.lib().lbm_synchronize(self._h))

    def time_steps(self, steps: int) -> float:
        """Run `steps` coarse steps bracketed by CUDA events; returns device ms."""
        ms = C.c_float()
        A.check(A.lib().lbm_time_steps(self._h, int(steps), C.byref(ms)))
        return ms.value

    def time_steps_graph(self, steps: int) -> float:
        """Run `steps` coarse steps as replayed CUDA graphs; returns device ms."""
        ms = C.c_float()
        A.check(A.lib().lbm_time_steps_graph(self._h, int(steps), C.byref(ms)))
        return ms.value

    def set_graphs(self, enabled: bool):
        A.check(A.lib().lbm_set_graphs(self._h, int(bool(enabled))))

    def last_launch_count(self) -> int:
        """Every kernel launch of the last time_steps call."""
        n = C.c_longlong()
        A.check(A.lib().lbm_last_launch_count(self._h, C.byref(n)))
        return n.value

    def last_kernel_time(self):
        """(summed ms, launch count) of the collide-stream launches of the last time_steps."""
        ms, n = C.c_float(), C.c_int()
        A.check(A.lib().lbm_last_kernel_time(self._h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    # inspection
    def level_count(self) -> int:
        return A.check(A.lib().lbm_level_count(self._h))

    def info(self, level: int = 0) -> A.LbmGridInfo:
        out = A.LbmGridInfo()
        A.check(A.lib().lbm_get_grid_info(self._h, level, C.byref(out)))
        return out

    def array(self, name: str, level: int = 0) -> np.ndarray:
        which = _INT_ARRAYS[name]
        n = _int_len(self.info(level), which)
        out = np.empty(n, dtype=np.int32)
        A.check(A.lib().lbm_read_array(self._h, level, which, out.ctypes.data_as(C.c_void_p), out.nbytes))
        return out

    def populations(self, level: int = 0) -> np.ndarray:
        """Raw slot array float32 [27][cellCount] (current esotwist slot order)."""
        n = self.info(level).cell_count
        out = np.empty((27, n), dtype=np.float32)
        A.check(A.lib().lbm_read_array(self._h, level, A.ARRAY_F, out.ctypes.data_as(C.c_void_p), out.nbytes))
        return out

    def set_populations(self, f: np.ndarray, level: int = 0):
        f = np.ascontiguousarray(f, dtype=np.float32)
        A.check(A.lib().lbm_write_f(self._h, level, f.ctypes.data_as(C.c_void_p), f.nbytes))

    def macro(self, level: int = 0) -> np.ndarray:
        """dRho, ux, uy, uz of every cell: float32 [4][cellCount]."""
        n = self.info(level).cell_count
        out = np.empty((4, n), dtype=np.float32)
        A.check(A.lib().lbm_read_array(self._h, level, A.ARRAY_MACRO, out.ctypes.data_as(C.c_void_p),
                                       out.nbytes))
        return out

    def kinetic_energy(self, u_ref_phys: float, domain_length: float) -> float:
        out = C.c_double()
        A.check(A.lib().lbm_kinetic_energy(self._h, u_ref_phys, domain_length, C.byref(out)))
        return out.value

    def global_sums(self) -> dict:
        """FP64 accumulators over the fluid cells: mass, mass deviation,
        momentum (SI), fluid cell count, and the lattice sums of rho and dRho."""
        out = (C.c_double * 8)()
        A.check(A.lib().lbm_global_sums(self._h, out))
        keys = ("mass", "mass_deviation", "momentum_x", "momentum_y", "momentum_z", "cells", "sum_rho",
                "sum_drho")
        return dict(zip(keys, out[:]))

    def wall_force(self, wall_id: int, reset: bool = False) -> np.ndarray:
        """{Fx, Fy, Fz [N], Tx, Ty, Tz [N m]} on a body, averaged since the last reset."""
        out = (C.c_double * 6)()
        A.check(A.lib().lbm_wall_force(self._h, wall_id, int(reset), out))
        return np.array(out[:])

    def flow_report(self, plane: int, cut: float, bounds=None) -> dict:
        """getFlowReportXY/ZY/ZX: flow through the layer nearest to `cut` (mm)."""
        out = (C.c_double * 7)()
        b = None
        if bounds is not None:
            barr = (C.c_float * 6)(*bounds)
            b = C.cast(barr, C.c_void_p)
        A.check(A.lib().lbm_flow_report(self._h, int(plane), float(cut), b, out))
        keys = ("normal_velocity", "mass_flow", "momentum_thrust", "pressure", "pressure_power",
                "normal_kinetic_power", "area_mm2")
        return dict(zip(keys, out[:]))

    def export_vtk(self, path) -> None:
        """exportVTK: every cell of every level as a legacy ASCII VTK file."""
        A.check(A.lib().lbm_export_vtk(self._h, str(path).encode()))

    def save_state(self) -> bytes:
        """Checkpoint of everything the run carries between steps."""
        n = C.c_size_t()
        A.check(A.lib().lbm_state_bytes(self._h, C.byref(n)))
        buf = (C.c_ubyte * n.value)()
        A.check(A.lib().lbm_save_state(self._h, buf, n.value))
        return bytes(buf)

    def load_state(self, state: bytes):
        """Resume from a checkpoint of grids built from the same case."""
        buf = (C.c_ubyte * len(state)).from_buffer_copy(state)
        A.check(A.lib().lbm_load_state(self._h, buf, len(state)))

    def rotor_info(self, r: int, level: int = 0) -> A.LbmRotorInfo:
        info = A.LbmRotorInfo()
        A.check(A.lib().lbm_get_rotor_info(self._h, level, r, C.byref(info)))
        return info

    def set_rotor_speed(self, r: int, radians_per_second: float):
        A.check(A.lib().lbm_set_rotor_speed(self._h, r, radians_per_second))

    def rotor_force(self, r: int, reset: bool = False) -> np.ndarray:
        """{Fx, Fy, Fz [N], Tx, Ty, Tz [N m]} the rotor exerts on the fluid, rotor
        frame, averaged since the last tracker reset."""
        out = (C.c_double * 6)()
        A.check(A.lib().lbm_rotor_force(self._h, r, int(reset), out))
        return np.array(out[:])

    def rotor_bins(self, r: int, level: int = 0) -> np.ndarray:
        """Force bins of rotor r, float32 [3][27 * nonzero] (lattice units, rotor frame)."""
        n = self.rotor_info(r, level).nonzero_block_count
        out = np.empty((3, 27 * n), dtype=np.float32)
        A.check(A.lib().lbm_read_array(self._h, level, A.ARRAY_ROTOR_BASE + 4 * r + 3,
                                       out.ctypes.data_as(C.c_void_p), out.nbytes))
        return out

    def open_boundary_flow(self, open_bc_id: int, reset: bool = False) -> dict:
        """Flow through one open boundary averaged since the last tracker reset
        (SI units; the normal is the outer normal)."""
        out = (C.c_double * 7)()
        A.check(A.lib().lbm_open_boundary_flow(self._h, open_bc_id, int(reset), out))
        keys = ("area", "normal_velocity", "mass_flow", "momentum_thrust", "pressure", "pressure_power",
                "normal_kinetic_power")
        return dict(zip(keys, out[:]))

    def _float_pair(self, which: int, level: int) -> np.ndarray:
        m = self.info(level).open_bc_count
        out = np.empty((2, m), dtype=np.float32)
        A.check(A.lib().lbm_read_array(self._h, level, which, out.ctypes.data_as(C.c_void_p), out.nbytes))
        return out

    def open_reference(self, level: int = 0) -> np.ndarray:
        """Reference values of the open boundary: float32 [2][openBCCount] (dRho, uNormal)."""
        return self._float_pair(A.ARRAY_OPEN_REFERENCE, level)

    def open_cumulative(self, level: int = 0) -> np.ndarray:
        """Tracked sums since the last reset: float32 [2][openBCCount] (dRho, uNormal)."""
        return self._float_pair(A.ARRAY_OPEN_CUMULATIVE, level)

    def wall_force_raw(self, level: int = 0) -> np.ndarray:
        """Per-cell force accumulators float32 [3][wallCount] (lattice units)."""
        n = self.info(level).wall_adjacent_count
        out = np.empty((3, n), dtype=np.float32)
        A.check(A.lib().lbm_read_array(self._h, level, A.ARRAY_WALL_FORCE, out.ctypes.data_as(C.c_void_p),
                                       out.nbytes))
        return out


def update_batch(grids, coarse_steps: int = 1):
    """Advance independent domains together, each on its own stream (set with
    Grids.set_stream), so that their kernels overlap on the GPU."""
    arr = (C.c_void_p * len(grids))(*[g.handle for g in grids])
    A.check(A.lib().lbm_update_batch(arr, len(grids), int(coarse_steps)))


class PackedBatch:
    """Single-level domains advanced by one packed launch per kernel kind
    (lbm_batch_create): one persistent collide-stream over the packed
    {domain, item} table of all members, one open-boundary and one
    periodic-ghost launch; each member's result is bit-identical to the member
    run as a batch of one and agrees to FP32 rounding with update_all_grids.
    Free (close) the batch before its members."""

    def __init__(self, grids):
        self.members = list(grids)
        arr = (C.c_void_p * len(self.members))(*[g.handle for g in self.members])
        h = C.c_void_p()
        A.check(A.lib().lbm_batch_create(arr, len(self.members), C.byref(h)))
        self._h = h

    def close(self):
        if self._h:
            A.lib().lbm_batch_free(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def update(self, coarse_steps: int = 1):
        """Advance every member by `coarse_steps` (asynchronous; members must
        be at the same esotwist parity)."""
        A.check(A.lib().lbm_batch_update(self._h, int(coarse_steps)))

    def time_steps(self, coarse_steps: int) -> float:
        """Device milliseconds of `coarse_steps` packed steps."""
        ms = C.c_float()
        A.check(A.lib().lbm_batch_time_steps(self._h, int(coarse_steps), C.byref(ms)))
        return ms.value

    def info(self) -> A.LbmBatchInfo:
        out = A.LbmBatchInfo()
        A.check(A.lib().lbm_batch_get_info(self._h, C.byref(out)))
        return out


def build_grids(case: A.LbmCase) -> Grids:
    """buildGrids (include/gridBuilderFunctions.h:1577-1670) on the current device."""
    return Grids(case)


def apply_collision_batch(d_f_ptr: int, n: int, nu: float, limiter: float = 0.05,
                          nu_multiplier: float = 1.0, g=(0.0, 0.0, 0.0), stream_ptr: int = 0):
    """In-place cumulant collision of a device [27][n] float32 batch."""
    A.check(A.lib().lbm_apply_collision_batch(C.c_void_p(d_f_ptr), int(n), nu, limiter, nu_multiplier,
                                              g[0], g[1], g[2], C.c_void_p(stream_ptr)))
