"""TEST INFRASTRUCTURE ONLY: ctypes loader for the CPU oracle (lbm_oracle.c).

Only tests/, ``__graft_entry__.smoke`` and bench.py's CPU-baseline leg use
this module, always as the checker or the timed CPU baseline, never as the
product path.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"


class OBC(C.Structure):
    _fields_ = [
        ("dRho", C.c_float), ("ux", C.c_float), ("uy", C.c_float), ("uz", C.c_float),
        ("gx", C.c_float), ("gy", C.c_float), ("gz", C.c_float),
        ("wallID", C.c_int), ("openBCID", C.c_int),
        ("useIBB", C.c_int), ("dirichletU", C.c_int), ("dirichletRho", C.c_int),
        ("periodic", C.c_int), ("nonReflective", C.c_int),
        ("nonReflectiveBeta", C.c_float), ("collisionLimiter", C.c_float), ("nuMultiplier", C.c_float),
    ]


_IP = C.POINTER(C.c_int)


class FaceBC(C.Structure):
    """lbm_face_bc of the public header (same layout)."""
    _fields_ = [
        ("kind", C.c_int), ("open_bc_id", C.c_int), ("priority", C.c_int),
        ("non_reflective", C.c_int), ("non_reflective_beta", C.c_float),
        ("dRho", C.c_float), ("ux", C.c_float), ("uy", C.c_float), ("uz", C.c_float),
    ]


class OGrid(C.Structure):
    _fields_ = [
        ("gridID", C.c_int), ("res", C.c_float), ("ox", C.c_float), ("oy", C.c_float), ("oz", C.c_float),
        ("nu", C.c_float), ("dtPhys", C.c_float),
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("cellCount", C.c_int),
        ("flip", C.c_int), ("iterationsFinished", C.c_int),
        ("I", _IP), ("J", _IP), ("K", _IP), ("jPlus", _IP), ("kPlus", _IP),
        ("geomBits", C.POINTER(C.c_ubyte)), ("wallMarker", C.POINTER(C.c_ubyte)),
        ("shifter", _IP), ("rowCount", C.c_int),
        ("rowI", _IP), ("rowJ", _IP), ("rowK", _IP), ("rowJP", _IP), ("rowKP", _IP), ("rowJKP", _IP),
        ("wallMap", _IP), ("perCount", C.c_int), ("perIndex", _IP), ("perSource", _IP),
        ("openBCCount", C.c_int), ("f", C.POINTER(C.c_float)), ("fluidUpdates", C.c_longlong),
        ("limiter", C.c_float), ("nuMultiplier", C.c_float),
        ("gx", C.c_float), ("gy", C.c_float), ("gz", C.c_float), ("useIBB", C.c_int),
        ("wallCount", C.c_int), ("wallIndex", _IP), ("wallData", C.POINTER(C.c_uint)),
        ("linkLength", C.POINTER(C.c_uint)), ("wallVel", C.POINTER(C.c_float)),
        ("wallForce", C.POINTER(C.c_float)), ("trackWallForce", C.c_int),
        ("face", FaceBC * 6), ("openCount", C.c_int), ("openIndex", _IP),
        ("openRef", C.POINTER(C.c_float)), ("openCum", C.POINTER(C.c_float)), ("trackOpen", C.c_int), ("openImpedance", C.c_int), ("openTolerance", C.c_float),
        ("rotorCount", C.c_int), ("rotors", C.c_void_p), ("trackRotorForce", C.c_int),
        ("openHook", C.c_void_p), ("hookUser", C.c_void_p),
    ]


class OInterface(C.Structure):
    _fields_ = [("f2cCount", C.c_int), ("c2fCount", C.c_int), ("leftCount", C.c_int),
                ("f2cIndex", _IP), ("f2cChild", _IP), ("c2fIndex", _IP), ("c2fChild", _IP),
                ("leftIndex", _IP), ("leftParent", _IP), ("leftNbr", _IP)]


MAX_LEVELS = 4


class ODomain(C.Structure):
    _fields_ = [("levelCount", C.c_int), ("level", OGrid * MAX_LEVELS), ("itf", OInterface * MAX_LEVELS)]


_lib = None


def build() -> Path:
    """Compile the oracle with its Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        sources = ("lbm_oracle.c", "oracle_geometry.c", "lbm_oracle.h", "oracle_internal.h")
        if not LIB.exists() or any(LIB.stat().st_mtime < (HERE / f).stat().st_mtime for f in sources):
            build()
        h = C.CDLL(str(LIB))
        h.oracle_default_bc.argtypes = [C.POINTER(OBC)]
        h.oracle_apply_collision.argtypes = [C.POINTER(C.c_float), C.POINTER(OBC), C.c_float]
        h.oracle_apply_collision_batch.argtypes = [C.POINTER(C.c_float), C.c_int, C.c_float, C.c_float,
                                                   C.c_float, C.c_float, C.c_float, C.c_float]
        h.oracle_get_feq.argtypes = [C.c_float] * 4 + [C.POINTER(C.c_float)]
        h.oracle_get_drho_u.argtypes = [C.POINTER(C.c_float), C.POINTER(C.c_float)]
        h.oracle_build.argtypes = [C.c_void_p, C.POINTER(OGrid)]
        h.oracle_build.restype = C.c_int
        h.oracle_free.argtypes = [C.POINTER(OGrid)]
        h.oracle_step.argtypes = [C.POINTER(OGrid), C.c_int]
        h.oracle_kinetic_energy.argtypes = [C.POINTER(OGrid), C.c_float, C.c_float]
        h.oracle_kinetic_energy.restype = C.c_double
        h.oracle_macro.argtypes = [C.POINTER(OGrid), C.POINTER(C.c_float)]
        h.oracle_global_sums.argtypes = [C.POINTER(OGrid), C.POINTER(C.c_double)]
        h.oracle_threads.restype = C.c_int
        h.oracle_collide_range.argtypes = [C.POINTER(OGrid), C.c_int, C.c_int]
        h.oracle_from_tables.argtypes = [C.c_void_p, C.POINTER(OGrid), C.c_int, C.c_int] + [C.c_void_p] * 8 + \
            [C.c_int, C.c_void_p, C.c_void_p, C.c_int] + [C.c_void_p] * 4
        h.oracle_from_tables.restype = C.c_int
        h.oracle_wall_force.argtypes = [C.POINTER(OGrid), C.c_int, C.POINTER(C.c_double)]
        h.oracle_set_rotor.argtypes = [C.POINTER(OGrid), C.c_int, C.c_float, C.c_void_p, C.c_void_p, C.c_int,
                                       C.c_void_p, C.c_float, C.c_void_p, C.c_int, C.c_void_p, C.c_int]
        h.oracle_set_rotor.restype = C.c_int
        h.oracle_rotor_bins.argtypes = [C.POINTER(OGrid), C.c_int, C.POINTER(C.c_float)]
        h.oracle_rotor_tables.argtypes = [C.POINTER(OGrid), C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                          C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                          C.POINTER(C.POINTER(C.c_int)), C.POINTER(C.POINTER(C.c_uint))]
        h.oracle_rotor_tables.restype = C.c_int
        h.oracle_flow_sums.argtypes = [C.POINTER(OGrid)] + [C.c_int] * 6 + [C.POINTER(C.c_double)]
        h.oracle_mbbc_apply.argtypes = [C.c_int] + [C.c_float] * 4 + [C.POINTER(C.c_float)]
        h.oracle_mbbc_restore_rho.argtypes = [C.c_int] + [C.c_float] * 3 + [C.POINTER(C.c_float)] * 2
        h.oracle_mbbc_restore_u.argtypes = [C.c_int, C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        h.oracle_domain_build.argtypes = [C.c_void_p, C.POINTER(ODomain)]
        h.oracle_domain_build.restype = C.c_int
        h.oracle_flow_image.argtypes = [C.POINTER(ODomain), C.c_int, C.c_float, C.POINTER(C.c_float),
                                        C.POINTER(C.c_double), C.POINTER(C.c_int)]
        h.oracle_flow_image.restype = C.c_int
        h.oracle_domain_free.argtypes = [C.POINTER(ODomain)]
        h.oracle_domain_step.argtypes = [C.POINTER(ODomain), C.c_int]
        h.oracle_domain_kinetic_energy.argtypes = [C.POINTER(ODomain), C.c_float, C.c_float]
        h.oracle_domain_kinetic_energy.restype = C.c_double
        h.oracle_fit_check.argtypes = [C.POINTER(C.c_float), C.c_float, C.c_float, C.c_float, C.POINTER(C.c_float)]
        _lib = h
    return _lib


def _fp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def threads() -> int:
    return lib().oracle_threads()


def default_bc() -> OBC:
    bc = OBC()
    lib().oracle_default_bc(C.byref(bc))
    return bc


def apply_collision(f: np.ndarray, nu: float, limiter: float = 0.05, nu_multiplier: float = 1.0,
                    g=(0.0, 0.0, 0.0)) -> np.ndarray:
    """Collide a single cell (27 shifted populations); returns a new array."""
    v = np.ascontiguousarray(f, dtype=np.float32).copy()
    bc = default_bc()
    bc.collisionLimiter = limiter
    bc.nuMultiplier = nu_multiplier
    bc.gx, bc.gy, bc.gz = g
    lib().oracle_apply_collision(_fp(v), C.byref(bc), nu)
    return v


def apply_collision_batch(f: np.ndarray, nu: float, limiter: float = 0.05, nu_multiplier: float = 1.0,
                          g=(0.0, 0.0, 0.0)) -> np.ndarray:
    v = np.ascontiguousarray(f, dtype=np.float32).copy()
    n = v.shape[1]
    lib().oracle_apply_collision_batch(_fp(v), n, nu, limiter, nu_multiplier, g[0], g[1], g[2])
    return v


def feq(dRho: float, ux: float, uy: float, uz: float) -> np.ndarray:
    out = np.empty(27, dtype=np.float32)
    lib().oracle_get_feq(dRho, ux, uy, uz, _fp(out))
    return out


def drho_u(f: np.ndarray) -> np.ndarray:
    v = np.ascontiguousarray(f, dtype=np.float32)
    out = np.empty(4, dtype=np.float32)
    lib().oracle_get_drho_u(_fp(v), _fp(out))
    return out


def mbbc_apply(code: int, rho: float, u, f: np.ndarray) -> np.ndarray:
    """applyMBBC on full populations; returns the completed 27 values."""
    v = np.ascontiguousarray(f, dtype=np.float32).copy()
    if lib().oracle_mbbc_apply(int(code), rho, u[0], u[1], u[2], _fp(v)) != 0:
        raise ValueError(f"no outer normal with code {code}")
    return v


def mbbc_restore_rho(code: int, u, f: np.ndarray) -> float:
    v = np.ascontiguousarray(f, dtype=np.float32)
    out = np.zeros(1, dtype=np.float32)
    if lib().oracle_mbbc_restore_rho(int(code), u[0], u[1], u[2], _fp(v), _fp(out)) != 0:
        raise ValueError(f"no outer normal with code {code}")
    return out[0]


def mbbc_restore_u(code: int, rho: float, f: np.ndarray) -> np.ndarray:
    v = np.ascontiguousarray(f, dtype=np.float32)
    out = np.zeros(3, dtype=np.float32)
    if lib().oracle_mbbc_restore_u(int(code), rho, _fp(v), _fp(out)) != 0:
        raise ValueError(f"no outer normal with code {code}")
    return out


def _vp(a):
    return a.ctypes.data_as(C.c_void_p)


class OracleGrid:
    """Single-level domain run by the oracle.  By default the oracle builds
    every table itself from the case (voxelizer, markers, wall links, rotors:
    its own restatement of the reference's setup chain); passing a host
    ``plan`` instead loads the product's tables (used only to isolate a time
    step difference from a setup difference)."""

    def __init__(self, case, plan=None):
        self.g = OGrid()
        if plan is None:
            rc = lib().oracle_build(C.cast(C.byref(case), C.c_void_p), C.byref(self.g))
            if rc != 0:
                raise RuntimeError(f"oracle_build failed with status {rc}")
            self._rotor_nonzero = [self.rotor_tables(r)["nonzero"] for r in range(self.g.rotorCount)]
            return
        info = plan.info()
        arrays = {k: plan.array(k) for k in ("shifter", "row_i", "row_j", "row_k", "row_jplus", "row_kplus",
                                              "row_jkplus", "wall_map", "periodic_index", "periodic_source",
                                              "wall_index")}
        wd = plan.uint_array("wall_data")
        ll = plan.uint_array("link_length")
        wv = np.ascontiguousarray(plan.wall_velocity(), dtype=np.float32)
        self._keep = (arrays, wd, ll, wv)
        rc = lib().oracle_from_tables(
            C.cast(C.byref(case), C.c_void_p), C.byref(self.g), info.cell_count, info.row_count,
            *[_vp(arrays[k]) for k in ("shifter", "row_i", "row_j", "row_k", "row_jplus", "row_kplus",
                                       "row_jkplus", "wall_map")],
            info.periodic_count, _vp(arrays["periodic_index"]), _vp(arrays["periodic_source"]),
            info.wall_adjacent_count, _vp(arrays["wall_index"]), _vp(wd), _vp(ll), _vp(wv))
        if rc != 0:
            raise RuntimeError(f"oracle_from_tables failed with status {rc}")
        self._rotor_nonzero = []
        for r in range(plan.rotor_count()):
            ri = plan.rotor_info(r)
            self._rotor_nonzero.append(ri.nonzero_block_count)
            rmap = plan.rotor_array(r, "map")
            interp = plan.rotor_array(r, "interpolation")
            bounds = np.array(ri.bounds[:], dtype=np.float32)
            counts = np.array(ri.cell_count[:], dtype=np.int32)
            origin = np.array(ri.origin[:], dtype=np.float32)
            self._keep += (rmap, interp, bounds, counts, origin)
            if lib().oracle_set_rotor(C.byref(self.g), r, ri.res, _vp(bounds), _vp(counts), ri.axis, _vp(origin),
                                      ri.radians_per_second, _vp(rmap), len(rmap), _vp(interp),
                                      ri.nonzero_block_count) != 0:
                raise RuntimeError("oracle_set_rotor failed")

    def wall_force(self, wall_id: int) -> np.ndarray:
        out = (C.c_double * 6)()
        lib().oracle_wall_force(C.byref(self.g), wall_id, out)
        return np.array(out[:])

    def close(self):
        if self.g.f:
            lib().oracle_free(C.byref(self.g))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def cell_count(self) -> int:
        return self.g.cellCount

    def step(self, steps: int = 1):
        lib().oracle_step(C.byref(self.g), int(steps))

    def collide_range(self, c0: int, c1: int):
        """Collide-stream of cells [c0, c1) of the current step (timing sample)."""
        lib().oracle_collide_range(C.byref(self.g), int(c0), int(c1))

    def kinetic_energy(self, u_ref_phys: float, domain_length: float) -> float:
        return lib().oracle_kinetic_energy(C.byref(self.g), u_ref_phys, domain_length)

    def global_sums(self) -> np.ndarray:
        """{sum rho, sum dRho, momentum x, y, z, cells} in lattice units (FP64)."""
        out = (C.c_double * 6)()
        lib().oracle_global_sums(C.byref(self.g), out)
        return np.array(out[:])

    def macro(self) -> np.ndarray:
        out = np.empty((4, self.g.cellCount), dtype=np.float32)
        lib().oracle_macro(C.byref(self.g), _fp(out))
        return out

    def populations(self) -> np.ndarray:
        n = self.g.cellCount
        return np.ctypeslib.as_array(self.g.f, shape=(27 * n,)).reshape(27, n).copy()

    def set_populations(self, f: np.ndarray):
        n = self.g.cellCount
        dst = np.ctypeslib.as_array(self.g.f, shape=(27 * n,))
        dst[:] = np.ascontiguousarray(f, dtype=np.float32).reshape(-1)

    def rotor_bins(self, r: int) -> np.ndarray:
        """Force bins of rotor r, float32 [3][27 * nonzero]."""
        import ctypes as _C
        R = self._rotor_nonzero[r]
        out = np.empty(3 * 27 * R, dtype=np.float32)
        lib().oracle_rotor_bins(C.byref(self.g), r, _fp(out))
        return out.reshape(3, -1)

    def flow_sums(self, plane: int, layer: int, h0: int, h1: int, v0: int, v1: int) -> np.ndarray:
        out = (C.c_double * 6)()
        lib().oracle_flow_sums(C.byref(self.g), plane, layer, h0, h1, v0, v1, out)
        return np.array(out[:])

    def open_index(self) -> np.ndarray:
        m = self.g.openCount
        return np.ctypeslib.as_array(self.g.openIndex, shape=(m,)).copy() if m else np.empty(0, np.int32)

    def open_reference(self) -> np.ndarray:
        """[2][openCount]: dRhoRef, uNormalRef."""
        m = self.g.openCount
        return np.ctypeslib.as_array(self.g.openRef, shape=(2 * m,)).reshape(2, m).copy()

    def open_cumulative(self) -> np.ndarray:
        m = self.g.openCount
        return np.ctypeslib.as_array(self.g.openCum, shape=(2 * m,)).reshape(2, m).copy()

    def wall_arrays(self) -> dict:
        """Wall-adjacent tables: index [nW], wall_data [nW] (uint32),
        link_length [7][nW] (uint32), wall_velocity [3][nW] (float32)."""
        nw = self.g.wallCount
        if nw == 0:
            return {"index": np.empty(0, np.int32), "wall_data": np.empty(0, np.uint32),
                    "link_length": np.empty((7, 0), np.uint32), "wall_velocity": np.empty((3, 0), np.float32)}
        return {"index": np.ctypeslib.as_array(self.g.wallIndex, shape=(nw,)).copy(),
                "wall_data": np.ctypeslib.as_array(self.g.wallData, shape=(nw,)).copy(),
                "link_length": np.ctypeslib.as_array(self.g.linkLength, shape=(7 * nw,)).reshape(7, nw).copy(),
                "wall_velocity": np.ctypeslib.as_array(self.g.wallVel, shape=(3 * nw,)).reshape(3, nw).copy()}

    def rotor_tables(self, r: int) -> dict:
        """Rotor r as the oracle built it: res, bounds, cell counts, rotorMap,
        interpolation (uint32 [64 * nonzero])."""
        res = C.c_float()
        bounds = (C.c_float * 6)()
        counts = (C.c_int * 3)()
        blocks, nonzero = C.c_int(), C.c_int()
        rmap = C.POINTER(C.c_int)()
        interp = C.POINTER(C.c_uint)()
        if lib().oracle_rotor_tables(C.byref(self.g), r, C.byref(res), bounds, counts, C.byref(blocks),
                                     C.byref(nonzero), C.byref(rmap), C.byref(interp)) != 0:
            raise IndexError(f"no rotor {r}")
        nz = nonzero.value
        return {"res": res.value, "bounds": np.array(bounds[:], np.float32), "cell_count": np.array(counts[:]),
                "block_count": blocks.value, "nonzero": nz,
                "map": np.ctypeslib.as_array(rmap, shape=(blocks.value,)).copy(),
                "interpolation": np.ctypeslib.as_array(interp, shape=(64 * nz,)).copy() if nz
                else np.empty(0, np.uint32)}

    def int_array(self, name: str) -> np.ndarray:
        lengths = {"I": self.g.cellCount, "J": self.g.cellCount, "K": self.g.cellCount,
                   "jPlus": self.g.cellCount, "kPlus": self.g.cellCount, "shifter": self.g.cellCount,
                   "wallMap": self.g.cellCount, "rowI": self.g.rowCount, "rowJ": self.g.rowCount,
                   "rowK": self.g.rowCount, "rowJP": self.g.rowCount, "rowKP": self.g.rowCount,
                   "rowJKP": self.g.rowCount, "perIndex": self.g.perCount, "perSource": self.g.perCount}
        n = lengths[name]
        ptr = getattr(self.g, name)
        if n == 0:
            return np.empty(0, dtype=np.int32)
        return np.ctypeslib.as_array(ptr, shape=(n,)).copy()


class OracleLevel(OracleGrid):
    """One level of an :class:`OracleDomain` (a view; the domain owns it)."""

    def __init__(self, view: OGrid, owner):
        self.g = view
        self._owner = owner
        self._rotor_nonzero = [self.rotor_tables(r)["nonzero"] for r in range(self.g.rotorCount)]

    def close(self):
        pass

    def step(self, steps: int = 1):
        raise RuntimeError("step a multilevel domain with OracleDomain.step")


class OracleDomain:
    """Every level of a domain run by the oracle: its own multilevel build
    (refinement markers, finer grids, interfaces) and the recursive time step
    with the interface exchange."""

    def __init__(self, case):
        self.d = ODomain()
        rc = lib().oracle_domain_build(C.cast(C.byref(case), C.c_void_p), C.byref(self.d))
        if rc != 0:
            raise RuntimeError(f"oracle_domain_build failed with status {rc}")
        self.levels = [OracleLevel(self.d.level[l], self) for l in range(self.d.levelCount)]

    def level(self, l: int) -> OracleLevel:
        return self.levels[l]

    @property
    def level_count(self) -> int:
        return self.d.levelCount

    def step(self, coarse_steps: int = 1):
        lib().oracle_domain_step(C.byref(self.d), int(coarse_steps))

    def kinetic_energy(self, u_ref_phys: float, domain_length: float) -> float:
        return lib().oracle_domain_kinetic_energy(C.byref(self.d), u_ref_phys, domain_length)

    def flow_image(self, plane: int, cut: float, bounds=None):
        """Raw section-image sums of every level and the image's level."""
        out = (C.c_double * 6)()
        lvl = C.c_int()
        b = (C.c_float * 6)(*bounds) if bounds is not None else None
        rc = lib().oracle_flow_image(C.byref(self.d), int(plane), float(cut), b, out, C.byref(lvl))
        if rc != 0:
            raise ValueError(f"oracle_flow_image failed with status {rc}")
        return np.array(out[:]), lvl.value

    def macro(self, l: int = 0) -> np.ndarray:
        return self.levels[l].macro()

    def interface(self, l: int) -> dict:
        """Interface lists of level l towards level l + 1."""
        it = self.d.itf[l]

        def arr(ptr, n):
            return np.ctypeslib.as_array(ptr, shape=(n,)).copy() if n else np.empty(0, np.int32)
        return {"f2c_index": arr(it.f2cIndex, it.f2cCount), "f2c_child": arr(it.f2cChild, it.f2cCount),
                "c2f_index": arr(it.c2fIndex, it.c2fCount), "c2f_child": arr(it.c2fChild, it.c2fCount),
                "leftover_index": arr(it.leftIndex, it.leftCount),
                "leftover_parent": arr(it.leftParent, it.leftCount),
                "leftover_nbr": arr(it.leftNbr, 3 * it.leftCount)}

    def close(self):
        if self.d.levelCount:
            self.levels = []
            lib().oracle_domain_free(C.byref(self.d))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def fit_check(corners: np.ndarray, x: float, y: float, z: float) -> np.ndarray:
    """The interface fit of 8 corner records [8][9] at (x, y, z): {dRho, u, G}."""
    c = np.ascontiguousarray(corners, dtype=np.float32).reshape(-1)
    out = np.empty(13, dtype=np.float32)
    lib().oracle_fit_check(_fp(c), x, y, z, _fp(out))
    return out
