"""Case descriptions: the runtime form of a reference driver's constants and hooks.

A reference driver (``cases/*/…Main.cu``) fixes its configuration with
``constexpr float`` constants and four ``__cuda_callable__`` hooks.  Here each
driver becomes a function returning an :class:`LbmCase`; constants are
evaluated in float32, operation by operation, so the grid geometry and the
lattice viscosity are bit-identical to what the driver's compiler computes.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _abi as A

f32 = np.float32


def _face(kind, open_bc_id=0, priority=0, non_reflective=False, beta=7.0,
          dRho=0.0, ux=0.0, uy=0.0, uz=0.0) -> A.LbmFaceBC:
    return A.LbmFaceBC(kind, open_bc_id, priority, int(non_reflective), beta, dRho, ux, uy, uz)


def _blank_case() -> A.LbmCase:
    c = A.LbmCase()
    c.grid_level_count = 1
    c.wall_refinement_count = 0
    c.rho_phys = 1.0
    c.collision_limiter = 0.05   # BCStruct default (include/types.h:131-136)
    c.nu_multiplier = 1.0
    c.use_ibb = 1                # BCStruct.useIBB default
    c.storage = A.LBM_STORE_F32
    for f in range(6):
        c.face[f] = _face(A.LBM_BC_PERIODIC)
    return c


@dataclass
class TGVSetup:
    """Numbers a Taylor–Green run needs next to its LbmCase."""
    case: A.LbmCase
    cells_per_domain: int
    u_initial: float          # lattice amplitude u0
    u_initial_phys: float     # m/s
    domain_length: float      # mm, periodic length
    reference_time: float     # s
    dt: float                 # s per step
    iteration_count: int      # steps to t* = end_time_star

    def time_star(self, steps: int) -> float:
        return steps * float(self.dt) / float(self.reference_time)


def taylor_green(cells_per_domain: int = 128, reynolds: float = 1600.0, mach: float = 0.1,
                 end_time_star: float = 20.0, storage: int = A.LBM_STORE_F32,
                 u_lattice: float | None = None, nu_lattice: float | None = None) -> TGVSetup:
    """Periodic Taylor–Green vortex (cases/taylorGreenVortex/taylorGreenVortexMain.cu:1-105, :187-204).

    With the default arguments this is the reference driver (Re 1600, Ma 0.1,
    one level).  ``u_lattice`` / ``nu_lattice`` override the Mach/Reynolds
    derived values, which expresses the plain-method configuration
    u0 = 0.05, nu = 0.01 on 64^3 in the same physical-unit framework.
    """
    PI = f32(3.14159265358979323846)
    reference_length = f32(1000.0)          # mm
    u_phys = f32(1.0)                       # m/s
    domain = f32(f32(2.0) * PI) * reference_length
    if u_lattice is None:
        u0 = f32(f32(mach) * f32(0.5773502691896258))
    else:
        u0 = f32(u_lattice)
    res = f32(domain / f32(cells_per_domain))
    dt = f32(f32(u0 / u_phys) * f32(res / f32(1000.0)))
    if nu_lattice is None:
        nu_phys = f32(f32(u_phys * f32(reference_length / f32(1000.0))) / f32(reynolds))
    else:
        # choose NU_PHYS so that dt * NU_PHYS / (res/1000)^2 == nu_lattice
        r = float(res) / 1000.0
        nu_phys = f32(float(nu_lattice) * r * r / float(dt))
    ref_time = f32(f32(reference_length / f32(1000.0)) / u_phys)
    iters = int(f32(f32(f32(end_time_star) * ref_time) / dt) + f32(0.5))

    c = _blank_case()
    c.res_global = res
    c.nu_phys = nu_phys
    c.rho_phys = 1.0
    c.dt_phys_global = dt
    half = f32(f32(0.5) * domain)
    eps = f32(f32(1e-6) * domain)
    lo = f32(f32(-half - res) - eps)
    hi = f32(f32(half + res) + eps)
    for a in range(3):
        c.bounds[a] = lo
        c.bounds[a + 3] = hi
    c.ic_kind = A.LBM_IC_TAYLOR_GREEN
    c.tgv_u0 = u0
    c.tgv_length = reference_length
    c.storage = storage
    return TGVSetup(c, cells_per_domain, float(u0), float(u_phys), float(domain),
                    float(ref_time), float(dt), iters)


def set_refine_box(case: A.LbmCase, level: int, lo, hi) -> A.LbmCase:
    """Refine the cells of `level` whose centres lie strictly inside the box
    [lo, hi] (mm) to the next level (getRefinementModifier as a table)."""
    for a in range(3):
        case.refine_box[level][a] = f32(lo[a])
        case.refine_box[level][a + 3] = f32(hi[a])
    return case


def taylor_green_refined(cells_per_domain: int = 128, storage: int = A.LBM_STORE_F32, **kw) -> TGVSetup:
    """The refined Taylor–Green run of the reference driver: two levels, the
    central cube [-pi L/2, pi L/2]^3 on the fine level
    (cases/taylorGreenVortex/taylorGreenVortexMain.cu:8-12, :53-67)."""
    s = taylor_green(cells_per_domain, storage=storage, **kw)
    s.case.grid_level_count = 2
    half = f32(f32(0.25) * f32(s.domain_length))
    set_refine_box(s.case, 0, (-half,) * 3, (half,) * 3)
    return s


def tgv_plain_method(storage: int = A.LBM_STORE_F32) -> TGVSetup:
    """Plain-method Taylor–Green: periodic 64^3, u0 = 0.05, nu = 0.01, 1000 steps."""
    s = taylor_green(64, u_lattice=0.05, nu_lattice=0.01, storage=storage)
    s.iteration_count = 1000
    return s


def periodic_box(nx: int, ny: int, nz: int, nu_lattice: float = 0.01, ux: float = 0.0,
                 uy: float = 0.0, uz: float = 0.0, storage: int = A.LBM_STORE_F32) -> A.LbmCase:
    """Fully periodic box of nx*ny*nz active cells (one ghost layer per face)
    with a uniform initial state.  nx, ny, nz must be even after adding the
    two ghost layers, i.e. even themselves."""
    if nx % 2 or ny % 2 or nz % 2:
        raise ValueError("active cell counts must be even")
    c = _blank_case()
    res = f32(1.0)
    c.res_global = res
    c.dt_phys_global = f32(1e-3)
    c.nu_phys = f32(float(nu_lattice) * 1e-6 / 1e-3)
    eps = f32(1e-3)
    for a, n in enumerate((nx, ny, nz)):
        c.bounds[a] = f32(-0.5 * n - 1.0) - eps
        c.bounds[a + 3] = f32(0.5 * n + 1.0) + eps
    c.ic_kind = A.LBM_IC_UNIFORM
    c.ic_ux, c.ic_uy, c.ic_uz = ux, uy, uz
    c.storage = storage
    return c


def open_channel(nx: int, ny: int, nz: int, u_in: float = 0.04, nu_lattice: float = 0.01,
                 sides: str = "velocity", outlet_non_reflective: bool = True, inlet_non_reflective: bool = False,
                 beta: float = 7.0, collision_limiter: float = 0.1, storage: int = A.LBM_STORE_F32) -> A.LbmCase:
    """Channel along x with nx*ny*nz cells (boundary layers included), 1 mm
    cells, uniform initial flow u_in.

    Faces follow the reference's flow-around-sphere driver
    (cases/flowAroundSphere/flowAroundSphereMain.cu:104-134): velocity inlet
    at x = 0 (openBCID 0), pressure outlet dRho = 0 at x = nx-1 (openBCID 1,
    non-reflective), and on the four sides either a strict velocity boundary
    u = (u_in, 0, 0) that also owns every edge and corner (``sides =
    "velocity"``, openBCID 2) or periodic faces (``sides = "periodic"``).
    The time step is chosen so that u_in is 1 m/s.
    """
    if nx % 2 or ny % 2 or nz % 2:
        raise ValueError("cell counts must be even")
    c = _blank_case()
    res = f32(1.0)
    c.res_global = res
    dt = f32(f32(u_in) * f32(res / f32(1000.0)))  # u_in lattice == 1 m/s
    c.dt_phys_global = dt
    r = float(res) / 1000.0
    c.nu_phys = f32(float(nu_lattice) * r * r / float(dt))
    eps = f32(1e-3)
    for a, n in enumerate((nx, ny, nz)):
        c.bounds[a] = -eps
        c.bounds[a + 3] = f32(n) + eps
    c.face[A.FACE_XMIN] = _face(A.LBM_BC_VELOCITY, open_bc_id=0, priority=1,
                                    non_reflective=inlet_non_reflective, beta=beta, ux=u_in)
    c.face[A.FACE_XMAX] = _face(A.LBM_BC_PRESSURE, open_bc_id=1, priority=1,
                                    non_reflective=outlet_non_reflective, beta=beta, dRho=0.0)
    for f in (A.FACE_YMIN, A.FACE_YMAX, A.FACE_ZMIN, A.FACE_ZMAX):
        if sides == "velocity":
            c.face[f] = _face(A.LBM_BC_VELOCITY, open_bc_id=2, priority=2, ux=u_in)
        elif sides == "periodic":
            c.face[f] = _face(A.LBM_BC_PERIODIC, priority=0)
        else:
            raise ValueError("sides must be 'velocity' or 'periodic'")
    c.ic_kind = A.LBM_IC_UNIFORM
    c.ic_ux = u_in
    c.collision_limiter = collision_limiter
    c.track_open_boundaries = 1
    c.storage = storage
    return c


@dataclass
class PipeSetup:
    """The non-reflective boundary study: the case and the inlet profile."""
    case: A.LbmCase
    u_mean: float             # lattice mean inlet velocity
    radius_mm: float
    dt: float                 # s per step

    def inlet_target(self, i: int, j: int, info) -> float:
        """Lattice uz the inlet prescribes at cell (i, j), as getOpenBC forms it."""
        return _pipe_profile(i, j, info, self.u_mean, self.radius_mm)


def _pipe_profile(i, j, info, u_mean, radius):
    # getXYZFromIJKCellIndex and the radius as device code forms them, with
    # contracted multiply-adds: x = fma(i, res, ox), r2 = fma(x, x, y * y)
    # (the products are exact in FP64, so one FP32 rounding of the sum is the fma)
    x = f32(float(i) * float(f32(info.res)) + float(f32(info.ox)))
    y = f32(float(j) * float(f32(info.res)) + float(f32(info.oy)))
    r2 = f32(float(x) * float(x) + float(f32(y * y)))
    return f32(f32(2.0) * f32(u_mean) * max(f32(0.0), f32(f32(1.0) - f32(r2 / f32(f32(radius) * f32(radius))))))


def non_reflective_pipe(scheme: str = "characteristic", tolerance: float = 2e-5, cells_per_mm: int = 5,
                        storage: int = A.LBM_STORE_F32) -> PipeSetup:
    """The reference's non-reflective boundary study
    (cases/nonReflectiveTest/nonReflectiveTestMain.cu): a pipe of 20 mm
    diameter, the bore of a 25 mm square block (a 90-sided polygon, vertices
    every 4 degrees), cut to 100 mm along z at 0.2 mm cells, Re 1000 on the
    mean velocity 0.03 (air: nu 1.5e-5 m^2/s, rho 1.225 kg/m^3), fluid at
    rest initially.  The inlet (k = 0, openBCID 0) prescribes the parabolic
    profile 2 u (1 - r^2 / R^2); the outlet (last k, openBCID 1) dRho = 0.
    `scheme`: "dirichlet" (plain inlet), "characteristic" (the stock
    non-reflective inlet) or "impedance" (the impedance scheme with
    RHO_REFLECTION_TOLERANCE = `tolerance`).  Walls without interpolation,
    AllOne collision (collision limiter 0)."""
    from .geometry import bored_block, set_bodies
    u_mean = f32(0.03)
    reynolds = f32(1000.0)
    diameter = f32(20.0)
    length = f32(100.0)
    radius = f32(f32(0.5) * diameter)
    nu_phys = f32(1.5e-5)
    res = f32(f32(1.0) / f32(cells_per_mm))
    u_phys = f32(reynolds * nu_phys / f32(diameter / f32(1000.0)))
    dt = f32(f32(u_mean / u_phys) * f32(res / f32(1000.0)))
    c = _blank_case()
    c.res_global = res
    c.nu_phys = nu_phys
    c.rho_phys = f32(1.225)
    c.dt_phys_global = dt
    tris = bored_block(12.5, float(radius), -100.0, 100.0, segments=90)
    set_bodies(c, [tris])
    lo, hi = tris.reshape(-1, 3).min(axis=0), tris.reshape(-1, 3).max(axis=0)
    c.bounds[0], c.bounds[1], c.bounds[3], c.bounds[4] = lo[0], lo[1], hi[0], hi[1]
    c.bounds[2], c.bounds[5] = -f32(length * f32(0.5)), f32(length * f32(0.5))
    c.collision_limiter = 0.0
    c.use_ibb = 0
    c.track_open_boundaries = 1
    c.storage = storage
    if scheme == "impedance":
        c.open_bc_scheme = A.LBM_OPEN_IMPEDANCE
        c.rho_reflection_tolerance = tolerance
    elif scheme not in ("characteristic", "dirichlet"):
        raise ValueError("scheme must be 'dirichlet', 'characteristic' or 'impedance'")
    non_reflective = scheme != "dirichlet"

    def open_bc(bc, i, j, k, info):
        if k == 0:
            bc.dirichletU = 1
            bc.ux, bc.uy = 0.0, 0.0
            bc.uz = _pipe_profile(i, j, info, u_mean, radius)
            bc.nonReflective = int(non_reflective)
            bc.openBCID = 0
        elif k == info.cell_count_z - 1:
            bc.dirichletRho = 1
            bc.dRho = 0.0
            bc.nonReflective = 0
            bc.openBCID = 1

    def local_bc(bc, i, j, k, info):
        bc.collisionLimiter = 0.0
        if bc.wallID >= 0:
            bc.ux = bc.uy = bc.uz = 0.0
        bc.useIBB = 0

    set_hooks(c, open_bc=open_bc, local_bc=local_bc)
    return PipeSetup(c, float(u_mean), float(radius), float(dt))


@dataclass
class SphereSetup:
    """Flow around a sphere: the case and what the drag coefficient needs."""
    case: A.LbmCase
    diameter_cells: float
    u_lattice: float
    u_phys: float            # m/s
    rho_phys: float          # kg/m^3
    diameter_m: float

    def drag_coefficient(self, fx: float) -> float:
        """Cd from the tracked x force, which acts on the fluid: drag = -Fx
        (cases/flowAroundSphere/flowAroundSphereMain.cu:212-213)."""
        area = math.pi * self.diameter_m ** 2 / 4.0
        return -fx / (0.5 * self.rho_phys * self.u_phys ** 2 * area)


def flow_around_sphere(nx: int = 256, ny: int = 128, nz: int = 128, diameter: float = 24.0,
                       center=(64.0, 64.0, 64.0), u_in: float = 0.04, nu_lattice: float = 0.0096,
                       subdivisions: int = 5, storage: int = A.LBM_STORE_F32,
                       sides: str = "velocity") -> SphereSetup:
    """Single-level flow around an icosphere (20 * 4**subdivisions triangles)
    of `diameter` cells centred at `center` (cell units, cell i spans
    [i, i+1)), in an open channel (see :func:`open_channel`), Re = u_in D / nu.
    The body is treated with interpolated bounceback and its force tracked."""
    from .geometry import icosphere, set_bodies
    c = open_channel(nx, ny, nz, u_in=u_in, nu_lattice=nu_lattice, sides=sides, storage=storage)
    c.track_wall_force = 1
    c.use_ibb = 1
    tris = icosphere(subdivisions, 0.5 * diameter, center)
    set_bodies(c, [tris])
    return SphereSetup(c, float(diameter), float(u_in), 1.0, float(c.rho_phys), float(diameter) / 1000.0)


@dataclass
class MultilevelSphereSetup:
    case: A.LbmCase
    diameter_finest: float    # sphere diameter in finest-level cells
    u_in: float
    reynolds: float


def multilevel_sphere(nx: int = 128, ny: int = 64, nz: int = 64, levels: int = 3, diameter_finest: float = 48.0,
                      reynolds: float = 300.0, u_in: float = 0.04, wall_refinement_count: int = 2,
                      subdivisions: int = 5, storage: int = A.LBM_STORE_F32,
                      fine_boxes=((96, 64, 64), (112, 80, 80))) -> MultilevelSphereSetup:
    """Flow around a sphere on nested refinement levels (ratio 2): an
    nx*ny*nz base channel (see :func:`open_channel`), the sphere of
    `diameter_finest` finest-level cells with its centre at a quarter of the
    channel length, and per level below the finest a refinement box around
    it of fine_boxes[level] cells of the next level, starting one third of
    its length upstream of the centre.  The sphere's own cells are refined to
    the finest level by its walls (markAllFinerWalls + WALL_REFINEMENT_COUNT).
    nu is set on the base level so that Re = u_in D / nu on every level.
    Level 0 collides with AllOne (limiter 0) and the finer levels with K17
    at limiter 0.1, as the reference's sphere driver does
    (cases/flowAroundSphere/flowAroundSphereMain.cu:136-149)."""
    from .geometry import icosphere, set_bodies
    scale = 2 ** (levels - 1)
    d0 = float(diameter_finest) / scale            # diameter in base cells
    nu0 = u_in * d0 / reynolds
    c = open_channel(nx, ny, nz, u_in=u_in, nu_lattice=nu0, collision_limiter=0.1, storage=storage)
    centre = (nx / 4.0, ny / 2.0, nz / 2.0)
    set_bodies(c, [icosphere(subdivisions, 0.5 * d0, centre)])
    c.grid_level_count = levels
    c.wall_refinement_count = wall_refinement_count
    c.track_wall_force = 1
    for l in range(levels - 1):
        cells = fine_boxes[l]
        size = [v / 2.0 ** (l + 1) for v in cells]       # in base cells
        lo = (centre[0] - size[0] / 3.0, centre[1] - size[1] / 2.0, centre[2] - size[2] / 2.0)
        set_refine_box(c, l, lo, (lo[0] + size[0], lo[1] + size[1], lo[2] + size[2]))

    def local(bc, i, j, k, info):
        if bc.wallID < 0:
            bc.collisionLimiter = 0.0 if info.grid_id == 0 else 0.1
    set_hooks(c, local_bc=local)
    return MultilevelSphereSetup(c, float(diameter_finest), float(u_in), float(reynolds))


def set_hooks(case: A.LbmCase, open_bc=None, initial_condition=None, local_bc=None,
              refinement=None) -> A.LbmCase:
    """Attach per-cell driver hooks (getOpenBC, getInitialCondition, getLocalBC)
    written in Python: each is called as hook(bc, i, j, k, info) with an
    lbm_bc to fill (the reference's BCStruct defaults, bc.wallID set for
    getLocalBC) and the level's lbm_grid_info, on the host while the grid is
    built.  `refinement(i, j, k, mark, info)` (getRefinementModifier)
    returns the refinement marker of a cell of a level below the finest.
    The callbacks are kept alive on the case object."""
    keep = []

    def wrap(fn):
        if fn is None:
            return None

        def tramp(user, bc, i, j, k, info):
            fn(bc.contents, i, j, k, info.contents)
        cb = A.CELL_HOOK(tramp)
        keep.append(cb)
        return C.cast(cb, C.c_void_p).value

    case.open_bc_hook = wrap(open_bc)
    case.initial_condition_hook = wrap(initial_condition)
    case.local_bc_hook = wrap(local_bc)
    if refinement is None:
        case.refinement_hook = None
    else:
        # refinement(i, j, k, mark, info) -> new mark (getRefinementModifier)
        def rtramp(user, i, j, k, mark, info):
            mark[0] = int(bool(refinement(i, j, k, bool(mark[0]), info.contents)))
        rcb = A.REFINEMENT_HOOK(rtramp)
        keep.append(rcb)
        case.refinement_hook = C.cast(rcb, C.c_void_p).value
    case.hook_user = None
    case._hook_refs = keep
    return case
