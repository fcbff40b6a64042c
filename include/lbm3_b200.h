/*
 * lbm3_b200.h — C ABI of the B200-native D3Q27 cumulant lattice-Boltzmann time step.
 *
 * Plain C types only (pointers, sizes, PODs); no C++ or torch types cross this
 * boundary.  Every call returns an int status (LBM_OK == 0, negative on error)
 * and leaves a human-readable message behind lbm_last_error().  Exceptions
 * never cross the boundary.
 *
 * The reference (stepanmuller/LBM3) exposes a header-level C++ API whose case
 * configuration is compile-time: constants such as RES_GLOBAL / NU_PHYS and
 * four __cuda_callable__ hooks (getOpenBC, getLocalBC, getInitialCondition,
 * getRefinementModifier) defined in the driver translation unit.  Here those
 * become the runtime, table-driven `lbm_case` description below.  Each entry
 * point names the reference function it replaces (path:line inside the
 * reference project).
 */
#ifndef LBM3_B200_H
#define LBM3_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define LBM_OK               0
#define LBM_ERR_INVALID     -1  /* bad argument or inconsistent case            */
#define LBM_ERR_CUDA        -2  /* a CUDA runtime call failed                   */
#define LBM_ERR_OOM         -3  /* device allocation failed                     */
#define LBM_ERR_BUILD       -4  /* setup failed (the reference throws
                                   std::runtime_error at these points, e.g.
                                   include/gridBuilderFunctions.h:1479,:1563) */
#define LBM_ERR_UNSUPPORTED -5  /* feature not available in this build          */
#define LBM_ERR_NO_DEVICE   -6  /* no CUDA device visible                       */
#define LBM_ERR_DEVICE_WAIT -7  /* a bounded wait inside a kernel gave up; the
                                   step that reported it is not trustworthy */

/* ---- boundary kinds for a domain face (replaces the getOpenBC hook) ------ */
#define LBM_BC_PERIODIC   0   /* BCStruct.periodic     (include/types.h:131-136) */
#define LBM_BC_VELOCITY   1   /* BCStruct.dirichletU                             */
#define LBM_BC_PRESSURE   2   /* BCStruct.dirichletRho                           */

/* face order inside lbm_case.face[] */
#define LBM_FACE_XMIN 0
#define LBM_FACE_XMAX 1
#define LBM_FACE_YMIN 2
#define LBM_FACE_YMAX 3
#define LBM_FACE_ZMIN 4
#define LBM_FACE_ZMAX 5

/* initial condition kinds (replaces the getInitialCondition hook) */
#define LBM_IC_UNIFORM      0  /* dRho, ux, uy, uz constant                      */
#define LBM_IC_TAYLOR_GREEN 1  /* cases/taylorGreenVortex/taylorGreenVortexMain.cu:66-87 */

/* population storage precision (arithmetic is FP32 for the first three) */
#define LBM_STORE_F32  0
#define LBM_STORE_F16  1      /* shifted populations f_i - w_i as IEEE half     */
#define LBM_STORE_BF16 2      /* shifted populations f_i - w_i as bfloat16      */
                              /* (16-bit stores of collided, boundary and
                                 interface values round stochastically; see
                                 lbm_build_grids)                               */
#define LBM_STORE_F64  3      /* FP64 populations and FP64 arithmetic: the
                                 double-precision build of the same kernels,
                                 the reference of the storage-precision study */

/* arrays that lbm_read_array can copy out (per level) */
#define LBM_ARRAY_F            0  /* float  [27][cellCount] (always returned as FP32) */
#define LBM_ARRAY_SHIFTER      1  /* int32  [cellCount]     IJKNBR.shifterArray   */
#define LBM_ARRAY_ROW_I        2  /* int32  [rowCount]      IJKNBR.iArray         */
#define LBM_ARRAY_ROW_J        3  /* int32  [rowCount]      IJKNBR.jArray         */
#define LBM_ARRAY_ROW_K        4  /* int32  [rowCount]      IJKNBR.kArray         */
#define LBM_ARRAY_ROW_JPLUS    5  /* int32  [rowCount]      IJKNBR.jPlusArray     */
#define LBM_ARRAY_ROW_KPLUS    6  /* int32  [rowCount]      IJKNBR.kPlusArray     */
#define LBM_ARRAY_ROW_JKPLUS   7  /* int32  [rowCount]      IJKNBR.jkPlusArray    */
#define LBM_ARRAY_WALL_MAP     8  /* int32  [cellCount]     Wall.wallMapArray     */
#define LBM_ARRAY_PERIODIC_INDEX  9  /* int32 [periodicCount] PeriodicBC.indexArray  */
#define LBM_ARRAY_PERIODIC_SOURCE 10 /* int32 [periodicCount] PeriodicBC.sourceArray */
#define LBM_ARRAY_MACRO        11 /* float  [4][cellCount]  dRho, ux, uy, uz of the
                                     current pre-collision state (getDRhoUxUyUz)  */
#define LBM_ARRAY_WALL_INDEX   12 /* int32  [wallAdjacentCount] Wall.indexArray    */
#define LBM_ARRAY_WALL_DATA    13 /* uint32 [wallAdjacentCount] Wall.wallDataArray */
#define LBM_ARRAY_LINK_LENGTH  14 /* uint32 [7][wallAdjacentCount] Wall.linkLengthArray */
#define LBM_ARRAY_WALL_FORCE   15 /* float  [3][wallAdjacentCount] Wall.gx/gy/gzArray
                                     accumulated since the last tracker reset   */
#define LBM_ARRAY_WALL_VELOCITY 16 /* float [3][wallAdjacentCount] wall velocity the
                                     body motion gives each wall-adjacent cell   */
#define LBM_ARRAY_OPEN_INDEX   17 /* int32  [openBCCount]   openBCs[id].indexArray of all
                                     IDs concatenated in ID order               */
#define LBM_ARRAY_OPEN_SOURCE  18 /* int32  [openBCCount]   openBCs[id].sourceArray, same order */
#define LBM_ARRAY_OPEN_REFERENCE 19 /* float [2][openBCCount] dRhoRefArray, uNormalRefArray */
/* rotor tables: id = LBM_ARRAY_ROTOR_BASE + 4 * rotor + one of:
 *   0 int32  [block_count]              rotorMapArray (-1 or compact block index)
 *   1 int32  [nonzero_block_count]      indexArray
 *   2 uint32 [64 * nonzero_block_count] interpolationArray (8 x 4-bit counts)
 *   3 float  [3][27 * nonzero_block_count] gx, gy, gz force bins in the rotor
 *            frame, accumulated since the last tracker reset (grids only) */
#define LBM_ARRAY_ROTOR_BASE   32
#define LBM_ARRAY_OPEN_CUMULATIVE 20 /* float [2][openBCCount] dRhoCumulativeArray,
                                     uNormalCumulativeArray since the last tracker reset */
/* Interfaces between a level (coarse) and the next finer one, read on the
 * coarse level (InterfaceStruct, include/types.h:198-200): */
#define LBM_ARRAY_F2C_INDEX      21 /* int32 [f2cCount] FineToCoarseInterface.indexArray (coarse cells) */
#define LBM_ARRAY_F2C_CHILD      22 /* int32 [f2cCount] childMapArray (fine cell (2i,2j,2k))          */
#define LBM_ARRAY_C2F_INDEX      23 /* int32 [c2fCount] CoarseToFineInterface.indexArray: coarse
                                       stencil corner (the block's -x,-y,-z coarse cell)           */
#define LBM_ARRAY_C2F_CHILD      24 /* int32 [c2fCount] childMapArray: fine cell (2i+1,2j+1,2k+1)   */
#define LBM_ARRAY_LEFTOVER_INDEX 25 /* int32 [leftoverCount] leftoverIndexArray (fine cells)        */
#define LBM_ARRAY_LEFTOVER_PARENT 26 /* int32 [leftoverCount] leftoverParentMapArray (coarse cells)  */
#define LBM_ARRAY_LEFTOVER_NBR   27 /* int32 [3][leftoverCount] leftoverNbrI/J/KArray: the coarse
                                       neighbour on the fine cell's side, or -(cell)-1 for the
                                       opposite side                                               */

/* A rotor forced towards rigid rotation (RotorStruct, include/types.h:206-219):
 * triangles of its surface at angle 0 (mm), the axis it turns about (parallel
 * to x, y or z through `origin`) and its speed.  Cells inside the rotor, in
 * the rotor's own frame, are forced towards the rotor velocity with a
 * smooth volume fraction (processRotor, include/rotorFunctions.h:211-304). */
#define LBM_MAX_ROTORS 4
typedef struct lbm_rotor {
    const float* triangles;     /* [triangle_count][9]                        */
    int   triangle_count;
    int   axis;                 /* 0: rotateAlongX, 1: Y, 2: Z                */
    float origin[3];            /* InfoRotor.ox, oy, oz (mm)                  */
    float radians_per_second;   /* InfoRotor.radiansPerSecond                 */
} lbm_rotor;

/* Rotor tables of one level (RotorInfoStruct plus table sizes). */
typedef struct lbm_rotor_info {
    float res;                  /* half the level spacing (mm)                */
    float bounds[6];            /* xMin, yMin, zMin, xMax, yMax, zMax (mm)    */
    int   cell_count[3];        /* interpolation cells, multiples of 4        */
    int   block_count;          /* 4x4x4 blocks in the bounds                 */
    int   nonzero_block_count;  /* blocks with rotor volume                   */
    int   axis;
    float origin[3];
    float radians_per_second;
    double radians_elapsed;
} lbm_rotor_info;

/* ---- case description -------------------------------------------------- */

/* One domain face.  `priority` decides edge and corner cells: a boundary cell
 * that touches several faces takes the description of the touching face with
 * the highest priority (ties: lower face index).  This reproduces drivers
 * such as cases/flowAroundSphere/flowAroundSphereMain.cu:103-135, where
 * edges of the inlet/outlet faces belong to the side faces. */
typedef struct lbm_face_bc {
    int   kind;                 /* LBM_BC_*                                   */
    int   open_bc_id;           /* BCStruct.openBCID                          */
    int   priority;
    int   non_reflective;       /* BCStruct.nonReflective                     */
    float non_reflective_beta;  /* BCStruct.nonReflectiveBeta (default 7)     */
    float dRho, ux, uy, uz;     /* target values                              */
} lbm_face_bc;

/* wall motion of a static body (replaces the per-wallID branch of getLocalBC,
 * e.g. cases/torqueTest/torqueTestMain.cu:100-122) */
#define LBM_WALL_STATIC   0   /* u_wall = 0                                   */
#define LBM_WALL_ROTATING 1   /* rigid rotation about an axis parallel to x/y/z */

#define LBM_MAX_BODIES 16     /* wallID is packed into 5 bits of wallData      */

#define LBM_MAX_LEVELS 4      /* grid levels of one domain, refinement ratio 2  */

/* non-reflective open-boundary scheme (lbm_case.open_bc_scheme) */
#define LBM_OPEN_CHARACTERISTIC 0  /* outgoing characteristic against exponentially
                                      averaged reference values (include/updateGrid.h:250-347) */
#define LBM_OPEN_IMPEDANCE      1  /* impedance scheme: the given density / normal
                                      velocity is clamped to within a density tolerance
                                      of the non-reflecting state computed from the
                                      previous completed boundary state
                                      (cases/nonReflectiveTest/updateGrid_SCHLAFFER_IMPEDANCE_SCHEME.h) */

/* One static body: a triangle soup in mm (the reference's gridStaticSTLs
 * entry; its index is the body's wallID). */
typedef struct lbm_body {
    const float* triangles;     /* [triangle_count][9]: ax ay az bx by bz cx cy cz */
    int   triangle_count;
    int   motion;               /* LBM_WALL_*                                  */
    int   axis;                 /* 0, 1, 2: rotation axis parallel to x, y, z  */
    float origin[3];            /* a point on the rotation axis, mm            */
    float radians_per_second;   /* signed angular speed                        */
} lbm_body;

/* BCStruct (include/types.h:131-136) as a hook fills it.  A hook receives it
 * with the reference's defaults (lbm_default_bc) and the cell's wallID. */
typedef struct lbm_bc {
    float dRho, ux, uy, uz;     /* target / initial / wall values              */
    float gx, gy, gz;           /* body force                                  */
    int   wallID, openBCID;
    int   useIBB, dirichletU, dirichletRho, periodic, nonReflective;
    float nonReflectiveBeta, collisionLimiter, nuMultiplier;
} lbm_bc;

struct lbm_grid_info;
/* A per-cell hook of a reference driver (getOpenBC, getInitialCondition,
 * getLocalBC, include/updateGrid.h:95,256), called on the host while the grid
 * is built, with the cell's (i, j, k) on its level and the level's info. */
typedef void (*lbm_cell_hook)(void* user, lbm_bc* bc, int i, int j, int k, const struct lbm_grid_info* info);
/* getRefinementModifier (include/markerFunctions.h:254-271), called on the host
 * for every cell of every level but the finest while the grids are built:
 * `*mark` arrives as the deep-refinement marker from the walls (and from
 * lbm_case.refine_box) and the hook may set it (1) or clear it (0). */
typedef void (*lbm_refinement_hook)(void* user, int i, int j, int k, int* mark, const struct lbm_grid_info* info);

typedef struct lbm_case {
    /* compile-time constants of a reference driver */
    int   grid_level_count;     /* GRID_LEVEL_COUNT, 1 .. LBM_MAX_LEVELS       */
    int   wall_refinement_count;/* WALL_REFINEMENT_COUNT                       */
    float res_global;           /* RES_GLOBAL, mm                              */
    float nu_phys;              /* NU_PHYS, m^2/s                              */
    float rho_phys;             /* RHO_PHYS, kg/m^3                            */
    float dt_phys_global;       /* DT_PHYS_GLOBAL, s                           */
    float bounds[6];            /* BoundsStruct: xMin,yMin,zMin,xMax,yMax,zMax (mm) */
    int   track_wall_force;     /* TRACK_WALL_FORCE                            */
    int   track_open_boundaries;/* TRACK_OPEN_BOUNDARIES                       */

    /* getOpenBC */
    lbm_face_bc face[6];

    /* getInitialCondition */
    int   ic_kind;
    float ic_dRho, ic_ux, ic_uy, ic_uz;   /* LBM_IC_UNIFORM                   */
    float tgv_u0;               /* LBM_IC_TAYLOR_GREEN: lattice amplitude      */
    float tgv_length;           /* X = x / tgv_length (x in mm)                */

    /* getLocalBC (uniform over the domain) */
    float collision_limiter;    /* BCStruct.collisionLimiter; <= 0 selects AllOne */
    float nu_multiplier;        /* BCStruct.nuMultiplier                       */
    float gx, gy, gz;           /* BCStruct.gx/gy/gz body force, lattice units */
    int   use_ibb;              /* BCStruct.useIBB: 1 interpolated, 0 gamma=1/2 */

    /* gridStaticSTLs */
    int      body_count;
    lbm_body body[LBM_MAX_BODIES];

    /* storage */
    int   storage;              /* LBM_STORE_*                                 */

    /* rotorSTLs: volume-fraction forcing rotors (include/rotorFunctions.h) */
    int       rotor_count;
    lbm_rotor rotor[LBM_MAX_ROTORS];
    int       track_rotor_force;  /* TRACK_ROTOR_FORCE                         */

    /* Per-cell hooks; NULL keeps the tables above.  open_bc_hook replaces the
     * face table for every boundary cell (getOpenBC); initial_condition_hook
     * gives dRho, ux, uy, uz of every cell (getInitialCondition);
     * local_bc_hook gives the wall velocity (bc.ux, uy, uz) of every
     * wall-adjacent cell, called with bc.wallID = its body (the per-wallID
     * branch of getLocalBC).  The kernels keep the collision limiter, nu
     * multiplier, body force and IBB switch uniform over a level: the fields
     * above, or, with a local_bc_hook, what the hook returns for them when it
     * is called once per level for a fluid cell (wallID -1) at the level's
     * first cell (so a hook may, e.g., pick another limiter on level 0). */
    lbm_cell_hook open_bc_hook;
    lbm_cell_hook initial_condition_hook;
    lbm_cell_hook local_bc_hook;
    void*         hook_user;

    /* Refinement (getRefinementModifier) on a level L < grid_level_count - 1:
     * a cell whose centre lies strictly inside refine_box[L] (xMin, yMin, zMin,
     * xMax, yMax, zMax in mm; a box with min >= max on some axis marks
     * nothing) is deep-refined, in addition to the cells the walls mark
     * (WALL_REFINEMENT_COUNT spreads around every finer level's walls);
     * refinement_hook, if set, then sees the marker and may change it. */
    float refine_box[LBM_MAX_LEVELS][6];
    lbm_refinement_hook refinement_hook;

    /* Non-reflective open boundaries (cells whose BC sets nonReflective):
     * LBM_OPEN_*; rho_reflection_tolerance is the impedance scheme's
     * RHO_REFLECTION_TOLERANCE (>= 0; 1 or more turns the scheme off). */
    int   open_bc_scheme;
    float rho_reflection_tolerance;
} lbm_case;

/* The reference's BCStruct defaults (include/types.h:131-136). */
void lbm_default_bc(lbm_bc* bc);

/* Per-level summary (InfoStruct, include/types.h:120-129, plus table sizes). */
typedef struct lbm_grid_info {
    int   grid_id;
    int   cell_count, cell_count_x, cell_count_y, cell_count_z;
    int   row_count;            /* compressed IJKNBR rows                      */
    int   wall_cell_count;      /* wallMap == -3                               */
    int   wall_adjacent_count;  /* Wall.wallAdjacentCount                      */
    int   periodic_count;       /* PeriodicBC.periodicBCCount                  */
    int   open_bc_count;        /* total open-boundary cells over all IDs      */
    int   esotwist_flipper;
    int   iterations_finished;
    int   storage;
    float res, ox, oy, oz, nu, dt_phys;
    unsigned long long grid_memory_bytes;
    /* interfaces to the next finer level (0 on the finest) */
    int   f2c_count;            /* FineToCoarseInterface.interfaceCount        */
    int   c2f_count;            /* CoarseToFineInterface.interfaceCount (blocks) */
    int   leftover_count;       /* CoarseToFineInterface.leftoverCount         */
} lbm_grid_info;

typedef struct lbm_grids lbm_grids;   /* opaque: all levels of one domain */
typedef struct lbm_plan lbm_plan;     /* opaque: host-side tables, no device memory */

/* Last error message of the calling thread ("" when none). */
const char* lbm_last_error(void);

/* Number of visible CUDA devices, or a negative status. */
int lbm_device_count(void);

/* Run the grid construction on the host only: every table of every level
 * and its device footprint, without touching a GPU.  Used for footprint
 * admission before allocation and for table parity checks.
 * Replaces the host-visible part of buildGrids (include/gridBuilderFunctions.h:1577-1649,
 * including the per-level memory accounting printed at :1630-1663). */
int lbm_plan_grids(const lbm_case* c, lbm_plan** out, long long* fluid_updates_per_iteration);
void lbm_free_plan(lbm_plan* p);
int lbm_plan_level_count(lbm_plan* p);
int lbm_plan_info(lbm_plan* p, int level, lbm_grid_info* out);
/* Same array ids as lbm_read_array except the device state: LBM_ARRAY_F,
 * LBM_ARRAY_MACRO, LBM_ARRAY_WALL_FORCE, LBM_ARRAY_OPEN_REFERENCE and
 * LBM_ARRAY_OPEN_CUMULATIVE. */
int lbm_plan_read_array(lbm_plan* p, int level, int which, void* host, size_t bytes);

/* Build every grid level on the current CUDA device, allocate the populations
 * and apply the initial condition.
 * Replaces buildGrids (include/gridBuilderFunctions.h:1577-1670) together with
 * applyInitialCondition (include/boundaryConditions/applyInitialCondition.h:8-84).
 * `fluid_updates_per_iteration` receives Σ_level (cells − wall cells)·2^level
 * (include/gridBuilderFunctions.h:1601-1608); it may be NULL.
 * With LBM_STORE_F16 / LBM_STORE_BF16, every store of a collided, boundary
 * or interpolated population rounds stochastically (up with probability equal
 * to the distance from the lower representable neighbour, so the rounding
 * error has zero mean and does not repeat step after step in a steady state);
 * the random bits are a hash of a per-level step seed, the cell and the
 * direction, so a run is deterministic and reproducible.  The initial
 * condition, periodic ghost copies and lbm_write_f round to nearest. */
int lbm_build_grids(const lbm_case* c, lbm_grids** out,
                    long long* fluid_updates_per_iteration);

/* Release all device and host memory of a domain. */
void lbm_free_grids(lbm_grids* g);

/* Launch subsequent work on this CUDA stream (cudaStream_t passed as void*,
 * NULL = legacy default stream). */
int lbm_set_stream(lbm_grids* g, void* stream);

/* Advance `coarse_steps` coarse time steps (asynchronous on the grid stream).
 * Replaces the driver loop `updateAllGrids(grids, 0)`
 * (include/updateGrid.h:388-396, one call per coarse step). */
int lbm_update_all_grids(lbm_grids* g, int coarse_steps);

/* Many-domain batch: advance `count` independent domains by `coarse_steps`,
 * issuing every domain's step schedule on its own stream, step by step
 * interleaved, so that the kernels of different domains overlap on the GPU
 * (small domains alone leave it mostly idle between launches).  Give each
 * grids object its own stream with lbm_set_stream; domains sharing a stream
 * run one after the other.  Asynchronous like lbm_update_all_grids; each
 * domain's result is the one it gets when stepped alone.
 * No counterpart in the reference (one domain per driver process). */
int lbm_update_batch(lbm_grids* const* grids, int count, int coarse_steps);

/* Packed batch: single-level domains (without rotors, of one storage type,
 * FP32, FP16 or BF16) advanced by ONE persistent collide-stream launch over a
 * packed table of all domains' work items (per domain its listed-cell chunks
 * and 128-cell bulk tiles, with an item counter each: a CTA works through its
 * home domain, then helps the others), one open-boundary launch over all
 * domains' chunks
 * and one periodic-ghost launch, instead of a launch set per domain; step
 * pairs replay as a CUDA graph.  A member's result is bit-identical to the
 * member stepped as a batch of one (the per-item work does not depend on the
 * other members) and agrees to FP32 rounding with lbm_update_all_grids, whose
 * kernel takes the level descriptor as a kernel parameter.  The batch runs on its own stream, ordered after the
 * work already queued on the members' streams and before what they get
 * next.  Members keep their own state (trackers, readbacks, lbm_update_all_grids
 * between batch updates); all members must be at the same esotwist parity
 * when lbm_batch_update is called (a domain that has made an odd number of
 * steps more than the others steps once on its own first).  Free the batch
 * before its members.  No counterpart in the reference (one domain per
 * driver process). */
typedef struct lbm_batch lbm_batch;
typedef struct lbm_batch_info {
    int domain_count;
    long long cells;          /* sum of the members' cells (ghosts included) */
    int collide_items;        /* collide-stream work items of all members     */
    int open_chunks;          /* open-boundary CTAs per step                  */
    int periodic_cells;       /* periodic ghost cells per step                */
    int launches_per_step;    /* kernels one packed step launches (<= 3)      */
} lbm_batch_info;
int lbm_batch_create(lbm_grids* const* grids, int count, lbm_batch** out);
int lbm_batch_update(lbm_batch* b, int coarse_steps);
/* Device time of `coarse_steps` packed steps (graphs captured first). */
int lbm_batch_time_steps(lbm_batch* b, int coarse_steps, float* ms);
int lbm_batch_get_info(lbm_batch* b, lbm_batch_info* out);
void lbm_batch_free(lbm_batch* b);

/* Graph replay of the step schedule.  lbm_update_all_grids and
 * lbm_update_batch advance step pairs by launching a CUDA graph of two steps
 * (captured on first use, one per starting esotwist parity) instead of the
 * individual kernels; domains with rotors, whose rotating frame is host
 * state, launch directly.  Results are identical either way.  `enabled` = 0
 * turns replay off for these grids (LBM3_GRAPHS=0 turns it off everywhere).
 * No counterpart in the reference. */
int lbm_set_graphs(lbm_grids* g, int enabled);

/* Time `steps` coarse steps as replayed graphs (graphs captured before the
 * timed region), device time in *ms; no per-kernel events.
 * No counterpart in the reference. */
int lbm_time_steps_graph(lbm_grids* g, int steps, float* ms);

/* Block until the grid stream is idle; returns a pending CUDA error, if any. */
int lbm_synchronize(lbm_grids* g);

/* Time `steps` coarse steps with CUDA events on the grid stream; *ms receives
 * the elapsed device time. */
int lbm_time_steps(lbm_grids* g, int steps, float* ms);

/* Device time of the collide-stream launches inside the most recent
 * lbm_time_steps call, each bracketed by CUDA events on the grid stream:
 * summed kernel milliseconds and the number of launches. */
int lbm_last_kernel_time(lbm_grids* g, float* kernel_ms, int* launches);
/* Number of kernels the last lbm_time_steps call launched, all kernels of the
 * step schedule (collide-stream, special cells, open boundary, periodic copy).
 * No counterpart in the reference (instrumentation). */
int lbm_last_launch_count(lbm_grids* g, long long* kernels);

int lbm_level_count(lbm_grids* g);
int lbm_get_grid_info(lbm_grids* g, int level, lbm_grid_info* out);

/* Copy a device array of one level to host memory (replaces drivers reading
 * GridStruct fields directly, e.g. cases/taylorGreenVortex/taylorGreenVortexMain.cu:123-156).
 * `bytes` must equal the array size; see LBM_ARRAY_* for element types. */
int lbm_read_array(lbm_grids* g, int level, int which, void* host, size_t bytes);

/* Overwrite the populations of one level (float [27][cellCount], shifted
 * f_i - w_i, in the current esotwist slot order). */
int lbm_write_f(lbm_grids* g, int level, const float* host, size_t bytes);

/* Normalised kinetic energy of the Taylor–Green driver
 * (cases/taylorGreenVortex/taylorGreenVortexMain.cu:116-180), accumulated in
 * FP64 on the device.  `u_ref_phys` is the physical reference velocity (m/s)
 * and `domain_length` the physical periodic length (mm). */
int lbm_kinetic_energy(lbm_grids* g, float u_ref_phys, float domain_length,
                       double* out);

/* The same kinetic energy for callers that cannot allocate device memory:
 * a serving loop that admits domains by HBM footprint has committed all of
 * it, and an allocation on the side can fail or (cudaFree) synchronize the
 * device mid-pipeline.  Its scratch (FP64 partial sums of 256-cell blocks and
 * the total) is a fixed static device array of 128 KB that every GPU loading
 * the library holds until exit, so the call allocates nothing.  Every level
 * must have at most LBM_KINETIC_ENERGY_NOALLOC_MAX_CELLS cells; larger ones
 * are rejected with LBM_ERR_INVALID.  Call it with the grids' device current;
 * its first call on a device looks up the array's device address, so make
 * that call before any stream capture begins.  The address is kept for the
 * life of the process: after a cudaDeviceReset of a device, do not call this
 * entry point on that device again.  All calls on a device share
 * the array: calls that overlap on the GPU race.  The sum is deterministic
 * (fixed order, no atomics).
 * No counterpart in the reference. */
#define LBM_KINETIC_ENERGY_NOALLOC_MAX_CELLS 4194304
int lbm_kinetic_energy_noalloc(lbm_grids* g, float u_ref_phys, float domain_length,
                               double* out);

/* Global FP64 accumulators over the fluid cells of every level (walls,
 * periodic ghosts and interface duplicates excluded), summed on the device:
 * out = {mass [kg], mass minus the rest mass [kg], momentum x, y, z [kg m/s]
 * (the domain's mass flow rate times its length), fluid cells, sum of rho and
 * sum of dRho in lattice units}.  The momentum is the sum of c_i f_i, without
 * the half body-force shift.  Mass drift of a closed domain is the change of
 * out[7] between calls.
 * The north star's global mass and flow-rate accumulators; the reference
 * tracks only open-boundary and wall quantities (include/trackerFunctions.h:120-497). */
int lbm_global_sums(lbm_grids* g, double* out);

/* Momentum-exchange force and torque on one body (wallID), accumulated in
 * FP64 on the device over the wall-adjacent cells and averaged over the
 * steps since the last reset: out = {Fx, Fy, Fz [N], Tx, Ty, Tz [N m]} about
 * the coordinate origin.  `reset` != 0 zeroes the accumulators afterwards.
 * Replaces the wall branch of updateTracker (include/trackerFunctions.h:366-497). */
int lbm_wall_force(lbm_grids* g, int wall_id, int reset, double* out);

/* Flow through one open boundary (openBCID), from the sums the open-boundary
 * update accumulates while the case's track_open_boundaries is set, averaged
 * over the steps since the last tracker reset and converted to SI units:
 * out = {area [m^2], area-averaged normal velocity [m/s], mass flow [kg/s],
 * momentum thrust [N], area-averaged pressure [Pa], pressure power [W],
 * normal kinetic power [W]}; the normal is the outer normal.  Sums are FP64
 * on the device.  `reset` != 0 then resets every tracker accumulator of the
 * grids (wall forces and open-boundary sums), as updateTracker does.
 * Replaces the open-boundary branch of updateTracker
 * (include/trackerFunctions.h:127-214). */
int lbm_open_boundary_flow(lbm_grids* g, int open_bc_id, int reset, double* out);

/* Rotor tables of one level of a plan or of built grids. */
int lbm_plan_rotor_info(lbm_plan* p, int level, int rotor, lbm_rotor_info* out);
int lbm_get_rotor_info(lbm_grids* g, int level, int rotor, lbm_rotor_info* out);

/* Change a rotor's speed between steps, as drivers set
 * rotors[i].Info.radiansPerSecond (cases/BruteforcePumpOnly/BruteforcePump.cu:226-229). */
int lbm_set_rotor_speed(lbm_grids* g, int rotor, float radians_per_second);

/* Force and torque the rotor exerts on the fluid, in the rotor frame,
 * averaged over the steps since the last tracker reset and summed in FP64 on
 * the device: out = {Fx, Fy, Fz [N], Tx, Ty, Tz [N m]} about the rotor
 * origin.  `reset` != 0 then resets every tracker accumulator.
 * Replaces the rotor branch of updateTracker (include/trackerFunctions.h:225-300). */
int lbm_rotor_force(lbm_grids* g, int rotor, int reset, double* out);

/* Section planes of lbm_flow_report; the normal is the +axis direction. */
#define LBM_PLANE_XY 0   /* cut at z */
#define LBM_PLANE_ZY 1   /* cut at x */
#define LBM_PLANE_ZX 2   /* cut at y */

/* Flow through a section plane (FlowReportStruct): the cell layer nearest to
 * the coordinate `cut` (mm), cropped to `bounds` {xMin, yMin, zMin, xMax,
 * yMax, zMax} (mm; NULL or all zero: no crop).  Pixels that are walls or
 * mostly rotor volume are left out.  out = {area-averaged normal velocity
 * [m/s], mass flow [kg/s], momentum thrust [N], area-averaged pressure [Pa],
 * pressure power [W], normal kinetic power [W], fluid area [mm^2]}; sums in
 * FP64 on the device.  A cut outside the grid is LBM_ERR_INVALID.  With
 * several levels the cut is the finest level's layer and the report is taken
 * on a section image at the finest level whose pixel count fits 16,000,000,
 * filled level by level (finer levels overwrite coarser ones; a coarser level
 * whose layers bracket the cut blends the two); areas are that level's pixels.
 * Replaces getFlowReportXY/ZY/ZX (include/flowReportFunctions.h:11-373). */
int lbm_flow_report(lbm_grids* g, int plane, float cut, const float* bounds, double* out);

/* Write every cell of every level to a legacy ASCII VTK file (POLYDATA, one
 * vertex per cell centre in mm) with point data wall (0/1), velocity_m_s,
 * pressure_Pa, grid_id, grid_resolution_mm and interface_overlap (0/1);
 * walls carry zero velocity and pressure.  Fields come from the device state
 * at the call (FP64 accumulators are not involved).
 * Replaces exportVTK (include/exportVTK.h:17-158). */
int lbm_export_vtk(lbm_grids* g, const char* filename);

/* Checkpoint and resume (preemption of long runs and of served domains).
 * The state is everything a run carries from step to step: the populations at
 * their storage precision, the esotwist flipper, the iteration counters, the
 * open-boundary reference and cumulative values, the wall and rotor force
 * accumulators, and the rotor angles and speeds.  It is restored into grids
 * built from the same case; a mismatch of sizes is LBM_ERR_INVALID.
 * No counterpart in the reference. */
int lbm_state_bytes(lbm_grids* g, size_t* bytes);
int lbm_save_state(lbm_grids* g, void* host, size_t bytes);
int lbm_load_state(lbm_grids* g, const void* host, size_t bytes);

/* Cell-wise collision on a device batch of shifted populations laid out as
 * float [27][n] (structure of arrays), in place.
 * Replaces applyCollision (include/applyCollision.h:17-491) applied per cell
 * with a uniform BCStruct {gx,gy,gz, collisionLimiter, nuMultiplier}. */
int lbm_apply_collision_batch(float* d_f, int n, float nu,
                              float collision_limiter, float nu_multiplier,
                              float gx, float gy, float gz, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* LBM3_B200_H */
