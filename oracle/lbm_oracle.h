/*
 * lbm_oracle.h — TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference's D3Q27 cumulant time step
 * (stepanmuller/LBM3, include/updateGrid.h and the headers it uses), in
 * plain C with no floating-point contraction.  Only tests/, the smoke check
 * and bench.py's CPU-baseline leg may load it; the product never does.
 *
 * Parity pin: the reference itself needs the absent TNL library, so it is
 * unbuildable here.  The restatement is pinned against the reference's own
 * stored Taylor–Green kinetic-energy curves
 * (cases/taylorGreenVortex/results/COARSE_kineticEnergy.txt and its siblings), committed as
 * fixtures under tests/golden/.
 */
#ifndef LBM_ORACLE_H
#define LBM_ORACLE_H

#include "../include/lbm3_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* BCStruct (include/types.h:131-136) */
typedef struct obc {
    float dRho, ux, uy, uz, gx, gy, gz;
    int wallID, openBCID;
    int useIBB, dirichletU, dirichletRho, periodic, nonReflective;
    float nonReflectiveBeta, collisionLimiter, nuMultiplier;
} obc;

void oracle_default_bc(obc* bc);

/* applyCollision, include/applyCollision.h:17-491 */
void oracle_apply_collision(float f[27], const obc* bc, float nu);
/* the same over a [27][n] batch (OpenMP) */
void oracle_apply_collision_batch(float* f, int n, float nu, float limiter, float nuMultiplier,
                                  float gx, float gy, float gz);
/* getFeq, include/cellFunctions.h:125-148 */
void oracle_get_feq(float dRho, float ux, float uy, float uz, float feq[27]);
/* getDRhoUxUyUz, include/cellFunctions.h:257-279; out = {dRho, ux, uy, uz} */
void oracle_get_drho_u(const float f[27], float out[4]);

/* One grid level: InfoStruct + the tables updateSingleGrid reads. */
typedef struct ogrid {
    /* Info */
    int gridID;
    float res, ox, oy, oz, nu, dtPhys;
    int nx, ny, nz, cellCount;
    int flip;
    int iterationsFinished;
    /* builder arrays (sorted full IJK, NBR plus) */
    int *I, *J, *K, *jPlus, *kPlus;
    unsigned char* geomBits;
    unsigned char* wallMarker;
    /* compressed IJK/NBR */
    int* shifter;
    int rowCount;
    int *rowI, *rowJ, *rowK, *rowJP, *rowKP, *rowJKP;
    int* wallMap;
    int perCount;
    int *perIndex, *perSource;
    int openBCCount;
    /* populations [27][cellCount] */
    float* f;
    long long fluidUpdates;
    /* uniform getLocalBC */
    float limiter, nuMultiplier;
    float gx, gy, gz;
    int useIBB;
    /* wall-adjacent cells */
    int wallCount;
    int *wallIndex;
    unsigned *wallData, *linkLength; /* linkLength [7][wallCount] */
    float *wallVel;                  /* [3][wallCount] */
    float *wallForce;                /* [3][wallCount] */
    int trackWallForce;
    /* open boundaries (OpenBCArrayStruct, all IDs concatenated in ID order) */
    lbm_face_bc face[6];             /* the case's face table (getOpenBC) */
    int openCount;
    int* openIndex;
    float* openRef;                  /* [2][openCount] dRhoRef, uNormalRef */
    float* openCum;                  /* [2][openCount] dRho, uNormal sums */
    int trackOpen;
    int openImpedance;       /* LBM_OPEN_IMPEDANCE for non-reflective face cells */
    float openTolerance;     /* its RHO_REFLECTION_TOLERANCE */
    /* forcing rotors (RotorStruct), set with oracle_set_rotor */
    int rotorCount;
    void* rotors;                    /* orotor[4], private to lbm_oracle.c */
    int trackRotorForce;
    /* the case's getOpenBC hook (NULL: the face table) */
    lbm_cell_hook openHook;
    void* hookUser;
} ogrid;

/* buildGrids (include/gridBuilderFunctions.h:1577-1670) for one level,
 * followed by applyInitialCondition: the oracle's own restatement of the
 * setup chain (readSTL bounds, sortSTLToBins, voxelizeSTL + sumRayMaps,
 * markKeepCells on the skeleton, deleteExcessCells, buildWallMarkers,
 * buildLinkExistenceMarkerArray, buildLinkLengthArray, packWallData, the
 * compressed rows, wallMap, open-boundary and periodic lists, buildRotors).
 * Returns 0 or a negative LBM_ERR_* code. */
int oracle_build(const lbm_case* c, ogrid* g);
void oracle_free(ogrid* g);

/* Single-level grid from tables built elsewhere (the product's host plan),
 * followed by applyInitialCondition.  Arrays are copied. */
int oracle_from_tables(const lbm_case* c, ogrid* g, int cellCount, int rowCount, const int* shifter,
                       const int* rowI, const int* rowJ, const int* rowK, const int* rowJP,
                       const int* rowKP, const int* rowJKP, const int* wallMap, int perCount,
                       const int* perIndex, const int* perSource, int wallCount, const int* wallIndex,
                       const unsigned* wallData, const unsigned* linkLength, const float* wallVel);

/* Σ g and Σ r x g (lattice units, FP64) over the wall-adjacent cells of
 * one wallID: out[6]. */
void oracle_wall_force(const ogrid* g, int wallID, double* out);

/* updateSingleGrid (include/updateGrid.h:16-386) `steps` times. */
void oracle_step(ogrid* g, int steps);

/* the collide-stream of cells [c0, c1) of one step, flipper unchanged
 * (bounded CPU timing sample) */
void oracle_collide_range(ogrid* g, int c0, int c1);

/* getKineticEnergy (cases/taylorGreenVortex/taylorGreenVortexMain.cu:116-180). */
double oracle_kinetic_energy(const ogrid* g, float uRefPhys, float domainLength);

/* FP64 sums over the fluid cells: {sum rho, sum dRho, momentum x, y, z, cells}. */
void oracle_global_sums(const ogrid* g, double* out);

/* dRho,ux,uy,uz of every cell: out[4][cellCount]. */
void oracle_macro(const ogrid* g, float* out);

/* Moment-based open boundary of one cell with outer normal code
 * (nx+5)*100+(ny+5)*10+(nz+5), on full (weight-compensated) populations:
 * applyMBBC, restoreRho and restoreUxUyUz
 * (include/boundaryConditions/{applyMBBC,restoreRho,restoreUxUyUz}.h).
 * Return 0, or -1 for a code without an outer normal. */
int oracle_mbbc_apply(int code, float rho, float ux, float uy, float uz, float f[27]);
int oracle_mbbc_restore_rho(int code, float ux, float uy, float uz, const float f[27], float* rho);
int oracle_mbbc_restore_u(int code, float rho, const float f[27], float u[3]);

/* Attach rotor `r` of a grid: its info (RotorInfoStruct) and tables as a
 * plan built them (rotorMap [blocks], interpolation [64 * nonzero]).  Arrays
 * are copied; force bins [3][27 * nonzero] start at zero.  Returns 0 or -1. */
int oracle_set_rotor(ogrid* g, int r, float res, const float* bounds, const int* cellCount, int axis,
                     const float* origin, float radiansPerSecond, const int* rotorMap, int blocks,
                     const unsigned* interpolation, int nonzero);
/* force bins of rotor r: out[3][27 * nonzero] */
void oracle_rotor_bins(const ogrid* g, int r, float* out);
/* tables of rotor r (built by oracle_build from the case's rotor triangles,
 * or attached with oracle_set_rotor); pointers stay owned by the grid */
int oracle_rotor_tables(const ogrid* g, int r, float* res, float* bounds, int* cellCount, int* blocks, int* nonzero,
                        const int** rotorMap, const unsigned** interpolation);

/* Section-plane sums of getFlowReportGeneral (include/flowReportFunctions.h:11-352)
 * on a single level: cells of layer `layer` along the plane normal (plane 0:
 * z, 1: x, 2: y) inside in-plane index ranges [h0,h1) x [v0,v1); out[6] =
 * {sum u, sum dRho u, sum (1+dRho) u |u|, sum dRho, sum (1+dRho) u^3/2, count}. */
void oracle_flow_sums(const ogrid* g, int plane, int layer, int h0, int h1, int v0, int v1, double* out);

/* number of OpenMP threads the oracle uses */
int oracle_threads(void);

/* Interface lists between a level and the next finer one (InterfaceStruct,
 * include/types.h:198-200). */
typedef struct ointerface {
    int f2cCount, c2fCount, leftCount;
    int *f2cIndex, *f2cChild, *c2fIndex, *c2fChild, *leftIndex, *leftParent, *leftNbr; /* leftNbr [3][leftCount] */
} ointerface;

/* Every level of a domain (std::vector<GridStruct>) and the interfaces
 * between consecutive levels, owned by the coarser one. */
typedef struct odomain {
    int levelCount;
    ogrid level[LBM_MAX_LEVELS];
    ointerface itf[LBM_MAX_LEVELS];
} odomain;

/* buildGrids over all levels (include/gridBuilderFunctions.h:1577-1670):
 * refinement markers, finer grids, excess-cell deletion, walls with parent
 * inheritance, interfaces, then applyInitialCondition on every level.  A
 * single-level case builds exactly as oracle_build.  Returns 0 or a negative
 * LBM_ERR_* code. */
int oracle_domain_build(const lbm_case* c, odomain* d);

/* getFlowReportGeneral over every level of a domain
 * (include/flowReportFunctions.h:11-318): the finest level's layer nearest
 * to `cut` (mm), a section image at the finest level within 16,000,000
 * pixels (cropped to `bounds`, NULL or all zero: none), filled level by
 * level (finer overwrite coarser, a coarser level whose layers bracket the
 * cut blends them); out[6] as oracle_flow_sums over the fluid pixels and
 * *imageLevel the image's level.  Returns 0, or < 0 for a cut outside the
 * grid or an empty / oversized image. */
int oracle_flow_image(const odomain* d, int plane, float cut, const float* bounds, double* out, int* imageLevel);
void oracle_domain_free(odomain* d);
/* updateAllGrids(grids, 0) `coarseSteps` times (include/updateGrid.h:388-396):
 * level L steps 2^L times per coarse step, each finer pair followed by
 * updateInterface (include/updateInterface.h:887-891). */
void oracle_domain_step(odomain* d, int coarseSteps);
/* getKineticEnergy over every level (cases/taylorGreenVortex/taylorGreenVortexMain.cu:116-180) */
double oracle_domain_kinetic_energy(const odomain* d, float uRefPhys, float domainLength);
/* The interface fit of 8 corner records {dRho, ux, uy, uz, kxy, kyz, kxz,
 * kxx-kyy, kxx-kzz} (corners self, +i, +j, +ij, +k, +ik, +jk, +ijk at
 * (+-1/2)^3) evaluated at (x, y, z): out[13] = {dRho, ux, uy, uz, the
 * velocity gradient G[a][b] = d u_a / d x_b row by row}. */
void oracle_fit_check(const float* corners, float x, float y, float z, float* out);

#ifdef __cplusplus
}
#endif
#endif
