// lbm3/gridBuilderFunctions.h — buildGrids and GridStruct of the reference
// driver API (include/gridBuilderFunctions.h:1577-1670) over the C ABI.
//
// Include after the driver's constants (RES_GLOBAL, NU_PHYS, RHO_PHYS,
// DT_PHYS_GLOBAL, GRID_LEVEL_COUNT, WALL_REFINEMENT_COUNT, TRACK_WALL_FORCE,
// TRACK_ROTOR_FORCE, TRACK_OPEN_BOUNDARIES) and its four hooks
// (getRefinementModifier, getInitialCondition, getOpenBC, getLocalBC).  The
// hooks are evaluated on the host while the grid is built:
//   getOpenBC             every boundary cell (kind, targets, openBCID, non-reflective)
//   getInitialCondition   every cell (dRho, ux, uy, uz)
//   getLocalBC            every wall-adjacent cell with BC.wallID set (wall
//                         velocity); once with wallID -1 for the uniform
//                         collision limiter, nu multiplier, body force and
//                         IBB switch the kernels apply everywhere
//   getRefinementModifier every cell of every level but the finest, with the
//                         marker the walls set (markRefinementCells)
#pragma once

#include "types.h"

namespace lbm3_detail {

inline InfoStruct infoFromGridInfo(const lbm_grid_info& g) {
    InfoStruct I;
    I.gridID = static_cast<float>(g.grid_id);
    I.gridMemoryBytes = g.grid_memory_bytes;
    I.iterationsFinished = g.iterations_finished;
    I.res = g.res;
    I.ox = g.ox;
    I.oy = g.oy;
    I.oz = g.oz;
    I.nu = g.nu;
    I.dtPhys = g.dt_phys;
    I.cellCountX = g.cell_count_x;
    I.cellCountY = g.cell_count_y;
    I.cellCountZ = g.cell_count_z;
    I.cellCount = g.cell_count;
    I.esotwistFlipper = g.esotwist_flipper != 0;
    return I;
}

inline BCStruct bcFromC(const lbm_bc& h) {
    BCStruct b;
    b.dRho = h.dRho; b.ux = h.ux; b.uy = h.uy; b.uz = h.uz;
    b.gx = h.gx; b.gy = h.gy; b.gz = h.gz;
    b.wallID = h.wallID; b.openBCID = h.openBCID;
    b.useIBB = h.useIBB != 0; b.dirichletU = h.dirichletU != 0; b.dirichletRho = h.dirichletRho != 0;
    b.periodic = h.periodic != 0; b.nonReflective = h.nonReflective != 0;
    b.nonReflectiveBeta = h.nonReflectiveBeta; b.collisionLimiter = h.collisionLimiter;
    b.nuMultiplier = h.nuMultiplier;
    return b;
}

inline void bcToC(const BCStruct& b, lbm_bc* h) {
    h->dRho = b.dRho; h->ux = b.ux; h->uy = b.uy; h->uz = b.uz;
    h->gx = b.gx; h->gy = b.gy; h->gz = b.gz;
    h->wallID = b.wallID; h->openBCID = b.openBCID;
    h->useIBB = b.useIBB; h->dirichletU = b.dirichletU; h->dirichletRho = b.dirichletRho;
    h->periodic = b.periodic; h->nonReflective = b.nonReflective;
    h->nonReflectiveBeta = b.nonReflectiveBeta; h->collisionLimiter = b.collisionLimiter;
    h->nuMultiplier = b.nuMultiplier;
}

// trampolines from the C ABI's hooks to the driver's functions
inline void openBCHook(void*, lbm_bc* bc, int i, int j, int k, const lbm_grid_info* info) {
    BCStruct b = bcFromC(*bc);
    ::getOpenBC(b, i, j, k, infoFromGridInfo(*info));
    bcToC(b, bc);
}
inline void initialConditionHook(void*, lbm_bc* bc, int i, int j, int k, const lbm_grid_info* info) {
    BCStruct b = bcFromC(*bc);
    ::getInitialCondition(b, i, j, k, infoFromGridInfo(*info));
    bcToC(b, bc);
}
inline void localBCHook(void*, lbm_bc* bc, int i, int j, int k, const lbm_grid_info* info) {
    BCStruct b = bcFromC(*bc);
    ::getLocalBC(b, i, j, k, infoFromGridInfo(*info));
    bcToC(b, bc);
}

inline void refinementHook(void*, int i, int j, int k, int* mark, const lbm_grid_info* info) {
    bool m = *mark != 0;
    ::getRefinementModifier(i, j, k, m, infoFromGridInfo(*info));
    *mark = m ? 1 : 0;
}

inline void check(int rc) {
    if (rc < 0) throw std::runtime_error(lbm_last_error());
}

struct GridsDeleter {
    void operator()(lbm_grids* g) const { lbm_free_grids(g); }
};

}  // namespace lbm3_detail

// GridStruct (include/types.h:230-236): one grid level of a domain.  All
// levels share the domain's device state; Info mirrors InfoStruct and is
// refreshed by updateAllGrids.
struct GridStruct {
    InfoStruct Info;
    std::shared_ptr<lbm_grids> domain;
    int level = 0;

    lbm_grids* handle() const { return domain.get(); }
    void refresh() {
        lbm_grid_info gi;
        lbm3_detail::check(lbm_get_grid_info(domain.get(), level, &gi));
        const InfoStruct fresh = lbm3_detail::infoFromGridInfo(gi);
        const int sinceReset = Info.iterationsSinceTrackerReset;
        const bool useRotors = Info.useRotors;
        Info = fresh;
        Info.iterationsSinceTrackerReset = sinceReset;
        Info.useRotors = useRotors;
    }
    // dRho, ux, uy, uz of every cell (getDRhoUxUyUz of the current state)
    std::vector<float> macro() const {
        std::vector<float> out(4 * static_cast<size_t>(Info.cellCount));
        lbm3_detail::check(lbm_read_array(domain.get(), level, LBM_ARRAY_MACRO, out.data(), out.size() * 4));
        return out;
    }
};

// buildGrids (include/gridBuilderFunctions.h:1577-1670): voxelize the static
// STLs and rotors, build every level and apply the initial condition; returns
// the fluid cell updates of one coarse iteration.
inline long long buildGrids(std::vector<GridStruct>& grids, std::vector<STLStruct>& gridStaticSTLs,
                            std::vector<STLStruct>& rotorSTLs, const BoundsStruct& Bounds) {
    if (GRID_LEVEL_COUNT < 1 || GRID_LEVEL_COUNT > LBM_MAX_LEVELS)
        throw std::runtime_error("buildGrids: GRID_LEVEL_COUNT must be in [1, LBM_MAX_LEVELS]");
    if (gridStaticSTLs.size() > LBM_MAX_BODIES) throw std::runtime_error("buildGrids: too many static STLs");
    if (rotorSTLs.size() > LBM_MAX_ROTORS) throw std::runtime_error("buildGrids: too many rotor STLs");
    lbm_case c;
    std::memset(&c, 0, sizeof(c));
    c.grid_level_count = GRID_LEVEL_COUNT;
    c.wall_refinement_count = WALL_REFINEMENT_COUNT;
    c.res_global = RES_GLOBAL;
    c.nu_phys = NU_PHYS;
    c.rho_phys = RHO_PHYS;
    c.dt_phys_global = DT_PHYS_GLOBAL;
    c.bounds[0] = Bounds.xMin; c.bounds[1] = Bounds.yMin; c.bounds[2] = Bounds.zMin;
    c.bounds[3] = Bounds.xMax; c.bounds[4] = Bounds.yMax; c.bounds[5] = Bounds.zMax;
    c.track_wall_force = TRACK_WALL_FORCE ? 1 : 0;
    c.track_open_boundaries = TRACK_OPEN_BOUNDARIES ? 1 : 0;
    c.track_rotor_force = TRACK_ROTOR_FORCE ? 1 : 0;
    for (int f = 0; f < 6; ++f) c.face[f].kind = LBM_BC_PERIODIC;  // replaced by getOpenBC
    c.ic_kind = LBM_IC_UNIFORM;
    // the uniform part of getLocalBC
    {
        BCStruct b;
        InfoStruct I;
        I.res = RES_GLOBAL;
        I.dtPhys = DT_PHYS_GLOBAL;
        ::getLocalBC(b, 0, 0, 0, I);
        c.collision_limiter = b.collisionLimiter;
        c.nu_multiplier = b.nuMultiplier;
        c.gx = b.gx;
        c.gy = b.gy;
        c.gz = b.gz;
        c.use_ibb = b.useIBB ? 1 : 0;
    }
    c.body_count = static_cast<int>(gridStaticSTLs.size());
    for (size_t b = 0; b < gridStaticSTLs.size(); ++b) {
        c.body[b].triangles = gridStaticSTLs[b].triangles.data();
        c.body[b].triangle_count = gridStaticSTLs[b].triangleCount;
        c.body[b].motion = LBM_WALL_STATIC;  // wall velocity from getLocalBC
    }
    c.rotor_count = static_cast<int>(rotorSTLs.size());
    for (size_t r = 0; r < rotorSTLs.size(); ++r) {
        const STLStruct& R = rotorSTLs[r];
        c.rotor[r].triangles = R.triangles.data();
        c.rotor[r].triangle_count = R.triangleCount;
        c.rotor[r].axis = R.rotateAlongX ? 0 : R.rotateAlongY ? 1 : 2;
        c.rotor[r].origin[0] = R.ox;
        c.rotor[r].origin[1] = R.oy;
        c.rotor[r].origin[2] = R.oz;
        c.rotor[r].radians_per_second = R.radiansPerSecond;
    }
    c.storage = LBM_STORE_F32;
    c.open_bc_hook = &lbm3_detail::openBCHook;
    c.initial_condition_hook = &lbm3_detail::initialConditionHook;
    c.local_bc_hook = &lbm3_detail::localBCHook;
    c.refinement_hook = &lbm3_detail::refinementHook;
    lbm_grids* raw = nullptr;
    long long fluidUpdates = 0;
    lbm3_detail::check(lbm_build_grids(&c, &raw, &fluidUpdates));
    std::shared_ptr<lbm_grids> domain(raw, lbm3_detail::GridsDeleter{});
    grids.resize(static_cast<size_t>(lbm_level_count(raw)));
    for (size_t l = 0; l < grids.size(); ++l) {
        grids[l].domain = domain;
        grids[l].level = static_cast<int>(l);
        grids[l].refresh();
    }
    return fluidUpdates;
}
