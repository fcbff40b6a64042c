// lbm3/updateGrid.h — the time step and trackers of the reference driver API
// over the C ABI: updateAllGrids (include/updateGrid.h:388-396), the wall,
// rotor and open-boundary branches of updateTracker
// (include/trackerFunctions.h:127-497) and exportVTK (include/exportVTK.h:17-158).
#pragma once

#include "gridBuilderFunctions.h"

// One coarse time step of every level (the recursion over finer levels and
// their interfaces runs behind the C ABI).  `level` must be 0.
inline void updateAllGrids(std::vector<GridStruct>& grids, const int level) {
    if (level != 0 || grids.empty()) throw std::runtime_error("updateAllGrids: call with level 0");
    lbm3_detail::check(lbm_update_all_grids(grids[0].handle(), 1));
    for (GridStruct& G : grids) {
        G.refresh();
        G.Info.iterationsSinceTrackerReset++;
    }
}

// {Fx, Fy, Fz [N], Tx, Ty, Tz [N m]} on body wallID, averaged since the last
// reset (FP64 on the device); reset != 0 restarts every tracker accumulator.
inline std::vector<double> getWallForce(std::vector<GridStruct>& grids, int wallID, bool reset) {
    std::vector<double> out(6);
    lbm3_detail::check(lbm_wall_force(grids[0].handle(), wallID, reset ? 1 : 0, out.data()));
    if (reset)
        for (GridStruct& G : grids) G.Info.iterationsSinceTrackerReset = 0;
    return out;
}

// Flow through open boundary openBCID: {area, normal velocity, mass flow,
// thrust, pressure, pressure power, normal kinetic power} (SI).
inline std::vector<double> getOpenBoundaryFlow(std::vector<GridStruct>& grids, int openBCID, bool reset) {
    std::vector<double> out(7);
    lbm3_detail::check(lbm_open_boundary_flow(grids[0].handle(), openBCID, reset ? 1 : 0, out.data()));
    if (reset)
        for (GridStruct& G : grids) G.Info.iterationsSinceTrackerReset = 0;
    return out;
}

inline void exportVTK(const std::vector<GridStruct>& grids, const std::string& filename) {
    lbm3_detail::check(lbm_export_vtk(grids[0].handle(), filename.c_str()));
}
