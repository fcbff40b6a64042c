// A Taylor-Green vortex case driver written the way the reference's drivers
// are (cases/taylorGreenVortex/taylorGreenVortexMain.cu): compile-time
// constants, the types header, four __cuda_callable__ hooks, then the grid
// builder and time-step headers; here against this library's include/lbm3/.
// Usage: tgv_driver <steps>; prints "steps energy" lines.
#include <cstdio>
#include <cstdlib>

constexpr float PI = 3.14159265358979323846f;
constexpr int cellsPerDomain = 32;
#ifndef TGV_LEVELS
#define TGV_LEVELS 1
#endif
// one level, or the central cube refined on a second level (the reference's
// refined run, cases/taylorGreenVortex/taylorGreenVortexMain.cu:8-12)
constexpr int GRID_LEVEL_COUNT = TGV_LEVELS;
constexpr float reynoldsNumber = 1600.f;
constexpr float machNumber = 0.1f;
constexpr float referenceLengthPhys = 1000.f;  // mm
constexpr float uInitialPhys = 1.f;            // m/s
constexpr float RHO_PHYS = 1.f;                // kg/m3
constexpr float domainSizePhys = 2.f * PI * referenceLengthPhys;
constexpr float uInitial = machNumber * 0.5773502691896258f;
constexpr float RES_GLOBAL = domainSizePhys / cellsPerDomain;
constexpr float NU_PHYS = uInitialPhys * (referenceLengthPhys / 1000.f) / reynoldsNumber;
constexpr float DT_PHYS_GLOBAL = (uInitial / uInitialPhys) * (RES_GLOBAL / 1000.f);
constexpr int WALL_REFINEMENT_COUNT = 0;
constexpr bool TRACK_WALL_FORCE = false;
constexpr bool TRACK_ROTOR_FORCE = false;
constexpr bool TRACK_OPEN_BOUNDARIES = false;

#include "lbm3/types.h"

__cuda_callable__ void getRefinementModifier(const int& iCell, const int& jCell, const int& kCell,
                                             bool& refinementMarker, const InfoStruct& Info) {
    refinementMarker = false;
    if (GRID_LEVEL_COUNT == 1 || Info.gridID != 0) return;
    float x, y, z;
    getXYZFromIJKCellIndex(iCell, jCell, kCell, x, y, z, Info);
    const float half = 0.25f * domainSizePhys;
    refinementMarker = x > -half && x < half && y > -half && y < half && z > -half && z < half;
}

__cuda_callable__ void getInitialCondition(BCStruct& BC, const int& iCell, const int& jCell, const int& kCell,
                                           const InfoStruct& Info) {
    float x, y, z;
    getXYZFromIJKCellIndex(iCell, jCell, kCell, x, y, z, Info);
    const float X = x / referenceLengthPhys;
    const float Y = y / referenceLengthPhys;
    const float Z = z / referenceLengthPhys;
    BC.ux = uInitial * std::sin(X) * std::cos(Y) * std::cos(Z);
    BC.uy = -uInitial * std::cos(X) * std::sin(Y) * std::cos(Z);
    BC.uz = 0.f;
    BC.dRho = (3.f * uInitial * uInitial / 16.f) * (std::cos(2.f * X) + std::cos(2.f * Y)) *
              (2.f + std::cos(2.f * Z));
}

__cuda_callable__ void getOpenBC(BCStruct& BC, const int& iCell, const int& jCell, const int& kCell,
                                 const InfoStruct& Info) {
    BC.periodic = true;
}

__cuda_callable__ void getLocalBC(BCStruct& BC, const int& iCell, const int& jCell, const int& kCell,
                                  const InfoStruct& Info) {
}

#include "lbm3/gridBuilderFunctions.h"
#include "lbm3/updateGrid.h"

static double kineticEnergy(std::vector<GridStruct>& grids) {
    double e = 0.0;
    if (lbm_kinetic_energy(grids[0].handle(), uInitialPhys, domainSizePhys, &e) != 0)
        throw std::runtime_error(lbm_last_error());
    return e;
}

int main(int argc, char** argv) {
    const int steps = argc > 1 ? std::atoi(argv[1]) : 10;
    std::vector<STLStruct> gridStaticSTLs(0);
    std::vector<STLStruct> rotorSTLs(0);
    std::vector<GridStruct> grids(GRID_LEVEL_COUNT);
    const float halfDomain = 0.5f * domainSizePhys;
    const float eps = 1e-6f * domainSizePhys;
    BoundsStruct DomainBounds;
    DomainBounds.xMin = -halfDomain - RES_GLOBAL - eps;
    DomainBounds.xMax = halfDomain + RES_GLOBAL + eps;
    DomainBounds.yMin = -halfDomain - RES_GLOBAL - eps;
    DomainBounds.yMax = halfDomain + RES_GLOBAL + eps;
    DomainBounds.zMin = -halfDomain - RES_GLOBAL - eps;
    DomainBounds.zMax = halfDomain + RES_GLOBAL + eps;
    try {
        const long long fluidUpdates = buildGrids(grids, gridStaticSTLs, rotorSTLs, DomainBounds);
        std::printf("fluid_updates %lld cells %d\n", fluidUpdates, grids[0].Info.cellCount);
        std::printf("0 %.17g\n", kineticEnergy(grids));
        for (int it = 1; it <= steps; ++it) updateAllGrids(grids, 0);
        std::printf("%d %.17g\n", grids[0].Info.iterationsFinished, kineticEnergy(grids));
    } catch (const std::exception& e) {
        std::fprintf(stderr, "driver failed: %s\n", e.what());
        return 1;
    }
    return 0;
}
