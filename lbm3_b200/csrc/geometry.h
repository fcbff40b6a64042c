// Static geometry for grid construction: triangle soups, spatial bins, the
// integer ray-casting voxelizer and per-ray solid intervals.
//
// The voxelizer follows the reference's voxelizeSTL
// (include/voxelizerFunctions.h:5-535): triangles are snapped to an integer
// grid 1000x finer than the lattice with odd coordinates while rays sit on
// even ones, a ray (i, j) is tested against each triangle with exact 64-bit
// edge functions (ties on an edge resolved by the same above/below rules),
// the hit height is evaluated on the float triangle and stored as
// k = ceil(z / res), and every ray's hits are sorted so that consecutive
// pairs [kStart, kEnd) are solid.  Work is organised per triangle on the
// host; since the hit lists are sorted afterwards, the order in which hits
// are found does not matter.
#pragma once

#include <cstdint>
#include <vector>

namespace lbm {

struct Triangles {
    int count = 0;
    std::vector<float> ax, ay, az, bx, by, bz, cx, cy, cz;
    float xMin = 0, yMin = 0, zMin = 0, xMax = 0, yMax = 0, zMax = 0;
    // spatial bins (sortSTLToBins, include/STLFunctions.h:5-128)
    float binSize = 0, oxBin = 0, oyBin = 0, ozBin = 0;
    int binCountX = 0, binCountY = 0, binCountZ = 0;
    std::vector<int> firstInBin, bin;
};

// readSTL's triangle handling (include/STLFunctions.h:317-462): triangles with
// two identical vertices are dropped; bounds over the remaining vertices.
void loadTriangles(const float* tri9, int n, Triangles& out);

// Spatial bins with the reference's size rule (about 10 triangles per bin)
// and tolerance; `resGlobal` is the coarsest lattice spacing.
void sortToBins(Triangles& t, float resGlobal);

// Sorted solid intervals along z for every (i, j) ray of a level.
struct RayMap {
    int nx = 0, ny = 0;
    std::vector<long long> scan;  // [nx*ny + 1]
    std::vector<int> hits;        // pairs kStart, kEnd per ray
};

// voxelizeSTL for one body on a level with origin (ox, oy, oz), spacing res and
// nx*ny rays.  Throws on an empty body.
void voxelize(const Triangles& t, float ox, float oy, float oz, float res, int nx, int ny, RayMap& out);

// sumRayMaps (include/voxelizerFunctions.h:537-690): union of solid intervals.
void unionRayMaps(RayMap& sum, const RayMap& bonus);

// markWallCells (include/markerFunctions.h:18-55): is cell (i, j, k) solid?
bool isSolid(const RayMap& m, int i, int j, int k);

// markSingleFinerFluid (include/markerFunctions.h:57-112): does the coarse
// cell (i, j, k) cover at least one fluid cell of the `downsample`x finer map?
bool coarseHasFluid(const RayMap& fine, int downsample, int i, int j, int k);

// markSingleFinerWall (include/markerFunctions.h:174-220): does the coarse
// cell (i, j, k) cover at least one solid cell of the `downsample`x finer map?
bool coarseHasWall(const RayMap& fine, int downsample, int i, int j, int k);

// intersectRayTriangle (include/boundaryConditions/interpolatedBouncebackFunctions.h:400-480),
// ray from the origin along e; returns the ray parameter t.
bool intersectRayTriangle(float ax, float ay, float az, float bx, float by, float bz, float cx, float cy,
                          float cz, float ex, float ey, float ez, float edgeTol, float& t);

}  // namespace lbm
