// Host-side grid construction for one domain (all levels).
//
// Produces the same tables as the reference's buildGrids pipeline
// (include/gridBuilderFunctions.h:1577-1670): k-j-i sorted cell list,
// compressed IJK/NBR rows, wallMap, periodic ghost lists and open-boundary
// lists.  The kernels in step.cu consume exactly these tables.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/lbm3_b200.h"

namespace lbm {

// BCStruct (include/types.h:131-136) as produced by the table-driven hooks.
struct BC {
    float dRho = 0.f, ux = 0.f, uy = 0.f, uz = 0.f;
    float gx = 0.f, gy = 0.f, gz = 0.f;
    int wallID = -1, openBCID = 0;
    bool useIBB = true, dirichletU = false, dirichletRho = false, periodic = false;
    bool nonReflective = true;
    float nonReflectiveBeta = 7.f, collisionLimiter = 0.05f, nuMultiplier = 1.f;
};

// InfoStruct (include/types.h:120-129), the fields the time step uses.
struct Info {
    int gridID = 0;
    float res = 1.f, ox = 0.f, oy = 0.f, oz = 0.f;
    float nu = 1.f, dtPhys = 1.f;
    int nx = 0, ny = 0, nz = 0, cellCount = 0;
    bool esotwistFlipper = false;
    int iterationsFinished = 0;
};

// One open-boundary ID (OpenBCArrayStruct, include/types.h:223-226).
struct OpenBCList {
    int openBCID = 0;
    std::vector<int> index, source;
    int trackFlowCount = 0;
};

// What the open-boundary kernel needs per boundary cell: getOpenBC of the
// cell resolved at setup.  info bits: 0-1 kind (1 velocity, 2 pressure),
// 2 non-reflective, 3-8 outer normal (nx+1, ny+1, nz+1 in 2 bits each),
// 9 track flow, 10-14 row of the normal in the boundary tables, 16-31 openBCID.
struct OpenBCCell {
    int cell;
    int info;
    float dRho, ux, uy, uz, beta;
};

// One rotor of a level (RotorStruct, include/types.h:206-219): the rotor is
// voxelized at half the level spacing; its bounds (with margins) are cut into
// 4x4x4 blocks of interpolation cells, and for every block that holds rotor
// volume each interpolation cell stores its 8 corner counts (0..8 marked
// voxels around the corner) as 4-bit fields.
struct HostRotor {
    float res = 0.f;
    float xMin = 0, yMin = 0, zMin = 0, xMax = 0, yMax = 0, zMax = 0;
    int cntX = 0, cntY = 0, cntZ = 0;
    int axis = 2;
    float ox = 0, oy = 0, oz = 0;
    float radiansPerSecond = 0.f;
    double radiansElapsed = 0.0;
    std::vector<int> rotorMap;            // [blocks] compact index or -1
    std::vector<int> index;               // [nonzero] block of each compact index
    std::vector<uint32_t> interpolation;  // [64 * nonzero]
};

struct HostLevel {
    Info info;
    // builder view: sorted full IJK of the kept cells
    std::vector<int> I, J, K;
    std::vector<int> jPlus, kPlus, jMinus, kMinus;
    std::vector<uint8_t> geomBits;
    std::vector<uint8_t> wallMarker;
    // compressed IJK/NBR (CompressedIJKNBRStruct, include/types.h:162-164)
    std::vector<int> shifter, rowI, rowJ, rowK, rowJP, rowKP, rowJKP;
    // Wall.wallMapArray: -3 wall, -2 no-track fluid, -1 fluid, >=0 wall-adjacent index
    std::vector<int> wallMap;
    // periodic ghost copies (PeriodicBCStruct)
    std::vector<int> perIndex, perSource;
    std::vector<OpenBCList> openBCs;
    std::vector<OpenBCCell> openCells;   // all IDs, in ID then cell order
    int wallCellCount = 0;
    int wallAdjacentCount = 0;
    // wall-adjacent fluid cells (WallStruct, include/types.h:202-204)
    std::vector<int> wallIndex;          // cell of each wall-adjacent entry
    std::vector<uint32_t> wallData;      // bit 0 overlap, bits 1-26 links, 27-31 wallID
    std::vector<uint32_t> linkLength;    // [7][wallAdjacentCount] 8-bit link codes
    std::vector<float> wallVelocity;     // [3][wallAdjacentCount] wall velocity, lattice units
    int linksTotal = 0, linksNotFound = 0;
    // Bulk segments: runs of at most kSegmentCells plain-fluid cells (wallMap
    // -1 or -2) inside one compressed row.  Inside such a run every neighbour
    // index is the run's base plus the lane offset, so the bulk kernel needs
    // one descriptor per tile and no per-cell metadata.
    std::vector<int> segCell, segJP, segKP, segJKP, segLen;
    // cells outside the bulk segments that still collide (wall-adjacent, or
    // whose +1 neighbour wraps around the end of the cell list)
    std::vector<int> specialCells;
    // rotors, and the cells their swept volume can reach (collided with the
    // special cells, since they need their position)
    std::vector<HostRotor> rotors;
    std::vector<uint8_t> rotorCell;
    std::vector<int> rotorCells;          // collided by the rotor kernel
    // cells whose values another level supplies: this level's fine-to-coarse
    // cells and the cells under the parent's coarse-to-fine band (no force or
    // flow tracking, wallMap -2 / wallData bit 0)
    std::vector<uint8_t> interfaceOverlap;
    // Interfaces to the next finer level, owned by the coarse level
    // (InterfaceStruct, include/types.h:198-200).  Fine-to-coarse: coarse cell
    // and its fine child (2i,2j,2k).  Coarse-to-fine: the -x-y-z coarse corner
    // of a full 2x2x2 coarse stencil and the fine cell (2i+1,2j+1,2k+1) that
    // starts the 2x2x2 fine block at its centre.  Leftovers: fine cells of the
    // band no full block covers, their coarse parent and the coarse neighbour
    // per axis on the fine cell's side (-cell-1: the opposite side).
    std::vector<int> f2cIndex, f2cChild, c2fIndex, c2fChild;
    std::vector<int> leftIndex, leftParent, leftNbr;  // leftNbr [3][leftoverCount]
};

constexpr int kSegmentCells = 128;

struct HostDomain {
    lbm_case c;
    std::vector<HostLevel> levels;
    long long fluidUpdatesPerIteration = 0;
};

// getOpenBC from the face table (see lbm_face_bc in include/lbm3_b200.h).
BC evalOpenBC(const lbm_case& c, const Info& info, int i, int j, int k);
// getLocalBC: uniform limiter / nuMultiplier.
void evalLocalBC(const lbm_case& c, BC& bc);
// getInitialCondition.
BC evalInitialCondition(const lbm_case& c, const Info& info, int i, int j, int k);

struct HostLevel;
// getLocalBC as the collide kernels use it, uniform over a level: the case's
// limiter, nu multiplier, body force and IBB switch; with a local_bc_hook,
// what the hook makes of them for a fluid cell (wallID -1) at the level's
// first cell (a driver may, e.g., use another limiter on the coarsest level,
// cases/flowAroundSphere/flowAroundSphereMain.cu:136-149).
BC levelLocalBC(const lbm_case& c, const HostLevel& L);

// buildRotors (include/rotorFunctions.h:315-585) for one level, plus the
// rotorCell marks of the cells inside any rotor's swept cylinder.
void buildRotors(const lbm_case& c, HostLevel& L);

// Split the compressed rows into bulk segments (needs wallMap and rotorCell).
void buildSegments(HostLevel& L);

// Build all tables of every level; throws std::runtime_error on an invalid
// case (the reference's setup throws at the same points).
void buildDomain(const lbm_case& c, HostDomain& out);

}  // namespace lbm
