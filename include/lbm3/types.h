// lbm3/types.h — the reference's driver-facing types over the C ABI.
//
// A reference case driver (e.g. cases/taylorGreenVortex/taylorGreenVortexMain.cu)
// defines its constants, includes the types header, defines its four
// __cuda_callable__ hooks, then includes the grid builder and time-step
// headers.  This header set keeps that structure and those names:
//   lbm3/types.h                 InfoStruct, BCStruct, BoundsStruct, STLStruct,
//                                getXYZFromIJKCellIndex, readSTL
//   lbm3/gridBuilderFunctions.h  GridStruct, buildGrids
//   lbm3/updateGrid.h            updateAllGrids and the trackers
// Device state lives behind the C ABI (include/lbm3_b200.h): drivers read
// fields through the GridStruct accessors instead of TNL views.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../lbm3_b200.h"

#ifndef __cuda_callable__
#ifdef __CUDACC__
#define __cuda_callable__ __host__ __device__
#else
#define __cuda_callable__
#endif
#endif

// BoundsStruct (include/types.h:114-118)
struct BoundsStruct {
    float xMin = 0.f, yMin = 0.f, zMin = 0.f, xMax = 0.f, yMax = 0.f, zMax = 0.f;
    float rxMax = 0.f, ryMax = 0.f, rzMax = 0.f;
};

// InfoStruct (include/types.h:120-129): the fields a hook or driver reads.
struct InfoStruct {
    float gridID = 0;
    unsigned long long gridMemoryBytes = 0;
    int iterationsFinished = 0, iterationsSinceTrackerReset = 0;
    float res = 1.f, ox = 0.f, oy = 0.f, oz = 0.f;
    BoundsStruct Bounds;
    float nu = 1.f, dtPhys = 1.f;
    int cellCountX = 0, cellCountY = 0, cellCountZ = 0, cellCount = 0;
    bool esotwistFlipper = false;
    bool useRotors = true;
};

// BCStruct (include/types.h:131-136) with the reference's defaults.
struct BCStruct {
    float dRho = 0.f, ux = 0.f, uy = 0.f, uz = 0.f;
    float gx = 0.f, gy = 0.f, gz = 0.f;
    int wallID = -1, openBCID = 0;
    bool useIBB = true, dirichletU = false, dirichletRho = false, periodic = false;
    bool nonReflective = true;
    float nonReflectiveBeta = 7.f, collisionLimiter = 0.05f, nuMultiplier = 1.f;
};

// STLStruct (include/types.h:244-256): the triangles of one body or rotor
// (mm), nine floats each, and their bounds.
struct STLStruct {
    int triangleCount = 0;
    std::vector<float> triangles;
    BoundsStruct Bounds;
    // rotor frame of a rotor STL (RotorInfoStruct, include/types.h:206-210)
    float ox = 0.f, oy = 0.f, oz = 0.f, radiansPerSecond = 0.f;
    bool rotateAlongX = false, rotateAlongY = false, rotateAlongZ = false;
};

// getXYZFromIJKCellIndex (include/cellFunctions.h:103-108)
__cuda_callable__ inline void getXYZFromIJKCellIndex(const int& iCell, const int& jCell, const int& kCell, float& x,
                                                     float& y, float& z, const InfoStruct& Info) {
    x = iCell * Info.res + Info.ox;
    y = jCell * Info.res + Info.oy;
    z = kCell * Info.res + Info.oz;
}

// readSTL (include/STLFunctions.h:317-460) without the device copy: binary
// STL, triangles with two identical vertices dropped, bounds of the rest.
inline void readSTL(STLStruct& STL, const std::string& filename) {
    std::ifstream file(filename, std::ios::binary);
    if (!file.is_open()) throw std::runtime_error("Failed to open STL file");
    char header[80];
    file.read(header, 80);
    uint32_t count = 0;
    file.read(reinterpret_cast<char*>(&count), 4);
    STL.triangles.clear();
    STL.Bounds = BoundsStruct{};
    STL.Bounds.xMin = STL.Bounds.yMin = STL.Bounds.zMin = 3.402823466e38f;
    STL.Bounds.xMax = STL.Bounds.yMax = STL.Bounds.zMax = -3.402823466e38f;
    for (uint32_t t = 0; t < count; ++t) {
        float rec[12];
        uint16_t attr;
        file.read(reinterpret_cast<char*>(rec), 48);
        file.read(reinterpret_cast<char*>(&attr), 2);
        if (!file) throw std::runtime_error("truncated STL file: " + filename);
        const float* v = rec + 3;  // the normal is skipped
        const bool ab = v[0] == v[3] && v[1] == v[4] && v[2] == v[5];
        const bool cb = v[6] == v[3] && v[7] == v[4] && v[8] == v[5];
        const bool ca = v[6] == v[0] && v[7] == v[1] && v[8] == v[2];
        if (ab || cb || ca) continue;
        STL.triangles.insert(STL.triangles.end(), v, v + 9);
        for (int p = 0; p < 3; ++p) {
            STL.Bounds.xMin = std::min(STL.Bounds.xMin, v[3 * p]);
            STL.Bounds.yMin = std::min(STL.Bounds.yMin, v[3 * p + 1]);
            STL.Bounds.zMin = std::min(STL.Bounds.zMin, v[3 * p + 2]);
            STL.Bounds.xMax = std::max(STL.Bounds.xMax, v[3 * p]);
            STL.Bounds.yMax = std::max(STL.Bounds.yMax, v[3 * p + 1]);
            STL.Bounds.zMax = std::max(STL.Bounds.zMax, v[3 * p + 2]);
        }
    }
    STL.triangleCount = static_cast<int>(STL.triangles.size() / 9);
}
