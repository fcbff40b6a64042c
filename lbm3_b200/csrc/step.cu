// Time-step kernels of one grid level.
//
//   collideStream  K1: fused read -> cumulant collision -> esotwist write
//                  (updateSingleGrid cell lambda, include/updateGrid.h:51-178)
//   openBoundary   K2: moment-based open boundary on the streamed state (:181-355)
//   periodicCopy   K3: ghost <- interior pre-collision copy (:358-382)
//   interfaceExchange  K4-K6: fine-to-coarse, coarse-to-fine and leftover
//                  interface updates between two levels (updateInterface.h)
//   initFeq        equilibrium initial condition (applyInitialCondition.h:23-41)
//   kineticEnergy  FP64 reduction of the Taylor–Green driver's energy
//   macroFields    dRho, ux, uy, uz of every cell
//   collideBatch   cell-wise collision of a [27][n] batch (applyCollision)
//
// One thread per cell; consecutive threads take consecutive cells of the
// k-j-i sorted list, so each of the 27 gathers and 27 scatters of a warp
// touches one contiguous run of a population plane (coalesced, off by at
// most one cell).  The esotwist scheme makes every slot read and written by
// exactly one thread per step, so the kernel needs no second buffer and no
// synchronisation between cells.
#define LBM_MBBC_TYPES_ONLY
#include "builder.h"
#include "interface.cuh"
#include "mbbc.h"
#include "step_launch.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <type_traits>
#include <utility>

// One storage type and one kernel family per translation unit, so the
// kernel sets build in parallel.  LBM3_STEP_PART selects the family:
// 1 the packed persistent collide-stream (one domain, or a batch with its
// open-boundary and periodic launches), 2 the other collide-stream
// variants, 3 open boundary, periodic ghosts, interface and initial
// condition, 4 reductions and field transfers (with the storage-independent
// launchers in the FP32 unit), 0 everything.  Templates a part does not
// launch are never instantiated in its unit.
#ifndef LBM3_STEP_STORAGE
#define LBM3_STEP_STORAGE 0
#endif
#ifndef LBM3_STEP_PART
#define LBM3_STEP_PART 0
#endif
#define LBM3_PART(n) (LBM3_STEP_PART == 0 || LBM3_STEP_PART == (n))
#define LBM3_SHARED_UNIT (LBM3_PART(4) && LBM3_STEP_STORAGE == 0)
#if LBM3_STEP_STORAGE == 1
#define LBM3_STEP_SUFFIX F16
#elif LBM3_STEP_STORAGE == 2
#define LBM3_STEP_SUFFIX BF16
#elif LBM3_STEP_STORAGE == 3
#define LBM3_STEP_SUFFIX F64
#else
#define LBM3_STEP_SUFFIX F32
#endif
#define LBM3_STEP_JOIN2(a, b) a##b
#define LBM3_STEP_JOIN(a, b) LBM3_STEP_JOIN2(a, b)

namespace lbm {

#if LBM3_STEP_STORAGE == 1
using StepStore = __half;
#elif LBM3_STEP_STORAGE == 2
using StepStore = __nv_bfloat16;
#elif LBM3_STEP_STORAGE == 3
using StepStore = double;  // the FP64 build: FP64 storage and arithmetic
#else
using StepStore = float;
#endif

namespace {

constexpr int kBlock = 256;

// ---- rotors ---------------------------------------------------------------
// Volume-fraction forcing towards rigid rotation (processRotor,
// include/rotorFunctions.h:211-304, and its call in the cell update,
// include/updateGrid.h:97-128).  For the cell at (x, y, z): rotate the point
// into each rotor's frame, look up the rotor volume fraction by trilinear
// interpolation of the packed corner counts, and add the forcing
// rho (u_rotor - u) times the smoothstep of the fraction, the fractions of
// all rotors capped at 1 in total.  The collision limiter is scaled by
// 1 - total fraction.  uxPre.. is the velocity after the local body force.
template <class T>
__device__ __forceinline__ void rotorForcing(const DevLevel& g, float x, float y, float z, T rho, T uxPre, T uyPre,
                                             T uzPre, bool trackForce, T& gx, T& gy, T& gz, T& lambda) {
    T cum = T(0);
    for (int r = 0; r < g.rotorCount; ++r) {
        const DevRotor& R = g.rotor[r];
        const float dx = x - R.ox, dy = y - R.oy, dz = z - R.oz;
        float xr = x, yr = y, zr = z;
        if (R.axis == 0) {
            yr = R.oy + R.c * dy + R.s * dz;
            zr = R.oz - R.s * dy + R.c * dz;
        } else if (R.axis == 1) {
            xr = R.ox + R.c * dx - R.s * dz;
            zr = R.oz + R.s * dx + R.c * dz;
        } else {
            xr = R.ox + R.c * dx + R.s * dy;
            yr = R.oy - R.s * dx + R.c * dy;
        }
        if (xr < R.xMin || xr >= R.xMax || yr < R.yMin || yr >= R.yMax || zr < R.zMin || zr >= R.zMax) continue;
        const float xRel = xr - R.xMin, yRel = yr - R.yMin, zRel = zr - R.zMin;
        const int ii = static_cast<int>(xRel / R.res);
        const int jj = static_cast<int>(yRel / R.res);
        const int kk = static_cast<int>(zRel / R.res);
        if (ii >= R.cntX || jj >= R.cntY || kk >= R.cntZ) continue;
        const int bx = R.cntX / 4, by = R.cntY / 4;
        const int block = (kk / 4) * bx * by + (jj / 4) * bx + ii / 4;
        const int map = __ldg(R.rotorMap + block);
        if (map < 0) continue;
        const unsigned packedCounts = __ldg(R.interp + map * 64 + (kk % 4) * 16 + (jj % 4) * 4 + (ii % 4));
        const float xw = xRel / R.res - ii, yw = yRel / R.res - jj, zw = zRel / R.res - kk;
        float v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = static_cast<float>((packedCounts >> (4u * q)) & 0xFu);
        const float v00 = v[0] + xw * (v[1] - v[0]);
        const float v10 = v[2] + xw * (v[3] - v[2]);
        const float v01 = v[4] + xw * (v[5] - v[4]);
        const float v11 = v[6] + xw * (v[7] - v[6]);
        const float v0 = v00 + yw * (v10 - v00);
        const float v1 = v01 + yw * (v11 - v01);
        const float frac = (v0 + zw * (v1 - v0)) * 0.125f;
        if (frac == 0.f) continue;
        // target: rigid rotation about the axis, in lattice units
        float ut[3] = {0.f, 0.f, 0.f};
        if (R.axis == 0) { ut[1] = -R.scale * dz; ut[2] = R.scale * dy; }
        else if (R.axis == 1) { ut[0] = R.scale * dz; ut[2] = -R.scale * dx; }
        else { ut[0] = -R.scale * dy; ut[1] = R.scale * dx; }
        T gxR = rho * (T(ut[0]) - uxPre), gyR = rho * (T(ut[1]) - uyPre), gzR = rho * (T(ut[2]) - uzPre);
        T ff = T(frac) * T(frac) * (T(3) - T(2) * T(frac));
        if (cum + ff > T(1)) {
            ff = T(1) - cum;
            cum = T(1);
        } else {
            cum += ff;
        }
        gxR *= ff;
        gyR *= ff;
        gzR *= ff;
        gx += gxR;
        gy += gyR;
        gz += gzR;
        if (g.trackRotorForce && trackForce) {
            // the force in the rotor frame, binned 3x3x3 per block
            T fx = gxR, fy = gyR, fz = gzR;
            if (R.axis == 0) { fy = R.c * gyR + R.s * gzR; fz = -R.s * gyR + R.c * gzR; }
            else if (R.axis == 1) { fx = R.c * gxR - R.s * gzR; fz = R.s * gxR + R.c * gzR; }
            else { fx = R.c * gxR + R.s * gyR; fy = -R.s * gxR + R.c * gyR; }
            const int iF = max(0, min(2, static_cast<int>(0.75f * ((ii % 4) + xw))));
            const int jF = max(0, min(2, static_cast<int>(0.75f * ((jj % 4) + yw))));
            const int kF = max(0, min(2, static_cast<int>(0.75f * ((kk % 4) + zw))));
            const int bin = map * 27 + kF * 9 + jF * 3 + iF;
            const int nb = 27 * R.nonzero;
            atomicAdd(R.force + bin, static_cast<float>(fx));
            atomicAdd(R.force + nb + bin, static_cast<float>(fy));
            atomicAdd(R.force + 2 * nb + bin, static_cast<float>(fz));
        }
        if (cum >= T(1)) break;
    }
    if (cum > T(0)) lambda *= T(1) - (cum < T(0) ? T(0) : cum > T(1) ? T(1) : cum);
}

// Rotor forcing of one cell before its collision (needs the cell's indices).
template <bool F, class S, class T>
__device__ __forceinline__ void cellRotorForcing(const DevLevel& g, const int (&ijk)[3], int wm, const T (&f)[27],
                                                 T& gx, T& gy, T& gz, T& lambda) {
    T dRho, ux, uy, uz;
    macroFromF(f, dRho, ux, uy, uz);
    const T rho = dRho + T(1);
    const T rhoInv = T(1) / rho;
    const T uxPre = (ux * rho + gx) * rhoInv;
    const T uyPre = (uy * rho + gy) * rhoInv;
    const T uzPre = (uz * rho + gz) * rhoInv;
    bool track = wm != -2;
    if (wm >= 0 && (__ldg(g.wallData + wm) & 1u)) track = false;
    const float x = ijk[0] * g.res + g.ox, y = ijk[1] * g.res + g.oy, z = ijk[2] * g.res + g.oz;
    rotorForcing(g, x, y, z, rho, uxPre, uyPre, uzPre, track, gx, gy, gz, lambda);
}

template <bool F, class S>
__global__ void __launch_bounds__(kBlock) collideStream(DevLevel g) {
    advanceDither<F, S>(g);
    const int cell = blockIdx.x * kBlock + threadIdx.x;
    if (cell >= g.cellCount) return;
    const int wm = __ldg(g.wallMap + cell);
    if (wm == -3) return;  // the cell itself is a wall
    int nb[8], ijk[3];
    decodeNbr(g, cell, nb, g.rotorCount > 0 ? ijk : nullptr);
    using T = Real<S>;
    T f[27];
    readPre<F, S>(g, nb, f);
    T gx = g.gx, gy = g.gy, gz = g.gz, lambda = collConsts<T>(g).lambda;
    if (g.rotorCount > 0) cellRotorForcing<F, S>(g, ijk, wm, f, gx, gy, gz, lambda);
    collideCumulantT(f, collConsts<T>(g), lambda, gx, gy, gz);
    writePost<F, S>(g, nb, f, stepDither<F, S>(g, kSaltCollide));
}

// Rotor volume fraction at (x, y, z) of one rotor (getRotorFraction,
// include/rotorFunctions.h:155-209).
__device__ __forceinline__ float rotorFractionAt(const DevRotor& R, float x, float y, float z) {
    const float dx = x - R.ox, dy = y - R.oy, dz = z - R.oz;
    float xr = x, yr = y, zr = z;
    if (R.axis == 0) {
        yr = R.oy + R.c * dy + R.s * dz;
        zr = R.oz - R.s * dy + R.c * dz;
    } else if (R.axis == 1) {
        xr = R.ox + R.c * dx - R.s * dz;
        zr = R.oz + R.s * dx + R.c * dz;
    } else {
        xr = R.ox + R.c * dx + R.s * dy;
        yr = R.oy - R.s * dx + R.c * dy;
    }
    if (xr < R.xMin || xr >= R.xMax || yr < R.yMin || yr >= R.yMax || zr < R.zMin || zr >= R.zMax) return 0.f;
    const float xRel = xr - R.xMin, yRel = yr - R.yMin, zRel = zr - R.zMin;
    const int ii = static_cast<int>(xRel / R.res), jj = static_cast<int>(yRel / R.res), kk = static_cast<int>(zRel / R.res);
    if (ii >= R.cntX || jj >= R.cntY || kk >= R.cntZ) return 0.f;
    const int bx = R.cntX / 4, by = R.cntY / 4;
    const int map = __ldg(R.rotorMap + (kk / 4) * bx * by + (jj / 4) * bx + ii / 4);
    if (map < 0) return 0.f;
    const unsigned packedCounts = __ldg(R.interp + map * 64 + (kk % 4) * 16 + (jj % 4) * 4 + (ii % 4));
    const float xw = xRel / R.res - ii, yw = yRel / R.res - jj, zw = zRel / R.res - kk;
    float v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = static_cast<float>((packedCounts >> (4u * q)) & 0xFu);
    const float v00 = v[0] + xw * (v[1] - v[0]);
    const float v10 = v[2] + xw * (v[3] - v[2]);
    const float v01 = v[4] + xw * (v[5] - v[4]);
    const float v11 = v[6] + xw * (v[7] - v[6]);
    const float v0 = v00 + yw * (v10 - v00);
    const float v1 = v01 + yw * (v11 - v01);
    return (v0 + zw * (v1 - v0)) * 0.125f;
}

// Solid fraction of all rotors at (x, y, z), clamped to [0, 1].
__device__ __forceinline__ float rotorMarkerAt(const DevLevel& g, float x, float y, float z) {
    float m = 0.f;
    for (int r = 0; r < g.rotorCount; ++r) m += rotorFractionAt(g.rotor[r], x, y, z);
    return fminf(fmaxf(m, 0.f), 1.f);
}

// One level's cells written into the section image img[3][pixelsV][pixelsH]
// (dRho, normal velocity, solid marker); finer levels run later and
// overwrite (include/flowReportFunctions.h:133-262).
template <bool F, class S>
__global__ void __launch_bounds__(kBlock) flowImageLevel(DevLevel g, FlowImagePass a, float* img) {
    const int cell = blockIdx.x * kBlock + threadIdx.x;
    if (cell >= g.cellCount) return;
    int nb[8], ijk[3];
    decodeNbr(g, cell, nb, ijk);
    const int normal = a.plane == LBM_PLANE_XY ? ijk[2] : a.plane == LBM_PLANE_ZY ? ijk[0] : ijk[1];
    if (normal != a.lowerNormal) return;
    const int ch = a.plane == LBM_PLANE_XY ? ijk[0] : ijk[2];
    const int cv = a.plane == LBM_PLANE_ZX ? ijk[0] : ijk[1];
    if (ch % a.downsample != 0 || cv % a.downsample != 0) return;
    const int ih = (ch / a.downsample) * a.upsample, iv = (cv / a.downsample) * a.upsample;
    if (ih + a.upsample <= a.startH || ih >= a.startH + a.pixelsH) return;
    if (iv + a.upsample <= a.startV || iv >= a.startV + a.pixelsV) return;
    // the next layer along the normal: an actual adjacent centre, or no sample
    int upper = cell, nu[8], uijk[3];
    if (a.interpolate) {
        upper = a.plane == LBM_PLANE_XY ? nb[4] : a.plane == LBM_PLANE_ZY ? nb[1] : nb[2];
        if (upper < 0 || upper >= g.cellCount) return;
        decodeNbr(g, upper, nu, uijk);
        if (uijk[0] != ijk[0] + (a.plane == LBM_PLANE_ZY) || uijk[1] != ijk[1] + (a.plane == LBM_PLANE_ZX) ||
            uijk[2] != ijk[2] + (a.plane == LBM_PLANE_XY))
            return;
    } else {
#pragma unroll
        for (int q = 0; q < 8; ++q) nu[q] = nb[q];
    }
    const bool lowerSolid = __ldg(g.wallMap + cell) == -3, upperSolid = __ldg(g.wallMap + upper) == -3;
    const bool solid = a.alpha <= 0.5f ? lowerSolid : upperSolid;
    float marker = solid ? 1.f : 0.f;
    float dRho = 0.f, ux = 0.f, uy = 0.f, uz = 0.f;
    if (!solid) {
        const bool blend = a.interpolate && !lowerSolid && !upperSolid;
        float f[27];
        if (lowerSolid) readPre<F, S>(g, nu, f);
        else readPre<F, S>(g, nb, f);
        macroFromF(f, dRho, ux, uy, uz);
        marker = rotorMarkerAt(g, ijk[0] * g.res + g.ox, ijk[1] * g.res + g.oy, ijk[2] * g.res + g.oz);
        if (blend) {
            readPre<F, S>(g, nu, f);
            float dU, xU, yU, zU;
            macroFromF(f, dU, xU, yU, zU);
            dRho += a.alpha * (dU - dRho);
            ux += a.alpha * (xU - ux);
            uy += a.alpha * (yU - uy);
            uz += a.alpha * (zU - uz);
            const int pi = ijk[0] + (a.plane == LBM_PLANE_ZY), pj = ijk[1] + (a.plane == LBM_PLANE_ZX),
                      pk = ijk[2] + (a.plane == LBM_PLANE_XY);
            const float mU = rotorMarkerAt(g, pi * g.res + g.ox, pj * g.res + g.oy, pk * g.res + g.oz);
            marker += a.alpha * (mU - marker);
        }
    }
    const float un = a.plane == LBM_PLANE_XY ? uz : a.plane == LBM_PLANE_ZY ? ux : uy;
    const long long plane = (long long)a.pixelsH * a.pixelsV;
    for (int sv = 0; sv < a.upsample; ++sv) {
        const int y = iv + sv - a.startV;
        if (y < 0 || y >= a.pixelsV) continue;
        for (int sh = 0; sh < a.upsample; ++sh) {
            const int x = ih + sh - a.startH;
            if (x < 0 || x >= a.pixelsH) continue;
            const long long p = (long long)y * a.pixelsH + x;
            img[p] = dRho;
            img[plane + p] = un;
            img[2 * plane + p] = marker;
        }
    }
}

// Section-plane flow sums (getFlowReportGeneral, include/flowReportFunctions.h:11-352)
// on one level: cells of layer `layer` along the plane normal inside the
// in-plane index ranges [h0, h1) x [v0, v1); walls and pixels that are at
// least half rotor are skipped.  Per pixel, in FP32 as the reference forms
// them: {u, dRho u, (1 + dRho) u |u|, dRho, (1 + dRho) u^3 / 2, 1}, summed in
// FP64 into out[6].
template <bool F, class S>
__global__ void __launch_bounds__(kBlock) flowReportSum(DevLevel g, int plane, int layer, int h0, int h1, int v0,
                                                        int v1, double* out) {
    const int cell = blockIdx.x * kBlock + threadIdx.x;
    double v[6] = {0, 0, 0, 0, 0, 0};
    if (cell < g.cellCount) {
        int nb[8], ijk[3];
        decodeNbr(g, cell, nb, ijk);
        const int normal = plane == LBM_PLANE_XY ? ijk[2] : plane == LBM_PLANE_ZY ? ijk[0] : ijk[1];
        const int horiz = plane == LBM_PLANE_XY ? ijk[0] : ijk[2];
        const int vert = plane == LBM_PLANE_ZX ? ijk[0] : ijk[1];
        if (normal == layer && horiz >= h0 && horiz < h1 && vert >= v0 && vert < v1 && __ldg(g.wallMap + cell) != -3) {
            float f[27];
            readPre<F, S>(g, nb, f);
            float dRho, ux, uy, uz;
            macroFromF(f, dRho, ux, uy, uz);
            float marker = 0.f;
            const float x = ijk[0] * g.res + g.ox, y = ijk[1] * g.res + g.oy, z = ijk[2] * g.res + g.oz;
            for (int r = 0; r < g.rotorCount; ++r) marker += rotorFractionAt(g.rotor[r], x, y, z);
            marker = fminf(fmaxf(marker, 0.f), 1.f);
            if (marker < 0.5f) {
                const float u = plane == LBM_PLANE_XY ? uz : plane == LBM_PLANE_ZY ? ux : uy;
                const float rhoU = fmaf(dRho, u, u);
                v[0] = u;
                v[1] = dRho * u;
                v[2] = rhoU * fabsf(u);
                v[3] = dRho;
                v[4] = 0.5f * rhoU * u * u;
                v[5] = 1.0;
            }
        }
    }
    __shared__ double part[6][kBlock / 32];
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        double a = v[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
        if ((threadIdx.x & 31) == 0) part[q][threadIdx.x >> 5] = a;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        double a = 0.0;
        for (int k = 0; k < kBlock / 32; ++k) a += part[threadIdx.x][k];
        atomicAdd(out + threadIdx.x, a);
    }
}

// ---- bulk collide-stream ---------------------------------------------------
// Persistent CTAs walk the bulk segments: runs of up to kSegmentCells plain
// fluid cells inside one compressed row, one segment per CTA iteration, one
// cell per thread.  Inside a segment the 8 esotwist neighbours of lane t are
// the segment's base indices + t, so a CTA reads one 20-byte descriptor per
// tile and no per-cell metadata.  For every direction q the tile's 27
// pre-collision values form one contiguous run of a population plane.
//
// collidePrefetch (default): the next tile's 27 gathers are issued into
// registers before the current tile is collided.
// collideBulkTma (LBM3_COLLIDE_KERNEL=tma): one elected thread copies those 27 runs with
// cp.async.bulk (the TMA engine, global -> shared, completion counted on an
// mbarrier) into a ring of kStages tiles, kStages-1 tiles ahead of the tile
// being collided.  The copies bypass L1 and hold no registers, so many tiles
// stay in flight per SM while the cumulant arithmetic runs.  Runs are copied
// from the 16-byte boundary below their first element; the lane offset of a
// run inside its stage slot is that misalignment.
// On B200 the small (about 0.5 KB) bulk copies of 128-cell tiles make the TMA
// variant slower than register prefetch, which is therefore the default.
constexpr int kTile = 128;  // == kSegmentCells
static_assert(kTile == kSegmentCells, "tile and segment length differ");

#ifndef LBM3_TMA_STAGES
#define LBM3_TMA_STAGES 4
#endif
#ifndef LBM3_TMA_MIN_BLOCKS
#define LBM3_TMA_MIN_BLOCKS 3
#endif
#ifndef LBM3_PREFETCH_MIN_BLOCKS
#define LBM3_PREFETCH_MIN_BLOCKS 4
#endif
constexpr int kStages = LBM3_TMA_STAGES;
// bytes of one run slot: kTile elements plus the 16-byte alignment slack
template <class S> constexpr int runBytes() { return kTile * int(sizeof(S)) + 16; }
template <class S> constexpr int stageBytes() { return 27 * runBytes<S>(); }
template <class S> constexpr int tmaSmemBytes() { return kStages * stageBytes<S>() + kStages * 8; }
// bound on mbarrier polls before a wait is declared lost (~0.1 s)
constexpr int kWaitPolls = 1 << 22;

__device__ __forceinline__ void segNbr(const DevLevel& g, const int4& d, int t, int (&nb)[8]) {
    // segments never contain a lane whose +1 neighbour wraps (the builder
    // sends those cells to the special list), so +1 is plain addition
    nb[0] = d.x + t;
    nb[1] = d.x + t + 1;
    nb[2] = d.y + t;
    nb[3] = d.y + t + 1;
    nb[4] = d.z + t;
    nb[5] = d.z + t + 1;
    nb[6] = d.w + t;
    nb[7] = d.w + t + 1;
}

__device__ __forceinline__ void loadDesc(const DevLevel& g, int tile, int4& d, int& l) {
    if (tile < g.segCount) {
        d = __ldg(g.seg + tile);
        l = __ldg(g.segLen + tile);
    } else {
        d = make_int4(0, 0, 0, 0);
        l = 0;
    }
}

__device__ __forceinline__ unsigned smemAddr(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbarInit(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smemAddr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbarArriveExpectTx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;\n" ::"r"(smemAddr(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbarTestWait(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smemAddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase with the given parity to complete.
__device__ __forceinline__ bool mbarWait(uint64_t* bar, unsigned parity) {
    for (int i = 0; i < kWaitPolls; ++i) {
        if (mbarTestWait(bar, parity)) return true;
        if (i > 64) __nanosleep(20);
    }
    return false;
}

__device__ __forceinline__ void bulkLoad(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
            smemAddr(dst)),
        "l"(src), "r"(bytes), "r"(smemAddr(bar))
        : "memory");
}

// Plane base index of direction q's run for a tile starting at descriptor d.
template <bool F>
__device__ __forceinline__ long long runStart(const DevLevel& g, const int4& d, int q) {
    const int k = preNbr(q);
    const int b = (k >> 1) == 0 ? d.x : (k >> 1) == 1 ? d.y : (k >> 1) == 2 ? d.z : d.w;
    return (long long)preSlot<F>(q) * g.stride + b + (k & 1);
}

// Elected thread: start the 27 run copies of a tile into `stage`.
template <bool F, class S>
__device__ __forceinline__ void produceTile(const DevLevel& g, const int4& d, int len, unsigned char* stage,
                                            uint64_t* bar) {
    const char* base = static_cast<const char*>(g.f);
    unsigned total = 0;
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        const uintptr_t a = reinterpret_cast<uintptr_t>(base + runStart<F>(g, d, q) * (long long)sizeof(S));
        const uintptr_t a0 = a & ~uintptr_t(15);
        const uintptr_t a1 = (a + uintptr_t(len) * sizeof(S) + 15) & ~uintptr_t(15);
        total += static_cast<unsigned>(a1 - a0);
    }
    mbarArriveExpectTx(bar, total);
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        const uintptr_t a = reinterpret_cast<uintptr_t>(base + runStart<F>(g, d, q) * (long long)sizeof(S));
        const uintptr_t a0 = a & ~uintptr_t(15);
        const uintptr_t a1 = (a + uintptr_t(len) * sizeof(S) + 15) & ~uintptr_t(15);
        bulkLoad(stage + q * runBytes<S>(), reinterpret_cast<const void*>(a0), static_cast<unsigned>(a1 - a0),
                 bar);
    }
}

template <bool F, class S>
__global__ void __launch_bounds__(kTile, LBM3_TMA_MIN_BLOCKS) collideBulkTma(DevLevel g) {
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kStages * stageBytes<S>());
    const int T = g.segCount;
    const int G = gridDim.x;
    const int t = threadIdx.x;
    advanceDither<F, S>(g);
    const Dither D = stepDither<F, S>(g, kSaltCollide);
    if (t == 0) {
#pragma unroll
        for (int k = 0; k < kStages; ++k) mbarInit(&bar[k], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();

    int4 d[kStages];
    int l[kStages];
    unsigned parity = 0;   // bit k: parity of the next phase of stage k
    unsigned pending = 0;  // bit k: copies issued into stage k not yet consumed
#pragma unroll
    for (int k = 0; k < kStages - 1; ++k) {
        loadDesc(g, blockIdx.x + k * G, d[k], l[k]);
        if (t == 0 && l[k] > 0) produceTile<F, S>(g, d[k], l[k], smem + k * stageBytes<S>(), &bar[k]);
        if (l[k] > 0) pending |= 1u << k;
    }
    int4 dNext;
    int lNext;
    loadDesc(g, blockIdx.x + (kStages - 1) * G, dNext, lNext);
    bool lost = false;
    for (int base = blockIdx.x; base < T; base += kStages * G) {
        bool stop = false;
#pragma unroll
        for (int k = 0; k < kStages; ++k) {
            const int tile = base + k * G;
            // every thread is done with the stage consumed last iteration, and
            // a lost wait anywhere in the CTA stops all of it
            if (__syncthreads_or(lost) || tile >= T) {
                stop = true;
                break;
            }
            const int ks = (k + kStages - 1) % kStages;
            d[ks] = dNext;
            l[ks] = lNext;
            if (l[ks] > 0) {
                if (t == 0) produceTile<F, S>(g, d[ks], l[ks], smem + ks * stageBytes<S>(), &bar[ks]);
                pending |= 1u << ks;
            }
            loadDesc(g, tile + kStages * G, dNext, lNext);
            if (l[k] > 0) {
                if (!mbarWait(&bar[k], (parity >> k) & 1u)) {
                    lost = true;
                    continue;
                }
                parity ^= 1u << k;
                pending &= ~(1u << k);
            }
            if (t < l[k]) {
                int nb[8];
                segNbr(g, d[k], t, nb);
                const unsigned char* st = smem + k * stageBytes<S>();
                Real<S> f[27];
#pragma unroll
                for (int q = 0; q < 27; ++q) {
                    const int off = static_cast<int>((runStart<F>(g, d[k], q) * (long long)sizeof(S)) & 15) /
                                    int(sizeof(S));
                    f[q] = Store<S>::ld(reinterpret_cast<const S*>(st + q * runBytes<S>()) + off + t);
                }
                collideCumulantT(f, collConsts<Real<S>>(g), collConsts<Real<S>>(g).lambda, Real<S>(g.gx),
                                 Real<S>(g.gy), Real<S>(g.gz));
                writePost<F, S>(g, nb, f, D);
            }
        }
        if (stop) break;
    }
    if (lost) {
        if (t == 0) {
            atomicExch(g.errorFlag, 1);
            // let copies still in flight land before the CTA's shared memory goes away
#pragma unroll
            for (int k = 0; k < kStages; ++k)
                if ((pending >> k) & 1u) mbarWait(&bar[k], (parity >> k) & 1u);
        }
        __syncthreads();
    }
}

// Cells outside the bulk segments, one thread per listed cell: wall-adjacent
// fluid cells get the interpolated bounceback of Zhao & Yong (2017) with a
// moving-wall term and momentum-exchange force
// (applyIBB, include/boundaryConditions/interpolatedBouncebackFunctions.h:43-157,
// and the write loop of include/updateGrid.h:143-176); the rest (cells whose
// +1 neighbour wraps) collide and stream like bulk cells.
template <bool F, class S, bool kRotors = false>
__device__ __forceinline__ void collideSpecialCell(const DevLevel& g, int cell) {
    const int wm = __ldg(g.wallMap + cell);
    int nb[8], ijk[3];
    decodeNbr(g, cell, nb, kRotors ? ijk : nullptr);
    using T = Real<S>;
    T f[27];
    readPre<F, S>(g, nb, f);
    T gx = g.gx, gy = g.gy, gz = g.gz, lambda = collConsts<T>(g).lambda;
    if (kRotors) cellRotorForcing<F, S>(g, ijk, wm, f, gx, gy, gz, lambda);
    collideCumulantT(f, collConsts<T>(g), lambda, gx, gy, gz);
    const Dither D = stepDither<F, S>(g, kSaltCollide);
    if (wm < 0) {
        writePost<F, S>(g, nb, f, D);
        return;
    }
    const unsigned wallData = __ldg(g.wallData + wm);
    const int nw = g.wallCount;
    const T uwx = __ldg(g.wallVel + wm), uwy = __ldg(g.wallVel + nw + wm), uwz = __ldg(g.wallVel + 2 * nw + wm);
    T dRho, ux, uy, uz;
    macroFromF(f, dRho, ux, uy, uz);
    T out[27];
#pragma unroll
    for (int d = 0; d < 27; ++d) out[d] = f[d];
    T fx = T(0), fy = T(0), fz = T(0);
    int link = 0;
    unsigned code = 0u;
    const S* base = static_cast<const S*>(g.f);
#pragma unroll
    for (int d = 1; d < 27; ++d) {
        if (!((wallData >> d) & 1u)) continue;
        const int id = inv(d);
        const T eu = T(cx(id)) * uwx + T(cy(id)) * uwy + T(cz(id)) * uwz;
        const T wallTerm = T(6) * weightT<T>(id) * (T(1) + dRho) * eu;
        T gamma = T(0.5);
        if (g.useIBB) {
            if ((link & 3) == 0) code = __ldg(g.linkLength + (link >> 2) * nw + wm);
            const unsigned c8 = (code >> (8 * (link & 3))) & 255u;
            const T q = static_cast<T>(c8) / T(254);
            gamma = q < T(0.01f) ? T(0.01f) : q > T(1) ? T(1) : q;
            ++link;
        }
        // pre-collision value of direction d, still unchanged in memory
        const T fPre = Store<S>::ld(base + (long long)preSlot<F>(d) * g.stride + nb[preNbr(d)]);
        const T invDen = T(1) / (T(1) + gamma);
        const T r = ((T(1) - gamma) * invDen) * fPre + (gamma * invDen) * f[id] + (gamma * invDen) * f[d] +
                    invDen * wallTerm;
        fx += -f[d] * (T(cx(d)) - uwx) + r * (T(cx(id)) - uwx);
        fy += -f[d] * (T(cy(d)) - uwy) + r * (T(cy(id)) - uwy);
        fz += -f[d] * (T(cz(d)) - uwz) + r * (T(cz(id)) - uwz);
        out[d] = r;
    }
    // writes: a linked direction goes to the next pre-collision slot of its
    // inverse (inside the wall cell), the others stream as usual
    S* wbase = static_cast<S*>(g.f);
    const unsigned cb = D.cell(cell);
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        const bool linked = d != 0 && ((wallData >> d) & 1u);
        const int slot = linked ? (F ? inv(d) : d) : postSlot<F>(d);
        stD(wbase + (long long)slot * g.stride + nb[postNbr(d)], out[d], D, cb, d);
    }
    if (g.trackWallForce && !(wallData & 1u)) {
        g.wallForce[wm] += double(fx);
        g.wallForce[nw + wm] += double(fy);
        g.wallForce[2 * nw + wm] += double(fz);
    }
}

template <bool F, class S>
__global__ void __launch_bounds__(kBlock) collideList(DevLevel g) {
    advanceDither<F, S>(g);
    const int idx = blockIdx.x * kBlock + threadIdx.x;
    if (idx >= g.specialCount) return;
    collideSpecialCell<F, S>(g, __ldg(g.special + idx));
}

// Cells a rotor can reach while it turns, one thread each: special-cell
// update with the rotor forcing before the collision.
template <bool F, class S>
__global__ void __launch_bounds__(kBlock) collideRotorList(DevLevel g) {
    advanceDither<F, S>(g);
    const int idx = blockIdx.x * kBlock + threadIdx.x;
    if (idx >= g.rotorCellCount) return;
    collideSpecialCell<F, S, true>(g, __ldg(g.rotorCells + idx));
}

// Work items of one launch: special chunks [0, S) first (kTile listed cells
// each), then the bulk segments [S, S + segCount).  CTAs take items from an
// atomic counter, so the long-latency wall-adjacent cells land on whichever
// CTAs are free first and the bulk tail stays balanced; the last CTA to
// finish resets the counter for the next launch.  Thread 0 fetches; the
// value reaches the CTA through a two-slot shared buffer and one barrier.
template <bool F, class S>
__global__ void __launch_bounds__(kTile, LBM3_PREFETCH_MIN_BLOCKS) collidePrefetch(DevLevel g) {
    __shared__ int slot[2];
    const int nSpecial = (g.specialCount + kTile - 1) / kTile;
    const int t = threadIdx.x;
    int parity = 0;
    advanceDither<F, S>(g);
    const Dither D = stepDither<F, S>(g, kSaltCollide);
    auto fetch = [&]() {
        if (t == 0) slot[parity] = atomicAdd(g.work, 1);
        __syncthreads();
        const int v = slot[parity];
        parity ^= 1;
        return v;
    };
    int item = fetch();
    while (item < nSpecial) {
        const int q = item * kTile + t;
        if (q < g.specialCount) collideSpecialCell<F, S>(g, __ldg(g.special + q));
        item = fetch();
    }
    int4 dCur, dNext;
    int lCur, lNext;
    loadDesc(g, item - nSpecial, dCur, lCur);
    loadDesc(g, fetch() - nSpecial, dNext, lNext);
    int nb[8];
    segNbr(g, dCur, t, nb);
    using T = Real<S>;
    const CollisionConstsT<T>& P = collConsts<T>(g);
    T fn[27];
    if (t < lCur) readPre<F, S>(g, nb, fn);
    while (lCur > 0) {  // CTA-uniform: lengths come from the shared descriptors
        int4 dAfter;
        int lAfter;
        loadDesc(g, fetch() - nSpecial, dAfter, lAfter);
        T f[27];
#pragma unroll
        for (int q = 0; q < 27; ++q) f[q] = fn[q];
        int nbn[8];
        segNbr(g, dNext, t, nbn);
        if (t < lNext) readPre<F, S>(g, nbn, fn);
        if (t < lCur) {
            collideCumulantT(f, P, P.lambda, T(g.gx), T(g.gy), T(g.gz));
            writePost<F, S>(g, nb, f, D);
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) nb[q] = nbn[q];
        lCur = lNext;
        dNext = dAfter;
        lNext = lAfter;
    }
    if (t == 0) {
        __threadfence();
        if (atomicAdd(g.work + 1, 1) == int(gridDim.x) - 1) {
            g.work[0] = 0;
            g.work[1] = 0;
            __threadfence();
        }
    }
}

// ---- paired bulk collide-stream ---------------------------------------------
// collidePair (default): CTAs of kHalf threads; thread t collides cells t and
// t + kHalf of a 128-cell segment as one Pair, so every add/mul/fma of the
// cumulant transform is one packed FP32x2 instruction for both cells (the
// kernel is bounded by instruction issue, not by the FMA pipe), and the
// second cell's 27 loads and 27 stores reuse the first cell's address with
// an immediate offset.  Population offsets are 32-bit element indices
// (27 x stride < 2^31; larger grids take collidePrefetch).  The CTA fetches
// its next work item while the current tile's loads are in flight; with
// LBM3_PAIR_PREFETCH the next tile's populations are also loaded into
// registers during the current tile's collision.
constexpr int kHalf = kTile / 2;

#ifndef LBM3_PAIR_MIN_BLOCKS
#define LBM3_PAIR_MIN_BLOCKS 8
#endif
#ifndef LBM3_PAIR_PREFETCH
#define LBM3_PAIR_PREFETCH 0
#endif

// Element offset of direction q's pre- (Pre) or post-collision run for the
// tile with descriptor d: slot x stride + the neighbour row start.  The
// callers read the stride once: a descriptor held in shared memory would
// otherwise be read again after every store through a generic pointer.
template <bool F, bool Pre>
__device__ __forceinline__ int runOffset32(int stride, const int4& d, int q) {
    const int k = Pre ? preNbr(q) : postNbr(q);
    const int b = (k >> 1) == 0 ? d.x : (k >> 1) == 1 ? d.y : (k >> 1) == 2 ? d.z : d.w;
    const int slot = Pre ? preSlot<F>(q) : postSlot<F>(q);
    return slot * stride + b + (k & 1);
}

// Load the 27 pre-collision values of lanes t and t + kHalf.  A partial tile
// clamps lane A to the last cell (its store is masked) and skips lane B.
template <bool F, class S, bool kFull>
__device__ __forceinline__ void loadPair(const DevLevel& g, const int4& d, int t, int len, Pair (&f)[27]) {
    const S* base = static_cast<const S*>(g.f);
    const int stride = static_cast<int>(g.stride);
    const int tA = kFull ? t : min(t, len - 1);
    const bool okB = kFull || t + kHalf < len;
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        const S* p = base + (runOffset32<F, true>(stride, d, q) + tA);
        const float a = Store<S>::ld(p);
        const float b = okB ? Store<S>::ld(p + kHalf) : 0.f;
        f[q] = mkPair(a, b);
    }
}

// For 16-bit storage one stochastic conversion rounds both lanes' values (cells
// d.x + t and d.x + t + kHalf) from one 32-bit draw.
template <bool F, class S>
__device__ __forceinline__ void storePair(const DevLevel& g, const int4& d, int t, int len, const Pair (&f)[27],
                                          const Dither& D) {
    S* base = static_cast<S*>(g.f);
    const int stride = static_cast<int>(g.stride);
    const bool okA = t < len, okB = t + kHalf < len;
    if constexpr (sizeof(S) == 2) {
        // one full hash per lane, then a 32-bit linear congruential step per
        // direction (Numerical Recipes' constants) with its high half folded
        // into the low half: three instructions per draw instead of a full
        // finaliser in the hottest store loop
        unsigned x = mix32(D.cell(d.x + t));
#pragma unroll
        for (int q = 0; q < 27; ++q) {
            S* p = base + (runOffset32<F, false>(stride, d, q) + t);
            x = x * 1664525u + 1013904223u;
            Store<S>::st2R(p, p + kHalf, f[q].v.x, f[q].v.y, x ^ (x >> 16), okA, okB);
        }
    } else {
#pragma unroll
        for (int q = 0; q < 27; ++q) {
            S* p = base + (runOffset32<F, false>(stride, d, q) + t);
            if (okA) Store<S>::st(p, f[q].v.x);
            if (okB) Store<S>::st(p + kHalf, f[q].v.y);
        }
    }
}

template <bool F, class S>
__device__ __forceinline__ void loadTilePair(const DevLevel& g, const int4& d, int t, int len, Pair (&f)[27]) {
    if (len == kTile) loadPair<F, S, true>(g, d, t, len, f);
    else if (len > 0) loadPair<F, S, false>(g, d, t, len, f);
}

template <bool F, class S>
__global__ void __launch_bounds__(kHalf, LBM3_PAIR_MIN_BLOCKS) collidePair(DevLevel g) {
    __shared__ int slot[2];
    const int nSpecial = (g.specialCount + kTile - 1) / kTile;
    const int t = threadIdx.x;
    int parity = 0;
    advanceDither<F, S>(g);
    const Dither D = stepDither<F, S>(g, kSaltCollide);
    auto fetch = [&]() {
        if (t == 0) slot[parity] = atomicAdd(g.work, 1);
        __syncthreads();
        const int v = slot[parity];
        parity ^= 1;
        return v;
    };
    int item = fetch();
    while (item < nSpecial) {
        const int q = item * kTile + t;
        if (q < g.specialCount) collideSpecialCell<F, S>(g, __ldg(g.special + q));
        if (q + kHalf < g.specialCount) collideSpecialCell<F, S>(g, __ldg(g.special + q + kHalf));
        item = fetch();
    }
    int4 dCur;
    int lCur;
    loadDesc(g, item - nSpecial, dCur, lCur);
    int next = fetch();
#if LBM3_PAIR_PREFETCH
    Pair fn[27];
    loadTilePair<F, S>(g, dCur, t, lCur, fn);
#endif
    while (lCur > 0) {  // CTA-uniform: lengths come from the shared descriptors
        Pair f[27];
#if LBM3_PAIR_PREFETCH
#pragma unroll
        for (int q = 0; q < 27; ++q) f[q] = fn[q];
#else
        loadTilePair<F, S>(g, dCur, t, lCur, f);
#endif
        int4 dNext;
        int lNext;
        loadDesc(g, next - nSpecial, dNext, lNext);
        next = fetch();  // the atomic's latency overlaps the loads in flight
#if LBM3_PAIR_PREFETCH
        loadTilePair<F, S>(g, dNext, t, lNext, fn);
#endif
        collideCumulantT(f, g.coll, g.coll.lambda, g.gx, g.gy, g.gz);
        storePair<F, S>(g, dCur, t, lCur, f, D);
        dCur = dNext;
        lCur = lNext;
    }
    if (t == 0) {
        __threadfence();
        if (atomicAdd(g.work + 1, 1) == int(gridDim.x) - 1) {
            g.work[0] = 0;
            g.work[1] = 0;
            __threadfence();
        }
    }
}

#if LBM3_SHARED_UNIT
// Section image cleared to solid (marker 1, values 0).
__global__ void __launch_bounds__(kBlock) flowImageClear(float* img, long long pixels) {
    const long long p = blockIdx.x * (long long)kBlock + threadIdx.x;
    if (p >= pixels) return;
    img[p] = 0.f;
    img[pixels + p] = 0.f;
    img[2 * pixels + p] = 1.f;
}

// Flow sums over the fluid pixels of a section image
// (include/flowReportFunctions.h:263-318): {u, dRho u, (1+dRho) u |u|, dRho,
// (1+dRho) u^3 / 2, pixels}, each pixel's terms in FP32, summed in FP64.
__global__ void __launch_bounds__(kBlock) flowImageSum(const float* img, long long pixels, double* out) {
    const long long p = blockIdx.x * (long long)kBlock + threadIdx.x;
    double v[6] = {0, 0, 0, 0, 0, 0};
    if (p < pixels && img[2 * pixels + p] < 0.5f) {
        const float dRho = img[p], u = img[pixels + p];
        const float rhoU = fmaf(dRho, u, u);
        v[0] = u;
        v[1] = dRho * u;
        v[2] = rhoU * fabsf(u);
        v[3] = dRho;
        v[4] = 0.5f * rhoU * u * u;
        v[5] = 1.0;
    }
    __shared__ double part[6][kBlock / 32];
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        double x = v[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == 0) part[q][threadIdx.x >> 5] = x;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        double x = 0.0;
        for (int k = 0; k < kBlock / 32; ++k) x += part[threadIdx.x][k];
        atomicAdd(out + threadIdx.x, x);
    }
}

// FP64 force and torque about the origin of the cells of one wall ID
// (updateTracker wall branch, include/trackerFunctions.h:386-428).
__global__ void __launch_bounds__(kBlock) wallForceSum(DevLevel g, int wallID, double* out) {
    const int w = blockIdx.x * kBlock + threadIdx.x;
    double v[6] = {0, 0, 0, 0, 0, 0};
    if (w < g.wallCount) {
        const unsigned data = __ldg(g.wallData + w);
        if (static_cast<int>((data >> 27) & 31u) == wallID) {
            const int cell = __ldg(g.wallIndex + w);
            int nb[8], ijk[3];
            decodeNbr(g, cell, nb, ijk);
            const double x = double(ijk[0] * g.res + g.ox), y = double(ijk[1] * g.res + g.oy),
                         z = double(ijk[2] * g.res + g.oz);
            const double gx = g.wallForce[w], gy = g.wallForce[g.wallCount + w], gz = g.wallForce[2 * g.wallCount + w];
            v[0] = gx; v[1] = gy; v[2] = gz;
            v[3] = y * gz - z * gy;
            v[4] = z * gx - x * gz;
            v[5] = x * gy - y * gx;
        }
    }
    __shared__ double part[6][kBlock / 32];
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        double a = v[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
        if ((threadIdx.x & 31) == 0) part[q][threadIdx.x >> 5] = a;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        double a = 0.0;
        for (int k = 0; k < kBlock / 32; ++k) a += part[threadIdx.x][k];
        atomicAdd(out + threadIdx.x, a);
    }
}

// FP64 force and torque of one rotor from its force bins, about the rotor
// origin in the rotor frame (updateTracker rotor branch,
// include/trackerFunctions.h:240-290); one thread per nonzero block.
__global__ void __launch_bounds__(kBlock) rotorForceSum(DevRotor R, const int* index, double* out) {
    const int n = blockIdx.x * kBlock + threadIdx.x;
    double v[6] = {0, 0, 0, 0, 0, 0};
    if (n < R.nonzero) {
        const int b = __ldg(index + n);
        const int bx = R.cntX / 4, by = R.cntY / 4;
        const int kb = b / (bx * by), rem = b % (bx * by), jb = rem / bx, ib = rem % bx;
        const float resBlock = R.res * 4.f;
        const float resForce = resBlock / 3.f;
        const float x0 = ib * resBlock + R.xMin - R.ox + 0.5f * resForce;
        const float y0 = jb * resBlock + R.yMin - R.oy + 0.5f * resForce;
        const float z0 = kb * resBlock + R.zMin - R.oz + 0.5f * resForce;
        const int nb = 27 * R.nonzero;
        for (int q = 0; q < 27; ++q) {
            const int kF = q / 9, jF = (q / 3) % 3, iF = q % 3;
            const double x = x0 + iF * resForce, y = y0 + jF * resForce, z = z0 + kF * resForce;
            const double fx = R.force[n * 27 + q], fy = R.force[nb + n * 27 + q], fz = R.force[2 * nb + n * 27 + q];
            v[0] += fx; v[1] += fy; v[2] += fz;
            v[3] += y * fz - z * fy;
            v[4] += z * fx - x * fz;
            v[5] += x * fy - y * fx;
        }
    }
    __shared__ double part[6][kBlock / 32];
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        double a = v[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
        if ((threadIdx.x & 31) == 0) part[q][threadIdx.x >> 5] = a;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        double a = 0.0;
        for (int k = 0; k < kBlock / 32; ++k) a += part[threadIdx.x][k];
        atomicAdd(out + threadIdx.x, a);
    }
}

// Flow sums of one open boundary from the cumulative arrays
// (include/trackerFunctions.h:143-172): per cell, in FP32 as the reference
// forms them, {uN, rho uN, rho uN |uN|, dRho, dRho uN, rho uN^3 / 2}; summed
// in FP64 into out[6].
__global__ void __launch_bounds__(kBlock) openFlowSum(DevLevel g, int openBCID, float invSpan, double* out) {
    __shared__ double part[6][kBlock / 32];
    const int idx = blockIdx.x * kBlock + threadIdx.x;
    double v[6] = {0, 0, 0, 0, 0, 0};
    if (idx < g.obCount && (__ldg(g.obInfo + idx) >> 16) == openBCID) {
        const float dRho = g.obRhoCum[idx] * invSpan;
        const float uN = g.obUnCum[idx] * invSpan;
        const float rho = 1.0f + dRho;
        v[0] = uN;
        v[1] = rho * uN;
        v[2] = rho * uN * fabsf(uN);
        v[3] = dRho;
        v[4] = dRho * uN;
        v[5] = 0.5f * rho * uN * uN * uN;
    }
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        double a = v[q];
        for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
        if ((threadIdx.x & 31) == 0) part[q][threadIdx.x >> 5] = a;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        double a = 0.0;
        for (int w = 0; w < kBlock / 32; ++w) a += part[threadIdx.x][w];
        atomicAdd(out + threadIdx.x, a);
    }
}
#endif

// F is the flipper after streaming, i.e. the state the ghosts are read in.
template <bool F, class S>
__device__ __forceinline__ void periodicCell(const DevLevel& g, int idx) {
    const int cell = __ldg(g.perIndex + idx);
    const int src = __ldg(g.perSource + idx);
    int nb[8];
    Real<S> f[27];
    decodeNbr(g, src, nb, nullptr);
    readPre<F, S>(g, nb, f);
    decodeNbr(g, cell, nb, nullptr);
    writePre<F, S>(g, nb, f);
}

template <bool F, class S>
__global__ void __launch_bounds__(kBlock) periodicCopy(DevLevel g) {
    const int idx = blockIdx.x * kBlock + threadIdx.x;
    if (idx < g.perCount) periodicCell<F, S>(g, idx);
}

// K4-K6 (updateInterface, include/updateInterface.h:155-891): the interface
// between coarse level C and fine level Fn after the fine level's two
// substeps; FC and FF are the two levels' flippers after streaming.  Work
// units of 8 lanes: fine-to-coarse items, then coarse-to-fine blocks, then
// the leftover fine cells, 8 per unit (one per lane).  Reads and writes are
// disjoint: fine-to-coarse reads fine cells under fine-to-coarse coarse cells
// and writes those coarse cells; coarse-to-fine reads coarse-to-fine coarse
// cells and writes fine cells between their centres.
template <bool FC, bool FF, class S>
__global__ void __launch_bounds__(kBlock) interfaceExchange(DevLevel C, DevLevel Fn, DevInterface I) {
    using T = Real<S>;
    const int lane = threadIdx.x & 7;
    const unsigned mask = 0xFFu << (threadIdx.x & 24);
    const int unit = (blockIdx.x * kBlock + threadIdx.x) >> 3;
    const T omegaC = static_cast<T>(I.omegaCoarse), omegaF = static_cast<T>(I.omegaFine);
    if (unit < I.f2cCount) {
        // fine to coarse: the 8 children of the coarse cell, fitted at their centre
        int nb[8], nr[8];
        decodeNbr(Fn, __ldg(I.f2cChild + unit), nb, nullptr);
        decodeNbr(Fn, nb[lane], nr, nullptr);
        T f[27];
        readPre<FF, S>(Fn, nr, f);
        const itf::Fit<T> fit = itf::fitStencil(itf::cellMoments(f, omegaF), lane, mask, false);
        T out[27];
        itf::populationsFromGradient(out, fit.d0, fit.c0[0], fit.c0[1], fit.c0[2], fit.g, T(2) / omegaC);
        const int coarse = __ldg(I.f2cIndex + unit);
        decodeNbr(C, coarse, nb, nullptr);
        S* base = static_cast<S*>(C.f);
        const Dither D = stepDither<FC, S>(C, kSaltInterface);
        const unsigned cb = D.cell(coarse);
#pragma unroll
        for (int d = 0; d < 27; ++d)
            if ((d & 7) == lane) stD(base + (long long)preSlot<FC>(d) * C.stride + nb[preNbr(d)], out[d], D, cb, d);
        return;
    }
    if (unit < I.f2cCount + I.c2fCount) {
        // coarse to fine: the 8 coarse cells around a block of 8 fine cells
        const int u = unit - I.f2cCount;
        int nb[8], nr[8];
        decodeNbr(C, __ldg(I.c2fIndex + u), nb, nullptr);
        decodeNbr(C, nb[lane], nr, nullptr);
        T f[27];
        readPre<FC, S>(C, nr, f);
        const itf::Fit<T> fit = itf::fitStencil(itf::cellMoments(f, omegaC), lane, mask, true);
        // this lane's fine cell sits at +-1/4 coarse spacing from the centre
        const T x = itf::sgnX<T>(lane) * T(0.25), y = itf::sgnY<T>(lane) * T(0.25), z = itf::sgnZ<T>(lane) * T(0.25);
        T dRho, uv[3], G[3][3];
        itf::evalFit(fit, x, y, z, dRho, uv, G);
        T out[27];
        itf::populationsFromGradient(out, dRho, uv[0], uv[1], uv[2], G, T(0.5) / omegaF);
        decodeNbr(Fn, __ldg(I.c2fChild + u), nb, nullptr);
        decodeNbr(Fn, nb[lane], nr, nullptr);
        writePreD<FF, S>(Fn, nr, out, stepDither<FF, S>(Fn, kSaltInterface));
        return;
    }
    // leftovers: the parent plus one coarse neighbour per axis, linear
    // (include/updateInterface.h:694-884)
    const int idx = (unit - I.f2cCount - I.c2fCount) * 8 + lane;
    if (idx >= I.leftCount) return;
    const int parent = __ldg(I.leftParent + idx);
    int nb[8];
    T f[27];
    decodeNbr(C, parent, nb, nullptr);
    readPre<FC, S>(C, nb, f);
    const itf::CellMoments<T> mc = itf::cellMoments(f, omegaC);
    const int wm = __ldg(C.wallMap + parent);
    const unsigned wallData = wm >= 0 ? __ldg(C.wallData + wm) : 0u;
    T uw[3] = {mc.ux, mc.uy, mc.uz};
    if (wm >= 0)
        for (int a = 0; a < 3; ++a) uw[a] = static_cast<T>(__ldg(C.wallVel + (long long)a * C.wallCount + wm));
    T r[9] = {mc.d, mc.ux, mc.uy, mc.uz, mc.kxy, mc.kyz, mc.kxz, mc.kxxMyy, mc.kxxMzz};
    const T cen[9] = {mc.d, mc.ux, mc.uy, mc.uz, mc.kxy, mc.kyz, mc.kxz, mc.kxxMyy, mc.kxxMzz};
#pragma unroll 1
    for (int a = 0; a < 3; ++a) {
        int cell = __ldg(I.leftNbr + (long long)a * I.leftCount + idx);
        const bool opposite = cell < 0;
        if (opposite) cell = -cell - 1;
        decodeNbr(C, cell, nb, nullptr);
        readPre<FC, S>(C, nb, f);
        const itf::CellMoments<T> m = itf::cellMoments(f, omegaC);
        const T v[9] = {m.d, m.ux, m.uy, m.uz, m.kxy, m.kyz, m.kxz, m.kxxMyy, m.kxxMzz};
        if (!opposite) {
#pragma unroll
            for (int t = 0; t < 9; ++t) r[t] += T(0.25) * (v[t] - cen[t]);
            continue;
        }
        // extrapolate from the opposite side: density and moments always;
        // the velocity towards a wall bends to the wall velocity instead
        r[0] -= T(0.25) * (v[0] - cen[0]);
#pragma unroll
        for (int t = 4; t < 9; ++t) r[t] -= T(0.25) * (v[t] - cen[t]);
        const int dir = a == 0 ? POO : a == 1 ? OPO : OOP;
        const bool wall = (wallData & (1u << dir)) || (wallData & (1u << inv(dir)));
#pragma unroll
        for (int t = 1; t < 4; ++t)
            r[t] = wall ? r[t] + (T(1) / T(24)) * (T(10) * uw[t - 1] - T(9) * cen[t] - v[t]) : r[t] - T(0.25) * (v[t] - cen[t]);
    }
    // the moments are strain estimates: (kxy, kyz, kxz) = off-diagonal
    // gradient sums, kxxMyy / kxxMzz = diagonal differences
    const T G[3][3] = {{T(0), r[4], r[6]}, {T(0), -r[7], r[5]}, {T(0), T(0), -r[8]}};
    T out[27];
    itf::populationsFromGradient(out, r[0], r[1], r[2], r[3], G, T(0.5) / omegaF);
    decodeNbr(Fn, __ldg(I.leftIndex + idx), nb, nullptr);
    writePreD<FF, S>(Fn, nb, out, stepDither<FF, S>(Fn, kSaltInterface));
}

// Characteristic (non-reflective) normal velocity of a face cell: the
// outgoing Riemann invariant of the streamed state against the reference
// values (include/updateGrid.h:268-308).
// Non-reflecting density of the impedance scheme from the previous completed
// boundary state (dRhoPrev, uNormalPrev) and the streamed partial density
// sum dRhoZ: the root of the characteristic quadratic in dRho, written as
// H / (B + sqrt(B^2 + D H)) so that it stays well conditioned
// (cases/nonReflectiveTest/updateGrid_SCHLAFFER_IMPEDANCE_SCHEME.h:268-280).
template <class V>
__device__ __forceinline__ V impedanceDRho(V dRhoPrev, V uNormalPrev, V dRhoZ) {
    const V cs = V(0.57735026918962576f);  // INVSQRT3 of the FP32 build
    const V cs2 = cs * cs;
    const V bracket = uNormalPrev + cs + V(1);
    const V t = uNormalPrev - dRhoZ;
    const V Dq = fma(bracket, bracket, cs2);
    const V B = fma(bracket, cs + t, -cs2 * dRhoPrev);
    const V H = fma(-t, V(2) * cs + t, V(2) * cs2 * dRhoPrev);
    const V disc = fma(Dq, H, B * B);
    return H / (B + sqrt(disc));
}

template <class V>
__device__ __forceinline__ V nonReflectiveUNormal(V uTarget, V dRhoZ, V dRhoRef) {
    const V cs = V(0.57735026918962576);  // 1/sqrt(3)
    const V rhoRef = dRhoRef + V(1);
    const V rhoTerm = (dRhoZ - dRhoRef) / rhoRef;
    const V numerator = V(2) * (uTarget + cs * rhoTerm);
    const V root = (V(1) + cs - uTarget) * (V(1) + cs - uTarget) + V(4) * (uTarget + cs * rhoTerm);
    const V denominator = V(1) + cs - uTarget + sqrt(root);
    return numerator / denominator;
}

// K2 (include/updateGrid.h:181-355), run after the flip, so F is the flipper
// of the next step's pre-collision read.  Open cells are grouped by outer
// normal into chunks of kOpenChunk; one CTA takes one chunk and stages that
// normal's direction-indexed closure tables in shared memory, so every thread
// of the CTA follows the same branches and its 27 populations stay in
// registers.  Known populations (c.n >= 0 on every axis) are read and
// weight-compensated, the missing macroscopic quantity is restored, the
// unknown populations are closed from equilibrium moments and written to the
// cell's own pre-collision slots.  All open-boundary IDs go in one launch:
// their cells are disjoint and a cell touches only its own 27 slots, so the
// reference's loop over IDs gives the same result in any order.
#ifndef LBM3_OPEN_MIN_BLOCKS
#define LBM3_OPEN_MIN_BLOCKS 8
#endif
// The open-boundary launch's last CTA advances the device iteration count.
__device__ __forceinline__ void openBoundaryDone(const DevLevel& g) {
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(g.obCounter + 1, 1) == g.obChunkCount - 1) {
            g.obCounter[1] = 0;
            g.obCounter[0] += 1;
            __threadfence();
        }
    }
}

// One open cell's inputs: its records and its known populations after streaming.
template <class V> struct OpenCell {
    int idx, info;
    int4 rows;
    float dRhoRef, uNormalRef, beta;
    float4 target;
    V f[27];
};

// Issue the loads of open cell `idx` (records and the known populations of a
// chunk with unknown-direction mask `unknown`); nothing waits on them here.
template <bool F, class S>
__device__ __forceinline__ void openLoad(const DevLevel& g, int idx, unsigned unknown, bool active,
                                         OpenCell<Real<S>>& c) {
    using V = Real<S>;
    c.idx = idx;
    c.info = __ldg(g.obInfo + idx);
    c.rows = __ldg(g.obNbr + idx);
    c.dRhoRef = g.obRhoRef[idx];
    c.uNormalRef = g.obUnRef[idx];
    c.target = __ldg(g.obTarget + idx);
    c.beta = __ldg(g.obBeta + idx);
    const int n = g.cellCount;
    int nb[8];
    nb[0] = c.rows.x;
    nb[1] = c.rows.x + 1 < n ? c.rows.x + 1 : 0;
    nb[2] = c.rows.y;
    nb[3] = c.rows.y + 1 < n ? c.rows.y + 1 : 0;
    nb[4] = c.rows.z;
    nb[5] = c.rows.z + 1 < n ? c.rows.z + 1 : 0;
    nb[6] = c.rows.w;
    nb[7] = c.rows.w + 1 < n ? c.rows.w + 1 : 0;
    const S* base = static_cast<const S*>(g.f);
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        c.f[d] = V(0);
        if (active && !(unknown >> d & 1u))
            c.f[d] = Store<S>::ldL2(base + (long long)preSlot<F>(d) * g.stride + nb[preNbr(d)]);
    }
}

// Close one open cell with the table T of its outer normal: restore the
// missing macroscopic quantity, write the unknown populations, update the
// reference averages and the flow sums.
template <bool F, class S>
__device__ __forceinline__ void openClose(const DevLevel& g, const MbbcDirT<Real<S>>& T, unsigned unknown,
                                          int iterationsFinished, OpenCell<Real<S>>& c) {
    using V = Real<S>;
    const int info = c.info;
    const int nx = ((info >> 3) & 3) - 1, ny = ((info >> 5) & 3) - 1, nz = ((info >> 7) & 3) - 1;
    const int n = g.cellCount;
    S* base = static_cast<S*>(g.f);
    V dRhoZ = V(0);
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        if (unknown >> d & 1u) continue;
        if (nx * cx(d) + ny * cy(d) + nz * cz(d) == 0) dRhoZ += c.f[d];
        else dRhoZ += V(2) * c.f[d];
        c.f[d] += weightT<V>(d);  // the closure is ill-conditioned on shifted populations
    }
    V dRho = c.target.x, ux = c.target.y, uy = c.target.z, uz = c.target.w;
    // face cells only (the host clears the flag on edges and corners)
    const bool nonReflective = (info & 4) && !g.obImpedance;
    // impedance scheme: clamp the given value to within the tolerance of the
    // non-reflecting state of the previous completed boundary state, which
    // the reference arrays hold under this scheme
    const bool impedance = (info & 4) && g.obImpedance && g.obTolerance < 1.f;
    const V tol = V(g.obTolerance);
    const V dRhoNR = impedance ? impedanceDRho<V>(V(c.dRhoRef), V(c.uNormalRef), dRhoZ) : V(0);
    if ((info & 3) == 2) {  // pressure: density given, velocity restored
        if (nonReflective) {
            const V uNormal = nonReflectiveUNormal<V>(c.uNormalRef, dRhoZ, dRho);
            dRho = (dRhoZ - uNormal) / (V(1) + uNormal);
        }
        if (impedance) dRho = fmin(fmax(dRho, dRhoNR - tol), dRhoNR + tol);
        mbbcRestoreU(T, dRho + V(1), c.f, ux, uy, uz);
    } else if ((info & 3) == 1) {  // velocity: velocity given, density restored
        if (impedance) {
            const V uMin = (dRhoZ - dRhoNR - tol) / (dRhoNR + V(1) + tol);
            const V uMax = (dRhoZ - dRhoNR + tol) / (dRhoNR + V(1) - tol);
            if (nx > 0) ux = fmin(fmax(ux, uMin), uMax);
            if (nx < 0) ux = fmin(fmax(ux, -uMax), -uMin);
            if (ny > 0) uy = fmin(fmax(uy, uMin), uMax);
            if (ny < 0) uy = fmin(fmax(uy, -uMax), -uMin);
            if (nz > 0) uz = fmin(fmax(uz, uMin), uMax);
            if (nz < 0) uz = fmin(fmax(uz, -uMax), -uMin);
        }
        if (nonReflective) {
            V uTarget = V(0);
            if (nx != 0) uTarget = nx > 0 ? ux : -ux;
            if (ny != 0) uTarget = ny > 0 ? uy : -uy;
            if (nz != 0) uTarget = nz > 0 ? uz : -uz;
            const V uNormal = nonReflectiveUNormal<V>(uTarget, dRhoZ, c.dRhoRef);
            if (nx != 0) ux = nx > 0 ? uNormal : -uNormal;
            if (ny != 0) uy = ny > 0 ? uNormal : -uNormal;
            if (nz != 0) uz = nz > 0 ? uNormal : -uNormal;
        }
        dRho = mbbcRestoreRho(T, ux, uy, uz, c.f) - V(1);
    }
    // closure: all unknown rows at once, each written to its pre-collision
    // slot (F ? inv(d) : d) in the neighbour offset by max(0, -c_d)
    V closed[kMbbcRowPad];
    {
        V meq[kMbbcMoments];
        mbbcMomentsEq(dRho + V(1), ux, uy, uz, meq);
        mbbcClose(T, unknown, (T.nu + 3) >> 2, meq, c.f, closed);
    }
    const Dither D = stepDither<F, S>(g, kSaltOpen);
    const unsigned cb = D.cell(c.rows.x);
#pragma unroll
    for (int r = 0; r < kMbbcRowPad; ++r) {
        if (r >= T.nu) break;
        const int k = T.unknownNbr[r];
        const int sel = k >> 1;
        int cell = sel == 0 ? c.rows.x : sel == 1 ? c.rows.y : sel == 2 ? c.rows.z : c.rows.w;
        if (k & 1) cell = cell + 1 < n ? cell + 1 : 0;
        const int slot = F ? T.unknownInv[r] : T.unknownDir[r];
        stD(base + (long long)slot * g.stride + cell, closed[r] - T.unknownW[r], D, cb, r);
    }
    // reference values: exponential average whose weight decays with the
    // iteration count; below 1e-5 the weight is tripled and the update runs
    // every 3^k iterations instead (include/updateGrid.h:325-347)
    const float uNormal = float(V(nx) * ux + V(ny) * uy + V(nz) * uz);
    if (g.obImpedance) {
        // the completed state, for the next step's non-reflecting state
        g.obRhoRef[c.idx] = float(dRho);
        g.obUnRef[c.idx] = uNormal;
    } else {
        float alpha = c.beta / ((float)iterationsFinished + c.beta + 10.f);
        int updateEvery = 1;
        while (alpha < 1.e-5f) {
            alpha *= 3.f;
            updateEvery *= 3;
        }
        if (iterationsFinished % updateEvery == 0) {
            g.obRhoRef[c.idx] = fmaf(alpha, float(dRho) - c.dRhoRef, c.dRhoRef);
            g.obUnRef[c.idx] = fmaf(alpha, uNormal - c.uNormalRef, c.uNormalRef);
        }
    }
    if (g.trackOpen && (info & 512)) {
        g.obRhoCum[c.idx] += float(dRho);
        g.obUnCum[c.idx] += uNormal;
    }
}

// Stage the closure tables of normal row `row` in shared memory.
template <class V> __device__ __forceinline__ void openStageTable(const DevLevel& g, int row, MbbcDirT<V>& T) {
    const int4* src = reinterpret_cast<const int4*>(static_cast<const MbbcDirT<V>*>(g.obTables) + row);
    int4* dst = reinterpret_cast<int4*>(&T);
    for (int q = threadIdx.x; q < int(sizeof(MbbcDirT<V>) / 16); q += blockDim.x) dst[q] = __ldg(src + q);
}

// One chunk of open cells on one CTA: the table staging overlaps the gathers.
template <bool F, class S>
__device__ __forceinline__ void openBoundaryChunk(const DevLevel& g, int chunkIndex, MbbcDirT<Real<S>>& T) {
    using V = Real<S>;
    // the level's finished iterations live on the device (obCounter[0]), so
    // a captured step graph replays with the right count; the last CTA of the
    // level's chunks advances it once every CTA has read it
    const int iterationsFinished = __ldcg(g.obCounter);
    const int4 chunk = __ldg(g.obChunk + chunkIndex);  // {first, count, normal row, unknown mask}
    openStageTable(g, chunk.z, T);
    const bool active = int(threadIdx.x) < chunk.y;
    OpenCell<V> c;
    openLoad<F, S>(g, chunk.x + (active ? int(threadIdx.x) : 0), static_cast<unsigned>(chunk.w), active, c);
    __syncthreads();
    if (active) openClose<F, S>(g, T, static_cast<unsigned>(chunk.w), iterationsFinished, c);
    openBoundaryDone(g);  // thread 0 is always active
}

// One chunk per CTA.
template <bool F, class S>
__global__ void __launch_bounds__(kOpenChunk, LBM3_OPEN_MIN_BLOCKS) openBoundary(DevLevel g) {
    __shared__ MbbcDirT<Real<S>> T;
    openBoundaryChunk<F, S>(g, blockIdx.x, T);
}


// Initial reference values of the open boundary (applyInitialCondition.h:43-81).
template <bool F, class S>
__global__ void __launch_bounds__(kBlock) openBoundaryInit(DevLevel g) {
    const int idx = blockIdx.x * kBlock + threadIdx.x;
    if (idx >= g.obCount) return;
    const int cell = __ldg(g.obCell + idx);
    const int info = __ldg(g.obInfo + idx);
    const int nx = ((info >> 3) & 3) - 1, ny = ((info >> 5) & 3) - 1, nz = ((info >> 7) & 3) - 1;
    int nb[8];
    decodeNbr(g, cell, nb, nullptr);
    using V = Real<S>;
    V f[27];
    readPre<F, S>(g, nb, f);
    V dRho, ux, uy, uz;
    macroFromF(f, dRho, ux, uy, uz);
    g.obRhoRef[idx] = float(dRho);
    g.obUnRef[idx] = float(V(nx) * ux + V(ny) * uy + V(nz) * uz);
}

// getFeq (include/cellFunctions.h:125-148) with rounding-exact intrinsics so
// the initial state is bit-identical to a host evaluation.
__device__ __forceinline__ void feqExact(float dRho, float ux, float uy, float uz, float (&feq)[27]) {
    const float ux2 = __fmul_rn(ux, ux), uy2 = __fmul_rn(uy, uy), uz2 = __fmul_rn(uz, uz);
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        const float X = float(cx(q)), Y = float(cy(q)), Z = float(cz(q));
        const float dx = __fadd_rn(__fmul_rn(__fmul_rn(3.f, X), ux),
                                   __fmul_rn(__fadd_rn(__fmul_rn(__fmul_rn(4.5f, X), X), -1.5f), ux2));
        const float dy = __fadd_rn(__fmul_rn(__fmul_rn(3.f, Y), uy),
                                   __fmul_rn(__fadd_rn(__fmul_rn(__fmul_rn(4.5f, Y), Y), -1.5f), uy2));
        const float dz = __fadd_rn(__fmul_rn(__fmul_rn(3.f, Z), uz),
                                   __fmul_rn(__fadd_rn(__fmul_rn(__fmul_rn(4.5f, Z), Z), -1.5f), uz2));
        const float xy = __fadd_rn(__fadd_rn(dx, dy), __fmul_rn(dx, dy));
        const float corr = __fadd_rn(__fadd_rn(xy, dz), __fmul_rn(xy, dz));
        feq[q] = __fmul_rn(weight(q), __fadd_rn(__fadd_rn(dRho, corr), __fmul_rn(dRho, corr)));
    }
}

// getFeq in double for the FP64 build (the same expression, FP64 throughout).
__device__ __forceinline__ void feqExact(double dRho, double ux, double uy, double uz, double (&feq)[27]) {
    const double ux2 = ux * ux, uy2 = uy * uy, uz2 = uz * uz;
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        const double X = cx(q), Y = cy(q), Z = cz(q);
        const double dx = 3.0 * X * ux + (4.5 * X * X - 1.5) * ux2;
        const double dy = 3.0 * Y * uy + (4.5 * Y * Y - 1.5) * uy2;
        const double dz = 3.0 * Z * uz + (4.5 * Z * Z - 1.5) * uz2;
        const double xy = dx + dy + dx * dy;
        const double corr = xy + dz + xy * dz;
        feq[q] = weightT<double>(q) * (dRho + corr + dRho * corr);
    }
}

template <bool F, class S>
__global__ void __launch_bounds__(kBlock) initFeq(DevLevel g, const float4* macro, float4 uniform) {
    const int cell = blockIdx.x * kBlock + threadIdx.x;
    if (cell >= g.cellCount) return;
    const float4 m = macro ? macro[cell] : uniform;
    int nb[8];
    decodeNbr(g, cell, nb, nullptr);
    using V = Real<S>;
    V f[27];
    feqExact(V(m.x), V(m.y), V(m.z), V(m.w), f);
    writePre<F, S>(g, nb, f);
}

__device__ __forceinline__ double warpSum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

template <bool F, class S>
__global__ void __launch_bounds__(kBlock) kineticEnergy(DevLevel g, double* out) {
    const int cell = blockIdx.x * kBlock + threadIdx.x;
    double e = 0.0;
    if (cell < g.cellCount) {
        const int wm = __ldg(g.wallMap + cell);
        // walls, interface duplicates and periodic ghosts are excluded
        // (cases/taylorGreenVortex/taylorGreenVortexMain.cu:139-141)
        const bool overlap = wm >= 0 && (__ldg(g.wallData + wm) & 1u);
        if (wm != -3 && wm != -2 && !overlap) {
            int nb[8];
            decodeNbr(g, cell, nb, nullptr);
            Real<S> f[27];
            readPre<F, S>(g, nb, f);
            Real<S> dRho, ux, uy, uz;
            macroFromF(f, dRho, ux, uy, uz);
            e = 0.5 * (1.0 + double(dRho)) *
                (double(ux) * ux + double(uy) * uy + double(uz) * uz);
        }
    }
    __shared__ double part[kBlock / 32];
    e = warpSum(e);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = e;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < kBlock / 32 ? part[threadIdx.x] : 0.0;
        v = warpSum(v);
        if (threadIdx.x == 0) atomicAdd(out, v);
    }
}

// FP64 global sums over the fluid cells (walls, periodic ghosts and
// interface duplicates excluded, as in the kinetic energy): out[0] sum of rho,
// out[1] sum of dRho, out[2..4] sum of rho u (momentum), out[5] cell count.
// The populations are read in the kernel's arithmetic type and each cell's
// contribution is formed in FP64.
template <bool F, class S>
__global__ void __launch_bounds__(kBlock) globalSums(DevLevel g, double* out) {
    const int cell = blockIdx.x * kBlock + threadIdx.x;
    double v[6] = {0, 0, 0, 0, 0, 0};
    if (cell < g.cellCount) {
        const int wm = __ldg(g.wallMap + cell);
        const bool overlap = wm >= 0 && (__ldg(g.wallData + wm) & 1u);
        if (wm != -3 && wm != -2 && !overlap) {
            int nb[8];
            decodeNbr(g, cell, nb, nullptr);
            Real<S> f[27];
            readPre<F, S>(g, nb, f);
            double dRho = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
#pragma unroll
            for (int d = 0; d < 27; ++d) {
                const double fd = f[d];
                dRho += fd;
                mx += cx(d) * fd;
                my += cy(d) * fd;
                mz += cz(d) * fd;
            }
            v[0] = 1.0 + dRho;
            v[1] = dRho;
            v[2] = mx;
            v[3] = my;
            v[4] = mz;
            v[5] = 1.0;
        }
    }
    __shared__ double part[6][kBlock / 32];
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        double a = v[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
        if ((threadIdx.x & 31) == 0) part[q][threadIdx.x >> 5] = a;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        double a = 0.0;
        for (int k = 0; k < kBlock / 32; ++k) a += part[threadIdx.x][k];
        atomicAdd(out + threadIdx.x, a);
    }
}

template <bool F, class S>
__global__ void __launch_bounds__(kBlock) macroFields(DevLevel g, float* out) {
    const int cell = blockIdx.x * kBlock + threadIdx.x;
    if (cell >= g.cellCount) return;
    int nb[8];
    decodeNbr(g, cell, nb, nullptr);
    Real<S> f[27];
    readPre<F, S>(g, nb, f);
    Real<S> dRho, ux, uy, uz;
    macroFromF(f, dRho, ux, uy, uz);
    const long long n = g.cellCount;
    out[cell] = float(dRho);
    out[n + cell] = float(ux);
    out[2 * n + cell] = float(uy);
    out[3 * n + cell] = float(uz);
}

template <bool F, class S>
__global__ void __launch_bounds__(kBlock) gatherF(DevLevel g, float* out) {
    // raw slot copy: out[slot][cell] = f[slot][cell] as FP32 (planes are
    // stride apart on the device, cellCount apart in the output)
    const long long i = (long long)blockIdx.x * kBlock + threadIdx.x;
    const long long n = g.cellCount;
    if (i >= 27 * n) return;
    const long long slot = i / n, cell = i - slot * n;
    out[i] = Store<S>::ld(static_cast<const S*>(g.f) + slot * g.stride + cell);
}

template <class S>
__global__ void __launch_bounds__(kBlock) scatterF(DevLevel g, const float* in) {
    const long long i = (long long)blockIdx.x * kBlock + threadIdx.x;
    const long long n = g.cellCount;
    if (i >= 27 * n) return;
    const long long slot = i / n, cell = i - slot * n;
    Store<S>::st(static_cast<S*>(g.f) + slot * g.stride + cell, in[i]);
}

#if LBM3_SHARED_UNIT
__global__ void __launch_bounds__(kBlock) collideBatch(float* f, int n, CollisionConsts P,
                                                       float gx, float gy, float gz) {
    const int c = blockIdx.x * kBlock + threadIdx.x;
    if (c >= n) return;
    float v[27];
#pragma unroll
    for (int d = 0; d < 27; ++d) v[d] = f[(long long)d * n + c];
    collideCumulant(v, P, P.lambda, gx, gy, gz);
#pragma unroll
    for (int d = 0; d < 27; ++d) f[(long long)d * n + c] = v[d];
}
#endif

// ---- packed batch ------------------------------------------------------------
// Domains of a batch advance together: one persistent collide-stream launch
// takes work items from the packed table of all domains (listed-cell chunks
// and bulk tiles of domain 0, then of domain 1, ...), so small domains fill
// the GPU together instead of one underfilled launch each, and the open
// boundary and periodic ghosts of all domains take one launch each.  A CTA
// stages the level descriptor of its item's domain in shared memory when the
// domain changes (a domain's items are contiguous, so that happens a few
// times per CTA and launch); the work per item is the paired kernel's, so a
// domain's result is bit-identical to stepping it alone.

// Copy a level descriptor into shared memory (all threads of the CTA).
__device__ __forceinline__ void stageLevel(const DevLevel* src, DevLevel& dst) {
    static_assert(sizeof(DevLevel) % 8 == 0, "descriptor copied in 8-byte words");
    const long long* s = reinterpret_cast<const long long*>(src);
    long long* d = reinterpret_cast<long long*>(&dst);
    for (int q = threadIdx.x; q < int(sizeof(DevLevel) / 8); q += blockDim.x) d[q] = __ldg(s + q);
}

template <bool F, class S>
__global__ void __launch_bounds__(kHalf, LBM3_PAIR_MIN_BLOCKS) collidePacked(DevBatch b) {
    __shared__ int slot[2];
    __shared__ DevLevel sg;
    const int t = threadIdx.x;
    if constexpr (sizeof(S) == 2) {
        // every domain's next step seed (advanceDither of the single-domain launch)
        if (blockIdx.x == 0)
            for (int q = t; q < b.domainCount; q += kHalf) {
                unsigned* seed = b.levels[q].seed;
                seed[F ? 0 : 1] = mix32(seed[F ? 1 : 0] + 0x6D2B79F5u);
            }
    }
    int parity = 0;
    auto fetch = [&](int domain) {
        if (t == 0) slot[parity] = atomicAdd(b.work + domain, 1);
        __syncthreads();
        const int v = slot[parity];
        parity ^= 1;
        return v;
    };
    // Each domain has its own item counter.  A CTA starts on its home domain
    // (blockIdx modulo the domain count) and moves on to the next domain when
    // that one runs out, so it stages a descriptor at most once per domain.
    const int D = b.domainCount;
    int dom = static_cast<int>(blockIdx.x % unsigned(D));
    for (int visited = 0; visited < D; ++visited, dom = dom + 1 == D ? 0 : dom + 1) {
        const int count = b.itemStart ? __ldg(b.itemStart + dom + 1) - __ldg(b.itemStart + dom) : b.collideCount;
        if (count <= 0) continue;
        int item = fetch(dom);
        if (item >= count) continue;  // CTA-uniform
        __syncthreads();              // every thread is done with the previous descriptor
        stageLevel(b.levels + dom, sg);
        __syncthreads();
        const int nSpecial = (sg.specialCount + kTile - 1) / kTile;
        while (item < count) {  // CTA-uniform: items come through shared memory
            int next;
            if (item < nSpecial) {  // CTA-uniform branch: both sides fetch once
                next = fetch(dom);
                const int q = item * kTile + t;
                if (q < sg.specialCount) collideSpecialCell<F, S>(sg, __ldg(sg.special + q));
                if (q + kHalf < sg.specialCount) collideSpecialCell<F, S>(sg, __ldg(sg.special + q + kHalf));
            } else {
                int4 d;
                int l;
                loadDesc(sg, item - nSpecial, d, l);
                Pair f[27];
                loadTilePair<F, S>(sg, d, t, l, f);
                next = fetch(dom);  // the atomic and the barrier overlap the tile's loads in flight
                collideCumulantT(f, sg.coll, sg.coll.lambda, sg.gx, sg.gy, sg.gz);
                storePair<F, S>(sg, d, t, l, f, stepDither<F, S>(sg, kSaltCollide));
            }
            item = next;
        }
    }
    if (t == 0) {
        __threadfence();
        if (atomicAdd(b.work + D, 1) == int(gridDim.x) - 1) {
            for (int q = 0; q <= D; ++q) b.work[q] = 0;
            __threadfence();
        }
    }
}

// One open-boundary chunk of one domain per CTA.
template <bool F, class S>
__global__ void __launch_bounds__(kOpenChunk, LBM3_OPEN_MIN_BLOCKS) openPacked(DevBatch b) {
    __shared__ MbbcDirT<Real<S>> T;
    __shared__ DevLevel sg;
    const int2 it = __ldg(b.openItems + blockIdx.x);
    stageLevel(b.levels + it.x, sg);
    __syncthreads();
    openBoundaryChunk<F, S>(sg, it.y, T);
}

// Periodic ghosts of all domains, one thread per ghost.
template <bool F, class S>
__global__ void __launch_bounds__(kBlock) periodicPacked(DevBatch b) {
    const int idx = blockIdx.x * kBlock + threadIdx.x;
    if (idx >= b.periodicCount) return;
    // the last domain whose first ghost is at or before idx (domains without
    // ghosts share their start with the next one)
    int lo = 0, hi = b.domainCount - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(b.periodicStart + mid) <= idx) lo = mid;
        else hi = mid - 1;
    }
    periodicCell<F, S>(b.levels[lo], idx - __ldg(b.periodicStart + lo));
}

inline unsigned blocksFor(long long n) { return static_cast<unsigned>((n + kBlock - 1) / kBlock); }

// Dispatch on the flipper; this translation unit holds the kernels of one
// storage type (LBM3_STEP_STORAGE), step_dispatch.cu picks the unit.
template <template <bool, class> class K, class... A>
void dispatch(const DevLevel& g, bool flip, A&&... args) {
    flip ? K<true, StepStore>::run(g, args...) : K<false, StepStore>::run(g, args...);
}

// Persistent grid size of a kernel on the current device: SMs x resident
// CTAs.  Cached per device and kernel (devices may differ in SM count); a
// kernel that needs more than the default dynamic shared memory gets the
// attribute set before its occupancy is queried.
template <class K> int persistentGrid(K kernel, int block, int smem) {
    static std::mutex m;
    static std::map<std::pair<int, const void*>, int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    const std::pair<int, const void*> key(dev, reinterpret_cast<const void*>(kernel));
    std::lock_guard<std::mutex> lock(m);
    const auto hit = cache.find(key);
    if (hit != cache.end()) return hit->second;
    int sms = 0, perSm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (smem > 0) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, block, smem);
    const int grid = (sms > 0 ? sms : 1) * (perSm > 0 ? perSm : 1);
    cache[key] = grid;
    return grid;
}

// The paired persistent kernel: listed cells and bulk tiles in one launch
// (FP32 arithmetic on two cells per thread), then the rotor cells.
// One domain through the packed batch's kernel (a batch of one, its
// descriptor read from the device copy): the same machine code as the
// domain inside a batch, so the same results bit for bit
// (LBM3_COLLIDE_KERNEL=packed; a one-member lbm_batch does the same).
template <bool F, class S> struct RunCollidePair {
    static void run(const DevLevel& g, cudaStream_t s) {
        if constexpr (!std::is_same<S, double>::value) {
            const int items = g.segCount + (g.specialCount + kTile - 1) / kTile;
            if (items > 0) {
                DevBatch b{};
                b.levels = g.self;
                b.domainCount = 1;
                b.itemStart = nullptr;
                b.collideCount = items;
                b.work = g.work;
                const int grid = persistentGrid(collidePacked<F, S>, kHalf, 0);
                collidePacked<F, S><<<std::min(grid, items), kHalf, 0, s>>>(b);
            }
            if (g.rotorCellCount > 0) collideRotorList<F, S><<<blocksFor(g.rotorCellCount), kBlock, 0, s>>>(g);
        }
    }
};

// One step of a packed batch: collide-stream at flipper F, then the open
// boundary and periodic ghosts on the streamed state (!F).
template <bool F, class S> struct RunPackedStep {
    static void run(const DevBatch& b, cudaStream_t s) {
        if constexpr (!std::is_same<S, double>::value) {
            if (b.collideCount > 0) {
                const int grid = persistentGrid(collidePacked<F, S>, kHalf, 0);
                collidePacked<F, S><<<std::min(grid, b.collideCount), kHalf, 0, s>>>(b);
            }
            if (b.openCount > 0) openPacked<!F, S><<<b.openCount, kOpenChunk, 0, s>>>(b);
            if (b.periodicCount > 0) periodicPacked<!F, S><<<blocksFor(b.periodicCount), kBlock, 0, s>>>(b);
        }
    }
};

// The other collide-stream variants (LBM3_COLLIDE_KERNEL), the FP64 build
// and grids too large for the paired kernel's 32-bit offsets.
template <bool F, class S> struct RunCollideOther {
    static void run(const DevLevel& g, cudaStream_t s, CollideVariant v) {
        if (v == CollideVariant::Simple) {
            collideStream<F, S><<<blocksFor(g.cellCount), kBlock, 0, s>>>(g);
            return;
        }
        if (v == CollideVariant::Pair) {
            // the paired kernel with the descriptor as a kernel parameter
            // (faster on one large domain than the packed kernel's staged copy)
            if constexpr (!std::is_same<S, double>::value) {
                const int items = g.segCount + (g.specialCount + kTile - 1) / kTile;
                if (items > 0) {
                    const int grid = persistentGrid(collidePair<F, S>, kHalf, 0);
                    collidePair<F, S><<<std::min(grid, items), kHalf, 0, s>>>(g);
                }
            }
        } else if (v == CollideVariant::Tma) {
            if (g.segCount > 0) {
                const int grid = persistentGrid(collideBulkTma<F, S>, kTile, tmaSmemBytes<S>());
                persistentGrid(collideBulkTma<!F, S>, kTile, tmaSmemBytes<S>());
                collideBulkTma<F, S><<<std::min(grid, g.segCount), kTile, tmaSmemBytes<S>(), s>>>(g);
            }
            if (g.specialCount > 0) collideList<F, S><<<blocksFor(g.specialCount), kBlock, 0, s>>>(g);
        } else {
            // bulk segments and listed cells in one persistent launch
            const int items = g.segCount + (g.specialCount + kTile - 1) / kTile;
            if (items > 0) {
                const int grid = persistentGrid(collidePrefetch<F, S>, kTile, 0);
                collidePrefetch<F, S><<<std::min(grid, items), kTile, 0, s>>>(g);
            }
        }
        if (g.rotorCellCount > 0) collideRotorList<F, S><<<blocksFor(g.rotorCellCount), kBlock, 0, s>>>(g);
    }
};

template <class S> void runInterface(const DevLevel& c, const DevLevel& f, const DevInterface& I, bool flipC,
                                     bool flipF, cudaStream_t s) {
    const long long units = static_cast<long long>(I.f2cCount) + I.c2fCount + (I.leftCount + 7) / 8;
    if (units <= 0) return;
    const unsigned blocks = static_cast<unsigned>((units * 8 + kBlock - 1) / kBlock);
    if (flipC)
        flipF ? interfaceExchange<true, true, S><<<blocks, kBlock, 0, s>>>(c, f, I)
              : interfaceExchange<true, false, S><<<blocks, kBlock, 0, s>>>(c, f, I);
    else
        flipF ? interfaceExchange<false, true, S><<<blocks, kBlock, 0, s>>>(c, f, I)
              : interfaceExchange<false, false, S><<<blocks, kBlock, 0, s>>>(c, f, I);
}

template <bool F, class S> struct RunPeriodic {
    static void run(const DevLevel& g, cudaStream_t s) {
        if (g.perCount > 0) periodicCopy<F, S><<<blocksFor(g.perCount), kBlock, 0, s>>>(g);
    }
};
template <bool F, class S> struct RunOpen {
    static void run(const DevLevel& g, cudaStream_t s) {
        if (g.obChunkCount > 0) openBoundary<F, S><<<g.obChunkCount, kOpenChunk, 0, s>>>(g);
    }
};
template <bool F, class S> struct RunOpenInit {
    static void run(const DevLevel& g, cudaStream_t s) {
        if (g.obCount > 0) openBoundaryInit<F, S><<<blocksFor(g.obCount), kBlock, 0, s>>>(g);
    }
};
template <bool F, class S> struct RunFlowReport {
    static void run(const DevLevel& g, cudaStream_t s, int plane, int layer, int h0, int h1, int v0, int v1,
                    double* out) {
        flowReportSum<F, S><<<blocksFor(g.cellCount), kBlock, 0, s>>>(g, plane, layer, h0, h1, v0, v1, out);
    }
};
template <bool F, class S> struct RunFlowImage {
    static void run(const DevLevel& g, cudaStream_t s, const FlowImagePass& a, float* img) {
        flowImageLevel<F, S><<<blocksFor(g.cellCount), kBlock, 0, s>>>(g, a, img);
    }
};
template <bool F, class S> struct RunInit {
    static void run(const DevLevel& g, cudaStream_t s, const float4* macro, float4 u) {
        initFeq<F, S><<<blocksFor(g.cellCount), kBlock, 0, s>>>(g, macro, u);
    }
};
template <bool F, class S> struct RunEnergy {
    static void run(const DevLevel& g, cudaStream_t s, double* out) {
        kineticEnergy<F, S><<<blocksFor(g.cellCount), kBlock, 0, s>>>(g, out);
    }
};
template <bool F, class S> struct RunGlobalSums {
    static void run(const DevLevel& g, cudaStream_t s, double* out) {
        globalSums<F, S><<<blocksFor(g.cellCount), kBlock, 0, s>>>(g, out);
    }
};
template <bool F, class S> struct RunMacro {
    static void run(const DevLevel& g, cudaStream_t s, float* out) {
        macroFields<F, S><<<blocksFor(g.cellCount), kBlock, 0, s>>>(g, out);
    }
};
template <bool F, class S> struct RunGather {
    static void run(const DevLevel& g, cudaStream_t s, float* out) {
        gatherF<F, S><<<blocksFor(27LL * g.cellCount), kBlock, 0, s>>>(g, out);
    }
};
template <bool F, class S> struct RunScatter {
    static void run(const DevLevel& g, cudaStream_t s, const float* in) {
        scatterF<S><<<blocksFor(27LL * g.cellCount), kBlock, 0, s>>>(g, in);
    }
};

}  // namespace

#define LBM3_FN(name) LBM3_STEP_JOIN(name, LBM3_STEP_SUFFIX)

#if LBM3_PART(1)
void LBM3_FN(launchCollidePair)(const DevLevel& g, bool flip, cudaStream_t s) { dispatch<RunCollidePair>(g, flip, s); }
#endif
#if LBM3_PART(2)
void LBM3_FN(launchCollideOther)(const DevLevel& g, bool flip, cudaStream_t s, CollideVariant v) {
    dispatch<RunCollideOther>(g, flip, s, v);
}
#endif
#if LBM3_PART(3)
void LBM3_FN(launchPeriodic)(const DevLevel& g, bool flip, cudaStream_t s) { dispatch<RunPeriodic>(g, flip, s); }
void LBM3_FN(launchInterface)(const DevLevel& coarse, const DevLevel& fine, const DevInterface& I, bool flipCoarse,
                              bool flipFine, cudaStream_t s) {
    runInterface<StepStore>(coarse, fine, I, flipCoarse, flipFine, s);
}
void LBM3_FN(launchOpenBoundary)(const DevLevel& g, bool flip, cudaStream_t s) {
    dispatch<RunOpen>(g, flip, s);
}
void LBM3_FN(launchOpenBoundaryInit)(const DevLevel& g, bool flip, cudaStream_t s) { dispatch<RunOpenInit>(g, flip, s); }
void LBM3_FN(launchInit)(const DevLevel& g, bool flip, cudaStream_t s, const float4* macro, float4 uniform) {
    dispatch<RunInit>(g, flip, s, macro, uniform);
}
#endif
#if LBM3_PART(4)
void LBM3_FN(launchKineticEnergy)(const DevLevel& g, bool flip, cudaStream_t s, double* out) {
    dispatch<RunEnergy>(g, flip, s, out);
}
void LBM3_FN(launchMacro)(const DevLevel& g, bool flip, cudaStream_t s, float* out) { dispatch<RunMacro>(g, flip, s, out); }
void LBM3_FN(launchGlobalSums)(const DevLevel& g, bool flip, cudaStream_t s, double* out) {
    dispatch<RunGlobalSums>(g, flip, s, out);
}
void LBM3_FN(launchGatherF)(const DevLevel& g, cudaStream_t s, float* out) { dispatch<RunGather>(g, false, s, out); }
void LBM3_FN(launchScatterF)(const DevLevel& g, cudaStream_t s, const float* in) { dispatch<RunScatter>(g, false, s, in); }
void LBM3_FN(launchFlowImage)(const DevLevel& g, bool flip, cudaStream_t s, const FlowImagePass& a, float* img) {
    dispatch<RunFlowImage>(g, flip, s, a, img);
}
void LBM3_FN(launchFlowReport)(const DevLevel& g, bool flip, cudaStream_t s, int plane, int layer, int h0, int h1,
                               int v0, int v1, double* out) {
    dispatch<RunFlowReport>(g, flip, s, plane, layer, h0, h1, v0, v1, out);
}
#endif

#if LBM3_PART(1)
void LBM3_FN(launchPackedStep)(const DevBatch& b, bool flip, cudaStream_t s) {
    flip ? RunPackedStep<true, StepStore>::run(b, s) : RunPackedStep<false, StepStore>::run(b, s);
}
#endif

#if LBM3_SHARED_UNIT
// storage-independent launchers live in the FP32 unit of part 4
int stepLaunchCount(const DevLevel& g) {
    int n = 0;
    const CollideVariant v = collideVariant();
    if (v == CollideVariant::Simple) n += g.cellCount > 0;
    else if (v == CollideVariant::Prefetch || v == CollideVariant::Pair || v == CollideVariant::Packed)
        n += ((g.segCount + g.specialCount) > 0) + (g.rotorCellCount > 0);
    else n += (g.segCount > 0) + (g.specialCount > 0) + (g.rotorCellCount > 0);
    return n + (g.obCount > 0) + (g.perCount > 0);
}
void launchWallForce(const DevLevel& g, int wallID, cudaStream_t s, double* out) {
    if (g.wallCount > 0) wallForceSum<<<blocksFor(g.wallCount), kBlock, 0, s>>>(g, wallID, out);
}
void launchRotorForce(const DevRotor& R, const int* index, cudaStream_t s, double* out) {
    if (R.nonzero > 0) rotorForceSum<<<blocksFor(R.nonzero), kBlock, 0, s>>>(R, index, out);
}
void launchOpenFlow(const DevLevel& g, int openBCID, float invSpan, cudaStream_t s, double* out) {
    if (g.obCount > 0) openFlowSum<<<blocksFor(g.obCount), kBlock, 0, s>>>(g, openBCID, invSpan, out);
}
void launchCollideBatch(float* f, int n, const CollisionConsts& P, float gx, float gy, float gz,
                        cudaStream_t s) {
    collideBatch<<<blocksFor(n), kBlock, 0, s>>>(f, n, P, gx, gy, gz);
}
void launchFlowImageClear(float* img, long long pixels, cudaStream_t s) {
    flowImageClear<<<blocksFor(pixels), kBlock, 0, s>>>(img, pixels);
}
void launchFlowImageSum(const float* img, long long pixels, cudaStream_t s, double* out) {
    flowImageSum<<<blocksFor(pixels), kBlock, 0, s>>>(img, pixels, out);
}
#endif

}  // namespace lbm
