// Host-callable launchers of the level kernels.  step.cu is compiled once per
// population storage type (launchers suffixed F32, F16, BF16, F64);
// step_dispatch.cu selects the unit by DevLevel::storage.
#pragma once

#include <cuda_runtime.h>

#include "../../include/lbm3_b200.h"
#include "step.cuh"

namespace lbm {

// Collide-stream kernel choice (LBM3_COLLIDE_KERNEL = simple | tma | prefetch |
// packed; default: the paired persistent kernel with the level descriptor as
// a kernel parameter)
enum class CollideVariant { Tma, Prefetch, Simple, Pair, Packed };
CollideVariant collideVariant();
// The paired kernel indexes populations with 32-bit element offsets.
inline bool pairFits(const DevLevel& g) { return 27LL * g.stride + 128 < (1LL << 31); }  // 128: one tile

void launchCollideStream(const DevLevel& g, bool flip, cudaStream_t s);
// kernels one updateSingleGrid launches for this level
int stepLaunchCount(const DevLevel& g);
void launchPeriodic(const DevLevel& g, bool flip, cudaStream_t s);
// K4-K6: fine-to-coarse, coarse-to-fine and leftover interface updates
// between a level and the next finer one, after the finer level's substeps;
// the flippers are the two levels' after streaming
void launchInterface(const DevLevel& coarse, const DevLevel& fine, const DevInterface& I, bool flipCoarse,
                     bool flipFine, cudaStream_t s);
// K2; reads and advances the device iteration count (DevLevel::obCounter)
void launchOpenBoundary(const DevLevel& g, bool flip, cudaStream_t s);
void launchOpenBoundaryInit(const DevLevel& g, bool flip, cudaStream_t s);
void launchInit(const DevLevel& g, bool flip, cudaStream_t s, const float4* macro, float4 uniform);
void launchKineticEnergy(const DevLevel& g, bool flip, cudaStream_t s, double* out);
void launchMacro(const DevLevel& g, bool flip, cudaStream_t s, float* out);
// FP64 sums over the fluid cells: {rho, dRho, rho ux, rho uy, rho uz, cells}
void launchGlobalSums(const DevLevel& g, bool flip, cudaStream_t s, double* out);
void launchGatherF(const DevLevel& g, cudaStream_t s, float* out);
void launchScatterF(const DevLevel& g, cudaStream_t s, const float* in);
void launchWallForce(const DevLevel& g, int wallID, cudaStream_t s, double* out);
void launchFlowReport(const DevLevel& g, bool flip, cudaStream_t s, int plane, int layer, int h0, int h1, int v0,
                      int v1, double* out);
void launchRotorForce(const DevRotor& R, const int* index, cudaStream_t s, double* out);
void launchOpenFlow(const DevLevel& g, int openBCID, float invSpan, cudaStream_t s, double* out);
void launchCollideBatch(float* f, int n, const CollisionConsts& P, float gx, float gy, float gz,
                        cudaStream_t s);
// Section image of a flow report over several levels: clear, one pass per
// level (finer levels later), then the sums over the fluid pixels.
void launchFlowImageClear(float* img, long long pixels, cudaStream_t s);
void launchFlowImage(const DevLevel& g, bool flip, cudaStream_t s, const FlowImagePass& a, float* img);
void launchFlowImageSum(const float* img, long long pixels, cudaStream_t s, double* out);
// One step of a packed batch of single-level domains of one storage type
// (FP32, FP16 or BF16), all at esotwist flipper `flip`.
void launchPackedStep(const DevBatch& b, int storage, bool flip, cudaStream_t s);

// per-storage launchers (one set per step.cu unit)
#define LBM3_DECLARE_STORAGE_LAUNCHERS(SUF)                                                                      \
    void launchCollidePair##SUF(const DevLevel& g, bool flip, cudaStream_t s);                                 \
    void launchCollideOther##SUF(const DevLevel& g, bool flip, cudaStream_t s, CollideVariant v);              \
    void launchPeriodic##SUF(const DevLevel& g, bool flip, cudaStream_t s);                                    \
    void launchInterface##SUF(const DevLevel& coarse, const DevLevel& fine, const DevInterface& I, bool flipC,  \
                              bool flipF, cudaStream_t s);                                                     \
    void launchOpenBoundary##SUF(const DevLevel& g, bool flip, cudaStream_t s);                                \
    void launchOpenBoundaryInit##SUF(const DevLevel& g, bool flip, cudaStream_t s);                            \
    void launchInit##SUF(const DevLevel& g, bool flip, cudaStream_t s, const float4* macro, float4 uniform);   \
    void launchKineticEnergy##SUF(const DevLevel& g, bool flip, cudaStream_t s, double* out);                  \
    void launchMacro##SUF(const DevLevel& g, bool flip, cudaStream_t s, float* out);                           \
    void launchGlobalSums##SUF(const DevLevel& g, bool flip, cudaStream_t s, double* out);                     \
    void launchGatherF##SUF(const DevLevel& g, cudaStream_t s, float* out);                                    \
    void launchScatterF##SUF(const DevLevel& g, cudaStream_t s, const float* in);                              \
    void launchFlowReport##SUF(const DevLevel& g, bool flip, cudaStream_t s, int plane, int layer, int h0,     \
                               int h1, int v0, int v1, double* out);                                           \
    void launchPackedStep##SUF(const DevBatch& b, bool flip, cudaStream_t s);                                   \
    void launchFlowImage##SUF(const DevLevel& g, bool flip, cudaStream_t s, const FlowImagePass& a, float* img);
LBM3_DECLARE_STORAGE_LAUNCHERS(F32)
LBM3_DECLARE_STORAGE_LAUNCHERS(F16)
LBM3_DECLARE_STORAGE_LAUNCHERS(BF16)
LBM3_DECLARE_STORAGE_LAUNCHERS(F64)
#undef LBM3_DECLARE_STORAGE_LAUNCHERS

}  // namespace lbm
