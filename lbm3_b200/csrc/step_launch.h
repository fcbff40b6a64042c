// Host-callable launchers of the level kernels (implemented in step.cu).
#pragma once

#include <cuda_runtime.h>

#include "../../include/lbm3_b200.h"
#include "step.cuh"

namespace lbm {

void launchCollideStream(const DevLevel& g, bool flip, cudaStream_t s);
// kernels one updateSingleGrid launches for this level
int stepLaunchCount(const DevLevel& g);
void launchPeriodic(const DevLevel& g, bool flip, cudaStream_t s);
void launchOpenBoundary(const DevLevel& g, bool flip, cudaStream_t s, int iterationsFinished);
void launchOpenBoundaryInit(const DevLevel& g, bool flip, cudaStream_t s);
void launchInit(const DevLevel& g, bool flip, cudaStream_t s, const float4* macro, float4 uniform);
void launchKineticEnergy(const DevLevel& g, bool flip, cudaStream_t s, double* out);
void launchMacro(const DevLevel& g, bool flip, cudaStream_t s, float* out);
void launchGatherF(const DevLevel& g, cudaStream_t s, float* out);
void launchScatterF(const DevLevel& g, cudaStream_t s, const float* in);
void launchWallForce(const DevLevel& g, int wallID, cudaStream_t s, double* out);
void launchFlowReport(const DevLevel& g, bool flip, cudaStream_t s, int plane, int layer, int h0, int h1, int v0,
                      int v1, double* out);
void launchRotorForce(const DevRotor& R, const int* index, cudaStream_t s, double* out);
void launchOpenFlow(const DevLevel& g, int openBCID, float invSpan, cudaStream_t s, double* out);
void launchCollideBatch(float* f, int n, const CollisionConsts& P, float gx, float gy, float gz,
                        cudaStream_t s);

}  // namespace lbm
