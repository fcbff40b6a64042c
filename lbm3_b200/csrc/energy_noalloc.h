// Kinetic-energy reduction that allocates no device memory (host side).
#pragma once

#include <cuda_runtime.h>

#include "../../include/lbm3_b200.h"
#include "step.cuh"

namespace lbm {

// Cells per reduction block and the number of per-block partial sums the
// static scratch array holds; a level with more cells than their product is
// rejected by the caller.
constexpr int kNoAllocEnergyBlock = 256;
constexpr int kNoAllocEnergyMaxBlocks = 16384;
constexpr long long kNoAllocEnergyMaxCells = 1LL * kNoAllocEnergyBlock * kNoAllocEnergyMaxBlocks;

// Σ 0.5 (1 + dRho) |u|^2 over the level's fluid cells (the same cells and
// terms as the allocating path), summed in FP64 in a fixed order, written to
// *sum after a stream synchronize.  g.cellCount must not exceed
// kNoAllocEnergyMaxCells.  Returns the first CUDA error, if any.
cudaError_t kineticEnergyNoAlloc(const DevLevel& g, bool flip, cudaStream_t s, double* sum);

}  // namespace lbm
