// Storage dispatch of the level launchers: step.cu is compiled once per
// population storage type, and these entry points forward to its unit.
#include "step_launch.h"

#include <cstdlib>
#include <string>

namespace lbm {

#define LBM3_BY_STORAGE(name, ...)                                          \
    switch (g.storage) {                                                    \
        case LBM_STORE_F16: name##F16(__VA_ARGS__); break;                  \
        case LBM_STORE_BF16: name##BF16(__VA_ARGS__); break;                \
        case LBM_STORE_F64: name##F64(__VA_ARGS__); break;                  \
        default: name##F32(__VA_ARGS__);                                    \
    }

CollideVariant collideVariant() {
    static const CollideVariant v = [] {
        const char* e = std::getenv("LBM3_COLLIDE_KERNEL");
        const std::string s = e ? e : "";
        return s == "simple" ? CollideVariant::Simple
               : s == "tma"  ? CollideVariant::Tma
               : s == "prefetch" ? CollideVariant::Prefetch
               : s == "packed" ? CollideVariant::Packed
                                 : CollideVariant::Pair;
    }();
    return v;
}

// The paired kernel packs two FP32 cells per thread; the FP64 build collides
// one cell per thread in the prefetching kernel.
void launchCollideStream(const DevLevel& g, bool flip, cudaStream_t s) {
    const CollideVariant v = collideVariant();
    const bool paired = v == CollideVariant::Pair || v == CollideVariant::Packed;
    if (v == CollideVariant::Packed && pairFits(g) && g.storage != LBM_STORE_F64 && g.self) {
        LBM3_BY_STORAGE(launchCollidePair, g, flip, s)
    } else {
        LBM3_BY_STORAGE(launchCollideOther, g, flip, s,
                        paired && (!pairFits(g) || g.storage == LBM_STORE_F64) ? CollideVariant::Prefetch : v)
    }
}
void launchPeriodic(const DevLevel& g, bool flip, cudaStream_t s) { LBM3_BY_STORAGE(launchPeriodic, g, flip, s) }
void launchInterface(const DevLevel& coarse, const DevLevel& fine, const DevInterface& I, bool flipCoarse,
                     bool flipFine, cudaStream_t s) {
    const DevLevel& g = coarse;
    LBM3_BY_STORAGE(launchInterface, coarse, fine, I, flipCoarse, flipFine, s)
}
void launchOpenBoundary(const DevLevel& g, bool flip, cudaStream_t s) {
    LBM3_BY_STORAGE(launchOpenBoundary, g, flip, s)
}
void launchOpenBoundaryInit(const DevLevel& g, bool flip, cudaStream_t s) {
    LBM3_BY_STORAGE(launchOpenBoundaryInit, g, flip, s)
}
void launchInit(const DevLevel& g, bool flip, cudaStream_t s, const float4* macro, float4 uniform) {
    LBM3_BY_STORAGE(launchInit, g, flip, s, macro, uniform)
}
void launchKineticEnergy(const DevLevel& g, bool flip, cudaStream_t s, double* out) {
    LBM3_BY_STORAGE(launchKineticEnergy, g, flip, s, out)
}
void launchMacro(const DevLevel& g, bool flip, cudaStream_t s, float* out) { LBM3_BY_STORAGE(launchMacro, g, flip, s, out) }
void launchGlobalSums(const DevLevel& g, bool flip, cudaStream_t s, double* out) {
    LBM3_BY_STORAGE(launchGlobalSums, g, flip, s, out)
}
void launchGatherF(const DevLevel& g, cudaStream_t s, float* out) { LBM3_BY_STORAGE(launchGatherF, g, s, out) }
void launchScatterF(const DevLevel& g, cudaStream_t s, const float* in) { LBM3_BY_STORAGE(launchScatterF, g, s, in) }
void launchFlowReport(const DevLevel& g, bool flip, cudaStream_t s, int plane, int layer, int h0, int h1, int v0,
                      int v1, double* out) {
    LBM3_BY_STORAGE(launchFlowReport, g, flip, s, plane, layer, h0, h1, v0, v1, out)
}

void launchFlowImage(const DevLevel& g, bool flip, cudaStream_t s, const FlowImagePass& a, float* img) {
    LBM3_BY_STORAGE(launchFlowImage, g, flip, s, a, img)
}

void launchPackedStep(const DevBatch& b, int storage, bool flip, cudaStream_t s) {
    switch (storage) {
        case LBM_STORE_F16: launchPackedStepF16(b, flip, s); break;
        case LBM_STORE_BF16: launchPackedStepBF16(b, flip, s); break;
        case LBM_STORE_F32: launchPackedStepF32(b, flip, s); break;
        default: break;  // FP64 domains are not packed
    }
}

#undef LBM3_BY_STORAGE

}  // namespace lbm
