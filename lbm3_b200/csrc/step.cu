// Time-step kernels of one grid level.
//
//   collideStream  K1: fused read -> cumulant collision -> esotwist write
//                  (updateSingleGrid cell lambda, include/updateGrid.h:51-178)
//   periodicCopy   K3: ghost <- interior pre-collision copy (:358-382)
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
#include "builder.h"
#include "step_launch.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <string>
#include <type_traits>

namespace lbm {

namespace {

constexpr int kBlock = 256;

template <bool F, class S>
__global__ void __launch_bounds__(kBlock) collideStream(DevLevel g) {
    const int cell = blockIdx.x * kBlock + threadIdx.x;
    if (cell >= g.cellCount) return;
    const int wm = __ldg(g.wallMap + cell);
    if (wm == -3) return;  // the cell itself is a wall
    int nb[8];
    decodeNbr(g, cell, nb, nullptr);
    float f[27];
    readPre<F, S>(g, nb, f);
    collideCumulant(f, g.coll, g.coll.lambda, 0.f, 0.f, 0.f);
    writePost<F, S>(g, nb, f);
}

// ---- bulk collide-stream ---------------------------------------------------
// Persistent CTAs walk the bulk segments (runs of up to kSegmentCells plain
// fluid cells inside one compressed row; one segment per CTA iteration, one
// cell per thread).  Inside a segment the 8 esotwist neighbours of lane t are
// the segment's base indices + t, so no per-cell metadata is loaded: a CTA
// reads one 20-byte descriptor per tile, two tiles ahead.  The 27 gathers of
// the next tile are issued as cp.async copies into shared memory before the
// current tile is collided, so HBM traffic overlaps the cumulant arithmetic.
// A thread reads back only the stage slots its own copies filled, hence no
// block barrier; esotwist gives every global slot a single owning cell, so
// prefetching the next tile never reads a value the current tile writes.
// 16-bit storage stages the aligned 32-bit word that holds the element.
constexpr int kTile = 128;  // == kSegmentCells
static_assert(kTile == kSegmentCells, "tile and segment length differ");

__device__ __forceinline__ void cpAsync4(void* smem, const void* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cpAsyncWaitPrev() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

__device__ __forceinline__ void segNbr(const DevLevel& g, const int4& d, int t, int (&nb)[8]) {
    const int n = g.cellCount;
    nb[0] = d.x + t;
    nb[2] = d.y + t;
    nb[4] = d.z + t;
    nb[6] = d.w + t;
    nb[1] = nb[0] + 1 < n ? nb[0] + 1 : 0;
    nb[3] = nb[2] + 1 < n ? nb[2] + 1 : 0;
    nb[5] = nb[4] + 1 < n ? nb[4] + 1 : 0;
    nb[7] = nb[6] + 1 < n ? nb[6] + 1 : 0;
}

template <class S> __device__ __forceinline__ float fromWord(unsigned w, const S* p);
template <> __device__ __forceinline__ float fromWord<float>(unsigned w, const float*) {
    return __uint_as_float(w);
}
template <> __device__ __forceinline__ float fromWord<__half>(unsigned w, const __half* p) {
    const unsigned short h = (reinterpret_cast<uintptr_t>(p) & 2) ? (w >> 16) : (w & 0xffffu);
    return __half2float(__ushort_as_half(h));
}
template <> __device__ __forceinline__ float fromWord<__nv_bfloat16>(unsigned w, const __nv_bfloat16* p) {
    const unsigned short h = (reinterpret_cast<uintptr_t>(p) & 2) ? (w >> 16) : (w & 0xffffu);
    return __bfloat162float(__ushort_as_bfloat16(h));
}

template <bool F, class S>
__device__ __forceinline__ const S* preAddr(const DevLevel& g, const int (&nb)[8], int d) {
    return static_cast<const S*>(g.f) + (long long)preSlot<F>(d) * g.stride + nb[preNbr(d)];
}

template <bool F, class S>
__device__ __forceinline__ void issueGathers(const DevLevel& g, const int (&nb)[8], unsigned* stage) {
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        const S* p = preAddr<F, S>(g, nb, d);
        const void* w = reinterpret_cast<const void*>(reinterpret_cast<uintptr_t>(p) & ~uintptr_t(3));
        cpAsync4(stage + d * kTile + threadIdx.x, w);
    }
}

// resident CTAs per SM the register allocation is sized for
#ifndef LBM3_BULK_MIN_BLOCKS
#define LBM3_BULK_MIN_BLOCKS 6
#endif

template <bool F, class S>
__global__ void __launch_bounds__(kTile, LBM3_BULK_MIN_BLOCKS) collideBulk(DevLevel g) {
    extern __shared__ unsigned stages[];  // [2][27][kTile] words
    const int T = g.segCount;
    const int G = gridDim.x;
    const int t = threadIdx.x;
    int tile = blockIdx.x;
    int4 dCur = make_int4(0, 0, 0, 0), dNext = dCur;
    int lCur = 0, lNext = 0;
    if (tile < T) {
        dCur = __ldg(g.seg + tile);
        lCur = __ldg(g.segLen + tile);
    }
    if (tile + G < T) {
        dNext = __ldg(g.seg + tile + G);
        lNext = __ldg(g.segLen + tile + G);
    }
    int nbCur[8];
    segNbr(g, dCur, t, nbCur);
    if (t < lCur) issueGathers<F, S>(g, nbCur, stages);
    cpAsyncCommit();
    int b = 0;
    for (; tile < T; tile += G) {
        // descriptor two tiles ahead: consumed by the next iteration's issue
        int4 dAfter = make_int4(0, 0, 0, 0);
        int lAfter = 0;
        if (tile + 2 * G < T) {
            dAfter = __ldg(g.seg + tile + 2 * G);
            lAfter = __ldg(g.segLen + tile + 2 * G);
        }
        int nbNext[8];
        segNbr(g, dNext, t, nbNext);
        if (t < lNext) issueGathers<F, S>(g, nbNext, stages + (b ^ 1) * 27 * kTile);
        cpAsyncCommit();
        cpAsyncWaitPrev();  // this thread's copies for the current tile have landed
        if (t < lCur) {
            float f[27];
#pragma unroll
            for (int d = 0; d < 27; ++d)
                f[d] = fromWord<S>(stages[(b * 27 + d) * kTile + t], preAddr<F, S>(g, nbCur, d));
            collideCumulant(f, g.coll, g.coll.lambda, 0.f, 0.f, 0.f);
            writePost<F, S>(g, nbCur, f);
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) nbCur[q] = nbNext[q];
        lCur = lNext;
        dNext = dAfter;
        lNext = lAfter;
        b ^= 1;
    }
}

// Cells outside the bulk segments (wall-adjacent), one thread per listed cell.
template <bool F, class S>
__global__ void __launch_bounds__(kBlock) collideList(DevLevel g) {
    const int idx = blockIdx.x * kBlock + threadIdx.x;
    if (idx >= g.specialCount) return;
    const int cell = __ldg(g.special + idx);
    int nb[8];
    decodeNbr(g, cell, nb, nullptr);
    float f[27];
    readPre<F, S>(g, nb, f);
    collideCumulant(f, g.coll, g.coll.lambda, 0.f, 0.f, 0.f);
    writePost<F, S>(g, nb, f);
}

// F is the flipper after streaming, i.e. the state the ghosts are read in.
template <bool F, class S>
__global__ void __launch_bounds__(kBlock) periodicCopy(DevLevel g) {
    const int idx = blockIdx.x * kBlock + threadIdx.x;
    if (idx >= g.perCount) return;
    const int cell = __ldg(g.perIndex + idx);
    const int src = __ldg(g.perSource + idx);
    int nb[8];
    float f[27];
    decodeNbr(g, src, nb, nullptr);
    readPre<F, S>(g, nb, f);
    decodeNbr(g, cell, nb, nullptr);
    writePre<F, S>(g, nb, f);
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

template <bool F, class S>
__global__ void __launch_bounds__(kBlock) initFeq(DevLevel g, const float4* macro, float4 uniform) {
    const int cell = blockIdx.x * kBlock + threadIdx.x;
    if (cell >= g.cellCount) return;
    const float4 m = macro ? macro[cell] : uniform;
    int nb[8];
    decodeNbr(g, cell, nb, nullptr);
    float f[27];
    feqExact(m.x, m.y, m.z, m.w, f);
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
        if (wm != -3 && wm != -2) {
            int nb[8];
            decodeNbr(g, cell, nb, nullptr);
            float f[27];
            readPre<F, S>(g, nb, f);
            float dRho, ux, uy, uz;
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

template <bool F, class S>
__global__ void __launch_bounds__(kBlock) macroFields(DevLevel g, float* out) {
    const int cell = blockIdx.x * kBlock + threadIdx.x;
    if (cell >= g.cellCount) return;
    int nb[8];
    decodeNbr(g, cell, nb, nullptr);
    float f[27];
    readPre<F, S>(g, nb, f);
    float dRho, ux, uy, uz;
    macroFromF(f, dRho, ux, uy, uz);
    const long long n = g.cellCount;
    out[cell] = dRho;
    out[n + cell] = ux;
    out[2 * n + cell] = uy;
    out[3 * n + cell] = uz;
}

template <bool F, class S>
__global__ void __launch_bounds__(kBlock) gatherF(DevLevel g, float* out) {
    // raw slot copy: out[slot][cell] = f[slot][cell] as FP32
    const long long i = (long long)blockIdx.x * kBlock + threadIdx.x;
    const long long total = 27LL * g.stride;
    if (i >= total) return;
    out[i] = Store<S>::ld(static_cast<const S*>(g.f) + i);
}

template <class S>
__global__ void __launch_bounds__(kBlock) scatterF(DevLevel g, const float* in) {
    const long long i = (long long)blockIdx.x * kBlock + threadIdx.x;
    const long long total = 27LL * g.stride;
    if (i >= total) return;
    Store<S>::st(static_cast<S*>(g.f) + i, in[i]);
}

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

inline unsigned blocksFor(long long n) { return static_cast<unsigned>((n + kBlock - 1) / kBlock); }

// Dispatch on (flipper, storage type).
template <template <bool, class> class K, class... A>
void dispatch(const DevLevel& g, bool flip, A&&... args) {
    switch (g.storage) {
        case LBM_STORE_F16:
            flip ? K<true, __half>::run(g, args...) : K<false, __half>::run(g, args...);
            break;
        case LBM_STORE_BF16:
            flip ? K<true, __nv_bfloat16>::run(g, args...) : K<false, __nv_bfloat16>::run(g, args...);
            break;
        default:
            flip ? K<true, float>::run(g, args...) : K<false, float>::run(g, args...);
    }
}

constexpr int kStageBytes = 2 * 27 * kTile * 4;

template <class S> int bulkGrid() {
    static int grid = 0;
    if (grid == 0) {
        int dev = 0, sms = 0, perSm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaFuncSetAttribute(collideBulk<false, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, kStageBytes);
        cudaFuncSetAttribute(collideBulk<true, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, kStageBytes);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, collideBulk<false, S>, kTile, kStageBytes);
        grid = sms * (perSm > 0 ? perSm : 1);
    }
    return grid;
}

bool useBulk() {
    static int v = -1;
    if (v < 0) {
        const char* e = std::getenv("LBM3_COLLIDE_KERNEL");
        v = (e && std::string(e) == "simple") ? 0 : 1;
    }
    return v == 1;
}

template <bool F, class S> struct RunCollide {
    static void run(const DevLevel& g, cudaStream_t s) {
        if (useBulk()) {
            if (g.segCount > 0) {
                const int grid = std::min(bulkGrid<S>(), g.segCount);
                collideBulk<F, S><<<grid, kTile, kStageBytes, s>>>(g);
            }
            if (g.specialCount > 0) collideList<F, S><<<blocksFor(g.specialCount), kBlock, 0, s>>>(g);
        } else {
            collideStream<F, S><<<blocksFor(g.cellCount), kBlock, 0, s>>>(g);
        }
    }
};

template <bool F, class S> struct RunPeriodic {
    static void run(const DevLevel& g, cudaStream_t s) {
        if (g.perCount > 0) periodicCopy<F, S><<<blocksFor(g.perCount), kBlock, 0, s>>>(g);
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
template <bool F, class S> struct RunMacro {
    static void run(const DevLevel& g, cudaStream_t s, float* out) {
        macroFields<F, S><<<blocksFor(g.cellCount), kBlock, 0, s>>>(g, out);
    }
};
template <bool F, class S> struct RunGather {
    static void run(const DevLevel& g, cudaStream_t s, float* out) {
        gatherF<F, S><<<blocksFor(27LL * g.stride), kBlock, 0, s>>>(g, out);
    }
};
template <bool F, class S> struct RunScatter {
    static void run(const DevLevel& g, cudaStream_t s, const float* in) {
        scatterF<S><<<blocksFor(27LL * g.stride), kBlock, 0, s>>>(g, in);
    }
};

}  // namespace

void launchCollideStream(const DevLevel& g, bool flip, cudaStream_t s) { dispatch<RunCollide>(g, flip, s); }
void launchPeriodic(const DevLevel& g, bool flip, cudaStream_t s) { dispatch<RunPeriodic>(g, flip, s); }
void launchInit(const DevLevel& g, bool flip, cudaStream_t s, const float4* macro, float4 uniform) {
    dispatch<RunInit>(g, flip, s, macro, uniform);
}
void launchKineticEnergy(const DevLevel& g, bool flip, cudaStream_t s, double* out) {
    dispatch<RunEnergy>(g, flip, s, out);
}
void launchMacro(const DevLevel& g, bool flip, cudaStream_t s, float* out) { dispatch<RunMacro>(g, flip, s, out); }
void launchGatherF(const DevLevel& g, cudaStream_t s, float* out) { dispatch<RunGather>(g, false, s, out); }
void launchScatterF(const DevLevel& g, cudaStream_t s, const float* in) { dispatch<RunScatter>(g, false, s, in); }
void launchCollideBatch(float* f, int n, const CollisionConsts& P, float gx, float gy, float gz,
                        cudaStream_t s) {
    collideBatch<<<blocksFor(n), kBlock, 0, s>>>(f, n, P, gx, gy, gz);
}

}  // namespace lbm
