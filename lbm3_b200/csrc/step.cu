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

// ---- pipelined collide-stream (FP32 storage) --------------------------------
// Persistent CTAs walk tiles of kPipeBlock consecutive cells.  While a tile is
// collided from registers, the 27 gathers of the thread's next cell are already
// in flight as cp.async copies into shared memory (two stages).  Each thread
// reads back only the stage slots its own copies filled, so no block-level
// barrier is needed; in-place esotwist streaming keeps every global slot owned
// by exactly one cell, so the prefetch never reads a value this step writes.
constexpr int kPipeBlock = 128;

__device__ __forceinline__ void cpAsync4(float* smem, const float* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cpAsyncWaitPrev() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// Decode the tile's cell for this thread and start its 27 gathers into stage `buf`.
template <bool F>
__device__ __forceinline__ bool issueTile(const DevLevel& g, int tile, float* stage, int (&nb)[8]) {
    const int cell = tile * kPipeBlock + threadIdx.x;
    if (cell >= g.cellCount) return false;
    if (__ldg(g.wallMap + cell) == -3) return false;
    decodeNbr(g, cell, nb, nullptr);
    const float* base = static_cast<const float*>(g.f);
#pragma unroll
    for (int d = 0; d < 27; ++d)
        cpAsync4(stage + d * kPipeBlock + threadIdx.x,
                 base + (long long)preSlot<F>(d) * g.stride + nb[preNbr(d)]);
    return true;
}

template <bool F>
__global__ void __launch_bounds__(kPipeBlock) collideStreamPipelined(DevLevel g, int tiles) {
    extern __shared__ float stages[];  // [2][27][kPipeBlock]
    float* stage[2] = {stages, stages + 27 * kPipeBlock};
    int tile = blockIdx.x;
    int nbCur[8];
    bool cur = tile < tiles && issueTile<F>(g, tile, stage[0], nbCur);
    cpAsyncCommit();
    int b = 0;
    for (; tile < tiles; tile += gridDim.x) {
        const int next = tile + gridDim.x;
        int nbNext[8];
        const bool nxt = next < tiles && issueTile<F>(g, next, stage[b ^ 1], nbNext);
        cpAsyncCommit();
        cpAsyncWaitPrev();  // this thread's copies of the current tile have landed
        if (cur) {
            float f[27];
#pragma unroll
            for (int d = 0; d < 27; ++d) f[d] = stage[b][d * kPipeBlock + threadIdx.x];
            collideCumulant(f, g.coll, g.coll.lambda, 0.f, 0.f, 0.f);
            writePost<F, float>(g, nbCur, f);
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) nbCur[q] = nbNext[q];
        cur = nxt;
        b ^= 1;
    }
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

int pipelineGrid() {
    static int grid = 0;
    if (grid == 0) {
        int dev = 0, sms = 0, perSm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const int smem = 2 * 27 * kPipeBlock * sizeof(float);
        cudaFuncSetAttribute(collideStreamPipelined<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        cudaFuncSetAttribute(collideStreamPipelined<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, collideStreamPipelined<false>, kPipeBlock, smem);
        grid = sms * (perSm > 0 ? perSm : 1);
    }
    return grid;
}

bool usePipelined() {
    static int v = -1;
    if (v < 0) {
        const char* e = std::getenv("LBM3_COLLIDE_KERNEL");
        v = (e && std::string(e) == "simple") ? 0 : 1;
    }
    return v == 1;
}

template <bool F, class S> struct RunCollide {
    static void run(const DevLevel& g, cudaStream_t s) {
        if (std::is_same<S, float>::value && usePipelined()) {
            const int tiles = (g.cellCount + kPipeBlock - 1) / kPipeBlock;
            const int grid = std::min(pipelineGrid(), tiles);
            collideStreamPipelined<F><<<grid, kPipeBlock, 2 * 27 * kPipeBlock * sizeof(float), s>>>(g, tiles);
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
