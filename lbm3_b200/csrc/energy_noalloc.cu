// Kinetic-energy reduction with its scratch in a static device array.
//
// Some callers cannot allocate device memory while a simulation runs: a
// serving loop that admits domains by HBM footprint has committed every byte
// to resident populations, so any allocation on the side (cudaMalloc,
// cudaFree, a framework's caching allocator) may fail, and cudaFree also
// synchronizes the device in the middle of the step pipeline.  This path
// needs no allocation by anyone: the per-block partial sums and the total
// live in `gEnergyScratch`, a file-scope array of fixed size that the CUDA
// runtime places when the module loads and keeps until the process exits.
//
// Host code must not hand `gEnergyScratch` itself to a kernel: on the host the
// name is only a stand-in, not a device address.  The first call on a device
// (with that device current) looks up the array's device address with
// cudaGetSymbolAddress and caches it per device; make that first call before
// any stream capture begins.
//
// Every call on a device shares the one array, which keeps the last call's
// contents.  Nothing in it has to start at zero: pass 1 overwrites one
// partial per block and pass 2 overwrites the total.  Calls that overlap on
// the GPU (issued on different streams, or from different threads, without
// ordering between them) race on the array and may return each other's sums;
// serialize them.
#include "energy_noalloc.h"

#include <mutex>

namespace lbm {

namespace {

constexpr int kTotalSlot = kNoAllocEnergyMaxBlocks;  // index of the total
constexpr int kMaxDevices = 64;

// [0, kNoAllocEnergyMaxBlocks): partial sum of each pass-1 block;
// [kTotalSlot]: the level total.  128 KB + 256 B on every device.
static __device__ __align__(256) double gEnergyScratch[kNoAllocEnergyMaxBlocks + 32];

std::mutex gScratchMutex;
double* gScratchPtr[kMaxDevices] = {};

// Device address of gEnergyScratch on the current device (set-up on the first
// call per device).  The address is cached for the life of the process: a
// cudaDeviceReset destroys the context that owns it, so a process that resets
// a device must not call lbm_kinetic_energy_noalloc on that device afterwards.
cudaError_t scratchPointer(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(gScratchMutex);
    if (!gScratchPtr[dev]) {
        double* p = nullptr;
        e = cudaGetSymbolAddress((void**)&p, gEnergyScratch);
        if (e != cudaSuccess) return e;
        gScratchPtr[dev] = p;
    }
    *out = gScratchPtr[dev];
    return cudaSuccess;
}

__device__ __forceinline__ double warpSum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Block sum of v in a fixed order (lane tree, then warps in order); the
// result is valid in thread 0.
__device__ __forceinline__ double blockSum(double v, double* part) {
    v = warpSum(v);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x < 32) {
        r = threadIdx.x < blockDim.x / 32 ? part[threadIdx.x] : 0.0;
        r = warpSum(r);
    }
    return r;
}

// Pass 1: one partial per block of kNoAllocEnergyBlock cells.  Cell selection
// and the per-cell term are those of the Taylor–Green driver's energy
// (cases/taylorGreenVortex/taylorGreenVortexMain.cu:116-180).
template <bool F, class S>
__global__ void __launch_bounds__(kNoAllocEnergyBlock) energyPartials(DevLevel g, double* partial) {
    __shared__ double part[kNoAllocEnergyBlock / 32];
    const int cell = blockIdx.x * kNoAllocEnergyBlock + threadIdx.x;
    double e = 0.0;
    if (cell < g.cellCount) {
        const int wm = __ldg(g.wallMap + cell);
        const bool overlap = wm >= 0 && (__ldg(g.wallData + wm) & 1u);
        if (wm != -3 && wm != -2 && !overlap) {
            int nb[8];
            decodeNbr(g, cell, nb, nullptr);
            Real<S> f[27];
            readPre<F, S>(g, nb, f);
            Real<S> dRho, ux, uy, uz;
            macroFromF(f, dRho, ux, uy, uz);
            e = 0.5 * (1.0 + double(dRho)) * (double(ux) * ux + double(uy) * uy + double(uz) * uz);
        }
    }
    const double b = blockSum(e, part);
    if (threadIdx.x == 0) partial[blockIdx.x] = b;
}

// Pass 2: one block adds the partials, each thread a fixed strided subset.
constexpr int kTotalBlock = 1024;
__global__ void __launch_bounds__(kTotalBlock) energyTotal(const double* partial, int count, double* total) {
    __shared__ double part[kTotalBlock / 32];
    double v = 0.0;
    for (int q = threadIdx.x; q < count; q += kTotalBlock) v += partial[q];
    const double b = blockSum(v, part);
    if (threadIdx.x == 0) *total = b;
}

template <bool F, class S> void launchPartials(const DevLevel& g, cudaStream_t s, int blocks, double* scratch) {
    energyPartials<F, S><<<blocks, kNoAllocEnergyBlock, 0, s>>>(g, scratch);
}

}  // namespace

cudaError_t kineticEnergyNoAlloc(const DevLevel& g, bool flip, cudaStream_t s, double* sum) {
    if (g.cellCount > kNoAllocEnergyMaxCells) return cudaErrorInvalidValue;
    double* scratch = nullptr;
    cudaError_t e = scratchPointer(&scratch);
    if (e != cudaSuccess) return e;
    *sum = 0.0;
    if (g.cellCount <= 0) return cudaSuccess;
    const int blocks = static_cast<int>((g.cellCount + kNoAllocEnergyBlock - 1) / kNoAllocEnergyBlock);
    switch (g.storage) {
        case LBM_STORE_F16:
            flip ? launchPartials<true, __half>(g, s, blocks, scratch)
                 : launchPartials<false, __half>(g, s, blocks, scratch);
            break;
        case LBM_STORE_BF16:
            flip ? launchPartials<true, __nv_bfloat16>(g, s, blocks, scratch)
                 : launchPartials<false, __nv_bfloat16>(g, s, blocks, scratch);
            break;
        case LBM_STORE_F64:
            flip ? launchPartials<true, double>(g, s, blocks, scratch)
                 : launchPartials<false, double>(g, s, blocks, scratch);
            break;
        default:
            flip ? launchPartials<true, float>(g, s, blocks, scratch)
                 : launchPartials<false, float>(g, s, blocks, scratch);
    }
    energyTotal<<<1, kTotalBlock, 0, s>>>(scratch, blocks, scratch + kTotalSlot);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(sum, scratch + kTotalSlot, sizeof(double), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        return e;
    return cudaStreamSynchronize(s);
}

}  // namespace lbm
