// Device-side data of one grid level and the small helpers every kernel
// shares: neighbour decode from the compressed rows, typed population access
// and the esotwist slot maps.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cstdint>

#include "cumulant.cuh"
#include "lattice.h"

namespace lbm {

// open-boundary cells per CTA of the boundary kernel
constexpr int kOpenChunk = 128;


// One forcing rotor as the collide kernels see it (RotorViewStruct,
// include/types.h:217-219), with this step's angle as cosine and sine.
struct DevRotor {
    const int* rotorMap;           // [blocks] compact block index or -1
    const unsigned* interp;        // [64 * nonzero] packed corner counts
    float* force;                  // [3][27 * nonzero] force bins, rotor frame
    int nonzero;
    int cntX, cntY, cntZ, axis;
    float res, xMin, yMin, zMin, xMax, yMax, zMax;
    float ox, oy, oz;
    float c, s;                    // cos, sin of radiansElapsed (float angle)
    float scale;                   // radiansPerSecond * dtPhys / res of the level
};
constexpr int kMaxRotors = 4;

// Everything a kernel needs for one level, passed by value.
struct DevLevel {
    void* f;                 // populations [27][stride], element type per storage
    long long stride;        // == cellCount
    int cellCount;
    int storage;             // LBM_STORE_*
    const int* shifter;      // [cellCount]
    const int* rowI;
    const int* rowJ;
    const int* rowK;
    const int* rowJP;
    const int* rowKP;
    const int* rowJKP;       // [rowCount]
    const int* wallMap;      // [cellCount]
    const int* perIndex;     // [perCount]
    const int* perSource;
    int perCount;
    // bulk segments: {first cell, its jPlus, kPlus, jkPlus} and length
    const int4* seg;
    const int* segLen;
    int segCount;
    // cells collided outside the bulk segments (wall-adjacent)
    const int* special;
    int specialCount;
    int* errorFlag;          // set to nonzero when a bounded device wait gives up
    int* work;               // [2] work-item counter and finished-CTA count of the
                             // persistent collide-stream (zero between launches)
    const DevLevel* self;    // device copy of this descriptor (the one-domain
                             // launch of the packed collide-stream reads it)
    unsigned* seed;          // [2] step seeds of the stochastic rounding of 16-bit
                             // storage, by esotwist parity (null for FP32 / FP64)
    // wall-adjacent cells (WallStruct)
    const unsigned* wallData;      // [wallCount]
    const unsigned* linkLength;    // [7][wallCount] packed 8-bit link codes
    const float* wallVel;          // [3][wallCount] wall velocity, lattice units
    double* wallForce;             // [3][wallCount] momentum-exchange force accumulators (FP64)
    const int* wallIndex;          // [wallCount] cell of each entry
    int wallCount;
    int trackWallForce;
    int useIBB;
    float gx, gy, gz;              // body force (getLocalBC)
    // open-boundary cells (OpenBCArrayStruct, all IDs), in kernel order
    const int* obCell;
    const int4* obNbr;             // {cell, jPlus, kPlus, jkPlus} row neighbours
    const int* obInfo;             // packed, see OpenBCCell
    const float4* obTarget;        // dRho, ux, uy, uz of getOpenBC
    const float* obBeta;
    float* obRhoRef;               // dRhoRefArray
    float* obUnRef;                // uNormalRefArray
    float* obRhoCum;               // dRhoCumulativeArray
    float* obUnCum;                // uNormalCumulativeArray
    int obCount;
    int trackOpen;
    int obImpedance;               // LBM_OPEN_IMPEDANCE scheme for non-reflective cells
    float obTolerance;             // its RHO_REFLECTION_TOLERANCE
    // cells are grouped by outer normal; each chunk {first, count, normal row,
    // unknown-direction mask} is one CTA of the boundary kernel
    const int4* obChunk;
    int* obCounter;                   // [2] iterations finished, CTAs done in the running launch
    int obChunkCount;
    const void* obTables;             // [26] direction-indexed closure tables (MbbcDirT of the
                                      // arithmetic type)
    int nx, ny, nz;
    float res, ox, oy, oz;
    CollisionConsts coll;
    CollisionConstsT<double> coll64;  // the same constants for the FP64 build
    DevRotor rotor[kMaxRotors];
    int rotorCount;
    const int* rotorCells;         // cells inside a rotor's swept cylinder
    int rotorCellCount;
    int trackRotorForce;
};

// A packed batch of single-level domains advanced together (one launch per
// kernel kind for all of them): the domains' level descriptors on the device
// and the packed tables of work items.
struct DevBatch {
    const DevLevel* levels;    // [domainCount] device copies
    int domainCount;
    const int* itemStart;      // [domainCount + 1] prefix sums of the domains' collide-stream
                               // items (listed-cell chunks first, then bulk tiles); null:
                               // one domain with collideCount items
    int collideCount;
    int* work;                 // [domainCount + 1] per-domain item counters, then the
                               // finished-CTA count (zero between launches)
    const int2* openItems;     // {domain, chunk} of the open-boundary kernel
    int openCount;
    const int* periodicStart;  // [domainCount + 1] prefix sums of the ghost counts
    int periodicCount;
};

// One level's pass over the section image of a flow report
// (getFlowReportGeneral, include/flowReportFunctions.h:96-262): the cells of
// layer `lowerNormal` (blended with the next layer by `alpha` when
// `interpolate`), sampled every `downsample` cells in plane and written over
// upsample x upsample pixels of the image of pixelsH x pixelsV starting at
// (startH, startV) in image-level cell units.
struct FlowImagePass {
    int plane, lowerNormal, interpolate;
    float alpha;
    int downsample, upsample, startH, startV, pixelsH, pixelsV;
};

// Interface lists between a coarse level and the next finer one
// (InterfaceStruct, include/types.h:198-200) and the two levels' omega1.
struct DevInterface {
    const int* f2cIndex;     // [f2cCount] coarse cell
    const int* f2cChild;     // [f2cCount] its fine child (2i, 2j, 2k)
    int f2cCount;
    const int* c2fIndex;     // [c2fCount] -x-y-z coarse corner of a full stencil
    const int* c2fChild;     // [c2fCount] fine cell (2i+1, 2j+1, 2k+1)
    int c2fCount;
    const int* leftIndex;    // [leftCount] fine cell
    const int* leftParent;   // [leftCount] its coarse parent
    const int* leftNbr;      // [3][leftCount] coarse neighbour per axis (-cell-1: opposite side)
    int leftCount;
    double omegaCoarse, omegaFine;  // 1 / (3 nu + 1/2) of each level
};

// Collision constants in the arithmetic type T.
template <class T> __device__ __forceinline__ const CollisionConstsT<T>& collConsts(const DevLevel& g);
template <> __device__ __forceinline__ const CollisionConstsT<float>& collConsts<float>(const DevLevel& g) {
    return g.coll;
}
template <> __device__ __forceinline__ const CollisionConstsT<double>& collConsts<double>(const DevLevel& g) {
    return g.coll64;
}

// Neighbour cells of `cell` in the order self, +i, +j, +ij, +k, +ik, +jk, +ijk
// (bit 0 = i, bit 1 = j, bit 2 = k), from the compressed rows
// (getCompressedIJKNBR, include/cellFunctions.h:21-49; finishNBRPlus,
// include/NBRFunctions.h:5-11: +i neighbours are index + 1 with wrap).
__device__ __forceinline__ void decodeNbr(const DevLevel& g, int cell, int (&nb)[8], int* ijk) {
    const int shift = __ldg(g.shifter + cell);
    int row, off;
    if (shift >= 0) {
        row = shift;
        off = 0;
    } else {
        row = __ldg(g.shifter + cell + shift);
        off = -shift;
    }
    const int jP = __ldg(g.rowJP + row) + off;
    const int kP = __ldg(g.rowKP + row) + off;
    const int jkP = __ldg(g.rowJKP + row) + off;
    const int n = g.cellCount;
    nb[0] = cell;
    nb[1] = cell + 1 < n ? cell + 1 : 0;
    nb[2] = jP;
    nb[3] = jP + 1 < n ? jP + 1 : 0;
    nb[4] = kP;
    nb[5] = kP + 1 < n ? kP + 1 : 0;
    nb[6] = jkP;
    nb[7] = jkP + 1 < n ? jkP + 1 : 0;
    if (ijk) {
        ijk[0] = __ldg(g.rowI + row) + off;
        ijk[1] = __ldg(g.rowJ + row);
        ijk[2] = __ldg(g.rowK + row);
    }
}

// Typed population storage.  Half and bfloat16 hold the shifted value
// f_i - w_i directly (the reference already stores shifted FP32).  ldL2
// reads through L2 only (no L1 line allocation): scattered single-value
// gathers then move one 32-byte sector instead of a whole 128-byte line.  Arithmetic
// is FP32 for every storage type except double, which is the FP64 build of
// the kernels (FP64 storage and arithmetic).
template <class S> struct Compute { using type = float; };
template <> struct Compute<double> { using type = double; };
template <class S> using Real = typename Compute<S>::type;

template <class S> struct Store;
template <> struct Store<double> {
    static __device__ __forceinline__ double ld(const double* p) { return *p; }
    static __device__ __forceinline__ double ldL2(const double* p) { return __ldcg(p); }
    static __device__ __forceinline__ void st(double* p, double v) { *p = v; }
};
template <> struct Store<float> {
    static __device__ __forceinline__ float ld(const float* p) { return *p; }
    static __device__ __forceinline__ float ldL2(const float* p) { return __ldcg(p); }
    static __device__ __forceinline__ void st(float* p, float v) { *p = v; }
};
// stR / st2R round stochastically with the random bits r: cvt.rs adds random
// bits below the kept mantissa and truncates, so a value rounds up with
// probability equal to its distance from the lower neighbour in units of the
// spacing.  st2R converts two values with one instruction (a to *pa, b to *pb).
template <> struct Store<__half> {
    static __device__ __forceinline__ float ld(const __half* p) { return __half2float(*p); }
    static __device__ __forceinline__ float ldL2(const __half* p) { return __half2float(__ldcg(p)); }
    static __device__ __forceinline__ void st(__half* p, float v) { *p = __float2half_rn(v); }
    static __device__ __forceinline__ void stR(__half* p, float v, unsigned r) {
        unsigned d;
        asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(0.f), "f"(v), "r"(r));
        *reinterpret_cast<unsigned short*>(p) = static_cast<unsigned short>(d & 0xFFFFu);
    }
    static __device__ __forceinline__ void st2R(__half* pa, __half* pb, float a, float b, unsigned r, bool okA,
                                                bool okB) {
        unsigned d;
        asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(b), "f"(a), "r"(r));
        if (okA) *reinterpret_cast<unsigned short*>(pa) = static_cast<unsigned short>(d & 0xFFFFu);
        if (okB) *reinterpret_cast<unsigned short*>(pb) = static_cast<unsigned short>(d >> 16);
    }
};
template <> struct Store<__nv_bfloat16> {
    static __device__ __forceinline__ float ld(const __nv_bfloat16* p) { return __bfloat162float(*p); }
    static __device__ __forceinline__ float ldL2(const __nv_bfloat16* p) { return __bfloat162float(__ldcg(p)); }
    static __device__ __forceinline__ void st(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }
    static __device__ __forceinline__ void stR(__nv_bfloat16* p, float v, unsigned r) {
        unsigned d;
        asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(0.f), "f"(v), "r"(r));
        *reinterpret_cast<unsigned short*>(p) = static_cast<unsigned short>(d & 0xFFFFu);
    }
    static __device__ __forceinline__ void st2R(__nv_bfloat16* pa, __nv_bfloat16* pb, float a, float b, unsigned r,
                                                bool okA, bool okB) {
        unsigned d;
        asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(b), "f"(a), "r"(r));
        if (okA) *reinterpret_cast<unsigned short*>(pa) = static_cast<unsigned short>(d & 0xFFFFu);
        if (okB) *reinterpret_cast<unsigned short*>(pb) = static_cast<unsigned short>(d >> 16);
    }
};

// Stochastic rounding of 16-bit storage.  With round-to-nearest, a steady
// state rounds every population the same way step after step, and that fixed
// error is a constant forcing that the slowly relaxing hydrodynamic modes add
// up; with random rounding the error has zero mean and averages out.  The bits
// are a counter-based hash of (step seed, kernel salt, cell, direction) with
// the lowbias32 finaliser (C. Wellons, "Prospecting for hash functions",
// 2018), so results are deterministic: a replayed graph, a domain stepped
// alone or inside a batch draw the same bits.  Kernels of esotwist parity F
// read seed[F]; every collide-stream launch of the step writes the next value
// into seed[!F], which no kernel of that step reads.
__device__ __forceinline__ unsigned mix32(unsigned x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

struct Dither {
    unsigned seed;
    // bits of one cell; dir() then gives one 32-bit draw per direction
    __device__ __forceinline__ unsigned cell(int c) const { return seed ^ (static_cast<unsigned>(c) * 0x9E3779B1u); }
    static __device__ __forceinline__ unsigned dir(unsigned cellBits, int q) {
        return mix32(cellBits + static_cast<unsigned>(q) * 0x632BE5ABu);
    }
};

enum : unsigned { kSaltCollide = 0u, kSaltOpen = 0x51ED270Bu, kSaltInterface = 0xA3C59AC3u };

// The rounding is fixed per storage type at compile time: a run-time choice
// between the two roundings in every store multiplies the code the
// assembler has to schedule.
template <bool F, class S>
__device__ __forceinline__ Dither stepDither(const DevLevel& g, unsigned salt) {
    if constexpr (sizeof(S) == 2) return Dither{g.seed[F ? 1 : 0] ^ salt};
    else return Dither{0u};
}

template <bool F, class S>
__device__ __forceinline__ void advanceDither(const DevLevel& g) {
    if constexpr (sizeof(S) == 2) {
        if (blockIdx.x == 0 && threadIdx.x == 0) g.seed[F ? 0 : 1] = mix32(g.seed[F ? 1 : 0] + 0x6D2B79F5u);
    }
}

// Store one collided value: stochastic for 16-bit storage, as is otherwise.
template <class S, class T>
__device__ __forceinline__ void stD(S* p, T v, const Dither& D, unsigned cellBits, int q) {
    if constexpr (sizeof(S) == 2) Store<S>::stR(p, v, Dither::dir(cellBits, q));
    else Store<S>::st(p, v);
}

// Esotwist: with flipper F, direction d is read from the cell offset by
// max(0,-c_d) in slot (F ? inv(d) : d) and written after collision to the
// cell offset by max(0,+c_d) in slot (F ? d : inv(d))
// (include/esotwistStreamingFunctions.h:17-127).
template <bool F> __device__ __forceinline__ constexpr int preSlot(int d) { return F ? inv(d) : d; }
template <bool F> __device__ __forceinline__ constexpr int postSlot(int d) { return F ? d : inv(d); }

template <bool F, class S, class T>
__device__ __forceinline__ void readPre(const DevLevel& g, const int (&nb)[8], T (&f)[27]) {
    const S* base = static_cast<const S*>(g.f);
    // g.stride is read where it is used: holding it across the loop here and
    // in writePost (both inlined into the packed collide kernel's listed-cell
    // path) made that kernel 7% slower on a batch
#pragma unroll
    for (int d = 0; d < 27; ++d)
        f[d] = Store<S>::ld(base + (long long)preSlot<F>(d) * g.stride + nb[preNbr(d)]);
}

template <bool F, class S, class T>
__device__ __forceinline__ void writePost(const DevLevel& g, const int (&nb)[8], const T (&f)[27], const Dither& D) {
    S* base = static_cast<S*>(g.f);
    const unsigned cb = D.cell(nb[0]);
#pragma unroll
    for (int d = 0; d < 27; ++d) stD(base + (long long)postSlot<F>(d) * g.stride + nb[postNbr(d)], f[d], D, cb, d);
}

// Write f as pre-collision values of the cell (used by initial condition and
// periodic ghost copies, which both write with getPreCollisionIndex).
template <bool F, class S, class T>
__device__ __forceinline__ void writePre(const DevLevel& g, const int (&nb)[8], const T (&f)[27]) {
    S* base = static_cast<S*>(g.f);
    const long long stride = g.stride;  // once: stores may alias a descriptor in memory
#pragma unroll
    for (int d = 0; d < 27; ++d)
        Store<S>::st(base + (long long)preSlot<F>(d) * stride + nb[preNbr(d)], f[d]);
}

// writePre of interpolated values (interface), rounded like collided ones.
template <bool F, class S, class T>
__device__ __forceinline__ void writePreD(const DevLevel& g, const int (&nb)[8], const T (&f)[27], const Dither& D) {
    S* base = static_cast<S*>(g.f);
    const long long stride = g.stride;  // once: stores may alias a descriptor in memory
    const unsigned cb = D.cell(nb[0]);
#pragma unroll
    for (int d = 0; d < 27; ++d) stD(base + (long long)preSlot<F>(d) * stride + nb[preNbr(d)], f[d], D, cb, d);
}

}  // namespace lbm

namespace lbm {

// Density deviation and velocity from shifted populations with the
// reference's pairwise summation (getDRhoUxUyUz, include/cellFunctions.h:257-279).
template <class T>
__host__ __device__ __forceinline__ void macroFromF(const T (&f)[27], T& dRho, T& ux, T& uy, T& uz) {
    dRho = (((f[PPP] + f[MMM]) + (f[PMP] + f[MPM])) + ((f[PPM] + f[MMP]) + (f[PMM] + f[MPP]))) +
           (((f[OPP] + f[OMM]) + (f[OPM] + f[OMP])) + ((f[POP] + f[MOM]) + (f[POM] + f[MOP])) +
            ((f[PPO] + f[MMO]) + (f[PMO] + f[MPO]))) +
           ((f[POO] + f[MOO]) + (f[OPO] + f[OMO]) + (f[OOP] + f[OOM])) + f[OOO];
    const T rhoInv = T(1) / (dRho + T(1));
    const T a = f[PPP] - f[MMM], b = f[PMP] - f[MPM], c = f[PPM] - f[MMP], d = f[PMM] - f[MPP];
    const T mx = (((a + b) + (c + d)) + (((f[POP] - f[MOM]) + (f[POM] - f[MOP])) +
                                             ((f[PPO] - f[MMO]) + (f[PMO] - f[MPO])))) +
                     (f[POO] - f[MOO]);
    const T my = (((a - b) + (c - d)) + (((f[OPP] - f[OMM]) + (f[OPM] - f[OMP])) +
                                             ((f[PPO] - f[MMO]) - (f[PMO] - f[MPO])))) +
                     (f[OPO] - f[OMO]);
    const T mz = (((a + b) - (c + d)) + (((f[OPP] - f[OMM]) - (f[OPM] - f[OMP])) +
                                             ((f[POP] - f[MOM]) - (f[POM] - f[MOP])))) +
                     (f[OOP] - f[OOM]);
    ux = mx * rhoInv;
    uy = my * rhoInv;
    uz = mz * rhoInv;
}

}  // namespace lbm
