// D3Q27 lattice: direction numbering, velocities, inverse directions, weights.
//
// The numbering is the reference's (include/D3Q27Directions.h:8-34): it is a
// storage format (slot d of the population array holds direction d), so it
// has to be the same for dumped fields to be comparable.
#pragma once

#ifdef __CUDACC__
#define LBM_HD __host__ __device__ __forceinline__
#else
#define LBM_HD inline
#endif

namespace lbm {

enum Dir : int {
    OOO = 0, POO, MOO, OOM, OOP, OMO, OPO, POM, MOP, POP, MOM, MMO, PPO, OPM,
    OMP, MPO, PMO, OPP, OMM, MPM, PMP, MMP, PPM, PMM, MPP, MMM, PPP
};

constexpr int Q = 27;

// Velocity components packed per direction as (cx+1) + 3(cy+1) + 9(cz+1).
// A switch rather than an array so the helpers fold to constants in device
// code without constant memory.
LBM_HD constexpr int packed(int d) {
    switch (d) {
        case 0: return 13;  case 1: return 14;  case 2: return 12;  case 3: return 4;
        case 4: return 22;  case 5: return 10;  case 6: return 16;  case 7: return 5;
        case 8: return 21;  case 9: return 23;  case 10: return 3;  case 11: return 9;
        case 12: return 17; case 13: return 7;  case 14: return 19; case 15: return 15;
        case 16: return 11; case 17: return 25; case 18: return 1;  case 19: return 6;
        case 20: return 20; case 21: return 18; case 22: return 8;  case 23: return 2;
        case 24: return 24; case 25: return 0;  default: return 26;
    }
}

LBM_HD constexpr int cx(int d) { return packed(d) % 3 - 1; }
LBM_HD constexpr int cy(int d) { return (packed(d) / 3) % 3 - 1; }
LBM_HD constexpr int cz(int d) { return packed(d) / 9 - 1; }

// Direction with velocity (x, y, z), each in {-1, 0, 1}.
LBM_HD constexpr int dirOf(int x, int y, int z) {
    const int key = (x + 1) + 3 * (y + 1) + 9 * (z + 1);
    int r = 0;
    for (int d = 0; d < Q; ++d)
        if (packed(d) == key) r = d;
    return r;
}

LBM_HD constexpr int inv(int d) { return dirOf(-cx(d), -cy(d), -cz(d)); }

LBM_HD constexpr float weight(int d) {
    return (cx(d) * cx(d) + cy(d) * cy(d) + cz(d) * cz(d)) == 0 ? 8.f / 27.f
         : (cx(d) * cx(d) + cy(d) * cy(d) + cz(d) * cz(d)) == 1 ? 2.f / 27.f
         : (cx(d) * cx(d) + cy(d) * cy(d) + cz(d) * cz(d)) == 2 ? 1.f / 54.f
                                                                 : 1.f / 216.f;
}

// Weight in the arithmetic type T (exact fraction rounded once).
template <class T> LBM_HD constexpr T weightT(int d) {
    return (cx(d) * cx(d) + cy(d) * cy(d) + cz(d) * cz(d)) == 0 ? T(8) / T(27)
         : (cx(d) * cx(d) + cy(d) * cy(d) + cz(d) * cz(d)) == 1 ? T(2) / T(27)
         : (cx(d) * cx(d) + cy(d) * cy(d) + cz(d) * cz(d)) == 2 ? T(1) / T(54)
                                                                 : T(1) / T(216);
}

// Esotwist neighbour used by a direction: the cell offset by max(0, -c) on
// every axis holds the pre-collision value (include/esotwistStreamingFunctions.h:17-74);
// the post-collision value goes to the cell offset by max(0, +c) (:76-127).
// Offsets are encoded as bit 0 = +i, bit 1 = +j, bit 2 = +k.
LBM_HD constexpr int preNbr(int d) {
    return (cx(d) < 0 ? 1 : 0) | (cy(d) < 0 ? 2 : 0) | (cz(d) < 0 ? 4 : 0);
}
LBM_HD constexpr int postNbr(int d) {
    return (cx(d) > 0 ? 1 : 0) | (cy(d) > 0 ? 2 : 0) | (cz(d) > 0 ? 4 : 0);
}

}  // namespace lbm
