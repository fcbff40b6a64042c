// Moment-based open boundary in the form the device evaluates: the
// coefficient tables of one outer normal (mbbc_tables.h) re-indexed by
// population direction, so a kernel sweeps all 27 directions with static
// indices (populations stay in registers) and plain FMA chains (zero
// coefficients of unknown or unused populations add nothing).
//
// Sums run in ascending direction order, which is the order of the known
// populations in the generated tables and in the reference's generated code
// (include/boundaryConditions/{restoreRho,restoreUxUyUz,applyMBBC}.h), so the
// results agree with it to rounding.  Populations are full (weight-
// compensated) f, as at the reference's call site (include/updateGrid.h:223-240).
#pragma once

#include "lattice.h"
#include "mbbc_tables.h"

namespace lbm {

// T: the arithmetic type of the kernel (the FP64 build holds the same
// coefficients, the generated float values, widened to double).
template <class T> struct MbbcDirT {
    T smf[LBM_MBBC_MAX_UNKNOWN][27];  // S Mfk: weight of population d in equation i
    T inv[27][LBM_MBBC_MAX_UNKNOWN];  // row of (S Mfu)^-1 producing unknown population d
    T rhoMfk[27];                     // restoreRho numerator weights
    T uMfk[3][27];                    // restoreUxUyUz (edges, corners)
    T uInv[3][3];
    T uQ[3];
    T rhoQ, rhoQu[3];
    signed char moment[LBM_MBBC_MAX_UNKNOWN];  // equilibrium moment of equation i
    int nu;                                    // unknown count
    int face;                                  // 1: velocity from the face closed form
    unsigned unknownMask;                      // bit d: population d is unknown
    int nx, ny, nz;                            // outer normal
};
using MbbcDir = MbbcDirT<float>;

LBM_HD float mfma(float a, float b, float c) { return fmaf(a, b, c); }
LBM_HD double mfma(double a, double b, double c) { return fma(a, b, c); }

// Direction-indexed form of one generated table (host, at grid build).
template <class V = float> inline MbbcDirT<V> mbbcDirFromTable(const LbmMbbcTable& T) {
    MbbcDirT<V> D{};
    D.nu = T.nu;
    D.face = T.face;
    D.nx = T.code / 100 - 5;
    D.ny = (T.code / 10) % 10 - 5;
    D.nz = T.code % 10 - 5;
    for (int i = 0; i < T.nu; ++i) {
        D.moment[i] = T.moment[i];
        for (int k = 0; k < T.nk; ++k) D.smf[i][T.known[k]] = V(T.smfk[i][k]);
    }
    for (int r = 0; r < T.nu; ++r) {
        D.unknownMask |= 1u << T.unknown[r];
        for (int j = 0; j < T.nu; ++j) D.inv[T.unknown[r]][j] = T.inv[r][j];
    }
    for (int k = 0; k < T.nk; ++k) {
        D.rhoMfk[T.known[k]] = T.rhoMfk[k];
        for (int a = 0; a < 3; ++a) D.uMfk[a][T.known[k]] = T.uMfk[a][k];
    }
    for (int a = 0; a < 3; ++a) {
        D.uQ[a] = T.uQ[a];
        D.rhoQu[a] = T.rhoQu[a];
        for (int b = 0; b < 3; ++b) D.uInv[a][b] = T.uInv[a][b];
    }
    D.rhoQ = T.rhoQ;
    return D;
}

// Equilibrium value of moment m (the 23 moments in table order).
template <class V> LBM_HD V mbbcMomentEq(int m, V rho, V ux, V uy, V uz) {
    const V t = V(1) / V(3), n = V(1) / V(9);
    switch (m) {
        case 0: return rho;
        case 1: return rho * ux;
        case 2: return rho * uy;
        case 3: return rho * uz;
        case 4: return t * rho + rho * ux * ux;
        case 5: return t * rho + rho * uy * uy;
        case 6: return t * rho + rho * uz * uz;
        case 7: return rho * uy * uz;
        case 8: return rho * ux * uz;
        case 9: return rho * ux * uy;
        case 10: return V(0);
        case 11: return t * rho * uy + rho * ux * ux * uy;
        case 12: return t * rho * uz + rho * ux * ux * uz;
        case 13: return t * rho * ux + rho * ux * uy * uy;
        case 14: return t * rho * uz + rho * uy * uy * uz;
        case 15: return t * rho * ux + rho * ux * uz * uz;
        case 16: return t * rho * uy + rho * uy * uz * uz;
        case 17: return n * rho + t * rho * uy * uy + t * rho * uz * uz + rho * uy * uy * uz * uz;
        case 18: return n * rho + t * rho * ux * ux + t * rho * uz * uz + rho * ux * ux * uz * uz;
        case 19: return n * rho + t * rho * ux * ux + t * rho * uy * uy + rho * ux * ux * uy * uy;
        case 20: return t * rho * uy * uz;
        case 21: return t * rho * ux * uz;
        default: return t * rho * ux * uy;
    }
}

// applyMBBC: overwrite the unknown populations of f.
template <class V>
LBM_HD void mbbcApply(const MbbcDirT<V>& T, V rho, V ux, V uy, V uz, V (&f)[27]) {
    V s[LBM_MBBC_MAX_UNKNOWN];
#pragma unroll
    for (int i = 0; i < LBM_MBBC_MAX_UNKNOWN; ++i) {
        s[i] = V(0);
        if (i >= T.nu) continue;
        V smf = V(0);
#pragma unroll
        for (int d = 0; d < 27; ++d) smf = mfma(T.smf[i][d], f[d], smf);
        s[i] = mbbcMomentEq(T.moment[i], rho, ux, uy, uz) - smf;
    }
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        if (!(T.unknownMask >> d & 1u)) continue;
        V v = V(0);
#pragma unroll
        for (int j = 0; j < LBM_MBBC_MAX_UNKNOWN; ++j) v = mfma(T.inv[d][j], s[j], v);
        f[d] = v;
    }
}

// restoreRho: density from the known populations and the velocity.
template <class V>
LBM_HD V mbbcRestoreRho(const MbbcDirT<V>& T, V ux, V uy, V uz, const V (&f)[27]) {
    const V scqu = T.rhoQu[0] * ux + T.rhoQu[1] * uy + T.rhoQu[2] * uz;
    const V s = T.rhoQ + scqu;
    V scmf = V(0);
#pragma unroll
    for (int d = 0; d < 27; ++d) scmf = mfma(T.rhoMfk[d], f[d], scmf);
    return scmf / s;
}

// restoreUxUyUz: faces by the closed form (normal velocity from the
// known-population density, tangential velocity from a vanishing k_nnt),
// edges and corners from three moment relations free of the unknowns.
template <class V>
LBM_HD void mbbcRestoreU(const MbbcDirT<V>& T, V rho, const V (&f)[27], V& ux, V& uy, V& uz) {
    const int nx = T.nx, ny = T.ny, nz = T.nz;
    if (T.face) {
        V fZero = V(0), fPlus = V(0);
#pragma unroll
        for (int d = 0; d < 27; ++d) {
            const int cn = cx(d) * nx + cy(d) * ny + cz(d) * nz;
            if (cn == 0) fZero = fZero + f[d];
            else if (cn == 1) fPlus = fPlus + f[d];
        }
        const V uNormal = (fZero + V(2) * fPlus) / rho - V(1);
        const V den = fZero + V(2) * (uNormal + V(1)) * rho * uNormal;
        V u[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const int na = a == 0 ? nx : a == 1 ? ny : nz;
            if (na != 0) {
                u[a] = na > 0 ? uNormal : -uNormal;
                continue;
            }
            V jZero = V(0), jPlus = V(0);
#pragma unroll
            for (int d = 0; d < 27; ++d) {
                const int cn = cx(d) * nx + cy(d) * ny + cz(d) * nz;
                const int ca = a == 0 ? cx(d) : a == 1 ? cy(d) : cz(d);
                if (ca == 0) continue;
                if (cn == 0) jZero = ca > 0 ? jZero + f[d] : jZero - f[d];
                else if (cn == 1) jPlus = ca > 0 ? jPlus + f[d] : jPlus - f[d];
            }
            u[a] = ((V(2) * uNormal + V(1)) * jZero + V(4) * uNormal * jPlus) / den;
        }
        ux = u[0];
        uy = u[1];
        uz = u[2];
        return;
    }
    V s[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        V acc = V(0);
#pragma unroll
        for (int d = 0; d < 27; ++d) acc = mfma(T.uMfk[i][d], f[d], acc);
        s[i] = acc / rho - T.uQ[i];
    }
    V u[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        V v = V(0);
#pragma unroll
        for (int j = 0; j < 3; ++j) v = mfma(T.uInv[a][j], s[j], v);
        u[a] = v;
    }
    ux = u[0];
    uy = u[1];
    uz = u[2];
}

}  // namespace lbm
