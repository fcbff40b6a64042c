// Moment-based open boundary in the form the device evaluates: the
// coefficient tables of one outer normal (mbbc_tables.h) re-indexed by
// population direction, so a kernel sweeps all 27 directions with static
// indices (populations stay in registers) and plain FMA chains (zero
// coefficients of unknown or unused populations add nothing).
//
// The closure (applyMBBC) solves S Mfu f_u = m_eq - S Mfk f_k for the unknown
// populations.  The host folds the two steps of the generated code into one
// row per unknown population u:
//   f_u = sum_m E[u][m] m_eq[m] + sum_d C[u][d] f_d,
// E = (S Mfu)^-1 grouped by equilibrium moment and C = -(S Mfu)^-1 S Mfk,
// formed in double and rounded once, so the kernel runs one short loop over
// the unknowns (equal to the generated code to rounding).  Populations are
// full (weight-compensated) f, as at the reference's call site
// (include/updateGrid.h:223-240); restoreRho and restoreUxUyUz keep the
// generated sums in ascending direction order.
#pragma once

#include "lattice.h"
#include "mbbc_tables.h"

namespace lbm {

// T: the arithmetic type of the kernel (the FP64 build holds the same
// coefficients, the generated float values, widened to double).
constexpr int kMbbcMoments = 23;  // equilibrium moments of the closure, in table order

template <class T> struct MbbcDirT {
    T E[LBM_MBBC_MAX_UNKNOWN][kMbbcMoments];  // unknown row r: weights of the equilibrium moments
    T C[LBM_MBBC_MAX_UNKNOWN][27];            // unknown row r: weights of the known populations
    T rhoMfk[27];                     // restoreRho numerator weights
    T uMfk[3][27];                    // restoreUxUyUz (edges, corners)
    T uInv[3][3];
    T uQ[3];
    T rhoQ, rhoQu[3];
    signed char unknownDir[LBM_MBBC_MAX_UNKNOWN];  // population d of unknown row r
    signed char unknownInv[LBM_MBBC_MAX_UNKNOWN];  // its inverse direction
    signed char unknownNbr[LBM_MBBC_MAX_UNKNOWN];  // esotwist pre-collision neighbour of d
    T unknownW[LBM_MBBC_MAX_UNKNOWN];              // lattice weight of d
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
    for (int r = 0; r < T.nu; ++r) {
        D.unknownMask |= 1u << T.unknown[r];
        D.unknownDir[r] = T.unknown[r];
        D.unknownInv[r] = static_cast<signed char>(inv(T.unknown[r]));
        D.unknownNbr[r] = static_cast<signed char>(preNbr(T.unknown[r]));
        D.unknownW[r] = weightT<V>(T.unknown[r]);
        double e[kMbbcMoments] = {};
        double c[27] = {};
        for (int j = 0; j < T.nu; ++j) {
            e[T.moment[j]] += double(T.inv[r][j]);
            for (int k = 0; k < T.nk; ++k) c[T.known[k]] -= double(T.inv[r][j]) * double(T.smfk[j][k]);
        }
        for (int m = 0; m < kMbbcMoments; ++m) D.E[r][m] = V(e[m]);
        for (int d = 0; d < 27; ++d) D.C[r][d] = V(c[d]);
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

// The 23 equilibrium moments of the closure, in table order.
template <class V> LBM_HD void mbbcMomentsEq(V rho, V ux, V uy, V uz, V (&m)[kMbbcMoments]) {
    const V t = V(1) / V(3), n = V(1) / V(9);
    m[0] = rho;
    m[1] = rho * ux;
    m[2] = rho * uy;
    m[3] = rho * uz;
    m[4] = t * rho + rho * ux * ux;
    m[5] = t * rho + rho * uy * uy;
    m[6] = t * rho + rho * uz * uz;
    m[7] = rho * uy * uz;
    m[8] = rho * ux * uz;
    m[9] = rho * ux * uy;
    m[10] = V(0);
    m[11] = t * rho * uy + rho * ux * ux * uy;
    m[12] = t * rho * uz + rho * ux * ux * uz;
    m[13] = t * rho * ux + rho * ux * uy * uy;
    m[14] = t * rho * uz + rho * uy * uy * uz;
    m[15] = t * rho * ux + rho * ux * uz * uz;
    m[16] = t * rho * uy + rho * uy * uz * uz;
    m[17] = n * rho + t * rho * uy * uy + t * rho * uz * uz + rho * uy * uy * uz * uz;
    m[18] = n * rho + t * rho * ux * ux + t * rho * uz * uz + rho * ux * ux * uz * uz;
    m[19] = n * rho + t * rho * ux * ux + t * rho * uy * uy + rho * ux * ux * uy * uy;
    m[20] = t * rho * uy * uz;
    m[21] = t * rho * ux * uz;
    m[22] = t * rho * ux * uy;
}

// applyMBBC for unknown row r: the closed (full) population T.unknownDir[r].
template <class V>
LBM_HD V mbbcUnknown(const MbbcDirT<V>& T, int r, const V (&meq)[kMbbcMoments], const V (&f)[27]) {
    V v = V(0);
#pragma unroll
    for (int m = 0; m < kMbbcMoments; ++m) v = mfma(T.E[r][m], meq[m], v);
#pragma unroll
    for (int d = 0; d < 27; ++d) v = mfma(T.C[r][d], f[d], v);
    return v;
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
