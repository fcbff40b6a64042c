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
// formed in double and rounded once (equal to the generated code to
// rounding).  The tables are stored transposed, column m (or d) holding the
// weights of every unknown row, padded to kMbbcRowPad, so that a kernel
// forms all rows at once: one 16-byte shared-memory load feeds four FMAs,
// and the columns of unknown populations (zero weights) are skipped.  Populations are
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

constexpr int kMbbcRowPad = 20;   // LBM_MBBC_MAX_UNKNOWN rounded up to a multiple of 4

template <class T> struct alignas(16) MbbcDirT {
    T ET[kMbbcMoments][kMbbcRowPad];  // column m: weight of equilibrium moment m in every unknown row
    T CT[27][kMbbcRowPad];            // column d: weight of known population d in every unknown row
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
        for (int m = 0; m < kMbbcMoments; ++m) D.ET[m][r] = V(e[m]);
        for (int d = 0; d < 27; ++d) D.CT[d][r] = V(c[d]);
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

// Four consecutive table entries (16 bytes for float, two 16-byte loads for double).
LBM_HD void mbbcLoad4(const float* p, float (&o)[4]) {
#ifdef __CUDA_ARCH__
    const float4 v = *reinterpret_cast<const float4*>(p);
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
#else
    for (int k = 0; k < 4; ++k) o[k] = p[k];
#endif
}
LBM_HD void mbbcLoad4(const double* p, double (&o)[4]) {
#ifdef __CUDA_ARCH__
    const double2 a = *reinterpret_cast<const double2*>(p), b = *reinterpret_cast<const double2*>(p + 2);
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
#else
    for (int k = 0; k < 4; ++k) o[k] = p[k];
#endif
}

// applyMBBC for every unknown row at once: out[r] is the closed (full)
// population T.unknownDir[r] for r < T.nu.  `unknown` is T.unknownMask (the
// skipped columns) and `groups` = (T.nu + 3) / 4, both uniform over a CTA.
template <class V>
LBM_HD void mbbcClose(const MbbcDirT<V>& T, unsigned unknown, int groups, const V (&meq)[kMbbcMoments],
                      const V (&f)[27], V (&out)[kMbbcRowPad]) {
#pragma unroll
    for (int r = 0; r < kMbbcRowPad; ++r) out[r] = V(0);
#pragma unroll
    for (int m = 0; m < kMbbcMoments; ++m) {
        if (m == 10) continue;  // the moment is zero at equilibrium
#pragma unroll
        for (int q = 0; q < kMbbcRowPad / 4; ++q) {
            if (q >= groups) break;
            V w[4];
            mbbcLoad4(&T.ET[m][4 * q], w);
#pragma unroll
            for (int k = 0; k < 4; ++k) out[4 * q + k] = mfma(w[k], meq[m], out[4 * q + k]);
        }
    }
#pragma unroll
    for (int d = 0; d < 27; ++d) {
        if ((unknown >> d) & 1u) continue;
#pragma unroll
        for (int q = 0; q < kMbbcRowPad / 4; ++q) {
            if (q >= groups) break;
            V w[4];
            mbbcLoad4(&T.CT[d][4 * q], w);
#pragma unroll
            for (int k = 0; k < 4; ++k) out[4 * q + k] = mfma(w[k], f[d], out[4 * q + k]);
        }
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
