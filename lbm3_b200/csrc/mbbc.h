// Moment-based open boundary: restore the missing macroscopic quantity and
// close the unknown populations of a boundary cell from the generated tables
// (mbbc_tables.h).  Sums run over the known populations in direction order
// and products are formed as the reference's generated code forms them
// (include/boundaryConditions/{restoreRho,restoreUxUyUz,applyMBBC}.h), so the
// results agree with it to rounding.  All populations here are full
// (weight-compensated) f, as at the reference's call site
// (include/updateGrid.h:223-240).
#pragma once

#include "lattice.h"
#include "mbbc_tables.h"

namespace lbm {

// Table code of an outer normal; the row holding a code is found on the host
// (the tables live in device memory for device code).
LBM_HD int mbbcCode(int nx, int ny, int nz) { return (nx + 5) * 100 + (ny + 5) * 10 + (nz + 5); }

// Equilibrium value of moment m (the 23 moments in table order), with the
// reference generator's expressions (helperMain.py meq list).
LBM_HD float mbbcMomentEq(int m, float rho, float ux, float uy, float uz) {
    switch (m) {
        case 0: return rho;
        case 1: return rho * ux;
        case 2: return rho * uy;
        case 3: return rho * uz;
        case 4: return (1.f / 3.f) * rho + rho * ux * ux;
        case 5: return (1.f / 3.f) * rho + rho * uy * uy;
        case 6: return (1.f / 3.f) * rho + rho * uz * uz;
        case 7: return rho * uy * uz;
        case 8: return rho * ux * uz;
        case 9: return rho * ux * uy;
        case 10: return 0.f;
        case 11: return (1.f / 3.f) * rho * uy + rho * ux * ux * uy;
        case 12: return (1.f / 3.f) * rho * uz + rho * ux * ux * uz;
        case 13: return (1.f / 3.f) * rho * ux + rho * ux * uy * uy;
        case 14: return (1.f / 3.f) * rho * uz + rho * uy * uy * uz;
        case 15: return (1.f / 3.f) * rho * ux + rho * ux * uz * uz;
        case 16: return (1.f / 3.f) * rho * uy + rho * uy * uz * uz;
        case 17: return (1.f / 9.f) * rho + (1.f / 3.f) * rho * uy * uy + (1.f / 3.f) * rho * uz * uz +
                        rho * uy * uy * uz * uz;
        case 18: return (1.f / 9.f) * rho + (1.f / 3.f) * rho * ux * ux + (1.f / 3.f) * rho * uz * uz +
                        rho * ux * ux * uz * uz;
        case 19: return (1.f / 9.f) * rho + (1.f / 3.f) * rho * ux * ux + (1.f / 3.f) * rho * uy * uy +
                        rho * ux * ux * uy * uy;
        case 20: return (1.f / 3.f) * rho * uy * uz;
        case 21: return (1.f / 3.f) * rho * ux * uz;
        default: return (1.f / 3.f) * rho * ux * uy;
    }
}

// acc + c * v written the way the generated code writes the term.
LBM_HD float mbbcTerm(float acc, float c, float v) {
    if (c == 1.f) return acc + v;
    if (c == -1.f) return acc - v;
    return acc + c * v;
}

// applyMBBC: fill the unknown populations of f.
LBM_HD void mbbcApply(const LbmMbbcTable& T, float rho, float ux, float uy, float uz, float (&f)[27]) {
    float s[LBM_MBBC_MAX_UNKNOWN];
    for (int i = 0; i < T.nu; ++i) {
        float smf = 0.f;
        for (int k = 0; k < T.nk; ++k) {
            const int c = T.smfk[i][k];
            if (c != 0) smf = mbbcTerm(smf, float(c), f[T.known[k]]);
        }
        s[i] = mbbcMomentEq(T.moment[i], rho, ux, uy, uz) - smf;
    }
    for (int r = 0; r < T.nu; ++r) {
        float v = 0.f;
        for (int j = 0; j < T.nu; ++j) {
            const float c = T.inv[r][j];
            if (c != 0.f) v = mbbcTerm(v, c, s[j]);
        }
        f[T.unknown[r]] = v;
    }
}

// restoreRho: density from the known populations and the velocity.
LBM_HD float mbbcRestoreRho(const LbmMbbcTable& T, float ux, float uy, float uz, const float (&f)[27]) {
    const float scqu = T.rhoQu[0] * ux + T.rhoQu[1] * uy + T.rhoQu[2] * uz;
    const float s = T.rhoQ + scqu;
    float scmf = 0.f;
    for (int k = 0; k < T.nk; ++k) {
        const float c = T.rhoMfk[k];
        if (c != 0.f) scmf = mbbcTerm(scmf, c, f[T.known[k]]);
    }
    return scmf / s;
}

// restoreUxUyUz: velocity from the known populations and the density.
// Faces use the closed form (normal velocity from rhoZ, tangential velocity
// from k_nnt = 0); edges and corners solve the table's 3x3 relation.
LBM_HD void mbbcRestoreU(const LbmMbbcTable& T, int nx, int ny, int nz, float rho, const float (&f)[27],
                         float& ux, float& uy, float& uz) {
    if (T.face) {
        const int n[3] = {nx, ny, nz};
        float fZero = 0.f, fPlus = 0.f;
        for (int d = 0; d < 27; ++d) {
            const int cn = cx(d) * nx + cy(d) * ny + cz(d) * nz;
            if (cn == 0) fZero = fZero + f[d];
            else if (cn == 1) fPlus = fPlus + f[d];
        }
        const float uNormal = (fZero + 2.f * fPlus) / rho - 1.f;
        const float den = fZero + 2.f * (uNormal + 1.f) * rho * uNormal;
        float u[3];
        for (int a = 0; a < 3; ++a) {
            if (n[a] != 0) {
                u[a] = n[a] > 0 ? uNormal : -uNormal;
                continue;
            }
            float jZero = 0.f, jPlus = 0.f;
            for (int d = 0; d < 27; ++d) {
                const int cn = cx(d) * nx + cy(d) * ny + cz(d) * nz;
                const int ca = a == 0 ? cx(d) : a == 1 ? cy(d) : cz(d);
                if (ca == 0) continue;
                if (cn == 0) jZero = ca > 0 ? jZero + f[d] : jZero - f[d];
                else if (cn == 1) jPlus = ca > 0 ? jPlus + f[d] : jPlus - f[d];
            }
            u[a] = ((2.f * uNormal + 1.f) * jZero + 4.f * uNormal * jPlus) / den;
        }
        ux = u[0];
        uy = u[1];
        uz = u[2];
        return;
    }
    float s[3];
    for (int i = 0; i < 3; ++i) {
        float acc = 0.f;
        for (int k = 0; k < T.nk; ++k) {
            const float c = T.uMfk[i][k];
            if (c != 0.f) acc = mbbcTerm(acc, c, f[T.known[k]]);
        }
        s[i] = acc / rho - T.uQ[i];
    }
    float u[3];
    for (int a = 0; a < 3; ++a) {
        float v = 0.f;
        for (int j = 0; j < 3; ++j) {
            const float c = T.uInv[a][j];
            if (c != 0.f) v = mbbcTerm(v, c, s[j]);
        }
        u[a] = v;
    }
    ux = u[0];
    uy = u[1];
    uz = u[2];
}

}  // namespace lbm
