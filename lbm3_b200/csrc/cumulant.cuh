// Well-conditioned D3Q27 cumulant collision (Geier et al. 2017), in registers.
//
// Follows the reference's applyCollision (include/applyCollision.h:17-491):
// shifted populations f_i - w_i are transformed to central moments with the
// weight-moment constants K (chimera transform z, then y, then x), converted
// to cumulants, relaxed (K17 with limiter, or AllOne when the limiter is
// <= 0), and transformed back (x, then y, then z).  The grouping of every
// sum and product is kept as in the reference so FP32 results agree to
// rounding.  What differs is where the work is done: every quantity that
// depends only on the viscosity (omega1, omega3..5, A, B) is computed once
// per grid on the host (CollisionConsts) instead of once per cell.
#pragma once

#include "lattice.h"

namespace lbm {

struct CollisionConsts {
    float omega1;      // 1 / (3 nu nuMultiplier + 1/2)
    float omega3, omega4, omega5, A, B;  // K17 parameters (:241-262)
    float tauTerm;     // 1/omega1 - 1/2
    float lambda;      // collision limiter (K17 when > 0 and nuMultiplier <= 1)
    int useK17;
    // products of the above that every cell needs, formed in the order the
    // reference multiplies them so the per-cell result rounds the same way
    float mHalfW1;     // -omega1 * 0.5
    float w1x15;       // 1.5 * omega1
    float mW1x3;       // -3 * omega1
    float oneMinusW1;  // 1 - omega1
    float halfW1c;     // 1 - 0.5 * omega1
    float oneMinusW3, oneMinusW4, oneMinusW5;
    float c43;         // (2/3) * tauTerm * A
    float c45;         // -(4/3) * tauTerm * A
    float cB;          // -(1/3) * tauTerm * B
};

// Host-side evaluation of the per-grid constants, with the reference's
// expressions (include/applyCollision.h:193-262).
inline CollisionConsts makeCollisionConsts(float nu, float nuMultiplier, float limiter) {
    CollisionConsts k{};
    const float omega1 = 1.f / (3.f * (nu * nuMultiplier) + 0.5f);
    const float omega2 = 1.f;
    k.omega1 = omega1;
    k.omega3 = 8.f * (omega1 - 2.f) * (omega2 * (3.f * omega1 - 1.f) - 5.f * omega1) /
               (8.f * (5.f - 2.f * omega1) * omega1 + omega2 * (8.f + omega1 * (9.f * omega1 - 26.f)));
    k.omega4 = 8.f * (omega1 - 2.f) * (omega1 + omega2 * (3.f * omega1 - 7.f)) /
               (omega2 * (56.f - 42.f * omega1 + 9.f * omega1 * omega1) - 8.f * omega1);
    k.omega5 = 24.f * (omega1 - 2.f) *
               (4.f * omega1 * omega1 + omega1 * omega2 * (18.f - 13.f * omega1) +
                omega2 * omega2 * (2.f + omega1 * (6.f * omega1 - 11.f))) /
               (16.f * omega1 * omega1 * (omega1 - 6.f) -
                2.f * omega1 * omega2 * (216.f + 5.f * omega1 * (9.f * omega1 - 46.f)) +
                omega2 * omega2 * (omega1 * (3.f * omega1 - 10.f) * (15.f * omega1 - 28.f) - 48.f));
    k.A = (4.f * omega1 * omega1 + 2.f * omega1 * omega2 * (omega1 - 6.f) +
           omega2 * omega2 * (omega1 * (10.f - 3.f * omega1) - 4.f)) /
          ((omega1 - omega2) * (omega2 * (2.f + 3.f * omega1) - 8.f * omega1));
    k.B = (4.f * omega1 * omega2 * (9.f * omega1 - 16.f) - 4.f * omega1 * omega1 -
           2.f * omega2 * omega2 * (2.f + 9.f * omega1 * (omega1 - 2.f))) /
          (3.f * (omega1 - omega2) * (omega2 * (2.f + 3.f * omega1) - 8.f * omega1));
    k.tauTerm = 1.f / omega1 - 0.5f;
    k.lambda = limiter;
    k.useK17 = (limiter > 0.f) && (nuMultiplier <= 1.f);
    k.mHalfW1 = -omega1 * 0.5f;
    k.w1x15 = 1.5f * omega1;
    k.mW1x3 = -3.f * omega1;
    k.oneMinusW1 = 1.f - omega1;
    k.halfW1c = 1.f - 0.5f * omega1;
    k.oneMinusW3 = 1.f - k.omega3;
    k.oneMinusW4 = 1.f - k.omega4;
    k.oneMinusW5 = 1.f - k.omega5;
    k.c43 = (2.f / 3.f) * k.tauTerm * k.A;
    k.c45 = -(4.f / 3.f) * k.tauTerm * k.A;
    k.cB = -(1.f / 3.f) * k.tauTerm * k.B;
    return k;
}

namespace detail {

constexpr float kThird = 1.f / 3.f;
constexpr float kNinth = 1.f / 9.f;
constexpr float k27th = 1.f / 27.f;

// a / b for the limiter weights: the hardware reciprocal on the device
// (two ulp), an exact division on the host.
LBM_HD float limDiv(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fdividef(a, b);
#else
    return a / b;
#endif
}

// Weight moments of the shifted transform, as the literal fractions the
// reference uses (K_aa0 ... K_c02, include/applyCollision.h:24-38).
// Index 0 = -1, 1 = 0, 2 = +1 along an axis.
LBM_HD constexpr float kZ(int a, int b) {  // z stage: sum of w over the (a,b) line
    return (a == 1 && b == 1) ? 4.f / 9.f : (a == 1 || b == 1) ? 1.f / 9.f : 1.f / 36.f;
}
LBM_HD constexpr float kY(int a, int n) {  // y stage: order-n z moment of the x=a plane
    return n == 1 ? 0.f
         : n == 0 ? (a == 1 ? 2.f / 3.f : 1.f / 6.f)
                  : (a == 1 ? 2.f / 9.f : 1.f / 18.f);
}

// Forward chimera step on one line (minus, zero, plus) -> orders 0,1,2.
// k0 is passed in when the caller already holds the order-0 sum.
LBM_HD void fwdLine(float m, float o, float p, float u, float u2, float K, float k0,
                    float& r1, float& r2) {
    r1 = (p - m) - u * (k0 + K);
    r2 = (p + m) - 2.f * u * (p - m) + u2 * (k0 + K);
}

}  // namespace detail

// f: shifted populations, in place.  gx,gy,gz: body force (half applied
// before and half after collision, :70-72 and the sign flip of first-order
// moments before the back transform).  lambda: limiter for this cell.
LBM_HD void collideCumulant(float (&f)[27], const CollisionConsts& P, float lambda,
                            float gx, float gy, float gz) {
    using namespace detail;
    // m[x][y][z]: after the z stage z holds the moment order, etc.
    float m[3][3][3];
    // ---- z stage: populations -> (x,y) lines of z moments ----
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const float pm = f[dirOf(a - 1, b - 1, -1)];
            const float po = f[dirOf(a - 1, b - 1, 0)];
            const float pp = f[dirOf(a - 1, b - 1, 1)];
            m[a][b][0] = (pp + pm) + po;
        }
    // density and momentum from the zeroth z moments (:49-69)
    const float dRho = ((m[0][0][0] + m[0][1][0]) + m[0][2][0]) +
                       ((m[1][0][0] + m[1][1][0]) + m[1][2][0]) +
                       ((m[2][0][0] + m[2][1][0]) + m[2][2][0]);
    const float rho = 1.f + dRho;
    const float rhoInv = 1.f / rho;
    const float momX = ((m[2][0][0] + m[2][1][0]) + m[2][2][0]) -
                       ((m[0][0][0] + m[0][1][0]) + m[0][2][0]);
    const float momY = ((m[0][2][0] + m[1][2][0]) + m[2][2][0]) -
                       ((m[0][0][0] + m[1][0][0]) + m[2][0][0]);
    // z momentum: pairs (P - M) summed in the reference's grouping (:62-65)
    const float dz00 = f[MMP] - f[MMM], dz01 = f[MOP] - f[MOM], dz02 = f[MPP] - f[MPM];
    const float dz10 = f[OMP] - f[OMM], dz11 = f[OOP] - f[OOM], dz12 = f[OPP] - f[OPM];
    const float dz20 = f[PMP] - f[PMM], dz21 = f[POP] - f[POM], dz22 = f[PPP] - f[PPM];
    const float momZ = (((dz00 + dz01) + (dz02 + dz10)) + ((dz11 + dz12) + (dz20 + dz21))) + dz22;

    const float ux = (momX + 0.5f * gx) * rhoInv;
    const float uy = (momY + 0.5f * gy) * rhoInv;
    const float uz = (momZ + 0.5f * gz) * rhoInv;
    const float ux2 = ux * ux, uy2 = uy * uy, uz2 = uz * uz;

#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const float pm = f[dirOf(a - 1, b - 1, -1)];
            const float pp = f[dirOf(a - 1, b - 1, 1)];
            fwdLine(pm, 0.f, pp, uz, uz2, kZ(a, b), m[a][b][0], m[a][b][1], m[a][b][2]);
        }
    // ---- y stage ----
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int n = 0; n < 3; ++n) {
            const float lo = m[a][0][n], mid = m[a][1][n], hi = m[a][2][n];
            const float K = kY(a, n);
            const float k0 = (hi + lo) + mid;
            float r1, r2;
            fwdLine(lo, mid, hi, uy, uy2, K, k0, r1, r2);
            m[a][0][n] = k0;
            m[a][1][n] = r1;
            m[a][2][n] = r2;
        }
    // ---- x stage: central moments k[ord x][ord y][ord z] ----
    float k[3][3][3];
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int n = 0; n < 3; ++n) {
            const float lo = m[0][b][n], mid = m[1][b][n], hi = m[2][b][n];
            const float K = (b == 1 || n == 1) ? 0.f
                          : (b == 0 && n == 0) ? 1.f
                          : (b == 2 && n == 2) ? 1.f / 9.f
                                               : 1.f / 3.f;
            const float k0 = (b == 0 && n == 0) ? dRho : (hi + lo) + mid;
            float r1, r2;
            fwdLine(lo, mid, hi, ux, ux2, K, k0, r1, r2);
            k[0][b][n] = k0;
            k[1][b][n] = r1;
            k[2][b][n] = r2;
        }

    // ---- central moments -> cumulants (:164-187) ----
    const float C110 = k[1][1][0], C101 = k[1][0][1], C011 = k[0][1][1];
    const float C200 = k[2][0][0], C020 = k[0][2][0], C002 = k[0][0][2];
    const float C111 = k[1][1][1];
    const float C120 = k[1][2][0], C102 = k[1][0][2], C210 = k[2][1][0];
    const float C012 = k[0][1][2], C201 = k[2][0][1], C021 = k[0][2][1];
    const float third = kThird;
    const float dRhoNinth = dRho * rhoInv * kNinth;
    // C211, C121, C112, C220, C022, C202 (:170-187) only enter the reference's
    // relaxation multiplied by (1 - omega6..8) = 0, so they are not formed.
    const float k000 = dRho;

    // ---- relaxation (:193-342); omega2 = omega6 = omega7 = omega8 = 1, so
    // the (1 - omega) terms of those rates vanish and are not evaluated ----
    const float Dxu = P.mHalfW1 * rhoInv * (2.f * C200 - C020 - C002) -
                      0.5f * rhoInv * (C200 + C020 + C002 - k000);
    const float Dyv = Dxu + P.w1x15 * rhoInv * (C200 - C020);
    const float Dzw = Dxu + P.w1x15 * rhoInv * (C200 - C002);
    const float DxvDyu = P.mW1x3 * rhoInv * C110;
    const float DxwDzu = P.mW1x3 * rhoInv * C101;
    const float DywDzv = P.mW1x3 * rhoInv * C011;

    const float Cs110 = P.oneMinusW1 * C110;
    const float Cs101 = P.oneMinusW1 * C101;
    const float Cs011 = P.oneMinusW1 * C011;
    const float r3 = 3.f * rho * P.halfW1c;
    const float e33 = P.oneMinusW1 * (C200 - C020) - r3 * (ux2 * Dxu - uy2 * Dyv);
    const float e34 = P.oneMinusW1 * (C200 - C002) - r3 * (ux2 * Dxu - uz2 * Dzw);
    const float e35 = k000 - 3.f * rho * 0.5f * (ux2 * Dxu + uy2 * Dyv + uz2 * Dzw);
    const float Cs200 = (e33 + e34 + e35) * kThird;
    const float Cs020 = (e34 - 2.f * e33 + e35) * kThird;
    const float Cs002 = (e33 - 2.f * e34 + e35) * kThird;

    float Cs120 = 0.f, Cs102 = 0.f, Cs210 = 0.f, Cs012 = 0.f, Cs201 = 0.f, Cs021 = 0.f;
    float Cs111 = 0.f, Cs220 = 0.f, Cs202 = 0.f, Cs022 = 0.f, Cs211 = 0.f, Cs121 = 0.f, Cs112 = 0.f;
    if (P.useK17 && lambda > 0.f) {
        // K17 with limiter: third-order rates pushed from omega3..5 towards 1
        // where the cumulant is large compared with lambda (:270-306)
        const float p1 = C120 + C102, p2 = C210 + C012, p3 = C201 + C021;
        const float q1 = C120 - C102, q2 = C210 - C012, q3 = C201 - C021;
        // 1 - (om + (1 - om) |v| / (lambda + |v|)) applied to v
        auto relax = [&](float om, float oneMinusOm, float v) {
            const float av = fabsf(v);
            return (1.f - (om + limDiv(oneMinusOm * av, lambda + av))) * v;
        };
        const float e117 = relax(P.omega3, P.oneMinusW3, p1);
        const float e118 = relax(P.omega3, P.oneMinusW3, p2);
        const float e119 = relax(P.omega3, P.oneMinusW3, p3);
        const float e120 = relax(P.omega4, P.oneMinusW4, q1);
        const float e121 = relax(P.omega4, P.oneMinusW4, q2);
        const float e122 = relax(P.omega4, P.oneMinusW4, q3);
        Cs120 = 0.5f * (e120 + e117);
        Cs102 = 0.5f * (-e120 + e117);
        Cs210 = 0.5f * (e121 + e118);
        Cs012 = 0.5f * (-e121 + e118);
        Cs201 = 0.5f * (e122 + e119);
        Cs021 = 0.5f * (-e122 + e119);
        Cs111 = relax(P.omega5, P.oneMinusW5, C111);
        // fourth order (:310-323)
        const float e43 = P.c43 * rho * (Dxu - 2.f * Dyv + Dzw);
        const float e44 = P.c43 * rho * (-2.f * Dxu + Dyv + Dzw);
        const float e45 = P.c45 * rho * (Dxu + Dyv + Dzw);
        Cs220 = (e43 + e44 + e45) * kThird;
        Cs202 = (-e43 + e45) * kThird;
        Cs022 = (-e44 + e45) * kThird;
        Cs211 = P.cB * rho * DywDzv;
        Cs121 = P.cB * rho * DxwDzu;
        Cs112 = P.cB * rho * DxvDyu;
    }

    // ---- cumulants -> central moments (:348-384) ----
    float s[3][3][3];
    s[0][1][1] = Cs011; s[1][0][1] = Cs101; s[1][1][0] = Cs110; s[1][1][1] = Cs111;
    s[0][0][2] = Cs002; s[0][2][0] = Cs020; s[2][0][0] = Cs200;
    s[0][1][2] = Cs012; s[0][2][1] = Cs021; s[1][0][2] = Cs102;
    s[2][0][1] = Cs201; s[1][2][0] = Cs120; s[2][1][0] = Cs210;
    s[2][1][1] = Cs211 + ((Cs200 + third) * Cs011 + 2.f * Cs101 * Cs110) * rhoInv;
    s[1][2][1] = Cs121 + ((Cs020 + third) * Cs101 + 2.f * Cs110 * Cs011) * rhoInv;
    s[1][1][2] = Cs112 + ((Cs002 + third) * Cs110 + 2.f * Cs011 * Cs101) * rhoInv;
    s[2][2][0] = Cs220 + ((Cs020 * Cs200 + 2.f * Cs110 * Cs110 + (Cs200 + Cs020) * kThird) * rhoInv - dRhoNinth);
    s[0][2][2] = Cs022 + ((Cs002 * Cs020 + 2.f * Cs011 * Cs011 + (Cs002 + Cs020) * kThird) * rhoInv - dRhoNinth);
    s[2][0][2] = Cs202 + ((Cs200 * Cs002 + 2.f * Cs101 * Cs101 + (Cs200 + Cs002) * kThird) * rhoInv - dRhoNinth);
    s[1][2][2] = (Cs020 * Cs102 + Cs002 * Cs120 + 4.f * Cs011 * Cs111 +
                  2.f * (Cs110 * Cs012 + Cs101 * Cs021) + (Cs120 + Cs102) * kThird) * rhoInv;
    s[2][1][2] = (Cs002 * Cs210 + Cs200 * Cs012 + 4.f * Cs101 * Cs111 +
                  2.f * (Cs011 * Cs201 + Cs110 * Cs102) + (Cs210 + Cs012) * kThird) * rhoInv;
    s[2][2][1] = (Cs200 * Cs021 + Cs020 * Cs201 + 4.f * Cs110 * Cs111 +
                  2.f * (Cs101 * Cs120 + Cs011 * Cs210) + (Cs021 + Cs201) * kThird) * rhoInv;
    {
        const float a200 = Cs200, a020 = Cs020, a002 = Cs002;
        const float a110 = Cs110, a101 = Cs101, a011 = Cs011, a111 = Cs111;
        s[2][2][2] =
            (4.f * a111 * a111 + a200 * s[0][2][2] + a020 * s[2][0][2] + a002 * s[2][2][0] +
             4.f * (a011 * s[2][1][1] + a101 * s[1][2][1] + a110 * s[1][1][2]) +
             2.f * (Cs120 * Cs102 + Cs210 * Cs012 + Cs201 * Cs021)) * rhoInv -
            (16.f * a110 * a101 * a011 +
             4.f * (a101 * a101 * a020 + a011 * a011 * a200 + a110 * a110 * a002) +
             2.f * a200 * a020 * a002) * rhoInv * rhoInv +
            (3.f * (s[0][2][2] + s[2][0][2] + s[2][2][0]) + (a200 + a020 + a002)) * rhoInv * kNinth -
            (2.f / 3.f) *
                (2.f * (a101 * a101 + a011 * a011 + a110 * a110) +
                 (a002 * a020 + a002 * a200 + a020 * a200) + (a002 + a020 + a200) * kThird) *
                rhoInv * rhoInv -
            (dRho * dRho - dRho) * rhoInv * rhoInv * k27th;
    }
    s[0][0][0] = k000;
    s[1][0][0] = -k[1][0][0];
    s[0][1][0] = -k[0][1][0];
    s[0][0][1] = -k[0][0][1];

    // ---- back transform, x stage (:390-418): s[ord x][..] -> m[pop x][ord y][ord z]
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int n = 0; n < 3; ++n) {
            const float s0 = s[0][b][n], s1 = s[1][b][n], s2 = s[2][b][n];
            const bool hasK = (b != 1 && n != 1);
            const float K = !hasK ? 0.f
                          : (b == 0 && n == 0) ? 1.f
                          : (b == 2 && n == 2) ? 1.f / 9.f
                                               : 1.f / 3.f;
            const float div = (b == 0 && n == 0) ? 1.f : (b == 2 && n == 2) ? 9.f : 3.f;
            float mid = s0 * (1.f - ux2) - 2.f * ux * s1 - s2;
            if (hasK) mid = mid - ((b == 0 && n == 0) ? ux2 : ux2 * (1.f / div));
            m[1][b][n] = mid;
            m[0][b][n] = ((s0 + K) * (ux2 - ux) + s1 * (2.f * ux - 1.f) + s2) * 0.5f;
            m[2][b][n] = ((s0 + K) * (ux2 + ux) + s1 * (2.f * ux + 1.f) + s2) * 0.5f;
        }
    // ---- y stage (:420-448)
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int n = 0; n < 3; ++n) {
            const float s0 = m[a][0][n], s1 = m[a][1][n], s2 = m[a][2][n];
            const bool hasK = n != 1;
            const float K = kY(a, n);
            float mid = s0 * (1.f - uy2) - 2.f * uy * s1 - s2;
            if (hasK) mid = mid - K * uy2;
            m[a][1][n] = mid;
            m[a][0][n] = ((s0 + K) * (uy2 - uy) + s1 * (2.f * uy - 1.f) + s2) * 0.5f;
            m[a][2][n] = ((s0 + K) * (uy2 + uy) + s1 * (2.f * uy + 1.f) + s2) * 0.5f;
        }
    // ---- z stage (:450-490): back to populations
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const float s0 = m[a][b][0], s1 = m[a][b][1], s2 = m[a][b][2];
            const float K = kZ(a, b);
            f[dirOf(a - 1, b - 1, 0)] = s0 * (1.f - uz2) - 2.f * uz * s1 - s2 - K * uz2;
            f[dirOf(a - 1, b - 1, -1)] = ((s0 + K) * (uz2 - uz) + s1 * (2.f * uz - 1.f) + s2) * 0.5f;
            f[dirOf(a - 1, b - 1, 1)] = ((s0 + K) * (uz2 + uz) + s1 * (2.f * uz + 1.f) + s2) * 0.5f;
        }
}

}  // namespace lbm
