// Well-conditioned D3Q27 cumulant collision (Geier et al. 2017), in registers.
//
// Follows the reference's applyCollision (include/applyCollision.h:17-491):
// shifted populations f_i - w_i are transformed to central moments with the
// weight-moment constants K (chimera transform z, then y, then x), converted
// to cumulants, relaxed (K17 with limiter, or AllOne when the limiter is
// <= 0), and transformed back (x, then y, then z).  Sums in the forward
// transform and the cumulant algebra keep the reference's grouping; the back
// transform is refactored into fused multiply-adds with per-cell constants
// (algebraically the reference's Eqs. 57-65, rounded differently).  Every
// quantity that depends only on the viscosity (omega1, omega3..5, A, B) is
// computed once per grid on the host (CollisionConsts) instead of per cell.
//
// The arithmetic is a template over the value type: `float` collides one
// cell, `Pair` collides two cells at once with the packed FP32x2 instructions
// of sm_100 (add/mul/fma .rn.f32x2), which issue once for both cells (both
// lanes follow exactly the scalar sequence of operations), and `double` is
// the FP64 build that serves as the reference of the storage-precision study.
#pragma once

#include "lattice.h"

#ifdef __CUDACC__
#include <cuda_runtime.h>
#endif

namespace lbm {

template <class T> struct CollisionConstsT {
    T omega1;      // 1 / (3 nu nuMultiplier + 1/2)
    T omega3, omega4, omega5, A, B;  // K17 parameters (:241-262)
    T tauTerm;     // 1/omega1 - 1/2
    T lambda;      // collision limiter (K17 when > 0 and nuMultiplier <= 1)
    int useK17;
    // products of the above that every cell needs
    T mHalfW1;     // -omega1 * 0.5
    T w1x15;       // 1.5 * omega1
    T mW1x3;       // -3 * omega1
    T oneMinusW1;  // 1 - omega1
    T halfW1c;     // 1 - 0.5 * omega1
    T oneMinusW3, oneMinusW4, oneMinusW5;
    T c43;         // (2/3) * tauTerm * A
    T c45;         // -(4/3) * tauTerm * A
    T cB;          // -(1/3) * tauTerm * B
};
using CollisionConsts = CollisionConstsT<float>;

// Host-side evaluation of the per-grid constants, with the reference's
// expressions (include/applyCollision.h:193-262), in the arithmetic type T.
template <class T> inline CollisionConstsT<T> makeCollisionConstsT(T nu, T nuMultiplier, T limiter) {
    CollisionConstsT<T> k{};
    const T omega1 = T(1) / (T(3) * (nu * nuMultiplier) + T(0.5));
    const T omega2 = T(1);
    k.omega1 = omega1;
    k.omega3 = T(8) * (omega1 - T(2)) * (omega2 * (T(3) * omega1 - T(1)) - T(5) * omega1) /
               (T(8) * (T(5) - T(2) * omega1) * omega1 + omega2 * (T(8) + omega1 * (T(9) * omega1 - T(26))));
    k.omega4 = T(8) * (omega1 - T(2)) * (omega1 + omega2 * (T(3) * omega1 - T(7))) /
               (omega2 * (T(56) - T(42) * omega1 + T(9) * omega1 * omega1) - T(8) * omega1);
    k.omega5 = T(24) * (omega1 - T(2)) *
               (T(4) * omega1 * omega1 + omega1 * omega2 * (T(18) - T(13) * omega1) +
                omega2 * omega2 * (T(2) + omega1 * (T(6) * omega1 - T(11)))) /
               (T(16) * omega1 * omega1 * (omega1 - T(6)) -
                T(2) * omega1 * omega2 * (T(216) + T(5) * omega1 * (T(9) * omega1 - T(46))) +
                omega2 * omega2 * (omega1 * (T(3) * omega1 - T(10)) * (T(15) * omega1 - T(28)) - T(48)));
    k.A = (T(4) * omega1 * omega1 + T(2) * omega1 * omega2 * (omega1 - T(6)) +
           omega2 * omega2 * (omega1 * (T(10) - T(3) * omega1) - T(4))) /
          ((omega1 - omega2) * (omega2 * (T(2) + T(3) * omega1) - T(8) * omega1));
    k.B = (T(4) * omega1 * omega2 * (T(9) * omega1 - T(16)) - T(4) * omega1 * omega1 -
           T(2) * omega2 * omega2 * (T(2) + T(9) * omega1 * (omega1 - T(2)))) /
          (T(3) * (omega1 - omega2) * (omega2 * (T(2) + T(3) * omega1) - T(8) * omega1));
    k.tauTerm = T(1) / omega1 - T(0.5);
    k.lambda = limiter;
    k.useK17 = (limiter > T(0)) && (nuMultiplier <= T(1));
    k.mHalfW1 = -omega1 * T(0.5);
    k.w1x15 = T(1.5) * omega1;
    k.mW1x3 = T(-3) * omega1;
    k.oneMinusW1 = T(1) - omega1;
    k.halfW1c = T(1) - T(0.5) * omega1;
    k.oneMinusW3 = T(1) - k.omega3;
    k.oneMinusW4 = T(1) - k.omega4;
    k.oneMinusW5 = T(1) - k.omega5;
    k.c43 = (T(2) / T(3)) * k.tauTerm * k.A;
    k.c45 = -(T(4) / T(3)) * k.tauTerm * k.A;
    k.cB = -(T(1) / T(3)) * k.tauTerm * k.B;
    return k;
}
inline CollisionConsts makeCollisionConsts(float nu, float nuMultiplier, float limiter) {
    return makeCollisionConstsT<float>(nu, nuMultiplier, limiter);
}

// ---- value types -----------------------------------------------------------
// Scalar: plain float operators (the compiler fuses a*b+c on the device).
LBM_HD float fmaR(float a, float b, float c) { return a * b + c; }
LBM_HD float absR(float a) { return fabsf(a); }
LBM_HD float bcast(float a, float) { return a; }
// a / b for the limiter weights: the hardware reciprocal on the device
// (two ulp), an exact division on the host.
LBM_HD float divFast(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fdividef(a, b);
#else
    return a / b;
#endif
}
LBM_HD float rcpR(float a) {
#ifdef __CUDA_ARCH__
    return __frcp_rn(a);  // the correctly rounded 1 / a
#else
    return 1.f / a;
#endif
}
// Double: the FP64 build of the kernels (reference for storage precision).
LBM_HD double fmaR(double a, double b, double c) { return fma(a, b, c); }
LBM_HD double absR(double a) { return fabs(a); }
LBM_HD double bcast(double a, double) { return a; }
LBM_HD double divFast(double a, double b) { return a / b; }
LBM_HD double rcpR(double a) { return 1.0 / a; }

// Scalar type of a value type (the type of its constants).
template <class R> struct ScalarOf { using type = R; };

#ifdef __CUDACC__
// Two cells in the two lanes of a packed FP32x2 register pair.
struct Pair {
    float2 v;
};
__device__ __forceinline__ Pair mkPair(float a, float b) { return {make_float2(a, b)}; }
__device__ __forceinline__ Pair bcast(float a, Pair) { return {make_float2(a, a)}; }
__device__ __forceinline__ Pair operator+(Pair a, Pair b) { return {__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ Pair operator*(Pair a, Pair b) { return {__fmul2_rn(a.v, b.v)}; }
// a - b as a + (-1) b: one packed FMA, exact like a subtraction
__device__ __forceinline__ Pair operator-(Pair a, Pair b) { return {__ffma2_rn(b.v, make_float2(-1.f, -1.f), a.v)}; }
__device__ __forceinline__ Pair fmaR(Pair a, Pair b, Pair c) { return {__ffma2_rn(a.v, b.v, c.v)}; }
__device__ __forceinline__ Pair operator+(Pair a, float b) { return a + Pair{make_float2(b, b)}; }
__device__ __forceinline__ Pair operator+(float a, Pair b) { return Pair{make_float2(a, a)} + b; }
__device__ __forceinline__ Pair operator-(Pair a, float b) { return a + Pair{make_float2(-b, -b)}; }
__device__ __forceinline__ Pair operator-(float a, Pair b) { return Pair{make_float2(a, a)} - b; }
__device__ __forceinline__ Pair operator*(Pair a, float b) { return a * Pair{make_float2(b, b)}; }
__device__ __forceinline__ Pair operator*(float a, Pair b) { return Pair{make_float2(a, a)} * b; }
__device__ __forceinline__ Pair fmaR(Pair a, float b, Pair c) { return fmaR(a, Pair{make_float2(b, b)}, c); }
__device__ __forceinline__ Pair fmaR(float a, Pair b, Pair c) { return fmaR(Pair{make_float2(a, a)}, b, c); }
__device__ __forceinline__ Pair fmaR(Pair a, Pair b, float c) { return fmaR(a, b, Pair{make_float2(c, c)}); }
__device__ __forceinline__ Pair absR(Pair a) { return {make_float2(fabsf(a.v.x), fabsf(a.v.y))}; }
__device__ __forceinline__ Pair divFast(Pair a, Pair b) {
    return {make_float2(__fdividef(a.v.x, b.v.x), __fdividef(a.v.y, b.v.y))};
}
__device__ __forceinline__ Pair rcpR(Pair a) { return {make_float2(__frcp_rn(a.v.x), __frcp_rn(a.v.y))}; }
template <> struct ScalarOf<Pair> { using type = float; };
#endif

namespace detail {

// exact fractions rounded once to the scalar type
template <class Sc> struct Frac {
    static constexpr Sc third = Sc(1) / Sc(3);
    static constexpr Sc ninth = Sc(1) / Sc(9);
    static constexpr Sc n27th = Sc(1) / Sc(27);
    static constexpr Sc twoThirds = Sc(2) / Sc(3);
};

// Weight moments of the shifted transform, as the literal fractions the
// reference uses (K_aa0 ... K_c02, include/applyCollision.h:24-38).
// Index 0 = -1, 1 = 0, 2 = +1 along an axis.
template <class Sc = float> LBM_HD constexpr Sc kZ(int a, int b) {  // z stage: sum of w over the (a,b) line
    return (a == 1 && b == 1) ? Sc(4) / Sc(9) : (a == 1 || b == 1) ? Sc(1) / Sc(9) : Sc(1) / Sc(36);
}
template <class Sc = float> LBM_HD constexpr Sc kY(int a, int n) {  // y stage: order-n z moment of the x=a plane
    return n == 1 ? Sc(0)
         : n == 0 ? (a == 1 ? Sc(2) / Sc(3) : Sc(1) / Sc(6))
                  : (a == 1 ? Sc(2) / Sc(9) : Sc(1) / Sc(18));
}
template <class Sc = float> LBM_HD constexpr Sc kX(int b, int n) {  // x stage: order (y, z) moment of the weights
    return (b == 1 || n == 1) ? Sc(0) : (b == 0 && n == 0) ? Sc(1) : (b == 2 && n == 2) ? Sc(1) / Sc(9) : Sc(1) / Sc(3);
}

// Per-cell constants of one axis, for the line transforms.
template <class R> struct Axis {
    R mu, u2, m2u;       // -u, u^2, -2u
    R omu2, hlo, hhi;    // 1 - u^2, (u^2 - u) / 2, (u^2 + u) / 2
    R um, up;            // u - 1/2, u + 1/2
};
template <class R> LBM_HD Axis<R> axisOf(R u) {
    Axis<R> c;
    c.u2 = u * u;
    c.mu = u * -1.f;
    c.m2u = u * -2.f;
    c.omu2 = 1.f - c.u2;
    const R hu2 = c.u2 * 0.5f;
    c.hlo = fmaR(u, -0.5f, hu2);
    c.hhi = fmaR(u, 0.5f, hu2);
    c.um = u - 0.5f;
    c.up = u + 0.5f;
    return c;
}

// Forward chimera step of one line (minus m, zero o, plus p) with the order-0
// sum k0 and the weight moment K: orders 1 and 2 about velocity u,
//   r1 = (p - m) - u (k0 + K),  r2 = (p + m) - 2u (p - m) + u^2 (k0 + K).
template <class R, class Sc>
LBM_HD void fwd(R s, R d, R k0, Sc K, const Axis<R>& c, R& r1, R& r2) {
    const R kk = K != Sc(0) ? k0 + K : k0;
    r1 = fmaR(c.mu, kk, d);
    r2 = fmaR(c.u2, kk, fmaR(c.m2u, d, s));
}

// Backward chimera step of one line from orders (s0, s1, s2) to the values at
// velocities -1, 0, +1 (Eqs. 57-65 of the reference's applyCollision):
//   zero  = s0 (1 - u^2) - 2u s1 - s2 - K u^2,
//   minus = ((s0 + K)(u^2 - u) + s1 (2u - 1) + s2) / 2,
//   plus  = ((s0 + K)(u^2 + u) + s1 (2u + 1) + s2) / 2.
// mKu2 = -K u^2 of this line's K (a per-cell constant).
template <class R, class Sc>
LBM_HD void bwd(R s0, R s1, R s2, Sc K, R mKu2, const Axis<R>& c, R& lo, R& mid, R& hi) {
    const R h2 = s2 * 0.5f;
    const R sK = K != Sc(0) ? s0 + K : s0;
    lo = fmaR(sK, c.hlo, fmaR(s1, c.um, h2));
    hi = fmaR(sK, c.hhi, fmaR(s1, c.up, h2));
    const R t = K != Sc(0) ? fmaR(s2, -1.f, mKu2) : s2 * -1.f;
    mid = fmaR(s0, c.omu2, fmaR(c.m2u, s1, t));
}

}  // namespace detail

// f: shifted populations, in place.  gx,gy,gz: body force (half applied
// before and half after collision, :70-72 and the sign flip of first-order
// moments before the back transform).  lambda: limiter for this cell (the
// same for both lanes of a Pair).
template <class R>
LBM_HD void collideCumulantT(R (&f)[27], const CollisionConstsT<typename ScalarOf<R>::type>& P,
                             typename ScalarOf<R>::type lambda, typename ScalarOf<R>::type gx,
                             typename ScalarOf<R>::type gy, typename ScalarOf<R>::type gz) {
    using namespace detail;
    using Sc = typename ScalarOf<R>::type;
    constexpr Sc kThird = Frac<Sc>::third, kNinth = Frac<Sc>::ninth, k27th = Frac<Sc>::n27th;
    // m[x][y][z]: after the z stage z holds the moment order, etc.
    R m[3][3][3];
    R zs[3][3], zd[3][3];
    // ---- z stage: populations -> (x,y) lines of z moments ----
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const R pm = f[dirOf(a - 1, b - 1, -1)];
            const R po = f[dirOf(a - 1, b - 1, 0)];
            const R pp = f[dirOf(a - 1, b - 1, 1)];
            zs[a][b] = pp + pm;
            zd[a][b] = pp - pm;
            m[a][b][0] = zs[a][b] + po;
        }
    // density and momentum from the zeroth z moments (:49-69)
    const R dRho = ((m[0][0][0] + m[0][1][0]) + m[0][2][0]) +
                   ((m[1][0][0] + m[1][1][0]) + m[1][2][0]) +
                   ((m[2][0][0] + m[2][1][0]) + m[2][2][0]);
    const R rho = dRho + 1.f;
    const R rhoInv = rcpR(rho);
    const R momX = ((m[2][0][0] + m[2][1][0]) + m[2][2][0]) - ((m[0][0][0] + m[0][1][0]) + m[0][2][0]);
    const R momY = ((m[0][2][0] + m[1][2][0]) + m[2][2][0]) - ((m[0][0][0] + m[1][0][0]) + m[2][0][0]);
    // z momentum: pairs (P - M) summed in the reference's grouping (:62-65)
    const R momZ = (((zd[0][0] + zd[0][1]) + (zd[0][2] + zd[1][0])) + ((zd[1][1] + zd[1][2]) + (zd[2][0] + zd[2][1]))) +
                   zd[2][2];

    const R ux = (momX + 0.5f * gx) * rhoInv;
    const R uy = (momY + 0.5f * gy) * rhoInv;
    const R uz = (momZ + 0.5f * gz) * rhoInv;
    const Axis<R> X = axisOf(ux), Y = axisOf(uy), Z = axisOf(uz);

#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) fwd(zs[a][b], zd[a][b], m[a][b][0], kZ<Sc>(a, b), Z, m[a][b][1], m[a][b][2]);
    // ---- y stage ----
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int n = 0; n < 3; ++n) {
            const R lo = m[a][0][n], mid = m[a][1][n], hi = m[a][2][n];
            const R s = hi + lo;
            const R k0 = s + mid;
            fwd(s, hi - lo, k0, kY<Sc>(a, n), Y, m[a][1][n], m[a][2][n]);
            m[a][0][n] = k0;
        }
    // ---- x stage: central moments k[ord x][ord y][ord z] ----
    R k[3][3][3];
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int n = 0; n < 3; ++n) {
            const R lo = m[0][b][n], mid = m[1][b][n], hi = m[2][b][n];
            const R s = hi + lo;
            const R k0 = (b == 0 && n == 0) ? dRho : s + mid;
            fwd(s, hi - lo, k0, kX<Sc>(b, n), X, k[1][b][n], k[2][b][n]);
            k[0][b][n] = k0;
        }

    // ---- central moments -> cumulants (:164-187) ----
    const R C110 = k[1][1][0], C101 = k[1][0][1], C011 = k[0][1][1];
    const R C200 = k[2][0][0], C020 = k[0][2][0], C002 = k[0][0][2];
    const R C111 = k[1][1][1];
    const R C120 = k[1][2][0], C102 = k[1][0][2], C210 = k[2][1][0];
    const R C012 = k[0][1][2], C201 = k[2][0][1], C021 = k[0][2][1];
    const R dRhoNinth = dRho * rhoInv * kNinth;
    // C211, C121, C112, C220, C022, C202 (:170-187) only enter the reference's
    // relaxation multiplied by (1 - omega6..8) = 0, so they are not formed.
    const R k000 = dRho;

    // ---- relaxation (:193-342); omega2 = omega6 = omega7 = omega8 = 1, so
    // the (1 - omega) terms of those rates vanish and are not evaluated ----
    const R Dxu = P.mHalfW1 * rhoInv * (2.f * C200 - C020 - C002) - 0.5f * rhoInv * (C200 + C020 + C002 - k000);
    const R rw15 = P.w1x15 * rhoInv;
    const R Dyv = fmaR(rw15, C200 - C020, Dxu);
    const R Dzw = fmaR(rw15, C200 - C002, Dxu);
    const R rw3 = P.mW1x3 * rhoInv;
    const R DxvDyu = rw3 * C110;
    const R DxwDzu = rw3 * C101;
    const R DywDzv = rw3 * C011;

    const R Cs110 = P.oneMinusW1 * C110;
    const R Cs101 = P.oneMinusW1 * C101;
    const R Cs011 = P.oneMinusW1 * C011;
    const R r3 = rho * (3.f * P.halfW1c);
    const R xD = X.u2 * Dxu, yD = Y.u2 * Dyv, zD = Z.u2 * Dzw;
    const R e33 = P.oneMinusW1 * (C200 - C020) - r3 * (xD - yD);
    const R e34 = P.oneMinusW1 * (C200 - C002) - r3 * (xD - zD);
    const R e35 = k000 - rho * 1.5f * (xD + yD + zD);
    const R Cs200 = (e33 + e34 + e35) * kThird;
    const R Cs020 = (e34 - 2.f * e33 + e35) * kThird;
    const R Cs002 = (e33 - 2.f * e34 + e35) * kThird;

    R Cs120 = bcast(0.f, dRho), Cs102 = Cs120, Cs210 = Cs120, Cs012 = Cs120, Cs201 = Cs120, Cs021 = Cs120;
    R Cs111 = Cs120, Cs220 = Cs120, Cs202 = Cs120, Cs022 = Cs120, Cs211 = Cs120, Cs121 = Cs120, Cs112 = Cs120;
    const bool k17 = P.useK17 && lambda > Sc(0);
    if (k17) {
        // K17 with limiter: third-order rates pushed from omega3..5 towards 1
        // where the cumulant is large compared with lambda (:270-306)
        const R p1 = C120 + C102, p2 = C210 + C012, p3 = C201 + C021;
        const R q1 = C120 - C102, q2 = C210 - C012, q3 = C201 - C021;
        // 1 - (om + (1 - om) |v| / (lambda + |v|)) applied to v
        auto relax = [&](Sc om, Sc oneMinusOm, R v) {
            const R av = absR(v);
            return (1.f - (om + divFast(oneMinusOm * av, lambda + av))) * v;
        };
        const R e117 = relax(P.omega3, P.oneMinusW3, p1);
        const R e118 = relax(P.omega3, P.oneMinusW3, p2);
        const R e119 = relax(P.omega3, P.oneMinusW3, p3);
        const R e120 = relax(P.omega4, P.oneMinusW4, q1);
        const R e121 = relax(P.omega4, P.oneMinusW4, q2);
        const R e122 = relax(P.omega4, P.oneMinusW4, q3);
        Cs120 = 0.5f * (e120 + e117);
        Cs102 = 0.5f * (e117 - e120);
        Cs210 = 0.5f * (e121 + e118);
        Cs012 = 0.5f * (e118 - e121);
        Cs201 = 0.5f * (e122 + e119);
        Cs021 = 0.5f * (e119 - e122);
        Cs111 = relax(P.omega5, P.oneMinusW5, C111);
        // fourth order (:310-323)
        const R rc43 = rho * P.c43;
        const R e43 = rc43 * (Dxu - 2.f * Dyv + Dzw);
        const R e44 = rc43 * (-2.f * Dxu + Dyv + Dzw);
        const R e45 = rho * P.c45 * (Dxu + Dyv + Dzw);
        Cs220 = (e43 + e44 + e45) * kThird;
        Cs202 = (e45 - e43) * kThird;
        Cs022 = (e45 - e44) * kThird;
        const R rcB = rho * P.cB;
        Cs211 = rcB * DywDzv;
        Cs121 = rcB * DxwDzu;
        Cs112 = rcB * DxvDyu;
    }

    // ---- cumulants -> central moments (:348-384) ----
    R s[3][3][3];
    s[0][1][1] = Cs011; s[1][0][1] = Cs101; s[1][1][0] = Cs110; s[1][1][1] = Cs111;
    s[0][0][2] = Cs002; s[0][2][0] = Cs020; s[2][0][0] = Cs200;
    s[0][1][2] = Cs012; s[0][2][1] = Cs021; s[1][0][2] = Cs102;
    s[2][0][1] = Cs201; s[1][2][0] = Cs120; s[2][1][0] = Cs210;
    s[2][1][1] = fmaR(fmaR(Cs200 + kThird, Cs011, 2.f * Cs101 * Cs110), rhoInv, Cs211);
    s[1][2][1] = fmaR(fmaR(Cs020 + kThird, Cs101, 2.f * Cs110 * Cs011), rhoInv, Cs121);
    s[1][1][2] = fmaR(fmaR(Cs002 + kThird, Cs110, 2.f * Cs011 * Cs101), rhoInv, Cs112);
    s[2][2][0] = Cs220 + (fmaR(fmaR(Cs020, Cs200, 2.f * Cs110 * Cs110), rhoInv, (Cs200 + Cs020) * (kThird * rhoInv)) - dRhoNinth);
    s[0][2][2] = Cs022 + (fmaR(fmaR(Cs002, Cs020, 2.f * Cs011 * Cs011), rhoInv, (Cs002 + Cs020) * (kThird * rhoInv)) - dRhoNinth);
    s[2][0][2] = Cs202 + (fmaR(fmaR(Cs200, Cs002, 2.f * Cs101 * Cs101), rhoInv, (Cs200 + Cs002) * (kThird * rhoInv)) - dRhoNinth);
    if (k17) {
        s[1][2][2] = (Cs020 * Cs102 + Cs002 * Cs120 + 4.f * Cs011 * Cs111 +
                      2.f * (Cs110 * Cs012 + Cs101 * Cs021) + (Cs120 + Cs102) * kThird) * rhoInv;
        s[2][1][2] = (Cs002 * Cs210 + Cs200 * Cs012 + 4.f * Cs101 * Cs111 +
                      2.f * (Cs011 * Cs201 + Cs110 * Cs102) + (Cs210 + Cs012) * kThird) * rhoInv;
        s[2][2][1] = (Cs200 * Cs021 + Cs020 * Cs201 + 4.f * Cs110 * Cs111 +
                      2.f * (Cs101 * Cs120 + Cs011 * Cs210) + (Cs021 + Cs201) * kThird) * rhoInv;
    } else {
        // AllOne: every third-order cumulant is zero, and so are these moments
        s[1][2][2] = Cs120;
        s[2][1][2] = Cs120;
        s[2][2][1] = Cs120;
    }
    {
        const R a200 = Cs200, a020 = Cs020, a002 = Cs002;
        const R a110 = Cs110, a101 = Cs101, a011 = Cs011, a111 = Cs111;
        const R rhoInv2 = rhoInv * rhoInv;
        R lin = a200 * s[0][2][2] + a020 * s[2][0][2] + a002 * s[2][2][0] +
                4.f * (a011 * s[2][1][1] + a101 * s[1][2][1] + a110 * s[1][1][2]);
        if (k17) lin = lin + 4.f * a111 * a111 + 2.f * (Cs120 * Cs102 + Cs210 * Cs012 + Cs201 * Cs021);
        const R cub = 16.f * a110 * a101 * a011 +
                      4.f * (a101 * a101 * a020 + a011 * a011 * a200 + a110 * a110 * a002) +
                      2.f * a200 * a020 * a002;
        const R sq = 2.f * (a101 * a101 + a011 * a011 + a110 * a110) +
                     (a002 * a020 + a002 * a200 + a020 * a200) + (a002 + a020 + a200) * kThird;
        const R fourth = 3.f * (s[0][2][2] + s[2][0][2] + s[2][2][0]) + (a200 + a020 + a002);
        s[2][2][2] = lin * rhoInv - cub * rhoInv2 + fourth * (rhoInv * kNinth) - Frac<Sc>::twoThirds * sq * rhoInv2 -
                     (dRho * dRho - dRho) * (rhoInv2 * k27th);
    }
    s[0][0][0] = k000;
    s[1][0][0] = k[1][0][0] * -1.f;
    s[0][1][0] = k[0][1][0] * -1.f;
    s[0][0][1] = k[0][0][1] * -1.f;

    // ---- back transform, x stage (:390-418): s[ord x][..] -> m[pop x][ord y][ord z]
    {
        const R mK1 = X.u2 * -1.f, mK3 = X.u2 * -kThird, mK9 = X.u2 * -kNinth;
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int n = 0; n < 3; ++n) {
                const Sc K = kX<Sc>(b, n);
                const R mKu2 = (b == 0 && n == 0) ? mK1 : (b == 2 && n == 2) ? mK9 : mK3;
                bwd(s[0][b][n], s[1][b][n], s[2][b][n], K, mKu2, X, m[0][b][n], m[1][b][n], m[2][b][n]);
            }
    }
    // ---- y stage (:420-448)
    {
        const R mKa0 = Y.u2 * -kY<Sc>(0, 0), mKb0 = Y.u2 * -kY<Sc>(1, 0);
        const R mKa2 = Y.u2 * -kY<Sc>(0, 2), mKb2 = Y.u2 * -kY<Sc>(1, 2);
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int n = 0; n < 3; ++n) {
                const Sc K = kY<Sc>(a, n);
                const R mKu2 = n == 0 ? (a == 1 ? mKb0 : mKa0) : (a == 1 ? mKb2 : mKa2);
                const R s0 = m[a][0][n], s1 = m[a][1][n], s2 = m[a][2][n];
                bwd(s0, s1, s2, K, mKu2, Y, m[a][0][n], m[a][1][n], m[a][2][n]);
            }
    }
    // ---- z stage (:450-490): back to populations
    {
        const R mKc = Z.u2 * -kZ<Sc>(1, 1), mKe = Z.u2 * -kZ<Sc>(0, 1), mKv = Z.u2 * -kZ<Sc>(0, 0);
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const Sc K = kZ<Sc>(a, b);
                const R mKu2 = (a == 1 && b == 1) ? mKc : (a == 1 || b == 1) ? mKe : mKv;
                bwd(m[a][b][0], m[a][b][1], m[a][b][2], K, mKu2, Z, f[dirOf(a - 1, b - 1, -1)],
                    f[dirOf(a - 1, b - 1, 0)], f[dirOf(a - 1, b - 1, 1)]);
            }
    }
}

LBM_HD void collideCumulant(float (&f)[27], const CollisionConsts& P, float lambda, float gx, float gy, float gz) {
    collideCumulantT<float>(f, P, lambda, gx, gy, gz);
}

}  // namespace lbm
