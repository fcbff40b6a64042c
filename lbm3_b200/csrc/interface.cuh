// Grid-refinement interface between a coarse level and the next finer one
// (updateInterface, include/updateInterface.h:29-891): fine-to-coarse
// restriction, coarse-to-fine quadratic interpolation and the linear
// fallback for fine cells no full stencil reaches.
//
// Both directions interpolate the same way (Schoenherr 2015, as in the
// reference): each of the 8 cells of a 2x2x2 stencil contributes its density
// deviation, velocity and the non-equilibrium part of its second-order
// moments (Pxy, Pyz, Pxz, Pxx-Pyy, Pxx-Pzz scaled by -3 omega or -1.5 omega,
// i.e. velocity-gradient estimates); from these a velocity field quadratic in
// each coordinate and a trilinear density are fitted over the stencil.  The
// target cell's populations are rebuilt from the fitted density, velocity and
// second-order moments with the higher cumulants at rest (their equilibrium
// values) by the well-conditioned back transform.
//
// Design here: the 8 stencil cells of one interface item are loaded by 8
// lanes of a warp (one cell each, 27 gathers per lane instead of 8 x 27 in
// one thread), and every coefficient of the fit is written as a signed sum
// over the stencil corners, sum_q s(q) v(q) with s a product of the corner's
// axis signs; the sums are formed with three xor-shuffles inside the 8-lane
// group, so every lane holds every coefficient, bit-identical across lanes.
// A fine-to-coarse item then writes its one coarse cell with the 8 lanes
// sharing the 27 stores; a coarse-to-fine item writes 8 fine cells, one per
// lane.
#pragma once

#include "step.cuh"

namespace lbm {
namespace itf {

// Corner q of a 2x2x2 stencil in neighbour-decode order (self, +i, +j, +ij,
// +k, +ik, +jk, +ijk): its sign along each axis relative to the centre.
template <class T> __device__ __forceinline__ T sgnX(int q) { return (q & 1) ? T(1) : T(-1); }
template <class T> __device__ __forceinline__ T sgnY(int q) { return (q & 2) ? T(1) : T(-1); }
template <class T> __device__ __forceinline__ T sgnZ(int q) { return (q & 4) ? T(1) : T(-1); }

// Sum over the 8 lanes of a group (width 8, mask of the group): all lanes get
// the same value (each butterfly step adds the same two partials).
template <class T> __device__ __forceinline__ T groupSum(T v, unsigned mask) {
    v += __shfl_xor_sync(mask, v, 1, 8);
    v += __shfl_xor_sync(mask, v, 2, 8);
    v += __shfl_xor_sync(mask, v, 4, 8);
    return v;
}

// What one stencil cell contributes: density deviation, velocity, and the
// five non-equilibrium second-order moments as gradient estimates.
template <class T> struct CellMoments {
    T d, ux, uy, uz, kxy, kyz, kxz, kxxMyy, kxxMzz;
};

template <class T> __device__ __forceinline__ CellMoments<T> cellMoments(const T (&f)[27], T omega) {
    CellMoments<T> m;
    macroFromF(f, m.d, m.ux, m.uy, m.uz);
    T pxy = T(0), pyz = T(0), pxz = T(0), pxxMyy = T(0), pxxMzz = T(0);
#pragma unroll
    for (int d = 1; d < 27; ++d) {
        const int x = cx(d), y = cy(d), z = cz(d);
        if (x * y) pxy += T(x * y) * f[d];
        if (y * z) pyz += T(y * z) * f[d];
        if (x * z) pxz += T(x * z) * f[d];
        if (x * x - y * y) pxxMyy += T(x * x - y * y) * f[d];
        if (x * x - z * z) pxxMzz += T(x * x - z * z) * f[d];
    }
    const T rho = T(1) + m.d;
    m.kxy = T(-3) * omega * (pxy / rho - m.ux * m.uy);
    m.kyz = T(-3) * omega * (pyz / rho - m.uy * m.uz);
    m.kxz = T(-3) * omega * (pxz / rho - m.ux * m.uz);
    m.kxxMyy = T(-1.5) * omega * (pxxMyy / rho - (m.ux * m.ux - m.uy * m.uy));
    m.kxxMzz = T(-1.5) * omega * (pxxMzz / rho - (m.ux * m.ux - m.uz * m.uz));
    return m;
}

// Coefficients of the fitted fields over a stencil with corners at +-1/2:
//   dRho = d0 + d1 . r + dXY x y + dXZ x z + dYZ y z + dXYZ x y z,
//   u_a = c0[a] + g[a] . r + cXY[a] x y + cXZ[a] x z + cYZ[a] y z
//         + cXYZ[a] x y z + q[a] . (x^2, y^2, z^2).
template <class T> struct Fit {
    T d0, dx, dy, dz, dxy, dxz, dyz, dxyz;
    T c0[3], g[3][3], cxy[3], cxz[3], cyz[3], cxyz[3], q[3][3];
};

// Signed stencil sums of every field this lane's cell holds, and from them
// the fit.  `full` = false forms only what a point at the stencil centre
// needs (value and first derivatives).
template <class T>
__device__ __forceinline__ Fit<T> fitStencil(const CellMoments<T>& m, int lane, unsigned mask, bool full) {
    const T sx = sgnX<T>(lane), sy = sgnY<T>(lane), sz = sgnZ<T>(lane);
    const T u[3] = {m.ux, m.uy, m.uz};
    Fit<T> F;
    // first-order sums over the corners (divided by the 4 corner pairs)
    F.d0 = T(0.125) * groupSum(m.d, mask);
    F.dx = T(0.25) * groupSum(sx * m.d, mask);
    F.dy = T(0.25) * groupSum(sy * m.d, mask);
    F.dz = T(0.25) * groupSum(sz * m.d, mask);
    T su[3], sxy[3], sxz[3], syz[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        su[a] = groupSum(u[a], mask);
        F.g[a][0] = T(0.25) * groupSum(sx * u[a], mask);
        F.g[a][1] = T(0.25) * groupSum(sy * u[a], mask);
        F.g[a][2] = T(0.25) * groupSum(sz * u[a], mask);
        sxy[a] = groupSum(sx * sy * u[a], mask);
        sxz[a] = groupSum(sx * sz * u[a], mask);
        syz[a] = groupSum(sy * sz * u[a], mask);
    }
    // gradient-estimate sums that enter the centre value and the curvature
    const T kxyX = groupSum(sx * m.kxy, mask), kxyY = groupSum(sy * m.kxy, mask);
    const T kxzX = groupSum(sx * m.kxz, mask), kxzZ = groupSum(sz * m.kxz, mask);
    const T kyzY = groupSum(sy * m.kyz, mask), kyzZ = groupSum(sz * m.kyz, mask);
    const T myX = groupSum(sx * m.kxxMyy, mask), myY = groupSum(sy * m.kxxMyy, mask),
            myZ = groupSum(sz * m.kxxMyy, mask);
    const T mzX = groupSum(sx * m.kxxMzz, mask), mzY = groupSum(sy * m.kxxMzz, mask),
            mzZ = groupSum(sz * m.kxxMzz, mask);
    // centre values: the corner mean corrected by the curvature the gradient
    // estimates imply
    F.c0[0] = T(1.0 / 64.0) * (T(2) * (sxy[1] + sxz[2] - kxyY - kxzZ) + T(8) * su[0] - myX - mzX);
    F.c0[1] = T(1.0 / 64.0) * (T(2) * (sxy[0] + syz[2] + myY - kxyX - kyzZ) + T(8) * su[1] - mzY);
    F.c0[2] = T(1.0 / 64.0) * (T(2) * (sxz[0] + syz[1] + mzZ - kxzX - kyzY) + T(8) * su[2] - myZ);
    if (!full) return F;
    F.dxy = T(0.5) * groupSum(sx * sy * m.d, mask);
    F.dxz = T(0.5) * groupSum(sx * sz * m.d, mask);
    F.dyz = T(0.5) * groupSum(sy * sz * m.d, mask);
    F.dxyz = groupSum(sx * sy * sz * m.d, mask);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        F.cxy[a] = T(0.5) * sxy[a];
        F.cxz[a] = T(0.5) * sxz[a];
        F.cyz[a] = T(0.5) * syz[a];
        F.cxyz[a] = groupSum(sx * sy * sz * u[a], mask);
    }
    // curvature q[a][b] = coefficient of x_b^2 in u_a
    F.q[0][0] = T(1.0 / 16.0) * (T(2) * (sxy[1] + sxz[2]) + myX + mzX);
    F.q[1][0] = T(0.125) * (kxyX - T(2) * sxy[0]);
    F.q[2][0] = T(0.125) * (kxzX - T(2) * sxz[0]);
    F.q[0][1] = T(0.125) * (kxyY - T(2) * sxy[1]);
    F.q[1][1] = T(1.0 / 16.0) * (T(2) * (sxy[0] + syz[2] - myY) + mzY);
    F.q[2][1] = T(0.125) * (kyzY - T(2) * syz[1]);
    F.q[0][2] = T(0.125) * (kxzZ - T(2) * sxz[2]);
    F.q[1][2] = T(0.125) * (kyzZ - T(2) * syz[2]);
    F.q[2][2] = T(1.0 / 16.0) * (T(2) * (sxz[0] + syz[1] - mzZ) + myZ);
    return F;
}

// Populations of a cell from density deviation, velocity and the
// second-order central moments k011, k101, k110, k200, k020, k002, with every
// other central moment at its rest value (k220 = k202 = k022 = dRho/9,
// k222 = dRho/27, the rest zero): the back transform x, y, z of the
// well-conditioned cumulant scheme (reconstructInterpolatedF,
// include/updateInterface.h:29-153).
template <class T>
__device__ __forceinline__ void reconstruct(T (&f)[27], T dRho, T ux, T uy, T uz, T k011, T k101, T k110, T k200,
                                            T k020, T k002) {
    using namespace detail;
    T s[3][3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int c = 0; c < 3; ++c) s[a][b][c] = T(0);
    s[0][0][0] = dRho;
    s[2][0][0] = k200;
    s[0][2][0] = k020;
    s[0][0][2] = k002;
    s[1][1][0] = k110;
    s[1][0][1] = k101;
    s[0][1][1] = k011;
    s[2][2][0] = s[2][0][2] = s[0][2][2] = dRho / T(9);
    s[2][2][2] = dRho / T(27);
    const Axis<T> X = axisOf(ux), Y = axisOf(uy), Z = axisOf(uz);
    T m[3][3][3];
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int n = 0; n < 3; ++n) {
            const T K = kX<T>(b, n);
            bwd(s[0][b][n], s[1][b][n], s[2][b][n], K, X.u2 * -K, X, m[0][b][n], m[1][b][n], m[2][b][n]);
        }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int n = 0; n < 3; ++n) {
            const T K = kY<T>(a, n);
            const T s0 = m[a][0][n], s1 = m[a][1][n], s2 = m[a][2][n];
            bwd(s0, s1, s2, K, Y.u2 * -K, Y, m[a][0][n], m[a][1][n], m[a][2][n]);
        }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const T K = kZ<T>(a, b);
            bwd(m[a][b][0], m[a][b][1], m[a][b][2], K, Z.u2 * -K, Z, f[dirOf(a - 1, b - 1, -1)],
                f[dirOf(a - 1, b - 1, 0)], f[dirOf(a - 1, b - 1, 1)]);
        }
}

// Populations of a target cell from its density deviation, velocity and
// velocity gradient G[a][b] = d u_a / d x_b (in units of the stencil
// spacing): the non-equilibrium second-order moments follow from the strain
// rate, rescaled by sigma / omega to the target level (sigma = 2 fine to
// coarse, 1/2 coarse to fine).
template <class T>
__device__ __forceinline__ void populationsFromGradient(T (&f)[27], T dRho, T ux, T uy, T uz, const T (&G)[3][3],
                                                        T sigmaOverOmega) {
    const T rho = T(1) + dRho;
    const T sc = sigmaOverOmega * rho;
    const T k011 = -(T(1) / T(3)) * (G[1][2] + G[2][1]) * sc;
    const T k101 = -(T(1) / T(3)) * (G[0][2] + G[2][0]) * sc;
    const T k110 = -(T(1) / T(3)) * (G[0][1] + G[1][0]) * sc;
    const T mxxMyy = -(T(2) / T(3)) * (G[0][0] - G[1][1]) * sc;
    const T mxxMzz = -(T(2) / T(3)) * (G[0][0] - G[2][2]) * sc;
    const T k200 = (T(1) / T(3)) * (mxxMyy + mxxMzz + dRho);
    const T k020 = (T(1) / T(3)) * (T(-2) * mxxMyy + mxxMzz + dRho);
    const T k002 = (T(1) / T(3)) * (mxxMyy - T(2) * mxxMzz + dRho);
    reconstruct(f, dRho, ux, uy, uz, k011, k101, k110, k200, k020, k002);
}

// Value, velocity and velocity gradient of the fit at r = (x, y, z).
template <class T>
__device__ __forceinline__ void evalFit(const Fit<T>& F, T x, T y, T z, T& dRho, T (&u)[3], T (&G)[3][3]) {
    dRho = F.d0 + F.dx * x + F.dy * y + F.dz * z + F.dxy * x * y + F.dxz * x * z + F.dyz * y * z + F.dxyz * x * y * z;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        u[a] = F.c0[a] + F.g[a][0] * x + F.g[a][1] * y + F.g[a][2] * z + F.cxy[a] * x * y + F.cxz[a] * x * z +
               F.cyz[a] * y * z + F.cxyz[a] * x * y * z + F.q[a][0] * x * x + F.q[a][1] * y * y + F.q[a][2] * z * z;
        G[a][0] = F.g[a][0] + F.cxy[a] * y + F.cxz[a] * z + F.cxyz[a] * y * z + T(2) * F.q[a][0] * x;
        G[a][1] = F.g[a][1] + F.cxy[a] * x + F.cyz[a] * z + F.cxyz[a] * x * z + T(2) * F.q[a][1] * y;
        G[a][2] = F.g[a][2] + F.cxz[a] * x + F.cyz[a] * y + F.cxyz[a] * x * y + T(2) * F.q[a][2] * z;
    }
}

}  // namespace itf
}  // namespace lbm
