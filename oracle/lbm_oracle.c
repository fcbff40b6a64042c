/*
 * lbm_oracle.c — TEST INFRASTRUCTURE ONLY (see lbm_oracle.h).
 *
 * Scalar CPU restatement of the reference time step.  Built with
 * -ffp-contract=off so that every float operation rounds exactly as written.
 * Citations are path:line inside the reference project.
 */
#include "lbm_oracle.h"
#include "oracle_internal.h"
/* generated coefficient tables of the moment-based open boundary (plain C
 * data; pinned against the reference's generated code by the golden vectors) */
#include "../lbm3_b200/csrc/mbbc_tables.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ---- lattice (include/D3Q27Directions.h:8-54) --------------------------- */
enum { OOO, POO, MOO, OOM, OOP, OMO, OPO, POM, MOP, POP, MOM, MMO, PPO, OPM,
       OMP, MPO, PMO, OPP, OMM, MPM, PMP, MMP, PPM, PMM, MPP, MMM, PPP };
static const int CX[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, 0, 0, -1, 1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1};
static const int CY[27] = {0, 0, 0, 0, 0, -1, 1, 0, 0, 0, 0, -1, 1, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1, -1, 1};
static const int CZ[27] = {0, 0, 0, -1, 1, 0, 0, -1, 1, 1, -1, 0, 0, -1, 1, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, -1, 1};
static const int INV[27] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17, 20, 19, 22, 21, 24, 23, 26, 25};
static const float W[27] = {8.f / 27.f, 2.f / 27.f, 2.f / 27.f, 2.f / 27.f, 2.f / 27.f, 2.f / 27.f, 2.f / 27.f,
                            1.f / 54.f, 1.f / 54.f, 1.f / 54.f, 1.f / 54.f, 1.f / 54.f, 1.f / 54.f, 1.f / 54.f,
                            1.f / 54.f, 1.f / 54.f, 1.f / 54.f, 1.f / 54.f, 1.f / 54.f, 1.f / 216.f, 1.f / 216.f,
                            1.f / 216.f, 1.f / 216.f, 1.f / 216.f, 1.f / 216.f, 1.f / 216.f, 1.f / 216.f};

/* Neighbour slot used by the esotwist pre/post maps: 0 self, 1 iPlus, 2 jPlus,
 * 3 ijPlus, 4 kPlus, 5 ikPlus, 6 jkPlus, 7 ijkPlus
 * (include/esotwistStreamingFunctions.h:17-127). */
static int pre_nbr(int d) { return (CX[d] < 0) | ((CY[d] < 0) << 1) | ((CZ[d] < 0) << 2); }
static int post_nbr(int d) { return (CX[d] > 0) | ((CY[d] > 0) << 1) | ((CZ[d] > 0) << 2); }

int oracle_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void oracle_default_bc(obc* bc) {
    memset(bc, 0, sizeof(*bc));
    bc->wallID = -1;
    bc->useIBB = 1;
    bc->nonReflective = 1;
    bc->nonReflectiveBeta = 7.f;
    bc->collisionLimiter = 0.05f;
    bc->nuMultiplier = 1.f;
}

/* ---- getFeq / getDRhoUxUyUz -------------------------------------------- */
void oracle_get_feq(float dRho, float ux, float uy, float uz, float feq[27]) {
    const float ux2 = ux * ux, uy2 = uy * uy, uz2 = uz * uz;
    for (int q = 0; q < 27; ++q) {
        const float cx = (float)CX[q], cy = (float)CY[q], cz = (float)CZ[q];
        const float dx = 3.f * cx * ux + (4.5f * cx * cx - 1.5f) * ux2;
        const float dy = 3.f * cy * uy + (4.5f * cy * cy - 1.5f) * uy2;
        const float dz = 3.f * cz * uz + (4.5f * cz * cz - 1.5f) * uz2;
        const float xy = dx + dy + dx * dy;
        const float corr = xy + dz + xy * dz;
        feq[q] = W[q] * ((dRho + corr) + dRho * corr);
    }
}

void oracle_get_drho_u(const float f[27], float out[4]) {
    const float d = (((f[PPP] + f[MMM]) + (f[PMP] + f[MPM])) + ((f[PPM] + f[MMP]) + (f[PMM] + f[MPP]))) +
                    (((f[OPP] + f[OMM]) + (f[OPM] + f[OMP])) + ((f[POP] + f[MOM]) + (f[POM] + f[MOP])) +
                     ((f[PPO] + f[MMO]) + (f[PMO] + f[MPO]))) +
                    ((f[POO] + f[MOO]) + (f[OPO] + f[OMO]) + (f[OOP] + f[OOM])) + f[OOO];
    const float ri = 1.f / (d + 1.f);
    const float mx = ((((f[PPP] - f[MMM]) + (f[PMP] - f[MPM])) + ((f[PPM] - f[MMP]) + (f[PMM] - f[MPP]))) +
                      (((f[POP] - f[MOM]) + (f[POM] - f[MOP])) + ((f[PPO] - f[MMO]) + (f[PMO] - f[MPO]))) +
                      (f[POO] - f[MOO]));
    const float my = ((((f[PPP] - f[MMM]) - (f[PMP] - f[MPM])) + ((f[PPM] - f[MMP]) - (f[PMM] - f[MPP]))) +
                      (((f[OPP] - f[OMM]) + (f[OPM] - f[OMP])) + ((f[PPO] - f[MMO]) - (f[PMO] - f[MPO]))) +
                      (f[OPO] - f[OMO]));
    const float mz = ((((f[PPP] - f[MMM]) + (f[PMP] - f[MPM])) - ((f[PPM] - f[MMP]) + (f[PMM] - f[MPP]))) +
                      (((f[OPP] - f[OMM]) - (f[OPM] - f[OMP])) + ((f[POP] - f[MOM]) - (f[POM] - f[MOP]))) +
                      (f[OOP] - f[OOM]));
    out[0] = d;
    out[1] = mx * ri;
    out[2] = my * ri;
    out[3] = mz * ri;
}

/* ---- applyCollision ------------------------------------------------------
 * Variables are named after their (x,y,z) index; population lines use
 * a/b/c for -1/0/+1 and moments use 0/1/2 for the order, as in Geier 2017. */

/* population index of (x,y,z) in {0,1,2}^3 meaning {-1,0,+1} */
static const int PIDX[3][3][3] = {{{25, 11, 21}, {10, 2, 8}, {19, 15, 24}},
                                  {{18, 5, 14}, {3, 0, 4}, {13, 6, 17}},
                                  {{23, 16, 20}, {7, 1, 9}, {22, 12, 26}}};
#define pidx(x, y, z) PIDX[x][y][z]

/* weight moments (include/applyCollision.h:24-38) */
static float kw_z(int x, int y) {
    static const float t[3][3] = {{1.f / 36.f, 1.f / 9.f, 1.f / 36.f},
                                  {1.f / 9.f, 4.f / 9.f, 1.f / 9.f},
                                  {1.f / 36.f, 1.f / 9.f, 1.f / 36.f}};
    return t[x][y];
}
static float kw_y(int x, int zord) {
    if (zord == 1) return 0.f;
    if (zord == 0) return x == 1 ? 2.f / 3.f : 1.f / 6.f;
    return x == 1 ? 2.f / 9.f : 1.f / 18.f;
}

/* Back transform of the well-conditioned scheme (applyCollision.h:390-490):
 * central moments s[order x][order y][order z] about u -> shifted populations. */
static void back_transform(float s[3][3][3], float ux, float uy, float uz, float f[27]) {
    const float ux2 = ux * ux, uy2 = uy * uy, uz2 = uz * uz;
    /* back transform x (:390-418): X[x line][order y][order z] */
    float X[3][3][3];
    for (int m = 0; m < 3; ++m)
        for (int n = 0; n < 3; ++n) {
            const float s0 = s[0][m][n], s1 = s[1][m][n], s2 = s[2][m][n];
            float K = 0.f, centre = s0 * (1.f - ux2) - 2.f * ux * s1 - s2;
            if (m == 0 && n == 0) { K = 1.f; centre = centre - ux2; }
            else if ((m == 0 && n == 2) || (m == 2 && n == 0)) { K = 1.f / 3.f; centre = centre - ux2 / 3.f; }
            else if (m == 2 && n == 2) { K = 1.f / 9.f; centre = centre - ux2 / 9.f; }
            X[1][m][n] = centre;
            if (K != 0.f) {
                X[0][m][n] = ((s0 + K) * (ux2 - ux) + s1 * (2.f * ux - 1.f) + s2) * 0.5f;
                X[2][m][n] = ((s0 + K) * (ux2 + ux) + s1 * (2.f * ux + 1.f) + s2) * 0.5f;
            } else {
                X[0][m][n] = (s0 * (ux2 - ux) + s1 * (2.f * ux - 1.f) + s2) * 0.5f;
                X[2][m][n] = (s0 * (ux2 + ux) + s1 * (2.f * ux + 1.f) + s2) * 0.5f;
            }
        }
    /* back transform y (:420-448): V[x line][y line][order z] */
    float V[3][3][3];
    for (int x = 0; x < 3; ++x)
        for (int n = 0; n < 3; ++n) {
            const float s0 = X[x][0][n], s1 = X[x][1][n], s2 = X[x][2][n];
            if (n == 1) {
                V[x][1][n] = s0 * (1.f - uy2) - 2.f * uy * s1 - s2;
                V[x][0][n] = (s0 * (uy2 - uy) + s1 * (2.f * uy - 1.f) + s2) * 0.5f;
                V[x][2][n] = (s0 * (uy2 + uy) + s1 * (2.f * uy + 1.f) + s2) * 0.5f;
            } else {
                const float K = kw_y(x, n);
                V[x][1][n] = s0 * (1.f - uy2) - 2.f * uy * s1 - s2 - K * uy2;
                V[x][0][n] = ((s0 + K) * (uy2 - uy) + s1 * (2.f * uy - 1.f) + s2) * 0.5f;
                V[x][2][n] = ((s0 + K) * (uy2 + uy) + s1 * (2.f * uy + 1.f) + s2) * 0.5f;
            }
        }
    /* back transform z (:450-490) */
    for (int x = 0; x < 3; ++x)
        for (int y = 0; y < 3; ++y) {
            const float s0 = V[x][y][0], s1 = V[x][y][1], s2 = V[x][y][2];
            const float K = kw_z(x, y);
            f[pidx(x, y, 1)] = s0 * (1.f - uz2) - 2.f * uz * s1 - s2 - K * uz2;
            f[pidx(x, y, 0)] = ((s0 + K) * (uz2 - uz) + s1 * (2.f * uz - 1.f) + s2) * 0.5f;
            f[pidx(x, y, 2)] = ((s0 + K) * (uz2 + uz) + s1 * (2.f * uz + 1.f) + s2) * 0.5f;
        }
}

void oracle_apply_collision(float f[27], const obc* bc, float nu) {
    const float gx = bc->gx, gy = bc->gy, gz = bc->gz;
    float A0[3][3]; /* zeroth z moment of line (x,y): k_xy0 */
    for (int x = 0; x < 3; ++x)
        for (int y = 0; y < 3; ++y)
            A0[x][y] = (f[pidx(x, y, 2)] + f[pidx(x, y, 0)]) + f[pidx(x, y, 1)];

    /* :49-56 */
    const float dRho = ((A0[0][0] + A0[0][1]) + A0[0][2]) + ((A0[1][0] + A0[1][1]) + A0[1][2]) +
                       ((A0[2][0] + A0[2][1]) + A0[2][2]);
    const float rho = 1.f + dRho;
    const float rhoInv = 1.f / rho;
    /* :59-65 */
    const float momX = ((A0[2][0] + A0[2][1]) + A0[2][2]) - ((A0[0][0] + A0[0][1]) + A0[0][2]);
    const float momY = ((A0[0][2] + A0[1][2]) + A0[2][2]) - ((A0[0][0] + A0[1][0]) + A0[2][0]);
    const float momZ = (((f[MMP] - f[MMM]) + (f[MOP] - f[MOM])) + ((f[MPP] - f[MPM]) + (f[OMP] - f[OMM]))) +
                       (((f[OOP] - f[OOM]) + (f[OPP] - f[OPM])) + ((f[PMP] - f[PMM]) + (f[POP] - f[POM]))) +
                       (f[PPP] - f[PPM]);
    /* :70-72 */
    const float ux = (momX + 0.5f * gx) * rhoInv;
    const float uy = (momY + 0.5f * gy) * rhoInv;
    const float uz = (momZ + 0.5f * gz) * rhoInv;
    const float ux2 = ux * ux, uy2 = uy * uy, uz2 = uz * uz;

    /* z transform (:82-100): Z[x][y][order] */
    float Z[3][3][3];
    for (int x = 0; x < 3; ++x)
        for (int y = 0; y < 3; ++y) {
            const float p = f[pidx(x, y, 2)], m = f[pidx(x, y, 0)];
            const float K = kw_z(x, y);
            Z[x][y][0] = A0[x][y];
            Z[x][y][1] = (p - m) - uz * (A0[x][y] + K);
            Z[x][y][2] = (p + m) - 2.f * uz * (p - m) + uz2 * (A0[x][y] + K);
        }
    /* y transform (:102-130): Y[x][order y][order z] */
    float Y[3][3][3];
    for (int x = 0; x < 3; ++x)
        for (int n = 0; n < 3; ++n) {
            const float a = Z[x][0][n], b = Z[x][1][n], c = Z[x][2][n];
            const float K = kw_y(x, n);
            const float s0 = (c + a) + b;
            Y[x][0][n] = s0;
            if (n == 1) {
                Y[x][1][n] = (c - a) - uy * s0;
                Y[x][2][n] = (c + a) - 2.f * uy * (c - a) + uy2 * s0;
            } else {
                Y[x][1][n] = (c - a) - uy * (s0 + K);
                Y[x][2][n] = (c + a) - 2.f * uy * (c - a) + uy2 * (s0 + K);
            }
        }
    /* x transform (:134-159): k[order x][order y][order z] */
    float k[3][3][3];
    memset(k, 0, sizeof(k));
    for (int m = 0; m < 3; ++m)
        for (int n = 0; n < 3; ++n) {
            const float a = Y[0][m][n], b = Y[1][m][n], c = Y[2][m][n];
            const float s0 = (m == 0 && n == 0) ? dRho : (c + a) + b;
            k[0][m][n] = s0;
            float K = 0.f;
            int hasK = 0;
            if (m == 0 && n == 0) { K = 1.f; hasK = 1; }
            else if ((m == 0 && n == 2) || (m == 2 && n == 0)) { K = 1.f / 3.f; hasK = 1; }
            else if (m == 2 && n == 2) { K = 1.f / 9.f; hasK = 1; }
            if (hasK) {
                k[1][m][n] = (c - a) - ux * (s0 + K);
                k[2][m][n] = (c + a) - 2.f * ux * (c - a) + ux2 * (s0 + K);
            } else {
                k[1][m][n] = (c - a) - ux * s0;
                k[2][m][n] = (c + a) - 2.f * ux * (c - a) + ux2 * s0;
            }
        }

    /* cumulants (:164-187) */
    const float C110 = k[1][1][0], C101 = k[1][0][1], C011 = k[0][1][1];
    const float C200 = k[2][0][0], C020 = k[0][2][0], C002 = k[0][0][2];
    const float C111 = k[1][1][1];
    const float C120 = k[1][2][0], C102 = k[1][0][2], C210 = k[2][1][0];
    const float C012 = k[0][1][2], C201 = k[2][0][1], C021 = k[0][2][1];
    const float C211 = k[2][1][1] - ((k[2][0][0] + 1.f / 3.f) * k[0][1][1] + 2.f * k[1][0][1] * k[1][1][0]) * rhoInv;
    const float C121 = k[1][2][1] - ((k[0][2][0] + 1.f / 3.f) * k[1][0][1] + 2.f * k[1][1][0] * k[0][1][1]) * rhoInv;
    const float C112 = k[1][1][2] - ((k[0][0][2] + 1.f / 3.f) * k[1][1][0] + 2.f * k[0][1][1] * k[1][0][1]) * rhoInv;
    const float C220 = k[2][2][0] - ((k[0][2][0] * k[2][0][0] + 2.f * k[1][1][0] * k[1][1][0] +
                                      (k[2][0][0] + k[0][2][0]) / 3.f) * rhoInv - dRho * rhoInv / 9.f);
    const float C022 = k[0][2][2] - ((k[0][0][2] * k[0][2][0] + 2.f * k[0][1][1] * k[0][1][1] +
                                      (k[0][0][2] + k[0][2][0]) / 3.f) * rhoInv - dRho * rhoInv / 9.f);
    const float C202 = k[2][0][2] - ((k[2][0][0] * k[0][0][2] + 2.f * k[1][0][1] * k[1][0][1] +
                                      (k[2][0][0] + k[0][0][2]) / 3.f) * rhoInv - dRho * rhoInv / 9.f);
    const float k000 = dRho;

    /* relaxation (:193-342) */
    const float w1 = 1.f / (3.f * (nu * bc->nuMultiplier) + 0.5f);
    const float w2 = 1.f;
    const float Dxu = -w1 * 0.5f * rhoInv * (2.f * C200 - C020 - C002) - w2 * 0.5f * rhoInv * (C200 + C020 + C002 - k000);
    const float Dyv = Dxu + 1.5f * w1 * rhoInv * (C200 - C020);
    const float Dzw = Dxu + 1.5f * w1 * rhoInv * (C200 - C002);
    const float DxvDyu = -3.f * w1 * rhoInv * C110;
    const float DxwDzu = -3.f * w1 * rhoInv * C101;
    const float DywDzv = -3.f * w1 * rhoInv * C011;
    const float S110 = (1.f - w1) * C110, S101 = (1.f - w1) * C101, S011 = (1.f - w1) * C011;
    const float r33 = (1.f - w1) * (C200 - C020) - 3.f * rho * (1.f - 0.5f * w1) * (ux2 * Dxu - uy2 * Dyv);
    const float r34 = (1.f - w1) * (C200 - C002) - 3.f * rho * (1.f - 0.5f * w1) * (ux2 * Dxu - uz2 * Dzw);
    const float r35 = k000 * w2 + (1.f - w2) * (C200 + C020 + C002) -
                      3.f * rho * (1.f - 0.5f * w2) * (ux2 * Dxu + uy2 * Dyv + uz2 * Dzw);
    const float S200 = (r33 + r34 + r35) / 3.f;
    const float S020 = (r34 - 2.f * r33 + r35) / 3.f;
    const float S002 = (r33 - 2.f * r34 + r35) / 3.f;

    float S120 = 0.f, S102 = 0.f, S210 = 0.f, S012 = 0.f, S201 = 0.f, S021 = 0.f, S111 = 0.f;
    float S220 = 0.f, S202 = 0.f, S022 = 0.f, S211 = 0.f, S121 = 0.f, S112 = 0.f;
    const float w6 = 1.f, w7 = 1.f, w8 = 1.f;
    if (bc->collisionLimiter > 0.f && bc->nuMultiplier <= 1.f) {
        const float w3 = 8.f * (w1 - 2.f) * (w2 * (3.f * w1 - 1.f) - 5.f * w1) /
                         (8.f * (5.f - 2.f * w1) * w1 + w2 * (8.f + w1 * (9.f * w1 - 26.f)));
        const float w4 = 8.f * (w1 - 2.f) * (w1 + w2 * (3.f * w1 - 7.f)) /
                         (w2 * (56.f - 42.f * w1 + 9.f * w1 * w1) - 8.f * w1);
        const float w5 = 24.f * (w1 - 2.f) *
                         (4.f * w1 * w1 + w1 * w2 * (18.f - 13.f * w1) + w2 * w2 * (2.f + w1 * (6.f * w1 - 11.f))) /
                         (16.f * w1 * w1 * (w1 - 6.f) - 2.f * w1 * w2 * (216.f + 5.f * w1 * (9.f * w1 - 46.f)) +
                          w2 * w2 * (w1 * (3.f * w1 - 10.f) * (15.f * w1 - 28.f) - 48.f));
        const float A = (4.f * w1 * w1 + 2.f * w1 * w2 * (w1 - 6.f) + w2 * w2 * (w1 * (10.f - 3.f * w1) - 4.f)) /
                        ((w1 - w2) * (w2 * (2.f + 3.f * w1) - 8.f * w1));
        const float B = (4.f * w1 * w2 * (9.f * w1 - 16.f) - 4.f * w1 * w1 - 2.f * w2 * w2 * (2.f + 9.f * w1 * (w1 - 2.f))) /
                        (3.f * (w1 - w2) * (w2 * (2.f + 3.f * w1) - 8.f * w1));
        const float lam = bc->collisionLimiter;
        const float P1 = C120 + C102, P2 = C210 + C012, P3 = C201 + C021;
        const float M1 = C120 - C102, M2 = C210 - C012, M3 = C201 - C021;
        const float aP1 = fabsf(P1), aP2 = fabsf(P2), aP3 = fabsf(P3);
        const float aM1 = fabsf(M1), aM2 = fabsf(M2), aM3 = fabsf(M3), a111 = fabsf(C111);
        const float oP1 = w3 + (1.f - w3) * aP1 / (lam + aP1);
        const float oP2 = w3 + (1.f - w3) * aP2 / (lam + aP2);
        const float oP3 = w3 + (1.f - w3) * aP3 / (lam + aP3);
        const float oM1 = w4 + (1.f - w4) * aM1 / (lam + aM1);
        const float oM2 = w4 + (1.f - w4) * aM2 / (lam + aM2);
        const float oM3 = w4 + (1.f - w4) * aM3 / (lam + aM3);
        const float o111 = w5 + (1.f - w5) * a111 / (lam + a111);
        const float e117 = (1.f - oP1) * P1, e118 = (1.f - oP2) * P2, e119 = (1.f - oP3) * P3;
        const float e120 = (1.f - oM1) * M1, e121 = (1.f - oM2) * M2, e122 = (1.f - oM3) * M3;
        S120 = 0.5f * (e120 + e117);
        S102 = 0.5f * (-e120 + e117);
        S210 = 0.5f * (e121 + e118);
        S012 = 0.5f * (-e121 + e118);
        S201 = 0.5f * (e122 + e119);
        S021 = 0.5f * (-e122 + e119);
        S111 = (1.f - o111) * C111;
        const float e43 = (2.f / 3.f) * (1.f / w1 - 0.5f) * w6 * A * rho * (Dxu - 2.f * Dyv + Dzw) +
                          (1.f - w6) * (C220 - 2.f * C202 + C022);
        const float e44 = (2.f / 3.f) * (1.f / w1 - 0.5f) * w6 * A * rho * (-2.f * Dxu + Dyv + Dzw) +
                          (1.f - w6) * (C220 + C202 - 2.f * C022);
        const float e45 = -(4.f / 3.f) * (1.f / w1 - 0.5f) * w7 * A * rho * (Dxu + Dyv + Dzw) +
                          (1.f - w7) * (C220 + C202 + C022);
        S220 = (e43 + e44 + e45) / 3.f;
        S202 = (-e43 + e45) / 3.f;
        S022 = (-e44 + e45) / 3.f;
        S211 = -(1.f / 3.f) * (1.f / w1 - 0.5f) * w8 * B * rho * DywDzv + (1.f - w8) * C211;
        S121 = -(1.f / 3.f) * (1.f / w1 - 0.5f) * w8 * B * rho * DxwDzu + (1.f - w8) * C121;
        S112 = -(1.f / 3.f) * (1.f / w1 - 0.5f) * w8 * B * rho * DxvDyu + (1.f - w8) * C112;
    }

    /* cumulants -> central moments (:348-384) */
    float s[3][3][3];
    s[0][1][1] = S011; s[1][0][1] = S101; s[1][1][0] = S110; s[1][1][1] = S111;
    s[0][0][2] = S002; s[0][2][0] = S020; s[2][0][0] = S200;
    s[0][1][2] = S012; s[0][2][1] = S021; s[1][0][2] = S102; s[2][0][1] = S201;
    s[1][2][0] = S120; s[2][1][0] = S210;
    s[2][1][1] = S211 + ((S200 + 1.f / 3.f) * S011 + 2.f * S101 * S110) * rhoInv;
    s[1][2][1] = S121 + ((S020 + 1.f / 3.f) * S101 + 2.f * S110 * S011) * rhoInv;
    s[1][1][2] = S112 + ((S002 + 1.f / 3.f) * S110 + 2.f * S011 * S101) * rhoInv;
    s[2][2][0] = S220 + ((S020 * S200 + 2.f * S110 * S110 + (S200 + S020) / 3.f) * rhoInv - dRho * rhoInv / 9.f);
    s[0][2][2] = S022 + ((S002 * S020 + 2.f * S011 * S011 + (S002 + S020) / 3.f) * rhoInv - dRho * rhoInv / 9.f);
    s[2][0][2] = S202 + ((S200 * S002 + 2.f * S101 * S101 + (S200 + S002) / 3.f) * rhoInv - dRho * rhoInv / 9.f);
    s[1][2][2] = (S020 * S102 + S002 * S120 + 4.f * S011 * S111 + 2.f * (S110 * S012 + S101 * S021) +
                  (S120 + S102) / 3.f) * rhoInv;
    s[2][1][2] = (S002 * S210 + S200 * S012 + 4.f * S101 * S111 + 2.f * (S011 * S201 + S110 * S102) +
                  (S210 + S012) / 3.f) * rhoInv;
    s[2][2][1] = (S200 * S021 + S020 * S201 + 4.f * S110 * S111 + 2.f * (S101 * S120 + S011 * S210) +
                  (S021 + S201) / 3.f) * rhoInv;
    s[2][2][2] = (4.f * S111 * S111 + S200 * s[0][2][2] + S020 * s[2][0][2] + S002 * s[2][2][0] +
                  4.f * (S011 * s[2][1][1] + S101 * s[1][2][1] + S110 * s[1][1][2]) +
                  2.f * (S120 * S102 + S210 * S012 + S201 * S021)) * rhoInv -
                 (16.f * S110 * S101 * S011 + 4.f * (S101 * S101 * S020 + S011 * S011 * S200 + S110 * S110 * S002) +
                  2.f * S200 * S020 * S002) * rhoInv * rhoInv +
                 (3.f * (s[0][2][2] + s[2][0][2] + s[2][2][0]) + (S200 + S020 + S002)) * rhoInv / 9.f -
                 (2.f / 3.f) * (2.f * (S101 * S101 + S011 * S011 + S110 * S110) + (S002 * S020 + S002 * S200 + S020 * S200) +
                                (S002 + S020 + S200) / 3.f) * rhoInv * rhoInv -
                 (dRho * dRho - dRho) * rhoInv * rhoInv / 27.f;
    s[0][0][0] = k000;
    s[1][0][0] = -k[1][0][0];
    s[0][1][0] = -k[0][1][0];
    s[0][0][1] = -k[0][0][1];

    back_transform(s, ux, uy, uz, f);
}

void oracle_apply_collision_batch(float* f, int n, float nu, float limiter, float nuMultiplier, float gx,
                                  float gy, float gz) {
    obc bc;
    oracle_default_bc(&bc);
    bc.collisionLimiter = limiter;
    bc.nuMultiplier = nuMultiplier;
    bc.gx = gx; bc.gy = gy; bc.gz = gz;
#pragma omp parallel for schedule(static)
    for (int c = 0; c < n; ++c) {
        float v[27];
        for (int d = 0; d < 27; ++d) v[d] = f[(long long)d * n + c];
        oracle_apply_collision(v, &bc, nu);
        for (int d = 0; d < 27; ++d) f[(long long)d * n + c] = v[d];
    }
}

/* ---- moment-based open boundary ------------------------------------------ */

static const LbmMbbcTable* mbbc_table(int code) {
    for (int t = 0; t < LBM_MBBC_NORMALS; ++t)
        if (kLbmMbbc[t].code == code) return &kLbmMbbc[t];
    return NULL;
}

/* acc + c v, written as the generated code writes each term */
static float mbbc_term(float acc, float c, float v) {
    if (c == 1.f) return acc + v;
    if (c == -1.f) return acc - v;
    return acc + c * v;
}

/* equilibrium moment m of the 23 in table order (helperMain.py meq) */
static float mbbc_meq(int m, float rho, float ux, float uy, float uz) {
    const float t = 1.f / 3.f, n = 1.f / 9.f;
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
        case 10: return 0.f;
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

/* applyMBBC: unknowns = (S Mfu)^-1 (m_eq(S) - S Mfk f_k) */
int oracle_mbbc_apply(int code, float rho, float ux, float uy, float uz, float f[27]) {
    const LbmMbbcTable* T = mbbc_table(code);
    if (!T) return -1;
    float s[LBM_MBBC_MAX_UNKNOWN];
    for (int i = 0; i < T->nu; ++i) {
        float smf = 0.f;
        for (int k = 0; k < T->nk; ++k)
            if (T->smfk[i][k] != 0) smf = mbbc_term(smf, (float)T->smfk[i][k], f[T->known[k]]);
        s[i] = mbbc_meq(T->moment[i], rho, ux, uy, uz) - smf;
    }
    float out[LBM_MBBC_MAX_UNKNOWN];
    for (int r = 0; r < T->nu; ++r) {
        float v = 0.f;
        for (int j = 0; j < T->nu; ++j)
            if (T->inv[r][j] != 0.f) v = mbbc_term(v, T->inv[r][j], s[j]);
        out[r] = v;
    }
    for (int r = 0; r < T->nu; ++r) f[T->unknown[r]] = out[r];
    return 0;
}

/* restoreRho: rho = (C Mfk f_k) / (C Q + C Qu u) */
int oracle_mbbc_restore_rho(int code, float ux, float uy, float uz, const float f[27], float* rho) {
    const LbmMbbcTable* T = mbbc_table(code);
    if (!T) return -1;
    const float scqu = T->rhoQu[0] * ux + T->rhoQu[1] * uy + T->rhoQu[2] * uz;
    const float sden = T->rhoQ + scqu;
    float scmf = 0.f;
    for (int k = 0; k < T->nk; ++k)
        if (T->rhoMfk[k] != 0.f) scmf = mbbc_term(scmf, T->rhoMfk[k], f[T->known[k]]);
    *rho = scmf / sden;
    return 0;
}

/* restoreUxUyUz: faces by the closed form (normal velocity from the
 * known-population density, tangential from a vanishing k_nnt), edges and
 * corners from three unknown-free moment relations */
int oracle_mbbc_restore_u(int code, float rho, const float f[27], float u[3]) {
    const LbmMbbcTable* T = mbbc_table(code);
    if (!T) return -1;
    const int n[3] = {code / 100 - 5, (code / 10) % 10 - 5, code % 10 - 5};
    if (T->face) {
        float fZero = 0.f, fPlus = 0.f;
        for (int d = 0; d < 27; ++d) {
            const int cn = CX[d] * n[0] + CY[d] * n[1] + CZ[d] * n[2];
            if (cn == 0) fZero = fZero + f[d];
            else if (cn == 1) fPlus = fPlus + f[d];
        }
        const float uN = (fZero + 2.f * fPlus) / rho - 1.f;
        const float den = fZero + 2.f * (uN + 1.f) * rho * uN;
        for (int a = 0; a < 3; ++a) {
            if (n[a] != 0) { u[a] = n[a] > 0 ? uN : -uN; continue; }
            float jZero = 0.f, jPlus = 0.f;
            for (int d = 0; d < 27; ++d) {
                const int cn = CX[d] * n[0] + CY[d] * n[1] + CZ[d] * n[2];
                const int ca = a == 0 ? CX[d] : (a == 1 ? CY[d] : CZ[d]);
                if (ca == 0) continue;
                if (cn == 0) jZero = ca > 0 ? jZero + f[d] : jZero - f[d];
                else if (cn == 1) jPlus = ca > 0 ? jPlus + f[d] : jPlus - f[d];
            }
            u[a] = ((2.f * uN + 1.f) * jZero + 4.f * uN * jPlus) / den;
        }
        return 0;
    }
    float s[3];
    for (int i = 0; i < 3; ++i) {
        float acc = 0.f;
        for (int k = 0; k < T->nk; ++k)
            if (T->uMfk[i][k] != 0.f) acc = mbbc_term(acc, T->uMfk[i][k], f[T->known[k]]);
        s[i] = acc / rho - T->uQ[i];
    }
    for (int a = 0; a < 3; ++a) {
        float v = 0.f;
        for (int j = 0; j < 3; ++j)
            if (T->uInv[a][j] != 0.f) v = mbbc_term(v, T->uInv[a][j], s[j]);
        u[a] = v;
    }
    return 0;
}

/* ---- grid construction (include/gridBuilderFunctions.h) ------------------ */

static obc open_bc_faces(const lbm_face_bc* face, const ogrid* g, int i, int j, int k) {
    /* getOpenBC as the face table defines it (include/lbm3_b200.h) */
    obc bc;
    oracle_default_bc(&bc);
    const int touch[6] = {i == 0, i == g->nx - 1, j == 0, j == g->ny - 1, k == 0, k == g->nz - 1};
    int best = -1;
    for (int f = 0; f < 6; ++f)
        if (touch[f] && (best < 0 || face[f].priority > face[best].priority)) best = f;
    if (best < 0) return bc;
    const lbm_face_bc* fb = &face[best];
    bc.openBCID = fb->open_bc_id;
    bc.nonReflective = fb->non_reflective;
    bc.nonReflectiveBeta = fb->non_reflective_beta;
    if (fb->kind == LBM_BC_PERIODIC) bc.periodic = 1;
    else if (fb->kind == LBM_BC_VELOCITY) { bc.dirichletU = 1; bc.ux = fb->ux; bc.uy = fb->uy; bc.uz = fb->uz; }
    else if (fb->kind == LBM_BC_PRESSURE) { bc.dirichletRho = 1; bc.dRho = fb->dRho; }
    return bc;
}

/* A driver hook (getOpenBC / getInitialCondition / getLocalBC) on a
 * BCStruct that starts from `bc`, with the level's info. */
static obc call_hook(lbm_cell_hook hook, void* user, obc bc, const ogrid* g, int i, int j, int k) {
    lbm_bc h;
    h.dRho = bc.dRho; h.ux = bc.ux; h.uy = bc.uy; h.uz = bc.uz;
    h.gx = bc.gx; h.gy = bc.gy; h.gz = bc.gz;
    h.wallID = bc.wallID; h.openBCID = bc.openBCID;
    h.useIBB = bc.useIBB; h.dirichletU = bc.dirichletU; h.dirichletRho = bc.dirichletRho;
    h.periodic = bc.periodic; h.nonReflective = bc.nonReflective;
    h.nonReflectiveBeta = bc.nonReflectiveBeta; h.collisionLimiter = bc.collisionLimiter;
    h.nuMultiplier = bc.nuMultiplier;
    lbm_grid_info info;
    memset(&info, 0, sizeof(info));
    info.grid_id = g->gridID;
    info.cell_count = g->cellCount;
    info.cell_count_x = g->nx; info.cell_count_y = g->ny; info.cell_count_z = g->nz;
    info.res = g->res; info.ox = g->ox; info.oy = g->oy; info.oz = g->oz;
    info.nu = g->nu; info.dt_phys = g->dtPhys;
    info.iterations_finished = g->iterationsFinished;
    hook(user, &h, i, j, k, &info);
    obc r;
    r.dRho = h.dRho; r.ux = h.ux; r.uy = h.uy; r.uz = h.uz;
    r.gx = h.gx; r.gy = h.gy; r.gz = h.gz;
    r.wallID = h.wallID; r.openBCID = h.openBCID;
    r.useIBB = h.useIBB != 0; r.dirichletU = h.dirichletU != 0; r.dirichletRho = h.dirichletRho != 0;
    r.periodic = h.periodic != 0; r.nonReflective = h.nonReflective != 0;
    r.nonReflectiveBeta = h.nonReflectiveBeta; r.collisionLimiter = h.collisionLimiter;
    r.nuMultiplier = h.nuMultiplier;
    return r;
}

static obc open_bc_of(const ogrid* g, int i, int j, int k) {
    if (g->openHook) {
        obc bc;
        oracle_default_bc(&bc);
        return call_hook(g->openHook, g->hookUser, bc, g, i, j, k);
    }
    return open_bc_faces(g->face, g, i, j, k);
}

static obc open_bc(const lbm_case* c, const ogrid* g, int i, int j, int k) {
    (void)c;
    return open_bc_of(g, i, j, k);
}

static int cmp_kji(const void* a, const void* b) {
    const int* x = (const int*)a;
    const int* y = (const int*)b;
    if (x[2] != y[2]) return x[2] < y[2] ? -1 : 1;
    if (x[1] != y[1]) return x[1] < y[1] ? -1 : 1;
    if (x[0] != y[0]) return x[0] < y[0] ? -1 : 1;
    return 0;
}

/* connectNBRInRows (include/NBRFunctions.h:44-80) for rows keyed by `key` */
static void connect_rows(int n, const int* key, int keyCount, int* nbr) {
    int* counter = (int*)calloc((size_t)keyCount + 1, sizeof(int));
    int* temp = (int*)calloc((size_t)keyCount + 1, sizeof(int));
    int* rowMap = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int c = 0; c < n; ++c) counter[key[c]]++;
    /* exclusive scan */
    int run = 0;
    for (int r = 0; r <= keyCount; ++r) { const int v = counter[r]; counter[r] = run; run += v; }
    for (int c = 0; c < n; ++c) rowMap[counter[key[c]] + temp[key[c]]++] = c;
    for (int r = 0; r < keyCount; ++r) {
        const int start = counter[r], cnt = counter[r + 1] - start;
        if (cnt == 0) continue;
        for (int layer = 1; layer < cnt; ++layer) { /* insertion sort */
            const int v = rowMap[start + layer];
            int s = layer - 1;
            while (s >= 0 && rowMap[start + s] > v) { rowMap[start + s + 1] = rowMap[start + s]; --s; }
            rowMap[start + s + 1] = v;
        }
        for (int layer = 0; layer < cnt - 1; ++layer) nbr[rowMap[start + layer]] = rowMap[start + layer + 1];
        nbr[rowMap[start + cnt - 1]] = rowMap[start];
    }
    free(counter); free(temp); free(rowMap);
}

static int find_cell(const ogrid* g, int i, int j, int k) {
    int lo = 0, hi = g->cellCount;
    while (lo < hi) {
        const int mid = lo + (hi - lo) / 2;
        if (g->I[mid] == i && g->J[mid] == j && g->K[mid] == k) return mid;
        const int before = g->K[mid] < k || (g->K[mid] == k && g->J[mid] < j) ||
                           (g->K[mid] == k && g->J[mid] == j && g->I[mid] < i);
        if (before) lo = mid + 1; else hi = mid;
    }
    return -1;
}

static void get_nbr(const ogrid* g, int cell, int nb[8]);
static void init_info(const lbm_case* c, ogrid* g);
static void apply_initial_condition(const lbm_case* c, ogrid* g);
static void get_ijk(const ogrid* g, int cell, int* i, int* j, int* k);
static void build_open_list(ogrid* g);
static void free_rotors(ogrid* g);

/* buildNBRPlus (include/NBRFunctions.h:82-152) and markGeometricNBRPlus
 * (:154-194) over the current sorted cell list. */
static void nbr_plus(ogrid* g) {
    const int n = g->cellCount;
    free(g->jPlus); free(g->kPlus); free(g->geomBits);
    g->jPlus = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    g->kPlus = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int* key = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int q = 0; q < n; ++q) key[q] = g->K[q] * g->nx + g->I[q];
    connect_rows(n, key, g->nx * g->nz, g->jPlus);
    for (int q = 0; q < n; ++q) key[q] = g->J[q] * g->nx + g->I[q];
    connect_rows(n, key, g->nx * g->ny, g->kPlus);
    free(key);
    g->geomBits = (unsigned char*)calloc((size_t)(n > 0 ? n : 1), 1);
    for (int q = 0; q < n; ++q) {
        const int iP = q + 1 < n ? q + 1 : 0, jP = g->jPlus[q], ijP = jP + 1 < n ? jP + 1 : 0;
        const int kP = g->kPlus[q], ikP = kP + 1 < n ? kP + 1 : 0, jkP = g->jPlus[kP];
        const int ijkP = jkP + 1 < n ? jkP + 1 : 0;
        const int i = g->I[q], j = g->J[q], k = g->K[q];
        unsigned char bits = 0;
        if (g->I[iP] == i + 1 && g->J[iP] == j && g->K[iP] == k) bits |= 1;
        if (g->I[jP] == i && g->J[jP] == j + 1 && g->K[jP] == k) bits |= 2;
        if (g->I[ijP] == i + 1 && g->J[ijP] == j + 1 && g->K[ijP] == k) bits |= 4;
        if (g->I[kP] == i && g->J[kP] == j && g->K[kP] == k + 1) bits |= 8;
        if (g->I[ikP] == i + 1 && g->J[ikP] == j && g->K[ikP] == k + 1) bits |= 16;
        if (g->I[jkP] == i && g->J[jkP] == j + 1 && g->K[jkP] == k + 1) bits |= 32;
        if (g->I[ijkP] == i + 1 && g->J[ijkP] == j + 1 && g->K[ijkP] == k + 1) bits |= 64;
        g->geomBits[q] = bits;
    }
}

/* The 7 plus neighbours of spreadMarkers (include/markerFunctions.h:355-362). */
static void plus7(const ogrid* g, int q, int nb[7]) {
    const int n = g->cellCount;
    nb[0] = q + 1 < n ? q + 1 : 0;
    nb[1] = g->jPlus[q];
    nb[2] = nb[1] + 1 < n ? nb[1] + 1 : 0;
    nb[3] = g->kPlus[q];
    nb[4] = nb[3] + 1 < n ? nb[3] + 1 : 0;
    nb[5] = g->jPlus[nb[3]];
    nb[6] = nb[5] + 1 < n ? nb[5] + 1 : 0;
}

/* spreadMarkers on the cell list (include/markerFunctions.h:344-399): a cell
 * that is marked, or has a marked geometric plus neighbour, marks itself and
 * all its geometric plus neighbours in the target. */
static void spread_cells(const ogrid* g, const unsigned char* src, unsigned char* dst) {
    const int n = g->cellCount;
    memcpy(dst, src, (size_t)n);
    for (int q = 0; q < n; ++q) {
        int nb[7];
        plus7(g, q, nb);
        const unsigned bits = g->geomBits[q];
        int marker = src[q] != 0;
        for (int s = 0; s < 7 && !marker; ++s)
            if (((bits >> s) & 1u) && src[nb[s]]) marker = 1;
        if (!marker) continue;
        dst[q] = 1;
        for (int s = 0; s < 7; ++s)
            if ((bits >> s) & 1u) dst[nb[s]] = 1;
    }
}

/* spreadMarkers on the dense skeleton (include/markerFunctions.h:290-342). */
static void spread_dense(const unsigned char* src, unsigned char* dst, int nx, int ny, int nz) {
    const size_t total = (size_t)nx * ny * nz;
    memcpy(dst, src, total);
    for (size_t cell = 0; cell < total; ++cell) {
        if (src[cell]) continue;
        const int k = (int)(cell / ((size_t)nx * ny)), rem = (int)(cell % ((size_t)nx * ny));
        const int j = rem / nx, i = rem % nx;
        int hit = 0;
        for (int dk = -1; dk <= 1 && !hit; ++dk)
            for (int dj = -1; dj <= 1 && !hit; ++dj)
                for (int di = -1; di <= 1 && !hit; ++di) {
                    if (!di && !dj && !dk) continue;
                    const int a = i + di, b = j + dj, e = k + dk;
                    if (a < 0 || a >= nx || b < 0 || b >= ny || e < 0 || e >= nz) continue;
                    if (src[((size_t)e * ny + b) * nx + a]) hit = 1;
                }
        if (hit) dst[cell] = 1;
    }
}

/* Keep only the marked cells (deleteExcessCells steps 7-13,
 * include/gridBuilderFunctions.h:476-579): the list stays k-j-i sorted, the
 * plus neighbours are rebuilt. */
static void compact_cells(ogrid* g, const unsigned char* keep) {
    int w = 0;
    for (int q = 0; q < g->cellCount; ++q) {
        if (!keep[q]) continue;
        g->I[w] = g->I[q]; g->J[w] = g->J[q]; g->K[w] = g->K[q];
        ++w;
    }
    g->cellCount = w;
    nbr_plus(g);
}

/* Wall velocity a rotating body gives a wall-adjacent cell, evaluated at the
 * fluid cell centre: the per-wallID branch of getLocalBC in drivers with
 * moving walls (cases/torqueTest/torqueTestMain.cu:100-122). */
static void body_wall_velocity(const lbm_body* body, float x, float y, float z, float dtPhys, float res, float u[3]) {
    u[0] = u[1] = u[2] = 0.f;
    if (body->motion != LBM_WALL_ROTATING) return;
    const float dx = x - body->origin[0], dy = y - body->origin[1], dz = z - body->origin[2];
    const float s = body->radians_per_second * dtPhys / res;
    if (body->axis == 2) { u[0] = -s * dy; u[1] = s * dx; }
    else if (body->axis == 0) { u[1] = -s * dz; u[2] = s * dy; }
    else { u[2] = -s * dx; u[0] = s * dz; }
}

/* Full 26-neighbour list through the plus/minus chains
 * (interpolatedBouncebackFunctions.h:227-260). */
static void full_nbrs(const ogrid* g, const int* jMinus, const int* kMinus, int c, int nb[27]) {
    const int n = g->cellCount;
    const int* jP = g->jPlus;
    const int* kP = g->kPlus;
    const int iP = c + 1 >= n ? 0 : c + 1, iM = c - 1 < 0 ? n - 1 : c - 1;
    nb[OOO] = c; nb[POO] = iP; nb[MOO] = iM; nb[OOM] = kMinus[c]; nb[OOP] = kP[c];
    nb[OMO] = jMinus[c]; nb[OPO] = jP[c];
    nb[POM] = kMinus[iP]; nb[MOP] = kP[iM]; nb[POP] = kP[iP]; nb[MOM] = kMinus[iM];
    nb[MMO] = jMinus[iM]; nb[PPO] = jP[iP]; nb[OPM] = kMinus[jP[c]]; nb[OMP] = kP[jMinus[c]];
    nb[MPO] = jP[iM]; nb[PMO] = jMinus[iP]; nb[OPP] = jP[kP[c]]; nb[OMM] = kMinus[jMinus[c]];
    nb[MPM] = kMinus[jP[iM]]; nb[PMP] = kP[jMinus[iP]]; nb[MMP] = kP[jMinus[iM]]; nb[PPM] = kMinus[jP[iP]];
    nb[PMM] = kMinus[jMinus[iP]]; nb[MPP] = jP[kP[iM]]; nb[MMM] = kMinus[jMinus[iM]]; nb[PPP] = jP[kP[iP]];
}

/* buildLinkExistenceMarkerArray for one wall-adjacent cell:
 * interpolatedBouncebackFunctions.h:181-398.  Bit d set = link towards a wall
 * cell in direction d; `pierce` gets the links that start or end on an
 * interface cell (iface, NULL on a single level). */
static unsigned link_bits(const ogrid* g, const int* jMinus, const int* kMinus, int cell, const unsigned char* iface,
                          unsigned* pierce) {
    int nb[27];
    full_nbrs(g, jMinus, kMinus, cell, nb);
    const int i = g->I[cell], j = g->J[cell], k = g->K[cell];
    int geo[27];
    int all = 1, ip = 1, jp = 1, kp = 1, im = 1, jm = 1, km = 1;
    for (int d = 1; d < 27; ++d) {
        geo[d] = 1;
        const int ie = i + CX[d], je = j + CY[d], ke = k + CZ[d];
        const int q = nb[d];
        if (g->I[q] == ie && g->J[q] == je && g->K[q] == ke) continue;
        geo[d] = 0;
        if (ie < 0 || ie >= g->nx || je < 0 || je >= g->ny || ke < 0 || ke >= g->nz) continue;
        all = 0;
        if (CX[d] > 0) ip = 0;
        if (CY[d] > 0) jp = 0;
        if (CZ[d] > 0) kp = 0;
        if (CX[d] < 0) im = 0;
        if (CY[d] < 0) jm = 0;
        if (CZ[d] < 0) km = 0;
    }
    unsigned bits = 0;
    *pierce = 0;
    const int me = iface && iface[cell];
    if (i != 0 && i != g->nx - 1 && j != 0 && j != g->ny - 1 && k != 0 && k != g->nz - 1) {
        if (!all) return 0;
        for (int d = 1; d < 27; ++d)
            if (g->wallMarker[nb[d]]) {
                bits |= 1u << d;
                if (me || (iface && iface[nb[d]])) *pierce |= 1u << d;
            }
        return bits;
    }
    for (int d = 1; d < 27; ++d) {
        if (!geo[d] || !g->wallMarker[nb[d]]) continue;
        if ((CX[d] > 0 && !ip) || (CY[d] > 0 && !jp) || (CZ[d] > 0 && !kp)) continue;
        if ((CX[d] < 0 && !im) || (CY[d] < 0 && !jm) || (CZ[d] < 0 && !km)) continue;
        bits |= 1u << d;
        if (me || (iface && iface[nb[d]])) *pierce |= 1u << d;
    }
    return bits;
}

/* The coarser level of a level under construction: its grid, the parent of
 * every cell here (-1: none), its wallIDArrayFull and its body ray maps. */
typedef struct oparent {
    const ogrid* grid;
    const int* parent;
    const int* wallIDFull;
    const oraymap* maps;
} oparent;

/* buildWallMarkers (include/gridBuilderFunctions.h:590-739), then
 * buildLinkLengthArray (interpolatedBouncebackFunctions.h:471-660) and
 * packWallData (:662-695).  Fills wallMarker, the wall-adjacent list in cell
 * order, wallData, linkLength and the wall velocities.  On a finer level
 * (`up` set) a cell with a parent inherits the parent's wall state and body
 * marks, and the parent's wallID wins (steps 1-2); `iface` marks interface
 * cells (links from or to them get length 1/2), `overlap` the cells whose
 * wallData carries the overlap bit; `wallIDFull` (may be NULL) receives the
 * wallID of every cell. */
static void build_walls(const lbm_case* c, ogrid* g, const ostl* bodies, const oraymap* maps, const oraymap* total,
                        const oparent* up, const unsigned char* iface, const unsigned char* overlap,
                        int* wallIDFull) {
    const int n = g->cellCount;
    for (int q = 0; q < n; ++q) g->wallMarker[q] = (unsigned char)oray_solid(total, g->I[q], g->J[q], g->K[q]);
    if (up)
        for (int q = 0; q < n; ++q)
            if (up->parent[q] >= 0) g->wallMarker[q] = up->grid->wallMarker[up->parent[q]];
    int* wallID = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    unsigned char* src = (unsigned char*)malloc((size_t)(n > 0 ? n : 1));
    unsigned char* bw = (unsigned char*)malloc((size_t)(n > 0 ? n : 1));
    for (int q = 0; q < n; ++q) wallID[q] = -1;
    for (int b = 0; b < c->body_count; ++b) {
        for (int q = 0; q < n; ++q) src[q] = (unsigned char)oray_solid(&maps[b], g->I[q], g->J[q], g->K[q]);
        if (up)
            for (int q = 0; q < n; ++q) {
                const int pc = up->parent[q];
                if (pc >= 0)
                    src[q] = (unsigned char)oray_solid(&up->maps[b], up->grid->I[pc], up->grid->J[pc], up->grid->K[pc]);
            }
        spread_cells(g, src, bw);
        for (int q = 0; q < n; ++q) {
            if (!bw[q] || g->wallMarker[q]) continue;
            int id = b;  /* the last body wins, a parent's wallID above all */
            if (up && up->parent[q] >= 0 && up->wallIDFull[up->parent[q]] >= 0) id = up->wallIDFull[up->parent[q]];
            wallID[q] = id;
        }
    }
    if (wallIDFull) memcpy(wallIDFull, wallID, sizeof(int) * (size_t)n);
    free(src);
    free(bw);
    int nw = 0;
    for (int q = 0; q < n; ++q) nw += wallID[q] >= 0;
    g->wallCount = nw;
    g->wallIndex = (int*)malloc(sizeof(int) * (size_t)(nw > 0 ? nw : 1));
    int* ids = (int*)malloc(sizeof(int) * (size_t)(nw > 0 ? nw : 1));
    for (int q = 0, w = 0; q < n; ++q)
        if (wallID[q] >= 0) { g->wallIndex[w] = q; ids[w] = wallID[q]; ++w; }
    free(wallID);

    /* NBR minus as the inverse permutations (gridBuilderFunctions.h:565-575) */
    int* jMinus = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int* kMinus = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int q = 0; q < n; ++q) { jMinus[g->jPlus[q]] = q; kMinus[g->kPlus[q]] = q; }
    unsigned* links = (unsigned*)malloc(sizeof(unsigned) * (size_t)(nw > 0 ? nw : 1));
    unsigned* pierce = (unsigned*)malloc(sizeof(unsigned) * (size_t)(nw > 0 ? nw : 1));
    for (int w = 0; w < nw; ++w) links[w] = link_bits(g, jMinus, kMinus, g->wallIndex[w], iface, &pierce[w]);
    free(jMinus);
    free(kMinus);

    /* link lengths: the shortest accepted crossing over every body's triangles
     * in the bin of the cell centre */
    float* len = (float*)malloc(sizeof(float) * 27 * (size_t)(nw > 0 ? nw : 1));
    for (size_t q = 0; q < 27 * (size_t)nw; ++q) len[q] = 2.f;
    const float edgeTol = 0.1f * g->res, qTol = 0.2f;
    for (int b = 0; b < c->body_count; ++b) {
        const ostl* t = &bodies[b];
        const int bxy = t->binCountX * t->binCountY;
        for (int w = 0; w < nw; ++w) {
            if (!links[w]) continue;
            const int cell = g->wallIndex[w];
            const float x = g->I[cell] * g->res + g->ox, y = g->J[cell] * g->res + g->oy,
                        z = g->K[cell] * g->res + g->oz;
            const int ib = (int)((x - t->oxBin) / t->binSize), jb = (int)((y - t->oyBin) / t->binSize),
                      kb = (int)((z - t->ozBin) / t->binSize);
            if (ib < 0 || ib >= t->binCountX || jb < 0 || jb >= t->binCountY || kb < 0 || kb >= t->binCountZ)
                continue;
            const int bin = bxy * kb + t->binCountX * jb + ib;
            for (int r = t->firstInBin[bin]; r < t->firstInBin[bin + 1]; ++r) {
                const int tri = t->bin[r];
                const float ax = t->ax[tri] - x, ay = t->ay[tri] - y, az = t->az[tri] - z;
                const float bx = t->bx[tri] - x, by = t->by[tri] - y, bz = t->bz[tri] - z;
                const float cx = t->cx[tri] - x, cy = t->cy[tri] - y, cz = t->cz[tri] - z;
                for (int d = 1; d < 27; ++d) {
                    if (!((links[w] >> d) & 1u) || ((pierce[w] >> d) & 1u)) continue;
                    float tHit;
                    if (!oray_triangle(ax, ay, az, bx, by, bz, cx, cy, cz, (float)CX[d], (float)CY[d], (float)CZ[d],
                                       edgeTol, &tHit))
                        continue;
                    float qv = tHit / g->res;
                    float* slot = &len[(size_t)w * 27 + d];
                    if (qv > 0 && qv <= 1.f) {
                        qv = qv < 0.00001f ? 0.00001f : (qv > 1.f ? 1.f : qv);
                        if (*slot < 0.f || qv < *slot) *slot = qv;
                    } else if (qv > -qTol && qv <= 1.f + qTol) {
                        qv = qv < 0.00001f ? 0.00001f : (qv > 1.f ? 1.f : qv);
                        if (*slot < 0.f) {
                            if (qv < -*slot) *slot = -qv;
                        } else if (*slot > 1.f) {
                            *slot = -qv;
                        }
                    }
                }
            }
        }
    }
    g->wallData = (unsigned*)calloc((size_t)(nw > 0 ? nw : 1), sizeof(unsigned));
    g->linkLength = (unsigned*)calloc(7 * (size_t)(nw > 0 ? nw : 1), sizeof(unsigned));
    g->wallVel = (float*)calloc(3 * (size_t)(nw > 0 ? nw : 1), sizeof(float));
    g->wallForce = (float*)calloc(3 * (size_t)(nw > 0 ? nw : 1), sizeof(float));
    for (int w = 0; w < nw; ++w) {
        unsigned data = (unsigned)ids[w] << 27;
        if (overlap && overlap[g->wallIndex[w]]) data |= 1u;
        int li = 0;
        for (int d = 1; d < 27; ++d) {
            if (!((links[w] >> d) & 1u)) continue;
            float qv = len[(size_t)w * 27 + d];
            if ((pierce[w] >> d) & 1u) qv = 0.5f;  /* through an interface: as on the other level */
            else if (qv > 1.f) qv = 0.5f;      /* no crossing found: safe fallback */
            else if (qv < 0.f) qv = -qv;       /* near miss kept */
            qv = qv < 0.f ? 0.f : (qv > 1.f ? 1.f : qv);
            data |= 1u << d;
            const unsigned code = (unsigned)(qv * 254.f + 0.5f);
            g->linkLength[(size_t)(li / 4) * nw + w] |= code << (8 * (li % 4));
            ++li;
        }
        g->wallData[w] = data;
        const int cell = g->wallIndex[w];
        float u[3];
        if (c->local_bc_hook) {
            obc bc;
            oracle_default_bc(&bc);
            bc.wallID = ids[w];
            bc = call_hook(c->local_bc_hook, c->hook_user, bc, g, g->I[cell], g->J[cell], g->K[cell]);
            u[0] = bc.ux; u[1] = bc.uy; u[2] = bc.uz;
        } else {
            body_wall_velocity(&c->body[ids[w]], g->I[cell] * g->res + g->ox, g->J[cell] * g->res + g->oy,
                               g->K[cell] * g->res + g->oz, g->dtPhys, g->res, u);
        }
        for (int a = 0; a < 3; ++a) g->wallVel[(size_t)a * nw + w] = u[a];
    }
    free(ids);
    free(links);
    free(pierce);
    free(len);
}

static int build_rotor(ogrid* g, int r, const lbm_rotor* rt);
static int finish_level(const lbm_case* c, ogrid* g, const unsigned char* overlap);

int oracle_build(const lbm_case* c, ogrid* g) {
    memset(g, 0, sizeof(*g));
    if (c->grid_level_count != 1) return LBM_ERR_UNSUPPORTED;
    if (c->body_count < 0 || c->body_count > LBM_MAX_BODIES || c->rotor_count < 0 || c->rotor_count > 4)
        return LBM_ERR_INVALID;
    /* initializeGridInfo (:9-64), level 0 */
    init_info(c, g);
    if (g->nx < 2) return LBM_ERR_INVALID;
    const int snx = g->nx / 2, sny = g->ny / 2, snz = g->nz / 2;

    /* readSTL + sortSTLToBins for every static body, one ray map each on the
     * level and their union (initializeVoxelizers, voxelizerFunctions.h:692-728) */
    const int nb = c->body_count;
    ostl* bodies = (ostl*)calloc((size_t)(nb > 0 ? nb : 1), sizeof(ostl));
    oraymap* maps = (oraymap*)calloc((size_t)(nb > 0 ? nb : 1), sizeof(oraymap));
    oraymap total;
    for (int b = 0; b < nb; ++b) {
        if (!c->body[b].triangles || ostl_load(&bodies[b], c->body[b].triangles, c->body[b].triangle_count) == 0) {
            for (int q = 0; q <= b; ++q) ostl_free(&bodies[q]);
            for (int q = 0; q < b; ++q) oray_free(&maps[q]);
            free(bodies); free(maps);
            return LBM_ERR_BUILD;
        }
        ostl_bins(&bodies[b], c->res_global);
        oray_voxelize(&maps[b], &bodies[b], g->ox, g->oy, g->oz, g->res, g->nx, g->ny);
    }
    if (nb > 0) {
        oray_copy(&total, &maps[0]);
        for (int b = 1; b < nb; ++b) oray_union(&total, &maps[b]);
    } else {
        oray_empty(&total, g->nx, g->ny);
    }

    /* markKeepCells on the skeleton (markerFunctions.h:401-407): a skeleton
     * cell is kept when one of its 8 level cells is fluid, plus one layer */
    const size_t sc = (size_t)snx * sny * snz;
    unsigned char* keepS = (unsigned char*)malloc(sc);
    unsigned char* keepT = (unsigned char*)malloc(sc);
    for (size_t s = 0; s < sc; ++s) {
        const int ks = (int)(s / ((size_t)snx * sny)), rem = (int)(s % ((size_t)snx * sny));
        keepS[s] = (unsigned char)oray_block_has_fluid(&total, rem % snx, rem / snx, ks, 2);
    }
    spread_dense(keepS, keepT, snx, sny, snz);

    /* buildFinerGridBuilder from the skeleton (:66-132): 8 children per kept
     * skeleton cell, then sortIJK (:204-234) */
    int kept = 0;
    for (size_t s = 0; s < sc; ++s) kept += keepT[s];
    const int n0 = 8 * kept;
    int* ijk = (int*)malloc(sizeof(int) * 3 * (size_t)(n0 > 0 ? n0 : 1));
    int cf = 0;
    for (size_t s = 0; s < sc; ++s) {
        if (!keepT[s]) continue;
        const int ks = (int)(s / ((size_t)snx * sny)), rem = (int)(s % ((size_t)snx * sny)), js = rem / snx,
                  is = rem % snx;
        for (int ka = 0; ka < 2; ++ka)
            for (int ja = 0; ja < 2; ++ja)
                for (int ia = 0; ia < 2; ++ia) {
                    ijk[3 * cf] = 2 * is + ia;
                    ijk[3 * cf + 1] = 2 * js + ja;
                    ijk[3 * cf + 2] = 2 * ks + ka;
                    ++cf;
                }
    }
    free(keepS);
    free(keepT);
    qsort(ijk, (size_t)n0, 3 * sizeof(int), cmp_kji);
    g->cellCount = n0;
    g->I = (int*)malloc(sizeof(int) * (size_t)(n0 > 0 ? n0 : 1));
    g->J = (int*)malloc(sizeof(int) * (size_t)(n0 > 0 ? n0 : 1));
    g->K = (int*)malloc(sizeof(int) * (size_t)(n0 > 0 ? n0 : 1));
    for (int q = 0; q < n0; ++q) { g->I[q] = ijk[3 * q]; g->J[q] = ijk[3 * q + 1]; g->K[q] = ijk[3 * q + 2]; }
    free(ijk);
    nbr_plus(g);

    /* deleteExcessCells (:402-588), single level: keep the fluid cells plus one
     * layer of wall cells */
    {
        unsigned char* fluid = (unsigned char*)malloc((size_t)(n0 > 0 ? n0 : 1));
        unsigned char* keep = (unsigned char*)malloc((size_t)(n0 > 0 ? n0 : 1));
        for (int q = 0; q < n0; ++q) fluid[q] = (unsigned char)!oray_solid(&total, g->I[q], g->J[q], g->K[q]);
        spread_cells(g, fluid, keep);
        compact_cells(g, keep);
        free(fluid);
        free(keep);
    }
    const int n = g->cellCount;
    g->wallMarker = (unsigned char*)calloc((size_t)(n > 0 ? n : 1), 1);
    build_walls(c, g, bodies, maps, &total, NULL, NULL, NULL, NULL);
    for (int b = 0; b < nb; ++b) { ostl_free(&bodies[b]); oray_free(&maps[b]); }
    free(bodies);
    free(maps);
    oray_free(&total);

    return finish_level(c, g, NULL);
}

/* gridBuilderToGrid (include/gridBuilderFunctions.h:1032-1564) for one level
 * whose cells, NBR and walls are built, then buildRotors and
 * applyInitialCondition.  `overlap` (NULL: none) marks the cells under an
 * interface overlap (wallMap -2).  The level's uniform getLocalBC is the
 * case's, or the local hook's answer for a fluid cell at the first cell. */
static int finish_level(const lbm_case* c, ogrid* g, const unsigned char* overlap) {
    const int n = g->cellCount;
    if (c->local_bc_hook && n > 0) {
        obc bc;
        oracle_default_bc(&bc);
        bc.collisionLimiter = g->limiter;
        bc.nuMultiplier = g->nuMultiplier;
        bc.gx = g->gx; bc.gy = g->gy; bc.gz = g->gz;
        bc.useIBB = g->useIBB;
        bc.wallID = -1;
        bc = call_hook(c->local_bc_hook, c->hook_user, bc, g, g->I[0], g->J[0], g->K[0]);
        g->limiter = bc.collisionLimiter;
        g->nuMultiplier = bc.nuMultiplier;
        g->gx = bc.gx; g->gy = bc.gy; g->gz = bc.gz;
        g->useIBB = bc.useIBB;
    }
    /* gridBuilderToGrid (:1032-1126): first-in-row marks, inclusive max scan,
     * exclusive sum scan, compressed arrays */
    int* firstInRow = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int* scan = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int q = 0; q < n; ++q) {
        if (q == 0) { firstInRow[q] = 0; scan[q] = 1; continue; }
        const int jk = g->jPlus[g->kPlus[q]], jkPrev = g->jPlus[g->kPlus[q - 1]];
        const int brk = g->I[q] != g->I[q - 1] + 1 || g->J[q] != g->J[q - 1] || g->K[q] != g->K[q - 1] ||
                        g->jPlus[q] != g->jPlus[q - 1] + 1 || g->kPlus[q] != g->kPlus[q - 1] + 1 ||
                        jk != jkPrev + 1;
        firstInRow[q] = brk ? q : 0;
        scan[q] = brk ? 1 : 0;
    }
    for (int q = 1; q < n; ++q) if (firstInRow[q] < firstInRow[q - 1]) firstInRow[q] = firstInRow[q - 1];
    int rows = 0;
    for (int q = 0; q < n; ++q) { const int v = scan[q]; scan[q] = rows; rows += v; }
    g->rowCount = rows;
    g->shifter = (int*)malloc(sizeof(int) * n);
    g->rowI = (int*)malloc(sizeof(int) * rows); g->rowJ = (int*)malloc(sizeof(int) * rows);
    g->rowK = (int*)malloc(sizeof(int) * rows); g->rowJP = (int*)malloc(sizeof(int) * rows);
    g->rowKP = (int*)malloc(sizeof(int) * rows); g->rowJKP = (int*)malloc(sizeof(int) * rows);
    for (int q = 0; q < n; ++q) {
        if (q == firstInRow[q]) {
            const int r = scan[q];
            g->shifter[q] = r;
            g->rowI[r] = g->I[q]; g->rowJ[r] = g->J[q]; g->rowK[r] = g->K[q];
            g->rowJP[r] = g->jPlus[q]; g->rowKP[r] = g->kPlus[q]; g->rowJKP[r] = g->jPlus[g->kPlus[q]];
        } else {
            g->shifter[q] = firstInRow[q] - q;
        }
    }
    free(firstInRow); free(scan);

    /* wallMap (:1128-1149) and the periodic overlap (:1232-1274) */
    g->wallMap = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int q = 0; q < n; ++q) g->wallMap[q] = g->wallMarker[q] ? -3 : (overlap && overlap[q] ? -2 : -1);
    for (int w = 0; w < g->wallCount; ++w) g->wallMap[g->wallIndex[w]] = w;
    const int layers = 1 << g->gridID;
    for (int q = 0; q < n; ++q) {
        if (g->wallMarker[q]) continue;
        const int i = g->I[q], j = g->J[q], k = g->K[q];
        int ov = 0;
        if (i < layers || i >= g->nx - layers) ov |= open_bc(c, g, i < layers ? 0 : g->nx - 1, j, k).periodic;
        if (j < layers || j >= g->ny - layers) ov |= open_bc(c, g, i, j < layers ? 0 : g->ny - 1, k).periodic;
        if (k < layers || k >= g->nz - layers) ov |= open_bc(c, g, i, j, k < layers ? 0 : g->nz - 1).periodic;
        if (!ov) continue;
        if (g->wallMap[q] >= 0) g->wallData[g->wallMap[q]] |= 1u;
        else if (g->wallMap[q] == -1) g->wallMap[q] = -2;
    }
    build_open_list(g);

    /* periodic lists (:1486-1564) */
    g->perIndex = (int*)malloc(sizeof(int) * n);
    g->perSource = (int*)malloc(sizeof(int) * n);
    g->perCount = 0;
    const int per = (int)lround(pow(2.0, g->gridID));
    for (int q = 0; q < n; ++q) {
        if (g->wallMarker[q]) continue;
        int i = g->I[q], j = g->J[q], k = g->K[q];
        if (!(i == 0 || i == g->nx - 1 || j == 0 || j == g->ny - 1 || k == 0 || k == g->nz - 1)) continue;
        if (!open_bc(c, g, i, j, k).periodic) continue;
        if (i == 0) i = g->nx - 2 * per; else if (i == g->nx - 1) i = 2 * per - 1;
        if (j == 0) j = g->ny - 2 * per; else if (j == g->ny - 1) j = 2 * per - 1;
        if (k == 0) k = g->nz - 2 * per; else if (k == g->nz - 1) k = 2 * per - 1;
        const int src = find_cell(g, i, j, k);
        if (src < 0 || g->wallMarker[src]) { oracle_free(g); return LBM_ERR_BUILD; }
        g->perIndex[g->perCount] = q;
        g->perSource[g->perCount] = src;
        g->perCount++;
    }
    long long walls = 0;
    for (int q = 0; q < n; ++q) walls += g->wallMarker[q] != 0;
    g->fluidUpdates = (long long)n - walls;
    /* buildRotors (include/rotorFunctions.h:315-585) */
    for (int r = 0; r < c->rotor_count; ++r)
        if (build_rotor(g, r, &c->rotor[r]) != 0) { oracle_free(g); return LBM_ERR_BUILD; }
    apply_initial_condition(c, g);
    return 0;
}

void oracle_free(ogrid* g) {
    free(g->I); free(g->J); free(g->K); free(g->jPlus); free(g->kPlus); free(g->geomBits);
    free(g->wallMarker); free(g->shifter); free(g->rowI); free(g->rowJ); free(g->rowK);
    free(g->rowJP); free(g->rowKP); free(g->rowJKP); free(g->wallMap); free(g->perIndex);
    free(g->perSource); free(g->f);
    free(g->wallIndex); free(g->wallData); free(g->linkLength); free(g->wallVel); free(g->wallForce);
    free(g->openIndex); free(g->openRef); free(g->openCum);
    free_rotors(g);
    memset(g, 0, sizeof(*g));
}


static void init_info(const lbm_case* c, ogrid* g) {
    const float* b = c->bounds;
    g->res = c->res_global;
    const float sres = g->res * 2.f;
    const int snx = (int)((b[3] - b[0]) / sres), sny = (int)((b[4] - b[1]) / sres), snz = (int)((b[5] - b[2]) / sres);
    const float sox = b[0] + ((b[3] - b[0]) - (snx * sres) + sres) / 2.0f;
    const float soy = b[1] + ((b[4] - b[1]) - (sny * sres) + sres) / 2.0f;
    const float soz = b[2] + ((b[5] - b[2]) - (snz * sres) + sres) / 2.0f;
    g->nx = snx * 2; g->ny = sny * 2; g->nz = snz * 2;
    g->ox = sox - g->res * 0.5f; g->oy = soy - g->res * 0.5f; g->oz = soz - g->res * 0.5f;
    g->dtPhys = c->dt_phys_global;
    g->nu = (g->dtPhys * c->nu_phys) / ((g->res / 1000.f) * (g->res / 1000.f));
    g->limiter = c->collision_limiter;
    g->nuMultiplier = c->nu_multiplier;
    g->gx = c->gx; g->gy = c->gy; g->gz = c->gz;
    g->useIBB = c->use_ibb;
    g->trackWallForce = c->track_wall_force;
    g->trackOpen = c->track_open_boundaries;
    g->openImpedance = c->open_bc_scheme == LBM_OPEN_IMPEDANCE;
    g->openTolerance = c->rho_reflection_tolerance;
    g->trackRotorForce = c->track_rotor_force;
    memcpy(g->face, c->face, sizeof(g->face));
    g->openHook = c->open_bc_hook;
    g->hookUser = c->hook_user;
}

/* Open-boundary lists (gridBuilderFunctions.h:1276-1330): boundary cells that
 * are neither walls nor periodic, grouped by openBCID in ID order, each group
 * in cell order. */
static void build_open_list(ogrid* g) {
    const int n = g->cellCount;
    int* id = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int maxId = -1;
    for (int q = 0; q < n; ++q) {
        id[q] = -1;
        if (g->wallMap[q] == -3) continue;
        int i, j, k;
        get_ijk(g, q, &i, &j, &k);
        if (!(i == 0 || i == g->nx - 1 || j == 0 || j == g->ny - 1 || k == 0 || k == g->nz - 1)) continue;
        const obc bc = open_bc_of(g, i, j, k);
        if (bc.periodic) continue;
        id[q] = bc.openBCID;
        if (id[q] > maxId) maxId = id[q];
    }
    g->openCount = 0;
    g->openIndex = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int b = 0; b <= maxId; ++b)
        for (int q = 0; q < n; ++q)
            if (id[q] == b) g->openIndex[g->openCount++] = q;
    g->openBCCount = g->openCount;
    g->openRef = (float*)calloc(2 * (size_t)(g->openCount > 0 ? g->openCount : 1), sizeof(float));
    g->openCum = (float*)calloc(2 * (size_t)(g->openCount > 0 ? g->openCount : 1), sizeof(float));
    free(id);
}

static void outer_normal(const ogrid* g, int i, int j, int k, int n[3]) {
    /* getOuterNormal (include/cellFunctions.h:110-122) */
    n[0] = i == 0 ? -1 : (i == g->nx - 1 ? 1 : 0);
    n[1] = j == 0 ? -1 : (j == g->ny - 1 ? 1 : 0);
    n[2] = k == 0 ? -1 : (k == g->nz - 1 ? 1 : 0);
}

/* getCompressedIJK (include/cellFunctions.h:51-72) */
static void get_ijk(const ogrid* g, int cell, int* i, int* j, int* k) {
    const int shift = g->shifter[cell];
    if (shift >= 0) { *i = g->rowI[shift]; *j = g->rowJ[shift]; *k = g->rowK[shift]; }
    else {
        const int ci = g->shifter[cell + shift];
        *i = g->rowI[ci] - shift; *j = g->rowJ[ci]; *k = g->rowK[ci];
    }
}

/* allocateFArray + applyInitialCondition (applyInitialCondition.h:8-41) */
static void apply_initial_condition(const lbm_case* c, ogrid* g) {
    const int n = g->cellCount;
    free(g->f);
    g->f = (float*)malloc(sizeof(float) * 27 * (size_t)n);
#pragma omp parallel for schedule(static)
    for (int q = 0; q < n; ++q) {
        obc bc;
        oracle_default_bc(&bc);
        int ci, cj, ck;
        get_ijk(g, q, &ci, &cj, &ck);
        if (c->initial_condition_hook) {
            bc = call_hook(c->initial_condition_hook, c->hook_user, bc, g, ci, cj, ck);
        } else if (c->ic_kind == LBM_IC_TAYLOR_GREEN) {
            const float x = ci * g->res + g->ox, y = cj * g->res + g->oy, z = ck * g->res + g->oz;
            const float X = x / c->tgv_length, Y = y / c->tgv_length, Z = z / c->tgv_length;
            const float u0 = c->tgv_u0;
            bc.ux = u0 * sinf(X) * cosf(Y) * cosf(Z);
            bc.uy = -u0 * cosf(X) * sinf(Y) * cosf(Z);
            bc.uz = 0.f;
            bc.dRho = (3.f * u0 * u0 / 16.f) * (cosf(2.f * X) + cosf(2.f * Y)) * (2.f + cosf(2.f * Z));
        } else {
            bc.dRho = c->ic_dRho; bc.ux = c->ic_ux; bc.uy = c->ic_uy; bc.uz = c->ic_uz;
        }
        float feq[27];
        oracle_get_feq(bc.dRho, bc.ux, bc.uy, bc.uz, feq);
        int nb[8];
        get_nbr(g, q, nb);
        for (int d = 0; d < 27; ++d) {
            const int slot = g->flip ? INV[d] : d;
            g->f[(size_t)slot * n + nb[pre_nbr(d)]] = feq[d];
        }
    }
    /* previous values of the open boundary (applyInitialCondition.h:43-81) */
    for (int q = 0; q < g->openCount; ++q) {
        const int cell = g->openIndex[q];
        int ci, cj, ck, on[3], nb[8];
        get_ijk(g, cell, &ci, &cj, &ck);
        outer_normal(g, ci, cj, ck, on);
        get_nbr(g, cell, nb);
        float f[27], m[4];
        for (int d = 0; d < 27; ++d) f[d] = g->f[(size_t)(g->flip ? INV[d] : d) * n + nb[pre_nbr(d)]];
        oracle_get_drho_u(f, m);
        g->openRef[q] = m[0];
        g->openRef[g->openCount + q] = (float)on[0] * m[1] + (float)on[1] * m[2] + (float)on[2] * m[3];
    }
}

static int* copy_ints(const int* src, int n) {
    int* d = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    if (n > 0) memcpy(d, src, sizeof(int) * (size_t)n);
    return d;
}

int oracle_from_tables(const lbm_case* c, ogrid* g, int cellCount, int rowCount, const int* shifter,
                       const int* rowI, const int* rowJ, const int* rowK, const int* rowJP,
                       const int* rowKP, const int* rowJKP, const int* wallMap, int perCount,
                       const int* perIndex, const int* perSource, int wallCount, const int* wallIndex,
                       const unsigned* wallData, const unsigned* linkLength, const float* wallVel) {
    memset(g, 0, sizeof(*g));
    init_info(c, g);
    g->cellCount = cellCount;
    g->rowCount = rowCount;
    g->shifter = copy_ints(shifter, cellCount);
    g->rowI = copy_ints(rowI, rowCount); g->rowJ = copy_ints(rowJ, rowCount); g->rowK = copy_ints(rowK, rowCount);
    g->rowJP = copy_ints(rowJP, rowCount); g->rowKP = copy_ints(rowKP, rowCount); g->rowJKP = copy_ints(rowJKP, rowCount);
    g->wallMap = copy_ints(wallMap, cellCount);
    g->perCount = perCount;
    g->perIndex = copy_ints(perIndex, perCount);
    g->perSource = copy_ints(perSource, perCount);
    g->wallCount = wallCount;
    g->wallIndex = copy_ints(wallIndex, wallCount);
    g->wallData = (unsigned*)malloc(sizeof(unsigned) * (size_t)(wallCount > 0 ? wallCount : 1));
    g->linkLength = (unsigned*)malloc(sizeof(unsigned) * 7 * (size_t)(wallCount > 0 ? wallCount : 1));
    g->wallVel = (float*)malloc(sizeof(float) * 3 * (size_t)(wallCount > 0 ? wallCount : 1));
    g->wallForce = (float*)calloc(3 * (size_t)(wallCount > 0 ? wallCount : 1), sizeof(float));
    if (wallCount > 0) {
        memcpy(g->wallData, wallData, sizeof(unsigned) * (size_t)wallCount);
        memcpy(g->linkLength, linkLength, sizeof(unsigned) * 7 * (size_t)wallCount);
        memcpy(g->wallVel, wallVel, sizeof(float) * 3 * (size_t)wallCount);
    }
    long long walls = 0;
    for (int q = 0; q < cellCount; ++q) walls += g->wallMap[q] == -3;
    g->fluidUpdates = (long long)cellCount - walls;
    build_open_list(g);
    apply_initial_condition(c, g);
    return 0;
}

void oracle_wall_force(const ogrid* g, int wallID, double* out) {
    for (int q = 0; q < 6; ++q) out[q] = 0.0;
    for (int w = 0; w < g->wallCount; ++w) {
        if ((int)((g->wallData[w] >> 27) & 31u) != wallID) continue;
        int ci, cj, ck;
        get_ijk(g, g->wallIndex[w], &ci, &cj, &ck);
        const double x = (double)(ci * g->res + g->ox), y = (double)(cj * g->res + g->oy),
                     z = (double)(ck * g->res + g->oz);
        const double fx = g->wallForce[w], fy = g->wallForce[g->wallCount + w], fz = g->wallForce[2 * g->wallCount + w];
        out[0] += fx; out[1] += fy; out[2] += fz;
        out[3] += y * fz - z * fy;
        out[4] += z * fx - x * fz;
        out[5] += x * fy - y * fx;
    }
}

/* getCompressedNBR + finishNBRPlus (include/cellFunctions.h:74-94,
 * include/NBRFunctions.h:5-11) */
static void get_nbr(const ogrid* g, int cell, int nb[8]) {
    const int shift = g->shifter[cell];
    int jP, kP, jkP;
    if (shift >= 0) {
        jP = g->rowJP[shift]; kP = g->rowKP[shift]; jkP = g->rowJKP[shift];
    } else {
        const int ci = g->shifter[cell + shift];
        jP = g->rowJP[ci] - shift; kP = g->rowKP[ci] - shift; jkP = g->rowJKP[ci] - shift;
    }
    const int n = g->cellCount;
    nb[0] = cell;
    nb[1] = cell + 1 >= n ? 0 : cell + 1;
    nb[2] = jP;
    nb[3] = jP + 1 >= n ? 0 : jP + 1;
    nb[4] = kP;
    nb[5] = kP + 1 >= n ? 0 : kP + 1;
    nb[6] = jkP;
    nb[7] = jkP + 1 >= n ? 0 : jkP + 1;
}

/* one open-boundary cell after streaming (include/updateGrid.h:191-353) */
static void open_boundary(ogrid* g) {
    const size_t n = (size_t)g->cellCount;
    const int m = g->openCount;
#pragma omp parallel for schedule(static)
    for (int q = 0; q < m; ++q) {
        const int cell = g->openIndex[q];
        const int wm = g->wallMap[cell];
        int trackFlow = wm != -2;
        if (wm >= 0 && (g->wallData[wm] & 1u)) trackFlow = 0;
        int ci, cj, ck, on[3], nb[8];
        get_ijk(g, cell, &ci, &cj, &ck);
        outer_normal(g, ci, cj, ck, on);
        get_nbr(g, cell, nb);
        float f[27];
        float dRhoZ = 0.f;
        for (int d = 0; d < 27; ++d) {
            f[d] = 0.f;
            if (on[0] * CX[d] < 0 || on[1] * CY[d] < 0 || on[2] * CZ[d] < 0) continue;
            f[d] = g->f[(size_t)(g->flip ? INV[d] : d) * n + nb[pre_nbr(d)]];
            const int product = on[0] * CX[d] + on[1] * CY[d] + on[2] * CZ[d];
            if (product == 0) dRhoZ += f[d];
            else dRhoZ += 2.f * f[d];
            f[d] += W[d];
        }
        const float dRhoRef = g->openRef[q];
        const float uNormalRef = g->openRef[m + q];
        obc bc = open_bc_faces(g->face, g, ci, cj, ck);
        if (abs(on[0]) + abs(on[1]) + abs(on[2]) != 1) bc.nonReflective = 0;
        const float cs = 0.57735026918962576f;
        const int code = (on[0] + 5) * 100 + (on[1] + 5) * 10 + (on[2] + 5);
        /* the impedance scheme (cases/nonReflectiveTest/
         * updateGrid_SCHLAFFER_IMPEDANCE_SCHEME.h:250-310): the reference
         * arrays hold the previous completed boundary state; the given density
         * or normal velocity is clamped to within the tolerance of the
         * non-reflecting state computed from it */
        const int impedance = g->openImpedance && bc.nonReflective && g->openTolerance < 1.f;
        const float tol = g->openTolerance;
        float dRhoNR = 0.f;
        if (g->openImpedance) {
            if (impedance) {
                const float cs2 = cs * cs;
                const float bracket = uNormalRef + cs + 1.f;
                const float t = uNormalRef - dRhoZ;
                const float Dq = fmaf(bracket, bracket, cs2);
                const float B = fmaf(bracket, cs + t, -cs2 * dRhoRef);
                const float H = fmaf(-t, 2.f * cs + t, 2.f * cs2 * dRhoRef);
                const float disc = fmaf(Dq, H, B * B);
                dRhoNR = H / (B + sqrtf(disc));
            }
            bc.nonReflective = 0;
        }
        if (bc.dirichletRho && impedance) {
            if (bc.dRho < dRhoNR - tol) bc.dRho = dRhoNR - tol;
            if (bc.dRho > dRhoNR + tol) bc.dRho = dRhoNR + tol;
        }
        if (bc.dirichletU && impedance) {
            const float uMin = (dRhoZ - dRhoNR - tol) / (dRhoNR + 1.f + tol);
            const float uMax = (dRhoZ - dRhoNR + tol) / (dRhoNR + 1.f - tol);
            float* comp[3] = {&bc.ux, &bc.uy, &bc.uz};
            for (int a = 0; a < 3; ++a) {
                if (on[a] == 0) continue;
                const float lo = on[a] > 0 ? uMin : -uMax, hi = on[a] > 0 ? uMax : -uMin;
                if (*comp[a] < lo) *comp[a] = lo;
                if (*comp[a] > hi) *comp[a] = hi;
            }
        }
        if (bc.dirichletRho) {
            if (bc.nonReflective) {
                const float dRhoTarget = bc.dRho;
                const float rhoTarget = dRhoTarget + 1.f;
                const float rhoTerm = ((dRhoZ - dRhoTarget) / rhoTarget);
                const float numerator = 2.f * (uNormalRef + cs * rhoTerm);
                const float rootContent = (1.f + cs - uNormalRef) * (1.f + cs - uNormalRef) +
                                          4.f * (uNormalRef + cs * rhoTerm);
                const float denominator = 1.f + cs - uNormalRef + sqrtf(rootContent);
                const float uNormal = numerator / denominator;
                bc.dRho = (dRhoZ - uNormal) / (1.f + uNormal);
            }
            float u[3];
            oracle_mbbc_restore_u(code, bc.dRho + 1.f, f, u);
            bc.ux = u[0]; bc.uy = u[1]; bc.uz = u[2];
        } else if (bc.dirichletU) {
            if (bc.nonReflective) {
                float uT = 0.f;
                if (on[0] > 0) uT = bc.ux;
                if (on[0] < 0) uT = -bc.ux;
                if (on[1] > 0) uT = bc.uy;
                if (on[1] < 0) uT = -bc.uy;
                if (on[2] > 0) uT = bc.uz;
                if (on[2] < 0) uT = -bc.uz;
                const float rhoRef = dRhoRef + 1.f;
                const float rhoTerm = ((dRhoZ - dRhoRef) / rhoRef);
                const float numerator = 2.f * (uT + cs * rhoTerm);
                const float rootContent = (1.f + cs - uT) * (1.f + cs - uT) + 4.f * (uT + cs * rhoTerm);
                const float denominator = 1.f + cs - uT + sqrtf(rootContent);
                const float uNormal = numerator / denominator;
                if (on[0] > 0) bc.ux = uNormal;
                if (on[0] < 0) bc.ux = -uNormal;
                if (on[1] > 0) bc.uy = uNormal;
                if (on[1] < 0) bc.uy = -uNormal;
                if (on[2] > 0) bc.uz = uNormal;
                if (on[2] < 0) bc.uz = -uNormal;
            }
            float rho;
            oracle_mbbc_restore_rho(code, bc.ux, bc.uy, bc.uz, f, &rho);
            bc.dRho = rho - 1.f;
        }
        oracle_mbbc_apply(code, bc.dRho + 1.f, bc.ux, bc.uy, bc.uz, f);
        for (int d = 0; d < 27; ++d) {
            if (!(on[0] * CX[d] < 0 || on[1] * CY[d] < 0 || on[2] * CZ[d] < 0)) continue;
            f[d] -= W[d];
            g->f[(size_t)(g->flip ? INV[d] : d) * n + nb[pre_nbr(d)]] = f[d];
        }
        const float uNormal = (float)on[0] * bc.ux + (float)on[1] * bc.uy + (float)on[2] * bc.uz;
        if (g->openImpedance) {
            g->openRef[q] = bc.dRho;  /* the completed state */
            g->openRef[m + q] = uNormal;
        } else {
            const float beta = bc.nonReflectiveBeta;
            float alpha = beta / (g->iterationsFinished + beta + 10.f);
            int updateEvery = 1;
            while (alpha < 1.e-5f) { alpha *= 3.f; updateEvery *= 3; }
            if (g->iterationsFinished % updateEvery == 0) {
                g->openRef[q] = fmaf(alpha, bc.dRho - dRhoRef, dRhoRef);
                g->openRef[m + q] = fmaf(alpha, uNormal - uNormalRef, uNormalRef);
            }
        }
        if (!g->trackOpen || !trackFlow) continue;
        g->openCum[q] += bc.dRho;
        g->openCum[m + q] += uNormal;
    }
}

/* ---- rotors (include/rotorFunctions.h) ---------------------------------- */

typedef struct orotor {
    float res, xMin, yMin, zMin, xMax, yMax, zMax;
    int cntX, cntY, cntZ, axis;
    float ox, oy, oz, radiansPerSecond;
    double radiansElapsed;
    int blocks, nonzero;
    int* rotorMap;
    unsigned* interp;
    float* force;
} orotor;

int oracle_set_rotor(ogrid* g, int r, float res, const float* bounds, const int* cellCount, int axis,
                     const float* origin, float radiansPerSecond, const int* rotorMap, int blocks,
                     const unsigned* interpolation, int nonzero) {
    if (r < 0 || r >= 4) return -1;
    if (!g->rotors) g->rotors = calloc(4, sizeof(orotor));
    orotor* R = (orotor*)g->rotors + r;
    R->res = res;
    R->xMin = bounds[0]; R->yMin = bounds[1]; R->zMin = bounds[2];
    R->xMax = bounds[3]; R->yMax = bounds[4]; R->zMax = bounds[5];
    R->cntX = cellCount[0]; R->cntY = cellCount[1]; R->cntZ = cellCount[2];
    R->axis = axis;
    R->ox = origin[0]; R->oy = origin[1]; R->oz = origin[2];
    R->radiansPerSecond = radiansPerSecond;
    R->radiansElapsed = 0.0;
    R->blocks = blocks;
    R->nonzero = nonzero;
    R->rotorMap = (int*)malloc(sizeof(int) * (size_t)(blocks > 0 ? blocks : 1));
    memcpy(R->rotorMap, rotorMap, sizeof(int) * (size_t)blocks);
    R->interp = (unsigned*)malloc(sizeof(unsigned) * 64 * (size_t)(nonzero > 0 ? nonzero : 1));
    memcpy(R->interp, interpolation, sizeof(unsigned) * 64 * (size_t)nonzero);
    R->force = (float*)calloc(3 * 27 * (size_t)(nonzero > 0 ? nonzero : 1), sizeof(float));
    if (r + 1 > g->rotorCount) g->rotorCount = r + 1;
    return 0;
}

/* buildRotors for one rotor (include/rotorFunctions.h:315-470): voxelize the
 * rotor at half the level spacing over its own bounds, flag every 4x4x4 block
 * of interpolation cells whose 6x6x6 voxel neighbourhood holds rotor volume,
 * and pack per interpolation cell the eight 4-bit corner counts (how many of
 * the 2x2x2 voxels around each corner are inside). */
static int build_rotor(ogrid* g, int r, const lbm_rotor* rt) {
    if (!rt->triangles || rt->axis < 0 || rt->axis > 2) return -1;
    ostl t;
    if (ostl_load(&t, rt->triangles, rt->triangle_count) == 0) { ostl_free(&t); return -1; }
    const float vres = g->res * 0.5f;
    const int vnx = (int)((t.xMax - t.xMin) / vres) + 2;
    const int vny = (int)((t.yMax - t.yMin) / vres) + 2;
    const int vnz = (int)((t.zMax - t.zMin) / vres) + 2;
    oraymap m;
    oray_voxelize(&m, &t, t.xMin, t.yMin, t.zMin, vres, vnx, vny);
    (void)vnz;
    float bounds[6];
    bounds[0] = t.xMin - 1.5f * vres;
    bounds[1] = t.yMin - 1.5f * vres;
    bounds[2] = t.zMin - 1.5f * vres;
    int cnt[3];
    cnt[0] = ((vnx + 2 + 3) / 4) * 4;
    cnt[1] = ((vny + 2 + 3) / 4) * 4;
    cnt[2] = ((vnz + 2 + 3) / 4) * 4;
    bounds[3] = bounds[0] + vres * (float)cnt[0];
    bounds[4] = bounds[1] + vres * (float)cnt[1];
    bounds[5] = bounds[2] + vres * (float)cnt[2];
    ostl_free(&t);
    const int bx = cnt[0] / 4, by = cnt[1] / 4, bz = cnt[2] / 4, bxy = bx * by, blocks = bx * by * bz;
    int* rotorMap = (int*)malloc(sizeof(int) * (size_t)blocks);
    unsigned char(*marks)[216] = malloc(sizeof(*marks) * (size_t)blocks);
    int nonzero = 0;
    for (int b = 0; b < blocks; ++b) {
        const int kb = b / bxy, rem = b % bxy, jb = rem / bx, ib = rem % bx;
        memset(marks[b], 0, 216);
        int any = 0;
        for (int jc = (jb * 4 - 2 > 0 ? jb * 4 - 2 : 0); jc < (vny < jb * 4 + 4 ? vny : jb * 4 + 4); ++jc)
            for (int ic = (ib * 4 - 2 > 0 ? ib * 4 - 2 : 0); ic < (vnx < ib * 4 + 4 ? vnx : ib * 4 + 4); ++ic)
                for (int kc = kb * 4 - 2; kc < kb * 4 + 4; ++kc)
                    if (oray_solid(&m, ic, jc, kc)) {
                        marks[b][(kc - (kb * 4 - 2)) * 36 + (jc - (jb * 4 - 2)) * 6 + (ic - (ib * 4 - 2))] = 1;
                        any = 1;
                    }
        rotorMap[b] = any ? nonzero++ : -1;
    }
    oray_free(&m);
    unsigned* interp = (unsigned*)calloc(64 * (size_t)(nonzero > 0 ? nonzero : 1), sizeof(unsigned));
    int* index = (int*)malloc(sizeof(int) * (size_t)(nonzero > 0 ? nonzero : 1));
    for (int b = 0; b < blocks; ++b) {
        const int z = rotorMap[b];
        if (z < 0) continue;
        index[z] = b;
        unsigned char counter[125];
        for (int kc = 0; kc < 5; ++kc)
            for (int jc = 0; jc < 5; ++jc)
                for (int ic = 0; ic < 5; ++ic) {
                    int v = 0;
                    for (int km = kc; km <= kc + 1; ++km)
                        for (int jm = jc; jm <= jc + 1; ++jm)
                            for (int im = ic; im <= ic + 1; ++im) v += marks[b][km * 36 + jm * 6 + im];
                    counter[kc * 25 + jc * 5 + ic] = (unsigned char)v;
                }
        for (int ki = 0; ki < 4; ++ki)
            for (int ji = 0; ji < 4; ++ji)
                for (int ii = 0; ii < 4; ++ii) {
                    unsigned packed = 0u;
                    unsigned corner = 0;
                    for (int kc = ki; kc <= ki + 1; ++kc)
                        for (int jc = ji; jc <= ji + 1; ++jc)
                            for (int ic = ii; ic <= ii + 1; ++ic, ++corner)
                                packed |= (unsigned)counter[kc * 25 + jc * 5 + ic] << (4u * corner);
                    interp[(size_t)z * 64 + ki * 16 + ji * 4 + ii] = packed;
                }
    }
    free(marks);
    const int rc = oracle_set_rotor(g, r, vres, bounds, cnt, rt->axis, rt->origin, rt->radians_per_second, rotorMap,
                                    blocks, interp, nonzero);
    free(rotorMap);
    free(interp);
    free(index);
    return rc;
}

int oracle_rotor_tables(const ogrid* g, int r, float* res, float* bounds, int* cellCount, int* blocks, int* nonzero,
                        const int** rotorMap, const unsigned** interpolation) {
    if (r < 0 || r >= g->rotorCount || !g->rotors) return -1;
    const orotor* R = (const orotor*)g->rotors + r;
    *res = R->res;
    bounds[0] = R->xMin; bounds[1] = R->yMin; bounds[2] = R->zMin;
    bounds[3] = R->xMax; bounds[4] = R->yMax; bounds[5] = R->zMax;
    cellCount[0] = R->cntX; cellCount[1] = R->cntY; cellCount[2] = R->cntZ;
    *blocks = R->blocks;
    *nonzero = R->nonzero;
    *rotorMap = R->rotorMap;
    *interpolation = R->interp;
    return 0;
}

void oracle_rotor_bins(const ogrid* g, int r, float* out) {
    const orotor* R = (const orotor*)g->rotors + r;
    memcpy(out, R->force, sizeof(float) * 3 * 27 * (size_t)R->nonzero);
}

static void free_rotors(ogrid* g) {
    if (!g->rotors) return;
    orotor* R = (orotor*)g->rotors;
    for (int r = 0; r < g->rotorCount; ++r) { free(R[r].rotorMap); free(R[r].interp); free(R[r].force); }
    free(g->rotors);
    g->rotors = NULL;
    g->rotorCount = 0;
}

/* processRotor (include/rotorFunctions.h:211-304) for every rotor, with the
 * cumulative fraction cap and break of include/updateGrid.h:113-128 */
static void rotor_forcing(ogrid* g, float x, float y, float z, float rho, float uxPre, float uyPre, float uzPre,
                          int trackForce, obc* bc) {
    float cum = 0.f;
    for (int r = 0; r < g->rotorCount; ++r) {
        orotor* R = (orotor*)g->rotors + r;
        const float angle = (float)R->radiansElapsed;
        const float c = cosf(angle), s = sinf(angle);
        float xr = x, yr = y, zr = z;
        const float dx = x - R->ox, dy = y - R->oy, dz = z - R->oz;
        if (R->axis == 0) { yr = R->oy + c * dy + s * dz; zr = R->oz - s * dy + c * dz; }
        else if (R->axis == 1) { xr = R->ox + c * dx - s * dz; zr = R->oz + s * dx + c * dz; }
        else { xr = R->ox + c * dx + s * dy; yr = R->oy - s * dx + c * dy; }
        if (xr < R->xMin || xr >= R->xMax || yr < R->yMin || yr >= R->yMax || zr < R->zMin || zr >= R->zMax) continue;
        const float xRel = xr - R->xMin, yRel = yr - R->yMin, zRel = zr - R->zMin;
        const int ii = (int)(xRel / R->res), jj = (int)(yRel / R->res), kk = (int)(zRel / R->res);
        if (ii >= R->cntX || jj >= R->cntY || kk >= R->cntZ) continue;
        const int bx = R->cntX / 4, by = R->cntY / 4;
        const int block = (kk / 4) * bx * by + (jj / 4) * bx + ii / 4;
        const int map = R->rotorMap[block];
        if (map < 0) continue;
        const unsigned packed = R->interp[map * 64 + (kk % 4) * 16 + (jj % 4) * 4 + (ii % 4)];
        const float xw = (xRel / R->res) - ii, yw = (yRel / R->res) - jj, zw = (zRel / R->res) - kk;
        float v[8];
        for (int q = 0; q < 8; ++q) v[q] = (float)((packed >> (4u * q)) & 0xFu);
        const float v00 = v[0] + xw * (v[1] - v[0]);
        const float v10 = v[2] + xw * (v[3] - v[2]);
        const float v01 = v[4] + xw * (v[5] - v[4]);
        const float v11 = v[6] + xw * (v[7] - v[6]);
        const float v0 = v00 + yw * (v10 - v00);
        const float v1 = v01 + yw * (v11 - v01);
        const float frac = (v0 + zw * (v1 - v0)) * 0.125f;
        if (frac == 0.f) continue;
        /* getRotorForcing: rho (u_target - u) with rigid rotation about the axis */
        const float scale = R->radiansPerSecond * g->dtPhys / g->res;
        float ut[3] = {0.f, 0.f, 0.f};
        if (R->axis == 0) { ut[1] = -scale * dz; ut[2] = scale * dy; }
        else if (R->axis == 1) { ut[0] = scale * dz; ut[2] = -scale * dx; }
        else { ut[0] = -scale * dy; ut[1] = scale * dx; }
        float gx = rho * (ut[0] - uxPre), gy = rho * (ut[1] - uyPre), gz = rho * (ut[2] - uzPre);
        float ff = frac * frac * (3.f - 2.f * frac);
        if (cum + ff > 1.f) { ff = 1.f - cum; cum = 1.f; }
        else cum += ff;
        gx *= ff; gy *= ff; gz *= ff;
        bc->gx += gx; bc->gy += gy; bc->gz += gz;
        if (g->trackRotorForce && trackForce) {
            float fx = gx, fy = gy, fz = gz;
            if (R->axis == 0) { fy = c * gy + s * gz; fz = -s * gy + c * gz; }
            else if (R->axis == 1) { fx = c * gx - s * gz; fz = s * gx + c * gz; }
            else { fx = c * gx + s * gy; fy = -s * gx + c * gy; }
            int iF = (int)(0.75f * ((ii % 4) + xw)), jF = (int)(0.75f * ((jj % 4) + yw)), kF = (int)(0.75f * ((kk % 4) + zw));
            iF = iF < 0 ? 0 : (iF > 2 ? 2 : iF);
            jF = jF < 0 ? 0 : (jF > 2 ? 2 : jF);
            kF = kF < 0 ? 0 : (kF > 2 ? 2 : kF);
            const int bin = map * 27 + kF * 9 + jF * 3 + iF, nb = 27 * R->nonzero;
#pragma omp atomic
            R->force[bin] += fx;
#pragma omp atomic
            R->force[nb + bin] += fy;
#pragma omp atomic
            R->force[2 * nb + bin] += fz;
        }
        if (cum >= 1.f) break;
    }
    if (cum > 0.f) bc->collisionLimiter *= 1.f - (cum < 0.f ? 0.f : (cum > 1.f ? 1.f : cum));
}

/* getRotorFraction (include/rotorFunctions.h:155-209) */
static float rotor_fraction(const orotor* R, float x, float y, float z) {
    const float angle = (float)R->radiansElapsed;
    const float c = cosf(angle), s = sinf(angle);
    float xr = x, yr = y, zr = z;
    const float dx = x - R->ox, dy = y - R->oy, dz = z - R->oz;
    if (R->axis == 0) { yr = R->oy + c * dy + s * dz; zr = R->oz - s * dy + c * dz; }
    else if (R->axis == 1) { xr = R->ox + c * dx - s * dz; zr = R->oz + s * dx + c * dz; }
    else { xr = R->ox + c * dx + s * dy; yr = R->oy - s * dx + c * dy; }
    if (xr < R->xMin || xr >= R->xMax || yr < R->yMin || yr >= R->yMax || zr < R->zMin || zr >= R->zMax) return 0.f;
    const float xRel = xr - R->xMin, yRel = yr - R->yMin, zRel = zr - R->zMin;
    const int ii = (int)(xRel / R->res), jj = (int)(yRel / R->res), kk = (int)(zRel / R->res);
    if (ii >= R->cntX || jj >= R->cntY || kk >= R->cntZ) return 0.f;
    const int bx = R->cntX / 4, by = R->cntY / 4;
    const int map = R->rotorMap[(kk / 4) * bx * by + (jj / 4) * bx + ii / 4];
    if (map < 0) return 0.f;
    const unsigned packed = R->interp[map * 64 + (kk % 4) * 16 + (jj % 4) * 4 + (ii % 4)];
    const float xw = (xRel / R->res) - ii, yw = (yRel / R->res) - jj, zw = (zRel / R->res) - kk;
    float v[8];
    for (int q = 0; q < 8; ++q) v[q] = (float)((packed >> (4u * q)) & 0xFu);
    const float v00 = v[0] + xw * (v[1] - v[0]), v10 = v[2] + xw * (v[3] - v[2]);
    const float v01 = v[4] + xw * (v[5] - v[4]), v11 = v[6] + xw * (v[7] - v[6]);
    const float v0 = v00 + yw * (v10 - v00), v1 = v01 + yw * (v11 - v01);
    return (v0 + zw * (v1 - v0)) * 0.125f;
}

/* Section image of getFlowReportGeneral over every level of a domain
 * (include/flowReportFunctions.h:11-318); see oracle_flow_image in the header. */
static float rotor_marker(const ogrid* g, float x, float y, float z) {
    float m = 0.f;
    for (int r = 0; r < g->rotorCount; ++r) m += rotor_fraction((const orotor*)g->rotors + r, x, y, z);
    return m < 0.f ? 0.f : (m > 1.f ? 1.f : m);
}

static void read_macro(const ogrid* g, int cell, float m[4]) {
    const size_t n = (size_t)g->cellCount;
    int nb[8];
    get_nbr(g, cell, nb);
    float f[27];
    for (int d = 0; d < 27; ++d) f[d] = g->f[(size_t)(g->flip ? INV[d] : d) * n + nb[pre_nbr(d)]];
    oracle_get_drho_u(f, m);
}

int oracle_flow_image(const odomain* dom, int plane, float cut, const float* bounds, double* out, int* imageLevelOut) {
    const long long limit = 16000000;
    const int levels = dom->levelCount;
    const ogrid* fin = &dom->level[levels - 1];
    const int n[3] = {fin->nx, fin->ny, fin->nz};
    const float o[3] = {fin->ox, fin->oy, fin->oz};
    const int axis = plane == 0 ? 2 : (plane == 1 ? 0 : 1);
    const int cutIndex = (int)((cut - o[axis]) / fin->res + 0.5f);
    if (cutIndex < 0 || cutIndex >= n[axis]) return -1;
    const double cutPosition = (double)o[axis] + (double)cutIndex * fin->res;
    int lo[3] = {0, 0, 0}, hi[3] = {n[0], n[1], n[2]};
    if (bounds && (bounds[0] != 0.f || bounds[1] != 0.f || bounds[2] != 0.f || bounds[3] != 0.f || bounds[4] != 0.f ||
                   bounds[5] != 0.f))
        for (int a = 0; a < 3; ++a) {
            const float tMin = o[a] - 0.5f * fin->res, tMax = o[a] + fin->res * (n[a] - 0.5f);
            const int l0 = (int)ceilf((bounds[a] - tMin) / fin->res);
            const int h0 = n[a] - (int)ceilf((tMax - bounds[a + 3]) / fin->res);
            lo[a] = l0 > 0 ? l0 : 0;
            hi[a] = h0 < n[a] ? h0 : n[a];
        }
    const int hA = plane == 0 ? 0 : 2, vA = plane == 2 ? 0 : 1;
    int pH = hi[hA] - lo[hA], pV = hi[vA] - lo[vA], sH = lo[hA], sV = lo[vA];
    int imageLevel = levels - 1;
    long long pixels = (long long)pH * pV;
    while (pixels > limit && imageLevel > 0) {
        --imageLevel;
        pH /= 2; sH /= 2; pV /= 2; sV /= 2;
        pixels = (long long)pH * pV;
    }
    if (pH <= 0 || pV <= 0 || pixels > limit) return -2;
    float* img = (float*)malloc(3 * (size_t)pixels * sizeof(float));
    if (!img) return -3;
    for (long long p = 0; p < pixels; ++p) { img[p] = 0.f; img[pixels + p] = 0.f; img[2 * pixels + p] = 1.f; }
    for (int l = 0; l < levels; ++l) {
        const ogrid* g = &dom->level[l];
        const int count = plane == 0 ? g->nz : (plane == 1 ? g->nx : g->ny);
        if (g->cellCount <= 0 || count <= 0) continue;
        const double origin = plane == 0 ? g->oz : (plane == 1 ? g->ox : g->oy);
        double index = (cutPosition - origin) / (double)g->res;
        if (index < 0.0) index = 0.0;
        if (index > count - 1) index = count - 1;
        const int lower = (int)floor(index);
        const float alpha = (float)(index - lower);
        const int interpolate = alpha > 0.f;
        const int down = l > imageLevel ? 1 << (l - imageLevel) : 1, up = l < imageLevel ? 1 << (imageLevel - l) : 1;
        for (int cell = 0; cell < g->cellCount; ++cell) {
            int ci, cj, ck;
            get_ijk(g, cell, &ci, &cj, &ck);
            if ((plane == 0 ? ck : (plane == 1 ? ci : cj)) != lower) continue;
            const int ch = plane == 0 ? ci : ck, cv = plane == 2 ? ci : cj;
            if (ch % down || cv % down) continue;
            const int ih = (ch / down) * up, iv = (cv / down) * up;
            if (ih + up <= sH || ih >= sH + pH || iv + up <= sV || iv >= sV + pV) continue;
            int upper = cell;
            if (interpolate) {
                int nb[8];
                get_nbr(g, cell, nb);
                upper = plane == 0 ? nb[4] : (plane == 1 ? nb[1] : nb[2]);
                if (upper < 0 || upper >= g->cellCount) continue;
                int ui, uj, uk;
                get_ijk(g, upper, &ui, &uj, &uk);
                if (ui != ci + (plane == 1) || uj != cj + (plane == 2) || uk != ck + (plane == 0)) continue;
            }
            const int lowerSolid = g->wallMap[cell] == -3, upperSolid = g->wallMap[upper] == -3;
            const int solid = alpha <= 0.5f ? lowerSolid : upperSolid;
            float marker = solid ? 1.f : 0.f, m[4] = {0.f, 0.f, 0.f, 0.f};
            if (!solid) {
                read_macro(g, lowerSolid ? upper : cell, m);
                marker = rotor_marker(g, ci * g->res + g->ox, cj * g->res + g->oy, ck * g->res + g->oz);
                if (interpolate && !lowerSolid && !upperSolid) {
                    float mu[4];
                    read_macro(g, upper, mu);
                    for (int q = 0; q < 4; ++q) m[q] += alpha * (mu[q] - m[q]);
                    const float mk = rotor_marker(g, (ci + (plane == 1)) * g->res + g->ox,
                                                  (cj + (plane == 2)) * g->res + g->oy,
                                                  (ck + (plane == 0)) * g->res + g->oz);
                    marker += alpha * (mk - marker);
                }
            }
            const float un = plane == 0 ? m[3] : (plane == 1 ? m[1] : m[2]);
            for (int yv = 0; yv < up; ++yv) {
                const int y = iv + yv - sV;
                if (y < 0 || y >= pV) continue;
                for (int xh = 0; xh < up; ++xh) {
                    const int x = ih + xh - sH;
                    if (x < 0 || x >= pH) continue;
                    const long long p = (long long)y * pH + x;
                    img[p] = m[0];
                    img[pixels + p] = un;
                    img[2 * pixels + p] = marker;
                }
            }
        }
    }
    for (int q = 0; q < 6; ++q) out[q] = 0.0;
    for (long long p = 0; p < pixels; ++p) {
        if (!(img[2 * pixels + p] < 0.5f)) continue;
        const float dRho = img[p], u = img[pixels + p];
        const float rhoU = fmaf(dRho, u, u);
        out[0] += u;
        out[1] += dRho * u;
        out[2] += rhoU * fabsf(u);
        out[3] += dRho;
        out[4] += 0.5f * rhoU * u * u;
        out[5] += 1.0;
    }
    free(img);
    *imageLevelOut = imageLevel;
    return 0;
}

void oracle_flow_sums(const ogrid* g, int plane, int layer, int h0, int h1, int v0, int v1, double* out) {
    for (int q = 0; q < 6; ++q) out[q] = 0.0;
    const size_t n = (size_t)g->cellCount;
    for (int cell = 0; cell < g->cellCount; ++cell) {
        int ci, cj, ck;
        get_ijk(g, cell, &ci, &cj, &ck);
        const int normal = plane == 0 ? ck : (plane == 1 ? ci : cj);
        const int horiz = plane == 0 ? ci : ck;
        const int vert = plane == 2 ? ci : cj;
        if (normal != layer || horiz < h0 || horiz >= h1 || vert < v0 || vert >= v1) continue;
        if (g->wallMap[cell] == -3) continue;
        int nb[8];
        get_nbr(g, cell, nb);
        float f[27], m[4];
        for (int d = 0; d < 27; ++d) f[d] = g->f[(size_t)(g->flip ? INV[d] : d) * n + nb[pre_nbr(d)]];
        oracle_get_drho_u(f, m);
        float marker = 0.f;
        const float x = ci * g->res + g->ox, y = cj * g->res + g->oy, z = ck * g->res + g->oz;
        for (int r = 0; r < g->rotorCount; ++r) marker += rotor_fraction((const orotor*)g->rotors + r, x, y, z);
        marker = marker < 0.f ? 0.f : (marker > 1.f ? 1.f : marker);
        if (!(marker < 0.5f)) continue;
        const float u = plane == 0 ? m[3] : (plane == 1 ? m[1] : m[2]);
        const float rhoU = fmaf(m[0], u, u);
        out[0] += u;
        out[1] += m[0] * u;
        out[2] += rhoU * fabsf(u);
        out[3] += m[0];
        out[4] += 0.5f * rhoU * u * u;
        out[5] += 1.0;
    }
}

/* ---- updateSingleGrid (include/updateGrid.h:16-386) --------------------- */
void oracle_step(ogrid* g, int steps) {
    const long long n = g->cellCount;
    for (int s = 0; s < steps; ++s) {
        const int flip = g->flip;
        /* advance the rotors (include/updateGrid.h:36-49) */
        for (int r = 0; r < g->rotorCount; ++r) {
            orotor* R = (orotor*)g->rotors + r;
            const double twoPi = 6.283185307179586476925286766559;
            R->radiansElapsed = fmod(R->radiansElapsed + (double)g->dtPhys * R->radiansPerSecond, twoPi);
            if (R->radiansElapsed < 0.0) R->radiansElapsed += twoPi;
            if (R->radiansElapsed >= twoPi) R->radiansElapsed = 0.0;
        }
        /* K1: cell lambda (:51-177) */
#pragma omp parallel for schedule(static)
        for (int cell = 0; cell < g->cellCount; ++cell) {
            const int wm = g->wallMap[cell];
            if (wm == -3) continue;
            int nb[8];
            get_nbr(g, cell, nb);
            float f[27];
            for (int d = 0; d < 27; ++d) f[d] = g->f[(size_t)(flip ? INV[d] : d) * n + nb[pre_nbr(d)]];
            obc bc;
            oracle_default_bc(&bc);
            float m[4];
            oracle_get_drho_u(f, m);
            bc.dRho = m[0]; bc.ux = m[1]; bc.uy = m[2]; bc.uz = m[3];
            unsigned wallData = 0u;
            if (wm >= 0) {
                wallData = g->wallData[wm];
                bc.wallID = (int)((wallData >> 27) & 31u);
            }
            /* getLocalBC: limiter, forcing, IBB switch and the wall velocity */
            bc.collisionLimiter = g->limiter;
            bc.nuMultiplier = g->nuMultiplier;
            bc.gx = g->gx; bc.gy = g->gy; bc.gz = g->gz;
            bc.useIBB = g->useIBB;
            if (wm >= 0) {
                bc.ux = g->wallVel[wm];
                bc.uy = g->wallVel[g->wallCount + wm];
                bc.uz = g->wallVel[2 * g->wallCount + wm];
            }
            if (g->rotorCount > 0) {
                /* include/updateGrid.h:97-128 */
                int ci, cj, ck;
                get_ijk(g, cell, &ci, &cj, &ck);
                const float x = ci * g->res + g->ox, y = cj * g->res + g->oy, z = ck * g->res + g->oz;
                const float rho = m[0] + 1.f;
                const float rhoInv = 1.f / rho;
                const float uxPre = (m[1] * rho + bc.gx) * rhoInv;
                const float uyPre = (m[2] * rho + bc.gy) * rhoInv;
                const float uzPre = (m[3] * rho + bc.gz) * rhoInv;
                const int track = wm != -2 && !(wm >= 0 && (wallData & 1u));
                rotor_forcing(g, x, y, z, rho, uxPre, uyPre, uzPre, track, &bc);
            }
            oracle_apply_collision(f, &bc, g->nu);
            if (wm < 0) {
                for (int d = 0; d < 27; ++d) g->f[(size_t)(flip ? d : INV[d]) * n + nb[post_nbr(d)]] = f[d];
                continue;
            }
            /* applyIBB (interpolatedBouncebackFunctions.h:43-157) */
            float dr[4];
            oracle_get_drho_u(f, dr);
            float res[27];
            for (int d = 0; d < 27; ++d) res[d] = f[d];
            float gxw = 0.f, gyw = 0.f, gzw = 0.f;
            int linkIndex = 0;
            unsigned code = 0u;
            for (int d = 1; d < 27; ++d) {
                if (!(wallData & (1u << d))) continue;
                const int id = INV[d];
                const float eiDotFi = (float)CX[id] * bc.ux + (float)CY[id] * bc.uy + (float)CZ[id] * bc.uz;
                const float wallTerm = 6.f * W[id] * (1.f + dr[0]) * eiDotFi;
                float gamma = 0.5f;
                if (bc.useIBB) {
                    if (linkIndex % 4 == 0) code = g->linkLength[(size_t)(linkIndex / 4) * g->wallCount + wm];
                    const unsigned c8 = (code >> (8 * (linkIndex % 4))) & 255u;
                    gamma = (float)c8 / 254.f;
                    if (gamma < 0.01f) gamma = 0.01f;
                    if (gamma > 1.f) gamma = 1.f;
                    ++linkIndex;
                }
                const float fPre = g->f[(size_t)(flip ? INV[d] : d) * n + nb[pre_nbr(d)]];
                const float invDen = 1.f / (1.f + gamma);
                const float r = ((1.f - gamma) * invDen) * fPre + (gamma * invDen) * f[id] +
                                (gamma * invDen) * f[d] + invDen * wallTerm;
                gxw += -(f[d]) * (CX[d] - bc.ux) + (r) * (CX[id] - bc.ux);
                gyw += -(f[d]) * (CY[d] - bc.uy) + (r) * (CY[id] - bc.uy);
                gzw += -(f[d]) * (CZ[d] - bc.uz) + (r) * (CZ[id] - bc.uz);
                res[d] = r;
            }
            /* writes (updateGrid.h:150-170) */
            for (int d = 0; d < 27; ++d) {
                const int linked = d != 0 && (wallData & (1u << d));
                if (linked) {
                    /* next pre-collision slot of the inverse direction */
                    g->f[(size_t)(flip ? INV[d] : d) * n + nb[post_nbr(d)]] = res[d];
                } else {
                    g->f[(size_t)(flip ? d : INV[d]) * n + nb[post_nbr(d)]] = res[d];
                }
            }
            if (g->trackWallForce && !(wallData & 1u)) {
                g->wallForce[wm] += gxw;
                g->wallForce[g->wallCount + wm] += gyw;
                g->wallForce[2 * g->wallCount + wm] += gzw;
            }
        }
        /* applyStreaming (esotwistStreamingFunctions.h:6-9) */
        g->flip = !flip;
        /* K2: open boundaries (:181-355) */
        open_boundary(g);
        /* K3: periodic copy (:358-382) */
#pragma omp parallel for schedule(static)
        for (int p = 0; p < g->perCount; ++p) {
            int nb[8];
            float f[27];
            get_nbr(g, g->perSource[p], nb);
            for (int d = 0; d < 27; ++d) f[d] = g->f[(size_t)(g->flip ? INV[d] : d) * n + nb[pre_nbr(d)]];
            get_nbr(g, g->perIndex[p], nb);
            for (int d = 0; d < 27; ++d) g->f[(size_t)(g->flip ? INV[d] : d) * n + nb[pre_nbr(d)]] = f[d];
        }
        g->iterationsFinished++;
    }
}

/* K1 over cells [c0, c1) only, without the flip: a bounded slice of one step
 * for timing the CPU implementation on large grids. */
void oracle_collide_range(ogrid* g, int c0, int c1) {
    const long long n = g->cellCount;
    const int flip = g->flip;
    if (c0 < 0) c0 = 0;
    if (c1 > g->cellCount) c1 = g->cellCount;
#pragma omp parallel for schedule(static)
    for (int cell = c0; cell < c1; ++cell) {
        if (g->wallMap[cell] == -3) continue;
        int nb[8];
        get_nbr(g, cell, nb);
        float f[27];
        for (int d = 0; d < 27; ++d) f[d] = g->f[(size_t)(flip ? INV[d] : d) * n + nb[pre_nbr(d)]];
        obc bc;
        oracle_default_bc(&bc);
        float m[4];
        oracle_get_drho_u(f, m);
        bc.dRho = m[0]; bc.ux = m[1]; bc.uy = m[2]; bc.uz = m[3];
        bc.collisionLimiter = g->limiter;
        bc.nuMultiplier = g->nuMultiplier;
        oracle_apply_collision(f, &bc, g->nu);
        for (int d = 0; d < 27; ++d) g->f[(size_t)(flip ? d : INV[d]) * n + nb[post_nbr(d)]] = f[d];
    }
}

/* FP64 sums over the fluid cells (walls, periodic ghosts and interface
 * duplicates excluded): out = {sum rho, sum dRho, sum c_x f, sum c_y f,
 * sum c_z f, cells}, lattice units. */
void oracle_global_sums(const ogrid* g, double* out) {
    for (int q = 0; q < 6; ++q) out[q] = 0.0;
    const int n = g->cellCount;
    for (int c = 0; c < n; ++c) {
        const int wm = g->wallMap[c];
        if (wm == -3 || wm == -2) continue;
        if (wm >= 0 && (g->wallData[wm] & 1u)) continue;
        int nb[8];
        get_nbr(g, c, nb);
        double dRho = 0.0, m[3] = {0.0, 0.0, 0.0};
        for (int d = 0; d < 27; ++d) {
            const int slot = g->flip ? INV[d] : d;
            const double f = g->f[(size_t)slot * n + nb[pre_nbr(d)]];
            dRho += f;
            m[0] += CX[d] * f;
            m[1] += CY[d] * f;
            m[2] += CZ[d] * f;
        }
        out[0] += 1.0 + dRho;
        out[1] += dRho;
        out[2] += m[0];
        out[3] += m[1];
        out[4] += m[2];
        out[5] += 1.0;
    }
}

double oracle_kinetic_energy(const ogrid* g, float uRefPhys, float domainLength) {
    const long long n = g->cellCount;
    double sum = 0.0;
#pragma omp parallel for reduction(+ : sum) schedule(static)
    for (int cell = 0; cell < g->cellCount; ++cell) {
        const int wm = g->wallMap[cell];
        if (wm == -3 || wm == -2) continue;
        if (wm >= 0 && (g->wallData[wm] & 1u)) continue;
        int nb[8];
        get_nbr(g, cell, nb);
        float f[27], m[4];
        for (int d = 0; d < 27; ++d) f[d] = g->f[(size_t)(g->flip ? INV[d] : d) * n + nb[pre_nbr(d)]];
        oracle_get_drho_u(f, m);
        sum += 0.5 * (1.0 + (double)m[0]) * ((double)m[1] * m[1] + (double)m[2] * m[2] + (double)m[3] * m[3]);
    }
    const double dx = (double)g->res / 1000.0;
    const double vs = dx / ((double)g->dtPhys * uRefPhys);
    const double len = (double)domainLength / 1000.0;
    return sum * dx * dx * dx * vs * vs / (len * len * len);
}

void oracle_macro(const ogrid* g, float* out) {
    const long long n = g->cellCount;
#pragma omp parallel for schedule(static)
    for (int cell = 0; cell < g->cellCount; ++cell) {
        int nb[8];
        get_nbr(g, cell, nb);
        float f[27], m[4];
        for (int d = 0; d < 27; ++d) f[d] = g->f[(size_t)(g->flip ? INV[d] : d) * n + nb[pre_nbr(d)]];
        oracle_get_drho_u(f, m);
        for (int q = 0; q < 4; ++q) out[q * n + cell] = m[q];
    }
}

/* ---- multilevel domains ------------------------------------------------------
 * buildGrids over several levels (include/gridBuilderFunctions.h:9-64,
 * :66-201, :299-739, :741-1231), the recursive time step (updateAllGrids,
 * include/updateGrid.h:388-396) and the interface exchange (updateInterface,
 * include/updateInterface.h:29-891). */

static unsigned char* ucalloc(int n) { return (unsigned char*)calloc((size_t)(n > 0 ? n : 1), 1); }
static int* imalloc(int n) { return (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1)); }

/* initializeGridInfo for a finer level (gridBuilderFunctions.h:50-62) */
static void finer_info(const lbm_case* c, const ogrid* cg, ogrid* fg, int level) {
    init_info(c, fg);
    fg->gridID = level;
    fg->res = cg->res * 0.5f;
    fg->nx = cg->nx * 2; fg->ny = cg->ny * 2; fg->nz = cg->nz * 2;
    fg->ox = cg->ox - fg->res * 0.5f;
    fg->oy = cg->oy - fg->res * 0.5f;
    fg->oz = cg->oz - fg->res * 0.5f;
    fg->dtPhys = cg->dtPhys * 0.5f;
    fg->nu = (fg->dtPhys * c->nu_phys) / ((fg->res / 1000.f) * (fg->res / 1000.f));
}

/* GridBuilderStruct markers of one level while the domain is built
 * (include/types.h:181-190) */
typedef struct omarks {
    unsigned char *deep, *f2c, *c2f, *refine;
    int* parent;
    unsigned char *parentInterface, *parentF2C, *needValues;
    int* wallIDFull;
} omarks;

static void omarks_free(omarks* M) {
    free(M->deep); free(M->f2c); free(M->c2f); free(M->refine); free(M->parent);
    free(M->parentInterface); free(M->parentF2C); free(M->needValues); free(M->wallIDFull);
    memset(M, 0, sizeof(*M));
}

/* spreadMarkers in place: the result replaces `m` */
static void spread_in_place(const ogrid* g, unsigned char* m) {
    unsigned char* t = ucalloc(g->cellCount);
    spread_cells(g, m, t);
    memcpy(m, t, (size_t)g->cellCount);
    free(t);
}

/* markRefinementCells (include/markerFunctions.h:419-450) with markKeepCells
 * (:411-417), markAllFinerFluids/Walls (:222-252) and
 * applyUserRefinementModification (:254-271) */
static void mark_refinement(const lbm_case* c, const ogrid* g, omarks* M, const oraymap* total, int NL) {
    const int n = g->cellCount, lv = g->gridID;
    unsigned char* keep = ucalloc(n);
    M->deep = ucalloc(n);
    for (int q = 0; q < n; ++q)
        for (int m = lv; m < NL; ++m) {
            if (oray_block_has_fluid(&total[m], g->I[q], g->J[q], g->K[q], 1 << (m - lv))) keep[q] = 1;
            if (oray_block_has_wall(&total[m], g->I[q], g->J[q], g->K[q], 1 << (m - lv))) M->deep[q] = 1;
        }
    spread_in_place(g, keep);
    if (lv > 0)
        for (int q = 0; q < n; ++q) keep[q] = keep[q] || M->parentInterface[q];
    for (int r = 0; r < c->wall_refinement_count; ++r) spread_in_place(g, M->deep);
    const float* box = c->refine_box[lv];
    const int useBox = box[0] < box[3] && box[1] < box[4] && box[2] < box[5];
    lbm_grid_info info;
    memset(&info, 0, sizeof(info));
    info.grid_id = g->gridID;
    info.cell_count = n;
    info.cell_count_x = g->nx; info.cell_count_y = g->ny; info.cell_count_z = g->nz;
    info.res = g->res; info.ox = g->ox; info.oy = g->oy; info.oz = g->oz;
    info.nu = g->nu; info.dt_phys = g->dtPhys;
    for (int q = 0; q < n; ++q) {
        int mark = M->deep[q];
        if (useBox) {
            const float x = g->I[q] * g->res + g->ox, y = g->J[q] * g->res + g->oy, z = g->K[q] * g->res + g->oz;
            if (x > box[0] && x < box[3] && y > box[1] && y < box[4] && z > box[2] && z < box[5]) mark = 1;
        }
        if (c->refinement_hook) c->refinement_hook(c->hook_user, g->I[q], g->J[q], g->K[q], &mark, &info);
        M->deep[q] = mark != 0;
    }
    for (int q = 0; q < n; ++q) {
        if (lv > 0 && M->parentInterface[q]) M->deep[q] = 0;
        M->deep[q] = M->deep[q] && keep[q];
    }
    M->f2c = ucalloc(n);
    spread_cells(g, M->deep, M->f2c);
    for (int q = 0; q < n; ++q) M->f2c[q] = M->f2c[q] && keep[q] && !M->deep[q];
    M->c2f = ucalloc(n);
    memcpy(M->c2f, M->f2c, (size_t)n);
    spread_in_place(g, M->c2f);
    spread_in_place(g, M->c2f);
    for (int q = 0; q < n; ++q) M->c2f[q] = M->c2f[q] && keep[q] && !M->deep[q] && !M->f2c[q];
    M->refine = ucalloc(n);
    for (int q = 0; q < n; ++q) M->refine[q] = M->deep[q] || M->f2c[q] || M->c2f[q];
    free(keep);
}

/* buildFinerGridBuilder (gridBuilderFunctions.h:134-201): 8 children of every
 * refinement-marked coarse cell, then sortIJK (:204-234), buildNBRPlus, and
 * buildIJKFull steps 6-7 (parent map, parent-interface marks) */
static void build_finer(const ogrid* cg, const omarks* CM, ogrid* fg, omarks* FM) {
    int count = 0;
    for (int q = 0; q < cg->cellCount; ++q) count += CM->refine[q];
    const int n = 8 * count;
    int* ijk = imalloc(3 * n);
    int w = 0;
    for (int q = 0; q < cg->cellCount; ++q) {
        if (!CM->refine[q]) continue;
        for (int ka = 0; ka < 2; ++ka)
            for (int ja = 0; ja < 2; ++ja)
                for (int ia = 0; ia < 2; ++ia) {
                    ijk[3 * w] = 2 * cg->I[q] + ia;
                    ijk[3 * w + 1] = 2 * cg->J[q] + ja;
                    ijk[3 * w + 2] = 2 * cg->K[q] + ka;
                    ++w;
                }
    }
    qsort(ijk, (size_t)n, 3 * sizeof(int), cmp_kji);
    fg->cellCount = n;
    fg->I = imalloc(n); fg->J = imalloc(n); fg->K = imalloc(n);
    for (int q = 0; q < n; ++q) { fg->I[q] = ijk[3 * q]; fg->J[q] = ijk[3 * q + 1]; fg->K[q] = ijk[3 * q + 2]; }
    free(ijk);
    nbr_plus(fg);
    FM->parent = imalloc(n);
    FM->parentInterface = ucalloc(n);
    FM->parentF2C = ucalloc(n);
    for (int q = 0; q < n; ++q) {
        const int pc = find_cell(cg, fg->I[q] / 2, fg->J[q] / 2, fg->K[q] / 2);
        FM->parent[q] = pc;
        if (pc < 0) continue;
        FM->parentInterface[q] = CM->c2f[pc] || CM->f2c[pc];
        FM->parentF2C[q] = CM->f2c[pc];
    }
}

/* deleteExcessCells (gridBuilderFunctions.h:402-588) for one level */
static void delete_excess(ogrid* g, omarks* M, const ogrid* cg, const oraymap* total, int finest) {
    const int n = g->cellCount;
    if (cg)
        for (int q = 0; q < n; ++q) {
            M->parent[q] = find_cell(cg, g->I[q] / 2, g->J[q] / 2, g->K[q] / 2);
            M->parentInterface[q] = M->parent[q] >= 0;
        }
    unsigned char* keep = ucalloc(n);
    for (int q = 0; q < n; ++q) {
        keep[q] = !oray_solid(total, g->I[q], g->J[q], g->K[q]);
        if (cg && M->parentInterface[q]) keep[q] = 1;
    }
    spread_in_place(g, keep);
    if (!finest)
        for (int q = 0; q < n; ++q) keep[q] = keep[q] && !M->deep[q];
    if (cg) {
        unsigned char* s1 = ucalloc(n);
        unsigned char* s3 = ucalloc(n);
        spread_cells(g, M->parentF2C, s1);
        memcpy(s3, s1, (size_t)n);
        spread_in_place(g, s3);
        spread_in_place(g, s3);
        M->needValues = ucalloc(n);
        for (int q = 0; q < n; ++q) {
            if (M->parentInterface[q] && !s3[q]) keep[q] = 0;
            M->needValues[q] = M->parentInterface[q] && keep[q] && !s1[q];
        }
        free(s1);
        free(s3);
    }
    /* fullToKeep scan and compaction of the per-cell arrays */
    int w = 0;
    for (int q = 0; q < n; ++q) {
        if (!keep[q]) continue;
        g->I[w] = g->I[q]; g->J[w] = g->J[q]; g->K[w] = g->K[q];
        if (cg) { M->parent[w] = M->parent[q]; M->needValues[w] = M->needValues[q]; }
        if (!finest) { M->f2c[w] = M->f2c[q]; M->c2f[w] = M->c2f[q]; }
        ++w;
    }
    g->cellCount = w;
    nbr_plus(g);
    free(keep);
}

/* fillFineToCoarseInterface and fillCoarseToFineInterface
 * (gridBuilderFunctions.h:741-1030) with the child map of :1192-1222 */
static void build_interface(const ogrid* cg, const omarks* CM, const ogrid* fg, const omarks* FM, ointerface* I) {
    const int nc = cg->cellCount, nf = fg->cellCount;
    int* child = imalloc(nc);
    for (int q = 0; q < nc; ++q) child[q] = -1;
    for (int q = 0; q < nf; ++q) {
        const int pc = FM->parent[q];
        if (pc >= 0 && fg->I[q] % 2 == 0 && fg->J[q] % 2 == 0 && fg->K[q] % 2 == 0) child[pc] = q;
    }
    /* fine to coarse: marked coarse cells that are not walls */
    I->f2cCount = 0;
    for (int q = 0; q < nc; ++q) I->f2cCount += CM->f2c[q] && !cg->wallMarker[q];
    I->f2cIndex = imalloc(I->f2cCount);
    I->f2cChild = imalloc(I->f2cCount);
    for (int q = 0, t = 0; q < nc; ++q)
        if (CM->f2c[q] && !cg->wallMarker[q]) { I->f2cIndex[t] = q; I->f2cChild[t] = child[q]; ++t; }
    /* coarse to fine: cells that see a full block of marked coarse cells
     * around the centre of 8 existing fine cells */
    unsigned char* mark = ucalloc(nc);
    for (int q = 0; q < nc; ++q) mark[q] = CM->c2f[q] && !cg->wallMarker[q];
    int* jMinusF = imalloc(nf);
    int* kMinusF = imalloc(nf);
    for (int q = 0; q < nf; ++q) { jMinusF[fg->jPlus[q]] = q; kMinusF[fg->kPlus[q]] = q; }
    int* jMinusC = imalloc(nc);
    int* kMinusC = imalloc(nc);
    for (int q = 0; q < nc; ++q) { jMinusC[cg->jPlus[q]] = q; kMinusC[cg->kPlus[q]] = q; }
    int* sees = imalloc(nc);
    I->c2fCount = 0;
    for (int q = 0; q < nc; ++q) {
        sees[q] = -1;
        if (!mark[q]) continue;
        /* NBR of the coarse cell (finishNBRPlus, NBRFunctions.h:5-11) */
        const int iP = q + 1 < nc ? q + 1 : 0, jP = cg->jPlus[q], kP = cg->kPlus[q], jkP = cg->jPlus[kP];
        const int ijP = jP + 1 < nc ? jP + 1 : 0, ikP = kP + 1 < nc ? kP + 1 : 0, ijkP = jkP + 1 < nc ? jkP + 1 : 0;
        const int nb[7] = {iP, jP, ijP, kP, ikP, jkP, ijkP};
        const int di[7] = {1, 0, 1, 0, 1, 0, 1}, dj[7] = {0, 1, 1, 0, 0, 1, 1}, dk[7] = {0, 0, 0, 1, 1, 1, 1};
        int ok = 1;
        for (int t = 0; t < 7; ++t) if (!mark[nb[t]]) ok = 0;
        for (int t = 0; t < 7 && ok; ++t)
            if (cg->I[nb[t]] != cg->I[q] + di[t] || cg->J[nb[t]] != cg->J[q] + dj[t] || cg->K[nb[t]] != cg->K[q] + dk[t])
                ok = 0;
        if (!ok) continue;
        const int top = child[ijkP];
        if (top < 0) continue;
        int fjk = top - 1;
        if (fjk < 0) fjk = nf - 1;
        const int fk = jMinusF[fjk];
        const int fs = kMinusF[fk];
        const int fj = fg->jPlus[fs];
        const int fiP = fs + 1 < nf ? fs + 1 : 0, fijP = fj + 1 < nf ? fj + 1 : 0, fikP = fk + 1 < nf ? fk + 1 : 0;
        const int fijkP = fjk + 1 < nf ? fjk + 1 : 0;
        const int fb[8] = {fs, fiP, fj, fijP, fk, fikP, fjk, fijkP};
        const int ei[8] = {1, 2, 1, 2, 1, 2, 1, 2}, ej[8] = {1, 1, 2, 2, 1, 1, 2, 2}, ek[8] = {1, 1, 1, 1, 2, 2, 2, 2};
        for (int t = 0; t < 8 && ok; ++t)
            if (fg->I[fb[t]] != 2 * cg->I[q] + ei[t] || fg->J[fb[t]] != 2 * cg->J[q] + ej[t] ||
                fg->K[fb[t]] != 2 * cg->K[q] + ek[t])
                ok = 0;
        if (!ok) continue;
        sees[q] = fs;
        I->c2fCount++;
    }
    I->c2fIndex = imalloc(I->c2fCount);
    I->c2fChild = imalloc(I->c2fCount);
    unsigned char* received = ucalloc(nf);
    for (int q = 0, t = 0; q < nc; ++q) {
        if (sees[q] < 0) continue;
        I->c2fIndex[t] = q;
        I->c2fChild[t] = sees[q];
        ++t;
        const int fs = sees[q], fj = fg->jPlus[fs], fk = fg->kPlus[fs], fjk = fg->jPlus[fk];
        const int cells[8] = {fs, fs + 1 < nf ? fs + 1 : 0, fj, fj + 1 < nf ? fj + 1 : 0,
                              fk, fk + 1 < nf ? fk + 1 : 0, fjk, fjk + 1 < nf ? fjk + 1 : 0};
        for (int u = 0; u < 8; ++u) received[cells[u]] = 1;
    }
    /* leftovers (:919-1029): fine cells that need coarse values and got none */
    I->leftCount = 0;
    for (int q = 0; q < nf; ++q) I->leftCount += FM->needValues[q] && !fg->wallMarker[q] && !received[q];
    const int m = I->leftCount;
    I->leftIndex = imalloc(m);
    I->leftParent = imalloc(m);
    I->leftNbr = imalloc(3 * m);
    for (int q = 0, t = 0; q < nf; ++q) {
        if (!(FM->needValues[q] && !fg->wallMarker[q] && !received[q])) continue;
        const int pc = FM->parent[q];
        const int ic = cg->I[pc], jc = cg->J[pc], kc = cg->K[pc];
        /* per axis: the neighbour on the fine cell's side if it is marked and
         * in place, else the opposite one coded as -cell-1, else the parent */
        const int plus[3] = {pc + 1 >= nc ? 0 : pc + 1, cg->jPlus[pc], cg->kPlus[pc]};
        const int minus[3] = {pc - 1 < 0 ? nc - 1 : pc - 1, jMinusC[pc], kMinusC[pc]};
        const int odd[3] = {fg->I[q] % 2 == 1, fg->J[q] % 2 == 1, fg->K[q] % 2 == 1};
        for (int a = 0; a < 3; ++a) {
            const int e[3] = {a == 0, a == 1, a == 2};
            int pick = pc;
            const int first = odd[a] ? plus[a] : minus[a], second = odd[a] ? minus[a] : plus[a];
            const int sf = odd[a] ? 1 : -1;
            if (mark[first] && cg->I[first] == ic + sf * e[0] && cg->J[first] == jc + sf * e[1] &&
                cg->K[first] == kc + sf * e[2])
                pick = first;
            else if (mark[second] && cg->I[second] == ic - sf * e[0] && cg->J[second] == jc - sf * e[1] &&
                     cg->K[second] == kc - sf * e[2])
                pick = -second - 1;
            I->leftNbr[(size_t)a * m + t] = pick;
        }
        I->leftIndex[t] = q;
        I->leftParent[t] = pc;
        ++t;
    }
    free(child); free(mark); free(jMinusF); free(kMinusF); free(jMinusC); free(kMinusC); free(sees); free(received);
}

int oracle_domain_build(const lbm_case* c, odomain* d) {
    memset(d, 0, sizeof(*d));
    const int NL = c->grid_level_count;
    if (NL < 1 || NL > LBM_MAX_LEVELS) return LBM_ERR_INVALID;
    if (NL == 1) {
        d->levelCount = 1;
        return oracle_build(c, &d->level[0]);
    }
    if (c->body_count < 0 || c->body_count > LBM_MAX_BODIES || c->rotor_count < 0 || c->rotor_count > 4)
        return LBM_ERR_INVALID;
    d->levelCount = NL;
    init_info(c, &d->level[0]);
    for (int l = 1; l < NL; ++l) finer_info(c, &d->level[l - 1], &d->level[l], l);
    /* bodies on every level (initializeVoxelizers, voxelizerFunctions.h:692-728) */
    const int nb = c->body_count;
    ostl* bodies = (ostl*)calloc((size_t)(nb > 0 ? nb : 1), sizeof(ostl));
    oraymap* maps = (oraymap*)calloc((size_t)NL * (nb > 0 ? nb : 1), sizeof(oraymap));
    oraymap total[LBM_MAX_LEVELS];
    for (int b = 0; b < nb; ++b) {
        if (!c->body[b].triangles || ostl_load(&bodies[b], c->body[b].triangles, c->body[b].triangle_count) == 0) {
            for (int q = 0; q <= b; ++q) ostl_free(&bodies[q]);
            free(bodies); free(maps);
            return LBM_ERR_BUILD;
        }
        ostl_bins(&bodies[b], c->res_global);
    }
    for (int l = 0; l < NL; ++l) {
        const ogrid* g = &d->level[l];
        for (int b = 0; b < nb; ++b) oray_voxelize(&maps[l * nb + b], &bodies[b], g->ox, g->oy, g->oz, g->res, g->nx, g->ny);
        if (nb > 0) {
            oray_copy(&total[l], &maps[l * nb]);
            for (int b = 1; b < nb; ++b) oray_union(&total[l], &maps[l * nb + b]);
        } else {
            oray_empty(&total[l], g->nx, g->ny);
        }
    }
    /* buildIJKFull (:299-400): level 0 from the skeleton (a skeleton cell is
     * kept when it covers fluid on any level, plus one layer) */
    {
        ogrid* g = &d->level[0];
        const int snx = g->nx / 2, sny = g->ny / 2, snz = g->nz / 2;
        const size_t sc = (size_t)snx * sny * snz;
        unsigned char* keepS = (unsigned char*)calloc(sc, 1);
        unsigned char* keepT = (unsigned char*)calloc(sc, 1);
        for (size_t sIdx = 0; sIdx < sc; ++sIdx) {
            const int ks = (int)(sIdx / ((size_t)snx * sny)), rem = (int)(sIdx % ((size_t)snx * sny));
            for (int m = 0; m < NL && !keepS[sIdx]; ++m)
                keepS[sIdx] = (unsigned char)oray_block_has_fluid(&total[m], rem % snx, rem / snx, ks, 2 << m);
        }
        spread_dense(keepS, keepT, snx, sny, snz);
        int kept = 0;
        for (size_t q = 0; q < sc; ++q) kept += keepT[q];
        const int n0 = 8 * kept;
        int* ijk = imalloc(3 * n0);
        int cf = 0;
        for (size_t sIdx = 0; sIdx < sc; ++sIdx) {
            if (!keepT[sIdx]) continue;
            const int ks = (int)(sIdx / ((size_t)snx * sny)), rem = (int)(sIdx % ((size_t)snx * sny));
            for (int ka = 0; ka < 2; ++ka)
                for (int ja = 0; ja < 2; ++ja)
                    for (int ia = 0; ia < 2; ++ia) {
                        ijk[3 * cf] = 2 * (rem % snx) + ia;
                        ijk[3 * cf + 1] = 2 * (rem / snx) + ja;
                        ijk[3 * cf + 2] = 2 * ks + ka;
                        ++cf;
                    }
        }
        free(keepS); free(keepT);
        qsort(ijk, (size_t)n0, 3 * sizeof(int), cmp_kji);
        g->cellCount = n0;
        g->I = imalloc(n0); g->J = imalloc(n0); g->K = imalloc(n0);
        for (int q = 0; q < n0; ++q) { g->I[q] = ijk[3 * q]; g->J[q] = ijk[3 * q + 1]; g->K[q] = ijk[3 * q + 2]; }
        free(ijk);
        nbr_plus(g);
    }
    omarks marks[LBM_MAX_LEVELS];
    memset(marks, 0, sizeof(marks));
    for (int l = 0; l + 1 < NL; ++l) {
        mark_refinement(c, &d->level[l], &marks[l], total, NL);
        build_finer(&d->level[l], &marks[l], &d->level[l + 1], &marks[l + 1]);
    }
    for (int l = 0; l < NL; ++l)
        delete_excess(&d->level[l], &marks[l], l > 0 ? &d->level[l - 1] : NULL, &total[l], l == NL - 1);
    /* buildWallMarkers (:590-739) with the interface overlap (step 7) */
    int rc = 0;
    for (int l = 0; l < NL && rc == 0; ++l) {
        ogrid* g = &d->level[l];
        omarks* M = &marks[l];
        const int n = g->cellCount;
        unsigned char* overlap = ucalloc(n);
        unsigned char* iface = ucalloc(n);
        for (int q = 0; q < n; ++q) {
            if (l + 1 < NL) {
                overlap[q] = M->f2c[q];
                iface[q] = M->f2c[q] || M->c2f[q];
            }
            if (l > 0 && M->parent[q] >= 0) {
                iface[q] = 1;
                if (marks[l - 1].c2f[M->parent[q]]) overlap[q] = 1;
            }
        }
        g->wallMarker = ucalloc(n);
        M->wallIDFull = imalloc(n);
        oparent up = {l > 0 ? &d->level[l - 1] : NULL, M->parent, l > 0 ? marks[l - 1].wallIDFull : NULL,
                      l > 0 ? &maps[(l - 1) * nb] : NULL};
        build_walls(c, g, bodies, &maps[l * nb], &total[l], l > 0 ? &up : NULL, iface, overlap, M->wallIDFull);
        rc = finish_level(c, g, overlap);
        free(overlap);
        free(iface);
    }
    for (int l = 0; rc == 0 && l + 1 < NL; ++l)
        build_interface(&d->level[l], &marks[l], &d->level[l + 1], &marks[l + 1], &d->itf[l]);
    for (int l = 0; l < NL; ++l) omarks_free(&marks[l]);
    for (int b = 0; b < nb; ++b) ostl_free(&bodies[b]);
    for (int q = 0; q < NL * nb; ++q) oray_free(&maps[q]);
    for (int l = 0; l < NL; ++l) oray_free(&total[l]);
    free(bodies);
    free(maps);
    if (rc != 0) oracle_domain_free(d);
    return rc;
}

void oracle_domain_free(odomain* d) {
    for (int l = 0; l < d->levelCount; ++l) {
        oracle_free(&d->level[l]);
        ointerface* I = &d->itf[l];
        free(I->f2cIndex); free(I->f2cChild); free(I->c2fIndex); free(I->c2fChild);
        free(I->leftIndex); free(I->leftParent); free(I->leftNbr);
    }
    memset(d, 0, sizeof(*d));
}

/* pre-collision populations of a cell in the current esotwist state */
static void read_pre(const ogrid* g, int cell, float f[27]) {
    int nb[8];
    get_nbr(g, cell, nb);
    const size_t n = (size_t)g->cellCount;
    for (int dd = 0; dd < 27; ++dd) f[dd] = g->f[(size_t)(g->flip ? INV[dd] : dd) * n + nb[pre_nbr(dd)]];
}

static void write_pre(ogrid* g, int cell, const float f[27]) {
    int nb[8];
    get_nbr(g, cell, nb);
    const size_t n = (size_t)g->cellCount;
    for (int dd = 0; dd < 27; ++dd) g->f[(size_t)(g->flip ? INV[dd] : dd) * n + nb[pre_nbr(dd)]] = f[dd];
}

/* Density deviation, velocity and the five velocity-gradient estimates of a
 * cell from its populations (the stencil loops of updateInterface.h:204-239):
 * out = {dRho, ux, uy, uz, kxy, kyz, kxz, kxx-kyy, kxx-kzz}; sums of the
 * second moments run over the directions in index order. */
static void interface_moments(const float f[27], float omega, float out[9]) {
    float m[4];
    oracle_get_drho_u(f, m);
    const float rho = 1.f + m[0];
    float pxy = 0.f, pyz = 0.f, pxz = 0.f, pmy = 0.f, pmz = 0.f;
    for (int dd = 1; dd < 27; ++dd) {
        const int xy = CX[dd] * CY[dd], yz = CY[dd] * CZ[dd], xz = CX[dd] * CZ[dd];
        const int my = CX[dd] * CX[dd] - CY[dd] * CY[dd], mz = CX[dd] * CX[dd] - CZ[dd] * CZ[dd];
        if (xy > 0) pxy = pxy + f[dd]; else if (xy < 0) pxy = pxy - f[dd];
        if (yz > 0) pyz = pyz + f[dd]; else if (yz < 0) pyz = pyz - f[dd];
        if (xz > 0) pxz = pxz + f[dd]; else if (xz < 0) pxz = pxz - f[dd];
        if (my > 0) pmy = pmy + f[dd]; else if (my < 0) pmy = pmy - f[dd];
        if (mz > 0) pmz = pmz + f[dd]; else if (mz < 0) pmz = pmz - f[dd];
    }
    out[0] = m[0]; out[1] = m[1]; out[2] = m[2]; out[3] = m[3];
    out[4] = -3.f * omega * (pxy / rho - m[1] * m[2]);
    out[5] = -3.f * omega * (pyz / rho - m[2] * m[3]);
    out[6] = -3.f * omega * (pxz / rho - m[1] * m[3]);
    out[7] = -1.5f * omega * (pmy / rho - (m[1] * m[1] - m[2] * m[2]));
    out[8] = -1.5f * omega * (pmz / rho - (m[1] * m[1] - m[3] * m[3]));
}

/* reconstructInterpolatedF (updateInterface.h:29-153): populations from
 * dRho, u and the second-order central moments, every other central moment
 * at its rest value; the back transform x, y, z of applyCollision
 * (applyCollision.h:390-490). */
static void reconstruct_f(float f[27], float dRho, float ux, float uy, float uz, float k011, float k101, float k110,
                          float k200, float k020, float k002) {
    float s[3][3][3];
    memset(s, 0, sizeof(s));
    s[0][0][0] = dRho;
    s[2][0][0] = k200; s[0][2][0] = k020; s[0][0][2] = k002;
    s[1][1][0] = k110; s[1][0][1] = k101; s[0][1][1] = k011;
    s[2][2][0] = dRho / 9.f; s[0][2][2] = dRho / 9.f; s[2][0][2] = dRho / 9.f;
    s[2][2][2] = dRho / 27.f;
    back_transform(s, ux, uy, uz, f);
}

/* Quadratic fit over a 2x2x2 stencil (Schoenherr 2015, the coefficient set
 * of updateInterface.h:262-306 and :443-545): corners q = self, +i, +j, +ij,
 * +k, +ik, +jk, +ijk at (+-1/2)^3; v[q] = interface_moments of corner q.
 * Each coefficient is the signed corner sum of updateInterface.h, formed
 * corner by corner. */
typedef struct ofit {
    float d[8];                /* 1, x, y, z, xy, xz, yz, xyz */
    float u[3][11];            /* 1, x, y, z, xy, xz, yz, xyz, xx, yy, zz */
} ofit;

static float corner_sum(const float v[8][9], int field, int px, int py, int pz) {
    float s = 0.f;
    for (int q = 0; q < 8; ++q) {
        const int sx = (q & 1) ? 1 : -1, sy = (q & 2) ? 1 : -1, sz = (q & 4) ? 1 : -1;
        const int sign = (px ? sx : 1) * (py ? sy : 1) * (pz ? sz : 1);
        s = sign > 0 ? s + v[q][field] : s - v[q][field];
    }
    return s;
}

static void fit_stencil(const float v[8][9], ofit* F) {
    enum { D = 0, UX = 1, KXY = 4, KYZ = 5, KXZ = 6, KMY = 7, KMZ = 8 };
    F->d[0] = 0.125f * corner_sum(v, D, 0, 0, 0);
    F->d[1] = 0.25f * corner_sum(v, D, 1, 0, 0);
    F->d[2] = 0.25f * corner_sum(v, D, 0, 1, 0);
    F->d[3] = 0.25f * corner_sum(v, D, 0, 0, 1);
    F->d[4] = 0.5f * corner_sum(v, D, 1, 1, 0);
    F->d[5] = 0.5f * corner_sum(v, D, 1, 0, 1);
    F->d[6] = 0.5f * corner_sum(v, D, 0, 1, 1);
    F->d[7] = corner_sum(v, D, 1, 1, 1);
    for (int a = 0; a < 3; ++a) {
        F->u[a][1] = 0.25f * corner_sum(v, UX + a, 1, 0, 0);
        F->u[a][2] = 0.25f * corner_sum(v, UX + a, 0, 1, 0);
        F->u[a][3] = 0.25f * corner_sum(v, UX + a, 0, 0, 1);
        F->u[a][4] = 0.5f * corner_sum(v, UX + a, 1, 1, 0);
        F->u[a][5] = 0.5f * corner_sum(v, UX + a, 1, 0, 1);
        F->u[a][6] = 0.5f * corner_sum(v, UX + a, 0, 1, 1);
        F->u[a][7] = corner_sum(v, UX + a, 1, 1, 1);
    }
    const float sux = corner_sum(v, UX, 0, 0, 0), suy = corner_sum(v, UX + 1, 0, 0, 0), suz = corner_sum(v, UX + 2, 0, 0, 0);
    const float uxXY = corner_sum(v, UX, 1, 1, 0), uxXZ = corner_sum(v, UX, 1, 0, 1);
    const float uyXY = corner_sum(v, UX + 1, 1, 1, 0), uyYZ = corner_sum(v, UX + 1, 0, 1, 1);
    const float uzXZ = corner_sum(v, UX + 2, 1, 0, 1), uzYZ = corner_sum(v, UX + 2, 0, 1, 1);
    const float kxyX = corner_sum(v, KXY, 1, 0, 0), kxyY = corner_sum(v, KXY, 0, 1, 0);
    const float kxzX = corner_sum(v, KXZ, 1, 0, 0), kxzZ = corner_sum(v, KXZ, 0, 0, 1);
    const float kyzY = corner_sum(v, KYZ, 0, 1, 0), kyzZ = corner_sum(v, KYZ, 0, 0, 1);
    const float myX = corner_sum(v, KMY, 1, 0, 0), myY = corner_sum(v, KMY, 0, 1, 0), myZ = corner_sum(v, KMY, 0, 0, 1);
    const float mzX = corner_sum(v, KMZ, 1, 0, 0), mzY = corner_sum(v, KMZ, 0, 1, 0), mzZ = corner_sum(v, KMZ, 0, 0, 1);
    /* a000, b000, c000 */
    F->u[0][0] = 0.015625f * (2.f * (uyXY + uzXZ - kxyY - kxzZ) + 8.f * sux - myX - mzX);
    F->u[1][0] = 0.015625f * (2.f * (uxXY + uzYZ + myY - kxyX - kyzZ) + 8.f * suy - mzY);
    F->u[2][0] = 0.015625f * (2.f * (uxXZ + uyYZ + mzZ - kxzX - kyzY) + 8.f * suz - myZ);
    /* a200 .. c002 */
    F->u[0][8] = 0.0625f * (2.f * (uyXY + uzXZ) + myX + mzX);
    F->u[1][8] = 0.125f * (kxyX - 2.f * uxXY);
    F->u[2][8] = 0.125f * (kxzX - 2.f * uxXZ);
    F->u[0][9] = 0.125f * (kxyY - 2.f * uyXY);
    F->u[1][9] = 0.0625f * (2.f * (uxXY + uzYZ - myY) + mzY);
    F->u[2][9] = 0.125f * (kyzY - 2.f * uyYZ);
    F->u[0][10] = 0.125f * (kxzZ - 2.f * uzXZ);
    F->u[1][10] = 0.125f * (kyzZ - 2.f * uzYZ);
    F->u[2][10] = 0.0625f * (2.f * (uxXZ + uyYZ - mzZ) + myZ);
}

/* velocity gradient of the fit at (x, y, z): G[a][b] = d u_a / d x_b */
static void fit_gradient(const ofit* F, float x, float y, float z, float G[3][3]) {
    for (int a = 0; a < 3; ++a) {
        const float* c = F->u[a];
        G[a][0] = c[1] + c[4] * y + c[5] * z + c[7] * y * z + 2.f * c[8] * x;
        G[a][1] = c[2] + c[4] * x + c[6] * z + c[7] * x * z + 2.f * c[9] * y;
        G[a][2] = c[3] + c[5] * x + c[6] * y + c[7] * x * y + 2.f * c[10] * z;
    }
}

/* second-order central moments from the strain rate, rescaled by
 * sigma / omega of the target level (updateInterface.h:334-346, :645-660) */
static void populations_from_gradient(float f[27], float dRho, const float u[3], const float G[3][3], float sigma,
                                      float omega) {
    const float rho = 1.f + dRho;
    const float k011 = -(1.f / 3.f) * (G[1][2] + G[2][1]) * sigma / omega * rho;
    const float k101 = -(1.f / 3.f) * (G[0][2] + G[2][0]) * sigma / omega * rho;
    const float k110 = -(1.f / 3.f) * (G[0][1] + G[1][0]) * sigma / omega * rho;
    const float mxxMyy = -(2.f / 3.f) * (G[0][0] - G[1][1]) * sigma / omega * rho;
    const float mxxMzz = -(2.f / 3.f) * (G[0][0] - G[2][2]) * sigma / omega * rho;
    const float k200 = (1.f / 3.f) * (mxxMyy + mxxMzz + dRho);
    const float k020 = (1.f / 3.f) * (-2.f * mxxMyy + mxxMzz + dRho);
    const float k002 = (1.f / 3.f) * (mxxMyy - 2.f * mxxMzz + dRho);
    reconstruct_f(f, dRho, u[0], u[1], u[2], k011, k101, k110, k200, k020, k002);
}

/* updateInterface (updateInterface.h:155-891) between level c and level c+1 */
static void interface_update(ogrid* cg, ogrid* fg, const ointerface* I) {
    const float omegaC = 1.f / (3.f * cg->nu + 0.5f), omegaF = 1.f / (3.f * fg->nu + 0.5f);
    /* fine to coarse (:155-359) */
#pragma omp parallel for schedule(static)
    for (int t = 0; t < I->f2cCount; ++t) {
        int nb[8];
        get_nbr(fg, I->f2cChild[t], nb);
        float v[8][9], f[27];
        for (int q = 0; q < 8; ++q) { read_pre(fg, nb[q], f); interface_moments(f, omegaF, v[q]); }
        ofit F;
        fit_stencil(v, &F);
        float G[3][3], u[3] = {F.u[0][0], F.u[1][0], F.u[2][0]};
        fit_gradient(&F, 0.f, 0.f, 0.f, G);
        populations_from_gradient(f, F.d[0], u, G, 2.f, omegaC);
        write_pre(cg, I->f2cIndex[t], f);
    }
    /* coarse to fine blocks (:362-676) */
#pragma omp parallel for schedule(static)
    for (int t = 0; t < I->c2fCount; ++t) {
        int nb[8], fb[8];
        get_nbr(cg, I->c2fIndex[t], nb);
        float v[8][9], f[27];
        for (int q = 0; q < 8; ++q) { read_pre(cg, nb[q], f); interface_moments(f, omegaC, v[q]); }
        ofit F;
        fit_stencil(v, &F);
        get_nbr(fg, I->c2fChild[t], fb);
        for (int q = 0; q < 8; ++q) {
            const float x = (q & 1) ? 0.25f : -0.25f, y = (q & 2) ? 0.25f : -0.25f, z = (q & 4) ? 0.25f : -0.25f;
            const float dRho = F.d[0] + F.d[1] * x + F.d[2] * y + F.d[3] * z + F.d[4] * x * y + F.d[5] * x * z +
                               F.d[6] * y * z + F.d[7] * x * y * z;
            float u[3], G[3][3];
            for (int a = 0; a < 3; ++a) {
                const float* c = F.u[a];
                u[a] = c[0] + c[1] * x + c[2] * y + c[3] * z + c[4] * x * y + c[5] * x * z + c[6] * y * z +
                       c[7] * x * y * z + c[8] * x * x + c[9] * y * y + c[10] * z * z;
            }
            fit_gradient(&F, x, y, z, G);
            populations_from_gradient(f, dRho, u, G, 0.5f, omegaF);
            write_pre(fg, fb[q], f);
        }
    }
    /* leftovers (:678-884) */
#pragma omp parallel for schedule(static)
    for (int t = 0; t < I->leftCount; ++t) {
        const int pc = I->leftParent[t];
        float f[27], cen[9], r[9], uw[3];
        read_pre(cg, pc, f);
        interface_moments(f, omegaC, cen);
        const int wm = cg->wallMap[pc];
        const unsigned wallData = wm >= 0 ? cg->wallData[wm] : 0u;
        for (int a = 0; a < 3; ++a) uw[a] = wm >= 0 ? cg->wallVel[(size_t)a * cg->wallCount + wm] : cen[1 + a];
        for (int q = 0; q < 9; ++q) r[q] = cen[q];
        const int dirs[3] = {1, 6, 4}; /* POO, OPO, OOP */
        for (int a = 0; a < 3; ++a) {
            int cell = I->leftNbr[(size_t)a * I->leftCount + t];
            const int opposite = cell < 0;
            if (opposite) cell = -cell - 1;
            float v[9];
            read_pre(cg, cell, f);
            interface_moments(f, omegaC, v);
            if (!opposite) {
                for (int q = 0; q < 9; ++q) r[q] += 0.25f * (v[q] - cen[q]);
                continue;
            }
            r[0] -= 0.25f * (v[0] - cen[0]);
            for (int q = 4; q < 9; ++q) r[q] -= 0.25f * (v[q] - cen[q]);
            const int wall = (wallData & (1u << dirs[a])) || (wallData & (1u << INV[dirs[a]]));
            for (int q = 1; q < 4; ++q) {
                if (!wall) r[q] -= 0.25f * (v[q] - cen[q]);
                else r[q] += (1.f / 24.f) * (10.f * uw[q - 1] - 9.f * cen[q] - v[q]);
            }
        }
        const float G[3][3] = {{0.f, r[4], r[6]}, {0.f, -r[7], r[5]}, {0.f, 0.f, -r[8]}};
        const float u[3] = {r[1], r[2], r[3]};
        populations_from_gradient(f, r[0], u, G, 0.5f, omegaF);
        write_pre(fg, I->leftIndex[t], f);
    }
}

static void domain_update(odomain* d, int level) {
    oracle_step(&d->level[level], 1);
    if (level + 1 < d->levelCount && level + 1 < LBM_MAX_LEVELS) {
        for (int i = 0; i < 2; ++i) domain_update(d, level + 1);
        interface_update(&d->level[level], &d->level[level + 1], &d->itf[level]);
    }
}

void oracle_domain_step(odomain* d, int coarseSteps) {
    for (int s = 0; s < coarseSteps; ++s) domain_update(d, 0);
}

double oracle_domain_kinetic_energy(const odomain* d, float uRefPhys, float domainLength) {
    double e = 0.0;
    for (int l = 0; l < d->levelCount; ++l) e += oracle_kinetic_energy(&d->level[l], uRefPhys, domainLength);
    return e;
}

void oracle_fit_check(const float* corners, float x, float y, float z, float* out) {
    /* test hook: the fit of 8 corner records {dRho, ux, uy, uz, kxy, kyz, kxz,
     * kxx-kyy, kxx-kzz} evaluated at (x, y, z): out = {dRho, ux, uy, uz, G} */
    float v[8][9];
    for (int q = 0; q < 8; ++q)
        for (int t = 0; t < 9; ++t) v[q][t] = corners[q * 9 + t];
    ofit F;
    fit_stencil(v, &F);
    out[0] = F.d[0] + F.d[1] * x + F.d[2] * y + F.d[3] * z + F.d[4] * x * y + F.d[5] * x * z + F.d[6] * y * z +
             F.d[7] * x * y * z;
    for (int a = 0; a < 3; ++a) {
        const float* c = F.u[a];
        out[1 + a] = c[0] + c[1] * x + c[2] * y + c[3] * z + c[4] * x * y + c[5] * x * z + c[6] * y * z +
                     c[7] * x * y * z + c[8] * x * x + c[9] * y * y + c[10] * z * z;
    }
    float G[3][3];
    fit_gradient(&F, x, y, z, G);
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) out[4 + 3 * a + b] = G[a][b];
}
