/*
 * oracle_geometry.c — TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference's geometry setup: triangle soup and
 * spatial bins (include/STLFunctions.h), z-ray voxelization and interval
 * unions (include/voxelizerFunctions.h), the ray-map queries of the marker
 * functions (include/markerFunctions.h) and the ray/triangle intersection
 * of the link-length builder
 * (include/boundaryConditions/interpolatedBouncebackFunctions.h).
 * Plain C, serial, no floating-point contraction: the reference's parallel
 * formulation (thread-to-triangle balancing, atomics, scans) is replaced by
 * direct loops that produce the same sorted ray maps.  Used by the oracle's
 * grid builder; the product never links it.
 */
#include "oracle_internal.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static float fmin3(float a, float b, float c) { return a < b ? (a < c ? a : c) : (b < c ? b : c); }
static float fmax3(float a, float b, float c) { return a > b ? (a > c ? a : c) : (b > c ? b : c); }
static int imin(int a, int b) { return a < b ? a : b; }
static int imax(int a, int b) { return a > b ? a : b; }

/* readSTL without the file I/O (include/STLFunctions.h:317-440): triangles
 * with two identical vertices are dropped, bounds over the kept vertices. */
int ostl_load(ostl* t, const float* tri, int n) {
    memset(t, 0, sizeof(*t));
    float** arr[9] = {&t->ax, &t->ay, &t->az, &t->bx, &t->by, &t->bz, &t->cx, &t->cy, &t->cz};
    for (int q = 0; q < 9; ++q) *arr[q] = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
    t->xMin = t->yMin = t->zMin = 3.402823466e38f;
    t->xMax = t->yMax = t->zMax = -3.402823466e38f;
    int w = 0;
    for (int q = 0; q < n; ++q) {
        const float* v = tri + 9 * (size_t)q;
        const float ax = v[0], ay = v[1], az = v[2], bx = v[3], by = v[4], bz = v[5], cx = v[6], cy = v[7], cz = v[8];
        if ((ax == bx && ay == by && az == bz) || (cx == bx && cy == by && cz == bz) ||
            (cx == ax && cy == ay && cz == az))
            continue;
        t->ax[w] = ax; t->ay[w] = ay; t->az[w] = az;
        t->bx[w] = bx; t->by[w] = by; t->bz[w] = bz;
        t->cx[w] = cx; t->cy[w] = cy; t->cz[w] = cz;
        ++w;
        const float xl = fmin3(ax, bx, cx), yl = fmin3(ay, by, cy), zl = fmin3(az, bz, cz);
        const float xh = fmax3(ax, bx, cx), yh = fmax3(ay, by, cy), zh = fmax3(az, bz, cz);
        if (xl < t->xMin) t->xMin = xl;
        if (yl < t->yMin) t->yMin = yl;
        if (zl < t->zMin) t->zMin = zl;
        if (xh > t->xMax) t->xMax = xh;
        if (yh > t->yMax) t->yMax = yh;
        if (zh > t->zMax) t->zMax = zh;
    }
    t->count = w;
    return w;
}

/* sortSTLToBins (include/STLFunctions.h:5-127): cubic bins sized for about
 * 10 triangles each; every triangle is listed in each bin its tolerance-grown
 * bounding box touches.  Within a bin, triangles are in index order (the
 * reference's atomic order only changes ties of a minimum search). */
void ostl_bins(ostl* t, float resGlobal) {
    const float totalVolume = (t->xMax - t->xMin) * (t->yMax - t->yMin) * (t->zMax - t->zMin);
    const float targetBinVolume = totalVolume / ((float)t->count / (float)10);
    t->binSize = powf(targetBinVolume, 1.f / 3.f);
    const float bs = t->binSize;
    t->oxBin = t->xMin - bs - 2.f * resGlobal;
    t->oyBin = t->yMin - bs - 2.f * resGlobal;
    t->ozBin = t->zMin - bs - 2.f * resGlobal;
    t->binCountX = (int)((t->xMax - t->xMin + 2.f * bs + 4.f * resGlobal) / bs) + 1;
    t->binCountY = (int)((t->yMax - t->yMin + 2.f * bs + 4.f * resGlobal) / bs) + 1;
    t->binCountZ = (int)((t->zMax - t->zMin + 2.f * bs + 4.f * resGlobal) / bs) + 1;
    const int bxy = t->binCountX * t->binCountY;
    const int nb = bxy * t->binCountZ;
    const float tol = bs * 0.2f + resGlobal * 3.f;
    t->firstInBin = (int*)calloc((size_t)nb + 1, sizeof(int));
    int pass;
    int* fill = (int*)calloc((size_t)nb + 1, sizeof(int));
    for (pass = 0; pass < 2; ++pass) {
        for (int q = 0; q < t->count; ++q) {
            const float ax = t->ax[q] - t->oxBin, ay = t->ay[q] - t->oyBin, az = t->az[q] - t->ozBin;
            const float bx = t->bx[q] - t->oxBin, by = t->by[q] - t->oyBin, bz = t->bz[q] - t->ozBin;
            const float cx = t->cx[q] - t->oxBin, cy = t->cy[q] - t->oyBin, cz = t->cz[q] - t->ozBin;
            const float xl = fmin3(ax, bx, cx) - tol, yl = fmin3(ay, by, cy) - tol, zl = fmin3(az, bz, cz) - tol;
            const float xh = fmax3(ax, bx, cx) + tol, yh = fmax3(ay, by, cy) + tol, zh = fmax3(az, bz, cz) + tol;
            const int i0 = imax(0, (int)(xl / bs)), j0 = imax(0, (int)(yl / bs)), k0 = imax(0, (int)(zl / bs));
            const int i1 = imin(t->binCountX, (int)(xh / bs) + 1), j1 = imin(t->binCountY, (int)(yh / bs) + 1),
                      k1 = imin(t->binCountZ, (int)(zh / bs) + 1);
            for (int kb = k0; kb < k1; ++kb)
                for (int jb = j0; jb < j1; ++jb)
                    for (int ib = i0; ib < i1; ++ib) {
                        const int bin = bxy * kb + t->binCountX * jb + ib;
                        if (pass == 0) t->firstInBin[bin]++;
                        else t->bin[t->firstInBin[bin] + fill[bin]++] = q;
                    }
        }
        if (pass == 0) {
            int run = 0;
            for (int b = 0; b <= nb; ++b) { const int v = t->firstInBin[b]; t->firstInBin[b] = run; run += v; }
            t->bin = (int*)malloc(sizeof(int) * (size_t)(run > 0 ? run : 1));
        }
    }
    free(fill);
}

void ostl_free(ostl* t) {
    free(t->ax); free(t->ay); free(t->az); free(t->bx); free(t->by); free(t->bz);
    free(t->cx); free(t->cy); free(t->cz); free(t->firstInBin); free(t->bin);
    memset(t, 0, sizeof(*t));
}

/* getRayHitYesNo (include/voxelizerFunctions.h:5-65): strict interior, or an
 * exact edge hit decided by the above/below rule for the edge. */
static int ray_hit(int i, int j, long long wab, long long wbc, long long wca, int axI, int ayI, int bxI, int byI,
                   int cxI, int cyI, long long abx, long long bcx, long long cax) {
    if (wab > 0 && wbc > 0 && wca > 0) return 1;
    if (wab < 0 || wbc < 0 || wca < 0) return 0;
    const long long ax0 = axI - i * 1000, ay0 = ayI - j * 1000;
    const long long bx0 = bxI - i * 1000, by0 = byI - j * 1000;
    const long long cx0 = cxI - i * 1000, cy0 = cyI - j * 1000;
    if (wab == 0) {
        if (abx == 0) return cx0 < 0;
        if (bx0 > 0 && cy0 * bx0 > by0 * cx0) return 1;
        if (bx0 < 0 && cy0 * bx0 < by0 * cx0) return 1;
    }
    if (wbc == 0) {
        if (bcx == 0) return ax0 < 0;
        if (cx0 > 0 && ay0 * cx0 > cy0 * ax0) return 1;
        if (cx0 < 0 && ay0 * cx0 < cy0 * ax0) return 1;
    }
    if (wca == 0) {
        if (cax == 0) return bx0 < 0;
        if (ax0 > 0 && by0 * ax0 > ay0 * bx0) return 1;
        if (ax0 < 0 && by0 * ax0 < ay0 * bx0) return 1;
    }
    return 0;
}

/* Per-triangle ray setup shared by the counting and filling passes. */
typedef struct tri_rays {
    int i0, i1, j0, j1;
    int axI, ayI, bxI, byI, cxI, cyI;
    long long abx, bcx, cax;
    long long wab0, wbc0, wca0, dab_i, dab_j, dbc_i, dbc_j, dca_i, dca_j;
    float ax, ay, az, nx, ny, nz, minZ, maxZ, midZ;
} tri_rays;

/* The integer triangle and ray range of voxelizeSTL (:95-250 and :369-445). */
static int tri_setup(const ostl* t, int q, float ox, float oy, float oz, float res, int nx, int ny, tri_rays* r) {
    const float ax = t->ax[q] - ox, ay = t->ay[q] - oy, az = t->az[q] - oz;
    const float bx = t->bx[q] - ox, by = t->by[q] - oy, bz = t->bz[q] - oz;
    const float cx = t->cx[q] - ox, cy = t->cy[q] - oy, cz = t->cz[q] - oz;
    const float scale = 500.0f / res;
    r->axI = (int)roundf(ax * scale) * 2 + 1;
    r->ayI = (int)roundf(ay * scale) * 2 + 1;
    r->bxI = (int)roundf(bx * scale) * 2 + 1;
    r->byI = (int)roundf(by * scale) * 2 + 1;
    r->cxI = (int)roundf(cx * scale) * 2 + 1;
    r->cyI = (int)roundf(cy * scale) * 2 + 1;
    const int xLim = (nx - 1) * 1000, yLim = (ny - 1) * 1000;
    const int xIMin = imax(0, imin(imin(r->axI, r->bxI), imin(r->cxI, xLim)));
    const int xIMax = imin(xLim, imax(imax(r->axI, r->bxI), imax(r->cxI, 0)));
    const int yIMin = imax(0, imin(imin(r->ayI, r->byI), imin(r->cyI, yLim)));
    const int yIMax = imin(yLim, imax(imax(r->ayI, r->byI), imax(r->cyI, 0)));
    r->i0 = (xIMin + 999) / 1000;
    r->i1 = xIMax / 1000 + 1;
    r->j0 = (yIMin + 999) / 1000;
    r->j1 = yIMax / 1000 + 1;
    const long long x0 = 1000LL * r->i0, y0 = 1000LL * r->j0;
    const long long aX = r->axI - x0, aY = r->ayI - y0, bX = r->bxI - x0, bY = r->byI - y0;
    const long long cX = r->cxI - x0, cY = r->cyI - y0;
    const long long abx = bX - aX, aby = bY - aY, bcx = cX - bX, bcy = cY - bY, cax = aX - cX, cay = aY - cY;
    const long long area = abx * bcy - aby * bcx;
    if (area == 0) return 0;
    const long long s = area < 0 ? -1 : 1;
    r->abx = abx; r->bcx = bcx; r->cax = cax;
    r->wab0 = s * (abx * (-bY) - aby * (-bX));
    r->wbc0 = s * (bcx * (-cY) - bcy * (-cX));
    r->wca0 = s * (cax * (-aY) - cay * (-aX));
    r->dab_i = -s * aby * 1000; r->dab_j = s * abx * 1000;
    r->dbc_i = -s * bcy * 1000; r->dbc_j = s * bcx * 1000;
    r->dca_i = -s * cay * 1000; r->dca_j = s * cax * 1000;
    if (r->i1 - r->i0 == 0 || r->j1 - r->j0 == 0) return 0;
    const float v1x = bx - ax, v1y = by - ay, v1z = bz - az;
    const float v2x = cx - ax, v2y = cy - ay, v2z = cz - az;
    r->nx = v1y * v2z - v1z * v2y;
    r->ny = v1z * v2x - v1x * v2z;
    r->nz = v1x * v2y - v1y * v2x;
    r->ax = ax; r->ay = ay; r->az = az;
    r->maxZ = fmax3(az, bz, cz);
    r->minZ = fmin3(az, bz, cz);
    r->midZ = 0.5f * (r->maxZ + r->minZ);
    return 1;
}

/* voxelizeSTL (include/voxelizerFunctions.h:67-535): every (i, j) ray along
 * z through the cell centres of a grid with origin (ox, oy, oz) and spacing
 * res; a hit at height z is recorded as k = ceil(z / res); each ray's hits
 * are sorted, so consecutive pairs bound the solid intervals [k0, k1). */
void oray_voxelize(oraymap* m, const ostl* t, float ox, float oy, float oz, float res, int nx, int ny) {
    m->nx = nx;
    m->ny = ny;
    const size_t rays = (size_t)nx * ny;
    m->scan = (long long*)calloc(rays + 1, sizeof(long long));
    long long* fill = (long long*)calloc(rays + 1, sizeof(long long));
    m->map = NULL;
    for (int pass = 0; pass < 2; ++pass) {
        for (int q = 0; q < t->count; ++q) {
            tri_rays r;
            if (!tri_setup(t, q, ox, oy, oz, res, nx, ny, &r)) continue;
            for (int j = r.j0; j < r.j1; ++j)
                for (int i = r.i0; i < r.i1; ++i) {
                    const long long wab = r.wab0 + (long long)(j - r.j0) * r.dab_j + (long long)(i - r.i0) * r.dab_i;
                    const long long wbc = r.wbc0 + (long long)(j - r.j0) * r.dbc_j + (long long)(i - r.i0) * r.dbc_i;
                    const long long wca = r.wca0 + (long long)(j - r.j0) * r.dca_j + (long long)(i - r.i0) * r.dca_i;
                    if (!ray_hit(i, j, wab, wbc, wca, r.axI, r.ayI, r.bxI, r.byI, r.cxI, r.cyI, r.abx, r.bcx, r.cax))
                        continue;
                    const size_t ray = (size_t)j * nx + i;
                    if (pass == 0) { m->scan[ray]++; continue; }
                    const float rayX = i * res, rayY = j * res;
                    float rayZ;
                    if (r.nz != 0.0f) {
                        rayZ = r.az - (r.nx * (rayX - r.ax) + r.ny * (rayY - r.ay)) / r.nz;
                        if (rayZ > r.maxZ) rayZ = r.maxZ;
                        else if (rayZ < r.minZ) rayZ = r.minZ;
                    } else {
                        rayZ = r.midZ;
                    }
                    m->map[m->scan[ray] + fill[ray]++] = (int)ceilf(rayZ / res);
                }
        }
        if (pass == 0) {
            long long run = 0;
            for (size_t ray = 0; ray <= rays; ++ray) { const long long v = m->scan[ray]; m->scan[ray] = run; run += v; }
            m->map = (int*)malloc(sizeof(int) * (size_t)(run > 0 ? run : 1));
        }
    }
    free(fill);
    /* insertion sort of every ray's hits (:517-534) */
    for (size_t ray = 0; ray < rays; ++ray) {
        const long long s0 = m->scan[ray], cnt = m->scan[ray + 1] - s0;
        for (long long l = 1; l < cnt; ++l) {
            const int key = m->map[s0 + l];
            long long s = l - 1;
            while (s >= 0 && m->map[s0 + s] > key) { m->map[s0 + s + 1] = m->map[s0 + s]; --s; }
            m->map[s0 + s + 1] = key;
        }
    }
}

/* sumRayMaps (include/voxelizerFunctions.h:537-690): per ray, the union of
 * both maps' solid intervals, touching intervals merged. */
void oray_union(oraymap* sum, const oraymap* bonus) {
    const size_t rays = (size_t)sum->nx * sum->ny;
    long long* scan = (long long*)calloc(rays + 1, sizeof(long long));
    int* out = NULL;
    for (int pass = 0; pass < 2; ++pass) {
        for (size_t ray = 0; ray < rays; ++ray) {
            long long si = sum->scan[ray], se = sum->scan[ray + 1];
            long long bi = bonus->scan[ray], be = bonus->scan[ray + 1];
            long long w = pass ? scan[ray] : 0;
            int active = 0;
            long long lastStart = 0, lastEnd = 0;
            while (si < se || bi < be) {
                long long cs, ce;
                if (bi >= be || (si < se && sum->map[si] <= bonus->map[bi])) {
                    cs = sum->map[si]; ce = sum->map[si + 1]; si += 2;
                } else {
                    cs = bonus->map[bi]; ce = bonus->map[bi + 1]; bi += 2;
                }
                if (!active) { lastStart = cs; lastEnd = ce; active = 1; }
                else if (cs <= lastEnd) { if (ce > lastEnd) lastEnd = ce; }
                else {
                    if (pass) { out[w] = (int)lastStart; out[w + 1] = (int)lastEnd; }
                    w += 2;
                    lastStart = cs; lastEnd = ce;
                }
            }
            if (active) {
                if (pass) { out[w] = (int)lastStart; out[w + 1] = (int)lastEnd; }
                w += 2;
            }
            if (!pass) scan[ray] = w;
        }
        if (pass == 0) {
            long long run = 0;
            for (size_t ray = 0; ray <= rays; ++ray) { const long long v = scan[ray]; scan[ray] = run; run += v; }
            out = (int*)malloc(sizeof(int) * (size_t)(run > 0 ? run : 1));
        }
    }
    free(sum->scan);
    free(sum->map);
    sum->scan = scan;
    sum->map = out;
}

void oray_copy(oraymap* dst, const oraymap* src) {
    const size_t rays = (size_t)src->nx * src->ny;
    dst->nx = src->nx;
    dst->ny = src->ny;
    dst->scan = (long long*)malloc(sizeof(long long) * (rays + 1));
    memcpy(dst->scan, src->scan, sizeof(long long) * (rays + 1));
    const long long total = src->scan[rays];
    dst->map = (int*)malloc(sizeof(int) * (size_t)(total > 0 ? total : 1));
    if (total > 0) memcpy(dst->map, src->map, sizeof(int) * (size_t)total);
}

void oray_empty(oraymap* m, int nx, int ny) {
    m->nx = nx;
    m->ny = ny;
    m->scan = (long long*)calloc((size_t)nx * ny + 1, sizeof(long long));
    m->map = (int*)malloc(sizeof(int));
}

void oray_free(oraymap* m) {
    free(m->scan);
    free(m->map);
    memset(m, 0, sizeof(*m));
}

/* markWallCells for one cell (include/markerFunctions.h:18-53). */
int oray_solid(const oraymap* m, int i, int j, int k) {
    if (i < 0 || i >= m->nx || j < 0 || j >= m->ny) return 0;
    const size_t ray = (size_t)m->nx * j + i;
    for (long long s = m->scan[ray]; s < m->scan[ray + 1]; s += 2) {
        if (m->map[s] > k) break;
        if (m->map[s + 1] > k) return 1;
    }
    return 0;
}

/* markSingleFinerFluid for one coarse cell (include/markerFunctions.h:55-113):
 * 1 unless every fine cell of the down^3 block is inside a solid interval. */
int oray_block_has_fluid(const oraymap* m, int ic, int jc, int kc, int down) {
    const int kFirst = kc * down, kLast = kFirst + down - 1;
    for (int ja = 0; ja < down; ++ja)
        for (int ia = 0; ia < down; ++ia) {
            const size_t ray = (size_t)m->nx * (jc * down + ja) + (ic * down + ia);
            const long long s0 = m->scan[ray], s1 = m->scan[ray + 1];
            if (s0 == s1) return 1;
            int covered = 0;
            for (long long s = s0; s < s1; s += 2) {
                const int kEnd = m->map[s + 1];
                if (kEnd < kFirst) {
                    if (s + 2 < s1) continue;
                    return 1;
                } else if (kEnd <= kLast) {
                    return 1;
                }
                if (m->map[s] <= kFirst) { covered = 1; break; }
                return 1;
            }
            if (!covered) return 1;
        }
    return 0;
}

/* markSingleFinerWall for one coarse cell (include/markerFunctions.h:174-220):
 * 1 when some fine cell of the down^3 block is inside a solid interval. */
int oray_block_has_wall(const oraymap* m, int ic, int jc, int kc, int down) {
    const int kFirst = kc * down, kLast = kFirst + down - 1;
    for (int ja = 0; ja < down; ++ja)
        for (int ia = 0; ia < down; ++ia) {
            const size_t ray = (size_t)m->nx * (jc * down + ja) + (ic * down + ia);
            for (long long s = m->scan[ray]; s < m->scan[ray + 1]; s += 2) {
                const int kStart = m->map[s];
                if (kStart > kLast) break;
                if (kStart >= kFirst) return 1;
                if (m->map[s + 1] <= kFirst) continue;
                return 1;
            }
        }
    return 0;
}

/* intersectRayTriangle (interpolatedBouncebackFunctions.h:400-469): the ray
 * from the origin along e against triangle abc with an edge tolerance;
 * returns 1 and the ray parameter t on a hit (t may be <= 0 or > 1). */
int oray_triangle(float ax, float ay, float az, float bx, float by, float bz, float cx, float cy, float cz, float ex,
                  float ey, float ez, float edgeTol, float* tOut) {
    const float e1x = bx - ax, e1y = by - ay, e1z = bz - az;
    const float e2x = cx - ax, e2y = cy - ay, e2z = cz - az;
    const float nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
    const float area2 = sqrtf(nx * nx + ny * ny + nz * nz);
    if (area2 == 0.f) return 0;
    const float px = ey * e2z - ez * e2y, py = ez * e2x - ex * e2z, pz = ex * e2y - ey * e2x;
    const float det = e1x * px + e1y * py + e1z * pz;
    if (det > -1e-8f && det < 1e-8f) return 0;
    const float invDet = 1.f / det;
    const float lenAB = sqrtf(e1x * e1x + e1y * e1y + e1z * e1z);
    const float lenAC = sqrtf(e2x * e2x + e2y * e2y + e2z * e2z);
    const float bcx = cx - bx, bcy = cy - by, bcz = cz - bz;
    const float lenBC = sqrtf(bcx * bcx + bcy * bcy + bcz * bcz);
    const float uTol = edgeTol * lenAC / area2, vTol = edgeTol * lenAB / area2, wTol = edgeTol * lenBC / area2;
    const float tx = -ax, ty = -ay, tz = -az;
    const float u = (tx * px + ty * py + tz * pz) * invDet;
    if (u < -uTol) return 0;
    const float qx = ty * e1z - tz * e1y, qy = tz * e1x - tx * e1z, qz = tx * e1y - ty * e1x;
    const float v = (ex * qx + ey * qy + ez * qz) * invDet;
    if (v < -vTol || u + v > 1.f + wTol) return 0;
    *tOut = (e2x * qx + e2y * qy + e2z * qz) * invDet;
    return 1;
}
