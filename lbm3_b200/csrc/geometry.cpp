// Static geometry: triangle loading, spatial bins, integer ray-casting
// voxelizer, solid-interval queries and the link ray-triangle test.
#include "geometry.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <stdexcept>

namespace lbm {

void loadTriangles(const float* tri, int n, Triangles& t) {
    t = Triangles{};
    t.xMin = t.yMin = t.zMin = std::numeric_limits<float>::max();
    t.xMax = t.yMax = t.zMax = std::numeric_limits<float>::lowest();
    for (int q = 0; q < n; ++q) {
        const float* p = tri + 9 * static_cast<size_t>(q);
        const float ax = p[0], ay = p[1], az = p[2], bx = p[3], by = p[4], bz = p[5], cx = p[6], cy = p[7],
                    cz = p[8];
        // two identical vertices: zero area, dropped
        if ((ax == bx && ay == by && az == bz) || (cx == bx && cy == by && cz == bz) ||
            (cx == ax && cy == ay && cz == az))
            continue;
        t.ax.push_back(ax); t.ay.push_back(ay); t.az.push_back(az);
        t.bx.push_back(bx); t.by.push_back(by); t.bz.push_back(bz);
        t.cx.push_back(cx); t.cy.push_back(cy); t.cz.push_back(cz);
        t.xMin = std::min(t.xMin, std::min({ax, bx, cx}));
        t.yMin = std::min(t.yMin, std::min({ay, by, cy}));
        t.zMin = std::min(t.zMin, std::min({az, bz, cz}));
        t.xMax = std::max(t.xMax, std::max({ax, bx, cx}));
        t.yMax = std::max(t.yMax, std::max({ay, by, cy}));
        t.zMax = std::max(t.zMax, std::max({az, bz, cz}));
    }
    t.count = static_cast<int>(t.ax.size());
}

namespace {

struct BinRange {
    int i0, i1, j0, j1, k0, k1;
};

BinRange binRange(const Triangles& t, int q, float tol) {
    const float ax = t.ax[q] - t.oxBin, ay = t.ay[q] - t.oyBin, az = t.az[q] - t.ozBin;
    const float bx = t.bx[q] - t.oxBin, by = t.by[q] - t.oyBin, bz = t.bz[q] - t.ozBin;
    const float cx = t.cx[q] - t.oxBin, cy = t.cy[q] - t.oyBin, cz = t.cz[q] - t.ozBin;
    const float xMin = std::min(ax, std::min(bx, cx)) - tol, xMax = std::max(ax, std::max(bx, cx)) + tol;
    const float yMin = std::min(ay, std::min(by, cy)) - tol, yMax = std::max(ay, std::max(by, cy)) + tol;
    const float zMin = std::min(az, std::min(bz, cz)) - tol, zMax = std::max(az, std::max(bz, cz)) + tol;
    BinRange r;
    r.i0 = std::max(0, static_cast<int>(xMin / t.binSize));
    r.j0 = std::max(0, static_cast<int>(yMin / t.binSize));
    r.k0 = std::max(0, static_cast<int>(zMin / t.binSize));
    r.i1 = std::min(t.binCountX, static_cast<int>(xMax / t.binSize) + 1);
    r.j1 = std::min(t.binCountY, static_cast<int>(yMax / t.binSize) + 1);
    r.k1 = std::min(t.binCountZ, static_cast<int>(zMax / t.binSize) + 1);
    return r;
}

}  // namespace

void sortToBins(Triangles& t, float resGlobal) {
    if (t.count == 0) throw std::runtime_error("sortToBins: body has no triangles");
    const float volume = (t.xMax - t.xMin) * (t.yMax - t.yMin) * (t.zMax - t.zMin);
    const float target = volume / (static_cast<float>(t.count) / 10.f);
    t.binSize = std::pow(target, 1.f / 3.f);
    if (!(t.binSize > 0.f) || !std::isfinite(t.binSize))
        throw std::runtime_error("sortToBins: a body with zero bounding volume cannot be binned");
    t.oxBin = t.xMin - t.binSize - 2.f * resGlobal;
    t.oyBin = t.yMin - t.binSize - 2.f * resGlobal;
    t.ozBin = t.zMin - t.binSize - 2.f * resGlobal;
    t.binCountX = static_cast<int>((t.xMax - t.xMin + 2.f * t.binSize + 4.f * resGlobal) / t.binSize) + 1;
    t.binCountY = static_cast<int>((t.yMax - t.yMin + 2.f * t.binSize + 4.f * resGlobal) / t.binSize) + 1;
    t.binCountZ = static_cast<int>((t.zMax - t.zMin + 2.f * t.binSize + 4.f * resGlobal) / t.binSize) + 1;
    const long long bins = 1LL * t.binCountX * t.binCountY * t.binCountZ;
    if (bins > (1LL << 28)) throw std::runtime_error("sortToBins: too many bins");
    const float tol = t.binSize * 0.2f + resGlobal * 3.f;
    t.firstInBin.assign(static_cast<size_t>(bins) + 1, 0);
    for (int q = 0; q < t.count; ++q) {
        const BinRange r = binRange(t, q, tol);
        for (int k = r.k0; k < r.k1; ++k)
            for (int j = r.j0; j < r.j1; ++j)
                for (int i = r.i0; i < r.i1; ++i)
                    ++t.firstInBin[static_cast<size_t>((1LL * k * t.binCountY + j) * t.binCountX + i)];
    }
    long long run = 0;
    for (auto& v : t.firstInBin) {
        const long long c = v;
        v = static_cast<int>(run);
        run += c;
    }
    t.bin.assign(static_cast<size_t>(run), 0);
    std::vector<int> fill(static_cast<size_t>(bins), 0);
    for (int q = 0; q < t.count; ++q) {
        const BinRange r = binRange(t, q, tol);
        for (int k = r.k0; k < r.k1; ++k)
            for (int j = r.j0; j < r.j1; ++j)
                for (int i = r.i0; i < r.i1; ++i) {
                    const size_t b = static_cast<size_t>((1LL * k * t.binCountY + j) * t.binCountX + i);
                    t.bin[static_cast<size_t>(t.firstInBin[b]) + fill[b]++] = q;
                }
    }
}

namespace {

// getRayHitYesNo (include/voxelizerFunctions.h:5-65): strictly inside, or on
// an edge with the triangle's third vertex on the agreed side.
bool rayHit(int i, int j, long long wab, long long wbc, long long wca, int axI, int ayI, int bxI, int byI,
            int cxI, int cyI, long long abx, long long bcx, long long cax) {
    if (wab > 0 && wbc > 0 && wca > 0) return true;
    if (wab < 0 || wbc < 0 || wca < 0) return false;
    const long long rx = 1000LL * i, ry = 1000LL * j;
    const long long ax0 = axI - rx, ay0 = ayI - ry, bx0 = bxI - rx, by0 = byI - ry, cx0 = cxI - rx,
                    cy0 = cyI - ry;
    if (wab == 0) {
        if (abx == 0) return cx0 < 0;
        if (bx0 > 0 && cy0 * bx0 > by0 * cx0) return true;
        if (bx0 < 0 && cy0 * bx0 < by0 * cx0) return true;
    }
    if (wbc == 0) {
        if (bcx == 0) return ax0 < 0;
        if (cx0 > 0 && ay0 * cx0 > cy0 * ax0) return true;
        if (cx0 < 0 && ay0 * cx0 < cy0 * ax0) return true;
    }
    if (wca == 0) {
        if (cax == 0) return bx0 < 0;
        if (ax0 > 0 && by0 * ax0 > ay0 * bx0) return true;
        if (ax0 < 0 && by0 * ax0 < ay0 * bx0) return true;
    }
    return false;
}

}  // namespace

void voxelize(const Triangles& t, float ox, float oy, float oz, float res, int nx, int ny, RayMap& out) {
    if (t.count == 0) throw std::runtime_error("voxelize: the body has 0 triangles");
    out.nx = nx;
    out.ny = ny;
    const size_t rays = static_cast<size_t>(nx) * ny;
    std::vector<std::vector<int>> lists(rays);
    const float scale = 500.0f / res;
    const int xLim = (nx - 1) * 1000, yLim = (ny - 1) * 1000;
    for (int q = 0; q < t.count; ++q) {
        // coordinates relative to the level origin
        const float ax = t.ax[q] - ox, ay = t.ay[q] - oy, az = t.az[q] - oz;
        const float bx = t.bx[q] - ox, by = t.by[q] - oy, bz = t.bz[q] - oz;
        const float cx = t.cx[q] - ox, cy = t.cy[q] - oy, cz = t.cz[q] - oz;
        // odd integer coordinates, rays on even ones: no ray meets a vertex
        const int axI = static_cast<int>(std::round(ax * scale)) * 2 + 1;
        const int ayI = static_cast<int>(std::round(ay * scale)) * 2 + 1;
        const int bxI = static_cast<int>(std::round(bx * scale)) * 2 + 1;
        const int byI = static_cast<int>(std::round(by * scale)) * 2 + 1;
        const int cxI = static_cast<int>(std::round(cx * scale)) * 2 + 1;
        const int cyI = static_cast<int>(std::round(cy * scale)) * 2 + 1;
        const int xMinI = std::max(0, std::min({axI, bxI, cxI, xLim}));
        const int xMaxI = std::min(xLim, std::max({axI, bxI, cxI, 0}));
        const int yMinI = std::max(0, std::min({ayI, byI, cyI, yLim}));
        const int yMaxI = std::min(yLim, std::max({ayI, byI, cyI, 0}));
        const int i0 = (xMinI + 999) / 1000, i1 = xMaxI / 1000 + 1;
        const int j0 = (yMinI + 999) / 1000, j1 = yMaxI / 1000 + 1;
        if (i1 - i0 <= 0 || j1 - j0 <= 0) continue;
        // exact edge functions relative to the first ray (i0, j0)
        const long long xo = 1000LL * i0, yo = 1000LL * j0;
        const long long axL = axI - xo, ayL = ayI - yo, bxL = bxI - xo, byL = byI - yo, cxL = cxI - xo,
                        cyL = cyI - yo;
        const long long abx = bxL - axL, aby = byL - ayL, bcx = cxL - bxL, bcy = cyL - byL, cax = axL - cxL,
                        cay = ayL - cyL;
        const long long area = abx * bcy - aby * bcx;
        if (area == 0) continue;  // projection has no area: no hits
        const long long s = area < 0 ? -1 : 1;
        const long long wab0 = s * (abx * (-byL) - aby * (-bxL));
        const long long wbc0 = s * (bcx * (-cyL) - bcy * (-cxL));
        const long long wca0 = s * (cax * (-ayL) - cay * (-axL));
        const long long dab_i = -s * aby * 1000, dab_j = s * abx * 1000;
        const long long dbc_i = -s * bcy * 1000, dbc_j = s * bcx * 1000;
        const long long dca_i = -s * cay * 1000, dca_j = s * cax * 1000;
        // hit height on the float triangle (plane through a with normal n)
        const float v1x = bx - ax, v1y = by - ay, v1z = bz - az;
        const float v2x = cx - ax, v2y = cy - ay, v2z = cz - az;
        const float nxv = v1y * v2z - v1z * v2y;
        const float nyv = v1z * v2x - v1x * v2z;
        const float nzv = v1x * v2y - v1y * v2x;
        const float maxZ = std::max({az, bz, cz}), minZ = std::min({az, bz, cz});
        const float midZ = 0.5f * (maxZ + minZ);
        for (int j = j0; j < j1; ++j) {
            long long wab = wab0 + (j - j0) * dab_j, wbc = wbc0 + (j - j0) * dbc_j,
                      wca = wca0 + (j - j0) * dca_j;
            for (int i = i0; i < i1; ++i) {
                if (rayHit(i, j, wab, wbc, wca, axI, ayI, bxI, byI, cxI, cyI, abx, bcx, cax)) {
                    const float rayX = i * res, rayY = j * res;
                    float z;
                    if (nzv != 0.0f) {
                        z = az - (nxv * (rayX - ax) + nyv * (rayY - ay)) / nzv;
                        if (z > maxZ) z = maxZ;
                        else if (z < minZ) z = minZ;
                    } else {
                        z = midZ;
                    }
                    lists[static_cast<size_t>(j) * nx + i].push_back(static_cast<int>(std::ceil(z / res)));
                }
                wab += dab_i;
                wbc += dbc_i;
                wca += dca_i;
            }
        }
    }
    out.scan.assign(rays + 1, 0);
    for (size_t r = 0; r < rays; ++r) out.scan[r + 1] = out.scan[r] + static_cast<long long>(lists[r].size());
    out.hits.resize(static_cast<size_t>(out.scan[rays]));
    for (size_t r = 0; r < rays; ++r) {
        std::sort(lists[r].begin(), lists[r].end());
        std::copy(lists[r].begin(), lists[r].end(), out.hits.begin() + out.scan[r]);
    }
}

void unionRayMaps(RayMap& sum, const RayMap& bonus) {
    if (sum.nx != bonus.nx || sum.ny != bonus.ny)
        throw std::runtime_error("sumRayMaps failed: ray maps have different ray counts.");
    const size_t rays = static_cast<size_t>(sum.nx) * sum.ny;
    RayMap out;
    out.nx = sum.nx;
    out.ny = sum.ny;
    out.scan.assign(rays + 1, 0);
    std::vector<int> merged;
    for (size_t r = 0; r < rays; ++r) {
        long long a = sum.scan[r];
        const long long aEnd = sum.scan[r + 1];
        long long b = bonus.scan[r];
        const long long bEnd = bonus.scan[r + 1];
        bool active = false;
        long long lastStart = 0, lastEnd = 0;
        while (a < aEnd || b < bEnd) {
            long long s0, e0;
            if (b >= bEnd || (a < aEnd && sum.hits[a] <= bonus.hits[b])) {
                s0 = sum.hits[a];
                e0 = sum.hits[a + 1];
                a += 2;
            } else {
                s0 = bonus.hits[b];
                e0 = bonus.hits[b + 1];
                b += 2;
            }
            if (!active) {
                lastStart = s0;
                lastEnd = e0;
                active = true;
            } else if (s0 <= lastEnd) {
                if (e0 > lastEnd) lastEnd = e0;
            } else {
                merged.push_back(static_cast<int>(lastStart));
                merged.push_back(static_cast<int>(lastEnd));
                lastStart = s0;
                lastEnd = e0;
            }
        }
        if (active) {
            merged.push_back(static_cast<int>(lastStart));
            merged.push_back(static_cast<int>(lastEnd));
        }
        out.scan[r + 1] = static_cast<long long>(merged.size());
    }
    out.hits = std::move(merged);
    sum = std::move(out);
}

bool isSolid(const RayMap& m, int i, int j, int k) {
    const size_t r = static_cast<size_t>(m.nx) * j + i;
    for (long long s = m.scan[r]; s < m.scan[r + 1]; s += 2) {
        if (m.hits[s] > k) break;
        if (m.hits[s + 1] > k) return true;
    }
    return false;
}

bool coarseHasFluid(const RayMap& fine, int down, int i, int j, int k) {
    const int kFirst = k * down, kLast = kFirst + down - 1;
    for (int jAdd = 0; jAdd < down; ++jAdd)
        for (int iAdd = 0; iAdd < down; ++iAdd) {
            const size_t r = static_cast<size_t>(fine.nx) * (j * down + jAdd) + (i * down + iAdd);
            const long long s0 = fine.scan[r], s1 = fine.scan[r + 1];
            if (s0 == s1) return true;  // no solid on this fine ray
            for (long long s = s0; s < s1; s += 2) {
                const int kEnd = fine.hits[s + 1];
                if (kEnd < kFirst) {
                    if (s + 2 < s1) continue;
                    return true;  // fluid above the last interval
                }
                if (kEnd <= kLast) return true;  // fluid starts inside the coarse cell
                if (fine.hits[s] <= kFirst) break;  // this fine column is solid throughout
                return true;  // fluid below the interval
            }
        }
    return false;
}

bool coarseHasWall(const RayMap& fine, int down, int i, int j, int k) {
    const int kFirst = k * down, kLast = kFirst + down - 1;
    for (int jAdd = 0; jAdd < down; ++jAdd)
        for (int iAdd = 0; iAdd < down; ++iAdd) {
            const size_t r = static_cast<size_t>(fine.nx) * (j * down + jAdd) + (i * down + iAdd);
            for (long long s = fine.scan[r]; s < fine.scan[r + 1]; s += 2) {
                const int kStart = fine.hits[s];
                if (kStart > kLast) break;            // intervals above the coarse cell
                if (kStart >= kFirst) return true;    // solid starts inside it
                if (fine.hits[s + 1] <= kFirst) continue;  // interval ends below it
                return true;                          // interval covers its bottom
            }
        }
    return false;
}

bool intersectRayTriangle(float ax, float ay, float az, float bx, float by, float bz, float cx, float cy,
                          float cz, float ex, float ey, float ez, float edgeTol, float& t) {
    const float e1x = bx - ax, e1y = by - ay, e1z = bz - az;
    const float e2x = cx - ax, e2y = cy - ay, e2z = cz - az;
    const float nx = e1y * e2z - e1z * e2y;
    const float ny = e1z * e2x - e1x * e2z;
    const float nz = e1x * e2y - e1y * e2x;
    const float area2 = std::sqrt(nx * nx + ny * ny + nz * nz);
    if (area2 == 0.f) return false;
    const float px = ey * e2z - ez * e2y;
    const float py = ez * e2x - ex * e2z;
    const float pz = ex * e2y - ey * e2x;
    const float det = e1x * px + e1y * py + e1z * pz;
    if (det > -1e-8f && det < 1e-8f) return false;
    const float invDet = 1.f / det;
    const float lenAB = std::sqrt(e1x * e1x + e1y * e1y + e1z * e1z);
    const float lenAC = std::sqrt(e2x * e2x + e2y * e2y + e2z * e2z);
    const float bcx = cx - bx, bcy = cy - by, bcz = cz - bz;
    const float lenBC = std::sqrt(bcx * bcx + bcy * bcy + bcz * bcz);
    const float uTol = edgeTol * lenAC / area2;
    const float vTol = edgeTol * lenAB / area2;
    const float wTol = edgeTol * lenBC / area2;
    const float tx = -ax, ty = -ay, tz = -az;
    const float u = (tx * px + ty * py + tz * pz) * invDet;
    if (u < -uTol) return false;
    const float qx = ty * e1z - tz * e1y;
    const float qy = tz * e1x - tx * e1z;
    const float qz = tx * e1y - ty * e1x;
    const float v = (ex * qx + ey * qy + ez * qz) * invDet;
    if (v < -vTol || u + v > 1.f + wTol) return false;
    t = (e2x * qx + e2y * qy + e2z * qz) * invDet;
    return true;
}

}  // namespace lbm
