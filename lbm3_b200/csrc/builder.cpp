// Host-side construction of the sparse, k-j-i sorted grid tables.
//
// Design: the reference builds its tables with ~40 GPU lambdas, atomic row
// binning, sorts and host-synchronising reductions
// (include/gridBuilderFunctions.h, include/NBRFunctions.h).  Setup is not on
// the timed path, so this builder works on the host over a dense occupancy
// map of the level's bounding box: cells are emitted directly in k-j-i order
// (no sort), and the row neighbours jPlus/kPlus come from one sweep per
// column instead of bin + insertion sort.  The resulting tables are the same
// as the reference's (the oracle checks them element by element).
#include "builder.h"

#include <algorithm>
#include <cmath>
#include <stdexcept>

namespace lbm {

namespace {

// Faces touched by (i,j,k); returns the winning face index or -1.
int winningFace(const lbm_case& c, const Info& info, int i, int j, int k) {
    const bool touch[6] = {i == 0, i == info.nx - 1, j == 0, j == info.ny - 1,
                           k == 0, k == info.nz - 1};
    int best = -1;
    for (int f = 0; f < 6; ++f) {
        if (!touch[f]) continue;
        if (best < 0 || c.face[f].priority > c.face[best].priority) best = f;
    }
    return best;
}

}  // namespace

BC evalOpenBC(const lbm_case& c, const Info& info, int i, int j, int k) {
    BC bc;
    const int f = winningFace(c, info, i, j, k);
    if (f < 0) return bc;
    const lbm_face_bc& fb = c.face[f];
    bc.openBCID = fb.open_bc_id;
    bc.nonReflective = fb.non_reflective != 0;
    bc.nonReflectiveBeta = fb.non_reflective_beta;
    switch (fb.kind) {
        case LBM_BC_PERIODIC: bc.periodic = true; break;
        case LBM_BC_VELOCITY:
            bc.dirichletU = true;
            bc.ux = fb.ux; bc.uy = fb.uy; bc.uz = fb.uz;
            break;
        case LBM_BC_PRESSURE:
            bc.dirichletRho = true;
            bc.dRho = fb.dRho;
            break;
        default: break;
    }
    return bc;
}

void evalLocalBC(const lbm_case& c, BC& bc) {
    bc.collisionLimiter = c.collision_limiter;
    bc.nuMultiplier = c.nu_multiplier;
}

BC evalInitialCondition(const lbm_case& c, const Info& info, int i, int j, int k) {
    BC bc;
    if (c.ic_kind == LBM_IC_TAYLOR_GREEN) {
        // cases/taylorGreenVortex/taylorGreenVortexMain.cu:66-87
        const float x = i * info.res + info.ox;
        const float y = j * info.res + info.oy;
        const float z = k * info.res + info.oz;
        const float X = x / c.tgv_length, Y = y / c.tgv_length, Z = z / c.tgv_length;
        const float u0 = c.tgv_u0;
        bc.ux = u0 * std::sin(X) * std::cos(Y) * std::cos(Z);
        bc.uy = -u0 * std::cos(X) * std::sin(Y) * std::cos(Z);
        bc.uz = 0.f;
        bc.dRho = (3.f * u0 * u0 / 16.f) * (std::cos(2.f * X) + std::cos(2.f * Y)) *
                  (2.f + std::cos(2.f * Z));
    } else {
        bc.dRho = c.ic_dRho;
        bc.ux = c.ic_ux; bc.uy = c.ic_uy; bc.uz = c.ic_uz;
    }
    return bc;
}

namespace {

void validateCase(const lbm_case& c) {
    if (c.grid_level_count != 1)
        throw std::runtime_error("grid_level_count must be 1 in this build");
    if (!(c.res_global > 0.f)) throw std::runtime_error("res_global must be > 0");
    if (!(c.dt_phys_global > 0.f)) throw std::runtime_error("dt_phys_global must be > 0");
    if (!(c.nu_phys > 0.f)) throw std::runtime_error("nu_phys must be > 0");
    for (int a = 0; a < 3; ++a)
        if (!(c.bounds[a + 3] > c.bounds[a]))
            throw std::runtime_error("bounds must satisfy min < max on every axis");
    for (int f = 0; f < 6; ++f) {
        const int kind = c.face[f].kind;
        if (kind != LBM_BC_PERIODIC && kind != LBM_BC_VELOCITY && kind != LBM_BC_PRESSURE)
            throw std::runtime_error("unknown face boundary kind");
        if (kind != LBM_BC_PERIODIC && c.face[f].open_bc_id < 0)
            throw std::runtime_error("open_bc_id must be >= 0");
    }
    if (c.storage != LBM_STORE_F32 && c.storage != LBM_STORE_F16 && c.storage != LBM_STORE_BF16)
        throw std::runtime_error("unknown storage precision");
}

// initializeGridInfo, level 0 (include/gridBuilderFunctions.h:9-64): the
// coarsest grid is laid on a skeleton of twice the resolution so that every
// kept skeleton cell contributes 2x2x2 cells.
void initLevel0(const lbm_case& c, Info& info, Info& skel) {
    const float* b = c.bounds;
    info.res = c.res_global;
    skel.res = info.res * 2.f;
    skel.nx = static_cast<int>((b[3] - b[0]) / skel.res);
    skel.ny = static_cast<int>((b[4] - b[1]) / skel.res);
    skel.nz = static_cast<int>((b[5] - b[2]) / skel.res);
    if (skel.nx < 1 || skel.ny < 1 || skel.nz < 1)
        throw std::runtime_error("domain smaller than two cells on some axis");
    skel.ox = b[0] + ((b[3] - b[0]) - (skel.nx * skel.res) + skel.res) / 2.0f;
    skel.oy = b[1] + ((b[4] - b[1]) - (skel.ny * skel.res) + skel.res) / 2.0f;
    skel.oz = b[2] + ((b[5] - b[2]) - (skel.nz * skel.res) + skel.res) / 2.0f;
    info.nx = skel.nx * 2;
    info.ny = skel.ny * 2;
    info.nz = skel.nz * 2;
    info.ox = skel.ox - info.res * 0.5f;
    info.oy = skel.oy - info.res * 0.5f;
    info.oz = skel.oz - info.res * 0.5f;
    info.dtPhys = c.dt_phys_global;
    info.nu = (info.dtPhys * c.nu_phys) / ((info.res / 1000.f) * (info.res / 1000.f));
    info.gridID = 0;
}

// Emit the kept cells in k-j-i order and wire jPlus/kPlus with periodic wrap
// inside each (i,k) and (i,j) line, as buildNBRPlus/connectNBRInRows do
// (include/NBRFunctions.h:44-152).
void buildCellsAndNBR(HostLevel& L, const std::vector<uint8_t>& keepFull) {
    const Info& in = L.info;
    const long long nx = in.nx, ny = in.ny, nz = in.nz;
    std::vector<int> idx(static_cast<size_t>(nx * ny * nz), -1);
    L.I.clear(); L.J.clear(); L.K.clear();
    int n = 0;
    for (long long k = 0; k < nz; ++k)
        for (long long j = 0; j < ny; ++j)
            for (long long i = 0; i < nx; ++i) {
                const size_t p = static_cast<size_t>((k * ny + j) * nx + i);
                if (!keepFull[p]) continue;
                idx[p] = n++;
                L.I.push_back(static_cast<int>(i));
                L.J.push_back(static_cast<int>(j));
                L.K.push_back(static_cast<int>(k));
            }
    L.info.cellCount = n;
    L.jPlus.assign(n, 0);
    L.kPlus.assign(n, 0);
    // jPlus: walk each (i,k) column along j.
    for (long long k = 0; k < nz; ++k)
        for (long long i = 0; i < nx; ++i) {
            int first = -1, prev = -1;
            for (long long j = 0; j < ny; ++j) {
                const int cidx = idx[static_cast<size_t>((k * ny + j) * nx + i)];
                if (cidx < 0) continue;
                if (prev >= 0) L.jPlus[prev] = cidx; else first = cidx;
                prev = cidx;
            }
            if (prev >= 0) L.jPlus[prev] = first;
        }
    // kPlus: walk each (i,j) column along k.
    for (long long j = 0; j < ny; ++j)
        for (long long i = 0; i < nx; ++i) {
            int first = -1, prev = -1;
            for (long long k = 0; k < nz; ++k) {
                const int cidx = idx[static_cast<size_t>((k * ny + j) * nx + i)];
                if (cidx < 0) continue;
                if (prev >= 0) L.kPlus[prev] = cidx; else first = cidx;
                prev = cidx;
            }
            if (prev >= 0) L.kPlus[prev] = first;
        }
    // geometric-validity bits (markGeometricNBRPlus, include/NBRFunctions.h:154-194)
    L.geomBits.assign(n, 0);
    auto wrap = [n](int v) { return v + 1 < n ? v + 1 : 0; };
    for (int cidx = 0; cidx < n; ++cidx) {
        const int i = L.I[cidx], j = L.J[cidx], k = L.K[cidx];
        const int iP = wrap(cidx), jP = L.jPlus[cidx], ijP = wrap(jP);
        const int kP = L.kPlus[cidx], ikP = wrap(kP), jkP = L.jPlus[kP], ijkP = wrap(jkP);
        const int nb[7] = {iP, jP, ijP, kP, ikP, jkP, ijkP};
        const int di[7] = {1, 0, 1, 0, 1, 0, 1};
        const int dj[7] = {0, 1, 1, 0, 0, 1, 1};
        const int dk[7] = {0, 0, 0, 1, 1, 1, 1};
        uint8_t bits = 0;
        for (int q = 0; q < 7; ++q)
            if (L.I[nb[q]] == i + di[q] && L.J[nb[q]] == j + dj[q] && L.K[nb[q]] == k + dk[q])
                bits |= static_cast<uint8_t>(1u << q);
        L.geomBits[cidx] = bits;
    }
}

// Compressed IJK/NBR (include/gridBuilderFunctions.h:1043-1126): a new row
// starts wherever i, j, k or any of jPlus/kPlus/jkPlus stops advancing by one.
void compressRows(HostLevel& L) {
    const int n = L.info.cellCount;
    L.shifter.assign(n, 0);
    L.rowI.clear(); L.rowJ.clear(); L.rowK.clear();
    L.rowJP.clear(); L.rowKP.clear(); L.rowJKP.clear();
    int head = 0;
    for (int c = 0; c < n; ++c) {
        bool newRow = (c == 0);
        if (!newRow) {
            const int jk = L.jPlus[L.kPlus[c]], jkPrev = L.jPlus[L.kPlus[c - 1]];
            newRow = L.I[c] != L.I[c - 1] + 1 || L.J[c] != L.J[c - 1] || L.K[c] != L.K[c - 1] ||
                     L.jPlus[c] != L.jPlus[c - 1] + 1 || L.kPlus[c] != L.kPlus[c - 1] + 1 ||
                     jk != jkPrev + 1;
        }
        if (newRow) {
            head = c;
            L.shifter[c] = static_cast<int>(L.rowI.size());
            L.rowI.push_back(L.I[c]);
            L.rowJ.push_back(L.J[c]);
            L.rowK.push_back(L.K[c]);
            L.rowJP.push_back(L.jPlus[c]);
            L.rowKP.push_back(L.kPlus[c]);
            L.rowJKP.push_back(L.jPlus[L.kPlus[c]]);
        } else {
            L.shifter[c] = head - c;
        }
    }
}

int findCell(const HostLevel& L, int i, int j, int k) {
    // binary search over the k-j-i sorted cells
    int lo = 0, hi = L.info.cellCount;
    while (lo < hi) {
        const int mid = lo + (hi - lo) / 2;
        const bool before = L.K[mid] < k || (L.K[mid] == k && L.J[mid] < j) ||
                            (L.K[mid] == k && L.J[mid] == j && L.I[mid] < i);
        if (L.I[mid] == i && L.J[mid] == j && L.K[mid] == k) return mid;
        if (before) lo = mid + 1; else hi = mid;
    }
    return -1;
}

void buildBoundaryLists(const lbm_case& c, HostLevel& L) {
    const Info& in = L.info;
    const int n = in.cellCount;
    L.wallMap.assign(n, -1);
    L.wallCellCount = 0;
    for (int cidx = 0; cidx < n; ++cidx)
        if (L.wallMarker[cidx]) { L.wallMap[cidx] = -3; ++L.wallCellCount; }
    L.wallAdjacentCount = 0;

    // Periodic overlap: no force/flow tracking in the ghost layers
    // (include/gridBuilderFunctions.h:1232-1274).
    const int layers = 1 << in.gridID;
    for (int cidx = 0; cidx < n; ++cidx) {
        if (L.wallMarker[cidx]) continue;
        const int i = L.I[cidx], j = L.J[cidx], k = L.K[cidx];
        bool overlap = false;
        if (i < layers || i >= in.nx - layers)
            overlap |= evalOpenBC(c, in, i < layers ? 0 : in.nx - 1, j, k).periodic;
        if (j < layers || j >= in.ny - layers)
            overlap |= evalOpenBC(c, in, i, j < layers ? 0 : in.ny - 1, k).periodic;
        if (k < layers || k >= in.nz - layers)
            overlap |= evalOpenBC(c, in, i, j, k < layers ? 0 : in.nz - 1).periodic;
        if (overlap && L.wallMap[cidx] == -1) L.wallMap[cidx] = -2;
    }

    // Open boundaries: one list per openBCID (:1276-1484).
    std::vector<int> bcid(n, -1);
    int maxId = -1;
    for (int cidx = 0; cidx < n; ++cidx) {
        if (L.wallMarker[cidx]) continue;
        const int i = L.I[cidx], j = L.J[cidx], k = L.K[cidx];
        if (i == 0 || i == in.nx - 1 || j == 0 || j == in.ny - 1 || k == 0 || k == in.nz - 1) {
            const BC bc = evalOpenBC(c, in, i, j, k);
            bcid[cidx] = bc.periodic ? -1 : bc.openBCID;
            maxId = std::max(maxId, bcid[cidx]);
        }
    }
    L.openBCs.assign(maxId + 1, OpenBCList{});
    for (int id = 0; id <= maxId; ++id) L.openBCs[id].openBCID = id;
    for (int cidx = 0; cidx < n; ++cidx)
        if (bcid[cidx] >= 0) L.openBCs[bcid[cidx]].index.push_back(cidx);
    for (auto& ob : L.openBCs) {
        ob.source.assign(ob.index.size(), -1);
        ob.trackFlowCount = 0;
        for (size_t q = 0; q < ob.index.size(); ++q) {
            const int cidx = ob.index[q];
            if (L.wallMap[cidx] != -2) ++ob.trackFlowCount;
            const int i = L.I[cidx], j = L.J[cidx], k = L.K[cidx];
            const int onx = i == 0 ? -1 : (i == in.nx - 1 ? 1 : 0);
            const int ony = j == 0 ? -1 : (j == in.ny - 1 ? 1 : 0);
            const int onz = k == 0 ? -1 : (k == in.nz - 1 ? 1 : 0);
            const int faces = (onx != 0) + (ony != 0) + (onz != 0);
            const BC bc = evalOpenBC(c, in, i, j, k);
            const bool edgeFallback = bc.dirichletU && faces == 2;
            int pref = 0;
            if (edgeFallback) {
                if (onx == 0) pref = i <= in.nx - 1 - i ? 1 : -1;
                else if (ony == 0) pref = j <= in.ny - 1 - j ? 1 : -1;
                else pref = k <= in.nz - 1 - k ? 1 : -1;
            }
            const int candidates = edgeFallback ? 3 : 1;
            int src = -1;
            for (int cand = 0; cand < candidates && src < 0; ++cand) {
                int is = i - onx, js = j - ony, ks = k - onz;
                if (cand > 0) {
                    const int sh = cand == 1 ? pref : -pref;
                    if (onx == 0) is += sh; else if (ony == 0) js += sh; else ks += sh;
                }
                if (is <= 0 || is >= in.nx - 1 || js <= 0 || js >= in.ny - 1 || ks <= 0 ||
                    ks >= in.nz - 1)
                    continue;
                const int found = findCell(L, is, js, ks);
                if (found < 0) continue;
                if (bc.dirichletU && faces > 1 && L.wallMarker[found]) continue;
                src = found;
            }
            if (src < 0)
                throw std::runtime_error(
                    "Building open BC failed: no valid source for some cells");
            ob.source[q] = src;
        }
    }

    // Periodic ghost lists (:1486-1564).
    L.perIndex.clear();
    L.perSource.clear();
    const int per = static_cast<int>(std::lround(std::pow(2.0, in.gridID)));
    for (int cidx = 0; cidx < n; ++cidx) {
        if (L.wallMarker[cidx]) continue;
        int i = L.I[cidx], j = L.J[cidx], k = L.K[cidx];
        if (!(i == 0 || i == in.nx - 1 || j == 0 || j == in.ny - 1 || k == 0 || k == in.nz - 1))
            continue;
        if (!evalOpenBC(c, in, i, j, k).periodic) continue;
        if (i == 0) i = in.nx - 2 * per; else if (i == in.nx - 1) i = 2 * per - 1;
        if (j == 0) j = in.ny - 2 * per; else if (j == in.ny - 1) j = 2 * per - 1;
        if (k == 0) k = in.nz - 2 * per; else if (k == in.nz - 1) k = 2 * per - 1;
        int src = findCell(L, i, j, k);
        if (src >= 0 && L.wallMarker[src]) src = -1;
        if (src < 0)
            throw std::runtime_error(
                "Building periodic BC failed, some source cells do not exist or are marked as wall");
        L.perIndex.push_back(cidx);
        L.perSource.push_back(src);
    }
}

}  // namespace

void buildSegments(HostLevel& L) {
    L.segCell.clear(); L.segJP.clear(); L.segKP.clear(); L.segJKP.clear(); L.segLen.clear();
    L.specialCells.clear();
    const int n = L.info.cellCount;
    int c = 0;
    while (c < n) {
        // extent of the compressed row starting at c
        int end = c + 1;
        while (end < n && L.shifter[end] < 0) ++end;
        const int row = L.shifter[c];
        // neighbours of the cell at offset `off` in this row
        auto jP = [&](int off) { return L.rowJP[row] + off; };
        auto kP = [&](int off) { return L.rowKP[row] + off; };
        auto jkP = [&](int off) { return L.rowJKP[row] + off; };
        // a +1 neighbour that wraps to cell 0 (finishNBRPlus) breaks the
        // linear run, so such a cell is collided from the special list
        auto wraps = [&](int q) {
            const int off = q - c;
            return q + 1 >= n || jP(off) + 1 >= n || kP(off) + 1 >= n || jkP(off) + 1 >= n;
        };
        auto bulk = [&](int q) {
            return (L.wallMap[q] == -1 || L.wallMap[q] == -2) && !wraps(q);
        };
        for (int q = c; q < end;) {
            if (L.wallMap[q] == -3) { ++q; continue; }
            if (!bulk(q)) { L.specialCells.push_back(q); ++q; continue; }
            int r = q;
            while (r < end && r - q < kSegmentCells && bulk(r)) ++r;
            const int off = q - c;
            L.segCell.push_back(q);
            L.segJP.push_back(jP(off));
            L.segKP.push_back(kP(off));
            L.segJKP.push_back(jkP(off));
            L.segLen.push_back(r - q);
            q = r;
        }
        c = end;
    }
}

void buildDomain(const lbm_case& c, HostDomain& out) {
    validateCase(c);
    out.c = c;
    out.levels.assign(1, HostLevel{});
    HostLevel& L = out.levels[0];
    Info skel;
    initLevel0(c, L.info, skel);

    // Without static geometry every skeleton cell is kept (markKeepCells,
    // include/markerFunctions.h:401-409, over an empty ray map).
    const size_t full = static_cast<size_t>(L.info.nx) * L.info.ny * L.info.nz;
    std::vector<uint8_t> keep(full, 1);
    buildCellsAndNBR(L, keep);
    L.wallMarker.assign(L.info.cellCount, 0);
    compressRows(L);
    buildBoundaryLists(c, L);
    buildSegments(L);

    out.fluidUpdatesPerIteration = 0;
    for (const HostLevel& lv : out.levels)
        out.fluidUpdatesPerIteration +=
            static_cast<long long>(lv.info.cellCount - lv.wallCellCount) *
            (1LL << lv.info.gridID);
}

}  // namespace lbm
