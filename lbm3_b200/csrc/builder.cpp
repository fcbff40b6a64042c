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
#include "mbbc_tables.h"
#include "geometry.h"
#include "lattice.h"

#include <algorithm>
#include <cstdlib>
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

namespace {

lbm_bc toHookBC(const BC& b) {
    lbm_bc h;
    h.dRho = b.dRho; h.ux = b.ux; h.uy = b.uy; h.uz = b.uz;
    h.gx = b.gx; h.gy = b.gy; h.gz = b.gz;
    h.wallID = b.wallID; h.openBCID = b.openBCID;
    h.useIBB = b.useIBB; h.dirichletU = b.dirichletU; h.dirichletRho = b.dirichletRho;
    h.periodic = b.periodic; h.nonReflective = b.nonReflective;
    h.nonReflectiveBeta = b.nonReflectiveBeta; h.collisionLimiter = b.collisionLimiter;
    h.nuMultiplier = b.nuMultiplier;
    return h;
}

BC fromHookBC(const lbm_bc& h) {
    BC b;
    b.dRho = h.dRho; b.ux = h.ux; b.uy = h.uy; b.uz = h.uz;
    b.gx = h.gx; b.gy = h.gy; b.gz = h.gz;
    b.wallID = h.wallID; b.openBCID = h.openBCID;
    b.useIBB = h.useIBB != 0; b.dirichletU = h.dirichletU != 0; b.dirichletRho = h.dirichletRho != 0;
    b.periodic = h.periodic != 0; b.nonReflective = h.nonReflective != 0;
    b.nonReflectiveBeta = h.nonReflectiveBeta; b.collisionLimiter = h.collisionLimiter;
    b.nuMultiplier = h.nuMultiplier;
    return b;
}

// The level's InfoStruct as a hook sees it.
lbm_grid_info hookInfo(const Info& in) {
    lbm_grid_info g{};
    g.grid_id = in.gridID;
    g.cell_count = in.cellCount;
    g.cell_count_x = in.nx;
    g.cell_count_y = in.ny;
    g.cell_count_z = in.nz;
    g.res = in.res;
    g.ox = in.ox;
    g.oy = in.oy;
    g.oz = in.oz;
    g.nu = in.nu;
    g.dt_phys = in.dtPhys;
    g.iterations_finished = in.iterationsFinished;
    return g;
}

// Call a driver hook on a BCStruct that starts from `start`.
BC callHook(const lbm_case& c, lbm_cell_hook hook, const BC& start, const Info& info, int i, int j, int k) {
    lbm_bc h = toHookBC(start);
    const lbm_grid_info gi = hookInfo(info);
    hook(c.hook_user, &h, i, j, k, &gi);
    return fromHookBC(h);
}

}  // namespace

BC evalOpenBC(const lbm_case& c, const Info& info, int i, int j, int k) {
    if (c.open_bc_hook) return callHook(c, c.open_bc_hook, BC{}, info, i, j, k);
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

BC levelLocalBC(const lbm_case& c, const HostLevel& L) {
    BC bc;
    evalLocalBC(c, bc);
    bc.gx = c.gx;
    bc.gy = c.gy;
    bc.gz = c.gz;
    bc.useIBB = c.use_ibb != 0;
    bc.wallID = -1;
    if (c.local_bc_hook && L.info.cellCount > 0) bc = callHook(c, c.local_bc_hook, bc, L.info, L.I[0], L.J[0], L.K[0]);
    return bc;
}

BC evalInitialCondition(const lbm_case& c, const Info& info, int i, int j, int k) {
    if (c.initial_condition_hook) return callHook(c, c.initial_condition_hook, BC{}, info, i, j, k);
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
    if (c.grid_level_count < 1 || c.grid_level_count > LBM_MAX_LEVELS)
        throw std::runtime_error("grid_level_count must be in [1, LBM_MAX_LEVELS]");
    if (c.wall_refinement_count < 0) throw std::runtime_error("wall_refinement_count must be >= 0");
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
    if (c.storage != LBM_STORE_F32 && c.storage != LBM_STORE_F16 && c.storage != LBM_STORE_BF16 &&
        c.storage != LBM_STORE_F64)
        throw std::runtime_error("unknown storage precision");
    if (c.open_bc_scheme != LBM_OPEN_CHARACTERISTIC && c.open_bc_scheme != LBM_OPEN_IMPEDANCE)
        throw std::runtime_error("unknown open-boundary scheme");
    if (c.open_bc_scheme == LBM_OPEN_IMPEDANCE && !(c.rho_reflection_tolerance >= 0.f))
        throw std::runtime_error("RHO_REFLECTION_TOLERANCE must be non-negative");
    if (c.body_count < 0 || c.body_count > LBM_MAX_BODIES)
        throw std::runtime_error("body_count must be in [0, LBM_MAX_BODIES]");
    for (int b = 0; b < c.body_count; ++b) {
        const lbm_body& bd = c.body[b];
        if (bd.triangle_count <= 0 || !bd.triangles)
            throw std::runtime_error("voxelizeSTL failed: the passed STL has 0 triangles.");
        if (bd.motion != LBM_WALL_STATIC && bd.motion != LBM_WALL_ROTATING)
            throw std::runtime_error("unknown wall motion");
        if (bd.motion == LBM_WALL_ROTATING && (bd.axis < 0 || bd.axis > 2))
            throw std::runtime_error("rotation axis must be 0, 1 or 2");
    }
    if (c.rotor_count < 0 || c.rotor_count > LBM_MAX_ROTORS)
        throw std::runtime_error("rotor_count must be in [0, LBM_MAX_ROTORS]");
    for (int r = 0; r < c.rotor_count; ++r) {
        const lbm_rotor& rt = c.rotor[r];
        if (rt.triangle_count <= 0 || !rt.triangles)
            throw std::runtime_error("voxelizeSTL failed: the passed STL has 0 triangles.");
        if (rt.axis < 0 || rt.axis > 2) throw std::runtime_error("rotor axis must be 0, 1 or 2");
    }
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
    // NBR minus as the inverse of the plus permutations (gridBuilderFunctions.h:565-575)
    L.jMinus.assign(n, 0);
    L.kMinus.assign(n, 0);
    for (int cidx = 0; cidx < n; ++cidx) {
        L.jMinus[L.jPlus[cidx]] = cidx;
        L.kMinus[L.kPlus[cidx]] = cidx;
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
    for (int cidx = 0; cidx < n; ++cidx) {
        if (L.wallMarker[cidx]) { L.wallMap[cidx] = -3; ++L.wallCellCount; }
        else if (!L.interfaceOverlap.empty() && L.interfaceOverlap[cidx]) L.wallMap[cidx] = -2;
    }
    L.wallAdjacentCount = static_cast<int>(L.wallIndex.size());
    for (int w = 0; w < L.wallAdjacentCount; ++w) L.wallMap[L.wallIndex[w]] = w;

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
        if (!overlap) continue;
        if (L.wallMap[cidx] >= 0) L.wallData[L.wallMap[cidx]] |= 1u;
        else if (L.wallMap[cidx] == -1) L.wallMap[cidx] = -2;
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
            const int wmap = L.wallMap[cidx];
            if (wmap != -2 && !(wmap >= 0 && (L.wallData[wmap] & 1u))) ++ob.trackFlowCount;
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
    // per-cell records for the open-boundary kernel (include/updateGrid.h:183-355)
    L.openCells.clear();
    for (const auto& ob : L.openBCs)
        for (size_t q = 0; q < ob.index.size(); ++q) {
            const int cidx = ob.index[q];
            const int i = L.I[cidx], j = L.J[cidx], k = L.K[cidx];
            const int onx = i == 0 ? -1 : (i == in.nx - 1 ? 1 : 0);
            const int ony = j == 0 ? -1 : (j == in.ny - 1 ? 1 : 0);
            const int onz = k == 0 ? -1 : (k == in.nz - 1 ? 1 : 0);
            const BC bc = evalOpenBC(c, in, i, j, k);
            // non-reflectivity is defined for face cells only (:262-265)
            const bool nonRefl = bc.nonReflective && (std::abs(onx) + std::abs(ony) + std::abs(onz) == 1);
            int kind = bc.dirichletRho ? 2 : (bc.dirichletU ? 1 : 0);
            const int wm = L.wallMap[cidx];
            bool track = wm != -2;
            if (wm >= 0 && (L.wallData[wm] & 1u)) track = false;
            const int code = (onx + 5) * 100 + (ony + 5) * 10 + (onz + 5);
            int row = -1;
            for (int t = 0; t < LBM_MBBC_NORMALS; ++t)
                if (kLbmMbbc[t].code == code) row = t;
            if (row < 0) throw std::logic_error("open boundary cell without an outer normal");
            OpenBCCell oc;
            oc.cell = cidx;
            oc.info = kind | (nonRefl ? 4 : 0) | ((onx + 1) << 3) | ((ony + 1) << 5) | ((onz + 1) << 7) |
                      (track ? 512 : 0) | (row << 10) | (ob.openBCID << 16);
            oc.dRho = bc.dRho;
            oc.ux = bc.ux;
            oc.uy = bc.uy;
            oc.uz = bc.uz;
            oc.beta = bc.nonReflectiveBeta;
            L.openCells.push_back(oc);
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

namespace {

// The 7 plus neighbours of a cell (iPlus, jPlus, ijPlus, kPlus, ikPlus,
// jkPlus, ijkPlus) with the +1 wrap of finishNBRPlus.
void plusNbrs(const HostLevel& L, int c, int (&nb)[7]) {
    const int n = L.info.cellCount;
    auto wrap = [n](int v) { return v + 1 < n ? v + 1 : 0; };
    nb[0] = wrap(c);
    nb[1] = L.jPlus[c];
    nb[2] = wrap(nb[1]);
    nb[3] = L.kPlus[c];
    nb[4] = wrap(nb[3]);
    nb[5] = L.jPlus[nb[3]];
    nb[6] = wrap(nb[5]);
}

// spreadMarkers over the cell list (include/markerFunctions.h:344-399): a cell
// is marked when it or a geometric plus neighbour is; a marked cell also marks
// all its geometric plus neighbours.
std::vector<uint8_t> spreadCells(const HostLevel& L, const std::vector<uint8_t>& src) {
    std::vector<uint8_t> out = src;
    const int n = L.info.cellCount;
    for (int c = 0; c < n; ++c) {
        int nb[7];
        plusNbrs(L, c, nb);
        const uint8_t bits = L.geomBits[c];
        bool marker = src[c] != 0;
        for (int q = 0; q < 7 && !marker; ++q)
            if (((bits >> q) & 1u) && src[nb[q]]) marker = true;
        if (!marker) continue;
        out[c] = 1;
        for (int q = 0; q < 7; ++q)
            if ((bits >> q) & 1u) out[nb[q]] = 1;
    }
    return out;
}

// spreadMarkers on the dense skeleton (include/markerFunctions.h:290-342): 26 neighbours.
std::vector<uint8_t> spreadDense(const std::vector<uint8_t>& src, int nx, int ny, int nz) {
    std::vector<uint8_t> out = src;
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const size_t c = (static_cast<size_t>(k) * ny + j) * nx + i;
                if (src[c]) continue;
                bool hit = false;
                for (int dk = -1; dk <= 1 && !hit; ++dk)
                    for (int dj = -1; dj <= 1 && !hit; ++dj)
                        for (int di = -1; di <= 1 && !hit; ++di) {
                            if (!dk && !dj && !di) continue;
                            const int a = i + di, b = j + dj, e = k + dk;
                            if (a < 0 || a >= nx || b < 0 || b >= ny || e < 0 || e >= nz) continue;
                            if (src[(static_cast<size_t>(e) * ny + b) * nx + a]) hit = true;
                        }
                if (hit) out[c] = 1;
            }
    return out;
}

// Full 26-neighbour list of a cell reached through the plus/minus chains, as
// buildLinkExistenceMarkerArray forms it (interpolatedBouncebackFunctions.h:227-260).
void fullNbrList(const HostLevel& L, int c, int (&nb)[27]) {
    const int n = L.info.cellCount;
    const auto& jP = L.jPlus;
    const auto& kP = L.kPlus;
    const auto& jM = L.jMinus;
    const auto& kM = L.kMinus;
    const int iPlus = c + 1 >= n ? 0 : c + 1;
    const int iMinus = c - 1 < 0 ? n - 1 : c - 1;
    nb[OOO] = c;
    nb[POO] = iPlus;
    nb[MOO] = iMinus;
    nb[OOM] = kM[c];
    nb[OOP] = kP[c];
    nb[OMO] = jM[c];
    nb[OPO] = jP[c];
    nb[POM] = kM[iPlus];
    nb[MOP] = kP[iMinus];
    nb[POP] = kP[iPlus];
    nb[MOM] = kM[iMinus];
    nb[MMO] = jM[iMinus];
    nb[PPO] = jP[iPlus];
    nb[OPM] = kM[jP[c]];
    nb[OMP] = kP[jM[c]];
    nb[MPO] = jP[iMinus];
    nb[PMO] = jM[iPlus];
    nb[OPP] = jP[kP[c]];
    nb[OMM] = kM[jM[c]];
    nb[MPM] = kM[jP[iMinus]];
    nb[PMP] = kP[jM[iPlus]];
    nb[MMP] = kP[jM[iMinus]];
    nb[PPM] = kM[jP[iPlus]];
    nb[PMM] = kM[jM[iPlus]];
    nb[MPP] = jP[kP[iMinus]];
    nb[MMM] = kM[jM[iMinus]];
    nb[PPP] = jP[kP[iPlus]];
}

// Links of one wall-adjacent cell (buildLinkExistenceMarkerArray,
// interpolatedBouncebackFunctions.h:181-398).  `iface` marks the cells of an
// interface band (a parent on the coarser level, or fine-to-coarse /
// coarse-to-fine on this one; empty on a single level); a link from or to such
// a cell is returned in `pierce` and later gets length 1/2.
uint32_t linkBits(const HostLevel& L, int c, const std::vector<uint8_t>& iface, uint32_t& pierce) {
    const Info& in = L.info;
    int nb[27];
    fullNbrList(L, c, nb);
    const int i = L.I[c], j = L.J[c], k = L.K[c];
    bool geom[27];
    bool all = true, ip = true, jp = true, kp = true, im = true, jm = true, km = true;
    for (int d = 1; d < 27; ++d) {
        geom[d] = true;
        const int ie = i + cx(d), je = j + cy(d), ke = k + cz(d);
        const int q = nb[d];
        if (L.I[q] == ie && L.J[q] == je && L.K[q] == ke) continue;
        geom[d] = false;
        if (ie < 0 || ie >= in.nx || je < 0 || je >= in.ny || ke < 0 || ke >= in.nz) continue;
        all = false;
        if (cx(d) > 0) ip = false;
        if (cy(d) > 0) jp = false;
        if (cz(d) > 0) kp = false;
        if (cx(d) < 0) im = false;
        if (cy(d) < 0) jm = false;
        if (cz(d) < 0) km = false;
    }
    uint32_t bits = 0;
    pierce = 0;
    const bool meInterface = !iface.empty() && iface[c];
    auto add = [&](int d) {
        bits |= 1u << d;
        if (meInterface || (!iface.empty() && iface[nb[d]])) pierce |= 1u << d;
    };
    const bool interior = i != 0 && i != in.nx - 1 && j != 0 && j != in.ny - 1 && k != 0 && k != in.nz - 1;
    if (interior) {
        if (!all) return 0;
        for (int d = 1; d < 27; ++d)
            if (L.wallMarker[nb[d]]) add(d);
        return bits;
    }
    for (int d = 1; d < 27; ++d) {
        if (!geom[d] || !L.wallMarker[nb[d]]) continue;
        if ((cx(d) > 0 && !ip) || (cy(d) > 0 && !jp) || (cz(d) > 0 && !kp)) continue;
        if ((cx(d) < 0 && !im) || (cy(d) < 0 && !jm) || (cz(d) < 0 && !km)) continue;
        add(d);
    }
    return bits;
}

// Markers of one level that live only while the domain is built
// (GridBuilderStruct, include/types.h:181-190).
struct LevelMarks {
    std::vector<uint8_t> deep, f2c, c2f, refine;  // levels with a finer one
    std::vector<int> parent;                        // levels with a coarser one: parent cell or -1
    std::vector<uint8_t> parentInterface, parentF2C, needValues;
    std::vector<int> wallIDFull;                    // wallIDArrayFull: body of a wall-adjacent cell or -1
};

// Wall markers, wall IDs, wall-adjacent list, link existence and link lengths
// (buildWallMarkers, include/gridBuilderFunctions.h:590-739, and
// buildLinkLengthArray, interpolatedBouncebackFunctions.h:482-660), then the
// packed wallData / linkLength words (packWallData, :662-695).
// On a finer level (`coarse` set) cells with a parent inherit the parent's
// wall state and body marks, and a wall-adjacent cell takes its parent's
// wallID when the parent has one (buildWallMarkers steps 1-2).
void buildWalls(const lbm_case& c, HostLevel& L, LevelMarks& M, const HostLevel* coarse, const LevelMarks* CM,
                const std::vector<Triangles>& bodies, const std::vector<RayMap>& maps, const RayMap& total,
                const std::vector<RayMap>* coarseMaps, const std::vector<uint8_t>& iface) {
    const Info& in = L.info;
    const int n = in.cellCount;
    L.wallMarker.assign(n, 0);
    for (int q = 0; q < n; ++q) L.wallMarker[q] = isSolid(total, L.I[q], L.J[q], L.K[q]) ? 1 : 0;
    if (coarse)
        for (int q = 0; q < n; ++q)
            if (M.parent[q] >= 0) L.wallMarker[q] = coarse->wallMarker[M.parent[q]];
    std::vector<int> wallID(n, -1);
    for (size_t b = 0; b < maps.size(); ++b) {
        std::vector<uint8_t> body(n, 0);
        for (int q = 0; q < n; ++q) body[q] = isSolid(maps[b], L.I[q], L.J[q], L.K[q]) ? 1 : 0;
        if (coarse)
            for (int q = 0; q < n; ++q) {
                const int p = M.parent[q];
                if (p >= 0) body[q] = isSolid((*coarseMaps)[b], coarse->I[p], coarse->J[p], coarse->K[p]) ? 1 : 0;
            }
        body = spreadCells(L, body);
        for (int q = 0; q < n; ++q) {
            if (!body[q] || L.wallMarker[q]) continue;
            int id = static_cast<int>(b);  // last body wins
            if (coarse && M.parent[q] >= 0 && CM->wallIDFull[M.parent[q]] >= 0) id = CM->wallIDFull[M.parent[q]];
            wallID[q] = id;
        }
    }
    M.wallIDFull = wallID;
    L.wallIndex.clear();
    std::vector<int> ids;
    for (int q = 0; q < n; ++q)
        if (wallID[q] >= 0) {
            L.wallIndex.push_back(q);
            ids.push_back(wallID[q]);
        }
    const int nw = static_cast<int>(L.wallIndex.size());
    std::vector<uint32_t> links(nw, 0), pierce(nw, 0);
    for (int w = 0; w < nw; ++w) links[w] = linkBits(L, L.wallIndex[w], iface, pierce[w]);

    // link lengths: nearest triangle crossing of each link, per body bins
    std::vector<float> len(static_cast<size_t>(nw) * 27, 2.f);
    const float edgeTol = 0.1f * in.res;
    const float qTol = 0.2f;
    for (const Triangles& t : bodies) {
        const int bxy = t.binCountX * t.binCountY;
        for (int w = 0; w < nw; ++w) {
            if (!links[w]) continue;
            const int cell = L.wallIndex[w];
            const float x = L.I[cell] * in.res + in.ox;
            const float y = L.J[cell] * in.res + in.oy;
            const float z = L.K[cell] * in.res + in.oz;
            const int ib = static_cast<int>((x - t.oxBin) / t.binSize);
            const int jb = static_cast<int>((y - t.oyBin) / t.binSize);
            const int kb = static_cast<int>((z - t.ozBin) / t.binSize);
            if (ib < 0 || ib >= t.binCountX || jb < 0 || jb >= t.binCountY || kb < 0 || kb >= t.binCountZ)
                continue;
            const int bin = bxy * kb + t.binCountX * jb + ib;
            for (int r = t.firstInBin[bin]; r < t.firstInBin[bin + 1]; ++r) {
                const int tri = t.bin[r];
                const float ax = t.ax[tri] - x, ay = t.ay[tri] - y, az = t.az[tri] - z;
                const float bx = t.bx[tri] - x, by = t.by[tri] - y, bz = t.bz[tri] - z;
                const float cxv = t.cx[tri] - x, cyv = t.cy[tri] - y, czv = t.cz[tri] - z;
                for (int d = 1; d < 27; ++d) {
                    if (!((links[w] >> d) & 1u) || ((pierce[w] >> d) & 1u)) continue;
                    float tHit;
                    if (!intersectRayTriangle(ax, ay, az, bx, by, bz, cxv, cyv, czv, float(cx(d)), float(cy(d)),
                                              float(cz(d)), edgeTol, tHit))
                        continue;
                    float q = tHit / in.res;
                    float& slot = len[static_cast<size_t>(w) * 27 + d];
                    if (q > 0 && q <= 1.f) {  // accurate crossing
                        q = std::clamp(q, 0.00001f, 1.f);
                        if (slot < 0.f || q < slot) slot = q;
                    } else if (q > -qTol && q <= 1.f + qTol) {  // near miss, kept as negative
                        q = std::clamp(q, 0.00001f, 1.f);
                        if (slot < 0.f) {
                            if (q < -slot) slot = -q;
                        } else if (slot > 1.f) {
                            slot = -q;
                        }
                    }
                }
            }
        }
    }
    L.linksTotal = 0;
    L.linksNotFound = 0;
    for (int w = 0; w < nw; ++w)
        for (int d = 1; d < 27; ++d) {
            if (!((links[w] >> d) & 1u)) continue;
            ++L.linksTotal;
            float& slot = len[static_cast<size_t>(w) * 27 + d];
            if ((pierce[w] >> d) & 1u) {
                slot = 0.5f;  // crosses an interface: the same length on both levels
            } else if (slot > 1.f) {
                slot = 0.5f;  // no crossing found: safe fallback
                ++L.linksNotFound;
            } else if (slot < 0.f) {
                slot = -slot;
            }
        }

    // pack
    L.wallData.assign(nw, 0);
    L.linkLength.assign(static_cast<size_t>(7) * nw, 0);
    L.wallVelocity.assign(static_cast<size_t>(3) * nw, 0.f);
    for (int w = 0; w < nw; ++w) {
        uint32_t data = static_cast<uint32_t>(ids[w]) << 27;
        if (!L.interfaceOverlap.empty() && L.interfaceOverlap[L.wallIndex[w]]) data |= 1u;
        int li = 0;
        for (int d = 1; d < 27; ++d) {
            if (!((links[w] >> d) & 1u)) continue;
            data |= 1u << d;
            const float q = std::clamp(len[static_cast<size_t>(w) * 27 + d], 0.f, 1.f);
            const uint32_t code = static_cast<uint32_t>(q * 254.f + 0.5f);
            L.linkLength[static_cast<size_t>(li / 4) * nw + w] |= code << (8 * (li % 4));
            ++li;
        }
        L.wallData[w] = data;
        // getLocalBC wall velocity of the body (evaluated at the fluid cell centre)
        const lbm_body& body = c.body[ids[w]];
        if (c.local_bc_hook) {
            const int cell = L.wallIndex[w];
            BC start;
            start.wallID = ids[w];
            const BC bc = callHook(c, c.local_bc_hook, start, in, L.I[cell], L.J[cell], L.K[cell]);
            L.wallVelocity[static_cast<size_t>(0) * nw + w] = bc.ux;
            L.wallVelocity[static_cast<size_t>(1) * nw + w] = bc.uy;
            L.wallVelocity[static_cast<size_t>(2) * nw + w] = bc.uz;
        } else if (body.motion == LBM_WALL_ROTATING) {
            const int cell = L.wallIndex[w];
            const float x = L.I[cell] * in.res + in.ox - body.origin[0];
            const float y = L.J[cell] * in.res + in.oy - body.origin[1];
            const float z = L.K[cell] * in.res + in.oz - body.origin[2];
            const float s = body.radians_per_second * in.dtPhys / in.res;
            float u[3] = {0.f, 0.f, 0.f};
            if (body.axis == 2) { u[0] = -s * y; u[1] = s * x; }
            else if (body.axis == 0) { u[1] = -s * z; u[2] = s * y; }
            else { u[2] = -s * x; u[0] = s * z; }
            for (int a = 0; a < 3; ++a) L.wallVelocity[static_cast<size_t>(a) * nw + w] = u[a];
        }
    }
}

}  // namespace

void buildRotors(const lbm_case& c, HostLevel& L) {
    L.rotors.clear();
    L.rotorCell.assign(L.info.cellCount, 0);
    for (int r = 0; r < c.rotor_count; ++r) {
        const lbm_rotor& rt = c.rotor[r];
        Triangles t;
        loadTriangles(rt.triangles, rt.triangle_count, t);
        if (t.count == 0) throw std::runtime_error("voxelizeSTL failed: the passed STL has 0 triangles.");
        // 1) voxelize at half the level spacing over the rotor's own bounds
        const float vres = L.info.res * 0.5f;
        const int vnx = static_cast<int>((t.xMax - t.xMin) / vres) + 2;
        const int vny = static_cast<int>((t.yMax - t.yMin) / vres) + 2;
        const int vnz = static_cast<int>((t.zMax - t.zMin) / vres) + 2;
        RayMap map;
        voxelize(t, t.xMin, t.yMin, t.zMin, vres, vnx, vny, map);
        HostRotor R;
        R.res = vres;
        R.xMin = t.xMin - 1.5f * vres;
        R.yMin = t.yMin - 1.5f * vres;
        R.zMin = t.zMin - 1.5f * vres;
        // two cells of overlap, rounded up to whole blocks of 4
        R.cntX = ((vnx + 2 + 3) / 4) * 4;
        R.cntY = ((vny + 2 + 3) / 4) * 4;
        R.cntZ = ((vnz + 2 + 3) / 4) * 4;
        R.xMax = R.xMin + R.res * static_cast<float>(R.cntX);
        R.yMax = R.yMin + R.res * static_cast<float>(R.cntY);
        R.zMax = R.zMin + R.res * static_cast<float>(R.cntZ);
        R.axis = rt.axis;
        R.ox = rt.origin[0];
        R.oy = rt.origin[1];
        R.oz = rt.origin[2];
        R.radiansPerSecond = rt.radians_per_second;
        const int bx = R.cntX / 4, by = R.cntY / 4, bz = R.cntZ / 4;
        const int blocks = bx * by * bz;
        // 6x6x6 voxel marks around a block: voxel v of block b sits at
        // local (v - (4 b - 2)); its corner counters are local c..c+1
        auto marks = [&](int ib, int jb, int kb, uint8_t (&m)[216]) {
            bool any = false;
            for (int q = 0; q < 216; ++q) m[q] = 0;
            for (int j = std::max(0, jb * 4 - 2); j < std::min(vny, jb * 4 + 4); ++j)
                for (int i = std::max(0, ib * 4 - 2); i < std::min(vnx, ib * 4 + 4); ++i)
                    for (int k = kb * 4 - 2; k < kb * 4 + 4; ++k)
                        if (isSolid(map, i, j, k)) {
                            m[(k - (kb * 4 - 2)) * 36 + (j - (jb * 4 - 2)) * 6 + (i - (ib * 4 - 2))] = 1;
                            any = true;
                        }
            return any;
        };
        // 2-3) rotorMap and the compact block index
        R.rotorMap.assign(blocks, -1);
        for (int b = 0; b < blocks; ++b) {
            const int kb = b / (bx * by), rem = b % (bx * by), jb = rem / bx, ib = rem % bx;
            uint8_t m[216];
            if (marks(ib, jb, kb, m)) {
                R.rotorMap[b] = static_cast<int>(R.index.size());
                R.index.push_back(b);
            }
        }
        // 4) counter points (5x5x5 per block) and packed corner counts
        R.interpolation.assign(R.index.size() * 64, 0u);
        for (size_t n = 0; n < R.index.size(); ++n) {
            const int b = R.index[n];
            const int kb = b / (bx * by), rem = b % (bx * by), jb = rem / bx, ib = rem % bx;
            uint8_t m[216];
            marks(ib, jb, kb, m);
            uint8_t counter[125];
            for (int kc = 0; kc < 5; ++kc)
                for (int jc = 0; jc < 5; ++jc)
                    for (int ic = 0; ic < 5; ++ic) {
                        int cnt = 0;
                        for (int km = kc; km <= kc + 1; ++km)
                            for (int jm = jc; jm <= jc + 1; ++jm)
                                for (int im = ic; im <= ic + 1; ++im) cnt += m[km * 36 + jm * 6 + im];
                        counter[kc * 25 + jc * 5 + ic] = static_cast<uint8_t>(cnt);
                    }
            for (int ki = 0; ki < 4; ++ki)
                for (int ji = 0; ji < 4; ++ji)
                    for (int ii = 0; ii < 4; ++ii) {
                        uint32_t packedCounts = 0u;
                        int corner = 0;
                        for (int kc = ki; kc <= ki + 1; ++kc)
                            for (int jc = ji; jc <= ji + 1; ++jc)
                                for (int ic = ii; ic <= ii + 1; ++ic, ++corner)
                                    packedCounts |= static_cast<uint32_t>(counter[kc * 25 + jc * 5 + ic]) << (4 * corner);
                        R.interpolation[n * 64 + ki * 16 + ji * 4 + ii] = packedCounts;
                    }
        }
        // cells the rotor can reach while it turns: inside the cylinder about
        // the axis that the bounds sweep (radius of the farthest corner)
        const float lo[3] = {R.xMin, R.yMin, R.zMin}, hi[3] = {R.xMax, R.yMax, R.zMax};
        const float org[3] = {R.ox, R.oy, R.oz};
        const int a = R.axis, p1 = (a + 1) % 3, p2 = (a + 2) % 3;
        double r2max = 0.0;
        for (int u = 0; u < 2; ++u)
            for (int v = 0; v < 2; ++v) {
                const double d1 = (u ? hi[p1] : lo[p1]) - org[p1], d2 = (v ? hi[p2] : lo[p2]) - org[p2];
                r2max = std::max(r2max, d1 * d1 + d2 * d2);
            }
        const double margin = 0.01 * L.info.res;
        const double rmax = std::sqrt(r2max) + margin;
        for (int q = 0; q < L.info.cellCount; ++q) {
            const double pos[3] = {L.I[q] * L.info.res + L.info.ox, L.J[q] * L.info.res + L.info.oy,
                                   L.K[q] * L.info.res + L.info.oz};
            if (pos[a] < lo[a] - margin || pos[a] > hi[a] + margin) continue;
            const double d1 = pos[p1] - org[p1], d2 = pos[p2] - org[p2];
            if (d1 * d1 + d2 * d2 <= rmax * rmax) L.rotorCell[q] = 1;
        }
        L.rotors.push_back(std::move(R));
    }
}

void buildSegments(HostLevel& L) {
    L.segCell.clear(); L.segJP.clear(); L.segKP.clear(); L.segJKP.clear(); L.segLen.clear();
    L.specialCells.clear();
    L.rotorCells.clear();
    const int n = L.info.cellCount;
    int c = 0;
    while (c < n) {
        // extent of the compressed row starting at c
        int end = c + 1;
        while (end < n && L.shifter[end] < 0) ++end;
        int row = L.shifter[c];
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
            return (L.wallMap[q] == -1 || L.wallMap[q] == -2) && !wraps(q) &&
                   (L.rotorCell.empty() || !L.rotorCell[q]);
        };
        for (int q = c; q < end;) {
            if (L.wallMap[q] == -3) { ++q; continue; }
            if (!L.rotorCell.empty() && L.rotorCell[q]) { L.rotorCells.push_back(q); ++q; continue; }
            if (!bulk(q)) { L.specialCells.push_back(q); ++q; continue; }
            int r = q;
            while (r < end && r - q < kSegmentCells && bulk(r)) ++r;
            const int off = q - c;
            // A run that reaches the end of its row continues into the next
            // rows while their neighbour rows continue the same arithmetic
            // progression (a dense block of full rows): the +1 neighbour is
            // index + 1 everywhere, so the lane offsets stay valid and short
            // rows still fill whole tiles.
            int rowEnd = end, rowStart = c, rowId = row;
            static const bool rowSegments = std::getenv("LBM3_ROW_SEGMENTS") != nullptr;  // tuning: one row per segment
            while (!rowSegments && r == rowEnd && r - q < kSegmentCells && rowEnd < n) {
                const int next = L.shifter[rowEnd];
                const int len = rowEnd - rowStart;
                if (next < 0 || L.rowJP[next] != L.rowJP[rowId] + len || L.rowKP[next] != L.rowKP[rowId] + len ||
                    L.rowJKP[next] != L.rowJKP[rowId] + len)
                    break;
                int nextEnd = rowEnd + 1;
                while (nextEnd < n && L.shifter[nextEnd] < 0) ++nextEnd;
                const int nextStart = rowEnd;
                auto bulkIn = [&L, n, next, nextStart](int x) {
                    const int o = x - nextStart;
                    const bool w = x + 1 >= n || L.rowJP[next] + o + 1 >= n || L.rowKP[next] + o + 1 >= n ||
                                   L.rowJKP[next] + o + 1 >= n;
                    return (L.wallMap[x] == -1 || L.wallMap[x] == -2) && !w &&
                           (L.rotorCell.empty() || !L.rotorCell[x]);
                };
                if (!bulkIn(rowEnd)) break;
                rowStart = rowEnd;
                rowId = next;
                rowEnd = nextEnd;
                while (r < rowEnd && r - q < kSegmentCells && bulkIn(r)) ++r;
            }
            L.segCell.push_back(q);
            L.segJP.push_back(jP(off));
            L.segKP.push_back(kP(off));
            L.segJKP.push_back(jkP(off));
            L.segLen.push_back(r - q);
            if (r > end) {
                // the run ended inside a later row: carry on from there
                c = rowStart;
                end = rowEnd;
                row = rowId;
            }
            q = r;
        }
        c = end;
    }
}

namespace {

size_t denseIndex(const Info& in, int i, int j, int k) {
    return (static_cast<size_t>(k) * in.ny + j) * in.nx + i;
}

// initializeGridInfo for a finer level (include/gridBuilderFunctions.h:50-62):
// half the spacing, twice the cells per axis, origin shifted by half a fine
// cell, half the time step.
void initFinerInfo(const lbm_case& c, const Info& coarse, Info& fine, int level) {
    fine.gridID = level;
    fine.res = coarse.res * 0.5f;
    fine.nx = coarse.nx * 2;
    fine.ny = coarse.ny * 2;
    fine.nz = coarse.nz * 2;
    fine.ox = coarse.ox - fine.res * 0.5f;
    fine.oy = coarse.oy - fine.res * 0.5f;
    fine.oz = coarse.oz - fine.res * 0.5f;
    fine.dtPhys = coarse.dtPhys * 0.5f;
    fine.nu = (fine.dtPhys * c.nu_phys) / ((fine.res / 1000.f) * (fine.res / 1000.f));
}

// Keep the marked cells of a level (deleteExcessCells steps 7-13): the cell
// list is re-emitted in k-j-i order with fresh neighbours; returns the new
// index of every old cell (-1 when deleted).
std::vector<int> compactLevel(HostLevel& L, const std::vector<uint8_t>& keepCell) {
    const Info& in = L.info;
    std::vector<uint8_t> dense(static_cast<size_t>(in.nx) * in.ny * in.nz, 0);
    std::vector<int> remap(keepCell.size(), -1);
    int n = 0;
    for (size_t q = 0; q < keepCell.size(); ++q)
        if (keepCell[q]) {
            dense[denseIndex(in, L.I[q], L.J[q], L.K[q])] = 1;
            remap[q] = n++;
        }
    buildCellsAndNBR(L, dense);
    return remap;
}

template <class T>
std::vector<T> remapCells(const std::vector<T>& v, const std::vector<int>& remap, int n) {
    std::vector<T> out(n);
    if (v.empty()) return {};
    for (size_t q = 0; q < remap.size(); ++q)
        if (remap[q] >= 0) out[remap[q]] = v[q];
    return out;
}

std::vector<uint8_t> andNot(std::vector<uint8_t> a, const std::vector<uint8_t>& b) {
    for (size_t q = 0; q < a.size(); ++q) a[q] = a[q] && !b[q];
    return a;
}

// markRefinementCells (include/markerFunctions.h:419-450) on a level with a
// finer one: keep marks (cells that cover fluid on any finer level, spread
// once, plus the parent interface), deep refinement (cells that cover a wall
// on any finer level, spread WALL_REFINEMENT_COUNT times, then the user
// modification), the fine-to-coarse ring (one layer) and the coarse-to-fine
// band (two layers) around it.
void markRefinement(const lbm_case& c, const HostLevel& L, LevelMarks& M, const std::vector<RayMap>& total) {
    const Info& in = L.info;
    const int n = in.cellCount, lv = in.gridID, NL = c.grid_level_count;
    std::vector<uint8_t> keep(n, 0), deep(n, 0);
    for (int q = 0; q < n; ++q) {
        bool fluid = false, wall = false;
        for (int m = lv; m < NL; ++m) {
            const int down = 1 << (m - lv);
            fluid = fluid || coarseHasFluid(total[m], down, L.I[q], L.J[q], L.K[q]);
            wall = wall || coarseHasWall(total[m], down, L.I[q], L.J[q], L.K[q]);
        }
        keep[q] = fluid;
        deep[q] = wall;
    }
    keep = spreadCells(L, keep);
    if (lv > 0)
        for (int q = 0; q < n; ++q) keep[q] = keep[q] || M.parentInterface[q];
    for (int r = 0; r < c.wall_refinement_count; ++r) deep = spreadCells(L, deep);
    // applyUserRefinementModification (:254-271): the refinement box of this
    // level, then the driver's hook
    const float* box = c.refine_box[lv];
    const bool useBox = box[0] < box[3] && box[1] < box[4] && box[2] < box[5];
    lbm_grid_info hi = hookInfo(in);
    hi.cell_count = n;
    for (int q = 0; q < n; ++q) {
        int mark = deep[q];
        if (useBox) {
            const float x = L.I[q] * in.res + in.ox, y = L.J[q] * in.res + in.oy, z = L.K[q] * in.res + in.oz;
            if (x > box[0] && x < box[3] && y > box[1] && y < box[4] && z > box[2] && z < box[5]) mark = 1;
        }
        if (c.refinement_hook) c.refinement_hook(c.hook_user, L.I[q], L.J[q], L.K[q], &mark, &hi);
        deep[q] = mark != 0;
    }
    if (lv > 0) deep = andNot(deep, M.parentInterface);
    for (int q = 0; q < n; ++q) deep[q] = deep[q] && keep[q];
    std::vector<uint8_t> f2c = spreadCells(L, deep);
    for (int q = 0; q < n; ++q) f2c[q] = f2c[q] && keep[q] && !deep[q];
    std::vector<uint8_t> c2f = spreadCells(L, spreadCells(L, f2c));
    for (int q = 0; q < n; ++q) c2f[q] = c2f[q] && keep[q] && !deep[q] && !f2c[q];
    M.refine.assign(n, 0);
    for (int q = 0; q < n; ++q) M.refine[q] = deep[q] || f2c[q] || c2f[q];
    M.deep = std::move(deep);
    M.f2c = std::move(f2c);
    M.c2f = std::move(c2f);
}

// buildFinerGridBuilder (include/gridBuilderFunctions.h:134-201) + sortIJK:
// the 2x2x2 children of every refinement-marked coarse cell, emitted in k-j-i
// order; then the parent map and the parent-interface marks (buildIJKFull
// steps 6-7).
void buildFinerLevel(const HostLevel& C, const LevelMarks& CM, HostLevel& F, LevelMarks& FM) {
    const Info& fin = F.info;
    std::vector<uint8_t> dense(static_cast<size_t>(fin.nx) * fin.ny * fin.nz, 0);
    for (int q = 0; q < C.info.cellCount; ++q) {
        if (!CM.refine[q]) continue;
        for (int a = 0; a < 2; ++a)
            for (int b = 0; b < 2; ++b)
                for (int e = 0; e < 2; ++e)
                    dense[denseIndex(fin, 2 * C.I[q] + e, 2 * C.J[q] + b, 2 * C.K[q] + a)] = 1;
    }
    buildCellsAndNBR(F, dense);
    const int n = F.info.cellCount;
    FM.parent.assign(n, -1);
    FM.parentInterface.assign(n, 0);
    FM.parentF2C.assign(n, 0);
    for (int q = 0; q < n; ++q) {
        const int p = findCell(C, F.I[q] / 2, F.J[q] / 2, F.K[q] / 2);
        FM.parent[q] = p;
        if (p < 0) continue;
        FM.parentInterface[q] = CM.c2f[p] || CM.f2c[p];
        FM.parentF2C[q] = CM.f2c[p];
    }
}

// deleteExcessCells (include/gridBuilderFunctions.h:402-588) for one level,
// after its coarser level has been compacted.
void deleteExcess(const lbm_case& c, HostLevel& L, LevelMarks& M, const HostLevel* coarse, const RayMap& total) {
    const int NL = c.grid_level_count;
    const int lv = L.info.gridID;
    const int n = L.info.cellCount;
    if (coarse) {
        for (int q = 0; q < n; ++q) {
            M.parent[q] = findCell(*coarse, L.I[q] / 2, L.J[q] / 2, L.K[q] / 2);
            M.parentInterface[q] = M.parent[q] >= 0;
        }
    }
    std::vector<uint8_t> keep(n, 0);
    for (int q = 0; q < n; ++q) keep[q] = !isSolid(total, L.I[q], L.J[q], L.K[q]);
    if (coarse)
        for (int q = 0; q < n; ++q) keep[q] = keep[q] || M.parentInterface[q];
    keep = spreadCells(L, keep);
    if (lv < NL - 1) keep = andNot(keep, M.deep);
    if (coarse) {
        // the outermost layer of the parent interface goes: the coarse-to-fine
        // blocks reach the fine cells between coarse centres only
        const std::vector<uint8_t> s1 = spreadCells(L, M.parentF2C);
        const std::vector<uint8_t> s3 = spreadCells(L, spreadCells(L, s1));
        for (int q = 0; q < n; ++q)
            if (M.parentInterface[q] && !s3[q]) keep[q] = 0;
        M.needValues.assign(n, 0);
        for (int q = 0; q < n; ++q) M.needValues[q] = M.parentInterface[q] && keep[q] && !s1[q];
    }
    const std::vector<int> remap = compactLevel(L, keep);
    const int m = L.info.cellCount;
    if (coarse) {
        M.parent = remapCells(M.parent, remap, m);
        M.needValues = remapCells(M.needValues, remap, m);
        M.parentInterface = remapCells(M.parentInterface, remap, m);
        M.parentF2C = remapCells(M.parentF2C, remap, m);
    }
    if (lv < NL - 1) {
        M.f2c = remapCells(M.f2c, remap, m);
        M.c2f = remapCells(M.c2f, remap, m);
    }
    M.deep.clear();
    M.refine.clear();
}

// The 8 plus neighbours of a builder cell in the order self, +i, +j, +ij, +k,
// +ik, +jk, +ijk (finishNBRPlus, include/NBRFunctions.h:5-11).
void blockNbrs(const HostLevel& L, int c, int (&nb)[8]) {
    const int n = L.info.cellCount;
    auto wrap = [n](int v) { return v + 1 < n ? v + 1 : 0; };
    nb[0] = c;
    nb[1] = wrap(c);
    nb[2] = L.jPlus[c];
    nb[3] = wrap(nb[2]);
    nb[4] = L.kPlus[c];
    nb[5] = wrap(nb[4]);
    nb[6] = L.jPlus[nb[4]];
    nb[7] = wrap(nb[6]);
}

// Interface lists of a coarse level towards the next finer one
// (gridBuilderToGrid step 6, include/gridBuilderFunctions.h:1192-1231, with
// fillFineToCoarseInterface :741-769 and fillCoarseToFineInterface :771-1030).
void buildInterfaces(HostLevel& C, const LevelMarks& CM, const HostLevel& F, const LevelMarks& FM) {
    const int nc = C.info.cellCount, nf = F.info.cellCount;
    // childMapArrayGlobal: the (2i,2j,2k) child of every coarse cell
    std::vector<int> child(nc, -1);
    for (int q = 0; q < nf; ++q) {
        const int p = FM.parent[q];
        if (p >= 0 && F.I[q] % 2 == 0 && F.J[q] % 2 == 0 && F.K[q] % 2 == 0) child[p] = q;
    }
    C.f2cIndex.clear(); C.f2cChild.clear();
    for (int q = 0; q < nc; ++q)
        if (CM.f2c[q] && !C.wallMarker[q]) {
            C.f2cIndex.push_back(q);
            C.f2cChild.push_back(child[q]);
        }
    // coarse-to-fine: full 2x2x2 coarse stencils whose centre block of fine
    // cells exists in full
    std::vector<uint8_t> mark(nc, 0);
    for (int q = 0; q < nc; ++q) mark[q] = CM.c2f[q] && !C.wallMarker[q];
    C.c2fIndex.clear(); C.c2fChild.clear();
    std::vector<uint8_t> received(nf, 0);
    for (int q = 0; q < nc; ++q) {
        if (!mark[q]) continue;
        int nb[8];
        blockNbrs(C, q, nb);
        bool ok = true;
        for (int t = 1; t < 8 && ok; ++t) {
            const int r = nb[t];
            ok = mark[r] && C.I[r] == C.I[q] + (t & 1) && C.J[r] == C.J[q] + ((t >> 1) & 1) &&
                 C.K[r] == C.K[q] + ((t >> 2) & 1);
        }
        if (!ok) continue;
        const int top = child[nb[7]];
        if (top < 0) continue;
        // walk back from the top child: jkPlus = top - 1, kPlus = jMinus,
        // self = kMinus
        int jk = top - 1;
        if (jk < 0) jk = nf - 1;
        const int kp = F.jMinus[jk];
        const int self = F.kMinus[kp];
        int fb[8];
        blockNbrs(F, self, fb);
        for (int t = 0; t < 8 && ok; ++t) {
            const int r = fb[t];
            ok = F.I[r] == 2 * C.I[q] + 1 + (t & 1) && F.J[r] == 2 * C.J[q] + 1 + ((t >> 1) & 1) &&
                 F.K[r] == 2 * C.K[q] + 1 + ((t >> 2) & 1);
        }
        if (!ok) continue;
        C.c2fIndex.push_back(q);
        C.c2fChild.push_back(self);
        for (int t = 0; t < 8; ++t) received[fb[t]] = 1;
    }
    // leftovers: fine cells that need coarse values and no block reached
    C.leftIndex.clear(); C.leftParent.clear();
    std::vector<int> nbI, nbJ, nbK;
    for (int q = 0; q < nf; ++q) {
        if (!(FM.needValues[q] && !F.wallMarker[q] && !received[q])) continue;
        const int p = FM.parent[q];
        const int ic = C.I[p], jc = C.J[p], kc = C.K[p];
        auto at = [&](int r, int di, int dj, int dk) {
            return mark[r] && C.I[r] == ic + di && C.J[r] == jc + dj && C.K[r] == kc + dk;
        };
        auto pick = [&](bool plusFirst, int plusCell, int minusCell, int di, int dj, int dk) {
            const int first = plusFirst ? plusCell : minusCell, second = plusFirst ? minusCell : plusCell;
            const int s = plusFirst ? 1 : -1;
            if (at(first, s * di, s * dj, s * dk)) return first;
            if (at(second, -s * di, -s * dj, -s * dk)) return -second - 1;
            return p;
        };
        const int iPlus = p + 1 >= nc ? 0 : p + 1, iMinus = p - 1 < 0 ? nc - 1 : p - 1;
        nbI.push_back(pick(F.I[q] % 2 == 1, iPlus, iMinus, 1, 0, 0));
        nbJ.push_back(pick(F.J[q] % 2 == 1, C.jPlus[p], C.jMinus[p], 0, 1, 0));
        nbK.push_back(pick(F.K[q] % 2 == 1, C.kPlus[p], C.kMinus[p], 0, 0, 1));
        C.leftIndex.push_back(q);
        C.leftParent.push_back(p);
    }
    C.leftNbr.clear();
    C.leftNbr.insert(C.leftNbr.end(), nbI.begin(), nbI.end());
    C.leftNbr.insert(C.leftNbr.end(), nbJ.begin(), nbJ.end());
    C.leftNbr.insert(C.leftNbr.end(), nbK.begin(), nbK.end());
}

}  // namespace

void buildDomain(const lbm_case& c, HostDomain& out) {
    validateCase(c);
    out.c = c;
    out.c.body_count = 0;  // triangle pointers and hooks are not kept past this call
    out.c.open_bc_hook = nullptr;
    out.c.initial_condition_hook = nullptr;
    out.c.local_bc_hook = nullptr;
    out.c.refinement_hook = nullptr;
    out.c.hook_user = nullptr;
    for (int r = 0; r < LBM_MAX_ROTORS; ++r) out.c.rotor[r].triangles = nullptr;
    const int NL = c.grid_level_count;
    out.levels.assign(NL, HostLevel{});
    Info skel;
    initLevel0(c, out.levels[0].info, skel);
    for (int l = 1; l < NL; ++l) initFinerInfo(c, out.levels[l - 1].info, out.levels[l].info, l);

    // bodies: triangles and bins once, a ray map per body and level plus
    // their union (readSTL/sortSTLToBins, initializeVoxelizers:
    // voxelizerFunctions.h:692-728)
    std::vector<Triangles> bodies(c.body_count);
    for (int b = 0; b < c.body_count; ++b) {
        loadTriangles(c.body[b].triangles, c.body[b].triangle_count, bodies[b]);
        sortToBins(bodies[b], c.res_global);
    }
    std::vector<std::vector<RayMap>> maps(NL, std::vector<RayMap>(c.body_count));
    std::vector<RayMap> total(NL);
    for (int l = 0; l < NL; ++l) {
        const Info& in = out.levels[l].info;
        total[l].nx = in.nx;
        total[l].ny = in.ny;
        total[l].scan.assign(static_cast<size_t>(in.nx) * in.ny + 1, 0);
        for (int b = 0; b < c.body_count; ++b) {
            voxelize(bodies[b], in.ox, in.oy, in.oz, in.res, in.nx, in.ny, maps[l][b]);
            if (b == 0) total[l] = maps[l][0];
            else unionRayMaps(total[l], maps[l][b]);
        }
    }

    // buildIJKFull (include/gridBuilderFunctions.h:299-400).  Level 0 from the
    // skeleton: a skeleton cell is kept when it covers fluid on any level,
    // plus one layer (markKeepCells, markerFunctions.h:401-409), and
    // contributes its 2x2x2 children.
    std::vector<LevelMarks> marks(NL);
    {
        HostLevel& L0 = out.levels[0];
        const Info& in = L0.info;
        const int snx = skel.nx, sny = skel.ny, snz = skel.nz;
        std::vector<uint8_t> keepSkel(static_cast<size_t>(snx) * sny * snz, 1);
        if (c.body_count > 0) {
            for (int k = 0; k < snz; ++k)
                for (int j = 0; j < sny; ++j)
                    for (int i = 0; i < snx; ++i) {
                        bool fluid = false;
                        for (int m = 0; m < NL && !fluid; ++m) fluid = coarseHasFluid(total[m], 2 << m, i, j, k);
                        keepSkel[(static_cast<size_t>(k) * sny + j) * snx + i] = fluid ? 1 : 0;
                    }
            keepSkel = spreadDense(keepSkel, snx, sny, snz);
        }
        std::vector<uint8_t> keep(static_cast<size_t>(in.nx) * in.ny * in.nz, 0);
        for (int k = 0; k < in.nz; ++k)
            for (int j = 0; j < in.ny; ++j)
                for (int i = 0; i < in.nx; ++i)
                    keep[denseIndex(in, i, j, k)] = keepSkel[(static_cast<size_t>(k / 2) * sny + j / 2) * snx + i / 2];
        buildCellsAndNBR(L0, keep);
    }
    // finer levels: refinement marks on the coarser level, then its children
    for (int l = 0; l + 1 < NL; ++l) {
        markRefinement(c, out.levels[l], marks[l], total);
        buildFinerLevel(out.levels[l], marks[l], out.levels[l + 1], marks[l + 1]);
    }
    // deleteExcessCells, coarse to fine
    for (int l = 0; l < NL; ++l)
        deleteExcess(c, out.levels[l], marks[l], l > 0 ? &out.levels[l - 1] : nullptr, total[l]);

    // buildWallMarkers (include/gridBuilderFunctions.h:590-739), coarse to fine
    for (int l = 0; l < NL; ++l) {
        HostLevel& L = out.levels[l];
        LevelMarks& M = marks[l];
        const int n = L.info.cellCount;
        // interface overlap (step 7): this level's fine-to-coarse cells and
        // the cells under the parent's coarse-to-fine band
        L.interfaceOverlap.assign(n, 0);
        std::vector<uint8_t> iface;
        if (NL > 1) {
            iface.assign(n, 0);
            for (int q = 0; q < n; ++q) {
                bool ov = false, in = false;
                if (l + 1 < NL) {
                    ov = M.f2c[q];
                    in = M.f2c[q] || M.c2f[q];
                }
                if (l > 0 && M.parent[q] >= 0) {
                    in = true;
                    if (marks[l - 1].c2f[M.parent[q]]) ov = true;
                }
                L.interfaceOverlap[q] = ov;
                iface[q] = in;
            }
        }
        if (c.body_count > 0) {
            buildWalls(c, L, M, l > 0 ? &out.levels[l - 1] : nullptr, l > 0 ? &marks[l - 1] : nullptr, bodies,
                       maps[l], total[l], l > 0 ? &maps[l - 1] : nullptr, iface);
        } else {
            L.wallMarker.assign(n, 0);
            M.wallIDFull.assign(n, -1);
            L.wallIndex.clear();
            L.wallData.clear();
            L.linkLength.clear();
            L.wallVelocity.clear();
        }
    }

    // gridBuilderToGrid (include/gridBuilderFunctions.h:1032-1564) per level
    for (int l = 0; l < NL; ++l) {
        HostLevel& L = out.levels[l];
        compressRows(L);
        buildBoundaryLists(c, L);
        if (l + 1 < NL) buildInterfaces(L, marks[l], out.levels[l + 1], marks[l + 1]);
        buildRotors(c, L);
        buildSegments(L);
    }

    out.fluidUpdatesPerIteration = 0;
    for (const HostLevel& lv : out.levels)
        out.fluidUpdatesPerIteration +=
            static_cast<long long>(lv.info.cellCount - lv.wallCellCount) *
            (1LL << lv.info.gridID);
}

}  // namespace lbm
