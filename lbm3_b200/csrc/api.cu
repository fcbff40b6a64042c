// C ABI (include/lbm3_b200.h): owns device memory of every level, runs the
// per-step schedule of updateAllGrids on one CUDA stream, and converts every
// failure into a status code plus a thread-local message.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <functional>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/lbm3_b200.h"
#include "builder.h"
#include "energy_noalloc.h"
#include "mbbc.h"
#include "step_launch.h"

namespace {

thread_local std::string gLastError;

int fail(int code, const std::string& msg) {
    gLastError = msg;
    return code;
}

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

template <class T> T* devAlloc(size_t n) {
    if (n == 0) return nullptr;
    void* p = nullptr;
    const cudaError_t e = cudaMalloc(&p, n * sizeof(T));
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        throw std::bad_alloc();
    }
    return static_cast<T*>(p);
}

template <class T> T* upload(const std::vector<T>& v, cudaStream_t s) {
    T* p = devAlloc<T>(v.size());
    if (p) ck(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s), "upload");
    return p;
}

size_t storageBytes(int storage) {
    return storage == LBM_STORE_F64 ? 8 : storage == LBM_STORE_F32 ? 4 : 2;
}

// bytes of one direction-indexed closure table in the kernels' arithmetic type
size_t mbbcTableBytes(int storage) {
    return storage == LBM_STORE_F64 ? sizeof(lbm::MbbcDirT<double>) : sizeof(lbm::MbbcDirT<float>);
}

// Distance between consecutive population planes, in elements.  Planes start
// on 128-byte boundaries and are an odd number of 128-byte granules apart, so
// the 27 read and 27 write streams of a step do not all map onto the same
// DRAM channels when the cell count is a power of two.  LBM3_PLANE_PAD_LINES
// adds further 128-byte granules (tuning).
long long planeStride(long long n, int storage) {
    const long long perLine = 128 / static_cast<long long>(storageBytes(storage));
    long long lines = (n + perLine - 1) / perLine;
    if (lines % 2 == 0) ++lines;
    if (const char* e = std::getenv("LBM3_PLANE_PAD_LINES")) lines += std::atoll(e);
    return lines * perLine;
}

}  // namespace

struct LevelState {
    lbm::Info info;
    int iterationsSinceTrackerReset = 0;
    int rowCount = 0;
    int wallCellCount = 0;
    int wallAdjacentCount = 0;
    int openBCCount = 0;
    std::vector<int> openTrackCount;   // trackFlowCount per openBCID
    int* obSource = nullptr;           // openBCs[id].sourceArray, concatenated (ID order)
    std::vector<int> obPerm;           // kernel position -> ID-order index of open cells
    std::vector<lbm::HostRotor> rotors;  // host copies: info, tables (device copies in dev.rotor)
    std::vector<int*> rotorIndex;        // device indexArray per rotor
    unsigned long long memBytes = 0;
    lbm::DevLevel dev{};
    // interface to the next finer level (empty on the finest): device lists
    // and host copies for readback
    lbm::DevInterface itf{};
    std::vector<int> f2cIndex, f2cChild, c2fIndex, c2fChild, leftIndex, leftParent, leftNbr;
    std::vector<void*> owned;
};

struct lbm_grids {
    lbm_case c{};
    std::vector<LevelState> levels;
    cudaStream_t stream = nullptr;
    // CUDA graphs of two consecutive steps, one per starting esotwist parity,
    // replayed by lbm_update_all_grids / lbm_update_batch (domains without
    // rotors: their per-step frame is host state); captured on captureStream
    bool graphsEnabled = true;
    cudaStream_t captureStream = nullptr;
    cudaGraphExec_t pairExec[2] = {nullptr, nullptr};
    // per level with a finer one: a side stream on which the level's own
    // update runs while the finer levels' substeps run on the grid stream
    // (they touch disjoint state until the interface joins them)
    std::vector<cudaStream_t> sideStreams;
    std::vector<cudaEvent_t> forkEvents, joinEvents;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double* scratch = nullptr;
    int* errorFlag = nullptr;  // device word the kernels set when a bounded wait gives up
    float lastKernelMs = 0.f;
    int lastLaunches = 0;
    long long lastStepKernels = 0;  // every kernel launch of the last lbm_time_steps
    // event pairs bracketing collide-stream launches while lbm_time_steps runs
    std::vector<cudaEvent_t> kernelEvents;
    bool timingKernels = false;
    int kernelEventsUsed = 0;

    ~lbm_grids() {
        for (cudaEvent_t e : kernelEvents) cudaEventDestroy(e);
        for (auto& L : levels)
            for (void* p : L.owned) cudaFree(p);
        if (scratch) cudaFree(scratch);
        if (errorFlag) cudaFree(errorFlag);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        for (cudaGraphExec_t e : pairExec)
            if (e) cudaGraphExecDestroy(e);
        if (captureStream) cudaStreamDestroy(captureStream);
        // levels without a finer one have no side stream (null entries): a
        // destroy of a null handle would leave an error for the next check
        for (cudaStream_t t : sideStreams)
            if (t) cudaStreamDestroy(t);
        for (cudaEvent_t e : forkEvents)
            if (e) cudaEventDestroy(e);
        for (cudaEvent_t e : joinEvents)
            if (e) cudaEventDestroy(e);
    }
};

struct lbm_plan {
    lbm::HostDomain host;
};

namespace {

// Open-boundary chunks of the boundary kernel: cells grouped by outer normal
// (table row), kOpenChunk per CTA.
size_t openChunkCount(const lbm::HostLevel& H) {
    std::vector<size_t> perRow(LBM_MBBC_NORMALS, 0);
    for (const auto& oc : H.openCells) ++perRow[(oc.info >> 10) & 31];
    size_t chunks = 0;
    for (size_t c : perRow) chunks += (c + lbm::kOpenChunk - 1) / lbm::kOpenChunk;
    return chunks;
}

// Device bytes of one level: every array lbm_build_grids allocates for it,
// with the same size expressions (the reference prints a similar per-level
// account, gridBuilderFunctions.h:1630-1649).  The domain-wide words (FP64
// reduction scratch, error flag) are counted with level 0.
unsigned long long levelBytes(const lbm::HostLevel& H, int storage) {
    using ull = unsigned long long;
    auto bytes = [](size_t count, size_t each) { return static_cast<ull>(count) * each; };
    const size_t n = static_cast<size_t>(H.info.cellCount);
    ull b = 27ULL * planeStride(static_cast<long long>(n), storage) * storageBytes(storage) + 256;  // populations
    b += bytes(2, sizeof(int));                                     // work counter
    b += bytes(1, sizeof(lbm::DevLevel));                           // device copy of the descriptor
    if (storage == LBM_STORE_F16 || storage == LBM_STORE_BF16)
        b += bytes(2, sizeof(unsigned));                            // stochastic-rounding seeds
    b += bytes(n, sizeof(int)) * 2;                                 // shifter, wallMap
    b += bytes(H.rowI.size(), sizeof(int)) * 6;                     // compressed rows
    b += bytes(H.perIndex.size(), sizeof(int)) * 2;                 // periodic index, source
    b += bytes(H.segCell.size(), sizeof(int4)) + bytes(H.segLen.size(), sizeof(int));  // bulk segments
    b += bytes(H.specialCells.size(), sizeof(int)) + bytes(H.rotorCells.size(), sizeof(int));
    for (const auto& R : H.rotors)
        b += bytes(R.rotorMap.size(), sizeof(int)) + bytes(R.interpolation.size(), sizeof(unsigned)) +
             bytes(R.index.size(), sizeof(int)) + bytes(3 * 27 * R.index.size(), sizeof(float));
    b += bytes(H.wallIndex.size(), sizeof(int)) + bytes(H.wallData.size(), sizeof(unsigned)) +
         bytes(H.linkLength.size(), sizeof(unsigned)) + bytes(H.wallVelocity.size(), sizeof(float)) +
         bytes(3 * H.wallIndex.size(), sizeof(double));            // wall tables and FP64 force accumulators
    const size_t m = H.openCells.size();
    size_t sources = 0;
    for (const auto& ob : H.openBCs) sources += ob.source.size();
    b += bytes(m, sizeof(int)) * 2 + bytes(m, sizeof(int4)) + bytes(m, sizeof(float4)) + bytes(m, sizeof(float)) +
         bytes(sources, sizeof(int)) + bytes(4 * m, sizeof(float));  // cell, info, nbr, target, beta, source, refs
    b += bytes(openChunkCount(H), sizeof(int4)) + (m ? bytes(LBM_MBBC_NORMALS, mbbcTableBytes(storage)) : 0);
    b += m ? bytes(2, sizeof(int)) : 0;                             // device iteration counter
    b += bytes(H.f2cIndex.size() + H.f2cChild.size() + H.c2fIndex.size() + H.c2fChild.size(), sizeof(int));
    b += bytes(H.leftIndex.size() + H.leftParent.size() + H.leftNbr.size(), sizeof(int));  // interface lists
    if (H.info.gridID == 0) b += bytes(8, sizeof(double)) + bytes(1, sizeof(int));
    return b;
}

void fillInfo(const lbm::HostLevel& H, int storage, lbm_grid_info* out) {
    std::memset(out, 0, sizeof(*out));
    out->grid_id = H.info.gridID;
    out->cell_count = H.info.cellCount;
    out->cell_count_x = H.info.nx;
    out->cell_count_y = H.info.ny;
    out->cell_count_z = H.info.nz;
    out->row_count = static_cast<int>(H.rowI.size());
    out->wall_cell_count = H.wallCellCount;
    out->wall_adjacent_count = H.wallAdjacentCount;
    out->periodic_count = static_cast<int>(H.perIndex.size());
    int ob = 0;
    for (const auto& o : H.openBCs) ob += static_cast<int>(o.index.size());
    out->open_bc_count = ob;
    out->esotwist_flipper = H.info.esotwistFlipper ? 1 : 0;
    out->iterations_finished = H.info.iterationsFinished;
    out->storage = storage;
    out->res = H.info.res;
    out->ox = H.info.ox;
    out->oy = H.info.oy;
    out->oz = H.info.oz;
    out->nu = H.info.nu;
    out->dt_phys = H.info.dtPhys;
    out->grid_memory_bytes = levelBytes(H, storage);
    out->f2c_count = static_cast<int>(H.f2cIndex.size());
    out->c2f_count = static_cast<int>(H.c2fIndex.size());
    out->leftover_count = static_cast<int>(H.leftIndex.size());
}

}  // namespace

namespace {

// updateSingleGrid (include/updateGrid.h:16-386): K1, flip, open boundary,
// periodic copy.
// Advance every rotor's angle by one step (include/updateGrid.h:36-49) and
// hand its cosine and sine to the kernels.
void advanceRotors(LevelState& L) {
    constexpr double twoPi = 6.283185307179586476925286766559;
    for (size_t r = 0; r < L.rotors.size(); ++r) {
        lbm::HostRotor& R = L.rotors[r];
        R.radiansElapsed = std::fmod(R.radiansElapsed + static_cast<double>(L.info.dtPhys) * R.radiansPerSecond, twoPi);
        if (R.radiansElapsed < 0.0) R.radiansElapsed += twoPi;
        if (R.radiansElapsed >= twoPi) R.radiansElapsed = 0.0;
        const float angle = static_cast<float>(R.radiansElapsed);
        L.dev.rotor[r].c = std::cos(angle);
        L.dev.rotor[r].s = std::sin(angle);
        L.dev.rotor[r].scale = R.radiansPerSecond * L.info.dtPhys / L.info.res;
    }
}

void updateSingleGrid(lbm_grids* g, LevelState& L, cudaStream_t stream) {
    if (!L.rotors.empty()) advanceRotors(L);
    const bool flip = L.info.esotwistFlipper;
    if (g->timingKernels) {
        const size_t k = static_cast<size_t>(g->kernelEventsUsed);
        ck(cudaEventRecord(g->kernelEvents[k], stream), "event");
        lbm::launchCollideStream(L.dev, flip, stream);
        ck(cudaEventRecord(g->kernelEvents[k + 1], stream), "event");
        g->kernelEventsUsed += 2;
    } else {
        lbm::launchCollideStream(L.dev, flip, stream);
    }
    L.info.esotwistFlipper = !flip;  // applyStreaming
    lbm::launchOpenBoundary(L.dev, L.info.esotwistFlipper, stream);
    lbm::launchPeriodic(L.dev, L.info.esotwistFlipper, stream);
    L.info.iterationsFinished++;
    L.iterationsSinceTrackerReset++;
}

// Host bookkeeping of one step whose kernels ran inside a replayed graph.
void advanceHostState(LevelState& L) {
    L.info.esotwistFlipper = !L.info.esotwistFlipper;
    L.info.iterationsFinished++;
    L.iterationsSinceTrackerReset++;
}

// updateAllGrids (include/updateGrid.h:388-396): a level steps once, the
// next finer level twice (recursively), then the interface between them.
// The level's own update and the finer substeps read and write disjoint
// state (the interface of the previous coarse step is their only link), so
// the level's update runs on a side stream forked from the grid stream and
// joined before the interface; kernel timing keeps everything on one stream.
void updateAllGrids(lbm_grids* g, int level) {
    const bool finer = level + 1 < static_cast<int>(g->levels.size());
    if (!finer) {
        updateSingleGrid(g, g->levels[level], g->stream);
        return;
    }
    const bool fork = !g->timingKernels;
    if (fork) {
        if (g->sideStreams.size() < g->levels.size()) {
            g->sideStreams.resize(g->levels.size(), nullptr);
            g->forkEvents.resize(g->levels.size(), nullptr);
            g->joinEvents.resize(g->levels.size(), nullptr);
        }
        if (!g->sideStreams[level]) {
            ck(cudaStreamCreateWithFlags(&g->sideStreams[level], cudaStreamNonBlocking), "side stream");
            ck(cudaEventCreateWithFlags(&g->forkEvents[level], cudaEventDisableTiming), "fork event");
            ck(cudaEventCreateWithFlags(&g->joinEvents[level], cudaEventDisableTiming), "join event");
        }
        cudaStream_t side = g->sideStreams[level];
        ck(cudaEventRecord(g->forkEvents[level], g->stream), "fork");
        ck(cudaStreamWaitEvent(side, g->forkEvents[level], 0), "fork wait");
        updateSingleGrid(g, g->levels[level], side);
        ck(cudaEventRecord(g->joinEvents[level], side), "join");
    } else {
        updateSingleGrid(g, g->levels[level], g->stream);
    }
    for (int i = 0; i < 2; ++i) updateAllGrids(g, level + 1);
    if (fork) ck(cudaStreamWaitEvent(g->stream, g->joinEvents[level], 0), "join wait");
    LevelState& C = g->levels[level];
    LevelState& F = g->levels[level + 1];
    lbm::launchInterface(C.dev, F.dev, C.itf, C.info.esotwistFlipper, F.info.esotwistFlipper, g->stream);
}

// Host bookkeeping of one coarse step whose kernels ran inside a replayed
// graph: level L advances 2^L substeps.
void advanceHostStep(lbm_grids* g) {
    for (LevelState& L : g->levels)
        for (int k = 0; k < (1 << L.info.gridID); ++k) advanceHostState(L);
}

// Graph replay applies when no level has rotors (their frame is advanced
// on the host every step) and LBM3_GRAPHS is not "0".
bool graphable(const lbm_grids* g) {
    static const bool env = [] {
        const char* e = std::getenv("LBM3_GRAPHS");
        return !(e && std::string(e) == "0");
    }();
    if (!env || !g->graphsEnabled) return false;
    for (const LevelState& L : g->levels)
        if (!L.rotors.empty()) return false;
    return true;
}

// The instantiated graph of two steps starting at esotwist parity `parity`
// (captured on first use; kernel arguments are fixed per grids object).
cudaGraphExec_t pairGraph(lbm_grids* g, int parity) {
    if (g->pairExec[parity]) return g->pairExec[parity];
    if (!g->captureStream) ck(cudaStreamCreateWithFlags(&g->captureStream, cudaStreamNonBlocking), "stream");
    // capture changes no host state: save and restore the step bookkeeping
    std::vector<lbm::Info> saved;
    std::vector<int> savedReset;
    for (LevelState& L : g->levels) {
        saved.push_back(L.info);
        savedReset.push_back(L.iterationsSinceTrackerReset);
    }
    g->levels[0].info.esotwistFlipper = parity != 0;
    cudaStream_t user = g->stream;
    g->stream = g->captureStream;
    cudaGraph_t graph = nullptr;
    ck(cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    try {
        updateAllGrids(g, 0);
        updateAllGrids(g, 0);
    } catch (...) {
        cudaStreamEndCapture(g->stream, &graph);
        if (graph) cudaGraphDestroy(graph);
        g->stream = user;
        for (size_t l = 0; l < g->levels.size(); ++l) {
            g->levels[l].info = saved[l];
            g->levels[l].iterationsSinceTrackerReset = savedReset[l];
        }
        throw;
    }
    const cudaError_t e = cudaStreamEndCapture(g->stream, &graph);
    g->stream = user;
    for (size_t l = 0; l < g->levels.size(); ++l) {
        g->levels[l].info = saved[l];
        g->levels[l].iterationsSinceTrackerReset = savedReset[l];
    }
    ck(e, "end capture");
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    ck(ei, "graph instantiate");
    g->pairExec[parity] = exec;
    return exec;
}

// Launch two steps of a grids object from its graph, on its stream.
void launchPair(lbm_grids* g) {
    const int parity = g->levels[0].info.esotwistFlipper ? 1 : 0;
    cudaGraphExec_t exec = pairGraph(g, parity);
    ck(cudaGraphLaunch(exec, g->stream), "graph launch");
    for (int k = 0; k < 2; ++k) advanceHostStep(g);
}

struct DeviceWaitError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// After the stream is idle: report (and clear) a bounded device wait that gave up.
void checkDeviceFlag(lbm_grids* g) {
    int flag = 0;
    ck(cudaMemcpyAsync(&flag, g->errorFlag, sizeof(int), cudaMemcpyDeviceToHost, g->stream), "flag copy");
    ck(cudaStreamSynchronize(g->stream), "flag sync");
    if (flag) {
        ck(cudaMemsetAsync(g->errorFlag, 0, sizeof(int), g->stream), "flag reset");
        ck(cudaStreamSynchronize(g->stream), "flag sync");
        throw DeviceWaitError("a bounded device wait in the collide-stream kernel gave up");
    }
}

int guarded(const char* where, const std::function<void()>& body) {
    try {
        body();
        gLastError.clear();
        return LBM_OK;
    } catch (const CudaError& e) {
        return fail(LBM_ERR_CUDA, std::string(where) + ": " + e.what());
    } catch (const DeviceWaitError& e) {
        return fail(LBM_ERR_DEVICE_WAIT, std::string(where) + ": " + e.what());
    } catch (const std::bad_alloc&) {
        return fail(LBM_ERR_OOM, std::string(where) + ": device or host allocation failed");
    } catch (const std::invalid_argument& e) {
        return fail(LBM_ERR_INVALID, std::string(where) + ": " + e.what());
    } catch (const std::runtime_error& e) {
        return fail(LBM_ERR_BUILD, std::string(where) + ": " + e.what());
    } catch (const std::exception& e) {
        return fail(LBM_ERR_INVALID, std::string(where) + ": " + e.what());
    }
}
}  // namespace

// ---- packed batch --------------------------------------------------------------

struct lbm_batch {
    std::vector<lbm_grids*> members;
    int storage = LBM_STORE_F32;
    lbm::DevBatch dev{};
    lbm_batch_info info{};
    std::vector<void*> owned;
    cudaStream_t stream = nullptr;         // the batch's launches
    cudaStream_t captureStream = nullptr;  // graph capture
    cudaEvent_t sync = nullptr;            // orders the batch after / before its members
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaGraphExec_t pairExec[2] = {nullptr, nullptr};
    ~lbm_batch() {
        for (cudaGraphExec_t e : pairExec)
            if (e) cudaGraphExecDestroy(e);
        if (stream) cudaStreamSynchronize(stream);
        for (void* p : owned) cudaFree(p);
        if (sync) cudaEventDestroy(sync);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (captureStream) cudaStreamDestroy(captureStream);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

void batchStep(lbm_batch* b, bool flip, cudaStream_t s) { lbm::launchPackedStep(b->dev, b->storage, flip, s); }

// Graph of two packed steps starting at esotwist parity `parity`.
cudaGraphExec_t batchPairGraph(lbm_batch* b, int parity) {
    if (b->pairExec[parity]) return b->pairExec[parity];
    cudaGraph_t graph = nullptr;
    ck(cudaStreamBeginCapture(b->captureStream, cudaStreamCaptureModeThreadLocal), "begin capture");
    batchStep(b, parity != 0, b->captureStream);
    batchStep(b, parity == 0, b->captureStream);
    const cudaError_t e = cudaStreamEndCapture(b->captureStream, &graph);
    ck(e, "end capture");
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    ck(ei, "graph instantiate");
    b->pairExec[parity] = exec;
    return exec;
}

// Advance `steps` packed steps on the batch stream (members already waited for).
void batchAdvance(lbm_batch* b, int steps) {
    bool flip = b->members[0]->levels[0].info.esotwistFlipper;
    int s = 0;
    if (graphable(b->members[0]))
        for (; s + 2 <= steps; s += 2) ck(cudaGraphLaunch(batchPairGraph(b, flip ? 1 : 0), b->stream), "graph launch");
    for (; s < steps; ++s) {
        batchStep(b, flip, b->stream);
        flip = !flip;
    }
    ck(cudaGetLastError(), "batch launch");
    for (lbm_grids* g : b->members)
        for (int k = 0; k < steps; ++k) advanceHostState(g->levels[0]);
}

void batchCheckParity(const lbm_batch* b) {
    const bool flip = b->members[0]->levels[0].info.esotwistFlipper;
    for (const lbm_grids* g : b->members)
        if (g->levels[0].info.esotwistFlipper != flip)
            throw std::invalid_argument(
                "members are at different esotwist parities (step the odd ones once on their own)");
}

}  // namespace

namespace {

// Flow report of a domain with several levels (getFlowReportGeneral,
// include/flowReportFunctions.h:11-352): a section image at the finest level
// whose pixel count fits FLOW_REPORT_PIXEL_LIMIT, filled level by level (a
// finer level overwrites a coarser one; a coarser level's cut between two
// layers blends them), then summed over its fluid pixels.
int flowReportLevels(lbm_grids* g, int plane, float cut, const float* bounds, double* out) {
    constexpr long long kPixelLimit = 16000000;  // FLOW_REPORT_PIXEL_LIMIT
    const int levels = static_cast<int>(g->levels.size());
    const lbm::Info& fin = g->levels[levels - 1].info;
    const int n[3] = {fin.nx, fin.ny, fin.nz};
    const float o[3] = {fin.ox, fin.oy, fin.oz};
    const int axis = plane == LBM_PLANE_XY ? 2 : plane == LBM_PLANE_ZY ? 0 : 1;
    // getIJKCellIndexFromXYZ on the finest level (include/flowReportFunctions.h:355-372)
    const int cutIndex = static_cast<int>((cut - o[axis]) / fin.res + 0.5f);
    if (cutIndex < 0 || cutIndex >= n[axis]) return fail(LBM_ERR_INVALID, "lbm_flow_report: cut outside the grid");
    const double cutPosition = double(o[axis]) + double(cutIndex) * fin.res;
    int lo[3] = {0, 0, 0}, hi[3] = {n[0], n[1], n[2]};
    if (bounds && (bounds[0] != 0.f || bounds[1] != 0.f || bounds[2] != 0.f || bounds[3] != 0.f ||
                   bounds[4] != 0.f || bounds[5] != 0.f))
        for (int a = 0; a < 3; ++a) {
            const float tMin = o[a] - 0.5f * fin.res;
            const float tMax = o[a] + fin.res * (n[a] - 0.5f);
            lo[a] = std::max(0, static_cast<int>(std::ceil((bounds[a] - tMin) / fin.res)));
            hi[a] = std::min(n[a], n[a] - static_cast<int>(std::ceil((tMax - bounds[a + 3]) / fin.res)));
        }
    const int hAxis = plane == LBM_PLANE_XY ? 0 : 2, vAxis = plane == LBM_PLANE_ZX ? 0 : 1;
    int pixelsH = hi[hAxis] - lo[hAxis], pixelsV = hi[vAxis] - lo[vAxis];
    int startH = lo[hAxis], startV = lo[vAxis];
    int imageLevel = levels - 1;
    long long pixels = (long long)pixelsH * pixelsV;
    while (pixels > kPixelLimit && imageLevel > 0) {
        --imageLevel;
        pixelsH /= 2; startH /= 2;
        pixelsV /= 2; startV /= 2;
        pixels = (long long)pixelsH * pixelsV;
    }
    if (pixelsH <= 0 || pixelsV <= 0 || pixels > kPixelLimit)
        return fail(LBM_ERR_INVALID, "lbm_flow_report: empty crop or image above the pixel limit");
    return guarded("lbm_flow_report", [&] {
        float* img = devAlloc<float>(3 * size_t(pixels));
        struct Free { float* p; ~Free() { cudaFree(p); } } keep{img};
        lbm::launchFlowImageClear(img, pixels, g->stream);
        for (int l = 0; l < levels; ++l) {
            LevelState& L = g->levels[l];
            const lbm::Info& in = L.info;
            const int count = plane == LBM_PLANE_XY ? in.nz : plane == LBM_PLANE_ZY ? in.nx : in.ny;
            if (in.cellCount <= 0 || count <= 0) continue;
            const double origin = plane == LBM_PLANE_XY ? in.oz : plane == LBM_PLANE_ZY ? in.ox : in.oy;
            const double index = std::clamp((cutPosition - origin) / double(in.res), 0.0, double(count - 1));
            lbm::FlowImagePass a{};
            a.plane = plane;
            a.lowerNormal = static_cast<int>(std::floor(index));
            a.alpha = static_cast<float>(index - a.lowerNormal);
            a.interpolate = a.alpha > 0.f;
            a.downsample = l > imageLevel ? 1 << (l - imageLevel) : 1;
            a.upsample = l < imageLevel ? 1 << (imageLevel - l) : 1;
            a.startH = startH;
            a.startV = startV;
            a.pixelsH = pixelsH;
            a.pixelsV = pixelsV;
            lbm::launchFlowImage(L.dev, in.esotwistFlipper, g->stream, a, img);
        }
        ck(cudaMemsetAsync(g->scratch, 0, 6 * sizeof(double), g->stream), "memset");
        lbm::launchFlowImageSum(img, pixels, g->stream, g->scratch);
        ck(cudaGetLastError(), "flow report launch");
        double t[6];
        ck(cudaMemcpyAsync(t, g->scratch, sizeof(t), cudaMemcpyDeviceToHost, g->stream), "copy");
        ck(cudaStreamSynchronize(g->stream), "sync");
        for (int q = 0; q < 7; ++q) out[q] = 0.0;
        if (t[5] == 0.0) return;
        // unit conversion with the pixel size of the image level
        // (include/flowReportFunctions.h:322-351)
        const lbm::Info& in = g->levels[imageLevel].info;
        const double px = double(in.res) / 1000.0, area = px * px, vs = px / double(in.dtPhys);
        const double ps = double(g->c.rho_phys) * vs * vs / 3.0;
        const double mfs = double(g->c.rho_phys) * area * vs;
        out[0] = t[0] / t[5] * vs;
        out[1] = (t[0] + t[1]) * mfs;
        out[2] = t[2] * mfs * vs;
        out[3] = t[3] / t[5] * ps;
        out[4] = t[1] * area * ps * vs;
        out[5] = t[4] * mfs * vs * vs;
        out[6] = t[5] * double(in.res) * in.res;
    });
}

}  // namespace

extern "C" {

const char* lbm_last_error(void) { return gLastError.c_str(); }

int lbm_device_count(void) {
    int n = 0;
    const cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return 0;
        return fail(LBM_ERR_CUDA, cudaGetErrorString(e));
    }
    return n;
}

int lbm_plan_grids(const lbm_case* c, lbm_plan** out, long long* fluidUpdates) {
    if (!c || !out) return fail(LBM_ERR_INVALID, "lbm_plan_grids: null argument");
    *out = nullptr;
    lbm_plan* p = new lbm_plan();
    const int rc = guarded("lbm_plan_grids", [&] {
        lbm::buildDomain(*c, p->host);
        if (fluidUpdates) *fluidUpdates = p->host.fluidUpdatesPerIteration;
    });
    if (rc != LBM_OK) {
        delete p;
        return rc;
    }
    *out = p;
    return LBM_OK;
}

void lbm_free_plan(lbm_plan* p) { delete p; }

int lbm_plan_level_count(lbm_plan* p) {
    if (!p) return fail(LBM_ERR_INVALID, "lbm_plan_level_count: null plan");
    return static_cast<int>(p->host.levels.size());
}

int lbm_plan_info(lbm_plan* p, int level, lbm_grid_info* out) {
    if (!p || !out || level < 0 || level >= (int)p->host.levels.size())
        return fail(LBM_ERR_INVALID, "lbm_plan_info: bad argument");
    fillInfo(p->host.levels[level], p->host.c.storage, out);
    return LBM_OK;
}

int lbm_plan_read_array(lbm_plan* p, int level, int which, void* host, size_t bytes) {
    if (!p || !host || level < 0 || level >= (int)p->host.levels.size())
        return fail(LBM_ERR_INVALID, "lbm_plan_read_array: bad argument");
    const lbm::HostLevel& H = p->host.levels[level];
    const std::vector<int>* v = nullptr;
    const std::vector<uint32_t>* u = nullptr;
    std::vector<int> openIndex, openSource;
    for (const auto& ob : H.openBCs) {
        openIndex.insert(openIndex.end(), ob.index.begin(), ob.index.end());
        openSource.insert(openSource.end(), ob.source.begin(), ob.source.end());
    }
    if (which >= LBM_ARRAY_ROTOR_BASE) {
        const int r = (which - LBM_ARRAY_ROTOR_BASE) / 4, part = (which - LBM_ARRAY_ROTOR_BASE) % 4;
        if (r >= (int)H.rotors.size() || part == 3)
            return fail(LBM_ERR_INVALID, "lbm_plan_read_array: no such rotor table in a plan");
        const lbm::HostRotor& R = H.rotors[r];
        const void* src = part == 0 ? (const void*)R.rotorMap.data() : part == 1 ? (const void*)R.index.data()
                                                                                 : (const void*)R.interpolation.data();
        const size_t need = 4 * (part == 0 ? R.rotorMap.size() : part == 1 ? R.index.size() : R.interpolation.size());
        if (bytes != need) return fail(LBM_ERR_INVALID, "lbm_plan_read_array: byte count does not match array size");
        if (bytes) std::memcpy(host, src, bytes);
        return LBM_OK;
    }
    {
        const std::vector<int>* lists[7] = {&H.f2cIndex, &H.f2cChild, &H.c2fIndex, &H.c2fChild,
                                            &H.leftIndex, &H.leftParent, &H.leftNbr};
        if (which >= LBM_ARRAY_F2C_INDEX && which <= LBM_ARRAY_LEFTOVER_NBR) {
            const std::vector<int>& v = *lists[which - LBM_ARRAY_F2C_INDEX];
            if (bytes != v.size() * sizeof(int))
                return fail(LBM_ERR_INVALID, "lbm_plan_read_array: byte count does not match array size");
            if (bytes) std::memcpy(host, v.data(), bytes);
            return LBM_OK;
        }
    }
    if (which == LBM_ARRAY_WALL_VELOCITY) {
        const size_t need = H.wallVelocity.size() * sizeof(float);
        if (bytes != need) return fail(LBM_ERR_INVALID, "lbm_plan_read_array: byte count does not match array size");
        if (bytes) std::memcpy(host, H.wallVelocity.data(), bytes);
        return LBM_OK;
    }
    switch (which) {
        case LBM_ARRAY_SHIFTER: v = &H.shifter; break;
        case LBM_ARRAY_ROW_I: v = &H.rowI; break;
        case LBM_ARRAY_ROW_J: v = &H.rowJ; break;
        case LBM_ARRAY_ROW_K: v = &H.rowK; break;
        case LBM_ARRAY_ROW_JPLUS: v = &H.rowJP; break;
        case LBM_ARRAY_ROW_KPLUS: v = &H.rowKP; break;
        case LBM_ARRAY_ROW_JKPLUS: v = &H.rowJKP; break;
        case LBM_ARRAY_WALL_MAP: v = &H.wallMap; break;
        case LBM_ARRAY_PERIODIC_INDEX: v = &H.perIndex; break;
        case LBM_ARRAY_PERIODIC_SOURCE: v = &H.perSource; break;
        case LBM_ARRAY_WALL_INDEX: v = &H.wallIndex; break;
        case LBM_ARRAY_OPEN_INDEX: v = &openIndex; break;
        case LBM_ARRAY_OPEN_SOURCE: v = &openSource; break;
        case LBM_ARRAY_WALL_DATA: u = &H.wallData; break;
        case LBM_ARRAY_LINK_LENGTH: u = &H.linkLength; break;
        default: return fail(LBM_ERR_INVALID, "lbm_plan_read_array: array not available in a plan");
    }
    if (u) {
        if (bytes != u->size() * sizeof(uint32_t))
            return fail(LBM_ERR_INVALID, "lbm_plan_read_array: byte count does not match array size (expected " +
                                             std::to_string(u->size() * sizeof(uint32_t)) + ")");
        if (bytes) std::memcpy(host, u->data(), bytes);
        return LBM_OK;
    }
    if (bytes != v->size() * sizeof(int))
        return fail(LBM_ERR_INVALID, "lbm_plan_read_array: byte count does not match array size (expected " +
                                         std::to_string(v->size() * sizeof(int)) + ")");
    if (bytes) std::memcpy(host, v->data(), bytes);
    return LBM_OK;
}

void lbm_default_bc(lbm_bc* bc) {
    if (!bc) return;
    const lbm::BC d;
    bc->dRho = d.dRho; bc->ux = d.ux; bc->uy = d.uy; bc->uz = d.uz;
    bc->gx = d.gx; bc->gy = d.gy; bc->gz = d.gz;
    bc->wallID = d.wallID; bc->openBCID = d.openBCID;
    bc->useIBB = d.useIBB; bc->dirichletU = d.dirichletU; bc->dirichletRho = d.dirichletRho;
    bc->periodic = d.periodic; bc->nonReflective = d.nonReflective;
    bc->nonReflectiveBeta = d.nonReflectiveBeta; bc->collisionLimiter = d.collisionLimiter;
    bc->nuMultiplier = d.nuMultiplier;
}

int lbm_build_grids(const lbm_case* c, lbm_grids** out, long long* fluidUpdates) {
    if (!c || !out) return fail(LBM_ERR_INVALID, "lbm_build_grids: null argument");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        (void)cudaGetLastError();
        return fail(LBM_ERR_NO_DEVICE, "lbm_build_grids: no CUDA device visible");
    }
    lbm_grids* g = new lbm_grids();
    const int rc = guarded("lbm_build_grids", [&] {
        g->c = *c;
        lbm::HostDomain host;
        lbm::buildDomain(*c, host);
        ck(cudaEventCreate(&g->ev0), "cudaEventCreate");
        ck(cudaEventCreate(&g->ev1), "cudaEventCreate");
        g->scratch = devAlloc<double>(8);
        g->errorFlag = devAlloc<int>(1);
        cudaStream_t s = g->stream;
        ck(cudaMemsetAsync(g->errorFlag, 0, sizeof(int), s), "memset");
        g->levels.resize(host.levels.size());
        for (size_t l = 0; l < host.levels.size(); ++l) {
            const lbm::HostLevel& H = host.levels[l];
            LevelState& L = g->levels[l];
            L.info = H.info;
            L.rowCount = static_cast<int>(H.rowI.size());
            L.wallCellCount = H.wallCellCount;
            L.wallAdjacentCount = H.wallAdjacentCount;
            L.openBCCount = 0;
            for (const auto& ob : H.openBCs) {
                L.openBCCount += static_cast<int>(ob.index.size());
                L.openTrackCount.push_back(ob.trackFlowCount);
            }
            const long long n = H.info.cellCount;
            lbm::DevLevel& d = L.dev;
            d.cellCount = H.info.cellCount;
            d.stride = planeStride(n, c->storage);
            d.storage = c->storage;
            d.nx = H.info.nx; d.ny = H.info.ny; d.nz = H.info.nz;
            d.res = H.info.res; d.ox = H.info.ox; d.oy = H.info.oy; d.oz = H.info.oz;
            auto own = [&](auto* p) { if (p) L.owned.push_back(p); return p; };
            // 256 bytes of tail so bulk copies rounded up to 16 bytes stay inside
            d.f = own(devAlloc<unsigned char>(27ULL * d.stride * storageBytes(c->storage) + 256));
            d.errorFlag = g->errorFlag;
            d.work = own(devAlloc<int>(2));
            ck(cudaMemsetAsync(d.work, 0, 2 * sizeof(int), s), "memset");
            d.seed = nullptr;
            if (c->storage == LBM_STORE_F16 || c->storage == LBM_STORE_BF16) {
                // the two parities' first step seeds, distinct per level
                const std::vector<unsigned> seeds = {0x243F6A88u + 0x9E3779B9u * unsigned(l),
                                                     0x85A308D3u + 0x7F4A7C15u * unsigned(l)};
                d.seed = own(upload(seeds, s));
            }
            d.shifter = own(upload(H.shifter, s));
            d.rowI = own(upload(H.rowI, s));
            d.rowJ = own(upload(H.rowJ, s));
            d.rowK = own(upload(H.rowK, s));
            d.rowJP = own(upload(H.rowJP, s));
            d.rowKP = own(upload(H.rowKP, s));
            d.rowJKP = own(upload(H.rowJKP, s));
            d.wallMap = own(upload(H.wallMap, s));
            d.perIndex = own(upload(H.perIndex, s));
            d.perSource = own(upload(H.perSource, s));
            d.perCount = static_cast<int>(H.perIndex.size());
            {
                std::vector<int4> seg(H.segCell.size());
                for (size_t q = 0; q < seg.size(); ++q)
                    seg[q] = make_int4(H.segCell[q], H.segJP[q], H.segKP[q], H.segJKP[q]);
                d.seg = own(upload(seg, s));
                d.segLen = own(upload(H.segLen, s));
                d.segCount = static_cast<int>(seg.size());
                d.special = own(upload(H.specialCells, s));
                d.specialCount = static_cast<int>(H.specialCells.size());
                d.rotorCells = own(upload(H.rotorCells, s));
                d.rotorCellCount = static_cast<int>(H.rotorCells.size());
            }
            {
                // rotors: tables, force bins, and the per-step frame in dev.rotor
                L.rotors = H.rotors;
                d.rotorCount = static_cast<int>(H.rotors.size());
                d.trackRotorForce = c->track_rotor_force ? 1 : 0;
                for (size_t r = 0; r < H.rotors.size(); ++r) {
                    const lbm::HostRotor& R = H.rotors[r];
                    lbm::DevRotor& D = d.rotor[r];
                    D.rotorMap = own(upload(R.rotorMap, s));
                    D.interp = own(upload(R.interpolation, s));
                    D.nonzero = static_cast<int>(R.index.size());
                    D.force = own(devAlloc<float>(3 * 27 * R.index.size()));
                    if (D.force) ck(cudaMemsetAsync(D.force, 0, 3 * 27 * R.index.size() * sizeof(float), s), "memset");
                    L.rotorIndex.push_back(own(upload(R.index, s)));
                    D.cntX = R.cntX; D.cntY = R.cntY; D.cntZ = R.cntZ; D.axis = R.axis;
                    D.res = R.res;
                    D.xMin = R.xMin; D.yMin = R.yMin; D.zMin = R.zMin;
                    D.xMax = R.xMax; D.yMax = R.yMax; D.zMax = R.zMax;
                    D.ox = R.ox; D.oy = R.oy; D.oz = R.oz;
                    D.c = 1.f; D.s = 0.f;
                    D.scale = R.radiansPerSecond * H.info.dtPhys / H.info.res;
                }
            }
            d.wallCount = static_cast<int>(H.wallIndex.size());
            d.wallIndex = own(upload(H.wallIndex, s));
            d.wallData = own(upload(H.wallData, s));
            d.linkLength = own(upload(H.linkLength, s));
            d.wallVel = own(upload(H.wallVelocity, s));
            d.wallForce = own(devAlloc<double>(3 * H.wallIndex.size()));
            if (d.wallForce) ck(cudaMemsetAsync(d.wallForce, 0, 3 * H.wallIndex.size() * sizeof(double), s), "memset");
            {
                // open boundaries.  The device keeps the per-cell records in
                // kernel order: cells grouped by outer normal (table row) into
                // CTA-sized chunks, each group in ID order.  obPerm maps a
                // kernel position back to the ID order the ABI reports.
                const size_t m = H.openCells.size();
                std::vector<lbm::MbbcDir> tables(LBM_MBBC_NORMALS);
                for (int t = 0; t < LBM_MBBC_NORMALS; ++t) tables[t] = lbm::mbbcDirFromTable(kLbmMbbc[t]);
                std::vector<int> order;
                std::vector<int4> chunks;
                order.reserve(m);
                for (int row = 0; row < LBM_MBBC_NORMALS; ++row) {
                    const int first = static_cast<int>(order.size());
                    for (size_t q = 0; q < m; ++q)
                        if (((H.openCells[q].info >> 10) & 31) == row) order.push_back(static_cast<int>(q));
                    const int count = static_cast<int>(order.size()) - first;
                    for (int c0 = 0; c0 < count; c0 += lbm::kOpenChunk)
                        chunks.push_back(make_int4(first + c0, std::min(lbm::kOpenChunk, count - c0), row,
                                                   static_cast<int>(tables[row].unknownMask)));
                }
                std::vector<int> cell(m), info(m), source;
                std::vector<int4> nbr(m);
                std::vector<float4> target(m);
                std::vector<float> beta(m);
                for (size_t p = 0; p < m; ++p) {
                    const lbm::OpenBCCell& oc = H.openCells[order[p]];
                    cell[p] = oc.cell;
                    const int jp = H.jPlus[oc.cell], kp = H.kPlus[oc.cell];
                    nbr[p] = make_int4(oc.cell, jp, kp, H.jPlus[kp]);
                    info[p] = oc.info;
                    target[p] = make_float4(oc.dRho, oc.ux, oc.uy, oc.uz);
                    beta[p] = oc.beta;
                }
                for (const auto& ob : H.openBCs) source.insert(source.end(), ob.source.begin(), ob.source.end());
                L.obPerm = order;
                d.obCount = static_cast<int>(m);
                d.obCell = own(upload(cell, s));
                d.obNbr = own(upload(nbr, s));
                d.obInfo = own(upload(info, s));
                d.obTarget = own(upload(target, s));
                d.obBeta = own(upload(beta, s));
                L.obSource = own(upload(source, s));
                d.obRhoRef = own(devAlloc<float>(2 * m));
                d.obUnRef = d.obRhoRef ? d.obRhoRef + m : nullptr;
                d.obRhoCum = own(devAlloc<float>(2 * m));
                d.obUnCum = d.obRhoCum ? d.obRhoCum + m : nullptr;
                if (m) ck(cudaMemsetAsync(d.obRhoCum, 0, 2 * m * sizeof(float), s), "memset");
                d.trackOpen = c->track_open_boundaries ? 1 : 0;
                d.obImpedance = c->open_bc_scheme == LBM_OPEN_IMPEDANCE ? 1 : 0;
                d.obTolerance = c->rho_reflection_tolerance;
                d.obChunk = own(upload(chunks, s));
                d.obCounter = m ? own(devAlloc<int>(2)) : nullptr;
                if (m) ck(cudaMemsetAsync(d.obCounter, 0, 2 * sizeof(int), s), "memset");
                d.obChunkCount = static_cast<int>(chunks.size());
                if (m && c->storage == LBM_STORE_F64) {
                    std::vector<lbm::MbbcDirT<double>> wide(LBM_MBBC_NORMALS);
                    for (int t = 0; t < LBM_MBBC_NORMALS; ++t) wide[t] = lbm::mbbcDirFromTable<double>(kLbmMbbc[t]);
                    d.obTables = own(upload(wide, s));
                } else {
                    d.obTables = m ? own(upload(tables, s)) : nullptr;
                }
            }
            d.trackWallForce = c->track_wall_force ? 1 : 0;
            const lbm::BC bc = lbm::levelLocalBC(*c, H);
            d.useIBB = bc.useIBB ? 1 : 0;
            d.gx = bc.gx;
            d.gy = bc.gy;
            d.gz = bc.gz;
            d.coll = lbm::makeCollisionConsts(H.info.nu, bc.nuMultiplier, bc.collisionLimiter);
            d.coll64 = lbm::makeCollisionConstsT<double>(H.info.nu, bc.nuMultiplier, bc.collisionLimiter);
            // memory accounting as the reference prints it (gridBuilderFunctions.h:1630-1649),
            // scaled by the population storage size
            L.memBytes = levelBytes(H, c->storage);

            // initial condition: macroscopic fields from the host (exactly the
            // getInitialCondition hook), equilibrium populations on the device
            float4 uni = make_float4(c->ic_dRho, c->ic_ux, c->ic_uy, c->ic_uz);
            float4* dm = nullptr;
            if (c->ic_kind != LBM_IC_UNIFORM || c->initial_condition_hook) {
                std::vector<float4> macro(n);
                for (long long q = 0; q < n; ++q) {
                    const lbm::BC ic = lbm::evalInitialCondition(*c, H.info, H.I[q], H.J[q], H.K[q]);
                    macro[q] = make_float4(ic.dRho, ic.ux, ic.uy, ic.uz);
                }
                dm = upload(macro, s);
                lbm::launchInit(d, L.info.esotwistFlipper, s, dm, uni);
                ck(cudaStreamSynchronize(s), "init");
                cudaFree(dm);
            } else {
                lbm::launchInit(d, L.info.esotwistFlipper, s, nullptr, uni);
            }
            // reference values of the open boundary from the initial state
            lbm::launchOpenBoundaryInit(d, L.info.esotwistFlipper, s);
            ck(cudaGetLastError(), "init launch");
        }
        // interface lists between consecutive levels (owned by the coarse level)
        for (size_t l = 0; l + 1 < host.levels.size(); ++l) {
            const lbm::HostLevel& H = host.levels[l];
            LevelState& L = g->levels[l];
            auto own = [&](auto* p) { if (p) L.owned.push_back(p); return p; };
            L.f2cIndex = H.f2cIndex; L.f2cChild = H.f2cChild;
            L.c2fIndex = H.c2fIndex; L.c2fChild = H.c2fChild;
            L.leftIndex = H.leftIndex; L.leftParent = H.leftParent; L.leftNbr = H.leftNbr;
            lbm::DevInterface& I = L.itf;
            I.f2cIndex = own(upload(H.f2cIndex, s));
            I.f2cChild = own(upload(H.f2cChild, s));
            I.f2cCount = static_cast<int>(H.f2cIndex.size());
            I.c2fIndex = own(upload(H.c2fIndex, s));
            I.c2fChild = own(upload(H.c2fChild, s));
            I.c2fCount = static_cast<int>(H.c2fIndex.size());
            I.leftIndex = own(upload(H.leftIndex, s));
            I.leftParent = own(upload(H.leftParent, s));
            I.leftNbr = own(upload(H.leftNbr, s));
            I.leftCount = static_cast<int>(H.leftIndex.size());
            // omega1 = 1 / (3 nu + 1/2) of each level, in the arithmetic type
            auto omega = [&](float nu) {
                return c->storage == LBM_STORE_F64 ? 1.0 / (3.0 * static_cast<double>(nu) + 0.5)
                                                   : static_cast<double>(1.f / (3.f * nu + 0.5f));
            };
            I.omegaCoarse = omega(H.info.nu);
            I.omegaFine = omega(host.levels[l + 1].info.nu);
        }
        // each level's descriptor on the device, for the collide-stream launch
        // that reads it there (the fields it uses do not change after the build)
        for (LevelState& L : g->levels) {
            lbm::DevLevel* self = devAlloc<lbm::DevLevel>(1);
            L.owned.push_back(self);
            L.dev.self = self;
            ck(cudaMemcpyAsync(self, &L.dev, sizeof(lbm::DevLevel), cudaMemcpyHostToDevice, s), "descriptor copy");
        }
        ck(cudaStreamSynchronize(s), "build sync");
        if (fluidUpdates) *fluidUpdates = host.fluidUpdatesPerIteration;
        // the driver's hooks are evaluated during the build only
        g->c.open_bc_hook = nullptr;
        g->c.initial_condition_hook = nullptr;
        g->c.local_bc_hook = nullptr;
        g->c.hook_user = nullptr;
    });
    if (rc != LBM_OK) {
        delete g;
        return rc;
    }
    *out = g;
    return LBM_OK;
}

void lbm_free_grids(lbm_grids* g) {
    if (!g) return;
    cudaStreamSynchronize(g->stream);
    delete g;
}

int lbm_set_stream(lbm_grids* g, void* stream) {
    if (!g) return fail(LBM_ERR_INVALID, "lbm_set_stream: null grids");
    g->stream = static_cast<cudaStream_t>(stream);
    return LBM_OK;
}

int lbm_update_all_grids(lbm_grids* g, int steps) {
    if (!g || steps < 0) return fail(LBM_ERR_INVALID, "lbm_update_all_grids: bad argument");
    return guarded("lbm_update_all_grids", [&] {
        int s = 0;
        if (graphable(g))
            for (; s + 2 <= steps; s += 2) launchPair(g);
        for (; s < steps; ++s) updateAllGrids(g, 0);
        ck(cudaGetLastError(), "step launch");
    });
}

int lbm_update_batch(lbm_grids* const* grids, int count, int steps) {
    if (!grids || count < 0 || steps < 0) return fail(LBM_ERR_INVALID, "lbm_update_batch: bad argument");
    for (int q = 0; q < count; ++q)
        if (!grids[q]) return fail(LBM_ERR_INVALID, "lbm_update_batch: null grids in the batch");
    return guarded("lbm_update_batch", [&] {
        // step pairs from each domain's graph, interleaved across domains;
        // domains without graphs (rotors) and a trailing odd step launch directly
        int s = 0;
        for (; s + 2 <= steps; s += 2)
            for (int q = 0; q < count; ++q) {
                if (graphable(grids[q])) {
                    launchPair(grids[q]);
                } else {
                    updateAllGrids(grids[q], 0);
                    updateAllGrids(grids[q], 0);
                }
            }
        for (; s < steps; ++s)
            for (int q = 0; q < count; ++q) updateAllGrids(grids[q], 0);
        ck(cudaGetLastError(), "step launch");
    });
}

int lbm_batch_create(lbm_grids* const* grids, int count, lbm_batch** out) {
    if (!grids || count <= 0 || !out) return fail(LBM_ERR_INVALID, "lbm_batch_create: bad argument");
    *out = nullptr;
    for (int q = 0; q < count; ++q) {
        if (!grids[q]) return fail(LBM_ERR_INVALID, "lbm_batch_create: null grids in the batch");
        for (int r = 0; r < q; ++r)
            if (grids[r] == grids[q]) return fail(LBM_ERR_INVALID, "lbm_batch_create: a domain is listed twice");
    }
    lbm_batch* b = new lbm_batch();
    const int rc = guarded("lbm_batch_create", [&] {
        b->members.assign(grids, grids + count);
        b->storage = grids[0]->c.storage;
        for (lbm_grids* g : b->members) {
            if (g->levels.size() != 1) throw std::invalid_argument("a packed batch holds single-level domains");
            const LevelState& L = g->levels[0];
            if (!L.rotors.empty()) throw std::invalid_argument("a packed batch holds domains without rotors");
            if (g->c.storage != b->storage) throw std::invalid_argument("members have different storage types");
            if (b->storage == LBM_STORE_F64) throw std::invalid_argument("FP64 domains are not packed");
            if (!lbm::pairFits(L.dev)) throw std::invalid_argument("a member is too large for 32-bit offsets");
        }
        // packed tables: every member's items, member by member
        std::vector<lbm::DevLevel> levels;
        std::vector<int2> open;
        std::vector<int> itemStart{0};
        std::vector<int> perStart{0};
        long long cells = 0;
        for (int q = 0; q < count; ++q) {
            const lbm::DevLevel& d = b->members[q]->levels[0].dev;
            levels.push_back(d);
            const int items = d.segCount + (d.specialCount + 127) / 128;
            itemStart.push_back(itemStart.back() + items);
            for (int i = 0; i < d.obChunkCount; ++i) open.push_back(make_int2(q, i));
            perStart.push_back(perStart.back() + d.perCount);
            cells += d.cellCount;
        }
        ck(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "stream");
        ck(cudaStreamCreateWithFlags(&b->captureStream, cudaStreamNonBlocking), "stream");
        ck(cudaEventCreateWithFlags(&b->sync, cudaEventDisableTiming), "event");
        ck(cudaEventCreate(&b->ev0), "event");
        ck(cudaEventCreate(&b->ev1), "event");
        auto own = [&](auto* p) { if (p) b->owned.push_back(p); return p; };
        lbm::DevBatch& D = b->dev;
        D.levels = own(upload(levels, b->stream));
        D.domainCount = count;
        D.itemStart = own(upload(itemStart, b->stream));
        D.collideCount = itemStart.back();
        D.work = own(devAlloc<int>(count + 1));
        ck(cudaMemsetAsync(D.work, 0, (count + 1) * sizeof(int), b->stream), "memset");
        D.openItems = open.empty() ? nullptr : own(upload(open, b->stream));
        D.openCount = static_cast<int>(open.size());
        D.periodicStart = own(upload(perStart, b->stream));
        D.periodicCount = perStart.back();
        ck(cudaStreamSynchronize(b->stream), "batch upload");
        b->info.domain_count = count;
        b->info.cells = cells;
        b->info.collide_items = D.collideCount;
        b->info.open_chunks = D.openCount;
        b->info.periodic_cells = D.periodicCount;
        b->info.launches_per_step = (D.collideCount > 0) + (D.openCount > 0) + (D.periodicCount > 0);
    });
    if (rc != LBM_OK) {
        delete b;
        return rc;
    }
    *out = b;
    return LBM_OK;
}

int lbm_batch_update(lbm_batch* b, int coarse_steps) {
    if (!b || coarse_steps < 0) return fail(LBM_ERR_INVALID, "lbm_batch_update: bad argument");
    return guarded("lbm_batch_update", [&] {
        if (coarse_steps == 0) return;
        batchCheckParity(b);
        // after whatever the members' streams hold, and before what they get next
        for (lbm_grids* g : b->members) {
            ck(cudaEventRecord(b->sync, g->stream), "event");
            ck(cudaStreamWaitEvent(b->stream, b->sync, 0), "wait");
        }
        batchAdvance(b, coarse_steps);
        ck(cudaEventRecord(b->sync, b->stream), "event");
        for (lbm_grids* g : b->members) ck(cudaStreamWaitEvent(g->stream, b->sync, 0), "wait");
    });
}

int lbm_batch_time_steps(lbm_batch* b, int coarse_steps, float* ms) {
    if (!b || !ms || coarse_steps < 0) return fail(LBM_ERR_INVALID, "lbm_batch_time_steps: bad argument");
    return guarded("lbm_batch_time_steps", [&] {
        batchCheckParity(b);
        for (lbm_grids* g : b->members) ck(cudaStreamSynchronize(g->stream), "sync");
        if (graphable(b->members[0])) {  // capture outside the timed region
            batchPairGraph(b, 0);
            batchPairGraph(b, 1);
        }
        ck(cudaEventRecord(b->ev0, b->stream), "event");
        batchAdvance(b, coarse_steps);
        ck(cudaEventRecord(b->ev1, b->stream), "event");
        ck(cudaEventSynchronize(b->ev1), "event sync");
        ck(cudaEventElapsedTime(ms, b->ev0, b->ev1), "elapsed");
    });
}

int lbm_batch_get_info(lbm_batch* b, lbm_batch_info* out) {
    if (!b || !out) return fail(LBM_ERR_INVALID, "lbm_batch_get_info: bad argument");
    *out = b->info;
    return LBM_OK;
}

void lbm_batch_free(lbm_batch* b) { delete b; }

int lbm_set_graphs(lbm_grids* g, int enabled) {
    if (!g) return fail(LBM_ERR_INVALID, "lbm_set_graphs: null grids");
    g->graphsEnabled = enabled != 0;
    return LBM_OK;
}

int lbm_time_steps_graph(lbm_grids* g, int steps, float* ms) {
    if (!g || !ms || steps < 0) return fail(LBM_ERR_INVALID, "lbm_time_steps_graph: bad argument");
    return guarded("lbm_time_steps_graph", [&] {
        // capture outside the timed region
        if (graphable(g) && steps >= 2) {
            pairGraph(g, 0);
            pairGraph(g, 1);
        }
        ck(cudaEventRecord(g->ev0, g->stream), "event");
        int s = 0;
        if (graphable(g))
            for (; s + 2 <= steps; s += 2) launchPair(g);
        for (; s < steps; ++s) updateAllGrids(g, 0);
        ck(cudaEventRecord(g->ev1, g->stream), "event");
        ck(cudaEventSynchronize(g->ev1), "event sync");
        checkDeviceFlag(g);
        ck(cudaEventElapsedTime(ms, g->ev0, g->ev1), "elapsed");
    });
}

int lbm_synchronize(lbm_grids* g) {
    if (!g) return fail(LBM_ERR_INVALID, "lbm_synchronize: null grids");
    return guarded("lbm_synchronize", [&] {
        ck(cudaStreamSynchronize(g->stream), "sync");
        checkDeviceFlag(g);
    });
}

int lbm_time_steps(lbm_grids* g, int steps, float* ms) {
    if (!g || !ms || steps < 0) return fail(LBM_ERR_INVALID, "lbm_time_steps: bad argument");
    return guarded("lbm_time_steps", [&] {
        // one collide-stream launch per level substep: 2^level per coarse step
        size_t launches = 0;
        for (const LevelState& L : g->levels) launches += size_t(steps) << L.info.gridID;
        while (g->kernelEvents.size() < 2 * launches) {
            cudaEvent_t e;
            ck(cudaEventCreate(&e), "cudaEventCreate");
            g->kernelEvents.push_back(e);
        }
        g->kernelEventsUsed = 0;
        g->timingKernels = true;
        try {
            ck(cudaEventRecord(g->ev0, g->stream), "event");
            for (int s = 0; s < steps; ++s) updateAllGrids(g, 0);
            ck(cudaEventRecord(g->ev1, g->stream), "event");
        } catch (...) {
            g->timingKernels = false;
            throw;
        }
        g->timingKernels = false;
        ck(cudaEventSynchronize(g->ev1), "event sync");
        checkDeviceFlag(g);
        ck(cudaEventElapsedTime(ms, g->ev0, g->ev1), "elapsed");
        float kernel = 0.f;
        for (int k = 0; k + 1 < g->kernelEventsUsed; k += 2) {
            float t = 0.f;
            ck(cudaEventElapsedTime(&t, g->kernelEvents[k], g->kernelEvents[k + 1]), "elapsed");
            kernel += t;
        }
        g->lastKernelMs = kernel;
        g->lastLaunches = g->kernelEventsUsed / 2;
        g->lastStepKernels = 0;
        for (size_t l = 0; l < g->levels.size(); ++l) {
            const LevelState& L = g->levels[l];
            g->lastStepKernels += (static_cast<long long>(steps) << L.info.gridID) * lbm::stepLaunchCount(L.dev);
            const lbm::DevInterface& I = L.itf;
            if (l + 1 < g->levels.size() && I.f2cCount + I.c2fCount + I.leftCount > 0)
                g->lastStepKernels += static_cast<long long>(steps) << L.info.gridID;
        }
    });
}

int lbm_last_kernel_time(lbm_grids* g, float* kernel_ms, int* launches) {
    if (!g || !kernel_ms || !launches) return fail(LBM_ERR_INVALID, "lbm_last_kernel_time: bad argument");
    *kernel_ms = g->lastKernelMs;
    *launches = g->lastLaunches;
    return LBM_OK;
}

int lbm_last_launch_count(lbm_grids* g, long long* kernels) {
    if (!g || !kernels) return fail(LBM_ERR_INVALID, "lbm_last_launch_count: bad argument");
    *kernels = g->lastStepKernels;
    return LBM_OK;
}

int lbm_level_count(lbm_grids* g) {
    if (!g) return fail(LBM_ERR_INVALID, "lbm_level_count: null grids");
    return static_cast<int>(g->levels.size());
}

int lbm_get_grid_info(lbm_grids* g, int level, lbm_grid_info* out) {
    if (!g || !out || level < 0 || level >= (int)g->levels.size())
        return fail(LBM_ERR_INVALID, "lbm_get_grid_info: bad argument");
    const LevelState& L = g->levels[level];
    std::memset(out, 0, sizeof(*out));
    out->grid_id = L.info.gridID;
    out->cell_count = L.info.cellCount;
    out->cell_count_x = L.info.nx;
    out->cell_count_y = L.info.ny;
    out->cell_count_z = L.info.nz;
    out->row_count = L.rowCount;
    out->wall_cell_count = L.wallCellCount;
    out->wall_adjacent_count = L.wallAdjacentCount;
    out->periodic_count = L.dev.perCount;
    out->open_bc_count = L.openBCCount;
    out->esotwist_flipper = L.info.esotwistFlipper ? 1 : 0;
    out->iterations_finished = L.info.iterationsFinished;
    out->storage = L.dev.storage;
    out->res = L.info.res;
    out->ox = L.info.ox;
    out->oy = L.info.oy;
    out->oz = L.info.oz;
    out->nu = L.info.nu;
    out->dt_phys = L.info.dtPhys;
    out->grid_memory_bytes = L.memBytes;
    out->f2c_count = L.itf.f2cCount;
    out->c2f_count = L.itf.c2fCount;
    out->leftover_count = L.itf.leftCount;
    return LBM_OK;
}

int lbm_read_array(lbm_grids* g, int level, int which, void* host, size_t bytes) {
    if (!g || !host || level < 0 || level >= (int)g->levels.size())
        return fail(LBM_ERR_INVALID, "lbm_read_array: bad argument");
    LevelState& L = g->levels[level];
    const lbm::DevLevel& d = L.dev;
    const size_t n = static_cast<size_t>(d.cellCount);
    const size_t r = static_cast<size_t>(L.rowCount);
    const void* src = nullptr;
    size_t need = 0;
    switch (which) {
        case LBM_ARRAY_SHIFTER: src = d.shifter; need = n * 4; break;
        case LBM_ARRAY_ROW_I: src = d.rowI; need = r * 4; break;
        case LBM_ARRAY_ROW_J: src = d.rowJ; need = r * 4; break;
        case LBM_ARRAY_ROW_K: src = d.rowK; need = r * 4; break;
        case LBM_ARRAY_ROW_JPLUS: src = d.rowJP; need = r * 4; break;
        case LBM_ARRAY_ROW_KPLUS: src = d.rowKP; need = r * 4; break;
        case LBM_ARRAY_ROW_JKPLUS: src = d.rowJKP; need = r * 4; break;
        case LBM_ARRAY_WALL_MAP: src = d.wallMap; need = n * 4; break;
        case LBM_ARRAY_PERIODIC_INDEX: src = d.perIndex; need = size_t(d.perCount) * 4; break;
        case LBM_ARRAY_PERIODIC_SOURCE: src = d.perSource; need = size_t(d.perCount) * 4; break;
        case LBM_ARRAY_WALL_INDEX: src = d.wallIndex; need = size_t(d.wallCount) * 4; break;
        case LBM_ARRAY_WALL_DATA: src = d.wallData; need = size_t(d.wallCount) * 4; break;
        case LBM_ARRAY_LINK_LENGTH: src = d.linkLength; need = size_t(d.wallCount) * 7 * 4; break;
        case LBM_ARRAY_WALL_FORCE: need = size_t(d.wallCount) * 3 * 4; break;  // FP64 on the device
        case LBM_ARRAY_WALL_VELOCITY: src = d.wallVel; need = size_t(d.wallCount) * 3 * 4; break;
        case LBM_ARRAY_OPEN_INDEX: src = d.obCell; need = size_t(d.obCount) * 4; break;
        case LBM_ARRAY_OPEN_SOURCE: src = L.obSource; need = size_t(d.obCount) * 4; break;
        case LBM_ARRAY_OPEN_REFERENCE: src = d.obRhoRef; need = size_t(d.obCount) * 2 * 4; break;
        case LBM_ARRAY_OPEN_CUMULATIVE: src = d.obRhoCum; need = size_t(d.obCount) * 2 * 4; break;
        case LBM_ARRAY_F: need = 27 * n * 4; break;
        default:
            if (which >= LBM_ARRAY_F2C_INDEX && which <= LBM_ARRAY_LEFTOVER_NBR) {
                const std::vector<int>* lists[7] = {&L.f2cIndex, &L.f2cChild, &L.c2fIndex, &L.c2fChild,
                                                    &L.leftIndex, &L.leftParent, &L.leftNbr};
                const std::vector<int>& v = *lists[which - LBM_ARRAY_F2C_INDEX];
                if (bytes != v.size() * sizeof(int))
                    return fail(LBM_ERR_INVALID, "lbm_read_array: byte count does not match array size");
                if (bytes) std::memcpy(host, v.data(), bytes);
                return LBM_OK;
            }
            if (which >= LBM_ARRAY_ROTOR_BASE && (which - LBM_ARRAY_ROTOR_BASE) / 4 < d.rotorCount) {
                const int r = (which - LBM_ARRAY_ROTOR_BASE) / 4, part = (which - LBM_ARRAY_ROTOR_BASE) % 4;
                const lbm::HostRotor& R = L.rotors[r];
                if (part == 0) { src = d.rotor[r].rotorMap; need = R.rotorMap.size() * 4; }
                else if (part == 1) { src = L.rotorIndex[r]; need = R.index.size() * 4; }
                else if (part == 2) { src = d.rotor[r].interp; need = R.interpolation.size() * 4; }
                else { src = d.rotor[r].force; need = 3 * 27 * R.index.size() * 4; }
                break;
            }
            return fail(LBM_ERR_INVALID, "lbm_read_array: unknown array id");
        case LBM_ARRAY_MACRO: need = 4 * n * 4; break;
    }
    if (bytes != need)
        return fail(LBM_ERR_INVALID, "lbm_read_array: byte count does not match array size (expected " +
                                         std::to_string(need) + ")");
    return guarded("lbm_read_array", [&] {
        if (need == 0) return;
        if (which == LBM_ARRAY_WALL_FORCE) {
            std::vector<double> tmp(need / 4);
            ck(cudaMemcpyAsync(tmp.data(), d.wallForce, tmp.size() * sizeof(double), cudaMemcpyDeviceToHost,
                               g->stream), "copy");
            ck(cudaStreamSynchronize(g->stream), "sync");
            float* out = static_cast<float*>(host);
            for (size_t q = 0; q < tmp.size(); ++q) out[q] = static_cast<float>(tmp[q]);
        } else if (which == LBM_ARRAY_F || which == LBM_ARRAY_MACRO) {
            float* tmp = devAlloc<float>(need / 4);
            try {
                if (which == LBM_ARRAY_F) lbm::launchGatherF(d, g->stream, tmp);
                else lbm::launchMacro(d, L.info.esotwistFlipper, g->stream, tmp);
                ck(cudaGetLastError(), "read launch");
                ck(cudaMemcpyAsync(host, tmp, need, cudaMemcpyDeviceToHost, g->stream), "copy");
                ck(cudaStreamSynchronize(g->stream), "sync");
            } catch (...) {
                cudaFree(tmp);
                throw;
            }
            cudaFree(tmp);
        } else if (which == LBM_ARRAY_OPEN_INDEX || which == LBM_ARRAY_OPEN_REFERENCE ||
                   which == LBM_ARRAY_OPEN_CUMULATIVE) {
            // device arrays are in kernel order; report them in ID order
            std::vector<uint32_t> tmp(need / 4);
            ck(cudaMemcpyAsync(tmp.data(), src, need, cudaMemcpyDeviceToHost, g->stream), "copy");
            ck(cudaStreamSynchronize(g->stream), "sync");
            const size_t m = L.obPerm.size();
            uint32_t* out = static_cast<uint32_t*>(host);
            for (size_t part = 0; part < tmp.size() / (m ? m : 1); ++part)
                for (size_t p = 0; p < m; ++p) out[part * m + L.obPerm[p]] = tmp[part * m + p];
        } else {
            ck(cudaMemcpyAsync(host, src, need, cudaMemcpyDeviceToHost, g->stream), "copy");
            ck(cudaStreamSynchronize(g->stream), "sync");
        }
    });
}

int lbm_write_f(lbm_grids* g, int level, const float* host, size_t bytes) {
    if (!g || !host || level < 0 || level >= (int)g->levels.size())
        return fail(LBM_ERR_INVALID, "lbm_write_f: bad argument");
    LevelState& L = g->levels[level];
    const size_t need = 27ULL * L.dev.cellCount * 4;
    if (bytes != need) return fail(LBM_ERR_INVALID, "lbm_write_f: byte count does not match");
    return guarded("lbm_write_f", [&] {
        float* tmp = devAlloc<float>(need / 4);
        try {
            ck(cudaMemcpyAsync(tmp, host, need, cudaMemcpyHostToDevice, g->stream), "copy");
            lbm::launchScatterF(L.dev, g->stream, tmp);
            ck(cudaGetLastError(), "write launch");
            ck(cudaStreamSynchronize(g->stream), "sync");
        } catch (...) {
            cudaFree(tmp);
            throw;
        }
        cudaFree(tmp);
    });
}

// Zero every tracker accumulator of every level (trackerFunctions.h:474-497).
static void resetTracker(lbm_grids* g) {
    for (LevelState& L : g->levels) {
        const lbm::DevLevel& d = L.dev;
        if (d.wallForce) ck(cudaMemsetAsync(d.wallForce, 0, 3 * size_t(d.wallCount) * sizeof(double), g->stream), "memset");
        if (d.obRhoCum) ck(cudaMemsetAsync(d.obRhoCum, 0, 2 * size_t(d.obCount) * sizeof(float), g->stream), "memset");
        for (int r = 0; r < d.rotorCount; ++r)
            if (d.rotor[r].force)
                ck(cudaMemsetAsync(d.rotor[r].force, 0, 3 * 27 * size_t(d.rotor[r].nonzero) * sizeof(float), g->stream),
                   "memset");
        L.iterationsSinceTrackerReset = 0;
    }
    ck(cudaStreamSynchronize(g->stream), "sync");
}

int lbm_kinetic_energy(lbm_grids* g, float uRefPhys, float domainLength, double* out) {
    if (!g || !out) return fail(LBM_ERR_INVALID, "lbm_kinetic_energy: bad argument");
    return guarded("lbm_kinetic_energy", [&] {
        double energy = 0.0;
        for (LevelState& L : g->levels) {
            ck(cudaMemsetAsync(g->scratch, 0, sizeof(double), g->stream), "memset");
            lbm::launchKineticEnergy(L.dev, L.info.esotwistFlipper, g->stream, g->scratch);
            ck(cudaGetLastError(), "energy launch");
            double sum = 0.0;
            ck(cudaMemcpyAsync(&sum, g->scratch, sizeof(double), cudaMemcpyDeviceToHost, g->stream), "copy");
            ck(cudaStreamSynchronize(g->stream), "sync");
            const double dx = double(L.info.res) / 1000.0;
            const double vs = dx / (double(L.info.dtPhys) * uRefPhys);
            energy += sum * dx * dx * dx * vs * vs;
        }
        const double len = double(domainLength) / 1000.0;
        *out = energy / (len * len * len);
    });
}

int lbm_global_sums(lbm_grids* g, double* out) {
    if (!g || !out) return fail(LBM_ERR_INVALID, "lbm_global_sums: bad argument");
    return guarded("lbm_global_sums", [&] {
        double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (LevelState& L : g->levels) {
            ck(cudaMemsetAsync(g->scratch, 0, 6 * sizeof(double), g->stream), "memset");
            lbm::launchGlobalSums(L.dev, L.info.esotwistFlipper, g->stream, g->scratch);
            ck(cudaGetLastError(), "global sums launch");
            double sum[6];
            ck(cudaMemcpyAsync(sum, g->scratch, sizeof(sum), cudaMemcpyDeviceToHost, g->stream), "copy");
            ck(cudaStreamSynchronize(g->stream), "sync");
            const double dx = double(L.info.res) / 1000.0;                // m
            const double cellMass = double(g->c.rho_phys) * dx * dx * dx;  // kg per unit lattice density
            const double vel = dx / double(L.info.dtPhys);                 // m/s per lattice velocity
            acc[0] += cellMass * sum[0];
            acc[1] += cellMass * sum[1];
            for (int a = 0; a < 3; ++a) acc[2 + a] += cellMass * vel * sum[2 + a];
            acc[5] += sum[5];
            acc[6] += sum[0];
            acc[7] += sum[1];
        }
        for (int q = 0; q < 8; ++q) out[q] = acc[q];
    });
}

int lbm_kinetic_energy_noalloc(lbm_grids* g, float uRefPhys, float domainLength, double* out) {
    static_assert(lbm::kNoAllocEnergyMaxCells == LBM_KINETIC_ENERGY_NOALLOC_MAX_CELLS,
                  "header limit and scratch size disagree");
    if (!g || !out) return fail(LBM_ERR_INVALID, "lbm_kinetic_energy_noalloc: bad argument");
    for (const LevelState& L : g->levels)
        if (L.dev.cellCount > lbm::kNoAllocEnergyMaxCells)
            return fail(LBM_ERR_INVALID, "lbm_kinetic_energy_noalloc: level " + std::to_string(L.info.gridID) +
                                             " has " + std::to_string(L.dev.cellCount) +
                                             " cells; the static scratch covers at most " +
                                             std::to_string(lbm::kNoAllocEnergyMaxCells));
    return guarded("lbm_kinetic_energy_noalloc", [&] {
        double energy = 0.0;
        for (LevelState& L : g->levels) {
            double sum = 0.0;
            ck(lbm::kineticEnergyNoAlloc(L.dev, L.info.esotwistFlipper, g->stream, &sum), "energy");
            const double dx = double(L.info.res) / 1000.0;
            const double vs = dx / (double(L.info.dtPhys) * uRefPhys);
            energy += sum * dx * dx * dx * vs * vs;
        }
        const double len = double(domainLength) / 1000.0;
        *out = energy / (len * len * len);
    });
}

int lbm_wall_force(lbm_grids* g, int wallID, int reset, double* out) {
    if (!g || !out || wallID < 0 || wallID >= LBM_MAX_BODIES)
        return fail(LBM_ERR_INVALID, "lbm_wall_force: bad argument");
    return guarded("lbm_wall_force", [&] {
        double acc[6] = {0, 0, 0, 0, 0, 0};
        for (LevelState& L : g->levels) {
            ck(cudaMemsetAsync(g->scratch, 0, 6 * sizeof(double), g->stream), "memset");
            lbm::launchWallForce(L.dev, wallID, g->stream, g->scratch);
            ck(cudaGetLastError(), "force launch");
            double r[6];
            ck(cudaMemcpyAsync(r, g->scratch, sizeof(r), cudaMemcpyDeviceToHost, g->stream), "copy");
            ck(cudaStreamSynchronize(g->stream), "sync");
            const double span = L.iterationsSinceTrackerReset > 0 ? L.iterationsSinceTrackerReset : 1;
            // convertToPhysicalForce (include/cellFunctions.h:296-301); torque from N mm to N m
            const double rm = double(L.info.res) / 1000.0;
            const double conv = double(g->c.rho_phys) * rm * rm * rm * rm / (double(L.info.dtPhys) * L.info.dtPhys);
            for (int q = 0; q < 3; ++q) acc[q] += r[q] / span * conv;
            for (int q = 3; q < 6; ++q) acc[q] += r[q] / span * conv * 0.001;
        }
        if (reset) resetTracker(g);
        for (int q = 0; q < 6; ++q) out[q] = acc[q];
    });
}

static void fillRotorInfo(const lbm::HostRotor& R, lbm_rotor_info* out) {
    std::memset(out, 0, sizeof(*out));
    out->res = R.res;
    out->bounds[0] = R.xMin; out->bounds[1] = R.yMin; out->bounds[2] = R.zMin;
    out->bounds[3] = R.xMax; out->bounds[4] = R.yMax; out->bounds[5] = R.zMax;
    out->cell_count[0] = R.cntX; out->cell_count[1] = R.cntY; out->cell_count[2] = R.cntZ;
    out->block_count = static_cast<int>(R.rotorMap.size());
    out->nonzero_block_count = static_cast<int>(R.index.size());
    out->axis = R.axis;
    out->origin[0] = R.ox; out->origin[1] = R.oy; out->origin[2] = R.oz;
    out->radians_per_second = R.radiansPerSecond;
    out->radians_elapsed = R.radiansElapsed;
}

int lbm_plan_rotor_info(lbm_plan* p, int level, int rotor, lbm_rotor_info* out) {
    if (!p || !out || level < 0 || level >= (int)p->host.levels.size() || rotor < 0 ||
        rotor >= (int)p->host.levels[level].rotors.size())
        return fail(LBM_ERR_INVALID, "lbm_plan_rotor_info: bad argument");
    fillRotorInfo(p->host.levels[level].rotors[rotor], out);
    return LBM_OK;
}

int lbm_get_rotor_info(lbm_grids* g, int level, int rotor, lbm_rotor_info* out) {
    if (!g || !out || level < 0 || level >= (int)g->levels.size() || rotor < 0 ||
        rotor >= (int)g->levels[level].rotors.size())
        return fail(LBM_ERR_INVALID, "lbm_get_rotor_info: bad argument");
    fillRotorInfo(g->levels[level].rotors[rotor], out);
    return LBM_OK;
}

int lbm_set_rotor_speed(lbm_grids* g, int rotor, float radiansPerSecond) {
    if (!g || rotor < 0) return fail(LBM_ERR_INVALID, "lbm_set_rotor_speed: bad argument");
    bool found = false;
    for (LevelState& L : g->levels) {
        if (rotor >= (int)L.rotors.size()) continue;
        L.rotors[rotor].radiansPerSecond = radiansPerSecond;
        L.dev.rotor[rotor].scale = radiansPerSecond * L.info.dtPhys / L.info.res;
        found = true;
    }
    if (!found) return fail(LBM_ERR_INVALID, "lbm_set_rotor_speed: no rotor with this index");
    return LBM_OK;
}

int lbm_rotor_force(lbm_grids* g, int rotor, int reset, double* out) {
    if (!g || !out || rotor < 0) return fail(LBM_ERR_INVALID, "lbm_rotor_force: bad argument");
    return guarded("lbm_rotor_force", [&] {
        double acc[6] = {0, 0, 0, 0, 0, 0};
        bool found = false;
        for (LevelState& L : g->levels) {
            if (rotor >= L.dev.rotorCount) continue;
            found = true;
            ck(cudaMemsetAsync(g->scratch, 0, 6 * sizeof(double), g->stream), "memset");
            lbm::launchRotorForce(L.dev.rotor[rotor], L.rotorIndex[rotor], g->stream, g->scratch);
            ck(cudaGetLastError(), "rotor force launch");
            double r[6];
            ck(cudaMemcpyAsync(r, g->scratch, sizeof(r), cudaMemcpyDeviceToHost, g->stream), "copy");
            ck(cudaStreamSynchronize(g->stream), "sync");
            const double span = L.iterationsSinceTrackerReset > 0 ? L.iterationsSinceTrackerReset : 1;
            // convertToPhysicalForce (include/cellFunctions.h:296-301); torque from N mm to N m
            const double rm = double(L.info.res) / 1000.0;
            const double conv = double(g->c.rho_phys) * rm * rm * rm * rm / (double(L.info.dtPhys) * L.info.dtPhys);
            for (int q = 0; q < 3; ++q) acc[q] += r[q] / span * conv;
            for (int q = 3; q < 6; ++q) acc[q] += r[q] / span * conv * 0.001;
        }
        if (!found) throw std::invalid_argument("no rotor with this index");
        if (reset) resetTracker(g);
        for (int q = 0; q < 6; ++q) out[q] = acc[q];
    });
}

int lbm_export_vtk(lbm_grids* g, const char* filename) {
    if (!g || !filename) return fail(LBM_ERR_INVALID, "lbm_export_vtk: null argument");
    return guarded("lbm_export_vtk", [&] {
        // per level: cell centres (mm), wall flag, velocity (m/s), pressure
        // (Pa), interface overlap flag, all computed as the reference does
        struct LevelFields {
            std::vector<float> x, y, z, ux, uy, uz, p;
            std::vector<unsigned char> wall, overlap;
            int gridID = 0;
            float res = 0.f;
        };
        std::vector<LevelFields> lf(g->levels.size());
        size_t total = 0;
        const float invSqrt3 = 0.57735026918962576f;
        for (size_t l = 0; l < g->levels.size(); ++l) {
            LevelState& L = g->levels[l];
            const lbm::DevLevel& d = L.dev;
            const size_t n = static_cast<size_t>(d.cellCount);
            const size_t rows = static_cast<size_t>(L.rowCount);
            auto fetch = [&](const void* src, size_t bytes, void* dst) {
                if (bytes) ck(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, g->stream), "copy");
            };
            std::vector<int> shifter(n), rI(rows), rJ(rows), rK(rows), wallMap(n);
            std::vector<unsigned> wallData(static_cast<size_t>(d.wallCount));
            fetch(d.shifter, n * 4, shifter.data());
            fetch(d.rowI, rows * 4, rI.data());
            fetch(d.rowJ, rows * 4, rJ.data());
            fetch(d.rowK, rows * 4, rK.data());
            fetch(d.wallMap, n * 4, wallMap.data());
            fetch(d.wallData, wallData.size() * 4, wallData.data());
            std::vector<float> macro(4 * n);
            if (n) {
                float* tmp = devAlloc<float>(4 * n);
                try {
                    lbm::launchMacro(d, L.info.esotwistFlipper, g->stream, tmp);
                    ck(cudaGetLastError(), "macro launch");
                    fetch(tmp, 4 * n * 4, macro.data());
                    ck(cudaStreamSynchronize(g->stream), "sync");
                } catch (...) {
                    cudaFree(tmp);
                    throw;
                }
                cudaFree(tmp);
            }
            ck(cudaStreamSynchronize(g->stream), "sync");
            LevelFields& F = lf[l];
            F.gridID = L.info.gridID;
            F.res = L.info.res;
            for (auto* v : {&F.x, &F.y, &F.z, &F.ux, &F.uy, &F.uz, &F.p}) v->assign(n, 0.f);
            F.wall.assign(n, 0);
            F.overlap.assign(n, 0);
            const lbm::Info& in = L.info;
            const float scale = (in.res / 1000.f);
            const float cs = invSqrt3 * (in.res / 1000.f) / in.dtPhys;
            for (size_t c = 0; c < n; ++c) {
                // getCompressedIJK (include/cellFunctions.h:51-72)
                const int sh = shifter[c];
                const int head = sh >= 0 ? static_cast<int>(c) : static_cast<int>(c) + sh;
                const int row = shifter[static_cast<size_t>(head)];
                const int i = rI[row] + (static_cast<int>(c) - head), j = rJ[row], k = rK[row];
                F.x[c] = i * in.res + in.ox;
                F.y[c] = j * in.res + in.oy;
                F.z[c] = k * in.res + in.oz;
                const int wm = wallMap[c];
                if (wm == -3) {
                    F.wall[c] = 1;
                    continue;
                }
                F.overlap[c] = (wm == -2 || (wm >= 0 && (wallData[static_cast<size_t>(wm)] & 1u))) ? 1 : 0;
                // convertToPhysicalVelocity / convertToPhysicalPressure (include/cellFunctions.h:281-294)
                F.ux[c] = macro[n + c] * scale / in.dtPhys;
                F.uy[c] = macro[2 * n + c] * scale / in.dtPhys;
                F.uz[c] = macro[3 * n + c] * scale / in.dtPhys;
                F.p[c] = macro[c] * g->c.rho_phys * cs * cs;
            }
            total += n;
        }
        FILE* fp = std::fopen(filename, "w");
        if (!fp) throw std::runtime_error(std::string("cannot open VTK file: ") + filename);
        std::string buf;
        buf.reserve(1 << 22);
        char tmp[128];
        auto flush = [&](bool force) {
            if (force || buf.size() > (1u << 21)) {
                if (std::fwrite(buf.data(), 1, buf.size(), fp) != buf.size()) {
                    std::fclose(fp);
                    throw std::runtime_error(std::string("failed writing VTK file: ") + filename);
                }
                buf.clear();
            }
        };
        auto add = [&](const char* fmt, auto... v) {
            const int k = std::snprintf(tmp, sizeof(tmp), fmt, v...);
            buf.append(tmp, static_cast<size_t>(k));
            flush(false);
        };
        // legacy VTK POLYDATA, one vertex per cell (include/exportVTK.h:17-158);
        // floats with 9 significant digits (max_digits10 of float)
        add("# vtk DataFile Version 3.0\nLBM snapshot; coordinates in mm; grid count %zu\nASCII\nDATASET POLYDATA\n",
            lf.size());
        add("POINTS %zu float\n", total);
        for (const auto& F : lf)
            for (size_t c = 0; c < F.x.size(); ++c) add("%.9g %.9g %.9g\n", double(F.x[c]), double(F.y[c]), double(F.z[c]));
        add("VERTICES %zu %zu\n", total, 2 * total);
        for (size_t c = 0; c < total; ++c) add("1 %zu\n", c);
        add("POINT_DATA %zu\nSCALARS wall int 1\nLOOKUP_TABLE default\n", total);
        for (const auto& F : lf)
            for (unsigned char w : F.wall) add("%d\n", int(w));
        add("VECTORS velocity_m_s float\n");
        for (const auto& F : lf)
            for (size_t c = 0; c < F.ux.size(); ++c)
                add("%.9g %.9g %.9g\n", double(F.ux[c]), double(F.uy[c]), double(F.uz[c]));
        add("SCALARS pressure_Pa float 1\nLOOKUP_TABLE default\n");
        for (const auto& F : lf)
            for (float v : F.p) add("%.9g\n", double(v));
        add("SCALARS grid_id int 1\nLOOKUP_TABLE default\n");
        for (const auto& F : lf)
            for (size_t c = 0; c < F.x.size(); ++c) add("%d\n", F.gridID);
        add("SCALARS grid_resolution_mm float 1\nLOOKUP_TABLE default\n");
        for (const auto& F : lf)
            for (size_t c = 0; c < F.x.size(); ++c) add("%.9g\n", double(F.res));
        add("SCALARS interface_overlap int 1\nLOOKUP_TABLE default\n");
        for (const auto& F : lf)
            for (unsigned char o : F.overlap) add("%d\n", int(o));
        flush(true);
        if (std::fclose(fp) != 0) throw std::runtime_error(std::string("failed writing VTK file: ") + filename);
    });
}

int lbm_flow_report(lbm_grids* g, int plane, float cut, const float* bounds, double* out) {
    if (!g || !out || plane < 0 || plane > 2) return fail(LBM_ERR_INVALID, "lbm_flow_report: bad argument");
    if (g->levels.size() != 1) return flowReportLevels(g, plane, cut, bounds, out);
    LevelState& L = g->levels[0];
    const lbm::Info& in = L.info;
    const int n[3] = {in.nx, in.ny, in.nz};
    const float o[3] = {in.ox, in.oy, in.oz};
    const int axis = plane == LBM_PLANE_XY ? 2 : plane == LBM_PLANE_ZY ? 0 : 1;
    // getIJKCellIndexFromXYZ (include/cellFunctions.h:96-101)
    const int layer = static_cast<int>((cut - o[axis]) / in.res + 0.5f);
    if (layer < 0 || layer >= n[axis]) return fail(LBM_ERR_INVALID, "lbm_flow_report: cut outside the grid");
    // crop (include/flowReportFunctions.h:36-55)
    int lo[3] = {0, 0, 0}, hi[3] = {n[0], n[1], n[2]};
    if (bounds && (bounds[0] != 0.f || bounds[1] != 0.f || bounds[2] != 0.f || bounds[3] != 0.f ||
                   bounds[4] != 0.f || bounds[5] != 0.f))
        for (int a = 0; a < 3; ++a) {
            const float tMin = o[a] - 0.5f * in.res;
            const float tMax = o[a] + in.res * (n[a] - 0.5f);
            lo[a] = std::max(0, static_cast<int>(std::ceil((bounds[a] - tMin) / in.res)));
            hi[a] = std::min(n[a], n[a] - static_cast<int>(std::ceil((tMax - bounds[a + 3]) / in.res)));
        }
    const int hAxis = plane == LBM_PLANE_XY ? 0 : 2, vAxis = plane == LBM_PLANE_ZX ? 0 : 1;
    if (hi[hAxis] <= lo[hAxis] || hi[vAxis] <= lo[vAxis])
        return fail(LBM_ERR_INVALID, "lbm_flow_report: empty crop");
    return guarded("lbm_flow_report", [&] {
        ck(cudaMemsetAsync(g->scratch, 0, 6 * sizeof(double), g->stream), "memset");
        lbm::launchFlowReport(L.dev, in.esotwistFlipper, g->stream, plane, layer, lo[hAxis], hi[hAxis], lo[vAxis],
                              hi[vAxis], g->scratch);
        ck(cudaGetLastError(), "flow report launch");
        double t[6];
        ck(cudaMemcpyAsync(t, g->scratch, sizeof(t), cudaMemcpyDeviceToHost, g->stream), "copy");
        ck(cudaStreamSynchronize(g->stream), "sync");
        for (int q = 0; q < 7; ++q) out[q] = 0.0;
        if (t[5] == 0.0) return;
        // unit conversion (include/flowReportFunctions.h:322-351)
        const double px = double(in.res) / 1000.0, area = px * px, vs = px / double(in.dtPhys);
        const double ps = double(g->c.rho_phys) * vs * vs / 3.0;  // convertToPhysicalPressure of 1
        const double mfs = double(g->c.rho_phys) * area * vs;
        out[0] = t[0] / t[5] * vs;
        out[1] = (t[0] + t[1]) * mfs;
        out[2] = t[2] * mfs * vs;
        out[3] = t[3] / t[5] * ps;
        out[4] = t[1] * area * ps * vs;
        out[5] = t[4] * mfs * vs * vs;
        out[6] = t[5] * double(in.res) * in.res;
    });
}

namespace {

// One device region of the saved state of a level.
struct StateRegion {
    void* ptr;
    size_t bytes;
};

std::vector<StateRegion> stateRegions(LevelState& L) {
    lbm::DevLevel& d = L.dev;
    std::vector<StateRegion> r;
    r.push_back({d.f, 27ULL * size_t(d.stride) * storageBytes(d.storage)});
    if (d.obCount) {
        r.push_back({d.obRhoRef, 2ULL * d.obCount * sizeof(float)});
        r.push_back({d.obRhoCum, 2ULL * d.obCount * sizeof(float)});
    }
    if (d.wallCount) r.push_back({d.wallForce, 3ULL * d.wallCount * sizeof(double)});
    for (int q = 0; q < d.rotorCount; ++q)
        if (d.rotor[q].nonzero) r.push_back({d.rotor[q].force, 3ULL * 27 * d.rotor[q].nonzero * sizeof(float)});
    // the stochastic rounding's step seeds, so a resumed run draws the same bits
    if (d.seed) r.push_back({d.seed, 2 * sizeof(unsigned)});
    return r;
}

// host scalars of a level: counts (to check the target), flipper, counters,
// rotor angle and speed
struct StateHeader {
    long long cellCount, stride;
    int storage, obCount, wallCount, rotorCount;
    int flipper, iterationsFinished, iterationsSinceTrackerReset, pad;
    double radiansElapsed[LBM_MAX_ROTORS];
    float radiansPerSecond[LBM_MAX_ROTORS];
};

constexpr unsigned long long kStateMagic = 0x3154504b43334d42ULL;  // "BM3CKPT1"

size_t stateSize(lbm_grids* g) {
    size_t n = 16;
    for (LevelState& L : g->levels) {
        n += sizeof(StateHeader);
        for (const StateRegion& r : stateRegions(L)) n += r.bytes;
    }
    return n;
}

}  // namespace

int lbm_state_bytes(lbm_grids* g, size_t* bytes) {
    if (!g || !bytes) return fail(LBM_ERR_INVALID, "lbm_state_bytes: bad argument");
    *bytes = stateSize(g);
    return LBM_OK;
}

int lbm_save_state(lbm_grids* g, void* host, size_t bytes) {
    if (!g || !host) return fail(LBM_ERR_INVALID, "lbm_save_state: bad argument");
    if (bytes != stateSize(g))
        return fail(LBM_ERR_INVALID, "lbm_save_state: byte count does not match lbm_state_bytes");
    return guarded("lbm_save_state", [&] {
        unsigned char* out = static_cast<unsigned char*>(host);
        const unsigned long long head[2] = {kStateMagic, g->levels.size()};
        std::memcpy(out, head, 16);
        out += 16;
        for (LevelState& L : g->levels) {
            StateHeader h{};
            h.cellCount = L.dev.cellCount;
            h.stride = L.dev.stride;
            h.storage = L.dev.storage;
            h.obCount = L.dev.obCount;
            h.wallCount = L.dev.wallCount;
            h.rotorCount = L.dev.rotorCount;
            h.flipper = L.info.esotwistFlipper ? 1 : 0;
            h.iterationsFinished = L.info.iterationsFinished;
            h.iterationsSinceTrackerReset = L.iterationsSinceTrackerReset;
            for (size_t q = 0; q < L.rotors.size(); ++q) {
                h.radiansElapsed[q] = L.rotors[q].radiansElapsed;
                h.radiansPerSecond[q] = L.rotors[q].radiansPerSecond;
            }
            std::memcpy(out, &h, sizeof(h));
            out += sizeof(h);
            for (const StateRegion& r : stateRegions(L)) {
                ck(cudaMemcpyAsync(out, r.ptr, r.bytes, cudaMemcpyDeviceToHost, g->stream), "copy");
                out += r.bytes;
            }
        }
        ck(cudaStreamSynchronize(g->stream), "sync");
    });
}

int lbm_load_state(lbm_grids* g, const void* host, size_t bytes) {
    if (!g || !host) return fail(LBM_ERR_INVALID, "lbm_load_state: bad argument");
    if (bytes != stateSize(g))
        return fail(LBM_ERR_INVALID, "lbm_load_state: the state does not belong to grids of this size");
    const unsigned char* in = static_cast<const unsigned char*>(host);
    unsigned long long head[2];
    std::memcpy(head, in, 16);
    if (head[0] != kStateMagic || head[1] != g->levels.size())
        return fail(LBM_ERR_INVALID, "lbm_load_state: not a saved state of these grids");
    // check every level header before changing anything
    {
        const unsigned char* p = in + 16;
        for (LevelState& L : g->levels) {
            StateHeader h;
            std::memcpy(&h, p, sizeof(h));
            if (h.cellCount != L.dev.cellCount || h.stride != L.dev.stride || h.storage != L.dev.storage ||
                h.obCount != L.dev.obCount || h.wallCount != L.dev.wallCount || h.rotorCount != L.dev.rotorCount)
                return fail(LBM_ERR_INVALID, "lbm_load_state: the state belongs to a different case");
            p += sizeof(h);
            for (const StateRegion& r : stateRegions(L)) p += r.bytes;
        }
    }
    return guarded("lbm_load_state", [&] {
        const unsigned char* p = in + 16;
        for (LevelState& L : g->levels) {
            StateHeader h;
            std::memcpy(&h, p, sizeof(h));
            p += sizeof(h);
            L.info.esotwistFlipper = h.flipper != 0;
            L.info.iterationsFinished = h.iterationsFinished;
            L.iterationsSinceTrackerReset = h.iterationsSinceTrackerReset;
            for (size_t q = 0; q < L.rotors.size(); ++q) {
                L.rotors[q].radiansElapsed = h.radiansElapsed[q];
                L.rotors[q].radiansPerSecond = h.radiansPerSecond[q];
                L.dev.rotor[q].scale = h.radiansPerSecond[q] * L.info.dtPhys / L.info.res;
            }
            for (const StateRegion& r : stateRegions(L)) {
                ck(cudaMemcpyAsync(r.ptr, p, r.bytes, cudaMemcpyHostToDevice, g->stream), "copy");
                p += r.bytes;
            }
            if (L.dev.obCounter) {
                const int counter[2] = {L.info.iterationsFinished, 0};
                ck(cudaMemcpyAsync(L.dev.obCounter, counter, sizeof(counter), cudaMemcpyHostToDevice, g->stream),
                   "copy");
                ck(cudaStreamSynchronize(g->stream), "sync");
            }
        }
        ck(cudaStreamSynchronize(g->stream), "sync");
    });
}

int lbm_open_boundary_flow(lbm_grids* g, int openBCID, int reset, double* out) {
    if (!g || !out || openBCID < 0) return fail(LBM_ERR_INVALID, "lbm_open_boundary_flow: bad argument");
    return guarded("lbm_open_boundary_flow", [&] {
        double area = 0.0, acc[6] = {0, 0, 0, 0, 0, 0};
        bool found = false;
        for (LevelState& L : g->levels) {
            if (openBCID >= static_cast<int>(L.openTrackCount.size())) continue;
            found = true;
            ck(cudaMemsetAsync(g->scratch, 0, 6 * sizeof(double), g->stream), "memset");
            const double span = L.iterationsSinceTrackerReset > 0 ? L.iterationsSinceTrackerReset : 1;
            lbm::launchOpenFlow(L.dev, openBCID, static_cast<float>(1.0 / span), g->stream, g->scratch);
            ck(cudaGetLastError(), "flow launch");
            double r[6];
            ck(cudaMemcpyAsync(r, g->scratch, sizeof(r), cudaMemcpyDeviceToHost, g->stream), "copy");
            ck(cudaStreamSynchronize(g->stream), "sync");
            // unit conversion of updateTracker (include/trackerFunctions.h:176-186)
            const double cellArea = (double(L.info.res) / 1000.0) * (double(L.info.res) / 1000.0);
            const double v = (double(L.info.res) / 1000.0) / double(L.info.dtPhys);
            const double rho = g->c.rho_phys;
            const double cs = v / std::sqrt(3.0);
            const double p = rho * cs * cs;  // convertToPhysicalPressure
            acc[0] += r[0] * cellArea * v;
            acc[1] += r[1] * cellArea * v * rho;
            acc[2] += r[2] * cellArea * v * v * rho;
            acc[3] += r[3] * p * cellArea;
            acc[4] += r[4] * p * cellArea * v;
            acc[5] += r[5] * cellArea * v * v * v * rho;
            area += L.openTrackCount[openBCID] * cellArea;
        }
        if (!found) throw std::invalid_argument("no open boundary with this ID");
        out[0] = area;
        out[1] = area > 0 ? acc[0] / area : 0.0;
        out[2] = acc[1];
        out[3] = acc[2];
        out[4] = area > 0 ? acc[3] / area : 0.0;
        out[5] = acc[4];
        out[6] = acc[5];
        if (reset) resetTracker(g);
    });
}

int lbm_apply_collision_batch(float* d_f, int n, float nu, float limiter, float nuMultiplier, float gx,
                              float gy, float gz, void* stream) {
    if (!d_f || n < 0) return fail(LBM_ERR_INVALID, "lbm_apply_collision_batch: bad argument");
    return guarded("lbm_apply_collision_batch", [&] {
        if (n == 0) return;
        const lbm::CollisionConsts P = lbm::makeCollisionConsts(nu, nuMultiplier, limiter);
        lbm::launchCollideBatch(d_f, n, P, gx, gy, gz, static_cast<cudaStream_t>(stream));
        ck(cudaGetLastError(), "collision launch");
    });
}

}  // extern "C"
