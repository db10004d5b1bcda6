// Working set of one rewriting pass and the execution context its stages
// share.  Stage functions live in rw_front.cu, rw_eval.cu, rw_replace.cu and
// rw_choice.cu; Engine::rw (rw_pass.cu) runs them in order.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "engine.cuh"
#include "kernels.cuh"

namespace culs {

struct ExecCtx {
    cudaStream_t s = nullptr;
    Arena *ar = nullptr;
    int *status = nullptr;    // device status word
    int *counters = nullptr;  // 64 device ints of scratch
    int *hostSmall = nullptr; // 64 pinned host ints
    const RwLib *lib = nullptr;
    int sms = 148;
    bool clusters = true;  // thread-block clusters may be launched on s (not on an SM-partition stream)
    int *launches = nullptr;
    std::string *err = nullptr;
    const Tune *tune = nullptr;  // launch and schedule parameters
    cudaEvent_t *ev = nullptr;  // profiling marks (null when profiling is off)
    bool *evSet = nullptr;
    void mark(int m) {
        if (ev) {
            cudaEventRecord(ev[m], s);
            evSet[m] = true;
        }
    }

    int fail(int code, const std::string &m) {
        if (err) *err = m;
        return code;
    }
    int check(cudaError_t e, const char *what) {
        if (e == cudaSuccess) return 0;
        if (err) *err = std::string(what) + ": " + cudaGetErrorString(e);
        return CULS_E_DEVICE;
    }
    int sync() { return check(cudaStreamSynchronize(s), "stream sync"); }
    // Reads the device status word (after a sync) and maps it to an error.
    int status_check(const char *what);
    void launched(int k = 1) {
        if (launches) *launches += k;
    }
    unsigned grid(int64_t n, int block = kBlock) const { return grid_1d(n, block, sms * 16); }
};

// Objects of the batch in the level-major working layout W: position q holds
// the node the reference numbers levelCount[level-1] + rank after
// rw::CPUSolver::Reorder (src/algorithms/rewrite.cu:1245-1279), graphs
// interleaved inside a level.  Literals are AIGER convention (0 = FALSE).
struct RwWork {
    int G = 0;
    int64_t N = 0;    // original objects (all graphs)
    int64_t nL0 = 0;  // constants and PIs: W positions [0, nL0)
    int64_t nPO = 0;
    int maxLevel = 0;
    int64_t width = 1;  // Batch::flow_width of the batch: nodes a level-ordered pass can work on at once
    unsigned long long *warpPairs = nullptr;  // device counter (RwStats::warpPairs)
    bool useZeros = false;
    DevGraph *dg = nullptr;  // device graph table (cpos = constant's W position)

    int *w0 = nullptr, *w1 = nullptr;  // fanin literals, w0 <= w1 for AND nodes
    int *wg = nullptr, *wl = nullptr;  // graph id, local (reordered) id
    uint8_t *lidLow = nullptr;         // local id & 31 (cut signatures)
    int *wlev = nullptr;               // level (0 = constant / PI)
    uint8_t *wph = nullptr;            // value under the all-zero input
    int *ref = nullptr;                // fanout counts incl. PO references
    int *wpo = nullptr;                // PO literals
    int4 *cutL = nullptr;              // 8 cut slots per object: leaves
    int2 *cutM = nullptr;              //   {sign, packed}
    int *byGraph = nullptr;            // W positions grouped by graph (W order inside a graph)
    RegionTable tab{};                 // existence table, one region per graph
    int8_t *bestCut = nullptr;  // chosen slot or -1
    uint8_t *bestOut = nullptr; // chosen subgraph root index

    int64_t nCand = 0;
    int *cand = nullptr;  // W positions of nodes with a chosen cut, W order
    int *repW = nullptr;  // per candidate: replacement literal (rebuilt ids) or -1

    // after the replacement stage: W positions [N, N + nNew) hold new nodes
    int64_t nNew = 0;
    int *L0 = nullptr, *L1 = nullptr;  // fanin literals of [0, N + nNew)
    int *gidAll = nullptr;             // graph of [0, N + nNew)
    uint8_t *del = nullptr;            // isDeleted over [0, N + nNew)
    int *newOwnLev = nullptr;          // per new node: W level of its owner candidate (non-decreasing)
    int *choice = nullptr;             // per candidate outcome code
};

// choice outcome codes (same numbering as the oracle's dump)
enum ChoiceCode : int {
    kChNotVisited = 0,
    kChNoCut = 1,
    kChSmallCut = 2,
    kChNoReplace = 3,
    kChSelfRef = 4,
    kChCompromised = 5,
    kChCommitted = 6,
    kChReverted = 7,
};

int rw_front(ExecCtx &X, Batch &b, RwWork &w);     // levelize, reorder, refs
int rw_enumerate(ExecCtx &X, RwWork &w);           // cut enumeration
int rw_evaluate(ExecCtx &X, RwWork &w, const Batch &b);  // table + evaluation + candidates
int rw_replace(ExecCtx &X, Batch &b, RwWork &w);   // subgraph build + rebuild ids
int rw_choice(ExecCtx &X, Batch &b, RwWork &w, RwStats *stats);  // sequential choice per graph
int rw_redundancy(ExecCtx &X, Batch &b, RwWork &w);  // buffer chasing

}  // namespace culs
