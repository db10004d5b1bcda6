// Existence table and per-node evaluation: BuildHashTable + EvaluateNode
// (CULS src/algorithms/rewrite.cu:378-471).  The chained table of the
// reference becomes an open-addressing table on 64-bit CAS keys (fanin0 id,
// fanin1 id, compl0, compl1) with one region per graph.  Both the build and
// the evaluation visit the nodes graph by graph (the front's byGraph order),
// so the region, cuts and fanin arrays a block touches belong to the few
// graphs in flight.
//
// One thread evaluates one AND node: its cuts in slot order, each walked
// through the NPN class's library forest, with the 54-entry match/level
// scratch in shared memory laid out entry-major, so lanes reading the same
// library entry hit distinct banks.
#include <vector>

#include "rw_work.cuh"

namespace culs {

namespace {

constexpr int kEvalBlock = 64;
constexpr int kLibSlots = 54;  // 4 inputs + at most 50 library nodes

__global__ void k_table_clear(int64_t n, TabSlot *slots) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        reinterpret_cast<int4 *>(slots)[i] = make_int4(-1, -1, 0x7FFFFFFF, 0);
}

__global__ void k_table_build(int64_t nL0, int64_t N, const int *byGraph, const int *w0, const int *w1, const int *wg,
                              const int *wlev, const DevGraph *dg, RegionTable tab, int *status) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += stride) {
        const int q = byGraph[i];
        if (q < nL0) continue;  // constant or PI
        int f0 = w0[q], f1 = w1[q];
        const int g = wg[q];
        int cp = dg[g].cpos;
        // rewrite.cu:454 skips nodes whose fanins are both the constant
        if ((f0 >> 1) == cp && (f1 >> 1) == cp) continue;
        region_insert(table_region(tab, g), and_key(f0 >> 1, f1 >> 1, f0 & 1, f1 & 1), q, wlev[q], status);
    }
}

struct EvalArgs {
    int64_t nL0, N;
    const int *byGraph;
    EvalIn E;
    RegionTable tab;
    const int4 *cutL;
    const int2 *cutM;
    const int *wg;
    const DevGraph *dg;
    int useZeros;
    int8_t *bestCut;
    uint8_t *bestOut;
    uint8_t *candFlag;
};

__global__ void __launch_bounds__(kEvalBlock) k_evaluate(EvalArgs A) {
    __shared__ int s_match[kLibSlots * kEvalBlock];
    __shared__ int s_mlev[kLibSlots * kEvalBlock];
    int *match = s_match + threadIdx.x;
    int *mlev = s_mlev + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < A.N; i += stride) {
        const int64_t q = A.byGraph[i];
        if (q < A.nL0) continue;  // constant or PI
        const int g = A.wg[q];
        const int cpos = A.dg[g].cpos;
        EvalIn E = A.E;
        E.tab = table_region(A.tab, g);
        int bc = -1, bo = -1, gain = 0, level = 0;
        for (int k = 0; k < 8; k++) {
            const uint32_t pk = (uint32_t)A.cutM[q * 8 + k].y;
            if (!packed_used(pk) || packed_nleaves(pk) < 3) continue;
            const CutBest b =
                eval_cut(E, (int)q, cpos, pk, A.cutL[q * 8 + k], A.useZeros != 0, match, mlev, kEvalBlock);
            fold_cut_best(b, k, bc, bo, gain, level);
        }
        A.bestCut[q] = (int8_t)bc;
        A.bestOut[q] = (uint8_t)(bo < 0 ? 0 : bo);
        A.candFlag[q] = bc >= 0;
    }
}

}  // namespace

int rw_evaluate(ExecCtx &X, RwWork &w, const Batch &b) {
    const int64_t N = w.N;
    cudaStream_t s = X.s;
    int64_t nAnd = N - w.nL0;
    // region of graph g: 2 * its AND count + 8 slots (load factor <= 1/2)
    std::vector<int64_t> off(w.G + 1);
    off[0] = 0;
    for (int g = 0; g < w.G; g++) off[g + 1] = off[g] + 2 * (int64_t)b.hg[g].nAnds + 8;
    const int64_t nSlots = off[w.G];
    TabSlot *slots = X.ar->get<TabSlot>(nSlots);
    int64_t *dOff = X.ar->get<int64_t>(w.G + 1);
    w.bestCut = X.ar->get<int8_t>(N);
    w.bestOut = X.ar->get<uint8_t>(N);
    uint8_t *candFlag = X.ar->get<uint8_t>(N);
    w.cand = X.ar->get<int>(N);
    if (!slots || !dOff || !w.bestCut || !w.bestOut || !candFlag || !w.cand)
        return X.fail(CULS_E_OOM, "rw: scratch arena exhausted (table)");
    w.tab = RegionTable{slots, dOff};
    int rc;
    if ((rc = X.check(cudaMemcpyAsync(dOff, off.data(), sizeof(int64_t) * (w.G + 1), cudaMemcpyHostToDevice, s),
                      "h2d")))
        return rc;
    if ((rc = X.check(cudaMemsetAsync(w.bestCut, 0xFF, N, s), "memset"))) return rc;
    if ((rc = X.check(cudaMemsetAsync(candFlag, 0, N, s), "memset"))) return rc;
    if (nAnd > 0) {
        k_table_clear<<<X.grid(nSlots), kBlock, 0, s>>>(nSlots, slots);
        k_table_build<<<X.grid(N), kBlock, 0, s>>>(w.nL0, N, w.byGraph, w.w0, w.w1, w.wg, w.wlev, w.dg, w.tab,
                                                   X.status);
        EvalArgs A{w.nL0, N, w.byGraph, EvalIn{w.w0, w.w1, w.ref, w.wlev, X.lib, TabRegion{}, X.status}, w.tab,
                   w.cutL, w.cutM, w.wg, w.dg, w.useZeros ? 1 : 0, w.bestCut, w.bestOut, candFlag};
        X.mark(kMkEvalK0);
        k_evaluate<<<X.grid(N, kEvalBlock), kEvalBlock, 0, s>>>(A);
        X.mark(kMkEvalK1);
        X.launched(3);
    }
    if ((rc = X.check(compact_flags(candFlag, N, w.cand, X.counters + 8, *X.ar, s), "compact"))) return rc;
    if ((rc = X.check(cudaMemcpyAsync(X.hostSmall + 8, X.counters + 8, sizeof(int), cudaMemcpyDeviceToHost, s), "d2h")))
        return rc;
    if ((rc = X.sync())) return rc;
    if ((rc = X.status_check("rw evaluate"))) return rc;
    w.nCand = X.hostSmall[8];
    return 0;
}

}  // namespace culs
