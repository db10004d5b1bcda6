// Existence table and per-node evaluation: BuildHashTable + EvaluateNode
// (CULS src/algorithms/rewrite.cu:378-471).  The chained table of the
// reference becomes an open-addressing table on 64-bit CAS keys (fanin0 id,
// fanin1 id, compl0, compl1) with one region per graph.  Both the build and
// the evaluation visit the nodes graph by graph (the front's byGraph order),
// so the region, cuts and fanin arrays a block touches belong to the few
// graphs in flight.
//
// Evaluation works on (node, cut) items grouped by NPN class per warp (see
// k_evaluate); the match/level scratch of a library walk lives in shared
// memory laid out entry-major, so lanes reading the same library entry hit
// distinct banks.
#include <algorithm>
#include <vector>

#include "rw_work.cuh"

namespace culs {

namespace {

constexpr int kEvalBlock = 64;
constexpr int kLibSlots = 54;  // 4 inputs + at most 50 library nodes
// Library scratch entries kept in shared memory per thread: forests of up to
// kLibFast - 4 nodes (every frequent class) evaluate there; larger ones use
// a per-thread column of a global scratch array.  The smaller shared
// footprint keeps 22 warps resident per SM instead of 16.
constexpr int kLibFast = 38;
constexpr int kClassSlots = 224;  // >= the library's 222 classes, a multiple of 32
static_assert(kClassSlots >= kNumClasses && kClassSlots % 32 == 0, "class slots");

__global__ void k_table_clear(int64_t n, TabSlot *slots) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        reinterpret_cast<int4 *>(slots)[i] = make_int4(-1, -1, 0x7FFFFFFF, 0);
}

// Inserts the AND nodes at graph-major indices [lo, hi) of byGraph.
__global__ void k_table_build(int64_t nL0, int64_t lo, int64_t hi, const int *byGraph, const int *w0, const int *w1,
                              const int *wg, const int *wlev, const DevGraph *dg, RegionTable tab, int *status) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = lo + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < hi; i += stride) {
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
    int64_t nL0, lo, hi;  // evaluates the nodes at graph-major indices [lo, hi) of byGraph
    const int *byGraph;
    int *scratch;  // 2 * kLibSlots ints per thread of the grid, thread-minor
    EvalIn E;
    RegionTable tab;
    const int4 *cutL;
    const int2 *cutM;
    const int *wg;
    const DevGraph *dg;
    int useZeros;
    int *mffcNodes;  // per warp of the grid, per item: up to 8 MFFC node positions
    int8_t *bestCut;
    uint8_t *bestOut;
    uint8_t *candFlag;
};

// Per-warp shared state of k_evaluate: the warp's nodes' evaluable cuts as
// items grouped by class slot, and one result per (node, cut slot).
// Nodes per lane in a warp's window: two (about 210 cut items to sort per
// warp instead of 105) fill rounds better but measured slower on the
// 4,096-graph batch.
constexpr int kNodesPerLane = 1;
constexpr int kWarpNodes = 32 * kNodesPerLane;
struct WarpItems {
    int off[kClassSlots];          // class-slot counts, then exclusive offsets
    uint16_t item[kWarpNodes * 8];  // local node * 8 + cut slot, in class-slot order
    int2 res[kWarpNodes * 8];       // {gain * 16 + root index, level} or {-1, 0}
    uint16_t full[kWarpNodes * 8];  // items whose MFFC needs the full traversal
    uint8_t saved[kWarpNodes * 8];  // per item: CalcMFFC's count
    uint8_t nDel[kWarpNodes * 8];   // per item: its MFFC nodes (in EvalArgs::mffcNodes)
};

// A warp takes 32 * kNodesPerLane consecutive nodes of the graph-major
// order, sorts their evaluable cuts by NPN class -- classes ordered by their
// forests' batch counts -- and evaluates them 32 at a time, so the lanes of
// a round mostly walk the same library forest, or forests of as many
// batches (the forests' sizes differ several-fold between classes).  Each
// lane then folds its own nodes' results in slot order, the order of the
// reference's loop.  Warps never wait for one another.  LevT is the type of
// the library-node levels in the scratch (16-bit when the graph is shallow
// enough, which halves that part of the shared memory).
template <class LevT>
__global__ void __launch_bounds__(kEvalBlock, 8) k_evaluate(EvalArgs A) {
    __shared__ int s_match[kLibFast * kEvalBlock];
    __shared__ LevT s_mlev[kLibFast * kEvalBlock];
    __shared__ WarpItems s_w[kEvalBlock / 32];
    int *match = s_match + threadIdx.x;
    LevT *mlev = s_mlev + threadIdx.x;
    const int lane = threadIdx.x & 31;
    WarpItems &W = s_w[threadIdx.x >> 5];
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int gstride = gridDim.x * blockDim.x;
    int *gmatch = A.scratch + gtid;
    LevT *gmlev = reinterpret_cast<LevT *>(A.scratch + (int64_t)kLibSlots * gstride) + gtid;
    const int64_t nWarpChunks = (A.hi - A.lo + kWarpNodes - 1) / kWarpNodes;
    const int64_t warpStride = (int64_t)gridDim.x * (kEvalBlock / 32);
    for (int64_t wc = (int64_t)blockIdx.x * (kEvalBlock / 32) + (threadIdx.x >> 5); wc < nWarpChunks;
         wc += warpStride) {
        const int64_t base = A.lo + wc * kWarpNodes;
        for (int c = lane; c < kClassSlots; c += 32) W.off[c] = 0;
        __syncwarp();
        // 1. this lane's nodes: their evaluable cuts and class slots
        int64_t q[kNodesPerLane];
        uint32_t clsRank[kNodesPerLane][8];
#pragma unroll
        for (int h = 0; h < kNodesPerLane; h++) {
            const int local = h * 32 + lane;
            q[h] = -1;
            if (base + local < A.hi) {
                q[h] = A.byGraph[base + local];
                if (q[h] < A.nL0) q[h] = -1;  // constant or PI
            }
#pragma unroll
            for (int k = 0; k < 8; k++) {
                clsRank[h][k] = 0xFFFFFFFFu;
                W.res[local * 8 + k] = make_int2(-1, 0);
                if (q[h] >= 0) {
                    const uint32_t pk = (uint32_t)A.cutM[q[h] * 8 + k].y;
                    if (packed_used(pk) && packed_nleaves(pk) >= 3) {
                        const int cs = A.E.lib->classSlot[npn_class(A.E.lib->npn[pk & 0xFFFFu])];
                        clsRank[h][k] = ((uint32_t)cs << 16) | (uint32_t)atomicAdd(&W.off[cs], 1);
                    }
                }
            }
        }
        __syncwarp();
        // 2. exclusive scan of the class-slot counts, kClassSlots / 32 per lane
        int v[kClassSlots / 32], sum = 0;
#pragma unroll
        for (int t = 0; t < kClassSlots / 32; t++) {
            v[t] = W.off[lane * (kClassSlots / 32) + t];
            sum += v[t];
        }
        int inc = sum;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, inc, d);
            if (lane >= d) inc += y;
        }
        const int nItems = __shfl_sync(0xffffffffu, inc, 31);
        int run = inc - sum;
        __syncwarp();
#pragma unroll
        for (int t = 0; t < kClassSlots / 32; t++) {
            W.off[lane * (kClassSlots / 32) + t] = run;
            run += v[t];
        }
        __syncwarp();
#pragma unroll
        for (int h = 0; h < kNodesPerLane; h++)
#pragma unroll
            for (int k = 0; k < 8; k++)
                if (clsRank[h][k] != 0xFFFFFFFFu)
                    W.item[W.off[clsRank[h][k] >> 16] + (clsRank[h][k] & 0xFFFFu)] =
                        (uint16_t)((h * 32 + lane) * 8 + k);
        __syncwarp();
        // 3. every item's MFFC: the trivial ones (the root alone, nothing
        // deleted) at once, the others gathered and traversed 32 at a time,
        // so the traversal runs in full rounds instead of in every round
        int *const mffcNodes =
            A.mffcNodes + ((int64_t)blockIdx.x * (kEvalBlock / 32) + (threadIdx.x >> 5)) * (kWarpNodes * 8 * 8);
        int nFull = 0;
        for (int it0 = 0; it0 < nItems; it0 += 32) {
            const int it = it0 + lane;
            bool full = false;
            if (it < nItems) {
                const int slot = W.item[it];
                const int qq = A.byGraph[base + (slot >> 3)];
                const int64_t idx = (int64_t)qq * 8 + (slot & 7);
                const int4 l = A.cutL[idx];
                const int leaves[4] = {l.x, l.y, l.z,
                                       packed_nleaves((uint32_t)A.cutM[idx].y) == 3 ? A.dg[A.wg[qq]].cpos : l.w};
                full = !mffc_trivial(A.E, qq, leaves);
                W.saved[it] = 1;
                W.nDel[it] = 0;
            }
            const unsigned b = __ballot_sync(0xffffffffu, full);
            if (full) W.full[nFull + __popc(b & ((1u << lane) - 1u))] = (uint16_t)it;
            nFull += __popc(b);
        }
        __syncwarp();
        for (int k = lane; k < nFull; k += 32) {
            const int it = W.full[k];
            const int slot = W.item[it];
            const int qq = A.byGraph[base + (slot >> 3)];
            const int64_t idx = (int64_t)qq * 8 + (slot & 7);
            const int4 l = A.cutL[idx];
            const int leaves[4] = {l.x, l.y, l.z,
                                   packed_nleaves((uint32_t)A.cutM[idx].y) == 3 ? A.dg[A.wg[qq]].cpos : l.w};
            MffcTab tab;
            tab.size = 0;
            const int saved = mffc_size(A.E, qq, leaves, tab);
            const uint32_t zero = mffc_zero_mask(tab);
            int *del = mffcNodes + it * 8;
            int n = 0;
#define CULS_KEEP(k)             \
    if ((zero >> k) & 1u) del[n++] = tab.id[k];
            CULS_EACH8(CULS_KEEP)
#undef CULS_KEEP
            W.saved[it] = (uint8_t)saved;
            W.nDel[it] = (uint8_t)n;
        }
        __syncwarp();
        // 4. evaluate the items, 32 per round, in class-slot order
        for (int it = lane; it < nItems; it += 32) {
            const int slot = W.item[it];
            const int qq = A.byGraph[base + (slot >> 3)];
            const int g = A.wg[qq];
            EvalIn E = A.E;
            E.tab = table_region(A.tab, g);
            const int64_t idx = (int64_t)qq * 8 + (slot & 7);
            const uint32_t pk = (uint32_t)A.cutM[idx].y;
            const int4 l = A.cutL[idx];
            const int cpos = A.dg[g].cpos;
            CutBest b;
            const int saved = W.saved[it], nDel = W.nDel[it];
            const int *del = mffcNodes + it * 8;
            if (4 + A.E.lib->nNodes[npn_class(A.E.lib->npn[pk & 0xFFFFu])] <= kLibFast)
                b = eval_cut(E, qq, cpos, pk, l, A.useZeros != 0, match, mlev, kEvalBlock, saved, nDel, del);
            else  // a large forest: scratch in global memory
                b = eval_cut(E, qq, cpos, pk, l, A.useZeros != 0, gmatch, gmlev, gstride, saved, nDel, del);
            if (b.out >= 0) W.res[slot] = make_int2(b.gain * 16 + b.out, b.level);
        }
        __syncwarp();
        // 5. fold each of this lane's nodes' cuts in slot order
#pragma unroll
        for (int h = 0; h < kNodesPerLane; h++) {
            if (q[h] < 0) continue;
            const int local = h * 32 + lane;
            int bc = -1, bo = -1, gain = 0, level = 0;
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const int2 r = W.res[local * 8 + k];
                if (r.x >= 0) fold_cut_best(CutBest{r.x >> 4, r.y, r.x & 15}, k, bc, bo, gain, level);
            }
            A.bestCut[q[h]] = (int8_t)bc;
            A.bestOut[q[h]] = (uint8_t)(bo < 0 ? 0 : bo);
            A.candFlag[q[h]] = bc >= 0;
        }
        __syncwarp();
    }
}

}  // namespace

int rw_evaluate(ExecCtx &X, RwWork &w, const Batch &b) {
    const int64_t N = w.N;
    cudaStream_t s = X.s;
    int64_t nAnd = N - w.nL0;
    // region of graph g: 4 * its AND count + 8 slots.  At load factor <= 1/4
    // a linear probe ends in its home slot for ~80% of misses and ~90% of
    // hits (at 1/2 a miss scans 2.5 slots on average), and every extra slot
    // is a dependent load the whole warp waits for.
    std::vector<int64_t> off(w.G + 1);
    off[0] = 0;
    for (int g = 0; g < w.G; g++) off[g + 1] = off[g] + 4 * (int64_t)b.hg[g].nAnds + 8;
    const int64_t nSlots = off[w.G];
    TabSlot *slots = X.ar->get<TabSlot>(nSlots);
    int64_t *dOff = X.ar->get<int64_t>(w.G + 1);
    w.bestCut = X.ar->get<int8_t>(N);
    w.bestOut = X.ar->get<uint8_t>(N);
    uint8_t *candFlag = X.ar->get<uint8_t>(N);
    w.cand = X.ar->get<int>(N);
    // one resident wave: 8 blocks an SM (registers and shared memory); a
    // second wave of a grid-stride kernel would only start as the first ends
    const unsigned evalGrid = grid_1d(N, kEvalBlock, X.sms * 8);
    int *scratch = X.ar->get<int>((size_t)2 * kLibSlots * evalGrid * kEvalBlock);
    int *mffcNodes = X.ar->get<int>((size_t)evalGrid * (kEvalBlock / 32) * kWarpNodes * 8 * 8);
    if (!slots || !dOff || !w.bestCut || !w.bestOut || !candFlag || !w.cand || !scratch || !mffcNodes)
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
        X.mark(kMkEvalK0);
        // Graphs in groups of at most kGroupSlots table slots (16M by
        // default: 256 MB of regions; a tuned parameter), each group's
        // regions built right before its nodes are evaluated, so the probes
        // find them in L2 instead of DRAM (a single larger graph is a group
        // of its own).
        const int64_t kGroupSlots = (int64_t)X.tune->evalGroupMSlots << 20;
        const bool lev16 = w.maxLevel + 64 < 0xFFFF;  // see the launch below
        int g0 = 0;
        while (g0 < w.G) {
            int g1 = g0 + 1;
            while (g1 < w.G && off[g1 + 1] - off[g0] <= kGroupSlots) g1++;
            const int64_t lo = b.hg[g0].base, hi = g1 < w.G ? (int64_t)b.hg[g1].base : N;
            k_table_build<<<X.grid(hi - lo), kBlock, 0, s>>>(w.nL0, lo, hi, w.byGraph, w.w0, w.w1, w.wg, w.wlev,
                                                             w.dg, w.tab, X.status);
            EvalArgs A{w.nL0,  lo,     hi,     w.byGraph, scratch,
                       EvalIn{w.w0, w.w1, w.ref, w.wlev, X.lib, TabRegion{}, X.status},
                       w.tab,  w.cutL, w.cutM, w.wg,      w.dg,
                       w.useZeros ? 1 : 0, mffcNodes, w.bestCut, w.bestOut, candFlag};
            const unsigned grid = std::min(evalGrid, X.grid(hi - lo, kEvalBlock));
            // 16-bit library levels when no level of the batch, plus a
            // forest's depth (at most 50 nodes), can reach 65,535
            if (lev16)
                k_evaluate<uint16_t><<<grid, kEvalBlock, 0, s>>>(A);
            else
                k_evaluate<int><<<grid, kEvalBlock, 0, s>>>(A);
            X.launched(2);
            g0 = g1;
        }
        X.mark(kMkEvalK1);
        X.launched(1);
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
