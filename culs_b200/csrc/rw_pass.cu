// Engine::rw -- AIGMan::rewrite (CULS src/aig_manager.cu:632-672): reset,
// rewrite and the deduplication through strash, every stage on the device.
#include <algorithm>
#include <vector>

#include "rw_work.cuh"

namespace culs {

namespace {

// AIGER -> AIGMan constant convention (processRwmanFanins/Outs,
// src/aig_manager.cu:405-430); constants and PIs become -1 for strash_core.
__global__ void k_rw_to_aigman(int64_t N, int64_t M, const int *wlev, const int *gidAll, const DevGraph *dg,
                               const int *L0, const int *L1, int *o0, int *o1, int64_t nPO, const int *po, int *opo) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < M; q += stride) {
        if (q < N && wlev[q] == 0) {
            o0[q] = o1[q] = -1;
            continue;
        }
        int cp = dg[gidAll[q]].cpos;
        int a = L0[q], b = L1[q];
        o0[q] = (a >> 1) == cp ? a ^ 1 : a;
        o1[q] = (b >> 1) == cp ? b ^ 1 : b;
    }
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nPO; k += stride) {
        int l = po[k];
        int cp = dg[gidAll[l >> 1]].cpos;
        opo[k] = (l >> 1) == cp ? l ^ 1 : l;
    }
}

// The deduplication's processing order over W positions [0, M): each
// level's original nodes in W order, then the new nodes whose owner
// candidate is on that level, in position order (new positions are numbered
// by owner, and owners in W order, so their owner levels never decrease).
// Original fanins are on lower levels; a new node's fanins are its owner's
// cut leaves, new nodes numbered before it, or existing nodes the
// replacement reused, which may lie on the owner's level or above; buffers
// left by the choice point at their replacement.  The order is thus
// topological up to those last two kinds of fanins, which the level pass
// resolves in later passes.
//   lvEnd[l]    = W positions on levels <= l
//   newStart[l] = new nodes whose owner is on a level < l
__global__ void k_level_ends(int64_t N, const int *wlev, int maxLevel, int *lvEnd) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += stride) {
        const int l = wlev[p];
        const int next = p + 1 < N ? wlev[p + 1] : maxLevel + 1;
        for (int k = l; k < next; k++) lvEnd[k] = (int)(p + 1);
    }
}

__global__ void k_new_starts(int64_t nNew, const int *ownLev, int maxLevel, int *newStart) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j <= nNew; j += stride) {
        const int prev = j > 0 ? ownLev[j - 1] : -1;
        const int cur = j < nNew ? ownLev[j] : maxLevel + 1;
        for (int k = prev + 1; k <= cur; k++) newStart[k] = (int)j;
    }
}

__global__ void k_proc_order(int64_t N, int64_t M, const int *wlev, const int *ownLev, const int *lvEnd,
                             const int *newStart, int *inv, int *posOf, int *status) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < M; x += stride) {
        const int64_t pos = x < N ? x + newStart[wlev[x]] : lvEnd[ownLev[x - N]] + (x - N);
        if (pos < 0 || pos >= M) {
            set_status(status, kDevBadGraph);
            continue;
        }
        inv[pos] = (int)x;
        posOf[x] = (int)pos;
    }
}

void canon_cut(int4 l, int2 m, int *q) {
    Cut c;
    cut_unpack((uint32_t)m.y, c);
    if (!c.used) {
        for (int k = 0; k < 9; k++) q[k] = 0;
        return;
    }
    int lv[4] = {l.x, l.y, l.z, l.w};
    q[0] = 1;
    q[1] = (int)c.nLeaves;
    for (int k = 0; k < 4; k++) q[2 + k] = k < (int)c.nLeaves ? lv[k] : 0;
    q[6] = (int)c.tt;
    q[7] = m.x;
    q[8] = (int)c.value;
}

}  // namespace

int Engine::rw(Batch &b, bool useZeros, bool gpuDedup, RwStats *stats, RwDump *dump) {
    if (stats) *stats = RwStats{};
    bool anyAnd = false;
    for (auto &g : b.hg) anyAnd |= g.nAnds > 0;
    if (!anyAnd) return 0;  // AIGMan::rewrite returns at once without AND nodes
    int rc;
    if (b.keep) {  // the previous command was a rewrite: no Reset (src/aig_manager.cu:654-655)
        b.restore_kept();
        if ((rc = check(cudaMemcpyAsync(b.dg, b.hg.data(), sizeof(DevGraph) * b.G, cudaMemcpyHostToDevice, s_),
                        "h2d")))
            return rc;
    }
    const int64_t N = b.nObj;
    if ((rc = ensure_arena((size_t)N * 640 + (size_t)b.nPO * 16 + ((size_t)256 << 20)))) return rc;
    ar_.reset();
    ExecCtx X = ctx();
    RwWork w;
    w.useZeros = useZeros;
    const bool wantDump = dump && dump->enabled && b.G == 1;
    X.mark(kMkRwStart);
    if ((rc = rw_front(X, b, w))) return rc;
    X.mark(kMkFront);
    if ((rc = rw_enumerate(X, w))) return rc;
    X.mark(kMkEnum);
    if ((rc = rw_evaluate(X, w, b))) return rc;
    X.mark(kMkEval);
    if (wantDump) {
        std::vector<int4> L(N * 8);
        std::vector<int2> Mt(N * 8);
        std::vector<int8_t> bc(N);
        std::vector<uint8_t> bo(N);
        dump->reorderF0.resize(N);
        dump->reorderF1.resize(N);
        dump->reorderOut.resize(b.nPO);
        cudaMemcpy(dump->reorderF0.data(), w.w0, sizeof(int) * N, cudaMemcpyDeviceToHost);
        cudaMemcpy(dump->reorderF1.data(), w.w1, sizeof(int) * N, cudaMemcpyDeviceToHost);
        if (b.nPO) cudaMemcpy(dump->reorderOut.data(), w.wpo, sizeof(int) * b.nPO, cudaMemcpyDeviceToHost);
        cudaMemcpy(L.data(), w.cutL, sizeof(int4) * N * 8, cudaMemcpyDeviceToHost);
        cudaMemcpy(Mt.data(), w.cutM, sizeof(int2) * N * 8, cudaMemcpyDeviceToHost);
        cudaMemcpy(bc.data(), w.bestCut, N, cudaMemcpyDeviceToHost);
        cudaMemcpy(bo.data(), w.bestOut, N, cudaMemcpyDeviceToHost);
        dump->cuts.assign(N * 8 * 9, 0);
        dump->selected.assign(N * 10, 0);
        for (int64_t q = 0; q < N; q++) {
            for (int k = 0; k < 8; k++) canon_cut(L[q * 8 + k], Mt[q * 8 + k], &dump->cuts[(q * 8 + k) * 9]);
            int *sel = &dump->selected[q * 10];
            if (bc[q] >= 0) {
                canon_cut(L[q * 8 + bc[q]], Mt[q * 8 + bc[q]], sel);
                sel[9] = bo[q];
            } else {
                sel[9] = -1;
            }
        }
    }
    if ((rc = rw_replace(X, b, w))) return rc;
    X.mark(kMkReplace);
    if (wantDump) {
        std::vector<int> cand(w.nCand), rep(w.nCand);
        if (w.nCand) {
            cudaMemcpy(cand.data(), w.cand, sizeof(int) * w.nCand, cudaMemcpyDeviceToHost);
            cudaMemcpy(rep.data(), w.repW, sizeof(int) * w.nCand, cudaMemcpyDeviceToHost);
        }
        dump->replace.assign(N, -1);
        for (int64_t c = 0; c < w.nCand; c++) dump->replace[cand[c]] = rep[c];
        dump->newF0.resize(w.nNew);
        dump->newF1.resize(w.nNew);
        if (w.nNew) {
            cudaMemcpy(dump->newF0.data(), w.L0 + N, sizeof(int) * w.nNew, cudaMemcpyDeviceToHost);
            cudaMemcpy(dump->newF1.data(), w.L1 + N, sizeof(int) * w.nNew, cudaMemcpyDeviceToHost);
        }
    }
    if ((rc = rw_choice(X, b, w, stats))) return rc;
    X.mark(kMkChoice);
    if (wantDump) {
        std::vector<int> cand(w.nCand), ch(w.nCand), lev(N);
        if (w.nCand) {
            cudaMemcpy(cand.data(), w.cand, sizeof(int) * w.nCand, cudaMemcpyDeviceToHost);
            cudaMemcpy(ch.data(), w.choice, sizeof(int) * w.nCand, cudaMemcpyDeviceToHost);
        }
        cudaMemcpy(lev.data(), w.wlev, sizeof(int) * N, cudaMemcpyDeviceToHost);
        dump->choice.assign(N, kChNotVisited);
        for (int64_t q = 0; q < N; q++)
            if (lev[q] > 0) dump->choice[q] = kChNoCut;
        for (int64_t c = 0; c < w.nCand; c++) dump->choice[cand[c]] = ch[c];
    }
    if ((rc = rw_redundancy(X, b, w))) return rc;
    X.mark(kMkRedund);
    const int64_t M = N + w.nNew;
    int *o0 = ar_.get<int>(M), *o1 = ar_.get<int>(M), *opo = ar_.get<int>(b.nPO + 1);
    if (!o0 || !o1 || !opo) return fail(CULS_E_OOM, "rw: arena exhausted (dedup)");
    k_rw_to_aigman<<<X.grid(std::max<int64_t>(M, b.nPO)), kBlock, 0, s_>>>(N, M, w.wlev, w.gidAll, w.dg, w.L0, w.L1, o0,
                                                                           o1, b.nPO, w.wpo, opo);
    launches_ += 1;
    int *procInv = ar_.get<int>(M + 1), *procPos = ar_.get<int>(M + 1);
    int *lvEnd = ar_.get<int>(w.maxLevel + 2), *newStart = ar_.get<int>(w.maxLevel + 3);
    if (!procInv || !procPos || !lvEnd || !newStart) return fail(CULS_E_OOM, "rw: arena exhausted (dedup)");
    if ((rc = check(fill_i32(procInv, -1, M, s_), "fill"))) return rc;
    k_level_ends<<<X.grid(N), kBlock, 0, s_>>>(N, w.wlev, w.maxLevel, lvEnd);
    k_new_starts<<<X.grid(w.nNew + 1), kBlock, 0, s_>>>(w.nNew, w.newOwnLev, w.maxLevel, newStart);
    k_proc_order<<<X.grid(M), kBlock, 0, s_>>>(N, M, w.wlev, w.newOwnLev, lvEnd, newStart, procInv, procPos, status_);
    launches_ += 3;
    if ((rc = X.sync()) || (rc = X.status_check("rw dedup order"))) return rc;
    if (gpuDedup) {
        // updateFromRewriteManager(2): GPU strash, which also ends the
        // rewrite manager's state (src/aig_manager.cu:523-546)
        rc = strash_core(b, M, o0, o1, w.gidAll, w.wl, opo, false, true, true, false, false, procInv, procPos);
        if (stats) stats->hashRounds = hashRounds_;
        b.keep = false;
    } else {
        // updateFromRewriteManager(1): the manager's graph (every node, in
        // its final Reorder numbering) is kept for a following rewrite, then
        // deduplicated in id order (src/aig_manager.cu:454-522)
        rc = strash_core(b, M, o0, o1, w.gidAll, w.wl, opo, false, false, false, false, true, procInv, procPos);
        if (!rc) rc = check(b.keep_current(s_), "keep");
        if (!rc) {
            rc = strash_batch(b, false, false, false);
            if (stats) stats->hashRounds = hashRounds_;
            b.keep = rc == 0;
        }
    }
    X.mark(kMkRwEnd);
    return rc;
}

}  // namespace culs
