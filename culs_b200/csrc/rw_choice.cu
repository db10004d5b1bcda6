// Conflict-free replacement and redundancy removal: the sequential choice
// loop of rw::CPUSolver::Rewrite (CULS src/algorithms/rewrite.cu:830-921,
// rewrite.h:118-124,208-220) moved onto the GPU.
//
// Choice: one thread per graph walks that graph's candidates in id order and
// replays install / FastDelete with explicit stacks that follow the
// reference's recursion step by step (FastDelete's order of reference-count
// updates matters when a cone reaches a node along two paths).
//
// Redundancy removal chases buffer chains.  The reference does it in one
// sequential sweep in which a node's fanins, once rewritten, can make it
// redundant for later nodes only.  Here every node computes its chased fanins
// in parallel, judging each node it passes "as of its own id"; the sweep is
// repeated until nothing changes, which reproduces the sequential result
// because a node's outcome depends only on nodes with smaller ids.
#include <algorithm>
#include <climits>

#include "rw_work.cuh"

namespace culs {

namespace {

struct ChoiceArgs {
    int64_t N;
    const int *wlev;
    const DevGraph *dg;
    int *L0, *L1, *ref;
    uint8_t *del;
    const int *cand, *candByG, *gStart, *gCount;
    const int8_t *bestCut;
    const int4 *cutL;
    const int2 *cutM;
    const int *repW;
    int useZeros;
    int4 *stack;
    int stackCap;
    int *choice;
    unsigned long long *stats;  // replaced, pos, zero, reverted, compromised, newIdx, selfRef, expected
    int *status;
};

struct GraphCtx {
    const ChoiceArgs *A;
    int trueLit;
    int4 *stk;
};

__device__ __forceinline__ bool ch_is_pi(const ChoiceArgs &A, int x) { return x < A.N && A.wlev[x] == 0; }
__device__ __forceinline__ int ch_red(const GraphCtx &C, int x) {
    const ChoiceArgs &A = *C.A;
    if (ch_is_pi(A, x)) return 0;
    int a = A.L0[x];
    return a == A.L1[x] || a == C.trueLit;
}

// install lambda, rewrite.cu:835-847
__device__ int ch_install(const GraphCtx &C, int root) {
    const ChoiceArgs &A = *C.A;
    if (!A.del[root]) return 0;
    int sp = 0;
    A.del[root] = 0;
    C.stk[0] = make_int4(root, 0, 1 - ch_red(C, root), 0);
    while (true) {
        int4 F = C.stk[sp];
        if (F.y < 2) {
            int child = (F.y == 0 ? A.L0[F.x] : A.L1[F.x]) >> 1;
            F.y++;
            C.stk[sp] = F;
            if (A.del[child]) {
                if (sp + 1 >= A.stackCap) {
                    set_status(A.status, kDevStackOverflow);
                    return 0;
                }
                A.del[child] = 0;
                C.stk[++sp] = make_int4(child, 0, 1 - ch_red(C, child), 0);
            }
            continue;
        }
        A.ref[A.L0[F.x] >> 1]++;
        A.ref[A.L1[F.x] >> 1]++;
        if (sp == 0) return F.z;
        sp--;
        C.stk[sp].z += F.z;
    }
}

// FastDelete, rewrite.h:208-220
__device__ int ch_fast_delete(const GraphCtx &C, int root) {
    const ChoiceArgs &A = *C.A;
    if (ch_is_pi(A, root)) return 0;
    int sp = 0;
    {
        A.ref[A.L0[root] >> 1]--;
        A.ref[A.L1[root] >> 1]--;
        C.stk[0] = make_int4(root, 1, 1 - ch_red(C, root), 0);
    }
    while (true) {
        int4 F = C.stk[sp];
        if (F.y < 3) {
            int child = (F.y == 1 ? A.L0[F.x] : A.L1[F.x]) >> 1;
            F.y++;
            C.stk[sp] = F;
            if (A.ref[child] == 0 && !ch_is_pi(A, child)) {
                if (sp + 1 >= A.stackCap) {
                    set_status(A.status, kDevStackOverflow);
                    return 0;
                }
                A.ref[A.L0[child] >> 1]--;
                A.ref[A.L1[child] >> 1]--;
                C.stk[++sp] = make_int4(child, 1, 1 - ch_red(C, child), 0);
            }
            continue;
        }
        A.del[F.x] = 1;
        if (sp == 0) return F.z;
        sp--;
        C.stk[sp].z += F.z;
    }
}

__global__ void k_choice(ChoiceArgs A, int G) {
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
    const int cpos = A.dg[g].cpos;
    GraphCtx C{&A, 2 * cpos + 1, A.stack + (int64_t)g * A.stackCap};
    unsigned long long replaced = 0, pos = 0, zero = 0, reverted = 0, comp = 0, noRep = 0, selfRef = 0;
    long long expected = 0;
    const int e = A.gStart[g] + A.gCount[g];
    for (int i = A.gStart[g]; i < e; i++) {
        const int c = A.candByG[i];
        const int q = A.cand[c];
        const int rep = A.repW[c];
        const int newIdx = rep >> 1;
        if (newIdx < 0) {
            noRep++;
            A.choice[c] = kChNoReplace;
            continue;
        }
        if (newIdx == q || (A.L1[newIdx] >> 1) == q) {
            selfRef++;
            A.choice[c] = kChSelfRef;
            continue;
        }
        const int slot = A.bestCut[q];
        int4 l = A.cutL[(int64_t)q * 8 + slot];
        const int nl = (int)packed_nleaves((uint32_t)A.cutM[(int64_t)q * 8 + slot].y);
        int leaves[4] = {l.x, l.y, l.z, nl == 3 ? cpos : l.w};
        bool compromised = false;
        for (int j = 0; j < 4; j++) compromised |= A.del[leaves[j]] != 0;
        if (compromised) {
            comp++;
            A.choice[c] = kChCompromised;
            continue;
        }
        int added = ch_install(C, newIdx);
        A.ref[newIdx]++;
        int saved = ch_fast_delete(C, q);
        A.ref[newIdx]--;
        if (saved - added > 0 || (saved == added && A.useZeros)) {
            replaced++;
            if (saved - added > 0)
                pos++;
            else
                zero++;
            expected += saved - added;
            A.del[q] = 0;
            A.L0[q] = C.trueLit;
            A.L1[q] = rep;
            A.ref[cpos]++;
            A.ref[newIdx]++;
            A.choice[c] = kChCommitted;
        } else {
            reverted++;
            ch_install(C, q);
            A.ref[q]++;
            if (A.ref[newIdx] == 0) ch_fast_delete(C, newIdx);
            A.ref[q]--;
            A.choice[c] = kChReverted;
        }
    }
    atomicAdd(&A.stats[0], replaced);
    atomicAdd(&A.stats[1], pos);
    atomicAdd(&A.stats[2], zero);
    atomicAdd(&A.stats[3], reverted);
    atomicAdd(&A.stats[4], comp);
    atomicAdd(&A.stats[5], noRep);
    atomicAdd(&A.stats[6], selfRef);
    atomicAdd(&A.stats[7], (unsigned long long)expected);
}

__global__ void k_cand_gid(int64_t n, const int *cand, const int *wg, uint32_t *keys, int *vals, int *gCount) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += stride) {
        int g = wg[cand[c]];
        keys[c] = (uint32_t)g;
        vals[c] = (int)c;
        atomicAdd(&gCount[g], 1);
    }
}

}  // namespace

int rw_choice(ExecCtx &X, Batch &b, RwWork &w, RwStats *stats) {
    const int G = w.G;
    const int64_t nCand = w.nCand;
    cudaStream_t s = X.s;
    Arena &ar = *X.ar;
    int rc;
    int *gCount = ar.get<int>(G + 1), *gStart = ar.get<int>(G + 1), *candByG = ar.get<int>(nCand + 1);
    uint32_t *keys = ar.get<uint32_t>(nCand + 1), *keys2 = ar.get<uint32_t>(nCand + 1);
    int *vals = ar.get<int>(nCand + 1);
    w.choice = ar.get<int>(nCand + 1);
    unsigned long long *dstats = ar.get<unsigned long long>(8);
    // explicit recursion stacks: deep enough for any chain through the
    // levels plus the new nodes
    int64_t stackCap = (int64_t)w.maxLevel + 64;
    for (int g = 0; g < G; g++) stackCap = std::max<int64_t>(stackCap, 64);
    stackCap = std::min<int64_t>(2 * stackCap + w.nNew / std::max(G, 1) + 64, 1 << 20);
    int4 *stack = ar.get<int4>((size_t)stackCap * G);
    if (!gCount || !gStart || !candByG || !keys || !keys2 || !vals || !w.choice || !dstats || !stack)
        return X.fail(CULS_E_OOM, "rw: arena exhausted (choice)");
    if ((rc = X.check(cudaMemsetAsync(gCount, 0, sizeof(int) * (G + 1), s), "memset"))) return rc;
    if ((rc = X.check(cudaMemsetAsync(dstats, 0, sizeof(unsigned long long) * 8, s), "memset"))) return rc;
    if (nCand > 0) {
        k_cand_gid<<<X.grid(nCand), kBlock, 0, s>>>(nCand, w.cand, w.wg, keys, vals, gCount);
        X.launched(1);
        if (G > 1) {
            int bits = 1;
            while ((1ll << bits) < G) bits++;
            if ((rc = X.check(radix_sort_pairs(keys, vals, keys2, candByG, nCand, bits, ar, s), "sort"))) return rc;
        } else {
            if ((rc = X.check(iota_i32(candByG, 0, nCand, s), "iota"))) return rc;
        }
    }
    if ((rc = X.check(scan_exclusive(gCount, gStart, G, nullptr, ar, s), "scan"))) return rc;
    ChoiceArgs A{w.N,      w.wlev,  w.dg,       w.L0,   w.L1,   w.ref,       w.del,
                 w.cand,   candByG, gStart,     gCount, w.bestCut, w.cutL,   w.cutM,
                 w.repW,   w.useZeros ? 1 : 0,  stack,  (int)stackCap,       w.choice, dstats, X.status};
    k_choice<<<(G + 63) / 64, 64, 0, s>>>(A, G);
    X.launched(1);
    unsigned long long hs[8], warpPairs = 0;
    if ((rc = X.check(cudaMemcpyAsync(hs, dstats, sizeof hs, cudaMemcpyDeviceToHost, s), "d2h"))) return rc;
    if (w.warpPairs &&
        (rc = X.check(cudaMemcpyAsync(&warpPairs, w.warpPairs, sizeof warpPairs, cudaMemcpyDeviceToHost, s), "d2h")))
        return rc;
    if ((rc = X.sync())) return rc;
    if ((rc = X.status_check("rw choice"))) return rc;
    if (stats) {
        int64_t nAnd = w.N - w.nL0;
        stats->replaced = (long long)hs[0];
        stats->replacedPos = (long long)hs[1];
        stats->replacedZero = (long long)hs[2];
        stats->reverted = (long long)hs[3];
        stats->compromised = (long long)hs[4];
        stats->newIdx = (long long)hs[5];
        stats->expected = (long long)hs[7];
        stats->preEval = nAnd - nCand;
        stats->smallCut = 0;
        stats->newNodes = w.nNew;
        stats->candidates = nCand;
        stats->warpPairs = (long long)warpPairs;
    }
    (void)b;
    return 0;
}

namespace {

struct RedArgs {
    int64_t N, M;
    const int *wlev, *gidAll;
    const DevGraph *dg;
    const int *pre0, *pre1;
    const uint8_t *del;
    const int *postIn1;
    const uint8_t *nredIn;
    int *post0, *post1;
    uint8_t *nredOut;
    int *changed;
    int *status;
};

__device__ __forceinline__ bool rd_is_pi(const RedArgs &A, int x) { return x < A.N && A.wlev[x] == 0; }
__device__ __forceinline__ bool rd_r0(const RedArgs &A, int x) {
    if (rd_is_pi(A, x)) return false;
    int a = A.pre0[x];
    return a == A.pre1[x] || a == 2 * A.dg[A.gidAll[x]].cpos + 1;
}
__device__ __forceinline__ bool rd_chased(const RedArgs &A, int x) { return !rd_is_pi(A, x) && !A.del[x] && !rd_r0(A, x); }

// Fanin() of rewrite.h:121-124 as seen by the sweep at node `time`
// (time = INT_MAX after the sweep).
__device__ int rd_chase(const RedArgs &A, int lit, int time) {
    int c = 0;
    for (int step = 0; step < (1 << 20); step++) {
        int u = lit >> 1;
        if (rd_is_pi(A, u)) return lit ^ c;
        bool done = u < time && rd_chased(A, u);
        bool red = done ? A.nredIn[u] != 0 : rd_r0(A, u);
        if (!red) return lit ^ c;
        c ^= lit & 1;
        lit = done ? A.postIn1[u] : A.pre1[u];
    }
    set_status(A.status, kDevBadGraph);
    return lit ^ c;
}

__global__ void k_redundancy(RedArgs A) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < A.M; x += stride) {
        if (!rd_chased(A, (int)x)) {
            A.post0[x] = A.pre0[x];
            A.post1[x] = A.pre1[x];
            A.nredOut[x] = 0;
            continue;
        }
        int a = rd_chase(A, A.pre0[x], (int)x);
        int b = rd_chase(A, A.pre1[x], (int)x);
        int t = 2 * A.dg[A.gidAll[x]].cpos + 1;
        uint8_t nr = (a == b || a == t) ? 1 : 0;
        if (nr != A.nredIn[x] || b != A.postIn1[x]) atomicExch(A.changed, 1);
        A.post0[x] = a;
        A.post1[x] = b;
        A.nredOut[x] = nr;
    }
}

__global__ void k_redundancy_finish(RedArgs A, int *L0, int *L1, uint8_t *delOut, int64_t nPO, int *po) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < A.M; x += stride) {
        if (rd_chased(A, (int)x)) {
            L0[x] = A.post0[x];
            L1[x] = A.post1[x];
        } else if (!rd_is_pi(A, (int)x) && !A.del[x]) {
            delOut[x] = 1;  // redundant before the sweep: rewrite.cu:916-917
        }
    }
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nPO; k += stride) po[k] = rd_chase(A, po[k], INT_MAX);
}

}  // namespace

int rw_redundancy(ExecCtx &X, Batch &b, RwWork &w) {
    (void)b;
    const int64_t M = w.N + w.nNew;
    cudaStream_t s = X.s;
    Arena &ar = *X.ar;
    int rc;
    int *pre0 = ar.get<int>(M), *pre1 = ar.get<int>(M);
    int *P0[2] = {ar.get<int>(M), ar.get<int>(M)};
    int *P1[2] = {ar.get<int>(M), ar.get<int>(M)};
    uint8_t *NR[2] = {ar.get<uint8_t>(M), ar.get<uint8_t>(M)};
    uint8_t *del0 = ar.get<uint8_t>(M);
    if (!pre0 || !pre1 || !P0[0] || !P0[1] || !P1[0] || !P1[1] || !NR[0] || !NR[1] || !del0)
        return X.fail(CULS_E_OOM, "rw: arena exhausted (redundancy)");
    if ((rc = X.check(cudaMemcpyAsync(pre0, w.L0, sizeof(int) * M, cudaMemcpyDeviceToDevice, s), "copy"))) return rc;
    if ((rc = X.check(cudaMemcpyAsync(pre1, w.L1, sizeof(int) * M, cudaMemcpyDeviceToDevice, s), "copy"))) return rc;
    if ((rc = X.check(cudaMemcpyAsync(P1[0], w.L1, sizeof(int) * M, cudaMemcpyDeviceToDevice, s), "copy"))) return rc;
    if ((rc = X.check(cudaMemcpyAsync(del0, w.del, M, cudaMemcpyDeviceToDevice, s), "copy"))) return rc;
    if ((rc = X.check(cudaMemsetAsync(NR[0], 0, M, s), "memset"))) return rc;
    int *changed = X.counters + 24;
    // state k holds (post0, post1, nred) after sweep k; state 0 = no chase yet
    int cur = 0;
    for (int it = 0;; it++) {
        if (it >= 64) return X.fail(CULS_E_INVALID, "rw: redundancy sweep did not converge");
        int nxt = cur ^ 1;
        RedArgs A{w.N, M, w.wlev, w.gidAll, w.dg, pre0, pre1, del0, P1[cur], NR[cur], P0[nxt], P1[nxt], NR[nxt],
                  changed, X.status};
        if ((rc = X.check(cudaMemsetAsync(changed, 0, sizeof(int), s), "memset"))) return rc;
        k_redundancy<<<X.grid(M), kBlock, 0, s>>>(A);
        X.launched(1);
        if ((rc = X.check(cudaMemcpyAsync(X.hostSmall + 24, changed, sizeof(int), cudaMemcpyDeviceToHost, s), "d2h")))
            return rc;
        if ((rc = X.sync())) return rc;
        cur = nxt;
        if (!X.hostSmall[24]) break;
    }
    // state `cur` is a fix-point: sweeping it again reproduces it
    RedArgs F{w.N, M, w.wlev, w.gidAll, w.dg, pre0, pre1, del0, P1[cur], NR[cur], P0[cur], P1[cur], NR[cur], changed,
              X.status};
    k_redundancy_finish<<<X.grid(std::max<int64_t>(M, w.nPO)), kBlock, 0, s>>>(F, w.L0, w.L1, w.del, w.nPO, w.wpo);
    X.launched(1);
    if ((rc = X.sync())) return rc;
    return X.status_check("rw redundancy");
}

}  // namespace culs
