// Conflict-free replacement and redundancy removal: the sequential choice
// loop of rw::CPUSolver::Rewrite (CULS src/algorithms/rewrite.cu:830-921,
// rewrite.h:118-124,208-220) moved onto the GPU.
//
// Choice: one thread per graph walks that graph's candidates in id order and
// replays install / FastDelete with explicit stacks that follow the
// reference's recursion step by step (FastDelete's order of reference-count
// updates matters when a cone reaches a node along two paths).  The walk is
// a chain of dependent memory accesses, so it is written to shorten that
// chain: each candidate's record (node, replacement, cut leaves) is gathered
// beforehand in graph order and read one candidate ahead; the loads a
// candidate needs before its first store are issued together; a traversal
// frame carries its node's two fanins, the top frame lives in registers and
// the next ones in shared memory; reference-count updates whose old value is
// not needed are fire-and-forget atomics (a thread's own later loads of the
// same word observe them).
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

constexpr int kChoiceBlock = 32;   // graphs per block, one thread each
constexpr int kChoiceFrames = 64;  // frames per graph held in shared memory

struct ChoiceArgs {
    int64_t nL0;  // W positions [0, nL0) are constants and PIs
    const DevGraph *dg;
    int *L0, *L1, *ref;
    uint8_t *del;
    const int4 *recA, *recB;  // per candidate in graph order: {c, q, rep, -}, leaves
    const int *gStart, *gCount;
    int useZeros;
    int4 *stack;
    int stackCap;
    int *choice;
    unsigned long long *stats;  // replaced, pos, zero, reverted, compromised, newIdx, selfRef, expected
    int *status;
};

// frame {node, step | count << 2, fanin0 literal, fanin1 literal}; frames
// below kChoiceFrames in shared memory, deeper ones in the graph's global
// stack
struct GraphCtx {
    const ChoiceArgs *A;
    int trueLit;
    int4 (*sh)[kChoiceBlock];
    int lane;
    int4 *stk;
    __device__ __forceinline__ void push(int sp, int4 f) const {
        if (sp < kChoiceFrames)
            sh[sp][lane] = f;
        else
            stk[sp] = f;
    }
    __device__ __forceinline__ int4 pop(int sp) const { return sp < kChoiceFrames ? sh[sp][lane] : stk[sp]; }
};

__device__ __forceinline__ int ch_red(const GraphCtx &C, int x, int l0, int l1) {
    return x >= C.A->nL0 && (l0 == l1 || l0 == C.trueLit);
}
__device__ __forceinline__ void ref_add(int *ref, int x, int d) { atomicAdd(ref + x, d); }

// A pushed frame's two fanins are read together: their (del or ref, L0,
// L1).  L0 and L1 do not change during install / FastDelete, and del / ref
// of the second fanin change only inside the first fanin's subtree, so the
// second fanin is read again only when its frame resumes after that
// subtree.

// install lambda, rewrite.cu:835-847; rootDel, r0, r1 = del, L0, L1 of root
__device__ int ch_install(const GraphCtx &C, int root, int rootDel, int r0, int r1) {
    const ChoiceArgs &A = *C.A;
    if (!rootDel) return 0;
    A.del[root] = 0;
    int4 f = make_int4(root, (1 - ch_red(C, root, r0, r1)) << 2, r0, r1);
    int d0 = A.del[r0 >> 1], a0 = A.L0[r0 >> 1], b0 = A.L1[r0 >> 1];
    int d1 = A.del[r1 >> 1], a1 = A.L0[r1 >> 1], b1 = A.L1[r1 >> 1];
    int sp = 0;
    while (true) {
        const int step = f.y & 3;
        if (step < 2) {
            const int child = (step == 0 ? f.z : f.w) >> 1;
            const int d = step == 0 ? d0 : d1, c0 = step == 0 ? a0 : a1, c1 = step == 0 ? b0 : b1;
            f.y++;
            if (d) {
                if (sp + 1 >= A.stackCap) {
                    set_status(A.status, kDevStackOverflow);
                    return 0;
                }
                A.del[child] = 0;
                C.push(sp++, f);
                f = make_int4(child, (1 - ch_red(C, child, c0, c1)) << 2, c0, c1);
                d0 = A.del[c0 >> 1], a0 = A.L0[c0 >> 1], b0 = A.L1[c0 >> 1];
                d1 = A.del[c1 >> 1], a1 = A.L0[c1 >> 1], b1 = A.L1[c1 >> 1];
            }
            continue;
        }
        ref_add(A.ref, f.z >> 1, 1);
        ref_add(A.ref, f.w >> 1, 1);
        const int cnt = f.y >> 2;
        if (sp == 0) return cnt;
        f = C.pop(--sp);
        f.y += cnt << 2;
        if ((f.y & 3) == 1) {  // resumes at fanin 1 after fanin 0's subtree
            const int c = f.w >> 1;
            d1 = A.del[c], a1 = A.L0[c], b1 = A.L1[c];
        }
    }
}

// FastDelete's two reference-count decrements of a frame's fanins, whose
// returned values give the fanins' counts; L0 / L1 of both fanins
__device__ __forceinline__ void fd_open(const ChoiceArgs &A, int l0, int l1, int &v0, int &a0, int &b0, int &v1, int &a1,
                                        int &b1) {
    const int c0 = l0 >> 1, c1 = l1 >> 1;
    const int o0 = atomicAdd(A.ref + c0, -1);
    const int o1 = atomicAdd(A.ref + c1, -1);
    a0 = A.L0[c0], b0 = A.L1[c0], a1 = A.L0[c1], b1 = A.L1[c1];
    v1 = o1 - 1;
    v0 = c0 == c1 ? v1 : o0 - 1;  // one node twice: both decrements precede the first check
}

// FastDelete, rewrite.h:208-220; r0, r1 = L0, L1 of root
__device__ int ch_fast_delete(const GraphCtx &C, int root, int r0, int r1) {
    const ChoiceArgs &A = *C.A;
    if (root < A.nL0) return 0;
    int v0, a0, b0, v1, a1, b1;
    fd_open(A, r0, r1, v0, a0, b0, v1, a1, b1);
    int4 f = make_int4(root, 1 | ((1 - ch_red(C, root, r0, r1)) << 2), r0, r1);
    int sp = 0;
    while (true) {
        const int step = f.y & 3;
        if (step < 3) {
            const int child = (step == 1 ? f.z : f.w) >> 1;
            const int r = step == 1 ? v0 : v1, c0 = step == 1 ? a0 : a1, c1 = step == 1 ? b0 : b1;
            f.y++;
            if (r == 0 && child >= A.nL0) {
                if (sp + 1 >= A.stackCap) {
                    set_status(A.status, kDevStackOverflow);
                    return 0;
                }
                fd_open(A, c0, c1, v0, a0, b0, v1, a1, b1);
                C.push(sp++, f);
                f = make_int4(child, 1 | ((1 - ch_red(C, child, c0, c1)) << 2), c0, c1);
            }
            continue;
        }
        A.del[f.x] = 1;
        const int cnt = f.y >> 2;
        if (sp == 0) return cnt;
        f = C.pop(--sp);
        f.y += cnt << 2;
        if ((f.y & 3) == 2) {  // resumes at fanin 1 after fanin 0's subtree
            const int c = f.w >> 1;
            v1 = A.ref[c], a1 = A.L0[c], b1 = A.L1[c];
        }
    }
}

__global__ void __launch_bounds__(kChoiceBlock) k_choice(ChoiceArgs A, int G) {
    __shared__ int4 sh[kChoiceFrames][kChoiceBlock];
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
    const int cpos = A.dg[g].cpos;
    GraphCtx C{&A, 2 * cpos + 1, sh, (int)threadIdx.x, A.stack + (int64_t)g * A.stackCap};
    unsigned long long replaced = 0, pos = 0, zero = 0, reverted = 0, comp = 0, noRep = 0, selfRef = 0;
    long long expected = 0;
    int i = A.gStart[g];
    const int e = i + A.gCount[g];
    int4 na = make_int4(-1, -1, -1, -1), nb = na;
    if (i < e) {
        na = A.recA[i];
        nb = A.recB[i];
    }
    for (; i < e; i++) {
        const int4 a = na, lv = nb;
        if (i + 1 < e) {
            na = A.recA[i + 1];
            nb = A.recB[i + 1];
        }
        if (i + 1 < e && (na.z >> 1) >= 0) {
            // the next candidate's first loads, into L1 while this one runs
            // (a prefetch carries no value, so later stores cannot make it stale)
            const int nn = na.z >> 1, nq = na.y;
            asm volatile("prefetch.global.L1 [%0];" ::"l"(A.L0 + nn));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(A.L1 + nn));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(A.del + nn));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(A.L0 + nq));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(A.L1 + nq));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(A.del + nb.x));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(A.del + nb.y));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(A.del + nb.z));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(A.del + nb.w));
        }
        const int c = a.x, q = a.y, rep = a.z;
        const int newIdx = rep >> 1;
        if (newIdx < 0) {
            noRep++;
            A.choice[c] = kChNoReplace;
            continue;
        }
        // everything read before this candidate's first store
        const int n0 = A.L0[newIdx], n1 = A.L1[newIdx];
        const int dn = A.del[newIdx];
        const int dl = A.del[lv.x] | A.del[lv.y] | A.del[lv.z] | A.del[lv.w];
        const int q0 = A.L0[q], q1 = A.L1[q];
        if (newIdx == q || (n1 >> 1) == q) {
            selfRef++;
            A.choice[c] = kChSelfRef;
            continue;
        }
        if (dl) {
            comp++;
            A.choice[c] = kChCompromised;
            continue;
        }
        int added = ch_install(C, newIdx, dn, n0, n1);
        ref_add(A.ref, newIdx, 1);
        int saved = ch_fast_delete(C, q, q0, q1);
        ref_add(A.ref, newIdx, -1);
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
            ref_add(A.ref, cpos, 1);
            ref_add(A.ref, newIdx, 1);
            A.choice[c] = kChCommitted;
        } else {
            reverted++;
            ch_install(C, q, A.del[q], q0, q1);
            ref_add(A.ref, q, 1);
            if (A.ref[newIdx] == 0) ch_fast_delete(C, newIdx, n0, n1);
            ref_add(A.ref, q, -1);
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

// the choice's record of the i-th candidate in graph order: {c, q, rep, -}
// and the chosen cut's four leaves (the constant in the fourth place of a
// three-leaf cut); leaves are read only for candidates with a replacement
__global__ void k_cand_records(int64_t n, const int *candByG, const int *cand, const int *repW, const int8_t *bestCut,
                               const int4 *cutL, const int2 *cutM, const int *wg, const DevGraph *dg, int4 *recA,
                               int4 *recB) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int c = candByG[i];
        const int q = cand[c];
        const int rep = repW[c];
        int4 l = make_int4(0, 0, 0, 0);
        if ((rep >> 1) >= 0) {
            const int slot = bestCut[q];
            l = cutL[(int64_t)q * 8 + slot];
            if (packed_nleaves((uint32_t)cutM[(int64_t)q * 8 + slot].y) == 3) l.w = dg[wg[q]].cpos;
        }
        recA[i] = make_int4(c, q, rep, 0);
        recB[i] = l;
    }
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
    int4 *recA = ar.get<int4>(nCand + 1), *recB = ar.get<int4>(nCand + 1);
    w.choice = ar.get<int>(nCand + 1);
    unsigned long long *dstats = ar.get<unsigned long long>(8);
    // explicit recursion stacks: deep enough for any chain through the
    // levels plus the new nodes
    int64_t stackCap = (int64_t)w.maxLevel + 64;
    for (int g = 0; g < G; g++) stackCap = std::max<int64_t>(stackCap, 64);
    stackCap = std::min<int64_t>(2 * stackCap + w.nNew / std::max(G, 1) + 64, 1 << 20);
    int4 *stack = ar.get<int4>((size_t)stackCap * G);
    if (!gCount || !gStart || !candByG || !keys || !keys2 || !vals || !recA || !recB || !w.choice || !dstats || !stack)
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
        k_cand_records<<<X.grid(nCand), kBlock, 0, s>>>(nCand, candByG, w.cand, w.repW, w.bestCut, w.cutL, w.cutM, w.wg,
                                                        w.dg, recA, recB);
        X.launched(1);
    }
    if ((rc = X.check(scan_exclusive(gCount, gStart, G, nullptr, ar, s), "scan"))) return rc;
    ChoiceArgs A{w.nL0, w.dg,   w.L0,   w.L1,     w.ref,    w.del,       recA,   recB,  gStart,
                 gCount, w.useZeros ? 1 : 0,    stack,  (int)stackCap,       w.choice, dstats, X.status};
    // the walk's working set is the graph's fanins, flags and counts: the
    // smallest shared-memory carveout leaves the most L1 for it
    cudaFuncSetAttribute(k_choice, cudaFuncAttributePreferredSharedMemoryCarveout, 0);
    k_choice<<<(G + kChoiceBlock - 1) / kChoiceBlock, kChoiceBlock, 0, s>>>(A, G);
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

// per node, fixed during the sweeps
enum : uint8_t { kRdPi = 1, kRdDel = 2, kRdR0 = 4 };  // PI or constant; deleted; redundant before the sweep

struct RedArgs {
    int64_t M;
    const int *gidAll;
    const DevGraph *dg;
    const int *pre0, *pre1;
    const uint8_t *st;
    const int *postIn1;
    const uint8_t *nredIn;
    int *post1;
    uint8_t *nredOut;
    int *changed;
    int *status;
};

__global__ void k_red_state(int64_t M, int64_t nL0, const int *gidAll, const DevGraph *dg, const int *L0, const int *L1,
                            const uint8_t *del, uint8_t *st) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < M; x += stride) {
        if (x < nL0) {
            st[x] = kRdPi;
            continue;
        }
        const int a = L0[x];
        const bool r0 = a == L1[x] || a == 2 * dg[gidAll[x]].cpos + 1;
        st[x] = (uint8_t)((del[x] ? kRdDel : 0) | (r0 ? kRdR0 : 0));
    }
}

// Fanin() of rewrite.h:121-124 as seen by the sweep at node `time`
// (time = INT_MAX after the sweep).  A node is chased (its fanins are
// rewritten by the sweep) when it is no PI, not deleted and not redundant
// before the sweep: state byte 0.
__device__ int rd_chase(const RedArgs &A, int lit, int time) {
    int c = 0;
    for (int step = 0; step < (1 << 20); step++) {
        const int u = lit >> 1;
        const int s = A.st[u];
        if (s & kRdPi) return lit ^ c;
        const bool done = u < time && s == 0;
        const bool red = done ? A.nredIn[u] != 0 : (s & kRdR0) != 0;
        if (!red) return lit ^ c;
        c ^= lit & 1;
        lit = done ? A.postIn1[u] : A.pre1[u];
    }
    set_status(A.status, kDevBadGraph);
    return lit ^ c;
}

// one sweep over the chased nodes; the others keep their fanins and are
// never read as sweep state
__global__ void k_redundancy(RedArgs A) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < A.M; x += stride) {
        if (A.st[x]) continue;
        const int a = rd_chase(A, A.pre0[x], (int)x);
        const int b = rd_chase(A, A.pre1[x], (int)x);
        const int t = 2 * A.dg[A.gidAll[x]].cpos + 1;
        const uint8_t nr = (a == b || a == t) ? 1 : 0;
        if (nr != A.nredIn[x] || b != A.postIn1[x]) atomicExch(A.changed, 1);
        A.post1[x] = b;
        A.nredOut[x] = nr;
    }
}

// pre0 aliases L0 (each node reads and writes only its own entry); pre1 is a
// copy, since other nodes' chases read it
__global__ void k_redundancy_finish(RedArgs A, int *L0, int *L1, uint8_t *delOut, int64_t nPO, int *po) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < A.M; x += stride) {
        const int s = A.st[x];
        if (s == 0) {
            L0[x] = rd_chase(A, A.pre0[x], (int)x);
            L1[x] = A.postIn1[x];
        } else if (!(s & (kRdPi | kRdDel))) {
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
    int *pre1 = ar.get<int>(M);
    int *P1[2] = {ar.get<int>(M), ar.get<int>(M)};
    uint8_t *NR[2] = {ar.get<uint8_t>(M), ar.get<uint8_t>(M)};
    uint8_t *st = ar.get<uint8_t>(M);
    if (!pre1 || !P1[0] || !P1[1] || !NR[0] || !NR[1] || !st) return X.fail(CULS_E_OOM, "rw: arena exhausted (redundancy)");
    if ((rc = X.check(cudaMemcpyAsync(pre1, w.L1, sizeof(int) * M, cudaMemcpyDeviceToDevice, s), "copy"))) return rc;
    if ((rc = X.check(cudaMemsetAsync(NR[0], 0, M, s), "memset"))) return rc;
    k_red_state<<<X.grid(M), kBlock, 0, s>>>(M, w.nL0, w.gidAll, w.dg, w.L0, w.L1, w.del, st);
    X.launched(1);
    int *changed = X.counters + 24;
    // sweep state: (post1, nred) of the chased nodes; state 0 (no chase
    // yet) is (pre1, 0), read from pre1 itself
    const int *in1 = pre1;
    const uint8_t *inR = NR[0];
    int cur = 1;
    for (int it = 0;; it++) {
        if (it >= 64) return X.fail(CULS_E_INVALID, "rw: redundancy sweep did not converge");
        RedArgs A{M, w.gidAll, w.dg, w.L0, pre1, st, in1, inR, P1[cur], NR[cur], changed, X.status};
        if ((rc = X.check(cudaMemsetAsync(changed, 0, sizeof(int), s), "memset"))) return rc;
        k_redundancy<<<X.grid(M), kBlock, 0, s>>>(A);
        X.launched(1);
        if ((rc = X.check(cudaMemcpyAsync(X.hostSmall + 24, changed, sizeof(int), cudaMemcpyDeviceToHost, s), "d2h")))
            return rc;
        if ((rc = X.sync())) return rc;
        in1 = P1[cur];
        inR = NR[cur];
        cur ^= 1;
        if (!X.hostSmall[24]) break;
    }
    // (in1, inR) is a fix-point: sweeping it again reproduces it
    RedArgs F{M, w.gidAll, w.dg, w.L0, pre1, st, in1, inR, nullptr, nullptr, changed, X.status};
    k_redundancy_finish<<<X.grid(std::max<int64_t>(M, w.nPO)), kBlock, 0, s>>>(F, w.L0, w.L1, w.del, w.nPO, w.wpo);
    X.launched(1);
    if ((rc = X.sync())) return rc;
    return X.status_check("rw redundancy");
}

}  // namespace culs
