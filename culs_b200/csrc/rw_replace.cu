// Replacement subgraphs: ReplaceSubgr/BuildSubgr on the device plus the
// host-side DFS renumbering `rebuild` of GPUSolver::ReplaceSubgraphs (CULS
// src/algorithms/rewrite.cu:473-555,716-770), made deterministic and kept on
// the GPU.
//
// The reference builds new nodes with atomicAdd ids and deduplicates them in
// a second chained table.  Here, per candidate, the nodes BuildSubgr would
// visit are listed in its DFS post-order, so the id the sequential emulation
// (candidates in id order) would give each visited node is a prefix sum plus
// its post-order index.  Equal nodes are merged round by round in depth order
// through an atomicMin table, so every structural key keeps the smallest such
// id -- the node the sequential emulation creates first.  The rebuild's DFS
// numbering is reproduced from each new node's owner (the first candidate
// whose replacement cone contains it).
#include <algorithm>
#include <climits>

#include "rw_work.cuh"

namespace culs {

namespace {

struct RepArgs {
    int64_t N;
    const int *cand;
    const int8_t *bestCut;
    const uint8_t *bestOut;
    const int4 *cutL;
    const int2 *cutM;
    const int *wg;
    const DevGraph *dg;
    const RwLib *lib;
    RegionTable tab;
    const uint8_t *wph;
    int *status;
    // outputs
    int *kcnt;       // visited nodes per candidate (count pass)
    const int *koff; // prefix of kcnt (fill pass)
    int *recCand, *r0, *r1, *depth;
    uint8_t *rc0, *rc1;
    int *rootRef;  // per candidate: original position, -(T+1) for a built root, INT_MIN for none
    int *maxDepth;
};

// Recomputes the match of ReplaceSubgr for candidate c and walks BuildSubgr's
// visit order.  With fill == false only the count is written.
__device__ void rep_candidate(const RepArgs &A, int c, bool fill) {
    const int q = A.cand[c];
    const int slot = A.bestCut[q];
    const int g = A.wg[q];
    const int cpos = A.dg[g].cpos;
    const TabRegion T = table_region(A.tab, g);
    int4 l = A.cutL[(int64_t)q * 8 + slot];
    Cut cut;
    cut_unpack((uint32_t)A.cutM[(int64_t)q * 8 + slot].y, cut);
    int leaves[4] = {l.x, l.y, l.z, cut.nLeaves == 3 ? cpos : l.w};
    uint32_t npn = A.lib->npn[cut.tt];
    int uPhase = npn_phase(npn), cls = npn_class(npn);
    const uint8_t *perm = A.lib->perm4[npn_perm(npn)];
    int match[54];
    int isC = 0;
    for (int j = 0; j < 54; j++) match[j] = -1;
    for (int j = 0; j < 4; j++) {
        match[j] = leaves[perm[j]];
        if (uPhase >> j & 1) isC |= 1 << j;
    }
    const int rt = A.lib->roots[cls][A.bestOut[q]];
    uint64_t used = 1ull << rt;
    for (int j = rt; j >= 4; j--)
        if ((used >> j) & 1ull) {
            uint32_t w = A.lib->node[cls][j - 4];
            used |= 1ull << ln_f0(w);
            used |= 1ull << ln_f1(w);
        }
    const int nn = A.lib->nNodes[cls];
    for (int j = 0; j < nn; j++) {
        if (!((used >> (j + 4)) & 1ull)) continue;
        uint32_t w = A.lib->node[cls][j];
        int in0 = ln_f0(w), in1 = ln_f1(w);
        if (match[in0] == -1 || match[in1] == -1) continue;
        int cc0 = (in0 < 4 ? ((isC >> in0) & 1) : 0) ^ ln_c0(w);
        int cc1 = (in1 < 4 ? ((isC >> in1) & 1) : 0) ^ ln_c1(w);
        int id = region_and_lookup(T, match[in0], match[in1], cc0, cc1, A.status);
        if (id != -1) match[j + 4] = id;
    }
    if (match[rt] == q) {  // the whole subgraph exists already: no replacement
        if (fill)
            A.rootRef[c] = INT_MIN;
        else
            A.kcnt[c] = 0;
        return;
    }
    // BuildSubgr visit order: post-order over library nodes still unmatched;
    // a built node's match becomes -(2 + post-order index).
    int stk[56], st[56];
    int depth[54];
    int sp = 0, nb = 0;
    const int T0 = fill ? A.koff[c] : 0;
    stk[0] = rt;
    st[0] = 0;
    while (sp >= 0) {
        int cur = stk[sp];
        if (st[sp] == 0) {
            if (match[cur] != -1) {
                sp--;
                continue;
            }
            st[sp] = 1;
            stk[sp + 1] = ln_f0(A.lib->node[cls][cur - 4]);
            st[sp + 1] = 0;
            sp++;
            continue;
        }
        if (st[sp] == 1) {
            st[sp] = 2;
            stk[sp + 1] = ln_f1(A.lib->node[cls][cur - 4]);
            st[sp + 1] = 0;
            sp++;
            continue;
        }
        // build cur
        uint32_t w = A.lib->node[cls][cur - 4];
        int in0 = ln_f0(w), in1 = ln_f1(w);
        int idx = nb++;
        match[cur] = -(2 + idx);
        if (fill) {
            int T = T0 + idx;
            int m0 = match[in0], m1 = match[in1];
            int d0 = m0 <= -2 ? depth[-m0 - 2] : 0;
            int d1 = m1 <= -2 ? depth[-m1 - 2] : 0;
            depth[idx] = 1 + (d0 > d1 ? d0 : d1);
            A.recCand[T] = c;
            A.r0[T] = m0 >= 0 ? m0 : -(T0 + (-m0 - 2)) - 1;
            A.r1[T] = m1 >= 0 ? m1 : -(T0 + (-m1 - 2)) - 1;
            A.rc0[T] = (uint8_t)((in0 < 4 ? ((isC >> in0) & 1) : 0) ^ ln_c0(w));
            A.rc1[T] = (uint8_t)((in1 < 4 ? ((isC >> in1) & 1) : 0) ^ ln_c1(w));
            A.depth[T] = depth[idx];
            atomicMax(A.maxDepth, depth[idx]);
        }
        sp--;
    }
    if (fill) {
        int m = match[rt];
        A.rootRef[c] = m >= 0 ? m : -(T0 + (-m - 2)) - 1;
    } else {
        A.kcnt[c] = nb;
    }
}

__global__ void k_rep_count(int64_t nCand, RepArgs A) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nCand; c += stride) rep_candidate(A, (int)c, false);
}

__global__ void k_rep_fill(int64_t nCand, RepArgs A) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nCand; c += stride) rep_candidate(A, (int)c, true);
}

struct MergeArgs {
    int64_t N, K;
    const int *r0, *r1, *depth;
    const uint8_t *rc0, *rc1;
    const uint8_t *wph;
    int *canon;  // canonical T of each T (min T with the same key)
    uint8_t *nph;
    int *f0, *f1;  // resolved, oriented fanins (position space: < N original, N + C new)
    uint8_t *c0, *c1;
    int *slot;
    AndTable tab;
    int *status;
};

__device__ __forceinline__ int rep_resolve(const MergeArgs &A, int r) {
    return r >= 0 ? r : (int)A.N + A.canon[-r - 1];
}
__device__ __forceinline__ int rep_phase(const MergeArgs &A, int f) {
    return f < A.N ? A.wph[f] : A.nph[f - A.N];
}

// Round d: nodes of depth d have all children canonical.  BuildSubgr's
// orientation (rewrite.cu:491-498) compares the children's ids.
__global__ void k_rep_insert(int d, MergeArgs A) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t T = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; T < A.K; T += stride) {
        if (A.depth[T] != d) continue;
        int f0 = rep_resolve(A, A.r0[T]), f1 = rep_resolve(A, A.r1[T]);
        int c0 = A.rc0[T], c1 = A.rc1[T];
        A.nph[T] = (uint8_t)((rep_phase(A, f0) ^ c0) & (rep_phase(A, f1) ^ c1));
        if (f0 > f1) {
            int x = f0;
            f0 = f1;
            f1 = x;
            x = c0;
            c0 = c1;
            c1 = x;
        }
        A.f0[T] = f0;
        A.f1[T] = f1;
        A.c0[T] = (uint8_t)c0;
        A.c1[T] = (uint8_t)c1;
        A.slot[T] = table_insert(A.tab, and_key(f0, f1, c0, c1), (int)T, (int)T, A.status);
    }
}

__global__ void k_rep_canon(int d, MergeArgs A) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t T = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; T < A.K; T += stride) {
        if (A.depth[T] != d) continue;
        int sl = A.slot[T];
        A.canon[T] = sl >= 0 ? slot_rank(A.tab.slots[sl].rp) : (int)T;
    }
}

// replace[] before renumbering: literal over position space.
__global__ void k_rep_root(int64_t nCand, int64_t N, const int *cand, const int *rootRef, const int *canon,
                           const uint8_t *nph, const uint8_t *wph, int *repT) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nCand; c += stride) {
        int r = rootRef[c];
        int q = cand[c];
        if (r == INT_MIN) {
            repT[c] = -1;
        } else if (r >= 0) {
            repT[c] = 2 * r + (wph[r] ^ wph[q]);
        } else {
            int C = canon[-r - 1];
            repT[c] = 2 * ((int)N + C) + (nph[C] ^ wph[q]);
        }
    }
}

__global__ void k_rep_owner(int64_t K, const int *recCand, const int *canon, int *owner) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t T = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; T < K; T += stride)
        atomicMin(&owner[canon[T]], recCand[T]);
}

// The rebuild lambda of ReplaceSubgraphs (rewrite.cu:743-762) numbers new
// nodes in DFS post-order, fanin0 first, candidates in id order, skipping
// nodes numbered earlier.  Candidate c numbers exactly the nodes of its cone
// whose owner is c, in the same post-order.  With newPos == nullptr only the
// count is returned.
__device__ int rep_rebuild_dfs(int c, int rootX, int64_t N, const int *f0, const int *f1, const int *owner,
                               int *newPos, int posBase, int *status) {
    int vis[64], nv = 0;
    int stk[64], st[64];
    int sp = 0, idx = 0;
    if (owner[rootX] != c) return 0;
    stk[0] = rootX;
    st[0] = 0;
    vis[nv++] = rootX;
    while (sp >= 0) {
        int X = stk[sp];
        if (st[sp] < 2) {
            int f = st[sp] == 0 ? f0[X] : f1[X];
            st[sp]++;
            if (f < N) continue;
            int Y = f - (int)N;
            if (owner[Y] != c) continue;
            bool seen = false;
            for (int k = 0; k < nv; k++) seen |= vis[k] == Y;
            if (seen) continue;
            if (nv >= 64 || sp + 1 >= 64) {
                set_status(status, kDevStackOverflow);
                return idx;
            }
            vis[nv++] = Y;
            sp++;
            stk[sp] = Y;
            st[sp] = 0;
            continue;
        }
        if (newPos) newPos[X] = posBase + idx;
        idx++;
        sp--;
    }
    return idx;
}

__global__ void k_rep_rebuild(int64_t nCand, int64_t N, const int *rootRef, const int *canon, const int *f0,
                              const int *f1, const int *owner, int *kcnt, const int *koff, int *newPos, int *status) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nCand; c += stride) {
        int r = rootRef[c];
        if (r == INT_MIN || r >= 0) {
            if (!newPos) kcnt[c] = 0;
            continue;
        }
        int X = canon[-r - 1];
        if (newPos)
            rep_rebuild_dfs((int)c, X, N, f0, f1, owner, newPos, (int)N + koff[c], status);
        else
            kcnt[c] = rep_rebuild_dfs((int)c, X, N, f0, f1, owner, nullptr, 0, status);
    }
}

__global__ void k_rep_newnodes(int64_t K, int64_t N, const int *canon, const int *f0, const int *f1, const uint8_t *c0,
                               const uint8_t *c1, const int *newPos, const int *owner, const int *cand, const int *wg,
                               const int *wlev, int *L0, int *L1, int *gidAll, int *ownLev) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t T = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; T < K; T += stride) {
        if (canon[T] != T) continue;
        int q = newPos[T];
        if (q < 0) continue;
        int a = f0[T], b = f1[T];
        L0[q] = (a < N ? 2 * a : 2 * newPos[a - N]) + c0[T];
        L1[q] = (b < N ? 2 * b : 2 * newPos[b - N]) + c1[T];
        gidAll[q] = wg[cand[owner[T]]];
        ownLev[q - N] = wlev[cand[owner[T]]];
    }
}

__global__ void k_rep_final(int64_t nCand, int64_t N, const int *repT, const int *newPos, int *repW) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nCand; c += stride) {
        int r = repT[c];
        repW[c] = (r >= 2 * N) ? 2 * newPos[(r >> 1) - N] + (r & 1) : r;
    }
}

__global__ void k_rep_extend(int64_t N, int64_t M, const int *w0, const int *w1, const int *wg, const int *ref, int *L0,
                             int *L1, int *gidAll, int *ref2, uint8_t *del) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < M; q += stride) {
        if (q < N) {
            L0[q] = w0[q];
            L1[q] = w1[q];
            gidAll[q] = wg[q];
            ref2[q] = ref[q];
            del[q] = 0;
        } else {
            ref2[q] = 0;
            del[q] = 1;
        }
    }
}

}  // namespace

static int rep_extend_only(ExecCtx &X, RwWork &w, int64_t nNew) {
    const int64_t M = w.N + nNew;
    w.L0 = X.ar->get<int>(M);
    w.L1 = X.ar->get<int>(M);
    w.gidAll = X.ar->get<int>(M);
    int *ref2 = X.ar->get<int>(M);
    w.del = X.ar->get<uint8_t>(M);
    if (!w.L0 || !w.L1 || !w.gidAll || !ref2 || !w.del) return X.fail(CULS_E_OOM, "rw: arena exhausted (replace)");
    k_rep_extend<<<X.grid(M), kBlock, 0, X.s>>>(w.N, M, w.w0, w.w1, w.wg, w.ref, w.L0, w.L1, w.gidAll, ref2, w.del);
    X.launched(1);
    w.ref = ref2;
    w.nNew = nNew;
    return 0;
}

int rw_replace(ExecCtx &X, Batch &b, RwWork &w) {
    (void)b;
    const int64_t N = w.N, nCand = w.nCand;
    cudaStream_t s = X.s;
    Arena &ar = *X.ar;
    int rc;
    w.repW = ar.get<int>(nCand + 1);
    if (!w.repW) return X.fail(CULS_E_OOM, "rw: arena exhausted (replace)");
    if (nCand == 0) return rep_extend_only(X, w, 0);
    int *kcnt = ar.get<int>(nCand + 1), *koff = ar.get<int>(nCand + 1), *rootRef = ar.get<int>(nCand + 1);
    int *repT = ar.get<int>(nCand + 1);
    if (!kcnt || !koff || !rootRef || !repT) return X.fail(CULS_E_OOM, "rw: arena exhausted (replace)");
    int *cnt = X.counters + 16;
    if ((rc = X.check(cudaMemsetAsync(cnt, 0, sizeof(int) * 8, s), "memset"))) return rc;
    RepArgs A{N,    w.cand, w.bestCut, w.bestOut, w.cutL,  w.cutM,  w.wg,    w.dg,    X.lib,   w.tab,   w.wph,
              X.status, kcnt, koff,    nullptr,   nullptr, nullptr, nullptr, nullptr, nullptr, rootRef, cnt + 1};
    k_rep_count<<<X.grid(nCand, 64), 64, 0, s>>>(nCand, A);
    X.launched(1);
    if ((rc = X.check(scan_exclusive(kcnt, koff, nCand, cnt + 0, ar, s), "scan"))) return rc;
    if ((rc = X.check(cudaMemcpyAsync(X.hostSmall + 16, cnt, sizeof(int) * 8, cudaMemcpyDeviceToHost, s), "d2h")))
        return rc;
    if ((rc = X.sync())) return rc;
    const int64_t K = X.hostSmall[16];
    if (N + K >= (1ll << 29)) return X.fail(CULS_E_INVALID, "rw: batch too large for 30-bit node positions");
    int *recCand = ar.get<int>(K + 1), *r0 = ar.get<int>(K + 1), *r1 = ar.get<int>(K + 1), *depth = ar.get<int>(K + 1);
    uint8_t *rc0 = ar.get<uint8_t>(K + 1), *rc1 = ar.get<uint8_t>(K + 1);
    int *canon = ar.get<int>(K + 1), *f0 = ar.get<int>(K + 1), *f1 = ar.get<int>(K + 1), *slot = ar.get<int>(K + 1);
    uint8_t *nph = ar.get<uint8_t>(K + 1), *c0 = ar.get<uint8_t>(K + 1), *c1 = ar.get<uint8_t>(K + 1);
    int *owner = ar.get<int>(K + 1), *newPos = ar.get<int>(K + 1), *kp = ar.get<int>(nCand + 1),
        *kpo = ar.get<int>(nCand + 1);
    uint32_t cap = 1024;
    while ((int64_t)cap < 2 * K) cap <<= 1;
    AndSlot *ts = ar.get<AndSlot>(cap);
    if (!recCand || !r0 || !r1 || !depth || !rc0 || !rc1 || !canon || !f0 || !f1 || !slot || !nph || !c0 || !c1 ||
        !owner || !newPos || !kp || !kpo || !ts)
        return X.fail(CULS_E_OOM, "rw: arena exhausted (replace)");
    A.recCand = recCand;
    A.r0 = r0;
    A.r1 = r1;
    A.depth = depth;
    A.rc0 = rc0;
    A.rc1 = rc1;
    k_rep_fill<<<X.grid(nCand, 64), 64, 0, s>>>(nCand, A);
    X.launched(1);
    if ((rc = X.check(cudaMemcpyAsync(X.hostSmall + 16, cnt, sizeof(int) * 8, cudaMemcpyDeviceToHost, s), "d2h")))
        return rc;
    if ((rc = X.sync())) return rc;
    if ((rc = X.status_check("rw replace match"))) return rc;
    const int maxDepth = X.hostSmall[17];
    if ((rc = X.check(and_table_clear(ts, cap, s), "fill"))) return rc;
    MergeArgs Mg{N, K, r0, r1, depth, rc0, rc1, w.wph, canon, nph, f0, f1, c0, c1, slot, AndTable{ts, cap - 1},
                 X.status};
    for (int d = 1; d <= maxDepth; d++) {
        k_rep_insert<<<X.grid(K), kBlock, 0, s>>>(d, Mg);
        k_rep_canon<<<X.grid(K), kBlock, 0, s>>>(d, Mg);
        X.launched(2);
    }
    k_rep_root<<<X.grid(nCand), kBlock, 0, s>>>(nCand, N, w.cand, rootRef, canon, nph, w.wph, repT);
    if ((rc = X.check(fill_i32(owner, INT_MAX, K, s), "fill"))) return rc;
    if (K > 0) k_rep_owner<<<X.grid(K), kBlock, 0, s>>>(K, recCand, canon, owner);
    k_rep_rebuild<<<X.grid(nCand, 64), 64, 0, s>>>(nCand, N, rootRef, canon, f0, f1, owner, kp, nullptr, nullptr,
                                                     X.status);
    X.launched(3);
    if ((rc = X.check(scan_exclusive(kp, kpo, nCand, cnt + 2, ar, s), "scan"))) return rc;
    if ((rc = X.check(cudaMemcpyAsync(X.hostSmall + 16, cnt, sizeof(int) * 8, cudaMemcpyDeviceToHost, s), "d2h")))
        return rc;
    if ((rc = X.sync())) return rc;
    const int64_t nNew = X.hostSmall[18];
    if ((rc = X.check(fill_i32(newPos, -1, K, s), "fill"))) return rc;
    k_rep_rebuild<<<X.grid(nCand, 64), 64, 0, s>>>(nCand, N, rootRef, canon, f0, f1, owner, nullptr, kpo, newPos,
                                                     X.status);
    X.launched(1);
    if ((rc = rep_extend_only(X, w, nNew))) return rc;
    w.newOwnLev = ar.get<int>(nNew + 1);
    if (!w.newOwnLev) return X.fail(CULS_E_OOM, "rw: arena exhausted (replace)");
    if (K > 0)
        k_rep_newnodes<<<X.grid(K), kBlock, 0, s>>>(K, N, canon, f0, f1, c0, c1, newPos, owner, w.cand, w.wg, w.wlev,
                                                    w.L0, w.L1, w.gidAll, w.newOwnLev);
    k_rep_final<<<X.grid(nCand), kBlock, 0, s>>>(nCand, N, repT, newPos, w.repW);
    X.launched(2);
    if ((rc = X.sync())) return rc;
    return X.status_check("rw replace");
}

}  // namespace culs
