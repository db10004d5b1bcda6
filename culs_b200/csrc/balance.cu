// AIG balancing `b` on the GPU: the result of CULS's balancePerformV2 with
// sortDecId = 1 (src/algorithms/balance.cu:912-1382) and AIGMan::balance
// (src/aig_manager.cu:682-737), equal node for node.
//
// Phase 1, covers.  Starting from the AND nodes that drive POs, level L's
// frontier lists the nodes whose cover (supergate) is needed; every
// frontier node records L as its last appear level, collects its cover once
// (the DFS of localCoverTravToTable, balance.cu:666-751, leaves in pop
// order), and the AND leaves of its cover form level L + 1's frontier.  The
// reference rebuilds each frontier by a copy_if over all nodes; here the
// frontier is an append list deduplicated by a per-node level stamp, and
// levels are launched sixteen at a time without a host round trip.  A DFS
// keeps up to 32 leaves in registers; a larger cover (up to 1,024 leaves) is
// redone by a second kernel with a leaf buffer in global memory.
//
// Phase 2, reconstruction.  Covers are taken deepest level first, in
// increasing node id, in chunks of 32,768 (the reference's iterLen): each
// cover's inputs (their covers' new literals, with levels) sorted by
// decreasing level then literal; then lockstep steps, one thread per cover,
// two kernels per step:
//   1. the shared-node permutation and the pairing of the two lowest inputs
//      (balance.cu:113-247): a pair that is trivial or already built is
//      reused, else it is inserted into the table with id counter + cover
//      index (atomicMin keeps the smallest id of a key);
//   2. the pair's winning id, the step's largest id (the next counter), the
//      new node's level, and the pair's result put back in level order
//      (balance.cu:429-467).
// Lookups in step 1 must see the table as it was before the step: every
// entry carries the step that inserted it, and entries of the current step
// are invisible.  A chunk needs at most (longest cover - 1) steps, known on
// the host from phase 1, so steps are launched back to back.
//
// Phase 3 renumbers the built nodes in id order (balance.cu:1285-1318) and
// maps the POs (balance.cu:882-910).  Graphs of a batch are balanced one
// after another; `b` then strashes the batch (AIGMan::balance with
// updateLevel).
#include <algorithm>
#include <climits>
#include <vector>

#include "kernels.cuh"

namespace culs {

namespace {

constexpr int kBalMaxCover = 1024;  // MAX_LOCAL_COVER_SIZE, balance.cu:17
constexpr int kBalStack = 128;      // DFS_COVER_STACK_SIZE, balance.cu:18
constexpr int kBalChunk = 32768;    // iterLen, balance.cu:1125
constexpr int kBalLocal = 32;       // leaves a DFS keeps in registers
constexpr int kBalBigThreads = 2048;  // threads (each with a 1,024-leaf buffer) for the large covers
constexpr int kBalLevelsPerSync = 16;
constexpr unsigned kNoId = 0xFFFFFFFFu;
constexpr int kNoEpoch = INT_MAX;
constexpr int64_t kBalProbeCap = 1 << 20;

__device__ __forceinline__ int lit_id_(int l) { return l >> 1; }

struct BalView {  // one graph: local AIGMan literals, objects [0, nObj)
    const int *F0, *F1, *PO;
    int nPIs, nPO, nObj;
};

// ------------------------------------------------------------- phase 1
__global__ void k_bal_fanouts(BalView V, int *nfo) {
    const int stride = gridDim.x * blockDim.x;
    for (int v = V.nPIs + 1 + blockIdx.x * blockDim.x + threadIdx.x; v < V.nObj; v += stride) {
        atomicAdd(&nfo[lit_id_(V.F0[v])], 1);
        atomicAdd(&nfo[lit_id_(V.F1[v])], 1);
    }
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < V.nPO; k += stride) atomicAdd(&nfo[lit_id_(V.PO[k])], 1);
}

// The AND nodes driving POs, each once: level 0's frontier
// (checkCoverTravEnd, balance.cu:38-74).
__global__ void k_bal_roots(BalView V, int *stamp, int *list, int *cnt) {
    const int stride = gridDim.x * blockDim.x;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < V.nPO; k += stride) {
        const int v = lit_id_(V.PO[k]);
        if (v > V.nPIs && atomicCAS(&stamp[v], 0, 1) == 0) list[atomicAdd(cnt, 1)] = v;
    }
}

// The supergate DFS of localCoverTravToTable (balance.cu:666-751) into
// leaves[0..cap).  Returns the leaf count, -1 for a constant-false cover (a
// leaf and its complement), or -2 when more than cap leaves are needed.
__device__ int bal_cover_dfs(const BalView &V, const int *nfo, int v, int *leaves, int cap) {
    int stk[kBalStack];
    int top = -1, n = 0;
    stk[++top] = 2 * v;
    while (top >= 0) {
        const int cur = stk[top--];
        bool same = false;
        for (int j = 0; j < n; j++) {
            const int x = leaves[j];
            if (x == cur) {
                same = true;
                break;
            }
            if (x == (cur ^ 1)) return -1;
        }
        if (same) continue;
        const int id = lit_id_(cur);
        if (cur != 2 * v && ((cur & 1) || id <= V.nPIs || nfo[id] > 1 || top + 2 >= kBalStack ||
                             n + 2 * (top + 1) + 1 >= kBalMaxCover)) {
            if (n == cap) return -2;
            leaves[n++] = cur;
            continue;
        }
        stk[++top] = V.F1[id];
        stk[++top] = V.F0[id];
    }
    return n;
}

struct BalCovers {
    int *covLen;     // -1 not collected, -2 waiting for the large-cover kernel, else leaf count (0: constant false)
    int *covOff;     // first leaf in flat
    int *lastLevel;  // last frontier level the node is on
    int *flat;       // every collected cover's leaves
    int *cursor;     // leaves used in flat
    int64_t flatCap;
    int *status;
};

__device__ __forceinline__ void bal_store_cover(const BalCovers &K, int v, const int *leaves, int n) {
    int off = 0;
    if (n > 0) {
        off = atomicAdd(K.cursor, n);
        if ((int64_t)off + n > K.flatCap) {
            set_status(K.status, kDevCapacity);
            n = 0;
        } else {
            for (int j = 0; j < n; j++) K.flat[off + j] = leaves[j];
        }
    }
    K.covOff[v] = off;
    K.covLen[v] = n;
}

// Level L's frontier: last appear level, and the covers not yet collected
// (those over kBalLocal leaves are listed for k_bal_cover_big).
__global__ void k_bal_level(BalView V, const int *nfo, BalCovers K, const int *list, const int *cnt, int L, int *big,
                            int *bigCnt) {
    const int n = *cnt;
    const int stride = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int v = list[i];
        K.lastLevel[v] = L;
        if (K.covLen[v] != -1) continue;
        int leaves[kBalLocal];
        const int r = bal_cover_dfs(V, nfo, v, leaves, kBalLocal);
        if (r == -2) {
            K.covLen[v] = -2;
            big[atomicAdd(bigCnt, 1)] = v;
        } else {
            bal_store_cover(K, v, leaves, r < 0 ? 0 : r);
        }
    }
}

// The frontier's large covers, each thread with a 1,024-leaf buffer of its own.
__global__ void k_bal_cover_big(BalView V, const int *nfo, BalCovers K, const int *big, const int *bigCnt,
                                int *scratch) {
    const int n = *bigCnt;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    int *leaves = scratch + (int64_t)t * kBalMaxCover;
    for (int i = t; i < n; i += gridDim.x * blockDim.x) {
        const int v = big[i];
        const int r = bal_cover_dfs(V, nfo, v, leaves, kBalMaxCover);
        if (r == -2) set_status(K.status, kDevCapacity);  // cannot happen: the DFS stops at 1,024 leaves
        bal_store_cover(K, v, leaves, r < 0 ? 0 : r);
    }
}

// Level L + 1's frontier: the AND leaves of level L's covers, each once.
__global__ void k_bal_next(BalView V, BalCovers K, const int *list, const int *cnt, int L, int *stamp, int *next,
                           int *nextCnt) {
    const int n = *cnt;
    const int stride = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int v = list[i];
        const int len = K.covLen[v];
        for (int j = 0; j < len; j++) {
            const int x = lit_id_(K.flat[K.covOff[v] + j]);
            if (x > V.nPIs && atomicExch(&stamp[x], L + 2) != L + 2) next[atomicAdd(nextCnt, 1)] = x;
        }
    }
}

__global__ void k_bal_cover_flags(int n, const int *covLen, uint8_t *flags) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) flags[v] = covLen[v] >= 0;
}

// per cover (in id order): its last level as the sort key, and per level the
// cover count and the longest cover
__global__ void k_bal_cover_keys(int n, const int *ids, const int *lastLevel, const int *covLen, uint32_t *keys,
                                 int *lvCnt, int *lvMax) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int v = ids[i], L = lastLevel[v];
        keys[i] = (uint32_t)L;
        atomicAdd(&lvCnt[L], 1);
        atomicMax(&lvMax[L], covLen[v]);
    }
}

// ------------------------------------------------------------- phase 2
struct BalTables {
    unsigned long long *key;  // built pairs: (lit0 << 32) | lit1, lit0 < lit1
    unsigned *id;             //   smallest id inserted with the key
    int *epoch;               //   step that inserted the key
    uint32_t rMask;
    unsigned *lvKey;  // levels of built nodes by id
    int *lvVal;
    uint32_t lMask;
    int *status;
};

__device__ __forceinline__ uint32_t bal_hash(unsigned long long k) { return (uint32_t)mix64(k); }

// insert_batch_update_min_masked (src/hash_table/hash_table.h:247-269), the
// entry tagged with the inserting step
__device__ void bal_insert(const BalTables &T, unsigned long long key, unsigned id, int step) {
    uint32_t h = bal_hash(key) & T.rMask;
    for (int64_t p = 0; p <= T.rMask && p < kBalProbeCap; p++) {
        const unsigned long long prev = atomicCAS(&T.key[h], kEmptyKey, key);
        if (prev == kEmptyKey) T.epoch[h] = step;
        if (prev == kEmptyKey || prev == key) {
            atomicMin(&T.id[h], id);
            return;
        }
        h = (h + 1) & T.rMask;
    }
    set_status(T.status, kDevTableFull);
}

// Id of a built pair as of the start of step `step` (entries of that step
// invisible), or kNoId.
__device__ unsigned bal_find(const BalTables &T, unsigned long long key, int step) {
    uint32_t h = bal_hash(key) & T.rMask;
    for (int64_t p = 0; p <= T.rMask && p < kBalProbeCap; p++) {
        const unsigned long long k = T.key[h];
        if (k == key) return T.epoch[h] < step ? T.id[h] : kNoId;
        if (k == kEmptyKey) return kNoId;
        h = (h + 1) & T.rMask;
    }
    set_status(T.status, kDevTableFull);
    return kNoId;
}

__device__ void bal_level_insert(const BalTables &T, unsigned id, int lvl) {
    uint32_t h = bal_hash(id) & T.lMask;
    for (int64_t p = 0; p <= T.lMask && p < kBalProbeCap; p++) {
        const unsigned prev = atomicCAS(&T.lvKey[h], kNoId, id);
        if (prev == kNoId || prev == id) {
            atomicMin(&T.lvVal[h], lvl);
            return;
        }
        h = (h + 1) & T.lMask;
    }
    set_status(T.status, kDevTableFull);
}

__device__ int bal_level_of(const BalTables &T, int lit, int nPIs) {
    const unsigned id = (unsigned)lit_id_(lit);
    if ((int)id <= nPIs) return 0;
    uint32_t h = bal_hash(id) & T.lMask;
    for (int64_t p = 0; p <= T.lMask && p < kBalProbeCap; p++) {
        const unsigned k = T.lvKey[h];
        if (k == id) return T.lvVal[h];
        if (k == kNoId) break;
        h = (h + 1) & T.lMask;
    }
    set_status(T.status, kDevBadGraph);  // a built node without a level
    return 0;
}

// retrieveAndNode (balance.cu:85-110): the literal of l1 AND l2 when it is
// trivial (checkTrivialAndCases, src/hash_table/hash_table.h:435-449) or
// built before `step`, else kNoId.  AIGMan literals: 0 = TRUE, 1 = FALSE.
__device__ unsigned bal_and_lookup(const BalTables &T, int l1, int l2, int step) {
    if (l1 == l2) return (unsigned)l1;
    if (l1 == (l2 ^ 1)) return 1u;
    if (l1 == 0) return (unsigned)l2;
    if (l2 == 0) return (unsigned)l1;
    if (l1 == 1 || l2 == 1) return 1u;
    if (l1 > l2) {
        const int t = l1;
        l1 = l2;
        l2 = t;
    }
    const unsigned id = bal_find(T, ((unsigned long long)(uint32_t)l1 << 32) | (uint32_t)l2, step);
    return id == kNoId ? kNoId : id << 1;
}

struct BalChunk {
    const int *covers;  // the chunk's cover roots
    int n;
    int *off, *len;     // per cover: its array in work, current length
    int2 *work;         // {literal, level} arrays, longest level first
    int *mask;          // step outcome: 0 done, 1 new pair, 2 reused
    unsigned long long *key;
    unsigned *val;
    int *lvl;
    int *ctr, *smax;    // id counter and largest winning id, rings of 4 by step
};

// prepareReconstructArrays (balance.cu:272-426) with sortDecId = 1: the
// inputs' new literals and levels, sorted by decreasing level, then literal.
__global__ void k_bal_prepare(BalChunk C, BalTables T, const int *covOff, const int *covLen, const int *flat,
                              const int *newLit, int nPIs) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < C.n; i += gridDim.x * blockDim.x) {
        const int v = C.covers[i];
        const int off = covOff[v], n = covLen[v];
        C.off[i] = off;
        C.len[i] = n;
        int2 *a = C.work + off;
        for (int j = 0; j < n; j++) {
            const int x = flat[off + j];
            const int nl = lit_id_(x) <= nPIs ? x : (newLit[lit_id_(x)] ^ (x & 1));
            int2 e = make_int2(nl, bal_level_of(T, nl, nPIs));
            int k = j;
            // insertion sort: (level desc, literal desc)
            while (k > 0 && (a[k - 1].y < e.y || (a[k - 1].y == e.y && a[k - 1].x < e.x))) {
                a[k] = a[k - 1];
                k--;
            }
            a[k] = e;
        }
    }
}

// Step `step`, part 1: sharedNodeDrivenPermute (balance.cu:187-247) and
// prepareDataToInsert (balance.cu:113-184), then the new pairs' insertion.
__global__ void k_bal_step1(BalChunk C, BalTables T, int step, int nPIs) {
    const int prev = (step - 1) & 3;
    const int counter = C.smax[prev] ? C.smax[prev] + 1 : C.ctr[prev];  // newIdCounter of this step
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        C.ctr[step & 3] = counter;
        C.smax[(step + 1) & 3] = 0;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < C.n; i += gridDim.x * blockDim.x) {
        const int len = C.len[i];
        if (len <= 1) {
            C.mask[i] = 0;
            continue;
        }
        int2 *a = C.work + C.off[i];
        int left = 0;
        if (len >= 3) {
            left = len - 2;
            const int border = a[left].y;
            for (left--; left >= 0 && a[left].y == border; left--) {
            }
            left++;
        }
        const int right = len - 2;
        if (left < right) {
            const int l1 = a[right + 1].x, l2 = a[right].x;
            for (int k = right; k >= left; k--) {
                const int l3 = a[k].x;
                if (bal_and_lookup(T, l1, l3, step) != kNoId) {
                    if (l3 != l2) {
                        const int2 t = a[k];
                        a[k] = a[right];
                        a[right] = t;
                    }
                    break;
                }
            }
        }
        int l1 = a[len - 1].x, l2 = a[len - 2].x;
        const int lv1 = a[len - 1].y, lv2 = a[len - 2].y;
        C.len[i] = len - 2;
        const unsigned got = bal_and_lookup(T, l1, l2, step);
        if (got != kNoId) {
            C.mask[i] = 2;
            C.val[i] = got;
            C.lvl[i] = bal_level_of(T, (int)got, nPIs);
        } else {
            if (l1 > l2) {
                const int t = l1;
                l1 = l2;
                l2 = t;
            }
            const unsigned long long key = ((unsigned long long)(uint32_t)l1 << 32) | (uint32_t)l2;
            C.mask[i] = 1;
            C.key[i] = key;
            C.lvl[i] = (lv1 > lv2 ? lv1 : lv2) + 1;
            bal_insert(T, key, (unsigned)(counter + i), step);
        }
    }
}

// Step `step`, part 2: the winning ids (retrieve_batch_masked), the step's
// largest id, the new nodes' levels, and addBackLocalArrays.
__global__ void k_bal_step2(BalChunk C, BalTables T, int step) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < C.n; i += gridDim.x * blockDim.x) {
        const int m = C.mask[i];
        if (m == 0) continue;
        int lit;
        if (m == 1) {
            const unsigned id = bal_find(T, C.key[i], INT_MAX);
            if (id == kNoId) {
                set_status(T.status, kDevTableFull);
                continue;
            }
            atomicMax(&C.smax[step & 3], (int)id);
            bal_level_insert(T, id, C.lvl[i]);
            lit = (int)(id << 1);
        } else {
            lit = (int)C.val[i];
        }
        int2 *a = C.work + C.off[i];
        const int len = C.len[i];
        bool dup = false;
        for (int j = 0; j < len && !dup; j++) dup = a[j].x == lit;
        if (dup) continue;
        int k = len;
        const int2 e = make_int2(lit, C.lvl[i]);
        while (k > 0 && e.y > a[k - 1].y) {
            a[k] = a[k - 1];
            k--;
        }
        a[k] = e;
        C.len[i] = len + 1;
    }
}

// recordReconstructedCovers (balance.cu:469-491)
__global__ void k_bal_record(BalChunk C, int *newLit) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < C.n; i += gridDim.x * blockDim.x)
        newLit[C.covers[i]] = C.len[i] == 0 ? 1 : C.work[C.off[i]].x;
}

// ------------------------------------------------------------- phase 3
__global__ void k_bal_used(uint32_t cap, const unsigned long long *key, uint8_t *flags) {
    for (int64_t h = blockIdx.x * blockDim.x + threadIdx.x; h < cap; h += (int64_t)gridDim.x * blockDim.x)
        flags[h] = key[h] != kEmptyKey;
}

__global__ void k_bal_ids(int n, const int *slots, const unsigned *id, uint32_t *keys) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) keys[i] = id[slots[i]];
}

// built node id -> new literal: nPIs + 1 + its rank among the built ids
__device__ __forceinline__ int bal_out_lit(int lit, int nPIs, const uint32_t *ids, int n) {
    const unsigned id = (unsigned)lit_id_(lit);
    if ((int)id <= nPIs) return lit;
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (ids[mid] < id)
            lo = mid + 1;
        else
            hi = mid;
    }
    return 2 * (nPIs + 1 + lo) + (lit & 1);
}

__global__ void k_bal_out(int n, const uint32_t *ids, const int *slots, const unsigned long long *key, BalView V,
                          const int *newLit, int *F0n, int *F1n, int *POn) {
    const int stride = gridDim.x * blockDim.x;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride) {
        const unsigned long long k = key[slots[r]];
        F0n[V.nPIs + 1 + r] = bal_out_lit((int)(uint32_t)(k >> 32), V.nPIs, ids, n);
        F1n[V.nPIs + 1 + r] = bal_out_lit((int)(uint32_t)k, V.nPIs, ids, n);
    }
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r <= V.nPIs; r += stride) F0n[r] = F1n[r] = -1;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < V.nPO; k += stride) {
        const int o = V.PO[k];
        POn[k] = lit_id_(o) <= V.nPIs ? o : (bal_out_lit(newLit[lit_id_(o)], V.nPIs, ids, n) ^ (o & 1));
    }
}

__global__ void k_bal_init_tables(BalTables T, int64_t rCap, int64_t lCap) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t h = blockIdx.x * blockDim.x + threadIdx.x; h < rCap; h += stride) {
        T.key[h] = kEmptyKey;
        T.id[h] = kNoId;
        T.epoch[h] = kNoEpoch;
    }
    for (int64_t h = blockIdx.x * blockDim.x + threadIdx.x; h < lCap; h += stride) {
        T.lvKey[h] = kNoId;
        T.lvVal[h] = INT_MAX;
    }
}

__global__ void k_bal_copy_graph(BalView V, int *F0n, int *F1n, int *POn) {
    const int stride = gridDim.x * blockDim.x;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < V.nObj; v += stride) {
        F0n[v] = V.F0[v];
        F1n[v] = V.F1[v];
    }
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < V.nPO; k += stride) POn[k] = V.PO[k];
}

uint32_t pow2_at_least(int64_t n) {
    uint32_t c = 1024;
    while ((int64_t)c < n && c < (1u << 31)) c <<= 1;
    return c;
}

}  // namespace

// One graph: F0n/F1n/POn receive the balanced graph (nPIs + 1 + *nAnds
// objects); the caller's buffers hold at least the input's object count.
int Engine::balance_graph(const int *F0, const int *F1, const int *PO, int nPIs, int nPO, int nObj, int *F0n,
                          int *F1n, int *POn, int *nAndsOut) {
    cudaStream_t s = s_;
    const BalView V{F0, F1, PO, nPIs, nPO, nObj};
    const int nAnd = nObj - 1 - nPIs;
    const unsigned g1 = grid_1d(std::max(nObj, nPO), kBlock, sms_ * 8);
    if (nAnd == 0) {
        k_bal_copy_graph<<<g1, kBlock, 0, s>>>(V, F0n, F1n, POn);
        launches_ += 1;
        *nAndsOut = 0;
        return check(cudaGetLastError(), "balance launch");
    }
    const int64_t flatCap = 4 * (int64_t)nAnd + 16;  // leaves of all covers: at most 2 per AND fanin edge visit
    int rc;
    // per object: 15 arrays of 4 bytes; per cover leaf (at most flatCap):
    // leaf, work pair, and the two tables with their renumbering scratch at
    // up to four slots per leaf
    if ((rc = ensure_arena((size_t)nObj * 64 + (size_t)flatCap * 192 + (size_t)kBalChunk * 48 +
                           (size_t)kBalBigThreads * kBalMaxCover * 4 + ((size_t)64 << 20))))
        return rc;
    ar_.reset();
    int *nfo = ar_.get<int>(nObj), *stamp = ar_.get<int>(nObj), *covLen = ar_.get<int>(nObj),
        *covOff = ar_.get<int>(nObj), *lastLevel = ar_.get<int>(nObj), *newLit = ar_.get<int>(nObj);
    int *lists[2] = {ar_.get<int>(nObj), ar_.get<int>(nObj)};
    int *big = ar_.get<int>(nObj);
    int *flat = ar_.get<int>(flatCap);
    int *scratch = ar_.get<int>((size_t)kBalBigThreads * kBalMaxCover);
    int *cnt = ar_.get<int>((size_t)nObj + 2 + kBalLevelsPerSync);  // frontier size per level
    int *misc = ar_.get<int>(16);  // [0] flat cursor, [1] large covers of the current level
    if (!nfo || !stamp || !covLen || !covOff || !lastLevel || !newLit || !lists[0] || !lists[1] || !big || !flat ||
        !scratch || !cnt || !misc)
        return fail(CULS_E_OOM, "balance: arena exhausted");
    check(cudaMemsetAsync(nfo, 0, sizeof(int) * nObj, s), "memset");
    check(cudaMemsetAsync(stamp, 0, sizeof(int) * nObj, s), "memset");
    check(cudaMemsetAsync(covLen, 0xFF, sizeof(int) * nObj, s), "memset");  // -1: not collected
    check(cudaMemsetAsync(lastLevel, 0xFF, sizeof(int) * nObj, s), "memset");
    check(cudaMemsetAsync(cnt, 0, sizeof(int) * ((size_t)nObj + 2 + kBalLevelsPerSync), s), "memset");
    check(cudaMemsetAsync(misc, 0, sizeof(int) * 16, s), "memset");
    k_bal_fanouts<<<g1, kBlock, 0, s>>>(V, nfo);
    k_bal_roots<<<g1, kBlock, 0, s>>>(V, stamp, lists[0], cnt);
    launches_ += 2;
    // ---- phase 1: frontier levels, sixteen per host check
    BalCovers K{covLen, covOff, lastLevel, flat, misc, flatCap, status_};
    const unsigned gL = (unsigned)(sms_ * 4);
    int levels = -1;
    std::vector<int> hc(kBalLevelsPerSync);
    for (int L0 = 0; levels < 0; L0 += kBalLevelsPerSync) {
        for (int L = L0; L < L0 + kBalLevelsPerSync; L++) {
            int *cur = lists[L & 1], *nxt = lists[(L + 1) & 1];
            check(cudaMemsetAsync(misc + 1, 0, sizeof(int), s), "memset");
            k_bal_level<<<gL, kBlock, 0, s>>>(V, nfo, K, cur, cnt + L, L, big, misc + 1);
            k_bal_cover_big<<<kBalBigThreads / 128, 128, 0, s>>>(V, nfo, K, big, misc + 1, scratch);
            k_bal_next<<<gL, kBlock, 0, s>>>(V, K, cur, cnt + L, L, stamp, nxt, cnt + L + 1);
            launches_ += 3;
        }
        if ((rc = check(cudaMemcpyAsync(hostSmall_, cnt + L0 + 1, sizeof(int) * kBalLevelsPerSync,
                                        cudaMemcpyDeviceToHost, s), "d2h")))
            return rc;
        if ((rc = sync())) return rc;
        for (int k = 0; k < kBalLevelsPerSync; k++)
            if (hostSmall_[k] == 0) {
                levels = L0 + 1 + k;
                break;
            }
        if (levels < 0 && L0 + kBalLevelsPerSync > nObj) return fail(CULS_E_INVALID, "balance: frontier does not end");
    }
    if ((rc = check_status("balance covers"))) return rc;
    // ---- covers by (last level, id); per level: count and longest cover
    uint8_t *flags = ar_.get<uint8_t>(nObj);
    int *ids = ar_.get<int>(nObj), *sorted = ar_.get<int>(nObj), *ncov = ar_.get<int>(1);
    uint32_t *keys = ar_.get<uint32_t>(nObj), *keys2 = ar_.get<uint32_t>(nObj);
    int *lvCnt = ar_.get<int>(levels + 1), *lvMax = ar_.get<int>(levels + 1);
    if (!flags || !ids || !sorted || !ncov || !keys || !keys2 || !lvCnt || !lvMax)
        return fail(CULS_E_OOM, "balance: arena exhausted");
    k_bal_cover_flags<<<g1, kBlock, 0, s>>>(nObj, covLen, flags);
    check(compact_flags(flags, nObj, ids, ncov, ar_, s), "compact");
    check(cudaMemsetAsync(lvCnt, 0, sizeof(int) * (levels + 1), s), "memset");
    check(cudaMemsetAsync(lvMax, 0, sizeof(int) * (levels + 1), s), "memset");
    check(cudaMemcpyAsync(hostSmall_, ncov, sizeof(int), cudaMemcpyDeviceToHost, s), "d2h");
    check(cudaMemcpyAsync(hostSmall_ + 1, misc, sizeof(int), cudaMemcpyDeviceToHost, s), "d2h");
    if ((rc = sync())) return rc;
    const int nCov = hostSmall_[0];
    const int64_t nLeaves = hostSmall_[1];
    int keyBits = 1;
    while ((1 << keyBits) <= levels) keyBits++;
    k_bal_cover_keys<<<grid_1d(nCov, kBlock, sms_ * 8), kBlock, 0, s>>>(nCov, ids, lastLevel, covLen, keys, lvCnt,
                                                                        lvMax);
    launches_ += 2;
    if ((rc = check(radix_sort_pairs(keys, ids, keys2, sorted, nCov, keyBits, ar_, s), "sort"))) return rc;
    std::vector<int> hCnt(levels), hMax(levels);
    check(cudaMemcpyAsync(hCnt.data(), lvCnt, sizeof(int) * levels, cudaMemcpyDeviceToHost, s), "d2h");
    check(cudaMemcpyAsync(hMax.data(), lvMax, sizeof(int) * levels, cudaMemcpyDeviceToHost, s), "d2h");
    if ((rc = sync())) return rc;
    // ---- phase 2: tables and chunks
    const uint32_t rCap = pow2_at_least(2 * nLeaves + 64), lCap = pow2_at_least(2 * nLeaves + 64);
    BalTables T;
    T.key = ar_.get<unsigned long long>(rCap);
    T.id = ar_.get<unsigned>(rCap);
    T.epoch = ar_.get<int>(rCap);
    T.rMask = rCap - 1;
    T.lvKey = ar_.get<unsigned>(lCap);
    T.lvVal = ar_.get<int>(lCap);
    T.lMask = lCap - 1;
    T.status = status_;
    int2 *work = ar_.get<int2>(nLeaves + 1);
    BalChunk C;
    C.off = ar_.get<int>(kBalChunk);
    C.len = ar_.get<int>(kBalChunk);
    C.mask = ar_.get<int>(kBalChunk);
    C.key = ar_.get<unsigned long long>(kBalChunk);
    C.val = ar_.get<unsigned>(kBalChunk);
    C.lvl = ar_.get<int>(kBalChunk);
    C.ctr = ar_.get<int>(8);
    C.smax = C.ctr + 4;
    C.work = work;
    if (!T.key || !T.id || !T.epoch || !T.lvKey || !T.lvVal || !work || !C.off || !C.len || !C.mask || !C.key ||
        !C.val || !C.lvl || !C.ctr)
        return fail(CULS_E_OOM, "balance: arena exhausted");
    k_bal_init_tables<<<grid_1d(std::max<int64_t>(rCap, lCap), kBlock, sms_ * 16), kBlock, 0, s>>>(T, rCap, lCap);
    {
        // the counter before the first step: nPIs + 1 (balance.cu:1167)
        const int init[8] = {0, 0, 0, nPIs + 1, 0, 0, 0, 0};
        check(cudaMemcpyAsync(C.ctr, init, sizeof init, cudaMemcpyHostToDevice, s), "h2d");
    }
    launches_ += 1;
    std::vector<int64_t> start(levels + 1, 0);
    for (int L = 0; L < levels; L++) start[L + 1] = start[L] + hCnt[L];
    int step = 0;
    for (int L = levels - 1; L >= 0; L--) {
        for (int64_t c0 = start[L]; c0 < start[L + 1]; c0 += kBalChunk) {
            C.covers = sorted + c0;
            C.n = (int)std::min<int64_t>(kBalChunk, start[L + 1] - c0);
            const unsigned gc = grid_1d(C.n, kBlock, sms_ * 8);
            k_bal_prepare<<<gc, kBlock, 0, s>>>(C, T, covOff, covLen, flat, newLit, nPIs);
            for (int k = 0; k + 1 < hMax[L]; k++, step++) {
                k_bal_step1<<<gc, kBlock, 0, s>>>(C, T, step, nPIs);
                k_bal_step2<<<gc, kBlock, 0, s>>>(C, T, step);
            }
            k_bal_record<<<gc, kBlock, 0, s>>>(C, newLit);
            launches_ += 2 + 2 * std::max(0, hMax[L] - 1);
        }
        if ((L & 63) == 0 && (rc = check(cudaGetLastError(), "balance launch"))) return rc;
    }
    if ((rc = sync()) || (rc = check_status("balance reconstruction"))) return rc;
    // ---- phase 3: renumbering in id order
    uint8_t *used = ar_.get<uint8_t>(rCap);
    int *slots = ar_.get<int>(rCap), *slots2 = ar_.get<int>(rCap), *nBuilt = ar_.get<int>(1);
    uint32_t *bid = ar_.get<uint32_t>(rCap), *bid2 = ar_.get<uint32_t>(rCap);
    if (!used || !slots || !slots2 || !nBuilt || !bid || !bid2) return fail(CULS_E_OOM, "balance: arena exhausted");
    k_bal_used<<<grid_1d(rCap, kBlock, sms_ * 16), kBlock, 0, s>>>(rCap, T.key, used);
    check(compact_flags(used, rCap, slots, nBuilt, ar_, s), "compact");
    check(cudaMemcpyAsync(hostSmall_, nBuilt, sizeof(int), cudaMemcpyDeviceToHost, s), "d2h");
    if ((rc = sync())) return rc;
    const int nB = hostSmall_[0];
    if (nB > nAnd) return fail(CULS_E_INVALID, "balance: more nodes built than the input holds");
    k_bal_ids<<<grid_1d(std::max(nB, 1), kBlock, sms_ * 8), kBlock, 0, s>>>(nB, slots, T.id, bid);
    if ((rc = check(radix_sort_pairs(bid, slots, bid2, slots2, nB, 32, ar_, s), "sort"))) return rc;
    k_bal_out<<<grid_1d(std::max(std::max(nB, nPIs + 1), nPO), kBlock, sms_ * 8), kBlock, 0, s>>>(
        nB, bid2, slots2, T.key, V, newLit, F0n, F1n, POn);
    launches_ += 3;
    if ((rc = sync()) || (rc = check_status("balance output"))) return rc;
    *nAndsOut = nB;
    return 0;
}

// AIGMan::balance(sortDecId = 1, updateLevel) over every graph of b.
int Engine::balance(Batch &b, bool updateLevel) {
    b.keep = false;  // prevCmdRewrite = 0 (aig_manager.cu:729)
    if (!b.pool) b.pool = pool_;
    int rc;
    if ((rc = check(b.reserve_spare(b.nObj + 1, b.nPO + 1), "cudaMalloc"))) return rc;
    std::vector<DevGraph> ng = b.hg;
    int64_t base = 0;
    for (int g = 0; g < b.G; g++) {
        const DevGraph &d = b.hg[g];
        const int nObj = 1 + d.nPIs + d.nAnds;
        int nA = 0;
        rc = balance_graph(b.F0 + d.base, b.F1 + d.base, b.PO + d.poOff, d.nPIs, d.nPOs, nObj, b.F0s + base,
                           b.F1s + base, b.POs + d.poOff, &nA);
        if (rc) return rc;
        ng[g].nAnds = nA;
        ng[g].base = (int)base;
        base += 1 + d.nPIs + nA;
    }
    ar_.reset();
    if ((rc = check(cudaMemcpyAsync(b.dg, ng.data(), sizeof(DevGraph) * b.G, cudaMemcpyHostToDevice, s_), "h2d")))
        return rc;
    if ((rc = sync())) return rc;
    b.swap_spare();
    b.hg = ng;
    b.nObj = base;
    // levels: a strash (the `b` command), else the depth as read
    return updateLevel ? st(b, false) : batch_depth(b);
}

}  // namespace culs
