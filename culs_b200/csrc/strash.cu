// Structural hashing with dangling-node removal (`st`, and the
// deduplication that ends `rw`): a B200 restatement of Aig::strash (CULS
// src/aig/strash.cu:190-314) and of the CPU variants (src/aig/strash.cu:
// 322-466, src/aig_manager.cu:454-522).
//
// Reference semantics kept:
//  * dangling AND nodes are those outside the transitive fanin of the POs
//    (the fix-point of markDanglingNodesIter, strash.cu:175-188);
//  * nodes are hashed frontier by frontier, where a node's frontier is its
//    ASAP level among the remaining nodes, and inside a frontier in id order
//    (strash.cu:247-277);
//  * fanins are mapped to new literals, sorted, folded by
//    checkTrivialAndCases (src/hash_table/hash_table.h:435-449), then hashed
//    on the 64-bit key (lit0 << 32 | lit1) (hash_table.h:427-433);
//  * survivors are renumbered consecutively in (frontier, id) order and the
//    frontier count becomes the AIG level (strash.cu:279-300,483).
// Deterministic choice: among equal keys the earliest node in (frontier, id)
// order wins (the reference keeps whichever insertion lands first).
//
// B200 design: no per-frontier host loop.  Liveness is a reverse Kahn
// worklist, levels an in-order dataflow (a forward Kahn worklist over a
// fanout CSR as the fallback), and hashing either a few full-width rounds
// that iterate the mapping to its fixed point (batches of up to 16M live
// nodes) or a single in-order dataflow pass whose dependency waits are
// per-level completion counters (bounded spins).
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "kernels.cuh"
#include "rw_work.cuh"
#include "sched.cuh"

namespace culs {

namespace {

__device__ __forceinline__ bool is_and(const int *L0, int v) { return L0[v] >= 0; }

__global__ void k_fanout_count(int64_t M, const int *L0, const int *L1, const int *po, int64_t nPO, int *cnt) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < M; v += stride) {
        int a = L0[v];
        if (a < 0) continue;
        atomicAdd(&cnt[a >> 1], 1);
        atomicAdd(&cnt[L1[v] >> 1], 1);
    }
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nPO; k += stride) atomicAdd(&cnt[po[k] >> 1], 1);
}

__global__ void k_dead_seed_flags(int64_t M, const int *L0, const int *cnt, uint8_t *flags) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < M; v += stride)
        flags[v] = (L0[v] >= 0 && cnt[v] == 0) ? 1 : 0;
}

// Reverse Kahn: a node whose fanout count reaches zero is dangling.
__global__ void __launch_bounds__(kBlock) k_dead_queue(WorkQueue q, const int *L0, const int *L1, int *cnt,
                                                        uint8_t *dead, int *status) {
    int h = -1;
    bool fin = false;
    int64_t idle = 0;
    while (true) {
        const int v = queue_try_pop_warp(q, h, fin);
        int p0 = -1, p1 = -1;
        if (v >= 0) {
            dead[v] = 1;
            int u0 = L0[v] >> 1, u1 = L1[v] >> 1;
            if (L0[u0] >= 0 && atomicSub(&cnt[u0], 1) == 1) p0 = u0;
            if (L0[u1] >= 0 && atomicSub(&cnt[u1], 1) == 1) p1 = u1;
        }
        queue_push_warp(q, p0);
        queue_push_warp(q, p1);
        queue_done_warp(q, v >= 0);
        if (queue_round_end(fin, v >= 0, idle, status)) break;
    }
}

// level[v] = 1 for a live AND node without AND fanins (the seeds), -1 for the
// other AND nodes, 0 for the constant and PIs; outdeg[u] = live AND fanouts
// (a node whose two fanins are one node counts once).
__global__ void k_live_degrees(int64_t M, const int *L0, const int *L1, const uint8_t *dead, int *level, int *outdeg,
                               uint8_t *liveFlag, uint8_t *seedFlag) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < M; v += stride) {
        int a = L0[v];
        bool live = a >= 0 && !dead[v];
        liveFlag[v] = live;
        int pend = 0;
        if (live) {
            int u0 = a >> 1, u1 = L1[v] >> 1;
            if (L0[u0] >= 0) {
                pend++;
                atomicAdd(&outdeg[u0], 1);
            }
            if (L0[u1] >= 0 && u1 != u0) {
                pend++;
                atomicAdd(&outdeg[u1], 1);
            }
        }
        level[v] = a < 0 ? 0 : (live && pend == 0 ? 1 : -1);
        seedFlag[v] = live && pend == 0;
    }
}

__global__ void k_csr_fill(int64_t M, const int *L0, const int *L1, const uint8_t *liveFlag, int *cursor, int *adj) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < M; v += stride) {
        if (!liveFlag[v]) continue;
        int u0 = L0[v] >> 1, u1 = L1[v] >> 1;
        if (L0[u0] >= 0) adj[atomicAdd(&cursor[u0], 1)] = (int)v;
        if (L0[u1] >= 0 && u1 != u0) adj[atomicAdd(&cursor[u1], 1)] = (int)v;
    }
}

// Level-synchronous Kahn: ASAP level of every live AND node (PIs and
// constant: 0), one launch per level.  The queue's levels are consecutive
// segments of `items`; launch L reads its segment's start and size from a
// three-slot ring (written by launch L - 1, which has finished), releases
// the fanouts of every node of level L, and appends to level L + 1's
// segment each fanout whose other fanin finished earlier (no pending
// counters: a node's level is written when it is appended, so the levels up
// to L are all known when launch L starts, and of two fanins on the same
// level the one at the higher position appends).  Thread 0 of block 0
// sets the next segment's start and clears the slot that launch L + 1 will
// append to, which no other block of launch L touches.  No thread waits on
// another.  ring[0..2]: segment sizes, ring[3..5]: segment starts, both by
// level mod 3.
__global__ void __launch_bounds__(kBlock) k_level_step(int L, int *items, int *ring, const int *off, const int *adj,
                                                        const int *L0, const int *L1, int *level, const int *gid,
                                                        int *graphLevels, int *maxLevel) {
    const int r = L % 3;
    const int start = ring[3 + r], n = ring[r];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ring[3 + (L + 1) % 3] = start + n;
        ring[(L + 2) % 3] = 0;
        if (n > 0) atomicMax(maxLevel, L);
    }
    if (n == 0) return;
    int *nextCnt = ring + (L + 1) % 3;
    const int nextBase = start + n;
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t i0 = ((int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32; i0 < n; i0 += warps * 32) {
        const int64_t i = i0 + lane;
        int k = 0, e = 0, v = -1;
        if (i < n) {
            v = items[start + i];
            agg_max(graphLevels, gid[v], L);
            k = off[v];
            e = off[v + 1];
        }
        // release the fanouts, one fanout per lane per round: v pushes w when
        // w's other fanin is not an AND node, is below level L, or is on
        // level L at a lower position (levels up to L are all set when the
        // launch starts; later ones read as -1 or L + 1)
        while (__any_sync(0xffffffffu, k < e)) {
            bool push = false;
            int w = 0;
            if (k < e) {
                w = adj[k++];
                const int a = L0[w] >> 1, b = L1[w] >> 1;
                const int u = a == v ? b : a;
                if (u == v || L0[u] < 0) {
                    push = true;
                } else {
                    const int lu = level[u];
                    push = lu >= 0 && (lu < L || (lu == L && u < v));
                }
                if (push) level[w] = L + 1;
            }
            const unsigned b = __ballot_sync(0xffffffffu, push);
            if (b) {
                int base = 0;
                if (lane == 0) base = atomicAdd(nextCnt, __popc(b));
                base = __shfl_sync(0xffffffffu, base, 0);
                if (push) items[nextBase + base + __popc(b & ((1u << lane) - 1u))] = w;
            }
        }
    }
}

__global__ void k_live_flags(int64_t M, const int *L0, const uint8_t *dead, uint8_t *liveFlag, int *done) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < M; v += stride) {
        const bool isAnd = L0[v] >= 0;
        liveFlag[v] = isAnd && !dead[v];
        done[v] = isAnd ? 0 : 1;
    }
}

// Levels of a graph-major batch whose positions are topological (`st`):
// the in-order dataflow of the rw front over the interleaved chunk schedule
// (sched.cuh), instead of a worklist over a fanout CSR.  Every AND node gets
// its ASAP level; only live nodes count towards a graph's depth.  An AND
// node publishes its level (>= 1) in done[], the one word its fanouts wait
// on and read.
__global__ void __launch_bounds__(kBlock) k_st_levelize(ChunkSched S, const int *L0, const int *L1,
                                                         const uint8_t *liveFlag, const int *gid, int *level,
                                                         int *done, int *graphLevels, int *counter, int *maxLevel,
                                                         int *status) {
    __shared__ int64_t s_begin, s_end;
    int myMax = 0;
    while (true) {
        if (threadIdx.x == 0) {
            const int64_t c = atomicAdd(counter, 1);
            if (c < S.total) {
                sched_chunk(S, c, s_begin, s_end);
            } else {
                s_begin = s_end = -1;
            }
        }
        __syncthreads();
        const int64_t begin = s_begin, end = s_end;
        __syncthreads();
        if (begin < 0) break;
        const int64_t p = begin + threadIdx.x;
        if (p >= end) continue;
        const int a = L0[p];
        if (a < 0) continue;  // constant or PI: level 0, done preset
        const int u0 = a >> 1, u1 = L1[p] >> 1;
        int l0 = 0, l1 = 0;
        if (L0[u0] >= 0 && !wait_word(&done[u0], 1, status, &l0)) continue;
        if (L0[u1] >= 0 && !wait_word(&done[u1], 1, status, &l1)) continue;
        const int lv = 1 + (l0 > l1 ? l0 : l1);
        st_relaxed(&done[p], lv);
        __stcg(&level[p], lv);
        if (liveFlag[p]) {
            agg_max(graphLevels, gid[p], lv);
            myMax = lv > myMax ? lv : myMax;
        }
    }
    // every thread of the block leaves the loop at the same claim
    myMax = __reduce_max_sync(0xffffffffu, myMax);
    if ((threadIdx.x & 31) == 0 && myMax > 0) atomicMax(maxLevel, myMax);
}

// Levels over an order that is topological up to a few fanins placed later
// (the rewrite's deduplication: see k_proc_order).  A pass runs the nodes of
// `list` in order; a node waits only for AND fanins earlier in the order.  A
// fanin later in the order that is not done yet, or one left unresolved,
// leaves the node unresolved (done = 2), and the unresolved nodes form the
// next pass's list.  Every wait is on a node whose chunk was claimed
// earlier, so no pass can deadlock, and each pass resolves at least the
// unresolved nodes whose fanins are all resolved.  done[] is the word a node
// publishes: 0 pending, 2 unresolved, level + 2 once resolved.
__global__ void __launch_bounds__(kBlock) k_order_levelize(int64_t n, const int *list, const int *posOf, const int *L0,
                                                            const int *L1, const uint8_t *liveFlag, const int *gid,
                                                            int *level, int *done, int *graphLevels, int *counter,
                                                            int *maxLevel, int *status) {
    __shared__ int64_t s_begin;
    int myMax = 0;
    const int64_t nChunks = (n + kBlock - 1) / kBlock;
    while (true) {
        if (threadIdx.x == 0) {
            const int64_t c = atomicAdd(counter, 1);
            s_begin = c < nChunks ? c * kBlock : -1;
        }
        __syncthreads();
        const int64_t begin = s_begin;
        __syncthreads();
        if (begin < 0) break;
        const int64_t i = begin + threadIdx.x;
        if (i >= n) continue;
        const int v = list[i];
        if (v < 0 || !liveFlag[v]) continue;
        const int pv = posOf[v];
        int lv = 0;
        bool ok = true;
        for (int k = 0; k < 2 && ok; k++) {
            const int u = (k == 0 ? L0[v] : L1[v]) >> 1;
            if (L0[u] < 0) continue;  // constant or PI: level 0
            int d = ld_relaxed(&done[u]);
            if (d == 0 && posOf[u] < pv && !wait_word(&done[u], 1, status, &d)) {
                ok = false;
                break;
            }
            if (d < 3) {  // pending behind this node in the order, or unresolved
                ok = false;
                break;
            }
            const int l = d - 2;
            lv = l > lv ? l : lv;
        }
        if (!ok) {
            st_relaxed(&done[v], 2);
            continue;
        }
        lv += 1;
        st_relaxed(&done[v], lv + 2);
        __stcg(&level[v], lv);
        agg_max(graphLevels, gid[v], lv);
        myMax = lv > myMax ? lv : myMax;
    }
    myMax = __reduce_max_sync(0xffffffffu, myMax);
    if ((threadIdx.x & 31) == 0 && myMax > 0) atomicMax(maxLevel, myMax);
}

__global__ void k_unresolved_flags(int64_t n, const int *list, const int *done, uint8_t *flag) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int v = list[i];
        flag[i] = v >= 0 && done[v] == 2;
    }
}

// next list = list[idx[k]], reset to pending
__global__ void k_unresolved_next(int64_t n, const int *idx, const int *list, int *next, int *done) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
        const int v = list[idx[k]];
        next[k] = v;
        done[v] = 0;
    }
}

// lvlCnt has nBins counters (levels 0 .. nBins - 1)
__global__ void k_gather_levels(int64_t n, const int *idx, const int *level, uint32_t *keys, int *lvlCnt, int nBins) {
    __shared__ int h[kHistBins];
    hist_begin(h, nBins);
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        int l = level[idx[i]];
        keys[i] = (uint32_t)l;
        hist_add(h, nBins, lvlCnt, l);
    }
    hist_end(h, nBins, lvlCnt);
}

__global__ void k_inverse(int64_t n, const int *srt, int *tOf) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += stride) tOf[srt[t]] = (int)t;
}

struct DedupArgs {
    int64_t nLive;
    const int *srt;        // live AND positions in processing order
    const int *rankOf;     // per position: tentative rank (min wins)
    const int *L0, *L1;
    const int *level;
    const int *lvlCnt;     // live AND nodes per level
    const int *lvlStart;   // first processing index of each level
    const int *chunkStart; // first chunk of each level (maxLevel + 2 entries)
    int maxLevel;
    int *lvlDone;
    const int *gid;
    const DevGraph *dg;
    AndTable tab;
    int *mapEnc;  // per position: mapped literal (>= 0) or -(slot+1)
    int *kl0, *kl1;
    int *slotT;   // per processing index: table slot, -1 when folded
    int foldTrivial;
    int unique;  // key each node by its position: nothing merges
    int *counter;
    int *status;
};

constexpr int kDedupChunk = kBlock;

__device__ __forceinline__ int resolve_map(const DedupArgs &A, int u) {
    int e = __ldcg(&A.mapEnc[u]);
    if (e >= 0) return e;
    return 2 * slot_pos(__ldcg(&A.tab.slots[-e - 1].rp));
}

// chunks per level, for the level-aligned claim order of k_dedup
__global__ void k_level_chunks(int n, const int *lvlCnt, int *cc) {
    int stride = gridDim.x * blockDim.x;
    for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < n; l += stride)
        cc[l] = (lvlCnt[l] + kDedupChunk - 1) / kDedupChunk;
}

// Dataflow over the processing order in chunks that never cross a level.
// A chunk of level L needs its fanins' levels (< L) hashed: one thread waits
// for the highest of them, since a level completes only after the level
// below it has (every node of level L has a fanin on level L - 1).  The
// chunk then maps, folds and hashes its nodes and adds its size to its
// level's completion counter with one atomic.
__global__ void __launch_bounds__(kDedupChunk) k_dedup(DedupArgs A) {
    __shared__ int s_begin, s_end, s_level, s_need, s_ok;
    while (true) {
        if (threadIdx.x == 0) {
            const int c = atomicAdd(A.counter, 1);
            if (c < A.chunkStart[A.maxLevel + 1]) {
                int lo = 0, hi = A.maxLevel;
                while (lo < hi) {  // last level whose first chunk is <= c
                    int mid = (lo + hi + 1) >> 1;
                    if (A.chunkStart[mid] <= c)
                        lo = mid;
                    else
                        hi = mid - 1;
                }
                const int b = A.lvlStart[lo] + (c - A.chunkStart[lo]) * kDedupChunk;
                const int e = A.lvlStart[lo] + A.lvlCnt[lo];
                s_begin = b;
                s_end = b + kDedupChunk < e ? b + kDedupChunk : e;
                s_level = lo;
            } else {
                s_begin = -1;
            }
            s_need = -1;
        }
        __syncthreads();
        const int begin = s_begin, end = s_end, lv = s_level;
        if (begin < 0) break;
        const int t = begin + (int)threadIdx.x;
        const bool valid = t < end;
        int v = 0, lits[2] = {0, 0};
        if (valid) {
            v = A.srt[t];
            lits[0] = A.L0[v];
            lits[1] = A.L1[v];
            int need = -1;
            for (int k = 0; k < 2; k++) {
                const int u = lits[k] >> 1;
                if (A.L0[u] >= 0) need = max(need, A.level[u]);
            }
            if (need >= 0) atomicMax(&s_need, need);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            const int need = s_need;
            s_ok = need < 0 ? 1 : (wait_ge(&A.lvlDone[need], A.lvlCnt[need], A.status) ? 1 : 0);
        }
        __syncthreads();
        if (valid && s_ok) {
            for (int k = 0; k < 2; k++) {
                const int u = lits[k] >> 1;
                if (A.L0[u] < 0) continue;  // PI or constant keeps its literal
                lits[k] = resolve_map(A, u) ^ (lits[k] & 1);
            }
            int l0 = lits[0], l1 = lits[1];
            if (l0 > l1) {
                int x = l0;
                l0 = l1;
                l1 = x;
            }
            const int T = 2 * A.dg[A.gid[v]].cpos;  // AIGMan: constant TRUE
            const int F = T + 1;
            int triv = -1;
            if (A.foldTrivial) {
                if (l0 == l1)
                    triv = l0;
                else if (l0 == (l1 ^ 1))
                    triv = F;
                else if (l0 == T)
                    triv = l1;
                else if (l1 == T)
                    triv = l0;
                else if (l0 == F || l1 == F)
                    triv = F;
            }
            if (triv >= 0) {
                A.mapEnc[v] = triv;
                A.slotT[t] = -1;
            } else {
                // literals are non-negative, so a key with the top bit set
                // is never a real one
                const unsigned long long key = A.unique ? (1ull << 63) | (unsigned long long)(uint32_t)v
                                                        : ((unsigned long long)(uint32_t)l0 << 32) | (uint32_t)l1;
                int slot = table_insert(A.tab, key, A.rankOf[v], v, A.status);
                A.kl0[t] = l0;
                A.kl1[t] = l1;
                A.mapEnc[v] = slot >= 0 ? -(slot + 1) : 0;
                A.slotT[t] = slot;
            }
        }
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(&A.lvlDone[lv], end - begin);
        }
    }
}

// ------------------------------------------------- deduplication in rounds
// The mapping k_dedup computes is the unique fixed point of one parallel
// step: a node's key is its fanins' mapped literals (folded when trivial),
// and it maps to the position of the lowest-ranked live node with the same
// key.  (By induction over the levels: a node's key reads only lower
// levels, so any fixed point equals the level-by-level result.)  Starting
// from the identity, round r makes every node of level <= r final, and the
// rounds stop at the first one that changes nothing -- after one round when
// nothing merges, after a few when merges cascade, since a node's key
// changes only when a fanin's mapping did.  Each round is two passes over
// the live nodes with no dependency waits, so a deep, narrow graph costs a
// few launches instead of one wait latency per level.

struct RoundArgs {
    int64_t nLive;
    const int *srt, *rankOf;
    const int *L0, *L1;
    const int *gid;
    const DevGraph *dg;
    AndTable tab;
    const int *cur;  // per position: the literal an AND node maps to this round
    int *nxt;        // the same after this round
    int *slotT;      // per processing index: table slot, -1 when folded
    int *mapEnc, *kl0, *kl1;
    int foldTrivial, unique;
    int *changed;
    int *status;
};

__global__ void k_round_init(int64_t n, const int *srt, int *cur) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += stride) {
        const int v = srt[t];
        cur[v] = 2 * v;
    }
}

// keys from this round's mapping: fold (as k_dedup does) or insert
__global__ void k_round_insert(RoundArgs A) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < A.nLive; t += stride) {
        const int v = A.srt[t];
        int lits[2] = {A.L0[v], A.L1[v]};
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const int u = lits[k] >> 1;
            if (A.L0[u] >= 0) lits[k] = A.cur[u] ^ (lits[k] & 1);
        }
        int l0 = lits[0], l1 = lits[1];
        if (l0 > l1) {
            const int x = l0;
            l0 = l1;
            l1 = x;
        }
        const int T = 2 * A.dg[A.gid[v]].cpos;  // AIGMan: constant TRUE
        const int F = T + 1;
        int triv = -1;
        if (A.foldTrivial) {
            if (l0 == l1)
                triv = l0;
            else if (l0 == (l1 ^ 1))
                triv = F;
            else if (l0 == T)
                triv = l1;
            else if (l1 == T)
                triv = l0;
            else if (l0 == F || l1 == F)
                triv = F;
        }
        if (triv >= 0) {
            A.mapEnc[v] = triv;
            A.nxt[v] = triv;
            A.slotT[t] = -1;
            if (triv != A.cur[v]) *A.changed = 1;
        } else {
            const unsigned long long key = A.unique ? (1ull << 63) | (unsigned long long)(uint32_t)v
                                                    : ((unsigned long long)(uint32_t)l0 << 32) | (uint32_t)l1;
            const int slot = table_insert(A.tab, key, A.rankOf[v], v, A.status);
            A.kl0[t] = l0;
            A.kl1[t] = l1;
            A.mapEnc[v] = slot >= 0 ? -(slot + 1) : 0;
            A.slotT[t] = slot;
        }
    }
}

// every key's lowest rank is known: the inserted nodes map to its position
__global__ void k_round_resolve(RoundArgs A) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < A.nLive; t += stride) {
        const int slot = A.slotT[t];
        if (slot < 0) continue;
        const int v = A.srt[t];
        const int m = 2 * slot_pos(A.tab.slots[slot].rp);
        A.nxt[v] = m;
        if (m != A.cur[v]) *A.changed = 1;
    }
}

// A node wins when its key's lowest rank is its own: its rank is its
// processing index, or (id order) rankOf of its position.
__global__ void k_winner_flags(int64_t n, const int *srt, const int *rankOf, bool idOrder, const int *slotT,
                               const AndSlot *slots, uint8_t *flags) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += stride) {
        const int slot = slotT[t];
        const int rank = idOrder ? rankOf[srt[t]] : (int)t;
        flags[t] = (slot >= 0 && slot_rank(slots[slot].rp) == rank) ? 1 : 0;
    }
}

__global__ void k_gather_rank(int64_t n, const int *wl, const int *srt, const int *rankOf, uint32_t *keys) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        keys[i] = (uint32_t)rankOf[srt[wl[i]]];
}

// Winners of each graph in output order: key = gid, stable.
__global__ void k_winner_keys(int64_t n, const int *wl, const int *srt, const int *gid, uint32_t *keys, int *cntG) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        int g = gid[srt[wl[i]]];
        keys[i] = (uint32_t)g;
        agg_add(cntG, g, 1);
    }
}

__global__ void k_winner_local(int64_t n, const int *wlByG, const int *srt, const int *gid, const int *gStart,
                               const DevGraph *dg, int *newLocalT) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        int t = wlByG[i];
        int g = gid[srt[t]];
        newLocalT[t] = dg[g].nPIs + 1 + (int)(i - gStart[g]);
    }
}

struct OutArgs {
    const int *srt, *tOf, *gid, *lidIn, *L0, *kl0, *kl1, *newLocalT, *mapEnc;
    const AndSlot *slots;
    const int *po;
    const DevGraph *dgNew;
    int *F0, *F1, *PO;
    int64_t nPO;
    int G;
};

__device__ __forceinline__ int local_lit(const OutArgs &A, int lit) {
    int u = lit >> 1;
    if (A.L0[u] < 0) return 2 * A.lidIn[u] + (lit & 1);
    return 2 * A.newLocalT[A.tOf[u]] + (lit & 1);
}

__global__ void k_strash_out(int64_t nW, const int *wl, OutArgs A) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nW; i += stride) {
        int t = wl[i];
        int v = A.srt[t];
        int g = A.gid[v];
        int p = A.dgNew[g].base + A.newLocalT[t];
        // the reference forms keys over the final numbering, so the
        // smaller literal comes first there
        int a = local_lit(A, A.kl0[t]), b = local_lit(A, A.kl1[t]);
        A.F0[p] = a < b ? a : b;
        A.F1[p] = a < b ? b : a;
    }
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < A.nPO; k += stride) {
        int lit = A.po[k];
        int u = lit >> 1;
        int m = lit;
        if (A.L0[u] >= 0) {
            int e = A.mapEnc[u];
            int base = e >= 0 ? e : 2 * slot_pos(A.slots[-e - 1].rp);
            m = base ^ (lit & 1);
        }
        A.PO[k] = local_lit(A, m);
    }
}

}  // namespace

int Engine::strash_core(Batch &b, int64_t M, const int *L0, const int *L1, const int *gidA, const int *lidIn,
                        const int *po, bool idOrder, bool removeDangling, bool foldTrivial, bool topo,
                        bool unique, const int *procInv, const int *procPos) {
    const int G = b.G;
    const int64_t nPO = b.nPO;
    cudaStream_t s = s_;
    size_t mark = ar_.used();
    int *cnt = ar_.get<int>(M + 1);
    uint8_t *dead = ar_.get<uint8_t>(M + 1);
    uint8_t *flags = ar_.get<uint8_t>(M + 1);
    uint8_t *liveFlag = ar_.get<uint8_t>(M + 1);
    int *items = ar_.get<int>(M + 1);
    int *level = ar_.get<int>(M + 1);
    int *pending = ar_.get<int>(M + 1);
    int *off = ar_.get<int>(M + 2);
    int *graphLevels = ar_.get<int>(G + 1);
    if (!cnt || !dead || !flags || !liveFlag || !items || !level || !pending || !off || !graphLevels)
        return fail(CULS_E_OOM, "strash: scratch arena exhausted");
    int *qc = counters_;  // [0]=head [1]=tail [2]=done [3]=count [4]=maxLevel [5]=counter
    const unsigned gridM = grid_1d(std::max<int64_t>(M, nPO), kBlock, sms_ * 16);
    const unsigned gridQ = flow_blocks(b.flow_width(), kBlock, (unsigned)(sms_ * 8), sms_);

    // 1. liveness
    check(cudaMemsetAsync(dead, 0, (size_t)M + 1, s), "memset");
    if (removeDangling) {
        check(cudaMemsetAsync(cnt, 0, sizeof(int) * (M + 1), s), "memset");
        k_fanout_count<<<gridM, kBlock, 0, s>>>(M, L0, L1, po, nPO, cnt);
        k_dead_seed_flags<<<gridM, kBlock, 0, s>>>(M, L0, cnt, flags);
        check(fill_i32(items, -1, M + 1, s), "fill");
        check(cudaMemsetAsync(qc, 0, sizeof(int) * 8, s), "memset");
        check(compact_flags(flags, M, items, qc + 1, ar_, s), "compact");
        k_dead_queue<<<gridQ, kBlock, 0, s>>>(WorkQueue{items, qc + 0, qc + 1, qc + 2, (int)(M + 1)}, L0, L1, cnt,
                                              dead, status_);
        launches_ += 4;
    }
    // 2. levels of live AND nodes
    int *liveIdx = nullptr;
    if (topo) {
        liveIdx = ar_.get<int>(M + 1);
        int *done = pending;  // reuse
        if (!liveIdx) return fail(CULS_E_OOM, "strash: scratch arena exhausted");
        ExecCtx X = ctx();
        ChunkSched sched;
        int rc;
        if ((rc = build_chunk_sched(X, b, kBlock, sched))) return rc;
        check(cudaMemsetAsync(qc, 0, sizeof(int) * 8, s), "memset");
        check(cudaMemsetAsync(graphLevels, 0, sizeof(int) * (G + 1), s), "memset");
        check(cudaMemsetAsync(level, 0, sizeof(int) * (M + 1), s), "memset");
        k_live_flags<<<gridM, kBlock, 0, s>>>(M, L0, dead, liveFlag, done);
        check(compact_flags(liveFlag, M, liveIdx, qc + 3, ar_, s), "compact");  // live list and count
        if (prof_) this->mark(kMkLevelK0);
        k_st_levelize<<<gridQ, kBlock, 0, s>>>(sched, L0, L1, liveFlag, gidA, level, done, graphLevels, qc + 5,
                                               qc + 4, status_);
        if (prof_) this->mark(kMkLevelK1);
        launches_ += 2;
    } else {
    // in-order passes over procInv; the worklist below is the fallback if a
    // pass stops making progress (a cycle) or a wait times out, and runs
    // alone when CULS_DEDUP_WORKLIST is set (the tests compare the two)
    bool leveled = false;
    if (procInv && !getenv("CULS_DEDUP_WORKLIST")) {
        liveIdx = ar_.get<int>(M + 1);
        if (!liveIdx) return fail(CULS_E_OOM, "strash: scratch arena exhausted");
        int *done = pending;
        int *lists[2] = {cnt, off};  // free until the levels are known
        int *idx = items;
        check(cudaMemsetAsync(qc, 0, sizeof(int) * 8, s), "memset");
        // qc[7] is these passes' own status word; qc[8] its spin bound
        check(cudaMemcpyAsync(qc + 8, status_ + 1, sizeof(int), cudaMemcpyDeviceToDevice, s), "copy");
        check(cudaMemsetAsync(graphLevels, 0, sizeof(int) * (G + 1), s), "memset");
        check(cudaMemsetAsync(level, 0, sizeof(int) * (M + 1), s), "memset");
        k_live_flags<<<gridM, kBlock, 0, s>>>(M, L0, dead, liveFlag, done);
        check(compact_flags(liveFlag, M, liveIdx, qc + 3, ar_, s), "compact");  // live list and count
        launches_ += 1;
        if (prof_) this->mark(kMkLevelK0);
        const int *list = procInv;
        int64_t n = M;
        for (int pass = 0; pass < 64; pass++) {
            check(cudaMemsetAsync(qc + 5, 0, sizeof(int), s), "memset");
            k_order_levelize<<<gridQ, kBlock, 0, s>>>(n, list, procPos, L0, L1, liveFlag, gidA, level, done,
                                                      graphLevels, qc + 5, qc + 4, qc + 7);
            k_unresolved_flags<<<grid_1d(n, kBlock, sms_ * 16), kBlock, 0, s>>>(n, list, done, flags);
            launches_ += 2;
            check(compact_flags(flags, n, idx, qc + 6, ar_, s), "compact");
            check(cudaMemcpyAsync(hostSmall_, qc, sizeof(int) * 8, cudaMemcpyDeviceToHost, s), "d2h");
            if (int e = sync()) return e;
            const int64_t nu = hostSmall_[6];
            if (hostSmall_[7] != 0) break;  // a wait timed out
            if (nu == 0) {
                leveled = true;
                break;
            }
            if (pass > 0 && nu == n) break;  // no progress
            int *next = lists[pass & 1];
            k_unresolved_next<<<grid_1d(nu, kBlock, sms_ * 16), kBlock, 0, s>>>(nu, idx, list, next, done);
            launches_ += 1;
            list = next;
            n = nu;
        }
        if (leveled) {
            // every live node has its level
            check(cudaMemcpyAsync(qc + 1, qc + 3, sizeof(int), cudaMemcpyDeviceToDevice, s), "copy");
            if (prof_) this->mark(kMkLevelK1);
        }
    }
    if (!leveled) {
    check(cudaMemsetAsync(off, 0, sizeof(int) * (M + 2), s), "memset");
    k_live_degrees<<<gridM, kBlock, 0, s>>>(M, L0, L1, dead, level, off, liveFlag, flags);
    check(scan_exclusive(off, off, M + 1, nullptr, ar_, s), "scan");
    int *cursor = cnt;  // reuse
    check(cudaMemcpyAsync(cursor, off, sizeof(int) * (M + 1), cudaMemcpyDeviceToDevice, s), "copy");
    // number of live edges = off[M]
    check(cudaMemcpyAsync(hostSmall_, off + M, sizeof(int), cudaMemcpyDeviceToHost, s), "d2h");
    if (int e = sync()) return e;
    int64_t nEdges = hostSmall_[0];
    int *adj = ar_.get<int>(nEdges + 1);
    if (!adj) return fail(CULS_E_OOM, "strash: scratch arena exhausted");
    k_csr_fill<<<gridM, kBlock, 0, s>>>(M, L0, L1, liveFlag, cursor, adj);
    liveIdx = ar_.get<int>(M + 1);
    int *ring = ar_.get<int>(8);
    if (!liveIdx || !ring) return fail(CULS_E_OOM, "strash: scratch arena exhausted");
    check(cudaMemsetAsync(qc, 0, sizeof(int) * 8, s), "memset");
    check(cudaMemsetAsync(ring, 0, sizeof(int) * 8, s), "memset");
    check(cudaMemsetAsync(graphLevels, 0, sizeof(int) * (G + 1), s), "memset");
    check(compact_flags(flags, M, items, ring + 1, ar_, s), "compact");     // level 1: the seeds
    check(compact_flags(liveFlag, M, liveIdx, qc + 3, ar_, s), "compact");  // live list and count
    launches_ += 2;
    if (prof_) this->mark(kMkLevelK0);
    // levels in launches of 64, until a level comes out empty; the ring
    // then holds the number of nodes given a level (all live ones unless
    // there is a cycle)
    int L = 1;
    while (true) {
        for (int t = 0; t < 64; t++, L++)
            k_level_step<<<gridQ, kBlock, 0, s>>>(L, items, ring, off, adj, L0, L1, level, gidA, graphLevels, qc + 4);
        launches_ += 64;
        check(cudaMemcpyAsync(hostSmall_, ring, sizeof(int) * 6, cudaMemcpyDeviceToHost, s), "d2h");
        if (int e = sync()) return e;
        if (hostSmall_[L % 3] == 0) break;
    }
    check(cudaMemcpyAsync(qc + 1, ring + 3 + L % 3, sizeof(int), cudaMemcpyDeviceToDevice, s), "copy");
    if (prof_) this->mark(kMkLevelK1);
    }
    }
    // 3. processing order (level, position) and tentative ranks
    check(cudaMemcpyAsync(hostSmall_, qc, sizeof(int) * 8, cudaMemcpyDeviceToHost, s), "d2h");
    if (int e = sync()) return e;
    if (int e = check_status("strash levels")) return e;
    int64_t nLive = hostSmall_[3];
    int maxLevel = hostSmall_[4];
    if (!topo && hostSmall_[1] != nLive) return fail(CULS_E_INVALID, "strash: the AIG has a cycle");
    int *srt = ar_.get<int>(nLive + 1);
    uint32_t *keys = ar_.get<uint32_t>(nLive + 1);
    uint32_t *keys2 = ar_.get<uint32_t>(nLive + 1);
    int *vals2 = ar_.get<int>(nLive + 1);
    int *lvlCnt = ar_.get<int>(maxLevel + 2);
    int *lvlDone = ar_.get<int>(maxLevel + 2);
    int *lvlStart = ar_.get<int>(maxLevel + 2);
    int *chunkCnt = ar_.get<int>(maxLevel + 2);
    int *chunkStart = ar_.get<int>(maxLevel + 2);
    int *tOf = pending;  // reuse
    int *rankOf = off;   // reuse (only needs M entries)
    if (!srt || !keys || !keys2 || !vals2 || !lvlCnt || !lvlDone || !lvlStart || !chunkCnt || !chunkStart)
        return fail(CULS_E_OOM, "strash: arena exhausted");
    check(cudaMemsetAsync(lvlCnt, 0, sizeof(int) * (maxLevel + 2), s), "memset");
    check(cudaMemsetAsync(lvlDone, 0, sizeof(int) * (maxLevel + 2), s), "memset");
    if (nLive > 0) {
        unsigned gl = grid_1d(nLive, kBlock, sms_ * 16);
        k_gather_levels<<<gl, kBlock, 0, s>>>(nLive, liveIdx, level, keys, lvlCnt, maxLevel + 1);
        int bits = 1;
        while ((1ll << bits) <= maxLevel) bits++;
        check(cudaMemcpyAsync(vals2, liveIdx, sizeof(int) * nLive, cudaMemcpyDeviceToDevice, s), "copy");
        check(radix_sort_pairs(keys, vals2, keys2, srt, nLive, bits, ar_, s), "sort");
        k_inverse<<<gl, kBlock, 0, s>>>(nLive, srt, tOf);
        // tentative rank: processing order, or id order for the CPU variants
        k_inverse<<<gl, kBlock, 0, s>>>(nLive, idOrder ? liveIdx : srt, rankOf);
        // level-aligned chunks for the hashing dataflow
        k_level_chunks<<<grid_1d(maxLevel + 1, kBlock, sms_ * 16), kBlock, 0, s>>>(maxLevel + 1, lvlCnt, chunkCnt);
        launches_ += 4;
        check(scan_exclusive(lvlCnt, lvlStart, maxLevel + 1, nullptr, ar_, s), "scan");
        check(scan_exclusive(chunkCnt, chunkStart, maxLevel + 1, chunkStart + maxLevel + 1, ar_, s), "scan");
    }
    // 4. hash: fixed-point rounds or the level dataflow (below)
    uint32_t cap = 1024;
    while (cap < (uint32_t)std::min<int64_t>(nLive * 2, 1ll << 31)) cap <<= 1;
    // CULS_STRASH_TABLE_CAP lowers the capacity (rounded up to a power of
    // two): the tests use it to make the bounded probes run out and check
    // that the call reports CULS_E_PROBE and leaves the graph as it was
    if (const char *env = getenv("CULS_STRASH_TABLE_CAP")) {
        const long long want = atoll(env);
        if (want >= 1) {
            uint32_t c = 1;
            while ((long long)c < want && c < (1u << 31)) c <<= 1;
            cap = std::min(cap, c);
        }
    }
    AndSlot *ts = ar_.get<AndSlot>(cap);
    int *mapEnc = ar_.get<int>(M + 1);
    int *kl0 = ar_.get<int>(nLive + 1), *kl1 = ar_.get<int>(nLive + 1);
    uint8_t *wflags = ar_.get<uint8_t>(nLive + 1);
    int *wl = ar_.get<int>(nLive + 1);
    if (!ts || !mapEnc || !kl0 || !kl1 || !wflags || !wl) return fail(CULS_E_OOM, "strash: arena exhausted");
    check(cudaMemsetAsync(qc + 5, 0, sizeof(int), s), "memset");
    // Rounds (k_round_*) for batches of up to 16M live nodes, where a few
    // full passes cost less than one wait latency per level (the 10M-AND
    // single graph: each strash 22 -> 6 ms); the level dataflow (k_dedup)
    // for larger ones, whose rounds each move gigabytes and whose merges
    // can cascade for many rounds, and whenever the rounds do not settle
    // within kMaxRounds.  CULS_DEDUP_MODE=levels|rounds forces either
    // (the tests run both on the same graphs).
    constexpr int64_t kRoundsMaxLive = 16ll << 20;
    constexpr int kMaxRounds = 24;
    bool useRounds = nLive > 0 && nLive <= kRoundsMaxLive;
    if (const char *env = getenv("CULS_DEDUP_MODE")) {
        if (!strcmp(env, "levels")) useRounds = false;
        if (!strcmp(env, "rounds")) useRounds = nLive > 0;
    }
    bool settled = false;
    hashRounds_ = 0;
    int *slotT = ar_.get<int>(nLive + 1);
    if (!slotT) return fail(CULS_E_OOM, "strash: arena exhausted");
    if (useRounds) {
        int *cur = ar_.get<int>(M + 1), *nxt = ar_.get<int>(M + 1);
        if (!cur || !nxt) return fail(CULS_E_OOM, "strash: arena exhausted");
        const unsigned gl = grid_1d(nLive, kBlock, sms_ * 16);
        if (prof_) this->mark(kMkDedupK0);
        k_round_init<<<gl, kBlock, 0, s>>>(nLive, srt, cur);
        launches_ += 1;
        for (int r = 0; r < kMaxRounds; r++) {
            check(and_table_clear(ts, cap, s), "fill");
            check(cudaMemsetAsync(qc + 16, 0, sizeof(int), s), "memset");
            RoundArgs R{nLive,  srt,   rankOf, L0, L1, gidA, b.dg, AndTable{ts, cap - 1},
                        cur,    nxt,   slotT,  mapEnc, kl0, kl1, foldTrivial ? 1 : 0, unique ? 1 : 0, qc + 16, status_};
            k_round_insert<<<gl, kBlock, 0, s>>>(R);
            k_round_resolve<<<gl, kBlock, 0, s>>>(R);
            launches_ += 2;
            check(cudaMemcpyAsync(hostSmall_ + 16, qc + 16, sizeof(int), cudaMemcpyDeviceToHost, s), "d2h");
            if (int e = sync()) return e;
            if (int e = check_status("strash hashing")) return e;
            std::swap(cur, nxt);
            if (hostSmall_[16] == 0) {
                settled = true;
                hashRounds_ = r + 1;
                break;
            }
        }
        if (prof_) this->mark(kMkDedupK1);
    }
    if (nLive > 0 && !settled) {
        check(and_table_clear(ts, cap, s), "fill");
        DedupArgs A{nLive,      srt,      rankOf,
                    L0,         L1,       level,   lvlCnt,
                    lvlStart,   chunkStart, maxLevel, lvlDone,
                    gidA,       b.dg,     AndTable{ts, cap - 1}, mapEnc,
                    kl0,        kl1,      slotT,   foldTrivial ? 1 : 0, unique ? 1 : 0,
                    qc + 5,     status_};
        if (prof_) this->mark(kMkDedupK0);
        k_dedup<<<gridQ, kBlock, 0, s>>>(A);
        if (prof_) this->mark(kMkDedupK1);
        launches_ += 1;
    }
    if (nLive > 0) {
        k_winner_flags<<<grid_1d(nLive, kBlock, sms_ * 16), kBlock, 0, s>>>(nLive, srt, rankOf, idOrder, slotT, ts, wflags);
        launches_ += 1;
    }
    check(compact_flags(wflags, nLive, wl, qc + 6, ar_, s), "compact");
    // In id order (CPU variants) the winners are ranked by position, not by
    // processing order: sort the winner list by rank.
    check(cudaMemcpyAsync(hostSmall_, qc, sizeof(int) * 8, cudaMemcpyDeviceToHost, s), "d2h");
    if (int e = sync()) return e;
    if (int e = check_status("strash hashing")) return e;
    int64_t nW = hostSmall_[6];
    int *newLocalT = ar_.get<int>(nLive + 1);
    int *cntG = ar_.get<int>(G + 1);
    int *gStart = ar_.get<int>(G + 1);
    int *wlByG = ar_.get<int>(nW + 1);
    uint32_t *wk = ar_.get<uint32_t>(nW + 1), *wk2 = ar_.get<uint32_t>(nW + 1);
    int *wv = ar_.get<int>(nW + 1);
    if (!newLocalT || !cntG || !gStart || !wlByG || !wk || !wk2 || !wv) return fail(CULS_E_OOM, "strash: arena");
    if (idOrder && nW > 0) {
        // re-order winners by id order: key = rank (position order)
        // (ranks fit in 31 bits)
        int bits = 1;
        while ((1ll << bits) <= nLive) bits++;
        k_gather_rank<<<grid_1d(nW, kBlock, sms_ * 16), kBlock, 0, s>>>(nW, wl, srt, rankOf, wk);
        check(cudaMemcpyAsync(wv, wl, sizeof(int) * nW, cudaMemcpyDeviceToDevice, s), "copy");
        check(radix_sort_pairs(wk, wv, wk2, wl, nW, bits, ar_, s), "sort");
        launches_ += 1;
    }
    check(cudaMemsetAsync(cntG, 0, sizeof(int) * (G + 1), s), "memset");
    if (nW > 0) {
        unsigned gw = grid_1d(nW, kBlock, sms_ * 16);
        k_winner_keys<<<gw, kBlock, 0, s>>>(nW, wl, srt, gidA, wk, cntG);
        launches_ += 1;
        if (G > 1) {
            int bits = 1;
            while ((1ll << bits) < G) bits++;
            check(cudaMemcpyAsync(wv, wl, sizeof(int) * nW, cudaMemcpyDeviceToDevice, s), "copy");
            check(radix_sort_pairs(wk, wv, wk2, wlByG, nW, bits, ar_, s), "sort");
        } else {
            check(cudaMemcpyAsync(wlByG, wl, sizeof(int) * nW, cudaMemcpyDeviceToDevice, s), "copy");
        }
    }
    check(scan_exclusive(cntG, gStart, G, nullptr, ar_, s), "scan");
    std::vector<int> hCnt(G), hLev(G);
    check(cudaMemcpyAsync(hCnt.data(), cntG, sizeof(int) * G, cudaMemcpyDeviceToHost, s), "d2h");
    check(cudaMemcpyAsync(hLev.data(), graphLevels, sizeof(int) * G, cudaMemcpyDeviceToHost, s), "d2h");
    if (int e = sync()) return e;
    // new graph table
    std::vector<DevGraph> ng = b.hg;
    int64_t base = 0;
    for (int g = 0; g < G; g++) {
        ng[g].nAnds = hCnt[g];
        // the CPU strash reports maxDelay, -1 without AND nodes
        // (src/aig/strash.cu:396,454)
        ng[g].nLevels = (idOrder && hCnt[g] == 0) ? -1 : hLev[g];
        ng[g].base = (int)base;
        base += 1 + ng[g].nPIs + hCnt[g];
    }
    int64_t nObjNew = base;
    DevGraph *dgNew = reinterpret_cast<DevGraph *>(ar_.get<char>(sizeof(DevGraph) * (G + 1)));
    if (!dgNew) return fail(CULS_E_OOM, "strash: arena");
    // the output goes to the batch's spare buffers, swapped in at the end
    if (!b.pool) b.pool = pool_;
    if (int e = check(b.reserve_spare(nObjNew + 1, nPO + 1), "cudaMalloc")) return e;
    int *F0n = b.F0s, *F1n = b.F1s, *POn = b.POs;
    check(cudaMemcpyAsync(dgNew, ng.data(), sizeof(DevGraph) * G, cudaMemcpyHostToDevice, s), "h2d");
    check(fill_i32(F0n, -1, nObjNew, s), "fill");
    check(fill_i32(F1n, -1, nObjNew, s), "fill");
    if (nW > 0) {
        unsigned gw = grid_1d(nW, kBlock, sms_ * 16);
        k_winner_local<<<gw, kBlock, 0, s>>>(nW, wlByG, srt, gidA, gStart, b.dg, newLocalT);
        launches_ += 1;
    }
    OutArgs O{srt, tOf, gidA, lidIn, L0, kl0, kl1, newLocalT, mapEnc, ts, po, dgNew, F0n, F1n, POn, nPO, G};
    k_strash_out<<<grid_1d(std::max<int64_t>(std::max<int64_t>(nW, nPO), 1), kBlock, sms_ * 16), kBlock, 0, s>>>(nW, wl,
                                                                                                             O);
    launches_ += 1;
    check(cudaMemcpyAsync(b.dg, ng.data(), sizeof(DevGraph) * G, cudaMemcpyHostToDevice, s), "h2d");
    if (int e = sync()) return e;
    b.swap_spare();
    b.hg = ng;
    b.nObj = nObjNew;
    ar_.reset();
    (void)mark;
    return check_status("strash output");
}

namespace {

// AIGMan literals of graph-major arrays to position literals (-1 for the
// constant and PIs), and each position's graph.
__global__ void k_depth_prep(int64_t N, int G, const DevGraph *dg, const int *F0, const int *F1, int *L0, int *L1,
                             int *gid) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += stride) {
        const int g = graph_of_pos(dg, G, (int)p);
        const int base = dg[g].base;
        gid[p] = g;
        if ((int)p - base <= dg[g].nPIs) {
            L0[p] = L1[p] = -1;
        } else {
            L0[p] = F0[p] + 2 * base;
            L1[p] = F1[p] + 2 * base;
        }
    }
}

}  // namespace

// AIGMan::readFromMemory's nLevels for every graph of b (the level of its
// deepest AND node, dangling ones included), by the st levelization.
int Engine::batch_depth(Batch &b) {
    const int64_t N = b.nObj;
    const int G = b.G;
    int rc;
    if ((rc = ensure_arena((size_t)N * 24 + ((size_t)64 << 20)))) return rc;
    ar_.reset();
    int *L0 = ar_.get<int>(N + 1), *L1 = ar_.get<int>(N + 1), *gid = ar_.get<int>(N + 1), *level = ar_.get<int>(N + 1),
        *done = ar_.get<int>(N + 1), *graphLevels = ar_.get<int>(G + 1);
    uint8_t *dead = ar_.get<uint8_t>(N + 1), *live = ar_.get<uint8_t>(N + 1);
    if (!L0 || !L1 || !gid || !level || !done || !graphLevels || !dead || !live)
        return fail(CULS_E_OOM, "depth: arena exhausted");
    cudaStream_t s = s_;
    ExecCtx X = ctx();
    for (auto &g : b.hg) g.cpos = g.base;
    if ((rc = check(cudaMemcpyAsync(b.dg, b.hg.data(), sizeof(DevGraph) * G, cudaMemcpyHostToDevice, s), "h2d")))
        return rc;
    ChunkSched sched;
    if ((rc = build_chunk_sched(X, b, kBlock, sched))) return rc;
    int *qc = counters_;
    if ((rc = check(cudaMemsetAsync(qc, 0, sizeof(int) * 8, s), "memset"))) return rc;
    if ((rc = check(cudaMemsetAsync(graphLevels, 0, sizeof(int) * (G + 1), s), "memset"))) return rc;
    if ((rc = check(cudaMemsetAsync(level, 0, sizeof(int) * (N + 1), s), "memset"))) return rc;
    if ((rc = check(cudaMemsetAsync(dead, 0, (size_t)N + 1, s), "memset"))) return rc;
    k_depth_prep<<<X.grid(N), kBlock, 0, s>>>(N, G, b.dg, b.F0, b.F1, L0, L1, gid);
    k_live_flags<<<X.grid(N), kBlock, 0, s>>>(N, L0, dead, live, done);
    k_st_levelize<<<flow_blocks(b.flow_width(), kBlock, (unsigned)(sms_ * 8), sms_), kBlock, 0, s>>>(sched, L0, L1, live, gid, level, done, graphLevels, qc + 5,
                                                          qc + 4, status_);
    launches_ += 3;
    std::vector<int> hl(G);
    if ((rc = check(cudaMemcpyAsync(hl.data(), graphLevels, sizeof(int) * G, cudaMemcpyDeviceToHost, s), "d2h")))
        return rc;
    if ((rc = sync())) return rc;
    if ((rc = check_status("depth"))) return rc;
    for (int g = 0; g < G; g++) b.hg[g].nLevels = hl[g];
    rc = check(cudaMemcpyAsync(b.dg, b.hg.data(), sizeof(DevGraph) * G, cudaMemcpyHostToDevice, s), "h2d");
    ar_.reset();
    return rc ? rc : sync();
}

}  // namespace culs
