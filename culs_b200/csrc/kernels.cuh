// Kernel-side helpers shared by the engine's translation units.
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"
#include "engine.cuh"

namespace culs {

constexpr int kBlock = 256;

// Graph owning a position in a graph-major layout (bases increase strictly).
__device__ __forceinline__ int graph_of_pos(const DevGraph *g, int G, int p) {
    int lo = 0, hi = G - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (g[mid].base <= p)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Graph owning PO index k (poOff non-decreasing; empty graphs share an offset
// with the next graph, so the last graph with poOff <= k owns k).
__device__ __forceinline__ int graph_of_po(const DevGraph *g, int G, int k) {
    int lo = 0, hi = G - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (g[mid].poOff <= k)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Work queue shared by the persistent worklist kernels.  items[] starts at -1
// beyond the seeds; tail counts pushed items, done counts processed ones.
struct WorkQueue {
    int *items;
    int *head;
    int *tail;
    int *done;
    int cap;
};

// ------------------------------------------------ warp-aggregated atomics
// Per-item atomics on a handful of hot addresses (a level's completion
// counter, a queue tail, a graph's counter) serialise in L2; these helpers
// issue one atomic per group of converged lanes that share the address.

// atomicAdd(&base[key], v), one atomic per group of lanes with equal key.
__device__ __forceinline__ void agg_add(int *base, int key, int v) {
    const unsigned mask = __activemask();
    const unsigned peers = __match_any_sync(mask, key);
    const int sum = __reduce_add_sync(peers, v);
    if ((int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&base[key], sum);
}

// atomicMax(&base[key], v), one atomic per group of lanes with equal key.
__device__ __forceinline__ void agg_max(int *base, int key, int v) {
    const unsigned mask = __activemask();
    const unsigned peers = __match_any_sync(mask, key);
    const int mx = __reduce_max_sync(peers, v);
    if ((int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicMax(&base[key], mx);
}

// agg_add for a completion counter: every lane's earlier writes are visible
// (at GPU scope) before the group's single increment is.
__device__ __forceinline__ void agg_add_release(int *base, int key, int v) {
    __threadfence();
    const unsigned mask = __activemask();
    const unsigned peers = __match_any_sync(mask, key);
    const int sum = __reduce_add_sync(peers, v);
    __syncwarp(peers);
    if ((int)(threadIdx.x & 31) == __ffs(peers) - 1) {
        __threadfence();
        atomicAdd(&base[key], sum);
    }
}

// Pushes v (when v >= 0) of every lane; all 32 lanes of the warp must call it
// together.  One tail reservation per warp.
__device__ __forceinline__ void queue_push_warp(const WorkQueue &q, int v) {
    const unsigned b = __ballot_sync(0xffffffffu, v >= 0);
    if (!b) return;
    const int lane = threadIdx.x & 31;
    int base = 0;
    if (lane == 0) base = atomicAdd(q.tail, __popc(b));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (v >= 0) {
        __threadfence();
        st_release(&q.items[base + __popc(b & ((1u << lane) - 1u))], v);
    }
}

// Counts the items this warp finished (lanes with `finished`); all 32 lanes
// call it after their pushes, so tail never lags done.
__device__ __forceinline__ void queue_done_warp(const WorkQueue &q, bool finished) {
    const unsigned b = __ballot_sync(0xffffffffu, finished);
    __syncwarp();
    if (b && (threadIdx.x & 31) == 0) {
        __threadfence();
        atomicAdd(q.done, __popc(b));
    }
}

// Warp-cooperative, non-blocking pop; all 32 lanes call it together.  Each
// lane keeps the queue index it claimed in h (-1: claim a new one) and fin
// (true once the queue is drained for it).  Returns the lane's item, or -1
// when it has none this round.  A lane never blocks on its own index, so a
// lane whose item is pushed by a warp-mate cannot stall that warp-mate.
__device__ __forceinline__ int queue_try_pop_warp(const WorkQueue &q, int &h, bool &fin) {
    const int lane = threadIdx.x & 31;
    const unsigned need = __ballot_sync(0xffffffffu, !fin && h < 0);
    if (need) {
        int base = 0;
        if (lane == 0) base = atomicAdd(q.head, __popc(need));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (!fin && h < 0) h = base + __popc(need & ((1u << lane) - 1u));
    }
    if (fin) return -1;
    if (h < q.cap) {
        const int v = ld_acquire(&q.items[h]);
        if (v >= 0) {
            h = -1;
            return v;
        }
    }
    // drained: every pushed item is processed and this index lies beyond them
    const int d = ld_acquire(q.done);
    const int t = ld_acquire(q.tail);
    if (d == t && h >= t) fin = true;
    return -1;
}

// End-of-round bookkeeping of a worklist warp: returns true when the warp
// must leave (all lanes drained; the status word already holds an error; or
// no progress for spin_limit(status) rounds, which is recorded in *status).
// The decision is uniform across the warp.
__device__ __forceinline__ bool queue_round_end(bool fin, bool progressed, int64_t &idle, int *status) {
    if (__all_sync(0xffffffffu, fin)) return true;
    if (__any_sync(0xffffffffu, progressed)) {
        idle = 0;
        return false;
    }
    int failed = (threadIdx.x & 31) == 0 ? (ld_cg(status) != kDevOk) : 0;
    if (__shfl_sync(0xffffffffu, failed, 0)) return true;
    if (++idle > spin_limit(status)) {
        if ((threadIdx.x & 31) == 0) set_status(status, kDevWaitTimeout);
        return true;
    }
    backoff(idle);
    return false;
}

// Per-block histogram of small keys in shared memory (a few hundred levels
// for millions of nodes: global counters would serialise in L2).  Usage, by
// every thread of the block: hist_begin, hist_add per key, hist_end.  With
// nBins > kHistBins the keys go straight to the global counters.
constexpr int kHistBins = 4096;
__device__ __forceinline__ void hist_begin(int *h, int nBins) {
    if (nBins <= kHistBins)
        for (int i = threadIdx.x; i < nBins; i += blockDim.x) h[i] = 0;
    __syncthreads();
}
__device__ __forceinline__ void hist_add(int *h, int nBins, int *global, int key) {
    if (nBins <= kHistBins)
        atomicAdd(&h[key], 1);
    else
        agg_add(global, key, 1);
}
__device__ __forceinline__ void hist_end(const int *h, int nBins, int *global) {
    __syncthreads();
    if (nBins <= kHistBins)
        for (int i = threadIdx.x; i < nBins; i += blockDim.x)
            if (h[i]) atomicAdd(&global[i], h[i]);
}

// Blocks for a persistent dataflow kernel over a batch `width` nodes wide
// (Batch::flow_width): enough for about sixteen levels' worth of nodes in
// flight at itemsPerBlock nodes per block, at least minBlocks (one per SM:
// a narrow graph's waits still spread over the SMs), at most `full`.  A
// narrow, deep batch then leaves the rest of the GPU to other streams (the
// served mode runs several batches at once) instead of filling every SM with
// blocks that wait on its critical path.  Any grid is correct: chunks are
// claimed in order by running blocks.
inline unsigned flow_blocks(int64_t width, int itemsPerBlock, unsigned full, int minBlocks) {
    int64_t b = (16 * width + itemsPerBlock - 1) / itemsPerBlock;
    if (b < minBlocks) b = minBlocks;
    return (unsigned)(b < (int64_t)full ? b : (int64_t)full);
}

inline unsigned grid_1d(int64_t n, int block = kBlock, int maxBlocks = 1 << 20) {
    int64_t b = (n + block - 1) / block;
    if (b < 1) b = 1;
    if (b > maxBlocks) b = maxBlocks;
    return (unsigned)b;
}

}  // namespace culs
