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

__device__ __forceinline__ void queue_push(const WorkQueue &q, int v) {
    int t = atomicAdd(q.tail, 1);
    __threadfence();
    st_release(&q.items[t], v);
}

// Each lane takes one queue index; returns -1 when the queue is drained (or a
// wait expired, recorded in *status).
__device__ __forceinline__ int queue_pop_wait(const WorkQueue &q, int h, int *status) {
    int64_t it = 0;
    while (true) {
        if (h < q.cap) {
            int v = ld_acquire(&q.items[h]);
            if (v >= 0) return v;
        }
        int d = ld_acquire(q.done);
        int t = ld_acquire(q.tail);
        if (d == t && h >= t) return -1;
        if (++it > kSpinLimit) {
            set_status(status, kDevWaitTimeout);
            return -1;
        }
        backoff(it);
    }
}

inline unsigned grid_1d(int64_t n, int block = kBlock, int maxBlocks = 1 << 20) {
    int64_t b = (n + block - 1) / block;
    if (b < 1) b = 1;
    if (b > maxBlocks) b = maxBlocks;
    return (unsigned)b;
}

}  // namespace culs
