// Interleaved chunk schedule for in-order dataflow passes over a graph-major
// batch.
//
// A dataflow pass claims fixed-size chunks in increasing order, and every
// node waits (bounded) for its fanins, which sit at lower positions of the
// same graph.  Claiming the batch's positions in plain graph-major order
// keeps the in-flight window inside one or two graphs, so the pass advances
// about one graph layer per wait latency.  This schedule claims chunk k of
// every graph before chunk k+1 of any graph (graphs with more chunks first
// within a round): a chunk's fanins lie in chunks of the same graph with a
// lower or equal round, which were claimed before it, so no claimed chunk
// ever waits on an unclaimed one, and the window spans many graphs.
#pragma once

#include <cstdint>

#include "engine.cuh"

namespace culs {

struct ChunkSched {
    const DevGraph *dg = nullptr;
    const int *order = nullptr;          // graph ids, most chunks first
    const int64_t *roundStart = nullptr; // K + 1 prefix counts of chunks per round
    int K = 0;                           // rounds (chunks of the largest graph)
    int chunk = 256;
    int64_t total = 0;                   // chunks over all graphs
};

// Positions [begin, end) of schedule entry c (0 <= c < total).
__device__ __forceinline__ void sched_chunk(const ChunkSched &S, int64_t c, int64_t &begin, int64_t &end) {
    int lo = 0, hi = S.K - 1;
    while (lo < hi) {  // last round with roundStart <= c
        int mid = (lo + hi + 1) >> 1;
        if (S.roundStart[mid] <= c)
            lo = mid;
        else
            hi = mid - 1;
    }
    const int g = S.order[c - S.roundStart[lo]];
    const DevGraph d = S.dg[g];
    begin = (int64_t)d.base + (int64_t)lo * S.chunk;
    end = (int64_t)d.base + 1 + d.nPIs + d.nAnds;
    if (end > begin + S.chunk) end = begin + S.chunk;
}

struct ExecCtx;
struct Batch;
// Builds the schedule of batch b (object counts from the host graph table)
// into the context's arena and copies it to the device on the context's
// stream.  Returns a CULS status.
int build_chunk_sched(ExecCtx &X, const Batch &b, int chunk, ChunkSched &S);

}  // namespace culs
