// Host side of the interleaved chunk schedule (sched.cuh).
#include <algorithm>
#include <numeric>
#include <vector>

#include "rw_work.cuh"
#include "sched.cuh"

namespace culs {

int build_chunk_sched(ExecCtx &X, const Batch &b, int chunk, ChunkSched &S) {
    const int G = b.G;
    std::vector<int64_t> nChunks(G);
    for (int g = 0; g < G; g++) {
        const int64_t objs = 1 + (int64_t)b.hg[g].nPIs + b.hg[g].nAnds;
        nChunks[g] = (objs + chunk - 1) / chunk;
    }
    std::vector<int> order(G);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return nChunks[x] > nChunks[y]; });
    const int64_t K = G ? nChunks[order[0]] : 0;
    std::vector<int64_t> roundStart(K + 1);
    int64_t acc = 0;
    int live = G;  // graphs with more than k chunks
    for (int64_t k = 0; k < K; k++) {
        while (live > 0 && nChunks[order[live - 1]] <= k) live--;
        roundStart[k] = acc;
        acc += live;
    }
    roundStart[K] = acc;
    int *dOrder = X.ar->get<int>(std::max(G, 1));
    int64_t *dRound = X.ar->get<int64_t>(K + 1);
    if (!dOrder || !dRound) return X.fail(CULS_E_OOM, "scratch arena exhausted (chunk schedule)");
    int rc;
    if (G && (rc = X.check(cudaMemcpyAsync(dOrder, order.data(), sizeof(int) * G, cudaMemcpyHostToDevice, X.s),
                           "h2d")))
        return rc;
    if ((rc = X.check(cudaMemcpyAsync(dRound, roundStart.data(), sizeof(int64_t) * (K + 1), cudaMemcpyHostToDevice,
                                      X.s),
                      "h2d")))
        return rc;
    S.dg = b.dg;
    S.order = dOrder;
    S.roundStart = dRound;
    S.K = (int)K;
    S.chunk = chunk;
    S.total = acc;
    return 0;
}

}  // namespace culs
