// Front of the rewriting pass: CPUSolver::Reset + Reorder + Init
// (CULS src/algorithms/rewrite.cu:780-809,1229-1279, rewrite.h:291-307).
//
//  * literals switch to the AIGER constant convention (invertConstTrueFalse,
//    src/common.h:24-27);
//  * ASAP levels and phases (value under the all-zero input) come from one
//    in-order dataflow pass over the graph-major input, whose ids are
//    topological, instead of the reference's recursive TopoSort;
//  * a stable radix sort by level yields the level-major working layout, in
//    which each graph's nodes appear in (level, old id) order -- exactly the
//    renumbering of Reorder, since that sort is stable by old id;
//  * fanins are re-pointed, oriented (lit0 <= lit1) and counted into refs
//    together with the PO references.
#include <algorithm>

#include "rw_work.cuh"
#include "sched.cuh"

namespace culs {

namespace {

__global__ void k_front_load(int64_t N, int G, const DevGraph *dg, const int *F0, const int *F1, int *gidIn, int *a0,
                             int *a1, int *lp) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += stride) {
        int g = graph_of_pos(dg, G, (int)p);
        int base = dg[g].base;
        int local = (int)p - base;
        gidIn[p] = g;
        if (local <= dg[g].nPIs) {
            a0[p] = a1[p] = 2 * base;
            lp[p] = 0;
        } else {
            int l0 = F0[p], l1 = F1[p];
            l0 = l0 < 2 ? 1 - l0 : l0;
            l1 = l1 < 2 ? 1 - l1 : l1;
            a0[p] = l0 + 2 * base;
            a1[p] = l1 + 2 * base;
            lp[p] = -1;
        }
    }
}

// lp = 2*level + phase, -1 until known: the word a node publishes and its
// fanouts wait on.  Fanins precede their node inside its graph, and the
// chunks are claimed in the interleaved schedule order (sched.cuh), so a
// claimed chunk never waits on an unclaimed one.
__global__ void __launch_bounds__(kBlock) k_front_levelize(ChunkSched S, const int *a0, const int *a1, int *lp,
                                                            int *counter, int *maxLevel, int *status) {
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
        int64_t p = begin + threadIdx.x;
        if (p >= end || lp[p] != -1) continue;
        int f0 = a0[p], f1 = a1[p];
        int u0 = f0 >> 1, u1 = f1 >> 1;
        int x0, x1;
        if (!wait_word(&lp[u0], 0, status, &x0) || !wait_word(&lp[u1], 0, status, &x1)) continue;
        int lv = 1 + max(x0 >> 1, x1 >> 1);
        int ph = ((x0 & 1) ^ (f0 & 1)) & ((x1 & 1) ^ (f1 & 1));
        st_relaxed(&lp[p], 2 * lv + ph);
        myMax = lv > myMax ? lv : myMax;
    }
    // every thread of the block leaves the loop at the same claim
    myMax = __reduce_max_sync(0xffffffffu, myMax);
    if ((threadIdx.x & 31) == 0 && myMax > 0) atomicMax(maxLevel, myMax);
}

__global__ void k_front_keys(int64_t N, const int *lp, uint32_t *keys, int *vals) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += stride) {
        keys[p] = (uint32_t)(lp[p] >> 1);
        vals[p] = (int)p;
    }
}

__global__ void k_front_keys_gid(int64_t N, const int *wg, uint32_t *keys, int *vals) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < N; q += stride) {
        keys[q] = (uint32_t)wg[q];
        vals[q] = (int)q;
    }
}

__global__ void k_front_inverse(int64_t N, const int *order, int *newPos) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < N; q += stride) newPos[order[q]] = (int)q;
}

__global__ void k_front_permute(int64_t N, const int *order, const int *newPos, const int *gidIn, const int *a0,
                                const int *a1, const int *lp, DevGraph *dg, int *w0, int *w1, int *wg, int *wlev,
                                uint8_t *wph) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < N; q += stride) {
        int p = order[q];
        int g = gidIn[p];
        int x0 = a0[p], x1 = a1[p];
        int n0 = 2 * newPos[x0 >> 1] + (x0 & 1);
        int n1 = 2 * newPos[x1 >> 1] + (x1 & 1);
        if (n0 > n1) {  // rw::CPUSolver::Init orientation, rewrite.cu:1230-1232
            int t = n0;
            n0 = n1;
            n1 = t;
        }
        w0[q] = n0;
        w1[q] = n1;
        wg[q] = g;
        wlev[q] = lp[p] >> 1;
        wph[q] = (uint8_t)(lp[p] & 1);
        if (p == dg[g].base) dg[g].cpos = (int)q;
    }
}

__global__ void k_front_local_ids(int64_t N, const int *byGraph, const int *wg, const DevGraph *dg, int *wl,
                                  uint8_t *lidLow) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += stride) {
        int q = byGraph[i];
        int l = (int)i - dg[wg[q]].base;
        wl[q] = l;
        lidLow[q] = (uint8_t)(l & 31);
    }
}

__global__ void k_front_po(int64_t nPO, int G, const DevGraph *dg, const int *PO, const int *newPos, int *wpo) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nPO; k += stride) {
        int g = graph_of_po(dg, G, (int)k);
        int l = PO[k];
        l = l < 2 ? 1 - l : l;
        wpo[k] = 2 * newPos[dg[g].base + (l >> 1)] + (l & 1);
    }
}

__global__ void k_front_refs(int64_t N, const int *w0, const int *w1, const int *wlev, int64_t nPO, const int *wpo,
                             int *ref) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < N; q += stride) {
        if (wlev[q] == 0) continue;
        atomicAdd(&ref[w0[q] >> 1], 1);
        atomicAdd(&ref[w1[q] >> 1], 1);
    }
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nPO; k += stride) atomicAdd(&ref[wpo[k] >> 1], 1);
}

}  // namespace

int rw_front(ExecCtx &X, Batch &b, RwWork &w) {
    w.width = b.flow_width();
    const int64_t N = b.nObj;
    const int G = b.G;
    cudaStream_t s = X.s;
    Arena &ar = *X.ar;
    w.G = G;
    w.dg = b.dg;
    w.N = N;
    w.nPO = b.nPO;
    w.nL0 = 0;
    for (int g = 0; g < G; g++) w.nL0 += 1 + b.hg[g].nPIs;

    int *gidIn = ar.get<int>(N), *a0 = ar.get<int>(N), *a1 = ar.get<int>(N), *lp = ar.get<int>(N);
    int *done = ar.get<int>(N), *order = ar.get<int>(N), *newPos = ar.get<int>(N);
    uint32_t *keys = ar.get<uint32_t>(N), *keys2 = ar.get<uint32_t>(N);
    int *vals = ar.get<int>(N);
    w.w0 = ar.get<int>(N);
    w.w1 = ar.get<int>(N);
    w.wg = ar.get<int>(N);
    w.wl = ar.get<int>(N);
    w.wlev = ar.get<int>(N);
    w.wph = ar.get<uint8_t>(N);
    w.lidLow = ar.get<uint8_t>(N);
    w.ref = ar.get<int>(N);
    w.wpo = ar.get<int>(b.nPO + 1);
    if (!gidIn || !a0 || !a1 || !lp || !done || !order || !newPos || !keys || !keys2 || !vals || !w.w0 || !w.w1 ||
        !w.wg || !w.wl || !w.wlev || !w.wph || !w.lidLow || !w.ref || !w.wpo)
        return X.fail(CULS_E_OOM, "rw: scratch arena exhausted (front)");
    int *cnt = X.counters;
    int rc;
    if ((rc = X.check(cudaMemsetAsync(cnt, 0, sizeof(int) * 8, s), "memset"))) return rc;
    ChunkSched sched;
    if ((rc = build_chunk_sched(X, b, kBlock, sched))) return rc;
    k_front_load<<<X.grid(N), kBlock, 0, s>>>(N, G, b.dg, b.F0, b.F1, gidIn, a0, a1, lp);
    k_front_levelize<<<flow_blocks(w.width, kBlock, (unsigned)(X.sms * 8), X.sms), kBlock, 0, s>>>(sched, a0, a1, lp, cnt + 0, cnt + 1, X.status);
    k_front_keys<<<X.grid(N), kBlock, 0, s>>>(N, lp, keys, vals);
    X.launched(3);
    if ((rc = X.check(cudaMemcpyAsync(X.hostSmall, cnt, sizeof(int) * 8, cudaMemcpyDeviceToHost, s), "d2h"))) return rc;
    if ((rc = X.sync())) return rc;
    if ((rc = X.status_check("rw levelize"))) return rc;
    w.maxLevel = X.hostSmall[1];
    int bits = 1;
    while ((1ll << bits) <= w.maxLevel) bits++;
    if ((rc = X.check(radix_sort_pairs(keys, vals, keys2, order, N, bits, ar, s), "sort"))) return rc;
    k_front_inverse<<<X.grid(N), kBlock, 0, s>>>(N, order, newPos);
    k_front_permute<<<X.grid(N), kBlock, 0, s>>>(N, order, newPos, gidIn, a0, a1, lp, b.dg, w.w0, w.w1, w.wg, w.wlev,
                                                  w.wph);
    X.launched(2);
    // local ids: rank of each W position among its graph's positions
    int *byGraph = done;  // reuse
    if (G == 1) {
        if ((rc = X.check(iota_i32(byGraph, 0, N, s), "iota"))) return rc;
    } else {
        int gb = 1;
        while ((1ll << gb) < G) gb++;
        // keys = graph id of W position q, values = q
        k_front_keys_gid<<<X.grid(N), kBlock, 0, s>>>(N, w.wg, keys, vals);
        X.launched(1);
        if ((rc = X.check(radix_sort_pairs(keys, vals, keys2, byGraph, N, gb, ar, s), "sort"))) return rc;
    }
    w.byGraph = byGraph;
    k_front_local_ids<<<X.grid(N), kBlock, 0, s>>>(N, byGraph, w.wg, b.dg, w.wl, w.lidLow);
    if (b.nPO > 0) k_front_po<<<X.grid(b.nPO), kBlock, 0, s>>>(b.nPO, G, b.dg, b.PO, newPos, w.wpo);
    if ((rc = X.check(cudaMemsetAsync(w.ref, 0, sizeof(int) * N, s), "memset"))) return rc;
    k_front_refs<<<X.grid(std::max<int64_t>(N, b.nPO)), kBlock, 0, s>>>(N, w.w0, w.w1, w.wlev, b.nPO, w.wpo, w.ref);
    X.launched(3);
    // graph table now carries the constant positions of W
    if ((rc = X.check(cudaMemcpyAsync(b.hg.data(), b.dg, sizeof(DevGraph) * G, cudaMemcpyDeviceToHost, s), "d2h")))
        return rc;
    return X.sync();
}

}  // namespace culs
