// Existence table and per-node evaluation: BuildHashTable + EvaluateNode
// (CULS src/algorithms/rewrite.cu:378-471).  One thread per AND node; the
// 54-entry match/level scratch of EvaluateNode lives in shared memory.  The
// chained table of the reference becomes an open-addressing table on 64-bit
// CAS keys (fanin0 id, fanin1 id, compl0, compl1).
#include "rw_work.cuh"

namespace culs {

namespace {

constexpr int kEvalBlock = 64;

__global__ void k_table_build(int64_t nL0, int64_t N, const int *w0, const int *w1, const int *wg, const DevGraph *dg,
                              AndTable tab, int *status) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t q = nL0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < N; q += stride) {
        int f0 = w0[q], f1 = w1[q];
        int cp = dg[wg[q]].cpos;
        // rewrite.cu:454 skips nodes whose fanins are both the constant
        if ((f0 >> 1) == cp && (f1 >> 1) == cp) continue;
        table_insert(tab, and_key(f0 >> 1, f1 >> 1, f0 & 1, f1 & 1), (int)q, status);
    }
}

struct EvalArgs {
    int64_t nL0, N;
    EvalIn E;
    const int4 *cutL;
    const int2 *cutM;
    const int *wg;
    const DevGraph *dg;
    int useZeros;
    int8_t *bestCut;
    uint8_t *bestOut;
    uint8_t *candFlag;
};

__global__ void __launch_bounds__(kEvalBlock) k_evaluate(EvalArgs A) {
    __shared__ int s_match[kEvalBlock * 54];
    __shared__ int s_mlev[kEvalBlock * 54];
    int *match = &s_match[threadIdx.x * 54];
    int *mlev = &s_mlev[threadIdx.x * 54];
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t q = A.nL0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < A.N; q += stride) {
        Cut cuts[8];
        bool any = false;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            int2 m = A.cutM[q * 8 + k];
            cut_unpack((uint32_t)m.y, cuts[k]);
            cuts[k].sign = (uint32_t)m.x;
            if (cuts[k].used && cuts[k].nLeaves >= 3) {
                int4 l = A.cutL[q * 8 + k];
                cuts[k].leaves[0] = l.x;
                cuts[k].leaves[1] = l.y;
                cuts[k].leaves[2] = l.z;
                cuts[k].leaves[3] = l.w;
                any = true;
            }
        }
        int bc = -1, bo = -1;
        if (any) eval_node(A.E, (int)q, A.dg[A.wg[q]].cpos, cuts, A.useZeros != 0, match, mlev, bc, bo);
        A.bestCut[q] = (int8_t)bc;
        A.bestOut[q] = (uint8_t)(bo < 0 ? 0 : bo);
        A.candFlag[q] = bc >= 0;
    }
}

}  // namespace

int rw_evaluate(ExecCtx &X, RwWork &w) {
    const int64_t N = w.N;
    cudaStream_t s = X.s;
    int64_t nAnd = N - w.nL0;
    uint32_t cap = 1024;
    while ((int64_t)cap < nAnd * 2 && cap < (1u << 31)) cap <<= 1;
    unsigned long long *tk = X.ar->get<unsigned long long>(cap);
    int *tv = X.ar->get<int>(cap);
    w.bestCut = X.ar->get<int8_t>(N);
    w.bestOut = X.ar->get<uint8_t>(N);
    uint8_t *candFlag = X.ar->get<uint8_t>(N);
    w.cand = X.ar->get<int>(N);
    if (!tk || !tv || !w.bestCut || !w.bestOut || !candFlag || !w.cand)
        return X.fail(CULS_E_OOM, "rw: scratch arena exhausted (table)");
    w.tab = AndTable{tk, tv, cap - 1};
    int rc;
    if ((rc = X.check(cudaMemsetAsync(tk, 0xFF, sizeof(unsigned long long) * cap, s), "memset"))) return rc;
    if ((rc = X.check(cudaMemsetAsync(tv, 0x7F, sizeof(int) * cap, s), "memset"))) return rc;
    if ((rc = X.check(cudaMemsetAsync(w.bestCut, 0xFF, N, s), "memset"))) return rc;
    if ((rc = X.check(cudaMemsetAsync(candFlag, 0, N, s), "memset"))) return rc;
    if (nAnd > 0) {
        k_table_build<<<X.grid(nAnd), kBlock, 0, s>>>(w.nL0, N, w.w0, w.w1, w.wg, w.dg, w.tab, X.status);
        EvalArgs A{w.nL0, N, EvalIn{w.w0, w.w1, w.ref, w.wlev, X.lib, w.tab, X.status}, w.cutL, w.cutM, w.wg, w.dg,
                   w.useZeros ? 1 : 0, w.bestCut, w.bestOut, candFlag};
        X.mark(kMkEvalK0);
        k_evaluate<<<X.grid(nAnd, kEvalBlock), kEvalBlock, 0, s>>>(A);
        X.mark(kMkEvalK1);
        X.launched(2);
    }
    if ((rc = X.check(compact_flags(candFlag, N, w.cand, X.counters + 8, *X.ar, s), "compact"))) return rc;
    if ((rc = X.check(cudaMemcpyAsync(X.hostSmall + 8, X.counters + 8, sizeof(int), cudaMemcpyDeviceToHost, s), "d2h")))
        return rc;
    if ((rc = X.sync())) return rc;
    if ((rc = X.status_check("rw evaluate"))) return rc;
    w.nCand = X.hostSmall[8];
    return 0;
}

}  // namespace culs
