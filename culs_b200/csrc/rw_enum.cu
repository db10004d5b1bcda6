// 4-input cut enumeration with 16-bit truth tables: the B200 form of
// Inputs + CutEnumerate (CULS src/algorithms/rewrite.cu:63-74,268-294).
//
// The reference launches one kernel per level (rewrite.cu:703-704).  Here a
// single persistent dataflow kernel walks the level-major layout in order:
// each thread owns one node, waits (bounded) until both fanins have published
// their cut sets, and replays the reference's per-pair slot policy exactly in
// a private shared-memory copy of its 8 slots.  Pairs whose 32-bit signatures
// already exceed 4 leaves are rejected from the fanins' {sign, packed} words
// before any leaf data is fetched.
#include "rw_work.cuh"

namespace culs {

namespace {

constexpr int kEnumBlock = 128;

struct EnumArgs {
    int64_t nL0, N;
    const int *w0, *w1;
    const int *ref;
    const uint8_t *lidLow;
    int4 *cutL;
    int2 *cutM;
    int *done;
    int *counter;
    int *status;
};

__global__ void k_enum_init(int64_t N, const int *wlev, const int *wl, const uint8_t *lidLow, int4 *cutL, int2 *cutM,
                            int *done) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < N; q += stride) {
        bool lev0 = wlev[q] == 0;
        done[q] = lev0 ? 1 : 0;
        if (lev0 && wl[q] != 0) {  // primary input: the trivial cut only
            Cut c;
            c.leaves[0] = (int)q;
            c.leaves[1] = c.leaves[2] = c.leaves[3] = 0;
            c.sign = 1u << lidLow[q];
            c.tt = 0xAAAAu;
            c.nLeaves = 1;
            c.used = 1;
            c.value = 1001u;  // CutFindValue of a one-leaf cut
            cutL[q * 8] = make_int4(c.leaves[0], 0, 0, 0);
            cutM[q * 8] = make_int2((int)c.sign, (int)cut_pack(c));
        }
    }
}

__device__ __forceinline__ void load_cut(const int4 *cutL, int2 m, int64_t idx, Cut &c) {
    int4 l = __ldcg(&cutL[idx]);
    c.leaves[0] = l.x;
    c.leaves[1] = l.y;
    c.leaves[2] = l.z;
    c.leaves[3] = l.w;
    c.sign = (uint32_t)m.x;
    cut_unpack((uint32_t)m.y, c);
}

__global__ void __launch_bounds__(kEnumBlock) k_enumerate(EnumArgs A) {
    __shared__ Cut sm[kEnumBlock * 8];
    __shared__ int s_chunk;
    Cut *s = &sm[threadIdx.x * 8];
    while (true) {
        if (threadIdx.x == 0) s_chunk = atomicAdd(A.counter, 1);
        __syncthreads();
        int64_t start = A.nL0 + (int64_t)s_chunk * kEnumBlock;
        __syncthreads();
        if (start >= A.N) break;
        int64_t q = start + threadIdx.x;
        if (q >= A.N) continue;
        for (int k = 0; k < 8; k++) s[k].used = 0;
        s[0].leaves[0] = (int)q;
        s[0].leaves[1] = s[0].leaves[2] = s[0].leaves[3] = 0;
        s[0].sign = 1u << A.lidLow[q];
        s[0].tt = 0xAAAAu;
        s[0].nLeaves = 1;
        s[0].used = 1;
        s[0].value = 1001u;
        const int f0 = A.w0[q], f1 = A.w1[q];
        const int u0 = f0 >> 1, u1 = f1 >> 1, c0 = f0 & 1, c1 = f1 & 1;
        bool ok = wait_ge(&A.done[u0], 1, A.status) && wait_ge(&A.done[u1], 1, A.status);
        if (ok) {
            int2 m0[8], m1[8];
#pragma unroll
            for (int k = 0; k < 8; k++) {
                m0[k] = __ldcg(&A.cutM[(int64_t)u0 * 8 + k]);
                m1[k] = __ldcg(&A.cutM[(int64_t)u1 * 8 + k]);
            }
            bool stop = false;
            for (int i = 0; i < 8 && !stop; i++) {
                if (!packed_used((uint32_t)m0[i].y)) continue;
                Cut a;
                load_cut(A.cutL, m0[i], (int64_t)u0 * 8 + i, a);
                for (int j = 0; j < 8; j++) {
                    if (!packed_used((uint32_t)m1[j].y)) continue;
                    if (popc32((uint32_t)m0[i].x | (uint32_t)m1[j].x) > 4) continue;
                    Cut b;
                    load_cut(A.cutL, m1[j], (int64_t)u1 * 8 + j, b);
                    if (enum_pair(s, a, b, c0, c1, A.ref, A.lidLow)) {
                        stop = true;
                        break;
                    }
                }
            }
        }
#pragma unroll
        for (int k = 0; k < 8; k++) {
            A.cutL[q * 8 + k] = make_int4(s[k].leaves[0], s[k].leaves[1], s[k].leaves[2], s[k].leaves[3]);
            A.cutM[q * 8 + k] = make_int2((int)s[k].sign, (int)cut_pack(s[k]));
        }
        __threadfence();
        st_release(&A.done[q], 1);
    }
}

}  // namespace

int rw_enumerate(ExecCtx &X, RwWork &w) {
    const int64_t N = w.N;
    cudaStream_t s = X.s;
    w.cutL = X.ar->get<int4>(N * 8);
    w.cutM = X.ar->get<int2>(N * 8);
    int *done = X.ar->get<int>(N);
    if (!w.cutL || !w.cutM || !done) return X.fail(CULS_E_OOM, "rw: scratch arena exhausted (cuts)");
    int rc;
    if ((rc = X.check(cudaMemsetAsync(w.cutM, 0, sizeof(int2) * N * 8, s), "memset"))) return rc;
    if ((rc = X.check(cudaMemsetAsync(X.counters, 0, sizeof(int) * 4, s), "memset"))) return rc;
    k_enum_init<<<X.grid(N), kBlock, 0, s>>>(N, w.wlev, w.wl, w.lidLow, w.cutL, w.cutM, done);
    EnumArgs A{w.nL0, N, w.w0, w.w1, w.ref, w.lidLow, w.cutL, w.cutM, done, X.counters, X.status};
    X.mark(kMkEnumK0);
    k_enumerate<<<(unsigned)(X.sms * 6), kEnumBlock, 0, s>>>(A);
    X.mark(kMkEnumK1);
    X.launched(2);
    if ((rc = X.check(cudaGetLastError(), "enumerate launch"))) return rc;
    return 0;
}

}  // namespace culs
