// 4-input cut enumeration with 16-bit truth tables: the B200 form of
// Inputs + CutEnumerate (CULS src/algorithms/rewrite.cu:63-74,268-294).
//
// The reference launches one kernel per level (rewrite.cu:703-704).  Here a
// single persistent dataflow kernel walks the level-major layout in order:
// each thread owns one node, waits (bounded) until both fanins have published
// their cut sets, and replays the reference's per-pair slot policy exactly.
// The 8 slots live in registers (fully unrolled slot loops), and every cut
// record carries its leaves' reference counts and local-id bits (cutA), so a
// node reads nothing but its two fanins' 16 cut records.  Pairs whose 32-bit
// signatures already exceed 4 leaves are rejected from the fanins' {sign,
// packed} words before any leaf data is fetched.
#include "enum_regs.cuh"
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
    int2 *cutA;
    int *done;
    int *counter;
    int *status;
};

__device__ __forceinline__ uint32_t clamp_ref(int r) { return r > 1001 ? 1001u : (uint32_t)r; }

__global__ void k_enum_init(int64_t N, const int *wlev, const int *wl, const uint8_t *lidLow, const int *ref,
                            int4 *cutL, int2 *cutM, int2 *cutA, int *done) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < N; q += stride) {
        bool lev0 = wlev[q] == 0;
        done[q] = lev0 ? 1 : 0;
        if (lev0 && wl[q] != 0) {  // primary input: the trivial cut only
            Cut c;
            c.sign = 1u << lidLow[q];
            c.tt = 0xAAAAu;
            c.nLeaves = 1;
            c.used = 1;
            c.value = 1001u;  // CutFindValue of a one-leaf cut
            cutL[q * 8] = make_int4((int)q, 0, 0, 0);
            cutM[q * 8] = make_int2((int)c.sign, (int)cut_pack(c));
            cutA[q * 8] = make_int2((int)clamp_ref(ref[q]), (int)((uint32_t)lidLow[q] << 12));
        }
    }
}

// A slot in registers: leaves, signature, packed tt/value/nLeaves/used.  The
// slot's aux word is written straight to cutA when the slot is filled: this
// node never reads it back.
struct Slot {
    int l[4];
    uint32_t sign, pk;
};

__device__ __forceinline__ uint32_t sl_n(const Slot &s) { return packed_nleaves(s.pk); }
__device__ __forceinline__ uint32_t sl_used(const Slot &s) { return packed_used(s.pk); }
__device__ __forceinline__ uint32_t sl_value(const Slot &s) { return (s.pk >> 16) & 0x7FFu; }
__device__ __forceinline__ void sl_clear_used(Slot &s) { s.pk &= ~(1u << 30); }

// every leaf of (al, an) appears among the leaves of (bl, bn)
__device__ __forceinline__ bool leaves_subset(const int (&al)[4], uint32_t an, const int (&bl)[4], uint32_t bn) {
    bool all = true;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        bool in = false;
#pragma unroll
        for (int j = 0; j < 4; j++) in |= ((uint32_t)j < bn) && bl[j] == al[i];
        all &= ((uint32_t)i >= an) || in;
    }
    return all;
}

// CutFilter (rewrite.cu:178-193) for the cut X sitting in slot id: visits the
// other used slots in index order, drops larger slots that contain X and
// stops (dropping X) at the first slot contained in X.
__device__ __forceinline__ bool filter_slots(Slot (&S)[8], int id, const int (&xl)[4], uint32_t xn, uint32_t xs) {
    bool dropped = false;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        if (dropped || k == id || !sl_used(S[k])) continue;
        const uint32_t kn = sl_n(S[k]);
        if (kn > xn) {
            if ((S[k].sign & xs) == xs && leaves_subset(xl, xn, S[k].l, kn)) sl_clear_used(S[k]);
        } else {
            if ((S[k].sign & xs) == S[k].sign && leaves_subset(S[k].l, kn, xl, xn)) dropped = true;
        }
    }
    return dropped;
}

__device__ __forceinline__ void load_rcut(const EnumArgs &A, int64_t idx, int2 m, RCut &c) {
    int4 l = A.cutL[idx];
    int2 x = A.cutA[idx];
    c.l[0] = l.x;
    c.l[1] = l.y;
    c.l[2] = l.z;
    c.l[3] = l.w;
    c.sign = (uint32_t)m.x;
    c.tt = (uint32_t)m.y & 0xFFFFu;
    c.n = packed_nleaves((uint32_t)m.y);
    c.used = 1;
    rc_unpack_aux((uint32_t)x.x, (uint32_t)x.y, c);
}

// Warps claim 32 consecutive positions at a time.  A lane publishes its node
// before it next waits on its warp, and fanins lie at lower positions, so a
// lane never waits on a warp-mate that waits on it.
__global__ void __launch_bounds__(kEnumBlock, 4) k_enumerate(EnumArgs A) {
    const int lane = threadIdx.x & 31;
    while (true) {
        int chunk = 0;
        if (lane == 0) chunk = atomicAdd(A.counter, 1);
        chunk = __shfl_sync(0xffffffffu, chunk, 0);
        const int64_t start = A.nL0 + (int64_t)chunk * 32;
        if (start >= A.N) break;
        const int64_t q = start + lane;
        if (q >= A.N) continue;
        Slot S[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            S[k].pk = 0;
            S[k].sign = 0;
            S[k].l[0] = S[k].l[1] = S[k].l[2] = S[k].l[3] = 0;
        }
        {
            Cut c;
            c.sign = 1u << A.lidLow[q];
            c.tt = 0xAAAAu;
            c.nLeaves = 1;
            c.used = 1;
            c.value = 1001u;
            S[0].l[0] = (int)q;
            S[0].sign = c.sign;
            S[0].pk = cut_pack(c);
            A.cutA[q * 8] = make_int2((int)clamp_ref(A.ref[q]), (int)((uint32_t)A.lidLow[q] << 12));
        }
        const int f0 = A.w0[q], f1 = A.w1[q];
        const int u0 = f0 >> 1, u1 = f1 >> 1, c0 = f0 & 1, c1 = f1 & 1;
        bool ok = wait_ge(&A.done[u0], 1, A.status) && wait_ge(&A.done[u1], 1, A.status);
        if (ok) {
            const int2 *M0 = A.cutM + (int64_t)u0 * 8, *M1 = A.cutM + (int64_t)u1 * 8;
            // the pairs CutEnumerate tries (both slots used, at most 4 leaves
            // by signature), bit i * 8 + j: visiting the set bits in order is
            // the reference's i-major loop, and every lane takes its k-th pair
            // in the same iteration
            uint64_t pairs = 0;
            {
                uint32_t s1[8], used1 = 0;
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const int2 mj = M1[j];
                    s1[j] = (uint32_t)mj.x;
                    used1 |= packed_used((uint32_t)mj.y) << j;
                }
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    const int2 mi = M0[i];
                    if (!packed_used((uint32_t)mi.y)) continue;
#pragma unroll
                    for (int j = 0; j < 8; j++)
                        if (((used1 >> j) & 1u) && popc32((uint32_t)mi.x | s1[j]) <= 4)
                            pairs |= 1ull << (i * 8 + j);
                }
            }
            while (pairs) {
                const int p = __ffsll((long long)pairs) - 1;
                pairs &= pairs - 1;
                const int i = p >> 3, j = p & 7;
                {
                    RCut a, b;
                    load_rcut(A, (int64_t)u0 * 8 + i, M0[i], a);
                    load_rcut(A, (int64_t)u1 * 8 + j, M1[j], b);
                    // FindCut: first unused slot, else lowest value among
                    // >2-leaf, then 2-leaf, then smaller cuts (rewrite.cu:84-109)
                    int id = -1;
#pragma unroll
                    for (int k = 0; k < 8; k++)
                        if (id < 0 && !sl_used(S[k])) id = k;
                    if (id < 0) {
                        uint32_t best = 0xFFFFFFFFu;
#pragma unroll
                        for (int k = 0; k < 8; k++) {
                            uint32_t n = sl_n(S[k]);
                            uint32_t cls = n > 2 ? 0u : (n == 2 ? 1u : 2u);
                            uint32_t key = (cls << 20) | (sl_value(S[k]) << 3) | (uint32_t)k;
                            best = key < best ? key : best;
                        }
                        id = (int)(best & 7u);
                    }
#pragma unroll
                    for (int k = 0; k < 8; k++)
                        if (k == id) sl_clear_used(S[k]);
                    RCut m;
                    if (!rc_merge(a, b, m)) continue;
                    if (filter_slots(S, id, m.l, m.n, m.sign)) continue;  // dropped: slot stays free
                    m.tt = rc_truth(m, a, b, c0, c1);
                    const bool mini = rc_minimize(m);
                    m.value = 0;
                    Cut pc;
                    pc.tt = m.tt;
                    pc.nLeaves = m.n;
                    pc.used = 1;
                    pc.value = 0;
                    uint32_t a0, a1;
                    rc_pack_aux(m, a0, a1);
                    A.cutA[q * 8 + id] = make_int2((int)a0, (int)a1);
#pragma unroll
                    for (int k = 0; k < 8; k++)
                        if (k == id) {
                            S[k].l[0] = m.l[0];
                            S[k].l[1] = m.l[1];
                            S[k].l[2] = m.l[2];
                            S[k].l[3] = m.l[3];
                            S[k].sign = m.sign;
                            S[k].pk = cut_pack(pc);
                        }
                    bool keep = true;
                    if (mini) keep = !filter_slots(S, id, m.l, m.n, m.sign);
                    pc.value = rc_value(m);
                    pc.used = keep ? 1u : 0u;
#pragma unroll
                    for (int k = 0; k < 8; k++)
                        if (k == id) S[k].pk = cut_pack(pc);
                    if (m.n < 2) pairs = 0;  // enumeration of this node stops (rewrite.cu:291)
                }
            }
        }
#pragma unroll
        for (int k = 0; k < 8; k++) {
            A.cutL[q * 8 + k] = make_int4(S[k].l[0], S[k].l[1], S[k].l[2], S[k].l[3]);
            A.cutM[q * 8 + k] = make_int2((int)S[k].sign, (int)S[k].pk);
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
    int2 *cutA = X.ar->get<int2>(N * 8);
    int *done = X.ar->get<int>(N);
    if (!w.cutL || !w.cutM || !cutA || !done) return X.fail(CULS_E_OOM, "rw: scratch arena exhausted (cuts)");
    int rc;
    if ((rc = X.check(cudaMemsetAsync(w.cutM, 0, sizeof(int2) * N * 8, s), "memset"))) return rc;
    if ((rc = X.check(cudaMemsetAsync(X.counters, 0, sizeof(int) * 4, s), "memset"))) return rc;
    k_enum_init<<<X.grid(N), kBlock, 0, s>>>(N, w.wlev, w.wl, w.lidLow, w.ref, w.cutL, w.cutM, cutA, done);
    EnumArgs A{w.nL0, N, w.w0, w.w1, w.ref, w.lidLow, w.cutL, w.cutM, cutA, done, X.counters, X.status};
    X.mark(kMkEnumK0);
    k_enumerate<<<(unsigned)(X.sms * 8), kEnumBlock, 0, s>>>(A);
    X.mark(kMkEnumK1);
    X.launched(2);
    if ((rc = X.check(cudaGetLastError(), "enumerate launch"))) return rc;
    return 0;
}

}  // namespace culs
