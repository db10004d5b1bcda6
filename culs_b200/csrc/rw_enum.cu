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
    const int *lvlCnt;      // AND nodes per level (level 0: none)
    const int *lvlStart;    // first W position of each level
    const int *chunkStart;  // first chunk of each level; maxLevel + 2 entries
    int maxLevel;
    int wideMin;            // levels at least this wide run thread-per-node
    const int *w0, *w1;
    const int *ref;
    const uint8_t *lidLow;
    int4 *cutL;
    int2 *cutM;
    int2 *cutA;
    int *done;
    int *counter;
    unsigned long long *warpPairs;  // pairs replayed by enum_node_warp
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

// ------------------------------------------------- warp-per-node variant
// One candidate of a node's enumeration: the pair's merged cut (the first
// CutFilter sees it) and its final form after the truth table and
// MinimizeCutSupport, with value and aux.
struct Cand {
    int x0, x1, x2, x3;  // merged leaves
    uint32_t xs, xn;     // merged signature, leaf count
    int y0, y1, y2, y3;  // final leaves
    uint32_t ys, yn, ytt, yval, a0, a1;
    uint32_t ok, mini;   // merge succeeded; minimisation removed leaves
};

__device__ __forceinline__ void make_cand(const RCut &a, const RCut &b, int c0, int c1, Cand &c) {
    RCut m;
    c.ok = rc_merge(a, b, m) ? 1u : 0u;
    c.x0 = m.l[0];
    c.x1 = m.l[1];
    c.x2 = m.l[2];
    c.x3 = m.l[3];
    c.xs = m.sign;
    c.xn = m.n;
    m.tt = rc_truth(m, a, b, c0, c1);
    c.mini = rc_minimize(m) ? 1u : 0u;
    c.y0 = m.l[0];
    c.y1 = m.l[1];
    c.y2 = m.l[2];
    c.y3 = m.l[3];
    c.ys = m.sign;
    c.yn = m.n;
    c.ytt = m.tt;
    c.yval = rc_value(m);
    rc_pack_aux(m, c.a0, c.a1);
}

// A candidate in shared memory: four 16-byte words, written once by the lane
// that built it and read by the whole warp (a broadcast) when its turn in
// the slot policy comes.
__device__ __forceinline__ void put_cand(int4 *d, const Cand &c) {
    d[0] = make_int4(c.x0, c.x1, c.x2, c.x3);
    d[1] = make_int4(c.y0, c.y1, c.y2, c.y3);
    d[2] = make_int4((int)c.xs, (int)(c.xn | (c.ok << 8) | (c.mini << 9)), (int)c.ys, (int)c.yn);
    d[3] = make_int4((int)c.ytt, (int)c.yval, (int)c.a0, (int)c.a1);
}

__device__ __forceinline__ void get_cand(const int4 *d, Cand &c) {
    const int4 w0 = d[0], w1 = d[1], w2 = d[2], w3 = d[3];
    c.x0 = w0.x, c.x1 = w0.y, c.x2 = w0.z, c.x3 = w0.w;
    c.y0 = w1.x, c.y1 = w1.y, c.y2 = w1.z, c.y3 = w1.w;
    c.xs = (uint32_t)w2.x;
    c.xn = (uint32_t)w2.y & 0xFFu;
    c.ok = ((uint32_t)w2.y >> 8) & 1u;
    c.mini = ((uint32_t)w2.y >> 9) & 1u;
    c.ys = (uint32_t)w2.z, c.yn = (uint32_t)w2.w;
    c.ytt = (uint32_t)w3.x, c.yval = (uint32_t)w3.y, c.a0 = (uint32_t)w3.z, c.a1 = (uint32_t)w3.w;
}

// CutFilter (rewrite.cu:178-193) with slot k on lane k (k < 8): visiting the
// slots in index order, a larger slot containing X is dropped and the first
// slot contained in X drops X and ends the visit.  So every slot lane tests
// its own slot, one ballot finds the first containing slot, and only the
// supersets before it are dropped.  Returns true when X is dropped.
__device__ __forceinline__ bool warp_filter(int lane, int id, const int (&sl)[4], uint32_t ssign, uint32_t &spk,
                                            const int (&xl)[4], uint32_t xn, uint32_t xs) {
    bool clr = false, inX = false;
    if (lane < 8 && lane != id && packed_used(spk)) {
        const uint32_t kn = packed_nleaves(spk);
        if (kn > xn)
            clr = (ssign & xs) == xs && leaves_subset(xl, xn, sl, kn);
        else
            inX = (ssign & xs) == ssign && leaves_subset(sl, kn, xl, xn);
    }
    const unsigned C = __ballot_sync(0xffffffffu, clr), D = __ballot_sync(0xffffffffu, inX);
    const unsigned drop = D ? (C & ((1u << (__ffs(D) - 1)) - 1u)) : C;
    if ((drop >> lane) & 1u) spk &= ~(1u << 30);
    return D != 0;
}

// Fanin slot `lane` of the warp's node, read from the lane holding it.
__device__ __forceinline__ void fetch_slot(int src, int4 L, int2 M, int2 X, RCut &c, uint32_t &used) {
    const unsigned F = 0xffffffffu;
    c.l[0] = __shfl_sync(F, L.x, src);
    c.l[1] = __shfl_sync(F, L.y, src);
    c.l[2] = __shfl_sync(F, L.z, src);
    c.l[3] = __shfl_sync(F, L.w, src);
    const uint32_t sign = (uint32_t)__shfl_sync(F, M.x, src), pk = (uint32_t)__shfl_sync(F, M.y, src);
    const uint32_t x0 = (uint32_t)__shfl_sync(F, X.x, src), x1 = (uint32_t)__shfl_sync(F, X.y, src);
    c.sign = sign;
    c.tt = pk & 0xFFFFu;
    c.n = packed_nleaves(pk);
    c.used = 1;
    used = packed_used(pk);
    rc_unpack_aux(x0, x1, c);
}

// Position of the k-th (from 0) set bit of m; m has more than k set bits.
__device__ __forceinline__ int select_bit64(uint64_t m, int k) {
    int p = 0;
#pragma unroll
    for (int w = 32; w >= 1; w >>= 1) {
        const int c = __popcll(m & ((1ull << w) - 1ull));
        const bool up = k >= c;
        k -= up ? c : 0;
        m = up ? m >> w : m;
        p += up ? w : 0;
    }
    return p;
}

// A warp enumerates one node at a time: lanes 0-7 hold u0's cut slots and
// lanes 8-15 u1's.  The admissible pairs (pair bit i * 8 + j, the
// reference's i-major order; both slots used, at most four leaves by
// signature) are found from the slots' signatures first and dealt out in
// order, the k-th to lane k % 32, so a node with at most 32 of them -- most
// nodes -- builds its candidates in one round; each lands in shared memory.
// Then the warp replays
// CutEnumerate's slot policy over them in order with the node's 8 slots on
// lanes 0-7 -- FindCut is a min over those lanes, CutFilter two ballots --
// and lanes 0-7 write the slots.  Same results as the per-thread replay,
// with a node's latency cut to its sequential core.
__device__ __forceinline__ void enum_node_warp(const EnumArgs &A, int64_t q, int lane, int4 (*sc)[4]) {
    const unsigned F = 0xffffffffu;
    const int f0 = A.w0[q], f1 = A.w1[q];
    const int u0 = f0 >> 1, u1 = f1 >> 1, c0 = f0 & 1, c1 = f1 & 1;
    int ok = 1;
    if (lane == 0) ok = wait_ge(&A.done[u0], 1, A.status) && wait_ge(&A.done[u1], 1, A.status);
    ok = __shfl_sync(F, ok, 0);
    __syncwarp();
    // the node's slots: slot 0 the trivial cut
    int sl[4] = {0, 0, 0, 0};
    uint32_t ssign = 0, spk = 0, sa0 = 0, sa1 = 0;
    if (lane == 0) {
        Cut c;
        c.sign = 1u << A.lidLow[q];
        c.tt = 0xAAAAu;
        c.nLeaves = 1;
        c.used = 1;
        c.value = 1001u;
        sl[0] = (int)q;
        ssign = c.sign;
        spk = cut_pack(c);
        sa0 = clamp_ref(A.ref[q]);
        sa1 = (uint32_t)A.lidLow[q] << 12;
    }
    if (ok) {
        int4 L = make_int4(0, 0, 0, 0);
        int2 M = make_int2(0, 0), X = make_int2(0, 0);
        if (lane < 16) {
            const int64_t idx = (int64_t)(lane < 8 ? u0 : u1) * 8 + (lane & 7);
            L = __ldcg(&A.cutL[idx]);
            M = __ldcg(&A.cutM[idx]);
            X = __ldcg(&A.cutA[idx]);
        }
        // admissible pairs from the signatures: pair lane (i = lane / 8)
        // and pair lane + 32 (i = 4 + lane / 8), both with j = lane % 8
        const uint32_t sA = (uint32_t)__shfl_sync(F, M.x, lane >> 3), pA = (uint32_t)__shfl_sync(F, M.y, lane >> 3);
        const uint32_t sB = (uint32_t)__shfl_sync(F, M.x, 4 + (lane >> 3)),
                       pB = (uint32_t)__shfl_sync(F, M.y, 4 + (lane >> 3));
        const uint32_t sJ = (uint32_t)__shfl_sync(F, M.x, 8 + (lane & 7)),
                       pJ = (uint32_t)__shfl_sync(F, M.y, 8 + (lane & 7));
        const bool adm0 = packed_used(pA) && packed_used(pJ) && popc32(sA | sJ) <= 4;
        const bool adm1 = packed_used(pB) && packed_used(pJ) && popc32(sB | sJ) <= 4;
        const uint64_t pairs = (uint64_t)__ballot_sync(F, adm0) | ((uint64_t)__ballot_sync(F, adm1) << 32);
        const int nPairs = __popcll(pairs);
        // candidate k built by lane k % 32, kept in sc[k]
#pragma unroll
        for (int r = 0; r < 2; r++) {
            if (r * 32 >= nPairs) break;
            const int k = r * 32 + lane;
            const int p = k < nPairs ? select_bit64(pairs, k) : 0;
            RCut a, b;
            uint32_t ua, ub;
            fetch_slot(p >> 3, L, M, X, a, ua);
            fetch_slot(8 + (p & 7), L, M, X, b, ub);
            if (k < nPairs) {
                Cand c;
                make_cand(a, b, c0, c1, c);
                put_cand(sc[k], c);
            }
        }
        __syncwarp();
        int k = 0;
        for (; k < nPairs; k++) {
            Cand m;
            get_cand(sc[k], m);
            // FindCut (rewrite.cu:84-109): the first free slot, else the
            // lowest (class, value, index); both computed, one kept
            const unsigned freeSlots = __ballot_sync(F, lane < 8 && !packed_used(spk)) & 0xFFu;
            uint32_t key = 0xFFFFFFFFu;
            if (lane < 8) {
                const uint32_t n = packed_nleaves(spk);
                const uint32_t cls = n > 2 ? 0u : (n == 2 ? 1u : 2u);
                key = (cls << 20) | (((spk >> 16) & 0x7FFu) << 3) | (uint32_t)lane;
            }
            const uint32_t lowest = __reduce_min_sync(F, key);
            const int id = freeSlots ? __ffs(freeSlots) - 1 : (int)(lowest & 7u);
            if (lane == id) spk &= ~(1u << 30);
            if (!m.ok) continue;
            const int xl[4] = {m.x0, m.x1, m.x2, m.x3};
            if (warp_filter(lane, id, sl, ssign, spk, xl, m.xn, m.xs)) continue;  // slot stays free
            Cut pc;
            pc.tt = m.ytt;
            pc.nLeaves = m.yn;
            pc.used = 1;
            pc.value = 0;
            if (lane == id) {
                sl[0] = m.y0;
                sl[1] = m.y1;
                sl[2] = m.y2;
                sl[3] = m.y3;
                ssign = m.ys;
                spk = cut_pack(pc);
                sa0 = m.a0;
                sa1 = m.a1;
            }
            bool keep = true;
            if (m.mini) {
                const int yl[4] = {m.y0, m.y1, m.y2, m.y3};
                keep = !warp_filter(lane, id, sl, ssign, spk, yl, m.yn, m.ys);
            }
            pc.value = m.yval;
            pc.used = keep ? 1u : 0u;
            if (lane == id) spk = cut_pack(pc);
            if (m.yn < 2) {  // enumeration of this node stops (rewrite.cu:291)
                k++;
                break;
            }
        }
        if (lane == 0 && k > 0) atomicAdd(A.warpPairs, (unsigned long long)k);  // pairs replayed
    }
    if (lane < 8) {
        A.cutL[q * 8 + lane] = make_int4(sl[0], sl[1], sl[2], sl[3]);
        A.cutM[q * 8 + lane] = make_int2((int)ssign, (int)spk);
        A.cutA[q * 8 + lane] = make_int2((int)sa0, (int)sa1);
        __threadfence();
    }
    __syncwarp();  // also: every lane is done reading sc before the next node overwrites it
    if (lane == 0) st_release(&A.done[q], 1);
}

// One node on one thread (wide levels): the slots in registers, the
// admissible pairs visited in order.  All lanes of the warp call it (valid:
// the lane has a node) and run as many rounds as the lane with the most
// admissible pairs, one pair per round and back in step after each, so
// lanes that finish a pair early do not drift into later pairs alone.
__device__ __forceinline__ void enum_node_thread(const EnumArgs &A, int64_t q, bool valid) {
    Slot S[8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
        S[k].pk = 0;
        S[k].sign = 0;
        S[k].l[0] = S[k].l[1] = S[k].l[2] = S[k].l[3] = 0;
    }
    if (valid) {
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
    const int f0 = valid ? A.w0[q] : 0, f1 = valid ? A.w1[q] : 0;
    const int u0 = f0 >> 1, u1 = f1 >> 1, c0 = f0 & 1, c1 = f1 & 1;
    bool ok = valid && wait_ge(&A.done[u0], 1, A.status) && wait_ge(&A.done[u1], 1, A.status);
    uint64_t pairs = 0;
    const int2 *M0 = A.cutM + (int64_t)u0 * 8, *M1 = A.cutM + (int64_t)u1 * 8;
    if (ok) {
        // the pairs CutEnumerate tries (both slots used, at most 4 leaves
        // by signature), bit i * 8 + j: visiting the set bits in order is
        // the reference's i-major loop, and every lane takes its k-th pair
        // in the same iteration
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
    }
    // every lane runs the warp's largest number of admissible pairs, in step;
    // `continue` in the do-while below ends the lane's current pair
    const int rounds = __reduce_max_sync(0xffffffffu, (unsigned)popc64(pairs));
    for (int t = 0; t < rounds; t++) {
        if (pairs) {
            const int p = __ffsll((long long)pairs) - 1;
            pairs &= pairs - 1;
            const int i = p >> 3, j = p & 7;
            do {
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
            } while (false);
        }
        __syncwarp();
    }
    if (!valid) return;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        A.cutL[q * 8 + k] = make_int4(S[k].l[0], S[k].l[1], S[k].l[2], S[k].l[3]);
        A.cutM[q * 8 + k] = make_int2((int)S[k].sign, (int)S[k].pk);
    }
    __threadfence();
    st_release(&A.done[q], 1);
}

// Levels are cut into chunks that never cross a level: a wide level into
// 32-node chunks, each node on one thread (throughput), a narrow level into
// one-node chunks, each node on a whole warp (latency: a narrow level's
// time is the time of its slowest node).  Warps claim chunks in level
// order, so every fanin of a claimed node lies in an earlier, claimed chunk.
__global__ void __launch_bounds__(kEnumBlock, 4) k_enumerate(EnumArgs A) {
    __shared__ int4 s_cand[kEnumBlock / 32][64][4];
    const unsigned F = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int total = A.chunkStart[A.maxLevel + 1];
    while (true) {
        int c = 0;
        if (lane == 0) c = atomicAdd(A.counter, 1);
        c = __shfl_sync(F, c, 0);
        if (c >= total) break;
        int lo = 1, hi = A.maxLevel;
        while (lo < hi) {  // last level whose first chunk is <= c
            const int mid = (lo + hi + 1) >> 1;
            if (A.chunkStart[mid] <= c)
                lo = mid;
            else
                hi = mid - 1;
        }
        const int w = A.lvlCnt[lo];
        const int64_t base = A.nL0 + A.lvlStart[lo];
        const int64_t k = c - A.chunkStart[lo];
        if (w >= A.wideMin) {
            const int64_t q = base + k * 32 + lane;
            enum_node_thread(A, q, q < base + w);
        } else {
            enum_node_warp(A, base + k, lane, s_cand[threadIdx.x >> 5]);
        }
    }
}

// lvlCnt has nBins counters (levels 0 .. nBins - 1)
__global__ void k_level_count(int64_t nL0, int64_t N, const int *wlev, int *lvlCnt, int nBins) {
    __shared__ int h[kHistBins];
    hist_begin(h, nBins);
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t q = nL0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < N; q += stride)
        hist_add(h, nBins, lvlCnt, wlev[q]);
    hist_end(h, nBins, lvlCnt);
}

__global__ void k_level_chunks(int n, const int *lvlCnt, int wideMin, int *cc) {
    int stride = gridDim.x * blockDim.x;
    for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < n; l += stride) {
        const int w = lvlCnt[l];
        cc[l] = w >= wideMin ? (w + 31) / 32 : w;
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
    w.warpPairs = X.ar->get<unsigned long long>(1);
    if (!w.cutL || !w.cutM || !cutA || !done || !w.warpPairs)
        return X.fail(CULS_E_OOM, "rw: scratch arena exhausted (cuts)");
    int rc;
    if ((rc = X.check(cudaMemsetAsync(w.cutM, 0, sizeof(int2) * N * 8, s), "memset"))) return rc;
    if ((rc = X.check(cudaMemsetAsync(X.counters, 0, sizeof(int) * 4, s), "memset"))) return rc;
    if ((rc = X.check(cudaMemsetAsync(w.warpPairs, 0, sizeof(unsigned long long), s), "memset"))) return rc;
    // per-level widths, starts and chunk offsets
    const int L = w.maxLevel + 2;
    int *lvlCnt = X.ar->get<int>(L), *lvlStart = X.ar->get<int>(L), *cc = X.ar->get<int>(L),
        *chunkStart = X.ar->get<int>(L);
    if (!lvlCnt || !lvlStart || !cc || !chunkStart) return X.fail(CULS_E_OOM, "rw: scratch arena exhausted (levels)");
    if ((rc = X.check(cudaMemsetAsync(lvlCnt, 0, sizeof(int) * L, s), "memset"))) return rc;
    k_level_count<<<X.grid(N - w.nL0), kBlock, 0, s>>>(w.nL0, N, w.wlev, lvlCnt, w.maxLevel + 1);
    k_level_chunks<<<grid_1d(L, kBlock, X.sms * 16), kBlock, 0, s>>>(L - 1, lvlCnt, X.tune->enumWideMin, cc);
    if ((rc = X.check(scan_exclusive(lvlCnt, lvlStart, L - 1, nullptr, *X.ar, s), "scan"))) return rc;
    if ((rc = X.check(scan_exclusive(cc, chunkStart, L - 1, chunkStart + L - 1, *X.ar, s), "scan"))) return rc;
    k_enum_init<<<X.grid(N), kBlock, 0, s>>>(N, w.wlev, w.wl, w.lidLow, w.ref, w.cutL, w.cutM, cutA, done);
    // lvlStart counts AND nodes only: the AND positions of W start at nL0
    EnumArgs A{w.nL0, N,       lvlCnt, lvlStart, chunkStart, w.maxLevel, X.tune->enumWideMin, w.w0, w.w1,
               w.ref, w.lidLow, w.cutL, w.cutM, cutA,       done,       X.counters, w.warpPairs, X.status};
    X.mark(kMkEnumK0);
    // a wide batch fills the GPU; a narrow one runs about sixteen levels'
    // worth of chunks at a time (32 nodes a warp on wide levels, 1 on narrow)
    const int perBlock = (kEnumBlock / 32) * (w.width >= X.tune->enumWideMin ? 32 : 1);
    k_enumerate<<<flow_blocks(w.width, perBlock, (unsigned)(X.sms * X.tune->enumBlocksPerSm), X.sms), kEnumBlock, 0, s>>>(A);
    X.mark(kMkEnumK1);
    X.launched(6);
    if ((rc = X.check(cudaGetLastError(), "enumerate launch"))) return rc;
    return 0;
}

}  // namespace culs
