// Register-resident cut enumeration for one node (device side of
// k_enumerate).  Same semantics as enum_pair()/CutEnumerate
// (src/algorithms/rewrite.cu:268-294): the 8 slots live in registers (every
// slot index is a compile-time constant after unrolling), and every cut
// carries, beside its leaves, each leaf's reference count (clamped to 1001)
// and local-id bits, so cut values and minimised signatures need no memory
// access.
#pragma once

#include "rw_core.cuh"

namespace culs {

// A cut in registers.  aux0 = ref of leaf 0 | ref of leaf 1 << 11 |
// (ref of leaf 2 & 0x3FF) << 22; aux1 = ref of leaf 2 >> 10 | ref of leaf 3
// << 1 | lid5 of leaves 0..3 << 12 + 5*i.  Refs are clamped to 1001, which
// leaves CutFindValue's result unchanged (it caps the sum at 1000).
struct RCut {
    int l[4];
    uint32_t sign, tt, value, n, used;
    uint32_t ref[4];
    uint32_t lid[4];
};

__device__ __forceinline__ void rc_unpack_aux(uint32_t a0, uint32_t a1, RCut &c) {
    c.ref[0] = a0 & 0x7FFu;
    c.ref[1] = (a0 >> 11) & 0x7FFu;
    c.ref[2] = ((a0 >> 22) & 0x3FFu) | ((a1 & 1u) << 10);
    c.ref[3] = (a1 >> 1) & 0x7FFu;
#pragma unroll
    for (int i = 0; i < 4; i++) c.lid[i] = (a1 >> (12 + 5 * i)) & 31u;
}

__device__ __forceinline__ void rc_pack_aux(const RCut &c, uint32_t &a0, uint32_t &a1) {
    a0 = (c.ref[0] & 0x7FFu) | ((c.ref[1] & 0x7FFu) << 11) | ((c.ref[2] & 0x3FFu) << 22);
    a1 = ((c.ref[2] >> 10) & 1u) | ((c.ref[3] & 0x7FFu) << 1);
#pragma unroll
    for (int i = 0; i < 4; i++) a1 |= (c.lid[i] & 31u) << (12 + 5 * i);
}

// CutFindValue from the carried refs.
__device__ __forceinline__ uint32_t rc_value(const RCut &c) {
    if (c.n < 2) return 1001u;
    uint32_t v = 0, ones = 0;
#pragma unroll
    for (int i = 0; i < 4; i++)
        if ((uint32_t)i < c.n) {
            v += c.ref[i];
            ones += c.ref[i] == 1u;
        }
    int value = v > 1000u ? 1000 : (int)v;
    if (ones > 3) value = 5 - (int)ones;
    return (uint32_t)value & 0x7FFu;
}

template <class T>
__device__ __forceinline__ T pick4(const T (&v)[4], int i) {
    return i == 0 ? v[0] : (i == 1 ? v[1] : (i == 2 ? v[2] : v[3]));
}

// MergeCutOrdered / MergeCut with the leaf attributes carried along: four
// merge steps, each taking the smaller head leaf (both when equal), without
// branches -- the lanes of the warp-wide enumeration merge different cuts.
__device__ __forceinline__ bool rc_merge(const RCut &a0, const RCut &b0, RCut &o) {
    const bool sw = a0.n < b0.n;
    const RCut &a = sw ? b0 : a0;
    const RCut &b = sw ? a0 : b0;
    int i = 0, k = 0, c = 0;
    const int na = (int)a.n, nb = (int)b.n;
#pragma unroll
    for (int s = 0; s < 4; s++) {
        const bool ea = i >= na, eb = k >= nb;
        const bool act = !(ea && eb);
        const int ai = ea ? 0x7FFFFFFF : pick4(a.l, i);
        const int bk = eb ? 0x7FFFFFFF : pick4(b.l, k);
        const int take = eb ? 0 : (ea ? 1 : (ai < bk ? 0 : (ai > bk ? 1 : 2)));  // 0 = a, 1 = b, 2 = equal
        o.l[s] = act ? (take == 1 ? bk : ai) : 0;
        o.ref[s] = act ? (take == 1 ? pick4(b.ref, k) : pick4(a.ref, i)) : 0u;
        o.lid[s] = act ? (take == 1 ? pick4(b.lid, k) : pick4(a.lid, i)) : 0u;
        i += (act && take != 1) ? 1 : 0;
        k += (act && take != 0) ? 1 : 0;
        c = act ? s + 1 : c;
    }
    o.n = (uint32_t)c;
    o.sign = a0.sign | b0.sign;
    o.used = 1;
    return i >= na && k >= nb;
}

// CutTruthPhase over register leaves.
__device__ __forceinline__ int rc_phase(const RCut &x, const RCut &cut) {
    int ph = 0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        if ((uint32_t)i >= cut.n) continue;
        bool in = false;
#pragma unroll
        for (int j = 0; j < 4; j++) in |= ((uint32_t)j < x.n) && x.l[j] == cut.l[i];
        if (in) ph |= 1 << i;
    }
    return ph;
}

__device__ __forceinline__ uint32_t rc_truth(const RCut &cut, const RCut &a, const RCut &b, int ca, int cb) {
    uint32_t t0 = ca ? (~a.tt & 0xFFFFu) : a.tt;
    uint32_t t1 = cb ? (~b.tt & 0xFFFFu) : b.tt;
    t0 = tt_stretch_flat(t0, (int)a.n, rc_phase(a, cut));
    t1 = tt_stretch_flat(t1, (int)b.n, rc_phase(b, cut));
    return (t0 & t1) & 0xFFFFu;
}

// MinimizeCutSupport with carried attributes; returns true when leaves were
// removed.
__device__ __forceinline__ bool rc_minimize(RCut &c) {
    const uint32_t m0[4] = {0x5555u, 0x3333u, 0x0F0Fu, 0x00FFu};
    const uint32_t m1[4] = {0xAAAAu, 0xCCCCu, 0xF0F0u, 0xFF00u};
    int ph = 0, nl = (int)c.n;
    const uint32_t t = c.tt & 0xFFFFu;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        if ((uint32_t)i >= c.n) continue;
        if ((t & m0[i]) == ((t & m1[i]) >> (1 << i)))
            nl--;
        else
            ph |= 1 << i;
    }
    if (nl == (int)c.n) return false;
    c.tt = tt_shrink_flat(t, ph) & 0xFFFFu;
    RCut o = c;
    int k = 0;
    uint32_t sign = 0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        if ((uint32_t)i < c.n && (ph >> i & 1)) {
            // k <= i, so writing slot k never clobbers an unread slot
#pragma unroll
            for (int s = 0; s < 4; s++)
                if (s == k) {
                    o.l[s] = c.l[i];
                    o.ref[s] = c.ref[i];
                    o.lid[s] = c.lid[i];
                }
            sign |= 1u << c.lid[i];
            k++;
        }
    }
    o.sign = sign;
    o.n = (uint32_t)nl;
    c = o;
    return true;
}

// leaves(a) subset of leaves(b)
__device__ __forceinline__ bool rc_subset(const RCut &a, const RCut &b) {
    bool all = true;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        if ((uint32_t)i >= a.n) continue;
        bool in = false;
#pragma unroll
        for (int j = 0; j < 4; j++) in |= ((uint32_t)j < b.n) && b.l[j] == a.l[i];
        all &= in;
    }
    return all;
}

}  // namespace culs
