// Checks the branch-free helpers of the warp-wide cut enumeration against
// their sequential forms on the CPU: tt_stretch_flat / tt_shrink_flat against
// tt_stretch / tt_shrink (CutTruthStretch / CutTruthShrink, CULS
// src/algorithms/rewrite.cu:213-241) for every 16-bit table and phase, and
// rc_merge against the step-by-step merge with early exits (MergeCutOrdered,
// rewrite.cu:111-176) on two million random cut pairs.  Built and run by
// tests/test_flat_helpers.py.
#include <cstdio>
#include <random>
#include <algorithm>
#include <vector_types.h>
#define __device__
#define __forceinline__ inline
#include "enum_regs.cuh"
using namespace culs;
// the merge with early exits: stop when both inputs are used up, fail when
// leaves remain after four steps
static bool seq_merge(const RCut &a0, const RCut &b0, RCut &o) {
    const bool sw = a0.n < b0.n;
    const RCut &a = sw ? b0 : a0;
    const RCut &b = sw ? a0 : b0;
    int i = 0, k = 0, c = 0;
    const int na = (int)a.n, nb = (int)b.n;
    for (int s = 0; s < 4; s++) { o.l[s] = 0; o.ref[s] = 0; o.lid[s] = 0; }
    for (int s = 0; s < 4; s++) {
        if (c != s) break;
        int ai = i < na ? pick4(a.l, i) : 0x7FFFFFFF;
        int bk = k < nb ? pick4(b.l, k) : 0x7FFFFFFF;
        if (i == na && k == nb) break;
        int take;
        if (k == nb) take = 0; else if (i == na) take = 1; else take = ai < bk ? 0 : (ai > bk ? 1 : 2);
        int leaf = take == 1 ? bk : ai;
        uint32_t r = take == 1 ? pick4(b.ref, k) : pick4(a.ref, i);
        uint32_t d = take == 1 ? pick4(b.lid, k) : pick4(a.lid, i);
        o.l[s] = leaf; o.ref[s] = r; o.lid[s] = d;
        if (take != 1) i++;
        if (take != 0) k++;
        c = s + 1;
    }
    if (i < na || k < nb) return false;
    o.n = (uint32_t)c; o.sign = a0.sign | b0.sign; o.used = 1;
    return true;
}
int main() {
    long bad = 0, n = 0;
    for (uint32_t t = 0; t < 65536; t++)
        for (int ph = 0; ph < 16; ph++) {
            const int nv = __builtin_popcount(ph);
            if (tt_stretch(t, nv, ph) != tt_stretch_flat(t, nv, ph)) bad++;
            if (tt_shrink(t, ph) != tt_shrink_flat(t, ph)) bad++;
        }
    printf("truth tables: bad %ld\n", bad);
    std::mt19937 rng(1);
    for (int it = 0; it < 2000000; it++) {
        RCut a{}, b{};
        for (RCut *x : {&a, &b}) {
            x->n = rng() % 5;
            int v[8]; int m = 0;
            while (m < (int)x->n) { int c = rng() % 9; bool dup = false; for (int j = 0; j < m; j++) dup |= v[j] == c; if (!dup) v[m++] = c; }
            std::sort(v, v + m);
            for (int j = 0; j < 4; j++) { x->l[j] = j < m ? v[j] : 0; x->ref[j] = rng() % 1002; x->lid[j] = rng() % 32; }
            x->sign = rng();
        }
        RCut o1{}, o2{};
        bool r1 = seq_merge(a, b, o1), r2 = rc_merge(a, b, o2);
        n++;
        if (r1 != r2) { bad++; continue; }
        if (!r1) continue;
        bool same = o1.n == o2.n && o1.sign == o2.sign;
        for (int j = 0; j < 4; j++) same &= o1.l[j] == o2.l[j] && o1.ref[j] == o2.ref[j] && o1.lid[j] == o2.lid[j];
        if (!same) bad++;
    }
    printf("checked %ld bad %ld\n", n, bad);
    return bad != 0;
}
