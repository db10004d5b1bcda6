// Per-item logic of the rewriting pass, written as __host__ __device__
// functions over plain arrays.  The engine's kernels (engine.cu) call these;
// each function names the reference code whose semantics it reproduces
// (paths relative to the CULS source tree).
//
// Node addressing: every object of a batch has a storage position; literals
// are 2*position + complement.  Within one graph, storage order equals id
// order, so comparisons of positions reproduce the reference's comparisons of
// node ids.  Per graph, `cpos` is the position of the constant node.
#pragma once

#include "common.cuh"
#ifdef __CUDACC__
#include "prim.cuh"
#endif

namespace culs {

// ----------------------------------------------------------- library
// The 4-input rewriting library (same values as CULS
// src/algorithms/rewrite_library.inc, decoded as rw::CPUSolver::ReadLibrary
// does, src/algorithms/rewrite.cu:1281-1307), repacked for single loads.
constexpr int kNumClasses = 222;
constexpr int kMaxLibNodes = 56;  // <= 50 internal nodes + 4 inputs fit in 54
struct RwLib {
    // per truth table: phase (bits 0-4) | perm index (bits 8-12) | class (bits 16-23)
    uint32_t npn[1 << 16];
    uint8_t perm4[24][4];
    uint8_t nNodes[kNumClasses], nRoots[kNumClasses];
    // per class and internal node j (library index j+4):
    // fanin0 (bits 0-7) | fanin1 (bits 8-15) | compl0 (bit 16) | compl1 (bit 17)
    uint32_t node[kNumClasses][kMaxLibNodes];
    uint8_t roots[kNumClasses][16];
    // The same internal nodes regrouped for evaluation: batches of up to
    // kLibBatch nodes of equal depth (every fanin in an earlier batch), in
    // order of depth.  Entry = node word | index j (bits 18-23), or
    // kNoLibNode for an unused entry.  Nodes of one batch never read each
    // other, so their table probes are issued together.
    uint4 batch[kNumClasses][kMaxLibNodes];
    uint8_t nBatches[kNumClasses];
    // Per class and root: bit j set for every internal node j (j >= 4) in
    // the root's cone, the root included.
    unsigned long long rootCone[kNumClasses][16];
    // Evaluation order of the classes: by number of batches, then class, so
    // that cut items sorted by this slot put forests of equal batch count
    // side by side.
    uint8_t classSlot[kNumClasses];
};
constexpr int kLibBatch = 4;
constexpr uint32_t kNoLibNode = 0xFFFFFFFFu;
static_assert(kLibBatch == 4, "a batch is one uint4");

CULS_HD int npn_phase(uint32_t w) { return (int)(w & 31u); }
CULS_HD int npn_perm(uint32_t w) { return (int)((w >> 8) & 31u); }
CULS_HD int npn_class(uint32_t w) { return (int)((w >> 16) & 255u); }
CULS_HD int ln_f0(uint32_t w) { return (int)(w & 255u); }
CULS_HD int ln_f1(uint32_t w) { return (int)((w >> 8) & 255u); }
CULS_HD int ln_c0(uint32_t w) { return (int)((w >> 16) & 1u); }
CULS_HD int ln_c1(uint32_t w) { return (int)((w >> 17) & 1u); }

// --------------------------------------------------------------- cuts
// A cut slot (rw::Cut, src/algorithms/rewrite.h:10-16).  In device memory a
// slot is an int4 of leaves plus an int2 {sign, packed}, packed =
// tt (bits 0-15) | value (bits 16-26) | nLeaves (bits 27-29) | used (bit 30).
struct Cut {
    int leaves[4];
    uint32_t sign;
    uint32_t tt;
    uint32_t value;
    uint32_t nLeaves;
    uint32_t used;
};

CULS_HD uint32_t cut_pack(const Cut &c) {
    return (c.tt & 0xFFFFu) | ((c.value & 0x7FFu) << 16) | ((c.nLeaves & 7u) << 27) | ((c.used & 1u) << 30);
}
CULS_HD void cut_unpack(uint32_t w, Cut &c) {
    c.tt = w & 0xFFFFu;
    c.value = (w >> 16) & 0x7FFu;
    c.nLeaves = (w >> 27) & 7u;
    c.used = (w >> 30) & 1u;
}
CULS_HD uint32_t packed_used(uint32_t w) { return (w >> 30) & 1u; }
CULS_HD uint32_t packed_nleaves(uint32_t w) { return (w >> 27) & 7u; }

CULS_HD int popc32(uint32_t x) {
#if defined(__CUDA_ARCH__)
    return __popc(x);
#else
    return __builtin_popcount(x);
#endif
}
CULS_HD int popc64(uint64_t x) {
#if defined(__CUDA_ARCH__)
    return __popcll(x);
#else
    return __builtin_popcountll(x);
#endif
}

// CutFindValue, src/algorithms/rewrite.cu:49-61
CULS_HD uint32_t cut_value(const Cut &c, const int *ref) {
    int value = 0, nOnes = 0;
    for (uint32_t i = 0; i < c.nLeaves; i++) {
        int r = ref[c.leaves[i]];
        value += r;
        nOnes += (r == 1);
    }
    if (c.nLeaves < 2) return 1001u;
    if (value > 1000) value = 1000;
    if (nOnes > 3) value = 5 - nOnes;
    return (uint32_t)value & 0x7FFu;
}

// FindCut, src/algorithms/rewrite.cu:84-109: first unused slot, else the
// lowest-value slot among >2-leaf cuts, then 2-leaf, then smaller cuts; the
// chosen slot is marked unused before any merge is tried.
CULS_HD int find_slot(Cut *s) {
    for (int i = 0; i < 8; i++)
        if (s[i].used == 0) return i;
    int ans = -1;
    for (int i = 0; i < 8; i++)
        if (s[i].nLeaves > 2 && (ans == -1 || s[i].value < s[ans].value)) ans = i;
    if (ans == -1)
        for (int i = 0; i < 8; i++)
            if (s[i].nLeaves == 2 && (ans == -1 || s[i].value < s[ans].value)) ans = i;
    if (ans == -1)
        for (int i = 0; i < 8; i++)
            if (s[i].nLeaves < 2 && (ans == -1 || s[i].value < s[ans].value)) ans = i;
    s[ans].used = 0;
    return ans;
}

// MergeCutOrdered / MergeCut, src/algorithms/rewrite.cu:112-164.  Merges
// the sorted leaf lists of a and b into out (at most 4 leaves).  Returns 0
// when the union exceeds 4 leaves; out's leaves may be partly written then.
CULS_HD int merge_cuts(const Cut &a0, const Cut &b0, Cut *out) {
    const Cut &a = (a0.nLeaves >= b0.nLeaves) ? a0 : b0;
    const Cut &b = (a0.nLeaves >= b0.nLeaves) ? b0 : a0;
    int c = 0, i = 0, k = 0;
    const int na = (int)a.nLeaves, nb = (int)b.nLeaves;
    for (c = 0; c < 4; c++) {
        if (k == nb) {
            if (i == na) {
                out->nLeaves = (uint32_t)c;
                out->sign = a0.sign | b0.sign;
                out->used = 1;
                return 1;
            }
            out->leaves[c] = a.leaves[i++];
            continue;
        }
        if (i == na) {
            out->leaves[c] = b.leaves[k++];
            continue;
        }
        if (a.leaves[i] < b.leaves[k]) {
            out->leaves[c] = a.leaves[i++];
            continue;
        }
        if (a.leaves[i] > b.leaves[k]) {
            out->leaves[c] = b.leaves[k++];
            continue;
        }
        out->leaves[c] = a.leaves[i++];
        k++;
    }
    if (i < na || k < nb) return 0;
    out->nLeaves = (uint32_t)c;
    out->sign = a0.sign | b0.sign;
    out->used = 1;
    return 1;
}

// CutDominance, src/algorithms/rewrite.cu:167-175: leaves(a) subset of leaves(b)
CULS_HD int cut_subset(const Cut &a, const Cut &b) {
    for (uint32_t i = 0; i < a.nLeaves; i++) {
        int ok = 0;
        for (uint32_t j = 0; j < b.nLeaves; j++)
            if (b.leaves[j] == a.leaves[i]) ok = 1;
        if (!ok) return 0;
    }
    return 1;
}

// CutFilter, src/algorithms/rewrite.cu:178-193
CULS_HD int cut_filter(Cut *s, int id) {
    for (int i = 0; i < 8; i++) {
        if (i == id || !s[i].used) continue;
        if (s[i].nLeaves > s[id].nLeaves) {
            if ((s[i].sign & s[id].sign) != s[id].sign) continue;
            if (cut_subset(s[id], s[i])) s[i].used = 0;
        } else {
            if ((s[i].sign & s[id].sign) != s[i].sign) continue;
            if (cut_subset(s[i], s[id])) {
                s[id].used = 0;
                return 1;
            }
        }
    }
    return 0;
}

// CutTruthSwapAdjacentVars, src/algorithms/rewrite.cu:203-211, on 16 bits.
CULS_HD uint32_t tt_swap_adj(uint32_t t, int v) {
    if (v == 0) return (t & 0x9999u) | ((t & 0x2222u) << 1) | ((t & 0x4444u) >> 1);
    if (v == 1) return (t & 0xC3C3u) | ((t & 0x0C0Cu) << 2) | ((t & 0x3030u) >> 2);
    if (v == 2) return (t & 0xF00Fu) | ((t & 0x00F0u) << 4) | ((t & 0x0F00u) >> 4);
    return 0;
}

// CutTruthPhase, src/algorithms/rewrite.cu:195-201
CULS_HD int tt_phase(const Cut &x, const Cut &cut) {
    int ph = 0;
    for (uint32_t i = 0; i < cut.nLeaves; i++)
        for (uint32_t j = 0; j < x.nLeaves; j++)
            if (x.leaves[j] == cut.leaves[i]) ph |= 1 << i;
    return ph;
}

// CutTruthStretch, src/algorithms/rewrite.cu:213-221
CULS_HD uint32_t tt_stretch(uint32_t t, int nVar, int ph) {
    int var = nVar - 1;
    for (int i = 3; i >= 0; i--)
        if (ph >> i & 1) {
            for (int k = var; k < i; k++) t = tt_swap_adj(t, k);
            var--;
        }
    return t;
}

// tt_swap_adj with the variable known at compile time
template <int V>
CULS_HD uint32_t tt_swap_adj_c(uint32_t t) {
    return V == 0   ? (t & 0x9999u) | ((t & 0x2222u) << 1) | ((t & 0x4444u) >> 1)
           : V == 1 ? (t & 0xC3C3u) | ((t & 0x0C0Cu) << 2) | ((t & 0x3030u) >> 2)
                    : (t & 0xF00Fu) | ((t & 0x00F0u) << 4) | ((t & 0x0F00u) >> 4);
}

// tt_stretch without branches, for the warp-wide enumeration (lanes with
// different phases take one path): every swap the loops could make, in the
// loops' order, applied when the loops would make it.  Equal to tt_stretch
// whenever ph has nVar bits set, which holds for every call (a fanin cut's
// leaves all appear in the merged cut).
CULS_HD uint32_t tt_stretch_flat(uint32_t t, int nVar, int ph) {
    int var = nVar - 1;
#define CULS_SW(K, I)                                                          \
    {                                                                          \
        const uint32_t sw = tt_swap_adj_c<K>(t);                               \
        t = (((ph >> (I)) & 1) && (K) >= var) ? sw : t;                        \
    }
    CULS_SW(0, 3) CULS_SW(1, 3) CULS_SW(2, 3) var -= (ph >> 3) & 1;
    CULS_SW(0, 2) CULS_SW(1, 2) var -= (ph >> 2) & 1;
    CULS_SW(0, 1)
#undef CULS_SW
    return t;
}

// CutTruthtable, src/algorithms/rewrite.cu:223-229
CULS_HD uint32_t cut_truth(const Cut &cut, const Cut &a, const Cut &b, int ca, int cb) {
    uint32_t t0 = ca ? (~a.tt & 0xFFFFu) : a.tt;
    uint32_t t1 = cb ? (~b.tt & 0xFFFFu) : b.tt;
    t0 = tt_stretch(t0, (int)a.nLeaves, tt_phase(a, cut));
    t1 = tt_stretch(t1, (int)b.nLeaves, tt_phase(b, cut));
    return (t0 & t1) & 0xFFFFu;
}

// CutTruthShrink, src/algorithms/rewrite.cu:231-241
CULS_HD uint32_t tt_shrink(uint32_t t, int ph) {
    int var = 0;
    for (int i = 0; i < 4; i++)
        if (ph & (1 << i)) {
            for (int k = i - 1; k >= var; k--) t = tt_swap_adj(t, k);
            var++;
        }
    return t;
}

// tt_shrink without branches (see tt_stretch_flat): equal to tt_shrink for
// every phase.
CULS_HD uint32_t tt_shrink_flat(uint32_t t, int ph) {
    int var = (ph & 1);
#define CULS_SW(K, I)                                                          \
    {                                                                          \
        const uint32_t sw = tt_swap_adj_c<K>(t);                               \
        t = (((ph >> (I)) & 1) && (K) >= var) ? sw : t;                        \
    }
    CULS_SW(0, 1) var += (ph >> 1) & 1;
    CULS_SW(1, 2) CULS_SW(0, 2) var += (ph >> 2) & 1;
    CULS_SW(2, 3) CULS_SW(1, 3) CULS_SW(0, 3)
#undef CULS_SW
    return t;
}

// MinimizeCutSupport, src/algorithms/rewrite.cu:243-266.  `lsb` holds
// (local id & 31) of each leaf position so that the recomputed sign uses
// graph-local ids; it is read through lidLow[leaf].
CULS_HD int cut_minimize(Cut *c, const uint8_t *lidLow) {
    const uint32_t m0[4] = {0x5555u, 0x3333u, 0x0F0Fu, 0x00FFu};
    const uint32_t m1[4] = {0xAAAAu, 0xCCCCu, 0xF0F0u, 0xFF00u};
    int ph = 0;
    uint32_t t = c->tt & 0xFFFFu;
    int nl = (int)c->nLeaves;
    for (uint32_t i = 0; i < c->nLeaves; i++) {
        if ((t & m0[i]) == ((t & m1[i]) >> (1 << i)))
            nl--;
        else
            ph |= 1 << i;
    }
    if (nl == (int)c->nLeaves) return 0;
    t = tt_shrink(t, ph);
    c->tt = t & 0xFFFFu;
    c->sign = 0;
    for (uint32_t i = 0, k = 0; i < c->nLeaves; i++)
        if (ph >> i & 1) {
            c->leaves[k++] = c->leaves[i];
            c->sign |= 1u << (lidLow[c->leaves[i]] & 31u);
        }
    c->nLeaves = (uint32_t)nl;
    return 1;
}

// The CutEnumerate body for one pair (src/algorithms/rewrite.cu:282-291).
// Returns 1 when enumeration of this node must stop (a cut with fewer than
// two leaves was produced).
CULS_HD int enum_pair(Cut *s, const Cut &a, const Cut &b, int ca, int cb, const int *ref, const uint8_t *lidLow) {
    if (popc32(a.sign | b.sign) > 4) return 0;
    int id = find_slot(s);
    if (!merge_cuts(a, b, &s[id])) return 0;
    if (cut_filter(s, id)) return 0;
    s[id].tt = cut_truth(s[id], a, b, ca, cb);
    if (cut_minimize(&s[id], lidLow)) cut_filter(s, id);
    s[id].value = cut_value(s[id], ref);
    return s[id].nLeaves < 2 ? 1 : 0;
}

// ------------------------------------------------------ existence table
// Open-addressing table of AND nodes keyed by (fanin0 id, fanin1 id,
// compl0, compl1): the role of BuildHashTable/TableLookup
// (src/algorithms/rewrite.cu:328-367,450-471).  Duplicate keys keep the
// smallest position.
CULS_HD unsigned long long and_key(int in0, int in1, int c0, int c1) {
    return ((unsigned long long)(uint32_t)in0 << 32) | ((unsigned long long)(uint32_t)in1 << 2) |
           ((unsigned long long)c0 << 1) | (unsigned long long)c1;
}

// A slot holds its key and, in one 64-bit word, the lowest rank inserted
// with it and that insertion's position (rank << 32 | position), so that an
// insertion's CAS and min touch one 32-byte sector and a lookup finds the
// winner's position without a rank-to-position table.  Empty: key
// kEmptyKey, rank and position kEmptyRp.
struct alignas(16) AndSlot {
    unsigned long long key;
    unsigned long long rp;
};
constexpr unsigned long long kEmptyRp = 0x7F7F7F7F7F7F7F7Full;
CULS_HD int slot_rank(unsigned long long rp) { return (int)(rp >> 32); }
CULS_HD int slot_pos(unsigned long long rp) { return (int)(uint32_t)rp; }

struct AndTable {
    AndSlot *slots;
    uint32_t mask;  // capacity - 1 (capacity is a power of two)
};

#ifdef __CUDACC__
// Empties n slots on stream s.
inline cudaError_t and_table_clear(AndSlot *slots, int64_t n, cudaStream_t s) {
    return fill_i4(reinterpret_cast<int4 *>(slots), make_int4(-1, -1, 0x7F7F7F7F, 0x7F7F7F7F), n, s);
}
#endif

// Inserts key with (rank, pos): the slot keeps the lowest rank and its
// position.  Returns the slot, or -1 (and kDevTableFull) when the probe
// sequence runs out.
CULS_HD int table_insert(const AndTable &t, unsigned long long key, int rank, int pos, int *status) {
    uint32_t h = (uint32_t)mix64(key) & t.mask;
    for (uint32_t probe = 0; probe <= t.mask; probe++) {
        unsigned long long prev = at_cas(&t.slots[h].key, kEmptyKey, key);
        if (prev == kEmptyKey || prev == key) {
            at_min(&t.slots[h].rp, ((unsigned long long)(uint32_t)rank << 32) | (uint32_t)pos);
            return (int)h;
        }
        h = (h + 1) & t.mask;
    }
    set_status(status, kDevTableFull);
    return -1;
}

// Returns the lowest rank stored for key, or -1 when absent.
CULS_HD int table_find(const AndTable &t, unsigned long long key, int *status) {
    uint32_t h = (uint32_t)mix64(key) & t.mask;
    for (uint32_t probe = 0; probe <= t.mask; probe++) {
        unsigned long long k = t.slots[h].key;
        if (k == key) return slot_rank(t.slots[h].rp);
        if (k == kEmptyKey) return -1;
        h = (h + 1) & t.mask;
    }
    set_status(status, kDevTableFull);
    return -1;
}

// TableLookup, src/algorithms/rewrite.cu:346-367 (ids swapped, not literals)
CULS_HD int and_lookup(const AndTable &t, int in0, int in1, int c0, int c1, int *status) {
    if (in0 > in1) {
        int x = in0;
        in0 = in1;
        in1 = x;
        x = c0;
        c0 = c1;
        c1 = x;
    }
    return table_find(t, and_key(in0, in1, c0, c1), status);
}

// ---------------------------------------- per-graph existence table
// The existence table of one rewriting pass, split by graph: graph g owns
// slots [off[g], off[g + 1]) and only its own nodes are inserted into or
// looked up in that region, so passes that visit the nodes graph by graph
// keep the region they probe resident in L2.  A slot is 16 bytes {key,
// value}, so a probe touches one sector.  Duplicate keys keep the smallest
// position, as in AndTable.
struct alignas(16) TabSlot {
    unsigned long long key;
    int val;  // smallest position with this key
    int lvl;  // its level (equal for all nodes with one key: same fanins)
};

struct RegionTable {
    TabSlot *slots;
    const int64_t *off;  // G + 1 slot offsets
};

struct TabRegion {
    TabSlot *slots;
    uint32_t size;
};

CULS_HD TabRegion table_region(const RegionTable &t, int g) {
    const int64_t a = t.off[g], b = t.off[g + 1];
    return TabRegion{t.slots + a, (uint32_t)(b - a)};
}

// Home slot: a multiplicative hash of the key's two 32-bit halves (odd
// constants from the golden ratio and MurmurHash3), its high bits scaled
// onto [0, size) by a multiply-high.  Two 32-bit multiplies keep the probe
// short; linear probing at load <= 1/2 tolerates its weaker mixing.
CULS_HD uint32_t region_home(unsigned long long key, uint32_t size) {
    const uint32_t h = (uint32_t)(key >> 32) * 0x9E3779B1u + (uint32_t)key * 0x85EBCA6Bu;
    return (uint32_t)(((unsigned long long)(h ^ (h >> 15)) * size) >> 32);
}

CULS_HD int region_insert(const TabRegion &t, unsigned long long key, int val, int lvl, int *status) {
    uint32_t h = region_home(key, t.size);
    for (uint32_t probe = 0; probe < t.size; probe++) {
        unsigned long long prev = at_cas(&t.slots[h].key, kEmptyKey, key);
        if (prev == kEmptyKey || prev == key) {
            at_min(&t.slots[h].val, val);
            t.slots[h].lvl = lvl;
            return (int)h;
        }
        if (++h == t.size) h = 0;
    }
    set_status(status, kDevTableFull);
    return -1;
}

// Lookup in a region that no thread writes during the calling kernel.
CULS_HD int region_find(const TabRegion &t, unsigned long long key, int *status) {
    uint32_t h = region_home(key, t.size);
    for (uint32_t probe = 0; probe < t.size; probe++) {
#if defined(__CUDA_ARCH__)
        const int4 s = *reinterpret_cast<const int4 *>(&t.slots[h]);
        const unsigned long long k = ((unsigned long long)(uint32_t)s.y << 32) | (uint32_t)s.x;
        if (k == key) return s.z;
#else
        const unsigned long long k = t.slots[h].key;
        if (k == key) return t.slots[h].val;
#endif
        if (k == kEmptyKey) return -1;
        if (++h == t.size) h = 0;
    }
    set_status(status, kDevTableFull);
    return -1;
}

CULS_HD int4 region_load(const TabRegion &t, uint32_t h) {
#if defined(__CUDA_ARCH__)
    return *reinterpret_cast<const int4 *>(&t.slots[h]);
#else
    const TabSlot &x = t.slots[h];
    return int4{(int)(uint32_t)x.key, (int)(uint32_t)(x.key >> 32), x.val, x.lvl};
#endif
}

// Finishes a lookup whose home slot was already loaded into s: returns
// {position, level} of the key, or {-1, 0} when absent.  The home index is
// recomputed only when the probe goes on past it.
CULS_HD int2 region_resolve(const TabRegion &t, unsigned long long key, int4 s, int *status) {
    uint32_t h = 0;
    for (uint32_t probe = 0; probe < t.size; probe++) {
        if (probe > 0) {
            if (probe == 1) h = region_home(key, t.size);
            if (++h == t.size) h = 0;
            s = region_load(t, h);
        }
        const unsigned long long k = ((unsigned long long)(uint32_t)s.y << 32) | (uint32_t)s.x;
        if (k == key) return int2{s.z, s.w};
        if (k == kEmptyKey) return int2{-1, 0};
    }
    set_status(status, kDevTableFull);
    return int2{-1, 0};
}

// TableLookup (src/algorithms/rewrite.cu:346-367) on a graph's region.
CULS_HD int region_and_lookup(const TabRegion &t, int in0, int in1, int c0, int c1, int *status) {
    if (in0 > in1) {
        int x = in0;
        in0 = in1;
        in1 = x;
        x = c0;
        c0 = c1;
        c1 = x;
    }
    return region_find(t, and_key(in0, in1, c0, c1), status);
}

// --------------------------------------------------------- evaluation
struct EvalIn {
    const int *L0, *L1;  // fanin literals (the constant and PIs point at the constant)
    const int *ref;      // fanout counts incl. PO references
    const int *level;
    const RwLib *lib;
    TabRegion tab;       // the region of the evaluated node's graph
    int *status;
};

// 8-entry reference table of CalcMFFC (src/algorithms/rewrite.cu:296-316).
// Every access below names its entry by a literal index (CULS_EACH8), never
// by a loop variable left to the unroller, so the table stays in registers
// however large the calling kernel grows.
struct MffcTab {
    int size;
    int id[8];
    int num[8];
};

#define CULS_EACH8(X) X(0) X(1) X(2) X(3) X(4) X(5) X(6) X(7)

CULS_HD int pick8(const int (&v)[8], int i) {
    int r = v[0];
#define CULS_PICK8(k) \
    if (k == i) r = v[k];
    CULS_EACH8(CULS_PICK8)
#undef CULS_PICK8
    return r;
}

// Decrease, src/algorithms/rewrite.cu:296-309.  *slot receives the table
// entry whose count was returned (unchanged for leaves and a full table).
CULS_HD int mffc_decrease(int v, MffcTab &t, const int (&leaves)[4], const int *ref, int *slot) {
    if (v == leaves[0] || v == leaves[1] || v == leaves[2] || v == leaves[3]) return 1;
    int found = -1;
#define CULS_FIND8(k) \
    if (found < 0 && k < t.size && t.id[k] == v) found = k;
    CULS_EACH8(CULS_FIND8)
#undef CULS_FIND8
    if (found >= 0) {
        int r = 0;
#define CULS_DEC8(k) \
    if (k == found) r = --t.num[k];
        CULS_EACH8(CULS_DEC8)
#undef CULS_DEC8
        *slot = found;
        return r;
    }
    if (t.size == 8) return 1;
    const int r = ref[v] - 1;
#define CULS_ADD8(k)    \
    if (k == t.size) {  \
        t.id[k] = v;    \
        t.num[k] = r;   \
    }
    CULS_EACH8(CULS_ADD8)
#undef CULS_ADD8
    *slot = t.size;
    t.size++;
    return r;
}

// Bit i set when table entry i exists with a zero count: the entries
// IsDeleted (src/algorithms/rewrite.cu:312-316) reports.  Table ids are
// distinct, so the counts are no longer needed once this mask is taken.
CULS_HD uint32_t mffc_zero_mask(const MffcTab &t) {
    uint32_t z = 0;
#define CULS_ZERO8(k) \
    if (k < t.size && t.num[k] == 0) z |= 1u << k;
    CULS_EACH8(CULS_ZERO8)
#undef CULS_ZERO8
    return z;
}

// IsDeleted, src/algorithms/rewrite.cu:312-316, on the ids and zero mask
CULS_HD int mffc_deleted(int v, const int (&id)[8], uint32_t zero) {
    if (!zero) return 0;  // the common case: the MFFC is the root alone
    int del = 0;
#define CULS_DEL8(k) del |= ((zero >> k) & 1u) && id[k] == v;
    CULS_EACH8(CULS_DEL8)
#undef CULS_DEL8
    return del;
}

// CalcMFFC, src/algorithms/rewrite.cu:319-326, with the recursion replayed
// on a register stack.  A frame above the root is entered only when a table
// count reaches zero, so it is named by its table entry (3 bits); its state
// (next fanin to visit) takes 2 bits.  At most nine frames exist (eight
// table entries plus the root), and the result -- the root plus every node
// entered -- is the number of frames pushed.
CULS_HD int mffc_size(const EvalIn &E, int root, const int (&leaves)[4], MffcTab &t) {
    uint32_t idxs = 0, states = 0;
    int sp = 0, count = 1;
    while (true) {
        const int cur = sp == 0 ? root : pick8(t.id, (int)((idxs >> (3 * sp)) & 7u));
        const uint32_t st = (states >> (2 * sp)) & 3u;
        if (st < 2) {
            const int v = (st == 0 ? E.L0[cur] : E.L1[cur]) >> 1;
            states += 1u << (2 * sp);
            int slot = 0;
            if (mffc_decrease(v, t, leaves, E.ref, &slot) == 0) {
                if (sp + 1 >= 10) {
                    set_status(E.status, kDevStackOverflow);
                    return count;
                }
                sp++;
                idxs = (idxs & ~(7u << (3 * sp))) | ((uint32_t)slot << (3 * sp));
                states &= ~(3u << (2 * sp));
                count++;
            }
            continue;
        }
        if (sp == 0) return count;
        sp--;
    }
}

// True when CalcMFFC of root w.r.t. these leaves is the root alone and no
// table count reaches zero: its first two Decrease calls (the root's
// fanins) are then all that runs.  A count reaches zero only for a fanin that
// is not a leaf and has one reference, or -- both fanins the same node -- two.
CULS_HD bool mffc_trivial(const EvalIn &E, int root, const int (&leaves)[4]) {
    const int f0 = E.L0[root] >> 1, f1 = E.L1[root] >> 1;
    const bool l0 = f0 == leaves[0] || f0 == leaves[1] || f0 == leaves[2] || f0 == leaves[3];
    const bool l1 = f1 == leaves[0] || f1 == leaves[1] || f1 == leaves[2] || f1 == leaves[3];
    if (f0 == f1) return l0 || E.ref[f0] > 2;
    return (l0 || E.ref[f0] >= 2) && (l1 || E.ref[f1] >= 2);
}

CULS_HD int clz64(uint64_t x) {
#if defined(__CUDA_ARCH__)
    return __clzll((long long)x);
#else
    return __builtin_clzll(x);
#endif
}

// Number of library nodes the subgraph rooted at rt adds: unmatched nodes
// reachable from rt through unmatched nodes (Eval, rewrite.cu:369-374).
// unmatched has bit j set for library node j without a match.  A node is
// matched only when both its fanins are (inputs always are), so a matched
// node's whole cone is matched and every unmatched node of rt's cone is
// reached through unmatched nodes: the count is the unmatched part of the
// cone.
CULS_HD int lib_added(const RwLib *lib, int cls, int out, uint64_t unmatched) {
    return popc64(lib->rootCone[cls][out] & unmatched);
}

// One library node of an evaluation batch (the body of EvaluateNode's node
// loop, src/algorithms/rewrite.cu:400-428), split in two so that a batch's
// table probes are in flight together: lib_probe_issue sets the node's level
// from its fanins and, when both fanins are matched (and not to the root),
// loads the home slot of its structural-hash key; lib_probe_finish resolves
// the probe into a match or marks the node unmatched.
struct LibProbe {
    unsigned long long key;
    int4 slot;  // the key's home slot
    int num;    // library index, or -1 when no probe is pending
};

template <class LevT>
CULS_HD void lib_probe_issue(const EvalIn &E, int q, uint32_t w, int isC, int *match, LevT *mlev, int stride,
                             uint64_t &unmatched, LibProbe &p) {
    p.num = -1;
    if (w == kNoLibNode) return;
    const int num = (int)((w >> 18) & 63u) + 4;
    const int in0 = ln_f0(w), in1 = ln_f1(w);
    const int m0 = match[in0 * stride], m1 = match[in1 * stride];
    const int lv0 = mlev[in0 * stride], lv1 = mlev[in1 * stride];
    mlev[num * stride] = (LevT)(1 + (lv0 > lv1 ? lv0 : lv1));
    match[num * stride] = -1;
    const bool uin0 = in0 >= 4 && ((unmatched >> in0) & 1ull);
    const bool uin1 = in1 >= 4 && ((unmatched >> in1) & 1ull);
    if (uin0 || uin1 || m0 == q || m1 == q) {
        unmatched |= 1ull << num;
        return;
    }
    // the reference's isC mask only has input bits (0..3)
    int cc0 = (in0 < 4 ? ((isC >> in0) & 1) : 0) ^ ln_c0(w);
    int cc1 = (in1 < 4 ? ((isC >> in1) & 1) : 0) ^ ln_c1(w);
    int a = m0, b = m1;
    if (a > b) {  // TableLookup orders the ids
        const int x = a;
        a = b;
        b = x;
        const int y = cc0;
        cc0 = cc1;
        cc1 = y;
    }
    p.key = and_key(a, b, cc0, cc1);
    p.slot = region_load(E.tab, region_home(p.key, E.tab.size));
    p.num = num;
}

// IsDeleted (src/algorithms/rewrite.cu:312-316) on the MFFC's nodes: the
// table entries whose count reached zero, nDel of them at del.
CULS_HD bool mffc_member(int v, int nDel, const int *del) {
    for (int j = 0; j < nDel; j++)
        if (del[j] == v) return true;
    return false;
}

template <class LevT>
CULS_HD void lib_probe_finish(const EvalIn &E, const LibProbe &p, int nDel, const int *del, int *match, LevT *mlev,
                              int stride, uint64_t &unmatched) {
    if (p.num < 0) return;
    // the slot carries the node's level, so a hit needs no second load
    const int2 r = region_resolve(E.tab, p.key, p.slot, E.status);
    if (r.x != -1 && !mffc_member(r.x, nDel, del)) {
        match[p.num * stride] = r.x;
        mlev[p.num * stride] = (LevT)r.y;
    } else {
        unmatched |= 1ull << p.num;
    }
}

template <class T>
CULS_HD T pick4v(const T (&v)[4], int i) {
    return i == 0 ? v[0] : (i == 1 ? v[1] : (i == 2 ? v[2] : v[3]));
}

// Best replacement of one cut: the body of EvaluateNode's cut loop
// (src/algorithms/rewrite.cu:386-445) for cut slot packed word pk with
// leaves l.  match/mlev are 54-entry scratch arrays with element j at
// index j * stride.  Returns the first root (in root order) with the highest
// gain and, among equal gains, the lowest level: out < 0 when no root
// qualifies.
struct CutBest {
    int gain, level, out;
};

// LevT holds library-node levels: int, or uint16_t when every level of the
// graph plus the forest depth stays below 65,535.
//
// saved is CalcMFFC's count for this cut, and del its nDel MFFC nodes (the
// table entries whose count reached zero), computed beforehand.
template <class LevT>
CULS_HD CutBest eval_cut(const EvalIn &E, int q, int cpos, uint32_t pk, int4 l, bool useZeros, int *match, LevT *mlev,
                         int stride, int saved, int nDel, const int *del) {
    CutBest best{-1, 0, -1};
    const uint32_t nLeaves = packed_nleaves(pk);
    const int leaves[4] = {l.x, l.y, l.z, nLeaves == 3 ? cpos : l.w};
    const uint32_t npn = E.lib->npn[pk & 0xFFFFu];
    const int uPhase = npn_phase(npn), cls = npn_class(npn);
    const uint32_t perm = *reinterpret_cast<const uint32_t *>(E.lib->perm4[npn_perm(npn)]);
    int isC = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int m = pick4v(leaves, (int)((perm >> (8 * j)) & 255u));
        match[j * stride] = m;
        mlev[j * stride] = (LevT)E.level[m];
        if (uPhase >> j & 1) isC |= 1 << j;
    }
    // The library nodes in the reference's index order, regrouped into
    // batches of equal depth: every node reads only its fanins' entries, so
    // this order yields the same match, level and unmatched bits.
    uint64_t unmatched = 0;
    const int nb = E.lib->nBatches[cls];
    const uint4 *lbatch = E.lib->batch[cls];
    for (int bi = 0; bi < nb; bi++) {
        const uint4 bw = lbatch[bi];
        LibProbe p0, p1, p2, p3;  // the batch's probes in flight together
        lib_probe_issue(E, q, bw.x, isC, match, mlev, stride, unmatched, p0);
        lib_probe_issue(E, q, bw.y, isC, match, mlev, stride, unmatched, p1);
        lib_probe_issue(E, q, bw.z, isC, match, mlev, stride, unmatched, p2);
        lib_probe_issue(E, q, bw.w, isC, match, mlev, stride, unmatched, p3);
        lib_probe_finish(E, p0, nDel, del, match, mlev, stride, unmatched);
        lib_probe_finish(E, p1, nDel, del, match, mlev, stride, unmatched);
        lib_probe_finish(E, p2, nDel, del, match, mlev, stride, unmatched);
        lib_probe_finish(E, p3, nDel, del, match, mlev, stride, unmatched);
    }
    const int nr = E.lib->nRoots[cls];
    for (int out = 0; out < nr; out++) {
        const int rt = E.lib->roots[cls][out];
        if (match[rt * stride] == q) continue;
        const int added = lib_added(E.lib, cls, out, unmatched);
        const int rtLevel = mlev[rt * stride];
        const int gain = saved - added;
        if (gain < 0 || (gain == 0 && !useZeros)) continue;
        if (best.out >= 0 && (gain < best.gain || (gain == best.gain && rtLevel >= best.level))) continue;
        best = CutBest{gain, rtLevel, out};
    }
    return best;
}

// EvaluateNode's choice across cuts (src/algorithms/rewrite.cu:378-447):
// cuts in slot order, a later cut wins only with a higher gain or an equal
// gain at a lower level.  Folds cut i's best into (bestCut, bestOut, gain,
// level).
CULS_HD void fold_cut_best(const CutBest &c, int i, int &bestCut, int &bestOut, int &gain, int &level) {
    if (c.out < 0) return;
    if (bestCut >= 0 && (c.gain < gain || (c.gain == gain && c.level >= level))) return;
    bestCut = i;
    bestOut = c.out;
    gain = c.gain;
    level = c.level;
}

}  // namespace culs
