// ORACLE -- test infrastructure only.
//
// A sequential CPU restatement of CULS's `rw` (AIG rewriting, DAC'22
// "NovelRewrite") followed by its GPU-strash deduplication, and of `st`.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
// load this library, and only as the checker or the timed CPU baseline.  The
// product path (libculs_b200.so) never links or calls it.
//
// Every function names the reference code it restates (paths relative to the
// CULS source tree).  Where the reference is nondeterministic the oracle fixes
// one deterministic outcome and says which:
//   * strash duplicate keys inside one frontier: the smallest tentative id
//     wins (reference: whichever thread's atomicCAS lands first,
//     src/hash_table/hash_table.h:472-491);
//   * new-node ids in ReplaceSubgr: assigned as if the per-node threads ran
//     one after another in node-id order (reference: atomicAdd order,
//     src/algorithms/rewrite.cu:482);
//   * duplicate keys in the rewrite's chained existence table: the smallest
//     node id is returned (reference: first entry in the chain; never
//     ambiguous on a strashed input).
// The GPU strash in the reference never assigns a consecutive id to the first
// winner when that winner's tentative id is not nPIs+1
// (src/aig/strash.cu:113-123); the oracle assigns ranks to every winner.

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

namespace orc {

static const int kNtt = 1 << 16;
static const int kNcls = 222;

// Rewriting library, decoded from the project's rwlib.bin (same values as
// CULS src/algorithms/rewrite_library.inc, see culs_b200/data/make_rwlib.py).
struct Lib {
    uint8_t phase[kNtt], perm[kNtt], perm4[24][4], cls[kNtt];
    uint8_t nNodes[kNcls], nRoots[kNcls];
    uint8_t f0[kNcls][56], f1[kNcls][56], c0[kNcls][56], c1[kNcls][56];
    uint8_t roots[kNcls][16];
};

static bool load_lib(const char *path, Lib &L) {
    FILE *f = fopen(path, "rb");
    if (!f) return false;
    std::vector<uint8_t> b;
    uint8_t buf[65536];
    size_t k;
    while ((k = fread(buf, 1, sizeof buf, f)) > 0) b.insert(b.end(), buf, buf + k);
    fclose(f);
    if (b.size() < 40 || memcmp(b.data(), "CULSRWL1", 8) != 0) return false;
    size_t cur = 40;
    auto take = [&](uint8_t *dst, size_t n) {
        if (cur + n > b.size()) return false;
        memcpy(dst, b.data() + cur, n);
        cur += n;
        return true;
    };
    if (!take(L.phase, kNtt) || !take(L.perm, kNtt) || !take(&L.perm4[0][0], 96) ||
        !take(L.cls, kNtt) || !take(L.nNodes, kNcls) || !take(L.nRoots, kNcls))
        return false;
    memset(L.f0, 0, sizeof L.f0);
    memset(L.f1, 0, sizeof L.f1);
    memset(L.c0, 0, sizeof L.c0);
    memset(L.c1, 0, sizeof L.c1);
    memset(L.roots, 0, sizeof L.roots);
    for (int c = 0; c < kNcls; c++) {
        for (int i = 0; i < L.nNodes[c]; i++) {
            uint8_t q[4];
            if (!take(q, 4)) return false;
            L.f0[c][i] = q[0];
            L.f1[c][i] = q[1];
            L.c0[c][i] = q[2];
            L.c1[c][i] = q[3];
        }
        if (!take(L.roots[c], L.nRoots[c])) return false;
    }
    return cur == b.size();
}

// One cut slot: the fields of rw::Cut (src/algorithms/rewrite.h:10-16).
struct Cut {
    uint32_t sign;
    int32_t leaves[4];
    uint32_t tt;      // 16 bits used
    uint32_t value;   // 11 bits used
    uint32_t nLeaves; // 4 bits used
    uint32_t used;
};

static inline int lid(int lit) { return lit >> 1; }
static inline int lc(int lit) { return lit & 1; }
// AIGMan keeps literal 0 as constant TRUE; AIGER (and rw::CPUSolver) keep 0
// as FALSE.  src/common.h:24-27.
static inline int invConst(int lit) { return (lit >= 0 && lit < 2) ? 1 - lit : lit; }

// ---------------------------------------------------------------- cut helpers
// src/algorithms/rewrite.cu:49-61
static uint32_t cut_value(const Cut &c, const int *nRef) {
    int value = 0, nOnes = 0;
    for (uint32_t i = 0; i < c.nLeaves; i++) {
        value += nRef[c.leaves[i]];
        nOnes += (nRef[c.leaves[i]] == 1);
    }
    if (c.nLeaves < 2) return 1001;
    if (value > 1000) value = 1000;
    if (nOnes > 3) value = 5 - nOnes;
    return (uint32_t)value & 0x7FF;
}

// src/algorithms/rewrite.cu:84-109
static int find_slot(Cut *s) {
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

// src/algorithms/rewrite.cu:112-153 (a has at least as many leaves as b)
static int merge_ordered(const Cut &a, const Cut &b, Cut *out) {
    int c = 0, i = 0, k = 0;
    int na = (int)a.nLeaves, nb = (int)b.nLeaves;
    for (c = 0; c < 4; c++) {
        if (k == nb) {
            if (i == na) {
                out->nLeaves = c;
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
    out->nLeaves = c;
    return 1;
}

// src/algorithms/rewrite.cu:155-164
static int merge(const Cut &a, const Cut &b, Cut *out) {
    if (a.nLeaves >= b.nLeaves) {
        if (!merge_ordered(a, b, out)) return 0;
    } else {
        if (!merge_ordered(b, a, out)) return 0;
    }
    out->sign = a.sign | b.sign;
    out->used = 1;
    return 1;
}

// src/algorithms/rewrite.cu:167-175: every leaf of a is a leaf of b
static int subset(const Cut &a, const Cut &b) {
    for (uint32_t i = 0; i < a.nLeaves; i++) {
        int ok = 0;
        for (uint32_t j = 0; j < b.nLeaves; j++)
            if (b.leaves[j] == a.leaves[i]) ok = 1;
        if (!ok) return 0;
    }
    return 1;
}

// src/algorithms/rewrite.cu:178-193
static int filter(Cut *s, int id) {
    for (int i = 0; i < 8; i++) {
        if (i == id || !s[i].used) continue;
        if (s[i].nLeaves > s[id].nLeaves) {
            if ((s[i].sign & s[id].sign) != s[id].sign) continue;
            if (subset(s[id], s[i])) s[i].used = 0;
        } else {
            if ((s[i].sign & s[id].sign) != s[i].sign) continue;
            if (subset(s[i], s[id])) {
                s[id].used = 0;
                return 1;
            }
        }
    }
    return 0;
}

// src/algorithms/rewrite.cu:203-211 (operates on the low 16 bits only; the
// reference's 32-bit ints carry the same low half)
static uint32_t swap_adj(uint32_t t, int v) {
    if (v == 0) return (t & 0x9999u) | ((t & 0x2222u) << 1) | ((t & 0x4444u) >> 1);
    if (v == 1) return (t & 0xC3C3u) | ((t & 0x0C0Cu) << 2) | ((t & 0x3030u) >> 2);
    if (v == 2) return (t & 0xF00Fu) | ((t & 0x00F0u) << 4) | ((t & 0x0F00u) >> 4);
    return 0;
}

// src/algorithms/rewrite.cu:195-201
static int truth_phase(const Cut &x, const Cut &cut) {
    int ph = 0;
    for (uint32_t i = 0; i < cut.nLeaves; i++)
        for (uint32_t j = 0; j < x.nLeaves; j++)
            if (x.leaves[j] == cut.leaves[i]) ph |= 1 << i;
    return ph;
}

// src/algorithms/rewrite.cu:213-221
static uint32_t stretch(uint32_t t, int nVar, int ph) {
    int var = nVar - 1;
    for (int i = 3; i >= 0; i--)
        if (ph >> i & 1) {
            for (int k = var; k < i; k++) t = swap_adj(t, k);
            var--;
        }
    return t;
}

// src/algorithms/rewrite.cu:223-229
static uint32_t cut_truth(const Cut &cut, const Cut &a, const Cut &b, int ca, int cb) {
    uint32_t t0 = ca ? (~a.tt & 0xFFFFu) : a.tt;
    uint32_t t1 = cb ? (~b.tt & 0xFFFFu) : b.tt;
    t0 = stretch(t0, (int)a.nLeaves, truth_phase(a, cut));
    t1 = stretch(t1, (int)b.nLeaves, truth_phase(b, cut));
    return (t0 & t1) & 0xFFFFu;
}

// src/algorithms/rewrite.cu:231-241
static uint32_t shrink(uint32_t t, int ph) {
    int var = 0;
    for (int i = 0; i < 4; i++)
        if (ph & (1 << i)) {
            for (int k = i - 1; k >= var; k--) t = swap_adj(t, k);
            var++;
        }
    return t;
}

// src/algorithms/rewrite.cu:243-266
static int minimize(Cut *c) {
    static const uint32_t m0[4] = {0x5555, 0x3333, 0x0F0F, 0x00FF};
    static const uint32_t m1[4] = {0xAAAA, 0xCCCC, 0xF0F0, 0xFF00};
    int ph = 0;
    uint32_t t = c->tt & 0xFFFF;
    int nl = (int)c->nLeaves;
    for (uint32_t i = 0; i < c->nLeaves; i++) {
        if ((t & m0[i]) == ((t & m1[i]) >> (1 << i)))
            nl--;
        else
            ph |= 1 << i;
    }
    if (nl == (int)c->nLeaves) return 0;
    t = shrink(t, ph);
    c->tt = t & 0xFFFF;
    c->sign = 0;
    for (uint32_t i = 0, k = 0; i < c->nLeaves; i++)
        if (ph >> i & 1) {
            c->leaves[k++] = c->leaves[i];
            c->sign |= 1u << (31 & c->leaves[i]);
        }
    c->nLeaves = (uint32_t)nl;
    return 1;
}

// ------------------------------------------------------------ choice codes
enum ChoiceCode {
    kNotVisited = 0,
    kNoCut = 1,      // selected cut unused
    kSmallCut = 2,   // fewer than 3 leaves
    kNoReplace = 3,  // replace[i] == -1
    kSelfRef = 4,    // newIdx == i or fanin1(newIdx) == i
    kCompromised = 5,
    kCommitted = 6,
    kReverted = 7,
};

struct Graph {  // AIGMan layout (src/aig_manager.h:51-58), lit 0 = TRUE
    int nPIs = 0, nPOs = 0, nObjs = 1;
    std::vector<int> f0, f1, outs;
    int nLevels = 0;
};

struct Stats {
    long long replaced = 0, replacedPos = 0, replacedZero = 0, reverted = 0, compromised = 0, preEval = 0,
              smallCut = 0, newIdx = 0, expected = 0, nNewNodes = 0;
};

// ------------------------------------------------------------- rw solver
// Restates rw::CPUSolver (src/algorithms/rewrite.h:67-325,
// src/algorithms/rewrite.cu:780-938,1229-1307) together with the kernels of
// rw::GPUSolver run sequentially (src/algorithms/rewrite.cu:63-555,634-770).
struct Solver {
    const Lib *lib = nullptr;
    int n = 0, numInputs = 0, numOutputs = 0, nLevels = -1;
    std::vector<int> fanin0, fanin1, ref, phase, level, isDeleted, output, order, temp0, temp1;
    std::vector<int> levelCount;

    // dumps
    std::vector<int> dReorderF0, dReorderF1, dReorderOut;
    std::vector<Cut> dCuts, dSelected;
    std::vector<int> dBestOut, dReplace, dNewF0, dNewF1, dChoice;
    int dN0 = 0, dN1 = 0;
    Stats st;

    void ensure(size_t m) {
        if (fanin0.size() < m) {
            size_t cap = std::max(m, fanin0.size() * 2);
            for (auto *v : {&fanin0, &fanin1, &ref, &phase, &level, &isDeleted, &order, &temp0, &temp1})
                v->resize(cap, 0);
        }
    }

    // src/algorithms/rewrite.cu:780-809
    void reset(const Graph &g) {
        numInputs = g.nPIs;
        numOutputs = g.nPOs;
        n = g.nObjs - 1;
        fanin0.assign(n + 1, 0);
        fanin1.assign(n + 1, 0);
        ref.assign(n + 1, 0);
        phase.assign(n + 1, 0);
        level.assign(n + 1, 0);
        isDeleted.assign(n + 1, 0);
        order.assign(n + 1, 0);
        temp0.assign(n + 1, 0);
        temp1.assign(n + 1, 0);
        for (int i = numInputs + 1; i <= n; i++) {
            fanin0[i] = invConst(g.f0[i]);
            fanin1[i] = invConst(g.f1[i]);
        }
        output.assign(numOutputs, 0);
        for (int i = 0; i < numOutputs; i++) output[i] = invConst(g.outs[i]);
        reorder();
    }

    // rw::CPUSolver::TopoSort, src/algorithms/rewrite.h:291-294 (iterative
    // post-order; same result as the recursion)
    int topo(int root) {
        if (level[root] != -1) return level[root];
        std::vector<int> stk;
        stk.push_back(root);
        while (!stk.empty()) {
            int v = stk.back();
            if (level[v] != -1) {
                stk.pop_back();
                continue;
            }
            int a = lid(fanin0[v]), b = lid(fanin1[v]);
            bool ready = true;
            if (level[a] == -1) {
                stk.push_back(a);
                ready = false;
            }
            if (level[b] == -1) {
                stk.push_back(b);
                ready = false;
            }
            if (ready) {
                level[v] = 1 + std::max(level[a], level[b]);
                stk.pop_back();
            }
        }
        return level[root];
    }

    // src/algorithms/rewrite.h:296-307
    void count_levels() {
        int maxLevel = 0;
        for (int i = 1; i <= n; i++)
            if (!isDeleted[i]) maxLevel = std::max(maxLevel, level[i]);
        levelCount.assign(maxLevel + 1, 0);
        for (int i = 1; i <= n; i++)
            if (!isDeleted[i]) levelCount[level[i]]++;
        for (int i = 1; i <= maxLevel; i++) levelCount[i] += levelCount[i - 1];
        nLevels = maxLevel;
    }

    // src/algorithms/rewrite.cu:1245-1279
    void reorder() {
        for (int i = 1; i <= n; i++) level[i] = i <= numInputs ? 0 : -1;
        level[0] = 0;
        for (int i = numInputs + 1; i <= n; i++) isDeleted[i] = 0;
        for (int i = numInputs + 1; i <= n; i++)
            if (!isDeleted[i]) topo(i);
        count_levels();
        int newN = levelCount.back();
        std::vector<int> lc = levelCount;
        for (int i = n; i >= 1; i--)
            if (!isDeleted[i]) order[i] = lc[level[i]]--;
        order[0] = 0;
        for (int i = numInputs + 1; i <= n; i++) {
            temp0[i] = fanin0[i];
            temp1[i] = fanin1[i];
        }
        for (int i = numInputs + 1; i <= n; i++)
            if (!isDeleted[i]) fanin0[order[i]] = order[lid(temp0[i])] * 2 + lc_(temp0[i]);
        for (int i = numInputs + 1; i <= n; i++)
            if (!isDeleted[i]) fanin1[order[i]] = order[lid(temp1[i])] * 2 + lc_(temp1[i]);
        for (int i = 0; i < numOutputs; i++) output[i] = order[lid(output[i])] * 2 + lc_(output[i]);
        n = newN;
        init();
    }
    static int lc_(int lit) { return lit & 1; }

    // src/algorithms/rewrite.cu:1229-1243
    void init() {
        for (int i = numInputs + 1; i <= n; i++)
            if (fanin0[i] > fanin1[i]) std::swap(fanin0[i], fanin1[i]);
        std::fill(isDeleted.begin(), isDeleted.begin() + n + 1, 0);
        std::fill(ref.begin(), ref.begin() + n + 1, 0);
        for (int i = numInputs + 1; i <= n; i++) {
            ref[lid(fanin0[i])]++;
            ref[lid(fanin1[i])]++;
            level[i] = std::max(level[lid(fanin0[i])], level[lid(fanin1[i])]) + 1;
            phase[i] = (phase[lid(fanin0[i])] ^ lc(fanin0[i])) & (phase[lid(fanin1[i])] ^ lc(fanin1[i]));
        }
        for (int i = 0; i < numOutputs; i++) ref[lid(output[i])]++;
    }

    int isRedundant(int node) const {
        return node > numInputs && (fanin0[node] == fanin1[node] || fanin0[node] == 1);
    }
    // src/algorithms/rewrite.h:121-124
    int Fanin(int lit) const {
        int c = 0;
        while (isRedundant(lid(lit))) {
            c ^= lc(lit);
            lit = fanin1[lid(lit)];
        }
        return lit ^ c;
    }

    // src/algorithms/rewrite.h:208-220
    int fastDelete(int node) {
        if (node <= numInputs) return 0;
        int in0 = lid(fanin0[node]), in1 = lid(fanin1[node]);
        ref[in0]--;
        ref[in1]--;
        int cnt = !isRedundant(node);
        if (ref[in0] == 0) cnt += fastDelete(in0);
        if (ref[in1] == 0) cnt += fastDelete(in1);
        isDeleted[node] = 1;
        return cnt;
    }

    // install lambda, src/algorithms/rewrite.cu:835-847
    int install(int idx) {
        if (!isDeleted[idx]) return 0;
        isDeleted[idx] = 0;
        int cnt = !isRedundant(idx);
        cnt += install(lid(fanin0[idx]));
        cnt += install(lid(fanin1[idx]));
        ref[lid(fanin0[idx])]++;
        ref[lid(fanin1[idx])]++;
        return cnt;
    }

    // ------------------------------------------------ GPU stage, sequential
    // Device arrays of rw::GPUSolver after Convert (rewrite.cu:610-616).
    std::vector<int> gF0, gF1, gC0, gC1, gPhase;
    std::vector<Cut> cuts, selected;
    std::vector<int> bestOut;
    std::unordered_map<uint64_t, int> origTable, newTable;

    static uint64_t tkey(int in0, int in1, int c0, int c1) {
        return ((uint64_t)(uint32_t)in0 << 34) | ((uint64_t)(uint32_t)in1 << 2) | ((uint64_t)c0 << 1) | (uint64_t)c1;
    }

    // TableLookup, src/algorithms/rewrite.cu:346-367
    int lookup(std::unordered_map<uint64_t, int> &T, int in0, int in1, int c0, int c1) {
        if (in0 > in1) {
            std::swap(in0, in1);
            std::swap(c0, c1);
        }
        auto it = T.find(tkey(in0, in1, c0, c1));
        return it == T.end() ? -1 : it->second;
    }

    // CutEnumerate, src/algorithms/rewrite.cu:268-294
    void enum_node(int idx) {
        Cut *s = &cuts[(size_t)idx * 8];
        s[0].used = 1;
        s[0].sign = 1u << (idx & 31);
        s[0].tt = 0xAAAA;
        s[0].nLeaves = 1;
        s[0].leaves[0] = idx;
        s[0].value = cut_value(s[0], ref.data());
        int in0 = gF0[idx], in1 = gF1[idx];
        for (int i = 0; i < 8; i++) {
            if (cuts[(size_t)in0 * 8 + i].used != 1) continue;
            for (int j = 0; j < 8; j++) {
                if (cuts[(size_t)in1 * 8 + j].used != 1) continue;
                Cut a = cuts[(size_t)in0 * 8 + i], b = cuts[(size_t)in1 * 8 + j];
                if (__builtin_popcount(a.sign | b.sign) > 4) continue;
                int id = find_slot(s);
                if (!merge(a, b, &s[id])) continue;
                if (filter(s, id)) continue;
                s[id].tt = cut_truth(s[id], a, b, gC0[idx], gC1[idx]);
                if (minimize(&s[id])) filter(s, id);
                s[id].value = cut_value(s[id], ref.data());
                if (s[id].nLeaves < 2) return;
            }
        }
    }

    // Decrease / IsDeleted / CalcMFFC, src/algorithms/rewrite.cu:296-326
    struct MffcTab {
        int size = 0, id[8], num[8];
    };
    int decrease(int v, MffcTab &t, const Cut &cut) {
        for (uint32_t i = 0; i < cut.nLeaves; i++)
            if (v == cut.leaves[i]) return 1;
        for (int i = 0; i < t.size; i++)
            if (t.id[i] == v) return --t.num[i];
        if (t.size == 8) return 1;
        t.id[t.size] = v;
        t.num[t.size] = ref[v] - 1;
        t.size++;
        return ref[v] - 1;
    }
    static int tab_deleted(int v, const MffcTab &t) {
        for (int i = 0; i < t.size; i++)
            if (t.id[i] == v) return t.num[i] == 0;
        return 0;
    }
    int calc_mffc(int cur, const Cut &cut, MffcTab &t) {
        int ans = 1;
        if (decrease(gF0[cur], t, cut) == 0) ans += calc_mffc(gF0[cur], cut, t);
        if (decrease(gF1[cur], t, cut) == 0) ans += calc_mffc(gF1[cur], cut, t);
        return ans;
    }
    // Eval, src/algorithms/rewrite.cu:369-374
    int eval_added(int cur, int *match, int cls, int mark) {
        if (match[cur] > -1) return 0;
        if (match[cur] == mark) return 0;
        match[cur] = mark;
        return 1 + eval_added(lib->f0[cls][cur - 4], match, cls, mark) +
               eval_added(lib->f1[cls][cur - 4], match, cls, mark);
    }

    // EvaluateNode, src/algorithms/rewrite.cu:378-447
    void eval_node(int id, bool fUseZeros) {
        int reduction = -1, bestLevel = 99999999, bestCut = -1, bOut = -1;
        int match[54], matchLevel[54];
        for (int i = 0; i < 8; i++) {
            Cut *cut = &cuts[(size_t)id * 8 + i];
            if (cut->used == 0 || cut->nLeaves < 3) continue;
            int nleaves = (int)cut->nLeaves;
            if (nleaves == 3) cut->leaves[cut->nLeaves++] = 0;
            MffcTab tab;
            int saved = calc_mffc(id, *cut, tab);
            int uPhase = lib->phase[cut->tt];
            int cls = lib->cls[cut->tt];
            const uint8_t *perm = lib->perm4[lib->perm[cut->tt]];
            for (int j = 0; j < 54; j++) match[j] = matchLevel[j] = -1;
            uint64_t isC = 0;
            for (int j = 0; j < 4; j++) {
                match[j] = cut->leaves[perm[j]];
                matchLevel[j] = level[match[j]];
                if (uPhase >> j & 1) isC |= 1ull << j;
            }
            for (int j = 0; j < lib->nNodes[cls]; j++) {
                int num = j + 4;
                int in0 = lib->f0[cls][j], in1 = lib->f1[cls][j];
                matchLevel[num] = 1 + std::max(matchLevel[in0], matchLevel[in1]);
                if (match[in0] == -1 || match[in1] == -1 || match[in0] == id || match[in1] == id) continue;
                int nodeId = lookup(origTable, match[in0], match[in1], (int)((isC >> in0) & 1) ^ lib->c0[cls][j],
                                    (int)((isC >> in1) & 1) ^ lib->c1[cls][j]);
                if (nodeId != -1 && !tab_deleted(nodeId, tab)) {
                    match[num] = nodeId;
                    matchLevel[num] = level[nodeId];
                }
            }
            for (int out = 0; out < lib->nRoots[cls]; out++) {
                int rt = lib->roots[cls][out];
                if (match[rt] == id) continue;
                int added = eval_added(rt, match, cls, -out - 2);
                int rtLevel = matchLevel[rt];
                int gain = saved - added;
                if (gain < 0 || (gain == 0 && !fUseZeros)) continue;
                if (gain < reduction || (gain == reduction && rtLevel >= bestLevel)) continue;
                reduction = gain;
                bestLevel = rtLevel;
                bestCut = i;
                bOut = out;
            }
            cut->nLeaves = (uint32_t)nleaves;
        }
        if (bestCut != -1) {
            selected[id] = cuts[(size_t)id * 8 + bestCut];
            selected[id].used = 1;
            bestOut[id] = bOut;
        } else {
            selected[id].used = 0;
            bestOut[id] = -1;
        }
    }

    // BuildSubgr, src/algorithms/rewrite.cu:473-509 (new ids in node-id order)
    int N = 0;
    void build_subgr(int cur, int cls, int *match, uint64_t isC) {
        if (match[cur] != -1) return;
        int in0 = lib->f0[cls][cur - 4], in1 = lib->f1[cls][cur - 4];
        build_subgr(in0, cls, match, isC);
        build_subgr(in1, cls, match, isC);
        int node = ++N;
        if ((size_t)node >= gF0.size()) {
            size_t cap = gF0.size() * 2 + 16;
            for (auto *v : {&gF0, &gF1, &gC0, &gC1, &gPhase}) v->resize(cap, 0);
        }
        gF0[node] = match[in0];
        gF1[node] = match[in1];
        gC0[node] = lib->c0[cls][cur - 4] ^ (int)((isC >> in0) & 1);
        gC1[node] = lib->c1[cls][cur - 4] ^ (int)((isC >> in1) & 1);
        gPhase[node] = (gPhase[gF0[node]] ^ gC0[node]) & (gPhase[gF1[node]] ^ gC1[node]);
        if (gF0[node] > gF1[node]) {
            std::swap(gF0[node], gF1[node]);
            std::swap(gC0[node], gC1[node]);
        }
        uint64_t k = tkey(gF0[node], gF1[node], gC0[node], gC1[node]);
        auto it = newTable.find(k);
        if (it != newTable.end()) {
            gF0[node] = gF1[node] = -1;
            match[cur] = it->second;
        } else {
            newTable.emplace(k, node);
            match[cur] = node;
        }
    }

    // ReplaceSubgr, src/algorithms/rewrite.cu:511-555
    void replace_node(int id, std::vector<int> &replace) {
        Cut cut = selected[id];
        if (cut.used == 0 || cut.nLeaves < 3) return;
        if (cut.nLeaves == 3) cut.leaves[cut.nLeaves++] = 0;
        int uPhase = lib->phase[cut.tt];
        int cls = lib->cls[cut.tt];
        const uint8_t *perm = lib->perm4[lib->perm[cut.tt]];
        int match[54];
        uint64_t isC = 0;
        for (int j = 0; j < 54; j++) match[j] = -1;
        for (int j = 0; j < 4; j++) {
            match[j] = cut.leaves[perm[j]];
            if (uPhase >> j & 1) isC |= 1ull << j;
        }
        int rt = lib->roots[cls][bestOut[id]];
        uint64_t used = 1ull << rt;
        for (int j = rt; j >= 4; j--)
            if (used >> j & 1) {
                used |= 1ull << lib->f0[cls][j - 4];
                used |= 1ull << lib->f1[cls][j - 4];
            }
        for (int j = 0; j < lib->nNodes[cls]; j++) {
            if (!(used >> (j + 4) & 1)) continue;
            int num = j + 4;
            int in0 = lib->f0[cls][j], in1 = lib->f1[cls][j];
            if (match[in0] == -1 || match[in1] == -1) continue;
            int nodeId = lookup(origTable, match[in0], match[in1], (int)((isC >> in0) & 1) ^ lib->c0[cls][j],
                                (int)((isC >> in1) & 1) ^ lib->c1[cls][j]);
            if (nodeId != -1) match[num] = nodeId;
        }
        if (match[rt] == id) return;
        build_subgr(rt, cls, match, isC);
        replace[id] = match[rt] * 2 + (gPhase[match[rt]] ^ gPhase[id]);
    }

    // CPUSolver::Rewrite, src/algorithms/rewrite.cu:811-938 (GPUReplace=true)
    void rewrite(bool fUseZeros) {
        st = Stats();
        count_levels();
        dN0 = n;
        dReorderF0.assign(fanin0.begin(), fanin0.begin() + n + 1);
        dReorderF1.assign(fanin1.begin(), fanin1.begin() + n + 1);
        dReorderOut = output;

        // EnumerateAndPreEvaluate, rewrite.cu:689-714
        gF0.assign(n + 1, 0);
        gF1.assign(n + 1, 0);
        gC0.assign(n + 1, 0);
        gC1.assign(n + 1, 0);
        gPhase.assign(n + 1, 0);
        for (int i = 0; i <= n; i++) {
            int l0 = (i > numInputs) ? fanin0[i] : 0, l1 = (i > numInputs) ? fanin1[i] : 0;
            gF0[i] = l0 >> 1;
            gC0[i] = l0 & 1;
            gF1[i] = l1 >> 1;
            gC1[i] = l1 & 1;
        }
        cuts.assign((size_t)(n + 1) * 8, Cut{});
        for (int idx = 1; idx <= levelCount[0]; idx++) {  // Inputs, rewrite.cu:63-74
            Cut *c = &cuts[(size_t)idx * 8];
            c->used = 1;
            c->sign = 1u << (idx & 31);
            c->tt = 0xAAAA;
            c->nLeaves = 1;
            c->leaves[0] = idx;
            c->value = cut_value(*c, ref.data());
        }
        for (size_t l = 1; l < levelCount.size(); l++)
            for (int idx = levelCount[l - 1] + 1; idx <= levelCount[l]; idx++) enum_node(idx);
        // BuildHashTable, rewrite.cu:450-471
        origTable.clear();
        origTable.reserve((size_t)n * 2 + 16);
        for (int id = n; id >= 1; id--) {  // descending so the smallest id stays
            if (gF0[id] == 0 && gF1[id] == 0) continue;
            origTable[tkey(gF0[id], gF1[id], gC0[id], gC1[id])] = id;
        }
        selected.assign(n + 1, Cut{});
        bestOut.assign(n + 1, -1);
        for (int id = 1; id <= n; id++) eval_node(id, fUseZeros);
        dCuts = cuts;
        dSelected = selected;
        dBestOut = bestOut;

        // ReplaceSubgraphs, rewrite.cu:716-770
        for (int i = 0; i <= n; i++) gPhase[i] = phase[i];
        std::vector<int> replace(n + 1, -1);
        newTable.clear();
        N = n;
        for (int id = 1; id <= n; id++) replace_node(id, replace);
        st.nNewNodes = N - n;
        // Revert + host rebuild (DFS renumbering of new nodes into n+1..)
        int nn = n;
        std::vector<int> mapping((size_t)N + 1, -1);
        ensure((size_t)nn + (N - nn) + 2);
        std::vector<int> stackR;
        auto litOf = [&](int node, int which) {
            return which == 0 ? gF0[node] * 2 + gC0[node] : gF1[node] * 2 + gC1[node];
        };
        // rebuild, iterative post-order (fanin0 subtree first)
        auto rebuild = [&](int r0) -> int {
            if (r0 <= nn) return r0;
            if (mapping[r0] != -1) return mapping[r0];
            stackR.clear();
            stackR.push_back(r0);
            while (!stackR.empty()) {
                int r = stackR.back();
                if (mapping[r] != -1) {
                    stackR.pop_back();
                    continue;
                }
                int a = litOf(r, 0) / 2, b = litOf(r, 1) / 2;
                if (a > nn && mapping[a] == -1) {
                    stackR.push_back(a);
                    continue;
                }
                if (b > nn && mapping[b] == -1) {
                    stackR.push_back(b);
                    continue;
                }
                int ma = a > nn ? mapping[a] : a, mb = b > nn ? mapping[b] : b;
                n++;
                ensure((size_t)n + 2);
                fanin0[n] = ma * 2 + (litOf(r, 0) & 1);
                fanin1[n] = mb * 2 + (litOf(r, 1) & 1);
                mapping[r] = n;
                stackR.pop_back();
            }
            return mapping[r0];
        };
        for (int id = 1; id <= nn; id++) {
            if (replace[id] == -1) continue;
            replace[id] = rebuild(replace[id] / 2) * 2 + (replace[id] & 1);
        }
        dN1 = n;
        dReplace = replace;
        dNewF0.assign(fanin0.begin() + nn + 1, fanin0.begin() + n + 1);
        dNewF1.assign(fanin1.begin() + nn + 1, fanin1.begin() + n + 1);

        // choice loop, rewrite.cu:830-893
        for (int i = nn + 1; i <= n; i++) {
            isDeleted[i] = 1;
            ref[i] = 0;
        }
        dChoice.assign(nn + 1, kNotVisited);
        for (int i = numInputs + 1; i <= nn; i++) {
            Cut cut = selected[i];
            int newIdx = replace[i] >> 1;
            if (cut.used == 0) {
                st.preEval++;
                dChoice[i] = kNoCut;
                continue;
            }
            if (cut.nLeaves < 3) {
                st.smallCut++;
                dChoice[i] = kSmallCut;
                continue;
            }
            if (newIdx == -1) {
                st.newIdx++;
                dChoice[i] = kNoReplace;
                continue;
            }
            if (newIdx == i || lid(fanin1[newIdx]) == i) {
                dChoice[i] = kSelfRef;
                continue;
            }
            if (cut.nLeaves == 3) cut.leaves[cut.nLeaves++] = 0;
            bool compromised = false;
            for (uint32_t j = 0; j < cut.nLeaves; j++)
                if (isDeleted[cut.leaves[j]]) compromised = true;
            if (compromised) {
                st.compromised++;
                dChoice[i] = kCompromised;
                continue;
            }
            int added = install(newIdx);
            ref[newIdx]++;
            int saved = fastDelete(i);
            ref[newIdx]--;
            if (saved - added > 0 || (saved == added && fUseZeros)) {
                st.replaced++;
                if (saved - added > 0)
                    st.replacedPos++;
                else
                    st.replacedZero++;
                st.expected += saved - added;
                isDeleted[i] = 0;
                fanin0[i] = 1;
                fanin1[i] = replace[i];
                ref[0]++;
                ref[newIdx]++;
                dChoice[i] = kCommitted;
            } else {
                st.reverted++;
                install(i);
                ref[i]++;
                if (ref[newIdx] == 0) fastDelete(newIdx);
                ref[i]--;
                dChoice[i] = kReverted;
            }
        }
        // redundancy removal, rewrite.cu:911-921
        for (int i = numInputs + 1; i <= n; i++) {
            if (isDeleted[i]) continue;
            if (!isRedundant(i)) {
                fanin0[i] = Fanin(fanin0[i]);
                fanin1[i] = Fanin(fanin1[i]);
            } else {
                isDeleted[i] = 1;
            }
        }
        for (int i = 0; i < numOutputs; i++) output[i] = Fanin(output[i]);
        reorder();
    }
};

// ----------------------------------------------------------------- strash
// GPU strash + dangling removal, src/aig/strash.cu:190-314, with the
// deterministic duplicate rule described at the top of this file.
static Graph strash_gpu(const Graph &g) {
    int nPIs = g.nPIs, nObjs = g.nObjs;
    // dangling = AND nodes outside the transitive fanin of the POs; this is
    // the fix-point of markDanglingNodesIter (strash.cu:175-188,223-229)
    std::vector<char> live(nObjs, 0);
    std::vector<int> stk;
    for (int i = 0; i <= nPIs; i++) live[i] = 1;
    for (int o : g.outs) {
        int v = lid(o);
        if (!live[v]) {
            live[v] = 1;
            stk.push_back(v);
        }
    }
    while (!stk.empty()) {
        int v = stk.back();
        stk.pop_back();
        for (int lit : {g.f0[v], g.f1[v]}) {
            int u = lid(lit);
            if (!live[u]) {
                live[u] = 1;
                stk.push_back(u);
            }
        }
    }
    // frontier round of each remaining node = ASAP level in the remaining
    // graph; frontiers list nodes in ascending old id (strash.cu:247-277)
    std::vector<int> rnd(nObjs, 0);
    int maxRound = 0;
    std::vector<int> remain;
    for (int v = nPIs + 1; v < nObjs; v++)
        if (live[v]) remain.push_back(v);
    // inputs are topologically ordered by id (AIGER and every stage here)
    for (int v : remain) {
        rnd[v] = 1 + std::max(rnd[lid(g.f0[v])], rnd[lid(g.f1[v])]);
        maxRound = std::max(maxRound, rnd[v]);
    }
    std::vector<int> byRound(remain);
    std::stable_sort(byRound.begin(), byRound.end(), [&](int a, int b) { return rnd[a] < rnd[b]; });
    std::vector<int> map(nObjs, -1);
    for (int i = 0; i <= nPIs; i++) map[i] = 2 * i;
    std::unordered_map<uint64_t, int> table;
    table.reserve(remain.size() * 2 + 16);
    std::vector<int> winnerKey0, winnerKey1;  // tentative lits, in tentative-id order
    std::vector<int> winnerTent;
    int tent = nPIs + 1;
    for (int v : byRound) {
        int t = tent++;
        int l0 = map[lid(g.f0[v])] ^ lc(g.f0[v]);
        int l1 = map[lid(g.f1[v])] ^ lc(g.f1[v]);
        if (l0 > l1) std::swap(l0, l1);
        // checkTrivialAndCases, src/hash_table/hash_table.h:435-449
        int triv = -1;
        if (l0 == l1)
            triv = l0;
        else if (l0 == (l1 ^ 1))
            triv = 1;
        else if (l0 == 0)
            triv = l1;
        else if (l1 == 0)
            triv = l0;
        else if (l0 == 1 || l1 == 1)
            triv = 1;
        if (triv != -1) {
            map[v] = triv;
            continue;
        }
        uint64_t k = ((uint64_t)(uint32_t)l0 << 32) | (uint32_t)l1;
        auto it = table.find(k);
        if (it != table.end()) {
            map[v] = 2 * it->second;
        } else {
            table.emplace(k, t);
            map[v] = 2 * t;
            winnerKey0.push_back(l0);
            winnerKey1.push_back(l1);
            winnerTent.push_back(t);
        }
    }
    // consecutive renumbering (assignOld2NewConsecutiveIds / unbindKeysReId /
    // poReId, strash.cu:113-160)
    std::unordered_map<int, int> t2n;
    t2n.reserve(winnerTent.size() * 2 + 16);
    for (size_t r = 0; r < winnerTent.size(); r++) t2n[winnerTent[r]] = nPIs + 1 + (int)r;
    auto remap = [&](int lit) {
        int v = lid(lit);
        if (v <= nPIs) return lit;
        return 2 * t2n.at(v) + lc(lit);
    };
    Graph o;
    o.nPIs = nPIs;
    o.nPOs = g.nPOs;
    o.nObjs = nPIs + 1 + (int)winnerTent.size();
    o.f0.assign(o.nObjs, -1);
    o.f1.assign(o.nObjs, -1);
    for (size_t r = 0; r < winnerTent.size(); r++) {
        o.f0[nPIs + 1 + r] = remap(winnerKey0[r]);
        o.f1[nPIs + 1 + r] = remap(winnerKey1[r]);
    }
    o.outs.resize(g.nPOs);
    for (int i = 0; i < g.nPOs; i++) {
        int lit = map[lid(g.outs[i])] ^ lc(g.outs[i]);
        o.outs[i] = remap(lit);
    }
    o.nLevels = maxRound;
    return o;
}

// CPU strash (`st -c`), src/aig/strash.cu:322-466: dangling nodes removed,
// one pass in id order, no trivial-case folding, level = true depth.
static Graph strash_cpu(const Graph &g) {
    int nPIs = g.nPIs, nObjs = g.nObjs;
    std::vector<int> fo(nObjs, 0);
    for (int v = nPIs + 1; v < nObjs; v++) {
        fo[lid(g.f0[v])]++;
        fo[lid(g.f1[v])]++;
    }
    for (int o : g.outs) fo[lid(o)]++;
    std::vector<char> dead(nObjs, 0);
    std::vector<int> stk;
    for (int v = nPIs + 1; v < nObjs; v++) {
        if (fo[v] != 0 || dead[v]) continue;
        stk.push_back(v);
        while (!stk.empty()) {
            int u = stk.back();
            stk.pop_back();
            if (u <= nPIs || dead[u]) continue;
            dead[u] = 1;
            int a = lid(g.f0[u]), b = lid(g.f1[u]);
            if (--fo[a] == 0) stk.push_back(a);
            if (--fo[b] == 0) stk.push_back(b);
        }
    }
    std::vector<int> o2n(nObjs, -1), delay(nObjs, -1);
    for (int i = 0; i <= nPIs; i++) {
        o2n[i] = i;
        delay[i] = 0;
    }
    std::unordered_map<uint64_t, int> table;
    Graph o;
    o.nPIs = nPIs;
    o.nPOs = g.nPOs;
    o.f0.assign(nObjs, -1);
    o.f1.assign(nObjs, -1);
    int idc = nPIs + 1, maxDelay = -1;
    for (int v = nPIs + 1; v < nObjs; v++) {
        if (dead[v]) continue;
        int l0 = 2 * o2n[lid(g.f0[v])] + lc(g.f0[v]);
        int l1 = 2 * o2n[lid(g.f1[v])] + lc(g.f1[v]);
        if (l0 > l1) std::swap(l0, l1);
        uint64_t k = ((uint64_t)(uint32_t)l0 << 32) | (uint32_t)l1;
        auto it = table.find(k);
        if (it == table.end()) {
            table.emplace(k, idc);
            o2n[v] = idc;
            o.f0[idc] = l0;
            o.f1[idc] = l1;
            delay[idc] = 1 + std::max(delay[lid(l0)], delay[lid(l1)]);
            maxDelay = std::max(maxDelay, delay[idc]);
            idc++;
        } else {
            o2n[v] = it->second;
        }
    }
    o.nObjs = idc;
    o.f0.resize(idc);
    o.f1.resize(idc);
    o.outs.resize(g.nPOs);
    for (int i = 0; i < g.nPOs; i++) o.outs[i] = 2 * o2n[lid(g.outs[i])] + lc(g.outs[i]);
    o.nLevels = maxDelay;
    return o;
}

// CPU deduplicate of the rw result, src/aig_manager.cu:454-522 (no dangling
// removal, no trivial folding); level taken from the rewrite's Reorder.
static Graph dedup_cpu(const Graph &g) {
    int nPIs = g.nPIs, nObjs = g.nObjs;
    std::vector<int> o2n(nObjs, -1);
    for (int i = 0; i <= nPIs; i++) o2n[i] = i;
    std::unordered_map<uint64_t, int> table;
    Graph o;
    o.nPIs = nPIs;
    o.nPOs = g.nPOs;
    o.f0.assign(nObjs, -1);
    o.f1.assign(nObjs, -1);
    int idc = nPIs + 1;
    for (int v = nPIs + 1; v < nObjs; v++) {
        int l0 = 2 * o2n[lid(g.f0[v])] + lc(g.f0[v]);
        int l1 = 2 * o2n[lid(g.f1[v])] + lc(g.f1[v]);
        if (l0 > l1) std::swap(l0, l1);
        uint64_t k = ((uint64_t)(uint32_t)l0 << 32) | (uint32_t)l1;
        auto it = table.find(k);
        if (it == table.end()) {
            table.emplace(k, idc);
            o2n[v] = idc;
            o.f0[idc] = l0;
            o.f1[idc] = l1;
            idc++;
        } else {
            o2n[v] = it->second;
        }
    }
    o.nObjs = idc;
    o.f0.resize(idc);
    o.f1.resize(idc);
    o.outs.resize(g.nPOs);
    for (int i = 0; i < g.nPOs; i++) o.outs[i] = 2 * o2n[lid(g.outs[i])] + lc(g.outs[i]);
    o.nLevels = g.nLevels;
    return o;
}

// ---------------------------------------------------------------- balance
// AIG balancing `b` (src/algorithms/balance.cu:912-1382, called by
// AIGMan::balance, src/aig_manager.cu:682-737), sortDecId = 1 (the `b`
// default: inputs sorted by decreasing level, then decreasing literal).
// Sequential restatement of the reference's two phases:
//  1. cover finding, level by level from the POs (balance.cu:970-1039):
//     the next level is every AND input of the covers of this level, in
//     increasing id order; a node's cover is its supergate, collected by the
//     DFS of localCoverTravToTable (balance.cu:666-751), and its "last
//     appear level" the last level it is listed on;
//  2. reconstruction, deepest covers first (balance.cu:1175-1283): covers of
//     one level in increasing node id, in chunks of 32,768; all covers of a
//     chunk pair their two lowest inputs in lockstep steps against one table
//     of built nodes (existing pairs are reused, new ones get id counter +
//     cover index, the smallest id of a key wins), and finally nodes are
//     renumbered in id order (balance.cu:1285-1318).
// The reference is deterministic here: duplicate keys inside a step resolve
// by atomicMin and every other step is order independent.
static const int kBalMaxCover = 1024;   // MAX_LOCAL_COVER_SIZE
static const int kBalStack = 128;       // DFS_COVER_STACK_SIZE
static const int kBalChunk = 32768;     // iterLen
static const unsigned kBalEmpty = 0xFFFFFFFFu;

// checkTrivialAndCases + TableLookup of the reconstruction
// (src/hash_table/hash_table.h:435-449, balance.cu:85-110): literal of the
// AND of lit1 and lit2 if it is trivial or already built, else kBalEmpty.
static unsigned bal_lookup(int l1, int l2, const std::unordered_map<uint64_t, unsigned> &tab) {
    if (l1 == l2) return (unsigned)l1;
    if (l1 == (l2 ^ 1)) return 1u;  // AigConst0 (AIGMan literal 1 = FALSE)
    if (l1 == 0) return (unsigned)l2;  // AigConst1
    if (l2 == 0) return (unsigned)l1;
    if (l1 == 1 || l2 == 1) return 1u;
    if (l1 > l2) std::swap(l1, l2);
    auto it = tab.find(((uint64_t)(uint32_t)l1 << 32) | (uint32_t)l2);
    return it == tab.end() ? kBalEmpty : it->second << 1;
}

static Graph balance_core(const Graph &g, std::string *err) {
    const int nPIs = g.nPIs, nObjs = g.nObjs, nPOs = g.nPOs;
    Graph r;
    r.nPIs = nPIs;
    r.nPOs = nPOs;
    std::vector<int> nfo(nObjs, 0);  // fanouts incl. PO references (aig_manager.cu:203-221)
    for (int v = nPIs + 1; v < nObjs; v++) {
        nfo[lid(g.f0[v])]++;
        nfo[lid(g.f1[v])]++;
    }
    for (int o : g.outs) nfo[lid(o)]++;
    // ---- phase 1: covers
    std::vector<int> covLen(nObjs, -1), lastLevel(nObjs, -1);
    std::vector<std::vector<int>> cover(nObjs);
    std::vector<int> list;
    {
        std::vector<char> seen(nObjs, 0);
        for (int o : g.outs) {  // checkCoverTravEnd: AND drivers, first occurrence
            int v = lid(o);
            if (v > nPIs && !seen[v]) {
                seen[v] = 1;
                list.push_back(v);
            }
        }
    }
    if (list.empty()) {  // no AND node drives a PO: no AND node is kept
        r.nObjs = nPIs + 1;
        r.f0.assign(r.nObjs, -1);
        r.f1.assign(r.nObjs, -1);
        r.outs = g.outs;
        return r;
    }
    int levelCount = 0;
    std::vector<char> status(nObjs);
    while (!list.empty()) {
        std::fill(status.begin(), status.end(), 0);
        for (int v : list) {
            lastLevel[v] = levelCount;
            if (covLen[v] < 0) {
                // localCoverTravToTable (balance.cu:666-751)
                std::vector<int> &cv = cover[v];
                int stk[kBalStack];
                int top = -1;
                stk[++top] = 2 * v;
                bool constFalse = false;
                while (top >= 0) {
                    const int cur = stk[top--];
                    bool same = false;
                    for (int x : cv) {
                        if (x == cur) {
                            same = true;
                            break;
                        }
                        if (x == (cur ^ 1)) {
                            constFalse = true;
                            break;
                        }
                    }
                    if (constFalse) break;
                    if (same) continue;
                    const int id = lid(cur);
                    if (cur != 2 * v && ((cur & 1) || id <= nPIs || nfo[id] > 1 || top + 2 >= kBalStack ||
                                         (int)cv.size() + 2 * (top + 1) + 1 >= kBalMaxCover)) {
                        cv.push_back(cur);
                        continue;
                    }
                    stk[++top] = g.f1[id];
                    stk[++top] = g.f0[id];
                }
                if (constFalse) cv.clear();
                covLen[v] = (int)cv.size();
            }
            if (covLen[v] == 0) continue;  // constant false: inputs not followed
            for (int x : cover[v])
                if (lid(x) > nPIs) status[lid(x)] = 1;
        }
        list.clear();
        for (int v = 0; v < nObjs; v++)
            if (status[v]) list.push_back(v);
        levelCount++;
    }
    // ---- phase 2: reconstruction
    std::vector<int> covers;  // cover roots by (last level, id)
    for (int v = 0; v < nObjs; v++)
        if (covLen[v] >= 0) covers.push_back(v);
    std::stable_sort(covers.begin(), covers.end(), [&](int a, int b) { return lastLevel[a] < lastLevel[b]; });
    std::vector<int> newLit(nObjs, -1);  // per cover root: its reconstructed literal
    std::unordered_map<uint64_t, unsigned> tab;  // key (lit0 < lit1) -> new id
    std::unordered_map<unsigned, unsigned> lev;  // new id -> level
    auto level_of = [&](int lit) -> int {
        const unsigned id = (unsigned)lid(lit);
        if ((int)id <= nPIs) return 0;
        auto it = lev.find(id);
        if (it == lev.end()) {
            if (err) *err = "balance: level of a built node missing";
            return 0;
        }
        return (int)it->second;
    };
    long long newIdCounter = nPIs + 1;
    std::vector<size_t> lvEnd(levelCount + 1, 0);  // covers of level L: [lvEnd[L-1], lvEnd[L])
    for (int v : covers) lvEnd[lastLevel[v]]++;
    for (int L = 1; L < levelCount; L++) lvEnd[L] += lvEnd[L - 1];
    for (int L = levelCount - 1; L >= 0; L--) {
        const size_t pos = L ? lvEnd[L - 1] : 0, end = lvEnd[L];
        for (size_t c0 = pos; c0 < end; c0 += kBalChunk) {
            const int n = (int)std::min<size_t>(kBalChunk, end - c0);
            // prepareReconstructArrays (balance.cu:272-426), sortDecId = 1
            std::vector<std::vector<std::pair<int, int>>> arr(n);  // (literal, level)
            for (int i = 0; i < n; i++) {
                const int v = covers[c0 + i];
                for (int x : cover[v]) {
                    int nl;
                    if (lid(x) <= nPIs)
                        nl = x;
                    else
                        nl = newLit[lid(x)] ^ (x & 1);
                    arr[i].push_back({nl, level_of(nl)});
                }
                std::sort(arr[i].begin(), arr[i].end(), [](const std::pair<int, int> &a, const std::pair<int, int> &b) {
                    return a.second == b.second ? a.first > b.first : a.second > b.second;
                });
            }
            // steps (balance.cu:1207-1262)
            std::vector<int> mask(n);
            std::vector<uint64_t> keys(n);
            std::vector<unsigned> vals(n), lvls(n);
            while (true) {
                int maxMask = 0;
                for (int i = 0; i < n; i++) {
                    auto &a = arr[i];
                    const int len = (int)a.size();
                    mask[i] = 0;
                    if (len <= 1) continue;
                    // sharedNodeDrivenPermute (balance.cu:187-247)
                    int left = 0;
                    if (len >= 3) {
                        left = len - 2;
                        const int border = a[left].second;
                        for (left--; left >= 0 && a[left].second == border; left--) {
                        }
                        left++;
                    }
                    const int right = len - 2;
                    if (left < right) {
                        const int l1 = a[right + 1].first, l2 = a[right].first;
                        for (int k = right; k >= left; k--) {
                            const int l3 = a[k].first;
                            if (bal_lookup(l1, l3, tab) != kBalEmpty) {
                                if (l3 != l2) std::swap(a[k], a[right]);
                                break;
                            }
                        }
                    }
                    // prepareDataToInsert (balance.cu:113-184)
                    int l1 = a[len - 1].first, l2 = a[len - 2].first;
                    const int lv1 = a[len - 1].second, lv2 = a[len - 2].second;
                    a.resize(len - 2);
                    const unsigned got = bal_lookup(l1, l2, tab);
                    if (got != kBalEmpty) {
                        mask[i] = 2;
                        vals[i] = got;
                        lvls[i] = (unsigned)level_of((int)got);
                    } else {
                        if (l1 > l2) std::swap(l1, l2);
                        mask[i] = 1;
                        keys[i] = ((uint64_t)(uint32_t)l1 << 32) | (uint32_t)l2;
                        vals[i] = (unsigned)(newIdCounter + i);
                        lvls[i] = (unsigned)std::max(lv1, lv2) + 1;
                    }
                    maxMask = std::max(maxMask, mask[i]);
                }
                if (maxMask == 0) break;
                // insert_batch_update_min_masked + retrieve_batch_masked
                for (int i = 0; i < n; i++)
                    if (mask[i] == 1) {
                        auto it = tab.find(keys[i]);
                        if (it == tab.end())
                            tab[keys[i]] = vals[i];
                        else
                            it->second = std::min(it->second, vals[i]);
                    }
                unsigned maxId = 0;
                for (int i = 0; i < n; i++)
                    if (mask[i] == 1) {
                        vals[i] = tab[keys[i]];
                        maxId = std::max(maxId, vals[i]);
                    }
                if (maxId != 0) newIdCounter = (long long)maxId + 1;
                for (int i = 0; i < n; i++)
                    if (mask[i] == 1) {
                        auto it = lev.find(vals[i]);
                        if (it == lev.end())
                            lev[vals[i]] = lvls[i];
                        else
                            it->second = std::min(it->second, lvls[i]);
                    }
                // addBackLocalArrays (balance.cu:429-467)
                for (int i = 0; i < n; i++) {
                    if (mask[i] == 0) continue;
                    const int lit = mask[i] == 2 ? (int)vals[i] : (int)(vals[i] << 1);
                    auto &a = arr[i];
                    bool dup = false;
                    for (auto &e : a)
                        if (e.first == lit) {
                            dup = true;
                            break;
                        }
                    if (dup) continue;
                    a.push_back({lit, (int)lvls[i]});
                    for (int k = (int)a.size() - 1; k > 0 && a[k].second > a[k - 1].second; k--) std::swap(a[k], a[k - 1]);
                }
            }
            // recordReconstructedCovers (balance.cu:469-491)
            for (int i = 0; i < n; i++) {
                const int v = covers[c0 + i];
                newLit[v] = arr[i].empty() ? 1 : arr[i][0].first;
            }
        }
    }
    // renumbering in id order (balance.cu:1285-1318)
    std::vector<std::pair<unsigned, uint64_t>> built;
    built.reserve(tab.size());
    for (auto &kv : tab) built.push_back({kv.second, kv.first});
    std::sort(built.begin(), built.end());
    std::unordered_map<unsigned, int> outId;
    for (size_t k = 0; k < built.size(); k++) outId[built[k].first] = nPIs + 1 + (int)k;
    auto map_lit = [&](unsigned lit) -> int {
        const unsigned id = lit >> 1;
        if ((int)id <= nPIs) return (int)lit;
        return 2 * outId[id] + (int)(lit & 1);
    };
    r.nObjs = nPIs + 1 + (int)built.size();
    r.f0.assign(r.nObjs, -1);
    r.f1.assign(r.nObjs, -1);
    for (size_t k = 0; k < built.size(); k++) {
        const uint64_t key = built[k].second;
        r.f0[nPIs + 1 + k] = map_lit((unsigned)(key >> 32));
        r.f1[nPIs + 1 + k] = map_lit((unsigned)(key & 0xFFFFFFFFu));
    }
    // processPO (balance.cu:882-910)
    r.outs.resize(nPOs);
    for (int i = 0; i < nPOs; i++) {
        const int o = g.outs[i];
        if (lid(o) <= nPIs) {
            r.outs[i] = o;
            continue;
        }
        const int nl = newLit[lid(o)];
        r.outs[i] = map_lit((unsigned)nl) ^ (o & 1);
    }
    r.nLevels = -1;  // the balance does not compute levels (aig_manager.cu:727)
    return r;
}

struct Oracle {
    Lib lib;
    Graph g;
    Solver s;
    Graph preDedup;
    // AIGMan::prevCmdRewrite (src/aig_manager.h:97): the solver still holds
    // the last rewrite's graph, so the next rewrite starts from it instead
    // of resetting from g.  Set by every rewrite (aig_manager.cu:662) and
    // cleared by a strash (src/aig/strash.cu:498) -- the GPU deduplication
    // of a rewrite is one -- and by reading a graph (aig_manager.cu:101).
    bool keepRw = false;
    std::string err;
};

}  // namespace orc

using orc::Oracle;

extern "C" {

void *orc_create(const char *libpath) {
    Oracle *o = new Oracle();
    if (!orc::load_lib(libpath, o->lib)) {
        delete o;
        return nullptr;
    }
    o->s.lib = &o->lib;
    return o;
}

void orc_destroy(void *h) { delete (Oracle *)h; }

// Graph in AIGMan convention: arrays of nObjs = 1 + nPIs + nAnds entries
// (entries 0..nPIs ignored), literal 0 = constant TRUE.
int orc_set_graph(void *h, int nPIs, int nPOs, int nAnds, const int *f0, const int *f1, const int *outs) {
    Oracle *o = (Oracle *)h;
    orc::Graph &g = o->g;
    o->keepRw = false;
    g.nPIs = nPIs;
    g.nPOs = nPOs;
    g.nObjs = 1 + nPIs + nAnds;
    g.f0.assign(g.nObjs, -1);
    g.f1.assign(g.nObjs, -1);
    for (int i = nPIs + 1; i < g.nObjs; i++) {
        g.f0[i] = f0[i];
        g.f1[i] = f1[i];
        if (f0[i] < 0 || f1[i] < 0 || (f0[i] >> 1) >= i || (f1[i] >> 1) >= i) return -1;
    }
    g.outs.assign(outs, outs + nPOs);
    for (int i = 0; i < nPOs; i++)
        if (outs[i] < 0 || (outs[i] >> 1) >= g.nObjs) return -1;
    // level of the input as AIGMan::readFromMemory computes it
    std::vector<int> d(g.nObjs, 0);
    int mx = 0;
    for (int i = nPIs + 1; i < g.nObjs; i++) {
        d[i] = 1 + std::max(d[g.f0[i] >> 1], d[g.f1[i] >> 1]);
        mx = std::max(mx, d[i]);
    }
    g.nLevels = nAnds > 0 ? mx : 0;
    return 0;
}

// AIGMan::rewrite(fUseZeros, fGPUDeduplicate) (src/aig_manager.cu:632-672);
// dedupMode 2 = GPU deduplicate (strash), 1 = CPU deduplicate, 0 = none.
int orc_rw(void *h, int fUseZeros, int dedupMode) {
    Oracle *o = (Oracle *)h;
    orc::Graph &g = o->g;
    if (g.nObjs - 1 - g.nPIs == 0) return 0;  // rewrite: nothing to do
    orc::Solver &s = o->s;
    if (!o->keepRw) s.reset(g);  // src/aig_manager.cu:654-655
    s.rewrite(fUseZeros != 0);
    // updateFromRewriteManager, src/aig_manager.cu:432-564
    orc::Graph r;
    r.nPIs = s.numInputs;
    r.nPOs = s.numOutputs;
    r.nObjs = s.n + 1;
    r.nLevels = s.nLevels;
    r.f0.assign(r.nObjs, -1);
    r.f1.assign(r.nObjs, -1);
    for (int i = r.nPIs + 1; i < r.nObjs; i++) {
        r.f0[i] = orc::invConst(s.fanin0[i]);
        r.f1[i] = orc::invConst(s.fanin1[i]);
    }
    r.outs.resize(r.nPOs);
    for (int i = 0; i < r.nPOs; i++) r.outs[i] = orc::invConst(s.output[i]);
    o->preDedup = r;
    if (dedupMode == 2)
        g = orc::strash_gpu(r);
    else if (dedupMode == 1)
        g = orc::dedup_cpu(r);
    else
        g = r;
    o->keepRw = dedupMode != 2;
    return 0;
}

// AIGMan::strash(fCPU) (src/aig/strash.cu:317-503)
int orc_st(void *h, int fCPU) {
    Oracle *o = (Oracle *)h;
    o->g = fCPU ? orc::strash_cpu(o->g) : orc::strash_gpu(o->g);
    o->keepRw = false;
    return 0;
}

// AIGMan::balance(sortDecId = 1, updateLevel) (src/aig_manager.cu:682-737):
// balance, then a GPU strash when updateLevel (the `b` command).  Returns
// -1 when the restatement met an inconsistency.
int orc_b(void *h, int updateLevel) {
    Oracle *o = (Oracle *)h;
    if (o->g.nObjs - 1 - o->g.nPIs == 0) return 0;
    std::string err;
    orc::Graph r = orc::balance_core(o->g, &err);
    if (!err.empty()) {
        o->err = err;
        return -1;
    }
    o->g = updateLevel ? orc::strash_gpu(r) : r;
    o->keepRw = false;
    return 0;
}

int orc_get_sizes(void *h, int *nPIs, int *nPOs, int *nAnds, int *nLevels) {
    Oracle *o = (Oracle *)h;
    *nPIs = o->g.nPIs;
    *nPOs = o->g.nPOs;
    *nAnds = o->g.nObjs - 1 - o->g.nPIs;
    *nLevels = o->g.nLevels;
    return 0;
}

int orc_get_graph(void *h, int *f0, int *f1, int *outs) {
    Oracle *o = (Oracle *)h;
    for (int i = 0; i < o->g.nObjs; i++) {
        f0[i] = o->g.f0[i];
        f1[i] = o->g.f1[i];
    }
    for (int i = 0; i < o->g.nPOs; i++) outs[i] = o->g.outs[i];
    return 0;
}

// Sizes of the dumps of the last rw: n (objects after Reset, ids 0..n) and
// the object count after the DFS rebuild of new nodes.
int orc_dump_sizes(void *h, int *n0, int *n1) {
    Oracle *o = (Oracle *)h;
    *n0 = o->s.dN0;
    *n1 = o->s.dN1;
    return 0;
}

// Fanin literals (AIGER convention, lit 0 = FALSE) after Reset/Reorder, ids 0..n.
int orc_dump_reorder(void *h, int *f0, int *f1, int *outs) {
    Oracle *o = (Oracle *)h;
    int n = o->s.dN0;
    for (int i = 0; i <= n; i++) {
        f0[i] = o->s.dReorderF0[i];
        f1[i] = o->s.dReorderF1[i];
    }
    for (size_t i = 0; i < o->s.dReorderOut.size(); i++) outs[i] = o->s.dReorderOut[i];
    return 0;
}

static void put_cut(const orc::Cut &c, int *q) {
    // canonical record: used, nLeaves, leaves[4] (0 past nLeaves), tt, sign, value
    if (!c.used) {
        for (int k = 0; k < 9; k++) q[k] = 0;
        return;
    }
    q[0] = 1;
    q[1] = (int)c.nLeaves;
    for (int k = 0; k < 4; k++) q[2 + k] = k < (int)c.nLeaves ? c.leaves[k] : 0;
    q[6] = (int)c.tt;
    q[7] = (int)c.sign;
    q[8] = (int)c.value;
}

// All 8 cut slots per node, 9 ints per slot, ids 0..n.
int orc_dump_cuts(void *h, int *out) {
    Oracle *o = (Oracle *)h;
    size_t m = (size_t)(o->s.dN0 + 1) * 8;
    for (size_t i = 0; i < m; i++) put_cut(o->s.dCuts[i], out + i * 9);
    return 0;
}

// Selected cut per node (9 ints) followed by the chosen root index (-1 if none).
int orc_dump_selected(void *h, int *out) {
    Oracle *o = (Oracle *)h;
    for (int i = 0; i <= o->s.dN0; i++) {
        put_cut(o->s.dSelected[i], out + (size_t)i * 10);
        out[(size_t)i * 10 + 9] = o->s.dSelected[i].used ? o->s.dBestOut[i] : -1;
    }
    return 0;
}

// replace[] after the DFS rebuild (ids 0..n) and the rebuilt new nodes'
// fanin literals (AIGER convention), ids n+1..n1.
int orc_dump_replace(void *h, int *replace, int *newF0, int *newF1) {
    Oracle *o = (Oracle *)h;
    for (int i = 0; i <= o->s.dN0; i++) replace[i] = o->s.dReplace[i];
    for (size_t i = 0; i < o->s.dNewF0.size(); i++) {
        newF0[i] = o->s.dNewF0[i];
        newF1[i] = o->s.dNewF1[i];
    }
    return 0;
}

// Outcome of the sequential choice loop per node id 0..n (orc::ChoiceCode).
int orc_dump_choice(void *h, int *codes) {
    Oracle *o = (Oracle *)h;
    for (int i = 0; i <= o->s.dN0; i++) codes[i] = o->s.dChoice[i];
    return 0;
}

// replaced, replacedPos, replacedZero, reverted, compromised, preEval,
// smallCut, newIdx, expected (real reduction), new nodes created.
int orc_dump_stats(void *h, long long *out) {
    Oracle *o = (Oracle *)h;
    const orc::Stats &s = o->s.st;
    long long v[10] = {s.replaced, s.replacedPos, s.replacedZero, s.reverted, s.compromised,
                       s.preEval,  s.smallCut,    s.newIdx,       s.expected, s.nNewNodes};
    for (int i = 0; i < 10; i++) out[i] = v[i];
    return 0;
}

// The rewritten AIG before deduplication (AIGMan convention) and its sizes.
int orc_prededup_sizes(void *h, int *nObjs, int *nLevels) {
    Oracle *o = (Oracle *)h;
    *nObjs = o->preDedup.nObjs;
    *nLevels = o->preDedup.nLevels;
    return 0;
}
int orc_prededup_graph(void *h, int *f0, int *f1, int *outs) {
    Oracle *o = (Oracle *)h;
    for (int i = 0; i < o->preDedup.nObjs; i++) {
        f0[i] = o->preDedup.f0[i];
        f1[i] = o->preDedup.f1[i];
    }
    for (int i = 0; i < o->preDedup.nPOs; i++) outs[i] = o->preDedup.outs[i];
    return 0;
}

}  // extern "C"

// Bit-parallel simulation of an AIG (AIGMan layout) on `words` 64-bit random
// patterns per PI drawn from splitmix64(seed, pi, word); writes nPOs * words
// output words.  Used to check functional equivalence of large results.
extern "C" int orc_simulate(int nPIs, int nPOs, int nAnds, const int *f0, const int *f1, const int *outs, int words,
                            unsigned long long seed, unsigned long long *out) {
    const int n = 1 + nPIs + nAnds;
    std::vector<unsigned long long> val((size_t)n * words);
    auto mix = [](unsigned long long x) {
        x += 0x9E3779B97F4A7C15ull;
        x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
        x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
        return x ^ (x >> 31);
    };
    for (int w = 0; w < words; w++) val[w] = ~0ull;
    for (int i = 1; i <= nPIs; i++)
        for (int w = 0; w < words; w++) val[(size_t)i * words + w] = mix(seed ^ mix((unsigned long long)i * 1000003ull + w));
    for (int v = nPIs + 1; v < n; v++) {
        int a = f0[v], b = f1[v];
        if ((a >> 1) >= v || (b >> 1) >= v || a < 0 || b < 0) return -1;
        const unsigned long long ca = (a & 1) ? ~0ull : 0ull, cb = (b & 1) ? ~0ull : 0ull;
        const unsigned long long *pa = &val[(size_t)(a >> 1) * words], *pb = &val[(size_t)(b >> 1) * words];
        unsigned long long *pv = &val[(size_t)v * words];
        for (int w = 0; w < words; w++) pv[w] = (pa[w] ^ ca) & (pb[w] ^ cb);
    }
    for (int k = 0; k < nPOs; k++) {
        int o = outs[k];
        const unsigned long long c = (o & 1) ? ~0ull : 0ull;
        for (int w = 0; w < words; w++) out[(size_t)k * words + w] = val[(size_t)(o >> 1) * words + w] ^ c;
    }
    return 0;
}
