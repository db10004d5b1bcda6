// Seeded synthetic AIG generators for the rw;st workloads.
//
// The generators emit AIGs in the AIGMan layout (src/aig_manager.h:51-58 of
// CULS): objects 0..nObjs-1, object 0 the constant, PIs 1..nPIs, AND nodes
// after them in topological order, literal 2*id+complement with literal 0 =
// constant TRUE.  Every generated AIG is strashed: no two AND nodes share a
// fanin pair, no AND has both fanins on the same node, no constant fanins, and
// AND nodes outside the transitive fanin of the POs are removed (ids stay in
// generation order).  They have no counterpart in CULS, whose benchmark
// inputs are not shipped.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <climits>
#include <vector>

#include "culs_b200.h"
#include "guard.hpp"

namespace {

struct Rng {
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed) {}
    uint64_t next() {  // splitmix64
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    uint64_t below(uint64_t n) { return n ? next() % n : 0; }
    double unit() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
};

uint64_t splitmix(uint64_t x) {
    Rng r(x);
    return r.next();
}

struct Aig {
    int nPIs = 0;
    std::vector<int> f0, f1;  // indexed by object id; PIs/const hold -1
    std::vector<int> outs;
};

// Keep the transitive fanin of the POs, renumbering in id order.
void remove_dangling(Aig &g) {
    int nObjs = (int)g.f0.size();
    std::vector<char> live(nObjs, 0);
    for (int i = 0; i <= g.nPIs; i++) live[i] = 1;
    for (int o : g.outs) live[o >> 1] = 1;
    for (int v = nObjs - 1; v > g.nPIs; v--)
        if (live[v]) {
            live[g.f0[v] >> 1] = 1;
            live[g.f1[v] >> 1] = 1;
        }
    std::vector<int> map(nObjs, -1);
    int k = 0;
    for (int v = 0; v < nObjs; v++)
        if (live[v]) map[v] = k++;
    Aig o;
    o.nPIs = g.nPIs;
    o.f0.assign(k, -1);
    o.f1.assign(k, -1);
    for (int v = g.nPIs + 1; v < nObjs; v++)
        if (live[v]) {
            o.f0[map[v]] = 2 * map[g.f0[v] >> 1] + (g.f0[v] & 1);
            o.f1[map[v]] = 2 * map[g.f1[v] >> 1] + (g.f1[v] & 1);
        }
    for (int ol : g.outs) o.outs.push_back(2 * map[ol >> 1] + (ol & 1));
    g.f0.swap(o.f0);
    g.f1.swap(o.f1);
    g.outs.swap(o.outs);
}

// Layered random AIG.  Layer 0 holds the PIs; layer L (1..nLayers) holds its
// share of nAnds AND nodes.  A fanin is drawn, with probability 1-pFar,
// uniformly from the `window` previous layers (plus all PIs when withPIs), and
// otherwise uniformly from every earlier object except the constant.  Each
// fanin edge is complemented with probability 1/2.  POs are the first nPOs
// nodes of the last layer (all of it when it is narrower), or, with
// sinksArePOs, every AND node without fanouts (then no node dangles and the
// AIG keeps exactly nAnds AND nodes).  Returns false when a layer has more
// nodes than its window offers distinct fanin pairs (no strashed AIG has that
// shape).
bool layered(Aig &g, uint64_t seed, int nPIs, int nPOs, int64_t nAnds, int nLayers, int window, double pFar,
             bool withPIs, bool sinksArePOs = false) {
    Rng r(seed);
    g = Aig();
    g.nPIs = nPIs;
    int64_t nObjs = 1 + nPIs + nAnds;
    g.f0.assign(nObjs, -1);
    g.f1.assign(nObjs, -1);
    std::vector<int64_t> layerStart(nLayers + 2);
    layerStart[0] = 1;
    layerStart[1] = 1 + nPIs;
    for (int L = 1; L <= nLayers; L++) {
        int64_t w = nAnds / nLayers + (L <= nAnds % nLayers ? 1 : 0);
        layerStart[L + 1] = layerStart[L] + w;
    }
    std::unordered_set<uint64_t> seen;
    seen.reserve((size_t)nAnds * 2);
    int64_t id = 1 + nPIs;
    for (int L = 1; L <= nLayers; L++) {
        int lo = std::max(0, L - window);
        int64_t nearLo = layerStart[lo], nearHi = layerStart[L];  // [nearLo, nearHi)
        int64_t nearCnt = nearHi - nearLo;
        bool addPIs = withPIs && lo > 0;
        for (int64_t v = layerStart[L]; v < layerStart[L + 1]; v++, id++) {
            auto draw = [&]() -> int64_t {
                if (pFar > 0 && r.unit() < pFar) return 1 + (int64_t)r.below((uint64_t)(v - 1));
                int64_t span = nearCnt + (addPIs ? nPIs : 0);
                int64_t k = (int64_t)r.below((uint64_t)span);
                return k < nearCnt ? nearLo + k : 1 + (k - nearCnt);
            };
            int a = 0, b = 0;
            for (int tries = 0;; tries++) {
                int64_t x = draw(), y = draw();
                if (x == y) continue;
                a = (int)(2 * x + (r.next() & 1));
                b = (int)(2 * y + (r.next() & 1));
                if (a > b) std::swap(a, b);
                uint64_t key = ((uint64_t)(uint32_t)a << 32) | (uint32_t)b;
                if (seen.insert(key).second) break;
                if (tries > 1000) return false;  // the window's pairs are used up
            }
            g.f0[v] = a;
            g.f1[v] = b;
        }
    }
    if (sinksArePOs) {
        std::vector<char> hasFanout(nObjs, 0);
        for (int64_t v = 1 + nPIs; v < nObjs; v++) {
            hasFanout[g.f0[v] >> 1] = 1;
            hasFanout[g.f1[v] >> 1] = 1;
        }
        for (int64_t v = 1 + nPIs; v < nObjs; v++)
            if (!hasFanout[v]) g.outs.push_back((int)(2 * v));
    } else {
        int64_t lastLo = layerStart[nLayers], lastHi = layerStart[nLayers + 1];
        for (int64_t v = lastLo; v < lastHi && (int)g.outs.size() < nPOs; v++) g.outs.push_back((int)(2 * v));
    }
    remove_dangling(g);
    return true;
}

// Structural-hashing AIG builder used by the arithmetic generators.
struct Builder {
    Aig g;
    std::unordered_map<uint64_t, int> table;
    static const int T = 0, F = 1;  // AIGMan constants: literal 0 = TRUE
    explicit Builder(int nPIs) {
        g.nPIs = nPIs;
        g.f0.assign(1 + nPIs, -1);
        g.f1.assign(1 + nPIs, -1);
    }
    int pi(int i) const { return 2 * (1 + i); }
    int And(int a, int b) {
        if (a > b) std::swap(a, b);
        if (a == b) return a;
        if (a == (b ^ 1)) return F;
        if (a == T) return b;
        if (a == F) return F;
        uint64_t key = ((uint64_t)(uint32_t)a << 32) | (uint32_t)b;
        auto it = table.find(key);
        if (it != table.end()) return 2 * it->second;
        int id = (int)g.f0.size();
        g.f0.push_back(a);
        g.f1.push_back(b);
        table.emplace(key, id);
        return 2 * id;
    }
    int Or(int a, int b) { return And(a ^ 1, b ^ 1) ^ 1; }
    int Xor(int a, int b) { return And(And(a, b ^ 1) ^ 1, And(a ^ 1, b) ^ 1) ^ 1; }
};

// n x n unsigned array multiplier: AND partial products and ripple-carry rows
// of half/full adders (XOR as three ANDs).  PIs a0..a{n-1}, b0..b{n-1}; POs
// the 2n product bits, least significant first.
Aig multiplier(int n) {
    Builder B(2 * n);
    auto A = [&](int i) { return B.pi(i); };
    auto Bb = [&](int j) { return B.pi(n + j); };
    std::vector<int> out(2 * n, Builder::F);
    std::vector<int> S;
    for (int i = 0; i < n; i++) S.push_back(B.And(A(i), Bb(0)));
    out[0] = S[0];
    S.erase(S.begin());
    for (int j = 1; j < n; j++) {
        std::vector<int> res;
        int carry = -1;
        for (int k = 0; k < n; k++) {
            int x = B.And(A(k), Bb(j));
            bool hasY = k < (int)S.size();
            int y = hasY ? S[k] : -1;
            if (!hasY && carry < 0) {
                res.push_back(x);
            } else if (!hasY || carry < 0) {
                int o = hasY ? y : carry;
                res.push_back(B.Xor(x, o));
                carry = B.And(x, o);
            } else {
                int t = B.Xor(x, y);
                res.push_back(B.Xor(t, carry));
                carry = B.Or(B.And(x, y), B.And(carry, t));
            }
        }
        if (carry >= 0) res.push_back(carry);
        out[j] = res[0];
        S.assign(res.begin() + 1, res.end());
    }
    for (size_t k = 0; k < S.size() && n + (int)k < 2 * n; k++) out[n + k] = S[k];
    B.g.outs = out;
    remove_dangling(B.g);
    return B.g;
}

int export_graph(const Aig &g, culs_host_graph *out) {
    int nObjs = (int)g.f0.size();
    out->nPIs = g.nPIs;
    out->nPOs = (int)g.outs.size();
    out->nAnds = nObjs - 1 - g.nPIs;
    out->fanin0 = (int32_t *)malloc(sizeof(int32_t) * (size_t)nObjs);
    out->fanin1 = (int32_t *)malloc(sizeof(int32_t) * (size_t)nObjs);
    out->outs = (int32_t *)malloc(sizeof(int32_t) * (size_t)std::max(1, out->nPOs));
    if (!out->fanin0 || !out->fanin1 || !out->outs) {
        culs_host_graph_free(out);
        return CULS_E_OOM;
    }
    memcpy(out->fanin0, g.f0.data(), sizeof(int32_t) * (size_t)nObjs);
    memcpy(out->fanin1, g.f1.data(), sizeof(int32_t) * (size_t)nObjs);
    if (out->nPOs) memcpy(out->outs, g.outs.data(), sizeof(int32_t) * (size_t)out->nPOs);
    return CULS_OK;
}

}  // namespace

extern "C" {

int culs_gen_layered(uint64_t seed, int nPIs, int nPOs, int64_t nAnds, int nLayers, int window, double pFar,
                     int withPIs, culs_host_graph *out) {
    return culs::guard_call(nullptr, [&]() -> int {
        if (!out || nPIs < 2 || nAnds < 0 || nLayers < 1 || window < 1 || nAnds + nPIs + 1 > INT32_MAX / 2)
            return CULS_E_INVALID;
        if (nAnds > 0 && nAnds < nLayers) return CULS_E_INVALID;
        Aig g;
        if (!layered(g, seed, nPIs, nPOs, nAnds, nLayers, window, pFar, withPIs != 0)) return CULS_E_INVALID;
        return export_graph(g, out);
    });
}

int culs_gen_multiplier(int n, culs_host_graph *out) {
    return culs::guard_call(nullptr, [&]() -> int {
        if (!out || n < 1 || n > 4096) return CULS_E_INVALID;
        return export_graph(multiplier(n), out);
    });
}

// Batch of `count` layered graphs with sizes log-uniform in [minAnds,
// maxAnds], PI counts uniform in [minPIs, maxPIs], nLayers = round(sqrt(nAnds)),
// a 4-layer window plus PIs; every sink is a PO, so each graph keeps its drawn
// AND count.  Graph i is seeded with splitmix64(tag * 2^32 + i).  Generated on
// `threads` host threads; output order is graph order.
int culs_gen_batch(uint64_t tag, int first, int count, int64_t minAnds, int64_t maxAnds, int minPIs, int maxPIs,
                   int threads, culs_host_graph *out) {
    return culs::guard_call(nullptr, [&]() -> int {
        if (!out || count < 0 || minAnds < 1 || maxAnds < minAnds || minPIs < 2 || maxPIs < minPIs) return CULS_E_INVALID;
        if (threads < 1) threads = 1;
        std::vector<int> rc(count, CULS_E_INVALID);  // until the graph is made
        auto work = [&](int t) {
            for (int k = t; k < count; k += threads) {
                rc[k] = culs::guard_call(nullptr, [&]() -> int {
                    uint64_t seed = splitmix((tag << 32) + (uint64_t)(first + k));
                    Rng r(seed);
                    double u = r.unit();
                    int64_t nAnds = (int64_t)std::llround(
                        std::exp(std::log((double)minAnds) + u * (std::log((double)maxAnds) - std::log((double)minAnds))));
                    int nPIs = minPIs + (int)r.below((uint64_t)(maxPIs - minPIs + 1));
                    int nLayers = std::max(1, (int)std::llround(std::sqrt((double)nAnds)));
                    Aig g;
                    return layered(g, r.next(), nPIs, 0, nAnds, nLayers, 4, 0.0, true, true) ? export_graph(g, &out[k])
                                                                                              : CULS_E_INVALID;
                });
            }
        };
        std::vector<std::thread> th;
        try {
            for (int t = 0; t < threads; t++) th.emplace_back(work, t);
        } catch (...) {
            for (auto &x : th) x.join();
            for (int j = 0; j < count; j++)
                if (rc[j] == CULS_OK) culs_host_graph_free(&out[j]);
            throw;
        }
        for (auto &x : th) x.join();
        for (int k = 0; k < count; k++) {
            if (rc[k] == CULS_OK) continue;
            for (int j = 0; j < count; j++)  // no graph is returned on failure
                if (rc[j] == CULS_OK) culs_host_graph_free(&out[j]);
            return rc[k];
        }
        return CULS_OK;
    });
}

void culs_host_graph_free(culs_host_graph *g) {
    if (!g) return;
    free(g->fanin0);
    free(g->fanin1);
    free(g->outs);
    g->fanin0 = g->fanin1 = g->outs = nullptr;
}

}  // extern "C"
