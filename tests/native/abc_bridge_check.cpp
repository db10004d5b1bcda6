// Checks the ABC-patch bridge (culs_b200/abc_patch/abc_bridge.hpp) without
// ABC: a mock network with a structurally hashing AND constructor (as
// Abc_AigAnd folds and merges) stands in for Abc_Ntk_t.  Built and run by
// tests/test_abc_bridge.py; with --gpu it also runs the command session
// (gget; grw; gst; gput and the others) through libculs_b200.so.
#include <cstdio>
#include <cstring>
#include <map>
#include <random>
#include <string>
#include <vector>

#include "abc_bridge.hpp"

using culs_abc::HostAig;
using culs_abc::NtkView;

namespace {

int g_bad = 0;
#define CHECK(c)                                                  \
    do {                                                          \
        if (!(c)) {                                               \
            printf("FAIL %s:%d: %s\n", __FILE__, __LINE__, #c);   \
            g_bad++;                                              \
        }                                                         \
    } while (0)

// A strashed network: node 0 is constant 1, then inputs, outputs and AND
// nodes in creation order.
struct MockNtk {
    enum Kind { kConst, kPi, kPo, kAnd };
    struct Obj {
        Kind kind;
        int f0 = -1, c0 = 0, f1 = -1, c1 = 0;
    };
    std::vector<Obj> objs{Obj{kConst}};
    std::vector<int> pis, pos;
    std::map<std::pair<int, int>, int> strash;  // (lit0, lit1), lit0 <= lit1 -> AND node
};

struct MockBuilder {
    using Handle = int;
    MockNtk &n;
    Handle const1() { return 0; }
    Handle pi() {
        n.objs.push_back({MockNtk::kPi});
        n.pis.push_back((int)n.objs.size() - 1);
        return n.pis.back();
    }
    Handle po() {
        n.objs.push_back({MockNtk::kPo});
        n.pos.push_back((int)n.objs.size() - 1);
        return n.pos.back();
    }
    // x' & y' over literals 2*id + c with id 0 the constant 1
    Handle and2(Handle x, bool cx, Handle y, bool cy, bool *c) {
        int a = 2 * x + cx, b = 2 * y + cy;
        if (a > b) std::swap(a, b);
        *c = false;
        if (a == b) return *c = (a & 1), a >> 1;        // x & x
        if ((a ^ 1) == b) return *c = true, 0;          // x & !x = !1
        if (a == 0) return *c = (b & 1), b >> 1;        // 1 & y
        if (a == 1) return *c = true, 0;                // 0 & y = !1
        auto it = n.strash.find({a, b});
        if (it != n.strash.end()) return it->second;
        n.objs.push_back({MockNtk::kAnd, a >> 1, a & 1, b >> 1, b & 1});
        const int id = (int)n.objs.size() - 1;
        n.strash[{a, b}] = id;
        return id;
    }
    void drive(Handle po, Handle d, bool c) {
        n.objs[po].f0 = d;
        n.objs[po].c0 = c;
    }
};

// gget's reading of the mock: inputs, AND nodes in DFS order from the
// outputs (fanin 0 first), outputs
NtkView view_of(const MockNtk &n) {
    NtkView v;
    v.const1 = 0;
    v.ci = n.pis;
    std::vector<char> seen(n.objs.size(), 0);
    std::vector<std::pair<int, int>> stk;
    for (int po : n.pos) {
        stk.push_back({n.objs[po].f0, 0});
        while (!stk.empty()) {
            auto &[x, st] = stk.back();
            const MockNtk::Obj &o = n.objs[x];
            if (o.kind != MockNtk::kAnd || seen[x]) {
                stk.pop_back();
                continue;
            }
            if (st == 0) {
                st = 1;
                stk.push_back({o.f0, 0});
            } else if (st == 1) {
                st = 2;
                stk.push_back({o.f1, 0});
            } else {
                seen[x] = 1;
                v.ands.push_back({x, o.f0, o.c0, o.f1, o.c1});
                stk.pop_back();
            }
        }
        v.co.push_back({n.objs[po].f0, n.objs[po].c0});
    }
    return v;
}

// output values of an AIGMan-layout AIG on `words` x 64 seeded patterns
std::vector<uint64_t> simulate(const HostAig &a, int words, uint64_t seed) {
    std::mt19937_64 rng(seed);
    const int n = (int)a.F0.size();
    std::vector<uint64_t> val((size_t)n * words), out(a.outs.size() * (size_t)words);
    for (int w = 0; w < words; w++) val[w] = ~0ull;  // literal 0 is TRUE
    for (int i = 1; i <= a.nPIs; i++)
        for (int w = 0; w < words; w++) val[(size_t)i * words + w] = rng();
    auto lit = [&](int l, int w) { return val[(size_t)(l >> 1) * words + w] ^ ((l & 1) ? ~0ull : 0ull); };
    for (int i = a.nPIs + 1; i < n; i++)
        for (int w = 0; w < words; w++) val[(size_t)i * words + w] = lit(a.F0[i], w) & lit(a.F1[i], w);
    for (size_t k = 0; k < a.outs.size(); k++)
        for (int w = 0; w < words; w++) out[k * words + w] = lit(a.outs[k], w);
    return out;
}

HostAig from_host(const culs_host_graph &g) {
    HostAig a;
    a.nPIs = g.nPIs;
    const int n = 1 + g.nPIs + g.nAnds;
    a.F0.assign(g.fanin0, g.fanin0 + n);
    a.F1.assign(g.fanin1, g.fanin1 + n);
    a.outs.assign(g.outs, g.outs + g.nPOs);
    return a;
}

// A -> mock network (gput's order) -> view (gget's order) -> B
HostAig round_trip(const HostAig &a, MockNtk &n) {
    MockBuilder b{n};
    std::string err;
    CHECK(culs_abc::aig_to_ntk(a, b, err));
    HostAig r;
    CHECK(culs_abc::view_to_aig(view_of(n), r, err));
    return r;
}

std::vector<HostAig> cases() {
    std::vector<HostAig> v;
    culs_host_graph g;
    if (culs_gen_multiplier(8, &g) == CULS_OK) v.push_back(from_host(g)), culs_host_graph_free(&g);
    if (culs_gen_layered(7, 32, 16, 3000, 30, 4, 0.1, 1, &g) == CULS_OK) v.push_back(from_host(g)), culs_host_graph_free(&g);
    // constants and inputs on the outputs, x & x, x & !x, a duplicate node,
    // a dangling node: 2 inputs (ids 1, 2), ANDs 3..7
    HostAig e;
    e.nPIs = 2;
    e.F0 = {-1, -1, -1, 2, 4, 2, 2, 2};
    e.F1 = {-1, -1, -1, 4, 4, 3, 4, 5};
    e.outs = {0, 1, 3, 11, 13, 14, 8, 10};
    v.push_back(e);
    return v;
}

void cpu_checks() {
    int k = 0;
    for (const HostAig &a : cases()) {
        MockNtk n;
        const HostAig r = round_trip(a, n);
        CHECK(r.nPIs == a.nPIs && r.outs.size() == a.outs.size());
        CHECK(r.nAnds() <= a.nAnds());
        CHECK(simulate(r, 4, 11) == simulate(a, 4, 11));
        // a second trip finds nothing left to merge (the numbering may move:
        // the constructor orders fanins by their new ids)
        MockNtk n2;
        const HostAig r2 = round_trip(r, n2);
        CHECK(r2.nAnds() == r.nAnds());
        CHECK(simulate(r2, 4, 12) == simulate(a, 4, 12));
        printf("case %d: %d -> %d AND nodes\n", k++, a.nAnds(), r.nAnds());
    }
    // the hand-made case strashes down to its two distinct AND nodes
    {
        MockNtk n;
        const HostAig r = round_trip(cases().back(), n);
        CHECK(r.nAnds() == 2);
        CHECK(r.outs[0] == 0 && r.outs[1] == 1);  // constants stay constants
    }
    // refusals
    NtkView bad;
    bad.const1 = 0;
    bad.ci = {1, 2};
    bad.ands = {{4, 3, 0, 1, 0}, {3, 1, 0, 2, 0}};  // 4 reads 3 before 3 is numbered
    HostAig out;
    std::string err;
    CHECK(!culs_abc::view_to_aig(bad, out, err) && !err.empty());
    HostAig cyc;
    cyc.nPIs = 1;
    cyc.F0 = {-1, -1, 6};
    cyc.F1 = {-1, -1, 2};
    cyc.outs = {4};
    MockNtk n;
    MockBuilder b{n};
    CHECK(!culs_abc::aig_to_ntk(cyc, b, err));
}

// one command line's words
int run(culs_abc::Session &s, std::vector<std::string> words) {
    std::vector<char *> argv;
    for (std::string &w : words) argv.push_back(&w[0]);
    return s.command((int)argv.size(), argv.data());
}

void gpu_checks() {
    culs_abc::Session s;
    CHECK(run(s, {"grw"}) == 1);  // no graph yet
    for (const HostAig &a : cases()) {
        MockNtk n;
        MockBuilder b{n};
        std::string err;
        CHECK(culs_abc::aig_to_ntk(a, b, err));
        CHECK(s.get(view_of(n)) == 0);  // gget
        for (const char *line : {"grw", "gst", "grw -z -d", "gb", "grw", "grw", "gst -c", "gps"}) {
            std::vector<std::string> words;
            std::string w;
            for (const char *p = line;; p++) {
                if (*p == ' ' || !*p) {
                    if (!w.empty()) words.push_back(w);
                    w.clear();
                    if (!*p) break;
                } else {
                    w += *p;
                }
            }
            CHECK(run(s, words) == 0);
        }
        CHECK(run(s, {"gb", "-s"}) == 1);
        CHECK(run(s, {"gresyn2"}) == 1);
        CHECK(run(s, {"grw", "-q"}) == 1);
        HostAig r;
        CHECK(s.put(r) == 0);  // gput
        CHECK(!s.active());
        MockNtk back;
        MockBuilder bb{back};
        CHECK(culs_abc::aig_to_ntk(r, bb, err));
        HostAig rr;
        CHECK(culs_abc::view_to_aig(view_of(back), rr, err));
        CHECK(simulate(rr, 4, 5) == simulate(a, 4, 5));
        printf("gpu: %d -> %d AND nodes\n", a.nAnds(), rr.nAnds());
    }
}

}  // namespace

int main(int argc, char **argv) {
    cpu_checks();
    if (argc > 1 && !strcmp(argv[1], "--gpu")) gpu_checks();
    printf("bad %d\n", g_bad);
    return g_bad != 0;
}
