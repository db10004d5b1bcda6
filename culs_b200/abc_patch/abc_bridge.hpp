// The ABC-patch commands (`gget`, `gput`, `grw`, `gst`, `gb`, `gps`) of CULS
// (src/abc_patch/abc_patch_gpucmd.cpp:110-251, abc_patch_transform.cpp:5-149)
// over the C ABI, written against a neutral view of an ABC network so that
// everything but the last adaptation compiles and is tested without an ABC
// tree.  culs_abc_patch.cpp adapts ABC's Abc_Ntk_t to it and registers the
// commands; that file needs ABC's headers and is built only when an ABC
// tree is supplied (build_abc_patch.sh).
//
//  * gget (AbcNtkToGpuMan): a strashed network's combinational inputs
//    become objects 1..nPIs in their order, the constant-1 node object 0,
//    the AND nodes of a DFS from the outputs objects nPIs+1.. in DFS order;
//    literal = 2*id + complement, so literal 0 is constant TRUE (AIGMan).
//  * gput (GpuManToAbcNtk): a new strashed network gets the constant, the
//    inputs and the outputs, then every AND node in id order through the
//    network's own AND constructor (which may merge or fold, as Abc_AigAnd
//    does), then the outputs' drivers.
//  * grw [-z] [-d], gst [-c], gb: culs_rw / culs_st / culs_b on the graph
//    held since the last gget.  As in the reference, grw deduplicates on the
//    CPU side unless -d is given, gst on the GPU unless -c is given, and a
//    grw without -d keeps the rewrite manager's graph for a following grw
//    (the C ABI keeps it inside the graph handle).
//  * gb -s (sortDecId 0) and grf / gresyn2 (refactoring) are not provided
//    by this library; they fail with a message, as a bad option does.
#pragma once

#include <cstdint>
#include <cstdio>
#include <string>
#include <unordered_map>
#include <vector>

#include "culs_b200.h"

namespace culs_abc {

// What gget reads from a strashed network (node ids are the network's).
struct NtkView {
    int const1 = -1;        // id of the constant-1 node
    std::vector<int> ci;    // combinational inputs, in order
    struct And {
        int id, f0, c0, f1, c1;
    };
    std::vector<And> ands;  // AND nodes, every fanin before its node
    struct Co {
        int f, c;
    };
    std::vector<Co> co;     // combinational outputs' drivers, in order
};

// An AIG in the AIGMan layout of culs_b200.h.
struct HostAig {
    int nPIs = 0;
    std::vector<int32_t> F0, F1, outs;  // 1 + nPIs + nAnds entries; nPOs
    int nAnds() const { return (int)F0.size() - 1 - nPIs; }
};

inline int lit_of(int id, int c) { return 2 * id + (c ? 1 : 0); }

// gget's numbering (abc_patch_transform.cpp:5-83).  False, with err set,
// when a fanin has no number yet (the ANDs are not in DFS order) or an id
// repeats.
inline bool view_to_aig(const NtkView &v, HostAig &a, std::string &err) {
    std::unordered_map<int, int> num;
    num.reserve(2 * (v.ci.size() + v.ands.size()) + 2);
    num[v.const1] = 0;
    for (size_t i = 0; i < v.ci.size(); i++)
        if (!num.emplace(v.ci[i], (int)i + 1).second) return err = "an input id repeats", false;
    a.nPIs = (int)v.ci.size();
    const size_t nObjs = 1 + v.ci.size() + v.ands.size();
    a.F0.assign(nObjs, -1);
    a.F1.assign(nObjs, -1);
    for (size_t k = 0; k < v.ands.size(); k++) {
        const NtkView::And &n = v.ands[k];
        const auto i0 = num.find(n.f0), i1 = num.find(n.f1);
        if (i0 == num.end() || i1 == num.end()) return err = "the AND nodes are not in DFS order", false;
        const int id = a.nPIs + 1 + (int)k;
        a.F0[id] = lit_of(i0->second, n.c0);
        a.F1[id] = lit_of(i1->second, n.c1);
        if (!num.emplace(n.id, id).second) return err = "an AND node id repeats", false;
    }
    a.outs.resize(v.co.size());
    for (size_t i = 0; i < v.co.size(); i++) {
        const auto f = num.find(v.co[i].f);
        if (f == num.end()) return err = "an output's driver is not numbered", false;
        a.outs[i] = lit_of(f->second, v.co[i].c);
    }
    return true;
}

// gput's construction order (abc_patch_transform.cpp:85-149) over a
// builder B with
//   Handle const1(); Handle pi(); Handle po();
//   Handle and2(Handle x, bool cx, Handle y, bool cy, bool *c);
//   void drive(Handle po, Handle driver, bool c);
// and2 returns the node that realises x' & y' (x' = x complemented when cx)
// and sets *c when the AND equals that node's complement (a constructor
// that folds x & !x onto the constant returns the constant-1 node with *c
// set); an AND equal to an existing node may return that node.
template <class B>
bool aig_to_ntk(const HostAig &a, B &b, std::string &err) {
    using H = typename B::Handle;
    const int nObjs = (int)a.F0.size();
    std::vector<H> obj(nObjs);
    std::vector<char> cmp(nObjs, 0);
    std::vector<char> made(nObjs, 0);
    obj[0] = b.const1();
    made[0] = 1;
    for (int i = 1; i <= a.nPIs; i++) obj[i] = b.pi(), made[i] = 1;
    std::vector<H> pos(a.outs.size());
    for (size_t i = 0; i < a.outs.size(); i++) pos[i] = b.po();
    for (int i = a.nPIs + 1; i < nObjs; i++) {
        const int l0 = a.F0[i], l1 = a.F1[i];
        if (l0 < 0 || l1 < 0 || (l0 >> 1) >= i || (l1 >> 1) >= i || !made[l0 >> 1] || !made[l1 >> 1])
            return err = "an AND node's fanin is not an earlier object", false;
        bool c = false;
        obj[i] = b.and2(obj[l0 >> 1], ((l0 & 1) != 0) != (cmp[l0 >> 1] != 0), obj[l1 >> 1],
                        ((l1 & 1) != 0) != (cmp[l1 >> 1] != 0), &c);
        cmp[i] = c;
        made[i] = 1;
    }
    for (size_t i = 0; i < a.outs.size(); i++) {
        const int l = a.outs[i];
        if (l < 0 || (l >> 1) >= nObjs) return err = "an output literal is out of range", false;
        b.drive(pos[i], obj[l >> 1], ((l & 1) != 0) != (cmp[l >> 1] != 0));
    }
    return true;
}

// The command state of abc_patch.cpp (s_gpuFrame): one context and the
// graph taken by the last gget.  Every method returns 0 on success and 1 on
// failure after printing why, the ABC command convention.
class Session {
  public:
    ~Session() {
        if (g_) culs_graph_free(g_);
        if (ctx_) culs_destroy(ctx_);
    }
    bool active() const { return g_ != nullptr; }

    int get(const NtkView &v) {
        HostAig a;
        std::string err;
        if (!view_to_aig(v, a, err)) return fail(err.c_str());
        return get(a);
    }
    int get(const HostAig &a) {
        if (!ensure_ctx()) return 1;
        drop();
        if (culs_graph_upload(ctx_, a.F0.data(), a.F1.data(), a.outs.data(), a.nPIs, (int32_t)a.outs.size(),
                              a.nAnds(), &g_) != CULS_OK)
            return fail(culs_last_error(ctx_));
        return 0;
    }
    // gput: the held graph, which is released afterwards
    int put(HostAig &a) {
        if (!check_active()) return 1;
        int32_t nPIs, nPOs, nAnds, nLevels;
        if (culs_graph_stats(g_, 0, &nPIs, &nPOs, &nAnds, &nLevels) != CULS_OK) return fail(culs_last_error(ctx_));
        a.nPIs = nPIs;
        a.F0.assign((size_t)1 + nPIs + nAnds, -1);
        a.F1.assign((size_t)1 + nPIs + nAnds, -1);
        a.outs.assign((size_t)nPOs, 0);
        if (culs_graph_download(ctx_, g_, 0, a.F0.data(), a.F1.data(), a.outs.data()) != CULS_OK)
            return fail(culs_last_error(ctx_));
        drop();
        return 0;
    }
    int rw(bool zeros, bool gpuDedup) {
        if (!check_active()) return 1;
        const uint32_t f = (zeros ? CULS_RW_ZEROS : 0u) | (gpuDedup ? CULS_RW_GPU_DEDUP : 0u);
        return culs_rw(ctx_, g_, f) == CULS_OK ? 0 : fail(culs_last_error(ctx_));
    }
    int st(bool cpu) {
        if (!check_active()) return 1;
        return culs_st(ctx_, g_, cpu ? CULS_ST_CPU : 0u) == CULS_OK ? 0 : fail(culs_last_error(ctx_));
    }
    int b(bool sortWithoutDecId) {
        if (!check_active()) return 1;
        if (sortWithoutDecId) return fail("gb -s (sortDecId 0) is not provided by this library");
        return culs_b(ctx_, g_, 0u) == CULS_OK ? 0 : fail(culs_last_error(ctx_));
    }
    int print_stats() {
        if (!check_active()) return 1;
        int32_t nPIs, nPOs, nAnds, nLevels;
        if (culs_graph_stats(g_, 0, &nPIs, &nPOs, &nAnds, &nLevels) != CULS_OK) return fail(culs_last_error(ctx_));
        printf("pi = %d, po = %d, and = %d, lev = %d\n", nPIs, nPOs, nAnds, nLevels);
        return 0;
    }

    // Runs one command line's words (argv[0] = the command name).
    int command(int argc, char **argv) {
        const std::string cmd = argc > 0 ? argv[0] : "";
        bool z = false, d = false, c = false, s = false;
        for (int i = 1; i < argc; i++) {
            const std::string o = argv[i];
            if (o == "-z" && cmd == "grw")
                z = true;
            else if (o == "-d" && cmd == "grw")
                d = true;
            else if (o == "-c" && cmd == "gst")
                c = true;
            else if (o == "-s" && cmd == "gb")
                s = true;
            else
                return fail(("unknown option " + o + " of " + cmd).c_str());
        }
        if (cmd == "grw") return rw(z, d);
        if (cmd == "gst") return st(c);
        if (cmd == "gb") return b(s);
        if (cmd == "gps") return print_stats();
        if (cmd == "grf" || cmd == "gresyn2") return fail("refactoring (grf, gresyn2) is not provided by this library");
        return fail(("unknown command " + cmd).c_str());
    }

  private:
    bool ensure_ctx() {
        if (!ctx_) ctx_ = culs_create(0);
        if (!ctx_) fail(culs_last_error(nullptr));
        return ctx_ != nullptr;
    }
    bool check_active() {
        if (g_) return true;
        fail("no graph: run gget first");
        return false;
    }
    void drop() {
        if (g_) culs_graph_free(g_);
        g_ = nullptr;
    }
    int fail(const char *why) {
        fprintf(stderr, "culs: %s\n", why ? why : "error");
        return 1;
    }
    culs_ctx *ctx_ = nullptr;
    culs_graph *g_ = nullptr;
};

}  // namespace culs_abc
