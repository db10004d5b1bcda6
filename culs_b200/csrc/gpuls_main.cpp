// gpuls-compatible command line over the C ABI: the command surface of CULS's
// `gpuls` (src/main.cpp, src/command_manager.cpp) for the commands on the
// rewriting path.
//
//   gpuls -c "read in.aig; rw; st; ps; write out.aig"   (script mode)
//   gpuls                                               (reads commands from stdin)
//
// Commands: read <file.aig>, write <file.aig>, ps / print_stats, time,
// rw / rewrite [-z] [-d] [-v N], st / strash [-c] [-v N].  As in the
// reference, `rw` always deduplicates on the GPU (its -d flag defaults to
// true, src/command_manager.cpp:81-95), and a command that fails prints a
// message and the script goes on.  The other optimisation commands of the
// reference (b, rf, rs, resyn2, resyn2rs) are outside this library.
#include <chrono>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "culs_b200.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Shell {
    culs_ctx *ctx = nullptr;
    culs_graph *g = nullptr;
    bool loaded = false;
    double prevAlg = 0, prevFull = 0, totalAlg = 0, totalFull = 0;

    ~Shell() {
        culs_graph_free(g);
        culs_destroy(ctx);
    }

    bool ensure_ctx() {
        if (ctx) return true;
        ctx = culs_create(0);
        if (!ctx) printf("gpuls: %s\n", culs_last_error(nullptr));
        return ctx != nullptr;
    }

    void report(int rc, const char *what) {
        if (rc != CULS_OK) printf("%s: %s\n", what, culs_last_error(ctx));
    }

    void account(Clock::time_point t0, Clock::time_point t1, Clock::time_point t2) {
        prevAlg = std::chrono::duration<double>(t2 - t1).count();
        prevFull = std::chrono::duration<double>(t2 - t0).count();
        totalAlg += prevAlg;
        totalFull += prevFull;
    }

    // AIGMan::readFile (src/aig_manager.cu:80-108)
    void read(const std::string &path) {
        if (!ensure_ctx()) return;
        auto t0 = Clock::now();
        culs_host_graph h{};
        int rc = culs_aiger_read(path.c_str(), &h);
        if (rc != CULS_OK) {
            printf("read: cannot read %s as binary AIGER\n", path.c_str());
            return;
        }
        culs_graph *ng = nullptr;
        rc = culs_graph_upload(ctx, h.fanin0, h.fanin1, h.outs, h.nPIs, h.nPOs, h.nAnds, &ng);
        culs_host_graph_free(&h);
        if (rc != CULS_OK) {
            report(rc, "read");
            return;
        }
        culs_graph_free(g);
        g = ng;
        loaded = true;
        auto t1 = Clock::now();
        account(t0, t0, t1);
    }

    // AIGMan::saveFile (src/aig_manager.cu:231-267)
    void write(const std::string &path) {
        if (!loaded) {
            printf("saveFile: AIG is null! \n");
            return;
        }
        int32_t nPIs, nPOs, nAnds, nLevels;
        culs_graph_stats(g, 0, &nPIs, &nPOs, &nAnds, &nLevels);
        const size_t n = 1 + (size_t)nPIs + nAnds;
        std::vector<int32_t> f0(n), f1(n), outs(nPOs > 0 ? nPOs : 1);
        int rc = culs_graph_download(ctx, g, 0, f0.data(), f1.data(), outs.data());
        if (rc != CULS_OK) {
            report(rc, "write");
            return;
        }
        culs_host_graph h{nPIs, nPOs, nAnds, f0.data(), f1.data(), outs.data()};
        if (culs_aiger_write(path.c_str(), &h) != CULS_OK) printf("write: cannot write %s\n", path.c_str());
    }

    // AIGMan::printStats (src/aig_manager.cu:604-612)
    void ps() {
        if (!loaded) {
            printf("AIG stats: i/o = 0/0 and = 0 level = 0\n");
            return;
        }
        int32_t nPIs, nPOs, nAnds, nLevels;
        culs_graph_stats(g, 0, &nPIs, &nPOs, &nAnds, &nLevels);
        printf("AIG stats: i/o = %d/%d and = %d level = %d\n", nPIs, nPOs, nAnds, nLevels);
    }

    // AIGMan::printTime (src/aig_manager.cu:269-273)
    void time() {
        printf("{time} prev cmd: alg %.2lf s, full %.2lf s; total: alg %.2lf s, full %.2lf s.\n", prevAlg, prevFull,
               totalAlg, totalFull);
    }

    void rw(bool zeros) {
        if (!loaded) return;
        auto t0 = Clock::now();
        int rc = culs_rw(ctx, g, CULS_RW_GPU_DEDUP | (zeros ? CULS_RW_ZEROS : 0));
        if (rc == CULS_OK) rc = culs_sync(ctx);
        auto t1 = Clock::now();
        report(rc, "rw");
        account(t0, t0, t1);
    }

    void b() {
        if (!loaded) return;
        auto t0 = Clock::now();
        int rc = culs_b(ctx, g, 0);
        if (rc == CULS_OK) rc = culs_sync(ctx);
        auto t1 = Clock::now();
        report(rc, "b");
        account(t0, t0, t1);
    }

    void st(bool cpu) {
        if (!loaded) return;
        auto t0 = Clock::now();
        int rc = culs_st(ctx, g, cpu ? CULS_ST_CPU : 0);
        if (rc == CULS_OK) rc = culs_sync(ctx);
        auto t1 = Clock::now();
        report(rc, "st");
        account(t0, t0, t1);
    }
};

// Flags of a command: every literal after the command must be one of the
// allowed flags, or an option taking a value (-v N).
bool parse_flags(const std::vector<std::string> &lit, const char *flags, bool *seen) {
    for (size_t i = 1; i < lit.size(); i++) {
        const std::string &a = lit[i];
        if (a == "-v") {
            if (++i >= lit.size()) return false;
            continue;
        }
        if (a.size() != 2 || a[0] != '-') return false;
        const char *p = strchr(flags, a[1]);
        if (!p) return false;
        seen[p - flags] = true;
    }
    return true;
}

void run_command(Shell &sh, const std::string &line) {
    std::istringstream in(line);
    std::vector<std::string> lit;
    for (std::string w; in >> w;) lit.push_back(w);
    if (lit.empty()) return;
    const std::string &cmd = lit[0];
    bool ok = true;
    if (cmd == "read") {
        if (lit.size() < 2)
            ok = false;
        else
            sh.read(lit[1]);
    } else if (cmd == "write") {
        if (lit.size() < 2) {
            ok = false;
        } else if (lit[1].size() < 4 || lit[1].compare(lit[1].size() - 4, 4, ".aig") != 0) {
            printf("write: only support .aig format!\n");
            ok = false;
        } else {
            sh.write(lit[1]);
        }
    } else if (cmd == "ps" || cmd == "print_stats") {
        sh.ps();
    } else if (cmd == "time") {
        sh.time();
    } else if (cmd == "rw" || cmd == "rewrite") {
        bool seen[2] = {false, false};
        ok = parse_flags(lit, "zd", seen);
        if (ok) sh.rw(seen[0]);
    } else if (cmd == "st" || cmd == "strash") {
        bool seen[1] = {false};
        ok = parse_flags(lit, "c", seen);
        if (ok) sh.st(seen[0]);
    } else if (cmd == "b" || cmd == "balance") {
        bool seen[1] = {false};
        ok = parse_flags(lit, "s", seen);
        if (ok && seen[0]) {
            printf("balance -s (seeded shuffle of equal-level inputs) is not provided, ignored.\n");
            return;
        }
        if (ok) sh.b();
    } else if (cmd == "rf" || cmd == "refactor" || cmd == "rs" || cmd == "resub" || cmd == "resyn2" ||
               cmd == "resyn2rs" || cmd == "r2rs") {
        printf("Command %s is not part of this library (rw, st and b only), ignored.\n", cmd.c_str());
        return;
    } else {
        printf("Command %s not registered, ignored.\n", cmd.c_str());
        return;
    }
    if (!ok) printf("Command %s not recognized or in wrong format!\n", cmd.c_str());
}

void split_script(const std::string &script, std::vector<std::string> &out) {
    std::string cur;
    for (char c : script) {
        if (c == ';') {
            out.push_back(cur);
            cur.clear();
        } else {
            cur += c;
        }
    }
    out.push_back(cur);
}

}  // namespace

int main(int argc, char **argv) {
    std::string script;
    for (int i = 1; i < argc; i++) {
        if ((!strcmp(argv[i], "-c") || !strcmp(argv[i], "--script")) && i + 1 < argc) {
            script = argv[++i];
        } else {
            fprintf(stderr, "usage: %s [-c \"cmd; cmd; ...\"]\n", argv[0]);
            return 1;
        }
    }
    Shell sh;
    if (!script.empty()) {
        std::cout << "Running in script mode: \"" << script << "\"." << std::endl;
        std::cout << "============================================" << std::endl;
        std::vector<std::string> cmds;
        split_script(script, cmds);
        for (const auto &c : cmds) run_command(sh, c);
        return 0;
    }
    std::cout << "Starting interactive mode" << std::endl;
    for (std::string line; std::cout << "gpuls> " << std::flush, std::getline(std::cin, line);) {
        if (line == "exit" || line == "quit") break;
        std::vector<std::string> cmds;
        split_script(line, cmds);
        for (const auto &c : cmds) run_command(sh, c);
    }
    std::cout << "gpuls terminated." << std::endl;
    return 0;
}
