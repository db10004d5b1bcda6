// ORACLE -- test infrastructure only: drives the reference CULS `rw`/`st`
// code, compiled from the reference sources by oracle/build_ref.sh, to record
// golden results for the oracle and the GPU path.  Nothing in the product
// links this file.
//
//   rw_harness full <in.aig> <out.aig> <zeros 0|1>
//   rw_harness time <reps> <in.aig>...   (the reference rw;st timed per graph)
//       AIGMan::readFile; AIGMan::rewrite(zeros, true); AIGMan::strash();
//       AIGMan::saveFile -- the sequence of `read; rw [-z]; st; write`
//       (command handlers src/command_manager.cpp:32-128).
//   rw_harness chain <in.aig> <out.aig> <script>
//       a command sequence on one AIGMan, script = comma-separated tokens
//       rw | rwz | rwc | rwzc | st | b | bn: AIGMan::rewrite(zeros = 'z',
//       fGPUDeduplicate = no 'c'), AIGMan::strash(false, true), or
//       AIGMan::balance(1, updateLevel = true for b, false for bn), printing
//       the AND count and level after each, then AIGMan::saveFile.
//   rw_harness dump <in.aig> <prefix>
//       the first half of rw::CPUSolver::Rewrite (src/algorithms/
//       rewrite.cu:811-826) step by step, writing the reordered fanins, all
//       cut slots, the selected cuts and replace[] after the rebuild.
#include <cuda_runtime.h>
#include <thrust/device_vector.h>

#include <algorithm>
#include <cassert>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>
#include <tuple>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "robin_hood.h"

// The harness reads private members of the reference's solver classes.
#define private public
#include "aig_manager.h"
#include "algorithms/rewrite.cu"
#undef private

static void put(FILE *f, const std::vector<int> &v) {
    int n = (int)v.size();
    fwrite(&n, sizeof n, 1, f);
    if (n) fwrite(v.data(), sizeof(int), v.size(), f);
}

static void canon(const rw::Cut &c, int *q) {
    if (!c.used) {
        for (int k = 0; k < 9; k++) q[k] = 0;
        return;
    }
    q[0] = 1;
    q[1] = (int)c.nLeaves;
    for (int k = 0; k < 4; k++) q[2 + k] = k < (int)c.nLeaves ? c.leaves[k] : 0;
    q[6] = (int)c.truthtable;
    q[7] = c.sign;
    q[8] = (int)c.value;
}

static int run_dump(const char *in, const char *prefix) {
    AIGMan man;
    if (!man.readFile(in)) return 2;
    rw::CPUSolver &S = man.rwMan;
    S.Reset(man.nPIs, man.nPOs, man.nObjs - 1, man.pFanin0, man.pFanin1, man.pOuts);
    const int n = S.n;
    std::vector<int> f0(S.fanin0, S.fanin0 + n + 1), f1(S.fanin1, S.fanin1 + n + 1), outs(S.output,
                                                                                         S.output + S.numOutputs);
    for (int i = 0; i <= S.numInputs; i++) f0[i] = f1[i] = 0;
    S.expected = 0;
    S.gpuSolver = new rw::GPUSolver(n);
    S.ReadLibrary();
    S.gpuSolver->CopyLib(S.lib);
    S.LevelCount();
    S.gpuSolver->EnumerateAndPreEvaluate(S.level, S.levelCount, n, S.fanin0, S.fanin1, S.ref, false);
    std::vector<rw::Cut> cuts((size_t)(n + 1) * CUT_SET_SIZE);
    cudaMemcpy(cuts.data(), S.gpuSolver->cuts, sizeof(rw::Cut) * cuts.size(), cudaMemcpyDeviceToHost);
    S.gpuSolver->GetResults(n, S.bestOut, S.bestCut);
    std::vector<int> cutv(cuts.size() * 9), sel((size_t)(n + 1) * 10);
    for (size_t i = 0; i < cuts.size(); i++) canon(cuts[i], &cutv[i * 9]);
    for (int i = 0; i <= n; i++) {
        canon(S.bestCut[i], &sel[(size_t)i * 10]);
        sel[(size_t)i * 10 + 9] = S.bestCut[i].used ? S.bestOut[i] : -1;
    }
    std::vector<int> rep(n + 1, -1);
    int n1 = S.gpuSolver->ReplaceSubgraphs(n, S.fanin0, S.fanin1, S.phase, rep.data());
    std::vector<int> nf0(S.fanin0 + n + 1, S.fanin0 + n1 + 1), nf1(S.fanin1 + n + 1, S.fanin1 + n1 + 1);
    std::string path = std::string(prefix) + ".bin";
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) return 3;
    std::vector<int> hdr = {n, n1, S.numInputs, S.numOutputs};
    put(f, hdr);
    put(f, f0);
    put(f, f1);
    put(f, outs);
    put(f, cutv);
    put(f, sel);
    put(f, rep);
    put(f, nf0);
    put(f, nf1);
    fclose(f);
    delete S.gpuSolver;
    S.gpuSolver = nullptr;
    return 0;
}

static int run_full(const char *in, const char *out, bool zeros) {
    AIGMan man;
    if (!man.readFile(in)) return 2;
    man.rewrite(zeros, true);
    printf("HARNESS after rw: and = %d level = %d\n", man.nNodes, man.nLevels);
    man.strash(false, true);
    printf("HARNESS after st: and = %d level = %d\n", man.nNodes, man.nLevels);
    man.saveFile(out);
    fflush(stdout);
    return 0;
}

static int run_chain(const char *in, const char *out, const char *script) {
    AIGMan man;
    if (!man.readFile(in)) return 2;
    std::stringstream ss(script);
    std::string tok;
    while (std::getline(ss, tok, ',')) {
        if (tok == "st") {
            man.strash(false, true);
        } else if (tok == "b") {
            man.balance(1, true);  // the `b` command: balance, then strash
        } else if (tok == "bn") {
            man.balance(1, false);  // balance as resyn2 calls it, no strash
        } else if (tok.rfind("rw", 0) == 0) {
            const bool zeros = tok.find('z') != std::string::npos;
            const bool gpuDedup = tok.find('c') == std::string::npos;
            man.rewrite(zeros, gpuDedup);
        } else {
            fprintf(stderr, "chain: unknown command %s\n", tok.c_str());
            return 4;
        }
        printf("HARNESS after %s: and = %d level = %d\n", tok.c_str(), man.nNodes, man.nLevels);
    }
    man.saveFile(out);
    fflush(stdout);
    return 0;
}

// The reference's own rw;st timed per graph (its GPU path, one AIG at a
// time): read each file, then time AIGMan::rewrite + AIGMan::strash with a
// device synchronisation on both sides; best of `reps` runs per file after
// one untimed warm-up run.
static int run_time(int reps, int nfiles, char **files) {
    long long nodes = 0;
    double ms = 0;
    for (int f = 0; f < nfiles; f++) {
        double best = -1;
        for (int r = -1; r < reps; r++) {
            AIGMan man;
            if (!man.readFile(files[f])) return 2;
            const long long n = man.nNodes;
            cudaDeviceSynchronize();
            auto t0 = std::chrono::steady_clock::now();
            man.rewrite(false, true);
            man.strash(false, true);
            cudaDeviceSynchronize();
            const double t = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            if (r >= 0 && (best < 0 || t < best)) best = t;
            if (r == 0) nodes += n;
        }
        ms += best;
    }
    printf("HARNESS time files=%d and_nodes=%lld ms=%.3f\n", nfiles, nodes, ms);
    fflush(stdout);
    return 0;
}

int main(int argc, char **argv) {
    if (argc >= 5 && !strcmp(argv[1], "full")) return run_full(argv[2], argv[3], atoi(argv[4]) != 0);
    if (argc >= 4 && !strcmp(argv[1], "time")) return run_time(atoi(argv[2]), argc - 3, argv + 3);
    if (argc >= 4 && !strcmp(argv[1], "dump")) return run_dump(argv[2], argv[3]);
    if (argc >= 5 && !strcmp(argv[1], "chain")) return run_chain(argv[2], argv[3], argv[4]);
    fprintf(stderr, "usage: rw_harness full <in.aig> <out.aig> <zeros> | dump <in.aig> <prefix>\n");
    return 1;
}
