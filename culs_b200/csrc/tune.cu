// Autotuner of the launch and schedule parameters (engine.cuh, Tune).
//
// The parameters change only speed, never results.  The enumeration's
// schedule -- which levels run one node per thread and which one node per
// warp, and how many persistent blocks share the SMs -- depends on the
// workload's level widths and depths, so it is chosen by timing rw's cut
// enumeration (device events around the kernel) on clones of a sample of
// the workload: first the width threshold at the default grid, then the
// grid at the chosen threshold.  Then the evaluation's group size (how many
// graphs' existence tables are built and probed together, which decides
// whether they stay in L2), timed on the evaluation's marks.
#include <cfloat>

#include "engine.cuh"

namespace culs {

int Engine::autotune(const Batch &sample, int rounds) {
    if (sample.G < 1) return fail(CULS_E_INVALID, "autotune: empty sample");
    if (rounds < 1) rounds = 1;
    const bool prof = prof_;
    prof_ = true;
    Batch work;
    // rw's time between marks m0 and m1, the best of `rounds` runs
    int m0 = kMkEnumK0, m1 = kMkEnumK1;
    auto measure = [&](const Tune &t, float &ms) -> int {
        tune_ = t;
        ms = FLT_MAX;
        for (int r = 0; r < rounds; r++) {
            int rc = clone(sample, work);
            RwStats st{};
            if (rc == CULS_OK) rc = rw(work, false, true, &st, nullptr);
            if (rc != CULS_OK) return rc;
            const float e = elapsed(m0, m1);
            if (e >= 0.f && e < ms) ms = e;
        }
        return CULS_OK;
    };
    Tune best = tune_;
    float bestMs = FLT_MAX;
    int rc = CULS_OK;
    {  // one untimed pass first: clocks, caches and the arena settle
        float ms;
        if ((rc = measure(best, ms))) {
            tune_ = best;
            prof_ = prof;
            return rc;
        }
    }
    const int wides[] = {2048, 4096, 8192, 16384, 32768, 65536, 1 << 30};
    for (int w : wides) {
        Tune t = best;
        t.enumWideMin = w;
        float ms;
        if ((rc = measure(t, ms))) break;
        if (ms < bestMs) {
            bestMs = ms;
            best = t;
        }
    }
    const int grids[] = {4, 6, 12, 16};
    for (int b : grids) {
        if (rc) break;
        Tune t = best;
        t.enumBlocksPerSm = b;
        float ms;
        if ((rc = measure(t, ms))) break;
        if (ms < bestMs) {
            bestMs = ms;
            best = t;
        }
    }
    // the evaluation's group size, at the chosen enumeration schedule
    m0 = kMkEvalK0, m1 = kMkEvalK1;
    if (!rc) {
        float ms;
        rc = measure(best, ms);
        bestMs = ms;
    }
    const int groups[] = {4, 8, 32, 64};
    for (int gm : groups) {
        if (rc) break;
        Tune t = best;
        t.evalGroupMSlots = gm;
        float ms;
        if ((rc = measure(t, ms))) break;
        if (ms < bestMs) {
            bestMs = ms;
            best = t;
        }
    }
    tune_ = best;
    prof_ = prof;
    return rc;
}

}  // namespace culs
