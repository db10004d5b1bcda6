// Host side of batch transfers: upload (validation, AIGMan depth, staging)
// and whole-batch download.  Graphs are independent, so the host work runs
// on a few threads, each taking a contiguous run of graphs of about equal
// object count; data cross PCIe from one pinned staging buffer that the
// engine keeps and grows, so a transfer is one asynchronous copy per array.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <exception>
#include <mutex>
#include <thread>
#include <vector>

#include "engine.cuh"

namespace culs {

namespace {

// Splits graphs [0, G) into at most `parts` contiguous runs of about equal
// weight; returns the run starts (size runs + 1).
std::vector<int> split_runs(const std::vector<DevGraph> &hg, int64_t total, int parts) {
    std::vector<int> cut{0};
    int64_t acc = 0;
    const int G = (int)hg.size();
    for (int g = 0; g < G; g++) {
        acc += 1 + (int64_t)hg[g].nPIs + hg[g].nAnds;
        if ((int)cut.size() < parts && acc * parts >= total * (int64_t)cut.size() && g + 1 < G) cut.push_back(g + 1);
    }
    cut.push_back(G);
    return cut;
}

int host_threads(int64_t work, int G) {
    if (work < (1 << 20) || G < 2) return 1;
    const unsigned hw = std::thread::hardware_concurrency();
    return (int)std::max(1u, std::min({hw ? hw : 1u, 32u, (unsigned)G}));
}

// Runs fn(run) for every run on its own thread (the first on the caller's).
// An exception of any run is rethrown on the caller's thread once every
// started thread has been joined.
template <class F>
void run_parallel(int runs, F fn) {
    std::exception_ptr err;
    std::mutex mu;
    auto call = [&](int r) {
        try {
            fn(r);
        } catch (...) {
            std::lock_guard<std::mutex> lk(mu);
            if (!err) err = std::current_exception();
        }
    };
    std::vector<std::thread> th;
    try {
        for (int r = 1; r < runs; r++) th.emplace_back(call, r);
    } catch (...) {
        for (auto &t : th) t.join();
        throw;
    }
    call(0);
    for (auto &t : th) t.join();
    if (err) std::rethrow_exception(err);
}

}  // namespace

int Engine::prepare(int64_t nObj) {
    int rc = ensure_arena((size_t)nObj * 640 + ((size_t)256 << 20));
    if (rc == CULS_OK) rc = ensure_stage(3 * (size_t)nObj);
    return rc;
}

int Engine::ensure_stage(size_t ints) {
    ints = std::max<size_t>(ints, 1);
    if (stage_ && stageCap_ >= ints) return 0;
    if (stage_) cudaFreeHost(stage_);
    stage_ = nullptr;
    stageCap_ = 0;
    const size_t want = ints + ints / 8;  // headroom against regrowth
    if (cudaHostAlloc(&stage_, sizeof(int32_t) * want, cudaHostAllocDefault) != cudaSuccess) {
        stage_ = nullptr;
        return fail(CULS_E_OOM, "pinned staging buffer");
    }
    stageCap_ = want;
    return 0;
}

// AIGMan::readFromMemory + toDevice (src/aig_manager.cu:80-312) for a batch:
// every graph is validated (fanins precede their node, literals in range),
// its depth computed, and its arrays staged graph-major.
int Engine::upload(Batch &b, int count, const int32_t *const *f0, const int32_t *const *f1,
                   const int32_t *const *outs, const int32_t *nPIs, const int32_t *nPOs, const int32_t *nAnds) {
    if (count < 1) return fail(CULS_E_INVALID, "upload: no graphs");
    std::vector<DevGraph> hg(count);
    int64_t nObj = 0, nPO = 0;
    for (int g = 0; g < count; g++) {
        if (nPIs[g] < 0 || nPOs[g] < 0 || nAnds[g] < 0) return fail(CULS_E_INVALID, "upload: negative size");
        hg[g] = DevGraph{nPIs[g], nPOs[g], nAnds[g], 0, (int)nObj, (int)nPO, (int)nObj, 0};
        nObj += 1 + (int64_t)nPIs[g] + nAnds[g];
        nPO += nPOs[g];
        if (nObj >= (1ll << 29)) return fail(CULS_E_INVALID, "upload: batch too large for 30-bit node positions");
    }
    int rc;
    if ((rc = ensure_stage((size_t)2 * nObj + nPO))) return rc;
    if (!b.pool) b.pool = pool_;
    if ((rc = check(b.reserve(nObj, nPO, count), "cudaMalloc"))) return rc;
    int32_t *sF0 = stage_, *sF1 = stage_ + nObj, *sPO = stage_ + 2 * nObj;
    const std::vector<int> runs = split_runs(hg, nObj, host_threads(nObj, count));
    std::atomic<int> bad{0};
    std::mutex mu;
    std::string why;
    auto work = [&](int r) {
        std::vector<int> d;
        for (int g = runs[r]; g < runs[r + 1] && !bad.load(std::memory_order_relaxed); g++) {
            const int n = 1 + nPIs[g] + nAnds[g];
            const int64_t base = hg[g].base;
            d.assign(n, 0);
            int mx = 0;
            for (int i = 0; i <= nPIs[g]; i++) sF0[base + i] = sF1[base + i] = -1;
            for (int i = nPIs[g] + 1; i < n; i++) {
                const int a = f0[g][i], c = f1[g][i];
                if (a < 0 || c < 0 || (a >> 1) >= i || (c >> 1) >= i) {
                    std::lock_guard<std::mutex> lk(mu);
                    if (!bad.exchange(1)) why = "upload: fanin literal out of range or not topological";
                    return;
                }
                sF0[base + i] = a;
                sF1[base + i] = c;
                const int di = 1 + std::max(d[a >> 1], d[c >> 1]);
                d[i] = di;
                mx = di > mx ? di : mx;
            }
            for (int k = 0; k < nPOs[g]; k++) {
                const int o = outs[g][k];
                if (o < 0 || (o >> 1) >= n) {
                    std::lock_guard<std::mutex> lk(mu);
                    if (!bad.exchange(1)) why = "upload: PO literal out of range";
                    return;
                }
                sPO[hg[g].poOff + k] = o;
            }
            hg[g].nLevels = mx;  // AIGMan::readFromMemory's nLevels
        }
        // this run is staged: its copies overlap the other runs' staging
        const DevGraph &a = hg[runs[r]], &z = hg[runs[r + 1] - 1];
        const int64_t o0 = a.base, o1 = (int64_t)z.base + 1 + z.nPIs + z.nAnds;
        const int64_t p0 = a.poOff, p1 = (int64_t)z.poOff + z.nPOs;
        cudaMemcpyAsync(b.F0 + o0, sF0 + o0, sizeof(int) * (o1 - o0), cudaMemcpyHostToDevice, s_);
        cudaMemcpyAsync(b.F1 + o0, sF1 + o0, sizeof(int) * (o1 - o0), cudaMemcpyHostToDevice, s_);
        if (p1 > p0) cudaMemcpyAsync(b.PO + p0, sPO + p0, sizeof(int) * (p1 - p0), cudaMemcpyHostToDevice, s_);
    };
    run_parallel((int)runs.size() - 1, work);
    if (bad.load()) {
        sync();  // copies already issued read the staging buffer
        return fail(CULS_E_INVALID, why);
    }
    cudaMemcpyAsync(b.dg, hg.data(), sizeof(DevGraph) * count, cudaMemcpyHostToDevice, s_);
    b.G = count;
    b.nObj = nObj;
    b.nPO = nPO;
    b.hg = hg;
    // the staging buffer is reused by the next transfer: wait for the copies
    return sync();
}

// toHost (src/aig_manager.cu:314-350) for a whole batch.
int Engine::download_all(const Batch &b, int32_t *const *f0, int32_t *const *f1, int32_t *const *outs) {
    int rc;
    if ((rc = ensure_stage((size_t)2 * b.nObj + b.nPO))) return rc;
    int32_t *sF0 = stage_, *sF1 = stage_ + b.nObj, *sPO = stage_ + 2 * b.nObj;
    const std::vector<int> runs = split_runs(b.hg, b.nObj, host_threads(b.nObj, b.G));
    const int nr = (int)runs.size() - 1;
    // one event per run: a thread scatters its run as soon as it has landed
    std::vector<cudaEvent_t> ev(nr, nullptr);
    for (int r = 0; r < nr && rc == 0; r++) {
        const DevGraph &a = b.hg[runs[r]], &z = b.hg[runs[r + 1] - 1];
        const int64_t o0 = a.base, o1 = (int64_t)z.base + 1 + z.nPIs + z.nAnds;
        const int64_t p0 = a.poOff, p1 = (int64_t)z.poOff + z.nPOs;
        if (f0) rc = check(cudaMemcpyAsync(sF0 + o0, b.F0 + o0, sizeof(int) * (o1 - o0), cudaMemcpyDeviceToHost, s_),
                           "d2h");
        if (!rc && f1)
            rc = check(cudaMemcpyAsync(sF1 + o0, b.F1 + o0, sizeof(int) * (o1 - o0), cudaMemcpyDeviceToHost, s_), "d2h");
        if (!rc && outs && p1 > p0)
            rc = check(cudaMemcpyAsync(sPO + p0, b.PO + p0, sizeof(int) * (p1 - p0), cudaMemcpyDeviceToHost, s_), "d2h");
        if (!rc) rc = check(cudaEventCreateWithFlags(&ev[r], cudaEventDisableTiming), "event");
        if (!rc) rc = check(cudaEventRecord(ev[r], s_), "event");
    }
    if (rc) {
        sync();
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
        return rc;
    }
    std::atomic<int> bad{0};
    run_parallel(nr, [&](int r) {
        if (cudaEventSynchronize(ev[r]) != cudaSuccess) {
            bad.store(1);
            return;
        }
        for (int g = runs[r]; g < runs[r + 1]; g++) {
            const DevGraph &d = b.hg[g];
            const size_t n = 1 + (size_t)d.nPIs + d.nAnds;
            if (f0 && f0[g]) memcpy(f0[g], sF0 + d.base, sizeof(int32_t) * n);
            if (f1 && f1[g]) memcpy(f1[g], sF1 + d.base, sizeof(int32_t) * n);
            if (outs && outs[g] && d.nPOs) memcpy(outs[g], sPO + d.poOff, sizeof(int32_t) * d.nPOs);
        }
    });
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
    if (bad.load()) return check(cudaErrorUnknown, "d2h");
    return 0;
}

}  // namespace culs

namespace culs {

// Literals are graph-local, so joining batches moves arrays as they are and
// only the graph table's bases and PO offsets shift.
int Engine::concat(const std::vector<const Batch *> &parts, Batch &dst) {
    int64_t nObj = 0, nPO = 0;
    int G = 0;
    for (const Batch *p : parts) {
        nObj += p->nObj;
        nPO += p->nPO;
        G += p->G;
    }
    if (G < 1) return fail(CULS_E_INVALID, "concat: no graphs");
    if (nObj >= (1ll << 29)) return fail(CULS_E_INVALID, "concat: batch too large for 30-bit node positions");
    int rc;
    if (!dst.pool) dst.pool = pool_;
    if ((rc = check(dst.reserve(nObj, nPO, G), "cudaMalloc"))) return rc;
    std::vector<DevGraph> hg;
    hg.reserve(G);
    int64_t o = 0, po = 0;
    for (const Batch *p : parts) {
        if (p->nObj) {
            cudaMemcpyAsync(dst.F0 + o, p->F0, sizeof(int) * p->nObj, cudaMemcpyDeviceToDevice, s_);
            cudaMemcpyAsync(dst.F1 + o, p->F1, sizeof(int) * p->nObj, cudaMemcpyDeviceToDevice, s_);
        }
        if (p->nPO) cudaMemcpyAsync(dst.PO + po, p->PO, sizeof(int) * p->nPO, cudaMemcpyDeviceToDevice, s_);
        for (DevGraph d : p->hg) {
            d.base += (int)o;
            d.poOff += (int)po;
            d.cpos = d.base;
            hg.push_back(d);
        }
        o += p->nObj;
        po += p->nPO;
    }
    cudaMemcpyAsync(dst.dg, hg.data(), sizeof(DevGraph) * G, cudaMemcpyHostToDevice, s_);
    dst.G = G;
    dst.nObj = nObj;
    dst.nPO = nPO;
    dst.hg = hg;
    if ((rc = check(cudaGetLastError(), "concat"))) return rc;
    return sync();  // hg's host copy feeds the table copy above
}

int Engine::split(const Batch &src, const std::vector<Batch *> &parts) {
    int first = 0, rc;
    for (Batch *p : parts) {
        const int G = p->G;
        if (first + G > src.G) return fail(CULS_E_INVALID, "split: graph counts do not add up");
        const DevGraph &a = src.hg[first];
        const DevGraph &z = src.hg[first + G - 1];
        const int64_t objEnd = (int64_t)z.base + 1 + z.nPIs + z.nAnds;
        const int64_t nObj = objEnd - a.base, nPO = (int64_t)z.poOff + z.nPOs - a.poOff;
        if (!p->pool) p->pool = pool_;
        if ((rc = check(p->reserve(nObj, nPO, G), "cudaMalloc"))) return rc;
        cudaMemcpyAsync(p->F0, src.F0 + a.base, sizeof(int) * nObj, cudaMemcpyDeviceToDevice, s_);
        cudaMemcpyAsync(p->F1, src.F1 + a.base, sizeof(int) * nObj, cudaMemcpyDeviceToDevice, s_);
        if (nPO) cudaMemcpyAsync(p->PO, src.PO + a.poOff, sizeof(int) * nPO, cudaMemcpyDeviceToDevice, s_);
        std::vector<DevGraph> hg(src.hg.begin() + first, src.hg.begin() + first + G);
        for (DevGraph &d : hg) {
            d.base -= a.base;
            d.poOff -= a.poOff;
            d.cpos = d.base;
        }
        cudaMemcpyAsync(p->dg, hg.data(), sizeof(DevGraph) * G, cudaMemcpyHostToDevice, s_);
        p->nObj = nObj;
        p->nPO = nPO;
        p->hg = hg;
        if ((rc = sync())) return rc;  // before hg goes out of scope
        first += G;
    }
    return check(cudaGetLastError(), "split");
}

}  // namespace culs
