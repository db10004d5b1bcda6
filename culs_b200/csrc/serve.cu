// Served mode (serve.cuh).
#include <algorithm>

#include "serve.cuh"

namespace culs {

Server::Server(Engine &eng, std::mutex &engMu, size_t admitBytes, int maxBatch, int workers)
    : eng_(eng), engMu_(engMu), maxBatch_(maxBatch > 0 ? maxBatch : 1 << 20) {
    workers = workers < 1 ? 1 : workers;
    admit_ = admitBytes / (size_t)workers;  // every worker's batch within its share
    for (int w = 1; w < workers; w++) {
        auto e = std::make_unique<Engine>();
        if (e->init(eng.budget() / (size_t)workers) != CULS_OK) break;  // fewer workers
        own_.push_back(std::move(e));
        ownMu_.push_back(std::make_unique<std::mutex>());
    }
    th_ = std::thread([this] { worker(eng_, engMu_); });
    for (size_t i = 0; i < own_.size(); i++) {
        Engine *e = own_[i].get();
        std::mutex *m = ownMu_[i].get();
        extra_.emplace_back([this, e, m] { worker(*e, *m); });
    }
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_ = true;
    }
    cvWork_.notify_all();
    if (th_.joinable()) th_.join();
    for (auto &t : extra_)
        if (t.joinable()) t.join();
}

int Server::submit(const int32_t *f0, const int32_t *f1, const int32_t *outs, int32_t nPIs, int32_t nPOs,
                   int32_t nAnds, uint32_t rwFlags, uint32_t stFlags, int64_t *id) {
    if (!id || nPIs < 0 || nPOs < 0 || nAnds < 0 || (nAnds && (!f0 || !f1)) || (nPOs && !outs))
        return CULS_E_INVALID;
    auto job = std::make_unique<ServeJob>();
    const size_t n = 1 + (size_t)nPIs + nAnds;
    job->rwFlags = rwFlags;
    job->stFlags = stFlags;
    job->nPIs = nPIs;
    job->nPOs = nPOs;
    job->nAnds = nAnds;
    job->f0.assign(n, -1);
    job->f1.assign(n, -1);
    if (nAnds) {
        std::copy(f0 + nPIs + 1, f0 + n, job->f0.begin() + nPIs + 1);
        std::copy(f1 + nPIs + 1, f1 + n, job->f1.begin() + nPIs + 1);
    }
    job->outs.assign(outs, outs + nPOs);
    job->state = kQueued;
    job->tSubmit = std::chrono::steady_clock::now();
    {
        std::lock_guard<std::mutex> lk(mu_);
        job->id = nextId_++;
        *id = job->id;
        queue_.push_back(job->id);
        jobs_[job->id] = std::move(job);
    }
    cvWork_.notify_one();
    return CULS_OK;
}

int Server::poll(int64_t id, int32_t *nPIs, int32_t *nPOs, int32_t *nAnds, int32_t *nLevels) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = jobs_.find(id);
    if (it == jobs_.end()) return CULS_E_NOTFOUND;
    const ServeJob &j = *it->second;
    if (j.state == kQueued || j.state == kRunning) return CULS_E_BUSY;
    if (j.state != kDone) return j.state;
    if (nPIs) *nPIs = j.nPIs;
    if (nPOs) *nPOs = j.nPOs;
    if (nAnds) *nAnds = j.nAnds;
    if (nLevels) *nLevels = j.nLevels;
    return CULS_OK;
}

int Server::wait(int64_t id, int timeoutMs) {
    std::unique_lock<std::mutex> lk(mu_);
    auto finished = [&] {
        auto it = jobs_.find(id);
        return it == jobs_.end() || (it->second->state != kQueued && it->second->state != kRunning);
    };
    if (timeoutMs < 0)
        cvDone_.wait(lk, finished);
    else
        cvDone_.wait_for(lk, std::chrono::milliseconds(timeoutMs), finished);
    auto it = jobs_.find(id);
    if (it == jobs_.end()) return CULS_E_NOTFOUND;
    const int st = it->second->state;
    return (st == kQueued || st == kRunning) ? CULS_E_BUSY : st;
}

int Server::fetch(int64_t id, int32_t *f0, int32_t *f1, int32_t *outs, double *latencyMs) {
    std::unique_ptr<ServeJob> j;
    {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = jobs_.find(id);
        if (it == jobs_.end()) return CULS_E_NOTFOUND;
        const int st = it->second->state;
        if (st == kQueued || st == kRunning) return CULS_E_BUSY;
        j = std::move(it->second);
        jobs_.erase(it);
    }
    if (latencyMs) *latencyMs = std::chrono::duration<double, std::milli>(j->tDone - j->tSubmit).count();
    if (j->state != kDone) return j->state;
    if (f0) std::copy(j->f0.begin(), j->f0.end(), f0);
    if (f1) std::copy(j->f1.begin(), j->f1.end(), f1);
    if (outs) std::copy(j->outs.begin(), j->outs.end(), outs);
    return CULS_OK;
}

void Server::worker(Engine &eng, std::mutex &engMu) {
    cudaSetDevice(eng.device());  // the current device is per thread
    while (true) {
        std::vector<ServeJob *> batch;
        {
            std::unique_lock<std::mutex> lk(mu_);
            cvWork_.wait(lk, [&] { return stop_ || !queue_.empty(); });
            if (queue_.empty()) return;  // stop requested and nothing left
            // admission: arrival order, the head's flags, within the budget
            // (the head is always admitted; the engine refuses it if it alone
            // exceeds the context's budget)
            const ServeJob *head = jobs_[queue_.front()].get();
            size_t bytes = 0;
            std::deque<int64_t> rest;
            while (!queue_.empty()) {
                const int64_t id = queue_.front();
                queue_.pop_front();
                ServeJob *j = jobs_[id].get();
                const size_t need = kBytesPerObj * (1 + (size_t)j->nPIs + j->nAnds);
                const bool fits = batch.empty() || (bytes + need <= admit_ && (int)batch.size() < maxBatch_);
                if (j->rwFlags == head->rwFlags && j->stFlags == head->stFlags && fits) {
                    batch.push_back(j);
                    bytes += need;
                    j->state = kRunning;
                } else {
                    rest.push_back(id);
                    if (!fits) break;  // keep arrival order past a job that does not fit
                }
            }
            while (!rest.empty()) {
                queue_.push_front(rest.back());
                rest.pop_back();
            }
        }
        run_batch(eng, engMu, batch);
        cvDone_.notify_all();
    }
}

void Server::run_batch(Engine &eng, std::mutex &engMu, std::vector<ServeJob *> &batch) {
    const int n = (int)batch.size();
    std::vector<const int32_t *> f0(n), f1(n), po(n);
    std::vector<int32_t> nPIs(n), nPOs(n), nAnds(n);
    for (int i = 0; i < n; i++) {
        f0[i] = batch[i]->f0.data();
        f1[i] = batch[i]->f1.data();
        po[i] = batch[i]->outs.data();
        nPIs[i] = batch[i]->nPIs;
        nPOs[i] = batch[i]->nPOs;
        nAnds[i] = batch[i]->nAnds;
    }
    const uint32_t rwf = batch[0]->rwFlags, stf = batch[0]->stFlags;
    int rc;
    std::string why;
    {
        std::lock_guard<std::mutex> lk(engMu);
        Batch b;
        rc = eng.upload(b, n, f0.data(), f1.data(), po.data(), nPIs.data(), nPOs.data(), nAnds.data());
        if (rc == CULS_OK) {
            RwStats st{};
            rc = eng.rw(b, (rwf & CULS_RW_ZEROS) != 0, (rwf & CULS_RW_GPU_DEDUP) != 0, &st, nullptr);
        }
        if (rc == CULS_OK) rc = eng.st(b, (stf & CULS_ST_CPU) != 0);
        if (rc == CULS_OK) {
            std::vector<int32_t *> o0(n), o1(n), oo(n);
            for (int i = 0; i < n; i++) {
                const DevGraph &d = b.hg[i];
                const size_t m = 1 + (size_t)d.nPIs + d.nAnds;
                batch[i]->f0.resize(m);
                batch[i]->f1.resize(m);
                batch[i]->outs.resize(d.nPOs);
                batch[i]->nAnds = d.nAnds;
                batch[i]->nLevels = d.nLevels;
                o0[i] = batch[i]->f0.data();
                o1[i] = batch[i]->f1.data();
                oo[i] = batch[i]->outs.data();
            }
            rc = eng.download_all(b, o0.data(), o1.data(), oo.data());
        }
        if (rc != CULS_OK) why = eng.error();
    }
    const auto now = std::chrono::steady_clock::now();
    std::lock_guard<std::mutex> lk(mu_);
    if (rc != CULS_OK) err_ = why;
    for (ServeJob *j : batch) {
        j->state = rc == CULS_OK ? kDone : rc;
        j->tDone = now;
    }
}

}  // namespace culs
