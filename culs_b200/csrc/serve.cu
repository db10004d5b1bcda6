// Served mode (serve.cuh).
#include <algorithm>
#include <climits>
#include <cstring>

#include "guard.hpp"
#include "serve.cuh"

namespace culs {

Server::Server(Engine &eng, std::mutex &engMu, size_t admitBytes, int maxBatch, int workers)
    : eng_(eng), engMu_(engMu), maxBatch_(maxBatch > 0 ? maxBatch : 1 << 20) {
    workers = workers < 1 ? 1 : workers;
    admit_ = admitBytes / (size_t)workers;  // every worker's batch within its share
    // every worker has an engine of its own (stream, arena, staging) whose
    // HBM budget is its share of the admission budget (at least 1 GiB, room
    // for the arena's fixed part, and never more than the context's budget),
    // so the workers together stay near it whatever the context's own engine
    // holds
    const size_t engBudget = std::min<size_t>(eng.budget(), std::max<size_t>(admit_, (size_t)1 << 30));
    if (workers > 1 && !make_sm_partitions(eng.device(), workers, parts_, nullptr)) parts_.clear();
    for (int w = 0; w < workers; w++) {
        auto e = std::make_unique<Engine>();
        if (e->init(engBudget) != CULS_OK) break;  // fewer workers
        if (!parts_.empty()) {
            if (e->adopt_stream(parts_[w].stream, parts_[w].sms) != CULS_OK) break;
        } else {
            e->set_sm_share(workers);
        }
        // room for a typical batch (at most 16M objects within the share) up
        // front: growing it later would synchronise the whole device
        e->prepare(std::min<int64_t>((int64_t)(engBudget / kBytesPerObj), (int64_t)16 << 20));
        own_.push_back(std::move(e));
        ownMu_.push_back(std::make_unique<std::mutex>());
    }
    if (own_.empty()) {  // no room for an engine of its own: the context's
        th_ = std::thread([this] { worker(eng_, engMu_, INT64_MAX); });
        return;
    }
    // the first half of the workers (those beyond two) serve small jobs
    // only: a worker i < n/2 takes jobs below kSmallAnds * 8^i AND nodes, the
    // others take any job.  Small jobs then never wait behind a batch that
    // runs for a large graph's critical path.
    const int n = (int)own_.size();
    for (int i = 0; i < n; i++) {
        Engine *e = own_[i].get();
        std::mutex *m = ownMu_[i].get();
        const int64_t cap = (n > 2 && i < n / 2) ? kSmallAnds << (3 * i) : INT64_MAX;
        extra_.emplace_back([this, e, m, cap] { worker(*e, *m, cap); });
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
    own_.clear();  // the engines, before the partitions their streams belong to
    destroy_sm_partitions(parts_);
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
    cvWork_.notify_all();  // workers take different jobs
    return CULS_OK;
}

// The header fields of a binary AIGER file ("aig M I L O A"), as the host
// reader checks them (host_aiger.cpp): the job's sizes for admission.
static bool aiger_sizes(const uint8_t *p, size_t len, int32_t &nPIs, int32_t &nPOs, int32_t &nAnds) {
    const uint8_t *end = p + len;
    if (len < 4 || memcmp(p, "aig ", 4) != 0) return false;
    p += 4;
    long long v[5];
    for (int k = 0; k < 5; k++) {
        if (p >= end || *p < '0' || *p > '9') return false;
        long long x = 0;
        while (p < end && *p >= '0' && *p <= '9') {
            x = x * 10 + (*p++ - '0');
            if (x > INT32_MAX) return false;
        }
        if (p >= end || *p++ != (k < 4 ? ' ' : '\n')) return false;
        v[k] = x;
    }
    if (v[2] != 0 || v[0] != v[1] + v[4] || v[0] + 1 > INT32_MAX / 2) return false;
    nPIs = (int32_t)v[1];
    nPOs = (int32_t)v[3];
    nAnds = (int32_t)v[4];
    return true;
}

int Server::submit_aiger(const uint8_t *data, size_t len, uint32_t rwFlags, uint32_t stFlags, int64_t *id) {
    if (!id || !data) return CULS_E_INVALID;
    auto job = std::make_unique<ServeJob>();
    if (!aiger_sizes(data, len, job->nPIs, job->nPOs, job->nAnds)) return CULS_E_IO;
    job->rwFlags = rwFlags;
    job->stFlags = stFlags;
    job->aiger = true;
    job->file.assign(reinterpret_cast<const char *>(data), len);
    job->state = kQueued;
    job->tSubmit = std::chrono::steady_clock::now();
    {
        std::lock_guard<std::mutex> lk(mu_);
        job->id = nextId_++;
        *id = job->id;
        queue_.push_back(job->id);
        jobs_[job->id] = std::move(job);
    }
    cvWork_.notify_all();  // workers take different jobs
    return CULS_OK;
}

int Server::fetch_aiger(int64_t id, uint8_t *buf, size_t cap, size_t *len, double *latencyMs) {
    if (!len) return CULS_E_INVALID;
    std::unique_ptr<ServeJob> j;
    {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = jobs_.find(id);
        if (it == jobs_.end()) return CULS_E_NOTFOUND;
        const int st = it->second->state;
        if (st == kQueued || st == kRunning) return CULS_E_BUSY;
        if (!it->second->aiger) return CULS_E_INVALID;  // fetched with culs_fetch
        if (st == kDone) {
            *len = it->second->file.size();
            if (!buf) return CULS_OK;
            if (cap < *len) return CULS_E_INVALID;
        }
        j = std::move(it->second);
        jobs_.erase(it);
    }
    if (latencyMs) *latencyMs = std::chrono::duration<double, std::milli>(j->tDone - j->tSubmit).count();
    if (j->state != kDone) return j->state;
    memcpy(buf, j->file.data(), j->file.size());
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
        if (it->second->aiger) return CULS_E_INVALID;  // fetched with culs_fetch_aiger
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

int Server::cancel(int64_t id) {
    {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = jobs_.find(id);
        if (it == jobs_.end()) return CULS_E_NOTFOUND;
        ServeJob &j = *it->second;
        if (j.state == kRunning) return CULS_E_BUSY;
        if (j.state != kQueued) return CULS_E_INVALID;
        queue_.erase(std::find(queue_.begin(), queue_.end(), id));
        j.state = CULS_E_CANCELLED;
        j.tDone = std::chrono::steady_clock::now();
    }
    cvDone_.notify_all();
    return CULS_OK;
}

void Server::worker(Engine &eng, std::mutex &engMu, int64_t maxAnds) {
    cudaSetDevice(eng.device());  // the current device is per thread
    // the first queued job this worker takes (below maxAnds AND nodes)
    auto first = [&]() -> std::deque<int64_t>::iterator {
        for (auto it = queue_.begin(); it != queue_.end(); ++it)
            if (jobs_[*it]->nAnds < maxAnds) return it;
        return queue_.end();
    };
    while (true) {
        std::vector<ServeJob *> batch;
        {
            std::unique_lock<std::mutex> lk(mu_);
            cvWork_.wait(lk, [&] { return first() != queue_.end() || (stop_ && queue_.empty()); });
            if (queue_.empty()) return;  // stop requested and nothing left
            // the jobs before the first one this worker takes stay queued,
            // in order, for the other workers
            std::deque<int64_t> skipped(queue_.begin(), first());
            queue_.erase(queue_.begin(), first());
            // admission: arrival order, the head's flags and size class,
            // within the budget (the head is always admitted; the engine
            // refuses it if it alone exceeds the context's budget).  A batch
            // lasts as long as its deepest graph, and depth grows with size,
            // so a batch takes only jobs within kSizeRatio of the head's AND
            // count: small jobs then do not wait on a large one's critical
            // path, and the jobs left in the queue go to the next free worker.
            const ServeJob *head = jobs_[queue_.front()].get();
            const int64_t hs = 1 + (int64_t)head->nAnds;
            size_t bytes = 0;
            std::deque<int64_t> rest;
            while (!queue_.empty()) {
                const int64_t id = queue_.front();
                queue_.pop_front();
                ServeJob *j = jobs_[id].get();
                const size_t need = kBytesPerObj * (1 + (size_t)j->nPIs + j->nAnds);
                const bool fits = batch.empty() || (bytes + need <= admit_ && (int)batch.size() < maxBatch_);
                const int64_t js = 1 + (int64_t)j->nAnds;
                const bool alike = js <= hs * kSizeRatio && hs <= js * kSizeRatio && j->nAnds < maxAnds;
                if (j->rwFlags == head->rwFlags && j->stFlags == head->stFlags && j->aiger == head->aiger && fits &&
                    alike) {
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
            while (!skipped.empty()) {
                queue_.push_front(skipped.back());
                skipped.pop_back();
            }
        }
        // jobs this worker left to the others, or an emptied queue that
        // workers waiting to stop must see
        cvWork_.notify_all();
        // a host exception (an allocation) fails the batch's jobs, not the
        // worker thread and with it the process
        const int rc = guard_call(nullptr, [&]() -> int {
            run_batch(eng, engMu, batch);
            return CULS_OK;
        });
        if (rc != CULS_OK) {
            std::lock_guard<std::mutex> lk(mu_);
            const auto now = std::chrono::steady_clock::now();
            for (ServeJob *j : batch)
                if (j->state == kRunning) {
                    j->state = rc;
                    j->tDone = now;
                }
        }
        cvDone_.notify_all();
    }
}

// A batch of AIGER jobs: decoded on the device together; when the batch's
// bytes do not decode, every job is tried alone, so that a malformed file
// fails its own job only.  Results are encoded on the device.
void Server::run_aiger(Engine &eng, std::mutex &engMu, std::vector<ServeJob *> &batch) {
    std::vector<std::pair<ServeJob *, int>> failed;
    std::vector<ServeJob *> run = batch;
    int rc;
    std::string why;
    {
        std::lock_guard<std::mutex> lk(engMu);
        auto upload = [&](Batch &b, const std::vector<ServeJob *> &js) {
            std::vector<const uint8_t *> data(js.size());
            std::vector<size_t> len(js.size());
            for (size_t i = 0; i < js.size(); i++) {
                data[i] = reinterpret_cast<const uint8_t *>(js[i]->file.data());
                len[i] = js[i]->file.size();
            }
            return eng.upload_aiger(b, (int)js.size(), data.data(), len.data());
        };
        Batch b;
        rc = upload(b, run);
        if (rc == CULS_E_IO && run.size() > 1) {
            std::vector<ServeJob *> good;
            for (ServeJob *j : run) {
                Batch one;
                const int r = upload(one, std::vector<ServeJob *>{j});
                if (r == CULS_OK)
                    good.push_back(j);
                else
                    failed.emplace_back(j, r);
            }
            run = good;
            rc = run.empty() ? CULS_OK : upload(b, run);
        }
        if (rc == CULS_OK && !run.empty()) {
            const uint32_t rwf = run[0]->rwFlags, stf = run[0]->stFlags;
            RwStats st{};
            rc = eng.rw(b, (rwf & CULS_RW_ZEROS) != 0, (rwf & CULS_RW_GPU_DEDUP) != 0, &st, nullptr);
            if (rc == CULS_OK) rc = eng.st(b, (stf & CULS_ST_CPU) != 0);
            std::vector<size_t> off(run.size() + 1);
            if (rc == CULS_OK) rc = eng.download_aiger(b, nullptr, 0, off.data());
            std::string all;
            if (rc == CULS_OK) {
                all.resize(off[run.size()]);
                rc = eng.download_aiger(b, reinterpret_cast<uint8_t *>(&all[0]), all.size(), off.data());
            }
            if (rc == CULS_OK)
                for (size_t i = 0; i < run.size(); i++) {
                    const DevGraph &d = b.hg[i];
                    run[i]->file.assign(all, off[i], off[i + 1] - off[i]);
                    run[i]->nPIs = d.nPIs;
                    run[i]->nPOs = d.nPOs;
                    run[i]->nAnds = d.nAnds;
                    run[i]->nLevels = d.nLevels;
                }
        }
        if (rc != CULS_OK || !failed.empty()) why = eng.error();
    }
    const auto now = std::chrono::steady_clock::now();
    std::lock_guard<std::mutex> lk(mu_);
    if (rc != CULS_OK || !failed.empty()) err_ = why;
    for (ServeJob *j : run) {
        j->state = rc == CULS_OK ? kDone : rc;
        j->tDone = now;
    }
    for (auto &f : failed) {
        f.first->state = f.second;
        f.first->tDone = now;
    }
}

void Server::run_batch(Engine &eng, std::mutex &engMu, std::vector<ServeJob *> &batch) {
    if (batch[0]->aiger) {
        run_aiger(eng, engMu, batch);
        return;
    }
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
    bool written = false;  // the jobs' arrays hold (part of) the results
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
            written = true;
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
    if (rc != CULS_OK && n > 1 && !written && rc != CULS_E_DEVICE) {
        // one job's failure (a malformed graph, a cap) stays its own: each
        // job runs again alone
        for (ServeJob *j : batch) {
            std::vector<ServeJob *> one{j};
            run_batch(eng, engMu, one);
        }
        return;
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
