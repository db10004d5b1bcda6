// Served mode: AIGs submitted one by one are rewritten in dynamic batches.
//
// The reference runs one AIG per process invocation.  A server takes jobs
// (copied at submission, so the caller may free its arrays), and each of
// several worker threads, as soon as it is free, takes the queued jobs in
// arrival order -- those with the head job's flags and of a size like the
// head's, as long as their estimated device footprint stays within its share
// of the admission budget -- and runs them as one batch through its engine
// (upload, rw, st, download) under the context's lock, so served jobs and
// direct calls on the same context never overlap on the device.  Each job
// records its submit-to-done latency.
#pragma once

#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine.cuh"
#include "partition.cuh"

namespace culs {

struct ServeJob {
    int64_t id = 0;
    uint32_t rwFlags = 0, stFlags = 0;  // CULS_RW_* / CULS_ST_*
    int32_t nPIs = 0, nPOs = 0, nAnds = 0, nLevels = 0;
    std::vector<int32_t> f0, f1, outs;  // the input, replaced by the result
    bool aiger = false;                 // the job came and goes as binary AIGER bytes
    std::string file;                   // those bytes (input, replaced by the result)
    int state = 0;                      // kQueued, kRunning, kDone, or a CULS_E_* code
    std::chrono::steady_clock::time_point tSubmit, tDone;
};

class Server {
  public:
    static constexpr int kQueued = 1, kRunning = 2, kDone = 0;
    // Device bytes the admission rule charges per object of a batch (arena
    // of rw plus the graph arrays and their spares).
    static constexpr size_t kBytesPerObj = 720;
    // A batch takes only jobs whose AND count is within this factor of its
    // first job's (the batch runs as long as its deepest graph).
    static constexpr int64_t kSizeRatio = 8;
    // Workers reserved for small jobs take jobs below kSmallAnds * 8^i AND
    // nodes (worker i of the first half, when there are more than two).
    static constexpr int64_t kSmallAnds = 65536;

    // Every worker runs on an engine of the server's own (stream, arena,
    // staging) on the context's device, with its share of the admission
    // budget as HBM budget; workers' batches overlap on the GPU: a batch
    // waits on its deepest graph's critical path, during which most SMs
    // would sit idle.  With several workers each runs on a disjoint SM
    // partition of the GPU (a green context, partition.cuh), or, where the
    // driver cannot partition, sizes its grids for its share of the SMs.
    Server(Engine &eng, std::mutex &engMu, size_t admitBytes, int maxBatch, int workers = 1);
    ~Server();  // finishes every queued job, then stops the worker

    int submit(const int32_t *f0, const int32_t *f1, const int32_t *outs, int32_t nPIs, int32_t nPOs, int32_t nAnds,
               uint32_t rwFlags, uint32_t stFlags, int64_t *id);
    // A job given as a binary AIGER file's bytes; its result is fetched the
    // same way (fetch_aiger).  The header is checked here; the AND section
    // is decoded on the device with the rest of the job's batch.
    int submit_aiger(const uint8_t *data, size_t len, uint32_t rwFlags, uint32_t stFlags, int64_t *id);
    // With buf null *len receives the result's size; otherwise the result
    // (at most cap bytes) is copied and the job forgotten.
    int fetch_aiger(int64_t id, uint8_t *buf, size_t cap, size_t *len, double *latencyMs);
    // CULS_OK with the result's sizes when done, CULS_E_BUSY while queued or
    // running, CULS_E_NOTFOUND for an unknown id, or the job's error code.
    int poll(int64_t id, int32_t *nPIs, int32_t *nPOs, int32_t *nAnds, int32_t *nLevels);
    // Waits up to timeoutMs (< 0: without limit) for the job to finish.
    int wait(int64_t id, int timeoutMs);
    // Copies a finished job's result out and forgets the job.
    int fetch(int64_t id, int32_t *f0, int32_t *f1, int32_t *outs, double *latencyMs);
    // Takes a queued job out of the queue; it finishes with CULS_E_CANCELLED.
    int cancel(int64_t id);
    const std::string &lastError() const { return err_; }

  private:
    void worker(Engine &eng, std::mutex &engMu, int64_t maxAnds);
    void run_batch(Engine &eng, std::mutex &engMu, std::vector<ServeJob *> &batch);
    void run_aiger(Engine &eng, std::mutex &engMu, std::vector<ServeJob *> &batch);

    Engine &eng_;
    std::mutex &engMu_;
    std::vector<SmPartition> parts_;             // the workers' SM partitions (empty: shared SMs)
    std::vector<std::unique_ptr<Engine>> own_;  // the workers' engines
    std::vector<std::unique_ptr<std::mutex>> ownMu_;
    std::vector<std::thread> extra_;
    size_t admit_;
    int maxBatch_;
    std::mutex mu_;
    std::condition_variable cvWork_, cvDone_;
    std::deque<int64_t> queue_;
    std::unordered_map<int64_t, std::unique_ptr<ServeJob>> jobs_;
    int64_t nextId_ = 1;
    bool stop_ = false;
    std::string err_;
    std::thread th_;
};

}  // namespace culs
