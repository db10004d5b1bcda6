// Batch engine: many AIGs resident on one GPU, rewritten (`rw`) and strashed
// (`st`) together by the same kernels.
//
// At rest a batch stores its graphs one after another ("graph-major"): graph
// g owns positions base_g .. base_g + nObjs_g - 1 and keeps the AIGMan arrays
// of CULS (src/aig_manager.h:51-58) with graph-local literals: F0/F1 hold
// 2*localId + complement with literal 0 = constant TRUE (-1 for the constant
// and the PIs), POs hold local literals.  A single graph is a batch of one.
#pragma once

#include <algorithm>

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "culs_b200.h"
#include "prim.cuh"
#include "rw_core.cuh"

namespace culs {

struct ExecCtx;

// Launch and schedule parameters that do not change results, only speed
// (set by culs_set_param or culs_autotune).
struct Tune {
    int enumWideMin = 16384;   // levels this wide run one node per thread, narrower one per warp
    int enumBlocksPerSm = 8;   // persistent enumeration blocks per SM
    int evalGroupMSlots = 16;  // existence-table slots (millions) of a group of graphs built and evaluated together
};

struct DevGraph {
    int nPIs, nPOs, nAnds, nLevels;
    int base;   // first position of this graph in graph-major arrays
    int poOff;  // first PO of this graph in the PO array
    int cpos;   // position of the constant node in the current working layout
    int pad;
};

// Counters reported by the choice loop (CULS src/algorithms/rewrite.cu:849-897)
struct RwStats {
    long long replaced, replacedPos, replacedZero, reverted, compromised, preEval, smallCut, newIdx, expected,
        newNodes, candidates;
    long long warpPairs;  // fanin-cut pairs the one-node-per-warp enumeration replayed
    long long hashRounds; // rounds of the deduplication's hashing (0: the level dataflow)
};

// Device blocks freed by batches, kept for the next batch of a context (a
// served loop or a benchmark uploads batches of similar size again and
// again).  Shared by the engine and every batch it filled, so it outlives
// whichever goes first; cached bytes are bounded.
class DevPool {
  public:
    explicit DevPool(size_t limitBytes) : limit_(limitBytes) {}
    ~DevPool();
    // A block of at least `bytes` (the smallest cached one up to twice that
    // size, else a new allocation); *got receives its size.
    void *take(size_t bytes, size_t *got);
    void give(void *p, size_t bytes);  // caches the block, or frees it beyond the limit
    void flush();                      // frees every cached block

  private:
    std::mutex mu_;
    std::multimap<size_t, void *> free_;
    size_t cached_ = 0, limit_;
};

struct Batch {
    int G = 0;
    int64_t nObj = 0, nPO = 0;
    std::vector<DevGraph> hg;  // host copy of the graph table
    DevGraph *dg = nullptr;
    int *F0 = nullptr, *F1 = nullptr, *PO = nullptr;  // graph-local literals
    int64_t capObj = 0, capPO = 0;
    int capG = 0;
    // spare fanin/PO buffers: strash writes its output there and swaps
    int *F0s = nullptr, *F1s = nullptr, *POs = nullptr;
    int64_t capObjS = 0, capPOS = 0;
    // The rewrite manager's graph left by a rewrite with CPU deduplication
    // (AIGMan::prevCmdRewrite, src/aig_manager.cu:654-662): every node of the
    // rewritten graph in the manager's numbering, duplicates and dangling
    // nodes included.  The next rewrite starts from it instead of from the
    // deduplicated graph; a strash -- st, or a rewrite's GPU deduplication --
    // drops it (src/aig/strash.cu:498).
    bool keep = false;
    int *F0k = nullptr, *F1k = nullptr, *POk = nullptr;
    int64_t capObjK = 0, capPOK = 0, nObjK = 0;
    std::vector<DevGraph> hgk;
    std::shared_ptr<DevPool> pool;  // where the buffers come from and go back to (null: cudaMalloc)
    ~Batch();
    void release();
    // Grows the buffers to hold nObj objects, nPO POs and G graphs (their
    // contents are not kept, nor is the kept rewrite state); allocates
    // nothing when they are large enough.
    cudaError_t reserve(int64_t nObj, int64_t nPO, int G);
    cudaError_t reserve_spare(int64_t nObj, int64_t nPO);
    void swap_spare();
    // Objects per level summed over the graphs (+1): the number of nodes a
    // level-ordered dataflow pass over the batch can work on at once.
    int64_t flow_width() const {
        int64_t w = 1;
        for (const DevGraph &g : hg) w += (1 + (int64_t)g.nPIs + g.nAnds) / ((int64_t)g.nLevels + 1);
        return w;
    }
    // Copies the current graph into the kept buffers and sets keep.
    cudaError_t keep_current(cudaStream_t s);
    // Makes the kept graph current (the current one is discarded) and clears
    // keep; the caller uploads hg to dg.
    void restore_kept();
};

// Per-node dumps of the last rw (for parity checks); indexed by the graph's
// reordered local id (the numbering rw::CPUSolver::Reorder produces).
struct RwDump {
    bool enabled = false;
    // for graph 0 of the batch only
    std::vector<int> reorderF0, reorderF1, reorderOut;  // AIGER convention, local ids
    std::vector<int> cuts;                              // (n+1)*8*9
    std::vector<int> selected;                          // (n+1)*10
    std::vector<int> replace, newF0, newF1;             // local ids, rebuilt numbering
    std::vector<int> choice;                            // per node outcome code
};

// CUDA-event marks recorded on the engine stream when profiling is on.
enum Mark : int {
    kMkRwStart = 0,
    kMkFront,
    kMkEnum,
    kMkEval,
    kMkReplace,
    kMkChoice,
    kMkRedund,
    kMkRwEnd,
    kMkStStart,
    kMkStEnd,
    kMkEnumK0,
    kMkEnumK1,
    kMkEvalK0,
    kMkEvalK1,
    kMkDedupK0,
    kMkDedupK1,
    kMkUser0,
    kMkUser1,
    kMkLevelK0,
    kMkLevelK1,
    kNumMarks
};

class Engine {
  public:
    Engine();
    ~Engine();
    int init(size_t hbmBudget);  // loads the library, creates the stream
    const std::string &error() const { return err_; }

    int upload(Batch &b, int count, const int32_t *const *f0, const int32_t *const *f1, const int32_t *const *outs,
               const int32_t *nPIs, const int32_t *nPOs, const int32_t *nAnds);
    int download(const Batch &b, int g, int32_t *f0, int32_t *f1, int32_t *outs);
    // Whole-batch download into caller arrays (graph i's fanins into f0[i],
    // f1[i], its POs into outs[i]); a null array pointer skips that part.
    int download_all(const Batch &b, int32_t *const *f0, int32_t *const *f1, int32_t *const *outs);
    // Binary AIGER files' bytes in, decoded on the device (aiger_dev.cu).
    int upload_aiger(Batch &b, int count, const uint8_t *const *data, const size_t *len);
    // Every graph as a binary AIGER file's bytes, encoded on the device,
    // the files back to back in buf: offsets[0..G] (file g is
    // [offsets[g], offsets[g+1])).  With buf null only the offsets are set.
    int download_aiger(const Batch &b, uint8_t *buf, size_t cap, size_t *offsets);
    // Sets every graph's nLevels to its depth (AIGMan::readFromMemory).
    int batch_depth(Batch &b);
    int rw(Batch &b, bool useZeros, bool gpuDedup, RwStats *stats, RwDump *dump);
    int st(Batch &b, bool cpuOrder);
    // AIG balancing (`b`, sortDecId 1) of every graph of b, then a strash
    // when updateLevel (balance.cu).
    int balance(Batch &b, bool updateLevel);
    int sync();

    cudaStream_t stream() const { return s_; }
    size_t budget() const { return budget_; }
    int device() const { return device_; }  // the CUDA device the engine lives on
    // Sizes every grid of this engine for 1/share of the device's SMs, so
    // that `share` engines running at once (the served workers) overlap on
    // the GPU instead of queueing behind one another's persistent kernels.
    // Persistent kernels get one resident wave of blocks on that share (the
    // enumeration's blocks fit 4 to an SM).
    void set_sm_share(int share) {
        share_ = std::max(1, share);
        sms_ = std::max(8, num_sms() / share_);
        if (share_ > 1) tune_.enumBlocksPerSm = std::min(tune_.enumBlocksPerSm, 4);
    }
    int sm_share() const { return share_; }
    // Recreates the engine's stream at the device's highest stream priority
    // (high) or the default one: the block scheduler then starts this
    // engine's blocks before pending blocks of lower-priority streams.  Only
    // between calls (the stream is drained first).
    int set_high_priority(bool high);
    // Runs the engine's work on stream s, owned by the caller (a stream of
    // an SM partition of `sms` SMs, partition.cuh), with every grid sized for
    // those SMs.  Only between calls.
    int adopt_stream(cudaStream_t s, int sms);
    bool high_priority() const { return highPrio_; }
    // Grows the scratch arena and the pinned staging up front for batches of
    // up to nObj objects, so that serving them needs no allocation (freeing
    // device or pinned memory synchronises the whole device, stalling every
    // other engine's work).
    int prepare(int64_t nObj);
    size_t arenaHighWater() const { return ar_.high_water(); }
    int kernelLaunches() const { return launches_; }
    void setProfile(bool on) { prof_ = on; }
    void mark(int m);
    float elapsed(int a, int b);  // ms between two recorded marks (-1 if missing)
    int clone(const Batch &src, Batch &dst);
    // dst = the graphs of parts[0], parts[1], ... in order (device copies).
    int concat(const std::vector<const Batch *> &parts, Batch &dst);
    // Inverse of concat: parts[i] receives its graphs back from src.
    int split(const Batch &src, const std::vector<Batch *> &parts);
    void resetLaunchCount() { launches_ = 0; }
    Tune &tune() { return tune_; }
    // Times rw's enumeration on clones of `sample` for each candidate
    // schedule and keeps the fastest; `rounds` timings per candidate.
    int autotune(const Batch &sample, int rounds);

  private:
    int fail(int code, const std::string &msg);
    int check(cudaError_t e, const char *what);
    int check_status(const char *what);
    int ensure_arena(size_t bytes);
    int ensure_stage(size_t ints);  // pinned host staging of at least `ints` int32
    ExecCtx ctx();
    int balance_graph(const int *F0, const int *F1, const int *PO, int nPIs, int nPO, int nObj, int *F0n, int *F1n,
                      int *POn, int *nAndsOut);
    void apply_spin_limit();

    // stage helpers
    // Strash over M positions: L0/L1 are AIGMan-convention literals over
    // positions (L0 < 0 marks the constant and PIs), gid/lid give each
    // position's graph and local id (lid is read for the constant and PIs
    // only), po the PO literals over positions.  b.dg[g].cpos must hold each
    // graph's constant position.  Replaces b's arrays with the result.
    // topo: positions are topological and b's graph-major layout (levels by
    // an in-order dataflow instead of a worklist).
    // unique: every node is its own representative (no duplicate merged):
    // the output is the input graph renumbered in processing order.
    // procInv / procPos (not topo): an order of the positions that is
    // topological up to a few fanins placed later (procInv[k] = position at
    // order index k, procPos its inverse); levels then come from in-order
    // passes instead of the level-synchronous worklist.
    int strash_core(Batch &b, int64_t M, const int *L0, const int *L1, const int *gid, const int *lid, const int *po,
                    bool idOrder, bool removeDangling, bool foldTrivial, bool topo, bool unique = false,
                    const int *procInv = nullptr, const int *procPos = nullptr);
    // strash_core over b's own graph-major arrays (the body of st).
    int strash_batch(Batch &b, bool idOrder, bool removeDangling, bool foldTrivial);
    // rounds the last strash_core's hashing took to settle; 0 when it ran
    // as the level dataflow (by size, by CULS_DEDUP_MODE, or because the
    // rounds did not settle)
    int hashRounds_ = 0;

    std::string err_;
    cudaStream_t s_ = nullptr;
    RwLib *lib_ = nullptr;
    int *status_ = nullptr;     // device status word and spin bound (2 ints)
    int spinLimit_ = 0;         // the bound last written to status_[1]
    int *counters_ = nullptr;   // device scratch counters
    int *hostSmall_ = nullptr;  // pinned host scratch
    int32_t *stage_ = nullptr;  // pinned staging for uploads and downloads
    size_t stageCap_ = 0;       // in int32
    size_t budget_ = 0;
    int device_ = 0;
    Arena ar_;
    int launches_ = 0;
    int sms_ = 148;
    int share_ = 1;
    bool highPrio_ = false;
    bool ownStream_ = true;  // s_ was created by this engine
    bool prof_ = false;
    Tune tune_;
    std::shared_ptr<DevPool> pool_;
    cudaEvent_t ev_[kNumMarks] = {};
    bool evSet_[kNumMarks] = {};
};

}  // namespace culs
