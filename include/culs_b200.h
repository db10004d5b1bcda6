/*
 * culs_b200.h -- C ABI of the B200 implementation of CULS's `rw` (AIG
 * rewriting) and `st` (structural hashing with dangling-node removal).
 *
 * Every entry point takes plain pointers and sizes and returns CULS_OK (0) or
 * a negative CULS_E_* code; none of them exits the process.  The reference
 * reports through printf and calls exit() on a CUDA error
 * (CULS src/common.h:300-330).
 *
 * AIG layout (CULS AIGMan, src/aig_manager.h:51-58): objects 0..nObjs-1 with
 * nObjs = 1 + nPIs + nAnds; object 0 is the constant, objects 1..nPIs the
 * primary inputs, AND nodes follow in topological order.  A literal is
 * 2*id + complement and literal 0 is constant TRUE, literal 1 constant FALSE
 * (AIGMan convention; AIGER files use the opposite constant polarity).
 * fanin0/fanin1 are arrays of nObjs entries (entries 0..nPIs are ignored on
 * input and written as -1 on output); outs holds nPOs literals.
 */
#ifndef CULS_B200_H
#define CULS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define CULS_OK 0
#define CULS_E_INVALID (-1)  /* bad argument or malformed AIG */
#define CULS_E_OOM (-2)      /* device or host allocation failed */
#define CULS_E_BUDGET (-3)   /* request exceeds the context's HBM budget */
#define CULS_E_PROBE (-4)    /* a bounded device wait or probe hit its cap */
#define CULS_E_DEVICE (-5)   /* CUDA runtime error */
#define CULS_E_IO (-6)       /* file missing, unreadable or not binary AIGER */
#define CULS_E_BUSY (-7)     /* served job not finished yet */
#define CULS_E_NOTFOUND (-8) /* unknown job id */
#define CULS_E_CANCELLED (-9) /* served job cancelled before it ran */

/* ------------------------------------------------------- host-side graphs */
/* A graph held in host memory, arrays allocated with malloc by the library
 * (free with culs_host_graph_free). */
typedef struct culs_host_graph {
    int32_t nPIs, nPOs, nAnds;
    int32_t *fanin0, *fanin1, *outs;
} culs_host_graph;

void culs_host_graph_free(culs_host_graph *g);

/* Binary AIGER ("aig M I L O A") without latches, as
 * AIGMan::readFromMemory reads it (CULS src/aig_manager.cu:110-229). */
int culs_aiger_read(const char *path, culs_host_graph *out);
/* Writes binary AIGER as AIGMan::saveFile does (src/aig_manager.cu:231-267). */
int culs_aiger_write(const char *path, const culs_host_graph *g);

/* Seeded synthetic workloads (no reference counterpart; CULS ships no
 * benchmark inputs).  See culs_b200/csrc/host_gen.cpp for the rules. */
int culs_gen_layered(uint64_t seed, int nPIs, int nPOs, int64_t nAnds, int nLayers, int window, double pFar,
                     int withPIs, culs_host_graph *out);
int culs_gen_multiplier(int n, culs_host_graph *out);
int culs_gen_batch(uint64_t tag, int first, int count, int64_t minAnds, int64_t maxAnds, int minPIs, int maxPIs,
                   int threads, culs_host_graph *out);

/* ------------------------------------------------------ device engine */
typedef struct culs_ctx culs_ctx;     /* one GPU context: stream, library, scratch arena */
typedef struct culs_graph culs_graph; /* one or more AIGs resident in device memory */

/* flags of culs_rw: `rw -z` (fUseZeros) and `rw -d` (fGPUDeduplicate);
 * CULS_RW_DUMP records per-node intermediate results for parity checks
 * (single-graph handles only). */
#define CULS_RW_ZEROS 1u
#define CULS_RW_GPU_DEDUP 2u
#define CULS_RW_DUMP 4u
/* flag of culs_st: `st -c` (CPU strash ordering, no trivial folding) */
#define CULS_ST_CPU 1u

/* Creates a context on the current CUDA device.  hbm_budget (bytes, 0 = the
 * device's memory) bounds the scratch arena; a request above it fails with
 * CULS_E_BUDGET.  Replaces AIGMan construction (CULS src/aig_manager.cu:22-33).
 * Returns NULL on failure; culs_last_error(NULL) then explains why. */
culs_ctx *culs_create(size_t hbm_budget);
/* Selects the CUDA device that the next culs_create on this thread uses. */
int culs_set_device(int device);
void culs_destroy(culs_ctx *ctx);
const char *culs_last_error(culs_ctx *ctx);
int culs_sync(culs_ctx *ctx);

/* Copies one AIG (AIGMan layout, see above) into device memory; replaces
 * AIGMan::readFile + toDevice (src/aig_manager.cu:80-229,294-312).  The
 * caller keeps ownership of the input arrays. */
int culs_graph_upload(culs_ctx *ctx, const int32_t *fanin0, const int32_t *fanin1, const int32_t *outs, int32_t nPIs,
                      int32_t nPOs, int32_t nAnds, culs_graph **g);
/* Copies `count` AIGs into one device-resident batch. */
int culs_batch_upload(culs_ctx *ctx, int count, const culs_host_graph *graphs, culs_graph **g);
/* `count` binary AIGER files' contents (data[i], len[i] bytes) into one
 * batch: AIGMan::readFromMemory (src/aig_manager.cu:110-229, aigDecodeBinary
 * :861-869) with the header and output lines read on the host and the
 * delta-encoded AND section decoded on the device.  Accepts what
 * culs_aiger_read accepts; anything else is CULS_E_IO. */
int culs_batch_upload_aiger(culs_ctx *ctx, int count, const uint8_t *const *data, const size_t *len,
                            culs_graph **g);
/* Every graph of the handle as binary AIGER bytes, the file AIGMan::saveFile
 * writes (src/aig_manager.cu:231-267, aigEncodeBinary :871-880), the AND
 * section encoded on the device: data[i] receives a buffer of len[i] bytes
 * allocated by the library; free each with culs_buffer_free. */
int culs_batch_download_aiger(culs_ctx *ctx, const culs_graph *g, uint8_t **data, size_t *len);
void culs_buffer_free(void *p);
/* The same files back to back in one caller buffer: offsets receives
 * culs_graph_count(g) + 1 entries (file i is [offsets[i], offsets[i+1])).
 * With buf null only the offsets are written (call once for the size, then
 * with a buffer of at least offsets[count] bytes); a smaller cap is
 * CULS_E_INVALID. */
int culs_batch_download_aiger_into(culs_ctx *ctx, const culs_graph *g, uint8_t *buf, size_t cap, size_t *offsets);
void culs_graph_free(culs_graph *g);
int culs_graph_count(const culs_graph *g);
/* Sizes and level of graph `index` (AIGMan::printStats, src/aig_manager.cu:604-612). */
int culs_graph_stats(const culs_graph *g, int index, int32_t *nPIs, int32_t *nPOs, int32_t *nAnds, int32_t *nLevels);
/* culs_graph_stats for every graph of the handle at once: arrays of
 * culs_graph_count(g) entries (a null array is skipped). */
int culs_batch_stats(const culs_graph *g, int32_t *nPIs, int32_t *nPOs, int32_t *nAnds, int32_t *nLevels);
/* Copies graph `index` back (AIGMan::toHost, src/aig_manager.cu:314-336);
 * fanin arrays need 1 + nPIs + nAnds entries, outs nPOs. */
int culs_graph_download(culs_ctx *ctx, const culs_graph *g, int index, int32_t *fanin0, int32_t *fanin1,
                        int32_t *outs);

/* Copies every graph of the handle back into outs[0..count) (arrays
 * allocated by the library; free each with culs_host_graph_free). */
int culs_batch_download(culs_ctx *ctx, const culs_graph *g, culs_host_graph *outs);

/* The batch form of culs_graph_download (AIGMan::toHost for every graph of
 * the handle at once): graph i's fanins go to fanin0[i] / fanin1[i] (1 +
 * nPIs + nAnds entries each) and its POs to outs[i] (nPOs entries), arrays
 * the caller owns; a null outer pointer or a null entry skips that part.
 * One device-to-host transfer for the whole batch. */
int culs_batch_download_into(culs_ctx *ctx, const culs_graph *g, int32_t *const *fanin0, int32_t *const *fanin1,
                             int32_t *const *outs);

/* `rw` on every graph of the handle: AIGMan::rewrite(fUseZeros,
 * fGPUDeduplicate) (CULS src/aig_manager.cu:632-672, command handler
 * src/command_manager.cpp:81-95).  Without CULS_RW_GPU_DEDUP (the
 * ABC-patch `grw` default) the handle also keeps the rewrite manager's graph
 * -- every node of the rewritten graph before deduplication -- and the next
 * culs_rw on it starts from that graph, as the reference skips its Reset
 * after a rewrite (src/aig_manager.cu:654-662).  culs_st, a rewrite with
 * CULS_RW_GPU_DEDUP (whose deduplication is a strash, src/aig/strash.cu:498)
 * and writing a new graph into the handle drop it. */
int culs_rw(culs_ctx *ctx, culs_graph *g, uint32_t flags);
/* `st` on every graph of the handle: AIGMan::strash(fCPU)
 * (src/aig/strash.cu:317-503, handler src/command_manager.cpp:115-128). */
int culs_st(culs_ctx *ctx, culs_graph *g, uint32_t flags);
/* `b` on every graph of the handle: AIGMan::balance(sortDecId = 1,
 * updateLevel = true) (CULS src/aig_manager.cu:682-737 over
 * balancePerformV2, src/algorithms/balance.cu:912-1382; handler
 * src/command_manager.cpp:61-79): supergates rebuilt as balanced trees, then
 * a strash.  With CULS_B_NO_STRASH the strash is left out, as resyn2 calls
 * the balance (src/command_manager.cpp:151) -- the handle then reports the
 * graph's depth as its level.  `b -s` (sortDecId 0, a seeded shuffle of
 * equal-level inputs) is not provided: CULS_E_INVALID for any other flag.
 * Drops the rewrite manager's kept graph. */
#define CULS_B_NO_STRASH 1u
int culs_b(culs_ctx *ctx, culs_graph *g, uint32_t flags);
/* `rw; st` in one call (the rewrite-then-strash step of the reference's
 * scripts), on one graph or a whole batch. */
int culs_rw_st(culs_ctx *ctx, culs_graph *g, uint32_t rwFlags, uint32_t stFlags);

/* `rw; st` over several handles at once (each may hold one graph or a
 * batch): the handles are joined on the device, rewritten as one batch and
 * split back, each handle receiving its own graphs' results.  The batch
 * entry point of the served path; no counterpart in the reference, which
 * rewrites one AIG per process. */
int culs_rw_st_batch(culs_ctx *ctx, culs_graph *const *gs, int count, uint32_t rwFlags, uint32_t stFlags);

/* ------------------------------------------------------------ served mode
 * AIGs submitted one by one are rewritten (`rw; st`) in dynamic batches by
 * `workers` (<= 0: 2) worker threads of the context, each on an engine of its
 * own whose HBM budget is its share of the admission budget admitBytes (0:
 * the context's HBM budget), or 1 GiB if that is more, and at most the
 * context's HBM budget.  A worker, as soon as it is free,
 * takes the queued jobs in arrival order -- those with the first job's flags
 * and an AND count within 8x of its -- while their estimated device
 * footprint stays within its share and maxBatch (<= 0: no limit), runs them
 * as one batch, and holds every result until fetched.  Batches of several
 * workers overlap on the GPU, each worker on a disjoint partition of the SMs
 * (a green context) where the driver supports it: a batch waits on its
 * deepest graph while most of the GPU would sit idle.  With more than two
 * workers, the first half serve small jobs only (below 65,536 * 8^i AND
 * nodes for worker i).  Jobs and direct calls on the same context
 * never overlap on its engine.
 * No counterpart in the reference (one AIG per process invocation).
 *
 * culs_submit copies the graph (the caller may free its arrays) and returns
 * a job id.  culs_poll returns CULS_OK with the result's sizes once the job
 * is done, CULS_E_BUSY before, CULS_E_NOTFOUND for an unknown id, or the
 * job's error code.  culs_wait blocks up to timeoutMs (< 0: no limit) and
 * returns like culs_poll.  culs_fetch copies a finished result (fanin
 * arrays of 1 + nPIs + nAnds entries, nPOs outputs), reports the
 * submit-to-done latency in ms, and forgets the job.  culs_serve_stop
 * finishes every queued job, then ends the worker; results not fetched by
 * then are discarded.  Admission charges 720 device bytes per object. */
int culs_serve_start(culs_ctx *ctx, size_t admitBytes, int maxBatch, int workers);
int culs_serve_stop(culs_ctx *ctx);
int culs_submit(culs_ctx *ctx, const int32_t *fanin0, const int32_t *fanin1, const int32_t *outs, int32_t nPIs,
                int32_t nPOs, int32_t nAnds, uint32_t rwFlags, uint32_t stFlags, int64_t *job);
int culs_poll(culs_ctx *ctx, int64_t job, int32_t *nPIs, int32_t *nPOs, int32_t *nAnds, int32_t *nLevels);
int culs_wait(culs_ctx *ctx, int64_t job, int timeoutMs);
int culs_fetch(culs_ctx *ctx, int64_t job, int32_t *fanin0, int32_t *fanin1, int32_t *outs, double *latencyMs);
/* culs_cancel takes a job that is still queued out of the queue: it finishes
 * with CULS_E_CANCELLED (culs_poll, culs_wait and culs_fetch return that
 * code; culs_fetch then forgets it).  A job already in a running batch
 * completes (CULS_E_BUSY), a finished one is left as it is (CULS_E_INVALID),
 * and an unknown id gives CULS_E_NOTFOUND. */
int culs_cancel(culs_ctx *ctx, int64_t job);
/* A served job given as a binary AIGER file's bytes (copied): its header is
 * checked at once (CULS_E_IO when the host reader would refuse it), its AND
 * section decoded on the device with the rest of its batch, which holds AIGER
 * jobs only; a file whose bytes do not decode fails its own job with
 * CULS_E_IO.  culs_fetch_aiger returns the result as a binary AIGER file:
 * with buf null *len receives its size; otherwise it is copied (cap >=
 * *len) and the job forgotten.  culs_poll and culs_wait serve both kinds. */
int culs_submit_aiger(culs_ctx *ctx, const uint8_t *data, size_t len, uint32_t rwFlags, uint32_t stFlags,
                      int64_t *job);
int culs_fetch_aiger(culs_ctx *ctx, int64_t job, uint8_t *buf, size_t cap, size_t *len, double *latencyMs);

/* --------------------------------------------------------------- tuning
 * Launch and schedule parameters: they change speed only, never results.
 * CULS_PARAM_ENUM_WIDE_MIN: cut-enumeration levels with at least this many
 * AND nodes run one node per thread, narrower ones one node per warp
 * (default 16384).  CULS_PARAM_ENUM_BLOCKS_PER_SM: persistent enumeration
 * blocks per SM (default 8).  CULS_PARAM_SM_SHARE: size every grid of the
 * context for 1/value of the device's SMs (default 1), for contexts that run
 * at once on one GPU (the served workers use their share); setting it also
 * caps the enumeration blocks per SM at 4, one resident wave.
 * CULS_PARAM_HIGH_PRIORITY: 1 runs the context's work on a stream of the
 * device's highest priority, 0 (default) on a default-priority stream.
 * CULS_PARAM_EVAL_GROUP_MSLOTS: the evaluation builds and probes the
 * existence tables of groups of graphs whose tables hold at most this many
 * million slots (default 16), so that a group's tables stay in L2.
 * culs_autotune times rw's enumeration, then its evaluation, on clones of
 * `sample` (left unchanged) for candidate values, `rounds` times each, and
 * keeps the fastest in the context.  No reference counterpart. */
#define CULS_PARAM_ENUM_WIDE_MIN 1
#define CULS_PARAM_ENUM_BLOCKS_PER_SM 2
#define CULS_PARAM_SM_SHARE 4
#define CULS_PARAM_HIGH_PRIORITY 5
#define CULS_PARAM_EVAL_GROUP_MSLOTS 6
int culs_set_param(culs_ctx *ctx, int which, int64_t value);
int culs_get_param(culs_ctx *ctx, int which, int64_t *value);
int culs_autotune(culs_ctx *ctx, const culs_graph *sample, int rounds);

/* Counters of the last culs_rw (the summary CPUSolver::Rewrite prints,
 * src/algorithms/rewrite.cu:896-897,926): replaced, replaced with positive
 * gain, replaced with zero gain, reverted, compromised, without a cut, small
 * cut, without a replacement, real reduction, new nodes built, candidates;
 * then (no reference counterpart) the fanin-cut pairs the one-node-per-warp
 * cut enumeration replayed, and the rounds the deduplication's hashing took
 * to settle (0 when it ran level by level). */
int culs_rw_stats(culs_ctx *ctx, int64_t *out, int n);

/* Per-node intermediate results of the last culs_rw run with CULS_RW_DUMP,
 * indexed by the ids CPUSolver::Reorder assigns: fanin literals after the
 * reorder (AIGER constant convention), the 8 cut slots per node (9 ints:
 * used, nLeaves, leaves[4], truth table, signature, value), the selected cut
 * plus root index, replace[] after the rebuild, the rebuilt new nodes'
 * fanins, the choice-loop outcome per node.  For parity checks. */
#define CULS_DUMP_REORDER_F0 0
#define CULS_DUMP_REORDER_F1 1
#define CULS_DUMP_REORDER_OUT 2
#define CULS_DUMP_CUTS 3
#define CULS_DUMP_SELECTED 4
#define CULS_DUMP_REPLACE 5
#define CULS_DUMP_NEW_F0 6
#define CULS_DUMP_NEW_F1 7
#define CULS_DUMP_CHOICE 8
int64_t culs_dump_size(culs_ctx *ctx, int which);
int culs_dump_copy(culs_ctx *ctx, int which, int32_t *out);

/* ASAP level of every object of one AIG without allocating any memory.  No
 * counterpart in the reference: it serves callers that cannot call
 * cudaMalloc -- hosts whose device memory is owned and sized by another
 * runtime, and allocator-free embeddings that must not fragment a device
 * heap shared with other work.  d_fanin0/d_fanin1 are device pointers to the
 * AIGMan fanin arrays of one topologically ordered graph (1 + nPIs + nAnds
 * entries, constant and PIs ignored); d_levels receives one level per object
 * and d_maxLevel the depth (0 without AND nodes), both device pointers;
 * stream is a cudaStream_t (NULL = the default stream).  The call
 * synchronises that stream and reads a status word back to the host before
 * it returns: CULS_E_INVALID for a fanin that is not earlier than its node.
 * The scratch is a fixed device array of CULS_LEVELS_NOALLOC_MAX_OBJS objects
 * (about 8 MiB, held by every GPU that loads the library until exit); larger
 * graphs get CULS_E_INVALID before anything is launched.  All calls share
 * that array, so calls that overlap on the GPU race.  The first call on each
 * device looks the array's address up with that device current and should
 * come before any stream capture begins; a device reset in the same process
 * invalidates that address and is not supported.  Needs no culs_ctx. */
#define CULS_LEVELS_NOALLOC_MAX_OBJS (1 << 20)
int culs_levels_noalloc(const int32_t *d_fanin0, const int32_t *d_fanin1, int32_t nPIs, int32_t nAnds,
                        int32_t *d_levels, int32_t *d_maxLevel, void *stream);

/* Kernels this context has launched so far. */
int64_t culs_kernel_launches(culs_ctx *ctx);

/* Device copy of a handle's graphs into *dst (allocated when *dst is NULL),
 * e.g. to rerun a pass on the same input. */
int culs_graph_clone(culs_ctx *ctx, const culs_graph *src, culs_graph **dst);

/* Profiling: with profiling on, every pass records CUDA events on the
 * context's stream.  culs_mark(ctx, 0|1) records a user mark.
 * culs_profile_read fills up to n device-time intervals in ms: rw front
 * (reset/levelize/reorder), cut enumeration, evaluation, replacement,
 * choice, redundancy removal, rw's deduplication, `st`, the enumeration
 * kernel alone, the evaluation kernel alone, the last strash hashing kernel,
 * user mark 0 -> 1, the last strash level worklist kernel (-1 where an
 * interval was not recorded). */
int culs_profile(culs_ctx *ctx, int enable);
int culs_mark(culs_ctx *ctx, int slot);
int culs_profile_read(culs_ctx *ctx, float *ms, int n);

#ifdef __cplusplus
}
#endif

#endif /* CULS_B200_H */
