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

#ifdef __cplusplus
}
#endif

#endif /* CULS_B200_H */
