// Conflict-free replacement and redundancy removal: the sequential choice
// loop of rw::CPUSolver::Rewrite (CULS src/algorithms/rewrite.cu:830-921,
// rewrite.h:118-124,208-220) moved onto the GPU.
//
// Choice: one thread per graph walks that graph's candidates in id order and
// replays FastDelete with an explicit stack that follows the reference's
// recursion step by step (its order of reference-count updates matters when
// a cone reaches a node along two paths: a node can be deleted twice) and
// install with a worklist (its outcome does not depend on the order).  The walk is
// a chain of dependent memory accesses, so it is written to shorten that
// chain: each candidate's record (node, replacement, cut leaves) is gathered
// beforehand in graph order and read one candidate ahead; the loads a
// candidate needs before its first store are issued together; a traversal
// frame carries its node's two fanins, the top frame lives in registers and
// the next ones in shared memory; reference-count updates whose old value is
// not needed are fire-and-forget atomics (a thread's own later loads of the
// same word observe them).  A single graph of up to 65,536 objects runs on a
// thread-block cluster instead, with its arrays in the blocks' distributed
// shared memory (k_choice_cluster).
//
// Redundancy removal chases buffer chains.  The reference does it in one
// sequential sweep in which a node's fanins, once rewritten, can make it
// redundant for later nodes only.  Here every node computes its chased fanins
// in parallel, judging each node it passes "as of its own id"; the sweep is
// repeated until nothing changes, which reproduces the sequential result
// because a node's outcome depends only on nodes with smaller ids.
#include <algorithm>
#include <climits>
#include <cstdlib>

#include <cooperative_groups.h>

#include "rw_work.cuh"

namespace cg = cooperative_groups;

namespace culs {

namespace {

constexpr int kChoiceBlock = 32;   // graphs per block, one thread each
constexpr int kChoiceFrames = 64;  // frames per graph held in shared memory

struct ChoiceArgs {
    int64_t nL0;  // W positions [0, nL0) are constants and PIs
    const DevGraph *dg;
    int *L0, *L1, *ref;
    uint8_t *del;
    const int4 *recA, *recB;  // per candidate in graph order: {c, q, rep, -}, leaves
    const int *gStart, *gCount;
    int useZeros;
    int4 *stack;
    int stackCap;
    int *choice;
    unsigned long long *stats;  // replaced, pos, zero, reverted, compromised, newIdx, selfRef, expected
    int *status;
};

// The graph arrays the walk reads and writes.  GlobalMem: the arrays in HBM
// (one thread per graph of a batch).  ClusterMem: for a single graph small
// enough, the same arrays copied into the distributed shared memory of a
// thread-block cluster, object x at offset x & mask of block x >> shift, so
// that every access of the walk's dependent chain is a shared-memory access
// of this SM or a neighbour instead of an L2 round trip.  Only one thread
// walks, so the reference-count updates need no atomicity there; they stay
// atomics because a fire-and-forget `red` does not stall the thread.
struct GlobalMem {
    int *L0, *L1, *ref;
    uint8_t *del;
    __device__ __forceinline__ int l0(int x) const { return L0[x]; }
    __device__ __forceinline__ int l1(int x) const { return L1[x]; }
    __device__ __forceinline__ int dl(int x) const { return del[x]; }
    __device__ __forceinline__ int rf(int x) const { return ref[x]; }
    __device__ __forceinline__ void set_del(int x, int v) const { del[x] = (uint8_t)v; }
    __device__ __forceinline__ void set_fanins(int x, int a, int b) const {
        L0[x] = a;
        L1[x] = b;
    }
    __device__ __forceinline__ void rf_add(int x, int d) const { atomicAdd(ref + x, d); }
    __device__ __forceinline__ int rf_add_old(int x, int d) const { return atomicAdd(ref + x, d); }
    // del (or ref) and both fanins of x
    __device__ __forceinline__ void dab(int x, int &d, int &a, int &b) const {
        d = del[x];
        a = L0[x];
        b = L1[x];
    }
    __device__ __forceinline__ void rab(int x, int &r, int &a, int &b) const {
        r = ref[x];
        a = L0[x];
        b = L1[x];
    }
    __device__ __forceinline__ void ab(int x, int &a, int &b) const {
        a = L0[x];
        b = L1[x];
    }
    static constexpr bool kPrefetch = true;
};

struct ClusterMem {
    int4 *rec;  // this block's slice of {L0, L1, ref, del}; every block of the cluster has it at the same offset
    int shift, mask;
    __device__ __forceinline__ int4 *at(int x) const {
        return cg::this_cluster().map_shared_rank(rec + (x & mask), (unsigned)(x >> shift));
    }
    __device__ __forceinline__ int l0(int x) const { return at(x)->x; }
    __device__ __forceinline__ int l1(int x) const { return at(x)->y; }
    __device__ __forceinline__ int dl(int x) const { return at(x)->w; }
    __device__ __forceinline__ int rf(int x) const { return at(x)->z; }
    __device__ __forceinline__ void set_del(int x, int v) const { at(x)->w = v; }
    __device__ __forceinline__ void set_fanins(int x, int a, int b) const {
        *reinterpret_cast<int2 *>(at(x)) = make_int2(a, b);
    }
    __device__ __forceinline__ void rf_add(int x, int d) const { atomicAdd(&at(x)->z, d); }
    __device__ __forceinline__ int rf_add_old(int x, int d) const { return atomicAdd(&at(x)->z, d); }
    __device__ __forceinline__ void dab(int x, int &d, int &a, int &b) const {
        const int4 r = *at(x);
        d = r.w;
        a = r.x;
        b = r.y;
    }
    __device__ __forceinline__ void rab(int x, int &f, int &a, int &b) const {
        const int4 r = *at(x);
        f = r.z;
        a = r.x;
        b = r.y;
    }
    __device__ __forceinline__ void ab(int x, int &a, int &b) const {
        const int2 r = *reinterpret_cast<const int2 *>(at(x));
        a = r.x;
        b = r.y;
    }
    static constexpr bool kPrefetch = false;
};

// Stack frames: FastDelete's {node, step | count << 2, fanin0 literal,
// fanin1 literal}, install's {node, fanin0 literal, fanin1 literal, 0};
// frames below kChoiceFrames in shared memory (sh[sp * stride]), deeper ones
// in the graph's global stack.  The scalars the walk reads at every node are copies held here: read
// through the argument block, they would be reloaded after every store the
// compiler cannot tell apart from it.
template <class Mem>
struct GraphCtx {
    const ChoiceArgs *A;
    Mem m;
    int trueLit;
    int4 *sh;
    int stride;
    int4 *stk;
    int64_t nL0;
    int stackCap;
    int *status;
    __device__ __forceinline__ void push(int sp, int4 f) const {
        if (sp < kChoiceFrames)
            sh[sp * stride] = f;
        else
            stk[sp] = f;
    }
    __device__ __forceinline__ int4 pop(int sp) const { return sp < kChoiceFrames ? sh[sp * stride] : stk[sp]; }
};

template <class Mem>
__device__ __forceinline__ int ch_red(const GraphCtx<Mem> &C, int x, int l0, int l1) {
    return x >= C.nL0 && (l0 == l1 || l0 == C.trueLit);
}

// A pushed FastDelete frame's two fanins are read together: their (ref, L0,
// L1).  L0 and L1 do not change during FastDelete, and the ref of the second
// fanin changes only inside the first fanin's subtree, so the second fanin
// is read again only when its frame resumes after that subtree.

// install lambda, rewrite.cu:835-847; rootDel, r0, r1 = del, L0, L1 of root.
// Whether a node is installed depends only on the deletion flags, which the
// walk clears as it reaches nodes, and install reads no reference count, so
// every visiting order installs the same nodes, makes the same increments
// and returns the same count: a worklist (a node's deleted fanins are
// cleared and queued when the node is taken) instead of the recursion.
template <class Mem>
__device__ int ch_install(const GraphCtx<Mem> &C, int root, int rootDel, int r0, int r1) {
    const Mem &m = C.m;
    if (!rootDel) return 0;
    m.set_del(root, 0);
    int cnt = 0, sp = 0;
    int x = root, l0 = r0, l1 = r1;
    while (true) {
        cnt += 1 - ch_red(C, x, l0, l1);
        const int c0 = l0 >> 1, c1 = l1 >> 1;
        int d0, a0, b0, d1, a1, b1;
        m.dab(c0, d0, a0, b0);
        m.dab(c1, d1, a1, b1);
        m.rf_add(c0, 1);
        m.rf_add(c1, 1);
        if (d1 && c1 != c0) {
            if (sp + 1 >= C.stackCap) {
                set_status(C.status, kDevStackOverflow);
                return 0;
            }
            m.set_del(c1, 0);
            C.push(sp++, make_int4(c1, a1, b1, 0));
        }
        if (d0) {
            m.set_del(c0, 0);
            x = c0, l0 = a0, l1 = b0;
        } else if (sp > 0) {
            const int4 f = C.pop(--sp);
            x = f.x, l0 = f.y, l1 = f.z;
        } else {
            return cnt;
        }
    }
}

// FastDelete's two reference-count decrements of a frame's fanins, whose
// returned values give the fanins' counts; L0 / L1 of both fanins
template <class Mem>
__device__ __forceinline__ void fd_open(const Mem &m, int l0, int l1, int &v0, int &a0, int &b0, int &v1, int &a1,
                                        int &b1) {
    const int c0 = l0 >> 1, c1 = l1 >> 1;
    const int o0 = m.rf_add_old(c0, -1);
    const int o1 = m.rf_add_old(c1, -1);
    m.ab(c0, a0, b0);
    m.ab(c1, a1, b1);
    v1 = o1 - 1;
    v0 = c0 == c1 ? v1 : o0 - 1;  // one node twice: both decrements precede the first check
}

// FastDelete, rewrite.h:208-220; r0, r1 = L0, L1 of root.  The recursion
// replayed with an explicit stack: a node is opened (both fanins'
// decrements), then its fanin 0 entered if its count fell to zero, then --
// with fanin 1's count read again, since fanin 0's subtree may have changed
// it -- its fanin 1, then it is marked deleted and its count handed to its
// parent.  A pushed frame is {node, count << 2 | where to resume (1: at
// fanin 1, 2: at the end), fanin0 literal, fanin1 literal}.
template <class Mem>
__device__ int ch_fast_delete(const GraphCtx<Mem> &C, int root, int r0, int r1) {
    const Mem &m = C.m;
    if (root < C.nL0) return 0;
    int v0, a0, b0, v1, a1, b1;
    int x = root, l0 = r0, l1 = r1, sp = 0;
    fd_open(m, l0, l1, v0, a0, b0, v1, a1, b1);
    int cnt = 1 - ch_red(C, x, l0, l1);
    while (true) {
        // x is open: enter fanin 0 when its count fell to zero
        if (v0 == 0 && (l0 >> 1) >= C.nL0) {
            if (sp + 1 >= C.stackCap) {
                set_status(C.status, kDevStackOverflow);
                return 0;
            }
            C.push(sp++, make_int4(x, (cnt << 2) | 1, l0, l1));
            x = l0 >> 1, l0 = a0, l1 = b0;
            fd_open(m, l0, l1, v0, a0, b0, v1, a1, b1);
            cnt = 1 - ch_red(C, x, l0, l1);
            continue;
        }
        int resume = 1;  // 1: at fanin 1 of x, 2: x is finished
        while (true) {
            if (resume == 1 && v1 == 0 && (l1 >> 1) >= C.nL0) {
                if (sp + 1 >= C.stackCap) {
                    set_status(C.status, kDevStackOverflow);
                    return 0;
                }
                C.push(sp++, make_int4(x, (cnt << 2) | 2, l0, l1));
                x = l1 >> 1, l0 = a1, l1 = b1;
                fd_open(m, l0, l1, v0, a0, b0, v1, a1, b1);
                cnt = 1 - ch_red(C, x, l0, l1);
                break;  // the new node is open
            }
            m.set_del(x, 1);
            if (sp == 0) return cnt;
            const int4 f = C.pop(--sp);
            x = f.x, l0 = f.z, l1 = f.w;
            cnt += f.y >> 2;
            resume = f.y & 3;
            if (resume == 1) m.rab(l1 >> 1, v1, a1, b1);
        }
    }
}

// The choice loop over graph g's candidates in id order (rewrite.cu:849-897).
template <class Mem>
__device__ void choice_graph(const GraphCtx<Mem> &C, int g) {
    const ChoiceArgs &A = *C.A;
    const Mem &m = C.m;
    const int4 *recA = A.recA, *recB = A.recB;
    int *choice = A.choice;
    const bool useZeros = A.useZeros != 0;
    const int cpos = A.dg[g].cpos;
    unsigned long long replaced = 0, pos = 0, zero = 0, reverted = 0, comp = 0, noRep = 0, selfRef = 0;
    long long expected = 0;
    int i = A.gStart[g];
    const int e = i + A.gCount[g];
    int4 na = make_int4(-1, -1, -1, -1), nb = na;
    if (i < e) {
        na = recA[i];
        nb = recB[i];
    }
    for (; i < e; i++) {
        const int4 a = na, lv = nb;
        if (i + 1 < e) {
            na = recA[i + 1];
            nb = recB[i + 1];
        }
        if (Mem::kPrefetch && i + 1 < e && (na.z >> 1) >= 0) {
            // the next candidate's first loads, into L1 while this one runs
            // (a prefetch carries no value, so later stores cannot make it stale)
            const int nn = na.z >> 1, nq = na.y;
            asm volatile("prefetch.global.L1 [%0];" ::"l"(A.L0 + nn));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(A.L1 + nn));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(A.del + nn));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(A.L0 + nq));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(A.L1 + nq));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(A.del + nb.x));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(A.del + nb.y));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(A.del + nb.z));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(A.del + nb.w));
        }
        const int c = a.x, q = a.y, rep = a.z;
        const int newIdx = rep >> 1;
        if (newIdx < 0) {
            noRep++;
            choice[c] = kChNoReplace;
            continue;
        }
        // everything read before this candidate's first store
        int n0, n1, dn, q0, q1;
        m.dab(newIdx, dn, n0, n1);
        const int dl = m.dl(lv.x) | m.dl(lv.y) | m.dl(lv.z) | m.dl(lv.w);
        m.ab(q, q0, q1);
        if (newIdx == q || (n1 >> 1) == q) {
            selfRef++;
            choice[c] = kChSelfRef;
            continue;
        }
        if (dl) {
            comp++;
            choice[c] = kChCompromised;
            continue;
        }
        int added = ch_install(C, newIdx, dn, n0, n1);
        m.rf_add(newIdx, 1);
        int saved = ch_fast_delete(C, q, q0, q1);
        m.rf_add(newIdx, -1);
        if (saved - added > 0 || (saved == added && useZeros)) {
            replaced++;
            if (saved - added > 0)
                pos++;
            else
                zero++;
            expected += saved - added;
            m.set_del(q, 0);
            m.set_fanins(q, C.trueLit, rep);
            m.rf_add(cpos, 1);
            m.rf_add(newIdx, 1);
            choice[c] = kChCommitted;
        } else {
            reverted++;
            ch_install(C, q, m.dl(q), q0, q1);
            m.rf_add(q, 1);
            if (m.rf(newIdx) == 0) ch_fast_delete(C, newIdx, n0, n1);
            m.rf_add(q, -1);
            choice[c] = kChReverted;
        }
    }
    atomicAdd(&A.stats[0], replaced);
    atomicAdd(&A.stats[1], pos);
    atomicAdd(&A.stats[2], zero);
    atomicAdd(&A.stats[3], reverted);
    atomicAdd(&A.stats[4], comp);
    atomicAdd(&A.stats[5], noRep);
    atomicAdd(&A.stats[6], selfRef);
    atomicAdd(&A.stats[7], (unsigned long long)expected);
}

__global__ void __launch_bounds__(kChoiceBlock) k_choice(ChoiceArgs A, int G) {
    __shared__ int4 sh[kChoiceFrames * kChoiceBlock];
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
    GraphCtx<GlobalMem> C{&A,           GlobalMem{A.L0, A.L1, A.ref, A.del}, 2 * A.dg[g].cpos + 1,
                          sh + threadIdx.x, kChoiceBlock, A.stack + (int64_t)g * A.stackCap,
                          A.nL0,        A.stackCap,   A.status};
    choice_graph(C, g);
}

constexpr int kClusterBlock = 256;
constexpr int kClusterMaxBlocks = 8;  // the portable cluster size
constexpr int kClusterMaxShift = 13;  // objects per block: 8192 16-byte records, 128 KB of shared memory

// One graph (G = 1) on a cluster: its M objects' {L0, L1, ref, del} records
// are copied into the blocks' shared memory, thread 0 of block 0 walks the
// candidates on them (one 16-byte load gives a node's flag or count and
// both fanins), and every block writes its slice back.  The blocks that do
// not walk wait at the cluster barrier.
__global__ void __launch_bounds__(kClusterBlock) k_choice_cluster(ChoiceArgs A, int64_t M, int shift) {
    extern __shared__ __align__(16) unsigned char dyn[];
    __shared__ int4 sh[kChoiceFrames];
    const int per = 1 << shift;
    int4 *rec = reinterpret_cast<int4 *>(dyn);
    cg::cluster_group cl = cg::this_cluster();
    const int64_t base = (int64_t)cl.block_rank() << shift;
    for (int k = threadIdx.x; k < per; k += blockDim.x) {
        const int64_t x = base + k;
        if (x < M) rec[k] = make_int4(A.L0[x], A.L1[x], A.ref[x], A.del[x]);
    }
    cl.sync();
    if (cl.block_rank() == 0 && threadIdx.x == 0) {
        GraphCtx<ClusterMem> C{&A,    ClusterMem{rec, shift, per - 1}, 2 * A.dg[0].cpos + 1, sh, 1, A.stack,
                               A.nL0, A.stackCap,                      A.status};
        choice_graph(C, 0);
    }
    cl.sync();
    for (int k = threadIdx.x; k < per; k += blockDim.x) {
        const int64_t x = base + k;
        if (x < M) {
            const int4 r = rec[k];
            A.L0[x] = r.x;
            A.L1[x] = r.y;
            A.ref[x] = r.z;
            A.del[x] = (uint8_t)r.w;
        }
    }
}

// the choice's record of the i-th candidate in graph order: {c, q, rep, -}
// and the chosen cut's four leaves (the constant in the fourth place of a
// three-leaf cut); leaves are read only for candidates with a replacement
__global__ void k_cand_records(int64_t n, const int *candByG, const int *cand, const int *repW, const int8_t *bestCut,
                               const int4 *cutL, const int2 *cutM, const int *wg, const DevGraph *dg, int4 *recA,
                               int4 *recB) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int c = candByG[i];
        const int q = cand[c];
        const int rep = repW[c];
        int4 l = make_int4(0, 0, 0, 0);
        if ((rep >> 1) >= 0) {
            const int slot = bestCut[q];
            l = cutL[(int64_t)q * 8 + slot];
            if (packed_nleaves((uint32_t)cutM[(int64_t)q * 8 + slot].y) == 3) l.w = dg[wg[q]].cpos;
        }
        recA[i] = make_int4(c, q, rep, 0);
        recB[i] = l;
    }
}

__global__ void k_cand_gid(int64_t n, const int *cand, const int *wg, uint32_t *keys, int *vals, int *gCount) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += stride) {
        int g = wg[cand[c]];
        keys[c] = (uint32_t)g;
        vals[c] = (int)c;
        atomicAdd(&gCount[g], 1);
    }
}

}  // namespace

int rw_choice(ExecCtx &X, Batch &b, RwWork &w, RwStats *stats) {
    const int G = w.G;
    const int64_t nCand = w.nCand;
    cudaStream_t s = X.s;
    Arena &ar = *X.ar;
    int rc;
    int *gCount = ar.get<int>(G + 1), *gStart = ar.get<int>(G + 1), *candByG = ar.get<int>(nCand + 1);
    uint32_t *keys = ar.get<uint32_t>(nCand + 1), *keys2 = ar.get<uint32_t>(nCand + 1);
    int *vals = ar.get<int>(nCand + 1);
    int4 *recA = ar.get<int4>(nCand + 1), *recB = ar.get<int4>(nCand + 1);
    w.choice = ar.get<int>(nCand + 1);
    unsigned long long *dstats = ar.get<unsigned long long>(8);
    // explicit recursion stacks: deep enough for any chain through the
    // levels plus the new nodes
    int64_t stackCap = (int64_t)w.maxLevel + 64;
    for (int g = 0; g < G; g++) stackCap = std::max<int64_t>(stackCap, 64);
    stackCap = std::min<int64_t>(2 * stackCap + w.nNew / std::max(G, 1) + 64, 1 << 20);
    int4 *stack = ar.get<int4>((size_t)stackCap * G);
    if (!gCount || !gStart || !candByG || !keys || !keys2 || !vals || !recA || !recB || !w.choice || !dstats || !stack)
        return X.fail(CULS_E_OOM, "rw: arena exhausted (choice)");
    if ((rc = X.check(cudaMemsetAsync(gCount, 0, sizeof(int) * (G + 1), s), "memset"))) return rc;
    if ((rc = X.check(cudaMemsetAsync(dstats, 0, sizeof(unsigned long long) * 8, s), "memset"))) return rc;
    if (nCand > 0) {
        k_cand_gid<<<X.grid(nCand), kBlock, 0, s>>>(nCand, w.cand, w.wg, keys, vals, gCount);
        X.launched(1);
        if (G > 1) {
            int bits = 1;
            while ((1ll << bits) < G) bits++;
            if ((rc = X.check(radix_sort_pairs(keys, vals, keys2, candByG, nCand, bits, ar, s), "sort"))) return rc;
        } else {
            if ((rc = X.check(iota_i32(candByG, 0, nCand, s), "iota"))) return rc;
        }
        k_cand_records<<<X.grid(nCand), kBlock, 0, s>>>(nCand, candByG, w.cand, w.repW, w.bestCut, w.cutL, w.cutM, w.wg,
                                                        w.dg, recA, recB);
        X.launched(1);
    }
    if ((rc = X.check(scan_exclusive(gCount, gStart, G, nullptr, ar, s), "scan"))) return rc;
    ChoiceArgs A{w.nL0, w.dg,   w.L0,   w.L1,     w.ref,    w.del,       recA,   recB,  gStart,
                 gCount, w.useZeros ? 1 : 0,    stack,  (int)stackCap,       w.choice, dstats, X.status};
    // a single graph that fits: the cluster walk (not on an SM partition,
    // whose SMs need not hold a whole cluster)
    const int64_t M = w.N + w.nNew;  // extent of L0, L1, ref, del
    bool onCluster = false;
    if (G == 1 && X.clusters && M <= ((int64_t)kClusterMaxBlocks << kClusterMaxShift) && !getenv("CULS_CHOICE_GLOBAL")) {
        int shift = 8;
        while (((int64_t)kClusterMaxBlocks << shift) < M) shift++;
        const int blocks = (int)((M + (1 << shift) - 1) >> shift);
        const size_t smem = sizeof(int4) << shift;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)blocks);
        cfg.blockDim = dim3(kClusterBlock);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = s;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = (unsigned)blocks;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int fits = 0;
        if (cudaFuncSetAttribute(k_choice_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) ==
                cudaSuccess &&
            cudaOccupancyMaxActiveClusters(&fits, k_choice_cluster, &cfg) == cudaSuccess && fits > 0) {
            onCluster = cudaLaunchKernelEx(&cfg, k_choice_cluster, A, M, shift) == cudaSuccess;
        }
        (void)cudaGetLastError();  // a configuration the device refuses leaves no error behind
    }
    if (!onCluster) {
        // the walk's working set is the graph's fanins, flags and counts: the
        // smallest shared-memory carveout leaves the most L1 for it
        cudaFuncSetAttribute(k_choice, cudaFuncAttributePreferredSharedMemoryCarveout, 0);
        k_choice<<<(G + kChoiceBlock - 1) / kChoiceBlock, kChoiceBlock, 0, s>>>(A, G);
    }
    X.launched(1);
    unsigned long long hs[8], warpPairs = 0;
    if ((rc = X.check(cudaMemcpyAsync(hs, dstats, sizeof hs, cudaMemcpyDeviceToHost, s), "d2h"))) return rc;
    if (w.warpPairs &&
        (rc = X.check(cudaMemcpyAsync(&warpPairs, w.warpPairs, sizeof warpPairs, cudaMemcpyDeviceToHost, s), "d2h")))
        return rc;
    if ((rc = X.sync())) return rc;
    if ((rc = X.status_check("rw choice"))) return rc;
    if (stats) {
        int64_t nAnd = w.N - w.nL0;
        stats->replaced = (long long)hs[0];
        stats->replacedPos = (long long)hs[1];
        stats->replacedZero = (long long)hs[2];
        stats->reverted = (long long)hs[3];
        stats->compromised = (long long)hs[4];
        stats->newIdx = (long long)hs[5];
        stats->expected = (long long)hs[7];
        stats->preEval = nAnd - nCand;
        stats->smallCut = 0;
        stats->newNodes = w.nNew;
        stats->candidates = nCand;
        stats->warpPairs = (long long)warpPairs;
    }
    (void)b;
    return 0;
}

namespace {

// per node, fixed during the sweeps
enum : uint8_t { kRdPi = 1, kRdDel = 2, kRdR0 = 4 };  // PI or constant; deleted; redundant before the sweep

struct RedArgs {
    int64_t M;
    const int *gidAll;
    const DevGraph *dg;
    const int *pre0, *pre1;
    const uint8_t *st;
    const int *postIn1;
    const uint8_t *nredIn;
    int *post1;
    uint8_t *nredOut;
    int *changed;
    int *status;
};

__global__ void k_red_state(int64_t M, int64_t nL0, const int *gidAll, const DevGraph *dg, const int *L0, const int *L1,
                            const uint8_t *del, uint8_t *st) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < M; x += stride) {
        if (x < nL0) {
            st[x] = kRdPi;
            continue;
        }
        const int a = L0[x];
        const bool r0 = a == L1[x] || a == 2 * dg[gidAll[x]].cpos + 1;
        st[x] = (uint8_t)((del[x] ? kRdDel : 0) | (r0 ? kRdR0 : 0));
    }
}

// Fanin() of rewrite.h:121-124 as seen by the sweep at node `time`
// (time = INT_MAX after the sweep).  A node is chased (its fanins are
// rewritten by the sweep) when it is no PI, not deleted and not redundant
// before the sweep: state byte 0.
__device__ int rd_chase(const RedArgs &A, int lit, int time) {
    int c = 0;
    for (int step = 0; step < (1 << 20); step++) {
        const int u = lit >> 1;
        const int s = A.st[u];
        if (s & kRdPi) return lit ^ c;
        const bool done = u < time && s == 0;
        const bool red = done ? A.nredIn[u] != 0 : (s & kRdR0) != 0;
        if (!red) return lit ^ c;
        c ^= lit & 1;
        lit = done ? A.postIn1[u] : A.pre1[u];
    }
    set_status(A.status, kDevBadGraph);
    return lit ^ c;
}

// one sweep over the chased nodes; the others keep their fanins and are
// never read as sweep state
__global__ void k_redundancy(RedArgs A) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < A.M; x += stride) {
        if (A.st[x]) continue;
        const int a = rd_chase(A, A.pre0[x], (int)x);
        const int b = rd_chase(A, A.pre1[x], (int)x);
        const int t = 2 * A.dg[A.gidAll[x]].cpos + 1;
        const uint8_t nr = (a == b || a == t) ? 1 : 0;
        if (nr != A.nredIn[x] || b != A.postIn1[x]) atomicExch(A.changed, 1);
        A.post1[x] = b;
        A.nredOut[x] = nr;
    }
}

// pre0 aliases L0 (each node reads and writes only its own entry); pre1 is a
// copy, since other nodes' chases read it
__global__ void k_redundancy_finish(RedArgs A, int *L0, int *L1, uint8_t *delOut, int64_t nPO, int *po) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < A.M; x += stride) {
        const int s = A.st[x];
        if (s == 0) {
            L0[x] = rd_chase(A, A.pre0[x], (int)x);
            L1[x] = A.postIn1[x];
        } else if (!(s & (kRdPi | kRdDel))) {
            delOut[x] = 1;  // redundant before the sweep: rewrite.cu:916-917
        }
    }
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nPO; k += stride) po[k] = rd_chase(A, po[k], INT_MAX);
}

}  // namespace

int rw_redundancy(ExecCtx &X, Batch &b, RwWork &w) {
    (void)b;
    const int64_t M = w.N + w.nNew;
    cudaStream_t s = X.s;
    Arena &ar = *X.ar;
    int rc;
    int *pre1 = ar.get<int>(M);
    int *P1[2] = {ar.get<int>(M), ar.get<int>(M)};
    uint8_t *NR[2] = {ar.get<uint8_t>(M), ar.get<uint8_t>(M)};
    uint8_t *st = ar.get<uint8_t>(M);
    if (!pre1 || !P1[0] || !P1[1] || !NR[0] || !NR[1] || !st) return X.fail(CULS_E_OOM, "rw: arena exhausted (redundancy)");
    if ((rc = X.check(cudaMemcpyAsync(pre1, w.L1, sizeof(int) * M, cudaMemcpyDeviceToDevice, s), "copy"))) return rc;
    if ((rc = X.check(cudaMemsetAsync(NR[0], 0, M, s), "memset"))) return rc;
    k_red_state<<<X.grid(M), kBlock, 0, s>>>(M, w.nL0, w.gidAll, w.dg, w.L0, w.L1, w.del, st);
    X.launched(1);
    int *changed = X.counters + 24;
    // sweep state: (post1, nred) of the chased nodes; state 0 (no chase
    // yet) is (pre1, 0), read from pre1 itself
    const int *in1 = pre1;
    const uint8_t *inR = NR[0];
    int cur = 1;
    for (int it = 0;; it++) {
        if (it >= 64) return X.fail(CULS_E_INVALID, "rw: redundancy sweep did not converge");
        RedArgs A{M, w.gidAll, w.dg, w.L0, pre1, st, in1, inR, P1[cur], NR[cur], changed, X.status};
        if ((rc = X.check(cudaMemsetAsync(changed, 0, sizeof(int), s), "memset"))) return rc;
        k_redundancy<<<X.grid(M), kBlock, 0, s>>>(A);
        X.launched(1);
        if ((rc = X.check(cudaMemcpyAsync(X.hostSmall + 24, changed, sizeof(int), cudaMemcpyDeviceToHost, s), "d2h")))
            return rc;
        if ((rc = X.sync())) return rc;
        in1 = P1[cur];
        inR = NR[cur];
        cur ^= 1;
        if (!X.hostSmall[24]) break;
    }
    // (in1, inR) is a fix-point: sweeping it again reproduces it
    RedArgs F{M, w.gidAll, w.dg, w.L0, pre1, st, in1, inR, nullptr, nullptr, changed, X.status};
    k_redundancy_finish<<<X.grid(std::max<int64_t>(M, w.nPO)), kBlock, 0, s>>>(F, w.L0, w.L1, w.del, w.nPO, w.wpo);
    X.launched(1);
    if ((rc = X.sync())) return rc;
    return X.status_check("rw redundancy");
}

}  // namespace culs
