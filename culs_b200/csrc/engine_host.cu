// Engine set-up, batch upload/download and the `st` command.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "rw_work.cuh"

extern "C" const unsigned char culs_rwlib_blob[];
extern "C" const size_t culs_rwlib_blob_size;

namespace culs {

int ExecCtx::status_check(const char *what) {
    int st = 0;
    cudaError_t e = cudaMemcpy(&st, status, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return check(e, what);
    if (st == kDevOk) return 0;
    cudaMemset(status, 0, sizeof(int));
    static const char *names[] = {"ok", "dependency wait timed out", "hash table full", "traversal stack overflow",
                                  "malformed graph", "work buffer too small", "malformed binary AIGER"};
    if (err) *err = std::string(what) + ": " + (st >= 0 && st <= 6 ? names[st] : "device error");
    if (st == kDevWaitTimeout || st == kDevTableFull || st == kDevStackOverflow) return CULS_E_PROBE;
    if (st == kDevAigerFormat) return CULS_E_IO;
    return CULS_E_INVALID;
}

Batch::~Batch() { release(); }

DevPool::~DevPool() { flush(); }

void *DevPool::take(size_t bytes, size_t *got) {
    {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = free_.lower_bound(bytes);
        if (it != free_.end() && it->first <= 2 * bytes) {
            void *p = it->second;
            *got = it->first;
            cached_ -= it->first;
            free_.erase(it);
            return p;
        }
    }
    void *p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        flush();  // cached blocks may be what stands in the way
        if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
    }
    *got = bytes;
    return p;
}

void DevPool::give(void *p, size_t bytes) {
    if (!p) return;
    {
        std::lock_guard<std::mutex> lk(mu_);
        if (cached_ + bytes <= limit_) {
            free_.emplace(bytes, p);
            cached_ += bytes;
            return;
        }
    }
    cudaFree(p);
}

void DevPool::flush() {
    std::multimap<size_t, void *> all;
    {
        std::lock_guard<std::mutex> lk(mu_);
        all.swap(free_);
        cached_ = 0;
    }
    for (auto &kv : all) cudaFree(kv.second);
}

namespace {

template <class T>
void drop(const std::shared_ptr<DevPool> &pool, T *&p, size_t bytes) {
    if (p) {
        if (pool)
            pool->give(p, bytes);
        else
            cudaFree(p);
    }
    p = nullptr;
}

// Grows *p to at least `need` elements (contents not kept); cap is the
// block's real element count.
template <class T>
cudaError_t grow(const std::shared_ptr<DevPool> &pool, T *&p, int64_t &cap, int64_t need) {
    need = std::max<int64_t>(need, 1);
    if (p && cap >= need) return cudaSuccess;
    drop(pool, p, sizeof(T) * (size_t)cap);
    cap = 0;
    if (pool) {
        size_t got = 0;
        p = static_cast<T *>(pool->take(sizeof(T) * (size_t)need, &got));
        if (!p) return cudaErrorMemoryAllocation;
        cap = (int64_t)(got / sizeof(T));
        return cudaSuccess;
    }
    cudaError_t e = cudaMalloc(&p, sizeof(T) * (size_t)need);
    if (e == cudaSuccess) cap = need;
    return e;
}

}  // namespace

void Batch::release() {
    drop(pool, F0, sizeof(int) * (size_t)capObj);
    drop(pool, F1, sizeof(int) * (size_t)capObj);
    drop(pool, PO, sizeof(int) * (size_t)capPO);
    drop(pool, dg, sizeof(DevGraph) * (size_t)capG);
    drop(pool, F0s, sizeof(int) * (size_t)capObjS);
    drop(pool, F1s, sizeof(int) * (size_t)capObjS);
    drop(pool, POs, sizeof(int) * (size_t)capPOS);
    drop(pool, F0k, sizeof(int) * (size_t)capObjK);
    drop(pool, F1k, sizeof(int) * (size_t)capObjK);
    drop(pool, POk, sizeof(int) * (size_t)capPOK);
    capObjK = capPOK = nObjK = 0;
    keep = false;
    hgk.clear();
    capObj = capPO = capObjS = capPOS = 0;
    capG = 0;
    G = 0;
    nObj = nPO = 0;
    hg.clear();
}

cudaError_t Batch::reserve(int64_t n, int64_t np, int g) {
    keep = false;  // a new graph is written: no rewrite state carries over
    int64_t c0 = capObj, c1 = capObj, cg = capG;
    cudaError_t e;
    if ((e = grow(pool, F0, c0, n)) != cudaSuccess) return e;
    if ((e = grow(pool, F1, c1, n)) != cudaSuccess) return e;
    capObj = std::min(c0, c1);
    if ((e = grow(pool, PO, capPO, np)) != cudaSuccess) return e;
    if ((e = grow(pool, dg, cg, g)) != cudaSuccess) return e;
    capG = (int)cg;
    return cudaSuccess;
}

cudaError_t Batch::reserve_spare(int64_t n, int64_t np) {
    int64_t c0 = capObjS, c1 = capObjS;
    cudaError_t e;
    if ((e = grow(pool, F0s, c0, n)) != cudaSuccess) return e;
    if ((e = grow(pool, F1s, c1, n)) != cudaSuccess) return e;
    capObjS = std::min(c0, c1);
    return grow(pool, POs, capPOS, np);
}

cudaError_t Batch::keep_current(cudaStream_t s) {
    int64_t c0 = capObjK, c1 = capObjK;
    cudaError_t e;
    if ((e = grow(pool, F0k, c0, nObj)) != cudaSuccess) return e;
    if ((e = grow(pool, F1k, c1, nObj)) != cudaSuccess) return e;
    capObjK = std::min(c0, c1);
    if ((e = grow(pool, POk, capPOK, nPO)) != cudaSuccess) return e;
    if (nObj && (e = cudaMemcpyAsync(F0k, F0, sizeof(int) * nObj, cudaMemcpyDeviceToDevice, s))) return e;
    if (nObj && (e = cudaMemcpyAsync(F1k, F1, sizeof(int) * nObj, cudaMemcpyDeviceToDevice, s))) return e;
    if (nPO && (e = cudaMemcpyAsync(POk, PO, sizeof(int) * nPO, cudaMemcpyDeviceToDevice, s))) return e;
    hgk = hg;
    nObjK = nObj;
    keep = true;
    return cudaSuccess;
}

void Batch::restore_kept() {
    std::swap(F0, F0k);
    std::swap(F1, F1k);
    std::swap(PO, POk);
    std::swap(capObj, capObjK);
    std::swap(capPO, capPOK);
    hg = hgk;
    nObj = nObjK;
    keep = false;
}

void Batch::swap_spare() {
    std::swap(F0, F0s);
    std::swap(F1, F1s);
    std::swap(PO, POs);
    std::swap(capObj, capObjS);
    std::swap(capPO, capPOS);
}

// Decodes the embedded rwlib.bin (culs_b200/data/make_rwlib.py layout).
static bool decode_lib(const unsigned char *b, size_t n, RwLib &L) {
    if (n < 40 || memcmp(b, "CULSRWL1", 8) != 0) return false;
    size_t cur = 40;
    auto need = [&](size_t k) { return cur + k <= n; };
    const int kNtt = 1 << 16;
    if (!need(3 * (size_t)kNtt + 96 + 2 * kNumClasses)) return false;
    const unsigned char *ph = b + cur;
    const unsigned char *pe = ph + kNtt;
    const unsigned char *p4 = pe + kNtt;
    const unsigned char *cl = p4 + 96;
    const unsigned char *nn = cl + kNtt;
    const unsigned char *nr = nn + kNumClasses;
    cur = (size_t)(nr + kNumClasses - b);
    for (int t = 0; t < kNtt; t++) L.npn[t] = (uint32_t)ph[t] | ((uint32_t)pe[t] << 8) | ((uint32_t)cl[t] << 16);
    memcpy(&L.perm4[0][0], p4, 96);
    memcpy(L.nNodes, nn, kNumClasses);
    memcpy(L.nRoots, nr, kNumClasses);
    memset(L.node, 0, sizeof L.node);
    memset(L.roots, 0, sizeof L.roots);
    memset(L.batch, 0xFF, sizeof L.batch);
    memset(L.rootCone, 0, sizeof L.rootCone);
    for (int c = 0; c < kNumClasses; c++) {
        if (L.nNodes[c] > kMaxLibNodes - 4 || L.nRoots[c] > 16) return false;
        if (!need((size_t)L.nNodes[c] * 4 + L.nRoots[c])) return false;
        for (int i = 0; i < L.nNodes[c]; i++) {
            const unsigned char *q = b + cur;
            L.node[c][i] = (uint32_t)q[0] | ((uint32_t)q[1] << 8) | ((uint32_t)(q[2] & 1) << 16) |
                           ((uint32_t)(q[3] & 1) << 17);
            cur += 4;
        }
        memcpy(L.roots[c], b + cur, L.nRoots[c]);
        cur += L.nRoots[c];
        for (int i = 0; i < L.nNodes[c]; i++)  // fanins precede their node
            if (ln_f0(L.node[c][i]) >= i + 4 || ln_f1(L.node[c][i]) >= i + 4) return false;
        // evaluation batches: nodes by depth (inputs at depth 0), index order
        // within a depth, at most kLibBatch per batch
        int depth[kMaxLibNodes], maxDepth = 0;
        for (int i = 0; i < 4; i++) depth[i] = 0;
        for (int i = 0; i < L.nNodes[c]; i++) {
            const int d0 = depth[ln_f0(L.node[c][i])], d1 = depth[ln_f1(L.node[c][i])];
            depth[i + 4] = 1 + (d0 > d1 ? d0 : d1);
            maxDepth = depth[i + 4] > maxDepth ? depth[i + 4] : maxDepth;
        }
        int nb = 0;
        for (int d = 1; d <= maxDepth; d++) {
            uint32_t ent[kLibBatch];
            int k = 0;
            for (int i = 0; i <= L.nNodes[c]; i++) {
                const bool flush = k == kLibBatch || (i == L.nNodes[c] && k > 0);
                if (flush) {
                    for (int e = k; e < kLibBatch; e++) ent[e] = kNoLibNode;
                    L.batch[c][nb++] = uint4{ent[0], ent[1], ent[2], ent[3]};
                    k = 0;
                }
                if (i < L.nNodes[c] && depth[i + 4] == d) ent[k++] = L.node[c][i] | ((uint32_t)i << 18);
            }
        }
        L.nBatches[c] = (uint8_t)nb;
        // root cones over the internal nodes
        unsigned long long cone[kMaxLibNodes] = {0, 0, 0, 0};
        for (int i = 0; i < L.nNodes[c]; i++)
            cone[i + 4] = (1ull << (i + 4)) | cone[ln_f0(L.node[c][i])] | cone[ln_f1(L.node[c][i])];
        for (int r = 0; r < L.nRoots[c]; r++) {
            if (L.roots[c][r] >= 4 + L.nNodes[c]) return false;
            L.rootCone[c][r] = cone[L.roots[c][r]];
        }
    }
    int order[kNumClasses];
    for (int c = 0; c < kNumClasses; c++) order[c] = c;
    std::stable_sort(order, order + kNumClasses, [&](int a, int b) { return L.nBatches[a] < L.nBatches[b]; });
    for (int i = 0; i < kNumClasses; i++) L.classSlot[order[i]] = (uint8_t)i;
    return cur == n;
}

Engine::Engine() = default;

Engine::~Engine() {
    if (s_) cudaStreamSynchronize(s_);
    cudaFree(lib_);
    cudaFree(status_);
    cudaFree(counters_);
    if (hostSmall_) cudaFreeHost(hostSmall_);
    if (stage_) cudaFreeHost(stage_);
    for (auto &e : ev_)
        if (e) cudaEventDestroy(e);
    if (s_ && ownStream_) cudaStreamDestroy(s_);
}

int Engine::fail(int code, const std::string &msg) {
    err_ = msg;
    return code;
}

int Engine::check(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return 0;
    err_ = std::string(what) + ": " + cudaGetErrorString(e);
    return CULS_E_DEVICE;
}

int Engine::sync() { return check(cudaStreamSynchronize(s_), "stream sync"); }

int Engine::check_status(const char *what) {
    ExecCtx X = ctx();
    return X.status_check(what);
}

// CULS_SPIN_LIMIT (spin iterations, 0 or unset = the built-in bound of about
// one second) bounds every dependency wait of the next calls; the tests lower
// it to make waits run out on purpose.  Read at each call, like
// CULS_STRASH_TABLE_CAP.
void Engine::apply_spin_limit() {
    const char *env = getenv("CULS_SPIN_LIMIT");
    long long want = env ? atoll(env) : 0;
    if (want < 0 || want > (1ll << 30)) want = 0;
    if ((int)want == spinLimit_) return;
    const int v = (int)want;
    // pageable source: the call returns once v has been staged
    if (cudaMemcpyAsync(status_ + 1, &v, sizeof(int), cudaMemcpyHostToDevice, s_) == cudaSuccess) spinLimit_ = v;
}

ExecCtx Engine::ctx() {
    apply_spin_limit();
    ExecCtx X;
    X.s = s_;
    X.ar = &ar_;
    X.status = status_;
    X.counters = counters_;
    X.hostSmall = hostSmall_;
    X.lib = lib_;
    X.sms = sms_;
    X.clusters = ownStream_;
    X.launches = &launches_;
    X.err = &err_;
    X.ev = prof_ ? ev_ : nullptr;
    X.evSet = evSet_;
    X.tune = &tune_;
    return X;
}

int Engine::init(size_t hbmBudget) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return fail(CULS_E_DEVICE, "no CUDA device");
    int rc;
    if ((rc = check(cudaGetDevice(&device_), "device"))) return rc;
    if ((rc = check(cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking), "stream"))) return rc;
    sms_ = num_sms();
    RwLib *h = new RwLib;
    bool ok = decode_lib(culs_rwlib_blob, culs_rwlib_blob_size, *h);
    if (!ok) {
        delete h;
        return fail(CULS_E_INVALID, "embedded rewriting library is malformed");
    }
    rc = check(cudaMalloc(&lib_, sizeof(RwLib)), "cudaMalloc");
    if (!rc) rc = check(cudaMemcpy(lib_, h, sizeof(RwLib), cudaMemcpyHostToDevice), "library upload");
    delete h;
    if (rc) return rc;
    // status word and the spin bound of dependency waits (see common.cuh)
    if ((rc = check(cudaMalloc(&status_, sizeof(int) * 2), "cudaMalloc"))) return rc;
    if ((rc = check(cudaMemset(status_, 0, sizeof(int) * 2), "memset"))) return rc;
    if ((rc = check(cudaMalloc(&counters_, sizeof(int) * 64), "cudaMalloc"))) return rc;
    if ((rc = check(cudaMallocHost(&hostSmall_, sizeof(int) * 64), "cudaMallocHost"))) return rc;
    for (auto &e : ev_)
        if ((rc = check(cudaEventCreate(&e), "event"))) return rc;
    size_t freeB = 0, totalB = 0;
    cudaMemGetInfo(&freeB, &totalB);
    budget_ = hbmBudget ? hbmBudget : totalB;
    pool_ = std::make_shared<DevPool>(budget_ / 4);  // freed batch buffers kept for reuse
    return 0;
}

int Engine::set_high_priority(bool high) {
    int least = 0, greatest = 0;
    int rc = check(cudaDeviceGetStreamPriorityRange(&least, &greatest), "stream priorities");
    if (rc) return rc;
    if ((rc = sync())) return rc;
    cudaStream_t ns = nullptr;
    if ((rc = check(cudaStreamCreateWithPriority(&ns, cudaStreamNonBlocking, high ? greatest : least), "stream")))
        return rc;
    if (ownStream_) cudaStreamDestroy(s_);
    s_ = ns;
    ownStream_ = true;
    highPrio_ = high;
    return 0;
}

int Engine::adopt_stream(cudaStream_t s, int sms) {
    int rc = sync();
    if (rc) return rc;
    if (ownStream_) cudaStreamDestroy(s_);
    s_ = s;
    ownStream_ = false;
    sms_ = std::max(8, sms);
    share_ = std::max(1, num_sms() / sms_);
    tune_.enumBlocksPerSm = std::min(tune_.enumBlocksPerSm, 3);
    return 0;
}

int Engine::ensure_arena(size_t bytes) {
    bytes = (bytes + (64u << 20)) & ~(size_t)((1u << 20) - 1);
    if (bytes <= ar_.capacity()) return 0;
    if (bytes > budget_) return fail(CULS_E_BUDGET, "request exceeds the HBM budget");
    ar_.reset();
    cudaError_t e = ar_.reserve(bytes);
    if (e != cudaSuccess && pool_) {  // cached batch buffers may be in the way
        cudaGetLastError();
        pool_->flush();
        e = ar_.reserve(bytes);
    }
    if (e != cudaSuccess) return fail(CULS_E_OOM, std::string("device arena: ") + cudaGetErrorString(e));
    return 0;
}

void Engine::mark(int m) {
    if (m < 0 || m >= kNumMarks) return;
    cudaEventRecord(ev_[m], s_);
    evSet_[m] = true;
}

float Engine::elapsed(int a, int b) {
    if (a < 0 || b < 0 || a >= kNumMarks || b >= kNumMarks || !evSet_[a] || !evSet_[b]) return -1.f;
    float ms = -1.f;
    if (cudaEventSynchronize(ev_[b]) != cudaSuccess) return -1.f;
    if (cudaEventElapsedTime(&ms, ev_[a], ev_[b]) != cudaSuccess) return -1.f;
    return ms;
}

int Engine::clone(const Batch &src, Batch &dst) {
    if (&src == &dst) return 0;
    int rc;
    if (!dst.pool) dst.pool = pool_;
    if ((rc = check(dst.reserve(src.nObj, src.nPO, src.G), "cudaMalloc"))) return rc;
    cudaMemcpyAsync(dst.F0, src.F0, sizeof(int) * src.nObj, cudaMemcpyDeviceToDevice, s_);
    cudaMemcpyAsync(dst.F1, src.F1, sizeof(int) * src.nObj, cudaMemcpyDeviceToDevice, s_);
    if (src.nPO) cudaMemcpyAsync(dst.PO, src.PO, sizeof(int) * src.nPO, cudaMemcpyDeviceToDevice, s_);
    cudaMemcpyAsync(dst.dg, src.dg, sizeof(DevGraph) * src.G, cudaMemcpyDeviceToDevice, s_);
    dst.G = src.G;
    dst.nObj = src.nObj;
    dst.nPO = src.nPO;
    dst.hg = src.hg;
    return check(cudaGetLastError(), "clone");
}


int Engine::download(const Batch &b, int g, int32_t *f0, int32_t *f1, int32_t *outs) {
    if (g < 0 || g >= b.G) return fail(CULS_E_INVALID, "download: graph index out of range");
    const DevGraph &d = b.hg[g];
    const int64_t n = 1 + (int64_t)d.nPIs + d.nAnds;
    int rc;
    if (f0 && (rc = check(cudaMemcpyAsync(f0, b.F0 + d.base, sizeof(int) * n, cudaMemcpyDeviceToHost, s_), "d2h")))
        return rc;
    if (f1 && (rc = check(cudaMemcpyAsync(f1, b.F1 + d.base, sizeof(int) * n, cudaMemcpyDeviceToHost, s_), "d2h")))
        return rc;
    if (outs && d.nPOs &&
        (rc = check(cudaMemcpyAsync(outs, b.PO + d.poOff, sizeof(int) * d.nPOs, cudaMemcpyDeviceToHost, s_), "d2h")))
        return rc;
    return sync();
}

// ---------------------------------------------------------------- st
namespace {

__global__ void k_st_prep(int64_t N, int G, const DevGraph *dg, const int *F0, const int *F1, int *L0, int *L1,
                          int *gid, int *lid) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += stride) {
        int g = graph_of_pos(dg, G, (int)p);
        int base = dg[g].base;
        int local = (int)p - base;
        gid[p] = g;
        lid[p] = local;
        if (local <= dg[g].nPIs) {
            L0[p] = L1[p] = -1;
        } else {
            L0[p] = F0[p] + 2 * base;
            L1[p] = F1[p] + 2 * base;
        }
    }
}

__global__ void k_st_po(int64_t nPO, int G, const DevGraph *dg, const int *PO, int *po) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nPO; k += stride)
        po[k] = PO[k] + 2 * dg[graph_of_po(dg, G, (int)k)].base;
}

}  // namespace

int Engine::st(Batch &b, bool cpuOrder) {
    if (prof_) mark(kMkStStart);
    // `st` = GPU strash (frontier order, trivial folding); `st -c` = CPU strash
    // (id order, no folding), both with dangling removal
    const int rc = strash_batch(b, cpuOrder, true, !cpuOrder);
    if (prof_) mark(kMkStEnd);
    return rc;
}

int Engine::strash_batch(Batch &b, bool idOrder, bool removeDangling, bool foldTrivial) {
    const int64_t N = b.nObj;
    b.keep = false;  // a strash ends the rewrite manager's state (src/aig/strash.cu:498)
    int rc;
    if ((rc = ensure_arena((size_t)N * 160 + (size_t)b.nPO * 8 + ((size_t)64 << 20)))) return rc;
    ar_.reset();
    int *L0 = ar_.get<int>(N), *L1 = ar_.get<int>(N), *gid = ar_.get<int>(N), *lid = ar_.get<int>(N);
    int *po = ar_.get<int>(b.nPO + 1);
    if (!L0 || !L1 || !gid || !lid || !po) return fail(CULS_E_OOM, "st: arena exhausted");
    for (auto &g : b.hg) g.cpos = g.base;
    if ((rc = check(cudaMemcpyAsync(b.dg, b.hg.data(), sizeof(DevGraph) * b.G, cudaMemcpyHostToDevice, s_), "h2d")))
        return rc;
    ExecCtx X = ctx();
    k_st_prep<<<X.grid(N), kBlock, 0, s_>>>(N, b.G, b.dg, b.F0, b.F1, L0, L1, gid, lid);
    if (b.nPO) k_st_po<<<X.grid(b.nPO), kBlock, 0, s_>>>(b.nPO, b.G, b.dg, b.PO, po);
    launches_ += 2;
    return strash_core(b, N, L0, L1, gid, lid, po, idOrder, removeDangling, foldTrivial, true);
}

}  // namespace culs
