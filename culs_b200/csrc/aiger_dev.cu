// Binary AIGER decoded and encoded on the device, for whole batches: the
// B200 form of AIGMan::readFromMemory / aigDecodeBinary and AIGMan::saveFile
// / aigEncodeBinary (CULS src/aig_manager.cu:110-267,861-880), with the
// acceptance rules and byte layout of the host reader and writer in
// host_aiger.cpp.
//
// A file is a text header "aig M I L O A", O text lines of output literals,
// then 2A variable-length numbers (7 bits per byte, high bit = more bytes
// follow): for AND i, delta0 = lhs - rhs1 and delta1 = rhs1 - rhs0 with lhs =
// 2 (I + 1 + i) and rhs0 <= rhs1.  The header and output lines are short and
// parsed on the host; the number section of every graph crosses PCIe as
// bytes (about a third of the fanin arrays) and is decoded on the device:
//  1. each 4,096-byte tile counts its terminator bytes (high bit clear);
//  2. an exclusive scan of the tile counts gives every terminator its number
//     index, and per graph the index of its first number;
//  3. every terminator decodes its number (at most five bytes, scanning back
//     over continuation bytes) into its graph's slot, in parallel;
//  4. every AND turns its two numbers into the fanin literals of the AIGMan
//     layout (literal 0 = TRUE), checking that the fanins precede the node.
// Encoding runs the other way: every AND writes its two numbers' byte
// lengths, a scan places them, every AND writes its bytes, and the host
// frames each graph's bytes with the header, the output lines and "c".
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <exception>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "kernels.cuh"
#include "rw_work.cuh"

namespace culs {

namespace {

constexpr int kAigTile = 4096;   // bytes per block in the decoding passes
constexpr int kAigThreads = 256;  // 16 bytes per thread
constexpr int kAigPerThread = kAigTile / kAigThreads;

__host__ __device__ __forceinline__ int aig_inv_const(int lit) { return lit < 2 ? 1 - lit : lit; }

__host__ __device__ __forceinline__ int vlen(uint32_t x) {
    int n = 1;
    while (x & ~0x7fu) {
        x >>= 7;
        n++;
    }
    return n;
}

// Last index i in [0, n) with a[i] <= v (a sorted, a[0] <= v).
__device__ __forceinline__ int upper_index(const int64_t *a, int n, int64_t v) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (a[mid] <= v)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// 1. terminators per tile
__global__ void __launch_bounds__(kAigThreads) k_aig_count(const uint8_t *buf, int64_t n, int *tileCnt) {
    __shared__ int s[kAigThreads / 32];
    const int64_t t0 = (int64_t)blockIdx.x * kAigTile;
    int c = 0;
    for (int k = threadIdx.x; k < kAigTile; k += kAigThreads) {
        const int64_t i = t0 + k;
        if (i < n && !(buf[i] & 0x80)) c++;
    }
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < kAigThreads / 32; w++) t += s[w];
        tileCnt[blockIdx.x] = t;
    }
}

// 2. index of each graph's first number: terminators before its region
__global__ void k_aig_term_base(int G, const uint8_t *buf, int64_t n, const int64_t *regOff, const int64_t *tileBase,
                                int64_t *termBase) {
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g <= G; g += gridDim.x * blockDim.x) {
        const int64_t off = regOff[g];
        const int64_t tile = off / kAigTile;
        int64_t c = tileBase[tile];
        for (int64_t i = tile * kAigTile; i < off && i < n; i++) c += !(buf[i] & 0x80);
        termBase[g] = c;
    }
}

struct AigDecode {
    const uint8_t *buf;
    int64_t n;
    const int64_t *tileBase;
    int G;
    const int64_t *regOff;    // G + 1 region starts in buf
    const int64_t *termBase;  // G + 1: number index of each region's first number
    const int64_t *andBase;   // G + 1: first AND of each graph in the batch
    uint32_t *nums;           // 2 per AND
    int *status;
};

// 3. every terminator decodes the number it ends
__global__ void __launch_bounds__(kAigThreads) k_aig_numbers(AigDecode A) {
    __shared__ int s[kAigThreads / 32];
    const int64_t t0 = (int64_t)blockIdx.x * kAigTile + (int64_t)threadIdx.x * kAigPerThread;
    uint32_t term = 0;  // bit k: byte t0 + k ends a number
#pragma unroll
    for (int k = 0; k < kAigPerThread; k++) {
        const int64_t i = t0 + k;
        if (i < A.n && !(A.buf[i] & 0x80)) term |= 1u << k;
    }
    // exclusive scan of the per-thread counts over the block
    const int c = __popc(term), lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int inc = c;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, inc, d);
        if (lane >= d) inc += y;
    }
    if (lane == 31) s[wid] = inc;
    __syncthreads();
    int before = 0;
    for (int w = 0; w < wid; w++) before += s[w];
    int64_t t = A.tileBase[blockIdx.x] + before + inc - c;
    while (term) {
        const int k = __ffs(term) - 1;
        term &= term - 1;
        const int64_t i = t0 + k;
        const int g = upper_index(A.regOff, A.G + 1, i);
        const int64_t idx = t++ - A.termBase[g];
        if (g >= A.G || idx >= 2 * (A.andBase[g + 1] - A.andBase[g])) continue;  // past the numbers
        int64_t st = i;
        while (st > A.regOff[g] && (A.buf[st - 1] & 0x80) && i - st < 4) st--;
        if (st > A.regOff[g] && (A.buf[st - 1] & 0x80)) {  // more than five bytes
            set_status(A.status, kDevAigerFormat);
            continue;
        }
        uint32_t x = 0;
        for (int64_t j = st; j <= i; j++) x |= (uint32_t)(A.buf[j] & 0x7f) << (7 * (int)(j - st));
        A.nums[2 * A.andBase[g] + idx] = x;
    }
}

// 4. fanins of every AND
__global__ void k_aig_ands(int64_t nAnd, int G, const int64_t *andBase, const int64_t *termBase, const DevGraph *dg,
                           const uint32_t *nums, int *F0, int *F1, int *status) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; a < nAnd; a += stride) {
        const int g = upper_index(andBase, G + 1, a);
        const int64_t i = a - andBase[g];
        if (termBase[g + 1] - termBase[g] < 2 * (andBase[g + 1] - andBase[g])) {  // too few numbers
            set_status(status, kDevAigerFormat);
            continue;
        }
        const DevGraph &d = dg[g];
        const uint32_t lhs = 2u * (uint32_t)(i + 1 + d.nPIs), d0 = nums[2 * a], d1 = nums[2 * a + 1];
        if (d0 > lhs || d0 == 0 || d1 > lhs - d0) {
            set_status(status, kDevAigerFormat);
            continue;
        }
        const uint32_t r1 = lhs - d0, r0 = r1 - d1;
        const int64_t p = (int64_t)d.base + 1 + d.nPIs + i;
        F0[p] = aig_inv_const((int)r0);
        F1[p] = aig_inv_const((int)r1);
    }
}

// encoding: byte lengths of every AND's two numbers
__global__ void k_aig_enc_len(int64_t nAnd, int G, const int64_t *andBase, const DevGraph *dg, const int *F0,
                              const int *F1, long long *len, int *status) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; a < nAnd; a += stride) {
        const int g = upper_index(andBase, G + 1, a);
        const DevGraph &d = dg[g];
        const int64_t i = a - andBase[g];
        const int64_t p = (int64_t)d.base + 1 + d.nPIs + i;
        int l0 = aig_inv_const(F0[p]), l1 = aig_inv_const(F1[p]);
        if (l0 > l1) {
            const int x = l0;
            l0 = l1;
            l1 = x;
        }
        const int64_t lhs = 2 * (1 + d.nPIs + i);
        if (l0 < 0 || lhs - l1 <= 0) {
            set_status(status, kDevBadGraph);
            len[a] = 0;
            continue;
        }
        len[a] = vlen((uint32_t)(lhs - l1)) + vlen((uint32_t)(l1 - l0));
    }
}

__device__ __forceinline__ void put_uint(uint8_t *out, int64_t &o, uint32_t x) {
    while (x & ~0x7fu) {
        out[o++] = (uint8_t)((x & 0x7f) | 0x80);
        x >>= 7;
    }
    out[o++] = (uint8_t)x;
}

__global__ void k_aig_enc_write(int64_t nAnd, int G, const int64_t *andBase, const DevGraph *dg, const int *F0,
                                const int *F1, const long long *off, uint8_t *out) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; a < nAnd; a += stride) {
        const int g = upper_index(andBase, G + 1, a);
        const DevGraph &d = dg[g];
        const int64_t i = a - andBase[g];
        const int64_t p = (int64_t)d.base + 1 + d.nPIs + i;
        int l0 = aig_inv_const(F0[p]), l1 = aig_inv_const(F1[p]);
        if (l0 > l1) {
            const int x = l0;
            l0 = l1;
            l1 = x;
        }
        const int64_t lhs = 2 * (1 + d.nPIs + i);
        if (l0 < 0 || lhs - l1 <= 0) continue;  // reported by k_aig_enc_len
        int64_t o = off[a];
        put_uint(out, o, (uint32_t)(lhs - l1));
        put_uint(out, o, (uint32_t)(l1 - l0));
    }
}

__global__ void k_gather_i64(int n, const int64_t *idx, const long long *src, long long *dst) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) dst[k] = src[idx[k]];
}

// Graphs [0, G) in at most `parts` contiguous runs of about equal weight,
// each run on its own host thread (the first on the caller's).
template <class W, class F>
void for_runs(int G, W weight, F fn) {
    int64_t total = 0;
    for (int g = 0; g < G; g++) total += weight(g);
    const unsigned hw = std::thread::hardware_concurrency();
    const int parts = total < (1 << 20) ? 1 : (int)std::max(1u, std::min({hw ? hw : 1u, 32u, (unsigned)G}));
    std::vector<int> cut{0};
    int64_t acc = 0;
    for (int g = 0; g < G; g++) {
        acc += weight(g);
        if ((int)cut.size() < parts && acc * parts >= total * (int64_t)cut.size() && g + 1 < G) cut.push_back(g + 1);
    }
    cut.push_back(G);
    // an exception of any run is rethrown here once every started thread has
    // been joined
    std::exception_ptr err;
    std::mutex mu;
    auto call = [&](size_t r) {
        try {
            fn(cut[r], cut[r + 1]);
        } catch (...) {
            std::lock_guard<std::mutex> lk(mu);
            if (!err) err = std::current_exception();
        }
    };
    std::vector<std::thread> th;
    try {
        for (size_t r = 1; r + 1 < cut.size(); r++) th.emplace_back(call, r);
    } catch (...) {
        for (auto &t : th) t.join();
        throw;
    }
    call(0);
    for (auto &t : th) t.join();
    if (err) std::rethrow_exception(err);
}

// Decimal digits of v >= 0 followed by '\n' at p; returns the end.
char *put_line(char *p, int v) {
    char t[12];
    int n = 0;
    do {
        t[n++] = (char)('0' + v % 10);
        v /= 10;
    } while (v);
    while (n) *p++ = t[--n];
    *p++ = '\n';
    return p;
}

int line_len(int v) {
    int n = 2;
    while (v >= 10) {
        v /= 10;
        n++;
    }
    return n;
}

// Host side of the header: "aig M I L O A\n" and O output lines; returns
// false on anything the host reader (host_aiger.cpp) refuses.
bool read_dec(const uint8_t *&p, const uint8_t *end, long long &v) {
    if (p >= end || *p < '0' || *p > '9') return false;
    v = 0;
    while (p < end && *p >= '0' && *p <= '9') {
        v = v * 10 + (*p - '0');
        if (v > INT32_MAX) return false;
        p++;
    }
    return true;
}

bool parse_head(const uint8_t *data, size_t len, int &nPIs, int &nPOs, int &nAnds, std::vector<int> &outs,
                size_t &body) {
    const uint8_t *p = data, *end = data + len;
    if (len < 4 || memcmp(p, "aig ", 4) != 0) return false;
    p += 4;
    long long M, I, L, O, A;
    if (!read_dec(p, end, M) || p >= end || *p++ != ' ') return false;
    if (!read_dec(p, end, I) || p >= end || *p++ != ' ') return false;
    if (!read_dec(p, end, L) || p >= end || *p++ != ' ') return false;
    if (!read_dec(p, end, O) || p >= end || *p++ != ' ') return false;
    if (!read_dec(p, end, A) || p >= end || *p++ != '\n') return false;
    if (L != 0 || M != I + A || M + 1 > INT32_MAX / 2) return false;
    nPIs = (int)I;
    nPOs = (int)O;
    nAnds = (int)A;
    outs.resize(nPOs);
    for (int i = 0; i < nPOs; i++) {
        long long lit;
        if (!read_dec(p, end, lit) || p >= end || *p++ != '\n') return false;
        if (lit >= 2 * (M + 1)) return false;
        outs[i] = aig_inv_const((int)lit);
    }
    body = (size_t)(p - data);
    return true;
}

}  // namespace

int Engine::upload_aiger(Batch &b, int count, const uint8_t *const *data, const size_t *len) {
    if (count < 1 || !data || !len) return fail(CULS_E_INVALID, "upload: no graphs");
    std::vector<DevGraph> hg(count);
    std::vector<std::vector<int>> outs(count);
    std::vector<int64_t> regOff(count + 1), andBase(count + 1);
    int64_t nObj = 0, nPO = 0, nAnd = 0, bytes = 0;
    std::vector<size_t> body(count);
    std::vector<int> head(3 * (size_t)count);
    std::atomic<int> bad{-1};
    for_runs(count, [&](int g) { return (int64_t)len[g] / 64 + 1; }, [&](int g0, int g1) {
        for (int g = g0; g < g1; g++)
            if (!data[g] || !parse_head(data[g], len[g], head[3 * g], head[3 * g + 1], head[3 * g + 2], outs[g], body[g])) {
                int none = -1;
                bad.compare_exchange_strong(none, g);
                return;
            }
    });
    if (bad.load() >= 0) return fail(CULS_E_IO, "upload: not binary AIGER (graph " + std::to_string(bad.load()) + ")");
    for (int g = 0; g < count; g++) {
        const int nPIs = head[3 * g], nPOs = head[3 * g + 1], nAnds = head[3 * g + 2];
        hg[g] = DevGraph{nPIs, nPOs, nAnds, 0, (int)nObj, (int)nPO, (int)nObj, 0};
        regOff[g] = bytes;
        andBase[g] = nAnd;
        bytes += (int64_t)(len[g] - body[g]);
        nObj += 1 + (int64_t)nPIs + nAnds;
        nPO += nPOs;
        nAnd += nAnds;
        if (nObj >= (1ll << 29)) return fail(CULS_E_INVALID, "upload: batch too large for 30-bit node positions");
    }
    regOff[count] = bytes;
    andBase[count] = nAnd;
    int rc;
    // staging: the number sections, then the output literals
    if ((rc = ensure_stage((size_t)(bytes + 3) / 4 + (size_t)nPO + 1))) return rc;
    uint8_t *sB = reinterpret_cast<uint8_t *>(stage_);
    int32_t *sPO = stage_ + (bytes + 3) / 4;
    for_runs(count, [&](int g) { return regOff[g + 1] - regOff[g] + 1; }, [&](int g0, int g1) {
        for (int g = g0; g < g1; g++) {
            memcpy(sB + regOff[g], data[g] + body[g], len[g] - body[g]);
            if (!outs[g].empty()) memcpy(sPO + hg[g].poOff, outs[g].data(), sizeof(int32_t) * outs[g].size());
        }
    });
    if (!b.pool) b.pool = pool_;
    if ((rc = check(b.reserve(nObj, nPO, count), "cudaMalloc"))) return rc;
    const int64_t nTiles = (bytes + kAigTile - 1) / kAigTile;
    if ((rc = ensure_arena((size_t)bytes + 8 * (size_t)nAnd + 16 * (size_t)(nTiles + count) + ((size_t)64 << 20))))
        return rc;
    ar_.reset();
    uint8_t *dB = ar_.get<uint8_t>(bytes + 1);
    int *tileCnt = ar_.get<int>(nTiles + 1);
    int64_t *tileBase = ar_.get<int64_t>(nTiles + 2);
    int64_t *dReg = ar_.get<int64_t>(count + 1), *dTerm = ar_.get<int64_t>(count + 1),
            *dAnd = ar_.get<int64_t>(count + 1);
    uint32_t *nums = ar_.get<uint32_t>(2 * nAnd + 1);
    if (!dB || !tileCnt || !tileBase || !dReg || !dTerm || !dAnd || !nums)
        return fail(CULS_E_OOM, "upload: arena exhausted (AIGER)");
    cudaStream_t s = s_;
    ExecCtx X = ctx();
    if ((rc = check(cudaMemcpyAsync(dB, sB, (size_t)bytes, cudaMemcpyHostToDevice, s), "h2d"))) return rc;
    if (nPO && (rc = check(cudaMemcpyAsync(b.PO, sPO, sizeof(int32_t) * nPO, cudaMemcpyHostToDevice, s), "h2d")))
        return rc;
    if ((rc = check(cudaMemcpyAsync(dReg, regOff.data(), sizeof(int64_t) * (count + 1), cudaMemcpyHostToDevice, s),
                    "h2d")))
        return rc;
    if ((rc = check(cudaMemcpyAsync(dAnd, andBase.data(), sizeof(int64_t) * (count + 1), cudaMemcpyHostToDevice, s),
                    "h2d")))
        return rc;
    if ((rc = check(cudaMemcpyAsync(b.dg, hg.data(), sizeof(DevGraph) * count, cudaMemcpyHostToDevice, s), "h2d")))
        return rc;
    if ((rc = check(fill_i32(b.F0, -1, nObj, s), "fill"))) return rc;
    if ((rc = check(fill_i32(b.F1, -1, nObj, s), "fill"))) return rc;
    if (nTiles > 0) {
        k_aig_count<<<(unsigned)nTiles, kAigThreads, 0, s>>>(dB, bytes, tileCnt);
        // tile bases as 64-bit values: a prefix over 32-bit counts, widened
        std::vector<int> hc(nTiles);
        if ((rc = check(cudaMemcpyAsync(hc.data(), tileCnt, sizeof(int) * nTiles, cudaMemcpyDeviceToHost, s), "d2h")))
            return rc;
        if ((rc = sync())) return rc;
        std::vector<int64_t> hb(nTiles + 2);
        hb[0] = 0;
        for (int64_t t = 0; t < nTiles; t++) hb[t + 1] = hb[t] + hc[t];
        hb[nTiles + 1] = hb[nTiles];
        if ((rc = check(cudaMemcpyAsync(tileBase, hb.data(), sizeof(int64_t) * (nTiles + 2), cudaMemcpyHostToDevice, s),
                        "h2d")))
            return rc;
    } else if ((rc = check(cudaMemsetAsync(tileBase, 0, sizeof(int64_t) * 2, s), "memset"))) {
        return rc;
    }
    k_aig_term_base<<<grid_1d(count + 1, kBlock, sms_ * 4), kBlock, 0, s>>>(count, dB, bytes, dReg, tileBase, dTerm);
    if (nTiles > 0)
        k_aig_numbers<<<(unsigned)nTiles, kAigThreads, 0, s>>>(
            AigDecode{dB, bytes, tileBase, count, dReg, dTerm, dAnd, nums, status_});
    if (nAnd > 0)
        k_aig_ands<<<X.grid(nAnd), kBlock, 0, s>>>(nAnd, count, dAnd, dTerm, b.dg, nums, b.F0, b.F1, status_);
    launches_ += 4;
    if ((rc = sync())) return rc;
    if ((rc = check_status("upload (AIGER)"))) return rc;
    b.G = count;
    b.nObj = nObj;
    b.nPO = nPO;
    b.hg = hg;
    // AIGMan::readFromMemory's nLevels: the depth of every graph
    return batch_depth(b);
}

int Engine::download_aiger(const Batch &b, uint8_t *buf, size_t cap, size_t *offsets) {
    const int G = b.G;
    int64_t nAnd = 0;
    std::vector<int64_t> andBase(G + 1);
    for (int g = 0; g < G; g++) {
        andBase[g] = nAnd;
        nAnd += b.hg[g].nAnds;
    }
    andBase[G] = nAnd;
    int rc;
    if ((rc = ensure_arena(24 * (size_t)nAnd + 10 * (size_t)nAnd + 16 * (size_t)G + ((size_t)64 << 20)))) return rc;
    ar_.reset();
    int64_t *dAnd = ar_.get<int64_t>(G + 1);
    long long *lenA = ar_.get<long long>(nAnd + 1), *offA = ar_.get<long long>(nAnd + 1),
              *gOff = ar_.get<long long>(G + 1), *tot = ar_.get<long long>(1);
    if (!dAnd || !lenA || !offA || !gOff || !tot) return fail(CULS_E_OOM, "download: arena exhausted (AIGER)");
    cudaStream_t s = s_;
    ExecCtx X = ctx();
    if ((rc = check(cudaMemcpyAsync(dAnd, andBase.data(), sizeof(int64_t) * (G + 1), cudaMemcpyHostToDevice, s), "h2d")))
        return rc;
    long long total = 0;
    if (nAnd > 0) {
        k_aig_enc_len<<<X.grid(nAnd), kBlock, 0, s>>>(nAnd, G, dAnd, b.dg, b.F0, b.F1, lenA, status_);
        if ((rc = check(scan_exclusive(lenA, offA, nAnd, tot, ar_, s), "scan"))) return rc;
        if ((rc = check(cudaMemcpyAsync(&hostSmall_[0], tot, sizeof(long long), cudaMemcpyDeviceToHost, s), "d2h")))
            return rc;
        if ((rc = sync())) return rc;
        if ((rc = check_status("download (AIGER)"))) return rc;
        memcpy(&total, hostSmall_, sizeof total);
    }
    uint8_t *dB = ar_.get<uint8_t>(total + 1);
    if (!dB) return fail(CULS_E_OOM, "download: arena exhausted (AIGER)");
    // the graphs' first bytes: offA at each graph's first AND (total past the last)
    std::vector<long long> hOff(G + 1, total);
    if (nAnd > 0) {
        if (buf) k_aig_enc_write<<<X.grid(nAnd), kBlock, 0, s>>>(nAnd, G, dAnd, b.dg, b.F0, b.F1, offA, dB);
        std::vector<int64_t> firstAnd;
        std::vector<int> which;
        for (int g = 0; g < G; g++)
            if (andBase[g] < nAnd) {
                firstAnd.push_back(andBase[g]);
                which.push_back(g);
            }
        int64_t *dIdx = ar_.get<int64_t>(firstAnd.size() + 1);
        if (!dIdx) return fail(CULS_E_OOM, "download: arena exhausted (AIGER)");
        if ((rc = check(cudaMemcpyAsync(dIdx, firstAnd.data(), sizeof(int64_t) * firstAnd.size(), cudaMemcpyHostToDevice,
                                        s),
                        "h2d")))
            return rc;
        k_gather_i64<<<grid_1d((int64_t)firstAnd.size(), kBlock, sms_ * 4), kBlock, 0, s>>>((int)firstAnd.size(), dIdx,
                                                                                          offA, gOff);
        std::vector<long long> hg(firstAnd.size());
        if ((rc = check(cudaMemcpyAsync(hg.data(), gOff, sizeof(long long) * hg.size(), cudaMemcpyDeviceToHost, s),
                        "d2h")))
            return rc;
        launches_ += 3;
        if ((rc = sync())) return rc;
        for (size_t k = 0; k < which.size(); k++) hOff[which[k]] = hg[k];
        for (int g = G - 1; g >= 0; g--)  // graphs without ANDs start where the next graph does
            if (b.hg[g].nAnds == 0) hOff[g] = hOff[g + 1];
    }
    if ((rc = ensure_stage((size_t)(total + 3) / 4 + (size_t)b.nPO + 1))) return rc;
    uint8_t *sB = reinterpret_cast<uint8_t *>(stage_);
    int32_t *sPO = stage_ + (total + 3) / 4;
    if (buf && total && (rc = check(cudaMemcpyAsync(sB, dB, (size_t)total, cudaMemcpyDeviceToHost, s), "d2h")))
        return rc;  // (the sizes need the numbers' lengths and the output literals only)
    if (b.nPO && (rc = check(cudaMemcpyAsync(sPO, b.PO, sizeof(int32_t) * b.nPO, cudaMemcpyDeviceToHost, s), "d2h")))
        return rc;
    if ((rc = sync())) return rc;
    // file g = header, output lines, numbers, "c\n"; files back to back
    std::vector<int> headLen(G);
    std::vector<int64_t> textLen(G);
    char hline[96];
    for (int g = 0; g < G; g++) {
        const DevGraph &d = b.hg[g];
        headLen[g] = snprintf(hline, sizeof hline, "aig %d %d 0 %d %d\n", d.nPIs + d.nAnds, d.nPIs, d.nPOs, d.nAnds);
    }
    for_runs(G, [&](int g) { return (int64_t)b.hg[g].nPOs + 1; }, [&](int g0, int g1) {
        for (int g = g0; g < g1; g++) {
            int64_t t = 0;
            for (int o = 0; o < b.hg[g].nPOs; o++) t += line_len(aig_inv_const(sPO[b.hg[g].poOff + o]));
            textLen[g] = t;
        }
    });
    offsets[0] = 0;
    for (int g = 0; g < G; g++)
        offsets[g + 1] = offsets[g] + (size_t)headLen[g] + (size_t)textLen[g] + (size_t)(hOff[g + 1] - hOff[g]) + 2;
    if (!buf) return 0;  // sizes only
    if (cap < offsets[G]) return fail(CULS_E_INVALID, "download: AIGER buffer too small");
    for_runs(G, [&](int g) { return (int64_t)(offsets[g + 1] - offsets[g]); }, [&](int g0, int g1) {
        char line[96];
        for (int g = g0; g < g1; g++) {
            const DevGraph &d = b.hg[g];
            char *p = reinterpret_cast<char *>(buf + offsets[g]);
            snprintf(line, sizeof line, "aig %d %d 0 %d %d\n", d.nPIs + d.nAnds, d.nPIs, d.nPOs, d.nAnds);
            memcpy(p, line, (size_t)headLen[g]);
            p += headLen[g];
            for (int o = 0; o < d.nPOs; o++) p = put_line(p, aig_inv_const(sPO[d.poOff + o]));
            memcpy(p, sB + hOff[g], (size_t)(hOff[g + 1] - hOff[g]));
            p += hOff[g + 1] - hOff[g];
            *p++ = 'c';
            *p++ = '\n';
        }
    });
    return 0;
}

}  // namespace culs
