// Device-wide scan, compaction and stable radix sort (see prim.cuh).
#include "prim.cuh"

namespace culs {

// ------------------------------------------------------------------ arena
Arena::~Arena() {
    if (base_) cudaFree(base_);
}

cudaError_t Arena::reserve(size_t bytes) {
    if (bytes <= cap_) return cudaSuccess;
    if (used_ != 0) return cudaErrorInvalidValue;
    if (base_) cudaFree(base_);
    base_ = nullptr;
    cap_ = 0;
    cudaError_t e = cudaMalloc(&base_, bytes);
    if (e != cudaSuccess) {
        base_ = nullptr;
        return e;
    }
    cap_ = bytes;
    return cudaSuccess;
}

void *Arena::alloc(size_t bytes) {
    size_t off = (used_ + 255) & ~(size_t)255;
    if (off + bytes > cap_) return nullptr;
    used_ = off + bytes;
    if (used_ > high_) high_ = used_;
    return base_ + off;
}

int num_sms() {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    return v > 0 ? v : 1;
}

// ------------------------------------------------------------------- scan
template <class T>
__device__ __forceinline__ T warp_incl_scan(T v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T n = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += n;
    }
    return v;
}

// Exclusive scan across the kScanThreads threads of a block.  sm needs 33
// entries.  Every thread gets the block total.
template <class T>
__device__ __forceinline__ T block_excl_scan(T v, T *sm, T &total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    T inc = warp_incl_scan(v);
    if (lane == 31) sm[w] = inc;
    __syncthreads();
    if (w == 0) {
        T s = lane < (kScanThreads / 32) ? sm[lane] : T(0);
        T si = warp_incl_scan(s);
        if (lane < (kScanThreads / 32)) sm[lane] = si - s;
        if (lane == 31) sm[32] = si;
    }
    __syncthreads();
    T res = sm[w] + inc - v;
    total = sm[32];
    __syncthreads();
    return res;
}

template <class T>
__global__ void __launch_bounds__(kScanThreads) k_tile_reduce(const T *in, int64_t n, T *sums) {
    __shared__ T sm[33];
    int64_t b = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    T s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++)
        if (b + k < n) s += in[b + k];
    T tot;
    block_excl_scan(s, sm, tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

template <class T>
__global__ void __launch_bounds__(kScanThreads) k_scan_single(T *a, int64_t m, T *total) {
    __shared__ T sm[33];
    T carry = 0;
    for (int64_t base = 0; base < m; base += kScanTile) {
        T v[kScanItems];
        T s = 0;
        int64_t b = base + (int64_t)threadIdx.x * kScanItems;
#pragma unroll
        for (int k = 0; k < kScanItems; k++) {
            v[k] = (b + k < m) ? a[b + k] : T(0);
            s += v[k];
        }
        T tot;
        T run = carry + block_excl_scan(s, sm, tot);
#pragma unroll
        for (int k = 0; k < kScanItems; k++)
            if (b + k < m) {
                a[b + k] = run;
                run += v[k];
            }
        carry += tot;
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

template <class T>
__global__ void __launch_bounds__(kScanThreads) k_tile_scan(const T *in, T *out, int64_t n, const T *offs) {
    __shared__ T sm[33];
    int64_t b = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    T v[kScanItems];
    T s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        v[k] = (b + k < n) ? in[b + k] : T(0);
        s += v[k];
    }
    T tot;
    T run = offs[blockIdx.x] + block_excl_scan(s, sm, tot);
#pragma unroll
    for (int k = 0; k < kScanItems; k++)
        if (b + k < n) {
            out[b + k] = run;
            run += v[k];
        }
}

size_t scan_scratch_bytes(int64_t n) { return (size_t)((n + kScanTile - 1) / kScanTile + 1) * 8 + 512; }

template <class T>
static cudaError_t scan_impl(const T *in, T *out, int64_t n, T *total, Arena &ar, cudaStream_t s) {
    if (n <= 0) {
        if (total) return cudaMemsetAsync(total, 0, sizeof(T), s);
        return cudaSuccess;
    }
    int64_t tiles = (n + kScanTile - 1) / kScanTile;
    size_t mark = ar.used();
    T *sums = ar.get<T>((size_t)tiles);
    if (!sums) return cudaErrorMemoryAllocation;
    k_tile_reduce<T><<<(unsigned)tiles, kScanThreads, 0, s>>>(in, n, sums);
    k_scan_single<T><<<1, kScanThreads, 0, s>>>(sums, tiles, total);
    k_tile_scan<T><<<(unsigned)tiles, kScanThreads, 0, s>>>(in, out, n, sums);
    (void)mark;
    return cudaGetLastError();
}

cudaError_t scan_exclusive(const int *in, int *out, int64_t n, int *total, Arena &ar, cudaStream_t s) {
    return scan_impl<int>(in, out, n, total, ar, s);
}
cudaError_t scan_exclusive(const long long *in, long long *out, int64_t n, long long *total, Arena &ar,
                           cudaStream_t s) {
    return scan_impl<long long>(in, out, n, total, ar, s);
}

// ------------------------------------------------------------- compaction
__global__ void __launch_bounds__(kScanThreads) k_flag_count(const uint8_t *flags, int64_t n, int *sums) {
    __shared__ int sm[33];
    int64_t b = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++)
        if (b + k < n) s += flags[b + k] != 0;
    int tot;
    block_excl_scan(s, sm, tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kScanThreads) k_flag_scatter(const uint8_t *flags, int64_t n, const int *offs,
                                                                int *outIdx) {
    __shared__ int sm[33];
    int64_t b = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    uint8_t f[kScanItems];
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        f[k] = (b + k < n) ? flags[b + k] : 0;
        s += f[k] != 0;
    }
    int tot;
    int run = offs[blockIdx.x] + block_excl_scan(s, sm, tot);
#pragma unroll
    for (int k = 0; k < kScanItems; k++)
        if (f[k]) outIdx[run++] = (int)(b + k);
}

cudaError_t compact_flags(const uint8_t *flags, int64_t n, int *outIdx, int *count, Arena &ar, cudaStream_t s) {
    if (n <= 0) return cudaMemsetAsync(count, 0, sizeof(int), s);
    int64_t tiles = (n + kScanTile - 1) / kScanTile;
    int *sums = ar.get<int>((size_t)tiles);
    if (!sums) return cudaErrorMemoryAllocation;
    k_flag_count<<<(unsigned)tiles, kScanThreads, 0, s>>>(flags, n, sums);
    k_scan_single<int><<<1, kScanThreads, 0, s>>>(sums, tiles, count);
    k_flag_scatter<<<(unsigned)tiles, kScanThreads, 0, s>>>(flags, n, sums, outIdx);
    return cudaGetLastError();
}

// ------------------------------------------------------------- radix sort
constexpr int kRadixThreads = 256;
constexpr int kRadixRounds = 16;
constexpr int kRadixTile = kRadixThreads * kRadixRounds;

__global__ void __launch_bounds__(kRadixThreads) k_radix_hist(const uint32_t *keys, int64_t n, int shift, int *hist,
                                                               int numTiles) {
    __shared__ int h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    int64_t base = (int64_t)blockIdx.x * kRadixTile;
    for (int i = threadIdx.x; i < kRadixTile; i += kRadixThreads) {
        int64_t k = base + i;
        if (k < n) atomicAdd(&h[(keys[k] >> shift) & 255u], 1);
    }
    __syncthreads();
    hist[(int64_t)threadIdx.x * numTiles + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter: element order inside the tile is round-major, then thread
// index, which is the input order.
__global__ void __launch_bounds__(kRadixThreads) k_radix_scatter(const uint32_t *keysIn, const int *valsIn,
                                                                  uint32_t *keysOut, int *valsOut, int64_t n,
                                                                  int shift, const int *histScan, int numTiles) {
    __shared__ int s_base[256];
    __shared__ int s_w[kRadixThreads / 32][256];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    s_base[tid] = histScan[(int64_t)tid * numTiles + blockIdx.x];
    int64_t base = (int64_t)blockIdx.x * kRadixTile;
    const unsigned lt = (1u << lane) - 1u;
    for (int r = 0; r < kRadixRounds; r++) {
#pragma unroll
        for (int k = 0; k < kRadixThreads / 32; k++) s_w[k][tid] = 0;
        __syncthreads();
        int64_t idx = base + (int64_t)r * kRadixThreads + tid;
        bool valid = idx < n;
        uint32_t key = valid ? keysIn[idx] : 0u;
        int val = valid ? valsIn[idx] : 0;
        uint32_t d = valid ? ((key >> shift) & 255u) : 0x100u;
        unsigned peers = __match_any_sync(0xffffffffu, d);
        int rank = __popc(peers & lt);
        if (valid && rank == 0) s_w[w][d] = __popc(peers);
        __syncthreads();
        {
            int run = s_base[tid];
#pragma unroll
            for (int k = 0; k < kRadixThreads / 32; k++) {
                int c = s_w[k][tid];
                s_w[k][tid] = run;
                run += c;
            }
            s_base[tid] = run;
        }
        __syncthreads();
        if (valid) {
            int pos = s_w[w][d] + rank;
            keysOut[pos] = key;
            valsOut[pos] = val;
        }
        __syncthreads();
    }
}

cudaError_t radix_sort_pairs(uint32_t *keys, int *vals, uint32_t *keysOut, int *valsOut, int64_t n, int keyBits,
                             Arena &ar, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    int passes = (keyBits + 7) / 8;
    int numTiles = (int)((n + kRadixTile - 1) / kRadixTile);
    uint32_t *srcK = keys, *dstK = keysOut;
    int *srcV = vals, *dstV = valsOut;
    size_t mark = ar.used();
    int *hist = ar.get<int>((size_t)numTiles * 256);
    if (!hist) return cudaErrorMemoryAllocation;
    for (int p = 0; p < passes; p++) {
        int shift = 8 * p;
        k_radix_hist<<<numTiles, kRadixThreads, 0, s>>>(srcK, n, shift, hist, numTiles);
        cudaError_t e = scan_exclusive(hist, hist, (int64_t)numTiles * 256, nullptr, ar, s);
        if (e != cudaSuccess) return e;
        k_radix_scatter<<<numTiles, kRadixThreads, 0, s>>>(srcK, srcV, dstK, dstV, n, shift, hist, numTiles);
        uint32_t *tk = srcK;
        srcK = dstK;
        dstK = tk;
        int *tv = srcV;
        srcV = dstV;
        dstV = tv;
    }
    (void)mark;
    if (srcK != keysOut) {
        cudaMemcpyAsync(keysOut, srcK, sizeof(uint32_t) * (size_t)n, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(valsOut, srcV, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, s);
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------- fills
__global__ void k_fill_i32(int *d, int v, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        d[i] = v;
}
__global__ void k_fill_i4(int4 *d, int4 v, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        d[i] = v;
}
__global__ void k_iota_i32(int *d, int start, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        d[i] = start + (int)i;
}

static unsigned grid_for(int64_t n) {
    int64_t b = (n + 255) / 256;
    int64_t cap = (int64_t)num_sms() * 8;
    if (b > cap) b = cap;
    return (unsigned)(b < 1 ? 1 : b);
}

cudaError_t fill_i32(int *dst, int v, int64_t n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_fill_i32<<<grid_for(n), 256, 0, s>>>(dst, v, n);
    return cudaGetLastError();
}
cudaError_t fill_i4(int4 *dst, int4 v, int64_t n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_fill_i4<<<grid_for(n), 256, 0, s>>>(dst, v, n);
    return cudaGetLastError();
}
cudaError_t iota_i32(int *dst, int start, int64_t n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_iota_i32<<<grid_for(n), 256, 0, s>>>(dst, start, n);
    return cudaGetLastError();
}

}  // namespace culs
