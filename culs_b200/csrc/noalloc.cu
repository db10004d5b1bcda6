// culs_levels_noalloc: AIG level computation that allocates no memory.
//
// Some callers cannot call cudaMalloc: a host process whose device memory is
// owned and sized by another runtime, or an allocator-free embedding that
// must not fragment a device heap shared with other work.  For them this
// entry point computes the ASAP level of every object of one AIG (the same
// per-node recurrence as the levelization kernel of the rewriting pass,
// k_front_levelize in rw_front.cu) with its scratch -- completion flags,
// level words, a work counter, a status word and its spin bound -- in a
// fixed file-scope device array instead of the engine's arena.  The caller
// passes device pointers to the inputs and to the outputs.  The call
// synchronises the caller's stream and reads the status word back before it
// returns.
//
// Limits and sharing:
//  * at most CULS_LEVELS_NOALLOC_MAX_OBJS objects (1 + nPIs + nAnds); larger
//    graphs are refused with CULS_E_INVALID before anything is launched;
//  * the scratch array (about 8 MiB) is held by every GPU that loads the
//    library, until the process exits;
//  * every call uses the same array and it keeps the last call's contents;
//    each call clears what must start at zero.  Calls that overlap on the GPU
//    (different streams, or concurrent host threads) race on it and must be
//    serialised by the caller;
//  * the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) with that device current, so make that first
//    call before any stream capture begins.  The address is kept for the
//    life of the process: a device reset (cudaDeviceReset) in between
//    invalidates it, and calls after one are not supported.
#include <cuda_runtime.h>

#include <mutex>

#include "common.cuh"
#include "culs_b200.h"

namespace {

constexpr int kMaxObjs = CULS_LEVELS_NOALLOC_MAX_OBJS;
constexpr int kScratchInts = 2 * kMaxObjs + 64;  // done[], lp[], then counter / max level / status
constexpr int kBlockNA = 256;
constexpr int kMaxDevices = 64;

// The scratch.  Host code must not take this name as a device address; it
// uses the address cudaGetSymbolAddress returns for the current device.
static __device__ __align__(256) int g_levelsScratch[kScratchInts];

std::mutex g_mu;
int *g_scratchPtr[kMaxDevices] = {};

// Clears the completion flags and level words the dataflow pass relies on.
__global__ void k_na_init(int nObjs, int nPIs, int *done, int *lp, int *ctl) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nObjs; v += gridDim.x * blockDim.x) {
        bool lev0 = v <= nPIs;
        done[v] = lev0 ? 1 : 0;
        lp[v] = lev0 ? 0 : -1;
    }
    if (blockIdx.x == 0 && threadIdx.x < 4) ctl[threadIdx.x] = 0;
}

// Variant of k_front_levelize: the same in-order dataflow over a
// topologically ordered AIG (chunks claimed in increasing order, bounded
// waits on the fanins' completion flags), reading AIGMan literals of one
// graph and writing plain levels.  ctl = {counter, max level, status, spin
// bound}; the status and its spin bound are the pair culs::wait_ge reads.
__global__ void __launch_bounds__(kBlockNA) k_na_levelize(int nObjs, const int *f0, const int *f1, int *done, int *lp,
                                                           int *ctl, int *levels) {
    __shared__ int s_chunk;
    while (true) {
        if (threadIdx.x == 0) s_chunk = atomicAdd(&ctl[0], 1);
        __syncthreads();
        const long long start = (long long)s_chunk * kBlockNA;
        __syncthreads();
        if (start >= nObjs) break;
        const long long p = start + threadIdx.x;
        if (p >= nObjs) continue;
        if (lp[p] != -1) {  // constant or primary input
            levels[p] = 0;
            continue;
        }
        const int u0 = f0[p] >> 1, u1 = f1[p] >> 1;
        if (f0[p] < 0 || f1[p] < 0 || u0 >= p || u1 >= p) {
            culs::set_status(&ctl[2], culs::kDevBadGraph);
            culs::st_release(&done[p], 1);
            continue;
        }
        if (!culs::wait_ge(&done[u0], 1, &ctl[2]) || !culs::wait_ge(&done[u1], 1, &ctl[2])) continue;
        const int l0 = __ldcg(&lp[u0]), l1 = __ldcg(&lp[u1]);
        const int lv = 1 + (l0 > l1 ? l0 : l1);
        __stcg(&lp[p], lv);
        levels[p] = lv;
        atomicMax(&ctl[1], lv);
        __threadfence();
        culs::st_release(&done[p], 1);
    }
}

// Device address of the scratch array on the current device, looked up once
// per device (with that device current).
int scratch_for_current_device(int **out, int *devOut) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return CULS_E_DEVICE;
    *devOut = dev;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratchPtr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_levelsScratch);
        if (e != cudaSuccess || !p) return CULS_E_DEVICE;
        g_scratchPtr[dev] = static_cast<int *>(p);
    }
    *out = g_scratchPtr[dev];
    return CULS_OK;
}

}  // namespace

extern "C" int culs_levels_noalloc(const int32_t *d_fanin0, const int32_t *d_fanin1, int32_t nPIs, int32_t nAnds,
                                   int32_t *d_levels, int32_t *d_maxLevel, void *stream) {
    if (!d_fanin0 || !d_fanin1 || !d_levels || !d_maxLevel || nPIs < 0 || nAnds < 0) return CULS_E_INVALID;
    const long long nObjs = 1ll + nPIs + nAnds;
    if (nObjs > kMaxObjs) return CULS_E_INVALID;  // beyond the fixed scratch
    int *scratch = nullptr;
    int dev = 0;
    int rc = scratch_for_current_device(&scratch, &dev);
    if (rc != CULS_OK) return rc;
    int *done = scratch, *lp = scratch + kMaxObjs, *ctl = scratch + 2 * kMaxObjs;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int blocks = (int)((nObjs + kBlockNA - 1) / kBlockNA);
    if (blocks > 4096) blocks = 4096;
    k_na_init<<<blocks, kBlockNA, 0, s>>>((int)nObjs, nPIs, done, lp, ctl);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    k_na_levelize<<<sms * 4, kBlockNA, 0, s>>>((int)nObjs, d_fanin0, d_fanin1, done, lp, ctl, d_levels);
    if (cudaGetLastError() != cudaSuccess) return CULS_E_DEVICE;
    if (cudaMemcpyAsync(d_maxLevel, &ctl[1], sizeof(int32_t), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
        return CULS_E_DEVICE;
    int status = 0;
    if (cudaMemcpyAsync(&status, &ctl[2], sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess) return CULS_E_DEVICE;
    if (cudaStreamSynchronize(s) != cudaSuccess) return CULS_E_DEVICE;
    if (status == culs::kDevBadGraph) return CULS_E_INVALID;
    if (status != 0) return CULS_E_PROBE;
    return CULS_OK;
}
