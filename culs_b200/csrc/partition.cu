// SM partitions through green contexts (partition.cuh).  The driver entry
// points are looked up through the runtime (cudaGetDriverEntryPoint), so the
// library needs no link against the driver library.
#include <cuda.h>

#include "partition.cuh"

namespace culs {

namespace {

struct GreenApi {
    CUresult (*deviceGet)(CUdevice *, int) = nullptr;
    CUresult (*getResource)(CUdevice, CUdevResource *, CUdevResourceType) = nullptr;
    CUresult (*split)(CUdevResource *, unsigned *, const CUdevResource *, CUdevResource *, unsigned, unsigned) = nullptr;
    CUresult (*genDesc)(CUdevResourceDesc *, CUdevResource *, unsigned) = nullptr;
    CUresult (*create)(CUgreenCtx *, CUdevResourceDesc, CUdevice, unsigned) = nullptr;
    CUresult (*streamCreate)(CUstream *, CUgreenCtx, unsigned, int) = nullptr;
    CUresult (*destroy)(CUgreenCtx) = nullptr;
    CUresult (*streamDestroy)(CUstream) = nullptr;
    bool ok = false;
};

template <class F>
bool entry(const char *name, F &fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess ||
        !p) {
        cudaGetLastError();
        return false;
    }
    fn = reinterpret_cast<F>(p);
    return true;
}

GreenApi load_api() {
    GreenApi a;
    a.ok = entry("cuDeviceGet", a.deviceGet) && entry("cuDeviceGetDevResource", a.getResource) &&
           entry("cuDevSmResourceSplitByCount", a.split) && entry("cuDevResourceGenerateDesc", a.genDesc) &&
           entry("cuGreenCtxCreate", a.create) && entry("cuGreenCtxStreamCreate", a.streamCreate) &&
           entry("cuGreenCtxDestroy", a.destroy) && entry("cuStreamDestroy", a.streamDestroy);
    return a;
}

const GreenApi &api() {
    static const GreenApi a = load_api();
    return a;
}

}  // namespace

bool make_sm_partitions(int device, int n, std::vector<SmPartition> &out, std::string *why) {
    out.clear();
    auto no = [&](const char *w) {
        if (why) *why = w;
        destroy_sm_partitions(out);
        return false;
    };
    const GreenApi &g = api();
    if (n < 1 || !g.ok) return no("green contexts are not available");
    CUdevice dev;
    CUdevResource all;
    if (g.deviceGet(&dev, device) != CUDA_SUCCESS || g.getResource(dev, &all, CU_DEV_RESOURCE_TYPE_SM) != CUDA_SUCCESS)
        return no("cannot read the device's SM resources");
    // groups of the smallest partition size the hardware allows (8 SMs on
    // compute capability 9.0 and later), dealt out in turn
    unsigned nb = 0;
    if (g.split(nullptr, &nb, &all, nullptr, 0, 8) != CUDA_SUCCESS || nb < (unsigned)n)
        return no("fewer SM groups than partitions");
    std::vector<CUdevResource> grp(nb);
    CUdevResource rem{};
    if (g.split(grp.data(), &nb, &all, &rem, 0, 8) != CUDA_SUCCESS || nb < (unsigned)n)
        return no("SM split failed");
    for (int p = 0; p < n; p++) {
        std::vector<CUdevResource> mine;
        for (unsigned i = p; i < nb; i += (unsigned)n) mine.push_back(grp[i]);
        if (p == n - 1 && rem.sm.smCount > 0) mine.push_back(rem);
        int sms = 0;
        for (const CUdevResource &r : mine) sms += (int)r.sm.smCount;
        CUdevResourceDesc desc;
        CUgreenCtx ctx;
        if (g.genDesc(&desc, mine.data(), (unsigned)mine.size()) != CUDA_SUCCESS ||
            g.create(&ctx, desc, dev, CU_GREEN_CTX_DEFAULT_STREAM) != CUDA_SUCCESS)
            return no("green context creation failed");
        SmPartition part;
        part.green = ctx;
        part.sms = sms;
        out.push_back(part);
        CUstream st;
        if (g.streamCreate(&st, ctx, CU_STREAM_NON_BLOCKING, 0) != CUDA_SUCCESS) return no("green stream creation failed");
        out.back().stream = reinterpret_cast<cudaStream_t>(st);
    }
    return true;
}

void destroy_sm_partitions(std::vector<SmPartition> &parts) {
    const GreenApi &g = api();
    for (SmPartition &p : parts) {
        if (p.stream && g.streamDestroy) g.streamDestroy(reinterpret_cast<CUstream>(p.stream));
        if (p.green && g.destroy) g.destroy(static_cast<CUgreenCtx>(p.green));
        p.stream = nullptr;
        p.green = nullptr;
    }
    parts.clear();
}

}  // namespace culs
