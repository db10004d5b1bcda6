// C ABI (include/culs_b200.h) over the batch engine.
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "culs_b200.h"
#include "engine.cuh"
#include "guard.hpp"
#include "serve.cuh"

struct culs_ctx {
    culs::Engine eng;
    std::mutex mu;  // the engine owns one stream; calls on a context serialise
    culs::RwStats last{};
    culs::RwDump dump;
    std::string err;
    // served mode; its worker takes `mu` for every batch, so the pointer has
    // a lock of its own, and callers hold a reference while they use it
    std::mutex srvMu;
    std::shared_ptr<culs::Server> srv;  // destroyed first: finishes queued jobs
};

struct culs_graph {
    culs::Batch b;
    culs_ctx *owner = nullptr;
};

namespace {
thread_local std::string g_err;

int set_err(culs_ctx *c, int rc) {
    if (rc != CULS_OK && c) c->err = c->eng.error();
    return rc;
}
}  // namespace

extern "C" {

int culs_set_device(int device) {
    return culs::guard_call(&g_err, [&]() -> int {
        cudaError_t e = cudaSetDevice(device);
        if (e != cudaSuccess) {
            g_err = cudaGetErrorString(e);
            return CULS_E_DEVICE;
        }
        return CULS_OK;
    });
}

culs_ctx *culs_create(size_t hbm_budget) {
    culs_ctx *out = nullptr;
    culs::guard_call(&g_err, [&]() -> int {
        auto c = std::make_unique<culs_ctx>();
        int rc = c->eng.init(hbm_budget);
        if (rc != CULS_OK) {
            g_err = c->eng.error();
            return rc;
        }
        out = c.release();
        return CULS_OK;
    });
    return out;
}

void culs_destroy(culs_ctx *ctx) { delete ctx; }

const char *culs_last_error(culs_ctx *ctx) { return ctx ? ctx->err.c_str() : g_err.c_str(); }

int culs_graph_upload(culs_ctx *ctx, const int32_t *fanin0, const int32_t *fanin1, const int32_t *outs, int32_t nPIs,
                      int32_t nPOs, int32_t nAnds, culs_graph **g) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx || !g || (!fanin0 && nAnds) || (!fanin1 && nAnds) || (!outs && nPOs)) return CULS_E_INVALID;
        std::lock_guard<std::mutex> lk(ctx->mu);
        auto h = std::make_unique<culs_graph>();
        h->owner = ctx;
        int32_t zero = 0;
        const int32_t *p0 = fanin0 ? fanin0 : &zero, *p1 = fanin1 ? fanin1 : &zero, *po = outs ? outs : &zero;
        int rc = ctx->eng.upload(h->b, 1, &p0, &p1, &po, &nPIs, &nPOs, &nAnds);
        if (rc != CULS_OK) return set_err(ctx, rc);
        *g = h.release();
        return CULS_OK;
    });
}

int culs_batch_upload(culs_ctx *ctx, int count, const culs_host_graph *graphs, culs_graph **g) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx || !g || !graphs || count < 1) return CULS_E_INVALID;
        std::lock_guard<std::mutex> lk(ctx->mu);
        std::vector<const int32_t *> p0(count), p1(count), po(count);
        std::vector<int32_t> nPI(count), nPO(count), nA(count);
        int32_t zero = 0;
        for (int i = 0; i < count; i++) {
            p0[i] = graphs[i].fanin0 ? graphs[i].fanin0 : &zero;
            p1[i] = graphs[i].fanin1 ? graphs[i].fanin1 : &zero;
            po[i] = graphs[i].outs ? graphs[i].outs : &zero;
            nPI[i] = graphs[i].nPIs;
            nPO[i] = graphs[i].nPOs;
            nA[i] = graphs[i].nAnds;
        }
        auto h = std::make_unique<culs_graph>();
        h->owner = ctx;
        int rc = ctx->eng.upload(h->b, count, p0.data(), p1.data(), po.data(), nPI.data(), nPO.data(), nA.data());
        if (rc != CULS_OK) return set_err(ctx, rc);
        *g = h.release();
        return CULS_OK;
    });
}

void culs_graph_free(culs_graph *g) { delete g; }

int culs_graph_count(const culs_graph *g) { return g ? g->b.G : 0; }

int culs_graph_stats(const culs_graph *g, int index, int32_t *nPIs, int32_t *nPOs, int32_t *nAnds, int32_t *nLevels) {
    return culs::guard_call(&g_err, [&]() -> int {
        if (!g || index < 0 || index >= g->b.G) return CULS_E_INVALID;
        const culs::DevGraph &d = g->b.hg[index];
        if (nPIs) *nPIs = d.nPIs;
        if (nPOs) *nPOs = d.nPOs;
        if (nAnds) *nAnds = d.nAnds;
        if (nLevels) *nLevels = d.nLevels;
        return CULS_OK;
    });
}

int culs_batch_upload_aiger(culs_ctx *ctx, int count, const uint8_t *const *data, const size_t *len,
                            culs_graph **g) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx || !g || count < 1 || !data || !len) return CULS_E_INVALID;
        *g = nullptr;
        auto h = std::make_unique<culs_graph>();
        h->owner = ctx;
        std::lock_guard<std::mutex> lk(ctx->mu);
        const int rc = set_err(ctx, ctx->eng.upload_aiger(h->b, count, data, len));
        if (rc == CULS_OK) *g = h.release();
        return rc;
    });
}

int culs_batch_download_aiger_into(culs_ctx *ctx, const culs_graph *g, uint8_t *buf, size_t cap, size_t *offsets) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx || !g || !offsets) return CULS_E_INVALID;
        std::lock_guard<std::mutex> lk(ctx->mu);
        return set_err(ctx, ctx->eng.download_aiger(g->b, buf, cap, offsets));
    });
}

int culs_batch_download_aiger(culs_ctx *ctx, const culs_graph *g, uint8_t **data, size_t *len) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx || !g || !data || !len) return CULS_E_INVALID;
        const int G = g->b.G;
        std::vector<size_t> off(G + 1);
        int rc = culs_batch_download_aiger_into(ctx, g, nullptr, 0, off.data());
        if (rc != CULS_OK) return rc;
        uint8_t *all = static_cast<uint8_t *>(malloc(off[G] ? off[G] : 1));
        if (!all) return CULS_E_OOM;
        rc = culs_batch_download_aiger_into(ctx, g, all, off[G], off.data());
        for (int i = 0; i < G && rc == CULS_OK; i++) {
            data[i] = static_cast<uint8_t *>(malloc(off[i + 1] - off[i] ? off[i + 1] - off[i] : 1));
            if (!data[i]) {
                for (int j = 0; j < i; j++) free(data[j]);
                rc = CULS_E_OOM;
                break;
            }
            memcpy(data[i], all + off[i], off[i + 1] - off[i]);
            len[i] = off[i + 1] - off[i];
        }
        free(all);
        return rc;
    });
}

void culs_buffer_free(void *p) { free(p); }

int culs_batch_stats(const culs_graph *g, int32_t *nPIs, int32_t *nPOs, int32_t *nAnds, int32_t *nLevels) {
    return culs::guard_call(&g_err, [&]() -> int {
        if (!g) return CULS_E_INVALID;
        for (int i = 0; i < g->b.G; i++) {
            const culs::DevGraph &d = g->b.hg[i];
            if (nPIs) nPIs[i] = d.nPIs;
            if (nPOs) nPOs[i] = d.nPOs;
            if (nAnds) nAnds[i] = d.nAnds;
            if (nLevels) nLevels[i] = d.nLevels;
        }
        return CULS_OK;
    });
}

int culs_graph_download(culs_ctx *ctx, const culs_graph *g, int index, int32_t *fanin0, int32_t *fanin1,
                        int32_t *outs) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx || !g) return CULS_E_INVALID;
        std::lock_guard<std::mutex> lk(ctx->mu);
        return set_err(ctx, ctx->eng.download(g->b, index, fanin0, fanin1, outs));
    });
}

int culs_batch_download(culs_ctx *ctx, const culs_graph *g, culs_host_graph *outs) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx || !g || !outs) return CULS_E_INVALID;
        std::lock_guard<std::mutex> lk(ctx->mu);
        const culs::Batch &b = g->b;
        std::vector<int32_t *> f0(b.G), f1(b.G), po(b.G);
        bool oom = false;
        for (int i = 0; i < b.G; i++) {
            const culs::DevGraph &d = b.hg[i];
            const size_t n = 1 + (size_t)d.nPIs + d.nAnds;
            culs_host_graph &o = outs[i];
            o.nPIs = d.nPIs;
            o.nPOs = d.nPOs;
            o.nAnds = d.nAnds;
            o.fanin0 = f0[i] = (int32_t *)malloc(sizeof(int32_t) * n);
            o.fanin1 = f1[i] = (int32_t *)malloc(sizeof(int32_t) * n);
            o.outs = po[i] = (int32_t *)malloc(sizeof(int32_t) * (d.nPOs > 0 ? d.nPOs : 1));
            oom |= !o.fanin0 || !o.fanin1 || !o.outs;
        }
        if (oom) return CULS_E_OOM;
        return set_err(ctx, ctx->eng.download_all(b, f0.data(), f1.data(), po.data()));
    });
}

int culs_batch_download_into(culs_ctx *ctx, const culs_graph *g, int32_t *const *fanin0, int32_t *const *fanin1,
                             int32_t *const *outs) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx || !g) return CULS_E_INVALID;
        std::lock_guard<std::mutex> lk(ctx->mu);
        return set_err(ctx, ctx->eng.download_all(g->b, fanin0, fanin1, outs));
    });
}

int culs_rw(culs_ctx *ctx, culs_graph *g, uint32_t flags) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx || !g) return CULS_E_INVALID;
        std::lock_guard<std::mutex> lk(ctx->mu);
        ctx->dump.enabled = (flags & CULS_RW_DUMP) != 0;
        int rc = ctx->eng.rw(g->b, (flags & CULS_RW_ZEROS) != 0, (flags & CULS_RW_GPU_DEDUP) != 0, &ctx->last, &ctx->dump);
        return set_err(ctx, rc);
    });
}

int culs_st(culs_ctx *ctx, culs_graph *g, uint32_t flags) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx || !g) return CULS_E_INVALID;
        std::lock_guard<std::mutex> lk(ctx->mu);
        return set_err(ctx, ctx->eng.st(g->b, (flags & CULS_ST_CPU) != 0));
    });
}

int culs_b(culs_ctx *ctx, culs_graph *g, uint32_t flags) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx || !g || (flags & ~CULS_B_NO_STRASH)) return CULS_E_INVALID;
        std::lock_guard<std::mutex> lk(ctx->mu);
        return set_err(ctx, ctx->eng.balance(g->b, (flags & CULS_B_NO_STRASH) == 0));
    });
}

int culs_rw_st(culs_ctx *ctx, culs_graph *g, uint32_t rwFlags, uint32_t stFlags) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        int rc = culs_rw(ctx, g, rwFlags);
        if (rc != CULS_OK) return rc;
        return culs_st(ctx, g, stFlags);
    });
}

int culs_rw_st_batch(culs_ctx *ctx, culs_graph *const *gs, int count, uint32_t rwFlags, uint32_t stFlags) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx || !gs || count < 1) return CULS_E_INVALID;
        std::vector<const culs::Batch *> in;
        std::vector<culs::Batch *> out;
        for (int i = 0; i < count; i++) {
            if (!gs[i]) return CULS_E_INVALID;
            for (int k = 0; k < i; k++)
                if (gs[k] == gs[i]) return CULS_E_INVALID;  // a handle listed twice
            in.push_back(&gs[i]->b);
            out.push_back(&gs[i]->b);
        }
        std::lock_guard<std::mutex> lk(ctx->mu);
        culs::Batch all;
        int rc = ctx->eng.concat(in, all);
        if (rc == CULS_OK)
            rc = ctx->eng.rw(all, (rwFlags & CULS_RW_ZEROS) != 0, (rwFlags & CULS_RW_GPU_DEDUP) != 0, &ctx->last,
                             nullptr);
        if (rc == CULS_OK) rc = ctx->eng.st(all, (stFlags & CULS_ST_CPU) != 0);
        if (rc == CULS_OK) rc = ctx->eng.split(all, out);
        return set_err(ctx, rc);
    });
}

namespace {
std::shared_ptr<culs::Server> server_of(culs_ctx *ctx) {
    std::lock_guard<std::mutex> lk(ctx->srvMu);
    return ctx->srv;
}
}  // namespace

int culs_serve_start(culs_ctx *ctx, size_t admitBytes, int maxBatch, int workers) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx) return CULS_E_INVALID;
        std::lock_guard<std::mutex> lk(ctx->srvMu);
        if (ctx->srv) return CULS_E_INVALID;
        if (admitBytes == 0) admitBytes = ctx->eng.budget();
        if (workers <= 0) workers = 2;
        int dev = 0;
        cudaGetDevice(&dev);
        cudaSetDevice(ctx->eng.device());  // the server's own engines live beside the context's
        ctx->srv = std::make_shared<culs::Server>(ctx->eng, ctx->mu, admitBytes, maxBatch, workers);
        cudaSetDevice(dev);
        return CULS_OK;
    });
}

int culs_serve_stop(culs_ctx *ctx) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx) return CULS_E_INVALID;
        std::shared_ptr<culs::Server> s;
        {
            std::lock_guard<std::mutex> lk(ctx->srvMu);
            s.swap(ctx->srv);
        }
        return s ? CULS_OK : CULS_E_INVALID;  // the last reference finishes the queue
    });
}

int culs_submit(culs_ctx *ctx, const int32_t *fanin0, const int32_t *fanin1, const int32_t *outs, int32_t nPIs,
                int32_t nPOs, int32_t nAnds, uint32_t rwFlags, uint32_t stFlags, int64_t *job) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx) return CULS_E_INVALID;
        auto s = server_of(ctx);
        if (!s) return CULS_E_INVALID;
        return s->submit(fanin0, fanin1, outs, nPIs, nPOs, nAnds, rwFlags, stFlags, job);
    });
}

int culs_submit_aiger(culs_ctx *ctx, const uint8_t *data, size_t len, uint32_t rwFlags, uint32_t stFlags,
                      int64_t *job) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx) return CULS_E_INVALID;
        auto s = server_of(ctx);
        if (!s) return CULS_E_INVALID;
        return s->submit_aiger(data, len, rwFlags, stFlags, job);
    });
}

int culs_fetch_aiger(culs_ctx *ctx, int64_t job, uint8_t *buf, size_t cap, size_t *len, double *latencyMs) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx) return CULS_E_INVALID;
        auto s = server_of(ctx);
        if (!s) return CULS_E_NOTFOUND;
        int rc = s->fetch_aiger(job, buf, cap, len, latencyMs);
        if (rc < 0 && rc != CULS_E_BUSY && rc != CULS_E_NOTFOUND) {
            std::lock_guard<std::mutex> lk(ctx->mu);
            ctx->err = s->lastError();
        }
        return rc;
    });
}

int culs_poll(culs_ctx *ctx, int64_t job, int32_t *nPIs, int32_t *nPOs, int32_t *nAnds, int32_t *nLevels) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx) return CULS_E_INVALID;
        auto s = server_of(ctx);
        if (!s) return CULS_E_NOTFOUND;
        return s->poll(job, nPIs, nPOs, nAnds, nLevels);
    });
}

int culs_cancel(culs_ctx *ctx, int64_t job) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx) return CULS_E_INVALID;
        auto s = server_of(ctx);
        if (!s) return CULS_E_NOTFOUND;
        return s->cancel(job);
    });
}

int culs_wait(culs_ctx *ctx, int64_t job, int timeoutMs) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx) return CULS_E_INVALID;
        auto s = server_of(ctx);
        if (!s) return CULS_E_NOTFOUND;
        return s->wait(job, timeoutMs);
    });
}

int culs_fetch(culs_ctx *ctx, int64_t job, int32_t *fanin0, int32_t *fanin1, int32_t *outs, double *latencyMs) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx) return CULS_E_INVALID;
        auto s = server_of(ctx);
        if (!s) return CULS_E_NOTFOUND;
        int rc = s->fetch(job, fanin0, fanin1, outs, latencyMs);
        if (rc < 0 && rc != CULS_E_BUSY && rc != CULS_E_NOTFOUND) {
            std::lock_guard<std::mutex> lk(ctx->mu);
            ctx->err = s->lastError();
        }
        return rc;
    });
}

int culs_set_param(culs_ctx *ctx, int which, int64_t value) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx) return CULS_E_INVALID;
        std::lock_guard<std::mutex> lk(ctx->mu);
        culs::Tune &t = ctx->eng.tune();
        switch (which) {
            case CULS_PARAM_ENUM_WIDE_MIN:
                if (value < 1 || value > (1ll << 30)) return CULS_E_INVALID;
                t.enumWideMin = (int)value;
                return CULS_OK;
            case CULS_PARAM_ENUM_BLOCKS_PER_SM:
                if (value < 1 || value > 64) return CULS_E_INVALID;
                t.enumBlocksPerSm = (int)value;
                return CULS_OK;
            case CULS_PARAM_SM_SHARE:
                if (value < 1 || value > 64) return CULS_E_INVALID;
                ctx->eng.set_sm_share((int)value);
                return CULS_OK;
            case CULS_PARAM_HIGH_PRIORITY:
                if (value != 0 && value != 1) return CULS_E_INVALID;
                return set_err(ctx, ctx->eng.set_high_priority(value != 0));
            case CULS_PARAM_EVAL_GROUP_MSLOTS:
                if (value < 1 || value > 1024) return CULS_E_INVALID;
                t.evalGroupMSlots = (int)value;
                return CULS_OK;
            default:
                return CULS_E_INVALID;
        }
    });
}

int culs_get_param(culs_ctx *ctx, int which, int64_t *value) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx || !value) return CULS_E_INVALID;
        std::lock_guard<std::mutex> lk(ctx->mu);
        const culs::Tune &t = ctx->eng.tune();
        switch (which) {
            case CULS_PARAM_ENUM_WIDE_MIN: *value = t.enumWideMin; return CULS_OK;
            case CULS_PARAM_ENUM_BLOCKS_PER_SM: *value = t.enumBlocksPerSm; return CULS_OK;
            case CULS_PARAM_SM_SHARE: *value = ctx->eng.sm_share(); return CULS_OK;
            case CULS_PARAM_HIGH_PRIORITY: *value = ctx->eng.high_priority() ? 1 : 0; return CULS_OK;
            case CULS_PARAM_EVAL_GROUP_MSLOTS: *value = t.evalGroupMSlots; return CULS_OK;
            default: return CULS_E_INVALID;
        }
    });
}

int culs_autotune(culs_ctx *ctx, const culs_graph *sample, int rounds) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx || !sample) return CULS_E_INVALID;
        std::lock_guard<std::mutex> lk(ctx->mu);
        return set_err(ctx, ctx->eng.autotune(sample->b, rounds));
    });
}

int culs_rw_stats(culs_ctx *ctx, int64_t *out, int n) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx || !out) return CULS_E_INVALID;
        const culs::RwStats &s = ctx->last;
        int64_t v[13] = {s.replaced, s.replacedPos, s.replacedZero, s.reverted,   s.compromised,
                         s.preEval,  s.smallCut,    s.newIdx,       s.expected,   s.newNodes,
                         s.candidates, s.warpPairs, s.hashRounds};
        for (int i = 0; i < n && i < 13; i++) out[i] = v[i];
        return CULS_OK;
    });
}

int64_t culs_dump_size(culs_ctx *ctx, int which) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int64_t {
        if (!ctx) return -1;
        const culs::RwDump &d = ctx->dump;
        switch (which) {
            case CULS_DUMP_REORDER_F0: return (int64_t)d.reorderF0.size();
            case CULS_DUMP_REORDER_F1: return (int64_t)d.reorderF1.size();
            case CULS_DUMP_REORDER_OUT: return (int64_t)d.reorderOut.size();
            case CULS_DUMP_CUTS: return (int64_t)d.cuts.size();
            case CULS_DUMP_SELECTED: return (int64_t)d.selected.size();
            case CULS_DUMP_REPLACE: return (int64_t)d.replace.size();
            case CULS_DUMP_NEW_F0: return (int64_t)d.newF0.size();
            case CULS_DUMP_NEW_F1: return (int64_t)d.newF1.size();
            case CULS_DUMP_CHOICE: return (int64_t)d.choice.size();
            default: return -1;
        }
    });
}

int culs_dump_copy(culs_ctx *ctx, int which, int32_t *out) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx || !out) return CULS_E_INVALID;
        const culs::RwDump &d = ctx->dump;
        const std::vector<int> *v = nullptr;
        switch (which) {
            case CULS_DUMP_REORDER_F0: v = &d.reorderF0; break;
            case CULS_DUMP_REORDER_F1: v = &d.reorderF1; break;
            case CULS_DUMP_REORDER_OUT: v = &d.reorderOut; break;
            case CULS_DUMP_CUTS: v = &d.cuts; break;
            case CULS_DUMP_SELECTED: v = &d.selected; break;
            case CULS_DUMP_REPLACE: v = &d.replace; break;
            case CULS_DUMP_NEW_F0: v = &d.newF0; break;
            case CULS_DUMP_NEW_F1: v = &d.newF1; break;
            case CULS_DUMP_CHOICE: v = &d.choice; break;
            default: return CULS_E_INVALID;
        }
        if (!v->empty()) memcpy(out, v->data(), sizeof(int32_t) * v->size());
        return CULS_OK;
    });
}

int64_t culs_kernel_launches(culs_ctx *ctx) { return ctx ? ctx->eng.kernelLaunches() : 0; }

int culs_graph_clone(culs_ctx *ctx, const culs_graph *src, culs_graph **dst) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx || !src || !dst) return CULS_E_INVALID;
        std::lock_guard<std::mutex> lk(ctx->mu);
        std::unique_ptr<culs_graph> fresh(*dst ? nullptr : new culs_graph());
        culs_graph *h = *dst ? *dst : fresh.get();
        h->owner = ctx;
        int rc = ctx->eng.clone(src->b, h->b);
        if (rc != CULS_OK) return set_err(ctx, rc);
        if (fresh) *dst = fresh.release();
        return CULS_OK;
    });
}

int culs_profile(culs_ctx *ctx, int enable) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx) return CULS_E_INVALID;
        ctx->eng.setProfile(enable != 0);
        return CULS_OK;
    });
}

int culs_mark(culs_ctx *ctx, int slot) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx || slot < 0 || slot > 1) return CULS_E_INVALID;
        ctx->eng.mark(culs::kMkUser0 + slot);
        return CULS_OK;
    });
}

int culs_profile_read(culs_ctx *ctx, float *ms, int n) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx || !ms) return CULS_E_INVALID;
        using namespace culs;
        const int pairs[][2] = {{kMkRwStart, kMkFront}, {kMkFront, kMkEnum},     {kMkEnum, kMkEval},
                                {kMkEval, kMkReplace},  {kMkReplace, kMkChoice}, {kMkChoice, kMkRedund},
                                {kMkRedund, kMkRwEnd},  {kMkStStart, kMkStEnd},  {kMkEnumK0, kMkEnumK1},
                                {kMkEvalK0, kMkEvalK1}, {kMkDedupK0, kMkDedupK1}, {kMkUser0, kMkUser1},
                                {kMkLevelK0, kMkLevelK1}};
        const int np = (int)(sizeof pairs / sizeof pairs[0]);
        for (int i = 0; i < n && i < np; i++) ms[i] = ctx->eng.elapsed(pairs[i][0], pairs[i][1]);
        return CULS_OK;
    });
}

int culs_sync(culs_ctx *ctx) {
    return culs::guard_call(ctx ? &ctx->err : &g_err, [&]() -> int {
        if (!ctx) return CULS_E_INVALID;
        return set_err(ctx, ctx->eng.sync());
    });
}

}  // extern "C"
