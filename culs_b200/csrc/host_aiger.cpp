// Binary AIGER reader/writer in the AIGMan layout.
//
// Reader: the format AIGMan::readFromMemory accepts (CULS
// src/aig_manager.cu:110-229): header "aig M I L O A" with L == 0 and no
// extended header fields, one ASCII literal per output line, then the
// delta-encoded AND gates (aigDecodeBinary, src/aig_manager.cu:861-869).
// Where the reference asserts (latches, extended header, out-of-order
// literals) this reader returns CULS_E_IO instead.
// Writer: AIGMan::saveFile (src/aig_manager.cu:231-267): header, output
// literals, delta-encoded gates, then the comment marker "c".

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "culs_b200.h"
#include "guard.hpp"

namespace {

inline int inv_const(int lit) { return lit < 2 ? 1 - lit : lit; }

bool decode_uint(const unsigned char *&p, const unsigned char *end, uint32_t &x) {
    x = 0;
    int shift = 0;
    while (p < end) {
        unsigned char ch = *p++;
        if (shift > 28) return false;
        x |= (uint32_t)(ch & 0x7f) << shift;
        if (!(ch & 0x80)) return true;
        shift += 7;
    }
    return false;
}

void encode_uint(std::vector<unsigned char> &buf, uint32_t x) {
    while (x & ~0x7fu) {
        buf.push_back((unsigned char)((x & 0x7f) | 0x80));
        x >>= 7;
    }
    buf.push_back((unsigned char)x);
}

bool read_int(const unsigned char *&p, const unsigned char *end, long long &v) {
    if (p >= end || *p < '0' || *p > '9') return false;
    v = 0;
    while (p < end && *p >= '0' && *p <= '9') {
        v = v * 10 + (*p - '0');
        if (v > INT32_MAX) return false;
        p++;
    }
    return true;
}

}  // namespace

extern "C" {

int culs_aiger_read(const char *path, culs_host_graph *out) {
    return culs::guard_call(nullptr, [&]() -> int {
        if (!path || !out) return CULS_E_INVALID;
        memset(out, 0, sizeof *out);
        FILE *f = fopen(path, "rb");
        if (!f) return CULS_E_IO;
        std::vector<unsigned char> data;
        unsigned char buf[1 << 16];
        size_t k;
        while ((k = fread(buf, 1, sizeof buf, f)) > 0) data.insert(data.end(), buf, buf + k);
        fclose(f);
        const unsigned char *p = data.data(), *end = p + data.size();
        if (data.size() < 4 || memcmp(p, "aig ", 4) != 0) return CULS_E_IO;
        p += 4;
        long long M, I, L, O, A;
        if (!read_int(p, end, M) || p >= end || *p++ != ' ') return CULS_E_IO;
        if (!read_int(p, end, I) || p >= end || *p++ != ' ') return CULS_E_IO;
        if (!read_int(p, end, L) || p >= end || *p++ != ' ') return CULS_E_IO;
        if (!read_int(p, end, O) || p >= end || *p++ != ' ') return CULS_E_IO;
        if (!read_int(p, end, A) || p >= end || *p++ != '\n') return CULS_E_IO;
        if (L != 0 || M != I + A || M + 1 > INT32_MAX / 2) return CULS_E_IO;
        int nObjs = (int)(M + 1), nPIs = (int)I, nPOs = (int)O;
        std::vector<int32_t> f0(nObjs, -1), f1(nObjs, -1), outs(nPOs);
        for (int i = 0; i < nPOs; i++) {
            long long lit;
            if (!read_int(p, end, lit) || p >= end || *p++ != '\n') return CULS_E_IO;
            if (lit >= 2LL * nObjs) return CULS_E_IO;
            outs[i] = inv_const((int)lit);
        }
        for (int i = 0; i < (int)A; i++) {
            uint32_t lhs = 2u * (uint32_t)(i + 1 + nPIs), d0, d1;
            if (!decode_uint(p, end, d0) || !decode_uint(p, end, d1)) return CULS_E_IO;
            if (d0 > lhs) return CULS_E_IO;
            uint32_t r1 = lhs - d0;
            if (d1 > r1) return CULS_E_IO;
            uint32_t r0 = r1 - d1;
            if (r1 >= lhs) return CULS_E_IO;  // fanins precede the node
            f0[i + 1 + nPIs] = inv_const((int)r0);
            f1[i + 1 + nPIs] = inv_const((int)r1);
        }
        out->nPIs = nPIs;
        out->nPOs = nPOs;
        out->nAnds = (int)A;
        out->fanin0 = (int32_t *)malloc(sizeof(int32_t) * (size_t)nObjs);
        out->fanin1 = (int32_t *)malloc(sizeof(int32_t) * (size_t)nObjs);
        out->outs = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nPOs > 0 ? nPOs : 1));
        if (!out->fanin0 || !out->fanin1 || !out->outs) {
            culs_host_graph_free(out);
            return CULS_E_OOM;
        }
        memcpy(out->fanin0, f0.data(), sizeof(int32_t) * (size_t)nObjs);
        memcpy(out->fanin1, f1.data(), sizeof(int32_t) * (size_t)nObjs);
        if (nPOs) memcpy(out->outs, outs.data(), sizeof(int32_t) * (size_t)nPOs);
        return CULS_OK;
    });
}

int culs_aiger_write(const char *path, const culs_host_graph *g) {
    return culs::guard_call(nullptr, [&]() -> int {
        if (!path || !g || g->nPIs < 0 || g->nAnds < 0 || g->nPOs < 0) return CULS_E_INVALID;
        int nObjs = 1 + g->nPIs + g->nAnds;
        std::vector<unsigned char> body;
        body.reserve((size_t)g->nAnds * 4 + 16);
        for (int i = g->nPIs + 1; i < nObjs; i++) {
            int l0 = inv_const(g->fanin0[i]), l1 = inv_const(g->fanin1[i]);
            if (l0 > l1) {
                int t = l0;
                l0 = l1;
                l1 = t;
            }
            if (l0 < 0 || 2 * i - l1 <= 0) return CULS_E_INVALID;
            encode_uint(body, (uint32_t)(2 * i - l1));
            encode_uint(body, (uint32_t)(l1 - l0));
        }
        FILE *f = fopen(path, "wb");
        if (!f) return CULS_E_IO;
        fprintf(f, "aig %d %d 0 %d %d\n", nObjs - 1, g->nPIs, g->nPOs, g->nAnds);
        for (int i = 0; i < g->nPOs; i++) fprintf(f, "%d\n", inv_const(g->outs[i]));
        if (!body.empty()) fwrite(body.data(), 1, body.size(), f);
        fprintf(f, "c\n");
        int rc = ferror(f) ? CULS_E_IO : CULS_OK;
        fclose(f);
        return rc;
    });
}

}  // extern "C"
