// Data graph ingestion: text parser for the reference format and the
// label-major CSR that is made resident in HBM (layout in psm_internal.h).
// Replaces Graph::loadGraphFromFile / BuildReverseIndex / BuildNLF
// (graph/graph.cpp:15-52, :92-172): the per-vertex NLF hash maps become label
// runs inside each adjacency list, found by binary search on the device.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "host.h"

void psm_set_error(const std::string& msg);

namespace {

template <class T>
int upload(T** dst, const T* src, size_t n, std::string* err) {
    size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
    cudaError_t e = cudaMalloc((void**)dst, bytes);
    if (e != cudaSuccess) {
        *err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? PSM_ERR_OOM : PSM_ERR_CUDA;
    }
    if (n) {
        e = cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            *err = std::string("cudaMemcpy: ") + cudaGetErrorString(e);
            return PSM_ERR_CUDA;
        }
    }
    return PSM_OK;
}

void free_graph(psm_graph* g) {
    if (!g) return;
    cudaFree(g->d_off);
    cudaFree(g->d_nbr);
    cudaFree(g->d_lab_off);
    cudaFree(g->d_orig);
    delete g;
}

}  // namespace

int psm_graph_build(const uint32_t* off, const uint32_t* nbr, const uint32_t* labels, uint32_t V, psm_graph** out,
                    std::string* err) {
    if (!off || !labels || (!nbr && off[V] != 0)) {
        *err = "null CSR array";
        return PSM_ERR_ARG;
    }
    const u64 nnz = off[V];
    for (u32 v = 0; v < V; ++v)
        if (off[v + 1] < off[v]) {
            *err = "offsets must be non-decreasing";
            return PSM_ERR_ARG;
        }
    u32 maxlab = 0;
    for (u32 v = 0; v < V; ++v) maxlab = std::max(maxlab, labels[v]);
    const u32 L = V ? maxlab + 1 : 0;
    if ((u64)L > (u64)V + (1u << 24)) {
        *err = "label ids too sparse";
        return PSM_ERR_ARG;
    }
    auto* g = new psm_graph;
    g->V = V;
    g->L = L;
    g->nnz = nnz;
    g->lab_off.assign(L + 1, 0);
    for (u32 v = 0; v < V; ++v) g->lab_off[labels[v] + 1]++;
    for (u32 l = 0; l < L; ++l) {
        g->max_label_freq = std::max(g->max_label_freq, g->lab_off[l + 1]);
        g->lab_off[l + 1] += g->lab_off[l];
    }
    g->to_internal.resize(V);
    std::vector<u32> orig(V);
    {
        std::vector<u32> cur(g->lab_off.begin(), g->lab_off.end() - 1);
        for (u32 v = 0; v < V; ++v) {
            u32 id = cur[labels[v]]++;
            g->to_internal[v] = id;
            orig[id] = v;
        }
    }
    std::vector<u32> ioff(V + 1, 0);
    for (u32 i = 0; i < V; ++i) {
        u32 v = orig[i];
        u32 d = off[v + 1] - off[v];
        g->max_degree = std::max(g->max_degree, d);
        ioff[i + 1] = ioff[i] + d;
    }
    std::vector<u32> inbr(nnz);
    for (u32 i = 0; i < V; ++i) {
        u32 v = orig[i];
        u32* dst = inbr.data() + ioff[i];
        u32 d = off[v + 1] - off[v];
        for (u32 j = 0; j < d; ++j) {
            u32 w = nbr[off[v] + j];
            if (w >= V) {
                *err = "neighbour id out of range";
                delete g;
                return PSM_ERR_ARG;
            }
            dst[j] = g->to_internal[w];
        }
        std::sort(dst, dst + d);
    }
    g->lab_deg.assign(L, 0);
    if (L <= psm_graph::LAB_PAIR_MAX) g->lab_pair.assign((size_t)L * L, 0);
    for (u32 i = 0; i < V; ++i) {
        const u32 a = labels[orig[i]];
        g->lab_deg[a] += ioff[i + 1] - ioff[i];
        if (!g->lab_pair.empty()) {
            u64* row = g->lab_pair.data() + (size_t)a * L;
            // neighbours are sorted by internal id, i.e. grouped by label:
            // one run per label present
            const u32* r0 = inbr.data() + ioff[i];
            const u32* r1 = inbr.data() + ioff[i + 1];
            while (r0 < r1) {
                const u32 b = (u32)(std::upper_bound(g->lab_off.begin(), g->lab_off.end(), *r0) - g->lab_off.begin()) - 1;
                const u32* e = std::lower_bound(r0, r1, g->lab_off[b + 1]);
                row[b] += (u64)(e - r0);
                r0 = e;
            }
        }
    }
    cudaGetDevice(&g->device);
    int rc;
    if ((rc = upload(&g->d_off, ioff.data(), ioff.size(), err)) || (rc = upload(&g->d_nbr, inbr.data(), nnz, err)) ||
        (rc = upload(&g->d_lab_off, g->lab_off.data(), g->lab_off.size(), err)) ||
        (rc = upload(&g->d_orig, orig.data(), orig.size(), err))) {
        free_graph(g);
        return rc;
    }
    g->orig = std::move(orig);
    g->dev.V = V;
    g->dev.L = L;
    g->dev.off = g->d_off;
    g->dev.nbr = g->d_nbr;
    g->dev.lab_off = g->d_lab_off;
    g->dev.orig = g->d_orig;
    *out = g;
    return PSM_OK;
}

// Reference text format (graph/graph.cpp:92-172): "t V E", "v id label deg"
// lines, then "e u v" lines. Edges are stored in both directions; rows are
// sorted; duplicate edges are kept as the reference keeps them.
int psm_graph_parse(const char* path, psm_graph** out, std::string* err) {
    FILE* f = fopen(path, "rb");
    if (!f) {
        *err = std::string("cannot open ") + path;
        return PSM_ERR_IO;
    }
    std::vector<char> buf;
    {
        fseek(f, 0, SEEK_END);
        long sz = ftell(f);
        fseek(f, 0, SEEK_SET);
        buf.resize((size_t)std::max(sz, 0L) + 1);
        size_t rd = fread(buf.data(), 1, (size_t)std::max(sz, 0L), f);
        buf[rd] = 0;
        fclose(f);
    }
    char* p = buf.data();
    auto skip = [&]() {
        while (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\n') ++p;
    };
    auto num = [&]() -> unsigned long long {
        skip();
        unsigned long long x = 0;
        while (*p >= '0' && *p <= '9') x = x * 10 + (unsigned long long)(*p++ - '0');
        return x;
    };
    skip();
    if (*p != 't') {
        *err = "missing 't V E' header";
        return PSM_ERR_IO;
    }
    ++p;
    const u32 V = (u32)num();
    const u64 E = num();
    std::vector<u32> labels(V, 0), deg(V, 0);
    std::vector<u32> src, dst;
    src.reserve(E);
    dst.reserve(E);
    while (true) {
        skip();
        char c = *p;
        if (!c) break;
        ++p;
        if (c == 'v') {
            u32 id = (u32)num(), l = (u32)num();
            (void)num();
            if (id < V) labels[id] = l;
        } else if (c == 'e') {
            u32 a = (u32)num(), b = (u32)num();
            if (a >= V || b >= V) {
                *err = "edge endpoint out of range";
                return PSM_ERR_IO;
            }
            src.push_back(a);
            dst.push_back(b);
            deg[a]++;
            deg[b]++;
        } else {
            while (*p && *p != '\n') ++p;
        }
    }
    std::vector<u32> off(V + 1, 0);
    for (u32 v = 0; v < V; ++v) off[v + 1] = off[v] + deg[v];
    std::vector<u32> nbr(off[V]);
    std::vector<u32> cur(off.begin(), off.end() - 1);
    for (size_t i = 0; i < src.size(); ++i) {
        nbr[cur[src[i]]++] = dst[i];
        nbr[cur[dst[i]]++] = src[i];
    }
    for (u32 v = 0; v < V; ++v) std::sort(nbr.begin() + off[v], nbr.begin() + off[v + 1]);
    return psm_graph_build(off.data(), nbr.data(), labels.data(), V, out, err);
}

void psm_graph_destroy(psm_graph* g) { free_graph(g); }
