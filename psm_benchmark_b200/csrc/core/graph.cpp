// Data graph ingestion: text parser for the reference format and the
// label-major CSR that is made resident in HBM (layout in psm_internal.h).
// Replaces Graph::loadGraphFromFile / BuildReverseIndex / BuildNLF
// (graph/graph.cpp:15-52, :92-172): the per-vertex NLF hash maps become label
// runs inside each adjacency list, found by binary search on the device.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
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
    g->dev.loops = 0;
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
            if (w == v) g->dev.loops = 1;
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
// Host CSR of a graph file (original ids; rows sorted).
struct HostCsr {
    u32 V = 0;
    std::vector<u32> off, nbr, labels;
};

int parse_text(const char* path, HostCsr* g, std::string* err) {
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
    g->V = V;
    g->off = std::move(off);
    g->nbr = std::move(nbr);
    g->labels = std::move(labels);
    return PSM_OK;
}

int psm_graph_parse(const char* path, psm_graph** out, std::string* err) {
    HostCsr h;
    int rc = parse_text(path, &h, err);
    if (rc) return rc;
    return psm_graph_build(h.off.data(), h.nbr.data(), h.labels.data(), h.V, out, err);
}

// The reference's binary graph format (Graph::loadGraphFromFileCompressed /
// storeComparessedGraph, graph/graph.cpp:221-403; written by its
// GraphConverter, matching/GraphConverter.cpp): a degree file (int32 size of
// int = 4, uint32 |V|, uint32 |E| (undirected), uint32 degree[|V|]), an
// adjacency file (uint32 neighbours, row after row, 2|E| in all) and a label
// file (uint32 label[|V|]). Rows are sorted on load, as the reference does.
int read_binary(const char* deg_path, const char* adj_path, const char* label_path, HostCsr* g, std::string* err) {
    auto open = [&](const char* p) -> FILE* {
        FILE* f = fopen(p, "rb");
        if (!f) *err = std::string("cannot open ") + p;
        return f;
    };
    FILE* fd = open(deg_path);
    if (!fd) return PSM_ERR_IO;
    int32_t int_size = 0;
    u32 V = 0, E = 0;
    bool ok = fread(&int_size, 4, 1, fd) == 1 && fread(&V, 4, 1, fd) == 1 && fread(&E, 4, 1, fd) == 1;
    std::vector<u32> deg(V);
    ok = ok && int_size == 4 && (V == 0 || fread(deg.data(), 4, V, fd) == V);
    fclose(fd);
    if (!ok) {
        *err = std::string("malformed degree file ") + deg_path;
        return PSM_ERR_IO;
    }
    std::vector<u32> off(V + 1, 0);
    for (u32 v = 0; v < V; ++v) off[v + 1] = off[v] + deg[v];
    if ((u64)off[V] != 2ull * E) {
        *err = "degree sum differs from 2|E|";
        return PSM_ERR_IO;
    }
    std::vector<u32> nbr(off[V]);
    FILE* fa = open(adj_path);
    if (!fa) return PSM_ERR_IO;
    ok = nbr.empty() || fread(nbr.data(), 4, nbr.size(), fa) == nbr.size();
    fclose(fa);
    if (!ok) {
        *err = std::string("short adjacency file ") + adj_path;
        return PSM_ERR_IO;
    }
    std::vector<u32> labels(V);
    FILE* fl = open(label_path);
    if (!fl) return PSM_ERR_IO;
    ok = V == 0 || fread(labels.data(), 4, V, fl) == V;
    fclose(fl);
    if (!ok) {
        *err = std::string("short label file ") + label_path;
        return PSM_ERR_IO;
    }
    for (u32 v = 0; v < V; ++v) std::sort(nbr.begin() + off[v], nbr.begin() + off[v + 1]);
    g->V = V;
    g->off = std::move(off);
    g->nbr = std::move(nbr);
    g->labels = std::move(labels);
    return PSM_OK;
}

int write_binary(const u32* off, const u32* nbr, const u32* labels, u32 V, const char* deg_path, const char* adj_path,
                 const char* label_path, std::string* err) {
    if ((off[V] & 1u) != 0) {
        *err = "odd number of adjacency entries (an undirected CSR stores every edge twice)";
        return PSM_ERR_ARG;
    }
    const int32_t int_size = 4;
    const u32 E = off[V] / 2;
    std::vector<u32> deg(V);
    for (u32 v = 0; v < V; ++v) deg[v] = off[v + 1] - off[v];
    auto put = [&](const char* p, const void* a, size_t n, const void* h, size_t hn) -> bool {
        FILE* f = fopen(p, "wb");
        if (!f) {
            *err = std::string("cannot write ") + p;
            return false;
        }
        bool ok = (hn == 0 || fwrite(h, 1, hn, f) == hn) && (n == 0 || fwrite(a, 4, n, f) == n);
        ok = (fclose(f) == 0) && ok;
        if (!ok) *err = std::string("write failed: ") + p;
        return ok;
    };
    char head[12];
    memcpy(head, &int_size, 4);
    memcpy(head + 4, &V, 4);
    memcpy(head + 8, &E, 4);
    if (!put(deg_path, deg.data(), V, head, 12) || !put(adj_path, nbr, off[V], nullptr, 0) ||
        !put(label_path, labels, V, nullptr, 0))
        return PSM_ERR_IO;
    return PSM_OK;
}

int psm_graph_parse_binary(const char* deg_path, const char* adj_path, const char* label_path, psm_graph** out,
                           std::string* err) {
    HostCsr h;
    int rc = read_binary(deg_path, adj_path, label_path, &h, err);
    if (rc) return rc;
    return psm_graph_build(h.off.data(), h.nbr.data(), h.labels.data(), h.V, out, err);
}

int psm_text_to_binary(const char* text_path, const char* out_prefix, std::string* err) {
    HostCsr h;
    int rc = parse_text(text_path, &h, err);
    if (rc) return rc;
    const std::string pre(out_prefix);
    return write_binary(h.off.data(), h.nbr.data(), h.labels.data(), h.V, (pre + "_deg.bin").c_str(),
                        (pre + "_adj.bin").c_str(), (pre + "_label.bin").c_str(), err);
}

// Edge-list text -> the binary files above (matching/EdgeListToCSR.cpp, the
// reference's EdgeListConverter). One "u v" pair of vertex ids per line;
// lines starting with '#' and blank lines are skipped. Each pair is kept with
// its smaller id first and the pairs are sorted. A self loop (v, v) fails the
// whole conversion with nothing written (the reference prints "src >= dst"
// and writes no files); duplicate pairs are kept, as there. |V| = largest id
// + 1, |E| = number of pairs, and row v lists its neighbours in pair order:
// those below v, then those above, each ascending. Labels are uniform over
// [0, num_labels) from std::mt19937 seeded with `seed` (the reference seeds
// it from std::random_device, so its labels change from run to run). As the
// reference reads with getline until the stream is no longer good, a last
// line without a newline is not used.
int psm_edgelist_to_binary(const char* path, const char* out_prefix, u32 num_labels, u64 seed, std::string* err) {
    if (num_labels == 0) {
        *err = "number of labels must be positive";
        return PSM_ERR_ARG;
    }
    FILE* f = fopen(path, "rb");
    if (!f) {
        *err = std::string("cannot open ") + path;
        return PSM_ERR_IO;
    }
    std::string text;
    char buf[1 << 16];
    size_t got;
    while ((got = fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, got);
    fclose(f);
    std::vector<std::pair<u32, u32>> pairs;
    u64 max_id = 0;
    bool any = false;
    size_t line_no = 0;
    for (size_t pos = 0;;) {
        const size_t nl = text.find('\n', pos);
        if (nl == std::string::npos) break;  // unterminated last line: not used
        ++line_no;
        const std::string line = text.substr(pos, nl - pos);
        pos = nl + 1;
        if (!line.empty() && line[0] == '#') continue;
        const char* c = line.c_str();
        while (*c == ' ' || *c == '\t' || *c == '\r') ++c;
        if (*c == 0) continue;
        char* end = nullptr;
        long long ids[2];
        bool ok = true;
        for (int k = 0; k < 2 && ok; ++k) {
            ids[k] = strtoll(c, &end, 10);
            ok = end != c && ids[k] >= 0 && ids[k] < 0x7fffffffLL;
            c = end;
        }
        if (!ok) {
            *err = "line " + std::to_string(line_no) + ": expected two vertex ids in [0, 2^31 - 1)";
            return PSM_ERR_ARG;
        }
        u32 a = (u32)ids[0], b = (u32)ids[1];
        if (a > b) std::swap(a, b);
        if (a == b) {
            *err = "line " + std::to_string(line_no) + ": self loop (" + std::to_string(a) + ", " +
                   std::to_string(b) + "); nothing written";
            return PSM_ERR_ARG;
        }
        pairs.emplace_back(a, b);
        max_id = std::max<u64>(max_id, b);
        any = true;
    }
    std::sort(pairs.begin(), pairs.end());
    const u32 V = any ? (u32)(max_id + 1) : 0u;
    std::vector<u32> off(V + 1, 0);
    for (const auto& e : pairs) {
        off[e.first + 1]++;
        off[e.second + 1]++;
    }
    for (u32 v = 0; v < V; ++v) off[v + 1] += off[v];
    std::vector<u32> nbr(off[V]), fill(off.begin(), off.end() - 1);
    for (const auto& e : pairs) {
        nbr[fill[e.first]++] = e.second;
        nbr[fill[e.second]++] = e.first;
    }
    std::vector<u32> labels(V);
    std::mt19937 gen((std::mt19937::result_type)seed);
    std::uniform_int_distribution<int> dis(0, (int)num_labels - 1);
    for (u32 v = 0; v < V; ++v) labels[v] = (u32)dis(gen);
    const std::string pre(out_prefix);
    return write_binary(off.data(), nbr.data(), labels.data(), V, (pre + "_deg.bin").c_str(),
                        (pre + "_adj.bin").c_str(), (pre + "_label.bin").c_str(), err);
}

int psm_csr_write_binary(const u32* off, const u32* nbr, const u32* labels, u32 V, const char* deg_path,
                         const char* adj_path, const char* label_path, std::string* err) {
    return write_binary(off, nbr, labels, V, deg_path, adj_path, label_path, err);
}

void psm_graph_destroy(psm_graph* g) { free_graph(g); }
