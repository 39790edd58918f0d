// Seeded synthetic graph / query generators (host only). See include/psm_gen.h.
//
// Determinism: every random stream is a std::mt19937_64 seeded through
// splitmix64, and parallel work is cut into fixed-size chunks whose streams
// depend only on (seed, chunk index), so the output never depends on the
// number of threads.
#include "psm_gen.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <thread>
#include <vector>

namespace {

uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

double uniform01(std::mt19937_64& rng) {
    // 53 random bits -> [0, 1)
    return (double)(rng() >> 11) * (1.0 / 9007199254740992.0);
}

unsigned hw_threads() {
    unsigned t = std::thread::hardware_concurrency();
    return t == 0 ? 1 : std::min(t, 64u);
}

template <class F>
void parallel_chunks(uint64_t nchunks, F&& f) {
    unsigned nt = (unsigned)std::min<uint64_t>(hw_threads(), nchunks);
    if (nt <= 1) {
        for (uint64_t c = 0; c < nchunks; ++c) f(c);
        return;
    }
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t)
        th.emplace_back([&, t]() {
            for (uint64_t c = t; c < nchunks; c += nt) f(c);
        });
    for (auto& x : th) x.join();
}

// LSD radix sort of 64-bit keys on the low `bits` bits (16-bit digits).
void radix_sort_u64(std::vector<uint64_t>& a, unsigned bits) {
    std::vector<uint64_t> tmp(a.size());
    const unsigned passes = (bits + 15) / 16;
    std::vector<uint64_t> cnt(65537);
    for (unsigned p = 0; p < passes; ++p) {
        const unsigned sh = p * 16;
        std::fill(cnt.begin(), cnt.end(), 0);
        for (uint64_t k : a) cnt[((k >> sh) & 0xFFFF) + 1]++;
        for (int i = 0; i < 65536; ++i) cnt[i + 1] += cnt[i];
        for (uint64_t k : a) tmp[cnt[(k >> sh) & 0xFFFF]++] = k;
        a.swap(tmp);
    }
}

// Turns sampled endpoint pairs into a symmetric, deduplicated, loop-free CSR.
int pairs_to_csr(uint32_t n, std::vector<uint64_t>& keys, psmgen_csr* out) {
    unsigned bits = 1;
    while ((1ull << bits) < (uint64_t)n) ++bits;
    radix_sort_u64(keys, 32 + bits);
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    std::vector<uint64_t> deg(n + 1, 0);
    for (uint64_t k : keys) {
        deg[k >> 32]++;
        deg[k & 0xFFFFFFFFu]++;
    }
    uint64_t total = 0;
    for (uint32_t i = 0; i < n; ++i) {
        uint64_t d = deg[i];
        deg[i] = total;
        total += d;
    }
    deg[n] = total;
    if (total >= (1ull << 32)) return 2;  // uint32 offsets only
    out->num_vertices = n;
    out->num_entries = total;
    out->off = (uint32_t*)malloc(sizeof(uint32_t) * (n + 1));
    out->nbr = (uint32_t*)malloc(sizeof(uint32_t) * (total ? total : 1));
    if (!out->off || !out->nbr) return 3;
    for (uint32_t i = 0; i <= n; ++i) out->off[i] = (uint32_t)deg[i];
    // Keys are sorted by (u, v) with u < v, so appending in key order leaves
    // every row ascending: smaller endpoints arrive first, in order.
    std::vector<uint64_t> cur(deg.begin(), deg.end() - 1);
    for (uint64_t k : keys) {
        uint32_t u = (uint32_t)(k >> 32), v = (uint32_t)(k & 0xFFFFFFFFu);
        out->nbr[cur[u]++] = v;
        out->nbr[cur[v]++] = u;
    }
    return 0;
}

inline uint64_t pack_edge(uint32_t u, uint32_t v) {
    if (u > v) std::swap(u, v);
    return ((uint64_t)u << 32) | v;
}

bool has_edge(const uint32_t* off, const uint32_t* nbr, uint32_t u, uint32_t v) {
    const uint32_t* b = nbr + off[u];
    const uint32_t* e = nbr + off[u + 1];
    return std::binary_search(b, e, v);
}

}  // namespace

extern "C" {

int psmgen_chung_lu(uint32_t n, double gamma, double avg_degree, uint64_t seed, psmgen_csr* out) {
    if (!out || n < 2 || gamma <= 1.0 || avg_degree <= 0) return 1;
    std::vector<double> cdf(n);
    const double expo = -1.0 / (gamma - 1.0);
    double s = 0;
    for (uint32_t i = 0; i < n; ++i) {
        s += std::pow((double)(i + 1), expo);
        cdf[i] = s;
    }
    for (auto& x : cdf) x /= s;
    const uint64_t m = (uint64_t)std::llround((double)n * avg_degree / 2.0);
    std::mt19937_64 rng(splitmix64(seed));
    std::vector<uint64_t> keys;
    keys.reserve(m);
    auto draw = [&]() -> uint32_t {
        double r = uniform01(rng);
        uint32_t i = (uint32_t)(std::upper_bound(cdf.begin(), cdf.end(), r) - cdf.begin());
        return i >= n ? n - 1 : i;
    };
    for (uint64_t e = 0; e < m; ++e) {
        uint32_t u = draw(), v = draw();
        if (u != v) keys.push_back(pack_edge(u, v));
    }
    return pairs_to_csr(n, keys, out);
}

int psmgen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed,
                psmgen_csr* out) {
    if (!out || scale < 1 || scale > 31 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return 1;
    const uint32_t n = 1u << scale;
    const uint64_t m = (uint64_t)edge_factor << scale;
    const uint64_t chunk = 1ull << 20;
    const uint64_t nchunks = (m + chunk - 1) / chunk;
    std::vector<uint64_t> keys(m);
    std::vector<uint8_t> keep(m);
    const double ab = a + b, abc = a + b + c;
    parallel_chunks(nchunks, [&](uint64_t ch) {
        std::mt19937_64 rng(splitmix64(seed ^ splitmix64(ch + 1)));
        uint64_t lo = ch * chunk, hi = std::min(m, lo + chunk);
        for (uint64_t e = lo; e < hi; ++e) {
            uint32_t u = 0, v = 0;
            for (uint32_t lvl = 0; lvl < scale; ++lvl) {
                double r = uniform01(rng);
                uint32_t bu = 0, bv = 0;
                if (r < a) {
                } else if (r < ab) {
                    bv = 1;
                } else if (r < abc) {
                    bu = 1;
                } else {
                    bu = 1;
                    bv = 1;
                }
                u = (u << 1) | bu;
                v = (v << 1) | bv;
            }
            keep[e] = (u != v);
            keys[e] = pack_edge(u, v);
        }
    });
    uint64_t w = 0;
    for (uint64_t e = 0; e < m; ++e)
        if (keep[e]) keys[w++] = keys[e];
    keys.resize(w);
    std::vector<uint8_t>().swap(keep);
    return pairs_to_csr(n, keys, out);
}

int psmgen_labels(uint32_t n, uint32_t num_labels, double zipf_s, uint64_t seed, uint32_t* out) {
    if (!out || num_labels == 0) return 1;
    std::mt19937_64 rng(splitmix64(seed ^ 0x4C4142454Cull));
    if (zipf_s <= 0) {
        for (uint32_t i = 0; i < n; ++i) out[i] = (uint32_t)(rng() % num_labels);
        return 0;
    }
    std::vector<double> cdf(num_labels);
    double s = 0;
    for (uint32_t l = 0; l < num_labels; ++l) {
        s += std::pow((double)(l + 1), -zipf_s);
        cdf[l] = s;
    }
    for (auto& x : cdf) x /= s;
    for (uint32_t i = 0; i < n; ++i) {
        double r = uniform01(rng);
        uint32_t l = (uint32_t)(std::upper_bound(cdf.begin(), cdf.end(), r) - cdf.begin());
        out[i] = l >= num_labels ? num_labels - 1 : l;
    }
    return 0;
}

int psmgen_query(const uint32_t* off, const uint32_t* nbr, const uint32_t* labels, uint32_t num_vertices,
                 uint32_t k, int dense, uint64_t seed, uint32_t* q_labels, uint32_t* edges,
                 uint32_t max_edges, uint32_t* num_edges, uint32_t* data_ids) {
    if (!off || !nbr || !labels || k < 1 || k > 64 || !q_labels || !edges || !num_edges) return 1;
    std::mt19937_64 rng(splitmix64(seed));
    const int max_attempts = 2000;
    std::vector<uint32_t> best_verts;
    std::vector<std::pair<uint32_t, uint32_t>> best_edges;
    bool accepted = false;
    std::vector<uint32_t> verts;
    std::vector<std::pair<uint32_t, uint32_t>> tree, induced, chosen;
    for (int attempt = 0; attempt < max_attempts && !accepted; ++attempt) {
        uint32_t start = (uint32_t)(rng() % num_vertices);
        if (off[start + 1] == off[start]) continue;
        verts.assign(1, start);
        tree.clear();
        uint32_t cur = start, cur_idx = 0;
        const uint32_t max_steps = 64 * k + 64;
        for (uint32_t step = 0; verts.size() < k && step < max_steps; ++step) {
            uint32_t d = off[cur + 1] - off[cur];
            uint32_t nxt = nbr[off[cur] + (uint32_t)(rng() % d)];
            auto it = std::find(verts.begin(), verts.end(), nxt);
            uint32_t nxt_idx;
            if (it == verts.end()) {
                nxt_idx = (uint32_t)verts.size();
                verts.push_back(nxt);
                tree.emplace_back(cur_idx, nxt_idx);
            } else {
                nxt_idx = (uint32_t)(it - verts.begin());
            }
            cur = nxt;
            cur_idx = nxt_idx;
        }
        if (verts.size() < k) continue;
        induced.clear();
        for (uint32_t i = 0; i < k; ++i)
            for (uint32_t j = i + 1; j < k; ++j)
                if (has_edge(off, nbr, verts[i], verts[j])) induced.emplace_back(i, j);
        if (dense) {
            if (2.0 * (double)induced.size() / (double)k >= 3.0) {
                chosen = induced;
                accepted = true;
            } else if (induced.size() > best_edges.size() || best_verts.empty()) {
                best_verts = verts;
                best_edges = induced;
            }
        } else {
            chosen.clear();
            for (auto& e : tree) chosen.emplace_back(std::min(e.first, e.second), std::max(e.first, e.second));
            std::vector<std::pair<uint32_t, uint32_t>> rest;
            for (auto& e : induced)
                if (std::find(chosen.begin(), chosen.end(), e) == chosen.end()) rest.push_back(e);
            for (size_t i = rest.size(); i > 1; --i) std::swap(rest[i - 1], rest[(size_t)(rng() % i)]);
            for (auto& e : rest) {
                if (2.0 * (double)(chosen.size() + 1) / (double)k < 3.0)
                    chosen.push_back(e);
                else
                    break;
            }
            accepted = true;
        }
    }
    if (!accepted) {
        if (best_verts.empty()) return 2;
        verts = best_verts;
        chosen = best_edges;
    }
    std::sort(chosen.begin(), chosen.end());
    if (chosen.size() > max_edges) return 3;
    for (uint32_t i = 0; i < k; ++i) {
        q_labels[i] = labels[verts[i]];
        if (data_ids) data_ids[i] = verts[i];
    }
    for (size_t i = 0; i < chosen.size(); ++i) {
        edges[2 * i] = chosen[i].first;
        edges[2 * i + 1] = chosen[i].second;
    }
    *num_edges = (uint32_t)chosen.size();
    return 0;
}

int psmgen_write_text(const uint32_t* off, const uint32_t* nbr, const uint32_t* labels, uint32_t n,
                      const char* path) {
    FILE* f = fopen(path, "wb");
    if (!f) return 1;
    std::vector<char> buf;
    buf.reserve(1 << 22);
    char tmp[64];
    auto flush = [&]() {
        if (!buf.empty()) fwrite(buf.data(), 1, buf.size(), f);
        buf.clear();
    };
    auto put = [&](const char* s, int len) {
        buf.insert(buf.end(), s, s + len);
        if (buf.size() > (1u << 22)) flush();
    };
    uint64_t m = 0;
    for (uint32_t v = 0; v < n; ++v)
        for (uint32_t j = off[v]; j < off[v + 1]; ++j) m += nbr[j] > v;
    put(tmp, snprintf(tmp, sizeof(tmp), "t %u %llu\n", n, (unsigned long long)m));
    for (uint32_t v = 0; v < n; ++v)
        put(tmp, snprintf(tmp, sizeof(tmp), "v %u %u %u\n", v, labels[v], off[v + 1] - off[v]));
    for (uint32_t v = 0; v < n; ++v)
        for (uint32_t j = off[v]; j < off[v + 1]; ++j)
            if (nbr[j] > v) put(tmp, snprintf(tmp, sizeof(tmp), "e %u %u\n", v, nbr[j]));
    flush();
    return fclose(f) == 0 ? 0 : 2;
}

void psmgen_free(void* p) { free(p); }

}  // extern "C"
