// ORACLE -- TEST INFRASTRUCTURE ONLY.
//
// A single-threaded CPU restatement of the reference's subgraph-matching path
// (PSM_Benchmark, "-QorCandi C" mode): NLF / GQL / CFL candidate filtering,
// candidate sorting, candidate-edge tables, GQL / CFL matching orders and an
// LFTJ-style backtracking count with the optional embedding cap. Each function
// cites the reference file:line it restates. Only tests/, the smoke check and
// the bench's CPU-baseline leg load this library, and only as the checker;
// the product path never calls it.
//
// Parity pin: tests compare this oracle with fixtures dumped by the
// reference's own compiled code (tests/golden/) and with the reference's
// recorded HPRD counts.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <queue>
#include <vector>

namespace {

using u32 = uint32_t;
using u64 = uint64_t;
constexpr u32 INVALID = 100000000u;  // configuration/config.h:4 INVALID_VERTEX_ID

struct Graph {
    u32 n = 0;
    std::vector<u32> off, adj, lab;
    u32 labels_count = 0;
    u32 max_degree = 0;
    u32 max_label_freq = 0;
    std::vector<u32> label_freq;            // indexed by label id
    std::vector<u32> bucket_off, bucket;    // reverse index, ascending ids per label
    std::vector<u32> nlf_off, nlf_lab, nlf_cnt;  // per-vertex sorted (label, count)
    std::vector<int> core;

    u32 deg(u32 v) const { return off[v + 1] - off[v]; }
    u32 freq(u32 l) const { return l < label_freq.size() ? label_freq[l] : 0; }
    bool has_edge(u32 u, u32 v) const {
        return std::binary_search(adj.begin() + off[u], adj.begin() + off[u + 1], v);
    }
    // NLF count of label l around v (0 if none).
    u32 nlf(u32 v, u32 l) const {
        auto b = nlf_lab.begin() + nlf_off[v], e = nlf_lab.begin() + nlf_off[v + 1];
        auto it = std::lower_bound(b, e, l);
        return (it != e && *it == l) ? nlf_cnt[it - nlf_lab.begin()] : 0;
    }
    u32 nlf_size(u32 v) const { return nlf_off[v + 1] - nlf_off[v]; }
};

// graph/graph.cpp:92-172 (loadGraphFromFile), :15-33 (BuildReverseIndex),
// :36-52 (BuildNLF): label count = max(#distinct, max label + 1); buckets
// list ids ascending; NLF is the neighbour-label histogram.
void finalize(Graph& g) {
    g.max_degree = 0;
    u32 maxlab = 0;
    for (u32 v = 0; v < g.n; ++v) {
        g.max_degree = std::max(g.max_degree, g.deg(v));
        maxlab = std::max(maxlab, g.lab[v]);
    }
    g.labels_count = g.n ? maxlab + 1 : 0;
    g.label_freq.assign(g.labels_count, 0);
    for (u32 v = 0; v < g.n; ++v) g.label_freq[g.lab[v]]++;
    g.max_label_freq = 0;
    for (u32 f : g.label_freq) g.max_label_freq = std::max(g.max_label_freq, f);
    g.bucket_off.assign(g.labels_count + 1, 0);
    for (u32 l = 0; l < g.labels_count; ++l) g.bucket_off[l + 1] = g.bucket_off[l] + g.label_freq[l];
    g.bucket.resize(g.n);
    std::vector<u32> cur(g.bucket_off.begin(), g.bucket_off.end() - 1);
    for (u32 v = 0; v < g.n; ++v) g.bucket[cur[g.lab[v]]++] = v;
    g.nlf_off.assign(g.n + 1, 0);
    g.nlf_lab.clear();
    g.nlf_cnt.clear();
    std::vector<u32> tmp;
    for (u32 v = 0; v < g.n; ++v) {
        tmp.clear();
        for (u32 j = g.off[v]; j < g.off[v + 1]; ++j) tmp.push_back(g.lab[g.adj[j]]);
        std::sort(tmp.begin(), tmp.end());
        for (size_t i = 0; i < tmp.size();) {
            size_t k = i;
            while (k < tmp.size() && tmp[k] == tmp[i]) ++k;
            g.nlf_lab.push_back(tmp[i]);
            g.nlf_cnt.push_back((u32)(k - i));
            i = k;
        }
        g.nlf_off[v + 1] = (u32)g.nlf_lab.size();
    }
}

// k-core numbers (utility/graphoperations.cpp:5-76 getKCore computes the
// standard core decomposition, which is unique; this is plain peeling).
void build_core(Graph& g) {
    g.core.assign(g.n, 0);
    std::vector<u32> d(g.n);
    std::vector<char> removed(g.n, 0);
    for (u32 v = 0; v < g.n; ++v) d[v] = g.deg(v);
    for (u32 it = 0; it < g.n; ++it) {
        u32 best = INVALID, bd = INVALID;
        for (u32 v = 0; v < g.n; ++v)
            if (!removed[v] && d[v] < bd) bd = d[v], best = v;
        removed[best] = 1;
        g.core[best] = (int)bd;
        for (u32 j = g.off[best]; j < g.off[best + 1]; ++j) {
            u32 w = g.adj[j];
            if (!removed[w] && d[w] > bd) d[w]--;
        }
    }
}
u32 two_core_size(const Graph& q) {
    u32 c = 0;
    for (int x : q.core) c += x > 1;
    return c;
}

// matching/FilterVertices.cpp:767-813 computeCandidateWithNLF: scan the label
// bucket in ascending id order; keep v with deg(v) >= deg(u) whose NLF
// dominates u's NLF.
u32 nlf_candidates(const Graph& G, const Graph& Q, u32 u, std::vector<u32>* out) {
    u32 l = Q.lab[u], du = Q.deg(u), cnt = 0;
    if (l >= G.labels_count) return 0;
    for (u32 i = G.bucket_off[l]; i < G.bucket_off[l + 1]; ++i) {
        u32 v = G.bucket[i];
        if (G.deg(v) < du) continue;
        if (G.nlf_size(v) < Q.nlf_size(u)) continue;
        bool ok = true;
        for (u32 k = Q.nlf_off[u]; k < Q.nlf_off[u + 1] && ok; ++k)
            ok = G.nlf(v, Q.nlf_lab[k]) >= Q.nlf_cnt[k];
        if (!ok) continue;
        if (out) out->push_back(v);
        ++cnt;
    }
    return cnt;
}

using Cands = std::vector<std::vector<u32>>;

// matching/FilterVertices.cpp:48-65 NLFFilter: stops at the first empty set;
// the sets of later query vertices stay empty.
bool nlf_filter(const Graph& G, const Graph& Q, Cands& C) {
    C.assign(Q.n, {});
    for (u32 u = 0; u < Q.n; ++u) {
        nlf_candidates(G, Q, u, &C[u]);
        if (C[u].empty()) return false;
    }
    return true;
}

// Left-saturating bipartite matching test (Kuhn's augmenting paths). The
// reference's match_bfs (utility/graphoperations.cpp:95-149) computes a
// maximum matching too, so the saturating / not-saturating answer agrees.
struct Matcher {
    std::vector<std::vector<u32>> ladj;
    std::vector<int> rmatch;
    std::vector<u32> seen;
    u32 stamp = 0;
    bool aug(u32 l) {
        for (u32 r : ladj[l]) {
            if (seen[r] == stamp) continue;
            seen[r] = stamp;
            if (rmatch[r] < 0 || aug((u32)rmatch[r])) {
                rmatch[r] = (int)l;
                return true;
            }
        }
        return false;
    }
};

// matching/FilterVertices.cpp:704-741 verifyExactTwigIso: N(u) must match
// into N(v) where u' -- w iff w is a valid candidate of u'.
bool semi_perfect(const Graph& G, const Graph& Q, u32 u, u32 v, const std::vector<std::vector<char>>& valid,
                  Matcher& m) {
    u32 L = Q.deg(u), R = G.deg(v);
    m.ladj.assign(L, {});
    for (u32 i = 0; i < L; ++i) {
        u32 un = Q.adj[Q.off[u] + i];
        for (u32 j = 0; j < R; ++j)
            if (valid[un][G.adj[G.off[v] + j]]) m.ladj[i].push_back(j);
    }
    m.rmatch.assign(R, -1);
    m.seen.assign(R, 0);
    m.stamp = 0;
    for (u32 i = 0; i < L; ++i) {
        ++m.stamp;
        if (!m.aug(i)) return false;
    }
    return true;
}

// matching/FilterVertices.cpp:67-143 GQLFilter: NLF, then two rounds of
// in-place refinement over u = 0..q-1, then compaction.
bool gql_filter(const Graph& G, const Graph& Q, Cands& C) {
    if (!nlf_filter(G, Q, C)) return false;
    std::vector<std::vector<char>> valid(Q.n, std::vector<char>(G.n, 0));
    for (u32 u = 0; u < Q.n; ++u)
        for (u32 v : C[u]) valid[u][v] = 1;
    Matcher m;
    for (int round = 0; round < 2; ++round)
        for (u32 u = 0; u < Q.n; ++u)
            for (u32& v : C[u]) {
                if (v == INVALID) continue;
                if (!semi_perfect(G, Q, u, v, valid, m)) {
                    valid[u][v] = 0;
                    v = INVALID;
                }
            }
    for (auto& c : C) c.erase(std::remove(c.begin(), c.end(), INVALID), c.end());
    return true;
}

struct TreeNode {
    u32 parent = 0, level = 0;
    std::vector<u32> children, bn, fn, under;
};

// utility/graphoperations.cpp:156-195 bfsTraversal (neighbours in adjacency
// order, children in discovery order).
void bfs_tree(const Graph& Q, u32 root, std::vector<TreeNode>& tree, std::vector<u32>& order) {
    tree.assign(Q.n, TreeNode{});
    order.clear();
    std::vector<char> vis(Q.n, 0);
    std::queue<u32> qu;
    qu.push(root);
    vis[root] = 1;
    while (!qu.empty()) {
        u32 u = qu.front();
        qu.pop();
        order.push_back(u);
        for (u32 j = Q.off[u]; j < Q.off[u + 1]; ++j) {
            u32 w = Q.adj[j];
            if (vis[w]) continue;
            vis[w] = 1;
            qu.push(w);
            tree[w].parent = u;
            tree[w].level = tree[u].level + 1;
            tree[u].children.push_back(w);
        }
    }
}

// matching/GenerateFilteringPlan.cpp:343-385 selectCFLFilterStartVertex.
// The rank heap is a std::priority_queue with the same comparator, so ties
// pop in the same order as in the reference.
u32 cfl_start_vertex(const Graph& G, const Graph& Q) {
    auto cmp = [](std::pair<u32, double> l, std::pair<u32, double> r) { return l.second < r.second; };
    std::priority_queue<std::pair<u32, double>, std::vector<std::pair<u32, double>>, decltype(cmp)> pq(cmp);
    u32 core2 = two_core_size(Q);
    for (u32 u = 0; u < Q.n; ++u)
        if (core2 == 0 || Q.core[u] > 1) pq.push({u, G.freq(Q.lab[u]) / (double)Q.deg(u)});
    while (pq.size() > 3) pq.pop();
    u32 start = 0;
    double best = G.max_label_freq + 1;
    while (!pq.empty()) {
        u32 u = pq.top().first;
        double score = nlf_candidates(G, Q, u, nullptr) / (double)Q.deg(u);
        if (score < best) best = score, start = u;
        pq.pop();
    }
    return start;
}

// matching/GenerateFilteringPlan.cpp:81-140 generateCFLFilterPlan: BFS tree,
// levels, and per-vertex bn / fn / under-level neighbour lists.
void cfl_filter_plan(const Graph& G, const Graph& Q, std::vector<TreeNode>& tree, std::vector<u32>& order,
                     std::vector<u32>& level_off) {
    u32 root = cfl_start_vertex(G, Q);
    bfs_tree(Q, root, tree, order);
    std::vector<u32> idx(Q.n);
    for (u32 i = 0; i < Q.n; ++i) idx[order[i]] = i;
    level_off.assign(1, 0);
    u32 cur_level = INVALID;
    for (u32 i = 0; i < Q.n; ++i) {
        u32 u = order[i];
        if (tree[u].level != cur_level) {
            cur_level = tree[u].level;
            if (i) level_off.push_back(i);
        }
        for (u32 j = Q.off[u]; j < Q.off[u + 1]; ++j) {
            u32 w = Q.adj[j];
            if (tree[u].level == tree[w].level)
                (idx[w] < idx[u] ? tree[u].bn : tree[u].fn).push_back(w);
            else if (tree[u].level > tree[w].level)
                tree[u].bn.push_back(w);
            else
                tree[u].under.push_back(w);
        }
    }
    level_off.push_back(Q.n);
}

// matching/FilterVertices.cpp:841-912 generateCandidates as a set: label,
// degree, adjacent to a live candidate of every pivot, then NLF.
void cfl_generate(const Graph& G, const Graph& Q, u32 u, const std::vector<u32>& piv, Cands& C,
                  std::vector<u32>& flag) {
    std::vector<u32> touched;
    u32 cnt = 0;
    for (u32 p : piv) {
        for (u32 c : C[p]) {
            if (c == INVALID) continue;
            for (u32 j = G.off[c]; j < G.off[c + 1]; ++j) {
                u32 w = G.adj[j];
                if (flag[w] == cnt && G.lab[w] == Q.lab[u] && G.deg(w) >= Q.deg(u)) {
                    flag[w]++;
                    if (cnt == 0) touched.push_back(w);
                }
            }
        }
        ++cnt;
    }
    for (u32 w : touched) {
        if (flag[w] != cnt) continue;
        bool ok = G.nlf_size(w) >= Q.nlf_size(u);
        for (u32 k = Q.nlf_off[u]; k < Q.nlf_off[u + 1] && ok; ++k) ok = G.nlf(w, Q.nlf_lab[k]) >= Q.nlf_cnt[k];
        if (ok) C[u].push_back(w);
    }
    for (u32 w : touched) flag[w] = 0;
}

// matching/FilterVertices.cpp:914-966 pruneCandidates: drop candidates of u
// that are not adjacent to a live candidate of every pivot.
void cfl_prune(const Graph& G, const Graph& Q, u32 u, const std::vector<u32>& piv, Cands& C, std::vector<u32>& flag) {
    std::vector<u32> touched;
    u32 cnt = 0;
    for (u32 p : piv) {
        for (u32 c : C[p]) {
            if (c == INVALID) continue;
            for (u32 j = G.off[c]; j < G.off[c + 1]; ++j) {
                u32 w = G.adj[j];
                if (flag[w] == cnt && G.lab[w] == Q.lab[u] && G.deg(w) >= Q.deg(u)) {
                    flag[w]++;
                    if (cnt == 0) touched.push_back(w);
                }
            }
        }
        ++cnt;
    }
    for (u32& v : C[u])
        if (v != INVALID && flag[v] != cnt) v = INVALID;
    for (u32 w : touched) flag[w] = 0;
}

// matching/FilterVertices.cpp:188-250 CFLFilter.
void cfl_filter(const Graph& G, const Graph& Q, Cands& C) {
    std::vector<TreeNode> tree;
    std::vector<u32> order, lo;
    cfl_filter_plan(G, Q, tree, order, lo);
    C.assign(Q.n, {});
    nlf_candidates(G, Q, order[0], &C[order[0]]);
    std::vector<u32> flag(G.n, 0);
    u32 levels = (u32)lo.size() - 1;
    for (u32 i = 1; i < levels; ++i) {
        for (u32 j = lo[i]; j < lo[i + 1]; ++j) cfl_generate(G, Q, order[j], tree[order[j]].bn, C, flag);
        for (u32 j = lo[i + 1]; j-- > lo[i];)
            if (!tree[order[j]].fn.empty()) cfl_prune(G, Q, order[j], tree[order[j]].fn, C, flag);
    }
    for (int i = (int)levels - 2; i >= 0; --i)
        for (u32 j = lo[i]; j < lo[i + 1]; ++j)
            if (!tree[order[j]].under.empty()) cfl_prune(G, Q, order[j], tree[order[j]].under, C, flag);
    for (auto& c : C) c.erase(std::remove(c.begin(), c.end(), INVALID), c.end());
}

struct Table {
    std::vector<u32> off, adj;
};

// matching/BuildTable.cpp:9-151 buildTables: for every query edge (x, y),
// row i of T[x][y] lists ascending positions j in C(y) with
// (C(x)[i], C(y)[j]) a data edge.
void build_tables(const Graph& G, const Graph& Q, const Cands& C, std::vector<std::vector<Table>>& T) {
    T.assign(Q.n, std::vector<Table>(Q.n));
    std::vector<u32> pos(G.n, INVALID);
    for (u32 y = 0; y < Q.n; ++y) {
        for (u32 j = 0; j < C[y].size(); ++j) pos[C[y][j]] = j;
        for (u32 k = Q.off[y]; k < Q.off[y + 1]; ++k) {
            u32 x = Q.adj[k];
            Table& t = T[x][y];
            t.off.assign(C[x].size() + 1, 0);
            t.adj.clear();
            for (u32 i = 0; i < C[x].size(); ++i) {
                u32 v = C[x][i];
                for (u32 e = G.off[v]; e < G.off[v + 1]; ++e)
                    if (pos[G.adj[e]] != INVALID) t.adj.push_back(pos[G.adj[e]]);
                t.off[i + 1] = (u32)t.adj.size();
            }
        }
        for (u32 v : C[y]) pos[v] = INVALID;
    }
}

// matching/BuildTable.cpp:300-326 computeMemoryCostInBytes.
u64 memory_cost(const Graph& Q, const Cands& C, const std::vector<std::vector<Table>>& T) {
    u64 b = 0;
    for (u32 u = 0; u < Q.n; ++u) b += (u64)C[u].size() * 4;
    for (u32 a = 0; a < Q.n; ++a)
        for (u32 c = a + 1; c < Q.n; ++c)
            if (Q.has_edge(a, c))
                b += ((u64)T[a][c].adj.size() + C[a].size() + T[c][a].adj.size() + C[c].size()) * 4;
    return b;
}

// matching/GenerateQueryPlan.cpp:149-172 selectGQLStartVertex and :9-60
// generateGQLQueryPlan (greedy min-candidates, ties to higher degree; pivot =
// first earlier neighbour in the order).
void gql_order(const Graph& G, const Graph& Q, const Cands& C, std::vector<u32>& order, std::vector<u32>& pivot) {
    order.assign(Q.n, 0);
    pivot.assign(Q.n, 0);
    u32 start = 0;
    for (u32 u = 1; u < Q.n; ++u)
        if (C[u].size() < C[start].size() || (C[u].size() == C[start].size() && Q.deg(u) > Q.deg(start)))
            start = u;
    std::vector<char> vis(Q.n, 0), adjv(Q.n, 0);
    auto mark = [&](u32 u) {
        vis[u] = 1;
        for (u32 j = Q.off[u]; j < Q.off[u + 1]; ++j) adjv[Q.adj[j]] = 1;
    };
    order[0] = start;
    mark(start);
    for (u32 i = 1; i < Q.n; ++i) {
        u32 nxt = 0;
        u64 best = (u64)G.n + 1;
        for (u32 u = 0; u < Q.n; ++u) {
            if (vis[u] || !adjv[u]) continue;
            if (C[u].size() < best) {
                best = C[u].size();
                nxt = u;
            } else if (C[u].size() == best && Q.deg(u) > Q.deg(nxt)) {
                nxt = u;
            }
        }
        order[i] = nxt;
        mark(nxt);
    }
    for (u32 i = 1; i < Q.n; ++i)
        for (u32 j = 0; j < i; ++j)
            if (Q.has_edge(order[i], order[j])) {
                pivot[i] = order[j];
                break;
            }
}

// matching/GenerateQueryPlan.cpp:680-721 estimatePathEmbeddsingsNum.
std::vector<u64> path_estimates(const std::vector<u32>& path, const std::vector<std::vector<Table>>& T) {
    size_t k = path.size();
    std::vector<u64> est(k - 1), child, par;
    const Table& last = T[path[k - 2]][path[k - 1]];
    u32 rows = (u32)last.off.size() - 1;
    child.resize(rows);
    u64 s = 0;
    for (u32 i = 0; i < rows; ++i) s += (child[i] = last.off[i + 1] - last.off[i]);
    est[k - 2] = s;
    for (int i = (int)k - 2; i >= 1; --i) {
        const Table& t = T[path[i - 1]][path[i]];
        u32 r = (u32)t.off.size() - 1;
        par.assign(r, 0);
        s = 0;
        for (u32 j = 0; j < r; ++j) {
            u64 ls = 0;
            for (u32 e = t.off[j]; e < t.off[j + 1]; ++e) ls += child[t.adj[e]];
            par[j] = ls;
            s += ls;
        }
        est[i - 1] = s;
        par.swap(child);
    }
    return est;
}

void core_paths(const Graph& Q, const std::vector<TreeNode>& tree, u32 u, std::vector<u32>& cur,
                std::vector<std::vector<u32>>& out) {
    cur.push_back(u);
    bool leaf = true;
    for (u32 c : tree[u].children)
        if (Q.core[c] > 1) {
            core_paths(Q, tree, c, cur, out);
            leaf = false;
        }
    if (leaf) out.push_back(cur);
    cur.pop_back();
}

void tree_paths(const Graph& Q, const std::vector<TreeNode>& tree, u32 u, std::vector<u32>& cur,
                std::vector<std::vector<u32>>& out) {
    cur.push_back(u);
    bool leaf = true;
    for (u32 c : tree[u].children)
        if (Q.deg(c) > 1) {
            tree_paths(Q, tree, c, cur, out);
            leaf = false;
        }
    if (leaf && cur.size() > 1) out.push_back(cur);
    cur.pop_back();
}

// The unit query of "-QorCandi C" mode: the same vertices and edges with labels
// renumbered by first appearance (graph/graph.cpp:585-734 loadsubgFromGraph,
// labels at :659-666). The CFL order's start vertex is selected on it.
Graph relabelled_unit(const Graph& Q) {
    Graph U = Q;
    std::vector<u32> map;
    for (u32 v = 0; v < Q.n; ++v) {
        auto it = std::find(map.begin(), map.end(), Q.lab[v]);
        u32 nl = (u32)(it - map.begin());
        if (it == map.end()) map.push_back(Q.lab[v]);
        U.lab[v] = nl;
    }
    finalize(U);
    U.core = Q.core;
    return U;
}

// matching/GenerateQueryPlan.cpp:270-471 generateCFLQueryPlan(q, UnitArgs*),
// with the filtering tree of GenerateFilteringPlan.cpp:15-79 built on the unit
// query.
void cfl_order(const Graph& G, const Graph& Q, const Cands& C, const std::vector<std::vector<Table>>& T,
               std::vector<u32>& order, std::vector<u32>& pivot) {
    Graph U = relabelled_unit(Q);
    std::vector<TreeNode> tree;
    std::vector<u32> bfs;
    bfs_tree(U, cfl_start_vertex(G, U), tree, bfs);
    u32 root = bfs[0];
    order.assign(Q.n, 0);
    pivot.assign(Q.n, 0);
    std::vector<char> vis(Q.n, 0);
    std::vector<std::vector<u32>> cps;
    std::vector<std::vector<std::vector<u32>>> forests;
    std::vector<u32> leaves, cur;
    for (u32 u = 0; u < Q.n; ++u)
        if (Q.deg(u) == 1) leaves.push_back(u);
    if (Q.core[root] > 1) {
        core_paths(Q, tree, root, cur, cps);
        for (u32 u = 0; u < Q.n; ++u)
            if (Q.core[u] > 1) {
                std::vector<std::vector<u32>> tp;
                tree_paths(Q, tree, u, cur, tp);
                if (!tp.empty()) forests.push_back(tp);
            }
    } else {
        std::vector<std::vector<u32>> tp;
        tree_paths(Q, tree, root, cur, tp);
        if (!tp.empty()) forests.push_back(tp);
    }
    u32 cnt = 0;
    order[cnt++] = root;
    vis[root] = 1;
    auto csz = [&](u32 u) { return (double)C[u].size(); };
    if (!cps.empty()) {
        std::vector<std::vector<u64>> est;
        std::vector<u32> nte;
        for (auto& p : cps) {
            u32 x = Q.deg(p[0]) - (u32)tree[p[0]].children.size();
            for (size_t i = 1; i < p.size(); ++i) x += Q.deg(p[i]) - (u32)tree[p[i]].children.size() - 1;
            nte.push_back(x + 1);
            est.push_back(path_estimates(p, T));
        }
        double mn = 1.79769313486231570815e308;
        size_t sel = 0;
        for (size_t i = 0; i < cps.size(); ++i) {
            double v = est[i][0] / (double)nte[i];
            if (v < mn) mn = v, sel = i;
        }
        for (size_t i = 1; i < cps[sel].size(); ++i) {
            order[cnt] = cps[sel][i];
            pivot[cnt] = cps[sel][i - 1];
            ++cnt;
            vis[cps[sel][i]] = 1;
        }
        cps.erase(cps.begin() + sel);
        est.erase(est.begin() + sel);
        while (!cps.empty()) {
            mn = 1.79769313486231570815e308;
            sel = 0;
            for (size_t i = 0; i < cps.size(); ++i) {
                u32 ri = 0;
                for (u32 j = 0; j < cps[i].size(); ++j) {
                    if (vis[cps[i][j]]) continue;
                    ri = j - 1;
                    break;
                }
                double v = est[i][ri] / csz(cps[i][ri]);
                if (v < mn) mn = v, sel = i;
            }
            for (size_t i = 1; i < cps[sel].size(); ++i) {
                if (vis[cps[sel][i]]) continue;
                order[cnt] = cps[sel][i];
                pivot[cnt] = cps[sel][i - 1];
                ++cnt;
                vis[cps[sel][i]] = 1;
            }
            cps.erase(cps.begin() + sel);
            est.erase(est.begin() + sel);
        }
    }
    for (auto& tps : forests) {
        std::vector<std::vector<u64>> est;
        for (auto& p : tps) est.push_back(path_estimates(p, T));
        while (!tps.empty()) {
            double mn = 1.79769313486231570815e308;
            size_t sel = 0;
            for (size_t i = 0; i < tps.size(); ++i) {
                u32 ri = 0;
                for (u32 j = 0; j < tps[i].size(); ++j) {
                    if (vis[tps[i][j]]) continue;
                    ri = j == 0 ? j : j - 1;
                    break;
                }
                double v = est[i][ri] / csz(tps[i][ri]);
                if (v < mn) mn = v, sel = i;
            }
            for (size_t i = 0; i < tps[sel].size(); ++i) {
                if (vis[tps[sel][i]]) continue;
                order[cnt] = tps[sel][i];
                pivot[cnt] = i ? tps[sel][i - 1] : 0;  // path heads are always visited
                ++cnt;
                vis[tps[sel][i]] = 1;
            }
            tps.erase(tps.begin() + sel);
            est.erase(est.begin() + sel);
        }
    }
    while (!leaves.empty()) {
        double mn = 1.79769313486231570815e308;
        size_t sel = 0;
        for (size_t i = 0; i < leaves.size(); ++i) {
            double v = csz(leaves[i]);
            if (v < mn) mn = v, sel = i;
        }
        u32 l = leaves[sel];
        if (!vis[l]) {
            order[cnt] = l;
            pivot[cnt] = tree[l].parent;
            ++cnt;
            vis[l] = 1;
        }
        leaves.erase(leaves.begin() + sel);
    }
}

// matching/EvaluateQuery.cpp:231-372 LFTJ with generateValidCandidateIndex
// (:2024-2082): candidates at depth d are the intersection of the table rows
// of all earlier neighbours, visited vertices skipped when picked; counting
// stops once the cap is reached (EvaluateQuery.cpp:152,301-330).
struct Enumerator {
    const Graph& Q;
    const Cands& C;
    const std::vector<std::vector<Table>>& T;
    std::vector<u32> order;
    std::vector<std::vector<u32>> bn;   // by depth, query vertex ids
    std::vector<u32> emb_pos, emb_vid;  // by query vertex
    std::vector<std::vector<u32>> buf;
    u64 cap, count = 0, calls = 0;
    u64 emit_limit;
    std::vector<u32>* emit;
    // Per depth: partial embeddings accepted, candidates examined and
    // algorithmic bytes of the table rows read (8 B of offsets + 4 B per entry).
    std::vector<u64> depth_nodes, depth_cands, depth_bytes;

    Enumerator(const Graph& q, const Cands& c, const std::vector<std::vector<Table>>& t, const std::vector<u32>& o,
               u64 cap_, u64 emit_limit_, std::vector<u32>* emit_)
        : Q(q), C(c), T(t), order(o), cap(cap_), emit_limit(emit_limit_), emit(emit_) {
        bn.assign(Q.n, {});
        std::vector<char> seen(Q.n, 0);
        seen[order[0]] = 1;
        for (u32 d = 1; d < Q.n; ++d) {
            u32 u = order[d];
            for (u32 j = Q.off[u]; j < Q.off[u + 1]; ++j)
                if (seen[Q.adj[j]]) bn[d].push_back(Q.adj[j]);
            seen[u] = 1;
        }
        emb_pos.assign(Q.n, 0);
        emb_vid.assign(Q.n, INVALID);
        buf.assign(Q.n, {});
        depth_nodes.assign(Q.n, 0);
        depth_cands.assign(Q.n, 0);
        depth_bytes.assign(Q.n, 0);
    }

    bool used(u32 v) const {
        for (u32 x : emb_vid)
            if (x == v) return true;
        return false;
    }

    void candidates(u32 d, std::vector<u32>& out) {
        u32 u = order[d];
        out.clear();
        if (d == 0) {
            out.resize(C[u].size());
            std::iota(out.begin(), out.end(), 0u);
            return;
        }
        const Table& t0 = T[bn[d][0]][u];
        u32 r0 = emb_pos[bn[d][0]];
        out.assign(t0.adj.begin() + t0.off[r0], t0.adj.begin() + t0.off[r0 + 1]);
        for (u32 b : bn[d]) {
            const Table& t = T[b][u];
            u32 r = emb_pos[b];
            depth_bytes[d] += 8 + 4ull * (t.off[r + 1] - t.off[r]);
        }
        std::vector<u32> tmp;
        for (size_t i = 1; i < bn[d].size(); ++i) {
            const Table& t = T[bn[d][i]][u];
            u32 r = emb_pos[bn[d][i]];
            tmp.clear();
            std::set_intersection(out.begin(), out.end(), t.adj.begin() + t.off[r], t.adj.begin() + t.off[r + 1],
                                  std::back_inserter(tmp));
            out.swap(tmp);
        }
    }

    // Returns false once the cap is reached.
    bool dfs(u32 d) {
        candidates(d, buf[d]);
        u32 u = order[d];
        for (u32 p : buf[d]) {
            u32 v = C[u][p];
            ++calls;
            ++depth_cands[d];
            if (used(v)) continue;
            ++depth_nodes[d];
            if (d + 1 == Q.n) {
                ++count;
                if (emit && count <= emit_limit) {
                    emb_vid[u] = v;
                    emit->insert(emit->end(), emb_vid.begin(), emb_vid.end());
                    emb_vid[u] = INVALID;
                }
                if (cap && count >= cap) return false;
                continue;
            }
            emb_pos[u] = p;
            emb_vid[u] = v;
            bool go = dfs(d + 1);
            emb_vid[u] = INVALID;
            if (!go) return false;
        }
        return true;
    }
};

struct Result {
    int filter_ok = 1;
    u64 count = 0, calls = 0, memory = 0;
    Cands C;
    std::vector<std::vector<Table>> T;
    std::vector<u32> order, pivot, emb;
    std::vector<u64> depth_nodes, depth_cands, depth_bytes;
};

Graph make_graph(const u32* off, const u32* adj, const u32* lab, u32 n) {
    Graph g;
    g.n = n;
    g.off.assign(off, off + n + 1);
    g.adj.assign(adj, adj + off[n]);
    g.lab.assign(lab, lab + n);
    finalize(g);
    return g;
}

}  // namespace

extern "C" {

void* orc_graph_new(const u32* off, const u32* adj, const u32* lab, u32 n) {
    return new Graph(make_graph(off, adj, lab, n));
}
void orc_graph_free(void* g) { delete (Graph*)g; }

// filter: 0 = NLF, 1 = GQL, 2 = CFL; order: 0 = GQL, 1 = CFL.
// cap = 0 means no cap. emit_limit > 0 also records up to that many
// embeddings (query vertex order 0..q-1, data vertex ids).
void* orc_run(void* gp, const u32* qoff, const u32* qadj, const u32* qlab, u32 qn, int filter, int order,
              u64 cap, u64 emit_limit) {
    const Graph& G = *(const Graph*)gp;
    Graph Q = make_graph(qoff, qadj, qlab, qn);
    build_core(Q);
    Result* r = new Result;
    bool ok;
    if (filter == 0)
        ok = nlf_filter(G, Q, r->C);
    else if (filter == 1)
        ok = gql_filter(G, Q, r->C);
    else {
        cfl_filter(G, Q, r->C);
        ok = true;
    }
    r->filter_ok = ok;
    for (auto& c : r->C) std::sort(c.begin(), c.end());  // FilterVertices.cpp:1012-1016
    build_tables(G, Q, r->C, r->T);
    r->memory = memory_cost(Q, r->C, r->T);
    if (order == 0)
        gql_order(G, Q, r->C, r->order, r->pivot);
    else
        cfl_order(G, Q, r->C, r->T, r->order, r->pivot);
    bool any_empty = false;
    for (auto& c : r->C) any_empty |= c.empty();
    if (!any_empty) {
        Enumerator e(Q, r->C, r->T, r->order, cap, emit_limit, emit_limit ? &r->emb : nullptr);
        e.dfs(0);
        r->count = cap && e.count > cap ? cap : e.count;
        r->calls = e.calls;
        r->depth_nodes = e.depth_nodes;
        r->depth_cands = e.depth_cands;
        r->depth_bytes = e.depth_bytes;
    }
    return r;
}

u64 orc_res_count(void* r) { return ((Result*)r)->count; }
u64 orc_res_calls(void* r) { return ((Result*)r)->calls; }
u64 orc_res_memory(void* r) { return ((Result*)r)->memory; }
int orc_res_filter_ok(void* r) { return ((Result*)r)->filter_ok; }
// Per depth of the matching order (qn entries each): partial embeddings
// accepted, candidates examined, algorithmic bytes of table rows read.
// All zero when enumeration did not run.
void orc_res_depth_stats(void* r, u64* nodes, u64* cands, u64* bytes) {
    auto* x = (Result*)r;
    for (size_t d = 0; d < x->depth_nodes.size(); ++d) {
        nodes[d] = x->depth_nodes[d];
        cands[d] = x->depth_cands[d];
        bytes[d] = x->depth_bytes[d];
    }
}
u32 orc_res_cand_count(void* r, u32 u) { return (u32)((Result*)r)->C[u].size(); }
void orc_res_cands(void* r, u32 u, u32* out) {
    auto& c = ((Result*)r)->C[u];
    std::copy(c.begin(), c.end(), out);
}
// Number of entries of T[a][b], or 0xFFFFFFFF when (a, b) is not a query edge.
u32 orc_res_table_nnz(void* r, u32 a, u32 b) {
    auto& t = ((Result*)r)->T[a][b];
    return t.off.empty() ? 0xFFFFFFFFu : (u32)t.adj.size();
}
void orc_res_table(void* r, u32 a, u32 b, u32* off, u32* adj) {
    auto& t = ((Result*)r)->T[a][b];
    std::copy(t.off.begin(), t.off.end(), off);
    std::copy(t.adj.begin(), t.adj.end(), adj);
}
void orc_res_order(void* r, u32* order, u32* pivot) {
    auto* x = (Result*)r;
    std::copy(x->order.begin(), x->order.end(), order);
    std::copy(x->pivot.begin(), x->pivot.end(), pivot);
}
u64 orc_res_num_emb(void* r) {
    auto* x = (Result*)r;
    return x->C.empty() ? 0 : x->emb.size() / x->C.size();
}
void orc_res_emb(void* r, u32* out) {
    auto& e = ((Result*)r)->emb;
    std::copy(e.begin(), e.end(), out);
}
void orc_res_free(void* r) { delete (Result*)r; }

}  // extern "C"
