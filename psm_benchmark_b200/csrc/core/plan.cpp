// Host-side query analysis: everything about a query that does not depend on
// the data graph's adjacency is decided here, once, and shipped to the
// device in a QDesc:
//  - NLF lists (neighbour label histograms, graph/graph.cpp:36-52) and, per
//    label, the set of neighbours carrying it (the label groups of the GQL
//    matching test);
//  - the CFL start-vertex options: the rank heap of
//    matching/GenerateFilteringPlan.cpp:343-385 keeps three vertices, and the
//    device picks one of them from their NLF counts. The heap is a
//    std::priority_queue with the reference's comparator, so equal ranks pop
//    in the same order as in the reference;
//  - for every option, the CFL filtering plan (BFS tree, levels, bn / fn /
//    under-level neighbour sets: GenerateFilteringPlan.cpp:81-140) as a
//    sequence of generate / prune steps (FilterVertices.cpp:188-250);
//  - the CFL matching-order inputs for every option of the "unit" query, the
//    query with labels renumbered by first appearance that "-QorCandi C"
//    mode orders (graph/graph.cpp:659-666, GenerateQueryPlan.cpp:270-471):
//    BFS tree, core paths, tree-path forests, leaves.
#include <algorithm>
#include <cstring>
#include <queue>
#include <string>
#include <vector>

#include "host.h"

namespace {

struct QGraph {
    u32 n = 0;
    std::vector<u32> lab;
    std::vector<std::vector<u32>> nbrs;  // ascending
    std::vector<int> core;
    u32 deg(u32 u) const { return (u32)nbrs[u].size(); }
};

// k-core numbers by repeated removal of a minimum-degree vertex (the core
// decomposition is unique; utility/graphoperations.cpp:5-76 computes it with
// bin sort).
void core_numbers(QGraph& q) {
    q.core.assign(q.n, 0);
    std::vector<u32> d(q.n);
    std::vector<char> gone(q.n, 0);
    for (u32 v = 0; v < q.n; ++v) d[v] = q.deg(v);
    for (u32 it = 0; it < q.n; ++it) {
        u32 best = 0, bd = 0xFFFFFFFFu;
        for (u32 v = 0; v < q.n; ++v)
            if (!gone[v] && d[v] < bd) bd = d[v], best = v;
        gone[best] = 1;
        q.core[best] = (int)bd;
        for (u32 w : q.nbrs[best])
            if (!gone[w] && d[w] > bd) d[w]--;
    }
}

struct Tree {
    std::vector<u32> parent, level, order;
    std::vector<std::vector<u32>> children;
};

// utility/graphoperations.cpp:156-195 bfsTraversal.
Tree bfs(const QGraph& q, u32 root) {
    Tree t;
    t.parent.assign(q.n, 0);
    t.level.assign(q.n, 0);
    t.children.assign(q.n, {});
    std::vector<char> vis(q.n, 0);
    std::queue<u32> qu;
    qu.push(root);
    vis[root] = 1;
    while (!qu.empty()) {
        u32 u = qu.front();
        qu.pop();
        t.order.push_back(u);
        for (u32 w : q.nbrs[u]) {
            if (vis[w]) continue;
            vis[w] = 1;
            qu.push(w);
            t.parent[w] = u;
            t.level[w] = t.level[u] + 1;
            t.children[u].push_back(w);
        }
    }
    return t;
}

// The three start-vertex options of GenerateFilteringPlan.cpp:343-385 in
// the order the reference pops them.
std::vector<u32> start_options(const psm_graph& g, const QGraph& q) {
    auto cmp = [](std::pair<u32, double> l, std::pair<u32, double> r) { return l.second < r.second; };
    std::priority_queue<std::pair<u32, double>, std::vector<std::pair<u32, double>>, decltype(cmp)> pq(cmp);
    u32 core2 = 0;
    for (int c : q.core) core2 += c > 1;
    for (u32 u = 0; u < q.n; ++u)
        if (core2 == 0 || q.core[u] > 1) pq.push({u, g.freq(q.lab[u]) / (double)q.deg(u)});
    while (pq.size() > 3) pq.pop();
    std::vector<u32> out;
    while (!pq.empty()) {
        out.push_back(pq.top().first);
        pq.pop();
    }
    return out;
}

void fill_filter_plan(const QGraph& q, u32 root, FilterPlan& fp) {
    Tree t = bfs(q, root);
    std::vector<u32> idx(q.n);
    for (u32 i = 0; i < q.n; ++i) idx[t.order[i]] = i;
    std::vector<u32> bn(q.n, 0), fn(q.n, 0), under(q.n, 0);
    for (u32 u = 0; u < q.n; ++u)
        for (u32 w : q.nbrs[u]) {
            if (t.level[u] == t.level[w])
                (idx[w] < idx[u] ? bn[u] : fn[u]) |= 1u << w;
            else if (t.level[u] > t.level[w])
                bn[u] |= 1u << w;
            else
                under[u] |= 1u << w;
        }
    std::vector<u32> lo{0};
    for (u32 i = 1; i < q.n; ++i)
        if (t.level[t.order[i]] != t.level[t.order[i - 1]]) lo.push_back(i);
    lo.push_back(q.n);
    const u32 levels = (u32)lo.size() - 1;
    fp.root = root;
    fp.nsteps = 0;
    auto add = [&](u32 kind, u32 u, u32 mask) {
        fp.step_kind[fp.nsteps] = kind;
        fp.step_u[fp.nsteps] = u;
        fp.step_mask[fp.nsteps] = mask;
        fp.nsteps++;
    };
    for (u32 i = 1; i < levels; ++i) {
        for (u32 j = lo[i]; j < lo[i + 1]; ++j) add(STEP_GEN, t.order[j], bn[t.order[j]]);
        for (u32 j = lo[i + 1]; j-- > lo[i];)
            if (fn[t.order[j]]) add(STEP_PRUNE, t.order[j], fn[t.order[j]]);
    }
    for (int i = (int)levels - 2; i >= 0; --i)
        for (u32 j = lo[i]; j < lo[i + 1]; ++j)
            if (under[t.order[j]]) add(STEP_PRUNE, t.order[j], under[t.order[j]]);
}

void core_paths(const QGraph& q, const Tree& t, u32 u, std::vector<u32>& cur, std::vector<std::vector<u32>>& out) {
    cur.push_back(u);
    bool leaf = true;
    for (u32 c : t.children[u])
        if (q.core[c] > 1) {
            core_paths(q, t, c, cur, out);
            leaf = false;
        }
    if (leaf) out.push_back(cur);
    cur.pop_back();
}

void tree_paths(const QGraph& q, const Tree& t, u32 u, std::vector<u32>& cur, std::vector<std::vector<u32>>& out) {
    cur.push_back(u);
    bool leaf = true;
    for (u32 c : t.children[u])
        if (q.deg(c) > 1) {
            tree_paths(q, t, c, cur, out);
            leaf = false;
        }
    if (leaf && cur.size() > 1) out.push_back(cur);
    cur.pop_back();
}

// Serialises the CFL order inputs for start vertex `root` (layout documented
// in psm_internal.h). Returns false if the blob does not fit.
bool fill_order_plan(const QGraph& q, u32 root, std::vector<u32>& w) {
    Tree t = bfs(q, root);
    std::vector<std::vector<u32>> cps;
    std::vector<std::vector<std::vector<u32>>> forests;
    std::vector<u32> cur;
    if (q.core[root] > 1) {
        core_paths(q, t, root, cur, cps);
        for (u32 u = 0; u < q.n; ++u)
            if (q.core[u] > 1) {
                std::vector<std::vector<u32>> tp;
                tree_paths(q, t, u, cur, tp);
                if (!tp.empty()) forests.push_back(tp);
            }
    } else {
        std::vector<std::vector<u32>> tp;
        tree_paths(q, t, root, cur, tp);
        if (!tp.empty()) forests.push_back(tp);
    }
    if (cps.size() > 64) return false;
    for (auto& f : forests)
        if (f.size() > 64) return false;
    w.clear();
    w.push_back(root);
    for (u32 u = 0; u < q.n; ++u) w.push_back(t.parent[u]);
    for (u32 u = 0; u < q.n; ++u) w.push_back((u32)t.children[u].size());
    w.push_back((u32)cps.size());
    w.push_back((u32)forests.size());
    std::vector<std::vector<u32>> paths = cps;
    std::vector<u32> gfirst{(u32)cps.size()};
    for (auto& f : forests) {
        for (auto& p : f) paths.push_back(p);
        gfirst.push_back((u32)paths.size());
    }
    for (u32 x : gfirst) w.push_back(x);
    w.push_back((u32)paths.size());
    u32 acc = 0;
    w.push_back(0);
    for (auto& p : paths) {
        acc += (u32)p.size();
        w.push_back(acc);
    }
    for (auto& p : cps) {
        // GenerateQueryPlan.cpp:723-732 generateNoneTreeEdgesCount, plus one
        u32 x = q.deg(p[0]) - (u32)t.children[p[0]].size();
        for (size_t i = 1; i < p.size(); ++i) x += q.deg(p[i]) - (u32)t.children[p[i]].size() - 1;
        w.push_back(x + 1);
    }
    for (auto& p : paths)
        for (u32 v : p) w.push_back(v);
    std::vector<u32> leaves;
    for (u32 u = 0; u < q.n; ++u)
        if (q.deg(u) == 1) leaves.push_back(u);
    w.push_back((u32)leaves.size());
    for (u32 l : leaves) w.push_back(l);
    return true;
}

void nlf_lists(const QGraph& q, u32 u, std::vector<u32>& lab, std::vector<u32>& cnt, std::vector<u32>* grp) {
    std::vector<std::pair<u32, u32>> v;  // (label, neighbour)
    for (u32 w : q.nbrs[u]) v.push_back({q.lab[w], w});
    std::sort(v.begin(), v.end());
    for (size_t i = 0; i < v.size();) {
        size_t k = i;
        u32 m = 0;
        while (k < v.size() && v[k].first == v[i].first) m |= 1u << v[k++].second;
        lab.push_back(v[i].first);
        cnt.push_back((u32)(k - i));
        if (grp) grp->push_back(m);
        i = k;
    }
}

}  // namespace

size_t psm_qdesc_bytes(const QDesc& d) { return offsetof(QDesc, plan_words) + sizeof(u32) * d.plan_used; }

int psm_build_qdesc(const psm_graph& g, const psm_query_desc& qd, const psm_options& opt, QDesc* d, std::string* err) {
    const u32 n = qd.num_vertices;
    if (n == 0 || n > PSM_MAXQ) {
        *err = "query must have 1.." + std::to_string(PSM_MAXQ) + " vertices";
        return PSM_ERR_ARG;
    }
    if (!qd.labels || (qd.num_edges && !qd.edges)) {
        *err = "query labels / edges missing";
        return PSM_ERR_ARG;
    }
    if (opt.filter > PSM_FILTER_CFL || opt.order > PSM_ORDER_CFL) {
        *err = "unknown filter / order kind";
        return PSM_ERR_ARG;
    }
    QGraph q;
    q.n = n;
    q.lab.assign(qd.labels, qd.labels + n);
    q.nbrs.assign(n, {});
    std::vector<u32> adj(n, 0);
    for (u32 i = 0; i < qd.num_edges; ++i) {
        u32 a = qd.edges[2 * i], b = qd.edges[2 * i + 1];
        if (a >= n || b >= n || a == b) {
            *err = "query edge out of range or self-loop";
            return PSM_ERR_ARG;
        }
        if ((adj[a] >> b) & 1u) {
            *err = "duplicate query edge";
            return PSM_ERR_ARG;
        }
        adj[a] |= 1u << b;
        adj[b] |= 1u << a;
        q.nbrs[a].push_back(b);
        q.nbrs[b].push_back(a);
    }
    for (auto& v : q.nbrs) std::sort(v.begin(), v.end());
    {  // connectivity
        u32 seen = 1u, frontier = 1u;
        while (frontier) {
            u32 nxt = 0;
            for (u32 u = 0; u < n; ++u)
                if ((frontier >> u) & 1u) nxt |= adj[u];
            frontier = nxt & ~seen;
            seen |= nxt;
        }
        u32 all = n >= 32 ? ~0u : ((1u << n) - 1u);
        if ((seen & all) != all) {
            *err = "query graph must be connected";
            return PSM_ERR_ARG;
        }
    }
    if (n > 1)
        for (u32 u = 0; u < n; ++u)
            if (q.nbrs[u].empty()) {
                *err = "query vertex without edges";
                return PSM_ERR_ARG;
            }
    core_numbers(q);

    memset(d, 0, offsetof(QDesc, plan_words));
    d->n = n;
    d->filter = opt.filter;
    d->order = opt.order;
    d->data_label_count = g.L;
    for (u32 u = 0; u < n; ++u) {
        d->label[u] = q.lab[u];
        d->deg[u] = q.deg(u);
        d->adj[u] = adj[u];
        d->item_label[u] = q.lab[u];
        d->item_deg[u] = q.deg(u);
    }
    std::vector<u32> lab, cnt, grp;
    d->nlf_off[0] = 0;
    for (u32 u = 0; u < n; ++u) {
        nlf_lists(q, u, lab, cnt, &grp);
        d->nlf_off[u + 1] = (u32)lab.size();
    }
    // single-vertex queries have no edges; the CFL start vertex is vertex 0
    // and the order is trivial (degrees of 0 never divide).
    d->fopt_max_score_num = g.max_label_freq + 1;
    if (opt.filter == PSM_FILTER_CFL) {
        std::vector<u32> fo = n > 1 ? start_options(g, q) : std::vector<u32>{0};
        d->nfopt = (u32)fo.size();
        for (u32 k = 0; k < fo.size(); ++k) {
            d->fopt_vertex[k] = fo[k];
            fill_filter_plan(q, fo[k], d->fplan[k]);
        }
    }
    u32 used = 0;
    if (opt.order == PSM_ORDER_CFL) {
        // The unit query of "-QorCandi C": labels renumbered by first
        // appearance in vertex order.
        QGraph uq = q;
        std::vector<u32> map;
        for (u32 v = 0; v < n; ++v) {
            auto it = std::find(map.begin(), map.end(), q.lab[v]);
            uq.lab[v] = (u32)(it - map.begin());
            if (it == map.end()) map.push_back(q.lab[v]);
        }
        std::vector<u32> oo = n > 1 ? start_options(g, uq) : std::vector<u32>{0};
        d->noopt = (u32)oo.size();
        d->nvirt = (u32)oo.size();
        for (u32 k = 0; k < oo.size(); ++k) {
            const u32 u = oo[k], it = n + k;
            d->oopt_vertex[k] = u;
            d->oopt_item[k] = it;
            d->item_label[it] = uq.lab[u];
            d->item_deg[it] = uq.deg(u);
            nlf_lists(uq, u, lab, cnt, nullptr);
            grp.resize(lab.size(), 0);
            d->nlf_off[it + 1] = (u32)lab.size();
            std::vector<u32> w;
            if (!fill_order_plan(uq, u, w) || used + w.size() > PSM_PLAN_WORDS) {
                *err = "query too complex for the CFL order plan";
                return PSM_ERR_ARG;
            }
            d->oplan_off[k] = used;
            memcpy(d->plan_words + used, w.data(), w.size() * sizeof(u32));
            used += (u32)w.size();
        }
    }
    d->plan_used = used;
    if (lab.size() > PSM_MAXNLF) {
        *err = "too many neighbour-label entries";
        return PSM_ERR_ARG;
    }
    std::copy(lab.begin(), lab.end(), d->nlf_lab);
    std::copy(cnt.begin(), cnt.end(), d->nlf_cnt);
    std::copy(grp.begin(), grp.end(), d->nlf_grp);
    u32 e = 0;
    for (u32 x = 0; x < n; ++x) {
        d->e_first[x] = e;
        for (u32 y : q.nbrs[x]) {
            d->e_src[e] = x;
            d->e_dst[e++] = y;
        }
    }
    d->e_first[n] = e;
    return PSM_OK;
}
