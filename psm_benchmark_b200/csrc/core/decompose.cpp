// Query decomposition for the join path (host side).
//
// The reference splits a query into units with SplitGraph
// (utility/splitGraph/SplitGraph.cpp:23-36), enumerates every unit's
// embeddings and joins them: left-deep in unit order
// (JoinCollect::sequence_collect, matching/JoinCollect.cpp:237-315) or, for
// its path-tree pattern, bushy along a join tree
// (JoinCollect::recur_collect, :156-235). Its patterns:
//   STAR       stars around query vertices (greedyStarDecomposition,
//              SplitGraph.cpp:533-660);
//   TWINTWIG   units of one or two edges sharing a vertex, chosen by a
//              best-first search over the cost model card(m, n) =
//              (2M)^m / N^(2m - n) (optimalDecomposition, :671-872;
//              split_twintwig :875);
//   SEED       the same with triangles closed where the query has the third
//              edge (split_seed :913);
//   SKETCHTREE the root-to-leaf paths of a depth-first tree from the vertex
//              of highest degree, joined along the tree (split_hybrid_rnd
//              :38-108).
// This file builds units of the same shapes with its own search code (the
// reference's search visits hash-set order, so its exact units are not
// reproducible and need not be: every decomposition whose units cover all
// query edges and whose joins share a vertex gives the same embeddings).
// Units are always enumerated as induced subgraphs of the query (a twin-twig
// whose leaves are adjacent is enumerated as a triangle), which constrains
// the relations further without changing the joined result.
//
// Two patterns of this library bound the unit size, which the reference's
// patterns do not (their units of two or three vertices have about
// (2M)^2 / N embeddings each, far beyond device memory on large graphs):
//   BOUNDED connected units of at most max_unit vertices:
//     1. vertex order: the vertex of highest degree first (lowest id on
//        ties), then repeatedly the unplaced vertex with the most edges to
//        placed ones (ties: higher degree, then lower id);
//     2. the first unit takes the first max_unit vertices of that order;
//     3. each later unit takes the next vertices N of the order while
//        |N| + |B| <= max_unit, where B = earlier-covered vertices adjacent
//        to N (the join keys); a vertex with max_unit or more covered
//        neighbours gets star units of itself and max_unit - 1 of those
//        neighbours each;
//     4. a unit is the induced subgraph on N + B, split into its connected
//        components.
//   COST    BOUNDED decompositions for every start vertex and unit bounds
//     max_unit .. max_unit - 4, each with its join tree, costed by the
//     estimated number of rows the plan materialises, the cheapest kept.
//     With the device's candidate counts and candidate-edge table sizes the
//     estimate of a pattern is prod |C(u)| x prod p(a, b), p(a, b) = the
//     fraction of candidate pairs of query edge (a, b) that are data edges
//     (independent edges); without them the reference's card model.
// BUSHY join trees (the reference's JoinParadigm::BUSHY) pair, repeatedly,
// the two partial results that share a vertex and whose join has the
// smallest estimate.
//
// Inside a unit the enumeration order is the GQL rule on the query's
// candidate counts (matching/GenerateQueryPlan.cpp:9-83): start at the
// fewest candidates (ties: higher degree in the unit, then lower id), then
// repeatedly the adjacent unplaced vertex with the fewest candidates.
#include <algorithm>
#include <cmath>
#include <limits>
#include <string>
#include <vector>

#include "psm_b200.h"
#include "decompose.h"

namespace {

int popc(u32 x) { return __builtin_popcount(x); }

const double NEG_INF = -std::numeric_limits<double>::infinity();

// log(exp(a) + exp(b))
double log_add(double a, double b) {
    if (a == NEG_INF) return b;
    if (b == NEG_INF) return a;
    const double m = std::max(a, b);
    return m + std::log1p(std::exp(std::min(a, b) - m));
}

// Connected components of `mask` in the graph `adj` restricted to `mask`.
int components(const u32* adj, u32 mask, u32* out) {
    int k = 0;
    u32 left = mask;
    while (left) {
        u32 comp = left & (~left + 1u);
        for (;;) {
            u32 grow = comp;
            for (u32 m = comp; m; m &= m - 1) grow |= adj[__builtin_ctz(m)] & mask;
            if (grow == comp) break;
            comp = grow;
        }
        out[k++] = comp;
        left &= ~comp;
    }
    return k;
}

u32 edges_in(const u32* adj, u32 mask) {
    u32 m = 0;
    for (u32 r = mask; r; r &= r - 1) m += popc(adj[__builtin_ctz(r)] & mask);
    return m / 2;
}

struct Model {
    u32 n;
    const u32* adj;
    const PlanStats* st;
    double log_n, log_2m;
    Model(u32 n_, const u32* adj_, const PlanStats& s) : n(n_), adj(adj_), st(&s) {
        log_n = std::log(std::max(1.0, s.data_vertices));
        log_2m = std::log(std::max(1.0, 2.0 * s.data_edges));
    }
    // the reference's card(m, n) of a pattern with m edges and k vertices
    double log_card(u32 m, u32 k) const { return m * log_2m - (2.0 * m - k) * log_n; }
    // estimated embeddings of the induced pattern on `mask`
    double log_est(u32 mask) const {
        if (!st->cand || !st->edge_p) return log_card(edges_in(adj, mask), popc(mask));
        double s = 0;
        for (u32 r = mask; r; r &= r - 1) {
            const u32 u = __builtin_ctz(r);
            if (st->cand[u] <= 0) return NEG_INF;
            s += std::log(st->cand[u]);
        }
        for (u32 r = mask; r; r &= r - 1) {
            const u32 a = __builtin_ctz(r);
            for (u32 t = adj[a] & mask & ~((2u << a) - 1u); t; t &= t - 1) {
                const double p = st->edge_p[a * n + __builtin_ctz(t)];
                if (p <= 0) return NEG_INF;
                s += std::log(p);
            }
        }
        return s;
    }
};

// Vertex masks of the nodes of a join tree, and the log of the rows the plan
// materialises (every unit and every join result).
u32 tree_cost(const Model& md, const Decomposition& d, u32 node, double* cost) {
    const JoinNode& nd = d.nodes[node];
    if (nd.unit >= 0) {
        const u32 m = d.units[nd.unit].mask;
        *cost = log_add(*cost, md.log_est(m));
        return m;
    }
    u32 acc = tree_cost(md, d, nd.child[0], cost);
    for (u32 i = 1; i < nd.nchild; ++i) {
        acc |= tree_cost(md, d, nd.child[i], cost);
        *cost = log_add(*cost, md.log_est(acc));
    }
    return acc;
}

double plan_cost(const Model& md, const Decomposition& d) {
    double c = NEG_INF;
    tree_cost(md, d, d.root, &c);
    return c;
}

int bounded_sets(u32 n, const u32* adj, u32 max_unit, int start, std::vector<u32>& sets, std::string* err) {
    sets.clear();
    if (max_unit < 2) {
        *err = "units need at least two vertices";
        return 1;
    }
    u32 deg[PSM_MAXQ];
    for (u32 u = 0; u < n; ++u) deg[u] = popc(adj[u]);
    // 1. vertex order
    u32 order[PSM_MAXQ];
    u32 placed = 0;
    for (u32 i = 0; i < n; ++i) {
        int best = -1;
        int best_links = -1;
        if (i == 0 && start >= 0) {
            best = start;
        } else {
            for (u32 u = 0; u < n; ++u) {
                if ((placed >> u) & 1u) continue;
                const int links = popc(adj[u] & placed);
                if (i > 0 && links == 0) continue;
                if (best < 0 || links > best_links || (links == best_links && deg[u] > deg[best])) {
                    best = (int)u;
                    best_links = links;
                }
            }
        }
        if (best < 0) {
            *err = "query graph is not connected";
            return 1;
        }
        order[i] = (u32)best;
        placed |= 1u << best;
    }
    // 2.-4. units
    auto emit = [&](u32 mask) {
        u32 comp[PSM_MAXQ];
        const int k = components(adj, mask, comp);
        for (int c = 0; c < k; ++c)
            if (popc(comp[c]) >= 2) sets.push_back(comp[c]);  // a lone vertex carries no edge
    };
    u32 covered = 0;
    u32 i = 0;
    {
        u32 first = 0;
        for (; i < n && (u32)popc(first) < max_unit; ++i) first |= 1u << order[i];
        if (n == 1)
            sets.push_back(first);  // a single-vertex query is its own unit
        else
            emit(first);
        covered = first;
    }
    while (i < n) {
        u32 N = 0, B = 0;
        while (i < n) {
            const u32 v = order[i];
            const u32 bv = adj[v] & covered;
            if ((u32)(popc(N | (1u << v)) + popc(B | bv)) > max_unit) break;
            N |= 1u << v;
            B |= bv;
            ++i;
        }
        if (N == 0) {
            // one vertex with too many covered neighbours: stars of it
            const u32 v = order[i++];
            u32 bv = adj[v] & covered;
            while (bv) {
                u32 chunk = 0;
                while (bv && (u32)popc(chunk) < max_unit - 1) {
                    chunk |= bv & (~bv + 1u);
                    bv &= bv - 1;
                }
                sets.push_back(chunk | (1u << v));
            }
            covered |= 1u << v;
            continue;
        }
        emit(N | B);
        covered |= N;
    }
    return 0;
}

int store_units(u32 n, const u32* adj, const u32* cnt, const std::vector<u32>& sets, Decomposition* out,
                std::string* err) {
    if (sets.size() > PSM_MAX_UNITS) {
        *err = "more than " + std::to_string(PSM_MAX_UNITS) + " units";
        return 1;
    }
    for (u32 k = 0; k < sets.size(); ++k) {
        const u32 mask = sets[k];
        UnitPlan& up = out->units[k];
        up.mask = mask;
        up.n = 0;
        u32 done = 0;
        while (done != mask) {
            int best = -1;
            for (u32 u = 0; u < n; ++u) {
                if (!((mask >> u) & 1u) || ((done >> u) & 1u)) continue;
                if (done && !(adj[u] & done)) continue;
                if (best < 0) {
                    best = (int)u;
                    continue;
                }
                const u32 du = popc(adj[u] & mask), db = popc(adj[best] & mask);
                if (cnt[u] < cnt[best] || (cnt[u] == cnt[best] && du > db)) best = (int)u;
            }
            up.order[up.n++] = (u32)best;
            done |= 1u << best;
        }
    }
    out->nunits = (u32)sets.size();
    return 0;
}

// One inner node joining every unit in unit order (or the lone unit).
void left_deep(Decomposition* d) {
    const u32 U = d->nunits;
    for (u32 k = 0; k < U; ++k) {
        d->nodes[k].unit = (int)k;
        d->nodes[k].nchild = 0;
    }
    if (U == 1) {
        d->nnodes = 1;
        d->root = 0;
        return;
    }
    JoinNode& r = d->nodes[U];
    r.unit = -1;
    r.nchild = U;
    for (u32 k = 0; k < U; ++k) r.child[k] = k;
    d->nnodes = U + 1;
    d->root = U;
}

// Bushy tree: repeatedly joins the two partial results that share a vertex
// and whose join has the smallest estimate (ties: lower node indices).
void bushy(const Model& md, Decomposition* d) {
    const u32 U = d->nunits;
    if (U < 2) {
        left_deep(d);
        return;
    }
    std::vector<u32> node(U), mask(U);
    for (u32 k = 0; k < U; ++k) {
        d->nodes[k].unit = (int)k;
        d->nodes[k].nchild = 0;
        node[k] = k;
        mask[k] = d->units[k].mask;
    }
    u32 nn = U;
    while (node.size() > 1) {
        int bi = -1, bj = -1;
        double best = 0;
        for (u32 i = 0; i < node.size(); ++i)
            for (u32 j = i + 1; j < node.size(); ++j) {
                if (!(mask[i] & mask[j])) continue;
                const double c = md.log_est(mask[i] | mask[j]);
                if (bi < 0 || c < best) bi = (int)i, bj = (int)j, best = c;
            }
        if (bi < 0) {  // no two results share a vertex (cannot happen for a connected query)
            left_deep(d);
            return;
        }
        JoinNode& r = d->nodes[nn];
        r.unit = -1;
        r.nchild = 2;
        r.child[0] = node[bi];
        r.child[1] = node[bj];
        node[bi] = nn++;
        mask[bi] |= mask[bj];
        node.erase(node.begin() + bj);
        mask.erase(mask.begin() + bj);
    }
    d->nnodes = nn;
    d->root = node[0];
}

// Orders units so that each shares a vertex with the ones before it and
// adds an edge not yet covered (units adding none are dropped): the largest
// unit first, then the unit sharing most vertices (ties: most new edges,
// then listing order).
std::vector<u32> sequence(u32 n, const u32* adj, const std::vector<u32>& units) {
    std::vector<u32> out;
    std::vector<bool> used(units.size(), false);
    u32 cov[PSM_MAXQ] = {};
    u32 acc = 0;
    auto new_edges = [&](u32 m) {
        u32 c = 0;
        for (u32 r = m; r; r &= r - 1) {
            const u32 u = __builtin_ctz(r);
            c += popc(adj[u] & m & ~cov[u]);
        }
        return c / 2;
    };
    while (true) {
        int best = -1;
        u32 bs = 0, be = 0;
        for (u32 k = 0; k < units.size(); ++k) {
            if (used[k]) continue;
            const u32 s = acc ? (u32)popc(units[k] & acc) : (u32)popc(units[k]);
            if (acc && s == 0) continue;
            const u32 e = new_edges(units[k]);
            if (e == 0) {
                used[k] = true;
                continue;
            }
            if (best < 0 || s > bs || (s == bs && e > be)) best = (int)k, bs = s, be = e;
        }
        if (best < 0) break;
        used[best] = true;
        const u32 m = units[best];
        out.push_back(m);
        for (u32 r = m; r; r &= r - 1) {
            const u32 u = __builtin_ctz(r);
            cov[u] |= adj[u] & m;
        }
        acc |= m;
    }
    return out;
}

int star_sets(u32 n, const u32* adj, u32 max_unit, std::vector<u32>& sets, std::string* err) {
    // vertex cover: repeatedly the vertex with the most uncovered edges
    u32 left[PSM_MAXQ];
    for (u32 u = 0; u < n; ++u) left[u] = adj[u];
    std::vector<u32> units;
    while (true) {
        int best = -1;
        for (u32 u = 0; u < n; ++u)
            if (left[u] && (best < 0 || popc(left[u]) > popc(left[best]))) best = (int)u;
        if (best < 0) break;
        const u32 c = (u32)best;
        u32 leaves = adj[c];
        if (max_unit >= 2 && (u32)popc(leaves) + 1 > max_unit) {
            while (leaves) {
                u32 chunk = 0;
                while (leaves && (u32)popc(chunk) < max_unit - 1) {
                    chunk |= leaves & (~leaves + 1u);
                    leaves &= leaves - 1;
                }
                units.push_back(chunk | (1u << c));
            }
        } else {
            units.push_back(leaves | (1u << c));
        }
        for (u32 r = left[c]; r; r &= r - 1) left[__builtin_ctz(r)] &= ~(1u << c);
        left[c] = 0;
    }
    if (units.empty()) {
        if (n != 1) {
            *err = "query graph has no edge";
            return 1;
        }
        sets.assign(1, 1u);
        return 0;
    }
    sets = sequence(n, adj, units);
    return 0;
}

// Best-first search (beam) over twin-twig covers with the reference's cost
// terms: each step adds a twig t to the pattern P, costing 3 card(P + t) +
// card(t) + N (SplitGraph.cpp:790-800).
int twig_sets(const Model& md, u32 n, const u32* adj, bool seed, std::vector<u32>& sets, std::string* err) {
    struct Twig {
        u32 mask;
        double log_card;
    };
    std::vector<Twig> twigs;
    for (u32 c = 0; c < n; ++c) {
        const u32 nb = adj[c];
        for (u32 r = nb; r; r &= r - 1) {
            const u32 a = __builtin_ctz(r);
            if (a > c) twigs.push_back({(1u << c) | (1u << a), md.log_card(1, 2)});
            for (u32 t = r & (r - 1); t; t &= t - 1) {
                const u32 b = __builtin_ctz(t);
                const u32 m = (1u << c) | (1u << a) | (1u << b);
                const u32 me = seed ? edges_in(adj, m) : 2u;
                twigs.push_back({m, md.log_card(me, 3)});
            }
        }
    }
    if (twigs.empty()) {
        if (n != 1) {
            *err = "query graph has no edge";
            return 1;
        }
        sets.assign(1, 1u);
        return 0;
    }
    std::sort(twigs.begin(), twigs.end(), [](const Twig& x, const Twig& y) { return x.mask < y.mask; });
    twigs.erase(std::unique(twigs.begin(), twigs.end(), [](const Twig& x, const Twig& y) { return x.mask == y.mask; }),
                twigs.end());
    u32 total_edges = 0;
    for (u32 u = 0; u < n; ++u) total_edges += popc(adj[u]);
    total_edges /= 2;
    struct State {
        u32 cov[PSM_MAXQ];
        u32 vmask, ncov;
        double cost;
        std::vector<u32> units;
    };
    const double log_3 = std::log(3.0);
    auto grow = [&](const State& s, const Twig& t, State& o) -> bool {
        const u32 m = t.mask;
        u32 add = 0;
        for (u32 r = m; r; r &= r - 1) {
            const u32 u = __builtin_ctz(r);
            add += popc(adj[u] & m & ~s.cov[u]);
        }
        if (add == 0) return false;
        if (s.vmask && !(s.vmask & m)) return false;
        std::copy(s.cov, s.cov + PSM_MAXQ, o.cov);
        for (u32 r = m; r; r &= r - 1) {
            const u32 u = __builtin_ctz(r);
            o.cov[u] |= adj[u] & m;
        }
        o.ncov = s.ncov + add / 2;
        o.vmask = s.vmask | m;
        const double step =
            s.vmask ? log_add(log_add(log_3 + md.log_card(o.ncov, popc(o.vmask)), t.log_card), md.log_n) : t.log_card;
        o.cost = log_add(s.cost, step);
        o.units = s.units;
        o.units.push_back(m);
        return true;
    };
    const size_t BEAM = 6;
    std::vector<State> beam(1);
    beam[0].vmask = 0;
    beam[0].ncov = 0;
    beam[0].cost = NEG_INF;
    std::fill(beam[0].cov, beam[0].cov + PSM_MAXQ, 0u);
    for (u32 step = 0; step < PSM_MAX_UNITS; ++step) {  // a step adds one unit
        bool all_done = true;
        for (const State& s : beam) all_done &= s.ncov == total_edges;
        if (all_done) break;
        std::vector<State> next;
        for (const State& s : beam) {
            if (s.ncov == total_edges) {
                next.push_back(s);
                continue;
            }
            for (const Twig& t : twigs) {
                State o;
                if (grow(s, t, o)) next.push_back(std::move(o));
            }
        }
        std::stable_sort(next.begin(), next.end(), [](const State& x, const State& y) {
            if (x.cost != y.cost) return x.cost < y.cost;
            return x.units.size() < y.units.size();
        });
        beam.clear();
        for (State& s : next) {
            bool dup = false;
            for (const State& b : beam)
                if (b.vmask == s.vmask && std::equal(b.cov, b.cov + PSM_MAXQ, s.cov)) dup = true;
            if (!dup) beam.push_back(std::move(s));
            if (beam.size() == BEAM) break;
        }
    }
    const State& best = beam[0];
    if (best.ncov != total_edges) {
        *err = "the twin-twig cover needs more than " + std::to_string(PSM_MAX_UNITS) + " units";
        return 1;
    }
    sets = best.units;
    return 0;
}

// Depth-first tree from the vertex of highest degree (lowest id on ties),
// neighbours in ascending order; a unit per leaf (its root path), joined
// along the tree. Every non-tree edge of an undirected depth-first tree
// joins an ancestor and a descendant, so it lies on some root-to-leaf path.
int sketch_tree(u32 n, const u32* adj, const u32* cnt, Decomposition* out, std::string* err) {
    u32 root = 0;
    for (u32 u = 1; u < n; ++u)
        if (popc(adj[u]) > popc(adj[root])) root = u;
    int parent[PSM_MAXQ];
    std::vector<u32> kids[PSM_MAXQ];
    for (u32 u = 0; u < n; ++u) parent[u] = -2;
    parent[root] = -1;
    u32 path[PSM_MAXQ];
    u32 depth = 0;
    path[depth++] = root;
    u32 visited = 1u << root;
    std::vector<u32> leaves;
    std::vector<u32> leaf_mask;
    u32 on_path = 1u << root;
    while (depth) {
        const u32 u = path[depth - 1];
        const u32 nxt = adj[u] & ~visited;
        if (nxt) {
            const u32 v = __builtin_ctz(nxt);
            visited |= 1u << v;
            parent[v] = (int)u;
            kids[u].push_back(v);
            path[depth++] = v;
            on_path |= 1u << v;
            continue;
        }
        if (kids[u].empty() && (u != root || n == 1)) {
            leaves.push_back(u);
            leaf_mask.push_back(on_path);
        }
        on_path &= ~(1u << u);
        --depth;
    }
    if (visited != (n == 32 ? 0xFFFFFFFFu : ((1u << n) - 1u))) {
        *err = "query graph is not connected";
        return 1;
    }
    if (leaves.size() > PSM_MAX_UNITS) {
        *err = "more than " + std::to_string(PSM_MAX_UNITS) + " units";
        return 1;
    }
    if (int rc = store_units(n, adj, cnt, leaf_mask, out, err)) return rc;
    u32 unit_of[PSM_MAXQ];
    for (u32 k = 0; k < leaves.size(); ++k) unit_of[leaves[k]] = k;
    u32 nn = out->nunits;
    for (u32 k = 0; k < out->nunits; ++k) {
        out->nodes[k].unit = (int)k;
        out->nodes[k].nchild = 0;
    }
    // a vertex with several children joins its subtrees' results in child
    // order (JoinCollect::recur_collect); one child passes its result up
    auto build = [&](auto&& self, u32 u) -> u32 {
        if (kids[u].empty()) return unit_of[u];
        if (kids[u].size() == 1) return self(self, kids[u][0]);
        std::vector<u32> ch;
        for (u32 c : kids[u]) ch.push_back(self(self, c));
        const u32 id = nn++;
        JoinNode& r = out->nodes[id];
        r.unit = -1;
        r.nchild = (u32)ch.size();
        for (u32 i = 0; i < ch.size(); ++i) r.child[i] = ch[i];
        return id;
    };
    out->root = build(build, root);
    out->nnodes = nn;
    return 0;
}

}  // namespace

int psm_check_decomposition(u32 n, const u32* adj, const Decomposition& d, std::string* err) {
    u32 cov[PSM_MAXQ] = {};
    for (u32 k = 0; k < d.nunits; ++k) {
        const u32 m = d.units[k].mask;
        u32 comp[PSM_MAXQ];
        if (components(adj, m, comp) != 1) {
            *err = "unit " + std::to_string(k) + " is not connected";
            return 1;
        }
        for (u32 r = m; r; r &= r - 1) {
            const u32 u = __builtin_ctz(r);
            cov[u] |= adj[u] & m;
        }
    }
    for (u32 u = 0; u < n; ++u)
        if (cov[u] != adj[u]) {
            *err = "an edge of query vertex " + std::to_string(u) + " is in no unit";
            return 1;
        }
    bool ok = true;
    auto walk = [&](auto&& self, u32 node) -> u32 {
        const JoinNode& nd = d.nodes[node];
        if (nd.unit >= 0) return d.units[nd.unit].mask;
        u32 acc = self(self, nd.child[0]);
        for (u32 i = 1; i < nd.nchild; ++i) {
            const u32 m = self(self, nd.child[i]);
            if (!(acc & m)) ok = false;
            acc |= m;
        }
        return acc;
    };
    const u32 all = walk(walk, d.root);
    if (!ok) {
        *err = "a join of the plan shares no query vertex";
        return 1;
    }
    if (all != (n == 32 ? 0xFFFFFFFFu : ((1u << n) - 1u))) {
        *err = "the plan does not reach every query vertex";
        return 1;
    }
    return 0;
}

int psm_decompose_pattern(u32 n, const u32* adj, const u32* cnt, u32 pattern, u32 join_method, u32 max_unit,
                          const PlanStats& st, Decomposition* out, std::string* err) {
    out->nunits = 0;
    out->nnodes = 0;
    if (n == 0 || n > PSM_MAXQ) {
        *err = "bad query size";
        return 1;
    }
    const Model md(n, adj, st);
    std::vector<u32> sets;
    int rc = 0;
    switch (pattern) {
        case SPLIT_BOUNDED:
            rc = bounded_sets(n, adj, max_unit, -1, sets, err);
            break;
        case SPLIT_STAR:
            rc = star_sets(n, adj, max_unit, sets, err);
            break;
        case SPLIT_TWINTWIG:
        case SPLIT_SEED:
            rc = twig_sets(md, n, adj, pattern == SPLIT_SEED, sets, err);
            break;
        case SPLIT_SKETCHTREE:
            rc = sketch_tree(n, adj, cnt, out, err);
            if (!rc) {
                out->log_cost = plan_cost(md, *out);
                rc = psm_check_decomposition(n, adj, *out, err);
            }
            return rc;
        case SPLIT_COST: {
            bool have = false;
            Decomposition cand;
            const u32 lo = max_unit > 6 ? max_unit - 4 : std::min<u32>(max_unit, 2);
            for (u32 k = max_unit; k >= lo && k >= 2; --k) {
                for (u32 s = 0; s < n; ++s) {
                    std::string e2;
                    if (bounded_sets(n, adj, k, (int)s, sets, &e2) || store_units(n, adj, cnt, sets, &cand, &e2))
                        continue;
                    if (join_method == JOIN_BUSHY)
                        bushy(md, &cand);
                    else
                        left_deep(&cand);
                    if (psm_check_decomposition(n, adj, cand, &e2)) continue;
                    cand.log_cost = plan_cost(md, cand);
                    if (!have || cand.log_cost < out->log_cost ||
                        (cand.log_cost == out->log_cost && cand.nunits < out->nunits)) {
                        *out = cand;
                        have = true;
                    }
                }
                if (k == 2) break;
            }
            if (!have) {
                *err = "no bounded decomposition fits " + std::to_string(PSM_MAX_UNITS) + " units";
                return 1;
            }
            return 0;
        }
        default:
            *err = "unknown split pattern";
            return 1;
    }
    if (rc) return rc;
    if ((rc = store_units(n, adj, cnt, sets, out, err))) return rc;
    if (join_method == JOIN_BUSHY)
        bushy(md, out);
    else
        left_deep(out);
    out->log_cost = plan_cost(md, *out);
    return psm_check_decomposition(n, adj, *out, err);
}

int psm_decompose(u32 n, const u32* adj, const u32* cnt, u32 max_unit, Decomposition* out, std::string* err) {
    PlanStats st;
    return psm_decompose_pattern(n, adj, cnt, SPLIT_BOUNDED, JOIN_LEFTDEEP, max_unit, st, out, err);
}
