// Query decomposition for the join path (host side).
//
// The reference splits a query into units with SplitGraph
// (utility/splitGraph/SplitGraph.cpp:23-36; STAR: greedyStarDecomposition
// :533-660, a star around a vertex with all its neighbours) and joins the
// units' embeddings left-deep in unit order (JoinCollect::sequence_collect,
// matching/JoinCollect.cpp:237-315). Its patterns have no bound on unit
// size; here the decomposition bounds every unit by `max_unit` vertices:
//
//  1. vertex order: the vertex of highest degree first (lowest id on ties),
//     then repeatedly the unplaced vertex with the most edges to placed ones
//     (ties: higher degree, then lower id);
//  2. the first unit takes the first max_unit vertices of that order;
//  3. each later unit takes the next vertices N of the order while
//     |N| + |B| <= max_unit, where B = earlier-covered vertices adjacent to N
//     (the join keys); a vertex with max_unit or more covered neighbours gets
//     star units of itself and max_unit - 1 of those neighbours each;
//  4. a unit is the induced subgraph on N + B, split into its connected
//     components.
// Every query edge (a, b), a placed before b, lies in the unit that places b
// (a is in N or in B there), every unit after the first shares at least one
// vertex with the units before it, and every unit is connected, so a
// left-deep join over the units in order yields exactly the query's
// embeddings.
//
// Inside a unit the enumeration order is the GQL rule on the query's
// candidate counts (matching/GenerateQueryPlan.cpp:9-83): start at the
// fewest candidates (ties: higher degree in the unit, then lower id), then
// repeatedly the adjacent unplaced vertex with the fewest candidates.
#include <string>

#include "psm_b200.h"
#include "decompose.h"

namespace {

int popc(u32 x) { return __builtin_popcount(x); }

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

}  // namespace

int psm_decompose(u32 n, const u32* adj, const u32* cnt, u32 max_unit, Decomposition* out, std::string* err) {
    out->nunits = 0;
    if (n == 0 || n > PSM_MAXQ) {
        *err = "bad query size";
        return 1;
    }
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
        for (u32 u = 0; u < n; ++u) {
            if ((placed >> u) & 1u) continue;
            const int links = popc(adj[u] & placed);
            if (i > 0 && links == 0) continue;
            if (best < 0 || links > best_links || (links == best_links && deg[u] > deg[best])) {
                best = (int)u;
                best_links = links;
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
    u32 sets[2 * PSM_MAXQ * PSM_MAXQ];
    u32 nsets = 0;
    const u32 cap_sets = sizeof(sets) / sizeof(sets[0]);
    auto emit = [&](u32 mask) -> bool {
        u32 comp[PSM_MAXQ];
        const int k = components(adj, mask, comp);
        for (int c = 0; c < k; ++c) {
            if (popc(comp[c]) < 2) continue;  // a lone vertex carries no edge
            if (nsets >= cap_sets) return false;
            sets[nsets++] = comp[c];
        }
        return true;
    };
    u32 covered = 0;
    u32 i = 0;
    {
        u32 first = 0;
        for (; i < n && (u32)popc(first) < max_unit; ++i) first |= 1u << order[i];
        if (n == 1) {
            sets[nsets++] = first;  // a single-vertex query is its own unit
        } else if (!emit(first)) {
            *err = "too many units";
            return 1;
        }
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
                if (nsets >= cap_sets) {
                    *err = "too many units";
                    return 1;
                }
                sets[nsets++] = chunk | (1u << v);
            }
            covered |= 1u << v;
            continue;
        }
        if (!emit(N | B)) {
            *err = "too many units";
            return 1;
        }
        covered |= N;
    }
    if (nsets > PSM_MAX_UNITS) {
        *err = "more than " + std::to_string(PSM_MAX_UNITS) + " units";
        return 1;
    }
    // unit orders
    for (u32 k = 0; k < nsets; ++k) {
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
    out->nunits = nsets;
    return 0;
}
