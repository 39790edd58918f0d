// Query decomposition for the join path (decompose.cpp).
#pragma once
#include <string>

#include "psm_internal.h"

#define PSM_MAX_UNITS 32

struct UnitPlan {
    u32 mask;            // unit vertices
    u32 n;               // their number
    u32 order[PSM_MAXQ]; // enumeration order (query vertex ids)
};

// Join tree: a node with unit >= 0 is a leaf (that unit's embeddings); an
// inner node joins the results of its children in child order (the first
// child's result is joined with the second's, that with the third's, ...).
// A left-deep plan is one inner node whose children are all units in order.
struct JoinNode {
    int unit;
    u32 nchild;
    u32 child[PSM_MAX_UNITS];
};

struct Decomposition {
    u32 nunits;
    UnitPlan units[PSM_MAX_UNITS];
    u32 nnodes;
    u32 root;
    JoinNode nodes[2 * PSM_MAX_UNITS];
    double log_cost;     // the plan's estimated materialised rows (natural log)
};

// Inputs of the cost model. Per query vertex u: cand[u] candidates; per
// ordered pair (a, b) of adjacent query vertices: edge_p[a * n + b], the
// fraction of candidate pairs (C(a) x C(b)) joined by a data edge. Without
// them (null), the reference's label-blind model card(m, n) = (2M)^m /
// N^(2m - n) of a pattern with m edges and n vertices is used
// (utility/splitGraph/SplitGraph.cpp:17-21).
struct PlanStats {
    double data_vertices = 1;  // N
    double data_edges = 1;     // M
    const double* cand = nullptr;
    const double* edge_p = nullptr;
};

// Decomposition patterns (the reference's -Qpattern values plus two of this
// library's own); values match psm_split_pattern in psm_b200.h.
enum : u32 {
    SPLIT_BOUNDED = 0,
    SPLIT_STAR = 1,
    SPLIT_TWINTWIG = 2,
    SPLIT_SEED = 3,
    SPLIT_SKETCHTREE = 4,
    SPLIT_COST = 5,
};
enum : u32 { JOIN_LEFTDEEP = 0, JOIN_BUSHY = 1 };

// adj: neighbour masks of the n query vertices; cnt: candidate counts (unit
// orders only). Bounded units, left-deep. Returns 0, or 1 with *err set.
int psm_decompose(u32 n, const u32* adj, const u32* cnt, u32 max_unit, Decomposition* out, std::string* err);
// Any pattern and join method (max_unit bounds BOUNDED, COST and STAR units;
// 0 = no bound for STAR).
int psm_decompose_pattern(u32 n, const u32* adj, const u32* cnt, u32 pattern, u32 join_method, u32 max_unit,
                          const PlanStats& st, Decomposition* out, std::string* err);
// Checks a decomposition: every query edge inside some unit, every unit
// connected, and every join of the tree between results that share a query
// vertex. Returns 0, or 1 with *err set.
int psm_check_decomposition(u32 n, const u32* adj, const Decomposition& d, std::string* err);
