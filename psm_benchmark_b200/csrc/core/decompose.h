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

struct Decomposition {
    u32 nunits;
    UnitPlan units[PSM_MAX_UNITS];
};

// adj: neighbour masks of the n query vertices; cnt: candidate counts (unit
// orders only). Returns 0, or 1 with *err set.
int psm_decompose(u32 n, const u32* adj, const u32* cnt, u32 max_unit, Decomposition* out, std::string* err);
