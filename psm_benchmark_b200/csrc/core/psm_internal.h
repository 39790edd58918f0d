// Internal layout shared by the host runtime and the sm_100a kernels.
//
// Data graph in HBM ("label-major CSR"): vertices are renumbered so that the
// internal id of v is lab_off[L(v)] + (rank of v among vertices of label
// L(v), by original id). Label buckets are therefore contiguous id ranges,
// every adjacency list (internal ids, ascending) is grouped by label, and the
// run of label l inside a row is found with two binary searches for
// lab_off[l] and lab_off[l+1]. Ascending internal ids within a bucket are
// ascending original ids, so candidate sets and candidate positions keep the
// reference's order (matching/FilterVertices.cpp:1012-1016 sorts them).
//
// Candidate sets of a query vertex u live in "bucket space": a bitmap over
// the positions of bucket L(u) plus a per-word exclusive popcount (rank), so
// membership and the position of a data vertex inside the sorted candidate
// list cost two loads.
#pragma once
#include <stdint.h>

#define PSM_MAXQ 32          // query vertices handled by the kernels
#define PSM_MAXNLF 1024      // sum over query vertices of distinct neighbour labels
#define PSM_MAXSTEPS 96      // CFL filter steps per plan (<= 3 per query vertex)
#define PSM_MAXOPT 3         // start-vertex options kept by the CFL rank heap
#define PSM_MAXDIR 992       // directed query edges (32 * 31)
#define PSM_PLAN_WORDS 4096  // CFL order plan blob capacity (u32 words)
#define PSM_TRACE_STEPS 256  // preparation steps recorded when tracing (+1 start stamp)
#define HYBRID_REQUEST 0xFFFFFFFFu  // QState.step_cursor on entry: use the hybrid grid driver
#define PSM_CACHE_BM_BITS 32768u    // candidate positions covered by an enumerator cache bitmap
#define PSM_MEMO_CAP 8192u          // last-depth candidates covered by the per-warp weight memo

typedef uint32_t u32;
typedef uint64_t u64;

struct DevGraph {
    u32 V, L;
    const u32* off;      // [V+1]
    const u32* nbr;      // [off[V]] internal ids
    const u32* lab_off;  // [L+1] bucket ranges
    const u32* orig;     // [V] internal -> original id
    u32 loops;           // some vertex is its own neighbour (a self loop)
};

#ifndef PSM_B200_H
enum { PSM_FILTER_NLF = 0, PSM_FILTER_GQL = 1, PSM_FILTER_CFL = 2 };  // same values as psm_b200.h
enum { PSM_ORDER_GQL = 0, PSM_ORDER_CFL = 1 };
#endif
enum { STEP_GEN = 0, STEP_PRUNE = 1 };

// One CFL filtering plan (matching/GenerateFilteringPlan.cpp:81-140 and the
// step sequence of matching/FilterVertices.cpp:188-250) for one start vertex.
struct FilterPlan {
    u32 root;
    u32 nsteps;
    u32 step_u[PSM_MAXSTEPS];
    u32 step_kind[PSM_MAXSTEPS];
    u32 step_mask[PSM_MAXSTEPS];  // pivot query vertices as a bitmask
};

// Query descriptor, built on the host, read by the kernels.
struct QDesc {
    u32 n;
    u32 filter;                 // PSM_FILTER_*
    u32 order;                  // PSM_ORDER_*
    u32 data_label_count;       // L of the data graph (labels >= L have no bucket)
    u32 label[PSM_MAXQ];
    u32 deg[PSM_MAXQ];
    u32 adj[PSM_MAXQ];          // neighbour bitmask
    // NLF items: 0..n-1 are the query vertices; n..n+nvirt-1 are the
    // relabelled unit-query vertices whose candidate counts pick the CFL order
    // start vertex (only counted).
    u32 nvirt;
    u32 item_label[PSM_MAXQ + PSM_MAXOPT];
    u32 item_deg[PSM_MAXQ + PSM_MAXOPT];
    u32 nlf_off[PSM_MAXQ + PSM_MAXOPT + 1];
    u32 nlf_lab[PSM_MAXNLF];
    u32 nlf_cnt[PSM_MAXNLF];
    u32 nlf_grp[PSM_MAXNLF];    // for real vertices: neighbours carrying nlf_lab (bitmask)
    // CFL filter start-vertex options in rank-heap pop order.
    u32 nfopt;
    u32 fopt_vertex[PSM_MAXOPT];
    u32 fopt_max_score_num;     // data max label frequency + 1 (initial min score)
    FilterPlan fplan[PSM_MAXOPT];
    // CFL order start-vertex options (on the relabelled unit query).
    u32 noopt;
    u32 oopt_item[PSM_MAXOPT];  // NLF item index holding its count
    u32 oopt_vertex[PSM_MAXOPT];
    u32 oplan_off[PSM_MAXOPT];  // offset of each order plan in plan_words
    // Directed query edges grouped by source: edges of x are
    // e_first[x] .. e_first[x+1]-1 with targets in ascending order.
    u32 e_first[PSM_MAXQ + 1];
    u32 e_dst[PSM_MAXDIR];
    u32 e_src[PSM_MAXDIR];
    u32 plan_used;              // words of plan_words in use (last member: only
    u32 plan_words[PSM_PLAN_WORDS];  // the used prefix is copied to the device)
};

// CFL order plan blob layout (u32 words, starting at plan_words[oplan_off[k]]):
//   root, parent[n], nchild[n],
//   ncore, ngroups, group_path_first[ngroups+1], npaths,
//   path_off[npaths+1], nte[ncore], path_v[...], nleaves, leaves[nleaves]
// Paths 0..ncore-1 are core paths; group g holds tree paths
// group_path_first[g] .. group_path_first[g+1]-1.

// Per-query state written by the preparation kernels.
struct QState {
    const QDesc* desc;
    // candidates
    u32* bm[PSM_MAXQ];      // bucket-space bitmaps
    u32* rank[PSM_MAXQ];    // per-word exclusive popcount
    u32* list[PSM_MAXQ];    // sorted internal ids
    u32 bwords[PSM_MAXQ];   // words per bitmap
    u32 cnt[PSM_MAXQ];      // candidate counts
    u32 item_cnt[PSM_MAXQ + PSM_MAXOPT];
    u32 nlf_all;            // CFL: stage 1 left every vertex's NLF set in bm (large teams)
    u32* acc;               // CFL accumulator bitmap (max bwords)
    u32* tmp;               // CFL per-pivot bitmap
    u32 acc_words;          // words of acc / tmp
    // tables: row counts / offsets for all directed edges, concatenated
    u32* P;                 // [total_rows + 1] absolute offsets into adj
    u32 e_row_base[PSM_MAXDIR + 1];
    u32 total_rows;
    u32* adj;               // candidate positions, allocated on the device
    u32 adj_cap;            // words available at adj (set by the allocator)
    // scratch for team scans / estimates
    u32* scan;              // >= team warps + 1 words
    u64* est_a;             // est_blocks x 2 x est_stride path-estimate buffers
    u32 est_stride;         // >= max candidate count
    u32 est_blocks;         // blocks that estimate paths concurrently
    u64* est_out;           // per path estimates (<= PSM_PLAN_WORDS)
    // plan
    u32 froot, oroot;
    u32 step_cursor;        // next preparation step (hybrid grid driver)
    u64* trace;             // optional: %globaltimer at the end of each step
    u32 order[PSM_MAXQ];
    u32 pivot[PSM_MAXQ];
    u32 empty;              // some candidate set is empty -> count 0
    u32 filter_ok;          // reference filter return value (GQL/NLF early exit)
    u32 status;             // PSM_* error code from the device
    u64 table_nnz;
    u64 memory_bytes;       // computeMemoryCostInBytes
    // enumeration plan (by depth)
    u32 nbn[PSM_MAXQ];
    u32 bn_depth[PSM_MAXQ][PSM_MAXQ - 1];
    u32 bn_tab[PSM_MAXQ][PSM_MAXQ - 1];   // row base into P for table T[bn][u_d]
    u32 same_mask[PSM_MAXQ];              // earlier depths with the same label
    u32 cbase[PSM_MAXQ];                  // first internal id of the bucket of u (by query vertex)
    // Prefix-intersection cache plan (by depth d): cmask[d] = backward
    // neighbours k (bits over bn index) whose depth is <= d - 2, when there are
    // at least two of them, or one of them together with a backward neighbour
    // at depth d - 1 and a bitmap-sized candidate set (else 0). Their rows'
    // intersection depends only on the prefix up to cdep[d] = the deepest of
    // them, so the enumerator keeps it per warp (sorted list, plus a bitmap
    // over candidate positions when bm_depths has bit d) and reuses it for
    // every node below that prefix. crow[d] = bn index of the backward
    // neighbour at depth d - 1 (0xFFFFFFFF if none). cinval[x] = depths whose
    // cache is invalidated when depth x changes (cmask[d] != 0, cdep[d] >= x).
    u32 cmask[PSM_MAXQ];
    u32 crow[PSM_MAXQ];
    u32 cinval[PSM_MAXQ];
    u32 bm_depths;                        // depths with |C(u_d)| <= PSM_CACHE_BM_BITS
    // Last-two-depth weight memo (d = n-2, l = n-1): when C(u_d) depends only
    // on depths <= d-2 (its cache S_d) and depth l intersects its cache S_l
    // with the row of the depth-d vertex, the completions below a depth-(d-1)
    // node are sum over x in S_l of w(x) = |T[u_l -> u_d][x] ∩ S_d| (less
    // exact corrections for used vertices); w is memoised per warp while S_d
    // stays valid. memo_ok enables it; memo_tab = row base of T[u_l -> u_d].
    u32 memo_ok;
    u32 memo_tab;
    u32 loops;              // the data graph has a self loop (DevGraph::loops)
    u32 root_cnt;
    // results
    u64 count;
    u64 cap;                // 0 = none
    u64 calls;              // extension candidates examined
    u64 alg_bytes;          // algorithmic bytes of the intersections
    u32 stop;               // cap reached / error -> stop enumerating
    u32 overtime;
    u64 done_ns;            // %globaltimer when the cap was reached (0 if never)
    // Depths the enumerator runs: the query's n, or the size of a
    // decomposition unit whose order lists only the unit's vertices (the
    // unit reuses the query's candidates and tables).
    u32 n_enum;
    // emit mode (rows of n_enum data ids: by query vertex in original ids,
    // or, with emit_by_depth, by depth in internal ids)
    u32 emit_by_depth;
    u32* emit_buf;
    u64 emit_cap_rows;
    u64 emit_rows;
};

// Compact per-query result gathered after enumeration.
struct DevResult {
    u64 count, calls, alg_bytes, memory_bytes, table_nnz, emit_rows;
    u64 count_internal;  // unclamped count (work done before the stop)
    u32 status, overtime, filter_ok, empty;
};

// Completion record of one query of an enumeration launch, written by the
// enumerator into host-mapped memory as soon as the query's last task ends
// (serving: results leave before the rest of their batch).
struct QDoneRec {
    u64 count;     // min(count, cap)
    u64 done_ns;   // %globaltimer at completion
    u32 overtime;
    u32 status;    // PSM_DEV_* of the query's preparation
    u32 flag;      // set last: 1 once the record is complete
    u32 pad;
};

// Launch-wide counters of the enumeration scheduler, read back by the host.
struct EnumStats {
    u32 error;
    u64 donations, tasks, idle_polls;
};

// Device-side bump allocator over an arena region.
struct DevArena {
    u64 base_words;          // unused, keeps the struct 16-byte sized
    u32* base;
    unsigned long long top;  // words used
    unsigned long long cap;  // words available
};

enum {
    PSM_DEV_OK = 0,
    PSM_DEV_OOM = 2,
    PSM_DEV_TIMEOUT = 3,
    PSM_DEV_INTERNAL = 9,
};
