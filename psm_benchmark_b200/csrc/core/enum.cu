// Backtracking enumeration of embeddings on the device.
//
// Semantics follow the reference's LFTJ engine
// (matching/EvaluateQuery.cpp:231-372 with generateValidCandidateIndex
// :2024-2082): at depth d the candidates of u_d are the intersection of the
// candidate-edge table rows of all earlier neighbours, and a data vertex
// already used by the partial embedding is skipped. All of the reference's
// engines (GQL, EXPLORE, LFTJ) count the same embeddings; this kernel serves
// all of them.
//
// Execution model (replaces TaskPool's threads, matching/TaskPool.cpp):
//  - a persistent grid of warps; each warp runs a depth-first search whose
//    stack (per depth: candidate position, data vertex, unexplored range of
//    the driving table row, and a 32-entry chunk of surviving candidates)
//    lives in shared memory;
//  - candidates are generated 32 at a time: lane i takes element i of the
//    shortest backward-neighbour row (the "driver"), binary-searches it in
//    the other rows and checks it against same-label earlier vertices; a
//    ballot compacts the survivors. The last two depths are fused: each lane
//    takes one candidate of depth n-2 and counts its completions itself;
//  - initial work: the edges of the first candidate-edge table (pairs of
//    depth-0 / depth-1 candidates) of every query of the launch, handed out
//    in chunks by one atomic ticket; queries of up to three vertices hand out
//    root candidates instead;
//  - load balance: an idle warp raises a "hungry" counter; while more warps
//    are hungry than tasks are queued, busy warps donate the upper half of
//    their shallowest unexplored range (the reference's "linear" split,
//    TaskPool.cpp:1407-1424) to a bounded lock-free queue;
//  - termination: a pending-work counter (the initial pool + live tasks)
//    reaches zero. Every wait is bounded by a deadline and an iteration cap;
//    on expiry the kernel records an error and returns.
#include <cuda_runtime.h>

#include "device_util.cuh"
#include "psm_internal.h"

namespace {

constexpr u32 QCAP = 4096;     // steal queue slots
constexpr u32 HDR_WORDS = 6;   // kind, qi, d0, b, e, drv
constexpr u32 TASK_WORDS = HDR_WORDS + PSM_MAXQ;
constexpr u32 WARPS_PER_BLOCK = 8;

enum : u32 {
    KIND_RANGE = 0,  // driver range [b, e) at depth d0, prefix pos[0, d0)
    KIND_FULL = 1,   // whole driver row of depth d0, prefix pos[0, d0)
    KIND_EDGES = 2,  // edges [b, e) of the first table (absolute entry indices)
};

struct TaskHdr {
    u32 kind, qi, d0, b, e, drv;
};

struct Slot {
    u32 seq;
    u32 w[TASK_WORDS];
};

}  // namespace

struct EnumCtl {
    u32 ticket;         // next grab of the initial pool
    u32 total_grabs;
    u32 hungry;
    u32 q_head;
    u32 q_tail;
    u32 error;
    u32 nq;
    u32 pad;
    unsigned long long pending;
    u64 deadline_ns;
    u64 donations;
    u64 tasks;
    u64 idle_polls;
    u32* remaining;     // per query: grabs + donated tasks not yet finished
    QDoneRec* done;     // per query completion records (host-mapped) or null
    u32 exit_keep;      // > 0: idle warps beyond this many leave once no work is left
    u32 pad2;
};

namespace {

// Level flags (WarpStack::flg). A level in cached mode intersects at most
// two sorted arrays: the depth's prefix-intersection cache S (the rows of
// the backward neighbours at depths <= d - 2, intersected once per prefix)
// and the row R of the backward neighbour at depth d - 1, if any.
enum : u32 {
    LV_CACHED = 1,     // cached mode
    LV_DRV_CACHE = 2,  // the driver range indexes S (else q.adj)
    LV_OTHER = 4,      // the array that is not the driver is tested: R at [olo, ohi), or S
    LV_OTHER_BM = 8,   // ... and S is tested through its bitmap
};
// Per warp and depth a slot of CACHE_CAP list entries and BM_WORDS bitmap
// words. A cache whose intersection is longer than CACHE_CAP is not kept;
// a single cached row stays in q.adj and only its bitmap is built.
constexpr u32 CACHE_CAP = 512;
constexpr u32 BM_WORDS = PSM_CACHE_BM_BITS / 32;
constexpr u32 SLOT_WORDS = CACHE_CAP + BM_WORDS;
constexpr u32 WARP_CACHE_WORDS = PSM_MAXQ * SLOT_WORDS + PSM_MEMO_CAP;  // slots + weight memo
constexpr u32 NO_ROW = 0xFFFFFFFFu;
constexpr u32 LONG_ROW = 24;     // per-lane binary-search walks longer than this go to the warp
constexpr u32 LONG_BM_ROW = 96;  // per-lane bitmap walks longer than this go to the warp
// With only `act` lanes holding a candidate, a lane's walk costs the warp its
// whole length while the cooperative walk costs about 1/32 of it plus a fixed
// setup: walks longer than these multiples of `act` go to the warp too.
constexpr u32 DEFER_BM_PER_LANE = 8;
constexpr u32 DEFER_ROW_PER_LANE = 2;

// Invariants of the cache state: cvalid bit d => S of depth d is the
// intersection for the current prefix; cbits bit d => the bitmap of depth d
// holds exactly the bits of the list S_d (clen[d] entries, in q.adj from
// clo[d] when cadj bit d, else in the slot). Every bitmap is all-zero while
// its bit in cbits is clear; run_task clears them all before it returns, so
// bitmaps start each task (and each launch) empty.
struct WarpStack {
    u32* cbuf;          // this warp's slots (null: caching off)
    u32* memo;          // this warp's weight memo [PSM_MEMO_CAP] (entries w + 1; 0 = not known)
    u64 rsum;           // memo: total length of the depth-l rows of S_d's candidates (valid with rsum_ok)
    u32 rsum_ok;
    u32 lvfull;         // depths whose driver range is the whole level (not a donated part)
    u32 cvalid;
    u32 cover;          // depths whose intersection overflowed CACHE_CAP for the current prefix
    u32 cbits;
    u32 cadj;
    u32 near_q;         // query within reach of its cap: publish in small steps (~0: none)
    u32 pos[PSM_MAXQ];
    u32 vid[PSM_MAXQ];
    u32 cur[PSM_MAXQ];
    u32 end[PSM_MAXQ];
    u32 drv[PSM_MAXQ];
    u32 cn[PSM_MAXQ];
    u32 ci[PSM_MAXQ];
    u32 flg[PSM_MAXQ];
    u32 olo[PSM_MAXQ];
    u32 ohi[PSM_MAXQ];
    u32 clen[PSM_MAXQ];
    u32 clo[PSM_MAXQ];
    u32 csum[PSM_MAXQ];  // total length of the rows behind S (algorithmic bytes)
    u32 chunk[PSM_MAXQ][32];
};

// Per query, filled by enum_init_kernel: how the initial pool of a query is
// cut into grabs.
struct PoolInfo {
    u32 kind;   // KIND_RANGE (roots) or KIND_EDGES
    u32 units;  // roots or first-table edges
    u32 grab;   // units per grab
    u32 first;  // absolute index of unit 0 (edges: P[base])
};

__device__ __forceinline__ u32 row_lo(const QState& q, u32 d, u32 k, const u32* pos) {
    return q.P[q.bn_tab[d][k] + pos[q.bn_depth[d][k]]];
}
__device__ __forceinline__ u32 row_hi(const QState& q, u32 d, u32 k, const u32* pos) {
    return q.P[q.bn_tab[d][k] + pos[q.bn_depth[d][k]] + 1];
}

__device__ __forceinline__ u32* slot_list(const WarpStack* ws, u32 d) { return ws->cbuf + d * SLOT_WORDS; }
__device__ __forceinline__ u32* slot_bm(const WarpStack* ws, u32 d) { return ws->cbuf + d * SLOT_WORDS + CACHE_CAP; }
// The sorted list S of depth d (valid while cvalid or cbits has bit d).
__device__ __forceinline__ const u32* cache_list(const QState& q, const WarpStack* ws, u32 d) {
    return ((ws->cadj >> d) & 1u) ? q.adj + ws->clo[d] : slot_list(ws, d);
}
__device__ __forceinline__ bool bm_test(const u32* bm, u32 x) { return (bm[x >> 5] >> (x & 31u)) & 1u; }
// Membership of candidate position x in S of depth d (bitmap when built).
__device__ __forceinline__ bool in_cache(const QState& q, const WarpStack* ws, u32 d, u32 x) {
    if ((ws->cbits >> d) & 1u) return bm_test(slot_bm(ws, d), x);
    return contains_rw(cache_list(q, ws, d), 0, ws->clen[d], x);
}

// Clears the bitmap bits of depth d (from its list), if any are set.
__device__ void clear_bits(const QState& q, WarpStack* ws, u32 d) {
    if (!((ws->cbits >> d) & 1u)) return;
    const u32* L = cache_list(q, ws, d);
    const u32 n = ws->clen[d];
    u32* bm = slot_bm(ws, d);
    for (u32 i = lane_id(); i < n; i += 32) bm[L[i] >> 5] = 0u;
    __syncwarp();
    if (lane_id() == 0) ws->cbits &= ~(1u << d);
    __syncwarp();
}

// Sets the bitmap bits of depth d from its (ascending) list: lanes holding
// positions of one word OR their bits together and one of them stores, so
// every word has a single writer per pass.
__device__ void set_bits(const QState& q, WarpStack* ws, u32 d) {
    const u32* L = cache_list(q, ws, d);
    const u32 n = ws->clen[d];
    u32* bm = slot_bm(ws, d);
    const u32 lane = lane_id();
    for (u32 j = 0; j < n; j += 32) {
        const bool valid = j + lane < n;
        const u32 x = valid ? L[j + lane] : 0u;
        const u32 w = valid ? (x >> 5) : 0xFFFFFFFFu;
        const u32 peers = __match_any_sync(FULL_MASK, w);
        const u32 bits = __reduce_or_sync(peers, valid ? (1u << (x & 31u)) : 0u);
        if (valid && lane == (u32)(__ffs(peers) - 1)) bm[w] |= bits;
        __syncwarp();
    }
    if (lane == 0) ws->cbits |= 1u << d;
    __syncwarp();
}

// Clears every bitmap this warp has set (end of a task).
__device__ void release_caches(const QState& q, WarpStack* ws) {
    for (u32 m = ws->cbits; m; m &= m - 1) clear_bits(q, ws, __ffs(m) - 1);
    __syncwarp();
    if (lane_id() == 0) {
        ws->cvalid = 0;
        ws->cover = 0;
        ws->cadj = 0;
    }
    __syncwarp();
}

// Makes the cache S of depth d hold the intersection of the rows q.cmask[d]
// for the current prefix, building it when needed (one row: kept in place;
// several: driver = shortest row, one lane per driver entry, ballot
// compaction into the slot), then its bitmap when the candidate set of the
// depth is small enough. Returns false when depth d has no cache plan,
// caching is off, or the intersection has more than CACHE_CAP entries; the
// level then intersects the table rows directly.
template <u32 IS>
__device__ bool ensure_cache(const QState& q, u32 d, WarpStack* ws, u64& bytes) {
    const u32 cm = q.cmask[d];
    if (cm == 0 || ws->cbuf == nullptr) return false;
    const u32 bit = 1u << d;
    if (ws->cvalid & bit) return true;
    if (ws->cover & bit) return false;
    clear_bits(q, ws, d);
    const u32 lane = lane_id();
    bool over = false;
    if (__popc(cm) == 1) {
        const u32 k = __ffs(cm) - 1;
        const u32 lo = row_lo(q, d, k, ws->pos), hi = row_hi(q, d, k, ws->pos);
        __syncwarp();
        if (lane == 0) {
            ws->cadj |= bit;
            ws->clo[d] = lo;
            ws->clen[d] = hi - lo;
            ws->csum[d] = hi - lo;
        }
        __syncwarp();
    } else {
        u32 best = 0, blo = 0, blen = 0xFFFFFFFFu, tot = 0;
        u32 best2 = 0, b2lo = 0, b2len = 0xFFFFFFFFu;
        for (u32 m = cm; m; m &= m - 1) {
            const u32 k = __ffs(m) - 1;
            const u32 lo = row_lo(q, d, k, ws->pos), hi = row_hi(q, d, k, ws->pos);
            tot += hi - lo;
            if (hi - lo < blen) {
                b2len = blen, b2lo = blo, best2 = best;
                blen = hi - lo, blo = lo, best = k;
            } else if (hi - lo < b2len) {
                b2len = hi - lo, b2lo = lo, best2 = k;
            }
        }
        u32* out = slot_list(ws, d);
        const u32 rest = cm & ~(1u << best);
        u32 n = 0;
        if (IS != ISECT_BINARY && warp_merge_pays(IS, blen, b2len)) {
            // merge path over the two shortest rows; their common entries
            // that are in every other row make the list
            const u32* A = q.adj + blo;
            const u32 rest2 = rest & ~(1u << best2);
            n = warp_merge_collect<true, true>(A, blen, q.adj + b2lo, b2len, &q.stop, out, CACHE_CAP, &over,
                                               [&](u32 i) {
                                                   const u32 x = __ldg(A + i);
                                                   for (u32 m = rest2; m; m &= m - 1) {
                                                       const u32 k = __ffs(m) - 1;
                                                       if (!contains_u32(q.adj, row_lo(q, d, k, ws->pos),
                                                                         row_hi(q, d, k, ws->pos), x))
                                                           return false;
                                                   }
                                                   return true;
                                               });
            blen = 0;  // the chunked walk below has nothing left to do
        }
        for (u32 j = 0; j < blen; j += 32) {
            // a stopped query's long intersections end early: the cache is
            // then not kept (the level falls back to the table rows)
            if (j && (j & 4095u) == 0 && warp_ld_volatile_u32(&q.stop)) {
                over = true;
                break;
            }
            bool ok = j + lane < blen;
            const u32 x = ok ? __ldg(q.adj + blo + j + lane) : 0u;
            for (u32 m = rest; m && ok; m &= m - 1) {
                const u32 k = __ffs(m) - 1;
                ok = contains_u32(q.adj, row_lo(q, d, k, ws->pos), row_hi(q, d, k, ws->pos), x);
            }
            const u32 bal = __ballot_sync(FULL_MASK, ok);
            const u32 c = __popc(bal);
            if (n + c > CACHE_CAP) {
                over = true;
                break;
            }
            if (ok) out[n + __popc(bal & ((1u << lane) - 1u))] = x;
            n += c;
        }
        __syncwarp();
        if (lane == 0) {
            ws->cadj &= ~bit;
            ws->clen[d] = over ? 0u : n;
            ws->csum[d] = tot;
        }
        __syncwarp();
    }
    if (!over && ((q.bm_depths >> d) & 1u)) set_bits(q, ws, d);
    if (q.memo_ok && d + 2 == q.n_enum) {
        // the weight memo belongs to S_d: start it afresh
        const u32 nl = q.cnt[q.order[d + 1]];
        for (u32 i = lane; i < nl; i += 32) ws->memo[i] = 0u;
        __syncwarp();
        if (lane == 0) ws->rsum_ok = 0;
        __syncwarp();
    }
    if (lane == 0) {
        if (over)
            ws->cover |= bit;
        else
            ws->cvalid |= bit;
    }
    __syncwarp();
    return !over;
}

// Whether to walk R (length r) and test S through its bitmap rather than
// walk the shorter side and binary-search the other.
__device__ __forceinline__ bool walk_r_with_bitmap(const WarpStack* ws, u32 d, u32 r, u32 s) {
    return ((ws->cbits >> d) & 1u) && r <= 2u * s + 32u;
}

// Sets up depth d for the current prefix: cached mode when the depth's cache
// is usable, else the shortest backward-neighbour row drives and the others
// are tested. Adds the algorithmic bytes of the level -- those of the
// reference's intersection of all backward-neighbour rows (8 B of offsets +
// 4 B per entry each), whether or not a cache saved reading them; returns
// the driver length.
template <u32 IS>
__device__ __forceinline__ u32 setup_level(const QState& q, u32 d, WarpStack* ws, u64& bytes) {
    u32 flg = 0, best = 0, dlo = 0, dhi = 0, olo = 0, ohi = 0;
    if (ensure_cache<IS>(q, d, ws, bytes)) {
        const u32 s = ws->clen[d];
        const u32 k = q.crow[d];
        flg = LV_CACHED | LV_DRV_CACHE;
        dhi = s;
        bytes += 8ull * q.nbn[d] + 4ull * ws->csum[d];
        if (k != NO_ROW) {
            const u32 lo = row_lo(q, d, k, ws->pos), hi = row_hi(q, d, k, ws->pos);
            bytes += 4ull * (hi - lo);
            if (walk_r_with_bitmap(ws, d, hi - lo, s)) {
                flg = LV_CACHED | LV_OTHER | LV_OTHER_BM;
                best = k, dlo = lo, dhi = hi;
            } else if (hi - lo < s) {
                flg = LV_CACHED | LV_OTHER;
                best = k, dlo = lo, dhi = hi, olo = 0, ohi = s;
            } else {
                flg |= LV_OTHER;
                olo = lo, ohi = hi;
            }
        }
    } else {
        const u32 nb = q.nbn[d];
        u32 blen = 0xFFFFFFFFu;
        u64 by = 0;
        for (u32 k = 0; k < nb; ++k) {
            u32 lo = row_lo(q, d, k, ws->pos), hi = row_hi(q, d, k, ws->pos);
            by += 8u + 4ull * (hi - lo);
            if (hi - lo < blen) blen = hi - lo, best = k, dlo = lo, dhi = hi;
        }
        bytes += by;
    }
    __syncwarp();
    if (lane_id() == 0) {
        ws->flg[d] = flg;
        ws->drv[d] = best;
        ws->cur[d] = dlo;
        ws->end[d] = dhi;
        ws->olo[d] = olo;
        ws->ohi[d] = ohi;
        ws->cn[d] = 0;
        ws->ci[d] = 0;
        ws->lvfull |= 1u << d;
    }
    __syncwarp();
    return dhi - dlo;
}

// Element idx of depth d's driver array (d >= 1).
__device__ __forceinline__ u32 drv_elem(const QState& q, const WarpStack* ws, u32 d, u32 idx) {
    return (ws->flg[d] & LV_DRV_CACHE) ? cache_list(q, ws, d)[idx] : q.adj[idx];
}

// True if position x lies in depth d's driver range [lo, hi).
__device__ __forceinline__ bool drv_contains(const QState& q, const WarpStack* ws, u32 d, u32 lo, u32 hi, u32 x) {
    return (ws->flg[d] & LV_DRV_CACHE) ? contains_rw(cache_list(q, ws, d), lo, hi, x)
                                       : contains_u32(q.adj, lo, hi, x);
}

// Position of data vertex v (same label as query vertex u) among the sorted
// candidates of u, from u's bitmap and rank; 0xFFFFFFFF if not a candidate.
__device__ __forceinline__ u32 cand_pos(const QState& q, u32 u, u32 v) {
    const u32 b = v - q.cbase[u];
    const u32 word = q.bm[u][b >> 5];
    if (!((word >> (b & 31u)) & 1u)) return 0xFFFFFFFFu;
    return q.rank[u][b >> 5] + __popc(word & ((1u << (b & 31u)) - 1u));
}

// Writes a finished query's completion record (its count is final: every
// task of the query published before the caller's counter reached zero).
__device__ void finish_query(QState& q, QDoneRec* rec) {
    __threadfence();
    const u64 c = atomicAdd((unsigned long long*)&q.count, 0ull);
    rec->count = q.cap && c > q.cap ? q.cap : c;
    rec->overtime = ld_volatile_u32(&q.overtime);
    rec->status = q.status;
    rec->done_ns = global_timer_ns();
    __threadfence_system();
    *(volatile u32*)&rec->flag = 1u;
}

// Marks the query stopped (cap reached); the first caller stamps the time.
__device__ __forceinline__ void cap_reached(QState& q) {
    if (atomicExch(&q.stop, 1u) == 0) q.done_ns = global_timer_ns();
}

// One lane's candidate test at depth d for driver element p (a position in
// C(u_d)): member of every other array of the level and not a data vertex
// already used by a same-label earlier depth.
__device__ __forceinline__ bool accept(const QState& q, u32 d, u32 p, const WarpStack* ws, const u32* list_d) {
    const u32 f = ws->flg[d];
    if (f & LV_CACHED) {
        if (f & LV_OTHER) {
            bool in;
            if (f & LV_OTHER_BM)
                in = bm_test(slot_bm(ws, d), p);
            else if (f & LV_DRV_CACHE)
                in = contains_u32(q.adj, ws->olo[d], ws->ohi[d], p);
            else
                in = contains_rw(cache_list(q, ws, d), ws->olo[d], ws->ohi[d], p);
            if (!in) return false;
        }
    } else {
        const u32 nb = q.nbn[d], drv = ws->drv[d];
        for (u32 k = 0; k < nb; ++k) {
            if (k == drv) continue;
            u32 lo = row_lo(q, d, k, ws->pos), hi = row_hi(q, d, k, ws->pos);
            if (!contains_u32(q.adj, lo, hi, p)) return false;
        }
    }
    u32 m = q.same_mask[d];
    if (m) {
        u32 v = list_d[p];
        while (m) {
            u32 j = __ffs(m) - 1;
            m &= m - 1;
            if (ws->vid[j] == v) return false;
        }
    }
    return true;
}

// Candidate test of one lane's driver element p at depth d (lanes whose
// element lies past the row end pass valid = false).
__device__ __forceinline__ bool chunk_accept(const QState& q, u32 d, u32 p, bool valid, WarpStack* ws,
                                             const u32* list_d) {
    return valid && accept(q, d, p, ws, list_d);
}

// Warp-level count of the candidates of the last depth d given the prefix.
template <u32 IS>
__device__ u64 count_last(const QState& q, u32 d, WarpStack* ws, u64& bytes, u64& calls) {
    const u32 lane = lane_id();
    const u32 u = q.order[d];
    const u32* list_d = q.list[u];
    const u32 len = setup_level<IS>(q, d, ws, bytes);
    calls += len;
    if (len == 0) return 0;
    const u32 f = ws->flg[d];
    const u32 lo = ws->cur[d], hi = ws->end[d];
    const bool single = (f & LV_CACHED) ? !(f & LV_OTHER) : q.nbn[d] == 1;
    if (single) {
        // every driver entry is a candidate: subtract the used same-label
        // vertices whose position is in the range
        const u32 same = q.same_mask[d];
        u32 hit = 0;
        if ((same >> lane) & 1u) {
            const u32 x = cand_pos(q, u, ws->vid[lane]);
            hit = (x != 0xFFFFFFFFu && drv_contains(q, ws, d, lo, hi, x)) ? 1u : 0u;
        }
        return len - __popc(__ballot_sync(FULL_MASK, hit));
    }
    u64 c = 0;
    for (u32 j = 0; j < len; j += 32) {
        const bool valid = j + lane < len;
        const u32 p = valid ? drv_elem(q, ws, d, lo + j + lane) : 0u;
        c += __popc(__ballot_sync(FULL_MASK, chunk_accept(q, d, p, valid, ws, list_d)));
    }
    return c;
}

// Emits the embeddings of the last depth (original data ids, indexed by
// query vertex) into q.emit_buf; returns how many were found.
template <u32 IS>
__device__ u64 emit_last(QState& q, const DevGraph& g, u32 d, WarpStack* ws, u64& bytes, u64& calls) {
    const u32 lane = lane_id();
    const u32 n = d + 1;
    const u32 u = q.order[d];
    const u32* list_d = q.list[u];
    // A capped query stops emitting as soon as the rows reach its cap (the
    // rows emitted so far are the rows counted): a stopped query emits
    // nothing more, and the chunk that crosses the cap is the warp's last.
    if (q.cap && warp_ld_volatile_u32(&q.stop)) return 0;
    u32 blen = setup_level<IS>(q, d, ws, bytes);
    calls += blen;
    const u32 bs = ws->cur[d];
    u64 c = 0;
    for (u32 j = 0; j < blen; j += 32) {
        // another warp may have reached the cap during a long level
        if (q.cap && j && (j & 511u) == 0 && warp_ld_volatile_u32(&q.stop)) break;
        bool ok = false;
        u32 p = 0;
        if (j + lane < blen) {
            p = drv_elem(q, ws, d, bs + j + lane);
            ok = accept(q, d, p, ws, list_d);
        }
        u32 bal = __ballot_sync(FULL_MASK, ok);
        u32 k = __popc(bal);
        if (!k) continue;
        unsigned long long base = 0;
        if (lane == 0) {
            base = atomicAdd((unsigned long long*)&q.emit_rows, (unsigned long long)k);
            if (q.cap && base + k >= q.cap) cap_reached(q);
        }
        base = __shfl_sync(FULL_MASK, base, 0);
        if (ok) {
            u64 row = base + __popc(bal & ((1u << lane) - 1u));
            if (row < q.emit_cap_rows) {
                u32* out = q.emit_buf + row * n;
                if (q.emit_by_depth) {
                    for (u32 i = 0; i < d; ++i) out[i] = ws->vid[i];
                    out[d] = list_d[p];
                } else {
                    for (u32 i = 0; i < d; ++i) out[q.order[i]] = g.orig[ws->vid[i]];
                    out[u] = g.orig[list_d[p]];
                }
            }
        }
        c += k;
        if (q.cap && base + k >= q.cap) break;  // warp-uniform: base is broadcast
    }
    return c;
}

// Last-depth counts of the fused last two depths. The lane's own candidate
// p (data vertex v) sits at depth dl - 1, the rest of the prefix is shared
// in ws. A count is the number of positions in the intersection of the
// backward-neighbour rows of depth dl whose data vertex differs from every
// same-label vertex of the embedding. With `cached`, depth dl's cache S
// (warp-shared, valid for the prefix) stands for the rows of depths
// <= dl - 2, and only the lane's own row R (when p's depth is a backward
// neighbour) is intersected with it: R walked against S's bitmap, or the
// shorter side binary-searched in the other. A walk longer than LONG_ROW
// (LONG_BM_ROW for bitmap walks) is not done by the lane: it sets *defer and
// the warp counts it cooperatively afterwards (warp_last_count), so one hub
// row does not stall 31 idle lanes.

// Used same-label vertices (the lane's own v at depth dl - 1, the rest from
// ws) whose position lies in S of dl and, when has_row, in R = adj[lo, hi).
// R is then v's own row, which holds v only through a self loop: without
// one, v is not looked up.
__device__ __forceinline__ u32 cached_exclusions(const QState& q, u32 dl, u32 v, const WarpStack* ws, bool has_row,
                                                 u32 lo, u32 hi) {
    const u32 u = q.order[dl];
    const u32 dp = dl - 1;
    u32 c = 0;
    for (u32 m = q.same_mask[dl]; m; m &= m - 1) {
        const u32 j = __ffs(m) - 1;
        if (j == dp && has_row && !q.loops) continue;
        const u32 x = cand_pos(q, u, j == dp ? v : ws->vid[j]);
        if (x != 0xFFFFFFFFu && in_cache(q, ws, dl, x) && (!has_row || contains_u32(q.adj, lo, hi, x))) ++c;
    }
    return c;
}

template <u32 IS>
__device__ u64 lane_last_count(const QState& q, u32 dl, bool cached, u32 p, u32 v, const WarpStack* ws, u64& bytes,
                               u64& calls, bool* defer, u32 act) {
    const u32 nb = q.nbn[dl];
    const u32 dp = dl - 1;
    const u32 long_bm = min(LONG_BM_ROW, DEFER_BM_PER_LANE * act);
    const u32 long_row = min(LONG_ROW, max(2u, DEFER_ROW_PER_LANE * act));
    if (cached) {
        const u32 s = ws->clen[dl];
        const u32 k = q.crow[dl];
        bytes += 8ull * nb + 4ull * ws->csum[dl];
        if (k == NO_ROW) {
            calls += s;
            return s - cached_exclusions(q, dl, v, ws, false, 0, 0);
        }
        const u32 base = q.bn_tab[dl][k] + p;
        const u32 lo = q.P[base], hi = q.P[base + 1], r = hi - lo;
        bytes += 4ull * r;
        if (s == 0 || r == 0) return 0;
        u64 c = 0;
        if (walk_r_with_bitmap(ws, dl, r, s)) {
            calls += r;
            if (r > long_bm) {
                *defer = true;
                return 0;
            }
            const u32* bm = slot_bm(ws, dl);
            for (u32 e = lo; e < hi; ++e) c += bm_test(bm, __ldg(q.adj + e));
        } else {
            calls += min(s, r);
            if (min(s, r) > long_row) {
                *defer = true;
                return 0;
            }
            const u32* S = cache_list(q, ws, dl);
            if constexpr (IS != ISECT_BINARY) {
                c = r <= s ? lane_isect_count<true, false>(q.adj + lo, r, S, s, IS)
                           : lane_isect_count<false, true>(S, s, q.adj + lo, r, IS);
            } else if (r <= s) {
                for (u32 e = lo; e < hi; ++e) c += contains_rw(S, 0, s, __ldg(q.adj + e));
            } else {
                for (u32 i = 0; i < s; ++i) c += contains_u32(q.adj, lo, hi, S[i]);
            }
        }
        return c - cached_exclusions(q, dl, v, ws, true, lo, hi);
    }
    u32 blo = 0, bhi = 0, blen = 0xFFFFFFFFu, bk = 0;
    u64 by = 0;
    for (u32 k = 0; k < nb; ++k) {
        const u32 bd = q.bn_depth[dl][k];
        const u32 base = q.bn_tab[dl][k] + (bd == dp ? p : ws->pos[bd]);
        const u32 lo = q.P[base], hi = q.P[base + 1];
        by += 8u + 4ull * (hi - lo);
        if (hi - lo < blen) blen = hi - lo, blo = lo, bhi = hi, bk = k;
    }
    bytes += by;
    calls += blen;
    if (blen == 0) return 0;
    if (nb > 1 && blen > long_row) {
        *defer = true;
        return 0;
    }
    const u32 u = q.order[dl];
    const u32 same = q.same_mask[dl];
    if (nb == 1) {
        u64 c = blen;
        u32 m = same;
        // the row of v's own depth holds v only through a self loop
        if (q.bn_depth[dl][0] == dp && !q.loops) m &= ~(1u << dp);
        while (m) {
            const u32 j = __ffs(m) - 1;
            m &= m - 1;
            const u32 x = cand_pos(q, u, j == dp ? v : ws->vid[j]);
            if (x != 0xFFFFFFFFu && contains_u32(q.adj, blo, bhi, x)) --c;
        }
        return c;
    }
    const u32* list = q.list[u];
    u64 c = 0;
    for (u32 e = blo; e < bhi; ++e) {
        const u32 x = __ldg(q.adj + e);
        bool ok = true;
        for (u32 k = 0; k < nb && ok; ++k) {
            if (k == bk) continue;
            const u32 bd = q.bn_depth[dl][k];
            const u32 base = q.bn_tab[dl][k] + (bd == dp ? p : ws->pos[bd]);
            ok = contains_u32(q.adj, q.P[base], q.P[base + 1], x);
        }
        if (ok && same) {
            const u32 vx = __ldg(list + x);
            u32 m = same;
            while (m && ok) {
                const u32 j = __ffs(m) - 1;
                m &= m - 1;
                ok = vx != (j == dp ? v : ws->vid[j]);
            }
        }
        c += ok;
    }
    return c;
}

// Warp-cooperative form of lane_last_count for one (p, v) (warp-uniform):
// the walked side is taken 32 entries at a time, each lane testing its entry
// against the other arrays. Rows and bytes were counted by the lane that
// deferred it.
template <u32 IS>
__device__ u64 warp_last_count(const QState& q, u32 dl, bool cached, u32 p, u32 v, const WarpStack* ws) {
    const u32 lane = lane_id();
    const u32 nb = q.nbn[dl];
    const u32 dp = dl - 1;
    if (cached) {
        // deferred only with a row at depth dl - 1
        const u32 s = ws->clen[dl];
        const u32 base = q.bn_tab[dl][q.crow[dl]] + p;
        const u32 lo = q.P[base], hi = q.P[base + 1], r = hi - lo;
        u64 c = 0;
        if (walk_r_with_bitmap(ws, dl, r, s)) {
            const u32* bm = slot_bm(ws, dl);
            for (u32 e0 = lo; e0 < hi; e0 += 32) {
                // a stopped query's hub-row walk ends early and counts
                // nothing (its count is final or partial anyway)
                if (((e0 - lo) & 8191u) == 8160u && warp_ld_volatile_u32(&q.stop)) return 0;
                const u32 e = e0 + lane;
                const bool ok = e < hi && bm_test(bm, __ldg(q.adj + e));
                c += __popc(__ballot_sync(FULL_MASK, ok));
            }
        } else {
            const u32* S = cache_list(q, ws, dl);
            if (IS != ISECT_BINARY && warp_merge_pays(IS, min(r, s), max(r, s))) {
                bool st = false;
                c = warp_merge_count<true, false>(q.adj + lo, r, S, s, &q.stop, &st,
                                                  [](u32, u32) { return true; });
            } else if (r <= s) {
                for (u32 e0 = lo; e0 < hi; e0 += 32) {
                    const u32 e = e0 + lane;
                    const bool ok = e < hi && contains_rw(S, 0, s, __ldg(q.adj + e));
                    c += __popc(__ballot_sync(FULL_MASK, ok));
                }
            } else {
                for (u32 i0 = 0; i0 < s; i0 += 32) {
                    const u32 i = i0 + lane;
                    const bool ok = i < s && contains_u32(q.adj, lo, hi, S[i]);
                    c += __popc(__ballot_sync(FULL_MASK, ok));
                }
            }
        }
        return c - cached_exclusions(q, dl, v, ws, true, lo, hi);
    }
    // the shortest row drives; the second shortest is its merge partner
    u32 blo = 0, bhi = 0, blen = 0xFFFFFFFFu, bk = 0;
    u32 b2lo = 0, b2len = 0xFFFFFFFFu, bk2 = 0xFFFFFFFFu;
    for (u32 k = 0; k < nb; ++k) {
        const u32 bd = q.bn_depth[dl][k];
        const u32 base = q.bn_tab[dl][k] + (bd == dp ? p : ws->pos[bd]);
        const u32 lo = q.P[base], hi = q.P[base + 1];
        if (hi - lo < blen) {
            b2len = blen, b2lo = blo, bk2 = blen == 0xFFFFFFFFu ? 0xFFFFFFFFu : bk;
            blen = hi - lo, blo = lo, bhi = hi, bk = k;
        } else if (hi - lo < b2len) {
            b2len = hi - lo, b2lo = lo, bk2 = k;
        }
    }
    const u32 u = q.order[dl];
    const u32 same = q.same_mask[dl];
    const u32* list = q.list[u];
    if (IS != ISECT_BINARY && bk2 != 0xFFFFFFFFu && warp_merge_pays(IS, blen, b2len)) {
        // merge path over the two shortest rows; each common entry is then
        // tested against the other rows and the used same-label vertices
        const u32* A = q.adj + blo;
        bool st = false;
        return warp_merge_count<true, true>(A, blen, q.adj + b2lo, b2len, &q.stop, &st, [&](u32 i, u32) {
            const u32 x = __ldg(A + i);
            for (u32 k = 0; k < nb; ++k) {
                if (k == bk || k == bk2) continue;
                const u32 bd = q.bn_depth[dl][k];
                const u32 base = q.bn_tab[dl][k] + (bd == dp ? p : ws->pos[bd]);
                if (!contains_u32(q.adj, q.P[base], q.P[base + 1], x)) return false;
            }
            if (same) {
                const u32 vx = __ldg(list + x);
                for (u32 m = same; m; m &= m - 1) {
                    const u32 j = __ffs(m) - 1;
                    if (vx == (j == dp ? v : ws->vid[j])) return false;
                }
            }
            return true;
        });
    }
    u64 c = 0;
    for (u32 e0 = blo; e0 < bhi; e0 += 32) {
        const u32 e = e0 + lane;
        bool ok = e < bhi;
        const u32 x = ok ? __ldg(q.adj + e) : 0u;
        for (u32 k = 0; k < nb && ok; ++k) {
            if (k == bk) continue;
            const u32 bd = q.bn_depth[dl][k];
            const u32 base = q.bn_tab[dl][k] + (bd == dp ? p : ws->pos[bd]);
            ok = contains_u32(q.adj, q.P[base], q.P[base + 1], x);
        }
        if (ok && same) {
            const u32 vx = __ldg(list + x);
            u32 m = same;
            while (m && ok) {
                const u32 j = __ffs(m) - 1;
                m &= m - 1;
                ok = vx != (j == dp ? v : ws->vid[j]);
            }
        }
        c += __popc(__ballot_sync(FULL_MASK, ok));
    }
    return c;
}

// Completions of every candidate of depth d (= n-2, whose candidate set is
// its cache S_d, a whole level) at depth l = d + 1 given the prefix, through
// the weight memo (QState::memo_ok):
//   sum over p in S_d \ U, x in S_l \ V of [x in R(p)]
//     = sum_{x in S_l \ V} w(x) - sum_{u in U ∩ S_d} |R(u) ∩ S_l \ V|,
// with w(x) = |T[u_l -> u_d][x] ∩ S_d| (memoised), R(p) = T[u_d -> u_l][p],
// U / V the data vertices used by earlier same-label depths of u_d / u_l
// (p's own vertex is never in R(p): no self loops). Warp-uniform. Adds the
// reference-equivalent bytes of the level's last-depth intersections.
struct MemoOut {
    u64 count, bytes, calls;
};

__device__ __forceinline__ MemoOut memo_count(const QState& q, u32 d, WarpStack* ws) {
    const u32 lane = lane_id();
    const u32 l = d + 1;
    const u32 ud = q.order[d], ul = q.order[l];
    const u32* Sd = cache_list(q, ws, d);
    const u32 sd = ws->clen[d];
    const u32* bmd = slot_bm(ws, d);
    const u32* Sl = cache_list(q, ws, l);
    const u32 sl = ws->clen[l];
    const u32* list_l = q.list[ul];
    const u32 rbase = q.bn_tab[l][q.crow[l]];  // rows R(p) of T[u_d -> u_l]
    const u32 umask = q.same_mask[d];
    const u32 vmask = q.same_mask[l] & ~(1u << d);
    u32* memo = ws->memo;
    auto in_v = [&](u32 y) {
        if (!vmask) return false;
        const u32 vy = list_l[y];
        for (u32 m = vmask; m; m &= m - 1)
            if (ws->vid[__ffs(m) - 1] == vy) return true;
        return false;
    };
    // sum of w(x) over S_l \ V
    u64 a = 0;
    bool cut = false;
    for (u32 i = lane; i < sl; i += 32) {
        const u32 x = Sl[i];
        if (in_v(x)) continue;
        u32 e = memo[x];
        if (e == 0) {
            const u32 lo = q.P[q.memo_tab + x], hi = q.P[q.memo_tab + x + 1];
            u32 w = 0;
            for (u32 k = lo; k < hi; ++k) {
                // a stopped query ends long row walks early (per lane: no
                // warp-wide primitive inside this divergent loop)
                if (((k - lo) & 2047u) == 2047u && ld_volatile_u32(&q.stop)) {
                    cut = true;
                    break;
                }
                w += bm_test(bmd, __ldg(q.adj + k));
            }
            if (cut) break;
            e = w + 1;
            memo[x] = e;
        }
        a += e - 1;
    }
    // used same-label vertices among S_d: their completions and their rows
    u64 b = 0, ru = 0, nu = 0;
    if ((umask >> lane) & 1u) {
        const u32 pu = cand_pos(q, ud, ws->vid[lane]);
        if (pu != 0xFFFFFFFFu && bm_test(bmd, pu)) {
            const u32 lo = q.P[rbase + pu], hi = q.P[rbase + pu + 1];
            for (u32 k = lo; k < hi; ++k) {
                const u32 y = __ldg(q.adj + k);
                b += in_cache(q, ws, l, y) && !in_v(y);
            }
            ru = hi - lo;
            nu = 1;
        }
    }
    // reference-equivalent bytes: each accepted p of depth d intersects all
    // of depth l's rows
    if (!ws->rsum_ok) {
        u64 rs = 0;
        for (u32 i = lane; i < sd; i += 32) {
            const u32 p = Sd[i];
            rs += q.P[rbase + p + 1] - q.P[rbase + p];
        }
        rs = warp_sum64(rs);
        __syncwarp();
        if (lane == 0) {
            ws->rsum = rs;
            ws->rsum_ok = 1;
        }
        __syncwarp();
    }
    a = warp_sum64(a);
    b = warp_sum64(b);
    ru = warp_sum64(ru);
    nu = warp_sum64(nu);
    const u64 accepted = sd - nu;
    // a level cut short by the stop counts nothing
    if (__any_sync(FULL_MASK, cut)) return MemoOut{0, 0, 0};
    return MemoOut{a - b, accepted * (8ull * q.nbn[l] + 4ull * ws->csum[l]) + 4ull * (ws->rsum - ru), accepted};
}

// ---------------------------------------------------------------- queue --

// Bounded lock-free MPMC ring with a sequence number per slot. Lane 0 claims
// a slot; the warp copies the task words. A failed claim backs off and gives
// up after a few tries (the caller keeps the work).
__device__ bool enqueue(EnumCtl* ctl, Slot* slots, const TaskHdr& h, const WarpStack* ws, u32 npos, u32 extra_at,
                        u32 extra_val) {
    const u32 lane = lane_id();
    u32 slot_idx = 0;
    int ok = 0;
    if (lane == 0) {
        u32 pos = ld_volatile_u32(&ctl->q_tail);
        for (int it = 0; it < 8; ++it) {
            Slot* s = slots + (pos % QCAP);
            u32 seq = ld_acquire_u32(&s->seq);
            int diff = (int)(seq - pos);
            if (diff == 0) {
                u32 prev = atomicCAS(&ctl->q_tail, pos, pos + 1);
                if (prev == pos) {
                    ok = 1;
                    slot_idx = pos;
                    break;
                }
                pos = prev;
            } else if (diff < 0) {
                break;  // full
            } else {
                pos = ld_volatile_u32(&ctl->q_tail);
            }
        }
    }
    ok = __shfl_sync(FULL_MASK, ok, 0);
    if (!ok) return false;
    slot_idx = __shfl_sync(FULL_MASK, slot_idx, 0);
    Slot* s = slots + (slot_idx % QCAP);
    if (lane < HDR_WORDS) {
        const u32 hv[HDR_WORDS] = {h.kind, h.qi, h.d0, h.b, h.e, h.drv};
        u32 val = 0;
#pragma unroll
        for (u32 i = 0; i < HDR_WORDS; ++i)
            if (lane == i) val = hv[i];
        s->w[lane] = val;
    }
    s->w[HDR_WORDS + lane] = lane == extra_at ? extra_val : (lane < npos ? ws->pos[lane] : 0u);
    __threadfence();
    __syncwarp();
    if (lane == 0) st_release_u32(&s->seq, slot_idx + 1);
    return true;
}

// Takes a task; its prefix positions go straight into ws->pos.
__device__ bool dequeue(EnumCtl* ctl, Slot* slots, TaskHdr& h, WarpStack* ws) {
    const u32 lane = lane_id();
    u32 slot_idx = 0;
    int ok = 0;
    if (lane == 0) {
        u32 pos = ld_volatile_u32(&ctl->q_head);
        for (int it = 0; it < 4; ++it) {
            Slot* s = slots + (pos % QCAP);
            u32 seq = ld_acquire_u32(&s->seq);
            int diff = (int)(seq - (pos + 1));
            if (diff == 0) {
                u32 prev = atomicCAS(&ctl->q_head, pos, pos + 1);
                if (prev == pos) {
                    ok = 1;
                    slot_idx = pos;
                    break;
                }
                pos = prev;
                __nanosleep(32u << it);
            } else if (diff < 0) {
                break;  // empty
            } else {
                pos = ld_volatile_u32(&ctl->q_head);
            }
        }
    }
    ok = __shfl_sync(FULL_MASK, ok, 0);
    if (!ok) return false;
    slot_idx = __shfl_sync(FULL_MASK, slot_idx, 0);
    Slot* s = slots + (slot_idx % QCAP);
    __threadfence();
    u32 hw = lane < HDR_WORDS ? ld_volatile_u32(&s->w[lane]) : 0u;
    h.kind = __shfl_sync(FULL_MASK, hw, 0);
    h.qi = __shfl_sync(FULL_MASK, hw, 1);
    h.d0 = __shfl_sync(FULL_MASK, hw, 2);
    h.b = __shfl_sync(FULL_MASK, hw, 3);
    h.e = __shfl_sync(FULL_MASK, hw, 4);
    h.drv = __shfl_sync(FULL_MASK, hw, 5);
    ws->pos[lane] = ld_volatile_u32(&s->w[HDR_WORDS + lane]);
    __threadfence();
    __syncwarp();
    if (lane == 0) st_release_u32(&s->seq, slot_idx + QCAP);
    return true;
}

// Hands the upper half of a range to the queue when more warps are hungry
// than tasks are queued. Returns true if it donated (the range end moved).
__device__ bool try_donate_range(EnumCtl* ctl, Slot* slots, u32 kind, u32 qi, u32 d0, u32 cur, u32& end, u32 drv,
                                 const WarpStack* ws, u32 min_len) {
    if (end - cur < min_len) return false;
    const u32 hungry = warp_ld_volatile_u32(&ctl->hungry);
    if (hungry == 0) return false;
    const u32 qlen = warp_ld_volatile_u32(&ctl->q_tail) - warp_ld_volatile_u32(&ctl->q_head);
    if (qlen >= hungry) return false;
    const u32 lane = lane_id();
    const u32 mid = cur + ((end - cur) >> 1);
    TaskHdr h{kind, qi, d0, mid, end, drv};
    if (lane == 0) {
        atomicAdd(&ctl->pending, 1ull);
        atomicAdd(&ctl->remaining[qi], 1u);
    }
    __threadfence();
    __syncwarp();
    if (enqueue(ctl, slots, h, ws, d0, 0xFFFFFFFFu, 0)) {
        if (lane == 0) atomicAdd((unsigned long long*)&ctl->donations, 1ull);
        end = mid;
        return true;
    }
    if (lane == 0) {
        atomicSub(&ctl->remaining[qi], 1u);  // the donor's own task still holds the query open
        atomicAdd(&ctl->pending, (unsigned long long)-1ll);
    }
    return false;
}

// Every 16 warp steps inside a search: donate work to hungry warps, publish
// the local count (so a capped query stops close to its cap) and stop on the
// cap or the time limit. Returns true when the search must stop.
__device__ bool periodic(QState& q, u32 qi, WarpStack* ws, u32 d, u32 d0, u32 iter, u64& count, EnumCtl* ctl,
                         Slot* slots) {
    const u32 lane = lane_id();
    if (warp_ld_volatile_u32(&ctl->hungry) > 0) {
        // (a) upper half of the shallowest driver range with >= 64 unexplored
        // elements, else (b) the last unexplored chunk entry of the
        // shallowest depth below d, as a task one level deeper.
        u32 dd = d0;
        for (; dd <= d; ++dd)
            if (ws->end[dd] - ws->cur[dd] >= 64u) break;
        if (dd <= d) {
            u32 end = ws->end[dd];
            // drv word: bn index of the driver | level flags << 16
            bool done = try_donate_range(ctl, slots, KIND_RANGE, qi, dd, ws->cur[dd], end,
                                         ws->drv[dd] | (ws->flg[dd] << 16), ws, 64u);
            __syncwarp();
            if (done && lane == 0) {
                ws->end[dd] = end;
                ws->lvfull &= ~(1u << dd);
            }
            __syncwarp();
        } else {
            u32 de = d0;
            for (; de < d; ++de)
                if (ws->cn[de] > ws->ci[de]) break;
            const u32 hungry = warp_ld_volatile_u32(&ctl->hungry);
            const u32 qlen = warp_ld_volatile_u32(&ctl->q_tail) - warp_ld_volatile_u32(&ctl->q_head);
            if (de < d && qlen < hungry) {
                TaskHdr h{KIND_FULL, qi, de + 1, 0, 0, 0};
                if (lane == 0) {
                    atomicAdd(&ctl->pending, 1ull);
                    atomicAdd(&ctl->remaining[qi], 1u);
                }
                __threadfence();
                __syncwarp();
                if (enqueue(ctl, slots, h, ws, de, de, ws->chunk[de][ws->cn[de] - 1])) {
                    __syncwarp();
                    if (lane == 0) {
                        ws->cn[de] -= 1;
                        atomicAdd((unsigned long long*)&ctl->donations, 1ull);
                    }
                } else if (lane == 0) {
                    atomicSub(&ctl->remaining[qi], 1u);
                    atomicAdd(&ctl->pending, (unsigned long long)-1ll);
                }
                __syncwarp();
            }
        }
    }
    // Far from the cap a warp publishes every 16 K embeddings. Once its own
    // publish shows the query within reach of the cap (every warp's
    // unpublished share, twice over, could cross it), it publishes every 1 K:
    // the query then stops close to the cap instead of up to a share per warp
    // beyond it. Only lane 0 reads and writes near_q.
    if (lane == 0 && count >= (ws->near_q == qi ? (1ull << 10) : (1ull << 14))) {
        unsigned long long old = atomicAdd((unsigned long long*)&q.count, count);
        if (q.cap) {
            const u64 total = old + count;
            if (total >= q.cap) cap_reached(q);
            if (total + ((u64)(gridDim.x * (blockDim.x >> 5)) << 17) >= q.cap) ws->near_q = qi;
        }
        count = 0;
    }
    count = __shfl_sync(FULL_MASK, count, 0);
    // Emission keeps q.emit_rows current (one atomic per chunk), so a capped
    // emitting query stops on it instead of on the lagging published count:
    // the rows emitted past the cap stay few and fit the caller's buffer.
    if (lane == 0 && q.emit_buf && q.cap &&
        *(volatile unsigned long long*)&q.emit_rows >= (unsigned long long)q.cap)
        cap_reached(q);
    u32 stop = warp_ld_volatile_u32(&q.stop);
    if (!stop && (iter & 255u) == 0 && global_timer_ns() > ctl->deadline_ns) {
        if (lane == 0) {
            atomicExch(&q.overtime, 1u);
            atomicExch(&q.stop, 1u);
        }
        stop = 1;
    }
    return __shfl_sync(FULL_MASK, stop, 0) != 0;
}

// Depth-first search below the prefix ws->pos[0, d0): the level d0 has been
// set up (driver range in ws). Returns false if the query stopped.
template <u32 IS>
__device__ bool dfs(const DevGraph& g, QState& q, u32 qi, u32 d0, WarpStack* ws, EnumCtl* ctl, Slot* slots, bool emit,
                    u64& count, u64& bytes, u64& calls, u32& iter) {
    const u32 lane = lane_id();
    const u32 n = q.n_enum;
    u32 d = d0;
    u64 bytes_l = 0, calls_l = 0;  // per-lane parts, summed at the end
    bool go = true;
    while (true) {
        if (d + 2 == n && !emit) {
            // The last two depths fused: each lane takes one driver element
            // of depth d and counts its completions at depth d + 1 on its own.
            if (ws->cur[d] < ws->end[d] && q.memo_ok && ((ws->lvfull >> d) & 1u) &&
                (ws->flg[d] & LV_CACHED) && ((ws->cbits >> d) & 1u) && ensure_cache<IS>(q, d + 1, ws, bytes)) {
                // the whole level at once through the weight memo
                const MemoOut mo = memo_count(q, d, ws);
                count += mo.count;
                bytes += mo.bytes;
                calls += mo.calls;
                __syncwarp();
                if (lane == 0) ws->cur[d] = ws->end[d];
                __syncwarp();
                if ((++iter & 15u) == 0 && periodic(q, qi, ws, d, d0, iter, count, ctl, slots)) {
                    go = false;
                    break;
                }
                continue;
            }
            if (ws->cur[d] < ws->end[d]) {
                const u32 cur = ws->cur[d], end = ws->end[d];
                const u32 idx = cur + lane;
                u64 c = 0;
                bool defer = false;
                const u32* list_d = q.list[q.order[d]];
                // the last depth's cache depends on depths <= d - 1 only
                const bool cached = ensure_cache<IS>(q, d + 1, ws, bytes);
                const bool valid = idx < end;
                const u32 p = valid ? (d == 0 ? idx : drv_elem(q, ws, d, idx)) : 0u;
                const bool ok = d == 0 ? valid : chunk_accept(q, d, p, valid, ws, list_d);
                const u32 v = ok ? list_d[p] : 0u;
                const u32 act = __popc(__ballot_sync(FULL_MASK, ok));
                if (ok) c = lane_last_count<IS>(q, d + 1, cached, p, v, ws, bytes_l, calls_l, &defer, act);
                count += warp_sum64(c);
                // long intersections deferred by their lanes: whole warp each
                u32 dm = __ballot_sync(FULL_MASK, defer);
                while (dm) {
                    const u32 src = __ffs(dm) - 1;
                    dm &= dm - 1;
                    count += warp_last_count<IS>(q, d + 1, cached, __shfl_sync(FULL_MASK, p, src),
                                             __shfl_sync(FULL_MASK, v, src), ws);
                }
                calls += min(32u, end - cur);
                __syncwarp();
                if (lane == 0) ws->cur[d] = min(end, cur + 32u);
                __syncwarp();
                if ((++iter & 15u) == 0 && periodic(q, qi, ws, d, d0, iter, count, ctl, slots)) {
                    go = false;
                    break;
                }
            } else {
                if (d == d0) break;
                d -= 1;
            }
            continue;
        }
        if (ws->ci[d] < ws->cn[d]) {
            const u32 p = ws->chunk[d][ws->ci[d]];
            __syncwarp();
            if (lane == 0) {
                ws->ci[d] += 1;
                ws->pos[d] = p;
                ws->vid[d] = q.list[q.order[d]][p];
                const u32 inv = q.cinval[d];  // caches that depend on depth d
                ws->cvalid &= ~inv;
                ws->cover &= ~inv;
            }
            __syncwarp();
            if (d + 2 == n) {
                count += emit ? emit_last<IS>(q, g, d + 1, ws, bytes, calls) : count_last<IS>(q, d + 1, ws, bytes, calls);
            } else {
                d += 1;
                setup_level<IS>(q, d, ws, bytes);
            }
        } else if (ws->cur[d] < ws->end[d]) {
            const u32 cur = ws->cur[d], end = ws->end[d];
            const u32 idx = cur + lane;
            const bool valid = idx < end;
            const u32 p = valid ? (d == 0 ? idx : drv_elem(q, ws, d, idx)) : 0u;
            const bool ok = d == 0 ? valid : chunk_accept(q, d, p, valid, ws, q.list[q.order[d]]);
            u32 bal = __ballot_sync(FULL_MASK, ok);
            if (ok) ws->chunk[d][__popc(bal & ((1u << lane) - 1u))] = p;
            calls += min(32u, end - cur);
            __syncwarp();
            if (lane == 0) {
                ws->cn[d] = __popc(bal);
                ws->ci[d] = 0;
                ws->cur[d] = min(end, cur + 32u);
            }
            __syncwarp();
            if ((++iter & 15u) == 0 && periodic(q, qi, ws, d, d0, iter, count, ctl, slots)) {
                go = false;
                break;
            }
        } else {
            if (d == d0) break;
            d -= 1;
        }
    }
    bytes += warp_sum64(bytes_l);
    calls += warp_sum64(calls_l);
    return go;
}

__device__ void publish(QState& q, u64 count, u64 bytes, u64 calls) {
    if (lane_id() == 0) {
        if (count) {
            unsigned long long old = atomicAdd((unsigned long long*)&q.count, count);
            if (q.cap && old + count >= q.cap) cap_reached(q);
        }
        if (calls) atomicAdd((unsigned long long*)&q.calls, calls);
        if (bytes) atomicAdd((unsigned long long*)&q.alg_bytes, bytes);
    }
}

// Runs one task (prefix positions already in ws->pos[0, d0)).
template <u32 IS>
__device__ void run_task(const DevGraph& g, QState* qs, const TaskHdr& t, WarpStack* ws, EnumCtl* ctl, Slot* slots,
                         bool emit) {
    const u32 lane = lane_id();
    QState& q = qs[t.qi];
    const u32 n = q.n_enum;
    if (warp_ld_volatile_u32(&q.stop)) return;
    u64 count = 0, bytes = 0, calls = 0;
    u32 iter = 0;
    // caches start empty (release_caches ran at the end of the last task)
    if (n == 1) {  // single-vertex query: every root candidate is an embedding
        count = t.e - t.b;
        calls = count;
        if (emit) {
            for (u32 i = t.b + lane; i < t.e; i += 32) {
                unsigned long long r = atomicAdd((unsigned long long*)&q.emit_rows, 1ull);
                const u32 v = q.list[q.order[0]][i];
                if (r < q.emit_cap_rows) q.emit_buf[r] = q.emit_by_depth ? v : g.orig[v];
            }
        }
        publish(q, count, bytes, calls);
        return;
    }
    if (t.kind == KIND_EDGES) {
        // Pairs (root r, depth-1 candidate c) taken from the entries [b, e)
        // of the first table T[u_0][u_1]; the root of an entry is found by
        // walking the table's row offsets.
        const u32 base = q.bn_tab[1][0];
        const u32* list0 = q.list[q.order[0]];
        const u32* list1 = q.list[q.order[1]];
        const bool same01 = q.same_mask[1] & 1u;
        u32 lo = 0, hi = q.root_cnt;  // largest r with P[base + r] <= b
        while (hi - lo > 1) {
            u32 mid = (lo + hi) >> 1;
            if (q.P[base + mid] <= t.b)
                lo = mid;
            else
                hi = mid;
        }
        u32 r = lo, last_r = 0xFFFFFFFFu;
        u32 end = t.e;
        for (u32 e = t.b; e < end; ++e) {
            while (q.P[base + r + 1] <= e) ++r;
            const u32 c = q.adj[e];
            const u32 v0 = list0[r], v1 = list1[c];
            calls += 1;
            if (same01 && v0 == v1) continue;
            __syncwarp();
            if (lane == 0) {
                ws->pos[0] = r;
                ws->vid[0] = v0;
                ws->pos[1] = c;
                ws->vid[1] = v1;
                const u32 inv = q.cinval[r == last_r ? 1 : 0];
                ws->cvalid &= ~inv;
                ws->cover &= ~inv;
            }
            last_r = r;
            __syncwarp();
            // edge pools are built for queries of four or more vertices
            setup_level<IS>(q, 2, ws, bytes);
            if (!dfs<IS>(g, q, t.qi, 2, ws, ctl, slots, emit, count, bytes, calls, iter)) break;
            if (e + 2 < end) try_donate_range(ctl, slots, KIND_EDGES, t.qi, 0, e + 1, end, 0, ws, 2u);
        }
        release_caches(q, ws);
        publish(q, count, bytes, calls);
        return;
    }
    // Restore the data vertices of the prefix.
    if (lane < t.d0) ws->vid[lane] = q.list[q.order[lane]][ws->pos[lane]];
    __syncwarp();
    const u32 d0 = t.d0;
    if (t.kind == KIND_FULL && d0 + 1 == n) {
        // donated entry whose children are the last depth
        count += emit ? emit_last<IS>(q, g, d0, ws, bytes, calls) : count_last<IS>(q, d0, ws, bytes, calls);
    } else {
        if (t.kind == KIND_FULL) {
            setup_level<IS>(q, d0, ws, bytes);
        } else {
            // a donated driver range: rebuild the level the donor had (its
            // cache is a function of the prefix, so the range indexes the
            // same array here)
            const u32 flg = t.drv >> 16, k = t.drv & 0xFFFFu;
            u32 olo = 0, ohi = 0;
            if (flg & LV_CACHED) {
                // the donor's flags need what the donor had: the cache, and
                // its bitmap when S is tested through it
                if (!ensure_cache<IS>(q, d0, ws, bytes) || ((flg & LV_OTHER_BM) && !((ws->cbits >> d0) & 1u))) {
                    if (lane == 0) atomicExch(&ctl->error, 1u);
                    release_caches(q, ws);
                    publish(q, count, bytes, calls);
                    return;
                }
                if ((flg & LV_OTHER) && !(flg & LV_OTHER_BM)) {
                    if (flg & LV_DRV_CACHE) {
                        olo = row_lo(q, d0, q.crow[d0], ws->pos);
                        ohi = row_hi(q, d0, q.crow[d0], ws->pos);
                    } else {
                        ohi = ws->clen[d0];
                    }
                }
            }
            __syncwarp();
            if (lane == 0) {
                ws->lvfull &= ~(1u << d0);  // a part of the donor's level
                ws->flg[d0] = flg;
                ws->cur[d0] = t.b;
                ws->end[d0] = t.e;
                ws->drv[d0] = k;
                ws->olo[d0] = olo;
                ws->ohi[d0] = ohi;
                ws->cn[d0] = 0;
                ws->ci[d0] = 0;
            }
            __syncwarp();
        }
        dfs<IS>(g, q, t.qi, d0, ws, ctl, slots, emit, count, bytes, calls, iter);
    }
    release_caches(q, ws);
    publish(q, count, bytes, calls);
}

// Initial pool: ticket -> (query, unit range); grab_prefix[i] = grabs of the
// queries before i.
__device__ bool take_initial(EnumCtl* ctl, const u32* grab_prefix, const PoolInfo* pools, QState* qs, TaskHdr& t) {
    const u32 lane = lane_id();
    // Once the ticket passes the end it never comes back; skipping the
    // pending increment then keeps idle warps from holding `pending` above
    // zero with transient increments.
    if (warp_ld_volatile_u32(&ctl->ticket) >= ctl->total_grabs) return false;
    u32 r = 0, crossing = 0;
    if (lane == 0) {
        atomicAdd(&ctl->pending, 1ull);
        __threadfence();
        r = atomicAdd(&ctl->ticket, 1u);
        if (r >= ctl->total_grabs) {
            atomicAdd(&ctl->pending, (unsigned long long)-1ll);
        } else if (r + 1 == ctl->total_grabs) {
            crossing = 1;  // this grab exhausts the pool: release the pool's token
        }
    }
    r = __shfl_sync(FULL_MASK, r, 0);
    crossing = __shfl_sync(FULL_MASK, crossing, 0);
    if (r >= ctl->total_grabs) return false;
    if (crossing && lane == 0) {
        __threadfence();
        atomicAdd(&ctl->pending, (unsigned long long)-1ll);
    }
    u32 lo = 0, hi = ctl->nq;  // query owning grab r
    while (hi - lo > 1) {
        u32 mid = (lo + hi) >> 1;
        if (grab_prefix[mid] <= r)
            lo = mid;
        else
            hi = mid;
    }
    // A stopped query (cap reached, time limit) would still hand out every
    // grab left in its pool, one ticket and three counter updates each, and
    // the launch ends only after the last of them: the warp that meets a
    // stopped query claims the rest of its grabs in one step instead. The
    // claimed grabs never run, so they leave the query's remaining count;
    // its own grab r still holds the query open, and whoever claims the
    // pool's last grab releases the pool's token.
    if (warp_ld_volatile_u32(&qs[lo].stop)) {
        if (lane == 0) {
            const u32 end = grab_prefix[lo + 1];
            u32 cur = ld_volatile_u32(&ctl->ticket);
            while (cur < end) {
                const u32 prev = atomicCAS(&ctl->ticket, cur, end);
                if (prev == cur) {
                    atomicSub(&ctl->remaining[lo], end - cur);
                    if (end == ctl->total_grabs) {
                        __threadfence();
                        atomicAdd(&ctl->pending, (unsigned long long)-1ll);
                    }
                    break;
                }
                cur = prev;
            }
        }
        __syncwarp();
    }
    const PoolInfo& pi = pools[lo];
    const u32 j = r - grab_prefix[lo];
    const u32 ub = j * pi.grab, ue = min(pi.units, ub + pi.grab);
    t.kind = pi.kind;
    t.qi = lo;
    t.d0 = 0;
    t.b = pi.first + ub;
    t.e = pi.first + ue;
    t.drv = 0;
    return true;
}

template <u32 IS>
__global__ void __launch_bounds__(WARPS_PER_BLOCK * 32, 3) enum_kernel(DevGraph g, QState* qs, EnumCtl* ctl,
                                                                    Slot* slots, const u32* grab_prefix,
                                                                    const PoolInfo* pools, int emit, u32* cache) {
    __shared__ WarpStack stacks[WARPS_PER_BLOCK];
    WarpStack* ws = &stacks[threadIdx.x >> 5];
    const u32 lane = lane_id();
    if (lane == 0) {
        const size_t warp = (size_t)blockIdx.x * WARPS_PER_BLOCK + (threadIdx.x >> 5);
        ws->cbuf = cache ? cache + warp * WARP_CACHE_WORDS : nullptr;
        ws->memo = cache ? ws->cbuf + PSM_MAXQ * SLOT_WORDS : nullptr;
        ws->rsum_ok = 0;
        ws->lvfull = 0;
        ws->cvalid = 0;
        ws->cover = 0;
        ws->cbits = 0;
        ws->cadj = 0;
        ws->near_q = 0xFFFFFFFFu;
    }
    __syncwarp();
    TaskHdr t;
    bool hungry = false;
    u64 spins = 0, ntasks = 0, npolls = 0;
    while (true) {
        bool got = take_initial(ctl, grab_prefix, pools, qs, t);
        if (!got) got = dequeue(ctl, slots, t, ws);
        if (got) {
            if (hungry && lane == 0) atomicSub(&ctl->hungry, 1u);
            hungry = false;
            spins = 0;
            run_task<IS>(g, qs, t, ws, ctl, slots, emit != 0);
            ++ntasks;
            __syncwarp();
            if (lane == 0) {
                __threadfence();
                // the query's last task publishes its result
                if (atomicSub(&ctl->remaining[t.qi], 1u) == 1u && ctl->done) finish_query(qs[t.qi], ctl->done + t.qi);
                atomicAdd(&ctl->pending, (unsigned long long)-1ll);
            }
            continue;
        }
        if (!hungry && lane == 0) atomicAdd(&ctl->hungry, 1u);
        hungry = true;
        unsigned long long pend = 0;
        if (lane == 0) pend = ld_acquire_u64((const u64*)&ctl->pending);
        pend = __shfl_sync(FULL_MASK, pend, 0);
        if (pend == 0) break;
        if (ctl->exit_keep && warp_ld_volatile_u32(&ctl->ticket) >= ctl->total_grabs &&
            warp_ld_volatile_u32(&ctl->q_tail) == warp_ld_volatile_u32(&ctl->q_head)) {
            // nothing to take: leave (freeing the SM for other launches)
            // while more than exit_keep warps stay to take donations
            u32 leave = 0;
            if (lane == 0) {
                const u32 old = atomicSub(&ctl->hungry, 1u);
                if (old > ctl->exit_keep)
                    leave = 1;
                else
                    atomicAdd(&ctl->hungry, 1u);
            }
            if (__shfl_sync(FULL_MASK, leave, 0)) break;
        }
        ++spins;
        ++npolls;
        if ((spins & 255u) == 0) {
            u32 bail = 0;
            if (lane == 0 && (global_timer_ns() > ctl->deadline_ns + 2000000000ull || spins > (1ull << 32))) {
                atomicExch(&ctl->error, 1u);
                bail = 1;
            }
            if (__shfl_sync(FULL_MASK, bail, 0)) break;
        }
        __nanosleep(256);
    }
    if (lane == 0) {
        atomicAdd((unsigned long long*)&ctl->tasks, (unsigned long long)ntasks);
        atomicAdd((unsigned long long*)&ctl->idle_polls, (unsigned long long)npolls);
    }
}

// Single block: per-query initial pools (edges of the first table for
// queries of four or more vertices, roots otherwise), their prefix in grabs,
// the per-query task counts and the queue's sequence numbers.
__global__ void enum_init_kernel(QState* qs, u32 nq, EnumCtl* ctl, Slot* slots, u32* grab_prefix, PoolInfo* pools,
                                 u32* remaining, QDoneRec* done, u32 exit_keep, u32 total_warps, u64 budget_ns,
                                 u32 grabs_per_warp) {
    __shared__ u32 s_carry;
    __shared__ u32 wt[32];
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (u32 base = 0; base < nq; base += blockDim.x) {
        const u32 i = base + threadIdx.x;
        u32 grabs = 0;
        if (i < nq) {
            const QState& q = qs[i];
            PoolInfo pi{KIND_RANGE, 0, 1, 0};
            if (q.status == PSM_DEV_OK && !q.stop && q.root_cnt > 0) {
                const u32 n = q.n_enum;
                if (n >= 4) {
                    const u32 tb = q.bn_tab[1][0];
                    pi.kind = KIND_EDGES;
                    pi.first = q.P[tb];
                    pi.units = q.P[tb + q.root_cnt] - pi.first;
                    // depth 1 reads the first table's row of every root
                    atomicAdd((unsigned long long*)&qs[i].alg_bytes, 8ull * q.root_cnt + 4ull * pi.units);
                } else {
                    pi.kind = KIND_RANGE;
                    pi.first = 0;
                    pi.units = q.root_cnt;
                }
                // about grabs_per_warp grabs per warp for a lone query (8 by
                // default); never below one unit
                const u32 target = total_warps * grabs_per_warp;
                pi.grab = max(1u, pi.units / max(1u, target));
                grabs = (pi.units + pi.grab - 1) / pi.grab;
            }
            pools[i] = pi;
            remaining[i] = grabs;
            if (grabs == 0 && done) finish_query(qs[i], done + i);  // nothing to enumerate
        }
        u32 incl = warp_incl_scan(grabs);
        if (lane_id() == 31) wt[threadIdx.x >> 5] = incl;
        __syncthreads();
        if (threadIdx.x < 32) {
            u32 x = threadIdx.x < (blockDim.x >> 5) ? wt[threadIdx.x] : 0;
            u32 xi = warp_incl_scan(x);
            wt[threadIdx.x] = xi - x;
        }
        __syncthreads();
        const u32 excl = s_carry + wt[threadIdx.x >> 5] + incl - grabs;
        if (i < nq) grab_prefix[i] = excl;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) s_carry = excl + grabs;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        grab_prefix[nq] = s_carry;
        ctl->total_grabs = s_carry;
        ctl->ticket = 0;
        ctl->hungry = 0;
        ctl->q_head = 0;
        ctl->q_tail = 0;
        ctl->error = 0;
        ctl->nq = nq;
        ctl->pending = s_carry > 0 ? 1ull : 0ull;  // the initial pool's token
        ctl->deadline_ns = global_timer_ns() + budget_ns;
        ctl->donations = 0;
        ctl->tasks = 0;
        ctl->idle_polls = 0;
        ctl->remaining = remaining;
        ctl->done = done;
        ctl->exit_keep = exit_keep;
    }
    for (u32 i = threadIdx.x; i < QCAP; i += blockDim.x) slots[i].seq = i;
}

__global__ void gather_kernel(const QState* qs, u32 nq, DevResult* out) {
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += gridDim.x * blockDim.x) {
        const QState& q = qs[i];
        DevResult r;
        r.count = q.cap && q.count > q.cap ? q.cap : q.count;
        r.count_internal = q.count;
        r.calls = q.calls;
        r.alg_bytes = q.alg_bytes;
        r.memory_bytes = q.memory_bytes;
        r.table_nnz = q.table_nnz;
        r.emit_rows = q.emit_rows;
        r.status = q.status;
        r.overtime = q.overtime;
        r.filter_ok = q.filter_ok;
        r.empty = q.empty;
        out[i] = r;
    }
}

size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }

}  // namespace

cudaError_t psm_launch_gather(const QState* qs, u32 nq, DevResult* out, cudaStream_t st) {
    u32 blocks = (nq + 255) / 256;
    gather_kernel<<<blocks ? blocks : 1, 256, 0, st>>>(qs, nq, out);
    return cudaGetLastError();
}

size_t psm_enum_scratch_bytes() { return align16(sizeof(EnumCtl)) + sizeof(Slot) * QCAP + 64; }

// Per-warp prefix-intersection caches of a launch of `blocks` blocks.
size_t psm_enum_cache_bytes(int blocks) {
    return (size_t)blocks * WARPS_PER_BLOCK * WARP_CACHE_WORDS * sizeof(u32);
}

// Per-query scratch of the enumeration: grab prefix (nq + 1 words), pool
// descriptors and remaining-task counts.
size_t psm_enum_query_bytes(u32 nq) {
    return align16(sizeof(u32) * (nq + 1)) + align16(sizeof(PoolInfo) * nq) + sizeof(u32) * nq;
}

cudaError_t psm_launch_enum(const DevGraph& g, QState* qs, u32 nq, void* scratch, void* query_scratch, u64 budget_ns,
                            int emit, int blocks, u32* cache, QDoneRec* done, u32 exit_keep, cudaStream_t st,
                            u32 grabs_per_warp, u32 isect) {
    EnumCtl* ctl = (EnumCtl*)scratch;
    Slot* slots = (Slot*)((char*)scratch + align16(sizeof(EnumCtl)));
    u32* grab_prefix = (u32*)query_scratch;
    PoolInfo* pools = (PoolInfo*)((char*)query_scratch + align16(sizeof(u32) * (nq + 1)));
    u32* remaining = (u32*)((char*)pools + align16(sizeof(PoolInfo) * nq));
    enum_init_kernel<<<1, 1024, 0, st>>>(qs, nq, ctl, slots, grab_prefix, pools, remaining, done, exit_keep,
                                         (u32)blocks * WARPS_PER_BLOCK, budget_ns, max(1u, grabs_per_warp));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // one instantiation per intersection variant: the merge paths cost the
    // binary-search one nothing (registers, instruction cache)
    if (isect == ISECT_AUTO)
        enum_kernel<ISECT_AUTO><<<blocks, WARPS_PER_BLOCK * 32, 0, st>>>(g, qs, ctl, slots, grab_prefix, pools, emit,
                                                                        cache);
    else if (isect == ISECT_MERGE)
        enum_kernel<ISECT_MERGE><<<blocks, WARPS_PER_BLOCK * 32, 0, st>>>(g, qs, ctl, slots, grab_prefix, pools,
                                                                         emit, cache);
    else
        enum_kernel<ISECT_BINARY><<<blocks, WARPS_PER_BLOCK * 32, 0, st>>>(g, qs, ctl, slots, grab_prefix, pools,
                                                                          emit, cache);
    return cudaGetLastError();
}

cudaError_t psm_enum_max_blocks(int* blocks) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, enum_kernel<ISECT_BINARY>, WARPS_PER_BLOCK * 32, 0);
    if (e != cudaSuccess) return e;
    *blocks = sms * (per_sm < 1 ? 1 : per_sm);
    return cudaSuccess;
}

// Size of the launch-wide control block (error flag, scheduling counters).
size_t psm_enum_ctl_bytes() { return sizeof(EnumCtl); }

// Queues a copy of the control block into host memory (pinned staging).
cudaError_t psm_enum_copy_ctl(const void* scratch, void* host, cudaStream_t st) {
    return cudaMemcpyAsync(host, scratch, sizeof(EnumCtl), cudaMemcpyDeviceToHost, st);
}

// Decodes a control block copied by psm_enum_copy_ctl.
void psm_enum_ctl_stats(const void* host, EnumStats* out) {
    EnumCtl h;
    memcpy(&h, host, sizeof(h));
    out->error = h.error;
    out->donations = h.donations;
    out->tasks = h.tasks;
    out->idle_polls = h.idle_polls;
}

// Reads back the launch-wide error flag and scheduling counters.
cudaError_t psm_enum_read_ctl(void* scratch, EnumStats* out, cudaStream_t st) {
    EnumCtl h;
    cudaError_t e = cudaMemcpyAsync(&h, scratch, sizeof(EnumCtl), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    out->error = h.error;
    out->donations = h.donations;
    out->tasks = h.tasks;
    out->idle_polls = h.idle_polls;
    return cudaSuccess;
}
