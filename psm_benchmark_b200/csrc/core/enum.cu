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
//    ballot compacts the survivors. The last depth is only counted (row
//    length directly when a single row has no possible collision);
//  - work: root candidates of all queries of a launch are handed out by an
//    atomic ticket; an idle warp raises a "hungry" counter and busy warps
//    donate the upper half of the unexplored driver range at their
//    shallowest depth to a bounded lock-free queue (the reference's
//    "linear" split, TaskPool.cpp:1407-1424);
//  - termination: a pending-work counter (root pool + live tasks) reaches
//    zero. Every wait is bounded by a deadline and an iteration cap; on
//    expiry the kernel records an error and returns.
#include <cuda_runtime.h>

#include "device_util.cuh"
#include "psm_internal.h"

namespace {

constexpr u32 QCAP = 4096;          // steal queue slots
constexpr u32 TASK_WORDS = 5 + PSM_MAXQ;
constexpr u32 WARPS_PER_BLOCK = 8;
constexpr u32 FULL_LEVEL = 0xFFFFFFFFu;  // task range: the whole driver row of d0

struct Task {
    u32 qi, d0, b, e, drv;
    u32 pos[PSM_MAXQ];
};

struct Slot {
    u32 seq;
    u32 w[TASK_WORDS];
};

}  // namespace

struct EnumCtl {
    u32 root_ticket;
    u32 total_roots;
    u32 hungry;
    u32 q_head;
    u32 q_tail;
    u32 error;
    u32 nq;
    u32 pad;
    unsigned long long pending;
    u64 deadline_ns;
    u64 donations;
};

namespace {

struct WarpStack {
    u32 pos[PSM_MAXQ];
    u32 vid[PSM_MAXQ];
    u32 cur[PSM_MAXQ];
    u32 end[PSM_MAXQ];
    u32 drv[PSM_MAXQ];
    u32 cn[PSM_MAXQ];
    u32 ci[PSM_MAXQ];
    u32 chunk[PSM_MAXQ][32];
};

__device__ __forceinline__ u32 row_lo(const QState& q, u32 d, u32 k, const u32* pos) {
    return q.P[q.bn_tab[d][k] + pos[q.bn_depth[d][k]]];
}
__device__ __forceinline__ u32 row_hi(const QState& q, u32 d, u32 k, const u32* pos) {
    return q.P[q.bn_tab[d][k] + pos[q.bn_depth[d][k]] + 1];
}

// Picks the shortest backward-neighbour row at depth d; returns its length
// and range, and adds the algorithmic bytes of reading all rows.
__device__ __forceinline__ u32 setup_level(const QState& q, u32 d, WarpStack* ws, u64& bytes) {
    const u32 nb = q.nbn[d];
    u32 best = 0, blen = 0xFFFFFFFFu, bs = 0;
    u64 by = 0;
    for (u32 k = 0; k < nb; ++k) {
        u32 lo = row_lo(q, d, k, ws->pos), hi = row_hi(q, d, k, ws->pos);
        u32 len = hi - lo;
        by += 8u + 4ull * len;
        if (len < blen) blen = len, best = k, bs = lo;
    }
    bytes += by;
    if (lane_id() == 0) {
        ws->drv[d] = best;
        ws->cur[d] = bs;
        ws->end[d] = bs + blen;
        ws->cn[d] = 0;
        ws->ci[d] = 0;
    }
    __syncwarp();
    return blen;
}

// One lane's candidate test at depth d for driver element p (a position in
// C(u_d)): member of every other row and not a data vertex already used by a
// same-label earlier depth.
__device__ __forceinline__ bool accept(const QState& q, u32 d, u32 p, const WarpStack* ws, const u32* list_d) {
    const u32 nb = q.nbn[d], drv = ws->drv[d];
    for (u32 k = 0; k < nb; ++k) {
        if (k == drv) continue;
        u32 lo = row_lo(q, d, k, ws->pos), hi = row_hi(q, d, k, ws->pos);
        if (!contains_u32(q.adj, lo, hi, p)) return false;
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

// Counts the candidates of the last depth d given the prefix in ws.
__device__ u64 count_last(const QState& q, u32 d, WarpStack* ws, u64& bytes, u64& calls) {
    const u32 lane = lane_id();
    const u32 u = q.order[d];
    const u32* list_d = q.list[u];
    const u32 nb = q.nbn[d];
    u32 best = 0, blen = 0xFFFFFFFFu, bs = 0;
    u64 by = 0;
    for (u32 k = 0; k < nb; ++k) {
        u32 lo = row_lo(q, d, k, ws->pos), hi = row_hi(q, d, k, ws->pos);
        u32 len = hi - lo;
        by += 8u + 4ull * len;
        if (len < blen) blen = len, best = k, bs = lo;
    }
    bytes += by;
    calls += blen;
    if (blen == 0) return 0;
    const u32 same = q.same_mask[d];
    if (nb == 1) {
        if (!same) return blen;
        // Subtract used same-label vertices that occur in the row: the
        // position of a vertex in C(u_d) comes from u_d's bitmap and rank.
        u32 hit = 0;
        if ((same >> lane) & 1u) {
            // position of the used vertex among C(u_d) (sorted list), then
            // membership of that position in the row
            u32 v = ws->vid[lane];
            u32 lo = 0, hi = q.cnt[u];
            while (lo < hi) {
                u32 mid = (lo + hi) >> 1;
                if (list_d[mid] < v)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            if (lo < q.cnt[u] && list_d[lo] == v) hit = contains_u32(q.adj, bs, bs + blen, lo) ? 1u : 0u;
        }
        u32 h = __popc(__ballot_sync(FULL_MASK, hit));
        return blen - h;
    }
    if (lane == 0) ws->drv[d] = best;
    __syncwarp();
    u64 c = 0;
    for (u32 j = 0; j < blen; j += 32) {
        bool ok = false;
        if (j + lane < blen) ok = accept(q, d, q.adj[bs + j + lane], ws, list_d);
        c += __popc(__ballot_sync(FULL_MASK, ok));
    }
    return c;
}

// Emits the embeddings of the last depth (original data ids, indexed by
// query vertex) into q.emit_buf; returns how many were found.
__device__ u64 emit_last(QState& q, const DevGraph& g, u32 d, WarpStack* ws, u64& bytes, u64& calls) {
    const u32 lane = lane_id();
    const u32 n = d + 1;
    const u32 u = q.order[d];
    const u32* list_d = q.list[u];
    u32 blen = setup_level(q, d, ws, bytes);
    calls += blen;
    const u32 bs = ws->cur[d];
    u64 c = 0;
    for (u32 j = 0; j < blen; j += 32) {
        bool ok = false;
        u32 p = 0;
        if (j + lane < blen) {
            p = q.adj[bs + j + lane];
            ok = accept(q, d, p, ws, list_d);
        }
        u32 bal = __ballot_sync(FULL_MASK, ok);
        u32 k = __popc(bal);
        if (!k) continue;
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd((unsigned long long*)&q.emit_rows, (unsigned long long)k);
        base = __shfl_sync(FULL_MASK, base, 0);
        if (ok) {
            u64 row = base + __popc(bal & ((1u << lane) - 1u));
            if (row < q.emit_cap_rows) {
                u32* out = q.emit_buf + row * n;
                for (u32 i = 0; i < d; ++i) out[q.order[i]] = g.orig[ws->vid[i]];
                out[u] = g.orig[list_d[p]];
            }
        }
        c += k;
    }
    return c;
}

// Bounded lock-free MPMC ring (sequence numbers per slot).
__device__ bool enqueue(EnumCtl* ctl, Slot* slots, const Task& t) {
    const u32 lane = lane_id();
    u32 slot_idx = 0;
    int ok = 0;
    if (lane == 0) {
        u32 pos = ld_volatile_u32(&ctl->q_tail);
        for (int it = 0; it < 64; ++it) {
            Slot* s = slots + (pos % QCAP);
            u32 seq = ld_acquire_u32(&s->seq);
            int diff = (int)(seq - pos);
            if (diff == 0) {
                if (atomicCAS(&ctl->q_tail, pos, pos + 1) == pos) {
                    ok = 1;
                    slot_idx = pos;
                    break;
                }
                pos = ld_volatile_u32(&ctl->q_tail);
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
    const u32* src = (const u32*)&t;
    for (u32 i = lane; i < TASK_WORDS; i += 32) s->w[i] = src[i];
    __threadfence();
    __syncwarp();
    if (lane == 0) st_release_u32(&s->seq, slot_idx + 1);
    return true;
}

__device__ bool dequeue(EnumCtl* ctl, Slot* slots, Task& t) {
    const u32 lane = lane_id();
    u32 slot_idx = 0;
    int ok = 0;
    if (lane == 0) {
        u32 pos = ld_volatile_u32(&ctl->q_head);
        for (int it = 0; it < 64; ++it) {
            Slot* s = slots + (pos % QCAP);
            u32 seq = ld_acquire_u32(&s->seq);
            int diff = (int)(seq - (pos + 1));
            if (diff == 0) {
                if (atomicCAS(&ctl->q_head, pos, pos + 1) == pos) {
                    ok = 1;
                    slot_idx = pos;
                    break;
                }
                pos = ld_volatile_u32(&ctl->q_head);
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
    u32* dst = (u32*)&t;
    for (u32 i = 0; i < TASK_WORDS; ++i) dst[i] = ld_volatile_u32(&s->w[i]);
    __syncwarp();
    if (lane == 0) {
        __threadfence();
        st_release_u32(&s->seq, slot_idx + QCAP);
    }
    return true;
}

// Last-depth count for one lane: the lane's own candidate p (data vertex v)
// sits at depth dl - 1, the rest of the prefix is shared in ws. Counts the
// positions in the intersection of the backward-neighbour rows of depth dl
// whose data vertex differs from every same-label vertex of the embedding.
__device__ u64 lane_last_count(const QState& q, u32 dl, u32 p, u32 v, const WarpStack* ws, u64& bytes, u64& calls) {
    const u32 nb = q.nbn[dl];
    const u32 dp = dl - 1;
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
    const u32 u = q.order[dl];
    const u32* list = q.list[u];
    const u32 same = q.same_mask[dl];
    if (nb == 1) {
        u64 c = blen;
        u32 m = same;
        while (m) {
            const u32 j = __ffs(m) - 1;
            m &= m - 1;
            const u32 vj = j == dp ? v : ws->vid[j];
            const u32 x = lower_bound_u32(list, 0, q.cnt[u], vj);
            if (x < q.cnt[u] && __ldg(list + x) == vj && contains_u32(q.adj, blo, bhi, x)) --c;
        }
        return c;
    }
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

// Every 16 warp steps: donate work when another warp is idle, publish the
// local count (so a capped query stops close to its cap) and stop on the
// cap or the time limit. Returns true when the task must stop.
__device__ bool periodic(QState& q, const Task& t, WarpStack* ws, u32 d, u32 d0, u32 iter, u64& count, u64 flush_at,
                         EnumCtl* ctl, Slot* slots) {
    const u32 lane = lane_id();
    if (ld_volatile_u32(&ctl->hungry) > 0) {
        // (a) upper half of the shallowest unexplored driver range of at
        // least 64 elements, else (b) the last unexplored chunk entry of the
        // shallowest depth below d, as a task starting one level deeper.
        u32 dd = d0;
        for (; dd <= d; ++dd)
            if (ws->end[dd] - ws->cur[dd] >= 64u) break;
        u32 de = d0;
        for (; de < d; ++de)
            if (ws->cn[de] > ws->ci[de]) break;
        Task nt;
        nt.qi = t.qi;
        bool have = false;
        if (dd <= d) {
            const u32 c0 = ws->cur[dd], e0 = ws->end[dd];
            nt.d0 = dd;
            nt.b = c0 + ((e0 - c0) >> 1);
            nt.e = e0;
            nt.drv = ws->drv[dd];
            for (u32 i = 0; i < PSM_MAXQ; ++i) nt.pos[i] = i < dd ? ws->pos[i] : 0;
            have = true;
        } else if (de < d) {
            nt.d0 = de + 1;
            nt.b = FULL_LEVEL;
            nt.e = FULL_LEVEL;
            nt.drv = 0;
            for (u32 i = 0; i < PSM_MAXQ; ++i) nt.pos[i] = i < de ? ws->pos[i] : 0;
            nt.pos[de] = ws->chunk[de][ws->cn[de] - 1];
            have = true;
        }
        if (have) {
            if (lane == 0) atomicAdd(&ctl->pending, 1ull);
            __threadfence();
            __syncwarp();
            if (enqueue(ctl, slots, nt)) {
                if (lane == 0) {
                    if (nt.b != FULL_LEVEL)
                        ws->end[dd] = nt.b;
                    else
                        ws->cn[de] -= 1;
                    atomicAdd((unsigned long long*)&ctl->donations, 1ull);
                }
            } else if (lane == 0) {
                atomicAdd(&ctl->pending, (unsigned long long)-1ll);
            }
            __syncwarp();
        }
    }
    if (count >= flush_at && lane == 0) {
        unsigned long long old = atomicAdd((unsigned long long*)&q.count, count);
        if (q.cap && old + count >= q.cap) atomicExch(&q.stop, 1u);
        count = 0;
    }
    count = __shfl_sync(FULL_MASK, count, 0);
    u32 stop = ld_volatile_u32(&q.stop);
    if (!stop && (iter & 255u) == 0 && global_timer_ns() > ctl->deadline_ns) {
        if (lane == 0) {
            atomicExch(&q.overtime, 1u);
            atomicExch(&q.stop, 1u);
        }
        stop = 1;
    }
    return __shfl_sync(FULL_MASK, stop, 0) != 0;
}

// Runs one task to completion (or until the query stops).
__device__ void run_task(const DevGraph& g, QState* qs, const Task& t, WarpStack* ws, EnumCtl* ctl, Slot* slots,
                         bool emit) {
    const u32 lane = lane_id();
    QState& q = qs[t.qi];
    const u32 n = q.desc->n;
    const u32 d0 = t.d0;
    if (ld_volatile_u32(&q.stop)) return;
    u64 count = 0, bytes = 0, calls = 0;
    // restore the prefix
    if (lane < d0) {
        ws->pos[lane] = t.pos[lane];
        ws->vid[lane] = q.list[q.order[lane]][t.pos[lane]];
    }
    if (lane == 0) {
        ws->cur[d0] = t.b;
        ws->end[d0] = t.e;
        ws->drv[d0] = t.drv;
        ws->cn[d0] = 0;
        ws->ci[d0] = 0;
    }
    __syncwarp();
    if (n == 1) {  // single-vertex query: every root candidate is an embedding
        count = t.e - t.b;
        calls = count;
        if (emit) {
            for (u32 i = t.b + lane; i < t.e; i += 32) {
                unsigned long long r = atomicAdd((unsigned long long*)&q.emit_rows, 1ull);
                if (r < q.emit_cap_rows) q.emit_buf[r] = g.orig[q.list[q.order[0]][i]];
            }
        }
    } else if (t.b == FULL_LEVEL && d0 + 1 == n) {
        // donated entry whose children are the last depth
        count += emit ? emit_last(q, g, d0, ws, bytes, calls) : count_last(q, d0, ws, bytes, calls);
    } else {
        u32 d = d0;
        if (t.b == FULL_LEVEL) setup_level(q, d0, ws, bytes);
        u32 iter = 0;
        u64 bytes_l = 0, calls_l = 0;  // per-lane parts, summed at the end
        const u64 flush_at = 1ull << 16;
        while (true) {
            if (d + 2 == n && !emit) {
                // The last two depths fused: each lane takes one driver
                // element of depth d and counts its completions at depth
                // d + 1 on its own (32 partial embeddings per warp step).
                if (ws->cur[d] < ws->end[d]) {
                    const u32 cur = ws->cur[d], end = ws->end[d];
                    const u32 idx = cur + lane;
                    u64 c = 0;
                    if (idx < end) {
                        const u32* list_d = q.list[q.order[d]];
                        u32 p = d == 0 ? idx : q.adj[idx];
                        if (d == 0 || accept(q, d, p, ws, list_d))
                            c = lane_last_count(q, d + 1, p, list_d[p], ws, bytes_l, calls_l);
                    }
                    count += warp_sum64(c);
                    calls += min(32u, end - cur);
                    __syncwarp();
                    if (lane == 0) ws->cur[d] = min(end, cur + 32u);
                    __syncwarp();
                    if ((++iter & 15u) == 0 && periodic(q, t, ws, d, d0, iter, count, flush_at, ctl, slots)) break;
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
                }
                __syncwarp();
                if (d + 2 == n) {
                    u64 c = emit ? emit_last(q, g, d + 1, ws, bytes, calls) : count_last(q, d + 1, ws, bytes, calls);
                    count += c;
                } else {
                    d += 1;
                    setup_level(q, d, ws, bytes);
                }
            } else if (ws->cur[d] < ws->end[d]) {
                const u32 cur = ws->cur[d], end = ws->end[d];
                const u32 idx = cur + lane;
                bool ok = false;
                u32 p = 0;
                if (d == 0) {
                    p = idx;
                    ok = idx < end;
                } else if (idx < end) {
                    p = q.adj[idx];
                    ok = accept(q, d, p, ws, q.list[q.order[d]]);
                }
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
                if ((++iter & 15u) == 0 && periodic(q, t, ws, d, d0, iter, count, flush_at, ctl, slots)) break;
            } else {
                if (d == d0) break;
                d -= 1;
            }
        }
        bytes += warp_sum64(bytes_l);
        calls += warp_sum64(calls_l);
    }
    if (lane == 0) {
        if (count) {
            unsigned long long old = atomicAdd((unsigned long long*)&q.count, count);
            if (q.cap && old + count >= q.cap) atomicExch(&q.stop, 1u);
        }
        if (calls) atomicAdd((unsigned long long*)&q.calls, calls);
        if (bytes) atomicAdd((unsigned long long*)&q.alg_bytes, bytes);
    }
}

// Root ticket -> (query, candidate range); prefix[i] = roots before query i.
__device__ bool take_root(EnumCtl* ctl, const u32* prefix, QState* qs, Task& t, u32 grab) {
    const u32 lane = lane_id();
    // Once the ticket passes the end it never comes back; skipping the
    // pending increment then keeps idle warps from holding `pending` above
    // zero with transient increments.
    if (ld_volatile_u32(&ctl->root_ticket) >= ctl->total_roots) return false;
    u32 r = 0, crossing = 0;
    if (lane == 0) {
        atomicAdd(&ctl->pending, 1ull);
        __threadfence();
        r = atomicAdd(&ctl->root_ticket, grab);
        if (r >= ctl->total_roots) {
            atomicAdd(&ctl->pending, (unsigned long long)-1ll);
        } else if (r + grab >= ctl->total_roots) {
            crossing = 1;  // this grab exhausts the pool: release the pool's token
        }
    }
    r = __shfl_sync(FULL_MASK, r, 0);
    crossing = __shfl_sync(FULL_MASK, crossing, 0);
    if (r >= ctl->total_roots) return false;
    if (crossing && lane == 0) {
        __threadfence();
        atomicAdd(&ctl->pending, (unsigned long long)-1ll);
    }
    // query owning root r
    u32 lo = 0, hi = ctl->nq;
    while (hi - lo > 1) {
        u32 mid = (lo + hi) >> 1;
        if (prefix[mid] <= r)
            lo = mid;
        else
            hi = mid;
    }
    t.qi = lo;
    t.d0 = 0;
    t.b = r - prefix[lo];
    t.e = min(prefix[lo + 1], r + grab) - prefix[lo];
    t.drv = 0;
    return true;
}

__global__ void __launch_bounds__(WARPS_PER_BLOCK * 32) enum_kernel(DevGraph g, QState* qs, EnumCtl* ctl,
                                                                    Slot* slots, const u32* prefix, int emit) {
    __shared__ WarpStack stacks[WARPS_PER_BLOCK];
    WarpStack* ws = &stacks[threadIdx.x >> 5];
    const u32 lane = lane_id();
    Task t;
    bool hungry = false;
    u64 spins = 0;
    while (true) {
        bool got = take_root(ctl, prefix, qs, t, 1);
        if (!got) got = dequeue(ctl, slots, t);
        if (got) {
            if (hungry && lane == 0) atomicSub(&ctl->hungry, 1u);
            hungry = false;
            spins = 0;
            run_task(g, qs, t, ws, ctl, slots, emit != 0);
            __syncwarp();
            if (lane == 0) {
                __threadfence();
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
        ++spins;
        if ((spins & 255u) == 0) {
            u32 bail = 0;
            if (lane == 0 && (global_timer_ns() > ctl->deadline_ns + 2000000000ull || spins > (1ull << 32))) {
                atomicExch(&ctl->error, 1u);
                bail = 1;
            }
            if (__shfl_sync(FULL_MASK, bail, 0)) break;
        }
        __nanosleep(200);
    }
}

__global__ void enum_init_kernel(QState* qs, u32 nq, EnumCtl* ctl, Slot* slots, u32* prefix, u64 budget_ns) {
    // single block: prefix of root counts, queue sequence numbers
    __shared__ u32 s_carry;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (u32 base = 0; base < nq; base += blockDim.x) {
        u32 i = base + threadIdx.x;
        u32 v = 0;
        if (i < nq) v = (qs[i].status == PSM_DEV_OK && !qs[i].stop) ? qs[i].root_cnt : 0u;
        // block scan (simple: warp scans + shared totals)
        __shared__ u32 wt[32];
        u32 incl = warp_incl_scan(v);
        if (lane_id() == 31) wt[threadIdx.x >> 5] = incl;
        __syncthreads();
        if (threadIdx.x < 32) {
            u32 x = threadIdx.x < (blockDim.x >> 5) ? wt[threadIdx.x] : 0;
            u32 xi = warp_incl_scan(x);
            wt[threadIdx.x] = xi - x;
        }
        __syncthreads();
        u32 excl = s_carry + wt[threadIdx.x >> 5] + incl - v;
        if (i < nq) prefix[i] = excl;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) s_carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        prefix[nq] = s_carry;
        ctl->total_roots = s_carry;
        ctl->root_ticket = 0;
        ctl->hungry = 0;
        ctl->q_head = 0;
        ctl->q_tail = 0;
        ctl->error = 0;
        ctl->nq = nq;
        ctl->pending = s_carry > 0 ? 1ull : 0ull;  // the root pool's token
        ctl->deadline_ns = global_timer_ns() + budget_ns;
        ctl->donations = 0;
    }
    for (u32 i = threadIdx.x; i < QCAP; i += blockDim.x) slots[i].seq = i;
}

__global__ void gather_kernel(const QState* qs, u32 nq, DevResult* out) {
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += gridDim.x * blockDim.x) {
        const QState& q = qs[i];
        DevResult r;
        r.count = q.cap && q.count > q.cap ? q.cap : q.count;
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

}  // namespace

cudaError_t psm_launch_gather(const QState* qs, u32 nq, DevResult* out, cudaStream_t st) {
    u32 blocks = (nq + 255) / 256;
    gather_kernel<<<blocks ? blocks : 1, 256, 0, st>>>(qs, nq, out);
    return cudaGetLastError();
}

size_t psm_enum_scratch_bytes() { return sizeof(EnumCtl) + sizeof(Slot) * QCAP + 64; }

cudaError_t psm_launch_enum(const DevGraph& g, QState* qs, u32 nq, void* scratch, u32* prefix, u64 budget_ns,
                            int emit, int blocks, cudaStream_t st) {
    EnumCtl* ctl = (EnumCtl*)scratch;
    Slot* slots = (Slot*)((char*)scratch + ((sizeof(EnumCtl) + 15) & ~(size_t)15));
    enum_init_kernel<<<1, 1024, 0, st>>>(qs, nq, ctl, slots, prefix, budget_ns);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    enum_kernel<<<blocks, WARPS_PER_BLOCK * 32, 0, st>>>(g, qs, ctl, slots, prefix, emit);
    return cudaGetLastError();
}

cudaError_t psm_enum_max_blocks(int* blocks) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, enum_kernel, WARPS_PER_BLOCK * 32, 0);
    if (e != cudaSuccess) return e;
    *blocks = sms * (per_sm < 1 ? 1 : per_sm);
    return cudaSuccess;
}

// Reads back the launch-wide error flag and donation count.
cudaError_t psm_enum_read_ctl(void* scratch, u32* error, u64* donations, cudaStream_t st) {
    EnumCtl h;
    cudaError_t e = cudaMemcpyAsync(&h, scratch, sizeof(EnumCtl), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    *error = h.error;
    *donations = h.donations;
    return cudaSuccess;
}
