// Query preparation on the device: NLF / GQL / CFL candidate filtering,
// candidate compaction, candidate-edge tables and the GQL / CFL matching
// orders. The reference runs these stages on one host thread:
//   filters    matching/FilterVertices.cpp:48-250, :704-966
//   tables     matching/BuildTable.cpp:9-151
//   orders     matching/GenerateQueryPlan.cpp:9-83, :270-471, :680-721
//   bn lists   matching/EvaluateQuery.cpp:1594-1625
// Here every stage is a data-parallel loop over a "team" of threads: one
// thread block per query when many queries are prepared in one persistent
// launch (batched / serving), or the whole grid for one query (plain path).
// Both kinds of team run the same code, so results cannot differ between the
// two paths. Stages that the reference performs in place in a fixed order
// (GQL refinement of u = 0..q-1, the CFL generate / prune steps) are
// separated by team barriers and keep that order, which makes the candidate
// sets identical to the reference's.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "device_util.cuh"
#include "psm_internal.h"

namespace cg = cooperative_groups;

namespace {

// ---------------------------------------------------------------- teams --

// kRowLanes: lanes per candidate row in the table passes. A small team keeps
// more rows in flight with 4; the 148-block grid has rows enough and gains
// from 8 on hub rows.
struct BlockTeam {
    static constexpr u32 kRowLanes = 4;
    __device__ u32 rank() const { return threadIdx.x; }
    __device__ u32 size() const { return blockDim.x; }
    __device__ u32 warp() const { return threadIdx.x >> 5; }
    __device__ u32 nwarps() const { return blockDim.x >> 5; }
    __device__ u32 block() const { return 0; }
    __device__ u32 nblocks() const { return 1; }
    __device__ bool sync() {
        __syncthreads();
        return true;
    }
};

struct GridBarrier {
    u32 count;  // arrivals; its top bit flips once per completed barrier
    u32 abort;
    u32 pad[2];
};

// Whole-grid team for a cooperative launch (all blocks co-resident). One
// release-add per block per barrier: block 0 adds 2^31 - (blocks - 1), the
// others add 1, so the top bit of `count` flips exactly when every block
// has arrived. Waits are bounded: past the deadline or the iteration cap a
// block raises `abort`, every later barrier returns false at once and the
// kernel unwinds; the host reports an internal error.
struct GridTeam {
    static constexpr u32 kRowLanes = 8;
    GridBarrier* bar;
    u64 deadline_ns;
    __device__ u32 rank() const { return blockIdx.x * blockDim.x + threadIdx.x; }
    __device__ u32 size() const { return gridDim.x * blockDim.x; }
    __device__ u32 warp() const { return rank() >> 5; }
    __device__ u32 nwarps() const { return size() >> 5; }
    __device__ u32 block() const { return blockIdx.x; }
    __device__ u32 nblocks() const { return gridDim.x; }
    __device__ bool sync() {
        __shared__ u32 s_abort;
        __syncthreads();
        if (threadIdx.x == 0) {
            u32 ab = ld_acquire_u32(&bar->abort);
            if (!ab) {
                const u32 add = blockIdx.x == 0 ? (0x80000000u - (gridDim.x - 1)) : 1u;
                u32 old;
                asm volatile("atom.add.release.gpu.u32 %0, [%1], %2;" : "=r"(old) : "l"(&bar->count), "r"(add)
                             : "memory");
                u32 it = 0;
                while (((ld_acquire_u32(&bar->count) ^ old) & 0x80000000u) == 0) {
                    ++it;
                    if ((it & 63u) == 0) {
                        if (ld_acquire_u32(&bar->abort)) break;
                        if ((it & 4095u) == 0 && (global_timer_ns() > deadline_ns || it > (1u << 30))) {
                            atomicExch(&bar->abort, 1u);
                            break;
                        }
                    }
                    if (it > 128) __nanosleep(32);
                }
                ab = ld_acquire_u32(&bar->abort);
            }
            s_abort = ab;
        }
        __syncthreads();
        return s_abort == 0;
    }
};

// Thread-block cluster team: the blocks of one cluster (co-scheduled on one
// GPC) share a hardware barrier, so a step costs far less than a grid-wide
// software barrier. Release/acquire at cluster scope makes the global-memory
// writes of every block visible to the others after sync().
struct ClusterTeam {
    static constexpr u32 kRowLanes = 4;
    __device__ u32 rank() const { return cg::this_cluster().block_rank() * blockDim.x + threadIdx.x; }
    __device__ u32 size() const { return cg::this_cluster().num_blocks() * blockDim.x; }
    __device__ u32 warp() const { return rank() >> 5; }
    __device__ u32 nwarps() const { return size() >> 5; }
    __device__ u32 block() const { return cg::this_cluster().block_rank(); }
    __device__ u32 nblocks() const { return cg::this_cluster().num_blocks(); }
    __device__ bool sync() {
        __threadfence();
        cg::this_cluster().sync();
        return true;
    }
};

#define TSYNC(t)                 \
    do {                         \
        if (!(t).sync()) return; \
    } while (0)
#define TSYNC_B(t)                     \
    do {                               \
        if (!(t).sync()) return false; \
    } while (0)

// Team-wide exclusive scan of val(0..N-1): emit(i, prefix) for every i and
// *total receives the sum (written by team rank 0). Two levels: warps inside
// a block through shared memory, blocks through `scratch` (>= nblocks words).
template <class Team, class ValF, class EmitF>
__device__ bool team_scan(Team& t, u32 N, u32* scratch, ValF val, EmitF emit, u32* total) {
    __shared__ u32 s_wt[32];
    __shared__ u32 s_bp;
    const u32 nb = t.nblocks(), b = t.block();
    const u32 lane = lane_id(), w = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    const u32 per_blk = ((N + nb - 1) / nb + 31u) & ~31u;
    const u32 b0 = min(N, b * per_blk), b1 = min(N, b0 + per_blk);
    const u32 per_w = ((b1 - b0 + wpb - 1) / wpb + 31u) & ~31u;
    const u32 w0 = min(b1, b0 + w * per_w), w1 = min(b1, w0 + per_w);
    u32 s = 0;
    for (u32 i = w0 + lane; i < w1; i += 32) s += val(i);
    s = warp_sum(s);
    if (lane == 0) s_wt[w] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        u32 tot = 0;
        for (u32 i = 0; i < wpb; ++i) tot += s_wt[i];
        scratch[b] = tot;
    }
    TSYNC_B(t);
    if (w == 0) {
        u32 x = 0, all = 0;
        for (u32 i = lane; i < nb; i += 32) {
            u32 v = ld_volatile_u32(scratch + i);
            if (i < b) x += v;
            all += v;
        }
        x = warp_sum(x);
        all = warp_sum(all);
        if (lane == 0) {
            s_bp = x;
            if (b == 0 && total) *total = all;
        }
    }
    __syncthreads();
    u32 carry = s_bp;
    for (u32 i = 0; i < w; ++i) carry += s_wt[i];
    for (u32 base = w0; base < w1; base += 32) {
        u32 i = base + lane;
        u32 v = i < w1 ? val(i) : 0;
        u32 incl = warp_incl_scan(v);
        if (i < w1) emit(i, carry + incl - v);
        carry += __shfl_sync(FULL_MASK, incl, 31);
    }
    __syncthreads();
    return true;
}

// ------------------------------------------------------------ filters --

// NLF test of item t (a query vertex or a relabelled one) against data vertex
// v: degree, then per neighbour label a run at least as long as required
// (matching/FilterVertices.cpp:767-813). Labels are ascending, so the search
// window shrinks from label to label.
__device__ bool nlf_ok(const DevGraph& g, const QDesc* d, u32 t, u32 v) {
    u32 lo = g.off[v], hi = g.off[v + 1];
    if (hi - lo < d->item_deg[t]) return false;
    for (u32 k = d->nlf_off[t]; k < d->nlf_off[t + 1]; ++k) {
        u32 l = d->nlf_lab[k], need = d->nlf_cnt[k];
        if (l >= g.L) return false;
        u32 s = lower_bound_u32(g.nbr, lo, hi, g.lab_off[l]);
        if (hi - s < need) return false;
        u32 e = lower_bound_u32(g.nbr, s, hi, g.lab_off[l + 1]);
        if (e - s < need) return false;
        lo = e;
    }
    return true;
}

// nlf_ok for the 8-lane group of this lane (t uniform in the warp, v and
// valid uniform in the group); the label runs come from group_lower_bound.
// Called by the whole warp.
__device__ bool group_nlf_ok(const DevGraph& g, const QDesc* d, u32 t, bool valid, u32 v) {
    u32 lo = 0, hi = 0;
    if (valid) {
        lo = g.off[v];
        hi = g.off[v + 1];
    }
    bool ok = valid && hi - lo >= d->item_deg[t];
    for (u32 k = d->nlf_off[t]; k < d->nlf_off[t + 1]; ++k) {
        if (!__any_sync(FULL_MASK, ok)) break;
        const u32 l = d->nlf_lab[k], need = d->nlf_cnt[k];
        if (l >= g.L) ok = false;
        const u32 s = group_lower_bound(g.nbr, ok ? lo : 0u, ok ? hi : 0u, ok ? g.lab_off[l] : 0u);
        if (ok && hi - s < need) ok = false;
        const u32 e = group_lower_bound(g.nbr, ok ? s : 0u, ok ? hi : 0u, ok ? g.lab_off[l + 1] : 0u);
        if (ok && e - s < need) ok = false;
        if (ok) lo = e;
    }
    return ok;
}

__device__ __forceinline__ u32 bucket_size(const DevGraph& g, u32 l) {
    return l < g.L ? g.lab_off[l + 1] - g.lab_off[l] : 0u;
}
__device__ __forceinline__ u32 bucket_base(const DevGraph& g, u32 l) { return l < g.L ? g.lab_off[l] : 0u; }

// Adds a right vertex with neighbourhood `m` (bitmask over left = query
// vertices) to a maximum bipartite matching kept in lane-distributed form:
// lane x holds in `rm` the neighbourhood of the right vertex matched to left
// vertex x. Searches an augmenting path from the new vertex with a BFS over
// left vertices. All arguments are warp-uniform except rm.
__device__ __forceinline__ void match_add(u32 m, u32& matched, u32& rm) {
    const u32 lane = lane_id();
    int parent = -1;  // lane-distributed: BFS parent (left vertex) of left vertex `lane`
    u32 visited = m, frontier = m;
    while (true) {
        u32 fr = visited & ~matched;
        if (fr) {
            u32 i = __ffs(fr) - 1;
            // Walk back to the new vertex, shifting matched right vertices.
            while (true) {
                int p = __shfl_sync(FULL_MASK, parent, i);
                u32 val = p < 0 ? m : __shfl_sync(FULL_MASK, rm, (u32)p);
                if (lane == i) rm = val;
                if (p < 0) break;
                i = (u32)p;
            }
            matched |= fr & (0u - fr);
            return;
        }
        u32 nw = 0;
        u32 f = frontier;
        while (f) {
            u32 j = __ffs(f) - 1;
            f &= f - 1;
            u32 nm = __shfl_sync(FULL_MASK, rm, j) & ~visited & ~nw;
            if ((nm >> lane) & 1u) parent = (int)j;
            nw |= nm;
        }
        if (!nw) return;
        visited |= nw;
        frontier = nw;
    }
}

// GQL local test of candidate v for query vertex u: N(u) must have a matching
// into N(v) that saturates N(u), where u' -- w iff w is still a candidate of
// u' (matching/FilterVertices.cpp:704-741). The bipartite graph splits by
// label, so each neighbour label is matched on its own; right vertices are
// streamed through an incremental maximum matching (warp-wide).
__device__ bool gql_check(const DevGraph& g, const QDesc* d, const QState& q, u32 u, u32 v) {
    const u32 lane = lane_id();
    u32 lo = g.off[v], hi = g.off[v + 1];
    for (u32 k = d->nlf_off[u]; k < d->nlf_off[u + 1]; ++k) {
        const u32 l = d->nlf_lab[k], S = d->nlf_grp[k];
        if (l >= g.L) return false;
        u32 s = lower_bound_u32(g.nbr, lo, hi, g.lab_off[l]);
        u32 e = lower_bound_u32(g.nbr, s, hi, g.lab_off[l + 1]);
        lo = e;
        const u32 base = g.lab_off[l];
        u32 matched = 0, rm = 0;
        for (u32 j = s; j < e && matched != S; j += 32) {
            u32 idx = j + lane, m = 0;
            if (idx < e) {
                u32 pos = __ldg(g.nbr + idx) - base;
                u32 x = S;
                while (x) {
                    u32 y = __ffs(x) - 1;
                    x &= x - 1;
                    if (test_bit(q.bm[y], pos)) m |= 1u << y;
                }
            }
            u32 nz = __ballot_sync(FULL_MASK, m != 0);
            while (nz && matched != S) {
                u32 src = __ffs(nz) - 1;
                nz &= nz - 1;
                u32 mm = __shfl_sync(FULL_MASK, m, src);
                match_add(mm, matched, rm);
            }
        }
        if (matched != S) return false;
    }
    return true;
}

template <class Team>
__device__ bool compact_vertex(Team& t, const DevGraph& g, QState& q, u32 u) {
    const u32* bm = q.bm[u];
    u32* rank = q.rank[u];
    u32* list = q.list[u];
    const u32 base = bucket_base(g, q.desc->label[u]);
    return team_scan(
        t, q.bwords[u], q.scan, [&](u32 i) { return (u32)__popc(bm[i]); },
        [&](u32 i, u32 pre) {
            rank[i] = pre;
            u32 x = bm[i];
            u32 j = pre;
            while (x) {
                u32 b = __ffs(x) - 1;
                x &= x - 1;
                list[j++] = base + 32u * i + b;
            }
        },
        &q.cnt[u]);
}

// compact_vertex for every vertex in `mask` with one team barrier: a warp
// per vertex sums the block's part of its bitmap into
// scratch[k * nblocks + block] (k: the vertex's rank in mask; scratch holds
// nblocks words per query vertex), then, after the barrier, adds the parts of
// the blocks before it and emits the block's ranks and list entries. Same
// word partition as team_scan. The caller syncs the team afterwards.
template <class Team>
__device__ bool multi_compact(Team& t, const DevGraph& g, QState& q, u32 mask) {
    const u32 nb = t.nblocks(), b = t.block();
    const u32 lane = lane_id(), w = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    const u32 m = __popc(mask);
    auto vertex = [&](u32 k) {
        u32 x = mask;
        for (u32 j = 0; j < k; ++j) x &= x - 1u;
        return (u32)__ffs(x) - 1u;
    };
    for (u32 k = w; k < m; k += wpb) {
        const u32 u = vertex(k), N = q.bwords[u];
        const u32 per_blk = ((N + nb - 1) / nb + 31u) & ~31u;
        const u32 b0 = min(N, b * per_blk), b1 = min(N, b0 + per_blk);
        u32 c = 0;
        for (u32 i = b0 + lane; i < b1; i += 32) c += __popc(q.bm[u][i]);
        c = warp_sum(c);
        if (lane == 0) q.scan[k * nb + b] = c;
    }
    TSYNC_B(t);
    for (u32 k = w; k < m; k += wpb) {
        const u32 u = vertex(k), N = q.bwords[u];
        const u32 per_blk = ((N + nb - 1) / nb + 31u) & ~31u;
        const u32 b0 = min(N, b * per_blk), b1 = min(N, b0 + per_blk);
        u32 before = 0, all = 0;
        for (u32 i = lane; i < nb; i += 32) {
            const u32 v = ld_volatile_u32(q.scan + k * nb + i);
            if (i < b) before += v;
            all += v;
        }
        before = warp_sum(before);
        all = warp_sum(all);
        if (b == 0 && lane == 0) q.cnt[u] = all;
        const u32* bm = q.bm[u];
        u32* rank = q.rank[u];
        u32* list = q.list[u];
        const u32 base = bucket_base(g, q.desc->label[u]);
        u32 carry = before;
        for (u32 i0 = b0; i0 < b1; i0 += 32) {
            const u32 i = i0 + lane;
            u32 x = i < b1 ? bm[i] : 0u;
            const u32 v = __popc(x);
            const u32 incl = warp_incl_scan(v);
            if (i < b1) {
                u32 j = carry + incl - v;
                rank[i] = j;
                while (x) {
                    const u32 bit = __ffs(x) - 1u;
                    x &= x - 1u;
                    list[j++] = base + 32u * i + bit;
                }
            }
            carry += __shfl_sync(FULL_MASK, incl, 31);
        }
    }
    return true;
}

// Stage 1: NLF candidates for every needed item, one warp per bitmap word.
template <class Team>
__device__ void stage_nlf(Team& t, const DevGraph& g, QState& q, u32 need_mask, bool want_virtual) {
    const QDesc* d = q.desc;
    const u32 n = d->n, nitems = n + d->nvirt;
    const u32 lane = lane_id();
    u32 total_words = 0;
    for (u32 it = 0; it < nitems; ++it) {
        bool needed = it < n ? ((need_mask >> it) & 1u) : want_virtual;
        if (needed) total_words += (bucket_size(g, d->item_label[it]) + 31u) >> 5;
    }
    for (u32 gw = t.warp(); gw < total_words; gw += t.nwarps()) {
        u32 it = 0, w = gw;
        for (; it < nitems; ++it) {
            bool needed = it < n ? ((need_mask >> it) & 1u) : want_virtual;
            if (!needed) continue;
            u32 nw = (bucket_size(g, d->item_label[it]) + 31u) >> 5;
            if (w < nw) break;
            w -= nw;
        }
        const u32 l = d->item_label[it];
        const u32 bsz = bucket_size(g, l);
        const u32 pos = 32u * w + lane;
        bool ok = pos < bsz && nlf_ok(g, d, it, g.lab_off[l] + pos);
        u32 word = __ballot_sync(FULL_MASK, ok);
        if (lane == 0) {
            if (it < n) q.bm[it][w] = word;
            if (word) atomicAdd(&q.item_cnt[it], (u32)__popc(word));
        }
    }
}

// matching/FilterVertices.cpp:841-912 (generateCandidates): candidates of u
// are the data vertices of u's label, with enough degree and NLF, adjacent to
// a live candidate of every pivot. Marks neighbours of each pivot's
// candidates into a bucket bitmap (8 lanes per candidate), ANDs across
// pivots, then applies the degree + NLF test per surviving bit.
template <class Team>
__device__ bool mark_neighbours(Team& t, const DevGraph& g, QState& q, u32 p, u32 lu, u32* out) {
    const u32 lane = lane_id(), grp = lane >> 3, lg = lane & 7u;
    const u32 base_u = bucket_base(g, lu);
    const u32 base_p = bucket_base(g, q.desc->label[p]);
    const u32 N = q.cnt[p];
    for (u32 i0 = t.warp() * 4u; i0 < N; i0 += t.nwarps() * 4u) {
        u32 i = i0 + grp;
        u32 c = 0, s, e;
        bool live = false;
        if (i < N) {
            c = q.list[p][i];
            live = test_bit(q.bm[p], c - base_p);
        }
        group_label_run(g, live, c, lu, s, e);
        u32 len = e - s;
        u32 mx = warp_max(len);
        for (u32 j = 0; j < mx; j += 32) {  // 4 loads in flight per lane
            u32 x[4];
#pragma unroll
            for (u32 k = 0; k < 4; ++k) {
                const u32 o = j + 8u * k + lg;
                x[k] = o < len ? __ldg(g.nbr + s + o) : 0u;
            }
#pragma unroll
            for (u32 k = 0; k < 4; ++k)
                if (j + 8u * k + lg < len) {
                    const u32 pos = x[k] - base_u;
                    atomicOr(out + (pos >> 5), 1u << (pos & 31u));
                }
        }
    }
    return true;
}

// Contiguous word range of block b in a team scan over N words (the same
// partition team_scan uses).
__device__ __forceinline__ u32 scan_block_words(u32 N, u32 nb) { return ((N + nb - 1) / nb + 31u) & ~31u; }

// Second half of a team scan whose per-block totals are already in
// scratch[0, nblocks): each warp recounts its own words, then emits rank and
// list entries of bitmap u. *total (by team rank 0) = candidate count.
template <class Team>
__device__ bool compact_from_totals(Team& t, const DevGraph& g, QState& q, u32 u) {
    __shared__ u32 s_wt[32];
    __shared__ u32 s_bp;
    const u32 N = q.bwords[u];
    const u32* bm = q.bm[u];
    u32* rank = q.rank[u];
    u32* list = q.list[u];
    const u32 base = bucket_base(g, q.desc->label[u]);
    const u32 nb = t.nblocks(), b = t.block();
    const u32 lane = lane_id(), w = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    const u32 per_blk = scan_block_words(N, nb);
    const u32 b0 = min(N, b * per_blk), b1 = min(N, b0 + per_blk);
    const u32 per_w = ((b1 - b0 + wpb - 1) / wpb + 31u) & ~31u;
    const u32 w0 = min(b1, b0 + w * per_w), w1 = min(b1, w0 + per_w);
    u32 s = 0;
    for (u32 i = w0 + lane; i < w1; i += 32) s += __popc(bm[i]);
    s = warp_sum(s);
    if (lane == 0) s_wt[w] = s;
    if (w == 0) {
        u32 x = 0, all = 0;
        for (u32 i = lane; i < nb; i += 32) {
            u32 v = ld_volatile_u32(q.scan + i);
            if (i < b) x += v;
            all += v;
        }
        x = warp_sum(x);
        all = warp_sum(all);
        if (lane == 0) {
            s_bp = x;
            if (b == 0) q.cnt[u] = all;
        }
    }
    __syncthreads();
    u32 carry = s_bp;
    for (u32 i = 0; i < w; ++i) carry += s_wt[i];
    for (u32 base_i = w0; base_i < w1; base_i += 32) {
        u32 i = base_i + lane;
        u32 x = i < w1 ? bm[i] : 0u;
        u32 v = __popc(x);
        u32 incl = warp_incl_scan(v);
        if (i < w1) {
            u32 j = carry + incl - v;
            rank[i] = j;
            while (x) {
                u32 bit = __ffs(x) - 1;
                x &= x - 1;
                list[j++] = base + 32u * i + bit;
            }
        }
        carry += __shfl_sync(FULL_MASK, incl, 31);
    }
    __syncthreads();
    return true;
}

// matching/FilterVertices.cpp:841-912 (generateCandidates): candidates of u
// are the data vertices of u's label, with enough degree and NLF, adjacent to
// a live candidate of every pivot. The accumulator bitmaps (acc, tmp) are
// all-zero between steps: they are cleared once at the start of the query
// and re-zeroed where they are consumed.
template <class Team>
__device__ bool step_generate(Team& t, const DevGraph& g, QState& q, u32 u, u32 pivots) {
    const QDesc* d = q.desc;
    const u32 lu = d->label[u];
    const u32 W = q.bwords[u];
    bool first = true;
    u32 pm = pivots;
    while (pm) {
        u32 p = __ffs(pm) - 1;
        pm &= pm - 1;
        if (first) {
            mark_neighbours(t, g, q, p, lu, q.acc);
        } else {
            mark_neighbours(t, g, q, p, lu, q.tmp);
            TSYNC_B(t);
            for (u32 i = t.rank(); i < W; i += t.size()) {
                q.acc[i] &= q.tmp[i];
                q.tmp[i] = 0;
            }
        }
        first = false;
        if (!pm)  // the scan's per-block totals start from zero
            for (u32 i = t.rank(); i < t.nblocks(); i += t.size()) q.scan[i] = 0;
        TSYNC_B(t);
    }
    // Survivors: degree + NLF per surviving bit (warp per word); the word's
    // popcount goes straight to the total of the block that will emit it.
    const u32 lane = lane_id();
    const u32 base = bucket_base(g, lu), bsz = bucket_size(g, lu);
    const u32 per_blk = scan_block_words(W, t.nblocks());
    const u32 grp = lane >> 3, lg = lane & 7u;
    const bool nlf_known = q.nlf_all;  // u's NLF set is in bm[u] (stage 1)
    for (u32 w = t.warp(); w < W; w += t.nwarps()) {
        u32 bits = q.acc[w];
        if (bsz - 32u * w < 32u) bits &= (1u << (bsz - 32u * w)) - 1u;  // W words cover bsz bits
        u32 word = 0;
        if (nlf_known) {
            word = bits & q.bm[u][w];
        } else if (__popc(bits) > 8u) {  // dense word: a lane per bit
            const bool ok = ((bits >> lane) & 1u) && nlf_ok(g, d, u, base + 32u * w + lane);
            word = __ballot_sync(FULL_MASK, ok);
        } else {
            while (bits) {  // sparse word: a lane group per bit, 4 bits a round
                u32 b = bits;
                for (u32 k = 0; k < grp; ++k) b &= b - 1u;
                const u32 bit = b ? __ffs(b) - 1u : 0u;
                const bool ok = group_nlf_ok(g, d, u, b != 0, base + 32u * w + bit);
                word |= __reduce_or_sync(FULL_MASK, ok && lg == 0 ? 1u << bit : 0u);
                for (u32 k = 0; k < 4u; ++k) bits &= bits - 1u;
            }
        }
        if (lane == 0) {
            q.bm[u][w] = word;
            q.acc[w] = 0;
            if (word) atomicAdd(q.scan + w / per_blk, (u32)__popc(word));
        }
    }
    TSYNC_B(t);
    if (!compact_from_totals(t, g, q, u)) return false;
    TSYNC_B(t);
    return true;
}

// matching/FilterVertices.cpp:914-966 (pruneCandidates): keep a candidate of
// u only if it is adjacent to a live candidate of every pivot. Only the bitmap
// changes: u's list, rank and count stay those of its generation (a superset
// whose dead entries have their bit clear), which every later filter step
// reads through the bitmap, and the filter's last step compacts each pruned
// vertex once.
template <class Team>
__device__ bool step_prune(Team& t, const DevGraph& g, QState& q, u32 u, u32 pivots) {
    const QDesc* d = q.desc;
    const u32 lane = lane_id(), grp = lane >> 3, lg = lane & 7u;
    const u32 base_u = bucket_base(g, d->label[u]);
    const u32 N = q.cnt[u];
    for (u32 i0 = t.warp() * 4u; i0 < N; i0 += t.nwarps() * 4u) {
        u32 i = i0 + grp;
        u32 v = i < N ? q.list[u][i] : 0;
        const bool live = i < N && test_bit(q.bm[u], v - base_u);  // the list may hold dead entries
        bool alive = live;
        u32 pm = pivots;
        while (pm) {  // warp-uniform loop over pivots
            u32 p = __ffs(pm) - 1;
            pm &= pm - 1;
            const u32 lp = d->label[p], base_p = bucket_base(g, lp);
            u32 s, e;
            group_label_run(g, alive, v, lp, s, e);  // alive is uniform in the group
            u32 len = e - s;
            u32 mx = warp_max(len);
            bool found = false;
            for (u32 j = 0; j < mx; j += 32) {  // 4 loads in flight per lane
                u32 x[4];
#pragma unroll
                for (u32 k = 0; k < 4; ++k) {
                    const u32 o = j + 8u * k + lg;
                    x[k] = o < len ? __ldg(g.nbr + s + o) : 0u;
                }
                bool hit = false;
#pragma unroll
                for (u32 k = 0; k < 4; ++k)
                    if (j + 8u * k + lg < len) hit |= test_bit(q.bm[p], x[k] - base_p);
                u32 bal = __ballot_sync(FULL_MASK, hit);
                if ((bal >> (grp * 8u)) & 0xffu) found = true;
                if (__all_sync(FULL_MASK, found || !alive || j + 32 >= len)) break;
            }
            if (alive && !found) alive = false;
        }
        if (live && !alive && lg == 0) {
            u32 pos = v - base_u;
            atomicAnd(q.bm[u] + (pos >> 5), ~(1u << (pos & 31u)));
        }
    }
    TSYNC_B(t);
    return true;
}

// ------------------------------------------------------------- tables --

__device__ __forceinline__ u32 edge_index(const QDesc* d, u32 x, u32 y) {
    return d->e_first[x] + __popc(d->adj[x] & ((1u << y) - 1u));
}

// Directed edge and row of a global table row index.
__device__ __forceinline__ void row_of(const QState& q, u32 ne, u32 r, u32& e, u32& i) {
    u32 lo = 0, hi = ne;  // largest e with e_row_base[e] <= r
    while (hi - lo > 1) {
        u32 mid = (lo + hi) >> 1;
        if (q.e_row_base[mid] <= r)
            lo = mid;
        else
            hi = mid;
    }
    e = lo;
    i = r - q.e_row_base[lo];
}

__device__ __forceinline__ u32 edge_src(const QDesc* d, u32 e) { return d->e_src[e]; }

// matching/BuildTable.cpp:9-151: row i of T[x][y] lists, ascending, the
// positions in C(y) of the data neighbours of C(x)[i]. Every directed query
// edge's table is built independently (count, team scan, device allocation,
// fill); all tables of a query share one offset array P and one entry array.
template <class Team>
__device__ bool stage_tables(Team& t, const DevGraph& g, QState& q, DevArena* arena) {
    const QDesc* d = q.desc;
    const u32 ne = d->e_first[d->n];
    if (t.warp() == 0) {  // row bases of the directed edges: warp prefix sum
        const u32 lane = lane_id();
        u32 carry = 0;
        for (u32 e0 = 0; e0 < ne; e0 += 32) {
            const u32 e = e0 + lane;
            const u32 v = e < ne ? q.cnt[edge_src(d, e)] : 0u;
            const u32 incl = warp_incl_scan(v);
            if (e < ne) q.e_row_base[e] = carry + incl - v;
            carry += __shfl_sync(FULL_MASK, incl, 31);
        }
        if (lane == 0) {
            q.e_row_base[ne] = carry;
            q.total_rows = carry;
        }
    }
    TSYNC_B(t);
    const u32 R = q.total_rows;
    // Rows go to groups of TW lanes, 32 / TW rows per warp per round.
    constexpr u32 TW = Team::kRowLanes, TG = 32 / TW, TM = (1u << TW) - 1u;
    const u32 lane = lane_id(), grp = lane / TW, lg = lane % TW;
    // count pass
    for (u32 r0 = t.warp() * TG; r0 < R; r0 += t.nwarps() * TG) {
        u32 r = r0 + grp;
        u32 s, e, y = 0, v = 0;
        if (r < R) {
            u32 ei, i;
            row_of(q, ne, r, ei, i);
            u32 x = edge_src(d, ei);
            y = d->e_dst[ei];
            v = q.list[x][i];
        }
        group_label_run<TW>(g, r < R, v, d->label[y], s, e);
        const u32 base_y = r < R ? bucket_base(g, d->label[y]) : 0;
        u32 len = e - s, mx = warp_max(len), c = 0;
        for (u32 j = 0; j < mx; j += 4u * TW) {  // 4 loads in flight per lane
            u32 x[4];
#pragma unroll
            for (u32 k = 0; k < 4; ++k) {
                const u32 o = j + TW * k + lg;
                x[k] = o < len ? __ldg(g.nbr + s + o) : 0u;
            }
#pragma unroll
            for (u32 k = 0; k < 4; ++k) {
                const bool hit = j + TW * k + lg < len && test_bit(q.bm[y], x[k] - base_y);
                c += __popc((__ballot_sync(FULL_MASK, hit) >> (grp * TW)) & TM);
            }
        }
        if (r < R && lg == 0) q.P[r] = c;
    }
    TSYNC_B(t);
    u32* P = q.P;
    // In-place exclusive scan: values are read in pass 1 and pass 2 of
    // team_scan before being overwritten, and every index is written by the
    // warp that owns it only after it read it.
    if (!team_scan(
            t, R, q.scan, [&](u32 i) { return P[i]; }, [&](u32 i, u32 pre) { P[i] = pre; }, &P[R]))
        return false;
    TSYNC_B(t);
    if (t.rank() == 0) {
        u64 nnz = P[R];
        q.table_nnz = nnz;
        unsigned long long at = atomicAdd(&arena->top, (unsigned long long)(nnz + 4));
        if (at + nnz + 4 > arena->cap) {
            q.status = PSM_DEV_OOM;
            q.adj = nullptr;
        } else {
            q.adj = arena->base + at;
        }
    }
    TSYNC_B(t);
    if (q.adj == nullptr) return true;
    // fill pass
    for (u32 r0 = t.warp() * TG; r0 < R; r0 += t.nwarps() * TG) {
        u32 r = r0 + grp;
        u32 s, e, y = 0, v = 0, out = 0;
        if (r < R) {
            u32 ei, i;
            row_of(q, ne, r, ei, i);
            u32 x = edge_src(d, ei);
            y = d->e_dst[ei];
            v = q.list[x][i];
            out = P[r];
        }
        group_label_run<TW>(g, r < R, v, d->label[y], s, e);
        const u32 base_y = r < R ? bucket_base(g, d->label[y]) : 0;
        u32 len = e - s, mx = warp_max(len), written = 0;
        for (u32 j = 0; j < mx; j += 4u * TW) {  // 4 loads in flight per lane, written in row order
            u32 pos[4], word[4];
#pragma unroll
            for (u32 k = 0; k < 4; ++k) {
                const u32 o = j + TW * k + lg;
                pos[k] = o < len ? __ldg(g.nbr + s + o) - base_y : 0u;
            }
#pragma unroll
            for (u32 k = 0; k < 4; ++k) word[k] = j + TW * k + lg < len ? q.bm[y][pos[k] >> 5] : 0u;
#pragma unroll
            for (u32 k = 0; k < 4; ++k) {
                const bool hit = (word[k] >> (pos[k] & 31u)) & 1u;
                const u32 bal = (__ballot_sync(FULL_MASK, hit) >> (grp * TW)) & TM;
                if (hit) {
                    const u32 cpos = q.rank[y][pos[k] >> 5] + __popc(word[k] & ((1u << (pos[k] & 31u)) - 1u));
                    q.adj[out + written + __popc(bal & ((1u << lg) - 1u))] = cpos;
                }
                written += __popc(bal);
            }
        }
    }
    TSYNC_B(t);
    return true;
}

// ------------------------------------------------------------- orders --

__device__ __forceinline__ u32 table_base(const QState& q, u32 a, u32 b) {
    return q.e_row_base[edge_index(q.desc, a, b)];
}

// matching/GenerateQueryPlan.cpp:149-172 + :9-60 (GQL order), one thread.
__device__ void gql_order(const DevGraph& g, QState& q) {
    const QDesc* d = q.desc;
    const u32 n = d->n;
    u32 start = 0;
    for (u32 u = 1; u < n; ++u)
        if (q.cnt[u] < q.cnt[start] || (q.cnt[u] == q.cnt[start] && d->deg[u] > d->deg[start])) start = u;
    u32 vis = 1u << start, adjm = d->adj[start];
    q.order[0] = start;
    for (u32 i = 1; i < n; ++i) {
        u32 nxt = 0;
        u64 best = (u64)g.V + 1;
        for (u32 u = 0; u < n; ++u) {
            if (((vis >> u) & 1u) || !((adjm >> u) & 1u)) continue;
            if (q.cnt[u] < best) {
                best = q.cnt[u];
                nxt = u;
            } else if (q.cnt[u] == best && d->deg[u] > d->deg[nxt]) {
                nxt = u;
            }
        }
        q.order[i] = nxt;
        vis |= 1u << nxt;
        adjm |= d->adj[nxt];
    }
    q.pivot[0] = 0;
    for (u32 i = 1; i < n; ++i)
        for (u32 j = 0; j < i; ++j)
            if ((d->adj[q.order[i]] >> q.order[j]) & 1u) {
                q.pivot[i] = q.order[j];
                break;
            }
}

// matching/GenerateQueryPlan.cpp:680-721 estimatePathEmbeddsingsNum for one
// path, by one thread block: est[k-2] = entries of the last table; walking
// back, a row's estimate is the sum of the estimates of its entries.
__device__ void estimate_path_block(QState& q, const u32* path, u32 k, u64* est, u64* child, u64* par) {
    {
        const u32 a = path[k - 2], b = path[k - 1];
        const u32 rb = table_base(q, a, b), rows = q.cnt[a];
        u64 s = 0;
        for (u32 i = threadIdx.x; i < rows; i += blockDim.x) {
            u64 c = q.P[rb + i + 1] - q.P[rb + i];
            child[i] = c;
            s += c;
        }
        s = warp_sum64(s);
        if (lane_id() == 0 && s) atomicAdd((unsigned long long*)&est[k - 2], (unsigned long long)s);
    }
    __syncthreads();
    for (int i = (int)k - 2; i >= 1; --i) {
        const u32 a = path[i - 1], b = path[i];
        const u32 rb = table_base(q, a, b), rows = q.cnt[a];
        u64 s = 0;
        for (u32 j = threadIdx.x; j < rows; j += blockDim.x) {
            u64 ls = 0;
            for (u32 e = q.P[rb + j]; e < q.P[rb + j + 1]; ++e) ls += child[q.adj[e]];
            par[j] = ls;
            s += ls;
        }
        s = warp_sum64(s);
        if (lane_id() == 0 && s) atomicAdd((unsigned long long*)&est[i - 1], (unsigned long long)s);
        __syncthreads();
        u64* tmp = child;
        child = par;
        par = tmp;
    }
}

// Estimates of all paths of the chosen CFL order plan; entry k of path p is
// est_out[path_off[p] - p + k] (a path of length l has l - 1 estimates).
// Paths are independent: with several blocks each block takes its own paths
// (its own child / parent buffers), so the whole step costs one team barrier.
template <class Team>
__device__ bool cfl_estimates(Team& t, QState& q, const u32* pw) {
    const QDesc* d = q.desc;
    const u32 n = d->n;
    const u32 ncore = pw[1 + 2 * n];
    const u32 ngroups = pw[2 + 2 * n];
    const u32* gfirst = pw + 3 + 2 * n;
    const u32 npaths = gfirst[ngroups + 1];
    const u32* poff = gfirst + ngroups + 2;
    const u32* pv = poff + npaths + 1 + ncore;
    for (u32 i = t.rank(); i < PSM_PLAN_WORDS; i += t.size()) q.est_out[i] = 0;
    TSYNC_B(t);
    const u32 eb = min(t.nblocks(), q.est_blocks);
    if (t.block() < eb) {
        u64* child = q.est_a + (size_t)t.block() * 2 * q.est_stride;
        u64* par = child + q.est_stride;
        for (u32 p = t.block(); p < npaths; p += eb)
            estimate_path_block(q, pv + poff[p], poff[p + 1] - poff[p], q.est_out + (poff[p] - p), child, par);
    }
    TSYNC_B(t);
    return true;
}

// matching/GenerateQueryPlan.cpp:270-471 generateCFLQueryPlan greedy
// selection (core paths, tree paths per forest, leaves), one thread. Ties
// keep the first minimum, as the reference's strict "<" does.
__device__ void cfl_order_select(QState& q, const u32* pw) {
    const QDesc* d = q.desc;
    const u32 n = d->n;
    const u32 root = pw[0];
    const u32* parent = pw + 1;
    const u32 ncore = pw[1 + 2 * n];
    const u32 ngroups = pw[1 + 2 * n + 1];
    const u32* gfirst = pw + 1 + 2 * n + 2;
    const u32 npaths = gfirst[ngroups + 1];
    const u32* poff = gfirst + ngroups + 2;
    const u32* nte = poff + npaths + 1;
    const u32* pv = nte + ncore;
    const u32 nleaves = pv[poff[npaths]];
    const u32* leaves = pv + poff[npaths] + 1;
    const double DMAX = 1.79769313486231570815e308;
    auto est = [&](u32 p, u32 k) { return q.est_out[poff[p] - p + k]; };
    auto path_v = [&](u32 p, u32 k) { return pv[poff[p] + k]; };
    auto plen = [&](u32 p) { return poff[p + 1] - poff[p]; };
    u32 vis = 1u << root;
    u32 cnt = 0;
    q.order[cnt] = root;
    q.pivot[cnt] = 0;
    ++cnt;
    u64 alive = 0;  // remaining paths of the current family (bitmask over <= 64)
    if (ncore > 0) {
        double mn = DMAX;
        u32 sel = 0;
        for (u32 i = 0; i < ncore; ++i) {
            double v = (double)est(i, 0) / (double)nte[i];
            if (v < mn) mn = v, sel = i;
        }
        for (u32 k = 1; k < plen(sel); ++k) {
            q.order[cnt] = path_v(sel, k);
            q.pivot[cnt] = path_v(sel, k - 1);
            ++cnt;
            vis |= 1u << path_v(sel, k);
        }
        alive = (ncore >= 64 ? ~0ull : ((1ull << ncore) - 1)) & ~(1ull << sel);
        while (alive) {
            mn = DMAX;
            sel = 0xFFFFFFFFu;
            for (u32 i = 0; i < ncore; ++i) {
                if (!((alive >> i) & 1ull)) continue;
                if (sel == 0xFFFFFFFFu) sel = i;  // reference starts from index 0 of the remaining list
                u32 ri = 0;
                for (u32 j = 0; j < plen(i); ++j) {
                    if ((vis >> path_v(i, j)) & 1u) continue;
                    ri = j - 1;
                    break;
                }
                double v = (double)est(i, ri) / (double)q.cnt[path_v(i, ri)];
                if (v < mn) mn = v, sel = i;
            }
            for (u32 k = 1; k < plen(sel); ++k) {
                u32 x = path_v(sel, k);
                if ((vis >> x) & 1u) continue;
                q.order[cnt] = x;
                q.pivot[cnt] = path_v(sel, k - 1);
                ++cnt;
                vis |= 1u << x;
            }
            alive &= ~(1ull << sel);
        }
    }
    for (u32 gi = 0; gi < ngroups; ++gi) {
        const u32 p0 = gfirst[gi], p1 = gfirst[gi + 1];
        alive = (p1 - p0 >= 64) ? ~0ull : ((1ull << (p1 - p0)) - 1);
        while (alive) {
            double mn = DMAX;
            u32 sel = 0xFFFFFFFFu;
            for (u32 i = p0; i < p1; ++i) {
                if (!((alive >> (i - p0)) & 1ull)) continue;
                if (sel == 0xFFFFFFFFu) sel = i;
                u32 ri = 0;
                for (u32 j = 0; j < plen(i); ++j) {
                    if ((vis >> path_v(i, j)) & 1u) continue;
                    ri = j == 0 ? j : j - 1;
                    break;
                }
                double v = (double)est(i, ri) / (double)q.cnt[path_v(i, ri)];
                if (v < mn) mn = v, sel = i;
            }
            for (u32 k = 0; k < plen(sel); ++k) {
                u32 x = path_v(sel, k);
                if ((vis >> x) & 1u) continue;
                q.order[cnt] = x;
                q.pivot[cnt] = k ? path_v(sel, k - 1) : 0;
                ++cnt;
                vis |= 1u << x;
            }
            alive &= ~(1ull << (sel - p0));
        }
    }
    u32 lalive = nleaves >= 32 ? ~0u : ((1u << nleaves) - 1u);
    while (lalive) {
        double mn = DMAX;
        u32 sel = 0xFFFFFFFFu;
        for (u32 i = 0; i < nleaves; ++i) {
            if (!((lalive >> i) & 1u)) continue;
            if (sel == 0xFFFFFFFFu) sel = i;
            double v = (double)q.cnt[leaves[i]];
            if (v < mn) mn = v, sel = i;
        }
        u32 l = leaves[sel];
        if (!((vis >> l) & 1u)) {
            q.order[cnt] = l;
            q.pivot[cnt] = parent[l];
            ++cnt;
            vis |= 1u << l;
        }
        lalive &= ~(1u << sel);
    }
    if (cnt != n) q.status = PSM_DEV_INTERNAL;
}

// Backward neighbours by depth (matching/EvaluateQuery.cpp:1594-1625: all
// earlier neighbours, in query-vertex id order), their table rows, the
// earlier depths sharing the label (only those can collide on a data
// vertex), and computeMemoryCostInBytes (BuildTable.cpp:300-326). One warp:
// lane i handles depth i; all loops are warp-uniform.
__device__ void enum_plan_warp(const DevGraph& g, QState& q) {
    const QDesc* d = q.desc;
    const u32 nv = d->n;       // query vertices
    const u32 n = q.n_enum;    // depths (n_enum < nv for a decomposition unit)
    const u32 lane = lane_id();
    const bool act = lane < n;
    const u32 u = act ? q.order[lane] : 0u;          // vertex at depth lane
    const u32 lab = act ? d->label[u] : 0xFFFFFFFFu;  // its label
    u32 depth_of = 0;                                 // depth of vertex `lane` (if ordered)
    for (u32 j = 0; j < n; ++j)
        if (__shfl_sync(FULL_MASK, u, j) == lane) depth_of = j;
    u32 seen_incl = act ? (1u << u) : 0u;  // vertices at depths <= lane
    for (u32 o = 1; o < 32; o <<= 1) {
        u32 y = __shfl_up_sync(FULL_MASK, seen_incl, o);
        if (lane >= o) seen_incl |= y;
    }
    const u32 seen = seen_incl & ~(act ? (1u << u) : 0u);
    const u32 m = act ? (d->adj[u] & seen) : 0u;
    u32 k = 0, same = 0;
    for (u32 b = 0; b < nv; ++b) {  // b: query vertex
        const u32 db = __shfl_sync(FULL_MASK, depth_of, b);
        if ((m >> b) & 1u) {
            q.bn_depth[lane][k] = db;
            q.bn_tab[lane][k] = table_base(q, b, u);
            ++k;
        }
    }
    for (u32 b = 0; b < n; ++b) {  // b: depth
        const u32 lb = __shfl_sync(FULL_MASK, lab, b);
        if (b < lane && lb == lab) same |= 1u << b;
    }
    // prefix-intersection cache plan (the bn rows of this lane's depth are in
    // bn_depth[lane][0, k), written by this lane above)
    u32 cm = 0, crow = 0xFFFFFFFFu, cdep = 0;
    for (u32 j = 0; j < k; ++j) {
        const u32 bd = q.bn_depth[lane][j];
        if (bd + 2 <= lane) {
            cm |= 1u << j;
            cdep = max(cdep, bd);
        } else {
            crow = j;  // bd == lane - 1
        }
    }
    const bool bm_ok = act && q.cnt[u] <= PSM_CACHE_BM_BITS;
    const u32 bm_depths = __ballot_sync(FULL_MASK, bm_ok);
    const u32 cm_all = cm;
    // one shallow row is worth caching only as a bitmap tested against the
    // depth-(d-1) row
    if (__popc(cm) < 2 && !(__popc(cm) == 1 && crow != 0xFFFFFFFFu && bm_ok)) cm = 0;
    // last-two-depth weight memo (see QState::memo_ok): depth n-1 has a cache
    // and a row at depth n-2; depth n-2 has rows at depths <= n-4 only, all
    // kept in its cache (even a single one) with a bitmap
    const u32 last = n >= 3 ? n - 1 : 0u;
    const u32 cm_l = __shfl_sync(FULL_MASK, cm, last), crow_l = __shfl_sync(FULL_MASK, crow, last);
    const u32 cnt_l = __shfl_sync(FULL_MASK, act ? q.cnt[u] : 0u, last);
    const u32 u_l = __shfl_sync(FULL_MASK, u, last);
    // (the memo's exclusions assume a vertex is never its own neighbour)
    const bool memo = !g.loops && n >= 3 && lane + 2 == n && crow == 0xFFFFFFFFu && cm_all != 0 && bm_ok &&
                      cm_l != 0 && crow_l != 0xFFFFFFFFu && cnt_l <= PSM_MEMO_CAP;
    if (memo) cm = cm_all;
    const u32 memo_any = __ballot_sync(FULL_MASK, memo);
    u32 inval = 0;
    for (u32 x = 0; x < n; ++x) {
        const u32 bal = __ballot_sync(FULL_MASK, act && cm != 0 && cdep >= x);
        if (lane == x) inval = bal;
    }
    if (lane < nv) q.cbase[lane] = bucket_base(g, d->label[lane]);  // by query vertex
    if (act) {
        q.nbn[lane] = k;
        q.same_mask[lane] = same;
        q.cmask[lane] = cm;
        q.crow[lane] = crow;
        q.cinval[lane] = inval;
    }
    if (lane == 0) {
        q.bm_depths = bm_depths;
        q.memo_ok = memo_any ? 1u : 0u;
        q.loops = g.loops;
    }
    if (memo) q.memo_tab = table_base(q, u_l, u);
    // memory cost: candidates of every vertex, both tables of every edge
    // (the query's; a unit keeps the value it was given)
    u64 mem = 0;
    if (lane < nv && n == nv) {
        const u32 a = lane;
        mem += (u64)q.cnt[a] * 4u;
        u32 mb = d->adj[a] & ~((2u << a) - 1u);  // neighbours b > a
        while (mb) {
            const u32 b = __ffs(mb) - 1;
            mb &= mb - 1;
            const u32 ab = table_base(q, a, b), ba = table_base(q, b, a);
            const u64 nab = q.P[ab + q.cnt[a]] - q.P[ab], nba = q.P[ba + q.cnt[b]] - q.P[ba];
            mem += (nab + q.cnt[a] + nba + q.cnt[b]) * 4u;
        }
    }
    mem = warp_sum64(mem);
    if (lane == 0) {
        if (n == nv) q.memory_bytes = mem;
        q.root_cnt = q.empty ? 0u : q.cnt[q.order[0]];
    }
}

// ------------------------------------------------------------ driver --

// ------------------------------------------------------------ driver --
//
// The preparation of a query is a fixed list of steps, each ending with a
// team barrier:
//   0 clear, 1 NLF, 2 pick start vertices,
//   GQL / NLF filter: compact every u, empty check, [GQL: refine (round, u)
//     for 2n steps, compact every u],
//   CFL filter: compact the start vertex, the plan's generate / prune steps,
//   then: empty check, tables, order, enumeration plan.
// run_step executes one step with any team; the drivers below choose teams.

__device__ __forceinline__ bool is_cfl(const QDesc* d) { return d->filter == PSM_FILTER_CFL; }

// Number of steps (valid once step 2 has picked the CFL start vertex).
__device__ u32 step_count(const QState& q) {
    const QDesc* d = q.desc;
    const u32 n = d->n;
    u32 mid;
    if (is_cfl(d))
        mid = 1 + d->fplan[q.froot].nsteps;
    else
        mid = n + 1 + (d->filter == PSM_FILTER_GQL ? 3 * n : 0);
    return 3 + mid + 4;
}

template <class Team>
__device__ bool run_step(Team& t, const DevGraph& g, QState& q, DevArena* arena, u32 k) {
    const QDesc* d = q.desc;
    const u32 n = d->n;
    const bool cfl = is_cfl(d);
    if (k == 0) {  // clear bitmaps and counters
        for (u32 u = 0; u < n; ++u)
            for (u32 i = t.rank(); i < q.bwords[u]; i += t.size()) q.bm[u][i] = 0;
        if (cfl)
            for (u32 i = t.rank(); i < q.acc_words; i += t.size()) {
                q.acc[i] = 0;
                q.tmp[i] = 0;
            }
        if (t.rank() == 0) {
            for (u32 i = 0; i < PSM_MAXQ + PSM_MAXOPT; ++i) q.item_cnt[i] = 0;
            q.empty = 0;
            q.filter_ok = 1;
            q.count = 0;
            q.calls = 0;
            q.alg_bytes = 0;
            q.stop = 0;
            q.overtime = 0;
            q.emit_rows = 0;
            q.n_enum = d->n;
            q.table_nnz = 0;
            q.memory_bytes = 0;
            q.root_cnt = 0;
            q.status = PSM_DEV_OK;
        }
        TSYNC_B(t);
        return true;
    }
    if (k == 1) {  // NLF candidates of the needed items
        // CFL needs the NLF sets of its start options only. A team of >= 1024
        // warps computes every vertex's set here, in one wide pass, and the
        // generate steps then test a bit instead of walking NLF label runs
        // (the sets are the same either way).
        u32 need = n >= 32 ? ~0u : ((1u << n) - 1u);
        const bool all = !cfl || t.nwarps() >= 1024u;
        if (!all) {
            need = 0;
            for (u32 j = 0; j < d->nfopt; ++j) need |= 1u << d->fopt_vertex[j];
        }
        stage_nlf(t, g, q, need, d->order == PSM_ORDER_CFL);
        if (t.rank() == 0) q.nlf_all = all;
        TSYNC_B(t);
        return true;
    }
    if (k == 2) {  // start vertices of the CFL filter plan and of the CFL order
        if (t.rank() == 0) {
            // matching/GenerateFilteringPlan.cpp:343-385: lowest count/degree
            // among the kept options, first one on ties.
            if (cfl) {
                double best = (double)d->fopt_max_score_num;
                u32 pick = 0;
                for (u32 j = 0; j < d->nfopt; ++j) {
                    u32 u = d->fopt_vertex[j];
                    double s = (double)q.item_cnt[u] / (double)d->deg[u];
                    if (s < best) best = s, pick = j;
                }
                q.froot = pick;
            }
            if (d->order == PSM_ORDER_CFL) {
                double best = (double)d->fopt_max_score_num;
                u32 pick = 0;
                for (u32 j = 0; j < d->noopt; ++j) {
                    u32 u = d->oopt_vertex[j];
                    double s = (double)q.item_cnt[d->oopt_item[j]] / (double)d->deg[u];
                    if (s < best) best = s, pick = j;
                }
                q.oroot = pick;
            }
        }
        TSYNC_B(t);
        return true;
    }
    u32 j = k - 3;
    if (!cfl) {
        if (j < n) {  // compact u (NLF result)
            if (!compact_vertex(t, g, q, j)) return false;
            TSYNC_B(t);
            return true;
        }
        j -= n;
        if (j == 0) {  // NLFFilter / GQLFilter stop at the first empty set
            if (t.rank() == 0) {
                for (u32 u = 0; u < n; ++u)
                    if (q.cnt[u] == 0) {
                        q.empty = 1;
                        q.filter_ok = 0;
                        for (u32 v = u + 1; v < n; ++v) q.cnt[v] = 0;
                        break;
                    }
            }
            TSYNC_B(t);
            return true;
        }
        j -= 1;
        if (d->filter == PSM_FILTER_GQL) {
            if (j < 2 * n) {  // refine (round j / n) of u = j % n
                const u32 u = j % n;
                if (!q.empty) {
                    const u32 base = bucket_base(g, d->label[u]);
                    const u32 N = q.cnt[u];
                    for (u32 i = t.warp(); i < N; i += t.nwarps()) {
                        u32 v = q.list[u][i];
                        u32 pos = v - base;
                        if (!test_bit(q.bm[u], pos)) continue;
                        if (!gql_check(g, d, q, u, v) && lane_id() == 0)
                            atomicAnd(q.bm[u] + (pos >> 5), ~(1u << (pos & 31u)));
                    }
                }
                TSYNC_B(t);
                return true;
            }
            j -= 2 * n;
            if (j < n) {
                if (!q.empty && !compact_vertex(t, g, q, j)) return false;
                TSYNC_B(t);
                return true;
            }
            j -= n;
        }
    } else {
        const FilterPlan& fp = d->fplan[q.froot];
        if (j == 0) {
            if (!compact_vertex(t, g, q, fp.root)) return false;
            TSYNC_B(t);
            return true;
        }
        j -= 1;
        if (j < fp.nsteps)
            return fp.step_kind[j] == STEP_GEN ? step_generate(t, g, q, fp.step_u[j], fp.step_mask[j])
                                               : step_prune(t, g, q, fp.step_u[j], fp.step_mask[j]);
        j -= fp.nsteps;
    }
    // tail: empty check, tables, order, enumeration plan
    if (j == 0) {
        if (cfl) {  // lists of pruned vertices to their final sets
            const FilterPlan& fp = d->fplan[q.froot];
            u32 dirty = 0;
            for (u32 s = 0; s < fp.nsteps; ++s)
                if (fp.step_kind[s] == STEP_PRUNE) dirty |= 1u << fp.step_u[s];
            if (dirty) {
                if (!multi_compact(t, g, q, dirty)) return false;
                TSYNC_B(t);  // the check below reads cnt
            }
        }
        if (t.rank() == 0)
            for (u32 u = 0; u < n; ++u)
                if (q.cnt[u] == 0) q.empty = 1;
        TSYNC_B(t);
        return true;
    }
    const bool skip = !q.filter_ok;  // GQL / NLF early exit: nothing more is built
    if (j == 1) {
        if (!skip && !stage_tables(t, g, q, arena)) return false;
        TSYNC_B(t);
        return true;
    }
    if (j == 2) {
        if (!skip && q.adj != nullptr) {
            if (d->order == PSM_ORDER_CFL) {
                const u32* pw = d->plan_words + d->oplan_off[q.oroot];
                if (!cfl_estimates(t, q, pw)) return false;
                TSYNC_B(t);
                if (t.rank() == 0) cfl_order_select(q, pw);
            } else if (t.rank() == 0) {
                gql_order(g, q);
            }
        }
        TSYNC_B(t);
        return true;
    }
    if (t.warp() == 0 && !skip && q.adj != nullptr) enum_plan_warp(g, q);
    TSYNC_B(t);
    return true;
}

// Whether step k is small enough for one block (decided on current counts).
__device__ bool step_small(const DevGraph& g, const QState& q, u32 k) {
    constexpr u32 SMALL_ITEMS = 4096;   // candidates / rows handled by one block
    constexpr u32 SMALL_WORDS = 2048;   // bitmap words handled by one block
    const QDesc* d = q.desc;
    const u32 n = d->n;
    if (k == 1) {
        u32 words = 0;
        for (u32 it = 0; it < n + d->nvirt; ++it) words += (bucket_size(g, d->item_label[it]) + 31u) >> 5;
        return words <= SMALL_WORDS;
    }
    if (k == 0 || k == 2) {
        u32 words = 0;
        for (u32 u = 0; u < n; ++u) words += q.bwords[u];
        return k == 2 || words <= 4 * SMALL_WORDS;
    }
    u32 j = k - 3;
    if (!is_cfl(d)) {
        if (j < n) return q.bwords[j] <= SMALL_WORDS;
        j -= n;
        if (j == 0) return true;
        j -= 1;
        if (d->filter == PSM_FILTER_GQL) {
            if (j < 2 * n) return q.cnt[j % n] <= SMALL_ITEMS / 8;
            j -= 2 * n;
            if (j < n) return q.bwords[j] <= SMALL_WORDS;
            j -= n;
        }
    } else {
        const FilterPlan& fp = d->fplan[q.froot];
        if (j == 0) return q.bwords[fp.root] <= SMALL_WORDS;
        j -= 1;
        if (j < fp.nsteps) {
            const u32 u = fp.step_u[j];
            if (q.bwords[u] > SMALL_WORDS) return false;
            if (fp.step_kind[j] == STEP_PRUNE) return q.cnt[u] <= SMALL_ITEMS;
            u32 work = 0, m = fp.step_mask[j];
            while (m) {
                work += q.cnt[__ffs(m) - 1];
                m &= m - 1;
            }
            return work <= SMALL_ITEMS;
        }
        j -= fp.nsteps;
    }
    if (j == 1) {  // tables: all rows of all directed edges
        u32 rows = 0;
        for (u32 x = 0; x < n; ++x) rows += q.cnt[x] * (d->e_first[x + 1] - d->e_first[x]);
        return rows <= SMALL_ITEMS;
    }
    if (j == 2) {
        u32 rows = 0;
        for (u32 x = 0; x < n; ++x) rows += q.cnt[x];
        return rows <= 4 * SMALL_ITEMS;
    }
    return true;
}

__device__ __forceinline__ void trace_step(QState& q, u32 k) {
    if (q.trace && k < PSM_TRACE_STEPS) q.trace[k] = global_timer_ns();
}

template <class Team>
__device__ void prepare_query(Team& t, const DevGraph& g, QState& q, DevArena* arena) {
    if (t.rank() == 0 && q.trace) q.trace[PSM_TRACE_STEPS] = global_timer_ns();
    for (u32 k = 0; k < step_count(q); ++k) {
        if (!run_step(t, g, q, arena, k)) return;
        if (t.rank() == 0) trace_step(q, k);
    }
}

// Plain path with the whole grid: block 0 runs consecutive small steps on
// its own (block barriers only); the grid joins for large steps. The other
// blocks wait at one grid barrier per run of small steps.
__device__ void prepare_query_hybrid(GridTeam& gt, const DevGraph& g, QState& q, DevArena* arena) {
    __shared__ u32 s_k;
    u32 k = 0;
    if (gt.rank() == 0 && q.trace) q.trace[PSM_TRACE_STEPS] = global_timer_ns();
    while (true) {
        if (blockIdx.x == 0) {
            BlockTeam bt;
            // Steps 0 and 1 (before the start vertex is picked) always
            // qualify by size alone.
            while (k < (k < 3 ? 3u : step_count(q)) && step_small(g, q, k)) {
                if (!run_step(bt, g, q, arena, k)) break;
                if (threadIdx.x == 0) trace_step(q, k);
                ++k;
            }
            if (threadIdx.x == 0) q.step_cursor = k;
        }
        if (!gt.sync()) return;
        if (threadIdx.x == 0) s_k = ld_volatile_u32(&q.step_cursor);
        __syncthreads();
        k = s_k;
        if (k >= 3 && k >= step_count(q)) break;
        if (!run_step(gt, g, q, arena, k)) return;
        if (gt.rank() == 0) trace_step(q, k);
        ++k;
    }
}

// Batched / serving preparation: blocks take queries from a ticket counter.
__global__ void __launch_bounds__(512) prep_block_kernel(DevGraph g, QState* qs, u32 nq, u32* ticket,
                                                         DevArena* arena) {
    __shared__ u32 s_q;
    BlockTeam t;
    while (true) {
        if (threadIdx.x == 0) s_q = atomicAdd(ticket, 1u);
        __syncthreads();
        u32 qi = s_q;
        __syncthreads();
        if (qi >= nq) break;
        prepare_query(t, g, qs[qi], arena);
        __syncthreads();
    }
}

// Batched path with cluster teams: each thread-block cluster takes the next
// query from a ticket (read by block 0, handed to the others through
// distributed shared memory) and prepares it with all of its blocks.
__global__ void __launch_bounds__(512) prep_cluster_batch_kernel(DevGraph g, QState* qs, u32 nq, u32* ticket,
                                                                 DevArena* arena) {
    __shared__ u32 s_q;
    ClusterTeam t;
    cg::cluster_group cl = cg::this_cluster();
    while (true) {
        if (cl.block_rank() == 0 && threadIdx.x == 0) s_q = atomicAdd(ticket, 1u);
        cl.sync();
        const u32 qi = *cl.map_shared_rank(&s_q, 0);
        cl.sync();  // every block has read it before block 0 takes the next
        if (qi >= nq) break;
        prepare_query(t, g, qs[qi], arena);
    }
}

// Plain path: one query prepared by one thread-block cluster.
__global__ void __launch_bounds__(512) prep_cluster_kernel(DevGraph g, QState* qs, DevArena* arena) {
    ClusterTeam t;
    prepare_query(t, g, qs[0], arena);
}

// Plain path: one query prepared by the whole (co-resident) grid.
__global__ void __launch_bounds__(512, 1) prep_grid_kernel(DevGraph g, QState* qs, GridBarrier* bar, DevArena* arena,
                                                        u64 budget_ns) {
    GridTeam t{bar, global_timer_ns() + budget_ns};
    if (qs[0].step_cursor == HYBRID_REQUEST)
        prepare_query_hybrid(t, g, qs[0], arena);
    else
        prepare_query(t, g, qs[0], arena);
}

}  // namespace

// Host launchers ----------------------------------------------------------

cudaError_t psm_launch_prep_block(const DevGraph& g, QState* qs, u32 nq, u32* ticket, DevArena* arena, int blocks,
                                  int threads, cudaStream_t st) {
    prep_block_kernel<<<blocks, threads, 0, st>>>(g, qs, nq, ticket, arena);
    return cudaGetLastError();
}

cudaError_t psm_launch_prep_grid(const DevGraph& g, QState* qs, void* barrier, DevArena* arena, u64 budget_ns,
                                 int blocks, int threads, cudaStream_t st) {
    GridBarrier* bar = (GridBarrier*)barrier;
    void* args[] = {(void*)&g, (void*)&qs, (void*)&bar, (void*)&arena, (void*)&budget_ns};
    return cudaLaunchCooperativeKernel((const void*)prep_grid_kernel, dim3(blocks), dim3(threads), args, 0, st);
}

// Largest supported cluster size (<= want) for the cluster preparation kernel.
cudaError_t psm_prep_cluster_size(int threads, int want, int* size) {
    cudaError_t e = cudaFuncSetAttribute(prep_cluster_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
    for (int cs = want; cs >= 1; cs >>= 1) {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = cs;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(cs);
        cfg.blockDim = dim3(threads);
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int clusters = 0;
        e = cudaOccupancyMaxActiveClusters(&clusters, prep_cluster_kernel, &cfg);
        if (e == cudaSuccess && clusters > 0) {
            *size = cs;
            return cudaSuccess;
        }
        cudaGetLastError();
    }
    *size = 1;
    return cudaSuccess;
}

cudaError_t psm_launch_prep_cluster(const DevGraph& g, QState* qs, DevArena* arena, int cluster, int threads,
                                    cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(cluster);
    cfg.blockDim = dim3(threads);
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, prep_cluster_kernel, g, qs, arena);
}

// Clusters of `cluster` blocks that fit the GPU at once for the batched
// cluster preparation kernel (0 if that cluster size cannot run).
cudaError_t psm_prep_cluster_batch_clusters(int threads, int cluster, int* clusters) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(cluster);
    cfg.blockDim = dim3(threads);
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    *clusters = 0;
    cudaError_t e = cudaOccupancyMaxActiveClusters(clusters, prep_cluster_batch_kernel, &cfg);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *clusters = 0;
    }
    return cudaSuccess;
}

cudaError_t psm_launch_prep_cluster_batch(const DevGraph& g, QState* qs, u32 nq, u32* ticket, DevArena* arena,
                                          int cluster, int clusters, int threads, cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(cluster * clusters);
    cfg.blockDim = dim3(threads);
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, prep_cluster_batch_kernel, g, qs, nq, ticket, arena);
}

cudaError_t psm_prep_grid_max_blocks(int threads, int* blocks) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, prep_grid_kernel, threads, 0);
    if (e != cudaSuccess) return e;
    *blocks = sms * (per_sm < 1 ? 1 : per_sm);
    return cudaSuccess;
}

// ------------------------------------------------------ decomposition units --
//
// A decomposition unit is enumerated on a copy of its query's QState whose
// order lists only the unit's vertices (n_enum of them); the unit reuses the
// query's candidate sets and tables. These kernels recompute the enumeration
// plan of such copies and arm their emission buffers.

namespace {

__global__ void unit_plan_kernel(DevGraph g, QState* qs, u32 nq) {
    if (blockIdx.x < nq && threadIdx.x < 32) enum_plan_warp(g, qs[blockIdx.x]);
}

__global__ void unit_emit_kernel(QState* qs, u32 nq, u32* const* bufs, const u64* caps) {
    for (u32 i = threadIdx.x; i < nq; i += blockDim.x) {
        QState& q = qs[i];
        q.emit_buf = bufs[i];
        q.emit_cap_rows = caps[i];
        q.emit_rows = 0;
        q.emit_by_depth = 1;
        q.count = 0;
        q.calls = 0;
        q.alg_bytes = 0;
        q.stop = 0;
        q.overtime = 0;
        q.done_ns = 0;
    }
}

}  // namespace

cudaError_t psm_launch_unit_plan(const DevGraph& g, QState* qs, u32 nq, cudaStream_t st) {
    unit_plan_kernel<<<nq, 32, 0, st>>>(g, qs, nq);
    return cudaGetLastError();
}

cudaError_t psm_launch_unit_emit(QState* qs, u32 nq, u32* const* bufs, const u64* caps, cudaStream_t st) {
    unit_emit_kernel<<<1, 256, 0, st>>>(qs, nq, bufs, caps);
    return cudaGetLastError();
}
