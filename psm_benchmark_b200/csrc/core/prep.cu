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
#include <cuda_runtime.h>

#include "device_util.cuh"
#include "psm_internal.h"

namespace {

// ---------------------------------------------------------------- teams --

struct BlockTeam {
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
    u32 count;
    u32 gen;
    u32 abort;
    u32 pad;
};

// Whole-grid team for a cooperative launch (all blocks co-resident). The
// barrier spins with a bounded wait: past the deadline or the iteration cap
// it raises `abort`, every later barrier returns false at once and the
// kernel unwinds; the host reports an internal error.
struct GridTeam {
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
                __threadfence();
                u32 g = ld_acquire_u32(&bar->gen);
                u32 arrived = atomicAdd(&bar->count, 1u);
                if (arrived == gridDim.x - 1) {
                    atomicExch(&bar->count, 0u);
                    __threadfence();
                    atomicAdd(&bar->gen, 1u);
                } else {
                    u32 it = 0;
                    while (ld_acquire_u32(&bar->gen) == g) {
                        if (ld_acquire_u32(&bar->abort)) break;
                        if ((++it & 1023u) == 0 && global_timer_ns() > deadline_ns) {
                            atomicExch(&bar->abort, 1u);
                            break;
                        }
                        if (it > (1u << 30)) {
                            atomicExch(&bar->abort, 1u);
                            break;
                        }
                        __nanosleep(64);
                    }
                }
                __threadfence();
                ab = ld_acquire_u32(&bar->abort);
            }
            s_abort = ab;
        }
        __syncthreads();
        return s_abort == 0;
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
        u32 s = 0, e = 0;
        if (i < N) {
            u32 c = q.list[p][i];
            if (test_bit(q.bm[p], c - base_p)) label_run(g, c, lu, s, e);
        }
        u32 len = e - s;
        u32 mx = warp_max(len);
        for (u32 j = 0; j < mx; j += 8) {
            if (j + lg < len) {
                u32 pos = __ldg(g.nbr + s + j + lg) - base_u;
                atomicOr(out + (pos >> 5), 1u << (pos & 31u));
            }
        }
    }
    return true;
}

template <class Team>
__device__ bool step_generate(Team& t, const DevGraph& g, QState& q, u32 u, u32 pivots) {
    const QDesc* d = q.desc;
    const u32 lu = d->label[u];
    const u32 W = q.bwords[u];
    for (u32 i = t.rank(); i < W; i += t.size()) q.acc[i] = 0;
    TSYNC_B(t);
    bool first = true;
    u32 pm = pivots;
    while (pm) {
        u32 p = __ffs(pm) - 1;
        pm &= pm - 1;
        if (first) {
            mark_neighbours(t, g, q, p, lu, q.acc);
            TSYNC_B(t);
        } else {
            for (u32 i = t.rank(); i < W; i += t.size()) q.tmp[i] = 0;
            TSYNC_B(t);
            mark_neighbours(t, g, q, p, lu, q.tmp);
            TSYNC_B(t);
            for (u32 i = t.rank(); i < W; i += t.size()) q.acc[i] &= q.tmp[i];
            TSYNC_B(t);
        }
        first = false;
    }
    const u32 lane = lane_id();
    const u32 base = bucket_base(g, lu), bsz = bucket_size(g, lu);
    for (u32 w = t.warp(); w < W; w += t.nwarps()) {
        u32 pos = 32u * w + lane;
        bool ok = pos < bsz && ((q.acc[w] >> lane) & 1u) && nlf_ok(g, d, u, base + pos);
        u32 word = __ballot_sync(FULL_MASK, ok);
        if (lane == 0) q.bm[u][w] = word;
    }
    TSYNC_B(t);
    if (!compact_vertex(t, g, q, u)) return false;
    TSYNC_B(t);
    return true;
}

// matching/FilterVertices.cpp:914-966 (pruneCandidates): keep a candidate of
// u only if it is adjacent to a live candidate of every pivot.
template <class Team>
__device__ bool step_prune(Team& t, const DevGraph& g, QState& q, u32 u, u32 pivots) {
    const QDesc* d = q.desc;
    const u32 lane = lane_id(), grp = lane >> 3, lg = lane & 7u;
    const u32 base_u = bucket_base(g, d->label[u]);
    const u32 N = q.cnt[u];
    for (u32 i0 = t.warp() * 4u; i0 < N; i0 += t.nwarps() * 4u) {
        u32 i = i0 + grp;
        u32 v = i < N ? q.list[u][i] : 0;
        bool alive = i < N;
        u32 pm = pivots;
        while (pm) {  // warp-uniform loop over pivots
            u32 p = __ffs(pm) - 1;
            pm &= pm - 1;
            const u32 lp = d->label[p], base_p = bucket_base(g, lp);
            u32 s = 0, e = 0;
            if (alive) label_run(g, v, lp, s, e);
            u32 len = e - s;
            u32 mx = warp_max(len);
            bool found = false;
            for (u32 j = 0; j < mx; j += 8) {
                bool hit = false;
                if (j + lg < len) hit = test_bit(q.bm[p], __ldg(g.nbr + s + j + lg) - base_p);
                u32 bal = __ballot_sync(FULL_MASK, hit);
                if ((bal >> (grp * 8u)) & 0xffu) found = true;
                if (__all_sync(FULL_MASK, found || !alive || j + 8 >= len)) break;
            }
            if (alive && !found) alive = false;
        }
        if (i < N && !alive && lg == 0) {
            u32 pos = v - base_u;
            atomicAnd(q.bm[u] + (pos >> 5), ~(1u << (pos & 31u)));
        }
    }
    TSYNC_B(t);
    if (!compact_vertex(t, g, q, u)) return false;
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

__device__ __forceinline__ u32 edge_src(const QDesc* d, u32 e) {
    u32 x = 0;
    while (d->e_first[x + 1] <= e) ++x;
    return x;
}

// matching/BuildTable.cpp:9-151: row i of T[x][y] lists, ascending, the
// positions in C(y) of the data neighbours of C(x)[i]. Every directed query
// edge's table is built independently (count, team scan, device allocation,
// fill); all tables of a query share one offset array P and one entry array.
template <class Team>
__device__ bool stage_tables(Team& t, const DevGraph& g, QState& q, DevArena* arena) {
    const QDesc* d = q.desc;
    const u32 ne = d->e_first[d->n];
    if (t.rank() == 0) {
        u32 acc = 0;
        for (u32 e = 0; e < ne; ++e) {
            q.e_row_base[e] = acc;
            acc += q.cnt[edge_src(d, e)];
        }
        q.e_row_base[ne] = acc;
        q.total_rows = acc;
    }
    TSYNC_B(t);
    const u32 R = q.total_rows;
    const u32 lane = lane_id(), grp = lane >> 3, lg = lane & 7u;
    // count pass
    for (u32 r0 = t.warp() * 4u; r0 < R; r0 += t.nwarps() * 4u) {
        u32 r = r0 + grp;
        u32 s = 0, e = 0, y = 0;
        if (r < R) {
            u32 ei, i;
            row_of(q, ne, r, ei, i);
            u32 x = edge_src(d, ei);
            y = d->e_dst[ei];
            label_run(g, q.list[x][i], d->label[y], s, e);
        }
        const u32 base_y = r < R ? bucket_base(g, d->label[y]) : 0;
        u32 len = e - s, mx = warp_max(len), c = 0;
        for (u32 j = 0; j < mx; j += 8) {
            bool hit = j + lg < len && test_bit(q.bm[y], __ldg(g.nbr + s + j + lg) - base_y);
            u32 bal = __ballot_sync(FULL_MASK, hit);
            c += __popc((bal >> (grp * 8u)) & 0xffu);
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
    for (u32 r0 = t.warp() * 4u; r0 < R; r0 += t.nwarps() * 4u) {
        u32 r = r0 + grp;
        u32 s = 0, e = 0, y = 0, out = 0;
        if (r < R) {
            u32 ei, i;
            row_of(q, ne, r, ei, i);
            u32 x = edge_src(d, ei);
            y = d->e_dst[ei];
            label_run(g, q.list[x][i], d->label[y], s, e);
            out = P[r];
        }
        const u32 base_y = r < R ? bucket_base(g, d->label[y]) : 0;
        u32 len = e - s, mx = warp_max(len), written = 0;
        for (u32 j = 0; j < mx; j += 8) {
            u32 pos = 0;
            bool hit = false;
            if (j + lg < len) {
                pos = __ldg(g.nbr + s + j + lg) - base_y;
                hit = test_bit(q.bm[y], pos);
            }
            u32 bal = (__ballot_sync(FULL_MASK, hit) >> (grp * 8u)) & 0xffu;
            if (hit) {
                u32 word = q.bm[y][pos >> 5];
                u32 cpos = q.rank[y][pos >> 5] + __popc(word & ((1u << (pos & 31u)) - 1u));
                q.adj[out + written + __popc(bal & ((1u << lg) - 1u))] = cpos;
            }
            written += __popc(bal);
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

// matching/GenerateQueryPlan.cpp:680-721 estimatePathEmbeddsingsNum for all
// paths of the chosen CFL order plan; est_out[path_off[p] - p + k] is entry k
// of path p (paths have path_len - 1 estimates).
template <class Team>
__device__ bool cfl_estimates(Team& t, QState& q, const u32* pw) {
    const QDesc* d = q.desc;
    const u32 n = d->n;
    const u32 ngroups = pw[1 + 2 * n + 1];
    const u32* gfirst = pw + 1 + 2 * n + 2;
    const u32 npaths = gfirst[ngroups + 1 - 1 + 1];
    const u32* poff = gfirst + ngroups + 2;
    const u32* ncore_p = pw + 1 + 2 * n;
    const u32* pv = poff + npaths + 1 + ncore_p[0];
    for (u32 i = t.rank(); i < PSM_PLAN_WORDS; i += t.size()) q.est_out[i] = 0;
    TSYNC_B(t);
    for (u32 p = 0; p < npaths; ++p) {
        const u32* path = pv + poff[p];
        const u32 k = poff[p + 1] - poff[p];
        u64* est = q.est_out + (poff[p] - p);
        u64* child = q.est_a;
        u64* par = q.est_b;
        {
            const u32 a = path[k - 2], b = path[k - 1];
            const u32 rb = table_base(q, a, b), rows = q.cnt[a];
            u64 s = 0;
            for (u32 i = t.rank(); i < rows; i += t.size()) {
                u64 c = q.P[rb + i + 1] - q.P[rb + i];
                child[i] = c;
                s += c;
            }
            s = warp_sum64(s);
            if (lane_id() == 0 && s) atomicAdd((unsigned long long*)&est[k - 2], (unsigned long long)s);
        }
        TSYNC_B(t);
        for (int i = (int)k - 2; i >= 1; --i) {
            const u32 a = path[i - 1], b = path[i];
            const u32 rb = table_base(q, a, b), rows = q.cnt[a];
            u64 s = 0;
            for (u32 j = t.rank(); j < rows; j += t.size()) {
                u64 ls = 0;
                for (u32 e = q.P[rb + j]; e < q.P[rb + j + 1]; ++e) ls += child[q.adj[e]];
                par[j] = ls;
                s += ls;
            }
            s = warp_sum64(s);
            if (lane_id() == 0 && s) atomicAdd((unsigned long long*)&est[i - 1], (unsigned long long)s);
            TSYNC_B(t);
            u64* tmp = child;
            child = par;
            par = tmp;
        }
    }
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
// earlier neighbours, in query-vertex id order), their table rows, and the
// earlier depths sharing the label (only those can collide on a data vertex).
__device__ void enum_plan(const DevGraph& g, QState& q) {
    const QDesc* d = q.desc;
    const u32 n = d->n;
    u32 depth_of[PSM_MAXQ];
    for (u32 i = 0; i < n; ++i) depth_of[q.order[i]] = i;
    u32 seen = 0;
    for (u32 i = 0; i < n; ++i) {
        const u32 u = q.order[i];
        u32 k = 0, same = 0;
        u32 m = d->adj[u] & seen;
        while (m) {
            u32 b = __ffs(m) - 1;
            m &= m - 1;
            q.bn_depth[i][k] = depth_of[b];
            q.bn_tab[i][k] = table_base(q, b, u);
            ++k;
        }
        for (u32 j = 0; j < i; ++j)
            if (d->label[q.order[j]] == d->label[u]) same |= 1u << j;
        q.nbn[i] = k;
        q.same_mask[i] = same;
        seen |= 1u << u;
    }
    for (u32 u = 0; u < n; ++u) q.cbase[u] = bucket_base(g, d->label[u]);
    q.root_cnt = q.cnt[q.order[0]];
    u64 mem = 0;
    for (u32 u = 0; u < n; ++u) mem += (u64)q.cnt[u] * 4u;
    for (u32 a = 0; a < n; ++a) {
        u32 m = d->adj[a] & ~((2u << a) - 1u);  // b > a
        while (m) {
            u32 b = __ffs(m) - 1;
            m &= m - 1;
            u32 ab = table_base(q, a, b), ba = table_base(q, b, a);
            u64 nab = q.P[ab + q.cnt[a]] - q.P[ab], nba = q.P[ba + q.cnt[b]] - q.P[ba];
            mem += (nab + q.cnt[a] + nba + q.cnt[b]) * 4u;
        }
    }
    q.memory_bytes = mem;
}

// ------------------------------------------------------------ driver --

template <class Team>
__device__ void prepare_query(Team& t, const DevGraph& g, QState& q, DevArena* arena) {
    const QDesc* d = q.desc;
    const u32 n = d->n;
    // Stage 0: clear bitmaps and counters.
    for (u32 u = 0; u < n; ++u)
        for (u32 i = t.rank(); i < q.bwords[u]; i += t.size()) q.bm[u][i] = 0;
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
        q.table_nnz = 0;
        q.memory_bytes = 0;
        q.status = PSM_DEV_OK;
    }
    TSYNC(t);
    const u32 all = n >= 32 ? ~0u : ((1u << n) - 1u);
    const bool cfl = d->filter == PSM_FILTER_CFL;
    u32 need = all;
    if (cfl) {
        need = 0;
        for (u32 k = 0; k < d->nfopt; ++k) need |= 1u << d->fopt_vertex[k];
    }
    stage_nlf(t, g, q, need, d->order == PSM_ORDER_CFL);
    TSYNC(t);
    if (t.rank() == 0) {
        if (cfl) {
            // matching/GenerateFilteringPlan.cpp:343-385: lowest count/degree
            // among the kept options, first one on ties.
            double best = (double)d->fopt_max_score_num;
            u32 pick = 0;
            for (u32 k = 0; k < d->nfopt; ++k) {
                u32 u = d->fopt_vertex[k];
                double s = (double)q.item_cnt[u] / (double)d->deg[u];
                if (s < best) best = s, pick = k;
            }
            q.froot = pick;
        }
        if (d->order == PSM_ORDER_CFL) {
            double best = (double)d->fopt_max_score_num;
            u32 pick = 0;
            for (u32 k = 0; k < d->noopt; ++k) {
                u32 u = d->oopt_vertex[k];
                double s = (double)q.item_cnt[d->oopt_item[k]] / (double)d->deg[u];
                if (s < best) best = s, pick = k;
            }
            q.oroot = pick;
        }
    }
    TSYNC(t);
    if (!cfl) {
        // NLFFilter / GQLFilter stop at the first empty set.
        for (u32 u = 0; u < n; ++u) {
            if (!compact_vertex(t, g, q, u)) return;
            TSYNC(t);
        }
        if (t.rank() == 0) {
            for (u32 u = 0; u < n; ++u)
                if (q.cnt[u] == 0) {
                    q.empty = 1;
                    q.filter_ok = 0;
                    for (u32 v = u + 1; v < n; ++v) q.cnt[v] = 0;
                    break;
                }
        }
        TSYNC(t);
        if (q.empty) return;
        if (d->filter == PSM_FILTER_GQL) {
            for (u32 round = 0; round < 2; ++round)
                for (u32 u = 0; u < n; ++u) {
                    const u32 base = bucket_base(g, d->label[u]);
                    const u32 N = q.cnt[u];
                    for (u32 i = t.warp(); i < N; i += t.nwarps()) {
                        u32 v = q.list[u][i];
                        u32 pos = v - base;
                        if (!test_bit(q.bm[u], pos)) continue;
                        if (!gql_check(g, d, q, u, v) && lane_id() == 0)
                            atomicAnd(q.bm[u] + (pos >> 5), ~(1u << (pos & 31u)));
                    }
                    TSYNC(t);
                }
            for (u32 u = 0; u < n; ++u) {
                if (!compact_vertex(t, g, q, u)) return;
                TSYNC(t);
            }
        }
    } else {
        const FilterPlan& fp = d->fplan[q.froot];
        const u32 r = fp.root;
        if (!compact_vertex(t, g, q, r)) return;
        TSYNC(t);
        for (u32 s = 0; s < fp.nsteps; ++s) {
            bool ok = fp.step_kind[s] == STEP_GEN ? step_generate(t, g, q, fp.step_u[s], fp.step_mask[s])
                                                  : step_prune(t, g, q, fp.step_u[s], fp.step_mask[s]);
            if (!ok) return;
        }
    }
    if (t.rank() == 0) {
        for (u32 u = 0; u < n; ++u)
            if (q.cnt[u] == 0) q.empty = 1;
    }
    TSYNC(t);
    if (!stage_tables(t, g, q, arena)) return;
    if (q.adj == nullptr) return;
    if (d->order == PSM_ORDER_CFL) {
        const u32* pw = d->plan_words + d->oplan_off[q.oroot];
        if (!cfl_estimates(t, q, pw)) return;
        TSYNC(t);
        if (t.rank() == 0) cfl_order_select(q, pw);
    } else {
        if (t.rank() == 0) gql_order(g, q);
    }
    TSYNC(t);
    if (t.rank() == 0) {
        enum_plan(g, q);
        if (q.empty) q.root_cnt = 0;
    }
    TSYNC(t);
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

// Plain path: one query prepared by the whole (co-resident) grid.
__global__ void __launch_bounds__(512) prep_grid_kernel(DevGraph g, QState* qs, GridBarrier* bar, DevArena* arena,
                                                        u64 budget_ns) {
    GridTeam t{bar, global_timer_ns() + budget_ns};
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
