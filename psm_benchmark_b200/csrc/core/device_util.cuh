// Small device helpers shared by the preparation and enumeration kernels.
#pragma once
#include <stdint.h>

#include "psm_internal.h"

#define FULL_MASK 0xffffffffu

__device__ __forceinline__ u32 lane_id() { return threadIdx.x & 31u; }

// First index i in [lo, hi) with a[i] >= key (hi if none).
__device__ __forceinline__ u32 lower_bound_u32(const u32* __restrict__ a, u32 lo, u32 hi, u32 key) {
    while (lo < hi) {
        u32 mid = (lo + hi) >> 1;
        if (__ldg(a + mid) < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// True if key occurs in the ascending range a[lo, hi).
__device__ __forceinline__ bool contains_u32(const u32* __restrict__ a, u32 lo, u32 hi, u32 key) {
    u32 i = lower_bound_u32(a, lo, hi, key);
    return i < hi && __ldg(a + i) == key;
}

// Plain-load forms for memory that the running kernel itself writes (the
// enumerator's per-warp intersection caches): the read-only path behind
// __ldg may serve lines that are stale for such memory.
__device__ __forceinline__ u32 lower_bound_rw(const u32* a, u32 lo, u32 hi, u32 key) {
    while (lo < hi) {
        u32 mid = (lo + hi) >> 1;
        if (a[mid] < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}
__device__ __forceinline__ bool contains_rw(const u32* a, u32 lo, u32 hi, u32 key) {
    u32 i = lower_bound_rw(a, lo, hi, key);
    return i < hi && a[i] == key;
}

// Range of neighbours of internal vertex v that carry label l.
__device__ __forceinline__ void label_run(const DevGraph& g, u32 v, u32 l, u32& s, u32& e) {
    u32 lo = g.off[v], hi = g.off[v + 1];
    if (l >= g.L) {
        s = e = lo;
        return;
    }
    s = lower_bound_u32(g.nbr, lo, hi, g.lab_off[l]);
    e = lower_bound_u32(g.nbr, s, hi, g.lab_off[l + 1]);
}

// lower_bound_u32 computed by the W (4 or 8) lanes of an aligned lane group
// together: each round probes W evenly spaced positions of the range (a
// (W + 1)-way split), so with W = 8 a row of 1,000 entries takes 4 dependent
// loads instead of 10. Called by the whole warp; lo, hi and key are uniform
// within each group, and a group with lo == hi loads nothing.
template <u32 W = 8>
__device__ __forceinline__ u32 group_lower_bound(const u32* __restrict__ a, u32 lo, u32 hi, u32 key) {
    static_assert(W == 4 || W == 8, "group width");
    constexpr u32 M = (1u << W) - 1u;
    const u32 lg = lane_id() & (W - 1u), sh = lane_id() & ~(W - 1u);
    while (__any_sync(FULL_MASK, hi - lo > W)) {
        const u32 n = hi - lo;
        // probes lo + floor(n (j + 1) / (W + 1)), j < W: distinct, inside (lo, hi)
        bool lt = false;
        if (n > W) lt = __ldg(a + lo + (u32)((u64)n * (lg + 1u) / (W + 1u))) < key;
        const u32 c = __popc((__ballot_sync(FULL_MASK, lt) >> sh) & M);  // probes below key: a prefix
        if (n > W) {
            const u32 nlo = c ? lo + (u32)((u64)n * c / (W + 1u)) + 1u : lo;
            const u32 nhi = c < W ? lo + (u32)((u64)n * (c + 1u) / (W + 1u)) : hi;
            lo = nlo;
            hi = nhi;
        }
    }
    const bool lt = lg < hi - lo && __ldg(a + lo + lg) < key;
    return lo + __popc((__ballot_sync(FULL_MASK, lt) >> sh) & M);
}

// label_run for the W-lane group of this lane (v and l group-uniform; a
// group with !valid gets an empty run). Called by the whole warp.
template <u32 W = 8>
__device__ __forceinline__ void group_label_run(const DevGraph& g, bool valid, u32 v, u32 l, u32& s, u32& e) {
    u32 lo = 0, hi = 0, k1 = 0, k2 = 0;
    if (valid && l < g.L) {
        lo = g.off[v];
        hi = g.off[v + 1];
        k1 = g.lab_off[l];
        k2 = g.lab_off[l + 1];
    }
    s = group_lower_bound<W>(g.nbr, lo, hi, k1);
    e = group_lower_bound<W>(g.nbr, s, hi, k2);
}

__device__ __forceinline__ bool test_bit(const u32* bm, u32 pos) { return (bm[pos >> 5] >> (pos & 31)) & 1u; }

__device__ __forceinline__ u32 warp_sum(u32 x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(FULL_MASK, x, o);
    return x;
}
__device__ __forceinline__ u64 warp_sum64(u64 x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(FULL_MASK, x, o);
    return x;
}
__device__ __forceinline__ u32 warp_max(u32 x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = max(x, __shfl_xor_sync(FULL_MASK, x, o));
    return x;
}
// Inclusive warp prefix sum.
__device__ __forceinline__ u32 warp_incl_scan(u32 x) {
    u32 lane = lane_id();
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        u32 y = __shfl_up_sync(FULL_MASK, x, o);
        if (lane >= (u32)o) x += y;
    }
    return x;
}

__device__ __forceinline__ u64 global_timer_ns() {
    u64 t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ u32 ld_acquire_u32(const u32* p) {
    u32 v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(u32* p, u32 v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ u64 ld_acquire_u64(const u64* p) {
    u64 v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ u32 ld_volatile_u32(const u32* p) { return *(const volatile u32*)p; }

// Volatile load by lane 0, broadcast to the warp: every lane sees the same
// value, so branches on it keep the warp converged (full-mask warp
// primitives after a branch on a per-lane volatile read are undefined).
__device__ __forceinline__ u32 warp_ld_volatile_u32(const u32* p) {
    u32 v = 0;
    if ((threadIdx.x & 31u) == 0) v = *(const volatile u32*)p;
    return __shfl_sync(0xffffffffu, v, 0);
}

// ---- intersections of two ascending arrays of distinct values ----
//
// The arrays are table rows (read-only for the kernel: RO = true, loads
// through __ldg) or the enumerator's cache lists (written by the kernel:
// plain loads). Values are vertex ids or candidate positions, below
// 0xFFFFFFFF, which therefore serves as the end-of-array sentinel.

template <bool RO>
__device__ __forceinline__ u32 ld_sorted(const u32* a, u32 i) {
    if constexpr (RO)
        return __ldg(a + i);
    else
        return a[i];
}

template <bool RO>
__device__ __forceinline__ u32 lower_bound_t(const u32* a, u32 lo, u32 hi, u32 key) {
    while (lo < hi) {
        const u32 mid = (lo + hi) >> 1;
        if (ld_sorted<RO>(a, mid) < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

__device__ __forceinline__ u32 log2_ceil(u32 x) { return x <= 1u ? 0u : 32u - __clz(x - 1u); }

// Intersection variants of the enumerator (psm_batch_tuning::intersect).
enum : u32 {
    ISECT_BINARY = 0,  // every entry of the shorter array binary-searched in the longer one
    ISECT_AUTO = 1,    // per intersection, the variant with the fewer dependent loads
    ISECT_MERGE = 2,   // merge whenever both arrays are non-empty (for tests of the merge paths)
};

// Whether a warp intersects arrays of n_short <= n_long entries faster by
// merge path than by walking the shorter one 32 entries at a time with a
// binary search of each in the longer one: dependent loads per lane,
// ceil(n_short / 32) * (log2 n_long + 1) against log2 n_short (the diagonal
// search) + (n_short + n_long) / 32 (the lane's run) + 3 (its first loads).
// Balanced arrays merge; an array 16 or more times the other's length is
// searched.
__device__ __forceinline__ bool warp_merge_pays(u32 mode, u32 n_short, u32 n_long) {
    if (mode == ISECT_BINARY || n_short == 0u) return false;
    if (mode == ISECT_MERGE) return true;
    const u32 bin = ((n_short + 31u) >> 5) * (log2_ceil(n_long + 1u) + 1u);
    const u32 mrg = log2_ceil(n_short + 1u) + ((n_short + n_long + 31u) >> 5) + 3u;
    return mrg < bin;
}

// The same choice for one lane intersecting on its own: a two-cursor merge
// (n_short + n_long loads) against a binary search of each entry of the
// shorter array (n_short * log2 n_long).
__device__ __forceinline__ bool lane_merge_pays(u32 mode, u32 n_short, u32 n_long) {
    if (mode == ISECT_BINARY || n_short == 0u) return false;
    if (mode == ISECT_MERGE) return true;
    return n_short + n_long < n_short * log2_ceil(n_long + 1u);
}

// |A ∩ B| by one lane, A the shorter array. A two-cursor merge when
// lane_merge_pays, else each entry of A searched in B from where the search
// of the previous entry ended (A ascends, so the range only shrinks).
template <bool RoA, bool RoB>
__device__ __forceinline__ u32 lane_isect_count(const u32* A, u32 na, const u32* B, u32 nb, u32 mode) {
    u32 c = 0;
    if (na == 0u || nb == 0u) return 0u;
    if (lane_merge_pays(mode, na, nb)) {
        u32 i = 0, j = 0;
        u32 a = ld_sorted<RoA>(A, 0), b = ld_sorted<RoB>(B, 0);
        while (true) {
            c += a == b;
            const bool ta = a <= b, tb = b <= a;
            if (ta) {
                if (++i == na) break;
                a = ld_sorted<RoA>(A, i);
            }
            if (tb) {
                if (++j == nb) break;
                b = ld_sorted<RoB>(B, j);
            }
        }
        return c;
    }
    u32 lo = 0;
    for (u32 i = 0; i < na; ++i) {
        const u32 x = ld_sorted<RoA>(A, i);
        lo = lower_bound_t<RoB>(B, lo, nb, x);
        if (lo == nb) break;
        c += ld_sorted<RoB>(B, lo) == x;
    }
    return c;
}

// One lane's run of a merge path (O. Green, R. McColl, D. A. Bader, "GPU
// merge path: a GPU merging algorithm", ICS 2012): merge steps [k0, k1) of
// the merge of A[0, na) and B[0, nb) in which, on a tie, A's entry goes
// first. The run's start (i entries of A and k0 - i of B taken) is found by
// a binary search along the cross diagonal k0; then the run is walked with
// one cursor per array. A common value A[i] == B[j] shows as the step that
// takes B[j] right after A[i]: hit(i, j) is called there, by the lane whose
// run holds that step, so every common value is seen exactly once.
template <bool RoA, bool RoB, class Hit>
__device__ __forceinline__ void merge_run(const u32* A, u32 na, const u32* B, u32 nb, u32 k0, u32 k1, Hit&& hit) {
    if (k0 >= k1) return;
    u32 lo = k0 > nb ? k0 - nb : 0u, hi = min(k0, na);
    while (lo < hi) {
        const u32 mid = (lo + hi) >> 1;
        if (ld_sorted<RoA>(A, mid) <= ld_sorted<RoB>(B, k0 - mid - 1u))
            lo = mid + 1u;
        else
            hi = mid;
    }
    u32 i = lo, j = k0 - lo;
    u32 a = i < na ? ld_sorted<RoA>(A, i) : 0xFFFFFFFFu;
    u32 b = j < nb ? ld_sorted<RoB>(B, j) : 0xFFFFFFFFu;
    u32 pa = i ? ld_sorted<RoA>(A, i - 1u) : 0xFFFFFFFFu;  // the last entry of A taken
    for (u32 k = k0; k < k1; ++k) {
        if (a <= b) {  // B exhausted (b = sentinel) also lands here
            pa = a;
            ++i;
            a = i < na ? ld_sorted<RoA>(A, i) : 0xFFFFFFFFu;
        } else {
            if (pa == b) hit(i - 1u, j);
            ++j;
            b = j < nb ? ld_sorted<RoB>(B, j) : 0xFFFFFFFFu;
        }
    }
}

// Merge steps per lane and tile of a warp merge path: a tile is 32 runs of
// at most MERGE_RUN steps; the warp checks a stop flag between tiles.
constexpr u32 MERGE_RUN = 256;

// Warp-cooperative |A ∩ B| by merge path, counting the common values for
// which keep(i, j) holds (A[i] == B[j]). With stop non-null, the warp reads
// *stop between tiles and returns its partial count with *stopped = true
// once it is set. Called by the whole warp; the result is warp-uniform.
template <bool RoA, bool RoB, class Keep>
__device__ u32 warp_merge_count(const u32* A, u32 na, const u32* B, u32 nb, const u32* stop, bool* stopped,
                                Keep&& keep) {
    const u32 lane = threadIdx.x & 31u;
    const u32 total = na + nb;
    const u32 per = min(MERGE_RUN, (total + 31u) >> 5);
    u32 c = 0;
    for (u32 t0 = 0; t0 < total; t0 += 32u * per) {
        if (t0 && stop) {
            u32 s = 0;
            if (lane == 0) s = *(const volatile u32*)stop;
            if (__shfl_sync(0xffffffffu, s, 0)) {
                *stopped = true;
                break;
            }
        }
        const u32 k0 = min(total, t0 + lane * per), k1 = min(total, k0 + per);
        merge_run<RoA, RoB>(A, na, B, nb, k0, k1, [&](u32 i, u32 j) { c += keep(i, j) ? 1u : 0u; });
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    return c;
}

// Warp-cooperative A ∩ B by merge path, written in ascending order: the
// common values A[i] for which keep(i) holds go to out[0, n) and n is
// returned. Each tile is walked twice: once to count every lane's values,
// once, after the warp has found each lane's offset, to write them. When
// more than cap values would be written, or with stop non-null *stop is seen
// set between tiles, *over is set and the count so far is returned. Called
// by the whole warp; the result is warp-uniform.
template <bool RoA, bool RoB, class Keep>
__device__ u32 warp_merge_collect(const u32* A, u32 na, const u32* B, u32 nb, const u32* stop, u32* out, u32 cap,
                                  bool* over, Keep&& keep) {
    const u32 lane = threadIdx.x & 31u;
    const u32 total = na + nb;
    const u32 per = min(MERGE_RUN, (total + 31u) >> 5);
    u32 n = 0;
    for (u32 t0 = 0; t0 < total; t0 += 32u * per) {
        if (t0 && stop) {
            u32 s = 0;
            if (lane == 0) s = *(const volatile u32*)stop;
            if (__shfl_sync(0xffffffffu, s, 0)) {
                *over = true;
                break;
            }
        }
        const u32 k0 = min(total, t0 + lane * per), k1 = min(total, k0 + per);
        u32 mine = 0;
        merge_run<RoA, RoB>(A, na, B, nb, k0, k1, [&](u32 i, u32) { mine += keep(i) ? 1u : 0u; });
        const u32 incl = warp_incl_scan(mine);
        const u32 tile = __shfl_sync(0xffffffffu, incl, 31);
        if (n + tile > cap) {
            *over = true;
            break;
        }
        u32 w = n + incl - mine;
        merge_run<RoA, RoB>(A, na, B, nb, k0, k1, [&](u32 i, u32) {
            if (keep(i)) out[w++] = ld_sorted<RoA>(A, i);
        });
        n += tile;
    }
    return n;
}

