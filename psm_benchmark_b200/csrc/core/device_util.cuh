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
