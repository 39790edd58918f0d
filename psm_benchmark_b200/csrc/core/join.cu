// Device hash join of two relations of partial embeddings (decomposition
// path). Replaces the reference's NoPartitionHashJoin
// (utility/hashjoin/hashjoin.cpp:337-572 execute, :591-779 constructRow) as
// driven by JoinCollect::concateTwoTabels (matching/JoinCollect.cpp:60-153):
//  - join keys are the query vertices present in both relations;
//  - a pair of rows with equal keys yields an output row iff the build row's
//    non-key data vertices do not occur among the probe row's vertices (the
//    injectivity test of constructRow). Two columns can hold the same data
//    vertex only if their query vertices share a label, so only same-label
//    column pairs are compared;
//  - output row = the probe row's columns, then the build row's non-key
//    columns.
// Rows are uint32 data vertex ids, row-major, in device memory.
//
// Layout of a join: an open-addressing table of 2^k slots (load factor
// <= 0.5) holding, per distinct key, the index of its first build row; a
// grouped member list (build rows by key: counts, exclusive scan, scatter);
// probing counts each probe row's output rows, an exclusive scan turns the
// counts into offsets and a second pass writes the rows (or, for the last
// join, only the total is accumulated).
#include <cuda_runtime.h>

#include "device_util.cuh"
#include "join.h"

namespace {

constexpr u32 EMPTY = 0xFFFFFFFFu;

__device__ __forceinline__ u64 key_hash(const u32* row, const u32* cols, u32 nk) {
    u64 h = 0x243F6A8885A308D3ull;
    for (u32 i = 0; i < nk; ++i) {
        h = (h ^ row[cols[i]]) * 0x9E3779B97F4A7C15ull;
        h ^= h >> 29;
    }
    h ^= h >> 32;
    h *= 0xD6E8FEB86659FD93ull;
    h ^= h >> 32;
    return h;
}

__device__ __forceinline__ bool keys_equal(const u32* a, const u32* acols, const u32* b, const u32* bcols, u32 nk) {
    for (u32 i = 0; i < nk; ++i)
        if (a[acols[i]] != b[bcols[i]]) return false;
    return true;
}

__global__ void hj_build(const u32* __restrict__ brows, u64 nb, JoinSpec sp, u32* slots, u32 mask, u32* grp,
                         u32* gcount, u32* error) {
    for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < nb; i += (u64)gridDim.x * blockDim.x) {
        const u32* r = brows + i * sp.bcols;
        u32 h = (u32)key_hash(r, sp.bkey, sp.nk) & mask;
        bool placed = false;
        for (u32 step = 0; step <= mask; ++step) {
            u32 cur = *(volatile u32*)&slots[h];
            if (cur == EMPTY) {
                const u32 prev = atomicCAS(&slots[h], EMPTY, (u32)i);
                if (prev == EMPTY) {
                    placed = true;
                    break;
                }
                cur = prev;
            }
            if (keys_equal(brows + (u64)cur * sp.bcols, sp.bkey, r, sp.bkey, sp.nk)) {
                placed = true;
                break;
            }
            h = (h + 1) & mask;
        }
        if (!placed) {
            atomicExch(error, 1u);  // cannot happen below load factor 1
            grp[i] = 0;
            continue;
        }
        grp[i] = h;
        atomicAdd(&gcount[h], 1u);
    }
}

__global__ void hj_scatter(u64 nb, const u32* grp, const u64* goff, u32* gfill, u32* members) {
    for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < nb; i += (u64)gridDim.x * blockDim.x) {
        const u32 h = grp[i];
        members[goff[h] + atomicAdd(&gfill[h], 1u)] = (u32)i;
    }
}

// One thread per probe row: finds the key's group, tests every member and
// counts (out == nullptr) or writes the output rows at out_off[j].
__global__ void hj_probe(const u32* __restrict__ prows, u64 np, const u32* __restrict__ brows, JoinSpec sp,
                         const u32* __restrict__ slots, u32 mask, const u64* __restrict__ goff,
                         const u32* __restrict__ gcount, const u32* __restrict__ members, u32* out_cnt, u32* out,
                         const u64* __restrict__ out_off, unsigned long long* total) {
    u64 acc = 0;
    const u32 ocols = sp.pcols + sp.nbx;
    for (u64 j = blockIdx.x * (u64)blockDim.x + threadIdx.x; j < np; j += (u64)gridDim.x * blockDim.x) {
        const u32* pr = prows + j * sp.pcols;
        u32 h = (u32)key_hash(pr, sp.pkey, sp.nk) & mask;
        u32 c = 0;
        for (u32 step = 0; step <= mask; ++step) {
            const u32 cur = slots[h];
            if (cur == EMPTY) break;
            if (keys_equal(brows + (u64)cur * sp.bcols, sp.bkey, pr, sp.pkey, sp.nk)) {
                const u64 m0 = goff[h], m1 = m0 + gcount[h];
                u32* o = out ? out + out_off[j] * ocols : nullptr;
                for (u64 m = m0; m < m1; ++m) {
                    const u32* br = brows + (u64)members[m] * sp.bcols;
                    bool ok = true;
                    for (u32 x = 0; x < sp.nbx && ok; ++x) {
                        const u32 v = br[sp.bx[x]];
                        for (u32 pm = sp.bx_same[x]; pm && ok; pm &= pm - 1) ok = pr[__ffs(pm) - 1] != v;
                    }
                    if (!ok) continue;
                    if (o) {
                        for (u32 k = 0; k < sp.pcols; ++k) o[k] = pr[k];
                        for (u32 x = 0; x < sp.nbx; ++x) o[sp.pcols + x] = br[sp.bx[x]];
                        o += ocols;
                    }
                    ++c;
                }
                break;
            }
            h = (h + 1) & mask;
        }
        if (out_cnt) out_cnt[j] = c;
        acc += c;
    }
    if (total) {
        acc = warp_sum64(acc);
        if (lane_id() == 0 && acc) atomicAdd(total, (unsigned long long)acc);
    }
}

// ---- exclusive scan of u32 counts into u64 offsets (three passes) ----
constexpr u32 SCAN_THREADS = 1024;
constexpr u32 SCAN_ITEMS = 4;
constexpr u32 SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__global__ void scan_tiles(const u32* in, u64 n, u64* tile_sum) {
    __shared__ u64 red[32];
    const u64 base = (u64)blockIdx.x * SCAN_TILE;
    u64 s = 0;
    for (u32 k = 0; k < SCAN_ITEMS; ++k) {
        const u64 i = base + (u64)k * SCAN_THREADS + threadIdx.x;
        if (i < n) s += in[i];
    }
    s = warp_sum64(s);
    if (lane_id() == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        u64 v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0;
        v = warp_sum64(v);
        if (threadIdx.x == 0) tile_sum[blockIdx.x] = v;
    }
}

// One block: exclusive scan of the tile sums in place; total at [ntiles].
__global__ void scan_tile_sums(u64* tile_sum, u64 ntiles) {
    __shared__ u64 wsum[32];
    __shared__ u64 carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const u32 lane = lane_id(), w = threadIdx.x >> 5;
    for (u64 b = 0; b < ntiles; b += blockDim.x) {
        const u64 i = b + threadIdx.x;
        const u64 x = i < ntiles ? tile_sum[i] : 0;
        u64 incl = x;
        for (int o = 1; o < 32; o <<= 1) {
            const u64 y = __shfl_up_sync(FULL_MASK, incl, o);
            if (lane >= (u32)o) incl += y;
        }
        if (lane == 31) wsum[w] = incl;
        __syncthreads();
        if (w == 0) {
            const u64 v = lane < (blockDim.x >> 5) ? wsum[lane] : 0;
            u64 vi = v;
            for (int o = 1; o < 32; o <<= 1) {
                const u64 y = __shfl_up_sync(FULL_MASK, vi, o);
                if (lane >= (u32)o) vi += y;
            }
            wsum[lane] = vi - v;
        }
        __syncthreads();
        const u64 excl = carry + wsum[w] + incl - x;
        __syncthreads();
        if (i < ntiles) tile_sum[i] = excl;
        if (threadIdx.x == blockDim.x - 1) carry = excl + x;
        __syncthreads();
    }
    if (threadIdx.x == 0) tile_sum[ntiles] = carry;
}

__global__ void scan_apply(const u32* in, u64 n, const u64* tile_off, u64* out) {
    __shared__ u64 wsum[32];
    __shared__ u64 carry;
    if (threadIdx.x == 0) carry = tile_off[blockIdx.x];
    __syncthreads();
    const u32 lane = lane_id(), w = threadIdx.x >> 5;
    const u64 base = (u64)blockIdx.x * SCAN_TILE;
    for (u32 k = 0; k < SCAN_ITEMS; ++k) {
        const u64 i = base + (u64)k * SCAN_THREADS + threadIdx.x;
        const u64 x = i < n ? in[i] : 0;
        u64 incl = x;
        for (int o = 1; o < 32; o <<= 1) {
            const u64 y = __shfl_up_sync(FULL_MASK, incl, o);
            if (lane >= (u32)o) incl += y;
        }
        if (lane == 31) wsum[w] = incl;
        __syncthreads();
        if (w == 0) {
            const u64 v = lane < (blockDim.x >> 5) ? wsum[lane] : 0;
            u64 vi = v;
            for (int o = 1; o < 32; o <<= 1) {
                const u64 y = __shfl_up_sync(FULL_MASK, vi, o);
                if (lane >= (u32)o) vi += y;
            }
            wsum[lane] = vi - v;
        }
        __syncthreads();
        const u64 excl = carry + wsum[w] + incl - x;
        __syncthreads();
        if (i < n) out[i] = excl;
        if (threadIdx.x == blockDim.x - 1) carry = excl + x;
        __syncthreads();
    }
}

int grid_for(u64 n, int threads) {
    u64 b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148ull * 16) b = 148ull * 16;
    return (int)b;
}

}  // namespace

size_t psm_scan_tmp_bytes(u64 n) { return sizeof(u64) * ((n + SCAN_TILE - 1) / SCAN_TILE + 2); }

cudaError_t psm_excl_scan(const u32* in, u64 n, u64* out, u64* tmp, u64* total_dev, cudaStream_t st) {
    const u64 ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (ntiles > 0) {
        scan_tiles<<<(unsigned)ntiles, SCAN_THREADS, 0, st>>>(in, n, tmp);
        scan_tile_sums<<<1, SCAN_THREADS, 0, st>>>(tmp, ntiles);
        scan_apply<<<(unsigned)ntiles, SCAN_THREADS, 0, st>>>(in, n, tmp, out);
        if (total_dev) cudaMemcpyAsync(total_dev, tmp + ntiles, sizeof(u64), cudaMemcpyDeviceToDevice, st);
    } else if (total_dev) {
        cudaMemsetAsync(total_dev, 0, sizeof(u64), st);
    }
    return cudaGetLastError();
}

cudaError_t psm_join_build(const u32* brows, u64 nb, const JoinSpec& sp, const JoinTable& t, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(t.slots, 0xFF, sizeof(u32) * (t.mask + 1ull), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(t.gcount, 0, sizeof(u32) * (t.mask + 1ull), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(t.gfill, 0, sizeof(u32) * (t.mask + 1ull), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(t.error, 0, sizeof(u32), st);
    if (e != cudaSuccess) return e;
    if (nb) hj_build<<<grid_for(nb, 256), 256, 0, st>>>(brows, nb, sp, t.slots, t.mask, t.grp, t.gcount, t.error);
    e = psm_excl_scan(t.gcount, t.mask + 1ull, t.goff, t.scan_tmp, nullptr, st);
    if (e != cudaSuccess) return e;
    if (nb) hj_scatter<<<grid_for(nb, 256), 256, 0, st>>>(nb, t.grp, t.goff, t.gfill, t.members);
    return cudaGetLastError();
}

cudaError_t psm_join_probe(const u32* prows, u64 np, const u32* brows, const JoinSpec& sp, const JoinTable& t,
                           u32* out_cnt, u32* out, const u64* out_off, unsigned long long* total, cudaStream_t st) {
    if (np == 0) return cudaSuccess;
    hj_probe<<<grid_for(np, 256), 256, 0, st>>>(prows, np, brows, sp, t.slots, t.mask, t.goff, t.gcount, t.members,
                                               out_cnt, out, out_off, total);
    return cudaGetLastError();
}
