// Self-check of the enumerator's intersection primitives (device_util.cuh)
// on arrays given by the host. One warp computes the intersection of two
// ascending arrays of distinct values in every form the enumerator uses:
//   counts[0]  |A ∩ B| by warp merge path (warp_merge_count)
//   counts[1]  |A ∩ B| by one lane's two-cursor merge (lane_isect_count, merge)
//   counts[2]  |A ∩ B| by one lane's shrinking search (lane_isect_count, search)
//   counts[3]  entries written by the warp merge path with output
//              (warp_merge_collect) into list[0, cap)
//   counts[4]  1 when that output would have exceeded cap
// With filter set, only common values not divisible by 3 are counted in
// counts[0] and written to the list (the predicate the enumerator uses there
// tests further rows; any predicate of the value serves the check). The host
// compares the results with its own intersection.
#include <cuda_runtime.h>

#include "host.h"  // before device_util.cuh: the C ABI's enums come first
#include "device_util.cuh"

namespace {

__global__ void isect_check_kernel(const u32* a, u32 na, const u32* b, u32 nb, u32 cap, u32 filter, u32* counts,
                                   u32* list) {
    const u32 lane = lane_id();
    auto keep_val = [&](u32 x) { return !filter || x % 3u != 0u; };
    const u32 c0 = warp_merge_count<true, false>(a, na, b, nb, nullptr, nullptr,
                                                 [&](u32 i, u32) { return keep_val(__ldg(a + i)); });
    u32 c1 = 0, c2 = 0;
    if (lane == 0) {
        // the shorter array first, as the enumerator calls it
        if (na <= nb) {
            c1 = lane_isect_count<true, false>(a, na, b, nb, ISECT_MERGE);
            c2 = lane_isect_count<true, false>(a, na, b, nb, ISECT_BINARY);
        } else {
            c1 = lane_isect_count<false, true>(b, nb, a, na, ISECT_MERGE);
            c2 = lane_isect_count<false, true>(b, nb, a, na, ISECT_BINARY);
        }
    }
    bool over = false;
    const u32 n = warp_merge_collect<true, true>(a, na, b, nb, nullptr, list, cap, &over,
                                                 [&](u32 i) { return keep_val(__ldg(a + i)); });
    if (lane == 0) {
        counts[0] = c0;
        counts[1] = c1;
        counts[2] = c2;
        counts[3] = n;
        counts[4] = over ? 1u : 0u;
    }
}

}  // namespace

extern "C" int psm_intersect_check(const uint32_t* a, uint32_t na, const uint32_t* b, uint32_t nb, uint32_t cap,
                                   uint32_t filter, uint32_t* counts, uint32_t* list) {
    if ((na && !a) || (nb && !b) || !counts || (cap && !list)) return psm_fail(PSM_ERR_ARG, "null argument");
    const size_t bytes = sizeof(u32) * ((size_t)na + nb + cap + 5 + 3);
    u32* d = nullptr;
    cudaError_t e = cudaMalloc(&d, bytes);
    if (e != cudaSuccess) return psm_fail(PSM_ERR_CUDA, cudaGetErrorString(e));
    u32* da = d;
    u32* db = da + na;
    u32* dc = db + nb;
    u32* dl = dc + 8;
    if (na) e = cudaMemcpy(da, a, sizeof(u32) * na, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && nb) e = cudaMemcpy(db, b, sizeof(u32) * nb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        isect_check_kernel<<<1, 32>>>(da, na, db, nb, cap, filter, dc, dl);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(counts, dc, sizeof(u32) * 5, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && cap) e = cudaMemcpy(list, dl, sizeof(u32) * cap, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return psm_fail(PSM_ERR_CUDA, cudaGetErrorString(e));
    return PSM_OK;
}
