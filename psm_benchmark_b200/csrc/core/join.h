// Hash join of partial-embedding relations (device side, join.cu).
#pragma once
#include <cuda_runtime.h>

#include "psm_internal.h"

#define PSM_JOIN_MAX_KEYS PSM_MAXQ

// What one join compares and writes. Columns are indices into rows.
struct JoinSpec {
    u32 nk;                        // key columns
    u32 bkey[PSM_JOIN_MAX_KEYS];   // key columns of build rows
    u32 pkey[PSM_JOIN_MAX_KEYS];   // the same keys in probe rows
    u32 bcols, pcols;              // row widths
    u32 nbx;                       // build non-key columns copied to the output
    u32 bx[PSM_MAXQ];              // their indices in build rows
    u32 bx_same[PSM_MAXQ];         // per bx column: probe columns with the same label (bit mask)
};

// Device buffers of one build side: 2^k slots (mask = 2^k - 1) and nb rows.
struct JoinTable {
    u32 mask;
    u32* slots;     // [mask+1] first build row of a key, or 0xFFFFFFFF
    u32* gcount;    // [mask+1] rows per key
    u32* gfill;     // [mask+1] scatter cursors
    u64* goff;      // [mask+1] exclusive scan of gcount
    u32* grp;       // [nb] slot of each build row
    u32* members;   // [nb] build rows grouped by key
    u64* scan_tmp;  // psm_scan_tmp_bytes(mask+1)
    u32* error;     // set if a key could not be placed
};

size_t psm_scan_tmp_bytes(u64 n);
// out[i] = sum of in[0..i); *total_dev (optional, device) = sum of all.
// tmp: psm_scan_tmp_bytes(n) bytes of device memory.
cudaError_t psm_excl_scan(const u32* in, u64 n, u64* out, u64* tmp, u64* total_dev, cudaStream_t st);
cudaError_t psm_join_build(const u32* brows, u64 nb, const JoinSpec& sp, const JoinTable& t, cudaStream_t st);
// Count pass (out == nullptr): out_cnt[j] = output rows of probe row j
// (optional) and *total += all. Write pass: rows at out_off[j].
cudaError_t psm_join_probe(const u32* prows, u64 np, const u32* brows, const JoinSpec& sp, const JoinTable& t,
                           u32* out_cnt, u32* out, const u64* out_off, unsigned long long* total, cudaStream_t st);
