// Host-side runtime types (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "psm_b200.h"
#include "psm_internal.h"

struct psm_graph {
    int device = 0;
    u32 V = 0, L = 0;
    u64 nnz = 0;
    u32 max_degree = 0, max_label_freq = 0;
    std::vector<u32> lab_off;      // host copy of the bucket ranges
    std::vector<u32> to_internal;  // original id -> internal id
    std::vector<u32> orig;         // internal id -> original id
    u32* d_off = nullptr;
    u32* d_nbr = nullptr;
    u32* d_lab_off = nullptr;
    u32* d_orig = nullptr;
    DevGraph dev{};
    // For memory estimates: sum of degrees per label, and (when L <=
    // LAB_PAIR_MAX) the number of directed edges per label pair.
    static constexpr u32 LAB_PAIR_MAX = 1024;
    std::vector<u64> lab_deg;
    std::vector<u64> lab_pair;  // [L * L]: edges from label a to label b at a * L + b
    u32 freq(u32 l) const { return l < L ? lab_off[l + 1] - lab_off[l] : 0u; }
    // Upper bound on the entries of a candidate-edge table from label a to b.
    u64 pair_edges(u32 a, u32 b) const {
        if (a >= L || b >= L) return 0;
        if (!lab_pair.empty()) return lab_pair[(u64)a * L + b];
        return std::min(lab_deg[a], lab_deg[b]);
    }
};

// Records msg as this thread's last error and returns code.
int psm_fail(int code, const std::string& msg);

// What the allocation-free recount needs from a finished run.
struct RunInternals {
    int device;
    cudaStream_t stream;
    QState* dq;
    const DevGraph* dev;
    int enum_blocks;
    u32 emit;
    u32 prep_status;  // PSM_DEV_* status the run's preparation ended with
    u32 isect;        // the context's intersection variant (PSM_ISECT_*)
};
int psm_run_internals(psm_run* run, RunInternals* out);

// PSM_OK if psm_context_set_batch_tuning would accept t for ctx (reads only
// the context's fixed launch shape, so any thread may call it).
int psm_batch_tuning_check(const psm_context* ctx, const psm_batch_tuning* t);
// Sizes the context's persistent grids to 1/parts of the GPU (serving lanes
// that run side by side).
void psm_context_share_gpu(psm_context* ctx, u32 parts);
// Arena bytes available to a batch (the arena minus its fixed region).
u64 psm_context_free_bytes(const psm_context* ctx);
// Warps of the context's enumeration launches.
int psm_context_enum_warps(const psm_context* ctx);
// Blocks that prepare one query of a batch of nq queries.
u32 psm_context_prep_blocks_per_query(const psm_context* ctx, u32 nq);
// Batched path with per-query completion: the enumerator writes a QDoneRec
// per query into done_dev (device address of host-mapped memory) as each
// query finishes, and poll(poll_arg) runs every 0.1 ms until the launch
// ends. exit_keep > 0 lets idle warps leave once no work is left.
int psm_batch_polled(psm_context* ctx, const psm_graph* g, const psm_query_desc* qs, u32 nq, const psm_options* opt,
                     psm_result* results, QDoneRec* done_dev, u32 exit_keep, void (*poll)(void*), void* poll_arg);

// Builds the device query descriptor (validation, NLF lists, CFL plans).
// Returns PSM_OK or PSM_ERR_ARG with *err set.
int psm_build_qdesc(const psm_graph& g, const psm_query_desc& q, const psm_options& opt, QDesc* d, std::string* err);

// Size in bytes of the prefix of a QDesc that must be copied to the device.
size_t psm_qdesc_bytes(const QDesc& d);

// Kernel launchers (prep.cu, enum.cu).
cudaError_t psm_launch_prep_block(const DevGraph& g, QState* qs, u32 nq, u32* ticket, DevArena* arena, int blocks,
                                  int threads, cudaStream_t st);
cudaError_t psm_launch_prep_grid(const DevGraph& g, QState* qs, void* barrier, DevArena* arena, u64 budget_ns,
                                 int blocks, int threads, cudaStream_t st);
cudaError_t psm_prep_grid_max_blocks(int threads, int* blocks);
cudaError_t psm_prep_cluster_batch_clusters(int threads, int cluster, int* clusters);
cudaError_t psm_launch_prep_cluster_batch(const DevGraph& g, QState* qs, u32 nq, u32* ticket, DevArena* arena,
                                          int cluster, int clusters, int threads, cudaStream_t st);
cudaError_t psm_prep_cluster_size(int threads, int want, int* size);
cudaError_t psm_launch_prep_cluster(const DevGraph& g, QState* qs, DevArena* arena, int cluster, int threads,
                                    cudaStream_t st);
size_t psm_enum_scratch_bytes();
size_t psm_enum_query_bytes(u32 nq);
size_t psm_enum_cache_bytes(int blocks);
// cache: psm_enum_cache_bytes(blocks) of device memory for the per-warp
// prefix-intersection caches, or null to run without them. done: per-query
// completion records in host-mapped memory (device address), or null.
// exit_keep > 0 lets idle warps beyond that many leave once no work is left.
// grabs_per_warp: how finely each query's initial work is cut (about that
// many pieces per warp of the launch for a lone query). isect: intersection
// variant (PSM_ISECT_*: binary search only, by cost per intersection, or
// merge wherever both arrays are non-empty); each has its own kernel.
cudaError_t psm_launch_enum(const DevGraph& g, QState* qs, u32 nq, void* scratch, void* query_scratch, u64 budget_ns,
                            int emit, int blocks, u32* cache, QDoneRec* done, u32 exit_keep, cudaStream_t st,
                            u32 grabs_per_warp = 8, u32 isect = 0);
cudaError_t psm_enum_max_blocks(int* blocks);
cudaError_t psm_launch_gather(const QState* qs, u32 nq, DevResult* out, cudaStream_t st);
cudaError_t psm_enum_read_ctl(void* scratch, EnumStats* out, cudaStream_t st);
// Split form for callers with pinned staging: queue the control block's copy
// on the stream, then read the stats once the stream has synchronised.
size_t psm_enum_ctl_bytes();
cudaError_t psm_enum_copy_ctl(const void* scratch, void* host, cudaStream_t st);
void psm_enum_ctl_stats(const void* host, EnumStats* out);
cudaError_t psm_launch_unit_plan(const DevGraph& g, QState* qs, u32 nq, cudaStream_t st);
cudaError_t psm_launch_unit_emit(QState* qs, u32 nq, u32* const* bufs, const u64* caps, cudaStream_t st);
