// C ABI implementation (include/psm_b200.h): contexts, device arena layout,
// kernel sequencing for the plain and batched paths, result read-back.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "host.h"
// after host.h (psm_b200.h first)
#include "decompose.h"
#include "join.h"

int psm_graph_build(const uint32_t* off, const uint32_t* nbr, const uint32_t* labels, uint32_t V, psm_graph** out,
                    std::string* err);
int psm_graph_parse(const char* path, psm_graph** out, std::string* err);
int psm_graph_parse_binary(const char* deg_path, const char* adj_path, const char* label_path, psm_graph** out,
                           std::string* err);
int psm_text_to_binary(const char* text_path, const char* out_prefix, std::string* err);
int psm_edgelist_to_binary(const char* path, const char* out_prefix, u32 num_labels, u64 seed, std::string* err);
int psm_csr_write_binary(const u32* off, const u32* nbr, const u32* labels, u32 V, const char* deg_path,
                         const char* adj_path, const char* label_path, std::string* err);
void psm_graph_destroy(psm_graph* g);

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    return fail(e == cudaErrorMemoryAllocation ? PSM_ERR_OOM : PSM_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                              \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call);   \
    } while (0)

constexpr size_t ALIGN = 256;
inline size_t align_up(size_t x, size_t a = ALIGN) { return (x + a - 1) / a * a; }

// Host-side bump allocator over the device arena.
struct Bump {
    char* base;
    size_t top, cap;
    template <class T>
    T* take(size_t count) {
        size_t bytes = align_up(std::max<size_t>(count, 1) * sizeof(T));
        if (top + bytes > cap) return nullptr;
        T* p = (T*)(base + top);
        top += bytes;
        return p;
    }
};

}  // namespace

struct psm_context {
    int device = 0;
    cudaStream_t st = nullptr;
    char* arena = nullptr;
    size_t arena_bytes = 0;
    size_t fixed_bytes = 0;       // permanent region at the start of the arena
    DevArena* d_devarena = nullptr;
    void* d_barrier = nullptr;
    u32* d_ticket = nullptr;
    void* d_enum_scratch = nullptr;
    u32* d_enum_cache = nullptr;  // per-warp prefix-intersection caches (own allocation)
    int prep_threads = 512;
    int prep_grid_blocks = 0;
    int prep_block_blocks = 0;
    int cluster_size = 0;  // > 0: plain-path preparation by one thread-block cluster of this size
    int batch_cluster = 0;   // > 0: batched preparation by clusters of this many blocks, one query each
    int batch_clusters = 0;  // clusters of that launch
    int enum_blocks = 0;
    // batched-path settings (psm_context_set_batch_tuning / psm_autotune_batch)
    u32 tune_team = PSM_TEAM_RULE;   // preparation team of a batch
    u32 tune_grabs = 8;              // initial work pieces per enumeration warp
    u32 tune_quarters = 4;           // enumeration grid: quarters of the co-resident blocks
    u32 tune_isect = PSM_ISECT_BINARY;  // intersection variant of every enumeration launch
    cudaEvent_t ev[4]{};
    char* pinned = nullptr;  // pinned host staging of descriptors, states and results
    size_t pinned_bytes = 0;
    bool run_live = false;
};

struct psm_run {
    psm_context* ctx = nullptr;
    const psm_graph* g = nullptr;
    QState* d_q = nullptr;
    QState hq{};
    QDesc* hdesc = nullptr;  // host copy (order / labels)
    u32 n = 0;
    size_t arena_free = 0;   // first arena byte not used by the run
};

int psm_fail(int code, const std::string& msg) { return fail(code, msg); }

void psm_context_share_gpu(psm_context* ctx, u32 parts) {
    if (!ctx || parts < 2) return;
    ctx->enum_blocks = std::max(1, ctx->enum_blocks / (int)parts);
    ctx->prep_block_blocks = std::max(1, ctx->prep_block_blocks / (int)parts);
    ctx->batch_clusters = std::max(1, ctx->batch_clusters / (int)parts);
}

u64 psm_context_free_bytes(const psm_context* ctx) { return ctx->arena_bytes - ctx->fixed_bytes; }

int psm_context_enum_warps(const psm_context* ctx) { return ctx->enum_blocks * 8; }

int psm_run_internals(psm_run* r, RunInternals* out) {
    if (!r || !r->ctx || !r->d_q) return fail(PSM_ERR_ARG, "run is not alive");
    out->device = r->ctx->device;
    out->stream = r->ctx->st;
    out->dq = r->d_q;
    out->dev = &r->g->dev;
    out->enum_blocks = r->ctx->enum_blocks;
    out->emit = r->hq.emit_buf != nullptr;
    out->prep_status = r->hq.status;
    out->isect = r->ctx->tune_isect;
    return PSM_OK;
}

namespace {

struct Layout {
    QDesc* d_desc;
    QState* d_q;
    char* d_enum_q;  // per-query enumeration scratch
    DevResult* d_res;
};

// Per-query device buffers and QState initialisation.
int setup_query(psm_context* ctx, const psm_graph& g, const QDesc& d, const psm_options& opt, Bump& b,
                QDesc* d_desc, u32 scan_words, QState& q) {
    memset(&q, 0, sizeof(q));
    q.desc = d_desc;
    u32 maxw = 1, maxb = 1;
    for (u32 u = 0; u < d.n; ++u) {
        u32 B = g.freq(d.label[u]);
        u32 W = (B + 31) / 32;
        q.bwords[u] = W;
        q.bm[u] = b.take<u32>(W);
        q.rank[u] = b.take<u32>(W);
        q.list[u] = b.take<u32>(B);
        if (!q.bm[u] || !q.rank[u] || !q.list[u]) return fail(PSM_ERR_OOM, "device arena exhausted (candidates)");
        maxw = std::max(maxw, W);
        maxb = std::max(maxb, B);
    }
    u64 rows = 0;
    for (u32 x = 0; x < d.n; ++x) rows += (u64)g.freq(d.label[x]) * (d.e_first[x + 1] - d.e_first[x]);
    if (rows >= 0xFFFFFFF0ull) return fail(PSM_ERR_ARG, "candidate tables too large for 32-bit offsets");
    q.acc = b.take<u32>(maxw);
    q.tmp = b.take<u32>(maxw);
    q.acc_words = maxw;
    q.P = b.take<u32>(rows + 1);
    q.scan = b.take<u32>((size_t)scan_words * std::max(d.n, 1u));  // multi_compact: a block's word per vertex
    if (d.order == PSM_ORDER_CFL) {
        // one buffer pair per block that estimates paths concurrently
        q.est_blocks = std::max(1u, std::min(64u, scan_words - 1));
        q.est_stride = maxb;
        q.est_a = b.take<u64>((size_t)q.est_blocks * 2 * maxb);
        q.est_out = b.take<u64>(PSM_PLAN_WORDS);
        if (!q.est_a || !q.est_out) return fail(PSM_ERR_OOM, "device arena exhausted (estimates)");
    }
    if (!q.acc || !q.tmp || !q.P || !q.scan) return fail(PSM_ERR_OOM, "device arena exhausted (tables)");
    q.cap = opt.cap;
    // Diagnostics: PSM_TRACE=1 records a device timestamp per preparation
    // step (printed to stderr); PSM_HYBRID=1 lets block 0 of the plain-path
    // grid run small steps alone.
    if (getenv("PSM_TRACE")) {
        q.trace = b.take<u64>(PSM_TRACE_STEPS + 1);
        if (!q.trace) return fail(PSM_ERR_OOM, "device arena exhausted (trace)");
    }
    if (getenv("PSM_HYBRID")) q.step_cursor = HYBRID_REQUEST;
    if (opt.emit) {
        q.emit_cap_rows = opt.emit_capacity;
        q.emit_buf = b.take<u32>((size_t)opt.emit_capacity * d.n);
        if (!q.emit_buf) return fail(PSM_ERR_OOM, "device arena exhausted (embeddings)");
    }
    return PSM_OK;
}

bool use_cluster_batch(const psm_context* ctx, u32 nq) {
    if (ctx->batch_cluster <= 0 || ctx->tune_team == PSM_TEAM_BLOCK) return false;
    if (ctx->tune_team == PSM_TEAM_CLUSTER) return true;
    return nq <= 4u * (u32)ctx->batch_clusters;
}

// Enumeration grid of a batched launch (the tuning's share of the co-resident blocks).
int batch_enum_blocks(const psm_context* ctx) {
    return std::max(1, ctx->enum_blocks * (int)ctx->tune_quarters / 4);
}

u64 budget_ns(const psm_options& o) {
    double s = o.time_limit_s > 0 ? o.time_limit_s : 60.0;
    return (u64)(s * 1e9);
}

void fill_result(const DevResult& r, float prep_ms, float enum_ms, u64 donations, psm_result* out) {
    out->count = r.count;
    out->count_internal = r.count_internal;
    out->calls = r.calls;
    out->memory_bytes = r.memory_bytes;
    out->table_entries = r.table_nnz;
    out->alg_bytes = r.alg_bytes;
    out->donations = donations;
    out->overtime = r.overtime;
    out->filter_ok = r.filter_ok;
    out->status = r.status == PSM_DEV_OK ? (r.overtime ? PSM_ERR_TIMEOUT : PSM_OK)
                                         : (r.status == PSM_DEV_OOM ? PSM_ERR_OOM : PSM_ERR_INTERNAL);
    out->reserved = 0;
    out->prep_ms = prep_ms;
    out->enum_ms = enum_ms;
}

// Pinned host staging of at least `bytes` (the context's stream is idle
// between calls, so the buffer can be replaced here).
char* staging(psm_context* ctx, size_t bytes) {
    if (bytes <= ctx->pinned_bytes) return ctx->pinned;
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    ctx->pinned = nullptr;
    ctx->pinned_bytes = 0;
    size_t want = std::max<size_t>(bytes, 1 << 20);
    if (cudaHostAlloc((void**)&ctx->pinned, want, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        ctx->pinned = nullptr;
        return nullptr;
    }
    ctx->pinned_bytes = want;
    return ctx->pinned;
}

// Runs nq queries. grid_team: prepare the (single) query with the whole grid
// (plain path); otherwise one block per query (batched path).
int run_queries(psm_context* ctx, const psm_graph* g, const psm_query_desc* qs, u32 nq, const psm_options& opt,
                bool grid_team, psm_result* results, psm_run* keep, bool prep_only = false, QDoneRec* done = nullptr,
                u32 exit_keep = 0, void (*poll)(void*) = nullptr, void* poll_arg = nullptr) {
    if (!ctx || !g || !qs || nq == 0) return fail(PSM_ERR_ARG, "null argument");
    if (ctx->run_live) return fail(PSM_ERR_ARG, "a psm_run is still alive on this context");
    CK(cudaSetDevice(ctx->device));
    Bump b{ctx->arena, ctx->fixed_bytes, ctx->arena_bytes};
    // descriptors
    std::vector<QDesc> descs(nq);
    std::string err;
    for (u32 i = 0; i < nq; ++i) {
        int rc = psm_build_qdesc(*g, qs[i], opt, &descs[i], &err);
        if (rc) return fail(rc, "query " + std::to_string(i) + ": " + err);
    }
    Layout lay;
    lay.d_desc = b.take<QDesc>(nq);
    lay.d_q = b.take<QState>(nq);
    lay.d_enum_q = b.take<char>(psm_enum_query_bytes(nq));
    lay.d_res = b.take<DevResult>(nq);
    if (!lay.d_desc || !lay.d_q || !lay.d_enum_q || !lay.d_res) return fail(PSM_ERR_OOM, "device arena exhausted");
    // Batched preparation team: a cluster per query while the batch is small
    // (latency: a query's preparation spreads over the cluster's SMs), a
    // block per query for large batches (throughput).
    const bool cluster_batch = !grid_team && use_cluster_batch(ctx, nq);
    // team scans need one word per block of the preparing team (+1)
    const u32 scan_words = grid_team ? (u32)std::max(ctx->prep_grid_blocks, ctx->cluster_size) + 1
                                     : (cluster_batch ? (u32)ctx->batch_cluster : 1u) + 1;
    std::vector<QState> hq(nq);
    for (u32 i = 0; i < nq; ++i) {
        int rc = setup_query(ctx, *g, descs[i], opt, b, lay.d_desc + i, scan_words, hq[i]);
        if (rc) return rc;
    }
    // the rest of the arena is the device-side allocator region (tables)
    DevArena da{};
    size_t start = align_up(b.top);
    if (start + 4096 > b.cap) return fail(PSM_ERR_OOM, "device arena exhausted (no table space)");
    da.base = (u32*)(ctx->arena + start);
    da.top = 0;
    da.cap = (b.cap - start) / sizeof(u32);
    // uploads from pinned staging: descriptors (used prefix only), states,
    // allocator; the results come back through the same buffer
    size_t desc_bytes = 0;
    for (u32 i = 0; i < nq; ++i) desc_bytes += align_up(psm_qdesc_bytes(descs[i]), 16);
    const size_t off_q = align_up(desc_bytes), off_a = off_q + align_up(sizeof(QState) * nq),
                 off_r = off_a + align_up(sizeof(DevArena)),
                 off_c = off_r + align_up(sizeof(DevResult) * nq), off_b = off_c + align_up(psm_enum_ctl_bytes());
    char* pin = staging(ctx, off_b + 16);
    if (!pin) return fail(PSM_ERR_OOM, "pinned host staging");
    {
        size_t o = 0;
        for (u32 i = 0; i < nq; ++i) {
            const size_t b = psm_qdesc_bytes(descs[i]);
            memcpy(pin + o, &descs[i], b);
            CK(cudaMemcpyAsync(lay.d_desc + i, pin + o, b, cudaMemcpyHostToDevice, ctx->st));
            o += align_up(b, 16);
        }
    }
    memcpy(pin + off_q, hq.data(), sizeof(QState) * nq);
    memcpy(pin + off_a, &da, sizeof(da));
    CK(cudaMemcpyAsync(lay.d_q, pin + off_q, sizeof(QState) * nq, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->d_devarena, pin + off_a, sizeof(da), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemsetAsync(ctx->d_barrier, 0, 64, ctx->st));
    CK(cudaMemsetAsync(ctx->d_ticket, 0, sizeof(u32), ctx->st));
    const u64 budget = budget_ns(opt);
    CK(cudaEventRecord(ctx->ev[0], ctx->st));
    if (grid_team && ctx->cluster_size > 0) {
        CK(psm_launch_prep_cluster(g->dev, lay.d_q, ctx->d_devarena, ctx->cluster_size, ctx->prep_threads, ctx->st));
    } else if (grid_team) {
        CK(psm_launch_prep_grid(g->dev, lay.d_q, ctx->d_barrier, ctx->d_devarena, budget, ctx->prep_grid_blocks,
                                ctx->prep_threads, ctx->st));
    } else if (cluster_batch) {
        const int clusters = std::min<int>(ctx->batch_clusters, (int)nq);
        CK(psm_launch_prep_cluster_batch(g->dev, lay.d_q, nq, ctx->d_ticket, ctx->d_devarena, ctx->batch_cluster,
                                         clusters, ctx->prep_threads, ctx->st));
    } else {
        int blocks = std::min<int>(ctx->prep_block_blocks, (int)nq);
        CK(psm_launch_prep_block(g->dev, lay.d_q, nq, ctx->d_ticket, ctx->d_devarena, blocks, ctx->prep_threads,
                                 ctx->st));
    }
    CK(cudaEventRecord(ctx->ev[1], ctx->st));
    if (!prep_only)
        CK(psm_launch_enum(g->dev, lay.d_q, nq, ctx->d_enum_scratch, lay.d_enum_q, budget, opt.emit ? 1 : 0,
                           grid_team ? ctx->enum_blocks : batch_enum_blocks(ctx), ctx->d_enum_cache, done, exit_keep,
                           ctx->st, grid_team ? 8u : ctx->tune_grabs, ctx->tune_isect));
    CK(cudaEventRecord(ctx->ev[2], ctx->st));
    CK(psm_launch_gather(lay.d_q, nq, lay.d_res, ctx->st));
    if (poll) {
        // the caller collects per-query completion records while the launch runs
        cudaError_t q;
        while ((q = cudaStreamQuery(ctx->st)) == cudaErrorNotReady) {
            poll(poll_arg);
            std::this_thread::sleep_for(std::chrono::microseconds(100));
        }
        if (q != cudaSuccess) return cuda_fail(q, "batch launch");
        poll(poll_arg);
    }
    std::vector<DevResult> res(nq);
    CK(cudaMemcpyAsync(pin + off_r, lay.d_res, sizeof(DevResult) * nq, cudaMemcpyDeviceToHost, ctx->st));
    // the enumerator's control block and the grid barrier's abort word come
    // back through the staging buffer too: one synchronisation per run
    if (!prep_only) CK(psm_enum_copy_ctl(ctx->d_enum_scratch, pin + off_c, ctx->st));
    if (grid_team)  // GridBarrier::abort (second word of the barrier)
        CK(cudaMemcpyAsync(pin + off_b, (char*)ctx->d_barrier + 4, sizeof(u32), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    EnumStats es{};
    if (!prep_only) psm_enum_ctl_stats(pin + off_c, &es);
    memcpy(res.data(), pin + off_r, sizeof(DevResult) * nq);
    const u32 enum_err = es.error;
    float prep_ms = 0, enum_ms = 0;
    CK(cudaEventElapsedTime(&prep_ms, ctx->ev[0], ctx->ev[1]));
    CK(cudaEventElapsedTime(&enum_ms, ctx->ev[1], ctx->ev[2]));
    u64 h2d = sizeof(QState) * (u64)nq + sizeof(DevArena) + 64 + 4, d2h = sizeof(DevResult) * (u64)nq + (prep_only ? 0 : psm_enum_ctl_bytes()) + (grid_team ? 4 : 0);
    for (u32 i = 0; i < nq; ++i) h2d += psm_qdesc_bytes(descs[i]);
    int worst = PSM_OK;
    for (u32 i = 0; i < nq; ++i) {
        fill_result(res[i], prep_ms, enum_ms, es.donations, &results[i]);
        results[i].tasks = es.tasks;
        results[i].idle_polls = es.idle_polls;
        results[i].h2d_bytes = h2d / nq;
        results[i].d2h_bytes = d2h / nq;
        if (enum_err) results[i].status = PSM_ERR_INTERNAL;
        if (results[i].status != PSM_OK && worst == PSM_OK) worst = (int)results[i].status;
    }
    if (grid_team) {
        u32 ab = 0;
        memcpy(&ab, pin + off_b, sizeof(u32));
        if (ab) {
            for (u32 i = 0; i < nq; ++i) results[i].status = PSM_ERR_INTERNAL;
            worst = PSM_ERR_INTERNAL;
        }
    }
    if (hq[0].trace && nq > 1) {
        // per-query time at which the cap was reached, relative to the first
        std::vector<QState> st(nq);
        CK(cudaMemcpy(st.data(), lay.d_q, sizeof(QState) * nq, cudaMemcpyDeviceToHost));
        u64 t0 = ~0ull;
        for (auto& s : st)
            if (s.done_ns) t0 = std::min(t0, s.done_ns);
        fprintf(stderr, "psm trace done(us):");
        for (u32 i = 0; i < nq; ++i)
            fprintf(stderr, " %u:%.0f", i, st[i].done_ns ? (st[i].done_ns - t0) / 1e3 : -1.0);
        fprintf(stderr, "\n");
    }
    if (hq[0].trace) {
        for (u32 i = 0; i < nq && i < 4; ++i) {
            std::vector<u64> tr(PSM_TRACE_STEPS + 1);
            CK(cudaMemcpy(tr.data(), hq[i].trace, tr.size() * sizeof(u64), cudaMemcpyDeviceToHost));
            fprintf(stderr, "psm trace q%u:", i);
            u64 prev = tr[PSM_TRACE_STEPS];
            for (u32 k = 0; k < PSM_TRACE_STEPS && tr[k] >= prev && tr[k] - prev < 10000000000ull; ++k) {
                fprintf(stderr, " %u:%.1f", k, (tr[k] - prev) / 1e3);
                prev = tr[k];
            }
            fprintf(stderr, " (us)\n");
        }
    }
    if (keep) {
        keep->ctx = ctx;
        keep->g = g;
        keep->d_q = lay.d_q;
        CK(cudaMemcpy(&keep->hq, lay.d_q, sizeof(QState), cudaMemcpyDeviceToHost));
        keep->hdesc = new QDesc;
        memcpy(keep->hdesc, &descs[0], sizeof(QDesc));
        keep->n = descs[0].n;
        DevArena top{};
        CK(cudaMemcpy(&top, ctx->d_devarena, sizeof(top), cudaMemcpyDeviceToHost));
        keep->arena_free = align_up(start + (size_t)std::min<u64>(top.top, top.cap) * sizeof(u32));
        ctx->run_live = true;
    }
    if (worst == PSM_ERR_INTERNAL) return fail(worst, enum_err ? "enumeration wait gave up" : "device error");
    if (worst == PSM_ERR_OOM) return fail(worst, "device arena exhausted (tables)");
    if (worst == PSM_ERR_TIMEOUT) return fail(worst, "time limit reached");
    return PSM_OK;
}

}  // namespace

extern "C" {

const char* psm_status_string(int s) {
    switch (s) {
        case PSM_OK: return "ok";
        case PSM_ERR_ARG: return "invalid argument";
        case PSM_ERR_OOM: return "out of device memory";
        case PSM_ERR_TIMEOUT: return "time limit reached";
        case PSM_ERR_CUDA: return "CUDA error";
        case PSM_ERR_IO: return "I/O error";
        case PSM_ERR_INTERNAL: return "internal error";
        default: return "unknown status";
    }
}

const char* psm_last_error(void) { return g_last_error.c_str(); }

const char* psm_version(void) { return "psm_b200 1.0 (sm_100a)"; }

int psm_graph_from_csr(const uint32_t* off, const uint32_t* nbr, const uint32_t* labels, uint32_t V, psm_graph** out) {
    if (!out) return fail(PSM_ERR_ARG, "null out");
    std::string err;
    int rc = psm_graph_build(off, nbr, labels, V, out, &err);
    return rc ? fail(rc, err) : PSM_OK;
}

int psm_graph_load(const char* path, psm_graph** out) {
    if (!path || !out) return fail(PSM_ERR_ARG, "null argument");
    std::string err;
    int rc = psm_graph_parse(path, out, &err);
    return rc ? fail(rc, err) : PSM_OK;
}

int psm_graph_load_binary(const char* degree_path, const char* adjacency_path, const char* label_path,
                          psm_graph** out) {
    if (!degree_path || !adjacency_path || !label_path || !out) return fail(PSM_ERR_ARG, "null argument");
    std::string err;
    int rc = psm_graph_parse_binary(degree_path, adjacency_path, label_path, out, &err);
    return rc ? fail(rc, err) : PSM_OK;
}

int psm_graph_store_binary(const uint32_t* offsets, const uint32_t* neighbors, const uint32_t* labels,
                           uint32_t num_vertices, const char* degree_path, const char* adjacency_path,
                           const char* label_path) {
    if (!offsets || !labels || (!neighbors && offsets[num_vertices]) || !degree_path || !adjacency_path ||
        !label_path)
        return fail(PSM_ERR_ARG, "null argument");
    std::string err;
    int rc = psm_csr_write_binary(offsets, neighbors, labels, num_vertices, degree_path, adjacency_path, label_path,
                                  &err);
    return rc ? fail(rc, err) : PSM_OK;
}

int psm_graph_convert(const char* text_path, const char* out_prefix) {
    if (!text_path || !out_prefix) return fail(PSM_ERR_ARG, "null argument");
    std::string err;
    int rc = psm_text_to_binary(text_path, out_prefix, &err);
    return rc ? fail(rc, err) : PSM_OK;
}

int psm_graph_convert_edgelist(const char* edge_list_path, const char* out_prefix, uint32_t num_labels,
                               uint64_t seed) {
    if (!edge_list_path || !out_prefix) return fail(PSM_ERR_ARG, "null argument");
    std::string err;
    int rc = psm_edgelist_to_binary(edge_list_path, out_prefix, num_labels, seed, &err);
    return rc ? fail(rc, err) : PSM_OK;
}

int psm_graph_info(const psm_graph* g, uint32_t* V, uint64_t* E, uint32_t* L, uint32_t* maxdeg, uint32_t* maxfreq) {
    if (!g) return fail(PSM_ERR_ARG, "null graph");
    if (V) *V = g->V;
    if (E) *E = g->nnz / 2;
    if (L) *L = g->L;
    if (maxdeg) *maxdeg = g->max_degree;
    if (maxfreq) *maxfreq = g->max_label_freq;
    return PSM_OK;
}

void psm_graph_free(psm_graph* g) { psm_graph_destroy(g); }

int psm_context_create(int device, uint64_t arena_bytes, psm_context** out) {
    if (!out) return fail(PSM_ERR_ARG, "null out");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(PSM_ERR_CUDA, "no CUDA device");
    if (device < 0 || device >= ndev) return fail(PSM_ERR_ARG, "bad device index");
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) return fail(PSM_ERR_CUDA, "this build targets sm_100a (B200) only");
    CK(cudaSetDevice(device));
    auto* c = new psm_context;
    c->device = device;
    if (arena_bytes == 0) arena_bytes = 4ull << 30;
    c->arena_bytes = arena_bytes;
    cudaError_t e = cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc((void**)&c->arena, arena_bytes);
    for (int i = 0; i < 4 && e == cudaSuccess; ++i) e = cudaEventCreate(&c->ev[i]);
    if (e != cudaSuccess) {
        psm_context_free(c);
        return cuda_fail(e, "context allocation");
    }
    Bump b{c->arena, 0, arena_bytes};
    c->d_devarena = b.take<DevArena>(1);
    c->d_barrier = b.take<char>(64);
    c->d_ticket = b.take<u32>(1);
    c->d_enum_scratch = b.take<char>(psm_enum_scratch_bytes());
    c->fixed_bytes = b.top;
    if (psm_prep_grid_max_blocks(c->prep_threads, &c->prep_grid_blocks) != cudaSuccess ||
        psm_enum_max_blocks(&c->enum_blocks) != cudaSuccess) {
        psm_context_free(c);
        return fail(PSM_ERR_CUDA, "occupancy query failed");
    }
    // Plain-path preparation grid: one block of 512 per SM. Its steps are
    // small, so the grid barrier's cost sets their time: measured on B200,
    // 148 blocks prepare the benchmark queries 13 % faster than 296 (and 74 or
    // a 16-block cluster are slower). PSM_PREP_BLOCKS overrides the size.
    const int coresident = c->prep_grid_blocks;  // cooperative launch limit
    c->prep_grid_blocks = std::min(coresident, prop.multiProcessorCount);
    if (const char* pb = getenv("PSM_PREP_BLOCKS")) {
        const int want = atoi(pb);
        if (want > 0) c->prep_grid_blocks = std::min(coresident, want);
    }
    c->prep_block_blocks = prop.multiProcessorCount * 4;
    // Batched preparation team: clusters of 8 blocks per query (default), or
    // one block per query (PSM_BATCH_TEAM=block).
    const char* bt = getenv("PSM_BATCH_TEAM");
    if (!(bt && strcmp(bt, "block") == 0)) {
        int clusters = 0;
        if (psm_prep_cluster_batch_clusters(c->prep_threads, 8, &clusters) == cudaSuccess && clusters > 0) {
            c->batch_cluster = 8;
            c->batch_clusters = clusters;
        }
    }
    // PSM_ENUM_CACHE=0 runs the enumerator without prefix-intersection caches.
    const char* ec = getenv("PSM_ENUM_CACHE");
    if (!(ec && strcmp(ec, "0") == 0)) {
        const size_t cb = psm_enum_cache_bytes(c->enum_blocks);
        e = cudaMalloc((void**)&c->d_enum_cache, cb);
        // the enumerator keeps its cache bitmaps all-zero between tasks
        if (e == cudaSuccess) e = cudaMemset(c->d_enum_cache, 0, cb);
        if (e != cudaSuccess) {
            psm_context_free(c);
            return cuda_fail(e, "enumeration cache allocation");
        }
    }
    // Plain-path preparation team: the whole grid (default; measured fastest
    // on B200) or one thread-block cluster (PSM_PLAIN_TEAM=cluster,
    // PSM_CLUSTER=size).
    const char* team = getenv("PSM_PLAIN_TEAM");
    if (team && strcmp(team, "cluster") == 0) {
        int want = 16;
        if (const char* cs = getenv("PSM_CLUSTER")) want = std::max(1, std::min(16, atoi(cs)));
        if (psm_prep_cluster_size(c->prep_threads, want, &c->cluster_size) != cudaSuccess) c->cluster_size = 0;
    }
    *out = c;
    return PSM_OK;
}

void psm_context_free(psm_context* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    for (auto& e : c->ev)
        if (e) cudaEventDestroy(e);
    if (c->arena) cudaFree(c->arena);
    if (c->pinned) cudaFreeHost(c->pinned);
    if (c->d_enum_cache) cudaFree(c->d_enum_cache);
    if (c->st) cudaStreamDestroy(c->st);
    delete c;
}

int psm_match(psm_context* ctx, const psm_graph* g, const psm_query_desc* q, const psm_options* opt,
              psm_result* res) {
    if (!opt || !res) return fail(PSM_ERR_ARG, "null argument");
    return run_queries(ctx, g, q, 1, *opt, true, res, nullptr);
}

int psm_match_batch(psm_context* ctx, const psm_graph* g, const psm_query_desc* qs, uint32_t nq,
                    const psm_options* opt, psm_result* results) {
    if (!opt || !results) return fail(PSM_ERR_ARG, "null argument");
    return run_queries(ctx, g, qs, nq, *opt, false, results, nullptr);
}

}  // extern "C"

int psm_batch_tuning_check(const psm_context* ctx, const psm_batch_tuning* t) {
    if (!ctx || !t) return fail(PSM_ERR_ARG, "null argument");
    if (t->team > PSM_TEAM_CLUSTER || t->grabs_per_warp < 1 || t->grabs_per_warp > 64 || t->enum_quarters < 1 ||
        t->enum_quarters > 4 || t->intersect > PSM_ISECT_MERGE)
        return fail(PSM_ERR_ARG, "tuning out of range");
    if (t->team == PSM_TEAM_CLUSTER && ctx->batch_cluster <= 0)
        return fail(PSM_ERR_ARG, "this context has no cluster preparation");
    return PSM_OK;
}

extern "C" {

int psm_context_set_batch_tuning(psm_context* ctx, const psm_batch_tuning* t) {
    int rc = psm_batch_tuning_check(ctx, t);
    if (rc) return rc;
    ctx->tune_team = t->team;
    ctx->tune_grabs = t->grabs_per_warp;
    ctx->tune_quarters = t->enum_quarters;
    ctx->tune_isect = t->intersect;
    return PSM_OK;
}

int psm_context_get_batch_tuning(psm_context* ctx, psm_batch_tuning* t) {
    if (!ctx || !t) return fail(PSM_ERR_ARG, "null argument");
    memset(t, 0, sizeof(*t));
    t->team = ctx->tune_team;
    t->grabs_per_warp = ctx->tune_grabs;
    t->enum_quarters = ctx->tune_quarters;
    t->intersect = ctx->tune_isect;
    return PSM_OK;
}

int psm_autotune_batch(psm_context* ctx, const psm_graph* g, const psm_query_desc* sample, uint32_t n,
                       const psm_options* opt, uint32_t repeats, psm_batch_tuning* best, psm_batch_tuning* tried,
                       uint32_t tried_cap, uint32_t* ntried) {
    if (!ctx || !g || !sample || n == 0 || !opt || !best) return fail(PSM_ERR_ARG, "null argument");
    if (opt->emit) return fail(PSM_ERR_ARG, "the tuner counts; emit is not supported");
    const psm_batch_tuning before{ctx->tune_team, ctx->tune_grabs, ctx->tune_quarters, ctx->tune_isect, 0.0};
    std::vector<psm_batch_tuning> cands;
    std::vector<psm_result> res(n);
    std::vector<u64> counts;
    int best_i = -1;
    // times the sample under cands[i] (run 0 warms up, then the best of
    // `repeats`); every setting must count the same embeddings
    auto measure = [&](size_t i) -> int {
        psm_context_set_batch_tuning(ctx, &cands[i]);
        double ms = 0;
        for (u32 r = 0; r <= std::max(1u, repeats); ++r) {
            int rc = run_queries(ctx, g, sample, n, *opt, false, res.data(), nullptr);
            if (rc && rc != PSM_ERR_TIMEOUT) return rc;
            const double t = res[0].prep_ms + res[0].enum_ms;
            if (r == 1 || (r > 1 && t < ms)) ms = t;
        }
        cands[i].ms = ms;
        std::vector<u64> c(n);
        for (u32 q = 0; q < n; ++q) c[q] = res[q].count;
        if (counts.empty())
            counts = c;
        else if (c != counts)
            return fail(PSM_ERR_INTERNAL, "counts differ between batch settings");
        if (best_i < 0 || ms < cands[best_i].ms) best_i = (int)i;
        return PSM_OK;
    };
    // stage 1: preparation team x work pieces per warp x enumeration grid,
    // under the installed intersection variant
    std::vector<u32> teams{PSM_TEAM_BLOCK};
    if (ctx->batch_cluster > 0) teams.push_back(PSM_TEAM_CLUSTER);
    for (u32 team : teams)
        for (u32 grabs : {2u, 8u, 32u})
            for (u32 quarters : {2u, 4u}) cands.push_back({team, grabs, quarters, before.intersect, 0.0});
    const size_t stage1 = cands.size();
    for (size_t i = 0; i < stage1; ++i) {
        int rc = measure(i);
        if (rc) {
            psm_context_set_batch_tuning(ctx, &before);
            return rc;
        }
    }
    // stage 2: the other intersection variants under stage 1's best setting
    for (u32 v : {(u32)PSM_ISECT_AUTO, (u32)PSM_ISECT_BINARY, (u32)PSM_ISECT_MERGE}) {
        if (v == before.intersect) continue;
        psm_batch_tuning c = cands[best_i];
        c.intersect = v;
        c.ms = 0.0;
        cands.push_back(c);
        int rc = measure(cands.size() - 1);
        if (rc) {
            psm_context_set_batch_tuning(ctx, &before);
            return rc;
        }
    }
    *best = cands[best_i];
    psm_context_set_batch_tuning(ctx, best);
    if (ntried) *ntried = (u32)std::min<size_t>(cands.size(), tried ? tried_cap : 0);
    if (tried)
        for (u32 i = 0; i < cands.size() && i < tried_cap; ++i) tried[i] = cands[i];
    return PSM_OK;
}

int psm_run_create(psm_context* ctx, const psm_graph* g, const psm_query_desc* q, const psm_options* opt,
                   psm_run** out, psm_result* res) {
    if (!opt || !res || !out) return fail(PSM_ERR_ARG, "null argument");
    auto* r = new psm_run;
    int rc = run_queries(ctx, g, q, 1, *opt, true, res, r);
    if (r->ctx == nullptr) {
        delete r;
        *out = nullptr;
        return rc;
    }
    *out = r;
    return rc;
}

int psm_run_candidates(psm_run* r, uint32_t u, uint32_t* buf, uint32_t buf_len, uint32_t* n) {
    if (!r || !n || u >= r->n) return fail(PSM_ERR_ARG, "bad run / vertex");
    u32 c = r->hq.cnt[u];
    *n = c;
    if (!buf) return PSM_OK;
    if (buf_len < c) return fail(PSM_ERR_ARG, "buffer too small");
    std::vector<u32> tmp(c);
    if (c) CK(cudaMemcpy(tmp.data(), r->hq.list[u], c * sizeof(u32), cudaMemcpyDeviceToHost));
    for (u32 i = 0; i < c; ++i) buf[i] = r->g->orig[tmp[i]];
    return PSM_OK;
}

int psm_run_table(psm_run* r, uint32_t a, uint32_t b, uint32_t* offsets, uint32_t offsets_len, uint32_t* entries,
                  uint32_t entries_len, uint32_t* rows, uint32_t* nnz) {
    if (!r || a >= r->n || b >= r->n) return fail(PSM_ERR_ARG, "bad run / vertices");
    const QDesc& d = *r->hdesc;
    if (!((d.adj[a] >> b) & 1u)) return fail(PSM_ERR_ARG, "not a query edge");
    if (r->hq.adj == nullptr) return fail(PSM_ERR_ARG, "tables were not built (empty candidate set)");
    u32 e = d.e_first[a] + (u32)__builtin_popcount(d.adj[a] & ((1u << b) - 1u));
    u32 base = r->hq.e_row_base[e], R = r->hq.cnt[a];
    std::vector<u32> P(R + 1);
    CK(cudaMemcpy(P.data(), r->hq.P + base, (R + 1) * sizeof(u32), cudaMemcpyDeviceToHost));
    u32 z = P[R] - P[0];
    if (rows) *rows = R;
    if (nnz) *nnz = z;
    if (offsets) {
        if (offsets_len < R + 1) return fail(PSM_ERR_ARG, "offsets buffer too small");
        for (u32 i = 0; i <= R; ++i) offsets[i] = P[i] - P[0];
    }
    if (entries) {
        if (entries_len < z) return fail(PSM_ERR_ARG, "entries buffer too small");
        if (z) CK(cudaMemcpy(entries, r->hq.adj + P[0], z * sizeof(u32), cudaMemcpyDeviceToHost));
    }
    return PSM_OK;
}

int psm_run_order(psm_run* r, uint32_t* order, uint32_t* pivot) {
    if (!r) return fail(PSM_ERR_ARG, "null run");
    for (u32 i = 0; i < r->n; ++i) {
        if (order) order[i] = r->hq.order[i];
        if (pivot) pivot[i] = r->hq.pivot[i];
    }
    return PSM_OK;
}

int psm_run_embeddings(psm_run* r, uint32_t* buf, uint64_t buf_rows, uint64_t* rows) {
    if (!r || !rows) return fail(PSM_ERR_ARG, "null argument");
    u64 have = std::min<u64>(r->hq.emit_rows, r->hq.emit_cap_rows);
    *rows = have;
    if (!buf || have == 0) return PSM_OK;
    if (buf_rows < have) return fail(PSM_ERR_ARG, "buffer too small");
    CK(cudaMemcpy(buf, r->hq.emit_buf, have * r->n * sizeof(u32), cudaMemcpyDeviceToHost));
    return PSM_OK;
}

void psm_run_free(psm_run* r) {
    if (!r) return;
    if (r->ctx) r->ctx->run_live = false;
    delete r->hdesc;
    delete r;
}

}  // extern "C"

// ------------------------------------------------------------ join path --

namespace {

// Two-ended allocator over the free part of the arena: relations grow from
// the bottom, per-join temporaries from the top (released after each join).
struct Arena2 {
    char* base;
    size_t lo, hi;  // [lo, hi) is free
    template <class T>
    T* low(size_t count) {
        size_t bytes = align_up(std::max<size_t>(count, 1) * sizeof(T));
        if (lo + bytes > hi) return nullptr;
        T* p = (T*)(base + lo);
        lo += bytes;
        return p;
    }
    template <class T>
    T* high(size_t count) {
        size_t bytes = align_up(std::max<size_t>(count, 1) * sizeof(T));
        if (hi < lo + bytes) return nullptr;
        hi -= bytes;
        return (T*)(base + hi);
    }
};

// A relation of partial embeddings in device memory: n rows of ncols data
// vertex ids; column c holds query vertex vert[c].
struct Rel {
    u32* rows = nullptr;
    u64 n = 0;
    u32 ncols = 0;
    u32 vert[PSM_MAXQ]{};
};

// Joins build side B and probe side P (keys: the query vertices in both).
// count_only: *total receives the number of output rows; otherwise *out
// holds them (probe columns, then B's non-key columns).
int join_rels(psm_context* ctx, Arena2& ar, const u32* label, const Rel& B, const Rel& P, bool count_only, Rel* out,
              u64* total, u64* peak_bytes) {
    JoinSpec sp{};
    sp.bcols = B.ncols;
    sp.pcols = P.ncols;
    for (u32 i = 0; i < B.ncols; ++i) {
        int in_p = -1;
        for (u32 j = 0; j < P.ncols; ++j)
            if (P.vert[j] == B.vert[i]) in_p = (int)j;
        if (in_p >= 0) {
            if (sp.nk >= PSM_JOIN_MAX_KEYS) return fail(PSM_ERR_ARG, "too many join keys");
            sp.bkey[sp.nk] = i;
            sp.pkey[sp.nk] = (u32)in_p;
            ++sp.nk;
        } else {
            u32 same = 0;
            for (u32 j = 0; j < P.ncols; ++j)
                if (!label || label[P.vert[j]] == label[B.vert[i]]) same |= 1u << j;
            sp.bx[sp.nbx] = i;
            sp.bx_same[sp.nbx] = same;
            ++sp.nbx;
        }
    }
    if (P.ncols + sp.nbx > PSM_MAXQ) return fail(PSM_ERR_ARG, "joined rows wider than 32 columns");
    if (B.n >= 0x7FFFFFFFull) return fail(PSM_ERR_OOM, "join build side above 2^31 rows");
    const size_t hi0 = ar.hi;
    u64 cap = 64;
    while (cap < 2 * B.n) cap <<= 1;
    JoinTable t{};
    t.mask = (u32)(cap - 1);
    t.slots = ar.high<u32>(cap);
    t.gcount = ar.high<u32>(cap);
    t.gfill = ar.high<u32>(cap);
    t.goff = ar.high<u64>(cap);
    t.grp = ar.high<u32>(B.n);
    t.members = ar.high<u32>(B.n);
    t.scan_tmp = ar.high<u64>(psm_scan_tmp_bytes(cap) / sizeof(u64) + 1);
    t.error = ar.high<u32>(1);
    u64* d_total = ar.high<u64>(1);
    if (!t.slots || !t.gcount || !t.gfill || !t.goff || !t.grp || !t.members || !t.scan_tmp || !t.error || !d_total)
        return fail(PSM_ERR_OOM, "device arena exhausted (join table)");
    CK(psm_join_build(B.rows, B.n, sp, t, ctx->st));
    CK(cudaMemsetAsync(d_total, 0, sizeof(u64), ctx->st));
    u64 n_out = 0;
    if (count_only) {
        CK(psm_join_probe(P.rows, P.n, B.rows, sp, t, nullptr, nullptr, nullptr, (unsigned long long*)d_total,
                          ctx->st));
        CK(cudaMemcpyAsync(&n_out, d_total, sizeof(u64), cudaMemcpyDeviceToHost, ctx->st));
    } else {
        u32* cnt = ar.high<u32>(P.n);
        u64* off = ar.high<u64>(P.n);
        u64* stmp = ar.high<u64>(psm_scan_tmp_bytes(P.n) / sizeof(u64) + 1);
        if (!cnt || !off || !stmp) return fail(PSM_ERR_OOM, "device arena exhausted (join counts)");
        CK(psm_join_probe(P.rows, P.n, B.rows, sp, t, cnt, nullptr, nullptr, nullptr, ctx->st));
        CK(psm_excl_scan(cnt, P.n, off, stmp, d_total, ctx->st));
        CK(cudaMemcpyAsync(&n_out, d_total, sizeof(u64), cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
        out->ncols = P.ncols + sp.nbx;
        for (u32 j = 0; j < P.ncols; ++j) out->vert[j] = P.vert[j];
        for (u32 x = 0; x < sp.nbx; ++x) out->vert[P.ncols + x] = B.vert[sp.bx[x]];
        out->n = n_out;
        out->rows = ar.low<u32>(n_out * out->ncols);
        if (!out->rows) return fail(PSM_ERR_OOM, "device arena exhausted (joined rows)");
        CK(psm_join_probe(P.rows, P.n, B.rows, sp, t, nullptr, out->rows, off, nullptr, ctx->st));
    }
    u32 err = 0;
    CK(cudaMemcpyAsync(&err, t.error, sizeof(u32), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    if (err) return fail(PSM_ERR_INTERNAL, "join table overflow");
    *total = n_out;
    *peak_bytes = std::max<u64>(*peak_bytes, ar.lo + (hi0 - ar.hi));
    ar.hi = hi0;
    return PSM_OK;
}

// Adjacency masks of a query description (validated like the matching path:
// simple, loop-free edges inside the vertex range).
int query_adjacency(const psm_query_desc& q, u32* adj) {
    if (q.num_vertices == 0 || q.num_vertices > PSM_MAXQ) return fail(PSM_ERR_ARG, "query size out of range");
    for (u32 u = 0; u < q.num_vertices; ++u) adj[u] = 0;
    for (u32 e = 0; e < q.num_edges; ++e) {
        const u32 a = q.edges[2 * e], b = q.edges[2 * e + 1];
        if (a >= q.num_vertices || b >= q.num_vertices || a == b) return fail(PSM_ERR_ARG, "bad query edge");
        adj[a] |= 1u << b;
        adj[b] |= 1u << a;
    }
    return PSM_OK;
}

// The plan as binary joins in execution order (operands: unit k, or
// nunits + i = the result of join i); returns the operand id of `node`.
u32 plan_ops(const Decomposition& d, u32 node, std::vector<u32>& ops) {
    const JoinNode& nd = d.nodes[node];
    if (nd.unit >= 0) return (u32)nd.unit;
    u32 acc = plan_ops(d, nd.child[0], ops);
    for (u32 i = 1; i < nd.nchild; ++i) {
        const u32 r = plan_ops(d, nd.child[i], ops);
        ops.push_back(acc);
        ops.push_back(r);
        acc = d.nunits + (u32)(ops.size() / 2 - 1);
    }
    return acc;
}

}  // namespace

extern "C" {

int psm_query_decompose(const psm_query_desc* q, uint32_t max_unit_vertices, uint32_t* num_units,
                        uint32_t* unit_masks) {
    if (!q || !num_units || !unit_masks) return fail(PSM_ERR_ARG, "null argument");
    u32 adj[PSM_MAXQ], cnt[PSM_MAXQ] = {};
    int rc = query_adjacency(*q, adj);
    if (rc) return rc;
    Decomposition dec;
    std::string err;
    if (psm_decompose(q->num_vertices, adj, cnt, max_unit_vertices, &dec, &err)) return fail(PSM_ERR_ARG, err);
    *num_units = dec.nunits;
    for (u32 k = 0; k < dec.nunits; ++k) unit_masks[k] = dec.units[k].mask;
    return PSM_OK;
}


int psm_query_decompose_ex(const psm_query_desc* q, const psm_join_options* jo, double data_vertices,
                           double data_edges, uint32_t* num_units, uint32_t* unit_masks, uint32_t* num_joins,
                           uint32_t* join_ops) {
    if (!q || !jo || !num_units || !unit_masks) return fail(PSM_ERR_ARG, "null argument");
    u32 adj[PSM_MAXQ], cnt[PSM_MAXQ] = {};
    int rc = query_adjacency(*q, adj);
    if (rc) return rc;
    PlanStats st;
    st.data_vertices = data_vertices;
    st.data_edges = data_edges;
    Decomposition dec;
    std::string err;
    if (psm_decompose_pattern(q->num_vertices, adj, cnt, jo->pattern, jo->join_method, jo->max_unit, st, &dec, &err))
        return fail(PSM_ERR_ARG, err);
    *num_units = dec.nunits;
    for (u32 k = 0; k < dec.nunits; ++k) unit_masks[k] = dec.units[k].mask;
    std::vector<u32> ops;
    plan_ops(dec, dec.root, ops);
    if (num_joins) *num_joins = (u32)(ops.size() / 2);
    if (join_ops)
        for (u32 i = 0; i < ops.size(); ++i) join_ops[i] = ops[i];
    return PSM_OK;
}

int psm_match_join(psm_context* ctx, const psm_graph* g, const psm_query_desc* q, const psm_options* opt,
                   uint32_t max_unit_vertices, psm_join_result* res) {
    const psm_join_options jo{PSM_SPLIT_BOUNDED, PSM_JOIN_LEFTDEEP, max_unit_vertices, 0};
    return psm_match_join_ex(ctx, g, q, opt, &jo, res);
}

int psm_match_join_ex(psm_context* ctx, const psm_graph* g, const psm_query_desc* q, const psm_options* opt,
                      const psm_join_options* jo, psm_join_result* res) {
    if (!ctx || !g || !q || !opt || !res || !jo) return fail(PSM_ERR_ARG, "null argument");
    memset(res, 0, sizeof(*res));
    if (opt->emit) return fail(PSM_ERR_ARG, "the join path counts; emit is not supported");
    u32 adj[PSM_MAXQ];
    int rc = query_adjacency(*q, adj);
    if (rc) return rc;
    // 1. the whole query: filter, tables, order (no enumeration)
    psm_run run;
    psm_result pr{};
    psm_options po = *opt;
    po.cap = 0;
    rc = run_queries(ctx, g, q, 1, po, true, &pr, &run, /*prep_only=*/true);
    struct Release {
        psm_run& r;
        ~Release() {
            if (r.ctx) r.ctx->run_live = false;
            delete r.hdesc;
        }
    } release{run};
    if (rc) return rc;
    res->prep_ms = pr.prep_ms;
    res->memory_bytes = pr.memory_bytes;
    const QState& hq = run.hq;
    const u32 n = q->num_vertices;
    // 2. units and join plan; the cost-based pattern reads the candidate
    // counts and the table sizes (fraction of candidate pairs that are data
    // edges) of the prepared query
    PlanStats st;
    st.data_vertices = g->V;
    st.data_edges = (double)g->nnz / 2;
    std::vector<double> cand(n), edge_p((size_t)n * n, 0.0);
    if (jo->pattern == PSM_SPLIT_COST && !hq.empty) {
        const QDesc& d = *run.hdesc;
        for (u32 u = 0; u < n; ++u) cand[u] = hq.cnt[u];
        for (u32 e = 0; e < d.e_first[n]; ++e) {
            const u32 a = d.e_src[e], b = d.e_dst[e];
            u32 ends[2] = {0, 0};
            CK(cudaMemcpy(&ends[0], hq.P + hq.e_row_base[e], sizeof(u32), cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(&ends[1], hq.P + hq.e_row_base[e] + hq.cnt[a], sizeof(u32), cudaMemcpyDeviceToHost));
            const double pairs = (double)hq.cnt[a] * hq.cnt[b];
            edge_p[(size_t)a * n + b] = pairs > 0 ? (ends[1] - ends[0]) / pairs : 0.0;
        }
        st.cand = cand.data();
        st.edge_p = edge_p.data();
    }
    Decomposition dec;
    std::string err;
    if (psm_decompose_pattern(n, adj, hq.cnt, jo->pattern, jo->join_method, jo->max_unit, st, &dec, &err))
        return fail(PSM_ERR_ARG, err);
    const u32 U = dec.nunits;
    res->units = U;
    for (u32 k = 0; k < U; ++k) res->unit_mask[k] = dec.units[k].mask;
    if (hq.empty) {
        res->status = PSM_OK;
        return PSM_OK;  // some candidate set is empty: no embedding
    }
    Arena2 ar{ctx->arena, run.arena_free, ctx->arena_bytes};
    std::vector<QState> uq(U, hq);
    for (u32 k = 0; k < U; ++k) {
        QState& s = uq[k];
        const UnitPlan& up = dec.units[k];
        for (u32 i = 0; i < PSM_MAXQ; ++i) s.order[i] = i < up.n ? up.order[i] : 0u;
        s.n_enum = up.n;
        s.emit_by_depth = 1;
        s.emit_buf = nullptr;
        s.emit_cap_rows = 0;
        s.emit_rows = 0;
        s.count = s.calls = s.alg_bytes = 0;
        s.cap = 0;
        s.stop = s.overtime = 0;
        s.done_ns = 0;
        s.trace = nullptr;
    }
    QState* d_uq = ar.low<QState>(U);
    char* d_enum_q = ar.low<char>(psm_enum_query_bytes(U));
    DevResult* d_res = ar.low<DevResult>(U);
    u32** d_bufs = ar.low<u32*>(U);
    u64* d_caps = ar.low<u64>(U);
    if (!d_uq || !d_enum_q || !d_res || !d_bufs || !d_caps) return fail(PSM_ERR_OOM, "device arena exhausted (units)");
    const u64 budget = budget_ns(*opt);
    CK(cudaMemcpyAsync(d_uq, uq.data(), sizeof(QState) * U, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaEventRecord(ctx->ev[0], ctx->st));
    CK(psm_launch_unit_plan(g->dev, d_uq, U, ctx->st));
    // 3. count every unit, then emit every unit (one launch each)
    std::vector<DevResult> dr(U);
    auto run_units = [&](int emit) -> int {
        CK(psm_launch_enum(g->dev, d_uq, U, ctx->d_enum_scratch, d_enum_q, budget, emit, ctx->enum_blocks,
                           ctx->d_enum_cache, nullptr, 0, ctx->st, 8u, ctx->tune_isect));
        CK(psm_launch_gather(d_uq, U, d_res, ctx->st));
        CK(cudaMemcpyAsync(dr.data(), d_res, sizeof(DevResult) * U, cudaMemcpyDeviceToHost, ctx->st));
        EnumStats es{};
        CK(psm_enum_read_ctl(ctx->d_enum_scratch, &es, ctx->st));
        if (es.error) return fail(PSM_ERR_INTERNAL, "enumeration wait gave up");
        for (u32 k = 0; k < U; ++k) {
            if (dr[k].overtime) return fail(PSM_ERR_TIMEOUT, "time limit reached (units)");
            if (dr[k].status != PSM_DEV_OK) return fail(PSM_ERR_INTERNAL, "unit enumeration failed");
        }
        return PSM_OK;
    };
    rc = run_units(0);
    if (rc) return rc;
    u64 used = 0;
    for (u32 k = 0; k < U; ++k) res->unit_rows[k] = dr[k].count;
    if (U == 1) {
        CK(cudaEventRecord(ctx->ev[1], ctx->st));
        CK(cudaEventSynchronize(ctx->ev[1]));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
        res->enum_ms = ms;
        res->join_rows[0] = dr[0].count;
        res->count = opt->cap && dr[0].count > opt->cap ? opt->cap : dr[0].count;
        res->status = PSM_OK;
        return PSM_OK;
    }
    std::vector<u32*> bufs(U);
    std::vector<u64> caps(U);
    for (u32 k = 0; k < U; ++k) {
        caps[k] = dr[k].count;
        bufs[k] = ar.low<u32>(dr[k].count * dec.units[k].n);
        if (!bufs[k]) return fail(PSM_ERR_OOM, "device arena exhausted (unit embeddings)");
    }
    CK(cudaMemcpyAsync(d_bufs, bufs.data(), sizeof(u32*) * U, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(d_caps, caps.data(), sizeof(u64) * U, cudaMemcpyHostToDevice, ctx->st));
    CK(psm_launch_unit_emit(d_uq, U, d_bufs, d_caps, ctx->st));
    rc = run_units(1);
    if (rc) return rc;
    for (u32 k = 0; k < U; ++k)
        if (dr[k].emit_rows != caps[k]) return fail(PSM_ERR_INTERNAL, "unit emission differs from its count");
    CK(cudaEventRecord(ctx->ev[1], ctx->st));
    // 4. the joins of the plan, in execution order; the last one is counted
    const u32* label = run.hdesc->label;
    std::vector<u32> ops;
    plan_ops(dec, dec.root, ops);
    const u32 J = (u32)(ops.size() / 2);
    std::vector<Rel> results(J);
    auto operand = [&](u32 id) -> Rel {
        if (id >= U) return results[id - U];
        Rel r;
        r.rows = bufs[id];
        r.n = caps[id];
        r.ncols = dec.units[id].n;
        for (u32 i = 0; i < r.ncols; ++i) r.vert[i] = dec.units[id].order[i];
        return r;
    };
    res->join_rows[0] = caps[ops[0]];
    u64 total = 0;
    for (u32 j = 0; j < J; ++j) {
        const Rel a = operand(ops[2 * j]), b = operand(ops[2 * j + 1]);
        const bool last = j + 1 == J;
        // build on the smaller side
        const bool build_a = a.n <= b.n;
        rc = join_rels(ctx, ar, label, build_a ? a : b, build_a ? b : a, last, &results[j], &total, &used);
        if (rc) return rc;
        if (j + 1 < PSM_MAX_UNITS) res->join_rows[j + 1] = total;
        if (total == 0) break;  // an empty partial result empties the query
    }
    CK(cudaEventRecord(ctx->ev[2], ctx->st));
    CK(cudaEventSynchronize(ctx->ev[2]));
    float e_ms = 0, j_ms = 0;
    CK(cudaEventElapsedTime(&e_ms, ctx->ev[0], ctx->ev[1]));
    CK(cudaEventElapsedTime(&j_ms, ctx->ev[1], ctx->ev[2]));
    res->enum_ms = e_ms;
    res->join_ms = j_ms;
    res->work_bytes = std::max<u64>(used, ar.lo) - run.arena_free;
    res->count = opt->cap && total > opt->cap ? opt->cap : total;
    res->status = PSM_OK;
    return PSM_OK;
}

int psm_hash_join(psm_context* ctx, const uint32_t* r_rows, uint64_t r_n, uint32_t r_cols, const uint32_t* r_vertex,
                  const uint32_t* s_rows, uint64_t s_n, uint32_t s_cols, const uint32_t* s_vertex,
                  const uint32_t* vertex_label, uint32_t* out_rows, uint64_t out_capacity, uint32_t* out_vertex,
                  uint32_t* out_cols, uint64_t* out_n) {
    if (!ctx || !r_vertex || !s_vertex || !out_n || (r_n && !r_rows) || (s_n && !s_rows))
        return fail(PSM_ERR_ARG, "null argument");
    if (r_cols == 0 || s_cols == 0 || r_cols > PSM_MAXQ || s_cols > PSM_MAXQ) return fail(PSM_ERR_ARG, "bad widths");
    for (u32 i = 0; i < r_cols; ++i)
        if (r_vertex[i] >= PSM_MAXQ) return fail(PSM_ERR_ARG, "query vertex id out of range");
    for (u32 i = 0; i < s_cols; ++i)
        if (s_vertex[i] >= PSM_MAXQ) return fail(PSM_ERR_ARG, "query vertex id out of range");
    if (ctx->run_live) return fail(PSM_ERR_ARG, "a psm_run is still alive on this context");
    CK(cudaSetDevice(ctx->device));
    Arena2 ar{ctx->arena, ctx->fixed_bytes, ctx->arena_bytes};
    Rel R, S;
    R.n = r_n;
    R.ncols = r_cols;
    S.n = s_n;
    S.ncols = s_cols;
    for (u32 i = 0; i < r_cols; ++i) R.vert[i] = r_vertex[i];
    for (u32 i = 0; i < s_cols; ++i) S.vert[i] = s_vertex[i];
    R.rows = ar.low<u32>(r_n * r_cols);
    S.rows = ar.low<u32>(s_n * s_cols);
    if (!R.rows || !S.rows) return fail(PSM_ERR_OOM, "device arena exhausted (relations)");
    if (r_n) CK(cudaMemcpyAsync(R.rows, r_rows, r_n * r_cols * sizeof(u32), cudaMemcpyHostToDevice, ctx->st));
    if (s_n) CK(cudaMemcpyAsync(S.rows, s_rows, s_n * s_cols * sizeof(u32), cudaMemcpyHostToDevice, ctx->st));
    u32 lab[PSM_MAXQ] = {};
    if (vertex_label)
        for (u32 i = 0; i < r_cols; ++i) lab[r_vertex[i]] = vertex_label[r_vertex[i]];
    if (vertex_label)
        for (u32 i = 0; i < s_cols; ++i) lab[s_vertex[i]] = vertex_label[s_vertex[i]];
    Rel out;
    u64 total = 0, used = 0;
    int rc = join_rels(ctx, ar, vertex_label ? lab : nullptr, R, S, out_rows == nullptr, &out, &total, &used);
    if (rc) return rc;
    *out_n = total;
    if (!out_rows) return PSM_OK;
    if (out_cols) *out_cols = out.ncols;
    if (out_vertex)
        for (u32 i = 0; i < out.ncols; ++i) out_vertex[i] = out.vert[i];
    if (out_capacity < total) return fail(PSM_ERR_ARG, "output buffer too small");
    if (total) CK(cudaMemcpy(out_rows, out.rows, total * out.ncols * sizeof(u32), cudaMemcpyDeviceToHost));
    return PSM_OK;
}

}  // extern "C"

int psm_batch_polled(psm_context* ctx, const psm_graph* g, const psm_query_desc* qs, u32 nq, const psm_options* opt,
                     psm_result* results, QDoneRec* done_dev, u32 exit_keep, void (*poll)(void*), void* poll_arg) {
    if (!opt || !results) return fail(PSM_ERR_ARG, "null argument");
    return run_queries(ctx, g, qs, nq, *opt, false, results, nullptr, false, done_dev, exit_keep, poll, poll_arg);
}
u32 psm_context_prep_blocks_per_query(const psm_context* ctx, u32 nq) {
    return use_cluster_batch(ctx, nq) ? (u32)ctx->batch_cluster : 1u;
}
