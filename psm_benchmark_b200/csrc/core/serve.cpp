// Serving runtime: a request loop over a resident data graph with
// continuous batching (no counterpart in the reference, which matches one
// query per process; each batch runs the reference's C-mode path).
//
// A server owns `lanes` execution lanes. A lane is a context (its own CUDA
// stream, device arena and enumerator scratch) plus a host thread. Requests
// are copied into an admission queue with an estimate of their device
// memory: candidate bitmaps, ranks and lists, table row offsets, CFL
// estimate buffers and descriptors (exact, as the batched path lays them
// out), and the candidate-edge tables bounded by the data graph's edge
// count between the two labels of each query edge. Whenever a lane is idle
// it admits, in arrival order, every queued request that fits its memory
// budget and the batch limit, and runs them as one batch: one preparation
// launch (a block per query) and one persistent enumeration launch. Requests
// that arrive while other lanes' batches are on the GPU are admitted by the
// next lane that frees up, so the work of several batches overlaps on the
// device. Each query's result leaves as soon as its own last enumeration task
// ends: the enumerator writes a completion record into host-mapped memory,
// which the lane thread polls while its batch runs; with several lanes, idle
// warps of a batch leave the GPU once no work is left so that the next
// batch's launches get the SMs. A batch whose tables outgrow the estimate is
// rerun query by query.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "host.h"

namespace {

u64 now_ns() {
    return (u64)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

size_t al(size_t x) { return (x + 255) / 256 * 256; }

struct Request {
    u64 ticket = 0;
    std::vector<u32> labels, edges;
    u64 est = 0;
    u64 submit_ns = 0;
};

}  // namespace

struct Lane {
    psm_context* ctx = nullptr;
    u64 tune_gen = 0;              // the server's tuning generation this lane's context has
    QDoneRec* rec_host = nullptr;  // host-mapped completion records [max_batch]
    QDoneRec* rec_dev = nullptr;
};

struct psm_server {
    int device = 0;
    const psm_graph* g = nullptr;
    psm_options opt{};
    psm_server_config cfg{};
    u64 budget = 0;  // admission budget per lane (arena bytes minus the fixed region)
    u32 prep_blocks = 1;  // largest number of blocks that prepare one query
    std::vector<Lane> lanes;
    std::vector<std::thread> threads;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request> queue;
    std::vector<psm_request_result> done;
    u64 next_ticket = 1;
    u64 running = 0;
    bool stopping = false;
    psm_batch_tuning tune{};  // psm_server_set_batch_tuning: applied by each lane before its next batch
    u64 tune_gen = 0;
};

namespace {

// Device bytes a query takes in a batch (see the file comment); prep_blocks:
// blocks preparing one query (each keeps its own CFL path-estimate buffers).
u64 estimate_bytes(const psm_graph& g, const psm_query_desc& q, const psm_options& opt, u32 prep_blocks) {
    const u32 n = q.num_vertices;
    u64 b = al(sizeof(QState)) + al(sizeof(QDesc)) + al(sizeof(DevResult)) + 64;
    u64 maxw = 1, maxb = 1, rows = 0;
    std::vector<u32> deg(n, 0);
    for (u32 e = 0; e < q.num_edges; ++e) {
        deg[q.edges[2 * e]]++;
        deg[q.edges[2 * e + 1]]++;
    }
    for (u32 u = 0; u < n; ++u) {
        const u64 B = g.freq(q.labels[u]), W = (B + 31) / 32;
        b += 2 * al(4 * std::max<u64>(W, 1)) + al(4 * std::max<u64>(B, 1));
        maxw = std::max(maxw, W);
        maxb = std::max(maxb, B);
        rows += B * deg[u];
    }
    b += 2 * al(4 * maxw) + al(4 * (rows + 1)) + al(4ull * (prep_blocks + 1) * std::max(n, 2u));
    if (opt.order == PSM_ORDER_CFL) b += al(8ull * 2 * prep_blocks * maxb) + al(8ull * PSM_PLAN_WORDS);
    for (u32 e = 0; e < q.num_edges; ++e) {
        const u32 la = q.labels[q.edges[2 * e]], lb = q.labels[q.edges[2 * e + 1]];
        b += 4 * (g.pair_edges(la, lb) + g.pair_edges(lb, la));
    }
    return b + b / 8;
}

void finish(psm_server* s, const Request& r, const psm_result& res, int status, u64 t0, u64 t1, u32 bs, u32 lane) {
    psm_request_result o{};
    o.ticket = r.ticket;
    o.count = res.count;
    o.status = (u32)status;
    o.overtime = res.overtime;
    o.submit_ns = r.submit_ns;
    o.start_ns = t0;
    o.done_ns = t1;
    o.batch_size = bs;
    o.lane = lane;
    o.prep_ms = res.prep_ms;
    o.enum_ms = res.enum_ms;
    s->done.push_back(o);
}

// Poll state of a lane's running batch.
struct Inflight {
    psm_server* s;
    Lane* ln;
    std::vector<Request>* batch;
    std::vector<char> sent;
    u64 t0;
    u32 lane;
    u32 base;  // first record of this (sub)batch
    u32 n;
};

void poll_records(void* arg) {
    auto* f = (Inflight*)arg;
    std::vector<u32> fresh;
    for (u32 i = 0; i < f->n; ++i) {
        if (f->sent[f->base + i]) continue;
        // a query whose preparation failed is reported from the batch's results
        if (*(volatile u32*)&f->ln->rec_host[i].flag && f->ln->rec_host[i].status == PSM_DEV_OK) fresh.push_back(i);
    }
    if (fresh.empty()) return;
    std::atomic_thread_fence(std::memory_order_acquire);  // record fields after their flag
    const u64 t1 = now_ns();
    std::lock_guard<std::mutex> lk(f->s->mu);
    for (u32 i : fresh) {
        const QDoneRec& r = f->ln->rec_host[i];
        psm_result res{};
        res.count = r.count;
        res.overtime = r.overtime;
        finish(f->s, (*f->batch)[f->base + i], res, r.overtime ? PSM_ERR_TIMEOUT : PSM_OK, f->t0, t1,
               (u32)f->n, f->lane);
        f->sent[f->base + i] = 1;
    }
    f->s->cv_done.notify_all();
}

void lane_loop(psm_server* s, u32 lane) {
    cudaSetDevice(s->device);
    Lane& ln = s->lanes[lane];
    psm_context* ctx = ln.ctx;
    const u32 keep = s->cfg.lanes > 1 ? (u32)std::max(8, psm_context_enum_warps(ctx) / 16) : 0u;
    psm_batch_tuning tune{};
    bool retune = false;
    for (;;) {
        std::vector<Request> batch;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] { return s->stopping || !s->queue.empty(); });
            if (s->stopping) return;
            u64 used = 0;
            while (!s->queue.empty() && batch.size() < s->cfg.max_batch) {
                const Request& r = s->queue.front();
                if (r.est > s->budget) {
                    // never fits a lane: fail it now
                    finish(s, r, psm_result{}, PSM_ERR_OOM, now_ns(), now_ns(), 0, lane);
                    s->queue.pop_front();
                    s->cv_done.notify_all();
                    continue;
                }
                if (used + r.est > s->budget) break;
                used += r.est;
                batch.push_back(std::move(s->queue.front()));
                s->queue.pop_front();
            }
            if (batch.empty()) continue;
            s->running += batch.size();
            if (ln.tune_gen != s->tune_gen) {
                tune = s->tune;
                retune = true;
                ln.tune_gen = s->tune_gen;
            }
        }
        // the lane's own thread changes its context's settings, between batches
        if (retune) psm_context_set_batch_tuning(ctx, &tune);
        retune = false;
        const u64 t0 = now_ns();
        std::vector<psm_query_desc> qs(batch.size());
        for (size_t i = 0; i < batch.size(); ++i)
            qs[i] = psm_query_desc{(u32)batch[i].labels.size(), (u32)(batch[i].edges.size() / 2),
                                   batch[i].labels.data(), batch[i].edges.data()};
        std::vector<psm_result> res(batch.size());
        Inflight f{s, &ln, &batch, std::vector<char>(batch.size(), 0), t0, lane, 0, (u32)batch.size()};
        memset(ln.rec_host, 0, sizeof(QDoneRec) * batch.size());
        int rc = psm_batch_polled(ctx, s->g, qs.data(), (u32)qs.size(), &s->opt, res.data(), ln.rec_dev, keep,
                                  poll_records, &f);
        std::vector<int> st(batch.size(), rc);
        if (rc == PSM_ERR_OOM && batch.size() > 1) {
            // the tables outgrew the estimate: one query at a time
            for (size_t i = 0; i < batch.size(); ++i) {
                if (f.sent[i]) continue;
                memset(ln.rec_host, 0, sizeof(QDoneRec));
                f.base = (u32)i;
                f.n = 1;
                st[i] = psm_batch_polled(ctx, s->g, &qs[i], 1, &s->opt, &res[i], ln.rec_dev, keep, poll_records, &f);
            }
        } else if (rc == PSM_OK || rc == PSM_ERR_TIMEOUT) {
            for (size_t i = 0; i < batch.size(); ++i) st[i] = (int)res[i].status;
        }
        const u64 t1 = now_ns();
        {
            std::lock_guard<std::mutex> lk(s->mu);
            for (size_t i = 0; i < batch.size(); ++i)
                if (!f.sent[i]) finish(s, batch[i], res[i], st[i], t0, t1, (u32)batch.size(), lane);
            s->running -= batch.size();
        }
        s->cv_done.notify_all();
    }
}

}  // namespace

extern "C" {

int psm_server_create(int device, const psm_graph* g, const psm_options* opt, const psm_server_config* cfg,
                      psm_server** out) {
    if (!g || !opt || !cfg || !out) return psm_fail(PSM_ERR_ARG, "null argument");
    if (cfg->lanes == 0 || cfg->lanes > 16 || cfg->max_batch == 0) return psm_fail(PSM_ERR_ARG, "bad server config");
    if (opt->emit) return psm_fail(PSM_ERR_ARG, "the server counts; emit is not supported");
    auto* s = new psm_server;
    s->device = device;
    s->g = g;
    s->opt = *opt;
    s->cfg = *cfg;
    auto cleanup = [&]() {
        for (auto& x : s->lanes) {
            if (x.ctx) psm_context_free(x.ctx);
            if (x.rec_host) cudaFreeHost(x.rec_host);
        }
        delete s;
    };
    for (u32 l = 0; l < cfg->lanes; ++l) {
        Lane ln;
        int rc = psm_context_create(device, cfg->lane_arena_bytes, &ln.ctx);
        if (rc) {
            cleanup();
            return rc;
        }
        if (cfg->lanes > 1 && !cfg->full_gpu_lanes) psm_context_share_gpu(ln.ctx, cfg->lanes);
        cudaError_t e = cudaHostAlloc((void**)&ln.rec_host, sizeof(QDoneRec) * cfg->max_batch,
                                      cudaHostAllocMapped | cudaHostAllocPortable);
        if (e == cudaSuccess) e = cudaHostGetDevicePointer((void**)&ln.rec_dev, ln.rec_host, 0);
        s->lanes.push_back(ln);
        if (e != cudaSuccess) {
            cleanup();
            return psm_fail(PSM_ERR_CUDA, std::string("completion records: ") + cudaGetErrorString(e));
        }
    }
    s->budget = psm_context_free_bytes(s->lanes[0].ctx);
    s->prep_blocks = psm_context_prep_blocks_per_query(s->lanes[0].ctx, 1);
    for (u32 l = 0; l < cfg->lanes; ++l) s->threads.emplace_back(lane_loop, s, l);
    *out = s;
    return PSM_OK;
}

int psm_server_submit(psm_server* s, const psm_query_desc* q, uint64_t* ticket) {
    if (!s || !q || !ticket || !q->labels || (q->num_edges && !q->edges)) return psm_fail(PSM_ERR_ARG, "null argument");
    if (q->num_vertices == 0 || q->num_vertices > PSM_MAX_QUERY_VERTICES)
        return psm_fail(PSM_ERR_ARG, "query size out of range");
    Request r;
    r.labels.assign(q->labels, q->labels + q->num_vertices);
    r.edges.assign(q->edges, q->edges + 2ull * q->num_edges);
    for (u32 x : r.edges)
        if (x >= q->num_vertices) return psm_fail(PSM_ERR_ARG, "edge endpoint out of range");
    r.est = estimate_bytes(*s->g, *q, s->opt, s->prep_blocks);
    r.submit_ns = now_ns();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        r.ticket = s->next_ticket++;
        *ticket = r.ticket;
        s->queue.push_back(std::move(r));
    }
    s->cv_work.notify_one();
    return PSM_OK;
}

int psm_server_poll(psm_server* s, psm_request_result* out, uint32_t max, uint32_t* n, double wait_s) {
    if (!s || !n || (max && !out)) return psm_fail(PSM_ERR_ARG, "null argument");
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->done.empty() && wait_s > 0)
        s->cv_done.wait_for(lk, std::chrono::duration<double>(wait_s), [&] { return !s->done.empty(); });
    const u32 k = (u32)std::min<size_t>(max, s->done.size());
    for (u32 i = 0; i < k; ++i) out[i] = s->done[i];
    s->done.erase(s->done.begin(), s->done.begin() + k);
    *n = k;
    return PSM_OK;
}

int psm_server_pending(psm_server* s, uint64_t* queued, uint64_t* running) {
    if (!s) return psm_fail(PSM_ERR_ARG, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    if (queued) *queued = s->queue.size();
    if (running) *running = s->running;
    return PSM_OK;
}

int psm_server_estimate(psm_server* s, const psm_query_desc* q, uint64_t* bytes, uint64_t* lane_budget) {
    if (!s || !q || !bytes) return psm_fail(PSM_ERR_ARG, "null argument");
    *bytes = estimate_bytes(*s->g, *q, s->opt, s->prep_blocks);
    if (lane_budget) *lane_budget = s->budget;
    return PSM_OK;
}

int psm_server_set_batch_tuning(psm_server* s, const psm_batch_tuning* t) {
    if (!s || !t) return psm_fail(PSM_ERR_ARG, "null argument");
    int rc = psm_batch_tuning_check(s->lanes[0].ctx, t);
    if (rc) return rc;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->tune = *t;
        s->tune_gen += 1;
    }
    return PSM_OK;
}

uint64_t psm_server_clock_ns(void) { return now_ns(); }

void psm_server_destroy(psm_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
    }
    s->cv_work.notify_all();
    for (auto& t : s->threads) t.join();
    for (auto& ln : s->lanes) {
        psm_context_free(ln.ctx);
        cudaFreeHost(ln.rec_host);
    }
    delete s;
}

}  // extern "C"
