/*
 * psm_b200.h - C ABI of the B200 (sm_100a) subgraph-matching engine.
 *
 * Drop-in for the hot path of PSM_Benchmark (reference project), which has
 * no plugin registry: its boundary is the static C++ API that
 * matching/StudyPerformance.cpp drives and the SubgraphMatching.out command
 * line. Each entry point below names the reference interface it replaces.
 * Plain pointers and sizes only; every call returns a psm_status; nothing
 * throws across the boundary. A context owns one CUDA stream and one device
 * arena; calls on one context must not overlap (use one context per host
 * thread), graphs may be shared by contexts on the same device.
 */
#ifndef PSM_B200_H
#define PSM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum psm_status {
    PSM_OK = 0,
    PSM_ERR_ARG = 1,      /* invalid argument / unsupported query          */
    PSM_ERR_OOM = 2,      /* device arena or device memory exhausted        */
    PSM_ERR_TIMEOUT = 3,  /* time limit hit: counts are partial (Overtime 1) */
    PSM_ERR_CUDA = 4,     /* CUDA runtime error, or no usable sm_100 device */
    PSM_ERR_IO = 5,       /* file could not be read                         */
    PSM_ERR_INTERNAL = 9  /* a device-side wait gave up / invariant broken  */
} psm_status;

enum { PSM_FILTER_NLF = 0, PSM_FILTER_GQL = 1, PSM_FILTER_CFL = 2 };
enum { PSM_ORDER_GQL = 0, PSM_ORDER_CFL = 1 };
/* Engines of the reference. All count the same embeddings; every engine is
 * served by the one set-intersection enumerator. */
enum { PSM_ENGINE_LFTJ = 0, PSM_ENGINE_GQL = 1, PSM_ENGINE_EXPLORE = 2 };

#define PSM_MAX_QUERY_VERTICES 32

typedef struct psm_graph psm_graph;
typedef struct psm_context psm_context;
typedef struct psm_run psm_run;

/* A query graph: labels[num_vertices], undirected edges as pairs
 * (edges[2i], edges[2i+1]), vertex ids 0..num_vertices-1. Must be connected
 * and simple, with at most PSM_MAX_QUERY_VERTICES vertices. */
typedef struct psm_query_desc {
    uint32_t num_vertices;
    uint32_t num_edges;
    const uint32_t* labels;
    const uint32_t* edges;
} psm_query_desc;

typedef struct psm_options {
    uint32_t filter;          /* PSM_FILTER_*  (-BackMethods field 1) */
    uint32_t order;           /* PSM_ORDER_*   (field 2)              */
    uint32_t engine;          /* PSM_ENGINE_*  (field 3)              */
    uint32_t emit;            /* 1: also materialise embeddings       */
    uint64_t cap;             /* -num; 0 = no cap (MAX)               */
    double time_limit_s;      /* -time_limit; <= 0 means 60           */
    uint64_t emit_capacity;   /* rows of embeddings kept when emit=1  */
} psm_options;

typedef struct psm_result {
    uint64_t count;           /* #Embeddings = min(total, cap)                  */
    uint64_t calls;           /* extension candidates examined                  */
    uint64_t memory_bytes;    /* candidates + tables, computeMemoryCostInBytes */
    uint64_t table_entries;   /* entries over all candidate-edge tables         */
    uint64_t alg_bytes;       /* algorithmic bytes read by the intersections    */
    uint64_t donations;       /* work-stealing donations during enumeration     */
    uint32_t overtime;        /* 1 if the time limit was hit                    */
    uint32_t filter_ok;       /* 0 if a candidate set came out empty            */
    uint32_t status;          /* psm_status of this query                       */
    uint32_t reserved;
    double prep_ms;           /* device time of filter + tables + order         */
    double enum_ms;           /* device time of the enumeration                 */
    uint64_t h2d_bytes;       /* host->device bytes of the call (its share)     */
    uint64_t d2h_bytes;       /* device->host bytes of the call (its share)     */
    uint64_t tasks;           /* enumeration tasks run (launch-wide)            */
    uint64_t idle_polls;      /* polls of idle warps waiting for work           */
    uint64_t count_internal;  /* embeddings the enumerator counted (unclamped:
                                 >= count when the cap stopped the query; the
                                 work and alg_bytes above correspond to it) */
} psm_result;

const char* psm_status_string(int status);
/* Message of the last failing call on this thread ("" if none). */
const char* psm_last_error(void);
/* Library / device banner, e.g. for the CLI log. */
const char* psm_version(void);

/* ---- data graph (replaces Graph::loadGraphFromFile, graph/graph.cpp:92-172,
 *      and the label index / NLF built by graph.cpp:15-52) ---- */
int psm_graph_from_csr(const uint32_t* offsets, const uint32_t* neighbors, const uint32_t* labels,
                       uint32_t num_vertices, psm_graph** out);
int psm_graph_load(const char* path, psm_graph** out); /* reference text format */
/* The reference's binary graph format (Graph::loadGraphFromFileCompressed,
 * graph/graph.cpp:221-310): degree file (int32 4, uint32 |V|, uint32 |E|,
 * uint32 degree[|V|]), adjacency file (uint32 neighbours row by row), label
 * file (uint32 label[|V|]). */
int psm_graph_load_binary(const char* degree_path, const char* adjacency_path, const char* label_path,
                          psm_graph** out);
/* Writes an undirected CSR in that format (Graph::storeComparessedGraph,
 * graph/graph.cpp:355-403). Host only. */
int psm_graph_store_binary(const uint32_t* offsets, const uint32_t* neighbors, const uint32_t* labels,
                           uint32_t num_vertices, const char* degree_path, const char* adjacency_path,
                           const char* label_path);
/* Text graph -> <prefix>_deg.bin, <prefix>_adj.bin, <prefix>_label.bin
 * (replaces matching/GraphConverter.cpp). Host only. */
int psm_graph_convert(const char* text_path, const char* out_prefix);
/* Edge list ("u v" per line, '#' comments) -> <prefix>_deg.bin, _adj.bin,
 * _label.bin (replaces matching/EdgeListToCSR.cpp, run there as
 * EdgeListConverter.out <edge list> <prefix> <number of labels>). Pairs are
 * stored smaller id first and sorted; duplicates are kept; a self loop fails
 * with nothing written. Labels are uniform over [0, num_labels) from
 * std::mt19937 seeded with `seed` (the reference draws its seed from
 * std::random_device). Host only. */
int psm_graph_convert_edgelist(const char* edge_list_path, const char* out_prefix, uint32_t num_labels,
                               uint64_t seed);
int psm_graph_info(const psm_graph* g, uint32_t* num_vertices, uint64_t* num_edges, uint32_t* num_labels,
                   uint32_t* max_degree, uint32_t* max_label_frequency);
void psm_graph_free(psm_graph* g);

/* ---- execution context: stream + device arena ---- */
int psm_context_create(int device, uint64_t arena_bytes, psm_context** out);
void psm_context_free(psm_context* ctx);

/* ---- plain path: one query on the whole GPU (replaces the per-query body of
 *      split_C_test, matching/StudyPerformance.cpp:1150-1781: FilterVertices::
 *      {NLF,GQL,CFL}Filter + sortCandidates, BuildTable::buildTables,
 *      GenerateQueryPlan::generate{GQL,CFL}QueryPlan, EvaluateQuery::
 *      ParallelExecute with the LFTJ/GQL/EXPLORE engine) ---- */
int psm_match(psm_context* ctx, const psm_graph* g, const psm_query_desc* q, const psm_options* opt,
              psm_result* res);

/* Same as psm_match but keeps the query's device state for inspection until
 * psm_run_free (one live run per context). */
int psm_run_create(psm_context* ctx, const psm_graph* g, const psm_query_desc* q, const psm_options* opt,
                   psm_run** out, psm_result* res);
/* Sorted candidate set of query vertex u in original data ids
 * (the reference's candidates[u] after sortCandidates). */
int psm_run_candidates(psm_run* run, uint32_t u, uint32_t* buf, uint32_t buf_len, uint32_t* n);
/* Candidate-edge table T[a][b] (the reference's Edges edge_matrix[a][b]):
 * offsets[rows+1] and entries[nnz], positions into candidates of b. */
int psm_run_table(psm_run* run, uint32_t a, uint32_t b, uint32_t* offsets, uint32_t offsets_len,
                  uint32_t* entries, uint32_t entries_len, uint32_t* rows, uint32_t* nnz);
/* Matching order and pivots (UnitArgs::order / pivots). */
int psm_run_order(psm_run* run, uint32_t* order, uint32_t* pivot);
/* Embeddings of an emit run: rows of num_vertices original ids, indexed by
 * query vertex. */
int psm_run_embeddings(psm_run* run, uint32_t* buf, uint64_t buf_rows, uint64_t* rows);
void psm_run_free(psm_run* run);

/* No counterpart in the reference. Re-counts the embeddings of a prepared
 * run (psm_run_create with emit = 0) without allocating: for callers that
 * cannot allocate device memory at this point (serving loops that must not
 * take an allocation's implicit device synchronisation, hosts whose device
 * memory belongs to another runtime's pool). The enumeration's scratch lives
 * in a static 1 MiB device array per GPU, held until process exit; the first
 * call on a device looks up that array's address, so make it before any
 * stream capture begins. The call runs on the run's context stream and waits
 * for it. All calls share the array: calls whose work overlaps on the GPU
 * race and must not be issued. A run whose preparation failed is refused with
 * that status (PSM_ERR_OOM / _TIMEOUT / _INTERNAL). Writes min(total, cap) to
 * *count (cap 0 = none). */
int psm_run_recount_noalloc(psm_run* run, uint64_t cap, double time_limit_s, uint64_t* count, uint32_t* overtime);

/* ---- decomposition + join path (replaces split_Q_test,
 *      matching/StudyPerformance.cpp:100-1037: SplitGraph units
 *      (utility/splitGraph/SplitGraph.cpp:23-36), per-unit enumeration into
 *      PartialMatch relations (Args.cpp:162-166), JoinCollect::sequence_collect
 *      (matching/JoinCollect.cpp:237-315) with NoPartitionHashJoin
 *      (utility/hashjoin/hashjoin.cpp:337-779)) ---- */
#define PSM_MAX_UNITS 32
typedef struct psm_join_result {
    uint64_t count;                      /* #Embeddings = rows of the last join (min with the cap) */
    uint32_t units;                      /* decomposition units */
    uint32_t status;                     /* psm_status */
    uint32_t unit_mask[PSM_MAX_UNITS];   /* query vertices of each unit (bit mask) */
    uint64_t unit_rows[PSM_MAX_UNITS];   /* embeddings of each unit */
    uint64_t join_rows[PSM_MAX_UNITS];   /* rows after joining units 0..k (join_rows[0] = unit_rows[0]) */
    double prep_ms;                      /* device time: filter + tables + order of the whole query */
    double enum_ms;                      /* device time: counting and emitting the units */
    double join_ms;                      /* device time: the hash joins */
    uint64_t work_bytes;                 /* device bytes of unit relations and join buffers */
    uint64_t memory_bytes;               /* computeMemoryCostInBytes of the whole query */
} psm_join_result;
/* Filters the whole query and builds its tables (as the reference does in Q
 * mode), splits it into connected units of at most max_unit_vertices
 * vertices (every query edge in some unit), enumerates every unit on the
 * query's candidates and tables, materialises the unit embeddings and joins
 * them left-deep on their shared query vertices with device hash tables
 * (load factor <= 0.5), keeping only injective rows; the last join is
 * counted, not materialised. opt->cap applies to the final count. */
int psm_match_join(psm_context* ctx, const psm_graph* g, const psm_query_desc* q, const psm_options* opt,
                   uint32_t max_unit_vertices, psm_join_result* res);
/* Decomposition patterns of the join path: the reference's -Qpattern values
 * (matching/StudyPerformance.cpp:429-437, utility/splitGraph/SplitGraph.cpp:
 * split_star :895, split_twintwig :875 with optimalDecomposition :671-872,
 * split_seed :913, split_hybrid_rnd :38-108) and two of this library's own
 * that bound the unit size. */
typedef enum psm_split_pattern {
    PSM_SPLIT_BOUNDED = 0,    /* connected units of at most max_unit vertices (psm_match_join) */
    PSM_SPLIT_STAR = 1,       /* stars around a vertex cover (max_unit > 1 splits larger stars) */
    PSM_SPLIT_TWINTWIG = 2,   /* units of one or two edges sharing a vertex, chosen by the card() cost model */
    PSM_SPLIT_SEED = 3,       /* twin-twigs, triangles where the query closes them */
    PSM_SPLIT_SKETCHTREE = 4, /* root-to-leaf paths of a depth-first tree, joined along the tree */
    PSM_SPLIT_COST = 5        /* bounded units and join tree of least estimated materialised rows */
} psm_split_pattern;
/* Join paradigms (the reference's -JoinMethod LEFTDEEP / BUSHY,
 * StudyPerformance.cpp:421-426); SKETCHTREE always joins along its tree
 * (JoinCollect::recur_collect, matching/JoinCollect.cpp:156-235). */
typedef enum psm_join_method { PSM_JOIN_LEFTDEEP = 0, PSM_JOIN_BUSHY = 1 } psm_join_method;
typedef struct psm_join_options {
    uint32_t pattern;      /* psm_split_pattern */
    uint32_t join_method;  /* psm_join_method */
    uint32_t max_unit;     /* unit bound of BOUNDED / COST (required) and STAR (0 = none) */
    uint32_t reserved;
} psm_join_options;
/* psm_match_join with a chosen decomposition pattern and join paradigm
 * (replaces split_Q_test's SplitGraph + sequence_collect / recur_collect).
 * res->join_rows[j] = rows out of the j-th join executed (join_rows[0] =
 * the first unit evaluated); the last join is counted, not materialised. */
int psm_match_join_ex(psm_context* ctx, const psm_graph* g, const psm_query_desc* q, const psm_options* opt,
                      const psm_join_options* jo, psm_join_result* res);
/* The decomposition and join plan psm_match_join_ex would use, on the host
 * (COST and the twin-twig searches then use the reference's label-blind
 * card model with data_vertices / data_edges): unit_masks[PSM_MAX_UNITS];
 * the plan as binary joins in execution order, join_ops[2 * j] and
 * join_ops[2 * j + 1] naming the operands of join j (a unit k < num_units,
 * or num_units + i = the result of join i); join_ops needs room for
 * 2 * (PSM_MAX_UNITS - 1) entries (num_joins <= PSM_MAX_UNITS - 1). */
int psm_query_decompose_ex(const psm_query_desc* q, const psm_join_options* jo, double data_vertices,
                           double data_edges, uint32_t* num_units, uint32_t* unit_masks, uint32_t* num_joins,
                           uint32_t* join_ops);
/* The decomposition psm_match_join uses (host only): *num_units units,
 * unit_masks[PSM_MAX_UNITS] their vertex sets. */
int psm_query_decompose(const psm_query_desc* q, uint32_t max_unit_vertices, uint32_t* num_units,
                        uint32_t* unit_masks);
/* One hash join of host relations (replaces JoinCollect::concateTwoTabels,
 * matching/JoinCollect.cpp:60-153): rows of r_cols / s_cols data vertex ids,
 * column c of R holds query vertex r_vertex[c] (likewise S). Keys are the
 * query vertices in both; R is the build side, S probes. An output row is
 * S's columns then R's non-key columns (out_vertex / *out_cols describe
 * them), kept iff no R non-key value occurs in the S row among columns of
 * the same label (vertex_label[query vertex]; NULL = one label for all).
 * out_rows == NULL counts only; otherwise out_capacity rows must suffice
 * (else PSM_ERR_ARG with *out_n set to the count). */
int psm_hash_join(psm_context* ctx, const uint32_t* r_rows, uint64_t r_n, uint32_t r_cols, const uint32_t* r_vertex,
                  const uint32_t* s_rows, uint64_t s_n, uint32_t s_cols, const uint32_t* s_vertex,
                  const uint32_t* vertex_label, uint32_t* out_rows, uint64_t out_capacity, uint32_t* out_vertex,
                  uint32_t* out_cols, uint64_t* out_n);
/* ---- batched path: many queries through one persistent preparation launch
 *      and one persistent enumeration launch (no counterpart in the
 *      reference, which runs queries one process at a time) ---- */
int psm_match_batch(psm_context* ctx, const psm_graph* g, const psm_query_desc* qs, uint32_t nq,
                    const psm_options* opt, psm_result* results);

/* Settings of a context's batched launches (psm_match_batch and the serving
 * lanes; no counterpart in the reference). */
#define PSM_TEAM_RULE 0     /* a cluster per query for small batches, a block per query for large ones */
#define PSM_TEAM_BLOCK 1    /* one thread block prepares each query */
#define PSM_TEAM_CLUSTER 2  /* one thread-block cluster prepares each query */
/* Intersection variants of the enumerator (the reference's
 * ComputeSetIntersection::ComputeCandidates picks galloping for skewed
 * pairs and a merge for balanced ones, utility/computesetintersection.cpp:5-30).
 * They change the work, never the counts. */
#define PSM_ISECT_BINARY 0  /* binary search of every entry of the shorter array, whole range (the
                               default of a new context: the fastest on every workload measured) */
#define PSM_ISECT_AUTO 1    /* per intersection, by its dependent loads: warp merge path for balanced
                               arrays, binary search of the shorter array in the longer one for skewed
                               ones, a two-cursor merge or a shrinking search for one lane's walk */
#define PSM_ISECT_MERGE 2   /* merge wherever both arrays are non-empty */
typedef struct psm_batch_tuning {
    uint32_t team;            /* PSM_TEAM_*: preparation team of a query */
    uint32_t grabs_per_warp;  /* 1..64: how finely a query's initial work is cut, per enumeration warp */
    uint32_t enum_quarters;   /* 1..4: enumeration grid in quarters of the co-resident blocks */
    uint32_t intersect;       /* PSM_ISECT_*: every enumeration launch of the context (plain, batched,
                                 join units, serving lanes) */
    double ms;                /* psm_autotune_batch: device time of the sample under this setting */
} psm_batch_tuning;
int psm_context_set_batch_tuning(psm_context* ctx, const psm_batch_tuning* t);
int psm_context_get_batch_tuning(psm_context* ctx, psm_batch_tuning* t);
/* Autotuner of the batched path: runs the sample batch under every candidate
 * setting (teams x grabs_per_warp {2, 8, 32} x enum_quarters {2, 4} under the
 * installed intersection variant, then the other intersection variants under
 * the best of those), keeps the one with the least device time (the best of
 * `repeats` runs after one warm-up), installs it in the context and returns
 * it in *best; every setting tried is written to tried[0 .. *ntried) (up to
 * tried_cap). The counts of every setting must be equal (PSM_ERR_INTERNAL
 * otherwise). */
int psm_autotune_batch(psm_context* ctx, const psm_graph* g, const psm_query_desc* sample, uint32_t n,
                       const psm_options* opt, uint32_t repeats, psm_batch_tuning* best, psm_batch_tuning* tried,
                       uint32_t tried_cap, uint32_t* ntried);

/* ---- serving: request loop with continuous batching over a resident graph
 *      (no counterpart in the reference, which runs one query per process) ---- */
typedef struct psm_server psm_server;
typedef struct psm_server_config {
    uint32_t lanes;             /* concurrent batches: each lane has its own stream, arena, enumerator */
    uint32_t max_batch;         /* queries per batch */
    uint64_t lane_arena_bytes;  /* device arena per lane; requests are admitted within it */
    uint32_t full_gpu_lanes;    /* 1: every lane's launches may fill the whole GPU; 0: grids of 1/lanes */
    uint32_t reserved;
} psm_server_config;
typedef struct psm_request_result {
    uint64_t ticket;
    uint64_t count;             /* #Embeddings = min(total, cap) */
    uint32_t status;            /* psm_status of the request */
    uint32_t overtime;
    uint64_t submit_ns;         /* psm_server_clock_ns() stamps */
    uint64_t start_ns;          /* its batch started */
    uint64_t done_ns;           /* its batch finished */
    uint32_t batch_size;        /* queries in its batch */
    uint32_t lane;
    double prep_ms;             /* device time of its batch's preparation */
    double enum_ms;             /* device time of its batch's enumeration */
} psm_request_result;
/* Starts the lanes (threads) of a server for graph g (which must outlive it)
 * with the method, cap and time limit of *opt. */
int psm_server_create(int device, const psm_graph* g, const psm_options* opt, const psm_server_config* cfg,
                      psm_server** out);
/* Queues a copy of the query; *ticket identifies its result. */
int psm_server_submit(psm_server* s, const psm_query_desc* q, uint64_t* ticket);
/* Takes up to max finished results, waiting up to wait_s seconds for one. */
int psm_server_poll(psm_server* s, psm_request_result* out, uint32_t max, uint32_t* n, double wait_s);
/* Requests queued (not admitted) and running. */
int psm_server_pending(psm_server* s, uint64_t* queued, uint64_t* running);
/* The device memory a request is admitted with, and a lane's budget. */
int psm_server_estimate(psm_server* s, const psm_query_desc* q, uint64_t* bytes, uint64_t* lane_budget);
uint64_t psm_server_clock_ns(void);
/* Settings of every lane's batches (psm_batch_tuning, e.g. from
 * psm_autotune_batch on a context of the same device; enum_quarters < 4 leaves
 * SMs free for the other lanes' launches): each lane applies them before its
 * next batch. Lanes start with a new context's settings. */
int psm_server_set_batch_tuning(psm_server* s, const psm_batch_tuning* t);
/* Finishes the running batches and stops; queued requests are dropped. */
void psm_server_destroy(psm_server* s);

/* ---- self-check of the enumerator's intersection primitives (test support;
 *      no counterpart in the reference) ----
 * One warp on the current device intersects the ascending arrays a[0, na)
 * and b[0, nb) (distinct values below 0xFFFFFFFF each) in every form the
 * enumerator uses: counts[0] = |a ∩ b| by warp merge path, counts[1] by one
 * lane's two-cursor merge, counts[2] by one lane's search, counts[3] = the
 * entries of the merge path with output written to list[0, cap) in
 * ascending order, counts[4] = 1 when they would have exceeded cap. With
 * filter != 0, counts[0] and the list keep only values not divisible by 3. */
int psm_intersect_check(const uint32_t* a, uint32_t na, const uint32_t* b, uint32_t nb, uint32_t cap,
                        uint32_t filter, uint32_t* counts, uint32_t* list);
#ifdef __cplusplus
}
#endif
#endif
