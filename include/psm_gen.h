/*
 * psm_gen.h - seeded synthetic data-graph and query-graph generators.
 *
 * The reference ships one real dataset (HPRD) and no generator for the
 * synthetic workloads it is benchmarked on, so this host-only library
 * produces them deterministically from a 64-bit seed:
 *   - Chung-Lu power-law graphs and R-MAT graphs (symmetrised, deduplicated,
 *     no self-loops), returned as an id-sorted undirected CSR;
 *   - uniform or Zipf vertex labels;
 *   - connected query graphs extracted by random walk (so every query has at
 *     least one embedding), in a sparse (walk tree plus induced edges while
 *     the average degree stays below 3) or dense (full induced subgraph with
 *     average degree >= 3) flavour.
 * Output is identical for the same seed on every host and thread count.
 * All buffers returned through a psmgen_* out-pointer are malloc'ed and are
 * released with psmgen_free().
 */
#ifndef PSM_GEN_H
#define PSM_GEN_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Undirected CSR: off[V+1], nbr[off[V]] with each list ascending. */
typedef struct psmgen_csr {
    uint32_t  num_vertices;
    uint64_t  num_entries;    /* = 2 * undirected edges */
    uint32_t* off;
    uint32_t* nbr;
} psmgen_csr;

/* Chung-Lu graph: expected degree of vertex i proportional to
 * (i+1)^(-1/(gamma-1)), scaled so the mean expected degree is avg_degree;
 * round(n*avg_degree/2) endpoint pairs are sampled. Returns 0 on success. */
int psmgen_chung_lu(uint32_t n, double gamma, double avg_degree, uint64_t seed, psmgen_csr* out);

/* R-MAT graph with 2^scale vertices and edge_factor * 2^scale sampled edges,
 * quadrant probabilities a, b, c (d = 1-a-b-c). Returns 0 on success. */
int psmgen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c,
                uint64_t seed, psmgen_csr* out);

/* Labels in [0, num_labels): uniform when zipf_s <= 0, else P(l) ~ 1/(l+1)^s. */
int psmgen_labels(uint32_t n, uint32_t num_labels, double zipf_s, uint64_t seed, uint32_t* out);

/* Random-walk query of k vertices. Writes labels[k] and edges as pairs
 * (edges[2*i], edges[2*i+1]) with edges capacity max_edges; *num_edges gets
 * the count. dense != 0 asks for the dense flavour. Query vertex i is the
 * i-th distinct data vertex the walk reached; data_ids[k] (may be NULL)
 * receives those data vertices. Returns 0 on success, nonzero if no walk of
 * k distinct vertices was found. */
int psmgen_query(const uint32_t* off, const uint32_t* nbr, const uint32_t* labels,
                 uint32_t num_vertices, uint32_t k, int dense, uint64_t seed,
                 uint32_t* q_labels, uint32_t* edges, uint32_t max_edges,
                 uint32_t* num_edges, uint32_t* data_ids);

/* Writes the graph in the reference's text format ("t V E", "v id label
 * degree", "e u v" with u < v). Returns 0 on success. */
int psmgen_write_text(const uint32_t* off, const uint32_t* nbr, const uint32_t* labels, uint32_t num_vertices,
                      const char* path);

void psmgen_free(void* p);

#ifdef __cplusplus
}
#endif
#endif
