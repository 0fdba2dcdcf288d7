/*
 * CPU oracle for the Khuzdul embedding-extension path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py may load this library; the product (libkhz_b200.so)
 * never links or calls it.  It is a plain-C restatement of the reference's
 * algorithm, one function per reference routine, each citing the file:line it
 * follows (paths are relative to the AmadeusChan/OpenKhuzdulGraph tree).
 *
 * Pins: the restatement is checked against the reference's own apps, compiled
 * unmodified under oracle/_ref (golden fixtures in tests/golden/), and against
 * brute-force subgraph enumeration on small graphs.  The four schedules the
 * reference does not ship (kgraphpi 4-cycle, house, tailed triangle; kautomine
 * 4-motif) are pinned by brute force and closed-form identities only.
 */
#ifndef KHZ_ORACLE_H
#define KHZ_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* application ids: identical numbering to khz_app_id in include/khz.h */
enum {
    ORC_KAUTO_TRIANGLE = 0,
    ORC_KAUTO_4CLIQUE = 1,
    ORC_KAUTO_5CLIQUE = 2,
    ORC_KAUTO_3MOTIF = 3,
    ORC_KGPI_TRIANGLE = 4,
    ORC_KGPI_4CLIQUE = 5,
    ORC_KGPI_5CLIQUE = 6,
    ORC_KGPI_3MOTIF = 7,
    ORC_KGPI_4CYCLE = 8,
    ORC_KGPI_HOUSE = 9,
    ORC_KGPI_TAILED_TRIANGLE = 10,
    ORC_KAUTO_4MOTIF = 11,
    ORC_NUM_APPS = 12
};

/* ---- deterministic generators (bit-identical to the device generator) ---- */
uint64_t orc_mix64(uint64_t x);
/* Raw R-MAT edge i (before dedupe): writes src/dst. */
void orc_rmat_raw_edge(int scale, uint64_t seed, uint32_t ta, uint32_t tab, uint32_t tabc, uint64_t i,
                       uint32_t *src, uint32_t *dst);
/* R-MAT scale/edge factor -> sorted unique canonical pairs (u < v) with isolated
 * vertices dropped and ids compacted in order.  pairs_out holds 2*cap uint32.
 * Returns the number of pairs written (or UINT64_MAX when cap is too small). */
uint64_t orc_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                  uint32_t *pairs_out, uint64_t cap, uint32_t *n_out);
/* Erdos-Renyi: the first m distinct non-loop pairs of the seeded candidate stream,
 * then isolated vertices dropped and ids compacted; pairs sorted canonical (u < v). */
uint64_t orc_er(uint32_t n, uint64_t m, uint64_t seed, uint32_t *pairs_out, uint32_t *n_out);
/* canonical pairs (u < v, sorted) -> both directions sorted by (src, dst); out holds 4*m uint32 */
void orc_symmetrize(const uint32_t *canon, uint64_t m, uint32_t *out);

/* ---- .dgraph format (graph_loader.h:31-42) ---- */
int orc_dgraph_header(const char *path, uint32_t *n, uint64_t *m, int32_t *has_node_label);
int orc_dgraph_read(const char *path, uint32_t *labels_or_null, uint32_t *pairs);
int orc_dgraph_write(const char *path, uint32_t n, uint64_t m, const uint32_t *labels_or_null,
                     const uint32_t *pairs);

/* ---- CSR (graph_loader.h:154-201) and degree orientation (to_oriented_dataset_converter.cc:27-124) ---- */
int orc_csr_from_edges(const uint32_t *pairs, uint64_t m, uint32_t n, uint64_t *off, uint32_t *adj);
int orc_orient(uint32_t n, const uint64_t *off, const uint32_t *adj, uint64_t *ooff, uint32_t *oadj,
               uint32_t *rank_out);

/* ---- VertexSet algebra (vertex_set.cc) and trims (utilities.h:64-86) ---- */
uint32_t orc_intersect(const uint32_t *a, uint32_t na, const uint32_t *b, uint32_t nb, uint32_t *out);
uint32_t orc_subtract(const uint32_t *a, uint32_t na, const uint32_t *b, uint32_t nb, uint32_t *out);
uint32_t orc_intersect_count(const uint32_t *a, uint32_t na, const uint32_t *b, uint32_t nb);
uint32_t orc_bounded_intersect(const uint32_t *a, uint32_t na, const uint32_t *b, uint32_t nb, uint32_t ub,
                               uint32_t *out);
uint32_t orc_bounded_subtract(const uint32_t *a, uint32_t na, const uint32_t *b, uint32_t nb, uint32_t ub,
                              uint32_t *out);
uint32_t orc_trim(const uint32_t *a, uint32_t na, uint32_t upper_bound);
uint32_t orc_trim_lower_bound(const uint32_t *a, uint32_t na, uint32_t lower_bound);

/* ---- pattern counting: the reference schedules restated ----
 * Processes start vertices v0 with v0 % v0_mod == v0_rem (v0_mod = 1: all).
 * counts[] receives orc_num_counts(app) values (already divided by multiplicities);
 * num_ext = the engine's NumExtensions (engine.cc:924) summed over the app's runs;
 * algo_bytes = 4 * sum over set operations of (|A| + |B| + |result|). */
int orc_num_counts(int app);
int orc_count(int app, uint32_t n, const uint64_t *off, const uint32_t *adj, uint32_t v0_mod, uint32_t v0_rem,
              int threads, uint64_t *counts, uint64_t *num_ext, uint64_t *algo_bytes);
/* The run restricted to the start vertices whose label is `label` (run(..., true, label),
 * distributed_application.h:54, engine.cc:1457-1496); raw_counts are the aggregators' values
 * before any multiplicity division. */
int orc_count_labeled(int app, uint32_t n, const uint64_t *off, const uint32_t *adj, const uint32_t *labels,
                      uint32_t label, int threads, uint64_t *raw_counts, uint64_t *num_ext, uint64_t *algo_bytes);

/* ---- brute force (small graphs only) ----
 * Counts subgraph copies by enumerating vertex subsets.  pattern ids:
 * 0 triangle, 1 4-clique, 2 5-clique, 3 wedge (non-induced), 4 wedge (induced),
 * 5 4-cycle (non-induced), 6 house (non-induced), 7 tailed triangle (non-induced),
 * 10..15 induced 4-motifs in the order 3-star, 4-path, tailed triangle, 4-cycle, diamond, 4-clique. */
uint64_t orc_brute(int pattern, uint32_t n, const uint64_t *off, const uint32_t *adj);

/* ---- 3-FSM (kautomine/three_fsm.cc:53-800) ----
 * The app's level driver on a symmetric labelled graph (labels dense in [0, L), L <= 48 as
 * MAX_NUM_LABELS, graph_loader.h:28): levels 0 single vertices, 1 edges, 2 wedges, 3 triangles,
 * 4 four-chains, 5 three-stars, each level's candidates generated from the frequent patterns before
 * it (three_fsm.cc:315-590) and each candidate's MNI support the least number of distinct vertices
 * its embeddings map to one position (engine.h:384-401).  Fills, per level, the number of
 * candidates, of frequent patterns (support >= threshold) and their support sum (level 0: the sum
 * over every label, as setup() prints it).  Returns 0, or -1 for bad labels or no memory. */
#define ORC_FSM_MAX_LABELS 48
int orc_fsm(uint32_t n, const uint64_t *off, const uint32_t *adj, const uint32_t *labels, uint32_t L,
            uint32_t threshold, int threads, uint32_t *num_candidates, uint32_t *num_frequent,
            uint64_t *support_sum);

#ifdef __cplusplus
}
#endif
#endif
