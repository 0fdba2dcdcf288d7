/*
 * khz.h — C ABI of the B200 embedding-extension engine (libkhz_b200.so).
 *
 * Plain C: pointers, sizes and opaque handles only.  Every entry point returns a
 * khz_status and never aborts; khz_last_error_string() describes the last failure
 * of the calling thread.  Streams are passed as void* (a cudaStream_t, NULL for the
 * legacy default stream).
 *
 * Each declaration names the reference interface it replaces (paths relative to
 * the AmadeusChan/OpenKhuzdulGraph tree).
 */
#ifndef KHZ_H
#define KHZ_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KHZ_ABI_VERSION 2

/* Error codes.  Replaces the reference's assert()/exit(-1) failure paths
 * (e.g. distributed_application.cc:281-282, engine.cc:53-55, kautomine/triangle.cc:112-119). */
typedef enum khz_status {
    KHZ_OK = 0,
    KHZ_ERR_ARG = 1,      /* bad handle, id or size: rejected before any launch */
    KHZ_ERR_OOM = 2,      /* device or pinned allocation failed */
    KHZ_ERR_OVERFLOW = 3, /* a device-side capacity check fired (result dropped) */
    KHZ_ERR_TIMEOUT = 4,  /* a bounded device or host wait ran out */
    KHZ_ERR_CUDA = 5,     /* a CUDA runtime call failed */
    KHZ_ERR_FORMAT = 6,   /* input graph violates the .dgraph contract */
    KHZ_ERR_BUSY = 7,     /* serving queue full / ticket not finished */
    KHZ_ERR_NOT_FOUND = 8,
    KHZ_ERR_MULTIPLICITY = 9, /* a raw count is not divisible by the pattern multiplicity: the input
                                 is not the undirected graph the app assumes (the reference asserts,
                                 kautomine/three_motif.cc:232,243) */
    KHZ_ERR_CANCELLED = 10    /* a served query was withdrawn before it ran (khz_server_cancel) */
} khz_status;

/* Pattern applications; the numbering is shared with the oracle.
 * 0-7 are the reference's apps, 8-11 are schedules written in the same idioms. */
typedef enum khz_app_id {
    KHZ_KAUTO_TRIANGLE = 0,        /* kautomine/triangle.cc:58-121 */
    KHZ_KAUTO_4CLIQUE = 1,         /* kautomine/four_clique.cc:58-153 */
    KHZ_KAUTO_5CLIQUE = 2,         /* kautomine/five_clique.cc:58-186 */
    KHZ_KAUTO_3MOTIF = 3,          /* kautomine/three_motif.cc:40-44,59-138 (2 counts) */
    KHZ_KGPI_TRIANGLE = 4,         /* kgraphpi/triangle.cc:53-122 */
    KHZ_KGPI_4CLIQUE = 5,          /* kgraphpi/four_clique.cc:53-159 */
    KHZ_KGPI_5CLIQUE = 6,          /* kgraphpi/five_clique.cc:53-195 */
    KHZ_KGPI_3MOTIF = 7,           /* kgraphpi/three_motif.cc:52-174 (2 counts) */
    KHZ_KGPI_4CYCLE = 8,           /* 4-cycle, kgraphpi idiom (edge-induced) */
    KHZ_KGPI_HOUSE = 9,            /* house, kgraphpi idiom (edge-induced) */
    KHZ_KGPI_TAILED_TRIANGLE = 10, /* tailed triangle, kgraphpi idiom (edge-induced) */
    KHZ_KAUTO_4MOTIF = 11,         /* vertex-induced 4-motifs, kautomine idiom (6 counts) */
    KHZ_NUM_APPS = 12
} khz_app_id;

#define KHZ_MAX_COUNTS 6

typedef struct khz_ctx khz_ctx;
typedef uint32_t khz_graph; /* 0 is never a valid handle */

/* graph flags */
#define KHZ_EDGES_ON_DEVICE 0x1u /* the pairs pointer is device memory */
#define KHZ_ORIENT 0x2u          /* store the degree-oriented DAG instead of the symmetric CSR */
#define KHZ_UNCHECKED 0x4u       /* skip the sortedness/range validation pass */
#define KHZ_SKIP_LABELS 0x8u     /* khz_graph_load_dgraph: do not keep the file's node labels
                                    (DistributedApplication's load_vertex_labels = false) */

/* engine choice (khz_config.engine) */
#define KHZ_ENGINE_AUTO 0
#define KHZ_ENGINE_DFS 1     /* per-warp DFS over the schedule with warp-cooperative set ops */
#define KHZ_ENGINE_BITMAP 2  /* clique apps: local-subgraph bitmap engine on the oriented DAG */
#define KHZ_ENGINE_WEDGE 3   /* 4-cycle app on symmetric graphs: wedge-endpoint counting */

typedef struct khz_graph_info {
    uint32_t num_vertices;
    uint32_t max_degree;
    uint64_t num_entries;  /* CSR entries: 2|E| symmetric, |E| oriented */
    int32_t oriented;      /* 1: every list holds only larger ids (a DAG in id order) */
    int32_t symmetric;     /* 1: every entry has its reverse (undirected form) */
    const uint64_t *d_offsets; /* device, num_vertices + 1 */
    const uint32_t *d_adj;     /* device, num_entries (+ 8 padding entries) */
    uint64_t device_bytes;     /* HBM held by this graph */
    uint32_t num_labels;       /* 0: no node labels */
    uint32_t reserved;
    const uint32_t *d_labels;  /* device, num_vertices, or NULL */
} khz_graph_info;

typedef struct khz_stats {
    uint64_t num_extensions; /* the engine's NumExtensions (engine.cc:924) for the app's schedule */
    uint64_t algo_bytes;     /* 4 * sum (|A|+|B|+|A op B|) of the schedule's set ops (when requested) */
    double kernel_ms;        /* device time of the counting launches (CUDA events) */
    uint32_t engine;         /* KHZ_ENGINE_* actually used */
    uint32_t launches;       /* kernels launched by the call */
    /* per phase: 0 bitmap warp tier, 1 bitmap mid block tier, 2 bitmap large block tier, 3 DFS engine */
    double phase_ms[4];       /* device time of the phase's kernel (CUDA events; 0 if not run) */
    uint64_t phase_bytes[4];  /* algorithmic bytes of the phase (instrumented runs only) */
    uint32_t phase_launches[4];
} khz_stats;

typedef struct khz_config {
    int32_t engine;            /* KHZ_ENGINE_*; AUTO picks per app and graph */
    int32_t want_algo_bytes;   /* 1: run the instrumented variant that also sums algorithmic bytes */
    int32_t dfs_warps_per_sm;  /* resident warps per SM for the DFS engine (0 = default) */
    int32_t dfs_chunk;         /* level-1 candidates claimed per warp per grab (0 = default) */
    int32_t bitmap_warp_max;   /* largest out-degree served by one warp in the bitmap engine (32|64) */
    int32_t bitmap_block_warps;/* warps per block of the bitmap engine's block tier */
    int32_t bitmap_hub_rows;   /* bitmap engine: rows of the hub adjacency triangle over the
                                  highest-ranked vertices (0 = auto, -1 = none, else rounded down
                                  to a multiple of 32 and capped at the vertex count) */
    int32_t device_mem_limit_mib; /* cap on the device memory the context holds for graphs and counting
                                     scratch, in MiB (0 = none): an allocation that would exceed it
                                     fails with KHZ_ERR_OOM, as if the device were that small */
    int32_t bitmap_tensor_cores;  /* bitmap engine, out-degrees above 256: 1 = count 4-cliques as a
                                     masked 0/1 matrix product on the tensor cores; 0 (auto) or -1 =
                                     per-edge popcounts on the CUDA cores */
    int32_t reserved[7];
} khz_config;

/* ---- context ---------------------------------------------------------------------- */
/* Replaces DistributedSys::init_distributed_sys + the engine's buffer setup
 * (distributed_sys.cc:11-35, engine.cc:1152-1244): one context owns all device memory. */
khz_status khz_ctx_create(int device, khz_ctx **out);
khz_status khz_ctx_destroy(khz_ctx *ctx);
khz_status khz_ctx_set_config(khz_ctx *ctx, const khz_config *cfg);
khz_status khz_ctx_get_config(khz_ctx *ctx, khz_config *cfg);
const char *khz_last_error_string(void);
int khz_abi_version(void);

/* ---- graphs ----------------------------------------------------------------------- */
/* Sorted (src,dst) edge list -> HBM-resident CSR built on the device.  Replaces
 * CSRGraphLoader::load_graph / construct_csr_format_for_empty (graph_loader.h:154-201,
 * 210-499) and the distributed loader's CSR build (graph_loader.h:621-703).  pairs holds
 * m packed (src, dst) uint32 pairs sorted by (src, dst) without duplicates or self-loops,
 * exactly the .dgraph edge section (graph_loader.h:31-42). */
khz_status khz_graph_from_edges(khz_ctx *ctx, const uint32_t *pairs, uint64_t m, uint32_t n,
                                uint32_t flags, khz_graph *out, void *stream);
/* Reads a .dgraph file (header, optional node labels, edges) and builds the CSR.
 * Replaces JointHashBasedNumaAwareDistGraphLoader::load_graphs (graph_loader.h:706-961). */
khz_status khz_graph_load_dgraph(khz_ctx *ctx, const char *path, uint32_t flags, khz_graph *out);
/* Degree orientation on the device: rank by (degree, id), keep rank(u) < rank(v), sorted
 * out-lists.  Replaces toolkits/to_oriented_dataset_converter.cc:27-124. */
khz_status khz_graph_orient(khz_ctx *ctx, khz_graph in, khz_graph *out, void *stream);
/* Device R-MAT generator: raw edges -> drop self-loops -> canonical dedupe -> drop isolated
 * vertices with order-preserving compaction -> symmetric CSR.  Follows the dataset pipeline
 * datasets/live_journal/standardize.cc:66-111 + toolkits/converter.cc:151-268. */
khz_status khz_graph_generate_rmat(khz_ctx *ctx, int scale, int edge_factor, double a, double b,
                                   double c, uint64_t seed, uint32_t flags, khz_graph *out, void *stream);
khz_status khz_graph_info_get(khz_ctx *ctx, khz_graph g, khz_graph_info *info);
/* Copies the CSR to host memory (offsets: n+1 uint64, adj: num_entries uint32). */
khz_status khz_graph_export_csr(khz_ctx *ctx, khz_graph g, uint64_t *offsets, uint32_t *adj);
/* Writes the graph as a .dgraph file (symmetric or oriented, as stored); labels may be NULL. */
khz_status khz_graph_write_dgraph(khz_ctx *ctx, khz_graph g, const char *path, const uint32_t *labels);
/* Attaches node labels (labels: host array of num_vertices uint32) to a graph, replacing any it
 * had.  Labels must be dense: every value in [0, max label] is used by some vertex, as the
 * reference's loader requires (graph_loader.h:795-804, which exits otherwise; here KHZ_ERR_FORMAT).
 * khz_graph_load_dgraph attaches a labelled file's labels itself (graph_loader.h:773-822).
 * Orientation relabels vertices and, like to_oriented_dataset_converter.cc:76, drops labels. */
khz_status khz_graph_set_labels(khz_ctx *ctx, khz_graph g, const uint32_t *labels, uint32_t num_vertices);
/* Frees the graph's HBM.  Replaces destroy_graphs (graph_loader.h:963-974). */
khz_status khz_graph_free(khz_ctx *ctx, khz_graph g);

/* ---- counting --------------------------------------------------------------------- */
/* One application on one graph: replaces `count->clear(); app->run(); count->evaluate()`
 * (kautomine/triangle.cc:211-216, distributed_application.cc:259-356, engine.h:615-673).
 * counts receives khz_app_num_counts(app) uint64 values, already divided by the app's
 * multiplicities.  Blocks until the result is on the host. */
khz_status khz_count(khz_ctx *ctx, khz_graph g, khz_app_id app, uint64_t *counts, khz_stats *stats,
                     void *stream);
/* Enqueues the same work without waiting: d_out (device, >= 8 uint64) receives
 * [0..5] counts, [6] NumExtensions, [7] algorithmic bytes (0 unless configured). */
khz_status khz_count_async(khz_ctx *ctx, khz_graph g, khz_app_id app, uint64_t *d_out, void *stream);
/* run(disable_output, restrict_starting_vertex_label = true, start_label): the same count with the
 * start vertices v_0 restricted to the vertices whose label is start_label
 * (distributed_application.h:54, WorkloadDistributer::fetch_next_batch_local, engine.cc:1457-1496).
 * The graph must carry labels.  counts receives the aggregators' RAW values (Aggregator::evaluate,
 * engine.h:630-645): on a slice of the start vertices a pattern's copies need not come in whole
 * multiples of its multiplicity, so the division is left to the caller, as the reference apps do
 * after run().  stats->num_extensions is the restricted run's NumExtensions.  Clique apps use the
 * bitmap engine only on a graph stored oriented (its start vertices are the stored ones); on other
 * graphs the schedule runs as stored on the DFS engine. */
khz_status khz_count_restricted(khz_ctx *ctx, khz_graph g, khz_app_id app, uint32_t start_label, uint64_t *counts,
                                khz_stats *stats, void *stream);
int khz_app_num_counts(khz_app_id app);
/* mirrors the reference's `multiplicities[]` tables (kautomine/three_motif.cc:44) */
int khz_app_multiplicity(khz_app_id app, int pattern);

/* ---- frequent labelled subgraph mining (3-FSM) ------------------------------------ */
/* The kautomine three_fsm app (kautomine/three_fsm.cc:53-800) on the device: single vertices,
 * then edges, wedges, triangles, four-chains and three-stars of node labels, each level's candidate
 * labellings generated from the previous levels' frequent patterns (three_fsm.cc:315-590); a
 * pattern is frequent when its MNI support (for every pattern vertex the number of distinct graph
 * vertices it maps to, the least of these: SharedMemoryPatternDomain::get_support,
 * engine.h:384-401) reaches `threshold`.  The graph must carry node labels (at most 48, the
 * reference's MAX_NUM_LABELS) and be the symmetric CSR of a validated graph (the undirected form
 * the app mines; KHZ_ERR_ARG otherwise, as for a graph without labels).  out->level[i] gives what the app prints per level (the number of
 * frequent patterns and the support sum; level 0's sum covers every label, as setup() computes
 * it).  patterns (may be NULL) receives up to `capacity` frequent canonical patterns in the order
 * found; *num_patterns their total number. */
typedef struct khz_fsm_level {
    uint32_t num_candidates;
    uint32_t num_frequent;
    uint64_t support_sum;
} khz_fsm_level;
typedef struct khz_fsm_result {
    khz_fsm_level level[6]; /* vertex, edge, wedge, triangle, four-chain, three-star */
    double ms;              /* host wall time of the whole mining run */
} khz_fsm_result;
typedef struct khz_fsm_pattern {
    uint32_t level;         /* index into khz_fsm_result.level */
    uint32_t size;          /* pattern vertices */
    uint32_t labels[4];     /* the canonical labelling, in the app's vertex order */
    uint32_t support;
    uint32_t reserved;
} khz_fsm_pattern;
khz_status khz_fsm(khz_ctx *ctx, khz_graph g, uint32_t threshold, khz_fsm_result *out, khz_fsm_pattern *patterns,
                   uint32_t capacity, uint32_t *num_patterns);

/* ---- apps that bring their own schedule ------------------------------------------ */
/* Replaces the ApplyFunction contract (engine.h:589) and the engine calls an apply() makes
 * (scatter / cached objects, engine.h:592-613, 846-859): an app describes its apply() levels as
 * data, and the DFS engine runs them on the device.  Level l binds vertex v_l (l = 1 .. k-2
 * enumerate, level k-1 counts).  A level's candidate set is `base op0 N(v_a) op1 N(v_b)`:
 *   base = N(v_i) (KHZ_BASE_NBR, arg i) or a set materialised earlier (KHZ_BASE_SET, arg 2 or 3 =
 *          the set of level 2 or 3, arg 4 = the level's cached set), op = intersect_with (AND) or
 *          subtracted_by (SUB) of the vertex_set.cc routines;
 * the filters are the generated code's `v > v_a` restrictions (gt_mask: keep x above every v_a of
 * the mask) and `v != v_a` exclusions (ne_mask, at most 4 bits); a level's set is materialised
 * (the reference's cached prefix) when it has an op; `cached` is computed when the level is
 * entered, as an apply() computes a cached object for its children.  The last level adds
 * |set passing its filters| to its counter (1 or 2 counting terms: compute-fused apps), optionally
 * only when v[guard_lo] < v[guard_hi].  `finalized` levels do not count towards NumExtensions
 * (a finalized scatter, engine.cc:1441-1452).  Level 1 must enumerate N(v_0) itself. */
#define KHZ_BASE_NBR 0
#define KHZ_BASE_SET 1
#define KHZ_OP_NONE 0
#define KHZ_OP_AND 1
#define KHZ_OP_SUB 2
typedef struct khz_set_expr {
    int8_t base_kind;  /* KHZ_BASE_NBR or KHZ_BASE_SET */
    int8_t base_arg;   /* vertex index, or set 2 / 3 / 4 */
    int8_t op[2];      /* KHZ_OP_* */
    int8_t op_arg[2];  /* vertex index b of N(v_b) */
} khz_set_expr;
typedef struct khz_term {
    khz_set_expr set;
    uint8_t gt_mask;
    uint8_t ne_mask;
    int8_t guard_lo, guard_hi; /* -1: unguarded */
    int8_t counter;            /* last level: the count this term adds to */
    int8_t reserved[3];
} khz_term;
typedef struct khz_level {
    khz_term term;
    int8_t has_cached;
    int8_t finalized;
    int8_t reserved[2];
    khz_set_expr cached;
} khz_level;
typedef struct khz_pattern_schedule {
    int8_t k;          /* pattern size, 3 .. 5 (MAX_PATTERN_SIZE, engine.h:23) */
    int8_t num_terms;  /* counting terms of the last level, 1 or 2 */
    int8_t reserved[2];
    khz_level levels[5]; /* levels[1 .. k-2] are used */
    khz_term last[2];
} khz_pattern_schedule;
typedef struct khz_app_desc {
    int32_t num_runs;      /* patterns run one after another, each from every start vertex (1..6) */
    int32_t num_counts;    /* counters (1..6) */
    uint32_t multiplicity[KHZ_MAX_COUNTS]; /* raw counter / multiplicity = the reported count */
    khz_pattern_schedule runs[6];
} khz_app_desc;
/* Validates the schedule and returns an app id (>= KHZ_NUM_APPS) usable everywhere a khz_app_id
 * is, process-wide; such apps run on the DFS engine.  KHZ_ERR_ARG names the first invalid field. */
khz_status khz_app_register(const khz_app_desc *desc, int32_t *app_id);

/* ---- batched counting (many graphs / apps in one persistent launch) --------------- */
typedef struct khz_job {
    khz_graph graph;
    int32_t app;
    int32_t reserved;
} khz_job;
/* counts: n_jobs * KHZ_MAX_COUNTS uint64 (row per job); num_ext: n_jobs uint64 or NULL. */
khz_status khz_count_batch(khz_ctx *ctx, const khz_job *jobs, int n_jobs, uint64_t *counts,
                           uint64_t *num_ext, khz_stats *stats, void *stream);

/* A prepared batch: device tables and scratch are built once, the launch sequence (one bitmap
 * launch sequence for the clique jobs, one persistent DFS launch for the rest, a finalize kernel)
 * has no host synchronisation and, with KHZ_BATCH_CUDA_GRAPH, is captured into a CUDA graph and
 * replayed by khz_batch_launch.  Results of the last launch: khz_batch_wait. */
#define KHZ_BATCH_CUDA_GRAPH 0x1u
typedef struct khz_batch khz_batch;
khz_status khz_batch_create(khz_ctx *ctx, const khz_job *jobs, int n_jobs, uint32_t flags, khz_batch **out,
                            void *stream);
khz_status khz_batch_launch(khz_batch *batch, void *stream);
/* counts: n_jobs * KHZ_MAX_COUNTS uint64; num_ext: n_jobs uint64 or NULL; blocks until ready */
khz_status khz_batch_wait(khz_batch *batch, uint64_t *counts, uint64_t *num_ext, void *stream);
khz_status khz_batch_destroy(khz_batch *batch);

/* ---- autotuner ---------------------------------------------------------------------- */
/* Times the given jobs (a representative sample of the workload) under candidate settings —
 * engine (the bitmap / wedge / identity engines vs the DFS engine's warp-cooperative binary-search
 * probes), DFS warps per SM {8, 16, 24}, DFS units per grab {2, 8, 32}, bitmap warp-tier degree
 * threshold {32, 64}, hub-triangle rows {auto, none, 8192} — by coordinate descent (two passes,
 * best of `reps` each), checks that every
 * candidate produces the same counts, and installs the fastest in the context. */
typedef struct khz_tune_report {
    int32_t trials;
    int32_t reserved;
    double baseline_ms; /* the context's settings on entry */
    double best_ms;
    khz_config best;    /* now the context's configuration */
} khz_tune_report;
khz_status khz_autotune(khz_ctx *ctx, const khz_job *jobs, int n_jobs, int reps, khz_tune_report *report);

/* ---- serving: continuous batching of counting queries ----------------------------- */
/* A server owns `slots` CUDA streams and a scheduler thread.  Queries (graph, app) are admitted in
 * arrival order as slots and HBM budget free up (a query's footprint is its engine scratch: DFS
 * stacks sized by the graph's largest degree, or the bitmap engine's start-vertex lists; graphs
 * are resident and not counted); up to `max_batch` admitted queries share one launch sequence;
 * different slots' work overlaps on the device.  hbm_budget 0 = half the free device memory.
 * Replaces nothing in the reference (its engine serves one run() at a time). */
typedef struct khz_server khz_server;
typedef uint64_t khz_ticket;
typedef struct khz_server_stats {
    uint64_t completed;          /* queries finished since creation / the last reset */
    uint64_t batches;            /* launch sequences dispatched */
    uint64_t pending;            /* queries waiting for admission */
    uint64_t max_bytes_in_flight;/* largest admitted scratch footprint seen */
    double p50_ms, p99_ms, max_ms;  /* submit-to-result latency */
    double queries_per_s;        /* completed / (last completion - first submission) */
} khz_server_stats;
khz_status khz_server_create(khz_ctx *ctx, int slots, int max_batch, uint64_t hbm_budget, khz_server **out);
khz_status khz_server_submit(khz_server *server, khz_graph g, khz_app_id app, khz_ticket *ticket);
/* Waits up to timeout_ms (0: poll) for the ticket; KHZ_ERR_BUSY (poll) / KHZ_ERR_TIMEOUT if not done.
 * A finished ticket is consumed by the call that returns its result. */
khz_status khz_server_wait(khz_server *server, khz_ticket ticket, uint64_t *counts, uint64_t *num_ext,
                           double *latency_ms, double timeout_ms);
khz_status khz_server_stats_get(khz_server *server, khz_server_stats *stats);
khz_status khz_server_reset_stats(khz_server *server);
/* Withdraws a query that has not been admitted yet: its ticket then reports KHZ_ERR_CANCELLED.
 * KHZ_ERR_BUSY if it already runs or has finished (its result stays available), KHZ_ERR_NOT_FOUND
 * for an unknown or consumed ticket. */
khz_status khz_server_cancel(khz_server *server, khz_ticket ticket);
/* Finishes every submitted query, then releases the server. */
khz_status khz_server_destroy(khz_server *server);

/* ---- VertexSet algebra as a batch (test / tool entry) ----------------------------- */
/* VertexSet::intersect_with / subtracted_by / intersect_and_count / bounded_* and the
 * trims (vertex_set.cc:20-184, utilities.h:64-86) over n_pairs independent pairs of
 * sorted strictly increasing uint32 lists, all buffers on the device.  Pair i uses
 * a[a_off[i] .. a_off[i+1]) and b[b_off[i] .. b_off[i+1]); results go to
 * out[a_off[i] ..] (capacity |A_i|), out_len[i] receives the size (or count).
 * bound[i] is the upper bound of the bounded ops (ignored otherwise; may be NULL). */
#define KHZ_SETOP_INTERSECT 0
#define KHZ_SETOP_SUBTRACT 1
#define KHZ_SETOP_INTERSECT_COUNT 2
#define KHZ_SETOP_BOUNDED_INTERSECT 3
#define KHZ_SETOP_BOUNDED_SUBTRACT 4
#define KHZ_SETOP_TRIM 5               /* trim_v_list(A, bound): #elements < bound */
#define KHZ_SETOP_TRIM_LOWER_BOUND 6   /* trim_v_list_lower_bound(A, bound): #elements <= bound */
khz_status khz_set_op_batch(int op, const uint64_t *a_off, const uint32_t *a, const uint64_t *b_off,
                            const uint32_t *b, const uint32_t *bound, uint32_t *out, uint32_t *out_len,
                            uint32_t n_pairs, void *stream);

/* ---- counting without device allocation ------------------------------------------ */
/* No counterpart in the reference.  For callers that cannot call cudaMalloc: host frameworks
 * that own all device memory through their own pool and forbid side allocations, or plugins
 * loaded into a process whose allocator is locked down.  Counts `app` on a caller-owned device
 * CSR (d_offsets: n + 1 uint64, d_adj: num_entries uint32) with the DFS engine and writes the
 * same 8 uint64 as khz_count_async to the caller's device buffer d_out: [0..5] counts,
 * [6] NumExtensions, [7] 0.  It allocates nothing: all scratch lives in one fixed device array
 * of 14,557,184 bytes (about 13.9 MiB) inside the library, which every GPU that loads the library
 * holds until the process exits.  Limits: graphs whose largest vertex degree is at most 1024
 * (larger ones get KHZ_ERR_ARG).  The first call on each device looks up the array's device
 * address with that device current, so make that first call before any stream capture.  Every
 * call shares the array: calls whose work overlaps on the GPU (other streams, other host threads)
 * race and must be serialised by the caller.  Each call waits on its stream twice (to read the
 * graph's largest degree before the launch and the divisibility flag after it) and returns once
 * d_out holds the result. */
khz_status khz_count_noalloc(const uint64_t *d_offsets, const uint32_t *d_adj, uint32_t n, uint64_t num_entries,
                             khz_app_id app, uint64_t *d_out, void *stream);

#ifdef __cplusplus
}
#endif
#endif
