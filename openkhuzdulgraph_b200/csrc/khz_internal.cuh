// Internal types shared by the engine's translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <string>
#include <vector>

#include "khz.h"

namespace khz {

constexpr int kMaxK = 5;       // MAX_PATTERN_SIZE (engine.h:23)
constexpr int kNumSlots = 6;   // per-warp materialised sets: 1..3 level prefixes, 4 extra, 5 temp
constexpr uint32_t kAdjPad = 8;  // padding entries after every adjacency array (vector loads)

// ---------------------------------------------------------------------------------
// Schedule IR.  Each reference apply() level becomes one KhzLevel: the candidate set of
// vertex v_l is `base OP1 N(x1) OP2 N(x2)` (base = N(v_a) or a materialised prefix), the
// filters are the generated code's `v > v_a` / `v != v_a` tests, and the last level is
// one or two counting terms (compute-fused apps, kautomine/three_motif.cc:87-127).
// ---------------------------------------------------------------------------------
enum : int8_t { BASE_NBR = 0, BASE_SLOT = 1 };
enum : int8_t { OP_NONE = 0, OP_AND = 1, OP_SUB = 2 };

struct SetExpr {
    int8_t base_kind;
    int8_t base_arg;   // vertex index (BASE_NBR) or slot id (BASE_SLOT)
    int8_t op[2];
    int8_t op_arg[2];  // vertex index b of N(v_b)
};

struct Term {
    SetExpr set;
    uint8_t gt_mask;   // keep x > v_a for every bit a
    uint8_t ne_mask;   // keep x != v_a for every bit a
    int8_t guard_lo;   // evaluate only when v[guard_lo] < v[guard_hi] (-1: always)
    int8_t guard_hi;
    int8_t counter;    // last level: output counter index
    int8_t pad[3];
};

struct Level {
    Term t;            // enumeration term of this level (counter unused)
    int8_t has_extra;  // compute `extra` into slot 4 on entry (a cached object)
    int8_t finalized;  // children are executed in place: no NumExtensions (engine.cc:1441-1452)
    int8_t pad[2];
    SetExpr extra;
};

struct Plan {
    int8_t k;          // pattern size; levels 1..k-2 enumerate, level k-1 counts
    int8_t num_terms;  // counting terms at level k-1 (1 or 2)
    int8_t bounded_sets;  // 1: every later use of a level's set filters above that level's own lower
                          // bound, so level sets may be materialised without their members below it
    int8_t pad;
    Level lv[kMaxK];   // lv[1..k-2]; lv[1] must enumerate N(v0) (the DFS unit is one CSR entry)
    Term last[2];
};

static_assert(sizeof(Plan) % 4 == 0, "plans are copied to shared memory word by word");

struct AppDef {
    int num_runs;          // sequential pattern runs (each re-scatters every v0)
    Plan plans[6];
    int num_counts;
    uint32_t mult[6];
    bool clique;           // counts k-cliques: eligible for the bitmap engine
    int clique_k;
};

const AppDef &app_def(int app);
bool app_known(int app);  // a built-in app or one registered with khz_app_register

// ---------------------------------------------------------------------------------
// Device graph
// ---------------------------------------------------------------------------------
struct Graph {
    uint32_t n = 0;
    uint64_t m = 0;          // CSR entries
    uint32_t max_degree = 0;
    bool oriented = false;   // every list holds only ids above its vertex (a DAG in id order)
    bool symmetric = false;  // every entry (u, v) has its reverse (v, u)
    uint64_t *off = nullptr; // device n+1
    uint32_t *adj = nullptr; // device m + kAdjPad
    khz_graph oriented_view = 0;  // cached orientation of a symmetric graph (owned)
    khz_graph degree_view = 0;    // cached degree-descending renumbering of a symmetric graph (owned)
    uint64_t bytes = 0;
    // optional node labels (the .dgraph label section, graph_loader.h:773-822): device n uint32,
    // labels dense in [0, num_labels), and the number of vertices of each label (host)
    uint32_t *labels = nullptr;
    uint32_t num_labels = 0;
    std::vector<uint64_t> label_count;
};

// Start-vertex restriction of one job (run(..., restrict_starting_vertex_label, label),
// engine.cc:1457-1496): only start vertices v_0 with labels[v_0] == label are extended.
// labels == nullptr: every start vertex.
struct StartFilter {
    const uint32_t *labels;
    uint32_t label;
    __device__ __forceinline__ bool keep(uint32_t v0) const { return labels == nullptr || __ldg(labels + v0) == label; }
};

// DFS job (one (graph, plan) run inside a launch)
struct DfsJob {
    const uint64_t *off;
    const uint32_t *adj;
    uint32_t n;
    uint32_t plan_idx;     // index into the launch's plan table
    uint64_t unit_begin;   // first global unit of this job
    uint64_t num_units;    // = CSR entries (one level-1 candidate per unit)
    uint32_t out_base;     // counter row (KHZ_MAX_COUNTS + 2 uint64 per job)
    uint32_t min_deg;      // skip start vertices whose degree is below this (handled elsewhere)
    StartFilter start;     // start-vertex label restriction
};

constexpr int kRowWords = KHZ_MAX_COUNTS + 2;  // counter row: counts[6], NumExtensions, algorithmic bytes

// one (oriented graph, clique app) job of a bitmap-engine launch; jobs are sorted by vbase and
// their start vertices form one global index space [0, sum n)
struct BJob {
    const uint64_t *off;
    const uint32_t *adj;
    uint32_t n;
    int32_t k;          // clique size 3, 4 or 5
    uint64_t vbase;
    uint32_t out_row;
    uint32_t hub_rows;  // rows H of the hub triangle (vertices n - H .. n - 1), 0 = none
    const uint32_t *hub;  // the triangle (set by bitmap_prepare)
    StartFilter start;    // start-vertex label restriction
};

// bump allocator over one device allocation
struct Arena {
    char *base = nullptr;
    size_t used = 0, cap = 0;
    static size_t round(size_t b) { return (b + 255) & ~(size_t)255; }
    template <typename T>
    T *take(size_t count) {
        const size_t b = round(sizeof(T) * std::max<size_t>(count, 1));
        if (used + b > cap) return nullptr;
        T *p = (T *)(base + used);
        used += b;
        return p;
    }
};

// device resources and launch shapes of one bitmap-engine launch sequence
struct BitmapLaunch {
    const BJob *d_jobs = nullptr;
    int n_jobs = 0;
    uint64_t n_total = 0;
    // block tiers: 0 mid, 1 lower large, 2 upper large (start-vertex lists in descending degree)
    static constexpr int kTiers = 3;
    uint32_t *lists[kTiers] = {};
    unsigned int *cnt = nullptr;
    unsigned long long *queues = nullptr;
    uint32_t warp_max = 64;  // out-degrees served by one warp (32 or 64)
    int kmax = 4;            // largest clique size among the jobs (4 or 5: selects the kernel build)
    bool has_tier[kTiers] = {}, stats = false;
    int sms = 0;
    size_t block_smem[kTiers] = {};
    int block_threads[kTiers] = {}, block_grid[kTiers] = {}, block_dcap[kTiers] = {};
    // tensor-memory accumulator tiles per pass of the large tiers' 4-clique count (0: CUDA cores)
    int block_mma_g[kTiers] = {};
    std::vector<BJob> hubs;  // jobs with a hub triangle to build before the counting kernels
};

// one (symmetric graph, 4-cycle app) job of a wedge-engine launch (global start-vertex index space)
struct WJob {
    const uint64_t *off;
    const uint32_t *adj;
    uint32_t n;
    uint32_t max_deg;
    uint64_t vbase;
    uint32_t out_row;
    uint32_t tri_row;   // with `tri`: the row whose count 0 receives sum over wedges of (c - 1)(t1 + t2)
    StartFilter start;  // start-vertex label restriction (then the level-1 extensions are counted on the device)
    // When off/adj are the degree-descending renumbering of the stored graph, the wedges walked are
    // not the schedule's level-2 embeddings: these point at the stored graph, whose level-2
    // NumExtensions are then summed by a formula (null: the walked wedges are the schedule's)
    const uint64_t *ext_off;
    const uint32_t *ext_adj;
    // Per entry of adj: the triangles on that edge, or null.  With it, a second walk over each start
    // vertex's wedges (v0, w, v2) adds (c - 1)(t(v0 w) + t(w v2)), c being the endpoint count of v2:
    // summed, every 4-cycle once with the triangle counts of its four edges (the house identity)
    const uint32_t *tri;
};

struct WedgeLaunch {
    const WJob *d_jobs = nullptr;
    int n_jobs = 0;
    uint64_t n_total = 0, list_cap = 0;
    uint32_t *lists = nullptr;   // warp, block and window tier lists (list_cap each)
    unsigned int *cnt = nullptr;
    unsigned long long *queues = nullptr;
    bool wide = false;           // 32-bit window counters (some degree reaches 65535)
    bool ext_formula = false;    // some job counts on a renumbered graph (WJob::ext_off)
    int sms = 0;
};

// One pattern job counted from identities (the vertex-induced 4-motif, the tailed triangle and
// the house on a symmetric graph): per-edge triangle counts on the oriented view give the
// triangle, diamond and tailed-triangle terms, degrees the star and path terms; the 4-clique and
// 4-cycle counts (and the house's triangle-weighted 4-cycle sum) come from the bitmap and wedge
// engines into auxiliary counter rows.
struct MotifJob {
    const uint64_t *ooff;  // oriented view
    const uint32_t *oadj;
    uint32_t n;
    int32_t kind;          // KHZ_KAUTO_4MOTIF, KHZ_KGPI_TAILED_TRIANGLE or KHZ_KGPI_HOUSE
    uint64_t om;           // oriented edges (= undirected edges)
    uint32_t out_row;      // the job's counter row
    uint32_t k4_row, c4_row;  // auxiliary rows: 4-cliques (4-motif), 4-cycles (4-motif, house)
    uint32_t house_row;    // auxiliary row: the 4-cycles' edge-triangle sum (house)
    // house only: the degree-descending renumbering walked by the wedge engine (vertex x is the
    // oriented view's n - 1 - x), the triangle count of each of its entries, and the stored graph
    const uint64_t *doff;
    const uint32_t *dadj;
    uint32_t *tdv;
    const uint64_t *soff;
    const uint32_t *sadj;
    uint32_t *tri;         // per oriented edge: triangles on it (om)
    unsigned long long *acc;  // per vertex: sum of its edges' triangle counts (n)
    uint32_t *deg;         // per vertex: undirected degree (n)
    unsigned long long *sums;  // kMotifSums accumulators
};
constexpr int kMotifSums = 8;

struct MotifLaunch {
    const MotifJob *d_jobs = nullptr;
    int n_jobs = 0;
    std::vector<MotifJob> jobs;  // host copy (grid sizes)
    unsigned long long *queue = nullptr;  // vertex claims of the triangle kernel, one per job
    int sms = 0;
};

// device resources and launch shape of one DFS-engine launch
struct DfsLaunch {
    const DfsJob *d_jobs = nullptr;
    int n_jobs = 0;
    const Plan *d_plans = nullptr;
    uint64_t total_units = 0;
    uint32_t *slots = nullptr;
    uint32_t slot_cap = 0;
    int blocks = 0, threads = 0;
    uint32_t chunk = 8;
    unsigned long long *queue = nullptr;
    bool stats = false;
};


// Device allocation for graphs and temporaries: from the context's stream-ordered pool when an
// AllocScope is active on this thread (cudaMallocFromPoolAsync / cudaFreeAsync on its stream),
// plain cudaMalloc / cudaFree otherwise.
struct AllocScope {
    AllocScope(cudaMemPool_t pool, cudaStream_t s);
    ~AllocScope();
    cudaMemPool_t prev_pool;
    cudaStream_t prev_stream;
};
cudaError_t dev_alloc(void **p, size_t bytes);
void dev_free(void *p);

void set_error(const char *fmt, ...);
khz_status cuda_fail(cudaError_t e, const char *what);

#define KHZ_CUDA(call)                                              \
    do {                                                            \
        cudaError_t _e = (call);                                    \
        if (_e != cudaSuccess) return ::khz::cuda_fail(_e, #call);  \
    } while (0)

// graph construction (graph.cu)
khz_status build_csr_from_device_pairs(const uint32_t *d_pairs, uint64_t m, uint32_t n, bool validate,
                                       Graph *g, cudaStream_t s);
khz_status orient_graph(const Graph &in, Graph *out, cudaStream_t s);
khz_status relabel_by_degree(const Graph &in, Graph *out, cudaStream_t s);
khz_status generate_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                         Graph *g, cudaStream_t s);
void free_graph_memory(Graph *g);

// engines
constexpr int kPhases = 4;  // bitmap warp tier, mid block tier, large block tier, DFS
struct LaunchStats {
    uint32_t launches = 0;
    // optional per-phase event pairs (recorded around each phase's kernel when non-null)
    cudaEvent_t *ev_begin = nullptr;
    cudaEvent_t *ev_end = nullptr;
    bool used[kPhases] = {false, false, false, false};
    uint32_t phase_launches[kPhases] = {0, 0, 0, 0};
    uint64_t *d_phase_bytes = nullptr;  // device [kPhases], instrumented runs add per-phase bytes
};
// DFS engine.  Jobs carry unit_begin (prefix of num_units); rows of kRowWords uint64 must be
// zeroed by the caller.  No host synchronisation in dfs_enqueue.
uint64_t dfs_total_warps(int warps_per_sm);
// slot scratch is either owned by the launch (own_slots) or passed to dfs_enqueue by the caller
// (dfs_slot_words words), e.g. one buffer shared by launches that never overlap
uint64_t dfs_slot_words(int warps_per_sm, uint32_t slot_cap);
size_t dfs_arena_bytes(int n_jobs, int n_plans, uint64_t total_warps, uint32_t slot_cap, bool own_slots);
khz_status dfs_prepare(const std::vector<DfsJob> &jobs, const std::vector<Plan> &plans, uint32_t slot_cap,
                       int warps_per_sm, int chunk, bool stats, bool own_slots, Arena *arena, DfsLaunch *dl,
                       cudaStream_t s);
khz_status dfs_enqueue(const DfsLaunch &dl, uint64_t *d_rows, cudaStream_t s, LaunchStats *ls,
                       uint32_t *slots = nullptr);
khz_status dfs_launch_prealloc(const DfsJob *d_jobs, int n_jobs, const Plan *d_plans, uint64_t total_units,
                               uint32_t chunk, uint32_t *slots, uint32_t slot_cap, unsigned long long *queue,
                               uint64_t *d_raw, int blocks, int threads, cudaStream_t s);
// Bitmap clique engine over oriented graphs.  Adds each job's count (row[0]), its NumExtensions
// beyond depth 0 (row[6]) and, instrumented, the algorithmic bytes (row[7]).  Start vertices of
// out-degree above bitmap_block_max_degree() are skipped: run them on the DFS engine with
// DfsJob::min_deg.  No host synchronisation in bitmap_enqueue.
// Wedge engine (4-cycle on symmetric graphs): adds each job's count (row[0]) and its level-2
// NumExtensions (row[6]); no host synchronisation in wedge_enqueue.
size_t motif_arena_bytes(const std::vector<MotifJob> &jobs);
khz_status motif_prepare(std::vector<MotifJob> jobs, Arena *arena, MotifLaunch *ml, cudaStream_t s);
// the per-edge and per-vertex sums (before the wedge launch, which reads the house's entry
// triangle counts), then the combination (after the 4-clique and 4-cycle counts it reads)
khz_status motif_enqueue_sums(const MotifLaunch &ml, cudaStream_t s, LaunchStats *ls);
khz_status motif_enqueue_combine(const MotifLaunch &ml, uint64_t *d_rows, cudaStream_t s, LaunchStats *ls);
size_t wedge_arena_bytes(int n_jobs, uint64_t n_total);
khz_status wedge_prepare(const std::vector<WJob> &jobs, Arena *arena, WedgeLaunch *wl, cudaStream_t s);
khz_status wedge_enqueue(const WedgeLaunch &wl, uint64_t *d_rows, cudaStream_t s, LaunchStats *ls);
// rows of the hub triangle for a job on an oriented graph of n vertices and m edges under the
// configured setting (0 = auto, < 0 = none)
uint32_t bitmap_hub_rows(int cfg_rows, uint32_t n, uint64_t m);
size_t bitmap_hub_bytes(uint32_t rows);
size_t bitmap_arena_bytes(const std::vector<BJob> &jobs, uint64_t list_cap);
// tensor_cores: the large tiers count 4-cliques as a masked 0/1 matrix product on the tensor cores
khz_status bitmap_prepare(const std::vector<BJob> &jobs, uint32_t max_outdeg, uint64_t list_cap, bool stats,
                          int warp_max, bool tensor_cores, Arena *arena, BitmapLaunch *bl, cudaStream_t s);
// d_err: bit 2 is set if a tensor-core pass did not complete within its poll limit
khz_status bitmap_enqueue(const BitmapLaunch &bl, uint64_t *d_rows, cudaStream_t s, LaunchStats *ls,
                          unsigned int *d_err);
uint32_t bitmap_block_max_degree();

}  // namespace khz
