// C ABI of the engine: context, graph table, counting dispatch, batching, set-op batch.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <thread>
#include <mutex>
#include <atomic>
#include <string>
#include <unordered_map>
#include <vector>

#include "khz_internal.cuh"
#include "khz_setops.cuh"

namespace khz {

// DFS engine: resident warps per SM by default (three 256-thread blocks: the register limit at
// 80 registers per thread; 19 % faster than two on the 4-motif at R-MAT scale 14, and four do not fit)
constexpr int kDfsDefaultWarps = 24;

static thread_local char g_err[512] = "";

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

khz_status cuda_fail(cudaError_t e, const char *what) {
    set_error("CUDA error in %s: %s", what, cudaGetErrorString(e));
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return KHZ_ERR_OOM;
    }
    return KHZ_ERR_CUDA;
}

namespace {


// divides the raw counters by the multiplicities and adds the host-known NumExtensions terms
__global__ void finalize_kernel(const uint64_t *raw, int rows, const uint32_t *mult, const uint64_t *ext_add,
                                uint64_t *out, unsigned int *bad) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    for (int c = 0; c < KHZ_MAX_COUNTS; ++c) {
        const uint64_t v = raw[(size_t)r * kRowWords + c];
        const uint32_t mu = mult[(size_t)r * KHZ_MAX_COUNTS + c];
        if (mu > 1 && v % mu) atomicOr(bad, 1u);
        out[(size_t)r * kRowWords + c] = mu > 1 ? v / mu : v;
    }
    out[(size_t)r * kRowWords + KHZ_MAX_COUNTS] = raw[(size_t)r * kRowWords + KHZ_MAX_COUNTS] + ext_add[r];
    out[(size_t)r * kRowWords + KHZ_MAX_COUNTS + 1] = raw[(size_t)r * kRowWords + KHZ_MAX_COUNTS + 1];
}

// 3-motif jobs counted from their triangle count: one block per job sums C(d, 2) over the
// symmetric graph and writes the wedge counter of its raw row (after the triangle launches):
//   kautomine (vertex-induced, multiplicity 2): raw = 2 * (sum C(d,2) - 3 T)
//   kgraphpi (edge-induced): sum C(d,2)
struct MJob {
    const uint64_t *off;
    uint32_t n;
    uint32_t out_row;
    int32_t vertex_induced;
    int32_t pad;
};

__global__ void motif3_combine_kernel(const MJob *__restrict__ jobs, uint64_t *rows) {
    const MJob J = jobs[blockIdx.x];
    __shared__ unsigned long long s_sum;
    if (threadIdx.x == 0) s_sum = 0;
    __syncthreads();
    unsigned long long part = 0;
    for (uint32_t v = threadIdx.x; v < J.n; v += blockDim.x) {
        const unsigned long long d = J.off[v + 1] - J.off[v];
        part += d * (d - (d > 0 ? 1 : 0)) / 2;
    }
    for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&s_sum, part);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t *row = rows + (size_t)J.out_row * kRowWords;
        const uint64_t t = row[0];
        row[1] = J.vertex_induced ? 2 * (s_sum - 3 * t) : s_sum;
    }
}

// VertexSet ops as a batch: one warp per pair (vertex_set.cc:20-184, utilities.h:64-86)
__global__ void setop_batch_kernel(int op, const uint64_t *a_off, const uint32_t *a, const uint64_t *b_off,
                                   const uint32_t *b, const uint32_t *bound, uint32_t *out, uint32_t *out_len,
                                   uint32_t n_pairs) {
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    const Filter none = {0, 0, 0, {0, 0, 0, 0}};
    for (uint32_t i = warp; i < n_pairs; i += nw) {
        const uint32_t *A = a + a_off[i];
        uint32_t na = (uint32_t)(a_off[i + 1] - a_off[i]);
        const uint32_t *Bp = b ? b + b_off[i] : nullptr;
        const uint32_t nb = b ? (uint32_t)(b_off[i + 1] - b_off[i]) : 0;
        uint32_t *O = out ? out + a_off[i] : nullptr;
        uint32_t res = 0;
        const uint32_t ub = bound ? bound[i] : 0;
        switch (op) {
            case KHZ_SETOP_INTERSECT:
            case KHZ_SETOP_INTERSECT_COUNT:
            case KHZ_SETOP_BOUNDED_INTERSECT: {
                if (op == KHZ_SETOP_BOUNDED_INTERSECT) na = lower_bound_plain(A, 0, na, ub);
                if (na == 0 || nb == 0) { res = 0; break; }
                uint32_t *w = op == KHZ_SETOP_INTERSECT_COUNT ? nullptr : O;
                // the result is written in A's order either way; probe with the shorter list
                res = na <= nb ? warp_probe<false>(A, na, Bp, nb, w, none).full
                               : warp_probe<false>(Bp, nb, A, na, w, none).full;
                break;
            }
            case KHZ_SETOP_SUBTRACT:
            case KHZ_SETOP_BOUNDED_SUBTRACT:
                if (op == KHZ_SETOP_BOUNDED_SUBTRACT) na = lower_bound_plain(A, 0, na, ub);
                res = na == 0 ? 0 : warp_probe<true>(A, na, Bp, nb, O, none).full;
                break;
            case KHZ_SETOP_TRIM:  // trim_v_list: #elements < bound
                res = lower_bound_plain(A, 0, na, ub);
                break;
            case KHZ_SETOP_TRIM_LOWER_BOUND:  // trim_v_list_lower_bound: #elements <= bound
                res = upper_bound_plain(A, 0, na, ub);
                break;
            default:
                res = 0;
        }
        if ((threadIdx.x & 31) == 0) out_len[i] = res;
    }
}

}  // namespace
}  // namespace khz

using namespace khz;

// A prepared counting launch over one or more (graph, app) jobs.  Device job tables, engine
// scratch and counter rows live in one allocation owned by the plan, so plans are independent of
// one another (different plans may run concurrently on different streams), and enqueueing a plan
// involves no host synchronisation, so its launch sequence can be captured into a CUDA graph.
struct BatchPlan {
    int rows = 0;
    int aux_rows = 0;  // counter rows after the jobs' own, for engines feeding identity-counted jobs
    MotifLaunch ml;
    std::vector<int> apps;
    bool stats = false;
    bool has_bitmap = false, has_dfs = false, has_wedge = false;
    MJob *d_mjobs = nullptr;
    int n_mjobs = 0;
    uint32_t engine = KHZ_ENGINE_DFS;
    BitmapLaunch bl;
    WedgeLaunch wl;
    DfsLaunch dl;
    void *mem = nullptr;
    Arena arena;
    uint64_t *d_raw = nullptr, *d_final = nullptr, *d_extadd = nullptr, *d_phase_bytes = nullptr;
    uint32_t *d_mult = nullptr;
    unsigned int *d_bad = nullptr;
    uint64_t *h_final = nullptr;  // pinned: rows * kRowWords, then the bad flag (own_scratch plans)
    bool own_scratch = true;      // false: DFS slots are the context's shared ones
    bool own_pinned = false;      // h_final was allocated by the plan
    uint64_t slot_words = 0;      // DFS slot words needed when they are shared
    size_t mem_bytes = 0;
    bool pool_mem = false;               // mem came from the context pool ...
    cudaStream_t pool_stream = nullptr;  // ... and is released on this stream (null: legacy stream)
    std::vector<khz_graph> graphs;       // graphs (and oriented views) whose pointers the plan holds
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::atomic<uint64_t> *direct_bytes = nullptr;  // the context's count of cudaMalloc'd bytes (mem not pooled)
    ~BatchPlan() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (mem) {
            if (pool_mem) {
                cudaFreeAsync(mem, pool_stream);
            } else {
                cudaFree(mem);
                if (direct_bytes) *direct_bytes -= mem_bytes;
            }
        }
        if (h_final && own_pinned) cudaFreeHost(h_final);
    }
};

struct khz_ctx {
    int device = 0;
    khz_config cfg{};
    std::vector<Graph> graphs;  // handle h -> graphs[h - 1]
    std::vector<bool> live;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t ph_begin[kPhases] = {}, ph_end[kPhases] = {};
    cudaMemPool_t pool = nullptr;  // graphs and temporaries (keeps up to 4 GiB cached between calls)
    std::unordered_map<std::string, std::unique_ptr<BatchPlan>> plans;  // khz_count's prepared launches
    // scratch shared by khz_count's launches, which the context serialises
    uint32_t *shared_slots = nullptr;
    uint64_t shared_slot_words = 0;
    uint64_t *h_pinned = nullptr;  // kRowWords + 1 words
    std::atomic<uint64_t> direct_bytes{0};  // device bytes held outside the pool (cudaMalloc)
    std::mutex mu;
};

struct khz_batch {
    khz_ctx *ctx;
    std::unique_ptr<BatchPlan> plan;
};

// ------------------------------------------------------------------------------------------
// Serving: continuous batching of counting queries on device-resident graphs.
// A scheduler thread owns S slots (CUDA streams).  Whenever a slot is free it admits the oldest
// pending queries whose estimated scratch footprint fits the remaining HBM budget, prepares one
// launch sequence for them (scratch from the context's stream-ordered pool) and enqueues it on the
// slot's stream; work of different slots overlaps on the device.  Completion is detected with
// events; results and submit-to-result latencies are handed back through tickets.
// ------------------------------------------------------------------------------------------
struct ServeRequest {
    khz_ticket id;
    khz_graph graph;
    int app;
    double t_submit;  // seconds, steady clock
    uint64_t footprint;
    int size_class;   // floor(log2(CSR entries + 1)): queries share a launch only within a class
};

struct ServeResult {
    bool done = false;
    khz_status status = KHZ_OK;
    uint64_t counts[KHZ_MAX_COUNTS] = {};
    uint64_t num_ext = 0;
    double latency_ms = 0;
    std::string error;  // why the query failed (the scheduler thread's error text)
};

struct ServeSlot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    std::unique_ptr<BatchPlan> plan;
    std::vector<ServeRequest> reqs;
    uint64_t *h_rows = nullptr;  // pinned: max_batch * kRowWords + 1
    uint64_t footprint = 0;
    bool busy = false;
};

struct khz_server {
    khz_ctx *ctx = nullptr;
    int max_batch = 64;
    uint64_t budget = 0, in_use = 0;
    std::vector<ServeSlot> slots;
    std::deque<ServeRequest> pending;
    std::unordered_map<khz_ticket, ServeResult> results;
    std::unordered_map<uint64_t, uint64_t> footprints;  // (graph, app) -> bytes, guarded by fp_mu
    std::mutex fp_mu;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::thread worker;
    bool stop = false;
    khz_ticket next_ticket = 1;
    std::vector<double> latencies;
    uint64_t completed = 0, batches = 0, max_in_flight = 0;
    double t_first = -1, t_last = 0;
};


namespace {

// Device bytes the context holds: its pool (graphs, pooled scratch) and its direct allocations.
uint64_t ctx_device_bytes(khz_ctx *ctx) {
    unsigned long long used = 0;  // the attribute's value is a 64-bit unsigned integer
    if (ctx->pool) cudaMemPoolGetAttribute(ctx->pool, cudaMemPoolAttrUsedMemCurrent, &used);
    return (uint64_t)used + ctx->direct_bytes.load();
}

// khz_config.device_mem_limit_mib: true (and the error set) when `more` bytes would pass the cap
bool over_mem_limit(khz_ctx *ctx, uint64_t more, const char *what) {
    const int32_t mib = ctx->cfg.device_mem_limit_mib;
    if (mib <= 0) return false;
    const uint64_t held = ctx_device_bytes(ctx), cap = (uint64_t)mib << 20;
    if (held + more <= cap) return false;
    set_error("%s: %llu more bytes would pass the context's device memory limit (%llu of %llu bytes held)", what,
              (unsigned long long)more, (unsigned long long)held, (unsigned long long)cap);
    return true;
}

khz_status check_ctx(khz_ctx *ctx) {
    if (!ctx) {
        set_error("null context");
        return KHZ_ERR_ARG;
    }
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    return KHZ_OK;
}

Graph *get_graph(khz_ctx *ctx, khz_graph g) {
    if (g == 0 || g > ctx->graphs.size() || !ctx->live[g - 1]) {
        set_error("invalid graph handle %u", g);
        return nullptr;
    }
    return &ctx->graphs[g - 1];
}

khz_graph add_graph(khz_ctx *ctx, const Graph &g) {
    ctx->graphs.push_back(g);
    ctx->live.push_back(true);
    return (khz_graph)ctx->graphs.size();
}

// a graph built by an API call: registered, or released again (KHZ_ERR_OOM) when holding it passes
// the context's device memory limit (the caller's AllocScope is still active, so the release
// goes back to the pool)
khz_status register_graph(khz_ctx *ctx, Graph &g, khz_graph *out) {
    if (over_mem_limit(ctx, 0, "graph")) {
        free_graph_memory(&g);
        return KHZ_ERR_OOM;
    }
    *out = add_graph(ctx, g);
    return KHZ_OK;
}

// oriented view of g (g itself when oriented; else a cached orientation)
khz_status oriented_of(khz_ctx *ctx, khz_graph h, Graph **out, cudaStream_t s) {
    Graph *g = get_graph(ctx, h);
    if (!g) return KHZ_ERR_ARG;
    if (g->oriented) {
        *out = g;
        return KHZ_OK;
    }
    if (g->oriented_view == 0) {
        Graph o;
        AllocScope scope(ctx->pool, s);
        khz_status st = orient_graph(*g, &o, s);
        if (st) return st;
        khz_graph oh = add_graph(ctx, o);
        g = get_graph(ctx, h);  // the table may have moved
        g->oriented_view = oh;
    }
    *out = get_graph(ctx, g->oriented_view);
    return KHZ_OK;
}

// degree-descending renumbering of a symmetric graph (built once, cached, freed with the graph)
khz_status degree_view_of(khz_ctx *ctx, khz_graph h, Graph **out, cudaStream_t s) {
    Graph *g = get_graph(ctx, h);
    if (!g) return KHZ_ERR_ARG;
    if (g->degree_view == 0) {
        Graph r;
        AllocScope scope(ctx->pool, s);
        khz_status st = relabel_by_degree(*g, &r, s);
        if (st) return st;
        khz_graph rh = add_graph(ctx, r);
        g = get_graph(ctx, h);  // the table may have moved
        g->degree_view = rh;
    }
    *out = get_graph(ctx, g->degree_view);
    return KHZ_OK;
}

// engine for one job under the context's configuration: the bitmap engine for clique apps on
// graphs that are a DAG in id order or symmetric (oriented once, cached); the DFS engine otherwise
// and the wedge engine for the 4-cycle app on symmetric graphs.  Instrumented runs
// (want_algo_bytes) of the 4-cycle use the DFS engine, which sums the schedule's set-op bytes.
// A start-vertex restriction keeps the start vertices of the graph as stored, so the bitmap engine
// (which starts from the oriented view's vertices) serves restricted clique jobs only on graphs
// stored oriented, and the 3-motif identity path (global degree sums) not at all.
int pick_engine(const khz_config &cfg, const AppDef &def, int app, const Graph &g, bool restricted = false) {
    const bool wedge_ok = app == KHZ_KGPI_4CYCLE && g.symmetric && !cfg.want_algo_bytes;
    const bool motif3 = (app == KHZ_KAUTO_3MOTIF || app == KHZ_KGPI_3MOTIF || app == KHZ_KAUTO_4MOTIF ||
                         app == KHZ_KGPI_TAILED_TRIANGLE || app == KHZ_KGPI_HOUSE) &&
                        g.symmetric && !cfg.want_algo_bytes && !restricted;
    int engine = cfg.engine;
    if (engine == KHZ_ENGINE_AUTO)
        engine = def.clique || motif3 ? KHZ_ENGINE_BITMAP : (wedge_ok ? KHZ_ENGINE_WEDGE : KHZ_ENGINE_DFS);
    if (engine == KHZ_ENGINE_BITMAP && motif3) return KHZ_ENGINE_BITMAP;
    if (engine == KHZ_ENGINE_BITMAP && !def.clique) engine = KHZ_ENGINE_DFS;
    if (engine == KHZ_ENGINE_BITMAP && !g.oriented && (!g.symmetric || restricted)) engine = KHZ_ENGINE_DFS;
    if (engine == KHZ_ENGINE_WEDGE && !wedge_ok) engine = KHZ_ENGINE_DFS;
    return engine;
}

// build options
constexpr unsigned kPlanOwnSlots = 1u;   // the plan owns its DFS slots (else the context's shared ones)
constexpr unsigned kPlanPinned = 2u;     // the plan owns a pinned result buffer
constexpr unsigned kPlanPoolMem = 4u;    // device scratch from the context's stream-ordered pool on `s`
constexpr unsigned kPlanFreeLegacy = 8u; // with kPlanPoolMem: release on the legacy stream (callers sync first)

// start_labels (may be null): per job, the label its start vertices are restricted to, or -1.
// Restricted jobs report raw counts (multiplicities not divided).
khz_status build_plan(khz_ctx *ctx, const khz_job *jobs, int n, cudaStream_t s, unsigned opts,
                      std::unique_ptr<BatchPlan> *out, const int64_t *start_labels = nullptr) {
    const bool own_scratch = (opts & kPlanOwnSlots) != 0;
    if (n <= 0) {
        set_error("empty batch");
        return KHZ_ERR_ARG;
    }
    for (int i = 0; i < n; ++i) {
        if (!app_known(jobs[i].app)) {
            set_error("invalid app id %d", jobs[i].app);
            return KHZ_ERR_ARG;
        }
        const Graph *g = get_graph(ctx, jobs[i].graph);
        if (!g) return KHZ_ERR_ARG;
        const int64_t lab = start_labels ? start_labels[i] : -1;
        if (lab >= 0 && !g->labels) {
            set_error("graph %u has no node labels to restrict the start vertices by", jobs[i].graph);
            return KHZ_ERR_ARG;
        }
        if (lab >= (int64_t)g->num_labels) {
            set_error("start label %lld out of range: the graph has %u labels", (long long)lab, g->num_labels);
            return KHZ_ERR_ARG;
        }
    }
    auto P = std::make_unique<BatchPlan>();
    P->rows = n;
    P->own_scratch = own_scratch;
    P->stats = ctx->cfg.want_algo_bytes != 0;
    std::vector<BJob> bjobs;
    std::vector<MJob> mjobs;
    std::vector<MotifJob> motif_jobs;
    std::vector<WJob> wjobs;
    std::vector<std::pair<size_t, size_t>> house_wjobs;  // (wedge job, motif job) of each house job
    std::vector<DfsJob> djobs;
    std::vector<Plan> plans;
    std::vector<uint64_t> ext_add(n, 0);
    std::vector<uint32_t> mult((size_t)n * KHZ_MAX_COUNTS, 1);
    uint32_t bmax = 0, slot_cap = 32;
    uint64_t vbase = 0, bm_entries = 0, unit_base = 0, wbase = 0;
    auto add_dfs = [&](const Graph &g, const Plan &pl, int row, uint32_t min_deg, StartFilter sf) {
        DfsJob j{};
        j.off = g.off;
        j.adj = g.adj;
        j.n = g.n;
        j.plan_idx = (uint32_t)plans.size();
        j.unit_begin = unit_base;
        j.num_units = g.m;
        j.out_base = (uint32_t)row;
        j.min_deg = min_deg;
        j.start = sf;
        plans.push_back(pl);
        djobs.push_back(j);
        unit_base += g.m;
        slot_cap = std::max(slot_cap, g.max_degree);
    };
    for (int i = 0; i < n; ++i) {
        const AppDef &def = app_def(jobs[i].app);
        P->apps.push_back(jobs[i].app);
        P->graphs.push_back(jobs[i].graph);  // an oriented view is owned by (and freed with) its source
        const int64_t lab = start_labels ? start_labels[i] : -1;
        const Graph &g0 = *get_graph(ctx, jobs[i].graph);
        const StartFilter sf = lab >= 0 ? StartFilter{g0.labels, (uint32_t)lab} : StartFilter{nullptr, 0};
        const uint64_t starts = lab >= 0 ? g0.label_count[(size_t)lab] : g0.n;  // depth-0 extensions
        if (lab < 0)
            for (int c = 0; c < def.num_counts; ++c) mult[(size_t)i * KHZ_MAX_COUNTS + c] = def.mult[c];
        const int engine = pick_engine(ctx->cfg, def, jobs[i].app, g0, lab >= 0);
        if (engine == KHZ_ENGINE_BITMAP && (jobs[i].app == KHZ_KAUTO_4MOTIF ||
                                            jobs[i].app == KHZ_KGPI_TAILED_TRIANGLE || jobs[i].app == KHZ_KGPI_HOUSE)) {
            // identities over per-edge triangle counts (motif.cu); the 4-motif's 4-cliques come from
            // the bitmap engine and its 4-cycles from the wedge engine, each into an auxiliary row;
            // the house's 4-cycles and their edge-triangle sum from one weighted wedge job
            Graph *og = nullptr;
            khz_status st = oriented_of(ctx, jobs[i].graph, &og, s);
            if (st) return st;
            const Graph og_copy = *og;
            MotifJob mj{};
            mj.ooff = og_copy.off;
            mj.oadj = og_copy.adj;
            mj.n = og_copy.n;
            mj.kind = jobs[i].app;
            mj.om = og_copy.m;
            mj.out_row = (uint32_t)i;
            auto aux_row = [&]() {
                ext_add.push_back(0);
                mult.insert(mult.end(), KHZ_MAX_COUNTS, 1u);
                return (uint32_t)(ext_add.size() - 1);
            };
            if (jobs[i].app == KHZ_KGPI_HOUSE) {
                Graph *dv = nullptr;
                st = degree_view_of(ctx, jobs[i].graph, &dv, s);
                if (st) return st;
                const Graph dv_copy = *dv;
                const Graph sg = *get_graph(ctx, jobs[i].graph);
                mj.c4_row = aux_row();
                mj.house_row = aux_row();
                mj.doff = dv_copy.off;
                mj.dadj = dv_copy.adj;
                mj.soff = sg.off;
                mj.sadj = sg.adj;
                // the entry triangle counts (WJob::tri) are placed once the motif arena is laid out
                house_wjobs.push_back({wjobs.size(), motif_jobs.size()});
                wjobs.push_back(WJob{dv_copy.off, dv_copy.adj, dv_copy.n, dv_copy.max_degree, wbase, mj.c4_row,
                                     mj.house_row, StartFilter{nullptr, 0}, nullptr, nullptr, nullptr});
                wbase += dv_copy.n;
            }
            if (jobs[i].app == KHZ_KAUTO_4MOTIF) {
                Graph *dv = nullptr;
                st = degree_view_of(ctx, jobs[i].graph, &dv, s);
                if (st) return st;
                const Graph dv_copy = *dv;
                const Graph sg = *get_graph(ctx, jobs[i].graph);
                mj.k4_row = aux_row();
                mj.c4_row = aux_row();
                bjobs.push_back(BJob{og_copy.off, og_copy.adj, og_copy.n, 4, vbase, mj.k4_row,
                                     bitmap_hub_rows(ctx->cfg.bitmap_hub_rows, og_copy.n, og_copy.m), nullptr,
                                     StartFilter{nullptr, 0}});
                vbase += og_copy.n;
                bm_entries += og_copy.m;
                bmax = std::max(bmax, og_copy.max_degree);
                if (og_copy.max_degree > bitmap_block_max_degree())
                    add_dfs(og_copy, app_def(KHZ_KAUTO_4CLIQUE).plans[0], (int)mj.k4_row, bitmap_block_max_degree() + 1,
                            StartFilter{nullptr, 0});
                wjobs.push_back(WJob{dv_copy.off, dv_copy.adj, dv_copy.n, dv_copy.max_degree, wbase, mj.c4_row, 0,
                                     StartFilter{nullptr, 0}, sg.off, sg.adj});
                wbase += dv_copy.n;
            }
            motif_jobs.push_back(mj);
            ext_add[i] = 0;  // the combine kernel writes the whole NumExtensions
            P->engine = KHZ_ENGINE_BITMAP;
        } else if (engine == KHZ_ENGINE_BITMAP && !def.clique) {
            // 3-motif: triangles on the oriented view (bitmap engine, k = 3) + degree sums
            const Graph sg = *get_graph(ctx, jobs[i].graph);
            Graph *og = nullptr;
            khz_status st = oriented_of(ctx, jobs[i].graph, &og, s);
            if (st) return st;
            bjobs.push_back(BJob{og->off, og->adj, og->n, 3, vbase, (uint32_t)i,
                                 bitmap_hub_rows(ctx->cfg.bitmap_hub_rows, og->n, og->m), nullptr});
            vbase += og->n;
            bm_entries += og->m;
            bmax = std::max(bmax, og->max_degree);
            if (og->max_degree > bitmap_block_max_degree())
                add_dfs(*og, app_def(KHZ_KAUTO_TRIANGLE).plans[0], i, bitmap_block_max_degree() + 1,
                        StartFilter{nullptr, 0});
            const bool kauto = jobs[i].app == KHZ_KAUTO_3MOTIF;
            mjobs.push_back(MJob{sg.off, sg.n, (uint32_t)i, kauto ? 1 : 0, 0});
            // the bitmap launch adds one level-1 extension per undirected edge; kautomine's fused run
            // extends every (v0, v1) pair (twice that), kgraphpi's wedge run adds only its start vertices
            ext_add[i] = kauto ? (uint64_t)sg.n + sg.m / 2 : 2ull * sg.n;
            P->engine = KHZ_ENGINE_BITMAP;
        } else if (engine == KHZ_ENGINE_BITMAP) {
            Graph *og = nullptr;
            khz_status st = oriented_of(ctx, jobs[i].graph, &og, s);
            if (st) return st;
            // restricted: og is the graph as stored (pick_engine), so its labels apply
            BJob b{og->off, og->adj, og->n, def.clique_k, vbase, (uint32_t)i,
                   bitmap_hub_rows(ctx->cfg.bitmap_hub_rows, og->n, og->m), nullptr, sf};
            bjobs.push_back(b);
            vbase += og->n;
            bm_entries += og->m;
            bmax = std::max(bmax, og->max_degree);
            if (og->max_degree > bitmap_block_max_degree())
                add_dfs(*og, def.plans[0], i, bitmap_block_max_degree() + 1, sf);
            ext_add[i] = lab >= 0 ? starts : og->n;
            P->engine = KHZ_ENGINE_BITMAP;
        } else if (engine == KHZ_ENGINE_WEDGE) {
            const Graph g = *get_graph(ctx, jobs[i].graph);
            if (lab >= 0) {
                // restricted: the start vertices are the stored ones, so walk the stored graph
                wjobs.push_back(WJob{g.off, g.adj, g.n, g.max_degree, wbase, (uint32_t)i, 0, sf, nullptr, nullptr});
            } else {
                // every 4-cycle once, from its highest-degree vertex: wedges walked on the
                // degree-descending renumbering (about half the schedule's on R-MAT graphs); the
                // schedule's level-2 NumExtensions come from the stored graph by formula
                Graph *dv = nullptr;
                khz_status st = degree_view_of(ctx, jobs[i].graph, &dv, s);
                if (st) return st;
                wjobs.push_back(
                    WJob{dv->off, dv->adj, dv->n, dv->max_degree, wbase, (uint32_t)i, 0, sf, g.off, g.adj});
            }
            wbase += g.n;
            // depth 0 and every undirected edge once at depth 1 (restricted: depth 1 counted on the device)
            ext_add[i] = lab >= 0 ? starts : (uint64_t)g.n + g.m / 2;
            if (P->engine == KHZ_ENGINE_DFS) P->engine = KHZ_ENGINE_WEDGE;
        } else {
            const Graph &g = *get_graph(ctx, jobs[i].graph);
            for (int r = 0; r < def.num_runs; ++r) add_dfs(g, def.plans[r], i, 0, sf);
            ext_add[i] = starts * def.num_runs;
        }
    }
    P->has_bitmap = !bjobs.empty();
    P->has_dfs = !djobs.empty();
    P->has_wedge = !wjobs.empty();
    const int warp_max = ctx->cfg.bitmap_warp_max == 32 ? 32 : 64;
    // every listed start vertex has more than warp_max out-edges
    const uint64_t list_cap = std::min<uint64_t>(std::max<uint64_t>(vbase, 1), bm_entries / (warp_max + 1) + 1);
    const uint64_t dfs_warps = dfs_total_warps(ctx->cfg.dfs_warps_per_sm);
    const int total = (int)ext_add.size();  // job rows, then auxiliary rows of identity-counted jobs
    P->aux_rows = total - n;
    size_t bytes = 2 * Arena::round(sizeof(uint64_t) * kRowWords * total) + Arena::round(sizeof(uint32_t) * mult.size()) +
                   Arena::round(sizeof(uint64_t) * total) + Arena::round(sizeof(unsigned int)) +
                   Arena::round(sizeof(uint64_t) * kPhases);
    if (P->has_bitmap) bytes += bitmap_arena_bytes(bjobs, list_cap);
    if (P->has_wedge) bytes += wedge_arena_bytes((int)wjobs.size(), wbase);
    if (!mjobs.empty()) bytes += Arena::round(sizeof(MJob) * mjobs.size());
    if (!motif_jobs.empty()) bytes += motif_arena_bytes(motif_jobs);
    if (P->has_dfs) bytes += dfs_arena_bytes((int)djobs.size(), (int)plans.size(), dfs_warps, slot_cap, own_scratch);
    P->slot_words = P->has_dfs ? dfs_slot_words(ctx->cfg.dfs_warps_per_sm, slot_cap) : 0;
    if (over_mem_limit(ctx, bytes, "counting launch scratch")) return KHZ_ERR_OOM;
    cudaError_t e;
    if (opts & kPlanPoolMem) {
        e = cudaMallocFromPoolAsync(&P->mem, bytes, ctx->pool, s);
        if (e == cudaSuccess) {
            P->pool_mem = true;
            P->pool_stream = (opts & kPlanFreeLegacy) ? nullptr : s;
        }
    } else {
        e = cudaMalloc(&P->mem, bytes);
        if (e == cudaSuccess) {
            ctx->direct_bytes += bytes;
            P->direct_bytes = &ctx->direct_bytes;
        }
    }
    P->mem_bytes = bytes;
    if (e != cudaSuccess) {
        cudaGetLastError();
        P->mem = nullptr;
        set_error("counting launch needs %llu bytes of device scratch: %s", (unsigned long long)bytes,
                  cudaGetErrorString(e));
        return KHZ_ERR_OOM;
    }
    P->arena.base = (char *)P->mem;
    P->arena.cap = bytes;
    P->d_raw = P->arena.take<uint64_t>((size_t)kRowWords * total);
    P->d_final = P->arena.take<uint64_t>((size_t)kRowWords * total);
    P->d_mult = P->arena.take<uint32_t>(mult.size());
    P->d_extadd = P->arena.take<uint64_t>(total);
    P->d_bad = P->arena.take<unsigned int>(1);
    P->d_phase_bytes = P->arena.take<uint64_t>(kPhases);
    KHZ_CUDA(cudaMemcpyAsync(P->d_mult, mult.data(), sizeof(uint32_t) * mult.size(), cudaMemcpyHostToDevice, s));
    KHZ_CUDA(cudaMemcpyAsync(P->d_extadd, ext_add.data(), sizeof(uint64_t) * total, cudaMemcpyHostToDevice, s));
    khz_status st = KHZ_OK;
    if (P->has_bitmap)
        st = bitmap_prepare(bjobs, bmax, list_cap, P->stats, warp_max, ctx->cfg.bitmap_tensor_cores > 0, &P->arena,
                            &P->bl, s);
    if (st) return st;
    if (!motif_jobs.empty()) st = motif_prepare(motif_jobs, &P->arena, &P->ml, s);
    if (st) return st;
    for (const auto &hw : house_wjobs) wjobs[hw.first].tri = P->ml.jobs[hw.second].tdv;
    if (P->has_wedge) st = wedge_prepare(wjobs, &P->arena, &P->wl, s);
    if (st) return st;
    if (!mjobs.empty()) {
        P->d_mjobs = P->arena.take<MJob>(mjobs.size());
        P->n_mjobs = (int)mjobs.size();
        KHZ_CUDA(cudaMemcpyAsync(P->d_mjobs, mjobs.data(), sizeof(MJob) * mjobs.size(), cudaMemcpyHostToDevice, s));
    }
    if (P->has_dfs)
        st = dfs_prepare(djobs, plans, slot_cap, ctx->cfg.dfs_warps_per_sm, ctx->cfg.dfs_chunk, P->stats, own_scratch,
                         &P->arena, &P->dl, s);
    if (st) return st;
    if ((opts & kPlanPinned) &&
        cudaMallocHost(&P->h_final, sizeof(uint64_t) * ((size_t)kRowWords * n + 1)) != cudaSuccess) {
        cudaGetLastError();
        P->h_final = nullptr;
        set_error("pinned result buffer allocation failed");
        return KHZ_ERR_OOM;
    }
    P->own_pinned = (opts & kPlanPinned) != 0;
    KHZ_CUDA(cudaStreamSynchronize(s));
    *out = std::move(P);
    return KHZ_OK;
}

// Enqueue the plan: zero the counters, the engines' launches, finalize.  `ls` (may be null)
// records per-phase events; ev_begin / ev_end (may be null) bracket the counting launches.
khz_status enqueue_plan(BatchPlan *P, cudaStream_t s, LaunchStats *ls, cudaEvent_t ev_begin, cudaEvent_t ev_end,
                        uint32_t *shared_slots = nullptr) {
    KHZ_CUDA(cudaMemsetAsync(P->d_raw, 0, sizeof(uint64_t) * kRowWords * (P->rows + P->aux_rows), s));
    KHZ_CUDA(cudaMemsetAsync(P->d_bad, 0, sizeof(unsigned int), s));
    KHZ_CUDA(cudaMemsetAsync(P->d_phase_bytes, 0, sizeof(uint64_t) * kPhases, s));
    if (ls) ls->d_phase_bytes = P->d_phase_bytes;
    if (ev_begin) KHZ_CUDA(cudaEventRecord(ev_begin, s));
    khz_status st = KHZ_OK;
    if (P->has_bitmap) st = bitmap_enqueue(P->bl, P->d_raw, s, ls, P->d_bad);
    if (st) return st;
    if (P->has_dfs) st = dfs_enqueue(P->dl, P->d_raw, s, ls, P->own_scratch ? nullptr : shared_slots);
    if (st) return st;
    if (P->n_mjobs) {  // after every launch that counts triangles
        motif3_combine_kernel<<<P->n_mjobs, 256, 0, s>>>(P->d_mjobs, P->d_raw);
        KHZ_CUDA(cudaGetLastError());
        if (ls) ls->launches += 1;
    }
    st = motif_enqueue_sums(P->ml, s, ls);  // before the wedge launch, which reads the house's entry counts
    if (st) return st;
    if (P->has_wedge) st = wedge_enqueue(P->wl, P->d_raw, s, ls);
    if (st) return st;
    st = motif_enqueue_combine(P->ml, P->d_raw, s, ls);  // after the 4-clique and 4-cycle counts it combines
    if (st) return st;
    if (ev_end) KHZ_CUDA(cudaEventRecord(ev_end, s));
    const int all_rows = P->rows + P->aux_rows;
    finalize_kernel<<<(unsigned)((all_rows + 127) / 128), 128, 0, s>>>(P->d_raw, all_rows, P->d_mult, P->d_extadd,
                                                                       P->d_final, P->d_bad);
    KHZ_CUDA(cudaGetLastError());
    if (ls) ls->launches += 1;
    return KHZ_OK;
}

// the status a launch's device flag word reports: bit 1 a count not divisible by the pattern's
// multiplicity (finalize), bit 2 a tensor-core pass of the bitmap engine that did not complete
// within its poll limit (the counts are then incomplete)
khz_status launch_flags_status(unsigned int flags) {
    if (flags & 2u) {
        set_error("a tensor-core counting pass did not complete within its wait limit; the counts are incomplete");
        return KHZ_ERR_CUDA;
    }
    if (flags) {
        set_error("raw count not divisible by the pattern multiplicity (input is not an undirected graph)");
        return KHZ_ERR_MULTIPLICITY;
    }
    return KHZ_OK;
}

// copy the finalized rows to pinned memory (the plan's, or `host` for shared-scratch plans)
// and wait for them
khz_status read_plan(BatchPlan *P, cudaStream_t s, uint64_t *host = nullptr) {
    if (host) P->h_final = host;
    const size_t words = (size_t)kRowWords * P->rows;
    KHZ_CUDA(cudaMemcpyAsync(P->h_final, P->d_final, sizeof(uint64_t) * words, cudaMemcpyDeviceToHost, s));
    KHZ_CUDA(cudaMemcpyAsync(P->h_final + words, P->d_bad, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
    KHZ_CUDA(cudaStreamSynchronize(s));
    return launch_flags_status(*(const unsigned int *)(P->h_final + words));
}

khz_status fill_stats(khz_ctx *ctx, BatchPlan *P, const LaunchStats &ls, bool timed, khz_stats *stats) {
    uint64_t ext = 0, bytes = 0;
    for (int r = 0; r < P->rows; ++r) {
        ext += P->h_final[(size_t)r * kRowWords + KHZ_MAX_COUNTS];
        bytes += P->h_final[(size_t)r * kRowWords + KHZ_MAX_COUNTS + 1];
    }
    stats->num_extensions = ext;
    stats->algo_bytes = bytes;
    stats->engine = P->engine;
    stats->launches = ls.launches;
    stats->kernel_ms = 0;
    uint64_t pb[kPhases] = {0, 0, 0, 0};
    KHZ_CUDA(cudaMemcpy(pb, P->d_phase_bytes, sizeof(pb), cudaMemcpyDeviceToHost));
    for (int p = 0; p < kPhases; ++p) {
        stats->phase_ms[p] = 0;
        stats->phase_bytes[p] = pb[p];
        stats->phase_launches[p] = ls.phase_launches[p];
        if (timed && ls.used[p]) {
            float f = 0;
            KHZ_CUDA(cudaEventElapsedTime(&f, ctx->ph_begin[p], ctx->ph_end[p]));
            stats->phase_ms[p] = f;
        }
    }
    if (timed) {
        float f = 0;
        KHZ_CUDA(cudaEventElapsedTime(&f, ctx->ev0, ctx->ev1));
        stats->kernel_ms = f;
    }
    return KHZ_OK;
}

// the cached prepared launch of one (graph, app) under the current configuration
khz_status cached_plan(khz_ctx *ctx, khz_graph g, int app, cudaStream_t s, BatchPlan **out, int64_t start_label = -1) {
    char key[192];
    snprintf(key, sizeof(key), "%u/%d/%d/%d/%d/%d/%d/%d/%lld", g, app, ctx->cfg.engine, ctx->cfg.want_algo_bytes,
             ctx->cfg.dfs_warps_per_sm, ctx->cfg.dfs_chunk, ctx->cfg.bitmap_warp_max, ctx->cfg.bitmap_hub_rows,
             (long long)start_label);
    auto it = ctx->plans.find(key);
    if (it != ctx->plans.end()) {
        *out = it->second.get();
        return KHZ_OK;
    }
    khz_job j{g, (int32_t)app, 0};
    std::unique_ptr<BatchPlan> P;
    khz_status st = build_plan(ctx, &j, 1, s, kPlanPoolMem | kPlanFreeLegacy, &P, &start_label);
    if (st) return st;
    *out = P.get();
    ctx->plans[key] = std::move(P);
    return KHZ_OK;
}

// the context's shared DFS slots (>= words) and pinned result buffer
khz_status ensure_shared(khz_ctx *ctx, uint64_t words) {
    if (!ctx->h_pinned) {
        if (cudaMallocHost(&ctx->h_pinned, sizeof(uint64_t) * (kRowWords + 1)) != cudaSuccess) {
            cudaGetLastError();
            ctx->h_pinned = nullptr;
            set_error("pinned result buffer allocation failed");
            return KHZ_ERR_OOM;
        }
    }
    if (words > ctx->shared_slot_words) {
        if (ctx->shared_slots) {
            cudaFree(ctx->shared_slots);  // waits for work still using it
            ctx->direct_bytes -= sizeof(uint32_t) * ctx->shared_slot_words;
        }
        ctx->shared_slots = nullptr;
        ctx->shared_slot_words = 0;
        if (over_mem_limit(ctx, sizeof(uint32_t) * words, "DFS scratch")) return KHZ_ERR_OOM;
        cudaError_t e = cudaMalloc(&ctx->shared_slots, sizeof(uint32_t) * words);
        if (e == cudaSuccess) ctx->direct_bytes += sizeof(uint32_t) * words;
        if (e != cudaSuccess) {
            cudaGetLastError();
            ctx->shared_slots = nullptr;
            set_error("DFS scratch of %llu bytes: %s", (unsigned long long)(4 * words), cudaGetErrorString(e));
            return KHZ_ERR_OOM;
        }
        ctx->shared_slot_words = words;
    }
    return KHZ_OK;
}


double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// HBM scratch one query needs while it runs: DFS slots sized by the graph's largest degree, or
// the bitmap engine's start-vertex lists; the CSR itself is resident and not counted
khz_status serve_footprint(khz_server *sv, khz_graph h, int app, uint64_t *bytes) {
    const uint64_t key = ((uint64_t)h << 20) | (uint64_t)app;
    std::lock_guard<std::mutex> fl(sv->fp_mu);  // lock order: fp_mu, then ctx->mu; never sv->mu here
    auto it = sv->footprints.find(key);
    if (it != sv->footprints.end()) {
        *bytes = it->second;
        return KHZ_OK;
    }
    khz_ctx *ctx = sv->ctx;
    std::lock_guard<std::mutex> lk(ctx->mu);
    Graph *g = get_graph(ctx, h);
    if (!g) return KHZ_ERR_ARG;
    const AppDef &def = app_def(app);
    uint64_t b = 1ull << 16;
    const int eng = pick_engine(ctx->cfg, def, app, *g);
    if (eng == KHZ_ENGINE_WEDGE) {
        b += 3 * 4 * (uint64_t)g->n;
    } else if (eng == KHZ_ENGINE_BITMAP) {
        Graph *og = nullptr;
        khz_status st = oriented_of(ctx, h, &og, nullptr);  // orient once, before any timing matters
        if (st) return st;
        b += BitmapLaunch::kTiers * 4 * (og->m / 33 + 1) +
             bitmap_hub_bytes(bitmap_hub_rows(ctx->cfg.bitmap_hub_rows, og->n, og->m));
        if (app == KHZ_KAUTO_4MOTIF || app == KHZ_KGPI_TAILED_TRIANGLE || app == KHZ_KGPI_HOUSE)  // identities
            b += 4 * og->m + 16 * (uint64_t)og->n + (app != KHZ_KGPI_TAILED_TRIANGLE ? 12 * (uint64_t)og->n : 0) +
                 (app == KHZ_KGPI_HOUSE ? 8 * og->m : 0);
        if (og->max_degree > bitmap_block_max_degree())
            b += 4 * dfs_slot_words(ctx->cfg.dfs_warps_per_sm, og->max_degree);
    } else {
        b += 4 * dfs_slot_words(ctx->cfg.dfs_warps_per_sm, g->max_degree);
    }
    sv->footprints[key] = b;
    *bytes = b;
    return KHZ_OK;
}

// finish every slot whose work is done; returns true if any slot is still busy
bool serve_reap(khz_server *sv) {
    bool any_busy = false;
    for (auto &sl : sv->slots) {
        if (!sl.busy) continue;
        const cudaError_t q = cudaEventQuery(sl.done);
        if (q == cudaErrorNotReady) {
            any_busy = true;
            continue;
        }
        const double t = now_s();
        khz_status st = KHZ_OK;
        if (q != cudaSuccess) st = cuda_fail(q, "serving slot");
        const size_t words = (size_t)kRowWords * sl.reqs.size();
        if (st == KHZ_OK) st = launch_flags_status(*(const unsigned int *)(sl.h_rows + words));
        {
            std::lock_guard<std::mutex> lk(sv->mu);
            for (size_t i = 0; i < sl.reqs.size(); ++i) {
                ServeResult &r = sv->results[sl.reqs[i].id];
                r.status = st;
                for (int c = 0; c < KHZ_MAX_COUNTS; ++c) r.counts[c] = sl.h_rows[i * kRowWords + c];
                r.num_ext = sl.h_rows[i * kRowWords + KHZ_MAX_COUNTS];
                r.latency_ms = (t - sl.reqs[i].t_submit) * 1000.0;
                r.done = true;
                sv->latencies.push_back(r.latency_ms);
                sv->completed += 1;
            }
            sv->t_last = t;
            sv->in_use -= sl.footprint;
        }
        sl.plan.reset();  // returns the scratch to the pool, ordered on the slot's stream
        sl.reqs.clear();
        sl.busy = false;
        sv->cv_done.notify_all();
    }
    return any_busy;
}

// admit pending queries into idle slots
void serve_dispatch(khz_server *sv) {
    for (auto &sl : sv->slots) {
        if (sl.busy) continue;
        std::vector<ServeRequest> take;
        uint64_t fp = 0;
        {
            std::lock_guard<std::mutex> lk(sv->mu);
            // the oldest query decides the size class of this launch; younger queries of the same
            // class join it (so a large query does not hold small ones back, and small ones batch)
            int cls = -1;
            for (auto it = sv->pending.begin(); it != sv->pending.end() && (int)take.size() < sv->max_batch;) {
                const ServeRequest &r = *it;
                if (cls >= 0 && r.size_class != cls) {
                    ++it;
                    continue;
                }
                const bool fits = sv->in_use + fp + r.footprint <= sv->budget;
                // a query larger than the whole budget still runs, alone, when nothing else does
                if (!fits && !(take.empty() && sv->in_use == 0)) break;
                cls = r.size_class;
                fp += r.footprint;
                take.push_back(r);
                it = sv->pending.erase(it);
            }
            if (take.empty()) return;
            sv->in_use += fp;
            sv->max_in_flight = std::max<uint64_t>(sv->max_in_flight, sv->in_use);
        }
        std::vector<khz_job> jobs(take.size());
        for (size_t i = 0; i < take.size(); ++i) jobs[i] = khz_job{take[i].graph, (int32_t)take[i].app, 0};
        khz_status st;
        {
            std::lock_guard<std::mutex> lk(sv->ctx->mu);
            st = build_plan(sv->ctx, jobs.data(), (int)jobs.size(), sl.stream, kPlanOwnSlots | kPlanPoolMem,
                            &sl.plan);
        }
        if (st == KHZ_OK) st = enqueue_plan(sl.plan.get(), sl.stream, nullptr, nullptr, nullptr);
        if (st == KHZ_OK) {
            const size_t words = (size_t)kRowWords * take.size();
            cudaError_t e = cudaMemcpyAsync(sl.h_rows, sl.plan->d_final, sizeof(uint64_t) * words,
                                            cudaMemcpyDeviceToHost, sl.stream);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(sl.h_rows + words, sl.plan->d_bad, sizeof(unsigned int), cudaMemcpyDeviceToHost,
                                    sl.stream);
            if (e == cudaSuccess) e = cudaEventRecord(sl.done, sl.stream);
            if (e != cudaSuccess) st = cuda_fail(e, "serving dispatch");
        }
        if (st != KHZ_OK) {
            const std::string why = khz_last_error_string();
            std::lock_guard<std::mutex> lk(sv->mu);
            for (auto &r : take) {
                ServeResult &res = sv->results[r.id];
                res.status = st;
                res.error = why;
                res.done = true;
            }
            sv->in_use -= fp;
            sl.plan.reset();
            sv->cv_done.notify_all();
            continue;
        }
        sl.reqs = std::move(take);
        sl.footprint = fp;
        sl.busy = true;
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->batches += 1;
    }
}

void serve_loop(khz_server *sv) {
    cudaSetDevice(sv->ctx->device);
    while (true) {
        serve_reap(sv);
        serve_dispatch(sv);
        bool busy = false;
        for (const auto &sl : sv->slots) busy = busy || sl.busy;
        std::unique_lock<std::mutex> lk(sv->mu);
        if (sv->stop && sv->pending.empty() && !busy) break;
        if (sv->pending.empty() && !busy) {
            sv->cv_work.wait_for(lk, std::chrono::milliseconds(50));
        } else {
            lk.unlock();
            std::this_thread::sleep_for(std::chrono::microseconds(20));
        }
    }
}

}  // namespace

extern "C" {

const char *khz_last_error_string(void) { return g_err; }
int khz_abi_version(void) { return KHZ_ABI_VERSION; }

khz_status khz_ctx_create(int device, khz_ctx **out) {
    if (!out) {
        set_error("null output pointer");
        return KHZ_ERR_ARG;
    }
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        set_error("no CUDA device available (%s)", cudaGetErrorString(e));
        return KHZ_ERR_CUDA;
    }
    if (device < 0 || device >= ndev) {
        set_error("device %d out of range [0, %d)", device, ndev);
        return KHZ_ERR_ARG;
    }
    KHZ_CUDA(cudaSetDevice(device));
    khz_ctx *c = new khz_ctx();
    c->device = device;
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    if (cudaMemPoolCreate(&c->pool, &props) != cudaSuccess) {
        cudaGetLastError();
        delete c;
        set_error("cudaMemPoolCreate failed");
        return KHZ_ERR_CUDA;
    }
    uint64_t keep = 4ull << 30;
    cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    c->cfg.engine = KHZ_ENGINE_AUTO;
    c->cfg.dfs_warps_per_sm = kDfsDefaultWarps;
    c->cfg.dfs_chunk = 8;
    c->cfg.bitmap_warp_max = 64;
    c->cfg.bitmap_block_warps = 16;
    bool ok = cudaEventCreate(&c->ev0) == cudaSuccess && cudaEventCreate(&c->ev1) == cudaSuccess;
    for (int p = 0; p < kPhases; ++p)
        ok = ok && cudaEventCreate(&c->ph_begin[p]) == cudaSuccess && cudaEventCreate(&c->ph_end[p]) == cudaSuccess;
    if (!ok) {
        delete c;
        set_error("cudaEventCreate failed");
        return KHZ_ERR_CUDA;
    }
    *out = c;
    return KHZ_OK;
}

khz_status khz_ctx_destroy(khz_ctx *ctx) {
    if (!ctx) return KHZ_OK;
    cudaSetDevice(ctx->device);
    cudaDeviceSynchronize();
    {
        AllocScope scope(ctx->pool, nullptr);
        for (size_t i = 0; i < ctx->graphs.size(); ++i)
            if (ctx->live[i]) free_graph_memory(&ctx->graphs[i]);
    }
    ctx->plans.clear();
    cudaDeviceSynchronize();  // the plans' pooled scratch is released on the legacy stream
    if (ctx->shared_slots) cudaFree(ctx->shared_slots);
    if (ctx->h_pinned) cudaFreeHost(ctx->h_pinned);
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    for (int p = 0; p < kPhases; ++p) {
        if (ctx->ph_begin[p]) cudaEventDestroy(ctx->ph_begin[p]);
        if (ctx->ph_end[p]) cudaEventDestroy(ctx->ph_end[p]);
    }
    delete ctx;
    return KHZ_OK;
}

khz_status khz_ctx_set_config(khz_ctx *ctx, const khz_config *cfg) {
    if (!ctx || !cfg) {
        set_error("null argument");
        return KHZ_ERR_ARG;
    }
    if (cfg->engine < 0 || cfg->engine > KHZ_ENGINE_WEDGE) {
        set_error("invalid engine %d", cfg->engine);
        return KHZ_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->cfg = *cfg;
    cudaDeviceSynchronize();  // a prepared launch of the previous configuration may still run
    ctx->plans.clear();
    if (ctx->cfg.dfs_warps_per_sm <= 0) ctx->cfg.dfs_warps_per_sm = kDfsDefaultWarps;
    if (ctx->cfg.dfs_chunk <= 0) ctx->cfg.dfs_chunk = 8;
    return KHZ_OK;
}

khz_status khz_ctx_get_config(khz_ctx *ctx, khz_config *cfg) {
    if (!ctx || !cfg) {
        set_error("null argument");
        return KHZ_ERR_ARG;
    }
    *cfg = ctx->cfg;
    return KHZ_OK;
}

khz_status khz_graph_from_edges(khz_ctx *ctx, const uint32_t *pairs, uint64_t m, uint32_t n, uint32_t flags,
                                khz_graph *out, void *stream) {
    khz_status st = check_ctx(ctx);
    if (st) return st;
    if (!out || (!pairs && m > 0)) {
        set_error("null argument");
        return KHZ_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaStream_t s = (cudaStream_t)stream;
    AllocScope scope(ctx->pool, s);
    const uint32_t *d_pairs = pairs;
    void *tmp = nullptr;
    if (!(flags & KHZ_EDGES_ON_DEVICE) && m > 0) {
        cudaError_t e = dev_alloc(&tmp, sizeof(uint32_t) * 2 * m);
        if (e != cudaSuccess) {
            cudaGetLastError();
            set_error("device allocation for %llu edges failed", (unsigned long long)m);
            return KHZ_ERR_OOM;
        }
        e = cudaMemcpyAsync(tmp, pairs, sizeof(uint32_t) * 2 * m, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) {
            dev_free(tmp);
            return cuda_fail(e, "edge upload");
        }
        d_pairs = (const uint32_t *)tmp;
    }
    Graph g;
    st = build_csr_from_device_pairs(d_pairs, m, n, !(flags & KHZ_UNCHECKED), &g, s);
    if (tmp) dev_free(tmp);
    if (st) return st;
    if (flags & KHZ_ORIENT) {
        Graph o;
        st = orient_graph(g, &o, s);
        free_graph_memory(&g);
        if (st) return st;
        g = o;
    }
    return register_graph(ctx, g, out);
}

khz_status khz_graph_load_dgraph(khz_ctx *ctx, const char *path, uint32_t flags, khz_graph *out) {
    if (!ctx || !path || !out) {
        set_error("null argument");
        return KHZ_ERR_ARG;
    }
    FILE *f = fopen(path, "rb");
    if (!f) {
        set_error("cannot open %s", path);
        return KHZ_ERR_NOT_FOUND;
    }
    unsigned char h[20];
    if (fread(h, 1, 20, f) != 20) {
        fclose(f);
        set_error("%s: short header", path);
        return KHZ_ERR_FORMAT;
    }
    uint32_t n;
    uint64_t m;
    int32_t has_label, has_edge_label;
    memcpy(&n, h, 4);
    memcpy(&m, h + 4, 8);
    memcpy(&has_label, h + 12, 4);
    memcpy(&has_edge_label, h + 16, 4);
    if (has_edge_label) {
        fclose(f);
        set_error("%s: edge labels are not supported (graph_loader.h:750)", path);
        return KHZ_ERR_FORMAT;
    }
    std::vector<uint32_t> labels;
    const bool keep_labels = has_label && !(flags & (KHZ_SKIP_LABELS | KHZ_ORIENT));
    if (keep_labels) {
        labels.resize(n);
        if (n > 0 && fread(labels.data(), 4, n, f) != n) {
            fclose(f);
            set_error("%s: truncated label section", path);
            return KHZ_ERR_FORMAT;
        }
    } else if (has_label) {
        fseek(f, 20 + 4 * (long)n, SEEK_SET);
    }
    uint32_t *pairs = nullptr;
    if (m > 0 && cudaMallocHost(&pairs, sizeof(uint32_t) * 2 * m) != cudaSuccess) {
        cudaGetLastError();
        fclose(f);
        set_error("pinned allocation for %llu edges failed", (unsigned long long)m);
        return KHZ_ERR_OOM;
    }
    const size_t got = m > 0 ? fread(pairs, 8, m, f) : 0;
    fclose(f);
    if (got != m) {
        cudaFreeHost(pairs);
        set_error("%s: truncated edge list (%llu of %llu)", path, (unsigned long long)got, (unsigned long long)m);
        return KHZ_ERR_FORMAT;
    }
    khz_status st = khz_graph_from_edges(ctx, pairs, m, n, flags & ~KHZ_EDGES_ON_DEVICE, out, nullptr);
    if (pairs) cudaFreeHost(pairs);
    if (st == KHZ_OK && keep_labels) {
        st = khz_graph_set_labels(ctx, *out, labels.data(), n);
        if (st != KHZ_OK) {
            const std::string why = khz_last_error_string();
            khz_graph_free(ctx, *out);
            *out = 0;
            set_error("%s: %s", path, why.c_str());
        }
    }
    return st;
}

khz_status khz_graph_orient(khz_ctx *ctx, khz_graph in, khz_graph *out, void *stream) {
    khz_status st = check_ctx(ctx);
    if (st) return st;
    std::lock_guard<std::mutex> lk(ctx->mu);
    Graph *g = get_graph(ctx, in);
    if (!g || !out) return KHZ_ERR_ARG;
    if (g->oriented) {
        set_error("graph %u is already oriented", in);
        return KHZ_ERR_ARG;
    }
    Graph o;
    AllocScope scope(ctx->pool, (cudaStream_t)stream);
    st = orient_graph(*g, &o, (cudaStream_t)stream);
    if (st) return st;
    return register_graph(ctx, o, out);
}

khz_status khz_graph_generate_rmat(khz_ctx *ctx, int scale, int edge_factor, double a, double b, double c,
                                   uint64_t seed, uint32_t flags, khz_graph *out, void *stream) {
    khz_status st = check_ctx(ctx);
    if (st) return st;
    if (!out) {
        set_error("null argument");
        return KHZ_ERR_ARG;
    }
    if (!(a >= 0 && b >= 0 && c >= 0 && a + b + c < 1.0)) {
        set_error("R-MAT probabilities must be >= 0 with a + b + c < 1");
        return KHZ_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    AllocScope scope(ctx->pool, (cudaStream_t)stream);
    Graph g;
    st = generate_rmat(scale, edge_factor, a, b, c, seed, &g, (cudaStream_t)stream);
    if (st) return st;
    if (flags & KHZ_ORIENT) {
        Graph o;
        st = orient_graph(g, &o, (cudaStream_t)stream);
        free_graph_memory(&g);
        if (st) return st;
        g = o;
    }
    return register_graph(ctx, g, out);
}

khz_status khz_graph_info_get(khz_ctx *ctx, khz_graph h, khz_graph_info *info) {
    if (!ctx || !info) {
        set_error("null argument");
        return KHZ_ERR_ARG;
    }
    Graph *g = get_graph(ctx, h);
    if (!g) return KHZ_ERR_ARG;
    memset(info, 0, sizeof(*info));
    info->num_vertices = g->n;
    info->num_entries = g->m;
    info->max_degree = g->max_degree;
    info->oriented = g->oriented ? 1 : 0;
    info->symmetric = g->symmetric ? 1 : 0;
    info->d_offsets = g->off;
    info->d_adj = g->adj;
    info->device_bytes = g->bytes;
    info->num_labels = g->num_labels;
    info->d_labels = g->labels;
    return KHZ_OK;
}

khz_status khz_graph_export_csr(khz_ctx *ctx, khz_graph h, uint64_t *offsets, uint32_t *adj) {
    khz_status st = check_ctx(ctx);
    if (st) return st;
    Graph *g = get_graph(ctx, h);
    if (!g) return KHZ_ERR_ARG;
    if (offsets) KHZ_CUDA(cudaMemcpy(offsets, g->off, sizeof(uint64_t) * ((size_t)g->n + 1), cudaMemcpyDeviceToHost));
    if (adj && g->m) KHZ_CUDA(cudaMemcpy(adj, g->adj, sizeof(uint32_t) * g->m, cudaMemcpyDeviceToHost));
    return KHZ_OK;
}

khz_status khz_graph_write_dgraph(khz_ctx *ctx, khz_graph h, const char *path, const uint32_t *labels) {
    khz_status st = check_ctx(ctx);
    if (st) return st;
    Graph *g = get_graph(ctx, h);
    if (!g || !path) return KHZ_ERR_ARG;
    std::vector<uint64_t> off(g->n + 1);
    std::vector<uint32_t> adj(g->m);
    st = khz_graph_export_csr(ctx, h, off.data(), adj.data());
    if (st) return st;
    FILE *f = fopen(path, "wb");
    if (!f) {
        set_error("cannot create %s", path);
        return KHZ_ERR_NOT_FOUND;
    }
    unsigned char hd[20];
    const uint32_t n = g->n;
    const uint64_t m = g->m;
    const int32_t hl = labels ? 1 : 0, he = 0;
    memcpy(hd, &n, 4);
    memcpy(hd + 4, &m, 8);
    memcpy(hd + 12, &hl, 4);
    memcpy(hd + 16, &he, 4);
    bool ok = fwrite(hd, 1, 20, f) == 20;
    if (labels) ok = ok && fwrite(labels, 4, n, f) == n;
    std::vector<uint32_t> buf;
    buf.reserve(1 << 20);
    for (uint32_t v = 0; v < n && ok; ++v) {
        for (uint64_t i = off[v]; i < off[v + 1]; ++i) {
            buf.push_back(v);
            buf.push_back(adj[i]);
        }
        if (buf.size() >= (1u << 20) || v + 1 == n) {
            ok = ok && fwrite(buf.data(), 4, buf.size(), f) == buf.size();
            buf.clear();
        }
    }
    fclose(f);
    if (!ok) {
        set_error("short write to %s", path);
        return KHZ_ERR_FORMAT;
    }
    return KHZ_OK;
}

khz_status khz_graph_set_labels(khz_ctx *ctx, khz_graph h, const uint32_t *labels, uint32_t num_vertices) {
    khz_status st = check_ctx(ctx);
    if (st) return st;
    if (!labels && num_vertices > 0) {
        set_error("null labels");
        return KHZ_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    Graph *g = get_graph(ctx, h);
    if (!g) return KHZ_ERR_ARG;
    if (num_vertices != g->n) {
        set_error("%u labels given for a graph of %u vertices", num_vertices, g->n);
        return KHZ_ERR_ARG;
    }
    // dense labels (graph_loader.h:784-804): num_labels = max + 1, every label used
    uint32_t mx = 0;
    for (uint32_t v = 0; v < num_vertices; ++v) mx = std::max(mx, labels[v]);
    if (num_vertices > 0 && mx == 0xffffffffu) {
        set_error("label 0xffffffff is out of range");
        return KHZ_ERR_FORMAT;
    }
    std::vector<uint64_t> cnt(num_vertices > 0 ? (size_t)mx + 1 : 0, 0);
    if (cnt.size() > (size_t)num_vertices) {
        set_error("the vertex labels should be continuous and range from 0 to num_labels - 1 (largest %u, %u vertices)",
                  mx, num_vertices);
        return KHZ_ERR_FORMAT;
    }
    for (uint32_t v = 0; v < num_vertices; ++v) cnt[labels[v]] += 1;
    for (size_t l = 0; l < cnt.size(); ++l) {
        if (cnt[l] == 0) {
            set_error("the vertex labels should be continuous and range from 0 to num_labels - 1 (label %zu unused)", l);
            return KHZ_ERR_FORMAT;
        }
    }
    KHZ_CUDA(cudaDeviceSynchronize());  // launches in flight may read the previous labels
    // prepared launches hold the label pointer: drop the graph's
    for (auto it = ctx->plans.begin(); it != ctx->plans.end();) {
        const auto &gs = it->second->graphs;
        if (std::find(gs.begin(), gs.end(), h) != gs.end()) it = ctx->plans.erase(it);
        else ++it;
    }
    AllocScope scope(ctx->pool, nullptr);
    dev_free(g->labels);
    g->labels = nullptr;
    g->num_labels = 0;
    g->label_count.clear();
    if (num_vertices == 0) return KHZ_OK;
    void *d = nullptr;
    cudaError_t e = dev_alloc(&d, sizeof(uint32_t) * num_vertices);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error("device allocation for %u labels failed", num_vertices);
        return KHZ_ERR_OOM;
    }
    e = cudaMemcpyAsync(d, labels, sizeof(uint32_t) * num_vertices, cudaMemcpyHostToDevice, nullptr);
    if (e == cudaSuccess) e = cudaStreamSynchronize(nullptr);
    if (e != cudaSuccess) {
        dev_free(d);
        return cuda_fail(e, "label upload");
    }
    g->labels = (uint32_t *)d;
    g->num_labels = (uint32_t)cnt.size();
    g->label_count = std::move(cnt);
    return KHZ_OK;
}

khz_status khz_graph_free(khz_ctx *ctx, khz_graph h) {
    khz_status st = check_ctx(ctx);
    if (st) return st;
    std::lock_guard<std::mutex> lk(ctx->mu);
    Graph *g = get_graph(ctx, h);
    if (!g) return KHZ_ERR_ARG;
    // work on any stream may still read the graph: order the release after all of it
    KHZ_CUDA(cudaDeviceSynchronize());
    const khz_graph ov = g->oriented_view, dv = g->degree_view;
    // prepared launches that hold the graph's (or its oriented view's) device pointers go with it;
    // the others stay cached
    for (auto it = ctx->plans.begin(); it != ctx->plans.end();) {
        const auto &gs = it->second->graphs;
        if (std::find(gs.begin(), gs.end(), h) != gs.end())
            it = ctx->plans.erase(it);
        else
            ++it;
    }
    AllocScope scope(ctx->pool, nullptr);
    free_graph_memory(g);
    ctx->live[h - 1] = false;
    for (const khz_graph view : {ov, dv}) {
        if (!view) continue;
        Graph *o = get_graph(ctx, view);
        if (o) {
            free_graph_memory(o);
            ctx->live[view - 1] = false;
        }
    }
    return KHZ_OK;
}

int khz_app_num_counts(khz_app_id app) {
    if (!app_known(app)) return 0;
    return app_def(app).num_counts;
}

int khz_app_multiplicity(khz_app_id app, int pattern) {
    if (!app_known(app)) return 0;
    const AppDef &d = app_def(app);
    if (pattern < 0 || pattern >= d.num_counts) return 0;
    return (int)d.mult[pattern];
}

khz_status khz_count_async(khz_ctx *ctx, khz_graph g, khz_app_id app, uint64_t *d_out, void *stream) {
    khz_status st = check_ctx(ctx);
    if (st) return st;
    if (!d_out) {
        set_error("null output");
        return KHZ_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaStream_t s = (cudaStream_t)stream;
    BatchPlan *P = nullptr;
    st = cached_plan(ctx, g, app, s, &P);
    if (st) return st;
    st = ensure_shared(ctx, P->slot_words);
    if (st) return st;
    st = enqueue_plan(P, s, nullptr, nullptr, nullptr, ctx->shared_slots);
    if (st) return st;
    KHZ_CUDA(cudaMemcpyAsync(d_out, P->d_final, sizeof(uint64_t) * kRowWords, cudaMemcpyDeviceToDevice, s));
    return KHZ_OK;
}

}  // extern "C"

namespace {
// khz_count and khz_count_restricted (start_label < 0: every start vertex)
khz_status count_one(khz_ctx *ctx, khz_graph g, khz_app_id app, int64_t start_label, uint64_t *counts,
                     khz_stats *stats, void *stream) {
    khz_status st = check_ctx(ctx);
    if (st) return st;
    if (!counts) {
        set_error("null counts");
        return KHZ_ERR_ARG;
    }
    if (!app_known(app)) {
        set_error("invalid app id %d", (int)app);
        return KHZ_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaStream_t s = (cudaStream_t)stream;
    BatchPlan *P = nullptr;
    st = cached_plan(ctx, g, app, s, &P, start_label);
    if (st) return st;
    st = ensure_shared(ctx, P->slot_words);
    if (st) return st;
    LaunchStats ls;
    ls.ev_begin = ctx->ph_begin;
    ls.ev_end = ctx->ph_end;
    st = enqueue_plan(P, s, &ls, ctx->ev0, ctx->ev1, ctx->shared_slots);
    if (st) return st;
    st = read_plan(P, s, ctx->h_pinned);
    if (st) return st;
    const int nc = app_def(app).num_counts;
    for (int c = 0; c < nc; ++c) counts[c] = P->h_final[c];
    if (stats) return fill_stats(ctx, P, ls, true, stats);
    return KHZ_OK;
}
}  // namespace

extern "C" {

khz_status khz_count(khz_ctx *ctx, khz_graph g, khz_app_id app, uint64_t *counts, khz_stats *stats, void *stream) {
    return count_one(ctx, g, app, -1, counts, stats, stream);
}

khz_status khz_count_restricted(khz_ctx *ctx, khz_graph g, khz_app_id app, uint32_t start_label, uint64_t *counts,
                                khz_stats *stats, void *stream) {
    return count_one(ctx, g, app, (int64_t)start_label, counts, stats, stream);
}

khz_status khz_count_batch(khz_ctx *ctx, const khz_job *jobs, int n_jobs, uint64_t *counts, uint64_t *num_ext,
                           khz_stats *stats, void *stream) {
    khz_status st = check_ctx(ctx);
    if (st) return st;
    if (!jobs || n_jobs <= 0 || !counts) {
        set_error("empty batch or null argument");
        return KHZ_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaStream_t s = (cudaStream_t)stream;
    std::unique_ptr<BatchPlan> P;
    st = build_plan(ctx, jobs, n_jobs, s, kPlanOwnSlots | kPlanPinned, &P);
    if (st) return st;
    LaunchStats ls;
    ls.ev_begin = ctx->ph_begin;
    ls.ev_end = ctx->ph_end;
    st = enqueue_plan(P.get(), s, &ls, ctx->ev0, ctx->ev1);
    if (st) return st;
    st = read_plan(P.get(), s);
    if (st) return st;
    for (int i = 0; i < n_jobs; ++i) {
        for (int c = 0; c < KHZ_MAX_COUNTS; ++c)
            counts[(size_t)i * KHZ_MAX_COUNTS + c] = P->h_final[(size_t)i * kRowWords + c];
        if (num_ext) num_ext[i] = P->h_final[(size_t)i * kRowWords + KHZ_MAX_COUNTS];
    }
    if (stats) return fill_stats(ctx, P.get(), ls, true, stats);
    return KHZ_OK;
}

khz_status khz_batch_create(khz_ctx *ctx, const khz_job *jobs, int n_jobs, uint32_t flags, khz_batch **out,
                            void *stream) {
    khz_status st = check_ctx(ctx);
    if (st) return st;
    if (!out || !jobs || n_jobs <= 0) {
        set_error("empty batch or null argument");
        return KHZ_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaStream_t s = (cudaStream_t)stream;
    std::unique_ptr<khz_batch> b(new khz_batch{ctx, nullptr});
    st = build_plan(ctx, jobs, n_jobs, s, kPlanOwnSlots | kPlanPinned, &b->plan);
    if (st) return st;
    if (flags & KHZ_BATCH_CUDA_GRAPH) {
        cudaStream_t cs = nullptr;
        KHZ_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            st = enqueue_plan(b->plan.get(), cs, nullptr, nullptr, nullptr);
            e = cudaStreamEndCapture(cs, &b->plan->graph);
        }
        if (e == cudaSuccess && st == KHZ_OK) e = cudaGraphInstantiate(&b->plan->exec, b->plan->graph, 0);
        cudaStreamDestroy(cs);
        if (st) return st;
        if (e != cudaSuccess) return cuda_fail(e, "capturing the batch into a CUDA graph");
    }
    *out = b.release();
    return KHZ_OK;
}

khz_status khz_batch_launch(khz_batch *b, void *stream) {
    if (!b) {
        set_error("null batch");
        return KHZ_ERR_ARG;
    }
    khz_status st = check_ctx(b->ctx);
    if (st) return st;
    cudaStream_t s = (cudaStream_t)stream;
    if (b->plan->exec) {
        KHZ_CUDA(cudaGraphLaunch(b->plan->exec, s));
        return KHZ_OK;
    }
    return enqueue_plan(b->plan.get(), s, nullptr, nullptr, nullptr);
}

khz_status khz_batch_wait(khz_batch *b, uint64_t *counts, uint64_t *num_ext, void *stream) {
    if (!b || !counts) {
        set_error("null argument");
        return KHZ_ERR_ARG;
    }
    khz_status st = check_ctx(b->ctx);
    if (st) return st;
    BatchPlan *P = b->plan.get();
    st = read_plan(P, (cudaStream_t)stream);
    if (st) return st;
    for (int i = 0; i < P->rows; ++i) {
        for (int c = 0; c < KHZ_MAX_COUNTS; ++c)
            counts[(size_t)i * KHZ_MAX_COUNTS + c] = P->h_final[(size_t)i * kRowWords + c];
        if (num_ext) num_ext[i] = P->h_final[(size_t)i * kRowWords + KHZ_MAX_COUNTS];
    }
    return KHZ_OK;
}

khz_status khz_batch_destroy(khz_batch *b) {
    if (!b) return KHZ_OK;
    cudaSetDevice(b->ctx->device);
    cudaDeviceSynchronize();
    delete b;
    return KHZ_OK;
}


khz_status khz_server_create(khz_ctx *ctx, int slots, int max_batch, uint64_t hbm_budget, khz_server **out) {
    khz_status st = check_ctx(ctx);
    if (st) return st;
    if (!out || slots < 1 || slots > 64 || max_batch < 1) {
        set_error("server needs 1..64 slots and max_batch >= 1");
        return KHZ_ERR_ARG;
    }
    std::unique_ptr<khz_server> sv(new khz_server());
    sv->ctx = ctx;
    sv->max_batch = max_batch;
    if (hbm_budget == 0) {
        size_t free_b = 0, total_b = 0;
        KHZ_CUDA(cudaMemGetInfo(&free_b, &total_b));
        hbm_budget = free_b / 2;
    }
    sv->budget = hbm_budget;
    sv->slots.resize(slots);
    for (auto &sl : sv->slots) {
        KHZ_CUDA(cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking));
        KHZ_CUDA(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming));
        if (cudaMallocHost(&sl.h_rows, sizeof(uint64_t) * ((size_t)kRowWords * max_batch + 1)) != cudaSuccess) {
            cudaGetLastError();
            set_error("pinned result buffer allocation failed");
            return KHZ_ERR_OOM;
        }
    }
    khz_server *p = sv.get();
    sv->worker = std::thread([p] { serve_loop(p); });
    *out = sv.release();
    return KHZ_OK;
}

khz_status khz_server_submit(khz_server *sv, khz_graph g, khz_app_id app, khz_ticket *ticket) {
    if (!sv || !ticket) {
        set_error("null argument");
        return KHZ_ERR_ARG;
    }
    if (!app_known(app)) {
        set_error("invalid app id %d", (int)app);
        return KHZ_ERR_ARG;
    }
    cudaSetDevice(sv->ctx->device);
    uint64_t fp = 0;
    khz_status st;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        if (sv->stop) {
            set_error("server is shutting down");
            return KHZ_ERR_BUSY;
        }
    }
    st = serve_footprint(sv, g, app, &fp);
    if (st) return st;
    int cls = 0;
    {
        std::lock_guard<std::mutex> lk(sv->ctx->mu);
        Graph *gp = get_graph(sv->ctx, g);
        if (!gp) return KHZ_ERR_ARG;
        for (uint64_t m = gp->m + 1; m > 1; m >>= 1) ++cls;
    }
    const double t = now_s();
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        const khz_ticket id = sv->next_ticket++;
        sv->pending.push_back(ServeRequest{id, g, (int)app, t, fp, cls});
        sv->results[id] = ServeResult{};
        if (sv->t_first < 0) sv->t_first = t;
        *ticket = id;
    }
    sv->cv_work.notify_one();
    return KHZ_OK;
}

khz_status khz_server_wait(khz_server *sv, khz_ticket ticket, uint64_t *counts, uint64_t *num_ext, double *latency_ms,
                           double timeout_ms) {
    if (!sv) {
        set_error("null server");
        return KHZ_ERR_ARG;
    }
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->results.find(ticket);
    if (it == sv->results.end()) {
        set_error("unknown ticket %llu", (unsigned long long)ticket);
        return KHZ_ERR_NOT_FOUND;
    }
    const auto deadline = std::chrono::steady_clock::now() +
                          std::chrono::microseconds((int64_t)(std::max(timeout_ms, 0.0) * 1000.0));
    while (!sv->results[ticket].done) {
        if (sv->cv_done.wait_until(lk, deadline) == std::cv_status::timeout && !sv->results[ticket].done) {
            set_error("ticket %llu not finished within %.3f ms", (unsigned long long)ticket, timeout_ms);
            return timeout_ms <= 0 ? KHZ_ERR_BUSY : KHZ_ERR_TIMEOUT;
        }
    }
    ServeResult r = sv->results[ticket];
    sv->results.erase(ticket);
    if (r.status == KHZ_ERR_CANCELLED) {
        set_error("ticket %llu was cancelled before it ran", (unsigned long long)ticket);
        return r.status;
    }
    if (r.status != KHZ_OK) {
        set_error("query failed (status %d): %s", (int)r.status, r.error.c_str());
        return r.status;
    }
    if (counts)
        for (int c = 0; c < KHZ_MAX_COUNTS; ++c) counts[c] = r.counts[c];
    if (num_ext) *num_ext = r.num_ext;
    if (latency_ms) *latency_ms = r.latency_ms;
    return KHZ_OK;
}

khz_status khz_server_stats_get(khz_server *sv, khz_server_stats *out) {
    if (!sv || !out) {
        set_error("null argument");
        return KHZ_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(sv->mu);
    memset(out, 0, sizeof(*out));
    out->completed = sv->completed;
    out->batches = sv->batches;
    out->pending = sv->pending.size();
    out->max_bytes_in_flight = sv->max_in_flight;
    std::vector<double> l = sv->latencies;
    if (!l.empty()) {
        std::sort(l.begin(), l.end());
        out->p50_ms = l[(size_t)(0.50 * (l.size() - 1))];
        out->p99_ms = l[(size_t)(0.99 * (l.size() - 1))];
        out->max_ms = l.back();
    }
    if (sv->completed > 0 && sv->t_last > sv->t_first) out->queries_per_s = sv->completed / (sv->t_last - sv->t_first);
    return KHZ_OK;
}

khz_status khz_server_reset_stats(khz_server *sv) {
    if (!sv) return KHZ_ERR_ARG;
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->latencies.clear();
    sv->completed = 0;
    sv->batches = 0;
    sv->max_in_flight = sv->in_use;
    sv->t_first = -1;
    return KHZ_OK;
}

khz_status khz_server_cancel(khz_server *sv, khz_ticket ticket) {
    if (!sv) {
        set_error("null server");
        return KHZ_ERR_ARG;
    }
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        auto it = sv->results.find(ticket);
        if (it == sv->results.end()) {
            set_error("unknown ticket %llu", (unsigned long long)ticket);
            return KHZ_ERR_NOT_FOUND;
        }
        auto p = std::find_if(sv->pending.begin(), sv->pending.end(),
                              [&](const ServeRequest &r) { return r.id == ticket; });
        if (p == sv->pending.end()) {
            set_error("ticket %llu is already admitted or finished", (unsigned long long)ticket);
            return KHZ_ERR_BUSY;
        }
        sv->pending.erase(p);
        it->second.status = KHZ_ERR_CANCELLED;
        it->second.done = true;
    }
    sv->cv_done.notify_all();
    return KHZ_OK;
}

khz_status khz_server_destroy(khz_server *sv) {
    if (!sv) return KHZ_OK;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stop = true;
    }
    sv->cv_work.notify_all();
    if (sv->worker.joinable()) sv->worker.join();
    cudaSetDevice(sv->ctx->device);
    for (auto &sl : sv->slots) {
        if (sl.stream) cudaStreamSynchronize(sl.stream);
        sl.plan.reset();
        if (sl.stream) cudaStreamDestroy(sl.stream);
        if (sl.done) cudaEventDestroy(sl.done);
        if (sl.h_rows) cudaFreeHost(sl.h_rows);
    }
    delete sv;
    return KHZ_OK;
}


khz_status khz_autotune(khz_ctx *ctx, const khz_job *jobs, int n_jobs, int reps, khz_tune_report *report) {
    khz_status st = check_ctx(ctx);
    if (st) return st;
    if (!jobs || n_jobs <= 0) {
        set_error("empty job list");
        return KHZ_ERR_ARG;
    }
    if (reps < 1) reps = 1;
    std::lock_guard<std::mutex> lk(ctx->mu);
    const khz_config base = ctx->cfg;
    cudaStream_t s = nullptr;
    KHZ_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    std::vector<uint64_t> ref;
    int trials = 0;
    // one measurement: prepare the launch under `c`, run it once to warm, then best of `reps`
    auto measure = [&](const khz_config &c, double *ms) -> khz_status {
        ctx->cfg = c;
        ctx->cfg.want_algo_bytes = 0;
        std::unique_ptr<BatchPlan> P;
        khz_status e = build_plan(ctx, jobs, n_jobs, s, kPlanOwnSlots | kPlanPinned, &P);
        if (e) return e;
        double best = 1e300;
        for (int r = 0; r <= reps; ++r) {
            e = enqueue_plan(P.get(), s, nullptr, ctx->ev0, ctx->ev1);
            if (e) return e;
            e = read_plan(P.get(), s);
            if (e) return e;
            float f = 0;
            KHZ_CUDA(cudaEventElapsedTime(&f, ctx->ev0, ctx->ev1));
            if (r > 0) best = std::min(best, (double)f);
        }
        std::vector<uint64_t> rows;
        for (int i = 0; i < n_jobs; ++i)
            for (int c2 = 0; c2 <= KHZ_MAX_COUNTS; ++c2) rows.push_back(P->h_final[(size_t)i * kRowWords + c2]);
        if (ref.empty()) ref = rows;
        else if (rows != ref) {
            set_error("autotuner: candidate configurations disagree on the counts");
            return KHZ_ERR_OVERFLOW;
        }
        ++trials;
        *ms = best;
        return KHZ_OK;
    };
    khz_config best = base;
    best.want_algo_bytes = 0;
    double best_ms = 0, base_ms = 0;
    st = measure(best, &base_ms);
    best_ms = base_ms;
    // coordinate descent over the knobs, each from the current best
    const int engines[] = {KHZ_ENGINE_AUTO, KHZ_ENGINE_DFS};
    const int warps[] = {8, 16, 24};
    const int chunks[] = {2, 8, 32};
    const int warp_max[] = {32, 64};
    const int hub_rows[] = {0, -1, 8192};  // auto (32768 on large graphs), none, a small triangle
    for (int pass = 0; pass < 2 && st == KHZ_OK; ++pass) {
        for (int knob = 0; knob < 5 && st == KHZ_OK; ++knob) {
            const int *vals = knob == 0 ? engines : knob == 1 ? warps : knob == 2 ? chunks : knob == 3 ? warp_max : hub_rows;
            const int nv = knob == 0 ? 2 : knob == 1 ? 3 : knob == 2 ? 3 : knob == 3 ? 2 : 3;
            for (int v = 0; v < nv && st == KHZ_OK; ++v) {
                khz_config c = best;
                int *field = knob == 0   ? &c.engine
                             : knob == 1 ? &c.dfs_warps_per_sm
                             : knob == 2 ? &c.dfs_chunk
                             : knob == 3 ? &c.bitmap_warp_max
                                         : &c.bitmap_hub_rows;
                if (*field == vals[v]) continue;
                *field = vals[v];
                double ms = 0;
                st = measure(c, &ms);
                if (st == KHZ_OK && ms < best_ms) {
                    best_ms = ms;
                    best = c;
                }
            }
        }
    }
    cudaStreamDestroy(s);
    ctx->cfg = st == KHZ_OK ? best : base;
    ctx->cfg.want_algo_bytes = base.want_algo_bytes;
    cudaDeviceSynchronize();
    ctx->plans.clear();
    if (st) return st;
    if (report) {
        report->trials = trials;
        report->baseline_ms = base_ms;
        report->best_ms = best_ms;
        report->best = ctx->cfg;
    }
    return KHZ_OK;
}

khz_status khz_set_op_batch(int op, const uint64_t *a_off, const uint32_t *a, const uint64_t *b_off,
                            const uint32_t *b, const uint32_t *bound, uint32_t *out, uint32_t *out_len,
                            uint32_t n_pairs, void *stream) {
    if (op < KHZ_SETOP_INTERSECT || op > KHZ_SETOP_TRIM_LOWER_BOUND) {
        set_error("invalid set op %d", op);
        return KHZ_ERR_ARG;
    }
    const bool needs_b = op <= KHZ_SETOP_BOUNDED_SUBTRACT;
    const bool needs_bound = op >= KHZ_SETOP_BOUNDED_INTERSECT;
    const bool writes = op == KHZ_SETOP_INTERSECT || op == KHZ_SETOP_SUBTRACT ||
                        op == KHZ_SETOP_BOUNDED_INTERSECT || op == KHZ_SETOP_BOUNDED_SUBTRACT;
    if (!a_off || !a || !out_len || (needs_b && (!b_off || !b)) || (needs_bound && !bound) || (writes && !out)) {
        set_error("null argument for set op %d", op);
        return KHZ_ERR_ARG;
    }
    if (n_pairs == 0) return KHZ_OK;
    int dev = 0, sms = 0;
    KHZ_CUDA(cudaGetDevice(&dev));
    KHZ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int blocks = (int)std::min<uint64_t>(((uint64_t)n_pairs + 7) / 8, (uint64_t)sms * 16);
    setop_batch_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(op, a_off, a, needs_b ? b_off : nullptr,
                                                                  needs_b ? b : nullptr, bound, out, out_len, n_pairs);
    KHZ_CUDA(cudaGetLastError());
    return KHZ_OK;
}

}  // extern "C"
