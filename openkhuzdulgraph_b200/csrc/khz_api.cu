// C ABI of the engine: context, graph table, counting dispatch, batching, set-op batch.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "khz_internal.cuh"
#include "setops.cuh"

namespace khz {

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

constexpr int kRow = KHZ_MAX_COUNTS + 2;

// divides the raw counters by the multiplicities and adds the host-known NumExtensions terms
__global__ void finalize_kernel(const uint64_t *raw, int rows, const uint32_t *mult, const uint64_t *ext_add,
                                uint64_t *out, unsigned int *bad) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    for (int c = 0; c < KHZ_MAX_COUNTS; ++c) {
        const uint64_t v = raw[(size_t)r * kRow + c];
        const uint32_t mu = mult[(size_t)r * KHZ_MAX_COUNTS + c];
        if (mu > 1 && v % mu) atomicOr(bad, 1u);
        out[(size_t)r * kRow + c] = mu > 1 ? v / mu : v;
    }
    out[(size_t)r * kRow + KHZ_MAX_COUNTS] = raw[(size_t)r * kRow + KHZ_MAX_COUNTS] + ext_add[r];
    out[(size_t)r * kRow + KHZ_MAX_COUNTS + 1] = raw[(size_t)r * kRow + KHZ_MAX_COUNTS + 1];
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

struct khz_ctx {
    int device = 0;
    khz_config cfg{};
    std::vector<Graph> graphs;  // handle h -> graphs[h - 1]
    std::vector<bool> live;
    Workspace ws;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t ph_begin[kPhases] = {}, ph_end[kPhases] = {};
    uint64_t *d_rows = nullptr;  // raw + final counter rows
    uint32_t *d_mult = nullptr;
    uint64_t *d_extadd = nullptr;
    unsigned int *d_bad = nullptr;
    size_t rows_cap = 0;
    cudaMemPool_t pool = nullptr;  // graphs and temporaries (keeps up to 4 GiB cached between calls)
    std::mutex mu;
};

namespace {

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

khz_status ensure_rows(khz_ctx *ctx, size_t rows) {
    if (ctx->rows_cap >= rows) return KHZ_OK;
    if (ctx->d_rows) cudaFree(ctx->d_rows);
    if (ctx->d_mult) cudaFree(ctx->d_mult);
    if (ctx->d_extadd) cudaFree(ctx->d_extadd);
    ctx->d_rows = nullptr;
    ctx->d_mult = nullptr;
    ctx->d_extadd = nullptr;
    ctx->rows_cap = 0;
    KHZ_CUDA(cudaMalloc(&ctx->d_rows, sizeof(uint64_t) * kRow * rows * 2));
    KHZ_CUDA(cudaMalloc(&ctx->d_mult, sizeof(uint32_t) * KHZ_MAX_COUNTS * rows));
    KHZ_CUDA(cudaMalloc(&ctx->d_extadd, sizeof(uint64_t) * rows));
    ctx->rows_cap = rows;
    return KHZ_OK;
}

khz_status ensure_counters(Workspace *ws) {
    if (ws->counters) return KHZ_OK;
    KHZ_CUDA(cudaMalloc(&ws->counters, 4096));
    ws->counters_bytes = 4096;
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
        g = get_graph(ctx, h);  // vector may have moved
        g->oriented_view = oh;
    }
    *out = get_graph(ctx, g->oriented_view);
    return KHZ_OK;
}

struct Enq {
    uint32_t launches = 0;
    uint32_t engine = 0;
    LaunchStats ls;  // per-phase events / bytes (timed calls only)
};

// Enqueue one (graph, app) count into raw row `row` (zeroed by the caller); returns the host-side
// NumExtensions addend (one depth-0 embedding per start vertex per run).
khz_status enqueue_count(khz_ctx *ctx, khz_graph h, int app, size_t row, std::vector<DfsJob> *dfs_jobs,
                         std::vector<Plan> *dfs_plans, uint64_t *ext_add, uint32_t *slot_cap, Enq *enq,
                         cudaStream_t s, bool batched) {
    const AppDef &def = app_def(app);
    Graph *g = get_graph(ctx, h);
    if (!g) return KHZ_ERR_ARG;
    const bool stats = ctx->cfg.want_algo_bytes != 0;
    int engine = ctx->cfg.engine;
    if (engine == KHZ_ENGINE_AUTO) engine = def.clique ? KHZ_ENGINE_BITMAP : KHZ_ENGINE_DFS;
    if (engine == KHZ_ENGINE_BITMAP && !def.clique) engine = KHZ_ENGINE_DFS;
    uint64_t *raw = ctx->d_rows + row * kRow;
    // the bitmap engine needs a DAG in id order; a symmetric graph is oriented first (cached);
    // any other shape runs the schedule as stored, like the reference does
    if (engine == KHZ_ENGINE_BITMAP && !g->oriented && !g->symmetric) engine = KHZ_ENGINE_DFS;
    if (engine == KHZ_ENGINE_BITMAP && !batched) {
        Graph *og = nullptr;
        khz_status st = oriented_of(ctx, h, &og, s);
        if (st) return st;
        uint32_t overflow = 0;
        const uint32_t before = enq->ls.launches;
        st = bitmap_clique_run(*og, def.clique_k, stats, ctx->cfg.bitmap_warp_max, ctx->cfg.bitmap_block_warps,
                               raw, &ctx->ws, s, &enq->ls, &overflow);
        if (st) return st;
        enq->launches += enq->ls.launches - before;
        if (overflow > 0) {
            DfsJob j{};
            j.off = og->off;
            j.adj = og->adj;
            j.n = og->n;
            j.num_units = og->m;
            j.out_base = (uint32_t)row;
            j.min_deg = bitmap_block_max_degree() + 1;
            j.plan_idx = (uint32_t)dfs_plans->size();
            dfs_plans->push_back(def.plans[0]);
            dfs_jobs->push_back(j);
            *slot_cap = std::max(*slot_cap, og->max_degree);
        }
        *ext_add = og->n;
        enq->engine = KHZ_ENGINE_BITMAP;
        return KHZ_OK;
    }
    // DFS engine on the graph as stored (oriented graphs use the oriented lists)
    for (int r = 0; r < def.num_runs; ++r) {
        DfsJob j{};
        j.off = g->off;
        j.adj = g->adj;
        j.n = g->n;
        j.num_units = g->m;
        j.out_base = (uint32_t)row;
        j.min_deg = 0;
        j.plan_idx = (uint32_t)dfs_plans->size();
        dfs_plans->push_back(def.plans[r]);
        dfs_jobs->push_back(j);
    }
    *slot_cap = std::max(*slot_cap, g->max_degree);
    *ext_add = (uint64_t)g->n * def.num_runs;
    enq->engine = KHZ_ENGINE_DFS;
    return KHZ_OK;
}

khz_status run_dfs(khz_ctx *ctx, std::vector<DfsJob> &jobs, std::vector<Plan> &plans, uint32_t slot_cap,
                   Enq *enq, cudaStream_t s) {
    if (jobs.empty()) return KHZ_OK;
    uint64_t begin = 0;
    for (auto &j : jobs) {
        j.unit_begin = begin;
        begin += j.num_units;
    }
    const uint32_t before = enq->ls.launches;
    khz_status st = dfs_run(jobs.data(), (int)jobs.size(), plans.data(), (int)plans.size(), slot_cap,
                            ctx->cfg.want_algo_bytes != 0, ctx->cfg.dfs_warps_per_sm, ctx->cfg.dfs_chunk,
                            ctx->d_rows, &ctx->ws, s, &enq->ls);
    enq->launches += enq->ls.launches - before;
    return st;
}

khz_status finalize(khz_ctx *ctx, const std::vector<int> &apps, const std::vector<uint64_t> &ext_add,
                    uint64_t *d_final, cudaStream_t s) {
    const size_t rows = apps.size();
    std::vector<uint32_t> mult(rows * KHZ_MAX_COUNTS, 1);
    for (size_t r = 0; r < rows; ++r) {
        const AppDef &d = app_def(apps[r]);
        for (int c = 0; c < KHZ_MAX_COUNTS; ++c) mult[r * KHZ_MAX_COUNTS + c] = c < d.num_counts ? d.mult[c] : 1;
    }
    KHZ_CUDA(cudaMemcpyAsync(ctx->d_mult, mult.data(), sizeof(uint32_t) * mult.size(), cudaMemcpyHostToDevice, s));
    KHZ_CUDA(cudaMemcpyAsync(ctx->d_extadd, ext_add.data(), sizeof(uint64_t) * rows, cudaMemcpyHostToDevice, s));
    finalize_kernel<<<(unsigned)((rows + 127) / 128), 128, 0, s>>>(ctx->d_rows, (int)rows, ctx->d_mult,
                                                                   ctx->d_extadd, d_final, ctx->d_bad);
    KHZ_CUDA(cudaGetLastError());
    return KHZ_OK;
}

khz_status count_many(khz_ctx *ctx, const khz_job *jobs, int n_jobs, uint64_t *d_final, cudaStream_t s,
                      Enq *enq, bool timed, double *ms) {
    for (int i = 0; i < n_jobs; ++i) {
        if (jobs[i].app < 0 || jobs[i].app >= KHZ_NUM_APPS) {
            set_error("invalid app id %d", jobs[i].app);
            return KHZ_ERR_ARG;
        }
        if (!get_graph(ctx, jobs[i].graph)) return KHZ_ERR_ARG;
    }
    khz_status st = ensure_rows(ctx, (size_t)n_jobs);
    if (st) return st;
    st = ensure_counters(&ctx->ws);
    if (st) return st;
    if (!ctx->d_bad) KHZ_CUDA(cudaMalloc(&ctx->d_bad, sizeof(unsigned int)));
    KHZ_CUDA(cudaMemsetAsync(ctx->d_bad, 0, sizeof(unsigned int), s));
    KHZ_CUDA(cudaMemsetAsync(ctx->d_rows, 0, sizeof(uint64_t) * kRow * n_jobs, s));
    // orientations are prepared before the timed region
    const bool batched = n_jobs > 1;
    if (!batched) {
        const AppDef &def = app_def(jobs[0].app);
        int engine = ctx->cfg.engine;
        Graph *g0 = get_graph(ctx, jobs[0].graph);
        if ((engine == KHZ_ENGINE_AUTO || engine == KHZ_ENGINE_BITMAP) && def.clique && !g0->oriented &&
            g0->symmetric) {
            Graph *og;
            st = oriented_of(ctx, jobs[0].graph, &og, s);
            if (st) return st;
        }
    }
    uint64_t *d_phase_bytes = ctx->ws.counters + 16;
    KHZ_CUDA(cudaMemsetAsync(d_phase_bytes, 0, sizeof(uint64_t) * kPhases, s));
    if (timed) {
        enq->ls.ev_begin = ctx->ph_begin;
        enq->ls.ev_end = ctx->ph_end;
        enq->ls.d_phase_bytes = d_phase_bytes;
    }
    if (timed) KHZ_CUDA(cudaEventRecord(ctx->ev0, s));
    std::vector<DfsJob> djobs;
    std::vector<Plan> plans;
    std::vector<uint64_t> ext_add(n_jobs, 0);
    std::vector<int> apps(n_jobs);
    uint32_t slot_cap = 32;
    for (int i = 0; i < n_jobs; ++i) {
        apps[i] = jobs[i].app;
        st = enqueue_count(ctx, jobs[i].graph, jobs[i].app, (size_t)i, &djobs, &plans, &ext_add[i], &slot_cap, enq,
                           s, batched);
        if (st) return st;
    }
    st = run_dfs(ctx, djobs, plans, slot_cap, enq, s);
    if (st) return st;
    if (timed) KHZ_CUDA(cudaEventRecord(ctx->ev1, s));
    st = finalize(ctx, apps, ext_add, d_final, s);
    if (st) return st;
    enq->launches += 1;
    if (timed) {
        KHZ_CUDA(cudaEventSynchronize(ctx->ev1));
        float f = 0;
        KHZ_CUDA(cudaEventElapsedTime(&f, ctx->ev0, ctx->ev1));
        *ms = f;
    }
    return KHZ_OK;
}

khz_status fill_phases(khz_ctx *ctx, const Enq &enq, khz_stats *stats, cudaStream_t s) {
    uint64_t pb[kPhases] = {0, 0, 0, 0};
    KHZ_CUDA(cudaMemcpyAsync(pb, ctx->ws.counters + 16, sizeof(pb), cudaMemcpyDeviceToHost, s));
    KHZ_CUDA(cudaStreamSynchronize(s));
    for (int p = 0; p < kPhases; ++p) {
        stats->phase_ms[p] = 0;
        stats->phase_bytes[p] = pb[p];
        stats->phase_launches[p] = enq.ls.phase_launches[p];
        if (enq.ls.used[p]) {
            float f = 0;
            KHZ_CUDA(cudaEventElapsedTime(&f, ctx->ph_begin[p], ctx->ph_end[p]));
            stats->phase_ms[p] = f;
        }
    }
    return KHZ_OK;
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
    c->cfg.dfs_warps_per_sm = 16;
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
    cudaDeviceSynchronize();
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    if (ctx->ws.slots) cudaFree(ctx->ws.slots);
    if (ctx->ws.counters) cudaFree(ctx->ws.counters);
    if (ctx->ws.tmp) cudaFree(ctx->ws.tmp);
    if (ctx->d_rows) cudaFree(ctx->d_rows);
    if (ctx->d_mult) cudaFree(ctx->d_mult);
    if (ctx->d_extadd) cudaFree(ctx->d_extadd);
    if (ctx->d_bad) cudaFree(ctx->d_bad);
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
    if (cfg->engine < 0 || cfg->engine > KHZ_ENGINE_BITMAP) {
        set_error("invalid engine %d", cfg->engine);
        return KHZ_ERR_ARG;
    }
    ctx->cfg = *cfg;
    if (ctx->cfg.dfs_warps_per_sm <= 0) ctx->cfg.dfs_warps_per_sm = 16;
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
    *out = add_graph(ctx, g);
    return KHZ_OK;
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
    if (has_label) fseek(f, 20 + 4 * (long)n, SEEK_SET);
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
    *out = add_graph(ctx, o);
    return KHZ_OK;
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
    *out = add_graph(ctx, g);
    return KHZ_OK;
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

khz_status khz_graph_free(khz_ctx *ctx, khz_graph h) {
    khz_status st = check_ctx(ctx);
    if (st) return st;
    std::lock_guard<std::mutex> lk(ctx->mu);
    Graph *g = get_graph(ctx, h);
    if (!g) return KHZ_ERR_ARG;
    // work on any stream may still read the graph: order the release after all of it
    KHZ_CUDA(cudaDeviceSynchronize());
    AllocScope scope(ctx->pool, nullptr);
    const khz_graph ov = g->oriented_view;
    free_graph_memory(g);
    ctx->live[h - 1] = false;
    if (ov) {
        Graph *o = get_graph(ctx, ov);
        if (o) {
            free_graph_memory(o);
            ctx->live[ov - 1] = false;
        }
    }
    return KHZ_OK;
}

int khz_app_num_counts(khz_app_id app) {
    if (app < 0 || app >= KHZ_NUM_APPS) return 0;
    return app_def(app).num_counts;
}

int khz_app_multiplicity(khz_app_id app, int pattern) {
    if (app < 0 || app >= KHZ_NUM_APPS) return 0;
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
    khz_job j{g, (int32_t)app, 0};
    Enq enq;
    double ms = 0;
    return count_many(ctx, &j, 1, d_out, (cudaStream_t)stream, &enq, false, &ms);
}

khz_status khz_count(khz_ctx *ctx, khz_graph g, khz_app_id app, uint64_t *counts, khz_stats *stats, void *stream) {
    khz_status st = check_ctx(ctx);
    if (st) return st;
    if (!counts) {
        set_error("null counts");
        return KHZ_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaStream_t s = (cudaStream_t)stream;
    khz_job j{g, (int32_t)app, 0};
    Enq enq;
    double ms = 0;
    st = ensure_rows(ctx, 1);
    if (st) return st;
    uint64_t *d_final = ctx->d_rows + ctx->rows_cap * kRow;
    st = count_many(ctx, &j, 1, d_final, s, &enq, true, &ms);
    if (st) return st;
    uint64_t row[kRow];
    unsigned int bad = 0;
    KHZ_CUDA(cudaMemcpyAsync(row, d_final, sizeof(row), cudaMemcpyDeviceToHost, s));
    KHZ_CUDA(cudaMemcpyAsync(&bad, ctx->d_bad, sizeof(bad), cudaMemcpyDeviceToHost, s));
    KHZ_CUDA(cudaStreamSynchronize(s));
    if (bad) {
        set_error("raw count not divisible by the pattern multiplicity (input is not an undirected graph)");
        return KHZ_ERR_MULTIPLICITY;
    }
    const int nc = app_def(app).num_counts;
    for (int c = 0; c < nc; ++c) counts[c] = row[c];
    if (stats) {
        stats->num_extensions = row[KHZ_MAX_COUNTS];
        stats->algo_bytes = row[KHZ_MAX_COUNTS + 1];
        stats->kernel_ms = ms;
        stats->engine = enq.engine;
        stats->launches = enq.launches;
        st = fill_phases(ctx, enq, stats, s);
        if (st) return st;
    }
    return KHZ_OK;
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
    st = ensure_rows(ctx, (size_t)n_jobs);
    if (st) return st;
    uint64_t *d_final = ctx->d_rows + ctx->rows_cap * kRow;
    Enq enq;
    double ms = 0;
    st = count_many(ctx, jobs, n_jobs, d_final, s, &enq, true, &ms);
    if (st) return st;
    std::vector<uint64_t> rows((size_t)n_jobs * kRow);
    unsigned int bad = 0;
    KHZ_CUDA(cudaMemcpyAsync(rows.data(), d_final, sizeof(uint64_t) * rows.size(), cudaMemcpyDeviceToHost, s));
    KHZ_CUDA(cudaMemcpyAsync(&bad, ctx->d_bad, sizeof(bad), cudaMemcpyDeviceToHost, s));
    KHZ_CUDA(cudaStreamSynchronize(s));
    if (bad) {
        set_error("raw count not divisible by the pattern multiplicity (input is not an undirected graph)");
        return KHZ_ERR_MULTIPLICITY;
    }
    for (int i = 0; i < n_jobs; ++i) {
        for (int c = 0; c < KHZ_MAX_COUNTS; ++c) counts[(size_t)i * KHZ_MAX_COUNTS + c] = rows[(size_t)i * kRow + c];
        if (num_ext) num_ext[i] = rows[(size_t)i * kRow + KHZ_MAX_COUNTS];
    }
    if (stats) {
        uint64_t ext = 0, bytes = 0;
        for (int i = 0; i < n_jobs; ++i) {
            ext += rows[(size_t)i * kRow + KHZ_MAX_COUNTS];
            bytes += rows[(size_t)i * kRow + KHZ_MAX_COUNTS + 1];
        }
        stats->num_extensions = ext;
        stats->algo_bytes = bytes;
        stats->kernel_ms = ms;
        stats->engine = KHZ_ENGINE_DFS;
        stats->launches = enq.launches;
        st = fill_phases(ctx, enq, stats, s);
        if (st) return st;
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
