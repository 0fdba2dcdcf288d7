// Per-warp DFS engine: the device form of EmbeddingExplorationEngine::extend_embeddings
// (engine.cc:914-1118) + scatter (engine.cc:1385-1453) + the apps' apply() levels.
//
// The reference runs levels breadth-first through bounded global queues of 36-byte
// compact embeddings and rebuilds each embedding through a parent chain.  Here one
// warp owns one partial embedding at a time and walks its subtree depth-first: the
// matched vertices live in registers, every materialised prefix ("cached object",
// engine.h:592-613) lives in the warp's stack frame in shared memory (or, when it can hold
// more than 256 members, in the warp's slot of a global arena), and every set operation is
// warp-cooperative
// (include/khz_setops.cuh).  Work distribution replaces WorkloadDistributer (engine.cc:1457-1496):
// a unit is one level-1 candidate, i.e. one CSR entry (v0, adj[e]); warps grab
// contiguous chunks of units from one atomic counter, so hub start vertices are split
// across many warps.  Per-job counters replace Aggregator<EdgeId> (engine.h:615-673):
// lanes accumulate in registers and a warp flushes with one atomicAdd per counter.
#include <cuda_runtime.h>

#include <algorithm>

#include "khz_internal.cuh"
#include "khz_setops.cuh"

namespace khz {

namespace {

constexpr int kOutStride = KHZ_MAX_COUNTS + 2;  // counts[6], num_ext, algo_bytes

// The warp's materialised sets (slots 2..5: level prefixes, the cached set, the two-op temporary)
// live in the warp's own shared-memory frame when the set can hold at most kSmemSlotWords members
// (bounded before the operation runs: |A n B| <= min(|A|, |B|), |A \ B| <= |A|), else in its slot
// of the global arena.  Deeper levels re-read these prefixes once per partial embedding, so the
// common small ones are read at shared-memory latency.
constexpr uint32_t kSmemSlotWords = 256;
constexpr int kSmemSlots = 4;  // slots 2, 3, 4, 5
// dynamic shared memory of a launch: one frame per warp (4 KiB)
size_t dfs_smem_bytes(int threads) { return (size_t)(threads / 32) * kSmemSlots * kSmemSlotWords * sizeof(uint32_t); }

struct WarpCtx {
    const Plan *plan;
    const uint64_t *off;
    const uint32_t *adj;
    uint32_t *slot_base;  // this warp's kNumSlots * slot_cap words of the global arena
    uint32_t *smem_base;  // this warp's kSmemSlots * kSmemSlotWords words of shared memory
    uint32_t slot_cap;
    uint32_t in_smem;     // bit s: slot s currently lives in shared memory
    uint32_t v[kMaxK];
    uint32_t slot_len[kNumSlots];
    uint64_t acc[KHZ_MAX_COUNTS];
    uint64_t ext;
    uint64_t bytes;
    __device__ __forceinline__ uint32_t *slot(int s) const {
        return ((in_smem >> s) & 1u) ? smem_base + (size_t)(s - 2) * kSmemSlotWords : slot_base + (size_t)s * slot_cap;
    }
    // choose where slot s is written for a set of at most `bound` members, and return it
    __device__ __forceinline__ uint32_t *place(int s, uint32_t bound) {
        if (bound <= kSmemSlotWords) in_smem |= 1u << s;
        else in_smem &= ~(1u << s);
        return slot(s);
    }
    __device__ __forceinline__ const uint32_t *nbr(uint32_t v) const { return adj + off[v]; }
    __device__ __forceinline__ uint32_t deg(uint32_t v) const { return (uint32_t)(off[v + 1] - off[v]); }
};

__device__ __forceinline__ Filter make_filter(const WarpCtx &c, uint8_t gt_mask, uint8_t ne_mask, bool bounded) {
    Filter f;
    f.lb = 0;
    f.has_lb = 0;
    f.nne = 0;
#pragma unroll
    for (int a = 0; a < kMaxK; ++a) {
        if (gt_mask & (1u << a)) {
            if (!f.has_lb || c.v[a] > f.lb) f.lb = c.v[a];
            f.has_lb = 1;
        }
    }
#pragma unroll
    for (int a = 0; a < kMaxK; ++a) {
        if ((ne_mask & (1u << a)) && f.nne < 4) f.ne[f.nne++] = c.v[a];
    }
    (void)bounded;
    return f;
}

__device__ __forceinline__ void base_of(WarpCtx &c, const SetExpr &e, const uint32_t *&p, uint32_t &n) {
    if (e.base_kind == BASE_NBR) {
        const uint32_t v = c.v[e.base_arg];
        p = c.nbr(v);
        n = c.deg(v);
    } else {
        p = c.slot(e.base_arg);
        n = c.slot_len[e.base_arg];
    }
}

// One set operation A op N(x) -> either written to `out` or only counted.
// When `trim_lb` the operands are first cut to their members > f.lb (valid for counting
// and for bounded materialisation; never used in the instrumented variant).
template <bool STATS>
__device__ ProbeResult apply_op(WarpCtx &c, int8_t op, const uint32_t *A, uint32_t na, uint32_t x, uint32_t *out,
                                const Filter &f, bool trim_lb) {
    const uint32_t *B = c.nbr(x);
    uint32_t nb = c.deg(x);
    const uint32_t na_full = na, nb_full = nb;
    if (!STATS && trim_lb && f.has_lb) {
        const uint32_t sa = upper_bound_plain(A, 0, na, f.lb);
        A += sa;
        na -= sa;
        const uint32_t sb = upper_bound_u32(B, 0, nb, f.lb);
        B += sb;
        nb -= sb;
    }
    ProbeResult r;
    if (op == OP_AND) {
        if (na <= nb) r = warp_probe<false>(A, na, B, nb, out, f);
        else r = warp_probe<false>(B, nb, A, na, out, f);
    } else {
        r = warp_probe<true>(A, na, B, nb, out, f);
    }
    if (STATS) c.bytes += 4ull * ((uint64_t)na_full + nb_full + r.full);
    return r;
}

// most members `A op N(x)` can have
__device__ __forceinline__ uint32_t op_bound(const WarpCtx &c, int8_t op, uint32_t na, uint32_t x) {
    return op == OP_AND ? min(na, c.deg(x)) : na;
}

// Materialise expression e (with 1 or 2 ops) into slot `dst`; returns its size.
template <bool STATS>
__device__ uint32_t materialise(WarpCtx &c, const SetExpr &e, int dst, const Filter &f, bool bounded) {
    const uint32_t *A;
    uint32_t na;
    base_of(c, e, A, na);
    const Filter none = {0, 0, 0, {0, 0, 0, 0}};
    __syncwarp();  // every lane is done reading the previous contents of the slots
    const uint32_t b0 = op_bound(c, e.op[0], na, c.v[e.op_arg[0]]);
    if (e.op[1] == OP_NONE) {
        ProbeResult r = apply_op<STATS>(c, e.op[0], A, na, c.v[e.op_arg[0]], c.place(dst, b0), bounded ? f : none,
                                        bounded);
        return r.full;
    }
    ProbeResult t = apply_op<STATS>(c, e.op[0], A, na, c.v[e.op_arg[0]], c.place(5, b0), bounded ? f : none, bounded);
    c.slot_len[5] = t.full;
    __syncwarp();
    ProbeResult r = apply_op<STATS>(c, e.op[1], c.slot(5), t.full, c.v[e.op_arg[1]],
                                    c.place(dst, op_bound(c, e.op[1], t.full, c.v[e.op_arg[1]])), bounded ? f : none,
                                    bounded);
    return r.full;
}

// Count-only `A op N(x)` filtered by f.  A subtraction is counted as |A passing f| minus
// |A n N(x) passing f|, which probes the shorter of the two lists instead of all of A (the
// instrumented variant keeps the reference's full subtraction so its byte count is the schedule's).
template <bool STATS>
__device__ __forceinline__ uint32_t count_op(WarpCtx &c, int8_t op, const uint32_t *A, uint32_t na, uint32_t x,
                                            const Filter &f) {
    if (!STATS && op == OP_SUB) {
        const uint32_t pass_a = warp_count_plain(A, na, f);
        return pass_a - apply_op<STATS>(c, OP_AND, A, na, x, nullptr, f, true).filtered;
    }
    return apply_op<STATS>(c, op, A, na, x, nullptr, f, true).filtered;
}

template <bool STATS>
__device__ void count_last(WarpCtx &c) {
    const Plan &p = *c.plan;
    for (int ti = 0; ti < p.num_terms; ++ti) {
        const Term &t = p.last[ti];
        if (t.guard_lo >= 0 && !(c.v[t.guard_lo] < c.v[t.guard_hi])) continue;
        const Filter f = make_filter(c, t.gt_mask, t.ne_mask, true);
        const uint32_t *A;
        uint32_t na;
        base_of(c, t.set, A, na);
        uint32_t cnt;
        if (t.set.op[0] == OP_NONE) {
            cnt = warp_count_plain(A, na, f);
        } else if (t.set.op[1] == OP_NONE) {
            cnt = count_op<STATS>(c, t.set.op[0], A, na, c.v[t.set.op_arg[0]], f);
        } else {
            const Filter none = {0, 0, 0, {0, 0, 0, 0}};
            // first op materialised (bounded by the term's lower bound when not instrumented)
            __syncwarp();
            ProbeResult r0 = apply_op<STATS>(c, t.set.op[0], A, na, c.v[t.set.op_arg[0]],
                                             c.place(5, op_bound(c, t.set.op[0], na, c.v[t.set.op_arg[0]])),
                                             STATS ? none : f, !STATS);
            __syncwarp();
            cnt = count_op<STATS>(c, t.set.op[1], c.slot(5), r0.full, c.v[t.set.op_arg[1]], f);
        }
        if (lane_id() == 0) c.acc[t.counter] += cnt;
    }
}

template <int L, bool STATS>
__device__ void dfs_level(WarpCtx &c) {
    const Plan &p = *c.plan;
    if (L == p.k - 1) {
        count_last<STATS>(c);
        return;
    }
    if constexpr (L < kMaxK - 1) {
        const Level &lv = p.lv[L];
        if (lv.has_extra) {
            const Filter none = {0, 0, 0, {0, 0, 0, 0}};
            c.slot_len[4] = materialise<STATS>(c, lv.extra, 4, none, false);
            __syncwarp();
        }
        const Filter f = make_filter(c, lv.t.gt_mask, lv.t.ne_mask, false);
        const uint32_t *S;
        uint32_t ns;
        if (lv.t.set.op[0] == OP_NONE) {
            base_of(c, lv.t.set, S, ns);
        } else {
            // bounded materialisation where the plan allows it: level sets then are only ever
            // re-read above their own lower bound (every later use filters by a larger matched vertex)
            c.slot_len[L] = materialise<STATS>(c, lv.t.set, L, f, !STATS && p.bounded_sets);
            __syncwarp();
            S = c.slot(L);
            ns = c.slot_len[L];
        }
        uint32_t i = f.has_lb ? upper_bound_plain(S, 0, ns, f.lb) : 0;
        for (; i < ns; ++i) {
            const uint32_t x = S[i];
            if (!f.pass(x)) continue;
            c.v[L] = x;
            if (!lv.finalized && lane_id() == 0) c.ext++;
            dfs_level<L + 1, STATS>(c);
        }
    }
}

__device__ __forceinline__ void flush(WarpCtx &c, uint64_t *row, int ncounters, uint64_t *phase_bytes) {
    if (lane_id() == 0) {
        for (int k = 0; k < ncounters; ++k)
            if (c.acc[k]) atomicAdd((unsigned long long *)&row[k], (unsigned long long)c.acc[k]);
        if (c.ext) atomicAdd((unsigned long long *)&row[KHZ_MAX_COUNTS], (unsigned long long)c.ext);
        if (c.bytes) atomicAdd((unsigned long long *)&row[KHZ_MAX_COUNTS + 1], (unsigned long long)c.bytes);
        if (c.bytes && phase_bytes) atomicAdd((unsigned long long *)phase_bytes, (unsigned long long)c.bytes);
    }
    for (int k = 0; k < KHZ_MAX_COUNTS; ++k) c.acc[k] = 0;
    c.ext = 0;
    c.bytes = 0;
}

template <bool STATS>
__global__ void __launch_bounds__(256) dfs_kernel(const DfsJob *__restrict__ jobs, int n_jobs,
                                                  const Plan *__restrict__ plans, uint64_t total_units,
                                                  uint32_t chunk, uint32_t *slots, uint32_t slot_cap,
                                                  unsigned long long *queue, uint64_t *out,
                                                  uint64_t *phase_bytes) {
    __shared__ Plan s_plans[4];
    const int n_plans_cached = 4;
    for (int i = threadIdx.x; i < (int)(sizeof(Plan) * n_plans_cached / 4); i += blockDim.x) {
        // plans are small PODs: copy the first few into shared memory word by word
        ((uint32_t *)s_plans)[i] = ((const uint32_t *)plans)[i];
    }
    __syncthreads();
    extern __shared__ __align__(16) uint32_t dsm[];  // kSmemSlots * kSmemSlotWords words per warp
    const unsigned lane = lane_id();
    const uint32_t warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    WarpCtx c;
    c.slot_base = slots + (size_t)warp_global * kNumSlots * slot_cap;
    c.smem_base = dsm + (size_t)(threadIdx.x >> 5) * kSmemSlots * kSmemSlotWords;
    c.in_smem = 0;
    c.slot_cap = slot_cap;
    for (int k = 0; k < KHZ_MAX_COUNTS; ++k) c.acc[k] = 0;
    c.ext = 0;
    c.bytes = 0;
    int cur_job = -1;
    uint32_t v0 = 0;
    uint64_t v0_end = 0;
    while (true) {
        unsigned long long u0 = 0;
        if (lane == 0) u0 = atomicAdd(queue, (unsigned long long)chunk);
        u0 = __shfl_sync(kFull, u0, 0);
        if (u0 >= total_units) break;
        const uint64_t u1 = (uint64_t)u0 + chunk < total_units ? (uint64_t)u0 + chunk : total_units;
        for (uint64_t u = u0; u < u1; ++u) {
            // locate the job (jobs are sorted by unit_begin)
            if (cur_job < 0 || u < jobs[cur_job].unit_begin ||
                u >= jobs[cur_job].unit_begin + jobs[cur_job].num_units) {
                if (cur_job >= 0) flush(c, out + (size_t)jobs[cur_job].out_base * kOutStride, KHZ_MAX_COUNTS, phase_bytes);
                int lo = 0, hi = n_jobs - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (jobs[mid].unit_begin <= u) lo = mid; else hi = mid - 1;
                }
                cur_job = lo;
                const DfsJob &J = jobs[cur_job];
                c.off = J.off;
                c.adj = J.adj;
                c.plan = J.plan_idx < (uint32_t)n_plans_cached ? &s_plans[J.plan_idx] : &plans[J.plan_idx];
                v0_end = 0;
            }
            const DfsJob &J = jobs[cur_job];
            const uint64_t e = u - J.unit_begin;
            if (e >= v0_end || e < (v0_end == 0 ? 0 : c.off[v0])) {
                // find v0 with off[v0] <= e < off[v0 + 1]
                uint32_t lo = 0, hi = J.n - 1;
                while (lo < hi) {
                    const uint32_t mid = (lo + hi + 1) >> 1;
                    if (c.off[mid] <= e) lo = mid; else hi = mid - 1;
                }
                v0 = lo;
                v0_end = c.off[v0 + 1];
            }
            if (v0_end - c.off[v0] < J.min_deg || !J.start.keep(v0)) {
                // no unit of this start vertex is extended: skip to its last unit in the chunk
                const uint64_t next = J.unit_begin + v0_end;
                u = (next < u1 ? next : u1) - 1;
                continue;
            }
            const Plan &p = *c.plan;
            const Level &l1 = p.lv[1];
            c.v[0] = v0;
            const uint32_t x = c.adj[e];
            const Filter f1 = make_filter(c, l1.t.gt_mask, l1.t.ne_mask, false);
            if (!f1.pass(x)) continue;
            c.v[1] = x;
            if (!l1.finalized && lane == 0) c.ext++;
            dfs_level<2, STATS>(c);
        }
    }
    if (cur_job >= 0) flush(c, out + (size_t)jobs[cur_job].out_base * kOutStride, KHZ_MAX_COUNTS, phase_bytes);
}

}  // namespace

// Launch the (uninstrumented) DFS kernel on caller-provided device tables and scratch; no
// allocation and no host synchronisation.
khz_status dfs_launch_prealloc(const DfsJob *d_jobs, int n_jobs, const Plan *d_plans, uint64_t total_units,
                               uint32_t chunk, uint32_t *slots, uint32_t slot_cap, unsigned long long *queue,
                               uint64_t *d_raw, int blocks, int threads, cudaStream_t s) {
    dfs_kernel<false><<<blocks, threads, dfs_smem_bytes(threads), s>>>(d_jobs, n_jobs, d_plans, total_units, chunk, slots, slot_cap, queue,
                                                 d_raw, nullptr);
    KHZ_CUDA(cudaGetLastError());
    return KHZ_OK;
}

namespace {
constexpr int kDfsWarpsPerBlock = 8;
int num_sms_dfs() {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms > 0 ? sms : 1;
}
int dfs_blocks(int warps_per_sm) {
    if (warps_per_sm <= 0) warps_per_sm = 16;
    return num_sms_dfs() * ((warps_per_sm + kDfsWarpsPerBlock - 1) / kDfsWarpsPerBlock);
}
uint32_t round_cap(uint32_t slot_cap) { return slot_cap == 0 ? 32u : ((slot_cap + 31u) & ~31u); }
}  // namespace

uint64_t dfs_total_warps(int warps_per_sm) { return (uint64_t)dfs_blocks(warps_per_sm) * kDfsWarpsPerBlock; }

uint64_t dfs_slot_words(int warps_per_sm, uint32_t slot_cap) {
    return dfs_total_warps(warps_per_sm) * kNumSlots * round_cap(slot_cap);
}

size_t dfs_arena_bytes(int n_jobs, int n_plans, uint64_t total_warps, uint32_t slot_cap, bool own_slots) {
    return Arena::round(sizeof(DfsJob) * (size_t)std::max(n_jobs, 1)) +
           Arena::round(sizeof(Plan) * (size_t)std::max(n_plans, 4)) +
           (own_slots ? Arena::round(total_warps * kNumSlots * round_cap(slot_cap) * sizeof(uint32_t)) : 0) +
           Arena::round(sizeof(unsigned long long));
}

khz_status dfs_prepare(const std::vector<DfsJob> &jobs, const std::vector<Plan> &plans, uint32_t slot_cap,
                       int warps_per_sm, int chunk, bool stats, bool own_slots, Arena *arena, DfsLaunch *dl,
                       cudaStream_t s) {
    DfsLaunch L;
    L.n_jobs = (int)jobs.size();
    L.stats = stats;
    L.chunk = chunk > 0 ? (uint32_t)chunk : 8u;
    L.blocks = dfs_blocks(warps_per_sm);
    L.threads = kDfsWarpsPerBlock * 32;
    L.slot_cap = round_cap(slot_cap);
    for (const auto &j : jobs) L.total_units = std::max(L.total_units, j.unit_begin + j.num_units);
    DfsJob *d_jobs = arena->take<DfsJob>(jobs.size());
    // the kernel stages the first four plans into shared memory: keep at least four readable
    Plan *d_plans = arena->take<Plan>(std::max<size_t>(plans.size(), 4));
    L.slots = own_slots ? arena->take<uint32_t>((size_t)L.blocks * kDfsWarpsPerBlock * kNumSlots * L.slot_cap)
                        : nullptr;
    L.queue = arena->take<unsigned long long>(1);
    if (!d_jobs || !d_plans || (own_slots && !L.slots) || !L.queue) {
        set_error("DFS launch arena too small");
        return KHZ_ERR_OOM;
    }
    if (!jobs.empty())
        KHZ_CUDA(cudaMemcpyAsync(d_jobs, jobs.data(), sizeof(DfsJob) * jobs.size(), cudaMemcpyHostToDevice, s));
    KHZ_CUDA(cudaMemsetAsync(d_plans, 0, sizeof(Plan) * std::max<size_t>(plans.size(), 4), s));
    if (!plans.empty())
        KHZ_CUDA(cudaMemcpyAsync(d_plans, plans.data(), sizeof(Plan) * plans.size(), cudaMemcpyHostToDevice, s));
    L.d_jobs = d_jobs;
    L.d_plans = d_plans;
    *dl = L;
    return KHZ_OK;
}

khz_status dfs_enqueue(const DfsLaunch &L, uint64_t *d_rows, cudaStream_t s, LaunchStats *ls, uint32_t *slots) {
    if (L.n_jobs == 0 || L.total_units == 0) return KHZ_OK;
    if (!slots) slots = L.slots;
    if (!slots) {
        set_error("DFS launch has no slot scratch");
        return KHZ_ERR_ARG;
    }
    KHZ_CUDA(cudaMemsetAsync(L.queue, 0, sizeof(unsigned long long), s));
    uint64_t *pb = ls && ls->d_phase_bytes ? ls->d_phase_bytes + 3 : nullptr;
    if (ls && ls->ev_begin) cudaEventRecord(ls->ev_begin[3], s);
    if (L.stats)
        dfs_kernel<true><<<L.blocks, L.threads, dfs_smem_bytes(L.threads), s>>>(L.d_jobs, L.n_jobs, L.d_plans, L.total_units, L.chunk, slots,
                                                        L.slot_cap, L.queue, d_rows, pb);
    else
        dfs_kernel<false><<<L.blocks, L.threads, dfs_smem_bytes(L.threads), s>>>(L.d_jobs, L.n_jobs, L.d_plans, L.total_units, L.chunk,
                                                         slots, L.slot_cap, L.queue, d_rows, pb);
    KHZ_CUDA(cudaGetLastError());
    if (ls && ls->ev_begin) {
        cudaEventRecord(ls->ev_end[3], s);
        ls->used[3] = true;
        ls->phase_launches[3] += 1;
    }
    if (ls) ls->launches += 1;
    return KHZ_OK;
}

}  // namespace khz
