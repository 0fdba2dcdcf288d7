// Wedge engine for the 4-cycle app on symmetric graphs.
//
// The schedule (kgraphpi idiom: v1 > v0, v2 in N(v1) with v2 > v0, last level
// |{v3 in N(v0) n N(v2) : v3 > v1}| minus matched vertices) intersects N(v0) with N(v2) once per
// partial embedding (v0, v1, v2).  Grouped by (v0, v2) its count is C(c, 2) with
// c = |{w in N(v0) n N(v2) : w > v0}|, so this engine enumerates every wedge (v0, w, v2) with
// w > v0 and v2 > v0 exactly once and counts wedge endpoints v2 per start vertex.  An increment
// that returns the previous count `old` adds `old` to the result: summed over a run of c increments
// that is C(c, 2), so no second pass is needed.  The wedges enumerated are exactly the schedule's
// level-2 embeddings, so NumExtensions = n + |E| + #wedges.
//
// Tiers by the number of wedges of v0 (an upper bound on distinct endpoints): one warp with a
// 512-slot shared hash (<= 384 wedges), one block with an 8192-slot shared hash (<= 6144), or one
// 1024-thread block with dense counters in shared memory over a window of endpoint ids (106496
// 16-bit counters, or 53248 32-bit ones when a degree reaches 65535), the endpoints v2 > v0 taken
// one window at a time; each neighbour list's part inside the window is bounded by splitters.
//
// House jobs (WJob::tri set) walk each start vertex's wedges (or window) a second time once the
// endpoint counts are final, reading them without atomics: a pair (v0, v2) with c common
// neighbours closes C(c, 2) 4-cycles, and over those cycles each wedge (v0, w, v2) appears in c - 1,
// so sum over wedges of (c - 1)(t(v0 w) + t(w v2)) is the sum over 4-cycles of the triangle counts
// of their four edges.
#include <cuda_runtime.h>

#include "khz_internal.cuh"
#include "khz_setops.cuh"

namespace khz {
namespace {

constexpr uint32_t kEmptyKey = 0xffffffffu;
constexpr int kWarpSlots = 512, kWarpWedges = 384;
constexpr int kBlockSlots = 8192, kBlockWedges = 6144;
constexpr int kBlockThreads = 512;
constexpr int kWinThreads = 1024;
constexpr uint32_t kWinWords = 53248;  // 208 KiB of shared counters per block

__device__ __forceinline__ int wjob_of(const WJob *jobs, int n_jobs, uint64_t gv) {
    int lo = 0, hi = n_jobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].vbase <= gv) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ uint64_t *wrow(uint64_t *rows, const WJob &j) { return rows + (size_t)j.out_row * kRowWords; }

// the count of v2 (0 if the table does not hold it; the probe visits each slot at most once)
__device__ __forceinline__ uint32_t hash_count(const uint32_t *keys, const uint32_t *cnts, uint32_t mask,
                                               uint32_t v2) {
    uint32_t h = (v2 * 0x9E3779B1u) & mask;
    for (uint32_t p = 0; p <= mask; ++p, h = (h + 1) & mask) {
        const uint32_t k = keys[h];
        if (k == v2) return cnts[h];
        if (k == kEmptyKey) break;
    }
    return 0;
}

// add v2 to an open-addressing (key, count) table; returns the count before the increment
__device__ __forceinline__ uint32_t hash_increment(uint32_t *keys, uint32_t *cnts, uint32_t mask, uint32_t v2) {
    uint32_t h = (v2 * 0x9E3779B1u) & mask;
    while (true) {
        const uint32_t k = keys[h];
        if (k == v2) return atomicAdd(&cnts[h], 1u);
        if (k == kEmptyKey) {
            const uint32_t prev = atomicCAS(&keys[h], kEmptyKey, v2);
            if (prev == kEmptyKey || prev == v2) return atomicAdd(&cnts[h], 1u);
        }
        h = (h + 1) & mask;
    }
}

// pass 1, one warp per start vertex: its wedge count (level-2 extensions) and its tier list
__global__ void wedge_classify_kernel(const WJob *__restrict__ jobs, int n_jobs, uint64_t n_total,
                                      unsigned int *cnt, uint32_t *lists, uint64_t list_cap, uint64_t *rows) {
    const unsigned lane = lane_id();
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t gv = warp; gv < n_total; gv += nwarps) {
        const int j = wjob_of(jobs, n_jobs, gv);
        const WJob &J = jobs[j];
        const uint32_t v0 = (uint32_t)(gv - J.vbase);
        if (!J.start.keep(v0)) continue;
        const uint64_t b = J.off[v0], e = J.off[v0 + 1];
        const uint32_t start = upper_bound_u32(J.adj + b, 0, (uint32_t)(e - b), v0);
        // with a start-vertex restriction the level-1 extensions (v1 > v0) are counted here
        if (J.start.labels && lane == 0 && e - b > start)
            atomicAdd((unsigned long long *)&wrow(rows, J)[KHZ_MAX_COUNTS], (unsigned long long)(e - b - start));
        uint64_t wedges = 0;
        for (uint64_t i = b + start + lane; i < e; i += 32) {
            const uint32_t w = J.adj[i];
            const uint64_t wb = J.off[w], we = J.off[w + 1];
            wedges += (we - wb) - upper_bound_u32(J.adj + wb, 0, (uint32_t)(we - wb), v0);
        }
        for (int o = 16; o > 0; o >>= 1) wedges += __shfl_down_sync(kFull, wedges, o);
        if (lane == 0 && wedges > 0) {
            if (!J.ext_off)  // the wedges walked are the schedule's level-2 embeddings
                atomicAdd((unsigned long long *)&wrow(rows, J)[KHZ_MAX_COUNTS], (unsigned long long)wedges);
            const int t = wedges <= (uint64_t)kWarpWedges ? 0 : (wedges <= (uint64_t)kBlockWedges ? 1 : 2);
            const unsigned int pos = atomicAdd(&cnt[t], 1u);
            lists[(size_t)t * list_cap + pos] = (uint32_t)gv;
        }
    }
}

// Level-2 NumExtensions of the 4-cycle schedule on the stored graph, for jobs that count on its
// degree-descending renumbering: the level-1 embeddings (v0, v1) are the v0 < v1 in N(v1), and each
// extends to every v2 in N(v1) above v0; with p = #{v0 in N(v1) : v0 < v1} that is
// sum_{k < p} (deg(v1) - 1 - k) = p (deg(v1) - 1) - p (p - 1) / 2 per v1.  One thread per v1,
// one atomic per distinct job per warp.
__global__ void wedge_ext_formula_kernel(const WJob *__restrict__ jobs, int n_jobs, uint64_t n_total, uint64_t *rows) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;  // a multiple of 32: whole warps iterate together
    for (uint64_t gv = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; gv < ((n_total + 31) & ~31ull);
         gv += stride) {
        int j = -1;
        uint64_t val = 0;
        if (gv < n_total) {
            j = wjob_of(jobs, n_jobs, gv);
            const WJob &J = jobs[j];
            if (J.ext_off) {
                const uint32_t v = (uint32_t)(gv - J.vbase);
                const uint64_t b = J.ext_off[v];
                const uint64_t d = J.ext_off[v + 1] - b;
                const uint64_t p = lower_bound_u32(J.ext_adj + b, 0, (uint32_t)d, v);
                val = p * (d - 1) - p * (p - (p > 0 ? 1 : 0)) / 2;
            } else {
                j = -1;
            }
        }
        const unsigned peers = __match_any_sync(kFull, j);
        uint64_t sum = 0;
        for (int l = 0; l < 32; ++l) {
            const uint64_t x = __shfl_sync(kFull, val, l);
            if ((peers >> l) & 1u) sum += x;
        }
        if (j >= 0 && (int)lane_id() == __ffs(peers) - 1 && sum)
            atomicAdd((unsigned long long *)&wrow(rows, jobs[j])[KHZ_MAX_COUNTS], (unsigned long long)sum);
    }
}

// The part of the sorted list L[0, len) inside [lo, hi), widened to whole gaps between 32 evenly
// spaced splitters (lane l holds splitter l, read in one warp-wide load) instead of two binary
// searches of dependent loads; entries outside [lo, hi) in the range are filtered by the caller.
struct Span {
    uint32_t begin, end;
};
__device__ __forceinline__ uint32_t load_splitter(const uint32_t *__restrict__ L, uint32_t len) {
    const uint64_t sidx = lane_id() * (((uint64_t)len + 31) >> 5);
    return sidx < len ? __ldg(L + sidx) : kEmptyKey;
}
__device__ __forceinline__ Span splitter_span(uint32_t sp, uint32_t len, uint32_t lo, uint32_t hi) {
    const uint64_t step = ((uint64_t)len + 31) >> 5;
    const uint64_t k_lo = __popc(__ballot_sync(kFull, sp < lo));
    const uint64_t k_hi = __popc(__ballot_sync(kFull, sp < hi));
    Span r;
    r.begin = (uint32_t)(k_lo == 0 ? 0 : (k_lo - 1) * step + 1);
    r.end = (uint32_t)min((uint64_t)len, k_hi * step);
    return r;
}

// Walk the wedges (v0, w, v2) of one start vertex with w > v0 and v2 in [lo, hi) (lo > v0), with
// the calling threads: warp `wid` of `nw` takes every nw-th w, its lanes take consecutive v2.  The
// list bounds of a warp's next 32 w are read together (one per lane), and the next list's
// splitters are loaded before the current list is walked, so the round trips of one w overlap the
// previous one's work.  f(v2, iw, k) is called once per wedge, iw and k being the positions in adj
// of the entries (v0, w) and (w, v2).
template <typename F>
__device__ __forceinline__ void walk_wedges(const WJob &J, uint32_t v0, int wid, int nw, uint32_t lo, uint32_t hi,
                                            F f) {
    const unsigned lane = lane_id();
    const uint64_t b = J.off[v0], e = J.off[v0 + 1];
    const uint32_t start = upper_bound_u32(J.adj + b, 0, (uint32_t)(e - b), v0);
    for (uint64_t i0 = b + start + wid; i0 < e; i0 += 32ull * nw) {
        const uint64_t mine = i0 + (uint64_t)lane * nw;
        uint64_t my_b = 0;
        uint32_t my_len = 0;
        if (mine < e) {
            const uint32_t w = J.adj[mine];
            my_b = J.off[w];
            my_len = (uint32_t)(J.off[w + 1] - my_b);
        }
        const int nr = (int)min((uint64_t)32, (e - i0 + nw - 1) / nw);
        uint32_t sp_next = load_splitter(J.adj + __shfl_sync(kFull, my_b, 0), __shfl_sync(kFull, my_len, 0));
        for (int r = 0; r < nr; ++r) {
            const uint64_t wb = __shfl_sync(kFull, my_b, r);
            const uint32_t len = __shfl_sync(kFull, my_len, r);
            const uint32_t sp = sp_next;
            if (r + 1 < nr)
                sp_next = load_splitter(J.adj + __shfl_sync(kFull, my_b, r + 1), __shfl_sync(kFull, my_len, r + 1));
            const Span s2 = splitter_span(sp, len, lo, hi);
            const uint64_t iw = i0 + (uint64_t)r * nw;
            for (uint64_t k = wb + s2.begin + lane; k < wb + s2.end; k += 32) {
                const uint32_t v2 = __ldg(J.adj + k);
                if (v2 - lo < hi - lo) f(v2, iw, k);
            }
        }
    }
}

__device__ __forceinline__ void flush_count(uint64_t &acc, uint64_t *row) {
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(kFull, acc, o);
    if (lane_id() == 0 && acc) atomicAdd((unsigned long long *)&row[0], (unsigned long long)acc);
    acc = 0;
}

// the endpoint count and the weighted sum of a job, into its rows
__device__ __forceinline__ void flush_job(uint64_t &acc, uint64_t &acc_t, uint64_t *rows, const WJob &J) {
    flush_count(acc, wrow(rows, J));
    if (J.tri) flush_count(acc_t, rows + (size_t)J.tri_row * kRowWords);
}

// one wedge's term of the triangle-weighted sum, c being its endpoint's count
__device__ __forceinline__ uint64_t tri_term(const WJob &J, uint32_t c, uint64_t iw, uint64_t k) {
    return c > 1 ? (uint64_t)(c - 1) * ((uint64_t)__ldg(J.tri + iw) + __ldg(J.tri + k)) : 0;
}

__global__ void __launch_bounds__(256) wedge_warp_kernel(const WJob *__restrict__ jobs, int n_jobs,
                                                         const uint32_t *__restrict__ list,
                                                         const unsigned int *__restrict__ list_len,
                                                         unsigned long long *queue, uint64_t *rows) {
    __shared__ uint32_t s_keys[8][kWarpSlots];
    __shared__ uint32_t s_cnts[8][kWarpSlots];
    const unsigned lane = lane_id();
    const int wib = threadIdx.x >> 5;
    uint32_t *keys = s_keys[wib], *cnts = s_cnts[wib];
    const unsigned int n_list = *list_len;
    uint64_t acc = 0, acc_t = 0;
    int cur = -1;
    while (true) {
        unsigned long long t = 0;
        if (lane == 0) t = atomicAdd(queue, 1ull);
        t = __shfl_sync(kFull, t, 0);
        if (t >= n_list) break;
        const uint64_t gv = list[t];
        const int j = wjob_of(jobs, n_jobs, gv);
        if (j != cur) {
            if (cur >= 0) flush_job(acc, acc_t, rows, jobs[cur]);
            cur = j;
        }
        __syncwarp();
        for (int k = lane; k < kWarpSlots; k += 32) {
            keys[k] = kEmptyKey;
            cnts[k] = 0;
        }
        __syncwarp();
        const WJob &J = jobs[j];
        const uint32_t v0 = (uint32_t)(gv - J.vbase);
        walk_wedges(J, v0, 0, 1, v0 + 1, J.n,
                    [&](uint32_t v2, uint64_t, uint64_t) { acc += hash_increment(keys, cnts, kWarpSlots - 1, v2); });
        if (J.tri) {
            __syncwarp();
            walk_wedges(J, v0, 0, 1, v0 + 1, J.n, [&](uint32_t v2, uint64_t iw, uint64_t k) {
                acc_t += tri_term(J, hash_count(keys, cnts, kWarpSlots - 1, v2), iw, k);
            });
        }
    }
    if (cur >= 0) flush_job(acc, acc_t, rows, jobs[cur]);
}

__global__ void __launch_bounds__(kBlockThreads) wedge_block_kernel(const WJob *__restrict__ jobs, int n_jobs,
                                                                    const uint32_t *__restrict__ list,
                                                                    const unsigned int *__restrict__ list_len,
                                                                    unsigned long long *queue, uint64_t *rows) {
    extern __shared__ __align__(16) uint32_t smem[];
    __shared__ uint64_t s_gv;
    uint32_t *keys = smem, *cnts = smem + kBlockSlots;
    const int wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const unsigned int n_list = *list_len;
    uint64_t acc = 0, acc_t = 0;
    int cur = -1;
    while (true) {
        if (threadIdx.x == 0) {
            const unsigned long long t = atomicAdd(queue, 1ull);
            s_gv = t < n_list ? list[t] : ~0ull;
        }
        __syncthreads();
        const uint64_t gv = s_gv;
        if (gv == ~0ull) break;
        const int j = wjob_of(jobs, n_jobs, gv);
        if (j != cur) {
            if (cur >= 0) flush_job(acc, acc_t, rows, jobs[cur]);
            cur = j;
        }
        for (int k = threadIdx.x; k < kBlockSlots; k += blockDim.x) {
            keys[k] = kEmptyKey;
            cnts[k] = 0;
        }
        __syncthreads();
        const WJob &J = jobs[j];
        const uint32_t v0 = (uint32_t)(gv - J.vbase);
        walk_wedges(J, v0, wid, nw, v0 + 1, J.n,
                    [&](uint32_t v2, uint64_t, uint64_t) { acc += hash_increment(keys, cnts, kBlockSlots - 1, v2); });
        __syncthreads();
        if (J.tri) {
            walk_wedges(J, v0, wid, nw, v0 + 1, J.n, [&](uint32_t v2, uint64_t iw, uint64_t k) {
                acc_t += tri_term(J, hash_count(keys, cnts, kBlockSlots - 1, v2), iw, k);
            });
            __syncthreads();
        }
    }
    if (cur >= 0) flush_job(acc, acc_t, rows, jobs[cur]);
}

// One block per heavy start vertex: the endpoints v2 in (v0, n) are counted one window of `span`
// ids at a time in shared memory (16-bit counters packed two to a word unless WIDE: a count is at
// most the graph's largest degree).
template <bool WIDE>
__global__ void __launch_bounds__(kWinThreads, 1) wedge_window_kernel(const WJob *__restrict__ jobs, int n_jobs,
                                                                      const uint32_t *__restrict__ list,
                                                                      const unsigned int *__restrict__ list_len,
                                                                      unsigned long long *queue, uint64_t *rows) {
    extern __shared__ __align__(16) uint32_t win[];
    __shared__ uint64_t s_gv;
    constexpr uint64_t span = WIDE ? kWinWords : 2ull * kWinWords;
    const unsigned lane = lane_id();
    const int wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const unsigned int n_list = *list_len;
    uint64_t acc = 0, acc_t = 0;
    int cur = -1;
    while (true) {
        if (threadIdx.x == 0) {
            const unsigned long long t = atomicAdd(queue, 1ull);
            s_gv = t < n_list ? list[t] : ~0ull;
        }
        __syncthreads();
        const uint64_t gv = s_gv;
        if (gv == ~0ull) break;
        const int j = wjob_of(jobs, n_jobs, gv);
        if (j != cur) {
            if (cur >= 0) flush_job(acc, acc_t, rows, jobs[cur]);
            cur = j;
        }
        const WJob &J = jobs[j];
        const uint32_t v0 = (uint32_t)(gv - J.vbase);
        for (uint64_t base = (uint64_t)v0 + 1; base < J.n; base += span) {
            for (uint32_t t = threadIdx.x; t < kWinWords; t += blockDim.x) win[t] = 0;
            __syncthreads();
            const uint32_t top = (uint32_t)min((uint64_t)J.n, base + span);
            walk_wedges(J, v0, wid, nw, (uint32_t)base, top, [&](uint32_t v2, uint64_t, uint64_t) {
                const uint32_t x = v2 - (uint32_t)base;
                if (WIDE) {
                    acc += atomicAdd(&win[x], 1u);
                } else {
                    const uint32_t sh = (x & 1u) << 4;
                    acc += (atomicAdd(&win[x >> 1], 1u << sh) >> sh) & 0xffffu;
                }
            });
            __syncthreads();
            if (J.tri) {
                walk_wedges(J, v0, wid, nw, (uint32_t)base, top, [&](uint32_t v2, uint64_t iw, uint64_t k) {
                    const uint32_t x = v2 - (uint32_t)base;
                    const uint32_t c = WIDE ? win[x] : (win[x >> 1] >> ((x & 1u) << 4)) & 0xffffu;
                    acc_t += tri_term(J, c, iw, k);
                });
                __syncthreads();
            }
        }
    }
    if (cur >= 0) flush_job(acc, acc_t, rows, jobs[cur]);
}

}  // namespace

size_t wedge_arena_bytes(int n_jobs, uint64_t n_total) {
    return Arena::round(sizeof(WJob) * (size_t)std::max(n_jobs, 1)) +
           Arena::round(sizeof(uint32_t) * 3 * std::max<uint64_t>(n_total, 1)) + Arena::round(sizeof(unsigned int) * 8) +
           Arena::round(sizeof(unsigned long long) * 4);
}

khz_status wedge_prepare(const std::vector<WJob> &jobs, Arena *arena, WedgeLaunch *wl, cudaStream_t s) {
    WedgeLaunch L;
    L.n_jobs = (int)jobs.size();
    L.n_total = jobs.empty() ? 0 : jobs.back().vbase + jobs.back().n;
    if (L.n_total >= (1ull << 32)) {
        set_error("a wedge launch serves at most 2^32 - 1 start vertices");
        return KHZ_ERR_ARG;
    }
    for (const auto &j : jobs) {
        L.wide = L.wide || j.max_deg >= 65535u;
        L.ext_formula = L.ext_formula || j.ext_off != nullptr;
    }
    WJob *d_jobs = arena->take<WJob>(jobs.size());
    L.lists = arena->take<uint32_t>(3 * std::max<uint64_t>(L.n_total, 1));
    L.cnt = arena->take<unsigned int>(8);
    L.queues = arena->take<unsigned long long>(4);
    if (!d_jobs || !L.lists || !L.cnt || !L.queues) {
        set_error("wedge launch arena too small");
        return KHZ_ERR_OOM;
    }
    L.list_cap = std::max<uint64_t>(L.n_total, 1);
    if (!jobs.empty())
        KHZ_CUDA(cudaMemcpyAsync(d_jobs, jobs.data(), sizeof(WJob) * jobs.size(), cudaMemcpyHostToDevice, s));
    KHZ_CUDA(cudaFuncSetAttribute(wedge_block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(2 * kBlockSlots * sizeof(uint32_t))));
    KHZ_CUDA(cudaFuncSetAttribute(wedge_window_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(kWinWords * sizeof(uint32_t))));
    KHZ_CUDA(cudaFuncSetAttribute(wedge_window_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(kWinWords * sizeof(uint32_t))));
    int dev = 0;
    KHZ_CUDA(cudaGetDevice(&dev));
    KHZ_CUDA(cudaDeviceGetAttribute(&L.sms, cudaDevAttrMultiProcessorCount, dev));
    L.d_jobs = d_jobs;
    *wl = L;
    return KHZ_OK;
}

khz_status wedge_enqueue(const WedgeLaunch &L, uint64_t *d_rows, cudaStream_t s, LaunchStats *ls) {
    if (L.n_jobs == 0 || L.n_total == 0) return KHZ_OK;
    KHZ_CUDA(cudaMemsetAsync(L.cnt, 0, sizeof(unsigned int) * 8, s));
    KHZ_CUDA(cudaMemsetAsync(L.queues, 0, sizeof(unsigned long long) * 4, s));
    const int cgrid = (int)std::max<uint64_t>(1, std::min<uint64_t>((L.n_total + 7) / 8, (uint64_t)L.sms * 16));
    wedge_classify_kernel<<<cgrid, 256, 0, s>>>(L.d_jobs, L.n_jobs, L.n_total, L.cnt, L.lists, L.list_cap, d_rows);
    if (L.ext_formula) {
        const int fgrid = (int)std::max<uint64_t>(1, std::min<uint64_t>((L.n_total + 255) / 256, (uint64_t)L.sms * 8));
        wedge_ext_formula_kernel<<<fgrid, 256, 0, s>>>(L.d_jobs, L.n_jobs, L.n_total, d_rows);
        if (ls) ls->launches += 1;
    }
    wedge_warp_kernel<<<L.sms * 8, 256, 0, s>>>(L.d_jobs, L.n_jobs, L.lists, L.cnt + 0, &L.queues[0], d_rows);
    wedge_block_kernel<<<L.sms * 2, kBlockThreads, 2 * kBlockSlots * sizeof(uint32_t), s>>>(
        L.d_jobs, L.n_jobs, L.lists + L.list_cap, L.cnt + 1, &L.queues[1], d_rows);
    (L.wide ? wedge_window_kernel<true> : wedge_window_kernel<false>)<<<L.sms, kWinThreads,
                                                                      kWinWords * sizeof(uint32_t), s>>>(
        L.d_jobs, L.n_jobs, L.lists + 2 * L.list_cap, L.cnt + 2, &L.queues[2], d_rows);
    KHZ_CUDA(cudaGetLastError());
    if (ls) ls->launches += 4;
    return KHZ_OK;
}

}  // namespace khz
