// Bitmap clique engine for the clique apps on the degree-oriented DAG.
//
// The reference schedule (kautomine/four_clique.cc:58-153, five_clique.cc:58-186 and
// the kgraphpi equivalents) intersects the prefix N(v0) n N(v1) n ... with one more
// neighbour list per level.  On the oriented DAG every prefix is a subset of
// C = N+(v0), so this engine intersects each list only once per start vertex: it
// builds the subgraph induced on C as a bit matrix (row i = positions j of C[j] in
// N+(C[i]); only j > i can be set), and every deeper intersection becomes an AND of
// rows plus a popcount in shared memory:
//   triangles through v0  = sum_i popc(row_i)
//   4-cliques             = sum_i sum_{j in row_i} popc(row_i & row_j)
//   5-cliques             = sum_i sum_{j in row_i} sum_{l in row_i & row_j} popc(row_i & row_j & row_l)
// The NumExtensions of the reference schedule (engine.cc:924) follow from the same
// popcounts: n + m + #triangles (+ #4-cliques for k = 5).  The instrumented variant
// also sums the schedule's algorithmic bytes 4 * (|A| + |B| + |A n B|) per set op.
//
// Tiers by out-degree d of v0: one warp per v0 for d <= 64 (rows of 2 words), one
// block per v0 for 64 < d <= kBlockMax (rows in up to ~195 KB of shared memory, block
// size chosen per tier); larger d are left to the DFS engine.  Blocks and warps take
// start vertices from atomic queues, heaviest first.
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include "khz_internal.cuh"
#include "setops.cuh"

namespace khz {

namespace {

constexpr int kWarpMax = 64;          // warp tier: d <= 64 -> 2 words per row
constexpr int kMidMax = 256;          // mid block tier
constexpr int kBlockMax = 1248;       // large block tier: 1248 rows x 39 words = 190 KiB

// position of the n-th (0-based) set bit of x; x must have more than n set bits
__device__ __forceinline__ int nth_set_bit(uint32_t x, int n) {
    int pos = 0;
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        const uint32_t low = x & ((1u << s) - 1u);
        const int c = __popc(low);
        if (n >= c) {
            n -= c;
            x >>= s;
            pos += s;
        } else {
            x = low;
        }
    }
    return pos;
}

struct Acc {
    uint64_t cnt, t3, t4, bytes, ext1;  // ext1: level-1 extensions (v0, v1) of the processed v0s
};

__device__ __forceinline__ uint32_t odeg(const uint64_t *off, uint32_t v) {
    return (uint32_t)(__ldg(off + v + 1) - __ldg(off + v));
}

// Build rows [row_begin, d - 1) with stride row_step; the calling warp owns those rows.
__device__ void build_rows(uint32_t *rows, int W, int d, const uint32_t *sC, const uint64_t *__restrict__ off,
                           const uint32_t *__restrict__ adj, int row_begin, int row_step) {
    const unsigned lane = lane_id();
    const uint32_t hi_val = sC[d - 1];
    for (int i = row_begin; i < d - 1; i += row_step) {
        const uint32_t v = sC[i];
        const uint64_t b0 = __ldg(off + v);
        const uint32_t len = (uint32_t)(__ldg(off + v + 1) - b0);
        const uint32_t *L = adj + b0;
        uint32_t start = lower_bound_u32(L, 0, len, sC[i + 1]);
        uint32_t *row = rows + (size_t)i * W;
        uint32_t lo = (uint32_t)i + 1;
        for (uint32_t b = start; b < len; b += 32) {
            const uint32_t idx = b + lane;
            const uint32_t x = idx < len ? __ldg(L + idx) : 0xffffffffu;
            uint32_t j = (uint32_t)d;
            if (x <= hi_val) {
                j = lower_bound_plain(sC, lo, (uint32_t)d, x);
                if (j < (uint32_t)d && sC[j] == x) atomicOr(row + (j >> 5), 1u << (j & 31));
            }
            const uint32_t xl = __shfl_sync(kFull, x, 31);
            const uint32_t jl = __shfl_sync(kFull, j, 31);
            if (xl >= hi_val) break;
            lo = jl < (uint32_t)d ? jl : lo;
        }
    }
}

template <int K, bool STATS>
__device__ __forceinline__ void process_item(const uint32_t *rows, int W, int i, int j, const uint32_t *sC,
                                             const uint64_t *off, Acc &a) {
    const uint32_t *ri = rows + (size_t)i * W;
    const uint32_t *rj = rows + (size_t)j * W;
    const int w0 = j >> 5;
    uint32_t s = 0;
    for (int w = w0; w < W; ++w) s += __popc(ri[w] & rj[w]);
    if (STATS) {
        uint32_t pi = 0;
        for (int w = 0; w < W; ++w) pi += __popc(ri[w]);
        a.bytes += 4ull * ((uint64_t)pi + odeg(off, sC[j]) + s);
    }
    if (K == 4) {
        a.cnt += s;
        return;
    }
    a.t4 += s;
    for (int w1 = w0; w1 < W; ++w1) {
        uint32_t m = ri[w1] & rj[w1];
        while (m) {
            const int l = (w1 << 5) + __ffs(m) - 1;
            m &= m - 1;
            const uint32_t *rl = rows + (size_t)l * W;
            uint32_t t = 0;
            for (int w = l >> 5; w < W; ++w) t += __popc(ri[w] & rj[w] & rl[w]);
            a.cnt += t;
            if (STATS) a.bytes += 4ull * ((uint64_t)s + odeg(off, sC[l]) + t);
        }
    }
}

// Count over rows [row_begin, d) with stride row_step; (i, j) items are dealt to the
// lanes of the calling warp in batches of 32.
template <int K, bool STATS>
__device__ void count_rows(const uint32_t *rows, int W, int d, const uint32_t *sC, const uint64_t *off,
                           int row_begin, int row_step, Acc &a) {
    const unsigned lane = lane_id();
    int pc = 0;           // pending items held by lanes [0, pc)
    int my_i = 0, my_j = 0;
    for (int i = row_begin; i < d; i += row_step) {
        const uint32_t *ri = rows + (size_t)i * W;
        uint32_t pop = 0;
        for (int w = (i + 1) >> 5; w < W; ++w) pop += __popc(ri[w]);
        if (lane == 0) a.t3 += pop;
        if (STATS && lane == 0) a.bytes += 4ull * ((uint64_t)d + odeg(off, sC[i]) + pop);
        if (K == 3) {
            if (lane == 0) a.cnt += pop;
            continue;
        }
        for (int ww = (i + 1) >> 5; ww < W; ++ww) {
            const uint32_t bits = ri[ww];
            const int c = __popc(bits);
            if (c == 0) continue;
            const int q = (int)lane;
            if (q >= pc && q < pc + c) {
                my_i = i;
                my_j = (ww << 5) + nth_set_bit(bits, q - pc);
            }
            if (pc + c >= 32) {
                process_item<K, STATS>(rows, W, my_i, my_j, sC, off, a);
                const int rem = pc + c - 32;
                if (q < rem) {
                    my_i = i;
                    my_j = (ww << 5) + nth_set_bit(bits, (32 - pc) + q);
                }
                pc = rem;
            } else {
                pc += c;
            }
        }
    }
    if (K > 3 && (int)lane < pc) process_item<K, STATS>(rows, W, my_i, my_j, sC, off, a);
}

__device__ __forceinline__ void flush_acc(Acc &a, int K, uint64_t *out, uint64_t *phase_bytes) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a.cnt += __shfl_down_sync(kFull, a.cnt, o);
        a.t3 += __shfl_down_sync(kFull, a.t3, o);
        a.t4 += __shfl_down_sync(kFull, a.t4, o);
        a.bytes += __shfl_down_sync(kFull, a.bytes, o);
        a.ext1 += __shfl_down_sync(kFull, a.ext1, o);
    }
    if (lane_id() == 0) {
        const uint64_t ext = a.ext1 + (K >= 4 ? a.t3 : 0) + (K >= 5 ? a.t4 : 0);
        if (a.cnt) atomicAdd((unsigned long long *)&out[0], (unsigned long long)a.cnt);
        if (ext) atomicAdd((unsigned long long *)&out[KHZ_MAX_COUNTS], (unsigned long long)ext);
        if (a.bytes) atomicAdd((unsigned long long *)&out[KHZ_MAX_COUNTS + 1], (unsigned long long)a.bytes);
        if (a.bytes && phase_bytes) atomicAdd((unsigned long long *)phase_bytes, (unsigned long long)a.bytes);
    }
}

// Warp tier: one warp per start vertex with dmin <= d <= 64; vertices taken in descending id
// order (heaviest first on the oriented DAG, whose ids are degree ranks).
template <int K, bool STATS>
__global__ void __launch_bounds__(256) clique_warp_kernel(const uint64_t *__restrict__ off,
                                                          const uint32_t *__restrict__ adj, uint32_t n,
                                                          uint32_t dmin, unsigned long long *queue,
                                                          uint64_t *out, uint64_t *phase_bytes) {
    constexpr int W = kWarpMax / 32;
    __shared__ uint32_t s_c[8][kWarpMax];
    __shared__ uint32_t s_rows[8][kWarpMax * W];
    const unsigned lane = lane_id();
    const int wib = threadIdx.x >> 5;
    uint32_t *sC = s_c[wib];
    uint32_t *rows = s_rows[wib];
    Acc a = {0, 0, 0, 0, 0};
    constexpr uint32_t kChunk = 32;
    while (true) {
        unsigned long long c0 = 0;
        if (lane == 0) c0 = atomicAdd(queue, (unsigned long long)kChunk);
        c0 = __shfl_sync(kFull, c0, 0);
        if (c0 >= n) break;
        const uint32_t c1 = (uint32_t)min((unsigned long long)n, c0 + kChunk);
        // vertex candidates of this chunk, one per lane
        const uint32_t myc = (uint32_t)c0 + lane;
        uint32_t myv = 0, myd = 0;
        if (myc < c1) {
            myv = n - 1 - myc;
            myd = odeg(off, myv);
        }
        if (myc < c1 && myd <= (uint32_t)kWarpMax) a.ext1 += myd;
        unsigned todo = __ballot_sync(kFull, myc < c1 && myd >= dmin && myd <= (uint32_t)kWarpMax);
        while (todo) {
            const int src = __ffs(todo) - 1;
            todo &= todo - 1;
            const uint32_t v0 = __shfl_sync(kFull, myv, src);
            const int d = (int)__shfl_sync(kFull, myd, src);
            const uint64_t b0 = __ldg(off + v0);
            __syncwarp();
            for (int t = lane; t < kWarpMax; t += 32) sC[t] = t < d ? __ldg(adj + b0 + t) : 0xffffffffu;
            for (int t = lane; t < kWarpMax * W; t += 32) rows[t] = 0;
            __syncwarp();
            if (d >= 2) build_rows(rows, W, d, sC, off, adj, 0, 1);
            __syncwarp();
            count_rows<K, STATS>(rows, W, d, sC, off, 0, 1, a);
        }
    }
    flush_acc(a, K, out, phase_bytes);
}

// Block tier: one block per start vertex from a degree-descending list.
template <int K, bool STATS>
__global__ void clique_block_kernel(const uint64_t *__restrict__ off, const uint32_t *__restrict__ adj,
                                    const uint32_t *__restrict__ list, uint32_t list_n, int dcap,
                                    unsigned long long *queue, uint64_t *out, uint64_t *phase_bytes) {
    extern __shared__ uint32_t smem[];
    __shared__ uint32_t s_v0;
    uint32_t *sC = smem;
    uint32_t *rows = smem + ((dcap + 31) & ~31);
    const int warps = blockDim.x >> 5;
    const int wib = threadIdx.x >> 5;
    Acc a = {0, 0, 0, 0, 0};
    while (true) {
        if (threadIdx.x == 0) {
            const unsigned long long t = atomicAdd(queue, 1ull);
            s_v0 = t < list_n ? list[t] : 0xffffffffu;
        }
        __syncthreads();
        const uint32_t v0 = s_v0;
        if (v0 == 0xffffffffu) break;
        const int d = (int)odeg(off, v0);
        const int W = (d + 31) >> 5;
        if (threadIdx.x == 0) a.ext1 += (uint64_t)d;
        const uint64_t b0 = __ldg(off + v0);
        for (int t = threadIdx.x; t < d; t += blockDim.x) sC[t] = __ldg(adj + b0 + t);
        for (int t = threadIdx.x; t < d * W; t += blockDim.x) rows[t] = 0;
        __syncthreads();
        build_rows(rows, W, d, sC, off, adj, wib, warps);
        __syncthreads();
        count_rows<K, STATS>(rows, W, d, sC, off, wib, warps, a);
        __syncthreads();
    }
    flush_acc(a, K, out, phase_bytes);
}

__global__ void classify_kernel(const uint64_t *__restrict__ off, uint32_t n, uint32_t *keys, uint32_t *vals,
                                unsigned int *counts) {
    // counts[0]: mid tier (64, 256], counts[1]: large tier (256, kBlockMax], counts[2]: overflow
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const uint32_t d = odeg(off, v);
        int t = -1;
        if (d > kWarpMax && d <= kMidMax) t = 0;
        else if (d > kMidMax && d <= kBlockMax) t = 1;
        else if (d > kBlockMax) t = 2;
        if (t >= 0) {
            const unsigned int pos = atomicAdd(&counts[t], 1u);
            keys[(size_t)t * n + pos] = d;
            vals[(size_t)t * n + pos] = v;
        }
    }
}

template <int K, bool STATS>
khz_status launch_all(const Graph &g, uint64_t *d_out, Workspace *ws, cudaStream_t s, LaunchStats *ls,
                      uint32_t *n_overflow) {
    int dev = 0, sms = 0;
    KHZ_CUDA(cudaGetDevice(&dev));
    KHZ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const uint32_t n = g.n;
    // temp layout: keys[3n], vals[3n], sorted keys/vals [n], counts, cub temp
    size_t cub_bytes = 0;
    cub::DeviceRadixSort::SortPairsDescending(nullptr, cub_bytes, (uint32_t *)nullptr, (uint32_t *)nullptr,
                                              (uint32_t *)nullptr, (uint32_t *)nullptr, (int)std::max(n, 1u));
    const size_t lists = (size_t)3 * std::max(n, 1u) * sizeof(uint32_t);
    const size_t sorted = (size_t)std::max(n, 1u) * sizeof(uint32_t);
    const size_t need = 2 * lists + 2 * sorted + 256 + cub_bytes + 256;
    if (ws->tmp_bytes < need) {
        if (ws->tmp) cudaFree(ws->tmp);
        ws->tmp = nullptr;
        ws->tmp_bytes = 0;
        KHZ_CUDA(cudaMalloc(&ws->tmp, need));
        ws->tmp_bytes = need;
    }
    char *p = (char *)ws->tmp;
    uint32_t *keys = (uint32_t *)p; p += lists;
    uint32_t *vals = (uint32_t *)p; p += lists;
    uint32_t *skeys = (uint32_t *)p; p += sorted;
    uint32_t *svals = (uint32_t *)p; p += sorted;
    unsigned int *tier_counts = (unsigned int *)p; p += 256;
    void *cub_tmp = p;
    unsigned long long *queues = (unsigned long long *)ws->counters;  // [0] warp, [1] mid, [2] large
    KHZ_CUDA(cudaMemsetAsync(tier_counts, 0, 16, s));
    KHZ_CUDA(cudaMemsetAsync(queues, 0, 4 * sizeof(unsigned long long), s));
    classify_kernel<<<sms * 4, 256, 0, s>>>(g.off, n, keys, vals, tier_counts);
    KHZ_CUDA(cudaGetLastError());
    unsigned int h_counts[3];
    KHZ_CUDA(cudaMemcpyAsync(h_counts, tier_counts, sizeof(h_counts), cudaMemcpyDeviceToHost, s));
    KHZ_CUDA(cudaStreamSynchronize(s));
    if (ls) ls->launches += 1;
    auto pb = [&](int phase) -> uint64_t * { return ls && ls->d_phase_bytes ? ls->d_phase_bytes + phase : nullptr; };
    auto mark = [&](int phase, bool begin) {
        if (!ls || !ls->ev_begin) return;
        cudaEventRecord(begin ? ls->ev_begin[phase] : ls->ev_end[phase], s);
        if (!begin) {
            ls->used[phase] = true;
            ls->phase_launches[phase] += 1;
        }
    };
    // warp tier
    mark(0, true);
    clique_warp_kernel<K, STATS><<<sms * 8, 256, 0, s>>>(g.off, g.adj, n, STATS ? 1u : 2u, &queues[0], d_out,
                                                          pb(0));
    KHZ_CUDA(cudaGetLastError());
    mark(0, false);
    if (ls) ls->launches += 1;
    // block tiers, each list sorted by degree descending
    const int tier_dcap[2] = {kMidMax, kBlockMax};
    const int tier_threads[2] = {128, 512};
    for (int t = 0; t < 2; ++t) {
        const unsigned int cnt = h_counts[t];
        if (cnt == 0) continue;
        size_t cb = cub_bytes;
        KHZ_CUDA(cub::DeviceRadixSort::SortPairsDescending(cub_tmp, cb, keys + (size_t)t * n, skeys,
                                                           vals + (size_t)t * n, svals, (int)cnt, 0, 32, s));
        const int dcap = tier_dcap[t];
        const size_t smem = (size_t)((dcap + 31) & ~31) * 4 + (size_t)dcap * ((dcap + 31) / 32) * 4;
        auto kern = clique_block_kernel<K, STATS>;
        KHZ_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 0;
        KHZ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, tier_threads[t], smem));
        if (per_sm < 1) per_sm = 1;
        const int blocks = (int)std::min<size_t>((size_t)sms * per_sm, cnt);
        mark(1 + t, true);
        kern<<<blocks, tier_threads[t], smem, s>>>(g.off, g.adj, svals, cnt, dcap, &queues[1 + t], d_out,
                                                   pb(1 + t));
        KHZ_CUDA(cudaGetLastError());
        mark(1 + t, false);
        if (ls) ls->launches += 2;
    }
    *n_overflow = h_counts[2];
    return KHZ_OK;
}

}  // namespace

uint32_t bitmap_block_max_degree() { return kBlockMax; }

khz_status bitmap_clique_run(const Graph &g, int k, bool stats, int warp_max, int block_warps, uint64_t *d_out,
                             Workspace *ws, cudaStream_t s, LaunchStats *ls, uint32_t *n_overflow) {
    (void)warp_max;
    (void)block_warps;
    if (!g.oriented) {
        set_error("bitmap clique engine needs an oriented graph");
        return KHZ_ERR_ARG;
    }
    if (g.n == 0) {
        *n_overflow = 0;
        return KHZ_OK;
    }
    switch (k * 2 + (stats ? 1 : 0)) {
        case 6: return launch_all<3, false>(g, d_out, ws, s, ls, n_overflow);
        case 7: return launch_all<3, true>(g, d_out, ws, s, ls, n_overflow);
        case 8: return launch_all<4, false>(g, d_out, ws, s, ls, n_overflow);
        case 9: return launch_all<4, true>(g, d_out, ws, s, ls, n_overflow);
        case 10: return launch_all<5, false>(g, d_out, ws, s, ls, n_overflow);
        case 11: return launch_all<5, true>(g, d_out, ws, s, ls, n_overflow);
        default:
            set_error("bitmap clique engine supports k = 3, 4, 5 (got %d)", k);
            return KHZ_ERR_ARG;
    }
}

}  // namespace khz
