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
constexpr int kBlockMax = 1216;       // large block tier: 1216 rows x 38 words = 180 KiB (+ hash 24 KiB)

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

constexpr uint32_t kEmpty = 0xffffffffu;

// The subgraph induced on C = N+(v0), in shared memory:
//   c[d]            the candidates (sorted vertex ids)
//   hkey/hidx[T]    open-addressing hash of c: vertex id -> position (T = 2^logt >= 2d)
//   rows[d * W]     bit j of row i set iff c[j] in N+(c[i])   (only j > i)
//   rlo/rhi[d]      first / one-past-last non-zero word of each row
struct Local {
    uint32_t *c;
    uint32_t *hkey;
    uint16_t *hidx;
    uint32_t *rows;
    uint16_t *rlo, *rhi;
    int d, W, logt;
    __device__ __forceinline__ uint32_t slot(uint32_t x) const { return (x * 0x9E3779B1u) >> (32 - logt); }
    __device__ __forceinline__ int find(uint32_t x) const {
        const uint32_t mask = (1u << logt) - 1u;
        uint32_t h = slot(x);
        while (true) {
            const uint32_t k = hkey[h];
            if (k == x) return hidx[h];
            if (k == kEmpty) return -1;
            h = (h + 1) & mask;
        }
    }
};

// insert c[t] for t in [tid, d) step nthr (the table was set to kEmpty before a barrier)
__device__ __forceinline__ void hash_insert(const Local &g, int tid, int nthr) {
    const uint32_t mask = (1u << g.logt) - 1u;
    for (int t = tid; t < g.d; t += nthr) {
        const uint32_t x = g.c[t];
        uint32_t h = g.slot(x);
        while (atomicCAS(&g.hkey[h], kEmpty, x) != kEmpty) h = (h + 1) & mask;
        g.hidx[h] = (uint16_t)t;
    }
}

// Build rows [row_begin, d - 1) with stride row_step; the calling warp owns those rows.
// Members of N+(c[i]) outside [c[i+1], c[d-1]] cannot be in C and are skipped.
__device__ void build_rows(const Local &g, const uint64_t *__restrict__ off, const uint32_t *__restrict__ adj,
                           int row_begin, int row_step) {
    const unsigned lane = lane_id();
    const int d = g.d;
    const uint32_t hi_val = g.c[d - 1];
    for (int i = row_begin; i < d - 1; i += row_step) {
        const uint32_t v = g.c[i];
        const uint64_t b0 = __ldg(off + v);
        const uint32_t len = (uint32_t)(__ldg(off + v + 1) - b0);
        const uint32_t *L = adj + b0;
        const uint32_t start = lower_bound_u32(L, 0, len, g.c[i + 1]);
        uint32_t *row = g.rows + (size_t)i * g.W;
        for (uint32_t b = start; b < len; b += 32) {
            const uint32_t idx = b + lane;
            const uint32_t x = idx < len ? __ldg(L + idx) : kEmpty;
            if (x <= hi_val) {
                const int j = g.find(x);
                if (j >= 0) atomicOr(row + (j >> 5), 1u << (j & 31));
            }
            if (__shfl_sync(kFull, x, 31) >= hi_val) break;
        }
    }
}

// first / one-past-last non-zero word of rows [tid, d) step nthr
__device__ __forceinline__ void row_extents(const Local &g, int tid, int nthr) {
    for (int i = tid; i < g.d; i += nthr) {
        const uint32_t *r = g.rows + (size_t)i * g.W;
        int lo = g.W, hi = 0;
        for (int w = (i + 1) >> 5; w < g.W; ++w) {
            if (r[w]) {
                lo = min(lo, w);
                hi = w + 1;
            }
        }
        g.rlo[i] = (uint16_t)(hi == 0 ? g.W : lo);
        g.rhi[i] = (uint16_t)hi;
    }
}

template <int K, bool STATS>
__device__ __forceinline__ void process_item(const Local &g, int i, int j, const uint64_t *off, Acc &a) {
    const uint32_t *ri = g.rows + (size_t)i * g.W;
    const uint32_t *rj = g.rows + (size_t)j * g.W;
    const int lo = max((int)g.rlo[i], (int)g.rlo[j]);
    const int hi = min((int)g.rhi[i], (int)g.rhi[j]);
    uint32_t s = 0;
    for (int w = lo; w < hi; ++w) s += __popc(ri[w] & rj[w]);
    if (STATS) {
        uint32_t pi = 0;
        for (int w = g.rlo[i]; w < g.rhi[i]; ++w) pi += __popc(ri[w]);
        a.bytes += 4ull * ((uint64_t)pi + odeg(off, g.c[j]) + s);
    }
    if (K == 4) {
        a.cnt += s;
        return;
    }
    a.t4 += s;
    for (int w1 = lo; w1 < hi; ++w1) {
        uint32_t m = ri[w1] & rj[w1];
        while (m) {
            const int l = (w1 << 5) + __ffs(m) - 1;
            m &= m - 1;
            const uint32_t *rl = g.rows + (size_t)l * g.W;
            const int lo3 = max(lo, (int)g.rlo[l]);
            const int hi3 = min(hi, (int)g.rhi[l]);
            uint32_t t = 0;
            for (int w = lo3; w < hi3; ++w) t += __popc(ri[w] & rj[w] & rl[w]);
            a.cnt += t;
            if (STATS) a.bytes += 4ull * ((uint64_t)s + odeg(off, g.c[l]) + t);
        }
    }
}

// Count over rows [row_begin, d) with stride row_step; (i, j) items are dealt to the
// lanes of the calling warp in batches of 32.
template <int K, bool STATS>
__device__ void count_rows(const Local &g, const uint64_t *off, int row_begin, int row_step, Acc &a) {
    const unsigned lane = lane_id();
    int pc = 0;  // pending items held by lanes [0, pc)
    int my_i = 0, my_j = 0;
    for (int i = row_begin; i < g.d; i += row_step) {
        const uint32_t *ri = g.rows + (size_t)i * g.W;
        const int lo = g.rlo[i], hi = g.rhi[i];
        uint32_t pop = 0;
        for (int w = lo; w < hi; ++w) pop += __popc(ri[w]);
        if (lane == 0) a.t3 += pop;
        if (STATS && lane == 0) a.bytes += 4ull * ((uint64_t)g.d + odeg(off, g.c[i]) + pop);
        if (K == 3) {
            if (lane == 0) a.cnt += pop;
            continue;
        }
        for (int ww = lo; ww < hi; ++ww) {
            const uint32_t bits = ri[ww];
            const int c = __popc(bits);
            if (c == 0) continue;
            const int q = (int)lane;
            if (q >= pc && q < pc + c) {
                my_i = i;
                my_j = (ww << 5) + nth_set_bit(bits, q - pc);
            }
            if (pc + c >= 32) {
                process_item<K, STATS>(g, my_i, my_j, off, a);
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
    if (K > 3 && (int)lane < pc) process_item<K, STATS>(g, my_i, my_j, off, a);
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
constexpr int kWarpHashLog = 7;  // 128-slot table per warp
template <int K, bool STATS>
__global__ void __launch_bounds__(256) clique_warp_kernel(const uint64_t *__restrict__ off,
                                                          const uint32_t *__restrict__ adj, uint32_t n,
                                                          uint32_t dmin, unsigned long long *queue,
                                                          uint64_t *out, uint64_t *phase_bytes) {
    constexpr int W = kWarpMax / 32;
    constexpr int T = 1 << kWarpHashLog;
    __shared__ uint32_t s_c[8][kWarpMax];
    __shared__ uint32_t s_rows[8][kWarpMax * W];
    __shared__ uint32_t s_hkey[8][T];
    __shared__ uint16_t s_hidx[8][T];
    __shared__ uint16_t s_rlo[8][kWarpMax], s_rhi[8][kWarpMax];
    const unsigned lane = lane_id();
    const int wib = threadIdx.x >> 5;
    Local g;
    g.c = s_c[wib];
    g.rows = s_rows[wib];
    g.hkey = s_hkey[wib];
    g.hidx = s_hidx[wib];
    g.rlo = s_rlo[wib];
    g.rhi = s_rhi[wib];
    g.W = W;
    g.logt = kWarpHashLog;
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
            g.d = (int)__shfl_sync(kFull, myd, src);
            const uint64_t b0 = __ldg(off + v0);
            __syncwarp();
            for (int t = lane; t < kWarpMax; t += 32) g.c[t] = t < g.d ? __ldg(adj + b0 + t) : kEmpty;
            for (int t = lane; t < kWarpMax * W; t += 32) g.rows[t] = 0;
            for (int t = lane; t < T; t += 32) g.hkey[t] = kEmpty;
            __syncwarp();
            hash_insert(g, lane, 32);
            __syncwarp();
            if (g.d >= 2) build_rows(g, off, adj, 0, 1);
            __syncwarp();
            row_extents(g, lane, 32);
            __syncwarp();
            count_rows<K, STATS>(g, off, 0, 1, a);
        }
    }
    flush_acc(a, K, out, phase_bytes);
}

// shared-memory footprint of a block-tier launch serving out-degrees up to dcap
__host__ __device__ __forceinline__ int block_logt(int dcap) {
    int l = 5;
    while ((1 << l) < 2 * dcap) ++l;
    return l;
}
__host__ __device__ __forceinline__ size_t block_smem(int dcap) {
    const size_t dp = (size_t)((dcap + 31) & ~31);
    const size_t t = (size_t)1 << block_logt(dcap);
    const size_t w = (size_t)((dcap + 31) / 32);
    return dp * 4 + t * 4 + t * 2 + dp * 2 * 2 + dp * w * 4;
}

// Block tier: one block per start vertex from a degree-descending list.
template <int K, bool STATS>
__global__ void clique_block_kernel(const uint64_t *__restrict__ off, const uint32_t *__restrict__ adj,
                                    const uint32_t *__restrict__ list, uint32_t list_n, int dcap,
                                    unsigned long long *queue, uint64_t *out, uint64_t *phase_bytes) {
    extern __shared__ __align__(16) uint32_t smem[];
    __shared__ uint32_t s_v0;
    const int dp = (dcap + 31) & ~31;
    const int logt = block_logt(dcap);
    const int T = 1 << logt;
    Local g;
    g.c = smem;
    g.hkey = smem + dp;
    g.hidx = (uint16_t *)(g.hkey + T);
    g.rlo = g.hidx + T;
    g.rhi = g.rlo + dp;
    g.rows = (uint32_t *)(g.rhi + dp);
    g.logt = logt;
    const int warps = blockDim.x >> 5;
    const int wib = threadIdx.x >> 5;
    Acc a = {0, 0, 0, 0, 0};
    while (true) {
        if (threadIdx.x == 0) {
            const unsigned long long t = atomicAdd(queue, 1ull);
            s_v0 = t < list_n ? list[t] : kEmpty;
        }
        __syncthreads();
        const uint32_t v0 = s_v0;
        if (v0 == kEmpty) break;
        g.d = (int)odeg(off, v0);
        g.W = (g.d + 31) >> 5;
        if (threadIdx.x == 0) a.ext1 += (uint64_t)g.d;
        const uint64_t b0 = __ldg(off + v0);
        for (int t = threadIdx.x; t < g.d; t += blockDim.x) g.c[t] = __ldg(adj + b0 + t);
        for (int t = threadIdx.x; t < g.d * g.W; t += blockDim.x) g.rows[t] = 0;
        for (int t = threadIdx.x; t < T; t += blockDim.x) g.hkey[t] = kEmpty;
        __syncthreads();
        hash_insert(g, threadIdx.x, blockDim.x);
        __syncthreads();
        build_rows(g, off, adj, wib, warps);
        __syncthreads();
        row_extents(g, threadIdx.x, blockDim.x);
        __syncthreads();
        count_rows<K, STATS>(g, off, wib, warps, a);
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
    const int large_cap = (int)std::min<uint32_t>((uint32_t)kBlockMax, std::max<uint32_t>(g.max_degree, kMidMax + 1));
    const int tier_dcap[2] = {kMidMax, large_cap};
    const int tier_threads[2] = {256, 1024};
    for (int t = 0; t < 2; ++t) {
        const unsigned int cnt = h_counts[t];
        if (cnt == 0) continue;
        size_t cb = cub_bytes;
        KHZ_CUDA(cub::DeviceRadixSort::SortPairsDescending(cub_tmp, cb, keys + (size_t)t * n, skeys,
                                                           vals + (size_t)t * n, svals, (int)cnt, 0, 32, s));
        const int dcap = tier_dcap[t];
        const size_t smem = block_smem(dcap);
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
