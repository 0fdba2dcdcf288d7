// Device graph construction: CSR from a sorted edge list, degree orientation and the
// R-MAT generator.
//
// CSR build (graph_loader.h:154-201, 621-703): the .dgraph edge section is sorted by
// (src, dst), so offsets are the first positions of each source; a boundary kernel writes
// off[v] for every v in (src[i-1], src[i]] with no atomics and no scan, and a strided copy
// extracts the destinations.  A validation pass flags unsorted, duplicate, self-loop and
// out-of-range entries (the loader's asserts, graph_loader.h:891-898, become an error code).
//
// Orientation (toolkits/to_oriented_dataset_converter.cc:27-124): rank by (degree, id)
// with one 64-bit key sort, one warp per vertex counts and compacts its higher-ranked
// neighbours (ballot), an exclusive scan gives the offsets, and a segmented sort orders
// each out-list.  Sorting and scans use CUB.
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>

#include "khz_internal.cuh"

namespace khz {

static thread_local cudaMemPool_t t_pool = nullptr;
static thread_local cudaStream_t t_stream = nullptr;

AllocScope::AllocScope(cudaMemPool_t pool, cudaStream_t s) : prev_pool(t_pool), prev_stream(t_stream) {
    t_pool = pool;
    t_stream = s;
}
AllocScope::~AllocScope() {
    t_pool = prev_pool;
    t_stream = prev_stream;
}
cudaError_t dev_alloc(void **p, size_t bytes) {
    if (t_pool) return cudaMallocFromPoolAsync(p, bytes, t_pool, t_stream);
    return cudaMalloc(p, bytes);
}
void dev_free(void *p) {
    if (!p) return;
    if (t_pool) cudaFreeAsync(p, t_stream);
    else cudaFree(p);
}

namespace {

__global__ void validate_pairs_kernel(const uint32_t *__restrict__ pairs, uint64_t m, uint32_t n,
                                      unsigned int *bad) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t s = pairs[2 * i], d = pairs[2 * i + 1];
        bool ok = s < n && d < n && s != d;
        if (i > 0) {
            const uint64_t pk = ((uint64_t)pairs[2 * i - 2] << 32) | pairs[2 * i - 1];
            const uint64_t ck = ((uint64_t)s << 32) | d;
            ok = ok && ck > pk;
        }
        if (!ok) atomicOr(bad, 1u);
        if (s >= d) atomicOr(bad + 1, 1u);  // not upper-triangular
    }
}

// every entry (u, v) must have its reverse (v, u): one binary search per entry
__global__ void symmetry_kernel(const uint64_t *__restrict__ off, const uint32_t *__restrict__ adj, uint32_t n,
                                unsigned int *asym) {
    const unsigned lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t u = warp; u < n; u += nwarps) {
        const uint64_t b = off[u], e = off[u + 1];
        bool bad = false;
        for (uint64_t i = b + lane; i < e; i += 32) {
            const uint32_t v = adj[i];
            uint64_t l = off[v], r = off[v + 1];
            while (l < r) {
                const uint64_t mid = (l + r) >> 1;
                if (adj[mid] < u) l = mid + 1; else r = mid;
            }
            bad = bad || !(l < off[v + 1] && adj[l] == u);
        }
        if (__any_sync(0xffffffffu, bad)) {
            if (lane == 0) atomicOr(asym, 1u);
        }
    }
}

// off[v] = first i with src[i] >= v
__global__ void boundaries_kernel(const uint32_t *__restrict__ pairs, uint64_t m, uint32_t n, uint64_t *off) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i <= m; i += (uint64_t)gridDim.x * blockDim.x) {
        const int64_t prev = i == 0 ? -1 : (int64_t)pairs[2 * (i - 1)];
        const int64_t cur = i == m ? (int64_t)n : (int64_t)pairs[2 * i];
        for (int64_t v = prev + 1; v <= cur; ++v) off[v] = i;
    }
}

__global__ void extract_dst_kernel(const uint32_t *__restrict__ pairs, uint64_t m, uint32_t *adj) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x)
        adj[i] = pairs[2 * i + 1];
}

__global__ void max_degree_kernel(const uint64_t *__restrict__ off, uint32_t n, unsigned int *out) {
    unsigned int best = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        best = max(best, (unsigned int)(off[v + 1] - off[v]));
    for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_down_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, best);
}

__global__ void degree_keys_kernel(const uint64_t *__restrict__ off, uint32_t n, uint64_t *keys) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        keys[v] = ((uint64_t)(off[v + 1] - off[v]) << 32) | v;
}

__global__ void rank_kernel(const uint64_t *__restrict__ sorted_keys, uint32_t n, uint32_t *rank) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
        rank[(uint32_t)sorted_keys[r]] = r;
}

// one warp per rank r: count (or write) the ranks of u = order[r]'s neighbours above r
template <bool WRITE>
__global__ void orient_kernel(const uint64_t *__restrict__ off, const uint32_t *__restrict__ adj,
                              const uint64_t *__restrict__ sorted_keys, const uint32_t *__restrict__ rank,
                              uint32_t n, uint64_t *odeg_or_ooff, uint32_t *oadj) {
    const unsigned lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t r = warp; r < n; r += nwarps) {
        const uint32_t u = (uint32_t)sorted_keys[r];
        const uint64_t b = off[u], e = off[u + 1];
        uint64_t pos = WRITE ? odeg_or_ooff[r] : 0;
        uint64_t cnt = 0;
        for (uint64_t i = b; i < e; i += 32) {
            const uint64_t idx = i + lane;
            uint32_t rv = 0;
            bool keep = false;
            if (idx < e) {
                rv = rank[adj[idx]];
                keep = rv > r;
            }
            const unsigned bal = __ballot_sync(0xffffffffu, keep);
            if (WRITE && keep) oadj[pos + cnt + __popc(bal & ((1u << lane) - 1u))] = rv;
            cnt += __popc(bal);
        }
        if (!WRITE && lane == 0) odeg_or_ooff[r] = cnt;
    }
}

// degree-descending relabelling: new vertex q = n - 1 - r is u = order[r]; its list holds the new
// ids of all of u's neighbours (one warp per new vertex; lists sorted afterwards)
__global__ void relabel_degree_count_kernel(const uint64_t *__restrict__ off, const uint64_t *__restrict__ sorted_keys,
                                            uint32_t n, uint64_t *deg) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const uint32_t u = (uint32_t)sorted_keys[n - 1 - q];
        deg[q] = off[u + 1] - off[u];
    }
}
__global__ void relabel_degree_write_kernel(const uint64_t *__restrict__ off, const uint32_t *__restrict__ adj,
                                            const uint64_t *__restrict__ sorted_keys, const uint32_t *__restrict__ rank,
                                            uint32_t n, const uint64_t *__restrict__ noff, uint32_t *nadj) {
    const unsigned lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t q = warp; q < n; q += nwarps) {
        const uint32_t u = (uint32_t)sorted_keys[n - 1 - q];
        const uint64_t b = off[u], e = off[u + 1], o = noff[q];
        for (uint64_t i = b + lane; i < e; i += 32) nadj[o + (i - b)] = n - 1 - rank[adj[i]];
    }
}

__global__ void rmat_kernel(int scale, uint64_t base, uint32_t ta, uint32_t tab, uint32_t tabc, uint64_t raw,
                            uint64_t *keys) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < raw; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t s = 0, d = 0;
        for (int l = 0; l < scale; ++l) {
            // splitmix64 finaliser of (base ^ (64 i + l))
            uint64_t z = (base ^ (i * 64u + (uint64_t)l)) + 0x9E3779B97F4A7C15ULL;
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
            z ^= z >> 31;
            const uint32_t u = (uint32_t)(z >> 32);
            const uint32_t sb = u >= tab ? 1u : 0u;
            const uint32_t db = (u >= ta && u < tab) || u >= tabc ? 1u : 0u;
            s |= sb << (scale - 1 - l);
            d |= db << (scale - 1 - l);
        }
        keys[i] = s == d ? ~0ull : (((uint64_t)min(s, d) << 32) | max(s, d));
    }
}

__global__ void mark_present_kernel(const uint64_t *__restrict__ keys, uint64_t m, uint32_t *present) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
        present[keys[i] >> 32] = 1;
        present[(uint32_t)keys[i]] = 1;
    }
}

// both directions of every relabelled canonical edge
__global__ void relabel_sym_kernel(const uint64_t *__restrict__ keys, uint64_t m, const uint32_t *__restrict__ newid,
                                   uint64_t *sym) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t a = newid[keys[i] >> 32], b = newid[(uint32_t)keys[i]];
        sym[2 * i] = ((uint64_t)a << 32) | b;
        sym[2 * i + 1] = ((uint64_t)b << 32) | a;
    }
}

// a sorted 64-bit key (src << 32 | dst) array viewed as packed (dst, src) little-endian words:
// swap halves into (src, dst) pairs in place
__global__ void keys_to_pairs_kernel(uint64_t *keys, uint64_t m) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = keys[i];
        keys[i] = (k >> 32) | (k << 32);
    }
}

int grid_for(uint64_t work, int sms) {
    const uint64_t g = (work + 255) / 256;
    return (int)std::max<uint64_t>(1, std::min<uint64_t>(g, (uint64_t)sms * 32));
}

int num_sms() {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms > 0 ? sms : 1;
}

template <typename T>
khz_status dalloc(T **p, size_t count) {
    *p = nullptr;
    cudaError_t e = dev_alloc((void **)p, std::max<size_t>(count, 1) * sizeof(T));
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error("device allocation of %llu bytes failed: %s", (unsigned long long)(count * sizeof(T)),
                  cudaGetErrorString(e));
        return KHZ_ERR_OOM;
    }
    return KHZ_OK;
}

struct DevBuf {
    void *p = nullptr;
    ~DevBuf() { dev_free(p); }
};

}  // namespace

void free_graph_memory(Graph *g) {
    dev_free(g->off);
    dev_free(g->adj);
    dev_free(g->labels);
    g->off = nullptr;
    g->adj = nullptr;
    g->labels = nullptr;
    g->num_labels = 0;
    g->label_count.clear();
}

khz_status build_csr_from_device_pairs(const uint32_t *d_pairs, uint64_t m, uint32_t n, bool validate, Graph *g,
                                       cudaStream_t s) {
    const int sms = num_sms();
    if (n == 0 && m > 0) {
        set_error("edges given for a graph with 0 vertices");
        return KHZ_ERR_FORMAT;
    }
    DevBuf flag;
    KHZ_CUDA(dev_alloc(&flag.p, sizeof(unsigned int) * 4));
    KHZ_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(unsigned int) * 4, s));
    unsigned int hflags[4] = {0, 1, 1, 0};  // bad, not_upper, asym (unknown without validation)
    if (validate && m > 0) {
        validate_pairs_kernel<<<grid_for(m, sms), 256, 0, s>>>(d_pairs, m, n, (unsigned int *)flag.p);
        KHZ_CUDA(cudaGetLastError());
        KHZ_CUDA(cudaMemcpyAsync(hflags, flag.p, sizeof(unsigned int) * 2, cudaMemcpyDeviceToHost, s));
        KHZ_CUDA(cudaStreamSynchronize(s));
        if (hflags[0]) {
            set_error("edge list is not sorted by (src, dst), has duplicates or self-loops, or ids >= n");
            return KHZ_ERR_FORMAT;
        }
    } else if (validate) {
        hflags[1] = 0;  // an empty graph is both upper-triangular and symmetric
        hflags[2] = 0;
    }
    Graph out;
    out.n = n;
    out.m = m;
    khz_status st = dalloc(&out.off, (size_t)n + 1);
    if (st) return st;
    st = dalloc(&out.adj, (size_t)m + kAdjPad);
    if (st) {
        free_graph_memory(&out);
        return st;
    }
    cudaMemsetAsync(out.adj + m, 0xff, kAdjPad * sizeof(uint32_t), s);
    boundaries_kernel<<<grid_for(m + 1, sms), 256, 0, s>>>(d_pairs, m, n, out.off);
    if (m > 0) extract_dst_kernel<<<grid_for(m, sms), 256, 0, s>>>(d_pairs, m, out.adj);
    unsigned int *d_max = (unsigned int *)flag.p + 3;
    KHZ_CUDA(cudaMemsetAsync(d_max, 0, sizeof(unsigned int), s));
    if (validate && m > 0 && hflags[1]) {
        // not a DAG in id order: find out whether it is the symmetric (undirected) form
        symmetry_kernel<<<grid_for((uint64_t)n * 32, sms), 256, 0, s>>>(out.off, out.adj, n,
                                                                         (unsigned int *)flag.p + 2);
        KHZ_CUDA(cudaMemcpyAsync(&hflags[2], (unsigned int *)flag.p + 2, sizeof(unsigned int),
                                 cudaMemcpyDeviceToHost, s));
    }
    if (n > 0) max_degree_kernel<<<grid_for(n, sms), 256, 0, s>>>(out.off, n, d_max);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        free_graph_memory(&out);
        return cuda_fail(e, "csr build kernels");
    }
    unsigned int mx = 0;
    KHZ_CUDA(cudaMemcpyAsync(&mx, d_max, sizeof(mx), cudaMemcpyDeviceToHost, s));
    KHZ_CUDA(cudaStreamSynchronize(s));
    out.max_degree = mx;
    out.oriented = hflags[1] == 0;
    out.symmetric = hflags[2] == 0;
    out.bytes = ((uint64_t)n + 1) * 8 + (m + kAdjPad) * 4;
    *g = out;
    return KHZ_OK;
}

khz_status orient_graph(const Graph &in, Graph *outg, cudaStream_t s) {
    const int sms = num_sms();
    const uint32_t n = in.n;
    Graph out;
    out.n = n;
    out.oriented = true;
    DevBuf keys, skeys, rank, tmp;
    KHZ_CUDA(dev_alloc(&keys.p, sizeof(uint64_t) * ((size_t)n + 1)));
    KHZ_CUDA(dev_alloc(&skeys.p, sizeof(uint64_t) * std::max<uint32_t>(n, 1)));
    KHZ_CUDA(dev_alloc(&rank.p, sizeof(uint32_t) * std::max<uint32_t>(n, 1)));
    khz_status st = dalloc(&out.off, (size_t)n + 1);
    if (st) return st;
    if (n > 0) {
        degree_keys_kernel<<<grid_for(n, sms), 256, 0, s>>>(in.off, n, (uint64_t *)keys.p);
        size_t tb = 0;
        cub::DeviceRadixSort::SortKeys(nullptr, tb, (uint64_t *)keys.p, (uint64_t *)skeys.p, (int)n);
        size_t tb2 = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tb2, out.off, out.off, (int)n + 1);
        KHZ_CUDA(dev_alloc(&tmp.p, std::max(tb, tb2)));
        KHZ_CUDA(cub::DeviceRadixSort::SortKeys(tmp.p, tb, (uint64_t *)keys.p, (uint64_t *)skeys.p, (int)n, 0, 64, s));
        rank_kernel<<<grid_for(n, sms), 256, 0, s>>>((uint64_t *)skeys.p, n, (uint32_t *)rank.p);
        const int wblocks = (int)std::max<uint64_t>(1, std::min<uint64_t>(((uint64_t)n + 7) / 8, (uint64_t)sms * 16));
        // out-degrees into the (now free) key buffer, then offsets = exclusive scan
        uint64_t *odeg = (uint64_t *)keys.p;
        KHZ_CUDA(cudaMemsetAsync(odeg + n, 0, sizeof(uint64_t), s));
        orient_kernel<false><<<wblocks, 256, 0, s>>>(in.off, in.adj, (uint64_t *)skeys.p, (uint32_t *)rank.p, n,
                                                     odeg, nullptr);
        tb2 = std::max(tb, tb2);
        KHZ_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tb2, odeg, out.off, (int)n + 1, s));
        uint64_t m = 0;
        KHZ_CUDA(cudaMemcpyAsync(&m, out.off + n, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
        KHZ_CUDA(cudaStreamSynchronize(s));
        out.m = m;
        st = dalloc(&out.adj, (size_t)m + kAdjPad);
        if (st) {
            free_graph_memory(&out);
            return st;
        }
        KHZ_CUDA(cudaMemsetAsync(out.adj + m, 0xff, kAdjPad * sizeof(uint32_t), s));
        orient_kernel<true><<<wblocks, 256, 0, s>>>(in.off, in.adj, (uint64_t *)skeys.p, (uint32_t *)rank.p, n,
                                                    out.off, out.adj);
        KHZ_CUDA(cudaGetLastError());
        if (m > 0) {
            DevBuf sorted, stmp;
            KHZ_CUDA(dev_alloc(&sorted.p, sizeof(uint32_t) * m));
            size_t sb = 0;
            cub::DeviceSegmentedSort::SortKeys(nullptr, sb, out.adj, (uint32_t *)sorted.p, (int64_t)m, (int64_t)n,
                                               out.off, out.off + 1);
            KHZ_CUDA(dev_alloc(&stmp.p, std::max<size_t>(sb, 1)));
            KHZ_CUDA(cub::DeviceSegmentedSort::SortKeys(stmp.p, sb, out.adj, (uint32_t *)sorted.p, (int64_t)m,
                                                        (int64_t)n, out.off, out.off + 1, s));
            KHZ_CUDA(cudaMemcpyAsync(out.adj, sorted.p, sizeof(uint32_t) * m, cudaMemcpyDeviceToDevice, s));
            KHZ_CUDA(cudaStreamSynchronize(s));
        }
    } else {
        KHZ_CUDA(cudaMemsetAsync(out.off, 0, sizeof(uint64_t), s));
        st = dalloc(&out.adj, kAdjPad);
        if (st) return st;
    }
    unsigned int *d_max = nullptr;
    KHZ_CUDA(dev_alloc((void **)&d_max, sizeof(unsigned int)));
    cudaMemsetAsync(d_max, 0, sizeof(unsigned int), s);
    if (n > 0) max_degree_kernel<<<grid_for(n, sms), 256, 0, s>>>(out.off, n, d_max);
    unsigned int mx = 0;
    cudaMemcpyAsync(&mx, d_max, sizeof(mx), cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    dev_free(d_max);
    if (e != cudaSuccess) {
        free_graph_memory(&out);
        return cuda_fail(e, "orientation");
    }
    out.max_degree = mx;
    out.oriented = true;
    out.symmetric = out.m == 0;
    out.bytes = ((uint64_t)n + 1) * 8 + (out.m + kAdjPad) * 4;
    *outg = out;
    return KHZ_OK;
}

// The same undirected graph with vertices renumbered by descending (degree, id): new id
// n - 1 - rank, rank being the orientation's (degree, id) order.  Every list keeps all neighbours,
// sorted.  Counting with the smallest new id as the start vertex then starts each copy of a
// pattern at its highest-degree vertex.
khz_status relabel_by_degree(const Graph &in, Graph *outg, cudaStream_t s) {
    const int sms = num_sms();
    const uint32_t n = in.n;
    Graph out;
    out.n = n;
    out.m = in.m;
    DevBuf keys, skeys, rank, tmp;
    KHZ_CUDA(dev_alloc(&keys.p, sizeof(uint64_t) * ((size_t)n + 1)));
    KHZ_CUDA(dev_alloc(&skeys.p, sizeof(uint64_t) * std::max<uint32_t>(n, 1)));
    KHZ_CUDA(dev_alloc(&rank.p, sizeof(uint32_t) * std::max<uint32_t>(n, 1)));
    khz_status st = dalloc(&out.off, (size_t)n + 1);
    if (st) return st;
    st = dalloc(&out.adj, (size_t)in.m + kAdjPad);
    if (st) {
        free_graph_memory(&out);
        return st;
    }
    KHZ_CUDA(cudaMemsetAsync(out.adj + in.m, 0xff, kAdjPad * sizeof(uint32_t), s));
    if (n > 0) {
        degree_keys_kernel<<<grid_for(n, sms), 256, 0, s>>>(in.off, n, (uint64_t *)keys.p);
        size_t tb = 0, tb2 = 0;
        cub::DeviceRadixSort::SortKeys(nullptr, tb, (uint64_t *)keys.p, (uint64_t *)skeys.p, (int)n);
        cub::DeviceScan::ExclusiveSum(nullptr, tb2, out.off, out.off, (int)n + 1);
        KHZ_CUDA(dev_alloc(&tmp.p, std::max(tb, tb2)));
        KHZ_CUDA(cub::DeviceRadixSort::SortKeys(tmp.p, tb, (uint64_t *)keys.p, (uint64_t *)skeys.p, (int)n, 0, 64, s));
        rank_kernel<<<grid_for(n, sms), 256, 0, s>>>((uint64_t *)skeys.p, n, (uint32_t *)rank.p);
        uint64_t *deg = (uint64_t *)keys.p;
        KHZ_CUDA(cudaMemsetAsync(deg + n, 0, sizeof(uint64_t), s));
        relabel_degree_count_kernel<<<grid_for(n, sms), 256, 0, s>>>(in.off, (uint64_t *)skeys.p, n, deg);
        tb2 = std::max(tb, tb2);
        KHZ_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tb2, deg, out.off, (int)n + 1, s));
        const int wblocks = (int)std::max<uint64_t>(1, std::min<uint64_t>(((uint64_t)n + 7) / 8, (uint64_t)sms * 16));
        relabel_degree_write_kernel<<<wblocks, 256, 0, s>>>(in.off, in.adj, (uint64_t *)skeys.p, (uint32_t *)rank.p, n,
                                                            out.off, out.adj);
        KHZ_CUDA(cudaGetLastError());
        if (in.m > 0) {
            DevBuf sorted, stmp;
            KHZ_CUDA(dev_alloc(&sorted.p, sizeof(uint32_t) * in.m));
            size_t sb = 0;
            cub::DeviceSegmentedSort::SortKeys(nullptr, sb, out.adj, (uint32_t *)sorted.p, (int64_t)in.m, (int64_t)n,
                                               out.off, out.off + 1);
            KHZ_CUDA(dev_alloc(&stmp.p, std::max<size_t>(sb, 1)));
            KHZ_CUDA(cub::DeviceSegmentedSort::SortKeys(stmp.p, sb, out.adj, (uint32_t *)sorted.p, (int64_t)in.m,
                                                        (int64_t)n, out.off, out.off + 1, s));
            KHZ_CUDA(cudaMemcpyAsync(out.adj, sorted.p, sizeof(uint32_t) * in.m, cudaMemcpyDeviceToDevice, s));
        }
    } else {
        KHZ_CUDA(cudaMemsetAsync(out.off, 0, sizeof(uint64_t), s));
    }
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        free_graph_memory(&out);
        return cuda_fail(e, "degree relabelling");
    }
    out.max_degree = in.max_degree;
    out.symmetric = in.symmetric;
    out.oriented = in.m == 0;
    out.bytes = ((uint64_t)n + 1) * 8 + (out.m + kAdjPad) * 4;
    *outg = out;
    return KHZ_OK;
}

khz_status generate_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed, Graph *g,
                         cudaStream_t s) {
    if (scale < 1 || scale > 31 || edge_factor < 1) {
        set_error("R-MAT scale must be in [1, 31] and edge factor >= 1");
        return KHZ_ERR_ARG;
    }
    const int sms = num_sms();
    const uint64_t raw = (uint64_t)edge_factor << scale;
    const uint32_t ta = (uint32_t)(a * 4294967296.0);
    const uint32_t tab = (uint32_t)((a + b) * 4294967296.0);
    const uint32_t tabc = (uint32_t)((a + b + c) * 4294967296.0);
    // splitmix64 of the seed, as in the oracle's generator
    uint64_t base = seed + 0x9E3779B97F4A7C15ULL;
    base = (base ^ (base >> 30)) * 0xBF58476D1CE4E5B9ULL;
    base = (base ^ (base >> 27)) * 0x94D049BB133111EBULL;
    base ^= base >> 31;
    DevBuf keys, keys2, tmp, uniq_count, present, newid;
    KHZ_CUDA(dev_alloc(&keys.p, sizeof(uint64_t) * raw));
    KHZ_CUDA(dev_alloc(&keys2.p, sizeof(uint64_t) * raw));
    rmat_kernel<<<grid_for(raw, sms), 256, 0, s>>>(scale, base, ta, tab, tabc, raw, (uint64_t *)keys.p);
    KHZ_CUDA(cudaGetLastError());
    size_t tb_sort = 0, tb_uniq = 0, tb_scan = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, tb_sort, (uint64_t *)keys.p, (uint64_t *)keys2.p, (int64_t)raw);
    cub::DeviceSelect::Unique(nullptr, tb_uniq, (uint64_t *)keys2.p, (uint64_t *)keys.p, (uint64_t *)nullptr,
                              (int64_t)raw);
    const uint32_t id_space = 1u << scale;
    cub::DeviceScan::ExclusiveSum(nullptr, tb_scan, (uint32_t *)nullptr, (uint32_t *)nullptr, (int)id_space + 1);
    // the symmetric key array (2m) is sorted later with the same temp size bound (2m <= 2 raw)
    size_t tb_sort2 = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, tb_sort2, (uint64_t *)keys.p, (uint64_t *)keys2.p, (int64_t)(2 * raw));
    const size_t tb = std::max(std::max(tb_sort, tb_uniq), std::max(tb_scan, tb_sort2));
    KHZ_CUDA(dev_alloc(&tmp.p, tb));
    KHZ_CUDA(dev_alloc(&uniq_count.p, sizeof(uint64_t)));
    size_t t1 = tb;
    KHZ_CUDA(cub::DeviceRadixSort::SortKeys(tmp.p, t1, (uint64_t *)keys.p, (uint64_t *)keys2.p, (int64_t)raw, 0, 64, s));
    t1 = tb;
    KHZ_CUDA(cub::DeviceSelect::Unique(tmp.p, t1, (uint64_t *)keys2.p, (uint64_t *)keys.p, (uint64_t *)uniq_count.p,
                                       (int64_t)raw, s));
    uint64_t nuniq = 0;
    KHZ_CUDA(cudaMemcpyAsync(&nuniq, uniq_count.p, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    KHZ_CUDA(cudaStreamSynchronize(s));
    // the self-loop sentinel sorts last
    uint64_t last = 0;
    if (nuniq > 0) {
        KHZ_CUDA(cudaMemcpy(&last, (uint64_t *)keys.p + nuniq - 1, sizeof(uint64_t), cudaMemcpyDeviceToHost));
        if (last == ~0ull) nuniq -= 1;
    }
    const uint64_t m = nuniq;
    KHZ_CUDA(dev_alloc(&present.p, sizeof(uint32_t) * ((size_t)id_space + 1)));
    KHZ_CUDA(dev_alloc(&newid.p, sizeof(uint32_t) * ((size_t)id_space + 1)));
    KHZ_CUDA(cudaMemsetAsync(present.p, 0, sizeof(uint32_t) * ((size_t)id_space + 1), s));
    if (m > 0) mark_present_kernel<<<grid_for(m, sms), 256, 0, s>>>((uint64_t *)keys.p, m, (uint32_t *)present.p);
    t1 = tb;
    KHZ_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, t1, (uint32_t *)present.p, (uint32_t *)newid.p, (int)id_space + 1, s));
    uint32_t n = 0;
    KHZ_CUDA(cudaMemcpyAsync(&n, (uint32_t *)newid.p + id_space, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    // symmetric keys: reuse keys2 (raw entries) when 2m fits, otherwise allocate
    DevBuf sym, sym_sorted;
    KHZ_CUDA(dev_alloc(&sym.p, sizeof(uint64_t) * std::max<uint64_t>(2 * m, 1)));
    KHZ_CUDA(dev_alloc(&sym_sorted.p, sizeof(uint64_t) * std::max<uint64_t>(2 * m, 1)));
    if (m > 0)
        relabel_sym_kernel<<<grid_for(m, sms), 256, 0, s>>>((uint64_t *)keys.p, m, (uint32_t *)newid.p,
                                                             (uint64_t *)sym.p);
    // release the raw buffers before the second sort
    KHZ_CUDA(cudaStreamSynchronize(s));
    dev_free(keys.p);
    keys.p = nullptr;
    dev_free(keys2.p);
    keys2.p = nullptr;
    t1 = tb;
    if (m > 0)
        KHZ_CUDA(cub::DeviceRadixSort::SortKeys(tmp.p, t1, (uint64_t *)sym.p, (uint64_t *)sym_sorted.p,
                                                (int64_t)(2 * m), 0, 64, s));
    if (m > 0) keys_to_pairs_kernel<<<grid_for(2 * m, sms), 256, 0, s>>>((uint64_t *)sym_sorted.p, 2 * m);
    KHZ_CUDA(cudaGetLastError());
    khz_status st = build_csr_from_device_pairs((const uint32_t *)sym_sorted.p, 2 * m, n, false, g, s);
    if (st == KHZ_OK) {
        g->symmetric = true;  // both directions of every edge by construction
        g->oriented = m == 0;
    }
    return st;
}

}  // namespace khz
