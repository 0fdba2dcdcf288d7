// Identity engine for the patterns on symmetric graphs whose schedules the DFS engine would run
// with work growing with the square of hub degrees: the kautomine-idiom vertex-induced 4-motif
// (six counts), the kgraphpi tailed triangle and the kgraphpi house.
//
// Non-induced counts from per-edge triangle counts t(e), per-vertex triangle counts
// t(v) = sum_{e at v} t(e) / 2 and degrees d(v):
//   triangles T  = sum_e t(e) / 3          diamonds D   = sum_e C(t(e), 2)
//   3-stars S    = sum_v C(d(v), 3)        tailed Tl    = sum_v t(v) (d(v) - 2)
//   4-paths P    = sum_{edges uv} (d(u) - 1)(d(v) - 1) - 3 T
// with the 4-cycles C4 (wedge engine) and 4-cliques K4 (bitmap engine) counted into auxiliary rows.
// The vertex-induced counts follow by inclusion-exclusion over the copies of each pattern in the
// denser ones:
//   K4, diamond = D - 6 K4, 4-cycle = C4 - D + 3 K4, tailed triangle = Tl - 4 D + 12 K4,
//   4-path = P - 2 Tl - 4 C4 + 6 D - 12 K4, 3-star = S - Tl + 2 D - 4 K4.
// NumExtensions of the schedules (every queued embedding, engine.cc:924), from the same sums with
// E undirected edges and W = sum_v C(d(v), 2):
//   4-motif (six runs, three_motif.cc:87-127 idiom)     6 n + 10 E + 5 W - 8 T
//   tailed triangle (kgraphpi/four_clique.cc idiom)      n + 2 E + 3 T
// The per-edge triangle counts come from the oriented view: each triangle a < b < c (rank order)
// is found once, at its edge (a, b), as a common out-neighbour c, and adds one to its three edges.
//
// House (square v0 v1 v2 v3, roof v4 on v0 and v1; edge-induced, one automorphism broken by
// v1 > v0): every house is one 4-cycle plus one apex over one of the cycle's edges, the apex outside
// the cycle.  Summing over the 4-cycles the triangle counts of their four edges counts those, plus
// the apexes inside the cycle: a cycle with a chord is a diamond, and each diamond (cycle p x q y,
// chord x y) has one such apex on each of its four cycle edges.  So
//   houses = sum over 4-cycles of sum over their edges of t(e)  -  4 D,
// the first term from the wedge engine (WJob::tri), walking the degree-descending renumbering with
// the triangle count of each of its entries.  The schedule's NumExtensions: n + E at depths 0-1,
// sum over edges v0 < v1 of (d(v1) - 1) at depth 2, and at depth 3 each 4-cycle once per edge
// (v3 in N(v0) n N(v2) other than v1): n + E + sum_v (d(v) - 1) #{u in N(v) : u < v} + 4 C4.
#include <cuda_runtime.h>

#include <algorithm>

#include "khz_internal.cuh"
#include "khz_setops.cuh"

namespace khz {
namespace {

enum : int { kSumT3 = 0, kSumD = 1, kSumTl = 2, kSumS = 3, kSumW = 4, kSumPE = 5, kSumL2 = 6 };

__device__ __forceinline__ void warp_add(unsigned long long *dst, unsigned long long v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
    if (lane_id() == 0 && v) atomicAdd(dst, v);
}

// warp per start vertex a (claimed from a counter): for each out-neighbour b (edge e_ab), the
// members c of N+(a) after b found in N+(b) close the triangles (a, b, c)
__global__ void __launch_bounds__(256) motif_tri_kernel(MotifJob J, unsigned long long *queue) {
    const unsigned lane = lane_id();
    while (true) {
        unsigned long long a = 0;
        if (lane == 0) a = atomicAdd(queue, 1ull);
        a = __shfl_sync(kFull, a, 0);
        if (a >= J.n) break;
        const uint64_t ba = J.ooff[a];
        const uint32_t da = (uint32_t)(J.ooff[a + 1] - ba);
        for (uint32_t ib = 0; ib + 1 < da; ++ib) {
            const uint32_t b = __ldg(J.oadj + ba + ib);
            const uint64_t bb = J.ooff[b];
            const uint32_t db = (uint32_t)(J.ooff[b + 1] - bb);
            if (db == 0) continue;
            uint32_t found = 0;
            for (uint32_t k = ib + 1 + lane; k < da; k += 32) {
                const uint32_t c = __ldg(J.oadj + ba + k);
                const uint32_t jb = lower_bound_u32(J.oadj + bb, 0, db, c);
                if (jb < db && __ldg(J.oadj + bb + jb) == c) {
                    atomicAdd(&J.tri[ba + k], 1u);
                    atomicAdd(&J.tri[bb + jb], 1u);
                    ++found;
                }
            }
            for (int o = 16; o > 0; o >>= 1) found += __shfl_down_sync(kFull, found, o);
            if (lane == 0 && found) atomicAdd(&J.tri[ba + ib], found);
        }
    }
}

// per out-edge (a, b): the diamond and triangle sums, t(e) into both endpoints' accumulators, and
// the undirected degrees (out-degree plus in-degree); warp per vertex a
__global__ void __launch_bounds__(256) motif_edge_kernel(MotifJob J) {
    const unsigned lane = lane_id();
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    unsigned long long t3 = 0, dia = 0;
    for (uint32_t a = warp; a < J.n; a += nw) {
        const uint64_t ba = J.ooff[a], ea = J.ooff[a + 1];
        unsigned long long acc_a = 0;
        for (uint64_t e = ba + lane; e < ea; e += 32) {
            const unsigned long long t = J.tri[e];
            const uint32_t b = J.oadj[e];
            t3 += t;
            dia += t * (t - (t > 0 ? 1 : 0)) / 2;
            acc_a += t;
            if (t) atomicAdd(&J.acc[b], t);
            atomicAdd(&J.deg[b], 1u);
        }
        for (int o = 16; o > 0; o >>= 1) acc_a += __shfl_down_sync(kFull, acc_a, o);
        if (lane == 0) {
            if (acc_a) atomicAdd(&J.acc[a], acc_a);
            atomicAdd(&J.deg[a], (unsigned int)(ea - ba));
        }
    }
    warp_add(&J.sums[kSumT3], t3);
    warp_add(&J.sums[kSumD], dia);
}

// per vertex: tailed-triangle, 3-star and wedge sums
__global__ void motif_vertex_kernel(MotifJob J) {
    unsigned long long tl = 0, st = 0, w = 0;
    const uint32_t stride = gridDim.x * blockDim.x;  // a multiple of 32
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < ((J.n + 31) & ~31u); v += stride) {
        if (v < J.n) {
            const unsigned long long d = J.deg[v];
            const unsigned long long tv = J.acc[v] / 2;
            if (d >= 2) {
                tl += tv * (d - 2);
                w += d * (d - 1) / 2;
            }
            if (d >= 3) st += d * (d - 1) * (d - 2) / 6;
        }
    }
    warp_add(&J.sums[kSumTl], tl);
    warp_add(&J.sums[kSumS], st);
    warp_add(&J.sums[kSumW], w);
}

// per edge: (d(a) - 1)(d(b) - 1); warp per vertex a
__global__ void __launch_bounds__(256) motif_path_kernel(MotifJob J) {
    const unsigned lane = lane_id();
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    unsigned long long pe = 0;
    for (uint32_t a = warp; a < J.n; a += nw) {
        const unsigned long long da = J.deg[a];
        for (uint64_t e = J.ooff[a] + lane; e < J.ooff[a + 1]; e += 32)
            pe += (da - 1) * ((unsigned long long)J.deg[J.oadj[e]] - 1);
    }
    warp_add(&J.sums[kSumPE], pe);
}

// House: the triangle count of every entry of the degree-descending renumbering (vertex x is the
// oriented view's a = n - 1 - x).  x's entries below x are a's out-list in reverse order; an entry
// y above x is the out-edge (n - 1 - y, a), found by binary search.  Warp per x.
__global__ void __launch_bounds__(256) motif_house_entries_kernel(MotifJob J) {
    const unsigned lane = lane_id();
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t x = warp; x < J.n; x += nw) {
        const uint32_t a = J.n - 1 - x;
        const uint64_t ba = J.ooff[a];
        const uint32_t p = (uint32_t)(J.ooff[a + 1] - ba);
        const uint64_t bx = J.doff[x];
        const uint32_t dx = (uint32_t)(J.doff[x + 1] - bx);
        for (uint32_t i = lane; i < dx; i += 32) {
            uint32_t t;
            if (i < p) {
                t = J.tri[ba + (p - 1 - i)];
            } else {
                const uint32_t b = J.n - 1 - J.dadj[bx + i];
                const uint64_t bb = J.ooff[b];
                t = J.tri[bb + lower_bound_u32(J.oadj + bb, 0, (uint32_t)(J.ooff[b + 1] - bb), a)];
            }
            J.tdv[bx + i] = t;
        }
    }
}

// House NumExtensions at depth 2: sum over the stored graph's vertices of (d(v) - 1) times the
// number of neighbours below v
__global__ void motif_house_depth2_kernel(MotifJob J) {
    unsigned long long l2 = 0;
    const uint32_t stride = gridDim.x * blockDim.x;  // a multiple of 32
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < ((J.n + 31) & ~31u); v += stride) {
        if (v < J.n) {
            const uint64_t b = J.soff[v];
            const uint32_t d = (uint32_t)(J.soff[v + 1] - b);
            if (d > 1) l2 += (unsigned long long)(d - 1) * lower_bound_u32(J.sadj + b, 0, d, v);
        }
    }
    warp_add(&J.sums[kSumL2], l2);
}

// the job's raw counters (the finalize kernel divides by the multiplicities) and NumExtensions
__global__ void motif_combine_kernel(MotifJob J, uint64_t *rows) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const long long t = (long long)(J.sums[kSumT3] / 3), d = (long long)J.sums[kSumD],
                    tl = (long long)J.sums[kSumTl], s = (long long)J.sums[kSumS], w = (long long)J.sums[kSumW];
    const long long n = J.n, e = (long long)J.om;
    uint64_t *row = rows + (size_t)J.out_row * kRowWords;
    if (J.kind == KHZ_KGPI_HOUSE) {
        const long long c4 = (long long)rows[(size_t)J.c4_row * kRowWords];
        const long long tsum = (long long)rows[(size_t)J.house_row * kRowWords];
        row[0] = (uint64_t)(tsum - 4 * d);
        row[KHZ_MAX_COUNTS] = (uint64_t)(n + e + (long long)J.sums[kSumL2] + 4 * c4);
        return;
    }
    if (J.kind == KHZ_KGPI_TAILED_TRIANGLE) {
        row[0] = (uint64_t)tl;
        row[KHZ_MAX_COUNTS] = (uint64_t)(n + 2 * e + 3 * t);
        return;
    }
    const long long k4 = (long long)rows[(size_t)J.k4_row * kRowWords];
    const long long c4 = (long long)rows[(size_t)J.c4_row * kRowWords];
    const long long p = (long long)J.sums[kSumPE] - 3 * t;
    const long long induced[6] = {s - tl + 2 * d - 4 * k4,         p - 2 * tl - 4 * c4 + 6 * d - 12 * k4,
                                  tl - 4 * d + 12 * k4,             c4 - d + 3 * k4,
                                  d - 6 * k4,                       k4};
    const long long mult[6] = {1, 2, 1, 8, 1, 1};  // the schedule's raw counters before division
    for (int c = 0; c < 6; ++c) row[c] = (uint64_t)(induced[c] * mult[c]);
    row[KHZ_MAX_COUNTS] = (uint64_t)(6 * n + 10 * e + 5 * w - 8 * t);
}

}  // namespace

size_t motif_arena_bytes(const std::vector<MotifJob> &jobs) {
    size_t b = Arena::round(sizeof(MotifJob) * std::max<size_t>(jobs.size(), 1)) +
               Arena::round(sizeof(unsigned long long) * std::max<size_t>(jobs.size(), 1));
    for (const auto &j : jobs) {
        b += Arena::round(sizeof(uint32_t) * std::max<uint64_t>(j.om, 1)) +
             Arena::round(sizeof(unsigned long long) * std::max<uint32_t>(j.n, 1)) +
             Arena::round(sizeof(uint32_t) * std::max<uint32_t>(j.n, 1)) +
             Arena::round(sizeof(unsigned long long) * kMotifSums);
        if (j.kind == KHZ_KGPI_HOUSE) b += Arena::round(sizeof(uint32_t) * std::max<uint64_t>(2 * j.om, 1));
    }
    return b;
}

khz_status motif_prepare(std::vector<MotifJob> jobs, Arena *arena, MotifLaunch *ml, cudaStream_t s) {
    MotifLaunch L;
    for (auto &j : jobs) {
        j.tri = arena->take<uint32_t>(j.om);
        j.acc = arena->take<unsigned long long>(j.n);
        j.deg = arena->take<uint32_t>(j.n);
        j.sums = arena->take<unsigned long long>(kMotifSums);
        j.tdv = j.kind == KHZ_KGPI_HOUSE ? arena->take<uint32_t>(std::max<uint64_t>(2 * j.om, 1)) : nullptr;
        if (!j.tri || !j.acc || !j.deg || !j.sums || (j.kind == KHZ_KGPI_HOUSE && !j.tdv)) {
            set_error("motif launch arena too small");
            return KHZ_ERR_OOM;
        }
    }
    L.queue = arena->take<unsigned long long>(jobs.size());
    if (!L.queue) {
        set_error("motif launch arena too small");
        return KHZ_ERR_OOM;
    }
    L.n_jobs = (int)jobs.size();
    L.jobs = jobs;
    int dev = 0;
    KHZ_CUDA(cudaGetDevice(&dev));
    KHZ_CUDA(cudaDeviceGetAttribute(&L.sms, cudaDevAttrMultiProcessorCount, dev));
    *ml = L;
    (void)s;
    return KHZ_OK;
}

khz_status motif_enqueue_sums(const MotifLaunch &L, cudaStream_t s, LaunchStats *ls) {
    if (L.n_jobs == 0) return KHZ_OK;
    KHZ_CUDA(cudaMemsetAsync(L.queue, 0, sizeof(unsigned long long) * L.n_jobs, s));
    for (int i = 0; i < L.n_jobs; ++i) {
        const MotifJob &J = L.jobs[i];
        KHZ_CUDA(cudaMemsetAsync(J.tri, 0, sizeof(uint32_t) * std::max<uint64_t>(J.om, 1), s));
        KHZ_CUDA(cudaMemsetAsync(J.acc, 0, sizeof(unsigned long long) * std::max<uint32_t>(J.n, 1), s));
        KHZ_CUDA(cudaMemsetAsync(J.deg, 0, sizeof(uint32_t) * std::max<uint32_t>(J.n, 1), s));
        KHZ_CUDA(cudaMemsetAsync(J.sums, 0, sizeof(unsigned long long) * kMotifSums, s));
        const int wgrid = (int)std::max<uint64_t>(1, std::min<uint64_t>(((uint64_t)J.n + 7) / 8, (uint64_t)L.sms * 16));
        const int vgrid = (int)std::max<uint64_t>(1, std::min<uint64_t>(((uint64_t)J.n + 255) / 256, (uint64_t)L.sms * 8));
        motif_tri_kernel<<<wgrid, 256, 0, s>>>(J, L.queue + i);
        motif_edge_kernel<<<wgrid, 256, 0, s>>>(J);
        if (J.kind == KHZ_KGPI_HOUSE) {
            motif_house_entries_kernel<<<wgrid, 256, 0, s>>>(J);
            motif_house_depth2_kernel<<<vgrid, 256, 0, s>>>(J);
        } else {
            motif_vertex_kernel<<<vgrid, 256, 0, s>>>(J);
            if (J.kind == KHZ_KAUTO_4MOTIF) motif_path_kernel<<<wgrid, 256, 0, s>>>(J);
        }
        KHZ_CUDA(cudaGetLastError());
        if (ls) ls->launches += J.kind == KHZ_KGPI_TAILED_TRIANGLE ? 3 : 4;
    }
    return KHZ_OK;
}

khz_status motif_enqueue_combine(const MotifLaunch &L, uint64_t *d_rows, cudaStream_t s, LaunchStats *ls) {
    for (int i = 0; i < L.n_jobs; ++i) {
        motif_combine_kernel<<<1, 32, 0, s>>>(L.jobs[i], d_rows);
        KHZ_CUDA(cudaGetLastError());
        if (ls) ls->launches += 1;
    }
    return KHZ_OK;
}

}  // namespace khz
