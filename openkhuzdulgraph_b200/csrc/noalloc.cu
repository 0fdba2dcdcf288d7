// Counting without any device allocation.
//
// Some callers cannot call cudaMalloc: code that runs inside a host framework which owns
// all device memory through its own pool and forbids side allocations, or a plugin loaded
// into a process whose allocator is locked down.  For them, khz_count_noalloc runs the per-warp
// DFS engine with all of its scratch (work-queue head, raw counters, job and schedule
// tables, per-warp materialised prefixes) in one file-scope device array of fixed size.
// The caller still provides the graph (device CSR) and the output buffer.
//
// The array is part of the library's device image: every GPU that loads the library holds
// it (kNoAllocBytes = 14,557,184 bytes, about 13.9 MiB) until the process exits.  Its size fixes the limits:
// at most kNoAllocWarps resident warps, and no vertex of degree above kNoAllocMaxDegree.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "khz_internal.cuh"

namespace khz {
namespace {

constexpr uint32_t kNoAllocWarps = 592;        // 148 SMs x 4 warps
constexpr uint32_t kNoAllocMaxDegree = 1024;   // slot capacity: largest vertex degree served
constexpr size_t kHeaderBytes = 8192;
constexpr size_t kSlotBytes = (size_t)kNoAllocWarps * kNumSlots * kNoAllocMaxDegree * sizeof(uint32_t);
constexpr size_t kNoAllocBytes = kHeaderBytes + kSlotBytes;
// header layout (bytes)
constexpr size_t kOffQueue = 0;      // unsigned long long work-queue head
constexpr size_t kOffMaxDeg = 8;     // unsigned int max degree of the caller's graph
constexpr size_t kOffBad = 12;       // unsigned int: raw count not divisible by the multiplicity
constexpr size_t kOffRaw = 64;       // KHZ_MAX_COUNTS + 2 raw counters
constexpr size_t kOffJobs = 256;     // up to 6 DfsJob
constexpr size_t kOffPlans = 1024;   // up to 6 Plan (the kernel reads 4 Plans' worth at least)
static_assert(kOffJobs + 6 * sizeof(DfsJob) <= kOffPlans, "job table overlaps the plan table");
static_assert(kOffPlans + 6 * sizeof(Plan) <= kHeaderBytes, "plan table overlaps the slots");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char *g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device.  The first call on each device
// resolves it with cudaGetSymbolAddress (with that device current) and caches it.
khz_status scratch_address(int dev, unsigned char **out) {
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("device %d beyond the no-allocation table (%d devices)", dev, kMaxDevices);
        return KHZ_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-allocation scratch)");
        g_scratch_ptr[dev] = (unsigned char *)p;
    }
    *out = g_scratch_ptr[dev];
    return KHZ_OK;
}

__global__ void noalloc_max_degree_kernel(const uint64_t *__restrict__ off, uint32_t n, unsigned int *out) {
    unsigned int best = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        best = max(best, (unsigned int)(off[v + 1] - off[v]));
    for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_down_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, best);
}

struct Mult {
    uint32_t m[KHZ_MAX_COUNTS];
};

__global__ void noalloc_finalize_kernel(const uint64_t *raw, Mult mult, uint64_t ext_add, uint64_t *out,
                                        unsigned int *bad) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int c = 0; c < KHZ_MAX_COUNTS; ++c) {
        const uint64_t v = raw[c];
        const uint32_t mu = mult.m[c];
        if (mu > 1 && v % mu) *bad = 1u;
        out[c] = mu > 1 ? v / mu : v;
    }
    out[KHZ_MAX_COUNTS] = raw[KHZ_MAX_COUNTS] + ext_add;
    out[KHZ_MAX_COUNTS + 1] = raw[KHZ_MAX_COUNTS + 1];
}

}  // namespace
}  // namespace khz

using namespace khz;

extern "C" khz_status khz_count_noalloc(const uint64_t *d_offsets, const uint32_t *d_adj, uint32_t n,
                                        uint64_t num_entries, khz_app_id app, uint64_t *d_out, void *stream) {
    if (app < 0 || app >= KHZ_NUM_APPS) {
        set_error("invalid app id %d", (int)app);
        return KHZ_ERR_ARG;
    }
    if (!d_out || !d_offsets || (num_entries > 0 && !d_adj)) {
        set_error("null graph or output pointer");
        return KHZ_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    int dev = 0;
    KHZ_CUDA(cudaGetDevice(&dev));
    unsigned char *base = nullptr;
    khz_status st = scratch_address(dev, &base);
    if (st) return st;
    unsigned long long *queue = (unsigned long long *)(base + kOffQueue);
    unsigned int *d_maxdeg = (unsigned int *)(base + kOffMaxDeg);
    unsigned int *d_bad = (unsigned int *)(base + kOffBad);
    uint64_t *d_raw = (uint64_t *)(base + kOffRaw);
    DfsJob *d_jobs = (DfsJob *)(base + kOffJobs);
    Plan *d_plans = (Plan *)(base + kOffPlans);
    uint32_t *slots = (uint32_t *)(base + kHeaderBytes);

    // the array keeps the previous call's contents: clear everything that must start at zero
    KHZ_CUDA(cudaMemsetAsync(base, 0, kOffJobs, s));
    int sms = 0;
    KHZ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (n > 0) {
        const int blocks = (int)std::min<uint64_t>(((uint64_t)n + 255) / 256, (uint64_t)sms * 8);
        noalloc_max_degree_kernel<<<blocks, 256, 0, s>>>(d_offsets, n, d_maxdeg);
        KHZ_CUDA(cudaGetLastError());
    }
    unsigned int maxdeg = 0;
    KHZ_CUDA(cudaMemcpyAsync(&maxdeg, d_maxdeg, sizeof(maxdeg), cudaMemcpyDeviceToHost, s));
    KHZ_CUDA(cudaStreamSynchronize(s));
    if (maxdeg > kNoAllocMaxDegree) {
        set_error("vertex degree %u exceeds the no-allocation limit of %u; use khz_count", maxdeg,
                  kNoAllocMaxDegree);
        return KHZ_ERR_ARG;
    }

    const AppDef &def = app_def(app);
    DfsJob jobs[6];
    Plan plans[6];
    for (int r = 0; r < def.num_runs; ++r) {
        DfsJob j{};
        j.off = d_offsets;
        j.adj = d_adj;
        j.n = n;
        j.plan_idx = (uint32_t)r;
        j.unit_begin = (uint64_t)r * num_entries;
        j.num_units = num_entries;
        j.out_base = 0;
        j.min_deg = 0;
        jobs[r] = j;
        plans[r] = def.plans[r];
    }
    KHZ_CUDA(cudaMemcpyAsync(d_jobs, jobs, sizeof(DfsJob) * def.num_runs, cudaMemcpyHostToDevice, s));
    KHZ_CUDA(cudaMemcpyAsync(d_plans, plans, sizeof(Plan) * def.num_runs, cudaMemcpyHostToDevice, s));
    const uint64_t total_units = (uint64_t)def.num_runs * num_entries;
    const int blocks = (int)std::min<uint32_t>((uint32_t)sms, kNoAllocWarps / 4);
    st = dfs_launch_prealloc(d_jobs, def.num_runs, d_plans, total_units, 8, slots, kNoAllocMaxDegree, queue, d_raw,
                             blocks, 128, s);
    if (st) return st;
    Mult mult;
    for (int c = 0; c < KHZ_MAX_COUNTS; ++c) mult.m[c] = c < def.num_counts ? def.mult[c] : 1;
    noalloc_finalize_kernel<<<1, 32, 0, s>>>(d_raw, mult, (uint64_t)n * def.num_runs, d_out, d_bad);
    KHZ_CUDA(cudaGetLastError());
    unsigned int bad = 0;
    KHZ_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof(bad), cudaMemcpyDeviceToHost, s));
    KHZ_CUDA(cudaStreamSynchronize(s));
    if (bad) {
        set_error("raw count not divisible by the pattern multiplicity (input is not an undirected graph)");
        return KHZ_ERR_MULTIPLICITY;
    }
    return KHZ_OK;
}
