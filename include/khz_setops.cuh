// Warp-cooperative sorted-set algebra on uint32 vertex lists (the device form of
// VertexSet, vertex_set.cc:20-184, and the trims of utilities.h:64-86).
//
// Every function here is called by all 32 lanes of a warp with identical arguments
// and returns the same value in every lane.  Lists are sorted strictly increasing.
// The merge loops of the reference are replaced by a probe scheme: each lane takes
// one element of the probe list (32 consecutive elements per step, one coalesced
// 128-byte load) and binary-searches it in the other list; the search window of the
// next step starts where the previous step's last lane stopped, so a step costs
// O(log(window)) dependent loads per lane.  Results are compacted in order with a
// ballot + popc prefix, so materialised outputs stay sorted.
#pragma once
#include <stdint.h>

namespace khz {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

// number of elements < x in a[0, n)  (std::lower_bound position)
__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t *__restrict__ a, uint32_t lo, uint32_t n,
                                                    uint32_t x) {
    uint32_t l = lo, r = n;
    while (l < r) {
        uint32_t m = (l + r) >> 1;
        if (__ldg(a + m) < x) l = m + 1; else r = m;
    }
    return l;
}
// number of elements <= x in a[0, n)  (std::upper_bound position)
__device__ __forceinline__ uint32_t upper_bound_u32(const uint32_t *__restrict__ a, uint32_t lo, uint32_t n,
                                                    uint32_t x) {
    uint32_t l = lo, r = n;
    while (l < r) {
        uint32_t m = (l + r) >> 1;
        if (__ldg(a + m) <= x) l = m + 1; else r = m;
    }
    return l;
}
// same on a generic (possibly shared or freshly written) pointer, without the read-only path
__device__ __forceinline__ uint32_t upper_bound_plain(const uint32_t *a, uint32_t lo, uint32_t n, uint32_t x) {
    uint32_t l = lo, r = n;
    while (l < r) {
        uint32_t m = (l + r) >> 1;
        if (a[m] <= x) l = m + 1; else r = m;
    }
    return l;
}
__device__ __forceinline__ uint32_t lower_bound_plain(const uint32_t *a, uint32_t lo, uint32_t n, uint32_t x) {
    uint32_t l = lo, r = n;
    while (l < r) {
        uint32_t m = (l + r) >> 1;
        if (a[m] < x) l = m + 1; else r = m;
    }
    return l;
}

// Filter applied to the members of a result: x > lb (when has_lb) and x not in ne[0..nne).
struct Filter {
    uint32_t lb;
    int has_lb;
    int nne;
    uint32_t ne[4];
    __device__ __forceinline__ bool pass(uint32_t x) const {
        bool ok = !has_lb || x > lb;
#pragma unroll
        for (int i = 0; i < 4; ++i) ok = ok && (i >= nne || x != ne[i]);
        return ok;
    }
};

// Result of a probe pass
struct ProbeResult {
    uint32_t full;      // |A op B| (unfiltered)
    uint32_t filtered;  // members passing the filter
};

// A op B with op = intersect (SUB = false) or subtract (SUB = true).
// P is the probe list, Q the searched list.  For intersection the caller passes the
// smaller list as P; for subtraction P = A and Q = B.  When out != nullptr the full
// result is written (sorted).  Sets are read through the generic path because the
// probe list may be a warp's own freshly materialised prefix.
template <bool SUB>
__device__ ProbeResult warp_probe(const uint32_t *P, uint32_t np, const uint32_t *Q, uint32_t nq, uint32_t *out,
                                  const Filter &f) {
    const unsigned lane = lane_id();
    uint32_t lo = 0, written = 0, filtered = 0;
    for (uint32_t base = 0; base < np; base += 32) {
        const uint32_t idx = base + lane;
        const bool valid = idx < np;
        const uint32_t x = valid ? P[idx] : 0xffffffffu;
        uint32_t pos = nq;
        if (valid) pos = lower_bound_plain(Q, lo, nq, x);
        const bool found = valid && pos < nq && Q[pos] == x;
        const bool keep = SUB ? (valid && !found) : found;
        const unsigned bal = __ballot_sync(kFull, keep);
        if (out != nullptr && keep) out[written + __popc(bal & ((1u << lane) - 1u))] = x;
        written += __popc(bal);
        filtered += __popc(__ballot_sync(kFull, keep && f.pass(x)));
        // next window starts at the last valid lane's position
        const uint32_t last = (np - base) >= 32 ? 31u : (np - base - 1);
        lo = __shfl_sync(kFull, pos, last);
        if (lo >= nq && !SUB) break;  // nothing left to intersect with
        if (lo >= nq && SUB) {
            // the rest of P survives the subtraction unchanged
            const uint32_t rest_begin = base + 32;
            for (uint32_t b2 = rest_begin; b2 < np; b2 += 32) {
                const uint32_t i2 = b2 + lane;
                const bool v2 = i2 < np;
                const uint32_t y = v2 ? P[i2] : 0;
                const unsigned b = __ballot_sync(kFull, v2);
                if (out != nullptr && v2) out[written + __popc(b & ((1u << lane) - 1u))] = y;
                written += __popc(b);
                filtered += __popc(__ballot_sync(kFull, v2 && f.pass(y)));
            }
            break;
        }
    }
    return {written, filtered};
}

// |{x in a[0,n) : filter}| for a plain sorted list (no set op): lower-bound trim + exclusions
// (the kgraphpi last level, kgraphpi/three_motif.cc:151-158).
__device__ __forceinline__ uint32_t warp_count_plain(const uint32_t *a, uint32_t n, const Filter &f) {
    uint32_t start = f.has_lb ? upper_bound_plain(a, 0, n, f.lb) : 0;
    uint32_t c = n - start;
    for (int i = 0; i < f.nne; ++i) {
        const uint32_t x = f.ne[i];
        bool dup = false;
        for (int j = 0; j < i; ++j) dup = dup || f.ne[j] == x;
        if (dup || (f.has_lb && x <= f.lb)) continue;
        const uint32_t p = lower_bound_plain(a, start, n, x);
        c -= (p < n && a[p] == x) ? 1u : 0u;
    }
    return c;
}

}  // namespace khz
