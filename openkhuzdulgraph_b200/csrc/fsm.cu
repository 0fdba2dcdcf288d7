// Frequent labelled subgraph mining (3-FSM) on the device: the kautomine three_fsm app
// (kautomine/three_fsm.cc:53-800) with its MNI support domains (SharedMemoryPatternDomain,
// engine.h:303-403).
//
// The host side mirrors the app's level-by-level driver: single-vertex patterns, then edges,
// wedges, triangles, four-chains and three-stars, each level's candidate labellings generated from
// the frequent patterns of the levels before it (three_fsm.cc:315-590), a candidate frequent when
// its support reaches the threshold.  A pattern's support is minimum-image based: for every
// pattern vertex, the number of distinct graph vertices it is mapped to over all embeddings; the
// support is the least of these (get_support, engine.h:384-401).
//
// Where the reference runs the engine once per candidate (run(..., restrict_starting_vertex_label,
// labels[0])), the device answers all of a level's candidates at once.  Edges: every embedding is
// enumerated once (a warp per v0); triangles: each is listed once, from its lowest vertex in
// (degree, id) order (a warp per (v0, v1) pair, lanes over v2), and its six vertex orders are the
// embeddings.  An embedding whose label tuple is a candidate (one lookup in a dense table indexed by
// the labels) sets its vertices' bits in that candidate's per-position domain bitmaps (a word is
// read before the atomicOr, so repeated images cost no atomics).  Wedges,
// four-chains and three-stars, whose embeddings are far more numerous: each (candidate, position,
// vertex) is decided by a search for one witness embedding over label counts of the neighbour lists
// (see below).  A
// popcount kernel then gives every (candidate, position) domain size.  Candidates whose bitmaps
// would not fit the memory budget at once are processed in groups.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <set>
#include <vector>

#include "khz_internal.cuh"
#include "khz_setops.cuh"

namespace khz {
namespace {

constexpr int kFsmMaxLabels = 48;  // MAX_NUM_LABELS (graph_loader.h:28)

enum Template : int { kEdge = 0, kWedge = 1, kTriangle = 2, kFourChain = 3, kThreeStar = 4 };
constexpr int kPatSize[5] = {2, 3, 3, 4, 4};

struct FsmArgs {
    const uint64_t *off;
    const uint32_t *adj;
    const uint32_t *labels;
    uint32_t n;
    uint32_t L;             // number of labels
    const int32_t *table;   // L^size entries: candidate index of a label tuple (group-local), or -1
    uint32_t *domains;      // [candidate][position][words]
    uint32_t words;         // ceil(n / 32)
    uint64_t m;             // CSR entries (the (v0, v1) pairs)
    unsigned long long *queue;  // pair claims of one launch (zeroed before it)
};

__device__ __forceinline__ void mark(const FsmArgs &a, int cand, int pos, uint32_t v) {
    uint32_t *w = a.domains + ((size_t)cand * 4 + pos) * a.words + (v >> 5);
    const uint32_t bit = 1u << (v & 31);
    if (!(*(volatile uint32_t *)w & bit)) atomicOr(w, bit);
}

__device__ __forceinline__ void mark_all(const FsmArgs &a, int cand, int k, const uint32_t *v) {
    for (int p = 0; p < k; ++p) mark(a, cand, p, v[p]);
}

__device__ __forceinline__ bool contains(const uint32_t *list, uint32_t len, uint32_t x) {
    const uint32_t p = lower_bound_u32(list, 0, len, x);
    return p < len && __ldg(list + p) == x;
}

// The embeddings enumerated are exactly those the app's apply() inserts into its pattern domain
// with enable = true (three_fsm.cc:53-262):
//   edge        v1 in N(v0)
//   wedge       v1 in N(v0); v2 in N(v0), v2 != v1
//   triangle    v1 in N(v0); v2 in N(v0) n N(v1)
//   four-chain  v1 in N(v0); v2 in N(v0), v2 != v1; v3 in N(v1), v3 != v0, v3 != v2
//   three-star  v1 in N(v0); v2 in N(v1), v2 != v0; v3 in N(v1), v3 != v0, v3 != v2
// Edges and triangles are enumerated here (wedges, four-chains and three-stars by fsm_exist_kernel,
// under the same constraints).  The edge template takes one warp per v0; triangles one warp per
// (v0, v1) pair: pairs are CSR entries, claimed in chunks from a counter, so a hub's pairs spread
// over many warps.  All of it assumes the symmetric CSR of a simple graph (validated: no self-loops),
// which khz_fsm requires.

// (degree, id) order: each triangle is listed once, from its lowest-ranked vertex
__device__ __forceinline__ bool ranks_below(uint32_t da, uint32_t va, uint32_t db, uint32_t vb) {
    return da < db || (da == db && va < vb);
}

__device__ __forceinline__ void mark_tri(const FsmArgs &a, int cand, uint32_t x, uint32_t y, uint32_t z) {
    if (cand < 0) return;
    mark(a, cand, 0, x);
    mark(a, cand, 1, y);
    mark(a, cand, 2, z);
}

// the triangles {v0, v1, v2} with v0 < v1 < v2 in (degree, id) order; lanes take v2.  The app's
// enumeration reaches each triangle of a symmetric graph in all six vertex orders, so every order
// whose label tuple is a candidate is marked here.  Listing from the lowest-ranked vertex scans
// sum d(v0) d+(v0) entries, d+ the neighbours ranked above v0, instead of sum d(v0)^2.
template <int T>
__device__ __forceinline__ void fsm_pair(const FsmArgs &a, uint32_t v0, uint32_t v1) {
    static_assert(T == kTriangle, "wedges, four-chains and three-stars use fsm_exist_kernel");
    const unsigned lane = lane_id();
    const uint64_t b0 = a.off[v0], b1 = a.off[v1];
    const uint32_t d0 = (uint32_t)(a.off[v0 + 1] - b0);
    const uint32_t d1 = (uint32_t)(a.off[v1 + 1] - b1);
    if (!ranks_below(d0, v0, d1, v1)) return;
    const uint32_t L = a.L;
    const uint32_t l0 = __ldg(a.labels + v0);
    const uint32_t l1 = __ldg(a.labels + v1);
    const uint32_t *n0 = a.adj + b0;
    const uint32_t *n1 = a.adj + b1;
    for (uint32_t i = lane; i < d0; i += 32) {
        const uint32_t v2 = __ldg(n0 + i);
        const uint32_t d2 = (uint32_t)(a.off[v2 + 1] - a.off[v2]);
        if (!ranks_below(d1, v1, d2, v2)) continue;
        const uint32_t l2 = __ldg(a.labels + v2);
        const int c012 = a.table[(l0 * L + l1) * L + l2], c021 = a.table[(l0 * L + l2) * L + l1];
        const int c102 = a.table[(l1 * L + l0) * L + l2], c120 = a.table[(l1 * L + l2) * L + l0];
        const int c201 = a.table[(l2 * L + l0) * L + l1], c210 = a.table[(l2 * L + l1) * L + l0];
        if (c012 < 0 && c021 < 0 && c102 < 0 && c120 < 0 && c201 < 0 && c210 < 0) continue;
        if (!contains(n1, d1, v2)) continue;
        mark_tri(a, c012, v0, v1, v2);
        mark_tri(a, c021, v0, v2, v1);
        mark_tri(a, c102, v1, v0, v2);
        mark_tri(a, c120, v1, v2, v0);
        mark_tri(a, c201, v2, v0, v1);
        mark_tri(a, c210, v2, v1, v0);
    }
}

template <int T>
__global__ void __launch_bounds__(256) fsm_domain_kernel(FsmArgs a) {
    const unsigned lane = lane_id();
    if constexpr (T == kEdge) {
        const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
        const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
        for (uint32_t v0 = warp; v0 < a.n; v0 += nwarps) {
            const uint32_t l0 = __ldg(a.labels + v0);
            const uint32_t *n0 = a.adj + a.off[v0];
            const uint32_t d0 = (uint32_t)(a.off[v0 + 1] - a.off[v0]);
            for (uint32_t i = lane; i < d0; i += 32) {
                const uint32_t v1 = __ldg(n0 + i);
                const int c = a.table[l0 * a.L + __ldg(a.labels + v1)];
                if (c >= 0) {
                    const uint32_t v[2] = {v0, v1};
                    mark_all(a, c, 2, v);
                }
            }
        }
    } else {
        constexpr uint64_t kChunk = 8;
        while (true) {
            unsigned long long e0 = 0;
            if (lane == 0) e0 = atomicAdd(a.queue, (unsigned long long)kChunk);
            e0 = __shfl_sync(kFull, e0, 0);
            if (e0 >= a.m) break;
            const uint64_t e1 = min((uint64_t)a.m, (uint64_t)e0 + kChunk);
            // v0 of entry e0: the largest v with off[v] <= e0 (its list holds e0, as e0 < m)
            uint32_t lo = 0, hi = a.n;
            while (lo < hi) {
                const uint32_t mid = (lo + hi + 1) >> 1;
                if (a.off[mid] <= e0) lo = mid; else hi = mid - 1;
            }
            uint32_t v0 = lo;
            for (uint64_t e = e0; e < e1; ++e) {
                while (a.off[v0 + 1] <= e) ++v0;
                fsm_pair<T>(a, v0, __ldg(a.adj + e));
            }
        }
    }
}

// ---- wedge, four-chain and three-star domains by existence ------------------------------------
// Enumerating every four-chain or three-star costs sum d(v0)^2 d(v1) steps (22 s at R-MAT scale 16),
// every wedge sum d(v0)^2, while a domain only asks, per (candidate, position, vertex x), whether
// SOME embedding of the enumeration above puts x at that position.  With lc(v, l), the number of
// neighbours of v with label l, each such question needs at most one pass over a neighbour list (or
// two nested for the chain's outer positions) and stops at the first witness.  The answers are the
// same sets the enumeration marks, since the conditions below are exactly its constraints with the
// other vertices left free:
//   wedge v1 - v0 - v2 with labels (c0, c1, c2), all three distinct;
//   four-chain v2 - v0 - v1 - v3 with labels (c0, c1, c2, c3), all four distinct;
//   three-star: centre v1 (c1), leaves v0, v2, v3 (c0, c2, c3), all four distinct.

// lc: one warp per vertex, a label histogram per warp in shared memory
__global__ void __launch_bounds__(256) fsm_label_count_kernel(const uint64_t *__restrict__ off,
                                                             const uint32_t *__restrict__ adj,
                                                             const uint32_t *__restrict__ labels, uint32_t n,
                                                             uint32_t L, uint32_t *lc) {
    __shared__ uint32_t hist[8][kFsmMaxLabels];
    const unsigned lane = lane_id();
    const int wib = threadIdx.x >> 5;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t v = warp; v < n; v += nwarps) {
        for (uint32_t l = lane; l < L; l += 32) hist[wib][l] = 0;
        __syncwarp();
        for (uint64_t e = off[v] + lane; e < off[v + 1]; e += 32) atomicAdd(&hist[wib][__ldg(labels + __ldg(adj + e))], 1u);
        __syncwarp();
        for (uint32_t l = lane; l < L; l += 32) lc[(size_t)v * L + l] = hist[wib][l];
        __syncwarp();
    }
}

struct FsmExistArgs {
    const uint64_t *off;
    const uint32_t *adj;
    const uint32_t *labels;
    const uint32_t *lc;      // n x L
    uint32_t n;
    uint32_t L;
    const uint8_t *cands;    // per candidate of the group: its 4 labels in enumeration order
    uint32_t num_cands;
    uint32_t *domains;       // [candidate][position][words]
    uint32_t words;
    unsigned long long *queue;  // (candidate, vertex) claims, zeroed before the launch
};

__device__ __forceinline__ uint32_t lcount(const FsmExistArgs &a, uint32_t v, uint32_t l) {
    return __ldg(a.lc + (size_t)v * a.L + l);
}

// four-chain: does the pair (v0, v1) (labels c0, c1, adjacent) extend by v2 in N(v0) with label c2
// and v3 in N(v1) with label c3, all four distinct?  A and B count the choices left for v2 and v3;
// only when each has exactly one and the labels agree must the two be compared (found by scans).
__device__ bool chain_pair(const FsmExistArgs &a, uint32_t v0, uint32_t v1, uint32_t c0, uint32_t c1, uint32_t c2,
                           uint32_t c3) {
    const uint32_t A = lcount(a, v0, c2) - (c1 == c2 ? 1u : 0u);
    const uint32_t B = lcount(a, v1, c3) - (c0 == c3 ? 1u : 0u);
    if (A == 0 || B == 0) return false;
    if (A >= 2 || B >= 2 || c2 != c3) return true;
    uint32_t as = 0xffffffffu, bs = 0xffffffffu;
    for (uint64_t e = a.off[v0]; e < a.off[v0 + 1]; ++e) {
        const uint32_t u = __ldg(a.adj + e);
        if (u != v1 && __ldg(a.labels + u) == c2) {
            as = u;
            break;
        }
    }
    for (uint64_t e = a.off[v1]; e < a.off[v1 + 1]; ++e) {
        const uint32_t w = __ldg(a.adj + e);
        if (w != v0 && __ldg(a.labels + w) == c3) {
            bs = w;
            break;
        }
    }
    return as != bs;
}

__device__ __forceinline__ bool has_nbr(const FsmExistArgs &a, uint32_t v, uint32_t x) {
    const uint64_t b = a.off[v];
    const uint32_t d = (uint32_t)(a.off[v + 1] - b);
    const uint32_t p = lower_bound_u32(a.adj + b, 0, d, x);
    return p < d && __ldg(a.adj + b + p) == x;
}

// three-star: with the leaf labels still to place as a multiset (up to 3 labels), does y have
// enough neighbours of each label once `ex` (a neighbour of y with label lex, or none) is left out?
__device__ __forceinline__ bool star_fits(const FsmExistArgs &a, uint32_t y, const uint32_t *need, int k,
                                          int lex) {
    for (int i = 0; i < k; ++i) {
        uint32_t mult = 0;
        for (int j = 0; j < k; ++j) mult += need[j] == need[i] ? 1u : 0u;
        const uint32_t have = lcount(a, y, need[i]) - ((int)need[i] == lex ? 1u : 0u);
        if (have < mult) return false;
    }
    return true;
}

__device__ __forceinline__ void set_domain_bit(const FsmExistArgs &a, uint32_t c, int p, uint32_t x) {
    atomicOr(a.domains + ((size_t)c * 4 + p) * a.words + (x >> 5), 1u << (x & 31));
}

// The positions p of candidate c (labels c0..c3) that x, with label lx, could take: cl[p] == lx and
// x's own label counts allow the position (necessary conditions of the searches below, so a
// position dropped here has no witness).  The wedge centre and the three-star centre need only x's
// label counts and are decided here outright.
template <int T>
__device__ __forceinline__ unsigned open_positions(const FsmExistArgs &a, uint32_t c, uint32_t x, uint32_t lx,
                                                   uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3) {
    unsigned pm = 0;
    if (T == kWedge) {
        // centre v0: a c1 neighbour and another c2 one, decided here; ends v1 / v2: a c0 neighbour
        const uint32_t same = c1 == c2 ? 1u : 0u;
        if (c0 == lx && lcount(a, x, c1) >= 1 && lcount(a, x, c2) >= 1 + same) set_domain_bit(a, c, 0, x);
        if ((c1 == lx || c2 == lx) && lcount(a, x, c0) >= 1) {
            if (c1 == lx) pm |= 2;
            if (c2 == lx) pm |= 4;
        }
    } else if (T == kFourChain) {
        // v0: a c1 neighbour and another c2 one; v1: a c0 neighbour and another c3 one;
        // v2: a c0 neighbour; v3: a c1 neighbour
        if (c0 == lx && lcount(a, x, c1) >= 1 && lcount(a, x, c2) >= 1 + (c1 == c2 ? 1u : 0u)) pm |= 1;
        if (c1 == lx && lcount(a, x, c0) >= 1 && lcount(a, x, c3) >= 1 + (c0 == c3 ? 1u : 0u)) pm |= 2;
        if (c2 == lx && lcount(a, x, c0) >= 1) pm |= 4;
        if (c3 == lx && lcount(a, x, c1) >= 1) pm |= 8;
    } else {
        if (c1 == lx) {
            const uint32_t need[3] = {c0, c2, c3};
            if (star_fits(a, x, need, 3, -1)) set_domain_bit(a, c, 1, x);
        }
        // a leaf needs a neighbour with the centre's label
        if ((c0 == lx || c2 == lx || c3 == lx) && lcount(a, x, c1) >= 1) {
            if (c0 == lx) pm |= 1;
            if (c2 == lx) pm |= 4;
            if (c3 == lx) pm |= 8;
        }
    }
    return pm;
}

// A warp claims 32 consecutive (candidate, vertex x) tasks at a time; each lane screens one of them
// (open_positions), and the warp then searches a witness embedding for every position left open,
// lane 0 setting x's domain bit when one is found.
template <int T>
__global__ void __launch_bounds__(256) fsm_exist_kernel(FsmExistArgs a) {
    const unsigned lane = lane_id();
    const uint64_t tasks = (uint64_t)a.num_cands * a.n;
    while (true) {
        unsigned long long t0 = 0;
        if (lane == 0) t0 = atomicAdd(a.queue, 32ull);
        t0 = __shfl_sync(kFull, t0, 0);
        if (t0 >= tasks) break;
        const uint64_t t = t0 + lane;
        uint32_t tc = 0, tx = 0;
        unsigned tpm = 0;
        if (t < tasks) {
            tc = (uint32_t)(t / a.n);
            tx = (uint32_t)(t % a.n);
            const uint8_t *cl = a.cands + (size_t)tc * 4;
            tpm = open_positions<T>(a, tc, tx, __ldg(a.labels + tx), cl[0], cl[1], cl[2], cl[3]);
        }
        for (unsigned todo = __ballot_sync(kFull, tpm != 0); todo; todo &= todo - 1) {
            const int src = __ffs(todo) - 1;
            const uint32_t c = __shfl_sync(kFull, tc, src), x = __shfl_sync(kFull, tx, src);
            const unsigned pm = __shfl_sync(kFull, tpm, src);
            const uint8_t *cl = a.cands + (size_t)c * 4;
            const uint32_t c0 = cl[0], c1 = cl[1], c2 = cl[2], c3 = cl[3];
            const uint32_t lx = __ldg(a.labels + x);
            const uint64_t bx = a.off[x], ex = a.off[x + 1];
            for (int p = 0; p < 4; ++p) {
                if (!(pm >> p & 1)) continue;
                bool found = false;
                if (T == kWedge) {
                    // x is end p: a centre y in N(x) with label c0 and a neighbour of the other end's
                    // label other than x
                    const uint32_t lend = p == 1 ? c2 : c1;
                    const uint32_t end_min = 1u + (c1 == c2 ? 1u : 0u);
                    for (uint64_t e0 = bx; e0 < ex && !found; e0 += 32) {
                        bool hit = false;
                        const uint64_t e = e0 + lane;
                        if (e < ex) {
                            const uint32_t y = __ldg(a.adj + e);
                            hit = __ldg(a.labels + y) == c0 && lcount(a, y, lend) >= end_min;
                        }
                        found = __any_sync(kFull, hit);
                    }
                } else if (T == kThreeStar) {
                    // x is leaf p: a centre y in N(x) with label c1 that still has the other two leaves
                    const uint32_t need[2] = {p == 0 ? c2 : c0, p == 3 ? c2 : c3};
                    for (uint64_t e0 = bx; e0 < ex && !found; e0 += 32) {
                        bool hit = false;
                        const uint64_t e = e0 + lane;
                        if (e < ex) {
                            const uint32_t y = __ldg(a.adj + e);
                            hit = __ldg(a.labels + y) == c1 && star_fits(a, y, need, 2, (int)lx);
                        }
                        found = __any_sync(kFull, hit);
                    }
                } else if (p <= 1) {
                    // four-chain, x = v0 (p = 0) or v1 (p = 1): a partner in N(x) completing the pair
                    const uint32_t want = p == 0 ? c1 : c0;
                    for (uint64_t e0 = bx; e0 < ex && !found; e0 += 32) {
                        bool hit = false;
                        const uint64_t e = e0 + lane;
                        if (e < ex) {
                            const uint32_t y = __ldg(a.adj + e);
                            if (__ldg(a.labels + y) == want)
                                hit = p == 0 ? chain_pair(a, x, y, c0, c1, c2, c3) : chain_pair(a, y, x, c0, c1, c2, c3);
                        }
                        found = __any_sync(kFull, hit);
                    }
                } else {
                    // four-chain, x = v2 (p = 2): v0 in N(x) (c0), v1 in N(v0) \ {x} (c1), and v1 keeps a
                    // neighbour of label c3 other than v0 and x; x = v3 (p = 3) is the mirror image
                    // (v1 in N(x) (c1), v0 in N(v1) \ {x} (c0), v0 keeps a c2 neighbour other than v1, x).
                    // The middle vertices m are screened 32 at a time: label lmid and an lfar neighbour
                    // other than x.
                    const uint32_t lmid = p == 2 ? c0 : c1, lfar = p == 2 ? c1 : c0, lend = p == 2 ? c3 : c2;
                    const uint32_t lmid_in_end = lmid == lend ? 1u : 0u;
                    const uint32_t far_min = 1u + (lx == lfar ? 1u : 0u);
                    for (uint64_t g0 = bx; g0 < ex && !found; g0 += 32) {
                        uint32_t mm = 0;
                        bool ok = false;
                        if (g0 + lane < ex) {
                            mm = __ldg(a.adj + g0 + lane);
                            ok = __ldg(a.labels + mm) == lmid && lcount(a, mm, lfar) >= far_min;
                        }
                        for (unsigned mids = __ballot_sync(kFull, ok); mids && !found; mids &= mids - 1) {
                            const uint32_t m = __shfl_sync(kFull, mm, __ffs(mids) - 1);  // v0 (p = 2) or v1 (p = 3)
                            const uint64_t bm = a.off[m], em = a.off[m + 1];
                            for (uint64_t e0 = bm; e0 < em && !found; e0 += 32) {
                                bool hit = false;
                                const uint64_t e = e0 + lane;
                                if (e < em) {
                                    const uint32_t f = __ldg(a.adj + e);  // v1 (p = 2) or v0 (p = 3)
                                    if (f != x && __ldg(a.labels + f) == lfar) {
                                        const uint32_t k = lcount(a, f, lend) - lmid_in_end;
                                        hit = k >= 2 || (k == 1 && (lx != lend || !has_nbr(a, f, x)));
                                    }
                                }
                                found = __any_sync(kFull, hit);
                            }
                        }
                    }
                }
                if (found && lane == 0) set_domain_bit(a, c, p, x);
            }
        }
    }
}

// sizes of the domains: one block per (candidate, position)
__global__ void fsm_popcount_kernel(const uint32_t *domains, uint32_t words, int k, uint32_t *sizes) {
    const uint32_t *d = domains + ((size_t)(blockIdx.x / k) * 4 + blockIdx.x % k) * words;
    uint32_t s = 0;
    for (uint32_t w = threadIdx.x; w < words; w += blockDim.x) s += __popc(d[w]);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(kFull, s, o);
    __shared__ uint32_t part[32];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(kFull, s, o);
        if (threadIdx.x == 0) sizes[blockIdx.x] = s;
    }
}

using Labels = std::vector<uint32_t>;

struct Candidate {
    Labels canonical;
    std::vector<Labels> automorphisms;  // non-canonical labellings of the same pattern
};

// ---- candidate generation, following three_fsm.cc:315-590 -------------------------------------
struct Frequent {
    std::vector<bool> vertex;
    std::set<Labels> edge, wedge, triangle, chain, star;
};

std::vector<Candidate> candidates_of(int t, uint32_t L, const Frequent &f) {
    std::vector<Candidate> out;
    auto fe = [&](uint32_t a, uint32_t b) { return f.edge.count({a, b}) > 0; };
    auto fw = [&](uint32_t a, uint32_t b, uint32_t c) { return f.wedge.count({a, b, c}) > 0; };
    for (uint32_t l0 = 0; l0 < L; ++l0) {
        if (!f.vertex[l0]) continue;
        for (uint32_t l1 = 0; l1 < L; ++l1) {
            if (t == kEdge) {
                if (f.vertex[l1] && l0 <= l1) out.push_back({{l0, l1}, {{l1, l0}}});
                continue;
            }
            if (!fe(l0, l1)) continue;
            for (uint32_t l2 = 0; l2 < L; ++l2) {
                if (t == kWedge) {
                    if (fe(l0, l2) && l1 <= l2) out.push_back({{l0, l1, l2}, {{l0, l2, l1}}});
                    continue;
                }
                if (!fw(l0, l1, l2)) continue;
                if (t == kTriangle) {
                    if (fw(l1, l0, l2) && fw(l2, l0, l1) && l0 <= l1 && l1 <= l2)
                        out.push_back({{l0, l1, l2},
                                       {{l0, l2, l1}, {l1, l0, l2}, {l1, l2, l0}, {l2, l0, l1}, {l2, l1, l0}}});
                    continue;
                }
                for (uint32_t l3 = 0; l3 < L; ++l3) {
                    if (t == kFourChain) {
                        if (fw(l1, l0, l3) && fe(l0, l2) && fe(l1, l3) && l0 <= l1)
                            out.push_back({{l0, l1, l2, l3}, {}});
                    } else {  // three-star centred at l0: the canonical labelling puts the centre second
                        if (fw(l0, l2, l3) && fw(l0, l1, l3) && l1 <= l2 && l2 <= l3)
                            out.push_back({{l1, l0, l2, l3}, {}});
                    }
                }
            }
        }
    }
    return out;
}

}  // namespace
}  // namespace khz

using namespace khz;

extern "C" khz_status khz_fsm(khz_ctx *ctx, khz_graph g, uint32_t threshold, khz_fsm_result *out,
                              khz_fsm_pattern *patterns, uint32_t capacity, uint32_t *num_patterns) {
    if (!out) {
        set_error("null result");
        return KHZ_ERR_ARG;
    }
    khz_graph_info gi;
    khz_status st = khz_graph_info_get(ctx, g, &gi);
    if (st) return st;
    if (!gi.d_labels || gi.num_labels == 0) {
        set_error("3-FSM needs a graph with node labels");
        return KHZ_ERR_ARG;
    }
    if (!gi.symmetric) {
        set_error("3-FSM needs the symmetric (undirected) CSR of a validated graph");
        return KHZ_ERR_ARG;
    }
    if (gi.num_labels > (uint32_t)kFsmMaxLabels) {
        set_error("3-FSM supports at most %d labels (the graph has %u)", kFsmMaxLabels, gi.num_labels);
        return KHZ_ERR_ARG;
    }
    const auto t0 = std::chrono::steady_clock::now();
    const uint32_t n = gi.num_vertices, L = gi.num_labels;
    memset(out, 0, sizeof(*out));
    if (num_patterns) *num_patterns = 0;
    auto emit = [&](int level, const Labels &lab, uint32_t support) {
        if (!patterns || !num_patterns) return;
        if (*num_patterns < capacity) {
            khz_fsm_pattern &p = patterns[*num_patterns];
            memset(&p, 0, sizeof(p));
            p.level = level;
            p.size = (uint32_t)lab.size();
            for (size_t i = 0; i < lab.size(); ++i) p.labels[i] = lab[i];
            p.support = support;
        }
        *num_patterns += 1;
    };
    // level 0: single vertices (setup, three_fsm.cc:289-310): the support sum counts every label
    std::vector<uint32_t> h_labels(n);
    KHZ_CUDA(cudaMemcpy(h_labels.data(), gi.d_labels, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost));
    std::vector<uint64_t> per_label(L, 0);
    for (uint32_t v = 0; v < n; ++v) per_label[h_labels[v]] += 1;
    Frequent f;
    f.vertex.assign(L, false);
    for (uint32_t l = 0; l < L; ++l) {
        f.vertex[l] = per_label[l] >= threshold;
        out->level[0].num_candidates += 1;
        out->level[0].num_frequent += f.vertex[l] ? 1 : 0;
        out->level[0].support_sum += per_label[l];
        if (f.vertex[l]) emit(0, {l}, (uint32_t)per_label[l]);
    }
    // device buffers: the label-tuple table of the edge and triangle levels (L^3 entries) and the
    // domains (grouped by budget)
    const size_t tsize = (size_t)L * L * L;
    const uint32_t words = (n + 31) / 32;
    size_t free_b = 0, total_b = 0;
    KHZ_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t budget = std::max<size_t>(free_b / 4, (size_t)64 << 20);
    const size_t per_cand = (size_t)4 * words * sizeof(uint32_t);
    // no level has more than L^4 candidates, so a larger buffer would only cost allocation time
    const size_t group_max = std::max<size_t>(1, std::min(budget / per_cand, tsize * L));
    int32_t *d_table = nullptr;
    uint32_t *d_dom = nullptr, *d_sizes = nullptr, *d_lc = nullptr;
    uint8_t *d_cands = nullptr;
    unsigned long long *d_queue = nullptr;
    auto release = [&]() {
        cudaFree(d_table);
        cudaFree(d_dom);
        cudaFree(d_sizes);
        cudaFree(d_queue);
        cudaFree(d_lc);
        cudaFree(d_cands);
    };
    cudaError_t e = cudaMalloc(&d_table, sizeof(int32_t) * tsize);
    if (e == cudaSuccess) e = cudaMalloc(&d_dom, per_cand * group_max);
    if (e == cudaSuccess) e = cudaMalloc(&d_sizes, sizeof(uint32_t) * 4 * group_max);
    if (e == cudaSuccess) e = cudaMalloc(&d_queue, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&d_lc, sizeof(uint32_t) * std::max<size_t>((size_t)n * L, 1));
    if (e == cudaSuccess) e = cudaMalloc(&d_cands, 4 * group_max);
    if (e != cudaSuccess) {
        cudaGetLastError();
        release();
        set_error("3-FSM device buffers: %s", cudaGetErrorString(e));
        return KHZ_ERR_OOM;
    }
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>(((uint64_t)n + 7) / 8, (uint64_t)sms * 16));
    // the label histogram of every neighbour list (the wedge, four-chain and three-star levels)
    if (n > 0) fsm_label_count_kernel<<<grid, 256>>>(gi.d_offsets, gi.d_adj, gi.d_labels, n, L, d_lc);
    std::vector<int32_t> table(tsize);
    std::vector<uint8_t> cand_labels(4 * group_max);
    for (int t = kEdge; t <= kThreeStar; ++t) {
        const std::vector<Candidate> cands = candidates_of(t, L, f);
        const int k = kPatSize[t];
        khz_fsm_level &lv = out->level[1 + t];
        lv.num_candidates = (uint32_t)cands.size();
        std::set<Labels> *freq = t == kEdge       ? &f.edge
                                 : t == kWedge    ? &f.wedge
                                 : t == kTriangle ? &f.triangle
                                 : t == kFourChain ? &f.chain
                                                   : &f.star;
        for (size_t g0 = 0; g0 < cands.size(); g0 += group_max) {
            const size_t gn = std::min(group_max, cands.size() - g0);
            // edges and triangles look label tuples up in the dense table; the witness searches read
            // the candidates' labels directly
            const bool enumerated = t == kEdge || t == kTriangle;
            size_t tn = 1;
            for (int p = 0; p < k; ++p) tn *= L;
            st = KHZ_OK;
            if (enumerated) {
                std::fill(table.begin(), table.begin() + tn, -1);
                for (size_t c = 0; c < gn; ++c) {
                    const Labels &lab = cands[g0 + c].canonical;
                    size_t idx = 0;
                    for (int p = 0; p < k; ++p) idx = idx * L + lab[p];
                    table[idx] = (int32_t)c;
                }
                if (cudaMemcpy(d_table, table.data(), sizeof(int32_t) * tn, cudaMemcpyHostToDevice) != cudaSuccess) {
                    release();
                    return cuda_fail(cudaGetLastError(), "3-FSM tables");
                }
            } else {
                for (size_t c = 0; c < gn; ++c)
                    for (int p = 0; p < 4; ++p)
                        cand_labels[4 * c + p] = p < k ? (uint8_t)cands[g0 + c].canonical[p] : (uint8_t)0;
                if (cudaMemcpy(d_cands, cand_labels.data(), 4 * gn, cudaMemcpyHostToDevice) != cudaSuccess) {
                    release();
                    return cuda_fail(cudaGetLastError(), "3-FSM candidates");
                }
            }
            if (cudaMemset(d_dom, 0, per_cand * gn) != cudaSuccess ||
                cudaMemset(d_queue, 0, sizeof(unsigned long long)) != cudaSuccess) {
                release();
                return cuda_fail(cudaGetLastError(), "3-FSM domains and claim counter");
            }
            FsmArgs a{gi.d_offsets, gi.d_adj, gi.d_labels, n, L, d_table, d_dom, words, gi.num_entries, d_queue};
            FsmExistArgs x{gi.d_offsets, gi.d_adj, gi.d_labels, d_lc, n, L, d_cands, (uint32_t)gn, d_dom, words, d_queue};
            const int xgrid = sms * 8;
            switch (t) {
                case kEdge: fsm_domain_kernel<kEdge><<<grid, 256>>>(a); break;
                case kWedge: fsm_exist_kernel<kWedge><<<xgrid, 256>>>(x); break;
                case kTriangle: fsm_domain_kernel<kTriangle><<<grid, 256>>>(a); break;
                case kFourChain: fsm_exist_kernel<kFourChain><<<xgrid, 256>>>(x); break;
                default: fsm_exist_kernel<kThreeStar><<<xgrid, 256>>>(x); break;
            }
            fsm_popcount_kernel<<<(unsigned)(gn * k), 256>>>(d_dom, words, k, d_sizes);
            std::vector<uint32_t> sizes(gn * k);
            e = cudaMemcpy(sizes.data(), d_sizes, sizeof(uint32_t) * gn * k, cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) {
                release();
                return cuda_fail(e, "3-FSM domains");
            }
            for (size_t c = 0; c < gn; ++c) {
                uint32_t support = n;  // get_support starts from the vertex count (engine.h:385)
                for (int p = 0; p < k; ++p) support = std::min(support, sizes[c * k + p]);
                if (support >= threshold) {
                    const Candidate &cd = cands[g0 + c];
                    freq->insert(cd.canonical);
                    for (const Labels &aut : cd.automorphisms) freq->insert(aut);
                    lv.num_frequent += 1;
                    lv.support_sum += support;
                    emit(1 + t, cd.canonical, support);
                }
            }
        }
    }
    release();
    out->ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return KHZ_OK;
}
