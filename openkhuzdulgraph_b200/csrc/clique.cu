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
// One launch sequence serves many (graph, clique app) jobs: their start vertices form one
// global index space.  Tiers by out-degree d of v0: one warp per v0 for d <= 64, one block per
// v0 for 64 < d <= 256 and 256 < d <= kBlockMax (rows in up to ~227 KB of shared memory, sized
// from the largest out-degree of the batch); larger d are left to the DFS engine.  Device-side
// classification sorts the block-tier start vertices by degree, heaviest first, so nothing
// waits on the host between launches.  Rows of the highest-ranked vertices come from a
// per-job hub triangle (one bit test per candidate pair); the others from splitter-bounded
// scans of the candidate's out-list against a hash of C.
#include <cuda_runtime.h>

#include "khz_internal.cuh"
#include "khz_setops.cuh"

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
    uint64_t cnt, t3, t4, bytes;
};

__device__ __forceinline__ uint32_t odeg(const uint64_t *off, uint32_t v) {
    return (uint32_t)(__ldg(off + v + 1) - __ldg(off + v));
}

constexpr uint32_t kEmpty = 0xffffffffu;

// Hub triangle.  For the H highest-ranked vertices (ids n - H .. n - 1 of the oriented graph,
// whose out-lists hold only larger ids, so ids of the same range) the adjacency is kept as a bit
// triangle: row h (vertex n - H + h) holds columns c > h, stored from word (h + 1) / 32 on.
// A row of the induced subgraph whose vertex is a hub is then read from the triangle with one
// bit test per candidate instead of a scan of the vertex's out-list.
constexpr uint32_t kHubRowsAuto = 32768;       // 64 MiB triangle
constexpr uint64_t kHubMinEdges = 1ull << 22;  // auto: graphs of at least 4 Mi oriented edges

// first word of row h: the sum over rows k < h of (wh - (k + 1) / 32) words
__host__ __device__ __forceinline__ uint64_t hub_row_offset(uint32_t h, uint32_t wh) {
    const uint64_t q = h >> 5, r = h & 31;
    return (uint64_t)h * wh - (16 * q * (q - 1) + q * (r + 1));
}

// The subgraph induced on C = N+(v0), in shared memory:
//   c[d]            the candidates (sorted vertex ids)
//   hkey/hidx[T]    open-addressing hash of c: vertex id -> position (T = 2^logt >= 2d)
//   rows[d * S]     bit j of row i set iff c[j] in N+(c[i])   (only j > i); W = ceil(d / 32)
//                   32-bit words, read as W64 = ceil(d / 64) 64-bit words by the counting loops,
//                   at a stride of S = 2 (W64 | 1) 32-bit words: odd in 64-bit words, so that
//                   lanes reading the same word offset of different rows hit different banks
//   rext[d]         per row, its first (low 16 bits) and one-past-last (high 16 bits) non-zero
//                   64-bit word: one shared load gives both
__device__ __forceinline__ int ext_lo(uint32_t e) { return (int)(e & 0xffffu); }
__device__ __forceinline__ int ext_hi(uint32_t e) { return (int)(e >> 16); }
struct Local {
    uint32_t *c;
    uint32_t *hkey;
    uint16_t *hidx;
    uint32_t *rows;
    uint32_t *rext;
    int d, W, W64, S, logt;
    __device__ __forceinline__ const uint64_t *row64(int i) const {
        return reinterpret_cast<const uint64_t *>(rows + (size_t)i * S);
    }
    const uint32_t *hub;  // the job's hub triangle, or null
    uint32_t hub_base, hub_wh;
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
// Only members of N+(c[i]) in [c[i+1], c[d-1]] can be in C.  32 evenly spaced splitters of the
// list, read in one load, bound that range to within one splitter gap at each end (lists of <= 32
// entries are the splitters themselves); the range is then read kScanUnroll x 32 entries per
// round with all loads of a round in flight together.  The list offsets of the warp's next 32 rows
// are fetched together, one per lane, and the next row's splitters are loaded before the current
// row is scanned, so a row's round trips overlap the previous row's work.  Rows of hub vertices
// come from the job's hub triangle instead.
constexpr int kScanUnroll = 4;

// Row i of a hub vertex from the triangle: lane l tests candidate j = 32 w + l (j > i), and the
// ballot over the warp is word w of the row, stored whole (the calling warp owns the row).
// U words per step (their loads in flight together): 4 in the large tiers, whose rows are long
// and almost all hub rows; 2 elsewhere.  (Lanes outside (i, d) skip their load: a variant that
// loaded on every lane and masked the ballot instead measured 12 % slower.)
template <int U>
__device__ __forceinline__ void hub_row(const Local &g, int i) {
    const int lane = (int)lane_id();
    const uint32_t h = g.c[i] - g.hub_base;
    const uint32_t *hrow = g.hub + hub_row_offset(h, g.hub_wh);
    const uint32_t wb = (h + 1) >> 5;
    uint32_t *row = g.rows + (size_t)i * g.S;
    for (int w = (i + 1) >> 5; w < g.W; w += U) {
        bool bit[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int j = ((w + u) << 5) + lane;
            bit[u] = false;
            if (j > i && j < g.d) {
                const uint32_t cc = g.c[j] - g.hub_base;
                bit[u] = (__ldg(hrow + ((cc >> 5) - wb)) >> (cc & 31)) & 1u;
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const unsigned m = __ballot_sync(kFull, bit[u]);
            if (lane == 0 && w + u < g.W) row[w + u] = m;
        }
    }
}

template <int U = 2>
__device__ void build_rows(const Local &g, const uint64_t *__restrict__ off, const uint32_t *__restrict__ adj,
                           int row_begin, int row_step) {
    const unsigned lane = lane_id();
    const int d = g.d;
    const uint32_t hi_val = g.c[d - 1];
    for (int i0 = row_begin; i0 < d - 1; i0 += 32 * row_step) {
        const int mine = i0 + (int)lane * row_step;
        uint64_t my_b = 0;
        uint32_t my_len = 0;
        if (mine < d - 1) {
            const uint32_t v = g.c[mine];
            my_b = __ldg(off + v);
            my_len = (uint32_t)(__ldg(off + v + 1) - my_b);
        }
        const int nrows = min(32, (d - 1 - i0 + row_step - 1) / row_step);
        // splitter `lane` of row r: entry lane * ceil(len / 32), or kEmpty past the end (or for
        // a hub row, which needs none)
        auto splitter = [&](int r) -> uint32_t {
            const uint64_t b0 = __shfl_sync(kFull, my_b, r);
            const uint32_t len = __shfl_sync(kFull, my_len, r);
            if (g.hub && g.c[i0 + r * row_step] >= g.hub_base) return kEmpty;
            const uint64_t sidx = lane * (((uint64_t)len + 31) >> 5);
            return sidx < len ? __ldg(adj + b0 + sidx) : kEmpty;
        };
        uint32_t sp_next = splitter(0);
        for (int r = 0; r < nrows; ++r) {
            const int i = i0 + r * row_step;
            if (g.hub && g.c[i] >= g.hub_base) {
                hub_row<U>(g, i);
                continue;
            }
            const uint32_t sp = sp_next;
            const uint64_t b0 = __shfl_sync(kFull, my_b, r);
            const uint32_t len = __shfl_sync(kFull, my_len, r);
            if (r + 1 < nrows) sp_next = splitter(r + 1);
            const uint32_t *L = adj + b0;
            const uint32_t lo_val = g.c[i + 1];
            uint32_t *row = g.rows + (size_t)i * g.S;
            auto probe = [&](uint32_t x) {
                if (x >= lo_val && x <= hi_val) {
                    const int j = g.find(x);
                    if (j >= 0) atomicOr(row + (j >> 5), 1u << (j & 31));
                }
            };
            const uint64_t step = ((uint64_t)len + 31) >> 5;
            if (step <= 1) {
                probe(sp);
                continue;
            }
            const uint64_t k_lo = __popc(__ballot_sync(kFull, sp < lo_val));
            const uint64_t k_hi = __popc(__ballot_sync(kFull, sp <= hi_val));
            const uint64_t begin = k_lo == 0 ? 0 : (k_lo - 1) * step + 1;
            const uint64_t end = min((uint64_t)len, k_hi * step);
            for (uint64_t b = begin; b < end; b += 32 * kScanUnroll) {
                uint32_t x[kScanUnroll];
#pragma unroll
                for (int u = 0; u < kScanUnroll; ++u) {
                    const uint64_t ix = b + 32 * u + lane;
                    x[u] = ix < end ? __ldg(L + ix) : kEmpty;
                }
#pragma unroll
                for (int u = 0; u < kScanUnroll; ++u) probe(x[u]);
            }
        }
    }
}

// first / one-past-last non-zero word of rows [tid, d) step nthr
__device__ __forceinline__ void row_extents(const Local &g, int tid, int nthr) {
    for (int i = tid; i < g.d; i += nthr) {
        const uint64_t *r = g.row64(i);
        int lo = g.W64, hi = 0;
        for (int w = (i + 1) >> 6; w < g.W64; ++w) {
            if (r[w]) {
                lo = min(lo, w);
                hi = w + 1;
            }
        }
        g.rext[i] = (uint32_t)(hi == 0 ? g.W64 : lo) | ((uint32_t)hi << 16);
    }
}

// WIDE: rows of many words (the large tiers), where the popcount loop runs two words per step
template <int K, bool STATS, bool WIDE = false>
__device__ __forceinline__ void process_item(const Local &g, int i, int j, const uint64_t *off, Acc &a) {
    const uint64_t *ri = g.row64(i);
    const uint64_t *rj = g.row64(j);
    const uint32_t ei = g.rext[i], ej = g.rext[j];
    const int lo = max(ext_lo(ei), ext_lo(ej));
    const int hi = min(ext_hi(ei), ext_hi(ej));
    uint32_t s = 0;
    if (!WIDE) {
        // the hot loop with 32-bit shared-window addresses stepped by one 64-bit word
        const uint32_t sb = (uint32_t)__cvta_generic_to_shared(g.rows);
        uint32_t ai = sb + (uint32_t)(i * g.S + 2 * lo) * 4u, aj = sb + (uint32_t)(j * g.S + 2 * lo) * 4u;
        for (int w = lo; w < hi; ++w, ai += 8, aj += 8) {
            uint64_t x, y;
            asm("ld.shared.u64 %0, [%1];" : "=l"(x) : "r"(ai));
            asm("ld.shared.u64 %0, [%1];" : "=l"(y) : "r"(aj));
            s += __popcll(x & y);
        }
    } else {
        // two 64-bit words per step with independent sums (the popcounts of one step do not
        // wait on each other)
        const uint32_t sb = (uint32_t)__cvta_generic_to_shared(g.rows);
        uint32_t ai = sb + (uint32_t)(i * g.S + 2 * lo) * 4u, aj = sb + (uint32_t)(j * g.S + 2 * lo) * 4u;
        uint32_t s1 = 0;
        int w = lo;
        for (; w + 1 < hi; w += 2, ai += 16, aj += 16) {
            uint64_t x0, y0, x1, y1;
            asm("ld.shared.u64 %0, [%1];" : "=l"(x0) : "r"(ai));
            asm("ld.shared.u64 %0, [%1];" : "=l"(y0) : "r"(aj));
            asm("ld.shared.u64 %0, [%1+8];" : "=l"(x1) : "r"(ai));
            asm("ld.shared.u64 %0, [%1+8];" : "=l"(y1) : "r"(aj));
            s += __popcll(x0 & y0);
            s1 += __popcll(x1 & y1);
        }
        if (w < hi) {
            uint64_t x, y;
            asm("ld.shared.u64 %0, [%1];" : "=l"(x) : "r"(ai));
            asm("ld.shared.u64 %0, [%1];" : "=l"(y) : "r"(aj));
            s += __popcll(x & y);
        }
        s += s1;
    }
    if (STATS) {
        uint32_t pi = 0;
        for (int w = ext_lo(ei); w < ext_hi(ei); ++w) pi += __popcll(ri[w]);
        a.bytes += 4ull * ((uint64_t)pi + odeg(off, g.c[j]) + s);
    }
    if (K == 4) {
        a.cnt += s;
        return;
    }
    a.t4 += s;
    for (int w1 = lo; w1 < hi; ++w1) {
        uint64_t m = ri[w1] & rj[w1];
        while (m) {
            const int l = (w1 << 6) + __ffsll((long long)m) - 1;
            m &= m - 1;
            const uint64_t *rl = g.row64(l);
            const uint32_t el = g.rext[l];
            const int lo3 = max(lo, ext_lo(el));
            const int hi3 = min(hi, ext_hi(el));
            uint32_t t = 0;
            for (int w = lo3; w < hi3; ++w) t += __popcll(ri[w] & rj[w] & rl[w]);
            a.cnt += t;
            if (STATS) a.bytes += 4ull * ((uint64_t)s + odeg(off, g.c[l]) + t);
        }
    }
}

// Items (i, j) = the set bits j of row i, dealt to the lanes of the calling warp in batches of
// 32.  Each lane holds one unit (row u_row, word u_word, its bits); an inclusive scan of the
// units' popcounts numbers their items, and each free lane finds its item's unit by a 5-step
// search over the lanes' prefix sums.  A partial batch (lanes [0, pc) hold items) carries over to
// the next call.  k is warp-uniform (one start vertex at a time).
template <bool STATS, int KMAX>
__device__ __forceinline__ void deal_units(const Local &g, int K, const uint64_t *off, int u_row, int u_word,
                                           uint32_t bits, int &pc, int &my_i, int &my_j, Acc &a) {
    const int lane = (int)lane_id();
    const int c = __popc(bits);
    a.t3 += c;
    if (STATS) a.bytes += 4ull * c;
    if (K == 3) {
        a.cnt += c;
        return;
    }
    int incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += y;
    }
    const int total = __shfl_sync(kFull, incl, 31);
    const int excl = incl - c;
    for (int consumed = 0; consumed < total;) {
        const int avail = min(32 - pc, total - consumed);
        const int t = consumed + lane - pc;
        int w = 0;
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) {
            const int e = __shfl_sync(kFull, excl, w + s);
            if (e <= t) w += s;
        }
        const uint32_t wb = __shfl_sync(kFull, bits, w);
        const int we = __shfl_sync(kFull, excl, w);
        const int wr = __shfl_sync(kFull, u_row, w);
        const int ww = __shfl_sync(kFull, u_word, w);
        if (lane >= pc && lane < pc + avail) {
            my_i = wr;
            my_j = (ww << 5) + nth_set_bit(wb, t - we);
        }
        consumed += avail;
        pc += avail;
        if (pc == 32) {
            if (KMAX == 4 || K == 4) process_item<4, STATS>(g, my_i, my_j, off, a);
            else process_item<5, STATS>(g, my_i, my_j, off, a);
            pc = 0;
        }
    }
}

template <bool STATS, int KMAX>
__device__ __forceinline__ void deal_flush(const Local &g, int K, const uint64_t *off, int pc, int my_i, int my_j,
                                           Acc &a) {
    if (K > 3 && (int)lane_id() < pc) {
        if (KMAX == 4 || K == 4) process_item<4, STATS>(g, my_i, my_j, off, a);
        else process_item<5, STATS>(g, my_i, my_j, off, a);
    }
}

// Count over rows [row_begin, d) with stride row_step for a k-clique job.  The items (i, j) of a
// 64-bit row word are appended to the warp's kRing-entry ring in shared memory (lane l writes the
// items of bits l and 32 + l at their ranks among the word's set bits), and while 32 items are
// pending the lanes take one each: items of consecutive words and rows pack into full batches.
// The triangles through the rows (NumExtensions) are the number of items dealt.
constexpr int kRing = 128;
template <bool STATS, int KMAX>
__device__ void count_rows(const Local &g, int K, const uint64_t *off, int row_begin, int row_step, uint32_t *ring,
                           Acc &a) {
    const int lane = (int)lane_id();
    const uint32_t lanebit = 1u << lane, below = lanebit - 1u;
    uint32_t head = 0, tail = 0;  // ring positions (warp-uniform); pending items tail - head < 32
    for (int i = row_begin; i < g.d; i += row_step) {
        const uint64_t *ri = g.row64(i);
        const uint32_t ei = g.rext[i];
        const int lo = ext_lo(ei), hi = ext_hi(ei);
        if (STATS && lane == 0) a.bytes += 4ull * ((uint64_t)g.d + odeg(off, g.c[i]));
        const uint32_t ibase = ((uint32_t)i << 16) + (uint32_t)lane;
        for (int w = lo; w < hi; ++w) {
            const uint64_t bits = ri[w];
            const uint32_t b0 = (uint32_t)bits, b1 = (uint32_t)(bits >> 32);
            const uint32_t c0 = __popc(b0);
            if (K == 3) {
                tail += c0 + __popc(b1);
                continue;
            }
            const uint32_t item = ibase + ((uint32_t)w << 6);
            if (b0 & lanebit) ring[(tail + __popc(b0 & below)) & (kRing - 1)] = item;
            if (b1 & lanebit) ring[(tail + c0 + __popc(b1 & below)) & (kRing - 1)] = item + 32;
            tail += c0 + __popc(b1);
            while (tail - head >= 32) {
                __syncwarp();
                const uint32_t it = ring[(head + lane) & (kRing - 1)];
                __syncwarp();
                head += 32;
                if (KMAX == 4 || K == 4) process_item<4, STATS, true>(g, (int)(it >> 16), (int)(it & 0xffffu), off, a);
                else process_item<5, STATS, true>(g, (int)(it >> 16), (int)(it & 0xffffu), off, a);
            }
        }
    }
    if (lane == 0) {
        a.t3 += tail;
        if (STATS) a.bytes += 4ull * tail;
        if (K == 3) a.cnt += tail;
    }
    __syncwarp();
    if (K > 3 && (uint32_t)lane < tail - head) {
        const uint32_t it = ring[(head + lane) & (kRing - 1)];
        if (KMAX == 4 || K == 4) process_item<4, STATS, true>(g, (int)(it >> 16), (int)(it & 0xffffu), off, a);
        else process_item<5, STATS, true>(g, (int)(it >> 16), (int)(it & 0xffffu), off, a);
    }
    __syncwarp();
}

// Rows of at most 8 words (the mid tier): one unit per 32-bit word, the words of 32 / wp rows per
// round (wp = 4 or 8, a power of two >= W), dealt as in the warp tier; per-row work is spread
// over the lanes instead of running row by row.
template <bool STATS, int KMAX>
__device__ void count_rows_units(const Local &g, int K, const uint64_t *off, int row_begin, int row_step, Acc &a) {
    const int lane = (int)lane_id();
    const int lg = g.W <= 4 ? 2 : 3;
    const int nrows = (g.d - row_begin + row_step - 1) / row_step;  // rows of this warp
    int pc = 0, my_i = 0, my_j = 0;
    for (int k0 = 0; k0 < nrows; k0 += 32 >> lg) {
        const int k = k0 + (lane >> lg), w = lane & ((1 << lg) - 1);
        const int i = row_begin + k * row_step;
        const bool ok = k < nrows && w < g.W;
        const uint32_t bits = ok ? g.rows[(size_t)i * g.S + w] : 0u;
        if (STATS && ok && w == 0) a.bytes += 4ull * ((uint64_t)g.d + odeg(off, g.c[i]));
        deal_units<STATS, KMAX>(g, K, off, i, w, bits, pc, my_i, my_j, a);
    }
    deal_flush<STATS, KMAX>(g, K, off, pc, my_i, my_j, a);
}

// The same over all rows of a warp-tier start vertex (W = 2 words per row): 16 rows per round.
template <bool STATS, int KMAX>
__device__ void count_rows_small(const Local &g, int K, const uint64_t *off, Acc &a) {
    const int lane = (int)lane_id();
    int pc = 0, my_i = 0, my_j = 0;
    if (STATS)
        for (int i = lane; i < g.d; i += 32) a.bytes += 4ull * ((uint64_t)g.d + odeg(off, g.c[i]));
    for (int u0 = 0; u0 < 2 * g.d; u0 += 32) {
        const int u = u0 + lane;
        const int i = u >> 1, w = u & 1;
        const uint32_t bits = i < g.d ? g.rows[(size_t)i * g.S + w] : 0u;
        deal_units<STATS, KMAX>(g, K, off, i, w, bits, pc, my_i, my_j, a);
    }
    deal_flush<STATS, KMAX>(g, K, off, pc, my_i, my_j, a);
}

// ---- Tensor-core 4-clique count (large block tiers) -------------------------------------------
// The induced subgraphs of the large tiers are dense (31 % of candidate pairs are edges for
// 256 < d <= 640 and 44 % above that on R-MAT s22), so their 4-cliques are counted as a masked
// matrix product: with A the d x d upper-triangular 0/1 matrix of the rows,
//   4-cliques through v0 = sum over i < j with A[i][j] = 1 of (A A^T)[i][j]
// (row i and row j share (A A^T)[i][j] columns, each closing a 4-clique).  A A^T runs on the
// tensor cores as tcgen05.mma kind::i8 (0/1 bytes, int32 accumulators in tensor memory) over
// 128 x 128 tiles of row blocks (ib, jb >= ib), only over columns >= 128 jb (row j has no bit at
// or below j).  Per 32-column step the block expands 32 bits of each needed row into bytes in a
// shared-memory stage (the canonical K-major layout without swizzle: 8-row core matrices of
// 16 bytes per row, the two 16-byte K halves 2048 bytes apart), one thread issues the MMAs of up
// to G accumulator tiles and commits them to an mbarrier, and the block waits (bounded) before the
// stage is rewritten.  The epilogue reads each accumulator row with tcgen05.ld and adds the
// entries whose bit is set in row i.
constexpr int kMmaRows = 128;                 // M = N = 128 rows of the 0/1 matrix per tile
constexpr uint32_t kMmaTileBytes = 128 * 32;  // one operand tile: 128 rows x 32 columns (bytes)
constexpr uint32_t kMmaWaitIters = 1u << 20;  // mbarrier polls before the launch reports a stall
constexpr int kMmaMaxTiles = 4;               // accumulator tiles per pass: 4 x 128 = all 512 TMEM columns
// tensor-memory columns a block allocates for g accumulator tiles (a power of two >= 32)
__host__ __device__ __forceinline__ uint32_t mma_tmem_cols(int g) { return g <= 1 ? 128u : (g == 2 ? 256u : 512u); }
// instruction descriptor: D int32 (bits 4-5 = 2), A and B unsigned 8-bit, K-major, N = 128, M = 128
constexpr uint32_t kMmaIdesc = (2u << 4) | ((uint32_t)(kMmaRows >> 3) << 17) | ((uint32_t)(kMmaRows >> 4) << 24);

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor of one operand tile: start address, K-half stride (LBO)
// 2048 bytes, 8-row-group stride (SBO) 128 bytes, descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t mma_desc(uint32_t addr) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)(2048u >> 4) << 16) | ((uint64_t)(128u >> 4) << 32) |
           (1ull << 46);
}

// bytes 0..3 of the result are bits 0..3 of x (as 0 / 1)
__device__ __forceinline__ uint32_t spread4(uint32_t x) { return ((x & 0xFu) * 0x00204081u) & 0x01010101u; }

// row r's 32 bits of one 32-column step as 32 bytes of the tile: bits 0-15 in the first K half,
// bits 16-31 in the second
__device__ __forceinline__ void expand_row_bits(uint8_t *tile, int r, uint32_t bits) {
    const uint4 lo = make_uint4(spread4(bits), spread4(bits >> 4), spread4(bits >> 8), spread4(bits >> 12));
    const uint4 hi = make_uint4(spread4(bits >> 16), spread4(bits >> 20), spread4(bits >> 24), spread4(bits >> 28));
    *reinterpret_cast<uint4 *>(tile + r * 16) = lo;
    *reinterpret_cast<uint4 *>(tile + 2048 + r * 16) = hi;
}

// true once the mbarrier's phase `parity` has completed, false after kMmaWaitIters polls
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    uint32_t done = 0;
    for (uint32_t it = 0; it < kMmaWaitIters && !done; ++it)
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
    return done != 0;
}

// mbarriers of the tensor-core count: operand stage s full (producer warps arrived) and empty (its
// MMAs completed), and the accumulators of a pass complete
enum : int { kBarFull = 0, kBarEmpty = 2, kBarAcc = 4, kMmaBars = 5 };

struct MmaState {
    uint32_t tmem;            // tensor-memory base of the accumulators (G x 128 columns)
    uint32_t bar[kMmaBars];   // shared addresses of the mbarriers
    uint32_t uses[2];         // fills of each operand stage so far (every thread keeps the count)
    uint32_t passes;          // accumulator passes so far
    int G;                    // accumulator tiles per pass
    uint8_t *stage;           // two stages of (G + 1) operand tiles each
    volatile int *abort;      // set when a wait ran out: every role then stops waiting
};

// poll an mbarrier phase; false after the poll limit, or early once another thread set the abort flag
__device__ __forceinline__ bool mbar_wait_abortable(uint32_t mbar, uint32_t parity, volatile int *abort) {
    uint32_t done = 0;
    for (uint32_t it = 0; it < kMmaWaitIters && !done; ++it) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (!done && (it & 63u) == 63u && *abort) break;
    }
    return done != 0;
}

__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}\n" ::"r"(mbar) : "memory");
}

// 4-clique count of one start vertex on the tensor cores, warp-specialised: warps 1.. expand the
// operand tiles of each 32-column step into one of two stages and arrive on its `full` barrier;
// thread 0 waits for it, issues the step's MMAs and commits them to the stage's `empty` barrier
// (and, after a pass's last step, to the accumulator barrier).  Producers wait for `empty` only
// before refilling a stage, so the expansion of step s + 1 overlaps the MMAs of step s, and no
// block-wide barrier is taken per step; all warps then read the pass's accumulators.  Every wait is
// bounded; one that runs out sets the abort flag, the others then give up at once, and the
// function returns false with the stall recorded in *err.
template <int THREADS>
__device__ bool count_rows_mma(const Local &g, MmaState &ms, unsigned int *err, Acc &a) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int kWarps = THREADS / 32;
    constexpr int kProducerThreads = THREADS - 32;
    const int d = g.d;
    // triangles through v0 (NumExtensions): every set bit of every row
    for (int i = tid; i < d; i += THREADS) {
        const uint32_t *r = g.rows + (size_t)i * g.S;
        uint32_t c = 0;
        for (int w = (i + 1) >> 5; w < g.W; ++w) c += __popc(r[w]);
        a.t3 += c;
    }
    const int nb = (d + kMmaRows - 1) / kMmaRows;
    const int kw = g.W;  // 32-column steps
    const uint32_t stage_bytes = (uint32_t)(ms.G + 1) * kMmaTileBytes;
    for (int ib = 0; ib < nb; ++ib) {
        for (int jb0 = ib; jb0 < nb; jb0 += ms.G) {
            const int ng = min(ms.G, nb - jb0);
            const int k0 = jb0 * (kMmaRows / 32);
            for (int kc = k0; kc < kw; ++kc) {
                const int st = (int)((ms.uses[0] + ms.uses[1]) & 1u);
                const uint32_t u = ms.uses[st];
                uint8_t *stage = ms.stage + st * stage_bytes;
                if (warp > 0) {
                    // producers: refill the stage once its previous MMAs completed
                    int go = 1;
                    if (lane == 0) {
                        if (u > 0 && !mbar_wait_abortable(ms.bar[kBarEmpty + st], (u - 1) & 1u, ms.abort)) *ms.abort = 1;
                        go = !*ms.abort;
                    }
                    go = __shfl_sync(kFull, go, 0);
                    if (go) {
                        // tile 0 = rows of block ib, tile 1 + t = rows of block jb0 + t
                        for (int task = tid - 32; task < (ng + 1) * kMmaRows; task += kProducerThreads) {
                            const int tile = task / kMmaRows, r = task % kMmaRows;
                            const int R = (tile == 0 ? ib : jb0 + tile - 1) * kMmaRows + r;
                            const uint32_t bits = R < d ? g.rows[(size_t)R * g.S + kc] : 0u;
                            expand_row_bits(stage + tile * kMmaTileBytes, r, bits);
                        }
                        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    }
                    __syncwarp();
                    if (lane == 0) mbar_arrive(ms.bar[kBarFull + st]);
                } else if (lane == 0) {
                    // the MMA thread
                    if (!mbar_wait_abortable(ms.bar[kBarFull + st], u & 1u, ms.abort)) *ms.abort = 1;
                    if (!*ms.abort) {
                        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                        const uint32_t s0 = smem_addr(stage);
                        const uint64_t da = mma_desc(s0);
                        const uint32_t acc = kc > k0 ? 1u : 0u;
                        for (int t = 0; t < ng; ++t) {
                            const uint64_t db = mma_desc(s0 + (uint32_t)(t + 1) * kMmaTileBytes);
                            asm volatile(
                                "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                                "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(
                                    ms.tmem + (uint32_t)(t * kMmaRows)),
                                "l"(da), "l"(db), "r"(kMmaIdesc), "r"(acc), "r"(0u));
                        }
                        asm volatile(
                            "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                ms.bar[kBarEmpty + st])
                            : "memory");
                        if (kc == kw - 1)
                            asm volatile(
                                "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                    ms.bar[kBarAcc])
                                : "memory");
                    }
                }
                ms.uses[st] = u + 1;
            }
            // the pass's accumulators
            const bool ok = mbar_wait_abortable(ms.bar[kBarAcc], ms.passes & 1u, ms.abort);
            ms.passes += 1;
            if (__syncthreads_or(!ok || *ms.abort)) {
                if (tid == 0) atomicOr(err, 2u);
                return false;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            // epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 (rows of block ib), columns
            // 16 c, 16 (c + kWarps / 4), ... of the ng accumulator tiles
            const int q = warp & 3, i = ib * kMmaRows + q * 32 + lane;
            const uint32_t *ri = g.rows + (size_t)min(i, d - 1) * g.S;
            uint64_t sum = 0;
            for (int col = (warp >> 2) * 16; col < ng * kMmaRows; col += (kWarps / 4) * 16) {
                uint32_t v[16];
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                    "[%16];\n"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                      "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                      "=r"(v[15])
                    : "r"(ms.tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)col));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                const int j0 = (jb0 + col / kMmaRows) * kMmaRows + col % kMmaRows;
                const uint32_t m = (i < d && j0 < d) ? (ri[j0 >> 5] >> (j0 & 31)) & 0xFFFFu : 0u;
#pragma unroll
                for (int t = 0; t < 16; ++t) sum += (m >> t) & 1u ? v[t] : 0u;
            }
            a.cnt += sum;
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();  // every accumulator read before the next pass overwrites it
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        }
    }
    return true;
}

// warp reduction of the accumulator and one atomicAdd per counter into the job's row
__device__ __forceinline__ void flush_acc(Acc &a, int K, uint64_t *row, uint64_t *phase_bytes) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a.cnt += __shfl_down_sync(kFull, a.cnt, o);
        a.t3 += __shfl_down_sync(kFull, a.t3, o);
        a.t4 += __shfl_down_sync(kFull, a.t4, o);
        a.bytes += __shfl_down_sync(kFull, a.bytes, o);
    }
    if (lane_id() == 0) {
        // NumExtensions beyond levels 0 and 1: the scattered triangles (k >= 4) and 4-cliques (k = 5)
        const uint64_t ext = (K >= 4 ? a.t3 : 0) + (K >= 5 ? a.t4 : 0);
        if (a.cnt) atomicAdd((unsigned long long *)&row[0], (unsigned long long)a.cnt);
        if (ext) atomicAdd((unsigned long long *)&row[KHZ_MAX_COUNTS], (unsigned long long)ext);
        if (a.bytes) atomicAdd((unsigned long long *)&row[KHZ_MAX_COUNTS + 1], (unsigned long long)a.bytes);
        if (a.bytes && phase_bytes) atomicAdd((unsigned long long *)phase_bytes, (unsigned long long)a.bytes);
    }
    a = Acc{0, 0, 0, 0};
}

// job of a global start-vertex index (jobs sorted by vbase)
__device__ __forceinline__ int job_of(const BJob *jobs, int n_jobs, uint64_t gv) {
    int lo = 0, hi = n_jobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].vbase <= gv) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ uint64_t *row_of(uint64_t *rows, const BJob &j) { return rows + (size_t)j.out_row * kRowWords; }

// Warp tier: one warp per start vertex with dmin <= d <= 64 over all jobs' vertices, taken in
// descending global index (per job: descending rank, i.e. heaviest first on the oriented DAG).
constexpr int kWarpHashLog = 8;  // 256-slot table per warp (at least 4 slots per candidate)
template <bool STATS, int KMAX>
__global__ void __launch_bounds__(256, 4) clique_warp_kernel(const BJob *__restrict__ jobs, int n_jobs,
                                                          uint64_t n_total, uint32_t dmin, uint32_t warp_max,
                                                          unsigned long long *queue, uint64_t *rows_out,
                                                          uint64_t *phase_bytes) {
    constexpr int W = kWarpMax / 32;
    constexpr int W64 = kWarpMax / 64;
    constexpr int S = 2 * (W64 | 1);
    constexpr int T = 1 << kWarpHashLog;
    __shared__ uint32_t s_c[8][kWarpMax];
    __shared__ uint64_t s_rows[8][kWarpMax * S / 2];
    __shared__ uint32_t s_hkey[8][T];
    __shared__ uint16_t s_hidx[8][T];
    __shared__ uint32_t s_rext[8][kWarpMax];
    const unsigned lane = lane_id();
    const int wib = threadIdx.x >> 5;
    Local g;
    g.c = s_c[wib];
    g.rows = reinterpret_cast<uint32_t *>(s_rows[wib]);
    g.hkey = s_hkey[wib];
    g.hidx = s_hidx[wib];
    g.rext = s_rext[wib];
    g.W = W;
    g.W64 = W64;
    g.S = S;
    g.logt = kWarpHashLog;
    Acc a = {0, 0, 0, 0};
    int cur_job = -1;
    constexpr uint32_t kChunk = 32;
    while (true) {
        unsigned long long c0 = 0;
        if (lane == 0) c0 = atomicAdd(queue, (unsigned long long)kChunk);
        c0 = __shfl_sync(kFull, c0, 0);
        if (c0 >= n_total) break;
        const unsigned long long c1 = min((unsigned long long)n_total, c0 + kChunk);
        // one candidate start vertex per lane
        const unsigned long long myc = c0 + lane;
        uint32_t myv = 0, myd = 0;
        int myj = 0;
        if (myc < c1) {
            const uint64_t gv = n_total - 1 - myc;
            myj = job_of(jobs, n_jobs, gv);
            myv = (uint32_t)(gv - jobs[myj].vbase);
            myd = jobs[myj].start.keep(myv) ? odeg(jobs[myj].off, myv) : 0u;
        }
        unsigned todo = __ballot_sync(kFull, myc < c1 && myd >= dmin && myd <= warp_max);
        while (todo) {
            const int src = __ffs(todo) - 1;
            todo &= todo - 1;
            const uint32_t v0 = __shfl_sync(kFull, myv, src);
            const int j = __shfl_sync(kFull, myj, src);
            g.d = (int)__shfl_sync(kFull, myd, src);
            if (j != cur_job) {
                if (cur_job >= 0) flush_acc(a, jobs[cur_job].k, row_of(rows_out, jobs[cur_job]), phase_bytes);
                cur_job = j;
            }
            const uint64_t *off = jobs[j].off;
            const uint32_t *adj = jobs[j].adj;
            g.hub = jobs[j].hub;
            g.hub_base = jobs[j].n - jobs[j].hub_rows;
            g.hub_wh = jobs[j].hub_rows >> 5;
            const uint64_t b0 = __ldg(off + v0);
            __syncwarp();
            for (int t = lane; t < kWarpMax; t += 32) g.c[t] = t < g.d ? __ldg(adj + b0 + t) : kEmpty;
            for (int t = lane; t < kWarpMax * S; t += 32) g.rows[t] = 0;
            for (int t = lane; t < T; t += 32) g.hkey[t] = kEmpty;
            __syncwarp();
            hash_insert(g, lane, 32);
            __syncwarp();
            if (g.d >= 2) build_rows(g, off, adj, 0, 1);
            __syncwarp();
            row_extents(g, lane, 32);
            __syncwarp();
            count_rows_small<STATS, KMAX>(g, jobs[j].k, off, a);
        }
    }
    if (cur_job >= 0) flush_acc(a, jobs[cur_job].k, row_of(rows_out, jobs[cur_job]), phase_bytes);
}

// shared-memory footprint of a block-tier launch serving out-degrees up to dcap
__host__ __device__ __forceinline__ int block_logt(int dcap) {
    // hash slots per candidate: 8 (almost every miss ends at the first slot) where shared memory
    // allows, 2 for larger candidate sets (at most 2048 slots, so that the large tier fits an SM)
    const int per = dcap <= kMidMax ? 8 : 2;
    int l = 5;
    while ((1 << l) < per * dcap) ++l;
    return (dcap <= kMidMax || l <= 11) ? l : 11;  // <= 2048 slots: >= 1.68 per candidate up to kBlockMax
}
__host__ __device__ __forceinline__ size_t block_rows_words(int dcap) {
    return (size_t)((dcap + 31) & ~31) * 2 * ((size_t)((dcap + 63) / 64) | 1);
}
// the item rings, which the tensor-core count reuses for its two operand stages of (mma_g + 1) tiles
__host__ __device__ __forceinline__ size_t block_smem(int dcap, int threads, int mma_g = 0) {
    const size_t dp = (size_t)((dcap + 31) & ~31);
    const size_t t = (size_t)1 << block_logt(dcap);
    const size_t rings = (size_t)(threads / 32) * kRing * 4;
    const size_t stage = mma_g > 0 ? (size_t)2 * (mma_g + 1) * kMmaTileBytes : 0;
    return dp * 4 + t * 4 + t * 2 + dp * 2 * 2 + block_rows_words(dcap) * 4 + (rings > stage ? rings : stage);
}

// Block tier: one block per start vertex; the list holds global start-vertex indices, heaviest
// degree bucket first, and its length is read from device memory.  The mid tier runs 256-thread
// blocks, several per SM (registers capped for that); the lower large tier (out-degree up to 640)
// two 512-thread blocks per SM, so that one block's barriers and phase tails overlap the other's
// work; the upper large tier one 1024-thread block per SM (its shared memory fills the SM).
constexpr int kMidThreads = 256, kLargeAThreads = 512, kLargeThreads = 1024;
constexpr int kMidMinBlocks = 5;
constexpr int kLargeAMax = 640;
// MMA: the build whose k = 4 jobs count on the tensor cores (mma_g accumulator tiles per pass); the
// other build has no tensor-core code at all, so its CUDA-core count compiles as before
template <bool STATS, int KMAX, int THREADS, bool MMA = false>
__global__ void __launch_bounds__(THREADS, THREADS == kLargeThreads ? 1 : (THREADS == kLargeAThreads ? 2 : kMidMinBlocks))
    clique_block_kernel(const BJob *__restrict__ jobs, int n_jobs, const uint32_t *__restrict__ list,
                                    const unsigned int *__restrict__ list_len, int dcap, unsigned long long *queue,
                                    uint64_t *rows_out, uint64_t *phase_bytes, int mma_g, unsigned int *err) {
    constexpr bool kMma = MMA && !STATS && THREADS != kMidThreads;
    extern __shared__ __align__(16) uint32_t smem[];
    __shared__ uint32_t s_v0;
    __shared__ int s_job;
    __shared__ __align__(8) uint64_t s_mbar[kMmaBars];
    __shared__ uint32_t s_tmem;
    __shared__ int s_abort;
    const int dp = (dcap + 31) & ~31;
    const int logt = block_logt(dcap);
    const int T = 1 << logt;
    Local g;
    g.c = smem;
    g.hkey = smem + dp;
    g.hidx = (uint16_t *)(g.hkey + T);
    g.rext = (uint32_t *)(g.hidx + T);  // T is a power of two >= 32: 4-byte aligned
    g.rows = g.rext + dp;
    g.logt = logt;
    const int warps = blockDim.x >> 5;
    const int wib = threadIdx.x >> 5;
    uint32_t *ring = g.rows + block_rows_words(dcap) + (size_t)wib * kRing;
    const bool use_mma = kMma && mma_g > 0;
    const uint32_t tmem_cols = mma_tmem_cols(mma_g);
    MmaState ms{0, {0, 0, 0, 0, 0}, {0, 0}, 0, mma_g,
                reinterpret_cast<uint8_t *>(g.rows + block_rows_words(dcap)),  // stages: over the rings
                &s_abort};
    if (use_mma) {
        if (wib == 0) {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&s_tmem)),
                         "r"(tmem_cols));
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
        }
        if (threadIdx.x == 0) {
            // `full` waits for one arrival per producer warp (all warps but warp 0); the others for
            // one tcgen05.commit
            for (int b = 0; b < kMmaBars; ++b) {
                const uint32_t count = b < kBarEmpty ? (uint32_t)(warps - 1) : 1u;
                asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&s_mbar[b])), "r"(count));
            }
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            s_abort = 0;
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        ms.tmem = s_tmem;
        for (int b = 0; b < kMmaBars; ++b) ms.bar[b] = smem_addr(&s_mbar[b]);
    }
    bool stalled = false;
    const unsigned int n_list = *list_len;
    Acc a = {0, 0, 0, 0};
    int cur_job = -1;
    while (true) {
        if (threadIdx.x == 0) {
            const unsigned long long t = atomicAdd(queue, 1ull);
            if (t < n_list) {
                const uint64_t gv = list[t];
                const int j = job_of(jobs, n_jobs, gv);
                s_job = j;
                s_v0 = (uint32_t)(gv - jobs[j].vbase);
            } else {
                s_job = -1;
            }
        }
        __syncthreads();
        const int j = s_job;
        if (j < 0) break;
        const uint32_t v0 = s_v0;
        if (j != cur_job) {
            if (cur_job >= 0) flush_acc(a, jobs[cur_job].k, row_of(rows_out, jobs[cur_job]), phase_bytes);
            cur_job = j;
        }
        const uint64_t *off = jobs[j].off;
        const uint32_t *adj = jobs[j].adj;
        g.hub = jobs[j].hub;
        g.hub_base = jobs[j].n - jobs[j].hub_rows;
        g.hub_wh = jobs[j].hub_rows >> 5;
        g.d = (int)odeg(off, v0);
        g.W = (g.d + 31) >> 5;
        g.W64 = (g.d + 63) >> 6;
        g.S = 2 * (g.W64 | 1);
        const uint64_t b0 = __ldg(off + v0);
        for (int t = threadIdx.x; t < g.d; t += blockDim.x) g.c[t] = __ldg(adj + b0 + t);
        for (int t = threadIdx.x; t < g.d * g.S; t += blockDim.x) g.rows[t] = 0;
        for (int t = threadIdx.x; t < T; t += blockDim.x) g.hkey[t] = kEmpty;
        __syncthreads();
        hash_insert(g, threadIdx.x, blockDim.x);
        __syncthreads();
        build_rows<THREADS == kMidThreads ? 2 : 4>(g, off, adj, wib, warps);
        __syncthreads();
        if (use_mma && jobs[j].k == 4) {
            if (!count_rows_mma<THREADS>(g, ms, err, a)) {
                stalled = true;
                break;
            }
        } else {
            row_extents(g, threadIdx.x, blockDim.x);
            __syncthreads();
            if (g.W <= 8) count_rows_units<STATS, KMAX>(g, jobs[j].k, off, wib, warps, a);
            else count_rows<STATS, KMAX>(g, jobs[j].k, off, wib, warps, ring, a);
        }
        __syncthreads();
    }
    if (cur_job >= 0) flush_acc(a, jobs[cur_job].k, row_of(rows_out, jobs[cur_job]), phase_bytes);
    if (use_mma) {
        // after a stall, give the outstanding MMAs one more bounded wait before the accumulators
        // are released (a completed phase makes the wait return at once)
        if (stalled && threadIdx.x == 0)
            for (int st = 0; st < 2; ++st)
                if (ms.uses[st] > 0) mbar_wait(ms.bar[kBarEmpty + st], (ms.uses[st] - 1) & 1u);
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (wib == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(ms.tmem), "r"(tmem_cols));
        }
    }
}

using BlockKernel = void (*)(const BJob *, int, const uint32_t *, const unsigned int *, int, unsigned long long *,
                             uint64_t *, uint64_t *, int, unsigned int *);
template <int THREADS>
BlockKernel block_kernel_of(bool stats, int kmax, bool mma) {
    if (mma && !stats && THREADS != kMidThreads)
        return kmax == 5 ? clique_block_kernel<false, 5, THREADS, true> : clique_block_kernel<false, 4, THREADS, true>;
    return stats ? (kmax == 5 ? clique_block_kernel<true, 5, THREADS> : clique_block_kernel<true, 4, THREADS>)
                 : (kmax == 5 ? clique_block_kernel<false, 5, THREADS> : clique_block_kernel<false, 4, THREADS>);
}
// tier 0: mid, tier 1: lower large, tier 2: upper large
BlockKernel block_kernel(bool stats, int kmax, int tier, bool mma = false) {
    return tier == 0   ? block_kernel_of<kMidThreads>(stats, kmax, false)
           : tier == 1 ? block_kernel_of<kLargeAThreads>(stats, kmax, mma)
                       : block_kernel_of<kLargeThreads>(stats, kmax, mma);
}
// out-degrees (lo, hi] of block tier t
__host__ __device__ __forceinline__ int tier_lo(int t, int warp_max) {
    return t == 0 ? warp_max : (t == 1 ? kMidMax : kLargeAMax);
}
__host__ __device__ __forceinline__ int tier_hi(int t) { return t == 0 ? kMidMax : (t == 1 ? kLargeAMax : kBlockMax); }
__host__ __device__ __forceinline__ int tier_of(uint32_t d) {
    return d <= (uint32_t)kMidMax ? 0 : (d <= (uint32_t)kLargeAMax ? 1 : 2);
}

// The hub triangle of one job (zeroed beforehand): one warp per hub row.
__global__ void hub_build_kernel(const uint64_t *__restrict__ off, const uint32_t *__restrict__ adj, uint32_t n,
                                 uint32_t rows, uint32_t *hub) {
    const uint32_t base = n - rows, wh = rows >> 5;
    const unsigned lane = lane_id();
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t h = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; h < rows; h += nw) {
        const uint32_t u = base + h;
        const uint64_t e = off[u + 1];
        uint32_t *row = hub + hub_row_offset(h, wh);
        const uint32_t wb = (h + 1) >> 5;
        for (uint64_t t = off[u] + lane; t < e; t += 32) {
            const uint32_t c = adj[t] - base;  // > h: out-lists hold larger ids only
            atomicOr(row + ((c >> 5) - wb), 1u << (c & 31));
        }
    }
}

// Block-tier lists in exact descending out-degree order, built without the host: a histogram
// over degrees, one prefix pass, one write pass (a counting sort).  Tier t's list holds the degrees
// (tier_lo(t), tier_hi(t)]; larger degrees go to the DFS engine.  Counter layout (unsigned int):
// hist[kCntDeg], cursor[kCntDeg], base[kCntDeg], then the tiers' list lengths.
constexpr int kCntDeg = kBlockMax + 1;
constexpr int kCntCursor = kCntDeg, kCntBase = 2 * kCntDeg, kCntLen = 3 * kCntDeg;
constexpr int kCntWords = 3 * kCntDeg + BitmapLaunch::kTiers;

// pass 1: degree histogram of block-tier start vertices, and the level-1 extensions (v0, v1) of
// every start vertex this engine serves (the reference counts one per scattered v1, engine.cc:924)
__global__ void classify_count_kernel(const BJob *__restrict__ jobs, int n_jobs, uint64_t n_total,
                                      uint32_t warp_max, unsigned int *cnt, uint64_t *rows_out) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;  // a multiple of 32: whole warps iterate together
    for (uint64_t gv = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; gv < ((n_total + 31) & ~31ull);
         gv += stride) {
        int j = -1;
        uint32_t d = 0;
        if (gv < n_total) {
            j = job_of(jobs, n_jobs, gv);
            const uint32_t v = (uint32_t)(gv - jobs[j].vbase);
            d = jobs[j].start.keep(v) ? odeg(jobs[j].off, v) : 0u;  // a filtered-out start vertex extends nothing
            if (d > warp_max && d <= (uint32_t)kBlockMax) atomicAdd(&cnt[d], 1u);
        }
        // one atomic per distinct job per warp
        const unsigned peers = __match_any_sync(kFull, j);
        const uint64_t mine = (j >= 0 && d <= (uint32_t)kBlockMax) ? d : 0;
        uint64_t sum = 0;
        for (int l = 0; l < 32; ++l) {
            const uint64_t v = __shfl_sync(kFull, mine, l);
            if ((peers >> l) & 1u) sum += v;
        }
        if (j >= 0 && (int)lane_id() == __ffs(peers) - 1 && sum)
            atomicAdd((unsigned long long *)&row_of(rows_out, jobs[j])[KHZ_MAX_COUNTS], (unsigned long long)sum);
    }
}

__global__ void classify_prefix_kernel(unsigned int *cnt, uint32_t warp_max) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int t = 0; t < BitmapLaunch::kTiers; ++t) {
        unsigned int acc = 0;
        for (int d = tier_hi(t); d > tier_lo(t, (int)warp_max); --d) {
            cnt[kCntBase + d] = acc;
            acc += cnt[d];
        }
        cnt[kCntLen + t] = acc;
    }
}

// pass 2: write each block-tier start vertex at its place in its list
__global__ void classify_write_kernel(const BJob *__restrict__ jobs, int n_jobs, uint64_t n_total,
                                      uint32_t warp_max, unsigned int *cnt, uint32_t *list0, uint32_t *list1,
                                      uint32_t *list2) {
    for (uint64_t gv = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; gv < n_total;
         gv += (uint64_t)gridDim.x * blockDim.x) {
        const int j = job_of(jobs, n_jobs, gv);
        const uint32_t v = (uint32_t)(gv - jobs[j].vbase);
        if (!jobs[j].start.keep(v)) continue;
        const uint32_t d = odeg(jobs[j].off, v);
        if (d <= warp_max || d > (uint32_t)kBlockMax) continue;
        const unsigned int pos = cnt[kCntBase + d] + atomicAdd(&cnt[kCntCursor + d], 1u);
        const int t = tier_of(d);
        (t == 0 ? list0 : (t == 1 ? list1 : list2))[pos] = (uint32_t)gv;
    }
}

}  // namespace

uint32_t bitmap_block_max_degree() { return kBlockMax; }

uint32_t bitmap_hub_rows(int cfg_rows, uint32_t n, uint64_t m) {
    if (cfg_rows < 0) return 0;
    const uint32_t want = cfg_rows == 0 ? (m >= kHubMinEdges ? kHubRowsAuto : 0u) : (uint32_t)cfg_rows;
    return std::min(want, n) & ~31u;
}

static size_t hub_words(uint32_t rows) { return rows ? (size_t)hub_row_offset(rows, rows >> 5) : 0; }
size_t bitmap_hub_bytes(uint32_t rows) { return sizeof(uint32_t) * hub_words(rows); }

size_t bitmap_arena_bytes(const std::vector<BJob> &jobs, uint64_t list_cap) {
    size_t b = Arena::round(sizeof(BJob) * std::max<size_t>(jobs.size(), 1)) +
               BitmapLaunch::kTiers * Arena::round(sizeof(uint32_t) * std::max<uint64_t>(list_cap, 1)) +
               Arena::round(sizeof(unsigned int) * kCntWords) + Arena::round(sizeof(unsigned long long) * 4);
    for (const auto &j : jobs) b += Arena::round(sizeof(uint32_t) * hub_words(j.hub_rows));
    return b;
}

khz_status bitmap_prepare(const std::vector<BJob> &jobs, uint32_t max_outdeg, uint64_t list_cap, bool stats,
                          int warp_max, bool tensor_cores, Arena *arena, BitmapLaunch *bl, cudaStream_t s) {
    BitmapLaunch L;
    L.warp_max = warp_max == 32 ? 32u : (uint32_t)kWarpMax;
    L.kmax = 4;
    for (const auto &j : jobs) L.kmax = std::max(L.kmax, (int)j.k);
    L.n_jobs = (int)jobs.size();
    L.n_total = jobs.empty() ? 0 : jobs.back().vbase + jobs.back().n;
    L.stats = stats;
    if (L.n_total >= (1ull << 32)) {
        set_error("a bitmap launch serves at most 2^32 - 1 start vertices (got %llu)", (unsigned long long)L.n_total);
        return KHZ_ERR_ARG;
    }
    BJob *d_jobs = arena->take<BJob>(jobs.size());
    bool lists_ok = true;
    for (int t = 0; t < BitmapLaunch::kTiers; ++t) {
        L.lists[t] = arena->take<uint32_t>(list_cap);
        lists_ok = lists_ok && L.lists[t];
    }
    L.cnt = arena->take<unsigned int>(kCntWords);
    L.queues = arena->take<unsigned long long>(4);
    if (!d_jobs || !lists_ok || !L.cnt || !L.queues) {
        set_error("bitmap launch arena too small");
        return KHZ_ERR_OOM;
    }
    std::vector<BJob> dj(jobs);
    for (auto &j : dj) {
        j.hub = nullptr;
        if (!j.hub_rows) continue;
        uint32_t *h = arena->take<uint32_t>(hub_words(j.hub_rows));
        if (!h) {
            set_error("bitmap launch arena too small");
            return KHZ_ERR_OOM;
        }
        j.hub = h;
        L.hubs.push_back(j);
    }
    if (!dj.empty())
        KHZ_CUDA(cudaMemcpyAsync(d_jobs, dj.data(), sizeof(BJob) * dj.size(), cudaMemcpyHostToDevice, s));
    L.d_jobs = d_jobs;
    int dev = 0;
    KHZ_CUDA(cudaGetDevice(&dev));
    KHZ_CUDA(cudaDeviceGetAttribute(&L.sms, cudaDevAttrMultiProcessorCount, dev));
    int optin = 0;
    KHZ_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const size_t smem_optin = (size_t)optin;
    // each tier's shared memory is sized for the largest degree it serves in this launch
    const int dcaps[BitmapLaunch::kTiers] = {
        kMidMax, (int)std::min<uint32_t>((uint32_t)kLargeAMax, std::max<uint32_t>(max_outdeg, kMidMax + 1)),
        (int)std::min<uint32_t>((uint32_t)kBlockMax, std::max<uint32_t>(max_outdeg, kLargeAMax + 1))};
    const int threads[BitmapLaunch::kTiers] = {kMidThreads, kLargeAThreads, kLargeThreads};
    for (int t = 0; t < BitmapLaunch::kTiers; ++t) {
        L.has_tier[t] = max_outdeg > (uint32_t)tier_lo(t, (int)L.warp_max);
        // large tiers: the most accumulator tiles per pass whose tensor memory fits every block
        // resident on an SM at once (512 columns per SM; an allocation would otherwise wait)
        int g = (t > 0 && tensor_cores && !stats) ? (t == 2 ? kMmaMaxTiles : 2) : 0;
        size_t smem = 0;
        int per_sm = 0;
        BlockKernel kern = nullptr;
        for (;; --g) {
            kern = block_kernel(stats, L.kmax, t, g > 0);
            // the attribute is per kernel, shared by every prepared launch: always allow the largest
            // footprint (up to the device's opt-in limit) so launches prepared earlier with more
            // shared memory stay valid
            cudaFuncAttributes fa;
            KHZ_CUDA(cudaFuncGetAttributes(&fa, kern));
            const size_t dyn_max = smem_optin - std::min(smem_optin, (size_t)fa.sharedSizeBytes);  // less static
            KHZ_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)std::min(block_smem(kBlockMax, 1024, kMmaMaxTiles), dyn_max)));
            smem = block_smem(dcaps[t], threads[t], g);
            per_sm = 0;
            if (smem <= dyn_max)
                KHZ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads[t], smem));
            if (g == 0 || (per_sm >= 1 && per_sm * (int)mma_tmem_cols(g) <= 512)) break;
        }
        if (per_sm < 1) {
            set_error("bitmap block kernel does not fit an SM (%d threads, %zu bytes of shared memory)", threads[t], smem);
            return KHZ_ERR_CUDA;
        }
        L.block_smem[t] = smem;
        L.block_threads[t] = threads[t];
        L.block_grid[t] = L.sms * std::max(per_sm, 1);
        L.block_dcap[t] = dcaps[t];
        L.block_mma_g[t] = g;
    }
    *bl = L;
    return KHZ_OK;
}

khz_status bitmap_enqueue(const BitmapLaunch &L, uint64_t *d_rows, cudaStream_t s, LaunchStats *ls,
                          unsigned int *d_err) {
    if (L.n_jobs == 0 || L.n_total == 0) return KHZ_OK;
    auto pb = [&](int phase) -> uint64_t * { return ls && ls->d_phase_bytes ? ls->d_phase_bytes + phase : nullptr; };
    auto mark = [&](int phase, bool begin) {
        if (!ls || !ls->ev_begin) return;
        cudaEventRecord(begin ? ls->ev_begin[phase] : ls->ev_end[phase], s);
        if (!begin) {
            ls->used[phase] = true;
            ls->phase_launches[phase] += 1;
        }
    };
    KHZ_CUDA(cudaMemsetAsync(L.cnt, 0, sizeof(unsigned int) * kCntWords, s));
    KHZ_CUDA(cudaMemsetAsync(L.queues, 0, sizeof(unsigned long long) * 4, s));
    for (const auto &j : L.hubs) {
        KHZ_CUDA(cudaMemsetAsync(const_cast<uint32_t *>(j.hub), 0, sizeof(uint32_t) * hub_words(j.hub_rows), s));
        hub_build_kernel<<<std::max(1, std::min<int>(L.sms * 8, (int)(j.hub_rows / 8))), 256, 0, s>>>(
            j.off, j.adj, j.n, j.hub_rows, const_cast<uint32_t *>(j.hub));
        if (ls) ls->launches += 1;
    }
    const int cgrid = (int)std::max<uint64_t>(1, std::min<uint64_t>((L.n_total + 255) / 256, (uint64_t)L.sms * 8));
    classify_count_kernel<<<cgrid, 256, 0, s>>>(L.d_jobs, L.n_jobs, L.n_total, L.warp_max, L.cnt, d_rows);
    if (L.has_tier[0]) {
        classify_prefix_kernel<<<1, 32, 0, s>>>(L.cnt, L.warp_max);
        classify_write_kernel<<<cgrid, 256, 0, s>>>(L.d_jobs, L.n_jobs, L.n_total, L.warp_max, L.cnt, L.lists[0],
                                                    L.lists[1], L.lists[2]);
    }
    KHZ_CUDA(cudaGetLastError());
    if (ls) ls->launches += L.has_tier[0] ? 3 : 1;
    mark(0, true);
    {
        auto wk = L.stats ? (L.kmax == 5 ? clique_warp_kernel<true, 5> : clique_warp_kernel<true, 4>)
                          : (L.kmax == 5 ? clique_warp_kernel<false, 5> : clique_warp_kernel<false, 4>);
        wk<<<L.sms * 8, 256, 0, s>>>(L.d_jobs, L.n_jobs, L.n_total, L.stats ? 1u : 2u, L.warp_max, &L.queues[0], d_rows,
                                     pb(0));
    }
    KHZ_CUDA(cudaGetLastError());
    mark(0, false);
    if (ls) ls->launches += 1;
    // phases: the mid tier is phase 1, the two large tiers together phase 2
    const int last_large = L.has_tier[2] ? 2 : 1;
    for (int t = 0; t < BitmapLaunch::kTiers; ++t) {
        if (!L.has_tier[t]) continue;
        const int phase = t == 0 ? 1 : 2;
        if (t != 2 || !L.has_tier[1]) mark(phase, true);
        const BlockKernel bk = block_kernel(L.stats, L.kmax, t, L.block_mma_g[t] > 0);
        bk<<<L.block_grid[t], L.block_threads[t], L.block_smem[t], s>>>(
            L.d_jobs, L.n_jobs, L.lists[t], L.cnt + kCntLen + t, L.block_dcap[t], &L.queues[1 + t], d_rows, pb(phase),
            L.block_mma_g[t], d_err);
        KHZ_CUDA(cudaGetLastError());
        if (t == 0 || t == last_large) mark(phase, false);
        if (ls) ls->launches += 1;
    }
    return KHZ_OK;
}

}  // namespace khz
