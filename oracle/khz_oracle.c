/*
 * CPU oracle for the Khuzdul embedding-extension path — TEST INFRASTRUCTURE ONLY.
 * See khz_oracle.h for who may call it and how it is pinned.  Every routine below
 * restates one reference routine; the reference file:line is given beside it.
 */
#define _GNU_SOURCE
#include "khz_oracle.h"

#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------- */
/* generators                                                                */
/* ------------------------------------------------------------------------- */

/* splitmix64 finaliser (Steele, Lea, Flood 2014): a bijective 64-bit mixer. */
uint64_t orc_mix64(uint64_t x) {
    uint64_t z = x + 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

/* R-MAT (Chakrabarti, Zhan, Faloutsos 2004): one quadrant draw per bit level,
 * most significant bit first; draw (i, l) = mix64(mix64(seed) ^ (64 i + l)). */
void orc_rmat_raw_edge(int scale, uint64_t seed, uint32_t ta, uint32_t tab, uint32_t tabc, uint64_t i,
                       uint32_t *src, uint32_t *dst) {
    uint64_t base = orc_mix64(seed);
    uint32_t s = 0, d = 0;
    for (int l = 0; l < scale; ++l) {
        uint32_t u = (uint32_t)(orc_mix64(base ^ (i * 64u + (uint64_t)l)) >> 32);
        uint32_t sb, db;
        if (u < ta) { sb = 0; db = 0; }
        else if (u < tab) { sb = 0; db = 1; }
        else if (u < tabc) { sb = 1; db = 0; }
        else { sb = 1; db = 1; }
        s |= sb << (scale - 1 - l);
        d |= db << (scale - 1 - l);
    }
    *src = s;
    *dst = d;
}

static void radix_sort_u64(uint64_t *keys, uint64_t n) {
    uint64_t *tmp = (uint64_t *)malloc(sizeof(uint64_t) * (n ? n : 1));
    uint64_t *cnt = (uint64_t *)malloc(sizeof(uint64_t) * 65536);
    uint64_t *src = keys, *dst = tmp;
    for (int pass = 0; pass < 4; ++pass) {
        int sh = pass * 16;
        memset(cnt, 0, sizeof(uint64_t) * 65536);
        for (uint64_t i = 0; i < n; ++i) cnt[(src[i] >> sh) & 0xffff]++;
        uint64_t acc = 0;
        for (int b = 0; b < 65536; ++b) { uint64_t c = cnt[b]; cnt[b] = acc; acc += c; }
        for (uint64_t i = 0; i < n; ++i) dst[cnt[(src[i] >> sh) & 0xffff]++] = src[i];
        uint64_t *t = src; src = dst; dst = t;
    }
    /* 4 passes: result is back in keys */
    free(tmp);
    free(cnt);
}

/* sorted canonical keys (u << 32 | v, u < v, unique) -> compacted pairs; returns n */
static uint32_t compact_pairs(const uint64_t *keys, uint64_t m, uint32_t id_space, uint32_t *pairs_out) {
    uint8_t *present = (uint8_t *)calloc(id_space ? id_space : 1, 1);
    uint32_t *newid = (uint32_t *)malloc(sizeof(uint32_t) * (id_space ? id_space : 1));
    for (uint64_t i = 0; i < m; ++i) { present[keys[i] >> 32] = 1; present[(uint32_t)keys[i]] = 1; }
    uint32_t n = 0;
    for (uint32_t v = 0; v < id_space; ++v) { newid[v] = n; n += present[v]; }
    for (uint64_t i = 0; i < m; ++i) {
        pairs_out[2 * i] = newid[keys[i] >> 32];
        pairs_out[2 * i + 1] = newid[(uint32_t)keys[i]];
    }
    free(present);
    free(newid);
    return n;
}

uint64_t orc_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                  uint32_t *pairs_out, uint64_t cap, uint32_t *n_out) {
    uint64_t raw = (uint64_t)edge_factor << scale;
    uint32_t ta = (uint32_t)(a * 4294967296.0);
    uint32_t tab = (uint32_t)((a + b) * 4294967296.0);
    uint32_t tabc = (uint32_t)((a + b + c) * 4294967296.0);
    uint64_t *keys = (uint64_t *)malloc(sizeof(uint64_t) * (raw ? raw : 1));
    uint64_t k = 0;
    for (uint64_t i = 0; i < raw; ++i) {
        uint32_t s, d;
        orc_rmat_raw_edge(scale, seed, ta, tab, tabc, i, &s, &d);
        if (s == d) continue;
        uint32_t lo = s < d ? s : d, hi = s < d ? d : s;
        keys[k++] = ((uint64_t)lo << 32) | hi;
    }
    radix_sort_u64(keys, k);
    uint64_t m = 0;
    for (uint64_t i = 0; i < k; ++i)
        if (i == 0 || keys[i] != keys[i - 1]) keys[m++] = keys[i];
    if (m > cap) { free(keys); return UINT64_MAX; }
    *n_out = compact_pairs(keys, m, scale >= 32 ? 0xffffffffu : (1u << scale), pairs_out);
    free(keys);
    return m;
}

uint64_t orc_er(uint32_t n, uint64_t m, uint64_t seed, uint32_t *pairs_out, uint32_t *n_out) {
    uint64_t base = orc_mix64(seed);
    uint64_t cap = 1;
    while (cap < 2 * m + 16) cap <<= 1;
    uint64_t *table = (uint64_t *)malloc(sizeof(uint64_t) * cap);
    memset(table, 0xff, sizeof(uint64_t) * cap);
    uint64_t *keys = (uint64_t *)malloc(sizeof(uint64_t) * (m ? m : 1));
    uint64_t got = 0;
    for (uint64_t k = 0; got < m; ++k) {
        uint64_t r1 = orc_mix64(base ^ (2 * k)), r2 = orc_mix64(base ^ (2 * k + 1));
        uint32_t u = (uint32_t)(((r1 >> 32) * (uint64_t)n) >> 32);
        uint32_t v = (uint32_t)(((r2 >> 32) * (uint64_t)n) >> 32);
        if (u == v) continue;
        uint32_t lo = u < v ? u : v, hi = u < v ? v : u;
        uint64_t key = ((uint64_t)lo << 32) | hi;
        uint64_t h = orc_mix64(key) & (cap - 1);
        int dup = 0;
        while (table[h] != UINT64_MAX) {
            if (table[h] == key) { dup = 1; break; }
            h = (h + 1) & (cap - 1);
        }
        if (dup) continue;
        table[h] = key;
        keys[got++] = key;
    }
    radix_sort_u64(keys, m);
    *n_out = compact_pairs(keys, m, n, pairs_out);
    free(table);
    free(keys);
    return m;
}

/* both directions, sorted by (src, dst): the converter's reverse-edge + counting sorts
 * (toolkits/converter.cc:52-131) */
void orc_symmetrize(const uint32_t *canon, uint64_t m, uint32_t *out) {
    uint64_t *keys = (uint64_t *)malloc(sizeof(uint64_t) * (2 * m + 1));
    for (uint64_t i = 0; i < m; ++i) {
        keys[2 * i] = ((uint64_t)canon[2 * i] << 32) | canon[2 * i + 1];
        keys[2 * i + 1] = ((uint64_t)canon[2 * i + 1] << 32) | canon[2 * i];
    }
    radix_sort_u64(keys, 2 * m);
    for (uint64_t i = 0; i < 2 * m; ++i) { out[2 * i] = (uint32_t)(keys[i] >> 32); out[2 * i + 1] = (uint32_t)keys[i]; }
    free(keys);
}

/* ------------------------------------------------------------------------- */
/* .dgraph: 20-byte packed header {u32 n; u64 m; i32 has_node_label; i32 has_edge_label},
 * optional u32 labels[n], then m packed (u32 src, u32 dst) (graph_loader.h:31-42)       */
/* ------------------------------------------------------------------------- */
int orc_dgraph_header(const char *path, uint32_t *n, uint64_t *m, int32_t *has_node_label) {
    FILE *f = fopen(path, "rb");
    if (!f) return -1;
    unsigned char h[20];
    size_t r = fread(h, 1, 20, f);
    fclose(f);
    if (r != 20) return -2;
    memcpy(n, h, 4);
    memcpy(m, h + 4, 8);
    memcpy(has_node_label, h + 12, 4);
    return 0;
}

int orc_dgraph_read(const char *path, uint32_t *labels_or_null, uint32_t *pairs) {
    uint32_t n; uint64_t m; int32_t hl;
    if (orc_dgraph_header(path, &n, &m, &hl)) return -1;
    FILE *f = fopen(path, "rb");
    if (!f) return -1;
    fseek(f, 20, SEEK_SET);
    if (hl) {
        if (labels_or_null) { if (fread(labels_or_null, 4, n, f) != n) { fclose(f); return -2; } }
        else fseek(f, 20 + 4 * (long)n, SEEK_SET);
    }
    if (fread(pairs, 8, m, f) != m) { fclose(f); return -3; }
    fclose(f);
    return 0;
}

int orc_dgraph_write(const char *path, uint32_t n, uint64_t m, const uint32_t *labels_or_null,
                     const uint32_t *pairs) {
    FILE *f = fopen(path, "wb");
    if (!f) return -1;
    unsigned char h[20];
    int32_t hl = labels_or_null ? 1 : 0, he = 0;
    memcpy(h, &n, 4);
    memcpy(h + 4, &m, 8);
    memcpy(h + 12, &hl, 4);
    memcpy(h + 16, &he, 4);
    int ok = fwrite(h, 1, 20, f) == 20;
    if (labels_or_null) ok = ok && fwrite(labels_or_null, 4, n, f) == n;
    ok = ok && fwrite(pairs, 8, m, f) == m;
    fclose(f);
    return ok ? 0 : -2;
}

/* ------------------------------------------------------------------------- */
/* CSR build: CSRGraphLoader::construct_csr_format_for_empty (graph_loader.h:154-201);
 * the input must be sorted by (src, dst) with no duplicates (graph_loader.h:31-35). */
/* ------------------------------------------------------------------------- */
int orc_csr_from_edges(const uint32_t *pairs, uint64_t m, uint32_t n, uint64_t *off, uint32_t *adj) {
    memset(off, 0, sizeof(uint64_t) * ((uint64_t)n + 1));
    for (uint64_t i = 0; i < m; ++i) {
        uint32_t s = pairs[2 * i], d = pairs[2 * i + 1];
        if (s >= n || d >= n) return -1;
        if (i > 0) {
            uint64_t pk = ((uint64_t)pairs[2 * i - 2] << 32) | pairs[2 * i - 1];
            uint64_t ck = ((uint64_t)s << 32) | d;
            if (ck <= pk) return -2;
        }
        off[s + 1]++;
        adj[i] = d;
    }
    for (uint32_t v = 0; v < n; ++v) off[v + 1] += off[v];
    return 0;
}

/* Degree orientation: to_oriented_dataset_converter.cc:27-124.  Vertices are ranked by
 * (degree, id) ascending (:40-53), relabelled (:62-67), and rank r keeps the relabelled
 * neighbours > r, sorted (:84-112). */
typedef struct { uint32_t deg, vtx; } orc_degvtx;
static int cmp_degvtx(const void *x, const void *y) {
    const orc_degvtx *a = (const orc_degvtx *)x, *b = (const orc_degvtx *)y;
    if (a->deg != b->deg) return a->deg < b->deg ? -1 : 1;
    return a->vtx < b->vtx ? -1 : (a->vtx > b->vtx);
}
static int cmp_u32(const void *x, const void *y) {
    uint32_t a = *(const uint32_t *)x, b = *(const uint32_t *)y;
    return a < b ? -1 : (a > b);
}
int orc_orient(uint32_t n, const uint64_t *off, const uint32_t *adj, uint64_t *ooff, uint32_t *oadj,
               uint32_t *rank_out) {
    orc_degvtx *dv = (orc_degvtx *)malloc(sizeof(orc_degvtx) * (n ? n : 1));
    uint32_t *map = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    for (uint32_t v = 0; v < n; ++v) { dv[v].deg = (uint32_t)(off[v + 1] - off[v]); dv[v].vtx = v; }
    qsort(dv, n, sizeof(orc_degvtx), cmp_degvtx);
    for (uint32_t r = 0; r < n; ++r) map[dv[r].vtx] = r;
    uint64_t e = 0;
    ooff[0] = 0;
    for (uint32_t r = 0; r < n; ++r) {
        uint32_t u = dv[r].vtx;
        uint64_t start = e;
        for (uint64_t i = off[u]; i < off[u + 1]; ++i) {
            uint32_t d = map[adj[i]];
            if (d > r) oadj[e++] = d;
        }
        qsort(oadj + start, e - start, sizeof(uint32_t), cmp_u32);
        ooff[r + 1] = e;
    }
    if (rank_out) memcpy(rank_out, map, sizeof(uint32_t) * n);
    free(dv);
    free(map);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* VertexSet algebra                                                          */
/* ------------------------------------------------------------------------- */
/* VertexSet::intersect_with, vertex_set.cc:20-49 (merge; result sorted) */
uint32_t orc_intersect(const uint32_t *a, uint32_t na, const uint32_t *b, uint32_t nb, uint32_t *out) {
    if (na == 0 || nb == 0) return 0;
    uint32_t j = 0, r = 0;
    for (uint32_t i = 0; i < na; ++i) {
        uint32_t v = a[i];
        while (j < nb && b[j] < v) ++j;
        if (j < nb && b[j] == v) { out[r++] = v; ++j; }
    }
    return r;
}
/* VertexSet::subtracted_by, vertex_set.cc:51-86 */
uint32_t orc_subtract(const uint32_t *a, uint32_t na, const uint32_t *b, uint32_t nb, uint32_t *out) {
    if (na == 0) return 0;
    uint32_t j = 0, r = 0;
    for (uint32_t i = 0; i < na; ++i) {
        uint32_t v = a[i];
        int found = 0;
        while (j < nb) {
            if (b[j] == v) { found = 1; ++j; break; }
            if (b[j] > v) break;
            ++j;
        }
        if (!found) out[r++] = v;
    }
    return r;
}
/* VertexSet::intersect_and_count, vertex_set.cc:88-111 */
uint32_t orc_intersect_count(const uint32_t *a, uint32_t na, const uint32_t *b, uint32_t nb) {
    if (na == 0 || nb == 0) return 0;
    uint32_t j = 0, r = 0;
    for (uint32_t i = 0; i < na; ++i) {
        uint32_t v = a[i];
        while (j < nb && b[j] < v) ++j;
        if (j < nb && b[j] == v) { ++r; ++j; }
    }
    return r;
}
/* VertexSet::bounded_intersect_with, vertex_set.cc:113-144 (stops at the first a[i] >= ub) */
uint32_t orc_bounded_intersect(const uint32_t *a, uint32_t na, const uint32_t *b, uint32_t nb, uint32_t ub,
                               uint32_t *out) {
    if (na == 0 || nb == 0) return 0;
    uint32_t j = 0, r = 0;
    for (uint32_t i = 0; i < na; ++i) {
        uint32_t v = a[i];
        if (v >= ub) break;
        while (j < nb && b[j] < v) ++j;
        if (j < nb && b[j] == v) { out[r++] = v; ++j; }
    }
    return r;
}
/* VertexSet::bounded_subtracted_by, vertex_set.cc:146-184 */
uint32_t orc_bounded_subtract(const uint32_t *a, uint32_t na, const uint32_t *b, uint32_t nb, uint32_t ub,
                              uint32_t *out) {
    if (na == 0) return 0;
    uint32_t j = 0, r = 0;
    for (uint32_t i = 0; i < na; ++i) {
        uint32_t v = a[i];
        if (v >= ub) break;
        int found = 0;
        while (j < nb) {
            if (b[j] == v) { found = 1; ++j; break; }
            if (b[j] > v) break;
            ++j;
        }
        if (!found) out[r++] = v;
    }
    return r;
}
/* trim_v_list, utilities.h:64-74: number of elements < upper_bound */
uint32_t orc_trim(const uint32_t *a, uint32_t na, uint32_t upper_bound) {
    if (na == 0 || a[0] >= upper_bound) return 0;
    if (a[na - 1] < upper_bound) return na;
    uint32_t l = 0, r = na;
    while (r - l > 1) {
        uint32_t mid = (l + r) >> 1;
        if (a[mid] < upper_bound) l = mid; else r = mid;
    }
    return l + 1;
}
/* trim_v_list_lower_bound, utilities.h:76-86: number of elements <= lower_bound */
uint32_t orc_trim_lower_bound(const uint32_t *a, uint32_t na, uint32_t lower_bound) {
    if (na == 0 || a[na - 1] <= lower_bound) return na;
    if (a[0] > lower_bound) return 0;
    uint32_t l = 0, r = na;
    while (r - l > 1) {
        uint32_t mid = (l + r) >> 1;
        if (a[mid] <= lower_bound) l = mid; else r = mid;
    }
    return l + 1;
}
/* std::binary_search as used by the kgraphpi last levels (kgraphpi/four_clique.cc:135-143) */
static int bsearch_u32(const uint32_t *a, uint32_t na, uint32_t x) {
    uint32_t l = 0, r = na;
    while (l < r) {
        uint32_t mid = (l + r) >> 1;
        if (a[mid] < x) l = mid + 1; else r = mid;
    }
    return l < na && a[l] == x;
}

/* ------------------------------------------------------------------------- */
/* pattern schedules                                                          */
/* ------------------------------------------------------------------------- */
typedef struct {
    const uint64_t *off;
    const uint32_t *adj;
    uint32_t *buf[5]; /* per-level prefix buffers (max degree each) */
    uint64_t cnt[6];
    uint64_t ext;
    uint64_t bytes;
} orc_tc;

#define NB(v) (t->adj + t->off[v])
#define DG(v) ((uint32_t)(t->off[(v) + 1] - t->off[v]))

static inline uint32_t op_and(orc_tc *t, const uint32_t *a, uint32_t na, const uint32_t *b, uint32_t nb, uint32_t *o) {
    uint32_t r = orc_intersect(a, na, b, nb, o);
    t->bytes += 4ull * ((uint64_t)na + nb + r);
    return r;
}
static inline uint32_t op_sub(orc_tc *t, const uint32_t *a, uint32_t na, const uint32_t *b, uint32_t nb, uint32_t *o) {
    uint32_t r = orc_subtract(a, na, b, nb, o);
    t->bytes += 4ull * ((uint64_t)na + nb + r);
    return r;
}

/* kautomine/triangle.cc:58-121 */
static void kauto_triangle(orc_tc *t, uint32_t v0) {
    t->ext++;
    const uint32_t *p0 = NB(v0); uint32_t n0 = DG(v0);
    for (uint32_t i = 0; i < n0; ++i) {
        uint32_t v1 = p0[i];
        if (!(v1 > v0)) continue;
        t->ext++;
        uint32_t n1 = op_and(t, p0, n0, NB(v1), DG(v1), t->buf[1]);
        uint64_t c = 0;
        for (uint32_t k = 0; k < n1; ++k) c += t->buf[1][k] > v1;
        t->cnt[0] += c;
    }
}

/* kautomine/four_clique.cc:58-153 and five_clique.cc:58-186 (k = 4, 5) */
static void kauto_clique(orc_tc *t, uint32_t v0, int k) {
    t->ext++;
    const uint32_t *p0 = NB(v0); uint32_t n0 = DG(v0);
    for (uint32_t i = 0; i < n0; ++i) {
        uint32_t v1 = p0[i];
        if (!(v1 > v0)) continue;
        t->ext++;
        uint32_t *p1 = t->buf[1];
        uint32_t n1 = op_and(t, p0, n0, NB(v1), DG(v1), p1);
        for (uint32_t j = 0; j < n1; ++j) {
            uint32_t v2 = p1[j];
            if (!(v2 > v1)) continue;
            t->ext++;
            uint32_t *p2 = t->buf[2];
            uint32_t n2 = op_and(t, p1, n1, NB(v2), DG(v2), p2);
            if (k == 4) {
                uint64_t c = 0;
                for (uint32_t x = 0; x < n2; ++x) c += p2[x] > v2;
                t->cnt[0] += c;
                continue;
            }
            for (uint32_t l = 0; l < n2; ++l) {
                uint32_t v3 = p2[l];
                if (!(v3 > v2)) continue;
                t->ext++;
                uint32_t *p3 = t->buf[3];
                uint32_t n3 = op_and(t, p2, n2, NB(v3), DG(v3), p3);
                uint64_t c = 0;
                for (uint32_t x = 0; x < n3; ++x) c += p3[x] > v3;
                t->cnt[0] += c;
            }
        }
    }
}

/* kautomine/three_motif.cc:59-138 (compute-fused; multiplicities {1, 2} at :44) */
static void kauto_3motif(orc_tc *t, uint32_t v0) {
    t->ext++;
    const uint32_t *p0 = NB(v0); uint32_t n0 = DG(v0);
    for (uint32_t i = 0; i < n0; ++i) {
        uint32_t v1 = p0[i];
        t->ext++;
        if (v0 < v1) {
            uint32_t n1 = op_and(t, p0, n0, NB(v1), DG(v1), t->buf[1]);
            uint64_t c = 0;
            for (uint32_t x = 0; x < n1; ++x) c += t->buf[1][x] > v1;
            t->cnt[0] += c;
        }
        uint32_t n2 = op_sub(t, p0, n0, NB(v1), DG(v1), t->buf[2]);
        uint64_t c = 0;
        for (uint32_t x = 0; x < n2; ++x) c += t->buf[2][x] != v1;
        t->cnt[1] += c;
    }
}

/* kgraphpi last level: |{x in P : x > lb}| minus the matched vertices found in that tail
 * (kgraphpi/four_clique.cc:131-143) */
static inline uint64_t kgpi_tail(const uint32_t *p, uint32_t np, uint32_t lb, const uint32_t *ex, int nex) {
    uint32_t tr = orc_trim_lower_bound(p, np, lb);
    uint64_t c = np - tr;
    for (int e = 0; e < nex; ++e) c -= bsearch_u32(p + tr, np - tr, ex[e]);
    return c;
}

/* kgraphpi/triangle.cc:53-122 */
static void kgpi_triangle(orc_tc *t, uint32_t v0, int slot) {
    t->ext++;
    const uint32_t *p0 = NB(v0); uint32_t n0 = DG(v0);
    for (uint32_t i = 0; i < n0; ++i) {
        uint32_t v1 = p0[i];
        if (v1 <= v0) continue;
        if (!(v1 != v0)) continue;
        t->ext++;
        uint32_t n1 = op_and(t, p0, n0, NB(v1), DG(v1), t->buf[1]);
        uint32_t ex[2] = {v0, v1};
        t->cnt[slot] += kgpi_tail(t->buf[1], n1, v1, ex, 2);
    }
}

/* kgraphpi/four_clique.cc:53-159 and five_clique.cc:53-195 */
static void kgpi_clique(orc_tc *t, uint32_t v0, int k) {
    t->ext++;
    const uint32_t *p0 = NB(v0); uint32_t n0 = DG(v0);
    for (uint32_t i = 0; i < n0; ++i) {
        uint32_t v1 = p0[i];
        if (v1 <= v0 || v1 == v0) continue;
        t->ext++;
        uint32_t *p1 = t->buf[1];
        uint32_t n1 = op_and(t, p0, n0, NB(v1), DG(v1), p1);
        for (uint32_t j = 0; j < n1; ++j) {
            uint32_t v2 = p1[j];
            if (v2 <= v1) continue;
            if (!(v2 != v0 && v2 != v1)) continue;
            t->ext++;
            uint32_t *p2 = t->buf[2];
            uint32_t n2 = op_and(t, p1, n1, NB(v2), DG(v2), p2);
            if (k == 4) {
                uint32_t lb = v0 > v2 ? v0 : v2;
                uint32_t ex[3] = {v0, v1, v2};
                t->cnt[0] += kgpi_tail(p2, n2, lb, ex, 3);
                continue;
            }
            for (uint32_t l = 0; l < n2; ++l) {
                uint32_t v3 = p2[l];
                if (v3 <= v0 || v3 <= v2) continue;
                if (!(v3 != v0 && v3 != v1 && v3 != v2)) continue;
                t->ext++;
                uint32_t *p3 = t->buf[3];
                uint32_t n3 = op_and(t, p2, n2, NB(v3), DG(v3), p3);
                uint32_t lb = v1 > v3 ? v1 : v3;
                uint32_t ex[4] = {v0, v1, v2, v3};
                t->cnt[0] += kgpi_tail(p3, n3, lb, ex, 4);
            }
        }
    }
}

/* kgraphpi/three_motif.cc:123-163, pattern 1: edge-induced wedge centred at v0; the
 * size-1 -> 2 step is a finalized scatter (engine.cc:1441-1452), so it adds no extension. */
static void kgpi_wedge(orc_tc *t, uint32_t v0) {
    t->ext++;
    const uint32_t *p0 = NB(v0); uint32_t n0 = DG(v0);
    for (uint32_t i = 0; i < n0; ++i) {
        uint32_t v1 = p0[i];
        if (!(v1 != v0)) continue;
        uint32_t ex[2] = {v0, v1};
        t->cnt[1] += kgpi_tail(p0, n0, v1, ex, 2);
    }
}

/* 4-cycle v0-v1-v2-v3-v0 (edge-induced), written in the kgraphpi idiom.  Restrictions
 * v1 > v0, v2 > v0, v3 > v1 break the 8 automorphisms (v0 is the cycle's minimum and
 * v1 < v3 are its two neighbours).  Not in the reference (kgraphpi/CMakeLists.txt:14-18). */
static void kgpi_4cycle(orc_tc *t, uint32_t v0) {
    t->ext++;
    const uint32_t *p0 = NB(v0); uint32_t n0 = DG(v0);
    for (uint32_t i = 0; i < n0; ++i) {
        uint32_t v1 = p0[i];
        if (v1 <= v0) continue;
        t->ext++;
        const uint32_t *q = NB(v1); uint32_t nq = DG(v1);
        for (uint32_t j = 0; j < nq; ++j) {
            uint32_t v2 = q[j];
            if (v2 <= v0) continue;
            if (!(v2 != v0 && v2 != v1)) continue;
            t->ext++;
            uint32_t n2 = op_and(t, p0, n0, NB(v2), DG(v2), t->buf[2]);
            uint32_t ex[3] = {v0, v1, v2};
            t->cnt[0] += kgpi_tail(t->buf[2], n2, v1, ex, 3);
        }
    }
}

/* House: square v0-v1-v2-v3-v0 with roof v4 adjacent to v0 and v1 (edge-induced).
 * v1 > v0 breaks the single non-trivial automorphism; the roof candidates
 * N(v0) n N(v1) are cached at size 2 like kgraphpi's cached prefixes. */
static void kgpi_house(orc_tc *t, uint32_t v0) {
    t->ext++;
    const uint32_t *p0 = NB(v0); uint32_t n0 = DG(v0);
    for (uint32_t i = 0; i < n0; ++i) {
        uint32_t v1 = p0[i];
        if (v1 <= v0) continue;
        t->ext++;
        uint32_t *p1 = t->buf[1];
        uint32_t n1 = op_and(t, p0, n0, NB(v1), DG(v1), p1);
        const uint32_t *q = NB(v1); uint32_t nq = DG(v1);
        for (uint32_t j = 0; j < nq; ++j) {
            uint32_t v2 = q[j];
            if (!(v2 != v0 && v2 != v1)) continue;
            t->ext++;
            uint32_t *p2 = t->buf[2];
            uint32_t n2 = op_and(t, p0, n0, NB(v2), DG(v2), p2);
            for (uint32_t l = 0; l < n2; ++l) {
                uint32_t v3 = p2[l];
                if (!(v3 != v0 && v3 != v1 && v3 != v2)) continue;
                t->ext++;
                uint64_t c = n1;
                c -= bsearch_u32(p1, n1, v0);
                c -= bsearch_u32(p1, n1, v1);
                c -= bsearch_u32(p1, n1, v2);
                c -= bsearch_u32(p1, n1, v3);
                t->cnt[0] += c;
            }
        }
    }
}

/* Tailed triangle: triangle v0 v1 v2 plus tail v3 on v0 (edge-induced); v2 > v1 breaks
 * the swap of v1 and v2. */
static void kgpi_tailed(orc_tc *t, uint32_t v0) {
    t->ext++;
    const uint32_t *p0 = NB(v0); uint32_t n0 = DG(v0);
    for (uint32_t i = 0; i < n0; ++i) {
        uint32_t v1 = p0[i];
        if (!(v1 != v0)) continue;
        t->ext++;
        uint32_t *p1 = t->buf[1];
        uint32_t n1 = op_and(t, p0, n0, NB(v1), DG(v1), p1);
        for (uint32_t j = 0; j < n1; ++j) {
            uint32_t v2 = p1[j];
            if (v2 <= v1) continue;
            if (!(v2 != v0 && v2 != v1)) continue;
            t->ext++;
            uint64_t c = n0;
            c -= bsearch_u32(p0, n0, v0);
            c -= bsearch_u32(p0, n0, v1);
            c -= bsearch_u32(p0, n0, v2);
            t->cnt[0] += c;
        }
    }
}

/* Vertex-induced 4-motifs in the kautomine idiom (kautomine/three_motif.cc:87-127 style:
 * intersect_with / subtracted_by per level, filter loop at the last level).  Patterns run
 * one after another; raw counts are divided by the multiplicities {1, 2, 1, 8, 1, 1}. */
static void kauto_4motif(orc_tc *t, uint32_t v0, int pat) {
    t->ext++;
    const uint32_t *p0 = NB(v0); uint32_t n0 = DG(v0);
    for (uint32_t i = 0; i < n0; ++i) {
        uint32_t v1 = p0[i];
        if ((pat == 4 || pat == 5) && !(v1 > v0)) continue;
        t->ext++;
        const uint32_t *q1 = NB(v1); uint32_t nq1 = DG(v1);
        uint32_t *p1 = t->buf[1], *aux = t->buf[3];
        uint32_t n1, naux = 0;
        if (pat == 0 || pat == 1 || pat == 3) n1 = op_sub(t, p0, n0, q1, nq1, p1);
        else n1 = op_and(t, p0, n0, q1, nq1, p1);
        if (pat == 1) naux = op_sub(t, q1, nq1, p0, n0, aux);   /* N(v1) \ N(v0) */
        if (pat == 2) naux = op_sub(t, p0, n0, q1, nq1, aux);   /* N(v0) \ N(v1) */
        for (uint32_t j = 0; j < n1; ++j) {
            uint32_t v2 = p1[j];
            int ok;
            switch (pat) {
                case 0: ok = v2 > v1; break;
                case 1: ok = v2 != v1; break;
                case 2: ok = v2 > v1; break;
                case 3: ok = v2 != v1; break;
                case 4: ok = 1; break;
                default: ok = v2 > v1; break;
            }
            if (!ok) continue;
            t->ext++;
            const uint32_t *q2 = NB(v2); uint32_t nq2 = DG(v2);
            uint32_t *p2 = t->buf[2];
            uint32_t n2;
            uint64_t c = 0;
            switch (pat) {
                case 0: /* 3-star */
                    n2 = op_sub(t, p1, n1, q2, nq2, p2);
                    for (uint32_t x = 0; x < n2; ++x) c += p2[x] > v2;
                    break;
                case 1: /* 4-path */
                    n2 = op_sub(t, aux, naux, q2, nq2, p2);
                    for (uint32_t x = 0; x < n2; ++x) c += p2[x] != v0;
                    break;
                case 2: /* tailed triangle */
                    n2 = op_sub(t, aux, naux, q2, nq2, p2);
                    for (uint32_t x = 0; x < n2; ++x) c += p2[x] != v1 && p2[x] != v2;
                    break;
                case 3: { /* 4-cycle */
                    uint32_t *tmp = t->buf[4];
                    uint32_t nt = op_and(t, q1, nq1, q2, nq2, tmp);
                    n2 = op_sub(t, tmp, nt, p0, n0, p2);
                    for (uint32_t x = 0; x < n2; ++x) c += p2[x] != v0;
                    break;
                }
                case 4: /* diamond */
                    n2 = op_sub(t, p1, n1, q2, nq2, p2);
                    for (uint32_t x = 0; x < n2; ++x) c += p2[x] > v2;
                    break;
                default: /* 4-clique */
                    n2 = op_and(t, p1, n1, q2, nq2, p2);
                    for (uint32_t x = 0; x < n2; ++x) c += p2[x] > v2;
                    break;
            }
            t->cnt[pat] += c;
        }
    }
}

int orc_num_counts(int app) {
    switch (app) {
        case ORC_KAUTO_3MOTIF: case ORC_KGPI_3MOTIF: return 2;
        case ORC_KAUTO_4MOTIF: return 6;
        default: return (app >= 0 && app < ORC_NUM_APPS) ? 1 : 0;
    }
}

/* number of sequential pattern runs of an app (each re-scatters every v0) */
static int num_runs(int app) {
    if (app == ORC_KGPI_3MOTIF) return 2;
    if (app == ORC_KAUTO_4MOTIF) return 6;
    return 1;
}

/* Start vertices: v0 % v0_mod == v0_rem, and, when labels is given, labels[v0] == label (the
 * restrict_starting_vertex_label run of WorkloadDistributer::fetch_next_batch_local,
 * engine.cc:1457-1496).  raw: keep the aggregators' raw values (no multiplicity division). */
static int count_impl(int app, uint32_t n, const uint64_t *off, const uint32_t *adj, const uint32_t *labels,
                      uint32_t label, uint32_t v0_mod, uint32_t v0_rem, int threads, int raw, uint64_t *counts,
                      uint64_t *num_ext, uint64_t *algo_bytes) {
    if (app < 0 || app >= ORC_NUM_APPS || v0_mod == 0) return -1;
    uint32_t maxd = 0;
    for (uint32_t v = 0; v < n; ++v) { uint32_t d = (uint32_t)(off[v + 1] - off[v]); if (d > maxd) maxd = d; }
    if (threads <= 0) threads = omp_get_max_threads();
    uint64_t tot[6] = {0}, ext = 0, bytes = 0;
    for (int run = 0; run < num_runs(app); ++run) {
#pragma omp parallel num_threads(threads) reduction(+ : ext, bytes)
        {
            orc_tc tc;
            memset(&tc, 0, sizeof(tc));
            tc.off = off;
            tc.adj = adj;
            for (int l = 0; l < 5; ++l) tc.buf[l] = (uint32_t *)malloc(sizeof(uint32_t) * (maxd + 1));
            orc_tc *t = &tc;
#pragma omp for schedule(dynamic, 64)
            for (uint32_t v0 = v0_rem; v0 < n; v0 += v0_mod) {
                if (labels && labels[v0] != label) continue;
                switch (app) {
                    case ORC_KAUTO_TRIANGLE: kauto_triangle(t, v0); break;
                    case ORC_KAUTO_4CLIQUE: kauto_clique(t, v0, 4); break;
                    case ORC_KAUTO_5CLIQUE: kauto_clique(t, v0, 5); break;
                    case ORC_KAUTO_3MOTIF: kauto_3motif(t, v0); break;
                    case ORC_KGPI_TRIANGLE: kgpi_triangle(t, v0, 0); break;
                    case ORC_KGPI_4CLIQUE: kgpi_clique(t, v0, 4); break;
                    case ORC_KGPI_5CLIQUE: kgpi_clique(t, v0, 5); break;
                    case ORC_KGPI_3MOTIF: if (run == 0) kgpi_triangle(t, v0, 0); else kgpi_wedge(t, v0); break;
                    case ORC_KGPI_4CYCLE: kgpi_4cycle(t, v0); break;
                    case ORC_KGPI_HOUSE: kgpi_house(t, v0); break;
                    case ORC_KGPI_TAILED_TRIANGLE: kgpi_tailed(t, v0); break;
                    case ORC_KAUTO_4MOTIF: kauto_4motif(t, v0, run); break;
                }
            }
#pragma omp critical
            for (int c = 0; c < 6; ++c) tot[c] += tc.cnt[c];
            ext += tc.ext;
            bytes += tc.bytes;
            for (int l = 0; l < 5; ++l) free(tc.buf[l]);
        }
    }
    /* multiplicities: kautomine/three_motif.cc:44 ({1, 2}); 4-motif {1, 2, 1, 8, 1, 1} */
    if (raw) {
        /* the aggregators' values as they are */
    } else if (app == ORC_KAUTO_3MOTIF) {
        if (tot[1] % 2) return -2;
        tot[1] /= 2;
    } else if (app == ORC_KAUTO_4MOTIF) {
        if (tot[1] % 2 || tot[3] % 8) return -2;
        tot[1] /= 2;
        tot[3] /= 8;
    }
    for (int c = 0; c < orc_num_counts(app); ++c) counts[c] = tot[c];
    if (num_ext) *num_ext = ext;
    if (algo_bytes) *algo_bytes = bytes;
    return 0;
}

int orc_count(int app, uint32_t n, const uint64_t *off, const uint32_t *adj, uint32_t v0_mod, uint32_t v0_rem,
              int threads, uint64_t *counts, uint64_t *num_ext, uint64_t *algo_bytes) {
    return count_impl(app, n, off, adj, NULL, 0, v0_mod, v0_rem, threads, 0, counts, num_ext, algo_bytes);
}

int orc_count_labeled(int app, uint32_t n, const uint64_t *off, const uint32_t *adj, const uint32_t *labels,
                      uint32_t label, int threads, uint64_t *raw_counts, uint64_t *num_ext, uint64_t *algo_bytes) {
    if (!labels) return -1;
    return count_impl(app, n, off, adj, labels, label, 1, 0, threads, 1, raw_counts, num_ext, algo_bytes);
}

/* ------------------------------------------------------------------------- */
/* brute force                                                                */
/* ------------------------------------------------------------------------- */
static int has_edge(const uint64_t *off, const uint32_t *adj, uint32_t u, uint32_t v) {
    return bsearch_u32(adj + off[u], (uint32_t)(off[u + 1] - off[u]), v);
}

/* pattern edge lists over k vertices, with |Aut| */
typedef struct { int k; int ne; int e[8][2]; int aut; } orc_pat;
static const orc_pat PATS[8] = {
    {3, 3, {{0, 1}, {1, 2}, {0, 2}}, 6},                                   /* triangle */
    {4, 6, {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}}, 24},          /* 4-clique */
    {5, 0, {{0, 0}}, 120},                                                 /* 5-clique: nested loops below */
    {3, 2, {{0, 1}, {0, 2}}, 2},                                           /* wedge */
    {3, 2, {{0, 1}, {0, 2}}, 2},                                           /* wedge (induced) */
    {4, 4, {{0, 1}, {1, 2}, {2, 3}, {3, 0}}, 8},                           /* 4-cycle */
    {5, 6, {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {0, 4}, {1, 4}}, 2},           /* house */
    {4, 4, {{0, 1}, {0, 2}, {1, 2}, {0, 3}}, 2},                           /* tailed triangle */
};
static const int MOTIF4[6][7][2] = {
    {{0, 1}, {0, 2}, {0, 3}, {-1, -1}},                                   /* 3-star */
    {{0, 1}, {1, 2}, {2, 3}, {-1, -1}},                                   /* 4-path */
    {{0, 1}, {0, 2}, {1, 2}, {0, 3}, {-1, -1}},                           /* tailed triangle */
    {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {-1, -1}},                           /* 4-cycle */
    {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {-1, -1}},                   /* diamond */
    {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}, {-1, -1}},           /* 4-clique */
};

static int next_perm(int *a, int k) {
    int i = k - 2;
    while (i >= 0 && a[i] >= a[i + 1]) --i;
    if (i < 0) return 0;
    int j = k - 1;
    while (a[j] <= a[i]) --j;
    int x = a[i]; a[i] = a[j]; a[j] = x;
    for (int l = i + 1, r = k - 1; l < r; ++l, --r) { x = a[l]; a[l] = a[r]; a[r] = x; }
    return 1;
}

/* copies of pattern p inside vertex set S (|S| = p.k): embeddings / |Aut| */
static uint64_t copies_in(const orc_pat *p, const uint32_t *S, const uint8_t adjm[5][5], int induced) {
    int perm[5] = {0, 1, 2, 3, 4};
    uint64_t emb = 0;
    uint8_t pe[5][5];
    memset(pe, 0, sizeof(pe));
    for (int e = 0; e < p->ne; ++e) { pe[p->e[e][0]][p->e[e][1]] = pe[p->e[e][1]][p->e[e][0]] = 1; }
    (void)S;
    do {
        int ok = 1;
        for (int a = 0; a < p->k && ok; ++a)
            for (int b = a + 1; b < p->k && ok; ++b) {
                int g = adjm[perm[a]][perm[b]];
                if (pe[a][b] && !g) ok = 0;
                if (induced && !pe[a][b] && g) ok = 0;
            }
        emb += ok;
    } while (next_perm(perm, p->k));
    return emb / p->aut;
}

uint64_t orc_brute(int pattern, uint32_t n, const uint64_t *off, const uint32_t *adj) {
    orc_pat pat;
    int induced = 0;
    if (pattern >= 10 && pattern <= 15) {
        int q = pattern - 10;
        pat.k = 4; pat.ne = 0;
        while (MOTIF4[q][pat.ne][0] >= 0) { pat.e[pat.ne][0] = MOTIF4[q][pat.ne][0]; pat.e[pat.ne][1] = MOTIF4[q][pat.ne][1]; pat.ne++; }
        static const int aut[6] = {6, 2, 2, 8, 4, 24};
        pat.aut = aut[q];
        induced = 1;
    } else if (pattern >= 0 && pattern <= 7) {
        pat = PATS[pattern];
        induced = pattern == 4;
    } else {
        return UINT64_MAX;
    }
    uint64_t total = 0;
    int k = pat.k;
    if (pattern == 2) {
        /* 5-clique: all 10 pairs */
        uint64_t c = 0;
        for (uint32_t a = 0; a < n; ++a)
            for (uint32_t b = a + 1; b < n; ++b) if (has_edge(off, adj, a, b))
                for (uint32_t cc = b + 1; cc < n; ++cc) if (has_edge(off, adj, a, cc) && has_edge(off, adj, b, cc))
                    for (uint32_t d = cc + 1; d < n; ++d) if (has_edge(off, adj, a, d) && has_edge(off, adj, b, d) && has_edge(off, adj, cc, d))
                        for (uint32_t e = d + 1; e < n; ++e)
                            if (has_edge(off, adj, a, e) && has_edge(off, adj, b, e) && has_edge(off, adj, cc, e) && has_edge(off, adj, d, e)) c++;
        return c;
    }
    uint32_t S[5];
    /* enumerate k-subsets in lexicographic order */
    if (n < (uint32_t)k) return 0;
    for (int i = 0; i < k; ++i) S[i] = (uint32_t)i;
    for (;;) {
        uint8_t adjm[5][5];
        memset(adjm, 0, sizeof(adjm));
        int nedges = 0;
        for (int a = 0; a < k; ++a)
            for (int b = a + 1; b < k; ++b)
                if (has_edge(off, adj, S[a], S[b])) { adjm[a][b] = adjm[b][a] = 1; nedges++; }
        if (nedges >= pat.ne) total += copies_in(&pat, S, (const uint8_t(*)[5])adjm, induced);
        int i = k - 1;
        while (i >= 0 && S[i] == n - (uint32_t)k + (uint32_t)i) --i;
        if (i < 0) break;
        S[i]++;
        for (int j = i + 1; j < k; ++j) S[j] = S[j - 1] + 1;
    }
    return total;
}

/* ------------------------------------------------------------------------- */
/* 3-FSM (kautomine/three_fsm.cc)                                            */
/* ------------------------------------------------------------------------- */

/* Neighbour lists regrouped by label: the label-l neighbours of v are
 * ladj[loff[v * L + l] .. loff[v * L + l + 1]), ascending ids (the CSR order kept). */
typedef struct {
    uint32_t n, L;
    uint64_t *loff;
    uint32_t *ladj;
    const uint32_t *labels;
    uint8_t *dom[4]; /* per pattern position: 1 where some embedding maps a vertex there */
} orc_fsm_graph;

static const uint32_t *fsm_nbrs(const orc_fsm_graph *g, uint32_t v, uint32_t l, uint32_t *len) {
    const uint64_t b = g->loff[(uint64_t)v * g->L + l];
    *len = (uint32_t)(g->loff[(uint64_t)v * g->L + l + 1] - b);
    return g->ladj + b;
}

static void fsm_mark(const orc_fsm_graph *g, int pos, uint32_t v) {
    __atomic_store_n(&g->dom[pos][v], (uint8_t)1, __ATOMIC_RELAXED);
}

/* The images of the pairs (a, b), a in A \ {skip_a}, b in B \ {skip_b}, a != b, at positions
 * pa and pb (the last two vertices of a wedge, four-chain or three-star, which the app's loops
 * pick independently under exactly these exclusions).  a has a partner iff B holds a vertex
 * other than skip_b and a; likewise b.  Returns whether any pair exists. */
static int fsm_pair_images(const orc_fsm_graph *g, const uint32_t *A, uint32_t na, uint32_t skip_a,
                           const uint32_t *B, uint32_t nb, uint32_t skip_b, int pa, int pb) {
    uint32_t ea = 0, eb = 0, a1 = 0, b1 = 0;
    for (uint32_t i = 0; i < na; ++i) if (A[i] != skip_a) { if (ea == 0) a1 = A[i]; ea++; }
    for (uint32_t i = 0; i < nb; ++i) if (B[i] != skip_b) { if (eb == 0) b1 = B[i]; eb++; }
    int any = 0;
    for (uint32_t i = 0; i < na; ++i) {
        const uint32_t a = A[i];
        if (a == skip_a) continue;
        if (eb >= 2 || (eb == 1 && b1 != a)) { fsm_mark(g, pa, a); any = 1; }
    }
    for (uint32_t i = 0; i < nb; ++i) {
        const uint32_t b = B[i];
        if (b == skip_b) continue;
        if (ea >= 2 || (ea == 1 && a1 != b)) fsm_mark(g, pb, b);
    }
    return any;
}

enum { FSM_EDGE = 0, FSM_WEDGE = 1, FSM_TRIANGLE = 2, FSM_FOUR_CHAIN = 3, FSM_THREE_STAR = 4 };

/* The embeddings one candidate's run inserts with enable = true (three_fsm.cc:53-262), started
 * from the vertices whose label is c[0] (run(true, true, labels[0]), three_fsm.cc:606):
 *   edge        v1 in N(v0)                                      (53-68)
 *   wedge       v1, v2 in N(v0), v2 != v1                        (69-107)
 *   triangle    v1 in N(v0), v2 in N(v0) n N(v1)                 (108-151)
 *   four-chain  v1, v2 in N(v0), v2 != v1; v3 in N(v1) \ {v0, v2} (152-200)
 *   three-star  v1 in N(v0); v2 in N(v1) \ {v0}; v3 in N(v1) \ {v0, v2} (201-250)
 * each with its vertices' labels equal to c.  The images per position are marked per (v0) or
 * (v0, v1) prefix without listing the last two vertices' pairs one by one. */
static void fsm_domains(const orc_fsm_graph *g, int t, const uint32_t *c, int threads) {
    const uint32_t n = g->n;
#pragma omp parallel for num_threads(threads) schedule(dynamic, 64)
    for (uint32_t v0 = 0; v0 < n; ++v0) {
        if (g->labels[v0] != c[0]) continue;
        uint32_t n1;
        const uint32_t *N1 = fsm_nbrs(g, v0, c[1], &n1);
        if (t == FSM_EDGE) {
            if (n1) fsm_mark(g, 0, v0);
            for (uint32_t i = 0; i < n1; ++i) fsm_mark(g, 1, N1[i]);
            continue;
        }
        if (t == FSM_WEDGE) {
            uint32_t n2;
            const uint32_t *N2 = fsm_nbrs(g, v0, c[2], &n2);
            if (fsm_pair_images(g, N1, n1, UINT32_MAX, N2, n2, UINT32_MAX, 1, 2)) fsm_mark(g, 0, v0);
            continue;
        }
        for (uint32_t i = 0; i < n1; ++i) {
            const uint32_t v1 = N1[i];
            int any = 0;
            if (t == FSM_TRIANGLE) {
                uint32_t na, nb;
                const uint32_t *A = fsm_nbrs(g, v0, c[2], &na), *B = fsm_nbrs(g, v1, c[2], &nb);
                for (uint32_t x = 0, y = 0; x < na && y < nb;) {
                    if (A[x] < B[y]) ++x;
                    else if (A[x] > B[y]) ++y;
                    else { fsm_mark(g, 2, A[x]); any = 1; ++x; ++y; }
                }
            } else if (t == FSM_FOUR_CHAIN) {
                uint32_t na, nb;
                const uint32_t *A = fsm_nbrs(g, v0, c[2], &na), *B = fsm_nbrs(g, v1, c[3], &nb);
                any = fsm_pair_images(g, A, na, v1, B, nb, v0, 2, 3);
            } else {
                uint32_t na, nb;
                const uint32_t *A = fsm_nbrs(g, v1, c[2], &na), *B = fsm_nbrs(g, v1, c[3], &nb);
                any = fsm_pair_images(g, A, na, v0, B, nb, v0, 2, 3);
            }
            if (any) { fsm_mark(g, 0, v0); fsm_mark(g, 1, v1); }
        }
    }
}

/* Candidate labellings of one level (CandidateLabeledPatternGenerator, three_fsm.cc:315-590), in
 * the generator's loop order.  fv / fe / fw: frequent vertex labels, edges (L^2) and wedges (L^3).
 * cand receives 4 labels per candidate (canonical order); returns the number of candidates. */
static uint32_t fsm_candidates(int t, uint32_t L, const uint8_t *fv, const uint8_t *fe, const uint8_t *fw,
                               uint32_t *cand) {
    uint32_t nc = 0;
#define FE(a, b) fe[(a) * L + (b)]
#define FW(a, b, c) fw[((a) * L + (b)) * L + (c)]
#define PUT(a, b, c, d) do { cand[4 * nc] = (a); cand[4 * nc + 1] = (b); cand[4 * nc + 2] = (c); \
                             cand[4 * nc + 3] = (d); nc++; } while (0)
    for (uint32_t l0 = 0; l0 < L; ++l0) {
        if (!fv[l0]) continue;
        for (uint32_t l1 = 0; l1 < L; ++l1) {
            if (t == FSM_EDGE) { /* 315-343 */
                if (fv[l1] && l0 <= l1) PUT(l0, l1, 0, 0);
                continue;
            }
            if (!FE(l0, l1)) continue;
            for (uint32_t l2 = 0; l2 < L; ++l2) {
                if (t == FSM_WEDGE) { /* 345-389 */
                    if (FE(l0, l2) && l1 <= l2) PUT(l0, l1, l2, 0);
                    continue;
                }
                if (!FW(l0, l1, l2)) continue;
                if (t == FSM_TRIANGLE) { /* 391-452 */
                    if (FW(l1, l0, l2) && FW(l2, l0, l1) && l0 <= l1 && l1 <= l2) PUT(l0, l1, l2, 0);
                    continue;
                }
                for (uint32_t l3 = 0; l3 < L; ++l3) {
                    if (t == FSM_FOUR_CHAIN) { /* 454-512 */
                        if (FW(l1, l0, l3) && FE(l0, l2) && FE(l1, l3) && l0 <= l1) PUT(l0, l1, l2, l3);
                    } else { /* 514-589: the centre's label l0 goes second */
                        if (FW(l0, l2, l3) && FW(l0, l1, l3) && l1 <= l2 && l2 <= l3) PUT(l1, l0, l2, l3);
                    }
                }
            }
        }
    }
#undef FE
#undef FW
#undef PUT
    return nc;
}

int orc_fsm(uint32_t n, const uint64_t *off, const uint32_t *adj, const uint32_t *labels, uint32_t L,
            uint32_t threshold, int threads, uint32_t *num_candidates, uint32_t *num_frequent,
            uint64_t *support_sum) {
    if (L == 0 || L > ORC_FSM_MAX_LABELS) return -1;
    for (uint32_t v = 0; v < n; ++v) if (labels[v] >= L) return -1;
    if (threads <= 0) threads = omp_get_max_threads();
    const uint64_t m = off[n];
    orc_fsm_graph g;
    memset(&g, 0, sizeof(g));
    g.n = n;
    g.L = L;
    g.labels = labels;
    g.loff = (uint64_t *)calloc((size_t)n * L + 1, sizeof(uint64_t));
    g.ladj = (uint32_t *)malloc(sizeof(uint32_t) * (m ? m : 1));
    const size_t L4 = (size_t)L * L * L * L;
    uint8_t *fe = (uint8_t *)calloc((size_t)L * L, 1), *fw = (uint8_t *)calloc((size_t)L * L * L, 1);
    uint32_t *cand = (uint32_t *)malloc(sizeof(uint32_t) * 4 * L4);
    uint8_t fv[ORC_FSM_MAX_LABELS] = {0};
    int rc = g.loff && g.ladj && fe && fw && cand ? 0 : -1;
    for (int p = 0; p < 4 && rc == 0; ++p) if (!(g.dom[p] = (uint8_t *)malloc(n ? n : 1))) rc = -1;
    if (rc == 0) {
        /* regroup every list by label: a counting pass, then a stable scatter */
        for (uint32_t v = 0; v < n; ++v)
            for (uint64_t e = off[v]; e < off[v + 1]; ++e) g.loff[(uint64_t)v * L + labels[adj[e]] + 1]++;
        for (uint64_t i = 0; i < (uint64_t)n * L; ++i) g.loff[i + 1] += g.loff[i];
        uint64_t *fill = (uint64_t *)malloc(sizeof(uint64_t) * ((size_t)n * L + 1));
        if (!fill) rc = -1;
        else {
            memcpy(fill, g.loff, sizeof(uint64_t) * ((size_t)n * L + 1));
            for (uint32_t v = 0; v < n; ++v)
                for (uint64_t e = off[v]; e < off[v + 1]; ++e) g.ladj[fill[(uint64_t)v * L + labels[adj[e]]]++] = adj[e];
            free(fill);
        }
    }
    if (rc == 0) {
        /* level 0, setup (three_fsm.cc:289-310): every label's vertex count enters the sum */
        uint64_t per[ORC_FSM_MAX_LABELS] = {0};
        for (uint32_t v = 0; v < n; ++v) per[labels[v]]++;
        num_candidates[0] = L;
        num_frequent[0] = 0;
        support_sum[0] = 0;
        for (uint32_t l = 0; l < L; ++l) {
            fv[l] = per[l] >= threshold;
            num_frequent[0] += fv[l];
            support_sum[0] += per[l];
        }
        static const int kSize[5] = {2, 3, 3, 4, 4};
        for (int t = FSM_EDGE; t <= FSM_THREE_STAR; ++t) {
            const uint32_t nc = fsm_candidates(t, L, fv, fe, fw, cand);
            const int k = kSize[t];
            /* the next levels read this level's frequent set: edges and wedges only */
            uint8_t *freq = t == FSM_EDGE ? fe : t == FSM_WEDGE ? fw : NULL;
            num_candidates[1 + t] = nc;
            num_frequent[1 + t] = 0;
            support_sum[1 + t] = 0;
            for (uint32_t ci = 0; ci < nc; ++ci) {
                const uint32_t *c = cand + 4 * ci;
                for (int p = 0; p < 4; ++p) memset(g.dom[p], 0, n);
                fsm_domains(&g, t, c, threads);
                /* get_support (engine.h:384-401): the least image count, starting from n */
                uint32_t support = n;
                for (int p = 0; p < k; ++p) {
                    uint32_t s = 0;
                    for (uint32_t v = 0; v < n; ++v) s += g.dom[p][v];
                    if (s < support) support = s;
                }
                if (support < threshold) continue;
                num_frequent[1 + t]++;
                support_sum[1 + t] += support;
                /* the canonical labelling and its automorphisms join the frequent set */
                if (t == FSM_EDGE) {
                    freq[c[0] * L + c[1]] = 1;
                    freq[c[1] * L + c[0]] = 1;
                } else if (t == FSM_WEDGE) {
                    freq[(c[0] * L + c[1]) * L + c[2]] = 1;
                    freq[(c[0] * L + c[2]) * L + c[1]] = 1;
                }
            }
        }
    }
    for (int p = 0; p < 4; ++p) free(g.dom[p]);
    free(g.loff);
    free(g.ladj);
    free(fe);
    free(fw);
    free(cand);
    return rc;
}
