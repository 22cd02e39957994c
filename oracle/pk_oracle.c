/*
 * CPU restatement of pickle's v2 HNSW query and insert path.  TEST
 * INFRASTRUCTURE (see pk_oracle.h): the checker for the device library, never
 * part of the product.
 *
 * Every function below names the reference code it restates.  Paths are
 * relative to the reference project (juelinl/pickle).
 *
 * Floating-point summation order.  The reference computes float distances in
 * 16 SIMD lanes, lane l summing elements i = l (mod 16), and then adds the 16
 * lanes left to right (include/distance/avx512.hpp:187-231, Sum16 in
 * include/marco.hpp:128-131).  It is compiled with
 * -funsafe-math-optimizations, so the compiler may reassociate both steps, and
 * in practice its fixed-Dim and dynamic-extent instantiations of the same
 * kernel return different last bits.  The restatement uses the source order
 * (16 lanes, fused multiply-add, then a left-to-right lane sum) under strict
 * IEEE semantics.  Integer types accumulate exactly in int32
 * (include/distance/avx512.hpp:14-149) and are bit-identical to the reference.
 */
#include "pk_oracle.h"
#include "pk_graphfile.h"

#include <float.h>
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ */
/* distances: include/distance.hpp:10-20, include/distance/avx512.hpp  */
/* ------------------------------------------------------------------ */

static inline float half_to_float(uint16_t h) {
    uint32_t s = (uint32_t)(h & 0x8000) << 16, e = (h >> 10) & 0x1f, m = h & 0x3ff, bits;
    if (e == 0) {
        if (m == 0) {
            bits = s;
        } else { /* subnormal: normalise */
            e = 127 - 15 + 1;
            while (!(m & 0x400)) { m <<= 1; e--; }
            m &= 0x3ff;
            bits = s | (e << 23) | (m << 13);
        }
    } else if (e == 31) {
        bits = s | 0x7f800000u | (m << 13);
    } else {
        bits = s | ((e + 127 - 15) << 23) | (m << 13);
    }
    float f;
    memcpy(&f, &bits, 4);
    return f;
}

static float dist_float(const float *a, const float *b, int64_t dim, int ip) {
    float lane[16] = {0};
    int64_t main_ = dim - dim % 16;
    for (int64_t i = 0; i < main_; i += 16)
        for (int l = 0; l < 16; l++) {
            if (ip) {
                lane[l] = fmaf(a[i + l], b[i + l], lane[l]);
            } else {
                float d = a[i + l] - b[i + l];
                lane[l] = fmaf(d, d, lane[l]);
            }
        }
    float remain = 0.0f;
    for (int64_t j = main_; j < dim; j++) {
        if (ip) {
            remain = fmaf(a[j], b[j], remain);
        } else {
            float d = a[j] - b[j];
            remain = fmaf(d, d, remain);
        }
    }
    float s = lane[0];
    for (int l = 1; l < 16; l++) s = s + lane[l];
    s = s + remain;
    return ip ? -s : s;
}

static float dist_half(const uint16_t *a, const uint16_t *b, int64_t dim, int ip) {
    float lane[16] = {0};
    int64_t main_ = dim - dim % 16;
    for (int64_t i = 0; i < main_; i += 16)
        for (int l = 0; l < 16; l++) {
            float x = half_to_float(a[i + l]), y = half_to_float(b[i + l]);
            if (ip) {
                lane[l] = fmaf(x, y, lane[l]);
            } else {
                float d = x - y;
                lane[l] = fmaf(d, d, lane[l]);
            }
        }
    float remain = 0.0f;
    for (int64_t j = main_; j < dim; j++) {
        float x = half_to_float(a[j]), y = half_to_float(b[j]);
        if (ip) {
            remain = fmaf(x, y, remain);
        } else {
            float d = x - y;
            remain = fmaf(d, d, remain);
        }
    }
    float s = lane[0];
    for (int l = 1; l < 16; l++) s = s + lane[l];
    s = s + remain;
    return ip ? -s : s;
}

static float dist_u8(const uint8_t *a, const uint8_t *b, int64_t dim, int ip) {
    int32_t s = 0;
    for (int64_t i = 0; i < dim; i++) s += ip ? (int32_t)a[i] * (int32_t)b[i] : ((int32_t)a[i] - b[i]) * ((int32_t)a[i] - b[i]);
    return ip ? -(float)s : (float)s;
}

static float dist_i8(const int8_t *a, const int8_t *b, int64_t dim, int ip) {
    int32_t s = 0;
    for (int64_t i = 0; i < dim; i++) s += ip ? (int32_t)a[i] * (int32_t)b[i] : ((int32_t)a[i] - b[i]) * ((int32_t)a[i] - b[i]);
    return ip ? -(float)s : (float)s;
}

/* The summation order of the device library's float distances
 * (pickle_b200/csrc/pk_warp.cuh, Acc / dist_rows / dist_rows_staged; lane
 * layout of lane_config in pk_internal.h): the row, zero padded to C 16-byte
 * chunks, is split over a group of G lanes (G the power of two >= C/4, from 2
 * to 32), lane g accumulating chunks g, g + G, ... in element order with fused
 * multiply-adds; the G partial sums are then combined by a butterfly
 * (partial[g] += partial[g ^ off] for off = G/2, ..., 1) and lane 0's sum is
 * the distance.  Restated here so that the oracle can replay a search with
 * the device's own float distances. */
static float dist_device_order(int dtype, const void *a, const void *b, int64_t dim, int ip) {
    const int64_t esz = dtype == 2 ? 4 : 2, per = 16 / esz;
    const int C = (int)((dim * esz + 15) / 16);
    const int want = (C + 3) / 4;
    int G = 2;
    while (G < want && G < 32) G *= 2;
    const int K = (C + G - 1) / G;
    float part[32], nxt[32];
    for (int g = 0; g < G; g++) {
        float acc = 0.0f;
        for (int k = 0; k < K; k++) {
            const int c = g + k * G;
            if (c >= C) continue;
            for (int64_t e = 0; e < per; e++) {
                const int64_t i = (int64_t)c * per + e;
                float x = 0.0f, y = 0.0f;
                if (i < dim) {
                    if (dtype == 2) {
                        x = ((const float *)a)[i];
                        y = ((const float *)b)[i];
                    } else {
                        x = half_to_float(((const uint16_t *)a)[i]);
                        y = half_to_float(((const uint16_t *)b)[i]);
                    }
                }
                if (ip) {
                    acc = fmaf(x, y, acc);
                } else {
                    const float d = x - y;
                    acc = fmaf(d, d, acc);
                }
            }
        }
        part[g] = acc;
    }
    for (int off = G >> 1; off > 0; off >>= 1) {
        for (int g = 0; g < G; g++) nxt[g] = part[g] + part[g ^ off];
        for (int g = 0; g < G; g++) part[g] = nxt[g];
    }
    return ip ? -part[0] : part[0];
}

static int g_float_order = ORA_ORDER_SOURCE;

void ora_set_float_order(int order) { g_float_order = order == ORA_ORDER_DEVICE ? ORA_ORDER_DEVICE : ORA_ORDER_SOURCE; }

static float distance_in_order(int order, int dtype, int metric, const void *a, const void *b, int64_t dim) {
    int ip = metric == 2;
    switch (dtype) {
        case 0: return dist_u8((const uint8_t *)a, (const uint8_t *)b, dim, ip);
        case 1: return dist_i8((const int8_t *)a, (const int8_t *)b, dim, ip);
        case 2:
            return order == ORA_ORDER_DEVICE ? dist_device_order(2, a, b, dim, ip)
                                             : dist_float((const float *)a, (const float *)b, dim, ip);
        case 3:
            return order == ORA_ORDER_DEVICE ? dist_device_order(3, a, b, dim, ip)
                                             : dist_half((const uint16_t *)a, (const uint16_t *)b, dim, ip);
        default: return NAN;
    }
}

float ora_distance(int dtype, int metric, const void *a, const void *b, int64_t dim) {
    return distance_in_order(g_float_order, dtype, metric, a, b, dim);
}

/* ------------------------------------------------------------------ */
/* binary heaps: include/queue.hpp:99-289                              */
/* ------------------------------------------------------------------ */

typedef struct {
    float d;
    int32_t id;
} ent;

typedef struct {
    ent *a;
    int64_t len, cap;
    int maxfirst; /* 1: MaxFirst (top = largest), 0: MinFirst (top = smallest) */
} heap;

/* Comparators look at the distance only (include/queue.hpp:30-40). */
static inline int hcmp(const heap *h, ent l, ent r) { return h->maxfirst ? (l.d < r.d) : (l.d > r.d); }

static void hinit(heap *h, int maxfirst) {
    h->cap = 512;
    h->len = 0;
    h->maxfirst = maxfirst;
    h->a = (ent *)malloc(sizeof(ent) * h->cap);
}
static void hfree(heap *h) { free(h->a); h->a = NULL; }
static void hclear(heap *h) { h->len = 0; }

/* insert(Entry) (custom sift-up, queue.hpp:191-202) and insert(dist, vid)
 * (std::push_heap, queue.hpp:204-216) move the new entry up while its parent
 * compares strictly before it; both leave the same array. */
static void hpush(heap *h, float d, int32_t id) {
    if (h->len >= h->cap) {
        h->cap *= 8;
        h->a = (ent *)realloc(h->a, sizeof(ent) * h->cap);
    }
    ent e = {d, id};
    int64_t i = h->len++;
    while (i > 0) {
        int64_t p = (i - 1) / 2;
        if (!hcmp(h, h->a[p], e)) break;
        h->a[i] = h->a[p];
        i = p;
    }
    h->a[i] = e;
}

/* pop: last entry to the root, then the custom sift-down of
 * queue.hpp:127-150 (left child wins ties with the right one). */
static void hpop(heap *h) {
    h->a[0] = h->a[h->len - 1];
    h->len--;
    if (h->len == 0) return;
    int64_t i = 0;
    for (;;) {
        int64_t l = 2 * i + 1, r = 2 * i + 2, best = i;
        if (l < h->len && hcmp(h, h->a[best], h->a[l])) best = l;
        if (r < h->len && hcmp(h, h->a[best], h->a[r])) best = r;
        if (best == i) return;
        ent t = h->a[i];
        h->a[i] = h->a[best];
        h->a[best] = t;
        i = best;
    }
}

static inline ent htop(const heap *h) { return h->a[0]; }
static inline ent hextract(heap *h) {
    ent e = h->a[0];
    hpop(h);
    return e;
}

/* ------------------------------------------------------------------ */
/* graph state: include/hnsw_layer.hpp:57-83, include/hnsw.hpp:127-140 */
/* ------------------------------------------------------------------ */

typedef struct {
    int64_t n, lcap, cap, alloc;
    int32_t ent;
    int32_t *ext;
    int16_t *deg, *heu;
    uint8_t *hasvec; /* 0: this layer's copy of the vector is the zero row */
    int32_t *adj;
    float *dist;
    int32_t *ext2in;
} olayer;

struct ora_graph {
    int metric, dtype, growth;
    int64_t dim, M, efc, capacity, esz;
    int enter_level, nlayers;
    olayer *L;
    char *data;       /* capacity rows, by external id */
    uint8_t *levels;  /* capacity */
    char *zero_row;
    int err;
};

/* Spill room after each layer's fixed-stride array, for the reference growth
 * mode: in the reference a list that outgrows its row runs into the next rows
 * and, for the last rows, past the array (undefined behaviour there).  Writes
 * that would land beyond this slack set g->err. */
#define ORA_SLACK_ROWS 64

static int layer_alloc(olayer *L, int64_t lcap, int64_t cap, int64_t capacity) {
    memset(L, 0, sizeof(*L));
    L->lcap = lcap;
    L->cap = cap;
    L->alloc = (lcap + ORA_SLACK_ROWS) * cap;
    L->ext = (int32_t *)malloc(sizeof(int32_t) * (lcap + 1));
    L->deg = (int16_t *)calloc((size_t)lcap + 1, sizeof(int16_t));
    L->heu = (int16_t *)calloc((size_t)lcap + 1, sizeof(int16_t));
    L->hasvec = (uint8_t *)calloc((size_t)lcap + 1, 1);
    L->adj = (int32_t *)malloc(sizeof(int32_t) * L->alloc);
    L->dist = (float *)malloc(sizeof(float) * L->alloc);
    L->ext2in = (int32_t *)malloc(sizeof(int32_t) * (capacity + 1));
    if (!L->ext || !L->deg || !L->heu || !L->hasvec || !L->adj || !L->dist || !L->ext2in) return -1;
    for (int64_t i = 0; i <= lcap; i++) L->ext[i] = -1;
    for (int64_t i = 0; i < L->alloc; i++) {
        L->adj[i] = -1;
        L->dist[i] = FLT_MAX;
    }
    for (int64_t i = 0; i <= capacity; i++) L->ext2in[i] = -1;
    return 0;
}

static void layer_free(olayer *L) {
    free(L->ext);
    free(L->deg);
    free(L->heu);
    free(L->hasvec);
    free(L->adj);
    free(L->dist);
    free(L->ext2in);
}

void ora_free(ora_graph *g) {
    if (!g) return;
    for (int l = 0; l < g->nlayers; l++) layer_free(&g->L[l]);
    free(g->L);
    free(g->data);
    free(g->levels);
    free(g->zero_row);
    free(g);
}

/* GetData(vid, level): a layer's row is the node's external row once AddNode
 * copied it there (include/hnsw_layer.hpp:304-307) and the zero row before
 * that, or forever if AddNode never ran for that level (include/hnsw.hpp:283-297). */
static inline const void *get_data(const ora_graph *g, int level, int32_t vid) {
    int32_t e = g->L[level].ext[vid];
    if (e < 0 || !g->L[level].hasvec[vid]) return g->zero_row;
    return g->data + (size_t)e * g->dim * g->esz;
}

static inline float dist_q(const ora_graph *g, const void *q, const void *row) {
    return ora_distance(g->dtype, g->metric, q, row, g->dim);
}

/* ------------------------------------------------------------------ */
/* visited sets: ByteMap, include/visited.hpp:248-297 (exact)           */
/* ------------------------------------------------------------------ */

typedef struct {
    uint32_t *stamp;
    int64_t size;
    uint32_t cur;
} vset;

static void vs_begin(vset *v, int64_t size) {
    if (v->size < size) {
        free(v->stamp);
        v->stamp = (uint32_t *)calloc((size_t)size, sizeof(uint32_t));
        v->size = size;
        v->cur = 0;
    }
    v->cur++;
    if (v->cur == 0) {
        memset(v->stamp, 0, sizeof(uint32_t) * v->size);
        v->cur = 1;
    }
}
static inline int vs_test(const vset *v, int32_t id) { return v->stamp[id] == v->cur; }
static inline void vs_mark(vset *v, int32_t id) { v->stamp[id] = v->cur; }

typedef struct {
    vset vis;
    heap cand, nn, w, wd;
} scratch;

static void scratch_init(scratch *s) {
    memset(s, 0, sizeof(*s));
    hinit(&s->cand, 0);
    hinit(&s->nn, 1);
    hinit(&s->w, 0);
    hinit(&s->wd, 0);
}
static void scratch_free(scratch *s) {
    free(s->vis.stamp);
    hfree(&s->cand);
    hfree(&s->nn);
    hfree(&s->w);
    hfree(&s->wd);
}

/* An adjacency entry that lies outside the layer would make the reference
 * index its visited table out of range; here it is skipped and flagged. */
static inline int bad_id(const ora_graph *g, const olayer *L, int32_t v) {
    if (v < 0 || v >= L->lcap) {
        ((ora_graph *)g)->err = 1;
        return 1;
    }
    return 0;
}

/* SlideLayer, include/hnsw.hpp:446-494: greedy descent, strict '<'. */
static int32_t slide_layer(const ora_graph *g, scratch *s, int32_t enter, int level, const void *q, int64_t *cnt) {
    const olayer *L = &g->L[level];
    vs_begin(&s->vis, L->lcap);
    int32_t c = enter;
    float cd = dist_q(g, q, get_data(g, level, enter));
    vs_mark(&s->vis, enter);
    int updated;
    do {
        updated = 0;
        int32_t cur = c;
        int64_t deg = L->deg[cur];
        const int32_t *adj = L->adj + (int64_t)cur * L->cap;
        if (cnt) { cnt[0]++; cnt[2] += deg; }
        for (int64_t i = 0; i < deg; i++) {
            int32_t v = adj[i];
            if (bad_id(g, L, v)) continue;
            if (!vs_test(&s->vis, v)) {
                if (cnt) cnt[1]++;
                float d = dist_q(g, q, get_data(g, level, v));
                if (d < cd) {
                    c = v;
                    cd = d;
                    updated = 1;
                }
                vs_mark(&s->vis, v);
            }
        }
    } while (updated);
    return c;
}

/* SearchLayer / SearchLayerFast, include/hnsw.hpp:304-444 (the two share one
 * algorithm; the fast one only adds prefetches).  The result heap is left in
 * s->nn. */
static void search_layer(const ora_graph *g, scratch *s, int32_t enter, int level, int ef, const void *q, int64_t *cnt) {
    const olayer *L = &g->L[level];
    vs_begin(&s->vis, L->lcap);
    hclear(&s->cand);
    hclear(&s->nn);
    float ed = dist_q(g, q, get_data(g, level, enter));
    hpush(&s->nn, ed, enter);
    hpush(&s->cand, ed, enter);
    vs_mark(&s->vis, enter);
    while (s->cand.len > 0) {
        ent c = hextract(&s->cand);
        if (c.d > htop(&s->nn).d) break;
        int64_t deg = L->deg[c.id];
        const int32_t *adj = L->adj + (int64_t)c.id * L->cap;
        if (cnt) { cnt[0]++; cnt[2] += deg; }
        for (int64_t i = 0; i < deg; i++) {
            int32_t v = adj[i];
            if (bad_id(g, L, v)) continue;
            if (!vs_test(&s->vis, v)) {
                if (cnt) cnt[1]++;
                vs_mark(&s->vis, v);
                float d = dist_q(g, q, get_data(g, level, v));
                if (s->nn.len < ef || htop(&s->nn).d > d) {
                    hpush(&s->nn, d, v);
                    hpush(&s->cand, d, v);
                    if (s->nn.len > ef) hpop(&s->nn);
                }
            }
        }
    }
}

/* GetEntInID, include/hnsw_layer.hpp:186-190. */
static inline int32_t ent_in(const ora_graph *g, int32_t ext, int level) {
    return ext < 0 ? g->L[level].ent : g->L[level].ext2in[ext];
}

/* AnnSearch (single), include/hnsw.hpp:509-525, then SelectSimpleExt /
 * extractMinTopK (include/hnsw.hpp:118-125, include/queue.hpp:265-286). */
static void ann_search(const ora_graph *g, scratch *s, const void *q, int k, int ef, int32_t *ids, float *dists,
                       int64_t *cnt) {
    int32_t enter_ext = -1, enter_in = -1;
    for (int level = g->enter_level; level >= 1; level--) {
        enter_in = ent_in(g, enter_ext, level);
        enter_in = slide_layer(g, s, enter_in, level, q, cnt);
        enter_ext = g->L[level].ext[enter_in];
    }
    enter_in = ent_in(g, enter_ext, 0);
    search_layer(g, s, enter_in, 0, ef, q, cnt ? cnt + 3 : NULL);
    heap *nn = &s->nn;
    int64_t kk = k < nn->len ? k : nn->len;
    while (nn->len > kk) hpop(nn);
    for (int64_t i = 0; i < k; i++) {
        ids[i] = -1;
        dists[i] = FLT_MAX;
    }
    for (int64_t i = 0; i < kk; i++) {
        ent e = hextract(nn);
        ids[kk - i - 1] = g->L[0].ext[e.id];
        dists[kk - i - 1] = e.d;
    }
}

int ora_search(const ora_graph *g, const void *queries, int64_t nq, int k, int ef, int nthreads, int32_t *ids,
               float *dists, int64_t *counters) {
    if (!g || k <= 0 || ef <= 0 || nq < 0 || g->nlayers == 0 || g->L[0].n == 0) return -1;
    if (nthreads > 0) omp_set_num_threads(nthreads);
    size_t qb = (size_t)g->dim * g->esz;
#pragma omp parallel
    {
        scratch s;
        scratch_init(&s);
#pragma omp for schedule(dynamic, 20)
        for (int64_t i = 0; i < nq; i++) {
            int64_t *cnt = counters ? counters + 6 * i : NULL;
            if (cnt) memset(cnt, 0, 6 * sizeof(int64_t));
            ann_search(g, &s, (const char *)queries + i * qb, k, ef, ids + i * k, dists + i * k, cnt);
        }
        scratch_free(&s);
    }
    return g->err ? -2 : 0;
}

/* ------------------------------------------------------------------ */
/* fork detector: AnnSearch replayed with two sets of float distances  */
/* ------------------------------------------------------------------ */
/* The same steps as slide_layer / search_layer / ann_search above, on entries
 * that carry a distance in the driving order (a) and in the compared order
 * (b).  Every decision follows a; each comparison of two distances is also
 * made with b, and the first one whose outcome differs is recorded. */

typedef struct {
    float a, b;
    int32_t id;
} dent;

typedef struct {
    dent *v;
    int64_t len, cap;
    int maxfirst;
} dheap;

typedef struct {
    const ora_graph *g;
    int order_a, order_b;
    const int32_t *tkey;
    const float *tval;
    int64_t tn;
    double *fork;
    int32_t *touched;
    int64_t tcap, tcount;
} fctx;

static void fk_note(fctx *c, int where, float xa, float ya, float xb, float yb) {
    if (c->fork[0] != 0.0) return;
    c->fork[0] = 1.0;
    c->fork[1] = where;
    c->fork[2] = xa;
    c->fork[3] = ya;
    c->fork[4] = xb;
    c->fork[5] = yb;
}

/* x < y in order a; a different outcome in order b is the fork. */
static inline int fk_lt(fctx *c, int where, float xa, float ya, float xb, float yb) {
    const int ra = xa < ya, rb = xb < yb;
    if (ra != rb) fk_note(c, where, xa, ya, xb, yb);
    return ra;
}

/* The heaps' comparator (include/queue.hpp:30-40): MaxFirst l < r, MinFirst l > r. */
static inline int dh_cmp(fctx *c, const dheap *h, dent l, dent r) {
    return h->maxfirst ? fk_lt(c, 4, l.a, r.a, l.b, r.b) : fk_lt(c, 4, r.a, l.a, r.b, l.b);
}

static void dh_init(dheap *h, int maxfirst) {
    h->cap = 512;
    h->len = 0;
    h->maxfirst = maxfirst;
    h->v = (dent *)malloc(sizeof(dent) * h->cap);
}

/* hpush / hpop above, step for step. */
static void dh_push(fctx *c, dheap *h, dent e) {
    if (h->len >= h->cap) {
        h->cap *= 8;
        h->v = (dent *)realloc(h->v, sizeof(dent) * h->cap);
    }
    int64_t i = h->len++;
    while (i > 0) {
        int64_t p = (i - 1) / 2;
        if (!dh_cmp(c, h, h->v[p], e)) break;
        h->v[i] = h->v[p];
        i = p;
    }
    h->v[i] = e;
}

static void dh_pop(fctx *c, dheap *h) {
    h->v[0] = h->v[h->len - 1];
    h->len--;
    if (h->len == 0) return;
    int64_t i = 0;
    for (;;) {
        int64_t l = 2 * i + 1, r = 2 * i + 2, best = i;
        if (l < h->len && dh_cmp(c, h, h->v[best], h->v[l])) best = l;
        if (r < h->len && dh_cmp(c, h, h->v[best], h->v[r])) best = r;
        if (best == i) return;
        dent t = h->v[i];
        h->v[i] = h->v[best];
        h->v[best] = t;
        i = best;
    }
}

static dent dh_extract(fctx *c, dheap *h) {
    dent e = h->v[0];
    dh_pop(c, h);
    return e;
}

/* The row a layer's node is compared with: its external id, or -1 for the
 * zero row (see get_data). */
static inline int32_t row_key(const ora_graph *g, int level, int32_t vid) {
    int32_t e = g->L[level].ext[vid];
    return (e < 0 || !g->L[level].hasvec[vid]) ? -1 : e;
}

static dent fk_dist(fctx *c, const void *q, int level, int32_t vid) {
    const ora_graph *g = c->g;
    const void *row = get_data(g, level, vid);
    const int32_t key = row_key(g, level, vid);
    if (c->touched && c->tcount < c->tcap) c->touched[c->tcount] = key;
    c->tcount++;
    dent e;
    e.id = vid;
    e.a = distance_in_order(c->order_a, g->dtype, g->metric, q, row, g->dim);
    if (c->order_b != ORA_ORDER_TABLE) {
        e.b = distance_in_order(c->order_b, g->dtype, g->metric, q, row, g->dim);
        return e;
    }
    int64_t lo = 0, hi = c->tn;
    while (lo < hi) {
        int64_t mid = lo + (hi - lo) / 2;
        if (c->tkey[mid] < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    if (lo < c->tn && c->tkey[lo] == key) {
        e.b = c->tval[lo];
    } else {
        e.b = e.a;
        fk_note(c, 5, e.a, e.a, NAN, NAN);
    }
    return e;
}

static int32_t fk_slide(fctx *c, scratch *s, int32_t enter, int level, const void *q) {
    const ora_graph *g = c->g;
    const olayer *L = &g->L[level];
    vs_begin(&s->vis, L->lcap);
    int32_t best = enter;
    dent cd = fk_dist(c, q, level, enter);
    vs_mark(&s->vis, enter);
    int updated;
    do {
        updated = 0;
        int32_t cur = best;
        int64_t deg = L->deg[cur];
        const int32_t *adj = L->adj + (int64_t)cur * L->cap;
        for (int64_t i = 0; i < deg; i++) {
            int32_t v = adj[i];
            if (bad_id(g, L, v)) continue;
            if (!vs_test(&s->vis, v)) {
                dent d = fk_dist(c, q, level, v);
                if (fk_lt(c, 1, d.a, cd.a, d.b, cd.b)) {
                    best = v;
                    cd = d;
                    updated = 1;
                }
                vs_mark(&s->vis, v);
            }
        }
    } while (updated);
    return best;
}

static void fk_search_layer(fctx *c, scratch *s, dheap *cand, dheap *nn, int32_t enter, int level, int ef,
                            const void *q) {
    const ora_graph *g = c->g;
    const olayer *L = &g->L[level];
    vs_begin(&s->vis, L->lcap);
    cand->len = 0;
    nn->len = 0;
    dent e = fk_dist(c, q, level, enter);
    dh_push(c, nn, e);
    dh_push(c, cand, e);
    vs_mark(&s->vis, enter);
    while (cand->len > 0) {
        dent x = dh_extract(c, cand);
        const dent t = nn->v[0];
        if (fk_lt(c, 2, t.a, x.a, t.b, x.b)) break; /* x.d > top.d */
        int64_t deg = L->deg[x.id];
        const int32_t *adj = L->adj + (int64_t)x.id * L->cap;
        for (int64_t i = 0; i < deg; i++) {
            int32_t v = adj[i];
            if (bad_id(g, L, v)) continue;
            if (!vs_test(&s->vis, v)) {
                vs_mark(&s->vis, v);
                dent d = fk_dist(c, q, level, v);
                int admit = nn->len < ef;
                if (!admit) {
                    const dent w = nn->v[0];
                    admit = fk_lt(c, 3, d.a, w.a, d.b, w.b); /* top.d > d */
                }
                if (admit) {
                    dh_push(c, nn, d);
                    dh_push(c, cand, d);
                    if (nn->len > ef) dh_pop(c, nn);
                }
            }
        }
    }
}

int ora_search_fork(const ora_graph *g, const void *queries, int64_t nq, int k, int ef, int order_a, int order_b,
                    const int64_t *tb_off, const int32_t *tb_key, const float *tb_val, int nthreads, int32_t *ids,
                    float *dists, double *fork, int32_t *touched, int64_t touched_cap, int64_t *touched_n) {
    if (!g || k <= 0 || ef <= 0 || nq < 0 || g->nlayers == 0 || g->L[0].n == 0) return -1;
    if (order_a == ORA_ORDER_TABLE) return -1;
    if (order_b == ORA_ORDER_TABLE && (!tb_off || !tb_key || !tb_val)) return -1;
    if (nthreads > 0) omp_set_num_threads(nthreads);
    size_t qb = (size_t)g->dim * g->esz;
#pragma omp parallel
    {
        scratch s;
        scratch_init(&s);
        dheap cand, nn;
        dh_init(&cand, 0);
        dh_init(&nn, 1);
#pragma omp for schedule(dynamic, 4)
        for (int64_t i = 0; i < nq; i++) {
            const void *q = (const char *)queries + i * qb;
            fctx c;
            memset(&c, 0, sizeof(c));
            c.g = g;
            c.order_a = order_a;
            c.order_b = order_b;
            c.fork = fork + 6 * i;
            memset(c.fork, 0, 6 * sizeof(double));
            if (order_b == ORA_ORDER_TABLE) {
                c.tkey = tb_key + tb_off[i];
                c.tval = tb_val + tb_off[i];
                c.tn = tb_off[i + 1] - tb_off[i];
            }
            if (touched) {
                c.touched = touched + i * touched_cap;
                c.tcap = touched_cap;
            }
            /* ann_search */
            int32_t enter_ext = -1, enter_in = -1;
            for (int level = g->enter_level; level >= 1; level--) {
                enter_in = ent_in(g, enter_ext, level);
                enter_in = fk_slide(&c, &s, enter_in, level, q);
                enter_ext = g->L[level].ext[enter_in];
            }
            enter_in = ent_in(g, enter_ext, 0);
            fk_search_layer(&c, &s, &cand, &nn, enter_in, 0, ef, q);
            int64_t kk = k < nn.len ? k : nn.len;
            while (nn.len > kk) dh_pop(&c, &nn);
            int32_t *oi = ids + i * k;
            float *od = dists + i * k;
            for (int64_t j = 0; j < k; j++) {
                oi[j] = -1;
                od[j] = FLT_MAX;
            }
            for (int64_t j = 0; j < kk; j++) {
                dent e = dh_extract(&c, &nn);
                oi[kk - j - 1] = g->L[0].ext[e.id];
                od[kk - j - 1] = e.a;
            }
            if (touched_n) touched_n[i] = c.tcount;
        }
        free(cand.v);
        free(nn.v);
        scratch_free(&s);
    }
    return g->err ? -2 : 0;
}

/* ------------------------------------------------------------------ */
/* insertion: include/hnsw.hpp:70-116, :247-302; hnsw_layer.hpp:297-465 */
/* ------------------------------------------------------------------ */

typedef struct {
    ent *a;
    int64_t n;
} elist;

/* SelectHeuristic, include/hnsw.hpp:70-116, keep_pruned = true. */
static void select_heuristic(const ora_graph *g, scratch *s, int level, int64_t top_k, elist *R, elist *P) {
    heap *W = &s->w, *Wd = &s->wd;
    hclear(W);
    hclear(Wd);
    for (int64_t i = 0; i < s->nn.len; i++) hpush(W, s->nn.a[i].d, s->nn.a[i].id);
    R->n = 0;
    P->n = 0;
    while (W->len > 0 && R->n < top_k) {
        ent v1 = htop(W);
        const void *v1d = get_data(g, level, v1.id);
        int ins = 1;
        for (int64_t j = 0; j < R->n; j++) {
            float d12 = ora_distance(g->dtype, g->metric, v1d, get_data(g, level, R->a[j].id), g->dim);
            if (v1.d > d12) {
                ins = 0;
                break;
            }
        }
        if (ins)
            R->a[R->n++] = v1;
        else
            hpush(Wd, v1.d, v1.id);
        hpop(W);
    }
    while (Wd->len > 0 && R->n + P->n < top_k) P->a[P->n++] = hextract(Wd);
}

/* std::lower_bound over floats: first index with !(a[i] < x). */
static int64_t lower_bound_f(const float *a, int64_t n, float x) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        int64_t mid = lo + (hi - lo) / 2;
        if (a[mid] < x)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

static inline int slot_ok(ora_graph *g, const olayer *L, int64_t flat) {
    if (flat < 0 || flat >= L->alloc) {
        g->err = 1;
        return 0;
    }
    return 1;
}

/* AddNode, include/hnsw_layer.hpp:297-332. */
static void add_node(ora_graph *g, int level, int32_t vid, const elist *R, const elist *P) {
    olayer *L = &g->L[level];
    int64_t base = (int64_t)vid * L->cap;
    int64_t heur = R->n < L->cap ? R->n : L->cap;
    for (int64_t i = 0; i < heur; i++) {
        L->adj[base + i] = R->a[i].id;
        L->dist[base + i] = R->a[i].d;
    }
    int64_t deg = heur + P->n < L->cap ? heur + P->n : L->cap;
    for (int64_t i = 0; i < deg - heur; i++) {
        L->adj[base + heur + i] = P->a[i].id;
        L->dist[base + heur + i] = P->a[i].d;
    }
    L->deg[vid] = (int16_t)deg;
    L->heu[vid] = (int16_t)heur;
    L->hasvec[vid] = 1;
}

/* AddEdge, include/hnsw_layer.hpp:360-465: reverse edge vid -> nid. */
static void add_edge(ora_graph *g, scratch *s, int level, int32_t vid, int32_t nid, float distance) {
    olayer *L = &g->L[level];
    int64_t cap = L->cap, base = (int64_t)vid * cap;
    int32_t *adj = L->adj + base;
    float *dist = L->dist + base;
    int64_t heur = L->heu[vid], degree = L->deg[vid];
    int64_t offset = lower_bound_f(dist, heur, distance);
    const void *nd = get_data(g, level, nid);
    int ins = 1;
    for (int64_t i = 0; i < offset; i++) {
        float d = ora_distance(g->dtype, g->metric, nd, get_data(g, level, adj[i]), g->dim);
        if (distance > d) {
            ins = 0;
            break;
        }
    }
    if (ins && g->growth == ORA_GROWTH_CAPPED && offset >= cap) ins = 0;
    if (!ins) {
        /* insert into the distance-sorted pruned suffix (:386-408) */
        int32_t *adj_p = adj + heur;
        float *dist_p = dist + heur;
        int64_t pruned = degree - heur;
        int64_t off = lower_bound_f(dist_p, pruned, distance);
        if (off == pruned && degree < cap) {
            adj_p[off] = nid;
            dist_p[off] = distance;
            L->deg[vid] = (int16_t)(degree + 1);
        } else if (off < pruned) {
            int64_t end = degree < cap ? pruned : pruned - 1;
            /* the reference's loop also runs i == off, copying the entry
             * before the suffix into slot off; the write below replaces it */
            for (int64_t i = end; i > off; i--) {
                adj_p[i] = adj_p[i - 1];
                dist_p[i] = dist_p[i - 1];
            }
            adj_p[off] = nid;
            dist_p[off] = distance;
            degree += degree < cap;
            L->deg[vid] = (int16_t)degree;
        }
        return;
    }
    /* re-run the heuristic over the tail (:409-463) */
    heap *W = &s->w, *Wd = &s->wd;
    hclear(W);
    hclear(Wd);
    for (int64_t i = offset; i < degree; i++) hpush(W, dist[i], adj[i]);
    if (!slot_ok(g, L, base + offset)) return;
    adj[offset] = nid;
    dist[offset] = distance;
    int64_t cur_h = offset + 1;
    while (W->len > 0) {
        ent v1 = hextract(W);
        const void *v1d = get_data(g, level, v1.id);
        int keep = 1;
        for (int64_t i = 0; i < cur_h; i++) {
            float d = ora_distance(g->dtype, g->metric, v1d, get_data(g, level, adj[i]), g->dim);
            if (d < v1.d) {
                keep = 0;
                break;
            }
        }
        if (keep && g->growth == ORA_GROWTH_CAPPED && cur_h >= cap) keep = 0;
        if (keep) {
            if (!slot_ok(g, L, base + cur_h)) return;
            adj[cur_h] = v1.id;
            dist[cur_h] = v1.d;
            cur_h++;
        } else {
            hpush(Wd, v1.d, v1.id);
        }
    }
    int64_t cur_deg = cur_h;
    while (cur_deg < cap && Wd->len > 0) {
        ent e = hextract(Wd);
        adj[cur_deg] = e.id;
        dist[cur_deg] = e.d;
        cur_deg++;
    }
    if (cur_h > 32767 || cur_deg > 32767) { g->err = 1; return; }
    L->heu[vid] = (int16_t)cur_h;
    L->deg[vid] = (int16_t)cur_deg;
}

/* NewInID, include/hnsw_layer.hpp:168-177. */
static int32_t new_in_id(ora_graph *g, int level, int32_t ext) {
    olayer *L = &g->L[level];
    if (L->n >= L->lcap) { g->err = 1; return -1; }
    int32_t id = (int32_t)L->n++;
    L->ext[id] = ext;
    L->ext2in[ext] = id;
    return id;
}

static int ora_insert_s(ora_graph *g, scratch *s, int32_t ext_id, const void *data, elist *Rs, elist *Ps) {
    if (ext_id < 0 || ext_id >= g->capacity) return -1;
    const void *q = (const char *)data + (size_t)ext_id * g->dim * g->esz;
    memcpy(g->data + (size_t)ext_id * g->dim * g->esz, q, (size_t)g->dim * g->esz);
    int l = g->levels[ext_id], Ltop = g->enter_level;
    int32_t enter_ext = -1, enter_in = -1;
    for (int level = Ltop; level >= l + 1; level--) {
        if (g->L[level].n > 0) {
            enter_in = ent_in(g, enter_ext, level);
            enter_in = slide_layer(g, s, enter_in, level, q, NULL);
            enter_ext = g->L[level].ext[enter_in];
        }
    }
    int top_search = l < Ltop ? l : Ltop, top_inserted = 0;
    for (int level = 0; level <= l; level++) {
        Rs[level].n = 0;
        Ps[level].n = 0;
    }
    for (int level = top_search; level >= 0; level--) {
        if (g->L[level].n > 0) {
            enter_in = ent_in(g, enter_ext, level);
            int64_t top_k = level == 0 ? 2 * g->M : g->M;
            search_layer(g, s, enter_in, level, (int)g->efc, q, NULL);
            select_heuristic(g, s, level, top_k, &Rs[level], &Ps[level]);
            enter_in = Rs[level].a[0].id;
            enter_ext = g->L[level].ext[enter_in];
            if (level > top_inserted) top_inserted = level;
        }
    }
    for (int level = 0; level <= l; level++) {
        int32_t vid = new_in_id(g, level, ext_id);
        if (vid < 0) return -3;
        if (level <= top_inserted) {
            add_node(g, level, vid, &Rs[level], &Ps[level]);
            for (int64_t i = 0; i < Rs[level].n; i++) add_edge(g, s, level, Rs[level].a[i].id, vid, Rs[level].a[i].d);
            for (int64_t i = 0; i < Ps[level].n; i++) add_edge(g, s, level, Ps[level].a[i].id, vid, Ps[level].a[i].d);
        }
    }
    if (l > g->enter_level) g->enter_level = l;
    return g->err ? -2 : 0;
}

static void alloc_lists(const ora_graph *g, elist **R, elist **P) {
    *R = (elist *)calloc((size_t)g->nlayers + 1, sizeof(elist));
    *P = (elist *)calloc((size_t)g->nlayers + 1, sizeof(elist));
    for (int l = 0; l <= g->nlayers; l++) {
        (*R)[l].a = (ent *)malloc(sizeof(ent) * (2 * g->M + 1));
        (*P)[l].a = (ent *)malloc(sizeof(ent) * (2 * g->M + 1));
    }
}
static void free_lists(const ora_graph *g, elist *R, elist *P) {
    for (int l = 0; l <= g->nlayers; l++) {
        free(R[l].a);
        free(P[l].a);
    }
    free(R);
    free(P);
}

int ora_insert(ora_graph *g, int32_t ext_id, const void *data) {
    scratch s;
    scratch_init(&s);
    elist *R, *P;
    alloc_lists(g, &R, &P);
    int rc = ora_insert_s(g, &s, ext_id, data, R, P);
    free_lists(g, R, P);
    scratch_free(&s);
    return rc;
}

int ora_build(ora_graph *g, const void *data, const int32_t *order, int64_t n) {
    scratch s;
    scratch_init(&s);
    elist *R, *P;
    alloc_lists(g, &R, &P);
    int rc = 0;
    for (int64_t i = 0; i < n && rc == 0; i++) rc = ora_insert_s(g, &s, order[i], data, R, P);
    free_lists(g, R, P);
    scratch_free(&s);
    return rc;
}

/* ------------------------------------------------------------------ */
/* construction, load, save                                            */
/* ------------------------------------------------------------------ */

int ora_cumulative_probability(int64_t M, double *out, int maxn) {
    /* get_cumulative_probability, include/util.hpp:13-25 */
    double r = 1.0 / log((double)M), c = 0.0;
    int n = 0;
    for (;;) {
        double delta = exp(-1.0 * n / r) * (1 - exp(-1.0 / r));
        if (delta < 1e-9) break;
        c += delta;
        if (n < maxn) out[n] = c;
        n++;
    }
    return n;
}

ora_graph *ora_new(int metric, int dtype, int64_t dim, int64_t M, int64_t efc, int64_t capacity,
                   const uint8_t *levels, int growth) {
    if ((metric != 1 && metric != 2) || pkf_elem_size(dtype) == 0 || dim <= 0 || M <= 1 || capacity <= 0) return NULL;
    ora_graph *g = (ora_graph *)calloc(1, sizeof(ora_graph));
    g->metric = metric;
    g->dtype = dtype;
    g->growth = growth;
    g->dim = dim;
    g->M = M;
    g->efc = efc;
    g->capacity = capacity;
    g->esz = pkf_elem_size(dtype);
    g->levels = (uint8_t *)malloc((size_t)capacity);
    memcpy(g->levels, levels, (size_t)capacity);
    int top = 0;
    for (int64_t i = 0; i < capacity; i++)
        if (levels[i] > top) top = levels[i];
    g->nlayers = top + 1;
    g->L = (olayer *)calloc((size_t)g->nlayers, sizeof(olayer));
    /* InitBuffer, include/hnsw.hpp:222-245: layer l holds every node whose
     * level is >= l; layer 0 has 2M slots per node, the others M. */
    for (int l = 0; l < g->nlayers; l++) {
        int64_t cnt = 0;
        for (int64_t i = 0; i < capacity; i++) cnt += levels[i] >= l;
        if (layer_alloc(&g->L[l], cnt, l == 0 ? 2 * M : M, capacity) != 0) {
            ora_free(g);
            return NULL;
        }
    }
    g->data = (char *)calloc((size_t)capacity, (size_t)dim * g->esz);
    g->zero_row = (char *)calloc(1, (size_t)dim * g->esz);
    g->enter_level = 0;
    return g;
}

ora_graph *ora_load(const char *path, int *rc) {
    pkf_graph F;
    int r = pkf_read(path, &F);
    if (rc) *rc = r;
    if (r != 0) return NULL;
    ora_graph *g = (ora_graph *)calloc(1, sizeof(ora_graph));
    g->metric = F.metric;
    g->dtype = F.dtype;
    g->growth = ORA_GROWTH_REFERENCE;
    g->dim = F.dim;
    g->M = F.max_degree;
    g->efc = F.build_ef;
    g->capacity = F.capacity;
    g->esz = pkf_elem_size(F.dtype);
    g->enter_level = F.enter_level;
    g->nlayers = F.num_layers;
    g->L = (olayer *)calloc((size_t)(g->nlayers ? g->nlayers : 1), sizeof(olayer));
    g->levels = (uint8_t *)calloc((size_t)g->capacity + 1, 1);
    g->data = (char *)calloc((size_t)g->capacity + 1, (size_t)g->dim * g->esz);
    g->zero_row = (char *)calloc(1, (size_t)g->dim * g->esz);
    for (int l = 0; l < g->nlayers; l++) {
        olayer *L = &g->L[l];
        pkf_layer *FL = &F.layers[l];
        if (layer_alloc(L, FL->layer_capacity, FL->cap, g->capacity) != 0) {
            pkf_free(&F);
            ora_free(g);
            if (rc) *rc = -6;
            return NULL;
        }
        L->n = FL->n;
        L->ent = FL->ent_id;
        for (int64_t i = 0; i < FL->n; i++) {
            int32_t e = FL->ext[i];
            if (e < 0 || e >= g->capacity) {
                pkf_free(&F);
                ora_free(g);
                if (rc) *rc = -4;
                return NULL;
            }
            L->ext[i] = e;
            L->deg[i] = FL->degree[i];
            L->heu[i] = FL->heuristic[i];
            L->hasvec[i] = FL->has_vector[i];
            L->ext2in[e] = (int32_t)i;
            if (g->levels[e] < l) g->levels[e] = (uint8_t)l;
        }
        memcpy(L->adj, FL->adj, sizeof(int32_t) * FL->layer_capacity * FL->cap);
        memcpy(L->dist, FL->dist, sizeof(float) * FL->layer_capacity * FL->cap);
    }
    if (g->nlayers > 0) {
        size_t rb = (size_t)g->dim * g->esz;
        for (int64_t i = 0; i < F.layers[0].n; i++)
            memcpy(g->data + (size_t)F.layers[0].ext[i] * rb, (const char *)F.vectors + i * rb, rb);
    }
    pkf_free(&F);
    return g;
}

int ora_save(const ora_graph *g, const char *path) {
    pkf_graph F;
    memset(&F, 0, sizeof(F));
    F.metric = g->metric;
    F.dtype = g->dtype;
    F.dim = g->dim;
    F.max_degree = g->M;
    F.build_ef = g->efc;
    F.capacity = g->capacity;
    F.enter_level = g->enter_level;
    F.num_layers = g->nlayers;
    F.layers = (pkf_layer *)calloc((size_t)(g->nlayers ? g->nlayers : 1), sizeof(pkf_layer));
    for (int l = 0; l < g->nlayers; l++) {
        const olayer *L = &g->L[l];
        pkf_layer *FL = &F.layers[l];
        FL->n = L->n;
        FL->layer_capacity = L->lcap;
        FL->cap = L->cap;
        FL->ent_id = L->ent;
        FL->ext = (int32_t *)malloc(4 * L->n + 4);
        FL->degree = (int16_t *)malloc(2 * L->n + 2);
        FL->heuristic = (int16_t *)malloc(2 * L->n + 2);
        FL->has_vector = (uint8_t *)malloc(L->n + 1);
        FL->adj = (int32_t *)malloc(4 * L->lcap * L->cap + 4);
        FL->dist = (float *)malloc(4 * L->lcap * L->cap + 4);
        memcpy(FL->ext, L->ext, 4 * L->n);
        memcpy(FL->degree, L->deg, 2 * L->n);
        memcpy(FL->heuristic, L->heu, 2 * L->n);
        memcpy(FL->has_vector, L->hasvec, L->n);
        memcpy(FL->adj, L->adj, 4 * L->lcap * L->cap);
        memcpy(FL->dist, L->dist, 4 * L->lcap * L->cap);
    }
    int64_t n0 = g->nlayers ? g->L[0].n : 0;
    size_t rb = (size_t)g->dim * g->esz;
    F.vectors = malloc(n0 * rb + 1);
    for (int64_t i = 0; i < n0; i++) memcpy((char *)F.vectors + i * rb, g->data + (size_t)g->L[0].ext[i] * rb, rb);
    int rc = pkf_write(path, &F);
    pkf_free(&F);
    return rc;
}

int ora_info(const ora_graph *g, int64_t *out) {
    out[0] = g->nlayers ? g->L[0].n : 0;
    out[1] = g->nlayers;
    out[2] = g->enter_level;
    out[3] = g->capacity;
    out[4] = g->dim;
    out[5] = g->M;
    out[6] = g->metric;
    out[7] = g->dtype;
    return g->err;
}

int ora_layer(const ora_graph *g, int level, int64_t *n, int64_t *cap, const int32_t **ext, const int16_t **degree,
              const int16_t **heuristic, const int32_t **adj, const float **dist) {
    if (level < 0 || level >= g->nlayers) return -1;
    const olayer *L = &g->L[level];
    *n = L->n;
    *cap = L->cap;
    *ext = L->ext;
    *degree = L->deg;
    *heuristic = L->heu;
    *adj = L->adj;
    *dist = L->dist;
    return 0;
}
