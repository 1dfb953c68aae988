/*
 * pdx_port.c -- CPU restatement of the PDXearch IVF / two-level-IVF search path.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle). Only tests/, the smoke check and bench.py's CPU
 * baseline leg load this library, and only as the checker or the timed CPU port. The product
 * (libpdx_b200.so) never links or calls it.
 *
 * Parity is pinned: tests/test_oracle.py checks this port bit-for-bit (ids and distances)
 * against the reference's own search code compiled from its headers (oracle/_ref, AVX2
 * flavour) on seeded indexes, and against the golden fixtures in tests/golden/.
 *
 * Semantics restated, with the reference lines they follow:
 *   - file format: index.hpp:242-267 (type byte, rotation), ivf_wrapper.hpp:89-131 (IVF),
 *     ivf_wrapper.hpp:218-312 (IVFTree), cluster.hpp:225-255 (compact PDX blocks)
 *   - GetPDXDimensionSplit: common.hpp:133-159
 *   - ADSampling ratios / threshold: adsampling.hpp:91-98, 147-157; searcher.hpp:75-91
 *   - NormalizeQuery: scalar.hpp:23-40; QuantizeEmbedding: scalar.hpp:76-94
 *   - GetClustersAccessOrderIVF: searcher.hpp:181-215
 *   - Start / Warmup / Prune / MergeIntoHeap / BuildResultSetFromHeap: searcher.hpp:217-585
 *   - FilteredStart / Warmup<true> / Prune<true> / FilteredSearch: searcher.hpp:283-372, 726-856
 *   - PDXTreeIndex::Search: index.hpp:545-566
 *   - Distance kernels: scalar_computers.hpp:79-194 (exact U8); the F32 horizontal reduction
 *     order of avx2_computers.hpp:47-98 (8 FMA lanes, pairwise double reduction, double tail).
 *     The F32 vertical update is one fused multiply-add per dimension (the -ffp-contract=fast
 *     form of `dist += d * d`).
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define H_DIM 64
static const uint32_t FETCH_SIZES[20] = {16,  16,  32,  32,   32,   32,   64,   64,   64,    64,
                                         128, 128, 128, 128, 256, 256, 512, 1024, 2048, 16384};

typedef struct {
    uint32_t n, max_cap;
    uint8_t* data; /* compact layout exactly as stored in the file (stride = n) */
    uint32_t* ids;
} pcluster;

typedef struct {
    int is_u8;
    uint32_t d, dv, dh, nclusters;
    pcluster* clusters;
    float* centroids; /* nclusters x d, may be NULL (tree L1 in the file) */
    int is_normalized;
    float base, scale, scale_sq, inv_scale_sq;
    size_t* offsets; /* cumulative max_cap, like IVF::cluster_offsets */
    size_t total_capacity;
    uint32_t max_n;
} plevel;

typedef struct {
    int type;
    uint32_t d;
    float* rotation; /* d x d row-major */
    plevel l1, l0;
    int is_tree;
    float ratios[16385];
    float eps0;
    uint32_t nprobe;
    uint32_t* rowid_cluster; /* row id -> cluster */
    uint32_t* rowid_pos;     /* row id -> position */
    size_t n_rows;
    char err[256];
} pindex;

/* ---------- small helpers ---------- */

static void dim_split(uint32_t d, uint32_t* dh_out, uint32_t* dv_out) {
    float prop = 0.75f;
    if (d <= 128) prop = 0.25f;
    uint32_t h = (uint32_t)((float)d * prop);
    uint32_t v = d - h;
    if (h % H_DIM > 0) {
        h = ((h + H_DIM / 2) / H_DIM) * H_DIM;
        v = d - h;
    }
    if (!v) {
        h = H_DIM;
        v = d - h;
    }
    if (d <= H_DIM) {
        h = 0;
        v = d;
    }
    *dh_out = h;
    *dv_out = v;
}

static float get_ratio(uint32_t visited, uint32_t d, float eps0) {
    if (visited == 0) return 1.0f;
    if (visited == d) return 1.0f;
    double a = 1.0 + (double)eps0 / sqrt((double)visited);
    double r = (double)((float)visited / (float)d);
    return (float)(r * a * a);
}

static float horiz_f32(const float* a, const float* b, size_t n) {
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    size_t i = 0;
    for (; i + 8 <= n; i += 8)
        for (int j = 0; j < 8; j++) {
            float t = a[i + j] - b[i + j];
            acc[j] = fmaf(t, t, acc[j]);
        }
    double s0 = (double)acc[0] + (double)acc[4];
    double s1 = (double)acc[1] + (double)acc[5];
    double s2 = (double)acc[2] + (double)acc[6];
    double s3 = (double)acc[3] + (double)acc[7];
    double d2 = (s0 + s2) + (s1 + s3);
    for (; i < n; i++) {
        float t = a[i] - b[i];
        float sq = t * t;
        d2 += (double)sq;
    }
    return (float)d2;
}

static uint32_t horiz_u8(const uint8_t* a, const uint8_t* b, size_t n) {
    uint32_t s = 0;
    for (size_t i = 0; i < n; i++) {
        int t = (int)a[i] - (int)b[i];
        s += (uint32_t)(t * t);
    }
    return s;
}

/* ---------- heap of (distance, id): max on top, strict-< admission ---------- */
typedef struct {
    float dist;
    uint32_t id;
} cand;
typedef struct {
    cand* a;
    size_t n, cap;
} heap_t;

static void heap_push(heap_t* h, cand c) {
    size_t i = h->n++;
    h->a[i] = c;
    while (i > 0) {
        size_t p = (i - 1) / 2;
        if (h->a[p].dist < h->a[i].dist) {
            cand t = h->a[p];
            h->a[p] = h->a[i];
            h->a[i] = t;
            i = p;
        } else
            break;
    }
}
static void heap_pop(heap_t* h) {
    h->a[0] = h->a[--h->n];
    size_t i = 0;
    for (;;) {
        size_t l = 2 * i + 1, r = l + 1, m = i;
        if (l < h->n && h->a[m].dist < h->a[l].dist) m = l;
        if (r < h->n && h->a[m].dist < h->a[r].dist) m = r;
        if (m == i) break;
        cand t = h->a[m];
        h->a[m] = h->a[i];
        h->a[i] = t;
        i = m;
    }
}

/* ---------- per-search scratch ---------- */
typedef struct {
    const pindex* ix;
    const plevel* lv;
    const void* q; /* float* (F32) or uint8_t* (U8) prepared query */
    uint32_t k;
    heap_t heap;
    uint32_t* dist_u; /* U8 partial distances */
    float* dist_f;    /* F32 partial distances */
    uint32_t* pos;
} sctx;

/* Vertical distance update over dims [d0, d1) for either all vectors (positions == NULL) or
 * the listed positions. For U8, d0 is a multiple of 4 and a tail group is reached only when
 * d1 == dv (scalar_computers.hpp:137-181). */
static void vertical(sctx* s, const pcluster* c, uint32_t d0, uint32_t d1, const uint32_t* positions,
                     size_t npos) {
    const uint32_t n = c->n;
    size_t count = positions ? npos : n;
    if (!s->lv->is_u8) {
        const float* data = (const float*)c->data;
        const float* q = (const float*)s->q;
        for (uint32_t j = d0; j < d1; j++) {
            const float* row = data + (size_t)j * n;
            for (size_t i = 0; i < count; i++) {
                uint32_t v = positions ? positions[i] : (uint32_t)i;
                float t = q[j] - row[v];
                s->dist_f[v] = fmaf(t, t, s->dist_f[v]);
            }
        }
    } else {
        const uint8_t* data = c->data;
        const uint8_t* q = (const uint8_t*)s->q;
        uint32_t j = d0;
        for (; j + 4 <= d1; j += 4) {
            const uint8_t* grp = data + (size_t)j * n;
            for (size_t i = 0; i < count; i++) {
                uint32_t v = positions ? positions[i] : (uint32_t)i;
                const uint8_t* x = grp + (size_t)v * 4;
                int a = (int)q[j] - x[0], b = (int)q[j + 1] - x[1];
                int cc = (int)q[j + 2] - x[2], dd = (int)q[j + 3] - x[3];
                s->dist_u[v] += (uint32_t)(a * a + b * b + cc * cc + dd * dd);
            }
        }
        if (j < d1) {
            uint32_t rem = d1 - j;
            const uint8_t* grp = data + (size_t)j * n;
            for (size_t i = 0; i < count; i++) {
                uint32_t v = positions ? positions[i] : (uint32_t)i;
                for (uint32_t t = 0; t < rem; t++) {
                    int df = (int)q[j + t] - grp[(size_t)v * rem + t];
                    s->dist_u[v] += (uint32_t)(df * df);
                }
            }
        }
    }
}

/* Adds the 64-dim horizontal block b (0-based) of vector v to its partial distance. */
static void horizontal_block(sctx* s, const pcluster* c, uint32_t b, uint32_t v) {
    const plevel* lv = s->lv;
    const size_t n = c->n;
    if (!lv->is_u8) {
        const float* base = (const float*)c->data + (size_t)lv->dv * n + (size_t)b * H_DIM * n;
        s->dist_f[v] += horiz_f32((const float*)s->q + lv->dv + b * H_DIM, base + (size_t)v * H_DIM, H_DIM);
    } else {
        const uint8_t* base = c->data + (size_t)lv->dv * n + (size_t)b * H_DIM * n;
        s->dist_u[v] += horiz_u8((const uint8_t*)s->q + lv->dv + b * H_DIM, base + (size_t)v * H_DIM, H_DIM);
    }
}

/* Threshold in the distance domain of the level (searcher.hpp:75-91). */
static float float_threshold(const sctx* s, uint32_t cur) {
    const float ratio = (cur == s->lv->d) ? 1.0f : s->ix->ratios[cur];
    return s->heap.a[0].dist * ratio;
}
static uint32_t u8_threshold(const sctx* s, uint32_t cur) {
    const float scaled = float_threshold(s, cur) * s->lv->scale_sq;
    return scaled >= (float)UINT32_MAX ? UINT32_MAX : (uint32_t)scaled;
}
static int is_pruned(const sctx* s, uint32_t v, float thr_f, uint32_t thr_u) {
    return s->lv->is_u8 ? (s->dist_u[v] >= thr_u) : (s->dist_f[v] >= thr_f);
}
static float reported(const sctx* s, uint32_t v) {
    if (s->lv->is_u8) return (float)s->dist_u[v] * s->lv->inv_scale_sq;
    return s->dist_f[v];
}
static void reset_dist(sctx* s, uint32_t n) {
    if (s->lv->is_u8)
        memset(s->dist_u, 0, sizeof(uint32_t) * n);
    else
        memset(s->dist_f, 0, sizeof(float) * n);
}
static void mask_dist(sctx* s, uint32_t v) {
    if (s->lv->is_u8)
        s->dist_u[v] = UINT32_MAX / 2;
    else
        s->dist_f[v] = FLT_MAX / 2;
}

static const uint32_t* g_sort_keys_u;
static const float* g_sort_keys_f;

typedef struct {
    double key;
    uint32_t idx;
} kv;
static int kv_cmp(const void* a, const void* b) {
    const kv* x = (const kv*)a;
    const kv* y = (const kv*)b;
    if (x->key < y->key) return -1;
    if (x->key > y->key) return 1;
    return (x->idx < y->idx) ? -1 : (x->idx > y->idx);
}

/* Pushes the m smallest partial distances of the cluster (searcher.hpp:256-280). */
static void push_smallest(sctx* s, const pcluster* c, size_t m) {
    kv* tmp = (kv*)malloc(sizeof(kv) * (c->n ? c->n : 1));
    for (uint32_t v = 0; v < c->n; v++) {
        tmp[v].key = s->lv->is_u8 ? (double)s->dist_u[v] : (double)s->dist_f[v];
        tmp[v].idx = v;
    }
    qsort(tmp, c->n, sizeof(kv), kv_cmp);
    for (size_t i = 0; i < m; i++) {
        cand cd;
        cd.id = c->ids[tmp[i].idx];
        cd.dist = reported(s, tmp[i].idx);
        heap_push(&s->heap, cd);
    }
    free(tmp);
}

/* searcher.hpp:217-281 */
static void start(sctx* s, const pcluster* c) {
    reset_dist(s, c->n);
    vertical(s, c, 0, s->lv->dv, NULL, 0);
    for (uint32_t b = 0; b * H_DIM < s->lv->dh; b++)
        for (uint32_t v = 0; v < c->n; v++) horizontal_block(s, c, b, v);
    size_t m = (size_t)s->k - s->heap.n;
    if (m > c->n) m = c->n;
    push_smallest(s, c, m);
}

/* searcher.hpp:283-372 */
static void filtered_start(sctx* s, const pcluster* c, const uint8_t* sel, uint32_t passing) {
    reset_dist(s, c->n);
    size_t nsurv = 0;
    for (uint32_t v = 0; v < c->n; v++) {
        s->pos[nsurv] = v;
        nsurv += sel[v] == 1;
    }
    const float selection = (float)passing / (float)c->n;
    for (uint32_t b = 0; b * H_DIM < s->lv->dh; b++)
        for (size_t i = 0; i < nsurv; i++) horizontal_block(s, c, b, s->pos[i]);
    if (selection > (1.0f - 0.80f))
        vertical(s, c, 0, s->lv->dv, NULL, 0);
    else
        vertical(s, c, 0, s->lv->dv, s->pos, nsurv);
    size_t m = (size_t)s->k - s->heap.n;
    if (m > passing) m = passing;
    for (uint32_t v = 0; v < c->n; v++)
        if (sel[v] == 0) mask_dist(s, v);
    push_smallest(s, c, m);
}

/* Warmup (searcher.hpp:374-435) then Prune (437-540) then MergeIntoHeap (542-566). */
static void warmup_prune_merge(sctx* s, const pcluster* c, const uint8_t* sel, uint32_t passing) {
    const plevel* lv = s->lv;
    const uint32_t n = c->n;
    uint32_t cur = 0;
    size_t step = 0;
    const size_t needed = (size_t)ceilf(0.80f * (float)n);
    reset_dist(s, n);
    int skip_warmup = 0;
    if (sel) {
        for (uint32_t v = 0; v < n; v++)
            if (sel[v] == 0) mask_dist(s, v);
        const float selection = (float)passing / (float)n;
        if (selection < (1.0f - 0.80f)) skip_warmup = 1;
    }
    if (!skip_warmup) {
        size_t n_pruned = 0;
        while (n_pruned < needed && cur < lv->dv) {
            uint32_t last = cur + FETCH_SIZES[step];
            if (last > lv->dv) last = lv->dv;
            vertical(s, c, cur, last, NULL, 0);
            cur = last;
            step++;
            const float tf = float_threshold(s, cur);
            const uint32_t tu = lv->is_u8 ? u8_threshold(s, cur) : 0;
            n_pruned = 0;
            for (uint32_t v = 0; v < n; v++) n_pruned += is_pruned(s, v, tf, tu);
        }
    }
    /* Prune */
    float tf = float_threshold(s, cur);
    uint32_t tu = lv->is_u8 ? u8_threshold(s, cur) : 0;
    size_t nsurv = 0;
    for (uint32_t v = 0; v < n; v++) {
        s->pos[nsurv] = v;
        nsurv += !is_pruned(s, v, tf, tu) && (!sel || sel[v] == 1);
    }
    uint32_t cur_v = cur, cur_h = 0;
    while (lv->dh && nsurv && cur_h < lv->dh) {
        const size_t cnt = nsurv;
        for (size_t i = 0; i < cnt; i++) horizontal_block(s, c, cur_h / H_DIM, s->pos[i]);
        cur_h += H_DIM;
        cur += H_DIM;
        tf = float_threshold(s, cur);
        tu = lv->is_u8 ? u8_threshold(s, cur) : 0;
        nsurv = 0;
        for (size_t i = 0; i < cnt; i++) {
            s->pos[nsurv] = s->pos[i];
            nsurv += !is_pruned(s, s->pos[i], tf, tu);
        }
    }
    while (nsurv && cur_v < lv->dv) {
        const size_t cnt = nsurv;
        uint32_t last = cur_v + H_DIM;
        if (last > lv->dv) last = lv->dv;
        vertical(s, c, cur_v, last, s->pos, cnt);
        cur = cur + H_DIM < lv->d ? cur + H_DIM : lv->d;
        cur_v = last;
        tf = float_threshold(s, cur);
        tu = lv->is_u8 ? u8_threshold(s, cur) : 0;
        nsurv = 0;
        for (size_t i = 0; i < cnt; i++) {
            s->pos[nsurv] = s->pos[i];
            nsurv += !is_pruned(s, s->pos[i], tf, tu);
        }
        if (cur == lv->d) break;
    }
    /* MergeIntoHeap */
    for (size_t i = 0; i < nsurv; i++) {
        const uint32_t v = s->pos[i];
        const float dd = reported(s, v);
        if (s->heap.n < s->k || dd < s->heap.a[0].dist) {
            cand cd;
            cd.dist = dd;
            cd.id = c->ids[v];
            if (s->heap.n >= s->k) heap_pop(&s->heap);
            heap_push(&s->heap, cd);
        }
    }
}

static int emit(heap_t* h, uint32_t k, uint32_t* ids, float* dists) {
    if (h->n && h->a[0].dist == FLT_MAX) heap_pop(h);
    size_t m = h->n < k ? h->n : k;
    for (size_t i = m; i > 0; i--) {
        ids[i - 1] = h->a[0].id;
        dists[i - 1] = h->a[0].dist;
        heap_pop(h);
    }
    return (int)m;
}

/* searcher.hpp:181-215: centroid distances then (partial) sort; ties by cluster id. */
static void access_order(const plevel* lv, const float* q, uint32_t* order) {
    kv* tmp = (kv*)malloc(sizeof(kv) * lv->nclusters);
    for (uint32_t c = 0; c < lv->nclusters; c++) {
        tmp[c].key = horiz_f32(q, lv->centroids + (size_t)c * lv->d, lv->d);
        tmp[c].idx = c;
    }
    qsort(tmp, lv->nclusters, sizeof(kv), kv_cmp);
    for (uint32_t c = 0; c < lv->nclusters; c++) order[c] = tmp[c].idx;
    free(tmp);
}

static void quantize(const plevel* lv, const float* x, uint8_t* out) {
    for (uint32_t i = 0; i < lv->d; i++) {
        const float v = (x[i] - lv->base) * lv->scale;
        const int r = (int)roundf(v);
        out[i] = r > 255 ? 255 : (r < 0 ? 0 : (uint8_t)r);
    }
}

/* y = M^T x with M row-major d x d (adsampling.hpp:225-245 calls column-major sgemm on it). */
static void rotate(const pindex* ix, const float* x, float* y) {
    const uint32_t d = ix->d;
    for (uint32_t j = 0; j < d; j++) y[j] = 0.0f;
    for (uint32_t i = 0; i < d; i++) {
        const float xi = x[i];
        const float* row = ix->rotation + (size_t)i * d;
        for (uint32_t j = 0; j < d; j++) y[j] = fmaf(row[j], xi, y[j]);
    }
}

/* scalar.hpp:23-40 */
static void normalize(const float* src, float* out, uint32_t d) {
    float sum = 0.0f;
    for (uint32_t i = 0; i < d; i++) sum = fmaf(src[i], src[i], sum);
    if (sum == 0.0f) {
        memcpy(out, src, sizeof(float) * d);
        return;
    }
    const float norm = sqrtf(sum);
    for (uint32_t i = 0; i < d; i++) out[i] = src[i] / norm;
}

static void prepare_query(const pindex* ix, const plevel* lv, const float* raw, int transformed, float* out) {
    if (transformed) {
        memcpy(out, raw, sizeof(float) * ix->d);
        return;
    }
    if (!lv->is_normalized) {
        rotate(ix, raw, out);
    } else {
        float* tmp = (float*)malloc(sizeof(float) * ix->d);
        normalize(raw, tmp, ix->d);
        rotate(ix, tmp, out);
        free(tmp);
    }
}

/* One PDXearch::Search / FilteredSearch over a level. order == NULL: centroid order. */
static int level_search(const pindex* ix, const plevel* lv, const float* qf, uint32_t k, uint32_t nprobe,
                        const uint32_t* order_in, size_t n_order, const uint8_t* selvec,
                        const uint32_t* passing, uint32_t* ids, float* dists) {
    size_t to_visit = (nprobe == 0 || nprobe > lv->nclusters) ? lv->nclusters : nprobe;
    uint32_t* order = (uint32_t*)malloc(sizeof(uint32_t) * (lv->nclusters ? lv->nclusters : 1));
    if (order_in) {
        if (n_order < to_visit) to_visit = n_order;
        memcpy(order, order_in, sizeof(uint32_t) * to_visit);
    } else {
        access_order(lv, qf, order);
    }
    sctx s;
    memset(&s, 0, sizeof(s));
    s.ix = ix;
    s.lv = lv;
    s.k = k;
    uint8_t* qu = NULL;
    if (lv->is_u8) {
        qu = (uint8_t*)malloc(lv->d);
        quantize(lv, qf, qu);
        s.q = qu;
    } else {
        s.q = qf;
    }
    s.heap.a = (cand*)malloc(sizeof(cand) * (k + 1));
    s.heap.cap = k + 1;
    size_t mx = lv->max_n ? lv->max_n : 1;
    s.dist_u = (uint32_t*)malloc(sizeof(uint32_t) * mx);
    s.dist_f = (float*)malloc(sizeof(float) * mx);
    s.pos = (uint32_t*)malloc(sizeof(uint32_t) * mx);
    for (size_t ci = 0; ci < to_visit; ci++) {
        const uint32_t cidx = order[ci];
        const pcluster* c = &lv->clusters[cidx];
        const uint8_t* sel = NULL;
        uint32_t pass = 0;
        if (selvec) {
            sel = selvec + lv->offsets[cidx];
            pass = passing[cidx];
            if (pass == 0) continue;
        }
        if (c->n == 0) continue;
        if (s.heap.n < k) {
            if (sel)
                filtered_start(&s, c, sel, pass);
            else
                start(&s, c);
            continue;
        }
        warmup_prune_merge(&s, c, sel, pass);
    }
    int m = emit(&s.heap, k, ids, dists);
    free(s.heap.a);
    free(s.dist_u);
    free(s.dist_f);
    free(s.pos);
    free(qu);
    free(order);
    return m;
}

/* ---------- loading ---------- */

static int read_level(const uint8_t** pp, const uint8_t* end, plevel* lv, uint32_t d, uint32_t dv, uint32_t dh,
                      uint32_t ncl, int is_u8) {
    const uint8_t* p = *pp;
    lv->is_u8 = is_u8;
    lv->d = d;
    lv->dv = dv;
    lv->dh = dh;
    lv->nclusters = ncl;
    lv->clusters = (pcluster*)calloc(ncl ? ncl : 1, sizeof(pcluster));
    lv->offsets = (size_t*)calloc(ncl ? ncl : 1, sizeof(size_t));
    if ((size_t)(end - p) < (size_t)ncl * 8) return -1;
    const size_t esz = is_u8 ? 1 : 4;
    for (uint32_t i = 0; i < ncl; i++) {
        memcpy(&lv->clusters[i].n, p + (size_t)i * 8, 4);
        memcpy(&lv->clusters[i].max_cap, p + (size_t)i * 8 + 4, 4);
    }
    p += (size_t)ncl * 8;
    lv->total_capacity = 0;
    lv->max_n = 0;
    for (uint32_t i = 0; i < ncl; i++) {
        pcluster* c = &lv->clusters[i];
        lv->offsets[i] = lv->total_capacity;
        lv->total_capacity += c->max_cap;
        if (c->n > lv->max_n) lv->max_n = c->n;
        const size_t bytes = (size_t)c->n * d * esz;
        if ((size_t)(end - p) < bytes) return -1;
        c->data = (uint8_t*)malloc(bytes ? bytes : 1);
        memcpy(c->data, p, bytes);
        p += bytes;
    }
    for (uint32_t i = 0; i < ncl; i++) {
        pcluster* c = &lv->clusters[i];
        const size_t bytes = (size_t)c->n * 4;
        if ((size_t)(end - p) < bytes) return -1;
        c->ids = (uint32_t*)malloc(bytes ? bytes : 4);
        memcpy(c->ids, p, bytes);
        p += bytes;
    }
    *pp = p;
    return 0;
}

static void free_level(plevel* lv) {
    if (!lv->clusters) return;
    for (uint32_t i = 0; i < lv->nclusters; i++) {
        free(lv->clusters[i].data);
        free(lv->clusters[i].ids);
    }
    free(lv->clusters);
    free(lv->offsets);
    free(lv->centroids);
    memset(lv, 0, sizeof(*lv));
}

static void set_ratios(pindex* ix, float eps0) {
    ix->eps0 = eps0;
    for (uint32_t i = 0; i < ix->d && i < 16385; i++) ix->ratios[i] = get_ratio(i, ix->d, eps0);
}

static void build_rowid_map(pindex* ix) {
    const plevel* lv = &ix->l1;
    size_t total = 0;
    for (uint32_t c = 0; c < lv->nclusters; c++) total += lv->clusters[c].n;
    ix->n_rows = total;
    ix->rowid_cluster = (uint32_t*)malloc(sizeof(uint32_t) * (total ? total : 1));
    ix->rowid_pos = (uint32_t*)malloc(sizeof(uint32_t) * (total ? total : 1));
    for (size_t i = 0; i < total; i++) ix->rowid_cluster[i] = UINT32_MAX;
    for (uint32_t c = 0; c < lv->nclusters; c++)
        for (uint32_t p = 0; p < lv->clusters[c].n; p++) {
            uint32_t r = lv->clusters[c].ids[p];
            if (r < total) {
                ix->rowid_cluster[r] = c;
                ix->rowid_pos[r] = p;
            }
        }
}

/* Rebuilds L1 centroids from the L0 vectors (the tree file stores them only there). */
static void tree_l1_centroids(pindex* ix) {
    plevel* l1 = &ix->l1;
    const plevel* l0 = &ix->l0;
    const uint32_t d = ix->d;
    l1->centroids = (float*)calloc((size_t)l1->nclusters * d + 1, sizeof(float));
    for (uint32_t c = 0; c < l0->nclusters; c++) {
        const pcluster* cl = &l0->clusters[c];
        const float* data = (const float*)cl->data;
        const size_t n = cl->n;
        for (uint32_t p = 0; p < cl->n; p++) {
            if (cl->ids[p] >= l1->nclusters) continue;
            float* dst = l1->centroids + (size_t)cl->ids[p] * d;
            for (uint32_t j = 0; j < l0->dv; j++) dst[j] = data[(size_t)j * n + p];
            for (uint32_t b = 0; b < l0->dh; b += H_DIM)
                for (uint32_t j = 0; j < H_DIM; j++)
                    dst[l0->dv + b + j] = data[(size_t)l0->dv * n + (size_t)b * n + (size_t)p * H_DIM + j];
        }
    }
}

void pdxport_free(pindex* ix);

pindex* pdxport_load_buffer(const uint8_t* buf, size_t size) {
    pindex* ix = (pindex*)calloc(1, sizeof(pindex));
    const uint8_t* p = buf;
    const uint8_t* end = buf + size;
    if (size < 9) goto bad;
    ix->type = p[0];
    if (ix->type > 3) goto bad;
    p += 1;
    uint32_t rows, cols;
    memcpy(&rows, p, 4);
    memcpy(&cols, p + 4, 4);
    p += 8;
    if ((size_t)(end - p) < (size_t)rows * cols * 4) goto bad;
    ix->rotation = (float*)malloc(sizeof(float) * (size_t)rows * cols + 4);
    memcpy(ix->rotation, p, sizeof(float) * (size_t)rows * cols);
    p += sizeof(float) * (size_t)rows * cols;
    if (end - p < 16) goto bad;
    uint32_t hdr[5];
    memcpy(hdr, p, 16);
    const int is_u8 = (ix->type == 1 || ix->type == 3);
    ix->is_tree = ix->type >= 2;
    const uint32_t d = hdr[0], dv = hdr[1], dh = hdr[2];
    if (d == 0 || d > 16384 || dv + dh != d || cols != d || (rows != d && rows != 1)) goto bad;
    ix->d = d;
    if (rows == 1) {
        /* adsampling.hpp:192-246, FFTW branch: flip the sign of dimension j where the stored
         * vector is negative, then the orthonormal DCT-II (FFTW_REDFT10 scaled by sqrt(1/(4d))
         * for output 0 and sqrt(1/(2d)) for the others). As the d x d matrix of y = x M:
         * M[j][k] = s_j c_k cos(pi (2j + 1) k / (2d)), c_0 = sqrt(1/d), c_k = sqrt(2/d). */
        float* dense = (float*)malloc(sizeof(float) * (size_t)d * d);
        for (uint32_t j = 0; j < d; ++j) {
            const double sj = ix->rotation[j] < 0.0f ? -1.0 : 1.0;
            for (uint32_t k = 0; k < d; ++k) {
                const double ck = k == 0 ? sqrt(1.0 / d) : sqrt(2.0 / d);
                dense[(size_t)j * d + k] = (float)(sj * ck * cos(3.14159265358979323846 * (2.0 * j + 1.0) * k / (2.0 * d)));
            }
        }
        free(ix->rotation);
        ix->rotation = dense;
    }
    if (!ix->is_tree) {
        const uint32_t ncl = hdr[3];
        p += 16;
        if (read_level(&p, end, &ix->l1, d, dv, dh, ncl, is_u8)) goto bad;
        if (end - p < 1) goto bad;
        ix->l1.is_normalized = p[0];
        p += 1;
        if ((size_t)(end - p) < (size_t)ncl * d * 4) goto bad;
        ix->l1.centroids = (float*)malloc(sizeof(float) * (size_t)ncl * d + 4);
        memcpy(ix->l1.centroids, p, sizeof(float) * (size_t)ncl * d);
        p += sizeof(float) * (size_t)ncl * d;
    } else {
        if (end - p < 20) goto bad;
        memcpy(hdr, p, 20);
        p += 20;
        const uint32_t n1 = hdr[3], n0 = hdr[4];
        if (read_level(&p, end, &ix->l0, d, dv, dh, n0, 0)) goto bad;
        if (read_level(&p, end, &ix->l1, d, dv, dh, n1, is_u8)) goto bad;
        if (end - p < 1) goto bad;
        ix->l1.is_normalized = ix->l0.is_normalized = p[0];
        p += 1;
        if ((size_t)(end - p) < (size_t)n0 * d * 4) goto bad;
        ix->l0.centroids = (float*)malloc(sizeof(float) * (size_t)n0 * d + 4);
        memcpy(ix->l0.centroids, p, sizeof(float) * (size_t)n0 * d);
        p += sizeof(float) * (size_t)n0 * d;
        tree_l1_centroids(ix);
    }
    ix->l1.base = 0.0f;
    ix->l1.scale = 1.0f;
    if (is_u8) {
        if (end - p < 8) goto bad;
        memcpy(&ix->l1.base, p, 4);
        memcpy(&ix->l1.scale, p + 4, 4);
        p += 8;
    }
    ix->l1.scale_sq = ix->l1.scale * ix->l1.scale;
    ix->l1.inv_scale_sq = 1.0f / ix->l1.scale_sq;
    ix->l0.scale = 1.0f;
    ix->l0.scale_sq = 1.0f;
    ix->l0.inv_scale_sq = 1.0f;
    set_ratios(ix, 1.5f);
    build_rowid_map(ix);
    return ix;
bad:
    pdxport_free(ix);
    return NULL;
}

pindex* pdxport_load(const char* path) {
    FILE* f = fopen(path, "rb");
    if (!f) return NULL;
    fseek(f, 0, SEEK_END);
    long sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    uint8_t* buf = (uint8_t*)malloc(sz > 0 ? (size_t)sz : 1);
    size_t got = fread(buf, 1, (size_t)sz, f);
    fclose(f);
    pindex* ix = (got == (size_t)sz) ? pdxport_load_buffer(buf, (size_t)sz) : NULL;
    free(buf);
    return ix;
}

void pdxport_free(pindex* ix) {
    if (!ix) return;
    free_level(&ix->l1);
    free_level(&ix->l0);
    free(ix->rotation);
    free(ix->rowid_cluster);
    free(ix->rowid_pos);
    free(ix);
}

int pdxport_type(const pindex* ix) { return ix->type; }
uint32_t pdxport_num_dimensions(const pindex* ix) { return ix->d; }
uint32_t pdxport_num_clusters(const pindex* ix) { return ix->l1.nclusters; }
void pdxport_set_nprobe(pindex* ix, uint32_t nprobe) { ix->nprobe = nprobe; }
void pdxport_set_pruning_aggressiveness(pindex* ix, float eps0) { set_ratios(ix, eps0); }
float pdxport_ratio(const pindex* ix, uint32_t i) { return ix->ratios[i]; }
void pdxport_dim_split(uint32_t d, uint32_t* dh, uint32_t* dv) { dim_split(d, dh, dv); }

/* Rotated (and, for normalized indexes, normalized) query, as PDXearch::Search prepares it. */
void pdxport_prepare_query(const pindex* ix, const float* raw, float* out) {
    prepare_query(ix, &ix->l1, raw, 0, out);
}
void pdxport_quantize(const pindex* ix, const float* x, uint8_t* out) { quantize(&ix->l1, x, out); }

/* Tree top level (index.hpp:545-566): returns the L1 cluster order and the L1 nprobe. */
static int tree_order(const pindex* ix, const float* qf, uint32_t* order, uint32_t* l1_nprobe) {
    uint32_t np = ix->nprobe == 0 ? ix->l1.nclusters : ix->nprobe;
    uint32_t top = ix->l0.nclusters;
    if (np < ix->l1.nclusters / 2) top /= 2;
    float* dtmp = (float*)malloc(sizeof(float) * (np ? np : 1));
    int m = level_search(ix, &ix->l0, qf, np, top, NULL, 0, NULL, NULL, order, dtmp);
    free(dtmp);
    *l1_nprobe = np;
    return m;
}

int pdxport_search(const pindex* ix, const float* raw, uint32_t k, int transformed, uint32_t* ids, float* dists) {
    float* qf = (float*)malloc(sizeof(float) * ix->d);
    prepare_query(ix, &ix->l1, raw, transformed, qf);
    int m;
    if (!ix->is_tree) {
        m = level_search(ix, &ix->l1, qf, k, ix->nprobe, NULL, 0, NULL, NULL, ids, dists);
    } else {
        uint32_t np;
        uint32_t* order = (uint32_t*)malloc(sizeof(uint32_t) * (ix->l1.nclusters + 1));
        int no = tree_order(ix, qf, order, &np);
        m = level_search(ix, &ix->l1, qf, k, np, order, (size_t)(no < 0 ? 0 : no), NULL, NULL, ids, dists);
        free(order);
    }
    free(qf);
    return m;
}

/* Tree top-level order only (for parity checks of the probing stage). */
int pdxport_tree_order(const pindex* ix, const float* raw, int transformed, uint32_t* order) {
    float* qf = (float*)malloc(sizeof(float) * ix->d);
    prepare_query(ix, &ix->l1, raw, transformed, qf);
    uint32_t np;
    int m = tree_order(ix, qf, order, &np);
    free(qf);
    return m;
}

/* Access order over the L1 centroids (GetClustersAccessOrderIVF), full permutation. */
void pdxport_access_order(const pindex* ix, const float* raw, int transformed, uint32_t* order) {
    float* qf = (float*)malloc(sizeof(float) * ix->d);
    prepare_query(ix, &ix->l1, raw, transformed, qf);
    access_order(&ix->l1, qf, order);
    free(qf);
}

int pdxport_search_with_order(const pindex* ix, const float* raw, uint32_t k, const uint32_t* order,
                              uint32_t n_order, int transformed, uint32_t* ids, float* dists) {
    float* qf = (float*)malloc(sizeof(float) * ix->d);
    prepare_query(ix, &ix->l1, raw, transformed, qf);
    uint32_t np = ix->nprobe;
    if (ix->is_tree && np == 0) np = ix->l1.nclusters;
    int m = level_search(ix, &ix->l1, qf, k, np, order, n_order, NULL, NULL, ids, dists);
    free(qf);
    return m;
}

/* FilteredSearch (searcher.hpp:726-856; index.hpp:421-446). Unknown row ids are ignored. */
int pdxport_filtered_search(const pindex* ix, const float* raw, uint32_t k, const uint64_t* row_ids, uint64_t n,
                            int transformed, uint32_t* ids, float* dists) {
    const plevel* lv = &ix->l1;
    uint8_t* sel = (uint8_t*)calloc(lv->total_capacity + 1, 1);
    uint32_t* passing = (uint32_t*)calloc(lv->nclusters + 1, sizeof(uint32_t));
    for (uint64_t i = 0; i < n; i++) {
        if (row_ids[i] >= ix->n_rows) continue;
        const uint32_t c = ix->rowid_cluster[row_ids[i]];
        if (c == UINT32_MAX) continue;
        passing[c]++;
        sel[lv->offsets[c] + ix->rowid_pos[row_ids[i]]] = 1;
    }
    float* qf = (float*)malloc(sizeof(float) * ix->d);
    prepare_query(ix, lv, raw, transformed, qf);
    int m = level_search(ix, lv, qf, k, ix->nprobe, NULL, 0, sel, passing, ids, dists);
    free(qf);
    free(sel);
    free(passing);
    return m;
}

int pdxport_search_batch(const pindex* ix, const float* q, uint32_t nq, uint32_t k, int transformed,
                         int n_threads, uint32_t* ids, float* dists, uint32_t* counts) {
    const uint32_t d = ix->d;
    if (n_threads <= 0) n_threads = 1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(n_threads)
    for (int64_t i = 0; i < (int64_t)nq; i++) {
        int m = pdxport_search(ix, q + (size_t)i * d, k, transformed, ids + (size_t)i * k, dists + (size_t)i * k);
        counts[i] = (uint32_t)(m < 0 ? 0 : m);
    }
    return 0;
}
