/*
 * sc_oracle.c -- TEST INFRASTRUCTURE ONLY (see sc_oracle.h).
 *
 * Plain-C restatement of the reference search path, used as the checker for
 * the CUDA library.  Build with -O2 -ffp-contract=off so that every float
 * multiply and add rounds on its own, as in the reference built for x86-64.
 *
 * Two traversal orders are provided:
 *   ORC_ORDER_HEAP  -- the reference's own array heap (sc_utilities.h:229-300,
 *                      :469-503, :546-585), including its index arithmetic and
 *                      its fixed capacity.  This pins the reference.
 *   ORC_ORDER_EXACT -- the same multi-sequence push rules with an exact binary
 *                      heap keyed by (key, rank1, rank2).  Cells then come out
 *                      in ascending key order, ties broken by rank1 then rank2.
 *                      This is the order the CUDA library implements.
 * The two agree except where the reference heap pops a non-minimum (its
 * sift-down stops when a node's only child is the last element) or where keys
 * tie exactly.
 */
#include "sc_oracle.h"

#include <float.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* distance_l2_square<float>: float difference, double accumulation
 * (lib/simple-cluster/include/utilities.h:195-207). */
double orc_distance_l2_square(const float *x, const float *y, int d) {
    double dis = 0.0, tmp;
    for (int i = 0; i < d; i++) {
        tmp = (double)(x[i] - y[i]);
        dis += tmp * tmp;
    }
    return dis;
}

/* BLAS sdot taken as a sequential float loop (query.h:166,178). */
static float sdot_seq(int n, const float *x, const float *y) {
    float s = 0.0f;
    for (int i = 0; i < n; i++) s += x[i] * y[i];
    return s;
}

/* PQQuery::pre_compute1, query.h:91-149. */
void orc_pre_compute1(int dim, int mc, int kc, int mp, int kp,
                      const float *cq, const float *pq,
                      float *norm_c, float *norm_r, float *dot_cr) {
    int bsc = dim / mc, bsp = dim / mp;
    const float *v = cq;
    for (long i = 0; i < (long)mc * kc; i++) {
        float d = 0.0f;
        for (int j = 0; j < bsc; j++) { float t = *v++; d += t * t; }
        norm_c[i] = d;
    }
    v = pq;
    for (long i = 0; i < (long)mp * kp; i++) {
        float d = 0.0f;
        for (int j = 0; j < bsp; j++) { float t = *v++; d += t * t; }
        norm_r[i] = d;
    }
    size_t base = 0;
    const float *v1 = cq, *v2 = pq;
    for (int i = 0; i < mc; i++) {
        for (int j = 0; j < kc; j++) {
            const float *v3 = v2;
            for (int i1 = 0; i1 < mp / mc; i1++) {
                for (int j1 = 0; j1 < kp; j1++) {
                    float d = 0.0f;
                    for (int k = 0; k < bsp; k++) d += v1[k] * v3[k];
                    dot_cr[base++] = 2.0f * d;
                    v3 += bsp;
                }
                v1 += bsp;
            }
        }
        v2 += (size_t)kp * bsc;
    }
}

/* PQQuery::pre_compute2, query.h:154-184, with the intended sequencing: entry
 * `base` of each table receives norm[base] - d - d for the same `base` (the
 * reference statement `diff_qc[base] = norm_c[base++] - d - d` shifts the
 * table by one slot when the right-hand side is evaluated first). */
void orc_pre_compute2(int dim, int mc, int kc, int mp, int kp,
                      const float *cq, const float *pq,
                      const float *norm_c, const float *norm_r,
                      const float *q, float *diff_qc, float *diff_qr) {
    int bsc = dim / mc, bsp = dim / mp;
    const float *v1 = q, *v2 = cq;
    size_t base = 0;
    for (int i = 0; i < mc; i++) {
        for (int j = 0; j < kc; j++) {
            float d = sdot_seq(bsc, v1, v2);
            diff_qc[base] = norm_c[base] - d - d;
            base++;
            v2 += bsc;
        }
        v1 += bsc;
    }
    v1 = q; v2 = pq; base = 0;
    for (int i = 0; i < mp; i++) {
        for (int j = 0; j < kp; j++) {
            float d = sdot_seq(bsp, v1, v2);
            diff_qr[base] = norm_r[base] - d - d;
            base++;
            v2 += bsp;
        }
        v1 += bsp;
    }
}

/* ------------------------------------------------------------------------ */
/* The reference's array heaps (sc_utilities.h:229-300, :469-503, :546-585). */

typedef struct { float *key; int *h[4]; int pos, cap; } heap4;

static void swap_int(int *a, int *b) { int t = *a; *a = *b; *b = t; }
static void swap_flt(float *a, float *b) { float t = *a; *a = *b; *b = t; }

/* pq_insert4, sc_utilities.h:469-503: inserts past capacity are dropped. */
static void ref_insert4(heap4 *hp, float data, int a, int b, int c, int d) {
    if (hp->pos >= hp->cap || hp->pos < 0) return;
    int p = hp->pos;
    hp->key[p] = data; hp->h[0][p] = a; hp->h[1][p] = b; hp->h[2][p] = c; hp->h[3][p] = d;
    hp->pos++;
    int i = hp->pos - 1, j = i >> 1;
    while (i > 0) {
        if (hp->key[i] < hp->key[j]) {
            swap_flt(&hp->key[i], &hp->key[j]);
            for (int t = 0; t < 4; t++) swap_int(&hp->h[t][i], &hp->h[t][j]);
        } else break;
        i = j; j = i >> 1;
    }
}

/* pq_pop4, sc_utilities.h:546-585 (sift-down compares children 2i and 2i+1
 * only while both exist). */
static void ref_pop4(heap4 *hp, int *a, int *b, int *c, int *d) {
    int *h0 = hp->h[0], *h1 = hp->h[1], *h2 = hp->h[2], *h3 = hp->h[3];
    float *key = hp->key;
    *a = h0[0]; *b = h1[0]; *c = h2[0]; *d = h3[0];
    int last = hp->pos - 1;
    key[0] = key[last]; h0[0] = h0[last]; h1[0] = h1[last]; h2[0] = h2[last]; h3[0] = h3[last];
    hp->pos--;
    int cur = hp->pos, i = 0, j = 0, m;
    while (j + 1 < cur) {
        m = (key[j] < key[j + 1]) ? j : j + 1;
        if (key[m] < key[i]) {
            for (int t = 0; t < 4; t++) swap_int(&hp->h[t][i], &hp->h[t][m]);
            swap_flt(&key[i], &key[m]);
            i = m;
        } else break;
        j = i << 1;
    }
}

/* Exact binary heap on (key, rank1, rank2); used by ORC_ORDER_EXACT. */
static int ex_less(const heap4 *hp, int x, int y) {
    if (hp->key[x] < hp->key[y]) return 1;
    if (hp->key[x] > hp->key[y]) return 0;
    if (hp->h[0][x] != hp->h[0][y]) return hp->h[0][x] < hp->h[0][y];
    return hp->h[1][x] < hp->h[1][y];
}
static void ex_swap(heap4 *hp, int x, int y) {
    swap_flt(&hp->key[x], &hp->key[y]);
    for (int t = 0; t < 4; t++) swap_int(&hp->h[t][x], &hp->h[t][y]);
}
static void ex_insert4(heap4 *hp, float data, int a, int b, int c, int d) {
    int p = hp->pos++;
    hp->key[p] = data; hp->h[0][p] = a; hp->h[1][p] = b; hp->h[2][p] = c; hp->h[3][p] = d;
    while (p > 0) {
        int par = (p - 1) >> 1;
        if (ex_less(hp, p, par)) { ex_swap(hp, p, par); p = par; } else break;
    }
}
static void ex_pop4(heap4 *hp, int *a, int *b, int *c, int *d) {
    *a = hp->h[0][0]; *b = hp->h[1][0]; *c = hp->h[2][0]; *d = hp->h[3][0];
    hp->pos--;
    if (hp->pos == 0) return;
    ex_swap(hp, 0, hp->pos);
    int i = 0;
    for (;;) {
        int l = 2 * i + 1, r = l + 1, m = i;
        if (l < hp->pos && ex_less(hp, l, m)) m = l;
        if (r < hp->pos && ex_less(hp, r, m)) m = r;
        if (m == i) break;
        ex_swap(hp, i, m); i = m;
    }
}

static int heap_alloc(heap4 *hp, int cap) {
    hp->pos = 0; hp->cap = cap;
    hp->key = (float *)malloc(sizeof(float) * (size_t)(cap > 0 ? cap : 1));
    for (int t = 0; t < 4; t++) hp->h[t] = (int *)malloc(sizeof(int) * (size_t)(cap > 0 ? cap : 1));
    return hp->key != NULL;
}
static void heap_free(heap4 *hp) {
    free(hp->key);
    for (int t = 0; t < 4; t++) free(hp->h[t]);
}

/* The six-payload heap of the three-list walk: pq_insert6 / pq_pop6
 * (sc_utilities.h:505-544, :629-675), and an exact binary heap on (key,
 * rank1, rank2, rank3) for ORC_ORDER_EXACT. */
typedef struct { float *key; int *h[6]; int pos, cap; } heap6;

static int heap6_alloc(heap6 *hp, int cap) {
    hp->pos = 0; hp->cap = cap;
    hp->key = (float *)malloc(sizeof(float) * (size_t)(cap > 0 ? cap : 1));
    for (int t = 0; t < 6; t++) hp->h[t] = (int *)malloc(sizeof(int) * (size_t)(cap > 0 ? cap : 1));
    return hp->key != NULL;
}
static void heap6_free(heap6 *hp) {
    free(hp->key);
    for (int t = 0; t < 6; t++) free(hp->h[t]);
}
static void h6_swap(heap6 *hp, int x, int y) {
    swap_flt(&hp->key[x], &hp->key[y]);
    for (int t = 0; t < 6; t++) swap_int(&hp->h[t][x], &hp->h[t][y]);
}
/* pq_insert6: inserts past capacity are dropped; parent of i is i >> 1. */
static void ref_insert6(heap6 *hp, float data, const int *v) {
    if (hp->pos >= hp->cap || hp->pos < 0) return;
    int p = hp->pos;
    hp->key[p] = data;
    for (int t = 0; t < 6; t++) hp->h[t][p] = v[t];
    hp->pos++;
    int i = hp->pos - 1, j = i >> 1;
    while (i > 0) {
        if (hp->key[i] < hp->key[j]) h6_swap(hp, i, j);
        else break;
        i = j; j = i >> 1;
    }
}
/* pq_pop6: the sift-down compares children 2i and 2i+1 only while both exist. */
static void ref_pop6(heap6 *hp, int *v) {
    for (int t = 0; t < 6; t++) v[t] = hp->h[t][0];
    int last = hp->pos - 1;
    hp->key[0] = hp->key[last];
    for (int t = 0; t < 6; t++) hp->h[t][0] = hp->h[t][last];
    hp->pos--;
    int cur = hp->pos, i = 0, j = 0, m;
    while (j + 1 < cur) {
        m = (hp->key[j] < hp->key[j + 1]) ? j : j + 1;
        if (hp->key[m] < hp->key[i]) { h6_swap(hp, i, m); i = m; }
        else break;
        j = i << 1;
    }
}
static int ex6_less(const heap6 *hp, int x, int y) {
    if (hp->key[x] < hp->key[y]) return 1;
    if (hp->key[x] > hp->key[y]) return 0;
    for (int t = 0; t < 3; t++)
        if (hp->h[t][x] != hp->h[t][y]) return hp->h[t][x] < hp->h[t][y];
    return 0;
}
static void ex_insert6(heap6 *hp, float data, const int *v) {
    int p = hp->pos++;
    hp->key[p] = data;
    for (int t = 0; t < 6; t++) hp->h[t][p] = v[t];
    while (p > 0) {
        int par = (p - 1) >> 1;
        if (ex6_less(hp, p, par)) { h6_swap(hp, p, par); p = par; } else break;
    }
}
static void ex_pop6(heap6 *hp, int *v) {
    for (int t = 0; t < 6; t++) v[t] = hp->h[t][0];
    hp->pos--;
    if (hp->pos == 0) return;
    h6_swap(hp, 0, hp->pos);
    int i = 0;
    for (;;) {
        int l = 2 * i + 1, r = l + 1, m = i;
        if (l < hp->pos && ex6_less(hp, l, m)) m = l;
        if (r < hp->pos && ex6_less(hp, r, m)) m = r;
        if (m == i) break;
        h6_swap(hp, i, m); i = m;
    }
}

/* ------------------------------------------------------------------------ */

typedef struct { float v; int id; } vid;
static int cmp_vid(const void *a, const void *b) {
    const vid *x = (const vid *)a, *y = (const vid *)b;
    if (x->v < y->v) return -1;
    if (x->v > y->v) return 1;
    return (x->id > y->id) - (x->id < y->id);
}

/* Sorts n coarse keys ascending (sort_id / nth_element_id with M = kc,
 * sc_algorithm.h:24-75); equal keys are ordered by centroid id. */
static void sort_keys(const float *v, int n, float *vs, int *ids) {
    vid *t = (vid *)malloc(sizeof(vid) * (size_t)n);
    for (int i = 0; i < n; i++) { t[i].v = v[i]; t[i].id = i; }
    qsort(t, (size_t)n, sizeof(vid), cmp_vid);
    for (int i = 0; i < n; i++) { vs[i] = t[i].v; ids[i] = t[i].id; }
    free(t);
}

static int cell_len(const int *L, long bid) { return bid > 0 ? L[bid] - L[bid - 1] : L[0]; }

/* The largest rank of any coarse list among the cells the last orc_search
 * popped, empty cells included (IMI and second candidate; -1 otherwise). */
static int g_max_rank = -1;
int orc_last_max_rank(void) { return g_max_rank; }

/* Rank limit of the IMI and second-candidate walks (the library's
 * scg_set_rank_limit; the reference has none -- it sorts only the top M
 * ranks, multi_query.h:125-128, but walks on into the rest): ranks 0..M-1
 * of each sorted coarse list only; 0 = all. */
static int g_rank_limit = 0;
void orc_set_rank_limit(int M) { g_rank_limit = M; }
static long cell_start(const int *L, long bid) { return bid > 0 ? L[bid - 1] : 0; }

/* One query of PQQuery::search_ivfadc (query.h:202-325),
 * MultiQuery::search_multi2 (multi_query.h:62-273) or
 * SCQuery::search_mr_ivf (sc_query.h:60-256).  Writes the `sum` candidate
 * distances and ids in visiting order (the arrays the reference fills before
 * its top-R step) and the visited non-empty cells.  Returns 0, or -1 for bad
 * arguments, -2 when cap or cap_cells is too small. */
int orc_search(const orc_index *ix, int mode, int order, const float *q,
               int w, int T, int real_dist,
               float *dist, int *ids, int cap,
               int *cells, int cap_cells, int *ncells_out,
               int *sum_out, int *empty_out) {
    const int dim = ix->dim, kc = ix->kc, kp = ix->kp, mp = ix->mp, mc = ix->mc;
    g_max_rank = -1;
    if ((mode == ORC_IMI && mc != 2) || (mode != ORC_IMI && mc != 1)) return -1;
    if (mode == ORC_SC3 && (long)kc * kc * kc > 0x7fffffffL) return -1;
    if (real_dist && !ix->raw) return -1;
    const int *L = ix->L;

    float *diff_qc = (float *)malloc(sizeof(float) * (size_t)mc * kc);
    float *diff_qr = (float *)malloc(sizeof(float) * (size_t)mp * kp);
    orc_pre_compute2(dim, mc, kc, mp, kp, ix->cq, ix->pq, ix->norm_c, ix->norm_r, q, diff_qc, diff_qr);

    /* visited non-empty cells: cell id and the two coarse centroid ids */
    int nvis = 0, sum = 0, empty = 0, rc = 0;
    int *vis_h3 = (int *)malloc(sizeof(int) * (size_t)(cap_cells > 0 ? cap_cells : 1));
    int *vis_h4 = (int *)malloc(sizeof(int) * (size_t)(cap_cells > 0 ? cap_cells : 1));
    float q_sum = 0.0f;

    if (mode == ORC_IVFADC) {
        /* query.h:223-259 */
        for (int i = 0; i < dim; i++) { float t = q[i]; q_sum += t * t; }
        float *keys = (float *)malloc(sizeof(float) * (size_t)kc);
        int *order_ids = (int *)malloc(sizeof(int) * (size_t)kc);
        for (int i = 0; i < kc; i++) keys[i] = q_sum + diff_qc[i];
        int npop = 0;
        if (order == ORC_ORDER_HEAP) {
            heap4 hp; heap_alloc(&hp, kc);
            for (int i = 0; i < kc; i++) ref_insert4(&hp, keys[i], i, 0, 0, 0);
            /* pq_pop (sc_utilities.h:269-300) is pq_pop4 with one payload */
            while (npop < kc && hp.pos > 0) {
                int a, b, c, d; ref_pop4(&hp, &a, &b, &c, &d);
                order_ids[npop++] = a;
            }
            heap_free(&hp);
        } else {
            float *vs = (float *)malloc(sizeof(float) * (size_t)kc);
            sort_keys(keys, kc, vs, order_ids);
            npop = kc;
            free(vs);
        }
        for (int i = 0; i < w && i < npop; i++) {
            int bid = order_ids[i];
            int l = cell_len(L, bid);
            if (l > 0) {
                if (nvis >= cap_cells) { rc = -2; break; }
                cells[nvis] = bid; vis_h3[nvis] = bid; vis_h4[nvis] = 0; nvis++;
            } else empty++;
            sum += l;
            if (sum >= T) break;
        }
        free(keys); free(order_ids);
    } else if (mode == ORC_SC3) {
        /* SCQuery::search_mr_ivf3, sc_query.h:265-405: one sorted coarse list,
         * a multi-sequence over rank triples (h1, h2, h3) with key
         * (v[h1] + v[h2]) + v[h3]; cell (t[h1], t[h2], t[h3]) = t[h1] kc^2 +
         * t[h2] kc + t[h3]; the residual is relative to t[h1]. */
        for (int i2 = 0; i2 < dim; i2++) { float t = q[i2]; q_sum += t * t; }
        float *keys = (float *)malloc(sizeof(float) * (size_t)kc);
        float *v = (float *)malloc(sizeof(float) * (size_t)kc);
        int *t = (int *)malloc(sizeof(int) * (size_t)kc);
        for (int j = 0; j < kc; j++) keys[j] = q_sum + diff_qc[j];
        sort_keys(keys, kc, v, t);
        free(keys);
        const long kc2 = (long)kc * kc, size3 = kc2 * kc;
        unsigned char *trav = (unsigned char *)calloc((size_t)size3, 1);
        heap6 hp;
        heap6_alloc(&hp, order == ORC_ORDER_HEAP ? w : (int)(3 * kc2 + 8));
        void (*ins)(heap6 *, float, const int *) = (order == ORC_ORDER_HEAP) ? ref_insert6 : ex_insert6;
        void (*pop)(heap6 *, int *) = (order == ORC_ORDER_HEAP) ? ref_pop6 : ex_pop6;
        const int lim = (g_rank_limit > 0 && g_rank_limit < kc) ? g_rank_limit : kc;
        int hv[6] = {0, 0, 0, t[0], t[0], t[0]};
        ins(&hp, 3.0f * v[0], hv);                     /* sc_query.h:316-324 */
        long i = 0, count2 = 0;
        int h1 = 0, h2 = 0, h3 = 0;
        /* while(count < w && sum < T && count2 < size2), sc_query.h:327 */
        while (nvis < w && sum < T && count2 < size3) {
            /* An empty heap: the whole grid is exhausted (exact order) or the
             * capped heap dropped cells; the reference then re-pushes the
             * last cell's neighbours, the restatement stops. */
            if (hp.pos <= 0) break;
            pop(&hp, hv);
            h1 = hv[0]; h2 = hv[1]; h3 = hv[2];
            for (int t2 = 0; t2 < 3; t2++)
                if (hv[t2] > g_max_rank) g_max_rank = hv[t2];
            long bid = (long)hv[3] * kc2 + (long)hv[4] * kc + hv[5];
            int l = bid > 0 ? L[bid] - L[bid - 1] : 0;  /* sc_query.h:336-339 */
            if (l > 0) {
                if (nvis >= cap_cells) { rc = -2; break; }
                cells[nvis] = (int)bid; vis_h3[nvis] = hv[3]; vis_h4[nvis] = 0; nvis++;
                sum += l;
            } else empty++;
            i = kc2 * h1 + (long)kc * h2 + h3;
            trav[i] = 1;
            count2++;
            if (sum < T) {
                /* sc_query.h:350-400: push each neighbour once all its other
                 * predecessors are traversed */
                const long m1 = i + kc2 - kc, m2 = i + kc2 - 1, m3 = i + kc - 1;
                const long m4 = i + kc - kc2, m5 = i - kc + 1, m6 = i - kc2 + 1;
                if (h1 < lim - 1 && (h2 == 0 || (m1 < size3 && trav[m1])) && (h3 == 0 || (m2 < size3 && trav[m2]))) {
                    int nv[6] = {h1 + 1, h2, h3, t[h1 + 1], t[h2], t[h3]};
                    ins(&hp, v[h1 + 1] + v[h2] + v[h3], nv);
                }
                if (h2 < lim - 1 && (h3 == 0 || (m3 < size3 && trav[m3])) && (h1 == 0 || (m4 >= 0 && trav[m4]))) {
                    int nv[6] = {h1, h2 + 1, h3, t[h1], t[h2 + 1], t[h3]};
                    ins(&hp, v[h1] + v[h2 + 1] + v[h3], nv);
                }
                if (h3 < lim - 1 && (h2 == 0 || (m5 >= 0 && trav[m5])) && (h1 == 0 || (m6 >= 0 && trav[m6]))) {
                    int nv[6] = {h1, h2, h3 + 1, t[h1], t[h2], t[h3 + 1]};
                    ins(&hp, v[h1] + v[h2] + v[h3 + 1], nv);
                }
            }
        }
        heap6_free(&hp);
        free(trav); free(v); free(t);
    } else {
        const int two = (mode == ORC_IMI);
        float *v1 = (float *)malloc(sizeof(float) * (size_t)kc);
        float *v2 = (float *)malloc(sizeof(float) * (size_t)kc);
        int *t1 = (int *)malloc(sizeof(int) * (size_t)kc);
        int *t2 = (int *)malloc(sizeof(int) * (size_t)kc);
        float *tmpk = (float *)malloc(sizeof(float) * (size_t)kc);
        if (two) {
            /* multi_query.h:102-128 */
            int bsc = dim / mc;
            float qn[2];
            for (int i = 0; i < 2; i++) {
                float acc = 0.0f;
                for (int j = 0; j < bsc; j++) { float t = q[i * bsc + j]; acc += t * t; }
                q_sum += acc;
                qn[i] = acc;
            }
            for (int j = 0; j < kc; j++) tmpk[j] = qn[0] + diff_qc[j];
            sort_keys(tmpk, kc, v1, t1);
            for (int j = 0; j < kc; j++) tmpk[j] = qn[1] + diff_qc[kc + j];
            sort_keys(tmpk, kc, v2, t2);
        } else {
            /* sc_query.h:90-106 */
            for (int i = 0; i < dim; i++) { float t = q[i]; q_sum += t * t; }
            for (int j = 0; j < kc; j++) tmpk[j] = q_sum + diff_qc[j];
            sort_keys(tmpk, kc, v1, t1);
            memcpy(v2, v1, sizeof(float) * (size_t)kc);
            memcpy(t2, t1, sizeof(int) * (size_t)kc);
        }
        free(tmpk);

        const size_t grid = (size_t)kc * kc;
        unsigned char *trav = (unsigned char *)calloc(grid, 1);
        /* The reference heap holds at most w entries; the exact heap is sized
         * for the whole frontier (at most kc + 1 cells of a down-set grid). */
        heap4 hp;
        int cap_heap = (order == ORC_ORDER_HEAP) ? w : kc + 2;
        heap_alloc(&hp, cap_heap);
        void (*ins)(heap4 *, float, int, int, int, int) = (order == ORC_ORDER_HEAP) ? ref_insert4 : ex_insert4;
        void (*pop)(heap4 *, int *, int *, int *, int *) = (order == ORC_ORDER_HEAP) ? ref_pop4 : ex_pop4;

        int count2 = 0, h1 = 0, h2 = 0, h3, h4;
        long i = 0;
        const int lim = (g_rank_limit > 0 && g_rank_limit < kc) ? g_rank_limit : kc;
        if (two) {
            /* multi_query.h:133-149 */
            ins(&hp, v1[0] + v2[0], 0, 0, t1[0], t2[0]);
        } else {
            /* sc_query.h:113-128; the caller presets traversed[0]
             * (test_sc_query.cpp:160-161). */
            trav[0] = 1;
            float d0 = v1[0] + v1[1];
            if (lim >= 2) {
                ins(&hp, d0, 0, 1, t1[0], t1[1]);
                ins(&hp, d0, 1, 0, t1[1], t1[0]);
            }
        }
        for (;;) {
            /* IMI: while(count2 < w && sum < T) (multi_query.h:151);
             * SC:  while(count < w && sum < T)  (sc_query.h:130) */
            if (two ? (count2 >= w) : (nvis >= w)) break;
            if (sum >= T) break;
            /* An empty heap means the whole grid is exhausted; the reference
             * keeps looping there, the restatement stops. */
            if (hp.pos <= 0) break;
            pop(&hp, &h1, &h2, &h3, &h4);
            if (h1 > g_max_rank) g_max_rank = h1;
            if (h2 > g_max_rank) g_max_rank = h2;
            long bid = (long)h3 * kc + h4;
            int l;
            if (two) l = cell_len(L, bid);                /* multi_query.h:160-164 */
            else l = bid > 0 ? L[bid] - L[bid - 1] : 0;  /* sc_query.h:138-140   */
            if (l > 0) {
                if (nvis >= cap_cells) { rc = -2; break; }
                cells[nvis] = (int)bid; vis_h3[nvis] = h3; vis_h4[nvis] = h4; nvis++;
                sum += l;
            } else empty++;
            i = (long)h1 * kc + h2;
            trav[i] = 1;
            count2++;
            if (sum < T) {
                /* multi_query.h:175-204, sc_query.h:154-185: push (h1+1,h2)
                 * once (h1+1,h2-1) is traversed, (h1,h2+1) once (h1-1,h2+1)
                 * is traversed. */
                if (h1 < lim - 1 && (h2 == 0 || ((size_t)(i + kc - 1) < grid && trav[i + kc - 1])))
                    ins(&hp, v1[h1 + 1] + v2[h2], h1 + 1, h2, t1[h1 + 1], t2[h2]);
                if (h2 < lim - 1 && (h1 == 0 || (i - kc + 1 >= 0 && trav[i - kc + 1])))
                    ins(&hp, v1[h1] + v2[h2 + 1], h1, h2 + 1, t1[h1], t2[h2 + 1]);
            }
        }
        heap_free(&hp);
        free(trav);
        free(v1); free(v2); free(t1); free(t2);
    }

    if (rc == 0 && sum > cap) rc = -2;
    if (rc == 0) {
        /* The ADC scan: query.h:269-318, multi_query.h:216-262,
         * sc_query.h:201-239. */
        const int bs = kp * mp / mc;
        const int c = mp >> 1;
        int count = 0;
        for (int v = 0; v < nvis; v++) {
            long bid = cells[v];
            int l = cell_len(L, bid);
            long st = cell_start(L, bid);
            const unsigned char *ct = ix->codes + (size_t)st * mp;
            memcpy(&ids[count], ix->pid + st, sizeof(int) * (size_t)l);
            if (real_dist) {
                for (int j = 0; j < l; j++) {
                    dist[count] = (float)orc_distance_l2_square(q, ix->raw + (size_t)ix->pid[st + j] * dim, dim);
                    count++;
                }
                continue;
            }
            if (mode == ORC_IMI) {
                int h3 = vis_h3[v], h4 = vis_h4[v];
                float d0 = q_sum + diff_qc[h3] + diff_qc[kc + h4];
                size_t b1 = (size_t)h3 * bs, b2 = (size_t)(h4 + kc - 1) * bs;
                for (int j = 0; j < l; j++) {
                    float d = d0;
                    int base = 0;
                    for (int k = 0; k < c; k++) {
                        int bc = base + *ct++;
                        d += diff_qr[bc];
                        d += ix->dot_cr[b1 + bc];
                        base += kp;
                    }
                    for (int k = c; k < mp; k++) {
                        int bc = base + *ct++;
                        d += diff_qr[bc];
                        d += ix->dot_cr[b2 + bc];
                        base += kp;
                    }
                    dist[count++] = d;
                }
            } else {
                int h3 = vis_h3[v];
                float d0 = q_sum + diff_qc[h3];
                size_t b1 = (size_t)h3 * bs;
                for (int j = 0; j < l; j++) {
                    float d = d0;
                    int base = 0;
                    for (int k = 0; k < mp; k++) {
                        int bc = base + *ct++;
                        d += (diff_qr[bc] + ix->dot_cr[b1 + bc]);
                        base += kp;
                    }
                    dist[count++] = d;
                }
            }
        }
    }
    *ncells_out = nvis;
    *sum_out = sum;
    *empty_out = empty;
    free(vis_h3); free(vis_h4);
    free(diff_qc); free(diff_qr);
    return rc;
}

/* The top-R step (nth_element_id + sort_id, query.h:321-324): the R smallest
 * distances ascending; equal distances are ordered by id.  Writes min(R, n)
 * entries. */
void orc_topk(const float *dist, const int *ids, int n, int R, float *out_d, int *out_i) {
    vid *t = (vid *)malloc(sizeof(vid) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; i++) { t[i].v = dist[i]; t[i].id = ids[i]; }
    qsort(t, (size_t)n, sizeof(vid), cmp_vid);
    int m = n < R ? n : R;
    for (int i = 0; i < m; i++) { out_d[i] = t[i].v; out_i[i] = t[i].id; }
    free(t);
}

int orc_rerank(const float *raw, int dim, const float *q, const int *ids, int L, int R,
               int *out_ids, float *out_d) {
    float *d = (float *)malloc(sizeof(float) * (size_t)(L > 0 ? L : 1));
    int *v = (int *)malloc(sizeof(int) * (size_t)(L > 0 ? L : 1));
    int n = 0;
    for (int i = 0; i < L; i++) {
        if (ids[i] < 0) continue;
        d[n] = (float)orc_distance_l2_square(q, raw + (size_t)ids[i] * dim, dim);
        v[n] = ids[i];
        n++;
    }
    orc_topk(d, v, n, R, out_d, out_ids);
    free(d);
    free(v);
    return n < R ? n : R;
}

/* Encoder::encode<T>, encoder.h:69-192: per part the first nearest coarse
 * centroid (double distances, strict '>'), the float residual, then per
 * subspace the first nearest PQ centroid. */
void orc_encode(int dim, int mc, int kc, int mp, int kp,
                const float *cq, const float *pq, const float *X, long n,
                unsigned short *cid, unsigned char *codes) {
    int bsc = dim / mc, bsp = dim / mp;
    float *r = (float *)malloc(sizeof(float) * (size_t)dim);
    for (long row = 0; row < n; row++) {
        const float *x = X + (size_t)row * dim;
        for (int j = 0; j < mc; j++) {
            double d = DBL_MAX;
            int minp = 0;
            for (int k = 0; k < kc; k++) {
                double dt = orc_distance_l2_square(x + j * bsc, cq + ((size_t)j * kc + k) * bsc, bsc);
                if (d > dt) { d = dt; minp = k; }
            }
            cid[row * mc + j] = (unsigned short)minp;
            const float *cc = cq + ((size_t)j * kc + minp) * bsc;
            for (int k = 0; k < bsc; k++) r[j * bsc + k] = x[j * bsc + k] - cc[k];
        }
        for (int j = 0; j < mp; j++) {
            double d = DBL_MAX;
            int minp = 0;
            for (int k = 0; k < kp; k++) {
                double dt = orc_distance_l2_square(r + j * bsp, pq + ((size_t)j * kp + k) * bsp, bsp);
                if (d > dt) { d = dt; minp = k; }
            }
            codes[row * mp + j] = (unsigned char)minp;
        }
    }
    free(r);
}

/* SCEncoder::encode<T>, sc_encoder.h:205-332 (mc = 1): coarse distances
 * rounded to float, the nc nearest in ascending order (equal distances by
 * centroid id), residual w.r.t. the nearest, then per subspace the first
 * nearest PQ centroid under float comparison. */
void orc_sc_encode(int dim, int kc, int mp, int kp, int nc,
                   const float *cq, const float *pq, const float *X, long n,
                   unsigned short *cid, unsigned char *codes) {
    int bsp = dim / mp;
    float *r = (float *)malloc(sizeof(float) * (size_t)dim);
    float *dk = (float *)malloc(sizeof(float) * (size_t)kc);
    float *vs = (float *)malloc(sizeof(float) * (size_t)kc);
    int *id = (int *)malloc(sizeof(int) * (size_t)kc);
    for (long row = 0; row < n; row++) {
        const float *x = X + (size_t)row * dim;
        for (int k = 0; k < kc; k++) dk[k] = (float)orc_distance_l2_square(x, cq + (size_t)k * dim, dim);
        sort_keys(dk, kc, vs, id);
        for (int k = 0; k < nc; k++) cid[row * nc + k] = (unsigned short)id[k];
        const float *cc = cq + (size_t)id[0] * dim;
        for (int k = 0; k < dim; k++) r[k] = x[k] - cc[k];
        for (int j = 0; j < mp; j++) {
            float d = FLT_MAX;
            int minp = 0;
            for (int k = 0; k < kp; k++) {
                float dt = (float)orc_distance_l2_square(r + j * bsp, pq + ((size_t)j * kp + k) * bsp, bsp);
                if (d > dt) { d = dt; minp = k; }
            }
            codes[row * mp + j] = (unsigned char)minp;
        }
    }
    free(r); free(dk); free(vs); free(id);
}

/* Encoder::distribution (encoder.cpp:170-205) and SCEncoder::distribution
 * (sc_encoder.cpp:17-60) followed by the CSR layout PQQuery::load_encoded_data
 * builds (query.cpp:82-165): rows are bucketed by cell id in row order; L is
 * the inclusive prefix count per cell.  mode: ORC_IVFADC/ORC_IMI use
 * vector_base(cid, mc, kc); ORC_SC uses nn1*kc + nn2 (nc = 2).
 * Returns the number of non-empty cells. */
int orc_distribution(int mode, int kc, int mc, int nc, int mp, long n,
                     const unsigned short *cid, const unsigned char *codes,
                     int *L, int *pid, unsigned char *codes_out) {
    long ncells = 1;
    int parts = (mode == ORC_SC) ? nc : mc;
    for (int i = 0; i < parts; i++) ncells *= kc;
    long *cnt = (long *)calloc((size_t)ncells + 1, sizeof(long));
    long *cell_of = (long *)malloc(sizeof(long) * (size_t)(n > 0 ? n : 1));
    for (long r = 0; r < n; r++) {
        long h = 0;
        for (int i = 0; i < parts; i++) h = h * kc + cid[r * parts + i];
        cell_of[r] = h;
        cnt[h]++;
    }
    int non_empty = 0;
    long acc = 0;
    for (long c = 0; c < ncells; c++) {
        if (cnt[c] > 0) non_empty++;
        long l = cnt[c];
        cnt[c] = acc;           /* becomes the write cursor */
        acc += l;
        L[c] = (int)acc;
    }
    for (long r = 0; r < n; r++) {
        long p = cnt[cell_of[r]]++;
        pid[p] = (int)r;
        memcpy(codes_out + (size_t)p * mp, codes + (size_t)r * mp, (size_t)mp);
    }
    free(cnt); free(cell_of);
    return non_empty;
}
