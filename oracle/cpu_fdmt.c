/*
 * TEST INFRASTRUCTURE ONLY — a CPU port of the dedispersion search for the
 * timed CPU baseline (bench.py's cpu_baseline leg and `--impl reference`).
 * frost's own CPU engine (dmt v0.8.0's FDMTBoxcar) is not available, so this
 * is this project's restatement, not dmt: its speed is not frost's shipped
 * CPU speed. It runs the same work as the GPU engine on one block with zero
 * history: the level-by-level FDMT of Zackay & Ofek (2017) under the split
 * rule of fdmt_oracle.c, in float with OpenMP over rows, then the boxcar
 * S/N of every searched row and width with run-based peak counting.
 *
 * Returns the number of above-threshold runs (peaks), or -1.
 */

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define KDISP 4.148808e3

typedef struct {
    int64_t a, m, b;     /* channels [a, b), split at m (leaf: b - a == 1) */
    int64_t lo, hi;      /* children */
    int64_t ndel, cap;
    int64_t* del;        /* sorted distinct delays */
    float* rows;         /* [ndel][T] */
    int keep;            /* rows still needed after the parent is computed */
} node_t;

static double kf(double a, double b) { return 1.0 / (a * a) - 1.0 / (b * b); }

typedef struct {
    node_t* n;
    int64_t count, cap;
    int64_t C;
    double fmin, fmax, tsamp;
} tree_t;

static double edge(const tree_t* t, int64_t c) {
    return t->fmin + (double)c * ((t->fmax - t->fmin) / (double)t->C);
}

static int64_t add_node(tree_t* t, int64_t a, int64_t m, int64_t b) {
    if (t->count == t->cap) {
        t->cap = t->cap ? 2 * t->cap : 1024;
        t->n   = (node_t*)realloc(t->n, sizeof(node_t) * (size_t)t->cap);
    }
    node_t* n = &t->n[t->count];
    memset(n, 0, sizeof(*n));
    n->a = a;
    n->m = m;
    n->b = b;
    n->lo = n->hi = -1;
    return t->count++;
}

static int64_t build(tree_t* t, int64_t a, int64_t b) {
    const int64_t m  = a + (b - a) / 2;
    const int64_t id = add_node(t, a, m, b);
    if (b - a > 1) {
        const int64_t lo = build(t, a, m);
        const int64_t hi = build(t, m, b);
        t->n[id].lo      = lo;
        t->n[id].hi      = hi;
    }
    return id;
}

static void push(node_t* n, int64_t d) {
    if (n->ndel == n->cap) {
        n->cap = n->cap ? 2 * n->cap : 16;
        n->del = (int64_t*)realloc(n->del, sizeof(int64_t) * (size_t)n->cap);
    }
    n->del[n->ndel++] = d;
}

static int cmp64(const void* x, const void* y) {
    const int64_t a = *(const int64_t*)x, b = *(const int64_t*)y;
    return (a > b) - (a < b);
}

static void uniq(node_t* n) {
    if (n->ndel == 0)
        return;
    qsort(n->del, (size_t)n->ndel, sizeof(int64_t), cmp64);
    int64_t k = 1;
    for (int64_t i = 1; i < n->ndel; ++i)
        if (n->del[i] != n->del[k - 1])
            n->del[k++] = n->del[i];
    n->ndel = k;
}

static int64_t find(const node_t* n, int64_t d) {
    int64_t lo = 0, hi = n->ndel - 1;
    while (lo <= hi) {
        const int64_t mid = (lo + hi) / 2;
        if (n->del[mid] == d)
            return mid;
        if (n->del[mid] < d)
            lo = mid + 1;
        else
            hi = mid - 1;
    }
    return -1;
}

static void split(const tree_t* t, const node_t* n, int64_t d, int64_t* dl, int64_t* dh) {
    const double r = kf(edge(t, n->m), edge(t, n->b)) / kf(edge(t, n->a), edge(t, n->b));
    *dh            = llround((double)d * r);
    *dl            = d - *dh;
}

/* Computes node rows bottom-up (recursion) from the [C][T] input. */
static void compute(tree_t* t, int64_t id, const float* in, int64_t T) {
    node_t* n = &t->n[id];
    if (n->ndel == 0 || n->rows != NULL)
        return;
    n->rows = (float*)malloc(sizeof(float) * (size_t)(n->ndel * T));
    if (n->b - n->a == 1) {
        const float* x = in + n->a * T;
#pragma omp parallel for schedule(static)
        for (int64_t r = 0; r < n->ndel; ++r) {
            const int64_t d = n->del[r];
            float* o        = n->rows + r * T;
            for (int64_t s = 0; s < T; ++s) {
                float acc = 0.0F;
                for (int64_t j = 0; j <= d && j <= s; ++j)
                    acc += x[s - j];
                o[s] = acc;
            }
        }
        return;
    }
    compute(t, n->lo, in, T);
    compute(t, n->hi, in, T);
    const node_t* lo = &t->n[n->lo];
    const node_t* hi = &t->n[n->hi];
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n->ndel; ++r) {
        int64_t dl, dh;
        split(t, n, n->del[r], &dl, &dh);
        const float* a = lo->rows + find(lo, dl) * T;
        const float* b = hi->rows + find(hi, dh) * T;
        float* o       = n->rows + r * T;
        for (int64_t s = 0; s < T; ++s)
            o[s] = a[s] + (s >= dl ? b[s - dl] : 0.0F);
    }
    /* children rows are no longer needed unless searched or shared */
    if (!t->n[n->lo].keep) {
        free(t->n[n->lo].rows);
        t->n[n->lo].rows = NULL;
    }
    if (!t->n[n->hi].keep) {
        free(t->n[n->hi].rows);
        t->n[n->hi].rows = NULL;
    }
}

/* Boxcar search of a node's searched rows; returns the peak count. */
static int64_t search_rows(const node_t* n, const int64_t* rows_idx, int64_t nrows, int64_t T,
                           const int64_t* widths, int64_t nw, const double* inv_sigma,
                           double thresh) {
    int64_t peaks = 0;
#pragma omp parallel for schedule(dynamic) reduction(+ : peaks)
    for (int64_t i = 0; i < nrows; ++i) {
        const float* x = n->rows + rows_idx[i] * T;
        float* pre     = (float*)malloc(sizeof(float) * (size_t)(T + 1));
        pre[0]         = 0.0F;
        for (int64_t s = 0; s < T; ++s)
            pre[s + 1] = pre[s] + x[s];
        for (int64_t w = 0; w < nw; ++w) {
            const int64_t W = widths[w];
            int open        = 0;
            const float inv = (float)inv_sigma[i * nw + w];
            for (int64_t s = W - 1; s < T; ++s) {
                const int up = (pre[s + 1] - pre[s + 1 - W]) * inv > (float)thresh;
                if (up && !open)
                    ++peaks;
                open = up;
            }
        }
        free(pre);
    }
    return peaks;
}

/* Searches the [C][T] block over the full band and, for depth >= 1, the
 * halving and staggered sub-bands. dm_list ascending. */
int64_t cpu_fdmt_search(const float* in, int64_t C, int64_t T, double f_min, double f_max,
                        double tsamp, const float* dm_list, int64_t ndm, int64_t depth,
                        const int64_t* widths, int64_t nw, double thresh) {
    tree_t t;
    memset(&t, 0, sizeof(t));
    t.C     = C;
    t.fmin  = f_min;
    t.fmax  = f_max;
    t.tsamp = tsamp;
    const int64_t root = build(&t, 0, C);
    /* searched bands: full band plus, per depth s, the tree bands and the
     * staggered merges of adjacent depth-(s+1) bands */
    int64_t nb = 1, capb = 64;
    int64_t* band = (int64_t*)malloc(sizeof(int64_t) * (size_t)capb);
    band[0]       = root;
    int64_t* cur  = (int64_t*)malloc(sizeof(int64_t) * (size_t)(2 * C + 2));
    int64_t* nxt  = (int64_t*)malloc(sizeof(int64_t) * (size_t)(2 * C + 2));
    int64_t ncur  = 1;
    cur[0]        = root;
    for (int64_t s = 1; s <= depth; ++s) {
        int64_t nn = 0;
        for (int64_t i = 0; i < ncur; ++i) {
            nxt[nn++] = t.n[cur[i]].lo;
            nxt[nn++] = t.n[cur[i]].hi;
        }
        for (int64_t i = 0; i < nn; ++i)
            band[nb++] = nxt[i];
        for (int64_t i = 0; i + 1 < nn; ++i) {
            const node_t* a = &t.n[t.n[nxt[i]].hi];
            const node_t* b = &t.n[t.n[nxt[i + 1]].lo];
            const int64_t id = add_node(&t, a->a, b->a, b->b);
            /* re-fetch after a possible realloc */
            t.n[id].lo = t.n[nxt[i]].hi;
            t.n[id].hi = t.n[nxt[i + 1]].lo;
            t.n[t.n[id].lo].keep = 1;
            t.n[t.n[id].hi].keep = 1;
            band[nb++] = id;
        }
        memcpy(cur, nxt, sizeof(int64_t) * (size_t)nn);
        ncur = nn;
    }
    /* demands: each band's distinct delays, then down the tree in order of
     * decreasing band width (parents before children) */
    int64_t** srows = (int64_t**)calloc((size_t)nb, sizeof(int64_t*));
    int64_t* nsr    = (int64_t*)calloc((size_t)nb, sizeof(int64_t));
    for (int64_t k = 0; k < nb; ++k) {
        node_t* n  = &t.n[band[k]];
        int64_t last = -1;
        for (int64_t i = 0; i < ndm; ++i) {
            const int64_t d = llround(KDISP * dm_list[i] * kf(edge(&t, n->a), edge(&t, n->b)) / tsamp);
            if (d != last)
                push(n, d);
            last = d;
        }
    }
    int64_t* order = (int64_t*)malloc(sizeof(int64_t) * (size_t)t.count);
    for (int64_t i = 0; i < t.count; ++i)
        order[i] = i;
    for (int64_t i = 1; i < t.count; ++i) { /* insertion sort by width, descending */
        const int64_t v = order[i];
        int64_t j       = i - 1;
        while (j >= 0 && (t.n[order[j]].b - t.n[order[j]].a) < (t.n[v].b - t.n[v].a)) {
            order[j + 1] = order[j];
            --j;
        }
        order[j + 1] = v;
    }
    for (int64_t i = 0; i < t.count; ++i) {
        node_t* n = &t.n[order[i]];
        uniq(n);
        if (n->b - n->a == 1)
            continue;
        for (int64_t r = 0; r < n->ndel; ++r) {
            int64_t dl, dh;
            split(&t, n, n->del[r], &dl, &dh);
            push(&t.n[n->lo], dl);
            push(&t.n[n->hi], dh);
        }
    }
    /* each node once: the regular tree, then the staggered bands from their
     * kept children; then every band is searched */
    for (int64_t k = 0; k < nb; ++k)
        t.n[band[k]].keep = 1;
    compute(&t, root, in, T);
    for (int64_t k = 0; k < nb; ++k)
        compute(&t, band[k], in, T);
    int64_t peaks = 0;
    for (int64_t k = 0; k < nb; ++k) {
        node_t* n = &t.n[band[k]];
        /* searched rows of this band: its distinct delays from the DM list */
        int64_t last = -1, ns = 0;
        int64_t* idx = (int64_t*)malloc(sizeof(int64_t) * (size_t)ndm);
        for (int64_t i = 0; i < ndm; ++i) {
            const int64_t d = llround(KDISP * dm_list[i] * kf(edge(&t, n->a), edge(&t, n->b)) / tsamp);
            if (d != last)
                idx[ns++] = find(n, d);
            last = d;
        }
        double* inv = (double*)malloc(sizeof(double) * (size_t)(ns * nw));
        for (int64_t i = 0; i < ns * nw; ++i)
            inv[i] = 1.0 / sqrt((double)(n->b - n->a) * (double)widths[i % nw]);
        peaks += search_rows(n, idx, ns, T, widths, nw, inv, thresh);
        free(n->rows);
        n->rows = NULL;
        free(idx);
        free(inv);
    }
    for (int64_t i = 0; i < t.count; ++i) {
        free(t.n[i].del);
        free(t.n[i].rows);
    }
    free(t.n);
    free(band);
    free(cur);
    free(nxt);
    free(srows);
    free(nsr);
    free(order);
    return peaks;
}
