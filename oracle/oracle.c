/*
 * oracle.c -- TEST INFRASTRUCTURE ONLY (see oracle.h).  CPU restatement of the
 * reference OIFT + relaxation path, used as the checker of the CUDA library.
 * Each routine cites the reference lines it restates.
 */
#include "oracle.h"

#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MAX(a, b) ((a) > (b) ? (a) : (b))
#define MIN(a, b) ((a) < (b) ? (a) : (b))

/* gft/src/gft_adjrel3.cpp:47-85: Spheric(r) enumerates dz, dy, dx in [-r0, r0] with
 * dx^2+dy^2+dz^2 <= (int)(r*r) and moves the centre to the front. */
int or_adjacency(int adj, int *dx, int *dy, int *dz) {
    int r2 = (adj == 26 || adj == 8) ? 3 : 1;
    int n = 0;
    for (int z = -1; z <= 1; z++)
        for (int y = -1; y <= 1; y++)
            for (int x = -1; x <= 1; x++) {
                if (x == 0 && y == 0 && z == 0) continue;
                if (x * x + y * y + z * z <= r2) {
                    dx[n] = x;
                    dy[n] = y;
                    dz[n] = z;
                    n++;
                }
            }
    return n;
}

static inline int in_bounds(int x, int y, int z, int X, int Y, int Z) {
    return x >= 0 && x < X && y >= 0 && y < Y && z >= 0 && z < Z;
}

void or_rbf_lut(double sigma, int wq, int len, uint16_t *lut) {
    for (int d = 0; d < len; d++) {
        double a = exp(-((double)d * (double)d) / (2.0 * sigma * sigma));
        double v = floor((double)wq * (1.0 - a) + 0.5);
        if (v < 0) v = 0;
        if (v > wq) v = wq;
        lut[d] = (uint16_t)v;
    }
}

long long or_build_weights(const int *img, int X, int Y, int Z, int adj, int mode, int wq,
                           const uint16_t *lut, int lut_len, const int *grad, float blend_a,
                           uint16_t *W) {
    int dx[26], dy[26], dz[26];
    int n = or_adjacency(adj, dx, dy, dz);
    int half = n / 2;
    size_t N = (size_t)X * Y * Z;
    long long nclamp = 0;
    int cap = (mode == OR_W_GRAD) ? OR_WMAX_BASE : MIN(wq, OR_WMAX_BASE);
    for (int k = 0; k < half; k++) {
        int d = half + k;
        uint16_t *plane = W + (size_t)k * N;
        for (int z = 0; z < Z; z++)
            for (int y = 0; y < Y; y++)
                for (int x = 0; x < X; x++) {
                    size_t p = (size_t)x + (size_t)y * X + (size_t)z * X * Y;
                    int qx = x + dx[d], qy = y + dy[d], qz = z + dz[d];
                    if (!in_bounds(qx, qy, qz, X, Y, Z)) {
                        plane[p] = 0;
                        continue;
                    }
                    size_t q = (size_t)qx + (size_t)qy * X + (size_t)qz * X * Y;
                    int ip = img[p], iq = img[q];
                    int ad = abs(ip - iq);
                    long long b;
                    switch (mode) {
                        case OR_W_GRAD:
                        case OR_W_GRAD_Q:
                            b = ad;
                            break;
                        case OR_W_RBF_Q:
                            b = (ad < lut_len) ? lut[ad] : lut[lut_len - 1];
                            break;
                        default: { /* BLEND_Q, exp_gradient_weight.cpp:244-247 */
                            float gavg = (float)(grad[p] + grad[q]) * 0.5f;
                            float wf = blend_a * (float)ad + (1.0f - blend_a) * gavg;
                            b = (long long)wf;
                            if (b < 0) b = 0;
                        }
                    }
                    if (b > cap) {
                        b = cap;
                        nclamp++;
                    }
                    uint16_t code = (uint16_t)b;
                    if (ip > iq) code |= 0x8000u;
                    if (ip < iq) code |= 0x4000u;
                    plane[p] = code;
                }
    }
    return nclamp;
}

/* gft/src/gft_ift.cpp:965-973: int w = |dI|; w *= (1.0 + per_pq/100.0) if I_p > I_q,
 * w *= (1.0 - per_pq/100.0) if I_p < I_q.  The int *= double truncates toward zero. */
int or_oriented(uint16_t base, int tail_gt, int tail_lt, float pol) {
    int w = base;
    if (tail_gt)
        w = (int)((double)w * (1.0 + (double)pol / 100.0));
    else if (tail_lt)
        w = (int)((double)w * (1.0 - (double)pol / 100.0));
    return w;
}

static inline float polarity_of(or_polarity pol, int lb) {
    if (lb >= 0 && lb < pol.ntable) return pol.table[lb];
    return pol.dflt;
}

/* Blend arc weight of OIFT_Multi_GradWeight (experiments/exp_gradient_weight.cpp:244-254):
 * wf = alpha |I_p - I_q| + (1 - alpha) (g_p + g_q) * 0.5f in float, oriented by
 * (int)(wf * (1 +/- per/100)) in float, (int)wf for equal intensities, at least 0. */
static inline int blend_weight(const int *img, const int *g, float alpha, size_t p, size_t q,
                               float pol) {
    float intensity_diff = (float)abs(img[p] - img[q]);
    float grad_avg = (g[p] + g[q]) * 0.5f;
    float wf = alpha * intensity_diff + (1.0f - alpha) * grad_avg;
    int w = (int)wf;
    if (img[p] > img[q])
        w = (int)(wf * (1.0f + pol / 100.0f));
    else if (img[p] < img[q])
        w = (int)(wf * (1.0f - pol / 100.0f));
    if (w < 0) w = 0;
    return w;
}

/* Arc p -> q of the 2D image graph, oriented from p's side with alpha = per/100 held in a
 * float: val = |I_p - I_q| + 1 (ImageGraph::ByEuclideanDistance, gft/src/gft_imagegraph.cpp:
 * 13-47), MAX(ROUND(val * (1.0 + alpha)), 1) if I_p > I_q, MAX(ROUND(val * (1.0 - alpha)), 1)
 * if I_p < I_q, val otherwise (Orient2Digraph, gft_imagegraph.cpp:981-1016; ROUND is
 * gft/include/gft_common.h:120). */
static inline int ig_link(const int *img, size_t p, size_t q, float alpha) {
    int val = abs(img[p] - img[q]) + 1;
    double x;
    if (img[p] > img[q])
        x = val * (1.0 + alpha);
    else if (img[p] < img[q])
        x = val * (1.0 - alpha);
    else
        return val;
    int w = (x < 0) ? (int)(x - 0.5) : (int)(x + 0.5);
    return w > 1 ? w : 1;
}

/* Alpha of a polarity given x100, as Orient2Digraph computes it: float alpha = per/100.0. */
static inline float ig_alpha(float per) { return (float)(per / 100.0); }

/* Where arc weights come from: edge-code planes W, the blend of image and gradient, or (ig)
 * the oriented image graph. */
typedef struct {
    const uint16_t *W;
    const int *img, *g;
    float alpha;
    int ig;
} wsrc;

/* Arc weight p -> q where q = p + d_i.  For i in the positive half the edge lives in
 * plane (i - half) at p; otherwise in plane (n-1-i - half) at q with the bits read
 * from q's side, i.e. swapped. */
static inline int arc_weight_codes(const uint16_t *W, size_t N, int n, int i, size_t p, size_t q,
                                   float pol) {
    int half = n / 2;
    uint16_t code;
    int gt, lt;
    if (i >= half) {
        code = W[(size_t)(i - half) * N + p];
        gt = (code >> 15) & 1;
        lt = (code >> 14) & 1;
    } else {
        code = W[(size_t)(n - 1 - i - half) * N + q];
        gt = (code >> 14) & 1; /* I_q < I_p seen from q means I_p > I_q */
        lt = (code >> 15) & 1;
    }
    return or_oriented((uint16_t)(code & 0x3fffu), gt, lt, pol);
}

static inline int arc_weight(const wsrc *ws, size_t N, int n, int i, size_t p, size_t q,
                             float pol) {
    /* OIFT(sImageGraph) (gft/src/gft_ift.cpp:1358-1439) takes n_link[p] for an object tail
     * and the transposed arc n_link[q] for a background tail: the arc from p's side with
     * the tail label's polarity (-per for label 0) */
    if (ws->ig) return ig_link(ws->img, p, q, ig_alpha(pol));
    if (ws->img) return blend_weight(ws->img, ws->g, ws->alpha, p, q, pol);
    return arc_weight_codes(ws->W, N, n, i, p, q, pol);
}

/* ---------------------------------------------------------------- binary heap --- */
typedef struct {
    uint64_t *k;
    size_t n, cap;
} heap64;

static void hpush(heap64 *h, uint64_t v) {
    if (h->n == h->cap) {
        h->cap = h->cap ? h->cap * 2 : 1024;
        h->k = (uint64_t *)realloc(h->k, h->cap * sizeof(uint64_t));
    }
    size_t i = h->n++;
    while (i > 0) {
        size_t par = (i - 1) / 2;
        if (h->k[par] <= v) break;
        h->k[i] = h->k[par];
        i = par;
    }
    h->k[i] = v;
}

static uint64_t hpop(heap64 *h) {
    uint64_t top = h->k[0];
    uint64_t v = h->k[--h->n];
    size_t i = 0;
    for (;;) {
        size_t l = 2 * i + 1, r = l + 1, m = i;
        uint64_t mv = v;
        if (l < h->n && h->k[l] < mv) { m = l; mv = h->k[l]; }
        if (r < h->n && h->k[r] < mv) { m = r; mv = h->k[r]; }
        if (m == i) break;
        h->k[i] = h->k[m];
        i = m;
    }
    if (h->n) h->k[i] = v;
    return top;
}

/* R2.  Key = (cost << 32 | label) << 24 | voxel would not fit; the heap holds
 * (cost << 48 | label << 32 | voxel) with voxel < 2^32, cost < 2^16, label < 2^16.
 * Ties inside one (cost,label) level pop in any order: the set conquered at a level
 * is a reachability closure, so the result does not depend on that order.  Seeds keep
 * their labels: OIFT_Multi enters them at value 0 and conquers a voxel only through
 * w < value[q] (gft/src/gft_ift.cpp:929-976), so no arc can take a seed from it. */
static int fmax_core(const wsrc *ws, int X, int Y, int Z, int adj, or_polarity pol,
                     const int *seeds, int nseeds, const int *label_in, int *cost, int *label,
                     int *pred) {
    int dx[26], dy[26], dz[26];
    int n = or_adjacency(adj, dx, dy, dz);
    size_t N = (size_t)X * Y * Z;
    unsigned char *done = (unsigned char *)calloc(N, 1);
    unsigned char *seed = (unsigned char *)calloc(N, 1);
    heap64 h = {0};
    for (size_t p = 0; p < N; p++) {
        cost[p] = INT32_MAX;
        label[p] = OR_NIL;
        if (pred) pred[p] = -1;
    }
    for (int i = 0; i < nseeds; i++) {
        int p = seeds[i];
        if (p < 0 || (size_t)p >= N) continue;
        int lb = label_in[p] < 0 ? 0 : label_in[p];
        seed[p] = 1;
        if (cost[p] == 0 && label[p] <= lb) continue;
        cost[p] = 0;
        label[p] = lb;
        hpush(&h, ((uint64_t)0 << 48) | ((uint64_t)lb << 32) | (uint64_t)p);
    }
    int levels = 0;
    uint64_t lastkey = UINT64_MAX;
    while (h.n) {
        uint64_t e = hpop(&h);
        size_t p = (size_t)(e & 0xffffffffu);
        int c = (int)(e >> 48), lb = (int)((e >> 32) & 0xffff);
        if (done[p] || c != cost[p] || lb != label[p]) continue; /* stale */
        done[p] = 1;
        if ((e >> 32) != lastkey) {
            levels++;
            lastkey = e >> 32;
        }
        float pl = polarity_of(pol, lb);
        int x = (int)(p % X), y = (int)((p / X) % Y), z = (int)(p / ((size_t)X * Y));
        for (int i = 0; i < n; i++) {
            int qx = x + dx[i], qy = y + dy[i], qz = z + dz[i];
            if (!in_bounds(qx, qy, qz, X, Y, Z)) continue;
            size_t q = (size_t)qx + (size_t)qy * X + (size_t)qz * X * Y;
            if (done[q] || seed[q]) continue;
            int w = arc_weight(ws, N, n, i, p, q, pl);
            int nc = MAX(c, w);
            if (nc < cost[q] || (nc == cost[q] && lb < label[q])) {
                cost[q] = nc;
                label[q] = lb;
                if (pred) pred[q] = (int)p;
                hpush(&h, ((uint64_t)nc << 48) | ((uint64_t)lb << 32) | (uint64_t)q);
            }
        }
    }
    free(h.k);
    free(done);
    free(seed);
    return levels;
}

int or_oift_fmax(const uint16_t *W, int X, int Y, int Z, int adj, or_polarity pol,
                 const int *seeds, int nseeds, const int *label_in,
                 int *cost, int *label, int *pred) {
    wsrc ws = {W, NULL, NULL, 0.0f};
    return fmax_core(&ws, X, Y, Z, adj, pol, seeds, nseeds, label_in, cost, label, pred);
}

/* R2 with the blend weights of OIFT_Multi_GradWeight. */
int or_oift_fmax_blend(const int *img, const int *g, float alpha, int X, int Y, int Z, int adj,
                       or_polarity pol, const int *seeds, int nseeds, const int *label_in,
                       int *cost, int *label) {
    wsrc ws = {NULL, img, g, alpha};
    return fmax_core(&ws, X, Y, Z, adj, pol, seeds, nseeds, label_in, cost, label, NULL);
}

/* R2 with the weights of the oriented 2D image graph. */
int or_oift_fmax_imagegraph(const int *img, int X, int Y, int adj, or_polarity pol,
                            const int *seeds, int nseeds, const int *label_in, int *cost,
                            int *label, int *pred) {
    wsrc ws = {NULL, img, NULL, 0.0f, 1};
    return fmax_core(&ws, X, Y, 1, adj, pol, seeds, nseeds, label_in, cost, label, pred);
}

/* ------------------------------------------------------- R1: Prim / Dial queue --- */
/* Restates PQueue32 (gft/src/gft_pqueue32.cpp:231-245 _BucketFIFO, 300-324
 * FastInsertElem with the backwards-moving minvalue at 312-313, 353-377
 * FastRemoveElem, 433-451 FastRemoveMinFIFO) and OIFT_Multi's loop
 * (gft/src/gft_ift.cpp:934-985). */
enum { WHITE = 0, GRAY = 1, BLACK = 2 };

typedef struct {
    int *first, *last, nb, minv;
    int *next, *prev;
    unsigned char *color;
    int *value;
} dialq;

static void dq_insert(dialq *Q, int e) {
    int b = Q->value[e];
    if (b < Q->minv) Q->minv = b;
    if (Q->first[b] == -1) {
        Q->first[b] = e;
        Q->prev[e] = -1;
    } else {
        Q->next[Q->last[b]] = e;
        Q->prev[e] = Q->last[b];
    }
    Q->last[b] = e;
    Q->next[e] = -1;
    Q->color[e] = GRAY;
}

static void dq_remove(dialq *Q, int e) {
    int b = Q->value[e], pv = Q->prev[e], nx = Q->next[e];
    if (Q->first[b] == e) {
        Q->first[b] = nx;
        if (nx == -1)
            Q->last[b] = -1;
        else
            Q->prev[nx] = -1;
    } else {
        Q->next[pv] = nx;
        if (nx == -1)
            Q->last[b] = pv;
        else
            Q->prev[nx] = pv;
    }
    Q->color[e] = BLACK;
}

static int dq_popmin(dialq *Q) {
    while (Q->first[Q->minv] == -1) Q->minv++;
    int b = Q->minv;
    int e = Q->first[b], nx = Q->next[e];
    if (nx == -1)
        Q->first[b] = Q->last[b] = -1;
    else {
        Q->first[b] = nx;
        Q->prev[nx] = -1;
    }
    Q->color[e] = BLACK;
    return e;
}

static void prim_core(const wsrc *ws, int X, int Y, int Z, int adj, or_polarity pol,
                      int wmax_buckets, const int *seeds, int nseeds, int *label,
                      int *value_out, int *pred_out, int *fmax_out) {
    int dx[26], dy[26], dz[26];
    int n = or_adjacency(adj, dx, dy, dz);
    size_t N = (size_t)X * Y * Z;
    dialq Q;
    Q.nb = wmax_buckets + 2;
    Q.first = (int *)malloc(sizeof(int) * (Q.nb + 1));
    Q.last = (int *)malloc(sizeof(int) * (Q.nb + 1));
    for (int b = 0; b <= Q.nb; b++) Q.first[b] = Q.last[b] = -1;
    Q.minv = Q.nb;
    Q.next = (int *)malloc(sizeof(int) * N);
    Q.prev = (int *)malloc(sizeof(int) * N);
    Q.color = (unsigned char *)calloc(N, 1);
    Q.value = (int *)malloc(sizeof(int) * N);
    int *pred = (int *)malloc(sizeof(int) * N);
    int *order = fmax_out ? (int *)malloc(sizeof(int) * N) : NULL;
    size_t norder = 0;
    for (size_t p = 0; p < N; p++) {
        Q.value[p] = (label[p] == OR_NIL) ? INT_MAX : 0;
        pred[p] = -1;
    }
    for (int i = 0; i < nseeds; i++) dq_insert(&Q, seeds[i]);
    /* Queue emptiness: count of GRAY elements. */
    size_t ingray = 0;
    for (size_t p = 0; p < N; p++) ingray += (Q.color[p] == GRAY);
    /* Duplicate seeds were inserted twice in the reference as well; mirror the list
     * semantics by counting list occupancy instead of colours. */
    long long occ = nseeds;
    (void)ingray;
    while (occ > 0) {
        int p = dq_popmin(&Q);
        occ--;
        if (order) order[norder++] = p;
        int x = p % X, y = (p / X) % Y, z = p / (X * Y);
        float pl = polarity_of(pol, label[p]);
        for (int i = 0; i < n; i++) {
            int qx = x + dx[i], qy = y + dy[i], qz = z + dz[i];
            if (!in_bounds(qx, qy, qz, X, Y, Z)) continue;
            int q = qx + qy * X + qz * X * Y;
            if (Q.color[q] == BLACK) continue;
            int w = arc_weight(ws, N, n, i, (size_t)p, (size_t)q, pl);
            if (w < Q.value[q]) {
                if (Q.color[q] == GRAY) {
                    dq_remove(&Q, q);
                    occ--;
                }
                Q.value[q] = w;
                label[q] = label[p];
                pred[q] = p;
                dq_insert(&Q, q);
                occ++;
            }
        }
    }
    if (value_out) memcpy(value_out, Q.value, sizeof(int) * N);
    if (pred_out) memcpy(pred_out, pred, sizeof(int) * N);
    if (fmax_out) {
        for (size_t p = 0; p < N; p++) fmax_out[p] = (label[p] == OR_NIL) ? INT32_MAX : 0;
        for (size_t k = 0; k < norder; k++) {
            int p = order[k];
            if (pred[p] >= 0) fmax_out[p] = MAX(fmax_out[pred[p]], Q.value[p]);
        }
        free(order);
    }
    free(pred);
    free(Q.first);
    free(Q.last);
    free(Q.next);
    free(Q.prev);
    free(Q.color);
    free(Q.value);
}

void or_oift_prim(const uint16_t *W, int X, int Y, int Z, int adj, or_polarity pol,
                  int wmax_buckets, const int *seeds, int nseeds, int *label,
                  int *value_out, int *pred_out, int *fmax_out) {
    wsrc ws = {W, NULL, NULL, 0.0f};
    prim_core(&ws, X, Y, Z, adj, pol, wmax_buckets, seeds, nseeds, label, value_out, pred_out,
              fmax_out);
}

/* R1 with the blend weights: OIFT_Multi_GradWeight (exp_gradient_weight.cpp:196-270). */
void or_oift_prim_blend(const int *img, const int *g, float alpha, int X, int Y, int Z, int adj,
                        or_polarity pol, int wmax_buckets, const int *seeds, int nseeds,
                        int *label) {
    wsrc ws = {NULL, img, g, alpha};
    prim_core(&ws, X, Y, Z, adj, pol, wmax_buckets, seeds, nseeds, label, NULL, NULL, NULL);
}

/* R1 on the oriented 2D image graph: OIFT(sImageGraph) (gft/src/gft_ift.cpp:1358-1439),
 * Dial queue of Wmax + 2 buckets, FIFO ties. */
void or_oift_prim_imagegraph(const int *img, int X, int Y, int adj, or_polarity pol,
                             int wmax, const int *seeds, int nseeds, int *label, int *value_out,
                             int *pred_out, int *fmax_out) {
    wsrc ws = {NULL, img, NULL, 0.0f, 1};
    prim_core(&ws, X, Y, 1, adj, pol, wmax, seeds, nseeds, label, value_out, pred_out, fmax_out);
}

/* sg->Wmax after Orient2Digraph (gft_imagegraph.cpp:981-1016): the largest oriented arc
 * weight over every in-image arc p -> q, seen from p with the global alpha; 0 without arcs. */
int or_imagegraph_wmax(const int *img, int X, int Y, int adj, float per) {
    int dx[26], dy[26], dz[26];
    int n = or_adjacency(adj, dx, dy, dz);
    float alpha = ig_alpha(per);
    int wmax = 0;
    for (int y = 0; y < Y; y++)
        for (int x = 0; x < X; x++)
            for (int i = 0; i < n; i++) {
                if (dz[i] != 0) continue;
                int qx = x + dx[i], qy = y + dy[i];
                if (qx < 0 || qx >= X || qy < 0 || qy >= Y) continue;
                int w = ig_link(img, (size_t)x + (size_t)y * X, (size_t)qx + (size_t)qy * X, alpha);
                if (w > wmax) wmax = w;
            }
    return wmax;
}

/* GetEnergy_Min(sImageGraph, label, lb) (gft/src/gft_ift.cpp:287-319): the smallest
 * oriented weight n_link[p] (global alpha, seen from p) over the arcs p -> q that leave
 * label lb; INT_MAX without such an arc. */
int or_energy_imagegraph(const int *img, int X, int Y, int adj, float per, const int *label,
                         int lb) {
    int dx[26], dy[26], dz[26];
    int n = or_adjacency(adj, dx, dy, dz);
    float alpha = ig_alpha(per);
    int e = INT_MAX;
    for (int y = 0; y < Y; y++)
        for (int x = 0; x < X; x++) {
            size_t p = (size_t)x + (size_t)y * X;
            if (label[p] != lb) continue;
            for (int i = 0; i < n; i++) {
                if (dz[i] != 0) continue;
                int qx = x + dx[i], qy = y + dy[i];
                if (qx < 0 || qx >= X || qy < 0 || qy >= Y) continue;
                size_t q = (size_t)qx + (size_t)qy * X;
                if (label[q] == lb) continue;
                int w = ig_link(img, p, q, alpha);
                if (w < e) e = w;
            }
        }
    return e;
}

/* ORelax_1(sImageGraph) (gft/src/gft_ift.cpp:7683-7847) in FP32: one membership value per
 * pixel, label / Imax at the start and at the seeds after every sweep; the mask starts at
 * the pixels with a differently-labelled neighbour and grows one ring after every sweep
 * but the last; a mask pixel takes sum(w m_q) / sum(w) over its neighbours with
 * w = (Wmax - n_link)^8, where n_link is the arc p -> q when m_q < 0.5 and q -> p
 * otherwise; the result is 1 where m >= 0.5 (and where it is NaN), else 0.  label is
 * replaced by that result and m_out receives the final memberships. */
void or_relax_imagegraph_f32(const int *img, int X, int Y, int adj, float per,
                             const int *seeds, int nseeds, int *label, int ntimes,
                             float *m_out) {
    int dx[26], dy[26], dz[26];
    int n0 = or_adjacency(adj, dx, dy, dz), n = 0;
    int ox[8], oy[8];
    for (int i = 0; i < n0; i++)
        if (dz[i] == 0) {
            ox[n] = dx[i];
            oy[n] = dy[i];
            n++;
        }
    size_t N = (size_t)X * Y;
    float alpha = ig_alpha(per);
    int wmax = or_imagegraph_wmax(img, X, Y, adj, per);
    int imax = label[0];
    for (size_t p = 1; p < N; p++) imax = label[p] > imax ? label[p] : imax;
    float *f1 = (float *)malloc(sizeof(float) * N), *f2 = (float *)malloc(sizeof(float) * N);
    unsigned char *mask = (unsigned char *)calloc(N, 1);
    int *nodes = (int *)malloc(sizeof(int) * N);
    size_t nn = 0;
    for (size_t p = 0; p < N; p++) {
        f1[p] = (float)label[p] / (float)imax;
        int px = (int)(p % X), py = (int)(p / X);
        for (int i = 0; i < n; i++) {
            int qx = px + ox[i], qy = py + oy[i];
            if (qx < 0 || qx >= X || qy < 0 || qy >= Y) continue;
            if (label[p] != label[qx + qy * X]) {
                mask[p] = 1;
                nodes[nn++] = (int)p;
                break;
            }
        }
    }
    size_t ninic = 0;
    while (ntimes > 0) {
        memcpy(f2, f1, sizeof(float) * N);
        for (size_t j = 0; j < nn; j++) {
            int p = nodes[j], px = p % X, py = p / X;
            float acc = 0.0f, sw = 0.0f;
            for (int i = 0; i < n; i++) {
                int qx = px + ox[i], qy = py + oy[i];
                if (qx < 0 || qx >= X || qy < 0 || qy >= Y) continue;
                int q = qx + qy * X;
                float w = (f1[q] < 0.5f) ? (float)ig_link(img, (size_t)p, (size_t)q, alpha)
                                         : (float)ig_link(img, (size_t)q, (size_t)p, alpha);
                w = (float)wmax - w;
                w = w * w;
                w = w * w;
                w = w * w;
                sw += w;
                acc += w * f1[q];
            }
            f2[p] = acc / sw;
        }
        float *t = f1;
        f1 = f2;
        f2 = t;
        for (int i = 0; i < nseeds; i++) f1[seeds[i]] = (float)label[seeds[i]] / (float)imax;
        ntimes--;
        if (ntimes > 0) {
            size_t last = nn;
            for (size_t j = ninic; j < nn; j++) {
                int p = nodes[j], px = p % X, py = p / X;
                for (int i = 0; i < n; i++) {
                    int qx = px + ox[i], qy = py + oy[i];
                    if (qx < 0 || qx >= X || qy < 0 || qy >= Y) continue;
                    int q = qx + qy * X;
                    if (!mask[q]) {
                        mask[q] = 1;
                        nodes[last++] = q;
                    }
                }
            }
            ninic = nn;
            nn = last;
        }
    }
    for (size_t p = 0; p < N; p++) {
        label[p] = (f1[p] < 0.5f) ? 0 : 1;
        if (m_out) m_out[p] = f1[p];
    }
    free(f1);
    free(f2);
    free(mask);
    free(nodes);
}

/* R4: gft/src/gft_ift.cpp:287-319 (GetEnergy_Min) in 3D with OIFT_Multi's oriented
 * arc weights (gft_ift.cpp:965-973), tail label selecting the polarity. */
int or_energy(const uint16_t *W, int X, int Y, int Z, int adj, or_polarity pol,
              const int *label, int nl, int *energy_lb) {
    int dx[26], dy[26], dz[26];
    int n = or_adjacency(adj, dx, dy, dz);
    size_t N = (size_t)X * Y * Z;
    int e = INT32_MAX;
    for (int l = 0; l < nl; l++) energy_lb[l] = INT32_MAX;
    for (int z = 0; z < Z; z++)
        for (int y = 0; y < Y; y++)
            for (int x = 0; x < X; x++) {
                size_t p = (size_t)x + (size_t)y * X + (size_t)z * X * Y;
                int lp = label[p];
                float pl = polarity_of(pol, lp);
                for (int i = 0; i < n; i++) {
                    int qx = x + dx[i], qy = y + dy[i], qz = z + dz[i];
                    if (!in_bounds(qx, qy, qz, X, Y, Z)) continue;
                    size_t q = (size_t)qx + (size_t)qy * X + (size_t)qz * X * Y;
                    if (label[q] == lp) continue;
                    int w = arc_weight_codes(W, N, n, i, p, q, pl);
                    e = MIN(e, w);
                    if (lp >= 0 && lp < nl) energy_lb[lp] = MIN(energy_lb[lp], w);
                }
            }
    return e;
}

/* Equal-cost tie accounting.  A label l "offers" voxel p its cost when some in-bounds
 * neighbour q labelled l reaches p at exactly cost[p]: MAX(cost[q], w_l(q -> p)) ==
 * cost[p], w_l the oriented weight of gft_ift.cpp:965-973 with the polarity of the
 * tail's label l.  Non-seed voxels only (seeds hold cost 0 by definition).
 *   out[0] = voxels offered their cost by >= 2 labels in labelling A (tie voxels of A);
 *   out[1] = voxels where labA != labB;
 *   out[2] = of those, voxels where labA[p] is offered in A and labB[p] is offered in B
 *            (both labellings' labels reach p at the same cost: an equal-cost tie);
 *   out[3] = out[1] - out[2] (differences that are not explained by a tie).
 * flags (optional, per voxel): bit 0 tie in A, bit 1 labels differ, bit 2 classified. */
static int offered(const uint16_t *W, size_t N, int n, const int *dx, const int *dy,
                   const int *dz, int X, int Y, int Z, or_polarity pol, const int *cost,
                   const int *lab, size_t p, int want) {
    int x = (int)(p % X), y = (int)((p / X) % Y), z = (int)(p / ((size_t)X * Y));
    for (int i = 0; i < n; i++) {
        int qx = x + dx[i], qy = y + dy[i], qz = z + dz[i];
        if (!in_bounds(qx, qy, qz, X, Y, Z)) continue;
        size_t q = (size_t)qx + (size_t)qy * X + (size_t)qz * X * Y;
        if (lab[q] != want || cost[q] == INT32_MAX) continue;
        /* the arc q -> p is direction n-1-i seen from q */
        int w = arc_weight_codes(W, N, n, n - 1 - i, q, p, polarity_of(pol, want));
        if (MAX(cost[q], w) == cost[p]) return 1;
    }
    return 0;
}

void or_tie_stats(const uint16_t *W, int X, int Y, int Z, int adj, or_polarity pol,
                  const int *cost, const int *labA, const int *labB,
                  const unsigned char *is_seed, long long *out, unsigned char *flags) {
    int dx[26], dy[26], dz[26];
    int n = or_adjacency(adj, dx, dy, dz);
    size_t N = (size_t)X * Y * Z;
    out[0] = out[1] = out[2] = out[3] = 0;
    for (size_t p = 0; p < N; p++) {
        unsigned char f = 0;
        if (!is_seed[p] && cost[p] != INT32_MAX) {
            /* labels offering p its cost in A: stop at the second distinct one */
            int first = OR_NIL, two = 0;
            int x = (int)(p % X), y = (int)((p / X) % Y), z = (int)(p / ((size_t)X * Y));
            for (int i = 0; i < n && !two; i++) {
                int qx = x + dx[i], qy = y + dy[i], qz = z + dz[i];
                if (!in_bounds(qx, qy, qz, X, Y, Z)) continue;
                size_t q = (size_t)qx + (size_t)qy * X + (size_t)qz * X * Y;
                int lq = labA[q];
                if (lq < 0 || lq == first || cost[q] == INT32_MAX) continue;
                int w = arc_weight_codes(W, N, n, n - 1 - i, q, p, polarity_of(pol, lq));
                if (MAX(cost[q], w) != cost[p]) continue;
                if (first == OR_NIL) first = lq;
                else two = 1;
            }
            if (two) {
                f |= 1;
                out[0]++;
            }
            if (labA[p] != labB[p]) {
                f |= 2;
                out[1]++;
                if (offered(W, N, n, dx, dy, dz, X, Y, Z, pol, cost, labA, p, labA[p]) &&
                    offered(W, N, n, dx, dy, dz, X, Y, Z, pol, cost, labB, p, labB[p])) {
                    f |= 4;
                    out[2]++;
                }
            }
        } else if (labA[p] != labB[p]) {
            f |= 2;
            out[1]++;
        }
        if (flags) flags[p] = f;
    }
    out[3] = out[1] - out[2];
}

/* gft/src/gft_ift.cpp:8684-8720 */
int or_relax_classes(const int *seeds, int nseeds, const int *label, int n,
                     int *class_labels, int cap) {
    int maxl = 0;
    for (int i = 0; i < nseeds; i++) {
        int p = seeds[i];
        if (p >= 0 && p < n) maxl = MAX(maxl, label[p]);
    }
    maxl = MAX(0, maxl);
    char *present = (char *)calloc((size_t)maxl + 1, 1);
    present[0] = 1;
    for (int i = 0; i < nseeds; i++) {
        int p = seeds[i];
        if (p >= 0 && p < n) {
            int lb = label[p];
            if (lb >= 0 && lb <= maxl) present[lb] = 1;
        }
    }
    int nc = 0;
    for (int l = 0; l <= maxl; l++)
        if (present[l]) {
            if (nc < cap) class_labels[nc] = l;
            nc++;
        }
    free(present);
    return nc;
}

/* ------------------------------------------------------------------ R3 relax --- */
/* One template body for FP32 and FP64: T is the membership / weight type.  The FP32
 * instance performs exactly the float operations of gft_ift.cpp:8778-8833 (global)
 * and 9058-9110 (per class) in the same order. */
#define RELAX_BODY(T, FABS, SQRT)                                                          \
    int dxa[26], dya[26], dza[26];                                                          \
    int na = or_adjacency(adj, dxa, dya, dza);                                              \
    int n = X * Y * Z;                                                                      \
    int cl[512];                                                                            \
    int nc = or_relax_classes(seeds, nseeds, label, n, cl, 512);                            \
    if (nc > 512) return -1;                                                                \
    int maxl = cl[nc - 1];                                                                  \
    int *l2c = (int *)malloc(sizeof(int) * (maxl + 1));                                     \
    for (int l = 0; l <= maxl; l++) l2c[l] = -1;                                            \
    for (int c = 0; c < nc; c++) l2c[cl[c]] = c;                                            \
    int bgc = l2c[0] < 0 ? 0 : l2c[0];                                                      \
    T pcm[512];                                                                             \
    float max_abs_per = 0.0f;                                                               \
    if (per_class) {                                                                        \
        for (int c = 0; c < nc; c++) {                                                      \
            float v = (cl[c] <= max_label) ? per_class[cl[c]] : 0.0f;                       \
            pcm[c] = (T)v;                                                                  \
            if (fabsf(v) > max_abs_per) max_abs_per = fabsf(v);                             \
        }                                                                                   \
    } else {                                                                                \
        max_abs_per = fabsf(per);                                                           \
    }                                                                                       \
    T Dpq[26];                                                                              \
    for (int i = 0; i < na; i++)                                                            \
        Dpq[i] = SQRT((T)(dxa[i] * dxa[i]) * (T)1 * (T)1 + (T)(dya[i] * dya[i]) * (T)1 * (T)1 + \
                      (T)(dza[i] * dza[i]) * (T)1 * (T)1) / (T)1;                           \
    int imax = img[0];                                                                      \
    for (int p = 1; p < n; p++) imax = MAX(imax, img[p]);                                   \
    T Wmax = (T)imax;                                                                       \
    if (blend) { /* exp_gradient_weight.cpp:338-339, in float */                            \
        float wm = (float)imax;                                                             \
        wm *= (1.0f + fabsf(per) / 100.0f);                                                 \
        Wmax = (T)wm;                                                                       \
    } else {                                                                                \
        Wmax = (T)((double)Wmax * (1.0 + (double)max_abs_per / 100.0));                     \
    }                                                                                       \
    size_t tot = (size_t)n * nc;                                                            \
    T *f1 = (T *)calloc(tot, sizeof(T)), *f2 = (T *)calloc(tot, sizeof(T));                 \
    int *mask_nodes = (int *)malloc(sizeof(int) * (n + 1));                                 \
    unsigned char *mask = (unsigned char *)calloc(n, 1);                                    \
    mask_nodes[0] = 0;                                                                      \
    for (int p = 0; p < n; p++) {                                                           \
        int lb = label[p], c = bgc;                                                         \
        if (lb >= 0 && lb <= maxl && l2c[lb] >= 0) c = l2c[lb];                             \
        f1[(size_t)p * nc + c] = (T)1;                                                      \
        int x = p % X, y = (p / X) % Y, z = p / (X * Y);                                    \
        for (int i = 0; i < na; i++) {                                                      \
            int qx = x + dxa[i], qy = y + dya[i], qz = z + dza[i];                          \
            if (!in_bounds(qx, qy, qz, X, Y, Z)) continue;                                  \
            int q = qx + qy * X + qz * X * Y;                                               \
            if (label[p] != label[q]) {                                                     \
                mask[p] = 1;                                                                \
                mask_nodes[++mask_nodes[0]] = p;                                            \
                break;                                                                      \
            }                                                                               \
        }                                                                                   \
    }                                                                                       \
    int ninic = 1;                                                                          \
    while (ntimes > 0) {                                                                    \
        memcpy(f2, f1, tot * sizeof(T));                                                    \
        for (int j = 1; j <= mask_nodes[0]; j++) {                                          \
            int p = mask_nodes[j];                                                          \
            int x = p % X, y = (p / X) % Y, z = p / (X * Y);                                \
            size_t po = (size_t)p * nc;                                                     \
            for (int k = 0; k < nc; k++) f2[po + k] = (T)0;                                 \
            T sw = (T)0;                                                                    \
            for (int i = 0; i < na; i++) {                                                  \
                int qx = x + dxa[i], qy = y + dya[i], qz = z + dza[i];                      \
                if (!in_bounds(qx, qy, qz, X, Y, Z)) continue;                              \
                int q = qx + qy * X + qz * X * Y;                                           \
                size_t qo = (size_t)q * nc;                                                 \
                T w = FABS((T)(img[p] - img[q]));                                           \
                if (blend) { /* exp_gradient_weight.cpp:403-405 */                          \
                    T grad_avg = (T)(g[p] + g[q]) * (T)0.5f;                                \
                    w = (T)alpha * w + ((T)1 - (T)alpha) * grad_avg;                        \
                }                                                                           \
                T per_pq;                                                                   \
                if (per_class) {                                                            \
                    per_pq = (T)0;                                                          \
                    for (int k = 0; k < nc; k++) per_pq += pcm[k] * f1[qo + k];             \
                } else {                                                                    \
                    T p_bg = f1[qo + bgc];                                                  \
                    per_pq = (T)per * ((T)2 * p_bg - (T)1);                                 \
                }                                                                           \
                if (img[p] > img[q])                                                        \
                    w *= ((T)1 + per_pq / (T)100);                                          \
                else if (img[p] < img[q])                                                   \
                    w *= ((T)1 - per_pq / (T)100);                                          \
                if (blend && w < (T)0) w = (T)0;                                            \
                w = Wmax - w;                                                               \
                if (w < (T)0) w = (T)0;                                                     \
                w = w * w;                                                                  \
                w = w * w;                                                                  \
                w = w * w;                                                                  \
                w /= Dpq[i];                                                                \
                sw += w;                                                                    \
                for (int k = 0; k < nc; k++) f2[po + k] += w * f1[qo + k];                  \
            }                                                                               \
            if (sw > (T)0) {                                                                \
                for (int k = 0; k < nc; k++) f2[po + k] /= sw;                              \
            } else {                                                                        \
                for (int k = 0; k < nc; k++) f2[po + k] = f1[po + k];                       \
            }                                                                               \
        }                                                                                   \
        T *tmp = f1;                                                                        \
        f1 = f2;                                                                            \
        f2 = tmp;                                                                           \
        for (int i = 0; i < nseeds; i++) {                                                  \
            int p = seeds[i];                                                               \
            if (p < 0 || p >= n) continue;                                                  \
            int lb = label[p], c = bgc;                                                     \
            if (lb >= 0 && lb <= maxl && l2c[lb] >= 0) c = l2c[lb];                         \
            size_t po = (size_t)p * nc;                                                     \
            for (int k = 0; k < nc; k++) f1[po + k] = (T)0;                                 \
            f1[po + c] = (T)1;                                                              \
        }                                                                                   \
        ntimes--;                                                                           \
        if (ntimes > 0) {                                                                   \
            int nlast = mask_nodes[0];                                                      \
            for (int j = ninic; j <= mask_nodes[0]; j++) {                                  \
                int p = mask_nodes[j];                                                      \
                int x = p % X, y = (p / X) % Y, z = p / (X * Y);                            \
                for (int i = 0; i < na; i++) {                                              \
                    int qx = x + dxa[i], qy = y + dya[i], qz = z + dza[i];                  \
                    if (!in_bounds(qx, qy, qz, X, Y, Z)) continue;                          \
                    int q = qx + qy * X + qz * X * Y;                                       \
                    if (!mask[q]) {                                                         \
                        mask[q] = 1;                                                        \
                        mask_nodes[++nlast] = q;                                            \
                    }                                                                       \
                }                                                                           \
            }                                                                               \
            ninic = mask_nodes[0] + 1;                                                      \
            mask_nodes[0] = nlast;                                                          \
        }                                                                                   \
    }                                                                                       \
    for (int p = 0; p < n; p++) {                                                           \
        size_t po = (size_t)p * nc;                                                         \
        int best = 0;                                                                       \
        T bv = f1[po];                                                                      \
        for (int k = 1; k < nc; k++)                                                        \
            if (f1[po + k] > bv) {                                                          \
                bv = f1[po + k];                                                            \
                best = k;                                                                   \
            }                                                                               \
        label[p] = cl[best];                                                                \
    }                                                                                       \
    if (membership)                                                                         \
        for (int k = 0; k < nc; k++)                                                        \
            for (int p = 0; p < n; p++) membership[(size_t)k * n + p] = f1[(size_t)p * nc + k]; \
    free(l2c);                                                                              \
    free(f1);                                                                               \
    free(f2);                                                                               \
    free(mask_nodes);                                                                       \
    free(mask);                                                                             \
    return nc;

int or_relax_f32(const int *img, int X, int Y, int Z, int adj, float per,
                 const float *per_class, int max_label,
                 const int *seeds, int nseeds, int *label, int ntimes, float *membership) {
    const int blend = 0, *g = NULL;
    const float alpha = 1.0f;
    RELAX_BODY(float, fabsf, sqrtf)
}

int or_relax_f64(const int *img, int X, int Y, int Z, int adj, float per,
                 const float *per_class, int max_label,
                 const int *seeds, int nseeds, int *label, int ntimes, double *membership) {
    const int blend = 0, *g = NULL;
    const float alpha = 1.0f;
    RELAX_BODY(double, fabs, sqrt)
}

/* ORelax_1_Multi_GradWeight (experiments/exp_gradient_weight.cpp:272-503): the relaxation
 * with blend weights wf = alpha |dI| + (1 - alpha)(g_p + g_q) * 0.5f, oriented by the soft
 * polarity and clamped at 0, and Wmax evaluated in float. */
int or_relax_blend_f32(const int *img, const int *g, float alpha, int X, int Y, int Z, int adj,
                       float per, const int *seeds, int nseeds, int *label, int ntimes,
                       float *membership) {
    const int blend = 1;
    const float *per_class = NULL;
    const int max_label = 0;
    RELAX_BODY(float, fabsf, sqrtf)
}

/* ----------------------------------------------------------------- Sobel --- */
/* Scene32::SobelFilter (gft/src/gft_filtering3.cpp:509-552): over the linear addresses
 * i in [1 + X + XY, N - 1 - X - XY) (neighbours by address arithmetic, rows and planes wrap
 * as in the reference), three 3x3 difference stencils with weights 1 2 1 / 2 4 2 / 1 2 1,
 * each >> 4, then ROUND(sqrtf((a^2 + b^2 + c^2) / 3.0)); other voxels 0.  Then the
 * normalisation of exp_gradient_weight.cpp:600-608: g = g * max(I) / max(g) in 64-bit
 * integers when both maxima are positive. */
void or_sobel_normalized(const int *img, int X, int Y, int Z, int *out) {
    static const int n0[9] = {-1, 0, 1, -1, 0, 1, -1, 0, 1};
    static const int n1[9] = {-1, -1, -1, 0, 0, 0, 1, 1, 1};
    static const int we[9] = {1, 2, 1, 2, 4, 2, 1, 2, 1};
    const long long N = (long long)X * Y * Z;
    const long long dx = 1, dy = X, dz = (long long)X * Y, di = dx + dy + dz;
    for (long long i = 0; i < N; i++) out[i] = 0;
    for (long long i = di; i < N - di; i++) {
        int acc[3] = {0, 0, 0};
        for (int m = 0; m < 9; m++)
            acc[0] += we[m] * (img[i + dz + dx * n0[m] + dy * n1[m]] - img[i - dz + dx * n0[m] + dy * n1[m]]);
        for (int m = 0; m < 9; m++)
            acc[1] += we[m] * (img[i + dx + dz * n0[m] + dy * n1[m]] - img[i - dx + dz * n0[m] + dy * n1[m]]);
        for (int m = 0; m < 9; m++)
            acc[2] += we[m] * (img[i + dy + dx * n0[m] + dz * n1[m]] - img[i - dy + dx * n0[m] + dz * n1[m]]);
        acc[0] >>= 4;
        acc[1] >>= 4;
        acc[2] >>= 4;
        float f0 = (float)acc[0], f1 = (float)acc[1], f2 = (float)acc[2];
        float r = sqrtf((f0 * f0 + f1 * f1 + f2 * f2) / 3.0);
        out[i] = (r < 0) ? (int)(r - 0.5) : (int)(r + 0.5);
    }
    int gmax = out[0], wmax = img[0];
    for (long long i = 1; i < N; i++) {
        gmax = MAX(gmax, out[i]);
        wmax = MAX(wmax, img[i]);
    }
    if (gmax > 0 && wmax > 0)
        for (long long i = 0; i < N; i++) out[i] = (int)((long long)out[i] * wmax / gmax);
}

/* ------------------------------------------------------------------- blur --- */
/* Kernel3::SphericalGaussian(scn, 1.0, 10.0, 1.0) + Normalize + Convolution
 * (gft_filtering3.cpp:106-126, 72-83, 321-346, 385-397) with unit voxel spacing. */
void or_gaussian_blur(const int *img, int X, int Y, int Z, int *out) {
    int dx[27], dy[27], dz[27];
    dx[0] = dy[0] = dz[0] = 0;
    int n = 1 + or_adjacency(6, dx + 1, dy + 1, dz + 1);
    float val[27], R = 1.0f, s = 10.0f, f = 1.0f, R2 = R * R;
    for (int i = 0; i < n; i++) {
        float r2 = (float)(dx[i] * dx[i]) + (float)(dy[i] * dy[i]) + (float)(dz[i] * dz[i]);
        val[i] = (float)(s * exp(-f * (r2 / R2)));
    }
    float wt = 0.0f;
    for (int i = 0; i < n; i++) wt += val[i];
    for (int i = 0; i < n; i++) val[i] /= wt;
    for (int z = 0; z < Z; z++)
        for (int y = 0; y < Y; y++)
            for (int x = 0; x < X; x++) {
                float conv = 0.0f;
                for (int i = 0; i < n; i++) {
                    int qx = x + dx[i], qy = y + dy[i], qz = z + dz[i];
                    if (!in_bounds(qx, qy, qz, X, Y, Z)) continue;
                    conv += ((float)img[qx + qy * X + qz * X * Y]) * val[i];
                }
                out[x + y * X + z * X * Y] = (conv < 0) ? (int)(conv - 0.5) : (int)(conv + 0.5);
            }
}

/* ------------------------------------------------------ conditional dilation --- */
/* oiftrelax.cpp:87-169 (get_dilation_border, condition_percentil, dilation_conditional):
 * border = label-0 voxels with a label-1 voxel within Spheric(radius); the border voxels
 * sorted by image value (stable: address order among equal values) up to index
 * (int)(float)((percentile / 100.0) * (n - 1)) become 1.  Returns the voxels relabelled.
 * n == 0 changes nothing (the reference indexes out of range there). */
typedef struct {
    int value, position;
} or_vp;

static int or_vp_cmp(const void *a, const void *b) {
    const or_vp *u = (const or_vp *)a, *v = (const or_vp *)b;
    if (u->value != v->value) return u->value < v->value ? -1 : 1;
    return u->position < v->position ? -1 : (u->position > v->position);
}

long long or_conditional_dilation(const int *img, int *label, int X, int Y, int Z,
                                  float radius, float percentile) {
    const long long N = (long long)X * Y * Z;
    const int r0 = (int)radius, r2 = (int)(radius * radius);
    or_vp *bv = (or_vp *)malloc(sizeof(or_vp) * (size_t)(N > 0 ? N : 1));
    long long n = 0;
    for (long long p = 0; p < N; p++) {
        if (label[p] != 0) continue;
        const int x = (int)(p % X), y = (int)((p / X) % Y), z = (int)(p / ((long long)X * Y));
        int hit = 0;
        for (int dz = -r0; dz <= r0 && !hit; dz++)
            for (int dy = -r0; dy <= r0 && !hit; dy++)
                for (int dx = -r0; dx <= r0 && !hit; dx++) {
                    if (dx * dx + dy * dy + dz * dz > r2) continue;
                    if (!in_bounds(x + dx, y + dy, z + dz, X, Y, Z)) continue;
                    if (label[(x + dx) + (long long)(y + dy) * X + (long long)(z + dz) * X * Y] == 1)
                        hit = 1;
                }
        if (hit) {
            bv[n].value = img[p];
            bv[n].position = (int)p;
            n++;
        }
    }
    long long added = 0;
    if (n > 0) {
        qsort(bv, (size_t)n, sizeof(or_vp), or_vp_cmp);
        const float index_percentile = (float)((percentile / 100.0) * (double)(n - 1));
        const double ipd = (double)index_percentile;
        long long vp = ipd >= 2147483647.0 ? 2147483647LL
                       : ipd <= -2147483648.0 ? -2147483648LL : (long long)(int)index_percentile;
        long long keep = vp + 1;
        if (keep < 0) keep = 0;
        if (keep > n) keep = n;
        for (long long i = 0; i < keep; i++) label[bv[i].position] = 1;
        added = keep;
    }
    free(bv);
    return added;
}

/* oiftrelax.cpp:175-224: face voxels on the stride grid (z, y, x order) whose label is
 * NIL become background seeds.  Returns how many were appended to out (cap entries). */
int or_inject_boundary_seeds(int *label, int X, int Y, int Z, int stride, int *out, int cap) {
    int n = 0;
    for (int z = 0; z < Z; z += stride)
        for (int y = 0; y < Y; y += stride)
            for (int x = 0; x < X; x += stride) {
                if (!(x == 0 || x == X - 1 || y == 0 || y == Y - 1 || z == 0 || z == Z - 1))
                    continue;
                const long long p = x + (long long)y * X + (long long)z * X * Y;
                if (label[p] != -1) continue;
                label[p] = 0;
                if (n < cap) out[n] = (int)p;
                n++;
            }
    return n;
}
