/* CPU oracle of the AprilTag detection path. TEST INFRASTRUCTURE ONLY:
   loaded by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
   leg as the checker of the GPU library; never part of the product.

   Plain scalar C, written for clarity rather than speed, restating the
   algorithm of the reference detector (bouk/apriltags-fast, files under
   fast/). Every function names the reference lines it follows. It must be
   compiled with -ffp-contract=off: the reference's floating point results
   depend on each operation being rounded on its own. */
#include "at_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define AO_MAX_FAMILIES 16

static void *xmalloc(size_t n) {
    void *p = malloc(n ? n : 1);
    if (!p) {
        fprintf(stderr, "oracle: out of memory\n");
        abort();
    }
    return p;
}
static void *xcalloc(size_t n) {
    void *p = calloc(n ? n : 1, 1);
    if (!p) {
        fprintf(stderr, "oracle: out of memory\n");
        abort();
    }
    return p;
}
static int64_t mini(int64_t a, int64_t b) { return a < b ? a : b; }
static int64_t maxi(int64_t a, int64_t b) { return a > b ? a : b; }

/* C's (int) of a double on x86-64 (INT_MIN when out of range or NaN), as
   fast/decode.c:8-11 models it. */
static int64_t c_int(double x) {
    if (x > -2147483649.0 && x < 2147483648.0) return (int64_t)x;
    return -2147483648LL;
}

float ao_atan2f(float y, float x) { return (float)atan2((double)y, (double)x); }
float ao_cosf(float x) { return (float)cos((double)x); }
float ao_sinf(float x) { return (float)sin((double)x); }

void ao_default_params(ao_params *p) {
    /* fast/detector.c:8-20 */
    p->quad_decimate = 2.0f;
    p->quad_sigma = 0.0f;
    p->refine_edges = 1;
    p->decode_sharpening = 0.25;
    p->min_cluster_pixels = 24;
    p->max_nmaxima = 10;
    p->cos_critical_rad = (float)cos(10.0 * M_PI / 180.0);
    p->max_line_fit_mse = 10.0f;
    p->min_white_black_diff = 5;
    p->deglitch = 0;
}

/* =====================================================================
   1. Decimation (fast/image.c:6-88). */

static void quad_size(int64_t w, int64_t h, float f, int64_t *qw, int64_t *qh) {
    if (f == 1.5f) {
        *qw = w / 3 * 2;
        *qh = h / 3 * 2;
        return;
    }
    int64_t k = (int64_t)f;
    if (k == 2) {
        *qw = w / 2;
        *qh = h / 2;
        return;
    }
    *qw = 1 + (w - 1) / k;
    *qh = 1 + (h - 1) / k;
}

/* Factor 2 is a 2x2 box filter. The columns below the largest multiple
   of 32 of the output width round twice, ((a+c+1)>>1 + (b+d+1)>>1 + 1)>>1,
   as the C library's AVX2 path; the others take the exact (sum+2)>>2
   (fast/image.c:26-46). 1.5 uses 3x3 weights over 9 (:50-62); other
   factors take every k-th pixel (:67-88). */
static void decimate(const uint8_t *src, int64_t stride, float f, uint8_t *out, int64_t qw, int64_t qh) {
    if (f == 1.5f) {
        for (int64_t oy = 0; oy < qh; oy += 2) {
            const uint8_t *r0 = src + (oy / 2) * 3 * stride, *r1 = r0 + stride, *r2 = r1 + stride;
            uint8_t *o0 = out + oy * qw, *o1 = o0 + qw;
            for (int64_t k = 0; k < qw / 2; k++) {
                int64_t x = 3 * k;
                int a = r0[x], b = r0[x + 1], c = r0[x + 2];
                int d = r1[x], e = r1[x + 1], g = r1[x + 2];
                int p = r2[x], q = r2[x + 1], r = r2[x + 2];
                o0[2 * k] = (uint8_t)((4 * a + 2 * b + 2 * d + e) / 9);
                o0[2 * k + 1] = (uint8_t)((4 * c + 2 * b + 2 * g + e) / 9);
                o1[2 * k] = (uint8_t)((4 * p + 2 * d + 2 * q + e) / 9);
                o1[2 * k + 1] = (uint8_t)((4 * r + 2 * g + 2 * q + e) / 9);
            }
        }
        return;
    }
    int64_t k = (int64_t)f;
    if (k == 2) {
        int64_t split = qw - qw % 32;
        for (int64_t oy = 0; oy < qh; oy++) {
            const uint8_t *r0 = src + 2 * oy * stride, *r1 = r0 + stride;
            uint8_t *o = out + oy * qw;
            for (int64_t x = 0; x < qw; x++) {
                int a = r0[2 * x], b = r0[2 * x + 1], c = r1[2 * x], d = r1[2 * x + 1];
                if (x < split)
                    o[x] = (uint8_t)((((a + c + 1) >> 1) + ((b + d + 1) >> 1) + 1) >> 1);
                else
                    o[x] = (uint8_t)((a + b + c + d + 2) >> 2);
            }
        }
        return;
    }
    for (int64_t oy = 0; oy < qh; oy++)
        for (int64_t x = 0; x < qw; x++) out[oy * qw + x] = src[oy * k * stride + x * k];
}

/* =====================================================================
   2. Blur or sharpen (fast/image.c:93-173). */

static int64_t blur_taps(float sigma) {
    if (sigma == 0.0f) return 0;
    int64_t n = (int64_t)(4.0f * fabsf(sigma));
    if ((n & 1) == 0) n++;
    return n;
}

/* One line. The wide variant (images of 65536 pixels or more) filters one
   more output pixel than the narrow one (fast/image.c:93-107). */
static void convolve_line(const uint8_t *x, uint8_t *y, int64_t n, const uint8_t *k, int64_t nk, bool wide) {
    int64_t r = nk / 2;
    for (int64_t i = 0; i < r && i < n; i++) y[i] = x[i];
    int64_t m = wide ? n - nk + 1 : n - nk;
    for (int64_t i = 0; i < m; i++) {
        uint32_t acc = 0;
        for (int64_t j = 0; j < nk; j++) acc += (uint32_t)k[j] * x[i + j];
        y[r + i] = (uint8_t)(acc >> 8);
    }
    int64_t tail = wide ? n - r : n - nk + r;
    for (int64_t i = maxi(tail, 0); i < n; i++) y[i] = x[i];
}

static bool blur_or_sharpen(uint8_t *im, int64_t w, int64_t h, float qsigma) {
    int64_t nk = blur_taps(qsigma);
    if (nk <= 1) return false;
    double sigma = fabsf(qsigma);
    double *dk = xmalloc(sizeof(double) * nk);
    for (int64_t i = 0; i < nk; i++) {
        double t = (double)(i - nk / 2) / sigma;
        dk[i] = exp(-0.5 * (t * t));
    }
    double sum = 0.0;
    for (int64_t i = 0; i < nk; i++) sum += dk[i];
    uint8_t *k = xmalloc(nk);
    for (int64_t i = 0; i < nk; i++) k[i] = (uint8_t)(dk[i] / sum * 255.0);
    free(dk);
    uint8_t *orig = NULL;
    if (qsigma < 0.0f) {
        orig = xmalloc(w * h);
        memcpy(orig, im, w * h);
    }
    bool wide = w * h >= 65536;
    uint8_t *a = xmalloc(maxi(w, h)), *b = xmalloc(maxi(w, h));
    for (int64_t y = 0; y < h; y++) {
        memcpy(a, im + y * w, w);
        convolve_line(a, im + y * w, w, k, nk, wide);
    }
    for (int64_t x = 0; x < w; x++) {
        for (int64_t y = 0; y < h; y++) a[y] = im[y * w + x];
        convolve_line(a, b, h, k, nk, wide);
        for (int64_t y = 0; y < h; y++) im[y * w + x] = b[y];
    }
    if (orig) {
        for (int64_t i = 0; i < w * h; i++) {
            int v = 2 * (int)orig[i] - im[i];
            im[i] = (uint8_t)(v < 0 ? 0 : v > 255 ? 255 : v);
        }
        free(orig);
    }
    free(a);
    free(b);
    free(k);
    return true;
}

/* =====================================================================
   3. Adaptive threshold (fast/threshold.c:15-161) and deglitch
   (:173-193). 4x4 tiles; each tile's min and max, then the max and min
   over its 3x3 tile neighbourhood (cells outside the grid left out);
   threshold lo + (hi-lo)/2, and 127 where hi-lo < diff. Pixels right of
   the last whole tile column use that column and are never 127; pixels
   below the last whole tile row use that row and are never 127. */

static void threshold(const uint8_t *im, int64_t w, int64_t h, int32_t diff, uint8_t *out) {
    int64_t tw = w / 4, th = h / 4;
    uint8_t *mx = xmalloc(tw * th), *mn = xmalloc(tw * th);
    uint8_t *mx3 = xmalloc(tw * th), *mn3 = xmalloc(tw * th);
    for (int64_t ty = 0; ty < th; ty++)
        for (int64_t tx = 0; tx < tw; tx++) {
            uint8_t hi = 0, lo = 255;
            for (int dy = 0; dy < 4; dy++)
                for (int dx = 0; dx < 4; dx++) {
                    uint8_t v = im[(4 * ty + dy) * w + 4 * tx + dx];
                    if (v > hi) hi = v;
                    if (v < lo) lo = v;
                }
            mx[ty * tw + tx] = hi;
            mn[ty * tw + tx] = lo;
        }
    for (int64_t ty = 0; ty < th; ty++)
        for (int64_t tx = 0; tx < tw; tx++) {
            uint8_t hi = 0, lo = 255;
            for (int64_t y = maxi(ty - 1, 0); y <= mini(ty + 1, th - 1); y++)
                for (int64_t x = maxi(tx - 1, 0); x <= mini(tx + 1, tw - 1); x++) {
                    if (mx[y * tw + x] > hi) hi = mx[y * tw + x];
                    if (mn[y * tw + x] < lo) lo = mn[y * tw + x];
                }
            mx3[ty * tw + tx] = hi;
            mn3[ty * tw + tx] = lo;
        }
    for (int64_t y = 0; y < h; y++)
        for (int64_t x = 0; x < w; x++) {
            int64_t ty = y / 4, tx = x / 4;
            bool may_flat = true;
            if (ty >= th) {
                ty = th - 1;
                may_flat = false;
            }
            if (tx >= tw) {
                tx = tw - 1;
                may_flat = false;
            }
            int hi = mx3[ty * tw + tx], lo = mn3[ty * tw + tx];
            uint8_t t = (uint8_t)(lo + (hi - lo) / 2);
            uint8_t v = im[y * w + x] > t ? 255 : 0;
            out[y * w + x] = may_flat && hi - lo < diff ? 127 : v;
        }
    free(mx);
    free(mn);
    free(mx3);
    free(mn3);
}

static void deglitch(uint8_t *t, int64_t w, int64_t h) {
    uint8_t *tmp = xcalloc(w * h);
    for (int64_t y = 1; y < h - 1; y++)
        for (int64_t x = 1; x < w - 1; x++) {
            uint8_t m = 0;
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++)
                    if (t[(y + dy) * w + x + dx] > m) m = t[(y + dy) * w + x + dx];
            tmp[y * w + x] = m;
        }
    for (int64_t y = 1; y < h - 1; y++)
        for (int64_t x = 1; x < w - 1; x++) {
            uint8_t m = 255;
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++)
                    if (tmp[(y + dy) * w + x + dx] < m) m = tmp[(y + dy) * w + x + dx];
            t[y * w + x] = m;
        }
    free(tmp);
}

/* =====================================================================
   4. Runs (fast/threshold.c:210-283): maximal runs of equal value over
   columns 0..w-2 of each row; runs of 127 are not kept. */

static int64_t row_runs(const uint8_t *row, int64_t w, uint16_t *s, uint16_t *e, uint8_t *v) {
    int64_t xmax = w - 2, n = 0, start = 0;
    uint8_t cur = row[0];
    for (int64_t x = 1; x <= xmax; x++) {
        if (row[x] == row[x - 1]) continue;
        if (cur != 127) {
            s[n] = (uint16_t)start;
            e[n] = (uint16_t)(x - 1);
            v[n] = cur;
            n++;
        }
        start = x;
        cur = row[x];
    }
    if (cur != 127) {
        s[n] = (uint16_t)start;
        e[n] = (uint16_t)xmax;
        v[n] = cur;
        n++;
    }
    return n;
}

/* =====================================================================
   5. Connected components over runs (fast/unionfind.c:13-298).

   Nodes: the runs in row-major order, then one node per row for pixel
   (w-1, y), which no run covers. Two runs of rows y-1 and y join when
   they have the same value and: they share a column x >= 1; or, for white
   (255), one is diagonal to the other at columns >= 1. The last run of
   row y, when white and ending at w-2, joins the node of pixel (w-1, y-1)
   if that pixel is white and (w-2, y-1) is not (unionfind.c:89-97).

   The reference's sequential pass: rows in order, the runs of a row in
   order, the candidate runs above in order (unionfind.c:112-146), then
   the last-column link. Union by size (pixels - 1 at a root; ties link
   the current row's tree under the other), so the root it picks depends
   on this exact sequence. */

typedef struct {
    uint32_t parent, size;
} ufnode;

static uint32_t uf_root(ufnode *u, uint32_t a) {
    while (u[a].parent != a) {
        uint32_t p = u[a].parent;
        u[a].parent = u[p].parent; /* path halving: roots unchanged */
        a = p;
    }
    return a;
}

/* a: node of the current row (or its tree), b: node above. */
static void uf_link(ufnode *u, uint32_t a, uint32_t b) {
    uint32_t ra = uf_root(u, a), rb = uf_root(u, b);
    if (ra == rb) return;
    uint32_t sa = u[ra].size + 1, sb = u[rb].size + 1;
    if (sa > sb) {
        u[rb].parent = ra;
        u[ra].size += sb;
    } else {
        u[ra].parent = rb;
        u[rb].size += sa;
    }
}

static bool runs_touch(int64_t a0, int64_t a1, int64_t b0, int64_t b1, uint8_t v) {
    if (maxi(maxi(a0, b0), 1) <= mini(a1, b1)) return true;
    if (v != 255) return false;
    if (maxi(maxi(a0, b0 + 1), 1) <= mini(a1, b1 + 1)) return true;
    return maxi(maxi(a0, b0 - 1), 1) <= mini(a1, b1 - 1);
}

static void components(const ao_result *r, const uint8_t *t, int64_t w, int64_t h, ufnode *u) {
    int64_t nruns = r->nruns;
    for (int64_t i = 0; i < nruns; i++) {
        u[i].parent = (uint32_t)i;
        u[i].size = (uint32_t)(r->run_end[i] - r->run_start[i]);
    }
    for (int64_t y = 0; y < h; y++) u[nruns + y] = (ufnode){(uint32_t)(nruns + y), 0};
    for (int64_t y = 1; y < h; y++) {
        int64_t p0 = r->row_off[y - 1], p1 = r->row_off[y], c1 = r->row_off[y + 1];
        int64_t j = p0;
        for (int64_t i = p1; i < c1; i++) {
            int64_t a0 = r->run_start[i], a1 = r->run_end[i];
            uint8_t v = r->run_v[i];
            while (j < p1 && (int64_t)r->run_end[j] + 1 < a0) j++;
            for (int64_t k = j; k < p1 && r->run_start[k] <= a1 + 1; k++) {
                if (r->run_v[k] != v) continue;
                if (runs_touch(a0, a1, r->run_start[k], r->run_end[k], v)) uf_link(u, (uint32_t)i, (uint32_t)k);
            }
        }
        if (c1 > p1) {
            int64_t last = c1 - 1;
            const uint8_t *above = t + (y - 1) * w;
            if (r->run_end[last] == w - 2 && r->run_v[last] == 255 && above[w - 1] == 255 && above[w - 2] != 255)
                uf_link(u, (uint32_t)last, (uint32_t)(nruns + y - 1));
        }
    }
}

/* =====================================================================
   6. Boundary points (fast/clusters.c:144-308).

   For pixel (x, y), x in 1..w-2 and y in 1..h-2, its neighbours (1,0),
   (0,1), (-1,1), (1,1) in that order: a point where one pixel is 0 and
   the other 255 and both components have at least min_cluster_pixels
   pixels. The (-1,1) point is left out when the pixel to the left gave a
   (1,1) point, except at x = 1. Pixel x = 0 gives only its (1,0) point.
   Points are at doubled coordinates (2x+dx, 2y+dy) with gradient
   (dx, dy) * (255 - 2 v), v the pixel's value. The cluster of a point is
   the unordered pair of the two components' labels. */

typedef struct {
    uint64_t pt;  /* x | y<<16 | gx<<32 | gy<<48 */
    uint64_t cid; /* (larger label << 32) + smaller label */
    uint64_t okey; /* cluster order key */
    uint64_t seq; /* emission index */
} emitted;

static int cmp_emitted(const void *pa, const void *pb) {
    const emitted *a = pa, *b = pb;
    if (a->okey != b->okey) return a->okey < b->okey ? -1 : 1;
    if (a->cid != b->cid) return a->cid < b->cid ? -1 : 1;
    return a->seq < b->seq ? -1 : a->seq > b->seq;
}

static int opp(uint8_t a, uint8_t b) { return (a ^ b) == 255; }

/* Per-pixel labels and size flags of one row; pixels of no run get flag 0
   and the last column the row's virtual node. */
static void label_row(const ao_result *r, const uint32_t *nlab, const uint8_t *nok, int64_t y, int64_t w,
                      uint32_t *lab, uint8_t *ok) {
    memset(ok, 0, w);
    memset(lab, 0, w * sizeof *lab);
    for (int64_t i = r->row_off[y]; i < (int64_t)r->row_off[y + 1]; i++)
        for (int64_t x = r->run_start[i]; x <= r->run_end[i]; x++) {
            lab[x] = nlab[i];
            ok[x] = nok[i];
        }
    lab[w - 1] = nlab[r->nruns + y];
    ok[w - 1] = nok[r->nruns + y];
}

static int64_t cluster_buckets(int64_t w, int64_t h) {
    /* cluster_map_size (fast/clusters.c:97-103) for one thread */
    int64_t chunk = 1 + (h - 1) / 6;
    int64_t n = 1024;
    while (n < chunk * w / 64 && n < 65536) n <<= 1;
    return n;
}

static emitted *boundary_points(const ao_result *r, const uint8_t *t, int64_t w, int64_t h, const uint32_t *nlab,
                                const uint8_t *nok, int32_t order_mode, int64_t *np_out) {
    int64_t cap = 1024, np = 0;
    emitted *out = xmalloc(cap * sizeof *out);
    uint32_t *la = xmalloc(w * 4), *lb = xmalloc(w * 4);
    uint8_t *oa = xmalloc(w), *ob = xmalloc(w);
    uint64_t bmask = (uint64_t)cluster_buckets(w, h) - 1;
    static const int ddx[4] = {1, 0, -1, 1}, ddy[4] = {0, 1, 1, 1};
    for (int64_t y = 1; y + 1 < h; y++) {
        const uint8_t *a = t + y * w, *b = a + w;
        label_row(r, nlab, nok, y, w, la, oa);
        label_row(r, nlab, nok, y + 1, w, lb, ob);
        for (int64_t x = 0; x + 1 < w; x++) {
            int m = 0;
            if (x == 0) {
                m = opp(a[0], a[1]) && oa[0] && oa[1];
            } else {
                uint8_t v = a[x];
                int c10 = opp(v, a[x + 1]) && oa[x + 1];
                int c01 = opp(v, b[x]) && ob[x];
                int cm1 = opp(v, b[x - 1]) && ob[x - 1];
                int c11 = opp(v, b[x + 1]) && ob[x + 1];
                int left11 = opp(a[x - 1], b[x]) && oa[x - 1] && ob[x];
                if (x == 1) left11 = 0;
                m = oa[x] ? (c10 | c01 << 1 | (cm1 && !left11) << 2 | c11 << 3) : 0;
            }
            for (int j = 0; j < 4; j++) {
                if (!(m >> j & 1)) continue;
                int64_t nx = x + ddx[j];
                uint32_t l0 = la[x], l1 = ddy[j] ? lb[nx] : la[nx];
                int g = a[x] == 0 ? 255 : -255;
                uint64_t px = (uint64_t)(2 * x + ddx[j]), py = (uint64_t)(2 * y + ddy[j]);
                uint64_t gx = (uint16_t)(int16_t)(ddx[j] * g), gy = (uint16_t)(int16_t)(ddy[j] * g);
                if (np == cap) {
                    cap *= 2;
                    out = realloc(out, cap * sizeof *out);
                    if (!out) abort();
                }
                emitted *e = &out[np];
                e->pt = px | py << 16 | gx << 32 | gy << 48;
                e->cid = l0 < l1 ? ((uint64_t)l1 << 32) + l0 : ((uint64_t)l0 << 32) + l1;
                /* the reference orders clusters by hash bucket, then id
                   (fast/clusters.c:44, 338-356) */
                e->okey = order_mode == AO_ORDER_REF ? ((e->cid * 2654435761u) >> 32) & bmask : 0;
                e->seq = (uint64_t)np;
                np++;
            }
        }
    }
    free(la);
    free(lb);
    free(oa);
    free(ob);
    *np_out = np;
    return out;
}

/* =====================================================================
   7. Quad fitting (fast/quads.c). */

/* The angle sort (fast/quads.c:48-208): a recursive merge sort whose
   leaves (at most 5 keys) are put in order by fixed compare-exchange
   networks that look at the upper 32 bits only (so keys with equal
   angles can stay out of order there), and whose merges compare whole
   keys. While half of a range has more than 5 keys it is cut in four
   (halves of halves), else in two. The networks are the reference's
   (they decide the order of equal angles). */
static void leaf_network(uint64_t *k, int64_t n) {
    static const int8_t net2[] = {0, 1};
    static const int8_t net3[] = {0, 1, 1, 2, 0, 1};
    static const int8_t net4[] = {0, 1, 2, 3, 0, 2, 1, 3, 1, 2};
    static const int8_t net5[] = {0, 1, 3, 4, 1, 2, 0, 1, 0, 3, 2, 4, 1, 2, 2, 3, 1, 2};
    const int8_t *net = NULL;
    int len = 0;
    if (n == 2) net = net2, len = 1;
    if (n == 3) net = net3, len = 3;
    if (n == 4) net = net4, len = 5;
    if (n == 5) net = net5, len = 9;
    for (int i = 0; i < len; i++) {
        int a = net[2 * i], b = net[2 * i + 1];
        if ((k[a] >> 32) > (k[b] >> 32)) {
            uint64_t t = k[a];
            k[a] = k[b];
            k[b] = t;
        }
    }
}

static void merge_keys(const uint64_t *a, int64_t na, const uint64_t *b, int64_t nb, uint64_t *out) {
    int64_t i = 0, j = 0, o = 0;
    while (i < na && j < nb) out[o++] = a[i] < b[j] ? a[i++] : b[j++];
    while (i < na) out[o++] = a[i++];
    while (j < nb) out[o++] = b[j++];
}

static void sort_halves(uint64_t *k, uint64_t *tmp, int64_t n) {
    if (n <= 5) {
        leaf_network(k, n);
        return;
    }
    int64_t h = n / 2;
    sort_halves(k, tmp, h);
    sort_halves(k + h, tmp + h, n - h);
    merge_keys(k, h, k + h, n - h, tmp);
    memcpy(k, tmp, n * 8);
}

static void sort_quarters(uint64_t *k, uint64_t *tmp, int64_t n) {
    if (n <= 5) {
        leaf_network(k, n);
        return;
    }
    int64_t half = n / 2;
    if (half <= 5) {
        sort_halves(k, tmp, n);
        return;
    }
    int64_t q1 = half / 2, q3 = half + (n - half) / 2;
    sort_quarters(k, tmp, q1);
    sort_quarters(k + q1, tmp + q1, half - q1);
    sort_quarters(k + half, tmp + half, q3 - half);
    sort_quarters(k + q3, tmp + q3, n - q3);
    merge_keys(k, q1, k + q1, half - q1, tmp);
    merge_keys(k + half, q3 - half, k + q3, n - q3, tmp + half);
    merge_keys(tmp, half, tmp + half, n - half, k);
}

void ao_keysort(uint64_t *keys, int64_t n) {
    if (n < 2) return;
    uint64_t *tmp = xmalloc(n * 8);
    sort_quarters(keys, tmp, n);
    free(tmp);
}

static uint32_t f32_bits(float f) {
    uint32_t b;
    memcpy(&b, &f, 4);
    return b;
}
static float bits_f32(uint32_t b) {
    float f;
    memcpy(&f, &b, 4);
    return f;
}

/* The angle key of a point (fast/quads.c:429-453): a pseudo-angle
   quadrant + slope in f32, its order-preserving bits above the
   complemented index. */
static uint64_t angle_key(float dx, float dy, uint32_t idx) {
    float quadrant;
    if (dy > 0.0f)
        quadrant = dx > 0.0f ? 65536.0f : 131072.0f;
    else
        quadrant = dx > 0.0f ? 0.0f : -65536.0f;
    float fx = dx, fy = dy;
    if (dy < 0.0f) {
        fx = bits_f32(f32_bits(dx) ^ 0x80000000u);
        fy = bits_f32(f32_bits(dy) ^ 0x80000000u);
    }
    float ndx = fx, ndy = fy;
    if (fx < 0.0f) {
        ndx = fy;
        ndy = -fx;
    }
    float slope = quadrant + ndy / ndx;
    uint32_t b = f32_bits(slope);
    uint32_t s = (uint32_t)((int32_t)b >> 31);
    uint32_t ord = b ^ (s | 0x80000000u);
    return (uint64_t)ord << 32 | (uint32_t)~idx;
}

typedef struct {
    double *mx, *my, *mxx, *mxy, *myy, *mw;
} moments;

/* Moments of points i0..i1 of the sorted cluster, wrapping past the end
   (fast/quads.c:539-569, 658-700, 885-921 sum them in these forms). */
typedef struct {
    double x, y, xx, xy, yy, w;
} msum;

static msum seg_moments(const moments *a, int64_t sz, int64_t i0, int64_t i1) {
    msum s;
    if (i0 <= i1) {
        s.x = a->mx[i1];
        s.y = a->my[i1];
        s.xx = a->mxx[i1];
        s.xy = a->mxy[i1];
        s.yy = a->myy[i1];
        s.w = a->mw[i1];
        if (i0 > 0) {
            s.x -= a->mx[i0 - 1];
            s.y -= a->my[i0 - 1];
            s.xx -= a->mxx[i0 - 1];
            s.xy -= a->mxy[i0 - 1];
            s.yy -= a->myy[i0 - 1];
            s.w -= a->mw[i0 - 1];
        }
    } else {
        s.x = (a->mx[sz - 1] - a->mx[i0 - 1]) + a->mx[i1];
        s.y = (a->my[sz - 1] - a->my[i0 - 1]) + a->my[i1];
        s.xx = (a->mxx[sz - 1] - a->mxx[i0 - 1]) + a->mxx[i1];
        s.xy = (a->mxy[sz - 1] - a->mxy[i0 - 1]) + a->mxy[i1];
        s.yy = (a->myy[sz - 1] - a->myy[i0 - 1]) + a->myy[i1];
        s.w = (a->mw[sz - 1] - a->mw[i0 - 1]) + a->mw[i1];
    }
    return s;
}

/* The error of a window of nn points (fast/quads.c:604-653). */
static double window_error(msum s, double nn) {
    double ex = s.x / s.w, ey = s.y / s.w;
    double cxx = s.xx / s.w - ex * ex;
    double cxy = s.xy / s.w - ex * ey;
    double cyy = s.yy / s.w - ey * ey;
    double d = cxx - cyy;
    double root = (double)sqrtf((float)(d * d + 4.0 * (cxy * cxy)));
    return nn * (0.5 * (cxx + cyy - root));
}

/* The line through the moments: the centroid, the unit normal and the
   smaller eigenvalue (fast/quads.c:570-600, 756-783). */
static void line_of(msum s, double lp[4], double *mse) {
    double ex = s.x / s.w, ey = s.y / s.w;
    double cxx = s.xx / s.w - ex * ex;
    double cxy = s.xy / s.w - ex * ey;
    double cyy = s.yy / s.w - ey * ey;
    double root = (double)sqrtf((float)((cxx - cyy) * (cxx - cyy) + 4.0 * cxy * cxy));
    double eig_small = 0.5 * (cxx + cyy - root);
    double eig = 0.5 * (cxx + cyy + root);
    double nx1 = cxx - eig, ny1 = cxy, m1 = nx1 * nx1 + ny1 * ny1;
    double nx2 = cxy, ny2 = cyy - eig, m2 = nx2 * nx2 + ny2 * ny2;
    double nx = nx2, ny = ny2, m = m2;
    if (m1 > m2) {
        nx = nx1;
        ny = ny1;
        m = m1;
    }
    double len = (double)sqrtf((float)m);
    lp[0] = ex;
    lp[1] = ey;
    lp[2] = 0.0;
    lp[3] = 0.0;
    if (!(fabs(len) < 1e-12)) {
        lp[2] = nx / len;
        lp[3] = ny / len;
    }
    *mse = eig_small;
}

static int cmp_desc(const void *pa, const void *pb) {
    double a = *(const double *)pa, b = *(const double *)pb;
    return a > b ? -1 : a < b;
}

typedef struct {
    int32_t min_px, max_nmaxima;
    double max_dot, max_mse;
    double qsm[7];
    int64_t tag_width;
    bool normal_border, reversed_border;
} fitcfg;

/* Corner search (fast/quads.c:788-959): window errors over 2*ksz+1
   points, a 7-tap low-pass (wrapping), local maxima (wrapping), the
   max_nmaxima largest kept when there are more, line fits between pairs
   of maxima, and the 4 maxima with the smallest total error. */
static bool segment_corners(const fitcfg *cfg, const moments *a, int64_t sz, int64_t idx[4]) {
    int64_t ksz = mini(20, sz / 12);
    if (ksz < 2) return false;
    double nn = (double)(2 * ksz + 1);
    double *errs = xmalloc(sz * 8), *filt = xmalloc(sz * 8);
    for (int64_t i = 0; i < sz; i++) {
        int64_t i0 = i - ksz, i1 = i + ksz;
        msum s;
        if (i0 >= 1 && i1 < sz) {
            /* middle windows (window_errors) */
            s.x = a->mx[i1] - a->mx[i0 - 1];
            s.y = a->my[i1] - a->my[i0 - 1];
            s.xx = a->mxx[i1] - a->mxx[i0 - 1];
            s.xy = a->mxy[i1] - a->mxy[i0 - 1];
            s.yy = a->myy[i1] - a->myy[i0 - 1];
            s.w = a->mw[i1] - a->mw[i0 - 1];
        } else if (i0 < 0) {
            s = seg_moments(a, sz, i0 + sz, i1);
        } else if (i0 == 0) {
            s = seg_moments(a, sz, 0, i1);
        } else {
            s = seg_moments(a, sz, i0, i1 - sz);
        }
        errs[i] = window_error(s, nn);
    }
    /* the low-pass: the middle outputs start from the first product, the
       six wrapping ones from 0.0 (fast/quads.c:706-735) */
    for (int64_t i = 0; i < sz; i++) {
        if (i >= 3 && i < sz - 3) {
            double acc = errs[i - 3] * cfg->qsm[0];
            for (int t = 1; t < 7; t++) acc += errs[i - 3 + t] * cfg->qsm[t];
            filt[i] = acc;
        } else {
            double acc = 0.0;
            for (int t = 0; t < 7; t++) {
                int64_t j = i - 3 + t;
                if (j < 0) j += sz;
                if (j >= sz) j -= sz;
                acc += errs[j] * cfg->qsm[t];
            }
            filt[i] = acc;
        }
    }
    int64_t *mxi = xmalloc(sz * 8);
    double *mxe = xmalloc(sz * 8);
    int64_t nm = 0;
    for (int64_t i = 0; i < sz; i++) {
        double e = filt[i], l = filt[(i + sz - 1) % sz], r = filt[(i + 1) % sz];
        if (e > l && e > r) {
            mxi[nm] = i;
            mxe[nm] = e;
            nm++;
        }
    }
    bool ok = false;
    if (nm < 4) goto done;
    if (nm > cfg->max_nmaxima) {
        double *sel = xmalloc(nm * 8);
        memcpy(sel, mxe, nm * 8);
        qsort(sel, nm, 8, cmp_desc);
        double thresh = sel[cfg->max_nmaxima];
        free(sel);
        int64_t o = 0;
        for (int64_t i = 0; i < nm; i++)
            if (mxe[i] > thresh) mxi[o++] = mxi[i];
        nm = o;
    }
    {
        double *perr = xmalloc(nm * nm * 8), *pmse = xmalloc(nm * nm * 8), *pnx = xmalloc(nm * nm * 8),
               *pny = xmalloc(nm * nm * 8);
        for (int64_t m0 = 0; m0 < nm; m0++)
            for (int64_t m1 = m0 + 1; m1 < nm; m1++) {
                for (int pass = 0; pass < 2; pass++) {
                    int64_t p, q;
                    if (pass == 0) {
                        p = m0;
                        q = m1;
                    } else {
                        if (m1 < m0 + 3) break;
                        p = m1;
                        q = m0;
                    }
                    int64_t i0 = mxi[p], i1 = mxi[q];
                    msum s = seg_moments(a, sz, i0, i1);
                    double n = (double)(i0 <= i1 ? i1 - i0 + 1 : sz - i0 + i1 + 1);
                    double lp[4], mse;
                    line_of(s, lp, &mse);
                    perr[p * nm + q] = n * mse;
                    pmse[p * nm + q] = mse;
                    pnx[p * nm + q] = lp[2];
                    pny[p * nm + q] = lp[3];
                }
            }
        double best = INFINITY;
        int64_t bi[4] = {0, 0, 0, 0};
        for (int64_t m0 = 0; m0 < nm - 3; m0++)
            for (int64_t m1 = m0 + 1; m1 < nm - 2; m1++) {
                int64_t p01 = m0 * nm + m1;
                if (pmse[p01] > cfg->max_mse) continue;
                for (int64_t m2 = m1 + 1; m2 < nm - 1; m2++) {
                    int64_t p12 = m1 * nm + m2;
                    if (pmse[p12] > cfg->max_mse) continue;
                    double dot = pnx[p01] * pnx[p12] + pny[p01] * pny[p12];
                    if (fabs(dot) > cfg->max_dot) continue;
                    double e012 = perr[p01] + perr[p12];
                    for (int64_t m3 = m2 + 1; m3 < nm; m3++) {
                        int64_t p23 = m2 * nm + m3, p30 = m3 * nm + m0;
                        double e23 = pmse[p23] > cfg->max_mse ? INFINITY : perr[p23];
                        double e30 = pmse[p30] > cfg->max_mse ? INFINITY : perr[p30];
                        double err = e012 + e23 + e30;
                        if (err < best) {
                            best = err;
                            bi[0] = mxi[m0];
                            bi[1] = mxi[m1];
                            bi[2] = mxi[m2];
                            bi[3] = mxi[m3];
                        }
                    }
                }
            }
        free(perr);
        free(pmse);
        free(pnx);
        free(pny);
        if (best == INFINITY) goto done;
        memcpy(idx, bi, sizeof bi);
        ok = best / (double)sz < cfg->max_mse;
    }
done:
    free(errs);
    free(filt);
    free(mxi);
    free(mxe);
    return ok;
}

static double sqd(double x) { return x * x; }

/* Fit one quad (fast/quads.c:1044-1141). pts: the cluster in emission
   order; im: the quad image. */
static bool fit_quad(const fitcfg *cfg, const uint64_t *pts, int64_t sz, const uint8_t *im, int64_t iw, int64_t ih,
                     ao_quad *q) {
    int64_t xmin = 0xffff, xmax = 0, ymin = 0xffff, ymax = 0;
    for (int64_t i = 0; i < sz; i++) {
        int64_t x = pts[i] & 0xffff, y = pts[i] >> 16 & 0xffff;
        xmin = mini(xmin, x);
        xmax = maxi(xmax, x);
        ymin = mini(ymin, y);
        ymax = maxi(ymax, y);
    }
    if ((xmax - xmin) * (ymax - ymin) < cfg->tag_width) return false;
    float cx = (float)((double)(xmin + xmax) * 0.5 + 0.05118);
    float cy = (float)((double)(ymin + ymax) * 0.5 + -0.028581);
    uint64_t *keys = xmalloc(sz * 8);
    float lanes[8] = {0};
    int64_t nv = sz - sz % 8;
    float dot = 0.0f;
    for (int64_t i = 0; i < sz; i++) {
        float x = (float)(pts[i] & 0xffff), y = (float)(pts[i] >> 16 & 0xffff);
        float gx = (float)(int16_t)(pts[i] >> 32 & 0xffff), gy = (float)(int16_t)(pts[i] >> 48);
        float dx = x - cx, dy = y - cy;
        keys[i] = angle_key(dx, dy, (uint32_t)i);
        /* 8 lanes (i mod 8) for the whole groups of 8, summed pairwise,
           then the rest in order (fast/quads.c:473-511) */
        if (i < nv) {
            lanes[i % 8] = lanes[i % 8] + (dx * gx + dy * gy);
        } else {
            if (i == nv)
                dot = ((lanes[0] + lanes[4]) + (lanes[2] + lanes[6])) + ((lanes[1] + lanes[5]) + (lanes[3] + lanes[7]));
            dot += dx * gx + dy * gy;
        }
    }
    if (nv == sz) dot = ((lanes[0] + lanes[4]) + (lanes[2] + lanes[6])) + ((lanes[1] + lanes[5]) + (lanes[3] + lanes[7]));
    q->reversed_border = dot < 0.0f;
    bool ok = false;
    double *buf = NULL;
    if (!cfg->reversed_border && q->reversed_border) goto out;
    if (!cfg->normal_border && !q->reversed_border) goto out;
    ao_keysort(keys, sz);
    /* cumulative weighted moments in angle order (fast/quads.c:968-1035):
       weight sqrt(gx^2 + gy^2) + 1 from the quad image at the point's
       pixel, 1 where a neighbour is off the image */
    buf = xmalloc(6 * sz * 8);
    moments m = {buf, buf + sz, buf + 2 * sz, buf + 3 * sz, buf + 4 * sz, buf + 5 * sz};
    double smx = 0, smy = 0, smxx = 0, smxy = 0, smyy = 0, sw = 0;
    for (int64_t k = 0; k < sz; k++) {
        uint32_t src = ~(uint32_t)keys[k];
        int32_t px = (int32_t)(pts[src] & 0xffff), py = (int32_t)(pts[src] >> 16 & 0xffff);
        int32_t ix = (px >> 1) + (px & 1), iy = (py >> 1) + (py & 1);
        int32_t g2 = 0;
        if (ix > 0 && ix + 1 < iw && iy > 0 && iy + 1 < ih) {
            int64_t c = (int64_t)iy * iw + ix;
            int32_t gx = (int32_t)im[c + 1] - im[c - 1];
            int32_t gy = (int32_t)im[c + iw] - im[c - iw];
            g2 = gx * gx + gy * gy;
        }
        double w = sqrt((double)g2) + 1.0;
        double fx = (double)px * 0.5 + 0.5, fy = (double)py * 0.5 + 0.5;
        smx += w * fx;
        smy += w * fy;
        smxx += w * fx * fx;
        smxy += w * fx * fy;
        smyy += w * fy * fy;
        sw += w;
        m.mx[k] = smx;
        m.my[k] = smy;
        m.mxx[k] = smxx;
        m.mxy[k] = smxy;
        m.myy[k] = smyy;
        m.mw[k] = sw;
    }
    int64_t idx[4];
    if (!segment_corners(cfg, &m, sz, idx)) goto out;
    double lines[4][4];
    for (int i = 0; i < 4; i++) {
        double mse;
        line_of(seg_moments(&m, sz, idx[i], idx[(i + 1) & 3]), lines[i], &mse);
        if (mse > cfg->max_mse) goto out;
    }
    for (int i = 0; i < 4; i++) {
        int j = (i + 1) & 3;
        double a00 = lines[i][3], a01 = -lines[j][3], a10 = -lines[i][2], a11 = lines[j][2];
        double b0 = -lines[i][0] + lines[j][0], b1 = -lines[i][1] + lines[j][1];
        double det = a00 * a11 - a10 * a01;
        if (fabs(det) < 0.001) goto out;
        double w00 = a11 / det, w01 = -a01 / det;
        double l0 = w00 * b0 + w01 * b1;
        q->p[i][0] = (float)(lines[i][0] + l0 * a00);
        q->p[i][1] = (float)(lines[i][1] + l0 * a10);
    }
    /* area of triangles (0,1,2) and (2,3,0) by Heron */
    {
        static const int tri[2][4] = {{0, 1, 2, 0}, {2, 3, 0, 2}};
        double area = 0.0;
        for (int t = 0; t < 2; t++) {
            double len[3];
            for (int i = 0; i < 3; i++) {
                int ia = tri[t][i], ib = tri[t][i + 1];
                float ddx = q->p[ib][0] - q->p[ia][0], ddy = q->p[ib][1] - q->p[ia][1];
                len[i] = sqrt(sqd(ddx) + sqd(ddy));
            }
            double p = (len[0] + len[1] + len[2]) / 2.0;
            area += sqrt(p * (p - len[0]) * (p - len[1]) * (p - len[2]));
        }
        if (area < 0.95 * (double)cfg->tag_width * (double)cfg->tag_width) goto out;
    }
    for (int i = 0; i < 4; i++) {
        int i0 = i, i1 = (i + 1) & 3, i2 = (i + 2) & 3;
        double dx1 = q->p[i1][0] - q->p[i0][0], dy1 = q->p[i1][1] - q->p[i0][1];
        double dx2 = q->p[i2][0] - q->p[i1][0], dy2 = q->p[i2][1] - q->p[i1][1];
        double den = sqrt((dx1 * dx1 + dy1 * dy1) * (dx2 * dx2 + dy2 * dy2));
        if (den == 0.0) goto out;
        double cs = (dx1 * dx2 + dy1 * dy2) / den;
        if ((cs > cfg->max_dot || cs < -cfg->max_dot) || dx1 * dy2 < dy1 * dx2) goto out;
    }
    ok = true;
out:
    free(keys);
    free(buf);
    return ok;
}

/* =====================================================================
   8. Decoding (fast/decode.c). */

typedef struct {
    const uint8_t *im;
    int64_t s, w, h;
} view;

/* Quick-decode tables (fast/decode.c:20-58): the codes split into 4
   chunks of (nbits+3)/4 bits; per chunk, the code indices of each chunk
   value, in index order. */
typedef struct {
    int64_t chunk, cap, ncodes, nbits, maxham;
    uint32_t *off; /* 4 * (cap + 1) */
    uint32_t *idx; /* 4 * ncodes */
    const uint64_t *codes;
} qdtab;

static void qd_build(qdtab *t, const ao_family *f, int bits) {
    t->nbits = f->nbits;
    t->ncodes = f->ncodes;
    t->chunk = (f->nbits + 3) / 4;
    t->cap = (int64_t)1 << t->chunk;
    t->maxham = bits;
    t->codes = f->codes;
    uint64_t mask = (uint64_t)t->cap - 1;
    t->off = xcalloc(4 * (t->cap + 1) * 4);
    t->idx = xmalloc(4 * t->ncodes * 4 + 4);
    for (int64_t i = 0; i < t->ncodes; i++)
        for (int j = 0; j < 4; j++) t->off[j * (t->cap + 1) + ((f->codes[i] >> (j * t->chunk)) & mask) + 1]++;
    for (int j = 0; j < 4; j++)
        for (int64_t v = 0; v < t->cap; v++) t->off[j * (t->cap + 1) + v + 1] += t->off[j * (t->cap + 1) + v];
    uint32_t *cur = xmalloc(4 * (t->cap + 1) * 4);
    memcpy(cur, t->off, 4 * (t->cap + 1) * 4);
    for (int64_t i = 0; i < t->ncodes; i++)
        for (int j = 0; j < 4; j++) {
            int64_t c = j * (t->cap + 1) + ((f->codes[i] >> (j * t->chunk)) & mask);
            t->idx[j * t->ncodes + cur[c]++] = (uint32_t)i;
        }
    free(cur);
}

static uint64_t rot90(uint64_t w0, int64_t nbits) {
    /* fast/decode.c:61-71 */
    int64_t p = nbits, l = 0;
    if (nbits % 4 == 1) {
        p = nbits - 1;
        l = 1;
    }
    uint64_t w = ((w0 >> l) << (p / 4 + l)) | (w0 >> (3 * p / 4 + l) << l) | (w0 & (uint64_t)l);
    return w & (((uint64_t)1 << nbits) - 1);
}

/* The first code (rotations, then chunks, then code index) within
   maxhamming bits (fast/decode.c:87-107). */
static void qd_lookup(const qdtab *t, uint64_t rcode, int64_t *id, int64_t *ham, int64_t *rot) {
    uint64_t mask = (uint64_t)t->cap - 1;
    for (int r = 0; r < 4; r++) {
        for (int j = 0; j < 4; j++) {
            int64_t v = (int64_t)((rcode >> (j * t->chunk)) & mask);
            for (uint32_t e = t->off[j * (t->cap + 1) + v]; e < t->off[j * (t->cap + 1) + v + 1]; e++) {
                uint32_t ci = t->idx[j * t->ncodes + e];
                int64_t hd = __builtin_popcountll(t->codes[ci] ^ rcode);
                if (hd <= t->maxham) {
                    *id = ci;
                    *ham = hd;
                    *rot = r;
                    return;
                }
            }
        }
        rcode = rot90(rcode, t->nbits);
    }
    *id = 65535;
    *ham = 255;
    *rot = 0;
}

/* The homography of 4 correspondences by 8x9 Gaussian elimination with
   partial pivoting (fast/decode.c:114-165). */
static bool homography(const double c[4][4], double H[9]) {
    double a[8][9];
    memset(a, 0, sizeof a);
    for (int i = 0; i < 4; i++) {
        double x = c[i][0], y = c[i][1], X = c[i][2], Y = c[i][3];
        a[2 * i][0] = x;
        a[2 * i][1] = y;
        a[2 * i][2] = 1.0;
        a[2 * i][6] = -x * X;
        a[2 * i][7] = -y * X;
        a[2 * i][8] = X;
        a[2 * i + 1][3] = x;
        a[2 * i + 1][4] = y;
        a[2 * i + 1][5] = 1.0;
        a[2 * i + 1][6] = -x * Y;
        a[2 * i + 1][7] = -y * Y;
        a[2 * i + 1][8] = Y;
    }
    for (int col = 0; col < 8; col++) {
        double best = 0.0;
        int piv = -1;
        for (int r = col; r < 8; r++)
            if (fabs(a[r][col]) > best) {
                best = fabs(a[r][col]);
                piv = r;
            }
        if (piv < 0 || best < 1e-10) return false;
        if (piv != col)
            for (int i = col; i < 9; i++) {
                double t = a[col][i];
                a[col][i] = a[piv][i];
                a[piv][i] = t;
            }
        for (int r = col + 1; r < 8; r++) {
            double f = a[r][col] / a[col][col];
            a[r][col] = 0.0;
            for (int i = col + 1; i < 9; i++) a[r][i] -= f * a[col][i];
        }
    }
    for (int col = 7; col >= 0; col--) {
        double s = 0.0;
        for (int i = col + 1; i < 8; i++) s += a[col][i] * a[i][8];
        a[col][8] = (a[col][8] - s) / a[col][col];
    }
    for (int i = 0; i < 8; i++) H[i] = a[i][8];
    H[8] = 1.0;
    return true;
}

/* Invertibility as the C library's PLU decomposition decides it
   (fast/decode.c:168-196). */
static bool invertible3(const double m[9]) {
    double lu[9];
    memcpy(lu, m, sizeof lu);
    for (int j = 0; j < 3; j++) {
        for (int i = 0; i < 3; i++) {
            int kmax = i < j ? i : j;
            double acc = 0.0;
            for (int k = 0; k < kmax; k++) acc += lu[i * 3 + k] * lu[k * 3 + j];
            lu[i * 3 + j] -= acc;
        }
        int p = j;
        for (int i = j + 1; i < 3; i++)
            if (fabs(lu[i * 3 + j]) > fabs(lu[p * 3 + j])) p = i;
        if (p != j)
            for (int k = 0; k < 3; k++) {
                double t = lu[p * 3 + k];
                lu[p * 3 + k] = lu[j * 3 + k];
                lu[j * 3 + k] = t;
            }
        double d = lu[j * 3 + j];
        if (fabs(d) < 1e-8) return false;
        if (d != 0.0) {
            double inv = 1.0 / d;
            for (int i = j + 1; i < 3; i++) lu[i * 3 + j] *= inv;
        }
    }
    return true;
}

static void project(const double H[9], double x, double y, double *ox, double *oy) {
    double xx = H[0] * x + H[1] * y + H[2];
    double yy = H[3] * x + H[4] * y + H[5];
    double zz = H[6] * x + H[7] * y + H[8];
    *ox = xx / zz;
    *oy = yy / zz;
}

/* Edge refinement (fast/decode.c:408-761). Along the normal of each edge
   at nsamples points, steps n = -range + 0.25 k; a step's weight is
   (g2 - g1)^2 of the bilinear values at n+1 and n-1 along the normal,
   kept when g1 >= g2 and both points are inside. Steps below the largest
   multiple of 4 of the step count go to 4 partial sums by k mod 4
   (combined (0+2)+(1+3)) with their bilinear sums pairwise; the rest are
   added in order with the bilinear sum left to right. */
static double bil_pair(double a, double b, const uint8_t *p, int64_t s) {
    double na = 1.0 - a, nb = 1.0 - b;
    return ((na * nb) * p[0] + (a * nb) * p[1]) + ((na * b) * p[s] + (a * b) * p[s + 1]);
}
static double bil_seq(double a, double b, const uint8_t *p, int64_t s) {
    return (1.0 - a) * (1.0 - b) * p[0] + a * (1.0 - b) * p[1] + (1.0 - a) * b * p[s] + a * b * p[s + 1];
}

static void refine_edges(float qdec, const view *v, ao_quad *q) {
    int64_t w = v->w, h = v->h;
    int64_t range = (int64_t)(qdec + 1.0f);
    int64_t nsteps = 2 * 4 * range + 1;
    int64_t vsteps = nsteps - nsteps % 4;
    double wl = (double)(w - 1), hl = (double)(h - 1);
    double lines[4][4];
    for (int edge = 0; edge < 4; edge++) {
        int a = edge, b = (edge + 1) & 3;
        double nx = (double)(q->p[b][1] - q->p[a][1]);
        double ny = (double)(-q->p[b][0] + q->p[a][0]);
        double mag = sqrt(nx * nx + ny * ny);
        nx /= mag;
        ny /= mag;
        if (q->reversed_border) {
            nx = -nx;
            ny = -ny;
        }
        int64_t nsamples = maxi(16, c_int(mag / 8.0));
        double mx = 0, my = 0, mxx = 0, mxy = 0, myy = 0, nn = 0;
        for (int64_t si = 0; si < nsamples; si++) {
            double alpha = (1.0 + (double)si) / (double)(nsamples + 1);
            double x0 = alpha * q->p[a][0] + (1.0 - alpha) * q->p[b][0];
            double y0 = alpha * q->p[a][1] + (1.0 - alpha) * q->p[b][1];
            double ln[4] = {0, 0, 0, 0}, lc[4] = {0, 0, 0, 0};
            for (int64_t k = 0; k < vsteps; k++) {
                double n = (double)-range + 0.25 * (double)k;
                double x1 = x0 + (n + 1.0) * nx - 0.5, y1 = y0 + (n + 1.0) * ny - 0.5;
                double x2 = x0 + (n - 1.0) * nx - 0.5, y2 = y0 + (n - 1.0) * ny - 0.5;
                double wgt = 0.0;
                if (x1 > -1.0 && x1 < wl && y1 > -1.0 && y1 < hl && x2 > -1.0 && x2 < wl && y2 > -1.0 && y2 < hl) {
                    double tx1 = trunc(x1), ty1 = trunc(y1), tx2 = trunc(x2), ty2 = trunc(y2);
                    double g1 = bil_pair(x1 - tx1, y1 - ty1, v->im + (int64_t)ty1 * v->s + (int64_t)tx1, v->s);
                    double g2 = bil_pair(x2 - tx2, y2 - ty2, v->im + (int64_t)ty2 * v->s + (int64_t)tx2, v->s);
                    double d = g2 - g1;
                    wgt = !(g1 < g2) ? d * d : 0.0;
                }
                ln[k % 4] += wgt * n;
                lc[k % 4] += wgt;
            }
            double mn = 0.0 + ((ln[0] + ln[2]) + (ln[1] + ln[3]));
            double mc = 0.0 + ((lc[0] + lc[2]) + (lc[1] + lc[3]));
            for (int64_t k = vsteps; k < nsteps; k++) {
                double n = (double)-range + 0.25 * (double)k;
                double x1 = x0 + (n + 1.0) * nx - 0.5, y1 = y0 + (n + 1.0) * ny - 0.5;
                int64_t x1i = c_int(x1), y1i = c_int(y1);
                if (x1i < 0 || x1i + 1 >= w || y1i < 0 || y1i + 1 >= h) continue;
                double x2 = x0 + (n - 1.0) * nx - 0.5, y2 = y0 + (n - 1.0) * ny - 0.5;
                int64_t x2i = c_int(x2), y2i = c_int(y2);
                if (x2i < 0 || x2i + 1 >= w || y2i < 0 || y2i + 1 >= h) continue;
                double g1 = bil_seq(x1 - (double)x1i, y1 - (double)y1i, v->im + y1i * v->s + x1i, v->s);
                double g2 = bil_seq(x2 - (double)x2i, y2 - (double)y2i, v->im + y2i * v->s + x2i, v->s);
                if (g1 < g2) continue;
                double wgt = (g2 - g1) * (g2 - g1);
                mn += wgt * n;
                mc += wgt;
            }
            if (mc == 0.0) continue;
            double n0 = mn / mc;
            double bx = x0 + n0 * nx, by = y0 + n0 * ny;
            mx += bx;
            my += by;
            mxx += bx * bx;
            mxy += bx * by;
            myy += by * by;
            nn += 1.0;
        }
        double ex = mx / nn, ey = my / nn;
        double cxx = mxx / nn - ex * ex, cxy = mxy / nn - ex * ey, cyy = myy / nn - ey * ey;
        double theta = 0.5 * (double)ao_atan2f((float)(-2.0 * cxy), (float)(cyy - cxx));
        lines[edge][0] = ex;
        lines[edge][1] = ey;
        lines[edge][2] = ao_cosf((float)theta);
        lines[edge][3] = ao_sinf((float)theta);
    }
    for (int i = 0; i < 4; i++) {
        int j = (i + 1) & 3;
        double a00 = lines[i][3], a01 = -lines[j][3], a10 = -lines[i][2], a11 = lines[j][2];
        double b0 = -lines[i][0] + lines[j][0], b1 = -lines[i][1] + lines[j][1];
        double det = a00 * a11 - a10 * a01;
        if (fabs(det) > 0.001) {
            double w00 = a11 / det, w01 = -a01 / det;
            double l0 = w00 * b0 + w01 * b1;
            q->p[j][0] = (float)(lines[i][0] + l0 * a00);
            q->p[j][1] = (float)(lines[i][1] + l0 * a10);
        }
    }
}

/* Least-squares gray model c0 x + c1 y + c2 (fast/decode.c:225-265). */
typedef struct {
    double a[9], b[3], c[3];
} graymodel;

static void gm_add(graymodel *g, double x, double y, double v) {
    g->a[0] += x * x;
    g->a[1] += x * y;
    g->a[2] += x;
    g->a[4] += y * y;
    g->a[5] += y;
    g->a[8] += 1.0;
    g->b[0] += x * v;
    g->b[1] += y * v;
    g->b[2] += v;
}

static void gm_solve(graymodel *g) {
    const double *a = g->a;
    double L0 = sqrt(a[0]);
    double L3 = a[1] / L0;
    double L6 = a[2] / L0;
    double L4 = sqrt(a[4] - L3 * L3);
    double L7 = (a[5] - L3 * L6) / L4;
    double L8 = sqrt(a[8] - L6 * L6 - L7 * L7);
    double M0 = 1.0 / L0;
    double M3 = -L3 * M0 / L4;
    double M4 = 1.0 / L4;
    double M6 = (-L6 * M0 - L7 * M3) / L8;
    double M7 = -L7 * M4 / L8;
    double M8 = 1.0 / L8;
    const double *b = g->b;
    double t0 = M0 * b[0];
    double t1 = M3 * b[0] + M4 * b[1];
    double t2 = M6 * b[0] + M7 * b[1] + M8 * b[2];
    g->c[0] = M0 * t0 + M3 * t1 + M6 * t2;
    g->c[1] = M4 * t1 + M7 * t2;
    g->c[2] = M8 * t2;
}

static double bilinear_at(const view *v, double px, double py) {
    int64_t x1 = c_int(floor(px - 0.5)), x2 = c_int(ceil(px - 0.5));
    double x = px - 0.5 - (double)x1;
    int64_t y1 = c_int(floor(py - 0.5)), y2 = c_int(ceil(py - 0.5));
    double y = py - 0.5 - (double)y1;
    if (x1 < 0 || x2 >= v->w || y1 < 0 || y2 >= v->h) return -1.0;
    const uint8_t *r1 = v->im + y1 * v->s, *r2 = v->im + y2 * v->s;
    return r1[x1] * (1.0 - x) * (1.0 - y) + r1[x2] * x * (1.0 - y) + r2[x1] * (1.0 - x) * y + r2[x2] * x * y;
}

/* Bit sampling (fast/decode.c:291-402): returns false when the border
   has the wrong polarity for the family. */
static bool sample_bits(const ao_family *f, double sharpening, const view *v, const double *H, float *margin,
                        uint64_t *rcode_out) {
    int32_t wab = f->width_at_border;
    float wf = (float)wab;
    const float pat[8][5] = {
        {-0.5f, 0.5f, 0.0f, 1.0f, 1.0f}, {0.5f, 0.5f, 0.0f, 1.0f, 0.0f},
        {(float)(wab + 0.5), 0.5f, 0.0f, 1.0f, 1.0f}, {(float)(wab - 0.5), 0.5f, 0.0f, 1.0f, 0.0f},
        {0.5f, -0.5f, 1.0f, 0.0f, 1.0f}, {0.5f, 0.5f, 1.0f, 0.0f, 0.0f},
        {0.5f, (float)(wab + 0.5), 1.0f, 0.0f, 1.0f}, {0.5f, (float)(wab - 0.5), 1.0f, 0.0f, 0.0f},
    };
    graymodel wm, bm;
    memset(&wm, 0, sizeof wm);
    memset(&bm, 0, sizeof bm);
    for (int pi = 0; pi < 8; pi++)
        for (int32_t i = 0; i < wab; i++) {
            double tx01 = (double)((pat[pi][0] + (float)i * pat[pi][2]) / wf);
            double ty01 = (double)((pat[pi][1] + (float)i * pat[pi][3]) / wf);
            double tx = 2.0 * (tx01 - 0.5), ty = 2.0 * (ty01 - 0.5);
            double zz = H[6] * tx + H[7] * ty + H[8];
            double px = (H[0] * tx + H[1] * ty + H[2]) / zz;
            double py = (H[3] * tx + H[4] * ty + H[5]) / zz;
            int64_t ix = c_int(px), iy = c_int(py);
            if (ix < 0 || iy < 0 || ix >= v->w || iy >= v->h) continue;
            gm_add(pat[pi][4] != 0.0f ? &wm : &bm, tx, ty, (double)v->im[iy * v->s + ix]);
        }
    gm_solve(&wm);
    if (wab > 1) {
        gm_solve(&bm);
    } else {
        bm.c[0] = 0.0;
        bm.c[1] = 0.0;
        bm.c[2] = bm.b[2] / 4.0;
    }
    double wi = wm.c[0] * 0.0 + wm.c[1] * 0.0 + wm.c[2];
    double bi = bm.c[0] * 0.0 + bm.c[1] * 0.0 + bm.c[2];
    if ((wi - bi < 0.0) != f->reversed_border) return false;
    int64_t tw = f->total_width;
    double *vals = xcalloc(tw * tw * 8), *sharp = xmalloc(tw * tw * 8);
    int64_t minc = (wab - tw) / 2;
    for (int64_t i = 0; i < f->nbits; i++) {
        int64_t bx = f->bit_x[i], by = f->bit_y[i];
        double tx = 2.0 * (((double)bx + 0.5) / wab - 0.5), ty = 2.0 * (((double)by + 0.5) / wab - 0.5);
        double zz = H[6] * tx + H[7] * ty + H[8];
        double px = (H[0] * tx + H[1] * ty + H[2]) / zz;
        double py = (H[3] * tx + H[4] * ty + H[5]) / zz;
        double val = bilinear_at(v, px, py);
        if (val == -1.0) continue;
        double thr = ((bm.c[0] * tx + bm.c[1] * ty + bm.c[2]) + (wm.c[0] * tx + wm.c[1] * ty + wm.c[2])) / 2.0;
        vals[tw * (by - minc) + (bx - minc)] = val - thr;
    }
    for (int64_t y = 0; y < tw; y++)
        for (int64_t x = 0; x < tw; x++) {
            double acc = 0.0;
            if (y > 0) acc += -vals[(y - 1) * tw + x];
            if (x > 0) acc += -vals[y * tw + x - 1];
            acc += vals[y * tw + x] * 4.0;
            if (x + 1 < tw) acc += -vals[y * tw + x + 1];
            if (y + 1 < tw) acc += -vals[(y + 1) * tw + x];
            sharp[y * tw + x] = acc;
        }
    for (int64_t i = 0; i < tw * tw; i++) vals[i] = vals[i] + sharpening * sharp[i];
    float bs = 0.0f, ws = 0.0f, bc = 1.0f, wc = 1.0f;
    uint64_t rcode = 0;
    for (int64_t i = 0; i < f->nbits; i++) {
        rcode <<= 1;
        double vv = vals[(f->bit_y[i] - minc) * tw + (f->bit_x[i] - minc)];
        if (vv > 0.0) {
            ws = (float)(ws + vv);
            wc += 1.0f;
            rcode |= 1;
        } else {
            bs = (float)(bs - vv);
            bc += 1.0f;
        }
    }
    free(vals);
    free(sharp);
    double x = (double)(ws / wc), y = (double)(bs / bc);
    double m = x != x ? y : y != y ? x : x < y ? x : y; /* fmin */
    *margin = (float)m;
    *rcode_out = rcode;
    return true;
}

static ao_detection detection_of(int64_t fi, int64_t id, int64_t ham, int64_t rot, float margin, const double qH[9]) {
    /* fast/detector.c:83-107: H = qH * R(rot * pi/2) with libm cos/sin */
    double th = (double)rot * M_PI / 2.0;
    double c = cos(th), s = sin(th);
    const double r[9] = {c, -s, 0.0, s, c, 0.0, 0.0, 0.0, 1.0};
    ao_detection d;
    memset(&d, 0, sizeof d);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double acc = 0.0;
            for (int k = 0; k < 3; k++) acc += qH[i * 3 + k] * r[k * 3 + j];
            d.H[i * 3 + j] = acc;
        }
    d.family = (int32_t)fi;
    d.id = (int32_t)id;
    d.hamming = (int32_t)ham;
    d.decision_margin = margin;
    project(d.H, 0.0, 0.0, &d.c[0], &d.c[1]);
    for (int i = 0; i < 4; i++) {
        double tx = i == 1 || i == 2 ? 1.0 : -1.0;
        double ty = i < 2 ? 1.0 : -1.0;
        project(d.H, tx, ty, &d.p[i][0], &d.p[i][1]);
    }
    return d;
}

/* =====================================================================
   9. Overlap removal (fast/decode.c:766-891) and the sort by id
   (fast/detector.c:164-179). */

typedef struct {
    double p[2], u[2];
} gline;

static gline gline_of(const double *p0, const double *p1) {
    double u0 = p1[0] - p0[0], u1 = p1[1] - p0[1];
    double mag = (double)sqrtf((float)(u0 * u0 + u1 * u1));
    gline l = {{p0[0], p0[1]}, {u0 / mag, u1 / mag}};
    return l;
}
static double gline_coord(const gline *l, const double *q) {
    return (q[0] - l->p[0]) * l->u[0] + (q[1] - l->p[1]) * l->u[1];
}
static bool segments_cross(const double *a0, const double *a1, const double *b0, const double *b1) {
    gline la = gline_of(a0, a1), lb = gline_of(b0, b1);
    double m00 = la.u[0], m01 = -lb.u[0], m10 = la.u[1], m11 = -lb.u[1];
    double det = m00 * m11 - m01 * m10;
    if (fabs(det) < 0.00000001) return false;
    double i00 = m11 / det, i01 = -m01 / det;
    double b00 = lb.p[0] - la.p[0], b10 = lb.p[1] - la.p[1];
    double x00 = i00 * b00 + i01 * b10;
    double t[2] = {la.u[0] * x00 + la.p[0], la.u[1] * x00 + la.p[1]};
    double a = gline_coord(&la, la.p), b = gline_coord(&la, a1), c = gline_coord(&la, t);
    if ((c < a && c < b) || (c > a && c > b)) return false;
    a = gline_coord(&lb, lb.p);
    b = gline_coord(&lb, b1);
    c = gline_coord(&lb, t);
    if ((c < a && c < b) || (c > a && c > b)) return false;
    return true;
}
static bool poly_contains(const double poly[4][2], const double *q) {
    int last = 0, acc = 0;
    for (int i = 0; i < 5; i++) {
        const double *p = poly[i % 4];
        int quad = p[0] < q[0] ? (p[1] < q[1] ? 2 : 1) : (p[1] < q[1] ? 3 : 0);
        if (i > 0) {
            int dq = quad - last;
            if (dq == -3 || dq == 1)
                acc++;
            else if (dq == -1 || dq == 3)
                acc--;
            else if (dq == -2 || dq == 2) {
                const double *p0 = poly[i - 1];
                double nx = p[1] - q[1], ny = -p[0] + q[0];
                double dot = nx * (p0[0] - q[0]) + ny * (p0[1] - q[1]);
                acc += dot < 0.0 ? -2 : 2;
            }
        }
        last = quad;
    }
    return acc >= 2 || acc <= -2;
}
static bool quads_overlap(const double pa[4][2], const double pb[4][2]) {
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++)
            if (segments_cross(pa[i], pa[(i + 1) % 4], pb[j], pb[(j + 1) % 4])) return true;
    double qb[2] = {(pb[0][0] + pb[1][0] + pb[2][0]) / 3.0, (pb[0][1] + pb[1][1] + pb[2][1]) / 3.0};
    if (poly_contains(pa, qb)) return true;
    double qa[2] = {(pa[0][0] + pa[1][0] + pa[2][0]) / 3.0, (pa[0][1] + pa[1][1] + pa[2][1]) / 3.0};
    return poly_contains(pb, qa);
}
static int prefer(int pref, double a, double b) { return pref ? pref : a < b ? -1 : b < a ? 1 : 0; }

static void drop_overlaps(ao_detection *d, int64_t *n) {
    int64_t i0 = 0;
    while (i0 < *n) {
        bool gone = false;
        int64_t i1 = i0 + 1;
        while (i1 < *n) {
            if (d[i0].id != d[i1].id || d[i0].family != d[i1].family || !quads_overlap(d[i0].p, d[i1].p)) {
                i1++;
                continue;
            }
            int pref = prefer(0, d[i0].hamming, d[i1].hamming);
            pref = prefer(pref, -(double)d[i0].decision_margin, -(double)d[i1].decision_margin);
            for (int i = 0; i < 4; i++) {
                pref = prefer(pref, d[i0].p[i][0], d[i1].p[i][0]);
                pref = prefer(pref, d[i0].p[i][1], d[i1].p[i][1]);
            }
            int64_t drop = pref < 0 ? i1 : i0;
            memmove(d + drop, d + drop + 1, (*n - drop - 1) * sizeof *d);
            (*n)--;
            if (drop == i0) {
                gone = true;
                break;
            }
        }
        if (!gone) i0++;
    }
}

static void stable_sort_by_id(ao_detection *d, int64_t n) {
    /* insertion sort: stable */
    for (int64_t i = 1; i < n; i++) {
        ao_detection x = d[i];
        int64_t j = i;
        while (j > 0 && d[j - 1].id > x.id) {
            d[j] = d[j - 1];
            j--;
        }
        d[j] = x;
    }
}

/* =====================================================================
   The frame (fast/detector.c:196-335). */

int ao_detect(const ao_params *prm, const ao_family *fams, const int32_t *bits, int32_t nfam, const uint8_t *img,
              int64_t w, int64_t h, int64_t stride, int32_t order_mode, ao_result *res) {
    memset(res, 0, sizeof *res);
    if (nfam > AO_MAX_FAMILIES) return -1;
    for (int i = 0; i < nfam; i++)
        if (bits[i] < 0 || bits[i] > 3 || fams[i].ncodes >= 65536 || fams[i].nbits <= 0 || fams[i].nbits > 64)
            return -1;
    if (nfam == 0 || w < 8 || h < 8) return 0;
    int64_t qw = w, qh = h;
    if (prm->quad_decimate > 1.0f) quad_size(w, h, prm->quad_decimate, &qw, &qh);
    res->qw = qw;
    res->qh = qh;
    uint8_t *qim = xmalloc(qw * qh);
    res->qim = qim;
    if (prm->quad_decimate > 1.0f)
        decimate(img, stride, prm->quad_decimate, qim, qw, qh);
    else
        for (int64_t y = 0; y < qh; y++) memcpy(qim + y * qw, img + y * stride, qw);
    bool blurred = blur_or_sharpen(qim, qw, qh, prm->quad_sigma);
    view v = {img, stride, w, h};
    if (blurred && !(prm->quad_decimate > 1.0f)) v = (view){qim, w, w, h};

    uint8_t *t = xmalloc(qw * qh);
    res->thresh = t;
    if (qw < 4 || qh < 4) return 0; /* no whole tile: nothing to threshold */
    threshold(qim, qw, qh, prm->min_white_black_diff, t);
    if (prm->deglitch) deglitch(t, qw, qh);

    /* runs */
    res->run_start = xmalloc(qw * qh * 2);
    res->run_end = xmalloc(qw * qh * 2);
    res->run_v = xmalloc(qw * qh);
    res->row_off = xmalloc((qh + 1) * 4);
    res->row_off[0] = 0;
    int64_t nr = 0;
    for (int64_t y = 0; y < qh; y++) {
        nr += row_runs(t + y * qw, qw, res->run_start + nr, res->run_end + nr, res->run_v + nr);
        res->row_off[y + 1] = (uint32_t)nr;
    }
    res->nruns = nr;
    int64_t nn = nr + qh;
    res->nnodes = nn;

    /* components: the reference's roots and sizes, then the labels */
    ufnode *u = xmalloc(nn * sizeof *u);
    components(res, t, qw, qh, u);
    res->ref_root = xmalloc(nn * 4);
    res->label = xmalloc(nn * 4);
    res->comp_pixels = xmalloc(nn * 4);
    uint32_t *minidx = xmalloc(nn * 4);
    for (int64_t i = 0; i < nn; i++) minidx[i] = 0xffffffffu;
    for (int64_t i = 0; i < nn; i++) {
        uint32_t r = uf_root(u, (uint32_t)i);
        res->ref_root[i] = r;
        if ((uint32_t)i < minidx[r]) minidx[r] = (uint32_t)i;
    }
    uint8_t *nok = xmalloc(nn);
    for (int64_t i = 0; i < nn; i++) {
        uint32_t r = res->ref_root[i];
        res->label[i] = minidx[r];
        res->comp_pixels[i] = u[r].size + 1;
        nok[i] = (int64_t)u[r].size + 1 >= prm->min_cluster_pixels;
    }
    free(minidx);
    free(u);

    /* boundary points and clusters */
    int64_t np = 0;
    emitted *em = NULL;
    if (qh >= 3)
        em = boundary_points(res, t, qw, qh, order_mode == AO_ORDER_REF ? res->ref_root : res->label, nok,
                             order_mode, &np);
    free(nok);
    if (np > 0) qsort(em, np, sizeof *em, cmp_emitted);
    res->npoints = np;
    res->pts = xmalloc(np * 8);
    res->cstart = xmalloc((np + 1) * 4);
    res->cid = xmalloc(np * 8);
    int64_t nc = 0;
    for (int64_t i = 0; i < np; i++) {
        if (i == 0 || em[i].cid != em[i - 1].cid) {
            res->cstart[nc] = (uint32_t)i;
            res->cid[nc] = em[i].cid;
            nc++;
        }
        res->pts[i] = em[i].pt;
    }
    res->cstart[nc] = (uint32_t)np;
    res->nclusters = nc;
    free(em);

    /* quads (fast/quads.c:1145-1160) */
    fitcfg cfg;
    cfg.min_px = prm->min_cluster_pixels;
    cfg.max_nmaxima = prm->max_nmaxima;
    cfg.max_dot = prm->cos_critical_rad;
    cfg.max_mse = prm->max_line_fit_mse;
    for (int i = 0; i < 7; i++) cfg.qsm[i] = (float)exp(-(double)((i - 3) * (i - 3)) / 2.0);
    {
        /* min_tag_width (fast/detector.c:67-81) */
        int32_t mtw = 1000000;
        cfg.normal_border = cfg.reversed_border = false;
        for (int i = 0; i < nfam; i++) {
            if (fams[i].width_at_border < mtw) mtw = fams[i].width_at_border;
            cfg.normal_border = cfg.normal_border || !fams[i].reversed_border;
            cfg.reversed_border = cfg.reversed_border || fams[i].reversed_border;
        }
        if (prm->quad_decimate > 1.0f) mtw = (int32_t)((float)mtw / prm->quad_decimate);
        if (mtw < 3) mtw = 3;
        cfg.tag_width = mtw;
    }
    int64_t max_px = 2 * (2 * qw + 2 * qh);
    res->quads = xmalloc((nc + 1) * sizeof(ao_quad));
    int64_t nq = 0;
    for (int64_t c = 0; c < nc; c++) {
        int64_t n = res->cstart[c + 1] - res->cstart[c];
        if (n < cfg.min_px || n > max_px) continue;
        ao_quad q;
        memset(&q, 0, sizeof q);
        if (fit_quad(&cfg, res->pts + res->cstart[c], n, qim, qw, qh, &q)) {
            q.cluster = (int32_t)c;
            res->quads[nq++] = q;
        }
    }
    res->nquads = nq;

    /* decode (fast/detector.c:113-139, 313-322) */
    qdtab tabs[AO_MAX_FAMILIES];
    for (int i = 0; i < nfam; i++) qd_build(&tabs[i], &fams[i], bits[i]);
    int64_t dcap = 16, nd = 0;
    ao_detection *dets = xmalloc(dcap * sizeof *dets);
    for (int64_t qi = 0; qi < nq; qi++) {
        ao_quad q = res->quads[qi];
        if (prm->quad_decimate > 1.0f)
            for (int j = 0; j < 4; j++) {
                q.p[j][0] *= prm->quad_decimate;
                q.p[j][1] *= prm->quad_decimate;
            }
        if (prm->refine_edges) refine_edges(prm->quad_decimate, &v, &q);
        double corr[4][4], H[9];
        for (int i = 0; i < 4; i++) {
            corr[i][0] = i == 0 || i == 3 ? -1.0 : 1.0;
            corr[i][1] = i == 0 || i == 1 ? -1.0 : 1.0;
            corr[i][2] = q.p[i][0];
            corr[i][3] = q.p[i][1];
        }
        if (!homography(corr, H) || !invertible3(H)) continue;
        for (int fi = 0; fi < nfam; fi++) {
            if (fams[fi].reversed_border != (q.reversed_border != 0)) continue;
            float margin;
            uint64_t rcode;
            if (!sample_bits(&fams[fi], prm->decode_sharpening, &v, H, &margin, &rcode)) continue;
            int64_t id, ham, rot;
            qd_lookup(&tabs[fi], rcode, &id, &ham, &rot);
            if (!(margin >= 0.0f && ham < 255)) continue;
            if (nd == dcap) {
                dcap *= 2;
                dets = realloc(dets, dcap * sizeof *dets);
                if (!dets) abort();
            }
            dets[nd++] = detection_of(fi, id, ham, rot, margin, H);
        }
    }
    for (int i = 0; i < nfam; i++) {
        free(tabs[i].off);
        free(tabs[i].idx);
    }
    drop_overlaps(dets, &nd);
    stable_sort_by_id(dets, nd);
    res->dets = dets;
    res->ndet = nd;
    return 0;
}

void ao_result_free(ao_result *r) {
    free(r->qim);
    free(r->thresh);
    free(r->run_start);
    free(r->run_end);
    free(r->run_v);
    free(r->row_off);
    free(r->label);
    free(r->ref_root);
    free(r->comp_pixels);
    free(r->cstart);
    free(r->cid);
    free(r->pts);
    free(r->quads);
    free(r->dets);
    memset(r, 0, sizeof *r);
}
