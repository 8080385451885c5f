/* A small baseline JPEG encoder for synthetic inputs (the JPEG-input
   benchmark and tests): gray or YCbCr, luma sampling up to 2x2 (chroma
   1x1), the ITU-T T.81 Annex K quantisation tables scaled by quality as the
   IJG library scales them, the Annex K Huffman tables or per-image optimal
   ones (Annex K.2), restart markers every n MCUs. Not part of the decoder:
   built into its own small library next to the package. */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

enum {
    SJ_OPTIMIZE = 1,  /* per-image optimal Huffman tables */
    SJ_NO_DHT = 2,    /* leave the Huffman tables out (Annex K ones used) */
    SJ_MARKERS = 4,   /* add APP0, APP13 and COM segments */
    SJ_ONE_DQT = 8,   /* both quantisation tables in one DQT segment */
};

/* Zig-zag position -> natural position. */
static const uint8_t ZIG[64] = {0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,
                                12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6,  7,  14, 21, 28,
                                35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
                                58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

/* The Annex K Huffman tables (ITU-T T.81, K.3). */
static const uint8_t K_DC_L_BITS[16] = {0, 1, 5, 1, 1, 1, 1, 1, 1, 0, 0, 0, 0, 0, 0, 0};
static const uint8_t K_DC_C_BITS[16] = {0, 3, 1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 0, 0, 0, 0};
static const uint8_t K_DC_VALS[12] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11};
static const uint8_t K_AC_L_BITS[16] = {0, 2, 1, 3, 3, 2, 4, 3, 5, 5, 4, 4, 0, 0, 1, 0x7d};
static const uint8_t K_AC_L_VALS[162] = {
    0x01, 0x02, 0x03, 0x00, 0x04, 0x11, 0x05, 0x12, 0x21, 0x31, 0x41, 0x06, 0x13, 0x51, 0x61, 0x07, 0x22, 0x71,
    0x14, 0x32, 0x81, 0x91, 0xa1, 0x08, 0x23, 0x42, 0xb1, 0xc1, 0x15, 0x52, 0xd1, 0xf0, 0x24, 0x33, 0x62, 0x72,
    0x82, 0x09, 0x0a, 0x16, 0x17, 0x18, 0x19, 0x1a, 0x25, 0x26, 0x27, 0x28, 0x29, 0x2a, 0x34, 0x35, 0x36, 0x37,
    0x38, 0x39, 0x3a, 0x43, 0x44, 0x45, 0x46, 0x47, 0x48, 0x49, 0x4a, 0x53, 0x54, 0x55, 0x56, 0x57, 0x58, 0x59,
    0x5a, 0x63, 0x64, 0x65, 0x66, 0x67, 0x68, 0x69, 0x6a, 0x73, 0x74, 0x75, 0x76, 0x77, 0x78, 0x79, 0x7a, 0x83,
    0x84, 0x85, 0x86, 0x87, 0x88, 0x89, 0x8a, 0x92, 0x93, 0x94, 0x95, 0x96, 0x97, 0x98, 0x99, 0x9a, 0xa2, 0xa3,
    0xa4, 0xa5, 0xa6, 0xa7, 0xa8, 0xa9, 0xaa, 0xb2, 0xb3, 0xb4, 0xb5, 0xb6, 0xb7, 0xb8, 0xb9, 0xba, 0xc2, 0xc3,
    0xc4, 0xc5, 0xc6, 0xc7, 0xc8, 0xc9, 0xca, 0xd2, 0xd3, 0xd4, 0xd5, 0xd6, 0xd7, 0xd8, 0xd9, 0xda, 0xe1, 0xe2,
    0xe3, 0xe4, 0xe5, 0xe6, 0xe7, 0xe8, 0xe9, 0xea, 0xf1, 0xf2, 0xf3, 0xf4, 0xf5, 0xf6, 0xf7, 0xf8, 0xf9, 0xfa};
static const uint8_t K_AC_C_BITS[16] = {0, 2, 1, 2, 4, 4, 3, 4, 7, 5, 4, 4, 0, 1, 2, 0x77};
static const uint8_t K_AC_C_VALS[162] = {
    0x00, 0x01, 0x02, 0x03, 0x11, 0x04, 0x05, 0x21, 0x31, 0x06, 0x12, 0x41, 0x51, 0x07, 0x61, 0x71, 0x13, 0x22,
    0x32, 0x81, 0x08, 0x14, 0x42, 0x91, 0xa1, 0xb1, 0xc1, 0x09, 0x23, 0x33, 0x52, 0xf0, 0x15, 0x62, 0x72, 0xd1,
    0x0a, 0x16, 0x24, 0x34, 0xe1, 0x25, 0xf1, 0x17, 0x18, 0x19, 0x1a, 0x26, 0x27, 0x28, 0x29, 0x2a, 0x35, 0x36,
    0x37, 0x38, 0x39, 0x3a, 0x43, 0x44, 0x45, 0x46, 0x47, 0x48, 0x49, 0x4a, 0x53, 0x54, 0x55, 0x56, 0x57, 0x58,
    0x59, 0x5a, 0x63, 0x64, 0x65, 0x66, 0x67, 0x68, 0x69, 0x6a, 0x73, 0x74, 0x75, 0x76, 0x77, 0x78, 0x79, 0x7a,
    0x82, 0x83, 0x84, 0x85, 0x86, 0x87, 0x88, 0x89, 0x8a, 0x92, 0x93, 0x94, 0x95, 0x96, 0x97, 0x98, 0x99, 0x9a,
    0xa2, 0xa3, 0xa4, 0xa5, 0xa6, 0xa7, 0xa8, 0xa9, 0xaa, 0xb2, 0xb3, 0xb4, 0xb5, 0xb6, 0xb7, 0xb8, 0xb9, 0xba,
    0xc2, 0xc3, 0xc4, 0xc5, 0xc6, 0xc7, 0xc8, 0xc9, 0xca, 0xd2, 0xd3, 0xd4, 0xd5, 0xd6, 0xd7, 0xd8, 0xd9, 0xda,
    0xe2, 0xe3, 0xe4, 0xe5, 0xe6, 0xe7, 0xe8, 0xe9, 0xea, 0xf2, 0xf3, 0xf4, 0xf5, 0xf6, 0xf7, 0xf8, 0xf9, 0xfa};


typedef struct {
    uint8_t *out;
    int64_t cap, n;
    uint32_t acc;
    int nacc, fail;
} bw_t;

static void bw_byte(bw_t *w, int b) {
    if (w->n < w->cap) w->out[w->n] = (uint8_t)b;
    else w->fail = 1;
    w->n++;
}
static void bw_u16(bw_t *w, int v) { bw_byte(w, (v >> 8) & 255); bw_byte(w, v & 255); }
static void bw_bits(bw_t *w, uint32_t code, int len) {
    for (int i = len - 1; i >= 0; i--) {
        w->acc = (w->acc << 1) | ((code >> i) & 1);
        if (++w->nacc == 8) {
            bw_byte(w, (int)(w->acc & 255));
            if ((w->acc & 255) == 255) bw_byte(w, 0);
            w->acc = 0;
            w->nacc = 0;
        }
    }
}
static void bw_pad(bw_t *w) { while (w->nacc) bw_bits(w, 1, 1); }

typedef struct {
    uint8_t bits[16];
    uint8_t vals[256];
    int nvals;
    uint16_t code[256];
    uint8_t size[256];
} enc_huff_t;

static void eh_codes(enc_huff_t *t) {
    memset(t->size, 0, sizeof(t->size));
    uint32_t code = 0;
    int k = 0;
    for (int l = 1; l <= 16; l++) {
        for (int i = 0; i < t->bits[l - 1]; i++, k++) {
            t->code[t->vals[k]] = (uint16_t)code++;
            t->size[t->vals[k]] = (uint8_t)l;
        }
        code <<= 1;
    }
}

static void eh_std(enc_huff_t *t, const uint8_t *bits, const uint8_t *vals) {
    memcpy(t->bits, bits, 16);
    t->nvals = 0;
    for (int l = 0; l < 16; l++) t->nvals += bits[l];
    memcpy(t->vals, vals, (size_t)t->nvals);
    eh_codes(t);
}

/* Code lengths from symbol counts, limited to 16 bits with the all-ones
   code left free (ITU-T T.81 Annex K.2, restated). */
static void eh_optimal(enc_huff_t *t, const int64_t *count) {
    int64_t f[257];
    int csize[257], next[257];
    for (int i = 0; i < 256; i++) f[i] = count[i];
    f[256] = 1; /* a reserved symbol keeps the all-ones code unused */
    for (int i = 0; i < 257; i++) { csize[i] = 0; next[i] = -1; }
    for (;;) {
        int v1 = -1, v2 = -1;
        for (int i = 0; i < 257; i++)
            if (f[i] > 0 && (v1 < 0 || f[i] <= f[v1])) v1 = i;
        for (int i = 0; i < 257; i++)
            if (f[i] > 0 && i != v1 && (v2 < 0 || f[i] <= f[v2])) v2 = i;
        if (v2 < 0) break;
        f[v1] += f[v2];
        f[v2] = 0;
        for (int v = v1;; v = next[v]) { csize[v]++; if (next[v] < 0) { next[v] = v2; break; } }
        for (int v = v2; v >= 0; v = next[v]) csize[v]++;
    }
    int nb[33] = {0};
    for (int i = 0; i < 257; i++)
        if (csize[i]) nb[csize[i] > 32 ? 32 : csize[i]]++;
    for (int i = 32; i > 16; i--)
        while (nb[i] > 0) {
            int j = i - 2;
            while (nb[j] == 0) j--;
            nb[i] -= 2;
            nb[i - 1] += 1;
            nb[j + 1] += 2;
            nb[j] -= 1;
        }
    int i = 16;
    while (nb[i] == 0) i--;
    nb[i]--; /* the reserved symbol's code */
    for (int l = 1; l <= 16; l++) t->bits[l - 1] = (uint8_t)nb[l];
    t->nvals = 0;
    for (int l = 1; l <= 32; l++)
        for (int s = 0; s < 256; s++)
            if (csize[s] == l) t->vals[t->nvals++] = (uint8_t)s;
    eh_codes(t);
}

static const uint8_t K_Q_LUMA[64] = {  /* Annex K.1, natural order */
    16, 11, 10, 16, 24, 40, 51, 61, 12, 12, 14, 19, 26, 58, 60, 55, 14, 13, 16, 24, 40, 57, 69, 56,
    14, 17, 22, 29, 51, 87, 80, 62, 18, 22, 37, 56, 68, 109, 103, 77, 24, 35, 55, 64, 81, 104, 113, 92,
    49, 64, 78, 87, 103, 121, 120, 101, 72, 92, 95, 98, 112, 100, 103, 99};
static const uint8_t K_Q_CHROMA[64] = {
    17, 18, 24, 47, 99, 99, 99, 99, 18, 21, 26, 66, 99, 99, 99, 99, 24, 26, 56, 99, 99, 99, 99, 99,
    47, 66, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99,
    99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99};

static void fdct_quant(const float *px, int64_t stride, const uint8_t *qz, int16_t *outz) {
    static float cs[8][8];
    static int init = 0;
    if (!init) {
        for (int u = 0; u < 8; u++)
            for (int x = 0; x < 8; x++)
                cs[u][x] = (float)((u ? 0.5 : 0.5 / sqrt(2.0)) * cos((2 * x + 1) * u * M_PI / 16));
        init = 1;
    }
    float tmp[8][8], F[8][8];
    for (int y = 0; y < 8; y++)
        for (int u = 0; u < 8; u++) {
            float a = 0;
            for (int x = 0; x < 8; x++) a += cs[u][x] * (px[y * stride + x] - 128.0f);
            tmp[y][u] = a;
        }
    for (int u = 0; u < 8; u++)
        for (int v = 0; v < 8; v++) {
            float a = 0;
            for (int y = 0; y < 8; y++) a += cs[v][y] * tmp[y][u];
            F[v][u] = a;
        }
    for (int k = 0; k < 64; k++) {
        int n = ZIG[k];
        long c = lroundf(F[n / 8][n % 8] / qz[k]);
        if (c > 1023) c = 1023;
        if (c < -1023) c = -1023;
        outz[k] = (int16_t)c;
    }
}

static int nbits_of(int v) {
    int a = v < 0 ? -v : v, n = 0;
    while (a) { n++; a >>= 1; }
    return n;
}

/* Walks every block in MCU order, calling emit for the DC difference and
   the AC run/size symbols; `pred` reset at every restart. */
typedef void (*sym_fn)(void *ctx, int table, int sym, int nb, int extra);

static void walk(const int16_t *coef, int64_t nmcu, int nb_mcu, const int *blk_comp, int restart, sym_fn fn,
                 void *ctx, bw_t *w) {
    int pred[3] = {0, 0, 0};
    int rst = 0;
    for (int64_t m = 0; m < nmcu; m++) {
        if (restart > 0 && m > 0 && m % restart == 0) {
            if (w) {
                bw_pad(w);
                bw_byte(w, 0xff);
                bw_byte(w, 0xd0 + rst);
            }
            rst = (rst + 1) & 7;
            pred[0] = pred[1] = pred[2] = 0;
        }
        for (int b = 0; b < nb_mcu; b++) {
            const int16_t *z = coef + (m * nb_mcu + b) * 64;
            int c = blk_comp[b], t = c ? 1 : 0;
            int d = z[0] - pred[c];
            pred[c] = z[0];
            int s = nbits_of(d);
            fn(ctx, t, s, s, d < 0 ? d + (1 << s) - 1 : d);
            int run = 0;
            for (int k = 1; k < 64; k++) {
                if (z[k] == 0) { run++; continue; }
                while (run > 15) { fn(ctx, 2 + t, 0xf0, 0, 0); run -= 16; }
                s = nbits_of(z[k]);
                fn(ctx, 2 + t, (run << 4) | s, s, z[k] < 0 ? z[k] + (1 << s) - 1 : z[k]);
                run = 0;
            }
            if (run) fn(ctx, 2 + t, 0, 0, 0);
        }
    }
    if (w) bw_pad(w);
}

static void count_sym(void *ctx, int table, int sym, int nb, int extra) {
    ((int64_t(*)[256])ctx)[table][sym]++;
}

typedef struct { bw_t *w; enc_huff_t *h; } put_ctx;
static void put_sym(void *ctx, int table, int sym, int nb, int extra) {
    put_ctx *p = (put_ctx *)ctx;
    bw_bits(p->w, p->h[table].code[sym], p->h[table].size[sym]);
    if (nb) bw_bits(p->w, (uint32_t)extra, nb);
}

int64_t sj_encode(const uint8_t *img, int w, int h, int64_t stride, int nc, int hs, int vs, int quality,
                  int restart, int flags, uint8_t *out, int64_t cap) {
    if ((nc != 1 && nc != 3) || hs < 1 || hs > 2 || vs < 1 || vs > 2 || quality < 1 || quality > 100 || w < 1 ||
        h < 1 || w > 65535 || h > 65535 || restart < 0 || restart > 65535)
        return -1;
    int scale = quality < 50 ? 5000 / quality : 200 - 2 * quality;
    uint8_t qz[2][64];
    for (int k = 0; k < 64; k++) {
        for (int t = 0; t < 2; t++) {
            int v = ((t ? K_Q_CHROMA : K_Q_LUMA)[ZIG[k]] * scale + 50) / 100;
            qz[t][k] = (uint8_t)(v < 1 ? 1 : v > 255 ? 255 : v);
        }
    }
    const int mw = 8 * hs, mh = 8 * vs;
    const int64_t mx = (w + mw - 1) / mw, my = (h + mh - 1) / mh, pw = mx * mw, ph = my * mh;
    const int64_t cw = mx * 8, ch = my * 8;
    float *Y = (float *)malloc(sizeof(float) * pw * ph);
    float *Cb = nc == 3 ? (float *)malloc(sizeof(float) * cw * ch) : NULL;
    float *Cr = nc == 3 ? (float *)malloc(sizeof(float) * cw * ch) : NULL;
    float *full = nc == 3 ? (float *)malloc(sizeof(float) * pw * ph * 2) : NULL;
    int nb_mcu = hs * vs + (nc == 3 ? 2 : 0);
    int16_t *coef = (int16_t *)malloc(sizeof(int16_t) * 64 * nb_mcu * mx * my);
    if (!Y || !coef || (nc == 3 && (!Cb || !Cr || !full))) {
        free(Y); free(Cb); free(Cr); free(full); free(coef);
        return -1;
    }
    for (int64_t y = 0; y < ph; y++)
        for (int64_t x = 0; x < pw; x++) {
            int64_t sx = x < w ? x : w - 1, sy = y < h ? y : h - 1;
            if (nc == 1) {
                Y[y * pw + x] = img[sy * stride + sx];
            } else {
                const uint8_t *p = img + sy * stride + 3 * sx;
                float r = p[0], g = p[1], b = p[2];
                Y[y * pw + x] = 0.299f * r + 0.587f * g + 0.114f * b;
                full[(y * pw + x) * 2] = -0.168736f * r - 0.331264f * g + 0.5f * b + 128.0f;
                full[(y * pw + x) * 2 + 1] = 0.5f * r - 0.418688f * g - 0.081312f * b + 128.0f;
            }
        }
    if (nc == 3)
        for (int64_t y = 0; y < ch; y++)
            for (int64_t x = 0; x < cw; x++) {
                float a = 0, b = 0;
                for (int dy = 0; dy < vs; dy++)
                    for (int dx = 0; dx < hs; dx++) {
                        int64_t o = ((y * vs + dy) * pw + x * hs + dx) * 2;
                        a += full[o];
                        b += full[o + 1];
                    }
                Cb[y * cw + x] = a / (hs * vs);
                Cr[y * cw + x] = b / (hs * vs);
            }
    int blk_comp[6];
    for (int64_t m = 0, i = 0; m < mx * my; m++) {
        int64_t bx = m % mx, by = m / mx;
        for (int sy = 0; sy < vs; sy++)
            for (int sx = 0; sx < hs; sx++, i++) {
                blk_comp[sy * hs + sx] = 0;
                fdct_quant(Y + (by * mh + sy * 8) * pw + bx * mw + sx * 8, pw, qz[0], coef + i * 64);
            }
        if (nc == 3) {
            blk_comp[hs * vs] = 1;
            blk_comp[hs * vs + 1] = 2;
            fdct_quant(Cb + by * 8 * cw + bx * 8, cw, qz[1], coef + i++ * 64);
            fdct_quant(Cr + by * 8 * cw + bx * 8, cw, qz[1], coef + i++ * 64);
        }
    }
    free(Y); free(Cb); free(Cr); free(full);

    enc_huff_t ht[4];
    if (flags & SJ_OPTIMIZE) {
        int64_t cnt[4][256];
        memset(cnt, 0, sizeof(cnt));
        walk(coef, mx * my, nb_mcu, blk_comp, restart, count_sym, cnt, NULL);
        const uint8_t *sb[4] = {K_DC_L_BITS, K_DC_C_BITS, K_AC_L_BITS, K_AC_C_BITS};
        const uint8_t *sv[4] = {K_DC_VALS, K_DC_VALS, K_AC_L_VALS, K_AC_C_VALS};
        for (int t = 0; t < 4; t++) {
            int used = 0;
            for (int k = 0; k < 256; k++) used |= cnt[t][k] != 0;
            if (used) eh_optimal(&ht[t], cnt[t]);
            else eh_std(&ht[t], sb[t], sv[t]);
        }
    } else {
        eh_std(&ht[0], K_DC_L_BITS, K_DC_VALS);
        eh_std(&ht[1], K_DC_C_BITS, K_DC_VALS);
        eh_std(&ht[2], K_AC_L_BITS, K_AC_L_VALS);
        eh_std(&ht[3], K_AC_C_BITS, K_AC_C_VALS);
    }

    bw_t bw = {out, cap, 0, 0, 0, 0};
    bw_t *W = &bw;
    bw_u16(W, 0xffd8);
    if (flags & SJ_MARKERS) {
        static const uint8_t app0[14] = {'J', 'F', 'I', 'F', 0, 1, 1, 0, 0, 1, 0, 1, 0, 0};
        bw_u16(W, 0xffe0); bw_u16(W, 16);
        for (int i = 0; i < 14; i++) bw_byte(W, app0[i]);
        bw_u16(W, 0xffed); bw_u16(W, 10);
        for (int i = 0; i < 8; i++) bw_byte(W, i & 1 ? 0xff : 0xd9);
        bw_u16(W, 0xfffe); bw_u16(W, 6);
        for (int i = 0; i < 4; i++) bw_byte(W, "test"[i]);
    }
    int nq = nc == 3 ? 2 : 1;
    for (int t = 0; t < nq; t++) {
        if (t == 0 || !(flags & SJ_ONE_DQT)) {
            bw_u16(W, 0xffdb);
            bw_u16(W, 2 + 65 * ((flags & SJ_ONE_DQT) ? nq : 1));
        }
        bw_byte(W, t);
        for (int k = 0; k < 64; k++) bw_byte(W, qz[t][k]);
    }
    bw_u16(W, 0xffc0);
    bw_u16(W, 8 + 3 * nc);
    bw_byte(W, 8);
    bw_u16(W, h);
    bw_u16(W, w);
    bw_byte(W, nc);
    for (int c = 0; c < nc; c++) {
        bw_byte(W, c + 1);
        bw_byte(W, c ? 0x11 : (hs << 4) | vs);
        bw_byte(W, c ? 1 : 0);
    }
    if (!(flags & SJ_NO_DHT)) {
        int order[4] = {0, 2, 1, 3}, cls[4] = {0x00, 0x10, 0x01, 0x11};
        int nt = nc == 3 ? 4 : 2, len = 2;
        for (int i = 0; i < nt; i++) len += 17 + ht[order[i]].nvals;
        bw_u16(W, 0xffc4);
        bw_u16(W, len);
        for (int i = 0; i < nt; i++) {
            enc_huff_t *t = &ht[order[i]];
            bw_byte(W, cls[i]);
            for (int l = 0; l < 16; l++) bw_byte(W, t->bits[l]);
            for (int k = 0; k < t->nvals; k++) bw_byte(W, t->vals[k]);
        }
    }
    if (restart > 0) {
        bw_u16(W, 0xffdd);
        bw_u16(W, 4);
        bw_u16(W, restart);
    }
    bw_u16(W, 0xffda);
    bw_u16(W, 6 + 2 * nc);
    bw_byte(W, nc);
    for (int c = 0; c < nc; c++) {
        bw_byte(W, c + 1);
        bw_byte(W, c ? 0x11 : 0x00);
    }
    bw_byte(W, 0);
    bw_byte(W, 63);
    bw_byte(W, 0);
    put_ctx pc = {W, ht};
    walk(coef, mx * my, nb_mcu, blk_comp, restart, put_sym, &pc, W);
    bw_u16(W, 0xffd9);
    free(coef);
    return W->fail ? -1 : W->n;
}
