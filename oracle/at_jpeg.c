/* CPU checker of the JPEG input path: a restatement of the reference's
   baseline decoder (common/pjpeg.c, common/pjpeg-idct.c) and a small
   encoder for test inputs. TEST INFRASTRUCTURE ONLY; see at_jpeg.h. */
#include "at_jpeg.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ */
/* Byte and bit reader (common/pjpeg.c:163-244).                       */
/* The stream a decoder sees: FF 00 reads as one FF byte; any other    */
/* byte, markers included, reads as itself; past the end of the        */
/* buffer the reader yields 1-bits without moving.                     */

typedef struct {
    const uint8_t *in;
    int64_t pos, len;
    uint32_t bits;   /* the low `avail` bits are the next bits of the stream */
    int avail;
} rd_t;

static void rd_fill(rd_t *r, int need) {
    while (r->avail < need) {
        uint8_t b = 0xff;
        if (r->pos < r->len) {
            b = r->in[r->pos++];
            if (b == 0xff && r->pos < r->len && r->in[r->pos] == 0)
                r->pos++;
        }
        r->bits = (r->bits << 8) | b;
        r->avail += 8;
    }
}

static uint32_t rd_peek(rd_t *r, int n) {
    rd_fill(r, n);
    return n ? (r->bits >> (r->avail - n)) & ((1u << n) - 1) : 0;
}

static uint32_t rd_take(rd_t *r, int n) {
    uint32_t v = rd_peek(r, n);
    r->avail -= n;
    return v;
}

static int rd_more(const rd_t *r) { return r->avail > 0 || r->pos < r->len; }
static void rd_align(rd_t *r) { r->avail -= r->avail & 7; }

/* ------------------------------------------------------------------ */
/* Huffman code space (common/pjpeg.c:386-436). Codes are laid out in  */
/* a 16-bit space in order of length; a code of n bits covers 2^(16-n) */
/* positions. A window past the last code decodes as 0 bits, symbol 0. */

typedef struct {
    int present;
    uint32_t lim[17];   /* end of the codes of length <= l in the 16-bit space */
    uint16_t first[17]; /* index of the first symbol of length l */
    uint8_t sym[256 * 17];
} huff_t;

static void huff_lookup(const huff_t *t, uint32_t w16, int *nbits, int *sym) {
    for (int l = 1; l <= 16; l++) {
        if (w16 < t->lim[l]) {
            uint32_t start = t->lim[l - 1];
            *nbits = l;
            *sym = t->sym[t->first[l] + ((w16 - start) >> (16 - l))];
            return;
        }
    }
    *nbits = 0;
    *sym = 0;
}

/* ------------------------------------------------------------------ */
/* The integer IDCT of the reference (common/pjpeg-idct.c:272-385):    */
/* the fixed-point butterfly of the MPEG-2 reference decoder as        */
/* NanoJPEG writes it, a row pass into 32-bit integers, then a column  */
/* pass that rounds, level-shifts and clamps. The rotation constants   */
/* are 2048 * sqrt(2) * cos(k*pi/16), k = 1, 2, 3, 5, 6, 7.            */

enum { C1 = 2841, C2 = 2676, C3 = 2408, C5 = 1609, C6 = 1108, C7 = 565 };

/* One 8-point pass over v[0], v[s], ..., v[7s]. Row pass (col == 0):
   in place, DC scaled by 2^11 with bias 128, results >> 8. Column pass:
   DC scaled by 2^8 with bias 8192, rotations rounded (+4) >> 3, results
   >> 14, + 128, clamped to a byte and stored to out[k * ostride]. */
static void idct_pass(int32_t *v, int s, int col, uint8_t *out, int64_t ostride) {
    const int sh = col ? 8 : 11;
    int32_t x1 = (int32_t)((uint32_t)v[4 * s] << sh);
    int32_t a2 = v[6 * s], a3 = v[2 * s], a4 = v[1 * s], a5 = v[7 * s], a6 = v[5 * s], a7 = v[3 * s];
    if (!(x1 | a2 | a3 | a4 | a5 | a6 | a7)) {
        if (!col) {
            int32_t d = v[0] * 8;
            for (int k = 0; k < 8; k++) v[k * s] = d;
        } else {
            int32_t d = ((v[0] + 32) >> 6) + 128;
            uint8_t b = d < 0 ? 0 : d > 255 ? 255 : (uint8_t)d;
            for (int k = 0; k < 8; k++) out[k * ostride] = b;
        }
        return;
    }
    const int32_t rb = col ? 4 : 0;
    int32_t x0 = (int32_t)((uint32_t)v[0] << sh) + (col ? 8192 : 128);
    int32_t t, o4, o5, o6, o7, e2, e3;
    t = C7 * (a4 + a5) + rb;
    o4 = t + (C1 - C7) * a4;
    o5 = t - (C1 + C7) * a5;
    t = C3 * (a6 + a7) + rb;
    o6 = t - (C3 - C5) * a6;
    o7 = t - (C3 + C5) * a7;
    t = C6 * (a3 + a2) + rb;
    e2 = t - (C2 + C6) * a2;
    e3 = t + (C2 - C6) * a3;
    if (col) { o4 >>= 3; o5 >>= 3; o6 >>= 3; o7 >>= 3; e2 >>= 3; e3 >>= 3; }
    int32_t e8 = x0 + x1, e0 = x0 - x1;
    int32_t s1 = o4 + o6, d4 = o4 - o6, s6 = o5 + o7, d5 = o5 - o7;
    int32_t f7 = e8 + e3, f8 = e8 - e3, f3 = e0 + e2, f0 = e0 - e2;
    int32_t g2 = (181 * (d4 + d5) + 128) >> 8, g4 = (181 * (d4 - d5) + 128) >> 8;
    int32_t r[8] = {f7 + s1, f3 + g2, f0 + g4, f8 + s6, f8 - s6, f0 - g4, f3 - g2, f7 - s1};
    if (!col) {
        for (int k = 0; k < 8; k++) v[k * s] = r[k] >> 8;
    } else {
        for (int k = 0; k < 8; k++) {
            int32_t d = (r[k] >> 14) + 128;
            out[k * ostride] = d < 0 ? 0 : d > 255 ? 255 : (uint8_t)d;
        }
    }
}

static void idct_block(int32_t blk[64], uint8_t *out, int64_t stride) {
    for (int r = 0; r < 8; r++) idct_pass(blk + 8 * r, 1, 0, NULL, 0);
    for (int c = 0; c < 8; c++) idct_pass(blk + c, 8, 1, out + c, stride);
}

/* Zig-zag position -> natural position. */
static const uint8_t ZIG[64] = {0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,
                                12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6,  7,  14, 21, 28,
                                35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
                                58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

/* The Annex K tables (ITU-T T.81, K.3), which the reference loads for
   files without DHT segments under its MJPEG flag. */
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

/* ------------------------------------------------------------------ */
/* Decoder (common/pjpeg.c:246-687).                                   */

typedef struct {
    uint32_t width, height;
    int ncomp;
    oj_plane comp[3];
    uint8_t q[4][64];     /* quantisation tables, zig-zag order */
    huff_t h[4];          /* DC 0, DC 1, AC 0, AC 1 */
    int restart;          /* MCUs per restart interval, 0: none */
    int rst_next;         /* the restart number expected next, kept across scans */
} dec_t;

static int read_dht(dec_t *d, rd_t *r) {
    uint16_t left = (uint16_t)(rd_take(r, 16) - 2);
    while (left > 0) {
        uint8_t tcth = (uint8_t)rd_take(r, 8);
        left--;
        int tc = tcth >> 4, th = tcth & 15;
        if (tc >= 2 || th >= 2) return OJ_ERR_DHT;
        huff_t *t = &d->h[tc * 2 + th];
        uint8_t cnt[17];
        cnt[0] = 0;
        for (int l = 1; l <= 16; l++) {
            cnt[l] = (uint8_t)rd_take(r, 8);
            left -= cnt[l];
        }
        left -= 16;
        memset(t, 0, sizeof(*t));
        uint32_t pos = 0;
        int nsym = 0;
        for (int l = 1; l <= 16; l++) {
            t->first[l] = (uint16_t)nsym;
            for (int k = 0; k < cnt[l]; k++) {
                uint8_t v = (uint8_t)rd_take(r, 8);
                if (pos + (1u << (16 - l)) > 0xffff) return OJ_ERR_DHT;
                t->sym[nsym++] = v;
                pos += 1u << (16 - l);
            }
            t->lim[l] = pos;
        }
        t->present = 1;
    }
    return OJ_OK;
}

/* One block: DC, then AC until end-of-block or position 63, dequantised
   into natural order (common/pjpeg.c:552-600). */
static void read_block(rd_t *r, const huff_t *dc, const huff_t *ac, const uint8_t *q, int32_t *pred,
                       int32_t blk[64]) {
    int nb, sym;
    memset(blk, 0, 64 * sizeof(int32_t));
    huff_lookup(dc, rd_peek(r, 16), &nb, &sym);
    rd_take(r, nb);
    int s = sym & 15;
    int32_t v = (int32_t)rd_take(r, s);
    if (s && !(v >> (s - 1))) v -= (1 << s) - 1;
    *pred += v;
    blk[0] = *pred * q[0];
    for (int k = 1; k < 64; k++) {
        huff_lookup(ac, rd_peek(r, 16), &nb, &sym);
        rd_take(r, nb);
        if (sym == 0) break;
        s = sym & 15;
        v = (int32_t)rd_take(r, s);
        if (s && !(v >> (s - 1))) v -= (1 << s) - 1;
        k += sym >> 4;
        if (k < 64) blk[ZIG[k]] = v * q[k];
    }
}

static int read_scan(dec_t *d, rd_t *r) {
    rd_take(r, 16);
    int ns = (int)rd_take(r, 8);
    int idx[256];
    for (int i = 0; i < ns; i++) {
        uint8_t id = (uint8_t)rd_take(r, 8);
        int found = -1;
        for (int j = 0; j < d->ncomp; j++)
            if (d->comp[j].id == id) { found = j; break; }
        if (found < 0) return OJ_ERR_SOS;
        d->comp[found].tda = (uint8_t)rd_take(r, 8);
        idx[i] = found;
    }
    uint8_t ss = (uint8_t)rd_take(r, 8), se = (uint8_t)rd_take(r, 8), a = (uint8_t)rd_take(r, 8);
    if (ss != 0 || se != 63 || a != 0) return OJ_ERR_SOS;
    int mw = 0, mh = 0;
    for (int i = 0; i < ns; i++) {
        oj_plane *c = &d->comp[idx[i]];
        if (c->scalex * 8 > mw) mw = c->scalex * 8;
        if (c->scaley * 8 > mh) mh = c->scaley * 8;
    }
    /* The reference divides by these (a zero sampling factor crashes it). */
    if (mw == 0 || mh == 0) return OJ_ERR_SOF;
    int mx = (int)((d->width + mw - 1) / mw), my = (int)((d->height + mh - 1) / mh);
    for (int i = 0; i < ns; i++) {
        oj_plane *c = &d->comp[idx[i]];
        c->width = (uint32_t)(mx * c->scalex * 8);
        c->height = (uint32_t)(my * c->scaley * 8);
        c->stride = (c->width + 31) / 32 * 32;
        free(c->data);
        c->data = (uint8_t *)calloc((size_t)c->height * c->stride + 1, 1);
        if (!c->data) return OJ_ERR_FILE;
    }
    int32_t pred[256] = {0};
    int count = 0;
    int32_t blk[64];
    for (int y = 0; y < my; y++) {
        for (int x = 0; x < mx; x++) {
            if (d->restart > 0 && count == d->restart) {
                rd_align(r);
                while (rd_take(r, 8) != 0xff) {}
                if (rd_take(r, 8) != 0xd0u + d->rst_next) return OJ_ERR_RESET;
                count = 0;
                d->rst_next = (d->rst_next + 1) & 7;
                pred[0] = 0; /* the reference zeroes the first predictor only */
            }
            for (int i = 0; i < ns; i++) {
                oj_plane *c = &d->comp[idx[i]];
                int hd = c->tda >> 4, ha = 2 + (c->tda & 15);
                for (int sy = 0; sy < c->scaley; sy++)
                    for (int sx = 0; sx < c->scalex; sx++) {
                        /* Table numbers past 3 index outside the reference's tables. */
                        if (hd > 3 || ha > 3 || !d->h[hd].present || !d->h[ha].present)
                            return OJ_ERR_MISSING_DHT;
                        read_block(r, &d->h[hd], &d->h[ha], d->q[c->tq], &pred[i], blk);
                        int64_t px = (int64_t)(x * c->scalex + sx) * 8, py = (int64_t)(y * c->scaley + sy) * 8;
                        idct_block(blk, c->data + py * c->stride + px, c->stride);
                    }
            }
            count++;
        }
    }
    return OJ_OK;
}

static int decode_into(dec_t *d, const uint8_t *buf, int64_t len) {
    rd_t r = {buf, 0, len, 0, 0};
    while (rd_more(&r)) {
        rd_align(&r);
        while (rd_take(&r, 8) != 0xff) {}
        uint8_t m = (uint8_t)rd_take(&r, 8);
        int e = OJ_OK;
        switch (m) {
        case 0xd8:
            break;
        case 0xdb: {
            int n = (int)rd_take(&r, 16);
            if ((n - 2) % 65 != 0) return OJ_ERR_DQT;
            for (int o = 0; o < n - 2; o += 65) {
                uint8_t pq = (uint8_t)rd_take(&r, 8);
                if ((pq & 0xf0) || (pq & 15) >= 4) return OJ_ERR_DQT;
                for (int k = 0; k < 64; k++) d->q[pq & 3][k] = (uint8_t)rd_take(&r, 8);
            }
            break;
        }
        case 0xc0: {
            rd_take(&r, 16);
            if (rd_take(&r, 8) != 8) return OJ_ERR_SOF;
            d->height = rd_take(&r, 16);
            d->width = rd_take(&r, 16);
            int nf = (int)rd_take(&r, 8);
            if (nf < 1 || nf > 3) return OJ_ERR_SOF;
            for (int i = 0; i < d->ncomp; i++) free(d->comp[i].data);
            memset(d->comp, 0, sizeof(d->comp));
            d->ncomp = nf;
            for (int i = 0; i < nf; i++) {
                oj_plane *c = &d->comp[i];
                c->id = (uint8_t)rd_take(&r, 8);
                c->hv = (uint8_t)rd_take(&r, 8);
                c->scalex = c->hv >> 4;
                c->scaley = c->hv & 15;
                c->tq = (uint8_t)rd_take(&r, 8);
                /* Table numbers past 3 index outside the reference's tables. */
                if (c->tq > 3) return OJ_ERR_SOF;
            }
            break;
        }
        case 0xc1: case 0xc2: case 0xc3: case 0xc5: case 0xc6: case 0xc7: case 0xc8:
        case 0xc9: case 0xca: case 0xcb: case 0xcd: case 0xce: case 0xcf:
            return OJ_ERR_UNSUPPORTED;
        case 0xc4:
            e = read_dht(d, &r);
            break;
        case 0xda:
            e = read_scan(d, &r);
            break;
        case 0xd9:
            return OJ_OK;
        case 0xdd:
            if (rd_take(&r, 16) != 4) return OJ_ERR_DRI;
            d->restart = (int)rd_take(&r, 16);
            break;
        default: { /* APPn, COM and anything unknown: skipped by length */
            int n = (int)rd_take(&r, 16);
            /* A length below 2 moves the reference's unsigned position past the end. */
            r.pos = n < 2 ? r.len : r.pos + (n - 2);
            break;
        }
        }
        if (e != OJ_OK) return e;
    }
    return OJ_OK;
}

int oj_decode(const uint8_t *buf, int64_t len, uint32_t flags, oj_image *out) {
    dec_t *d = (dec_t *)calloc(1, sizeof(dec_t));
    if (!d) return OJ_ERR_FILE;
    memset(out, 0, sizeof(*out));
    if (flags & OJ_MJPEG) {
        const uint8_t *bits[4] = {K_DC_L_BITS, K_DC_C_BITS, K_AC_L_BITS, K_AC_C_BITS};
        const uint8_t *vals[4] = {K_DC_VALS, K_DC_VALS, K_AC_L_VALS, K_AC_C_VALS};
        for (int t = 0; t < 4; t++) {
            huff_t *h = &d->h[t];
            uint32_t pos = 0;
            int nsym = 0;
            for (int l = 1; l <= 16; l++) {
                h->first[l] = (uint16_t)nsym;
                for (int k = 0; k < bits[t][l - 1]; k++, nsym++) {
                    h->sym[nsym] = vals[t][nsym];
                    pos += 1u << (16 - l);
                }
                h->lim[l] = pos;
            }
            h->present = 1;
        }
    }
    int e = decode_into(d, buf, len);
    if (e != OJ_OK) {
        for (int i = 0; i < 3; i++) free(d->comp[i].data);
        free(d);
        return e;
    }
    out->width = d->width;
    out->height = d->height;
    out->ncomponents = d->ncomp;
    memcpy(out->comp, d->comp, sizeof(d->comp));
    free(d);
    return OJ_OK;
}

void oj_free(oj_image *im) {
    for (int i = 0; i < 3; i++) free(im->comp[i].data);
    memset(im, 0, sizeof(*im));
}

int oj_gray(const oj_image *im, uint8_t *dst, int64_t stride) {
    const oj_plane *c = &im->comp[0];
    if (im->ncomponents < 1 || !c->data || c->width < im->width || c->height < im->height) return -1;
    for (uint32_t y = 0; y < im->height; y++) memcpy(dst + y * stride, c->data + (size_t)y * c->stride, im->width);
    return 0;
}
