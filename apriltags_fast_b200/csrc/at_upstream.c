/* The upstream AprilTag API (include/apriltag.h) over the native GPU
   detector (include/apriltag_fast.h). Follows apriltag.c of the reference:
   the parameters of apriltag_detector_t are copied into the native detector
   before each detection, the families are handed over again when they
   changed, and each native detection becomes a heap-allocated
   apriltag_detection_t with its own matd_t H. Also the small parts of the
   reference's common/ library that the API's callers use: matd_t, image_u8_t
   and the built-in families' create/destroy. */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "apriltag.h"
#include "apriltag_fast.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ---- matd_t (common/matd.c of the reference, the parts H needs) ---- */

matd_t *matd_create(int rows, int cols) {
    if (rows <= 0 || cols <= 0) return NULL;
    matd_t *m = (matd_t *)calloc(1, sizeof(matd_t));
    m->nrows = (unsigned)rows;
    m->ncols = (unsigned)cols;
    m->data = (double *)calloc((size_t)rows * cols, sizeof(double));
    return m;
}

matd_t *matd_create_data(int rows, int cols, const double *data) {
    matd_t *m = matd_create(rows, cols);
    if (m) memcpy(m->data, data, (size_t)rows * cols * sizeof(double));
    return m;
}

matd_t *matd_copy(const matd_t *m) {
    if (m == NULL) return NULL;
    return matd_create_data((int)m->nrows, (int)m->ncols, m->data);
}

void matd_destroy(matd_t *m) {
    if (m == NULL) return;
    free(m->data);
    free(m);
}

/* ---- image_u8_t (common/image_u8.c:40-120 of the reference) ---- */

image_u8_t *image_u8_create_stride(unsigned int width, unsigned int height, unsigned int stride) {
    uint8_t *buf = (uint8_t *)calloc((size_t)height * stride, 1);
    image_u8_t tmp = {.width = (int32_t)width, .height = (int32_t)height, .stride = (int32_t)stride, .buf = buf};
    image_u8_t *im = (image_u8_t *)calloc(1, sizeof(image_u8_t));
    memcpy(im, &tmp, sizeof tmp);
    return im;
}

image_u8_t *image_u8_create_alignment(unsigned int width, unsigned int height, unsigned int alignment) {
    unsigned int stride = width;
    if (alignment && stride % alignment) stride += alignment - stride % alignment;
    return image_u8_create_stride(width, height, stride);
}

image_u8_t *image_u8_create(unsigned int width, unsigned int height) {
    return image_u8_create_alignment(width, height, 96);
}

image_u8_t *image_u8_copy(const image_u8_t *in) {
    image_u8_t *im = image_u8_create_stride((unsigned)in->width, (unsigned)in->height, (unsigned)in->stride);
    memcpy(im->buf, in->buf, (size_t)in->height * in->stride);
    return im;
}

void image_u8_destroy(image_u8_t *im) {
    if (im == NULL) return;
    free(im->buf);
    free(im);
}

image_u8_t *image_u8_create_from_pnm(const char *path) {
    int64_t w = 0, h = 0;
    uint8_t *px = NULL;
    if (!at_read_pnm(path, &w, &h, &px)) return NULL;
    image_u8_t *im = image_u8_create((unsigned)w, (unsigned)h);
    for (int64_t y = 0; y < h; y++) memcpy(im->buf + y * im->stride, px + y * w, (size_t)w);
    free(px);
    return im;
}

int image_u8_write_pnm(const image_u8_t *im, const char *path) {
    uint8_t *px = (uint8_t *)malloc((size_t)im->width * im->height);
    for (int32_t y = 0; y < im->height; y++) memcpy(px + (size_t)y * im->width, im->buf + (size_t)y * im->stride, im->width);
    const bool ok = at_write_pgm(path, px, im->width, im->height);
    free(px);
    return ok ? 0 : -1;
}

/* ---- families ---- */

static bool family_to_native(const apriltag_family_t *src, at_family *dst) {
    if (src == NULL || src->nbits > 64) return false;
    memset(dst, 0, sizeof *dst);
    strncpy(dst->name, src->name ? src->name : "", sizeof dst->name - 1);
    dst->codes = src->codes;
    dst->ncodes = src->ncodes;
    dst->nbits = (int32_t)src->nbits;
    dst->h = (int32_t)src->h;
    dst->width_at_border = src->width_at_border;
    dst->total_width = src->total_width;
    dst->reversed_border = src->reversed_border;
    for (uint32_t i = 0; i < src->nbits; i++) {
        dst->bit_x[i] = (int32_t)src->bit_x[i];
        dst->bit_y[i] = (int32_t)src->bit_y[i];
    }
    return true;
}

static apriltag_family_t *family_from_native(const at_family *f) {
    if (f == NULL) return NULL;
    apriltag_family_t *tf = (apriltag_family_t *)calloc(1, sizeof *tf);
    tf->ncodes = (uint32_t)f->ncodes;
    tf->codes = (uint64_t *)f->codes; /* the library's static table */
    tf->width_at_border = f->width_at_border;
    tf->total_width = f->total_width;
    tf->reversed_border = f->reversed_border;
    tf->nbits = (uint32_t)f->nbits;
    tf->bit_x = (uint32_t *)calloc(f->nbits > 0 ? f->nbits : 1, sizeof(uint32_t));
    tf->bit_y = (uint32_t *)calloc(f->nbits > 0 ? f->nbits : 1, sizeof(uint32_t));
    for (int32_t i = 0; i < f->nbits; i++) {
        tf->bit_x[i] = (uint32_t)f->bit_x[i];
        tf->bit_y[i] = (uint32_t)f->bit_y[i];
    }
    tf->h = (uint32_t)f->h;
    tf->name = strdup(f->name);
    return tf;
}

static void family_free(apriltag_family_t *tf) {
    if (tf == NULL) return;
    free(tf->bit_x);
    free(tf->bit_y);
    free(tf->name);
    free(tf);
}

#define FAMILY(n)                                                         \
    apriltag_family_t *n##_create(void) { return family_from_native(at_##n()); } \
    void n##_destroy(apriltag_family_t *tf) { family_free(tf); }
FAMILY(tag16h5)
FAMILY(tag25h9)
FAMILY(tag36h10)
FAMILY(tag36h11)
FAMILY(tagCircle21h7)
FAMILY(tagCircle49h12)
FAMILY(tagCustom48h12)
FAMILY(tagStandard41h12)
FAMILY(tagStandard52h13)

/* ---- the detector (apriltag.c:21-208 of the reference) ---- */

apriltag_detector_t *apriltag_detector_create(void) {
    apriltag_detector_t *td = (apriltag_detector_t *)calloc(1, sizeof(apriltag_detector_t));
    td->nthreads = 1;
    td->quad_decimate = 2.0f;
    td->quad_sigma = 0.0f;
    td->qtp.max_nmaxima = 10;
    td->qtp.min_cluster_pixels = 24;
    td->qtp.max_line_fit_mse = 10.0f;
    td->qtp.cos_critical_rad = (float)cos(10 * M_PI / 180);
    td->qtp.deglitch = 0;
    td->qtp.min_white_black_diff = 5;
    td->tag_families = zarray_create(sizeof(apriltag_family_t *));
    td->family_bits = zarray_create(sizeof(int));
    pthread_mutex_init(&td->mutex, NULL);
    td->tp = timeprofile_create();
    td->refine_edges = true;
    td->decode_sharpening = 0.25;
    td->debug = false;
    td->fast = at_detector_create();
    return td;
}

void apriltag_detector_destroy(apriltag_detector_t *td) {
    if (td == NULL) return;
    at_detector_destroy(td->fast);
    timeprofile_destroy(td->tp);
    zarray_destroy(td->tag_families);
    zarray_destroy(td->family_bits);
    pthread_mutex_destroy(&td->mutex);
    free(td);
}

apriltag_detector_t *apriltag_detector_copy(apriltag_detector_t *src) {
    apriltag_detector_t *dst = (apriltag_detector_t *)malloc(sizeof(apriltag_detector_t));
    *dst = *src;
    dst->tag_families = zarray_create(sizeof(apriltag_family_t *));
    dst->family_bits = zarray_create(sizeof(int));
    dst->tp = timeprofile_create();
    dst->wp = NULL;
    pthread_mutex_init(&dst->mutex, NULL);
    dst->fast = at_detector_create();
    dst->families_changed = false;
    return dst;
}

void apriltag_detector_add_family_bits(apriltag_detector_t *td, apriltag_family_t *fam, int bits_corrected) {
    zarray_add(td->tag_families, &fam);
    zarray_add(td->family_bits, &bits_corrected);
    td->families_changed = true;
}

void apriltag_detector_remove_family(apriltag_detector_t *td, apriltag_family_t *fam) {
    for (int i = 0; i < zarray_size(td->tag_families); i++) {
        apriltag_family_t *f;
        zarray_get(td->tag_families, i, &f);
        if (f == fam) {
            zarray_remove_index(td->tag_families, i, 0);
            zarray_remove_index(td->family_bits, i, 0);
            td->families_changed = true;
            return;
        }
    }
}

void apriltag_detector_clear_families(apriltag_detector_t *td) {
    zarray_clear(td->tag_families);
    zarray_clear(td->family_bits);
    td->families_changed = true;
}

/* Contract of the family list: after any add/remove/clear, the next
   detection hands the upstream list to the native detector in list order,
   and a detection's `family` is the list entry at its native index. So an
   entry that the native detector refuses (bits_corrected out of range, a
   17th family, a table it cannot hold) must leave the upstream list too;
   the caller learns of it on stderr. */
static void sync_families(apriltag_detector_t *td) {
    const int n = zarray_size(td->tag_families);
    apriltag_family_t **fams = (apriltag_family_t **)malloc(sizeof(apriltag_family_t *) * (n > 0 ? n : 1));
    int *bits = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
    int kept = 0;
    at_clear_families(td->fast);
    for (int i = 0; i < n; i++) {
        zarray_get(td->tag_families, i, &fams[kept]);
        zarray_get(td->family_bits, i, &bits[kept]);
        at_family native;
        const bool taken = family_to_native(fams[kept], &native) && at_add_family(td->fast, &native, bits[kept]);
        if (taken) {
            kept++;
        } else {
            const char *nm = fams[kept] != NULL && fams[kept]->name != NULL ? fams[kept]->name : "(unnamed)";
            fprintf(stderr, "apriltag_b200: the GPU detector refused family %s at %d corrected bits; it is no "
                            "longer in the detector's list\n", nm, bits[kept]);
        }
    }
    zarray_clear(td->tag_families);
    zarray_clear(td->family_bits);
    for (int i = 0; i < kept; i++) {
        zarray_add(td->tag_families, &fams[i]);
        zarray_add(td->family_bits, &bits[i]);
    }
    free(fams);
    free(bits);
    td->families_changed = false;
}

/* td->tp after a detection: a stamp at the end of each stage, at the
   detection's start time plus the stage times so far (the GPU's event
   times). The stage names are the ones upstream users see in
   timeprofile_display. */
static const struct {
    const char *name;
    size_t field; /* offset of the stage's seconds in at_timing; SIZE_MAX: none */
} kStages[] = {
    {"init", (size_t)-1},
    {"decimate", offsetof(at_timing, decimate)},
    {"blur/sharp", offsetof(at_timing, blur)},
    {"threshold", offsetof(at_timing, threshold)},
    {"unionfind", offsetof(at_timing, unionfind)},
    {"make clusters", offsetof(at_timing, clusters)},
    {"fit quads to clusters", offsetof(at_timing, fit_quads)},
    {"decode+refinement", offsetof(at_timing, decode)},
    {"reconcile", offsetof(at_timing, reconcile)},
};

static void stamp_stages(timeprofile_t *tp, const at_timing *t) {
    const int64_t t0 = tp->utime;
    double elapsed = 0.0;
    zarray_clear(tp->stamps);
    tp->utime = t0;
    for (size_t k = 0; k < sizeof kStages / sizeof kStages[0]; k++) {
        if (kStages[k].field != (size_t)-1) elapsed += *(const double *)((const char *)t + kStages[k].field);
        struct timeprofile_entry e = {{0}, t0 + (int64_t)(elapsed * 1e6)};
        snprintf(e.name, sizeof e.name, "%s", kStages[k].name);
        zarray_add(tp->stamps, &e);
    }
}

/* The detector's parameters as the native detector takes them. */
static void push_params(apriltag_detector_t *td) {
    at_detector *fd = td->fast;
    fd->nthreads = td->nthreads > 0 ? td->nthreads : 1;
    fd->quad_decimate = td->quad_decimate;
    fd->quad_sigma = td->quad_sigma;
    fd->refine_edges = td->refine_edges;
    fd->decode_sharpening = td->decode_sharpening;
    fd->debug = td->debug;
    fd->qtp.min_cluster_pixels = td->qtp.min_cluster_pixels;
    fd->qtp.max_nmaxima = td->qtp.max_nmaxima;
    fd->qtp.critical_rad = td->qtp.critical_rad;
    fd->qtp.cos_critical_rad = td->qtp.cos_critical_rad;
    fd->qtp.max_line_fit_mse = td->qtp.max_line_fit_mse;
    fd->qtp.min_white_black_diff = td->qtp.min_white_black_diff;
    fd->qtp.deglitch = td->qtp.deglitch != 0;
}

/* Native detections [first, first + count) as upstream detections: each
   its own allocation, its H a 3x3 matd, its family the detector's. */
static zarray_t *to_upstream(apriltag_detector_t *td, const at_detection *dets, int64_t count) {
    zarray_t *out = zarray_create(sizeof(apriltag_detection_t *));
    zarray_ensure_capacity(out, (int)count);
    for (int64_t i = 0; i < count; i++) {
        const at_detection *d = &dets[i];
        apriltag_detection_t *det = (apriltag_detection_t *)calloc(1, sizeof(apriltag_detection_t));
        zarray_get(td->tag_families, d->family, &det->family);
        det->id = d->id;
        det->hamming = d->hamming;
        det->decision_margin = d->decision_margin;
        det->H = matd_create_data(3, 3, d->H);
        det->c[0] = d->c[0];
        det->c[1] = d->c[1];
        memcpy(det->p, d->p, sizeof det->p);
        zarray_add(out, &det);
    }
    return out;
}

zarray_t *apriltag_detector_detect(apriltag_detector_t *td, image_u8_t *im_orig) {
    if (zarray_size(td->tag_families) == 0 || im_orig->width < 8 || im_orig->height < 8)
        return zarray_create(sizeof(apriltag_detection_t *));
    if (td->families_changed) sync_families(td);
    push_params(td);
    at_detector *fd = td->fast;
    td->tp->utime = utime_now();
    at_detect(fd, im_orig->buf, im_orig->width, im_orig->height, im_orig->stride);
    stamp_stages(td->tp, &fd->timing);
    td->nquads = (uint32_t)fd->nquads;
    td->nedges = 0;
    td->nsegments = 0;
    return to_upstream(td, fd->detections, fd->ndetections);
}

void apriltag_detector_detect_batch(apriltag_detector_t *td, image_u8_t **ims, int n, zarray_t **results) {
    if (n <= 0) return;
    if (zarray_size(td->tag_families) == 0) {
        for (int i = 0; i < n; i++) results[i] = zarray_create(sizeof(apriltag_detection_t *));
        return;
    }
    if (td->families_changed) sync_families(td);
    push_params(td);
    at_detector *fd = td->fast;
    at_frame *frames = (at_frame *)calloc((size_t)n, sizeof(at_frame));
    at_frame_result *res = (at_frame_result *)calloc((size_t)n, sizeof(at_frame_result));
    for (int i = 0; i < n; i++) {
        /* a frame under 8 px a side is given no detections, as by the
           single-frame call */
        const int small = ims[i]->width < 8 || ims[i]->height < 8;
        frames[i].pixels = ims[i]->buf;
        frames[i].width = small ? 0 : ims[i]->width;
        frames[i].height = small ? 0 : ims[i]->height;
        frames[i].stride = ims[i]->stride;
        frames[i].family_mask = 0;
    }
    td->tp->utime = utime_now();
    at_detect_batch(fd, frames, n, res);
    stamp_stages(td->tp, &fd->timing);
    uint64_t nq = 0;
    for (int i = 0; i < n; i++) {
        results[i] = to_upstream(td, fd->detections + res[i].first, res[i].count);
        nq += (uint64_t)res[i].nquads;
    }
    td->nquads = (uint32_t)nq;
    td->nedges = 0;
    td->nsegments = 0;
    free(frames);
    free(res);
}

void apriltag_detection_destroy(apriltag_detection_t *det) {
    if (det == NULL) return;
    matd_destroy(det->H);
    free(det);
}

void apriltag_detections_destroy(zarray_t *detections) {
    for (int i = 0; i < zarray_size(detections); i++) {
        apriltag_detection_t *det;
        zarray_get(detections, i, &det);
        apriltag_detection_destroy(det);
    }
    zarray_destroy(detections);
}

/* Deep copies: the copy owns its own H (a new matd_t); the family pointer
   is shared, as families are owned by the caller. */
void apriltag_detection_copy(apriltag_detection_t *src, apriltag_detection_t *dst) {
    matd_t *old = dst->H;
    *dst = *src;
    dst->H = matd_copy(src->H);
    matd_destroy(old);
}

zarray_t *apriltag_detections_copy(zarray_t *detections) {
    const int n = zarray_size(detections);
    zarray_t *out = zarray_create(sizeof(apriltag_detection_t *));
    zarray_ensure_capacity(out, n);
    for (int i = 0; i < n; i++) {
        apriltag_detection_t *src = NULL;
        zarray_get(detections, i, &src);
        apriltag_detection_t *dup = (apriltag_detection_t *)malloc(sizeof *dup);
        *dup = *src;
        dup->H = matd_copy(src->H);
        zarray_add(out, &dup);
    }
    return out;
}

/* One pixel per module of a tag of `fam` with code index idx: 0 (black)
   everywhere except a white square ring of side w centred in the
   total_width grid (w = width_at_border + 2 for a normal border, the
   border width itself for a reversed one: the white module ring just
   inside a reversed border, just outside the black border of a normal
   one), and the code's bits, most significant first, at (bit_x, bit_y)
   relative to the border's corner. NULL for a bad index. */
image_u8_t *apriltag_to_image(apriltag_family_t *fam, uint32_t idx) {
    if (fam == NULL || idx >= fam->ncodes) return NULL;
    const int tw = fam->total_width;
    const int w = fam->width_at_border + (fam->reversed_border ? 0 : 2);
    const int lo = (tw - w) / 2, hi = tw - 1 - lo;  /* ring rows/columns */
    const int bs = (tw - fam->width_at_border) / 2; /* border corner */
    image_u8_t *im = image_u8_create((unsigned)tw, (unsigned)tw);
    for (int y = 0; y < tw; y++)
        for (int x = 0; x < tw; x++) {
            const bool inside = x >= lo && x <= hi && y >= lo && y <= hi;
            const bool edge = x == lo || x == hi || y == lo || y == hi;
            if (inside && edge) im->buf[y * im->stride + x] = 255;
        }
    for (uint32_t b = 0; b < fam->nbits; b++) {
        const uint32_t bit = fam->nbits - 1 - b; /* bit b of the code, counted from the top */
        if ((fam->codes[idx] >> bit) & 1u) im->buf[(fam->bit_y[b] + bs) * im->stride + fam->bit_x[b] + bs] = 255;
    }
    return im;
}
