/* Runs one image through the upstream API (apriltag.h) and through the
   native API (apriltag_fast.h) of the library and prints both detection
   lists in the same exact (%a) form, one line per detection, so that the
   GPU test can compare them; also exercises detections_copy, the family
   create/destroy pair, remove/clear families, apriltag_to_image, the batch
   call (the image three times and a crop too small to hold a tag) and a
   page-locked image buffer.
   usage: upstream_detect image.pgm family bits */
#include <stdio.h>
#include <string.h>

#include "apriltag.h"
#include "apriltag_fast.h"
#include "tag16h5.h"
#include "tag25h9.h"
#include "tag36h11.h"
#include "tagStandard41h12.h"

static apriltag_family_t *make_family(const char *name) {
    if (!strcmp(name, "tag36h11")) return tag36h11_create();
    if (!strcmp(name, "tag25h9")) return tag25h9_create();
    if (!strcmp(name, "tag16h5")) return tag16h5_create();
    if (!strcmp(name, "tagStandard41h12")) return tagStandard41h12_create();
    return NULL;
}

static void print_det(const char *tag, int id, int hamming, float margin, const double *H, const double *c,
                      const double (*p)[2]) {
    printf("%s %d %d %a", tag, id, hamming, (double)margin);
    for (int i = 0; i < 9; i++) printf(" %a", H[i]);
    printf(" %a %a", c[0], c[1]);
    for (int i = 0; i < 4; i++) printf(" %a %a", p[i][0], p[i][1]);
    printf("\n");
}

int main(int argc, char **argv) {
    if (argc < 4) return 2;
    const int bits = atoi(argv[3]);
    image_u8_t *im = image_u8_create_from_pnm(argv[1]);
    apriltag_family_t *fam = make_family(argv[2]);
    if (im == NULL || fam == NULL) return 3;

    apriltag_detector_t *td = apriltag_detector_create();
    apriltag_family_t *other = tag16h5_create();
    apriltag_detector_add_family_bits(td, other, 1);
    apriltag_detector_remove_family(td, other);
    apriltag_detector_add_family_bits(td, fam, bits);
    zarray_t *dets = apriltag_detector_detect(td, im);
    zarray_t *copy = apriltag_detections_copy(dets);
    for (int i = 0; i < zarray_size(copy); i++) {
        apriltag_detection_t *d;
        zarray_get(copy, i, &d);
        if (d->family != fam || d->H->nrows != 3 || d->H->ncols != 3) return 4;
        print_det("U", d->id, d->hamming, d->decision_margin, d->H->data, d->c, (const double (*)[2])d->p);
    }
    printf("nquads %u stamps %d\n", td->nquads, zarray_size(td->tp->stamps));
    /* the same image three times and a 4x4 crop through the batch call */
    image_u8_t tiny = {4, 4, im->stride, im->buf};
    image_u8_t *batch[4] = {im, &tiny, im, im};
    zarray_t *bres[4];
    apriltag_detector_detect_batch(td, batch, 4, bres);
    for (int k = 0; k < 4; k++) {
        for (int i = 0; i < zarray_size(bres[k]); i++) {
            apriltag_detection_t *d;
            zarray_get(bres[k], i, &d);
            char tag[8];
            snprintf(tag, sizeof tag, "B%d", k);
            print_det(tag, d->id, d->hamming, d->decision_margin, d->H->data, d->c, (const double (*)[2])d->p);
        }
        apriltag_detections_destroy(bres[k]);
    }
    printf("batch nquads %u\n", td->nquads);
    apriltag_detections_destroy(copy);
    apriltag_detections_destroy(dets);
    apriltag_detector_clear_families(td);
    zarray_t *none = apriltag_detector_detect(td, im);
    printf("after clear %d\n", zarray_size(none));
    apriltag_detections_destroy(none);

    at_detector *fd = at_detector_create();
    at_add_family(fd, at_family_by_name(argv[2]), bits);
    at_detect(fd, im->buf, im->width, im->height, im->stride);
    for (int64_t i = 0; i < fd->ndetections; i++) {
        const at_detection *d = &fd->detections[i];
        print_det("N", d->id, d->hamming, d->decision_margin, d->H, d->c, d->p);
    }
    printf("native nquads %lld\n", (long long)fd->nquads);
    /* the image's buffer page-locked: the same detections */
    const int reg = at_register_host_buffer(im->buf, (size_t)im->stride * im->height);
    at_detect(fd, im->buf, im->width, im->height, im->stride);
    for (int64_t i = 0; i < fd->ndetections; i++) {
        const at_detection *d = &fd->detections[i];
        print_det("R", d->id, d->hamming, d->decision_margin, d->H, d->c, d->p);
    }
    printf("registered %d unregistered %d\n", reg, at_unregister_host_buffer(im->buf));

    image_u8_t *tagim = apriltag_to_image(fam, 0);
    printf("tag image %d %d\n", tagim->width, tagim->height);
    image_u8_destroy(tagim);
    at_detector_destroy(fd);
    apriltag_detector_destroy(td);
    tag16h5_destroy(other);
    tag36h11_destroy(fam == NULL ? NULL : (strcmp(argv[2], "tag36h11") ? NULL : fam));
    image_u8_destroy(im);
    return 0;
}
