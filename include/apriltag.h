/* The upstream AprilTag API (apriltag.h of bouk/apriltags-fast, which keeps
   the API of AprilRobotics apriltag 3) over the GPU detector of
   apriltag_fast.h. Same names, arguments and struct layouts as the
   reference's apriltag.h:57-300, so a program written against it builds
   unchanged and links -lapriltag_b200. The image is read in place (host or
   device memory). As in the reference, nedges/nsegments stay 0 and wp stays
   NULL, and the last three fields of apriltag_detector_t belong to the
   library. */
#pragma once

#include <pthread.h>
#include <stdbool.h>
#include <stdint.h>
#include <stdlib.h>

#include "common/image_u8.h"
#include "common/matd.h"
#include "common/timeprofile.h"
#include "common/workerpool.h"
#include "common/zarray.h"

#ifdef __cplusplus
extern "C" {
#endif

/* A tag family (apriltag.h:72-100). */
typedef struct apriltag_family apriltag_family_t;
struct apriltag_family {
    uint32_t ncodes;
    uint64_t *codes;
    int width_at_border;
    int total_width;
    bool reversed_border;
    uint32_t nbits;
    uint32_t *bit_x;
    uint32_t *bit_y;
    uint32_t h;
    char *name;
    void *impl; /* unused here */
};

/* Quad detection parameters (apriltag.h:103-133). */
struct apriltag_quad_thresh_params {
    int min_cluster_pixels;
    int max_nmaxima;
    float critical_rad;
    float cos_critical_rad;
    float max_line_fit_mse;
    int min_white_black_diff;
    int deglitch;
};

/* The detector (apriltag.h:138-210). */
struct at_detector;
typedef struct apriltag_detector apriltag_detector_t;
struct apriltag_detector {
    int nthreads;
    float quad_decimate;
    float quad_sigma;
    bool refine_edges;
    double decode_sharpening;
    bool debug;
    struct apriltag_quad_thresh_params qtp;
    timeprofile_t *tp;
    uint32_t nedges;
    uint32_t nsegments;
    uint32_t nquads;
    zarray_t *tag_families;
    workerpool_t *wp;
    pthread_mutex_t mutex;
    struct at_detector *fast;  /* the GPU detector */
    zarray_t *family_bits;     /* bits_corrected per entry of tag_families */
    bool families_changed;
};

/* A detection (apriltag.h:214-250). */
typedef struct apriltag_detection apriltag_detection_t;
struct apriltag_detection {
    apriltag_family_t *family;
    int id;
    int hamming;
    float decision_margin;
    matd_t *H;
    double c[2];
    double p[4][2];
};

/* apriltag.c:21-52: defaults nthreads 1, decimate 2, refine_edges, sharpening 0.25. */
apriltag_detector_t *apriltag_detector_create(void);
/* apriltag.c:85-90 */
void apriltag_detector_add_family_bits(apriltag_detector_t *td, apriltag_family_t *fam, int bits_corrected);
static inline void apriltag_detector_add_family(apriltag_detector_t *td, apriltag_family_t *fam) {
    apriltag_detector_add_family_bits(td, fam, 2);
}
/* apriltag.c:92-105 */
void apriltag_detector_remove_family(apriltag_detector_t *td, apriltag_family_t *fam);
/* apriltag.c:107-112 */
void apriltag_detector_clear_families(apriltag_detector_t *td);
/* apriltag.c:54-64 */
void apriltag_detector_destroy(apriltag_detector_t *td);
/* apriltag.c:152-208: a zarray of apriltag_detection_t *, sorted by id. */
zarray_t *apriltag_detector_detect(apriltag_detector_t *td, image_u8_t *im_orig);
/* Not in apriltag.c: n images through one batched pass on the GPU;
   results[i] gets image i's detections exactly as apriltag_detector_detect
   would return them (the caller destroys each with
   apriltag_detections_destroy). td->nquads is the batch's total and td->tp
   holds the batch's stage times. */
void apriltag_detector_detect_batch(apriltag_detector_t *td, image_u8_t **ims, int n, zarray_t **results);
/* apriltag.c:210-229 */
void apriltag_detection_destroy(apriltag_detection_t *det);
void apriltag_detections_destroy(zarray_t *detections);
/* apriltag.c:231-267 */
void apriltag_detection_copy(apriltag_detection_t *src, apriltag_detection_t *dst);
zarray_t *apriltag_detections_copy(zarray_t *detections);
/* apriltag.c:66-83: the parameters, no families. */
apriltag_detector_t *apriltag_detector_copy(apriltag_detector_t *src);
/* apriltag.c:269-297 */
image_u8_t *apriltag_to_image(apriltag_family_t *fam, uint32_t idx);

#ifdef __cplusplus
}
#endif
