/* CPU oracle of the AprilTag detection path. TEST INFRASTRUCTURE ONLY.

   A plain-C restatement of the reference detector's algorithm (bouk/
   apriltags-fast, the files under fast/), written for this project, used by the tests,
   smoke() and bench.py's CPU-baseline leg as the checker of the GPU
   library. It is never linked into, loaded by or called from the product.

   Order modes. The reference numbers its components by the root that its
   sequential union-by-size union-find happens to pick, and orders the
   clusters (and so the quads, and detections with equal ids) by a hash of
   those roots (fast/clusters.c:338-356). AO_ORDER_REF reproduces that
   exactly (byte-identical to the reference's goldens). AO_ORDER_CANON
   numbers each component by its smallest node index and orders clusters
   by (larger label, smaller label): the order the GPU library uses. Both
   modes give the same clusters, quads and detections; only the order of
   clusters (hence of quads and of detections that share an id) differs. */
#ifndef AT_ORACLE_H
#define AT_ORACLE_H

#include <stdbool.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same layout as the reference's at_family (fast/apriltag_fast.h:24-36). */
typedef struct ao_family {
    char name[32];
    const uint64_t *codes;
    int64_t ncodes;
    int32_t nbits;
    int32_t h;
    int32_t width_at_border;
    int32_t total_width;
    bool reversed_border;
    int32_t bit_x[64];
    int32_t bit_y[64];
} ao_family;

/* Same layout as the reference's at_detection (fast/apriltag_fast.h:52-64). */
typedef struct ao_detection {
    int32_t family, id, hamming;
    float decision_margin;
    double H[9];
    double c[2];
    double p[4][2];
} ao_detection;

/* The detector parameters (fast/apriltag_fast.h:40-96). */
typedef struct ao_params {
    float quad_decimate;
    float quad_sigma;
    int32_t refine_edges;
    double decode_sharpening;
    int32_t min_cluster_pixels;
    int32_t max_nmaxima;
    float cos_critical_rad;
    float max_line_fit_mse;
    int32_t min_white_black_diff;
    int32_t deglitch;
} ao_params;

enum { AO_ORDER_REF = 0, AO_ORDER_CANON = 1 };

/* A quad candidate as fit on the quad image (before corner scaling). */
typedef struct ao_quad {
    float p[4][2];
    int32_t reversed_border;
    int32_t cluster; /* index of the cluster it was fit to */
} ao_quad;

/* Everything one frame produced. Arrays are malloc'd; ao_result_free. */
typedef struct ao_result {
    int64_t qw, qh;
    uint8_t *qim;          /* quad image qw*qh (decimated, blurred) */
    uint8_t *thresh;       /* thresholded image qw*qh (0/127/255) */
    int64_t nruns;
    uint16_t *run_start, *run_end; /* nruns each */
    uint8_t *run_v;        /* nruns */
    uint32_t *row_off;     /* qh+1 */
    int64_t nnodes;        /* nruns + qh (virtual last-column nodes) */
    uint32_t *label;       /* nnodes: smallest node index of the component */
    uint32_t *ref_root;    /* nnodes: the reference union-find's root */
    uint32_t *comp_pixels; /* nnodes: pixels of the node's component */
    int64_t npoints;
    int64_t nclusters;
    uint32_t *cstart;      /* nclusters+1 offsets into pts */
    uint64_t *cid;         /* nclusters cluster ids (pair of labels of the mode) */
    uint64_t *pts;         /* npoints: x | y<<16 | gx<<32 | gy<<48 (u16 each) */
    int64_t nquads;
    ao_quad *quads;
    int64_t ndet;
    ao_detection *dets;
} ao_result;

/* Default parameters (fast/detector.c:8-20). */
void ao_default_params(ao_params *p);

/* Detect. fams/bits: nfam families with their bits_corrected (0..3).
   Returns 0, or -1 on bad arguments (as the reference's at_add_family
   refusal). */
int ao_detect(const ao_params *prm, const ao_family *fams, const int32_t *bits, int32_t nfam, const uint8_t *img,
              int64_t w, int64_t h, int64_t stride, int32_t order_mode, ao_result *res);
void ao_result_free(ao_result *res);

/* The sort order of fit_quad's angle keys (fast/quads.c:159-208): the
   reference's recursive merge sort with its leaf networks, restated. Used
   by the tests to check the GPU's characterisation on random keys. */
void ao_keysort(uint64_t *keys, int64_t n);

/* Correctly rounded f32 trig as the golden vectors need (double, then one
   rounding). Exposed for the tests of the GPU's versions. */
float ao_atan2f(float y, float x);
float ao_cosf(float x);
float ao_sinf(float x);

#ifdef __cplusplus
}
#endif
#endif
