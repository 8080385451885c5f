/* apriltags-b200: the native C API of the GPU AprilTag detector.

   A drop-in for the native API of bouk/apriltags-fast
   (fast/apriltag_fast.h:99-141): the same function names, arguments and
   struct layouts (at_detection is 168 bytes, at_detector 160 bytes, at_family
   584 bytes; checked with offsetof in the tests), so code written against
   that header links against libapriltag_b200.so unchanged:

       at_detector *td = at_detector_create();
       at_add_family(td, at_tag36h11(), 2);
       at_detect(td, pixels, width, height, stride);
       for (int64_t i = 0; i < td->ndetections; i++) use(td->detections[i]);
       at_detector_destroy(td);

   Every stage of at_detect runs as sm_100a CUDA kernels on the current
   device; there is no CPU path. The detections are bit-identical to the
   reference built with -ffp-contract=off, in the reference's order (same-id
   detections too: the order its union-find roots give their quads). See
   at_detector_last_error below for the error model. */
#ifndef APRILTAG_FAST_H
#define APRILTAG_FAST_H

#include <stdbool.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* A tag family (fast/apriltag_fast.h:24-36). `codes` stays owned by the
   caller (or is static for the built-in families). */
typedef struct at_family {
    char name[32];
    const uint64_t *codes;
    int64_t ncodes;
    int32_t nbits;
    int32_t h;
    int32_t width_at_border;
    int32_t total_width;
    bool reversed_border;
    int32_t bit_x[64]; /* bit positions in tag coordinates, MSB first */
    int32_t bit_y[64];
} at_family;

/* Quad detection parameters (fast/apriltag_fast.h:40-48). */
typedef struct at_quad_thresh_params {
    int32_t min_cluster_pixels;   /* default 24 */
    int32_t max_nmaxima;          /* default 10 */
    float critical_rad;           /* unused, kept for the layout */
    float cos_critical_rad;       /* default (float)cos(10 degrees) */
    float max_line_fit_mse;       /* default 10 */
    int32_t min_white_black_diff; /* default 5 */
    bool deglitch;                /* default false */
} at_quad_thresh_params;

/* One detection (fast/apriltag_fast.h:52-64). `family` indexes the
   detector's families in the order they were added. H maps tag coordinates
   in [-1, 1] to pixels (row major); p holds the corners counter-clockwise
   from tag coordinate (-1, -1). */
typedef struct at_detection {
    int32_t family;
    int32_t id;
    int32_t hamming;
    float decision_margin;
    double H[9];
    double c[2];
    double p[4][2];
} at_detection;

/* Seconds spent per stage in the last at_detect (fast/apriltag_fast.h:67-69),
   measured with CUDA events around each stage's kernels. */
typedef struct at_timing {
    double decimate, blur, threshold, unionfind, clusters, fit_quads, decode, reconcile, total;
} at_timing;

struct at_internal;

/* The detector (fast/apriltag_fast.h:73-96). nthreads is accepted and
   ignored: the results do not depend on it. */
typedef struct at_detector {
    int32_t nthreads;
    float quad_decimate;   /* 1.5, or an integer factor; default 2 */
    float quad_sigma;      /* blur (>0) or sharpen (<0) of the quad image */
    bool refine_edges;     /* default true */
    double decode_sharpening; /* default 0.25 */
    bool debug;            /* writes debug_preprocess.pnm / debug_threshold.pnm */
    at_quad_thresh_params qtp;

    at_detection *detections; /* valid until the next at_detect */
    int64_t ndetections;
    int64_t nquads;
    at_timing timing;

    struct at_internal *in;
} at_detector;

/* Replaces at_detector_create (fast/detector.c:4-31): default parameters,
   no families. Aborts if no CUDA device can be used. */
at_detector *at_detector_create(void);
/* Replaces at_detector_destroy (fast/detector.c:35-43). */
void at_detector_destroy(at_detector *td);
/* Replaces at_add_family (fast/detector.c:45-54): false for
   bits_corrected outside 0..3, a 17th family, ncodes >= 65536 or nbits
   outside 1..64. The decode tables are built once and kept on the device. */
bool at_add_family(at_detector *td, const at_family *fam, int bits_corrected);
/* Replaces at_clear_families (fast/detector.c:56-60). */
void at_clear_families(at_detector *td);
/* Replaces at_family_name (fast/detector.c:62-64). */
const char *at_family_name(const at_detector *td, const at_detection *d);
/* Replaces at_detect (fast/detector.c:246-335). pixels is host memory
   (pageable or pinned) or device memory; it is never written. */
void at_detect(at_detector *td, const uint8_t *pixels, int64_t width, int64_t height, int64_t stride);
/* Replaces at_shutdown (fast/detector.c:33): releases the detector's
   device arenas (and those of its batch helper detectors); the next
   at_detect allocates them again. */
void at_shutdown(at_detector *td);

/* The built-in families (fast/families.c:44-78): the AprilTag code
   tables, built into the library. */
const at_family *at_tag16h5(void);
const at_family *at_tag25h9(void);
const at_family *at_tag36h10(void);
const at_family *at_tag36h11(void);
const at_family *at_tagCircle21h7(void);
const at_family *at_tagCircle49h12(void);
const at_family *at_tagCustom48h12(void);
const at_family *at_tagStandard41h12(void);
const at_family *at_tagStandard52h13(void);
/* Replaces at_family_by_name (fast/families.c:64-68). */
const at_family *at_family_by_name(const char *name);

/* PNM files (fast/image.c:204-266): same behaviour as the reference. */
bool at_read_pnm(const char *path, int64_t *width, int64_t *height, uint8_t **pixels);
bool at_read_pnm_into(const char *path, int64_t *width, int64_t *height, uint8_t **pixels, int64_t *cap);
bool at_write_pgm(const char *path, const uint8_t *pixels, int64_t width, int64_t height);

/* ---------------------------------------------------------------------
   Additions of the GPU library (no counterpart in the reference). */

/* The last error of the detector: 0 for none. A failed CUDA call or a
   device-side check (a buffer bound, a bounded wait) makes at_detect return
   no detections and sets this; the message is kept until the next call. */
int at_detector_last_error(const at_detector *td, const char **message);

/* One frame of a batch. */
typedef struct at_frame {
    const uint8_t *pixels; /* host or device memory */
    int64_t width, height, stride;
    uint32_t family_mask;  /* bit i: decode with family i (0: all) */
} at_frame;

/* The result of one frame of a batch: detections [first, first + count)
   of td->detections, and that frame's quad count. */
typedef struct at_frame_result {
    int64_t first, count, nquads;
} at_frame_result;

/* Detect tags in n frames of any sizes in one pass over the GPU: each
   stage runs once for all frames. results[i] is what at_detect would give
   for frame i alone (bit-identical). td->detections holds all frames'
   detections, frame by frame; td->ndetections their total. */
void at_detect_batch(at_detector *td, const at_frame *frames, int64_t n, at_frame_result *results);

/* Page-locks a caller's host buffer for the GPU (cudaHostRegister): frames
   in it are then copied to the device by DMA straight from it, instead of
   through the driver's staging of pageable memory. Returns 0, or -1 when
   the buffer cannot be registered (it is then used as before). A buffer
   stays registered until at_unregister_host_buffer, which must come before
   the buffer is freed. */
int at_register_host_buffer(void *ptr, size_t bytes);
int at_unregister_host_buffer(void *ptr);

/* How many pipelines at_detect_batch spreads a large batch over (1 to 4;
   3 by default). Each pipeline takes a run of consecutive frames (at least
   10, with about equal pixel counts): the first runs on this detector, the
   others on helper detectors made like it (their own streams and device
   arenas, created at first use), each driven by its own host thread, so
   that their host synchronisations and latency-bound kernels overlap on the
   GPU. Results do not depend on the setting; at_timing and the diagnostics
   describe the first pipeline's part. Returns -1 for a value out of range. */
int at_detector_set_batch_split(at_detector *td, int pipelines);

/* Serving (no counterpart in the reference, which detects one frame per
   call). A server owns `workers` detectors made from `params` (its
   parameters and families at creation), each with its own stream and
   device arenas, and one thread each. Submitted frames queue oldest first;
   a free worker takes every queued frame, up to max_batch frames and its
   share (memory_budget / workers) of device memory at the learned bytes
   per pixel, and detects them as one batch, so frames that arrive while a
   batch is on the GPU are admitted to the next one and overlap it. A frame
   is rejected when it alone exceeds a worker's share, or when the device
   bytes of all pending and running frames with it would exceed the
   budget (bytes are estimated per input pixel from the batches so far, so
   a flood of requests is turned away instead of queued). Each frame's
   detections equal at_detect's for that frame alone. The pixels must stay
   valid and unchanged until the frame's result has been polled. */
typedef struct at_server at_server;
typedef struct at_server_config {
    int32_t workers;       /* concurrent batches (default 2) */
    int32_t max_batch;     /* frames per batch (default 16) */
    int64_t memory_budget; /* device bytes for all workers' frames (default 24 GiB) */
    uint32_t device_mask;  /* bit d: workers on GPU d, dealt out in turn (0: the current GPU) */
} at_server_config;
#define AT_SERVER_CANCELLED (-1) /* at_server_result.status of a cancelled request */
typedef struct at_server_result {
    uint64_t ticket, user;   /* from at_server_submit */
    int32_t status;          /* 0, AT_SERVER_CANCELLED, or the worker detector's at_detector_last_error */
    int32_t batch_frames;    /* frames in the batch it ran in */
    int32_t worker;
    int32_t pad;
    int64_t ndetections, nquads;
    at_detection *detections; /* owned by the result: at_server_free_result */
    double t_submit, t_start, t_done; /* seconds, steady clock */
} at_server_result;
typedef struct at_server_stats {
    int64_t admitted, rejected, completed, batches, in_flight, pending, cancelled;
    int64_t peak_arena_bytes; /* the largest worker arena seen */
    double bytes_per_pixel;   /* the admission estimate in use */
} at_server_stats;
at_server *at_server_create(const at_detector *params, const at_server_config *cfg);
/* Returns the request's ticket, or 0 when the frame is invalid or rejected. */
uint64_t at_server_submit(at_server *s, const at_frame *frame, uint64_t user);
/* Cancels a request that is still queued: it leaves the queue, and its
   result (status AT_SERVER_CANCELLED, no detections) is delivered by
   at_server_poll. Returns 1, or 0 when the ticket is unknown or its frame
   is already on the GPU or done (it then completes normally). */
int at_server_cancel(at_server *s, uint64_t ticket);
/* Copies up to max finished results (waiting up to wait_ms for the first);
   returns how many. */
int64_t at_server_poll(at_server *s, at_server_result *out, int64_t max, int32_t wait_ms);
void at_server_free_result(at_server_result *r);
void at_server_get_stats(at_server *s, at_server_stats *out);
/* The GPU that worker w runs on (at_server_result.worker), or -1. */
int at_server_worker_device(const at_server *s, int32_t worker);
/* Finishes the queued frames, stops the workers, frees everything. */
void at_server_destroy(at_server *s);

/* Diagnostics: copy an intermediate array of the last at_detect (or of
   frame 0 of the last batch) to host memory `dst` of `cap` bytes. Returns
   the array's size in bytes (copying min(size, cap)), or -1. `what`:
     AT_DIAG_QUAD_IMAGE  u8 qw*qh, the decimated (blurred) image
     AT_DIAG_THRESHOLD   u8 qw*qh, 0 / 127 / 255
     AT_DIAG_LABELS      u32 qw*qh, each pixel's component label (its
                         smallest union-find node id) or 0xffffffff
     AT_DIAG_POINTS      u64 per boundary point in cluster order:
                         x | y<<16 | gx<<32 | gy<<48
     AT_DIAG_CLUSTERS    u32 per cluster, the index of its first point
     AT_DIAG_QUADS       per fitted quad: 8 f32 corners (quad image
                         coordinates) then i32 reversed_border, i32 frame
     AT_DIAG_SIZES       i64 qw, qh, points, clusters, quads, and the number
                         of this library's kernels launched so far
     AT_DIAG_ORDER_ROOTS u32 pairs, one per component next to a quad whose
                         detection shares its id with another: the
                         component's smallest node and the root that the
                         reference's union order leaves it, both numbered
                         as the reference packs its union-find nodes */
enum {
    AT_DIAG_QUAD_IMAGE = 0,
    AT_DIAG_THRESHOLD = 1,
    AT_DIAG_LABELS = 2,
    AT_DIAG_POINTS = 3,
    AT_DIAG_CLUSTERS = 4,
    AT_DIAG_QUADS = 5,
    AT_DIAG_SIZES = 6,
    AT_DIAG_ORDER_ROOTS = 7
};
int64_t at_detector_diag(const at_detector *td, int what, void *dst, int64_t cap);

/* Tag poses of all detections of the last at_detect / at_detect_batch, in
   one launch on the GPU (a thread per detection): what the reference's
   estimate_tag_pose_orthogonal_iteration gives with 50 iterations for each
   detection (apriltag_pose.c:490-547), camera intrinsics fx, fy, cx, cy in
   pixels and the tag's side in metres: the refined pose (R row-major, t)
   and its object-space error, and the second local minimum (err2 HUGE_VAL
   when there is none; estimate_tag_pose picks the smaller error). out[i]
   belongs to td->detections[i]. Returns 0, 1 for bad arguments, 2 for a
   CUDA error. No counterpart in the native API of the reference. */
typedef struct at_pose {
    double R[9], t[3], err;
    double R2[9], t2[3], err2;
} at_pose;
int at_estimate_poses(const at_detector *td, double tagsize, double fx, double fy, double cx, double cy,
                      at_pose *out);

/* The threshold stage without any device allocation (it has no counterpart
   in the reference). For callers that cannot call cudaMalloc: a frame loop
   whose latency must not include the device-wide synchronisation that
   cudaMalloc/cudaFree imply, or a process whose device memory is all owned
   by one pool or framework that hands it only buffers. `image` (width x
   height u8, rows width bytes apart) and `out` (same size) are device
   memory of the caller; `stream` is a cudaStream_t (NULL: the default
   stream). The result equals the threshold image of at_detect for a quad
   image `image` (0 / 127 / 255, min_white_black_diff as qtp).
   The only scratch is a fixed 2 MiB array of the library that each GPU
   holds from the first call until the process exits: images above 1 Mi
   4x4 tiles (e.g. 4096 x 4096) are refused, as are images below one tile.
   The first call on a device finds that array's device address (once per
   device) and keeps it for the life of the process: make that first call
   before any stream capture, and do not call it again on a device after
   cudaDeviceReset there (the array may then live at another address). Every call
   shares the array: calls that overlap on the GPU race. Returns 0, 1 for
   a refused size, 2 for a CUDA error (message on stderr). */
int at_threshold_noalloc(const uint8_t *image, int64_t width, int64_t height, int32_t min_white_black_diff,
                         uint8_t *out, void *stream);

/* ---- JPEG input: baseline JPEG decoded on the GPU into 8-bit frames ----
   The pixels are those of the reference's decoder (common/pjpeg.c:
   pjpeg_create_from_buffer then pjpeg_to_u8_baseline, component 0 cropped
   to the image), byte for byte, and so are its error codes (PJPEG_ERR_* of
   common/pjpeg.h). The reference decodes on one CPU core; here the host
   reads the headers and cuts each scan at its restart markers, and the
   entropy decoding and the IDCT run on the GPU. pjpeg.h's calls are
   provided too, over the same decoder. No counterpart in the reference's
   native API. */
typedef struct at_jpeg at_jpeg;

/* A decoder with its own CUDA stream and memory on the current device. */
at_jpeg *at_jpeg_create(void);
void at_jpeg_destroy(at_jpeg *dec);

/* The size of the gray frame a decode of buf gives (the image's width and
   height, its component count). Returns 0 or the error the decode would
   return from its headers (PJPEG_ERR_*). */
int at_jpeg_info(const uint8_t *buf, int64_t len, uint32_t flags, int32_t *width, int32_t *height,
                 int32_t *ncomponents);

/* Decodes n JPEGs (bufs[i], lens[i] bytes, host memory) in one pass on the
   GPU into gray frames: frame i goes to dst[i], rows of strides[i] bytes,
   width x height as at_jpeg_info gives; dst is device memory of the
   decoder's GPU when on_device is non-zero, host memory otherwise. flags: PJPEG_MJPEG.
   errors[i] receives each image's PJPEG_ERR_* (0: written). Returns the
   number of images that failed, or -1 for a CUDA error (message on
   stderr). Returns when every frame is written. */
int at_jpeg_decode_gray(at_jpeg *dec, int32_t n, const uint8_t *const *bufs, const int64_t *lens, uint32_t flags,
                        uint8_t *const *dst, const int64_t *strides, int32_t on_device, int32_t *errors);

/* Figures of the last decode: [0] host parse ms, [1] copy in ms, [2] sync
   pass ms, [3] write and IDCT ms, [4] copy out ms (CUDA events), [5] sub-
   streams, [6] sync passes beyond the first, [7] entropy-coded bytes, [8]
   the most repeats a CTA needed within a pass, [9] unused. */
int at_jpeg_last_stats(const at_jpeg *dec, double *out10);

/* Bits of entropy-coded data per sub-stream (one GPU thread each); by
   default chosen per call from 256 to 1024 by the data's size (0 restores
   that); a multiple of 32 from 64 to 65536. Returns 0 or 1. */
int at_jpeg_set_sub_bits(at_jpeg *dec, int32_t bits);

/* Bits a sub-stream's first, speculative decode starts before the
   sub-stream (by default the larger of 512 and the sub-stream; 0 restores
   that): longer run-ins fall into step with the true decode more often, at
   the cost of decoding them. Returns 0 or 1. */
int at_jpeg_set_run_in(at_jpeg *dec, int32_t bits);

/* Host threads that parse the images of a batch (0, the default: up to
   16). Returns 0 or 1. */
int at_jpeg_set_threads(at_jpeg *dec, int32_t threads);

#ifdef __cplusplus
}
#endif

#endif
