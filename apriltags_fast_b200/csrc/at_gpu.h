// Shared host/device declarations of the GPU detection pipeline.
//
// A batch holds F frames of any sizes. All per-pixel arrays of the batch
// are concatenated: frame f's quad-image pixel (x, y) is at q_off + y*qw + x.
// Union-find nodes: frame f owns ids [node_off, node_off + qw*qh + qh): the
// run i of row y is node node_off + y*qw + i (a row never has qw runs), and
// the last-column node of row y is node_off + qw*qh + y. So within a frame
// the runs of earlier rows, and then the last-column nodes, have smaller
// ids, the order the reference's packed run numbering gives; and the ids of
// different frames never interleave.
#pragma once
#include <stdint.h>

#define AT_MAX_FAMILIES 16
#define AT_NOK 0xffffffffu          // label of a pixel whose component is too small
#define AT_MAX_NMAXIMA 16           // largest max_nmaxima the fit kernel supports
#define AT_MAX_TW 16                // largest family total_width supported
#define AT_FIT_THREADS 128
#define AT_DEC_THREADS 128

// Error bits set by device-side checks (read back by the host).
#define AT_ERR_CLUSTER_TOO_BIG 1u
#define AT_ERR_CAPACITY 2u
#define AT_ERR_ORDER 4u             // the reference's quad order could not be recovered
#define AT_ERR_SEGCAP 8u            // the clusters' row tables needed more room: the batch runs again

struct FrameDesc {
    int32_t w, h;          // input frame
    int32_t qw, qh;        // quad image
    const uint8_t *img;    // input pixels in device memory: the caller's, or a copy in the arena
    int64_t stride;        // bytes between rows of img
    int64_t q_off;         // into the quad-pixel arenas
    int64_t node_off;      // first union-find node id of the frame
    int64_t row0;          // global index of quad row 0
    int64_t tile_off;      // into the tile arenas ((qw/4) * (qh/4))
    uint32_t fam_mask;     // families decoded for this frame
    int32_t max_px;        // 2 * (2 qw + 2 qh)
    int32_t tag_width;     // min_tag_width of the frame's families (fast/detector.c:67-81)
    int32_t normal_border, reversed_border;  // whether any of them has a normal / reversed border
};

// Detector parameters that the kernels need (host copies them per call).
struct GpuParams {
    float quad_decimate;
    int32_t min_cluster_pixels;
    int32_t max_nmaxima;
    int32_t min_white_black_diff;
    int32_t refine_edges;
    int32_t decode_blurred;   // decode samples the blurred quad image
    int32_t nfam;
    double max_dot;           // (double)cos_critical_rad
    double max_mse;           // (double)max_line_fit_mse
    double decode_sharpening;
    double qsm[7];            // (float)exp(-j^2/2), host libm
    double rot_cs[4][2];      // cos, sin of r*pi/2, host libm
};

// One family on the device: geometry plus its quick-decode tables.
struct GpuFamily {
    int32_t nbits, wab, tw;
    int32_t reversed_border;
    int32_t chunk, maxham;
    int64_t cap;              // 1 << chunk
    int64_t ncodes;
    int32_t bit_x[64], bit_y[64];
    const uint32_t *off;      // 4 * (cap + 1)
    const uint16_t *idx;      // 4 * ncodes: code index per chunk bucket entry
    const uint64_t *codes;    // 4 * ncodes: the code of each entry
};

// A fitted quad (cluster order), before corner scaling.
struct GpuQuad {
    float p[4][2];
    int32_t reversed_border;
    int32_t frame;
};

// A detection in the reference's at_detection layout (168 bytes).
struct GpuDetection {
    int32_t family, id, hamming;
    float decision_margin;
    double H[9];
    double c[2];
    double p[4][2];
};
