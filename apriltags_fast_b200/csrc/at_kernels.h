// Launchers of the detection kernels (defined in at_kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "at_gpu.h"

// Run table and union-find nodes, indexed by node id.
struct RunArrays {
    uint16_t *start, *end;
    uint8_t *v;
    uint32_t *parent;  // union-find parent
    uint32_t *px;      // at a root: its component's pixel count
    uint32_t *minid;   // at a root: its component's smallest node id (the label)
};

// Per-point scratch of the quad fit, indexed by point position.
struct FitScratch {
    uint64_t *keys, *skey;
    uint32_t *sval;
    double *w, *fx, *fy;
    double *mx, *my, *mxx, *mxy, *myy, *mw;
    double *errs, *filt, *mxe;
    int32_t *mxi;
    uint32_t *lists;   // one list of cluster ids per size class, nclusters apart
    uint32_t *counts;  // per class: list length, then the next list index to take
};

struct BlurTaps {
    int n;
    uint8_t k[64];
};

// The grid of the per-frame kernels: x blocks per frame, one row of frames.
struct Launch {
    cudaStream_t stream;
    int nframes;
    int blocks_per_frame;
    int64_t max_qh;  // the tallest quad image of the batch
};

void launch_decimate(const Launch &L, const FrameDesc *frames, const uint8_t *img, uint8_t *qim, float factor);
void launch_blur(const Launch &L, const FrameDesc *frames, uint8_t *qim, uint8_t *tmp_a, uint8_t *tmp_b,
                 const BlurTaps &taps, bool sharpen);
void launch_threshold(const Launch &L, const FrameDesc *frames, const uint8_t *qim, uint8_t *tmax, uint8_t *tmin,
                      uint8_t *thr, int32_t diff);
void launch_deglitch(const Launch &L, const FrameDesc *frames, uint8_t *thr, uint8_t *tmp);
int launch_segment(const Launch &L, const FrameDesc *frames, const uint8_t *thr, RunArrays runs, uint32_t *row_nruns,
                   uint32_t *lab, int32_t min_px, int64_t max_qh);
void launch_point_count(const Launch &L, const FrameDesc *frames, const uint8_t *thr, const uint32_t *lab,
                        uint64_t *row_npts);
void launch_point_emit(const Launch &L, const FrameDesc *frames, const uint8_t *thr, const uint32_t *lab,
                       const uint64_t *row_pt_off, uint64_t *pt_key, uint64_t *pt_val, int nb);
void launch_cluster_heads(cudaStream_t s, const uint64_t *key, int64_t n, uint32_t *head);
void launch_cluster_hash(cudaStream_t s, const uint64_t *key, int64_t n, uint64_t *tkeys, uint32_t *tcount,
                         uint32_t mask, uint32_t *full);
void launch_cluster_collect(cudaStream_t s, const uint64_t *tkeys, uint32_t size, uint64_t *okeys, uint32_t *oslots,
                            uint32_t *count);
// Distinct 64-bit keys with 32-bit values in key order (a rank per key);
// false (nothing launched) above RANK_SORT_CAP keys.
#define RANK_SORT_CAP 16384
bool launch_sort_distinct(cudaStream_t s, const uint64_t *kin, const uint32_t *vin, int64_t n, uint64_t *kout,
                          uint32_t *vout);
void launch_cluster_rank(cudaStream_t s, const uint64_t *skeys, const uint32_t *sslots, int64_t ncl,
                         const uint32_t *tcount, uint32_t *rank_of_slot, uint32_t *ccount, int nb,
                         const FrameDesc *frames, int nframes, int32_t *cframe);
void launch_cluster_assign(cudaStream_t s, const uint64_t *key, int64_t n, const uint64_t *tkeys, uint32_t mask,
                           const uint32_t *rank_of_slot, uint32_t *cidx);
void launch_cluster_starts(cudaStream_t s, const uint64_t *key, const uint32_t *head, const uint32_t *head_scan,
                           int64_t n, int nb, const FrameDesc *frames, int nframes, uint32_t *cstart, int32_t *cframe);
void launch_fit_quads(cudaStream_t s, cudaStream_t side, cudaStream_t side2, cudaStream_t side3, cudaEvent_t fork,
                      cudaEvent_t join, cudaEvent_t join2, cudaEvent_t join3, const FrameDesc *frames, const GpuParams &prm, const uint8_t *qim,
                      const uint64_t *pts, const uint32_t *cstart, const int32_t *cframe, int64_t nclusters,
                      int64_t npoints, const FitScratch &scr, GpuQuad *quads, uint32_t *quad_ok, uint32_t *err);
void launch_gather_quads(cudaStream_t s, const GpuQuad *quads, const uint32_t *ok, const uint32_t *scan, int64_t n,
                         GpuQuad *out, uint32_t *nq);
void launch_frame_bounds(cudaStream_t s, const GpuQuad *quads, const uint32_t *nq, int nframes, int nfam,
                         int64_t *qstart, int64_t *out_off);
void launch_output(cudaStream_t s, int nframes, const int64_t *qstart, const GpuDetection *out,
                   const int64_t *out_off, const int64_t *out_n, int64_t *first, GpuDetection *host,
                   int64_t *meta, int64_t max_dets);
// per quad: refined corners (8 floats), homography (9 doubles), and whether
// the homography was found and is invertible
struct DecodeScratch {
    float *corners;
    double *h;
    uint32_t *hok;
    const uint32_t *nq;  // the number of quads, on the device
};
void launch_decode(cudaStream_t s, const FrameDesc *frames, const GpuParams &prm, const GpuFamily *fams,
                   const uint8_t *img, const uint8_t *qim, const GpuQuad *quads, int64_t max_quads,
                   const DecodeScratch &scr, GpuDetection *dets, uint32_t *det_ok);
void launch_finalize(cudaStream_t s, int nframes, const int64_t *frame_qstart, int nfam, const GpuDetection *dets,
                     const uint32_t *det_ok, uint32_t *idx, uint8_t *removed, GpuDetection *out,
                     const int64_t *out_off, int64_t *out_n);
