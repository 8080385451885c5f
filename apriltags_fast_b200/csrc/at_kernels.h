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
// Decimate 2 + tile max/min + threshold in one pass (no blur): max_blocks
// from decimate_threshold_blocks of the batch's largest frame.
void launch_decimate_threshold(const Launch &L, const FrameDesc *frames, int64_t max_blocks, uint8_t *qim,
                               uint8_t *thr, int32_t diff);
int64_t decimate_threshold_blocks(int64_t qw, int64_t qh);
void launch_deglitch(const Launch &L, const FrameDesc *frames, uint8_t *thr, uint8_t *tmp);
int launch_segment(const Launch &L, const FrameDesc *frames, const uint8_t *thr, RunArrays runs, uint32_t *row_nruns,
                   uint32_t *lab, int32_t min_px, int64_t max_qh);
void launch_point_count(const Launch &L, const FrameDesc *frames, const uint8_t *thr, const uint32_t *lab,
                        uint64_t *row_npts);
void launch_point_emit(const Launch &L, const FrameDesc *frames, const uint8_t *thr, const uint32_t *lab,
                       const uint64_t *row_pt_off, uint64_t *pt_key, uint64_t *pt_val, int nb);
void launch_cluster_heads(cudaStream_t s, const uint64_t *key, int64_t n, uint32_t *head);
void launch_cluster_collect(cudaStream_t s, const uint64_t *tkeys, uint32_t size, uint64_t *okeys, uint32_t *oslots,
                            uint32_t *count);
// Clusters without sorting the points (at_cluster.cu). The pair table:
// key (label pair), point count, first and last row with points, per slot.
struct PairTable {
    uint64_t *keys;
    uint32_t *count, *ymin, *ymax;
    uint32_t mask;
};
// Scratch of the pair ordering: per pair its frame, per frame its pair count,
// first pair (nframes + 1) and a cursor, the pairs grouped by frame, and
// the block sums of the scans (pair_scan_blocks each).
struct PairScratch {
    uint32_t *kframe, *fcount, *foff, *fcur;
    uint64_t *gkeys;
    uint32_t *gslots, *bsum_a, *bsum_b;
};
// The points of each row (rows 1 .. qh-2): records in emission order at
// rec + 2 (q_off + y qw), at most 2 qw a row (pair index in the row |
// neighbour << 11 | pixel is 0 << 13 | x << 14); the row's distinct pairs
// (slot in the pair table, points) at (row0 + y) nd_cap; info[row0 + y] =
// (records, pairs).
struct PointRows {
    uint32_t *rec;
    uint32_t *pslot, *pcnt;
    uint2 *info;
    int32_t nd_cap;
};
bool point_scan_set_smem();
void launch_point_scan(const Launch &L, const FrameDesc *frames, const uint8_t *thr, const uint32_t *lab, int nb,
                       const PairTable &T, const PointRows &P, uint32_t *full, unsigned long long *npoints);
void launch_pair_order(cudaStream_t s, const uint64_t *okeys, const uint32_t *oslots, int64_t ncl, int nb,
                       const FrameDesc *frames, int nframes, const PairTable &T, const PairScratch &P,
                       uint64_t *skeys, uint32_t *sslots, uint32_t *rank_of_slot, uint32_t *ccount, uint32_t *cspan,
                       uint32_t *cy0, int32_t *cframe, uint32_t *cstart, uint32_t *spanoff);
int64_t pair_scan_blocks(int64_t ncl);
int64_t scan_u32_scratch(int64_t n);
void launch_scan_u32(cudaStream_t s, const uint32_t *a, int64_t n, uint32_t *out, uint32_t *scratch);
void launch_point_place(const Launch &L, const FrameDesc *frames, const PointRows &P, const uint32_t *rank_of_slot,
                        const uint32_t *cstart, const uint32_t *spanoff, const uint32_t *cspan, const uint32_t *cy0,
                        int64_t ncl, uint32_t *seg, int64_t cap, uint64_t *out, int64_t npts, uint32_t *err);
void launch_cluster_starts(cudaStream_t s, const uint64_t *key, const uint32_t *head, const uint32_t *head_scan,
                           int64_t n, int nb, const FrameDesc *frames, int nframes, uint32_t *cstart, int32_t *cframe,
                           uint64_t *ckey);
void launch_fit_quads(cudaStream_t s, cudaStream_t side, cudaStream_t side2, cudaStream_t side3, cudaEvent_t fork,
                      cudaEvent_t join, cudaEvent_t join2, cudaEvent_t join3, const FrameDesc *frames, const GpuParams &prm, const uint8_t *qim,
                      const uint64_t *pts, const uint32_t *cstart, const int32_t *cframe, int64_t nclusters,
                      int64_t npoints, const FitScratch &scr, GpuQuad *quads, uint32_t *quad_ok, uint32_t *err);
// also each gathered quad's cluster index (qcl)
void launch_gather_quads(cudaStream_t s, const GpuQuad *quads, const uint32_t *ok, const uint32_t *scan, int64_t n,
                         GpuQuad *out, uint32_t *nq, uint32_t *qcl);
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
// The reference's order of the quads whose detections share an id
// (at_order.cu). Per frame: whether it has such detections (need), the
// target components (GPU labels, pixel counts, and after the replay their
// roots in the reference's packed node numbering); per node, the frame's
// target runs compacted by row (tlist); per row, their count (trow); per
// row plus one per frame, the runs above the row (rpre).
#define AT_REF_MAXT 192
#define REF_BAND 16         // rows per band of the replay, at most
#define REF_PCAP 4160       // target runs of a row, at most (quad images up to 4161 px wide)
#define REF_PCAP_MIN 2048   // target runs per band, at most, when every row has fewer
#define REF_SMALLR 256      // the replay's narrow class: rows of at most this many target runs
#define REF_BAND_BLOCKS 32  // replay blocks per frame when the replay works in a global scratch
struct RefOrder {
    uint32_t *need, *nt;
    uint32_t *tlabel, *tpx, *troot;
    uint64_t *tlist;
    uint32_t *trow;
    uint32_t *rpre;
    uint32_t *fin, *finb;     // per target: its root (node or symbol) and the band where it was found
    // per band (rows + one per frame each): first row (and the end after the
    // last band), the widest row, the band's summary (at_order.cu); per
    // frame: the band count
    uint32_t *bstart, *bwide;
    uint4 *desc;
    uint32_t *nband;
    // per node (at the rows of the band edges, at_order.cu):
    uint32_t *tch;            //   each target run: the target runs above it touches (first | last << 16)
    uint32_t *ltop, *lpx;     //   top row: each run's band component, their pixels
    uint32_t *lbot, *lpx2;    //   bottom row: each run's band component, the others' pixels
    uint16_t *bslot;          //   row above a band: each target run's slot
    uint64_t *binfo;          //   row above a band: each slot, pixels | first run << 32 | target << 48
    uint32_t *outroot;        //   row above a band: each slot's root after the band above
    uint32_t *bm;             // per row: slots at the row above a band
};
// The sizes the order replay runs at: capr, the most runs in a row of the
// batch; pcap, the most target runs of a band; global scratch regions (a
// frame's, a block's) for the frontier pass and the wide-row replay when
// their arrays exceed the shared memory (else null).
struct RefPlan {
    int64_t capr, pcap;
    uint8_t *front_scratch;
    size_t front_bytes;
    uint8_t *band_scratch;
    size_t band_bytes;
};
size_t ref_replay_bytes(int64_t capr);
size_t ref_band_bytes(int64_t capr, bool staged);
size_t ref_local_bytes(int64_t pcap);
size_t ref_frontier_bytes(int64_t capr, bool staged);
bool ref_replay_set_smem(size_t bytes);
int ref_order_launches(const RefPlan &P);
void launch_ref_order(const Launch &L, const FrameDesc *frames, const uint8_t *thr, RunArrays runs,
                      const uint32_t *row_nruns, int nfam, const int64_t *qstart, const GpuDetection *dets,
                      const uint32_t *det_ok, const uint32_t *qcl, const uint64_t *ckey, int nb,
                      const RefPlan &P, const RefOrder &ref, uint32_t *err);
// okey: 2 u64 + 1 u32 per detection slot (the order keys, a second index)
void launch_finalize(cudaStream_t s, int nframes, const int64_t *frame_qstart, int nfam, const GpuDetection *dets,
                     const uint32_t *det_ok, uint32_t *idx, uint8_t *removed, GpuDetection *out,
                     const int64_t *out_off, int64_t *out_n, const FrameDesc *frames, const RefOrder &ref,
                     const uint32_t *qcl, const uint64_t *ckey, int nb, uint64_t *okey, uint32_t *idx2,
                     uint32_t *err);
