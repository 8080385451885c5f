// The detector object and the C ABI (include/apriltag_fast.h).
//
// Host code only orchestrates: it sizes the device arenas, copies frames in,
// launches the stage kernels (at_kernels.cu) on the detector's stream and
// copies the detections out. Every computation of the detection path runs on
// the GPU. Compiled with -ffp-contract=off for the few host-side constants
// (blur taps, the low-pass taps, rotation cos/sin) that the reference takes
// from libm.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cub/cub.cuh>
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "apriltag_fast.h"
#include "at_gpu.h"
#include "at_kernels.h"

// batch splitting: at most this many pipelines, each given at least
// AT_SPLIT_MIN_FRAMES frames (measured on 1080p batches: copies from host
// memory overlap compute, +14% frames/s at 32 frames; below about 20
// frames one pipeline is as fast)
#define AT_BATCH_SPLIT_DEFAULT 3
#define AT_BATCH_SPLIT_MAX 4
#define AT_SPLIT_MIN_FRAMES 10

static_assert(sizeof(at_detection) == 168, "at_detection layout");
static_assert(sizeof(GpuDetection) == sizeof(at_detection), "detection layout");
static_assert(sizeof(at_detector) == 160, "at_detector layout");
static_assert(sizeof(at_family) == 584, "at_family layout");

// Tables of the built-in families, a C source that the build makes from
// csrc/families.bin (gen_families.py); a null-terminated list.
extern "C" {
extern const at_family *const at_builtin_families[];
}

namespace {

// A device buffer that only grows. Growing frees the old one (cudaFree
// synchronises the device first).
struct DBuf {
    void *p = nullptr;
    size_t cap = 0;
    size_t want = 0;  // the largest request of the current call
    cudaError_t ensure(size_t bytes) {
        if (bytes > want) want = bytes;
        if (bytes <= cap) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        size_t want = bytes + bytes / 2 + 4096;  // grow with headroom: growth synchronises the device
        cudaError_t e = cudaMalloc(&p, want);
        if (e == cudaSuccess) cap = want;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    template <class T> T *as() const { return static_cast<T *>(p); }
};

// Pinned host staging that only grows.
struct HBuf {
    void *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap) return cudaSuccess;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        size_t want = bytes + bytes / 2 + 4096;  // grow with headroom: growth synchronises the device
        cudaError_t e = cudaMallocHost(&p, want);
        if (e == cudaSuccess) cap = want;
        return e;
    }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
    }
    template <class T> T *as() const { return static_cast<T *>(p); }
};

enum {
    B_FRAMES, B_IMG, B_QIM, B_THR, B_TMPA, B_TMPB, B_TMAX, B_TMIN, B_LAB,
    B_RSTART, B_REND, B_RV, B_PARENT, B_PX, B_ROWRUNS, B_ROWPTS, B_ROWOFF,
    B_KEY, B_VAL, B_KEY2, B_VAL2, B_HEAD, B_HSCAN, B_CSTART, B_CFRAME,
    B_SKEYS, B_SSKEY, B_SSVAL, B_SW, B_SFX, B_SFY, B_SMX, B_SMY, B_SMXX, B_SMXY, B_SMYY, B_SMW, B_SERRS, B_SFILT,
    B_SMXE, B_SMXI, B_QUADS, B_QOK, B_QSCAN, B_QUADSC, B_DETS, B_DETOK, B_OUT, B_QSTART, B_OUTOFF, B_OUTN, B_DIDX, B_DRM, B_MINID, B_FLIST, B_FCNT, B_QCORN, B_QH, B_QHOK, B_QNUM, B_FIRST, B_HKEYS, B_HCOUNT, B_HRANK, B_HOKEYS, B_HOSLOTS, B_HSKEYS, B_HSSLOTS, B_HCCOUNT, B_HMISC,
    B_HYMIN, B_HYMAX, B_CSPAN, B_CY0, B_SPANOFF, B_PKFRAME, B_PGKEYS, B_PGSLOTS, B_PFRAMES, B_PBSUM, B_SEG,
    B_QCL, B_CKEY, B_RNEED, B_RNT, B_RTLAB, B_RTPX, B_RTROOT, B_RTLIST, B_RTROW, B_RPRE, B_ROKEY, B_RIDX2, B_RSCR,
    B_RFIN, B_RFINB, B_RBSLOT, B_RBINFO, B_ROUTROOT, B_RBM, B_RBSTART, B_RBWIDE, B_RDESC, B_RNBAND, B_RFSCR, B_RTCH, B_RLTOP, B_RLPX, B_RLBOT,
    B_RLPX2,
    B_PREC, B_PPSLOT, B_PPCNT, B_PINFO, B_QSCR,
    B_CUB, B_ERR, B_NBUF
};

// the replay of the reference's union order keeps its arrays in shared
// memory up to this size, else in a global scratch region per frame
#define AT_REF_SMEM_MAX (200 * 1024)

}  // namespace

struct at_internal {
    at_family families[AT_MAX_FAMILIES];
    int bits[AT_MAX_FAMILIES];
    int nfam = 0;
    GpuFamily gfam[AT_MAX_FAMILIES];
    std::vector<void *> fam_mem[AT_MAX_FAMILIES];
    DBuf dfam;
    bool fam_dirty = true;

    int device = 0;
    cudaStream_t stream = nullptr, side = nullptr, side2 = nullptr, side3 = nullptr;
    cudaEvent_t ev[12];
    cudaEvent_t fork = nullptr, join = nullptr, join2 = nullptr, join3 = nullptr;  // ordering only, no timing
    DBuf buf[B_NBUF];
    HBuf h_frames, h_small, h_out;
    std::vector<at_detection> dets;

    int err = 0;
    std::string msg;
    // sizes of the last run (frame 0), for at_detector_diag
    int64_t last_qw = 0, last_qh = 0, last_npts = 0, last_ncl = 0, last_nq = 0;
    int64_t launches = 0;  // kernels of this library launched so far
    size_t ref_smem = 0;     // the shared memory the replay kernel is allowed (set per device)
    bool scan_smem = false;  // the point scan's shared memory allowance is set
    int64_t seg_slack = 64;  // row-table entries per cluster beyond its points (grows on a shortfall)

    // A large batch is spread over up to `split` pipelines: this detector
    // and split - 1 helpers (each with its own streams and arenas), each
    // driven by its own host thread, so that one pipeline's host
    // synchronisations and latency-bound kernels overlap the others' work.
    int split = AT_BATCH_SPLIT_DEFAULT;
    at_detector *helper[AT_BATCH_SPLIT_MAX - 1] = {};
    uint64_t fam_gen = 0, helper_gen[AT_BATCH_SPLIT_MAX - 1] = {};
    struct CopyChain *chain = nullptr;  // the order of the pipelines' host copies
};

// ---------------------------------------------------------------------------
// Errors: a failed CUDA call ends the frame with no detections.

#define CK(call)                                                                            \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess) {                                                            \
            set_error(in, 1, std::string(#call) + ": " + cudaGetErrorString(e_));           \
            return false;                                                                   \
        }                                                                                   \
    } while (0)

static void set_error(at_internal *in, int code, const std::string &m) {
    in->err = code;
    in->msg = m;
    fprintf(stderr, "apriltag_b200: %s\n", m.c_str());
}

// ---------------------------------------------------------------------------
// Families and their quick-decode tables (fast/decode.c:20-58), built on the
// host once per at_add_family and kept on the device.

static bool upload_family(at_internal *in, int i) {
    const at_family *f = &in->families[i];
    GpuFamily g;
    memset(&g, 0, sizeof g);
    g.nbits = f->nbits;
    g.wab = f->width_at_border;
    g.tw = f->total_width;
    g.reversed_border = f->reversed_border ? 1 : 0;
    g.chunk = (f->nbits + 3) / 4;
    g.cap = (int64_t)1 << g.chunk;
    g.ncodes = f->ncodes;
    g.maxham = in->bits[i];
    for (int k = 0; k < 64; k++) {
        g.bit_x[k] = f->bit_x[k];
        g.bit_y[k] = f->bit_y[k];
    }
    uint64_t mask = (uint64_t)g.cap - 1;
    std::vector<uint32_t> off(4 * (g.cap + 1), 0);
    std::vector<uint16_t> idx(4 * g.ncodes + 1);
    std::vector<uint64_t> codes(4 * g.ncodes + 1);
    for (int64_t c = 0; c < g.ncodes; c++)
        for (int j = 0; j < 4; j++) off[j * (g.cap + 1) + ((f->codes[c] >> (j * g.chunk)) & mask) + 1]++;
    for (int j = 0; j < 4; j++)
        for (int64_t v = 0; v < g.cap; v++) off[j * (g.cap + 1) + v + 1] += off[j * (g.cap + 1) + v];
    std::vector<uint32_t> cur(off);
    for (int64_t c = 0; c < g.ncodes; c++)
        for (int j = 0; j < 4; j++) {
            int64_t b = j * (g.cap + 1) + ((f->codes[c] >> (j * g.chunk)) & mask);
            int64_t e = j * g.ncodes + cur[b]++;
            idx[e] = (uint16_t)c;
            codes[e] = f->codes[c];
        }
    for (void *p : in->fam_mem[i]) cudaFree(p);
    in->fam_mem[i].clear();
    void *d_off, *d_idx, *d_codes;
    CK(cudaMalloc(&d_off, off.size() * 4));
    in->fam_mem[i].push_back(d_off);
    CK(cudaMalloc(&d_idx, idx.size() * 2));
    in->fam_mem[i].push_back(d_idx);
    CK(cudaMalloc(&d_codes, codes.size() * 8));
    in->fam_mem[i].push_back(d_codes);
    CK(cudaMemcpy(d_off, off.data(), off.size() * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_idx, idx.data(), idx.size() * 2, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_codes, codes.data(), codes.size() * 8, cudaMemcpyHostToDevice));
    g.off = (const uint32_t *)d_off;
    g.idx = (const uint16_t *)d_idx;
    g.codes = (const uint64_t *)d_codes;
    in->gfam[i] = g;
    in->fam_dirty = true;
    return true;
}

// ---------------------------------------------------------------------------
// Host-side constants of the reference.

// The quad image size (fast/image.c:6-20).
static void quad_size(int64_t w, int64_t h, float f, int64_t *qw, int64_t *qh) {
    if (!(f > 1.0f)) {
        *qw = w;
        *qh = h;
    } else if (f == 1.5f) {
        *qw = w / 3 * 2;
        *qh = h / 3 * 2;
    } else if ((int64_t)f == 2) {
        *qw = w / 2;
        *qh = h / 2;
    } else {
        int64_t k = (int64_t)f;
        *qw = 1 + (w - 1) / k;
        *qh = 1 + (h - 1) / k;
    }
}

// Blur taps (fast/image.c:108-118, 476-482): 0 when nothing is filtered.
static int blur_taps(float qsigma, BlurTaps *t) {
    if (qsigma == 0.0f) return 0;
    int64_t n = (int64_t)(4.0f * fabsf(qsigma));
    if ((n & 1) == 0) n++;
    if (n <= 1) return 0;
    if (n > 63) return -1;
    double sigma = fabsf(qsigma);
    double dk[64], acc = 0.0;
    for (int64_t i = 0; i < n; i++) {
        double x = (double)(i - n / 2) / sigma;
        dk[i] = exp(-0.5 * (x * x));
    }
    for (int64_t i = 0; i < n; i++) acc += dk[i];
    t->n = (int)n;
    for (int64_t i = 0; i < n; i++) t->k[i] = (uint8_t)(dk[i] / acc * 255.0);
    return (int)n;
}

// min_tag_width (fast/detector.c:67-81) and the border kinds of the
// families in `mask`.
static void frame_families(const at_detector *td, const at_internal *in, uint32_t mask, FrameDesc *f) {
    int32_t mtw = 1000000;
    bool normal = false, reversed = false;
    for (int i = 0; i < in->nfam; i++) {
        if (!(mask >> i & 1u)) continue;
        if (in->families[i].width_at_border < mtw) mtw = in->families[i].width_at_border;
        normal = normal || !in->families[i].reversed_border;
        reversed = reversed || in->families[i].reversed_border;
    }
    if (td->quad_decimate > 1.0f) mtw = (int32_t)((float)mtw / td->quad_decimate);
    if (mtw < 3) mtw = 3;
    f->tag_width = mtw;
    f->normal_border = normal;
    f->reversed_border = reversed;
}

static void gpu_params(const at_detector *td, const at_internal *in, bool decode_blurred, GpuParams *p) {
    memset(p, 0, sizeof *p);
    p->quad_decimate = td->quad_decimate;
    p->min_cluster_pixels = td->qtp.min_cluster_pixels;
    p->max_nmaxima = td->qtp.max_nmaxima;
    p->min_white_black_diff = td->qtp.min_white_black_diff;
    p->refine_edges = td->refine_edges ? 1 : 0;
    p->decode_blurred = decode_blurred ? 1 : 0;
    p->nfam = in->nfam;
    p->max_dot = (double)td->qtp.cos_critical_rad;
    p->max_mse = (double)td->qtp.max_line_fit_mse;
    p->decode_sharpening = td->decode_sharpening;
    for (int i = 0; i < 7; i++) p->qsm[i] = (float)exp(-(double)((i - 3) * (i - 3)) / 2.0);
    for (int r = 0; r < 4; r++) {
        double th = (double)r * M_PI / 2.0;
        p->rot_cs[r][0] = cos(th);
        p->rot_cs[r][1] = sin(th);
    }
}

// ---------------------------------------------------------------------------
// The pipeline over a batch of frames.

static int bits_for(uint64_t n) {
    int b = 1;
    while (b < 63 && ((uint64_t)1 << b) < n) b++;
    return b;
}

template <class F> static bool cub_call(at_internal *in, F &&f) {
    size_t bytes = 0;
    CK(f(nullptr, bytes));
    CK(in->buf[B_CUB].ensure(bytes));
    CK(f(in->buf[B_CUB].p, bytes));
    return true;
}

// The pipelines of one split batch copy their host frames in pipeline
// order: pipeline k's copies start on the device once pipeline k - 1's are
// done, so the first pipeline computes while the later ones' frames are
// still crossing the bus (copies issued together share it and all end late).
struct CopyChain {
    std::mutex m;
    std::condition_variable cv;
    int done = 0;  // the pipelines whose copies are issued (their events recorded)
    cudaEvent_t ev[AT_BATCH_SPLIT_MAX] = {};
};

// A pipeline's turn in the chain; it is passed on when the pipeline's
// copies are issued, or when the pipeline ends without them.
struct CopyTurn {
    CopyChain *c = nullptr;
    int k = 0;
    cudaStream_t st = nullptr;
    bool passed = false;
    void wait() {
        if (!c || k == 0) return;
        std::unique_lock<std::mutex> l(c->m);
        // bounded: a pipeline that never passes its turn cannot stall this one
        c->cv.wait_for(l, std::chrono::seconds(10), [&] { return c->done >= k; });
        if (c->done >= k) cudaStreamWaitEvent(st, c->ev[k - 1], 0);
    }
    void pass() {
        if (!c || passed) return;
        passed = true;
        cudaEventRecord(c->ev[k], st);
        {
            std::lock_guard<std::mutex> l(c->m);
            c->done = std::max(c->done, k + 1);
        }
        c->cv.notify_all();
    }
    ~CopyTurn() { pass(); }
};

static bool run_batch(at_detector *td, const at_frame *frames, int64_t n, at_frame_result *res,
                      CopyChain *chain = nullptr, int link = 0) {
    at_internal *in = td->in;
    CopyTurn turn;
    turn.c = chain;
    turn.k = link;
    turn.st = in->stream;
    cudaStream_t st = in->stream;
    CK(cudaSetDevice(in->device));
    if (td->qtp.max_nmaxima > AT_MAX_NMAXIMA || td->qtp.max_nmaxima < 0) {
        set_error(in, 2, "max_nmaxima above the supported " + std::to_string(AT_MAX_NMAXIMA));
        return false;
    }
    BlurTaps taps;
    memset(&taps, 0, sizeof taps);
    int ntaps = blur_taps(td->quad_sigma, &taps);
    if (ntaps < 0) {
        set_error(in, 2, "quad_sigma too large (blur kernel above 63 taps)");
        return false;
    }
    const bool decimated = td->quad_decimate > 1.0f;
    GpuParams prm;
    gpu_params(td, in, ntaps > 1 && !decimated, &prm);

    // frame layout
    std::vector<FrameDesc> fd(n);
    std::vector<char> copied(n, 0);  // frames copied into the input arena
    int64_t img = 0, qpx = 0, nodes = 0, rows = 0, tiles = 0;
    uint32_t all = in->nfam >= 32 ? 0xffffffffu : ((1u << in->nfam) - 1u);
    for (int64_t i = 0; i < n; i++) {
        FrameDesc &f = fd[i];
        memset(&f, 0, sizeof f);
        const at_frame &fr = frames[i];
        // a frame whose family set is empty is detected as with no families
        bool live = in->nfam > 0 && fr.width >= 8 && fr.height >= 8 && (!fr.family_mask || (fr.family_mask & all));
        int64_t qw = 0, qh = 0;
        if (live) quad_size(fr.width, fr.height, td->quad_decimate, &qw, &qh);
        if (qw < 4 || qh < 4) live = false;
        f.w = live ? (int32_t)fr.width : 0;
        f.h = live ? (int32_t)fr.height : 0;
        f.qw = live ? (int32_t)qw : 0;
        f.qh = live ? (int32_t)qh : 0;
        // frames already in this device's memory are read in place; the
        // others are copied into the input arena (packed, stride w)
        f.img = nullptr;
        f.stride = f.w;
        if (live) {
            cudaPointerAttributes pa;
            int dev = -1;
            cudaGetDevice(&dev);
            if (cudaPointerGetAttributes(&pa, fr.pixels) == cudaSuccess &&
                (pa.type == cudaMemoryTypeDevice || pa.type == cudaMemoryTypeManaged) && pa.device == dev &&
                pa.devicePointer != nullptr) {
                f.img = static_cast<const uint8_t *>(pa.devicePointer);
                f.stride = fr.stride;
            } else {
                cudaGetLastError();  // clear the error an unregistered host pointer leaves
                f.img = reinterpret_cast<const uint8_t *>((uintptr_t)img);  // an offset until the arena exists
                img += (int64_t)f.w * f.h;
                copied[i] = 1;
            }
        }
        f.q_off = qpx;
        f.node_off = nodes;
        f.row0 = rows;
        f.tile_off = tiles;
        f.fam_mask = fr.family_mask ? (fr.family_mask & all) : all;
        frame_families(td, in, f.fam_mask, &f);
        f.max_px = (int32_t)(2 * (2 * f.qw + 2 * f.qh));
        qpx += (int64_t)f.qw * f.qh;
        nodes += (int64_t)f.qw * f.qh + f.qh;
        rows += f.qh;
        tiles += (int64_t)(f.qw / 4) * (f.qh / 4);
    }
    for (int64_t i = 0; i < n; i++) res[i] = at_frame_result{0, 0, 0};
    in->dets.clear();
    in->last_qw = n > 0 ? fd[0].qw : 0;
    in->last_qh = n > 0 ? fd[0].qh : 0;
    in->last_npts = in->last_ncl = in->last_nq = 0;
    if (qpx == 0) return true;
    if (nodes >= ((int64_t)1 << 32)) {
        set_error(in, 2, "batch too large (union-find ids exceed 32 bits)");
        return false;
    }
    const int nb = bits_for((uint64_t)nodes);
    Launch L{st, (int)n, 0, 0};
    for (auto &f : fd) L.max_qh = f.qh > L.max_qh ? f.qh : L.max_qh;
    int64_t maxq = 0;
    for (auto &f : fd) maxq = f.qw * (int64_t)f.qh > maxq ? f.qw * (int64_t)f.qh : maxq;
    L.blocks_per_frame = (int)((maxq + 255) / 256 < 148 * 4 ? (maxq + 255) / 256 : 148 * 4);
    if (L.blocks_per_frame < 1) L.blocks_per_frame = 1;

    // arenas
    DBuf *B = in->buf;
    for (int k = 0; k < B_NBUF; k++) B[k].want = 0;
    CK(B[B_FRAMES].ensure(n * sizeof(FrameDesc)));
    CK(B[B_IMG].ensure(img + 1));
    CK(B[B_QIM].ensure(qpx));
    CK(B[B_THR].ensure(qpx));
    CK(B[B_TMPA].ensure(qpx));
    CK(B[B_TMPB].ensure(qpx));
    CK(B[B_TMAX].ensure(tiles + 1));
    CK(B[B_TMIN].ensure(tiles + 1));
    CK(B[B_LAB].ensure(qpx * 4));
    CK(B[B_RSTART].ensure(nodes * 2));
    CK(B[B_REND].ensure(nodes * 2));
    CK(B[B_RV].ensure(nodes));
    CK(B[B_PARENT].ensure(nodes * 4));
    CK(B[B_PX].ensure(nodes * 4));
    CK(B[B_ROWRUNS].ensure(rows * 4));
    CK(B[B_ROWPTS].ensure((rows + 1) * 8));
    CK(B[B_ROWOFF].ensure((rows + 1) * 8));
    CK(B[B_ERR].ensure(4));
    // copied frames: their offsets into the arena become pointers
    for (int64_t i = 0; i < n; i++)
        if (copied[i]) fd[i].img = B[B_IMG].as<uint8_t>() + (uintptr_t)fd[i].img;
    CK(in->h_frames.ensure(n * sizeof(FrameDesc)));
    memcpy(in->h_frames.p, fd.data(), n * sizeof(FrameDesc));
    const FrameDesc *dfr = B[B_FRAMES].as<FrameDesc>();

    for (int k = 0; k < 12; k++) CK(cudaEventRecord(in->ev[k], st));  // keep all events valid
    CK(cudaEventRecord(in->ev[0], st));
    CK(cudaMemcpyAsync(B[B_FRAMES].p, in->h_frames.p, n * sizeof(FrameDesc), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(B[B_ERR].p, 0, 4, st));
    turn.wait();
    for (int64_t i = 0; i < n; i++) {
        if (!copied[i]) continue;
        CK(cudaMemcpy2DAsync(const_cast<uint8_t *>(fd[i].img), fd[i].w, frames[i].pixels, frames[i].stride, fd[i].w,
                             fd[i].h, cudaMemcpyDefault, st));
    }
    turn.pass();
    uint8_t *qim = B[B_QIM].as<uint8_t>(), *thr = B[B_THR].as<uint8_t>();
    // decimate 2 without blur: decimation and threshold in one pass (its
    // time is the threshold stage's, as when the reference fuses them)
    const bool fused = (int)td->quad_decimate == 2 && ntaps <= 1;
    if (fused) {
        int64_t blocks = 1;
        for (auto &f : fd) {
            const int64_t b = f.qw > 0 ? decimate_threshold_blocks(f.qw, f.qh) : 0;
            blocks = b > blocks ? b : blocks;
        }
        CK(cudaEventRecord(in->ev[1], st));
        CK(cudaEventRecord(in->ev[2], st));
        launch_decimate_threshold(L, dfr, blocks, qim, thr, td->qtp.min_white_black_diff);
        in->launches += 1;
    } else {
        launch_decimate(L, dfr, B[B_IMG].as<uint8_t>(), qim, td->quad_decimate);
        in->launches += 1;
        CK(cudaEventRecord(in->ev[1], st));
        if (ntaps > 1) {
            launch_blur(L, dfr, qim, B[B_TMPA].as<uint8_t>(), B[B_TMPB].as<uint8_t>(), taps, td->quad_sigma < 0);
            in->launches += 3;
        }
        CK(cudaEventRecord(in->ev[2], st));
        launch_threshold(L, dfr, qim, B[B_TMAX].as<uint8_t>(), B[B_TMIN].as<uint8_t>(), thr,
                         td->qtp.min_white_black_diff);
        in->launches += 2;
    }
    if (td->qtp.deglitch) {
        launch_deglitch(L, dfr, thr, B[B_TMPA].as<uint8_t>());
        in->launches += 2;
    }
    CK(cudaEventRecord(in->ev[3], st));
    CK(B[B_MINID].ensure(nodes * 4));
    RunArrays runs{B[B_RSTART].as<uint16_t>(), B[B_REND].as<uint16_t>(), B[B_RV].as<uint8_t>(),
                   B[B_PARENT].as<uint32_t>(), B[B_PX].as<uint32_t>(), B[B_MINID].as<uint32_t>()};
    uint32_t *lab = B[B_LAB].as<uint32_t>();
    int64_t max_qh = 0;
    for (auto &f : fd) max_qh = f.qh > max_qh ? f.qh : max_qh;
    in->launches += launch_segment(L, dfr, thr, runs, B[B_ROWRUNS].as<uint32_t>(), lab, td->qtp.min_cluster_pixels,
                                   max_qh);
    CK(cudaEventRecord(in->ev[4], st));
    CK(cudaGetLastError());

    // boundary points and clusters: the label pairs hashed straight from
    // the threshold image (at_cluster.cu); the only wait of this stage reads
    // the pair and point counts. If the pair table overflows, the points are
    // emitted in order and sorted by pair instead (at_kernels.cu, CUB).
    int64_t ncl = 0, nq = 0;
    uint64_t npts = 0;
    uint32_t hsize = 1u << 16;
    while ((int64_t)hsize < qpx / 32 && hsize < (1u << 30)) hsize <<= 1;
    CK(B[B_HKEYS].ensure((size_t)hsize * 8));
    CK(B[B_HCOUNT].ensure((size_t)hsize * 4));
    CK(B[B_HYMIN].ensure((size_t)hsize * 4));
    CK(B[B_HYMAX].ensure((size_t)hsize * 4));
    CK(B[B_HRANK].ensure((size_t)hsize * 4));
    CK(B[B_HMISC].ensure(32));
    const PairTable pt{B[B_HKEYS].as<uint64_t>(), B[B_HCOUNT].as<uint32_t>(), B[B_HYMIN].as<uint32_t>(),
                       B[B_HYMAX].as<uint32_t>(), hsize - 1};
    uint32_t *misc = B[B_HMISC].as<uint32_t>();  // [0] overflow, [1] pairs, [2..3] points (u64)
    CK(cudaMemsetAsync(pt.keys, 0xff, (size_t)hsize * 8, st));
    CK(cudaMemsetAsync(pt.count, 0, (size_t)hsize * 4, st));
    CK(cudaMemsetAsync(pt.ymin, 0xff, (size_t)hsize * 4, st));
    CK(cudaMemsetAsync(pt.ymax, 0, (size_t)hsize * 4, st));
    CK(cudaMemsetAsync(misc, 0, 32, st));
    // each row's points as records, its pairs gathered in shared memory
    int64_t max_qw = 0;
    for (auto &f : fd) max_qw = f.qw > max_qw ? f.qw : max_qw;
    int32_t nd_cap = 64;
    while (nd_cap < max_qw / 8 && nd_cap < 2048) nd_cap <<= 1;
    CK(B[B_PREC].ensure(qpx * 8));
    CK(B[B_PPSLOT].ensure(rows * nd_cap * 4));
    CK(B[B_PPCNT].ensure(rows * nd_cap * 4));
    CK(B[B_PINFO].ensure(rows * 8));
    if (!in->scan_smem) {
        if (!point_scan_set_smem()) {
            set_error(in, 1, "cudaFuncSetAttribute for the point scan failed");
            return false;
        }
        in->scan_smem = true;
    }
    const PointRows prow{B[B_PREC].as<uint32_t>(), B[B_PPSLOT].as<uint32_t>(), B[B_PPCNT].as<uint32_t>(),
                         B[B_PINFO].as<uint2>(), nd_cap};
    launch_point_scan(L, dfr, thr, lab, nb, pt, prow, misc, reinterpret_cast<unsigned long long *>(misc + 2));
    CK(B[B_HOKEYS].ensure((size_t)hsize * 8));
    CK(B[B_HOSLOTS].ensure((size_t)hsize * 4));
    launch_cluster_collect(st, pt.keys, hsize, B[B_HOKEYS].as<uint64_t>(), B[B_HOSLOTS].as<uint32_t>(), misc + 1);
    in->launches += 2;
    uint32_t hm[4];
    CK(cudaMemcpyAsync(hm, misc, 16, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const bool hashed = hm[0] == 0;
    npts = (uint64_t)hm[2] | (uint64_t)hm[3] << 32;
    CK(B[B_CKEY].ensure(8));
    if (npts > 0 && hashed) {
        ncl = hm[1];
        CK(B[B_VAL2].ensure(npts * 8));
        CK(B[B_CSTART].ensure(ncl * 4 + 4));
        CK(B[B_CFRAME].ensure(ncl * 4 + 4));
        CK(B[B_HSKEYS].ensure(ncl * 8 + 8));
        CK(B[B_HSSLOTS].ensure(ncl * 4 + 4));
        CK(B[B_HCCOUNT].ensure(ncl * 4 + 4));
        CK(B[B_CSPAN].ensure(ncl * 4 + 4));
        CK(B[B_CY0].ensure(ncl * 4 + 4));
        CK(B[B_SPANOFF].ensure(ncl * 4 + 4));
        CK(B[B_PKFRAME].ensure(ncl * 4 + 4));
        CK(B[B_PGKEYS].ensure(ncl * 8 + 8));
        CK(B[B_PGSLOTS].ensure(ncl * 4 + 4));
        CK(B[B_PFRAMES].ensure((3 * n + 1) * 4));
        CK(B[B_PBSUM].ensure(2 * pair_scan_blocks(ncl) * 4));
        const int64_t segcap = (int64_t)npts + in->seg_slack * ncl + 4096;
        CK(B[B_SEG].ensure(segcap * 4));
        uint32_t *pf = B[B_PFRAMES].as<uint32_t>();
        uint32_t *bs = B[B_PBSUM].as<uint32_t>();
        const PairScratch ps{B[B_PKFRAME].as<uint32_t>(), pf, pf + n, pf + 2 * n + 1, B[B_PGKEYS].as<uint64_t>(),
                             B[B_PGSLOTS].as<uint32_t>(), bs, bs + pair_scan_blocks(ncl)};
        launch_pair_order(st, B[B_HOKEYS].as<uint64_t>(), B[B_HOSLOTS].as<uint32_t>(), ncl, nb, dfr, (int)n, pt, ps,
                          B[B_HSKEYS].as<uint64_t>(), B[B_HSSLOTS].as<uint32_t>(), B[B_HRANK].as<uint32_t>(),
                          B[B_HCCOUNT].as<uint32_t>(), B[B_CSPAN].as<uint32_t>(), B[B_CY0].as<uint32_t>(),
                          B[B_CFRAME].as<int32_t>(), B[B_CSTART].as<uint32_t>(), B[B_SPANOFF].as<uint32_t>());
        launch_point_place(L, dfr, prow, B[B_HRANK].as<uint32_t>(), B[B_CSTART].as<uint32_t>(),
                           B[B_SPANOFF].as<uint32_t>(), B[B_CSPAN].as<uint32_t>(), B[B_CY0].as<uint32_t>(), ncl,
                           B[B_SEG].as<uint32_t>(), segcap, B[B_VAL2].as<uint64_t>(), (int64_t)npts,
                           B[B_ERR].as<uint32_t>());
        in->launches += 13;
    } else if (npts > 0) {
        // the pair table overflowed: points in emission order, sorted by pair
        uint64_t *row_npts = B[B_ROWPTS].as<uint64_t>(), *row_off = B[B_ROWOFF].as<uint64_t>();
        CK(cudaMemsetAsync(row_npts + rows, 0, 8, st));
        launch_point_count(L, dfr, thr, lab, row_npts);
        in->launches += 1;
        if (!cub_call(in, [&](void *t, size_t &b) {
                return cub::DeviceScan::ExclusiveSum(t, b, row_npts, row_off, rows + 1, st);
            }))
            return false;
        CK(B[B_KEY].ensure(npts * 8));
        CK(B[B_VAL].ensure(npts * 8));
        CK(B[B_KEY2].ensure(npts * 8));
        CK(B[B_VAL2].ensure(npts * 8));
        CK(B[B_HEAD].ensure(npts * 4));
        CK(B[B_HSCAN].ensure(npts * 4));
        CK(B[B_CKEY].ensure(npts * 8));
        launch_point_emit(L, dfr, thr, lab, row_off, B[B_KEY].as<uint64_t>(), B[B_VAL].as<uint64_t>(), nb);
        in->launches += 1;
        if (!cub_call(in, [&](void *t, size_t &b) {
                return cub::DeviceRadixSort::SortPairs(t, b, B[B_KEY].as<uint64_t>(), B[B_KEY2].as<uint64_t>(),
                                                       B[B_VAL].as<uint64_t>(), B[B_VAL2].as<uint64_t>(),
                                                       (int64_t)npts, 0, 2 * nb, st);
            }))
            return false;
        const uint64_t *skey = B[B_KEY2].as<uint64_t>();
        uint32_t *head = B[B_HEAD].as<uint32_t>(), *hscan = B[B_HSCAN].as<uint32_t>();
        launch_cluster_heads(st, skey, npts, head);
        in->launches += 1;
        if (!cub_call(in, [&](void *t, size_t &b) {
                return cub::DeviceScan::ExclusiveSum(t, b, head, hscan, (int64_t)npts, st);
            }))
            return false;
        uint32_t last[2];
        CK(cudaMemcpyAsync(&last[0], hscan + npts - 1, 4, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(&last[1], head + npts - 1, 4, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        ncl = (int64_t)last[0] + last[1];
        CK(B[B_CSTART].ensure(ncl * 4 + 4));
        CK(B[B_CFRAME].ensure(ncl * 4));
        launch_cluster_starts(st, skey, head, hscan, npts, nb, dfr, (int)n, B[B_CSTART].as<uint32_t>(),
                              B[B_CFRAME].as<int32_t>(), B[B_CKEY].as<uint64_t>());
        in->launches += 1;
    }
    if (npts > 0) {
        const uint64_t *spts = B[B_VAL2].as<uint64_t>();
        CK(cudaEventRecord(in->ev[5], st));
        // each cluster's label pair (the reference order of shared ids needs it)
        const uint64_t *ckey = hashed ? B[B_HSKEYS].as<uint64_t>() : B[B_CKEY].as<uint64_t>();

        // quads
        const int sc[] = {B_SKEYS, B_SSKEY, B_SW, B_SFX, B_SFY, B_SMX, B_SMY, B_SMXX, B_SMXY, B_SMYY, B_SMW,
                          B_SERRS, B_SFILT, B_SMXE};
        for (int b : sc) CK(B[b].ensure(npts * 8));
        CK(B[B_SSVAL].ensure(npts * 4));
        CK(B[B_SMXI].ensure(npts * 4));
        CK(B[B_QUADS].ensure(ncl * sizeof(GpuQuad)));
        CK(B[B_QOK].ensure(ncl * 4));
        CK(B[B_QSCAN].ensure((ncl + 1) * 4));
        CK(B[B_QSCR].ensure(scan_u32_scratch(ncl) * 4));
        CK(B[B_FLIST].ensure(ncl * 4 * 5));
        CK(B[B_FCNT].ensure(64));
        FitScratch scr{B[B_SKEYS].as<uint64_t>(), B[B_SSKEY].as<uint64_t>(), B[B_SSVAL].as<uint32_t>(),
                       B[B_SW].as<double>(),      B[B_SFX].as<double>(),    B[B_SFY].as<double>(),
                       B[B_SMX].as<double>(),     B[B_SMY].as<double>(),    B[B_SMXX].as<double>(),
                       B[B_SMXY].as<double>(),    B[B_SMYY].as<double>(),   B[B_SMW].as<double>(),
                       B[B_SERRS].as<double>(),   B[B_SFILT].as<double>(),  B[B_SMXE].as<double>(),
                       B[B_SMXI].as<int32_t>(),   B[B_FLIST].as<uint32_t>(), B[B_FCNT].as<uint32_t>()};
        uint32_t *qok = B[B_QOK].as<uint32_t>(), *qscan = B[B_QSCAN].as<uint32_t>();
        launch_fit_quads(st, in->side, in->side2, in->side3, in->fork, in->join, in->join2, in->join3, dfr, prm, qim, spts, B[B_CSTART].as<uint32_t>(), B[B_CFRAME].as<int32_t>(), ncl,
                         (int64_t)npts, scr, B[B_QUADS].as<GpuQuad>(), qok, B[B_ERR].as<uint32_t>());
        in->launches += 8;
        CK(cudaGetLastError());
        launch_scan_u32(st, qok, ncl, qscan, B[B_QSCR].as<uint32_t>());
        in->launches += 3;
        // the quads in cluster order (grouped by frame), their count and each
        // frame's first quad stay on the device: decode is sized by ncl
        CK(B[B_QUADSC].ensure(ncl * sizeof(GpuQuad)));
        CK(B[B_QNUM].ensure(8));
        CK(B[B_QCL].ensure(ncl * 4));
        uint32_t *nq_dev = B[B_QNUM].as<uint32_t>();
        CK(cudaMemsetAsync(nq_dev, 0, 4, st));
        launch_gather_quads(st, B[B_QUADS].as<GpuQuad>(), qok, qscan, ncl, B[B_QUADSC].as<GpuQuad>(), nq_dev,
                            B[B_QCL].as<uint32_t>());
        in->launches += 1;
        CK(cudaEventRecord(in->ev[6], st));
        // decode
        if (in->fam_dirty) {
            CK(in->dfam.ensure(sizeof(GpuFamily) * AT_MAX_FAMILIES));
            CK(cudaMemcpyAsync(in->dfam.p, in->gfam, sizeof(GpuFamily) * AT_MAX_FAMILIES, cudaMemcpyHostToDevice, st));
            in->fam_dirty = false;
        }
        const int64_t nd = ncl * in->nfam;
        CK(B[B_DETS].ensure(nd * sizeof(GpuDetection)));
        CK(B[B_DETOK].ensure(nd * 4));
        CK(B[B_OUT].ensure(nd * sizeof(GpuDetection)));
        CK(B[B_DIDX].ensure(nd * 4));
        CK(B[B_DRM].ensure(nd));
        CK(B[B_QSTART].ensure((n + 1) * 8));
        CK(B[B_OUTOFF].ensure((n + 1) * 8));
        CK(B[B_OUTN].ensure((n + 1) * 8));
        CK(B[B_FIRST].ensure((n + 1) * 8));
        launch_frame_bounds(st, B[B_QUADSC].as<GpuQuad>(), nq_dev, (int)n, in->nfam, B[B_QSTART].as<int64_t>(),
                            B[B_OUTOFF].as<int64_t>());
        CK(B[B_QCORN].ensure(ncl * 8 * sizeof(float)));
        CK(B[B_QH].ensure(ncl * 9 * sizeof(double)));
        CK(B[B_QHOK].ensure(ncl * sizeof(uint32_t)));
        const DecodeScratch dscr{B[B_QCORN].as<float>(), B[B_QH].as<double>(), B[B_QHOK].as<uint32_t>(), nq_dev};
        launch_decode(st, dfr, prm, in->dfam.as<GpuFamily>(), B[B_IMG].as<uint8_t>(), qim, B[B_QUADSC].as<GpuQuad>(),
                      ncl, dscr, B[B_DETS].as<GpuDetection>(), B[B_DETOK].as<uint32_t>());
        CK(cudaEventRecord(in->ev[7], st));
        in->launches += 4;
        // the reference's quad order for detections that share an id: the
        // roots its union order picks for their components (at_order.cu)
        CK(B[B_RNEED].ensure(n * 4));
        CK(B[B_RNT].ensure(n * 4));
        CK(B[B_RTLAB].ensure(n * AT_REF_MAXT * 4));
        CK(B[B_RTPX].ensure(n * AT_REF_MAXT * 4));
        CK(B[B_RTROOT].ensure(n * AT_REF_MAXT * 4));
        CK(B[B_RTLIST].ensure(nodes * 8));
        CK(B[B_RTROW].ensure(rows * 4));
        CK(B[B_RPRE].ensure((rows + n) * 4));
        CK(B[B_ROKEY].ensure(nd * 16));
        CK(B[B_RIDX2].ensure(nd * 4));
        CK(B[B_RFIN].ensure(n * AT_REF_MAXT * 4));
        CK(B[B_RFINB].ensure(n * AT_REF_MAXT * 4));
        CK(B[B_RBSLOT].ensure(nodes * 2));
        CK(B[B_RBINFO].ensure(nodes * 8));
        CK(B[B_ROUTROOT].ensure(nodes * 4));
        CK(B[B_RBM].ensure(rows * 4));
        CK(B[B_RBSTART].ensure((rows + n) * 4));
        CK(B[B_RBWIDE].ensure((rows + n) * 4));
        CK(B[B_RDESC].ensure((rows + n) * 16));
        CK(B[B_RNBAND].ensure(n * 4));
        CK(B[B_RTCH].ensure(nodes * 4));
        CK(B[B_RLTOP].ensure(nodes * 4));
        CK(B[B_RLPX].ensure(nodes * 4));
        CK(B[B_RLBOT].ensure(nodes * 4));
        CK(B[B_RLPX2].ensure(nodes * 4));
        CK(cudaMemsetAsync(B[B_RTROOT].p, 0xff, n * AT_REF_MAXT * 4, st));
        CK(cudaMemsetAsync(B[B_RFINB].p, 0xff, n * AT_REF_MAXT * 4, st));
        const RefOrder ro{B[B_RNEED].as<uint32_t>(),   B[B_RNT].as<uint32_t>(),     B[B_RTLAB].as<uint32_t>(),
                          B[B_RTPX].as<uint32_t>(),    B[B_RTROOT].as<uint32_t>(),  B[B_RTLIST].as<uint64_t>(),
                          B[B_RTROW].as<uint32_t>(),   B[B_RPRE].as<uint32_t>(),    B[B_RFIN].as<uint32_t>(),
                          B[B_RFINB].as<uint32_t>(),   B[B_RBSTART].as<uint32_t>(), B[B_RBWIDE].as<uint32_t>(),
                          B[B_RDESC].as<uint4>(),      B[B_RNBAND].as<uint32_t>(),  B[B_RTCH].as<uint32_t>(),
                          B[B_RLTOP].as<uint32_t>(),
                          B[B_RLPX].as<uint32_t>(),
                          B[B_RLBOT].as<uint32_t>(),   B[B_RLPX2].as<uint32_t>(),   B[B_RBSLOT].as<uint16_t>(),
                          B[B_RBINFO].as<uint64_t>(),  B[B_ROUTROOT].as<uint32_t>(), B[B_RBM].as<uint32_t>()};
        int64_t capr = 1;
        for (auto &f : fd) capr = f.qw - 1 > capr ? f.qw - 1 : capr;
        if (nodes >= ((int64_t)1 << 31)) {  // the replay marks symbols with the top bit of a node id
            set_error(in, 2, "batch too large for the order replay (node ids above 2^31)");
            return false;
        }
        if (capr > REF_PCAP) {
            set_error(in, 2, "quad image too wide for the order replay (" + std::to_string(capr + 1) + " px)");
            return false;
        }
        // the frontier pass and the wide-row replay work in global scratch
        // when their arrays do not fit the shared memory
        RefPlan plan{capr, capr > REF_PCAP_MIN ? capr : REF_PCAP_MIN, nullptr, 0, nullptr, 0};
        if (ref_frontier_bytes(capr, true) > AT_REF_SMEM_MAX) {
            plan.front_bytes = ref_frontier_bytes(capr, false);
            CK(B[B_RFSCR].ensure(plan.front_bytes * n));
            plan.front_scratch = B[B_RFSCR].as<uint8_t>();
        }
        if (capr > REF_SMALLR && ref_band_bytes(capr, true) > AT_REF_SMEM_MAX) {
            plan.band_bytes = ref_replay_bytes(capr);
            CK(B[B_RSCR].ensure(plan.band_bytes * n * REF_BAND_BLOCKS));
            plan.band_scratch = B[B_RSCR].as<uint8_t>();
        }
        if (in->ref_smem == 0) {
            if (!ref_replay_set_smem(AT_REF_SMEM_MAX)) {
                set_error(in, 1, "cudaFuncSetAttribute for the order replay failed");
                return false;
            }
            in->ref_smem = AT_REF_SMEM_MAX;
        }
        launch_ref_order(L, dfr, thr, runs, B[B_ROWRUNS].as<uint32_t>(), in->nfam, B[B_QSTART].as<int64_t>(),
                         B[B_DETS].as<GpuDetection>(), B[B_DETOK].as<uint32_t>(), B[B_QCL].as<uint32_t>(), ckey, nb,
                         plan, ro, B[B_ERR].as<uint32_t>());
        in->launches += ref_order_launches(plan);
        launch_finalize(st, (int)n, B[B_QSTART].as<int64_t>(), in->nfam, B[B_DETS].as<GpuDetection>(),
                        B[B_DETOK].as<uint32_t>(), B[B_DIDX].as<uint32_t>(), B[B_DRM].as<uint8_t>(),
                        B[B_OUT].as<GpuDetection>(), B[B_OUTOFF].as<int64_t>(), B[B_OUTN].as<int64_t>(), dfr, ro,
                        B[B_QCL].as<uint32_t>(), ckey, nb, B[B_ROKEY].as<uint64_t>(), B[B_RIDX2].as<uint32_t>(),
                        B[B_ERR].as<uint32_t>());
        // the frames' detections and counts straight into pinned host memory
        CK(in->h_out.ensure(nd * sizeof(GpuDetection) + 16));
        CK(in->h_small.ensure((3 * n + 4) * 8));
        launch_output(st, (int)n, B[B_QSTART].as<int64_t>(), B[B_OUT].as<GpuDetection>(), B[B_OUTOFF].as<int64_t>(),
                      B[B_OUTN].as<int64_t>(), B[B_FIRST].as<int64_t>(), in->h_out.as<GpuDetection>(),
                      in->h_small.as<int64_t>(), nd);
        in->launches += 4;
        CK(cudaGetLastError());
        CK(cudaEventRecord(in->ev[8], st));
        uint32_t derr = 0;
        CK(cudaMemcpyAsync(&derr, B[B_ERR].p, 4, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if ((derr & AT_ERR_SEGCAP) && in->seg_slack < ((int64_t)1 << 24)) {
            // the clusters' row tables were short (rows without points inside
            // a cluster's span): the batch again, with more room
            in->seg_slack *= 8;
            return run_batch(td, frames, n, res);
        }
        if (derr) {
            set_error(in, 3, "device check failed (code " + std::to_string(derr) + ")");
            return false;
        }
        const int64_t *meta = in->h_small.as<int64_t>();
        nq = meta[3 * n + 1];
        const GpuDetection *ho = in->h_out.as<GpuDetection>();
        const int64_t total = meta[3 * n];
        in->dets.resize(total);
        if (total) memcpy(in->dets.data(), ho, total * sizeof(at_detection));
        for (int64_t f = 0; f < n; f++) res[f] = at_frame_result{meta[3 * f], meta[3 * f + 1], meta[3 * f + 2]};
    } else {
        CK(cudaEventRecord(in->ev[6], st));
        CK(cudaEventRecord(in->ev[7], st));
        CK(cudaEventRecord(in->ev[8], st));
        CK(cudaStreamSynchronize(st));
    }
    in->last_npts = (int64_t)npts;
    in->last_ncl = ncl;
    in->last_nq = nq;
    // stage times from the events (at_timing, fast/apriltag_fast.h:67-69)
    auto dt = [&](int a, int b) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, in->ev[a], in->ev[b]);
        return (double)ms * 1e-3;
    };
    memset(&td->timing, 0, sizeof td->timing);
    td->timing.decimate = dt(0, 1);
    td->timing.blur = dt(1, 2);
    td->timing.threshold = dt(2, 3);
    td->timing.unionfind = dt(3, 4);
    if (npts > 0) {
        td->timing.clusters = dt(4, 5);
        td->timing.fit_quads = dt(5, 6);
    } else {
        td->timing.clusters = dt(4, 6);
    }
    td->timing.decode = dt(6, 7);
    td->timing.reconcile = dt(7, 8);
    td->timing.total = dt(0, 8);
    if (td->debug && n == 1 && fd[0].qw > 0) {
        std::vector<uint8_t> h((size_t)fd[0].qw * fd[0].qh);
        CK(cudaMemcpy(h.data(), qim, h.size(), cudaMemcpyDeviceToHost));
        at_write_pgm("debug_preprocess.pnm", h.data(), fd[0].qw, fd[0].qh);
        CK(cudaMemcpy(h.data(), thr, h.size(), cudaMemcpyDeviceToHost));
        at_write_pgm("debug_threshold.pnm", h.data(), fd[0].qw, fd[0].qh);
    }
    return true;
}

// ---------------------------------------------------------------------------
// The C ABI.

extern "C" {

at_detector *at_detector_create(void) {
    at_detector *td = (at_detector *)calloc(1, sizeof *td);
    at_internal *in = new at_internal();
    if (!td) abort();
    td->nthreads = 1;
    td->quad_decimate = 2.0f;
    td->quad_sigma = 0.0f;
    td->refine_edges = true;
    td->decode_sharpening = 0.25;
    td->debug = false;
    td->qtp.min_cluster_pixels = 24;
    td->qtp.max_nmaxima = 10;
    td->qtp.critical_rad = 0.0f;
    td->qtp.cos_critical_rad = (float)cos(10.0 * M_PI / 180.0);
    td->qtp.max_line_fit_mse = 10.0f;
    td->qtp.min_white_black_diff = 5;
    td->qtp.deglitch = false;
    td->in = in;
    if (cudaGetDevice(&in->device) != cudaSuccess || cudaStreamCreateWithFlags(&in->stream, cudaStreamNonBlocking) != cudaSuccess) {
        fprintf(stderr, "apriltag_b200: no usable CUDA device\n");
        abort();
    }
    for (int k = 0; k < 12; k++) cudaEventCreate(&in->ev[k]);
    cudaStreamCreateWithFlags(&in->side, cudaStreamNonBlocking);
    cudaStreamCreateWithFlags(&in->side2, cudaStreamNonBlocking);
    cudaStreamCreateWithFlags(&in->side3, cudaStreamNonBlocking);
    cudaEventCreateWithFlags(&in->fork, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&in->join, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&in->join2, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&in->join3, cudaEventDisableTiming);
    return td;
}

static void release_arenas(at_internal *in) {
    for (int b = 0; b < B_NBUF; b++) in->buf[b].release();
    in->h_frames.release();
    in->h_small.release();
    in->h_out.release();
}

void at_shutdown(at_detector *td) {
    if (!td) return;
    for (at_detector *h : td->in->helper) at_shutdown(h);  // the batch pipelines' arenas too
    cudaStreamSynchronize(td->in->stream);
    release_arenas(td->in);
}

void at_detector_destroy(at_detector *td) {
    if (!td) return;
    at_internal *in = td->in;
    for (at_detector *h : in->helper) at_detector_destroy(h);
    cudaStreamSynchronize(in->stream);
    release_arenas(in);
    for (int i = 0; i < AT_MAX_FAMILIES; i++)
        for (void *p : in->fam_mem[i]) cudaFree(p);
    in->dfam.release();
    for (int k = 0; k < 12; k++) cudaEventDestroy(in->ev[k]);
    if (in->chain) {
        for (cudaEvent_t e : in->chain->ev)
            if (e) cudaEventDestroy(e);
        delete in->chain;
    }
    cudaEventDestroy(in->fork);
    cudaEventDestroy(in->join);
    cudaEventDestroy(in->join2);
    cudaEventDestroy(in->join3);
    cudaStreamDestroy(in->side);
    cudaStreamDestroy(in->side2);
    cudaStreamDestroy(in->side3);
    cudaStreamDestroy(in->stream);
    delete in;
    free(td);
}

bool at_add_family(at_detector *td, const at_family *fam, int bits_corrected) {
    at_internal *in = td->in;
    if (bits_corrected < 0 || bits_corrected > 3) return false;
    if (in->nfam == AT_MAX_FAMILIES) return false;
    if (fam->ncodes >= 65536 || fam->nbits <= 0 || fam->nbits > 64) return false;
    if (fam->total_width > AT_MAX_TW || fam->width_at_border > AT_MAX_TW || fam->width_at_border < 1) {
        set_error(in, 2, "family total_width above the supported 16");
        return false;
    }
    // every bit must land in the total_width x total_width grid that the
    // sampler fills (fast/decode.c:340-361)
    int32_t minc = (fam->width_at_border - fam->total_width) / 2;
    for (int k = 0; k < fam->nbits; k++)
        if (fam->bit_x[k] - minc < 0 || fam->bit_x[k] - minc >= fam->total_width || fam->bit_y[k] - minc < 0 ||
            fam->bit_y[k] - minc >= fam->total_width) {
            set_error(in, 2, "family bit position outside the tag grid");
            return false;
        }
    int i = in->nfam;
    in->families[i] = *fam;
    in->bits[i] = bits_corrected;
    if (!upload_family(in, i)) return false;
    in->nfam++;
    in->fam_gen++;
    return true;
}

void at_clear_families(at_detector *td) {
    td->in->nfam = 0;
    td->in->fam_dirty = true;
    td->in->fam_gen++;
}

const char *at_family_name(const at_detector *td, const at_detection *d) { return td->in->families[d->family].name; }

at_detector *at_detector_clone(const at_detector *src);

// A batch spread over P pipelines (this detector and P - 1 helpers made
// like it), each taking a run of consecutive frames with about 1/P of the
// pixels; the results are joined in frame order, so they are those of one
// pipeline. Each helper runs on its own host thread.
static bool run_split(at_detector *td, const at_frame *frames, int64_t n, at_frame_result *res, int P) {
    at_internal *in = td->in;
    if (cudaSetDevice(in->device) != cudaSuccess) {
        set_error(in, 1, "cudaSetDevice failed");
        return false;
    }
    int64_t launched[AT_BATCH_SPLIT_MAX] = {};
    for (int k = 0; k < P - 1; k++) {
        if (!in->helper[k] || in->helper_gen[k] != in->fam_gen) {
            if (in->helper[k]) at_detector_destroy(in->helper[k]);
            in->helper[k] = at_detector_clone(td);
            in->helper_gen[k] = in->fam_gen;
        }
        at_detector *h = in->helper[k];
        h->quad_decimate = td->quad_decimate;
        h->quad_sigma = td->quad_sigma;
        h->refine_edges = td->refine_edges;
        h->decode_sharpening = td->decode_sharpening;
        h->qtp = td->qtp;
        h->in->err = 0;
        h->in->msg.clear();
        launched[k + 1] = h->in->launches;
    }
    // part boundaries by pixel count, each part at least one frame
    int64_t total = 0;
    for (int64_t i = 0; i < n; i++) total += frames[i].width * frames[i].height;
    int64_t cut[AT_BATCH_SPLIT_MAX + 1];
    cut[0] = 0;
    cut[P] = n;
    int64_t acc = 0, i = 0;
    for (int k = 1; k < P; k++) {
        while (i < n - (P - k) && (i < cut[k - 1] + 1 || P * (acc + frames[i].width * frames[i].height) <= k * total))
            acc += frames[i].width * frames[i].height, i++;
        cut[k] = i;
    }
    std::vector<at_frame_result> part(n);
    bool ok[AT_BATCH_SPLIT_MAX] = {};
    if (!in->chain) in->chain = new CopyChain;
    CopyChain &chain = *in->chain;
    for (int k = 0; k < P; k++)
        if (!chain.ev[k] && cudaEventCreateWithFlags(&chain.ev[k], cudaEventDisableTiming) != cudaSuccess) {
            set_error(in, 1, "cudaEventCreate failed");
            return false;
        }
    chain.done = 0;
    std::vector<std::thread> th;
    for (int k = 1; k < P; k++)
        th.emplace_back([&, k] {
            ok[k] = run_batch(in->helper[k - 1], frames + cut[k], cut[k + 1] - cut[k], part.data() + cut[k], &chain,
                              k);
        });
    ok[0] = run_batch(td, frames, cut[1], res, &chain, 0);
    for (auto &t : th) t.join();
    for (int k = 1; k < P; k++)
        if (!ok[k]) {
            if (ok[0]) set_error(in, in->helper[k - 1]->in->err, in->helper[k - 1]->in->msg);
            return false;
        }
    if (!ok[0]) return false;
    for (int k = 1; k < P; k++) {
        const at_internal *hin = in->helper[k - 1]->in;
        const int64_t base = (int64_t)in->dets.size();
        in->dets.insert(in->dets.end(), hin->dets.begin(), hin->dets.end());
        for (int64_t f = cut[k]; f < cut[k + 1]; f++)
            res[f] = at_frame_result{part[f].first + base, part[f].count, part[f].nquads};
        in->launches += hin->launches - launched[k];
    }
    return true;
}

void at_detect_batch(at_detector *td, const at_frame *frames, int64_t n, at_frame_result *results) {
    at_internal *in = td->in;
    in->err = 0;
    in->msg.clear();
    td->ndetections = 0;
    td->nquads = 0;
    int P = in->split;
    if (P > n / AT_SPLIT_MIN_FRAMES) P = (int)(n / AT_SPLIT_MIN_FRAMES);
    const bool ok = P > 1 ? run_split(td, frames, n, results, P) : run_batch(td, frames, n, results);
    if (!ok) {
        in->dets.clear();
        for (int64_t i = 0; i < n; i++) results[i] = at_frame_result{0, 0, 0};
    }
    td->detections = in->dets.data();
    td->ndetections = (int64_t)in->dets.size();
    int64_t nq = 0;
    for (int64_t i = 0; i < n; i++) nq += results[i].nquads;
    td->nquads = nq;
}

// For the server (at_server.cu): a detector with src's parameters and
// families, and the device bytes a detector's arenas hold.
at_detector *at_detector_clone(const at_detector *src) {
    at_detector *td = at_detector_create();
    at_internal *in = td->in;
    in->device = src->in->device;
    in->split = 1;  // a clone (a server worker, a batch helper) runs one pipeline
    td->nthreads = src->nthreads;
    td->quad_decimate = src->quad_decimate;
    td->quad_sigma = src->quad_sigma;
    td->refine_edges = src->refine_edges;
    td->decode_sharpening = src->decode_sharpening;
    td->debug = false;
    td->qtp = src->qtp;
    for (int i = 0; i < src->in->nfam; i++) at_add_family(td, &src->in->families[i], src->in->bits[i]);
    return td;
}

int at_register_host_buffer(void *ptr, size_t bytes) {
    if (!ptr || bytes == 0) return -1;
    if (cudaHostRegister(ptr, bytes, cudaHostRegisterPortable) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    return 0;
}

int at_unregister_host_buffer(void *ptr) {
    if (!ptr || cudaHostUnregister(ptr) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    return 0;
}

int at_detector_set_batch_split(at_detector *td, int pipelines) {
    if (pipelines < 1 || pipelines > AT_BATCH_SPLIT_MAX) return -1;
    td->in->split = pipelines;
    return 0;
}

int64_t at_detector_arena_bytes(const at_detector *td) {
    int64_t b = 0;
    for (int k = 0; k < B_NBUF; k++) b += (int64_t)td->in->buf[k].want;
    return b;
}

void at_detect(at_detector *td, const uint8_t *pixels, int64_t width, int64_t height, int64_t stride) {
    at_frame f{pixels, width, height, stride, 0};
    at_frame_result r;
    at_detect_batch(td, &f, 1, &r);
}

int64_t at_detector_diag(const at_detector *td, int what, void *dst, int64_t cap) {
    at_internal *in = td->in;
    const DBuf *B = in->buf;
    const void *src = nullptr;
    int64_t bytes = 0;
    int64_t sizes[6] = {in->last_qw, in->last_qh, in->last_npts, in->last_ncl, in->last_nq, in->launches};
    switch (what) {
    case AT_DIAG_QUAD_IMAGE: src = B[B_QIM].p, bytes = in->last_qw * in->last_qh; break;
    case AT_DIAG_THRESHOLD: src = B[B_THR].p, bytes = in->last_qw * in->last_qh; break;
    case AT_DIAG_LABELS: src = B[B_LAB].p, bytes = 4 * in->last_qw * in->last_qh; break;
    case AT_DIAG_POINTS: src = B[B_VAL2].p, bytes = 8 * in->last_npts; break;
    case AT_DIAG_CLUSTERS: src = B[B_CSTART].p, bytes = 4 * in->last_ncl; break;
    case AT_DIAG_QUADS: src = B[B_QUADSC].p, bytes = (int64_t)sizeof(GpuQuad) * in->last_nq; break;
    case AT_DIAG_SIZES:
        memcpy(dst, sizes, (size_t)(cap < 48 ? cap : 48));
        return 48;
    case AT_DIAG_ORDER_ROOTS: {
        // frame 0: the targets' GPU labels to packed numbers (node_off 0)
        uint32_t nt = 0;
        const int64_t qw = in->last_qw, qh = in->last_qh;
        if (qw * qh == 0 || !B[B_RNT].p || !B[B_RPRE].p) return 0;
        if (cudaMemcpy(&nt, B[B_RNT].p, 4, cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
        if (nt > AT_REF_MAXT) return -1;
        std::vector<uint32_t> lab(nt), root(nt), pre(qh + 1), out(2 * nt);
        if (nt > 0 && (cudaMemcpy(lab.data(), B[B_RTLAB].p, 4 * nt, cudaMemcpyDeviceToHost) != cudaSuccess ||
                       cudaMemcpy(root.data(), B[B_RTROOT].p, 4 * nt, cudaMemcpyDeviceToHost) != cudaSuccess ||
                       cudaMemcpy(pre.data(), B[B_RPRE].p, 4 * (qh + 1), cudaMemcpyDeviceToHost) != cudaSuccess))
            return -1;
        for (uint32_t t = 0; t < nt; t++) {
            const int64_t nd = lab[t];
            out[2 * t] = nd < qw * qh ? pre[nd / qw] + (uint32_t)(nd % qw) : pre[qh] + (uint32_t)(nd - qw * qh);
            out[2 * t + 1] = root[t];
        }
        const int64_t nbytes = 8 * (int64_t)nt;
        if (dst && cap > 0) memcpy(dst, out.data(), (size_t)(nbytes < cap ? nbytes : cap));
        return nbytes;
    }
    default: return -1;
    }
    int64_t n = bytes < cap ? bytes : cap;
    if (n > 0 && src && cudaMemcpy(dst, src, (size_t)n, cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    return bytes;
}

int at_detector_last_error(const at_detector *td, const char **message) {
    if (message) *message = td->in->msg.c_str();
    return td->in->err;
}

// Built-in families (fast/families.c:44-78).
static const at_family *builtin(const char *name) {
    if (name == nullptr) return nullptr;
    for (int i = 0; at_builtin_families[i]; i++)
        if (!strcmp(at_builtin_families[i]->name, name)) return at_builtin_families[i];
    return nullptr;
}
const at_family *at_family_by_name(const char *name) { return builtin(name); }
const at_family *at_tag16h5(void) { return builtin("tag16h5"); }
const at_family *at_tag25h9(void) { return builtin("tag25h9"); }
const at_family *at_tag36h10(void) { return builtin("tag36h10"); }
const at_family *at_tag36h11(void) { return builtin("tag36h11"); }
const at_family *at_tagCircle21h7(void) { return builtin("tagCircle21h7"); }
const at_family *at_tagCircle49h12(void) { return builtin("tagCircle49h12"); }
const at_family *at_tagCustom48h12(void) { return builtin("tagCustom48h12"); }
const at_family *at_tagStandard41h12(void) { return builtin("tagStandard41h12"); }
const at_family *at_tagStandard52h13(void) { return builtin("tagStandard52h13"); }

// PNM files. Contract (fast/apriltag_fast.h:126-131 of the reference):
// binary PGM (P5) or PPM (P6) with maxval 255 only; a PPM becomes gray as
// (r + 2 g + b) / 4 with integer division; at_read_pnm_into reuses
// *pixels when *cap holds width * height bytes and otherwise replaces it
// with a new malloc'd buffer (freeing the old one); false on any error.

// The next decimal number of a PNM header, after whitespace and '#'
// comments. The character after the number is left unread.
static bool pnm_number(FILE *fp, int64_t *value) {
    int c;
    for (;;) {
        c = getc(fp);
        if (c == '#') {
            do c = getc(fp);
            while (c != '\n' && c != EOF);
        } else if (!(c == ' ' || c == '\t' || c == '\r' || c == '\n')) {
            break;
        }
    }
    if (c < '0' || c > '9') return false;
    int64_t v = 0;
    for (; c >= '0' && c <= '9'; c = getc(fp)) {
        if (v > ((int64_t)1 << 40)) return false;  // no real image is this large
        v = v * 10 + (c - '0');
    }
    if (c != EOF) ungetc(c, fp);
    *value = v;
    return true;
}

static bool pnm_load(FILE *fp, int64_t *width, int64_t *height, uint8_t **pixels, int64_t *cap) {
    char magic[2];
    if (fread(magic, 1, 2, fp) != 2 || magic[0] != 'P' || (magic[1] != '5' && magic[1] != '6')) return false;
    const int channels = magic[1] == '5' ? 1 : 3;
    int64_t w = 0, h = 0, maxval = 0;
    if (!pnm_number(fp, &w) || !pnm_number(fp, &h) || !pnm_number(fp, &maxval)) return false;
    if (w <= 0 || h <= 0 || maxval != 255 || w > ((int64_t)1 << 20) || h > ((int64_t)1 << 20)) return false;
    if (getc(fp) == EOF) return false;  // the one whitespace byte that ends the header
    const size_t npx = (size_t)w * (size_t)h;
    uint8_t *dst = *pixels;
    const bool fresh = dst == nullptr || *cap < (int64_t)npx;
    if (fresh && (dst = (uint8_t *)malloc(npx)) == nullptr) return false;
    bool ok = true;
    if (channels == 1) {
        ok = fread(dst, 1, npx, fp) == npx;
    } else {
        std::vector<uint8_t> rgb((size_t)w * 3);
        for (int64_t y = 0; ok && y < h; y++) {
            ok = fread(rgb.data(), 1, rgb.size(), fp) == rgb.size();
            for (int64_t x = 0; ok && x < w; x++)
                dst[y * w + x] = (uint8_t)((rgb[3 * x] + 2 * rgb[3 * x + 1] + rgb[3 * x + 2]) / 4);
        }
    }
    if (!ok) {
        if (fresh) free(dst);
        return false;
    }
    if (fresh) {
        free(*pixels);
        *pixels = dst;
        *cap = (int64_t)npx;
    }
    *width = w;
    *height = h;
    return true;
}

bool at_read_pnm_into(const char *path, int64_t *width, int64_t *height, uint8_t **pixels, int64_t *cap) {
    FILE *fp = fopen(path, "rb");
    if (fp == nullptr) return false;
    const bool ok = pnm_load(fp, width, height, pixels, cap);
    fclose(fp);
    return ok;
}

bool at_read_pnm(const char *path, int64_t *width, int64_t *height, uint8_t **pixels) {
    int64_t cap = 0;
    *pixels = nullptr;
    return at_read_pnm_into(path, width, height, pixels, &cap);
}

bool at_write_pgm(const char *path, const uint8_t *pixels, int64_t width, int64_t height) {
    char header[64];
    const int hl = snprintf(header, sizeof header, "P5\n%lld %lld\n255\n", (long long)width, (long long)height);
    FILE *fp = fopen(path, "wb");
    if (fp == nullptr) return false;
    const size_t n = (size_t)width * (size_t)height;
    bool ok = fwrite(header, 1, (size_t)hl, fp) == (size_t)hl && fwrite(pixels, 1, n, fp) == n;
    ok = (fclose(fp) == 0) && ok;
    return ok;
}

}  // extern "C"
