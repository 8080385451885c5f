// The sm_100a kernels of the AprilTag detection path.
//
// Every kernel takes a batch of frames (FrameDesc array) and works on all
// of them at once: blockIdx.y is the frame, blockIdx.x strides over the
// frame's rows, pixels or items. Compiled with --fmad=false, -prec-div and
// -prec-sqrt: each floating point operation is rounded on its own, as the
// reference (built with -ffp-contract=off) rounds it, so the results are
// bit-identical. Each kernel names the reference lines it follows.
#include <cuda_runtime.h>
#include <stdint.h>

#include "at_gpu.h"
#include "at_device.cuh"
#include "at_kernels.h"

// ---------------------------------------------------------------------------
// Small helpers.

// C's (int) of a double on x86-64: truncation, INT_MIN out of range or NaN
// (fast/decode.c:8-11).
__device__ __forceinline__ int64_t c_int(double x) {
    if (x > -2147483649.0 && x < 2147483648.0) return (int64_t)x;
    return -2147483648LL;
}

#define FRAME_LOOP_BEGIN(n_items)                                                               \
    const FrameDesc fd = frames[blockIdx.y];                                                   \
    for (int64_t it = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; it < (n_items);          \
         it += (int64_t)gridDim.x * blockDim.x) {
#define FRAME_LOOP_END }

// ---------------------------------------------------------------------------
// 1. Decimation (fast/image.c:6-88). A block per output row, a thread per
// output pixel.

__global__ void k_decimate(const FrameDesc *frames, const uint8_t *img, uint8_t *qim, float factor) {
    const FrameDesc f = frames[blockIdx.y];
    const uint8_t *src = f.img;
    const int64_t stride = f.stride;
    const int qw = (int)f.qw, qh = (int)f.qh;
    for (int y = blockIdx.x; y < qh; y += gridDim.x) {
        uint8_t *out = qim + f.q_off + (int64_t)y * qw;
        if (factor == 1.5f) {
            // 3x3 weights over 9; output pixel (2k+dx, 2m+dy) from input
            // block (3k.., 3m..) (fast/image.c:50-62)
            const int m = y >> 1;
            const uint8_t *r0 = src + (int64_t)(3 * m) * stride, *r1 = r0 + stride, *r2 = r1 + stride;
            for (int x = threadIdx.x; x < qw; x += blockDim.x) {
                const int k3 = 3 * (x >> 1);
                const int e = r1[k3 + 1];
                int v;
                if ((y & 1) == 0)
                    v = (x & 1) == 0 ? 4 * r0[k3] + 2 * r0[k3 + 1] + 2 * r1[k3] + e
                                     : 4 * r0[k3 + 2] + 2 * r0[k3 + 1] + 2 * r1[k3 + 2] + e;
                else
                    v = (x & 1) == 0 ? 4 * r2[k3] + 2 * r1[k3] + 2 * r2[k3 + 1] + e
                                     : 4 * r2[k3 + 2] + 2 * r1[k3 + 2] + 2 * r2[k3 + 1] + e;
                out[x] = (uint8_t)(v / 9);
            }
        } else if (factor > 1.0f) {
            const int k = (int)factor;
            if (k == 2) {
                // 2x2 box; the part of the row below the largest multiple of
                // 32 rounds twice (the C library's AVX2 path), the rest once
                // (fast/image.c:26-46)
                const uint8_t *r0 = src + (int64_t)(2 * y) * stride, *r1 = r0 + stride;
                const int xv = qw - qw % 32;
                auto box = [&](int x, int a, int b, int c, int d) {
                    out[x] = x < xv ? (uint8_t)((((a + c + 1) >> 1) + ((b + d + 1) >> 1) + 1) >> 1)
                                    : (uint8_t)((a + b + c + d + 2) >> 2);
                };
                if ((((uintptr_t)r0 | (uintptr_t)r1) & 7) == 0) {
                    // four outputs a thread from 8-byte loads of both rows
                    for (int x4 = 4 * threadIdx.x; x4 < qw; x4 += 4 * blockDim.x) {
                        if (x4 + 3 < qw) {
                            const uint2 p = *reinterpret_cast<const uint2 *>(r0 + 2 * x4);
                            const uint2 q = *reinterpret_cast<const uint2 *>(r1 + 2 * x4);
#pragma unroll
                            for (int u = 0; u < 4; u++) {
                                const uint32_t pw = u < 2 ? p.x : p.y, qv = u < 2 ? q.x : q.y;
                                const int sh = 16 * (u & 1);
                                box(x4 + u, (pw >> sh) & 255, (pw >> (sh + 8)) & 255, (qv >> sh) & 255,
                                    (qv >> (sh + 8)) & 255);
                            }
                        } else {
                            for (int x = x4; x < qw; x++) box(x, r0[2 * x], r0[2 * x + 1], r1[2 * x], r1[2 * x + 1]);
                        }
                    }
                } else {
                    for (int x = threadIdx.x; x < qw; x += blockDim.x)
                        box(x, r0[2 * x], r0[2 * x + 1], r1[2 * x], r1[2 * x + 1]);
                }
            } else {
                const uint8_t *r0 = src + (int64_t)y * k * stride;
                for (int x = threadIdx.x; x < qw; x += blockDim.x) out[x] = r0[(int64_t)x * k];
            }
        } else {
            const uint8_t *r0 = src + (int64_t)y * stride;
            for (int x = threadIdx.x; x < qw; x += blockDim.x) out[x] = r0[x];
        }
    }
}

// ---------------------------------------------------------------------------
// 2. Blur / sharpen of the quad image (fast/image.c:93-173). The taps are
// integers made on the host. A separable pass: `dir` 0 filters rows, 1
// columns. The line's first nk/2 outputs and its tail copy the input; the
// wide variant (images of 65536 pixels or more) filters one more output.

__global__ void k_blur_pass(const FrameDesc *frames, const uint8_t *in, uint8_t *out, BlurTaps taps, int dir) {
    const FrameDesc f = frames[blockIdx.y];
    const int qw = (int)f.qw, qh = (int)f.qh;
    const bool wide = (int64_t)qw * qh >= 65536;
    const int nk = taps.n, r = nk / 2;
    const int len = dir == 0 ? qw : qh;
    const int m = wide ? len - nk + 1 : len - nk;
    const int64_t step = dir == 0 ? 1 : qw;
    for (int y = blockIdx.x; y < qh; y += gridDim.x) {
        for (int x = threadIdx.x; x < qw; x += blockDim.x) {
            const int pos = dir == 0 ? x : y;
            const uint8_t *line = in + f.q_off + (dir == 0 ? (int64_t)y * qw : (int64_t)x);
            uint8_t v;
            if (pos >= r && pos - r < m) {
                uint32_t acc = 0;
                for (int j = 0; j < nk; j++) acc += (uint32_t)taps.k[j] * line[(int64_t)(pos - r + j) * step];
                v = (uint8_t)(acc >> 8);
            } else {
                v = line[(int64_t)pos * step];
            }
            out[f.q_off + (int64_t)y * qw + x] = v;
        }
    }
}

// sharpen: im = clamp(2 * orig - blurred) (fast/image.c:484-489); else copy
__global__ void k_blur_finish(const FrameDesc *frames, const uint8_t *blurred, uint8_t *qim, int sharpen) {
    const FrameDesc f = frames[blockIdx.y];
    const int64_t n = (int64_t)f.qw * f.qh;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint8_t b = blurred[f.q_off + i];
        if (sharpen) {
            int v = 2 * (int)qim[f.q_off + i] - b;
            qim[f.q_off + i] = (uint8_t)(v < 0 ? 0 : v > 255 ? 255 : v);
        } else {
            qim[f.q_off + i] = b;
        }
    }
}

// ---------------------------------------------------------------------------
// 3. Adaptive threshold (fast/threshold.c:15-161). First each 4x4 tile's
// max and min, then per pixel the max and min of its tile's 3x3 tile
// neighbourhood (cells outside the grid left out).

__global__ void k_tile_minmax(const FrameDesc *frames, const uint8_t *qim, uint8_t *tmax, uint8_t *tmin) {
    const FrameDesc f = frames[blockIdx.y];
    const int64_t tw = f.qw / 4, th = f.qh / 4, n = tw * th;
    // 4-byte loads when every tile row is 4-byte aligned, else byte loads
    const bool al = (((uintptr_t)(qim + f.q_off)) & 3) == 0 && (f.qw & 3) == 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int64_t ty = i / tw, tx = i - ty * tw;
        const uint8_t *p = qim + f.q_off + 4 * ty * f.qw + 4 * tx;
        uint32_t hi = 0, lo = 255;
        if (al) {
            uint32_t mx = 0, mn = 0xffffffffu;
#pragma unroll
            for (int dy = 0; dy < 4; dy++) {
                const uint32_t v = *reinterpret_cast<const uint32_t *>(p + dy * f.qw);
                mx = __vmaxu4(mx, v);
                mn = __vminu4(mn, v);
            }
            hi = max(max(mx & 255u, mx >> 8 & 255u), max(mx >> 16 & 255u, mx >> 24));
            lo = min(min(mn & 255u, mn >> 8 & 255u), min(mn >> 16 & 255u, mn >> 24));
        } else {
#pragma unroll
            for (int dy = 0; dy < 4; dy++) {
                const uint8_t *r = p + dy * f.qw;
                hi = max(hi, (uint32_t)max(max(r[0], r[1]), max(r[2], r[3])));
                lo = min(lo, (uint32_t)min(min(r[0], r[1]), min(r[2], r[3])));
            }
        }
        tmax[f.tile_off + i] = (uint8_t)hi;
        tmin[f.tile_off + i] = (uint8_t)lo;
    }
}

// The streaming stages fused for decimate 2 without blur (fast/image.c:26-46
// and fast/threshold.c:15-161 in one pass): a block takes a region of
// DT_ROWS x DT_COLS 4x4 cells of one frame. It reads the input rows of the
// region's tiles and of a one-tile halo around them (16-byte loads), makes
// each tile's 16 quad pixels in registers, keeps the region's own quad
// pixels and every tile's max/min in shared memory, then per cell the 3x3
// tile neighbourhood's max/min and per pixel the threshold, and writes the
// quad image and the threshold image once (16-byte stores). Cells right of
// the last whole tile column or below the last whole tile row (no tile of
// their own) use the nearest tile's neighbourhood and are never flat.
#define DT_ROWS 16
#define DT_COLS 64
#define DT_THREADS 256

// 2x2 box of the reference's decimate2_row: columns below the largest
// multiple of 32 round twice (its AVX2 path), the rest once.
__device__ __forceinline__ uint32_t box2(int x, int xv, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    return x < xv ? ((((a + c + 1) >> 1) + ((b + d + 1) >> 1) + 1) >> 1) : ((a + b + c + d + 2) >> 2);
}

__global__ void __launch_bounds__(DT_THREADS) k_decimate_threshold(const FrameDesc *frames, uint8_t *qim, uint8_t *thr,
                                                                   int32_t diff) {
    __shared__ __align__(16) uint8_t s_q[4 * DT_ROWS][4 * DT_COLS];
    __shared__ uint8_t s_tmax[DT_ROWS + 2][DT_COLS + 4], s_tmin[DT_ROWS + 2][DT_COLS + 4];
    __shared__ uint16_t s_cell[DT_ROWS][DT_COLS];  // threshold | flat << 8
    const FrameDesc f = frames[blockIdx.y];
    const int qw = f.qw, qh = f.qh, tw = qw / 4, th = qh / 4;
    const int cw = (qw + 3) / 4, ch = (qh + 3) / 4;
    const int ncb = (cw + DT_COLS - 1) / DT_COLS;
    const int rb = blockIdx.x / ncb, cb = blockIdx.x - rb * ncb;
    const int cy0 = rb * DT_ROWS, cx0 = cb * DT_COLS;
    if (cy0 >= ch) return;
    const int cy1 = min(cy0 + DT_ROWS, ch), cx1 = min(cx0 + DT_COLS, cw);  // own cells
    // tiles needed: the own cells' tiles (clamped to the grid) and one around
    const int ty0 = max(min(cy0, th - 1) - 1, 0), ty1 = min(min(cy1 - 1, th - 1) + 1, th - 1);
    const int tx0 = max(min(cx0, tw - 1) - 1, 0), tx1 = min(min(cx1 - 1, tw - 1) + 1, tw - 1);
    const int px0 = tx0 & ~1;  // tiles go in pairs (16 input bytes) from an even tile
    const int npair = (tx1 - px0) / 2 + 1, ntr = ty1 - ty0 + 1;
    const int xv = qw - qw % 32;
    const uint8_t *img = f.img;
    const int64_t st = f.stride;
    const bool al16 = ((((uintptr_t)img) | (uintptr_t)st) & 15) == 0;
    // 1. tiles: max/min of each, and the own tiles' quad pixels
    for (int i = threadIdx.x; i < npair * ntr; i += DT_THREADS) {
        const int r = i / npair, tp = px0 + 2 * (i - r * npair);
        const int ty = ty0 + r;
        uint32_t qw4[2][4];  // [tile][row]: the tile row's 4 quad pixels as bytes of a word
        if (al16 && tp + 1 < tw && 4 * tp + 8 <= xv) {
            // 16 input bytes of two rows give 8 quad pixels: the byte average
            // of the rows, then of even and odd columns (the reference's two
            // rounded averages of its AVX2 path)
#pragma unroll
            for (int dy = 0; dy < 4; dy++) {
                const uint8_t *r0 = img + (int64_t)(8 * ty + 2 * dy) * st + 8 * tp;
                const uint4 u = *reinterpret_cast<const uint4 *>(r0), v = *reinterpret_cast<const uint4 *>(r0 + st);
                const uint32_t a0 = __vavgu4(u.x, v.x), a1 = __vavgu4(u.y, v.y), a2 = __vavgu4(u.z, v.z),
                               a3 = __vavgu4(u.w, v.w);
                qw4[0][dy] = __vavgu4(__byte_perm(a0, a1, 0x6420), __byte_perm(a0, a1, 0x7531));
                qw4[1][dy] = __vavgu4(__byte_perm(a2, a3, 0x6420), __byte_perm(a2, a3, 0x7531));
            }
        } else {
#pragma unroll
            for (int dy = 0; dy < 4; dy++) {
                const uint8_t *r0 = img + (int64_t)(8 * ty + 2 * dy) * st + 8 * tp, *r1 = r0 + st;
                uint32_t a[4], b[4];  // 16 input bytes of each row, as words
                if (al16 && tp + 1 < tw) {
                    const uint4 u = *reinterpret_cast<const uint4 *>(r0), v = *reinterpret_cast<const uint4 *>(r1);
                    a[0] = u.x, a[1] = u.y, a[2] = u.z, a[3] = u.w;
                    b[0] = v.x, b[1] = v.y, b[2] = v.z, b[3] = v.w;
                } else {
                    const int nb = tp + 1 < tw ? 16 : 8;
#pragma unroll
                    for (int w = 0; w < 4; w++) {
                        a[w] = b[w] = 0;
#pragma unroll
                        for (int k = 0; k < 4; k++)
                            if (4 * w + k < nb) {
                                a[w] |= (uint32_t)r0[4 * w + k] << (8 * k);
                                b[w] |= (uint32_t)r1[4 * w + k] << (8 * k);
                            }
                    }
                }
                qw4[0][dy] = qw4[1][dy] = 0;
#pragma unroll
                for (int o = 0; o < 8; o++) {  // quad pixel 4 tp + o of row 4 ty + dy
                    const uint32_t w0 = a[o >> 1], w1 = b[o >> 1];
                    const int sh = 16 * (o & 1);
                    qw4[o >> 2][dy] |= box2(4 * tp + o, xv, (w0 >> sh) & 255, (w0 >> (sh + 8)) & 255, (w1 >> sh) & 255,
                                            (w1 >> (sh + 8)) & 255)
                                       << (8 * (o & 3));
                }
            }
        }
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const int tx = tp + k;
            if (tx < tx0 || tx > tx1) continue;
            uint32_t mx = qw4[k][0], mn = qw4[k][0];
#pragma unroll
            for (int dy = 1; dy < 4; dy++) {
                mx = __vmaxu4(mx, qw4[k][dy]);
                mn = __vminu4(mn, qw4[k][dy]);
            }
            s_tmax[ty - ty0][tx - tx0] = (uint8_t)max(max(mx & 255u, mx >> 8 & 255u), max(mx >> 16 & 255u, mx >> 24));
            s_tmin[ty - ty0][tx - tx0] = (uint8_t)min(min(mn & 255u, mn >> 8 & 255u), min(mn >> 16 & 255u, mn >> 24));
            if (ty >= cy0 && ty < cy1 && tx >= cx0 && tx < cx1) {
#pragma unroll
                for (int dy = 0; dy < 4; dy++)
                    *reinterpret_cast<uint32_t *>(&s_q[4 * (ty - cy0) + dy][4 * (tx - cx0)]) = qw4[k][dy];
            }
        }
    }
    __syncthreads();
    // 2. per own cell: its tile's 3x3 neighbourhood (clipped to the grid)
    for (int i = threadIdx.x; i < (cy1 - cy0) * (cx1 - cx0); i += DT_THREADS) {
        const int cy = cy0 + i / (cx1 - cx0), cx = cx0 + i % (cx1 - cx0);
        const int ty = min(cy, th - 1), tx = min(cx, tw - 1);
        const bool may_flat = cy < th && cx < tw;
        uint32_t hi = 0, lo = 255;
        for (int yy = max(ty - 1, 0); yy <= min(ty + 1, th - 1); yy++)
            for (int xx = max(tx - 1, 0); xx <= min(tx + 1, tw - 1); xx++) {
                hi = max(hi, (uint32_t)s_tmax[yy - ty0][xx - tx0]);
                lo = min(lo, (uint32_t)s_tmin[yy - ty0][xx - tx0]);
            }
        const uint32_t t = lo + (hi - lo) / 2;
        const bool flat = may_flat && (int32_t)(hi - lo) < diff;
        s_cell[cy - cy0][cx - cx0] = (uint16_t)(t | (flat ? 256u : 0u));
    }
    __syncthreads();
    // 3. the own pixels, 16 a thread: quad image and threshold image
    const int y0 = 4 * cy0, y1 = min(4 * cy1, qh), x0 = 4 * cx0, x1 = min(4 * cx1, qw);
    const int nseg = (x1 - x0 + 15) / 16;
    const bool st16 = ((((uintptr_t)(qim + f.q_off)) | ((uintptr_t)(thr + f.q_off)) | (uintptr_t)qw) & 15) == 0;
    for (int i = threadIdx.x; i < (y1 - y0) * nseg; i += DT_THREADS) {
        const int y = y0 + i / nseg, xs = x0 + 16 * (i % nseg);
        const int n = min(16, x1 - xs);
        const bool whole_tiles = y < 4 * th;
        if (st16 && n == 16 && whole_tiles && xs + 16 <= 4 * tw) {
            // 16 pixels of 4 cells, 4 at a time: above the cell's threshold
            // 255, else 0; a flat cell 127
            const uint4 q = *reinterpret_cast<const uint4 *>(&s_q[y - y0][xs - x0]);
            const uint32_t qa[4] = {q.x, q.y, q.z, q.w};
            uint32_t t4[4];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const uint32_t c = s_cell[(y >> 2) - cy0][(xs >> 2) - cx0 + k];
                t4[k] = (c & 256u) ? 0x7f7f7f7fu : __vcmpgtu4(qa[k], (c & 255u) * 0x01010101u);
            }
            const int64_t o = f.q_off + (int64_t)y * qw + xs;
            *reinterpret_cast<uint4 *>(qim + o) = q;
            *reinterpret_cast<uint4 *>(thr + o) = make_uint4(t4[0], t4[1], t4[2], t4[3]);
            continue;
        }
        uint32_t qv[4] = {0, 0, 0, 0}, tv[4] = {0, 0, 0, 0};
#pragma unroll
        for (int o = 0; o < 16; o++) {
            if (o >= n) break;
            const int x = xs + o;
            uint32_t v;
            if (whole_tiles && x < 4 * tw) {
                v = s_q[y - y0][x - x0];
            } else {  // a pixel of no tile: decimated here
                const uint8_t *r0 = img + (int64_t)(2 * y) * st + 2 * x, *r1 = r0 + st;
                v = box2(x, xv, r0[0], r0[1], r1[0], r1[1]);
            }
            const uint32_t c = s_cell[(y >> 2) - cy0][(x >> 2) - cx0];
            const uint32_t tb = (c & 256u) ? 127u : (v > (c & 255u) ? 255u : 0u);
            qv[o >> 2] |= v << (8 * (o & 3));
            tv[o >> 2] |= tb << (8 * (o & 3));
        }
        const int64_t o = f.q_off + (int64_t)y * qw + xs;
        if (st16 && n == 16) {
            *reinterpret_cast<uint4 *>(qim + o) = make_uint4(qv[0], qv[1], qv[2], qv[3]);
            *reinterpret_cast<uint4 *>(thr + o) = make_uint4(tv[0], tv[1], tv[2], tv[3]);
        } else {
            for (int k = 0; k < n; k++) {
                qim[o + k] = (uint8_t)(qv[k >> 2] >> (8 * (k & 3)));
                thr[o + k] = (uint8_t)(tv[k >> 2] >> (8 * (k & 3)));
            }
        }
    }
}

// A thread per 4x4 tile: the max and min of its 3x3 tile neighbourhood
// (cells outside the grid left out) once, then its 16 pixels. Pixels right
// of the last whole tile column use that column and are never 127; rows
// below the last whole tile row use that row and are never 127
// (fast/threshold.c:85-91, 144-148): the partial tiles there clamp.
__global__ void k_threshold(const FrameDesc *frames, const uint8_t *qim, const uint8_t *tmax, const uint8_t *tmin,
                            uint8_t *thr, int32_t diff) {
    const FrameDesc f = frames[blockIdx.y];
    const int qw = (int)f.qw, qh = (int)f.qh;
    const int tw = qw / 4, th = qh / 4, cw = (qw + 3) / 4, ch = (qh + 3) / 4;
    const int n = cw * ch;
    const uint8_t *tx_max = tmax + f.tile_off, *tx_min = tmin + f.tile_off;
    const bool al = ((((uintptr_t)(qim + f.q_off)) | ((uintptr_t)(thr + f.q_off))) & 3) == 0 && (qw & 3) == 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int cy = i / cw, cx = i - cy * cw;
        int ty = cy, tx = cx;
        bool may_flat = true;
        if (ty >= th) {
            ty = th - 1;
            may_flat = false;
        }
        if (tx >= tw) {
            tx = tw - 1;
            may_flat = false;
        }
        uint32_t hi = 0, lo = 255;
        const int y0t = ty - 1 > 0 ? ty - 1 : 0, y1t = ty + 1 < th - 1 ? ty + 1 : th - 1;
        const int x0t = tx - 1 > 0 ? tx - 1 : 0, x1t = tx + 1 < tw - 1 ? tx + 1 : tw - 1;
        for (int yy = y0t; yy <= y1t; yy++)
            for (int xx = x0t; xx <= x1t; xx++) {
                hi = max(hi, (uint32_t)tx_max[yy * tw + xx]);
                lo = min(lo, (uint32_t)tx_min[yy * tw + xx]);
            }
        const uint32_t t = lo + (hi - lo) / 2;
        const bool flat = may_flat && (int32_t)(hi - lo) < diff;
        const int x0 = 4 * cx, y0 = 4 * cy;
        const int xe = x0 + 4 < qw ? x0 + 4 : qw, ye = y0 + 4 < qh ? y0 + 4 : qh;
        if (al && xe == x0 + 4) {
            // a whole tile row at a time: per byte 255 above t, else 0
            const uint32_t t4 = t * 0x01010101u;
            for (int y = y0; y < ye; y++) {
                const int64_t o = f.q_off + (int64_t)y * qw + x0;
                const uint32_t v = *reinterpret_cast<const uint32_t *>(qim + o);
                *reinterpret_cast<uint32_t *>(thr + o) = flat ? 0x7f7f7f7fu : __vcmpgtu4(v, t4);
            }
        } else {
            for (int y = y0; y < ye; y++) {
                const int64_t o = f.q_off + (int64_t)y * qw;
                for (int x = x0; x < xe; x++) thr[o + x] = flat ? 127 : (qim[o + x] > t ? 255 : 0);
            }
        }
    }
}

// Deglitch (fast/threshold.c:173-193): 3x3 dilate into tmp (its border
// zero), then 3x3 erode back; the image border keeps its values.
__global__ void k_morph(const FrameDesc *frames, const uint8_t *in, uint8_t *out, int dilate) {
    const FrameDesc f = frames[blockIdx.y];
    const int qw = (int)f.qw, qh = (int)f.qh;
    for (int y = blockIdx.x; y < qh; y += gridDim.x) {
        const int64_t row = f.q_off + (int64_t)y * qw;
        for (int x = threadIdx.x; x < qw; x += blockDim.x) {
            const bool border = x == 0 || y == 0 || x == qw - 1 || y == qh - 1;
            if (border) {
                if (dilate) out[row + x] = 0;
                continue;
            }
            uint32_t m = dilate ? 0 : 255;
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    const uint32_t v = in[row + (int64_t)dy * qw + x + dx];
                    m = dilate ? max(m, v) : min(m, v);
                }
            out[row + x] = (uint8_t)m;
        }
    }
}

// ---------------------------------------------------------------------------
// 4-5. Runs and connected components over runs.
//
// 5. Connected components over runs (fast/unionfind.c:89-196): the same
// pairs of runs join as in the reference; lock-free union that links the
// larger root under the smaller, so every component's root is its smallest
// node id (the label the cluster order is defined by).

__device__ __forceinline__ uint32_t uf_find(uint32_t *par, uint32_t x) {
    volatile uint32_t *p = par;
    uint32_t px = p[x];
    while (px != x) {
        uint32_t ppx = p[px];
        if (ppx == px) return px;
        p[x] = ppx;  // path halving: only ever an ancestor
        x = ppx;
        px = p[x];
    }
    return x;
}

// Roots are linked in the order of a bijective hash of their ids: one fixed
// total order, so concurrent links can never form a cycle, and a random one,
// so trees stay shallow (linking by id would chain the pieces of a row).
// The label of a component, its smallest node id, is tracked apart.
__device__ __forceinline__ uint32_t uf_rank(uint32_t x) {
    uint32_t h = x * 0x9e3779b1u;
    return h ^ (h >> 16);
}

__device__ __forceinline__ void uf_unite(uint32_t *par, uint32_t a, uint32_t b) {
    for (;;) {
        a = uf_find(par, a);
        b = uf_find(par, b);
        if (a == b) return;
        if (uf_rank(a) < uf_rank(b)) {
            uint32_t t = a;
            a = b;
            b = t;
        }
        if (atomicCAS(par + a, a, b) == a) return;
    }
}

// The runs of row y of slots [base, base + n) that touch run (a0, a1, v),
// in order, by binary search for the first with end + 1 >= a0.
#define FOR_TOUCHING(SE, V, base, n, a0, a1, v, k, BODY)                                 \
    {                                                                                     \
        int64_t lo_ = 0, hi_ = (n);                                                       \
        while (lo_ < hi_) {                                                               \
            int64_t mid_ = (lo_ + hi_) >> 1;                                              \
            if ((int64_t)((SE)[(base) + mid_] >> 16) + 1 < (a0))                          \
                lo_ = mid_ + 1;                                                           \
            else                                                                          \
                hi_ = mid_;                                                               \
        }                                                                                 \
        for (int64_t k = lo_; k < (n) && (int64_t)((SE)[(base) + k] & 0xffff) <= (a1) + 1; k++) { \
            if ((V)[(base) + k] != (v)) continue;                                         \
            if (runs_touch((a0), (a1), (SE)[(base) + k] & 0xffff, (SE)[(base) + k] >> 16, (v))) BODY \
        }                                                                                 \
    }

// The flat form of the same union-find: one block per row, one thread per
// run, links in global memory (hash-ordered, so trees stay shallow), then
// one pass that sums each component's pixels and smallest node at its root.
#define ROW_STAGE 4096

__global__ void __launch_bounds__(256) k_row_runs(const FrameDesc *frames, const uint8_t *thr, RunArrays runs,
                                                  uint32_t *row_nruns) {
    // a warp per row: runs of equal value over columns [0, qw - 2], 32
    // columns at a time (ballots of run starts), 127 runs not stored
    const FrameDesc f = frames[blockIdx.y];
    const int lane = threadIdx.x & 31;
    const uint32_t lt = (1u << lane) - 1u;
    const int64_t wpb = blockDim.x >> 5;
    for (int64_t y = blockIdx.x * wpb + (threadIdx.x >> 5); y < f.qh; y += gridDim.x * wpb) {
        const uint8_t *row = thr + f.q_off + y * f.qw;
        const int64_t base = f.node_off + y * f.qw;
        const int64_t xmax = f.qw - 2;
        int64_t count = 0, open = -1;
        for (int64_t x0 = 0; x0 <= xmax; x0 += 32) {
            int64_t x = x0 + lane;
            bool valid = x <= xmax;
            uint8_t v = valid ? row[x] : 0;
            bool start = valid && (x == 0 || row[x - 1] != v);
            uint32_t S = __ballot_sync(0xffffffffu, start);
            uint32_t N = __ballot_sync(0xffffffffu, start && v != 127);
            if (start) {
                uint32_t below = S & lt;
                int64_t prev_slot;
                if (below) {
                    int pl = 31 - __clz(below);
                    prev_slot = (N >> pl & 1u) ? count + __popc(N & ((1u << pl) - 1u)) : -1;
                } else {
                    prev_slot = open;
                }
                if (prev_slot >= 0) runs.end[base + prev_slot] = (uint16_t)(x - 1);
                if (v != 127) {
                    int64_t sl = base + count + __popc(N & lt);
                    runs.start[sl] = (uint16_t)x;
                    runs.v[sl] = v;
                    runs.parent[sl] = (uint32_t)sl;
                    runs.px[sl] = 0;
                    runs.minid[sl] = 0xffffffffu;
                }
            }
            if (S) {
                int ls = 31 - __clz(S);
                open = (N >> ls & 1u) ? count + __popc(N & ((1u << ls) - 1u)) : -1;
            }
            count += __popc(N);
        }
        if (lane == 0) {
            if (open >= 0) runs.end[base + open] = (uint16_t)xmax;
            row_nruns[f.row0 + y] = (uint32_t)count;
            int64_t vn = f.node_off + (int64_t)f.qw * f.qh + y;
            runs.parent[vn] = (uint32_t)vn;
            runs.px[vn] = 0;
            runs.minid[vn] = 0xffffffffu;
        }
    }
}

__global__ void __launch_bounds__(256) k_row_union(const FrameDesc *frames, const uint8_t *thr, RunArrays runs,
                                                   const uint32_t *row_nruns) {
    __shared__ uint32_t s_se[ROW_STAGE];
    __shared__ uint8_t s_v[ROW_STAGE];
    const FrameDesc f = frames[blockIdx.y];
    for (int64_t y = 1 + blockIdx.x; y < f.qh; y += gridDim.x) {
        const int64_t cur = f.node_off + y * f.qw, prev = cur - f.qw;
        const int64_t ncur = row_nruns[f.row0 + y], nprev = row_nruns[f.row0 + y - 1];
        const bool staged = nprev <= ROW_STAGE;
        __syncthreads();
        if (staged)
            for (int64_t t = threadIdx.x; t < nprev; t += blockDim.x) {
                s_se[t] = (uint32_t)runs.start[prev + t] | (uint32_t)runs.end[prev + t] << 16;
                s_v[t] = runs.v[prev + t];
            }
        __syncthreads();
        for (int64_t i = threadIdx.x; i < ncur; i += blockDim.x) {
            int64_t a0 = runs.start[cur + i], a1 = runs.end[cur + i];
            uint8_t v = runs.v[cur + i];
            if (staged) {
                FOR_TOUCHING(s_se, s_v, 0, nprev, a0, a1, v, kk,
                             { uf_unite(runs.parent, (uint32_t)(cur + i), (uint32_t)(prev + kk)); })
            } else {
                int64_t lo = 0, hi = nprev;
                while (lo < hi) {
                    int64_t mid = (lo + hi) >> 1;
                    if ((int64_t)runs.end[prev + mid] + 1 < a0)
                        lo = mid + 1;
                    else
                        hi = mid;
                }
                for (int64_t kk = lo; kk < nprev && (int64_t)runs.start[prev + kk] <= a1 + 1; kk++) {
                    if (runs.v[prev + kk] != v) continue;
                    if (runs_touch(a0, a1, runs.start[prev + kk], runs.end[prev + kk], v))
                        uf_unite(runs.parent, (uint32_t)(cur + i), (uint32_t)(prev + kk));
                }
            }
        }
        if (threadIdx.x == 0 && ncur > 0) {
            int64_t last = cur + ncur - 1;
            const uint8_t *above = thr + f.q_off + (y - 1) * f.qw;
            if (runs.end[last] == f.qw - 2 && runs.v[last] == 255 && above[f.qw - 1] == 255 && above[f.qw - 2] != 255)
                uf_unite(runs.parent, (uint32_t)last, (uint32_t)(f.node_off + (int64_t)f.qw * f.qh + y - 1));
        }
    }
}

// The same unions in bands: a block takes UB_ROWS rows of a frame and does
// the unions between those rows in shared memory over band-local ids (the
// larger id hooked under the smaller, lock-free, so a local root is its
// set's smallest node of the band); every node then points at its local
// root in global memory. k_band_join then joins the bands in global memory
// (each band's first row with the row above, hash-ordered links between
// roots as in uf_unite) and adds the last-column links of every row. The
// same pairs are joined as by k_row_union, so the partition is the same. A
// band with more than UB_CAP runs joins its rows in global memory instead.
#define UB_ROWS 8
#define UB_CAP 3072
#define UB_PAIRS 3072  // touching pairs listed per band, at most

__device__ __forceinline__ uint32_t lu_find(volatile uint32_t *par, uint32_t x) {
    uint32_t p = par[x];
    while (p != x) {
        const uint32_t pp = par[p];
        if (pp != p) par[x] = pp;  // path halving: only ever an ancestor
        x = p;
        p = par[x];
    }
    return x;
}

__device__ __forceinline__ void lu_unite(uint32_t *par, uint32_t a, uint32_t b) {
    volatile uint32_t *vp = par;
    for (;;) {
        a = lu_find(vp, a);
        b = lu_find(vp, b);
        if (a == b) return;
        if (a < b) {
            const uint32_t t = a;
            a = b;
            b = t;
        }
        if (atomicCAS(par + a, a, b) == a) return;
    }
}

__global__ void __launch_bounds__(256) k_band_union(const FrameDesc *frames, RunArrays runs,
                                                    const uint32_t *row_nruns) {
    __shared__ uint32_t s_se[UB_CAP];
    __shared__ uint32_t s_par[UB_CAP];
    __shared__ uint8_t s_v[UB_CAP];
    __shared__ uint8_t s_row[UB_CAP];
    __shared__ uint32_t s_roff[UB_ROWS + 1];
    __shared__ uint32_t s_pair[UB_PAIRS];  // touching pairs: run | run above << 16
    __shared__ uint32_t s_npair;
    static_assert(UB_ROWS <= 32, "one warp scans the band's row counts");
    static_assert(UB_CAP <= 65536, "band-local run ids fit 16 bits");
    const FrameDesc f = frames[blockIdx.y];
    const int tid = threadIdx.x;
    const int nband = (f.qh + UB_ROWS - 1) / UB_ROWS;
    for (int b = blockIdx.x; b < nband; b += gridDim.x) {
        const int y0 = b * UB_ROWS, nr = min(UB_ROWS, f.qh - y0);
        __syncthreads();
        if (tid < 32) {
            const uint32_t c = tid < nr ? row_nruns[f.row0 + y0 + tid] : 0u;
            uint32_t total;
            const uint32_t off = warp_excl_scan(c, &total);
            if (tid < nr) s_roff[tid] = off;
            if (tid == 0) s_roff[nr] = total;
        }
        __syncthreads();
        const uint32_t L = s_roff[nr];
        if (L > UB_CAP) {
            // too many runs to stage: the band's unions in global memory
            for (int r = 1; r < nr; r++) {
                const int64_t cur = f.node_off + (int64_t)(y0 + r) * f.qw, prev = cur - f.qw;
                const int64_t ncur = s_roff[r + 1] - s_roff[r], nprev = s_roff[r] - s_roff[r - 1];
                for (int64_t i = tid; i < ncur; i += blockDim.x) {
                    const int64_t a0 = runs.start[cur + i], a1 = runs.end[cur + i];
                    const uint8_t v = runs.v[cur + i];
                    int64_t lo = 0, hi = nprev;
                    while (lo < hi) {
                        const int64_t mid = (lo + hi) >> 1;
                        if ((int64_t)runs.end[prev + mid] + 1 < a0)
                            lo = mid + 1;
                        else
                            hi = mid;
                    }
                    for (int64_t k = lo; k < nprev && (int64_t)runs.start[prev + k] <= a1 + 1; k++)
                        if (runs.v[prev + k] == v && runs_touch(a0, a1, runs.start[prev + k], runs.end[prev + k], v))
                            uf_unite(runs.parent, (uint32_t)(cur + i), (uint32_t)(prev + k));
                }
            }
            continue;
        }
        // stage the band's runs (local id l = s_roff[row] + index)
        for (uint32_t l = tid; l < L; l += blockDim.x) {
            int r = 0;
            while (s_roff[r + 1] <= l) r++;
            const int64_t node = f.node_off + (int64_t)(y0 + r) * f.qw + (l - s_roff[r]);
            s_se[l] = (uint32_t)runs.start[node] | (uint32_t)runs.end[node] << 16;
            s_v[l] = runs.v[node];
            s_par[l] = l;
            s_row[l] = (uint8_t)r;
        }
        __syncthreads();
        // the unions of rows 1.. of the band with the row above, in shared
        // memory: the touching pairs listed first (a thread per run), then
        // one union per pair, the pairs spread evenly over the threads (a
        // run touching many runs above no longer holds its warp); a band
        // with more pairs than the list holds unites them where found
        if (tid == 0) s_npair = 0;
        __syncthreads();
        for (uint32_t l = s_roff[1] + tid; l < L; l += blockDim.x) {
            const int r = s_row[l];
            const uint32_t pb = s_roff[r - 1], pe = s_roff[r];
            const int a0 = (int)(s_se[l] & 0xffffu), a1 = (int)(s_se[l] >> 16);
            const uint8_t v = s_v[l];
            uint32_t lo = pb, hi = pe;
            while (lo < hi) {  // the first run above whose end reaches a0 - 1
                const uint32_t mid = (lo + hi) >> 1;
                if ((int)(s_se[mid] >> 16) + 1 < a0)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            for (uint32_t k = lo; k < pe && (int)(s_se[k] & 0xffffu) <= a1 + 1; k++)
                if (s_v[k] == v && runs_touch(a0, a1, s_se[k] & 0xffffu, s_se[k] >> 16, v)) {
                    const uint32_t p = atomicAdd(&s_npair, 1u);
                    if (p < UB_PAIRS)
                        s_pair[p] = l | k << 16;
                    else
                        lu_unite(s_par, l, k);
                }
        }
        __syncthreads();
        const uint32_t np = min(s_npair, (uint32_t)UB_PAIRS);
        for (uint32_t p = tid; p < np; p += blockDim.x) lu_unite(s_par, s_pair[p] & 0xffffu, s_pair[p] >> 16);
        __syncthreads();
        // every node points at its local root (read-only walks)
        for (uint32_t l = tid; l < L; l += blockDim.x) {
            uint32_t x = l;
            while (s_par[x] != x) x = s_par[x];
            const int r = s_row[l], rr = s_row[x];
            const int64_t node = f.node_off + (int64_t)(y0 + r) * f.qw + (l - s_roff[r]);
            const int64_t root = f.node_off + (int64_t)(y0 + rr) * f.qw + (x - s_roff[rr]);
            runs.parent[node] = (uint32_t)root;
        }
    }
}

// The joins between bands (each band's first row with the row above) and
// the last-column links of every row (fast/unionfind.c:89-97), in global
// memory: a block per band boundary row, then a thread per row for the
// last column.
#define BJ_CAP 4096  // runs of the two rows staged at once
__global__ void __launch_bounds__(256) k_band_join(const FrameDesc *frames, const uint8_t *thr, RunArrays runs,
                                                   const uint32_t *row_nruns) {
    __shared__ uint32_t s_se[BJ_CAP];
    __shared__ uint8_t s_v[BJ_CAP];
    const FrameDesc f = frames[blockIdx.y];
    const int tid = threadIdx.x;
    const int nband = (f.qh + UB_ROWS - 1) / UB_ROWS;
    for (int b = 1 + blockIdx.x; b < nband; b += gridDim.x) {
        const int64_t y = (int64_t)b * UB_ROWS;
        const int64_t cur = f.node_off + y * f.qw, prev = cur - f.qw;
        const uint32_t ncur = row_nruns[f.row0 + y], nprev = row_nruns[f.row0 + y - 1];
        const uint32_t L = ncur + nprev;  // staged: the row above [0, nprev), this row [nprev, L)
        const bool staged = L <= BJ_CAP;
        __syncthreads();
        if (staged)
            for (uint32_t l = tid; l < L; l += blockDim.x) {
                const int64_t node = l < nprev ? prev + l : cur + (l - nprev);
                s_se[l] = (uint32_t)runs.start[node] | (uint32_t)runs.end[node] << 16;
                s_v[l] = runs.v[node];
            }
        __syncthreads();
        auto se_at = [&](uint32_t l) -> uint32_t {
            if (staged) return s_se[l];
            const int64_t node = l < nprev ? prev + l : cur + (l - nprev);
            return (uint32_t)runs.start[node] | (uint32_t)runs.end[node] << 16;
        };
        auto v_at = [&](uint32_t l) -> uint8_t {
            if (staged) return s_v[l];
            return runs.v[l < nprev ? prev + l : cur + (l - nprev)];
        };
        // each run of either row: the runs of the other row covering its
        // start column and the column before (see k_band_union)
        for (uint32_t l = tid; l < L; l += blockDim.x) {
            const uint32_t se = se_at(l);
            const int a0 = (int)(se & 0xffffu), a1 = (int)(se >> 16);
            const uint8_t v = v_at(l);
            const uint32_t ob = l < nprev ? nprev : 0, oe = l < nprev ? L : nprev;
            uint32_t lo = ob, hi = oe;
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if ((int)(se_at(mid) & 0xffffu) <= a0)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            if (lo == ob) continue;
            const int64_t node = l < nprev ? prev + l : cur + (l - nprev);
            // runs_touch as the reference calls it: this row's run, then the
            // run above (it is not symmetric at column 0)
            const bool upper = l < nprev;
            for (uint32_t k = lo - 1, t = 0; t < 2; t++) {
                const uint32_t sk = se_at(k);
                const int b0 = (int)(sk & 0xffffu), b1 = (int)(sk >> 16);
                if (v_at(k) == v && (upper ? runs_touch(b0, b1, a0, a1, v) : runs_touch(a0, a1, b0, b1, v)))
                    uf_unite(runs.parent, (uint32_t)node, (uint32_t)(k < nprev ? prev + k : cur + (k - nprev)));
                if ((int)(sk & 0xffffu) != a0 || k == ob) break;
                k--;  // the run covering a0 - 1
            }
        }
    }
    for (int64_t y = 1 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; y < f.qh;
         y += (int64_t)gridDim.x * blockDim.x) {
        const int64_t ncur = row_nruns[f.row0 + y];
        if (ncur == 0) continue;
        const int64_t last = f.node_off + y * f.qw + ncur - 1;
        const uint8_t *above = thr + f.q_off + (y - 1) * f.qw;
        if (runs.end[last] == f.qw - 2 && runs.v[last] == 255 && above[f.qw - 1] == 255 && above[f.qw - 2] != 255)
            uf_unite(runs.parent, (uint32_t)last, (uint32_t)(f.node_off + (int64_t)f.qw * f.qh + y - 1));
    }
}

// The root of x without writes (after the unions: a path-halving write that
// read its value before another thread stored a root would undo it).
__device__ __forceinline__ uint32_t uf_root(const uint32_t *par, uint32_t x) {
    const volatile uint32_t *p = par;
    uint32_t px = p[x];
    while (px != x) {
        x = px;
        px = p[x];
    }
    return x;
}

// Each node adds its pixels and offers its id to its root (one atomic per
// distinct root of a warp), and from here on points at its root.
__global__ void __launch_bounds__(256) k_row_sums(const FrameDesc *frames, RunArrays runs, const uint32_t *row_nruns) {
    const FrameDesc f = frames[blockIdx.y];
    const int lane = threadIdx.x & 31;
    for (int64_t y = blockIdx.x; y < f.qh; y += gridDim.x) {
        const int64_t base = f.node_off + y * f.qw;
        const int64_t n = row_nruns[f.row0 + y];
        for (int64_t i0 = 0; i0 <= n; i0 += blockDim.x) {
            const int64_t i = i0 + threadIdx.x;
            const bool valid = i <= n;
            const uint32_t live = __ballot_sync(0xffffffffu, valid);
            if (!valid) continue;
            const int64_t node = i < n ? base + i : f.node_off + (int64_t)f.qw * f.qh + y;
            const uint32_t r = uf_root(runs.parent, (uint32_t)node);
            // no unions run any more: pointing straight at the root is safe
            // for the walks of other threads, and the labels read it once
            if (r != (uint32_t)node) runs.parent[node] = r;
            const uint32_t px = i < n ? (uint32_t)(runs.end[node] - runs.start[node] + 1) : 1u;
            const uint32_t peers = __match_any_sync(live, r);
            const uint32_t sum = __reduce_add_sync(peers, px), mn = __reduce_min_sync(peers, (uint32_t)node);
            if (lane == __ffs(peers) - 1) {
                atomicAdd(runs.px + r, sum);
                atomicMin(runs.minid + r, mn);
            }
        }
    }
}

// Per pixel: its component's label if the component has at least
// min_cluster_pixels pixels, else AT_NOK (no run: 127, or too small). A
// block per row: each run's label once (every node points at its root after
// k_row_sums), spread over the run's pixels by a max-scan of the run starts;
// the last column is the row's extra node.
#define LAB_THREADS 256
__global__ void __launch_bounds__(LAB_THREADS) k_labels(const FrameDesc *frames, const RunArrays runs,
                                                        const uint32_t *row_nruns, uint32_t *lab, int32_t min_px) {
    __shared__ uint32_t s_run[ROW_STAGE];
    __shared__ uint32_t s_rlab[ROW_STAGE];
    __shared__ uint16_t s_end[ROW_STAGE];
    __shared__ uint32_t s_wmax[LAB_THREADS / 32];
    const FrameDesc f = frames[blockIdx.y];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int qw = (int)f.qw, W = qw - 1;
    for (int y = blockIdx.x; y < (int)f.qh; y += gridDim.x) {
        const int64_t base = f.node_off + (int64_t)y * qw;
        const int nr = (int)row_nruns[f.row0 + y];
        uint32_t *out = lab + f.q_off + (int64_t)y * qw;
        if (tid == 0) {
            const uint32_t r = runs.parent[f.node_off + (int64_t)qw * f.qh + y];
            out[W] = (int64_t)runs.px[r] >= min_px ? runs.minid[r] : AT_NOK;
        }
        if (W > ROW_STAGE) {
            // rows too wide to stage: a binary search per pixel
            for (int x = tid; x < W; x += LAB_THREADS) {
                int lo = 0, hi = nr;
                while (lo < hi) {  // the first run with start > x
                    const int mid = (lo + hi) >> 1;
                    if ((int)runs.start[base + mid] <= x)
                        lo = mid + 1;
                    else
                        hi = mid;
                }
                uint32_t l = AT_NOK;
                if (lo > 0 && (int)runs.end[base + lo - 1] >= x) {
                    const uint32_t r = runs.parent[base + lo - 1];
                    if ((int64_t)runs.px[r] >= min_px) l = runs.minid[r];
                }
                out[x] = l;
            }
            continue;
        }
        __syncthreads();
        for (int x = tid; x < W; x += LAB_THREADS) s_run[x] = 0;
        __syncthreads();
        for (int i = tid; i < nr; i += LAB_THREADS) {
            s_run[runs.start[base + i]] = (uint32_t)i + 1;
            s_end[i] = runs.end[base + i];
            const uint32_t r = runs.parent[base + i];
            s_rlab[i] = (int64_t)runs.px[r] >= min_px ? runs.minid[r] : AT_NOK;
        }
        __syncthreads();
        // thread t owns pixels [t * seg, t * seg + seg): the largest run
        // number started at or before each of them
        const int seg = (W + LAB_THREADS - 1) / LAB_THREADS;
        const int x0 = tid * seg, x1 = x0 + seg < W ? x0 + seg : W;
        uint32_t m = 0;
        for (int x = x0; x < x1; x++) m = max(m, s_run[x]);
        uint32_t incl = m;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl = max(incl, t);
        }
        if (lane == 31) s_wmax[wid] = incl;
        uint32_t run = __shfl_up_sync(0xffffffffu, incl, 1);
        if (lane == 0) run = 0;
        __syncthreads();
        for (int w = 0; w < wid; w++) run = max(run, s_wmax[w]);
        for (int x = x0; x < x1; x++) {
            run = max(run, s_run[x]);
            s_run[x] = run && x <= (int)s_end[run - 1] ? s_rlab[run - 1] : AT_NOK;
        }
        __syncthreads();
        for (int x = tid; x < W; x += LAB_THREADS) out[x] = s_run[x];
    }
}

// The same labels with a warp per row (8 rows a block, for batches large
// enough to fill the GPU that way): the run starting at each column staged
// in the warp's slice of shared memory, then 128 columns at a time, 4 a
// lane: a max-scan gives each column its run (carried across chunks), the
// label is read through the run's root (the L1 cache holds the few roots of
// a row; a lane's 4 pixels usually share one run), and a pixel that no
// stored run covers is a 127 of the threshold image. Rows wider than
// LW_CAP columns search the runs per pixel instead.
#define LW_CAP 2048
__global__ void __launch_bounds__(256) k_labels_w(const FrameDesc *frames, const uint8_t *thr, const RunArrays runs,
                                                  const uint32_t *row_nruns, uint32_t *lab, int32_t min_px) {
    __shared__ __align__(16) uint16_t s_run[8][LW_CAP + 8];
    const FrameDesc f = frames[blockIdx.y];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int qw = (int)f.qw, W = qw - 1;
    uint16_t *sr = s_run[w];
    for (int y = (int)blockIdx.x * 8 + w; y < (int)f.qh; y += (int)gridDim.x * 8) {
        const int64_t base = f.node_off + (int64_t)y * qw;
        const int nr = (int)row_nruns[f.row0 + y];
        uint32_t *out = lab + f.q_off + (int64_t)y * qw;
        const uint8_t *row = thr + f.q_off + (int64_t)y * qw;
        auto label_of = [&](int i) -> uint32_t {
            const uint32_t r = runs.parent[base + i];
            return (int64_t)runs.px[r] >= min_px ? runs.minid[r] : AT_NOK;
        };
        if (lane == 0) {
            const uint32_t r = runs.parent[f.node_off + (int64_t)qw * f.qh + y];
            out[W] = (int64_t)runs.px[r] >= min_px ? runs.minid[r] : AT_NOK;
        }
        if (W > LW_CAP) {
            for (int x = lane; x < W; x += 32) {
                int lo = 0, hi = nr;
                while (lo < hi) {  // the first run with start > x
                    const int mid = (lo + hi) >> 1;
                    if ((int)runs.start[base + mid] <= x)
                        lo = mid + 1;
                    else
                        hi = mid;
                }
                out[x] = lo > 0 && (int)runs.end[base + lo - 1] >= x ? label_of(lo - 1) : AT_NOK;
            }
            continue;
        }
        const int Wp = (W + 3) & ~3;
        for (int x = lane; x < Wp; x += 32) sr[x] = 0;
        __syncwarp();
        for (int i = lane; i < nr; i += 32) sr[runs.start[base + i]] = (uint16_t)(i + 1);
        __syncwarp();
        // 16-byte stores when the row and the label array allow
        const bool v4 = ((((uintptr_t)out) | ((uintptr_t)row)) & 15) == 0;
        uint32_t carry = 0;
        for (int x0 = 0; x0 < W; x0 += 128) {
            const int x = x0 + 4 * lane;
            const uint2 pr = x < Wp ? *reinterpret_cast<const uint2 *>(sr + x) : make_uint2(0, 0);
            uint32_t m[4] = {pr.x & 0xffffu, pr.x >> 16, pr.y & 0xffffu, pr.y >> 16};
            m[1] = max(m[1], m[0]);
            m[2] = max(m[2], m[1]);
            m[3] = max(m[3], m[2]);
            uint32_t incl = m[3];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl = max(incl, t);
            }
            uint32_t excl = __shfl_up_sync(0xffffffffu, incl, 1);
            if (lane == 0) excl = 0;
            excl = max(excl, carry);
            carry = max(carry, __shfl_sync(0xffffffffu, incl, 31));
            uint32_t l4[4];
            uint32_t prev_run = 0, prev_lab = AT_NOK;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const uint32_t v = max(m[k], excl);
                uint32_t l = AT_NOK;
                if (x + k < W && v) {
                    if (v != prev_run) {
                        prev_run = v;
                        prev_lab = label_of((int)v - 1);
                    }
                    l = row[x + k] != 127 ? prev_lab : AT_NOK;
                }
                l4[k] = l;
            }
            if (v4 && x + 4 <= W) {
                *reinterpret_cast<uint4 *>(out + x) = make_uint4(l4[0], l4[1], l4[2], l4[3]);
            } else {
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (x + k < W) out[x + k] = l4[k];
            }
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// 6. Boundary points (fast/clusters.c:144-252). Pixel (x, y), y in
// 1..qh-2, against (1,0), (0,1), (-1,1), (1,1): a point where one pixel is
// 0 and the other 255 and both labels are not AT_NOK. The (-1,1) point is
// left out when the pixel to the left gave its (1,1) point, except at x=1;
// x = 0 gives only (1,0) (point_mask). Points are emitted in (y, x,
// neighbour) order.

// Block-per-row forms of the point passes (a block scan per 256 columns),
// for batches too small to fill the GPU with a warp per row.
__global__ void k_point_count_block(const FrameDesc *frames, const uint8_t *thr, const uint32_t *lab, uint64_t *row_npts) {
    __shared__ uint32_t sh[32];
    const FrameDesc f = frames[blockIdx.y];
    for (int64_t y = blockIdx.x; y < f.qh; y += gridDim.x) {
        uint32_t cnt = 0;
        if (y >= 1 && y + 1 < f.qh) {
            const uint8_t *a = thr + f.q_off + y * f.qw, *b = a + f.qw;
            const uint32_t *la = lab + f.q_off + y * f.qw, *lb = la + f.qw;
            for (int64_t x = threadIdx.x; x < f.qw; x += blockDim.x) cnt += __popc(point_mask(a, b, la, lb, x, f.qw));
        }
        uint32_t total;
        block_excl_scan(cnt, &total, sh);
        if (threadIdx.x == 0) row_npts[f.row0 + y] = total;
    }
}

__global__ void k_point_emit_block(const FrameDesc *frames, const uint8_t *thr, const uint32_t *lab,
                             const uint64_t *row_pt_off, uint64_t *pt_key, uint64_t *pt_val, int nb) {
    __shared__ uint32_t sh[32];
    const FrameDesc f = frames[blockIdx.y];
    for (int64_t y = 1 + blockIdx.x; y + 1 < f.qh; y += gridDim.x) {
        const uint8_t *a = thr + f.q_off + y * f.qw, *b = a + f.qw;
        const uint32_t *la = lab + f.q_off + y * f.qw, *lb = la + f.qw;
        uint64_t out = row_pt_off[f.row0 + y];
        for (int64_t x0 = 0; x0 < f.qw; x0 += blockDim.x) {
            int64_t x = x0 + threadIdx.x;
            uint32_t m = x < f.qw ? point_mask(a, b, la, lb, x, f.qw) : 0u;
            uint32_t total;
            uint32_t off = block_excl_scan(__popc(m), &total, sh);
            uint64_t o = out + off;
            int g = a[x < f.qw ? x : 0] == 0 ? 255 : -255;
            for (int j = 0; j < 4; j++) {
                if (!(m >> j & 1u)) continue;
                int dx = j == 0 || j == 3 ? 1 : j == 2 ? -1 : 0;
                int dy = j == 0 ? 0 : 1;
                uint32_t l0 = la[x], l1 = dy ? lb[x + dx] : la[x + dx];
                uint64_t hi = l0 > l1 ? l0 : l1, lo = l0 > l1 ? l1 : l0;
                uint64_t px = (uint64_t)(2 * x + dx), py = (uint64_t)(2 * y + dy);
                uint64_t gx = (uint16_t)(int16_t)(dx * g), gy = (uint16_t)(int16_t)(dy * g);
                pt_key[o] = hi << nb | lo;
                pt_val[o] = px | py << 16 | gx << 32 | gy << 48;
                o++;
            }
            out += total;
        }
    }
}

// A warp per row for both passes: the row's points counted, then emitted
// in (x, neighbour) order at the row's offset (warp scans, no block
// barriers).

__global__ void __launch_bounds__(256) k_point_count(const FrameDesc *frames, const uint8_t *thr,
                                                     const uint32_t *lab, uint64_t *row_npts) {
    const FrameDesc f = frames[blockIdx.y];
    const int lane = threadIdx.x & 31;
    const int64_t wpb = blockDim.x >> 5;
    for (int64_t y = blockIdx.x * wpb + (threadIdx.x >> 5); y < f.qh; y += gridDim.x * wpb) {
        uint32_t cnt = 0;
        if (y >= 1 && y + 1 < f.qh) {
            const uint8_t *a = thr + f.q_off + y * f.qw, *b = a + f.qw;
            const uint32_t *la = lab + f.q_off + y * f.qw, *lb = la + f.qw;
            for (int64_t x = lane; x < f.qw; x += 32) cnt += __popc(point_mask(a, b, la, lb, x, f.qw));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        if (lane == 0) row_npts[f.row0 + y] = cnt;
    }
}

// The cluster key of a point: (larger label, smaller label) packed as
// larger << nb | smaller, nb = bits of the largest node id.
__global__ void __launch_bounds__(256) k_point_emit(const FrameDesc *frames, const uint8_t *thr,
                                                    const uint32_t *lab, const uint64_t *row_pt_off,
                                                    uint64_t *pt_key, uint64_t *pt_val, int nb) {
    const FrameDesc f = frames[blockIdx.y];
    const int lane = threadIdx.x & 31;
    const int64_t wpb = blockDim.x >> 5;
    for (int64_t y = 1 + blockIdx.x * wpb + (threadIdx.x >> 5); y + 1 < f.qh; y += gridDim.x * wpb) {
        const uint8_t *a = thr + f.q_off + y * f.qw, *b = a + f.qw;
        const uint32_t *la = lab + f.q_off + y * f.qw, *lb = la + f.qw;
        uint64_t out = row_pt_off[f.row0 + y];
        for (int64_t x0 = 0; x0 < f.qw; x0 += 32) {
            const int64_t x = x0 + lane;
            const uint32_t m = x < f.qw ? point_mask(a, b, la, lb, x, f.qw) : 0u;
            uint32_t total;
            const uint32_t off = warp_excl_scan(__popc(m), &total);
            uint64_t o = out + off;
            const int g = a[x < f.qw ? x : 0] == 0 ? 255 : -255;
            for (int j = 0; j < 4; j++) {
                if (!(m >> j & 1u)) continue;
                const int dx = j == 0 || j == 3 ? 1 : j == 2 ? -1 : 0;
                const int dy = j == 0 ? 0 : 1;
                const uint32_t l0 = la[x], l1 = dy ? lb[x + dx] : la[x + dx];
                const uint64_t hi = l0 > l1 ? l0 : l1, lo = l0 > l1 ? l1 : l0;
                const uint64_t px = (uint64_t)(2 * x + dx), py = (uint64_t)(2 * y + dy);
                const uint64_t gx = (uint16_t)(int16_t)(dx * g), gy = (uint16_t)(int16_t)(dy * g);
                pt_key[o] = hi << nb | lo;
                pt_val[o] = px | py << 16 | gx << 32 | gy << 48;
                o++;
            }
            out += total;
        }
    }
}

// ---------------------------------------------------------------------------
// 7. Clusters (fast/clusters.c:16-66, 318-382). The pair table and the
// placing of the points are in at_cluster.cu; here the distinct pairs of
// the table, and the fallback when the table overflows.

// The occupied slots, in no particular order: (pair, slot).
__global__ void k_cluster_collect(const uint64_t *tkeys, uint32_t size, uint64_t *okeys, uint32_t *oslots,
                                  uint32_t *count) {
    const int lane = threadIdx.x & 31;
    for (uint32_t s0 = blockIdx.x * blockDim.x; s0 < size; s0 += gridDim.x * blockDim.x) {
        const uint32_t s = s0 + threadIdx.x;
        const uint64_t k = s < size ? tkeys[s] : CH_EMPTY;
        const bool occ = k != CH_EMPTY;
        const uint32_t bal = __ballot_sync(0xffffffffu, occ);
        if (!bal) continue;
        uint32_t at = 0;
        if (lane == __ffs(bal) - 1) at = atomicAdd(count, (uint32_t)__popc(bal));
        at = __shfl_sync(0xffffffffu, at, __ffs(bal) - 1) + __popc(bal & ((1u << lane) - 1u));
        if (occ) {
            okeys[at] = k;
            oslots[at] = s;
        }
    }
}

// ---------------------------------------------------------------------------
// 7b. Clusters by the full sort (the fallback): after the stable sort by
// key, each run of equal keys is a cluster (points in emission order).

__global__ void k_cluster_heads(const uint64_t *key, int64_t n, uint32_t *head) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        head[i] = i == 0 || key[i] != key[i - 1];
}

__global__ void k_cluster_starts(const uint64_t *key, const uint32_t *head, const uint32_t *head_scan, int64_t n,
                                 int nb, const FrameDesc *frames, int nframes, uint32_t *cstart, int32_t *cframe,
                                 uint64_t *ckey) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (!head[i]) continue;
        uint32_t c = head_scan[i];
        cstart[c] = (uint32_t)i;
        ckey[c] = key[i];
        int64_t node = (int64_t)(key[i] >> nb);
        int lo = 0, hi = nframes - 1;  // the frame whose node range holds node
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (frames[mid].node_off <= node)
                lo = mid;
            else
                hi = mid - 1;
        }
        cframe[c] = lo;
    }
}

// ---------------------------------------------------------------------------
// 8. Quad fitting, one block per cluster (fast/quads.c:429-1160).

__device__ __forceinline__ uint32_t f32_bits(float f) { return __float_as_uint(f); }

// The angle key (fast/quads.c:429-453): quadrant + slope in f32, as
// order-preserving bits, above the complemented point index.
__device__ __forceinline__ uint64_t angle_key(float dx, float dy, uint32_t idx) {
    float quadrant = dy > 0.0f ? (dx > 0.0f ? 65536.0f : 131072.0f) : (dx > 0.0f ? 0.0f : -65536.0f);
    float fx = dx, fy = dy;
    if (dy < 0.0f) {
        fx = __uint_as_float(f32_bits(dx) ^ 0x80000000u);
        fy = __uint_as_float(f32_bits(dy) ^ 0x80000000u);
    }
    float ndx = fx, ndy = fy;
    if (fx < 0.0f) {
        ndx = fy;
        ndy = -fx;
    }
    float slope = __fadd_rn(quadrant, __fdiv_rn(ndy, ndx));
    uint32_t b = f32_bits(slope);
    uint32_t s = (uint32_t)((int32_t)b >> 31);
    return (uint64_t)(b ^ (s | 0x80000000u)) << 32 | (uint32_t)~idx;
}

// The leaf of the reference's angle sort holding position p of n
// (fast/quads.c:181-237): cut in four while half the range has more than
// 5 keys, then in two down to 5 or fewer. Returns start << 8 | length.
__device__ __forceinline__ uint32_t leaf_of(int64_t n, int64_t p) {
    int64_t lo = 0, sz = n;
    while (sz / 2 > 5) {
        int64_t half = sz / 2, q1 = half / 2, q3 = half + (sz - half) / 2;
        int64_t r = p - lo;
        if (r < q1) {
            sz = q1;
        } else if (r < half) {
            lo += q1;
            sz = half - q1;
        } else if (r < q3) {
            lo += half;
            sz = q3 - half;
        } else {
            lo += q3;
            sz = sz - q3;
        }
    }
    while (sz > 5) {
        int64_t half = sz / 2;
        if (p - lo >= half) {
            lo += half;
            sz -= half;
        } else {
            sz = half;
        }
    }
    return (uint32_t)(lo << 8 | sz);
}

// The leaf of position p of n (see leaf_of), in 32-bit arithmetic.
__device__ __forceinline__ void leaf_of32(int n, int p, int &lo, int &len) {
    int l = 0, sz = n;
    while (sz / 2 > 5) {
        const int half = sz / 2, q1 = half / 2, q3 = half + (sz - half) / 2;
        const int r = p - l;
        if (r < q1) {
            sz = q1;
        } else if (r < half) {
            l += q1;
            sz = half - q1;
        } else if (r < q3) {
            l += half;
            sz = q3 - half;
        } else {
            l += q3;
            sz = sz - q3;
        }
    }
    while (sz > 5) {
        const int half = sz / 2;
        if (p - l >= half) {
            l += half;
            sz -= half;
        } else {
            sz = half;
        }
    }
    lo = l;
    len = sz;
}

// The leaf networks of the reference (fast/quads.c:56-85): compare-exchange
// on the upper 32 bits only.
__device__ __forceinline__ void leaf_network(uint64_t *k, int n) {
#define CX(a, b)                                      \
    if ((k[a] >> 32) > (k[b] >> 32)) {                \
        uint64_t t_ = k[a];                           \
        k[a] = k[b];                                  \
        k[b] = t_;                                    \
    }
    if (n == 2) {
        CX(0, 1)
    } else if (n == 3) {
        CX(0, 1) CX(1, 2) CX(0, 1)
    } else if (n == 4) {
        CX(0, 1) CX(2, 3) CX(0, 2) CX(1, 3) CX(1, 2)
    } else if (n == 5) {
        CX(0, 1) CX(3, 4) CX(1, 2) CX(0, 1) CX(0, 3) CX(2, 4) CX(1, 2) CX(2, 3) CX(1, 2)
    }
#undef CX
}


// Sort (key, val) pairs ascending by key (keys distinct): a merge sort of
// log2(n) levels; at each level every thread writes a contiguous chunk of
// the output, starting at the merge-path split of its first element (a
// binary search). kb/vb are scratch of n entries; the result is in ka/va.
__device__ void block_merge_sort(uint64_t *ka, uint32_t *va, uint64_t *kb, uint32_t *vb, int n) {
    uint64_t *sk = ka, *dk = kb;
    uint32_t *sv = va, *dv = vb;
    const int ipt = (n + (int)blockDim.x - 1) / (int)blockDim.x;
    for (int w = 1; w < n; w <<= 1) {
        const int o0 = (int)threadIdx.x * ipt, o1 = min(n, o0 + ipt);
        int o = o0;
        while (o < o1) {
            const int lo = (o / (2 * w)) * (2 * w);
            const int la = min(w, n - lo), lb = max(0, min(w, n - lo - la));
            const uint64_t *A = sk + lo, *B = sk + lo + la;
            const int k = o - lo, seg_end = min(o1, lo + la + lb);
            int l = max(0, k - lb), h = min(k, la);
            while (l < h) {
                const int m = (l + h) >> 1;
                if (A[m] < B[k - m - 1])
                    l = m + 1;
                else
                    h = m;
            }
            int i = l, j = k - l;
            for (; o < seg_end; o++) {
                const bool take_a = j >= lb || (i < la && A[i] < B[j]);
                if (take_a) {
                    dk[o] = A[i];
                    dv[o] = sv[lo + i];
                    i++;
                } else {
                    dk[o] = B[j];
                    dv[o] = sv[lo + la + j];
                    j++;
                }
            }
        }
        __syncthreads();
        uint64_t *tk = sk;
        sk = dk;
        dk = tk;
        uint32_t *tv = sv;
        sv = dv;
        dv = tv;
    }
    if (sk != ka) {
        for (int t = threadIdx.x; t < n; t += blockDim.x) {
            ka[t] = sk[t];
            va[t] = sv[t];
        }
        __syncthreads();
    }
}

struct MSum {
    double x, y, xx, xy, yy, w;
};

struct Moments {
    const double *mx, *my, *mxx, *mxy, *myy, *mw;
};

// Moments of sorted points i0..i1, wrapping past the end, summed in the
// reference's forms (fast/quads.c:539-569, 658-700, 885-921).
__device__ __forceinline__ MSum seg_moments(const Moments &a, int64_t sz, int64_t i0, int64_t i1) {
    MSum s;
    if (i0 <= i1) {
        s.x = a.mx[i1];
        s.y = a.my[i1];
        s.xx = a.mxx[i1];
        s.xy = a.mxy[i1];
        s.yy = a.myy[i1];
        s.w = a.mw[i1];
        if (i0 > 0) {
            s.x = s.x - a.mx[i0 - 1];
            s.y = s.y - a.my[i0 - 1];
            s.xx = s.xx - a.mxx[i0 - 1];
            s.xy = s.xy - a.mxy[i0 - 1];
            s.yy = s.yy - a.myy[i0 - 1];
            s.w = s.w - a.mw[i0 - 1];
        }
    } else {
        s.x = (a.mx[sz - 1] - a.mx[i0 - 1]) + a.mx[i1];
        s.y = (a.my[sz - 1] - a.my[i0 - 1]) + a.my[i1];
        s.xx = (a.mxx[sz - 1] - a.mxx[i0 - 1]) + a.mxx[i1];
        s.xy = (a.mxy[sz - 1] - a.mxy[i0 - 1]) + a.mxy[i1];
        s.yy = (a.myy[sz - 1] - a.myy[i0 - 1]) + a.myy[i1];
        s.w = (a.mw[sz - 1] - a.mw[i0 - 1]) + a.mw[i1];
    }
    return s;
}

// The moments of the window of 2 ksz + 1 points centred on i, wrapping
// around the ends (fast/quads.c:797-808).
__device__ __forceinline__ MSum window_moments(const Moments &a, int64_t sz, int64_t ksz, int64_t i) {
    const int64_t i0 = i - ksz, i1 = i + ksz;
    if (i0 < 0) return seg_moments(a, sz, i0 + sz, i1);
    if (i1 < sz) return seg_moments(a, sz, i0, i1);
    return seg_moments(a, sz, i0, i1 - sz);
}

// The smoothed error at i (fast/quads.c:809-826): the 7-tap filter over
// errs, wrapping around the ends; the sum in tap order.
template <typename I>
__device__ __forceinline__ double smooth_at(const double *e, I n, I i, const double *q) {
    double acc;
    if (i >= 3 && i < n - 3) {
        acc = e[i - 3] * q[0];
        for (int t = 1; t < 7; t++) acc = acc + e[i - 3 + t] * q[t];
    } else {
        acc = 0.0;
        for (int t = 0; t < 7; t++) {
            I j = i - 3 + t;
            if (j < 0) j += n;
            if (j >= n) j -= n;
            acc = acc + e[j] * q[t];
        }
    }
    return acc;
}

// The error of a window of nn points (fast/quads.c:604-653).
__device__ __forceinline__ double window_error(MSum s, double nn) {
    double ex = s.x / s.w, ey = s.y / s.w;
    double cxx = s.xx / s.w - ex * ex;
    double cxy = s.xy / s.w - ex * ey;
    double cyy = s.yy / s.w - ey * ey;
    double d = cxx - cyy;
    double root = (double)__fsqrt_rn((float)(d * d + 4.0 * (cxy * cxy)));
    return nn * (0.5 * (cxx + cyy - root));
}

// The line of the moments: centroid, unit normal, smaller eigenvalue
// (fast/quads.c:570-600, 756-783).
__device__ __forceinline__ void line_of(MSum s, double lp[4], double *mse) {
    double ex = s.x / s.w, ey = s.y / s.w;
    double cxx = s.xx / s.w - ex * ex;
    double cxy = s.xy / s.w - ex * ey;
    double cyy = s.yy / s.w - ey * ey;
    double root = (double)__fsqrt_rn((float)((cxx - cyy) * (cxx - cyy) + 4.0 * cxy * cxy));
    double eig_small = 0.5 * (cxx + cyy - root);
    double eig = 0.5 * (cxx + cyy + root);
    double nx1 = cxx - eig, ny1 = cxy, m1 = nx1 * nx1 + ny1 * ny1;
    double nx2 = cxy, ny2 = cyy - eig, m2 = nx2 * nx2 + ny2 * ny2;
    double nx = nx2, ny = ny2, m = m2;
    if (m1 > m2) {
        nx = nx1;
        ny = ny1;
        m = m1;
    }
    double len = (double)__fsqrt_rn((float)m);
    lp[0] = ex;
    lp[1] = ey;
    lp[2] = 0.0;
    lp[3] = 0.0;
    if (!(fabs(len) < 1e-12)) {
        lp[2] = nx / len;
        lp[3] = ny / len;
    }
    *mse = eig_small;
}


// A double as a 64-bit integer in the same order (negative values
// reversed below the positive ones); no NaN reaches it.
__device__ __forceinline__ uint64_t dorder_key(double d) {
    const uint64_t b = (uint64_t)__double_as_longlong(d);
    return (b >> 63) ? ~b : b | 0x8000000000000000ull;
}
__device__ __forceinline__ double dorder_val(uint64_t k) {
    return __longlong_as_double((long long)((k >> 63) ? k & 0x7fffffffffffffffull : ~k));
}

// The (r+1)-th largest of e[0, n) (r < n), by the whole block: a radix
// select over dorder_key, 8 bits a pass from the top. hist holds 256
// counters; *selp and *selr are the prefix found and the rank left.
// Warp 0 finds each pass's digit: lane l counts digits 255-8l .. 248-8l.
__device__ double block_select_desc(const double *e, int64_t n, uint32_t r, uint32_t *hist, uint64_t *selp,
                                    uint32_t *selr) {
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31;
    if (tid == 0) {
        *selp = 0;
        *selr = r;
    }
    for (int shift = 56; shift >= 0; shift -= 8) {
        for (int b = tid; b < 256; b += nt) hist[b] = 0;
        __syncthreads();
        const uint64_t prefix = *selp, mask = shift == 56 ? 0ull : ~0ull << (shift + 8);
        for (int64_t i = tid; i < n; i += nt) {
            const uint64_t key = dorder_key(e[i]);
            if ((key & mask) == prefix) atomicAdd(hist + ((key >> shift) & 255u), 1u);
        }
        __syncthreads();
        if (tid < 32) {
            const uint32_t rr = *selr;
            uint32_t c[8], sum = 0;
#pragma unroll
            for (int j = 0; j < 8; j++) {
                c[j] = hist[255 - 8 * lane - j];
                sum += c[j];
            }
            uint32_t inc = sum;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += t;
            }
            const uint32_t excl = inc - sum;
            if (excl <= rr && rr < inc) {
                uint32_t acc = excl;
                int bin = 255 - 8 * lane;
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    if (rr >= acc + c[j]) {
                        acc += c[j];
                        continue;
                    }
                    bin = 255 - 8 * lane - j;
                    break;
                }
                *selr = rr - acc;
                *selp = prefix | (uint64_t)bin << shift;
            }
        }
        __syncthreads();
    }
    return dorder_val(*selp);
}

// Two size classes of clusters, one kernel template: 128 threads for
// clusters of at most FIT_SMALL points (everything staged in shared
// memory), FIT_LARGE_NT threads for the larger ones (dynamic shared memory; sorts
// beyond FIT_LARGE_SORT points fall back to global scratch).
#define FIT_SMALL 1024
#define FIT_LARGE_SORT 6144
#define FIT_CHUNK_SMALL 256
#define FIT_CHUNK_LARGE 512
#define FIT_LARGE_NT 256  // threads of the largest class's blocks (two blocks an SM)

// dynamic shared memory of one block of the fit kernel
// Shared memory of the block fit kernel for clusters of up to sort_cap
// points: region X (the angle keys; then the radix sort's second buffers;
// then the staged moment terms of a chunk of points), the sort keys (4 B)
// and point indices (2 B), and the radix histograms (256 per warp). The
// moment terms take two chunks of six rows of chunk + 2 doubles (the pad
// puts the six rows that one warp walks in step on distinct banks).
__host__ __device__ constexpr size_t fit_x_bytes(int sort_cap, int chunk) {
    return (size_t)sort_cap * 8 > (size_t)(chunk + 2) * 96 ? (size_t)sort_cap * 8 : (size_t)(chunk + 2) * 96;
}
__host__ __device__ constexpr size_t fit_smem_bytes(int sort_cap, int chunk, int nwarps) {
    return fit_x_bytes(sort_cap, chunk) + (size_t)sort_cap * 6 + (size_t)256 * nwarps * 4;
}

// Stable sort of n (32-bit key, 16-bit value) pairs by key: four passes of
// 8 bits. Each pass counts digits per warp over the warp's contiguous range,
// scans the counts in (digit, warp) order, and scatters each warp's range in
// order, 32 at a time, ranking equal digits by lane (match_any). ka/va hold
// the input and get the result; kb/vb are the second buffers; hist holds
// 256 counters per warp.
__device__ void block_radix_sort32(uint32_t *ka, uint16_t *va, uint32_t *kb, uint16_t *vb, int n, uint32_t *hist) {
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, nw = blockDim.x >> 5;
    const int per = ((n + nw - 1) / nw + 31) & ~31;
    const int w0 = w * per < n ? w * per : n, w1 = w0 + per < n ? w0 + per : n;
    const int nh = 256 * nw;
    __shared__ uint32_t s_part[32];
    for (int shift = 0; shift < 32; shift += 8) {
        for (int i = tid; i < nh; i += blockDim.x) hist[i] = 0;
        __syncthreads();
        for (int i = w0 + lane; i < w1; i += 32) atomicAdd(hist + (int)(ka[i] >> shift & 255u) * nw + w, 1u);
        __syncthreads();
        // exclusive scan of hist: thread t owns entries [t * e, t * e + e)
        const int e = (nh + blockDim.x - 1) / blockDim.x;
        const int h0 = tid * e < nh ? tid * e : nh, h1 = h0 + e < nh ? h0 + e : nh;
        uint32_t sum = 0;
        for (int i = h0; i < h1; i++) sum += hist[i];
        uint32_t incl = sum;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) s_part[w] = incl;
        __syncthreads();
        if (w == 0) {
            uint32_t v = lane < nw ? s_part[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
                if (lane >= o) v += t;
            }
            if (lane < nw) s_part[lane] = v;
        }
        __syncthreads();
        uint32_t run = (w > 0 ? s_part[w - 1] : 0) + incl - sum;
        for (int i = h0; i < h1; i++) {
            const uint32_t c = hist[i];
            hist[i] = run;
            run += c;
        }
        __syncthreads();
        for (int i0 = w0; i0 < w1; i0 += 32) {
            const int i = i0 + lane;
            const bool valid = i < w1;
            const uint32_t k = valid ? ka[i] : 0;
            const int d = valid ? (int)(k >> shift & 255u) : 256 + lane;
            const uint32_t peers = __match_any_sync(0xffffffffu, d);
            const uint32_t base = valid ? hist[d * nw + w] : 0;
            if (valid) {
                const uint32_t at = base + __popc(peers & ((1u << lane) - 1u));
                kb[at] = k;
                vb[at] = va[i];
            }
            __syncwarp();
            if (valid && lane == __ffs(peers) - 1) hist[d * nw + w] = base + __popc(peers);
            __syncwarp();
        }
        __syncthreads();
        uint32_t *tk = ka;
        ka = kb;
        kb = tk;
        uint16_t *tv = va;
        va = vb;
        vb = tv;
    }
}


// Optional phase timers of the fit kernel (a -DAT_FIT_PROF build only).
#ifdef AT_FIT_PROF
#define FIT_PROF_N 32768
__device__ long long g_fitprof[FIT_PROF_N][12];
#define FIT_PROF(k)                                              \
    if (tid == 0 && c < FIT_PROF_N) g_fitprof[c][k] = clock64();
#define FITW_PROF(k)                                             \
    if (lane == 0 && c < FIT_PROF_N) g_fitprof[c][k] = clock64();
#define FITW_SIZE(n)                                             \
    if (lane == 0 && c < FIT_PROF_N) g_fitprof[c][0] = (n);
#define FITB_SIZE(n)                                             \
    if (tid == 0 && c < FIT_PROF_N) g_fitprof[c][0] = (n);
__device__ long long g_decprof[8192][8];
#define DEC_PROF(k)                                              \
    if (tid == 0 && qi < 8192) g_decprof[qi][k] = clock64();
extern "C" int at_dec_prof_copy(void *dst, int n) {
    return (int)cudaMemcpyFromSymbol(dst, g_decprof, (size_t)n * 8 * 8);
}
extern "C" int at_fit_prof_copy(void *dst, int n) {
    return (int)cudaMemcpyFromSymbol(dst, g_fitprof, (size_t)n * 12 * 8);
}
#else
#define FIT_PROF(k)
#define FITW_PROF(k)
#define FITW_SIZE(n)
#define FITB_SIZE(n)
#define DEC_PROF(k)
#endif

template <int NT>
__global__ void __launch_bounds__(NT, (NT <= 128 ? 4 : NT <= 256 ? 2 : 1)) k_fit_quads(const FrameDesc *frames, GpuParams prm, const uint8_t *qim,
                                                   const uint64_t *pts, const uint32_t *cstart,
                                                   const int32_t *cframe, int64_t nclusters, int64_t npoints,
                                                   FitScratch scr, GpuQuad *quads, uint32_t *quad_ok, uint32_t *err,
                                                   const uint32_t *list, const uint32_t *count, uint32_t *next,
                                                   int sort_cap, int chunk) {
    extern __shared__ __align__(16) unsigned char fit_smem[];
    const size_t xb = fit_x_bytes(sort_cap, chunk);
    uint64_t *s_key = reinterpret_cast<uint64_t *>(fit_smem);  // X: angle keys
    uint32_t *s_kb = reinterpret_cast<uint32_t *>(fit_smem);   // X: the sort's second buffers
    uint16_t *s_vb = reinterpret_cast<uint16_t *>(fit_smem + (size_t)sort_cap * 4);
    double *s_w = reinterpret_cast<double *>(fit_smem);        // X: six terms per staged point
    uint32_t *s_ka = reinterpret_cast<uint32_t *>(fit_smem + xb);
    uint16_t *s_val = reinterpret_cast<uint16_t *>(fit_smem + xb + (size_t)sort_cap * 4);
    uint32_t *s_hist = reinterpret_cast<uint32_t *>(fit_smem + xb + (size_t)sort_cap * 6);
    __shared__ float s_lane[8];
    __shared__ int s_rev, s_ok;
    __shared__ uint32_t s_bb[4][NT / 32];
    __shared__ uint32_t s_scan[32];
    __shared__ double s_perr[AT_MAX_NMAXIMA * AT_MAX_NMAXIMA], s_pmse[AT_MAX_NMAXIMA * AT_MAX_NMAXIMA],
        s_pnx[AT_MAX_NMAXIMA * AT_MAX_NMAXIMA], s_pny[AT_MAX_NMAXIMA * AT_MAX_NMAXIMA];
    __shared__ double s_be[NT / 32], s_lines[4][4], s_lmse[4], s_best;
    __shared__ int64_t s_bo[NT / 32];
    __shared__ uint32_t s_next;
    __shared__ uint64_t s_selp;
    __shared__ uint32_t s_selr;
    const int tid = threadIdx.x;
    const uint32_t ncl = *count;

    // the class's clusters, largest first, each to the next free block
    for (;;) {
        __syncthreads();
        if (tid == 0) s_next = atomicAdd(next, 1u);
        __syncthreads();
        if (s_next >= ncl) break;
        const int64_t c = list[s_next];
        const int64_t s0 = cstart[c];
        const int64_t sz = (c + 1 < nclusters ? (int64_t)cstart[c + 1] : npoints) - s0;
        const FrameDesc f = frames[cframe[c]];
        if (sz > 65535) {
            if (tid == 0) atomicOr(err, AT_ERR_CLUSTER_TOO_BIG);
            continue;
        }
        FIT_PROF(1)
        FITB_SIZE(sz)
        const uint64_t *P = pts + s0;
        // bounding box (fast/quads.c:515-528)
        uint32_t xmin = 0xffff, xmax = 0, ymin = 0xffff, ymax = 0;
        for (int64_t i = tid; i < sz; i += NT) {
            uint32_t x = (uint32_t)(P[i] & 0xffff), y = (uint32_t)(P[i] >> 16 & 0xffff);
            xmin = min(xmin, x);
            xmax = max(xmax, x);
            ymin = min(ymin, y);
            ymax = max(ymax, y);
        }
        for (int o = 16; o > 0; o >>= 1) {
            xmin = min(xmin, __shfl_xor_sync(0xffffffffu, xmin, o));
            xmax = max(xmax, __shfl_xor_sync(0xffffffffu, xmax, o));
            ymin = min(ymin, __shfl_xor_sync(0xffffffffu, ymin, o));
            ymax = max(ymax, __shfl_xor_sync(0xffffffffu, ymax, o));
        }
        __syncthreads();
        if ((tid & 31) == 0) {
            s_bb[0][tid >> 5] = xmin;
            s_bb[1][tid >> 5] = xmax;
            s_bb[2][tid >> 5] = ymin;
            s_bb[3][tid >> 5] = ymax;
        }
        __syncthreads();
        for (int w = 0; w < NT / 32; w++) {
            xmin = min(xmin, s_bb[0][w]);
            xmax = max(xmax, s_bb[1][w]);
            ymin = min(ymin, s_bb[2][w]);
            ymax = max(ymax, s_bb[3][w]);
        }
        if ((int64_t)(xmax - xmin) * (int64_t)(ymax - ymin) < f.tag_width) continue;
        const float cx = (float)((double)(xmin + xmax) * 0.5 + 0.05118);
        const float cy = (float)((double)(ymin + ymax) * 0.5 + -0.028581);

        FIT_PROF(2)
        // angle keys, and the dot product of offsets and gradients: 8 lanes
        // over the whole groups of 8, then the rest (fast/quads.c:467-512)
        // clusters that fit keep their keys in shared memory, where the
        // leaf step turns them into sort keys in place
        const bool in_smem = sz <= sort_cap;
        uint64_t *keys = in_smem ? s_key : scr.keys + s0;
        for (int64_t i = tid; i < sz; i += NT) {
            float dx = __fsub_rn((float)(P[i] & 0xffff), cx), dy = __fsub_rn((float)(P[i] >> 16 & 0xffff), cy);
            keys[i] = angle_key(dx, dy, (uint32_t)i);
        }
        const int64_t nv = sz - sz % 8;
        {
            // the terms dx*gx + dy*gy by all threads into shared memory (the
            // moment staging area, free here), then lane l < 8 sums terms
            // l, l+8, ... in order
            float *s_term = reinterpret_cast<float *>(s_ka);
            const int64_t tcap = sort_cap;  // a multiple of 8
            float acc = 0.0f;
            for (int64_t c0 = 0; c0 < nv; c0 += tcap) {
                const int64_t cn = dmin(tcap, nv - c0);
                for (int64_t i = tid; i < cn; i += NT) {
                    uint64_t pt = P[c0 + i];
                    float dx = __fsub_rn((float)(pt & 0xffff), cx), dy = __fsub_rn((float)(pt >> 16 & 0xffff), cy);
                    float gx = (float)(int16_t)(pt >> 32 & 0xffff), gy = (float)(int16_t)(pt >> 48);
                    s_term[i] = __fadd_rn(__fmul_rn(dx, gx), __fmul_rn(dy, gy));
                }
                __syncthreads();
                if (tid < 8) {
                    int64_t i = tid;
                    for (; i + 56 < cn; i += 64) {
                        float v[8];
#pragma unroll
                        for (int u = 0; u < 8; u++) v[u] = s_term[i + 8 * u];
#pragma unroll
                        for (int u = 0; u < 8; u++) acc = __fadd_rn(acc, v[u]);
                    }
                    for (; i < cn; i += 8) acc = __fadd_rn(acc, s_term[i]);
                }
                __syncthreads();
            }
            if (tid < 8) s_lane[tid] = acc;
        }
        __syncthreads();
        if (tid == 0) {
            float dot = __fadd_rn(__fadd_rn(__fadd_rn(s_lane[0], s_lane[4]), __fadd_rn(s_lane[2], s_lane[6])),
                                  __fadd_rn(__fadd_rn(s_lane[1], s_lane[5]), __fadd_rn(s_lane[3], s_lane[7])));
            for (int64_t i = nv; i < sz; i++) {
                float dx = __fsub_rn((float)(P[i] & 0xffff), cx), dy = __fsub_rn((float)(P[i] >> 16 & 0xffff), cy);
                float gx = (float)(int16_t)(P[i] >> 32 & 0xffff), gy = (float)(int16_t)(P[i] >> 48);
                dot = __fadd_rn(dot, __fadd_rn(__fmul_rn(dx, gx), __fmul_rn(dy, gy)));
            }
            int rev = dot < 0.0f;
            int ok = 1;
            if (!f.reversed_border && rev) ok = 0;
            if (!f.normal_border && !rev) ok = 0;
            s_ok = ok;
            s_rev = rev;
        }
        __syncthreads();
        if (!s_ok) continue;
        const int rev = s_rev;

        // The angle sort. The reference's merge sort keeps each leaf's
        // "blocks" (a key larger than all before it in the leaf's network
        // order, and the smaller keys after it) together and orders them by
        // their first key. So: per leaf, the network order, each key's
        // block head and its place in the leaf; then one sort by (head,
        // place), packed into 64 bits as head's slope bits, 0xffff - head's
        // index, and the place.
        FIT_PROF(3)
        uint64_t *sk = scr.skey + s0;
        uint32_t *sv = scr.sval + s0;
        if (in_smem) {
            // Lay the points out in (head index descending, place) order:
            // leaves in reverse order, and in each leaf its blocks by head
            // index descending, each block in network order. A stable sort
            // by the head's slope bits then gives the (head, place) order.
            // Each warp finds the leaves that start in its 32 points at a
            // time, queues them in its slice of the (still unused) radix
            // histograms, and arranges them 32 leaves at a time.
            auto arrange = [&](uint32_t lf) {
                const int lo = (int)(lf >> 8), len = (int)(lf & 255);
                // everything indexed by constants: registers only
                uint64_t k5[5];
#pragma unroll
                for (int t = 0; t < 5; t++) k5[t] = t < len ? keys[lo + t] : ~0ull;
                leaf_network(k5, len);
                uint32_t hid[5], hkey[5];
                int bs[5];
                uint64_t head = k5[0];
                int start = 0;
#pragma unroll
                for (int t = 0; t < 5; t++) {
                    if (t > 0 && k5[t] > head) {
                        head = k5[t];
                        start = t;
                    }
                    hid[t] = ~(uint32_t)head;
                    hkey[t] = (uint32_t)(head >> 32);
                    bs[t] = start;
                }
                const int base = (int)sz - lo - len;
#pragma unroll
                for (int t = 0; t < 5; t++) {
                    if (t >= len) continue;
                    int before = 0;  // points of blocks with a larger head index
#pragma unroll
                    for (int t2 = 0; t2 < 5; t2++) before += t2 < len && hid[t2] > hid[t];
                    const int pos = base + before + (t - bs[t]);
                    s_ka[pos] = hkey[t];
                    s_val[pos] = (uint16_t)~(uint32_t)k5[t];
                }
            };
            {
                const int lane = tid & 31;
                uint32_t *lq = s_hist + (tid >> 5) * 256;
                int qn = 0;
                for (int64_t p0 = (int64_t)(tid >> 5) * 32; p0 < sz; p0 += NT) {
                    const int64_t p = p0 + lane;
                    int llo = -1, llen = 0;
                    if (p < sz) leaf_of32((int)sz, (int)p, llo, llen);
                    const bool lead = llo == (int)p;
                    const uint32_t lf = (uint32_t)llo << 8 | (uint32_t)llen;
                    const uint32_t bal = __ballot_sync(0xffffffffu, lead);
                    if (lead) lq[qn + __popc(bal & ((1u << lane) - 1u))] = lf;
                    qn += __popc(bal);
                    __syncwarp();
                    if (qn >= 32) {
                        qn -= 32;
                        arrange(lq[qn + lane]);
                        __syncwarp();
                    }
                }
                if (lane < qn) arrange(lq[lane]);
            }
            __syncthreads();
            FIT_PROF(4)
            block_radix_sort32(s_ka, s_val, s_kb, s_vb, (int)sz, s_hist);
        } else {
            for (int64_t p = tid; p < sz; p += NT) {
                uint32_t lf = leaf_of(sz, p);
                int64_t lo = lf >> 8, len = lf & 255;
                if (p != lo) continue;
                uint64_t k5[5];
                for (int t = 0; t < len; t++) k5[t] = keys[lo + t];
                leaf_network(k5, (int)len);
                uint64_t head = 0;
                for (int t = 0; t < len; t++) {
                    if (t == 0 || k5[t] > head) head = k5[t];
                    uint32_t hidx = ~(uint32_t)head;
                    sk[lo + t] = (head & 0xffffffff00000000ull) | (uint64_t)(0xffffu - hidx) << 3 | (uint64_t)t;
                    sv[lo + t] = ~(uint32_t)k5[t];
                }
            }
            __syncthreads();
            FIT_PROF(4)
            // the merge's second buffer: two scratch arrays
            uint64_t *kb = reinterpret_cast<uint64_t *>(scr.w + s0);
            uint32_t *vb = reinterpret_cast<uint32_t *>(scr.fx + s0);
            block_merge_sort(sk, sv, kb, vb, (int)sz);
        }
        FIT_PROF(5)

        // cumulative weighted moments in angle order (fast/quads.c:968-1035):
        // w = sqrt(gx^2 + gy^2) + 1 on the quad image (1 at its border),
        // fx = x/2 + 1/2. Chunks of points get their six terms (w fx, w fy,
        // w fx fx, w fx fy, w fy fy, w; the reference's products) staged in
        // shared memory, two buffers deep: while lane q < 6 of warp 0 runs
        // prefix sum q over chunk c in point order, the other warps stage
        // chunk c + 1.
        const uint8_t *im = qim + f.q_off;
        double *M[6] = {scr.mx + s0, scr.my + s0, scr.mxx + s0, scr.mxy + s0, scr.myy + s0, scr.mw + s0};
        double run = 0.0;
        const int cs = chunk + 2;  // row stride of the staged terms
        auto stage = [&](int64_t k0, double *buf, int first, int stride) {
            const int64_t kn = dmin((int64_t)chunk, sz - k0);
            for (int64_t t = first; t < kn; t += stride) {
                const uint32_t src = in_smem ? (uint32_t)s_val[k0 + t] : sv[k0 + t];
                const uint64_t pt = P[src];
                const int32_t px = (int32_t)(pt & 0xffff), py = (int32_t)(pt >> 16 & 0xffff);
                const int32_t ix = (px >> 1) + (px & 1), iy = (py >> 1) + (py & 1);
                int32_t g2 = 0;
                if (ix > 0 && ix + 1 < f.qw && iy > 0 && iy + 1 < f.qh) {
                    const int64_t cc = (int64_t)iy * f.qw + ix;
                    const int32_t gx = (int32_t)im[cc + 1] - im[cc - 1];
                    const int32_t gy = (int32_t)im[cc + f.qw] - im[cc - f.qw];
                    g2 = gx * gx + gy * gy;
                }
                const double w = __dadd_rn(__dsqrt_rn((double)g2), 1.0);
                const double fx = __dadd_rn(__dmul_rn((double)px, 0.5), 0.5);
                const double fy = __dadd_rn(__dmul_rn((double)py, 0.5), 0.5);
                const double wx = __dmul_rn(w, fx), wy = __dmul_rn(w, fy);
                buf[0 * cs + t] = wx;
                buf[1 * cs + t] = wy;
                buf[2 * cs + t] = __dmul_rn(wx, fx);
                buf[3 * cs + t] = __dmul_rn(wx, fy);
                buf[4 * cs + t] = __dmul_rn(wy, fy);
                buf[5 * cs + t] = w;
            }
        };
        // the prefix sums are taken in place in shared memory; the other
        // warps copy a finished chunk out before staging into its buffer
        auto copy_out = [&](int64_t k0, const double *buf, int first, int stride) {
            const int64_t kn = dmin((int64_t)chunk, sz - k0);
            for (int64_t t = first; t < 6 * kn; t += stride) {
                const int64_t q = t / kn, i = t - q * kn;
                M[q][k0 + i] = buf[q * cs + i];
            }
        };
        stage(0, s_w, tid, NT);
        __syncthreads();
        int64_t ch = 0;
        for (int64_t k0 = 0; k0 < sz; k0 += chunk, ch++) {
            double *cur = s_w + (ch & 1) * 6 * cs, *oth = s_w + ((ch + 1) & 1) * 6 * cs;
            if (tid < 32) {
                if (tid < 6) {
                    const int64_t kn = dmin((int64_t)chunk, sz - k0);
                    double *src = cur + tid * cs;
                    int64_t t = 0;
                    // 16 loads, the 16 dependent additions, then 16 stores:
                    // stores between the additions would lengthen the chain
                    for (; t + 16 <= kn; t += 16) {
                        double v[16];
#pragma unroll
                        for (int u = 0; u < 16; u++) v[u] = src[t + u];
#pragma unroll
                        for (int u = 0; u < 16; u++) {
                            run = __dadd_rn(run, v[u]);
                            v[u] = run;
                        }
#pragma unroll
                        for (int u = 0; u < 16; u++) src[t + u] = v[u];
                    }
                    for (; t < kn; t++) {
                        run = __dadd_rn(run, src[t]);
                        src[t] = run;
                    }
                }
            } else {
                if (ch > 0) copy_out(k0 - chunk, oth, tid - 32, NT - 32);
                asm volatile("bar.sync 1, %0;" ::"r"(NT - 32));
                if (k0 + chunk < sz) stage(k0 + chunk, oth, tid - 32, NT - 32);
            }
            __syncthreads();
        }
        if (ch > 0) copy_out((ch - 1) * chunk, s_w + ((ch - 1) & 1) * 6 * cs, tid, NT);
        __syncthreads();
        const Moments mo = {M[0], M[1], M[2], M[3], M[4], M[5]};
        FIT_PROF(6)

        // corner search (fast/quads.c:788-959)
        const int64_t ksz = dmin(20, sz / 12);
        if (ksz < 2) continue;
        const double nn = (double)(2 * ksz + 1);
        double *errs = scr.errs + s0, *filt = scr.filt + s0;
        // two points a thread at a time: both windows' loads before either
        // store (a store could alias the next loads)
        for (int64_t i = tid; i < sz; i += 2 * NT) {
            const int64_t i2 = i + NT < sz ? i + NT : i;
            const MSum sa = window_moments(mo, sz, ksz, i), sb = window_moments(mo, sz, ksz, i2);
            const double ea = window_error(sa, nn), eb = window_error(sb, nn);
            errs[i] = ea;
            errs[i2] = eb;
        }
        __syncthreads();
        for (int64_t i = tid; i < sz; i += 2 * NT) {
            const int64_t i2 = i + NT < sz ? i + NT : i;
            const double fa = smooth_at(errs, sz, i, prm.qsm), fb = smooth_at(errs, sz, i2, prm.qsm);
            filt[i] = fa;
            filt[i2] = fb;
        }
        __syncthreads();
        FIT_PROF(7)
        // local maxima with wrap-around, compacted in index order
        int32_t *mxi = scr.mxi + s0;
        double *mxe = scr.mxe + s0;
        int64_t nm_run = 0;
        for (int64_t i0 = 0; i0 < sz; i0 += NT) {
            int64_t i = i0 + tid;
            uint32_t is_max = 0;
            double e = 0.0;
            if (i < sz) {
                e = filt[i];
                double l = filt[i == 0 ? sz - 1 : i - 1], r = filt[i + 1 == sz ? 0 : i + 1];
                is_max = e > l && e > r;
            }
            uint32_t total;
            uint32_t off = block_excl_scan(is_max, &total, s_scan);
            if (is_max) {
                mxi[nm_run + off] = (int32_t)i;
                mxe[nm_run + off] = e;
            }
            nm_run += total;
        }
        __syncthreads();
        int64_t nm = nm_run;
        if (nm < 4) continue;
        if (nm > prm.max_nmaxima) {
            // The reference keeps the maxima whose error is above the
            // (max_nmaxima+1)-th largest (its quickselect, quads.c:827-862).
            // e_i exceeds that order statistic exactly when at most
            // max_nmaxima errors are >= e_i: a parallel count, then an
            // order-keeping compaction.
            // The order statistic by a radix select over the errors'
            // order-preserving 64-bit images, 8 bits a pass: e_i is kept
            // exactly when e_i > T, T the (max_nmaxima+1)-th largest.
            const int64_t k = prm.max_nmaxima;
            double *e = in_smem && nm <= sort_cap ? reinterpret_cast<double *>(s_key) : filt;
            for (int64_t i = tid; i < nm; i += NT) e[i] = mxe[i];
            const double T = block_select_desc(e, nm, (uint32_t)k, s_hist, &s_selp, &s_selr);
            int64_t kept_run = 0;
            for (int64_t i0 = 0; i0 < nm; i0 += NT) {
                int64_t i = i0 + tid;
                uint32_t keep = 0;
                if (i < nm) keep = e[i] > T;
                uint32_t total;
                uint32_t off = block_excl_scan(keep, &total, s_scan);
                int32_t mi = i < nm ? mxi[i] : 0;
                __syncthreads();
                if (keep) mxi[kept_run + off] = mi;
                kept_run += total;
            }
            __syncthreads();
            nm = kept_run;
        }
        FIT_PROF(8)
        // line fits of pairs of maxima: (a, b), a < b, and the closing pair
        // (b, a) wrapping around for b >= a + 3
        for (int64_t t = tid; t < nm * nm; t += NT) {
            int64_t p = t / nm, q = t - p * nm;
            bool used = p < q || p >= q + 3;
            if (!used) continue;
            int64_t i0 = mxi[p], i1 = mxi[q];
            MSum s = seg_moments(mo, sz, i0, i1);
            double n = (double)(i0 <= i1 ? i1 - i0 + 1 : sz - i0 + i1 + 1);
            double lp[4], mse;
            line_of(s, lp, &mse);
            s_perr[t] = n * mse;
            s_pmse[t] = mse;
            s_pnx[t] = lp[2];
            s_pny[t] = lp[3];
        }
        __syncthreads();
        FIT_PROF(9)
        // the 4 maxima with the smallest total error (quads.c:931-958): the
        // reference keeps the first strictly smaller error in (m0, m1, m2, m3)
        // order, i.e. the smallest error and, among equal ones, the first in
        // that order. Each thread scans some (m0, m1, m2) triples; then a
        // block-wide minimum of (error, order).
        {
            const double inf = __longlong_as_double(0x7ff0000000000000ll);
            double be = inf;
            int64_t bo = INT64_MAX;
            for (int64_t t = tid; t < nm * nm * nm; t += NT) {
                const int64_t m0 = t / (nm * nm), m1 = (t / nm) % nm, m2 = t % nm;
                if (!(m0 < m1 && m1 < m2 && m2 < nm - 1)) continue;
                const int64_t p01 = m0 * nm + m1, p12 = m1 * nm + m2;
                if (s_pmse[p01] > prm.max_mse || s_pmse[p12] > prm.max_mse) continue;
                const double dot = s_pnx[p01] * s_pnx[p12] + s_pny[p01] * s_pny[p12];
                if (fabs(dot) > prm.max_dot) continue;
                const double e012 = s_perr[p01] + s_perr[p12];
                for (int64_t m3 = m2 + 1; m3 < nm; m3++) {
                    const int64_t p23 = m2 * nm + m3, p30 = m3 * nm + m0;
                    const double e23 = s_pmse[p23] > prm.max_mse ? inf : s_perr[p23];
                    const double e30 = s_pmse[p30] > prm.max_mse ? inf : s_perr[p30];
                    const double e = e012 + e23 + e30;
                    if (e < be) {  // within a thread: ascending order already
                        be = e;
                        bo = t * nm + m3;
                    }
                }
            }
            // block minimum of (be, bo)
            for (int o = 16; o > 0; o >>= 1) {
                double e2 = __shfl_xor_sync(0xffffffffu, be, o);
                int64_t o2 = __shfl_xor_sync(0xffffffffu, bo, o);
                if (e2 < be || (e2 == be && o2 < bo)) {
                    be = e2;
                    bo = o2;
                }
            }
            if ((tid & 31) == 0) {
                s_be[tid >> 5] = be;
                s_bo[tid >> 5] = bo;
            }
            __syncthreads();
            if (tid == 0) {
                for (int w = 1; w < NT / 32; w++)
                    if (s_be[w] < be || (s_be[w] == be && s_bo[w] < bo)) {
                        be = s_be[w];
                        bo = s_bo[w];
                    }
                s_be[0] = be;
                s_bo[0] = bo;
            }
            __syncthreads();
            be = s_be[0];
            bo = s_bo[0];
            // the 4 line fits (quads.c:1069-1075), one per thread
            if (be != inf && tid < 4) {
                const int64_t t = bo / nm, m3 = bo % nm;
                const int64_t mi[4] = {t / (nm * nm), (t / nm) % nm, t % nm, m3};
                double mse;
                line_of(seg_moments(mo, sz, mxi[mi[tid]], mxi[mi[(tid + 1) & 3]]), s_lines[tid], &mse);
                s_lmse[tid] = mse;
            }
            __syncthreads();
            if (tid == 0) s_best = be;
        }
        if (tid == 0) {
            const double inf = __longlong_as_double(0x7ff0000000000000ll);
            const double best = s_best;
            bool ok = best != inf && best / (double)sz < prm.max_mse;
            GpuQuad q;
            q.reversed_border = rev;
            q.frame = cframe[c];
            double lines[4][4];
            for (int i = 0; ok && i < 4; i++) {
                for (int k = 0; k < 4; k++) lines[i][k] = s_lines[i][k];
                if (s_lmse[i] > prm.max_mse) ok = false;
            }
            for (int i = 0; ok && i < 4; i++) {
                int j = (i + 1) & 3;
                double a00 = lines[i][3], a01 = -lines[j][3], a10 = -lines[i][2], a11 = lines[j][2];
                double b0 = -lines[i][0] + lines[j][0], b1 = -lines[i][1] + lines[j][1];
                double det = a00 * a11 - a10 * a01;
                if (fabs(det) < 0.001) {
                    ok = false;
                    break;
                }
                double w00 = a11 / det, w01 = -a01 / det;
                double l0 = w00 * b0 + w01 * b1;
                q.p[i][0] = (float)(lines[i][0] + l0 * a00);
                q.p[i][1] = (float)(lines[i][1] + l0 * a10);
            }
            if (ok) {
                // area of triangles (0,1,2) and (2,3,0) by Heron (quads.c:1094-1110)
                const int tri[2][4] = {{0, 1, 2, 0}, {2, 3, 0, 2}};
                double area = 0.0;
                for (int t = 0; t < 2; t++) {
                    double len[3];
                    for (int i = 0; i < 3; i++) {
                        int ia = tri[t][i], ib = tri[t][i + 1];
                        double ddx = (double)__fsub_rn(q.p[ib][0], q.p[ia][0]);
                        double ddy = (double)__fsub_rn(q.p[ib][1], q.p[ia][1]);
                        len[i] = sqrt(ddx * ddx + ddy * ddy);
                    }
                    double pp = (len[0] + len[1] + len[2]) / 2.0;
                    area = area + sqrt(pp * (pp - len[0]) * (pp - len[1]) * (pp - len[2]));
                }
                if (area < 0.95 * (double)f.tag_width * (double)f.tag_width) ok = false;
            }
            for (int i = 0; ok && i < 4; i++) {
                // convexity (quads.c:1112-1124)
                int i0 = i, i1 = (i + 1) & 3, i2 = (i + 2) & 3;
                double dx1 = (double)__fsub_rn(q.p[i1][0], q.p[i0][0]), dy1 = (double)__fsub_rn(q.p[i1][1], q.p[i0][1]);
                double dx2 = (double)__fsub_rn(q.p[i2][0], q.p[i1][0]), dy2 = (double)__fsub_rn(q.p[i2][1], q.p[i1][1]);
                double den = sqrt((dx1 * dx1 + dy1 * dy1) * (dx2 * dx2 + dy2 * dy2));
                if (den == 0.0) {
                    ok = false;
                    break;
                }
                double cs = (dx1 * dx2 + dy1 * dy2) / den;
                if ((cs > prm.max_dot || cs < -prm.max_dot) || dx1 * dy2 < dy1 * dx2) ok = false;
            }
            if (ok) {
                quads[c] = q;
                quad_ok[c] = 1;
            }
            FIT_PROF(10)
#ifdef AT_FIT_PROF
            if (c < 16384) g_fitprof[c][0] = sz;
#endif
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// The fit's size classes: clusters of at most 128, 256, 512 points (a warp
// each), at most 1024 (a block of 128), and larger (a block of 512). Each
// class gets a list of its clusters; clusters outside [min_cluster_pixels,
// max_px] of their frame get none (fast/quads.c:1180-1190). Every cluster's
// quad flag starts at 0.
#define FIT_NCLASS 5
__device__ __forceinline__ int fit_class(int64_t sz) {
    return sz <= 128 ? 0 : sz <= 256 ? 1 : sz <= 512 ? 2 : sz <= 1024 ? 3 : 4;
}

__global__ void k_fit_classify(const FrameDesc *frames, const uint32_t *cstart, const int32_t *cframe,
                               int64_t nclusters, int64_t npoints, int32_t min_px, uint32_t *quad_ok,
                               uint32_t *lists, uint32_t *counts) {
    const int lane = threadIdx.x & 31;
    for (int64_t c0 = (int64_t)blockIdx.x * blockDim.x; c0 < nclusters; c0 += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = c0 + threadIdx.x;
        int k = -1;
        if (c < nclusters) {
            quad_ok[c] = 0;
            const int64_t sz = (c + 1 < nclusters ? (int64_t)cstart[c + 1] : npoints) - cstart[c];
            if (sz >= min_px && sz <= frames[cframe[c]].max_px) k = fit_class(sz);
        }
#pragma unroll
        for (int q = 0; q < FIT_NCLASS; q++) {
            const uint32_t bal = __ballot_sync(0xffffffffu, k == q);
            if (!bal) continue;
            uint32_t at = 0;
            if (lane == __ffs(bal) - 1) at = atomicAdd(counts + q, (uint32_t)__popc(bal));
            at = __shfl_sync(0xffffffffu, at, __ffs(bal) - 1);
            if (k == q) lists[(int64_t)q * nclusters + at + __popc(bal & ((1u << lane) - 1u))] = (uint32_t)c;
        }
    }
}

// One block per list: the list by size, largest first (then by cluster),
// when it has at most FIT_ORDER_CAP clusters; a bitonic sort in shared
// memory.
#define FIT_ORDER_CAP 8192
__global__ void __launch_bounds__(1024) k_fit_order(const uint32_t *cstart, int64_t nclusters, int64_t npoints,
                                                   uint32_t *lists, const uint32_t *counts, int first_class) {
    extern __shared__ __align__(16) uint64_t s_ord[];
    const int q = first_class + blockIdx.x;
    const uint32_t n = counts[q];
    if (n < 2 || n > FIT_ORDER_CAP) return;
    uint32_t *list = lists + (int64_t)q * nclusters;
    uint32_t np = 2;
    while (np < n) np <<= 1;
    for (uint32_t i = threadIdx.x; i < np; i += blockDim.x) {
        uint64_t key = ~0ull;
        if (i < n) {
            const uint32_t c = list[i];
            const int64_t sz = (c + 1 < nclusters ? (int64_t)cstart[c + 1] : npoints) - cstart[c];
            key = (uint64_t)(0xffffffffu - (uint32_t)sz) << 32 | c;
        }
        s_ord[i] = key;
    }
    __syncthreads();
    for (uint32_t kk = 2; kk <= np; kk <<= 1)
        for (uint32_t j = kk >> 1; j > 0; j >>= 1) {
            for (uint32_t t = threadIdx.x; t < np / 2; t += blockDim.x) {
                const uint32_t i = ((t & ~(j - 1)) << 1) | (t & (j - 1)), l = i + j;
                const uint64_t a = s_ord[i], b = s_ord[l];
                if (((i & kk) == 0) == (a > b)) {
                    s_ord[i] = b;
                    s_ord[l] = a;
                }
            }
            __syncthreads();
        }
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) list[i] = (uint32_t)s_ord[i];
}

// ---------------------------------------------------------------------------
// Clusters of at most 32 * R points: one warp each, FIT_WPB per block, no
// block barriers. The same steps as k_fit_quads; the angle sort is a bitonic
// sort in registers, the prefix moments stay in shared memory.
#define FIT_WPB 2

// The 4-subsets {m0 < m1 < m2 < m3} of {0..15} in colex order (by m3, then
// m2, m1, m0), one per entry as nibbles m0 | m1 << 4 | m2 << 8 | m3 << 12:
// the first C(n, 4) entries are the 4-subsets of {0..n-1}.
struct Quad4Table {
    uint16_t v[1820];
};
constexpr Quad4Table make_quad4() {
    Quad4Table t{};
    int k = 0;
    for (int d = 3; d < 16; d++)
        for (int c = 2; c < d; c++)
            for (int b = 1; b < c; b++)
                for (int a = 0; a < b; a++) t.v[k++] = (uint16_t)(a | b << 4 | c << 8 | d << 12);
    return t;
}
__device__ const Quad4Table g_quad4 = make_quad4();
static_assert(AT_MAX_NMAXIMA <= 16, "the 4-subset table covers 16 maxima");

__host__ __device__ constexpr int binom4(int n) { return n < 4 ? 0 : n * (n - 1) * (n - 2) * (n - 3) / 24; }

// per warp: six prefix arrays, then region x0 (angle keys; errors; the
// maxima) and region x1 (dot terms; filtered errors; the pair fits)
__host__ __device__ constexpr size_t fit_warp_x1(int cap, int mm) {
    return (size_t)8 * cap > (size_t)32 * mm * mm ? (size_t)8 * cap : (size_t)32 * mm * mm;
}
// gp: the prefix arrays in global scratch (the largest warp class, where
// 48 B per point of shared memory would leave few warps per SM)
__host__ __device__ constexpr size_t fit_warp_smem(int cap, int mm, bool gp = false) {
    return (size_t)(gp ? 8 : 56) * cap + fit_warp_x1(cap, mm);
}



// Bitonic sort, ascending, of a warp's keys k[0, np) in shared memory (np
// a power of two): log2(np) (log2(np) + 1) / 2 steps of np / 2 exchanges.
__device__ void warp_bitonic(uint64_t *k, int np, int lane) {
    for (int kk = 2; kk <= np; kk <<= 1) {
        for (int j = kk >> 1; j > 0; j >>= 1) {
            for (int q = lane; q < np / 2; q += 32) {
                const int i = ((q & ~(j - 1)) << 1) | (q & (j - 1)), l = i + j;
                const uint64_t a = k[i], b = k[l];
                if (((i & kk) == 0) == (a > b)) {
                    k[i] = b;
                    k[l] = a;
                }
            }
            __syncwarp();
        }
    }
}

// Stable sort of a warp's n (32-bit key, 16-bit value) pairs by key: four
// passes of 8 bits; equal digits keep their order (ranked by lane among 32
// consecutive pairs, match_any). ka/va hold the input and get the result,
// kb/vb are the second buffers, hist 256 counters.
__device__ void warp_radix_sort32(uint32_t *ka, uint16_t *va, uint32_t *kb, uint16_t *vb, int n, uint32_t *hist,
                                  int lane) {
    for (int shift = 0; shift < 32; shift += 8) {
#pragma unroll
        for (int j = 0; j < 8; j++) hist[lane * 8 + j] = 0;
        __syncwarp();
        for (int i = lane; i < n; i += 32) atomicAdd(hist + (ka[i] >> shift & 255u), 1u);
        __syncwarp();
        uint32_t c[8], sum = 0;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            c[j] = hist[lane * 8 + j];
            sum += c[j];
        }
        uint32_t incl = sum;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        uint32_t run = incl - sum;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            hist[lane * 8 + j] = run;
            run += c[j];
        }
        __syncwarp();
        for (int i0 = 0; i0 < n; i0 += 32) {
            const int i = i0 + lane;
            const bool valid = i < n;
            const uint32_t k = valid ? ka[i] : 0;
            const int d = valid ? (int)(k >> shift & 255u) : 256 + lane;
            const uint32_t peers = __match_any_sync(0xffffffffu, d);
            const uint32_t base = valid ? hist[d] : 0;
            if (valid) {
                const uint32_t at = base + __popc(peers & ((1u << lane) - 1u));
                kb[at] = k;
                vb[at] = va[i];
            }
            __syncwarp();
            if (valid && lane == __ffs(peers) - 1) hist[d] = base + __popc(peers);
            __syncwarp();
        }
        uint32_t *tk = ka;
        ka = kb;
        kb = tk;
        uint16_t *tv = va;
        va = vb;
        vb = tv;
    }
}

template <int R>
__global__ void __launch_bounds__(FIT_WPB * 32, 12) k_fit_warp(const FrameDesc *frames, GpuParams prm, const uint8_t *qim,
                                                          const uint64_t *pts, const uint32_t *cstart,
                                                          const int32_t *cframe, int64_t nclusters, int64_t npoints,
                                                          const uint32_t *list, const uint32_t *count,
                                                          uint32_t *next, GpuQuad *quads, uint32_t *quad_ok, int mm,
                                                          FitScratch scr) {
    constexpr int CAP = 32 * R;
    constexpr bool GP = R >= 16;  // prefix arrays in global scratch
    extern __shared__ __align__(16) unsigned char fw_smem[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned FULL = 0xffffffffu;
    unsigned char *base = fw_smem + fit_warp_smem(CAP, mm, GP) * wid;
    double *pm = reinterpret_cast<double *>(base);  // prefix array q at pm + q * CAP (not GP)
    unsigned char *x0 = base + (GP ? 0 : 48 * CAP), *x1 = x0 + 8 * CAP;
    uint64_t *s_akey = reinterpret_cast<uint64_t *>(x0);
    double *s_err = reinterpret_cast<double *>(x0);
    double *s_mxe = reinterpret_cast<double *>(x0);
    int32_t *s_mxi = reinterpret_cast<int32_t *>(x0 + 4 * CAP);
    float *s_term = reinterpret_cast<float *>(x1);
    double *s_filt = reinterpret_cast<double *>(x1);
    double *s_perr = reinterpret_cast<double *>(x1), *s_pmse = s_perr + mm * mm, *s_pnx = s_pmse + mm * mm,
           *s_pny = s_pnx + mm * mm;
    const double inf = __longlong_as_double(0x7ff0000000000000ll);

    // one resident wave of warps, each taking the class's next cluster
    // from a shared counter as it finishes one (no static share to wait on)
    const uint32_t ncl = *count;
    for (;;) {
        uint32_t li = 0;
        if (lane == 0) li = atomicAdd(next, 1u);
        li = __shfl_sync(FULL, li, 0);
        if (li >= ncl) break;
        const int64_t c = list[li];
        const int64_t s0 = cstart[c];
        const int64_t sz = (c + 1 < nclusters ? (int64_t)cstart[c + 1] : npoints) - s0;
        const FrameDesc f = frames[cframe[c]];
        const int n = (int)sz;
        FITW_SIZE(n)
        FITW_PROF(1)
        const uint64_t *P = pts + s0;
        // bounding box (fast/quads.c:515-528)
        uint32_t xmin = 0xffff, xmax = 0, ymin = 0xffff, ymax = 0;
        for (int i = lane; i < n; i += 32) {
            const uint64_t pt = P[i];
            const uint32_t x = (uint32_t)(pt & 0xffff), y = (uint32_t)(pt >> 16 & 0xffff);
            xmin = min(xmin, x);
            xmax = max(xmax, x);
            ymin = min(ymin, y);
            ymax = max(ymax, y);
        }
        for (int o = 16; o > 0; o >>= 1) {
            xmin = min(xmin, __shfl_xor_sync(FULL, xmin, o));
            xmax = max(xmax, __shfl_xor_sync(FULL, xmax, o));
            ymin = min(ymin, __shfl_xor_sync(FULL, ymin, o));
            ymax = max(ymax, __shfl_xor_sync(FULL, ymax, o));
        }
        if ((int64_t)(xmax - xmin) * (int64_t)(ymax - ymin) < f.tag_width) continue;
        FITW_PROF(2)
        const float cx = (float)((double)(xmin + xmax) * 0.5 + 0.05118);
        const float cy = (float)((double)(ymin + ymax) * 0.5 + -0.028581);

        // angle keys (fast/quads.c:429-453) and the dot product of offsets
        // and gradients (fast/quads.c:467-512): lane l < 8 sums terms l,
        // l+8, ... of the whole groups of 8; then the rest in order
        const int nv = n - n % 8;
        for (int i = lane; i < n; i += 32) {
            const uint64_t pt = P[i];
            const float dx = __fsub_rn((float)(pt & 0xffff), cx), dy = __fsub_rn((float)(pt >> 16 & 0xffff), cy);
            s_akey[i] = angle_key(dx, dy, (uint32_t)i);
            const float gx = (float)(int16_t)(pt >> 32 & 0xffff), gy = (float)(int16_t)(pt >> 48);
            s_term[i] = __fadd_rn(__fmul_rn(dx, gx), __fmul_rn(dy, gy));
        }
        __syncwarp();
        float acc = 0.0f;
        if (lane < 8) {
            int i = lane;
            for (; i + 56 < nv; i += 64) {
                float v[8];
#pragma unroll
                for (int u = 0; u < 8; u++) v[u] = s_term[i + 8 * u];
#pragma unroll
                for (int u = 0; u < 8; u++) acc = __fadd_rn(acc, v[u]);
            }
            for (; i < nv; i += 8) acc = __fadd_rn(acc, s_term[i]);
        }
        float l8[8];
#pragma unroll
        for (int k = 0; k < 8; k++) l8[k] = __shfl_sync(FULL, acc, k);
        int okrev = 0;
        if (lane == 0) {
            float dot = __fadd_rn(__fadd_rn(__fadd_rn(l8[0], l8[4]), __fadd_rn(l8[2], l8[6])),
                                  __fadd_rn(__fadd_rn(l8[1], l8[5]), __fadd_rn(l8[3], l8[7])));
            for (int i = nv; i < n; i++) dot = __fadd_rn(dot, s_term[i]);
            const int rev = dot < 0.0f;
            int ok = 1;
            if (!f.reversed_border && rev) ok = 0;
            if (!f.normal_border && !rev) ok = 0;
            okrev = ok | rev << 1;
        }
        okrev = __shfl_sync(FULL, okrev, 0);
        if (!(okrev & 1)) continue;
        const int rev = okrev >> 1;
        FITW_PROF(3)

        // The angle sort (see k_fit_quads). Up to 256 points: a bitonic
        // sort of packed keys; above: the points laid out in (head index,
        // place) order and a stable radix sort by the head's slope bits.
        const uint16_t *s_order;  // point index of each sorted position
        if constexpr (R <= 8) {
            // The angle sort (see k_fit_quads): position i of leaf (lo, len)
            // takes place t = i - lo of the leaf's network order; its sort key
            // packs the slope bits of its block head, 0xffff - the head's index,
            // t, and (below the order, since the rest is distinct) the index of
            // its point. The keys live in the last prefix array until the moments.
            uint64_t *s_skey = reinterpret_cast<uint64_t *>(pm + 5 * CAP);
            int np = 32;
            while (np < n) np <<= 1;
            for (int i = lane; i < np; i += 32) {
                uint64_t key = ~0ull;
                if (i < n) {
                    int lo, len;
                    leaf_of32(n, i, lo, len);
                    uint64_t a[5];
    #pragma unroll
                    for (int t = 0; t < 5; t++) a[t] = t < len ? s_akey[lo + t] : ~0ull;
                    leaf_network(a, len);
                    const int tp = i - lo;
                    uint64_t head = a[0], e = a[0];
    #pragma unroll
                    for (int t = 1; t < 5; t++) {
                        if (t <= tp) {
                            if (a[t] > head) head = a[t];
                            e = a[t];
                        }
                    }
                    const uint32_t hidx = ~(uint32_t)head;
                    key = (head & 0xffffffff00000000ull) | (uint64_t)(0xffffu - hidx) << 16 | (uint64_t)tp << 13 |
                          (uint64_t)(~(uint32_t)e & 0x1fffu);
                }
                s_skey[i] = key;
            }
            __syncwarp();
            FITW_PROF(4)
            warp_bitonic(s_skey, np, lane);
            s_order = nullptr;
        } else {
            // The angle sort (see k_fit_quads): the points laid out in (head
            // index descending, place) order, a lane per leaf, then a stable
            // radix sort by the head's slope bits. The sort keys and indices
            // live in region x1, their second buffers and the histogram in the
            // prefix arrays (free until the moments).
            uint32_t *s_ka = reinterpret_cast<uint32_t *>(x1);
            uint16_t *s_va = reinterpret_cast<uint16_t *>(x1 + 4 * CAP);
            // second buffers: in x0 once the angle keys are read (GP: x0
            // holds 8 B per point of capacity, 4 + 2 for the buffers and
            // 1 KB for the histogram)
            unsigned char *sb = GP ? x0 : reinterpret_cast<unsigned char *>(pm);
            uint32_t *s_kb = reinterpret_cast<uint32_t *>(sb);
            uint16_t *s_vb = reinterpret_cast<uint16_t *>(sb + 4 * CAP);
            uint32_t *s_hist = reinterpret_cast<uint32_t *>(sb + (GP ? 6 : 8) * CAP);
            for (int p = lane; p < n; p += 32) {
                int lo, len;
                leaf_of32(n, p, lo, len);
                if (p != lo) continue;
                uint64_t a[5];
    #pragma unroll
                for (int t = 0; t < 5; t++) a[t] = t < len ? s_akey[lo + t] : ~0ull;
                leaf_network(a, len);
                uint32_t hid[5], hkey[5];
                int bs[5];
                uint64_t head = a[0];
                int start = 0;
    #pragma unroll
                for (int t = 0; t < 5; t++) {
                    if (t > 0 && a[t] > head) {
                        head = a[t];
                        start = t;
                    }
                    hid[t] = ~(uint32_t)head;
                    hkey[t] = (uint32_t)(head >> 32);
                    bs[t] = start;
                }
                const int base = n - lo - len;
    #pragma unroll
                for (int t = 0; t < 5; t++) {
                    if (t >= len) continue;
                    int before = 0;
    #pragma unroll
                    for (int t2 = 0; t2 < 5; t2++) before += t2 < len && hid[t2] > hid[t];
                    const int pos = base + before + (t - bs[t]);
                    s_ka[pos] = hkey[t];
                    s_va[pos] = (uint16_t)~(uint32_t)a[t];
                }
            }
            __syncwarp();
            FITW_PROF(4)
            warp_radix_sort32(s_ka, s_va, s_kb, s_vb, n, s_hist, lane);
            __syncwarp();
            s_order = s_va;
        }
        FITW_PROF(5)

        // cumulative weighted moments in angle order (fast/quads.c:968-1035):
        // every lane stages the six terms of its positions, then lane q < 6
        // turns array q into its prefix sums in place
        double *M0 = GP ? scr.mx + s0 : pm, *M1 = GP ? scr.my + s0 : pm + CAP, *M2 = GP ? scr.mxx + s0 : pm + 2 * CAP,
               *M3 = GP ? scr.mxy + s0 : pm + 3 * CAP, *M4 = GP ? scr.myy + s0 : pm + 4 * CAP,
               *M5 = GP ? scr.mw + s0 : pm + 5 * CAP;
        const uint8_t *im = qim + f.q_off;
        for (int k = lane; k < n; k += 32) {
            uint32_t src;
            if constexpr (R <= 8)
                src = (uint32_t)(reinterpret_cast<const uint64_t *>(pm + 5 * CAP)[k] & 0x1fffu);
            else
                src = s_order[k];
            const uint64_t p = P[src];
            const int32_t px = (int32_t)(p & 0xffff), py = (int32_t)(p >> 16 & 0xffff);
            const int32_t ix = (px >> 1) + (px & 1), iy = (py >> 1) + (py & 1);
            int32_t g2 = 0;
            if (ix > 0 && ix + 1 < f.qw && iy > 0 && iy + 1 < f.qh) {
                const int64_t cc = (int64_t)iy * f.qw + ix;
                const int32_t gx = (int32_t)im[cc + 1] - im[cc - 1];
                const int32_t gy = (int32_t)im[cc + f.qw] - im[cc - f.qw];
                g2 = gx * gx + gy * gy;
            }
            const double w = __dadd_rn(__dsqrt_rn((double)g2), 1.0);
            const double fx = __dadd_rn(__dmul_rn((double)px, 0.5), 0.5);
            const double fy = __dadd_rn(__dmul_rn((double)py, 0.5), 0.5);
            const double wx = __dmul_rn(w, fx), wy = __dmul_rn(w, fy);
            M0[k] = wx;
            M1[k] = wy;
            M2[k] = __dmul_rn(wx, fx);
            M3[k] = __dmul_rn(wx, fy);
            M4[k] = __dmul_rn(wy, fy);
            M5[k] = w;
        }
        __syncwarp();
        if (lane < 6) {
            double *o = lane == 0 ? M0 : lane == 1 ? M1 : lane == 2 ? M2 : lane == 3 ? M3 : lane == 4 ? M4 : M5;
            double run = 0.0;
            int t = 0;
            for (; t + 16 <= n; t += 16) {
                double v[16];
#pragma unroll
                for (int u = 0; u < 16; u++) v[u] = o[t + u];
#pragma unroll
                for (int u = 0; u < 16; u++) {
                    run = __dadd_rn(run, v[u]);
                    v[u] = run;
                }
#pragma unroll
                for (int u = 0; u < 16; u++) o[t + u] = v[u];
            }
            for (; t < n; t++) {
                run = __dadd_rn(run, o[t]);
                o[t] = run;
            }
        }
        __syncwarp();
        FITW_PROF(6)
        const Moments mo = {M0, M1, M2, M3, M4, M5};

        // corner search (fast/quads.c:788-959)
        const int ksz = min(20, n / 12);
        if (ksz < 2) continue;
        const double nn = (double)(2 * ksz + 1);
        for (int i = lane; i < n; i += 64) {
            const int i2 = i + 32 < n ? i + 32 : i;
            const MSum sa = window_moments(mo, n, ksz, i), sb = window_moments(mo, n, ksz, i2);
            const double ea = window_error(sa, nn), eb = window_error(sb, nn);
            s_err[i] = ea;
            s_err[i2] = eb;
        }
        __syncwarp();
        for (int i = lane; i < n; i += 64) {
            const int i2 = i + 32 < n ? i + 32 : i;
            const double fa = smooth_at(s_err, n, i, prm.qsm), fb = smooth_at(s_err, n, i2, prm.qsm);
            s_filt[i] = fa;
            s_filt[i2] = fb;
        }
        __syncwarp();
        FITW_PROF(7)
        int nm = 0;
        for (int i0 = 0; i0 < n; i0 += 32) {
            const int i = i0 + lane;
            bool is_max = false;
            double e = 0.0;
            if (i < n) {
                e = s_filt[i];
                const double lft = s_filt[i == 0 ? n - 1 : i - 1], rgt = s_filt[i + 1 == n ? 0 : i + 1];
                is_max = e > lft && e > rgt;
            }
            const uint32_t bal = __ballot_sync(FULL, is_max);
            if (is_max) {
                const int at = nm + __popc(bal & ((1u << lane) - 1u));
                s_mxi[at] = i;
                s_mxe[at] = e;
            }
            nm += __popc(bal);
        }
        __syncwarp();
        if (nm < 4) continue;
        if (nm > prm.max_nmaxima) {
            // keep e_i when at most max_nmaxima errors are >= e_i (quads.c:827-862)
            const int k = prm.max_nmaxima;
            int kept = 0;
            for (int i0 = 0; i0 < nm; i0 += 32) {
                const int i = i0 + lane;
                bool keep = false;
                int32_t mi = 0;
                if (i < nm) {
                    const double ei = s_mxe[i];
                    int ge = 0;
                    for (int j = 0; j < nm && ge <= k; j++) ge += s_mxe[j] >= ei;
                    keep = ge <= k;
                    mi = s_mxi[i];
                }
                const uint32_t bal = __ballot_sync(FULL, keep);
                __syncwarp();
                if (keep) s_mxi[kept + __popc(bal & ((1u << lane) - 1u))] = mi;
                kept += __popc(bal);
            }
            __syncwarp();
            nm = kept;
        }
        FITW_PROF(8)
        // line fits of pairs of maxima
        for (int t = lane; t < nm * nm; t += 32) {
            const int p = t / nm, q = t - p * nm;
            if (!(p < q || p >= q + 3)) continue;
            const int i0 = s_mxi[p], i1 = s_mxi[q];
            const MSum s = seg_moments(mo, n, i0, i1);
            const double cnt = (double)(i0 <= i1 ? i1 - i0 + 1 : n - i0 + i1 + 1);
            double lp[4], mse;
            line_of(s, lp, &mse);
            s_perr[t] = cnt * mse;
            s_pmse[t] = mse;
            s_pnx[t] = lp[2];
            s_pny[t] = lp[3];
        }
        __syncwarp();
        FITW_PROF(9)
        // the first smallest total error in (m0, m1, m2, m3) order: the
        // smallest (error, m0 m1 m2 m3) over the 4-subsets of the maxima
        double be = inf;
        int bo = 0xffff;
        const int nsub = binom4(nm);
        for (int t = lane; t < nsub; t += 32) {
            const int v = g_quad4.v[t];
            const int m0 = v & 15, m1 = v >> 4 & 15, m2 = v >> 8 & 15, m3 = v >> 12;
            const int p01 = m0 * nm + m1, p12 = m1 * nm + m2;
            if (s_pmse[p01] > prm.max_mse || s_pmse[p12] > prm.max_mse) continue;
            const double dot = s_pnx[p01] * s_pnx[p12] + s_pny[p01] * s_pny[p12];
            if (fabs(dot) > prm.max_dot) continue;
            const int p23 = m2 * nm + m3, p30 = m3 * nm + m0;
            const double e012 = s_perr[p01] + s_perr[p12];
            const double e23 = s_pmse[p23] > prm.max_mse ? inf : s_perr[p23];
            const double e30 = s_pmse[p30] > prm.max_mse ? inf : s_perr[p30];
            const double e = e012 + e23 + e30;
            const int ord = m0 << 12 | m1 << 8 | m2 << 4 | m3;
            if (e < be || (e == be && ord < bo)) {
                be = e;
                bo = ord;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double e2 = __shfl_xor_sync(FULL, be, o);
            const int o2 = __shfl_xor_sync(FULL, bo, o);
            if (e2 < be || (e2 == be && o2 < bo)) {
                be = e2;
                bo = o2;
            }
        }
        FITW_PROF(10)
        if (!(be != inf && be / (double)sz < prm.max_mse)) continue;
        // the 4 line fits, lanes 0-3 (quads.c:1069-1075)
        double ln[4] = {0.0, 0.0, 0.0, 0.0}, lmse = 0.0;
        if (lane < 4) {
            const int ma = bo >> (12 - 4 * lane) & 15, mb = bo >> (12 - 4 * ((lane + 1) & 3)) & 15;
            line_of(seg_moments(mo, n, s_mxi[ma], s_mxi[mb]), ln, &lmse);
        }
        double lines[4][4], lm[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            lm[i] = __shfl_sync(FULL, lmse, i);
#pragma unroll
            for (int k = 0; k < 4; k++) lines[i][k] = __shfl_sync(FULL, ln[k], i);
        }
        if (lane == 0) {
            bool ok = true;
            for (int i = 0; i < 4; i++)
                if (lm[i] > prm.max_mse) ok = false;
            GpuQuad q;
            q.reversed_border = rev;
            q.frame = cframe[c];
            for (int i = 0; ok && i < 4; i++) {
                int j = (i + 1) & 3;
                double a00 = lines[i][3], a01 = -lines[j][3], a10 = -lines[i][2], a11 = lines[j][2];
                double b0 = -lines[i][0] + lines[j][0], b1 = -lines[i][1] + lines[j][1];
                double det = a00 * a11 - a10 * a01;
                if (fabs(det) < 0.001) {
                    ok = false;
                    break;
                }
                double w00 = a11 / det, w01 = -a01 / det;
                double l0 = w00 * b0 + w01 * b1;
                q.p[i][0] = (float)(lines[i][0] + l0 * a00);
                q.p[i][1] = (float)(lines[i][1] + l0 * a10);
            }
            if (ok) {
                const int tri[2][4] = {{0, 1, 2, 0}, {2, 3, 0, 2}};
                double area = 0.0;
                for (int t = 0; t < 2; t++) {
                    double len[3];
                    for (int i = 0; i < 3; i++) {
                        int ia = tri[t][i], ib = tri[t][i + 1];
                        double ddx = (double)__fsub_rn(q.p[ib][0], q.p[ia][0]);
                        double ddy = (double)__fsub_rn(q.p[ib][1], q.p[ia][1]);
                        len[i] = sqrt(ddx * ddx + ddy * ddy);
                    }
                    double pp = (len[0] + len[1] + len[2]) / 2.0;
                    area = area + sqrt(pp * (pp - len[0]) * (pp - len[1]) * (pp - len[2]));
                }
                if (area < 0.95 * (double)f.tag_width * (double)f.tag_width) ok = false;
            }
            for (int i = 0; ok && i < 4; i++) {
                int i0 = i, i1 = (i + 1) & 3, i2 = (i + 2) & 3;
                double dx1 = (double)__fsub_rn(q.p[i1][0], q.p[i0][0]), dy1 = (double)__fsub_rn(q.p[i1][1], q.p[i0][1]);
                double dx2 = (double)__fsub_rn(q.p[i2][0], q.p[i1][0]), dy2 = (double)__fsub_rn(q.p[i2][1], q.p[i1][1]);
                double den = sqrt((dx1 * dx1 + dy1 * dy1) * (dx2 * dx2 + dy2 * dy2));
                if (den == 0.0) {
                    ok = false;
                    break;
                }
                double cs = (dx1 * dx2 + dy1 * dy2) / den;
                if ((cs > prm.max_dot || cs < -prm.max_dot) || dx1 * dy2 < dy1 * dx2) ok = false;
            }
            if (ok) {
                quads[c] = q;
                quad_ok[c] = 1;
            }
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// 9. Decoding, one block per quad (fast/decode.c, fast/detector.c:83-139).

struct DView {
    const uint8_t *im;
    int64_t s, w, h;
};

__device__ __forceinline__ double bil_seq(double a, double b, const uint8_t *p, int64_t s) {
    return (1.0 - a) * (1.0 - b) * p[0] + a * (1.0 - b) * p[1] + (1.0 - a) * b * p[s] + a * b * p[s + 1];
}

// One sample point of edge refinement (fast/decode.c:549-735): the
// weighted mean step n0 along the normal, or false when no step counts.
// The first vsteps steps (a multiple of 4) sum into 4 interleaved partial
// sums. They go 4 at a time, each step's 8 pixels loaded before any is
// used (a step outside the image loads pixel (0, 0) and counts 0), so the
// loads of the 4 steps overlap; the rest of the steps follow in order.
__device__ __forceinline__ double bil_vals(double a, double b, int p00, int p01, int p10, int p11) {
    double na = 1.0 - a, nb = 1.0 - b;
    return ((na * nb) * p00 + (a * nb) * p01) + ((na * b) * p10 + (a * b) * p11);
}

__device__ bool refine_sample(const DView &v, double x0, double y0, double nx, double ny, int64_t range,
                              int64_t vsteps, int64_t nsteps, double *n0) {
    const double wl = (double)(v.w - 1), hl = (double)(v.h - 1);
    double ln[4] = {0.0, 0.0, 0.0, 0.0}, lc[4] = {0.0, 0.0, 0.0, 0.0};
    const bool tiny = v.w < 2 || v.h < 2;
    for (int64_t k0 = 0; k0 < vsteps; k0 += 4) {
        bool in[4];
        double fx1[4], fy1[4], fx2[4], fy2[4];
        int px[4][8];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const double n = (double)-range + 0.25 * (double)(k0 + u);
            const double x1 = x0 + (n + 1.0) * nx - 0.5, y1 = y0 + (n + 1.0) * ny - 0.5;
            const double x2 = x0 + (n - 1.0) * nx - 0.5, y2 = y0 + (n - 1.0) * ny - 0.5;
            in[u] = x1 > -1.0 && x1 < wl && y1 > -1.0 && y1 < hl && x2 > -1.0 && x2 < wl && y2 > -1.0 && y2 < hl;
            const double tx1 = trunc(x1), ty1 = trunc(y1), tx2 = trunc(x2), ty2 = trunc(y2);
            fx1[u] = x1 - tx1;
            fy1[u] = y1 - ty1;
            fx2[u] = x2 - tx2;
            fy2[u] = y2 - ty2;
            const bool safe = in[u] || !tiny;
            const uint8_t *p1 = v.im + (in[u] ? (int64_t)ty1 * v.s + (int64_t)tx1 : 0);
            const uint8_t *p2 = v.im + (in[u] ? (int64_t)ty2 * v.s + (int64_t)tx2 : 0);
            if (safe) {
                px[u][0] = p1[0], px[u][1] = p1[1], px[u][2] = p1[v.s], px[u][3] = p1[v.s + 1];
                px[u][4] = p2[0], px[u][5] = p2[1], px[u][6] = p2[v.s], px[u][7] = p2[v.s + 1];
            } else {
#pragma unroll
                for (int t = 0; t < 8; t++) px[u][t] = 0;
            }
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const double n = (double)-range + 0.25 * (double)(k0 + u);
            double wgt = 0.0;
            if (in[u]) {
                const double g1 = bil_vals(fx1[u], fy1[u], px[u][0], px[u][1], px[u][2], px[u][3]);
                const double g2 = bil_vals(fx2[u], fy2[u], px[u][4], px[u][5], px[u][6], px[u][7]);
                const double d = g2 - g1;
                wgt = !(g1 < g2) ? d * d : 0.0;
            }
            ln[u] = ln[u] + wgt * n;
            lc[u] = lc[u] + wgt;
        }
    }
    double mn = 0.0 + ((ln[0] + ln[2]) + (ln[1] + ln[3]));
    double mc = 0.0 + ((lc[0] + lc[2]) + (lc[1] + lc[3]));
    for (int64_t k = vsteps; k < nsteps; k++) {
        double n = (double)-range + 0.25 * (double)k;
        double x1 = x0 + (n + 1.0) * nx - 0.5, y1 = y0 + (n + 1.0) * ny - 0.5;
        int64_t x1i = c_int(x1), y1i = c_int(y1);
        if (x1i < 0 || x1i + 1 >= v.w || y1i < 0 || y1i + 1 >= v.h) continue;
        double x2 = x0 + (n - 1.0) * nx - 0.5, y2 = y0 + (n - 1.0) * ny - 0.5;
        int64_t x2i = c_int(x2), y2i = c_int(y2);
        if (x2i < 0 || x2i + 1 >= v.w || y2i < 0 || y2i + 1 >= v.h) continue;
        double g1 = bil_seq(x1 - (double)x1i, y1 - (double)y1i, v.im + y1i * v.s + x1i, v.s);
        double g2 = bil_seq(x2 - (double)x2i, y2 - (double)y2i, v.im + y2i * v.s + x2i, v.s);
        if (g1 < g2) continue;
        double wgt = (g2 - g1) * (g2 - g1);
        mn = mn + wgt * n;
        mc = mc + wgt;
    }
    if (mc == 0.0) return false;
    *n0 = mn / mc;
    return true;
}

// Lane u's share of one sample's first vsteps steps (a multiple of 4): the
// steps k = u, u + 4, ..., summed in that order into (ln, lc), which is
// partial sum u of refine_sample, so four lanes give its four sums.
__device__ __forceinline__ void refine_part(const DView &v, double x0, double y0, double nx, double ny, int64_t range,
                                            int64_t vsteps, int u, double *ln, double *lc) {
    const double wl = (double)(v.w - 1), hl = (double)(v.h - 1);
    const bool tiny = v.w < 2 || v.h < 2;
    double sn = 0.0, sc = 0.0;
#pragma unroll 3
    for (int64_t k = u; k < vsteps; k += 4) {
        const double n = (double)-range + 0.25 * (double)k;
        const double x1 = x0 + (n + 1.0) * nx - 0.5, y1 = y0 + (n + 1.0) * ny - 0.5;
        const double x2 = x0 + (n - 1.0) * nx - 0.5, y2 = y0 + (n - 1.0) * ny - 0.5;
        const bool in = x1 > -1.0 && x1 < wl && y1 > -1.0 && y1 < hl && x2 > -1.0 && x2 < wl && y2 > -1.0 && y2 < hl;
        const double tx1 = trunc(x1), ty1 = trunc(y1), tx2 = trunc(x2), ty2 = trunc(y2);
        double wgt = 0.0;
        if (in || !tiny) {
            const uint8_t *p1 = v.im + (in ? (int64_t)ty1 * v.s + (int64_t)tx1 : 0);
            const uint8_t *p2 = v.im + (in ? (int64_t)ty2 * v.s + (int64_t)tx2 : 0);
            const int a0 = p1[0], a1 = p1[1], a2 = p1[v.s], a3 = p1[v.s + 1];
            const int b0 = p2[0], b1 = p2[1], b2 = p2[v.s], b3 = p2[v.s + 1];
            if (in) {
                const double g1 = bil_vals(x1 - tx1, y1 - ty1, a0, a1, a2, a3);
                const double g2 = bil_vals(x2 - tx2, y2 - ty2, b0, b1, b2, b3);
                const double d = g2 - g1;
                wgt = !(g1 < g2) ? d * d : 0.0;
            }
        }
        sn = sn + wgt * n;
        sc = sc + wgt;
    }
    *ln = sn;
    *lc = sc;
}

// The steps after the first vsteps of one sample, in order, added to the
// sums (mn, mc) (the tail of refine_sample).
__device__ __forceinline__ void refine_tail(const DView &v, double x0, double y0, double nx, double ny, int64_t range,
                                            int64_t vsteps, int64_t nsteps, double *mn, double *mc) {
    for (int64_t k = vsteps; k < nsteps; k++) {
        double n = (double)-range + 0.25 * (double)k;
        double x1 = x0 + (n + 1.0) * nx - 0.5, y1 = y0 + (n + 1.0) * ny - 0.5;
        int64_t x1i = c_int(x1), y1i = c_int(y1);
        if (x1i < 0 || x1i + 1 >= v.w || y1i < 0 || y1i + 1 >= v.h) continue;
        double x2 = x0 + (n - 1.0) * nx - 0.5, y2 = y0 + (n - 1.0) * ny - 0.5;
        int64_t x2i = c_int(x2), y2i = c_int(y2);
        if (x2i < 0 || x2i + 1 >= v.w || y2i < 0 || y2i + 1 >= v.h) continue;
        double g1 = bil_seq(x1 - (double)x1i, y1 - (double)y1i, v.im + y1i * v.s + x1i, v.s);
        double g2 = bil_seq(x2 - (double)x2i, y2 - (double)y2i, v.im + y2i * v.s + x2i, v.s);
        if (g1 < g2) continue;
        double wgt = (g2 - g1) * (g2 - g1);
        *mn = *mn + wgt * n;
        *mc = *mc + wgt;
    }
}

// Correctly rounded f32 trig as the golden vectors need: the double
// function, then one rounding (fast/decode.c:740-744).
__device__ __forceinline__ float cr_atan2f(float y, float x) { return (float)atan2((double)y, (double)x); }
__device__ __forceinline__ float cr_cosf(float x) { return (float)cos((double)x); }
__device__ __forceinline__ float cr_sinf(float x) { return (float)sin((double)x); }

// Homography of 4 correspondences by one warp: the 8x9 Gaussian elimination
// with partial pivoting of fast/decode.c:114-165. Lane l holds row l / 4,
// columns l % 4 and l % 4 + 4 (and column 8 when l % 4 == 0). Each cell
// takes the same operations as in the sequential elimination, so the result
// is the same; the pivot is the first largest |a[r][col]|, r >= col, as the
// scan for a strictly larger value finds it. The back substitution runs on
// lane 0 from shared memory (m: 72 doubles). Returns false on a failed pivot
// check, on every lane. The loops stay rolled: this runs once per quad, so
// its code size is its cost.
__device__ __noinline__ bool homography_warp(const float (*p)[2], double *m, double H[9], int lane) {
    const unsigned FULL = 0xffffffffu;
    const int r = lane >> 2, g = lane & 3;
    double cell[3];
    {
        const int i = r >> 1;
        const double x = i == 0 || i == 3 ? -1.0 : 1.0, y = i == 0 || i == 1 ? -1.0 : 1.0;
        const double X = (double)p[i][0], Y = (double)p[i][1];
#pragma unroll
        for (int sl = 0; sl < 3; sl++) {
            const int col = sl == 2 ? 8 : g + 4 * sl;
            double v = 0.0;
            if ((r & 1) == 0) {
                v = col == 0 ? x : col == 1 ? y : col == 2 ? 1.0 : col == 6 ? -x * X : col == 7 ? -y * X : col == 8 ? X : 0.0;
            } else {
                v = col == 3 ? x : col == 4 ? y : col == 5 ? 1.0 : col == 6 ? -x * Y : col == 7 ? -y * Y : col == 8 ? Y : 0.0;
            }
            cell[sl] = v;
        }
    }
    bool ok = true;
#pragma unroll 1
    for (int col = 0; col < 8; col++) {
        const int cg = col & 3, cs = col >> 2;
        // pivot: the largest |a[r][col]| over r >= col, first r on ties
        double v = -1.0;
        if (g == cg && r >= col) {
            const double a = fabs(cs ? cell[1] : cell[0]);
            if (a == a) v = a;
        }
        int pr = r;
        for (int o = 16; o > 0; o >>= 1) {
            const double v2 = __shfl_xor_sync(FULL, v, o);
            const int r2 = __shfl_xor_sync(FULL, pr, o);
            if (v2 > v || (v2 == v && r2 < pr)) {
                v = v2;
                pr = r2;
            }
        }
        if (!(v > 0.0) || v < 1e-10) ok = false;
        const int piv = v > 0.0 ? pr : col;
        // swap rows col and piv (their columns left of col are zero in both)
        const int src = r == col ? 4 * piv + g : r == piv ? 4 * col + g : lane;
#pragma unroll
        for (int sl = 0; sl < 3; sl++) cell[sl] = __shfl_sync(FULL, cell[sl], src);
        // eliminate below the pivot
        const double pv = __shfl_sync(FULL, cs ? cell[1] : cell[0], 4 * col + cg);
        const double mine = cs ? cell[1] : cell[0];
        const double fct = __shfl_sync(FULL, mine / pv, 4 * r + cg);
        double prow[3];
#pragma unroll
        for (int sl = 0; sl < 3; sl++) prow[sl] = __shfl_sync(FULL, cell[sl], 4 * col + g);
        if (r > col) {
#pragma unroll
            for (int sl = 0; sl < 3; sl++) {
                const int cc = sl == 2 ? 8 : g + 4 * sl;
                if (sl == 2 && g != 0) continue;
                if (cc == col)
                    cell[sl] = 0.0;
                else if (cc > col)
                    cell[sl] = cell[sl] - fct * prow[sl];
            }
        }
    }
    m[r * 9 + g] = cell[0];
    m[r * 9 + g + 4] = cell[1];
    if (g == 0) m[r * 9 + 8] = cell[2];
    __syncwarp();
    if (ok && lane == 0) {
#pragma unroll 1
        for (int col = 7; col >= 0; col--) {
            double s = 0.0;
#pragma unroll 1
            for (int i = col + 1; i < 8; i++) s = s + m[col * 9 + i] * m[i * 9 + 8];
            m[col * 9 + 8] = (m[col * 9 + 8] - s) / m[col * 9 + col];
        }
    }
    __syncwarp();
#pragma unroll
    for (int i = 0; i < 8; i++) H[i] = m[i * 9 + 8];
    H[8] = 1.0;
    return ok;
}

// Invertibility as the C library's PLU decomposition decides it
// (fast/decode.c:168-196).
__device__ bool invertible3(const double m[9]) {
    double lu[9];
    for (int i = 0; i < 9; i++) lu[i] = m[i];
    for (int j = 0; j < 3; j++) {
        for (int i = 0; i < 3; i++) {
            int kmax = i < j ? i : j;
            double acc = 0.0;
            for (int k = 0; k < kmax; k++) acc = acc + lu[i * 3 + k] * lu[k * 3 + j];
            lu[i * 3 + j] = lu[i * 3 + j] - acc;
        }
        int p = j;
        for (int i = j + 1; i < 3; i++)
            if (fabs(lu[i * 3 + j]) > fabs(lu[p * 3 + j])) p = i;
        if (p != j)
            for (int k = 0; k < 3; k++) {
                double t = lu[p * 3 + k];
                lu[p * 3 + k] = lu[j * 3 + k];
                lu[j * 3 + k] = t;
            }
        double d = lu[j * 3 + j];
        if (fabs(d) < 1e-8) return false;
        if (d != 0.0) {
            double inv = 1.0 / d;
            for (int i = j + 1; i < 3; i++) lu[i * 3 + j] = lu[i * 3 + j] * inv;
        }
    }
    return true;
}

__device__ __forceinline__ void project(const double H[9], double x, double y, double *ox, double *oy) {
    double xx = H[0] * x + H[1] * y + H[2];
    double yy = H[3] * x + H[4] * y + H[5];
    double zz = H[6] * x + H[7] * y + H[8];
    *ox = xx / zz;
    *oy = yy / zz;
}

struct GrayModel {
    double a[9], b[3], c[3];
};

// mat33_sym_solve as the C library does it (fast/decode.c:241-265).
__device__ __forceinline__ void gm_solve(GrayModel *g) {
    const double *a = g->a;
    double L0 = sqrt(a[0]);
    double L3 = a[1] / L0;
    double L6 = a[2] / L0;
    double L4 = sqrt(a[4] - L3 * L3);
    double L7 = (a[5] - L3 * L6) / L4;
    double L8 = sqrt(a[8] - L6 * L6 - L7 * L7);
    double M0 = 1.0 / L0;
    double M3 = -L3 * M0 / L4;
    double M4 = 1.0 / L4;
    double M6 = (-L6 * M0 - L7 * M3) / L8;
    double M7 = -L7 * M4 / L8;
    double M8 = 1.0 / L8;
    const double *b = g->b;
    double t0 = M0 * b[0];
    double t1 = M3 * b[0] + M4 * b[1];
    double t2 = M6 * b[0] + M7 * b[1] + M8 * b[2];
    g->c[0] = M0 * t0 + M3 * t1 + M6 * t2;
    g->c[1] = M4 * t1 + M7 * t2;
    g->c[2] = M8 * t2;
}

__device__ __forceinline__ double bilinear_at(const DView &v, double px, double py) {
    int64_t x1 = c_int(floor(px - 0.5)), x2 = c_int(ceil(px - 0.5));
    double x = px - 0.5 - (double)x1;
    int64_t y1 = c_int(floor(py - 0.5)), y2 = c_int(ceil(py - 0.5));
    double y = py - 0.5 - (double)y1;
    if (x1 < 0 || x2 >= v.w || y1 < 0 || y2 >= v.h) return -1.0;
    const uint8_t *r1 = v.im + y1 * v.s, *r2 = v.im + y2 * v.s;
    return r1[x1] * (1.0 - x) * (1.0 - y) + r1[x2] * x * (1.0 - y) + r2[x1] * (1.0 - x) * y + r2[x2] * x * y;
}

__device__ __forceinline__ uint64_t rot90(uint64_t w0, int64_t nbits) {
    int64_t p = nbits, l = 0;
    if (nbits % 4 == 1) {
        p = nbits - 1;
        l = 1;
    }
    uint64_t w = ((w0 >> l) << (p / 4 + l)) | (w0 >> (3 * p / 4 + l) << l) | (w0 & (uint64_t)l);
    return w & ((nbits >= 64) ? ~0ull : (((uint64_t)1 << nbits) - 1));
}

// The first code within maxham bits, by rotation, then chunk, then code
// index (fast/decode.c:87-107). Returns id | hamming << 16 | rot << 24.
__device__ uint32_t qd_lookup(const GpuFamily &F, uint64_t rcode, int lane) {
    // lane 4 r + j (r rotations, chunk j) scans its bucket; the first lane
    // with a match holds the first match in the sequential order
    const uint64_t mask = (uint64_t)F.cap - 1;
    uint32_t res = 0xffffffffu;
    if (lane < 16) {
        const int r = lane >> 2, j = lane & 3;
        uint64_t rc = rcode;
        for (int t = 0; t < r; t++) rc = rot90(rc, F.nbits);
        const int64_t val = (int64_t)((rc >> (j * F.chunk)) & mask);
        const int64_t ob = j * (F.cap + 1) + val, base = j * F.ncodes;
        for (int64_t e = base + F.off[ob]; e < base + F.off[ob + 1]; e++) {
            const int hd = __popcll(F.codes[e] ^ rc);
            if (hd <= F.maxham) {
                res = (uint32_t)F.idx[e] | (uint32_t)hd << 16 | (uint32_t)r << 24;
                break;
            }
        }
    }
    const uint32_t found = __ballot_sync(0xffffffffu, res != 0xffffffffu);
    if (!found) return 65535u | 255u << 16;
    return __shfl_sync(0xffffffffu, res, __ffs(found) - 1);
}

#define REF_CHUNK 128

__global__ void __launch_bounds__(AT_DEC_THREADS) k_refine(const FrameDesc *frames, GpuParams prm,
                                                              const uint8_t *img, const uint8_t *qim,
                                                              const GpuQuad *quads, const uint32_t *nq, float *corners,
                                                              uint32_t *det_ok) {
    const int64_t nquads = *nq;
    __shared__ float s_p[4][2];
    __shared__ double s_lines[4][4];
    __shared__ double s_bx[REF_CHUNK], s_by[REF_CHUNK];
    __shared__ int s_bok[REF_CHUNK];
    __shared__ double s_enx[4], s_eny[4];
    __shared__ int64_t s_ens[4];
    const int tid = threadIdx.x;
    for (int64_t qi = blockIdx.x; qi < nquads; qi += gridDim.x) {
        const GpuQuad q = quads[qi];
        DEC_PROF(0)
        const FrameDesc f = frames[q.frame];
        DView v;
        if (prm.decode_blurred)
            v = DView{qim + f.q_off, (int64_t)f.qw, (int64_t)f.qw, (int64_t)f.qh};
        else
            v = DView{f.img, f.stride, (int64_t)f.w, (int64_t)f.h};
        if (tid < 8) {
            float val = q.p[tid >> 1][tid & 1];
            if (prm.quad_decimate > 1.0f) val = __fmul_rn(val, prm.quad_decimate);
            s_p[tid >> 1][tid & 1] = val;
        }
        for (int fi = tid; fi < prm.nfam; fi += blockDim.x) det_ok[qi * prm.nfam + fi] = 0;
        __syncthreads();
        if (prm.refine_edges) {
            // fast/decode.c:657-761. The 4 edges are independent until the
            // corners are moved: their sample points, one per thread, are
            // refined together, and thread e < 4 sums edge e's in order.
            const int64_t range = (int64_t)__fadd_rn(prm.quad_decimate, 1.0f);
            const int64_t nsteps = 2 * 4 * range + 1;
            const int64_t vsteps = nsteps - nsteps % 4;
            if (tid < 4) {
                int a = tid, b = (tid + 1) & 3;
                double nx = (double)__fsub_rn(s_p[b][1], s_p[a][1]);
                double ny = (double)__fadd_rn(-s_p[b][0], s_p[a][0]);
                double mag = sqrt(nx * nx + ny * ny);
                nx = nx / mag;
                ny = ny / mag;
                if (q.reversed_border) {
                    nx = -nx;
                    ny = -ny;
                }
                s_enx[tid] = nx;
                s_eny[tid] = ny;
                s_ens[tid] = dmax(16, c_int(mag / 8.0));
            }
            __syncthreads();
            // the 4 edges' samples in one packed range, edge after edge
            const int64_t o1 = s_ens[0], o2 = o1 + s_ens[1], o3 = o2 + s_ens[2], total = o3 + s_ens[3];
            double mx = 0.0, my = 0.0, mxx = 0.0, mxy = 0.0, myy = 0.0, cnt = 0.0;
            for (int64_t c0 = 0; c0 < total; c0 += REF_CHUNK) {
                // four lanes per sample, lane u summing partial sum u
                const int u = tid & 3;
                for (int w0 = 0; w0 < REF_CHUNK; w0 += (int)(blockDim.x >> 2)) {
                    const int w = w0 + (tid >> 2);
                    const int64_t gi = c0 + w;
                    const bool valid = w < REF_CHUNK && gi < total;
                    double ln = 0.0, lc = 0.0, x0 = 0.0, y0 = 0.0, nx = 0.0, ny = 0.0;
                    if (valid) {
                        const int e = gi < o1 ? 0 : gi < o2 ? 1 : gi < o3 ? 2 : 3;
                        const int64_t si = gi - (e == 0 ? 0 : e == 1 ? o1 : e == 2 ? o2 : o3), ns = s_ens[e];
                        const int a = e, b = (e + 1) & 3;
                        nx = s_enx[e];
                        ny = s_eny[e];
                        double alpha = (1.0 + (double)si) / (double)(ns + 1);
                        x0 = alpha * (double)s_p[a][0] + (1.0 - alpha) * (double)s_p[b][0];
                        y0 = alpha * (double)s_p[a][1] + (1.0 - alpha) * (double)s_p[b][1];
                        refine_part(v, x0, y0, nx, ny, range, vsteps, u, &ln, &lc);
                    }
                    const double ln0 = __shfl_sync(0xffffffffu, ln, 0, 4), ln1 = __shfl_sync(0xffffffffu, ln, 1, 4),
                                 ln2 = __shfl_sync(0xffffffffu, ln, 2, 4), ln3 = __shfl_sync(0xffffffffu, ln, 3, 4);
                    const double lc0 = __shfl_sync(0xffffffffu, lc, 0, 4), lc1 = __shfl_sync(0xffffffffu, lc, 1, 4),
                                 lc2 = __shfl_sync(0xffffffffu, lc, 2, 4), lc3 = __shfl_sync(0xffffffffu, lc, 3, 4);
                    if (valid && u == 0) {
                        double mn = 0.0 + ((ln0 + ln2) + (ln1 + ln3));
                        double mc = 0.0 + ((lc0 + lc2) + (lc1 + lc3));
                        refine_tail(v, x0, y0, nx, ny, range, vsteps, nsteps, &mn, &mc);
                        const bool ok = mc != 0.0;
                        s_bok[w] = ok;
                        if (ok) {
                            const double n0 = mn / mc;
                            s_bx[w] = x0 + n0 * nx;
                            s_by[w] = y0 + n0 * ny;
                        }
                    }
                }
                __syncthreads();
                if (tid < 4) {
                    const int64_t eo = tid == 0 ? 0 : tid == 1 ? o1 : tid == 2 ? o2 : o3, ee = eo + s_ens[tid];
                    const int64_t lo = dmax(eo, c0), hi = dmin(ee, c0 + REF_CHUNK);
                    for (int64_t gi = lo; gi < hi; gi++) {
                        const int64_t t = gi - c0;
                        if (!s_bok[t]) continue;
                        double bx = s_bx[t], by = s_by[t];
                        mx = mx + bx;
                        my = my + by;
                        mxx = mxx + bx * bx;
                        mxy = mxy + bx * by;
                        myy = myy + by * by;
                        cnt = cnt + 1.0;
                    }
                }
                __syncthreads();
            }
            DEC_PROF(1)
            if (tid < 4) {
                double ex = mx / cnt, ey = my / cnt;
                double cxx = mxx / cnt - ex * ex, cxy = mxy / cnt - ex * ey, cyy = myy / cnt - ey * ey;
                double theta = 0.5 * (double)cr_atan2f((float)(-2.0 * cxy), (float)(cyy - cxx));
                s_lines[tid][0] = ex;
                s_lines[tid][1] = ey;
                s_lines[tid][2] = (double)cr_cosf((float)theta);
                s_lines[tid][3] = (double)cr_sinf((float)theta);
            }
            __syncthreads();
            if (tid == 0) {
                for (int i = 0; i < 4; i++) {
                    int j = (i + 1) & 3;
                    double a00 = s_lines[i][3], a01 = -s_lines[j][3], a10 = -s_lines[i][2], a11 = s_lines[j][2];
                    double b0 = -s_lines[i][0] + s_lines[j][0], b1 = -s_lines[i][1] + s_lines[j][1];
                    double det = a00 * a11 - a10 * a01;
                    if (fabs(det) > 0.001) {
                        double w00 = a11 / det, w01 = -a01 / det;
                        double l0 = w00 * b0 + w01 * b1;
                        s_p[j][0] = (float)(s_lines[i][0] + l0 * a00);
                        s_p[j][1] = (float)(s_lines[i][1] + l0 * a10);
                    }
                }
            }
            __syncthreads();
            DEC_PROF(2)
        }
        if (tid < 8) corners[qi * 8 + tid] = s_p[tid >> 1][tid & 1];
        __syncthreads();
    }
}

// The homography of each quad's corners (fast/decode.c:114-196), a warp
// per quad: H, and whether it was found and is invertible.
#define QH_WARPS 4
__global__ void __launch_bounds__(QH_WARPS * 32) k_quad_homography(const float *corners, const uint32_t *nq, double *hs,
                                                                     uint32_t *hok) {
    const int64_t nquads = *nq;
    __shared__ float s_p[QH_WARPS][4][2];
    __shared__ double s_hm[QH_WARPS][72];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int64_t qi = (int64_t)blockIdx.x * QH_WARPS + w; qi < nquads; qi += (int64_t)gridDim.x * QH_WARPS) {
        if (lane < 8) s_p[w][lane >> 1][lane & 1] = corners[qi * 8 + lane];
        __syncwarp();
        double H[9];
        const bool ok = homography_warp(s_p[w], s_hm[w], H, lane);
        if (lane == 0) {
            hok[qi] = ok && invertible3(H);
#pragma unroll
            for (int i = 0; i < 9; i++) hs[qi * 9 + i] = H[i];
        }
        __syncwarp();
    }
}

__global__ void __launch_bounds__(AT_DEC_THREADS) k_decode(const FrameDesc *frames, GpuParams prm,
                                                              const GpuFamily *fams, const uint8_t *img,
                                                              const uint8_t *qim, const GpuQuad *quads,
                                                              const uint32_t *nq, const double *hs, const uint32_t *hok,
                                                              GpuDetection *dets, uint32_t *det_ok) {
    const int64_t nquads = *nq;
    __shared__ double s_H[9];
    __shared__ double s_gx[8 * AT_MAX_TW], s_gy[8 * AT_MAX_TW], s_gv[8 * AT_MAX_TW];
    __shared__ int s_gk[8 * AT_MAX_TW];
    __shared__ double s_wc[3], s_bc[3];
    __shared__ int s_pol;
    __shared__ double s_vals[AT_MAX_TW * AT_MAX_TW], s_sharp[AT_MAX_TW * AT_MAX_TW];
    const int tid = threadIdx.x;
    for (int64_t qi = blockIdx.x; qi < nquads; qi += gridDim.x) {
        if (!hok[qi]) continue;
        const GpuQuad q = quads[qi];
        const FrameDesc f = frames[q.frame];
        DView v;
        if (prm.decode_blurred)
            v = DView{qim + f.q_off, (int64_t)f.qw, (int64_t)f.qw, (int64_t)f.qh};
        else
            v = DView{f.img, f.stride, (int64_t)f.w, (int64_t)f.h};
        __syncthreads();
        if (tid < 9) s_H[tid] = hs[qi * 9 + tid];
        __syncthreads();
        DEC_PROF(3)
        for (int fi = 0; fi < prm.nfam; fi++) {
            const GpuFamily &F = fams[fi];
            if (F.reversed_border != q.reversed_border) continue;
            if (!(f.fam_mask >> fi & 1u)) continue;
            // border gray models (fast/decode.c:291-337): 8 patterns x wab
            const int32_t wab = F.wab;
            const float wf = (float)wab;
            for (int t = tid; t < 8 * wab; t += blockDim.x) {
                int pi = t / wab, i = t - pi * wab;
                float pat[5];
                switch (pi) {
                case 0: pat[0] = -0.5f, pat[1] = 0.5f, pat[2] = 0.0f, pat[3] = 1.0f; break;
                case 1: pat[0] = 0.5f, pat[1] = 0.5f, pat[2] = 0.0f, pat[3] = 1.0f; break;
                case 2: pat[0] = (float)(wab + 0.5), pat[1] = 0.5f, pat[2] = 0.0f, pat[3] = 1.0f; break;
                case 3: pat[0] = (float)(wab - 0.5), pat[1] = 0.5f, pat[2] = 0.0f, pat[3] = 1.0f; break;
                case 4: pat[0] = 0.5f, pat[1] = -0.5f, pat[2] = 1.0f, pat[3] = 0.0f; break;
                case 5: pat[0] = 0.5f, pat[1] = 0.5f, pat[2] = 1.0f, pat[3] = 0.0f; break;
                case 6: pat[0] = 0.5f, pat[1] = (float)(wab + 0.5), pat[2] = 1.0f, pat[3] = 0.0f; break;
                default: pat[0] = 0.5f, pat[1] = (float)(wab - 0.5), pat[2] = 1.0f, pat[3] = 0.0f; break;
                }
                double tx01 = (double)__fdiv_rn(__fadd_rn(pat[0], __fmul_rn((float)i, pat[2])), wf);
                double ty01 = (double)__fdiv_rn(__fadd_rn(pat[1], __fmul_rn((float)i, pat[3])), wf);
                double tx = 2.0 * (tx01 - 0.5), ty = 2.0 * (ty01 - 0.5);
                double zz = s_H[6] * tx + s_H[7] * ty + s_H[8];
                double px = (s_H[0] * tx + s_H[1] * ty + s_H[2]) / zz;
                double py = (s_H[3] * tx + s_H[4] * ty + s_H[5]) / zz;
                int64_t ix = c_int(px), iy = c_int(py);
                int keep = !(ix < 0 || iy < 0 || ix >= v.w || iy >= v.h);
                s_gk[t] = keep;
                s_gx[t] = tx;
                s_gy[t] = ty;
                s_gv[t] = keep ? (double)v.im[iy * v.s + ix] : 0.0;
            }
            __syncthreads();
            if (tid < 32) {
                // lane 0 the white model (even patterns), lane 1 the black one
                // (odd patterns), each summed in pattern order in registers
                double a0 = 0.0, a1 = 0.0, a2 = 0.0, a4 = 0.0, a5 = 0.0, a8 = 0.0, b0 = 0.0, b1 = 0.0, b2 = 0.0;
                if (tid < 2) {
                    for (int pi = tid; pi < 8; pi += 2)
                        for (int i = 0; i < wab; i++) {
                            const int t = pi * wab + i;
                            if (!s_gk[t]) continue;
                            const double x = s_gx[t], y = s_gy[t], val = s_gv[t];
                            a0 = a0 + x * x;
                            a1 = a1 + x * y;
                            a2 = a2 + x;
                            a4 = a4 + y * y;
                            a5 = a5 + y;
                            a8 = a8 + 1.0;
                            b0 = b0 + x * val;
                            b1 = b1 + y * val;
                            b2 = b2 + val;
                        }
                }
                GrayModel gm;
                gm.a[0] = a0, gm.a[1] = a1, gm.a[2] = a2, gm.a[4] = a4, gm.a[5] = a5, gm.a[8] = a8;
                gm.a[3] = gm.a[6] = gm.a[7] = 0.0;
                gm.b[0] = b0, gm.b[1] = b1, gm.b[2] = b2;
                if (tid == 0 || (tid == 1 && wab > 1)) {
                    gm_solve(&gm);
                } else {
                    gm.c[0] = 0.0;
                    gm.c[1] = 0.0;
                    gm.c[2] = gm.b[2] / 4.0;
                }
                const double ci = gm.c[0] * 0.0 + gm.c[1] * 0.0 + gm.c[2];
                const double bi = __shfl_sync(0xffffffffu, ci, 1);
                if (tid == 0) s_pol = (ci - bi < 0.0) == (F.reversed_border != 0);
                if (tid < 2)
                    for (int i = 0; i < 3; i++) (tid == 0 ? s_wc : s_bc)[i] = gm.c[i];
            }
            __syncthreads();
            if (!s_pol) continue;
            DEC_PROF(4)
            // bit values less the local threshold, sharpened (decode.c:340-377)
            const int64_t tw = F.tw;
            const int64_t minc = (wab - tw) / 2;
            for (int64_t t = tid; t < tw * tw; t += blockDim.x) s_vals[t] = 0.0;
            __syncthreads();
            for (int64_t i = tid; i < F.nbits; i += blockDim.x) {
                int64_t bx = F.bit_x[i], by = F.bit_y[i];
                double tx = 2.0 * (((double)bx + 0.5) / wab - 0.5), ty = 2.0 * (((double)by + 0.5) / wab - 0.5);
                double zz = s_H[6] * tx + s_H[7] * ty + s_H[8];
                double px = (s_H[0] * tx + s_H[1] * ty + s_H[2]) / zz;
                double py = (s_H[3] * tx + s_H[4] * ty + s_H[5]) / zz;
                double val = bilinear_at(v, px, py);
                if (val == -1.0) continue;
                double thr = ((s_bc[0] * tx + s_bc[1] * ty + s_bc[2]) + (s_wc[0] * tx + s_wc[1] * ty + s_wc[2])) / 2.0;
                s_vals[tw * (by - minc) + (bx - minc)] = val - thr;
            }
            __syncthreads();
            for (int64_t t = tid; t < tw * tw; t += blockDim.x) {
                int64_t y = t / tw, x = t - y * tw;
                double acc = 0.0;
                if (y > 0) acc = acc + -s_vals[(y - 1) * tw + x];
                if (x > 0) acc = acc + -s_vals[y * tw + x - 1];
                acc = acc + s_vals[y * tw + x] * 4.0;
                if (x + 1 < tw) acc = acc + -s_vals[y * tw + x + 1];
                if (y + 1 < tw) acc = acc + -s_vals[(y + 1) * tw + x];
                s_sharp[t] = acc;
            }
            __syncthreads();
            DEC_PROF(5)
            if (tid < 32) {
                float bs = 0.0f, ws = 0.0f, bc = 1.0f, wc = 1.0f;
                uint64_t rcode = 0;
                if (tid == 0) {
                for (int64_t i = 0; i < F.nbits; i++) {
                    rcode <<= 1;
                    int64_t cell = (F.bit_y[i] - minc) * tw + (F.bit_x[i] - minc);
                    double vv = s_vals[cell] + prm.decode_sharpening * s_sharp[cell];
                    if (vv > 0.0) {
                        ws = (float)((double)ws + vv);
                        wc = __fadd_rn(wc, 1.0f);
                        rcode |= 1;
                    } else {
                        bs = (float)((double)bs - vv);
                        bc = __fadd_rn(bc, 1.0f);
                    }
                }
                }
                rcode = (uint64_t)__shfl_sync(0xffffffffu, (uint32_t)(rcode >> 32), 0) << 32 |
                        __shfl_sync(0xffffffffu, (uint32_t)rcode, 0);
                const uint32_t lk = qd_lookup(F, rcode, tid);
                double x = (double)__fdiv_rn(ws, wc), y = (double)__fdiv_rn(bs, bc);
                double m = x != x ? y : y != y ? x : x < y ? x : y;  // fmin
                float margin = (float)m;
                int64_t id = lk & 0xffff, ham = (lk >> 16) & 0xff, rot = lk >> 24;
                if (tid == 0 && margin >= 0.0f && ham < 255) {
                    // H = qH * R(rot * pi/2) (fast/detector.c:83-107)
                    double c = prm.rot_cs[rot][0], s = prm.rot_cs[rot][1];
                    const double r[9] = {c, -s, 0.0, s, c, 0.0, 0.0, 0.0, 1.0};
                    GpuDetection d;
                    for (int i = 0; i < 3; i++)
                        for (int j = 0; j < 3; j++) {
                            double acc = 0.0;
                            for (int k = 0; k < 3; k++) acc = acc + s_H[i * 3 + k] * r[k * 3 + j];
                            d.H[i * 3 + j] = acc;
                        }
                    d.family = fi;
                    d.id = (int32_t)id;
                    d.hamming = (int32_t)ham;
                    d.decision_margin = margin;
                    project(d.H, 0.0, 0.0, &d.c[0], &d.c[1]);
                    for (int i = 0; i < 4; i++) {
                        double tx = i == 1 || i == 2 ? 1.0 : -1.0;
                        double ty = i < 2 ? 1.0 : -1.0;
                        project(d.H, tx, ty, &d.p[i][0], &d.p[i][1]);
                    }
                    dets[qi * prm.nfam + fi] = d;
                    det_ok[qi * prm.nfam + fi] = 1;
                }
            }
            __syncthreads();
            DEC_PROF(6)
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// 10. Per frame: gather the detections in (quad, family) order, remove
// overlapping detections of one tag (fast/decode.c:766-891), stable sort by
// id (fast/detector.c:164-179). One thread per frame.

struct GLine {
    double p[2], u[2];
};

__device__ GLine gline_of(const double *p0, const double *p1) {
    double u0 = p1[0] - p0[0], u1 = p1[1] - p0[1];
    double mag = (double)__fsqrt_rn((float)(u0 * u0 + u1 * u1));
    GLine l;
    l.p[0] = p0[0];
    l.p[1] = p0[1];
    l.u[0] = u0 / mag;
    l.u[1] = u1 / mag;
    return l;
}
__device__ __forceinline__ double gline_coord(const GLine &l, const double *q) {
    return (q[0] - l.p[0]) * l.u[0] + (q[1] - l.p[1]) * l.u[1];
}
__device__ bool segments_cross(const double *a0, const double *a1, const double *b0, const double *b1) {
    GLine la = gline_of(a0, a1), lb = gline_of(b0, b1);
    double m00 = la.u[0], m01 = -lb.u[0], m10 = la.u[1], m11 = -lb.u[1];
    double det = m00 * m11 - m01 * m10;
    if (fabs(det) < 0.00000001) return false;
    double i00 = m11 / det, i01 = -m01 / det;
    double b00 = lb.p[0] - la.p[0], b10 = lb.p[1] - la.p[1];
    double x00 = i00 * b00 + i01 * b10;
    double t[2] = {la.u[0] * x00 + la.p[0], la.u[1] * x00 + la.p[1]};
    double a = gline_coord(la, la.p), b = gline_coord(la, a1), c = gline_coord(la, t);
    if ((c < a && c < b) || (c > a && c > b)) return false;
    a = gline_coord(lb, lb.p);
    b = gline_coord(lb, b1);
    c = gline_coord(lb, t);
    if ((c < a && c < b) || (c > a && c > b)) return false;
    return true;
}
__device__ bool poly_contains(const double (*poly)[2], const double *q) {
    int last = 0, acc = 0;
    for (int i = 0; i < 5; i++) {
        const double *p = poly[i % 4];
        int quad = p[0] < q[0] ? (p[1] < q[1] ? 2 : 1) : (p[1] < q[1] ? 3 : 0);
        if (i > 0) {
            int dq = quad - last;
            if (dq == -3 || dq == 1)
                acc++;
            else if (dq == -1 || dq == 3)
                acc--;
            else if (dq == -2 || dq == 2) {
                const double *p0 = poly[i - 1];
                double nx = p[1] - q[1], ny = -p[0] + q[0];
                double dot = nx * (p0[0] - q[0]) + ny * (p0[1] - q[1]);
                acc += dot < 0.0 ? -2 : 2;
            }
        }
        last = quad;
    }
    return acc >= 2 || acc <= -2;
}
__device__ bool quads_overlap(const double (*pa)[2], const double (*pb)[2]) {
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++)
            if (segments_cross(pa[i], pa[(i + 1) % 4], pb[j], pb[(j + 1) % 4])) return true;
    double qb[2] = {(pb[0][0] + pb[1][0] + pb[2][0]) / 3.0, (pb[0][1] + pb[1][1] + pb[2][1]) / 3.0};
    if (poly_contains(pa, qb)) return true;
    double qa[2] = {(pa[0][0] + pa[1][0] + pa[2][0]) / 3.0, (pa[0][1] + pa[1][1] + pa[2][1]) / 3.0};
    return poly_contains(pb, qa);
}
__device__ __forceinline__ int prefer(int pref, double a, double b) {
    return pref ? pref : a < b ? -1 : b < a ? 1 : 0;
}

// One block per frame. Overlap removal only ever drops a detection in favour
// of another with the same (family, id), and its outcome for one such
// group depends only on that group's detections in quad order; so the
// groups are resolved independently (one thread each, the rare groups of
// two or more), and the survivors are placed by their stable rank by id.
// The bucket count of the reference's cluster table for a quad image of
// w x h at one thread (fast/clusters.c:97-103, fast/detector.c:223).
__device__ __forceinline__ uint64_t ref_buckets(int64_t w, int64_t h) {
    const int64_t chunk = 1 + (h - 1) / 6;
    int64_t n = 1024;
    while (n < chunk * w / 64 && n < 65536) n <<= 1;
    return (uint64_t)n;
}

__global__ void k_finalize(int nframes, const int64_t *frame_qstart, int nfam, const GpuDetection *dets,
                           const uint32_t *det_ok, uint32_t *idx, uint8_t *removed, GpuDetection *out,
                           const int64_t *out_off, int64_t *out_n, const FrameDesc *frames, RefOrder ref,
                           const uint32_t *qcl, const uint64_t *ckey, int nb, uint64_t *okey, uint32_t *idx2,
                           uint32_t *err) {
    __shared__ uint32_t sh[32];
    const int f = blockIdx.x;
    if (f >= nframes) return;
    const int64_t a = frame_qstart[f] * nfam, b = frame_qstart[f + 1] * nfam;
    uint32_t *ix = idx + a;
    uint8_t *rm = removed + a;
    // the detections of the frame in (quad, family) order
    int64_t n = 0;
    for (int64_t s0 = a; s0 < b; s0 += blockDim.x) {
        int64_t s = s0 + threadIdx.x;
        uint32_t ok = s < b ? det_ok[s] : 0u;
        uint32_t total;
        uint32_t off = block_excl_scan(ok, &total, sh);
        if (ok) ix[n + off] = (uint32_t)s;
        n += total;
    }
    __syncthreads();
    if (ref.need[f]) {
        // detections that share an id take the reference's quad order:
        // (bucket, key) of their clusters' reference roots
        // (fast/clusters.c:44, 338-356), then family; the others keep
        // theirs (only detections of one id are ever compared)
        const FrameDesc fd = frames[f];
        const uint64_t nbuck = ref_buckets(fd.qw, fd.qh);
        const uint32_t nt = ref.nt[f];
        const uint32_t *tl = ref.tlabel + (int64_t)f * AT_REF_MAXT, *tr = ref.troot + (int64_t)f * AT_REF_MAXT;
        const uint64_t lmask = ((uint64_t)1 << nb) - 1;
        uint64_t *k0 = okey + 2 * a, *k1 = k0 + (b - a);
        for (int64_t p = threadIdx.x; p < n; p += blockDim.x) {
            const uint32_t s = ix[p];
            const uint64_t key = ckey[qcl[s / nfam]];
            const uint32_t lh = (uint32_t)(key >> nb), ll = (uint32_t)(key & lmask);
            uint32_t th = 0xffffffffu, tlo = 0xffffffffu;
            for (uint32_t t = 0; t < nt; t++) {
                if (tl[t] == lh) th = t;
                if (tl[t] == ll) tlo = t;
            }
            if (th != 0xffffffffu && tlo != 0xffffffffu) {
                const uint64_t rh = tr[th], rl = tr[tlo];
                if (rh == 0xffffffffu || rl == 0xffffffffu) atomicOr(err, AT_ERR_ORDER);
                const uint64_t hi = rh > rl ? rh : rl, lo = rh > rl ? rl : rh;
                const uint64_t cid = hi << 32 | lo;
                const uint64_t bucket = ((cid * 2654435761ull) >> 32) & (nbuck - 1);
                k0[p] = bucket << 32 | hi;
                k1[p] = lo << 8 | (uint64_t)(s % nfam);
            } else {
                k0[p] = ~0ull;
                k1[p] = (uint64_t)p;
            }
        }
        __syncthreads();
        for (int64_t p = threadIdx.x; p < n; p += blockDim.x) {
            int64_t r = 0;
            for (int64_t q = 0; q < n; q++) r += k0[q] < k0[p] || (k0[q] == k0[p] && k1[q] < k1[p]);
            idx2[a + r] = ix[p];
        }
        __syncthreads();
        for (int64_t p = threadIdx.x; p < n; p += blockDim.x) ix[p] = idx2[a + p];
        __syncthreads();
    }
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) rm[i] = 0;
    __syncthreads();
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const GpuDetection &di = dets[ix[i]];
        bool first = true, more = false;
        for (int64_t j = 0; j < n && first; j++)
            if (j != i && dets[ix[j]].id == di.id && dets[ix[j]].family == di.family) {
                if (j < i) first = false;
                else more = true;
            }
        if (!first || !more) continue;
        // the reference's loop (fast/decode.c:860-891) over this group only
        int64_t i0 = i;
        while (i0 < n) {
            if (rm[i0] || dets[ix[i0]].id != di.id || dets[ix[i0]].family != di.family) {
                i0++;
                continue;
            }
            for (int64_t i1 = i0 + 1; i1 < n; i1++) {
                const GpuDetection &d0 = dets[ix[i0]], &d1 = dets[ix[i1]];
                if (rm[i1] || d1.id != di.id || d1.family != di.family || !quads_overlap(d0.p, d1.p)) continue;
                int pref = prefer(0, d0.hamming, d1.hamming);
                pref = prefer(pref, -(double)d0.decision_margin, -(double)d1.decision_margin);
                for (int k = 0; k < 4; k++) {
                    pref = prefer(pref, d0.p[k][0], d1.p[k][0]);
                    pref = prefer(pref, d0.p[k][1], d1.p[k][1]);
                }
                if (pref < 0) {
                    rm[i1] = 1;
                    continue;
                }
                rm[i0] = 1;
                break;
            }
            i0++;
        }
    }
    __syncthreads();
    // stable sort by id (fast/detector.c:164-179): rank among survivors
    GpuDetection *o = out + out_off[f];
    uint32_t kept = 0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        if (rm[i]) continue;
        kept++;
        int32_t id = dets[ix[i]].id;
        int64_t r = 0;
        for (int64_t j = 0; j < n; j++)
            if (!rm[j] && (dets[ix[j]].id < id || (dets[ix[j]].id == id && j < i))) r++;
        o[r] = dets[ix[i]];
    }
    uint32_t total;
    block_excl_scan(kept, &total, sh);
    if (threadIdx.x == 0) out_n[f] = total;
}

// The quads in cluster order (so grouped by frame), and their count.
__global__ void k_gather_quads(const GpuQuad *quads, const uint32_t *ok, const uint32_t *scan, int64_t n,
                               GpuQuad *out, uint32_t *nq, uint32_t *qcl) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (ok[i]) {
            out[scan[i]] = quads[i];
            qcl[scan[i]] = (uint32_t)i;
        }
        if (i == n - 1) *nq = scan[i] + ok[i];
    }
}

// Per frame: its first quad and its first detection slot (nfam per quad).
__global__ void k_frame_bounds(const GpuQuad *quads, const uint32_t *nq, int nframes, int nfam, int64_t *qstart,
                               int64_t *out_off) {
    const int64_t n = *nq;
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f <= nframes; f += gridDim.x * blockDim.x) {
        int64_t lo = 0, hi = n;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (quads[mid].frame < f)
                lo = mid + 1;
            else
                hi = mid;
        }
        qstart[f] = lo;
        out_off[f] = lo * nfam;
    }
}

// Each frame's detections, packed frame after frame into host memory
// (mapped pinned). k_output_meta (one block): meta[3 f ..] = (first, count,
// quads) per frame, meta[3 n], meta[3 n + 1] = the totals of detections and
// quads, and the offsets again on the device (first, with the total last).
// k_output_copy: a warp per detection, its 21 words in one coalesced write.
__global__ void __launch_bounds__(256) k_output_meta(int nframes, const int64_t *qstart, const int64_t *out_n,
                                                     int64_t *first, int64_t *meta) {
    __shared__ uint32_t sh[32];
    int64_t base = 0;
    for (int f0 = 0; f0 < nframes; f0 += blockDim.x) {
        const int f = f0 + threadIdx.x;
        const uint32_t cnt = f < nframes ? (uint32_t)out_n[f] : 0u;
        uint32_t total;
        const uint32_t off = block_excl_scan(cnt, &total, sh);
        if (f < nframes) {
            first[f] = base + off;
            meta[3 * f] = base + off;
            meta[3 * f + 1] = cnt;
            meta[3 * f + 2] = qstart[f + 1] - qstart[f];
        }
        base += total;
    }
    if (threadIdx.x == 0) {
        first[nframes] = base;
        meta[3 * nframes] = base;
        meta[3 * nframes + 1] = qstart[nframes];
    }
}

__global__ void k_output_copy(int nframes, const GpuDetection *out, const int64_t *out_off, const int64_t *first,
                              GpuDetection *host) {
    constexpr int W = (int)(sizeof(GpuDetection) / 8);
    const int lane = threadIdx.x & 31;
    const int64_t total = first[nframes];
    for (int64_t j = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < total;
         j += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        int lo = 0, hi = nframes - 1;  // the frame holding detection j
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (first[mid] <= j)
                lo = mid;
            else
                hi = mid - 1;
        }
        const uint64_t *src = reinterpret_cast<const uint64_t *>(out + out_off[lo] + (j - first[lo]));
        uint64_t *dst = reinterpret_cast<uint64_t *>(host + j);
        if (lane < W) dst[lane] = src[lane];
    }
}

// ---------------------------------------------------------------------------
// Launchers.

static inline dim3 frame_grid(const Launch &L) { return dim3((unsigned)L.blocks_per_frame, (unsigned)L.nframes); }
// a warp per row when the batch has rows enough to fill the GPU with warps
// (16 per SM), else a block per row (lower latency for a few frames)
static inline bool warp_rows(const Launch &L) { return (int64_t)L.nframes * L.max_qh >= 148 * 16; }
// a warp per row, 8 rows a block
static inline dim3 row_warp_grid(const Launch &L) {
    const int64_t b = (L.max_qh + 7) / 8;
    return dim3((unsigned)(b < 1 ? 1 : b < 148 * 8 ? b : 148 * 8), (unsigned)L.nframes);
}
static inline unsigned flat_blocks(int64_t n, int threads) {
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148 * 32) b = 148 * 32;
    return (unsigned)b;
}

void launch_decimate(const Launch &L, const FrameDesc *frames, const uint8_t *img, uint8_t *qim, float factor) {
    k_decimate<<<frame_grid(L), 256, 0, L.stream>>>(frames, img, qim, factor);
}

void launch_blur(const Launch &L, const FrameDesc *frames, uint8_t *qim, uint8_t *tmp_a, uint8_t *tmp_b,
                 const BlurTaps &taps, bool sharpen) {
    k_blur_pass<<<frame_grid(L), 256, 0, L.stream>>>(frames, qim, tmp_a, taps, 0);
    k_blur_pass<<<frame_grid(L), 256, 0, L.stream>>>(frames, tmp_a, tmp_b, taps, 1);
    k_blur_finish<<<frame_grid(L), 256, 0, L.stream>>>(frames, tmp_b, qim, sharpen ? 1 : 0);
}

void launch_threshold(const Launch &L, const FrameDesc *frames, const uint8_t *qim, uint8_t *tmax, uint8_t *tmin,
                      uint8_t *thr, int32_t diff) {
    k_tile_minmax<<<frame_grid(L), 256, 0, L.stream>>>(frames, qim, tmax, tmin);
    k_threshold<<<frame_grid(L), 256, 0, L.stream>>>(frames, qim, tmax, tmin, thr, diff);
}

void launch_decimate_threshold(const Launch &L, const FrameDesc *frames, int64_t max_cells, uint8_t *qim, uint8_t *thr,
                               int32_t diff) {
    // blocks per frame: enough regions for the frame with the most cells
    // (each block finds its region from its frame's width; extra ones exit)
    k_decimate_threshold<<<dim3((unsigned)max_cells, (unsigned)L.nframes), DT_THREADS, 0, L.stream>>>(frames, qim, thr,
                                                                                                     diff);
}

int64_t decimate_threshold_blocks(int64_t qw, int64_t qh) {
    const int64_t cw = (qw + 3) / 4, ch = (qh + 3) / 4;
    return ((cw + DT_COLS - 1) / DT_COLS) * ((ch + DT_ROWS - 1) / DT_ROWS);
}

void launch_deglitch(const Launch &L, const FrameDesc *frames, uint8_t *thr, uint8_t *tmp) {
    k_morph<<<frame_grid(L), 256, 0, L.stream>>>(frames, thr, tmp, 1);
    k_morph<<<frame_grid(L), 256, 0, L.stream>>>(frames, tmp, thr, 0);
}

int launch_segment(const Launch &L, const FrameDesc *frames, const uint8_t *thr, RunArrays runs, uint32_t *row_nruns,
                   uint32_t *lab, int32_t min_px, int64_t max_qh) {
    dim3 rg((unsigned)(max_qh < 148 * 16 ? max_qh : 148 * 16), (unsigned)L.nframes);
    const int64_t rb = (max_qh + 7) / 8;
    k_row_runs<<<dim3((unsigned)(rb < 148 * 8 ? rb : 148 * 8), (unsigned)L.nframes), 256, 0, L.stream>>>(frames, thr,
                                                                                                        runs, row_nruns);
    const int64_t nb = (max_qh + UB_ROWS - 1) / UB_ROWS;
    k_band_union<<<dim3((unsigned)(nb < 148 * 4 ? nb : 148 * 4), (unsigned)L.nframes), 256, 0, L.stream>>>(
        frames, runs, row_nruns);
    k_band_join<<<dim3((unsigned)(nb < 148 * 4 ? nb : 148 * 4), (unsigned)L.nframes), 256, 0, L.stream>>>(
        frames, thr, runs, row_nruns);
    k_row_sums<<<rg, 256, 0, L.stream>>>(frames, runs, row_nruns);
    if (warp_rows(L))
        k_labels_w<<<row_warp_grid(L), 256, 0, L.stream>>>(frames, thr, runs, row_nruns, lab, min_px);
    else
        k_labels<<<rg, LAB_THREADS, 0, L.stream>>>(frames, runs, row_nruns, lab, min_px);
    return 5;
}

void launch_point_count(const Launch &L, const FrameDesc *frames, const uint8_t *thr, const uint32_t *lab,
                        uint64_t *row_npts) {
    if (warp_rows(L))
        k_point_count<<<row_warp_grid(L), 256, 0, L.stream>>>(frames, thr, lab, row_npts);
    else
        k_point_count_block<<<frame_grid(L), 256, 0, L.stream>>>(frames, thr, lab, row_npts);
}

void launch_point_emit(const Launch &L, const FrameDesc *frames, const uint8_t *thr, const uint32_t *lab,
                       const uint64_t *row_pt_off, uint64_t *pt_key, uint64_t *pt_val, int nb) {
    if (warp_rows(L))
        k_point_emit<<<row_warp_grid(L), 256, 0, L.stream>>>(frames, thr, lab, row_pt_off, pt_key, pt_val, nb);
    else
        k_point_emit_block<<<frame_grid(L), 256, 0, L.stream>>>(frames, thr, lab, row_pt_off, pt_key, pt_val, nb);
}

void launch_cluster_collect(cudaStream_t s, const uint64_t *tkeys, uint32_t size, uint64_t *okeys, uint32_t *oslots,
                            uint32_t *count) {
    k_cluster_collect<<<flat_blocks(size, 256), 256, 0, s>>>(tkeys, size, okeys, oslots, count);
}

void launch_cluster_heads(cudaStream_t s, const uint64_t *key, int64_t n, uint32_t *head) {
    k_cluster_heads<<<flat_blocks(n, 256), 256, 0, s>>>(key, n, head);
}

void launch_cluster_starts(cudaStream_t s, const uint64_t *key, const uint32_t *head, const uint32_t *head_scan,
                           int64_t n, int nb, const FrameDesc *frames, int nframes, uint32_t *cstart, int32_t *cframe,
                           uint64_t *ckey) {
    k_cluster_starts<<<flat_blocks(n, 256), 256, 0, s>>>(key, head, head_scan, n, nb, frames, nframes, cstart, cframe,
                                                         ckey);
}

// One size class of the warp fit kernel on stream s: enough blocks to fill
// every SM as far as shared memory allows.
template <int R>
static void launch_fit_warp(cudaStream_t s, const FrameDesc *frames, const GpuParams &prm, const uint8_t *qim,
                            const uint64_t *pts, const uint32_t *cstart, const int32_t *cframe, int64_t nclusters,
                            int64_t npoints, const FitScratch &scr, int q, GpuQuad *quads, uint32_t *quad_ok, int mm) {
    const size_t wsm = fit_warp_smem(32 * R, mm, R >= 16) * FIT_WPB;
    cudaFuncSetAttribute(k_fit_warp<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wsm);
    // as many blocks as fit on the SMs at once (registers and shared memory)
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fit_warp<R>, FIT_WPB * 32, wsm) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    const int64_t full = 148 * (int64_t)per_sm;
    const int64_t wb = (nclusters + FIT_WPB - 1) / FIT_WPB;
    k_fit_warp<R><<<(unsigned)(wb < full ? wb : full), FIT_WPB * 32, wsm, s>>>(
        frames, prm, qim, pts, cstart, cframe, nclusters, npoints, scr.lists + (int64_t)q * nclusters,
        scr.counts + q, scr.counts + FIT_NCLASS + q, quads, quad_ok, mm, scr);
}

void launch_fit_quads(cudaStream_t s, cudaStream_t side, cudaStream_t side2, cudaStream_t side3, cudaEvent_t fork,
                      cudaEvent_t join, cudaEvent_t join2, cudaEvent_t join3, const FrameDesc *frames, const GpuParams &prm, const uint8_t *qim,
                      const uint64_t *pts, const uint32_t *cstart, const int32_t *cframe, int64_t nclusters,
                      int64_t npoints, const FitScratch &scr, GpuQuad *quads, uint32_t *quad_ok, uint32_t *err) {
    if (nclusters <= 0) return;
    const size_t small = fit_smem_bytes(FIT_SMALL, FIT_CHUNK_SMALL, 128 / 32),
                 large = fit_smem_bytes(FIT_LARGE_SORT, FIT_CHUNK_LARGE, FIT_LARGE_NT / 32);
    cudaFuncSetAttribute(k_fit_quads<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)small);
    cudaFuncSetAttribute(k_fit_quads<FIT_LARGE_NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)large);
    cudaFuncSetAttribute(k_fit_order, cudaFuncAttributeMaxDynamicSharedMemorySize, FIT_ORDER_CAP * 8);
    const int mm = prm.max_nmaxima > 4 ? prm.max_nmaxima : 4;
    // the size classes' lists, the two block classes' largest first
    cudaMemsetAsync(scr.counts, 0, 2 * FIT_NCLASS * sizeof(uint32_t), s);
    k_fit_classify<<<flat_blocks(nclusters, 256), 256, 0, s>>>(frames, cstart, cframe, nclusters, npoints,
                                                                prm.min_cluster_pixels, quad_ok, scr.lists,
                                                                scr.counts);
    // four streams, one per group of classes: the large clusters (a block
    // of FIT_LARGE_NT each, two an SM); 513-1024 points (a block of 128);
    // 257-512 (a warp each); up to 256 (a warp each). Only the two block
    // classes are put largest first, each on its own stream, so the warp
    // classes start at once (unsorted, the 513-1024 class measured slower:
    // 175 vs 159 us, a long cluster last).
    cudaEventRecord(fork, s);
    cudaStreamWaitEvent(side, fork, 0);
    cudaStreamWaitEvent(side2, fork, 0);
    cudaStreamWaitEvent(side3, fork, 0);
    k_fit_order<<<1, 1024, FIT_ORDER_CAP * 8, side>>>(cstart, nclusters, npoints, scr.lists, scr.counts, 4);
    k_fit_order<<<1, 1024, FIT_ORDER_CAP * 8, side2>>>(cstart, nclusters, npoints, scr.lists, scr.counts, 3);
    // two blocks an SM: one cluster's serial steps overlap the other's
    const unsigned nbig = (unsigned)(nclusters < 2 * 148 ? nclusters : 2 * 148);
    k_fit_quads<FIT_LARGE_NT><<<nbig, FIT_LARGE_NT, large, side>>>(frames, prm, qim, pts, cstart, cframe, nclusters, npoints, scr,
                                                 quads, quad_ok, err, scr.lists + 4 * nclusters, scr.counts + 4,
                                                 scr.counts + FIT_NCLASS + 4, FIT_LARGE_SORT, FIT_CHUNK_LARGE);
    cudaEventRecord(join, side);
    const unsigned mid = (unsigned)(nclusters < 148 * 4 ? nclusters : 148 * 4);
    k_fit_quads<128><<<mid, 128, small, side2>>>(frames, prm, qim, pts, cstart, cframe, nclusters, npoints, scr,
                                                 quads, quad_ok, err, scr.lists + 3 * nclusters, scr.counts + 3,
                                                 scr.counts + FIT_NCLASS + 3, FIT_SMALL, FIT_CHUNK_SMALL);
    cudaEventRecord(join2, side2);
    launch_fit_warp<16>(side3, frames, prm, qim, pts, cstart, cframe, nclusters, npoints, scr, 2, quads, quad_ok, mm);
    cudaEventRecord(join3, side3);
    launch_fit_warp<4>(s, frames, prm, qim, pts, cstart, cframe, nclusters, npoints, scr, 0, quads, quad_ok, mm);
    launch_fit_warp<8>(s, frames, prm, qim, pts, cstart, cframe, nclusters, npoints, scr, 1, quads, quad_ok, mm);
    cudaStreamWaitEvent(s, join, 0);
    cudaStreamWaitEvent(s, join2, 0);
    cudaStreamWaitEvent(s, join3, 0);
}

void launch_gather_quads(cudaStream_t s, const GpuQuad *quads, const uint32_t *ok, const uint32_t *scan, int64_t n,
                         GpuQuad *out, uint32_t *nq, uint32_t *qcl) {
    if (n <= 0) return;
    k_gather_quads<<<flat_blocks(n, 256), 256, 0, s>>>(quads, ok, scan, n, out, nq, qcl);
}

void launch_frame_bounds(cudaStream_t s, const GpuQuad *quads, const uint32_t *nq, int nframes, int nfam,
                         int64_t *qstart, int64_t *out_off) {
    k_frame_bounds<<<flat_blocks(nframes + 1, 256), 256, 0, s>>>(quads, nq, nframes, nfam, qstart, out_off);
}

void launch_output(cudaStream_t s, int nframes, const int64_t *qstart, const GpuDetection *out,
                   const int64_t *out_off, const int64_t *out_n, int64_t *first, GpuDetection *host,
                   int64_t *meta, int64_t max_dets) {
    k_output_meta<<<1, 256, 0, s>>>(nframes, qstart, out_n, first, meta);
    const int64_t blocks = (max_dets + 7) / 8;
    k_output_copy<<<(unsigned)(blocks < 1 ? 1 : blocks < 148 * 4 ? blocks : 148 * 4), 256, 0, s>>>(nframes, out, out_off,
                                                                                                first, host);
}

void launch_decode(cudaStream_t s, const FrameDesc *frames, const GpuParams &prm, const GpuFamily *fams,
                   const uint8_t *img, const uint8_t *qim, const GpuQuad *quads, int64_t max_quads,
                   const DecodeScratch &scr, GpuDetection *dets, uint32_t *det_ok) {
    // grids for at most max_quads quads; the kernels read the count (scr.nq)
    if (max_quads <= 0) return;
    const unsigned blocks = (unsigned)(max_quads < 148 * 64 ? max_quads : 148 * 64);
    k_refine<<<blocks, AT_DEC_THREADS, 0, s>>>(frames, prm, img, qim, quads, scr.nq, scr.corners, det_ok);
    const int64_t hb = (max_quads + QH_WARPS - 1) / QH_WARPS;
    k_quad_homography<<<(unsigned)(hb < 148 * 16 ? hb : 148 * 16), QH_WARPS * 32, 0, s>>>(scr.corners, scr.nq,
                                                                                        scr.h, scr.hok);
    k_decode<<<blocks, AT_DEC_THREADS, 0, s>>>(frames, prm, fams, img, qim, quads, scr.nq, scr.h, scr.hok, dets,
                                               det_ok);
}

void launch_finalize(cudaStream_t s, int nframes, const int64_t *frame_qstart, int nfam, const GpuDetection *dets,
                     const uint32_t *det_ok, uint32_t *idx, uint8_t *removed, GpuDetection *out,
                     const int64_t *out_off, int64_t *out_n, const FrameDesc *frames, const RefOrder &ref,
                     const uint32_t *qcl, const uint64_t *ckey, int nb, uint64_t *okey, uint32_t *idx2,
                     uint32_t *err) {
    k_finalize<<<nframes, 256, 0, s>>>(nframes, frame_qstart, nfam, dets, det_ok, idx, removed, out, out_off, out_n,
                                       frames, ref, qcl, ckey, nb, okey, idx2, err);
}
