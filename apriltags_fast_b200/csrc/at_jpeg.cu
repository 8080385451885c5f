// Baseline JPEG decode into 8-bit frames on the GPU: the input side of the
// detector (the reference decodes camera photos with common/pjpeg.c, whose
// pjpeg_create_from_file / pjpeg_to_u8_baseline its tests and demo call).
//
// Output equals the reference's decoder byte for byte on every file it
// decodes: the same marker walk and error codes, the same Huffman code
// space (a code that matches nothing reads as 0 bits, symbol 0), the same
// restart handling (which zeroes the DC predictor of the scan's first
// component only, common/pjpeg.c:494-518), the same integer IDCT
// (common/pjpeg-idct.c:272-385) and the same component planes.
//
// Work split. The host parses the headers (a few hundred bytes) and walks
// each scan's bytes once, keeping the stream as the reference's reader
// sees it (FF 00 read as FF, markers read as data) and cutting it at the
// restart markers into segments that decode on their own. Everything else
// is on the device:
//
//  * k_jpeg_sync (cooperative, one launch): every segment is cut into
//    sub-streams of 256 to 1024 bits (by the call's data size), one thread
//    each. Pass 0 decodes each sub-stream from a run-in before its first
//    bit, as if a block started there; later passes re-decode a sub-stream
//    from the exit state (bit, coefficient, block of the MCU) of its
//    predecessor whenever that changed, a CTA repeating over its own
//    sub-streams until they settle. Huffman codes fall back into step
//    within a few codes, so the exits mostly settle in one or two passes;
//    a segment's first sub-stream starts exactly, so the passes end by
//    construction (at worst after one per sub-stream). The same launch
//    then scans, over the sub-streams, the block counts and the DC
//    differences of each scan component.
//  * k_jpeg_write: each sub-stream decodes again from its exact entry and
//    owns the blocks whose DC code lies inside it; it gathers each in
//    shared memory and stores its quantised coefficients whole, with its
//    DC value.
//  * k_jpeg_idct: 8 lanes per block dequantise, run the IDCT (rows, then
//    columns) and store the 8x8 pixels.
#include <cuda_runtime.h>
#include <stdint.h>
#if defined(__x86_64__) || defined(__i386__)
#include <emmintrin.h>
#define JSINK_STREAM 1
#endif
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "apriltag_fast.h"
#include "common/pjpeg.h"

namespace {

// Bits per sub-stream, by job: short sub-streams give one image more
// threads (latency), long ones spend less of a large batch on run-ins.
uint32_t jsub_for(int64_t stream_bytes) {
    uint32_t b = 256;
    while (b < 1024 && (uint64_t)stream_bytes * 8 / b > 65536) b *= 2;
    return b;
}
constexpr int JMAX_BPM = 64;        // blocks per MCU (the standard allows 10)
constexpr int JSYNC_THREADS = 128;
constexpr int JWRITE_THREADS = 128;
constexpr int JPAD = 32;            // 1-bytes after each scan's stream
constexpr uint32_t JSTUCK = 0xffffffffu;

// ---------------------------------------------------------------------
// Device data of one decode job (any number of scans of any number of
// images).

constexpr int JMAX_RUNS = 48;

// One Huffman table: runs of equal-length codes over the 16-bit code
// space, in order (run r ends at rend[r]; position w of it decodes as
// symbol pool[rsym[r] + ((w - rorigin[r]) >> (16 - rlen[r]))]), and a
// lookup of the codes of up to 9 bits by the window's first 9 bits.
struct JTab {
    uint16_t lut[512];    // (bits << 8) | symbol, 0 if the prefix needs the runs
    uint32_t nrun, r0;    // runs; the first run a lookup miss can land in
    uint32_t rend[JMAX_RUNS], rorigin[JMAX_RUNS], rsym[JMAX_RUNS];
    uint8_t rlen[JMAX_RUNS];
};

struct JScanDev {
    uint32_t tab0;        // this scan's 4 tables (DC 0, DC 1, AC 0, AC 1) in the job's table array
    uint32_t mcus_x, nmcu;
    uint32_t restart;     // MCUs per segment (0: one segment)
    uint32_t sub0;        // first sub-stream of the scan
    uint32_t bpm;         // blocks per MCU
    uint32_t ns;          // scan components
    uint8_t bcomp[JMAX_BPM], bsx[JMAX_BPM], bsy[JMAX_BPM];
    // the smallest block of the MCU from which the sequence of Huffman
    // tables continues exactly as from block b: decoders at the same bit
    // and coefficient in blocks b and bcanon[b] stay in step for ever
    uint8_t bcanon[JMAX_BPM];
    uint8_t dc[3], ac[3];
    int32_t plane[3];     // output plane of each scan component, -1: not written
};

struct JSegDev {
    uint32_t scan, start, end;   // bit range in the job's stream
    uint32_t sub0, nsub;         // its sub-streams
    uint32_t blk0, nblk;         // its blocks, in the scan's decode order
};

struct JPlaneDev {
    uint8_t *out;         // pixels, rows of `stride` bytes
    int64_t stride;
    uint32_t ow, oh;      // pixels written: x < ow, y < oh
    uint32_t sx, sy;      // blocks of the component per MCU
    uint32_t mcus_x;
    uint32_t blk0, nblk;  // its blocks in the job's coefficient arrays (MCU order)
    int32_t q[64];        // dequantisation, natural order
};

struct JJob {
    const uint32_t *stream;      // big-endian bit stream, word aligned
    const JTab *tabs;
    const uint8_t *syms;
    const JScanDev *scans;
    const JSegDev *segs;
    const uint32_t *sub_seg;
    const JPlaneDev *planes;
    int16_t *coef;               // per block written: 64 quantised coefficients, natural order
    int32_t *dc;                 // per block written: its DC value (the predictor after the block)
    uint32_t nplanes, nblocks;
    uint32_t nsub, sub_bits, back_bits, max_passes;
    // sync state and the scans over the sub-streams
    unsigned long long *exitst, *used;
    uint32_t *cnt;               // 4 per sub-stream: blocks, DC sums of scan components 0..2
    uint32_t *excl;              // 4 per sub-stream: exclusive scans of cnt
    uint32_t *totals;            // 4 per CTA
    uint32_t *seg_stuck;         // per segment: its first sub-stream whose decode stops moving (~0: none)
    uint32_t *seg_endbit;        // per segment: the bit where its last block ends (~0: not reached)
    unsigned int *bar;           // grid barrier: count, generation
    int *changed;                // per pass
    int *err;
};

// Loads and bit operations of the decode, also compiled for the host so
// that the decode itself can be stepped through on the CPU.
#ifdef __CUDA_ARCH__
#define JLDG(p) __ldg(p)
#else
#define JLDG(p) (*(p))
#endif
__host__ __device__ __forceinline__ uint32_t jbswap(uint32_t x) {
#ifdef __CUDA_ARCH__
    return __byte_perm(x, 0, 0x0123);
#else
    return __builtin_bswap32(x);
#endif
}
// the upper 32 bits of (hi:lo) << s, s in [0, 31]
__host__ __device__ __forceinline__ uint32_t jfunnel(uint32_t lo, uint32_t hi, uint32_t s) {
#ifdef __CUDA_ARCH__
    return __funnelshift_l(lo, hi, s);
#else
    return s ? (hi << s) | (lo >> (32 - s)) : hi;
#endif
}

__host__ __device__ __forceinline__ unsigned long long jpack(uint32_t p, int z, int b) {
    return (unsigned long long)p | ((unsigned long long)z << 32) | ((unsigned long long)b << 40);
}

// Reads the stream 32 bits at a time at any bit position, keeping the two
// words around the last position in registers.
struct JReader {
    const uint32_t *w;
    uint32_t k, a, b;
    __host__ __device__ __forceinline__ void init(const uint32_t *words) {
        w = words;
        k = 0xfffffffeu;
    }
    __host__ __device__ __forceinline__ uint32_t peek(uint32_t p) {
        const uint32_t kk = p >> 5;
        if (kk != k) {
            if (kk == k + 1) {
                a = b;
            } else {
                a = jbswap(JLDG(w + kk));
            }
            b = jbswap(JLDG(w + kk + 1));
            k = kk;
        }
        return jfunnel(b, a, p & 31);
    }
};

// One code of table t at the window `win` (the next 32 bits): its length
// in bits (0 when nothing matches) and symbol.
__host__ __device__ __forceinline__ int jdecode(const JTab *__restrict__ t, const uint8_t *__restrict__ syms, uint32_t win,
                                       int &sym) {
    const uint32_t e = JLDG(&t->lut[win >> 23]);
    if (e) {
        sym = e & 255;
        return (int)(e >> 8);
    }
    const uint32_t w16 = win >> 16;
    const uint32_t nr = JLDG(&t->nrun);
#pragma unroll 1
    for (uint32_t r = JLDG(&t->r0); r < nr; r++) {
        if (w16 < JLDG(&t->rend[r])) {
            const int l = JLDG(&t->rlen[r]);
            sym = JLDG(&syms[JLDG(&t->rsym[r]) + ((w16 - JLDG(&t->rorigin[r])) >> (16 - l))]);
            return l;
        }
    }
    sym = 0;
    return 0;
}

__host__ __device__ __forceinline__ int32_t jextend(uint32_t v, int s) {
    return (s && !(v >> (s - 1))) ? (int32_t)v - ((1 << s) - 1) : (int32_t)v;
}

// The decoder's position: bit p, next coefficient z (0: the DC code),
// block b of the MCU, and the tables of that block's component.
struct JPos {
    uint32_t p;
    int z, b;
    const JTab *dc, *ac;
    int comp;
};

__host__ __device__ __forceinline__ void jset_block(JPos &s, const JScanDev &S, const JTab *tabs) {
    const int c = S.bcomp[s.b];
    s.comp = c;
    s.dc = tabs + S.tab0 + S.dc[c];
    s.ac = tabs + S.tab0 + S.ac[c];
}

// Decodes from the state `in` up to the first code boundary at or past
// bit `end`: the exit state, and from the first code boundary at or past
// bit `from` (its state to *entry) the blocks ended and the DC differences
// of the blocks that start there, per scan component. A position that
// decodes no bits through a whole MCU of codes can never move again: the
// decode stops there with the exit state JSTUCK. Block numbers in states
// are kept as bcanon.
__host__ __device__ unsigned long long jrun_sync(const JJob &J, const JScanDev &S, unsigned long long in,
                                                 uint32_t from, uint32_t end, uint32_t *out4,
                                                 unsigned long long *entry) {
    uint32_t nblk = 0, dc0 = 0, dc1 = 0, dc2 = 0;
    bool counting = false;
    JPos s;
    s.p = (uint32_t)in;
    if (s.p == JSTUCK) {
        out4[0] = out4[1] = out4[2] = out4[3] = 0;
        *entry = in;
        return in;
    }
    s.z = (int)((in >> 32) & 0xff);
    s.b = (int)((in >> 40) & 0xff);
    jset_block(s, S, J.tabs);
    JReader R;
    R.init(J.stream);
    const int stall_max = 2 * (int)S.bpm + 2;
    int stall = 0;
    unsigned long long out = 0;
    while (true) {
        if (!counting && s.p >= from) {
            counting = true;
            *entry = jpack(s.p, s.z, S.bcanon[s.b]);
        }
        if (s.p >= end) {
            out = jpack(s.p, s.z, S.bcanon[s.b]);
            break;
        }
        const uint32_t win = R.peek(s.p);
        int sym;
        const int nb = jdecode(s.z == 0 ? s.dc : s.ac, J.syms, win, sym);
        const int sz = sym & 15;
        if (nb == 0) {
            if (++stall > stall_max) {
                out = jpack(JSTUCK, 0, 0);
                if (!counting) *entry = out;
                break;
            }
        } else {
            stall = 0;
        }
        if (s.z == 0) {
            const uint32_t v = sz ? (win << nb) >> (32 - sz) : 0;
            const uint32_t d = counting ? (uint32_t)jextend(v, sz) : 0u;
            if (s.comp == 0) dc0 += d;
            else if (s.comp == 1) dc1 += d;
            else dc2 += d;
            s.z = 1;
        } else if (sym == 0) {
            s.z = 64;
        } else {
            s.z += (sym >> 4) + 1;
        }
        s.p += nb + sz;
        if (s.z >= 64) {
            s.z = 0;
            if (++s.b == (int)S.bpm) s.b = 0;
            jset_block(s, S, J.tabs);
            nblk += counting;
        }
    }
    out4[0] = nblk;
    out4[1] = dc0;
    out4[2] = dc1;
    out4[3] = dc2;
    return out;
}

// A grid barrier for a cooperative launch (all CTAs resident). The wait is
// bounded: past the limit the CTA records an error and returns false.
__device__ bool jgrid_sync(unsigned int *bar, unsigned int nblocks, int *err) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        s_ok = 1;
        volatile unsigned int *gen = bar + 1;
        const unsigned int g = *gen;
        __threadfence();
        if (atomicAdd(bar, 1u) == nblocks - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            long long spins = 0;
            while (*gen == g) {
                if (++spins > (1ll << 24)) {
                    atomicExch(err, 1);
                    s_ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return s_ok;
}

// Sub-streams of CTA j: [j * per, (j + 1) * per), visited in rounds of
// blockDim.x consecutive ones.
__global__ void __launch_bounds__(JSYNC_THREADS, 8) k_jpeg_sync(JJob J, uint32_t per) {
    const uint32_t lo = blockIdx.x * per, hi = min(J.nsub, lo + per);
    const unsigned nb = gridDim.x;
    // pass 0: every sub-stream decoded from back_bits before its first bit
    // (the segment's first from its exact start), as if a block started
    // there: by its first bit the decode has mostly fallen into step with
    // the true one
    for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const JSegDev &G = J.segs[J.sub_seg[i]];
        const JScanDev &S = J.scans[G.scan];
        const uint32_t start = G.start + (i - G.sub0) * J.sub_bits;
        const uint32_t end = min(G.end, start + J.sub_bits);
        const uint32_t back = i == G.sub0 ? start : start - min(J.back_bits, start - G.start);
        uint32_t c4[4];
        unsigned long long entry;
        J.exitst[i] = jrun_sync(J, S, jpack(back, 0, 0), start, end, c4, &entry);
        J.used[i] = entry;
        for (int k = 0; k < 4; k++) J.cnt[4 * (size_t)i + k] = c4[k];
    }
    if (!jgrid_sync(J.bar, nb, J.err)) return;
    // passes: a sub-stream whose predecessor's exit moved is decoded again.
    // Within a pass a CTA repeats over its own sub-streams until none of
    // their exits moves; only a move of its last exit (the next CTA's
    // entry) needs another pass over the grid.
    for (uint32_t pass = 1; pass <= J.max_passes; pass++) {
      bool edge = false;
      for (uint32_t round = 0;; round++) {
        bool any = false;
        for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
            const JSegDev &G = J.segs[J.sub_seg[i]];
            if (i == G.sub0) continue;
            const unsigned long long in = *(volatile unsigned long long *)&J.exitst[i - 1];
            // An entry that never moves again gives nothing to decode: what
            // follows it in the segment is dead (decided below), and a
            // speculative one is replaced by a true exit in a later pass.
            if (in == J.used[i] || (uint32_t)in == JSTUCK) continue;
            const JScanDev &S = J.scans[G.scan];
            const uint32_t start = G.start + (i - G.sub0) * J.sub_bits;
            const uint32_t end = min(G.end, start + J.sub_bits);
            uint32_t c4[4];
            unsigned long long entry;
            const unsigned long long x = jrun_sync(J, S, in, start, end, c4, &entry);
            // a segment's last exit has no successor to move
            if (x != J.exitst[i] && i + 1 != G.sub0 + G.nsub) {
                any = true;
                edge |= i + 1 == hi;
            }
            *(volatile unsigned long long *)&J.exitst[i] = x;
            J.used[i] = in;
            for (int k = 0; k < 4; k++) J.cnt[4 * (size_t)i + k] = c4[k];
        }
        if (!__syncthreads_or(any)) {
            if (threadIdx.x == 0 && round) atomicMax(&J.changed[J.max_passes + 1], (int)round);
            break;
        }
        if (round >= 7) {
            // Long chains (a decode that stays out of step over many
            // sub-streams, as 4:2:0 MCUs give): one thread walks the CTA's
            // sub-streams in order instead, each decoded at most once more
            // (measured on one smooth-chroma 4:2:0 frame: 1.39 -> 1.00 ms;
            // walking from the fourth round cost batches of such frames
            // more than it saved, since one thread then does in turn what
            // parallel rounds did side by side).
            __shared__ int s_edge;
            if (threadIdx.x == 0) {
                s_edge = 0;
                for (uint32_t i = lo; i < hi; i++) {
                    const JSegDev &G = J.segs[J.sub_seg[i]];
                    if (i == G.sub0) continue;
                    const unsigned long long in = *(volatile unsigned long long *)&J.exitst[i - 1];
                    if (in == J.used[i] || (uint32_t)in == JSTUCK) continue;
                    const uint32_t start = G.start + (i - G.sub0) * J.sub_bits;
                    const uint32_t end = min(G.end, start + J.sub_bits);
                    uint32_t c4[4];
                    unsigned long long entry;
                    const unsigned long long x = jrun_sync(J, J.scans[G.scan], in, start, end, c4, &entry);
                    if (x != J.exitst[i] && i + 1 != G.sub0 + G.nsub && i + 1 == hi) s_edge = 1;
                    *(volatile unsigned long long *)&J.exitst[i] = x;
                    J.used[i] = in;
                    for (int k = 0; k < 4; k++) J.cnt[4 * (size_t)i + k] = c4[k];
                }
                atomicMax(&J.changed[J.max_passes + 1], (int)round + 1);
            }
            __syncthreads();
            edge |= s_edge != 0;
            break;
        }
      }
        if (edge) J.changed[pass] = 1;
        if (!jgrid_sync(J.bar, nb, J.err)) return;
        if (!*(volatile int *)&J.changed[pass]) {
            if (blockIdx.x == 0 && threadIdx.x == 0) J.changed[0] = (int)pass;
            break;
        }
        if (pass == J.max_passes && threadIdx.x == 0) atomicExch(J.err, 2);  // cannot happen: one pass per sub-stream suffices
    }
    // the first sub-stream of each segment whose decode stops moving: the
    // ones after it are dead (they count nothing and write nothing)
    for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x)
        if ((uint32_t)J.exitst[i] == JSTUCK) atomicMin(&J.seg_stuck[J.sub_seg[i]], i);
    if (!jgrid_sync(J.bar, nb, J.err)) return;
    for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x)
        if (*(volatile uint32_t *)&J.seg_stuck[J.sub_seg[i]] < i)
            for (int k = 0; k < 4; k++) J.cnt[4 * (size_t)i + k] = 0;
    // exclusive scans of the four counts over all sub-streams
    __shared__ uint32_t s_red[4][JSYNC_THREADS];
    __shared__ uint32_t s_base[4];
    uint32_t t4[4] = {0, 0, 0, 0};
    for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x)
        for (int k = 0; k < 4; k++) t4[k] += J.cnt[4 * (size_t)i + k];
    for (int k = 0; k < 4; k++) s_red[k][threadIdx.x] = t4[k];
    __syncthreads();
    if (threadIdx.x < 4) {
        uint32_t a = 0;
        for (int t = 0; t < JSYNC_THREADS; t++) a += s_red[threadIdx.x][t];
        J.totals[4 * blockIdx.x + threadIdx.x] = a;
    }
    if (!jgrid_sync(J.bar, nb, J.err)) return;
    if (threadIdx.x < 4) {
        uint32_t a = 0;
        for (uint32_t j = 0; j < blockIdx.x; j++) a += *(volatile uint32_t *)&J.totals[4 * j + threadIdx.x];
        s_base[threadIdx.x] = a;
    }
    __syncthreads();
    for (uint32_t r = lo; r < hi; r += blockDim.x) {
        const uint32_t i = r + threadIdx.x;
        uint32_t v[4] = {0, 0, 0, 0};
        if (i < hi)
            for (int k = 0; k < 4; k++) v[k] = J.cnt[4 * (size_t)i + k];
        for (int k = 0; k < 4; k++) s_red[k][threadIdx.x] = v[k];
        __syncthreads();
        // inclusive scan in shared memory (Hillis-Steele)
        for (int off = 1; off < JSYNC_THREADS; off <<= 1) {
            uint32_t add[4];
            for (int k = 0; k < 4; k++) add[k] = threadIdx.x >= (unsigned)off ? s_red[k][threadIdx.x - off] : 0;
            __syncthreads();
            for (int k = 0; k < 4; k++) s_red[k][threadIdx.x] += add[k];
            __syncthreads();
        }
        if (i < hi)
            for (int k = 0; k < 4; k++) J.excl[4 * (size_t)i + k] = s_base[k] + s_red[k][threadIdx.x] - v[k];
        __syncthreads();
        if (threadIdx.x < 4) s_base[threadIdx.x] += s_red[threadIdx.x][JSYNC_THREADS - 1];
        __syncthreads();
    }
}

// Zig-zag position -> natural position (ITU-T T.81 figure A.6).
const uint8_t H_ZIG[64] = {0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,
                           12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6,  7,  14, 21, 28,
                           35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
                           58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};
__constant__ uint8_t c_zig[64] = {0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,
                                  12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6,  7,  14, 21, 28,
                                  35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
                                  58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

// The reference's integer IDCT (common/pjpeg-idct.c:272-385): the
// fixed-point butterfly of the MPEG-2 reference decoder as NanoJPEG writes
// it; rotation constants 2048 * sqrt(2) * cos(k * pi / 16).
constexpr int JC1 = 2841, JC2 = 2676, JC3 = 2408, JC5 = 1609, JC6 = 1108, JC7 = 565;

// One 8-point pass over v[0], v[st], ..., v[7 st] (shared memory). Row
// pass: in place, DC << 11 with bias 128, results >> 8. Column pass: DC
// << 8 with bias 8192, rotations rounded (+4) >> 3, results >> 14 + 128,
// clamped to bytes in pix[0..7]; the column is left zeroed.
template <bool COL>
__host__ __device__ __forceinline__ void jidct_pass(int32_t *v, int st, uint8_t *pix) {
    constexpr int sh = COL ? 8 : 11;
    const int32_t x1 = (int32_t)((uint32_t)v[4 * st] << sh);
    const int32_t a2 = v[6 * st], a3 = v[2 * st], a4 = v[1 * st], a5 = v[7 * st], a6 = v[5 * st],
                  a7 = v[3 * st];
    const int32_t v0 = v[0];
    if (!(x1 | a2 | a3 | a4 | a5 | a6 | a7)) {
        if (!COL) {
#pragma unroll
            for (int k = 0; k < 8; k++) v[k * st] = v0 * 8;
        } else {
            const int32_t d = ((v0 + 32) >> 6) + 128;
            const uint8_t b = d < 0 ? 0 : d > 255 ? 255 : (uint8_t)d;
#pragma unroll
            for (int k = 0; k < 8; k++) pix[k] = b;
            v[0] = 0;
        }
        return;
    }
    constexpr int32_t rb = COL ? 4 : 0;
    const int32_t x0 = (int32_t)((uint32_t)v0 << sh) + (COL ? 8192 : 128);
    int32_t t, o4, o5, o6, o7, e2, e3;
    t = JC7 * (a4 + a5) + rb;
    o4 = t + (JC1 - JC7) * a4;
    o5 = t - (JC1 + JC7) * a5;
    t = JC3 * (a6 + a7) + rb;
    o6 = t - (JC3 - JC5) * a6;
    o7 = t - (JC3 + JC5) * a7;
    t = JC6 * (a3 + a2) + rb;
    e2 = t - (JC2 + JC6) * a2;
    e3 = t + (JC2 - JC6) * a3;
    if (COL) {
        o4 >>= 3; o5 >>= 3; o6 >>= 3; o7 >>= 3; e2 >>= 3; e3 >>= 3;
    }
    const int32_t e8 = x0 + x1, e0 = x0 - x1;
    const int32_t s1 = o4 + o6, d4 = o4 - o6, s6 = o5 + o7, d5 = o5 - o7;
    const int32_t f7 = e8 + e3, f8 = e8 - e3, f3 = e0 + e2, f0 = e0 - e2;
    const int32_t g2 = (181 * (d4 + d5) + 128) >> 8, g4 = (181 * (d4 - d5) + 128) >> 8;
    const int32_t r[8] = {f7 + s1, f3 + g2, f0 + g4, f8 + s6, f8 - s6, f0 - g4, f3 - g2, f7 - s1};
    if (!COL) {
#pragma unroll
        for (int k = 0; k < 8; k++) v[k * st] = r[k] >> 8;
    } else {
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const int32_t d = (r[k] >> 14) + 128;
            pix[k] = d < 0 ? 0 : d > 255 ? 255 : (uint8_t)d;
            v[k * st] = 0;
        }
    }
}

// The write pass of one sub-stream: it decodes from its exact entry and
// owns the blocks whose DC code lies in it. The last sub-stream of a
// segment decodes on until the segment's blocks are done (past its data
// the stream reads as the reference's reader reads it: markers as data,
// then 1-bits).
struct JWriter {
    JPos s;
    JReader R;
    const JScanDev *S;
    const JPlaneDev *P;   // plane of the block in progress (nullptr: not written)
    uint32_t seg, end, rel, nblk, mcu;
    int32_t pred0, pred1, pred2;  // DC predictors of the scan components
    bool last, own, done;
};

__host__ __device__ __forceinline__ void jwriter_init(JWriter &w, const JJob &J, uint32_t i, bool valid) {
    w.done = true;
    if (!valid) return;
    const uint32_t seg = J.sub_seg[i];
    const JSegDev G = J.segs[seg];
    if (J.seg_stuck[seg] < i) return;  // dead: the segment's decode stopped before it
    const JScanDev &S = J.scans[G.scan];
    w.S = &S;
    w.seg = seg;
    const unsigned long long in = i == G.sub0 ? jpack(G.start, 0, 0) : J.exitst[i - 1];
    w.last = i == G.sub0 + G.nsub - 1;
    w.end = min(G.end, G.start + (i - G.sub0 + 1) * J.sub_bits);
    w.nblk = G.nblk;
    w.rel = J.excl[4 * (size_t)i] - J.excl[4 * (size_t)G.sub0];
    // the first predictor restarts with each segment, the others run
    // through the scan
    w.pred0 = (int32_t)(J.excl[4 * (size_t)i + 1] - J.excl[4 * (size_t)G.sub0 + 1]);
    w.pred1 = (int32_t)(J.excl[4 * (size_t)i + 2] - J.excl[4 * (size_t)S.sub0 + 2]);
    w.pred2 = (int32_t)(J.excl[4 * (size_t)i + 3] - J.excl[4 * (size_t)S.sub0 + 3]);
    // the block in progress at the entry: its number in the MCU follows
    // from the block count (the entry state keeps an equivalent one)
    w.s.p = (uint32_t)in;
    w.s.z = (int)((in >> 32) & 0xff);
    w.s.b = (int)((G.blk0 + w.rel) % S.bpm);
    jset_block(w.s, S, J.tabs);
    w.mcu = (G.blk0 + w.rel) / S.bpm;
    w.own = w.s.z == 0;  // a block begun before the entry belongs to the previous sub-stream
    w.P = nullptr;
    w.R.init(J.stream);
    w.done = false;
}

// Decodes the sub-stream to its end. Each block it owns and writes is
// gathered in blk (64 quantised coefficients, natural order; left zeroed)
// and stored whole to the job's coefficient array, with its DC value.
__host__ __device__ __forceinline__ void jwriter_run(JWriter &w, const JJob &J, int16_t *blk) {
    JPos &s = w.s;
    const JScanDev &S = *w.S;
    int32_t dcv = 0;
    while (true) {
        if (s.z == 0) {
            if ((!w.last && s.p >= w.end) || w.rel >= w.nblk) break;
            w.own = true;
            const int pl = S.plane[s.comp];
            w.P = pl >= 0 ? J.planes + pl : nullptr;
        }
        const uint32_t win = w.R.peek(s.p);
        int sym;
        const int nb = jdecode(s.z == 0 ? s.dc : s.ac, J.syms, win, sym);
        const int sz = sym & 15;
        const int32_t v = jextend(sz ? (win << nb) >> (32 - sz) : 0, sz);
        s.p += nb + sz;
        const bool put = w.own && w.P;
        if (s.z == 0) {
            if (w.own) {
                if (s.comp == 0) dcv = w.pred0 += v;
                else if (s.comp == 1) dcv = w.pred1 += v;
                else dcv = w.pred2 += v;
            }
            s.z = 1;
        } else if (sym == 0) {
            s.z = 64;
        } else {
            s.z += sym >> 4;
            if (put && s.z < 64) {
#ifdef __CUDA_ARCH__
                blk[c_zig[s.z]] = (int16_t)v;
#else
                blk[H_ZIG[s.z]] = (int16_t)v;
#endif
            }
            s.z += 1;
        }
        if (s.z >= 64) {
            if (put) {
                const JPlaneDev &P = *w.P;
                const uint32_t gb = P.blk0 + w.mcu * (P.sx * P.sy) + S.bsy[s.b] * P.sx + S.bsx[s.b];
                J.dc[gb] = dcv;
                uint4 *src = (uint4 *)blk, *dst = (uint4 *)(J.coef + (size_t)gb * 64);
                const uint4 zero = make_uint4(0, 0, 0, 0);
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    dst[k] = src[k];
                    src[k] = zero;
                }
            }
            s.z = 0;
            // where the segment's decode ends: the reference looks for the
            // next restart marker from there
            if (++w.rel == w.nblk) J.seg_endbit[w.seg] = s.p;
            if (++s.b == (int)S.bpm) {
                s.b = 0;
                w.mcu++;
            }
            jset_block(s, S, J.tabs);
        }
    }
}

// One thread per sub-stream, each decoding on its own.
__global__ void __launch_bounds__(JWRITE_THREADS) k_jpeg_write(JJob J) {
    __shared__ __align__(16) int16_t s_blk[JWRITE_THREADS][64];
    const uint32_t i = blockIdx.x * JWRITE_THREADS + threadIdx.x;
    int16_t *blk = s_blk[threadIdx.x];
    for (int k = 0; k < 8; k++) ((uint4 *)blk)[k] = make_uint4(0, 0, 0, 0);
    JWriter w;
    jwriter_init(w, J, i, i < J.nsub);
    if (!w.done) jwriter_run(w, J, blk);
}

// The IDCT and pixel stores: 8 lanes per block (lane r: row r, then column
// r), 4 blocks per warp.
constexpr int JIDCT_THREADS = 256;
__global__ void __launch_bounds__(JIDCT_THREADS) k_jpeg_idct(JJob J) {
    __shared__ int32_t s_v[JIDCT_THREADS / 8][64];
    __shared__ __align__(16) uint8_t s_px[JIDCT_THREADS / 8][64];
    const uint32_t g = threadIdx.x >> 3, r = threadIdx.x & 7;
    const uint32_t gb = blockIdx.x * (JIDCT_THREADS / 8) + g;
    const bool live = gb < J.nblocks;
    // the block's plane (planes in order of blk0)
    uint32_t lo = 0, hi = J.nplanes;
    while (live && hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (J.planes[mid].blk0 <= gb) lo = mid;
        else hi = mid;
    }
    const JPlaneDev &P = J.planes[lo];
    int32_t *v = s_v[g];
    if (live) {
        const uint4 raw = *(const uint4 *)(J.coef + (size_t)gb * 64 + r * 8);
        const int16_t *c = (const int16_t *)&raw;
#pragma unroll
        for (int k = 0; k < 8; k++) v[r * 8 + k] = (int32_t)c[k] * P.q[r * 8 + k];
        if (r == 0) v[0] = J.dc[gb] * P.q[0];
        jidct_pass<false>(v + r * 8, 1, nullptr);
    }
    __syncwarp();
    uint8_t pix[8];
    if (live) {
        jidct_pass<true>(v + r, 8, pix);
#pragma unroll
        for (int k = 0; k < 8; k++) s_px[g][k * 8 + r] = pix[k];
    }
    __syncwarp();
    if (!live) return;
    const uint32_t L = gb - P.blk0, per = P.sx * P.sy;
    const uint32_t mcu = L / per, sub = L - mcu * per;
    const uint32_t px = ((mcu % P.mcus_x) * P.sx + sub % P.sx) * 8;
    const uint32_t py = ((mcu / P.mcus_x) * P.sy + sub / P.sx) * 8 + r;
    if (px >= P.ow || py >= P.oh) return;
    uint8_t *o = P.out + (int64_t)py * P.stride + px;
    const uint2 row = *(const uint2 *)&s_px[g][r * 8];
    if (px + 8 <= P.ow && !((uintptr_t)o & 7)) {
        *(uint2 *)o = row;
    } else {
        const uint32_t nx = min(8u, P.ow - px);
        for (uint32_t x = 0; x < nx; x++) o[x] = s_px[g][r * 8 + x];
    }
}

}  // namespace

// ---------------------------------------------------------------------
// Host: headers and scans, as the reference's decoder walks them
// (common/pjpeg.c:246-687).

namespace {

// The reference's reader (common/pjpeg.c:163-244): FF 00 reads as one FF,
// every other byte as itself; past the end, 1-bits without moving.
struct HReader {
    const uint8_t *in;
    int64_t pos, len;
    uint32_t bits = 0;
    int avail = 0;
    void fill(int need) {
        while (avail < need) {
            uint8_t b = 0xff;
            if (pos < len) {
                b = in[pos++];
                if (b == 0xff && pos < len && in[pos] == 0) pos++;
            }
            bits = (bits << 8) | b;
            avail += 8;
        }
    }
    uint32_t take(int n) {
        fill(n);
        const uint32_t v = n ? (bits >> (avail - n)) & ((1u << n) - 1) : 0;
        avail -= n;
        return v;
    }
    bool more() const { return avail > 0 || pos < len; }
};

// A Huffman table as runs of equal-length codes over the 16-bit code space
// (position w16 of run r decodes as syms[sym0 + ((w16 - origin) >> (16 -
// len))]). A table defined again keeps the old codes past the end of the
// new ones, as the reference's 65536-entry table does.
struct HRun {
    uint32_t start, end, origin, sym0;
    int len;
};
struct HTab {
    bool present = false;
    std::vector<HRun> runs;
    std::vector<uint8_t> syms;
};

// Defines table t from code counts and symbols; false if the codes pass
// the end of the code space (the reference's PJPEG_ERR_DHT).
bool htab_define(HTab &t, const uint8_t cnt[17], const uint8_t *vals) {
    HTab n;
    uint32_t pos = 0;
    int k = 0;
    for (int l = 1; l <= 16; l++) {
        if (!cnt[l]) continue;
        const uint32_t w = 1u << (16 - l);
        HRun r{pos, pos, pos, (uint32_t)n.syms.size(), l};
        for (int i = 0; i < cnt[l]; i++, k++) {
            if (pos + w > 0xffff) return false;
            n.syms.push_back(vals[k]);
            pos += w;
        }
        r.end = pos;
        n.runs.push_back(r);
    }
    const uint32_t off = (uint32_t)n.syms.size();
    for (const HRun &o : t.runs) {
        if (o.end <= pos) continue;
        HRun c = o;
        c.start = std::max(o.start, pos);
        c.sym0 += off;
        n.runs.push_back(c);
    }
    n.syms.insert(n.syms.end(), t.syms.begin(), t.syms.end());
    // A table defined again and again can pile up more runs than the
    // device form holds: refused.
    if (n.runs.size() > (size_t)JMAX_RUNS) return false;
    n.present = true;
    t = std::move(n);
    return true;
}

struct HComp {
    uint8_t id, hv, sx, sy, tq, tda;
    uint32_t pw, ph, pstride;
    int scan;  // the last scan that decodes it, -1: none
};

struct HScan {
    int ns = 0;
    int cidx[3];
    uint8_t tda[3];
    uint8_t qz[3][64];  // quantisation of each scan component, zig-zag order
    HTab tab[4];
    uint32_t restart = 0, mx = 0, my = 0, bpm = 0;
    uint8_t bcomp[JMAX_BPM], bsx[JMAX_BPM], bsy[JMAX_BPM];
    int64_t s_off = 0;                       // first byte in the job stream
    std::vector<uint32_t> seg_start, seg_end;  // byte ranges from s_off
};

struct HImage {
    uint32_t w = 0, h = 0;
    uint32_t w0 = 0, h0 = 0;  // the first frame header's size
    bool sof_seen = false, sos_seen = false;
    int ncomp = 0;
    HComp comp[3];
    std::vector<HScan> scans;
};

// Annex K tables (ITU-T T.81 K.3), loaded under PJPEG_MJPEG.
const uint8_t K_BITS[4][17] = {
    {0, 0, 1, 5, 1, 1, 1, 1, 1, 1, 0, 0, 0, 0, 0, 0, 0},
    {0, 0, 3, 1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 0, 0, 0, 0},
    {0, 0, 2, 1, 3, 3, 2, 4, 3, 5, 5, 4, 4, 0, 0, 1, 0x7d},
    {0, 0, 2, 1, 2, 4, 4, 3, 4, 7, 5, 4, 4, 0, 1, 2, 0x77}};
const uint8_t K_DCV[12] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11};
const uint8_t K_ACL[162] = {
    0x01, 0x02, 0x03, 0x00, 0x04, 0x11, 0x05, 0x12, 0x21, 0x31, 0x41, 0x06, 0x13, 0x51, 0x61, 0x07, 0x22, 0x71,
    0x14, 0x32, 0x81, 0x91, 0xa1, 0x08, 0x23, 0x42, 0xb1, 0xc1, 0x15, 0x52, 0xd1, 0xf0, 0x24, 0x33, 0x62, 0x72,
    0x82, 0x09, 0x0a, 0x16, 0x17, 0x18, 0x19, 0x1a, 0x25, 0x26, 0x27, 0x28, 0x29, 0x2a, 0x34, 0x35, 0x36, 0x37,
    0x38, 0x39, 0x3a, 0x43, 0x44, 0x45, 0x46, 0x47, 0x48, 0x49, 0x4a, 0x53, 0x54, 0x55, 0x56, 0x57, 0x58, 0x59,
    0x5a, 0x63, 0x64, 0x65, 0x66, 0x67, 0x68, 0x69, 0x6a, 0x73, 0x74, 0x75, 0x76, 0x77, 0x78, 0x79, 0x7a, 0x83,
    0x84, 0x85, 0x86, 0x87, 0x88, 0x89, 0x8a, 0x92, 0x93, 0x94, 0x95, 0x96, 0x97, 0x98, 0x99, 0x9a, 0xa2, 0xa3,
    0xa4, 0xa5, 0xa6, 0xa7, 0xa8, 0xa9, 0xaa, 0xb2, 0xb3, 0xb4, 0xb5, 0xb6, 0xb7, 0xb8, 0xb9, 0xba, 0xc2, 0xc3,
    0xc4, 0xc5, 0xc6, 0xc7, 0xc8, 0xc9, 0xca, 0xd2, 0xd3, 0xd4, 0xd5, 0xd6, 0xd7, 0xd8, 0xd9, 0xda, 0xe1, 0xe2,
    0xe3, 0xe4, 0xe5, 0xe6, 0xe7, 0xe8, 0xe9, 0xea, 0xf1, 0xf2, 0xf3, 0xf4, 0xf5, 0xf6, 0xf7, 0xf8, 0xf9, 0xfa};
const uint8_t K_ACC[162] = {
    0x00, 0x01, 0x02, 0x03, 0x11, 0x04, 0x05, 0x21, 0x31, 0x06, 0x12, 0x41, 0x51, 0x07, 0x61, 0x71, 0x13, 0x22,
    0x32, 0x81, 0x08, 0x14, 0x42, 0x91, 0xa1, 0xb1, 0xc1, 0x09, 0x23, 0x33, 0x52, 0xf0, 0x15, 0x62, 0x72, 0xd1,
    0x0a, 0x16, 0x24, 0x34, 0xe1, 0x25, 0xf1, 0x17, 0x18, 0x19, 0x1a, 0x26, 0x27, 0x28, 0x29, 0x2a, 0x35, 0x36,
    0x37, 0x38, 0x39, 0x3a, 0x43, 0x44, 0x45, 0x46, 0x47, 0x48, 0x49, 0x4a, 0x53, 0x54, 0x55, 0x56, 0x57, 0x58,
    0x59, 0x5a, 0x63, 0x64, 0x65, 0x66, 0x67, 0x68, 0x69, 0x6a, 0x73, 0x74, 0x75, 0x76, 0x77, 0x78, 0x79, 0x7a,
    0x82, 0x83, 0x84, 0x85, 0x86, 0x87, 0x88, 0x89, 0x8a, 0x92, 0x93, 0x94, 0x95, 0x96, 0x97, 0x98, 0x99, 0x9a,
    0xa2, 0xa3, 0xa4, 0xa5, 0xa6, 0xa7, 0xa8, 0xa9, 0xaa, 0xb2, 0xb3, 0xb4, 0xb5, 0xb6, 0xb7, 0xb8, 0xb9, 0xba,
    0xc2, 0xc3, 0xc4, 0xc5, 0xc6, 0xc7, 0xc8, 0xc9, 0xca, 0xd2, 0xd3, 0xd4, 0xd5, 0xd6, 0xd7, 0xd8, 0xd9, 0xda,
    0xe2, 0xe3, 0xe4, 0xe5, 0xe6, 0xe7, 0xe8, 0xe9, 0xea, 0xf2, 0xf3, 0xf4, 0xf5, 0xf6, 0xf7, 0xf8, 0xf9, 0xfa};

// Where a parse writes the scans' streams: `cap` bytes at p (over: it
// needed more; the count n keeps growing). Bytes gather in a small buffer
// and reach p by streaming stores, 4 KB at a time: the copy engine then
// reads them from memory instead of snooping them out of many cores'
// caches (which halved the copy rate when 16 threads parsed a batch).
struct JSink {
    uint8_t *p = nullptr;
    int64_t cap = 0, n = 0;
    bool over = false;
    int64_t flushed = 0;  // bytes already at p
    alignas(64) uint8_t buf[4096];
    void flush_full() {
        const int64_t k = n - flushed;  // == sizeof buf
        if (flushed + k <= cap) {
            uint8_t *d = p + flushed;
#ifdef JSINK_STREAM
            if (!((uintptr_t)d & 15)) {
                for (int64_t o = 0; o < k; o += 16)
                    _mm_stream_si128((__m128i *)(d + o), _mm_load_si128((const __m128i *)(buf + o)));
            } else {
                memcpy(d, buf, (size_t)k);
            }
#else
            memcpy(d, buf, (size_t)k);  // hosts without SSE2 streaming stores
#endif
        } else {
            over = true;
        }
        flushed = n;
    }
    void put(const uint8_t *b, int64_t k) {
        while (k > 0) {
            const int64_t room = (int64_t)sizeof buf - (n - flushed), t = k < room ? k : room;
            memcpy(buf + (n - flushed), b, (size_t)t);
            n += t;
            b += t;
            k -= t;
            if (n - flushed == (int64_t)sizeof buf) flush_full();
        }
    }
    void put1(uint8_t b) { put(&b, 1); }
    void fill(uint8_t b, int64_t k) {
        uint8_t t[64];
        memset(t, b, sizeof t);
        while (k > 0) {
            const int64_t c = k < 64 ? k : 64;
            put(t, c);
            k -= c;
        }
    }
    // writes what is left; the streaming stores are ordered before return
    void finish() {
        const int64_t k = n - flushed;
        if (k > 0) {
            if (flushed + k <= cap) memcpy(p + flushed, buf, (size_t)k);
            else over = true;
        }
        flushed = n;
#ifdef JSINK_STREAM
        _mm_sfence();
#endif
    }
};

// Appends the bytes of stream-position `from` on, as the reader sees them,
// up to `n` bytes, then JPAD 1-bytes: what a decode that runs past a
// scan's data reads next.
void append_tail(JSink *st, const uint8_t *in, int64_t len, int64_t from, int n) {
    if (!st) return;
    for (int64_t i = from; i < len && n > 0; n--) {
        uint8_t b = in[i++];
        if (b == 0xff && i < len && in[i] == 0) i++;
        st->put1(b);
    }
    st->fill(0xff, JPAD + ((4 - ((st->n + JPAD) & 3)) & 3));
}

// One scan (common/pjpeg.c:439-662): its header, then its bytes up to the
// next marker that is not a needed restart marker, cut into segments at
// the restart markers. `st` receives the stream (nullptr: headers only).
int parse_scan(HImage &im, HReader &r, const uint8_t q[4][64], const HTab tab[4], uint32_t restart, int &rst_next,
               JSink *st) {
    r.take(16);
    const int ns = (int)r.take(8);
    HScan sc;
    int found_idx[256];
    for (int i = 0; i < ns; i++) {
        const uint8_t id = (uint8_t)r.take(8);
        int f = -1;
        for (int j = 0; j < im.ncomp; j++)
            if (im.comp[j].id == id) { f = j; break; }
        if (f < 0) return PJPEG_ERR_SOS;
        im.comp[f].tda = (uint8_t)r.take(8);
        found_idx[i] = f;
    }
    const uint32_t ss = r.take(8), se = r.take(8), ah = r.take(8);
    if (ss != 0 || se != 63 || ah != 0) return PJPEG_ERR_SOS;
    // Not decodable here (the reference reads more scan components, writes
    // one component twice, or divides by a zero sampling factor): refused.
    if (ns > 3) return PJPEG_ERR_SOS;
    for (int i = 0; i < ns; i++)
        for (int j = 0; j < i; j++)
            if (found_idx[i] == found_idx[j]) return PJPEG_ERR_SOS;
    sc.ns = ns;
    int mw = 0, mh = 0, bpm = 0;
    for (int i = 0; i < ns; i++) {
        const HComp &c = im.comp[found_idx[i]];
        sc.cidx[i] = found_idx[i];
        sc.tda[i] = c.tda;
        mw = std::max(mw, c.sx * 8);
        mh = std::max(mh, c.sy * 8);
        bpm += c.sx * c.sy;
    }
    if (mw == 0 || mh == 0 || bpm > JMAX_BPM) return PJPEG_ERR_SOF;
    sc.mx = (im.w + mw - 1) / mw;
    sc.my = (im.h + mh - 1) / mh;
    sc.restart = restart;
    sc.bpm = (uint32_t)bpm;
    for (int i = 0, b = 0; i < ns; i++) {
        const HComp &c = im.comp[sc.cidx[i]];
        for (int y = 0; y < c.sy; y++)
            for (int x = 0; x < c.sx; x++, b++) {
                sc.bcomp[b] = (uint8_t)i;
                sc.bsx[b] = (uint8_t)x;
                sc.bsy[b] = (uint8_t)y;
            }
        memcpy(sc.qz[i], q[c.tq], 64);
    }
    const uint64_t nmcu = (uint64_t)sc.mx * sc.my;
    if (nmcu > 0) {
        for (int i = 0; i < ns; i++) {
            const HComp &c = im.comp[sc.cidx[i]];
            const int hd = c.tda >> 4, ha = 2 + (c.tda & 15);
            // table numbers past 3 index outside the reference's tables
            if (c.sx * c.sy && (hd > 3 || ha > 3 || !tab[hd].present || !tab[ha].present))
                return PJPEG_ERR_MISSING_DHT;
        }
    }
    for (int t = 0; t < 4; t++) sc.tab[t] = tab[t];
    const int scan_index = (int)im.scans.size();
    for (int i = 0; i < ns; i++) {
        HComp &c = im.comp[sc.cidx[i]];
        c.pw = sc.mx * c.sx * 8;
        c.ph = sc.my * c.sy * 8;
        c.pstride = (c.pw + 31) / 32 * 32;
        c.scan = scan_index;
    }
    if (nmcu == 0) {
        im.scans.push_back(std::move(sc));
        return PJPEG_OKAY;
    }
    // the scan's bytes
    const uint64_t need = restart ? (nmcu + restart - 1) / restart - 1 : 0;
    uint64_t nrst = 0;
    const uint8_t *in = r.in;
    const int64_t len = r.len;
    int64_t i = r.pos;
    if (st) sc.s_off = st->n;
    int64_t rel = 0;  // stream bytes of this scan so far
    sc.seg_start.push_back(0);
    while (i < len) {
        const uint8_t *f = (const uint8_t *)memchr(in + i, 0xff, (size_t)(len - i));
        const int64_t j = f ? f - in : len;
        if (st) st->put(in + i, j - i);
        rel += j - i;
        if (!f) { i = len; break; }
        if (j + 1 >= len) {
            if (st) st->put1(0xff);
            rel++;
            i = len;
            break;
        }
        const uint8_t m = in[j + 1];
        if (m == 0x00 || m == 0xff) {  // a stuffed FF, or a fill FF read as data
            if (st) st->put(in + j, 1);
            rel++;
            i = j + (m == 0 ? 2 : 1);
            continue;
        }
        if (m >= 0xd0 && m <= 0xd7 && nrst < need) {
            if (m != 0xd0 + rst_next) return PJPEG_ERR_RESET;
            rst_next = (rst_next + 1) & 7;
            nrst++;
            sc.seg_end.push_back((uint32_t)rel);
            if (st) { st->put1(0xff); st->put1(m); }
            rel += 2;
            sc.seg_start.push_back((uint32_t)rel);
            i = j + 2;
            continue;
        }
        if (m >= 0xd0 && m <= 0xd7) {  // a restart marker past the needed ones reads as data
            if (st) { st->put1(0xff); st->put1(m); }
            rel += 2;
            i = j + 2;
            continue;
        }
        i = j;  // the next marker
        break;
    }
    if (nrst < need) return PJPEG_ERR_RESET;
    sc.seg_end.push_back((uint32_t)rel);
    append_tail(st, in, len, i, 16);
    r.pos = i;
    r.avail = 0;
    im.scans.push_back(std::move(sc));
    return PJPEG_OKAY;
}

// The marker walk (common/pjpeg.c:246-687). `st` receives the scans'
// streams (their bytes mean nothing after an error); without it the walk
// stops at the first scan, having read the frame header.
int parse_image(const uint8_t *buf, int64_t len, uint32_t flags, HImage &im, JSink *st) {
    const int64_t st0 = 0;
    uint8_t q[4][64];
    memset(q, 0, sizeof(q));
    HTab tab[4];
    if (flags & PJPEG_MJPEG) {
        const uint8_t *vals[4] = {K_DCV, K_DCV, K_ACL, K_ACC};
        for (int t = 0; t < 4; t++) htab_define(tab[t], K_BITS[t], vals[t]);
    }
    uint32_t restart = 0;
    int rst_next = 0;
    HReader r{buf, 0, len};
    int e = PJPEG_OKAY;
    while (e == PJPEG_OKAY && r.more()) {
        r.avail -= r.avail & 7;
        while (r.take(8) != 0xff) {}
        const uint8_t m = (uint8_t)r.take(8);
        switch (m) {
        case 0xd8:
            break;
        case 0xdb: {
            const int n = (int)r.take(16);
            if ((n - 2) % 65 != 0) { e = PJPEG_ERR_DQT; break; }
            for (int o = 0; o < n - 2 && e == PJPEG_OKAY; o += 65) {
                const uint8_t pq = (uint8_t)r.take(8);
                if ((pq & 0xf0) || (pq & 15) >= 4) { e = PJPEG_ERR_DQT; break; }
                for (int k = 0; k < 64; k++) q[pq & 3][k] = (uint8_t)r.take(8);
            }
            break;
        }
        case 0xc0: {
            r.take(16);
            if (r.take(8) != 8) { e = PJPEG_ERR_SOF; break; }
            im.h = r.take(16);
            im.w = r.take(16);
            if (!im.sof_seen) {
                im.sof_seen = true;
                im.w0 = im.w;
                im.h0 = im.h;
            }
            const int nf = (int)r.take(8);
            if (nf < 1 || nf > 3) { e = PJPEG_ERR_SOF; break; }
            im.ncomp = nf;
            im.scans.clear();
            for (int i = 0; i < nf && e == PJPEG_OKAY; i++) {
                HComp &c = im.comp[i];
                c = HComp{};
                c.id = (uint8_t)r.take(8);
                c.hv = (uint8_t)r.take(8);
                c.sx = c.hv >> 4;
                c.sy = c.hv & 15;
                c.tq = (uint8_t)r.take(8);
                c.scan = -1;
                // table numbers past 3 index outside the reference's tables
                if (c.tq > 3) e = PJPEG_ERR_SOF;
            }
            break;
        }
        case 0xc1: case 0xc2: case 0xc3: case 0xc5: case 0xc6: case 0xc7: case 0xc8:
        case 0xc9: case 0xca: case 0xcb: case 0xcd: case 0xce: case 0xcf:
            e = PJEPG_ERR_UNSUPPORTED;
            break;
        case 0xc4: {
            uint16_t left = (uint16_t)(r.take(16) - 2);
            while (left > 0 && e == PJPEG_OKAY) {
                const uint8_t tcth = (uint8_t)r.take(8);
                left--;
                const int tc = tcth >> 4, th = tcth & 15;
                if (tc >= 2 || th >= 2) { e = PJPEG_ERR_DHT; break; }
                uint8_t cnt[17];
                cnt[0] = 0;
                int total = 0;
                for (int l = 1; l <= 16; l++) {
                    cnt[l] = (uint8_t)r.take(8);
                    left -= cnt[l];
                    total += cnt[l];
                }
                left -= 16;
                std::vector<uint8_t> vals((size_t)total);
                for (int k = 0; k < total; k++) vals[k] = (uint8_t)r.take(8);
                if (!htab_define(tab[tc * 2 + th], cnt, vals.data())) e = PJPEG_ERR_DHT;
            }
            break;
        }
        case 0xda:
            if (!st) {
                im.sos_seen = true;
                return im.ncomp ? PJPEG_OKAY : PJPEG_ERR_SOS;
            }
            e = parse_scan(im, r, q, tab, restart, rst_next, st);
            break;
        case 0xd9:
            return PJPEG_OKAY;
        case 0xdd:
            if (r.take(16) != 4) { e = PJPEG_ERR_DRI; break; }
            restart = r.take(16);
            break;
        default: {  // APPn, COM and anything unknown: skipped by length
            const int n = (int)r.take(16);
            // a length below 2 moves the reference's unsigned position past the end
            r.pos = n < 2 ? r.len : r.pos + (n - 2);
            break;
        }
        }
    }
    (void)st0;
    return e;
}

}  // namespace

// ---------------------------------------------------------------------
// Host: decode jobs.

namespace {

constexpr int64_t JMAX_STREAM = (int64_t)1 << 28;  // bytes per job (bit positions stay below 2^31)

struct HOut {           // a plane copied to the host after the decode
    size_t dev_off;     // in the arena's plane staging
    int64_t dev_stride;
    uint8_t *host;
    int64_t host_stride;
    uint32_t w, h;
};

struct HJob {
    int64_t stream_n = 0;                 // stream bytes (at the staging's start, or at stream_src)
    const uint8_t *stream_src = nullptr;  // copied to the staging's start by run_job
    std::vector<JTab> tabs;
    std::vector<uint8_t> syms;
    std::vector<JScanDev> scans;
    std::vector<JSegDev> segs;
    std::vector<uint32_t> sub_seg;
    std::vector<JPlaneDev> planes;
    std::vector<size_t> plane_stage;  // per plane: staging offset, or SIZE_MAX (written in place)
    std::vector<HOut> outs;
    size_t staging = 0;
    uint32_t max_seg_subs = 0;
    uint32_t nblocks = 0;  // blocks of the planes written
    uint32_t sub_bits = 512, back_bits = 1024;
    std::vector<int> scan_image;    // per scan: the index of its image in the call
    std::vector<uint32_t> seg_end;  // per segment after the decode: the bit its last block ends at
};

// The reference's restart check (common/pjpeg.c:494-518): after a
// segment's last block it reads on from the next byte boundary to the
// first FF, which must begin the expected restart marker; a damaged
// segment whose decode ends elsewhere fails there with PJPEG_ERR_RESET.
// Returns, per image of the call, whether one of its segments fails.
std::vector<char> restart_failures(const HJob &J, const uint8_t *stream, int nimages) {
    std::vector<char> bad((size_t)nimages, 0);
    for (size_t g = 0; g + 1 < J.segs.size(); g++) {
        const JSegDev &G = J.segs[g];
        if (J.segs[g + 1].scan != G.scan) continue;  // a scan's last segment ends at no marker
        const uint32_t e = J.seg_end[g];
        const uint64_t b0 = ((uint64_t)e + 7) / 8, m = G.end / 8;  // m: the marker's FF
        const bool ok = e != 0xffffffffu && b0 <= m && !memchr(stream + b0, 0xff, (size_t)(m - b0));
        if (!ok) bad[(size_t)J.scan_image[G.scan]] = 1;
    }
    return bad;
}

JTab make_tab(const HTab &t, std::vector<uint8_t> &pool) {
    JTab d;
    memset(&d, 0, sizeof d);
    const uint32_t base = (uint32_t)pool.size();
    pool.insert(pool.end(), t.syms.begin(), t.syms.end());
    d.nrun = (uint32_t)t.runs.size();
    for (size_t r = 0; r < t.runs.size(); r++) {
        d.rend[r] = t.runs[r].end;
        d.rorigin[r] = t.runs[r].origin;
        d.rsym[r] = base + t.runs[r].sym0;
        d.rlen[r] = (uint8_t)t.runs[r].len;
    }
    d.r0 = d.nrun;
    size_t r = 0;
    for (uint32_t p = 0; p < 512; p++) {
        const uint32_t lo = p << 7, hi = lo + 127;
        while (r < t.runs.size() && t.runs[r].end <= lo) r++;
        bool hit = false;
        if (r < t.runs.size() && t.runs[r].start <= lo && hi < t.runs[r].end && t.runs[r].len <= 9) {
            const HRun &u = t.runs[r];
            const uint32_t k = (lo - u.origin) >> (16 - u.len);
            if (k == ((hi - u.origin) >> (16 - u.len))) {
                d.lut[p] = (uint16_t)((u.len << 8) | t.syms[u.sym0 + k]);
                hit = true;
            }
        }
        if (!hit && r < d.r0) d.r0 = (uint32_t)r;
    }
    return d;
}

// Adds the scans of a parsed image to the job. want: which frame
// components to write (bit c); place(c, P) fills the output of component
// c (pointer, stride, clip) and returns its staging size (0: in place).
template <class Place>
void add_image(HJob &J, const HImage &im, int img, int64_t s_base, uint32_t sub_bits, unsigned want, Place place) {
    int plane_of[3] = {-1, -1, -1};
    for (int c = 0; c < im.ncomp; c++) {
        if (!(want & (1u << c)) || im.comp[c].scan < 0) continue;
        const HComp &hc = im.comp[c];
        const HScan &sc = im.scans[hc.scan];
        JPlaneDev P;
        memset(&P, 0, sizeof P);
        P.sx = hc.sx;
        P.sy = hc.sy;
        P.mcus_x = sc.mx;
        P.blk0 = J.nblocks;
        P.nblk = sc.mx * sc.my * hc.sx * hc.sy;
        J.nblocks += P.nblk;
        for (int i = 0; i < sc.ns; i++)
            if (sc.cidx[i] == c)
                for (int k = 0; k < 64; k++) P.q[H_ZIG[k]] = sc.qz[i][k];
        plane_of[c] = (int)J.planes.size();
        size_t stage = place(c, P);
        if (stage) {
            J.plane_stage.push_back(J.staging);
            J.staging += (stage + 255) / 256 * 256;
        } else {
            J.plane_stage.push_back(SIZE_MAX);
        }
        J.planes.push_back(P);
    }
    for (size_t s = 0; s < im.scans.size(); s++) {
        const HScan &sc = im.scans[s];
        const uint64_t nmcu = (uint64_t)sc.mx * sc.my;
        if (nmcu == 0) continue;
        JScanDev D;
        memset(&D, 0, sizeof D);
        D.tab0 = (uint32_t)J.tabs.size();
        for (int t = 0; t < 4; t++) J.tabs.push_back(make_tab(sc.tab[t], J.syms));
        D.mcus_x = sc.mx;
        D.nmcu = (uint32_t)nmcu;
        D.restart = sc.restart;
        D.sub0 = (uint32_t)J.sub_seg.size();
        D.bpm = sc.bpm;
        D.ns = (uint32_t)sc.ns;
        memcpy(D.bcomp, sc.bcomp, sizeof D.bcomp);
        memcpy(D.bsx, sc.bsx, sizeof D.bsx);
        memcpy(D.bsy, sc.bsy, sizeof D.bsy);
        for (uint32_t b = 0; b < sc.bpm; b++) {
            D.bcanon[b] = (uint8_t)b;
            for (uint32_t c = 0; c < b; c++) {
                bool same = true;
                for (uint32_t k = 0; k < sc.bpm && same; k++) {
                    const int u = sc.bcomp[(b + k) % sc.bpm], v = sc.bcomp[(c + k) % sc.bpm];
                    same = sc.tda[u] == sc.tda[v];
                }
                if (same) {
                    D.bcanon[b] = (uint8_t)c;
                    break;
                }
            }
        }
        for (int i = 0; i < sc.ns; i++) {
            D.dc[i] = (uint8_t)(sc.tda[i] >> 4);
            D.ac[i] = (uint8_t)(2 + (sc.tda[i] & 15));
            // a component with no blocks per MCU never looks its tables up
            if (D.dc[i] > 3) D.dc[i] = 0;
            if (D.ac[i] > 3) D.ac[i] = 2;
            const int c = sc.cidx[i];
            D.plane[i] = (im.comp[c].scan == (int)s) ? plane_of[c] : -1;
        }
        for (int i = sc.ns; i < 3; i++) D.plane[i] = -1;
        const uint32_t scan_id = (uint32_t)J.scans.size();
        J.scans.push_back(D);
        J.scan_image.push_back(img);
        const uint32_t per = sc.restart ? sc.restart : (uint32_t)nmcu;
        for (size_t g = 0; g < sc.seg_start.size(); g++) {
            JSegDev G;
            G.scan = scan_id;
            G.start = (uint32_t)((s_base + sc.s_off + sc.seg_start[g]) * 8);
            G.end = (uint32_t)((s_base + sc.s_off + sc.seg_end[g]) * 8);
            const uint32_t bits = G.end - G.start;
            G.nsub = std::max(1u, (bits + sub_bits - 1) / sub_bits);
            G.sub0 = (uint32_t)J.sub_seg.size();
            const uint64_t m0 = (uint64_t)g * per;
            G.blk0 = (uint32_t)(m0 * sc.bpm);
            G.nblk = (uint32_t)(std::min<uint64_t>(per, nmcu - m0) * sc.bpm);
            J.sub_seg.insert(J.sub_seg.end(), G.nsub, (uint32_t)J.segs.size());
            J.max_seg_subs = std::max(J.max_seg_subs, G.nsub);
            J.segs.push_back(G);
        }
    }
}

}  // namespace

// Host threads that parse a batch's images, kept for the decoder's life
// (starting threads for every call cost more than the parse of a batch).
struct JPool {
    std::vector<std::thread> th;
    std::mutex m;
    std::condition_variable go, fin;
    const std::function<void(int)> *fn = nullptr;
    int n = 0, busy = 0;
    uint64_t gen = 0;
    bool stop = false;
    std::atomic<int> next{0};
    void start(int nthreads) {
        for (int t = 0; t < nthreads; t++)
            th.emplace_back([this] {
                uint64_t seen = 0;
                while (true) {
                    const std::function<void(int)> *f;
                    int cnt;
                    {
                        std::unique_lock<std::mutex> lk(m);
                        go.wait(lk, [&] { return stop || gen != seen; });
                        if (stop) return;
                        seen = gen;
                        f = fn;
                        cnt = n;
                    }
                    for (int k; (k = next.fetch_add(1)) < cnt;) (*f)(k);
                    std::lock_guard<std::mutex> lk(m);
                    if (--busy == 0) fin.notify_all();
                }
            });
    }
    // runs f(0 .. n-1) on the workers and the calling thread
    void run(int cnt, const std::function<void(int)> &f) {
        {
            std::lock_guard<std::mutex> lk(m);
            fn = &f;
            n = cnt;
            next = 0;
            busy = (int)th.size();
            gen++;
        }
        go.notify_all();
        for (int k; (k = next.fetch_add(1)) < cnt;) f(k);
        std::unique_lock<std::mutex> lk(m);
        fin.wait(lk, [&] { return busy == 0; });
    }
    ~JPool() {
        {
            std::lock_guard<std::mutex> lk(m);
            stop = true;
        }
        go.notify_all();
        for (auto &t : th) t.join();
    }
};

struct at_jpeg {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[5] = {};
    uint8_t *h_stage = nullptr;
    size_t h_cap = 0;
    uint8_t *d_arena = nullptr;
    size_t d_cap = 0;
    uint32_t sub_bits = 0;   // 0: chosen per job (jsub_for)
    uint32_t back_bits = 0;  // 0: chosen per job
    int threads = 0;  // host threads parsing a batch (0: up to 16)
    JPool *pool = nullptr;
    int pool_threads = 0;
    int grid_max = 0;
    double stats[10] = {};
    std::mutex mu;
};

namespace {

bool jcheck(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return true;
    fprintf(stderr, "at_jpeg: %s: %s\n", what, cudaGetErrorString(e));
    return false;
}

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

// Page-locked staging of at least `need` bytes, its first `keep` bytes kept.
bool grow_host(at_jpeg *d, size_t need, size_t keep) {
    if (need <= d->h_cap) return true;
    uint8_t *n = nullptr;
    const size_t cap = need + need / 4;
    if (!jcheck(cudaMallocHost(&n, cap), "cudaMallocHost")) return false;
    if (keep && d->h_stage) memcpy(n, d->h_stage, keep);
    if (d->h_stage) cudaFreeHost(d->h_stage);
    d->h_stage = n;
    d->h_cap = cap;
    return true;
}

// Runs a job: one copy in, the sync pass, the write pass, the copies out.
// Returns 0, or -1 on a CUDA error.
int run_job(at_jpeg *d, HJob &J, double parse_ms) {
    const uint32_t nsub = (uint32_t)J.sub_seg.size();
    d->stats[0] = parse_ms;
    d->stats[5] = nsub;
    d->stats[6] = 0;
    d->stats[7] = (double)J.stream_n;
    for (int k = 1; k < 5; k++) d->stats[k] = 0;
    if (nsub == 0 && J.outs.empty()) return 0;
    // packed inputs: the stream first
    size_t off = 0;
    auto put = [&](size_t bytes) { size_t o = off; off = align256(off + bytes); return o; };
    const size_t o_stream = put((size_t)J.stream_n + 32);
    const size_t o_tabs = put(J.tabs.size() * sizeof(JTab));
    const size_t o_syms = put(J.syms.size() + 16);
    const size_t o_scans = put(J.scans.size() * sizeof(JScanDev));
    const size_t o_segs = put(J.segs.size() * sizeof(JSegDev));
    const size_t o_subs = put((size_t)nsub * 4);
    const size_t o_planes = put(J.planes.size() * sizeof(JPlaneDev));
    const size_t in_bytes = off;
    // scratch
    const uint32_t per_cta_min = JSYNC_THREADS;
    uint32_t grid = std::max(1u, std::min<uint32_t>((nsub + per_cta_min - 1) / per_cta_min, (uint32_t)d->grid_max));
    const uint32_t per = (nsub + grid - 1) / grid;
    grid = nsub ? (nsub + per - 1) / per : 1;
    const uint32_t max_passes = J.max_seg_subs + 1;
    const size_t o_exit = put((size_t)nsub * 8);
    const size_t o_used = put((size_t)nsub * 8);
    const size_t o_cnt = put((size_t)nsub * 16);
    const size_t o_excl = put((size_t)nsub * 16);
    const size_t o_tot = put((size_t)grid * 16);
    const size_t o_stuck = put(J.segs.size() * 4);
    const size_t o_endbit = put(J.segs.size() * 4);
    const size_t o_zero = off;  // zeroed: barrier, error, pass flags
    const size_t o_bar = put(8);
    const size_t o_err = put(4);
    const size_t o_chg = put((size_t)(max_passes + 2) * 4);
    const size_t zero_bytes = off - o_zero;
    const size_t o_stage = put(J.staging);
    const size_t o_coef = put((size_t)J.nblocks * 128);
    const size_t o_dc = put((size_t)J.nblocks * 4);
    if (off > d->d_cap) {
        if (d->d_arena) cudaFree(d->d_arena);
        d->d_arena = nullptr;
        d->d_cap = 0;
        if (!jcheck(cudaMalloc(&d->d_arena, off + off / 4), "cudaMalloc")) return -1;
        d->d_cap = off + off / 4;
    }
    if (!grow_host(d, in_bytes + 64 + J.segs.size() * 4, J.stream_src ? 0 : (size_t)J.stream_n)) return -1;
    uint8_t *D = d->d_arena, *H = d->h_stage;
    for (size_t p = 0; p < J.planes.size(); p++)
        if (J.plane_stage[p] != SIZE_MAX) J.planes[p].out = D + o_stage + J.plane_stage[p];
    if (J.stream_src) memcpy(H + o_stream, J.stream_src, (size_t)J.stream_n);
    memset(H + o_stream + J.stream_n, 0xff, 32);
    if (!J.tabs.empty()) memcpy(H + o_tabs, J.tabs.data(), J.tabs.size() * sizeof(JTab));
    if (!J.syms.empty()) memcpy(H + o_syms, J.syms.data(), J.syms.size());
    if (!J.scans.empty()) memcpy(H + o_scans, J.scans.data(), J.scans.size() * sizeof(JScanDev));
    if (!J.segs.empty()) memcpy(H + o_segs, J.segs.data(), J.segs.size() * sizeof(JSegDev));
    if (nsub) memcpy(H + o_subs, J.sub_seg.data(), (size_t)nsub * 4);
    if (!J.planes.empty()) memcpy(H + o_planes, J.planes.data(), J.planes.size() * sizeof(JPlaneDev));
    cudaStream_t s = d->stream;
    int32_t *hres = (int32_t *)(H + in_bytes);  // error word and pass count read back
    bool ok = jcheck(cudaEventRecord(d->ev[0], s), "event");
    ok = ok && jcheck(cudaMemcpyAsync(D, H, in_bytes, cudaMemcpyHostToDevice, s), "copy in");
    ok = ok && jcheck(cudaMemsetAsync(D + o_zero, 0, zero_bytes, s), "memset");
    ok = ok && jcheck(cudaMemsetAsync(D + o_stuck, 0xff, J.segs.size() * 4, s), "memset");
    ok = ok && jcheck(cudaMemsetAsync(D + o_endbit, 0xff, J.segs.size() * 4, s), "memset");
    ok = ok && jcheck(cudaEventRecord(d->ev[1], s), "event");
    if (ok && nsub) {
        JJob JJ;
        JJ.stream = (const uint32_t *)(D + o_stream);
        JJ.tabs = (const JTab *)(D + o_tabs);
        JJ.syms = D + o_syms;
        JJ.scans = (const JScanDev *)(D + o_scans);
        JJ.segs = (const JSegDev *)(D + o_segs);
        JJ.sub_seg = (const uint32_t *)(D + o_subs);
        JJ.planes = (const JPlaneDev *)(D + o_planes);
        JJ.coef = (int16_t *)(D + o_coef);
        JJ.dc = (int32_t *)(D + o_dc);
        JJ.nplanes = (uint32_t)J.planes.size();
        JJ.nblocks = J.nblocks;
        JJ.nsub = nsub;
        JJ.sub_bits = J.sub_bits;
        JJ.max_passes = max_passes;
        JJ.exitst = (unsigned long long *)(D + o_exit);
        JJ.used = (unsigned long long *)(D + o_used);
        JJ.cnt = (uint32_t *)(D + o_cnt);
        JJ.excl = (uint32_t *)(D + o_excl);
        JJ.totals = (uint32_t *)(D + o_tot);
        JJ.seg_stuck = (uint32_t *)(D + o_stuck);
        JJ.seg_endbit = (uint32_t *)(D + o_endbit);
        JJ.back_bits = J.back_bits;
        JJ.bar = (unsigned int *)(D + o_bar);
        JJ.changed = (int *)(D + o_chg);
        JJ.err = (int *)(D + o_err);
        uint32_t per_arg = per;
        void *args[] = {&JJ, &per_arg};
        ok = jcheck(cudaLaunchCooperativeKernel((const void *)k_jpeg_sync, dim3(grid), dim3(JSYNC_THREADS), args, 0, s),
                    "sync pass");
        ok = ok && jcheck(cudaEventRecord(d->ev[2], s), "event");
        if (ok) {
            k_jpeg_write<<<(nsub + JWRITE_THREADS - 1) / JWRITE_THREADS, JWRITE_THREADS, 0, s>>>(JJ);
            ok = jcheck(cudaGetLastError(), "write pass");
            constexpr uint32_t per_cta = JIDCT_THREADS / 8;
            if (ok && J.nblocks) {
                k_jpeg_idct<<<(J.nblocks + per_cta - 1) / per_cta, JIDCT_THREADS, 0, s>>>(JJ);
                ok = jcheck(cudaGetLastError(), "IDCT pass");
            }
        }
        ok = ok && jcheck(cudaMemcpyAsync(hres, D + o_err, 4, cudaMemcpyDeviceToHost, s), "copy out");
        ok = ok && jcheck(cudaMemcpyAsync(hres + 1, D + o_chg, 4, cudaMemcpyDeviceToHost, s), "copy out");
        ok = ok && jcheck(cudaMemcpyAsync(hres + 2, D + o_chg + 4 * (size_t)(max_passes + 1), 4,
                                          cudaMemcpyDeviceToHost, s),
                          "copy out");
        ok = ok && jcheck(cudaMemcpyAsync(hres + 16, D + o_endbit, J.segs.size() * 4, cudaMemcpyDeviceToHost, s),
                          "copy out");
    } else if (ok) {
        ok = jcheck(cudaEventRecord(d->ev[2], s), "event");
        hres[0] = hres[1] = hres[2] = 0;
    }
    ok = ok && jcheck(cudaEventRecord(d->ev[3], s), "event");
    for (const HOut &o : J.outs) {
        if (!ok) break;
        ok = jcheck(cudaMemcpy2DAsync(o.host, (size_t)o.host_stride, D + o_stage + o.dev_off, (size_t)o.dev_stride,
                                      o.w, o.h, cudaMemcpyDeviceToHost, s),
                    "copy out");
    }
    ok = ok && jcheck(cudaEventRecord(d->ev[4], s), "event");
    ok = ok && jcheck(cudaStreamSynchronize(s), "synchronize");
    if (!ok) return -1;
    if (nsub && hres[0]) {
        fprintf(stderr, "at_jpeg: the sync pass gave up waiting at a grid barrier\n");
        return -1;
    }
    float ms;
    for (int k = 1; k < 5; k++)
        if (cudaEventElapsedTime(&ms, d->ev[k - 1], d->ev[k]) == cudaSuccess) d->stats[k] = ms;
    J.seg_end.assign((const uint32_t *)(hres + 16), (const uint32_t *)(hres + 16) + J.segs.size());
    d->stats[6] = nsub ? hres[1] : 0;
    d->stats[8] = nsub ? hres[2] : 0;
    return 0;
}

double now_ms() {
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return t.tv_sec * 1e3 + t.tv_nsec * 1e-6;
}

}  // namespace

// ---------------------------------------------------------------------
// C ABI (apriltag_fast.h) and the reference's pjpeg.h calls.

extern "C" {

at_jpeg *at_jpeg_create(void) {
    at_jpeg *d = new at_jpeg();
    bool ok = jcheck(cudaGetDevice(&d->device), "cudaGetDevice");
    ok = ok && jcheck(cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    for (int k = 0; ok && k < 5; k++) ok = jcheck(cudaEventCreate(&d->ev[k]), "cudaEventCreate");
    int occ = 0, nsm = 0;
    ok = ok && jcheck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_jpeg_sync, JSYNC_THREADS, 0), "occupancy");
    ok = ok && jcheck(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, d->device), "attribute");
    d->grid_max = occ * nsm;
    if (!ok || d->grid_max <= 0) {
        at_jpeg_destroy(d);
        return nullptr;
    }
    return d;
}

void at_jpeg_destroy(at_jpeg *d) {
    if (!d) return;
    if (d->stream) cudaStreamSynchronize(d->stream);
    for (int k = 0; k < 5; k++)
        if (d->ev[k]) cudaEventDestroy(d->ev[k]);
    if (d->stream) cudaStreamDestroy(d->stream);
    if (d->d_arena) cudaFree(d->d_arena);
    if (d->h_stage) cudaFreeHost(d->h_stage);
    delete d->pool;
    delete d;
}

// The errors a gray decode reports beyond the reference's walk: a first
// component that no scan decodes, or whose plane is smaller than the image
// (the reference's pjpeg_to_u8_baseline reads past its planes there).
static int gray_check(const HImage &im) {
    if (im.ncomp < 1 || im.comp[0].scan < 0) return PJPEG_ERR_SOS;
    if (im.comp[0].pw < im.w || im.comp[0].ph < im.h) return PJPEG_ERR_SOF;
    return PJPEG_OKAY;
}

int at_jpeg_info(const uint8_t *buf, int64_t len, uint32_t flags, int32_t *width, int32_t *height,
                 int32_t *ncomponents) {
    if (!buf || len < 0) return PJPEG_ERR_FILE;
    HImage im;
    int e = parse_image(buf, len, flags, im, nullptr);
    if (e == PJPEG_OKAY && !im.sos_seen) e = PJPEG_ERR_SOS;  // no scan: nothing to decode
    if (width) *width = e ? 0 : (int32_t)im.w0;
    if (height) *height = e ? 0 : (int32_t)im.h0;
    if (ncomponents) *ncomponents = e ? 0 : im.ncomp;
    return e;
}

// The gray decode of images [a, b) as one job. Each image is parsed on a
// host thread straight into the page-locked staging, at a place sized
// from its file; an image that needs more (many scans) is parsed again at
// the end.
static int decode_group(at_jpeg *dec, int32_t a, int32_t b, const uint8_t *const *bufs, const int64_t *lens,
                        uint32_t flags, uint8_t *const *dst, const int64_t *strides, int32_t on_device,
                        int32_t *errors, const std::vector<int64_t> &cap) {
    const double t0 = now_ms();
    const int m = b - a;
    std::vector<int64_t> base(m + 1, 0);
    for (int k = 0; k < m; k++) base[k + 1] = base[k] + cap[a + k];
    if (!grow_host(dec, (size_t)base[m] + 64, 0)) return -1;
    std::vector<HImage> ims(m);
    std::vector<int> errs(m);
    std::vector<int64_t> used(m);
    auto parse_one = [&](int k, uint8_t *at, int64_t room) {
        const int32_t i = a + k;
        ims[k] = HImage();
        JSink sk;
        sk.p = at;
        sk.cap = room;
        int e = (!bufs[i] || lens[i] < 0 || lens[i] > JMAX_STREAM)
                    ? PJPEG_ERR_FILE
                    : parse_image(bufs[i], lens[i], flags, ims[k], &sk);
        sk.finish();
        if (e == PJPEG_OKAY && sk.over) e = -2;  // needs more room
        if (e == PJPEG_OKAY) e = gray_check(ims[k]);
        // the frame must be the size at_jpeg_info reports (its first header)
        if (e == PJPEG_OKAY && (ims[k].w != ims[k].w0 || ims[k].h != ims[k].h0)) e = PJPEG_ERR_SOF;
        errs[k] = e;
        used[k] = sk.n;
    };
    const int nt = std::min<int>(
        m, dec->threads > 0 ? dec->threads : std::min<int>(16, (int)std::max(1u, std::thread::hardware_concurrency())));
    if (nt <= 1) {
        for (int k = 0; k < m; k++) parse_one(k, dec->h_stage + base[k], cap[a + k]);
    } else {
        if (!dec->pool || dec->pool_threads != nt - 1) {
            delete dec->pool;
            dec->pool = new JPool();
            dec->pool->start(nt - 1);
            dec->pool_threads = nt - 1;
        }
        const std::function<void(int)> f = [&](int k) { parse_one(k, dec->h_stage + base[k], cap[a + k]); };
        dec->pool->run(m, f);
    }
    int64_t tail = base[m];
    for (int k = 0; k < m; k++) {
        if (errs[k] != -2) continue;
        const int64_t need = (used[k] + 63) / 64 * 64;
        if (!grow_host(dec, (size_t)(tail + need) + 64, (size_t)tail)) return -1;
        parse_one(k, dec->h_stage + tail, need);
        base[k] = tail;
        tail += need;
    }
    HJob J;
    J.stream_n = tail;
    int64_t total = 0;
    for (int k = 0; k < m; k++)
        if (!errs[k]) total += used[k];
    J.sub_bits = dec->sub_bits ? dec->sub_bits : jsub_for(total);
    J.back_bits = dec->back_bits ? dec->back_bits : std::max(512u, J.sub_bits);
    int failed = 0;
    for (int k = 0; k < m; k++) {
        const int32_t i = a + k;
        errors[i] = errs[k] == -2 ? PJPEG_ERR_FILE : errs[k];
        if (errors[i]) {
            failed++;
            continue;
        }
        const HImage &im = ims[k];
        add_image(J, im, k, base[k], J.sub_bits, 1u, [&](int, JPlaneDev &P) -> size_t {
            P.ow = im.w;
            P.oh = im.h;
            if (on_device) {
                P.out = dst[i];
                P.stride = strides[i];
                return 0;
            }
            P.stride = (im.w + 15) / 16 * 16;
            if ((size_t)im.w * im.h) J.outs.push_back(HOut{J.staging, P.stride, dst[i], strides[i], im.w, im.h});
            return (size_t)P.stride * im.h + 16;
        });
    }
    if (run_job(dec, J, now_ms() - t0) != 0) return -1;
    const std::vector<char> bad = restart_failures(J, dec->h_stage, m);
    for (int k = 0; k < m; k++)
        if (bad[k] && errors[a + k] == PJPEG_OKAY) {
            errors[a + k] = PJPEG_ERR_RESET;  // its frame's pixels mean nothing
            failed++;
        }
    return failed;
}

int at_jpeg_decode_gray(at_jpeg *dec, int32_t n, const uint8_t *const *bufs, const int64_t *lens, uint32_t flags,
                        uint8_t *const *dst, const int64_t *strides, int32_t on_device, int32_t *errors) {
    if (!dec || n < 0 || (n && (!bufs || !lens || !dst || !strides || !errors))) return -1;
    std::lock_guard<std::mutex> lk(dec->mu);
    if (!jcheck(cudaSetDevice(dec->device), "cudaSetDevice")) return -1;
    // room for each image's stream: its file and the tails of a few scans
    std::vector<int64_t> cap(n);
    for (int32_t i = 0; i < n; i++) cap[i] = (std::max<int64_t>(0, std::min(lens[i], JMAX_STREAM)) + 1024 + 63) / 64 * 64;
    int failed = 0;
    for (int32_t i = 0; i < n;) {
        int32_t j = i;
        int64_t tot = 0;
        while (j < n && (j == i || tot + cap[j] <= JMAX_STREAM)) tot += cap[j++];
        const int r = decode_group(dec, i, j, bufs, lens, flags, dst, strides, on_device, errors, cap);
        if (r < 0) return -1;
        failed += r;
        i = j;
    }
    return failed;
}

int at_jpeg_last_stats(const at_jpeg *dec, double *out10) {
    if (!dec || !out10) return 1;
    memcpy(out10, dec->stats, sizeof dec->stats);
    return 0;
}

int at_jpeg_set_run_in(at_jpeg *dec, int32_t bits) {
    if (!dec || bits < 0 || bits > (1 << 20)) return 1;
    dec->back_bits = (uint32_t)bits;
    return 0;
}

int at_jpeg_set_threads(at_jpeg *dec, int32_t threads) {
    if (!dec || threads < 0 || threads > 256) return 1;
    dec->threads = threads;
    return 0;
}

int at_jpeg_set_sub_bits(at_jpeg *dec, int32_t bits) {
    if (!dec || (bits && (bits < 64 || bits > 65536 || bits % 32))) return 1;
    dec->sub_bits = (uint32_t)bits;
    return 0;
}

// ---- pjpeg.h (common/pjpeg.c:689-894 of the reference) ----

static at_jpeg *g_pjpeg_dec = nullptr;
static std::mutex g_pjpeg_mu;

pjpeg_t *pjpeg_create_from_buffer(uint8_t *buf, int buflen, uint32_t flags, int *error) {
    HImage im;
    HJob J;
    const double t0 = now_ms();
    std::vector<uint8_t> sbuf(buf && buflen > 0 ? (size_t)buflen + 1024 : 1024);
    JSink sk;
    sk.p = sbuf.data();
    sk.cap = (int64_t)sbuf.size();
    int e = buf && buflen >= 0 ? parse_image(buf, buflen, flags, im, &sk) : PJPEG_ERR_FILE;
    sk.finish();
    if (e == PJPEG_OKAY && sk.over) {  // many scans: again with the room it needed
        sbuf.assign((size_t)sk.n + 64, 0);
        im = HImage();
        sk = JSink();
        sk.p = sbuf.data();
        sk.cap = (int64_t)sbuf.size();
        e = parse_image(buf, buflen, flags, im, &sk);
        sk.finish();
    }
    if (error) *error = e;
    if (e) return nullptr;
    J.stream_src = sbuf.data();
    J.stream_n = sk.n;
    pjpeg_t *pj = (pjpeg_t *)calloc(1, sizeof(pjpeg_t));
    pj->width = im.w;
    pj->height = im.h;
    pj->ncomponents = im.ncomp;
    pj->components = (pjpeg_component_t *)calloc((size_t)std::max(im.ncomp, 1), sizeof(pjpeg_component_t));
    for (int c = 0; c < im.ncomp; c++) {
        const HComp &h = im.comp[c];
        pjpeg_component_t &o = pj->components[c];
        o.id = h.id;
        o.hv = h.hv;
        o.scalex = h.sx;
        o.scaley = h.sy;
        o.tq = h.tq;
        o.tda = h.tda;
        if (h.scan >= 0) {
            o.width = h.pw;
            o.height = h.ph;
            o.stride = h.pstride;
            o.data = (uint8_t *)calloc((size_t)h.ph * h.pstride + 1, 1);
        }
    }
    J.sub_bits = jsub_for(sk.n);
    J.back_bits = std::max(512u, J.sub_bits);
    add_image(J, im, 0, 0, J.sub_bits, 7u, [&](int c, JPlaneDev &P) -> size_t {
        const pjpeg_component_t &o = pj->components[c];
        P.ow = o.width;
        P.oh = o.height;
        P.stride = o.stride;
        if ((size_t)o.width * o.height)
            J.outs.push_back(HOut{J.staging, (int64_t)o.stride, o.data, (int64_t)o.stride, o.width, o.height});
        return (size_t)o.stride * o.height + 16;
    });
    int rc;
    bool reset = false;
    {
        std::lock_guard<std::mutex> lk(g_pjpeg_mu);
        if (!g_pjpeg_dec) g_pjpeg_dec = at_jpeg_create();
        rc = g_pjpeg_dec ? run_job(g_pjpeg_dec, J, now_ms() - t0) : -1;
        if (rc == 0) reset = restart_failures(J, g_pjpeg_dec->h_stage, 1)[0] != 0;
    }
    if (rc != 0 || reset) {
        pjpeg_destroy(pj);
        if (error) *error = rc != 0 ? PJPEG_ERR_FILE : PJPEG_ERR_RESET;
        return nullptr;
    }
    return pj;
}

pjpeg_t *pjpeg_create_from_file(const char *path, uint32_t flags, int *error) {
    FILE *f = fopen(path, "rb");
    if (!f) return nullptr;
    fseek(f, 0, SEEK_END);
    const long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    uint8_t *buf = (uint8_t *)malloc(n > 0 ? (size_t)n : 1);
    const size_t got = n > 0 ? fread(buf, 1, (size_t)n, f) : 0;
    fclose(f);
    if (n < 0 || got != (size_t)n) {
        free(buf);
        if (error) *error = PJPEG_ERR_FILE;
        return nullptr;
    }
    pjpeg_t *pj = pjpeg_create_from_buffer(buf, (int)n, flags, error);
    free(buf);
    return pj;
}

void pjpeg_destroy(pjpeg_t *pj) {
    if (!pj) return;
    for (int c = 0; c < pj->ncomponents; c++) free(pj->components[c].data);
    free(pj->components);
    free(pj);
}

image_u8_t *pjpeg_to_u8_baseline(pjpeg_t *pj) {
    if (!pj || pj->ncomponents < 1) return nullptr;
    const pjpeg_component_t &c = pj->components[0];
    if (!c.data || c.width < pj->width || c.height < pj->height) return nullptr;
    image_u8_t *im = image_u8_create(pj->width, pj->height);
    for (uint32_t y = 0; y < pj->height; y++) memcpy(im->buf + (size_t)y * im->stride, c.data + (size_t)y * c.stride, pj->width);
    return im;
}

image_u8x3_t *image_u8x3_create_alignment(unsigned int width, unsigned int height, unsigned int alignment) {
    unsigned int stride = 3 * width;
    if (alignment && stride % alignment) stride += alignment - stride % alignment;
    image_u8x3_t tmp = {(int32_t)width, (int32_t)height, (int32_t)stride,
                        (uint8_t *)calloc((size_t)height * stride + 1, 1)};
    image_u8x3_t *im = (image_u8x3_t *)calloc(1, sizeof(image_u8x3_t));
    memcpy((void *)im, &tmp, sizeof tmp);
    return im;
}

image_u8x3_t *image_u8x3_create(unsigned int width, unsigned int height) {
    return image_u8x3_create_alignment(width, height, 192);
}

void image_u8x3_destroy(image_u8x3_t *im) {
    if (!im) return;
    free(im->buf);
    free(im);
}

static inline uint8_t clamp_i(int32_t v) { return v < 0 ? 0 : v > 255 ? 255 : (uint8_t)v; }
static inline uint8_t clamp_d(double v) { return v < 0 ? 0 : v > 255 ? 255 : (uint8_t)v; }

// YCbCr to RGB by the JFIF formulas (common/pjpeg.c:738-822): 16.16 fixed
// point when chroma is full size or both chroma planes are sampled alike
// (then only whole chroma cells are written), else in doubles.
image_u8x3_t *pjpeg_to_u8x3_baseline(pjpeg_t *pj) {
    if (!pj || pj->ncomponents != 3) return nullptr;
    const pjpeg_component_t &Y = pj->components[0], &Cb = pj->components[1], &Cr = pj->components[2];
    if (!Y.data || !Cb.data || !Cr.data || !Cb.width || !Cb.height || !Cr.width || !Cr.height) return nullptr;
    const int fby = (int)(Y.height / Cb.height), fbx = (int)(Y.width / Cb.width);
    const int fry = (int)(Y.height / Cr.height), frx = (int)(Y.width / Cr.width);
    if (!fby || !fbx || !fry || !frx) return nullptr;
    image_u8x3_t *im = image_u8x3_create(pj->width, pj->height);
    auto put = [&](uint32_t x, uint32_t y, int32_t r, int32_t g, int32_t b) {
        uint8_t *p = im->buf + (size_t)y * im->stride + 3 * (size_t)x;
        p[0] = clamp_i(r >> 16);
        p[1] = clamp_i(g >> 16);
        p[2] = clamp_i(b >> 16);
    };
    if (fby == 1 && fbx == 1 && fry == 1 && frx == 1) {
        for (uint32_t y = 0; y < pj->height; y++)
            for (uint32_t x = 0; x < pj->width; x++) {
                const int32_t yv = Y.data[y * Y.stride + x] * 65536;
                const int32_t cb = Cb.data[y * Cb.stride + x] - 128, cr = Cr.data[y * Cr.stride + x] - 128;
                put(x, y, yv + 91881 * cr, yv - 22554 * cb - 46802 * cr, yv + 116130 * cb);
            }
    } else if (fby == fry && fbx == frx) {
        for (uint32_t by = 0; by < pj->height / fby; by++)
            for (uint32_t bx = 0; bx < pj->width / fbx; bx++) {
                const int32_t cb = Cb.data[by * Cb.stride + bx] - 128, cr = Cr.data[by * Cr.stride + bx] - 128;
                const int32_t r0 = 91881 * cr, g0 = -22554 * cb - 46802 * cr, b0 = 116130 * cb;
                for (int dy = 0; dy < fby; dy++)
                    for (int dx = 0; dx < fbx; dx++) {
                        const uint32_t y = by * fby + dy, x = bx * fbx + dx;
                        const int32_t yv = Y.data[y * Y.stride + x] * 65536;
                        put(x, y, r0 + yv, g0 + yv, b0 + yv);
                    }
            }
    } else {
        for (uint32_t y = 0; y < pj->height; y++)
            for (uint32_t x = 0; x < pj->width; x++) {
                const int32_t yv = Y.data[y * Y.stride + x];
                const int32_t cb = Cb.data[(y / fby) * Cb.stride + x / fbx] - 128;
                const int32_t cr = Cr.data[(y / fry) * Cr.stride + x / frx] - 128;
                uint8_t *p = im->buf + (size_t)y * im->stride + 3 * (size_t)x;
                p[0] = clamp_d(yv + 1.402 * cr);
                p[1] = clamp_d(yv - 0.34414 * cb - 0.71414 * cr);
                p[2] = clamp_d(yv + 1.772 * cb);
            }
    }
    return im;
}

}  // extern "C"
