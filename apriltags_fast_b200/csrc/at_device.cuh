// Device helpers shared by the kernel files.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "at_gpu.h"

__device__ __forceinline__ int64_t dmin(int64_t a, int64_t b) { return a < b ? a : b; }
__device__ __forceinline__ int64_t dmax(int64_t a, int64_t b) { return a > b ? a : b; }

// Block-wide exclusive scan of one value per thread (blockDim <= 1024).
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t *total, uint32_t *sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    __syncthreads();
    if (lane == 31) sh[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        uint32_t s = lane < nw ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += t;
        }
        if (lane < nw) sh[lane] = s;
    }
    __syncthreads();
    uint32_t off = wid > 0 ? sh[wid - 1] : 0;
    *total = sh[nw - 1];
    return off + incl - v;
}

// Whether two runs of equal value v on adjacent rows are joined
// (fast/unionfind.c:112-146): they share a column x >= 1, or, for white
// (8-connected), one is diagonal to the other at columns >= 1.
__device__ __forceinline__ bool runs_touch(int64_t a0, int64_t a1, int64_t b0, int64_t b1, uint8_t v) {
    if (dmax(dmax(a0, b0), 1) <= dmin(a1, b1)) return true;
    if (v != 255) return false;
    if (dmax(dmax(a0, b0 + 1), 1) <= dmin(a1, b1 + 1)) return true;
    return dmax(dmax(a0, b0 - 1), 1) <= dmin(a1, b1 - 1);
}

// The boundary points of pixel x of row a (row b is the next row; la, lb
// their labels) as 4 bits, one per neighbour (1,0), (0,1), (-1,1), (1,1)
// (fast/clusters.c:144-252): a point where one pixel is 0, the other 255
// and both labels are not AT_NOK; (-1,1) left out when the pixel to the
// left gave its (1,1) point, except at x = 1; x = 0 gives only (1,0).
__device__ __forceinline__ uint32_t point_mask(const uint8_t *a, const uint8_t *b, const uint32_t *la,
                                               const uint32_t *lb, int64_t x, int64_t qw) {
    if (x >= qw - 1) return 0;
    if (x == 0) return ((a[0] ^ a[1]) == 255 && la[0] != AT_NOK && la[1] != AT_NOK) ? 1u : 0u;
    if (la[x] == AT_NOK) return 0;
    uint8_t v = a[x];
    uint32_t c10 = (v ^ a[x + 1]) == 255 && la[x + 1] != AT_NOK;
    uint32_t c01 = (v ^ b[x]) == 255 && lb[x] != AT_NOK;
    uint32_t cm1 = (v ^ b[x - 1]) == 255 && lb[x - 1] != AT_NOK;
    uint32_t c11 = (v ^ b[x + 1]) == 255 && lb[x + 1] != AT_NOK;
    uint32_t left11 = x > 1 && (a[x - 1] ^ b[x]) == 255 && la[x - 1] != AT_NOK && lb[x] != AT_NOK;
    return c10 | c01 << 1 | (cm1 & (left11 ^ 1u)) << 2 | c11 << 3;
}

// Warp-wide exclusive scan of one value per lane; *total gets the sum.
__device__ __forceinline__ uint32_t warp_excl_scan(uint32_t v, uint32_t *total) {
    const int lane = threadIdx.x & 31;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    *total = __shfl_sync(0xffffffffu, incl, 31);
    return incl - v;
}

// Open-addressing table of cluster keys (label pairs).
#define CH_EMPTY 0xffffffffffffffffull
#define CH_PROBES 64

__device__ __forceinline__ uint32_t ch_hash(uint64_t k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    return (uint32_t)k;
}
