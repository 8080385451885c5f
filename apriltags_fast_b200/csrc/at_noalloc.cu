// at_threshold_noalloc: the adaptive threshold stage for callers that must
// not allocate device memory.
//
// Some callers cannot call cudaMalloc: a camera loop that has to keep its
// latency bound (cudaMalloc and cudaFree synchronise the whole device, which
// stalls every other stream), a process whose device memory is all handed to
// one pool up front, or code that only receives device pointers from the
// framework that owns the GPU. This entry point takes the caller's input
// and output buffers and keeps its only scratch, the per-tile max and min
// of the 4x4 tiles, in a fixed array of this library that every GPU holds
// from the first use until the process exits (2 MiB: quad images up to
// 1 Mi tiles, e.g. 4096 x 4096).
//
// It computes exactly what the detector's own threshold stage computes
// (tile max/min, their 3x3 tile neighbourhood, lo + (hi - lo) / 2, 127 for
// flat tiles), so its output equals the threshold image of at_detect.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <mutex>

#include "apriltag_fast.h"

#define AT_NOALLOC_MAX_TILES (1024 * 1024)

// The scratch: tile max in [0, MAX_TILES), tile min in [MAX_TILES, 2 MAX).
// Every call writes every tile it reads, so nothing needs clearing between
// calls; calls that overlap on the GPU share it and race.
static __device__ __align__(256) uint8_t g_noalloc_tiles[2 * AT_NOALLOC_MAX_TILES];

__global__ void k_noalloc_tiles(const uint8_t *im, int64_t w, int64_t h, uint8_t *tiles) {
    const int64_t tw = w / 4, th = h / 4, n = tw * th;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int64_t ty = i / tw, tx = i - ty * tw;
        const uint8_t *p = im + 4 * ty * w + 4 * tx;
        uint32_t hi = 0, lo = 255;
        for (int dy = 0; dy < 4; dy++)
            for (int dx = 0; dx < 4; dx++) {
                uint32_t v = p[dy * w + dx];
                hi = v > hi ? v : hi;
                lo = v < lo ? v : lo;
            }
        tiles[i] = (uint8_t)hi;
        tiles[AT_NOALLOC_MAX_TILES + i] = (uint8_t)lo;
    }
}

__global__ void k_noalloc_threshold(const uint8_t *im, int64_t w, int64_t h, const uint8_t *tiles, int32_t diff,
                                    uint8_t *out) {
    const int64_t tw = w / 4, th = h / 4, n = w * h;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int64_t y = i / w, x = i - y * w;
        int64_t ty = y >> 2, tx = x >> 2;
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
        for (int64_t yy = ty > 0 ? ty - 1 : 0; yy <= (ty + 1 < th ? ty + 1 : th - 1); yy++)
            for (int64_t xx = tx > 0 ? tx - 1 : 0; xx <= (tx + 1 < tw ? tx + 1 : tw - 1); xx++) {
                uint32_t a = tiles[yy * tw + xx], b = tiles[AT_NOALLOC_MAX_TILES + yy * tw + xx];
                hi = a > hi ? a : hi;
                lo = b < lo ? b : lo;
            }
        uint32_t t = lo + (hi - lo) / 2;
        uint8_t v = im[i] > t ? 255 : 0;
        out[i] = may_flat && (int32_t)(hi - lo) < diff ? 127 : v;
    }
}

// The device address of the scratch on each device, found once per device
// (in host code the array's name is only a stand-in for it) and kept for the
// life of the process: a cudaDeviceReset unloads the module, after which the
// array may live elsewhere, so calls after a reset are not supported.
static uint8_t *g_tiles_addr[128];
static std::mutex g_tiles_mu;

extern "C" int at_threshold_noalloc(const uint8_t *image, int64_t width, int64_t height,
                                    int32_t min_white_black_diff, uint8_t *out, void *stream) {
    if (width < 4 || height < 4) {
        fprintf(stderr, "at_threshold_noalloc: image %lldx%lld below one 4x4 tile\n", (long long)width,
                (long long)height);
        return 1;
    }
    if ((width / 4) * (height / 4) > AT_NOALLOC_MAX_TILES) {
        fprintf(stderr, "at_threshold_noalloc: %lldx%lld has more than %d tiles (the fixed scratch)\n",
                (long long)width, (long long)height, AT_NOALLOC_MAX_TILES);
        return 1;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128) return 2;
    uint8_t *tiles;
    {
        std::lock_guard<std::mutex> lock(g_tiles_mu);
        if (!g_tiles_addr[dev]) {
            void *p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_tiles);
            if (e != cudaSuccess || !p) {
                fprintf(stderr, "at_threshold_noalloc: cudaGetSymbolAddress: %s\n", cudaGetErrorString(e));
                return 2;
            }
            g_tiles_addr[dev] = (uint8_t *)p;
        }
        tiles = g_tiles_addr[dev];
    }
    cudaStream_t st = (cudaStream_t)stream;
    int64_t ntiles = (width / 4) * (height / 4), npx = width * height;
    unsigned b1 = (unsigned)((ntiles + 255) / 256 < 148 * 8 ? (ntiles + 255) / 256 : 148 * 8);
    unsigned b2 = (unsigned)((npx + 255) / 256 < 148 * 16 ? (npx + 255) / 256 : 148 * 16);
    k_noalloc_tiles<<<b1, 256, 0, st>>>(image, width, height, tiles);
    k_noalloc_threshold<<<b2, 256, 0, st>>>(image, width, height, tiles, min_white_black_diff, out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "at_threshold_noalloc: %s\n", cudaGetErrorString(e));
        return 2;
    }
    return 0;
}
