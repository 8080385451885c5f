// Clusters of boundary points without sorting the points
// (fast/clusters.c:16-66, 123-252, 318-382).
//
// The reference groups the boundary points by the pair of components they
// lie between, each cluster's points in emission order (y, x, neighbour),
// and orders the clusters. Here each point is made once, from the
// threshold image and the labels, as a 4-byte record in its row's region;
// the records are then placed, each at its place in its cluster:
//
//   k_point_scan     a warp per row: the row's points, their label pairs
//                    gathered in the warp's table (shared memory), the
//                    records in emission order; at the row's end each pair
//                    of the row into the frame's pair table (point count,
//                    first and last row) and the row's pair list.
//   k_cluster_collect (at_kernels.cu): the distinct pairs.
//   -- the host reads the pair and point counts (its only wait here) --
//   k_pair_frame, k_pair_scatter, k_pair_rank: the distinct pairs in order.
//                    A frame's pairs sort before the next frame's (the
//                    larger label is a node of the frame), so each frame's
//                    pairs are ranked among themselves.
//   k_cluster_span   per cluster: count, frame, first row, rows spanned.
//   scans            each cluster's first point; its row table's offset.
//   k_seg_fill       a warp per row: its pairs' point counts into the
//                    clusters' row tables.
//   k_seg_scan       a warp per cluster: the counts of its rows become the
//                    places of each row's first point of the cluster.
//   k_point_place    a warp per row: every record to its place; records of
//                    a row are in emission order, so a cluster's points
//                    keep the reference's order.
#include <cuda_runtime.h>
#include <stdint.h>

#include "at_device.cuh"
#include "at_gpu.h"
#include "at_kernels.h"

// The cluster key and the packed value of point j (neighbour (1,0), (0,1),
// (-1,1), (1,1)) of pixel x of row y (la, lb: labels of rows y, y + 1).
__device__ __forceinline__ uint64_t point_key(const uint32_t *la, const uint32_t *lb, int64_t x, int j, int nb) {
    const int dx = j == 0 || j == 3 ? 1 : j == 2 ? -1 : 0;
    const uint32_t l0 = la[x], l1 = j == 0 ? la[x + dx] : lb[x + dx];
    const uint64_t hi = l0 > l1 ? l0 : l1, lo = l0 > l1 ? l1 : l0;
    return hi << nb | lo;
}

// Rows 1 .. qh-2 of each frame, a warp per row.
#define ROW_WARPS_BEGIN                                                                              \
    const FrameDesc f = frames[blockIdx.y];                                                          \
    const int lane = threadIdx.x & 31;                                                               \
    const int64_t wpb = blockDim.x >> 5;                                                             \
    for (int64_t y = 1 + blockIdx.x * wpb + (threadIdx.x >> 5); y + 1 < f.qh; y += gridDim.x * wpb) {
#define ROW_WARPS_END }

// A warp's table of the pairs of its row: open addressing over 2 nd_cap
// slots (key, index), and per index (the order pairs first appear in the
// row) the key, the slot and the number of points.
struct RowPairs {
    uint64_t *tkey, *ikey;
    uint32_t *icnt;
    uint16_t *tpos, *islot;
};
__host__ __device__ inline size_t row_pairs_bytes(int nd_cap) { return (size_t)34 * nd_cap; }
__device__ inline RowPairs row_pairs(uint8_t *base, int nd_cap) {
    RowPairs W;
    W.tkey = reinterpret_cast<uint64_t *>(base);
    W.ikey = W.tkey + 2 * nd_cap;
    W.icnt = reinterpret_cast<uint32_t *>(W.ikey + nd_cap);
    W.tpos = reinterpret_cast<uint16_t *>(W.icnt + nd_cap);
    W.islot = W.tpos + 2 * nd_cap;
    return W;
}

// Point records: pair index in the row | neighbour j << 11 | (pixel is 0)
// << 13 | x << 14.
#define PREC_ID 0x7ffu

// Every boundary point, once: its pair into the warp's row table, its
// record (emission order) into the row's region; at the row's end each of
// the row's pairs into the frame's pair table (count, first and last row)
// and, with its points in the row, into the row's pair list. Any capacity
// exceeded (pairs of a row, records of a row, probes of the pair table)
// sets *full and the batch takes the sorting path instead.
__global__ void __launch_bounds__(256, 5) k_point_scan(const FrameDesc *frames, const uint8_t *thr, const uint32_t *lab,
                                                    int nb, PairTable T, PointRows P, uint32_t *full,
                                                    unsigned long long *npoints) {
    extern __shared__ __align__(16) uint8_t s_mem[];
    const int nd_cap = P.nd_cap, rt = 2 * nd_cap;
    RowPairs W = row_pairs(s_mem + (threadIdx.x >> 5) * row_pairs_bytes(nd_cap), nd_cap);
    for (int i = threadIdx.x & 31; i < rt; i += 32) W.tkey[i] = CH_EMPTY;
    __syncwarp();
    const uint32_t lt = (1u << (threadIdx.x & 31)) - 1u;
    uint64_t pts = 0;
    ROW_WARPS_BEGIN
    const uint8_t *a = thr + f.q_off + y * f.qw, *b = a + f.qw;
    const uint32_t *la = lab + f.q_off + y * f.qw, *lb = la + f.qw;
    uint32_t *rec = P.rec + 2 * (f.q_off + y * f.qw);
    const uint32_t rcap = (uint32_t)(2 * f.qw);
    uint32_t nd = 0, nrec = 0;
    for (int64_t x0 = 0; x0 < f.qw; x0 += 32) {
        const int64_t x = x0 + lane;
        const uint32_t m = x < f.qw ? point_mask(a, b, la, lb, x, f.qw) : 0u;
        if (!__any_sync(0xffffffffu, m != 0)) continue;
        uint32_t total;
        const uint32_t o = warp_excl_scan(__popc(m), &total);
        if (nrec + total > rcap) {
            if (lane == 0) atomicOr(full, 1u);
            return;
        }
        uint32_t id4[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const bool has = (m >> j & 1u) != 0;
            const uint64_t k = has ? point_key(la, lb, x, j, nb) : CH_EMPTY;
            // the pair's index in the row, if the row has met it already
            uint32_t id = 0xffffffffu;
            if (has) {
                uint32_t h = ch_hash(k) & (uint32_t)(rt - 1);
                for (int p = 0; p < rt; p++) {
                    const uint64_t cur = W.tkey[h];
                    if (cur == k) {
                        id = W.tpos[h];
                        break;
                    }
                    if (cur == CH_EMPTY) break;
                    h = (h + 1) & (uint32_t)(rt - 1);
                }
            }
            const bool miss = has && id == 0xffffffffu;
            if (__any_sync(0xffffffffu, miss)) {
                // pairs new to the row: each one's leader adds it
                __syncwarp();
                const uint64_t km = miss ? k : CH_EMPTY;
                const uint32_t peers = __match_any_sync(0xffffffffu, km);
                const int leader = __ffs(peers) - 1;
                const bool lead = miss && lane == leader;
                uint32_t h = 0;
                bool added = false;
                if (lead) {
                    h = ch_hash(k) & (uint32_t)(rt - 1);
                    for (int p = 0; p < rt; p++) {
                        const unsigned long long old =
                            atomicCAS(reinterpret_cast<unsigned long long *>(W.tkey + h), CH_EMPTY, k);
                        if (old == CH_EMPTY) {
                            added = true;
                            break;
                        }
                        h = (h + 1) & (uint32_t)(rt - 1);
                    }
                }
                const uint32_t nadd = __ballot_sync(0xffffffffu, added);
                if (nd + __popc(nadd) > (uint32_t)nd_cap) {
                    if (lane == 0) atomicOr(full, 1u);
                    return;
                }
                uint32_t nid = 0;
                if (added) {
                    nid = nd + __popc(nadd & lt);
                    W.tpos[h] = (uint16_t)nid;
                    W.ikey[nid] = k;
                    W.islot[nid] = (uint16_t)h;
                    W.icnt[nid] = 0;
                }
                nd += __popc(nadd);
                nid = __shfl_sync(0xffffffffu, nid, leader);
                if (miss) id = nid;
                __syncwarp();
            }
            if (has) atomicAdd(W.icnt + id, 1u);
            id4[j] = id;
            __syncwarp();
        }
        // this lane's points, in emission order (x, then neighbour)
        if (m) {
            const uint32_t g = a[x] == 0 ? 1u : 0u;
            uint32_t t = nrec + o;
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (m >> j & 1u) rec[t++] = id4[j] | (uint32_t)j << 11 | g << 13 | (uint32_t)x << 14;
        }
        nrec += total;
    }
    __syncwarp();
    // the row's pairs into the frame's pair table; the table cleared
    uint32_t *ps = P.pslot + (f.row0 + y) * nd_cap, *pc = P.pcnt + (f.row0 + y) * nd_cap;
    for (uint32_t i = lane; i < nd; i += 32) {
        const uint64_t k = W.ikey[i];
        uint32_t slot = ch_hash(k) & T.mask;
        int p = 0;
        for (; p < CH_PROBES; p++) {
            uint64_t cur = *(volatile uint64_t *)(T.keys + slot);
            if (cur == CH_EMPTY) {
                const unsigned long long old = atomicCAS(reinterpret_cast<unsigned long long *>(T.keys + slot), CH_EMPTY, k);
                cur = old == CH_EMPTY ? k : old;
            }
            if (cur == k) break;
            slot = (slot + 1) & T.mask;
        }
        if (p == CH_PROBES) {
            atomicOr(full, 1u);
        } else {
            atomicAdd(T.count + slot, W.icnt[i]);
            atomicMin(T.ymin + slot, (uint32_t)y);
            atomicMax(T.ymax + slot, (uint32_t)y);
        }
        ps[i] = slot;
        pc[i] = W.icnt[i];
        W.tkey[W.islot[i]] = CH_EMPTY;
    }
    if (lane == 0) P.info[f.row0 + y] = make_uint2(nrec, nd);
    pts += nrec;
    __syncwarp();
    ROW_WARPS_END
    if ((threadIdx.x & 31) == 0 && pts) atomicAdd(npoints, (unsigned long long)pts);
}

__device__ __forceinline__ int frame_of_node(const FrameDesc *frames, int nframes, int64_t node) {
    int lo = 0, hi = nframes - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (frames[mid].node_off <= node)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Each distinct pair's frame; pairs per frame.
__global__ void k_pair_frame(const uint64_t *okeys, int64_t ncl, int nb, const FrameDesc *frames, int nframes,
                             uint32_t *kframe, uint32_t *fcount) {
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < ncl; r += (int64_t)gridDim.x * blockDim.x) {
        const int fr = frame_of_node(frames, nframes, (int64_t)(okeys[r] >> nb));
        kframe[r] = (uint32_t)fr;
        atomicAdd(fcount + fr, 1u);
    }
}

// One block: each frame's first pair (foff, nframes + 1 entries).
__global__ void __launch_bounds__(1024) k_pair_frame_offsets(const uint32_t *fcount, int nframes, uint32_t *foff,
                                                             uint32_t *fcur) {
    __shared__ uint32_t sh[32];
    uint32_t base = 0;
    for (int f0 = 0; f0 < nframes; f0 += blockDim.x) {
        const int f = f0 + threadIdx.x;
        const uint32_t c = f < nframes ? fcount[f] : 0u;
        uint32_t total;
        const uint32_t off = block_excl_scan(c, &total, sh);
        if (f < nframes) {
            foff[f] = base + off;
            fcur[f] = 0;
        }
        base += total;
    }
    if (threadIdx.x == 0) foff[nframes] = base;
}

__global__ void k_pair_scatter(const uint64_t *okeys, const uint32_t *oslots, int64_t ncl, const uint32_t *kframe,
                               const uint32_t *foff, uint32_t *fcur, uint64_t *gkeys, uint32_t *gslots) {
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < ncl; r += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t fr = kframe[r];
        const uint32_t p = foff[fr] + atomicAdd(fcur + fr, 1u);
        gkeys[p] = okeys[r];
        gslots[p] = oslots[r];
    }
}

// A warp per pair: its place = its frame's first place + the number of
// smaller pairs of the frame (the pairs are distinct).
__global__ void __launch_bounds__(256) k_pair_rank(const uint64_t *gkeys, const uint32_t *gslots, int64_t ncl,
                                                   const uint32_t *foff, int nframes, uint64_t *skeys,
                                                   uint32_t *sslots) {
    const int lane = threadIdx.x & 31;
    for (int64_t p = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < ncl;
         p += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        int lo = 0, hi = nframes - 1;  // the frame whose segment holds p
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (foff[mid] <= (uint32_t)p)
                lo = mid;
            else
                hi = mid - 1;
        }
        const uint64_t k = gkeys[p];
        uint32_t below = 0;
        for (uint32_t q = foff[lo] + lane; q < foff[lo + 1]; q += 32) below += gkeys[q] < k;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) below += __shfl_xor_sync(0xffffffffu, below, o);
        if (lane == 0) {
            skeys[foff[lo] + below] = k;
            sslots[foff[lo] + below] = gslots[p];
        }
    }
}

// Cluster c (in pair order): its slot's rank; its point count, frame,
// first row and rows spanned.
__global__ void k_cluster_span(const uint64_t *skeys, const uint32_t *sslots, int64_t ncl, PairTable T, int nb,
                               const FrameDesc *frames, int nframes, uint32_t *rank_of_slot, uint32_t *ccount,
                               uint32_t *cspan, uint32_t *cy0, int32_t *cframe) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncl; c += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t s = sslots[c];
        rank_of_slot[s] = (uint32_t)c;
        ccount[c] = T.count[s];
        cy0[c] = T.ymin[s];
        cspan[c] = T.ymax[s] - T.ymin[s] + 1;
        cframe[c] = frame_of_node(frames, nframes, (int64_t)(skeys[c] >> nb));
    }
}

// Exclusive scans of two arrays of n values at once (a pass per block of
// SCAN_ITEMS, one block over the block sums, a pass that adds them):
// out_a, out_b get n + 1 entries (the totals last).
#define SCAN_THREADS 256
#define SCAN_ITEMS (4 * SCAN_THREADS)

__global__ void __launch_bounds__(SCAN_THREADS) k_scan2_sums(const uint32_t *a, const uint32_t *b, int64_t n,
                                                             uint32_t *sa, uint32_t *sb) {
    __shared__ uint32_t sh[32];
    const int64_t i0 = (int64_t)blockIdx.x * SCAN_ITEMS + 4 * threadIdx.x;
    uint32_t va = 0, vb = 0;
    for (int k = 0; k < 4; k++)
        if (i0 + k < n) {
            va += a[i0 + k];
            vb += b[i0 + k];
        }
    uint32_t ta, tb;
    block_excl_scan(va, &ta, sh);
    block_excl_scan(vb, &tb, sh);
    if (threadIdx.x == 0) {
        sa[blockIdx.x] = ta;
        sb[blockIdx.x] = tb;
    }
}

__global__ void __launch_bounds__(1024) k_scan2_top(uint32_t *sa, uint32_t *sb, int64_t nblocks) {
    __shared__ uint32_t sh[32];
    uint32_t ba = 0, bb = 0;
    for (int64_t i0 = 0; i0 < nblocks; i0 += blockDim.x) {
        const int64_t i = i0 + threadIdx.x;
        const uint32_t va = i < nblocks ? sa[i] : 0u, vb = i < nblocks ? sb[i] : 0u;
        uint32_t ta, tb;
        const uint32_t oa = block_excl_scan(va, &ta, sh), ob = block_excl_scan(vb, &tb, sh);
        if (i < nblocks) {
            sa[i] = ba + oa;
            sb[i] = bb + ob;
        }
        ba += ta;
        bb += tb;
    }
    if (threadIdx.x == 0) {
        sa[nblocks] = ba;
        sb[nblocks] = bb;
    }
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan2_apply(const uint32_t *a, const uint32_t *b, int64_t n,
                                                              const uint32_t *sa, const uint32_t *sb,
                                                              int64_t nblocks, uint32_t *out_a, uint32_t *out_b) {
    __shared__ uint32_t sh[32];
    const int64_t i0 = (int64_t)blockIdx.x * SCAN_ITEMS + 4 * threadIdx.x;
    uint32_t xa[4], xb[4], va = 0, vb = 0;
    for (int k = 0; k < 4; k++) {
        xa[k] = i0 + k < n ? a[i0 + k] : 0u;
        xb[k] = i0 + k < n ? b[i0 + k] : 0u;
        va += xa[k];
        vb += xb[k];
    }
    uint32_t ta, tb;
    uint32_t oa = block_excl_scan(va, &ta, sh) + sa[blockIdx.x], ob = block_excl_scan(vb, &tb, sh) + sb[blockIdx.x];
    for (int k = 0; k < 4; k++)
        if (i0 + k < n) {
            out_a[i0 + k] = oa;
            out_b[i0 + k] = ob;
            oa += xa[k];
            ob += xb[k];
        }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        out_a[n] = sa[nblocks];
        out_b[n] = sb[nblocks];
    }
}

// The row tables: zeroed up to their total (checked against the capacity:
// a shortfall sets AT_ERR_SEGCAP and the host runs the batch again with
// room enough; the point kernels then skip their work).
__global__ void k_seg_zero(const uint32_t *spanoff, int64_t ncl, uint32_t *seg, int64_t cap, uint32_t *err) {
    const int64_t total = spanoff[ncl];
    if (total > cap) {
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(err, AT_ERR_SEGCAP);
        return;
    }
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
        seg[i] = 0;
}

// A warp per cluster: seg[spanoff[c] + r] = the place of the cluster's
// first point in row cy0[c] + r.
__global__ void __launch_bounds__(256) k_seg_scan(const uint32_t *cstart, const uint32_t *spanoff,
                                                  const uint32_t *cspan, int64_t ncl, uint32_t *seg, int64_t cap) {
    if (spanoff[ncl] > cap) return;
    const int lane = threadIdx.x & 31;
    for (int64_t c = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < ncl;
         c += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        uint32_t *row = seg + spanoff[c];
        const uint32_t n = cspan[c];
        uint32_t carry = cstart[c];
        for (uint32_t i0 = 0; i0 < n; i0 += 32) {
            const uint32_t i = i0 + lane;
            const uint32_t v = i < n ? row[i] : 0u;
            uint32_t total;
            const uint32_t o = warp_excl_scan(v, &total);
            if (i < n) row[i] = carry + o;
            carry += total;
        }
    }
}

// Each row's pairs: their point counts into the row tables
// (seg[spanoff[c] + y - cy0[c]] for the pair's cluster c).
__global__ void __launch_bounds__(256) k_seg_fill(const FrameDesc *frames, PointRows P, const uint32_t *rank_of_slot,
                                                  const uint32_t *spanoff, const uint32_t *cy0, int64_t ncl,
                                                  uint32_t *seg, int64_t cap) {
    if (spanoff[ncl] > cap) return;
    ROW_WARPS_BEGIN
    const uint32_t nd = P.info[f.row0 + y].y;
    const uint32_t *ps = P.pslot + (f.row0 + y) * P.nd_cap, *pc = P.pcnt + (f.row0 + y) * P.nd_cap;
    for (uint32_t i = lane; i < nd; i += 32) {
        const uint32_t c = rank_of_slot[ps[i]];
        seg[spanoff[c] + ((uint32_t)y - cy0[c])] = pc[i];
    }
    ROW_WARPS_END
}

// A warp per row: each record to its place, the row's first place of each
// pair's cluster (seg, after the scan) plus the pair's points before it in
// the row; the records are in emission order, so a cluster's points keep
// the reference's order.
__global__ void __launch_bounds__(256) k_point_place(const FrameDesc *frames, PointRows P,
                                                     const uint32_t *rank_of_slot, const uint32_t *spanoff,
                                                     const uint32_t *cy0, int64_t ncl, const uint32_t *seg, int64_t cap,
                                                     uint64_t *out, int64_t npts, uint32_t *err) {
    extern __shared__ __align__(16) uint32_t s_base[];
    if (spanoff[ncl] > cap) return;
    uint32_t *base = s_base + (threadIdx.x >> 5) * P.nd_cap;
    const uint32_t lt = (1u << (threadIdx.x & 31)) - 1u;
    ROW_WARPS_BEGIN
    const uint2 inf = P.info[f.row0 + y];
    const uint32_t *ps = P.pslot + (f.row0 + y) * P.nd_cap;
    for (uint32_t i = lane; i < inf.y; i += 32) {
        const uint32_t c = rank_of_slot[ps[i]];
        base[i] = seg[spanoff[c] + ((uint32_t)y - cy0[c])];
    }
    __syncwarp();
    const uint32_t *rec = P.rec + 2 * (f.q_off + y * f.qw);
    for (uint32_t r0 = 0; r0 < inf.x; r0 += 32) {
        const uint32_t r = r0 + lane;
        const bool valid = r < inf.x;
        const uint32_t rc = valid ? rec[r] : 0u;
        const uint32_t id = valid ? rc & PREC_ID : 0xffffffffu;
        const uint32_t peers = __match_any_sync(0xffffffffu, id);
        const uint32_t at = valid ? base[id] + __popc(peers & lt) : 0u;
        __syncwarp();
        if (valid && lane == __ffs(peers) - 1) base[id] += __popc(peers);
        if (valid) {
            const uint32_t j = (rc >> 11) & 3u, x = rc >> 14;
            const int dx = j == 0 || j == 3 ? 1 : j == 2 ? -1 : 0, dy = j == 0 ? 0 : 1;
            const int g = (rc >> 13 & 1u) ? 255 : -255;
            const uint64_t px = (uint64_t)(2 * (int64_t)x + dx), py = (uint64_t)(2 * y + dy);
            const uint64_t gx = (uint16_t)(int16_t)(dx * g), gy = (uint16_t)(int16_t)(dy * g);
            if (at < npts)  // always, unless the counts disagree: then an error, not a stray write
                out[at] = px | py << 16 | gx << 32 | gy << 48;
            else
                atomicOr(err, AT_ERR_CAPACITY);
        }
        __syncwarp();
    }
    ROW_WARPS_END
}

// ---------------------------------------------------------------------------
// Launchers.

static inline unsigned flat_grid(int64_t n, int threads) {
    const int64_t b = (n + threads - 1) / threads;
    return (unsigned)(b < 1 ? 1 : b < 148 * 16 ? b : 148 * 16);
}

static inline dim3 row_warps(const Launch &L) {
    const int64_t b = (L.max_qh + 7) / 8;
    return dim3((unsigned)(b < 1 ? 1 : b < 148 * 8 ? b : 148 * 8), (unsigned)L.nframes);
}

// Warps per block of the point scan: their row tables within 96 KB.
static inline int scan_warps(int nd_cap) {
    const int w = (int)((96 * 1024) / row_pairs_bytes(nd_cap));
    return w < 1 ? 1 : w > 8 ? 8 : w;
}

bool point_scan_set_smem() {
    return cudaFuncSetAttribute(k_point_scan, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024) == cudaSuccess &&
           cudaFuncSetAttribute(k_point_place, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024) == cudaSuccess;
}

void launch_point_scan(const Launch &L, const FrameDesc *frames, const uint8_t *thr, const uint32_t *lab, int nb,
                       const PairTable &T, const PointRows &P, uint32_t *full, unsigned long long *npoints) {
    const int w = scan_warps(P.nd_cap);
    const int64_t b = (L.max_qh + w - 1) / w;
    const dim3 grid((unsigned)(b < 1 ? 1 : b < 148 * 8 ? b : 148 * 8), (unsigned)L.nframes);
    k_point_scan<<<grid, 32 * w, w * row_pairs_bytes(P.nd_cap), L.stream>>>(frames, thr, lab, nb, T, P, full, npoints);
}

void launch_pair_order(cudaStream_t s, const uint64_t *okeys, const uint32_t *oslots, int64_t ncl, int nb,
                       const FrameDesc *frames, int nframes, const PairTable &T, const PairScratch &P,
                       uint64_t *skeys, uint32_t *sslots, uint32_t *rank_of_slot, uint32_t *ccount, uint32_t *cspan,
                       uint32_t *cy0, int32_t *cframe, uint32_t *cstart, uint32_t *spanoff) {
    if (ncl <= 0) return;
    cudaMemsetAsync(P.fcount, 0, (size_t)nframes * 4, s);
    k_pair_frame<<<flat_grid(ncl, 256), 256, 0, s>>>(okeys, ncl, nb, frames, nframes, P.kframe, P.fcount);
    k_pair_frame_offsets<<<1, 1024, 0, s>>>(P.fcount, nframes, P.foff, P.fcur);
    k_pair_scatter<<<flat_grid(ncl, 256), 256, 0, s>>>(okeys, oslots, ncl, P.kframe, P.foff, P.fcur, P.gkeys,
                                                       P.gslots);
    k_pair_rank<<<flat_grid(ncl * 32, 256), 256, 0, s>>>(P.gkeys, P.gslots, ncl, P.foff, nframes, skeys, sslots);
    k_cluster_span<<<flat_grid(ncl, 256), 256, 0, s>>>(skeys, sslots, ncl, T, nb, frames, nframes, rank_of_slot,
                                                       ccount, cspan, cy0, cframe);
    const int64_t nblk = (ncl + SCAN_ITEMS - 1) / SCAN_ITEMS;
    k_scan2_sums<<<(unsigned)nblk, SCAN_THREADS, 0, s>>>(ccount, cspan, ncl, P.bsum_a, P.bsum_b);
    k_scan2_top<<<1, 1024, 0, s>>>(P.bsum_a, P.bsum_b, nblk);
    k_scan2_apply<<<(unsigned)nblk, SCAN_THREADS, 0, s>>>(ccount, cspan, ncl, P.bsum_a, P.bsum_b, nblk, cstart,
                                                          spanoff);
}

int64_t pair_scan_blocks(int64_t ncl) { return (ncl + SCAN_ITEMS - 1) / SCAN_ITEMS + 1; }

// An exclusive scan of n u32 values into out (n + 1 entries, the total
// last) with the two-array kernels above, the second array the first
// again; scratch: scan_u32_scratch(n) values.
int64_t scan_u32_scratch(int64_t n) { return 2 * ((n + SCAN_ITEMS - 1) / SCAN_ITEMS + 1) + n + 1; }

void launch_scan_u32(cudaStream_t s, const uint32_t *a, int64_t n, uint32_t *out, uint32_t *scratch) {
    if (n <= 0) return;
    const int64_t nblk = (n + SCAN_ITEMS - 1) / SCAN_ITEMS;
    uint32_t *sa = scratch, *sb = scratch + nblk + 1, *ob = scratch + 2 * (nblk + 1);
    k_scan2_sums<<<(unsigned)nblk, SCAN_THREADS, 0, s>>>(a, a, n, sa, sb);
    k_scan2_top<<<1, 1024, 0, s>>>(sa, sb, nblk);
    k_scan2_apply<<<(unsigned)nblk, SCAN_THREADS, 0, s>>>(a, a, n, sa, sb, nblk, out, ob);
}

void launch_point_place(const Launch &L, const FrameDesc *frames, const PointRows &P, const uint32_t *rank_of_slot,
                        const uint32_t *cstart, const uint32_t *spanoff, const uint32_t *cspan, const uint32_t *cy0,
                        int64_t ncl, uint32_t *seg, int64_t cap, uint64_t *out, int64_t npts, uint32_t *err) {
    if (ncl <= 0) return;
    k_seg_zero<<<flat_grid(cap, 256), 256, 0, L.stream>>>(spanoff, ncl, seg, cap, err);
    k_seg_fill<<<row_warps(L), 256, 0, L.stream>>>(frames, P, rank_of_slot, spanoff, cy0, ncl, seg, cap);
    k_seg_scan<<<flat_grid(ncl * 32, 256), 256, 0, L.stream>>>(cstart, spanoff, cspan, ncl, seg, cap);
    k_point_place<<<row_warps(L), 256, 8 * P.nd_cap * 4, L.stream>>>(frames, P, rank_of_slot, spanoff, cy0, ncl, seg,
                                                                    cap, out, npts, err);
}
