// The reference's order of the quads whose detections share an id.
//
// Why it matters. The reference hands its detections to a stable sort by
// id in quad order (fast/detector.c:143-179), and its reconcile of
// overlapping detections of one tag walks them in that order
// (fast/decode.c:860-891). So the quad order decides the output exactly
// when two detections of a frame have the same id. Quad order is cluster
// order, and the reference orders clusters by (hash bucket, id) of the key
// (larger root << 32) + smaller root of the two components a cluster lies
// between (fast/clusters.c:44, 97-103, 338-356), where a component's root
// is the node that the reference's sequential union by size over the runs
// in raster order leaves at the top (fast/unionfind.c:15-45, 152-196,
// 284-298), numbered as the reference packs its nodes (the runs row after
// row, then one node per row for the last column).
//
// The GPU's union-find is parallel and labels a component by its smallest
// node, which fixes the partition but not the reference's root. These
// kernels find that root for the few components that matter and give the
// final stage the reference's order keys:
//
//   k_ref_targets  per frame: the ids that two or more detections share;
//                  the components of their quads are the targets (their GPU
//                  labels and pixel counts); the packed run numbering.
//   k_ref_mark     the runs of the target components, row by row, compacted
//                  (start, end, index in row, value, target).
//   k_ref_replay   a warp per frame sweeps the rows and replays the
//                  reference's unions of the target runs (see below).
//   k_finalize     (at_kernels.cu) orders those detections by the keys.
//
// The replay. Before row y, each set of target runs that touches row y-1
// is a "slot" with its root and pixel count. The reference's calls of row
// y (each run in order, its touching runs above in order, then the
// last-column link) join slots and the new runs into groups. A group in
// which one slot holds more pixels than all its other members together
// keeps that slot's root whatever the order (that slot's set wins every
// comparison it meets: the a side needs strictly more, the b side wins
// ties). Any other group is replayed call by call, a lane per group. A set
// that no longer touches the current row is a whole component; a set
// holding more than half of its component's pixels can never lose a
// comparison again; either way its root is final. The replay restricted
// to a component gives the reference's root because the sets of other
// components never meet it. Every frame without a shared id returns at
// once.
#include <cuda_runtime.h>
#include <stdint.h>

#include "at_device.cuh"
#include "at_gpu.h"
#include "at_kernels.h"

#define REF_HASH 1024          // open-addressing table of target labels (k_ref_targets, k_ref_mark)
#define REF_NONE 0xffu         // no target
#define REF_TOUCHED 1u
static_assert(AT_REF_MAXT < REF_NONE, "target indices fit a byte");
static_assert(2 * AT_REF_MAXT <= REF_HASH, "the label table stays half empty");

__device__ __forceinline__ uint32_t ref_hash(uint32_t x) {
    x *= 0x9e3779b1u;
    return x ^ (x >> 15);
}

// A label's target index in a table of (label + 1, index) pairs; REF_NONE
// when absent.
__device__ __forceinline__ uint32_t ref_lookup(const uint32_t *keys, const uint8_t *idx, uint32_t label) {
    uint32_t h = ref_hash(label) & (REF_HASH - 1);
    for (int p = 0; p < REF_HASH; p++) {
        const uint32_t k = keys[h];
        if (k == 0) return REF_NONE;
        if (k == label + 1) return idx[h];
        h = (h + 1) & (REF_HASH - 1);
    }
    return REF_NONE;
}

// ---------------------------------------------------------------------------
// Targets: a block per frame.

__global__ void __launch_bounds__(256) k_ref_targets(const FrameDesc *frames, int nfam, const int64_t *qstart,
                                                     const GpuDetection *dets, const uint32_t *det_ok,
                                                     const uint32_t *qcl, const uint64_t *ckey, int nb,
                                                     RunArrays runs, const uint32_t *row_nruns, RefOrder ref,
                                                     uint32_t *err) {
    __shared__ uint32_t s_key[REF_HASH];
    __shared__ uint32_t s_n, s_need, s_over;
    __shared__ uint32_t s_scan[32];
    const int f = blockIdx.x;
    const FrameDesc fd = frames[f];
    for (int i = threadIdx.x; i < REF_HASH; i += blockDim.x) s_key[i] = 0;
    if (threadIdx.x == 0) s_n = s_need = s_over = 0;
    __syncthreads();
    const int64_t a = qstart[f] * nfam, b = qstart[f + 1] * nfam;
    const uint64_t lmask = ((uint64_t)1 << nb) - 1;
    for (int64_t s = a + threadIdx.x; s < b; s += blockDim.x) {
        if (!det_ok[s]) continue;
        const int32_t id = dets[s].id;
        bool shared = false;
        for (int64_t s2 = a; s2 < b && !shared; s2++) shared = s2 != s && det_ok[s2] && dets[s2].id == id;
        if (!shared) continue;
        s_need = 1;
        const uint64_t key = ckey[qcl[s / nfam]];
        const uint32_t lab[2] = {(uint32_t)(key >> nb), (uint32_t)(key & lmask)};
        for (int k = 0; k < 2; k++) {
            uint32_t h = ref_hash(lab[k]) & (REF_HASH - 1);
            int p = 0;
            for (; p < REF_HASH; p++) {
                const uint32_t old = atomicCAS(&s_key[h], 0u, lab[k] + 1);
                if (old == 0u || old == lab[k] + 1) break;
                h = (h + 1) & (REF_HASH - 1);
            }
            if (p == REF_HASH) s_over = 1;
        }
    }
    __syncthreads();
    uint32_t *tl = ref.tlabel + (int64_t)f * AT_REF_MAXT;
    uint32_t *tp = ref.tpx + (int64_t)f * AT_REF_MAXT;
    for (int i = threadIdx.x; i < REF_HASH; i += blockDim.x) {
        if (!s_key[i]) continue;
        const uint32_t t = atomicAdd(&s_n, 1u);
        if (t >= AT_REF_MAXT) {
            s_over = 1;
            continue;
        }
        const uint32_t label = s_key[i] - 1;
        tl[t] = label;
        tp[t] = runs.px[runs.parent[label]];  // every node points at its root after the unions
    }
    __syncthreads();
    const bool need = s_need && !s_over;
    if (threadIdx.x == 0) {
        ref.need[f] = need ? 1u : 0u;
        ref.nt[f] = need ? s_n : 0u;
        if (s_over) atomicOr(err, AT_ERR_CAPACITY);
    }
    if (!need) return;
    // the reference's packed numbering: runs of the rows above row y
    uint32_t *pre = ref.rpre + fd.row0 + f;
    uint32_t base = 0;
    for (int64_t y0 = 0; y0 < fd.qh; y0 += blockDim.x) {
        const int64_t y = y0 + threadIdx.x;
        const uint32_t c = y < fd.qh ? row_nruns[fd.row0 + y] : 0u;
        uint32_t total;
        const uint32_t off = block_excl_scan(c, &total, s_scan);
        if (y < fd.qh) pre[y] = base + off;
        base += total;
    }
    if (threadIdx.x == 0) pre[fd.qh] = base;
}

// ---------------------------------------------------------------------------
// The target runs of each row, compacted, a warp per row:
//   tlist[node_off + y qw + j] = start | end << 16 | index << 32 | v << 48 | target << 56
//   trow[row0 + y] = count | (the last-column link joins a target run) << 31

__global__ void __launch_bounds__(256) k_ref_mark(const FrameDesc *frames, const uint8_t *thr, RunArrays runs,
                                                  const uint32_t *row_nruns, RefOrder ref) {
    __shared__ uint32_t s_key[REF_HASH];
    __shared__ uint8_t s_idx[REF_HASH];
    const int f = blockIdx.y;
    if (!ref.need[f]) return;
    const FrameDesc fd = frames[f];
    for (int i = threadIdx.x; i < REF_HASH; i += blockDim.x) s_key[i] = 0;
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint32_t nt = ref.nt[f];
        for (uint32_t t = 0; t < nt; t++) {
            const uint32_t label = ref.tlabel[(int64_t)f * AT_REF_MAXT + t];
            uint32_t h = ref_hash(label) & (REF_HASH - 1);
            while (s_key[h]) h = (h + 1) & (REF_HASH - 1);
            s_key[h] = label + 1;
            s_idx[h] = (uint8_t)t;
        }
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t wpb = blockDim.x >> 5;
    for (int64_t y = blockIdx.x * wpb + (threadIdx.x >> 5); y < fd.qh; y += gridDim.x * wpb) {
        const int64_t base = fd.node_off + y * fd.qw;
        const int64_t n = row_nruns[fd.row0 + y];
        uint32_t cnt = 0, last_t = REF_NONE;
        for (int64_t j0 = 0; j0 < n; j0 += 32) {
            const int64_t j = j0 + lane;
            uint32_t t = REF_NONE;
            if (j < n) t = ref_lookup(s_key, s_idx, runs.minid[runs.parent[base + j]]);
            const uint32_t bal = __ballot_sync(0xffffffffu, t != REF_NONE);
            if (t != REF_NONE) {
                const uint64_t e = (uint64_t)runs.start[base + j] | (uint64_t)runs.end[base + j] << 16 |
                                   (uint64_t)j << 32 | (uint64_t)runs.v[base + j] << 48 | (uint64_t)t << 56;
                ref.tlist[base + cnt + __popc(bal & ((1u << lane) - 1u))] = e;
            }
            if (j == n - 1) last_t = t;
            cnt += __popc(bal);
        }
        last_t = __shfl_sync(0xffffffffu, last_t, (int)((n - 1) & 31));
        if (lane == 0) {
            bool link = false;
            if (y >= 1 && n > 0 && last_t != REF_NONE) {
                const int64_t last = base + n - 1;
                const uint8_t *above = thr + fd.q_off + (y - 1) * fd.qw;
                link = runs.end[last] == fd.qw - 2 && runs.v[last] == 255 && above[fd.qw - 1] == 255 &&
                       above[fd.qw - 2] != 255;
            }
            ref.trow[fd.row0 + y] = cnt | (link ? 0x80000000u : 0u);
        }
    }
}

// ---------------------------------------------------------------------------
// The replay, a warp per frame. Its arrays live in shared memory, or for
// very wide frames in a global scratch of the same layout (one region per
// frame); `capr` bounds the runs of a row.

struct ReplayArrays {
    uint32_t *p_se;   // previous row's open target runs: start | end << 16
    uint8_t *p_v;
    uint16_t *p_slot;
    uint32_t *c_se;   // this row's target runs
    uint8_t *c_v, *c_t;
    uint16_t *c_j;
    uint16_t *call_a, *call_b;  // the calls in the reference's order: (run element, slot element)
    uint16_t *e_par, *e_fpar;   // elements: slots [0, m), runs [m, m + n), the last-column node m + n
    uint32_t *e_R, *e_Z, *e_tot, *e_c0, *e_c1;
    unsigned long long *e_max;
    uint8_t *e_flag;
    uint32_t *s_R, *s_Z;        // slots carried to the next row
    uint8_t *s_t;
};

__host__ __device__ inline size_t ref_align(size_t x) { return (x + 15) & ~(size_t)15; }

// Carves the arrays out of `base`; returns the bytes used.
__host__ __device__ inline size_t ref_carve(uint8_t *base, int64_t capr, ReplayArrays *A) {
    const int64_t cape = 2 * capr + 2, capc = 2 * capr + 2;
    size_t at = 0;
    auto take = [&](size_t bytes) {
        uint8_t *p = base + at;
        at = ref_align(at + bytes);
        return p;
    };
    ReplayArrays a;
    a.p_se = (uint32_t *)take(4 * capr);
    a.c_se = (uint32_t *)take(4 * capr);
    a.e_R = (uint32_t *)take(4 * cape);
    a.e_Z = (uint32_t *)take(4 * cape);
    a.e_tot = (uint32_t *)take(4 * cape);
    a.e_c0 = (uint32_t *)take(4 * cape);
    a.e_c1 = (uint32_t *)take(4 * cape);
    a.e_max = (unsigned long long *)take(8 * cape);
    a.s_R = (uint32_t *)take(4 * (capr + 1));
    a.s_Z = (uint32_t *)take(4 * (capr + 1));
    a.p_slot = (uint16_t *)take(2 * capr);
    a.c_j = (uint16_t *)take(2 * capr);
    a.call_a = (uint16_t *)take(2 * capc);
    a.call_b = (uint16_t *)take(2 * capc);
    a.e_par = (uint16_t *)take(2 * cape);
    a.e_fpar = (uint16_t *)take(2 * cape);
    a.p_v = take(capr);
    a.c_v = take(capr);
    a.c_t = take(capr);
    a.e_flag = take(cape);
    a.s_t = take(capr + 1);
    if (A) *A = a;
    return at;
}

size_t ref_replay_bytes(int64_t capr) { return ref_carve(nullptr, capr, nullptr); }

__device__ __forceinline__ uint32_t el_find(volatile uint16_t *par, uint32_t x) {
    uint32_t p = par[x];
    while (p != x) {
        const uint32_t pp = par[p];
        if (pp != p) par[x] = (uint16_t)pp;  // path halving: only ever an ancestor
        x = p;
        p = par[x];
    }
    return x;
}

// Connectivity only (the group of each element): lock-free hooking of the
// larger root under the smaller.
__device__ __forceinline__ void el_unite(uint16_t *par, uint32_t a, uint32_t b) {
    volatile uint16_t *vp = par;
    for (;;) {
        a = el_find(vp, a);
        b = el_find(vp, b);
        if (a == b) return;
        if (a < b) {
            const uint32_t t = a;
            a = b;
            b = t;
        }
        // 16-bit CAS on the aligned 32-bit word that holds par[a]
        uint32_t *word = reinterpret_cast<uint32_t *>(reinterpret_cast<uintptr_t>(par + a) & ~(uintptr_t)3);
        const int sh = (reinterpret_cast<uintptr_t>(par + a) & 2) ? 16 : 0;
        uint32_t old = *(volatile uint32_t *)word;
        if (((old >> sh) & 0xffffu) != a) continue;
        const uint32_t nw = (old & ~(0xffffu << sh)) | (b << sh);
        if (atomicCAS(word, old, nw) == old) return;
    }
}

__device__ __forceinline__ uint32_t fold_find(const uint16_t *par, uint32_t x) {
    while (par[x] != x) x = par[x];
    return x;
}

__global__ void __launch_bounds__(32) k_ref_replay(const FrameDesc *frames, RefOrder ref, int64_t capr,
                                                   uint8_t *scratch, size_t scratch_per_frame, uint32_t *err) {
    extern __shared__ __align__(16) uint8_t s_mem[];
    __shared__ uint8_t s_done[AT_REF_MAXT];
    __shared__ uint32_t s_ndone;
    const int f = blockIdx.x;
    if (!ref.need[f]) return;
    const int lane = threadIdx.x;
    const uint32_t lt = (1u << lane) - 1u;
    const FrameDesc fd = frames[f];
    ReplayArrays A;
    ref_carve(scratch ? scratch + (size_t)f * scratch_per_frame : s_mem, capr, &A);
    const uint32_t nt = ref.nt[f];
    const uint32_t *tpx = ref.tpx + (int64_t)f * AT_REF_MAXT;
    uint32_t *troot = ref.troot + (int64_t)f * AT_REF_MAXT;
    for (uint32_t t = lane; t < AT_REF_MAXT; t += 32) s_done[t] = t < nt ? 0 : 1;
    if (lane == 0) s_ndone = 0;
    __syncwarp();
    const uint32_t vbase = (uint32_t)(fd.node_off + (int64_t)fd.qw * fd.qh);
    int64_t m = 0, np = 0;  // slots carried, open target runs of the previous row
    for (int64_t y = 0; y < fd.qh && s_ndone < nt; y++) {
        const uint32_t tr = ref.trow[fd.row0 + y];
        const int64_t nraw = tr & 0x7fffffffu;
        if (nraw == 0 && np == 0) continue;  // nothing open above, nothing here: m is 0 too
        const uint32_t rbase = (uint32_t)(fd.node_off + y * fd.qw);
        // this row's target runs whose component is still open
        int64_t n = 0;
        bool last_kept = false;
        for (int64_t j0 = 0; j0 < nraw; j0 += 32) {
            const int64_t j = j0 + lane;
            uint64_t e = 0;
            bool keep = false;
            if (j < nraw) {
                e = ref.tlist[rbase + j];
                keep = !s_done[e >> 56];
            }
            const uint32_t bal = __ballot_sync(0xffffffffu, keep);
            if (keep) {
                const int64_t o = n + __popc(bal & lt);
                A.c_se[o] = (uint32_t)e;
                A.c_v[o] = (uint8_t)(e >> 48);
                A.c_j[o] = (uint16_t)(e >> 32);
                A.c_t[o] = (uint8_t)(e >> 56);
            }
            if (j == nraw - 1) last_kept = keep;
            n += __popc(bal);
        }
        last_kept = __shfl_sync(0xffffffffu, last_kept, (int)((nraw - 1) & 31)) && nraw > 0;
        const bool link = (tr >> 31) && last_kept;
        const int64_t E = m + n + 1, vn = m + n;
        __syncwarp();
        for (int64_t e = lane; e < E; e += 32) {
            A.e_par[e] = (uint16_t)e;
            A.e_fpar[e] = (uint16_t)e;
            A.e_tot[e] = 0;
            A.e_max[e] = 0;
            A.e_c0[e] = 0xffffffffu;
            A.e_c1[e] = 0;
            if (e < m) {
                A.e_R[e] = A.s_R[e];
                A.e_Z[e] = A.s_Z[e];
                A.e_flag[e] = 0;
            } else if (e < vn) {
                const uint32_t se = A.c_se[e - m];
                A.e_R[e] = rbase + A.c_j[e - m];
                A.e_Z[e] = (se >> 16) - (se & 0xffffu) + 1;
                A.e_flag[e] = REF_TOUCHED;
            } else {
                A.e_R[e] = vbase + (uint32_t)(y - 1);
                A.e_Z[e] = 1;
                A.e_flag[e] = link ? REF_TOUCHED : 0;
            }
        }
        // the calls, in the reference's order: each run, its touching runs
        // above in order (fast/unionfind.c:112-196), then the last column
        int64_t nc = 0;
        if (np > 0) {
            for (int64_t i0 = 0; i0 < n; i0 += 32) {
                const int64_t i = i0 + lane;
                int64_t k0 = 0, cnt = 0;
                int64_t a0 = 0, a1 = 0;
                uint8_t v = 0;
                if (i < n) {
                    a0 = A.c_se[i] & 0xffffu;
                    a1 = A.c_se[i] >> 16;
                    v = A.c_v[i];
                    int64_t lo = 0, hi = np;
                    while (lo < hi) {
                        const int64_t mid = (lo + hi) >> 1;
                        if ((int64_t)(A.p_se[mid] >> 16) + 1 < a0)
                            lo = mid + 1;
                        else
                            hi = mid;
                    }
                    k0 = lo;
                    for (int64_t k = k0; k < np && (int64_t)(A.p_se[k] & 0xffffu) <= a1 + 1; k++)
                        if (A.p_v[k] == v && runs_touch(a0, a1, A.p_se[k] & 0xffffu, A.p_se[k] >> 16, v)) cnt++;
                }
                uint32_t incl = (uint32_t)cnt;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += t;
                }
                const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
                if (nc + total + 1 > 2 * capr + 2) {  // more calls than the arrays hold
                    if (lane == 0) atomicOr(err, AT_ERR_ORDER);
                    return;
                }
                int64_t o = nc + incl - cnt;
                if (i < n)
                    for (int64_t k = k0; k < np && (int64_t)(A.p_se[k] & 0xffffu) <= a1 + 1; k++)
                        if (A.p_v[k] == v && runs_touch(a0, a1, A.p_se[k] & 0xffffu, A.p_se[k] >> 16, v)) {
                            A.call_a[o] = (uint16_t)(m + i);
                            A.call_b[o] = A.p_slot[k];
                            o++;
                        }
                nc += total;
            }
        }
        if (link) {
            if (lane == 0) {
                A.call_a[nc] = (uint16_t)(vn - 1);
                A.call_b[nc] = (uint16_t)vn;
            }
            nc++;
        }
        __syncwarp();
        // groups
        for (int64_t c = lane; c < nc; c += 32) {
            el_unite(A.e_par, A.call_a[c], A.call_b[c]);
            A.e_flag[A.call_b[c]] = REF_TOUCHED;
        }
        __syncwarp();
        // every element's group root (read-only walks into e_tot, then
        // copied: a halving write racing a final write could leave a
        // non-root parent)
        for (int64_t e = lane; e < E; e += 32) {
            uint32_t x = (uint32_t)e;
            while (A.e_par[x] != x) x = A.e_par[x];
            A.e_tot[e] = x;
        }
        __syncwarp();
        for (int64_t e = lane; e < E; e += 32) {
            A.e_par[e] = (uint16_t)A.e_tot[e];
            A.e_tot[e] = 0;
        }
        __syncwarp();
        // per group: pixels, the largest set that existed before the row,
        // and the range of its calls
        for (int64_t e = lane; e < E; e += 32) {
            if (!A.e_flag[e]) continue;
            const uint32_t g = A.e_par[e];
            atomicAdd(&A.e_tot[g], A.e_Z[e]);
            if (e < m || e == vn) atomicMax(&A.e_max[g], (unsigned long long)A.e_Z[e] << 16 | (uint64_t)e);
        }
        for (int64_t c = lane; c < nc; c += 32) {
            const uint32_t g = A.e_par[A.call_a[c]];
            atomicMin(&A.e_c0[g], (uint32_t)c);
            atomicMax(&A.e_c1[g], (uint32_t)c);
        }
        __syncwarp();
        // each group's root and pixels, into its root element
        for (int64_t g = lane; g < E; g += 32) {
            if (!A.e_flag[g] || A.e_par[g] != g) continue;
            const unsigned long long mx = A.e_max[g];
            const uint32_t zmax = (uint32_t)(mx >> 16), tot = A.e_tot[g];
            if (mx != 0 && zmax > tot - zmax) {
                A.e_R[g] = A.e_R[mx & 0xffffu];
                A.e_Z[g] = tot;
                continue;
            }
            // no set outweighs the rest: the reference's calls one by one
            for (uint32_t c = A.e_c0[g]; c <= A.e_c1[g] && c < (uint32_t)nc; c++) {
                const uint32_t a = A.call_a[c];
                if (A.e_par[a] != g) continue;
                const uint32_t ra = fold_find(A.e_fpar, a), rb = fold_find(A.e_fpar, A.call_b[c]);
                if (ra == rb) continue;
                const uint32_t za = A.e_Z[ra], zb = A.e_Z[rb];
                if (za > zb) {
                    A.e_fpar[rb] = (uint16_t)ra;
                    A.e_Z[ra] = za + zb;
                } else {
                    A.e_fpar[ra] = (uint16_t)rb;
                    A.e_Z[rb] = za + zb;
                }
            }
            const uint32_t r = fold_find(A.e_fpar, (uint32_t)g);
            const uint32_t R = A.e_R[r], Z = A.e_Z[r];
            A.e_R[g] = R;
            A.e_Z[g] = Z;
        }
        __syncwarp();
        // a slot no call reached is a whole component: its root is final
        for (int64_t e = lane; e < m; e += 32) {
            const uint32_t t = A.s_t[e];
            if (A.e_flag[e] || t == REF_NONE || s_done[t]) continue;
            troot[t] = A.s_R[e];
            s_done[t] = 1;
            atomicAdd(&s_ndone, 1u);
        }
        // the new slots: one per group of this row's runs, numbered by its
        // first run (e_tot of the root is free again and holds that run)
        for (int64_t i = lane; i < n; i += 32) A.e_tot[A.e_par[m + i]] = 0xffffffffu;
        __syncwarp();
        for (int64_t i = lane; i < n; i += 32) atomicMin(&A.e_tot[A.e_par[m + i]], (uint32_t)i);
        __syncwarp();
        int64_t mnew = 0;
        for (int64_t i0 = 0; i0 < n; i0 += 32) {
            const int64_t i = i0 + lane;
            uint32_t g = 0;
            bool first = false;
            if (i < n) {
                g = A.e_par[m + i];
                first = A.e_tot[g] == (uint32_t)i;
            }
            const uint32_t bal = __ballot_sync(0xffffffffu, first);
            if (first) {
                const int64_t k = mnew + __popc(bal & lt);
                A.e_c0[g] = (uint32_t)k;  // the group's new slot
                const uint32_t t = A.c_t[i], Z = A.e_Z[g];
                A.s_R[k] = A.e_R[g];
                A.s_Z[k] = Z;
                A.s_t[k] = (uint8_t)t;
                // more than half of the component: no later call can move the root
                if (!s_done[t] && Z > tpx[t] - Z) {
                    troot[t] = A.e_R[g];
                    s_done[t] = 1;
                    atomicAdd(&s_ndone, 1u);
                }
            }
            mnew += __popc(bal);
        }
        __syncwarp();
        // the open runs of this row, with their slots, for the next row
        int64_t npn = 0;
        for (int64_t i0 = 0; i0 < n; i0 += 32) {
            const int64_t i = i0 + lane;
            const bool keep = i < n && !s_done[A.c_t[i]];
            const uint32_t bal = __ballot_sync(0xffffffffu, keep);
            if (keep) {
                const int64_t o = npn + __popc(bal & lt);
                A.p_se[o] = A.c_se[i];
                A.p_v[o] = A.c_v[i];
                A.p_slot[o] = (uint16_t)A.e_c0[A.e_par[m + i]];
            }
            npn += __popc(bal);
        }
        m = mnew;
        np = npn;
        __syncwarp();
    }
    // the sets still open at the bottom are whole components
    for (int64_t k = lane; k < m; k += 32) {
        const uint32_t t = A.s_t[k];
        if (t == REF_NONE || s_done[t]) continue;
        troot[t] = A.s_R[k];
        s_done[t] = 1;
    }
    __syncwarp();
    // GPU node ids -> the reference's packed node numbers (a target left
    // without a root keeps 0xffffffff, which the final stage reports)
    const uint32_t *pre = ref.rpre + fd.row0 + f;
    for (uint32_t t = lane; t < nt; t += 32) {
        if (troot[t] == 0xffffffffu) continue;
        const int64_t nd = (int64_t)troot[t] - fd.node_off;
        const int64_t qpx = (int64_t)fd.qw * fd.qh;
        troot[t] = nd < qpx ? pre[nd / fd.qw] + (uint32_t)(nd % fd.qw) : pre[fd.qh] + (uint32_t)(nd - qpx);
    }
}

// ---------------------------------------------------------------------------
// Launchers.

void launch_ref_order(const Launch &L, const FrameDesc *frames, const uint8_t *thr, RunArrays runs,
                      const uint32_t *row_nruns, int nfam, const int64_t *qstart, const GpuDetection *dets,
                      const uint32_t *det_ok, const uint32_t *qcl, const uint64_t *ckey, int nb, int64_t capr,
                      uint8_t *scratch, size_t scratch_per_frame, const RefOrder &ref, uint32_t *err) {
    k_ref_targets<<<L.nframes, 256, 0, L.stream>>>(frames, nfam, qstart, dets, det_ok, qcl, ckey, nb, runs, row_nruns,
                                                   ref, err);
    const int64_t b = (L.max_qh + 7) / 8;
    const dim3 grid((unsigned)(b < 1 ? 1 : b < 148 ? b : 148), (unsigned)L.nframes);
    k_ref_mark<<<grid, 256, 0, L.stream>>>(frames, thr, runs, row_nruns, ref);
    const size_t smem = scratch ? 0 : ref_replay_bytes(capr);
    k_ref_replay<<<L.nframes, 32, smem, L.stream>>>(frames, ref, capr, scratch, scratch_per_frame, err);
}

bool ref_replay_set_smem(size_t bytes) {
    return cudaFuncSetAttribute(k_ref_replay, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) ==
           cudaSuccess;
}
