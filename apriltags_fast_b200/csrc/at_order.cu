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
//   k_ref_targets   per frame: the ids that two or more detections share;
//                   the components of their quads are the targets (their
//                   GPU labels and pixel counts); the packed run numbering.
//   k_ref_mark      the runs of the target components, row by row, compacted
//                   (start, end, index in row, value, target).
//   k_ref_cut       the rows of each frame in bands.
//   k_ref_local     the band's own components of target runs (all bands at
//                   once), summarised by those reaching its top and bottom.
//   k_ref_frontier  per frame, band after band: the sets of target runs at
//                   each band's upper edge as the reference has them there.
//   k_ref_band      a warp per band replays the reference's unions of the
//                   band's target runs (see below), the incoming sets'
//                   roots as symbols.
//   k_ref_resolve   per frame: the symbols resolved from the top down.
//   k_finalize      (at_kernels.cu) orders those detections by the keys.
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
// The replay of a band of rows, a warp each. Its arrays live in shared
// memory, or for very wide frames in a global scratch of the same layout
// (one region per block); `capr` bounds the runs of a row.

struct ReplayArrays {
    uint32_t *p_se;   // previous row's open target runs: start | end << 16
    uint8_t *p_v;
    uint16_t *p_slot;
    uint32_t *c_se;   // this row's target runs
    uint32_t *c_tch;  //   the range of runs above each touches (first | last << 16; 0xffff: none)
    uint8_t *c_v, *c_t;
    uint16_t *c_j;
    uint16_t *r_slot; //   the first slot each touches (0xffff: none)
    uint16_t *r_key;  //   its group key: the group's root slot, or m + i when it touches none
    // per slot (m): the union-find of the row's groups, each slot's group,
    // whether a run touches it; per group root: its slots' pixels, its
    // runs' pixels, its largest slot (pixels << 16 | slot)
    uint16_t *e_par, *e_grp;
    uint8_t *e_flag;
    uint32_t *e_c1, *e_tot;
    unsigned long long *e_max;
    // per element (slots [0, m), runs m + i): the call-by-call replay's
    // union-find, roots and pixels; per group key: its first run, and its
    // root and pixels after the row
    uint16_t *e_fpar;
    uint32_t *e_R, *e_Z, *e_c0, *f_R, *f_Z;
    uint32_t *s_R, *s_Z;        // slots carried to the next row
    uint8_t *s_t;
};

__host__ __device__ inline size_t ref_align(size_t x) { return (x + 15) & ~(size_t)15; }

// Carves the arrays out of `base`; returns the bytes used.
__host__ __device__ inline size_t ref_carve(uint8_t *base, int64_t capr, ReplayArrays *A) {
    const int64_t cape = 2 * capr + 2, caps = capr + 1;
    size_t at = 0;
    auto take = [&](size_t bytes) {
        uint8_t *p = base + at;
        at = ref_align(at + bytes);
        return p;
    };
    ReplayArrays a;
    a.p_se = (uint32_t *)take(4 * capr);
    a.c_se = (uint32_t *)take(4 * capr);
    a.c_tch = (uint32_t *)take(4 * capr);
    a.e_R = (uint32_t *)take(4 * cape);
    a.e_Z = (uint32_t *)take(4 * cape);
    a.e_c0 = (uint32_t *)take(4 * cape);
    a.f_R = (uint32_t *)take(4 * cape);
    a.f_Z = (uint32_t *)take(4 * cape);
    a.e_tot = (uint32_t *)take(4 * caps);
    a.e_c1 = (uint32_t *)take(4 * caps);
    a.e_max = (unsigned long long *)take(8 * caps);
    a.s_R = (uint32_t *)take(4 * caps);
    a.s_Z = (uint32_t *)take(4 * caps);
    a.p_slot = (uint16_t *)take(2 * capr);
    a.c_j = (uint16_t *)take(2 * capr);
    a.r_slot = (uint16_t *)take(2 * capr);
    a.r_key = (uint16_t *)take(2 * capr);
    a.e_par = (uint16_t *)take(2 * caps);
    a.e_grp = (uint16_t *)take(2 * caps);
    a.e_fpar = (uint16_t *)take(2 * cape);
    a.p_v = take(capr);
    a.c_v = take(capr);
    a.c_t = take(capr);
    a.e_flag = take(caps);
    a.s_t = take(caps);
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

// Roots in the band replay: a node id, or REF_SYM | j, "the root of the
// band's incoming slot j" (known only once the bands above are resolved).
#define REF_SYM 0x80000000u

// The state between rows of a band's replay: m slots (the sets of target
// runs that touch the previous row: s_R, s_Z, s_t) and the previous row's
// np target runs (p_*, each with its slot).
struct RowState {
    int m, np;
};

// Adds `val` to arr[key] for the active lanes, one atomic per distinct key
// in the warp. Every lane of the warp calls it.
__device__ __forceinline__ void warp_add_by_key(uint32_t *arr, uint32_t key, uint32_t val, bool active) {
    const uint32_t am = __ballot_sync(0xffffffffu, active);
    if (!active) return;
    const uint32_t peers = __match_any_sync(am, key);
    const uint32_t sum = __reduce_add_sync(peers, val);
    if ((int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&arr[key], sum);
}

__device__ __forceinline__ uint32_t run_len(uint32_t se) { return (se >> 16) - (se & 0xffffu) + 1; }

// A row of the reference's calls (fast/unionfind.c:112-196): each run of
// the row in order, with each run above it touches, in order; then the
// last-column link. A run joins the sets (slots) of the runs it touches, so
// the row's groups are the slots joined through runs that touch several
// slots, each with the runs that touch it, and the runs that touch none
// (each alone). A group in which one slot holds more pixels than all its
// other slots and runs together keeps that slot's root, whatever the order
// (that slot is the b side of each call it meets and wins: the a side
// needs strictly more). Any other group is replayed call by call by one
// lane. The link then joins one pixel to the last run's set, taking the
// root only from a set of one pixel.
__device__ __forceinline__ void replay_row(ReplayArrays &A, RowState &S, int n, bool link, uint32_t rbase,
                                           uint32_t vnode, uint32_t *fin, uint32_t *finb, uint32_t band) {
    const int lane = threadIdx.x & 31;
    const uint32_t lt = (1u << lane) - 1u;
    const int m = S.m;
    // slots: their own set (union-find over slots), roots and sizes for
    // the call-by-call replays, sums per group
    for (int s = lane; s < m; s += 32) {
        A.e_par[s] = (uint16_t)s;
        A.e_fpar[s] = (uint16_t)s;
        A.e_R[s] = A.s_R[s];
        A.e_Z[s] = A.s_Z[s];
        A.e_flag[s] = 0;
        A.e_tot[s] = 0;
        A.e_c1[s] = 0;
        A.e_max[s] = 0;
    }
    for (int e = lane; e < m + n; e += 32) A.e_c0[e] = 0xffffffffu;
    __syncwarp();
    // each run: the first slot it touches (r_slot, 0xffff: none); the
    // slots a run touches are joined
    for (int i = lane; i < n; i += 32) {
        uint32_t s1 = 0xffffu;
        const uint32_t tc = A.c_tch[i];
        const uint8_t v = A.c_v[i];
        if ((tc & 0xffffu) != 0xffffu)
            for (uint32_t k = tc & 0xffffu; k <= (tc >> 16); k++)
                if (A.p_v[k] == v) {
                    const uint32_t s = A.p_slot[k];
                    A.e_flag[s] = REF_TOUCHED;
                    if (s1 == 0xffffu)
                        s1 = s;
                    else if (s != s1)
                        el_unite(A.e_par, s1, s);
                }
        A.r_slot[i] = (uint16_t)s1;
    }
    __syncwarp();
    // each slot's group (its root slot)
    for (int s = lane; s < m; s += 32) {
        uint32_t x = (uint32_t)s;
        while (A.e_par[x] != x) x = A.e_par[x];
        A.e_grp[s] = (uint16_t)x;
    }
    __syncwarp();
    // per group: the pixels of its slots and of its runs, its largest slot;
    // per key (group root slot g, or m + i for a run that touches none,
    // r_key[i] for run i): its first run
    for (int s = lane; s < m; s += 32)
        if (A.e_flag[s]) {
            const uint32_t g = A.e_grp[s];
            atomicAdd(&A.e_c1[g], A.s_Z[s]);
            atomicMax(&A.e_max[g], (unsigned long long)A.s_Z[s] << 16 | (uint64_t)s);
        }
    for (int i0 = 0; i0 < n; i0 += 32) {
        const int i = i0 + lane;
        uint32_t key = 0, z = 0;
        bool touched = false;
        if (i < n) {
            const uint32_t s = A.r_slot[i];
            touched = s != 0xffffu;
            key = touched ? A.e_grp[s] : (uint32_t)(m + i);
            z = run_len(A.c_se[i]);
            A.r_key[i] = (uint16_t)key;
            atomicMin(&A.e_c0[key], (uint32_t)i);
        }
        warp_add_by_key(A.e_tot, key, z, touched);
    }
    __syncwarp();
    // each group's root and pixels after the row (f_R, f_Z at its key)
    for (int g = lane; g < m; g += 32) {
        if (!A.e_flag[g] || A.e_grp[g] != g) continue;
        const unsigned long long mx = A.e_max[g];
        const uint32_t zmax = (uint32_t)(mx >> 16), tot = A.e_c1[g] + A.e_tot[g];
        uint32_t R, Z;
        if (zmax > tot - zmax) {
            R = A.s_R[mx & 0xffffu];
            Z = tot;
        } else {  // the group's calls one by one
            for (int i = (int)A.e_c0[g]; i < n; i++) {
                if (A.r_key[i] != g) continue;
                const uint32_t a = (uint32_t)(m + i);
                A.e_fpar[a] = (uint16_t)a;
                A.e_Z[a] = run_len(A.c_se[i]);
                A.e_R[a] = rbase + A.c_j[i];
                const uint32_t tc = A.c_tch[i];
                const uint8_t v = A.c_v[i];
                for (uint32_t k = tc & 0xffffu; k <= (tc >> 16); k++) {
                    if (A.p_v[k] != v) continue;
                    const uint32_t ra = fold_find(A.e_fpar, a), rb = fold_find(A.e_fpar, A.p_slot[k]);
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
            }
            const uint32_t r = fold_find(A.e_fpar, (uint32_t)g);
            R = A.e_R[r];
            Z = A.e_Z[r];
        }
        A.f_R[g] = R;
        A.f_Z[g] = Z;
    }
    // a slot no run touches is a whole component: its root is final
    for (int s = lane; s < m; s += 32) {
        const uint32_t t = A.s_t[s];
        if (A.e_flag[s] || t == REF_NONE) continue;
        fin[t] = A.s_R[s];
        finb[t] = band;
    }
    for (int i = lane; i < n; i += 32)
        if (A.r_slot[i] == 0xffffu) {
            A.f_R[m + i] = rbase + A.c_j[i];
            A.f_Z[m + i] = run_len(A.c_se[i]);
        }
    __syncwarp();
    // the last-column link
    if (link && lane == 0) {
        const uint32_t key = A.r_key[n - 1];
        const uint32_t Z = A.f_Z[key];
        if (Z <= 1) A.f_R[key] = vnode;
        A.f_Z[key] = Z + 1;
    }
    __syncwarp();
    // the new slots, numbered by first run
    int mnew = 0;
    for (int i0 = 0; i0 < n; i0 += 32) {
        const int i = i0 + lane;
        uint32_t key = 0;
        bool first = false;
        if (i < n) {
            key = A.r_key[i];
            first = A.e_c0[key] == (uint32_t)i;
        }
        const uint32_t bal = __ballot_sync(0xffffffffu, first);
        if (first) {
            const int k = mnew + __popc(bal & lt);
            A.s_R[k] = A.f_R[key];
            A.s_Z[k] = A.f_Z[key];
            A.s_t[k] = A.c_t[i];
            A.e_c0[key] = 0x80000000u | (uint32_t)k;
        }
        mnew += __popc(bal);
    }
    __syncwarp();
    // this row's runs, with their slots, for the next row
    for (int i = lane; i < n; i += 32) {
        A.p_se[i] = A.c_se[i];
        A.p_v[i] = A.c_v[i];
        A.p_slot[i] = (uint16_t)(A.e_c0[A.r_key[i]] & 0xffffu);
    }
    S.m = mnew;
    S.np = n;
    __syncwarp();
}

// ---------------------------------------------------------------------------
// Bands. The rows of a frame go in bands (at most REF_BAND rows and pcap
// target runs each), replayed in parallel. A band's replay needs the sets
// of target runs that touch the row above it as the reference has them
// there, with their pixel counts. Which runs are together and how many
// pixels a set holds do not depend on which root wins, so these come from
// an order-free union-find in two steps: k_ref_local joins the runs inside
// each band (all bands at once) and summarises the band by its components
// that reach its top and bottom rows; k_ref_frontier then walks the bands
// of a frame from the top joining only those summaries. A band's replay
// carries the incoming sets' roots as symbols, and k_ref_resolve puts the
// roots in from the top down.
//
// Per band b (at row0 + frame + b): bstart[b] its first row (and the end
// after the last band), bwide[b] the most target runs of one of its rows or
// of the row above, desc[b] = (first row, end row, components reaching the
// top | others reaching the bottom << 16, runs of the top row | of the
// bottom row << 16). Node-indexed arrays, at the nodes of a row y
// (node_off + y qw + i):
//   ltop[j]    top row of a band: the band component of target run j,
//              numbered by first run among the components that reach it
//   lpx[c]     top row: pixels of band component c
//   lbot[j]    bottom row: run j's component, c (one reaching the top row)
//              or 0x80000000 | k (the k-th of the others)
//   lpx2[k]    bottom row: pixels of the k-th other component
//   bslot[j]   row above a band: the slot (prefix set) of target run j
//   binfo[s]   row above a band: slot s, pixels | first run << 32 |
//              target << 48
//   outroot[s] row above a band: the root of slot s's set after the band
//              above (a node or a symbol of that band)
// and per row: bm[y] the slots at the row above a band.

#define REF_KNONE 0x3fffffffu  // no run yet: above every run index, below the flags
#define REF_KTOP 0x80000000u   // numbered: the component's index
#define REF_KBOT 0x40000000u

__device__ __forceinline__ uint32_t pu_find(volatile uint32_t *par, uint32_t x) {
    uint32_t p = par[x];
    while (p != x) {
        const uint32_t pp = par[p];
        if (pp != p) par[x] = pp;
        x = p;
        p = par[x];
    }
    return x;
}

// Lock-free hooking of the larger root under the smaller (connectivity only).
__device__ __forceinline__ void pu_unite(uint32_t *par, uint32_t a, uint32_t b) {
    volatile uint32_t *vp = par;
    for (;;) {
        a = pu_find(vp, a);
        b = pu_find(vp, b);
        if (a == b) return;
        if (a < b) {
            const uint32_t t = a;
            a = b;
            b = t;
        }
        if (atomicCAS(par + a, a, b) == a) return;
    }
}

// The first index in runs [lo, hi) (start | end << 16, sorted) whose end
// reaches column a0 - 1.
__device__ __forceinline__ uint32_t first_reaching(const uint32_t *se, uint32_t lo, uint32_t hi, int64_t a0) {
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if ((int64_t)(se[mid] >> 16) + 1 < a0)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// Asynchronous global -> shared copies (sm_80 and later), for staging the
// next row or band while the current one is worked on.
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// The band cut of each frame, a warp per frame: the rows in blocks of
// REF_BAND, each block one band, or several when its target runs exceed
// pcap (cut greedily, whole rows). bwide[b]: the most target runs in a row
// of band b or in the row above it (the replay's row capacity).
__global__ void __launch_bounds__(32) k_ref_cut(const FrameDesc *frames, RefOrder ref, uint32_t pcap) {
    const int f = blockIdx.x;
    if (!ref.need[f]) return;
    const FrameDesc fd = frames[f];
    const int lane = threadIdx.x;
    uint32_t *bs = ref.bstart + fd.row0 + f, *bw = ref.bwide + fd.row0 + f;
    const uint32_t *tr = ref.trow + fd.row0;
    const int64_t nblk = (fd.qh + REF_BAND - 1) / REF_BAND;
    uint32_t base = 0;
    for (int64_t k0 = 0; k0 < nblk; k0 += 32) {
        const int64_t k = k0 + lane;
        const int64_t y0 = k * REF_BAND;
        const int nr = k < nblk ? (int)(fd.qh - y0 < REF_BAND ? fd.qh - y0 : REF_BAND) : 0;
        uint32_t c[REF_BAND];
        uint32_t above = 0, nbk = 0, acc = 0;
        if (nr > 0 && y0 > 0) above = tr[y0 - 1] & 0x7fffffffu;
#pragma unroll
        for (int r = 0; r < REF_BAND; r++) c[r] = r < nr ? (tr[y0 + r] & 0x7fffffffu) : 0u;
#pragma unroll
        for (int r = 0; r < REF_BAND; r++)
            if (r < nr) {
                if (r == 0 || acc + c[r] > pcap) {
                    nbk++;
                    acc = 0;
                }
                acc += c[r];
            }
        uint32_t total;
        const uint32_t off = warp_excl_scan(nbk, &total);
        if (nr > 0) {
            uint32_t bi = base + off, wide = 0;
            acc = 0;
#pragma unroll
            for (int r = 0; r < REF_BAND; r++)
                if (r < nr) {
                    if (r == 0 || acc + c[r] > pcap) {
                        if (r > 0) bw[bi++] = wide;
                        bs[bi] = (uint32_t)(y0 + r);
                        acc = 0;
                        wide = r == 0 ? above : c[r - 1];
                    }
                    acc += c[r];
                    wide = wide > c[r] ? wide : c[r];
                }
            bw[bi] = wide;
        }
        base += total;
    }
    if (lane == 0) {
        bs[base] = (uint32_t)fd.qh;
        ref.nband[f] = base;
    }
}

// The shared-memory layout of k_ref_local: pcap runs and a last-column
// node per row.
struct LocalArrays {
    uint32_t *se, *par, *Z, *tot, *key;
    uint8_t *v;
};
__host__ __device__ inline size_t ref_local_carve(uint8_t *base, int64_t pcap, LocalArrays *A) {
    const int64_t cape = pcap + REF_BAND;
    size_t at = 0;
    auto take = [&](size_t bytes) {
        uint8_t *p = base + at;
        at = ref_align(at + bytes);
        return p;
    };
    LocalArrays a;
    a.se = (uint32_t *)take(4 * pcap);
    a.par = (uint32_t *)take(4 * cape);
    a.Z = (uint32_t *)take(4 * cape);
    a.tot = (uint32_t *)take(4 * cape);
    a.key = (uint32_t *)take(4 * cape);
    a.v = take(pcap);
    if (A) *A = a;
    return at;
}
size_t ref_local_bytes(int64_t pcap) { return ref_local_carve(nullptr, pcap, nullptr); }

// A block per band (the frame's bands taken in turn by its blocks): the
// band's components, their pixels, and the summaries named above.
__global__ void __launch_bounds__(256) k_ref_local(const FrameDesc *frames, RefOrder ref, uint32_t pcap,
                                                   uint32_t *err) {
    extern __shared__ __align__(16) uint8_t s_mem[];
    __shared__ uint32_t s_roff[REF_BAND + 1];
    __shared__ uint8_t s_link[REF_BAND];
    __shared__ uint32_t s_ntop, s_nnon;
    const int f = blockIdx.y;
    if (!ref.need[f]) return;
    const FrameDesc fd = frames[f];
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31;
    const uint32_t lt = (1u << lane) - 1u;
    LocalArrays A;
    ref_local_carve(s_mem, pcap, &A);
    const uint32_t *bs = ref.bstart + fd.row0 + f;
    const int64_t nb = ref.nband[f];
    for (int64_t b = blockIdx.x; b < nb; b += gridDim.x) {
        const int64_t y0 = bs[b], y1 = bs[b + 1];
        const int nr = (int)(y1 - y0);
        if (tid < 32) {
            uint32_t c = 0, lk = 0;
            if (tid < nr) {
                const uint32_t tr = ref.trow[fd.row0 + y0 + tid];
                c = tr & 0x7fffffffu;
                lk = tr >> 31;
            }
            uint32_t total;
            const uint32_t off = warp_excl_scan(c, &total);
            if (tid < nr) {
                s_roff[tid] = off;
                s_link[tid] = (uint8_t)lk;
            }
            if (tid == 0) s_roff[nr] = total;
        }
        __syncthreads();
        const uint32_t L = s_roff[nr];
        if (L > pcap) {  // the cut keeps bands within pcap when a row fits
            if (tid == 0) atomicOr(err, AT_ERR_ORDER);
            return;
        }
        const int64_t E = L + nr;
        // elements: the band's runs [0, L), then the last-column node of
        // each row's link [L, L + nr)
        for (uint32_t l = tid; l < L; l += nt) {
            int r = 0;
            while (s_roff[r + 1] <= l) r++;
            const uint64_t e = ref.tlist[fd.node_off + (y0 + r) * fd.qw + (l - s_roff[r])];
            A.se[l] = (uint32_t)e;
            A.v[l] = (uint8_t)(e >> 48);
            A.par[l] = l;
            A.Z[l] = (((uint32_t)e >> 16) & 0xffffu) - ((uint32_t)e & 0xffffu) + 1;
            A.tot[l] = 0;
            A.key[l] = REF_KNONE;
        }
        for (int r = tid; r < nr; r += nt) {
            A.par[L + r] = L + r;
            A.Z[L + r] = s_link[r] ? 1u : 0u;
            A.tot[L + r] = 0;
            A.key[L + r] = REF_KNONE;
        }
        __syncthreads();
        for (uint32_t l = tid; l < L; l += nt) {
            int r = 0;
            while (s_roff[r + 1] <= l) r++;
            if (r == 0) continue;
            const int64_t a0 = A.se[l] & 0xffffu, a1 = A.se[l] >> 16;
            const uint8_t v = A.v[l];
            const uint32_t lo = s_roff[r - 1], hi = s_roff[r];
            uint32_t klo = 0xffffu, khi = 0;
            for (uint32_t k = first_reaching(A.se, lo, hi, a0); k < hi && (int64_t)(A.se[k] & 0xffffu) <= a1 + 1; k++)
                if (A.v[k] == v && runs_touch(a0, a1, A.se[k] & 0xffffu, A.se[k] >> 16, v)) {
                    pu_unite(A.par, l, k);
                    if (klo == 0xffffu) klo = k - lo;
                    khi = k - lo;
                }
            // the runs above that this run touches, for the replay
            ref.tch[fd.node_off + (y0 + r) * fd.qw + (l - s_roff[r])] = klo == 0xffffu ? 0xffffffffu : klo | khi << 16;
        }
        for (int r = tid; r < nr; r += nt)
            if (s_link[r] && s_roff[r + 1] > s_roff[r]) pu_unite(A.par, s_roff[r + 1] - 1, L + r);
        __syncthreads();
        // each element's component (into Z, once its pixels are read)
        for (int64_t e0 = 0; e0 < E; e0 += nt) {
            const int64_t e = e0 + tid;
            const bool act = e < E;
            uint32_t x = 0, z = 0;
            if (act) {
                x = (uint32_t)e;
                while (A.par[x] != x) x = A.par[x];
                z = A.Z[e];
                A.Z[e] = x;  // only this thread reads or writes Z[e] here
            }
            warp_add_by_key(A.tot, x, z, act);
        }
        __syncthreads();
        // the components that reach the top row, numbered by first run
        const uint32_t n0 = s_roff[1];
        const int64_t rt = fd.node_off + y0 * fd.qw, rb = fd.node_off + (y1 - 1) * fd.qw;
        for (uint32_t l = tid; l < n0; l += nt) atomicMin(&A.key[A.Z[l]], l);
        __syncthreads();
        if (tid < 32) {
            uint32_t k0 = 0;
            for (uint32_t i0 = 0; i0 < n0; i0 += 32) {
                const uint32_t i = i0 + tid;
                uint32_t g = 0;
                bool first = false;
                if (i < n0) {
                    g = A.Z[i];
                    first = A.key[g] == i;
                }
                const uint32_t bal = __ballot_sync(0xffffffffu, first);
                if (first) {
                    const uint32_t c = k0 + __popc(bal & lt);
                    A.key[g] = REF_KTOP | c;
                    ref.lpx[rt + c] = A.tot[g];
                }
                k0 += __popc(bal);
            }
            if (tid == 0) s_ntop = k0;
        }
        __syncthreads();
        for (uint32_t l = tid; l < n0; l += nt) ref.ltop[rt + l] = A.key[A.Z[l]] & 0xffffu;
        // the bottom row's other components, numbered by first run
        const uint32_t lb = s_roff[nr - 1], nbot = L - lb;
        for (uint32_t i = tid; i < nbot; i += nt) {
            const uint32_t g = A.Z[lb + i];
            if (A.key[g] < REF_KTOP) atomicMin(&A.key[g], i);
        }
        __syncthreads();
        if (tid < 32) {
            uint32_t k0 = 0;
            for (uint32_t i0 = 0; i0 < nbot; i0 += 32) {
                const uint32_t i = i0 + tid;
                uint32_t g = 0;
                bool first = false;
                if (i < nbot) {
                    g = A.Z[lb + i];
                    first = A.key[g] == i;
                }
                const uint32_t bal = __ballot_sync(0xffffffffu, first);
                if (first) {
                    const uint32_t k = k0 + __popc(bal & lt);
                    A.key[g] = REF_KBOT | k;
                    ref.lpx2[rb + k] = A.tot[g];
                }
                k0 += __popc(bal);
            }
            if (tid == 0) s_nnon = k0;
        }
        __syncthreads();
        for (uint32_t i = tid; i < nbot; i += nt) {
            const uint32_t kg = A.key[A.Z[lb + i]];
            ref.lbot[rb + i] = (kg & REF_KTOP) ? (kg & 0xffffu) : (0x80000000u | (kg & 0xffffu));
        }
        if (tid == 0)
            ref.desc[fd.row0 + f + b] = make_uint4((uint32_t)y0, (uint32_t)y1, s_ntop | s_nnon << 16, n0 | nbot << 16);
        __syncthreads();
    }
}

// The frontier pass's arrays (rows of at most capr runs), and the staging
// of one band's summaries (two of them, the next band's copies landing
// while this band is worked on).
struct FrontArrays {
    uint32_t *f_se, *s_Z, *par, *Z, *tot, *key, *bk, *cmin, *trng;
    uint16_t *f_slot;
    uint8_t *f_v;
};
struct FrontStage {
    const uint64_t *top_tl, *bot_tl;  // target runs of the band's top and bottom rows
    const uint32_t *top_c, *bot_c;    // their band components (ltop, lbot)
    const uint32_t *px, *px2;         // lpx, lpx2
};
__host__ __device__ inline size_t ref_front_carve(uint8_t *base, int64_t capr, FrontArrays *A) {
    const int64_t cape = 2 * capr + 2;
    size_t at = 0;
    auto take = [&](size_t bytes) {
        uint8_t *p = base + at;
        at = ref_align(at + bytes);
        return p;
    };
    FrontArrays a;
    a.f_se = (uint32_t *)take(4 * capr);
    a.s_Z = (uint32_t *)take(4 * (capr + 1));
    a.par = (uint32_t *)take(4 * cape);
    a.Z = (uint32_t *)take(4 * cape);
    a.tot = (uint32_t *)take(4 * cape);
    a.key = (uint32_t *)take(4 * (cape + capr + 1));
    a.bk = (uint32_t *)take(4 * capr);
    a.cmin = (uint32_t *)take(4 * (capr + 1));
    a.trng = (uint32_t *)take(4 * capr);
    a.f_slot = (uint16_t *)take(2 * capr);
    a.f_v = take(capr);
    if (A) *A = a;
    return at;
}
__host__ __device__ inline size_t ref_stage_carve(uint8_t *base, int64_t capr, FrontStage *S) {
    size_t at = 0;
    auto take = [&](size_t bytes) {
        uint8_t *p = base + at;
        at = ref_align(at + bytes);
        return p;
    };
    FrontStage s;
    s.top_tl = (const uint64_t *)take(8 * capr);
    s.bot_tl = (const uint64_t *)take(8 * capr);
    s.top_c = (const uint32_t *)take(4 * capr);
    s.bot_c = (const uint32_t *)take(4 * capr);
    s.px = (const uint32_t *)take(4 * capr);
    s.px2 = (const uint32_t *)take(4 * capr);
    if (S) *S = s;
    return at;
}
size_t ref_frontier_bytes(int64_t capr, bool staged) {
    return ref_front_carve(nullptr, capr, nullptr) + (staged ? 2 * ref_stage_carve(nullptr, capr, nullptr) : 0);
}

// A band's summaries: staged copies (issued by every thread of the block)
// or, without staging, the global arrays themselves.
__device__ __forceinline__ void front_issue(const FrontStage &S, const RefOrder &ref, const FrameDesc &fd, uint4 d,
                                            int tid, int nt) {
    const int64_t rt = fd.node_off + (int64_t)d.x * fd.qw, rb = fd.node_off + (int64_t)(d.y - 1) * fd.qw;
    const uint32_t ntop = d.z & 0xffffu, nnon = d.z >> 16, n0 = d.w & 0xffffu, nbot = d.w >> 16;
    for (uint32_t j = tid; j < n0; j += nt) {
        cp_async8((void *)(S.top_tl + j), ref.tlist + rt + j);
        cp_async4((void *)(S.top_c + j), ref.ltop + rt + j);
    }
    for (uint32_t j = tid; j < ntop; j += nt) cp_async4((void *)(S.px + j), ref.lpx + rt + j);
    for (uint32_t j = tid; j < nbot; j += nt) {
        cp_async8((void *)(S.bot_tl + j), ref.tlist + rb + j);
        cp_async4((void *)(S.bot_c + j), ref.lbot + rb + j);
    }
    for (uint32_t j = tid; j < nnon; j += nt) cp_async4((void *)(S.px2 + j), ref.lpx2 + rb + j);
}
__device__ __forceinline__ FrontStage front_direct(const RefOrder &ref, const FrameDesc &fd, uint4 d) {
    const int64_t rt = fd.node_off + (int64_t)d.x * fd.qw, rb = fd.node_off + (int64_t)(d.y - 1) * fd.qw;
    return FrontStage{ref.tlist + rt, ref.tlist + rb, ref.ltop + rt, ref.lbot + rb, ref.lpx + rt, ref.lpx2 + rb};
}

// A block per frame, band after band: the prefix sets at the bottom row of
// each band (slots), from the slots above and the band's summaries. With
// `scratch`, the arrays live there (a region per frame) and nothing is staged.
__global__ void __launch_bounds__(128) k_ref_frontier(const FrameDesc *frames, RefOrder ref, int64_t capr,
                                                      uint8_t *scratch, size_t scratch_per_block) {
    extern __shared__ __align__(16) uint8_t s_mem[];
    __shared__ uint32_t s_m;
    const int f = blockIdx.x;
    if (!ref.need[f]) return;
    const FrameDesc fd = frames[f];
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31;
    const uint32_t lt = (1u << lane) - 1u;
    const bool staged = scratch == nullptr;
    FrontArrays A;
    const size_t fb = ref_front_carve(staged ? s_mem : scratch + (size_t)f * scratch_per_block, capr, &A);
    const size_t sb = ref_stage_carve(nullptr, capr, nullptr);
    auto stage = [&](int64_t i) {  // staging buffer i (0 or 1)
        FrontStage S;
        ref_stage_carve(s_mem + fb + (size_t)i * sb, capr, &S);
        return S;
    };
    const uint4 *desc = ref.desc + fd.row0 + f;
    const int64_t nb = ref.nband[f];
    uint4 d0 = desc[0], d1 = nb > 1 ? desc[1] : make_uint4(0, 0, 0, 0);
    if (staged) front_issue(stage(0), ref, fd, d0, tid, nt);
    cp_async_commit();
    int64_t m = 0, nf = 0;  // the slots and runs of the row above the band
    for (int64_t b = 0; b < nb; b++) {
        const uint4 d2 = b + 2 < nb ? desc[b + 2] : make_uint4(0, 0, 0, 0);
        if (staged && b + 1 < nb) front_issue(stage((b + 1) & 1), ref, fd, d1, tid, nt);
        cp_async_commit();
        cp_async_wait_one();
        __syncthreads();
        const FrontStage S = staged ? stage(b & 1) : front_direct(ref, fd, d0);
        const int64_t y1 = d0.y;
        const int64_t ntop = d0.z & 0xffffu, nnon = d0.z >> 16, n0 = d0.w & 0xffffu, nbot = d0.w >> 16;
        const int64_t rb = fd.node_off + (y1 - 1) * fd.qw;
        const bool boundary = y1 < fd.qh;
        // elements: the slots [0, m), the band's components that reach its
        // top row [m, m + ntop); keys of the bottom row's sets: those
        // elements, then the band's other components [E, E + nnon)
        const int64_t E = m + ntop;
        for (int64_t e = tid; e < E; e += nt) {
            A.par[e] = (uint32_t)e;
            A.tot[e] = 0;
            A.Z[e] = e < m ? A.s_Z[e] : S.px[e - m];
        }
        for (int64_t e = tid; e < E + nnon; e += nt) A.key[e] = REF_KNONE;
        for (int64_t c = tid; c < ntop; c += nt) A.cmin[c] = 0xffffffffu;
        __syncthreads();
        // each top run's touching runs above (first and last; the runs of
        // its value between them touch it too), and each band component's
        // smallest touching slot
        const int64_t rt = fd.node_off + (int64_t)d0.x * fd.qw;
        for (int64_t j = tid; j < n0; j += nt) {
            const uint64_t te = S.top_tl[j];
            const uint32_t se = (uint32_t)te;
            const uint8_t v = (uint8_t)(te >> 48);
            const int64_t a0 = se & 0xffffu, a1 = se >> 16;
            const uint32_t c = S.top_c[j];
            uint32_t klo = 0xffffu, khi = 0, smin = 0xffffffffu;
            if (nf > 0)
                for (uint32_t k = first_reaching(A.f_se, 0, (uint32_t)nf, a0);
                     k < nf && (int64_t)(A.f_se[k] & 0xffffu) <= a1 + 1; k++)
                    if (A.f_v[k] == v && runs_touch(a0, a1, A.f_se[k] & 0xffffu, A.f_se[k] >> 16, v)) {
                        smin = min(smin, (uint32_t)A.f_slot[k]);
                        if (klo == 0xffffu) klo = k;
                        khi = k;
                    }
            if (smin != 0xffffffffu) atomicMin(A.cmin + c, smin);
            const uint32_t r = klo == 0xffffu ? 0xffffffffu : klo | khi << 16;
            A.trng[j] = r;
            ref.tch[rt + j] = r;  // for the replay
        }
        __syncthreads();
        // a component hangs under its smallest slot; the other slots it
        // reaches are joined to that one (the only unions left)
        for (int64_t c = tid; c < ntop; c += nt)
            if (A.cmin[c] != 0xffffffffu) A.par[m + c] = A.cmin[c];
        for (int64_t j = tid; j < n0; j += nt) {
            const uint32_t r = A.trng[j];
            if (r == 0xffffffffu) continue;
            const uint32_t s0 = A.cmin[S.top_c[j]];
            const uint8_t v = (uint8_t)(S.top_tl[j] >> 48);
            for (uint32_t k = r & 0xffffu; k <= (r >> 16); k++)
                if (A.f_v[k] == v && A.f_slot[k] != s0) pu_unite(A.par, A.f_slot[k], s0);
        }
        __syncthreads();
        for (int64_t e0 = 0; e0 < E; e0 += nt) {
            const int64_t e = e0 + tid;
            const bool act = e < E;
            uint32_t x = 0, z = 0;
            if (act) {
                x = (uint32_t)e;
                while (A.par[x] != x) x = A.par[x];
                z = A.Z[e];
                A.Z[e] = x;  // only this thread reads or writes Z[e] here
            }
            warp_add_by_key(A.tot, x, z, act);
        }
        __syncthreads();
        // the bottom row's sets, numbered by first run: the new slots
        for (int64_t j = tid; j < nbot; j += nt) {
            const uint32_t lb = S.bot_c[j];
            const uint32_t g = (lb & 0x80000000u) ? (uint32_t)E + (lb & 0xffffu) : A.Z[m + lb];
            A.bk[j] = g;
            atomicMin(&A.key[g], (uint32_t)j);
        }
        __syncthreads();
        if (tid < 32) {  // one warp numbers them in run order
            uint32_t k0 = 0;
            for (int64_t i0 = 0; i0 < nbot; i0 += 32) {
                const int64_t i = i0 + lane;
                uint32_t g = 0;
                bool first = false;
                if (i < nbot) {
                    g = A.bk[i];
                    first = A.key[g] == (uint32_t)i;
                }
                const uint32_t bal = __ballot_sync(0xffffffffu, first);
                if (first) {
                    const uint32_t k = k0 + __popc(bal & lt);
                    const uint32_t px = g < (uint32_t)E ? A.tot[g] : S.px2[g - E];
                    A.s_Z[k] = px;
                    A.key[g] = REF_KTOP | k;
                    if (boundary)
                        ref.binfo[rb + k] =
                            (uint64_t)px | (uint64_t)i << 32 | (uint64_t)(uint8_t)(S.bot_tl[i] >> 56) << 48;
                }
                k0 += __popc(bal);
            }
            if (lane == 0) {
                s_m = k0;
                if (boundary) ref.bm[fd.row0 + y1 - 1] = k0;
            }
        }
        __syncthreads();
        for (int64_t j = tid; j < nbot; j += nt) {
            const uint32_t slot = A.key[A.bk[j]] & 0xffffu;
            const uint64_t te = S.bot_tl[j];
            A.f_se[j] = (uint32_t)te;
            A.f_v[j] = (uint8_t)(te >> 48);
            A.f_slot[j] = (uint16_t)slot;
            if (boundary) ref.bslot[rb + j] = (uint16_t)slot;
        }
        m = s_m;
        nf = nbot;
        d0 = d1;
        d1 = d2;
        __syncthreads();
    }
    cp_async_wait_all();
}

size_t ref_band_bytes(int64_t capr, bool staged) {
    return ref_replay_bytes(capr) + (staged ? ref_align(8 * capr) + ref_align(4 * capr) : 0);
}

// The replay of one band, a warp each (the frame's bands taken in turn by
// its blocks), the incoming sets' roots as symbols. A launch takes the
// bands whose rows hold more than `lo` and at most `hi` target runs (bwide)
// and has arrays for capr; with `scratch` they live there (a region per
// block) and rows are read in place, else each row's runs are staged while
// the row above is replayed.
__global__ void __launch_bounds__(32) k_ref_band(const FrameDesc *frames, RefOrder ref, int64_t capr, uint32_t lo,
                                                 uint32_t hi, uint8_t *scratch, size_t scratch_per_block) {
    extern __shared__ __align__(16) uint8_t s_mem[];
    const int f = blockIdx.y;
    if (!ref.need[f]) return;
    const int lane = threadIdx.x;
    const FrameDesc fd = frames[f];
    const bool staged = scratch == nullptr;
    ReplayArrays A;
    const size_t rbytes =
        ref_carve(staged ? s_mem : scratch + ((size_t)blockIdx.y * gridDim.x + blockIdx.x) * scratch_per_block, capr, &A);
    uint64_t *stg = reinterpret_cast<uint64_t *>(s_mem + rbytes);
    uint32_t *stg_t = reinterpret_cast<uint32_t *>(s_mem + rbytes + ref_align(8 * capr));
    uint32_t *fin = ref.fin + (int64_t)f * AT_REF_MAXT, *finb = ref.finb + (int64_t)f * AT_REF_MAXT;
    const uint32_t vbase = (uint32_t)(fd.node_off + (int64_t)fd.qw * fd.qh);
    const uint4 *desc = ref.desc + fd.row0 + f;
    const uint32_t *bw = ref.bwide + fd.row0 + f;
    const int64_t nb = ref.nband[f];
    for (int64_t b = blockIdx.x; b < nb; b += gridDim.x) {
        const uint32_t wide = bw[b];
        if (wide <= lo || wide > hi) continue;
        const uint4 d = desc[b];
        const int64_t y0 = d.x, y1 = d.y;
        const int nr = (int)(y1 - y0);
        // the band's row records (count | link << 31), lane r for row y0 + r
        const uint32_t trl = lane < nr ? ref.trow[fd.row0 + y0 + lane] : 0u;
        if (staged) {
            const int64_t n = __shfl_sync(0xffffffffu, trl, 0) & 0x7fffffffu, rbase = fd.node_off + y0 * fd.qw;
            for (int64_t j = lane; j < n; j += 32) {
                cp_async8(stg + j, ref.tlist + rbase + j);
                cp_async4(stg_t + j, ref.tch + rbase + j);
            }
            cp_async_commit();
        }
        RowState S{0, 0};
        if (b > 0) {
            // the incoming sets: the row above with its slots, roots as symbols
            const int64_t ya = y0 - 1;
            const int64_t ra = fd.node_off + ya * fd.qw;
            const int64_t na = ref.trow[fd.row0 + ya] & 0x7fffffffu;
            const int64_t ma = ref.bm[fd.row0 + ya];
            for (int64_t j = lane; j < na; j += 32) {
                const uint64_t e = ref.tlist[ra + j];
                A.p_se[j] = (uint32_t)e;
                A.p_v[j] = (uint8_t)(e >> 48);
                A.p_slot[j] = ref.bslot[ra + j];
            }
            for (int64_t k = lane; k < ma; k += 32) {
                const uint64_t bi = ref.binfo[ra + k];
                A.s_R[k] = REF_SYM | (uint32_t)k;
                A.s_Z[k] = (uint32_t)bi;
                A.s_t[k] = (uint8_t)(bi >> 48);
            }
            S.m = (int)ma;
            S.np = (int)na;
        }
        for (int64_t y = y0; y < y1; y++) {
            const uint32_t tr = __shfl_sync(0xffffffffu, trl, (int)(y - y0));
            const int n = (int)(tr & 0x7fffffffu);
            const bool link = (tr >> 31) != 0;
            const int64_t rbase = fd.node_off + y * fd.qw;
            const uint64_t *src = ref.tlist + rbase;
            const uint32_t *srct = ref.tch + rbase;
            if (staged) {
                cp_async_wait_all();
                src = stg;
                srct = stg_t;
            }
            __syncwarp();
            for (int j = lane; j < n; j += 32) {
                const uint64_t e = src[j];
                A.c_se[j] = (uint32_t)e;
                A.c_v[j] = (uint8_t)(e >> 48);
                A.c_j[j] = (uint16_t)(e >> 32);
                A.c_t[j] = (uint8_t)(e >> 56);
                A.c_tch[j] = srct[j];
            }
            __syncwarp();
            if (staged && y + 1 < y1) {
                const uint32_t tn = __shfl_sync(0xffffffffu, trl, (int)(y + 1 - y0)) & 0x7fffffffu;
                for (uint32_t j = lane; j < tn; j += 32) {
                    cp_async8(stg + j, ref.tlist + rbase + fd.qw + j);
                    cp_async4(stg_t + j, ref.tch + rbase + fd.qw + j);
                }
                cp_async_commit();
            }
            if (n == 0 && S.np == 0) continue;
            replay_row(A, S, n, link && n > 0, (uint32_t)rbase, vbase + (uint32_t)(y - 1), fin, finb, (uint32_t)b);
        }
        // the roots of the sets at the band's last row, per slot of the
        // boundary below (through the slot's first run); after the last
        // band every open set is a whole component
        if (y1 < fd.qh) {
            const int64_t rb = fd.node_off + (y1 - 1) * fd.qw;
            const int64_t mb = ref.bm[fd.row0 + y1 - 1];
            for (int64_t k = lane; k < mb; k += 32) {
                const uint32_t rep = (uint32_t)(ref.binfo[rb + k] >> 32) & 0xffffu;
                ref.outroot[rb + k] = A.s_R[A.p_slot[rep]];
            }
        } else {
            for (int64_t k = lane; k < S.m; k += 32) {
                const uint32_t t = A.s_t[k];
                if (t == REF_NONE) continue;
                fin[t] = A.s_R[k];
                finb[t] = (uint32_t)b;
            }
        }
        __syncwarp();
    }
}

// A block per frame: the symbols replaced band by band from the top (the
// roots of a band's incoming slots are those of the slots' sets after the
// band above), each target's root, then the reference's packed node
// numbers. Each band is a barrier and a shared-memory step; the global
// reads of 8 bands are issued together.
#define REF_RES_CHUNK 8
__global__ void __launch_bounds__(256) k_ref_resolve(const FrameDesc *frames, RefOrder ref, int64_t capr) {
    extern __shared__ __align__(16) uint32_t s_res[];  // two arrays of capr + 1
    __shared__ int64_t s_rb[REF_RES_CHUNK];
    __shared__ uint32_t s_mb[REF_RES_CHUNK];
    const int f = blockIdx.x;
    if (!ref.need[f]) return;
    const int tid = threadIdx.x, nth = blockDim.x;
    const FrameDesc fd = frames[f];
    const uint32_t nt = ref.nt[f];
    uint32_t my_fin = 0, my_finb = 0xffffffffu, my_root = 0xffffffffu;
    if (tid < (int)nt) {
        my_fin = ref.fin[(int64_t)f * AT_REF_MAXT + tid];
        my_finb = ref.finb[(int64_t)f * AT_REF_MAXT + tid];
    }
    uint32_t *cur = s_res, *nxt = s_res + capr + 1;
    const uint4 *desc = ref.desc + fd.row0 + f;
    const int64_t nb = ref.nband[f];
    for (int64_t b0 = 0; b0 < nb; b0 += REF_RES_CHUNK) {
        if (tid < REF_RES_CHUNK) {
            const int64_t b = b0 + tid;
            uint32_t mb = 0;
            int64_t rb = 0;
            if (b + 1 < nb) {
                const int64_t yb = (int64_t)desc[b].y - 1;
                rb = fd.node_off + yb * fd.qw;
                mb = ref.bm[fd.row0 + yb];
            }
            s_rb[tid] = rb;
            s_mb[tid] = mb;
        }
        __syncthreads();
        uint32_t R[REF_RES_CHUNK];
#pragma unroll
        for (int i = 0; i < REF_RES_CHUNK; i++) R[i] = (uint32_t)tid < s_mb[i] ? ref.outroot[s_rb[i] + tid] : 0u;
#pragma unroll
        for (int i = 0; i < REF_RES_CHUNK; i++) {
            const int64_t b = b0 + i;
            if (b < nb) {
                if (my_finb == (uint32_t)b) my_root = (my_fin & REF_SYM) ? cur[my_fin & ~REF_SYM] : my_fin;
                if (b + 1 < nb) {
                    const uint32_t mb = s_mb[i];
                    if ((uint32_t)tid < mb) nxt[tid] = (R[i] & REF_SYM) ? cur[R[i] & ~REF_SYM] : R[i];
                    for (uint32_t k = tid + nth; k < mb; k += nth) {
                        const uint32_t Rk = ref.outroot[s_rb[i] + k];
                        nxt[k] = (Rk & REF_SYM) ? cur[Rk & ~REF_SYM] : Rk;
                    }
                    __syncthreads();
                    uint32_t *t = cur;
                    cur = nxt;
                    nxt = t;
                }
            }
        }
        __syncthreads();
    }
    // GPU node ids -> the reference's packed node numbers (a target left
    // without a root keeps 0xffffffff, which the final stage reports)
    if (tid < (int)nt) {
        uint32_t r = my_root;
        if (r != 0xffffffffu) {
            const uint32_t *pre = ref.rpre + fd.row0 + f;
            const int64_t nd = (int64_t)r - fd.node_off;
            const int64_t qpx = (int64_t)fd.qw * fd.qh;
            r = nd < qpx ? pre[nd / fd.qw] + (uint32_t)(nd % fd.qw) : pre[fd.qh] + (uint32_t)(nd - qpx);
        }
        ref.troot[(int64_t)f * AT_REF_MAXT + tid] = r;
    }
}

// ---------------------------------------------------------------------------
// Launchers.

void launch_ref_order(const Launch &L, const FrameDesc *frames, const uint8_t *thr, RunArrays runs,
                      const uint32_t *row_nruns, int nfam, const int64_t *qstart, const GpuDetection *dets,
                      const uint32_t *det_ok, const uint32_t *qcl, const uint64_t *ckey, int nb,
                      const RefPlan &P, const RefOrder &ref, uint32_t *err) {
    k_ref_targets<<<L.nframes, 256, 0, L.stream>>>(frames, nfam, qstart, dets, det_ok, qcl, ckey, nb, runs, row_nruns,
                                                   ref, err);
    const int64_t b = (L.max_qh + 7) / 8;
    const dim3 grid((unsigned)(b < 1 ? 1 : b < 148 ? b : 148), (unsigned)L.nframes);
    k_ref_mark<<<grid, 256, 0, L.stream>>>(frames, thr, runs, row_nruns, ref);
    k_ref_cut<<<L.nframes, 32, 0, L.stream>>>(frames, ref, (uint32_t)P.pcap);
    const int64_t gb = (L.max_qh + REF_BAND - 1) / REF_BAND;
    const unsigned bands = (unsigned)(gb < 1 ? 1 : gb);
    k_ref_local<<<dim3(bands, (unsigned)L.nframes), 256, ref_local_bytes(P.pcap), L.stream>>>(frames, ref,
                                                                                            (uint32_t)P.pcap, err);
    k_ref_frontier<<<L.nframes, 128, P.front_scratch ? 0 : ref_frontier_bytes(P.capr, true), L.stream>>>(
        frames, ref, P.capr, P.front_scratch, P.front_bytes);
    // bands of narrow rows, many blocks per SM; then the others
    const int64_t small = P.capr < REF_SMALLR ? P.capr : REF_SMALLR;
    k_ref_band<<<dim3(bands, (unsigned)L.nframes), 32, ref_band_bytes(small, true), L.stream>>>(
        frames, ref, small, 0u, (uint32_t)small, nullptr, 0);
    if (P.capr > REF_SMALLR)
        k_ref_band<<<dim3(P.band_scratch ? REF_BAND_BLOCKS : bands, (unsigned)L.nframes), 32,
                     P.band_scratch ? 0 : ref_band_bytes(P.capr, true), L.stream>>>(
            frames, ref, P.capr, (uint32_t)REF_SMALLR, 0xffffffffu, P.band_scratch, P.band_bytes);
    k_ref_resolve<<<L.nframes, 256, 8 * (P.capr + 1), L.stream>>>(frames, ref, P.capr);
}

int ref_order_launches(const RefPlan &P) { return P.capr > REF_SMALLR ? 8 : 7; }

bool ref_replay_set_smem(size_t bytes) {
    return cudaFuncSetAttribute(k_ref_band, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) == cudaSuccess &&
           cudaFuncSetAttribute(k_ref_local, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) == cudaSuccess &&
           cudaFuncSetAttribute(k_ref_frontier, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) ==
               cudaSuccess &&
           cudaFuncSetAttribute(k_ref_resolve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) == cudaSuccess;
}
