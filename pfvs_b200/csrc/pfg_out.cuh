// Output stage: the points the search emitted (direction, q, c) become the
// reference's output rows (M = Binter c, Kn = Z Binter c, q, pidx), grouped
// by direction and sorted by (M, Kn) within one (the canonical order of
// pfvs/gpu.py:155-159 and pfvs/coni.py:322-324; the reference sorts on the
// host, pfvs/fp_kernel/cuda/pfvs_gpu.cu:672-699).  All on the device:
//   k_count    kept points per direction (the direction succeeded, and the
//              point comes from the direction's last search pass)
//   k_scan     segment offsets, sort-chunk offsets, longest segment (one block)
//   k_scatter  point indices into their direction's segment
//   k_keys     per kept point its M row (h entries, stride ks): the sort key
//              (c -> M = Binter c is injective, so M alone orders the points)
//   k_segsort  one block per chunk (a segment's points in runs of SORT_CAP):
//              bitonic sort in shared memory on the first KEYN entries of M,
//              ties decided from the full row
//   k_merge    merges pairs of sorted runs of the longer segments, one
//              thread per point: its place is its rank in its own run plus
//              its rank in the partner run (binary search); log2 passes
//   k_order    the sorted positions -> point indices
//   k_rows     the M and Kn rows (MH wide, or compact: the call's widest h11),
//              q and pidx in output order
//
// The rows are exact in int64: the setup guarantees that every column of
// Binter^T and (Z Binter)^T has an absolute sum below 2^31 (so each entry fits
// int32) and the search |c| < 2^31, so every sum is below 2^62.
#pragma once
#include "pfg_types.cuh"

namespace pfg {

constexpr int KEYN = 4;           // M entries in a sort key
#ifndef PFG_SORT_CAP
#define PFG_SORT_CAP 2048
#endif
constexpr int SORT_CAP = PFG_SORT_CAP;   // run length sorted in shared memory

struct OutArgs {
    const Dir *dirs;
    const int64_t *slab;
    const PointHdr *hdr;
    const int32_t *coords;
    const int32_t *dir_pass;
    unsigned long long n_pts;
    int n_dirs;
    unsigned *count, *fill;       // per direction
    unsigned long long *seg;      // (n_dirs + 1) offsets
    unsigned *idx;                // (n_kept) point indices, segment-ordered (then sorted)
    int64_t *keys;                // (n_kept, ks) M rows
    int ks;                       // key stride: the largest h11 of the batch
    unsigned long long *cseg;     // (n_dirs + 1) sort-chunk offsets
    unsigned long long *summary;  // [0] kept points, [1] chunks, [2] longest segment
    unsigned *perm;               // (n_kept) segment-local positions in sorted order
};

__device__ __forceinline__ bool dir_ok(int st) { return st == ST_PENDING || st == ST_OK; }

__device__ __forceinline__ bool keep_point(const OutArgs &O, unsigned long long k)
{
    const int pid = O.hdr[k].pid;
    return dir_ok(O.dirs[pid].status) && O.hdr[k].pad == O.dir_pass[pid];
}

__global__ void k_count(OutArgs O)
{
    for (unsigned long long k = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; k < O.n_pts;
         k += (unsigned long long)gridDim.x * blockDim.x)
        if (keep_point(O, k)) atomicAdd(&O.count[O.hdr[k].pid], 1u);
}

// exclusive scans of count[0..n) into seg[0..n] and of the chunk counts
// ceil(count / SORT_CAP) into cseg[0..n]; the longest segment (one block of
// 1024 threads)
__global__ void __launch_bounds__(1024) k_scan(OutArgs O)
{
    __shared__ unsigned long long part[1024], cpart[1024];
    __shared__ unsigned mx[1024];
    const int t = threadIdx.x, nt = blockDim.x, n = O.n_dirs;
    const int per = (n + nt - 1) / nt, a = t * per, b = min(a + per, n);
    unsigned long long s = 0, cs = 0;
    unsigned m = 0;
    for (int i = a; i < b; ++i) {
        const unsigned c = O.count[i];
        s += c;
        cs += (c + SORT_CAP - 1) / SORT_CAP;
        m = max(m, c);
    }
    part[t] = s; cpart[t] = cs; mx[t] = m;
    __syncthreads();
    for (int o = 1; o < nt; o <<= 1) {
        const unsigned long long x = t >= o ? part[t - o] : 0, y = t >= o ? cpart[t - o] : 0;
        const unsigned z = t >= o ? mx[t - o] : 0;
        __syncthreads();
        part[t] += x; cpart[t] += y; mx[t] = max(mx[t], z);
        __syncthreads();
    }
    unsigned long long run = t ? part[t - 1] : 0, crun = t ? cpart[t - 1] : 0;
    for (int i = a; i < b; ++i) {
        const unsigned c = O.count[i];
        O.seg[i] = run; run += c;
        O.cseg[i] = crun; crun += (c + SORT_CAP - 1) / SORT_CAP;
    }
    if (t == nt - 1) {
        O.seg[n] = part[nt - 1];
        O.cseg[n] = cpart[nt - 1];
        O.summary[0] = part[nt - 1];
        O.summary[1] = cpart[nt - 1];
        O.summary[2] = mx[nt - 1];
    }
}

__global__ void k_scatter(OutArgs O)
{
    for (unsigned long long k = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; k < O.n_pts;
         k += (unsigned long long)gridDim.x * blockDim.x) {
        if (!keep_point(O, k)) continue;
        const int pid = O.hdr[k].pid;
        const unsigned pos = atomicAdd(&O.fill[pid], 1u);
        O.idx[O.seg[pid] + pos] = (unsigned)k;
    }
}

// entry r of M (T = BT) or Kn (T = ZT) of point k
__device__ __forceinline__ int64_t row_entry(const int64_t *T, const int32_t *c, int d, int h, int r)
{
    int64_t s = 0;
    for (int a = 0; a < d; ++a) s += (int64_t)(int32_t)T[a * h + r] * (int64_t)c[a];
    return s;
}

// warp per kept point: its M row into the keys (lanes own entries)
__global__ void k_keys(OutArgs O, unsigned long long n_kept)
{
    const int lane = threadIdx.x & 31;
    const unsigned long long w = (blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x) >> 5;
    const unsigned long long nw = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
    for (unsigned long long t = w; t < n_kept; t += nw) {
        const unsigned k = O.idx[t];
        const Dir D = O.dirs[O.hdr[k].pid];
        const int h = D.h, d = D.d;
        const int64_t *BT = O.slab + D.slab + slab_layout(h, d).bt;
        const int32_t *c = O.coords + (unsigned long long)k * MD;
        const int32_t c0 = lane < d ? c[lane] : 0, c1 = lane + 32 < d ? c[lane + 32] : 0;
        int64_t m0 = 0, m1 = 0;
        if (h <= 32) {                                  // (warp-uniform) one column per lane
            const int64_t *col = BT + (lane < h ? lane : 0);
            for (int a = 0; a < d; ++a) {
                const int32_t ca = __shfl_sync(FULL, c0, a);
                m0 += (int64_t)(int32_t)col[a * h] * ca;
            }
            if (lane >= h) m0 = 0;
        } else {
            for (int a = 0; a < d; ++a) {
                const int64_t ca = __shfl_sync(FULL, a < 32 ? c0 : c1, a & 31);
                if (lane < h) m0 += (int64_t)(int32_t)BT[a * h + lane] * ca;
                if (lane + 32 < h) m1 += (int64_t)(int32_t)BT[a * h + lane + 32] * ca;
            }
        }
        int64_t *key = O.keys + t * O.ks;
        if (lane < h) key[lane] = m0;
        if (lane + 32 < h) key[lane + 32] = m1;
    }
}

// x > y for segment positions x, y: first KEYN entries from `pre` (stride
// KEYN), the rest of the M rows from global memory
__device__ __forceinline__ bool key_greater(const OutArgs &O, const int64_t *pre, unsigned long long s0,
                                            unsigned x, unsigned y, int h)
{
    for (int r = 0; r < KEYN; ++r) {
        const int64_t a = pre[x * KEYN + r], b = pre[y * KEYN + r];
        if (a != b) return a > b;
    }
    const int64_t *kx = O.keys + (s0 + x) * O.ks, *ky = O.keys + (s0 + y) * O.ks;
    for (int r = KEYN; r < h; ++r)
        if (kx[r] != ky[r]) return kx[r] > ky[r];
    return x > y;                                   // (equal rows: the same point)
}

// x < y for segment-local positions of one segment (rows from global memory)
__device__ __forceinline__ bool key_less(const OutArgs &O, unsigned long long s0, unsigned x, unsigned y, int h)
{
    const int64_t *kx = O.keys + (s0 + x) * O.ks, *ky = O.keys + (s0 + y) * O.ks;
    for (int r = 0; r < h; ++r)
        if (kx[r] != ky[r]) return kx[r] < ky[r];
    return x < y;
}

// One block per chunk: bitonic sort (padded to a power of two with
// sentinels) of SORT_CAP or fewer consecutive points of one segment, the
// first KEYN entries of their M rows in shared memory.  Writes the chunk's
// segment-local positions in sorted order to perm.
__global__ void __launch_bounds__(256) k_segsort(OutArgs O)
{
#ifdef PFG_EMU
    static unsigned char smem_raw[SORT_CAP * KEYN * 8 + SORT_CAP * 4];
#else
    extern __shared__ __align__(16) unsigned char smem_raw[];
#endif
    int64_t *skeys = (int64_t *)smem_raw;                       // SORT_CAP x KEYN
    unsigned *a = (unsigned *)(skeys + SORT_CAP * KEYN);        // SORT_CAP
    constexpr unsigned NONE = 0xffffffffu;
    const unsigned long long nch = O.summary[1];
    for (unsigned long long ci = blockIdx.x; ci < nch; ci += gridDim.x) {
        int lo_p = 0, hi_p = O.n_dirs;              // the direction: cseg[pid] <= ci < cseg[pid + 1]
        while (hi_p - lo_p > 1) {
            const int mid = (lo_p + hi_p) >> 1;
            if (O.cseg[mid] <= ci) lo_p = mid; else hi_p = mid;
        }
        const int pid = lo_p;
        const unsigned long long s0 = O.seg[pid];
        const unsigned nseg = (unsigned)(O.seg[pid + 1] - s0);
        const unsigned lo = (unsigned)(ci - O.cseg[pid]) * SORT_CAP;
        const unsigned n = min((unsigned)SORT_CAP, nseg - lo);
        const int h = O.dirs[pid].h;
        unsigned np = 1;
        while (np < n) np <<= 1;
        for (unsigned e = threadIdx.x; e < n * KEYN; e += blockDim.x) {
            const unsigned t = e / KEYN, r = e % KEYN;
            skeys[e] = (int)r < h ? O.keys[(s0 + lo + t) * O.ks + r] : 0;
        }
        for (unsigned t = threadIdx.x; t < np; t += blockDim.x) a[t] = t < n ? t : NONE;
        __syncthreads();
        for (unsigned k = 2; k <= np; k <<= 1) {
            for (unsigned j = k >> 1; j > 0; j >>= 1) {
                for (unsigned t = threadIdx.x; t < np; t += blockDim.x) {
                    const unsigned u = t ^ j;
                    if (u <= t) continue;
                    const bool up = (t & k) == 0;
                    const unsigned x = a[t], y = a[u];
                    bool xgt;                       // x > y
                    if (x == NONE) xgt = y != NONE;
                    else if (y == NONE) xgt = false;
                    else xgt = key_greater(O, skeys, s0 + lo, x, y, h);
                    if (xgt == up) { a[t] = y; a[u] = x; }
                }
                __syncthreads();
            }
        }
        for (unsigned t = threadIdx.x; t < n; t += blockDim.x) O.perm[s0 + lo + t] = lo + a[t];
        __syncthreads();
    }
}

// One merge pass over runs of length L (segments longer than L only): the
// point at segment position i of run r goes to the merged run of runs
// (r & ~1, r | 1) at its rank in its own run plus its rank in the partner.
__global__ void k_merge(OutArgs O, unsigned long long n_kept, unsigned L, const unsigned *pin, unsigned *pout)
{
    for (unsigned long long t = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; t < n_kept;
         t += (unsigned long long)gridDim.x * blockDim.x) {
        const int pid = O.hdr[O.idx[t]].pid;
        const unsigned long long s0 = O.seg[pid];
        const unsigned n = (unsigned)(O.seg[pid + 1] - s0), i = (unsigned)(t - s0);
        if (n <= L) { pout[t] = pin[t]; continue; }
        const unsigned r = i / L, own_lo = r * L, part_lo = (r ^ 1u) * L, base = (r & ~1u) * L;
        const unsigned part_n = part_lo >= n ? 0 : min(L, n - part_lo);
        const unsigned x = pin[t];
        const int h = O.dirs[pid].h;
        unsigned lo = 0, hi = part_n;               // partner elements less than x
        while (lo < hi) {
            const unsigned mid = (lo + hi) >> 1;
            if (key_less(O, s0, pin[s0 + part_lo + mid], x, h)) lo = mid + 1; else hi = mid;
        }
        pout[s0 + base + (i - own_lo) + lo] = x;
    }
}

// sorted segment-local positions -> point indices (and key rows) in output order
__global__ void k_order(OutArgs O, unsigned long long n_kept, const unsigned *perm, unsigned *out_idx,
                        unsigned *out_key)
{
    for (unsigned long long t = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; t < n_kept;
         t += (unsigned long long)gridDim.x * blockDim.x) {
        const int pid = O.hdr[O.idx[t]].pid;
        const unsigned long long s0 = O.seg[pid];
        out_idx[t] = O.idx[s0 + perm[t]];
        out_key[t] = (unsigned)(s0 + perm[t]);
    }
}

struct RowArgs {
    const Dir *dirs;
    const int64_t *slab;
    const PointHdr *hdr;
    const int32_t *coords;
    const unsigned *idx;          // points in output order
    const unsigned *krow;         // their rows of keys (the M rows)
    const int64_t *keys;
    int ks;
    unsigned long long n_out;
    int64_t pid_base;
    int64_t *M, *Kn, *q, *pidx;   // output (n_out, rw), (n_out,)
    int rw;                       // row width: MH, or the call's widest h11 (compact rows)
};

// one warp per output row: lanes own entries r = lane, lane + 32
__global__ void k_rows(RowArgs R)
{
    const int lane = threadIdx.x & 31;
    const unsigned long long w = (blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x) >> 5;
    const unsigned long long nw = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
    for (unsigned long long t = w; t < R.n_out; t += nw) {
        const unsigned k = R.idx[t];
        const PointHdr P = R.hdr[k];
        const Dir D = R.dirs[P.pid];
        const int h = D.h, d = D.d;
        const Slab L = slab_layout(h, d);
        const int64_t *ZT = R.slab + D.slab + L.zt;
        const int32_t *c = R.coords + (unsigned long long)k * MD;
        const int32_t c0 = lane < d ? c[lane] : 0, c1 = lane + 32 < d ? c[lane + 32] : 0;
        const int64_t *key = R.keys + (unsigned long long)R.krow[t] * R.ks;
        const int64_t m0 = lane < h ? key[lane] : 0, m1 = lane + 32 < h ? key[lane + 32] : 0;
        int64_t k0 = 0, k1 = 0;
        if (h <= 32) {                                  // (warp-uniform) one column per lane
            const int64_t *col = ZT + (lane < h ? lane : 0);
            for (int a = 0; a < d; ++a) {
                const int32_t ca = __shfl_sync(FULL, c0, a);
                k0 += (int64_t)(int32_t)col[a * h] * ca;
            }
            if (lane >= h) k0 = 0;
        } else {
            for (int a = 0; a < d; ++a) {
                const int64_t ca = __shfl_sync(FULL, a < 32 ? c0 : c1, a & 31);
                if (lane < h) k0 += (int64_t)(int32_t)ZT[a * h + lane] * ca;
                if (lane + 32 < h) k1 += (int64_t)(int32_t)ZT[a * h + lane + 32] * ca;
            }
        }
        int64_t *Mr = R.M + t * R.rw, *Kr = R.Kn + t * R.rw;
        if (lane < R.rw) { Mr[lane] = m0; Kr[lane] = k0; }
        if (lane + 32 < R.rw) { Mr[lane + 32] = m1; Kr[lane + 32] = k1; }
        if (lane == 0) { R.q[t] = P.q; R.pidx[t] = R.pid_base + P.pid; }
    }
}

}  // namespace pfg
