// Output stage: the points the search emitted (direction, q, c) become the
// reference's output rows (M = Binter c, Kn = Z Binter c, q, pidx), grouped
// by direction and sorted by (M, Kn) within one (the canonical order of
// pfvs/gpu.py:155-159 and pfvs/coni.py:322-324; the reference sorts on the
// host, pfvs/fp_kernel/cuda/pfvs_gpu.cu:672-699).  All on the device:
//   k_count    kept points per direction (the direction succeeded, and the
//              point comes from the direction's last search pass)
//   k_scan     segment offsets (one block)
//   k_scatter  point indices into their direction's segment
//   k_keys     per kept point its M row (h entries, stride ks): the sort key
//              (c -> M = Binter c is injective, so M alone orders the points)
//   k_segsort  one block per segment: bitonic sort of the segment by M; up
//              to SORT_CAP points in shared memory with the first KEYN
//              entries of M there, ties on them decided from the full row
//   k_rows     the MH-wide M and Kn rows, q and pidx in output order
//
// The rows are exact in int64: the setup guarantees |Binter|, |Z Binter| <
// 2^25 and the search |c| < 2^31, so each product is below 2^56 and a sum of
// at most 63 of them below 2^62.
#pragma once
#include "pfg_types.cuh"

namespace pfg {

constexpr int KEYN = 4;           // M entries in a sort key
constexpr int SORT_CAP = 2048;    // segment size sorted in shared memory

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
    unsigned *pad;                // (2 n_kept + 64) scratch of the long segments
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

// exclusive scan of count[0..n) into seg[0..n] (one block, <= 1024 threads)
__global__ void k_scan(OutArgs O)
{
    __shared__ unsigned long long part[1024];
    const int t = threadIdx.x, nt = blockDim.x, n = O.n_dirs;
    const int per = (n + nt - 1) / nt, a = t * per, b = min(a + per, n);
    unsigned long long s = 0;
    for (int i = a; i < b; ++i) s += O.count[i];
    part[t] = s;
    __syncthreads();
    for (int o = 1; o < nt; o <<= 1) {
        unsigned long long x = t >= o ? part[t - o] : 0;
        __syncthreads();
        part[t] += x;
        __syncthreads();
    }
    unsigned long long run = t ? part[t - 1] : 0;
    for (int i = a; i < b; ++i) { O.seg[i] = run; run += O.count[i]; }
    if (t == nt - 1) O.seg[n] = part[nt - 1];
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

__global__ void k_keys(OutArgs O, unsigned long long n_kept)
{
    for (unsigned long long t = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; t < n_kept;
         t += (unsigned long long)gridDim.x * blockDim.x) {
        const unsigned k = O.idx[t];
        const Dir D = O.dirs[O.hdr[k].pid];
        const int64_t *BT = O.slab + D.slab + slab_layout(D.h, D.d).bt;
        const int32_t *c = O.coords + (unsigned long long)k * MD;
        int64_t *key = O.keys + t * O.ks;
        for (int r = 0; r < D.h; ++r) key[r] = row_entry(BT, c, D.d, D.h, r);
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

// One block per direction: bitonic sort of the segment's local positions by
// M, padded to a power of two with sentinels.  Segments up to SORT_CAP points
// sort in shared memory (with the first KEYN entries of each M row copied
// in); longer ones in the scratch region pad[2 s0, 2 s0 + np) with the rows
// read from global memory (np < 2 n, so the regions of different segments
// are disjoint).
__global__ void __launch_bounds__(256) k_segsort(OutArgs O)
{
#ifdef PFG_EMU
    static unsigned char smem_raw[SORT_CAP * KEYN * 8 + SORT_CAP * 4];
#else
    extern __shared__ __align__(16) unsigned char smem_raw[];
#endif
    int64_t *skeys = (int64_t *)smem_raw;                       // SORT_CAP x KEYN
    unsigned *sperm = (unsigned *)(skeys + SORT_CAP * KEYN);    // SORT_CAP
    constexpr unsigned NONE = 0xffffffffu;
    for (int pid = blockIdx.x; pid < O.n_dirs; pid += gridDim.x) {
        const unsigned long long s0 = O.seg[pid];
        const unsigned n = (unsigned)(O.seg[pid + 1] - s0);
        if (n < 2) continue;
        const Dir D = O.dirs[pid];
        unsigned np = 1;
        while (np < n) np <<= 1;
        const bool in_smem = np <= (unsigned)SORT_CAP;
        unsigned *a = in_smem ? sperm : O.pad + 2 * s0;
        if (in_smem)
            for (unsigned e = threadIdx.x; e < n * KEYN; e += blockDim.x) {
                const unsigned t = e / KEYN, r = e % KEYN;
                skeys[e] = (int)r < D.h ? O.keys[(s0 + t) * O.ks + r] : 0;
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
                    else if (in_smem) xgt = key_greater(O, skeys, s0, x, y, D.h);
                    else {                          // long segment: whole rows from global memory
                        const int64_t *kx = O.keys + (s0 + x) * O.ks, *ky = O.keys + (s0 + y) * O.ks;
                        int r = 0;
                        while (r < D.h && kx[r] == ky[r]) ++r;
                        xgt = r < D.h ? kx[r] > ky[r] : x > y;
                    }
                    if (xgt == up) { a[t] = y; a[u] = x; }
                }
                __syncthreads();
            }
        }
        // a holds the local positions in sorted order: map them to point indices in place
        for (unsigned t = threadIdx.x; t < n; t += blockDim.x) a[t] = O.idx[s0 + a[t]];
        __syncthreads();
        for (unsigned t = threadIdx.x; t < n; t += blockDim.x) O.idx[s0 + t] = a[t];
        __syncthreads();
    }
}

struct RowArgs {
    const Dir *dirs;
    const int64_t *slab;
    const PointHdr *hdr;
    const int32_t *coords;
    const unsigned *idx;          // points in output order
    unsigned long long n_out;
    int64_t pid_base;
    int64_t *M, *Kn, *q, *pidx;   // output (n_out, MH), (n_out,)
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
        const int64_t *BT = R.slab + D.slab + L.bt, *ZT = R.slab + D.slab + L.zt;
        const int32_t *c = R.coords + (unsigned long long)k * MD;
        const int32_t c0 = lane < d ? c[lane] : 0, c1 = lane + 32 < d ? c[lane + 32] : 0;
        int64_t m0 = 0, m1 = 0, k0 = 0, k1 = 0;
        for (int a = 0; a < d; ++a) {
            const int64_t ca = __shfl_sync(FULL, a < 32 ? c0 : c1, a & 31);
            if (lane < h) {
                m0 += (int64_t)(int32_t)BT[a * h + lane] * ca;
                k0 += (int64_t)(int32_t)ZT[a * h + lane] * ca;
            }
            if (lane + 32 < h) {
                m1 += (int64_t)(int32_t)BT[a * h + lane + 32] * ca;
                k1 += (int64_t)(int32_t)ZT[a * h + lane + 32] * ca;
            }
        }
        int64_t *Mr = R.M + t * MH, *Kr = R.Kn + t * MH;
        Mr[lane] = m0; Mr[lane + 32] = m1;
        Kr[lane] = k0; Kr[lane + 32] = k1;
        if (lane == 0) { R.q[t] = P.q; R.pidx[t] = R.pid_base + P.pid; }
    }
}

}  // namespace pfg
