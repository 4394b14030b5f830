// Output stage: the points the search emitted (direction, q, c) become the
// reference's output rows (M = Binter c, Kn = Z Binter c, q, pidx), grouped
// by direction and sorted by (M, Kn) within one (the canonical order of
// pfvs/gpu.py:155-159 and pfvs/coni.py:322-324; the reference sorts on the
// host, pfvs/fp_kernel/cuda/pfvs_gpu.cu:672-699).  All on the device:
//   k_expand   warp per point: M, Kn in int128 -> int64 (MH-wide rows)
//   k_count    kept points per direction (the direction succeeded, and the
//              point comes from the direction's last search pass)
//   k_scan     segment offsets (one block)
//   k_scatter  point indices into their direction's segment
//   k_segsort  one block per segment: bitonic sort of indices by (M, Kn)
//   k_gather   rows in output order
#pragma once
#include "pfg_types.cuh"

namespace pfg {

struct OutArgs {
    const Dir *dirs;
    const int64_t *slab;
    const PointHdr *hdr;
    const int32_t *coords;
    const int32_t *dir_pass;
    unsigned long long n_pts;
    int n_dirs;
    int64_t *Mfull, *Knfull;      // (n_pts, MH)
    int *dir_err;                 // per direction: an M/Kn overflow
    unsigned *count, *fill;       // per direction
    unsigned long long *seg;      // (n_dirs + 1) offsets
    unsigned *idx;                // (n_kept) point indices, segment-ordered
};

__device__ __forceinline__ bool dir_ok(int st) { return st == ST_PENDING || st == ST_OK; }

__global__ void k_expand(OutArgs O)
{
    const int lane = threadIdx.x & 31;
    const unsigned long long w = (blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x) >> 5;
    const unsigned long long nw = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
    for (unsigned long long k = w; k < O.n_pts; k += nw) {
        const int pid = O.hdr[k].pid;
        const Dir D = O.dirs[pid];
        const int h = D.h, d = D.d;
        const Slab L = slab_layout(h, d);
        const int64_t *BT = O.slab + D.slab + L.bt, *ZT = O.slab + D.slab + L.zt;
        const int32_t *c = O.coords + k * MD;
        bool bad = false;
        for (int r = lane; r < MH; r += 32) {
            int64_t mv = 0, kv = 0;
            if (r < h) {
                i128 am = 0, ak = 0;
                for (int a = 0; a < d; ++a) {
                    am += (i128)BT[a * h + r] * c[a];
                    ak += (i128)ZT[a * h + r] * c[a];
                }
                if (!fits64(am) || !fits64(ak)) bad = true;
                mv = (int64_t)am; kv = (int64_t)ak;
            }
            O.Mfull[k * MH + r] = mv;
            O.Knfull[k * MH + r] = kv;
        }
        if (__any_sync(FULL, bad) && lane == 0) atomicExch(&O.dir_err[pid], 1);
    }
}

__device__ __forceinline__ bool keep_point(const OutArgs &O, unsigned long long k)
{
    const int pid = O.hdr[k].pid;
    return dir_ok(O.dirs[pid].status) && !O.dir_err[pid] && O.hdr[k].pad == O.dir_pass[pid];
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

// lexicographic (M, Kn) comparison of two points of one direction
__device__ __forceinline__ bool row_less(const OutArgs &O, unsigned a, unsigned b, int h)
{
    const int64_t *Ma = O.Mfull + (unsigned long long)a * MH, *Mb = O.Mfull + (unsigned long long)b * MH;
    for (int r = 0; r < h; ++r) if (Ma[r] != Mb[r]) return Ma[r] < Mb[r];
    const int64_t *Ka = O.Knfull + (unsigned long long)a * MH, *Kb = O.Knfull + (unsigned long long)b * MH;
    for (int r = 0; r < h; ++r) if (Ka[r] != Kb[r]) return Ka[r] < Kb[r];
    return a < b;
}

constexpr int SORT_SMEM = 4096;

// One block per direction: bitonic sort of the segment's indices, padded to
// a power of two with +infinity sentinels.  Segments up to SORT_SMEM points
// sort in shared memory; longer ones in the scratch region pad[2 s0, 2 s0 + np)
// (np < 2 n, so the regions of different segments are disjoint).
__global__ void __launch_bounds__(256) k_segsort(OutArgs O, unsigned *pad)
{
    __shared__ unsigned sh[SORT_SMEM];
    for (int pid = blockIdx.x; pid < O.n_dirs; pid += gridDim.x) {
        const unsigned long long s0 = O.seg[pid];
        const unsigned n = (unsigned)(O.seg[pid + 1] - s0);
        if (n < 2) continue;
        const int h = O.dirs[pid].h;
        unsigned np = 1;
        while (np < n) np <<= 1;
        unsigned *g = O.idx + s0;
        unsigned *a = np <= SORT_SMEM ? sh : pad + 2 * s0;
        for (unsigned t = threadIdx.x; t < np; t += blockDim.x) a[t] = t < n ? g[t] : 0xffffffffu;
        __syncthreads();
        for (unsigned k = 2; k <= np; k <<= 1) {
            for (unsigned j = k >> 1; j > 0; j >>= 1) {
                for (unsigned t = threadIdx.x; t < np; t += blockDim.x) {
                    const unsigned u = t ^ j;
                    if (u <= t) continue;
                    const bool up = (t & k) == 0;
                    const unsigned x = a[t], y = a[u];
                    bool xgt;                       // x > y
                    if (x == 0xffffffffu) xgt = y != 0xffffffffu;
                    else if (y == 0xffffffffu) xgt = false;
                    else xgt = row_less(O, y, x, h);
                    if (xgt == up) { a[t] = y; a[u] = x; }
                }
                __syncthreads();
            }
        }
        for (unsigned t = threadIdx.x; t < n; t += blockDim.x) g[t] = a[t];
        __syncthreads();
    }
}

struct GatherArgs {
    const unsigned *idx;
    const PointHdr *hdr;
    const int64_t *Mfull, *Knfull;
    unsigned long long n_out;
    int64_t pid_base;
    int64_t *M, *Kn, *q, *pidx;   // output (n_out, MH), (n_out,)
};

__global__ void k_gather(GatherArgs G)
{
    const unsigned long long tid = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
    const unsigned long long nt = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long e = tid; e < G.n_out * MH; e += nt) {
        const unsigned long long t = e / MH, r = e % MH;
        const unsigned k = G.idx[t];
        G.M[e] = G.Mfull[(unsigned long long)k * MH + r];
        G.Kn[e] = G.Knfull[(unsigned long long)k * MH + r];
        if (r == 0) { G.q[t] = G.hdr[k].q; G.pidx[t] = G.pid_base + G.hdr[k].pid; }
    }
}

}  // namespace pfg
