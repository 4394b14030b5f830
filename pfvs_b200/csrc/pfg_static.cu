// pfg_coni_direction_static: the whole coni pipeline for ONE p-vector in one
// launch of one warp, with every scratch buffer in a file-scope static
// device array -- so the call allocates nothing.
//
// Who needs it: callers that must not (or cannot) call cudaMalloc while they
// run -- code inside a framework that owns all device memory through its own
// pool or arena (an XLA/JAX custom call, a TensorRT plugin, an inference
// server with a fixed budget), where an allocation of its own would go around
// that pool or fail, or a real-time path that may not block on the
// allocator.  They pass device
// buffers for the inputs and outputs; the scratch the kernels need (the
// lattice setup's working arrays, the direction's lattice data, the search's
// point staging and the sort indices) lives in g_static below, which every
// GPU that loads this library holds, about 3 MB, until the process exits.
//
// The work is the same as pfg_coni_batch's for that p-vector (setup, FP64-
// pruned search, M = Binter c / Kn = Z Binter c, canonical (M, Kn) order),
// with the same device functions, so its output is bit-identical.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/pfvs_gpu.h"

// The device sources, with internal linkage here: the batch pipeline's
// translation unit (pfg_abi.cu) defines the same kernels.
namespace {
#include "pfg_int.cuh"
#include "pfg_types.cuh"
#include "pfg_setup.cuh"
#include "pfg_search.cuh"
}  // namespace

namespace {
using namespace pfg;

constexpr int STATIC_MAX_POINTS = PFG_STATIC_MAX_POINTS;
// words of one direction's slab at h = MH (slab_layout in pfg_types.cuh)
constexpr int STATIC_SLAB_WORDS = 2 * MD * MH + 3 * MD * MD + (MD * MD + 1) / 2 + MD + (MD + 1) / 2;

struct StaticScratch {
    SetupScratch setup;                         // the setup's working arrays (one warp)
    int64_t slab[STATIC_SLAB_WORDS + 8];        // this direction's lattice data
    Geo geo;
    Dir dir;
    SearchCtl ctl;
    int32_t zero32[4];
    int64_t zero64[4];
    unsigned long long dir_nodes[2];
    PointHdr hdr[STATIC_MAX_POINTS];
    int32_t coords[STATIC_MAX_POINTS * MD];
    int64_t Mrow[STATIC_MAX_POINTS * MH];       // unsorted rows
    int64_t Krow[STATIC_MAX_POINTS * MH];
    unsigned idx[STATIC_MAX_POINTS];
    unsigned char stage[56 * 1024];             // the search's staging area (stage_bytes<double>(63, 64))
};

// The scratch.  In host code `g_static` names a host-side stand-in, not the
// device array: its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) StaticScratch g_static;

__device__ bool row_less_static(const StaticScratch &S, unsigned a, unsigned b, int h)
{
    const int64_t *Ma = S.Mrow + (size_t)a * MH, *Mb = S.Mrow + (size_t)b * MH;
    for (int r = 0; r < h; ++r) if (Ma[r] != Mb[r]) return Ma[r] < Mb[r];
    const int64_t *Ka = S.Krow + (size_t)a * MH, *Kb = S.Krow + (size_t)b * MH;
    for (int r = 0; r < h; ++r) if (Ka[r] != Kb[r]) return Ka[r] < Kb[r];
    return a < b;
}

__global__ void __launch_bounds__(32) k_direction_static(StaticScratch *S, int h, int64_t Q, int64_t qmax,
                                                         int64_t linmin, const int64_t *kappa,
                                                         const int64_t *Mbasis, const int64_t *p,
                                                         int64_t cap, int64_t *M, int64_t *Kn, int64_t *q,
                                                         int64_t *n_out, int32_t *status)
{
    const int lane = threadIdx.x & 31;
    const int d = h - 1;
    const Slab L = slab_layout(h, d);
    // everything the previous call left in the scratch that must start from zero
    if (lane == 0) {
        Geo &g = S->geo;
        g.h = h; g.d = d; g.use_f32 = 0; g.coni = 1;
        g.Q = Q; g.qmax = qmax; g.linmin = linmin;
        g.koff = 0; g.moff = 0; g.slab_len = L.len;
        S->zero32[0] = 0; S->zero64[0] = 0;
        memset(&S->ctl, 0, sizeof S->ctl);
        S->dir_nodes[0] = 0;
        Dir &D = S->dir;
        D.geo = 0; D.h = h; D.d = d; D.slab = 0; D.status = ST_PENDING;
        D.m0_level = -1; D.g_lin = 0; D.hrows = 0; D.slack_chol = 0.0; D.pad = 0; D.wide = 0;
    }
    __syncwarp();
    // setup (the batch kernel's per-direction step, pfg_setup.cuh)
    SetupArgs SA{&S->geo, kappa, Mbasis, p, S->zero32, S->zero64, S->slab, &S->dir, &S->setup, 1, nullptr};
    int stage = 0;
    if (lane == 0) S->setup.core.B = S->setup.Bstore;
    __syncwarp();
    int st = setup_one<MH>(SA, 0, lane, stage, &S->setup.core);
    if (lane == 0) { S->dir.status = st; S->dir.pad = st < 0 ? stage : 0; }
    __syncwarp();
    // search (FP64 pruning, no work sharing)
    unsigned long long npts = 0;
    if (st == ST_PENDING) {
        SearchArgs A{};
        A.geo = &S->geo; A.dirs = &S->dir; A.slab = S->slab; A.todo = S->zero32; A.n_todo = 1;
        A.pass = 1; A.ctl = &S->ctl; A.items = nullptr; A.ready = nullptr; A.q_cap = 0;
        A.hdr = S->hdr; A.coords = S->coords; A.pts_cap = STATIC_MAX_POINTS; A.npts = &S->ctl.npts;
        A.dir_nodes = S->dir_nodes; A.eps = 1e-4; A.donate = 0; A.n_warps = 1;
        A.wait_ns = 30ll * 1000000000ll; A.deadline_ns = 120ll * 1000000000ll;
        Tally T{0, 0, 0};
        static_assert(sizeof(StaticScratch::stage) >= 49664, "staging area");
        const Prob<double> P = load_prob<double>(A, 0, S->stage, lane);
        st = run_subtree<double, 2>(A, P, 0, nullptr, T, lane);
        npts = shfl(S->ctl.npts, 0);
        if (st == 0 && npts > (unsigned long long)cap) st = -2;   // more points than the caller's buffers
        if (st == 0 && npts > (unsigned long long)STATIC_MAX_POINTS) st = -2;
    } else if (st == ST_EMPTY) {
        st = 0;
    }
    // M, Kn (int128 -> int64) into the scratch rows, then the canonical order
    if (st == 0 && npts) {
        const int64_t *BT = S->slab + L.bt, *ZT = S->slab + L.zt;
        bool bad = false;
        for (unsigned long long k = 0; k < npts; ++k) {
            const int32_t *c = S->coords + k * MD;
            for (int r = lane; r < MH; r += 32) {
                int64_t mv = 0, kv = 0;
                if (r < h) {
                    i128 am = 0, ak = 0;
                    for (int a = 0; a < d; ++a) { am += (i128)BT[a * h + r] * c[a]; ak += (i128)ZT[a * h + r] * c[a]; }
                    if (!fits64(am) || !fits64(ak)) bad = true;
                    mv = (int64_t)am; kv = (int64_t)ak;
                }
                S->Mrow[k * MH + r] = mv;
                S->Krow[k * MH + r] = kv;
            }
        }
        if (__any_sync(FULL, bad)) st = ST_OVERFLOW;
        __syncwarp();
    }
    if (st == 0 && npts) {
        unsigned np = 1;
        while (np < npts) np <<= 1;
        for (unsigned t = lane; t < np; t += 32) S->idx[t] = t < npts ? t : 0xffffffffu;
        __syncwarp();
        for (unsigned k = 2; k <= np; k <<= 1)
            for (unsigned j = k >> 1; j > 0; j >>= 1) {
                for (unsigned t = lane; t < np; t += 32) {
                    const unsigned u = t ^ j;
                    if (u <= t) continue;
                    const bool up = (t & k) == 0;
                    const unsigned x = S->idx[t], y = S->idx[u];
                    bool xgt;
                    if (x == 0xffffffffu) xgt = y != 0xffffffffu;
                    else if (y == 0xffffffffu) xgt = false;
                    else xgt = row_less_static(*S, y, x, h);
                    if (xgt == up) { S->idx[t] = y; S->idx[u] = x; }
                }
                __syncwarp();
            }
        for (unsigned long long t = 0; t < npts; ++t) {
            const unsigned k = S->idx[t];
            for (int r = lane; r < MH; r += 32) {
                M[t * MH + r] = S->Mrow[(size_t)k * MH + r];
                Kn[t * MH + r] = S->Krow[(size_t)k * MH + r];
            }
            if (lane == 0) q[t] = S->hdr[k].q;
        }
    }
    if (lane == 0) {
        *n_out = st == 0 ? (int64_t)npts : 0;
        *status = (st == ST_OK || st == ST_PENDING) ? 0 : st;
    }
}

std::mutex g_sym_mu;
StaticScratch *g_sym_addr[64] = {};     // device address of g_static, per device

}  // namespace

// See include/pfvs_gpu.h.
extern "C" int pfg_coni_direction_static(int h, int64_t Q, int64_t qmax, int64_t linmin,
                                         const int64_t *kappa, const int64_t *Mbasis, const int64_t *p,
                                         int64_t cap, int64_t *M, int64_t *Kn, int64_t *q,
                                         int64_t *n_out, int32_t *status, void *stream)
{
    if (h < 3 || h > MH) {
        fprintf(stderr, "pfg_coni_direction_static: h11 = %d outside 3..%d\n", h, MH);
        return 1;
    }
    if (cap < 0 || cap > STATIC_MAX_POINTS) {
        fprintf(stderr, "pfg_coni_direction_static: cap = %lld outside 0..%d (the static scratch holds "
                        "at most %d points)\n", (long long)cap, STATIC_MAX_POINTS, STATIC_MAX_POINTS);
        return 1;
    }
    if (Q <= 0 || qmax < 0 || !kappa || !Mbasis || !p || !n_out || !status || (cap && (!M || !Kn || !q))) {
        fprintf(stderr, "pfg_coni_direction_static: bad arguments\n");
        return 1;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 1;
    StaticScratch *S = nullptr;
    {
        // once per device, with that device current (first call: before any stream capture)
        std::lock_guard<std::mutex> g(g_sym_mu);
        if (!g_sym_addr[dev]) {
            void *a = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&a, g_static);
            if (e != cudaSuccess) {
                fprintf(stderr, "pfg_coni_direction_static: cudaGetSymbolAddress: %s\n", cudaGetErrorString(e));
                return 1;
            }
            g_sym_addr[dev] = (StaticScratch *)a;
        }
        S = g_sym_addr[dev];
    }
    k_direction_static<<<1, 32, 0, (cudaStream_t)stream>>>(S, h, Q, qmax, linmin, kappa, Mbasis, p, cap, M, Kn,
                                                          q, n_out, status);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "pfg_coni_direction_static: launch: %s\n", cudaGetErrorString(e));
        return 1;
    }
    return 0;
}
