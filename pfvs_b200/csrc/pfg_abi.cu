// libpfvs_gpu.so: host side of the batched coni pipeline and its C ABI
// (include/pfvs_gpu.h).  Per batch of directions, on one stream:
//   k_setup<.,0..2>  lattice setup in three phase kernels, one warp per
//                direction                                 (pfg_setup.cuh)
//   k_search<f>  FP32-pruned persistent search            (pfg_search.cuh)
//   k_flip       FP32 successes -> done; -11 -> FP64 retry
//   k_search<d>  FP64-pruned search of the rest
//   k_count .. k_rows      canonical output rows              (pfg_out.cuh)
//   k_pfv_count .. k_pfv_rows   points -> PFVs (pfg_coni_pfvs)  (pfg_pfv.cuh)
// with one host synchronisation at the end of a batch (point count, output
// size).  The point rows of a batch go to the caller's pinned block on a
// second (copy) stream, overlapping the next batch when there are several.  No CPU fallback: a
// direction the device cannot finish exactly is reported with a negative
// status.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "../../include/pfvs_gpu.h"
#include "pfg_int.cuh"
#include "pfg_types.cuh"
#include "pfg_setup.cuh"
#include "pfg_search.cuh"
#include "pfg_out.cuh"
#include "pfg_pfv.cuh"
#include "pfg_mu0.cuh"
#include "pfg_zpk.cuh"

using namespace pfg;

namespace {

// Between the FP32 and FP64 passes: an FP32-searched direction is done, or
// (status -11) goes to the FP64 pass; every direction the FP64 pass will
// search keeps only that pass's points (dir_pass = 2).
__global__ void k_flip(Dir *dirs, const Geo *geo, int n, int f32_used, int32_t *dir_pass,
                       unsigned long long *retries)
{
    for (int pid = blockIdx.x * blockDim.x + threadIdx.x; pid < n; pid += gridDim.x * blockDim.x) {
        Dir &D = dirs[pid];
        if (!(f32_used && geo[D.geo].use_f32)) { dir_pass[pid] = 2; continue; }
        if (D.status == ST_PENDING) D.status = ST_OK;
        else if (D.status == ST_FLOAT) { D.status = ST_PENDING; dir_pass[pid] = 2; atomicAdd(retries, 1ull); }
    }
}

__global__ void k_fill_i32(int32_t *a, int32_t v, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = v;
}

enum {
    W_GEO, W_KAPPA, W_MB, W_PS, W_PGEO, W_SLABOFF, W_SLAB, W_DIRS, W_SCRATCH, W_TODO32, W_TODOALL, W_ORDER,
    W_CTL, W_ITEMS, W_READY, W_HDR, W_COORDS, W_DIRNODES, W_DIRPASS,
    W_KEYS, W_COUNT, W_FILL, W_SEG, W_IDX, W_CSEG, W_SUM, W_PERM, W_PERM2, W_SIDX, W_PCNT, W_PKG, W_PEPT, W_PEG, W_PEK0, W_PEORD, W_PNONS, W_PKEEP,
    W_PERR, W_PSORT, W_PK, W_PM, W_PP, W_PRIMES, W_OM, W_OK, W_OQ, W_OP, W_OM2, W_OK2, W_OQ2, W_OP2, W_RETRY,
    W_ROWS, W_MU_K, W_MU_P, W_MU_ST, W_MU_NUM, W_MU_DEN, W_MU_KO, W_MU_SCR, W_MU_CTR,
    W_ZK_MB, W_ZK_PS, W_ZK_SCR, W_ZK_CTR, W_ZK_ST, W_ZK_M, W_ZK_K, W_ZK_Q, W_ZK_P, W_N
};

struct Workspace {
    std::mutex mu;
    void *p[W_N] = {};
    size_t cap[W_N] = {};
    unsigned long long pts_cap = 1ull << 20;    // point buffer: grows to the largest batch seen
    double rows_per_dir = 0.0;                  // output rows per direction of the last call
    cudaStream_t copy = nullptr;                // device-to-host row copies (non-blocking)
    cudaEvent_t rows_done[2] = {}, copied[2] = {};  // per output slot: rows written / copied out
    bool copy_pending[2] = {false, false};
};

std::mutex g_ws_mu;
std::map<int, Workspace *> g_ws;

Workspace &workspace(int dev)
{
    std::lock_guard<std::mutex> g(g_ws_mu);
    Workspace *&w = g_ws[dev];
    if (!w) w = new Workspace();
    return *w;
}

// pfg_debug_fail_alloc: allocations left before the one made to fail (0: none)
std::atomic<int> g_fail_alloc{0};

cudaError_t ws_get(Workspace &W, int slot, size_t bytes, void **out)
{
    if (bytes == 0) bytes = 16;
    if (W.cap[slot] < bytes) {
        if (W.p[slot]) cudaFree(W.p[slot]);
        W.p[slot] = nullptr;
        W.cap[slot] = 0;
        size_t b = bytes + bytes / 8 + 256;
        if (g_fail_alloc.load() > 0 && g_fail_alloc.fetch_sub(1) == 1) return cudaErrorMemoryAllocation;
        cudaError_t e = cudaMalloc(&W.p[slot], b);
        if (e != cudaSuccess) { W.p[slot] = nullptr; return e; }
        W.cap[slot] = b;
    }
    *out = W.p[slot];
    return cudaSuccess;
}

void ws_release(Workspace &W, int keep_below = 0)
{
    for (int k = keep_below; k < W_N; ++k) {
        if (W.p[k]) cudaFree(W.p[k]);
        W.p[k] = nullptr;
        W.cap[k] = 0;
    }
}

// Pinned host blocks for the output arrays handed to the caller: the rows
// come back by DMA at full link speed, and pfg_output_free returns a block
// to an idle list for the next call instead of unpinning it.
struct PinnedPool {
    std::mutex mu;
    std::map<void *, size_t> live;              // handed out: block -> capacity
    std::multimap<size_t, void *> idle;         // capacity -> block
    size_t idle_bytes = 0;
};
constexpr size_t PINNED_IDLE_MAX = 24ull << 30;

PinnedPool &pinned()
{
    static PinnedPool *P = new PinnedPool();
    return *P;
}

void *pinned_get(size_t bytes)
{
    bytes = std::max<size_t>(bytes, 64);
    PinnedPool &P = pinned();
    {
        std::lock_guard<std::mutex> g(P.mu);
        auto it = P.idle.lower_bound(bytes);
        if (it != P.idle.end() && it->first <= 2 * bytes + (1u << 20)) {
            void *p = it->second;
            P.live[p] = it->first;
            P.idle_bytes -= it->first;
            P.idle.erase(it);
            return p;
        }
    }
    void *p = nullptr;
    if (cudaHostAlloc(&p, bytes, cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    std::lock_guard<std::mutex> g(P.mu);
    P.live[p] = bytes;
    return p;
}

// false if p is not a pinned block of this pool
bool pinned_put(void *p)
{
    if (!p) return true;
    PinnedPool &P = pinned();
    size_t cap;
    {
        std::lock_guard<std::mutex> g(P.mu);
        auto it = P.live.find(p);
        if (it == P.live.end()) return false;
        cap = it->second;
        P.live.erase(it);
        if (P.idle_bytes + cap <= PINNED_IDLE_MAX) {
            P.idle.emplace(cap, p);
            P.idle_bytes += cap;
            return true;
        }
    }
    cudaFreeHost(p);
    return true;
}

void pinned_release_idle()
{
    PinnedPool &P = pinned();
    std::multimap<size_t, void *> idle;
    {
        std::lock_guard<std::mutex> g(P.mu);
        idle.swap(P.idle);
        P.idle_bytes = 0;
    }
    for (auto &e : idle) cudaFreeHost(e.second);
}

// The caller's point rows: one pinned block per array, filled batch by batch
// by asynchronous copies on the workspace's copy stream.
struct RowSink {
    int64_t *M = nullptr, *Kn = nullptr, *q = nullptr, *pidx = nullptr;
    size_t n = 0, cap = 0;
    int w = MH;                                 // entries per M / Kn row
    bool alloc(size_t rows, int width)
    {
        w = width;
        M = (int64_t *)pinned_get(rows * w * 8);
        Kn = (int64_t *)pinned_get(rows * w * 8);
        q = (int64_t *)pinned_get(rows * 8);
        pidx = (int64_t *)pinned_get(rows * 8);
        cap = rows;
        return M && Kn && q && pidx;
    }
    void release()
    {
        for (int64_t *p : {M, Kn, q, pidx}) pinned_put(p);
        M = Kn = q = pidx = nullptr;
        n = cap = 0;
    }
};

// PFVs of a pfg_coni_pfvs call, per batch
struct PfvChunk { int64_t *K, *M, *pidx; size_t n; };
struct PfvSink {
    std::vector<PfvChunk> chunks;
    int64_t n_points = 0;
    void release()
    {
        for (auto &c : chunks) for (int64_t *p : {c.K, c.M, c.pidx}) pinned_put(p);
        chunks.clear();
    }
};

// the first n primes below 2^31, descending (deterministic Miller-Rabin for
// 32-bit numbers: bases 2, 3, 5, 7)
bool is_prime32(uint32_t n)
{
    if (n < 2) return false;
    for (uint32_t p : {2u, 3u, 5u, 7u}) if (n % p == 0) return n == p;
    uint32_t d = n - 1;
    int r = 0;
    while (!(d & 1)) { d >>= 1; ++r; }
    auto mulm = [n](uint64_t a, uint64_t b) { return (uint32_t)((a * b) % n); };
    for (uint32_t a : {2u, 3u, 5u, 7u}) {
        uint64_t x = 1, b = a, e = d;
        while (e) { if (e & 1) x = mulm(x, b); b = mulm(b, b); e >>= 1; }
        if (x == 1 || x == n - 1) continue;
        bool comp = true;
        for (int i = 1; i < r && comp; ++i) { x = mulm(x, x); if (x == n - 1) comp = false; }
        if (comp) return false;
    }
    return true;
}
const std::vector<uint32_t> &primes31()
{
    static std::vector<uint32_t> P = [] {
        std::vector<uint32_t> v;
        for (uint32_t n = 2147483647u; v.size() < 64; n -= 2) if (is_prime32(n)) v.push_back(n);
        return v;
    }();
    return P;
}

double dbits(unsigned long long b)
{
    double x;
    memcpy(&x, &b, sizeof x);
    return x;
}

void set_err(pfg_output *out, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(out->err, sizeof out->err, fmt, ap);
    va_end(ap);
}

}  // namespace

#define CK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { \
    set_err(out, "%s (%s:%d)", cudaGetErrorString(e_), __FILE__, __LINE__); rc = 1; goto fail; } } while (0)
#define WS(ptr, slot, bytes) CK(ws_get(W, slot, (size_t)(bytes), (void **)&(ptr)))
// inside the batch loop: out of device memory -> the batch again at half size
#define WSB(ptr, slot, bytes) do { cudaError_t eb_ = ws_get(W, slot, (size_t)(bytes), (void **)&(ptr)); \
    if (eb_ == cudaErrorMemoryAllocation && nb > 1) goto out_of_memory; CK(eb_); } while (0)

extern "C" int pfg_max_h11(void) { return MH; }

#ifdef PFG_STAGE_CLOCKS
// profiling build only: read (and zero) the setup's per-stage cycle counters
extern "C" int pfg_debug_stage_cycles(unsigned long long *out)
{
    if (cudaMemcpyFromSymbol(out, pfg::pfg_stage_cycles, sizeof(unsigned long long) * 64) != cudaSuccess) return 1;
    unsigned long long z[64] = {};
    return cudaMemcpyToSymbol(pfg::pfg_stage_cycles, z, sizeof z) != cudaSuccess;
}
// profiling build only: the search's busy / waiting cycles and subtree counts (and zero them)
extern "C" int pfg_debug_search_cycles(unsigned long long *out)
{
    if (cudaMemcpyFromSymbol(out, pfg::pfg_search_cycles, sizeof(unsigned long long) * 16) != cudaSuccess) return 1;
    unsigned long long z[16] = {};
    return cudaMemcpyToSymbol(pfg::pfg_search_cycles, z, sizeof z) != cudaSuccess;
}
#endif
extern "C" const char *pfg_backend(void) { return "cuda"; }

extern "C" int pfg_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

extern "C" void pfg_output_free(pfg_output *out)
{
    for (int64_t *p : {out->M, out->Kn, out->q, out->pidx})
        if (!pinned_put(p)) free(p);
    free(out->pstat);
    out->M = out->Kn = out->q = out->pidx = nullptr;
    out->pstat = nullptr;
    out->n = 0;
}

extern "C" void pfg_release(int device)
{
    Workspace &W = workspace(device);
    std::lock_guard<std::mutex> g(W.mu);
    if (cudaSetDevice(device) == cudaSuccess) ws_release(W);
    pinned_release_idle();
}

extern "C" void pfg_debug_fail_alloc(int k) { g_fail_alloc.store(k > 0 ? k : 0); }

extern "C" int pfg_coni_batch(const pfg_input *in, pfg_output *out)
{
    return pfg_coni_batch_ex(in, nullptr, out, nullptr, nullptr);
}

// Lattice points -> coni PFVs on the device (pfg_pfv.cuh) for n_out points in
// device memory (rows of MH, pidx from pid_base; dirs / geo / kappa as the
// setup wrote them): the PFVs are appended to pfv as one pinned chunk.
// Returns 0, 1 with err set, or 2 when a device allocation ran out of memory
// (err set too; the caller may retry with a smaller batch).
static int pfv_stage(Workspace &W, int nsm, const Dir *ddirs, const Geo *dgeo, const int64_t *dkappa,
                     const int64_t *oM, const int64_t *oK, const int64_t *oq, const int64_t *op,
                     unsigned long long n_out, int64_t pid_base, int hmax2, PfvSink *pfv, int64_t &launches,
                     char *err)
{
    cudaError_t e;
#define PCK(x) do { e = (x); if (e != cudaSuccess) { snprintf(err, 256, "%s (%s:%d)", cudaGetErrorString(e), \
    __FILE__, __LINE__); return 1; } } while (0)
#define PWS(ptr, slot, bytes) do { e = ws_get(W, slot, (size_t)(bytes), (void **)&(ptr)); \
    if (e != cudaSuccess) { snprintf(err, 256, "%s (%s:%d)", cudaGetErrorString(e), __FILE__, __LINE__); \
    return e == cudaErrorMemoryAllocation ? 2 : 1; } } while (0)
    pfv->n_points += (int64_t)n_out;
    unsigned long long *pcnt, *pkeep; uint64_t *pkg; unsigned *pept, *peord, *psort;
    int64_t *peg, *pek0; int *pnons, *perr; uint32_t *dprimes;
    PWS(pcnt, W_PCNT, (n_out + 1) * 8);
    PWS(pkg, W_PKG, n_out * 8);
    PWS(pnons, W_PNONS, n_out * 4);
    PWS(perr, W_PERR, 64);
    PWS(dprimes, W_PRIMES, primes31().size() * 4);
    PCK(cudaMemset(perr, 0, 64));
    PCK(cudaMemcpy(dprimes, primes31().data(), primes31().size() * 4, cudaMemcpyHostToDevice));
    PfvArgs PA{ddirs, dgeo, dkappa, oM, oK, oq, op, n_out, pid_base, pcnt, pkg, nullptr, nullptr, nullptr,
               nullptr, pnons, nullptr, perr, dprimes, (int)primes31().size(), hmax2 - 1};
    k_pfv_count<<<nsm * 4, 256>>>(PA); ++launches;
    k_scan64<<<1, 1024>>>(pcnt, n_out); ++launches;
    unsigned long long n_e = 0;
    PCK(cudaMemcpy(&n_e, pcnt + n_out, 8, cudaMemcpyDeviceToHost));
    unsigned long long n_pfv = 0;
    if (n_e) {
        unsigned np2 = 1;
        while (np2 < n_e) np2 <<= 1;
        PWS(pept, W_PEPT, n_e * 4);
        PWS(peg, W_PEG, n_e * 8);
        PWS(pek0, W_PEK0, n_e * 8);
        PWS(peord, W_PEORD, n_e * 4);
        PWS(pkeep, W_PKEEP, (n_e + 1) * 8);
        PWS(psort, W_PSORT, (size_t)np2 * 4);
        PA.e_pt = pept; PA.e_g = peg; PA.e_K0 = pek0; PA.e_ord = peord; PA.keep = pkeep;
        k_pfv_fill<<<nsm * 4, 256>>>(PA); ++launches;
        k_pfv_sort<<<1, 1024>>>(PA, n_e, np2, psort); ++launches;
        k_pfv_det<<<(int)std::min<unsigned long long>(n_out, (unsigned long long)nsm * 32), 32,
                    (size_t)(hmax2 - 1) * (hmax2 - 1) * 12>>>(PA); ++launches;
        k_pfv_keep<<<nsm * 4, 256>>>(PA, n_e); ++launches;
        k_scan64<<<1, 1024>>>(pkeep, n_e); ++launches;
        PCK(cudaGetLastError());
        PCK(cudaMemcpy(&n_pfv, pkeep + n_e, 8, cudaMemcpyDeviceToHost));
    }
    int herr[3] = {0, 0, 0};
    if (n_pfv) {
        int64_t *pK, *pM, *pP;
        PWS(pK, W_PK, n_pfv * MH * 8);
        PWS(pM, W_PM, n_pfv * MH * 8);
        PWS(pP, W_PP, n_pfv * 8);
        k_pfv_rows<<<nsm * 8, 256>>>(PA, n_e, pK, pM, pP); ++launches;
        PCK(cudaGetLastError());
        PfvChunk c{(int64_t *)pinned_get(n_pfv * MH * 8), (int64_t *)pinned_get(n_pfv * MH * 8),
                   (int64_t *)pinned_get(n_pfv * 8), (size_t)n_pfv};
        pfv->chunks.push_back(c);
        if (!c.K || !c.M || !c.pidx) { snprintf(err, 256, "out of pinned host memory"); return 1; }
        PCK(cudaMemcpy(c.K, pK, n_pfv * MH * 8, cudaMemcpyDeviceToHost));
        PCK(cudaMemcpy(c.M, pM, n_pfv * MH * 8, cudaMemcpyDeviceToHost));
        PCK(cudaMemcpy(c.pidx, pP, n_pfv * 8, cudaMemcpyDeviceToHost));
    }
    PCK(cudaMemcpy(herr, perr, sizeof herr, cudaMemcpyDeviceToHost));
    if (herr[0]) { snprintf(err, 256, "Tadpole violation: -dot(K,M) > Q"); return 1; }
    if (herr[1] == 2) { snprintf(err, 256, "determinant test: more primes needed than provided"); return 1; }
    if (herr[1]) { snprintf(err, 256, "PFV entries beyond int64"); return 1; }
    if (herr[2]) { snprintf(err, 256, "a point expands over more than 2^22 values of g"); return 1; }
    return 0;
#undef PCK
#undef PWS
}

// The pipeline over all batches: points into `out`, or, with `pfv`, the
// points' PFVs into `pfv` (the points stay on the device).
static int coni_run(const pfg_input *in, const pfg_options *opt_in, pfg_output *out, pfg_stats *stats,
                    int64_t *dir_nodes_out, PfvSink *pfv, int coni = 1)
{
    memset(out, 0, sizeof *out);
    if (stats) memset(stats, 0, sizeof *stats);
    pfg_options opt = {PFG_FORM_BATCHED, PFG_PREC_AUTO, 0, 0, 0.0, 0.0, 0.0, 0, 0};
    if (opt_in) opt = *opt_in;
    const long long wait_ns = opt.wait_s > 0 ? (long long)(opt.wait_s * 1e9) : 30ll * 1000000000ll;
    const long long deadline_ns = opt.deadline_s > 0 ? (long long)(opt.deadline_s * 1e9) : 120ll * 1000000000ll;
    const double gcd_min_tree = opt.gcd_min_tree == 0.0 ? GCD_MIN_TREE_DEFAULT
                                : (opt.gcd_min_tree < 0.0 ? 0.0 : opt.gcd_min_tree);
    const int64_t NP = in->n_p;
    if (NP < 0 || in->n_geo < 0) { set_err(out, "negative sizes"); return 1; }
    // width of the M / Kn rows handed back: MH (the reference's layout), or with
    // compact_rows the widest h11 of the call (the PFV path keeps MH internally)
    int rw = MH;
    if (opt.compact_rows && !pfv) {
        rw = 3;
        for (int gi = 0; gi < in->n_geo; ++gi) rw = std::max(rw, (int)in->h[gi]);
        rw = std::min(rw, MH);
    }
    std::vector<Geo> geos(in->n_geo);
    {
        int64_t koff = 0, moff = 0;
        for (int gi = 0; gi < in->n_geo; ++gi) {
            Geo &g = geos[gi];
            g.h = in->h[gi];
            g.d = g.h - 1;
            g.Q = in->Q[gi]; g.qmax = in->qmax[gi];
            g.coni = coni;
            g.linmin = coni ? in->linmin[gi] : 0;     // (non-coni: no M0 cut)
            // (a non-coni geometry's GCD rows start from all h rows of ZB: h <= MH - 1)
            if (g.h < 3 || g.h > MH - (coni ? 0 : 1) || g.Q <= 0 || g.qmax < 0) {
                set_err(out, "geometry %d: unsupported h11 = %d (3..%d), Q or qmax", gi, g.h, MH - (coni ? 0 : 1));
                return 1;
            }
            g.use_f32 = g.qmax < (1LL << 22) && opt.precision == PFG_PREC_FP32;
            g.koff = koff; g.moff = moff;
            g.slab_len = slab_layout(g.h, g.d).len;
            koff += (int64_t)g.h * g.h * g.h;
            moff += (int64_t)g.h * g.h;
        }
    }
    for (int64_t ip = 0; ip < NP; ++ip)
        if (in->pgeo[ip] < 0 || in->pgeo[ip] >= in->n_geo) {
            set_err(out, "p %lld: bad geometry index", (long long)ip);
            return 1;
        }
    out->pstat = (int8_t *)calloc(NP > 0 ? NP : 1, 1);
    if (!out->pstat) { set_err(out, "out of host memory"); return 1; }
    if (NP == 0) return 0;

    int rc = 0;
    int64_t launches = 0;
    Workspace &W = workspace(in->device);
    std::unique_lock<std::mutex> lock(W.mu);
    RowSink rows;
    int sub = 0;                                // batches done (output slot = sub & 1)
    const auto t_call = std::chrono::steady_clock::now();
    auto host_ms = [&]() {                      // host wall time since the call began (verbose)
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_call).count();
    };
    cudaEvent_t ev[8] = {};
    int64_t koff_total = 0, moff_total = 0;
    Geo *dgeo = nullptr;
    int64_t *dkappa = nullptr, *dmb = nullptr;
    int nsm = 148;
    for (auto &g : geos) { koff_total += (int64_t)g.h * g.h * g.h; moff_total += (int64_t)g.h * g.h; }

    CK(cudaSetDevice(in->device));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, in->device));
    for (auto &e : ev) CK(cudaEventCreate(&e));
    if (!W.copy) {
        CK(cudaStreamCreateWithFlags(&W.copy, cudaStreamNonBlocking));
        for (int k = 0; k < 2; ++k) {
            CK(cudaEventCreateWithFlags(&W.rows_done[k], cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&W.copied[k], cudaEventDisableTiming));
        }
    }
    WS(dgeo, W_GEO, geos.size() * sizeof(Geo));
    WS(dkappa, W_KAPPA, koff_total * 8);
    WS(dmb, W_MB, moff_total * 8);
    CK(cudaMemcpy(dgeo, geos.data(), geos.size() * sizeof(Geo), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dkappa, in->kappa, koff_total * 8, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dmb, in->Mbasis, moff_total * 8, cudaMemcpyHostToDevice));
    {
        // batch size: all directions whose slabs fit in a quarter of free memory
        size_t free_b = 0, total_b = 0;
        CK(cudaMemGetInfo(&free_b, &total_b));
        int64_t batch = in->batch > 0 ? in->batch : NP;
        {
            int64_t acc = 0, nb = 0;
            const int64_t budget = (int64_t)(free_b / 4 / 8);
            for (int64_t ip = 0; ip < NP && nb < batch; ++ip, ++nb) {
                acc += geos[in->pgeo[ip]].slab_len;
                if (acc > budget && nb > 0) break;
            }
            batch = std::max<int64_t>(1, std::min(batch, nb));
        }
        unsigned long long &pts_cap = W.pts_cap;
        const unsigned q_cap = 1u << 20;
        int64_t off = 0;
    next_batches:
        for (; off < NP;) {
            const int nb = (int)std::min<int64_t>(batch, NP - off);
            int64_t *dps; int32_t *dpgeo; int64_t *dslaboff, *dslab; Dir *ddirs; SetupScratch *dscr;
            int32_t *dtodo32, *dtodoall, *dorder; SearchCtl *dctl; WorkItem *ditems; int *dready;
            PointHdr *dhdr; int32_t *dcoords; unsigned long long *ddirnodes, *dretry; int32_t *ddirpass;
            std::vector<int64_t> slab_off(nb);
            std::vector<int32_t> todo32, todoall(nb);
            int64_t slab_total = 0;
            for (int k = 0; k < nb; ++k) {
                slab_off[k] = slab_total;
                slab_total += geos[in->pgeo[off + k]].slab_len;
                todoall[k] = k;
                if (geos[in->pgeo[off + k]].use_f32) todo32.push_back(k);
            }
            // setup order: the directions whose LLL working set is an LllMem<32> (shared
            // memory: h11 <= 32, or <= 31 without the coni row) then the rest, each
            // largest h11 first
            std::vector<int32_t> order(nb);
            for (int k = 0; k < nb; ++k) order[k] = k;
            auto small = [&](int32_t k) { const Geo &g = geos[in->pgeo[off + k]]; return g.h + (g.coni ? 0 : 1) <= 32; };
            std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
                const int ha = geos[in->pgeo[off + a]].h, hb = geos[in->pgeo[off + b]].h;
                if (small(a) != small(b)) return small(a);
                return ha > hb;
            });
            int n32 = 0;
            while (n32 < nb && small(order[n32])) ++n32;
            const int n64 = nb - n32;
            const size_t smem32 = sizeof(LllMem<32>);
            int grid32 = 0, grid64[3] = {0, 0, 0};
            if (n32) {
                CK(cudaFuncSetAttribute(k_setup<32, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem32));
                CK(cudaFuncSetAttribute(k_setup<32, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem32));
                CK(cudaFuncSetAttribute(k_setup<32, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem32));
                CK(cudaFuncSetAttribute(k_setup<32, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem32));
                int bpsm = 0;
                CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, k_setup<32, 1>, 32, smem32));
                grid32 = std::min(n32, nsm * std::max(1, bpsm));
            }
            if (n64) {
                // the global-scratch LLL is latency-bound: as many blocks per SM as each phase's
                // registers allow
                const void *f64[3] = {(const void *)k_setup<MH, 0>, (const void *)k_setup<MH, 1>,
                                      (const void *)k_setup<MH, 2>};
                for (int p = 0; p < 3; ++p) {
                    int bpsm = 0;
                    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, f64[p], 128, 0));
                    grid64[p] = std::min((n64 + 3) / 4, nsm * std::max(1, bpsm));
                }
            }
            const int setup_warps = std::max(grid32, 4 * std::max(grid64[0], std::max(grid64[1], grid64[2])));
            WSB(dps, W_PS, (size_t)nb * MH * 8);
            WSB(dpgeo, W_PGEO, (size_t)nb * 4);
            WSB(dslaboff, W_SLABOFF, (size_t)nb * 8);
            WSB(dslab, W_SLAB, (size_t)slab_total * 8);
            WSB(ddirs, W_DIRS, (size_t)nb * sizeof(Dir));
            WSB(dscr, W_SCRATCH, (size_t)setup_warps * sizeof(SetupScratch));
            WSB(dtodo32, W_TODO32, (size_t)std::max<size_t>(todo32.size(), 1) * 4);
            WSB(dtodoall, W_TODOALL, (size_t)nb * 4);
            WSB(dorder, W_ORDER, (size_t)nb * 4);
            WSB(dctl, W_CTL, 2 * sizeof(SearchCtl) + 64);
            WSB(ditems, W_ITEMS, (size_t)q_cap * sizeof(WorkItem));
            WSB(dready, W_READY, (size_t)q_cap * 4);
            WSB(ddirnodes, W_DIRNODES, (size_t)nb * 8);
            WSB(ddirpass, W_DIRPASS, (size_t)nb * 4);
            WSB(dretry, W_RETRY, 64);
            int32_t *drows;
            WSB(drows, W_ROWS, (size_t)nb * 4);
            CK(cudaMemcpy(dps, &in->ps[off * MH], (size_t)nb * MH * 8, cudaMemcpyHostToDevice));
            CK(cudaMemcpy(dpgeo, &in->pgeo[off], (size_t)nb * 4, cudaMemcpyHostToDevice));
            CK(cudaMemcpy(dslaboff, slab_off.data(), (size_t)nb * 8, cudaMemcpyHostToDevice));
            if (!todo32.empty())
                CK(cudaMemcpy(dtodo32, todo32.data(), todo32.size() * 4, cudaMemcpyHostToDevice));
            CK(cudaMemcpy(dtodoall, todoall.data(), (size_t)nb * 4, cudaMemcpyHostToDevice));
            CK(cudaMemcpy(dorder, order.data(), (size_t)nb * 4, cudaMemcpyHostToDevice));

        restart_search:
            WSB(dhdr, W_HDR, pts_cap * sizeof(PointHdr));
            WSB(dcoords, W_COORDS, pts_cap * MD * 4);
            CK(cudaMemset(dctl, 0, 2 * sizeof(SearchCtl) + 64));
            CK(cudaMemset(ddirnodes, 0, (size_t)nb * 8));
            CK(cudaMemset(dretry, 0, 64));
            k_fill_i32<<<(nb + 255) / 256, 256>>>(ddirpass, 1, nb); ++launches;
            CK(cudaGetLastError());
            // ---- setup ----
            CK(cudaEventRecord(ev[0]));
            {
                // work counters: [0..2] phases 0-2 (h11 <= 32), [3..5] (h11 > 32), [6], [7]
                // phase 3; [8], [9] the lengths of the two GCD-row queues phase 2 fills
                unsigned *counters = (unsigned *)((char *)dctl + 2 * sizeof(SearchCtl));
                // phases in order, each over all directions (one work counter per launch)
                SetupArgs SA32{dgeo, dkappa, dmb, dps, dpgeo, dslaboff, dslab, ddirs, dscr, n32,
                               counters, dorder, 1, gcd_min_tree, drows, counters + 8, nullptr};
                SetupArgs SA64{dgeo, dkappa, dmb, dps, dpgeo, dslaboff, dslab, ddirs, dscr, n64,
                               counters + 3, dorder + n32, 0, gcd_min_tree, drows + n32, counters + 9, nullptr};
                if (n32) { k_setup<32, 0><<<grid32, 32, smem32>>>(SA32); ++launches; }
                if (n64) { k_setup<MH, 0><<<grid64[0], 128>>>(SA64); ++launches; }
                SA32.next = counters + 1; SA64.next = counters + 4;
                if (n32) { k_setup<32, 1><<<grid32, 32, smem32>>>(SA32); ++launches; }
                if (n64) { k_setup<MH, 1><<<grid64[1], 128>>>(SA64); ++launches; }
                SA32.next = counters + 2; SA64.next = counters + 5;
                if (n32) { k_setup<32, 2><<<grid32, 32, smem32>>>(SA32); ++launches; }
                if (n64) { k_setup<MH, 2><<<grid64[2], 128>>>(SA64); ++launches; }
                // phase 3: the GCD rows of the queued (large-tree) directions, all at once
                SA32.next = counters + 6; SA32.todo = drows; SA32.n_dev = counters + 8;
                SA64.next = counters + 7; SA64.todo = drows + n32; SA64.n_dev = counters + 9;
                if (n32) { k_setup<32, 3><<<grid32, 32, smem32>>>(SA32); ++launches; }
                if (n64) { k_setup<MH, 3><<<grid64[2], 128>>>(SA64); ++launches; }
                CK(cudaGetLastError());
            }
            CK(cudaEventRecord(ev[1]));
            // ---- search ----
            {
                SearchArgs A{};
                A.geo = dgeo; A.dirs = ddirs; A.slab = dslab; A.pass = 1; A.items = ditems;
                A.ready = dready; A.q_cap = q_cap; A.hdr = dhdr; A.coords = dcoords; A.pts_cap = pts_cap;
                A.dir_nodes = ddirnodes; A.eps = 1e-4; A.wait_ns = wait_ns;
                A.npts = &dctl->npts;
                A.deadline_ns = deadline_ns;
                // per-warp staging area in shared memory, sized for the batch's largest h11
                int hmax = 3;
                for (int k = 0; k < nb; ++k) hmax = std::max(hmax, geos[in->pgeo[off + k]].h);
                const unsigned st32 = stage_bytes<float>(hmax - 1, hmax), st64 = stage_bytes<double>(hmax - 1, hmax);
                const int smem_max = 227 * 1024;
                auto warps_for = [&](unsigned st) {
                    const int w = opt.warps_per_block > 0 ? std::min(opt.warps_per_block, SEARCH_WARPS) : SEARCH_WARPS;
                    return std::max(1, std::min(w, smem_max / (int)st));
                };
                const int wpb32 = warps_for(st32), wpb64 = warps_for(st64);
                // one level per lane (NS = 1) when every h11 of the batch is <= 32, else two
                const bool one = hmax <= 32;
                void (*ks32)(SearchArgs) = one ? k_search<float, 1> : k_search<float, 2>;
                void (*ks64)(SearchArgs) = one ? k_search<double, 1> : k_search<double, 2>;
                void (*kplain)(SearchArgs, int) = one ? k_search_plain<double, 1> : k_search_plain<double, 2>;
                void (*kchk32)(SearchArgs, int) = one ? k_search_plain<float, 1, true> : k_search_plain<float, 2, true>;
                CK(cudaFuncSetAttribute((const void *)ks32, cudaFuncAttributeMaxDynamicSharedMemorySize, wpb32 * st32));
                CK(cudaFuncSetAttribute((const void *)ks64, cudaFuncAttributeMaxDynamicSharedMemorySize, wpb64 * st64));
                if (opt.form == PFG_FORM_PLAIN) {
                    // one launch, one warp per direction, FP64 pruning, no work sharing
                    CK(cudaFuncSetAttribute((const void *)kplain, cudaFuncAttributeMaxDynamicSharedMemorySize, st64));
                    k_flip<<<(nb + 255) / 256, 256>>>(ddirs, dgeo, nb, 0, ddirpass, dretry); ++launches;
                    A.donate = 0; A.n_warps = 1; A.ctl = dctl + 1; A.pass = 2; A.stage_bytes = st64;
                    A.todo = dtodoall; A.n_todo = nb;
                    kplain<<<nb, 32, st64>>>(A, -1); ++launches;
                    CK(cudaGetLastError());
                } else {
                    auto grid_for = [&](const void *fn, int wpb, unsigned st, int &grid) -> cudaError_t {
                        int bps = opt.blocks_per_sm;
                        if (bps <= 0) {
                            cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, fn, wpb * 32,
                                                                                          (size_t)wpb * st);
                            if (e != cudaSuccess) return e;
                            bps = std::max(1, bps);
                        }
                        grid = nsm * bps;
                        return cudaSuccess;
                    };
                    A.donate = 1;
                    // FP32 pass over the FP32 geometries' directions
                    if (!todo32.empty() && opt.check_fp32) {
                        // the bound-check form: one warp per direction with the FP64 shadow
                        CK(cudaFuncSetAttribute((const void *)kchk32, cudaFuncAttributeMaxDynamicSharedMemorySize, st32));
                        SearchArgs C = A;
                        C.donate = 0; C.n_warps = 1; C.stage_bytes = st32; C.ctl = dctl;
                        C.todo = dtodo32; C.n_todo = (int)todo32.size(); C.pass = 1;
                        kchk32<<<(int)todo32.size(), 32, st32>>>(C, -1); ++launches;
                        CK(cudaGetLastError());
                    } else if (!todo32.empty()) {
                        int grid = 0;
                        CK(grid_for((const void *)ks32, wpb32, st32, grid));
                        A.n_warps = grid * wpb32; A.stage_bytes = st32;
                        A.ctl = dctl; A.todo = dtodo32; A.n_todo = (int)todo32.size(); A.pass = 1;
                        CK(cudaMemset(dready, 0, (size_t)q_cap * 4));
                        ks32<<<grid, wpb32 * 32, (size_t)wpb32 * st32>>>(A); ++launches;
                        CK(cudaGetLastError());
                    }
                    k_flip<<<(nb + 255) / 256, 256>>>(ddirs, dgeo, nb, 1, ddirpass, dretry); ++launches;
                    // FP64 pass over everything still pending
                    int grid = 0;
                    CK(grid_for((const void *)ks64, wpb64, st64, grid));
                    A.n_warps = grid * wpb64; A.stage_bytes = st64;
                    A.ctl = dctl + 1; A.todo = dtodoall; A.n_todo = nb; A.pass = 2;
                    CK(cudaMemset(dready, 0, (size_t)q_cap * 4));
                    ks64<<<grid, wpb64 * 32, (size_t)wpb64 * st64>>>(A); ++launches;
                    CK(cudaGetLastError());
                }
            }
            CK(cudaEventRecord(ev[2]));
            SearchCtl hctl[2];
            if (in->verbose) fprintf(stderr, "pfg: [%.1f ms] batch @%lld: launched through the search\n", host_ms(), (long long)off);
            CK(cudaMemcpy(hctl, dctl, 2 * sizeof(SearchCtl), cudaMemcpyDeviceToHost));
            if (in->verbose) fprintf(stderr, "pfg: [%.1f ms] search done\n", host_ms());
            if (hctl[0].err || hctl[1].err) {
                set_err(out, "search: a bounded device wait ran out (status %d)", hctl[0].err ? hctl[0].err : hctl[1].err);
                rc = 1;
                goto fail;
            }
            const unsigned long long npts = hctl[0].npts;
            if (npts > pts_cap) {
                // the device time of the attempt counts; then again with room for every point
                float ms_a[2];
                CK(cudaEventElapsedTime(&ms_a[0], ev[0], ev[1]));
                CK(cudaEventElapsedTime(&ms_a[1], ev[1], ev[2]));
                out->seconds_gpu += (ms_a[0] + ms_a[1]) / 1e3;
                if (stats) { stats->ms_setup += ms_a[0]; stats->ms_search += ms_a[1]; }
                pts_cap = npts + npts / 4 + 1024;
                if (in->verbose) fprintf(stderr, "pfg: point buffer -> %llu\n", pts_cap);
                goto restart_search;
            }
            // ---- output ----
            unsigned *dcount, *dfill, *didx, *dperm, *dperm2, *dsidx;
            unsigned long long *dseg, *dcseg, *dsum; int64_t *dkeys;
            const unsigned long long np1 = std::max<unsigned long long>(npts, 1);
            WSB(dcount, W_COUNT, (size_t)nb * 4);
            WSB(dfill, W_FILL, (size_t)nb * 4);
            WSB(dseg, W_SEG, (size_t)(nb + 1) * 8);
            WSB(dcseg, W_CSEG, (size_t)(nb + 1) * 8);
            WSB(dsum, W_SUM, 64);
            WSB(didx, W_IDX, np1 * 4);
            WSB(dperm, W_PERM, np1 * 4);
            WSB(dperm2, W_PERM2, np1 * 4);
            WSB(dsidx, W_SIDX, np1 * 4);
            int ks = 3;
            for (int k = 0; k < nb; ++k) ks = std::max(ks, geos[in->pgeo[off + k]].h);
            WSB(dkeys, W_KEYS, np1 * ks * 8);
            CK(cudaMemset(dcount, 0, (size_t)nb * 4));
            CK(cudaMemset(dfill, 0, (size_t)nb * 4));
            CK(cudaEventRecord(ev[3]));
            OutArgs O{ddirs, dslab, dhdr, dcoords, ddirpass, npts, nb, dcount, dfill, dseg, didx, dkeys, ks,
                      dcseg, dsum, dperm};
            if (npts) { k_count<<<nsm * 4, 256>>>(O); ++launches; }
            k_scan<<<1, 1024>>>(O); ++launches;
            if (npts) { k_scatter<<<nsm * 4, 256>>>(O); ++launches; }
            CK(cudaGetLastError());
            unsigned long long summary[3] = {0, 0, 0};
            CK(cudaMemcpy(summary, dsum, sizeof summary, cudaMemcpyDeviceToHost));
            const unsigned long long n_out = summary[0], n_chunks = summary[1], longest = summary[2];
            // output slot of this batch: free once the copy of the batch before last is done
            const int slot = sub & 1;
            if (W.copy_pending[slot]) {
                CK(cudaEventSynchronize(W.copied[slot]));
                W.copy_pending[slot] = false;
            }
            int64_t *oM, *oK, *oq, *op;
            WSB(oM, slot ? W_OM2 : W_OM, std::max<unsigned long long>(n_out, 1) * rw * 8);
            WSB(oK, slot ? W_OK2 : W_OK, std::max<unsigned long long>(n_out, 1) * rw * 8);
            WSB(oq, slot ? W_OQ2 : W_OQ, std::max<unsigned long long>(n_out, 1) * 8);
            WSB(op, slot ? W_OP2 : W_OP, std::max<unsigned long long>(n_out, 1) * 8);
            if (n_out) {
                const int smem_sort = SORT_CAP * KEYN * 8 + SORT_CAP * 4;
                CK(cudaFuncSetAttribute(k_segsort, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_sort));
                k_keys<<<nsm * 8, 256>>>(O, n_out); ++launches;
                k_segsort<<<(int)std::min<unsigned long long>(n_chunks, (unsigned long long)nsm * 3), 256,
                            smem_sort>>>(O); ++launches;
                unsigned *pin = dperm, *pout = dperm2;
                for (unsigned long long L = SORT_CAP; L < longest; L *= 2) {
                    k_merge<<<nsm * 8, 256>>>(O, n_out, (unsigned)L, pin, pout); ++launches;
                    std::swap(pin, pout);
                }
                k_order<<<nsm * 4, 256>>>(O, n_out, pin, dsidx, pout); ++launches;
                RowArgs R{ddirs, dslab, dhdr, dcoords, dsidx, pout, dkeys, ks, n_out, off, oM, oK, oq, op, rw};
                k_rows<<<nsm * 8, 256>>>(R); ++launches;
                CK(cudaGetLastError());
            }
            if (pfv && n_out) {
                // ---- points -> PFVs (on the device) ----
                int hmax2 = 3;
                for (int k = 0; k < nb; ++k) hmax2 = std::max(hmax2, geos[in->pgeo[off + k]].h);
                const int prc = pfv_stage(W, nsm, ddirs, dgeo, dkappa, oM, oK, oq, op, n_out, off, hmax2, pfv,
                                          launches, out->err);
                if (prc == 2 && nb > 1) { out->err[0] = 0; goto out_of_memory; }
                if (prc) { rc = 1; goto fail; }
            }
            CK(cudaEventRecord(ev[4]));
            if (n_out && !pfv) {
                if (rows.n + n_out > rows.cap) {
                    // room for the whole call, from this batch's (or the last call's) rows per direction
                    const double per = std::max((double)n_out / nb, W.rows_per_dir);
                    const size_t cap = std::max<size_t>(rows.n + n_out, (size_t)(per * (double)NP * 1.1) + 4096);
                    RowSink bigger;
                    if (!bigger.alloc(cap, rw)) { bigger.release(); set_err(out, "out of pinned host memory"); rc = 1; goto fail; }
                    if (rows.n) {
                        CK(cudaStreamSynchronize(W.copy));
                        memcpy(bigger.M, rows.M, rows.n * rw * 8);
                        memcpy(bigger.Kn, rows.Kn, rows.n * rw * 8);
                        memcpy(bigger.q, rows.q, rows.n * 8);
                        memcpy(bigger.pidx, rows.pidx, rows.n * 8);
                        bigger.n = rows.n;
                    }
                    rows.release();
                    rows = bigger;
                }
                CK(cudaEventRecord(W.rows_done[slot], 0));
                CK(cudaStreamWaitEvent(W.copy, W.rows_done[slot], 0));
                CK(cudaMemcpyAsync(rows.M + rows.n * rw, oM, n_out * rw * 8, cudaMemcpyDeviceToHost, W.copy));
                CK(cudaMemcpyAsync(rows.Kn + rows.n * rw, oK, n_out * rw * 8, cudaMemcpyDeviceToHost, W.copy));
                CK(cudaMemcpyAsync(rows.q + rows.n, oq, n_out * 8, cudaMemcpyDeviceToHost, W.copy));
                CK(cudaMemcpyAsync(rows.pidx + rows.n, op, n_out * 8, cudaMemcpyDeviceToHost, W.copy));
                CK(cudaEventRecord(W.copied[slot], W.copy));
                W.copy_pending[slot] = true;
                rows.n += n_out;
                if (in->verbose) fprintf(stderr, "pfg: [%.1f ms] rows %llu queued for copy (block of %zu rows)\n",
                                         host_ms(), n_out, rows.cap);
            }
            // statuses
            {
                std::vector<Dir> hd(nb);
                CK(cudaMemcpy(hd.data(), ddirs, (size_t)nb * sizeof(Dir), cudaMemcpyDeviceToHost));
                std::map<std::pair<int, int>, int> fails;
                for (int k = 0; k < nb; ++k) {
                    const int st = hd[k].status;
                    out->pstat[off + k] = (st == ST_OK || st == ST_PENDING || st == ST_EMPTY) ? 0 : (int8_t)st;
                    if (out->pstat[off + k]) fails[{st, hd[k].pad}]++;
                }
                if (in->verbose)
                    for (auto &f : fails)
                        fprintf(stderr, "pfg: %d directions with status %d (setup step %d)\n", f.second,
                                f.first.first, f.first.second);
                if (dir_nodes_out) {
                    std::vector<unsigned long long> dn(nb);
                    CK(cudaMemcpy(dn.data(), ddirnodes, (size_t)nb * 8, cudaMemcpyDeviceToHost));
                    for (int k = 0; k < nb; ++k) dir_nodes_out[off + k] = (int64_t)dn[k];
                }
            }
            {
                float ms[4];
                CK(cudaEventElapsedTime(&ms[0], ev[0], ev[1]));
                CK(cudaEventElapsedTime(&ms[1], ev[1], ev[2]));
                CK(cudaEventElapsedTime(&ms[2], ev[3], ev[4]));
                out->seconds_gpu += (ms[0] + ms[1] + ms[2]) / 1e3;
                unsigned long long retries = 0;
                CK(cudaMemcpy(&retries, dretry, 8, cudaMemcpyDeviceToHost));
                if (stats) {
                    stats->ms_setup += ms[0]; stats->ms_search += ms[1]; stats->ms_output += ms[2];
                    stats->nodes += (int64_t)(hctl[0].nodes + hctl[1].nodes);
                    stats->candidates += (int64_t)(hctl[0].cands + hctl[1].cands);
                    stats->leaves += (int64_t)(hctl[0].leaves + hctl[1].leaves);
                    stats->points += (int64_t)npts;
                    stats->donated += (int64_t)(hctl[0].donated + hctl[1].donated);
                    stats->fp64_retries += (int64_t)retries;
                    if (opt.check_fp32) {
                        stats->fp32_rem_err = std::max(stats->fp32_rem_err, dbits(hctl[0].chk_rem));
                        stats->fp32_margin_frac = std::max(stats->fp32_margin_frac, dbits(hctl[0].chk_frac));
                        stats->fp32_end_err = std::max(stats->fp32_end_err, dbits(hctl[0].chk_end));
                        stats->fp32_narrower += (int64_t)hctl[0].chk_narrower;
                    }
                    stats->launches = launches;
                }
                if (in->verbose)
                    fprintf(stderr, "pfg: batch @%lld: %d p | setup %.2f ms, search %.2f ms, output %.2f ms | "
                                    "nodes %llu, points %llu -> %llu rows, donated %llu, fp64 retries %llu\n",
                            (long long)off, nb, ms[0], ms[1], ms[2], hctl[0].nodes + hctl[1].nodes, npts, n_out,
                            hctl[0].donated + hctl[1].donated, retries);
            }
            off += nb;
            ++sub;
        }
        goto batches_done;
    out_of_memory:
        // out of device memory (another process, a partly filled GPU): free the
        // per-batch buffers (copies in flight read the output slots: let them
        // finish first), halve the batch and do the current batch again
        cudaGetLastError();
        if (W.copy) cudaStreamSynchronize(W.copy);
        W.copy_pending[0] = W.copy_pending[1] = false;
        ws_release(W, W_PS);                    // (the geometries' buffers stay)
        batch = std::max<int64_t>(1, batch / 2);
        pts_cap = std::max<unsigned long long>(1ull << 16, pts_cap / 2);
        if (stats) stats->batch_retries++;
        if (in->verbose) fprintf(stderr, "pfg: out of device memory at p %lld; batch -> %lld\n",
                                 (long long)off, (long long)batch);
        goto next_batches;
    batches_done:;
    }
    if (in->verbose) fprintf(stderr, "pfg: [%.1f ms] all batches done\n", host_ms());
    CK(cudaStreamSynchronize(W.copy));
    if (in->verbose) fprintf(stderr, "pfg: [%.1f ms] copies done\n", host_ms());
    W.copy_pending[0] = W.copy_pending[1] = false;
    out->n = (int64_t)rows.n;
    out->M = rows.M; out->Kn = rows.Kn; out->q = rows.q; out->pidx = rows.pidx;
    if (!pfv) W.rows_per_dir = NP ? (double)rows.n / (double)NP : 0.0;
    rows = RowSink();
fail:
    if (W.copy) {
        cudaStreamSynchronize(W.copy);          // no copy may still write into a block released below
        W.copy_pending[0] = W.copy_pending[1] = false;
    }
    rows.release();
    for (auto &e : ev) if (e) cudaEventDestroy(e);
    if (rc) {
        cudaGetLastError();
        pfg_output_free(out);
        if (pfv) pfv->release();
    }
    return rc;
}

extern "C" int pfg_coni_batch_ex(const pfg_input *in, const pfg_options *opt, pfg_output *out,
                                 pfg_stats *stats, int64_t *dir_nodes)
{
    return coni_run(in, opt, out, stats, dir_nodes, nullptr);
}

extern "C" int pfg_zpm_batch(const pfg_input *in, const pfg_options *opt, pfg_output *out, pfg_stats *stats,
                             int64_t *dir_nodes)
{
    return coni_run(in, opt, out, stats, dir_nodes, nullptr, 0);
}

extern "C" int pfg_coni_pfvs(const pfg_input *in, const pfg_options *opt, pfg_pfv_output *out, pfg_stats *stats)
{
    memset(out, 0, sizeof *out);
    for (int gi = 0; gi < in->n_geo; ++gi)
        if (in->linmin[gi] <= 0) {
            snprintf(out->err, sizeof out->err, "coniZpM requires M0min > 0 (geometry %d)", gi);
            return 1;
        }
    pfg_output pts;
    PfvSink sink;
    const int rc = coni_run(in, opt, &pts, stats, nullptr, &sink);
    out->pstat = pts.pstat;
    pts.pstat = nullptr;
    out->seconds_gpu = pts.seconds_gpu;
    out->n_points = sink.n_points;
    if (rc) {
        memcpy(out->err, pts.err, sizeof out->err);
        sink.release();
        pfg_output_free(&pts);
        return rc;
    }
    pfg_output_free(&pts);
    size_t n = 0;
    for (auto &c : sink.chunks) n += c.n;
    out->n = (int64_t)n;
    if (sink.chunks.size() == 1) {
        out->K = sink.chunks[0].K; out->M = sink.chunks[0].M; out->pidx = sink.chunks[0].pidx;
        sink.chunks.clear();
        return 0;
    }
    out->K = (int64_t *)pinned_get(n * MH * 8);
    out->M = (int64_t *)pinned_get(n * MH * 8);
    out->pidx = (int64_t *)pinned_get(n * 8);
    if (!out->K || !out->M || !out->pidx) {
        snprintf(out->err, sizeof out->err, "out of pinned host memory");
        sink.release();
        pfg_pfv_output_free(out);
        return 1;
    }
    size_t base = 0;
    for (auto &c : sink.chunks) {
        memcpy(out->K + base * MH, c.K, c.n * MH * 8);
        memcpy(out->M + base * MH, c.M, c.n * MH * 8);
        memcpy(out->pidx + base, c.pidx, c.n * 8);
        base += c.n;
    }
    sink.release();
    return 0;
}

extern "C" void pfg_pfv_output_free(pfg_pfv_output *out)
{
    for (int64_t *p : {out->K, out->M, out->pidx})
        if (!pinned_put(p)) free(p);
    free(out->pstat);
    out->K = out->M = out->pidx = nullptr;
    out->pstat = nullptr;
    out->n = 0;
}

// The coni dilation bound mu0 of n_p directions of one geometry (pfg_mu0.cuh).
extern "C" int pfg_coni_mu0_batch(int h, const int64_t *kappa, int64_t n_p, const int64_t *p_r, int device,
                                  int32_t *status, int64_t *mu_num, int64_t *mu_den, int64_t *K, char *err)
{
    char msg[256] = "";
    int rc = 0;
    if (h < 3 || h > MU0_MAXH || n_p < 0 || n_p > INT32_MAX || (n_p && (!kappa || !p_r || !status || !mu_num ||
                                                                        !mu_den || !K))) {
        snprintf(msg, sizeof msg, "pfg_coni_mu0_batch: bad arguments (h11 = %d outside 3..%d, or null arrays)",
                 h, MU0_MAXH);
        if (err) memcpy(err, msg, sizeof msg);
        return 1;
    }
    if (n_p == 0) return 0;
    const int m = h - 1;
    Workspace &W = workspace(device);
    std::lock_guard<std::mutex> lock(W.mu);
    int64_t *dk, *dp, *dn, *dd, *dK; int32_t *ds; Mu0Scratch *dscr; unsigned *dctr;
    int bps = 0, nsm = 148, grid = 0;
    cudaError_t e;
#define MCK(x) do { e = (x); if (e != cudaSuccess) { snprintf(msg, sizeof msg, "%s (%s:%d)", cudaGetErrorString(e), \
    __FILE__, __LINE__); rc = 1; goto mu_fail; } } while (0)
    MCK(cudaSetDevice(device));
    MCK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
    MCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_mu0, 128, 0));
    grid = (int)std::min<int64_t>((n_p + 3) / 4, (int64_t)nsm * std::max(1, bps));
    MCK(ws_get(W, W_MU_K, (size_t)h * h * h * 8, (void **)&dk));
    MCK(ws_get(W, W_MU_P, (size_t)n_p * m * 8, (void **)&dp));
    MCK(ws_get(W, W_MU_ST, (size_t)n_p * 4, (void **)&ds));
    MCK(ws_get(W, W_MU_NUM, (size_t)n_p * 8, (void **)&dn));
    MCK(ws_get(W, W_MU_DEN, (size_t)n_p * 8, (void **)&dd));
    MCK(ws_get(W, W_MU_KO, (size_t)n_p * m * 8, (void **)&dK));
    MCK(ws_get(W, W_MU_SCR, (size_t)grid * 4 * sizeof(Mu0Scratch), (void **)&dscr));
    MCK(ws_get(W, W_MU_CTR, 64, (void **)&dctr));
    MCK(cudaMemcpy(dk, kappa, (size_t)h * h * h * 8, cudaMemcpyHostToDevice));
    MCK(cudaMemcpy(dp, p_r, (size_t)n_p * m * 8, cudaMemcpyHostToDevice));
    MCK(cudaMemset(dctr, 0, 64));
    {
        Mu0Args A{h, dk, dp, (int)n_p, dctr, dscr, ds, dn, dd, dK, 20000000ll};
        k_mu0<<<grid, 128>>>(A);
        MCK(cudaGetLastError());
    }
    MCK(cudaMemcpy(status, ds, (size_t)n_p * 4, cudaMemcpyDeviceToHost));
    MCK(cudaMemcpy(mu_num, dn, (size_t)n_p * 8, cudaMemcpyDeviceToHost));
    MCK(cudaMemcpy(mu_den, dd, (size_t)n_p * 8, cudaMemcpyDeviceToHost));
    MCK(cudaMemcpy(K, dK, (size_t)n_p * m * 8, cudaMemcpyDeviceToHost));
#undef MCK
mu_fail:
    if (rc) {
        cudaGetLastError();
        if (err) memcpy(err, msg, sizeof msg);
    }
    return rc;
}

// ---------------------------------------------------------------------------
// coniZpK above D0 (pfg_zpk.cuh)
// ---------------------------------------------------------------------------
namespace {

constexpr long long ZPK_STEP_BUDGET = 100000000ll;  // search nodes + (j, M0) steps per lane and direction

struct EventPair {
    cudaEvent_t a = nullptr, b = nullptr;
    ~EventPair() { if (a) cudaEventDestroy(a); if (b) cudaEventDestroy(b); }
};

// one call: one geometry (h, Q, M0min, kappa, Mbasis) and n_p directions
// (rows of ps_stride entries)
struct ZpkCall {
    int h;
    int64_t Q, M0min;
    const int64_t *kappa, *Mbasis;
    int64_t n_p;
    const int64_t *ps;
    int ps_stride;
    int64_t D0, max_out;
    int device;
};

// k_zpk over the call's directions; the points of the directions with status 0
// into host rows (MH wide), the statuses into `status`.  kappa stays on the
// device (*dkappa).  Returns 0 or 1 with err set.
int zpk_points(Workspace &W, const ZpkCall &C, int32_t *status, std::vector<int64_t> &M, std::vector<int64_t> &Kn,
               std::vector<int64_t> &q, std::vector<int64_t> &pidx, double &secs, int &nsm, int64_t **dkappa,
               char *err)
{
    cudaError_t e;
#define ZCK(x) do { e = (x); if (e != cudaSuccess) { snprintf(err, 256, "%s (%s:%d)", cudaGetErrorString(e), \
    __FILE__, __LINE__); return 1; } } while (0)
    const int64_t ksz = (int64_t)C.h * C.h * C.h, msz = (int64_t)C.h * C.h;
    int bps = 0;
    ZCK(cudaSetDevice(C.device));
    ZCK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, C.device));
    ZCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_zpk, 128, 0));
    const int grid = (int)std::min<int64_t>((C.n_p + 3) / 4, (int64_t)nsm * std::max(1, std::min(bps, 4)));
    int64_t *dk, *dmb, *dps, *dM, *dK, *dq, *dp; int32_t *dst;
    ZpkScratch *dscr; unsigned *dctr;
    ZCK(ws_get(W, W_MU_K, (size_t)ksz * 8, (void **)&dk));
    ZCK(ws_get(W, W_ZK_MB, (size_t)msz * 8, (void **)&dmb));
    ZCK(ws_get(W, W_ZK_PS, (size_t)C.n_p * C.ps_stride * 8, (void **)&dps));
    ZCK(ws_get(W, W_ZK_ST, (size_t)C.n_p * 4, (void **)&dst));
    ZCK(ws_get(W, W_ZK_SCR, (size_t)grid * 4 * sizeof(ZpkScratch), (void **)&dscr));
    ZCK(ws_get(W, W_ZK_CTR, 64, (void **)&dctr));
    ZCK(cudaMemcpy(dk, C.kappa, (size_t)ksz * 8, cudaMemcpyHostToDevice));
    ZCK(cudaMemcpy(dmb, C.Mbasis, (size_t)msz * 8, cudaMemcpyHostToDevice));
    ZCK(cudaMemcpy(dps, C.ps, (size_t)C.n_p * C.ps_stride * 8, cudaMemcpyHostToDevice));
    *dkappa = dk;
    EventPair ev;
    ZCK(cudaEventCreate(&ev.a));
    ZCK(cudaEventCreate(&ev.b));
    unsigned long long cap = std::max<unsigned long long>(1ull << 14, (unsigned long long)C.n_p * 8), count = 0;
    for (int pass = 0; pass < 2; ++pass) {
        ZCK(ws_get(W, W_ZK_M, cap * MH * 8, (void **)&dM));
        ZCK(ws_get(W, W_ZK_K, cap * MH * 8, (void **)&dK));
        ZCK(ws_get(W, W_ZK_Q, cap * 8, (void **)&dq));
        ZCK(ws_get(W, W_ZK_P, cap * 8, (void **)&dp));
        ZCK(cudaMemset(dctr, 0, 64));
        ZpkArgs A{C.h, dk, dmb, dps, C.ps_stride, (int)C.n_p, C.Q, C.M0min, C.D0, C.max_out,
                  dctr, dscr, dst, (unsigned long long *)(dctr + 2), cap, dM, dK, dq, dp, ZPK_STEP_BUDGET};
        ZCK(cudaEventRecord(ev.a));
        k_zpk<<<grid, 128>>>(A);
        ZCK(cudaGetLastError());
        ZCK(cudaEventRecord(ev.b));
        ZCK(cudaMemcpy(&count, dctr + 2, 8, cudaMemcpyDeviceToHost));
        if (count <= cap) break;
        cap = count;                            // (the same points again, with room for all of them)
    }
    float ms = 0.f;
    ZCK(cudaEventElapsedTime(&ms, ev.a, ev.b));
    secs = ms * 1e-3;
    ZCK(cudaMemcpy(status, dst, (size_t)C.n_p * 4, cudaMemcpyDeviceToHost));
    std::vector<int64_t> aM(count * MH), aK(count * MH), aq(count), ap(count);
    if (count) {
        ZCK(cudaMemcpy(aM.data(), dM, count * MH * 8, cudaMemcpyDeviceToHost));
        ZCK(cudaMemcpy(aK.data(), dK, count * MH * 8, cudaMemcpyDeviceToHost));
        ZCK(cudaMemcpy(aq.data(), dq, count * 8, cudaMemcpyDeviceToHost));
        ZCK(cudaMemcpy(ap.data(), dp, count * 8, cudaMemcpyDeviceToHost));
    }
    M.clear(); Kn.clear(); q.clear(); pidx.clear();
    for (unsigned long long t = 0; t < count; ++t) {
        if (status[ap[t]] != 0) continue;       // (a direction's points count only when it finished)
        M.insert(M.end(), aM.begin() + t * MH, aM.begin() + (t + 1) * MH);
        Kn.insert(Kn.end(), aK.begin() + t * MH, aK.begin() + (t + 1) * MH);
        q.push_back(aq[t]);
        pidx.push_back(ap[t]);
    }
    return 0;
#undef ZCK
}

// the call's points -> PFVs on the device (the coniZpM post-processing stage)
int zpk_pfvs(Workspace &W, const ZpkCall &C, int32_t *status, pfg_pfv_output *out)
{
    std::vector<int64_t> M, Kn, q, pidx;
    int nsm = 148;
    int64_t *dk = nullptr;
    PfvSink sink;
    if (zpk_points(W, C, status, M, Kn, q, pidx, out->seconds_gpu, nsm, &dk, out->err)) {
        cudaGetLastError();
        return 1;
    }
    const size_t n = q.size();
    if (n) {
        cudaError_t e;
        int64_t *dM, *dK, *dq, *dp, launches = 0;
        Dir *ddirs; Geo *dgeo;
        std::vector<Dir> dirs(C.n_p);
        for (int64_t i = 0; i < C.n_p; ++i) {
            dirs[i] = Dir{};
            dirs[i].geo = 0; dirs[i].h = C.h; dirs[i].d = C.h - 1;
        }
        Geo geo{};
        geo.h = C.h; geo.d = C.h - 1; geo.coni = 1; geo.Q = C.Q; geo.linmin = C.M0min; geo.koff = 0;
#define ZCK2(x) do { e = (x); if (e != cudaSuccess) { snprintf(out->err, sizeof out->err, "%s (%s:%d)", \
    cudaGetErrorString(e), __FILE__, __LINE__); cudaGetLastError(); sink.release(); return 1; } } while (0)
        ZCK2(ws_get(W, W_OM, n * MH * 8, (void **)&dM));
        ZCK2(ws_get(W, W_OK, n * MH * 8, (void **)&dK));
        ZCK2(ws_get(W, W_OQ, n * 8, (void **)&dq));
        ZCK2(ws_get(W, W_OP, n * 8, (void **)&dp));
        ZCK2(ws_get(W, W_DIRS, (size_t)C.n_p * sizeof(Dir), (void **)&ddirs));
        ZCK2(ws_get(W, W_GEO, sizeof(Geo), (void **)&dgeo));
        ZCK2(cudaMemcpy(dM, M.data(), n * MH * 8, cudaMemcpyHostToDevice));
        ZCK2(cudaMemcpy(dK, Kn.data(), n * MH * 8, cudaMemcpyHostToDevice));
        ZCK2(cudaMemcpy(dq, q.data(), n * 8, cudaMemcpyHostToDevice));
        ZCK2(cudaMemcpy(dp, pidx.data(), n * 8, cudaMemcpyHostToDevice));
        ZCK2(cudaMemcpy(ddirs, dirs.data(), (size_t)C.n_p * sizeof(Dir), cudaMemcpyHostToDevice));
        ZCK2(cudaMemcpy(dgeo, &geo, sizeof(Geo), cudaMemcpyHostToDevice));
#undef ZCK2
        if (pfv_stage(W, nsm, ddirs, dgeo, dk, dM, dK, dq, dp, n, 0, std::max(3, C.h), &sink, launches, out->err)) {
            cudaGetLastError();
            sink.release();
            return 1;
        }
    }
    size_t np_ = 0;
    for (auto &c : sink.chunks) np_ += c.n;
    out->n = (int64_t)np_;
    out->n_points = (int64_t)n;
    if (sink.chunks.size() == 1) {
        out->K = sink.chunks[0].K; out->M = sink.chunks[0].M; out->pidx = sink.chunks[0].pidx;
        sink.chunks.clear();
    }
    return 0;
}

bool zpk_args_ok(int h, const int64_t *kappa, const int64_t *Mbasis, int64_t n_p, const int64_t *ps,
                 const int32_t *status, char *err)
{
    if (h < 3 || h > ZPK_MAXH || n_p < 0 || n_p > INT32_MAX || (n_p && (!kappa || !Mbasis || !ps || !status))) {
        snprintf(err, 256, "coniZpK: bad arguments (h11 = %d outside 3..%d, or null arrays)", h, ZPK_MAXH);
        return false;
    }
    return true;
}

}  // namespace

extern "C" int pfg_coni_zpk_batch(int h, const int64_t *kappa, const int64_t *Mbasis, int64_t n_p, const int64_t *ps,
                                  int64_t Q, int64_t M0min, int64_t D0, int64_t max_out, int device,
                                  pfg_output *out, int32_t *status)
{
    memset(out, 0, sizeof *out);
    if (!zpk_args_ok(h, kappa, Mbasis, n_p, ps, status, out->err)) return 1;
    if (n_p == 0) return 0;
    Workspace &W = workspace(device);
    std::lock_guard<std::mutex> lock(W.mu);
    const ZpkCall C{h, Q, M0min, kappa, Mbasis, n_p, ps, h, D0, max_out, device};
    std::vector<int64_t> M, Kn, q, pidx;
    int nsm = 148;
    int64_t *dk = nullptr;
    if (zpk_points(W, C, status, M, Kn, q, pidx, out->seconds_gpu, nsm, &dk, out->err)) {
        cudaGetLastError();
        return 1;
    }
    const size_t n = q.size();
    out->n = (int64_t)n;
    out->M = (int64_t *)pinned_get(std::max<size_t>(n, 1) * MH * 8);
    out->Kn = (int64_t *)pinned_get(std::max<size_t>(n, 1) * MH * 8);
    out->q = (int64_t *)pinned_get(std::max<size_t>(n, 1) * 8);
    out->pidx = (int64_t *)pinned_get(std::max<size_t>(n, 1) * 8);
    if (!out->M || !out->Kn || !out->q || !out->pidx) {
        snprintf(out->err, sizeof out->err, "out of pinned host memory");
        pfg_output_free(out);
        return 1;
    }
    if (n) {
        memcpy(out->M, M.data(), n * MH * 8);
        memcpy(out->Kn, Kn.data(), n * MH * 8);
        memcpy(out->q, q.data(), n * 8);
        memcpy(out->pidx, pidx.data(), n * 8);
    }
    return 0;
}

extern "C" int pfg_coni_zpk_pfvs(int h, const int64_t *kappa, const int64_t *Mbasis, int64_t n_p, const int64_t *ps,
                                 int64_t Q, int64_t M0min, int64_t D0, int64_t max_out, int device,
                                 pfg_pfv_output *out, int32_t *status)
{
    memset(out, 0, sizeof *out);
    if (!zpk_args_ok(h, kappa, Mbasis, n_p, ps, status, out->err)) return 1;
    if (M0min <= 0) { snprintf(out->err, sizeof out->err, "coniZpK requires M0min > 0"); return 1; }
    if (n_p == 0) return 0;
    Workspace &W = workspace(device);
    std::lock_guard<std::mutex> lock(W.mu);
    const ZpkCall C{h, Q, M0min, kappa, Mbasis, n_p, ps, h, D0, max_out, device};
    return zpk_pfvs(W, C, status, out);
}
