// TEST INFRASTRUCTURE -- never part of the product.
//
// Runs the library's device kernels (pfvs_b200/csrc/*.cuh, compiled for the
// host against warp_emu.h) on CPU threads, in the same sequence as the
// library's host code (pfvs_b200/csrc/pfg_abi.cu): setup, FP32 search,
// flip, FP64 search, expand/count/scan/scatter/segsort/gather.  Exposed as
// emu_coni_batch() with the pfg_input/pfg_output structs, for CPU tests of
// the device logic and for debugging without a GPU.  Not loadable by the
// product (the product loads only libpfvs_gpu*.so).
#define PFG_EMU 1
#include "warp_emu.h"

#include <cstdio>
#include <cstdlib>
#include <vector>

#include "../../include/pfvs_gpu.h"
#include "../../pfvs_b200/csrc/pfg_int.cuh"
#include "../../pfvs_b200/csrc/pfg_types.cuh"
#include "../../pfvs_b200/csrc/pfg_setup.cuh"
#include "../../pfvs_b200/csrc/pfg_search.cuh"
#include "../../pfvs_b200/csrc/pfg_out.cuh"
#include "../../pfvs_b200/csrc/pfg_mu0.cuh"
#include "../../pfvs_b200/csrc/pfg_zpk.cuh"

using namespace pfg;

template <class K> static void launch(unsigned grid, K kernel)
{
    for (unsigned b = 0; b < grid; ++b) emu_run_warp(b, 0, 32, grid, kernel);
}

// GCD-row policy of the emulated setup (pfg_options.gcd_min_tree's meaning after
// the library maps it: 0 builds rows for every direction)
static double g_emu_gcd_min_tree = GCD_MIN_TREE_DEFAULT;
extern "C" void emu_set_gcd_min_tree(double v) { g_emu_gcd_min_tree = v < 0 ? 0.0 : (v == 0 ? GCD_MIN_TREE_DEFAULT : v); }

// the last bound-check run's maxima (remaining-norm error, its fraction of the
// FP32 margin, interval-endpoint error) and narrower-range count
static double g_emu_chk[4];
extern "C" void emu_last_fp32_check(double *out) { memcpy(out, g_emu_chk, sizeof g_emu_chk); }

// 1: the coni pipeline (pfg_coni_batch_ex); 0: non-coni ZpM (pfg_zpm_batch)
static int g_emu_coni = 1;
extern "C" void emu_set_coni(int coni) { g_emu_coni = coni; }

// precision: PFG_PREC_*, or 3 for FP32 pruning in the bound-check form
extern "C" int emu_coni_batch(const pfg_input *in, int precision, int n_warps, pfg_output *out,
                              int64_t *dir_nodes_out, int32_t *dir_debug)
{
    memset(out, 0, sizeof *out);
    const bool check_fp32 = precision == 3;
    if (check_fp32) precision = PFG_PREC_FP32;
    memset(g_emu_chk, 0, sizeof g_emu_chk);
    const int64_t NP = in->n_p;
    std::vector<Geo> geos(in->n_geo);
    int64_t koff = 0, moff = 0;
    for (int gi = 0; gi < in->n_geo; ++gi) {
        Geo &g = geos[gi];
        g.h = in->h[gi]; g.d = g.h - 1;
        g.Q = in->Q[gi]; g.qmax = in->qmax[gi];
        g.coni = g_emu_coni;
        g.linmin = g.coni ? in->linmin[gi] : 0;
        g.use_f32 = g.qmax < (1LL << 22) && precision == PFG_PREC_FP32;
        g.koff = koff; g.moff = moff;
        g.slab_len = slab_layout(g.h, g.d).len;
        koff += (int64_t)g.h * g.h * g.h;
        moff += (int64_t)g.h * g.h;
    }
    out->pstat = (int8_t *)calloc(NP > 0 ? NP : 1, 1);
    const int nb = (int)NP;
    std::vector<int64_t> slab_off(nb);
    std::vector<int32_t> todo32, todoall(nb), pgeo(in->pgeo, in->pgeo + nb);
    int64_t slab_total = 0;
    for (int k = 0; k < nb; ++k) {
        slab_off[k] = slab_total;
        slab_total += geos[pgeo[k]].slab_len;
        todoall[k] = k;
        if (geos[pgeo[k]].use_f32) todo32.push_back(k);
    }
    std::vector<int64_t> slab(slab_total + 1);
    std::vector<Dir> dirs(nb);
    const int setup_warps = 4;
    std::vector<SetupScratch> scratch(setup_warps);
    unsigned next = 0;
    // the device's split: h11 <= 32 through the LllMem<32> kernel, the rest through LllMem<64>
    std::vector<int32_t> o32, o64;
    for (int k = 0; k < nb; ++k) (geos[pgeo[k]].h + (g_emu_coni ? 0 : 1) <= 32 ? o32 : o64).push_back(k);
    unsigned next64 = 0;
    SetupArgs SA{geos.data(), in->kappa, in->Mbasis, in->ps, pgeo.data(), slab_off.data(), slab.data(),
                 dirs.data(), scratch.data(), (int)o32.size(), &next, o32.data(), 0, g_emu_gcd_min_tree};
    SetupArgs SA64 = SA;
    SA64.n = (int)o64.size(); SA64.next = &next64; SA64.todo = o64.data();
    // the library's split form: phase 2 queues the directions that want GCD rows
    std::vector<int32_t> rows32(nb + 1), rows64(nb + 1);
    unsigned nrows32 = 0, nrows64 = 0;
    SA.rows_list = rows32.data(); SA.rows_count = &nrows32;
    SA64.rows_list = rows64.data(); SA64.rows_count = &nrows64;
    fprintf(stderr, "emu: setup\n");
    // the three phase kernels in order, each with a fresh work counter
    if (!o32.empty()) launch(setup_warps, [&] { k_setup<32, 0>(SA); });
    if (!o64.empty()) launch(setup_warps, [&] { k_setup<MH, 0>(SA64); });
    next = 0; next64 = 0;
    if (!o32.empty()) launch(setup_warps, [&] { k_setup<32, 1>(SA); });
    if (!o64.empty()) launch(setup_warps, [&] { k_setup<MH, 1>(SA64); });
    next = 0; next64 = 0;
    if (!o32.empty()) launch(setup_warps, [&] { k_setup<32, 2>(SA); });
    if (!o64.empty()) launch(setup_warps, [&] { k_setup<MH, 2>(SA64); });
    next = 0; next64 = 0;
    SA.todo = rows32.data(); SA.n_dev = &nrows32;
    SA64.todo = rows64.data(); SA64.n_dev = &nrows64;
    if (!o32.empty()) launch(setup_warps, [&] { k_setup<32, 3>(SA); });
    if (!o64.empty()) launch(setup_warps, [&] { k_setup<MH, 3>(SA64); });
    fprintf(stderr, "emu: setup done (%u + %u directions with GCD rows)\n", nrows32, nrows64);

    const unsigned long long pts_cap = 1 << 20;
    const unsigned q_cap = 1 << 14;
    std::vector<SearchCtl> ctl(2);
    memset(ctl.data(), 0, 2 * sizeof(SearchCtl));
    std::vector<WorkItem> items(q_cap);
    std::vector<int> ready(q_cap, 0);
    std::vector<PointHdr> hdr(pts_cap);
    std::vector<int32_t> coords((size_t)pts_cap * MD);
    std::vector<unsigned long long> dnodes(nb, 0), retries(1, 0);
    std::vector<int32_t> dpass(nb, 1);
    SearchArgs A{};
    A.geo = geos.data(); A.dirs = dirs.data(); A.slab = slab.data(); A.items = items.data();
    A.ready = ready.data(); A.q_cap = q_cap; A.hdr = hdr.data(); A.coords = coords.data();
    A.pts_cap = pts_cap; A.npts = &ctl[0].npts; A.dir_nodes = dnodes.data(); A.eps = 1e-4;
    A.donate = 1; A.n_warps = n_warps; A.wait_ns = 30ll * 1000000000ll; A.deadline_ns = 600ll * 1000000000ll;
    // the device's choice of instantiation: one slot per lane when every h11 <= 32
    int hmax = 3;
    for (int k = 0; k < nb; ++k) hmax = std::max(hmax, geos[pgeo[k]].h);
    const bool one = hmax <= 32;
    if (!todo32.empty() && check_fp32) {
        // the FP32 bound-check form: one warp per direction with the FP64 shadow
        SearchArgs C = A;
        C.ctl = &ctl[0]; C.todo = todo32.data(); C.n_todo = (int)todo32.size(); C.pass = 1;
        C.donate = 0; C.n_warps = 1;
        launch((unsigned)todo32.size(), [&] {
            if (one) k_search_plain<float, 1, true>(C, -1); else k_search_plain<float, 2, true>(C, -1);
        });
        double m[3];
        memcpy(m, &ctl[0].chk_rem, sizeof m);
        g_emu_chk[0] = m[0]; g_emu_chk[1] = m[1]; g_emu_chk[2] = m[2];
        g_emu_chk[3] = (double)ctl[0].chk_narrower;
    } else if (!todo32.empty()) {
        A.ctl = &ctl[0]; A.todo = todo32.data(); A.n_todo = (int)todo32.size(); A.pass = 1;
        launch(n_warps, [&] { if (one) k_search<float, 1>(A); else k_search<float, 2>(A); });
    }
    for (int pid = 0; pid < nb; ++pid) {          // k_flip
        Dir &D = dirs[pid];
        if (!geos[D.geo].use_f32) { dpass[pid] = 2; continue; }
        if (D.status == ST_PENDING) D.status = ST_OK;
        else if (D.status == ST_FLOAT) { D.status = ST_PENDING; dpass[pid] = 2; retries[0]++; }
    }
    std::fill(ready.begin(), ready.end(), 0);
    A.ctl = &ctl[1]; A.todo = todoall.data(); A.n_todo = nb; A.pass = 2;
    launch(n_warps, [&] { if (one) k_search<double, 1>(A); else k_search<double, 2>(A); });
    if (ctl[0].err || ctl[1].err) { snprintf(out->err, sizeof out->err, "wait ran out"); return 1; }
    const unsigned long long npts = ctl[0].npts;
    if (npts > pts_cap) { snprintf(out->err, sizeof out->err, "point buffer overflow"); return 1; }
    const unsigned long long np1 = std::max<unsigned long long>(npts, 1);
    std::vector<unsigned> cnt(nb, 0), fill(nb, 0), idx(np1), perm(np1), perm2(np1), sidx(np1);
    int ks = 3;
    for (int k = 0; k < nb; ++k) ks = std::max(ks, geos[pgeo[k]].h);
    std::vector<int64_t> keys(np1 * ks);
    std::vector<unsigned long long> seg(nb + 1, 0), cseg(nb + 1, 0), summary(4, 0);
    OutArgs O{dirs.data(), slab.data(), hdr.data(), coords.data(), dpass.data(), npts, nb,
              cnt.data(), fill.data(), seg.data(), idx.data(), keys.data(), ks, cseg.data(), summary.data(),
              perm.data()};
    if (npts) launch(4, [&] { k_count(O); });
    launch(1, [&] { k_scan(O); });
    if (npts) launch(4, [&] { k_scatter(O); });
    const unsigned long long n_out = summary[0], n_chunks = summary[1], longest = summary[2];
    out->n = (int64_t)n_out;
    out->M = (int64_t *)malloc(n_out * MH * 8 + 8);
    out->Kn = (int64_t *)malloc(n_out * MH * 8 + 8);
    out->q = (int64_t *)malloc(n_out * 8 + 8);
    out->pidx = (int64_t *)malloc(n_out * 8 + 8);
    if (n_out) {
        launch(4, [&] { k_keys(O, n_out); });
        launch((unsigned)std::min<unsigned long long>(n_chunks, 8), [&] { k_segsort(O); });
        unsigned *pin = perm.data(), *pout = perm2.data();
        for (unsigned long long L = SORT_CAP; L < longest; L *= 2) {
            launch(4, [&] { k_merge(O, n_out, (unsigned)L, pin, pout); });
            std::swap(pin, pout);
        }
        launch(4, [&] { k_order(O, n_out, pin, sidx.data(), pout); });
        RowArgs R{dirs.data(), slab.data(), hdr.data(), coords.data(), sidx.data(), pout, keys.data(), ks, n_out, 0,
                  out->M, out->Kn, out->q, out->pidx, MH};
        launch(4, [&] { k_rows(R); });
    }
    for (int k = 0; k < nb; ++k) {
        const int st = dirs[k].status;
        out->pstat[k] = (st == ST_OK || st == ST_PENDING || st == ST_EMPTY) ? 0 : (int8_t)st;
        if (dir_nodes_out) dir_nodes_out[k] = (int64_t)dnodes[k];
        if (dir_debug) dir_debug[k] = dirs[k].pad;
    }
    return 0;
}

extern "C" void emu_output_free(pfg_output *out)
{
    free(out->M); free(out->Kn); free(out->q); free(out->pidx); free(out->pstat);
    memset(out, 0, sizeof *out);
}

// The setup's exact non-positive-definiteness witness (pfg_setup.cuh,
// witness_not_pd) on one emulated warp, for a d x d symmetric integer matrix:
// 1 if it proves A is not positive definite, else 0.
extern "C" int emu_witness_not_pd(const int64_t *A, int d)
{
    std::vector<double> U((size_t)d * d + 1), y((size_t)d + 1);
    int res = 0;
    emu_run_warp(0, 0, 32, 1, [&] {
        const bool w = witness_not_pd(A, d, U.data(), y.data(), threadIdx.x & 31);
        if ((threadIdx.x & 31) == 0) res = w ? 1 : 0;
    });
    return res;
}


// The device's coni dilation bound (pfg_mu0.cuh, k_mu0) on one emulated warp.
extern "C" int emu_coni_mu0_batch(int h, const int64_t *kappa, int64_t n_p, const int64_t *p_r, int32_t *status,
                                  int64_t *num, int64_t *den, int64_t *K)
{
    std::vector<Mu0Scratch> scr(1);
    unsigned next = 0;
    Mu0Args A{h, kappa, p_r, (int)n_p, &next, scr.data(), status, num, den, K, 20000000ll};
    emu_run_warp(0, 0, 32, 1, [&] { k_mu0(A); });
    return 0;
}


// The device's coniZpK above D0 (pfg_zpk.cuh, k_zpk) on one emulated warp:
// the points (rows of MH) into the caller's arrays of cap rows; returns the
// number of points emitted (more than cap: call again with room for them).
extern "C" long long emu_coni_zpk_batch(int h, const int64_t *kappa, const int64_t *Mbasis, const int64_t *ps,
                                        int64_t n_p, int64_t Q, int64_t M0min, int64_t D0, int64_t max_out,
                                        long long budget, unsigned long long cap, int64_t *M, int64_t *Kn,
                                        int64_t *q, int64_t *pidx, int32_t *status)
{
    std::vector<ZpkScratch> scr(1);
    memset((void *)scr.data(), 0xA5, sizeof(ZpkScratch));        // (the device's scratch is not zeroed either)
    unsigned next = 0;
    unsigned long long count = 0;
    ZpkArgs A{h, kappa, Mbasis, ps, h, (int)n_p, Q, M0min, D0, max_out, &next, scr.data(), status, &count, cap,
              M, Kn, q, pidx, budget};
    emu_run_warp(0, 0, 32, 1, [&] { k_zpk(A); });
    return (long long)count;
}

