/*
 * ORACLE / TEST INFRASTRUCTURE -- never part of the product path.
 *
 * A C driver around the reference's own CPU sources, compiled in place from
 * the reference tree (pfvs/fp_kernel/pfv_lattice.h, fpk_common.h,
 * fpk_search_impl.h, fp_kernel.h) by oracle/Makefile into oracle/_ref/.
 * It replays the loop of the reference's Cython batch driver
 * `_coni_batch` (pfvs/fp_kernel/fp_kernel.pyx:544-609): per p-vector
 * `pfl_build`, the int64 check of H (fp_kernel.pyx:551-559),
 * `fpk_enumerate`, and M = Binter c, Kn = ZB c in int128 -> int64
 * (fp_kernel.pyx:591-609), with the same status convention
 * (0 done, 1 "exact per-p path needed", < 0 kernel status).
 *
 * Also exposes the kernel boundary (`conipfv_kernel` / `pfv_kernel`,
 * fp_kernel.pyx:258-350 -> fpk_enumerate) with arbitrary-precision H rows,
 * and the lattice setup alone (`_lattice_build`, fp_kernel.pyx:355-401).
 *
 * Used by tests/ (to pin the oracle) and by bench.py's CPU baseline arm.
 */
#define FP_KERNEL_IMPLEMENTATION
#define PFV_LATTICE_IMPLEMENTATION
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "fp_kernel.h"
#include "pfv_lattice.h"

typedef struct {
    int64_t *M, *Kn, *q, *pidx;   /* (n, h), (n, h), (n,), (n,) */
    long n, cap;
} ref_points;

void ref_points_free(ref_points *P)
{
    free(P->M); free(P->Kn); free(P->q); free(P->pidx);
    memset(P, 0, sizeof *P);
}

static int ref_grow(ref_points *P, long need, int h)
{
    if (need <= P->cap) return 0;
    long cap = 2 * P->cap > need ? 2 * P->cap : need + 64;
    int64_t *M = realloc(P->M, (size_t)cap * h * 8);
    if (!M) return -7;
    P->M = M;
    int64_t *K = realloc(P->Kn, (size_t)cap * h * 8);
    if (!K) return -7;
    P->Kn = K;
    int64_t *q = realloc(P->q, (size_t)cap * 8);
    if (!q) return -7;
    P->q = q;
    int64_t *p = realloc(P->pidx, (size_t)cap * 8);
    if (!p) return -7;
    P->pidx = p;
    P->cap = cap;
    return 0;
}

/*
 * Row-style Hermite normal form in GMP (upper echelon, positive pivots,
 * entries above a pivot reduced into [0, pivot), zero rows last): the
 * canonical form flint's HNF returns, which the reference's per-p path
 * feeds to the kernel (pfvs/coni.py:172-202 `coni_H_matrix`).  Used when the
 * int128 HNF of pfl_build does not fit (pfl_build status -15).
 * Column-by-column Euclidean elimination; A is (r x n), overwritten.
 */
static void ref_hnf_mpz(mpz_t *A, int r, int n)
{
    mpz_t q;
    mpz_init(q);
    int row = 0;
    for (int col = 0; col < n && row < r; ++col) {
        for (;;) {
            int piv = -1;
            for (int i = row; i < r; ++i)
                if (mpz_sgn(A[i * n + col]) != 0 &&
                    (piv < 0 || mpz_cmpabs(A[i * n + col], A[piv * n + col]) < 0))
                    piv = i;
            if (piv < 0) break;
            if (piv != row)
                for (int c = 0; c < n; ++c) mpz_swap(A[row * n + c], A[piv * n + c]);
            int clean = 1;
            for (int i = row + 1; i < r; ++i) {
                if (mpz_sgn(A[i * n + col]) == 0) continue;
                mpz_fdiv_q(q, A[i * n + col], A[row * n + col]);
                for (int c = col; c < n; ++c) mpz_submul(A[i * n + c], q, A[row * n + c]);
                if (mpz_sgn(A[i * n + col]) != 0) clean = 0;
            }
            if (clean) break;
        }
        if (mpz_sgn(A[row * n + col]) == 0) continue;
        if (mpz_sgn(A[row * n + col]) < 0)
            for (int c = col; c < n; ++c) mpz_neg(A[row * n + c], A[row * n + c]);
        for (int i = 0; i < row; ++i) {
            mpz_fdiv_q(q, A[i * n + col], A[row * n + col]);
            if (mpz_sgn(q) == 0) continue;
            for (int c = col; c < n; ++c) mpz_submul(A[i * n + c], q, A[row * n + c]);
        }
        row++;
    }
    mpz_clear(q);
}

static int ref_grow_into(ref_points *out, long extra, int h) { return ref_grow(out, out->n + extra, h); }

/* M = Binter c, Kn = ZB c for the kernel's points; 1 if any entry is beyond
 * int64 (the reference then redoes the direction in Python ints). */
static int ref_emit(ref_points *out, const pfl_result *R, int h, const fpk_output *o, long pidx)
{
    const int d = h - 1;
    if (ref_grow_into(out, o->n, h)) return -7;
    long start = out->n;
    int bad = 0;
    for (long t = 0; t < o->n; ++t) {
        for (int i = 0; i < h; ++i) {
            pfl_i128 am = 0, ak = 0;
            for (int a = 0; a < d; ++a) {
                am += (pfl_i128)R->Binter[i * d + a] * o->pts[t * d + a];
                ak += (pfl_i128)R->ZB[i * d + a] * o->pts[t * d + a];
            }
            if (am > (pfl_i128)INT64_MAX || am < -(pfl_i128)INT64_MAX ||
                ak > (pfl_i128)INT64_MAX || ak < -(pfl_i128)INT64_MAX) bad = 1;
            out->M[out->n * h + i] = (int64_t)am;
            out->Kn[out->n * h + i] = (int64_t)ak;
        }
        out->q[out->n] = o->qs[t];
        out->pidx[out->n] = pidx;
        out->n++;
    }
    if (bad) { out->n = start; return 1; }
    return 0;
}

/*
 * Batched coni pipeline on the CPU, one geometry: the loop of
 * fp_kernel.pyx:544-609.  `pidx_base` is added to every emitted pidx (so
 * callers can split a batch over threads).  nodes[ip] receives the
 * kernel's n_nodes for p-vector ip (0 when it did not run).
 *
 * With per_p != 0, a direction the batch loop hands on (status 1) is also
 * finished the way the reference's per-p path finishes it
 * (pfvs/coni.py:1025-1141) whenever that path needs no python-flint lattice
 * code: the same pfl_build data, H from the int128 HNF (or, on pfl_build
 * status -15, the GMP HNF above), and fpk_enumerate with the H rows in GMP.
 * Such directions get status 0 (done) and their points are emitted; a
 * direction whose setup itself overflowed keeps status 1.
 */
int ref_coni_batch(int h, const int64_t *kappa, const int64_t *Mbasis,
                   const int64_t *ps, long n, int64_t Q, int64_t qmax,
                   int64_t linmin, long max_N_out, double eps, long pidx_base,
                   int per_p, ref_points *out, int32_t *status, int64_t *nodes)
{
    const int d = h - 1;
    pfl_setup S;
    S.h11 = h; S.kappa = kappa; S.Mbasis = Mbasis;
    S.coni = 1; S.extra_lll = 1; S.m0_basis = 1;
    fpk_problem P;
    memset(&P, 0, sizeof P);
    P.dim = d; P.qmax = qmax; P.Q = Q; P.strict = 1; P.linmin = linmin;
    P.max_N_out = max_N_out; P.eps = eps;
    pfl_result *R = malloc(sizeof *R);
    int64_t *H64 = malloc((size_t)h * d * 8);
    mpz_t *Hz = malloc((size_t)h * d * sizeof(mpz_t));
    if (!R || !H64 || !Hz) { free(R); free(H64); free(Hz); return -7; }
    for (int k = 0; k < h * d; ++k) mpz_init(Hz[k]);
    memset(out, 0, sizeof *out);
    for (long ip = 0; ip < n; ++ip) {
        status[ip] = 0;
        if (nodes) nodes[ip] = 0;
        int st = pfl_build(&S, &ps[ip * h], R);
        int use_mpz = 0;
        if (st == -15 && per_p) {
            /* H = canonical HNF of ZB[1:] in GMP */
            for (int k = 0; k < d * d; ++k) mpz_set_si(Hz[k], R->ZB[d + k]);
            ref_hnf_mpz(Hz, d, d);
            P.nrows = d;
            use_mpz = 1;
        } else if (st != 0) {
            status[ip] = 1;
            continue;
        } else {
            int bad = 0;
            for (int k = 0; k < R->nrows * d; ++k) {
                pfl_i128 hv = R->H[k];
                if (hv > (pfl_i128)INT64_MAX || hv < -(pfl_i128)INT64_MAX) { bad = 1; break; }
                H64[k] = (int64_t)hv;
            }
            P.nrows = R->nrows;
            if (bad) {
                if (!per_p) { status[ip] = 1; continue; }
                for (int k = 0; k < R->nrows * d; ++k) {
                    pfl_u128 a = R->H[k] < 0 ? (pfl_u128)0 - (pfl_u128)R->H[k] : (pfl_u128)R->H[k];
                    uint64_t w[2] = { (uint64_t)a, (uint64_t)(a >> 64) };
                    mpz_import(Hz[k], 2, -1, 8, 0, 0, w);
                    if (R->H[k] < 0) mpz_neg(Hz[k], Hz[k]);
                }
                use_mpz = 1;
            }
        }
        P.mat = R->mat; P.linvec = &R->Binter[0];
        P.H = use_mpz ? Hz : NULL;
        P.H64 = use_mpz ? NULL : H64;
        fpk_output o;
        memset(&o, 0, sizeof o);
        st = fpk_enumerate(&P, &o);
        if (nodes) nodes[ip] = o.n_nodes;
        if (st != 0) { status[ip] = st; fpk_output_free(&o); continue; }
        int e = ref_emit(out, R, h, &o, pidx_base + ip);
        fpk_output_free(&o);
        if (e < 0) status[ip] = -7;
        else if (e > 0) status[ip] = 1;
    }
    for (int k = 0; k < h * d; ++k) mpz_clear(Hz[k]);
    free(R); free(H64); free(Hz);
    return 0;
}

/*
 * The kernel boundary (fpk_enumerate) with H given as signed multi-limb
 * integers: entry e of H is sign[e] * sum_k limbs[e * nl + k] 2^(64k).
 * linvec may be NULL (pfv_kernel).  Points are written to *pts (n x dim
 * int32, malloc'd) and *qs (malloc'd); release with ref_free.
 */
int ref_kernel(int dim, const int64_t *mat, int64_t qmax, int64_t Q, int nrows,
               const int8_t *sign, const uint64_t *limbs, int nl, int strict,
               const int64_t *linvec, int64_t linmin, long max_N_out, double eps,
               int32_t **pts, int64_t **qs, long *n, long *n_nodes)
{
    mpz_t *H = NULL;
    if (nrows > 0) {
        H = malloc((size_t)nrows * dim * sizeof(mpz_t));
        if (!H) return -7;
        for (long e = 0; e < (long)nrows * dim; ++e) {
            mpz_init(H[e]);
            mpz_import(H[e], (size_t)nl, -1, 8, 0, 0, &limbs[e * nl]);
            if (sign[e] < 0) mpz_neg(H[e], H[e]);
        }
    }
    fpk_problem P;
    memset(&P, 0, sizeof P);
    P.dim = dim; P.mat = mat; P.qmax = qmax; P.Q = Q; P.nrows = nrows; P.H = H;
    P.H64 = NULL; P.strict = strict; P.linvec = linvec; P.linmin = linmin;
    P.max_N_out = max_N_out; P.eps = eps;
    fpk_output o;
    memset(&o, 0, sizeof o);
    int st = fpk_enumerate(&P, &o);
    *pts = o.pts; *qs = o.qs; *n = o.n; *n_nodes = o.n_nodes;
    if (H) {
        for (long e = 0; e < (long)nrows * dim; ++e) mpz_clear(H[e]);
        free(H);
    }
    return st;
}

void ref_free(void *p) { free(p); }

/*
 * The lattice setup alone (pfl_build, as fp_kernel.pyx:_lattice_build).
 * H is returned as int128 entries split into (lo, hi) int64 words.
 */
int ref_lattice_build(int h, const int64_t *kappa, const int64_t *Mbasis,
                      const int64_t *p, int coni, int extra_lll, int m0_basis,
                      int64_t *Z, int64_t *Binter, int64_t *ZB, int64_t *mat,
                      int64_t *H_lohi, int *nrows)
{
    pfl_setup S;
    S.h11 = h; S.kappa = kappa; S.Mbasis = Mbasis;
    S.coni = coni; S.extra_lll = extra_lll; S.m0_basis = m0_basis;
    pfl_result *R = malloc(sizeof *R);
    if (!R) return -7;
    int st = pfl_build(&S, p, R);
    if (st == 0 || st == -15) {
        const int d = h - 1;
        memcpy(Z, R->Z, (size_t)h * h * 8);
        memcpy(Binter, R->Binter, (size_t)h * d * 8);
        memcpy(ZB, R->ZB, (size_t)h * d * 8);
        memcpy(mat, R->mat, (size_t)d * d * 8);
        *nrows = st == 0 ? R->nrows : 0;
        if (st == 0)
            for (int k = 0; k < R->nrows * d; ++k) {
                H_lohi[2 * k] = (int64_t)(uint64_t)R->H[k];
                H_lohi[2 * k + 1] = (int64_t)(R->H[k] >> 64);
            }
    }
    free(R);
    return st;
}

/* The reference's coni dilation bound mu0 (pfvs/fp_kernel/coni_bound.h:255,
 * the C path of pfvs.dilation.coni_mu0, dilation.py:145): status 0 with
 * mu0 = *num / *den and K a minimizer (h - 1 entries), 1 when the bound's
 * hypotheses fail (A_rr singular, s > 0, S not positive definite on Lambda),
 * < 0 when the C path cannot decide (the reference then uses flint). */
#include "coni_bound.h"
int ref_coni_mu0(int h, const int64_t *kappa, const int64_t *p_r, int64_t *num, int64_t *den, int64_t *K)
{
    return cb_coni_mu0(h, kappa, p_r, num, den, K);
}

/* the same over the n rows of P ((n, h-1)): statuses into st */
void ref_coni_mu0_batch(int h, const int64_t *kappa, int64_t n, const int64_t *P, int32_t *st, int64_t *num,
                        int64_t *den, int64_t *K)
{
    for (int64_t i = 0; i < n; ++i)
        st[i] = cb_coni_mu0(h, kappa, P + i * (h - 1), num + i, den + i, K + i * (h - 1));
}

/* The reference's coniZpK above D0 (pfvs/fp_kernel/coni_zpk.h:714, czk_batch,
 * as its _coni_zpk_batch binding calls it, fp_kernel.pyx:434): for the n rows
 * of ps ((n, h), p[0] = 0), the lattice points (M, Kn rows of h; q; pidx) and
 * a status per row (points kept only where it is 0).  The arrays are
 * malloc'd here (ref_free); returns the number of points. */
#include "coni_zpk.h"
long ref_coni_zpk_batch(int h, const int64_t *kappa, const int64_t *Mbasis, const int64_t *ps, long n, int64_t Q,
                        int64_t M0min, int64_t D0, long max_out, int64_t **M, int64_t **Kn, int64_t **q,
                        int64_t **pidx, int32_t *status)
{
    czk_points P;
    memset(&P, 0, sizeof P);
    int *st = (int *)malloc(sizeof(int) * (n ? n : 1));
    for (long i = 0; i < n; ++i) st[i] = -20;
    if (n && h >= 3 && h <= CZK_MAX_H11) czk_batch(h, kappa, Mbasis, ps, n, Q, M0min, D0, max_out, &P, st);
    for (long i = 0; i < n; ++i) status[i] = st[i];
    free(st);
    *M = P.M; *Kn = P.Kn; *q = P.q; *pidx = P.pidx;
    return P.n;
}

