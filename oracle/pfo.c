/*
 * ORACLE / TEST INFRASTRUCTURE -- never part of the product path.
 * See pfo.h.  Restates pfvs/fp_kernel/fpk_search_impl.h:217-455 (search),
 * :64-78 (fpk_bounds), :30-62 (search constants, fpk_need, GCD test) and
 * pfvs/fp_kernel/fpk_common.h:96-178 (gcd helpers, exact q) in the double
 * instantiation, without the CPU-only sparse-candidate and residue modes
 * (they change which candidates are tried, not the output).
 */
#include "pfo.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef __int128 i128;
typedef unsigned __int128 u128;

#define PFO_MAXD 128
#define PFO_G 1e-9

static u128 uabs128(i128 x) { return x < 0 ? (u128)0 - (u128)x : (u128)x; }

static uint64_t gcd64(uint64_t a, uint64_t b)
{
    while (b) { uint64_t t = a % b; a = b; b = t; }
    return a;
}

static u128 gcd128(u128 a, u128 b)
{
    while (b) { u128 t = a % b; a = b; b = t; }
    return a;
}

/* fpk_need (fpk_search_impl.h:43-51): smallest gcd that can pass when q >= q_lb */
static uint64_t need_of(double q_lb, int64_t Q, int strict)
{
    if (!(q_lb > 0)) return 0;
    double t = q_lb / (double)Q;
    t -= PFO_G * (1.0 + t);
    if (t < 0) t = 0;
    if (t >= 1.8e19) return UINT64_MAX;
    return strict ? (uint64_t)floor(t) + 1 : (uint64_t)ceil(t);
}

/* fpk_gcd_fails (fpk_search_impl.h:56-62): 1 if the branch must fail the cut */
static int gcd_fails(u128 g, int64_t Q, double q_lb, int strict)
{
    if (g == 0 || (g >> 64) != 0) return 0;
    double Qg = (double)Q * (double)(uint64_t)g;
    return strict ? (Qg <= q_lb) : (Qg < q_lb);
}

/* fpk_bounds (fpk_search_impl.h:67-78) */
static int bounds_of(double R, double off, double uinv, int64_t *lo, int64_t *hi)
{
    double a = (-R - off) * uinv, b = (R - off) * uinv;
    a = ceil(a - PFO_G * (1.0 + fabs(a)));
    b = floor(b + PFO_G * (1.0 + fabs(b)));
    if (!(a >= -2147483647.0 && b <= 2147483647.0)) return -8;
    *lo = (int64_t)a;
    *hi = (int64_t)b;
    return 0;
}

/* exact q(c) = c^T mat c in int128 (fpk_common.h:158-178); 1 on overflow */
static int exact_q(const int64_t *mat, const int32_t *c, int d, i128 *out)
{
    i128 q = 0;
    for (int i = 0; i < d; ++i) {
        if (!c[i]) continue;
        i128 row = 0;
        for (int j = i + 1; j < d; ++j) row += (i128)mat[i * d + j] * c[j];
        i128 t;
        if (__builtin_mul_overflow(row, (i128)2, &t)) return 1;
        if (__builtin_add_overflow(t, (i128)mat[i * d + i] * c[i], &t)) return 1;
        if (__builtin_mul_overflow(t, (i128)c[i], &t)) return 1;
        if (__builtin_add_overflow(q, t, &q)) return 1;
    }
    *out = q;
    return 0;
}

typedef struct { int32_t *pts; int64_t *qs; long n, cap; int d; } pfo_out;

static int push(pfo_out *o, const int32_t *c, int64_t q, long max_out)
{
    if (o->n >= max_out) return -2;
    if (o->n == o->cap) {
        long cap = o->cap ? 2 * o->cap : 64;
        int32_t *p = realloc(o->pts, (size_t)cap * o->d * 4);
        if (!p) return -7;
        o->pts = p;
        int64_t *qq = realloc(o->qs, (size_t)cap * 8);
        if (!qq) return -7;
        o->qs = qq;
        o->cap = cap;
    }
    memcpy(&o->pts[o->n * o->d], c, (size_t)o->d * 4);
    o->qs[o->n++] = q;
    return 0;
}

void pfo_free(void *p) { free(p); }

int pfo_search(const pfo_problem *P, int32_t **pts_out, int64_t **qs_out, long *n_out, long *nodes_out)
{
    const int d = P->dim;
    *pts_out = NULL; *qs_out = NULL; *n_out = 0; *nodes_out = 0;
    if (d < 1 || d > PFO_MAXD) return -6;
    if (P->qmax < 0) return 0;
    const double *U = P->U;
    const double qd = (double)P->qmax;
    const double slack = fmax(P->eps, PFO_G * (qd + 1.0));
    const double Kerr = 2.0 * (d + 8) * 0x1p-53;
    const int64_t *lv = P->linvec;
    int m0_level = -1;
    if (lv) {
        for (int j = 0; j < d; ++j) if (lv[j]) { m0_level = j; break; }
        if (m0_level < 0 && 0 < P->linmin) return 0;
    }
    /* pruning rows grouped by first nonzero column */
    int np = P->nprune, use_gcd = np > 0;
    int level_start[PFO_MAXD + 1], *order = malloc((size_t)(np + 1) * sizeof(int));
    i128 *pre = malloc((size_t)(np + 1) * sizeof(i128));
    if (!order || !pre) { free(order); free(pre); return -7; }
    {
        int cnt[PFO_MAXD + 1] = {0}, lvl_of[1024];
        int *lvl = np <= 1024 ? lvl_of : malloc((size_t)np * sizeof(int));
        for (int r = 0; r < np; ++r) {
            lvl[r] = -1;
            for (int j = 0; j < d; ++j) if (P->Hp[r * d + j]) { lvl[r] = j; break; }
            if (lvl[r] >= 0) cnt[lvl[r]]++;
        }
        level_start[0] = 0;
        for (int l = 0; l < d; ++l) level_start[l + 1] = level_start[l] + cnt[l];
        int fill[PFO_MAXD + 1];
        memcpy(fill, level_start, sizeof(int) * (d + 1));
        for (int r = 0; r < np; ++r) if (lvl[r] >= 0) order[fill[lvl[r]]++] = r;
        if (lvl != lvl_of) free(lvl);
    }
    double uinv[PFO_MAXD];
    for (int i = 0; i < d; ++i) uinv[i] = 1.0 / U[i * d + i];

    int32_t c[PFO_MAXD];
    int64_t cur[PFO_MAXD], hi[PFO_MAXD];
    double rem[PFO_MAXD], err[PFO_MAXD], off[PFO_MAXD], aoff[PFO_MAXD];
    i128 m0p[PFO_MAXD];
    u128 g[PFO_MAXD + 1];
    for (int j = 0; j < d; ++j) c[j] = 0;
    pfo_out o = { NULL, NULL, 0, 0, d };
    long nodes = 0;
    int status = 0;

#define ENTER(I) do {                                                              \
        const int i_ = (I);                                                        \
        double o_ = 0, a_ = 0;                                                     \
        for (int j = i_ + 1; j < d; ++j) { double t = U[i_ * d + j] * c[j]; o_ += t; a_ += fabs(t); } \
        off[i_] = o_; aoff[i_] = a_;                                               \
        if (use_gcd)                                                               \
            for (int k = level_start[i_]; k < level_start[i_ + 1]; ++k) {          \
                int r = order[k]; i128 s = 0;                                      \
                for (int j = i_ + 1; j < d; ++j) s += (i128)P->Hp[r * d + j] * c[j]; \
                pre[r] = s;                                                        \
            }                                                                      \
        double R = sqrt(fmax(rem[i_] + slack + err[i_], 0.0));                    \
        R += Kerr * (R + 2.0 * a_) + 1e-300;                                       \
        int empty = 0;                                                             \
        if (use_gcd && g[i_ + 1] != 0 && (g[i_ + 1] >> 64) == 0) {                \
            double am = R + 2.0 * a_;                                              \
            double Rg2 = (double)P->Q * (double)(uint64_t)g[i_ + 1] - (qd - rem[i_]) \
                         + slack + err[i_] + Kerr * (am * am + rem[i_]);           \
            if (Rg2 < 0) empty = 1;                                                \
            else { double Rg = sqrt(Rg2); Rg += Kerr * (Rg + 2.0 * a_) + 1e-300; if (Rg < R) R = Rg; } \
        }                                                                          \
        if (!empty && lv && i_ >= m0_level && m0_level >= 0) {                     \
            double vc = 0, va = 0;                                                 \
            for (int j = i_ + 1; j < d; ++j) {                                     \
                vc += P->m0V[i_ * d + j] * c[j];                                   \
                va += P->m0Va[i_ * d + j] * fabs((double)c[j]);                    \
            }                                                                      \
            double sq = sqrt(fmax(P->m0N[i_] * (rem[i_] + slack + err[i_]), 0.0)); \
            double ub = (double)m0p[i_] - vc + sq + Kerr * (va + sq + fabs((double)m0p[i_])) + 1e-9; \
            if (ub < (double)P->linmin) empty = 1;                                 \
        }                                                                          \
        int64_t lo = 1, hh = 0;                                                    \
        if (!empty && bounds_of(R, off[i_], uinv[i_], &lo, &hh)) { status = -8; goto done; } \
        if (!empty && i_ == m0_level) {                                            \
            i128 need = (i128)P->linmin - m0p[i_], l = lv[i_];                     \
            if (l > 0) {                                                           \
                i128 b = need >= 0 ? (need + l - 1) / l : -((-need) / l);          \
                if (b > lo) lo = b > hh ? hh + 1 : (int64_t)b;                     \
            } else {                                                               \
                i128 nl = -l;                                                      \
                i128 b = need <= 0 ? (-need) / nl : -((need + nl - 1) / nl);       \
                if (b < hh) hh = b < lo ? lo - 1 : (int64_t)b;                     \
            }                                                                      \
        }                                                                          \
        cur[i_] = lo; hi[i_] = hh;                                                 \
        nodes++;                                                                   \
    } while (0)

    int i = d - 1;
    rem[i] = qd;
    err[i] = Kerr * qd;
    m0p[i] = 0;
    g[d] = 0;
    ENTER(i);
    while (i < d) {
        if (cur[i] > hi[i]) { c[i] = 0; i++; continue; }
        int32_t v = (int32_t)cur[i]++;
        c[i] = v;
        double x = U[i * d + i] * v + off[i];
        double nr = rem[i] - x * x;
        double ai = fabs(U[i * d + i] * v) + aoff[i];
        double en = err[i] + Kerr * (ai * ai + rem[i]);
        if (nr < -(slack + en)) continue;
        i128 m0 = m0p[i] + (lv ? (i128)lv[i] * v : 0);
        if (i == m0_level && m0 < P->linmin) continue;
        if (use_gcd) {
            u128 gn = g[i + 1];
            double q_lb = (qd - nr) - (slack + en);
            uint64_t need = need_of(q_lb, P->Q, P->strict);
            int pruned = 0;
            for (int k = level_start[i]; k < level_start[i + 1]; ++k) {
                if (gcd_fails(gn, P->Q, q_lb, P->strict)) { pruned = 1; break; }
                int r = order[k];
                u128 a = uabs128(pre[r] + (i128)P->Hp[r * d + i] * v);
                gn = ((gn >> 64) == 0 && (a >> 64) == 0) ? gcd64((uint64_t)gn, (uint64_t)a)
                                                          : gcd128(gn, a);
                if (gn != 0 && gn < need) { pruned = 1; break; }
            }
            if (pruned || gcd_fails(gn, P->Q, q_lb, P->strict)) continue;
            g[i] = gn;
        }
        if (i > 0) {
            m0p[i - 1] = m0; rem[i - 1] = nr; err[i - 1] = en;
            i--;
            ENTER(i);
            continue;
        }
        /* leaf: exact tests */
        i128 q;
        if (exact_q(P->mat, c, d, &q)) { status = -12; goto done; }
        if (q > P->qmax) continue;
        if (lv) {
            i128 m = 0;
            for (int j = 0; j < d; ++j) m += (i128)lv[j] * c[j];
            if (m < P->linmin) continue;
        }
        if (P->leaf_gcd) {
            u128 gg = 0;
            for (int r = 0; r < P->nleaf; ++r) {
                i128 s = 0;
                for (int j = 0; j < d; ++j) s += (i128)P->Hl[r * d + j] * c[j];
                gg = gcd128(gg, uabs128(s));
            }
            if (gg != 0 && (gg >> 64) == 0) {
                i128 Qg = (i128)P->Q * (i128)(uint64_t)gg;
                if (P->strict ? (Qg <= q) : (Qg < q)) continue;
            }
        }
        int rc = push(&o, c, (int64_t)q, P->max_out);
        if (rc) { status = rc; goto done; }
    }
done:
#undef ENTER
    free(order); free(pre);
    *pts_out = o.pts; *qs_out = o.qs; *n_out = o.n; *nodes_out = nodes;
    return status;
}
