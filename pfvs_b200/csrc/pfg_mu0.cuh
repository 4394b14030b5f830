// The coni dilation bound mu0 on the device, one warp per direction.
//
// For p_hat = (0, p_r) of a geometry kappa (the reference computes this on
// the CPU: pfvs/dilation.py:145-180, in C for h11 <= 20 in
// pfvs/fp_kernel/coni_bound.h:255):
//
//   A = kappa . p_hat,  s = a00 - a_r0^T A_rr^-1 a_r0,  S = -A_rr^-1
//   Lambda = {K in Z^(h-1) : p_r . K = 0}
//   mu0 = min over nonzero K in Lambda of K^T S K
//
// Every coni PFV with direction p_hat has dilation below Q / mu0 when s <= 0
// and S is positive definite on Lambda; otherwise there is no bound.
//
// Steps (exact integers throughout; floating point only prunes the last
// search, with a proven margin):
//   1. A in int64 (checked), a basis O of Lambda (rows 1.. of a unimodular U
//      with U p_r = (g, 0, ..)).
//   2. Fraction-free (Bareiss) elimination of [A_rr | O^T | a_r0] (entries in
//      int128, each step's products in 256 bits with a checked exact
//      division), then X = d A_rr^-1 [O^T | a_r0] by exact back substitution (d the
//      last pivot, +-det A_rr): s from X's last column, and the form of S on
//      O's basis as the integer matrix G = -O X[:, :n] / g * sign(d) with
//      L = |d| / g (g the gcd of d and -O X), so S = G / L there.
//   3. LLL of Lambda's basis w.r.t. G (the setup's warp LLL on the exact
//      Gram), then the minimum of y^T Gr y over nonzero integer y by a
//      depth-first search whose floating-point pruning is widened by the
//      Cholesky factor's certified backward error and the dot products'
//      rounding bounds; every leaf is decided in exact int128.
//   4. K = O^T V^T y for the LLL transform V; mu0 = min / L in lowest terms.
//
// Status: 0 decided; 1 no bound (A_rr singular, s > 0, or S not positive
// definite on Lambda); < 0 not decided here (a value beyond int128 / int64,
// a form too ill-conditioned for the pruning, the search's node budget).
#pragma once
#include "pfg_setup.cuh"

namespace pfg {

constexpr int MU0_MAXH = 32;                  // h11 of the device bound (int128 limits it in practice)
enum {
    MU0_OK = 0, MU0_NONE = 1,
    MU0_RANGE = -20, MU0_OVF_A = -1, MU0_ORTH = -2, MU0_OVF_SOLVE = -3, MU0_INEXACT = -4,
    MU0_OVF_GRAM = -5, MU0_LLL = -6, MU0_ILLCOND = -31, MU0_OVF_LEAF = -34, MU0_BUDGET = -35
};

// Signed 256-bit integers (two's complement, four 64-bit limbs) for the
// elimination's products: a Bareiss step (p_k a_ij - a_ik a_kj) / p_(k-1) has
// an int128 result whenever the minors fit, but its products do not.
struct W256 { uint64_t w[4]; };

PFG_HD W256 w256(i128 x)
{
    const uint64_t ext = x < 0 ? ~0ull : 0ull;
    return W256{{(uint64_t)(u128)x, (uint64_t)((u128)x >> 64), ext, ext}};
}
PFG_HD bool w_neg_sign(const W256 &a) { return (int64_t)a.w[3] < 0; }
PFG_HD W256 w_neg(const W256 &a)
{
    W256 r;
    uint64_t c = 1;
    for (int i = 0; i < 4; ++i) { const uint64_t v = ~a.w[i] + c; c = (c && v == 0) ? 1 : 0; r.w[i] = v; }
    return r;
}
// a + b; true on signed overflow
PFG_HD bool w_add(const W256 &a, const W256 &b, W256 *r)
{
    W256 s;
    uint64_t c = 0;
    for (int i = 0; i < 4; ++i) {
        const u128 t = (u128)a.w[i] + b.w[i] + c;
        s.w[i] = (uint64_t)t;
        c = (uint64_t)(t >> 64);
    }
    const bool ovf = w_neg_sign(a) == w_neg_sign(b) && w_neg_sign(s) != w_neg_sign(a);
    *r = s;
    return ovf;
}
PFG_HD bool w_sub(const W256 &a, const W256 &b, W256 *r) { return w_add(a, w_neg(b), r) || (b.w[3] == (1ull << 63) && !b.w[2] && !b.w[1] && !b.w[0]); }
// the exact product of two int128 values (|a b| < 2^254, so it always fits)
PFG_HD W256 w_mul(i128 a, i128 b)
{
    const u128 ua = uabs(a), ub = uabs(b);
    const uint64_t a0 = (uint64_t)ua, a1 = (uint64_t)(ua >> 64), b0 = (uint64_t)ub, b1 = (uint64_t)(ub >> 64);
    const u128 p00 = (u128)a0 * b0, p01 = (u128)a0 * b1, p10 = (u128)a1 * b0, p11 = (u128)a1 * b1;
    W256 r;
    r.w[0] = (uint64_t)p00;
    const u128 mid = (p00 >> 64) + (uint64_t)p01 + (uint64_t)p10;
    r.w[1] = (uint64_t)mid;
    const u128 hi = (mid >> 64) + (p01 >> 64) + (p10 >> 64) + (uint64_t)p11;
    r.w[2] = (uint64_t)hi;
    r.w[3] = (uint64_t)(hi >> 64) + (uint64_t)(p11 >> 64);
    return ((a < 0) != (b < 0)) ? w_neg(r) : r;
}
PFG_HD bool w_eq(const W256 &a, const W256 &b)
{
    return a.w[0] == b.w[0] && a.w[1] == b.w[1] && a.w[2] == b.w[2] && a.w[3] == b.w[3];
}
PFG_HD bool w_is_zero(const W256 &a) { return !(a.w[0] | a.w[1] | a.w[2] | a.w[3]); }
// whether a is an int128 value, and that value
PFG_HD bool w_fits128(const W256 &a)
{
    const uint64_t ext = (int64_t)a.w[1] < 0 ? ~0ull : 0ull;
    return a.w[2] == ext && a.w[3] == ext;
}
PFG_HD i128 w_lo(const W256 &a) { return (i128)(((u128)a.w[1] << 64) | a.w[0]); }

// Exact division by a fixed nonzero int128 divisor p = 2^t o (o odd): the
// quotient of an exact division x / p is (x >> t) o^-1 mod 2^128 when it fits
// int128, and the product back is compared with x, so a wrong (inexact or too
// large) quotient is always detected.
struct ExactDiv {
    i128 p;
    int t;
    u128 inv;                                   // o^-1 mod 2^128
};
PFG_HD ExactDiv exact_div(i128 p)
{
    ExactDiv D;
    D.p = p;
    D.t = ctz128((u128)p);
    const u128 o = (u128)(p >> D.t);            // (odd: p = 2^t o, an arithmetic shift keeping the sign)
    u128 x = o;                                 // (correct to 3 bits: o o = 1 mod 8)
    for (int i = 0; i < 6; ++i) x *= (u128)2 - o * x;      // Newton: 3 -> 192 bits
    D.inv = x;
    return D;
}
// x / D.p into *q; true when the division is not exact or the quotient is not an int128 value
PFG_HD bool exact_quot(const W256 &x, const ExactDiv &D, i128 *q)
{
    const int t = D.t;
    if (t && (t < 64 ? (x.w[0] & ((1ull << t) - 1)) : (x.w[0] || (x.w[1] & ((1ull << (t - 64)) - 1))))) return true;
    u128 lo;
    if (t == 0) lo = ((u128)x.w[1] << 64) | x.w[0];
    else if (t < 64) lo = (((u128)x.w[1] << 64) | x.w[0]) >> t | ((u128)x.w[2] << (128 - t));
    else lo = (((u128)x.w[2] << 64) | x.w[1]) >> (t - 64) | (t > 64 ? (u128)x.w[3] << (192 - t) : 0);
    // (t < 128: p != 0 fits int128; for t == 64 the second term is not needed)
    *q = (i128)(lo * D.inv);
    return !w_eq(w_mul(*q, D.p), x);
}

struct Mu0Scratch {
    int64_t U[(MU0_MAXH - 1) * MH];           // unimodular transform of p_r (rows, stride MH)
    int64_t w[MH];
    int perm[MH];
    i128 M[(MU0_MAXH - 1) * 64];              // [A_rr | O^T | a_r0], stride 64
    i128 X[(MU0_MAXH - 1) * 32];              // d A_rr^-1 [O^T | a_r0], stride 32
    int64_t Gr[32 * 32];                      // the reduced integral form
    double R[32 * 32];                        // its FP64 Cholesky factor
    LllMem<32> L;                             // LLL working set (basis of Lambda in O's coordinates)
    int64_t Lb[31 * 32];                      // its rows
};

struct Mu0Args {
    int h;
    const int64_t *kappa;                     // h^3
    const int64_t *pr;                        // (n_p, h - 1)
    int n_p;
    unsigned *next;                           // work counter
    Mu0Scratch *scratch;                      // one per warp
    int32_t *status;
    int64_t *mu_num, *mu_den, *K;             // (n_p,), (n_p,), (n_p, h - 1)
    long long node_budget;
};

// min y^T G y over nonzero integer y (lane 0 only; G n x n int64, positive
// definite by construction, LLL-reduced): *best enters as the smallest
// diagonal entry with y its unit vector.
//
// Pruning: the FP64 Cholesky R has R^T R = G + E, |E| <= g1 |R^T||R| (g1 =
// gamma_{n+1}), so y^T G y >= |R y|^2 (1 - g1 C), C = 2 ||R||_F^2 ||R^-1||_F^2;
// y^T G y < best therefore needs |R y|^2 < rad = best / (1 - g1 C).  A level's
// term t_i = (R y)_i is computed with error at most g2 a_i (g2 = gamma_n, a_i
// the sum of |R_ij y_j|), and a value is dropped only when the sum of the
// levels' lower bounds (|t_i| - g2 a_i)_+^2 exceeds rad; candidate ranges
// are widened by one on each side.
__device__ int mu0_min(const int64_t *G, double *R, int n, int64_t &best, int64_t *ybest, long long budget)
{
    for (int j = 0; j < n; ++j) {                                   // G = R^T R
        double dj = (double)G[j * 32 + j];
        for (int k = 0; k < j; ++k) dj -= R[k * 32 + j] * R[k * 32 + j];
        if (!(dj > 0)) return MU0_ILLCOND;
        R[j * 32 + j] = sqrt(dj);
        for (int i = j + 1; i < n; ++i) {
            double t = (double)G[j * 32 + i];
            for (int k = 0; k < j; ++k) t -= R[k * 32 + j] * R[k * 32 + i];
            R[j * 32 + i] = t / R[j * 32 + j];
        }
    }
    // ||R||_F^2 and ||R^-1||_F^2 (R^-1 column by column, into the lower triangle's mirror)
    double fR = 0, fRi = 0;
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i <= j; ++i) fR += R[i * 32 + j] * R[i * 32 + j];
        double col[32];
        for (int i = j; i >= 0; --i) {
            double t = (i == j) ? 1.0 : 0.0;
            for (int k = i + 1; k <= j; ++k) t -= R[i * 32 + k] * col[k];
            col[i] = t / R[i * 32 + i];
            fRi += col[i] * col[i];
        }
    }
    const double u = 0x1p-53;
    const double g1 = (n + 1) * u / (1 - (n + 1) * u), g2 = n * u / (1 - n * u);
    const double C = 2.0 * fR * fRi;
    if (!(g1 * C < 1e-6)) return MU0_ILLCOND;
    const double shrink = 1.0 / (1.0 - g1 * C) * (1.0 + 1e-12);
    double rad = (double)best * shrink;
    int64_t y[32], lo[32], hi[32];
    double rem[33], aoff[32];
    for (int k = 0; k < n; ++k) y[k] = 0;
    rem[n] = rad;
    long long nodes = 0;
    int i = n - 1;
    bool le0 = false;
    // enter level i: its candidate range from the centre and the room left
    auto enter = [&](int ii) -> bool {
        double o = 0, a = 0;
        for (int j = ii + 1; j < n; ++j) { const double t = R[ii * 32 + j] * (double)y[j]; o += t; a += fabs(t); }
        const double rii = R[ii * 32 + ii];
        const double ctr = -o / rii, wd = sqrt(fmax(rem[ii + 1], 0.0)) / rii;
        // rounding of the centre and width, as a multiple of a coordinate step: must stay below 1/2
        const double e = g2 * (fabs(ctr) + wd + 1.0 + a / rii) * 4.0 + 4.0 * u * (fabs(ctr) + wd);
        if (!(e < 0.5) || !(fabs(ctr) + wd < 1e15)) return false;
        lo[ii] = (int64_t)floor(ctr - wd) - 1;
        hi[ii] = (int64_t)ceil(ctr + wd) + 1;
        aoff[ii] = a;
        y[ii] = lo[ii];
        return true;
    };
    if (!enter(i)) return MU0_ILLCOND;
    for (;;) {
        if (++nodes > budget) return MU0_BUDGET;
        if (y[i] > hi[i]) {                                         // level done
            y[i] = 0;
            if (++i == n) break;
            y[i]++;
            continue;
        }
        double o = 0;
        for (int j = i + 1; j < n; ++j) o += R[i * 32 + j] * (double)y[j];
        const double t = R[i * 32 + i] * (double)y[i] + o;
        const double a = fabs(R[i * 32 + i] * (double)y[i]) + aoff[i];
        const double lb = fmax(fabs(t) - g2 * a, 0.0) * (1.0 - 4.0 * u);
        const double r = rem[i + 1] - lb * lb * (1.0 - 4.0 * u);
        if (r < 0) { y[i]++; continue; }                           // (rigorously) too long
        if (i > 0) {
            rem[i] = r;
            --i;
            if (!enter(i)) return MU0_ILLCOND;
            continue;
        }
        bool nz = false;
        for (int j = 0; j < n; ++j) nz |= y[j] != 0;
        if (nz) {                                                   // exact y^T G y
            i128 q = 0, tt, rr;
            bool ovf = false;
            for (int a2 = 0; a2 < n && !ovf; ++a2) {
                if (!y[a2]) continue;
                rr = 0;
                for (int b = 0; b < n; ++b)
                    if (y[b] && (mul_ovf((i128)G[a2 * 32 + b], (i128)y[b], &tt) || add_ovf(rr, tt, &rr))) ovf = true;
                if (mul_ovf(rr, (i128)y[a2], &tt) || add_ovf(q, tt, &q)) ovf = true;
            }
            if (ovf) return MU0_OVF_LEAF;
            if (q <= 0) le0 = true;
            else if (q < (i128)best) {
                best = (int64_t)q;
                for (int j = 0; j < n; ++j) ybest[j] = y[j];
                rad = (double)best * shrink;                        // tighten
                rem[n] = rad;
            }
        }
        y[i]++;
    }
    return le0 ? MU0_NONE : MU0_OK;
}

// mu0 of direction k (warp-collective)
__device__ int mu0_direction(const Mu0Args &P, int k, Mu0Scratch *W, int lane, int64_t &num, int64_t &den, int64_t *Kout)
{
    const int h = P.h, m = h - 1, n = h - 2, w = m + n + 1;
    const int64_t *kap = P.kappa, *pr = P.pr + (int64_t)k * m;
    bool bad = false;
    i128 my_a00 = 0;
    // 1. A_rr, a_r0 into M; a00 kept (lane 0 computes it: entry e = 0)
    for (int e = lane; e < h * h; e += 32) {
        const int a = e / h, b = e % h;
        if (a < b) continue;                                        // (symmetric: the lower triangle)
        i128 s = 0;
        for (int c = 1; c < h; ++c)
            if (add_ovf(s, (i128)kap[(a * h + b) * h + c] * pr[c - 1], &s)) bad = true;
        if (!fits64(s)) bad = true;
        const int64_t v = (int64_t)s;
        if (a >= 1 && b >= 1) { W->M[(a - 1) * 64 + (b - 1)] = v; W->M[(b - 1) * 64 + (a - 1)] = v; }
        if (a >= 1 && b == 0) W->M[(a - 1) * 64 + m + n] = v;      // a_r0
        if (a == 0 && b == 0) my_a00 = v;
    }
    __syncwarp();
    if (warp_any(bad)) return MU0_OVF_A;
    i128 a00;                                                       // (lane 0's value)
    {
        const long long lo = __shfl_sync(FULL, (long long)(uint64_t)my_a00, 0);
        const long long hi = __shfl_sync(FULL, (long long)(my_a00 >> 64), 0);
        a00 = (i128)(((u128)(uint64_t)hi << 64) | (uint64_t)lo);
    }
    // the original a_r0 (the elimination overwrites its column): lane i keeps entry i (m <= 31)
    int64_t ar0 = 0;
    if (lane < m) ar0 = (int64_t)W->M[lane * 64 + m + n];
    // Lambda: rows 1..m-1 of U with U p_r = (g, 0, ..)
    if (warp_unimodular(pr, m, W->U, W->w, W->perm, lane)) return MU0_ORTH;
    for (int e = lane; e < m * n; e += 32) {
        const int i = e / n, a = e % n;
        W->M[i * 64 + m + a] = W->U[(a + 1) * MH + i];              // O^T
    }
    __syncwarp();
    // 2. Bareiss: lower part eliminated, pivots on the diagonal
    i128 prev = 1;
    for (int kk = 0; kk < m; ++kk) {
        int piv = -1;
        for (int r = kk; r < m; ++r) if (W->M[r * 64 + kk] != 0) { piv = r; break; }
        __syncwarp();                                               // (every lane has read column kk)
        if (piv < 0) return MU0_NONE;                               // A_rr singular
        if (piv != kk) {
            for (int j = lane; j < w; j += 32) {
                const i128 t = W->M[kk * 64 + j];
                W->M[kk * 64 + j] = W->M[piv * 64 + j];
                W->M[piv * 64 + j] = t;
            }
            __syncwarp();
        }
        const i128 pk = W->M[kk * 64 + kk];
        const int rows = m - kk - 1, cols = w - kk - 1;
        const ExactDiv dv = exact_div(prev);
        for (int e = lane; e < rows * cols; e += 32) {
            const int i = kk + 1 + e / cols, j = kk + 1 + e % cols;
            W256 dlt;
            i128 q;
            // (the division is exact: Bareiss entries are minors; a quotient beyond int128 fails here)
            if (w_sub(w_mul(pk, W->M[i * 64 + j]), w_mul(W->M[i * 64 + kk], W->M[kk * 64 + j]), &dlt) ||
                exact_quot(dlt, dv, &q)) { bad = true; continue; }
            W->M[i * 64 + j] = q;
        }
        __syncwarp();
        if (warp_any(bad)) return MU0_OVF_SOLVE;
        for (int i = kk + 1 + lane; i < m; i += 32) W->M[i * 64 + kk] = 0;
        prev = pk;
        __syncwarp();
    }
    const i128 d = W->M[(m - 1) * 64 + (m - 1)];
    // X[:, c] = d A_rr^-1 rhs_c by back substitution (lanes own columns c)
    for (int i = m - 1; i >= 0; --i) {
        const ExactDiv dv = exact_div(W->M[i * 64 + i]);
        for (int c = lane; c <= n; c += 32) {
            W256 s = w_mul(d, W->M[i * 64 + m + c]);
            for (int j = i + 1; j < m; ++j)
                if (w_sub(s, w_mul(W->M[i * 64 + j], W->X[j * 32 + c]), &s)) { bad = true; break; }
            i128 q;
            if (exact_quot(s, dv, &q)) { bad = true; continue; }
            W->X[i * 32 + c] = q;
        }
        __syncwarp();
        if (warp_any(bad)) return MU0_OVF_SOLVE;
    }
    // -s d = a_r0 . X[:, n] - d a00: s <= 0 needs it 0 or of d's sign (in 256 bits: every
    // product is below 2^190 and there are at most 32 terms)
    i128 t;
    W256 part = lane < m ? w_mul((i128)ar0, W->X[lane * 32 + n]) : w256(0);
    for (int o = 16; o; o >>= 1) {
        W256 other;
        for (int q = 0; q < 4; ++q) other.w[q] = __shfl_xor_sync(FULL, part.w[q], o);
        w_add(part, other, &part);
    }
    W256 sn;
    w_sub(part, w_mul(d, a00), &sn);
    if (!w_is_zero(sn) && (w_neg_sign(sn) != (d < 0))) return MU0_NONE;          // s > 0
    // G_n = -O X[:, :n], g = gcd(|d|, G_n), G = G_n / g sign(d), L = |d| / g
    u128 g = uabs(d);
    for (int e = lane; e < n * n; e += 32) {
        const int a = e / n, b = e % n;
        W256 s = w256(0);
        for (int i = 0; i < m; ++i) {
            const int64_t oai = W->U[(a + 1) * MH + i];
            if (oai && w_sub(s, w_mul((i128)oai, W->X[i * 32 + b]), &s)) bad = true;
        }
        if (!w_fits128(s)) bad = true;
        W->M[a * 64 + b] = w_lo(s);                                 // (M's storage reused for G_n)
        g = gcd128(g, uabs(w_lo(s)));
    }
    if (warp_any(bad)) return MU0_OVF_SOLVE;
    for (int o = 16; o; o >>= 1) g = gcd128(g, (u128)shfl_xor_i128((i128)g, o));
    __syncwarp();
    const i128 L = (i128)(uabs(d) / g);
    if (!fits64(L)) return MU0_OVF_GRAM;
    for (int e = lane; e < n * n; e += 32) {
        const int a = e / n, b = e % n;
        const i128 v = (i128)((u128)uabs(W->M[a * 64 + b]) / g) * ((W->M[a * 64 + b] < 0) != (d < 0) ? -1 : 1);
        if (!fits64(v)) bad = true;
        W->Gr[a * 32 + b] = (int64_t)v;
    }
    __syncwarp();
    if (warp_any(bad)) return MU0_OVF_GRAM;
    for (int a = 0; a < n; ++a) if (W->Gr[a * 32 + a] <= 0) return MU0_NONE;      // not positive definite
    // 3. LLL of the identity basis w.r.t. G (exact Gram in the working set)
    LllMem<32> *S = &W->L;
    for (int e = lane; e < n * 32; e += 32) S->B[(e / 32) * 32 + e % 32] = (e / 32) == (e % 32) ? 1 : 0;
    for (int e = lane; e < n * n; e += 32) {
        const int a = e / n, b = e % n;
        if (b <= a) S->G[gix(a, b)] = (i128)W->Gr[a * 32 + b];
    }
    __syncwarp();
    if (n > 1) {
        Lll<32> LK{S, n, n};
        const int st = warp_lll(LK, n, false, 0.99, lane);
        if (st == ST_NONPOS) {
            // a non-positive norm under G: not positive definite when a witness says so (on
            // a compact n x n copy of G in U's storage; U is not needed on this path)
            for (int e = lane; e < n * n; e += 32) W->U[e] = W->Gr[(e / n) * 32 + e % n];
            __syncwarp();
            return witness_not_pd(W->U, n, W->R, W->R + n * n, lane) ? MU0_NONE : MU0_LLL;
        }
        if (st) return MU0_LLL;
    }
    for (int e = lane; e < n * n; e += 32) {
        const int a = e / n, b = e % n;
        const i128 v = S->G[gix(a, b)];
        if (!fits64(v)) bad = true;
        W->Gr[a * 32 + b] = (int64_t)v;
    }
    __syncwarp();
    if (warp_any(bad)) return MU0_OVF_GRAM;
    // the minimum, from the smallest basis vector
    int st = 0;
    int64_t best = 0, y[32];
    if (lane == 0) {
        int i0 = 0;
        for (int a = 1; a < n; ++a) if (W->Gr[a * 32 + a] < W->Gr[i0 * 32 + i0]) i0 = a;
        best = W->Gr[i0 * 32 + i0];
        for (int a = 0; a < n; ++a) y[a] = a == i0;
        st = mu0_min(W->Gr, W->R, n, best, y, P.node_budget);
        for (int a = 0; a < n; ++a) W->w[a] = y[a];
    }
    st = __shfl_sync(FULL, st, 0);
    best = __shfl_sync(FULL, best, 0);
    __syncwarp();
    if (st) return st;
    // 4. K = O^T V^T y (lanes own K's entries)
    for (int i = lane; i < m; i += 32) {
        i128 s = 0;
        for (int a = 0; a < n; ++a) {
            i128 z = 0;
            for (int b = 0; b < n; ++b)
                if (W->w[b] && (mul_ovf((i128)S->B[b * 32 + a], (i128)W->w[b], &t) || add_ovf(z, t, &z))) bad = true;
            const int64_t oai = W->U[(a + 1) * MH + i];
            if (oai && (mul_ovf((i128)oai, z, &t) || add_ovf(s, t, &s))) bad = true;
        }
        if (!fits64(s)) bad = true;
        Kout[i] = (int64_t)s;
    }
    if (warp_any(bad)) return MU0_OVF_GRAM;
    const uint64_t gg = gcd64((uint64_t)best, (uint64_t)L);
    num = best / (int64_t)gg;
    den = (int64_t)L / (int64_t)gg;
    return MU0_OK;
}

// One warp per direction, taken from a work counter.
__global__ void __launch_bounds__(128) k_mu0(Mu0Args P)
{
    const int lane = threadIdx.x & 31;
    Mu0Scratch *W = P.scratch + (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5));
    if (lane == 0) W->L.B = W->Lb;
    __syncwarp();
    for (;;) {
        unsigned t = 0;
        if (lane == 0) t = atomicAdd(P.next, 1u);
        t = __shfl_sync(FULL, t, 0);
        if (t >= (unsigned)P.n_p) break;
        int64_t num = 0, den = 0;
        const int st = P.h < 3 || P.h > MU0_MAXH ? (int)MU0_RANGE
                       : mu0_direction(P, (int)t, W, lane, num, den, P.K + (int64_t)t * (P.h - 1));
        if (lane == 0) {
            P.status[t] = st;
            P.mu_num[t] = st == 0 ? num : 0;
            P.mu_den[t] = st == 0 ? den : 0;
        }
        __syncwarp();
    }
}

}  // namespace pfg
