// coniZpK above D0 on the device, one warp per direction: the lattice points
// of every coni PFV whose dilation exceeds D0 (the reference computes this on
// the CPU: pfvs/fp_kernel/coni_zpk.h:267-714, called through coniZpK,
// pfvs/coni.py:554-637).  ZpM at ellipsoid dilation D0 finds the PFVs with
// dilation <= D0, so the two together are exhaustive.
//
// For p_hat = (0, p_r), A = kappa . p_hat, S = -A_rr^-1, -s = sn / sd and
// Lambda = {K in Z^m : p_r . K = 0} (m = h11 - 1, rank n = m - 1), a PFV with
// p = p_hat / delta has K_r in Lambda and tadpole
//
//     Q = M0 eps + (M0^2 / delta)(-s) + delta K_r^T S K_r,   eps > 0,
//
// so delta > D0 forces K_r^T S K_r < Q / D0: K_r is one of finitely many
// short vectors of Lambda.  With W = (Z Binter)_r (the rows 1.. of Z Binter)
// and Gamma = W Z^m, a short K_r = g K' (K' primitive, o its order in
// Lambda / Gamma) comes from the points c = j c1 + t kv (W c1 = o K', kv
// spanning ker W) with delta = j o / g; delta > D0 is j o > g D0, the tadpole
//
//     g L sn M0^2 < sd j o (Q L - g j o kn),   kn = L K'^T S K' (an integer),
//
// and M0 = l . c >= M0min (l = Binter row 0): a range of j and, for each j, an
// arithmetic progression of M0 (so of t).
//
// Steps (exact integers throughout; floating point only prunes the search,
// by a proven margin, and screens j with a wide one):
//   1. Z, the M-lattice basis Binter orthogonal to p.Z (a unimodular
//      transform of v = (Z p)^T Mbasis, its rows 1.. LLL-reduced), Z Binter.
//   2. A basis O of Lambda (rows 1.. of a unimodular U with U p_r = (g, 0, ..))
//      and U^-1 (a fraction-free elimination of [U | I]).
//   3. Bareiss elimination of [A_rr | O^T | a_r0]: -s = sn / sd and the form
//      of S on O's basis, G / L (as the dilation bound's kernel, pfg_mu0.cuh),
//      LLL-reduced: Gr = V G V^T.
//   4. The Lambda coordinates Y of W's columns, the Hermite normal form of [Y^T | I]
//      by unimodular row operations: [H | E] over [0 | kv^T], H upper
//      triangular (Gamma's basis in Lambda coordinates), kv spanning ker W;
//      Hdet = det H, Hadj = Hdet H^-T, Cs / Cden solving W c1 = v for v in
//      Gamma, HT = Hadj V^T, w = l Cs O^T V^T, lk = l . kv.
//   5. Every x != 0 with x^T Gr x D0 < Q L by depth-first walks, one per lane
//      (the nodes two levels below the top dealt to the lanes in turn), with
//      exact partial sums (Gr x, HT x, w . x, x^T Gr x) carried down the
//      levels; per short x the (j, M0) ranges above and the points, emitted
//      with M = Binter c, Kn = Z Binter c, q = c^T mat c = -M . Kn.
//
// Any basis of the M-lattice and of Lambda gives the same points (M, Kn, q):
// they are fixed by the PFVs, not by the coordinates, so the bases here need
// not be the reference's.
//
// Status (the reference's codes where it has the same failure): 0 done; 1 no
// ZpK for this direction (s >= 0, A_rr singular, S not positive definite on
// Lambda); < 0 not decided here (an exact value beyond int128 or int64, an
// ill-conditioned form, more than max_out points, the node budget): the
// caller searches the direction another way (ZpM up to its dilation bound).
#pragma once
#include "pfg_mu0.cuh"

namespace pfg {

constexpr int ZPK_MAXH = 32;

enum ZpkStatus {
    ZPK_OK = 0, ZPK_NONE = 1,
    ZPK_RANGE = -20, ZPK_LATTICE = -31, ZPK_ORTH = -32,
    ZPK_UNIMOD = -40, ZPK_OVF_Y = -41, ZPK_NOT_IN = -42, ZPK_OVF_HNF = -43, ZPK_RANK = -44,
    ZPK_OVF_H = -45, ZPK_INEXACT = -46,
    ZPK_OVF_SOLVE = -50, ZPK_OVF_S = -52, ZPK_LLL = -60, ZPK_OVF_GR = -61,
    ZPK_OVF_HT = -70, ZPK_LK0 = -71,
    ZPK_MAX_OUT = -80, ZPK_OVF_POINT = -82, ZPK_OVF_K = -90, ZPK_INEXACT_K = -91,
    ZPK_ARGS = -100, ZPK_OVF_QL = -101, ZPK_CHOL = -102, ZPK_ILLCOND = -103, ZPK_ENTER = -104,
    ZPK_COORD = -105, ZPK_BUDGET = -106
};

struct ZpkScratch {
    int64_t Z[32 * 32];                       // kappa . p_hat (h x h)
    int64_t Bi[32 * 32];                      // Binter (h x m): M = Binter c
    int64_t ZB[32 * 32];                      // Z Binter (h x m)
    int64_t U[32 * MH];                       // unimodular transforms (rows, stride MH)
    int64_t w[MH];
    int perm[MH];
    i128 M[31 * 64];                          // elimination workspace (stride 64)
    i128 X[31 * 32];                          // solutions (stride 32)
    i128 Ui[31 * 32];                         // U^-1 (m x m)
    i128 A[31 * 64];                          // [Y^T | I] -> [H | E ; 0 | kv^T] (stride 64)
    i128 Hadj[30 * 32];                       // Hdet H^-T (lower triangular)
    i128 HP[30 * 32];                         // Hadj Y(v) rows: (n x m)
    i128 lC[32];                              // l Cs, then l Cs O^T
    int64_t Cs[31 * 32];                      // (m x m)
    int64_t kv[32];
    int64_t Gr[32 * 32];                      // the reduced form (n x n)
    int64_t HT[32 * 32];                      // Hadj V^T (n x n)
    int64_t wv[32];                           // l Cs O^T V^T
    double R[32 * 32];                        // FP64 Cholesky factor of Gr
    // the search, one walk per lane: state interleaved by lane ([..][lane])
    i128 gx[31 * 32 * 32], hx[31 * 32 * 32];  // exact partial sums per level: Gr x, HT x
    i128 wx[32 * 32], vals[32 * 32];          // w . x, x^T Gr x per level
    int64_t x[32 * 32], lo[32 * 32], hi[32 * 32];
    double rem[32 * 32], aoff[32 * 32], ofs[32 * 32];
    i128 c1[32 * 32];                         // c1 of the lane's current short vector
    double rad, g2;                           // the search radius, the dot products' rounding factor
    i128 QL;                                  // Q L
    unsigned long long nout;                  // points of the direction so far
    int abort;                                // a lane ended with an error: the others stop
    LllMem<32> L;                             // LLL working set
    int64_t Lb[31 * 32];                      // its rows
};

struct ZpkArgs {
    int h;
    const int64_t *kappa;                     // h^3
    const int64_t *Mbasis;                    // h^2
    const int64_t *ps;                        // (n_p, ps_stride >= h), p[0] = 0 in the first h
    int ps_stride;
    int n_p;
    int64_t Q, M0min, D0, max_out;
    unsigned *next;                           // work counter
    ZpkScratch *scratch;                      // one per warp
    int32_t *status;                          // (n_p,)
    unsigned long long *count;                // points emitted (all directions; may exceed cap)
    unsigned long long cap;                   // rows the output arrays hold
    int64_t *M, *Kn, *q, *pidx;               // rows of MH (first h entries), (cap,)
    long long budget;                         // search nodes + (j, M0) steps per lane and direction
};

// int128 quotient (truncated, as C) and remainder, on the 64-bit path when both
// operands fit (the common case here; the 128-bit division is a long software routine)
__device__ __forceinline__ i128 q128(i128 a, i128 b)
{
    return fits64(a) && fits64(b) ? (i128)((int64_t)a / (int64_t)b) : a / b;
}
__device__ __forceinline__ i128 r128(i128 a, i128 b)
{
    return fits64(a) && fits64(b) ? (i128)((int64_t)a % (int64_t)b) : a % b;
}
__device__ __forceinline__ i128 fdivq(i128 a, i128 b)
{
    return fits64(a) && fits64(b) ? (i128)fdiv64((int64_t)a, (int64_t)b) : fdiv128(a, b);
}

// a b + c into *r; true on overflow
__device__ __forceinline__ bool muladd_ovf(i128 a, i128 b, i128 c, i128 *r)
{
    i128 p;
    return mul_ovf(a, b, &p) || add_ovf(c, p, r);
}

// Fraction-free elimination of the m x w matrix M (stride 64; its first m
// columns the square system), then X = d M_sq^-1 M_rhs (the w - m right-hand
// sides, stride 32) by exact back substitution, d the last pivot (+-det).
// Products in 256 bits, each quotient checked exact and within int128.
// Returns 0, 1 (singular) or -1 (a value beyond int128).  Warp-collective.
__device__ int zpk_solve(i128 *M, int m, int w, i128 *X, i128 &d, int lane)
{
    bool bad = false;
    i128 prev = 1;
    for (int k = 0; k < m; ++k) {
        int piv = -1;
        for (int r = k; r < m; ++r) if (M[r * 64 + k] != 0) { piv = r; break; }
        __syncwarp();
        if (piv < 0) return 1;
        if (piv != k) {
            for (int j = lane; j < w; j += 32) {
                const i128 t = M[k * 64 + j];
                M[k * 64 + j] = M[piv * 64 + j];
                M[piv * 64 + j] = t;
            }
            __syncwarp();
        }
        const i128 pk = M[k * 64 + k];
        const int rows = m - k - 1, cols = w - k - 1;
        const ExactDiv dv = exact_div(prev);
        for (int e = lane; e < rows * cols; e += 32) {
            const int i = k + 1 + e / cols, j = k + 1 + e % cols;
            W256 dlt;
            i128 q;
            if (w_sub(w_mul(pk, M[i * 64 + j]), w_mul(M[i * 64 + k], M[k * 64 + j]), &dlt) ||
                exact_quot(dlt, dv, &q)) { bad = true; continue; }
            M[i * 64 + j] = q;
        }
        __syncwarp();
        if (warp_any(bad)) return -1;
        for (int i = k + 1 + lane; i < m; i += 32) M[i * 64 + k] = 0;
        prev = pk;
        __syncwarp();
    }
    d = M[(m - 1) * 64 + (m - 1)];
    const int nr = w - m;
    for (int i = m - 1; i >= 0; --i) {
        const ExactDiv dv = exact_div(M[i * 64 + i]);
        for (int c = lane; c < nr; c += 32) {
            W256 s = w_mul(d, M[i * 64 + m + c]);
            for (int j = i + 1; j < m; ++j)
                if (w_sub(s, w_mul(M[i * 64 + j], X[j * 32 + c]), &s)) { bad = true; break; }
            i128 q;
            if (exact_quot(s, dv, &q)) { bad = true; continue; }
            X[i * 32 + c] = q;
        }
        __syncwarp();
        if (warp_any(bad)) return -1;
    }
    return 0;
}

// row i -= q row r over the columns c0 .. w-1 of A (stride 64); true on overflow.  Warp-collective.
__device__ __forceinline__ bool zpk_rowsub(i128 *A, int i, int r, i128 q, int c0, int w, int lane)
{
    bool bad = false;
    for (int j = c0 + lane; j < w; j += 32) {
        i128 pr;
        if (mul_ovf(q, A[r * 64 + j], &pr) || sub_ovf(A[i * 64 + j], pr, &A[i * 64 + j])) bad = true;
    }
    __syncwarp();
    return warp_any(bad);
}

// The Hermite normal form of the m x w matrix A (stride 64) by unimodular row
// operations.  Column by column, the rows not yet pivoted are reduced by the
// one with the smallest nonzero entry (nearest-integer quotients, so each
// round at least halves it) until a single nonzero is left; that pivot is
// made positive and the rows above are reduced modulo it.  Returns the rank,
// or -1 on overflow.  Warp-collective (every lane takes the same decisions).
__device__ int zpk_hnf(i128 *A, int m, int w, int lane)
{
    int r = 0;
    for (int c = 0; c < w && r < m; ++c) {
        bool pivot = false;
        for (int it = 0;; ++it) {
            if (it > 256) return -1;                                   // (each round halves the pivot)
            int p = -1;
            u128 best = 0;
            for (int i = r; i < m; ++i) {
                const i128 v = A[i * 64 + c];
                if (v != 0 && (p < 0 || uabs(v) < best)) { p = i; best = uabs(v); }
            }
            __syncwarp();
            if (p < 0) break;
            pivot = true;
            if (p != r) {
                for (int j = c + lane; j < w; j += 32) {
                    const i128 t = A[r * 64 + j];
                    A[r * 64 + j] = A[p * 64 + j];
                    A[p * 64 + j] = t;
                }
                __syncwarp();
            }
            const i128 pv = A[r * 64 + c];
            bool more = false;
            for (int i = r + 1; i < m; ++i) {
                const i128 v = A[i * 64 + c];
                __syncwarp();
                if (v == 0) continue;
                i128 q = fdiv128(v, pv);
                if (uabs(v - q * pv) > uabs(pv) / 2) q += 1;               // the nearest quotient
                if (q && zpk_rowsub(A, i, r, q, c, w, lane)) return -1;
                more |= A[i * 64 + c] != 0;
            }
            if (!more) break;
        }
        if (!pivot) continue;
        if (A[r * 64 + c] < 0) {
            __syncwarp();
            for (int j = c + lane; j < w; j += 32) A[r * 64 + j] = -A[r * 64 + j];
        }
        __syncwarp();
        for (int i = 0; i < r; ++i) {
            const i128 q = fdiv128(A[i * 64 + c], A[r * 64 + c]);
            __syncwarp();
            if (q && zpk_rowsub(A, i, r, q, c, w, lane)) return -1;
        }
        ++r;
    }
    return r;
}

// the scalars of one direction's setup
struct ZpkDir { int64_t Hdet, Cden, L, sn, sd, lk; };

// Steps 1-4 of direction k (warp-collective): the scratch then holds Bi, ZB,
// U (rows 1.. a basis O of Lambda), L.B (the LLL transform V), Gr, HT, wv,
// Cs, kv, and D the scalars.
__device__ int zpk_setup(const ZpkArgs &P, int k, ZpkScratch *W, ZpkDir &D, int lane)
{
    const int h = P.h, m = h - 1, n = h - 2;
    const int64_t *kap = P.kappa, *Mb = P.Mbasis, *p = P.ps + (int64_t)k * P.ps_stride;
    bool bad = false;
    // 1. Z = kappa . p, T = Z p (into x), v = T^T Mbasis (into wv)
    for (int e = lane; e < h * h; e += 32) {
        const int a = e / h, b = e % h;
        i128 s = 0;
        for (int c = 0; c < h; ++c)
            if (p[c] && muladd_ovf((i128)kap[(a * h + b) * h + c], (i128)p[c], s, &s)) bad = true;
        if (!fits64(s)) bad = true;
        W->Z[a * 32 + b] = (int64_t)s;
    }
    __syncwarp();
    if (warp_any(bad)) return ZPK_LATTICE;
    if (lane < h) {
        i128 s = 0;
        for (int j = 0; j < h; ++j)
            if (p[j] && muladd_ovf((i128)W->Z[lane * 32 + j], (i128)p[j], s, &s)) bad = true;
        if (!fits64(s)) bad = true;
        W->x[lane] = (int64_t)s;
    }
    __syncwarp();
    if (warp_any(bad)) return ZPK_LATTICE;
    if (lane < h) {
        i128 s = 0;
        for (int i = 0; i < h; ++i)
            if (muladd_ovf((i128)W->x[i], (i128)Mb[i * h + lane], s, &s)) bad = true;
        if (!fits64(s)) bad = true;
        W->wv[lane] = (int64_t)s;
    }
    __syncwarp();
    if (warp_any(bad)) return ZPK_LATTICE;
    // the M-lattice vectors orthogonal to v: rows 1.. of a unimodular transform, LLL-reduced
    if (warp_unimodular(W->wv, h, W->U, W->w, W->perm, lane)) return ZPK_ORTH;
    LllMem<32> *S = &W->L;
    for (int e = lane; e < m * 32; e += 32) {
        const int a = e / 32, c = e % 32;
        S->B[a * 32 + c] = c < h ? W->U[(a + 1) * MH + c] : 0;
    }
    __syncwarp();
    if (gram_euclid<32>(S, m, h, lane)) return ZPK_ORTH;
    {
        Lll<32> LL{S, h, m};
        if (warp_lll(LL, m, false, 0.99, lane)) return ZPK_ORTH;
    }
    for (int e = lane; e < h * m; e += 32) {
        const int i = e / m, a = e % m;
        i128 s = 0;
        for (int l = 0; l < h; ++l)
            if (S->B[a * 32 + l] && muladd_ovf((i128)Mb[i * h + l], (i128)S->B[a * 32 + l], s, &s)) bad = true;
        if (!fits64(s)) bad = true;
        W->Bi[i * 32 + a] = (int64_t)s;
    }
    __syncwarp();
    if (warp_any(bad)) return ZPK_LATTICE;
    for (int e = lane; e < h * m; e += 32) {
        const int i = e / m, a = e % m;
        i128 s = 0;
        for (int j = 0; j < h; ++j)
            if (W->Z[i * 32 + j] && muladd_ovf((i128)W->Z[i * 32 + j], (i128)W->Bi[j * 32 + a], s, &s)) bad = true;
        if (!fits64(s)) bad = true;
        W->ZB[i * 32 + a] = (int64_t)s;
    }
    __syncwarp();
    if (warp_any(bad)) return ZPK_LATTICE;

    // 2. Lambda: rows 1.. of U with U p_r = (g, 0, ..); U^-1 from [U | I]
    if (warp_unimodular(p + 1, m, W->U, W->w, W->perm, lane)) return ZPK_UNIMOD;
    for (int e = lane; e < m * 2 * m; e += 32) {
        const int i = e / (2 * m), j = e % (2 * m);
        W->M[i * 64 + j] = j < m ? (i128)W->U[i * MH + j] : (i128)(j - m == i);
    }
    __syncwarp();
    i128 d;
    if (zpk_solve(W->M, m, 2 * m, W->X, d, lane) || (d != 1 && d != -1)) return ZPK_UNIMOD;
    for (int e = lane; e < m * m; e += 32) {
        const int i = e / m, j = e % m;
        W->Ui[i * 32 + j] = d == 1 ? W->X[i * 32 + j] : -W->X[i * 32 + j];
    }
    __syncwarp();

    // 3. [A_rr | O^T | a_r0]: X = d A_rr^-1 [O^T | a_r0]
    const int wa = m + n + 1;
    for (int e = lane; e < m * wa; e += 32) {
        const int i = e / wa, j = e % wa;
        int64_t v;
        if (j < m) v = W->Z[(i + 1) * 32 + j + 1];
        else if (j < m + n) v = W->U[(j - m + 1) * MH + i];
        else v = W->Z[(i + 1) * 32];
        W->M[i * 64 + j] = v;
    }
    __syncwarp();
    {
        const int rc = zpk_solve(W->M, m, wa, W->X, d, lane);
        if (rc) return rc > 0 ? ZPK_NONE : ZPK_OVF_SOLVE;
    }
    // -s = sn / sd: sn = a_r0 . X[:, n] - d a00 over sd = d (products below 2^190, at most 31 terms)
    W256 part = lane < m ? w_mul((i128)W->Z[(lane + 1) * 32], W->X[lane * 32 + n]) : w256(0);
    for (int o = 16; o; o >>= 1) {
        W256 other;
        for (int qq = 0; qq < 4; ++qq) other.w[qq] = __shfl_xor_sync(FULL, part.w[qq], o);
        w_add(part, other, &part);
    }
    W256 snw;
    w_sub(part, w_mul(d, (i128)W->Z[0]), &snw);
    if (!w_fits128(snw)) return ZPK_OVF_SOLVE;
    {
        i128 sn = w_lo(snw), sd = d;
        if (sd < 0) { sd = -sd; sn = -sn; }
        if (sn <= 0) return ZPK_NONE;                                  // s >= 0
        const i128 gs = (i128)gcd128(uabs(sn), uabs(sd));
        sn /= gs; sd /= gs;
        if (!fits64(sn) || !fits64(sd)) return ZPK_OVF_S;
        D.sn = (int64_t)sn; D.sd = (int64_t)sd;
    }
    // G_n = -O X[:, :n] (into M), g = gcd(|d|, G_n), Gi = G_n / g sign(d), L = |d| / g
    u128 g = uabs(d);
    for (int e = lane; e < n * n; e += 32) {
        const int a = e / n, b = e % n;
        W256 s = w256(0);
        for (int i = 0; i < m; ++i) {
            const int64_t oai = W->U[(a + 1) * MH + i];
            if (oai && w_sub(s, w_mul((i128)oai, W->X[i * 32 + b]), &s)) bad = true;
        }
        if (!w_fits128(s)) bad = true;
        W->M[a * 64 + b] = w_lo(s);
        g = gcd128(g, uabs(w_lo(s)));
    }
    if (warp_any(bad)) return ZPK_OVF_SOLVE;
    for (int o = 16; o; o >>= 1) g = gcd128(g, (u128)shfl_xor_i128((i128)g, o));
    __syncwarp();
    {
        const i128 L = (i128)(uabs(d) / g);
        if (!fits64(L)) return ZPK_OVF_S;
        D.L = (int64_t)L;
    }
    for (int e = lane; e < n * n; e += 32) {
        const int a = e / n, b = e % n;
        const i128 gn = W->M[a * 64 + b];
        const i128 v = (i128)(uabs(gn) / g) * ((gn < 0) != (d < 0) ? -1 : 1);
        if (!fits64(v)) bad = true;
        W->Gr[a * 32 + b] = (int64_t)v;
    }
    __syncwarp();
    if (warp_any(bad)) return ZPK_OVF_S;
    for (int a = 0; a < n; ++a) if (W->Gr[a * 32 + a] <= 0) return ZPK_NONE;      // not positive definite
    // LLL of the identity basis w.r.t. Gi: rows of V in L.B, Gr = V Gi V^T exactly in L.G
    for (int e = lane; e < n * 32; e += 32) S->B[e] = (e / 32) == (e % 32) ? 1 : 0;
    for (int e = lane; e < n * n; e += 32) {
        const int a = e / n, b = e % n;
        if (b <= a) S->G[gix(a, b)] = (i128)W->Gr[a * 32 + b];
    }
    __syncwarp();
    if (n > 1) {
        Lll<32> LK{S, n, n};
        const int st = warp_lll(LK, n, false, 0.99, lane);
        if (st == ST_NONPOS) {
            // a non-positive norm: not positive definite when a witness says so (a compact copy in HT)
            for (int e = lane; e < n * n; e += 32) W->HT[e] = W->Gr[(e / n) * 32 + e % n];
            __syncwarp();
            return witness_not_pd(W->HT, n, W->R, W->R + n * n, lane) ? ZPK_NONE : ZPK_LLL;
        }
        if (st) return ZPK_LLL;
    }
    for (int e = lane; e < n * n; e += 32) {
        const int a = e / n, b = e % n;
        const i128 v = S->G[gix(a, b)];
        if (!fits64(v)) bad = true;
        W->Gr[a * 32 + b] = (int64_t)v;
    }
    __syncwarp();
    if (warp_any(bad)) return ZPK_OVF_GR;

    // 4. Y^T: the Lambda coordinates (v^T U^-1)[1:] of W's columns v = ZB[1:, c], into
    // [Y^T | I] (coordinate 0 must vanish: W's columns lie in Lambda)
    const int wA = n + m;
    bool notin = false;
    for (int e = lane; e < m * (n + 1); e += 32) {
        const int c = e / (n + 1), j = e % (n + 1);
        i128 s = 0;
        for (int i = 0; i < m; ++i)
            if (W->ZB[(i + 1) * 32 + c] && muladd_ovf((i128)W->ZB[(i + 1) * 32 + c], W->Ui[i * 32 + j], s, &s)) bad = true;
        if (j == 0) notin |= s != 0;
        else W->A[c * 64 + j - 1] = s;
    }
    for (int e = lane; e < m * m; e += 32) W->A[(e / m) * 64 + n + e % m] = (i128)((e / m) == (e % m));
    __syncwarp();
    if (warp_any(bad)) return ZPK_OVF_Y;
    if (warp_any(notin)) return ZPK_NOT_IN;
    // its Hermite normal form: rows 0..n-1 pivot on the diagonal (Y has rank n), row n is
    // [0 | kv^T] with its pivot in the identity part
    if (zpk_hnf(W->A, m, wA, lane) != m) return ZPK_OVF_HNF;
    for (int r = 0; r < n; ++r) if (W->A[r * 64 + r] <= 0) return ZPK_RANK;
    for (int j = 0; j < n; ++j) if (W->A[n * 64 + j] != 0) return ZPK_RANK;
    for (int i = lane; i < m; i += 32) {
        const i128 v = W->A[n * 64 + n + i];
        if (!fits64(v)) bad = true;
        W->kv[i] = (int64_t)v;
    }
    __syncwarp();
    if (warp_any(bad)) return ZPK_OVF_H;
    // Hdet = det H; Hadj = Hdet H^-T (lower triangular) by exact forward substitution, lanes own columns
    i128 dH = 1;
    for (int i = 0; i < n; ++i) if (mul_ovf(dH, W->A[i * 64 + i], &dH)) return ZPK_OVF_H;
    if (!fits64(dH)) return ZPK_OVF_H;
    bool inexact = false;
    if (lane < n) {
        const int j = lane;
        for (int i = 0; i < n; ++i) {
            if (i < j) { W->Hadj[i * 32 + j] = 0; continue; }
            i128 s = i == j ? dH : 0;
            for (int kk = j; kk < i; ++kk) {
                i128 pr;
                if (mul_ovf(W->A[kk * 64 + i], W->Hadj[kk * 32 + j], &pr) || sub_ovf(s, pr, &s)) bad = true;
            }
            const i128 piv = W->A[i * 64 + i];
            if (s % piv) inexact = true;
            W->Hadj[i * 32 + j] = s / piv;
        }
    }
    __syncwarp();
    if (warp_any(bad)) return ZPK_OVF_H;
    if (warp_any(inexact)) return ZPK_INEXACT;
    // HP = Hadj Y(v) for the unit vectors v (Y(v)[b] = U^-1[v][b + 1]); Cn = E^T HP; Cs = Cn / gC
    for (int e = lane; e < n * m; e += 32) {
        const int a = e / m, j = e % m;
        i128 s = 0;
        for (int b = 0; b <= a; ++b)
            if (W->Hadj[a * 32 + b] && muladd_ovf(W->Hadj[a * 32 + b], W->Ui[j * 32 + b + 1], s, &s)) bad = true;
        W->HP[a * 32 + j] = s;
    }
    __syncwarp();
    if (warp_any(bad)) return ZPK_OVF_H;
    u128 gC = uabs(dH);
    for (int e = lane; e < m * m; e += 32) {
        const int i = e / m, j = e % m;
        i128 s = 0;
        for (int a = 0; a < n; ++a)
            if (W->A[a * 64 + n + i] && muladd_ovf(W->A[a * 64 + n + i], W->HP[a * 32 + j], s, &s)) bad = true;
        W->M[i * 64 + j] = s;
        gC = gcd128(gC, uabs(s));
    }
    if (warp_any(bad)) return ZPK_OVF_H;
    for (int o = 16; o; o >>= 1) gC = gcd128(gC, (u128)shfl_xor_i128((i128)gC, o));
    __syncwarp();
    for (int e = lane; e < m * m; e += 32) {
        const int i = e / m, j = e % m;
        const i128 v = W->M[i * 64 + j] / (i128)gC;
        if (!fits64(v)) bad = true;
        W->Cs[i * 32 + j] = (int64_t)v;
    }
    __syncwarp();
    if (warp_any(bad)) return ZPK_OVF_H;
    D.Hdet = (int64_t)dH;
    D.Cden = (int64_t)(dH / (i128)gC);
    // HT = Hadj V^T; w = l Cs O^T V^T (l = Binter row 0); lk = l . kv
    for (int e = lane; e < n * n; e += 32) {
        const int a = e / n, b = e % n;
        i128 s = 0;
        for (int j = 0; j <= a; ++j)
            if (S->B[b * 32 + j] && muladd_ovf(W->Hadj[a * 32 + j], (i128)S->B[b * 32 + j], s, &s)) bad = true;
        if (!fits64(s)) bad = true;
        W->HT[a * 32 + b] = (int64_t)s;
    }
    for (int j = lane; j < m; j += 32) {
        i128 s = 0;
        for (int i = 0; i < m; ++i)
            if (W->Bi[i] && muladd_ovf((i128)W->Bi[i], (i128)W->Cs[i * 32 + j], s, &s)) bad = true;
        W->lC[j] = s;
    }
    __syncwarp();
    if (warp_any(bad)) return ZPK_OVF_HT;
    for (int b = lane; b < n; b += 32) {
        i128 s = 0;
        for (int j = 0; j < m; ++j)
            if (W->U[(b + 1) * MH + j] && muladd_ovf(W->lC[j], (i128)W->U[(b + 1) * MH + j], s, &s)) bad = true;
        W->X[b] = s;
    }
    __syncwarp();
    if (warp_any(bad)) return ZPK_OVF_HT;
    for (int b = lane; b < n; b += 32) {
        i128 s = 0;
        for (int j = 0; j < n; ++j)
            if (S->B[b * 32 + j] && muladd_ovf(W->X[j], (i128)S->B[b * 32 + j], s, &s)) bad = true;
        if (!fits64(s)) bad = true;
        W->wv[b] = (int64_t)s;
    }
    __syncwarp();
    if (warp_any(bad)) return ZPK_OVF_HT;
    i128 lk = 0;
    for (int i = 0; i < m; ++i)
        if (muladd_ovf((i128)W->Bi[i], (i128)W->kv[i], lk, &lk)) return ZPK_OVF_HT;
    if (!fits64(lk)) return ZPK_OVF_HT;
    if (lk == 0) return ZPK_LK0;                                       // (M0 independent of t)
    D.lk = (int64_t)lk;
    return ZPK_OK;
}

// one point c = j c1 + t kv: M = Binter c, Kn = Z Binter c, q = -M . Kn (one lane)
__device__ int zpk_emit(const ZpkArgs &P, int k, ZpkScratch *W, i128 j, i128 t, int lane)
{
    const int h = P.h, m = h - 1;
    int64_t c[32], Mr[32], Kr[32];
    for (int i = 0; i < m; ++i) {
        i128 s;
        if (mul_ovf(j, W->c1[(i << 5) + lane], &s) || muladd_ovf(t, (i128)W->kv[i], s, &s) || !fits64(s))
            return ZPK_OVF_POINT;
        c[i] = (int64_t)s;
    }
    i128 mk = 0;
    for (int i = 0; i < h; ++i) {
        i128 a = 0, b = 0;
        for (int l = 0; l < m; ++l) {
            if (!c[l]) continue;
            if (muladd_ovf((i128)W->Bi[i * 32 + l], (i128)c[l], a, &a) ||
                muladd_ovf((i128)W->ZB[i * 32 + l], (i128)c[l], b, &b)) return ZPK_OVF_POINT;
        }
        if (!fits64(a) || !fits64(b)) return ZPK_OVF_POINT;
        Mr[i] = (int64_t)a;
        Kr[i] = (int64_t)b;
        if (add_ovf(mk, (i128)Mr[i] * (i128)Kr[i], &mk)) return ZPK_OVF_POINT;
    }
    if (!fits64(-mk)) return ZPK_OVF_POINT;
    if (atomicAdd(&W->nout, 1ull) >= (unsigned long long)P.max_out) return ZPK_MAX_OUT;
    const unsigned long long slot = atomicAdd(P.count, 1ull);
    if (slot < P.cap) {
        for (int i = 0; i < MH; ++i) {
            P.M[slot * MH + i] = i < h ? Mr[i] : 0;
            P.Kn[slot * MH + i] = i < h ? Kr[i] : 0;
        }
        P.q[slot] = (int64_t)(-mk);
        P.pidx[slot] = k;
    }
    return ZPK_OK;
}

// the points of the lane's short vector x (level-0 sums hx = HT x, wx = w . x; val = x^T Gr x)
__device__ int zpk_per_short(const ZpkArgs &P, int k, ZpkScratch *W, const ZpkDir &D, i128 val, long long &steps,
                             int lane)
{
    const int n = P.h - 2, m = P.h - 1;
    const int64_t *x = W->x;
    uint64_t gu = 0;
    for (int i = 0; i < n; ++i) gu = gcd64(gu, uabs64(x[(i << 5) + lane]));
    const i128 g = (i128)gu, kn = gu == 1 ? val : q128(val, g * g);     // kn = L K'^T S K'
    // o = Hdet / gcd(Hdet, Hadj y'): the order of K' = K / g in Lambda / Gamma
    uint64_t og = (uint64_t)D.Hdet;
    for (int i = 0; i < n && og != 1; ++i) {
        const i128 hv = W->hx[(i << 5) + lane];
        const u128 av = uabs(gu == 1 ? hv : q128(hv, g));
        const uint64_t r = (av >> 64) ? (uint64_t)(av % (u128)og) : (uint64_t)av % og;
        if (r) og = gcd64(og, r);
    }
    const i128 o = (i128)((uint64_t)D.Hdet / og);
    // l . c1 = o (w . y') / Cden for W c1 = o K'
    i128 num, den;
    if (mul_ovf(o, W->wx[lane], &num) || mul_ovf(g, (i128)D.Cden, &den)) return ZPK_OVF_K;
    if (r128(num, den)) return ZPK_INEXACT_K;
    const i128 QL = W->QL, lc1 = q128(num, den), lk = D.lk, alk = lk < 0 ? -lk : lk;
    // j: j o > g D0 and g j o kn < Q L
    i128 gLsn, gokn, gD0;
    if (mul_ovf(g, (i128)D.L, &gLsn) || mul_ovf(gLsn, (i128)D.sn, &gLsn) || mul_ovf(g, o, &gokn) ||
        mul_ovf(gokn, kn, &gokn) || mul_ovf(g, (i128)P.D0, &gD0)) return ZPK_OVF_K;
    i128 jlo = fdivq(gD0, o) + 1, jhi = q128(QL - 1, gokn);
    if (jlo > jhi) return ZPK_OK;
    // per j: M0 = j lc1 + t lk >= M0min in one residue class mod |lk|, with
    // g L sn M0^2 < sd j o (Q L - g j o kn); a float screen (relative margin 1e-9)
    // skips the j whose smallest M0 fails, the rest is exact
    const double gLsn_d = (double)gLsn, sdo_d = (double)D.sd * (double)o;
    {
        // the screen fails at every j where even M0 = M0min does: outside the roots of
        // sd o j (Q L - g o kn j) = T, T = (M0min^2 g L sn - 1) / (1 + 1e-9) (a concave
        // parabola in j), so the loop runs between the roots, widened by a relative 1e-6
        // and two steps on each side (far beyond the roots' rounding)
        const double T = ((double)P.M0min * (double)P.M0min * gLsn_d - 1.0) / (1.0 + 1e-9);
        const double B = (double)QL, C = (double)gokn, Ta = T / sdo_d;
        const double disc = B * B - 4.0 * C * Ta;
        if (disc < -1e-6 * B * B) return ZPK_OK;                   // no j reaches T
        const double sq = sqrt(fmax(disc, 0.0));
        const double r1 = Ta > 0 ? 2.0 * Ta / (B + sq) : 0.0, r2 = (B + sq) / (2.0 * C);
        const double jl = floor(r1 - 1e-6 * (r1 + 1.0)) - 2.0, jr = ceil(r2 + 1e-6 * (r2 + 1.0)) + 2.0;
        if (jl > (double)jlo && jl < 1e30) jlo = (i128)jl;
        if (jr < (double)jhi && jr > -1e30) jhi = (i128)jr;
        if (jlo > jhi) return ZPK_OK;
    }
    const i128 step = r128(r128(lc1, alk) + alk, alk), m0m = r128(r128((i128)P.M0min, alk) + alk, alk);
    i128 res;
    if (mul_ovf(r128(jlo, alk), step, &res)) return ZPK_OVF_K;
    res = r128(res, alk);
    bool have_c1 = false;
    for (i128 j = jlo; j <= jhi; ++j, res = res + step >= alk ? res + step - alk : res + step) {
        if (++steps > P.budget) return ZPK_BUDGET;
        i128 off = res - m0m;
        if (off < 0) off += alk;
        const i128 M0c = (i128)P.M0min + off;
        i128 diff;
        if (mul_ovf(gokn, j, &diff) || sub_ovf(QL, diff, &diff)) return ZPK_OVF_K;
        const double Rd = sdo_d * (double)j * (double)diff;
        if ((double)M0c * (double)M0c * gLsn_d > Rd * (1 + 1e-9) + 1.0) continue;
        i128 R, jo;
        if (mul_ovf(j, o, &jo) || mul_ovf(jo, (i128)D.sd, &R) || mul_ovf(R, diff, &R)) return ZPK_OVF_K;
        for (i128 M0 = M0c;; M0 += alk) {
            if (++steps > P.budget) return ZPK_BUDGET;
            i128 lhs, t1;
            if (mul_ovf(M0, M0, &lhs) || mul_ovf(lhs, gLsn, &lhs)) break;      // (beyond R)
            if (lhs >= R) break;
            if (mul_ovf(j, lc1, &t1) || sub_ovf(M0, t1, &t1)) return ZPK_OVF_K;
            if (r128(t1, lk)) return ZPK_INEXACT_K;
            if (!have_c1) {
                // y = x V / g (Lambda coordinates of K'), v = o O^T y = o K', c1 = Cs v / Cden
                i128 y[32], v[32];
                for (int b = 0; b < n; ++b) {
                    i128 s = 0;
                    for (int a = 0; a < n; ++a) {
                        const int64_t xa = x[(a << 5) + lane];
                        if (xa && muladd_ovf((i128)xa, (i128)W->L.B[a * 32 + b], s, &s)) return ZPK_OVF_K;
                    }
                    y[b] = gu == 1 ? s : q128(s, g);
                }
                for (int i = 0; i < m; ++i) {
                    i128 s = 0;
                    for (int b = 0; b < n; ++b)
                        if (y[b] && muladd_ovf((i128)W->U[(b + 1) * MH + i], y[b], s, &s)) return ZPK_OVF_K;
                    if (mul_ovf(o, s, &v[i])) return ZPK_OVF_K;
                }
                for (int i = 0; i < m; ++i) {
                    i128 s = 0;
                    for (int kk = 0; kk < m; ++kk)
                        if (v[kk] && muladd_ovf((i128)W->Cs[i * 32 + kk], v[kk], s, &s)) return ZPK_OVF_K;
                    if (s % (i128)D.Cden) return ZPK_INEXACT_K;
                    W->c1[(i << 5) + lane] = s / (i128)D.Cden;
                }
                have_c1 = true;
            }
            const int rc = zpk_emit(P, k, W, j, q128(t1, lk), lane);
            if (rc) return rc;
        }
    }
    return ZPK_OK;
}

// lane 0, before the walks: the arguments, Q L, the FP64 Cholesky factor R of Gr
// and the radius.  As the dilation bound's search (pfg_mu0.cuh): R^T R = Gr + E,
// |E| <= g1 |R^T||R|, so x^T Gr x >= |R x|^2 (1 - g1 C), C = 2 ||R||_F^2 ||R^-1||_F^2,
// and x^T Gr x D0 < Q L needs |R x|^2 < rad = Q L / D0 / (1 - g1 C).
__device__ int zpk_prepare(const ZpkArgs &P, ZpkScratch *W, const ZpkDir &D)
{
    const int n = P.h - 2;
    if (P.D0 < 1 || P.M0min < 1) return ZPK_ARGS;
    i128 QL;
    if (mul_ovf((i128)P.Q, (i128)D.L, &QL) || QL < 1) return ZPK_OVF_QL;
    double *R = W->R;
    for (int j = 0; j < n; ++j) {
        double dj = (double)W->Gr[j * 32 + j];
        for (int kk = 0; kk < j; ++kk) dj -= R[kk * 32 + j] * R[kk * 32 + j];
        if (!(dj > 0)) return ZPK_CHOL;
        R[j * 32 + j] = sqrt(dj);
        for (int i = j + 1; i < n; ++i) {
            double t = (double)W->Gr[j * 32 + i];
            for (int kk = 0; kk < j; ++kk) t -= R[kk * 32 + j] * R[kk * 32 + i];
            R[j * 32 + i] = t / R[j * 32 + j];
        }
    }
    double fR = 0, fRi = 0;
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i <= j; ++i) fR += R[i * 32 + j] * R[i * 32 + j];
        double col[32];
        for (int i = j; i >= 0; --i) {
            double t = (i == j) ? 1.0 : 0.0;
            for (int kk = i + 1; kk <= j; ++kk) t -= R[i * 32 + kk] * col[kk];
            col[i] = t / R[i * 32 + i];
            fRi += col[i] * col[i];
        }
    }
    const double u = 0x1p-53;
    const double g1 = (n + 1) * u / (1 - (n + 1) * u);
    const double C = 2.0 * fR * fRi;
    if (!(g1 * C < 1e-6)) return ZPK_ILLCOND;
    W->rad = (double)QL / (double)P.D0 / (1.0 - g1 * C) * (1.0 + 1e-12);
    W->g2 = n * u / (1 - n * u);
    W->QL = QL;
    W->nout = 0;
    W->abort = 0;
    return ZPK_OK;
}

constexpr int ZPK_STOPPED = -1000;            // (internal) another lane of the warp failed

// Step 5, one depth-first walk per lane over every x != 0 with x^T Gr x D0 < Q L:
// the nodes that survive the pruning at the split level (two levels below the
// top) are dealt to the lanes in turn, each lane walking the levels above in
// full and below only under its own nodes.  A level's term is computed within
// g2 a_i; leaves are decided exactly from the partial sums carried down the
// levels (|x_i| < 2^20 keeps them far inside int128).
__device__ int zpk_walk(const ZpkArgs &P, int k, ZpkScratch *W, const ZpkDir &D, int lane)
{
    const int n = P.h - 2, split = n > 2 ? n - 2 : 0;
    const double *R = W->R, rad = W->rad, g2 = W->g2, u = 0x1p-53;
    i128 *gx = W->gx, *hx = W->hx, *wx = W->wx, *vals = W->vals;
    int64_t *x = W->x, *lo = W->lo, *hi = W->hi;
    double *rem = W->rem, *aoff = W->aoff, *ofs = W->ofs;
#define ZL(i) (((i) << 5) + lane)                 // entry i of this lane's vectors
#define ZLL(l, kk) (((((l) << 5) + (kk)) << 5) + lane)   // entry kk of level l
    for (int kk = 0; kk < n; ++kk) { gx[ZLL(n, kk)] = 0; hx[ZLL(n, kk)] = 0; x[ZL(kk)] = 0; }
    wx[ZL(n)] = 0; vals[ZL(n)] = 0; rem[ZL(n)] = rad;
    auto enter = [&](int ii) -> bool {
        double o = 0, a = 0;
        for (int j = ii + 1; j < n; ++j) { const double t = R[ii * 32 + j] * (double)x[ZL(j)]; o += t; a += fabs(t); }
        const double rii = R[ii * 32 + ii];
        const double ctr = -o / rii, wd = sqrt(fmax(rem[ZL(ii + 1)], 0.0)) / rii;
        // rounding of the centre and width, as a multiple of a coordinate step: must stay below 1/2
        const double e = g2 * (fabs(ctr) + wd + 1.0 + a / rii) * 4.0 + 4.0 * u * (fabs(ctr) + wd);
        if (!(e < 0.5) || !(fabs(ctr) + wd < 1e6)) return false;
        lo[ZL(ii)] = (int64_t)floor(ctr - wd) - 1;
        hi[ZL(ii)] = (int64_t)ceil(ctr + wd) + 1;
        aoff[ZL(ii)] = a;
        ofs[ZL(ii)] = o;
        x[ZL(ii)] = lo[ZL(ii)];
        return true;
    };
    long long steps = 0, dealt = 0;
    int i = n - 1;
    if (!enter(i)) return ZPK_ENTER;
    for (;;) {
        if (++steps > P.budget) return ZPK_BUDGET;
        if ((steps & 255) == 0 && *(volatile int *)&W->abort) return ZPK_STOPPED;
        if (x[ZL(i)] > hi[ZL(i)]) {                                  // level done
            if (++i == n) break;
            x[ZL(i)]++;
            continue;
        }
        const double xi_d = (double)x[ZL(i)];
        const double t = R[i * 32 + i] * xi_d + ofs[ZL(i)];
        const double a = fabs(R[i * 32 + i] * xi_d) + aoff[ZL(i)];
        const double lb = fmax(fabs(t) - g2 * a, 0.0) * (1.0 - 4.0 * u);
        const double r = rem[ZL(i + 1)] - lb * lb * (1.0 - 4.0 * u);
        if (r < 0) { x[ZL(i)]++; continue; }                         // (rigorously) too long
        if (i == split && ((dealt++) & 31) != lane) { x[ZL(i)]++; continue; }   // another lane's node
        const i128 xi = x[ZL(i)];
        if (xi >= (1 << 20) || xi <= -(1 << 20)) return ZPK_COORD;
        for (int kk = 0; kk < n; ++kk) {
            gx[ZLL(i, kk)] = gx[ZLL(i + 1, kk)] + (i128)W->Gr[kk * 32 + i] * xi;
            hx[ZLL(i, kk)] = hx[ZLL(i + 1, kk)] + (i128)W->HT[kk * 32 + i] * xi;
        }
        wx[ZL(i)] = wx[ZL(i + 1)] + (i128)W->wv[i] * xi;
        vals[ZL(i)] = vals[ZL(i + 1)] + xi * (2 * gx[ZLL(i + 1, i)] + (i128)W->Gr[i * 32 + i] * xi);
        if (i > 0) {
            rem[ZL(i)] = r;
            --i;
            if (!enter(i)) return ZPK_ENTER;
            continue;
        }
        const i128 val = vals[ZL(0)];
        if (val > 0) {                                               // a leaf, decided exactly
            i128 lhs;
            if (mul_ovf(val, (i128)P.D0, &lhs)) return ZPK_OVF_QL;
            if (lhs < W->QL) {
                const int rc = zpk_per_short(P, k, W, D, val, steps, lane);
                if (rc) return rc;
            }
        } else {
            bool nz = false;
            for (int j = 0; j < n; ++j) nz |= x[ZL(j)] != 0;
            if (nz) return ZPK_NONE;                                 // not positive definite (exactly)
        }
        x[ZL(i)]++;
    }
    return ZPK_OK;
#undef ZL
#undef ZLL
}

// Step 5 for the warp: the walks, then the status of the lowest lane that
// failed (the others stop at their next poll).
__device__ int zpk_search(const ZpkArgs &P, int k, ZpkScratch *W, const ZpkDir &D, int lane)
{
    int st = 0;
    if (lane == 0) st = zpk_prepare(P, W, D);
    st = __shfl_sync(FULL, st, 0);
    __syncwarp();
    if (st) return st;
    int my = zpk_walk(P, k, W, D, lane);
    if (my != ZPK_OK && my != ZPK_STOPPED) atomicExch(&W->abort, 1);
    const unsigned bad = __ballot_sync(FULL, my != ZPK_OK && my != ZPK_STOPPED);
    if (!bad) return ZPK_OK;
    return __shfl_sync(FULL, my, __ffs((int)bad) - 1);
}

// One warp per direction, taken from a work counter.
__global__ void __launch_bounds__(128) k_zpk(ZpkArgs P)
{
    const int lane = threadIdx.x & 31;
    ZpkScratch *W = P.scratch + (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5));
    if (lane == 0) W->L.B = W->Lb;
    __syncwarp();
    for (;;) {
        unsigned t = 0;
        if (lane == 0) t = atomicAdd(P.next, 1u);
        t = __shfl_sync(FULL, t, 0);
        if (t >= (unsigned)P.n_p) break;
        ZpkDir D{};
        int st = P.h < 3 || P.h > ZPK_MAXH ? (int)ZPK_RANGE : zpk_setup(P, (int)t, W, D, lane);
        if (st == ZPK_OK) st = zpk_search(P, (int)t, W, D, lane);
        if (lane == 0) P.status[t] = st;
        __syncwarp();
    }
}

}  // namespace pfg
