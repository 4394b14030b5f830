// Per-direction lattice setup on the device, one warp per direction.
//
// For direction p of a geometry (kappa, Mbasis), this builds the data the
// search needs (the reference does the same on the CPU in pfl_build,
// pfvs/fp_kernel/pfv_lattice.h:604-680, and its factorization in
// fpk_factor_fast/fpk_factor_exact, pfvs/fp_kernel/fpk_common.h:259-309):
//
//   Z = kappa.p, T = Z p, v = T Mbasis              exact, int128-checked
//   O = lattice orthogonal to v (Bezout steps)       pfv_lattice.h:162-188
//   LLL(O) (Euclidean)                               warp_lll
//   Binter = Mbasis O^T, coni column order           pfv_lattice.h:630-653
//   ZB = Z Binter, mat = -Binter^T ZB
//   cut-aware basis: T = [K | w], K an LLL basis of ker(Binter[0,:]) w.r.t.
//   mat, w size-reduced against K; then Binter[0,:] = (0, .., 0, g), so M0
//   is fixed at the root level by an exact interval  pfv_lattice.h:554-602
//   GCD rows: an echelon basis of the row lattice of ZB[1:] whose rows are
//   reduced against an LLL basis of the rows below them (the reference uses
//   the row-HNF, whose rows reach 77-367 bits here; any echelon basis of
//   the same lattice prunes identically, and this one keeps the rows small)
//   U: FP64 Cholesky factor of mat with a certified backward-error margin
//   (the reference rounds an exact GMP/int128 Bareiss factor; in FP64 the
//   factor is exact for mat + dA, |dA| <= gamma_{d+1} |U^T||U|, and the
//   search widens its slack by a bound on c^T dA c over the ellipsoid).
#pragma once
#include "pfg_types.cuh"

namespace pfg {

struct SetupScratch {
    int64_t Z[MH * MH];
    int64_t B[(MH + 1) * MH];       // LLL rows (+ the 'last' row)
    i128 G[(MH + 1) * (MH + 1)];    // exact Gram of B's rows
    double mu[MH * MH];
    double bb[MH + 1];
    int64_t V[MH * MH];             // unimodular transforms / temporaries
    int64_t S[MH * MH];
    double X[MH * MH];              // U^-1 for the certificate
    i128 y[MH];
    int64_t w[MH], v[MH];
    int order[MH];
};

constexpr int LDG = MH + 1;

struct SetupArgs {
    const Geo *geo;
    const int64_t *kappa, *Mbasis, *ps;     // ps: (n, MH)
    const int32_t *pgeo;
    const int64_t *slab_off;                // (n,) slab offset per direction
    int64_t *slab;
    Dir *dirs;
    SetupScratch *scratch;                  // one per warp
    int n;
    unsigned *next;                         // work counter
};

__device__ __forceinline__ double warp_sum(double x)
{
    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(FULL, x, o);
    return x;
}

__device__ __forceinline__ bool warp_any(bool b) { return __any_sync(FULL, b); }

// ---------------------------------------------------------------------------
// Warp LLL (delta 0.99) on the m rows of B (length n, stride MH) with exact
// Gram G (stride LDG) over M = m + has_last rows; row m is 'last', which is
// size-reduced against the reduced rows at the end.  Float Gram-Schmidt
// data (mu, bb) are recomputed from the exact Gram and only choose the
// unimodular steps.  Returns 0, or ST_OVERFLOW on an int64/int128 overflow
// or rank loss, or when the iteration budget runs out.
// ---------------------------------------------------------------------------
struct Lll {
    int64_t *B;
    i128 *G;
    double *mu, *bb;
    int n, M;
};

// b_k -= q b_j, on the vectors and the exact Gram; true on overflow
__device__ bool lll_sub(Lll &L, int k, int j, int64_t q, int lane)
{
    bool bad = false;
    for (int c = lane; c < L.n; c += 32) {
        i128 x = (i128)L.B[k * MH + c] - (i128)q * L.B[j * MH + c];
        if (!fits64(x)) bad = true;
        else L.B[k * MH + c] = (int64_t)x;
    }
    i128 gkk = 0;
    {
        i128 t, u;
        bool b = mul_ovf(L.G[j * LDG + j], (i128)q, &t) ||
                 sub_ovf(t, L.G[k * LDG + j], &t) || sub_ovf(t, L.G[k * LDG + j], &t) ||
                 mul_ovf(t, (i128)q, &u) || add_ovf(L.G[k * LDG + k], u, &gkk);
        bad |= b;
    }
    __syncwarp();
    for (int l = lane; l < L.M; l += 32) {
        if (l == k) continue;
        i128 t;
        if (mul_ovf(L.G[j * LDG + l], (i128)q, &t) || sub_ovf(L.G[k * LDG + l], t, &t)) { bad = true; continue; }
        L.G[k * LDG + l] = t;
        L.G[l * LDG + k] = t;
    }
    __syncwarp();
    if (lane == 0) L.G[k * LDG + k] = gkk;
    __syncwarp();
    return warp_any(bad);
}

// Gram-Schmidt data of row k from the exact Gram: r_j = mu_kj bb_j solves
// the unit lower-triangular system r_j = G_kj - sum_{l<j} mu_jl r_l
// (column-oriented forward substitution, lanes own rows).
__device__ void lll_gs(Lll &L, int k, int lane)
{
    double a0 = lane < k ? (double)L.G[k * LDG + lane] : 0.0;
    double a1 = lane + 32 < k ? (double)L.G[k * LDG + lane + 32] : 0.0;
    double s = 0.0;
    for (int j = 0; j < k; ++j) {
        double rj = __shfl_sync(FULL, j < 32 ? a0 : a1, j & 31);
        double mkj = rj / L.bb[j];
        if (lane == (j & 31)) L.mu[k * MH + j] = mkj;
        s += mkj * rj;
        if (lane > j && lane < k) a0 -= L.mu[lane * MH + j] * rj;
        if (lane + 32 > j && lane + 32 < k) a1 -= L.mu[(lane + 32) * MH + j] * rj;
    }
    if (lane == 0) L.bb[k] = (double)L.G[k * LDG + k] - s;
    __syncwarp();
}

__device__ void lll_swap(Lll &L, int k, int lane)
{
    for (int c = lane; c < L.n; c += 32) {
        int64_t t = L.B[k * MH + c]; L.B[k * MH + c] = L.B[(k - 1) * MH + c]; L.B[(k - 1) * MH + c] = t;
    }
    __syncwarp();
    for (int l = lane; l < L.M; l += 32) {
        i128 t = L.G[k * LDG + l]; L.G[k * LDG + l] = L.G[(k - 1) * LDG + l]; L.G[(k - 1) * LDG + l] = t;
    }
    __syncwarp();
    for (int l = lane; l < L.M; l += 32) {
        i128 t = L.G[l * LDG + k]; L.G[l * LDG + k] = L.G[l * LDG + k - 1]; L.G[l * LDG + k - 1] = t;
    }
    __syncwarp();
}

__device__ int warp_lll(Lll &L, int m, bool has_last, int lane)
{
    const double delta = 0.99;
    L.M = m + (has_last ? 1 : 0);
    if (m >= 1) {
        lll_gs(L, 0, lane);
        if (!(L.bb[0] > 0)) return ST_OVERFLOW;
    }
    if (m >= 2) lll_gs(L, 1, lane);
    int k = 1, iters = 0;
    while (k < m) {
        if (++iters > 200000) return ST_OVERFLOW;
        for (int pass = 0; pass < 4; ++pass) {
            bool changed = false;
            for (int j = k - 1; j >= 0; --j) {
                double q = rint(L.mu[k * MH + j]);
                if (q == 0.0) continue;
                if (!(fabs(q) <= 9.0e18)) return ST_OVERFLOW;
                int64_t qi = (int64_t)q;
                if (lll_sub(L, k, j, qi, lane)) return ST_OVERFLOW;
                for (int l = lane; l < j; l += 32) L.mu[k * MH + l] -= q * L.mu[j * MH + l];
                __syncwarp();
                if (lane == 0) L.mu[k * MH + j] -= q;
                __syncwarp();
                changed = true;
            }
            if (!changed) break;
            lll_gs(L, k, lane);
        }
        if (!(L.bb[k] > 0)) return ST_OVERFLOW;
        double mk = L.mu[k * MH + k - 1];
        if (L.bb[k] < (delta - mk * mk) * L.bb[k - 1]) {
            lll_swap(L, k, lane);
            k = k > 1 ? k - 1 : 1;
            if (k == 1) lll_gs(L, 0, lane);
            lll_gs(L, k - 1, lane);
            lll_gs(L, k, lane);
        } else {
            ++k;
            if (k < m) lll_gs(L, k, lane);
        }
    }
    if (has_last && m > 0) {            // size-reduce row m against rows 0..m-1
        double *mw = L.mu + m * MH;     // (row m of mu is free: m <= MD - 1)
        for (int pass = 0; pass < 4; ++pass) {
            // mw_j bb_j = G_mj - sum_{l<j} mu_jl mw_l bb_l  (forward substitution)
            double a0 = lane < m ? (double)L.G[m * LDG + lane] : 0.0;
            double a1 = lane + 32 < m ? (double)L.G[m * LDG + lane + 32] : 0.0;
            for (int j = 0; j < m; ++j) {
                double rj = __shfl_sync(FULL, j < 32 ? a0 : a1, j & 31);
                if (lane == (j & 31)) mw[j] = rj / L.bb[j];
                if (lane > j && lane < m) a0 -= L.mu[lane * MH + j] * rj;
                if (lane + 32 > j && lane + 32 < m) a1 -= L.mu[(lane + 32) * MH + j] * rj;
            }
            __syncwarp();
            bool changed = false;
            for (int j = m - 1; j >= 0; --j) {
                double q = rint(mw[j]);
                if (q == 0.0) continue;
                if (!(fabs(q) <= 9.0e18)) return ST_OVERFLOW;
                if (lll_sub(L, m, j, (int64_t)q, lane)) return ST_OVERFLOW;
                for (int l = lane; l < j; l += 32) mw[l] -= q * L.mu[j * MH + l];
                __syncwarp();
                if (lane == 0) mw[j] -= q;
                __syncwarp();
                changed = true;
            }
            if (!changed) break;
        }
    }
    return 0;
}

// Euclidean Gram of rows 0..m-1 of B (length n)
__device__ bool gram_euclid(SetupScratch *W, int m, int n, int lane)
{
    bool bad = false;
    for (int e = lane; e < m * m; e += 32) {
        int i = e / m, j = e % m;
        if (j > i) continue;
        i128 s = 0;
        for (int c = 0; c < n; ++c)
            if (add_ovf(s, (i128)W->B[i * MH + c] * W->B[j * MH + c], &s)) bad = true;
        W->G[i * LDG + j] = s;
        W->G[j * LDG + i] = s;
    }
    __syncwarp();
    return warp_any(bad);
}

// Unimodular U (n x n rows, stride MH, into Uo) with U v = (gcd, 0, ..., 0)
// by Bezout steps on (w0, wk) (as pfl_unimodular, pfvs/fp_kernel/pfv_lattice.h:
// 162-188), with one change against coefficient growth: the coordinates are
// first permuted so that a coprime pair of entries of v / gcd(v) (the one
// with the smallest larger entry) comes first.  After the first step the
// running gcd is then 1, every later step is (1, w_k) -> (1, 0), and the
// entries stay below about max|v|^2 instead of compounding.  Any unimodular
// U gives the same lattice; v is read from vin (length n).
__device__ int warp_unimodular(const int64_t *vin, int n, int64_t *Uo, int64_t *wtmp, int *perm, int lane)
{
    // g = gcd(v)
    uint64_t g = 0;
    for (int e = lane; e < n; e += 32) g = gcd64(g, uabs64(vin[e]));
    for (int o = 16; o; o >>= 1) g = gcd64(g, __shfl_xor_sync(FULL, g, o));
    if (g == 0) return ST_OVERFLOW;
    // coprime pair (i, j) of v / g minimising max(|v_i|, |v_j|)
    uint64_t best = ~0ull;
    int who = -1;
    for (int e = lane; e < n * n; e += 32) {
        const int i = e / n, j = e % n;
        if (j <= i || !vin[i] || !vin[j]) continue;
        const uint64_t a = uabs64(vin[i]) / g, b = uabs64(vin[j]) / g;
        const uint64_t sc = a > b ? a : b;
        if (sc < best && gcd64(a, b) == 1) { best = sc; who = e; }
    }
    for (int o = 16; o; o >>= 1) {
        uint64_t ob = __shfl_xor_sync(FULL, best, o);
        int ow = __shfl_xor_sync(FULL, who, o);
        if (ob < best || (ob == best && ow >= 0 && (who < 0 || ow < who))) { best = ob; who = ow; }
    }
    if (lane == 0) {
        for (int c = 0; c < n; ++c) perm[c] = c;
        if (who >= 0) {
            const int i = who / n, j = who % n;
            int t = perm[0]; perm[0] = perm[i]; perm[i] = t;
            int pj = -1;
            for (int c = 0; c < n; ++c) if (perm[c] == j) pj = c;
            t = perm[1]; perm[1] = perm[pj]; perm[pj] = t;
        }
    }
    __syncwarp();
    for (int e = lane; e < n * n; e += 32) Uo[(e / n) * MH + e % n] = (e / n) == (e % n);
    for (int e = lane; e < n; e += 32) wtmp[e] = vin[perm[e]];
    __syncwarp();
    bool bad = false;
    for (int k = 1; k < n; ++k) {
        int64_t wk = wtmp[k];
        if (wk == 0) continue;
        int64_t w0 = wtmp[0], s, t;
        int64_t gk = xgcd_floor(w0, wk, &s, &t);
        if (gk == 0) return ST_OVERFLOW;
        int64_t m10 = -fdiv64(wk, gk), m11 = fdiv64(w0, gk);
        __syncwarp();
        if (lane == 0) { wtmp[0] = gk; wtmp[k] = 0; }
        for (int c = lane; c < n; c += 32) {
            i128 t1 = (i128)s * Uo[c] + (i128)t * Uo[k * MH + c];
            i128 t2 = (i128)m10 * Uo[c] + (i128)m11 * Uo[k * MH + c];
            if (!fits64(t1) || !fits64(t2)) { bad = true; continue; }
            Uo[c] = (int64_t)t1;
            Uo[k * MH + c] = (int64_t)t2;
        }
        __syncwarp();
        if (warp_any(bad)) return ST_OVERFLOW;
    }
    // undo the permutation on the columns: U[row][perm[c]] = U'[row][c]
    for (int r = 0; r < n; ++r) {
        int64_t x0 = lane < n ? Uo[r * MH + lane] : 0;
        int64_t x1 = lane + 32 < n ? Uo[r * MH + lane + 32] : 0;
        __syncwarp();
        if (lane < n) Uo[r * MH + perm[lane]] = x0;
        if (lane + 32 < n) Uo[r * MH + perm[lane + 32]] = x1;
        __syncwarp();
    }
    return 0;
}

// warp argmin over rows r < nr of |B[r][col]| != 0 (-1 if the column is 0)
__device__ int argmin_nonzero(const int64_t *B, int nr, int col, int lane)
{
    uint64_t best = ~0ull;
    int who = -1;
    for (int r = lane; r < nr; r += 32) {
        uint64_t a = uabs64(B[r * MH + col]);
        if (a && a < best) { best = a; who = r; }
    }
    for (int o = 16; o; o >>= 1) {
        uint64_t ob = __shfl_xor_sync(FULL, best, o);
        int ow = __shfl_xor_sync(FULL, who, o);
        if (ob < best || (ob == best && ow >= 0 && (who < 0 || ow < who))) { best = ob; who = ow; }
    }
    return who;
}

// ---------------------------------------------------------------------------
// The setup of one direction.
// ---------------------------------------------------------------------------
__device__ int setup_one(const SetupArgs &A, int pid, int lane, int &stage)
{
    SetupScratch *W = A.scratch + (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5));
    const Geo g = A.geo[A.pgeo[pid]];
    const int h = g.h, d = h - 1;
    const int64_t *kap = A.kappa + g.koff, *Mb = A.Mbasis + g.moff, *p = A.ps + (int64_t)pid * MH;
    int64_t *slab = A.slab + A.slab_off[pid];
    const Slab L = slab_layout(h, d);
    Dir &D = A.dirs[pid];
    bool bad = false;

    stage = 1;
    // 1. Z = kappa . p
    for (int e = lane; e < h * h; e += 32) {
        i128 s = 0;
        for (int k = 0; k < h; ++k)
            if (add_ovf(s, (i128)kap[(int64_t)e * h + k] * p[k], &s)) bad = true;
        if (!fits64(s)) bad = true;
        W->Z[(e / h) * MH + e % h] = (int64_t)s;
    }
    __syncwarp();
    if (warp_any(bad)) return ST_OVERFLOW;
    stage = 2;
    // 2. T = Z p, v = T Mbasis
    for (int i = lane; i < h; i += 32) {
        i128 s = 0;
        for (int k = 0; k < h; ++k)
            if (add_ovf(s, (i128)W->Z[i * MH + k] * p[k], &s)) bad = true;
        if (!fits64(s)) bad = true;
        W->w[i] = (int64_t)s;
    }
    __syncwarp();
    if (warp_any(bad)) return ST_OVERFLOW;
    for (int j = lane; j < h; j += 32) {
        i128 s = 0;
        for (int i = 0; i < h; ++i)
            if (add_ovf(s, (i128)W->w[i] * Mb[i * h + j], &s)) bad = true;
        if (!fits64(s)) bad = true;
        W->v[j] = (int64_t)s;
    }
    __syncwarp();
    if (warp_any(bad)) return ST_OVERFLOW;
    stage = 3;
    // 3. orthogonal lattice: rows 1.. of the unimodular transform of v
    int st = warp_unimodular(W->v, h, W->V, W->w, W->order, lane);
    if (st) return st;
    for (int e = lane; e < d * h; e += 32) W->B[(e / h) * MH + e % h] = W->V[(e / h + 1) * MH + e % h];
    __syncwarp();
    stage = 4;
    // 4. Euclidean LLL of O
    if (gram_euclid(W, d, h, lane)) return ST_OVERFLOW;
    Lll LL{W->B, W->G, W->mu, W->bb, h, d};
    if ((st = warp_lll(LL, d, false, lane))) return st;
    stage = 5;
    // 5. (Mbasis O^T)^T rows, 6. coni order (rows with entry 0 == 0 first, stable)
    for (int e = lane; e < d * h; e += 32) {
        int a = e / h, i = e % h;
        i128 s = 0;
        for (int l = 0; l < h; ++l)
            if (add_ovf(s, (i128)Mb[i * h + l] * W->B[a * MH + l], &s)) bad = true;
        if (!fits64(s)) bad = true;
        W->S[a * MH + i] = (int64_t)s;
    }
    __syncwarp();
    if (warp_any(bad)) return ST_OVERFLOW;
    if (lane == 0) {
        int no = 0;
        for (int a = 0; a < d; ++a) if (W->S[a * MH] == 0) W->order[no++] = a;
        for (int a = 0; a < d; ++a) if (W->S[a * MH] != 0) W->order[no++] = a;
    }
    __syncwarp();
    int64_t *BT = slab + L.bt, *ZT = slab + L.zt, *MAT = slab + L.mat;
    for (int e = lane; e < d * h; e += 32) BT[e] = W->S[W->order[e / h] * MH + e % h];
    __syncwarp();
    stage = 7;
    // 7. ZT[a][r] = (Z Binter)[r][a], mat = -Binter^T Z Binter
    for (int e = lane; e < d * h; e += 32) {
        int a = e / h, r = e % h;
        i128 s = 0;
        for (int i = 0; i < h; ++i)
            if (add_ovf(s, (i128)W->Z[r * MH + i] * BT[a * h + i], &s)) bad = true;
        if (!fits64(s)) bad = true;
        ZT[e] = (int64_t)s;
    }
    __syncwarp();
    if (warp_any(bad)) return ST_OVERFLOW;
    for (int e = lane; e < d * d; e += 32) {
        int a = e / d, b = e % d;
        i128 s = 0;
        for (int r = 0; r < h; ++r)
            if (add_ovf(s, (i128)BT[a * h + r] * ZT[b * h + r], &s)) bad = true;
        if (!fits64(-s)) bad = true;
        MAT[e] = (int64_t)(-s);
    }
    __syncwarp();
    if (warp_any(bad)) return ST_OVERFLOW;

    stage = 8;
    // 8. cut-aware basis (pfv_lattice.h:554-602)
    for (int a = lane; a < d; a += 32) W->v[a] = BT[a * h];
    __syncwarp();
    bool lnz = false;
    for (int a = lane; a < d; a += 32) lnz |= W->v[a] != 0;
    lnz = warp_any(lnz);
    int m0_level = -1;
    int64_t g_lin = 0;
    if (lnz) {
        if ((st = warp_unimodular(W->v, d, W->V, W->w, W->order, lane))) return st;
        // B rows 0..d-2 = K = V[1..], row d-1 = w = V[0]
        for (int e = lane; e < d * d; e += 32) {
            int a = e / d, c = e % d;
            W->B[a * MH + c] = a < d - 1 ? W->V[(a + 1) * MH + c] : W->V[c];
        }
        __syncwarp();
        // Gram w.r.t. mat: G_ij = B_i^T mat B_j
        for (int j = 0; j < d; ++j) {
            for (int c = lane; c < d; c += 32) {
                i128 s = 0;
                for (int k = 0; k < d; ++k)
                    if (add_ovf(s, (i128)MAT[c * d + k] * W->B[j * MH + k], &s)) bad = true;
                W->y[c] = s;
            }
            __syncwarp();
            for (int i = lane; i <= j; i += 32) {
                i128 s = 0, t;
                for (int c = 0; c < d; ++c) {
                    if (!W->B[i * MH + c]) continue;
                    if (mul_ovf(W->y[c], (i128)W->B[i * MH + c], &t) || add_ovf(s, t, &s)) bad = true;
                }
                W->G[i * LDG + j] = s;
                W->G[j * LDG + i] = s;
            }
            __syncwarp();
        }
        if (warp_any(bad)) return ST_OVERFLOW;
        Lll LK{W->B, W->G, W->mu, W->bb, d, d};
        if ((st = warp_lll(LK, d - 1, true, lane))) return st;
        // new columns a of Binter: sum_b B[a][b] Binter[:, b]  (likewise ZB)
        for (int e = lane; e < d * h; e += 32) {
            int a = e / h, r = e % h;
            i128 s = 0, t = 0;
            for (int b = 0; b < d; ++b) {
                s += (i128)W->B[a * MH + b] * BT[b * h + r];
                t += (i128)W->B[a * MH + b] * ZT[b * h + r];
            }
            if (!fits64(s) || !fits64(t)) bad = true;
            W->S[a * MH + r] = (int64_t)s;
            W->V[a * MH + r] = (int64_t)t;
        }
        __syncwarp();
        if (warp_any(bad)) return ST_OVERFLOW;
        for (int e = lane; e < d * h; e += 32) {
            BT[e] = W->S[(e / h) * MH + e % h];
            ZT[e] = W->V[(e / h) * MH + e % h];
        }
        for (int e = lane; e < d * d; e += 32) {
            i128 x = W->G[(e / d) * LDG + e % d];
            if (!fits64(x)) bad = true;
            MAT[e] = (int64_t)x;
        }
        __syncwarp();
        if (warp_any(bad)) return ST_OVERFLOW;
        for (int a = lane; a < d - 1; a += 32) bad |= BT[a * h] != 0;
        if (warp_any(bad)) return ST_OVERFLOW;      // (cannot happen: K spans ker l)
        m0_level = d - 1;
        g_lin = BT[(d - 1) * h];
    } else if (g.linmin > 0) {
        if (lane == 0) { D.m0_level = -1; D.g_lin = 0; }
        return ST_EMPTY;
    }

    stage = 9;
    // 9. GCD rows: echelon basis of the row lattice of ZB[1:] with small rows.
    // The rows r_k = ZB[k][:], k = 1..d, satisfy sum_k p_k r_k = 0 (p^T Z Binter
    // = 0 and p_0 = 0); with V p' = e0 from Bezout steps, the rows of V^-T R
    // are the rows of R with row 0 = p'^T R = 0: drop it, the rest is a basis.
    for (int e = lane; e < d * d; e += 32) W->B[(e / d) * MH + e % d] = ZT[(e % d) * h + e / d + 1];
    for (int e = lane; e < d; e += 32) W->w[e] = p[e + 1];
    __syncwarp();
    for (int k = 1; k < d; ++k) {
        int64_t wk = W->w[k];
        if (wk == 0) continue;
        int64_t w0 = W->w[0], s, t;
        int64_t gg = xgcd_floor(w0, wk, &s, &t);
        int64_t m10 = -fdiv64(wk, gg), m11 = fdiv64(w0, gg);
        __syncwarp();
        if (lane == 0) { W->w[0] = gg; W->w[k] = 0; }
        for (int c = lane; c < d; c += 32) {
            i128 r0 = (i128)m11 * W->B[c] - (i128)m10 * W->B[k * MH + c];
            i128 rk = -(i128)t * W->B[c] + (i128)s * W->B[k * MH + c];
            if (!fits64(r0) || !fits64(rk)) { bad = true; continue; }
            W->B[c] = (int64_t)r0;
            W->B[k * MH + c] = (int64_t)rk;
        }
        __syncwarp();
        if (warp_any(bad)) return ST_OVERFLOW;
    }
    stage = 91;
    for (int c = lane; c < d; c += 32) bad |= W->B[c] != 0;
    if (warp_any(bad)) return ST_OVERFLOW;          // p'^T ZB[1:] must vanish exactly
    int nr = d - 1;
    // drop row 0 (staged through S: an in-place shift would race across lanes)
    for (int e = lane; e < nr * d; e += 32) W->S[(e / d) * MH + e % d] = W->B[(e / d + 1) * MH + e % d];
    __syncwarp();
    for (int e = lane; e < nr * d; e += 32) W->B[(e / d) * MH + e % d] = W->S[(e / d) * MH + e % d];
    __syncwarp();
    int64_t *H = slab + L.H;
    for (int e = lane; e < d * d; e += 32) H[e] = 0;
    uint64_t hrows = 0;
    if (nr > 0) {
        // Rows whose construction would leave int64 (the last pivots are
        // large: the lattice of rows vanishing on all but the last columns has
        // a huge covolume) are not built: the rows found so far are kept, and
        // any set of rows of the lattice gives a valid GCD bound.
        if (gram_euclid(W, nr, d, lane)) goto h_done;
        Lll LH{W->B, W->G, W->mu, W->bb, d, nr};
        if (warp_lll(LH, nr, false, lane)) goto h_done;
        for (int col = 0; col < d && nr > 0; ++col) {
            int pr = -1;
            for (int it = 0; ; ++it) {
                if (it > 256) goto h_done;
                pr = argmin_nonzero(W->B, nr, col, lane);
                PFG_UNIFORM(pr);
                if (pr < 0) break;
                bool other = false;
                LH.M = nr;
                for (int r = 0; r < nr; ++r) {
                    if (r == pr) continue;
                    int64_t x = W->B[r * MH + col];
                    PFG_UNIFORM(x);
                    if (!x) continue;
                    int64_t q = fdiv64(x, W->B[pr * MH + col]);
                    PFG_UNIFORM(q);
                    __syncwarp();           // (every lane has read row r before lll_sub writes it)
                    if (lll_sub(LH, r, pr, q, lane)) goto h_done;
                    other |= W->B[r * MH + col] != 0;
                }
                PFG_UNIFORM(other);
                if (!other) break;
            }
            if (pr < 0) continue;
            // move the pivot row to the end (index nr - 1), positive pivot
            LH.M = nr;
            for (int k2 = pr + 1; k2 < nr; ++k2) lll_swap(LH, k2, lane);
            const bool neg = W->B[(nr - 1) * MH + col] < 0;
            PFG_UNIFORM(neg);
            __syncwarp();                   // (read by every lane before the owner negates it)
            if (neg) {
                for (int c = lane; c < d; c += 32) W->B[(nr - 1) * MH + c] = -W->B[(nr - 1) * MH + c];
                for (int l = lane; l < nr; l += 32) {
                    if (l == nr - 1) continue;
                    W->G[(nr - 1) * LDG + l] = -W->G[(nr - 1) * LDG + l];
                    W->G[l * LDG + nr - 1] = -W->G[l * LDG + nr - 1];
                }
                __syncwarp();
            }
            // LLL the rows below (rows 0..nr-2), size-reduce the pivot row against them
            if (warp_lll(LH, nr - 1, true, lane)) goto h_done;
            bool fits = true;
            for (int c = lane; c < d; c += 32) fits &= uabs64(W->B[(nr - 1) * MH + c]) < (1ull << 62);
            fits = __all_sync(FULL, fits);
            if (fits) {
                for (int c = lane; c < d; c += 32) H[col * d + c] = W->B[(nr - 1) * MH + c];
                hrows |= 1ull << col;
            }
            __syncwarp();
            --nr;
        }
    }
h_done:

    stage = 10;
    // 10. FP64 Cholesky of mat, certificate, float copies
    double *U = (double *)(slab + L.u64);
    for (int e = lane; e < d * d; e += 32) U[e] = 0.0;
    __syncwarp();
    bool notpd = false;
    for (int j = 0; j < d; ++j) {
        // row j of U: U_jj = sqrt(A_jj - sum_{k<j} U_kj^2), U_ji = (A_ji - sum_k U_kj U_ki) / U_jj
        double s0 = 0.0;
        for (int k = 0; k < j; ++k) { double u = U[k * d + j]; s0 += u * u; }
        double pj = (double)MAT[j * d + j] - s0;
        if (!(pj > 0)) { notpd = true; break; }
        double ujj = sqrt(pj);
        for (int i = j + 1 + lane; i < d; i += 32) {
            double s = 0.0;
            for (int k = 0; k < j; ++k) s += U[k * d + j] * U[k * d + i];
            U[j * d + i] = ((double)MAT[j * d + i] - s) / ujj;
        }
        if (lane == 0) U[j * d + j] = ujj;
        __syncwarp();
    }
    if (notpd) return ST_PRECISION;          // not certified positive definite here
    // ||U||_F^2 and ||U^-1||_F^2
    double *X = W->X;
    for (int j = 0; j < d; ++j) {
        for (int i = lane; i <= j; i += 32) {
            double x;
            if (i == j) x = 1.0 / U[j * d + j];
            else {
                double s = 0.0;
                for (int k = i; k < j; ++k) s += X[i * MH + k] * U[k * d + j];
                x = -s / U[j * d + j];
            }
            X[i * MH + j] = x;
        }
        __syncwarp();
    }
    double f1 = 0.0, f2 = 0.0;
    for (int e = lane; e < d * d; e += 32) {
        int i = e / d, j = e % d;
        if (j < i) continue;
        f1 += U[e] * U[e];
        f2 += X[i * MH + j] * X[i * MH + j];
    }
    f1 = warp_sum(f1);
    f2 = warp_sum(f2);
    const double u = 0x1p-53, gam = (d + 1) * u / (1.0 - (d + 1) * u);
    const double K = 2.0 * f1 * f2;              // 2x for the rounding in computing f2
    if (!(gam * K <= 1e-3)) return ST_PRECISION;
    const double slack_chol = 2.0 * gam * K * ((double)g.qmax + 1.0);
    float *U32 = (float *)(slab + L.u32);
    double *UI = (double *)(slab + L.ui64);
    float *UI32 = (float *)(slab + L.ui32);
    for (int e = lane; e < d * d; e += 32) U32[e] = (float)U[e];
    __syncwarp();
    for (int i = lane; i < d; i += 32) { UI[i] = 1.0 / U[i * d + i]; UI32[i] = 1.0f / U32[i * d + i]; }
    stage = 11;
    // 11. the search keeps exact incremental sums mat c, ZB c, Binter c in int64
    // (|entry| < 2^25, |c| < 2^31, <= 64 terms)
    for (int e = lane; e < d * d; e += 32) bad |= uabs64(MAT[e]) >= (1ull << 25);
    for (int e = lane; e < d * h; e += 32) bad |= uabs64(BT[e]) >= (1ull << 25) || uabs64(ZT[e]) >= (1ull << 25);
    if (warp_any(bad)) return ST_OVERFLOW;
    if (lane == 0) {
        D.m0_level = m0_level;
        D.g_lin = g_lin;
        D.hrows = hrows;
        D.slack_chol = slack_chol;
    }
    __syncwarp();
    return ST_PENDING;
}

__global__ void __launch_bounds__(128) k_setup(SetupArgs A)
{
    const int lane = threadIdx.x & 31;
    for (;;) {
        unsigned pid = 0;
        if (lane == 0) pid = atomicAdd(A.next, 1u);
        pid = __shfl_sync(FULL, pid, 0);
        if (pid >= (unsigned)A.n) break;
        const Geo g = A.geo[A.pgeo[pid]];
        if (lane == 0) {
            Dir &D = A.dirs[pid];
            D.geo = A.pgeo[pid]; D.h = g.h; D.d = g.h - 1; D.slab = A.slab_off[pid];
            D.m0_level = -1; D.g_lin = 0; D.hrows = 0; D.slack_chol = 0.0;
        }
        __syncwarp();
        int stage = 0;
        int st = setup_one(A, (int)pid, lane, stage);
        if (lane == 0) { A.dirs[pid].status = st; A.dirs[pid].pad = st < 0 ? stage : 0; }
        __syncwarp();
    }
}

}  // namespace pfg
