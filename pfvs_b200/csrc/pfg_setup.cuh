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
//
// The lattice reductions work on an LllMem<N> (rows of length <= N, the
// exact Gram in int128 as a packed triangle, packed Gram-Schmidt data): for
// h11 <= 32 it lives in shared memory (20.8 KB per warp), above that in
// the warp's global scratch.
#pragma once
#include "pfg_types.cuh"

namespace pfg {

// ---------------------------------------------------------------------------
// LLL working set of one warp.
// ---------------------------------------------------------------------------
template <int N> struct LllMem {
    static constexpr int R = N - 1;             // rows: at most d = h11 - 1 <= N - 1 are ever used
                                                // (d basis rows in step 4; d - 1 plus the 'last'
                                                // row in step 8; fewer in step 9)
    int64_t *B;                                 // rows, stride N: R * N words in the warp's global
                                                // scratch (set by the owner), so that the shared-memory
                                                // working set of h11 <= 32 is only the Gram and
                                                // Gram-Schmidt data (12.9 KB: 16 warps per SM)
    i128 G[R * (R + 1) / 2];                    // exact Gram, lower triangle packed (gix)
    i128 T[R];                                  // a copied column of G / a temporary vector
    double mu[R * (R - 1) / 2];                 // Gram-Schmidt coefficients mu(k, j), j < k (mix)
    double bb[R], ibb[R];                       // squared Gram-Schmidt norms, their inverses
    int64_t q[R];                               // size-reduction / elimination multipliers
};

PFG_HD int gix(int i, int j) { return i >= j ? ((i * (i + 1)) >> 1) + j : ((j * (j + 1)) >> 1) + i; }
PFG_HD int mix(int k, int j) { return ((k * (k - 1)) >> 1) + j; }
// packed lower-triangle index e -> (i, j), j <= i
PFG_HD void tri_of(int e, int &i, int &j)
{
    int r = (int)((sqrt(8.0 * e + 1.0) - 1.0) * 0.5);
    while (((r + 1) * (r + 2) >> 1) <= e) ++r;
    while ((r * (r + 1) >> 1) > e) --r;
    i = r;
    j = e - ((r * (r + 1)) >> 1);
}

// Cold working arrays of one warp (global memory), plus an LllMem for the
// h11 > 32 path.
struct SetupScratch {
    int64_t Z[MH * MH];
    int64_t V[MH * MH];             // unimodular transforms / temporaries
    int64_t S[MH * MH];
    double X[MH * MH];              // U^-1 for the certificate
    int64_t w[MH], v[MH];
    int order[MH];
    LllMem<MH> core;
    int64_t Bstore[(MH - 1) * MH];  // the rows of the warp's LllMem (core or the shared-memory one)
};

struct SetupArgs {
    const Geo *geo;
    const int64_t *kappa, *Mbasis, *ps;     // ps: (n, MH)
    const int32_t *pgeo;
    const int64_t *slab_off;                // slab offset per direction
    int64_t *slab;
    Dir *dirs;
    SetupScratch *scratch;                  // one per warp
    int n;                                  // entries of todo
    unsigned *next;                         // work counter
    const int32_t *todo;                    // directions to set up (null: 0..n-1)
    int smem_core;                          // 1: the LllMem<32> lives in dynamic shared memory
    double gcd_min_tree;                    // GCD rows only for trees estimated at >= this many
                                            // nodes (<= 0: always)
    // split form (the batched path): phase 2 queues the directions that want GCD
    // rows into rows_list (rows_count entries) for phase 3; null: phase 2 builds them
    int32_t *rows_list;
    unsigned *rows_count;
    const unsigned *n_dev;                  // if set, the number of todo entries (device)
};

// Per-stage cycle accounting of the setup, compiled in only with
// -DPFG_STAGE_CLOCKS (a profiling build): lane 0 adds the clock64() cycles
// spent in each stage to pfg_stage_cycles[stage & 31]; counters [32..34]
// count LLL calls, swaps and size-reduction passes with non-zero
// multipliers, [40..43] the cycles in the LLL's Gram-Schmidt rows, Babai
// loops, exact updates and swaps, [44..45] the Gram-Schmidt rows and Babai
// loops run.
#ifdef PFG_STAGE_CLOCKS
__device__ unsigned long long pfg_stage_cycles[64];
struct StageClock {
    int &stage;
    int lane;
    long long t;
    __device__ StageClock(int &s, int l) : stage(s), lane(l), t(0)
    {
#ifdef __CUDA_ARCH__
        t = clock64();
#endif
    }
    __device__ void mark(int s)
    {
#ifdef __CUDA_ARCH__
        if (lane == 0) {
            long long n = clock64();
            atomicAdd(&pfg_stage_cycles[stage & 31], (unsigned long long)(n - t));
            t = n;
        }
#endif
        stage = s;
    }
    __device__ ~StageClock() { mark(stage); }
};
#define PFG_COUNT(i, v) do { if ((threadIdx.x & 31) == 0) atomicAdd(&pfg_stage_cycles[32 + (i)], (unsigned long long)(v)); } while (0)
#define PFG_T0(t) const long long t = clock64()
#define PFG_TACC(i, t) PFG_COUNT(i, clock64() - (t))
#else
struct StageClock {
    int &stage;
    __device__ StageClock(int &s, int) : stage(s) {}
    __device__ void mark(int s) { stage = s; }
};
#define PFG_COUNT(i, v) do { } while (0)
#define PFG_T0(t) do { } while (0)
#define PFG_TACC(i, t) do { } while (0)
#endif

__device__ __forceinline__ double warp_sum(double x)
{
    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(FULL, x, o);
    return x;
}

__device__ __forceinline__ bool warp_any(bool b) { return __any_sync(FULL, b); }

__device__ __forceinline__ i128 shfl_xor_i128(i128 x, int m)
{
    uint64_t lo = (uint64_t)x;
    long long hi = (long long)(x >> 64);
    lo = __shfl_xor_sync(FULL, lo, m);
    hi = __shfl_xor_sync(FULL, hi, m);
    return (i128)(((u128)(uint64_t)hi << 64) | lo);
}

// acc -= q * g; true on overflow
PFG_HD bool submul_ovf(i128 &acc, int64_t q, i128 g)
{
    i128 t;
    if (mul_ovf((i128)q, g, &t)) return true;
    return sub_ovf(acc, t, &acc);
}

// ---------------------------------------------------------------------------
// Warp LLL (Schnorr-Euchner style) on the m rows of B (length n) with the
// exact Gram over M = m + has_last rows; row m is 'last', size-reduced
// against the reduced rows at the end.  Row and Gram updates are exact
// (checked int64 / int128); the FP64 Gram-Schmidt data only choose the
// unimodular steps and are recomputed from the exact Gram whenever a row is
// visited.  Returns 0, or ST_OVERFLOW on an int64/int128 overflow, a
// non-positive Gram-Schmidt norm, or when the iteration budget runs out.
// ---------------------------------------------------------------------------
template <int N> struct Lll {
    LllMem<N> *S;
    int n, M;
};

// mu(k, j) (j < k) and bb[k] from G(k, .) and the rows above: r_j = mu_kj
// bb_j solves the unit lower-triangular system r_j = G_kj - sum_{l<j} mu_jl
// r_l (forward substitution by columns, lanes own rows); afterwards lane l
// holds r_l, so mu_kl = r_l / bb_l and bb_k = G_kk - sum_l mu_kl r_l are
// formed in parallel.
template <int N> PFG_NOINLINE __device__ void lll_gs(LllMem<N> *S, int k, int lane)
{
    PFG_T0(t_gs);
    PFG_COUNT(12, 1);
    double a0 = lane < k ? (double)S->G[gix(k, lane)] : 0.0;
    double a1 = 0.0;
    if (N > 32) a1 = lane + 32 < k ? (double)S->G[gix(k, lane + 32)] : 0.0;
    for (int j = 0; j < k - 1; ++j) {
        const double rj = __shfl_sync(FULL, (N > 32 && j >= 32) ? a1 : a0, j & 31);
        if (lane > j && lane < k) a0 = fma(-S->mu[mix(lane, j)], rj, a0);
        if (N > 32 && lane + 32 > j && lane + 32 < k) a1 = fma(-S->mu[mix(lane + 32, j)], rj, a1);
    }
    double *muk = S->mu + mix(k, 0);
    double s = 0.0;
    if (lane < k) {
        const double m = a0 * S->ibb[lane];
        muk[lane] = m;
        s = m * a0;
    }
    if (N > 32 && lane + 32 < k) {
        const double m = a1 * S->ibb[lane + 32];
        muk[lane + 32] = m;
        s = fma(m, a1, s);
    }
    s = warp_sum(s);
    if (lane == 0) {
        const double b = (double)S->G[gix(k, k)] - s;
        S->bb[k] = b;
        S->ibb[k] = 1.0 / b;
    }
    __syncwarp();
    PFG_TACC(8, t_gs);
}

// Size-reduce row k against rows 0..k-1: the multipliers q_j come from the
// Gram-Schmidt row (Babai), then b_k -= sum_j q_j b_j in one exact pass over
// B and G; repeated until no multiplier is non-zero.  Leaves row k's
// Gram-Schmidt data current.
template <int N> PFG_LLL_INLINE __device__ int lll_reduce(Lll<N> &L, int k, int lane)
{
    LllMem<N> *S = L.S;
    for (int pass = 0; pass < 16; ++pass) {
        PFG_T0(t_q);
        PFG_COUNT(13, 1);
        double r0 = lane < k ? S->mu[mix(k, lane)] : 0.0;
        double r1 = 0.0;
        if (N > 32) r1 = lane + 32 < k ? S->mu[mix(k, lane + 32)] : 0.0;
        // Babai from j = k-1 down: q_j = rint(x_j) of the running coefficient,
        // which is 0 exactly when |x_j| <= 1/2; so only the rows whose running
        // coefficient is outside [-1/2, 1/2] (or NaN, which fails the range
        // check) are visited, highest first, found by ballot.
        uint64_t qmask = 0;                             // rows j with q_j != 0 (uniform)
        int64_t q0 = 0, q1 = 0;                         // q_lane, q_{lane+32}
        int top = k;
        for (;;) {
            uint64_t cand = __ballot_sync(FULL, lane < top && !(fabs(r0) <= 0.5));
            if (N > 32) cand |= (uint64_t)__ballot_sync(FULL, lane + 32 < top && !(fabs(r1) <= 0.5)) << 32;
            if (!cand) break;
            const int j = 63 - __clzll((long long)cand);
            const double x = __shfl_sync(FULL, (N > 32 && j >= 32) ? r1 : r0, j & 31);
            const double qd = rint(x);
            PFG_UNIFORM(qd);
            if (!(fabs(qd) <= 9.0e18)) return ST_OVERFLOW;
            qmask |= 1ull << j;
            if (lane == (j & 31)) {
                if (N > 32 && j >= 32) q1 = (int64_t)qd;
                else q0 = (int64_t)qd;
            }
            if (lane < j) r0 = fma(-qd, S->mu[mix(j, lane)], r0);
            if (N > 32 && lane + 32 < j) r1 = fma(-qd, S->mu[mix(j, lane + 32)], r1);
            top = j;
        }
        PFG_TACC(9, t_q);
        if (!qmask) return 0;
        PFG_COUNT(2, 1);
        PFG_T0(t_u);
        if (lane < k) S->q[lane] = q0;
        if (N > 32 && lane + 32 < k) S->q[lane + 32] = q1;
        __syncwarp();                                   // q[] visible to all lanes
        bool bad = false;
        // new row k of B (lanes own columns)
        i128 b0 = 0, b1 = 0;
        if (lane < L.n) {
            b0 = S->B[k * N + lane];
            for (uint64_t m = qmask; m; m &= m - 1) {
                const int j = __ffsll((long long)m) - 1;
                bad |= submul_ovf(b0, S->q[j], (i128)S->B[j * N + lane]);
            }
        }
        if (N > 32 && lane + 32 < L.n) {
            b1 = S->B[k * N + lane + 32];
            for (uint64_t m = qmask; m; m &= m - 1) {
                const int j = __ffsll((long long)m) - 1;
                bad |= submul_ovf(b1, S->q[j], (i128)S->B[j * N + lane + 32]);
            }
        }
        bad |= !fits64(b0) || !fits64(b1);
        // new G(k, l), l != k (lanes own l)
        const int l0 = lane, l1 = lane + 32;
        i128 g0 = 0, g1 = 0;
        if (l0 < L.M && l0 != k) {
            g0 = S->G[gix(k, l0)];
            for (uint64_t m = qmask; m; m &= m - 1) {
                const int j = __ffsll((long long)m) - 1;
                bad |= submul_ovf(g0, S->q[j], S->G[gix(j, l0)]);
            }
        }
        if (N > 32 && l1 < L.M && l1 != k) {
            g1 = S->G[gix(k, l1)];
            for (uint64_t m = qmask; m; m &= m - 1) {
                const int j = __ffsll((long long)m) - 1;
                bad |= submul_ovf(g1, S->q[j], S->G[gix(j, l1)]);
            }
        }
        // G'(k, k) = G(k, k) - sum_{l<k} q_l (G(k, l) + G'(k, l))
        i128 t = 0;
        if (l0 < k && S->q[l0]) {
            i128 u, v;
            bad |= add_ovf(S->G[gix(k, l0)], g0, &u);
            bad |= mul_ovf((i128)S->q[l0], u, &v);
            t = v;
        }
        if (N > 32 && l1 < k && S->q[l1]) {
            i128 u, v;
            bad |= add_ovf(S->G[gix(k, l1)], g1, &u);
            bad |= mul_ovf((i128)S->q[l1], u, &v);
            bad |= add_ovf(t, v, &t);
        }
        for (int o = 16; o; o >>= 1) bad |= add_ovf(t, shfl_xor_i128(t, o), &t);
        i128 gkk;
        bad |= sub_ovf(S->G[gix(k, k)], t, &gkk);
        if (warp_any(bad)) return ST_OVERFLOW;
        __syncwarp();                                   // every lane has read the old row k
        if (lane < L.n) S->B[k * N + lane] = (int64_t)b0;
        if (N > 32 && lane + 32 < L.n) S->B[k * N + lane + 32] = (int64_t)b1;
        if (l0 < L.M && l0 != k) S->G[gix(k, l0)] = g0;
        if (N > 32 && l1 < L.M && l1 != k) S->G[gix(k, l1)] = g1;
        if (lane == 0) S->G[gix(k, k)] = gkk;
        __syncwarp();
        PFG_TACC(10, t_u);
        lll_gs(S, k, lane);
    }
    return 0;
}

// Exchange rows k-1 and k: B, G exactly; the Gram-Schmidt data of the two
// rows by the usual update formulas (rows > k are recomputed when visited).
template <int N> PFG_LLL_INLINE __device__ void lll_swap(Lll<N> &L, int k, int lane)
{
    LllMem<N> *S = L.S;
    for (int c = lane; c < L.n; c += 32) {
        const int64_t t = S->B[k * N + c];
        S->B[k * N + c] = S->B[(k - 1) * N + c];
        S->B[(k - 1) * N + c] = t;
    }
    for (int l = lane; l < L.M; l += 32) {
        if (l == k || l == k - 1) continue;
        const i128 t = S->G[gix(k, l)];
        S->G[gix(k, l)] = S->G[gix(k - 1, l)];
        S->G[gix(k - 1, l)] = t;
    }
    for (int j = lane; j < k - 1; j += 32) {
        const double t = S->mu[mix(k, j)];
        S->mu[mix(k, j)] = S->mu[mix(k - 1, j)];
        S->mu[mix(k - 1, j)] = t;
    }
    if (lane == 0) {
        const i128 t = S->G[gix(k, k)];
        S->G[gix(k, k)] = S->G[gix(k - 1, k - 1)];
        S->G[gix(k - 1, k - 1)] = t;
        // one division: 1/bb'_k = Bn / (b1 b2) from the old inverses
        const double m = S->mu[mix(k, k - 1)], b1 = S->bb[k - 1], b2 = S->bb[k];
        const double Bn = k == 1 ? (double)S->G[0] : fma(m * m, b1, b2);
        const double iBn = 1.0 / Bn;
        S->mu[mix(k, k - 1)] = m * b1 * iBn;
        S->bb[k] = b1 * b2 * iBn;
        S->bb[k - 1] = Bn;
        S->ibb[k] = Bn * S->ibb[k - 1] * S->ibb[k];
        S->ibb[k - 1] = iBn;
    }
    __syncwarp();
}

template <int N> PFG_NOINLINE __device__ int warp_lll(Lll<N> &L, int m, bool has_last, double delta, int lane)
{
    LllMem<N> *S = L.S;
    L.M = m + (has_last ? 1 : 0);
    PFG_COUNT(0, 1);
    if (m >= 1) {
        lll_gs(S, 0, lane);
        if (!(S->bb[0] > 0)) return ST_NONPOS;
    }
    if (m >= 2) lll_gs(S, 1, lane);
    int k = 1, iters = 0;
    while (k < m) {
        if (++iters > 200000) return ST_OVERFLOW;
        int st = lll_reduce(L, k, lane);
        if (st) return st;
        const double bk = S->bb[k], mk = S->mu[mix(k, k - 1)], bk1 = S->bb[k - 1];
        PFG_UNIFORM(bk);
        __syncwarp();                       // (every lane has read them before lll_swap writes)
        if (!(bk > 0)) return ST_NONPOS;
        if (bk < (delta - mk * mk) * bk1) {
            PFG_T0(t_s);
            lll_swap(L, k, lane);
            PFG_TACC(11, t_s);
            PFG_COUNT(1, 1);
            if (k > 1) --k;
        } else {
            ++k;
            if (k < m) lll_gs(S, k, lane);
        }
    }
    if (has_last && m > 0) {
        lll_gs(S, m, lane);
        int st = lll_reduce(L, m, lane);
        if (st) return st;
    }
    return 0;
}

// Euclidean Gram of rows 0..m-1 of B (length n); true on overflow
template <int N> PFG_NOINLINE __device__ bool gram_euclid(LllMem<N> *S, int m, int n, int lane)
{
    bool bad = false;
    for (int e = lane; e < (m * (m + 1)) / 2; e += 32) {
        int i, j;
        tri_of(e, i, j);
        i128 s = 0;
        for (int c = 0; c < n; ++c)
            if (add_ovf(s, (i128)S->B[i * N + c] * S->B[j * N + c], &s)) bad = true;
        S->G[e] = s;
    }
    __syncwarp();
    return warp_any(bad);
}

// Exchange rows a and b (any positions) of B and G; Gram-Schmidt data become stale.
template <int N> PFG_NOINLINE __device__ void lll_exchange(Lll<N> &L, int a, int b, int lane)
{
    if (a == b) return;
    LllMem<N> *S = L.S;
    for (int c = lane; c < L.n; c += 32) {
        const int64_t t = S->B[a * N + c];
        S->B[a * N + c] = S->B[b * N + c];
        S->B[b * N + c] = t;
    }
    for (int l = lane; l < L.M; l += 32) {
        if (l == a || l == b) continue;
        const i128 t = S->G[gix(a, l)];
        S->G[gix(a, l)] = S->G[gix(b, l)];
        S->G[gix(b, l)] = t;
    }
    if (lane == 0) {
        const i128 t = S->G[gix(a, a)];
        S->G[gix(a, a)] = S->G[gix(b, b)];
        S->G[gix(b, b)] = t;
    }
    __syncwarp();
}

// One elimination step of column col over rows 0..nr-1 with pivot row pr:
// b_r -= floor(b_r[col] / b_pr[col]) b_pr for every r != pr, exactly, with
// the Gram updated as E G E^T.  True on overflow.
template <int N> PFG_NOINLINE __device__ bool echelon_step(Lll<N> &L, int nr, int pr, int col, int lane)
{
    LllMem<N> *S = L.S;
    const int64_t piv = S->B[pr * N + col];
    for (int r = lane; r < nr; r += 32) S->q[r] = r == pr ? 0 : fdiv64(S->B[r * N + col], piv);
    for (int l = lane; l < nr; l += 32) S->T[l] = S->G[gix(pr, l)];
    __syncwarp();
    bool bad = false;
    for (int c = lane; c < L.n; c += 32) {
        const int64_t bp = S->B[pr * N + c];
        for (int r = 0; r < nr; ++r) {
            const int64_t qr = S->q[r];
            if (!qr) continue;
            const i128 x = (i128)S->B[r * N + c] - (i128)qr * bp;
            if (!fits64(x)) { bad = true; continue; }
            S->B[r * N + c] = (int64_t)x;
        }
    }
    const i128 tp = S->T[pr];
    for (int e = lane; e < (nr * (nr + 1)) / 2; e += 32) {
        int r, l;
        tri_of(e, r, l);
        const int64_t qr = S->q[r], ql = S->q[l];
        if (!qr && !ql) continue;
        i128 g;
        if (r == pr || l == pr) {                      // <b_o - q_o b_pr, b_pr>
            const int o = r == pr ? l : r;
            g = S->T[o];
            bad |= submul_ovf(g, S->q[o], tp);
        } else {                                       // G - q_r T_l - q_l T_r + q_r q_l T_pr
            g = S->G[e];
            bad |= submul_ovf(g, qr, S->T[l]);
            bad |= submul_ovf(g, ql, S->T[r]);
            i128 qq = (i128)qr * ql, t;
            if (mul_ovf(qq, tp, &t) || add_ovf(g, t, &g)) bad = true;
        }
        S->G[e] = g;
    }
    __syncwarp();
    return warp_any(bad);
}

// warp argmin over rows r < nr of |B[r][col]| != 0 (-1 if the column is 0)
template <int N> PFG_NOINLINE __device__ int argmin_nonzero(const int64_t *B, int nr, int col, int lane)
{
    uint64_t best = ~0ull;
    int who = -1;
    for (int r = lane; r < nr; r += 32) {
        uint64_t a = uabs64(B[r * N + col]);
        if (a && a < best) { best = a; who = r; }
    }
    for (int o = 16; o; o >>= 1) {
        uint64_t ob = __shfl_xor_sync(FULL, best, o);
        int ow = __shfl_xor_sync(FULL, who, o);
        if (ob < best || (ob == best && ow >= 0 && (who < 0 || ow < who))) { best = ob; who = ow; }
    }
    return who;
}

// Unimodular U (n x n rows, stride MH, into Uo) with U v = (gcd, 0, ..., 0)
// by Bezout steps on (w0, wk) (as pfl_unimodular, pfvs/fp_kernel/pfv_lattice.h:
// 162-188), with one change against coefficient growth: the coordinates are
// first permuted so that a coprime pair of entries of v / gcd(v) (the one
// with the smallest larger entry) comes first.  After the first step the
// running gcd is then 1, every later step is (1, w_k) -> (1, 0), and the
// entries stay below about max|v|^2 instead of compounding.  Any unimodular
// U gives the same lattice; v is read from vin (length n).
PFG_NOINLINE __device__ int warp_unimodular(const int64_t *vin, int n, int64_t *Uo, int64_t *wtmp, int *perm, int lane)
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

#ifndef PFG_DELTA_H
#define PFG_DELTA_H 0.75        // LLL parameter of the GCD-row reductions (they only keep the rows'
                                // entries small: any echelon basis of the row lattice prunes the
                                // same; against 0.99, 2 % less setup time on the mixed batch, and
                                // the rows that stay within int64 differ in a handful of directions,
                                // whose trees then differ by a few nodes)
#endif
#ifndef PFG_DELTA_O
#define PFG_DELTA_O 0.5         // LLL parameter of the Euclidean reduction of O (it only has to
                                // keep the entries small: the search basis is reduced again w.r.t.
                                // mat with PFG_DELTA_K; 0.5 takes 14 % less setup time than 0.99 for
                                // the same tree sizes)
#endif
#ifndef PFG_DELTA_K
#define PFG_DELTA_K 0.99        // LLL parameter of the cut-aware basis (the search basis)
#endif

// ---------------------------------------------------------------------------
// Exact proof that a symmetric integer matrix A (d x d, row-major) is NOT
// positive definite, for the directions whose FP64 factorization fails.
//
// An FP64 Cholesky A = U^T U runs until a pivot fails (or, if none does, to
// the pivot j with the smallest ratio pivot / A_jj).  With y the solution of
// A[<j, <j] y = A[<j, j] through the computed factor, x = (-y, 1, 0, ..) has
// x^T A x = A_jj - A[j, <j] y, the Schur complement the pivot estimates.  x
// is scaled by a power of two D = 2^t and rounded to integers, and x^T A x
// is evaluated exactly in int128.  A value <= 0 at the nonzero integer x
// proves A is not positive definite -- the decision the reference's exact
// Bareiss factorization reaches by a non-positive leading minor (status -9,
// fpk_common.h:259-309; Sylvester's criterion).  Rounding only moves x^T A x
// by O(D |x| |A|) against D^2 times the Schur complement, so a clearly
// negative pivot always gives a witness.  Returns false when none is found:
// A may still be indefinite with a pivot lost in rounding, or positive
// definite and too ill-conditioned to certify.  U: d*d doubles, y: d doubles
// of scratch (y is reused for the integer witness).
// ---------------------------------------------------------------------------
__device__ bool witness_not_pd(const int64_t *A, int d, double *U, double *y, int lane)
{
    int jw = -1;                                // the pivot the witness is built at
    double rmin = 1.0;
    for (int j = 0; j < d; ++j) {
        if (A[j * d + j] <= 0) return true;     // e_j itself: e_j^T A e_j = A_jj <= 0
        double s0 = 0.0;
        for (int k = 0; k < j; ++k) { const double u = U[k * d + j]; s0 += u * u; }
        const double ajj = (double)A[j * d + j], pj = ajj - s0;
        if (!(pj > 0)) { jw = j; break; }
        if (pj / ajj < rmin) { rmin = pj / ajj; jw = j; }
        const double ujj = sqrt(pj);
        for (int i = j + 1 + lane; i < d; i += 32) {
            double s = 0.0;
            for (int k = 0; k < j; ++k) s += U[k * d + j] * U[k * d + i];
            U[j * d + i] = ((double)A[j * d + i] - s) / ujj;
        }
        if (lane == 0) U[j * d + j] = ujj;
        __syncwarp();
    }
    PFG_UNIFORM(jw);
    if (jw <= 0) return false;
    const int j = jw, n = j + 1;
    // z = U[<j, j] (the forward substitution U^T z = A[<j, j] is column j of
    // U's first j rows), then U[<j, <j] y = z backwards
    for (int i = j - 1; i >= 0; --i) {
        double s = 0.0;
        for (int k = i + 1 + lane; k < j; k += 32) s += U[i * d + k] * y[k];
        s = warp_sum(s);
        if (lane == 0) y[i] = (U[i * d + j] - s) / U[i * d + i];
        __syncwarp();
    }
    double ymax = 1.0;
    uint64_t amax = 1;
    for (int i = lane; i < j; i += 32) ymax = fmax(ymax, fabs(y[i]));
    for (int e = lane; e < n * n; e += 32) {
        const uint64_t a = uabs64(A[(e / n) * d + e % n]);
        amax = a > amax ? a : amax;
    }
    for (int o = 16; o; o >>= 1) {
        ymax = fmax(ymax, __shfl_xor_sync(FULL, ymax, o));
        const uint64_t t = __shfl_xor_sync(FULL, amax, o);
        amax = t > amax ? t : amax;
    }
    if (!(ymax < 1e300)) return false;
    // |x| < 2^xb with 2 xb + bits(amax) + 2 bits(n) <= 124 keeps every partial sum of
    // x^T A x inside int128 (the checked arithmetic below still guards it)
    const int bits_a = 64 - __clzll((long long)amax), bits_n = 32 - __clz(n);
    const int xb = min(60, (124 - bits_a - 2 * bits_n) / 2);
    int ey = 0;
    frexp(ymax, &ey);                           // ymax < 2^ey
    const int t = xb - ey - 1;
    if (t < 0) return false;
    const double D = ldexp(1.0, t);
    int64_t *x = (int64_t *)y;
    for (int i = lane; i < n; i += 32) x[i] = i < j ? (int64_t)llrint(-y[i] * D) : ((int64_t)1 << t);
    __syncwarp();
    bool bad = false;
    i128 qf = 0;
    for (int i = lane; i < n; i += 32) {
        i128 r = 0, tt;
        for (int k = 0; k < n; ++k)
            if (mul_ovf((i128)A[i * d + k], (i128)x[k], &tt) || add_ovf(r, tt, &r)) bad = true;
        if (mul_ovf(r, (i128)x[i], &tt) || add_ovf(qf, tt, &qf)) bad = true;
    }
    for (int o = 16; o; o >>= 1) {
        const i128 other = shfl_xor_i128(qf, o);
        if (add_ovf(qf, other, &qf)) bad = true;
    }
    if (warp_any(bad)) return false;
    return qf <= 0;
}

// ---------------------------------------------------------------------------
// The setup of one direction in three phases, each a kernel of its own in the
// batched path so that the warps of an SM run the same code (the phases'
// code together does not fit the instruction caches).  They share only the
// direction's slab (BT, ZT, MAT, U, H) and Dir; S is the warp's LLL working
// set (N >= h11).  Each returns ST_PENDING to go on, else the final status.
//   phase 0: steps 1-7 (Z, v, orthogonal lattice, Euclidean LLL, Binter, mat)
//   phase 1: step 8 (cut-aware basis)
//   phase 2: step 10 (Cholesky and certificate, tree estimate), then 9 and 11
//            (GCD rows, bounds) -- or, in the split form, 11 only for the
//            directions without GCD rows, the others queued for
//   phase 3: steps 9 and 11 of the queued directions (the GCD rows of the
//            large trees then run side by side instead of trailing phase 2)
// ---------------------------------------------------------------------------
template <int N> __device__ int setup_phase0(const SetupArgs &A, int pid, int lane, int &stage, LllMem<N> *S)
{
    SetupScratch *W = A.scratch + (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5));
    const Geo g = A.geo[A.pgeo[pid]];
    const int h = g.h, d = h - 1;
    const int64_t *kap = A.kappa + g.koff, *Mb = A.Mbasis + g.moff, *p = A.ps + (int64_t)pid * MH;
    int64_t *slab = A.slab + A.slab_off[pid];
    const Slab L = slab_layout(h, d);
    Dir &D = A.dirs[pid];
    bool bad = false;
    StageClock clk(stage, lane);
    (void)D;

    clk.mark(1);
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
    clk.mark(2);
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
    clk.mark(3);
    // 3. orthogonal lattice: rows 1.. of the unimodular transform of v
    int st = warp_unimodular(W->v, h, W->V, W->w, W->order, lane);
    if (st) return st;
    for (int e = lane; e < d * h; e += 32) S->B[(e / h) * N + e % h] = W->V[(e / h + 1) * MH + e % h];
    __syncwarp();
    clk.mark(4);
    // 4. Euclidean LLL of O
    if (gram_euclid<N>(S, d, h, lane)) return ST_OVERFLOW;
    {
        Lll<N> LL{S, h, d};
        if ((st = warp_lll(LL, d, false, PFG_DELTA_O, lane))) return st == ST_NONPOS ? ST_OVERFLOW : st;
    }
    clk.mark(5);
    // 5. (Mbasis O^T)^T rows, 6. coni order (rows with entry 0 == 0 first, stable)
    for (int e = lane; e < d * h; e += 32) {
        int a = e / h, i = e % h;
        i128 s = 0;
        for (int l = 0; l < h; ++l)
            if (add_ovf(s, (i128)Mb[i * h + l] * S->B[a * N + l], &s)) bad = true;
        if (!fits64(s)) bad = true;
        W->S[a * MH + i] = (int64_t)s;
    }
    __syncwarp();
    if (warp_any(bad)) return ST_OVERFLOW;
    if (lane == 0) {
        int no = 0;
        if (g.coni) {
            for (int a = 0; a < d; ++a) if (W->S[a * MH] == 0) W->order[no++] = a;
            for (int a = 0; a < d; ++a) if (W->S[a * MH] != 0) W->order[no++] = a;
        } else {
            for (int a = 0; a < d; ++a) W->order[no++] = a;
        }
    }
    __syncwarp();
    int64_t *BT = slab + L.bt, *ZT = slab + L.zt, *MAT = slab + L.mat;
    for (int e = lane; e < d * h; e += 32) BT[e] = W->S[W->order[e / h] * MH + e % h];
    __syncwarp();
    clk.mark(7);
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
    return ST_PENDING;
}

template <int N> __device__ int setup_phase1(const SetupArgs &A, int pid, int lane, int &stage, LllMem<N> *S)
{
    SetupScratch *W = A.scratch + (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5));
    const Geo g = A.geo[A.pgeo[pid]];
    const int h = g.h, d = h - 1;
    const int64_t *kap = A.kappa + g.koff, *Mb = A.Mbasis + g.moff, *p = A.ps + (int64_t)pid * MH;
    int64_t *slab = A.slab + A.slab_off[pid];
    const Slab L = slab_layout(h, d);
    Dir &D = A.dirs[pid];
    bool bad = false;
    StageClock clk(stage, lane);
    (void)kap; (void)Mb; (void)p;
    int64_t *BT = slab + L.bt, *ZT = slab + L.zt, *MAT = slab + L.mat;
    int st = 0;
    clk.mark(8);
    // 8. cut-aware basis (pfv_lattice.h:554-602); without an M0 cut (a non-coni
    // geometry) the whole basis LLL-reduced w.r.t. mat instead (pfv_lattice.h:560-566)
    bool lnz = !g.coni;
    if (g.coni) {
        for (int a = lane; a < d; a += 32) W->v[a] = BT[a * h];
        __syncwarp();
        for (int a = lane; a < d; a += 32) lnz |= W->v[a] != 0;
        lnz = warp_any(lnz);
    }
    int m0_level = -1;
    int64_t g_lin = 0;
    if (lnz && !g.coni) {
        // B = the identity, its Gram w.r.t. mat is mat itself
        for (int e = lane; e < d * d; e += 32) S->B[(e / d) * N + e % d] = (e / d) == (e % d);
        for (int e = lane; e < d * d; e += 32) {
            const int i = e / d, j = e % d;
            if (j <= i) S->G[gix(i, j)] = (i128)MAT[i * d + j];
        }
        __syncwarp();
    } else if (lnz) {
        if ((st = warp_unimodular(W->v, d, W->V, W->w, W->order, lane))) return st;
        // B rows 0..d-2 = K = V[1..], row d-1 = w = V[0]
        for (int e = lane; e < d * d; e += 32) {
            int a = e / d, c = e % d;
            S->B[a * N + c] = a < d - 1 ? W->V[(a + 1) * MH + c] : W->V[c];
        }
        __syncwarp();
    }
    if (lnz && g.coni) {
        // Gram w.r.t. mat: G_ij = B_i^T mat B_j  (T holds mat B_j)
        for (int j = 0; j < d; ++j) {
            for (int c = lane; c < d; c += 32) {
                i128 s = 0;
                for (int k = 0; k < d; ++k)
                    if (add_ovf(s, (i128)MAT[c * d + k] * S->B[j * N + k], &s)) bad = true;
                S->T[c] = s;
            }
            __syncwarp();
            for (int i = lane; i <= j; i += 32) {
                i128 s = 0, t;
                for (int c = 0; c < d; ++c) {
                    if (!S->B[i * N + c]) continue;
                    if (mul_ovf(S->T[c], (i128)S->B[i * N + c], &t) || add_ovf(s, t, &s)) bad = true;
                }
                S->G[gix(j, i)] = s;
            }
            __syncwarp();
        }
        if (warp_any(bad)) return ST_OVERFLOW;
    }
    if (lnz) {
        {
            Lll<N> LK{S, d, d};
            // (coni: the d - 1 rows spanning ker l, then w size-reduced; else all d rows)
            if ((st = g.coni ? warp_lll(LK, d - 1, true, PFG_DELTA_K, lane) : warp_lll(LK, d, false, PFG_DELTA_K, lane))) {
                // a non-positive norm under mat: not positive definite when an
                // integer witness says so (exact), else not decided here
                if (st == ST_NONPOS)
                    st = witness_not_pd(MAT, d, W->X, W->X + d * d, lane) ? ST_NOT_PD : ST_PRECISION;
                return st;
            }
        }
        // new columns a of Binter: sum_b B[a][b] Binter[:, b]  (likewise ZB)
        for (int e = lane; e < d * h; e += 32) {
            int a = e / h, r = e % h;
            i128 s = 0, t = 0;
            for (int b = 0; b < d; ++b) {
                s += (i128)S->B[a * N + b] * BT[b * h + r];
                t += (i128)S->B[a * N + b] * ZT[b * h + r];
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
            i128 x = S->G[gix(e / d, e % d)];
            if (!fits64(x)) bad = true;
            MAT[e] = (int64_t)x;
        }
        __syncwarp();
        if (warp_any(bad)) return ST_OVERFLOW;
        if (g.coni) {
            for (int a = lane; a < d - 1; a += 32) bad |= BT[a * h] != 0;
            if (warp_any(bad)) return ST_OVERFLOW;      // (cannot happen: K spans ker l)
            m0_level = d - 1;
            g_lin = BT[(d - 1) * h];
        }
    } else if (g.linmin > 0) {
        if (lane == 0) { D.m0_level = -1; D.g_lin = 0; }
        return ST_EMPTY;
    }
    if (lane == 0) { D.m0_level = m0_level; D.g_lin = g_lin; }
    __syncwarp();
    return ST_PENDING;
}

// Steps 9 and 11 of one direction: its GCD rows (when wanted) and the int64
// bounds of the search's sums.
template <int N> __device__ int setup_rows_bounds(const SetupArgs &A, int pid, int lane, int &stage, LllMem<N> *S,
                                                  bool want_rows, double slack_chol)
{
    SetupScratch *W = A.scratch + (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5));
    const Geo g = A.geo[A.pgeo[pid]];
    const int h = g.h, d = h - 1;
    const int64_t *p = A.ps + (int64_t)pid * MH;
    int64_t *slab = A.slab + A.slab_off[pid];
    const Slab L = slab_layout(h, d);
    Dir &D = A.dirs[pid];
    bool bad = false;
    StageClock clk(stage, lane);
    int64_t *BT = slab + L.bt, *ZT = slab + L.zt, *MAT = slab + L.mat;
    int64_t *H = slab + L.H;
    for (int e = lane; e < d * d; e += 32) H[e] = 0;
    uint64_t hrows = 0;
    clk.mark(9);
    // 9. GCD rows: echelon basis of the row lattice of ZB[1:] with small rows.
    // The rows r_k = ZB[k][:], k = 1..d, satisfy sum_k p_k r_k = 0 (p^T Z Binter
    // = 0 and p_0 = 0); with V p' = e0 from Bezout steps, the rows of V^-T R
    // are the rows of R with row 0 = p'^T R = 0: drop it, the rest is a basis.
    // (Lanes own columns here, so the row operations need no staging.)  The
    // rows only prune: when one cannot be built, the search goes without it.
    // (A non-coni geometry cuts on all of K: the rows are those of ZB[0:], their
    // relation p, and nin = h rows in, h - 1 out; LllMem<N> holds N - 1 >= h rows.)
    const int r0 = g.coni ? 1 : 0, nin = h - r0;
    if (want_rows) {
        for (int c = lane; c < d; c += 32)
            for (int r = 0; r < nin; ++r) S->B[r * N + c] = ZT[c * h + r + r0];
        for (int e = lane; e < nin; e += 32) W->w[e] = p[e + r0];
        __syncwarp();
        for (int k = 1; k < nin; ++k) {
            int64_t wk = W->w[k];
            if (wk == 0) continue;
            int64_t w0 = W->w[0], s, t;
            int64_t gg = xgcd_floor(w0, wk, &s, &t);
            int64_t m10 = -fdiv64(wk, gg), m11 = fdiv64(w0, gg);
            __syncwarp();
            if (lane == 0) { W->w[0] = gg; W->w[k] = 0; }
            for (int c = lane; c < d; c += 32) {
                i128 r0 = (i128)m11 * S->B[c] - (i128)m10 * S->B[k * N + c];
                i128 rk = -(i128)t * S->B[c] + (i128)s * S->B[k * N + c];
                if (!fits64(r0) || !fits64(rk)) { bad = true; continue; }
                S->B[c] = (int64_t)r0;
                S->B[k * N + c] = (int64_t)rk;
            }
            __syncwarp();
            if (warp_any(bad)) { bad = false; want_rows = false; break; }
        }
    }
    clk.mark(91);
    if (want_rows) {
        for (int c = lane; c < d; c += 32) bad |= S->B[c] != 0;
        if (warp_any(bad)) return ST_OVERFLOW;      // p'^T ZB[1:] must vanish exactly
    }
    if (want_rows) {
        int nr = nin - 1;
        for (int c = lane; c < d; c += 32)          // drop row 0
            for (int r = 0; r < nr; ++r) S->B[r * N + c] = S->B[(r + 1) * N + c];
        __syncwarp();
        // Rows whose construction would leave int64 (the last pivots are
        // large: the lattice of rows vanishing on all but the last columns has
        // a huge covolume) are not built: the rows found so far are kept, and
        // any set of rows of the lattice gives a valid GCD bound.
        if (nr > 0) {
            if (gram_euclid<N>(S, nr, d, lane)) goto h_done;
            Lll<N> LH{S, d, nr};
            if (warp_lll(LH, nr, false, PFG_DELTA_H, lane)) goto h_done;
            for (int col = 0; col < d && nr > 0; ++col) {
                int pr = -1;
                LH.M = nr;
                for (int it = 0; ; ++it) {
                    if (it > 256) goto h_done;
                    pr = argmin_nonzero<N>(S->B, nr, col, lane);
                    PFG_UNIFORM(pr);
                    if (pr < 0) break;
                    bool other = false;
                    for (int r = lane; r < nr; r += 32) other |= r != pr && S->B[r * N + col] != 0;
                    if (!warp_any(other)) break;
                    if (echelon_step(LH, nr, pr, col, lane)) goto h_done;
                }
                if (pr < 0) continue;
                // the pivot row to the end (index nr - 1), positive pivot
                lll_exchange(LH, pr, nr - 1, lane);
                const bool neg = S->B[(nr - 1) * N + col] < 0;
                PFG_UNIFORM(neg);
                __syncwarp();                   // (read by every lane before the owner negates it)
                if (neg) {
                    for (int c = lane; c < d; c += 32) S->B[(nr - 1) * N + c] = -S->B[(nr - 1) * N + c];
                    for (int l = lane; l < nr - 1; l += 32) S->G[gix(nr - 1, l)] = -S->G[gix(nr - 1, l)];
                    __syncwarp();
                }
                // LLL the rows below (rows 0..nr-2), size-reduce the pivot row against them
                if (warp_lll(LH, nr - 1, true, PFG_DELTA_H, lane)) goto h_done;
                bool fits = true;
                for (int c = lane; c < d; c += 32) fits &= uabs64(S->B[(nr - 1) * N + c]) < (1ull << 62);
                fits = __all_sync(FULL, fits);
                if (fits) {
                    // stored transposed (H[c d + col] = entry c of the row with pivot col): the
                    // search updates every row's prefix with column c when coordinate c changes
                    for (int c = lane; c < d; c += 32) H[c * d + col] = S->B[(nr - 1) * N + c];
                    hrows |= 1ull << col;
                }
                __syncwarp();
                --nr;
            }
        }
    }
h_done:
    clk.mark(11);
    // 11. the search keeps exact sums mat c, ZB c, Binter c in int64 and stages
    // mat and ZB^T as int32: every row of mat and every column of Binter^T and
    // (Z Binter)^T has an absolute sum below 2^31, so with |c| < 2^31 every such
    // sum (and every partial one) stays below 2^62.  A mat beyond that (a long,
    // thin ellipsoid) is read from the slab instead (Dir.wide), with its sums
    // bounded through the coordinate ranges below.
    bool wide = false;
    for (int r = lane; r < d; r += 32) {
        uint64_t s = 0;
        for (int j = 0; j < d; ++j) {
            const uint64_t a = uabs64(MAT[r * d + j]);
            if (a >= (1ull << 31)) wide = true; else s += a;
        }
        wide |= s >= (1ull << 31);
    }
    wide = warp_any(wide);
    if (wide) {
        // Every coordinate value the search visits lies in a level interval of the
        // ellipsoid |U c|^2 <= rho (rho = qmax plus the pruning slack), so
        // |c_j| <= sqrt(rho) |row j of U^-1| + 1; the bound is taken twice over
        // (FP64 rounding of U^-1 is far below that), and then every row's
        // sum |mat_rj| R_j must stay below 2^62.
        const double *Uf = (const double *)(slab + L.u64);
        double *X = W->X;
        for (int j = 0; j < d; ++j) {
            for (int i = lane; i <= j; i += 32) {
                double x;
                if (i == j) x = 1.0 / Uf[j * d + j];
                else {
                    double s = 0.0;
                    for (int k = i; k < j; ++k) s += X[i * MH + k] * Uf[k * d + j];
                    x = -s / Uf[j * d + j];
                }
                X[i * MH + j] = x;
            }
            __syncwarp();
        }
        const double rho = 2.0 * ((double)g.qmax + slack_chol) + 16.0;
        for (int j = lane; j < d; j += 32) {
            double rn = 0.0;
            for (int k = j; k < d; ++k) rn += X[j * MH + k] * X[j * MH + k];
            const double rj = 2.0 * sqrt(rho * rn) + 2.0;
            W->w[j] = rj < 2147483648.0 && rj == rj ? (int64_t)ceil(rj) : (int64_t)(1ll << 31);
        }
        __syncwarp();
        for (int r = lane; r < d; r += 32) {
            u128 s = 0;
            for (int j = 0; j < d; ++j) s += (u128)uabs64(MAT[r * d + j]) * (uint64_t)W->w[j];
            bad |= s >= ((u128)1 << 62);
        }
    }
    for (int r = lane; r < h; r += 32) {
        uint64_t sb = 0, sz = 0;
        for (int a = 0; a < d; ++a) {
            const uint64_t x = uabs64(BT[a * h + r]), y = uabs64(ZT[a * h + r]);
            if (x >= (1ull << 31) || y >= (1ull << 31)) bad = true;
            else { sb += x; sz += y; }
        }
        bad |= sb >= (1ull << 31) || sz >= (1ull << 31);
    }
    if (warp_any(bad)) return ST_OVERFLOW;
    if (lane == 0) {
        D.hrows = hrows;
        D.slack_chol = slack_chol;
        D.wide = wide;
    }
    __syncwarp();
    return ST_PENDING;
}

// Phase 3 (split form): the GCD rows and bounds of a direction phase 2 queued.
template <int N> __device__ int setup_phase3(const SetupArgs &A, int pid, int lane, int &stage, LllMem<N> *S)
{
    return setup_rows_bounds<N>(A, pid, lane, stage, S, true, A.dirs[pid].slack_chol);
}

template <int N> __device__ int setup_phase2(const SetupArgs &A, int pid, int lane, int &stage, LllMem<N> *S)
{
    SetupScratch *W = A.scratch + (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5));
    const Geo g = A.geo[A.pgeo[pid]];
    const int h = g.h, d = h - 1;
    int64_t *slab = A.slab + A.slab_off[pid];
    const Slab L = slab_layout(h, d);
    Dir &D = A.dirs[pid];
    StageClock clk(stage, lane);
    int64_t *MAT = slab + L.mat;
    const int m0_level = D.m0_level;
    const int64_t g_lin = D.g_lin;
    clk.mark(10);
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
    if (notpd)                               // not positive definite, or not decided here
        return witness_not_pd(MAT, d, U, W->X, lane) ? ST_NOT_PD : ST_PRECISION;
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
    if (!(gam * K <= 1e-3))                  // ill-conditioned: maybe not positive definite
        return witness_not_pd(MAT, d, U, W->X, lane) ? ST_NOT_PD : ST_PRECISION;
    const double slack_chol = 2.0 * gam * K * ((double)g.qmax + 1.0);
    float *U32 = (float *)(slab + L.u32);
    double *UI = (double *)(slab + L.ui64);
    float *UI32 = (float *)(slab + L.ui32);
    for (int e = lane; e < d * d; e += 32) U32[e] = (float)U[e];
    __syncwarp();
    for (int i = lane; i < d; i += 32) { UI[i] = 1.0 / U[i * d + i]; UI32[i] = 1.0f / U32[i * d + i]; }
    // Tree estimate (Gaussian heuristic): the points of the projected lattice
    // of the last k coordinates inside the ellipsoid's shadow, summed over k.
    // The GCD rows below only prune, so a direction whose tree is small
    // (or whose root interval is empty) is searched without them: building
    // them costs more than they could save there.
    bool want_rows = A.gcd_min_tree <= 0.0;
    if (!want_rows) {
        double est = 0.0;
        if (lane == 0) {
            const double lq = log((double)g.qmax + 1.0) + 1.1447298858494002;   // + log(pi)
            double ldet = 0.0;
            for (int k = 1; k <= d; ++k) {
                ldet += log(U[(d - k) * d + (d - k)]);
                est += exp(0.5 * k * lq - lgamma(0.5 * k + 1.0) - ldet);
            }
            if (m0_level == d - 1 && g.linmin > 0) {          // root interval under the M0 cut
                const double rmax = sqrt((double)g.qmax + slack_chol + 1.0) / U[(d - 1) * d + (d - 1)];
                const double cmin = ceil((double)g.linmin / fabs((double)g_lin));
                if (cmin > rmax * (1.0 + 1e-9) + 1e-9) est = 0.0;
            }
        }
        est = __shfl_sync(FULL, est, 0);
        want_rows = est >= A.gcd_min_tree;
    }
    if (want_rows && A.rows_list) {
        // (split form) the GCD rows are built by phase 3, over the directions that want them
        if (lane == 0) {
            D.slack_chol = slack_chol;
            A.rows_list[atomicAdd(A.rows_count, 1u)] = pid;
        }
        __syncwarp();
        return ST_WANT_ROWS;
    }
    return setup_rows_bounds<N>(A, pid, lane, stage, S, want_rows, slack_chol);
}

template <int N, int PH> __device__ __forceinline__ int setup_phase(const SetupArgs &A, int pid, int lane, int &stage,
                                                                   LllMem<N> *S)
{
    if (PH == 0) return setup_phase0<N>(A, pid, lane, stage, S);
    if (PH == 1) return setup_phase1<N>(A, pid, lane, stage, S);
    if (PH == 2) return setup_phase2<N>(A, pid, lane, stage, S);
    return setup_phase3<N>(A, pid, lane, stage, S);
}

// All three phases of one direction in sequence (the no-allocation entry point).
template <int N> __device__ int setup_one(const SetupArgs &A, int pid, int lane, int &stage, LllMem<N> *S)
{
    int st = setup_phase0<N>(A, pid, lane, stage, S);
    if (st == ST_PENDING) st = setup_phase1<N>(A, pid, lane, stage, S);
    if (st == ST_PENDING) st = setup_phase2<N>(A, pid, lane, stage, S);
    return st;
}

// Persistent setup kernel of phase PH: warps take directions from A.todo
// through an atomic counter; phases 1 and 2 skip the directions an earlier
// phase finished.  N = 32 serves h11 <= 32 with the LLL working set in
// dynamic shared memory (one LllMem<32> per warp) when A.smem_core is set;
// otherwise (and for N = 64) the working set is the warp's global scratch.
// (N = 32: launched as one-warp blocks, 16 per SM -- 128 registers a thread,
// 16 x 12.9 KB of shared memory; N = 64: blocks of 4 warps, 4 per SM)
template <int N, int PH> __global__ void __launch_bounds__(N == 32 ? 32 : 128, N == 32 ? 16 : 4) k_setup(SetupArgs A)
{
#ifdef PFG_EMU
    unsigned char *smem_raw = nullptr;
#else
    extern __shared__ __align__(16) unsigned char smem_raw[];
#endif
    const int lane = threadIdx.x & 31;
    SetupScratch *Wg = A.scratch + (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5));
    LllMem<N> *S = A.smem_core ? (LllMem<N> *)smem_raw + (threadIdx.x >> 5) : (LllMem<N> *)&Wg->core;
    if (lane == 0) S->B = Wg->Bstore;
    __syncwarp();
    const unsigned n = A.n_dev ? *A.n_dev : (unsigned)A.n;
    for (;;) {
        unsigned t = 0;
        if (lane == 0) t = atomicAdd(A.next, 1u);
        t = __shfl_sync(FULL, t, 0);
        if (t >= n) break;
        const int pid = A.todo ? A.todo[t] : (int)t;
        const Geo g = A.geo[A.pgeo[pid]];
        if (PH == 0) {
            if (lane == 0) {
                Dir &D = A.dirs[pid];
                D.geo = A.pgeo[pid]; D.h = g.h; D.d = g.h - 1; D.slab = A.slab_off[pid];
                D.m0_level = -1; D.g_lin = 0; D.hrows = 0; D.slack_chol = 0.0; D.wide = 0;
            }
        } else if (A.dirs[pid].status != (PH == 3 ? ST_WANT_ROWS : ST_PENDING)) {
            continue;
        }
        __syncwarp();
        int stage = 0;
        int st = g.h + (g.coni ? 0 : 1) <= N ? setup_phase<N, PH>(A, pid, lane, stage, S) : ST_OVERFLOW;
        if (lane == 0) { A.dirs[pid].status = st; A.dirs[pid].pad = st < 0 ? stage : 0; }
        __syncwarp();
    }
}

}  // namespace pfg
