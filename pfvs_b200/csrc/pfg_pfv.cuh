// Lattice points -> coni PFVs on the device: coniZpM's post-processing
// (_pfvs_from_points, pfvs/coni.py:275-412) on the points in canonical
// order, all in exact integer arithmetic.
//
// For a point (M, Kn, q) of a direction with Q:
//   Kg = max(1, gcd(Kn[1:])); the strict cut q < Q Kg (the search already
//   keeps only such points); for g = 1 .. (Q Kg - 1) // q:
//     Qperp = g ((q + M0 Kn0) // Kg)
//     K0 in [ceil((Qperp - Q) / M0), min(floor((Qperp - Q) / M0), ceil(Kn0 g / Kg) - 1)]
//     K = (K0, g Kn[1:] / Kg), with -K.M <= Q checked (a violation is an error,
//     as the reference raises);
//   kept when det((kappa . M)[1:, 1:]) != 0; results grouped by direction,
//   then g, then point (canonical order), then K0 (coni.py:366-412).
//
// Kernels:
//   k_pfv_count  thread per point: Kg, the number of (g, K0) entries
//   k_scan64     offsets (one block)
//   k_pfv_fill   thread per point: its entries (point, g, K0)
//   k_pfv_sort   one block: entries into (direction, g, entry) order
//   k_pfv_det    warp per point with entries: the determinant test, exactly:
//                Gaussian elimination modulo 31-bit primes until one gives a
//                non-zero determinant (non-singular) or their product
//                exceeds twice the Hadamard bound of the matrix (singular)
//   k_pfv_keep   non-singular entries -> flags, k_scan64 -> positions
//   k_pfv_rows   the (K, M) rows, pidx, the tadpole check
#pragma once
#include "pfg_types.cuh"

namespace pfg {

struct PfvArgs {
    const Dir *dirs;
    const Geo *geo;
    const int64_t *kappa;            // all geometries (Geo::koff)
    const int64_t *M, *Kn, *q, *pidx;// points in canonical order, rows of MH
    unsigned long long n;            // points
    int64_t pid_base;                // pidx of the batch's first direction
    unsigned long long *cnt;         // (n + 1) entries per point, then their offsets
    uint64_t *Kg;                    // (n) gcd(Kn[1:]) (>= 1)
    unsigned *e_pt;                  // (n_e) entry -> point
    int64_t *e_g, *e_K0;             // (n_e)
    unsigned *e_ord;                 // (n_e) entries in output order
    int *nonsing;                    // (n) 1: det != 0 (per point with entries)
    unsigned long long *keep;        // (n_e + 1) kept flags, then offsets
    int *err;                        // [0] tadpole violation, [1] overflow, [2] expansion too long
    const uint32_t *primes;          // 31-bit primes, descending
    int n_primes;
    int mmax;                        // largest h11 - 1 of the batch (det matrix size)
};

constexpr long long PFV_MAX_G = 1ll << 22;     // most candidate g of one point

__device__ __forceinline__ bool pfv_prep(const PfvArgs &P, unsigned long long t, int &h, int64_t &Q, uint64_t &Kg,
                                         i128 &gcap, i128 &raw, int64_t &nat_K0, int64_t &M0)
{
    const int pid = (int)(P.pidx[t] - P.pid_base);
    const Dir D = P.dirs[pid];
    h = D.h;
    Q = P.geo[D.geo].Q;
    const int64_t *Kt = P.Kn + t * MH, *Mt = P.M + t * MH;
    uint64_t g = 0;
    for (int r = 1; r < h; ++r) g = gcd64(g, uabs64(Kt[r]));
    Kg = g ? g : 1;
    const int64_t q = P.q[t];
    const i128 QK = (i128)Q * (i128)Kg;
    if (!((i128)q < QK)) return false;                 // the strict cut
    gcap = (QK - 1) / (i128)(q > 1 ? q : 1);
    nat_K0 = Kt[0];
    M0 = Mt[0];
    raw = fdiv128((i128)q + (i128)M0 * nat_K0, (i128)Kg);
    return M0 > 0;
}

// The K0 range of expansion g is non-empty only when M0 divides g raw - Q
// (its ends are ceil and floor of (g raw - Q) / M0), i.e. g raw = Q (mod M0):
// the first such g >= 1 and the step between them, or false if there is none.
__device__ __forceinline__ bool pfv_g_progression(i128 raw, int64_t Q, int64_t M0, i128 &g0, i128 &step)
{
    const i128 m = M0;
    i128 r = raw % m;
    if (r < 0) r += m;
    i128 qm = (i128)Q % m;
    if (qm < 0) qm += m;
    // d = gcd(r, m); solvable iff d | qm
    i128 a = r, b = m;
    while (b) { const i128 t = a % b; a = b; b = t; }
    const i128 d = a;                               // (r = 0: d = m)
    if (qm % d) return false;
    const i128 m2 = m / d, r2 = r / d, q2 = qm / d;
    // inverse of r2 modulo m2 (extended Euclid)
    i128 x0 = 1, x1 = 0, a0 = r2 % m2, a1 = m2;
    while (a1) {
        const i128 qq = a0 / a1, t = a0 - qq * a1;
        a0 = a1; a1 = t;
        const i128 tx = x0 - qq * x1;
        x0 = x1; x1 = tx;
    }
    i128 inv = m2 > 1 ? x0 % m2 : 0;
    if (inv < 0) inv += m2;
    i128 g = m2 > 1 ? (q2 % m2) * inv % m2 : 0;
    if (g < 1) g += m2;
    g0 = g;
    step = m2;
    return true;
}

// The entries of a point in closed form.  For g in the progression above,
// K0 = (g raw - Q) / M0 exactly, and the cap K0 <= ceil(Kn0 g / Kg) - 1 is
// K0 Kg < Kn0 g, i.e. g (raw Kg - M0 Kn0) < Q Kg: with c = raw Kg - M0 Kn0,
// every g <= (Q Kg - 1) // c when c > 0, every g otherwise; and g <= gcap.
// Returns the number of entries; g0, step as pfv_g_progression.
__device__ __forceinline__ unsigned long long pfv_entries(i128 gcap, i128 raw, int64_t Q, int64_t M0, int64_t nat_K0,
                                                          uint64_t Kg, i128 &g0, i128 &step)
{
    if (!pfv_g_progression(raw, Q, M0, g0, step)) return 0;
    i128 G = gcap;
    const i128 c = raw * (i128)Kg - (i128)M0 * nat_K0, QK = (i128)Q * (i128)Kg;
    if (c > 0) {
        const i128 gc = (QK - 1) / c;
        if (gc < G) G = gc;
    }
    if (G < g0) return 0;
    const i128 n = (G - g0) / step + 1;
    return n > (i128)PFV_MAX_G ? ~0ull : (unsigned long long)n;
}

__global__ void k_pfv_count(PfvArgs P)
{
    for (unsigned long long t = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; t < P.n;
         t += (unsigned long long)gridDim.x * blockDim.x) {
        int h;
        int64_t Q, nat_K0, M0;
        uint64_t Kg;
        i128 gcap, raw, g0, step;
        unsigned long long c = 0;
        if (pfv_prep(P, t, h, Q, Kg, gcap, raw, nat_K0, M0)) {
            c = pfv_entries(gcap, raw, Q, M0, nat_K0, Kg, g0, step);
            if (c == ~0ull) { atomicExch(&P.err[2], 1); c = 0; }
        }
        P.Kg[t] = Kg;
        P.cnt[t] = c;
    }
}

// exclusive scan of a[0..n) in place, total in a[n] (one block of 1024 threads)
__global__ void __launch_bounds__(1024) k_scan64(unsigned long long *a, unsigned long long n)
{
    __shared__ unsigned long long part[1024];
    const unsigned long long t = threadIdx.x, nt = blockDim.x;
    const unsigned long long per = (n + nt - 1) / nt, lo = t * per, hi = min(lo + per, n);
    unsigned long long s = 0;
    for (unsigned long long i = lo; i < hi; ++i) s += a[i];
    part[t] = s;
    __syncthreads();
    for (unsigned o = 1; o < nt; o <<= 1) {
        const unsigned long long x = t >= o ? part[t - o] : 0;
        __syncthreads();
        part[t] += x;
        __syncthreads();
    }
    unsigned long long run = t ? part[t - 1] : 0;
    for (unsigned long long i = lo; i < hi; ++i) { const unsigned long long c = a[i]; a[i] = run; run += c; }
    if (t == nt - 1) a[n] = part[nt - 1];
}

__global__ void k_pfv_fill(PfvArgs P)
{
    for (unsigned long long t = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; t < P.n;
         t += (unsigned long long)gridDim.x * blockDim.x) {
        unsigned long long pos = P.cnt[t];
        const unsigned long long n = P.cnt[t + 1] - pos;
        if (!n) continue;
        int h;
        int64_t Q, nat_K0, M0;
        uint64_t Kg;
        i128 gcap, raw, g0, step;
        if (!pfv_prep(P, t, h, Q, Kg, gcap, raw, nat_K0, M0)) continue;
        if (!pfv_g_progression(raw, Q, M0, g0, step)) continue;
        for (unsigned long long j = 0; j < n; ++j) {
            const i128 g = g0 + (i128)j * step;
            const i128 k0 = (g * raw - (i128)Q) / (i128)M0;       // exact
            if (!fits64(k0)) { atomicExch(&P.err[1], 1); continue; }
            P.e_pt[pos] = (unsigned)t;
            P.e_g[pos] = (int64_t)g;
            P.e_K0[pos] = (int64_t)k0;
            ++pos;
        }
    }
}

// entry a before entry b: (direction, g, entry index) -- entries are made in
// (point, g, K0) order and points are in canonical order
__device__ __forceinline__ bool pfv_before(const PfvArgs &P, unsigned a, unsigned b)
{
    const int64_t pa = P.pidx[P.e_pt[a]], pb = P.pidx[P.e_pt[b]];
    if (pa != pb) return pa < pb;
    if (P.e_g[a] != P.e_g[b]) return P.e_g[a] < P.e_g[b];
    return a < b;
}

// one block: bitonic sort of the entry indices (padded to a power of two)
// in scratch (np entries)
__global__ void __launch_bounds__(1024) k_pfv_sort(PfvArgs P, unsigned long long n_e, unsigned np, unsigned *a)
{
    constexpr unsigned NONE = 0xffffffffu;
    for (unsigned t = threadIdx.x; t < np; t += blockDim.x) a[t] = t < n_e ? t : NONE;
    __syncthreads();
    for (unsigned k = 2; k <= np; k <<= 1)
        for (unsigned j = k >> 1; j > 0; j >>= 1) {
            for (unsigned t = threadIdx.x; t < np; t += blockDim.x) {
                const unsigned u = t ^ j;
                if (u <= t) continue;
                const bool up = (t & k) == 0;
                const unsigned x = a[t], y = a[u];
                bool xgt;
                if (x == NONE) xgt = y != NONE;
                else if (y == NONE) xgt = false;
                else xgt = pfv_before(P, y, x);
                if (xgt == up) { a[t] = y; a[u] = x; }
            }
            __syncthreads();
        }
    for (unsigned t = threadIdx.x; t < n_e; t += blockDim.x) P.e_ord[t] = a[t];
}

// arithmetic modulo a prime p < 2^31 with Barrett reduction (x < 2^64)
struct ModP {
    uint32_t p;
    uint64_t m;                                     // floor((2^64 - 1) / p)
    __device__ explicit ModP(uint32_t p_) : p(p_), m(~0ull / p_) {}
    __device__ __forceinline__ uint32_t red(uint64_t x) const
    {
        uint64_t r = x - __umul64hi(x, m) * (uint64_t)p;
        while (r >= p) r -= p;
        return (uint32_t)r;
    }
    __device__ __forceinline__ uint32_t mul(uint32_t a, uint32_t b) const { return red((uint64_t)a * b); }
    __device__ __forceinline__ uint32_t of(int64_t x) const
    {
        const uint32_t r = red(uabs64(x));
        return x < 0 && r ? p - r : r;
    }
    __device__ uint32_t pow(uint32_t a, uint32_t e) const
    {
        uint32_t r = 1;
        while (e) {
            if (e & 1) r = mul(r, a);
            a = mul(a, a);
            e >>= 1;
        }
        return r;
    }
};

// det(A) mod p for the m x m matrix in shared memory A (row stride m), lanes
// own columns; A is destroyed
__device__ uint32_t warp_det_mod(uint32_t *A, int m, const ModP &F, int lane)
{
    const uint32_t p = F.p;
    uint32_t det = 1;
    for (int c = 0; c < m; ++c) {
        const bool nz0 = lane >= c && lane < m && A[lane * m + c] != 0;
        const bool nz1 = lane + 32 >= c && lane + 32 < m && A[(lane + 32) * m + c] != 0;
        const unsigned b0 = __ballot_sync(FULL, nz0), b1 = __ballot_sync(FULL, nz1);
        const int r = b0 ? __ffs(b0) - 1 : (b1 ? 32 + __ffs(b1) - 1 : -1);
        if (r < 0) return 0;
        __syncwarp();
        if (r != c) {
            for (int j = c + lane; j < m; j += 32) {
                const uint32_t x = A[r * m + j];
                A[r * m + j] = A[c * m + j];
                A[c * m + j] = x;
            }
            det = det ? p - det : 0;
            __syncwarp();
        }
        const uint32_t piv = A[c * m + c];
        det = F.mul(det, piv);
        const uint32_t inv = F.pow(piv, p - 2);
        for (int i = c + 1; i < m; ++i) {
            const uint32_t f = F.mul(A[i * m + c], inv);
            if (f) {
                const uint64_t nf = p - f;
                for (int j = c + 1 + lane; j < m; j += 32)
                    A[i * m + j] = F.red(A[i * m + j] + nf * A[c * m + j]);
            }
        }
        __syncwarp();
    }
    return det;
}

// warp per point with entries: is det((kappa . M)[1:, 1:]) != 0 ?
__global__ void __launch_bounds__(32) k_pfv_det(PfvArgs P)
{
#ifdef PFG_EMU
    static int64_t Nx[MD * MD];
    static uint32_t A[MD * MD];
#else
    extern __shared__ __align__(16) int64_t Nx[];                  // exact matrix (mmax^2)
    uint32_t *A = (uint32_t *)(Nx + P.mmax * P.mmax);              // its residues (mmax^2)
#endif
    const int lane = threadIdx.x & 31;
    for (unsigned long long t = blockIdx.x; t < P.n; t += gridDim.x) {
        if (P.cnt[t + 1] == P.cnt[t]) continue;
        const int pid = (int)(P.pidx[t] - P.pid_base);
        const Dir D = P.dirs[pid];
        const int h = D.h, m = h - 1;
        const int64_t *kap = P.kappa + P.geo[D.geo].koff, *Mt = P.M + t * MH;
        // log2 of the Hadamard bound prod_i ||row i|| (an upper bound, rounded up)
        double lb = 0.0;
        for (int i = lane; i < m; i += 32) {
            double s2 = 0.0;
            for (int j = 0; j < m; ++j) {
                double a = 0.0;
                for (int k = 0; k < h; ++k)
                    a += fabs((double)kap[((int64_t)(i + 1) * h + (j + 1)) * h + k]) * fabs((double)Mt[k]);
                s2 += a * a;
            }
            lb += 0.5 * log2(s2 * (1.0 + 1e-9) + 1.0);
        }
        for (int o = 16; o; o >>= 1) lb += __shfl_xor_sync(FULL, lb, o);
        lb = lb * (1.0 + 1e-9) + 2.0;                   // (det = 0 iff |det| < prod p / 2)
        // the exact matrix once (int64 when it fits; otherwise residues are built per prime)
        bool big = false;
        for (int e = lane; e < m * m; e += 32) {
            const int i = e / m, j = e % m;
            const int64_t *kr = kap + ((int64_t)(i + 1) * h + (j + 1)) * h;
            i128 s = 0, t;
            for (int k = 0; k < h; ++k)
                if (mul_ovf((i128)kr[k], (i128)Mt[k], &t) || add_ovf(s, t, &s)) big = true;
            if (!fits64(s)) big = true;
            Nx[e] = (int64_t)s;
        }
        big = __any_sync(FULL, big);
        __syncwarp();
        int res = -1;
        double covered = 0.0;
        for (int pi = 0; pi < P.n_primes && res < 0; ++pi) {
            const ModP F(P.primes[pi]);
            const uint32_t p = F.p;
            for (int e = lane; e < m * m; e += 32) {
                if (!big) { A[e] = F.of(Nx[e]); continue; }
                const int i = e / m, j = e % m;
                const int64_t *kr = kap + ((int64_t)(i + 1) * h + (j + 1)) * h;
                uint32_t s = 0;
                for (int k = 0; k < h; ++k) s = F.red((uint64_t)s + (uint64_t)F.mul(F.of(kr[k]), F.of(Mt[k])));
                A[e] = s;
            }
            __syncwarp();
            const uint32_t dp = warp_det_mod(A, m, F, lane);
            if (dp != 0) res = 1;
            else {
                covered += log2((double)p);
                if (covered > lb) res = 0;
            }
            __syncwarp();
        }
        if (lane == 0) {
            if (res < 0) atomicExch(&P.err[1], 2);      // more primes needed than given
            P.nonsing[t] = res == 1;
        }
    }
}

__global__ void k_pfv_keep(PfvArgs P, unsigned long long n_e)
{
    for (unsigned long long e = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; e < n_e;
         e += (unsigned long long)gridDim.x * blockDim.x)
        P.keep[e] = P.nonsing[P.e_pt[P.e_ord[e]]] ? 1 : 0;
}

// warp per kept entry (in output order): K, M rows, pidx, tadpole check
__global__ void k_pfv_rows(PfvArgs P, unsigned long long n_e, int64_t *K, int64_t *Mo, int64_t *pidx)
{
    const int lane = threadIdx.x & 31;
    const unsigned long long w = (blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x) >> 5;
    const unsigned long long nw = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
    for (unsigned long long e = w; e < n_e; e += nw) {
        if (P.keep[e + 1] == P.keep[e]) continue;
        const unsigned long long o = P.keep[e];
        const unsigned x = P.e_ord[e];
        const unsigned t = P.e_pt[x];
        const int pid = (int)(P.pidx[t] - P.pid_base);
        const Dir D = P.dirs[pid];
        const int h = D.h;
        const int64_t Q = P.geo[D.geo].Q;
        const int64_t *Kt = P.Kn + (unsigned long long)t * MH, *Mt = P.M + (unsigned long long)t * MH;
        const int64_t g = P.e_g[x];
        const uint64_t Kg = P.Kg[t];
        i128 tad = 0;
        bool bad = false;
        for (int r = lane; r < MH; r += 32) {
            int64_t kv = 0, mv = 0;
            if (r < h) {
                mv = Mt[r];
                if (r == 0) kv = P.e_K0[x];
                else {
                    const i128 y = (i128)g * (i128)(Kt[r] / (int64_t)Kg);
                    if (!fits64(y)) bad = true;
                    kv = (int64_t)y;
                }
                tad -= (i128)kv * mv;
            }
            K[o * MH + r] = kv;
            Mo[o * MH + r] = mv;
        }
        for (int s = 16; s; s >>= 1) {
            long long lo = (long long)(uint64_t)tad, hi = (long long)(tad >> 64);
            lo = __shfl_xor_sync(FULL, lo, s);
            hi = __shfl_xor_sync(FULL, hi, s);
            tad += (i128)(((u128)(uint64_t)hi << 64) | (uint64_t)lo);
        }
        bad = __any_sync(FULL, bad);
        if (lane == 0) {
            pidx[o] = P.pidx[t];
            if (tad > (i128)Q) atomicExch(&P.err[0], 1);
            if (bad) atomicExch(&P.err[1], 1);
        }
        __syncwarp();
    }
}

}  // namespace pfg
