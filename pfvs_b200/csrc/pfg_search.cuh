// The Fincke-Pohst search on the device: one warp per subtree.
//
// Semantics are those of the reference search fpk_search
// (pfvs/fp_kernel/fpk_search_impl.h:217-455): c is set from its last
// coordinate to its first; per level the candidate range comes from the
// ellipsoid radius widened by a rigorous rounding-error bound, narrowed by
// the GCD bound of the rows already determined and, at the M0 level, by the
// exact interval M0 = g_lin c[d-1] >= M0min; each candidate is tested on the
// ellipsoid (with the error term en), exactly on M0, and on the GCD cut with
// an early-exit gcd; leaves are decided exactly (q in int128, gcd of
// Kn[1:] = (ZB c)[1:] exactly).  Floating point only prunes.
//
// B200 mapping.  The 32 lanes of a warp share one DFS: lane l keeps the
// state of levels l and l+32 in registers (candidate range, remaining norm,
// error bound, centre offset, gcd of the rows above, the GCD row's prefix,
// and c[l]); entering a level is a warp-wide dot product (lane j multiplies
// U[i][j] c[j]) reduced with shuffles; the 32 lanes test 32 sibling
// candidates at once and a ballot picks the next child (DFS order) or the
// passing leaves.  The exact sums mat c and ZB c are kept per lane
// (lane r owns rows r, r+32) and updated by one column whenever a coordinate
// changes, so a leaf costs O(1) exact work; the GCD rows' prefixes
// (H_r c over the coordinates above row r's pivot, lane r) are kept the
// same way, with the column of H that a coordinate change touches.  (M = Binter c is formed after
// the search from the emitted c.)  Warps take whole directions
// from a counter and donate the top of their DFS stack to a global queue
// when other warps run out of work (persistent kernel, work stealing).
#pragma once
#include "pfg_types.cuh"

namespace pfg {

struct WorkItem {                 // an entered node with its remaining candidates
    int32_t pid, level;
    int64_t cur, hi;
    double rem, err;
    uint64_t glo, ghi;            // gcd of the rows above (u128)
    int32_t c[MD + 1];            // c[level+1 .. d-1]
};

struct SearchCtl {
    unsigned roots_next;          // next index into the todo list
    unsigned q_tail, q_head;      // queue reservation / consumption
    int active;                   // warps holding work
    int err;                      // first error (ST_WAIT) if any
    int pad;
    unsigned long long npts;      // points emitted by all passes (see SearchArgs::npts)
    unsigned long long nodes, cands, leaves, donated;
    // FP32 bound check (k_search_plain<float, NS, true>): maxima as the bit
    // patterns of non-negative doubles, and a count
    unsigned long long chk_rem, chk_frac, chk_end, chk_narrower;
};

struct SearchArgs {
    const Geo *geo;
    Dir *dirs;
    const int64_t *slab;
    const int32_t *todo;          // directions to search (their status is ST_PENDING)
    int n_todo;
    int pass;                     // written into each point (stale passes are dropped)
    SearchCtl *ctl;
    WorkItem *items;
    int *ready;
    unsigned q_cap;
    PointHdr *hdr;
    int32_t *coords;              // (cap, MD)
    unsigned long long pts_cap;
    unsigned long long *npts;     // points emitted (shared by all passes; may exceed pts_cap)
    unsigned long long *dir_nodes;  // per direction
    double eps;
    int donate;                   // 0: the plain form (no queue)
    int n_warps;                  // warps of the persistent grid
    long long wait_ns;            // bound on idle waiting (globaltimer ns)
    long long deadline_ns;        // bound on one subtree's search (globaltimer ns)
    unsigned stage_bytes;         // per-warp staging area (dynamic shared memory), stage_bytes<R>(d max)
};

__device__ __forceinline__ unsigned long long gtimer()
{
#ifdef PFG_EMU
    return emu_now_ns();
#else
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
#endif
}

template <class T> __device__ __forceinline__ T shfl(T x, int src) { return __shfl_sync(FULL, x, src); }
__device__ __forceinline__ i128 shfl128(i128 x, int src)
{
    long long lo = (long long)(uint64_t)x, hi = (long long)(x >> 64);
    lo = __shfl_sync(FULL, lo, src);
    hi = __shfl_sync(FULL, hi, src);
    return (i128)(((u128)(uint64_t)hi << 64) | (uint64_t)lo);
}
__device__ __forceinline__ u128 shflu128(u128 x, int src) { return (u128)shfl128((i128)x, src); }
__device__ __forceinline__ i128 warp_sum128(i128 x)
{
    // every lane's term below 2^58 in magnitude (the usual case): the sum of 32
    // of them fits int64, so one 64-bit shuffle a round instead of two
    const int64_t lo64 = (int64_t)x;
    if (__all_sync(FULL, (i128)lo64 == x && lo64 < (1ll << 58) && lo64 > -(1ll << 58))) {
        long long t = lo64;
        for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(FULL, t, o);
        return (i128)t;
    }
    for (int o = 16; o; o >>= 1) {
        long long lo = (long long)(uint64_t)x, hi = (long long)(x >> 64);
        lo = __shfl_xor_sync(FULL, lo, o);
        hi = __shfl_xor_sync(FULL, hi, o);
        x += (i128)(((u128)(uint64_t)hi << 64) | (uint64_t)lo);
    }
    return x;
}
template <class R> __device__ __forceinline__ R warp_sumr(R x)
{
    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(FULL, x, o);
    return x;
}

template <class R> struct Num;
template <> struct Num<float> {
    static __device__ float U() { return 0x1p-24f; }
    static __device__ float G() { return 64 * 0x1p-24f; }
    static __device__ float tiny() { return 1e-30f; }
    static __device__ float i32max() { return 2147483520.0f; }
};
template <> struct Num<double> {
    static __device__ double U() { return 0x1p-53; }
    static __device__ double G() { return 1e-9; }
    static __device__ double tiny() { return 1e-300; }
    static __device__ double i32max() { return 2147483647.0; }
};

// The search data of one direction, staged by the warp that searches it:
// U packed by rows (upper triangle, row i holds U[i][i..d-1]), 1/U_ii, and
// mat and ZB^T as int32 (the setup bounds their row / column absolute sums by 2^31), and
// the GCD rows' pivots H_ii; the GCD-cut rows H themselves stay in global memory (only
// large trees have them), read one column per coordinate change.
PFG_HD int upk(int i, int j, int d) { return i * d - ((i * (i - 1)) >> 1) + (j - i); }
template <class R> PFG_HD unsigned stage_bytes(int d, int h)
{
    unsigned b = (unsigned)((d * (d + 1) / 2 + d) * sizeof(R));
    b = (b + 15u) & ~15u;
    b += (unsigned)(d * d + d * h) * 4u;
    b = (b + 15u) & ~15u;
    b += (unsigned)d * 8u;                      // H_ii
    return (b + 15u) & ~15u;
}

template <class R> struct Prob {
    const R *U, *UI;                  // staged: U packed (upk), 1/U_ii
    const int32_t *MAT, *ZT;          // staged: mat (d x d), ZT (d x h)
    const int64_t *HD;                // staged: the GCD rows' pivots H_ii (0 where no row is kept)
    const int64_t *H;                 // global, transposed: H[c d + r] = entry c of the row with pivot r
    const double *U64, *UI64;         // global: the FP64 factor (d x d row-major), 1/U_ii
    int d, h, m0_level;
    int coni;                         // 1: strict GCD cut on K[1:] (coni); 0: non-strict on all of K
    int wide;                         // mat has entries beyond int32: read in int64 from the slab,
                                      // where it lies just before H (H - d d), not from MAT
    int64_t g_lin, Q, qmax, linmin;
    uint64_t hrows;
    R qmax_r, slack, Kerr, max_err, invQ;
    double slack_chol;                // the FP64 factor's certified margin (part of slack)
};

// Set up the problem of direction pid and stage its data in `stage` (the
// warp's area: shared memory in the batched kernels).  Warp-collective.
template <class R> __device__ Prob<R> load_prob(const SearchArgs &A, int pid, void *stage, int lane)
{
    const Dir D = A.dirs[pid];
    const Geo g = A.geo[D.geo];
    const int d = D.d, h = D.h;
    const Slab L = slab_layout(h, d);
    const int64_t *s = A.slab + D.slab;
    const R *Ug = sizeof(R) == 4 ? (const R *)(s + L.u32) : (const R *)(s + L.u64);
    const R *UIg = sizeof(R) == 4 ? (const R *)(s + L.ui32) : (const R *)(s + L.ui64);
    const int64_t *MATg = s + L.mat, *ZTg = s + L.zt;
    R *U = (R *)stage, *UI = U + d * (d + 1) / 2;
    int32_t *MAT = (int32_t *)((char *)stage + ((((d * (d + 1) / 2 + d) * sizeof(R)) + 15) & ~(size_t)15));
    int32_t *ZT = MAT + d * d;
    int64_t *HD = (int64_t *)((char *)stage + ((((((d * (d + 1) / 2 + d) * sizeof(R)) + 15) & ~(size_t)15)
                                                 + (size_t)(d * d + d * h) * 4 + 15) & ~(size_t)15));
    __syncwarp();                                   // (the previous problem's readers are done)
    for (int e = lane; e < d * d; e += 32) {
        const int i = e / d, j = e - i * d;
        if (j >= i) U[upk(i, j, d)] = Ug[e];
        MAT[e] = (int32_t)MATg[e];
    }
    for (int e = lane; e < d; e += 32) UI[e] = UIg[e];
    for (int e = lane; e < d * h; e += 32) ZT[e] = (int32_t)ZTg[e];
    for (int e = lane; e < d; e += 32) HD[e] = ((D.hrows >> e) & 1) ? s[L.H + (int64_t)e * d + e] : 0;
    __syncwarp();
    Prob<R> P;
    P.d = d; P.h = h; P.m0_level = D.m0_level; P.coni = g.coni; P.wide = D.wide;
    P.g_lin = D.g_lin; P.Q = g.Q; P.qmax = g.qmax; P.linmin = g.linmin; P.hrows = D.hrows;
    P.U = U; P.UI = UI; P.MAT = MAT; P.ZT = ZT; P.HD = HD; P.H = s + L.H;
    P.U64 = (const double *)(s + L.u64); P.UI64 = (const double *)(s + L.ui64);
    const R qd = (R)g.qmax;
    P.qmax_r = qd;
    // search constants (fpk_search_impl.h:30-39), plus the certified margin
    // of the FP64 Cholesky factor
    R sl = (R)A.eps > Num<R>::G() * (qd + (R)1) ? (R)A.eps : Num<R>::G() * (qd + (R)1);
    P.slack = sl + (R)D.slack_chol;
    P.slack_chol = D.slack_chol;
    P.Kerr = (R)2 * (R)(D.d + 8) * Num<R>::U();
    P.max_err = sizeof(R) < sizeof(double) ? (R)1 + (R)0.05 * qd : (R)INFINITY;
    P.invQ = (R)1 / (R)g.Q;
    return P;
}

// smallest gcd that can pass the GCD cut when q >= q_lb (fpk_search_impl.h:43-51):
// Q g > q (strict, coni) or Q g >= q (non-coni); q_lb / Q as a product with the
// rounded 1/Q: its few units of rounding are far inside the G (1 + t) margin
// taken off below
template <class R> __device__ __forceinline__ uint64_t need_of(R q_lb, R invQ, int strict)
{
    if (!(q_lb > 0)) return 0;
    R t = q_lb * invQ;
    t -= Num<R>::G() * ((R)1 + t);
    if (t < 0) t = 0;
    if (t >= (R)1.8e19) return UINT64_MAX;
    return strict ? (uint64_t)floor((double)t) + 1 : (uint64_t)ceil((double)t);
}
// the branch must fail the cut when q >= q_lb (fpk_search_impl.h:56-62)
template <class R> __device__ __forceinline__ bool gcd_fails(u128 g, int64_t Q, R q_lb, int strict)
{
    if (g == 0 || (g >> 64) != 0) return false;
    R Qg = (R)Q * (R)(uint64_t)g;
    return strict ? Qg <= q_lb : Qg < q_lb;
}

struct Tally { unsigned long long nodes, cands, leaves; };

// Profiling build only (-DPFG_STAGE_CLOCKS): per pass (float 0, double 1)
// the warps' clock64() cycles spent searching [0/1] and waiting for work
// [2/3], the subtrees run [4/5], and within the search the cycles of the
// leaf level (exact q, GCD cut, emission) [6/7]; in the FP64 pass the
// cycles of backtracks [8], candidate evaluation at interior levels [9] and
// descents (incremental sums, entering the level) [10].
#ifdef PFG_STAGE_CLOCKS
__device__ unsigned long long pfg_search_cycles[16];
#define PFG_SCLK(v) long long v = clock64()
#define PFG_SADD(i, x) do { if (lane == 0) atomicAdd(&pfg_search_cycles[(i) + (sizeof(R) == 8)], (unsigned long long)(x)); } while (0)
#else
#define PFG_SCLK(v) do { } while (0)
#define PFG_SADD(i, x) do { } while (0)
#endif

// Per-lane register state: levels lane (slot 0) and lane + 32 (slot 1).
// The search code is instantiated for NS = 1 slot (h11 <= 32: every level
// and column has its own lane, and slot 1 is never touched, so the compiler
// drops its registers) and NS = 2 (h11 up to 64).
template <class R> struct Lanes {
    int64_t cur0, cur1, hi0, hi1;
    R rem0, rem1, err0, err1, off0, off1, aoff0, aoff1;
    u128 gab0, gab1;              // gcd of the rows above the level
    i128 hp0, hp1;                // H_r c over c[r+1:], r = lane, lane+32 (the GCD row's prefix)
    int32_t c0, c1;               // c[lane], c[lane+32]
    int64_t y0, y1;               // (mat c)_r, r = lane, lane+32, over c[1:]
    int64_t k0, k1;               // (ZB c)_r over c[1:]
};

#define LGET(S, f, i) shfl((NS > 1 && (i) >= 32) ? S.f##1 : S.f##0, (i) & 31)
#define LSET(S, f, i, val) do { if (lane == ((i) & 31)) { if (NS > 1 && (i) >= 32) S.f##1 = (val); else S.f##0 = (val); } } while (0)

// c[i] changes by dv (i >= 1): update the exact incremental sums (the GCD
// rows' prefixes of the levels below i with column i of H)
template <class R, int NS> __device__ __forceinline__ void apply_dc(Lanes<R> &S, const Prob<R> &P, int i, int64_t dv, int lane)
{
    if (dv == 0 || i == 0) return;
    const int d = P.d, h = P.h;
    if (lane < d) S.y0 += (P.wide ? P.H[(i - d) * d + lane] : (int64_t)P.MAT[i * d + lane]) * dv;
    if (NS > 1 && lane + 32 < d) S.y1 += (P.wide ? P.H[(i - d) * d + lane + 32] : (int64_t)P.MAT[i * d + lane + 32]) * dv;
    if (lane < h) S.k0 += (int64_t)P.ZT[i * h + lane] * dv;
    if (NS > 1 && lane + 32 < h) S.k1 += (int64_t)P.ZT[i * h + lane + 32] * dv;
    if (lane < i && ((P.hrows >> lane) & 1)) S.hp0 += (i128)P.H[i * d + lane] * dv;
    if (NS > 1 && lane + 32 < i && ((P.hrows >> (lane + 32)) & 1)) S.hp1 += (i128)P.H[i * d + lane + 32] * dv;
}

// the dot products of entering level i (c[i+1:] set): off, aoff, GCD prefix
template <class R, int NS> __device__ __forceinline__ void level_sums(const Lanes<R> &S, const Prob<R> &P, int i, int lane,
                                                              R &off, R &aoff, i128 &pre)
{
    const int d = P.d;
    R o = 0, a = 0;
    const bool hrow = (P.hrows >> i) & 1;
    const R *Ui = P.U + upk(i, i, d) - i;           // Ui[j] = U[i][j], j >= i
    int j = lane;
    if (j > i && j < d) {
        R t = Ui[j] * (R)S.c0;
        o += t; a += fabs(t);
    }
    j = lane + 32;
    if (NS > 1 && j > i && j < d) {
        R t = Ui[j] * (R)S.c1;
        o += t; a += fabs(t);
    }
    off = warp_sumr(o);
    aoff = warp_sumr(a);
    pre = hrow ? shfl128((NS > 1 && i >= 32) ? S.hp1 : S.hp0, i & 31) : (i128)0;
}

// The candidate range [lo, hi] (lo > hi: none) of level i from its entry
// values: remaining norm rem, its error bound err, the gcd bound gab of the
// rows above, the centre offset off and the absolute sum aoff
// (fpk_search_impl.h:241-348).  Returns ST_RANGE if a bound leaves int32.
// The real interval (a, b) of level i before rounding to integers (false:
// the GCD bound rules the level out), in precision R with the constants
// slack, Kerr, qmax and 1/U_ii given.
template <class R> __device__ __forceinline__ bool level_interval(R slack, R Kerr, R qmax_r, int64_t Q, R ui, R rem,
                                                                  R err, u128 gab, R off, R aoff, R &a, R &b)
{
    R Rr = sqrt(fmax(rem + slack + err, (R)0));
    Rr += Kerr * (Rr + (R)2 * aoff) + Num<R>::tiny();
    if (gab != 0 && (gab >> 64) == 0) {                 // GCD narrowing
        R am = Rr + (R)2 * aoff;
        R Rg2 = (R)Q * (R)(uint64_t)gab - (qmax_r - rem) + slack + err + Kerr * (am * am + rem);
        if (Rg2 < (R)0) return false;
        R Rg = sqrt(Rg2);
        Rg += Kerr * (Rg + (R)2 * aoff) + Num<R>::tiny();
        if (Rg < Rr) Rr = Rg;
    }
    a = (-Rr - off) * ui;
    b = (Rr - off) * ui;
    return true;
}

template <class R> __device__ __forceinline__ int level_range(const Prob<R> &P, int i, R rem, R err, u128 gab,
                                                              R off, R aoff, int64_t &lo_o, int64_t &hi_o)
{
    R a = 0, b = 0;
    const bool empty = !level_interval<R>(P.slack, P.Kerr, P.qmax_r, P.Q, P.UI[i], rem, err, gab, off, aoff, a, b);
    int64_t lo = 1, hi = 0;
    if (!empty) {
        a = ceil(a - Num<R>::G() * ((R)1 + fabs(a)));
        b = floor(b + Num<R>::G() * ((R)1 + fabs(b)));
        if (!(a >= -Num<R>::i32max() && b <= Num<R>::i32max())) return ST_RANGE;
        lo = (int64_t)a; hi = (int64_t)b;
        if (i == P.m0_level) {                          // exact M0 interval: g_lin v >= linmin
            const i128 need = (i128)P.linmin, l = P.g_lin;
            if (l > 0) {
                i128 bnd = need >= 0 ? (need + l - 1) / l : -((-need) / l);
                if (bnd > lo) lo = bnd > hi ? hi + 1 : (int64_t)bnd;
            } else {
                i128 nl = -l;
                i128 bnd = need <= 0 ? (-need) / nl : -((need + nl - 1) / nl);
                if (bnd < hi) hi = bnd < lo ? lo - 1 : (int64_t)bnd;
            }
        }
    }
    lo_o = lo; hi_o = hi;
    return 0;
}

// Enter level i (warp search): the level's sums and candidate range into
// the owner lanes' registers (kept for the return to this level and for
// donation), and to the caller (every lane).  Returns ST_RANGE if a bound
// leaves int32.
template <class R, int NS> __device__ int enter_level(Lanes<R> &S, const Prob<R> &P, int i, R rem, R err, u128 gab,
                                              int lane, int64_t &lo_o, int64_t &hi_o, R &off, R &aoff, i128 &pre)
{
#ifdef PFG_STAGE_CLOCKS
    const long long e0 = clock64();
#endif
    level_sums<R, NS>(S, P, i, lane, off, aoff, pre);
#ifdef PFG_STAGE_CLOCKS
    const long long e1 = clock64();
#endif
    int64_t lo, hi;
    const int st = level_range(P, i, rem, err, gab, off, aoff, lo, hi);
#ifdef PFG_STAGE_CLOCKS
    __syncwarp();
    if (lane == 0 && sizeof(R) == 8) {
        atomicAdd(&pfg_search_cycles[12], (unsigned long long)(e1 - e0));
        atomicAdd(&pfg_search_cycles[13], (unsigned long long)(clock64() - e1));
    }
#endif
    if (st) return st;
    LSET(S, cur, i, lo); LSET(S, hi, i, hi);
    LSET(S, rem, i, rem); LSET(S, err, i, err);
    LSET(S, off, i, off); LSET(S, aoff, i, aoff);
    LSET(S, gab, i, gab);
    lo_o = lo; hi_o = hi;
    return 0;
}

// exact leaf data of the level-0 node (c[1:] set): q(c) = A0 + 2 c0 B0 + m00 c0^2
template <class R, int NS> __device__ __forceinline__ void leaf_data(const Lanes<R> &S, const Prob<R> &P, int lane,
                                                             i128 &A0, int64_t &B0)
{
    i128 part = 0;
    if (lane >= 1 && lane < P.d) part += (i128)S.c0 * S.y0;
    if (NS > 1 && lane + 32 < P.d) part += (i128)S.c1 * S.y1;
    A0 = warp_sum128(part);
    B0 = shfl(S.y0, 0);
}

// FP32-versus-FP64 bound check.  The FP32 search is run with an FP64 shadow
// of its pruning quantities along the same path (the FP64 factor, FP64
// sums): per candidate the FP32 remaining norm nr against the FP64 one
// (abs difference, and its fraction of the FP32 safety margin slack + en
// that the pruning test allows), per level the real interval endpoints
// against the FP64 ones, and the levels whose FP32 integer range misses
// part of the FP64 one.  FP64's own error is ~2^-29 of FP32's, so the FP64
// values stand in for the exact ones.
struct BoundAcc { double rem, frac, end; unsigned long long narrower; };
struct Shadow64 { double rem0, rem1, err0, err1, off0, off1, aoff0, aoff1; };

template <int NS> __device__ __forceinline__ void shadow_sums(const Lanes<float> &S, const Prob<float> &P, int i,
                                                              int lane, double &off, double &aoff)
{
    const int d = P.d;
    double o = 0, a = 0;
    if (lane > i && lane < d) { const double t = P.U64[i * d + lane] * (double)S.c0; o += t; a += fabs(t); }
    if (NS > 1 && lane + 32 > i && lane + 32 < d) {
        const double t = P.U64[i * d + lane + 32] * (double)S.c1; o += t; a += fabs(t);
    }
    off = warp_sumr(o);
    aoff = warp_sumr(a);
}

// the interval endpoints of level i in both precisions
__device__ __forceinline__ void shadow_interval(const Prob<float> &P, int i, float rem, float err, u128 gab,
                                                float off, float aoff, double rem64, double err64, double off64,
                                                double aoff64, double slack64, double Kerr64, BoundAcc &acc)
{
    float a = 0, b = 0;
    double a64 = 0, b64 = 0;
    const bool ok32 = level_interval<float>(P.slack, P.Kerr, P.qmax_r, P.Q, P.UI[i], rem, err, gab, off, aoff, a, b);
    const bool ok64 = level_interval<double>(slack64, Kerr64, (double)P.qmax, P.Q, P.UI64[i], rem64, err64, gab,
                                             off64, aoff64, a64, b64);
    if (ok32 && ok64) acc.end = fmax(acc.end, fmax(fabs((double)a - a64), fabs((double)b - b64)));
    if (ok64) {
        const double lo64 = ceil(a64 - Num<double>::G() * (1.0 + fabs(a64)));
        const double hi64 = floor(b64 + Num<double>::G() * (1.0 + fabs(b64)));
        if (lo64 <= hi64) {
            if (!ok32) acc.narrower++;
            else {
                const float lo = ceil(a - Num<float>::G() * (1.0f + fabs(a)));
                const float hi = floor(b + Num<float>::G() * (1.0f + fabs(b)));
                if ((double)lo > lo64 || (double)hi < hi64) acc.narrower++;
            }
        }
    }
}

template <class R, int NS, bool CHK = false>
__device__ int run_subtree(const SearchArgs &A, const Prob<R> &P, int pid, const WorkItem *it, Tally &T, int lane,
                           BoundAcc *acc = nullptr)
{
    static_assert(!CHK || sizeof(R) == 4, "the bound check shadows the FP32 search");
    const int d = P.d, h = P.h;
    Lanes<R> S;
    S.cur0 = S.cur1 = 0; S.hi0 = S.hi1 = -1;
    S.rem0 = S.rem1 = S.err0 = S.err1 = S.off0 = S.off1 = S.aoff0 = S.aoff1 = 0;
    S.gab0 = S.gab1 = 0; S.hp0 = S.hp1 = 0;
    S.c0 = S.c1 = 0; S.y0 = S.y1 = S.k0 = S.k1 = 0;
    int top, i;
    // The current level's entry values, the same in every lane (its owner
    // lane keeps a copy for the return to it after the levels below).
    int64_t u_cur, u_hi;
    R u_rem, u_err, u_off, u_aoff;
    u128 u_gab;
    i128 u_pre;
    // FP32 bound check: the FP64 shadow of the current level and, per level, its owner's copy
    Shadow64 SH{};
    double w_rem = 0, w_err = 0, w_off = 0, w_aoff = 0;
    double slack64 = 0, Kerr64 = 0;
    if constexpr (CHK) {
        slack64 = fmax(A.eps, Num<double>::G() * ((double)P.qmax + 1.0)) + P.slack_chol;
        Kerr64 = 2.0 * (double)(d + 8) * Num<double>::U();
    }
    if (!it) {                                    // the root of the direction
        top = i = d - 1;
        u_rem = P.qmax_r; u_err = P.Kerr * P.qmax_r; u_gab = 0;
        int st = enter_level<R, NS>(S, P, i, u_rem, u_err, u_gab, lane, u_cur, u_hi, u_off, u_aoff, u_pre);
        if (st) return st;
        T.nodes++;
        if constexpr (CHK) {
            w_rem = (double)P.qmax; w_err = Kerr64 * w_rem; w_off = 0; w_aoff = 0;
            shadow_interval(P, i, u_rem, u_err, u_gab, u_off, u_aoff, w_rem, w_err, w_off, w_aoff, slack64, Kerr64, *acc);
            LSET(SH, rem, i, w_rem); LSET(SH, err, i, w_err); LSET(SH, off, i, w_off); LSET(SH, aoff, i, w_aoff);
        }
    } else {                                      // a donated node
        top = i = it->level;
        if (lane > i && lane < d) S.c0 = it->c[lane];
        if (NS > 1 && lane + 32 > i && lane + 32 < d) S.c1 = it->c[lane + 32];
        // exact incremental sums from scratch
        for (int j = i + 1; j < d; ++j) {
            int32_t cj = shfl((NS > 1 && j >= 32) ? S.c1 : S.c0, j & 31);
            apply_dc<R, NS>(S, P, j, cj, lane);
        }
        R off, aoff;
        i128 pre;
        level_sums<R, NS>(S, P, i, lane, off, aoff, pre);
        const u128 gab = ((u128)it->ghi << 64) | it->glo;
        LSET(S, cur, i, it->cur); LSET(S, hi, i, it->hi);
        LSET(S, rem, i, (R)it->rem); LSET(S, err, i, (R)it->err);
        LSET(S, off, i, off); LSET(S, aoff, i, aoff);
        LSET(S, gab, i, gab);
        u_cur = it->cur; u_hi = it->hi; u_rem = (R)it->rem; u_err = (R)it->err;
        u_off = off; u_aoff = aoff; u_gab = gab; u_pre = pre;
    }
    const R slack = P.slack, Kerr = P.Kerr;
    // leaf data for the current level-0 node: q(v) = A0 + 2 v B0 + m00 v^2
    i128 A0 = 0;
    int64_t B0 = 0;
    if (i == 0) leaf_data<R, NS>(S, P, lane, A0, B0);
    const int64_t m00 = P.wide ? P.H[-(int64_t)P.d * P.d] : (int64_t)P.MAT[0];
    unsigned poll = 0;
    const unsigned long long t0 = shfl(gtimer(), 0);
#ifdef PFG_STAGE_CLOCKS
    long long acc_bt = 0, acc_ev = 0, acc_ds = 0, acc_gcd = 0;
#endif
    for (;;) {
        if (i > top) break;
#ifdef PFG_STAGE_CLOCKS
        const long long k0 = clock64();
#endif
        if (u_cur > u_hi) {                       // backtrack
            // (c[i] keeps its last value: nothing reads it or its share of
            // the incremental sums until the next descent to level i, which
            // applies the change from it)
            ++i;
            if (i <= top) {                       // the parent's values from its owner lane
                u_cur = LGET(S, cur, i); u_hi = LGET(S, hi, i);
                u_rem = LGET(S, rem, i); u_err = LGET(S, err, i);
                u_off = LGET(S, off, i); u_aoff = LGET(S, aoff, i);
                u_gab = shflu128((NS > 1 && i >= 32) ? S.gab1 : S.gab0, i & 31);
                // (H_i c over c[i+1:] has not changed since level i was entered)
                u_pre = ((P.hrows >> i) & 1) ? shfl128((NS > 1 && i >= 32) ? S.hp1 : S.hp0, i & 31) : (i128)0;
                if constexpr (CHK) {
                    w_rem = LGET(SH, rem, i); w_err = LGET(SH, err, i);
                    w_off = LGET(SH, off, i); w_aoff = LGET(SH, aoff, i);
                }
            }
#ifdef PFG_STAGE_CLOCKS
            acc_bt += clock64() - k0;
#endif
            continue;
        }
        const int64_t cur = u_cur, hi = u_hi;
        // donate the top of the stack when other warps are idle
        if (((++poll) & 1023) == 0 && (long long)(shfl(gtimer(), 0) - t0) > A.deadline_ns)
            return ST_WAIT;                       // (uniform: lane 0's clock)
        if (A.donate && (poll & 63) == 0) {
            int hungry = 0;
            if (lane == 0) {
                volatile SearchCtl *C = A.ctl;
                const int queued = (int)(C->q_tail - C->q_head);
                hungry = C->roots_next >= (unsigned)A.n_todo && queued < A.n_warps - C->active;
            }
            hungry = shfl(hungry, 0);
            if (hungry) {
                // highest level j in (i, top] with candidates left
                bool has0 = lane > i && lane <= top && S.cur0 <= S.hi0;
                bool has1 = NS > 1 && lane + 32 > i && lane + 32 <= top && S.cur1 <= S.hi1;
                unsigned b1 = __ballot_sync(FULL, has1), b0 = __ballot_sync(FULL, has0);
                int j = b1 ? 32 + 31 - __clz(b1) : (b0 ? 31 - __clz(b0) : -1);
                if (j >= 0) {
                    unsigned slot = 0;
                    if (lane == 0) slot = atomicAdd(&A.ctl->q_tail, 1u);
                    slot = shfl(slot, 0);
                    if (slot < A.q_cap) {
                        WorkItem *dst = A.items + slot;
                        const int64_t jc = LGET(S, cur, j), jh = LGET(S, hi, j);
                        const R jr = LGET(S, rem, j), je = LGET(S, err, j);
                        const u128 jg = shflu128((NS > 1 && j >= 32) ? S.gab1 : S.gab0, j & 31);
                        if (lane == 0) {
                            dst->pid = pid; dst->level = j; dst->cur = jc; dst->hi = jh;
                            dst->rem = (double)jr; dst->err = (double)je;
                            dst->glo = (uint64_t)jg; dst->ghi = (uint64_t)(jg >> 64);
                        }
                        if (lane > j && lane < d) dst->c[lane] = S.c0;
                        if (NS > 1 && lane + 32 > j && lane + 32 < d) dst->c[lane + 32] = S.c1;
                        __threadfence();
                        __syncwarp();
                        if (lane == 0) { atomicExch(&A.ready[slot], 1); atomicAdd(&A.ctl->donated, 1ull); }
                        LSET(S, hi, j, jc - 1);       // (j > i: not the current level)
                    }
                }
            }
        }
        const R rem = u_rem, err = u_err, off = u_off, aoff = u_aoff;
        const u128 gab = u_gab;
        const i128 pre = u_pre;
        const bool hrow = (P.hrows >> i) & 1;
        const int64_t hii = P.HD[i];
        const R uii = P.U[upk(i, i, d)];
        const int64_t ncand = min((int64_t)32, hi - cur + 1);
        const int64_t v = cur + lane;
        bool pass = lane < ncand;
        R nr = 0, en = 0;
        u128 gn = gab;
        bool ferr = false;
        double nr64 = 0, en64 = 0;
        if (pass) {
            R x = uii * (R)v + off;
            nr = rem - x * x;
            R ai = fabs(uii * (R)v) + aoff;
            en = err + Kerr * (ai * ai + rem);
            if constexpr (CHK) {
                const double u64 = P.U64[i * d + i];
                const double x64 = u64 * (double)v + w_off;
                nr64 = w_rem - x64 * x64;
                const double ai64 = fabs(u64 * (double)v) + w_aoff;
                en64 = w_err + Kerr64 * (ai64 * ai64 + w_rem);
                const double dr = fabs((double)nr - nr64);
                acc->rem = fmax(acc->rem, dr);
                acc->frac = fmax(acc->frac, dr / ((double)slack + (double)en));
            }
            if (en > P.max_err) { ferr = true; pass = false; }
            else if (nr < -(slack + en)) pass = false;
        }
        if (pass && i == P.m0_level && (i128)P.g_lin * v < (i128)P.linmin) pass = false;
#ifdef PFG_STAGE_CLOCKS
        const long long kg0 = clock64();
#endif
        if (pass) {
            const R q_lb = (P.qmax_r - nr) - (slack + en);
            if (hrow) {
                if (gcd_fails(gn, P.Q, q_lb, P.coni)) pass = false;
                else {
                    u128 a = uabs(pre + (i128)hii * v);
                    if ((gn >> 64) == 0 && (a >> 64) == 0 && (gn | a) != 0) {
                        uint64_t gg = gcd64_ge_small((uint64_t)gn, (uint64_t)a, need_of(q_lb, P.invQ, P.coni));
                        if (!gg) pass = false;
                        gn = gg;
                    } else {
                        gn = gcd128(gn, a);
                    }
                }
            }
            if (pass && gcd_fails(gn, P.Q, q_lb, P.coni)) pass = false;
        }
#ifdef PFG_STAGE_CLOCKS
        __syncwarp();
        acc_gcd += clock64() - kg0;
#endif
        if (__any_sync(FULL, ferr)) return ST_FLOAT;
        T.cands += (unsigned long long)ncand;
        unsigned mask = __ballot_sync(FULL, pass);
#ifdef PFG_STAGE_CLOCKS
        const long long k1 = clock64();
        acc_ev += k1 - k0;
#endif
        if (i > 0) {
            if (!mask) { u_cur = cur + ncand; continue; }
            const int t0 = __ffs(mask) - 1;
            const int64_t vc = cur + t0;
            u_cur = vc + 1;
            LSET(S, cur, i, u_cur);               // (for the return to this level and for donation)
            const R nr0 = shfl(nr, t0), en0 = shfl(en, t0);
            const u128 g0 = shflu128(gn, t0);
            const int32_t ci = LGET(S, c, i);
            apply_dc<R, NS>(S, P, i, vc - ci, lane);
            LSET(S, c, i, (int32_t)vc);
            --i;
            u_rem = nr0; u_err = en0; u_gab = g0;
            int st = enter_level<R, NS>(S, P, i, u_rem, u_err, u_gab, lane, u_cur, u_hi, u_off, u_aoff, u_pre);
            if (st) return st;
            T.nodes++;
            if constexpr (CHK) {
                w_rem = shfl(nr64, t0); w_err = shfl(en64, t0);
                shadow_sums<NS>(S, P, i, lane, w_off, w_aoff);
                shadow_interval(P, i, u_rem, u_err, u_gab, u_off, u_aoff, w_rem, w_err, w_off, w_aoff, slack64,
                                Kerr64, *acc);
                LSET(SH, rem, i, w_rem); LSET(SH, err, i, w_err); LSET(SH, off, i, w_off); LSET(SH, aoff, i, w_aoff);
            }
            if (i == 0) leaf_data<R, NS>(S, P, lane, A0, B0);
#ifdef PFG_STAGE_CLOCKS
            acc_ds += clock64() - k1;
#endif
            continue;
        }
        // leaves: exact q, exact gcd of Kn[1:], emission
        u_cur = cur + ncand;
        if (!mask) continue;
        PFG_SCLK(c_leaf);
        T.leaves += __popc(mask);
        bool ok = pass;
        i128 q = 0;
        if (ok) {
            // (|v| < 2^31: 2 v and v^2 are int64 values, so both products are 64 x 64-bit)
            q = A0 + (i128)(2 * v) * (i128)B0 + (i128)m00 * (i128)(v * v);
            if (q > (i128)P.qmax) ok = false;
        }
        // Q g > q (coni: g = gcd(Kn[1:])) or Q g >= q (non-coni: g = gcd(Kn)) needs g exactly
        // where g = 1 would not already pass
        unsigned need_g = __ballot_sync(FULL, ok && (P.coni ? q >= (i128)P.Q : q > (i128)P.Q));
        const int k_lo = P.coni ? 1 : 0;
        while (need_g) {
            const int t = __ffs(need_g) - 1;
            need_g &= need_g - 1;
            const int64_t vt = cur + t;
            const i128 qt = shfl128(q, t);
            uint64_t g = 0;
            if (lane >= k_lo && lane < h) g = gcd64(g, uabs64(S.k0 + (int64_t)P.ZT[lane] * vt));
            if (NS > 1 && lane + 32 < h) g = gcd64(g, uabs64(S.k1 + (int64_t)P.ZT[lane + 32] * vt));
            for (int o = 16; o; o >>= 1) g = gcd64(g, __shfl_xor_sync(FULL, g, o));
            if (g != 0 && lane == t && (P.coni ? (i128)P.Q * (i128)g <= qt : (i128)P.Q * (i128)g < qt)) ok = false;
        }
        unsigned emit = __ballot_sync(FULL, ok);
#ifdef PFG_STAGE_CLOCKS
        if (!emit) { PFG_SCLK(c_leaf_end); PFG_SADD(6, c_leaf_end - c_leaf); continue; }
#else
        if (!emit) continue;
#endif
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(A.npts, (unsigned long long)__popc(emit));
        base = __shfl_sync(FULL, base, 0);
        unsigned e2 = emit;
        for (unsigned k = 0; e2; ++k) {
            const int t = __ffs(e2) - 1;
            e2 &= e2 - 1;
            const unsigned long long slot = base + k;
            if (slot >= A.pts_cap) continue;
            const int64_t vt = cur + t;
            const i128 qt = shfl128(q, t);
            if (lane == 0) {
                A.hdr[slot].pid = pid;
                A.hdr[slot].pad = A.pass;
                A.hdr[slot].q = (int64_t)qt;
            }
            int32_t *cc = A.coords + slot * MD;
            if (lane == 0) cc[0] = (int32_t)vt;
            else if (lane < d) cc[lane] = S.c0;
            if (NS > 1 && lane + 32 < d) cc[lane + 32] = S.c1;
        }
#ifdef PFG_STAGE_CLOCKS
        PFG_SCLK(c_leaf_end);
        PFG_SADD(6, c_leaf_end - c_leaf);
#endif
    }
#ifdef PFG_STAGE_CLOCKS
    if (lane == 0 && sizeof(R) == 8) {
        atomicAdd(&pfg_search_cycles[8], (unsigned long long)acc_bt);
        atomicAdd(&pfg_search_cycles[9], (unsigned long long)acc_ev);
        atomicAdd(&pfg_search_cycles[10], (unsigned long long)acc_ds);
        atomicAdd(&pfg_search_cycles[11], (unsigned long long)acc_gcd);
    }
#endif
    return 0;
}

template <class R>
__device__ void finish_item(const SearchArgs &A, int pid, int st, Tally &T, int lane)
{
    if (lane == 0) {
        atomicAdd(&A.dir_nodes[pid], T.nodes);
        atomicAdd(&A.ctl->nodes, T.nodes);
        atomicAdd(&A.ctl->cands, T.cands);
        atomicAdd(&A.ctl->leaves, T.leaves);
        if (st) atomicCAS(&A.dirs[pid].status, ST_PENDING, st);
    }
    T.nodes = T.cands = T.leaves = 0;
}

// Persistent batched search: warps take directions from the todo list, then
// donated nodes from the queue; all bounded waits report ST_WAIT.
#ifdef PFG_EMU
static unsigned char emu_stage[64 * 1024];
#define PFG_STAGE_AREA(A) ((void *)emu_stage)
#else
#define PFG_STAGE_AREA(A) ((void *)(pfg_stage_smem + (threadIdx.x >> 5) * (A).stage_bytes))
#endif

// Blocks of at most SEARCH_WARPS warps, SEARCH_BLOCKS(NS) per SM: the
// search's registers then fit without spilling to local memory.
constexpr int SEARCH_WARPS = 4;
#ifndef PFG_SEARCH_BLOCKS1
#define PFG_SEARCH_BLOCKS1 4
#endif
template <int NS> constexpr int search_blocks() { return NS == 1 ? PFG_SEARCH_BLOCKS1 : 3; }
template <class R, int NS>
__global__ void __launch_bounds__(SEARCH_WARPS * 32, search_blocks<NS>()) k_search(SearchArgs A)
{
#ifndef PFG_EMU
    extern __shared__ __align__(16) unsigned char pfg_stage_smem[];
#endif
    void *stage = PFG_STAGE_AREA(A);
    const int lane = threadIdx.x & 31;
    Tally T{0, 0, 0};
    const unsigned long long t_start = gtimer();
    for (;;) {
        PFG_SCLK(c_wait);
        int pid = -1;
        const WorkItem *it = nullptr;
        int got = 0;                              // 1 root, 2 queue item
        if (lane == 0) {
            volatile SearchCtl *C = A.ctl;
            for (;;) {
                // 'active' counts warps holding work; idle warps only read it.
                // A warp raises it just before grabbing an item it has seen,
                // and a worker pushes its donations before lowering it.
                if (C->roots_next < (unsigned)A.n_todo) {
                    atomicAdd(&A.ctl->active, 1);
                    unsigned r = atomicAdd(&A.ctl->roots_next, 1u);
                    if (r < (unsigned)A.n_todo) { got = 1; pid = A.todo[r]; break; }
                    atomicSub(&A.ctl->active, 1);
                }
                unsigned head = C->q_head, tail = C->q_tail;
                if (tail > A.q_cap) tail = A.q_cap;
                if (head < tail) {
                    atomicAdd(&A.ctl->active, 1);
                    if (atomicCAS(&A.ctl->q_head, head, head + 1) == head) {
                        volatile int *rd = A.ready + head;
                        long long spins = 0;
                        while (*rd == 0 && spins < (1LL << 22)) { __nanosleep(64); ++spins; }
                        __threadfence();
                        if (*rd) { got = 2; it = A.items + head; pid = it->pid; break; }
                        atomicCAS(&A.ctl->err, 0, ST_WAIT);     // a reserved slot never filled
                        atomicSub(&A.ctl->active, 1);
                        break;
                    }
                    atomicSub(&A.ctl->active, 1);
                    continue;
                }
                // finished when nobody holds work and, after that, nothing is queued
                if (C->active == 0) {
                    __threadfence();
                    unsigned h2 = C->q_head, t2 = C->q_tail;
                    if (t2 > A.q_cap) t2 = A.q_cap;
                    if (h2 >= t2 && C->roots_next >= (unsigned)A.n_todo) break;
                }
                if ((long long)(gtimer() - t_start) > A.wait_ns || C->err) {
                    atomicCAS(&A.ctl->err, 0, ST_WAIT);
                    break;
                }
                __nanosleep(256);
            }
        }
        got = shfl(got, 0);
        if (!got) break;
        pid = shfl(pid, 0);
        unsigned long long ip = shfl((unsigned long long)it, 0);
        it = (const WorkItem *)ip;
        int st = 0;
        int pending = 0;
        PFG_SCLK(c_run);
        if (lane == 0) pending = ((volatile Dir *)A.dirs)[pid].status == ST_PENDING;
        if (shfl(pending, 0)) {                   // (skip work of a direction that already failed)
            const Prob<R> P = load_prob<R>(A, pid, stage, lane);
            st = run_subtree<R, NS>(A, P, pid, it, T, lane);
        }
#ifdef PFG_STAGE_CLOCKS
        PFG_SCLK(c_end);
        PFG_SADD(0, c_end - c_run);
        PFG_SADD(2, c_run - c_wait);
        PFG_SADD(4, 1);
#endif
        finish_item<R>(A, pid, st, T, lane);
        __threadfence();
        if (lane == 0) atomicSub(&A.ctl->active, 1);
    }
}

// The plain form: one warp (block) per direction, no work sharing; pid < 0
// takes the block's direction todo[blockIdx.x].
template <class R, int NS, bool CHK = false>
__global__ void __launch_bounds__(32) k_search_plain(SearchArgs A, int pid)
{
    if (pid < 0) {
        if ((int)blockIdx.x >= A.n_todo) return;
        pid = A.todo[blockIdx.x];
    }
#ifndef PFG_EMU
    extern __shared__ __align__(16) unsigned char pfg_stage_smem[];
#endif
    void *stage = PFG_STAGE_AREA(A);
    const int lane = threadIdx.x & 31;
    Tally T{0, 0, 0};
    int pending = 0;
    if (lane == 0) pending = A.dirs[pid].status == ST_PENDING;
    if (!shfl(pending, 0)) return;
    const Prob<R> P = load_prob<R>(A, pid, stage, lane);
    BoundAcc acc{0, 0, 0, 0};
    int st = run_subtree<R, NS, CHK>(A, P, pid, nullptr, T, lane, &acc);
    finish_item<R>(A, pid, st, T, lane);
    if constexpr (CHK) {
        // the warp's maxima (each lane saw its own candidates), then the launch's
        double m[3] = {acc.rem, acc.frac, acc.end};
        for (int k = 0; k < 3; ++k)
            for (int o = 16; o; o >>= 1) m[k] = fmax(m[k], __shfl_xor_sync(FULL, m[k], o));
        if (lane == 0) {
            atomicMax(&A.ctl->chk_rem, (unsigned long long)__double_as_longlong(m[0]));
            atomicMax(&A.ctl->chk_frac, (unsigned long long)__double_as_longlong(m[1]));
            atomicMax(&A.ctl->chk_end, (unsigned long long)__double_as_longlong(m[2]));
            atomicAdd(&A.ctl->chk_narrower, acc.narrower);
        }
    }
}

}  // namespace pfg
