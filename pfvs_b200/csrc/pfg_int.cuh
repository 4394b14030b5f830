// Exact integer helpers for the device code: checked int128 arithmetic,
// binary gcd with an early exit, floor division, extended Euclid.
#pragma once
#include <cstdint>

typedef __int128 i128;
typedef unsigned __int128 u128;

#define PFG_HD __host__ __device__ __forceinline__

// Out-of-line device functions: the setup's reduction routines are called
// from several stages, and one shared copy keeps the kernel's hot code small
// enough for the instruction caches.
#ifdef PFG_EMU
#define PFG_NOINLINE
#else
#define PFG_NOINLINE __noinline__
#endif
// The LLL's size reduction and swap, inlined into the one out-of-line LLL: called
// once per loop iteration, a call there costs the saving and restoring of live
// registers through local memory.  (Its Gram-Schmidt row stays out of line: it is
// called from three places, and one copy of it keeps the loop's code smaller.)
#ifndef PFG_LLL_INLINE
#ifdef PFG_EMU
#define PFG_LLL_INLINE
#else
#define PFG_LLL_INLINE __forceinline__
#endif
#endif

// PFG_UNIFORM(v): v must be equal in all lanes of the warp (a warp-uniform
// branch input).  Checked only under the test-suite's CPU warp emulator.
#ifdef PFG_EMU
#define PFG_UNIFORM(v) emu_uniform((long long)(v), __LINE__)
#else
#define PFG_UNIFORM(v) ((void)0)
#endif

namespace pfg {

PFG_HD u128 uabs(i128 x) { return x < 0 ? (u128)0 - (u128)x : (u128)x; }
PFG_HD uint64_t uabs64(int64_t x) { return x < 0 ? (uint64_t)0 - (uint64_t)x : (uint64_t)x; }

// |x| < 2^63 and x != INT64_MIN (so negation and division by -1 are defined)
PFG_HD bool fits64(i128 x) { return x <= (i128)INT64_MAX && x > (i128)INT64_MIN; }

// a + b, a - b with overflow detection (true on overflow)
PFG_HD bool add_ovf(i128 a, i128 b, i128 *r)
{
    i128 s = (i128)((u128)a + (u128)b);
    *r = s;
    return ((a >= 0) == (b >= 0)) && ((s >= 0) != (a >= 0));
}
PFG_HD bool sub_ovf(i128 a, i128 b, i128 *r)
{
    i128 s = (i128)((u128)a - (u128)b);
    *r = s;
    return ((a >= 0) != (b >= 0)) && ((s >= 0) != (a >= 0));
}
// a * b with overflow detection: true iff |a b| > 2^127 - 1.  The magnitude
// product is formed from 64-bit limbs (no 128-bit division): when both
// magnitudes reach 2^64 it is at least 2^128; otherwise one factor x is below
// 2^64 and |a b| = hi(u) x 2^64 + lo(u) x for the other factor u.
PFG_HD bool mul_ovf(i128 a, i128 b, i128 *r)
{
    // both int64 values (the usual case): one 64 x 64 -> 128-bit product, which
    // always fits (|a b| <= 2^126), instead of a full 128 x 128-bit multiply
    const int64_t a64 = (int64_t)a, b64 = (int64_t)b;
    if ((i128)a64 == a && (i128)b64 == b) { *r = (i128)a64 * (i128)b64; return false; }
    u128 ua = uabs(a), ub = uabs(b);
    const u128 lim = (u128)1 << 63;
    if (ua < lim && ub < lim) { *r = a * b; return false; }
    if ((uint64_t)(ua >> 64) && (uint64_t)(ub >> 64)) return true;
    if (ub >> 64) { u128 t = ua; ua = ub; ub = t; }
    const uint64_t x = (uint64_t)ub;
    const u128 p0 = (u128)(uint64_t)ua * x, p1 = (u128)(uint64_t)(ua >> 64) * x;
    if ((uint64_t)(p1 >> 64)) return true;
    const u128 hi = (p0 >> 64) + (u128)(uint64_t)p1;
    if (hi >> 63) return true;
    const u128 m = (hi << 64) | (u128)(uint64_t)p0;
    *r = ((a < 0) != (b < 0)) ? -(i128)m : (i128)m;
    return false;
}

PFG_HD int ctz64(uint64_t x)
{
#ifdef __CUDA_ARCH__
    return __ffsll((long long)x) - 1;
#else
    return __builtin_ctzll(x);
#endif
}
PFG_HD int ctz128(u128 x)
{
    uint64_t lo = (uint64_t)x;
    return lo ? ctz64(lo) : 64 + ctz64((uint64_t)(x >> 64));
}

// Stein's binary gcd
PFG_HD uint64_t gcd64(uint64_t u, uint64_t v)
{
    if (u == 0) return v;
    if (v == 0) return u;
    int sh = ctz64(u | v);
    u >>= ctz64(u);
    do {
        v >>= ctz64(v);
        if (u > v) { uint64_t t = v; v = u; u = t; }
        v -= u;
    } while (v);
    return u << sh;
}

// gcd(u, v) if it is >= need, else 0 (u, v not both 0): the odd part of the
// gcd is at most min(u, v) after each step, so stop once that cannot reach need.
PFG_HD uint64_t gcd64_ge(uint64_t u, uint64_t v, uint64_t need)
{
    if (u == 0) return v >= need ? v : 0;
    if (v == 0) return u >= need ? u : 0;
    int sh = ctz64(u | v);
    uint64_t need_s = (need >> sh) + ((need & ((1ULL << sh) - 1)) != 0);
    u >>= ctz64(u);
    do {
        v >>= ctz64(v);
        if (u > v) { uint64_t t = v; v = u; u = t; }
        if (u < need_s) return 0;
        v -= u;
    } while (v);
    return u << sh;
}

PFG_HD int ctz32(uint32_t x)
{
#ifdef __CUDA_ARCH__
    return __ffs((int)x) - 1;
#else
    return __builtin_ctz(x);
#endif
}

// gcd64_ge on 32-bit operands (u != 0)
PFG_HD uint64_t gcd32_ge(uint32_t u, uint32_t v, uint64_t need)
{
    if (v == 0) return u >= need ? u : 0;
    const int sh = ctz32(u | v);
    const uint64_t need_s = (need >> sh) + ((need & ((1ULL << sh) - 1)) != 0);
    u >>= ctz32(u);
    do {
        v >>= ctz32(v);
        if (u > v) { uint32_t t = v; v = u; u = t; }
        if (u < need_s) return 0;
        v -= u;
    } while (v);
    return (uint64_t)u << sh;
}

// gcd64_ge(u, v, need) for a small u and a large v, the usual case of the
// search's GCD-row test (u = the gcd of the rows above): the binary
// algorithm needs about one step per bit of v there, so v is first reduced
// modulo u (gcd(u, v) = gcd(u, v mod u)) and the rest runs in 32 bits.
PFG_HD uint64_t gcd64_ge_small(uint64_t u, uint64_t v, uint64_t need)
{
    if (u != 0 && (u >> 32) == 0 && v > u) return gcd32_ge((uint32_t)u, (uint32_t)(v % u), need);
    return gcd64_ge(u, v, need);
}

PFG_HD u128 gcd128(u128 u, u128 v)
{
    if ((u >> 64) == 0 && (v >> 64) == 0) return gcd64((uint64_t)u, (uint64_t)v);
    if (u == 0) return v;
    if (v == 0) return u;
    int sh = ctz128(u | v);
    u >>= ctz128(u);
    do {
        v >>= ctz128(v);
        if (u > v) { u128 t = v; v = u; u = t; }
        v -= u;
        if ((u >> 64) == 0 && (v >> 64) == 0)
            return (u128)gcd64((uint64_t)u, (uint64_t)v) << sh;
    } while (v);
    return u << sh;
}

// floor division (Python //) for b != 0
PFG_HD int64_t fdiv64(int64_t a, int64_t b)
{
    int64_t q = a / b;
    if ((a % b != 0) && ((a < 0) != (b < 0))) q--;
    return q;
}
PFG_HD i128 fdiv128(i128 a, i128 b)
{
    i128 q = a / b;
    if ((a % b != 0) && ((a < 0) != (b < 0))) q--;
    return q;
}

// Extended Euclid with floor division: s a + t b = g (the sign convention of
// the reference's util.extended_euclidean / pfl_xgcd).
PFG_HD int64_t xgcd_floor(int64_t a, int64_t b, int64_t *s, int64_t *t)
{
    int64_t r0 = a, r1 = b, s0 = 1, s1 = 0, t0 = 0, t1 = 1;
    while (r1 != 0) {
        int64_t q = fdiv64(r0, r1), x;
        x = r0 - q * r1; r0 = r1; r1 = x;
        x = s0 - q * s1; s0 = s1; s1 = x;
        x = t0 - q * t1; t0 = t1; t1 = x;
    }
    *s = s0; *t = t0;
    return r0;
}

}  // namespace pfg
