// TEST INFRASTRUCTURE -- never part of the product.
//
// A CPU emulation of the CUDA warp model, enough to compile the library's
// device sources (pfvs_b200/csrc/*.cuh) with g++ and run their kernels on
// the host for tests and debugging without a GPU: each lane is a host
// thread; warp collectives (__shfl*_sync, __ballot_sync, __any_sync,
// __all_sync, __syncwarp) exchange values through a per-warp barrier;
// atomics map to GCC __atomic builtins.  Warps of a grid run one after
// another (the kernels' cross-warp protocols stay correct, only serial).
#pragma once
#include <atomic>
#include <sched.h>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <algorithm>
#include <cstdio>
#include <cstdlib>

#define __device__
#define __host__
#define __global__
#define __forceinline__ inline
#define __launch_bounds__(...)
#define __shared__ static    // (blocks of one warp run one at a time)

struct dim3 { unsigned x = 1, y = 1, z = 1; };

// Barrier of the 32 lane threads: spin with yield (lanes meet at every
// collective, far too often for a sleeping barrier to keep up).
struct EmuBarrier {
    std::atomic<int> count{0};
    std::atomic<unsigned> phase{0};
    void arrive_and_wait()
    {
        const unsigned ph = phase.load(std::memory_order_acquire);
        if (count.fetch_add(1, std::memory_order_acq_rel) == 31) {
            count.store(0, std::memory_order_relaxed);
            phase.fetch_add(1, std::memory_order_acq_rel);
        } else {
            while (phase.load(std::memory_order_acquire) == ph) sched_yield();
        }
    }
};

struct EmuWarp {
    EmuBarrier bar;
    unsigned char slot[32][16];
    int site[32];
    int hist[32][64];
    int nh[32] = {};
};

inline thread_local int emu_lane = 0;
inline thread_local EmuWarp *emu_warp = nullptr;
inline thread_local dim3 threadIdx, blockIdx, blockDim, gridDim;

// Every collective records its call site; lanes meeting at different sites
// (a divergent collective: undefined behaviour on the GPU) abort the test.
inline void emu_check_site(int line)
{
    EmuWarp *W = emu_warp;
    W->site[emu_lane] = line;
    W->hist[emu_lane][W->nh[emu_lane]++ & 63] = line;
    W->bar.arrive_and_wait();
    if (emu_lane == 0)
        for (int l = 1; l < 32; ++l)
            if (W->site[l] != W->site[0]) {
                fprintf(stderr, "warp_emu: divergent collective: lane 0 at line %d, lane %d at line %d\n",
                        W->site[0], l, W->site[l]);
                for (int ll : {0, l}) {
                    fprintf(stderr, "  lane %d recent sites:", ll);
                    for (int k = 40; k >= 1; --k) fprintf(stderr, " %d", W->hist[ll][(W->nh[ll] - k) & 63]);
                    fprintf(stderr, "\n");
                }
                abort();
            }
    W->bar.arrive_and_wait();
}
template <class T> inline T emu_exchange(T v, int src, int line)
{
    EmuWarp *W = emu_warp;
    static_assert(sizeof(T) <= 16, "shuffle width");
    emu_check_site(line);
    std::memcpy(W->slot[emu_lane], &v, sizeof(T));
    W->bar.arrive_and_wait();
    T r;
    std::memcpy(&r, W->slot[src & 31], sizeof(T));
    W->bar.arrive_and_wait();
    return r;
}
inline unsigned emu_ballot(bool p, int line)
{
    EmuWarp *W = emu_warp;
    emu_check_site(line);
    W->slot[emu_lane][0] = p ? 1 : 0;
    W->bar.arrive_and_wait();
    unsigned m = 0;
    for (int l = 0; l < 32; ++l) if (W->slot[l][0]) m |= 1u << l;
    W->bar.arrive_and_wait();
    return m;
}
inline void emu_uniform(long long v, int line)
{
    long long v0 = emu_exchange(v, 0, line);
    if (emu_ballot(v != v0, line)) {
        if (emu_lane == 0) fprintf(stderr, "warp_emu: non-uniform value at line %d\n", line);
        emu_warp->bar.arrive_and_wait();
        abort();
    }
}
#define __shfl_sync(m, v, s) emu_exchange((v), (s), __LINE__)
#define __shfl_xor_sync(m, v, o) emu_exchange((v), emu_lane ^ (o), __LINE__)
#define __ballot_sync(m, p) emu_ballot((p), __LINE__)
#define __any_sync(m, p) (emu_ballot((p), __LINE__) != 0)
#define __all_sync(m, p) (emu_ballot((p), __LINE__) == 0xffffffffu)
#define __syncwarp(...) emu_check_site(__LINE__)
#define __syncthreads() emu_check_site(__LINE__)
inline void __threadfence() { __atomic_thread_fence(__ATOMIC_SEQ_CST); }
inline void __nanosleep(unsigned) { std::this_thread::yield(); }

inline int __ffs(int x) { return __builtin_ffs(x); }
inline int __ffsll(long long x) { return __builtin_ffsll(x); }
inline int __popc(unsigned x) { return __builtin_popcount(x); }
inline int __clz(int x) { return x ? __builtin_clz((unsigned)x) : 32; }
inline int __clzll(long long x) { return x ? __builtin_clzll((unsigned long long)x) : 64; }
inline unsigned long long __umul64hi(unsigned long long a, unsigned long long b)
{
    return (unsigned long long)(((unsigned __int128)a * b) >> 64);
}

template <class T, class U> inline T atomicAdd(T *p, U v) { return __atomic_fetch_add(p, (T)v, __ATOMIC_SEQ_CST); }
template <class T, class U> inline T atomicSub(T *p, U v) { return __atomic_fetch_sub(p, (T)v, __ATOMIC_SEQ_CST); }
template <class T, class U> inline T atomicExch(T *p, U v) { return __atomic_exchange_n(p, (T)v, __ATOMIC_SEQ_CST); }
template <class T, class U, class V> inline T atomicCAS(T *p, U cmp, V val)
{
    T c = (T)cmp;
    __atomic_compare_exchange_n(p, &c, (T)val, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST);
    return c;
}
template <class T, class U> inline T atomicMax(T *p, U v)
{
    T cur = __atomic_load_n(p, __ATOMIC_SEQ_CST);
    while (cur < (T)v && !__atomic_compare_exchange_n(p, &cur, (T)v, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST)) {}
    return cur;
}
inline long long __double_as_longlong(double x) { long long r; memcpy(&r, &x, sizeof r); return r; }

using std::min;
using std::max;

inline unsigned long long emu_now_ns()
{
    return (unsigned long long)std::chrono::duration_cast<std::chrono::nanoseconds>(
        std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Run `body(lane)` as one warp: 32 host threads.
template <class F> inline void emu_run_warp(unsigned block, unsigned warp_in_block, unsigned bdim,
                                            unsigned gdim, F body)
{
    EmuWarp W;
    std::thread th[32];
    for (int l = 0; l < 32; ++l)
        th[l] = std::thread([&, l] {
            emu_lane = l;
            emu_warp = &W;
            threadIdx.x = warp_in_block * 32 + l;
            blockIdx.x = block;
            blockDim.x = bdim;
            gridDim.x = gdim;
            body();
        });
    for (auto &t : th) t.join();
}
