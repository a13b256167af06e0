// Host warp emulator for the warp-synchronous device code of libeimp_b200.
//
// Compiles a kernel's CUDA C++ source as host C++ (with the sanitizers) and
// runs each warp as 32 host threads.  Every warp collective (__syncwarp,
// __ballot_sync, __any_sync, __match_any_sync, __shfl*_sync) meets at a barrier and records the
// source line each lane called it from: lanes that reach different shuffles
// or ballots (a divergent collective, undefined on the device) are counted in
// emu_divergence; __syncwarp calls from different lines are reported but
// allowed (sm_70 and later permit them).  Lanes run truly concurrently, so
// unsynchronised reads and writes of shared state show up as wrong results
// or divergence instead of hiding behind lock-step execution.
#pragma once
#include <atomic>
#include <sched.h>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <climits>

#define __device__
#define __global__
#define __host__
#define __forceinline__ inline
#define __noinline__
#define __launch_bounds__(...)
#define __align__(n) __attribute__((aligned(n)))
#define __restrict__ __restrict

typedef int cudaError_t;
typedef void *cudaStream_t;
enum { cudaSuccess = 0, cudaErrorInvalidValue = 1 };

struct dim3 { unsigned x = 0, y = 0, z = 0; };
struct int2 { int x, y; };
struct short2 { short x, y; };
struct uint2 { unsigned x, y; };
struct uint4 { unsigned x, y, z, w; };
struct float4 { float x, y, z, w; };
struct int4 { int x, y, z, w; };
inline int2 make_int2(int x, int y) { return int2{x, y}; }
inline short2 make_short2(short x, short y) { return short2{x, y}; }
inline int4 make_int4(int x, int y, int z, int w) { return int4{x, y, z, w}; }
inline uint4 make_uint4(unsigned x, unsigned y, unsigned z, unsigned w) { return uint4{x, y, z, w}; }
inline uint2 make_uint2(unsigned x, unsigned y) { return uint2{x, y}; }
inline float4 make_float4(float x, float y, float z, float w) { return float4{x, y, z, w}; }

extern thread_local dim3 threadIdx, blockIdx, blockDim;

// Barrier of the 32 lane threads: the last to arrive opens the next
// generation; the others yield the core while they wait (lanes outnumber the
// cores, and a futex wake-up of 31 threads per collective costs far more).
struct EmuBarrier {
    std::atomic<int> count{0};
    std::atomic<unsigned> gen{0};
    int n = 32;   // participating threads
    void arrive_and_wait() {
        const unsigned g = gen.load(std::memory_order_acquire);
        if (count.fetch_add(1, std::memory_order_acq_rel) == n - 1) {
            count.store(0, std::memory_order_relaxed);
            gen.fetch_add(1, std::memory_order_release);
        } else {
            while (gen.load(std::memory_order_acquire) == g) sched_yield();
        }
    }
};

struct EmuWarp {
    EmuBarrier bar;
    uint64_t vals[32];
    int sites[32];
};
extern thread_local EmuWarp *emu_warp;
// __syncthreads: a barrier of all the block's threads (drivers that run whole
// blocks set emu_block; a block's __shared__ arrays are function statics,
// shared by its threads -- blocks run one after the other)
extern thread_local EmuBarrier *emu_block;
#define __shared__ static
#define __syncthreads() emu_block->arrive_and_wait()
extern thread_local uint8_t *emu_smem_ptr;
extern std::atomic<int> emu_divergence;

inline int emu_lane() { return threadIdx.x & 31; }

template <class T> inline uint64_t emu_bits(T v) { uint64_t u = 0; std::memcpy(&u, &v, sizeof(T)); return u; }
template <class T> inline T emu_from(uint64_t u) { T v; std::memcpy(&v, &u, sizeof(T)); return v; }

inline void emu_enter(int site, uint64_t v, bool strict) {
    EmuWarp *w = emu_warp;
    const int l = emu_lane();
    w->vals[l] = v;
    w->sites[l] = site;
    w->bar.arrive_and_wait();
    if (l == 0) {
        for (int i = 1; i < 32; i++)
            if (w->sites[i] != w->sites[0]) {
                std::fprintf(stderr, "%s: lanes at different collectives: lane 0 line %d, lane %d line %d\n",
                             strict ? "DIVERGENT COLLECTIVE" : "syncwarp sites differ", w->sites[0], i,
                             w->sites[i]);
                if (strict) emu_divergence++;
                break;
            }
    }
}
inline void emu_leave() { emu_warp->bar.arrive_and_wait(); }

inline void emu_syncwarp(int site) { emu_enter(site, 0, false); emu_leave(); }
inline unsigned emu_ballot(int site, bool p) {
    emu_enter(site, p ? 1 : 0, true);
    unsigned r = 0;
    for (int i = 0; i < 32; i++) if (emu_warp->vals[i]) r |= 1u << i;
    emu_leave();
    return r;
}
template <class T> inline T emu_shfl(int site, T v, int src) {
    emu_enter(site, emu_bits(v), true);
    T r = emu_from<T>(emu_warp->vals[src & 31]);
    emu_leave();
    return r;
}
template <class T> inline T emu_shfl_up(int site, T v, int d) {
    emu_enter(site, emu_bits(v), true);
    const int l = emu_lane();
    T r = l >= d ? emu_from<T>(emu_warp->vals[l - d]) : v;
    emu_leave();
    return r;
}
template <class T> inline T emu_shfl_down(int site, T v, int d) {
    emu_enter(site, emu_bits(v), true);
    const int l = emu_lane();
    T r = l + d < 32 ? emu_from<T>(emu_warp->vals[l + d]) : v;
    emu_leave();
    return r;
}
template <class T> inline T emu_shfl_xor(int site, T v, int m) {
    emu_enter(site, emu_bits(v), true);
    T r = emu_from<T>(emu_warp->vals[(emu_lane() ^ m) & 31]);
    emu_leave();
    return r;
}
inline unsigned emu_match_any(int site, uint64_t v) {
    emu_enter(site, v, true);
    unsigned r = 0;
    const uint64_t mine = emu_warp->vals[emu_lane()];
    for (int i = 0; i < 32; i++) if (emu_warp->vals[i] == mine) r |= 1u << i;
    emu_leave();
    return r;
}
#define __syncwarp(...) emu_syncwarp(__LINE__)
#define __match_any_sync(m, v) emu_match_any(__LINE__, emu_bits(v))
#define __ballot_sync(m, p) emu_ballot(__LINE__, (p))
#define __any_sync(m, p) (emu_ballot(__LINE__, (p)) != 0u)
#define __shfl_sync(m, v, s) emu_shfl(__LINE__, (v), (s))
#define __shfl_up_sync(m, v, d) emu_shfl_up(__LINE__, (v), (d))
#define __shfl_xor_sync(m, v, x) emu_shfl_xor(__LINE__, (v), (x))
#define __shfl_down_sync(m, v, d) emu_shfl_down(__LINE__, (v), (d))

inline int __popc(unsigned x) { return __builtin_popcount(x); }
inline int __popcll(unsigned long long x) { return __builtin_popcountll(x); }
inline int __clz(int x) { return x ? __builtin_clz((unsigned)x) : 32; }
inline int __clzll(long long x) { return x ? __builtin_clzll((unsigned long long)x) : 64; }
inline int __ffs(int x) { return __builtin_ffs(x); }
inline int __ffsll(long long x) { return __builtin_ffsll(x); }
inline unsigned __float_as_uint(float f) { unsigned u; std::memcpy(&u, &f, 4); return u; }
inline float __uint_as_float(unsigned u) { float f; std::memcpy(&f, &u, 4); return f; }
inline float __int_as_float(int u) { float f; std::memcpy(&f, &u, 4); return f; }
inline double __longlong_as_double(long long u) { double f; std::memcpy(&f, &u, 8); return f; }
inline long long __double_as_longlong(double f) { long long u; std::memcpy(&u, &f, 8); return u; }
// IEEE round-to-nearest, one operation each (built with -ffp-contract=off)
inline float __fadd_rn(float a, float b) { volatile float r = a + b; return r; }
inline float __fmul_rn(float a, float b) { volatile float r = a * b; return r; }
inline float __fdiv_rn(float a, float b) { volatile float r = a / b; return r; }
inline double __dadd_rn(double a, double b) { volatile double r = a + b; return r; }
inline double __dmul_rn(double a, double b) { volatile double r = a * b; return r; }
inline double __dsub_rn(double a, double b) { volatile double r = a - b; return r; }
inline double __ddiv_rn(double a, double b) { volatile double r = a / b; return r; }
inline float __fsub_rn(float a, float b) { volatile float r = a - b; return r; }
using std::ldexp;
inline int min(int a, int b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }

inline int atomicAdd(int *p, int v) { return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST); }
inline unsigned atomicAdd(unsigned *p, unsigned v) { return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST); }
inline int atomicSub(int *p, int v) { return __atomic_fetch_sub(p, v, __ATOMIC_SEQ_CST); }
inline int atomicCAS(int *p, int c, int v) {
    __atomic_compare_exchange_n(p, &c, v, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST);
    return c;
}
inline int atomicMin(int *p, int v) {
    int o = __atomic_load_n(p, __ATOMIC_SEQ_CST);
    while (v < o && !__atomic_compare_exchange_n(p, &o, v, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST)) {}
    return o;
}
inline unsigned atomicOr(unsigned *p, unsigned v) { return __atomic_fetch_or(p, v, __ATOMIC_SEQ_CST); }
inline unsigned long long atomicOr(unsigned long long *p, unsigned long long v) {
    return __atomic_fetch_or(p, v, __ATOMIC_SEQ_CST);
}
inline unsigned long long atomicAnd(unsigned long long *p, unsigned long long v) {
    return __atomic_fetch_and(p, v, __ATOMIC_SEQ_CST);
}
inline unsigned __funnelshift_r(unsigned lo, unsigned hi, unsigned sh) {
    const uint64_t v = ((uint64_t)hi << 32) | lo;
    return (unsigned)(v >> (sh & 31));
}
inline unsigned long long atomicAdd(unsigned long long *p, unsigned long long v) {
    return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST);
}
inline double atomicAdd(double *p, double v) {
    double o, n;
    __atomic_load(p, &o, __ATOMIC_SEQ_CST);
    do { n = o + v; } while (!__atomic_compare_exchange(p, &o, &n, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST));
    return o;
}
inline int atomicOr(int *p, int v) { return __atomic_fetch_or(p, v, __ATOMIC_SEQ_CST); }
