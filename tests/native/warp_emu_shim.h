// Host stand-ins for the CUDA built-ins the engine's device code uses, so that the device headers
// (rovaca_b200/csrc/phmm_device*.cuh, phmm_warp32.cuh, phmm_warp64.cuh) compile with g++ and run on
// 32 host threads standing for the 32 lanes of one warp (tests/native/warp_emu.cpp).
//
// Arithmetic: every rounded intrinsic is one IEEE operation (the build passes -ffp-contract=off and
// -mfma, so fmaf / fma are single fused instructions); packed float2 operations are two of them.
// The GPU kernels run with flush-to-zero single precision (-ftz=true); each lane thread sets the
// x86 FTZ and DAZ bits, which flush single-precision denormal results and inputs the same way.  The
// FP64 path flushes explicitly (ftz in phmm_device.cuh), so the bits change no double result it keeps.
//
// Warp collectives: each lane writes its value to a per-warp slot, all lanes meet at a barrier,
// read the slot they need and meet again; the device code calls them on every lane in the same
// order (its divergent branches hold no collective).
#pragma once

#include <pmmintrin.h>
#include <xmmintrin.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>

#define __device__
#define __host__
#define __global__
#define __forceinline__ inline

struct float2 {
    float x, y;
};
struct float4 {
    float x, y, z, w;
};
inline float2 make_float2(float x, float y) { return float2{x, y}; }

inline float __fmul_rn(float a, float b) { return a * b; }
inline float __fadd_rn(float a, float b) { return a + b; }
inline float __fmaf_rn(float a, float b, float c) { return std::fmaf(a, b, c); }
inline double __dmul_rn(double a, double b) { return a * b; }
inline double __dadd_rn(double a, double b) { return a + b; }
inline double __fma_rn(double a, double b, double c) { return std::fma(a, b, c); }
inline float2 __fmul2_rn(float2 a, float2 b) { return float2{a.x * b.x, a.y * b.y}; }
inline float2 __fadd2_rn(float2 a, float2 b) { return float2{a.x + b.x, a.y + b.y}; }
inline float2 __ffma2_rn(float2 a, float2 b, float2 c) { return float2{std::fmaf(a.x, b.x, c.x), std::fmaf(a.y, b.y, c.y)}; }
inline int __double2hiint(double x)
{
    uint64_t u;
    std::memcpy(&u, &x, 8);
    return (int)(uint32_t)(u >> 32);
}
inline unsigned int min(unsigned int a, unsigned int b) { return a < b ? a : b; }

inline unsigned int atomicAdd(unsigned int* p, unsigned int v) { return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST); }
inline unsigned int atomicOr(unsigned int* p, unsigned int v) { return __atomic_fetch_or(p, v, __ATOMIC_SEQ_CST); }

namespace warp_emu {

// Sense-reversing barrier of the 32 lane threads; a waiting lane yields its core (the lanes
// outnumber the cores), which costs far less than sleeping in the kernel at every collective.
struct Barrier {
    std::atomic<int> count{32};
    std::atomic<int> sense{0};
    void arrive_and_wait()
    {
        const int s = sense.load(std::memory_order_relaxed);
        if (count.fetch_sub(1, std::memory_order_acq_rel) == 1) {
            count.store(32, std::memory_order_relaxed);
            sense.store(s ^ 1, std::memory_order_release);
        } else {
            while (sense.load(std::memory_order_acquire) == s) std::this_thread::yield();
        }
    }
};

struct Warp {
    Barrier bar;
    uint64_t slot[32];
};
inline thread_local Warp* t_warp = nullptr;
inline thread_local int t_lane = 0;

inline void enter_lane(Warp* w, int lane)
{
    t_warp = w;
    t_lane = lane;
    _mm_setcsr(_mm_getcsr() | 0x8040);  // FTZ | DAZ
}

template <typename T>
inline uint64_t bits(T v)
{
    uint64_t u = 0;
    std::memcpy(&u, &v, sizeof(T));
    return u;
}
template <typename T>
inline T from_bits(uint64_t u)
{
    T v;
    std::memcpy(&v, &u, sizeof(T));
    return v;
}

// every lane publishes v; returns lane src's value
template <typename T>
inline T exchange(T v, int src)
{
    Warp* w = t_warp;
    w->slot[t_lane] = bits(v);
    w->bar.arrive_and_wait();
    const T r = from_bits<T>(w->slot[src]);
    w->bar.arrive_and_wait();
    return r;
}

inline uint32_t ballot(bool p)
{
    Warp* w = t_warp;
    w->slot[t_lane] = p ? 1 : 0;
    w->bar.arrive_and_wait();
    uint32_t m = 0;
    for (int k = 0; k < 32; ++k) m |= (uint32_t)w->slot[k] << k;
    w->bar.arrive_and_wait();
    return m;
}

}  // namespace warp_emu

template <typename T>
inline T __shfl_up_sync(unsigned, T v, int d)
{
    const int lane = warp_emu::t_lane;
    return warp_emu::exchange(v, lane >= d ? lane - d : lane);
}
template <typename T>
inline T __shfl_sync(unsigned, T v, int src)
{
    return warp_emu::exchange(v, src & 31);
}
inline int __any_sync(unsigned, int p) { return warp_emu::ballot(p != 0) != 0; }
inline int __all_sync(unsigned, int p) { return warp_emu::ballot(p != 0) == 0xffffffffu; }
inline void __syncwarp() { warp_emu::t_warp->bar.arrive_and_wait(); }
