// Shared device helpers for the nwgrad_b200 kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <mutex>

namespace nwg {

// Let `fn` launch with `bytes` of dynamic shared memory.  The attribute only ever grows, under
// a lock: a launch prepared (or captured) with a larger size by another bucket or thread stays
// valid.
inline cudaError_t allow_smem(const void* fn, size_t bytes) {
    if (bytes <= 48 * 1024) return cudaSuccess;
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, size_t> set;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(mu);
    size_t& cur = set[{dev, fn}];
    if (bytes <= cur) return cudaSuccess;
    const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
    if (e == cudaSuccess) cur = bytes;
    return e;
}

// The reference's max: std::max keeps the first argument on ties and on a NaN second
// argument: (a < b) ? b : a.  Kept as a compare + select (not fmaxf) so signed zeros and
// NaNs propagate exactly as in the reference's scalar fill.
template <class T> __device__ __forceinline__ T rmax(T a, T b) { return (a < b) ? b : a; }
template <class T> __device__ __forceinline__ T rmax3(T a, T b, T c) { return rmax(rmax(a, b), c); }

// The hardware max (FMNMX): equal to rmax except for the sign of an exact zero and NaNs.
__device__ __forceinline__ float hmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double hmax(double a, double b) { return fmax(a, b); }
template <class T> __device__ __forceinline__ T hmax3(T a, T b, T c) { return hmax(hmax(a, b), c); }

// The predecessor code of one state: 0 first argument (M), 1 second (X), 2 third (Y),
// by >= in M, X, Y order (aligner.hpp:3977-3980).
template <class T> __device__ __forceinline__ uint32_t pick3(T vm, T vx, T vy) {
    const uint32_t kxy = vx >= vy ? 1u : 2u;
    return vm >= hmax(vx, vy) ? 0u : kxy;
}

// Round-to-nearest multiply and add that the compiler never fuses into an FMA (the
// reference is compiled with -ffp-contract=off: its closed-form borders round twice).
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }

__device__ __forceinline__ float fmaf_t(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fmaf_t(double a, double b, double c) { return fma(a, b, c); }

template <class T> __device__ __forceinline__ T ninf();
template <> __device__ __forceinline__ float ninf<float>() { return __int_as_float(0xff800000u); }
template <> __device__ __forceinline__ double ninf<double>() { return __longlong_as_double(0xfff0000000000000ull); }

// Exact powers of two for the soft path's exponent bookkeeping: 2^e, flushed to 0 below
// the normal range and to +inf above it.
template <class T> __device__ __forceinline__ T pow2i(int e);
template <> __device__ __forceinline__ float pow2i<float>(int e) {
    if (e < -126) return 0.0f;
    if (e > 127) return __int_as_float(0x7f800000);
    return __int_as_float((e + 127) << 23);
}
template <> __device__ __forceinline__ double pow2i<double>(int e) {
    if (e < -1022) return 0.0;
    if (e > 1023) return __longlong_as_double(0x7ff0000000000000ll);
    return __longlong_as_double(static_cast<long long>(e + 1023) << 52);
}
// 2^e with gradual underflow: subnormal for float e in [-149, -127] (double: [-1074, -1023]),
// 0 below, so a value scaled by it loses at most half the smallest subnormal.
template <class T> __device__ __forceinline__ T pow2s(int e);
template <> __device__ __forceinline__ float pow2s<float>(int e) {
    if (e >= -126) return pow2i<float>(e);
    if (e < -149) return 0.0f;
    return __int_as_float(1 << (e + 149));
}
template <> __device__ __forceinline__ double pow2s<double>(int e) {
    if (e >= -1022) return pow2i<double>(e);
    if (e < -1074) return 0.0;
    return __longlong_as_double(1ll << (e + 1074));
}
// v * 2^d for d <= 0 with gradual underflow: the result is v * 2^d rounded once into the
// subnormal range (or 0 when below half the smallest subnormal for v < 2), never a
// flush of a value that float could still hold.
template <class T> __device__ __forceinline__ T scale_down(T v, int d) {
    constexpr int lo = sizeof(T) == 4 ? -126 : -1022;
    if (d >= lo) return v * pow2i<T>(d);
    v *= pow2i<T>(lo);
    return v * pow2s<T>(d - lo);
}
// floor(log2(x)) for a finite x > 0 (normal or subnormal handled via the bits).
template <class T> __device__ __forceinline__ int ilog2(T x);
template <> __device__ __forceinline__ int ilog2<float>(float x) {
    const uint32_t u = __float_as_uint(x);
    const int e = int((u >> 23) & 0xff);
    if (e) return e - 127;
    return -127 - __clz(u << 9);   // subnormal: position of the top set mantissa bit
}
template <> __device__ __forceinline__ int ilog2<double>(double x) {
    const unsigned long long u = __double_as_longlong(x);
    const int e = int((u >> 52) & 0x7ff);
    if (e) return e - 1023;
    return -1023 - __clzll(static_cast<long long>(u << 12));
}
// Bring [p, p + bytes) into L2 ahead of its use (the bulk-copy engine's prefetch: p 16-byte
// aligned, bytes a multiple of 16); no data returns to the issuing thread.
__device__ __forceinline__ void prefetch_l2_bulk(const void* p, unsigned bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}
__device__ __forceinline__ void prefetch_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p) : "memory");
}
// Work queue of one persistent launch: q[0] the next item of the launch's order (longest
// first), q[1] the groups that have found it empty.  A group's leader draws items until one is
// past the end; the last of the launch's ngroups groups to do so resets both counters, so the
// next launch (or graph replay) on the same counters starts at zero without a memset.
__device__ __forceinline__ int64_t wq_next(int* q, int ngroups, int64_t n_items) {
    const int64_t it = atomicAdd(q, 1);
    if (it >= n_items && atomicAdd(q + 1, 1) == ngroups - 1) {
        atomicExch(q, 0);
        atomicExch(q + 1, 0);
    }
    return it;
}
__device__ __forceinline__ bool is_finite(float x) { return (__float_as_uint(x) & 0x7f800000u) != 0x7f800000u; }
__device__ __forceinline__ bool is_finite(double x) {
    return (static_cast<unsigned long long>(__double_as_longlong(x)) & 0x7ff0000000000000ull) != 0x7ff0000000000000ull;
}

}  // namespace nwg
