// common.cuh -- shared device/host definitions for the PGGC B200 library.
//
// Canonical arithmetic (shared by definition with the CPU oracle):
//  * every FP32 operation is separately rounded (the library is compiled with
//    -fmad=false; no FMA contraction), including the int->float conversions the
//    reference performs implicitly (src/local_mover.cpp:484,498,324);
//  * weight sums are int64 for integer graphs and FP64 for FP32-weighted graphs;
//  * per-vertex FP64 edge reductions use 32 lane-strided partials combined by an
//    xor butterfly (degree < 15000) or 1024 thread-strided partials, butterfly per
//    warp, butterfly over the 32 warp totals (degree >= 15000);
//  * FP64 array reductions / scans are groups of 32 (xor butterfly / Kogge-Stone)
//    applied recursively to group totals.
#pragma once
#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <limits>
#include <stdexcept>
#include <string>
#include <type_traits>

namespace pggc {

using i32 = int32_t;
using i64 = int64_t;
using u32 = uint32_t;
using u64 = uint64_t;

// src/local_mover.cpp:74-80
constexpr float OBJ_MIN = -3.402823466e+38f;
constexpr i32 NULL_PART = -1;
constexpr i32 NO_MOVE = -3;
constexpr i32 NEW_PART = -4;
constexpr float AFTERBURNER_EPS = 0.1f;
// src/header/ordering.h:17-19
constexpr i64 MID_CUTOFF = 64;
constexpr i64 LARGE_CUTOFF = 128;
constexpr i64 MASSIVE_CUTOFF = 15000;
// src/leidenR.cpp:38-39
constexpr i32 ORD_MAX = 2147483647;
constexpr i32 SPLIT = 1000000000;

constexpr unsigned FULL = 0xffffffffu;
constexpr int NUM_SMS = 148;

// device-side error codes latched in Context::d_err
enum DevErr : int { DEV_OK = 0, DEV_ERR_PROBE = 1, DEV_ERR_CHASE = 2, DEV_ERR_LABEL = 3, DEV_ERR_WAIT = 4 };

struct CudaError : std::runtime_error {
    cudaError_t code;
    CudaError(cudaError_t c, const std::string& where)
        : std::runtime_error(where + ": " + cudaGetErrorString(c)), code(c) {}
};
struct InvalidArg : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct DeviceFault : std::runtime_error {
    using std::runtime_error::runtime_error;
};

#define PGGC_CUDA(x)                                                                   \
    do {                                                                               \
        cudaError_t _e = (x);                                                          \
        if (_e != cudaSuccess) throw ::pggc::CudaError(_e, std::string(#x) + " @ " + \
                                                       __FILE__ + ":" + std::to_string(__LINE__)); \
    } while (0)

// Every kernel launch is followed by exactly one PGGC_LAUNCH_CHECK(), which also
// counts the launch (pggc_launch_count()).
extern std::atomic<unsigned long long> g_kernel_launches;
#define PGGC_LAUNCH_CHECK()                                                        \
    do {                                                                           \
        PGGC_CUDA(cudaGetLastError());                                             \
        ::pggc::g_kernel_launches.fetch_add(1, std::memory_order_relaxed);         \
    } while (0)

template <class W> struct Traits;
template <> struct Traits<i32> { using V = i64; };
template <> struct Traits<float> { using V = double; };

// ---------------------------------------------------------------------------
// hashes
// ---------------------------------------------------------------------------
// src/local_mover.cpp:82-87
__host__ __device__ __forceinline__ u32 xorshift32(u32 x) {
    x ^= x << 13;
    x ^= x >> 17;
    x ^= x << 5;
    return x;
}

__host__ __device__ __forceinline__ u32 rotl32(u32 x, int r) { return (x << r) | (x >> (32 - r)); }

// MurmurHash3_x86_32 of one 4-byte key, seed 0 (the hash behind Kokkos::pod_hash,
// src/leidenR.cpp:37).
__host__ __device__ __forceinline__ u32 murmur3_32(u32 key) {
    u32 k = key * 0xcc9e2d51u;
    k = rotl32(k, 15);
    k *= 0x1b873593u;
    u32 h = k;
    h = rotl32(h, 13);
    h = h * 5u + 0xe6546b64u;
    h ^= 4u;
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

// splitmix64 seed stream (replaces std::random_device)
struct SplitMix64 {
    u64 s;
    explicit SplitMix64(u64 seed) : s(seed) {}
    u64 next() {
        u64 z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
};

// ---------------------------------------------------------------------------
// small device helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

template <class V>
__device__ __forceinline__ float to_f(V x) { return static_cast<float>(x); }

__device__ __forceinline__ double butterfly_sum(double v) {
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) v = v + __shfl_xor_sync(FULL, v, d);
    return v;
}
__device__ __forceinline__ i64 warp_sum_i64(i64 v) {
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) v += __shfl_xor_sync(FULL, v, d);
    return v;
}

// Canonical per-vertex FP64 edge sum, warp flavour (degree < MASSIVE_CUTOFF).
// Every lane returns the same total.
template <class F>
__device__ __forceinline__ double warp_canon_sum(i64 b, i64 e, F term) {
    double acc = 0.0;
    for (i64 j = b + lane_id(); j < e; j += 32) acc += term(j);
    return butterfly_sum(acc);
}

// Canonical per-vertex FP64 edge sum, block-of-1024 flavour (degree >=
// MASSIVE_CUTOFF).  Must be called by all 1024 threads; `red` is 32 doubles of
// shared memory.  Every thread returns the total.
template <class F>
__device__ __forceinline__ double block1024_canon_sum(i64 b, i64 e, F term, double* red) {
    double acc = 0.0;
    for (i64 j = b + threadIdx.x; j < e; j += 1024) acc += term(j);
    acc = butterfly_sum(acc);
    __syncthreads();
    if (lane_id() == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    double t = red[lane_id()];
    t = butterfly_sum(t);
    __syncthreads();
    return t;
}

// integer flavours (order-free)
template <class F>
__device__ __forceinline__ i64 warp_int_sum(i64 b, i64 e, F term) {
    i64 acc = 0;
    for (i64 j = b + lane_id(); j < e; j += 32) acc += term(j);
    return warp_sum_i64(acc);
}

template <class V>
struct VSum;
template <>
struct VSum<i64> {
    template <class F>
    __device__ static i64 warp(i64 b, i64 e, F f) { return warp_int_sum(b, e, f); }
};
template <>
struct VSum<double> {
    template <class F>
    __device__ static double warp(i64 b, i64 e, F f) { return warp_canon_sum(b, e, f); }
};

__host__ __device__ __forceinline__ u32 next_pow2_u32(u32 x) {
    if (x <= 1) return 1;
    x--;
    x |= x >> 1;
    x |= x >> 2;
    x |= x >> 4;
    x |= x >> 8;
    x |= x >> 16;
    return x + 1;
}

__host__ __device__ __forceinline__ i64 ceil_div(i64 a, i64 b) { return (a + b - 1) / b; }

// ---------------------------------------------------------------------------
// device graph view
// ---------------------------------------------------------------------------
template <class W>
struct DGraph {
    using V = typename Traits<W>::V;
    i64 n = 0, nnz = 0;
    const i64* rowptr = nullptr;
    const i32* col = nullptr;
    const W* w = nullptr;  // nullptr: unit weights
    const V* vtx_w = nullptr;
    __device__ __forceinline__ W wgt(i64 j) const { return w ? w[j] : W(1); }
};

}  // namespace pggc
