// scan.cuh -- device-wide primitives used by every hot-path kernel family:
//   * scan_apply: exclusive int64 prefix over a functor input with a per-element
//     epilogue (prefix sums, order-preserving stream compaction, bucket offsets).
//     The element count may live in device memory so a launch sequence needs no
//     host round trip.
//   * det_scan / det_reduce: FP64 scan and reduction in the fixed association
//     (groups of 32, Kogge-Stone / xor butterfly, recursive over group totals).
//   * radix_sort_pairs: stable LSD radix sort of u64 keys with a payload
//     (8-bit digits, one warp per 512-element tile, __match_any_sync ranking).
#pragma once
#include "context.cuh"

namespace pggc {

// ---------------------------------------------------------------------------
// fills
// ---------------------------------------------------------------------------
template <class T>
__global__ void k_fill(T* a, i64 n, T v) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) a[i] = v;
}
template <class T>
inline void fill(Context& ctx, T* a, i64 n, T v) {
    if (n <= 0) return;
    int grid = (int)std::min<i64>(ceil_div(n, 256), (i64)ctx.num_sms * 16);
    k_fill<T><<<grid, 256, 0, ctx.stream>>>(a, n, v);
    PGGC_LAUNCH_CHECK();
}
template <class T>
__global__ void k_iota(T* a, i64 n) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) a[i] = (T)i;
}
template <class T>
inline void iota(Context& ctx, T* a, i64 n) {
    if (n <= 0) return;
    int grid = (int)std::min<i64>(ceil_div(n, 256), (i64)ctx.num_sms * 16);
    k_iota<T><<<grid, 256, 0, ctx.stream>>>(a, n);
    PGGC_LAUNCH_CHECK();
}
template <class T>
inline void copy_d2d(Context& ctx, T* dst, const T* src, i64 n) {
    if (n <= 0) return;
    PGGC_CUDA(cudaMemcpyAsync(dst, src, sizeof(T) * (size_t)n, cudaMemcpyDeviceToDevice, ctx.stream));
}

// ---------------------------------------------------------------------------
// block-level int64 exclusive scan of one value per thread
// ---------------------------------------------------------------------------
template <int THREADS>
__device__ __forceinline__ i64 block_excl_scan_i64(i64 v, i64* red /* THREADS/32 + 1 */, i64* total) {
    const int lane = lane_id(), wid = threadIdx.x >> 5;
    i64 x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        i64 t = __shfl_up_sync(FULL, x, d);
        if (lane >= d) x += t;
    }
    if (lane == 31) red[wid] = x;
    __syncthreads();
    if (wid == 0) {
        constexpr int NW = THREADS / 32;
        i64 y = lane < NW ? red[lane] : 0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            i64 t = __shfl_up_sync(FULL, y, d);
            if (lane >= d) y += t;
        }
        if (lane < NW) red[lane] = y;  // inclusive warp totals
    }
    __syncthreads();
    i64 wprefix = wid > 0 ? red[wid - 1] : 0;
    if (total) *total = red[THREADS / 32 - 1];
    __syncthreads();
    return wprefix + x - v;
}

constexpr int SCAN_THREADS = 512;
constexpr int SCAN_ITEMS = 8;
constexpr i64 SCAN_TILE = (i64)SCAN_THREADS * SCAN_ITEMS;

template <class In>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tile_sums(In in, const i64* d_k, i64 k_max, i64* partial) {
    __shared__ i64 red[SCAN_THREADS / 32 + 1];
    i64 k = d_k ? min(*d_k, k_max) : k_max;
    i64 base = (i64)blockIdx.x * SCAN_TILE;
    i64 s = 0;
#pragma unroll
    for (int it = 0; it < SCAN_ITEMS; it++) {
        i64 i = base + (i64)it * SCAN_THREADS + threadIdx.x;
        if (i < k) s += in(i);
    }
    i64 tot;
    block_excl_scan_i64<SCAN_THREADS>(s, red, &tot);
    if (threadIdx.x == 0) partial[blockIdx.x] = tot;
}

template <class In, class Epi>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tile_apply(In in, Epi epi, const i64* d_k, i64 k_max,
                                                                   const i64* tile_off) {
    __shared__ i64 red[SCAN_THREADS / 32 + 1];
    i64 k = d_k ? min(*d_k, k_max) : k_max;
    i64 base = (i64)blockIdx.x * SCAN_TILE + (i64)threadIdx.x * SCAN_ITEMS;
    i64 v[SCAN_ITEMS];
    i64 s = 0;
#pragma unroll
    for (int it = 0; it < SCAN_ITEMS; it++) {
        i64 i = base + it;
        v[it] = (i < k) ? in(i) : 0;
        s += v[it];
    }
    i64 off = block_excl_scan_i64<SCAN_THREADS>(s, red, nullptr) + tile_off[blockIdx.x];
#pragma unroll
    for (int it = 0; it < SCAN_ITEMS; it++) {
        i64 i = base + it;
        if (i < k) epi(i, off, v[it]);
        off += v[it];
    }
}

struct ArrIn {
    const i64* a;
    __device__ i64 operator()(i64 i) const { return a[i]; }
};
struct ArrOutExcl {
    i64* a;
    __device__ void operator()(i64 i, i64 excl, i64) const { a[i] = excl; }
};

// the whole scan in one block when it fits one tile: the tile apply with a
// zero tile offset that also writes the grand total (one launch instead of
// three and a memset, for the many short scans of small levels)
template <class In, class Epi>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_single(In in, Epi epi, const i64* d_k, i64 k_max,
                                                               i64* d_total) {
    __shared__ i64 red[SCAN_THREADS / 32 + 1];
    i64 k = d_k ? min(*d_k, k_max) : k_max;
    i64 base = (i64)threadIdx.x * SCAN_ITEMS;
    i64 v[SCAN_ITEMS];
    i64 s = 0;
#pragma unroll
    for (int it = 0; it < SCAN_ITEMS; it++) {
        i64 i = base + it;
        v[it] = (i < k) ? in(i) : 0;
        s += v[it];
    }
    i64 tot;
    i64 off = block_excl_scan_i64<SCAN_THREADS>(s, red, &tot);
#pragma unroll
    for (int it = 0; it < SCAN_ITEMS; it++) {
        i64 i = base + it;
        if (i < k) epi(i, off, v[it]);
        off += v[it];
    }
    if (d_total && threadIdx.x == 0) *d_total = tot;
}

static __global__ void k_scan_total(const i64* tile_off, const i64* partial, i64 nt, i64* d_total) {
    *d_total = tile_off[nt - 1] + partial[nt - 1];
}

// Exclusive scan of in(0..k-1) with epi(i, exclusive_prefix, value) applied to
// every element; the grand total goes to *d_total when non-null.  k is
// min(*d_k, k_max) when d_k is non-null (device-resident count).
template <class In, class Epi>
void scan_apply(Context& ctx, In in, Epi epi, i64 k_max, const i64* d_k, i64* d_total) {
    if (k_max <= 0) {
        if (d_total) PGGC_CUDA(cudaMemsetAsync(d_total, 0, sizeof(i64), ctx.stream));
        return;
    }
    i64 nt = ceil_div(k_max, SCAN_TILE);
    if (nt == 1) {
        k_scan_single<In, Epi><<<1, SCAN_THREADS, 0, ctx.stream>>>(in, epi, d_k, k_max, d_total);
        PGGC_LAUNCH_CHECK();
        return;
    }
    Tmp<i64> partial(ctx, nt), tile_off(ctx, nt);
    k_scan_tile_sums<In><<<(unsigned)nt, SCAN_THREADS, 0, ctx.stream>>>(in, d_k, k_max, partial.p);
    PGGC_LAUNCH_CHECK();
    scan_apply(ctx, ArrIn{partial.p}, ArrOutExcl{tile_off.p}, nt, nullptr, nullptr);
    k_scan_tile_apply<In, Epi><<<(unsigned)nt, SCAN_THREADS, 0, ctx.stream>>>(in, epi, d_k, k_max, tile_off.p);
    PGGC_LAUNCH_CHECK();
    if (d_total) {
        k_scan_total<<<1, 1, 0, ctx.stream>>>(tile_off.p, partial.p, nt, d_total);
        PGGC_LAUNCH_CHECK();
    }
}

// ---------------------------------------------------------------------------
// fixed-association FP64 scan / reduction
// ---------------------------------------------------------------------------
template <class In>
__global__ void k_det_scan_groups(In in, double* out, i64 k, double* totals) {
    i64 g = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    i64 ngroups = ceil_div(k, 32);
    if (g >= ngroups) return;
    int l = lane_id();
    i64 idx = g * 32 + l;
    double v = idx < k ? in(idx) : 0.0;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        double t = __shfl_up_sync(FULL, v, d);
        if (l >= d) v = v + t;
    }
    if (idx < k) out[idx] = v;
    if (l == 31) totals[g] = v;
}
static __global__ void k_det_scan_add(double* out, i64 k, const double* S) {
    i64 idx = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    if (idx >= k) return;
    i64 g = idx >> 5;
    if (g >= 1) out[idx] = S[g - 1] + out[idx];
}
struct DArrIn {
    const double* a;
    __device__ double operator()(i64 i) const { return a[i]; }
};

// Inclusive FP64 scan in the canonical association (host-known k).
template <class In>
void det_scan(Context& ctx, In in, double* out, i64 k) {
    if (k <= 0) return;
    i64 groups = ceil_div(k, 32);
    Tmp<double> tot(ctx, groups);
    k_det_scan_groups<In><<<(unsigned)ceil_div(groups * 32, 256), 256, 0, ctx.stream>>>(in, out, k, tot.p);
    PGGC_LAUNCH_CHECK();
    if (groups > 1) {
        Tmp<double> S(ctx, groups);
        det_scan(ctx, DArrIn{tot.p}, S.p, groups);
        k_det_scan_add<<<(unsigned)ceil_div(k, 256), 256, 0, ctx.stream>>>(out, k, S.p);
        PGGC_LAUNCH_CHECK();
    }
}

template <class In>
__global__ void __launch_bounds__(1024) k_det_reduce_level(In in, i64 k, double* out) {
    __shared__ double wt[32];
    i64 idx = (i64)blockIdx.x * 1024 + threadIdx.x;
    double v = idx < k ? in(idx) : 0.0;
    v = butterfly_sum(v);
    if (lane_id() == 0) wt[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = butterfly_sum(wt[threadIdx.x]);
        if (threadIdx.x == 0) out[blockIdx.x] = t;
    }
}

// Canonical FP64 reduction of in(0..k-1) into *d_out (device).
template <class In>
void det_reduce(Context& ctx, In in, i64 k, double* d_out) {
    if (k <= 0) {
        PGGC_CUDA(cudaMemsetAsync(d_out, 0, sizeof(double), ctx.stream));
        return;
    }
    i64 nb = ceil_div(k, 1024);
    if (nb == 1) {
        k_det_reduce_level<In><<<1, 1024, 0, ctx.stream>>>(in, k, d_out);
        PGGC_LAUNCH_CHECK();
        return;
    }
    Tmp<double> part(ctx, nb);
    k_det_reduce_level<In><<<(unsigned)nb, 1024, 0, ctx.stream>>>(in, k, part.p);
    PGGC_LAUNCH_CHECK();
    det_reduce(ctx, DArrIn{part.p}, nb, d_out);
}

// int64 reduction (order-free)
template <class In>
__global__ void k_sum_i64(In in, i64 k, unsigned long long* out) {
    i64 s = 0;
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < k; i += (i64)gridDim.x * blockDim.x) s += in(i);
    s = warp_sum_i64(s);
    if (lane_id() == 0 && s != 0) atomicAdd(out, (unsigned long long)s);
}
template <class In>
void sum_i64(Context& ctx, In in, i64 k, i64* d_out) {
    PGGC_CUDA(cudaMemsetAsync(d_out, 0, sizeof(i64), ctx.stream));
    if (k <= 0) return;
    int grid = (int)std::min<i64>(ceil_div(k, 256), (i64)ctx.num_sms * 8);
    k_sum_i64<In><<<grid, 256, 0, ctx.stream>>>(in, k, (unsigned long long*)d_out);
    PGGC_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// stable LSD radix sort: u64 keys + payload
// ---------------------------------------------------------------------------
constexpr int RS_WARPS = 8;
constexpr int RS_ITEMS = 16;
constexpr i64 RS_TILE = 32 * RS_ITEMS;

static __global__ void __launch_bounds__(RS_WARPS * 32) k_rs_hist(const u64* keys, i64 k, int shift, i64 ntiles, i64* hist) {
    __shared__ u32 cnt[RS_WARPS][256];
    int w = threadIdx.x >> 5, l = lane_id();
    i64 tile = (i64)blockIdx.x * RS_WARPS + w;
    for (int d = l; d < 256; d += 32) cnt[w][d] = 0;
    __syncwarp();
    if (tile < ntiles) {
        i64 base = tile * RS_TILE;
#pragma unroll 4
        for (int it = 0; it < RS_ITEMS; it++) {
            i64 i = base + it * 32 + l;
            if (i < k) atomicAdd(&cnt[w][(keys[i] >> shift) & 255], 1u);
        }
        __syncwarp();
        for (int d = l; d < 256; d += 32) hist[(i64)d * ntiles + tile] = cnt[w][d];
    }
}

template <class P>
__global__ void __launch_bounds__(RS_WARPS * 32) k_rs_scatter(const u64* keys, const P* vals, u64* keys_out,
                                                              P* vals_out, i64 k, int shift, i64 ntiles,
                                                              const i64* off) {
    __shared__ i64 o[RS_WARPS][256];
    int w = threadIdx.x >> 5, l = lane_id();
    i64 tile = (i64)blockIdx.x * RS_WARPS + w;
    if (tile >= ntiles) return;
    for (int d = l; d < 256; d += 32) o[w][d] = off[(i64)d * ntiles + tile];
    __syncwarp();
    i64 base = tile * RS_TILE;
    for (int it = 0; it < RS_ITEMS; it++) {
        i64 i = base + it * 32 + l;
        bool valid = i < k;
        u64 key = valid ? keys[i] : 0;
        int d = valid ? (int)((key >> shift) & 255) : 256 + l;
        unsigned peers = __match_any_sync(FULL, d);
        int rank = __popc(peers & lanemask_lt());
        i64 pos = valid ? o[w][d] + rank : 0;
        __syncwarp();
        if (valid && rank == 0) o[w][d] += __popc(peers);
        __syncwarp();
        if (valid) {
            keys_out[pos] = key;
            vals_out[pos] = vals[i];
        }
    }
}

// Sorts keys[0..k) (with payload vals) on bits [begin_bit, end_bit).  Uses the
// provided temporaries; the result is left in keys/vals.
template <class P>
void radix_sort_pairs(Context& ctx, u64* keys, P* vals, i64 k, int begin_bit, int end_bit, u64* keys_tmp,
                      P* vals_tmp) {
    if (k <= 1) return;
    i64 ntiles = ceil_div(k, RS_TILE);
    Tmp<i64> hist(ctx, 256 * ntiles);
    u64 *ka = keys, *kb = keys_tmp;
    P *va = vals, *vb = vals_tmp;
    unsigned grid = (unsigned)ceil_div(ntiles, RS_WARPS);
    int passes = 0;
    for (int shift = begin_bit; shift < end_bit; shift += 8) {
        k_rs_hist<<<grid, RS_WARPS * 32, 0, ctx.stream>>>(ka, k, shift, ntiles, hist.p);
        PGGC_LAUNCH_CHECK();
        scan_apply(ctx, ArrIn{hist.p}, ArrOutExcl{hist.p}, 256 * ntiles, nullptr, nullptr);
        k_rs_scatter<P><<<grid, RS_WARPS * 32, 0, ctx.stream>>>(ka, va, kb, vb, k, shift, ntiles, hist.p);
        PGGC_LAUNCH_CHECK();
        std::swap(ka, kb);
        std::swap(va, vb);
        passes++;
    }
    if (passes & 1) {
        copy_d2d(ctx, keys, ka, k);
        copy_d2d(ctx, vals, va, k);
    }
}

inline int bits_for(u64 maxval) {
    int b = 0;
    while (b < 64 && (maxval >> b) != 0) b++;
    return b;
}

}  // namespace pggc
