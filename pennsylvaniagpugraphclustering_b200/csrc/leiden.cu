// leiden.cu -- Leiden refinement, coarsen_leidenR<top,uniform>
// (src/leidenR.cpp:41-500), for sm_100a.
//
//  * well-connectedness test, then a per-vertex neighbour pick inside the
//    constraint cluster: first qualifying neighbour in cyclic order from a
//    hashed start (unit weights; warp ballots find the first hit) or the
//    weighted-random heaviest edge (max of |h/ORD_MAX| * val^4, ties to the
//    last edge);
//  * hashed vertex order, forest connected components by bounded pointer
//    chasing (find_trees), order flip for the unassigned vertices;
//  * gamma-connectivity: one stable LSD radix sort by (cluster, order, id)
//    replaces the counting sort + sort_crs_matrix; prefix sums give cluster
//    sizes and outward connectivity, two breakpoint passes and one break pass;
//  * contiguous relabelling by a prefix sum.
// The random picks use MurmurHash3_x86_32 (the hash behind Kokkos::pod_hash).
#include "kernels.cuh"

namespace pggc {

template <class W>
__global__ void k_well(DGraph<W> g, const i32* constraint, const typename Traits<W>::V* pv,
                       const typename Traits<W>::V* td, float gamma, unsigned char* well) {
    using V = typename Traits<W>::V;
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < g.n; i += (i64)gridDim.x * blockDim.x) {
        i32 c = constraint[i];
        V wd = g.vtx_w[i];
        well[i] = to_f(pv[i]) >= (gamma * to_f(wd)) * to_f(V(td[c] - wd)) ? 1 : 0;
    }
}

template <class W>
struct PickArgs {
    DGraph<W> g;
    const i32* constraint;
    const unsigned char* well;
    float gamma;
    u32 seed;
    i32* hn;
};

template <class W>
__device__ __forceinline__ bool pick_ok_uniform(const PickArgs<W>& a, i32 i, i32 v, float multi) {
    if (a.constraint[i] != a.constraint[v]) return false;
    if (!a.well[v]) return false;
    return 1.0f >= multi * to_f(a.g.vtx_w[v]);
}

// select random edge (src/leidenR.cpp:296-336), warp per vertex
template <class W>
__global__ void __launch_bounds__(256) k_pick_uniform_warp(PickArgs<W> a, const i32* list, i64 count) {
    const int l = lane_id();
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
    for (i64 x = gw; x < count; x += nw) {
        i32 i = list[x];
        i64 b = a.g.rowptr[i], e = a.g.rowptr[i + 1];
        i64 width = e - b;
        i32 jxs = (i32)murmur3_32(a.seed + (u32)i);
        if (jxs % 1000 == 0 || !a.well[i] || width == 0) {
            if (l == 0) a.hn[i] = i;
            continue;
        }
        i64 jx = b + (i64)((u32)jxs % (u32)width);
        float multi = a.gamma * to_f(a.g.vtx_w[i]);
        i32 pick = i;
        for (i64 off = 0; off < width; off += 32) {
            i64 s = off + l;
            bool q = false;
            i32 v = -1;
            if (s < width) {
                i64 j = jx + s;
                if (j >= e) j -= width;
                v = a.g.col[j];
                q = pick_ok_uniform(a, i, v, multi);
            }
            unsigned m = __ballot_sync(FULL, q);
            if (m) {
                pick = __shfl_sync(FULL, v, __ffs(m) - 1);
                break;
            }
        }
        if (l == 0) a.hn[i] = pick;
    }
}

// the 1024-thread variant for degree >= 15000 (src/leidenR.cpp:342-393)
template <class W>
__global__ void __launch_bounds__(1024) k_pick_uniform_block(PickArgs<W> a, const i32* list, i64 count) {
    __shared__ long long first;
    for (i64 x = blockIdx.x; x < count; x += gridDim.x) {
        i32 i = list[x];
        i64 b = a.g.rowptr[i], e = a.g.rowptr[i + 1];
        i64 width = e - b;
        i32 jxs = (i32)murmur3_32(a.seed + (u32)i);
        if (jxs % 1000 == 0 || !a.well[i] || width == 0) {
            if (threadIdx.x == 0) a.hn[i] = i;
            continue;
        }
        i64 jx = b + (i64)((u32)jxs % (u32)width);
        float multi = a.gamma * to_f(a.g.vtx_w[i]);
        if (threadIdx.x == 0) first = width;
        __syncthreads();
        for (i64 off = 0; off < width; off += 1024) {
            i64 s = off + threadIdx.x;
            if (s < width) {
                i64 j = jx + s;
                if (j >= e) j -= width;
                if (pick_ok_uniform(a, i, a.g.col[j], multi)) atomicMin(&first, (long long)s);
            }
            __syncthreads();
            if (first < width) break;
        }
        if (threadIdx.x == 0) {
            if (first < width) {
                i64 j = jx + first;
                if (j >= e) j -= width;
                a.hn[i] = a.g.col[j];
            } else {
                a.hn[i] = i;
            }
        }
        __syncthreads();
    }
}

// select heaviest edge (src/leidenR.cpp:400-474): max sample, ties -> last edge
__device__ __forceinline__ bool sample_better(float s, i64 j, float bs, i64 bj) {
    return s > bs || (s == bs && j > bj);
}

template <class W>
__device__ __forceinline__ void heavy_eval(const PickArgs<W>& a, i32 i, i64 j, float multi, float& bs, i64& bj) {
    i32 v = a.g.col[j];
    if (a.constraint[i] != a.constraint[v]) return;
    if (!a.well[v]) return;
    float val = (float)a.g.wgt(j) - multi * to_f(a.g.vtx_w[v]);
    if (val >= 0.0f) {
        float sample = fabsf((float)murmur3_32(a.seed + (u32)(u64)j) / (float)ORD_MAX);
        float v2 = val * val;
        sample = sample * (v2 * v2);
        if (sample >= 0.0f && sample_better(sample, j, bs, bj)) {
            bs = sample;
            bj = j;
        }
    }
}

template <class W>
__global__ void __launch_bounds__(256) k_pick_heavy_warp(PickArgs<W> a, const i32* list, i64 count) {
    const int l = lane_id();
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
    for (i64 x = gw; x < count; x += nw) {
        i32 i = list[x];
        i64 b = a.g.rowptr[i], e = a.g.rowptr[i + 1];
        u32 h = murmur3_32(a.seed + (u32)i);
        if (h % 10000u == 0 || !a.well[i]) {
            if (l == 0) a.hn[i] = i;
            continue;
        }
        float multi = a.gamma * to_f(a.g.vtx_w[i]);
        float bs = -1.0f;
        i64 bj = -1;
        for (i64 j = b + l; j < e; j += 32) heavy_eval(a, i, j, multi, bs, bj);
        for (int d = 16; d >= 1; d >>= 1) {
            float os = __shfl_xor_sync(FULL, bs, d);
            i64 oj = __shfl_xor_sync(FULL, bj, d);
            if (sample_better(os, oj, bs, bj)) {
                bs = os;
                bj = oj;
            }
        }
        if (l == 0) a.hn[i] = bj >= b ? a.g.col[bj] : i;
    }
}

// One thread per vertex of low degree (the degree classes up to 32): per
// chunk of 8 edges the columns, constraints and well flags are gathered
// together, then the edges are evaluated in order; the argmax order (sample,
// then edge index) is total, so this equals the warp kernel's pick.
template <class W>
__global__ void __launch_bounds__(256, 3) k_pick_heavy_thr(PickArgs<W> a, Range rg) {
    const i64 lo = rg.begin(), hi = rg.end();
    for (i64 x = lo + blockIdx.x * (i64)blockDim.x + threadIdx.x; x < hi; x += (i64)gridDim.x * blockDim.x) {
        const i32 i = rg.list[x];
        const u32 h = murmur3_32(a.seed + (u32)i);
        if (h % 10000u == 0 || !a.well[i]) {
            a.hn[i] = i;
            continue;
        }
        const i64 b = a.g.rowptr[i], e = a.g.rowptr[i + 1];
        const float multi = a.gamma * to_f(a.g.vtx_w[i]);
        const i32 ci = a.constraint[i];
        float bs = -1.0f;
        i64 bj = -1;
        // edges in chunks of 8, in order
#pragma unroll 1
        for (i64 c0 = b; c0 < e; c0 += 8) {
            i32 cv[8];
#pragma unroll
            for (int t = 0; t < 8; t++) cv[t] = c0 + t < e ? a.g.col[c0 + t] : -1;
            bool ok[8];
#pragma unroll
            for (int t = 0; t < 8; t++) ok[t] = cv[t] >= 0 && a.constraint[cv[t]] == ci;
#pragma unroll
            for (int t = 0; t < 8; t++) ok[t] = ok[t] && a.well[cv[t]];
#pragma unroll
            for (int t = 0; t < 8; t++) {
                if (!ok[t]) continue;
                const i64 j = c0 + t;
                const float val = (float)a.g.wgt(j) - multi * to_f(a.g.vtx_w[cv[t]]);
                if (val >= 0.0f) {
                    float sample = fabsf((float)murmur3_32(a.seed + (u32)(u64)j) / (float)ORD_MAX);
                    const float v2 = val * val;
                    sample = sample * (v2 * v2);
                    if (sample >= 0.0f && sample_better(sample, j, bs, bj)) {
                        bs = sample;
                        bj = j;
                    }
                }
            }
        }
        a.hn[i] = bj >= b ? a.g.col[bj] : i;
    }
}

// G-lane groups for low-degree vertices (NG = 32 / G vertices per warp); the
// argmax order (sample, then edge index) is total, so any split of the edges
// over lanes gives the warp kernel's pick
template <class W, int G>
__global__ void __launch_bounds__(256) k_pick_heavy_grp(PickArgs<W> a, Range rg) {
    constexpr int NG = 32 / G;
    const int l = lane_id(), r = l & (G - 1), grp = l / G;
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
    const i64 lo = rg.begin(), count = rg.end();
    for (i64 base = lo + gw * NG; base < count; base += nw * NG) {
        const i64 x = base + grp;
        i32 i = -1;
        bool act = false;
        i64 b = 0, e = 0;
        float multi = 0.f;
        if (x < count) {
            i = rg.list[x];
            const u32 h = murmur3_32(a.seed + (u32)i);
            if (h % 10000u == 0 || !a.well[i]) {
                if (r == 0) a.hn[i] = i;
            } else {
                act = true;
                b = a.g.rowptr[i];
                e = a.g.rowptr[i + 1];
                multi = a.gamma * to_f(a.g.vtx_w[i]);
            }
        }
        float bs = -1.0f;
        i64 bj = -1;
        if (act)
            for (i64 j = b + r; j < e; j += G) heavy_eval(a, i, j, multi, bs, bj);
#pragma unroll
        for (int d = G / 2; d >= 1; d >>= 1) {
            float os = __shfl_xor_sync(FULL, bs, d);
            i64 oj = __shfl_xor_sync(FULL, bj, d);
            if (sample_better(os, oj, bs, bj)) {
                bs = os;
                bj = oj;
            }
        }
        if (r == 0 && act) a.hn[i] = bj >= b ? a.g.col[bj] : i;
    }
}

template <class W>
__global__ void __launch_bounds__(1024) k_pick_heavy_block(PickArgs<W> a, const i32* list, i64 count) {
    __shared__ float ws[32];
    __shared__ i64 wj[32];
    for (i64 x = blockIdx.x; x < count; x += gridDim.x) {
        i32 i = list[x];
        i64 b = a.g.rowptr[i], e = a.g.rowptr[i + 1];
        u32 h = murmur3_32(a.seed + (u32)i);
        if (h % 10000u == 0 || !a.well[i]) {
            if (threadIdx.x == 0) a.hn[i] = i;
            continue;
        }
        float multi = a.gamma * to_f(a.g.vtx_w[i]);
        float bs = -1.0f;
        i64 bj = -1;
        for (i64 j = b + threadIdx.x; j < e; j += 1024) heavy_eval(a, i, j, multi, bs, bj);
        for (int d = 16; d >= 1; d >>= 1) {
            float os = __shfl_xor_sync(FULL, bs, d);
            i64 oj = __shfl_xor_sync(FULL, bj, d);
            if (sample_better(os, oj, bs, bj)) {
                bs = os;
                bj = oj;
            }
        }
        if (lane_id() == 0) {
            ws[threadIdx.x >> 5] = bs;
            wj[threadIdx.x >> 5] = bj;
        }
        __syncthreads();
        if (threadIdx.x < 32) {
            bs = ws[threadIdx.x];
            bj = wj[threadIdx.x];
            for (int d = 16; d >= 1; d >>= 1) {
                float os = __shfl_xor_sync(FULL, bs, d);
                i64 oj = __shfl_xor_sync(FULL, bj, d);
                if (sample_better(os, oj, bs, bj)) {
                    bs = os;
                    bj = oj;
                }
            }
            if (threadIdx.x == 0) a.hn[i] = bj >= b ? a.g.col[bj] : i;
        }
        __syncthreads();
    }
}

// set order + unselect equal order edges (src/leidenR.cpp:482-494)
__global__ void k_set_order(i64 n, u32 seed, i32* order) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
        i32 o = (i32)murmur3_32((u32)i + seed);
        order[i] = abs(o % SPLIT);
    }
}
__global__ void k_unselect(i64 n, const i32* order, i32* hn) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
        i32 h = hn[i];
        if (order[i] == order[h]) hn[i] = (i32)i;
    }
}

// find_trees (src/leidenR.cpp:213-260); pointer chasing bounded by n steps
__global__ void k_trees_part1(i64 n, const i32* hn, const i32* order, i32* vcmap, int* err) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
        i32 now = (i32)i, then = hn[i];
        if (now == then) {
            vcmap[i] = (i32)i;
            continue;
        }
        i64 steps = 0;
        while (order[now] > order[then]) {
            now = then;
            then = hn[then];
            if (++steps > n) {
                atomicExch(err, (int)DEV_ERR_CHASE);
                break;
            }
        }
        if (now != (i32)i) {
            vcmap[i] = now;
            vcmap[now] = now;
        }
    }
}
__global__ void k_trees_flip(i64 n, const i32* vcmap, i32* order) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
        if (vcmap[i] == ORD_MAX) order[i] = 2 * SPLIT - order[i];
}
__global__ void k_trees_part2(i64 n, const i32* hn, const i32* order, i32* vcmap, int* err) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
        volatile i32* vc = vcmap;
        if (vc[i] != ORD_MAX) continue;
        i32 now = (i32)i, then = hn[i];
        i64 steps = 0;
        while (vc[now] == ORD_MAX && order[now] > order[then]) {
            now = then;
            then = hn[then];
            if (++steps > n) {
                atomicExch(err, (int)DEV_ERR_CHASE);
                break;
            }
        }
        vc[i] = vc[now];
    }
}

// ---- ensure_gamma_connectivity (src/leidenR.cpp:41-187) --------------------
__global__ void k_sort_keys(i64 n, const i32* vcmap, const i32* order, u64* keys, i32* ids) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
        keys[i] = ((u64)(u32)vcmap[i] << 31) | (u64)(u32)order[i];
        ids[i] = (i32)i;
    }
}
__global__ void k_hist(i64 n, const i32* lab, i64* cnt) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
        ::atomicAdd((unsigned long long*)&cnt[lab[i]], 1ull);
}

// The vertices grouped by tree and ordered by (order, id) inside each tree --
// the order of a stable sort on (tree, order) -- by a counting sort on the
// tree id (row_map: tree offsets) followed by per-tree sorts of the 64-bit
// keys (order << 32 | id): a thread per tree up to SEG_SMALL members (an
// odd-even transposition network in registers), a block per larger tree
// (bitonic network in shared memory, up to SEG_BIG members); trees above that
// fall back to a radix sort of all vertices.
constexpr int SEG_SMALL = 16;
constexpr int SEG_MID = 1024;
constexpr int SEG_BIG = 16384;

__global__ void k_seg_scatter(i64 n, const i32* vcmap, i64* cursor, i32* ids) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
        const i64 pos = (i64)::atomicAdd((unsigned long long*)&cursor[vcmap[i]], 1ull);
        ids[pos] = (i32)i;
    }
}

__device__ __forceinline__ u64 seg_key(const i32* order, i32 id) {
    return ((u64)(u32)order[id] << 32) | (u64)(u32)id;
}

// sorts the sz <= N ids of one tree by (order, id): an odd-even transposition
// network of N rounds over keys held in registers (padding ~0 sorts last)
template <int N>
__device__ __forceinline__ void seg_sort_net(const i32* order, i32* seg, int sz) {
    u64 k[N];
#pragma unroll
    for (int t = 0; t < N; t++) k[t] = t < sz ? seg_key(order, seg[t]) : ~0ull;
#pragma unroll
    for (int rd = 0; rd < N; rd++) {
#pragma unroll
        for (int t = rd & 1; t + 1 < N; t += 2) {
            const u64 lo = k[t] < k[t + 1] ? k[t] : k[t + 1];
            const u64 hi = k[t] < k[t + 1] ? k[t + 1] : k[t];
            k[t] = lo;
            k[t + 1] = hi;
        }
    }
#pragma unroll
    for (int t = 0; t < N; t++)
        if (t < sz) seg[t] = (i32)(u32)k[t];
}

// trees of 2..SEG_SMALL members sorted in registers; larger ones listed
// (big[0]: count of trees of up to SEG_MID members, big[1]: up to SEG_BIG,
// big[2]: above; the lists grow from the two ends of `lst`)
__global__ void k_seg_sort_small(i64 n, const i64* row_map, const i32* order, i32* ids, i32* lst,
                                 unsigned long long* big) {
    for (i64 r = blockIdx.x * (i64)blockDim.x + threadIdx.x; r < n; r += (i64)gridDim.x * blockDim.x) {
        const i64 b = row_map[r], sz = row_map[r + 1] - b;
        if (sz <= 1) continue;
        if (sz > SEG_SMALL) {
            if (sz <= SEG_MID) lst[::atomicAdd(&big[0], 1ull)] = (i32)r;
            else if (sz <= SEG_BIG) lst[n - 1 - (i64)::atomicAdd(&big[1], 1ull)] = (i32)r;
            else ::atomicAdd(&big[2], 1ull);
            continue;
        }
        if (sz <= 4) seg_sort_net<4>(order, ids + b, (int)sz);
        else if (sz <= 8) seg_sort_net<8>(order, ids + b, (int)sz);
        else seg_sort_net<SEG_SMALL>(order, ids + b, (int)sz);
    }
}

// a block per listed tree: keys in shared memory, bitonic network over
// next_pow2(size) slots padded with ~0
template <int THREADS>
__global__ void __launch_bounds__(THREADS) k_seg_sort_block(const i32* lst, i64 count, const i64* row_map,
                                                            const i32* order, i32* ids) {
    extern __shared__ __align__(16) u64 sk[];
    for (i64 x = blockIdx.x; x < count; x += gridDim.x) {
        const i32 r = lst[x];
        const i64 b = row_map[r];
        const u32 sz = (u32)(row_map[r + 1] - b);
        const u32 T = next_pow2_u32(sz);
        for (u32 s = threadIdx.x; s < T; s += THREADS) sk[s] = s < sz ? seg_key(order, ids[b + s]) : ~0ull;
        __syncthreads();
        for (u32 k = 2; k <= T; k <<= 1) {
            for (u32 j = k >> 1; j > 0; j >>= 1) {
                for (u32 t = threadIdx.x; t < T; t += THREADS) {
                    const u32 q = t ^ j;
                    if (q > t) {
                        const bool up = (t & k) == 0;
                        const u64 a0 = sk[t], a1 = sk[q];
                        if ((a0 > a1) == up) {
                            sk[t] = a1;
                            sk[q] = a0;
                        }
                    }
                }
                __syncthreads();
            }
        }
        for (u32 s = threadIdx.x; s < sz; s += THREADS) ids[b + s] = (i32)(u32)sk[s];
        __syncthreads();
    }
}

template <class V>
struct TsIn;
template <>
struct TsIn<i64> {
    const i32* ids;
    const i64* vw;
    i64 n;
    __device__ i64 operator()(i64 x) const { return x < n ? vw[ids[x]] : 0; }
};
template <>
struct TsIn<double> {
    const i32* ids;
    const double* vw;
    i64 n;
    __device__ double operator()(i64 x) const { return vw[ids[x]]; }
};

template <class W>
__device__ __forceinline__ typename Traits<W>::V inner_term(const DGraph<W>& g, const i32* vcmap, const i32* order,
                                                            i32 i, i64 j) {
    using V = typename Traits<W>::V;
    i32 v = g.col[j];
    return (vcmap[i] == vcmap[v] && order[v] < order[i]) ? V(g.wgt(j)) : V(0);
}

// Vertices of degree <= 2H (H = 8: degree classes 0 and 1, H = 16: class 2),
// one thread each: the 32-lane canonical association of the row's terms
// (canon_tree), no shuffles; the order of the neighbour is read only when
// its tree matches.
template <class W, int H>
__global__ void __launch_bounds__(256) k_inner_thr(DGraph<W> g, Range rg, const i32* vcmap, const i32* order,
                                                   typename Traits<W>::V* inner) {
    using V = typename Traits<W>::V;
    const i64 lo = rg.begin(), hi = rg.end();
    for (i64 x = lo + blockIdx.x * (i64)blockDim.x + threadIdx.x; x < hi; x += (i64)gridDim.x * blockDim.x) {
        const i32 i = rg.list[x];
        const i64 b = g.rowptr[i], e = g.rowptr[i + 1];
        const i32 ci = vcmap[i], oi = order[i];
        i32 cv[2 * H];
#pragma unroll
        for (int t = 0; t < 2 * H; t++) cv[t] = b + t < e ? g.col[b + t] : -1;
        bool in[2 * H];
#pragma unroll
        for (int t = 0; t < 2 * H; t++) in[t] = cv[t] >= 0 && vcmap[cv[t]] == ci;
#pragma unroll
        for (int t = 0; t < 2 * H; t++) in[t] = in[t] && order[cv[t]] < oi;
        V acc[H];
#pragma unroll
        for (int r = 0; r < H; r++) {
            acc[r] = V(0);
            if (b + r < e) acc[r] += in[r] ? V(g.wgt(b + r)) : V(0);
            if (b + r + H < e) acc[r] += in[r + H] ? V(g.wgt(b + r + H)) : V(0);
        }
        inner[i] = canon_tree<H, V>(acc);
    }
}

// warp per vertex (degree below MASSIVE_CUTOFF): the canonical warp sum
template <class W>
__global__ void __launch_bounds__(256) k_inner_warp(DGraph<W> g, Range rg, const i32* vcmap, const i32* order,
                                                    typename Traits<W>::V* inner) {
    using V = typename Traits<W>::V;
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
    const i64 lo = rg.begin(), hi = rg.end();
    for (i64 x = lo + gw; x < hi; x += nw) {
        i32 i = rg.list[x];
        V r = VSum<V>::warp(g.rowptr[i], g.rowptr[i + 1], [&](i64 j) { return inner_term(g, vcmap, order, i, j); });
        if (lane_id() == 0) inner[i] = r;
    }
}

template <class W>
__global__ void __launch_bounds__(1024) k_inner_block(DGraph<W> g, const i32* list, i64 count, const i32* vcmap,
                                                      const i32* order, typename Traits<W>::V* inner) {
    using V = typename Traits<W>::V;
    __shared__ double red[32];
    __shared__ unsigned long long acc;
    for (i64 x = blockIdx.x; x < count; x += gridDim.x) {
        i32 i = list[x];
        i64 b = g.rowptr[i], e = g.rowptr[i + 1];
        V r;
        if constexpr (std::is_same<V, double>::value) {
            r = block1024_canon_sum(b, e, [&](i64 j) { return inner_term(g, vcmap, order, i, j); }, red);
        } else {
            if (threadIdx.x == 0) acc = 0;
            __syncthreads();
            i64 s = 0;
            for (i64 j = b + threadIdx.x; j < e; j += 1024) s += inner_term(g, vcmap, order, i, j);
            s = warp_sum_i64(s);
            if (lane_id() == 0) ::atomicAdd(&acc, (unsigned long long)s);
            __syncthreads();
            r = (i64)acc;
        }
        if (threadIdx.x == 0) inner[i] = r;
        __syncthreads();
    }
}

template <class W>
struct GammaArgs {
    using V = typename Traits<W>::V;
    i64 n;
    const i32* ids;
    const i32* vcmap;
    const i64* row_map;
    const V* ts;
    const V* inner;
    const V* oc;
    const V* vw;
    const V* td;
    const i32* constraint;
    float gamma;
    long long* breakers;
};

template <class W>
__global__ void k_break_part1(GammaArgs<W> a) {
    using V = typename Traits<W>::V;
    for (i64 x = blockIdx.x * (i64)blockDim.x + threadIdx.x; x < a.n; x += (i64)gridDim.x * blockDim.x) {
        i32 i = a.ids[x];
        i32 c = a.vcmap[i];
        i64 cb = a.row_map[c];
        V prev = a.ts[x] - a.ts[cb];
        if (to_f(a.inner[i]) < (a.gamma * to_f(a.vw[i])) * to_f(prev)) atomicMin(&a.breakers[c], (long long)x);
    }
}
template <class W>
__global__ void k_break_part2(GammaArgs<W> a) {
    using V = typename Traits<W>::V;
    for (i64 x = blockIdx.x * (i64)blockDim.x + threadIdx.x; x < a.n; x += (i64)gridDim.x * blockDim.x) {
        i32 i = a.ids[x];
        i32 c = a.vcmap[i];
        i64 cb = a.row_map[c];
        V curr_size = (a.ts[x] + a.vw[i]) - a.ts[cb];
        V other = a.td[a.constraint[i]] - curr_size;
        V outer = a.oc[i];
        if (cb > 0) outer = outer - a.oc[a.ids[cb - 1]];
        if (to_f(outer) < (a.gamma * to_f(curr_size)) * to_f(other)) atomicMin(&a.breakers[c], (long long)(x + 1));
    }
}
__global__ void k_break_apply(i64 n, const i32* ids, const long long* breakers, i32* vcmap) {
    for (i64 x = blockIdx.x * (i64)blockDim.x + threadIdx.x; x < n; x += (i64)gridDim.x * blockDim.x) {
        i32 i = ids[x];
        i32 c = vcmap[i];
        if (x >= breakers[c]) vcmap[i] = i;
    }
}

template <class V>
struct OcInI {
    const i32* ids;
    const V* pv;
    const V* inner;
    __device__ i64 operator()(i64 x) const {
        i32 i = ids[x];
        return pv[i] - 2 * inner[i];
    }
};
struct OcEpiI {
    const i32* ids;
    i64* oc;
    __device__ void operator()(i64 x, i64 excl, i64 v) const { oc[ids[x]] = excl + v; }
};
struct OcInD {
    const i32* ids;
    const double* pv;
    const double* inner;
    __device__ double operator()(i64 x) const {
        i32 i = ids[x];
        return pv[i] - 2.0 * inner[i];
    }
};
__global__ void k_scatter_by_ids(i64 n, const i32* ids, const double* in, double* out) {
    for (i64 x = blockIdx.x * (i64)blockDim.x + threadIdx.x; x < n; x += (i64)gridDim.x * blockDim.x) out[ids[x]] = in[x];
}
__global__ void k_shift_excl(i64 n, const double* inc, double* ts) {
    for (i64 x = blockIdx.x * (i64)blockDim.x + threadIdx.x; x < n; x += (i64)gridDim.x * blockDim.x)
        ts[x] = x == 0 ? 0.0 : inc[x - 1];
}

// contigitize_clusters (src/leidenR.cpp:190-210)
struct RootFlag {
    const i32* vcmap;
    __device__ i64 operator()(i64 u) const { return vcmap[u] == (i32)u ? 1 : 0; }
};
struct RootEpi {
    i32* newid;
    __device__ void operator()(i64 u, i64 excl, i64 v) const {
        if (v) newid[u] = (i32)excl;
    }
};
__global__ void k_contig_apply(i64 n, const i32* vcmap, const i32* newid, i32* out) {
    for (i64 u = blockIdx.x * (i64)blockDim.x + threadIdx.x; u < n; u += (i64)gridDim.x * blockDim.x)
        out[u] = newid[vcmap[u]];
}

// Refinement temporaries live in grow-only workspace slots of the context
// (sized by the largest level and reused), so the level loop does not go
// through the allocator for them.
enum RefineSlot : int {
    RS_PV = 90, RS_WELL, RS_HN, RS_ORDER, RS_VCMAP, RS_KEYS, RS_KEYS2, RS_IDS, RS_IDS2, RS_CNT, RS_ROWMAP, RS_TS,
    RS_INNER, RS_OC, RS_INC, RS_BREAK, RS_NEWID, RS_TOT, RS_SEGBIG
};
template <class T>
struct RBuf {
    T* p;
    RBuf(Context& c, int slot, i64 count) : p(c.ws_get<T>(slot, std::max<i64>(count, 1))) {}
};

template <class W>
i64 coarsen_leidenR(Context& ctx, const Graph<W>& g, const Ordering& ord, const i32* constraint,
                    const ClusterState<typename Traits<W>::V>& cs, u32 seed_pick, u32 seed_order, i32* vcmap_out,
                    bool reuse_pvals) {
    using V = typename Traits<W>::V;
    const i64 n = g.n;
    if (n == 0) return 0;
    ProfScope ps(ctx, "leiden_refine");
    auto gv = g.view();
    const float gamma = (float)cs.lambda;
    const int grid = (int)std::min<i64>(ceil_div(n, 256), (i64)ctx.num_sms * 16);
    const i64 nsmall = ord.off_large2, nmass = n - ord.off_large2;
    const i32* small_list = ord.order1.p;
    const i32* mass_list = ord.order1.p + ord.off_large2;
    const int gw = (int)std::min<i64>(ceil_div(std::max<i64>(nsmall, 1), 8), (i64)ctx.num_sms * 16);
    const int gb = (int)std::min<i64>(std::max<i64>(nmass, 1), (i64)ctx.num_sms * 2);

    RBuf<V> pv(ctx, RS_PV, n);
    // constraint = the last local move's output on g: its own-cluster weights
    // are the context's retained ones
    if (reuse_pvals && ctx.pv_uid == g.uid && ctx.pv_n == n) copy_d2d(ctx, pv.p, (const V*)ctx.pv_ptr, n);
    else own_weights<W>(ctx, g, ord, constraint, pv.p);
    RBuf<unsigned char> well(ctx, RS_WELL, n);
    k_well<W><<<grid, 256, 0, ctx.stream>>>(gv, constraint, pv.p, cs.total_deg.p, gamma, well.p);
    PGGC_LAUNCH_CHECK();
    RBuf<i32> hn(ctx, RS_HN, n), order(ctx, RS_ORDER, n), vcmap(ctx, RS_VCMAP, n);
    PickArgs<W> pa{gv, constraint, well.p, gamma, seed_pick, hn.p};
    if (g.uniform) {
        if (nsmall > 0) {
            k_pick_uniform_warp<W><<<gw, 256, 0, ctx.stream>>>(pa, small_list, nsmall);
            PGGC_LAUNCH_CHECK();
        }
        if (nmass > 0) {
            k_pick_uniform_block<W><<<gb, 1024, 0, ctx.stream>>>(pa, mass_list, nmass);
            PGGC_LAUNCH_CHECK();
        }
    } else {
        // degree <= 32 (classes 0-2 of the graph's class lists): a thread per
        // vertex; 32 < degree < 128 (class 3): 8-lane groups; 128 <= degree <
        // 15000: a warp per vertex
        if (ord.off_large > 0) {
            const ClassLists cls = graph_class_lists<W>(ctx, g, ord);
            const int gt = (int)std::min<i64>(ceil_div(ord.off_large, 256), (i64)ctx.num_sms * 16);
            k_pick_heavy_thr<W><<<gt, 256, 0, ctx.stream>>>(pa, dev_range(cls.list, cls.off + 0, cls.off + 3));
            PGGC_LAUNCH_CHECK();
            const int g8 = (int)std::min<i64>(ceil_div(ord.off_large, 32), (i64)ctx.num_sms * 16);
            k_pick_heavy_grp<W, 8><<<g8, 256, 0, ctx.stream>>>(pa, dev_range(cls.list, cls.off + 3, cls.off + 4));
            PGGC_LAUNCH_CHECK();
        }
        if (nsmall > ord.off_large) {
            k_pick_heavy_warp<W><<<gw, 256, 0, ctx.stream>>>(pa, small_list + ord.off_large, nsmall - ord.off_large);
            PGGC_LAUNCH_CHECK();
        }
        if (nmass > 0) {
            k_pick_heavy_block<W><<<gb, 1024, 0, ctx.stream>>>(pa, mass_list, nmass);
            PGGC_LAUNCH_CHECK();
        }
    }
    k_set_order<<<grid, 256, 0, ctx.stream>>>(n, seed_order, order.p);
    PGGC_LAUNCH_CHECK();
    k_unselect<<<grid, 256, 0, ctx.stream>>>(n, order.p, hn.p);
    PGGC_LAUNCH_CHECK();
    fill<i32>(ctx, vcmap.p, n, ORD_MAX);
    k_trees_part1<<<grid, 256, 0, ctx.stream>>>(n, hn.p, order.p, vcmap.p, ctx.d_err);
    PGGC_LAUNCH_CHECK();
    k_trees_flip<<<grid, 256, 0, ctx.stream>>>(n, vcmap.p, order.p);
    PGGC_LAUNCH_CHECK();
    k_trees_part2<<<grid, 256, 0, ctx.stream>>>(n, hn.p, order.p, vcmap.p, ctx.d_err);
    PGGC_LAUNCH_CHECK();

    // --- gamma connectivity
    // tree offsets, then the vertices grouped by tree in (order, id) order
    RBuf<i64> cnt(ctx, RS_CNT, n + 1), row_map(ctx, RS_ROWMAP, n + 1);
    PGGC_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(i64) * (n + 1), ctx.stream));
    k_hist<<<grid, 256, 0, ctx.stream>>>(n, vcmap.p, cnt.p);
    PGGC_LAUNCH_CHECK();
    scan_apply(ctx, ArrIn{cnt.p}, ArrOutExcl{row_map.p}, n + 1, nullptr, nullptr);
    RBuf<i32> ids(ctx, RS_IDS, n), lst(ctx, RS_IDS2, n);
    {
        copy_d2d(ctx, cnt.p, row_map.p, n + 1);  // scatter cursors
        k_seg_scatter<<<grid, 256, 0, ctx.stream>>>(n, vcmap.p, cnt.p, ids.p);
        PGGC_LAUNCH_CHECK();
        RBuf<unsigned long long> big(ctx, RS_SEGBIG, 4);
        PGGC_CUDA(cudaMemsetAsync(big.p, 0, sizeof(unsigned long long) * 4, ctx.stream));
        k_seg_sort_small<<<grid, 256, 0, ctx.stream>>>(n, row_map.p, order.p, ids.p, lst.p, big.p);
        PGGC_LAUNCH_CHECK();
        const unsigned long long* hb = (const unsigned long long*)ctx.readback(big.p, 3 * sizeof(unsigned long long));
        const i64 n_mid = (i64)hb[0], n_big = (i64)hb[1], n_huge = (i64)hb[2];
        if (n_huge > 0) {
            // a tree above SEG_BIG members: the radix sort of every vertex on (tree, order)
            RBuf<u64> keys(ctx, RS_KEYS, n), keys2(ctx, RS_KEYS2, n);
            k_sort_keys<<<grid, 256, 0, ctx.stream>>>(n, vcmap.p, order.p, keys.p, ids.p);
            PGGC_LAUNCH_CHECK();
            radix_sort_pairs<i32>(ctx, keys.p, ids.p, n, 0, 31 + bits_for((u64)(n - 1)), keys2.p, lst.p);
        } else {
            if (n_mid > 0) {
                const int gm = (int)std::min<i64>(n_mid, (i64)ctx.num_sms * 8);
                k_seg_sort_block<256><<<gm, 256, sizeof(u64) * SEG_MID, ctx.stream>>>(lst.p, n_mid, row_map.p,
                                                                                     order.p, ids.p);
                PGGC_LAUNCH_CHECK();
            }
            if (n_big > 0) {
                set_dynamic_smem_once(k_seg_sort_block<1024>, (int)(sizeof(u64) * SEG_BIG), ctx.device);
                const int gb2 = (int)std::min<i64>(n_big, (i64)ctx.num_sms);
                k_seg_sort_block<1024><<<gb2, 1024, sizeof(u64) * SEG_BIG, ctx.stream>>>(lst.p + (n - n_big), n_big,
                                                                                         row_map.p, order.p, ids.p);
                PGGC_LAUNCH_CHECK();
            }
        }
    }
    RBuf<V> ts(ctx, RS_TS, n), inner(ctx, RS_INNER, n), oc(ctx, RS_OC, n);
    if constexpr (std::is_same<V, i64>::value) {
        scan_apply(ctx, TsIn<i64>{ids.p, g.vtx_w.p, n}, ArrOutExcl{ts.p}, n, nullptr, nullptr);
    } else {
        RBuf<double> inc(ctx, RS_INC, n);
        det_scan(ctx, TsIn<double>{ids.p, g.vtx_w.p, n}, inc.p, n);
        k_shift_excl<<<grid, 256, 0, ctx.stream>>>(n, inc.p, ts.p);
        PGGC_LAUNCH_CHECK();
    }
    if (nsmall > 0) {
        // degree <= 32 (classes 0-2 of the graph's class lists): a thread per
        // vertex; 32 < degree < 128 (class 3) and up to MASSIVE_CUTOFF: a warp
        const ClassLists cls = graph_class_lists<W>(ctx, g, ord);
        const int gt = (int)std::min<i64>(ceil_div(std::max<i64>(nsmall, 1), 256), (i64)ctx.num_sms * 16);
        k_inner_thr<W, 8><<<gt, 256, 0, ctx.stream>>>(gv, dev_range(cls.list, cls.off + 0, cls.off + 2), vcmap.p,
                                                      order.p, inner.p);
        PGGC_LAUNCH_CHECK();
        k_inner_thr<W, 16><<<gt, 256, 0, ctx.stream>>>(gv, dev_range(cls.list, cls.off + 2, cls.off + 3), vcmap.p,
                                                       order.p, inner.p);
        PGGC_LAUNCH_CHECK();
        k_inner_warp<W><<<gw, 256, 0, ctx.stream>>>(gv, dev_range(cls.list, cls.off + 3, cls.off + 4), vcmap.p,
                                                    order.p, inner.p);
        PGGC_LAUNCH_CHECK();
        if (nsmall > ord.off_large) {
            k_inner_warp<W><<<gw, 256, 0, ctx.stream>>>(gv, host_range(small_list, ord.off_large, nsmall), vcmap.p,
                                                        order.p, inner.p);
            PGGC_LAUNCH_CHECK();
        }
    }
    if (nmass > 0) {
        k_inner_block<W><<<gb, 1024, 0, ctx.stream>>>(gv, mass_list, nmass, vcmap.p, order.p, inner.p);
        PGGC_LAUNCH_CHECK();
    }
    RBuf<long long> breakers(ctx, RS_BREAK, n);
    fill<long long>(ctx, breakers.p, n, (long long)n);
    GammaArgs<W> ga{n, ids.p, vcmap.p, row_map.p, ts.p, inner.p, oc.p, g.vtx_w.p, cs.total_deg.p, constraint, gamma,
                    breakers.p};
    k_break_part1<W><<<grid, 256, 0, ctx.stream>>>(ga);
    PGGC_LAUNCH_CHECK();
    if constexpr (std::is_same<V, i64>::value) {
        scan_apply(ctx, OcInI<i64>{ids.p, pv.p, inner.p}, OcEpiI{ids.p, oc.p}, n, nullptr, nullptr);
    } else {
        RBuf<double> inc(ctx, RS_INC, n);
        det_scan(ctx, OcInD{ids.p, pv.p, inner.p}, inc.p, n);
        k_scatter_by_ids<<<grid, 256, 0, ctx.stream>>>(n, ids.p, inc.p, oc.p);
        PGGC_LAUNCH_CHECK();
    }
    k_break_part2<W><<<grid, 256, 0, ctx.stream>>>(ga);
    PGGC_LAUNCH_CHECK();
    k_break_apply<<<grid, 256, 0, ctx.stream>>>(n, ids.p, breakers.p, vcmap.p);
    PGGC_LAUNCH_CHECK();

    // --- contigitize
    RBuf<i32> newid(ctx, RS_NEWID, n);
    RBuf<i64> tot(ctx, RS_TOT, 2);
    scan_apply(ctx, RootFlag{vcmap.p}, RootEpi{newid.p}, n, nullptr, tot.p);
    k_contig_apply<<<grid, 256, 0, ctx.stream>>>(n, vcmap.p, newid.p, vcmap_out);
    PGGC_LAUNCH_CHECK();
    // the count and the device error word in one round trip
    PGGC_CUDA(cudaMemsetAsync(tot.p + 1, 0, sizeof(i64), ctx.stream));
    PGGC_CUDA(cudaMemcpyAsync(tot.p + 1, ctx.d_err, sizeof(int), cudaMemcpyDeviceToDevice, ctx.stream));
    const i64* ht = (const i64*)ctx.readback(tot.p, 2 * sizeof(i64));
    const i64 nc = ht[0];
    ctx.raise_device_error((int)ht[1]);
    // algorithmic bytes: two adjacency passes (pick, inner connectivity) each
    // reading column, weight, constraint and label of the neighbour; about ten
    // n-sized int32 passes (orderings, sort keys, trees, breaks, relabel)
    ctx.prof_add_bytes("leiden_refine", (double)g.nnz * 2.0 * (4.0 + (g.uniform ? 0.0 : sizeof(W)) + 4.0 + 4.0) +
                                            (double)n * 10.0 * 4.0);
    return nc;
}

template i64 coarsen_leidenR<i32>(Context&, const Graph<i32>&, const Ordering&, const i32*, const ClusterState<i64>&, u32,
                                  u32, i32*, bool);
template i64 coarsen_leidenR<float>(Context&, const Graph<float>&, const Ordering&, const i32*,
                                    const ClusterState<double>&, u32, u32, i32*, bool);

}  // namespace pggc
