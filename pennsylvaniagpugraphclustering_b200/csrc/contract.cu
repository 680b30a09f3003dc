// contract.cu -- build_coarse_graph (src/contract.cpp:234-336) for sm_100a.
//
// Pipeline:
//  1. one pass over the vertices counts members and the edge bound
//     (sum of member degrees) of every coarse vertex;
//  2. scans give member offsets and per-coarse-vertex scratch offsets; members
//     are scattered (counting sort by coarse id) and their degrees prefix-summed
//     so each coarse vertex owns one flat virtual edge list;
//  3. hashed merge of the (c_u, c_v) keys: a warp per coarse vertex with bound
//     <= 128 (per-warp shared-memory table, __match_any_sync chunk
//     pre-aggregation), a 256-thread block for bound <= 4096 (shared-memory
//     table), a block with a global-memory table above that; self-loops are
//     dropped (src/contract.cpp:191,209) and weights summed exactly (int64 /
//     FP64);
//  4. a prefix sum of the unique counts gives the coarse row offsets;
//  5. each row is sorted by column (warp rank sort, block bitonic sort in shared
//     memory, LSD radix sort for rows above 4096 entries) and written out.
// The output is the canonical (row, col)-sorted coarse CSR.
#include "kernels.cuh"

namespace pggc {

__device__ __forceinline__ void cvatomic_add(i64* a, i64 x) { ::atomicAdd((unsigned long long*)a, (unsigned long long)x); }
__device__ __forceinline__ void cvatomic_add(double* a, double x) { ::atomicAdd(a, x); }

template <class W>
__global__ void k_contract_count(DGraph<W> g, const i32* vcmap, i64* cnt, i64* bound) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < g.n; i += (i64)gridDim.x * blockDim.x) {
        i32 c = vcmap[i];
        ::atomicAdd((unsigned long long*)&cnt[c], 1ull);
        ::atomicAdd((unsigned long long*)&bound[c], (unsigned long long)(g.rowptr[i + 1] - g.rowptr[i]));
    }
}

__global__ void k_scatter_members(const i32* vcmap, i64 n, i64* cursor, i32* members) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
        i32 c = vcmap[i];
        i64 pos = (i64)::atomicAdd((unsigned long long*)&cursor[c], 1ull);
        members[pos] = (i32)i;
    }
}

struct MemberDegIn {
    const i64* rowptr;
    const i32* members;
    i64 n;
    __device__ i64 operator()(i64 m) const {
        if (m >= n) return 0;
        i32 i = members[m];
        return rowptr[i + 1] - rowptr[i];
    }
};

template <class W>
struct CArgs {
    using V = typename Traits<W>::V;
    DGraph<W> g;
    const i32* vcmap;
    const i64* cstart;   // member offsets [nc+1]
    const i32* members;
    const i64* P;        // exclusive prefix of member degrees in member order [n+1]
    i32* out_key;        // scratch, indexed by P[cstart[c]] + k
    V* out_val;
    i64* ucount;         // unique neighbours per coarse vertex
    int* err;
    u32 probe_cap;       // fault-injection cap on hash probes (0: none)
};

// Edge position j of virtual edge q (global flat index) of coarse vertex c.
__device__ __forceinline__ i64 flat_edge(const i64* P, const i32* members, const i64* rowptr, i64 m0, i64 m1, i64 q) {
    // largest m in [m0, m1) with P[m] <= q
    i64 lo = m0, hi = m1 - 1;
    while (lo < hi) {
        i64 mid = (lo + hi + 1) >> 1;
        if (P[mid] <= q) lo = mid;
        else hi = mid - 1;
    }
    return rowptr[members[lo]] + (q - P[lo]);
}

template <class V>
__device__ __forceinline__ void ctable_add(i32* keys, V* vals, u32 mask, i32 c, V x, int* err, u32 cap) {
    u32 s = xorshift32((u32)c) & mask;
    volatile i32* vk = keys;
    const u32 limit = (cap != 0 && cap <= mask) ? cap : mask + 1;
    for (u32 probe = 0; probe < limit; probe++) {
        i32 k = vk[s];
        if (k == c) {
            cvatomic_add(&vals[s], x);
            return;
        }
        if (k == -1) {
            i32 old = atomicCAS(&keys[s], -1, c);
            if (old == -1 || old == c) {
                cvatomic_add(&vals[s], x);
                return;
            }
        }
        s = (s + 1) & mask;
    }
    atomicExch(err, (int)DEV_ERR_PROBE);
}

template <class V>
__device__ __forceinline__ V cgroup_sum(unsigned peers, V val, bool leader) {
    int maxsize = __reduce_max_sync(FULL, (unsigned)__popc(peers));
    V s = V(0);
    unsigned rem = peers;
    const int l = lane_id();
    for (int r = 0; r < maxsize; r++) {
        int src = l;
        bool take = leader && rem;
        if (take) {
            src = __ffs(rem) - 1;
            rem &= rem - 1;
        }
        V x = __shfl_sync(FULL, val, src);
        if (take) s = s + x;
    }
    return s;
}

// one 32-edge chunk of coarse vertex c's flat list: q = base + lane
template <class W>
__device__ __forceinline__ void cchunk(const CArgs<W>& a, i32 c, i64 m0, i64 m1, i64 q, i64 qend, i32* keys,
                                       typename Traits<W>::V* vals, u32 mask) {
    using V = typename Traits<W>::V;
    bool valid = q < qend;
    i32 u = -1;
    V wv = V(0);
    if (valid) {
        i64 j = flat_edge(a.P, a.members, a.g.rowptr, m0, m1, q);
        u = a.vcmap[a.g.col[j]];
        wv = V(a.g.wgt(j));
    }
    bool keep = valid && u != c;
    i32 key = keep ? u : (i32)(0x80000000u | lane_id());
    unsigned peers = __match_any_sync(FULL, key);
    bool leader = keep && ((peers & lanemask_lt()) == 0);
    V s = a.g.w ? cgroup_sum<V>(peers, wv, leader) : V(__popc(peers));
    if (leader) ctable_add(keys, vals, mask, u, s, a.err, a.probe_cap);
}

// warp per coarse row with a per-warp shared-memory table of CW_T slots
// (rows with bound <= CW_T / 2)
template <class W, int CW_T, int CW_WARPS>
__global__ void __launch_bounds__(CW_WARPS * 32) k_contract_warp(CArgs<W> a, const i32* list, const i64* d_count) {
    using V = typename Traits<W>::V;
    __shared__ i32 tk[CW_WARPS][CW_T];
    __shared__ V tv[CW_WARPS][CW_T];
    const int l = lane_id(), w = threadIdx.x >> 5;
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
    const i64 count = *d_count;
    for (i64 x = gw; x < count; x += nw) {
        i32 c = list[x];
        i64 m0 = a.cstart[c], m1 = a.cstart[c + 1];
        i64 q0 = a.P[m0], q1 = a.P[m1];
        i64 bound = q1 - q0;
        u32 T = next_pow2_u32((u32)(2 * (bound > 1 ? bound : 1)));
        i32* keys = tk[w];
        V* vals = tv[w];
        for (u32 s = l; s < T; s += 32) {
            keys[s] = -1;
            vals[s] = V(0);
        }
        __syncwarp();
        for (i64 q = q0 + l; q - l < q1; q += 32) cchunk(a, c, m0, m1, q, q1, keys, vals, T - 1);
        __syncwarp();
        i64 written = 0;
        for (u32 s0 = 0; s0 < T; s0 += 32) {
            u32 s = s0 + l;
            bool occ = s < T && keys[s] != -1;
            unsigned m = __ballot_sync(FULL, occ);
            if (occ) {
                i64 pos = q0 + written + __popc(m & lanemask_lt());
                a.out_key[pos] = keys[s];
                a.out_val[pos] = vals[s];
            }
            written += __popc(m);
        }
        if (l == 0) a.ucount[c] = written;
        __syncwarp();
    }
}

// block per coarse row; the table is in shared memory (`gcap` slots, sized to
// the bucket's largest table) or, with GLOBAL, in a per-block global region
template <class W, bool GLOBAL>
__global__ void __launch_bounds__(256) k_contract_block(CArgs<W> a, const i32* list, const i64* d_count, i32* gkeys,
                                                        typename Traits<W>::V* gvals, i64 gcap, i64 nc) {
    using V = typename Traits<W>::V;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ unsigned long long wcount;
    V* svals = (V*)smem_raw;
    i32* skeys = (i32*)(smem_raw + sizeof(V) * (GLOBAL ? 0 : gcap));
    const int l = lane_id(), w = threadIdx.x >> 5;
    i32* keys = GLOBAL ? gkeys + (i64)blockIdx.x * gcap : skeys;
    V* vals = GLOBAL ? gvals + (i64)blockIdx.x * gcap : svals;
    const i64 count = *d_count;
    for (i64 x = blockIdx.x; x < count; x += gridDim.x) {
        i32 c = list[x];
        i64 m0 = a.cstart[c], m1 = a.cstart[c + 1];
        i64 q0 = a.P[m0], q1 = a.P[m1];
        i64 U = min(q1 - q0, nc);
        u32 T = next_pow2_u32((u32)(2 * (U > 1 ? U : 1)));
        for (u32 s = threadIdx.x; s < T; s += 256) {
            keys[s] = -1;
            vals[s] = V(0);
        }
        if (threadIdx.x == 0) wcount = 0;
        __syncthreads();
        for (i64 q = q0 + (i64)w * 32 + l; q - l < q1; q += 256) cchunk(a, c, m0, m1, q, q1, keys, vals, T - 1);
        __syncthreads();
        for (u32 s0 = w * 32; s0 < T; s0 += 256) {
            u32 s = s0 + l;
            bool occ = s < T && keys[s] != -1;
            unsigned m = __ballot_sync(FULL, occ);
            i64 base = 0;
            if (l == 0 && m) base = (i64)::atomicAdd(&wcount, (unsigned long long)__popc(m));
            base = __shfl_sync(FULL, base, 0);
            if (occ) {
                i64 pos = q0 + base + __popc(m & lanemask_lt());
                a.out_key[pos] = keys[s];
                a.out_val[pos] = vals[s];
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) a.ucount[c] = (i64)wcount;
        __syncthreads();
    }
}

// ---- per-row sort + placement ----------------------------------------------
template <class W>
__device__ __forceinline__ W to_w(typename Traits<W>::V v) {
    return (W)v;
}

template <class W>
__global__ void __launch_bounds__(256) k_place_warp(const i32* list, const i64* d_count, const i64* P, const i64* cstart,
                                                    const i64* ucount, const i64* rowptr, const i32* skey,
                                                    const typename Traits<W>::V* sval, i32* col, W* wout) {
    const int l = lane_id();
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
    const i64 count = *d_count;
    for (i64 x = gw; x < count; x += nw) {
        i32 c = list[x];
        i64 src = P[cstart[c]];
        i64 u = ucount[c];
        i32 key = l < u ? skey[src + l] : 2147483647;
        auto val = l < u ? sval[src + l] : typename Traits<W>::V(0);
        int rank = 0;
        for (int k = 0; k < 32; k++) {
            i32 o = __shfl_sync(FULL, key, k);
            rank += (o < key) ? 1 : 0;
        }
        if (l < u) {
            col[rowptr[c] + rank] = key;
            wout[rowptr[c] + rank] = to_w<W>(val);
        }
    }
}

// 32 < u <= PW_MAX: the warp stages the row in shared memory and each lane
// ranks its entries against all of them
constexpr int PW_MAX = 256;
constexpr int PW_WARPS = 8;

template <class W>
__global__ void __launch_bounds__(PW_WARPS * 32) k_place_warp_rank(const i32* list, const i64* d_count, const i64* P,
                                                                   const i64* cstart, const i64* ucount,
                                                                   const i64* rowptr, const i32* skey,
                                                                   const typename Traits<W>::V* sval, i32* col,
                                                                   W* wout) {
    __shared__ i32 kk[PW_WARPS][PW_MAX];
    const int l = lane_id(), w = threadIdx.x >> 5;
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
    const i64 count = *d_count;
    for (i64 x = gw; x < count; x += nw) {
        i32 c = list[x];
        i64 src = P[cstart[c]];
        int u = (int)ucount[c];
        for (int s = l; s < u; s += 32) kk[w][s] = skey[src + s];
        __syncwarp();
        for (int s = l; s < u; s += 32) {
            i32 key = kk[w][s];
            int rank = 0;
            for (int t = 0; t < u; t++) rank += kk[w][t] < key ? 1 : 0;
            col[rowptr[c] + rank] = key;
            wout[rowptr[c] + rank] = to_w<W>(sval[src + s]);
        }
        __syncwarp();
    }
}

constexpr int PB_MAX = 4096;

template <class W>
__global__ void __launch_bounds__(256) k_place_block(const i32* list, const i64* d_count, const i64* P, const i64* cstart,
                                                     const i64* ucount, const i64* rowptr, const i32* skey,
                                                     const typename Traits<W>::V* sval, i32* col, W* wout) {
    using V = typename Traits<W>::V;
    __shared__ i32 kk[PB_MAX];
    __shared__ V vv[PB_MAX];
    const i64 count = *d_count;
    for (i64 x = blockIdx.x; x < count; x += gridDim.x) {
        i32 c = list[x];
        i64 src = P[cstart[c]];
        i64 u = ucount[c];
        u32 T = next_pow2_u32((u32)u);
        for (u32 s = threadIdx.x; s < T; s += 256) {
            kk[s] = s < u ? skey[src + s] : 2147483647;
            vv[s] = s < u ? sval[src + s] : V(0);
        }
        __syncthreads();
        // bitonic sort of T keys (ascending)
        for (u32 k = 2; k <= T; k <<= 1) {
            for (u32 j = k >> 1; j > 0; j >>= 1) {
                for (u32 t = threadIdx.x; t < T; t += 256) {
                    u32 p = t ^ j;
                    if (p > t) {
                        bool up = (t & k) == 0;
                        i32 a0 = kk[t], a1 = kk[p];
                        if ((a0 > a1) == up) {
                            kk[t] = a1;
                            kk[p] = a0;
                            V v0 = vv[t];
                            vv[t] = vv[p];
                            vv[p] = v0;
                        }
                    }
                }
                __syncthreads();
            }
        }
        for (u32 s = threadIdx.x; s < u; s += 256) {
            col[rowptr[c] + s] = kk[s];
            wout[rowptr[c] + s] = to_w<W>(vv[s]);
        }
        __syncthreads();
    }
}

// big rows: gather into (row-major) temp with composite keys, radix sort, place
template <class V>
__global__ void k_big_gather(const i32* list, i64 count, const i64* tstart, const i64* P, const i64* cstart,
                             const i64* ucount, const i32* skey, const V* sval, u64* tkey, V* tval) {
    for (i64 x = blockIdx.x; x < count; x += gridDim.x) {
        i32 c = list[x];
        i64 src = P[cstart[c]];
        i64 u = ucount[c];
        i64 dst = tstart[x];
        for (i64 s = threadIdx.x; s < u; s += blockDim.x) {
            tkey[dst + s] = ((u64)x << 32) | (u64)(u32)skey[src + s];
            tval[dst + s] = sval[src + s];
        }
    }
}
template <class W>
__global__ void k_big_place(const i32* list, i64 count, const i64* tstart, const i64* rowptr, const u64* tkey,
                            const typename Traits<W>::V* tval, i32* col, W* wout) {
    for (i64 x = blockIdx.x; x < count; x += gridDim.x) {
        i32 c = list[x];
        i64 a = tstart[x], b = tstart[x + 1];
        for (i64 y = a + threadIdx.x; y < b; y += blockDim.x) {
            col[rowptr[c] + (y - a)] = (i32)(u32)(tkey[y] & 0xffffffffull);
            wout[rowptr[c] + (y - a)] = to_w<W>(tval[y]);
        }
    }
}

__global__ void k_max_bound(const i32* list, const i64* d_count, const i64* P, const i64* cstart,
                            unsigned long long* out) {
    const i64 count = *d_count;
    unsigned long long m = 0;
    for (i64 x = blockIdx.x * (i64)blockDim.x + threadIdx.x; x < count; x += (i64)gridDim.x * blockDim.x) {
        i32 c = list[x];
        unsigned long long b = (unsigned long long)(P[cstart[c + 1]] - P[cstart[c]]);
        m = b > m ? b : m;
    }
    for (int d = 16; d >= 1; d >>= 1) {
        unsigned long long o = __shfl_xor_sync(FULL, m, d);
        m = o > m ? o : m;
    }
    if (lane_id() == 0 && m) atomicMax(out, m);
}

struct BucketFlag {
    const i64* val;
    i64 lo, hi;  // lo < v <= hi
    __device__ i64 operator()(i64 c) const {
        i64 v = val[c];
        return (v > lo && v <= hi) ? 1 : 0;
    }
};
// lo < bound <= hi, and for mode 1 / 2 also U = min(bound, nc) <= / > 4096
struct BoundFlag {
    const i64* P;
    const i64* cstart;
    i64 lo, hi, nc;
    int mode;
    __device__ i64 operator()(i64 c) const {
        i64 v = P[cstart[c + 1]] - P[cstart[c]];
        if (!(v > lo && v <= hi)) return 0;
        i64 U = v < nc ? v : nc;
        if (mode == 1) return U <= HUGE_DEG ? 1 : 0;
        if (mode == 2) return U > HUGE_DEG ? 1 : 0;
        return 1;
    }
};
struct IdxEpiC {
    i32* dst;
    __device__ void operator()(i64 x, i64 excl, i64 v) const {
        if (v) dst[excl] = (i32)x;
    }
};
struct UcountIn {
    const i64* u;
    i64 nc;
    __device__ i64 operator()(i64 c) const { return c < nc ? u[c] : 0; }
};
struct RowptrOut {
    i64* rp;
    __device__ void operator()(i64 c, i64 excl, i64) const { rp[c] = excl; }
};
// unique count of the x-th row of a device-counted list (0 past the count)
struct ListUIn {
    const i32* list;
    const i64* u;
    const i64* d_count;
    __device__ i64 operator()(i64 x) const { return x < *d_count ? u[list[x]] : 0; }
};

template <class W>
std::unique_ptr<Graph<W>> build_coarse_graph(Context& ctx, const Graph<W>& g, const i32* vcmap, i64 nc) {
    using V = typename Traits<W>::V;
    ProfScope ps(ctx, "contract");
    auto cg = std::make_unique<Graph<W>>();
    cg->n = nc;
    cg->uniform = false;
    const i64 n = g.n;
    auto gv = g.view();
    cg->rowptr = DBuf<i64>(ctx, nc + 1);
    if (nc == 0 || n == 0) {
        PGGC_CUDA(cudaMemsetAsync(cg->rowptr.p, 0, sizeof(i64) * (nc + 1), ctx.stream));
        cg->nnz = 0;
        cg->col = DBuf<i32>(ctx, 1);
        cg->w = DBuf<W>(ctx, 1);
        return cg;
    }
    DBuf<i64> cnt(ctx, nc + 1), bound(ctx, nc + 1), cstart(ctx, nc + 1), P(ctx, n + 1), ucount(ctx, nc + 1);
    DBuf<i32> members(ctx, n);
    PGGC_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(i64) * (nc + 1), ctx.stream));
    PGGC_CUDA(cudaMemsetAsync(bound.p, 0, sizeof(i64) * (nc + 1), ctx.stream));
    int gridv = (int)std::min<i64>(ceil_div(n, 256), (i64)ctx.num_sms * 16);
    k_contract_count<W><<<gridv, 256, 0, ctx.stream>>>(gv, vcmap, cnt.p, bound.p);
    PGGC_LAUNCH_CHECK();
    scan_apply(ctx, ArrIn{cnt.p}, ArrOutExcl{cstart.p}, nc + 1, nullptr, nullptr);
    {
        DBuf<i64> cursor(ctx, nc + 1);
        copy_d2d(ctx, cursor.p, cstart.p, nc + 1);
        k_scatter_members<<<gridv, 256, 0, ctx.stream>>>(vcmap, n, cursor.p, members.p);
        PGGC_LAUNCH_CHECK();
    }
    DBuf<i64> tot(ctx, 4);
    scan_apply(ctx, MemberDegIn{gv.rowptr, members.p, n}, ArrOutExcl{P.p}, n + 1, nullptr, tot.p);
    const i64 total_bound = g.nnz;
    DBuf<i32> okey(ctx, std::max<i64>(total_bound, 1));
    DBuf<V> oval(ctx, std::max<i64>(total_bound, 1));

    // bucket lists by table size U = min(bound, nc) and bound:
    //   small warp rows (bound <= 32), medium warp rows (bound <= 256),
    //   block rows with a shared-memory table (U <= 4096), global-table rows
    DBuf<i32> lw(ctx, nc), lm(ctx, nc), lb(ctx, nc), lh(ctx, nc);
    DBuf<i64> counts(ctx, 12);
    PGGC_CUDA(cudaMemsetAsync(counts.p, 0, sizeof(i64) * 12, ctx.stream));
    scan_apply(ctx, BoundFlag{P.p, cstart.p, -1, 32, nc, 0}, IdxEpiC{lw.p}, nc, nullptr, counts.p + 0);
    scan_apply(ctx, BoundFlag{P.p, cstart.p, 32, 256, nc, 0}, IdxEpiC{lm.p}, nc, nullptr, counts.p + 8);
    scan_apply(ctx, BoundFlag{P.p, cstart.p, 256, (i64)1 << 62, nc, 1}, IdxEpiC{lb.p}, nc, nullptr, counts.p + 1);
    scan_apply(ctx, BoundFlag{P.p, cstart.p, 256, (i64)1 << 62, nc, 2}, IdxEpiC{lh.p}, nc, nullptr, counts.p + 2);
    k_max_bound<<<64, 256, 0, ctx.stream>>>(lh.p, counts.p + 2, P.p, cstart.p, (unsigned long long*)(counts.p + 7));
    PGGC_LAUNCH_CHECK();
    k_max_bound<<<64, 256, 0, ctx.stream>>>(lb.p, counts.p + 1, P.p, cstart.p, (unsigned long long*)(counts.p + 9));
    PGGC_LAUNCH_CHECK();
    // one round trip: bucket sizes and the largest bounds
    const i64* hc = (const i64*)ctx.readback(counts.p, 12 * sizeof(i64));
    const i64 n_w = hc[0], n_b = hc[1], n_h = hc[2], max_huge = hc[7], n_m = hc[8], max_block = hc[9];

    CArgs<W> a;
    a.g = gv;
    a.vcmap = vcmap;
    a.cstart = cstart.p;
    a.members = members.p;
    a.P = P.p;
    a.out_key = okey.p;
    a.out_val = oval.p;
    a.ucount = ucount.p;
    a.err = ctx.d_err;
    a.probe_cap = ctx.probe_cap;
    if (n_w > 0) {
        constexpr int WARPS = 8;
        int grid = (int)std::min<i64>(ceil_div(n_w, WARPS), (i64)ctx.num_sms * 16);
        k_contract_warp<W, 64, WARPS><<<grid, WARPS * 32, 0, ctx.stream>>>(a, lw.p, counts.p + 0);
        PGGC_LAUNCH_CHECK();
    }
    if (n_m > 0) {
        constexpr int WARPS = 4;
        int grid = (int)std::min<i64>(ceil_div(n_m, WARPS), (i64)ctx.num_sms * 16);
        k_contract_warp<W, 512, WARPS><<<grid, WARPS * 32, 0, ctx.stream>>>(a, lm.p, counts.p + 8);
        PGGC_LAUNCH_CHECK();
    }
    if (n_b > 0) {
        // table sized to the largest row of the bucket
        i64 tmax = next_pow2_u32((u32)(2 * std::max<i64>(std::min<i64>(max_block, nc), 1)));
        size_t sm = (sizeof(V) + sizeof(i32)) * (size_t)tmax;
        set_dynamic_smem_once(k_contract_block<W, false>, (int)((sizeof(V) + sizeof(i32)) * SEL_TS_MAX), ctx.device);
        int per_sm = 0;
        PGGC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_contract_block<W, false>, 256, sm));
        int grid = (int)std::min<i64>(n_b, (i64)ctx.num_sms * std::max(per_sm, 1));
        k_contract_block<W, false><<<grid, 256, sm, ctx.stream>>>(a, lb.p, counts.p + 1, nullptr, nullptr, tmax, nc);
        PGGC_LAUNCH_CHECK();
    }
    if (n_h > 0) {
        // global tables sized for the largest table among the huge rows, one
        // region per resident block, at most 2 GiB of tables
        i64 maxb = std::min<i64>(max_huge, nc);
        i64 gcap = next_pow2_u32((u32)std::min<i64>(2 * std::max<i64>(maxb, 1), (i64)1 << 30));
        i64 by_mem = std::max<i64>(1, ((i64)2 << 30) / (gcap * (i64)(sizeof(V) + sizeof(i32))));
        int grid = (int)std::min<i64>(std::min<i64>(n_h, (i64)ctx.num_sms * 2), by_mem);
        i32* gk = ctx.ws_get<i32>(WS_CONTRACT_GK, gcap * grid);
        V* gvv = ctx.ws_get<V>(WS_CONTRACT_GV, gcap * grid);
        k_contract_block<W, true><<<grid, 256, 0, ctx.stream>>>(a, lh.p, counts.p + 2, gk, gvv, gcap, nc);
        PGGC_LAUNCH_CHECK();
    }
    // coarse row offsets, placement buckets and the big-row total, then one round trip
    scan_apply(ctx, UcountIn{ucount.p, nc}, RowptrOut{cg->rowptr.p}, nc + 1, nullptr, tot.p + 1);
    DBuf<i32> pw(ctx, nc), pr(ctx, nc), pb(ctx, nc), ph(ctx, nc);
    scan_apply(ctx, BucketFlag{ucount.p, 0, 32}, IdxEpiC{pw.p}, nc, nullptr, counts.p + 3);
    scan_apply(ctx, BucketFlag{ucount.p, 32, PW_MAX}, IdxEpiC{pr.p}, nc, nullptr, counts.p + 10);
    scan_apply(ctx, BucketFlag{ucount.p, PW_MAX, PB_MAX}, IdxEpiC{pb.p}, nc, nullptr, counts.p + 4);
    scan_apply(ctx, BucketFlag{ucount.p, PB_MAX, (i64)1 << 62}, IdxEpiC{ph.p}, nc, nullptr, counts.p + 5);
    DBuf<i64> tstart(ctx, nc + 1);
    scan_apply(ctx, ListUIn{ph.p, ucount.p, counts.p + 5}, ArrOutExcl{tstart.p}, nc + 1, nullptr, tot.p + 2);
    PGGC_CUDA(cudaMemcpyAsync(counts.p + 6, tot.p + 1, 2 * sizeof(i64), cudaMemcpyDeviceToDevice, ctx.stream));
    const i64* pc = (const i64*)ctx.readback(counts.p, 12 * sizeof(i64));
    const i64 p_w = pc[3], p_b = pc[4], p_h = pc[5], nnz_c = pc[6], tn = pc[7], p_r = pc[10];
    ctx.check_device_error();
    cg->nnz = nnz_c;
    cg->col = DBuf<i32>(ctx, std::max<i64>(nnz_c, 1));
    cg->w = DBuf<W>(ctx, std::max<i64>(nnz_c, 1));
    if (p_w > 0) {
        int grid = (int)std::min<i64>(ceil_div(p_w, 8), (i64)ctx.num_sms * 8);
        k_place_warp<W><<<grid, 256, 0, ctx.stream>>>(pw.p, counts.p + 3, P.p, cstart.p, ucount.p, cg->rowptr.p, okey.p,
                                                      oval.p, cg->col.p, cg->w.p);
        PGGC_LAUNCH_CHECK();
    }
    if (p_r > 0) {
        int grid = (int)std::min<i64>(ceil_div(p_r, PW_WARPS), (i64)ctx.num_sms * 8);
        k_place_warp_rank<W><<<grid, PW_WARPS * 32, 0, ctx.stream>>>(pr.p, counts.p + 10, P.p, cstart.p, ucount.p,
                                                                     cg->rowptr.p, okey.p, oval.p, cg->col.p,
                                                                     cg->w.p);
        PGGC_LAUNCH_CHECK();
    }
    if (p_b > 0) {
        int grid = (int)std::min<i64>(p_b, (i64)ctx.num_sms * 4);
        k_place_block<W><<<grid, 256, 0, ctx.stream>>>(pb.p, counts.p + 4, P.p, cstart.p, ucount.p, cg->rowptr.p,
                                                       okey.p, oval.p, cg->col.p, cg->w.p);
        PGGC_LAUNCH_CHECK();
    }
    if (p_h > 0) {
        DBuf<u64> tk(ctx, tn), tk2(ctx, tn);
        DBuf<V> tv(ctx, tn), tv2(ctx, tn);
        int grid = (int)std::min<i64>(p_h, (i64)ctx.num_sms * 4);
        k_big_gather<V><<<grid, 256, 0, ctx.stream>>>(ph.p, p_h, tstart.p, P.p, cstart.p, ucount.p, okey.p, oval.p,
                                                      tk.p, tv.p);
        PGGC_LAUNCH_CHECK();
        int hib = 32 + bits_for((u64)p_h);
        radix_sort_pairs<V>(ctx, tk.p, tv.p, tn, 0, hib, tk2.p, tv2.p);
        k_big_place<W><<<grid, 256, 0, ctx.stream>>>(ph.p, p_h, tstart.p, cg->rowptr.p, tk.p, tv.p, cg->col.p,
                                                     cg->w.p);
        PGGC_LAUNCH_CHECK();
    }
    // algorithmic bytes: per fine edge its column, weight, the map of its head
    // and one table insert (key + value); per fine vertex its offset and map;
    // the coarse CSR written once
    {
        const double wb = g.uniform ? 0.0 : (double)sizeof(W);
        const double vb = (double)sizeof(V);
        ctx.prof_add_bytes("contract", (double)g.nnz * (4.0 + wb + 4.0 + 4.0 + vb) + (double)g.n * (8.0 + 4.0) +
                                           (double)nnz_c * (4.0 + sizeof(W)) + (double)(nc + 1) * 8.0);
    }
    return cg;
}

template <class W>
__global__ void k_coarsen_vtx_w(DGraph<W> g, const i32* vcmap, typename Traits<W>::V* out) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < g.n; i += (i64)gridDim.x * blockDim.x)
        cvatomic_add(&out[vcmap[i]], g.vtx_w[i]);
}

// coarsen_vtx_w (src/clustering_methods.cpp:33-38)
template <class W>
void coarsen_vtx_w(Context& ctx, const Graph<W>& g, const i32* vcmap, Graph<W>& cg) {
    using V = typename Traits<W>::V;
    cg.vtx_w = DBuf<V>(ctx, std::max<i64>(cg.n, 1));
    PGGC_CUDA(cudaMemsetAsync(cg.vtx_w.p, 0, sizeof(V) * std::max<i64>(cg.n, 1), ctx.stream));
    if (g.n == 0) return;
    int grid = (int)std::min<i64>(ceil_div(g.n, 256), (i64)ctx.num_sms * 16);
    k_coarsen_vtx_w<W><<<grid, 256, 0, ctx.stream>>>(g.view(), vcmap, cg.vtx_w.p);
    PGGC_LAUNCH_CHECK();
}

template std::unique_ptr<Graph<i32>> build_coarse_graph<i32>(Context&, const Graph<i32>&, const i32*, i64);
template std::unique_ptr<Graph<float>> build_coarse_graph<float>(Context&, const Graph<float>&, const i32*, i64);
template void coarsen_vtx_w<i32>(Context&, const Graph<i32>&, const i32*, Graph<i32>&);
template void coarsen_vtx_w<float>(Context&, const Graph<float>&, const i32*, Graph<float>&);

}  // namespace pggc
