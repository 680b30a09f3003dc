// local_move.cu -- the synchronous parallel local-move sweep
// (src/local_mover.cpp:100-1483) rebuilt for sm_100a.
//
// Design (vs. the reference's persistent per-vertex hash tables):
//  * No conn tables are kept between sweeps.  The DeltaQ argmax aggregates each
//    evaluated vertex's neighbour-cluster weights on the fly: a warp per vertex
//    (degree < 128) pre-aggregates each 32-edge chunk with __match_any_sync and
//    either reduces it directly (degree <= 32) or inserts group sums into a
//    per-warp shared-memory table; a 256-thread block per vertex with a
//    shared-memory table (degree <= 4096); global-memory tables for larger
//    degrees.  Aggregated sums are exact, so the result equals the reference's
//    table contents; ties go to the smallest cluster id.
//  * The own-cluster weights (pvals) are recomputed exactly for the vertices
//    whose neighbourhood changed, which is the set whose dest cache the
//    reference invalidates (moved vertices and their neighbours).
//  * Candidate / move lists are order-preserving compactions of order1, so new
//    cluster ids and the strict prefix follow the reference's move order.
//  * One host round trip per sweep (candidate and move counts); everything else
//    reads counts from device memory.
#include <mutex>
#include "kernels.cuh"
#include "bulk.cuh"
#include "filter.cuh"

namespace pggc {

template <class V>
struct LMScalars {
    i64 num_cand, split, num_moves, num_new, num_avail, avail_k;
    unsigned long long new_hint;  // NEW_PART moves counted while compacting the move list
    i64 label_count, best_label_count;
    V uncut, best_uncut, last_pval, pval_sum;
    i64 sumsq_i;
    double sumsq_d;
    double obj, best_obj;
    int improved;
    int err;  // copy of the context's device error word (end of a local move)
    int pad[2];
    i64 relabel_count;  // labels after the final relabel
};

__device__ __forceinline__ void vatomic_add(i64* a, i64 x) { ::atomicAdd((unsigned long long*)a, (unsigned long long)x); }
__device__ __forceinline__ void vatomic_add(double* a, double x) { ::atomicAdd(a, x); }

struct Best {
    float jc;
    i32 c;
};
__device__ __forceinline__ bool better(float jc, i32 c, const Best& b) { return jc > b.jc || (jc == b.jc && c < b.c); }
__device__ __forceinline__ Best none_best() { return Best{-INFINITY, 2147483647}; }
// Order-preserving map of a float onto u32 (no NaN here); with it the best
// (largest gain, then smallest cluster id) of a lane group is two hardware
// reductions instead of a shuffle butterfly.  Gains are never -0.0 (a
// candidate has f > 0 and f - x is +0.0 when equal), so float equality and
// key equality agree.
__device__ __forceinline__ u32 f2ord(float f) {
    const u32 b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ord2f(u32 k) { return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k); }
__device__ __forceinline__ void reduce_best(Best& b, unsigned mask) {
    const u32 k = f2ord(b.jc);
    const u32 mk = __reduce_max_sync(mask, k);
    const u32 mc = __reduce_min_sync(mask, k == mk ? (u32)b.c : 0xFFFFFFFFu);
    b = Best{ord2f(mk), (i32)mc};
}
__device__ __forceinline__ void warp_best(Best& b) { reduce_best(b, FULL); }


// canonical per-vertex sum by a G-lane group (exact match of the 32-lane
// association for degree <= 2G; integer sums are order-free)
template <int G, class V, class F>
__device__ __forceinline__ V group_vsum(i64 b, i64 e, int r, F term) {
    if constexpr (std::is_same<V, double>::value) {
        double acc = 0.0;
        for (i64 j = b + r; j < e; j += G) acc += term(j);
#pragma unroll
        for (int d = G / 2; d >= 1; d >>= 1) acc = acc + __shfl_xor_sync(FULL, acc, d);
        return acc;
    } else {
        i64 acc = 0;
        for (i64 j = b + r; j < e; j += G) acc += term(j);
#pragma unroll
        for (int d = G / 2; d >= 1; d >>= 1) acc += __shfl_xor_sync(FULL, acc, d);
        return acc;
    }
}

template <class W>
struct SelArgs {
    using V = typename Traits<W>::V;
    DGraph<W> g;
    const i32* part;
    i32* dest;
    float* gain;
    const V* pvals;
    const V* td;
    const i32* constraint;
    const i64* label_count;  // device
    const V* rsum;           // row weight sums (NULL: no bound check)
    int keys32;              // cluster ids < 2^29: group match keys fit 32 bits
    int dense;               // block kernels: every label indexes the shared table directly
    float pm;
    float fr;
    int initial;
    int* err;
    unsigned long long* prof;  // algorithmic-byte counter (profiling only)
    u32 probe_cap;             // fault-injection cap on hash probes (0: none)
    float inv_load;            // hash-table slots per distinct key (1 / load factor): 2 or 1/0.7
};

// table slots for up to U distinct keys at the tuned load factor (a power of two)
template <class W>
__device__ __forceinline__ u32 sel_table_slots(const SelArgs<W>& a, i64 U) {
    return next_pow2_u32((u32)ceilf((float)U * a.inv_load));
}

// algorithmic bytes of one select evaluation: list entry + dest read, then
// rowptr pair, vtx_w, part, pval, D[part], dest/gain writes, and per edge the
// column, weight and neighbour label (initial mode: column, weight, D[v])
template <class W>
__device__ __forceinline__ unsigned long long sel_bytes(const SelArgs<W>& a, i64 deg, bool evaluated) {
    if (!evaluated) return 8;
    const unsigned long long wb = a.g.w ? sizeof(W) : 0;
    return 60ull + (unsigned long long)deg * (a.initial ? (12ull + wb) : (8ull + wb));
}

struct VCtx {
    i32 p;
    float multi, p_conn, thr;
};

template <class W>
__device__ __forceinline__ VCtx sel_prologue(const SelArgs<W>& a, i32 i) {
    using V = typename Traits<W>::V;
    VCtx v;
    V w = a.g.vtx_w[i];
    v.multi = to_f(w) * a.pm;
    v.p = a.part[i];
    v.p_conn = to_f(a.pvals[i]) - to_f(V(a.td[v.p] - w)) * v.multi;
    v.thr = v.p_conn < 0.0f ? 0.0f : (float)((double)v.p_conn * (1.0 - (double)a.fr));
    return v;
}

// Exact skip: no neighbour cluster can carry more weight than the vertex's
// weight outside its own cluster, ext = rowsum - pval; when even ext rounds
// (one FP32 step up, covering FP64 rounding in either sum) below the
// candidate threshold, no cluster passes the `f >= thr` test of sel_eval and
// the edges need not be read: the outcome is the no-candidate outcome.
template <class W>
__device__ __forceinline__ bool sel_no_candidate(const SelArgs<W>& a, i32 i, const VCtx& vc) {
    if (!a.rsum || a.initial) return false;
    const float fe = nextafterf(to_f(a.rsum[i] - a.pvals[i]), INFINITY);
    return !(fe >= vc.thr);
}

template <class W, bool CON>
__device__ __forceinline__ void sel_eval(const SelArgs<W>& a, const VCtx& vc, i32 c, typename Traits<W>::V jv,
                                         Best& b) {
    using V = typename Traits<W>::V;
    if (!(jv > V(0))) return;
    float f = to_f(jv);
    if (!(f >= vc.thr)) return;
    if (CON && a.constraint[c] != a.constraint[vc.p]) return;
    float jc = f - to_f(a.td[c]) * vc.multi;
    if (jc >= vc.thr && better(jc, c, b)) b = Best{jc, c};
}

template <class W>
__device__ __forceinline__ void sel_finish(const SelArgs<W>& a, i32 i, const VCtx& vc, const Best& b) {
    if (b.c != 2147483647) {
        a.dest[i] = b.c;
        a.gain[i] = b.jc - vc.p_conn;
    } else if (vc.p_conn < 0.0f) {
        a.dest[i] = NEW_PART;
        a.gain[i] = -vc.p_conn;
    } else {
        a.dest[i] = NO_MOVE;
        a.gain[i] = OBJ_MIN;
    }
}

// Sum of `val` over the lanes of `peers` (lane order), valid at the group leader.
template <class V>
__device__ __forceinline__ V group_sum(unsigned peers, V val, bool leader) {
    int size = __popc(peers);
    int maxsize = __reduce_max_sync(FULL, (unsigned)size);
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

// Sum of the weights of the lanes in `peers` (equal neighbour clusters), valid
// at the leader: the lane-order shuffle sum, or the count for unit weights.
template <class W>
__device__ __forceinline__ typename Traits<W>::V peer_sum(const SelArgs<W>& a, unsigned peers, W wr, bool keep,
                                                          bool leader) {
    using V = typename Traits<W>::V;
    if (!a.g.w) return V(__popc(peers));
    return group_sum<V>(peers, keep ? V(wr) : V(0), leader);
}

// Linear-probing insert; gives up (latching DEV_ERR_PROBE) after the table size
// or `cap` probes, whichever is smaller (cap = 0: no extra limit).
template <class V>
__device__ __forceinline__ void table_add(i32* keys, V* vals, u32 mask, i32 c, V x, int* err, u32 cap) {
    u32 s = xorshift32((u32)c) & mask;
    volatile i32* vk = keys;
    const u32 limit = (cap != 0 && cap <= mask) ? cap : mask + 1;
    for (u32 probe = 0; probe < limit; probe++) {
        i32 k = vk[s];
        if (k == c) {
            vatomic_add(&vals[s], x);
            return;
        }
        if (k == -1) {
            i32 old = atomicCAS(&keys[s], -1, c);
            if (old == -1 || old == c) {
                vatomic_add(&vals[s], x);
                return;
            }
        }
        s = (s + 1) & mask;
    }
    atomicExch(err, (int)DEV_ERR_PROBE);
}

// Aggregates one 32-edge chunk (edges j = base + lane, valid if < e) into the
// table, skipping the vertex's own cluster.
template <class W>
__device__ __forceinline__ void chunk_to_table(const SelArgs<W>& a, const VCtx& vc, i64 j, i64 e, i32* keys,
                                               typename Traits<W>::V* vals, u32 mask) {
    using V = typename Traits<W>::V;
    bool valid = j < e;
    i32 c = valid ? a.part[a.g.col[j]] : -1;
    W wr = valid ? a.g.wgt(j) : W(0);
    bool keep = valid && c != vc.p;
    i32 key = keep ? c : (i32)(0x80000000u | lane_id());
    unsigned peers = __match_any_sync(FULL, key);
    bool leader = keep && ((peers & lanemask_lt()) == 0);
    V s = peer_sum<W>(a, peers, wr, keep, leader);
    if (leader) table_add(keys, vals, mask, c, s, a.err, a.probe_cap);
}

// Insert that gives up after TRY_PROBES probes (the caller sends the vertex
// to the global-table pass); a run that long means the table is nearly full.
constexpr u32 TRY_PROBES = 64;
template <class V>
__device__ __forceinline__ bool table_try_add(i32* keys, V* vals, u32 mask, i32 c, V x) {
    u32 s = xorshift32((u32)c) & mask;
    volatile i32* vk = keys;
    for (u32 probe = 0; probe < TRY_PROBES && probe <= mask; probe++) {
        i32 k = vk[s];
        if (k == c) {
            vatomic_add(&vals[s], x);
            return true;
        }
        if (k == -1) {
            i32 old = atomicCAS(&keys[s], -1, c);
            if (old == -1 || old == c) {
                vatomic_add(&vals[s], x);
                return true;
            }
        }
        s = (s + 1) & mask;
    }
    return false;
}

// chunk_to_table with table_try_add: false if this lane's insert failed
template <class W>
__device__ __forceinline__ bool chunk_to_table_try(const SelArgs<W>& a, const VCtx& vc, i64 j, i64 e, i32* keys,
                                                   typename Traits<W>::V* vals, u32 mask) {
    using V = typename Traits<W>::V;
    bool valid = j < e;
    i32 c = valid ? a.part[a.g.col[j]] : -1;
    W wr = valid ? a.g.wgt(j) : W(0);
    bool keep = valid && c != vc.p;
    i32 key = keep ? c : (i32)(0x80000000u | lane_id());
    unsigned peers = __match_any_sync(FULL, key);
    bool leader = keep && ((peers & lanemask_lt()) == 0);
    V s = peer_sum<W>(a, peers, wr, keep, leader);
    return leader ? table_try_add(keys, vals, mask, c, s) : true;
}

// ---- warp per vertex, degree < 128 (order1 bucket 0) ----------------------
constexpr int SELW_WARPS = 8;
constexpr int SELW_T = 256;

template <class W, bool CON>
__global__ void __launch_bounds__(SELW_WARPS * 32) k_select_warp(SelArgs<W> a, Range rg) {
    using V = typename Traits<W>::V;
    __shared__ i32 tk[SELW_WARPS][SELW_T];
    __shared__ V tv[SELW_WARPS][SELW_T];
    const int l = lane_id(), w = threadIdx.x >> 5;
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
    const i64 lo = rg.begin(), count = rg.end();
    unsigned long long pb = 0;
    for (i64 x = lo + gw; x < count; x += nw) {
        i32 i = rg.list[x];
        if (a.dest[i] == NO_MOVE) {
            pb += sel_bytes(a, 0, false);
            continue;
        }
        VCtx vc = sel_prologue(a, i);
        i64 b = a.g.rowptr[i], e = a.g.rowptr[i + 1];
        if (sel_no_candidate(a, i, vc)) e = b;
        pb += sel_bytes(a, e - b, true);
        Best best = none_best();
        if (a.initial) {
            for (i64 j = b + l; j < e; j += 32) sel_eval<W, CON>(a, vc, a.g.col[j], V(a.g.wgt(j)), best);
        } else if (e - b <= 32) {
            i64 j = b + l;
            bool valid = j < e;
            i32 c = valid ? a.part[a.g.col[j]] : -1;
            W wr = valid ? a.g.wgt(j) : W(0);
            bool keep = valid && c != vc.p;
            i32 key = keep ? c : (i32)(0x80000000u | l);
            unsigned peers = __match_any_sync(FULL, key);
            bool leader = keep && ((peers & lanemask_lt()) == 0);
            V s = peer_sum<W>(a, peers, wr, keep, leader);
            if (leader) sel_eval<W, CON>(a, vc, c, s, best);
        } else {
            u32 T = sel_table_slots(a, e - b);
            i32* keys = tk[w];
            V* vals = tv[w];
            for (u32 s = l; s < T; s += 32) {
                keys[s] = -1;
                vals[s] = V(0);
            }
            __syncwarp();
            for (i64 j = b + l; j - l < e; j += 32) chunk_to_table(a, vc, j, e, keys, vals, T - 1);
            __syncwarp();
            for (u32 s = l; s < T; s += 32) {
                i32 c = keys[s];
                if (c != -1) sel_eval<W, CON>(a, vc, c, vals[s], best);
            }
            __syncwarp();
        }
        warp_best(best);
        if (l == 0) sel_finish(a, i, vc, best);
    }
    if (a.prof && l == 0 && pb) atomicAdd(a.prof, pb);
}

// ---- degree classes ---------------------------------------------------------
// All vertices are split by degree into class 0 (<= 8), 1 (<= 16), 2 (<= 32),
// 3 (< 128: order1 bucket 0), 4 (<= 1024), 5 (<= 4096) and 6 (above), so that
// a warp can serve 4, 2 or 1 low-degree vertices at once and the block
// kernels get shared tables sized to their class (2048 or 8192 slots).  Order
// inside a class is irrelevant: every consumer treats vertices independently.
__device__ __forceinline__ int deg_class(i64 d) {
    return d <= 8 ? 0 : d <= 16 ? 1 : d <= 32 ? 2 : d < LARGE_CUTOFF ? 3 : d <= 1024 ? 4 : d <= HUGE_DEG ? 5 : 6;
}


__global__ void k_class_count(const i32* list, i64 count, const i64* rowptr, unsigned long long* cnt) {
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
    const int l = lane_id();
    for (i64 x0 = gw * 32; x0 < count; x0 += nw * 32) {
        i64 x = x0 + l;
        int k = -1;
        if (x < count) {
            i32 i = list[x];
            k = deg_class(rowptr[i + 1] - rowptr[i]);
        }
        for (int c = 0; c < NCLS; c++) {
            unsigned m = __ballot_sync(FULL, k == c);
            if (l == 0 && m) atomicAdd(&cnt[c], (unsigned long long)__popc(m));
        }
    }
}
__global__ void k_class_offsets(unsigned long long* cnt, i64* off) {
    i64 s = 0;
    for (int c = 0; c < NCLS; c++) {
        off[c] = s;
        i64 v = (i64)cnt[c];
        cnt[NCLS + c] = (unsigned long long)s;  // scatter cursor
        s += v;
    }
    off[NCLS] = s;
}
__global__ void k_class_scatter(const i32* list, i64 count, const i64* rowptr, unsigned long long* cnt, i32* out) {
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
    const int l = lane_id();
    for (i64 x0 = gw * 32; x0 < count; x0 += nw * 32) {
        i64 x = x0 + l;
        int k = -1;
        i32 i = -1;
        if (x < count) {
            i = list[x];
            k = deg_class(rowptr[i + 1] - rowptr[i]);
        }
        for (int c = 0; c < NCLS; c++) {
            unsigned m = __ballot_sync(FULL, k == c);
            unsigned long long base = 0;
            if (l == 0 && m) base = atomicAdd(&cnt[NCLS + c], (unsigned long long)__popc(m));
            base = __shfl_sync(FULL, base, 0);
            if (k == c) out[base + __popc(m & lanemask_lt())] = i;
        }
    }
}

// Builds the class lists of all vertices into cl's arrays (list: ord.n
// entries, off: NCLS + 1, cnt: 2 * NCLS).
inline void build_class_lists_into(Context& ctx, const i64* rowptr, const Ordering& ord, ClassLists& cl) {
    cl.count = ord.n;
    PGGC_CUDA(cudaMemsetAsync(cl.cnt, 0, sizeof(unsigned long long) * 2 * NCLS, ctx.stream));
    int grid = (int)std::max<i64>(1, std::min<i64>(ceil_div(std::max<i64>(cl.count, 1), 256), (i64)ctx.num_sms * 8));
    if (cl.count > 0) {
        k_class_count<<<grid, 256, 0, ctx.stream>>>(ord.order1.p, cl.count, rowptr, cl.cnt);
        PGGC_LAUNCH_CHECK();
    }
    k_class_offsets<<<1, 1, 0, ctx.stream>>>(cl.cnt, cl.off);
    PGGC_LAUNCH_CHECK();
    if (cl.count > 0) {
        k_class_scatter<<<grid, 256, 0, ctx.stream>>>(ord.order1.p, cl.count, rowptr, cl.cnt, cl.list);
        PGGC_LAUNCH_CHECK();
    }
}

// The graph's class lists (built on first use, kept with the graph).
template <class W>
ClassLists graph_class_lists(Context& ctx, const Graph<W>& g, const Ordering& ord) {
    GraphCache& c = *g.cache;
    std::lock_guard<std::mutex> lk(c.mu);
    ClassLists cl;
    if (!c.cls_ok) {
        c.cls_list = DBuf<i32>(ctx, std::max<i64>(ord.n, 1));
        c.cls_off = DBuf<i64>(ctx, NCLS + 1);
        c.cls_cnt = DBuf<unsigned long long>(ctx, 2 * NCLS);
        cl.list = c.cls_list.p;
        cl.off = c.cls_off.p;
        cl.cnt = c.cls_cnt.p;
        build_class_lists_into(ctx, g.view().rowptr, ord, cl);
        ctx.sync();  // other streams may read them next
        c.cls_ok = true;
    }
    cl.list = c.cls_list.p;
    cl.off = c.cls_off.p;
    cl.cnt = c.cls_cnt.p;
    cl.count = ord.n;
    return cl;
}

template <int G>
__device__ __forceinline__ void group_best(Best& b) {
    const unsigned mask = G == 32 ? FULL : (((1u << G) - 1u) << (lane_id() & ~(G - 1)));
    reduce_best(b, mask);
}

// G-lane groups, one vertex each, for vertices of degree <= G (single chunk):
// class k of the class lists.  Each group takes UV vertices per iteration and
// issues their loads together (the chains list -> row -> column -> label ->
// volume are latency-bound, so independent vertices in flight set the pace).
template <class W, bool CON, int G, int UV = 2>
__global__ void __launch_bounds__(256) k_select_grp(SelArgs<W> a, const i32* cls, const i64* off, int k) {
    using V = typename Traits<W>::V;
    constexpr int NG = 32 / G;
    const int l = lane_id(), r = l & (G - 1), grp = l / G;
    const i64 lo = off[k], hi = off[k + 1];
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
    unsigned long long pb = 0;
    for (i64 base = lo + gw * NG * UV; base < hi; base += nw * NG * UV) {
        i32 iv[UV];
        bool act[UV];
#pragma unroll
        for (int u = 0; u < UV; u++) {
            const i64 x = base + u * NG + grp;
            iv[u] = x < hi ? cls[x] : -1;
        }
#pragma unroll
        for (int u = 0; u < UV; u++) act[u] = iv[u] >= 0 && a.dest[iv[u]] != NO_MOVE;
        VCtx vc[UV];
        i64 b[UV], e[UV];
#pragma unroll
        for (int u = 0; u < UV; u++) {
            b[u] = 0;
            e[u] = 0;
            vc[u] = VCtx{};
            if (act[u]) {
                vc[u] = sel_prologue(a, iv[u]);
                b[u] = a.g.rowptr[iv[u]];
                e[u] = sel_no_candidate(a, iv[u], vc[u]) ? b[u] : a.g.rowptr[iv[u] + 1];
            }
            if (r == 0 && iv[u] >= 0) pb += sel_bytes(a, e[u] - b[u], act[u]);
        }
        if (a.initial) {
#pragma unroll
            for (int u = 0; u < UV; u++) {
                Best best = none_best();
                const i64 j = b[u] + r;
                if (act[u] && j < e[u]) sel_eval<W, CON>(a, vc[u], a.g.col[j], V(a.g.wgt(j)), best);
                group_best<G>(best);
                if (r == 0 && act[u]) sel_finish(a, iv[u], vc[u], best);
            }
        } else {
            i32 c[UV];
            W wv[UV];
#pragma unroll
            for (int u = 0; u < UV; u++) {
                const i64 j = b[u] + r;
                const bool valid = act[u] && j < e[u];
                c[u] = valid ? a.g.col[j] : -1;
                wv[u] = valid ? a.g.wgt(j) : W(0);
            }
#pragma unroll
            for (int u = 0; u < UV; u++) c[u] = c[u] >= 0 ? a.part[c[u]] : -1;
#pragma unroll
            for (int u = 0; u < UV; u++) {
                Best best = none_best();
                const bool keep = c[u] >= 0 && c[u] != vc[u].p;
                unsigned peers;
                if (a.keys32) {
                    // bit 31 marks lanes without a candidate (unique per lane),
                    // bits 29-30 the group
                    const u32 key = keep ? (((u32)grp << 29) | (u32)c[u]) : (0x80000000u | (u32)l);
                    peers = __match_any_sync(FULL, key);
                } else {
                    const u64 key = keep ? (((u64)grp << 32) | (u64)(u32)c[u]) : (0xFFFFFFFF00000000ull | (u64)l);
                    peers = __match_any_sync(FULL, key);
                }
                bool leader = keep && ((peers & lanemask_lt()) == 0);
                V sum = peer_sum<W>(a, peers, wv[u], keep, leader);
                if (leader) sel_eval<W, CON>(a, vc[u], c[u], sum, best);
                group_best<G>(best);
                if (r == 0 && act[u]) sel_finish(a, iv[u], vc[u], best);
            }
        }
    }
    if (a.prof) {
        pb = (unsigned long long)warp_sum_i64((i64)pb);
        if (l == 0 && pb) atomicAdd(a.prof, pb);
    }
}

// One thread per vertex for vertices of degree <= K (classes 0 and 1): the
// row sits in registers, equal neighbour clusters are merged by pairwise
// compares and summed from 0 in edge order -- the order of the lane-order
// group sum, so the gains are bit-identical -- and the best cluster is kept
// under the same total order (gain, then smaller id).  No shuffles or match
// instructions: the warp's 32 vertices are independent load chains.
template <class W, bool CON, int K>
__global__ void __launch_bounds__(256) k_select_thr(SelArgs<W> a, const i32* cls, const i64* off, int k) {
    using V = typename Traits<W>::V;
    const i64 lo = off[k], hi = off[k + 1];
    unsigned long long pb = 0;
    for (i64 x = lo + blockIdx.x * (i64)blockDim.x + threadIdx.x; x < hi; x += (i64)gridDim.x * blockDim.x) {
        const i32 i = cls[x];
        if (a.dest[i] == NO_MOVE) {
            pb += sel_bytes(a, 0, false);
            continue;
        }
        const VCtx vc = sel_prologue(a, i);
        const i64 b = a.g.rowptr[i];
        i64 e = a.g.rowptr[i + 1];
        if (sel_no_candidate(a, i, vc)) e = b;
        const int d = (int)(e - b);
        pb += sel_bytes(a, d, true);
        Best best = none_best();
        i32 c[K];
#pragma unroll
        for (int t = 0; t < K; t++) c[t] = t < d ? a.g.col[b + t] : -1;
        if (a.initial) {
#pragma unroll
            for (int t = 0; t < K; t++)
                if (t < d) sel_eval<W, CON>(a, vc, c[t], V(a.g.wgt(b + t)), best);
        } else {
#pragma unroll
            for (int t = 0; t < K; t++) c[t] = c[t] >= 0 ? a.part[c[t]] : -1;
            // weights are read where they are summed (the row is in L1)
#pragma unroll
            for (int t = 0; t < K; t++) {
                bool first = c[t] >= 0 && c[t] != vc.p;
#pragma unroll
                for (int m = 0; m < t; m++) first = first && c[m] != c[t];
                if (first) {
                    V sum = V(0);
#pragma unroll
                    for (int m = t; m < K; m++)
                        if (c[m] == c[t]) sum = sum + V(a.g.wgt(b + m));
                    sel_eval<W, CON>(a, vc, c[t], sum, best);
                }
            }
        }
        sel_finish(a, i, vc, best);
    }
    if (a.prof) {
        pb = (unsigned long long)warp_sum_i64((i64)pb);
        if (lane_id() == 0 && pb) atomicAdd(a.prof, pb);
    }
}

// ---- block per vertex, shared or global table -------------------------------
// With OVF (vertices above HUGE_DEG, shared tables of gcap slots that may be
// smaller than 2 * degree), a vertex whose distinct neighbour clusters do not
// fit is appended to `ovf_list` for the global-table pass instead.
template <class W, bool CON, bool GLOBAL, int THREADS = 256, bool OVF = false>
__global__ void __launch_bounds__(THREADS) k_select_block(SelArgs<W> a, Range rg, i32* gkeys,
                                                          typename Traits<W>::V* gvals, i64 gcap,
                                                          i32* ovf_list = nullptr, i64* ovf_count = nullptr) {
    using V = typename Traits<W>::V;
    constexpr int NW = THREADS / 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ Best wb[NW];
    __shared__ int full;
    V* svals = (V*)smem_raw;
    i32* skeys = (i32*)(smem_raw + sizeof(V) * (GLOBAL ? 0 : gcap));  // gcap = shared table slots
    const int l = lane_id(), w = threadIdx.x >> 5;
    i32* keys = GLOBAL ? gkeys + (i64)blockIdx.x * gcap : skeys;
    V* vals = GLOBAL ? gvals + (i64)blockIdx.x * gcap : svals;
    unsigned long long pb = 0;
    const i64 lo = rg.begin(), count = rg.end();
    for (i64 x = lo + blockIdx.x; x < count; x += gridDim.x) {
        i32 i = rg.list[x];
        i64 b = a.g.rowptr[i], e = a.g.rowptr[i + 1];
        if (!GLOBAL && !OVF && e - b > HUGE_DEG) continue;
        if (a.dest[i] == NO_MOVE) {
            pb += sel_bytes(a, 0, false);
            continue;
        }
        VCtx vc = sel_prologue(a, i);
        if (sel_no_candidate(a, i, vc)) e = b;
        Best best = none_best();
        if (a.initial) {
            for (i64 j = b + threadIdx.x; j < e; j += THREADS)
                sel_eval<W, CON>(a, vc, a.g.col[j], V(a.g.wgt(j)), best);
        } else if (!GLOBAL && a.dense) {
            // dense table: slot = cluster id (every label fits the shared
            // table); a cluster is present when its weight sum is positive,
            // the only sums sel_eval accepts
            const i64 L = *a.label_count;
            for (i64 s = threadIdx.x; s < L; s += THREADS) vals[s] = V(0);
            __syncthreads();
            for (i64 j = b + (i64)w * 32 + l; j - l < e; j += THREADS) {
                const bool valid = j < e;
                const i32 c = valid ? a.part[a.g.col[j]] : -1;
                const W wr = valid ? a.g.wgt(j) : W(0);
                const bool keep = valid && c != vc.p;
                const i32 key = keep ? c : (i32)(0x80000000u | l);
                const unsigned peers = __match_any_sync(FULL, key);
                const bool leader = keep && ((peers & lanemask_lt()) == 0);
                const V sum = peer_sum<W>(a, peers, wr, keep, leader);
                if (leader) vatomic_add(&vals[c], sum);
            }
            __syncthreads();
            for (i64 s = threadIdx.x; s < L; s += THREADS) {
                const V x = vals[s];
                if (x > V(0)) sel_eval<W, CON>(a, vc, (i32)s, x, best);
            }
        } else {
            i64 U = min(e - b, *a.label_count);
            u32 T = sel_table_slots(a, U);
            if (T > (u32)gcap) T = (u32)gcap;
            for (u32 s = threadIdx.x; s < T; s += THREADS) {
                keys[s] = -1;
                vals[s] = V(0);
            }
            if (OVF && threadIdx.x == 0) full = 0;
            __syncthreads();
            if (OVF) {
                for (i64 j = b + (i64)w * 32 + l; j - l < e; j += THREADS) {
                    if (!chunk_to_table_try(a, vc, j, e, keys, vals, T - 1)) full = 1;
                    if (__any_sync(FULL, *(volatile int*)&full != 0)) break;
                }
                __syncthreads();
                if (full) {
                    if (threadIdx.x == 0) {
                        i64 k = (i64)atomicAdd((unsigned long long*)ovf_count, 1ull);
                        ovf_list[k] = i;
                    }
                    __syncthreads();
                    continue;
                }
            } else {
                for (i64 j = b + (i64)w * 32 + l; j - l < e; j += THREADS)
                    chunk_to_table(a, vc, j, e, keys, vals, T - 1);
            }
            __syncthreads();
            for (u32 s = threadIdx.x; s < T; s += THREADS) {
                i32 c = keys[s];
                if (c != -1) sel_eval<W, CON>(a, vc, c, vals[s], best);
            }
        }
        pb += sel_bytes(a, e - b, true);
        warp_best(best);
        if (l == 0) wb[w] = best;
        __syncthreads();
        if (w == 0) {
            best = l < NW ? wb[l] : none_best();
            warp_best(best);
            if (l == 0) sel_finish(a, i, vc, best);
        }
        __syncthreads();
    }
    if (a.prof && threadIdx.x == 0 && pb) atomicAdd(a.prof, pb);
}

// ---- vertices whose distinct neighbour clusters overflow a 16384-slot shared
// table: the row is split across blocks ------------------------------------------
// Four launches per round of up to `count` such vertices, each vertex owning a
// global table of `gcap` slots: clear the tables; insert, one block per chunk of
// SPLIT_CHUNK edges (the chunk's columns and weights staged in shared memory by
// a TMA bulk copy, cp.async.bulk, from this GPU's own memory); scan, blocks over
// table slots with a packed 64-bit atomicMax of (gain, ~cluster) per vertex --
// the (larger gain, then smaller id) order of `better`; finish, one thread per
// vertex.  Sums are the exact table sums of the single-block pass, so the
// result is the same.
constexpr int SPLIT_CHUNK = 8192;
constexpr int SPLIT_THREADS = 256;
constexpr size_t SPLIT_SMEM = 16 + 2 * sizeof(i32) * (SPLIT_CHUNK + 4);
__device__ __forceinline__ unsigned long long pack_best(const Best& b) {
    return ((unsigned long long)f2ord(b.jc) << 32) | (unsigned long long)(~(u32)b.c);
}
__device__ __forceinline__ Best unpack_best(unsigned long long k) {
    return Best{ord2f((u32)(k >> 32)), (i32)(~(u32)(k & 0xFFFFFFFFull))};
}

template <class W>
__global__ void k_split_clear(SelArgs<W> a, const i32* list, i64 count, i64 gcap, i32* keys,
                              typename Traits<W>::V* vals, unsigned long long* best) {
    using V = typename Traits<W>::V;
    const i64 total = count * gcap;
    for (i64 x = blockIdx.x * (i64)blockDim.x + threadIdx.x; x < total; x += (i64)gridDim.x * blockDim.x) {
        keys[x] = -1;
        vals[x] = V(0);
    }
    for (i64 k = blockIdx.x * (i64)blockDim.x + threadIdx.x; k < count; k += (i64)gridDim.x * blockDim.x) best[k] = 0;
}

template <class W>
__global__ void __launch_bounds__(SPLIT_THREADS) k_split_insert(SelArgs<W> a, const i32* list, i64 count, i64 gcap,
                                                               i32* gkeys, typename Traits<W>::V* gvals) {
    using V = typename Traits<W>::V;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned long long* bar = (unsigned long long*)smem_raw;
    i32* s_col = (i32*)(smem_raw + 16);
    W* s_w = (W*)(smem_raw + 16 + sizeof(i32) * (SPLIT_CHUNK + 4));
    const i64 k = blockIdx.y;
    if (k >= count) return;
    const i32 i = list[k];
    const i64 b = a.g.rowptr[i], e = a.g.rowptr[i + 1];
    const i64 j0 = b + (i64)blockIdx.x * SPLIT_CHUNK;
    if (j0 >= e) return;
    const i64 j1 = min(e, j0 + (i64)SPLIT_CHUNK);
    const VCtx vc = sel_prologue(a, i);
    if (sel_no_candidate(a, i, vc)) return;
    const i64 U = min(e - b, *a.label_count);
    u32 T = sel_table_slots(a, U);
    if (T > (u32)gcap) T = (u32)gcap;
    i32* keys = gkeys + k * gcap;
    V* vals = gvals + k * gcap;
    // stage the chunk's columns (and weights) in shared memory
    const bool has_w = a.g.w != nullptr;
    const i64 lo16 = j0 & ~(i64)3;
    if (!stage_rows(a.g.col, has_w ? a.g.w : (const W*)nullptr, j0, j1, s_col, s_w, bar, a.err)) return;
    const int l = lane_id(), w = threadIdx.x >> 5;
    const i64 len = j1 - j0, base = j0 - lo16;
    for (i64 t = (i64)w * 32 + l; t - l < len; t += SPLIT_THREADS) {
        const bool valid = t < len;
        const i32 c = valid ? a.part[s_col[base + t]] : -1;
        const W wr = valid ? (has_w ? s_w[base + t] : W(1)) : W(0);
        const bool keep = valid && c != vc.p;
        const i32 key = keep ? c : (i32)(0x80000000u | l);
        const unsigned peers = __match_any_sync(FULL, key);
        const bool leader = keep && ((peers & lanemask_lt()) == 0);
        const V sum = peer_sum<W>(a, peers, wr, keep, leader);
        if (leader) table_add(keys, vals, T - 1, c, sum, a.err, a.probe_cap);
    }
}

template <class W, bool CON>
__global__ void __launch_bounds__(SPLIT_THREADS) k_split_scan(SelArgs<W> a, const i32* list, i64 count, i64 gcap,
                                                             const i32* gkeys, const typename Traits<W>::V* gvals,
                                                             unsigned long long* best) {
    __shared__ Best wb[SPLIT_THREADS / 32];
    const i64 k = blockIdx.y;
    if (k >= count) return;
    const i32 i = list[k];
    const i64 b = a.g.rowptr[i], e = a.g.rowptr[i + 1];
    const VCtx vc = sel_prologue(a, i);
    if (sel_no_candidate(a, i, vc)) return;
    const i64 U = min(e - b, *a.label_count);
    u32 T = sel_table_slots(a, U);
    if (T > (u32)gcap) T = (u32)gcap;
    const i32* keys = gkeys + k * gcap;
    const auto* vals = gvals + k * gcap;
    Best bst = none_best();
    for (i64 sl = blockIdx.x * (i64)SPLIT_THREADS + threadIdx.x; sl < T; sl += (i64)gridDim.x * SPLIT_THREADS) {
        const i32 c = keys[sl];
        if (c != -1) sel_eval<W, CON>(a, vc, c, vals[sl], bst);
    }
    warp_best(bst);
    const int l = lane_id(), w = threadIdx.x >> 5;
    if (l == 0) wb[w] = bst;
    __syncthreads();
    if (w == 0) {
        bst = l < SPLIT_THREADS / 32 ? wb[l] : none_best();
        warp_best(bst);
        if (l == 0 && bst.c != 2147483647) atomicMax(&best[k], pack_best(bst));
    }
}

template <class W>
__global__ void k_split_finish(SelArgs<W> a, const i32* list, i64 count, const unsigned long long* best) {
    for (i64 k = blockIdx.x * (i64)blockDim.x + threadIdx.x; k < count; k += (i64)gridDim.x * blockDim.x) {
        const i32 i = list[k];
        const VCtx vc = sel_prologue(a, i);
        const bool none = sel_no_candidate(a, i, vc) || best[k] == 0;
        const Best bst = none ? none_best() : unpack_best(best[k]);
        sel_finish(a, i, vc, bst);
        if (a.prof) {
            const i64 deg = none && sel_no_candidate(a, i, vc) ? 0 : a.g.rowptr[i + 1] - a.g.rowptr[i];
            atomicAdd(a.prof, sel_bytes(a, deg, true));
        }
    }
}

// ---------------------------------------------------------------------------
// own-cluster weights (pvals)
// ---------------------------------------------------------------------------
template <class W>
__device__ __forceinline__ typename Traits<W>::V own_warp(const DGraph<W>& g, const i32* lab, i32 i) {
    using V = typename Traits<W>::V;
    i64 b = g.rowptr[i], e = g.rowptr[i + 1];
    i32 li = lab[i];
    return VSum<V>::warp(b, e, [&](i64 j) -> V { return lab[g.col[j]] == li ? V(g.wgt(j)) : V(0); });
}

template <class W>
__device__ __forceinline__ typename Traits<W>::V own_block1024(const DGraph<W>& g, const i32* lab, i32 i, double* red) {
    using V = typename Traits<W>::V;
    i64 b = g.rowptr[i], e = g.rowptr[i + 1];
    i32 li = lab[i];
    if constexpr (std::is_same<V, double>::value) {
        return block1024_canon_sum(b, e, [&](i64 j) -> double { return lab[g.col[j]] == li ? (double)g.wgt(j) : 0.0; },
                                   red);
    } else {
        __shared__ unsigned long long acc;
        if (threadIdx.x == 0) acc = 0;
        __syncthreads();
        i64 s = 0;
        for (i64 j = b + threadIdx.x; j < e; j += 1024)
            if (lab[g.col[j]] == li) s += g.wgt(j);
        s = warp_sum_i64(s);
        if (lane_id() == 0) ::atomicAdd(&acc, (unsigned long long)s);
        __syncthreads();
        i64 r = (i64)acc;
        __syncthreads();
        return r;
    }
}

template <class W>
__global__ void __launch_bounds__(1024) k_own_massive(DGraph<W> g, const i32* lab, typename Traits<W>::V* out,
                                                      const i32* list, i64 count, int mode, unsigned char* flags,
                                                      i32* dest) {
    __shared__ double red[32];
    for (i64 x = blockIdx.x; x < count; x += gridDim.x) {
        i32 i = list[x];
        if (mode == 1 && !flags[i]) continue;
        auto r = own_block1024(g, lab, i, red);
        if (threadIdx.x == 0) {
            out[i] = r;
            if (mode == 1) {
                dest[i] = NULL_PART;
                flags[i] = 0;
            }
        }
        __syncthreads();
    }
}

// G-lane groups over a vertex range; mode 0: every vertex, mode 1: flagged
// vertices only (also resets their dest cache and clears the flag), mode 2:
// every vertex, resetting its dest cache (a list of affected vertices)
template <class W, int G>
__global__ void __launch_bounds__(256) k_own_grp(DGraph<W> g, const i32* lab, typename Traits<W>::V* out, Range rg,
                                                 int mode, unsigned char* flags, i32* dest,
                                                 unsigned long long* prof) {
    using V = typename Traits<W>::V;
    constexpr int NG = 32 / G;
    const int l = lane_id(), r = l & (G - 1), grp = l / G;
    const i64 lo = rg.begin(), hi = rg.end();
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
    unsigned long long pb = 0;
    for (i64 base = lo + gw * NG; base < hi; base += nw * NG) {
        const i64 x = base + grp;
        i32 i = -1;
        bool act = false;
        if (x < hi) {
            i = rg.list[x];
            act = mode != 1 || flags[i];
        }
        i64 b = 0, e = 0;
        i32 li = 0;
        if (act) {
            b = g.rowptr[i];
            e = g.rowptr[i + 1];
            li = lab[i];
        }
        V v = group_vsum<G, V>(b, e, r, [&](i64 j) -> V { return lab[g.col[j]] == li ? V(g.wgt(j)) : V(0); });
        if (r == 0 && act) {
            out[i] = v;
            if (mode == 1) {
                dest[i] = NULL_PART;
                flags[i] = 0;
            } else if (mode == 2) {
                dest[i] = NULL_PART;
            }
            // list entry, offsets, own label, result; per edge column, weight, label
            pb += 4 + 16 + 4 + sizeof(V) + (unsigned long long)(e - b) * (8 + (g.w ? sizeof(W) : 0));
        }
    }
    if (prof) {
        pb = (unsigned long long)warp_sum_i64((i64)pb);
        if (l == 0 && pb) atomicAdd(prof, pb);
    }
}

// Own-cluster weights of vertices of degree <= K * G: lane r of a G-lane group
// adds the terms of edges r, r + G, ... (at most K) in that order, then the
// group's xor butterfly -- the canonical association.  Each group takes UV
// vertices per iteration and issues their loads together.
template <class W, int G, int K, int UV = 2>
__global__ void __launch_bounds__(256) k_own_small(DGraph<W> g, const i32* lab, typename Traits<W>::V* out, Range rg,
                                                   int mode, unsigned char* flags, i32* dest,
                                                   unsigned long long* prof) {
    using V = typename Traits<W>::V;
    constexpr int NG = 32 / G;
    const int l = lane_id(), r = l & (G - 1), grp = l / G;
    const i64 lo = rg.begin(), hi = rg.end();
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
    unsigned long long pb = 0;
    for (i64 base = lo + gw * NG * UV; base < hi; base += nw * NG * UV) {
        i32 iv[UV];
        bool act[UV];
#pragma unroll
        for (int u = 0; u < UV; u++) {
            const i64 x = base + u * NG + grp;
            iv[u] = x < hi ? rg.list[x] : -1;
        }
#pragma unroll
        for (int u = 0; u < UV; u++) act[u] = iv[u] >= 0 && (mode == 0 || flags[iv[u]]);
        i64 b[UV], e[UV];
        i32 li[UV];
#pragma unroll
        for (int u = 0; u < UV; u++) {
            b[u] = act[u] ? g.rowptr[iv[u]] : 0;
            e[u] = act[u] ? g.rowptr[iv[u] + 1] : 0;
            li[u] = act[u] ? lab[iv[u]] : 0;
        }
        i32 cv[UV][K];
        V wv[UV][K];
#pragma unroll
        for (int u = 0; u < UV; u++)
#pragma unroll
            for (int t = 0; t < K; t++) {
                const i64 j = b[u] + r + (i64)t * G;
                const bool valid = j < e[u];
                cv[u][t] = valid ? g.col[j] : -1;
                wv[u][t] = valid ? V(g.wgt(j)) : V(0);
            }
#pragma unroll
        for (int u = 0; u < UV; u++)
#pragma unroll
            for (int t = 0; t < K; t++) cv[u][t] = cv[u][t] >= 0 ? lab[cv[u][t]] : -1;
#pragma unroll
        for (int u = 0; u < UV; u++) {
            V acc = V(0);
#pragma unroll
            for (int t = 0; t < K; t++)
                if (b[u] + r + (i64)t * G < e[u]) acc += cv[u][t] == li[u] ? wv[u][t] : V(0);
#pragma unroll
            for (int d = G / 2; d >= 1; d >>= 1) acc = acc + __shfl_xor_sync(FULL, acc, d);
            if (r == 0 && act[u]) {
                out[iv[u]] = acc;
                if (mode == 1) {
                    dest[iv[u]] = NULL_PART;
                    flags[iv[u]] = 0;
                }
                pb += 4 + 16 + 4 + sizeof(V) + (unsigned long long)(e[u] - b[u]) * (8 + (g.w ? sizeof(W) : 0));
            }
        }
    }
    if (prof) {
        pb = (unsigned long long)warp_sum_i64((i64)pb);
        if (l == 0 && pb) atomicAdd(prof, pb);
    }
}

// Own-cluster weights of vertices of degree <= 2H (H = 8: classes 0 and 1;
// H = 16: class 2), one thread per vertex, the association of
// k_own_small<W, H, 2> (canon_tree): no shuffles, 32 independent vertices
// per warp.
template <class W, int H>
__global__ void __launch_bounds__(256) k_own_thr(DGraph<W> g, const i32* lab, typename Traits<W>::V* out, Range rg,
                                                 int mode, unsigned char* flags, i32* dest,
                                                 unsigned long long* prof) {
    using V = typename Traits<W>::V;
    const i64 lo = rg.begin(), hi = rg.end();
    unsigned long long pb = 0;
    for (i64 x = lo + blockIdx.x * (i64)blockDim.x + threadIdx.x; x < hi; x += (i64)gridDim.x * blockDim.x) {
        const i32 i = rg.list[x];
        if (mode == 1 && !flags[i]) continue;
        const i64 b = g.rowptr[i], e = g.rowptr[i + 1];
        const i32 li = lab[i];
        i32 cv[2 * H];
#pragma unroll
        for (int t = 0; t < 2 * H; t++) cv[t] = b + t < e ? g.col[b + t] : -1;
#pragma unroll
        for (int t = 0; t < 2 * H; t++) cv[t] = cv[t] >= 0 ? lab[cv[t]] : -1;
        // weights are read only for own-cluster edges (the row is in L1)
        V acc[H];
#pragma unroll
        for (int r = 0; r < H; r++) {
            acc[r] = V(0);
            if (b + r < e) acc[r] += cv[r] == li ? V(g.wgt(b + r)) : V(0);
            if (b + r + H < e) acc[r] += cv[r + H] == li ? V(g.wgt(b + r + H)) : V(0);
        }
        out[i] = canon_tree<H, V>(acc);
        if (mode == 1) {
            dest[i] = NULL_PART;
            flags[i] = 0;
        }
        pb += 4 + 16 + 4 + sizeof(V) + (unsigned long long)(e - b) * (8 + (g.w ? sizeof(W) : 0));
    }
    if (prof) {
        pb = (unsigned long long)warp_sum_i64((i64)pb);
        if (lane_id() == 0 && pb) atomicAdd(prof, pb);
    }
}

template <class W>
void own_weights_impl(Context& ctx, const Graph<W>& g, const Ordering& ord, const i32* lab,
                      typename Traits<W>::V* out, int mode, unsigned char* flags, i32* dest,
                      const ClassLists* cls = nullptr) {
    auto gv = g.view();
    if (g.n == 0) return;
    ProfScope ps(ctx, "own_weights");
    unsigned long long* prof = ctx.prof_counter("own_weights");
    ClassLists local;
    if (!cls) {
        local = graph_class_lists<W>(ctx, g, ord);
        cls = &local;
    }
    const i64 c01 = cls->count;  // host upper bound of every class range
    if (c01 > 0) {
        int grid = (int)std::max<i64>(1, std::min<i64>(ceil_div(c01, 32), (i64)ctx.num_sms * 16));
        int grid_t = (int)std::max<i64>(1, std::min<i64>(ceil_div(c01, 256), (i64)ctx.num_sms * 16));
        k_own_thr<W, 8><<<grid_t, 256, 0, ctx.stream>>>(gv, lab, out, dev_range(cls->list, cls->off + 0, cls->off + 2),
                                                        mode, flags, dest, prof);
        PGGC_LAUNCH_CHECK();
        k_own_thr<W, 16><<<grid_t, 256, 0, ctx.stream>>>(gv, lab, out, dev_range(cls->list, cls->off + 2, cls->off + 3),
                                                         mode, flags, dest, prof);
        PGGC_LAUNCH_CHECK();
        k_own_small<W, 32, 4><<<grid, 256, 0, ctx.stream>>>(gv, lab, out,
                                                             dev_range(cls->list, cls->off + 3, cls->off + 4), mode,
                                                             flags, dest, prof);
        PGGC_LAUNCH_CHECK();
    }
    if (ord.off_large2 > ord.off_large) {
        int grid = (int)std::max<i64>(1, std::min<i64>(ceil_div(ord.off_large2 - ord.off_large, 8), (i64)ctx.num_sms * 16));
        k_own_grp<W, 32><<<grid, 256, 0, ctx.stream>>>(gv, lab, out,
                                                        host_range(ord.order1.p, ord.off_large, ord.off_large2), mode,
                                                        flags, dest, prof);
        PGGC_LAUNCH_CHECK();
    }
    i64 nm = g.n - ord.off_large2;
    if (nm > 0) {
        int gb = (int)std::min<i64>(nm, (i64)ctx.num_sms * 2);
        k_own_massive<W><<<gb, 1024, 0, ctx.stream>>>(gv, lab, out, ord.order1.p + ord.off_large2, nm, mode, flags,
                                                       dest);
        PGGC_LAUNCH_CHECK();
    }
}

// Own-cluster weights of a device list of vertices below MASSIVE_CUTOFF (at
// most `bound` entries, count in *d_count), warp per vertex (the 32-lane
// canonical association, equal to the class kernels' for every degree), then
// the flagged massive vertices; resets the dest cache of every one.
template <class W>
void own_weights_list(Context& ctx, const Graph<W>& g, const Ordering& ord, const i32* lab,
                      typename Traits<W>::V* out, const i32* list, const i64* d_count, i64 bound,
                      unsigned char* flags, i32* dest) {
    auto gv = g.view();
    ProfScope ps(ctx, "own_weights");
    unsigned long long* prof = ctx.prof_counter("own_weights");
    const int grid = (int)std::max<i64>(1, std::min<i64>(ceil_div(std::max<i64>(bound, 1), 8), (i64)ctx.num_sms * 16));
    k_own_grp<W, 32><<<grid, 256, 0, ctx.stream>>>(gv, lab, out, Range{list, nullptr, d_count, 0, 0}, 2, nullptr, dest,
                                                    prof);
    PGGC_LAUNCH_CHECK();
    const i64 nm = g.n - ord.off_large2;
    if (nm > 0) {
        int gb = (int)std::min<i64>(nm, (i64)ctx.num_sms * 2);
        k_own_massive<W><<<gb, 1024, 0, ctx.stream>>>(gv, lab, out, ord.order1.p + ord.off_large2, nm, 1, flags, dest);
        PGGC_LAUNCH_CHECK();
    }
}

template <class W>
void own_weights(Context& ctx, const Graph<W>& g, const Ordering& ord, const i32* labels, typename Traits<W>::V* out) {
    own_weights_impl<W>(ctx, g, ord, labels, out, 0, nullptr, nullptr);
}

// ---------------------------------------------------------------------------
// afterburner (src/local_mover.cpp:280-433)
// ---------------------------------------------------------------------------
template <class W>
struct ABArgs {
    using V = typename Traits<W>::V;
    DGraph<W> g;
    const i32* part;
    const i32* dest;
    const float* gain;
    float pm;
    const i32* cand;
    unsigned char* keep;
    const LMScalars<V>* sc;
    unsigned long long* prof;
};

// algorithmic bytes of one afterburner evaluation: candidate entry, its
// dest/part/vtx_w/gain, rowptr pair, keep flag; per edge column, weight, gain[v]
template <class W>
__device__ __forceinline__ unsigned long long ab_bytes(const ABArgs<W>& a, i64 deg) {
    const unsigned long long wb = a.g.w ? sizeof(W) : 0;
    return 41ull + (unsigned long long)deg * (8ull + wb);
}

template <class W>
__device__ __forceinline__ double ab_term(const ABArgs<W>& a, i64 j, i32 p, i32 best, float multi, float igain,
                                          i32 hi) {
    i32 v = a.g.col[j];
    float vgain = a.gain[v];
    float d = vgain - igain;
    if (d >= AFTERBURNER_EPS || (fabsf(d) < AFTERBURNER_EPS && (i32)xorshift32((u32)v) < hi)) {
        float q = (float)a.g.wgt(j) - multi * to_f(a.g.vtx_w[v]);
        int coef = 0;
        i32 vp = a.dest[v];
        if (vp == p) coef--;
        if (vp == best && best != NEW_PART) coef++;
        vp = a.part[v];
        if (vp == p) coef++;
        if (vp == best) coef--;
        return (double)coef * (double)q;
    }
    return 0.0;
}

// candidates (dest != NO_MOVE) of a vertex range, G-lane groups; keep is
// indexed by vertex
template <class W, int G>
__global__ void __launch_bounds__(256) k_afterburner_grp(ABArgs<W> a, Range rg) {
    constexpr int NG = 32 / G;
    const int l = lane_id(), r = l & (G - 1), grp = l / G;
    const i64 lo = rg.begin(), hi = rg.end();
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
    unsigned long long pb = 0;
    for (i64 base = lo + gw * NG; base < hi; base += nw * NG) {
        const i64 x = base + grp;
        i32 i = -1;
        bool act = false;
        if (x < hi) {
            i = rg.list[x];
            act = a.dest[i] != NO_MOVE;
        }
        i32 best = 0, p = 0, hv = 0;
        float multi = 0.f, igain = 0.f;
        i64 b = 0, e = 0;
        if (act) {
            best = a.dest[i];
            p = a.part[i];
            multi = to_f(a.g.vtx_w[i]) * a.pm;
            igain = a.gain[i];
            hv = (i32)xorshift32((u32)i);
            b = a.g.rowptr[i];
            e = a.g.rowptr[i + 1];
        }
        double ch = group_vsum<G, double>(b, e, r, [&](i64 j) { return ab_term(a, j, p, best, multi, igain, hv); });
        if (r == 0 && act) {
            a.keep[i] = (igain + (float)ch) >= 0.0f ? 1 : 0;
            pb += ab_bytes(a, e - b);
        }
    }
    if (a.prof) {
        pb = (unsigned long long)warp_sum_i64((i64)pb);
        if (l == 0 && pb) atomicAdd(a.prof, pb);
    }
}

// Afterburner for candidates of degree <= K * G, UV vertices per group per
// iteration, canonical association as in k_own_small.
template <class W, int G, int K, int UV = 2>
__global__ void __launch_bounds__(256) k_afterburner_small(ABArgs<W> a, Range rg) {
    constexpr int NG = 32 / G;
    const int l = lane_id(), r = l & (G - 1), grp = l / G;
    const i64 lo = rg.begin(), hi = rg.end();
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
    unsigned long long pb = 0;
    for (i64 base = lo + gw * NG * UV; base < hi; base += nw * NG * UV) {
        i32 iv[UV], bestv[UV], pv[UV], hv[UV];
        bool act[UV];
        float multi[UV], igain[UV];
        i64 b[UV], e[UV];
#pragma unroll
        for (int u = 0; u < UV; u++) {
            const i64 x = base + u * NG + grp;
            iv[u] = x < hi ? rg.list[x] : -1;
        }
#pragma unroll
        for (int u = 0; u < UV; u++) {
            bestv[u] = iv[u] >= 0 ? a.dest[iv[u]] : NO_MOVE;
            act[u] = bestv[u] != NO_MOVE;
        }
#pragma unroll
        for (int u = 0; u < UV; u++) {
            pv[u] = act[u] ? a.part[iv[u]] : 0;
            multi[u] = act[u] ? to_f(a.g.vtx_w[iv[u]]) * a.pm : 0.f;
            igain[u] = act[u] ? a.gain[iv[u]] : 0.f;
            hv[u] = act[u] ? (i32)xorshift32((u32)iv[u]) : 0;
            b[u] = act[u] ? a.g.rowptr[iv[u]] : 0;
            e[u] = act[u] ? a.g.rowptr[iv[u] + 1] : 0;
        }
        double acc[UV];
#pragma unroll
        for (int u = 0; u < UV; u++) {
            acc[u] = 0.0;
#pragma unroll
            for (int t = 0; t < K; t++) {
                const i64 j = b[u] + r + (i64)t * G;
                if (j < e[u]) acc[u] += ab_term(a, j, pv[u], bestv[u], multi[u], igain[u], hv[u]);
            }
        }
#pragma unroll
        for (int u = 0; u < UV; u++) {
            double ch = acc[u];
#pragma unroll
            for (int d = G / 2; d >= 1; d >>= 1) ch = ch + __shfl_xor_sync(FULL, ch, d);
            if (r == 0 && act[u]) {
                a.keep[iv[u]] = (igain[u] + (float)ch) >= 0.0f ? 1 : 0;
                pb += ab_bytes(a, e[u] - b[u]);
            }
        }
    }
    if (a.prof) {
        pb = (unsigned long long)warp_sum_i64((i64)pb);
        if (l == 0 && pb) atomicAdd(a.prof, pb);
    }
}

// Afterburner for candidates of degree <= 2H, one thread per vertex, the
// association of k_afterburner_small<W, H, 2> (canon_tree).
template <class W, int H>
__global__ void __launch_bounds__(256) k_afterburner_thr(ABArgs<W> a, Range rg) {
    const i64 lo = rg.begin(), hi = rg.end();
    unsigned long long pb = 0;
    for (i64 x = lo + blockIdx.x * (i64)blockDim.x + threadIdx.x; x < hi; x += (i64)gridDim.x * blockDim.x) {
        const i32 i = rg.list[x];
        const i32 best = a.dest[i];
        if (best == NO_MOVE) continue;
        const i32 p = a.part[i];
        const float multi = to_f(a.g.vtx_w[i]) * a.pm;
        const float igain = a.gain[i];
        const i32 hv = (i32)xorshift32((u32)i);
        const i64 b = a.g.rowptr[i], e = a.g.rowptr[i + 1];
        double acc[H];
#pragma unroll
        for (int r = 0; r < H; r++) {
            acc[r] = 0.0;
            if (b + r < e) acc[r] += ab_term(a, b + r, p, best, multi, igain, hv);
            if (b + r + H < e) acc[r] += ab_term(a, b + r + H, p, best, multi, igain, hv);
        }
        const double ch = canon_tree<H, double>(acc);
        a.keep[i] = (igain + (float)ch) >= 0.0f ? 1 : 0;
        pb += ab_bytes(a, e - b);
    }
    if (a.prof) {
        pb = (unsigned long long)warp_sum_i64((i64)pb);
        if (lane_id() == 0 && pb) atomicAdd(a.prof, pb);
    }
}

template <class W>
__global__ void __launch_bounds__(1024) k_afterburner_block(ABArgs<W> a, Range rg) {
    __shared__ double red[32];
    const i64 lo = rg.begin(), hi_x = rg.end();
    for (i64 x = lo + blockIdx.x; x < hi_x; x += gridDim.x) {
        i32 i = rg.list[x];
        if (a.dest[i] == NO_MOVE) continue;
        i32 best = a.dest[i], p = a.part[i];
        float multi = to_f(a.g.vtx_w[i]) * a.pm;
        float igain = a.gain[i];
        i32 hi = (i32)xorshift32((u32)i);
        double ch = block1024_canon_sum(a.g.rowptr[i], a.g.rowptr[i + 1],
                                        [&](i64 j) { return ab_term(a, j, p, best, multi, igain, hi); }, red);
        if (threadIdx.x == 0) a.keep[i] = (igain + (float)ch) >= 0.0f ? 1 : 0;
    }
}

// ---------------------------------------------------------------------------
// compactions
// ---------------------------------------------------------------------------
struct CandFlag {
    const i32* order1;
    const i32* dest;
    __device__ i64 operator()(i64 x) const { return dest[order1[x]] != NO_MOVE ? 1 : 0; }
};
struct CandEpi {
    const i32* order1;
    i32* cand;
    i64 split_at;
    i64* split;
    __device__ void operator()(i64 x, i64 excl, i64 v) const {
        if (v) cand[excl] = order1[x];
        if (x == split_at) *split = excl;
    }
};
struct KeepFlag {
    const i32* cand;
    const unsigned char* keep;  // indexed by vertex
    __device__ i64 operator()(i64 x) const { return keep[cand[x]]; }
};
// move-list compaction that also counts the NEW_PART moves
struct MoveEpi {
    const i32* cand;
    const i32* dest;
    i32* moves;
    unsigned long long* new_count;
    __device__ void operator()(i64 x, i64 excl, i64 v) const {
        if (v) {
            i32 i = cand[x];
            moves[excl] = i;
            if (dest[i] == NEW_PART) atomicAdd(new_count, 1ull);
        }
    }
};
struct ListEpi {
    const i32* src;
    i32* dst;
    __device__ void operator()(i64 x, i64 excl, i64 v) const {
        if (v) dst[excl] = src[x];
    }
};
struct NewFlag {
    const i32* moves;
    const i32* dest;
    __device__ i64 operator()(i64 x) const { return dest[moves[x]] == NEW_PART ? 1 : 0; }
};
struct UnusedFlag {
    const unsigned char* has;
    __device__ i64 operator()(i64 l) const { return has[l] ? 0 : 1; }
};
struct IdxEpi {
    i32* dst;
    __device__ void operator()(i64 x, i64 excl, i64 v) const {
        if (v) dst[excl] = (i32)x;
    }
};

template <class V>
__global__ void k_set_split_if_end(LMScalars<V>* sc) {
    sc->split = sc->num_cand;
}

// ---------------------------------------------------------------------------
// set_new_cluster_ids (src/local_mover.cpp:217-274)
// ---------------------------------------------------------------------------
template <class V>
__global__ void k_prep_new(LMScalars<V>* sc) {
    sc->avail_k = sc->num_new > 0 ? sc->label_count : 0;
}
template <class V>
__global__ void k_clear_has(unsigned char* has, const LMScalars<V>* sc) {
    i64 L = sc->avail_k;
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < L; i += (i64)gridDim.x * blockDim.x) has[i] = 0;
}
template <class V>
__global__ void k_mark_has(unsigned char* has, const i32* part, i64 n, const LMScalars<V>* sc) {
    if (sc->avail_k == 0) return;
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) has[part[i]] = 1;
}
template <class V>
__global__ void k_assign_new(const i32* newl, const i32* avail, i32* dest, const i32* part, i32* constraint, V* td,
                             LMScalars<V>* sc, i64 capacity, int* err) {
    i64 nn = sc->num_new, na = sc->num_avail, L = sc->label_count;
    for (i64 r = blockIdx.x * (i64)blockDim.x + threadIdx.x; r < nn; r += (i64)gridDim.x * blockDim.x) {
        i32 x = newl[r];
        i64 lab = r < na ? (i64)avail[r] : L + (r - na);
        if (lab >= capacity) {
            atomicExch(err, (int)DEV_ERR_LABEL);
            continue;
        }
        dest[x] = (i32)lab;
        if (constraint) constraint[lab] = constraint[part[x]];
        if (r >= na) td[lab] = V(0);
    }
}
template <class V>
__global__ void k_finish_new(LMScalars<V>* sc, i64 capacity) {
    if (sc->num_new > sc->num_avail) {
        sc->label_count += sc->num_new - sc->num_avail;
        if (sc->label_count > capacity) sc->label_count = capacity;
    }
}

// ---------------------------------------------------------------------------
// perform_moves (src/local_mover.cpp:1241-1279)
// ---------------------------------------------------------------------------
// csize / moved_at (NULL unless the learned filter is on) track cluster sizes
// and the sweep in which each vertex last moved
template <class W>
__global__ void k_apply_moves(DGraph<W> g, const i32* moves, i64 nm, const i32* dest, i32* part,
                              typename Traits<W>::V* td, int* err, i32* csize, i32* moved_at, i32 stamp) {
    for (i64 x = blockIdx.x * (i64)blockDim.x + threadIdx.x; x < nm; x += (i64)gridDim.x * blockDim.x) {
        i32 i = moves[x];
        i32 b = dest[i], p = part[i];
        if (b < 0) {  // an unresolved NEW_PART: never applied
            atomicExch(err, (int)DEV_ERR_LABEL);
            continue;
        }
        auto w = g.vtx_w[i];
        vatomic_add(&td[p], -w);
        vatomic_add(&td[b], w);
        part[i] = b;
        if (csize) {
            atomicSub(&csize[p], 1);
            atomicAdd(&csize[b], 1);
            moved_at[i] = stamp;
        }
    }
}

template <class W>
__global__ void k_mark_affected(DGraph<W> g, const i32* moves, i64 nm, unsigned char* flags) {
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
    for (i64 x = gw; x < nm; x += nw) {
        i32 i = moves[x];
        if (lane_id() == 0) flags[i] = 1;
        for (i64 j = g.rowptr[i] + lane_id(); j < g.rowptr[i + 1]; j += 32) flags[g.col[j]] = 1;
    }
}

// The same flags pulled instead of pushed: the movers are flagged 2 first
// (k_mark_movers), then a warp per vertex looks for a flagged-2 neighbour 32
// edges at a time and stops at the first one.  Pushing costs the movers'
// degrees, pulling about n / (moved fraction) edges, so dense graphs with
// many movers pull.  The graph is symmetric, so "has a moved neighbour" is
// "is a neighbour of a mover": the flagged set is the same.
__global__ void k_mark_movers(const i32* moves, i64 nm, unsigned char* flags) {
    for (i64 x = blockIdx.x * (i64)blockDim.x + threadIdx.x; x < nm; x += (i64)gridDim.x * blockDim.x)
        flags[moves[x]] = 2;
}

template <class W>
__global__ void k_mark_pull(DGraph<W> g, unsigned char* flags) {
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
    const int l = lane_id();
    for (i64 i = gw; i < g.n; i += nw) {
        if (flags[i] == 2) continue;
        const i64 b = g.rowptr[i], e = g.rowptr[i + 1];
        bool hit = false;
        for (i64 j0 = b; j0 < e && !hit; j0 += 32) {
            const i64 j = j0 + l;
            hit = __any_sync(FULL, j < e && flags[g.col[j]] == 2);
        }
        if (hit && l == 0) flags[i] = 1;
    }
}

// Affected vertices of a sweep (the movers and their neighbours), listed once
// each: vertices below MASSIVE_CUTOFF go to `list` (first marker of the
// epoch appends), massive ones are flagged for the block kernel.
template <class W>
__global__ void k_mark_list(DGraph<W> g, const i32* moves, i64 nm, u32* stamp, u32 epoch, i32* list, i64* cnt,
                            unsigned char* flags, int has_massive) {
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
    auto mark = [&](i32 v) {
        if (has_massive && g.rowptr[v + 1] - g.rowptr[v] >= MASSIVE_CUTOFF) flags[v] = 1;
        else if (atomicExch(&stamp[v], epoch) != epoch) list[atomicAdd((unsigned long long*)cnt, 1ull)] = v;
    };
    for (i64 x = gw; x < nm; x += nw) {
        const i32 i = moves[x];
        if (lane_id() == 0) mark(i);
        for (i64 j = g.rowptr[i] + lane_id(); j < g.rowptr[i + 1]; j += 32) mark(g.col[j]);
    }
}

template <class V>
struct SqIn;
template <>
struct SqIn<i64> {
    const i64* td;
    const i64* L;
    __device__ i64 operator()(i64 i) const { return i < *L ? td[i] * td[i] : 0; }
};
template <>
struct SqIn<double> {
    const double* td;
    const i64* L;
    __device__ double operator()(i64 i) const { return i < *L ? td[i] * td[i] : 0.0; }
};
struct PvI64In {
    const i64* a;
    __device__ i64 operator()(i64 i) const { return a[i]; }
};

template <class V>
__global__ void k_objective(LMScalars<V>* sc, double lambda) {
    V cut_change = sc->pval_sum - sc->last_pval;
    sc->last_pval = sc->pval_sum;
    sc->uncut = sc->uncut + cut_change;
    double m;
    if constexpr (std::is_same<V, i64>::value) {
        m = static_cast<double>(sc->uncut);
        m = m - lambda * static_cast<double>(sc->sumsq_i);
    } else {
        m = sc->uncut;
        m = m - lambda * sc->sumsq_d;
    }
    sc->obj = m;
    sc->improved = m > sc->best_obj ? 1 : 0;
    if (sc->improved) {
        sc->best_obj = m;
        sc->best_uncut = sc->uncut;
        sc->best_label_count = sc->label_count;
    }
}

// best state <- current state when the sweep improved the objective: the
// partition, the cluster volumes (label_count of them) and the own-cluster
// weights, in one grid-stride pass
template <class V>
__global__ void k_copy_if_improved(i32* best_part, const i32* part, V* td_best, const V* td, V* pv_best, const V* pv,
                                   i64 n, const LMScalars<V>* sc) {
    if (!sc->improved) return;
    const i64 L = sc->label_count;
    const i64 k = n > L ? n : L;
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < k; i += (i64)gridDim.x * blockDim.x) {
        if (i < n) {
            best_part[i] = part[i];
            pv_best[i] = pv[i];
        }
        if (i < L) td_best[i] = td[i];
    }
}

// ---------------------------------------------------------------------------
// afterburner_filter_strict (src/local_mover.cpp:131-213), O(k log k)
// ---------------------------------------------------------------------------
template <class W>
__global__ void __launch_bounds__(256) k_strict_nb_warp(DGraph<W> g, const i32* moves, i64 lo, i64 hi,
                                                        const i32* prio, const i32* dest, const i32* part,
                                                        typename Traits<W>::V* nb) {
    using V = typename Traits<W>::V;
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
    for (i64 x = lo + gw; x < hi; x += nw) {
        i32 i = moves[x];
        i32 best = dest[i], p = part[i];
        i32 pi = prio[i];
        V r = VSum<V>::warp(g.rowptr[i], g.rowptr[i + 1], [&](i64 j) -> V {
            i32 v = g.col[j];
            if (!(prio[v] < pi)) return V(0);
            int coef = 0;
            i32 vp = dest[v];
            if (vp == p) coef--;
            if (vp == best && best != NEW_PART) coef++;
            vp = part[v];
            if (vp == p) coef++;
            if (vp == best) coef--;
            return V(coef) * V(g.wgt(j));
        });
        if (lane_id() == 0) nb[x] = r;
    }
}

template <class W>
__global__ void __launch_bounds__(1024) k_strict_nb_block(DGraph<W> g, const i32* moves, i64 lo, i64 hi,
                                                          const i32* prio, const i32* dest, const i32* part,
                                                          typename Traits<W>::V* nb) {
    using V = typename Traits<W>::V;
    __shared__ double red[32];
    __shared__ unsigned long long acc;
    for (i64 x = lo + blockIdx.x; x < hi; x += gridDim.x) {
        i32 i = moves[x];
        i32 best = dest[i], p = part[i];
        i32 pi = prio[i];
        auto term = [&](i64 j) -> V {
            i32 v = g.col[j];
            if (!(prio[v] < pi)) return V(0);
            int coef = 0;
            i32 vp = dest[v];
            if (vp == p) coef--;
            if (vp == best && best != NEW_PART) coef++;
            vp = part[v];
            if (vp == p) coef++;
            if (vp == best) coef--;
            return V(coef) * V(g.wgt(j));
        };
        V r;
        if constexpr (std::is_same<V, double>::value) {
            r = block1024_canon_sum(g.rowptr[i], g.rowptr[i + 1], term, red);
        } else {
            if (threadIdx.x == 0) acc = 0;
            __syncthreads();
            i64 s = 0;
            for (i64 j = g.rowptr[i] + threadIdx.x; j < g.rowptr[i + 1]; j += 1024) s += term(j);
            s = warp_sum_i64(s);
            if (lane_id() == 0) ::atomicAdd(&acc, (unsigned long long)s);
            __syncthreads();
            r = (i64)acc;
        }
        if (threadIdx.x == 0) nb[x] = r;
        __syncthreads();
    }
}

__global__ void k_prio(const i32* moves, i64 k, i32* prio) {
    for (i64 x = blockIdx.x * (i64)blockDim.x + threadIdx.x; x < k; x += (i64)gridDim.x * blockDim.x)
        prio[moves[x]] = (i32)x;
}

template <class V>
__global__ void k_strict_keys(const i32* moves, i64 k, const i32* dest, const i32* part, u64* kd, u64* kp, i32* id,
                              i32* ip) {
    for (i64 x = blockIdx.x * (i64)blockDim.x + threadIdx.x; x < k; x += (i64)gridDim.x * blockDim.x) {
        i32 i = moves[x];
        kd[x] = ((u64)(u32)dest[i] << 32) | (u64)x;
        kp[x] = ((u64)(u32)part[i] << 32) | (u64)x;
        id[x] = (i32)x;
        ip[x] = (i32)x;
    }
}

template <class V>
__device__ __forceinline__ i64 lower_bound_u64(const u64* a, i64 k, u64 key) {
    i64 lo = 0, hi = k;
    while (lo < hi) {
        i64 mid = (lo + hi) >> 1;
        if (a[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

template <class V>
__device__ __forceinline__ V prefix_query(const u64* ks, const V* E, i64 k, i32 key, i64 x) {
    u64 hk = (u64)(u32)key << 32;
    i64 a = lower_bound_u64<V>(ks, k, hk | (u64)x);
    i64 s = lower_bound_u64<V>(ks, k, hk);
    return E[a] - E[s];
}

template <class W>
__global__ void k_strict_oc(DGraph<W> g, const i32* moves, i64 k, const i32* dest, const i32* part, const float* gain,
                            const typename Traits<W>::V* nb, const u64* ksd, const typename Traits<W>::V* Ed,
                            const u64* ksp, const typename Traits<W>::V* Ep, float pm, double* oc) {
    using V = typename Traits<W>::V;
    for (i64 x = blockIdx.x * (i64)blockDim.x + threadIdx.x; x < k; x += (i64)gridDim.x * blockDim.x) {
        i32 i = moves[x];
        i32 best = dest[i], p = part[i];
        float multi = to_f(g.vtx_w[i]) * pm;
        V A = prefix_query<V>(ksd, Ed, k, p, x);
        V B = best != NEW_PART ? prefix_query<V>(ksd, Ed, k, best, x) : V(0);
        V C = prefix_query<V>(ksp, Ep, k, p, x);
        V D = prefix_query<V>(ksp, Ep, k, best, x);
        V S = ((C - A) + B) - D;
        double t2 = -(double)multi * (double)S;
        oc[x] = ((double)gain[i] + (double)nb[x]) + t2;
    }
}

// first position of the maximum prefix value; writes num_moves = truncate
template <class V>
__global__ void __launch_bounds__(1024) k_strict_argmax(const double* pre, i64 k, LMScalars<V>* sc) {
    __shared__ double bv[32];
    __shared__ i64 bl[32];
    double v = -INFINITY;
    i64 loc = k;
    for (i64 x = threadIdx.x; x < k; x += 1024)
        if (pre[x] > v) {
            v = pre[x];
            loc = x;
        }
    for (int d = 16; d >= 1; d >>= 1) {
        double ov = __shfl_xor_sync(FULL, v, d);
        i64 ol = __shfl_xor_sync(FULL, loc, d);
        if (ov > v || (ov == v && ol < loc)) {
            v = ov;
            loc = ol;
        }
    }
    if (lane_id() == 0) {
        bv[threadIdx.x >> 5] = v;
        bl[threadIdx.x >> 5] = loc;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        v = bv[threadIdx.x];
        loc = bl[threadIdx.x];
        for (int d = 16; d >= 1; d >>= 1) {
            double ov = __shfl_xor_sync(FULL, v, d);
            i64 ol = __shfl_xor_sync(FULL, loc, d);
            if (ov > v || (ov == v && ol < loc)) {
                v = ov;
                loc = ol;
            }
        }
        if (threadIdx.x == 0) sc->num_moves = (loc < k && v > 0.0) ? loc + 1 : 0;
    }
}

template <class V>
__global__ void k_gather_vw(const i32* order, const i32* moves, const V* vw, i64 k, V* out) {
    for (i64 y = blockIdx.x * (i64)blockDim.x + threadIdx.x; y < k; y += (i64)gridDim.x * blockDim.x)
        out[y] = vw[moves[order[y]]];
}
struct I64ArrIn {
    const i64* a;
    i64 k;
    __device__ i64 operator()(i64 i) const { return i < k ? a[i] : 0; }
};
struct I64ExclOut {
    i64* E;
    __device__ void operator()(i64 i, i64 excl, i64) const { E[i] = excl; }
};

// ---------------------------------------------------------------------------
// relabel_contiguously (src/local_mover.cpp:100-129)
// ---------------------------------------------------------------------------
// labels outside [0, L) (only after a device error latched d_err, which the
// host raises right after) are left alone
__global__ void k_mark_used(unsigned char* used, const i32* lab, i64 n, i64 L) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
        const i32 l = lab[i];
        if (l >= 0 && l < L) used[l] = 1;
    }
}
struct UsedFlag {
    const unsigned char* used;
    __device__ i64 operator()(i64 l) const { return used[l] ? 1 : 0; }
};
template <class V>
struct RelabelEpi {
    i32* newid;
    const V* td;
    V* td_out;
    __device__ void operator()(i64 l, i64 excl, i64 v) const {
        if (v) {
            newid[l] = (i32)excl;
            td_out[excl] = td[l];
        }
    }
};
__global__ void k_remap(i32* lab, i64 n, const i32* newid, i64 L) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
        const i32 l = lab[i];
        if (l >= 0 && l < L) lab[i] = newid[l];
    }
}

// ---------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------
inline int grid_for(Context& ctx, i64 work, int per_block, int max_per_sm = 16) {
    return (int)std::max<i64>(1, std::min<i64>(ceil_div(std::max<i64>(work, 1), per_block), (i64)ctx.num_sms * max_per_sm));
}

// Row weight sums (8-lane groups per vertex; computed once per graph).  Only
// the no-candidate bound reads them, whose one-FP32-step margin covers any
// summation order.
template <class W>
__global__ void k_row_sums(DGraph<W> g, typename Traits<W>::V* out) {
    using V = typename Traits<W>::V;
    const int r = lane_id() & 7;
    const i64 gg = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 3;
    const i64 ng = ((i64)gridDim.x * blockDim.x) >> 3;
    for (i64 base = gg - (gg & 3); base < g.n; base += ng) {
        const i64 i = base + (gg & 3);
        V s = V(0);
        if (i < g.n)
            for (i64 j = g.rowptr[i] + r; j < g.rowptr[i + 1]; j += 8) s += V(g.wgt(j));
#pragma unroll
        for (int d = 4; d >= 1; d >>= 1) s = s + __shfl_xor_sync(FULL, s, d);
        if (r == 0 && i < g.n) out[i] = s;
    }
}

// graphs are created with their sums (make_graph) or by one context (coarse
// levels); the lock covers a graph first used by several threads
static std::mutex g_graph_cache_mu;

template <class W>
const typename Traits<W>::V* row_sums(Context& ctx, const Graph<W>& g) {
    using V = typename Traits<W>::V;
    if (g.n == 0) return nullptr;
    std::lock_guard<std::mutex> lk(g_graph_cache_mu);
    if (!g.rsum.p) {
        g.rsum = DBuf<V>(ctx, g.n);
        k_row_sums<W><<<(int)std::min<i64>(ceil_div(g.n, 32), (i64)ctx.num_sms * 16), 256, 0, ctx.stream>>>(g.view(),
                                                                                                          g.rsum.p);
        PGGC_LAUNCH_CHECK();
    }
    return g.rsum.p;
}

template <class W>
struct Mover {
    using V = typename Traits<W>::V;
    Context& ctx;
    const Graph<W>& g;
    const Ordering& ord;
    i64 n;
    i64 cap;  // label capacity
    // views of context workspace slots (reused across local_move calls)
    template <class T>
    struct View {
        T* p = nullptr;
    };
    View<i32> part, dest, cand, moves, newl, avail, prio;
    View<float> gain;
    View<V> pvals, pvals_clone, td_curr;
    View<unsigned char> flags, keep, has;
    // affected-vertex list of a sweep with few moves (stamp[v] == epoch: listed)
    View<u32> stamp;
    View<i32> aff;
    View<i64> aff_cnt;
    u32 epoch = 0;
    View<LMScalars<V>> sc;
    View<i32> gkeys;
    View<V> gvals;
    i64 gcap = 0;
    int gblocks = 0;  // global tables (one per block of the global-table pass)
    bool cdata_init = false;
    ClassLists cls;
    // learned filter state (allocated only when the context's filter is on)
    bool filt_on = false;
    View<i32> moved_at, csize;

    enum Slot { S_PART, S_DEST, S_CAND, S_MOVES, S_NEWL, S_AVAIL, S_PRIO, S_GAIN, S_PV, S_PVC, S_TD, S_FLAGS, S_KEEP,
                S_HAS, S_SC, S_GK, S_GV, S_CLS, S_CLS_OFF, S_CLS_CNT, S_MOVED_AT, S_CSIZE, S_OVF, S_OVF_CNT,
                S_STAMP, S_AFF, S_AFF_CNT, S_SPLIT_BEST };

    Mover(Context& c, const Graph<W>& gr, const Ordering& o, i64 capacity)
        : ctx(c), g(gr), ord(o), n(gr.n), cap(capacity) {
        i64 nn = std::max<i64>(n, 1), cc = std::max<i64>(cap, 1);
        part.p = ctx.ws_get<i32>(S_PART, nn);
        dest.p = ctx.ws_get<i32>(S_DEST, nn);
        cand.p = ctx.ws_get<i32>(S_CAND, nn);
        moves.p = ctx.ws_get<i32>(S_MOVES, nn);
        newl.p = ctx.ws_get<i32>(S_NEWL, nn);
        avail.p = ctx.ws_get<i32>(S_AVAIL, cc);
        gain.p = ctx.ws_get<float>(S_GAIN, nn);
        pvals.p = ctx.ws_get<V>(S_PV, nn);
        pvals_clone.p = ctx.ws_get<V>(S_PVC, nn);
        td_curr.p = ctx.ws_get<V>(S_TD, cc);
        flags.p = ctx.ws_get<unsigned char>(S_FLAGS, nn);
        keep.p = ctx.ws_get<unsigned char>(S_KEEP, nn);
        has.p = ctx.ws_get<unsigned char>(S_HAS, cc);
        sc.p = ctx.ws_get<LMScalars<V>>(S_SC, 1);
        PGGC_CUDA(cudaMemsetAsync(flags.p, 0, nn, ctx.stream));
        stamp.p = ctx.ws_get<u32>(S_STAMP, nn);
        aff.p = ctx.ws_get<i32>(S_AFF, nn);
        aff_cnt.p = ctx.ws_get<i64>(S_AFF_CNT, 1);
        PGGC_CUDA(cudaMemsetAsync(stamp.p, 0, sizeof(u32) * nn, ctx.stream));
        cls = graph_class_lists<W>(ctx, g, ord);
        if (ord.n_huge > 0) {
            gcap = next_pow2_u32((u32)std::min<i64>(2 * ord.max_deg, (i64)1 << 30));
            // at most 32 tables and at most GTABLE_BYTES of them in total (one
            // table when a single one is larger): a vertex of degree ~10^7
            // would otherwise ask for 32 tables of 2^25 slots
            constexpr i64 GTABLE_BYTES = (i64)1 << 30;
            const i64 per = gcap * (i64)(sizeof(i32) + sizeof(V));
            gblocks = (int)std::max<i64>(1, std::min<i64>(std::min<i64>(ord.n_huge, 32), GTABLE_BYTES / per));
            gkeys.p = ctx.ws_get<i32>(S_GK, gcap * gblocks);
            gvals.p = ctx.ws_get<V>(S_GV, gcap * gblocks);
        }
    }

    // learned filter: per-call state once `part` holds the starting partition
    void filter_init() {
        filt_on = ctx.filt.mode != 0;
        if (!filt_on) return;
        i64 nn = std::max<i64>(n, 1), cc = std::max<i64>(cap, 1);
        moved_at.p = ctx.ws_get<i32>(S_MOVED_AT, nn);
        csize.p = ctx.ws_get<i32>(S_CSIZE, cc);
        fill<i32>(ctx, moved_at.p, n, -1);
        PGGC_CUDA(cudaMemsetAsync(csize.p, 0, sizeof(i32) * cc, ctx.stream));
        PGGC_CUDA(cudaMemsetAsync(gain.p, 0, sizeof(float) * nn, ctx.stream));
        k_cluster_sizes<<<grid_for(ctx, n, 256), 256, 0, ctx.stream>>>(part.p, n, csize.p);
        PGGC_LAUNCH_CHECK();
    }

    // before a sweep's select: sample features (log mode) or drop the vertices
    // the network rejects (filter mode)
    void filter_pre(int sweep_idx, double vol_total) {
        if (!filt_on) return;
        auto& F = ctx.filt;
        F.stamp++;
        if (F.mode == 2 && (F.suspended || F.level < F.min_level || (F.max_pass >= 0 && F.pass >= F.max_pass)))
            return;
        ProfScope ps(ctx, "filter");
        FiltArgs<W> a;
        a.g = g.view();
        a.part = part.p;
        a.pvals = pvals.p;
        a.gain = gain.p;
        a.moved_at = moved_at.p;
        a.csize = csize.p;
        a.td = td_curr.p;
        a.dest = dest.p;
        a.inv_vol = vol_total > 0 ? (float)(1.0 / vol_total) : 0.f;
        a.inv_log_n = (float)(1.0 / std::log2(2.0 + (double)n));
        a.level_f = (float)F.level / 16.f;
        a.sweep_f = (float)sweep_idx / 8.f;
        a.prev_stamp = F.stamp - 1;
        a.mode = F.mode;
        a.net = F.net;
        a.threshold = F.threshold;
        a.log_x = F.log_x;
        a.log_v = F.log_v;
        a.log_y = F.log_y;
        a.log_cnt = F.log_cnt;
        a.log_cap = F.log_cap;
        a.rate = F.log_rate;
        a.salt = (u32)(F.log_seed ^ ((u64)(u32)F.stamp * 0x9E3779B9ull));
        a.stats = F.stats;
        if (F.mode == 1)
            PGGC_CUDA(cudaMemcpyAsync(F.log_cnt + 1, F.log_cnt, sizeof(unsigned long long), cudaMemcpyDeviceToDevice,
                                      ctx.stream));
        int grid = grid_for(ctx, ceil_div(n, 32 * FW_WARPS), 1, 8);
        k_filter_sweep<W><<<grid, FW_WARPS * 32, 0, ctx.stream>>>(a);
        PGGC_LAUNCH_CHECK();
    }

    // after the afterburner: label this sweep's logged samples
    void filter_post() {
        if (!filt_on || ctx.filt.mode != 1) return;
        auto& F = ctx.filt;
        k_filter_label<<<ctx.num_sms, 256, 0, ctx.stream>>>(F.log_v, F.log_y, F.log_cnt, F.log_cap, dest.p, keep.p,
                                                             F.log_label);
        PGGC_LAUNCH_CHECK();
    }

    SelArgs<W> sel_args(float fr, bool initial, const i32* constraint, const V* td, const i32* partp,
                        const V* pv, i32* destp, float* gainp, const i64* lcount, float pm) {
        SelArgs<W> a;
        a.g = g.view();
        a.part = partp;
        a.dest = destp;
        a.gain = gainp;
        a.pvals = pv;
        a.td = td;
        a.constraint = constraint;
        a.label_count = lcount;
        a.rsum = row_sums<W>(ctx, g);
        a.pm = pm;
        a.fr = fr;
        a.initial = initial ? 1 : 0;
        a.err = ctx.d_err;
        a.prof = nullptr;
        a.probe_cap = ctx.probe_cap;
        a.keys32 = cap < ((i64)1 << 29) ? 1 : 0;
        a.dense = 0;
        a.inv_load = ctx.tune.load >= 0.7f ? 1.0f / 0.7f : 2.0f;
        return a;
    }

    i64 label_bound_host = 0;  // host upper bound of the label count (table sizing)

    template <bool CON>
    void launch_select_t(SelArgs<W> a) {
        // degree classes 0..2 (<= 8, 16, 32) go to the thread kernels up to the
        // tuned thread bound, the rest below 128 to the warp kernel up to the
        // tuned warp bound, and everything above to the block kernels
        const TuneParams& tp = ctx.tune;
        const int tcls = tp.thread_max_deg >= 32 ? 3 : tp.thread_max_deg >= 16 ? 2 : tp.thread_max_deg >= 8 ? 1 : 0;
        const int wend = tp.warp_max_deg >= 127 ? 4 : 3;  // first class after the warp kernel's
        if (ord.off_large > 0) {
            ProfScope ps(ctx, "select_warp");
            a.prof = ctx.prof_counter("select_warp");
            int grid_t = grid_for(ctx, ceil_div(cls.count, 256), 1, 16);
            if (tcls > 0) {
                k_select_thr<W, CON, 8><<<grid_t, 256, 0, ctx.stream>>>(a, cls.list, cls.off, 0);
                PGGC_LAUNCH_CHECK();
            }
            if (tcls > 1) {
                k_select_thr<W, CON, 16><<<grid_t, 256, 0, ctx.stream>>>(a, cls.list, cls.off, 1);
                PGGC_LAUNCH_CHECK();
            }
            if (tcls > 2) {
                k_select_thr<W, CON, 32><<<grid_t, 256, 0, ctx.stream>>>(a, cls.list, cls.off, 2);
                PGGC_LAUNCH_CHECK();
            }
            if (tcls < wend) {
                int grid = grid_for(ctx, ceil_div(ord.off_large, SELW_WARPS), 1, 16);
                k_select_warp<W, CON><<<grid, SELW_WARPS * 32, 0, ctx.stream>>>(
                    a, dev_range(cls.list, cls.off + tcls, cls.off + wend));
                PGGC_LAUNCH_CHECK();
            }
        }
        i64 nb = n - ord.off_large;
        if (nb > 0 || (wend < 4 && ord.off_large > 0)) {
            ProfScope ps(ctx, "select_block");
            a.prof = ctx.prof_counter("select_block");
            // classes from the warp bound to 4 (degree <= 1024): 2048-slot
            // tables, 8 blocks of 256 per SM; class 5 (degree <= 4096):
            // 8192-slot tables, 2 blocks of 512 per SM
            const size_t slot = sizeof(V) + sizeof(i32);
            const i64 nb4 = wend < 4 ? n : nb;
            const i64 n4 = std::min<i64>(nb4, (i64)ctx.num_sms * 8), n5 = std::min<i64>(nb, (i64)ctx.num_sms * 2);
            // with at most as many labels as table slots, the table is indexed
            // by cluster id directly (no probing, no keys)
            SelArgs<W> a4 = a;
            a4.dense = label_bound_host <= 2048 ? 1 : 0;
            k_select_block<W, CON, false, 256><<<(int)n4, 256, slot * 2048, ctx.stream>>>(
                a4, dev_range(cls.list, cls.off + wend, cls.off + 5), nullptr, nullptr, 2048);
            PGGC_LAUNCH_CHECK();
            if (ord.max_deg > 1024) {
                SelArgs<W> a5 = a;
                a5.dense = label_bound_host <= SEL_TS_MAX ? 1 : 0;
                set_dynamic_smem_once(k_select_block<W, CON, false, 512>, (int)(slot * SEL_TS_MAX), ctx.device);
                // a dense table needs only the label_bound values: more blocks fit an SM
                const size_t smem5 =
                    a5.dense ? sizeof(V) * (size_t)std::max<i64>(label_bound_host, 1) : slot * SEL_TS_MAX;
                const int g5 = a5.dense ? (int)std::min<i64>(nb, (i64)ctx.num_sms * 4) : (int)n5;
                k_select_block<W, CON, false, 512><<<g5, 512, smem5, ctx.stream>>>(
                    a5, dev_range(cls.list, cls.off + 5, cls.off + 6), nullptr, nullptr, SEL_TS_MAX);
                PGGC_LAUNCH_CHECK();
            }
        }
        if (ord.n_huge > 0) {
            ProfScope ps(ctx, "select_huge");
            a.prof = ctx.prof_counter("select_huge");
            // 1024-thread blocks with 16384-slot shared tables; vertices with
            // more distinct neighbour clusters than fit go to the global pass
            const size_t slot = sizeof(V) + sizeof(i32);
            constexpr int TS = 16384;
            i32* ovf = ctx.ws_get<i32>(S_OVF, ord.n_huge);
            i64* ovf_cnt = ctx.ws_get<i64>(S_OVF_CNT, 1);
            PGGC_CUDA(cudaMemsetAsync(ovf_cnt, 0, sizeof(i64), ctx.stream));
            set_dynamic_smem_once(k_select_block<W, CON, false, 1024, true>, (int)(slot * TS), ctx.device);
            SelArgs<W> ah = a;
            ah.dense = label_bound_host <= TS ? 1 : 0;
            // a dense table needs only the label_bound values: two blocks fit an SM
            const size_t smemh = ah.dense ? sizeof(V) * (size_t)std::max<i64>(label_bound_host, 1) : slot * TS;
            const int grid = (int)std::min<i64>(ord.n_huge, (i64)ctx.num_sms * (smemh <= 100 * 1024 ? 2 : 1));
            k_select_block<W, CON, false, 1024, true><<<grid, 1024, smemh, ctx.stream>>>(
                ah, host_range(ord.huge.p, 0, ord.n_huge), nullptr, nullptr, TS, ovf, ovf_cnt);
            PGGC_LAUNCH_CHECK();
            // the vertices that overflowed: rows split across blocks, in rounds
            // of up to gblocks vertices (one table each)
            const i64 n_ovf = ctx.read1(ovf_cnt);
            unsigned long long* sbest = ctx.ws_get<unsigned long long>(S_SPLIT_BEST, gblocks);
            set_dynamic_smem_once(k_split_insert<W>, (int)SPLIT_SMEM, ctx.device);
            const unsigned chunks = (unsigned)std::max<i64>(1, ceil_div(ord.max_deg, SPLIT_CHUNK));
            for (i64 r0 = 0; r0 < n_ovf; r0 += gblocks) {
                const i64 cnt = std::min<i64>(gblocks, n_ovf - r0);
                const i32* lst = ovf + r0;
                const int cgrid = grid_for(ctx, cnt * gcap, 256, 16);
                k_split_clear<W><<<cgrid, 256, 0, ctx.stream>>>(a, lst, cnt, gcap, gkeys.p, gvals.p, sbest);
                PGGC_LAUNCH_CHECK();
                k_split_insert<W><<<dim3(chunks, (unsigned)cnt), SPLIT_THREADS, SPLIT_SMEM, ctx.stream>>>(
                    a, lst, cnt, gcap, gkeys.p, gvals.p);
                PGGC_LAUNCH_CHECK();
                const unsigned sblocks =
                    (unsigned)std::max<i64>(1, std::min<i64>(ceil_div(gcap, SPLIT_THREADS * 8), (i64)ctx.num_sms));
                k_split_scan<W, CON><<<dim3(sblocks, (unsigned)cnt), SPLIT_THREADS, 0, ctx.stream>>>(
                    a, lst, cnt, gcap, gkeys.p, gvals.p, sbest);
                PGGC_LAUNCH_CHECK();
                k_split_finish<W><<<1, 256, 0, ctx.stream>>>(a, lst, cnt, sbest);
                PGGC_LAUNCH_CHECK();
            }
        }
    }
    void launch_select(const SelArgs<W>& a, bool constrained) {
        if (constrained) launch_select_t<true>(a);
        else launch_select_t<false>(a);
    }

    // candidates (order1 order) -> cand, sc.num_cand, sc.split
    void compact_candidates() {
        LMScalars<V>* s = sc.p;
        scan_apply(ctx, CandFlag{ord.order1.p, dest.p},
                   CandEpi{ord.order1.p, cand.p, ord.off_large2 < n ? ord.off_large2 : -1, &s->split}, n, nullptr,
                   &s->num_cand);
        if (ord.off_large2 >= n) {
            k_set_split_if_end<V><<<1, 1, 0, ctx.stream>>>(s);
            PGGC_LAUNCH_CHECK();
        }
    }

    void afterburner(float pm) {
        ABArgs<W> a;
        a.g = g.view();
        a.part = part.p;
        a.dest = dest.p;
        a.gain = gain.p;
        a.pm = pm;
        a.cand = cand.p;
        a.keep = keep.p;
        a.sc = sc.p;
        a.prof = ctx.prof_counter("afterburner_warp");
        {
            ProfScope ps(ctx, "afterburner_warp");
            if (cls.count > 0) {
                int grid = grid_for(ctx, ceil_div(cls.count, 32), 1, 16);
                int grid_t = grid_for(ctx, ceil_div(cls.count, 256), 1, 16);
                k_afterburner_thr<W, 8><<<grid_t, 256, 0, ctx.stream>>>(a, dev_range(cls.list, cls.off + 0, cls.off + 2));
                PGGC_LAUNCH_CHECK();
                k_afterburner_thr<W, 16><<<grid_t, 256, 0, ctx.stream>>>(a, dev_range(cls.list, cls.off + 2, cls.off + 3));
                PGGC_LAUNCH_CHECK();
                k_afterburner_small<W, 32, 4><<<grid, 256, 0, ctx.stream>>>(
                    a, dev_range(cls.list, cls.off + 3, cls.off + 4));
                PGGC_LAUNCH_CHECK();
            }
            if (ord.off_large2 > ord.off_large) {
                int grid = grid_for(ctx, ceil_div(ord.off_large2 - ord.off_large, 8), 1, 16);
                k_afterburner_grp<W, 32><<<grid, 256, 0, ctx.stream>>>(
                    a, host_range(ord.order1.p, ord.off_large, ord.off_large2));
                PGGC_LAUNCH_CHECK();
            }
        }
        i64 nm = n - ord.off_large2;
        if (nm > 0) {
            ProfScope ps(ctx, "afterburner_block");
            a.prof = nullptr;
            k_afterburner_block<W><<<(int)std::min<i64>(nm, (i64)ctx.num_sms * 2), 1024, 0, ctx.stream>>>(
                a, host_range(ord.order1.p, ord.off_large2, n));
            PGGC_LAUNCH_CHECK();
        }
        PGGC_CUDA(cudaMemsetAsync(&sc.p->new_hint, 0, sizeof(unsigned long long), ctx.stream));
        scan_apply(ctx, KeepFlag{cand.p, keep.p}, MoveEpi{cand.p, dest.p, moves.p, &sc.p->new_hint}, n,
                   &sc.p->num_cand, &sc.p->num_moves);
    }

    void set_new_cluster_ids(i64 nmoves_host, i32* constraint) {
        LMScalars<V>* s = sc.p;
        scan_apply(ctx, NewFlag{moves.p, dest.p}, ListEpi{moves.p, newl.p}, nmoves_host, nullptr, &s->num_new);
        k_prep_new<V><<<1, 1, 0, ctx.stream>>>(s);
        PGGC_LAUNCH_CHECK();
        k_clear_has<V><<<grid_for(ctx, cap, 256), 256, 0, ctx.stream>>>(has.p, s);
        PGGC_LAUNCH_CHECK();
        k_mark_has<V><<<grid_for(ctx, n, 256), 256, 0, ctx.stream>>>(has.p, part.p, n, s);
        PGGC_LAUNCH_CHECK();
        scan_apply(ctx, UnusedFlag{has.p}, IdxEpi{avail.p}, cap, &s->avail_k, &s->num_avail);
        k_assign_new<V><<<grid_for(ctx, nmoves_host, 256), 256, 0, ctx.stream>>>(
            newl.p, avail.p, dest.p, part.p, constraint, td_curr.p, s, cap, ctx.d_err);
        PGGC_LAUNCH_CHECK();
        k_finish_new<V><<<1, 1, 0, ctx.stream>>>(s, cap);
        PGGC_LAUNCH_CHECK();
    }

    void perform_moves(i64 nm, double lambda, i64 label_bound) {
        auto gv = g.view();
        k_apply_moves<W><<<grid_for(ctx, nm, 256), 256, 0, ctx.stream>>>(
            gv, moves.p, nm, dest.p, part.p, td_curr.p, ctx.d_err, filt_on ? csize.p : nullptr,
            filt_on ? moved_at.p : nullptr, ctx.filt.stamp);
        PGGC_LAUNCH_CHECK();
        if (!cdata_init) {
            cdata_init = true;
            own_weights_impl<W>(ctx, g, ord, part.p, pvals.p, 0, nullptr, nullptr, &cls);
            fill<i32>(ctx, dest.p, n, NULL_PART);
        } else if (nm * 16 > n) {
            // push costs nm * avg_deg edges, pull about n * n / nm
            const double avg_deg = (double)g.nnz / (double)std::max<i64>(n, 1);
            if ((double)nm * (double)nm * avg_deg > 4.0 * (double)n * (double)n) {
                k_mark_movers<<<grid_for(ctx, nm, 256), 256, 0, ctx.stream>>>(moves.p, nm, flags.p);
                PGGC_LAUNCH_CHECK();
                k_mark_pull<W><<<grid_for(ctx, ceil_div(n, 8), 1, 16), 256, 0, ctx.stream>>>(gv, flags.p);
                PGGC_LAUNCH_CHECK();
            } else {
                k_mark_affected<W><<<grid_for(ctx, ceil_div(nm, 8), 1, 16), 256, 0, ctx.stream>>>(gv, moves.p, nm,
                                                                                                flags.p);
                PGGC_LAUNCH_CHECK();
            }
            own_weights_impl<W>(ctx, g, ord, part.p, pvals.p, 1, flags.p, dest.p, &cls);
        } else {
            // few moves: list the affected vertices once and recompute only them
            // (the same per-vertex association as the class kernels)
            if (++epoch == 0) {
                PGGC_CUDA(cudaMemsetAsync(stamp.p, 0, sizeof(u32) * std::max<i64>(n, 1), ctx.stream));
                epoch = 1;
            }
            PGGC_CUDA(cudaMemsetAsync(aff_cnt.p, 0, sizeof(i64), ctx.stream));
            k_mark_list<W><<<grid_for(ctx, ceil_div(nm, 8), 1, 16), 256, 0, ctx.stream>>>(gv, moves.p, nm, stamp.p,
                                                                                         epoch, aff.p, aff_cnt.p,
                                                                                         flags.p, ord.off_large2 < n);
            PGGC_LAUNCH_CHECK();
            own_weights_list<W>(ctx, g, ord, part.p, pvals.p, aff.p, aff_cnt.p, std::min<i64>(n, nm * (1 + ord.max_deg)),
                                flags.p, dest.p);
        }
        update_objective_dev(lambda, label_bound);
    }

    void update_objective_dev(double lambda, i64 label_bound) {
        LMScalars<V>* s = sc.p;
        if constexpr (std::is_same<V, i64>::value) {
            sum_i64(ctx, PvI64In{pvals.p}, n, &s->pval_sum);
            sum_i64(ctx, SqIn<i64>{td_curr.p, &s->label_count}, label_bound, &s->sumsq_i);
        } else {
            det_reduce(ctx, DArrIn{pvals.p}, n, &s->pval_sum);
            det_reduce(ctx, SqIn<double>{td_curr.p, &s->label_count}, label_bound, &s->sumsq_d);
        }
        k_objective<V><<<1, 1, 0, ctx.stream>>>(s, lambda);
        PGGC_LAUNCH_CHECK();
    }

    void copy_if_improved(i32* best_part, V* td_best, i64 label_bound) {
        LMScalars<V>* s = sc.p;
        k_copy_if_improved<V><<<grid_for(ctx, std::max<i64>(n, label_bound), 256), 256, 0, ctx.stream>>>(
            best_part, part.p, td_best, td_curr.p, pvals_clone.p, pvals.p, n, s);
        PGGC_LAUNCH_CHECK();
    }

    // strict prefix selection over moves[0..k); writes sc.num_moves
    void strict_filter(i64 k, i64 split_host, float pm) {
        auto gv = g.view();
        prio.p = ctx.ws_get<i32>(S_PRIO, std::max<i64>(n, 1));
        fill<i32>(ctx, prio.p, n, (i32)std::min<i64>(n + 1, 2147483647));
        k_prio<<<grid_for(ctx, k, 256), 256, 0, ctx.stream>>>(moves.p, k, prio.p);
        PGGC_LAUNCH_CHECK();
        DBuf<V> nb(ctx, k);
        if (split_host > 0) {
            k_strict_nb_warp<W><<<grid_for(ctx, ceil_div(split_host, 8), 1, 16), 256, 0, ctx.stream>>>(
                gv, moves.p, 0, split_host, prio.p, dest.p, part.p, nb.p);
            PGGC_LAUNCH_CHECK();
        }
        if (k > split_host) {
            k_strict_nb_block<W><<<(int)std::min<i64>(k - split_host, (i64)ctx.num_sms * 2), 1024, 0, ctx.stream>>>(
                gv, moves.p, split_host, k, prio.p, dest.p, part.p, nb.p);
            PGGC_LAUNCH_CHECK();
        }
        DBuf<u64> kd(ctx, k), kp(ctx, k), kt(ctx, k);
        DBuf<i32> od(ctx, k), op(ctx, k), ot(ctx, k);
        k_strict_keys<V><<<grid_for(ctx, k, 256), 256, 0, ctx.stream>>>(moves.p, k, dest.p, part.p, kd.p, kp.p, od.p,
                                                                        op.p);
        PGGC_LAUNCH_CHECK();
        radix_sort_pairs<i32>(ctx, kd.p, od.p, k, 32, 64, kt.p, ot.p);
        radix_sort_pairs<i32>(ctx, kp.p, op.p, k, 32, 64, kt.p, ot.p);
        DBuf<V> wd(ctx, k), wp(ctx, k), Ed(ctx, k + 1), Ep(ctx, k + 1);
        k_gather_vw<V><<<grid_for(ctx, k, 256), 256, 0, ctx.stream>>>(od.p, moves.p, g.vtx_w.p, k, wd.p);
        PGGC_LAUNCH_CHECK();
        k_gather_vw<V><<<grid_for(ctx, k, 256), 256, 0, ctx.stream>>>(op.p, moves.p, g.vtx_w.p, k, wp.p);
        PGGC_LAUNCH_CHECK();
        if constexpr (std::is_same<V, i64>::value) {
            scan_apply(ctx, I64ArrIn{wd.p, k}, I64ExclOut{Ed.p}, k + 1, nullptr, nullptr);
            scan_apply(ctx, I64ArrIn{wp.p, k}, I64ExclOut{Ep.p}, k + 1, nullptr, nullptr);
        } else {
            // exclusive prefix = shifted canonical inclusive scan
            PGGC_CUDA(cudaMemsetAsync(Ed.p, 0, sizeof(double), ctx.stream));
            PGGC_CUDA(cudaMemsetAsync(Ep.p, 0, sizeof(double), ctx.stream));
            det_scan(ctx, DArrIn{wd.p}, Ed.p + 1, k);
            det_scan(ctx, DArrIn{wp.p}, Ep.p + 1, k);
        }
        DBuf<double> oc(ctx, k), pre(ctx, k);
        k_strict_oc<W><<<grid_for(ctx, k, 256), 256, 0, ctx.stream>>>(gv, moves.p, k, dest.p, part.p, gain.p, nb.p, kd.p,
                                                                       Ed.p, kp.p, Ep.p, pm, oc.p);
        PGGC_LAUNCH_CHECK();
        det_scan(ctx, DArrIn{oc.p}, pre.p, k);
        k_strict_argmax<V><<<1, 1024, 0, ctx.stream>>>(pre.p, k, sc.p);
        PGGC_LAUNCH_CHECK();
    }

    // relabel_contiguously of the best partition, queued without a host round
    // trip: L bounds its label count; the new count lands in sc.relabel_count
    // and the compacted volumes in td2 (copied back by the caller)
    void relabel_async(i32* best_part, const V* td_best, i64 L, DBuf<V>& td2) {
        DBuf<unsigned char> used(ctx, std::max<i64>(L, 1));
        DBuf<i32> newid(ctx, std::max<i64>(L, 1));
        td2 = DBuf<V>(ctx, std::max<i64>(L, 1));
        PGGC_CUDA(cudaMemsetAsync(used.p, 0, std::max<i64>(L, 1), ctx.stream));
        k_mark_used<<<grid_for(ctx, n, 256), 256, 0, ctx.stream>>>(used.p, best_part, n, L);
        PGGC_LAUNCH_CHECK();
        scan_apply(ctx, UsedFlag{used.p}, RelabelEpi<V>{newid.p, td_best, td2.p}, L, nullptr, &sc.p->relabel_count);
        k_remap<<<grid_for(ctx, n, 256), 256, 0, ctx.stream>>>(best_part, n, newid.p, L);
        PGGC_LAUNCH_CHECK();
    }
};

template <class W>
void local_move(Context& ctx, const Graph<W>& g, const Ordering& ord, i32* best_part,
                ClusterState<typename Traits<W>::V>& best, bool is_initial, bool constrained, i32* constraint,
                bool enable_sa, bool strict, int sweep_limit, MoveStats* stats, bool reuse_pvals) {
    using V = typename Traits<W>::V;
    const i64 n = g.n;
    if (n == 0) return;
    if (best.capacity < best.label_count) throw InvalidArg("cluster state capacity below label count");
    ProfScope whole(ctx, strict ? "local_move_strict" : "local_move");
    Mover<W> m(ctx, g, ord, best.capacity);
    const float pm = (float)best.lambda;
    // curr_state.copy(best_state); part = best_part (src/local_mover.cpp:1365-1368)
    LMScalars<V> h{};
    h.label_count = best.label_count;
    h.best_label_count = best.label_count;
    h.uncut = best.uncut;
    h.best_uncut = best.uncut;
    h.obj = best.obj;
    h.best_obj = best.obj;
    copy_d2d(ctx, m.part.p, best_part, n);
    copy_d2d(ctx, m.td_curr.p, best.total_deg.p, best.label_count);
    fill<i32>(ctx, m.dest.p, n, NULL_PART);
    if (!strict) m.filter_init();
    ctx.prof_tag = "init";
    // the caller's partition is the previous local move's output on this graph:
    // its own-cluster weights are the ones left in pvals_clone
    const bool reuse = reuse_pvals && !is_initial && ctx.pv_uid == g.uid && ctx.pv_n == n &&
                       ctx.pv_ptr == (const void*)m.pvals_clone.p;
    ctx.pv_uid = 0;
    if (!is_initial) {
        m.cdata_init = true;
        if (reuse) copy_d2d(ctx, m.pvals.p, m.pvals_clone.p, n);
        else own_weights_impl<W>(ctx, g, ord, m.part.p, m.pvals.p, 0, nullptr, nullptr, &m.cls);
    } else {
        m.cdata_init = false;
        PGGC_CUDA(cudaMemsetAsync(m.pvals.p, 0, sizeof(V) * n, ctx.stream));
    }
    PGGC_CUDA(cudaMemcpyAsync(m.sc.p, &h, sizeof(h), cudaMemcpyHostToDevice, ctx.stream));
    if (!is_initial) {
        if constexpr (std::is_same<V, i64>::value) sum_i64(ctx, PvI64In{m.pvals.p}, n, &m.sc.p->last_pval);
        else det_reduce(ctx, DArrIn{m.pvals.p}, n, &m.sc.p->last_pval);
    }
    copy_d2d(ctx, m.pvals_clone.p, m.pvals.p, n);

    i64 label_bound = best.label_count;  // host upper bound of sc.label_count
    int sweeps = 0;
    i64 total_moves = 0;
    auto budget = [&]() { return sweep_limit < 0 || sweeps < sweep_limit; };

    if (!strict) {
        const float ratios[2] = {0.75f, 0.25f};
        const int limits[2] = {4, 2};
        int iter_count = 0;
        for (int x = 0; x < 2; x++) {
            float fr = enable_sa ? ratios[x] : 0.0f;
            int count = 0;
            while (count++ < limits[x]) {
                if (!budget()) break;
                sweeps++;
                iter_count++;
                ctx.prof_tag = iter_count == 1 ? (enable_sa ? "sa_first" : "first") : "later";
                m.filter_pre(iter_count - 1, best.vol_total);
                auto a = m.sel_args(fr, !m.cdata_init, constraint, m.td_curr.p, m.part.p, m.pvals.p, m.dest.p,
                                    m.gain.p, &m.sc.p->label_count, pm);
                m.label_bound_host = label_bound;
                m.launch_select(a, constrained);
                {
                    ProfScope pc(ctx, "lm_compact");
                    m.compact_candidates();
                }
                m.afterburner(pm);
                m.filter_post();
                const LMScalars<V>* hs;
                {
                    // the GPU's idle time while the host reads the sweep's counts
                    ProfScope pr(ctx, "lm_roundtrip");
                    hs = (const LMScalars<V>*)ctx.readback(m.sc.p, sizeof(LMScalars<V>));
                }
                i64 ncand = hs->num_cand, nm = hs->num_moves;
                const bool any_new = hs->new_hint != 0;
                if (ncand == 0 || nm == 0) break;
                // set_new_cluster_ids is a no-op without NEW_PART moves (src/local_mover.cpp:236)
                if ((iter_count > 1 || !is_initial) && any_new) {
                    ProfScope pn(ctx, "lm_newids");
                    m.set_new_cluster_ids(nm, constrained ? constraint : nullptr);
                }
                label_bound = std::min<i64>(label_bound + nm, m.cap);
                {
                    ProfScope pm_(ctx, "lm_moves");
                    m.perform_moves(nm, best.lambda, label_bound);
                }
                {
                    ProfScope pk(ctx, "lm_copy");
                    m.copy_if_improved(best_part, best.total_deg.p, label_bound);
                }
                total_moves += nm;
            }
        }
    } else {
        for (int it = 0; it < 6; it++) {
            if (!budget()) break;
            sweeps++;
            ctx.prof_tag = "strict";
            auto a = m.sel_args(0.0f, !m.cdata_init, constraint, m.td_curr.p, m.part.p, m.pvals.p, m.dest.p, m.gain.p,
                                &m.sc.p->label_count, pm);
            m.label_bound_host = label_bound;
            m.launch_select(a, constrained);
            m.compact_candidates();
            const LMScalars<V>* hs = (const LMScalars<V>*)ctx.readback(m.sc.p, sizeof(LMScalars<V>));
            i64 k = hs->num_cand, split = hs->split;
            if (k == 0) break;
            copy_d2d(ctx, m.moves.p, m.cand.p, k);
            PGGC_CUDA(cudaMemcpyAsync(&m.sc.p->num_moves, &m.sc.p->num_cand, sizeof(i64), cudaMemcpyDeviceToDevice,
                                      ctx.stream));
            if (it > 0 || !is_initial) m.set_new_cluster_ids(k, constrained ? constraint : nullptr);
            label_bound = std::min<i64>(label_bound + k, m.cap);
            m.strict_filter(k, split, pm);
            i64 nm = ctx.read1(&m.sc.p->num_moves);
            if (nm == 0) break;
            m.perform_moves(nm, best.lambda, label_bound);
            m.copy_if_improved(best_part, best.total_deg.p, label_bound);
            fill<i32>(ctx, m.dest.p, n, NULL_PART);
            total_moves += nm;
        }
    }
    ctx.prof_tag = "end";
    // the best state's scalars and the device error word in one round trip
    PGGC_CUDA(cudaMemcpyAsync(&m.sc.p->err, ctx.d_err, sizeof(int), cudaMemcpyDeviceToDevice, ctx.stream));
    const LMScalars<V>* hs = (const LMScalars<V>*)ctx.readback(m.sc.p, sizeof(LMScalars<V>));
    const int err = hs->err;
    best.label_count = hs->best_label_count;
    best.uncut = hs->best_uncut;
    best.obj = hs->best_obj;
    ctx.raise_device_error(err);
    DBuf<V> td2;
    m.relabel_async(best_part, best.total_deg.p, best.label_count, td2);
    best.label_count = ctx.read1(&m.sc.p->relabel_count);
    copy_d2d(ctx, best.total_deg.p, td2.p, best.label_count);
    ctx.prof_tag = nullptr;
    ctx.pv_uid = g.uid;
    ctx.pv_ptr = m.pvals_clone.p;
    ctx.pv_n = n;
    if (stats) {
        stats->sweeps += sweeps;
        stats->moves += total_moves;
    }
}

template <class W>
i64 select_pass(Context& ctx, const Graph<W>& g, const Ordering& ord, const i32* part,
                const typename Traits<W>::V* pvals, ClusterState<typename Traits<W>::V>& cs, i32* dest, float* gain,
                float filter_ratio, bool initial, bool constrained, const i32* constraint) {
    using V = typename Traits<W>::V;
    Mover<W> m(ctx, g, ord, cs.capacity);
    LMScalars<V> h{};
    h.label_count = cs.label_count;
    PGGC_CUDA(cudaMemcpyAsync(m.sc.p, &h, sizeof(h), cudaMemcpyHostToDevice, ctx.stream));
    auto a = m.sel_args(filter_ratio, initial, constraint, cs.total_deg.p, part, pvals, dest, gain,
                        &m.sc.p->label_count, (float)cs.lambda);
    m.label_bound_host = cs.label_count;
    m.launch_select(a, constrained);
    scan_apply(ctx, CandFlag{ord.order1.p, dest}, CandEpi{ord.order1.p, m.cand.p, -1, nullptr}, g.n, nullptr,
               &m.sc.p->num_cand);
    i64 k = ctx.read1(&m.sc.p->num_cand);
    ctx.check_device_error();
    return k;
}

#define PGGC_INST_LM(W)                                                                                             \
    template ClassLists graph_class_lists<W>(Context&, const Graph<W>&, const Ordering&);                           \
    template void local_move<W>(Context&, const Graph<W>&, const Ordering&, i32*, ClusterState<Traits<W>::V>&, bool, \
                                bool, i32*, bool, bool, int, MoveStats*, bool);                                     \
    template i64 select_pass<W>(Context&, const Graph<W>&, const Ordering&, const i32*, const Traits<W>::V*,         \
                                ClusterState<Traits<W>::V>&, i32*, float*, float, bool, bool, const i32*);          \
    template void own_weights<W>(Context&, const Graph<W>&, const Ordering&, const i32*, Traits<W>::V*);          \
    template const Traits<W>::V* row_sums<W>(Context&, const Graph<W>&);
PGGC_INST_LM(i32)
PGGC_INST_LM(float)

}  // namespace pggc
