// contract.cu -- build_coarse_graph (src/contract.cpp:234-336) for sm_100a.
//
// Pipeline:
//  1. one pass over the vertices counts members and the edge bound
//     (sum of member degrees) of every coarse vertex;
//  2. scans give member offsets and per-coarse-vertex scratch offsets; members
//     are scattered (counting sort by coarse id) and their degrees prefix-summed
//     so each coarse vertex owns one flat member-edge list;
//  3. flattening: one coalesced pass over the CSR writes every edge's coarse
//     key (or -1 inside the coarse vertex: dropped self-loops,
//     src/contract.cpp:191,209) and weight at its flat position;
//  4. one pass sorts the rows into buckets; hashed merge of the keys reads each
//     row as a contiguous stream: a warp per row with bound <= 256 (per-warp
//     shared table, __match_any_sync chunk pre-aggregation), a block with a
//     2048- or 8192-slot shared table up to 4096 distinct candidates, a
//     1024-thread block with a 16384-slot shared table above that, and a block
//     with a global table for the rows that overflow it; on coarse graphs of at
//     most 8192 vertices the block rows use a table indexed by coarse id
//     instead; weights are summed exactly (int64 / FP64);
//  5. a prefix sum of the unique counts gives the coarse row offsets;
//  6. each row is sorted by column and written out: register ranks (<= 32
//     entries), chunk ranks (sorted 32-key chunks plus binary searches into the
//     other chunks; warp <= 256, block <= 1024 entries), bitmap ranks when the
//     coarse graph has at most 262,144 vertices (and for rows above 1024
//     entries up to 928,768 vertices), block bitonic sort (<= 4096) and LSD
//     radix sort above.
// The output is the canonical (row, col)-sorted coarse CSR.
#include <optional>
#include "kernels.cuh"
#include "bulk.cuh"

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

__global__ void k_scatter_members(const i32* vcmap, i64 n, i64* cursor, i32* members, i64* memberpos) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
        i32 c = vcmap[i];
        i64 pos = (i64)::atomicAdd((unsigned long long*)&cursor[c], 1ull);
        members[pos] = (i32)i;
        memberpos[i] = pos;
    }
}

// Flattening: every fine edge (u, v) is written once, at its position in its
// coarse row's flat member-edge list (P[memberpos[u]] + rank within u's row),
// as the coarse key vcmap[v] (-1 for an edge inside the coarse vertex, a
// self-loop of the coarse graph) and its weight.  A warp streams the edge range
// of 32 consecutive vertices with coalesced loads; each lane finds its edge's
// source among the 32 by a 5-step shuffle search of the row offsets.  After
// this pass the hashing kernels read their rows as contiguous streams.
template <class W>
__global__ void __launch_bounds__(256) k_flatten(DGraph<W> g, const i32* vcmap, const i64* P, const i64* memberpos,
                                                 i32* fkey, W* fw) {
    const int l = lane_id();
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
    for (i64 u0 = gw * 32; u0 < g.n; u0 += nw * 32) {
        const i64 uu = u0 + l;
        const bool has = uu < g.n;
        const i64 R = has ? g.rowptr[uu] : (i64)1 << 62;  // row start of the lane's vertex
        const i64 B = has ? P[memberpos[uu]] : 0;          // its flat base
        const i32 C = has ? vcmap[uu] : -1;                // its coarse id
        const i64 e0 = g.rowptr[u0];
        const i64 e1 = g.rowptr[min(u0 + 32, g.n)];
        // FL_UNROLL chunks of 32 edges per iteration: their loads are issued
        // together so that several gathers are in flight per warp
        constexpr int FL_UNROLL = 4;
        for (i64 j0 = e0; j0 < e1; j0 += 32 * FL_UNROLL) {
            i32 col[FL_UNROLL];
            W wv[FL_UNROLL];
#pragma unroll
            for (int k = 0; k < FL_UNROLL; k++) {
                const i64 j = j0 + 32 * k + l;
                col[k] = j < e1 ? g.col[j] : 0;
                wv[k] = (g.w && j < e1) ? g.w[j] : W(0);
            }
            i32 cv[FL_UNROLL];
#pragma unroll
            for (int k = 0; k < FL_UNROLL; k++) cv[k] = j0 + 32 * k + l < e1 ? vcmap[col[k]] : 0;
#pragma unroll
            for (int k = 0; k < FL_UNROLL; k++) {
                const i64 j = j0 + 32 * k + l;
                // largest L with R_L <= j (vertices with no edges share R with the next)
                int lo = 0;
#pragma unroll
                for (int step = 16; step >= 1; step >>= 1) {
                    const int cand = lo + step;
                    const i64 rc = __shfl_sync(FULL, R, cand & 31);
                    if (cand < 32 && rc <= j) lo = cand;
                }
                const i64 rs = __shfl_sync(FULL, R, lo);
                const i64 bs = __shfl_sync(FULL, B, lo);
                const i32 cs = __shfl_sync(FULL, C, lo);
                if (j < e1) {
                    const i64 q = bs + (j - rs);
                    fkey[q] = cv[k] == cs ? -1 : cv[k];
                    if (g.w) fw[q] = wv[k];
                }
            }
        }
    }
}

// Flattening of graphs with long rows (mean degree >= FLW_MIN_DEG: the dense
// coarse levels, a few thousand vertices of thousands of edges): a warp per
// vertex copies its row, 4 chunks of 32 edges in flight, so the work spreads
// over n warps instead of n / 32.
constexpr i64 FLW_MIN_DEG = 128;

template <class W>
__global__ void __launch_bounds__(256) k_flatten_wide(DGraph<W> g, const i32* vcmap, const i64* P,
                                                      const i64* memberpos, i32* fkey, W* fw) {
    const int l = lane_id();
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
    for (i64 u = gw; u < g.n; u += nw) {
        const i64 b = g.rowptr[u], e = g.rowptr[u + 1];
        const i64 base = P[memberpos[u]] - b;  // flat position of edge j: base + j
        const i32 cu = vcmap[u];
        constexpr int UNR = 4;
        for (i64 j0 = b; j0 < e; j0 += 32 * UNR) {
            i32 col[UNR];
            W wv[UNR];
#pragma unroll
            for (int k = 0; k < UNR; k++) {
                const i64 j = j0 + 32 * k + l;
                col[k] = j < e ? g.col[j] : 0;
                wv[k] = (g.w && j < e) ? g.w[j] : W(0);
            }
#pragma unroll
            for (int k = 0; k < UNR; k++) {
                const i64 j = j0 + 32 * k + l;
                if (j < e) {
                    const i32 cv = vcmap[col[k]];
                    fkey[base + j] = cv == cu ? -1 : cv;
                    if (g.w) fw[base + j] = wv[k];
                }
            }
        }
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
    const i32* fkey;     // flattened coarse keys (-1: inside the coarse vertex) [nnz]
    const W* fw;         // flattened weights [nnz] (unused for unit weights)
    i32* out_key;        // scratch, indexed by P[cstart[c]] + k
    V* out_val;
    i64* ucount;         // unique neighbours per coarse vertex
    int* err;
    u32 probe_cap;       // fault-injection cap on hash probes (0: none)
};

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

// insert that gives up after CT_TRY_PROBES probes instead of latching an error
// (the caller falls back to a larger table); a run that long means the table
// is close to full, where further probing would cost O(table) per insert
constexpr u32 CT_TRY_PROBES = 64;
template <class V>
__device__ __forceinline__ bool ctable_try_add(i32* keys, V* vals, u32 mask, i32 c, V x) {
    u32 s = xorshift32((u32)c) & mask;
    volatile i32* vk = keys;
    for (u32 probe = 0; probe < CT_TRY_PROBES && probe <= mask; probe++) {
        i32 k = vk[s];
        if (k == c) {
            cvatomic_add(&vals[s], x);
            return true;
        }
        if (k == -1) {
            i32 old = atomicCAS(&keys[s], -1, c);
            if (old == -1 || old == c) {
                cvatomic_add(&vals[s], x);
                return true;
            }
        }
        s = (s + 1) & mask;
    }
    return false;
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

// one 32-entry chunk of a coarse row's flat list: q = base + lane; the
// warp pre-aggregates equal keys with __match_any_sync before the table insert
template <class W>
__device__ __forceinline__ typename Traits<W>::V cchunk_load(const CArgs<W>& a, i64 q, i64 qend, i32& key,
                                                             bool& keep, bool& leader) {
    using V = typename Traits<W>::V;
    const bool valid = q < qend;
    const i32 u = valid ? a.fkey[q] : -1;
    const V wv = (valid && a.g.w) ? V(a.fw[q]) : V(0);
    keep = valid && u >= 0;
    key = keep ? u : (i32)(0x80000000u | lane_id());
    const unsigned peers = __match_any_sync(FULL, key);
    leader = keep && ((peers & lanemask_lt()) == 0);
    return a.g.w ? cgroup_sum<V>(peers, wv, leader) : V(__popc(peers));
}

template <class W>
__device__ __forceinline__ void cchunk(const CArgs<W>& a, i64 q, i64 qend, i32* keys, typename Traits<W>::V* vals,
                                       u32 mask) {
    i32 key;
    bool keep, leader;
    auto s = cchunk_load(a, q, qend, key, keep, leader);
    if (leader) ctable_add(keys, vals, mask, key, s, a.err, a.probe_cap);
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
        for (i64 q = q0 + l; q - l < q1; q += 32) cchunk(a, q, q1, keys, vals, T - 1);
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
// the bucket's largest table) or, with GLOBAL, in a per-block global region.
// With OVF (shared tables of gcap slots smaller than 2U), a row whose distinct
// keys do not fit is appended to `ovf_list` for the global-table pass instead.
template <class W, bool GLOBAL, int THREADS = 256, bool OVF = false>
__global__ void __launch_bounds__(THREADS) k_contract_block(CArgs<W> a, const i32* list, const i64* d_count, i32* gkeys,
                                                            typename Traits<W>::V* gvals, i64 gcap, i64 nc,
                                                            i32* ovf_list = nullptr, i64* ovf_count = nullptr) {
    using V = typename Traits<W>::V;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ unsigned long long wcount;
    __shared__ int full;
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
        if (OVF && T > (u32)gcap) T = (u32)gcap;
        for (u32 s = threadIdx.x; s < T; s += THREADS) {
            keys[s] = -1;
            vals[s] = V(0);
        }
        if (threadIdx.x == 0) {
            wcount = 0;
            full = 0;
        }
        __syncthreads();
        if (OVF) {
            for (i64 q = q0 + (i64)w * 32 + l; q - l < q1; q += THREADS) {
                i32 key;
                bool keep, leader;
                auto sv = cchunk_load(a, q, q1, key, keep, leader);
                if (leader && !ctable_try_add(keys, vals, T - 1, key, sv)) full = 1;
                if (__any_sync(FULL, *(volatile int*)&full != 0)) break;
            }
            __syncthreads();
            if (full) {
                if (threadIdx.x == 0) {
                    i64 k = (i64)::atomicAdd((unsigned long long*)ovf_count, 1ull);
                    ovf_list[k] = c;
                }
                __syncthreads();
                continue;
            }
        } else {
            for (i64 q = q0 + (i64)w * 32 + l; q - l < q1; q += THREADS) cchunk(a, q, q1, keys, vals, T - 1);
        }
        __syncthreads();
        for (u32 s0 = w * 32; s0 < T; s0 += THREADS) {
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

// ---- block rows of small coarse graphs: a dense table ------------------------
// With at most DENSE_NC coarse vertices the table is indexed by coarse id:
// values plus a presence bitmap in shared memory (no keys, no probing, no
// overflow), and the row is written out in ascending column order by a scan
// of the bitmap.  The launch takes 8 nc + nc / 8 bytes of shared memory
// instead of the hash tables' 24-192 KB, so more blocks share an SM.
constexpr i64 DENSE_NC = 8192;

template <class W, int THREADS>
__global__ void __launch_bounds__(THREADS) k_contract_dense(CArgs<W> a, const i32* list, const i64* d_count, int nc) {
    using V = typename Traits<W>::V;
    constexpr int NW = THREADS / 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ u32 wsum[NW];
    V* vals = (V*)smem_raw;
    u32* pres = (u32*)(smem_raw + sizeof(V) * (size_t)nc);
    const int nwords = (nc + 31) >> 5;
    const int l = lane_id(), w = threadIdx.x >> 5, tid = threadIdx.x;
    const int per = (nwords + THREADS - 1) / THREADS;
    const int w0 = min(tid * per, nwords), w1 = min(w0 + per, nwords);
    const i64 count = *d_count;
    for (i64 x = blockIdx.x; x < count; x += gridDim.x) {
        const i32 c = list[x];
        const i64 q0 = a.P[a.cstart[c]], q1 = a.P[a.cstart[c + 1]];
        for (int s = tid; s < nc; s += THREADS) vals[s] = V(0);
        for (int s = tid; s < nwords; s += THREADS) pres[s] = 0u;
        __syncthreads();
        for (i64 q = q0 + (i64)w * 32 + l; q - l < q1; q += THREADS) {
            i32 key;
            bool keep, leader;
            const V sv = cchunk_load(a, q, q1, key, keep, leader);
            if (leader) {
                cvatomic_add(&vals[key], sv);
                atomicOr(&pres[key >> 5], 1u << (key & 31));
            }
        }
        __syncthreads();
        // exclusive prefix of the word popcounts over the threads' word ranges
        u32 local = 0;
        for (int q = w0; q < w1; q++) local += (u32)__popc(pres[q]);
        u32 incl = local;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const u32 t = __shfl_up_sync(FULL, incl, d);
            if (l >= d) incl += t;
        }
        if (l == 31) wsum[w] = incl;
        __syncthreads();
        u32 base = 0, tot = 0;
#pragma unroll
        for (int q = 0; q < NW; q++) {
            const u32 v = wsum[q];
            base += q < w ? v : 0u;
            tot += v;
        }
        u32 pos = base + incl - local;
        for (int q = w0; q < w1; q++) {
            u32 bits = pres[q];
            while (bits) {
                const int b = __ffs(bits) - 1;
                bits &= bits - 1;
                const i32 key = q * 32 + b;
                a.out_key[q0 + pos] = key;
                a.out_val[q0 + pos] = vals[key];
                pos++;
            }
        }
        if (tid == 0) a.ucount[c] = (i64)tot;
        __syncthreads();
    }
}

// ---- coarse rows that overflow a 16384-slot shared table: the row's flat list
// split across blocks ---------------------------------------------------------
// Per round of up to `count` such rows, each owning a global table of `gcap`
// slots: clear; insert, one block per chunk of CSPLIT_CHUNK flat entries (keys
// and weights staged in shared memory by TMA bulk copies); write, blocks over
// table slots appending the row's unique entries at q0 + (a per-row atomic
// counter, ucount[c]).  The order inside the row's scratch range depends on
// the blocks' race, but the placement sorts every row, so the coarse CSR is
// the same; the sums are exact.
constexpr int CSPLIT_CHUNK = 8192;
constexpr int CSPLIT_THREADS = 256;
constexpr size_t CSPLIT_SMEM = 16 + 2 * sizeof(i32) * (CSPLIT_CHUNK + 4);

template <class W>
__global__ void k_csplit_clear(CArgs<W> a, const i32* list, i64 count, i64 gcap, i32* keys,
                               typename Traits<W>::V* vals) {
    using V = typename Traits<W>::V;
    const i64 total = count * gcap;
    for (i64 x = blockIdx.x * (i64)blockDim.x + threadIdx.x; x < total; x += (i64)gridDim.x * blockDim.x) {
        keys[x] = -1;
        vals[x] = V(0);
    }
    for (i64 k = blockIdx.x * (i64)blockDim.x + threadIdx.x; k < count; k += (i64)gridDim.x * blockDim.x)
        a.ucount[list[k]] = 0;
}

template <class W>
__device__ __forceinline__ u32 csplit_slots(const CArgs<W>& a, i32 c, i64 nc, i64 gcap, i64& q0, i64& q1) {
    q0 = a.P[a.cstart[c]];
    q1 = a.P[a.cstart[c + 1]];
    const i64 U = min(q1 - q0, nc);
    u32 T = next_pow2_u32((u32)(2 * (U > 1 ? U : 1)));
    return T > (u32)gcap ? (u32)gcap : T;
}

template <class W>
__global__ void __launch_bounds__(CSPLIT_THREADS) k_csplit_insert(CArgs<W> a, const i32* list, i64 count, i64 gcap,
                                                                 i32* gkeys, typename Traits<W>::V* gvals, i64 nc) {
    using V = typename Traits<W>::V;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned long long* bar = (unsigned long long*)smem_raw;
    i32* s_key = (i32*)(smem_raw + 16);
    W* s_w = (W*)(smem_raw + 16 + sizeof(i32) * (CSPLIT_CHUNK + 4));
    const i64 k = blockIdx.y;
    if (k >= count) return;
    const i32 c = list[k];
    i64 q0, q1;
    const u32 T = csplit_slots(a, c, nc, gcap, q0, q1);
    const i64 j0 = q0 + (i64)blockIdx.x * CSPLIT_CHUNK;
    if (j0 >= q1) return;
    const i64 j1 = min(q1, j0 + (i64)CSPLIT_CHUNK);
    const bool has_w = a.g.w != nullptr;
    if (!stage_rows(a.fkey, has_w ? a.fw : (const W*)nullptr, j0, j1, s_key, s_w, bar, a.err)) return;
    i32* keys = gkeys + k * gcap;
    V* vals = gvals + k * gcap;
    const int l = lane_id(), w = threadIdx.x >> 5;
    const i64 len = j1 - j0, base = j0 - (j0 & ~(i64)3);
    for (i64 t = (i64)w * 32 + l; t - l < len; t += CSPLIT_THREADS) {
        const bool valid = t < len;
        const i32 u = valid ? s_key[base + t] : -1;
        const V wv = (valid && has_w) ? V(s_w[base + t]) : V(0);
        const bool keep = valid && u >= 0;
        const i32 key = keep ? u : (i32)(0x80000000u | l);
        const unsigned peers = __match_any_sync(FULL, key);
        const bool leader = keep && ((peers & lanemask_lt()) == 0);
        const V sum = has_w ? cgroup_sum<V>(peers, wv, leader) : V(__popc(peers));
        if (leader) ctable_add(keys, vals, T - 1, key, sum, a.err, a.probe_cap);
    }
}

template <class W>
__global__ void __launch_bounds__(CSPLIT_THREADS) k_csplit_write(CArgs<W> a, const i32* list, i64 count, i64 gcap,
                                                                const i32* gkeys,
                                                                const typename Traits<W>::V* gvals, i64 nc) {
    const i64 k = blockIdx.y;
    if (k >= count) return;
    const i32 c = list[k];
    i64 q0, q1;
    const u32 T = csplit_slots(a, c, nc, gcap, q0, q1);
    const i32* keys = gkeys + k * gcap;
    const auto* vals = gvals + k * gcap;
    const int l = lane_id();
    for (i64 s0 = blockIdx.x * (i64)CSPLIT_THREADS + (threadIdx.x & ~31); s0 < T;
         s0 += (i64)gridDim.x * CSPLIT_THREADS) {
        const i64 sl = s0 + l;
        const bool occ = sl < T && keys[sl] != -1;
        const unsigned m = __ballot_sync(FULL, occ);
        if (!m) continue;
        unsigned long long basepos = 0;
        if (l == 0) basepos = ::atomicAdd((unsigned long long*)&a.ucount[c], (unsigned long long)__popc(m));
        basepos = __shfl_sync(FULL, basepos, 0);
        if (occ) {
            const i64 pos = q0 + (i64)basepos + __popc(m & lanemask_lt());
            a.out_key[pos] = keys[sl];
            a.out_val[pos] = vals[sl];
        }
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

// Sorting by chunk ranks: the row's entries go in chunks of 32 (one warp
// each); a chunk is sorted by ranking every key against the chunk's other keys
// with shuffles (ties between padding keys broken by lane, so every slot of a
// chunk is written) and stored in shared memory; an entry's place in the row
// is its rank in its own chunk plus, for every other chunk, the number of that
// chunk's keys below it (a 6-step binary search of 32 sorted keys).  The keys
// of a row are distinct columns.  Cost per entry: 32 shuffles + 6 reads per
// other chunk, against the log^2 stages of a bitonic network.
constexpr i32 KEY_PAD = 2147483647;  // pads chunks; coarse ids are below it

__device__ __forceinline__ int chunk_rank(i32 key) {
    const int l = lane_id();
    int r = 0;
#pragma unroll
    for (int t = 0; t < 32; t++) {
        const i32 o = __shfl_sync(FULL, key, t);
        r += (o < key || (o == key && t < l)) ? 1 : 0;
    }
    return r;
}

// number of keys below `key` in a sorted chunk of 32 (padded with KEY_PAD)
__device__ __forceinline__ int chunk_below(const i32* ck, i32 key) {
    int pos = 0;
#pragma unroll
    for (int step = 16; step >= 1; step >>= 1)
        if (ck[pos + step - 1] < key) pos += step;
    return pos + (ck[pos] < key ? 1 : 0);
}

// 32 < u <= PW_MAX: a warp per row, entries held in registers (lane l has
// entries l, l + 32, ...), chunks sorted into shared memory, ranks summed
constexpr int PW_MAX = 256;
constexpr int PW_WARPS = 8;

template <class W>
__global__ void __launch_bounds__(PW_WARPS * 32) k_place_warp_rank(const i32* list, const i64* d_count, const i64* P,
                                                                   const i64* cstart, const i64* ucount,
                                                                   const i64* rowptr, const i32* skey,
                                                                   const typename Traits<W>::V* sval, i32* col,
                                                                   W* wout) {
    using V = typename Traits<W>::V;
    constexpr int NCH = PW_MAX / 32;
    __shared__ i32 kk[PW_WARPS][PW_MAX];
    const int l = lane_id(), w = threadIdx.x >> 5;
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
    const i64 count = *d_count;
    for (i64 x = gw; x < count; x += nw) {
        const i32 c = list[x];
        const i64 src = P[cstart[c]];
        const int u = (int)ucount[c];
        const i64 dst = rowptr[c];
        const int nch = (u + 31) >> 5;
        i32 key[NCH];
        V val[NCH];
        int rk[NCH];
#pragma unroll
        for (int k = 0; k < NCH; k++) {
            const int s = 32 * k + l;
            key[k] = s < u ? skey[src + s] : KEY_PAD;
            val[k] = s < u ? sval[src + s] : V(0);
        }
#pragma unroll
        for (int k = 0; k < NCH; k++) {
            if (k < nch) {
                rk[k] = chunk_rank(key[k]);
                kk[w][32 * k + rk[k]] = key[k];
            }
        }
        __syncwarp();
        // chunk by chunk, the searches of all the lane's entries together (independent, so
        // their shared-memory reads overlap)
        int g[NCH];
#pragma unroll
        for (int k = 0; k < NCH; k++) g[k] = k < nch ? rk[k] : 0;
        for (int j = 0; j < nch; j++) {
            const i32* ck = &kk[w][32 * j];
#pragma unroll
            for (int k = 0; k < NCH; k++)
                if (k < nch && k != j) g[k] += chunk_below(ck, key[k]);
        }
#pragma unroll
        for (int k = 0; k < NCH; k++) {
            if (k < nch && 32 * k + l < u) {
                col[dst + g[k]] = key[k];
                wout[dst + g[k]] = to_w<W>(val[k]);
            }
        }
        __syncwarp();
    }
}

// PW_MAX < u <= PB_MID: the same with a 256-thread block per row (warp w
// sorts chunks w, w + 8, ...)
constexpr int PBR_THREADS = 256;

template <class W>
__global__ void __launch_bounds__(PBR_THREADS) k_place_block_rank(const i32* list, const i64* d_count, const i64* P,
                                                                  const i64* cstart, const i64* ucount,
                                                                  const i64* rowptr, const i32* skey,
                                                                  const typename Traits<W>::V* sval, i32* col,
                                                                  W* wout) {
    using V = typename Traits<W>::V;
    constexpr int CAP = 1024, PER = CAP / PBR_THREADS;
    __shared__ i32 kk[CAP];
    const int t = threadIdx.x;
    const i64 count = *d_count;
    for (i64 x = blockIdx.x; x < count; x += gridDim.x) {
        const i32 c = list[x];
        const i64 src = P[cstart[c]];
        const int u = (int)ucount[c];
        const i64 dst = rowptr[c];
        const int nch = (u + 31) >> 5;
        i32 key[PER];
        V val[PER];
        int rk[PER];
#pragma unroll
        for (int m = 0; m < PER; m++) {
            const int s = t + PBR_THREADS * m;
            key[m] = s < u ? skey[src + s] : KEY_PAD;
            val[m] = s < u ? sval[src + s] : V(0);
        }
#pragma unroll
        for (int m = 0; m < PER; m++) {
            const int k = (t + PBR_THREADS * m) >> 5;  // warp-uniform
            if (k < nch) {
                rk[m] = chunk_rank(key[m]);
                kk[32 * k + rk[m]] = key[m];
            }
        }
        __syncthreads();
        int g[PER];
#pragma unroll
        for (int m = 0; m < PER; m++) g[m] = ((t + PBR_THREADS * m) >> 5) < nch ? rk[m] : 0;
        for (int j = 0; j < nch; j++) {
            const i32* ck = &kk[32 * j];
#pragma unroll
            for (int m = 0; m < PER; m++) {
                const int k = (t + PBR_THREADS * m) >> 5;
                if (k < nch && k != j) g[m] += chunk_below(ck, key[m]);
            }
        }
#pragma unroll
        for (int m = 0; m < PER; m++) {
            const int s = t + PBR_THREADS * m;
            if (s < u) {
                col[dst + g[m]] = key[m];
                wout[dst + g[m]] = to_w<W>(val[m]);
            }
        }
        __syncthreads();
    }
}

constexpr int PB_MID = 1024;
constexpr int PB_MAX = 4096;

// block per row of up to CAP entries: bitonic sort of (key, value) pairs in
// shared memory, T = next_pow2(u) padded with INT_MAX keys
template <class W, int THREADS, int CAP>
__global__ void __launch_bounds__(THREADS) k_place_block(const i32* list, const i64* d_count, const i64* P,
                                                         const i64* cstart, const i64* ucount, const i64* rowptr,
                                                         const i32* skey, const typename Traits<W>::V* sval, i32* col,
                                                         W* wout) {
    using V = typename Traits<W>::V;
    __shared__ i32 kk[CAP];
    __shared__ V vv[CAP];
    const i64 count = *d_count;
    for (i64 x = blockIdx.x; x < count; x += gridDim.x) {
        const i32 c = list[x];
        const i64 src = P[cstart[c]];
        const i64 u = ucount[c];
        const u32 T = next_pow2_u32((u32)u);
        for (u32 s = threadIdx.x; s < T; s += THREADS) {
            kk[s] = s < u ? skey[src + s] : 2147483647;
            vv[s] = s < u ? sval[src + s] : V(0);
        }
        __syncthreads();
        for (u32 k = 2; k <= T; k <<= 1) {
            for (u32 j = k >> 1; j > 0; j >>= 1) {
                for (u32 t = threadIdx.x; t < T; t += THREADS) {
                    const u32 q = t ^ j;
                    if (q > t) {
                        const bool up = (t & k) == 0;
                        const i32 a0 = kk[t], a1 = kk[q];
                        if ((a0 > a1) == up) {
                            kk[t] = a1;
                            kk[q] = a0;
                            const V v0 = vv[t];
                            vv[t] = vv[q];
                            vv[q] = v0;
                        }
                    }
                }
                // a stride below 32 keeps every pair inside one warp's
                // 32-aligned slices (THREADS is a multiple of 32), so only the
                // last step of each merge needs the block barrier
                if (j >= 32 || j == 1) __syncthreads();
                else __syncwarp();
            }
        }
        const i64 dst = rowptr[c];
        for (u32 s = threadIdx.x; s < u; s += THREADS) {
            col[dst + s] = kk[s];
            wout[dst + s] = to_w<W>(vv[s]);
        }
        __syncthreads();
    }
}

// Rows of a coarse graph with few vertices (nc <= BM_MAX_NC): a block per
// row sets one bit per unique column in a shared bitmap of nc bits; the rank
// of a column is the popcount of the bits before it (a prefix over the
// bitmap words plus the bits below it in its word), so every entry is written
// straight to its sorted position -- O(u + nc/32) per row instead of a
// comparison sort.
constexpr i64 BM_MAX_NC = 262144;
constexpr int BM_THREADS = 256;
// Rows above PB_MID entries of coarse graphs up to BM_BIG_MAX_NC vertices: the
// same with 1024 threads and a bitmap plus word prefix that fill the 227 KB a
// block may have -- a few rows per SM, each O(nc / 32 / 1024) per thread,
// against a 4096-slot bitonic network or the radix sort
constexpr i64 BM_BIG_MAX_NC = 29024 * 32;

template <class W, int BM_THREADS = BM_THREADS>
__global__ void __launch_bounds__(BM_THREADS) k_place_bitmap(const i32* list, const i64* d_count, const i64* P,
                                                            const i64* cstart, const i64* ucount, const i64* rowptr,
                                                            const i32* skey, const typename Traits<W>::V* sval,
                                                            i32* col, W* wout, int nwords) {
    extern __shared__ __align__(16) u32 bm_smem[];
    u32* bm = bm_smem;
    u32* pre = bm_smem + nwords;
    __shared__ u32 wsum[BM_THREADS / 32];
    const int tid = threadIdx.x, l = lane_id(), w = tid >> 5;
    const int per = (nwords + BM_THREADS - 1) / BM_THREADS;
    const int w0 = min(tid * per, nwords), w1 = min(w0 + per, nwords);
    const i64 count = *d_count;
    for (i64 x = blockIdx.x; x < count; x += gridDim.x) {
        const i32 c = list[x];
        const i64 src = P[cstart[c]];
        const i64 u = ucount[c];
        const i64 dst = rowptr[c];
        for (int s = tid; s < nwords; s += BM_THREADS) bm[s] = 0u;
        __syncthreads();
        for (i64 s = tid; s < u; s += BM_THREADS) {
            const u32 k = (u32)skey[src + s];
            atomicOr(&bm[k >> 5], 1u << (k & 31));
        }
        __syncthreads();
        // exclusive prefix of the word popcounts: thread chunks, then a block scan
        u32 local = 0;
        for (int q = w0; q < w1; q++) local += (u32)__popc(bm[q]);
        u32 incl = local;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const u32 t = __shfl_up_sync(FULL, incl, d);
            if (l >= d) incl += t;
        }
        if (l == 31) wsum[w] = incl;
        __syncthreads();
        u32 base = 0;
        for (int q = 0; q < w; q++) base += wsum[q];
        u32 run = base + incl - local;
        for (int q = w0; q < w1; q++) {
            pre[q] = run;
            run += (u32)__popc(bm[q]);
        }
        __syncthreads();
        for (i64 s = tid; s < u; s += BM_THREADS) {
            const u32 k = (u32)skey[src + s];
            const u32 r = pre[k >> 5] + (u32)__popc(bm[k >> 5] & ((1u << (k & 31)) - 1u));
            col[dst + r] = (i32)k;
            wout[dst + r] = to_w<W>(sval[src + s]);
        }
        __syncthreads();
    }
}

// big rows: gather into (row-major) temp with composite keys, radix sort, place
template <class V>
__global__ void k_big_gather(const i32* list, i64 count, const i64* tstart, const i64* P, const i64* cstart,
                             const i64* ucount, const i32* skey, const V* sval, u64* tkey, V* tval, int cbits) {
    for (i64 x = blockIdx.x; x < count; x += gridDim.x) {
        i32 c = list[x];
        i64 src = P[cstart[c]];
        i64 u = ucount[c];
        i64 dst = tstart[x];
        for (i64 s = threadIdx.x; s < u; s += blockDim.x) {
            tkey[dst + s] = ((u64)x << cbits) | (u64)(u32)skey[src + s];
            tval[dst + s] = sval[src + s];
        }
    }
}
template <class W>
__global__ void k_big_place(const i32* list, i64 count, const i64* tstart, const i64* rowptr, const u64* tkey,
                            const typename Traits<W>::V* tval, i32* col, W* wout, int cbits) {
    const u64 cmask = ((u64)1 << cbits) - 1;
    for (i64 x = blockIdx.x; x < count; x += gridDim.x) {
        i32 c = list[x];
        i64 a = tstart[x], b = tstart[x + 1];
        for (i64 y = a + threadIdx.x; y < b; y += blockDim.x) {
            col[rowptr[c] + (y - a)] = (i32)(u32)(tkey[y] & cmask);
            wout[rowptr[c] + (y - a)] = to_w<W>(tval[y]);
        }
    }
}

// Sorts the coarse rows into the hashing buckets in one pass (list order is
// irrelevant: rows are independent).  Buckets by bound (sum of member degrees)
// and U = min(bound, nc): 0: bound <= 32, 1: bound <= 256, 2: U <= 1024,
// 3: U <= 4096, 4: above.  cnt[k] counts bucket k; cnt[5] is the largest
// bound of bucket 4.
__global__ void k_bucket_rows(const i64* P, const i64* cstart, i64 nc, i32* l0, i32* l1, i32* l2, i32* l3, i32* l4,
                              unsigned long long* cnt) {
    const int l = lane_id();
    unsigned long long mx = 0;
    for (i64 c0 = (blockIdx.x * (i64)blockDim.x + threadIdx.x) - l; c0 < nc; c0 += (i64)gridDim.x * blockDim.x) {
        const i64 c = c0 + l;
        int k = -1;
        if (c < nc) {
            const i64 v = P[cstart[c + 1]] - P[cstart[c]];
            const i64 U = v < nc ? v : nc;
            k = v <= 32 ? 0 : v <= 256 ? 1 : U <= 1024 ? 2 : U <= HUGE_DEG ? 3 : 4;
            if (k == 4 && (unsigned long long)v > mx) mx = (unsigned long long)v;
        }
        i32* lists[5] = {l0, l1, l2, l3, l4};
#pragma unroll
        for (int b = 0; b < 5; b++) {
            const unsigned m = __ballot_sync(FULL, k == b);
            if (!m) continue;
            const int leader = __ffs(m) - 1;
            unsigned long long base = 0;
            if (l == leader) base = atomicAdd(&cnt[b], (unsigned long long)__popc(m));
            base = __shfl_sync(FULL, base, leader);
            if (k == b) lists[b][base + __popc(m & lanemask_lt())] = (i32)c;
        }
    }
    for (int d = 16; d >= 1; d >>= 1) {
        const unsigned long long o = __shfl_xor_sync(FULL, mx, d);
        mx = o > mx ? o : mx;
    }
    if (l == 0 && mx) atomicMax(&cnt[5], mx);
}

// Placement buckets by unique count u: 0: u <= 32, 1: u <= PW_MAX,
// 2: u <= PB_MID, 3: u <= PB_MAX, 4: above (rows with no entries are skipped).
__global__ void k_bucket_place(const i64* ucount, i64 nc, i32* l0, i32* l1, i32* l2, i32* l3, i32* l4,
                               unsigned long long* cnt) {
    const int l = lane_id();
    for (i64 c0 = (blockIdx.x * (i64)blockDim.x + threadIdx.x) - l; c0 < nc; c0 += (i64)gridDim.x * blockDim.x) {
        const i64 c = c0 + l;
        int k = -1;
        if (c < nc) {
            const i64 u = ucount[c];
            k = u <= 0 ? -1 : u <= 32 ? 0 : u <= PW_MAX ? 1 : u <= PB_MID ? 2 : u <= PB_MAX ? 3 : 4;
        }
        i32* lists[5] = {l0, l1, l2, l3, l4};
#pragma unroll
        for (int b = 0; b < 5; b++) {
            const unsigned m = __ballot_sync(FULL, k == b);
            if (!m) continue;
            const int leader = __ffs(m) - 1;
            unsigned long long base = 0;
            if (l == leader) base = atomicAdd(&cnt[b], (unsigned long long)__popc(m));
            base = __shfl_sync(FULL, base, leader);
            if (k == b) lists[b][base + __popc(m & lanemask_lt())] = (i32)c;
        }
    }
}

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

// Contraction temporaries live in grow-only workspace slots of the context
// (sized by the largest level, reused by every later contraction), so the
// level loop does not go through the allocator for them.
enum ContractSlot : int {
    CS_CNT = 50, CS_BOUND, CS_CSTART, CS_P, CS_UCOUNT, CS_MEMBERS, CS_MEMBERPOS, CS_CURSOR, CS_TOT, CS_FKEY, CS_FW,
    CS_OKEY, CS_OVAL, CS_LW, CS_LM, CS_LB, CS_LB2, CS_LH, CS_LO, CS_COUNTS, CS_PW, CS_PR, CS_PB, CS_PB2, CS_PH,
    CS_TSTART, CS_TK, CS_TK2, CS_TV, CS_TV2
};
template <class T>
struct WsBuf {
    T* p;
    WsBuf(Context& c, int slot, i64 count) : p(c.ws_get<T>(slot, std::max<i64>(count, 1))) {}
};

template <class W>
std::unique_ptr<Graph<W>> build_coarse_graph(Context& ctx, const Graph<W>& g, const i32* vcmap, i64 nc) {
    using V = typename Traits<W>::V;
    ProfScope ps(ctx, "contract");
    std::optional<ProfScope> phase;  // sub-phases: prep (count .. flatten), hash, place
    phase.emplace(ctx, "contract_prep");
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
    WsBuf<i64> cnt(ctx, CS_CNT, nc + 1), bound(ctx, CS_BOUND, nc + 1), cstart(ctx, CS_CSTART, nc + 1),
        P(ctx, CS_P, n + 1), ucount(ctx, CS_UCOUNT, nc + 1);
    WsBuf<i32> members(ctx, CS_MEMBERS, n);
    WsBuf<i64> memberpos(ctx, CS_MEMBERPOS, n);
    PGGC_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(i64) * (nc + 1), ctx.stream));
    PGGC_CUDA(cudaMemsetAsync(bound.p, 0, sizeof(i64) * (nc + 1), ctx.stream));
    int gridv = (int)std::min<i64>(ceil_div(n, 256), (i64)ctx.num_sms * 16);
    k_contract_count<W><<<gridv, 256, 0, ctx.stream>>>(gv, vcmap, cnt.p, bound.p);
    PGGC_LAUNCH_CHECK();
    scan_apply(ctx, ArrIn{cnt.p}, ArrOutExcl{cstart.p}, nc + 1, nullptr, nullptr);
    {
        WsBuf<i64> cursor(ctx, CS_CURSOR, nc + 1);
        copy_d2d(ctx, cursor.p, cstart.p, nc + 1);
        k_scatter_members<<<gridv, 256, 0, ctx.stream>>>(vcmap, n, cursor.p, members.p, memberpos.p);
        PGGC_LAUNCH_CHECK();
    }
    WsBuf<i64> tot(ctx, CS_TOT, 4);
    scan_apply(ctx, MemberDegIn{gv.rowptr, members.p, n}, ArrOutExcl{P.p}, n + 1, nullptr, tot.p);
    // flattened rows: coarse key and weight of every fine edge at its flat position
    WsBuf<i32> fkey(ctx, CS_FKEY, g.nnz);
    W* fw_p = gv.w ? ctx.ws_get<W>(CS_FW, std::max<i64>(g.nnz, 1)) : nullptr;
    if (g.nnz > 0 && g.nnz >= FLW_MIN_DEG * n) {
        int grid = (int)std::min<i64>(ceil_div(n, 8), (i64)ctx.num_sms * 16);
        k_flatten_wide<W><<<grid, 256, 0, ctx.stream>>>(gv, vcmap, P.p, memberpos.p, fkey.p, fw_p);
        PGGC_LAUNCH_CHECK();
    } else if (g.nnz > 0) {
        int grid = (int)std::min<i64>(ceil_div(ceil_div(n, 32), 8), (i64)ctx.num_sms * 16);
        k_flatten<W><<<grid, 256, 0, ctx.stream>>>(gv, vcmap, P.p, memberpos.p, fkey.p, fw_p);
        PGGC_LAUNCH_CHECK();
    }
    const i64 total_bound = g.nnz;
    WsBuf<i32> okey(ctx, CS_OKEY, total_bound);
    WsBuf<V> oval(ctx, CS_OVAL, total_bound);

    // bucket lists by bound (sum of member degrees) and table size U =
    // min(bound, nc): small warp rows (bound <= 32), medium warp rows
    // (bound <= 256), block rows with shared tables of 2048 slots (U <= 1024)
    // and 8192 slots (U <= 4096), big rows with 16384-slot shared tables
    // (U > 4096) whose overflow falls back to global tables
    WsBuf<i32> lw(ctx, CS_LW, nc), lm(ctx, CS_LM, nc), lb(ctx, CS_LB, nc), lb2(ctx, CS_LB2, nc), lh(ctx, CS_LH, nc),
        lo(ctx, CS_LO, nc);
    // counts: [0] small warp rows, [1] medium warp rows, [2] 2048-slot block
    // rows, [3] 8192-slot block rows, [4] big rows, [5] largest big-row bound,
    // [6] overflow rows, [7..11] placement buckets, [12] big-row placement
    // total, [14] coarse nnz
    WsBuf<i64> counts(ctx, CS_COUNTS, 16);
    PGGC_CUDA(cudaMemsetAsync(counts.p, 0, sizeof(i64) * 16, ctx.stream));
    {
        int grid = (int)std::max<i64>(1, std::min<i64>(ceil_div(nc, 256), (i64)ctx.num_sms * 8));
        k_bucket_rows<<<grid, 256, 0, ctx.stream>>>(P.p, cstart.p, nc, lw.p, lm.p, lb.p, lb2.p, lh.p,
                                                   (unsigned long long*)counts.p);
        PGGC_LAUNCH_CHECK();
    }
    // one round trip: bucket sizes and the largest big-row bound
    const i64* hc = (const i64*)ctx.readback(counts.p, 16 * sizeof(i64));
    const i64 n_w = hc[0], n_m = hc[1], n_b = hc[2], n_b2 = hc[3], n_h = hc[4], max_huge = hc[5];

    CArgs<W> a;
    a.g = gv;
    a.vcmap = vcmap;
    a.cstart = cstart.p;
    a.members = members.p;
    a.P = P.p;
    a.fkey = fkey.p;
    a.fw = fw_p;
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
        k_contract_warp<W, 512, WARPS><<<grid, WARPS * 32, 0, ctx.stream>>>(a, lm.p, counts.p + 1);
        PGGC_LAUNCH_CHECK();
    }
    phase.reset();
    phase.emplace(ctx, "contract_hash");
    const size_t slot = sizeof(V) + sizeof(i32);
    const bool dense = nc <= DENSE_NC;
    if (dense && (n_b > 0 || n_b2 > 0 || n_h > 0)) {
        // every block row on the dense table (256 threads up to U = 1024, 512 above)
        const size_t dsmem = sizeof(V) * (size_t)nc + sizeof(u32) * (size_t)ceil_div(nc, 32);
        const int dmax = (int)(sizeof(V) * DENSE_NC + sizeof(u32) * (DENSE_NC / 32));
        set_dynamic_smem_once(k_contract_dense<W, 256>, dmax, ctx.device);
        set_dynamic_smem_once(k_contract_dense<W, 512>, dmax, ctx.device);
        if (n_b > 0) {
            int grid = (int)std::min<i64>(n_b, (i64)ctx.num_sms * 8);
            k_contract_dense<W, 256><<<grid, 256, dsmem, ctx.stream>>>(a, lb.p, counts.p + 2, (int)nc);
            PGGC_LAUNCH_CHECK();
        }
        const i64 lists[2] = {n_b2, n_h};
        const i32* lp[2] = {lb2.p, lh.p};
        for (int q = 0; q < 2; q++) {
            if (lists[q] <= 0) continue;
            int grid = (int)std::min<i64>(lists[q], (i64)ctx.num_sms * 4);
            k_contract_dense<W, 512><<<grid, 512, dsmem, ctx.stream>>>(a, lp[q], counts.p + 3 + q, (int)nc);
            PGGC_LAUNCH_CHECK();
        }
    }
    if (!dense && n_b > 0) {
        constexpr int TS = 2048;
        int grid = (int)std::min<i64>(n_b, (i64)ctx.num_sms * 8);
        k_contract_block<W, false, 256><<<grid, 256, slot * TS, ctx.stream>>>(a, lb.p, counts.p + 2, nullptr, nullptr,
                                                                               TS, nc);
        PGGC_LAUNCH_CHECK();
    }
    if (!dense && n_b2 > 0) {
        constexpr int TS = 2 * HUGE_DEG;
        set_dynamic_smem_once(k_contract_block<W, false, 512>, (int)(slot * TS), ctx.device);
        int grid = (int)std::min<i64>(n_b2, (i64)ctx.num_sms * 2);
        k_contract_block<W, false, 512><<<grid, 512, slot * TS, ctx.stream>>>(a, lb2.p, counts.p + 3, nullptr, nullptr,
                                                                               TS, nc);
        PGGC_LAUNCH_CHECK();
    }
    if (!dense && n_h > 0) {
        // 16384-slot shared tables; rows with more distinct neighbours (a
        // 64-probe insert failure) go to the overflow list
        constexpr int TS = 16384;
        set_dynamic_smem_once(k_contract_block<W, false, 1024, true>, (int)(slot * TS), ctx.device);
        int grid = (int)std::min<i64>(n_h, (i64)ctx.num_sms);
        k_contract_block<W, false, 1024, true><<<grid, 1024, slot * TS, ctx.stream>>>(
            a, lh.p, counts.p + 4, nullptr, nullptr, TS, nc, lo.p, counts.p + 6);
        PGGC_LAUNCH_CHECK();
        // rows that overflowed: global tables sized for the largest table
        // among the big rows, one region per resident block, at most 2 GiB of
        // tables (allocated only when some row overflowed)
        const i64 n_ovf = ctx.read1(counts.p + 6);
        if (n_ovf > 0) {
            // split across blocks, in rounds of up to `per` rows (one table
            // each, at most 2 GiB of tables)
            i64 maxb = std::min<i64>(max_huge, nc);
            i64 gcap = next_pow2_u32((u32)std::min<i64>(2 * std::max<i64>(maxb, 1), (i64)1 << 30));
            i64 by_mem = std::max<i64>(1, ((i64)2 << 30) / (gcap * (i64)slot));
            const i64 per = std::min<i64>(std::min<i64>(n_ovf, 32), by_mem);
            i32* gk = ctx.ws_get<i32>(WS_CONTRACT_GK, gcap * per);
            V* gvv = ctx.ws_get<V>(WS_CONTRACT_GV, gcap * per);
            set_dynamic_smem_once(k_csplit_insert<W>, (int)CSPLIT_SMEM, ctx.device);
            const unsigned chunks = (unsigned)std::max<i64>(1, ceil_div(max_huge, CSPLIT_CHUNK));
            const unsigned wblocks =
                (unsigned)std::max<i64>(1, std::min<i64>(ceil_div(gcap, CSPLIT_THREADS * 8), (i64)ctx.num_sms));
            for (i64 r0 = 0; r0 < n_ovf; r0 += per) {
                const i64 cnt = std::min<i64>(per, n_ovf - r0);
                const i32* lst = lo.p + r0;
                const int cgrid = (int)std::max<i64>(1, std::min<i64>(ceil_div(cnt * gcap, 256),
                                                                      (i64)ctx.num_sms * 16));
                k_csplit_clear<W><<<cgrid, 256, 0, ctx.stream>>>(a, lst, cnt, gcap, gk, gvv);
                PGGC_LAUNCH_CHECK();
                k_csplit_insert<W><<<dim3(chunks, (unsigned)cnt), CSPLIT_THREADS, CSPLIT_SMEM, ctx.stream>>>(
                    a, lst, cnt, gcap, gk, gvv, nc);
                PGGC_LAUNCH_CHECK();
                k_csplit_write<W><<<dim3(wblocks, (unsigned)cnt), CSPLIT_THREADS, 0, ctx.stream>>>(a, lst, cnt, gcap,
                                                                                                    gk, gvv, nc);
                PGGC_LAUNCH_CHECK();
            }
        }
    }
    // coarse row offsets, placement buckets and the big-row total, then one round trip
    phase.reset();
    phase.emplace(ctx, "contract_place");
    scan_apply(ctx, UcountIn{ucount.p, nc}, RowptrOut{cg->rowptr.p}, nc + 1, nullptr, counts.p + 14);
    WsBuf<i32> pw(ctx, CS_PW, nc), pr(ctx, CS_PR, nc), pb(ctx, CS_PB, nc), pb2(ctx, CS_PB2, nc), ph(ctx, CS_PH, nc);
    {
        int grid = (int)std::max<i64>(1, std::min<i64>(ceil_div(nc, 256), (i64)ctx.num_sms * 8));
        k_bucket_place<<<grid, 256, 0, ctx.stream>>>(ucount.p, nc, pw.p, pr.p, pb.p, pb2.p, ph.p,
                                                    (unsigned long long*)(counts.p + 7));
        PGGC_LAUNCH_CHECK();
    }
    WsBuf<i64> tstart(ctx, CS_TSTART, nc + 1);
    scan_apply(ctx, ListUIn{ph.p, ucount.p, counts.p + 11}, ArrOutExcl{tstart.p}, nc + 1, nullptr, counts.p + 12);
    // the device error word rides along in counts[15] (zeroed above)
    PGGC_CUDA(cudaMemcpyAsync(counts.p + 15, ctx.d_err, sizeof(int), cudaMemcpyDeviceToDevice, ctx.stream));
    const i64* pc = (const i64*)ctx.readback(counts.p, 16 * sizeof(i64));
    const i64 p_w = pc[7], p_r = pc[8], p_b = pc[9], p_b2 = pc[10], p_h = pc[11], nnz_c = pc[14], tn = pc[12];
    ctx.raise_device_error((int)pc[15]);
    cg->nnz = nnz_c;
    cg->col = DBuf<i32>(ctx, std::max<i64>(nnz_c, 1));
    cg->w = DBuf<W>(ctx, std::max<i64>(nnz_c, 1));
    if (p_w > 0) {
        int grid = (int)std::min<i64>(ceil_div(p_w, 8), (i64)ctx.num_sms * 8);
        k_place_warp<W><<<grid, 256, 0, ctx.stream>>>(pw.p, counts.p + 7, P.p, cstart.p, ucount.p, cg->rowptr.p, okey.p,
                                                      oval.p, cg->col.p, cg->w.p);
        PGGC_LAUNCH_CHECK();
    }
    const bool bitmap = nc <= BM_MAX_NC;
    if (bitmap) {
        // every row above PW_MAX entries: bitmap ranks (lists pb, pb2, ph)
        const int nwords = (int)ceil_div(nc, 32);
        const size_t smem = sizeof(u32) * 2 * (size_t)nwords;
        set_dynamic_smem_once(k_place_bitmap<W>, (int)(sizeof(u32) * 2 * ceil_div(BM_MAX_NC, 32)), ctx.device);
        const i64 lists[3] = {p_b, p_b2, p_h};
        i32* lp[3] = {pb.p, pb2.p, ph.p};
        for (int q = 0; q < 3; q++) {
            if (lists[q] <= 0) continue;
            int grid = (int)std::min<i64>(lists[q], (i64)ctx.num_sms * 4);
            k_place_bitmap<W><<<grid, BM_THREADS, smem, ctx.stream>>>(lp[q], counts.p + 9 + q, P.p, cstart.p, ucount.p,
                                                                     cg->rowptr.p, okey.p, oval.p, cg->col.p,
                                                                     cg->w.p, nwords);
            PGGC_LAUNCH_CHECK();
        }
    }
    const bool bitmap_big = !bitmap && nc <= BM_BIG_MAX_NC;
    if (bitmap_big && (p_b2 > 0 || p_h > 0)) {
        const int nwords = (int)ceil_div(nc, 32);
        const size_t smem = sizeof(u32) * 2 * (size_t)nwords;
        set_dynamic_smem_once(k_place_bitmap<W, 1024>, (int)(sizeof(u32) * 2 * ceil_div(BM_BIG_MAX_NC, 32)),
                              ctx.device);
        const i64 lists[2] = {p_b2, p_h};
        i32* lp[2] = {pb2.p, ph.p};
        for (int q = 0; q < 2; q++) {
            if (lists[q] <= 0) continue;
            int grid = (int)std::min<i64>(lists[q], (i64)ctx.num_sms);
            k_place_bitmap<W, 1024><<<grid, 1024, smem, ctx.stream>>>(lp[q], counts.p + 10 + q, P.p, cstart.p,
                                                                     ucount.p, cg->rowptr.p, okey.p, oval.p,
                                                                     cg->col.p, cg->w.p, nwords);
            PGGC_LAUNCH_CHECK();
        }
    }
    // rows of 33..PW_MAX entries: chunk ranks in a warp (cheaper than the
    // bitmap's O(nc / 32) per row even for small nc)
    if (p_r > 0) {
        int grid = (int)std::min<i64>(ceil_div(p_r, PW_WARPS), (i64)ctx.num_sms * 8);
        k_place_warp_rank<W><<<grid, PW_WARPS * 32, 0, ctx.stream>>>(pr.p, counts.p + 8, P.p, cstart.p, ucount.p,
                                                                     cg->rowptr.p, okey.p, oval.p, cg->col.p,
                                                                     cg->w.p);
        PGGC_LAUNCH_CHECK();
    }
    if (!bitmap && p_b > 0) {
        int grid = (int)std::min<i64>(p_b, (i64)ctx.num_sms * 8);
        k_place_block_rank<W><<<grid, PBR_THREADS, 0, ctx.stream>>>(pb.p, counts.p + 9, P.p, cstart.p, ucount.p,
                                                                     cg->rowptr.p, okey.p, oval.p, cg->col.p,
                                                                     cg->w.p);
        PGGC_LAUNCH_CHECK();
    }
    if (!bitmap && !bitmap_big && p_b2 > 0) {
        int grid = (int)std::min<i64>(p_b2, (i64)ctx.num_sms * 2);
        k_place_block<W, 1024, PB_MAX><<<grid, 1024, 0, ctx.stream>>>(pb2.p, counts.p + 10, P.p, cstart.p, ucount.p,
                                                                      cg->rowptr.p, okey.p, oval.p, cg->col.p,
                                                                      cg->w.p);
        PGGC_LAUNCH_CHECK();
    }
    if (!bitmap && !bitmap_big && p_h > 0) {
        WsBuf<u64> tk(ctx, CS_TK, tn), tk2(ctx, CS_TK2, tn);
        WsBuf<V> tv(ctx, CS_TV, tn), tv2(ctx, CS_TV2, tn);
        int grid = (int)std::min<i64>(p_h, (i64)ctx.num_sms * 4);
        ProfScope pbig(ctx, "contract_place_big");
        ctx.prof_add_bytes("contract_place_big", (double)tn);
        // composite key (row rank, column): column bits for ids < nc only
        const int cbits = std::max(1, bits_for((u64)(nc - 1)));
        k_big_gather<V><<<grid, 256, 0, ctx.stream>>>(ph.p, p_h, tstart.p, P.p, cstart.p, ucount.p, okey.p, oval.p,
                                                      tk.p, tv.p, cbits);
        PGGC_LAUNCH_CHECK();
        int hib = cbits + bits_for((u64)p_h);
        radix_sort_pairs<V>(ctx, tk.p, tv.p, tn, 0, hib, tk2.p, tv2.p);
        k_big_place<W><<<grid, 256, 0, ctx.stream>>>(ph.p, p_h, tstart.p, cg->rowptr.p, tk.p, tv.p, cg->col.p,
                                                     cg->w.p, cbits);
        PGGC_LAUNCH_CHECK();
    }
    phase.reset();
    // algorithmic bytes: per fine edge its column, weight, the map of its head
    // and one table insert (key + output weight); per fine vertex its offset
    // and map; the coarse CSR written once
    {
        const double wb = g.uniform ? 0.0 : (double)sizeof(W);
        const double wout = (double)sizeof(W);
        ctx.prof_add_bytes("contract", (double)g.nnz * (4.0 + wb + 4.0 + 4.0 + wout) + (double)g.n * (8.0 + 4.0) +
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
