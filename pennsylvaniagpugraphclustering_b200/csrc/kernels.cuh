// kernels.cuh -- host-side entry points of the kernel families and the device
// state they share (weighted_graph, cluster_data, memory_store equivalents).
#pragma once
#include <atomic>
#include <memory>
#include <mutex>
#include <vector>
#include "scan.cuh"

// sets the thread-local message returned by pggc_last_error()
void pggc_set_last_error(const char* msg);

namespace pggc {

// Vertices of degree above HUGE_DEG aggregate into global-memory tables; all
// others use shared-memory tables.
constexpr i64 HUGE_DEG = 4096;
constexpr int SEL_TS_MAX = 8192;  // shared-memory table slots of the block kernels
// objective (modularity) the learned move filter may give up before its judge
// reports a fallback to the plain sweep (PGGC_FILTER_TOLERANCE)
constexpr double FILTER_TOLERANCE = 0.001;

// ---------------------------------------------------------------------------
// src/ordering.cpp:131-164 -- stable degree-bucket orderings
// ---------------------------------------------------------------------------
struct Ordering {
    DBuf<i32> order1, order2, huge;
    i64 n = 0;
    i64 off_large = 0, off_large2 = 0, off_mid = 0, off_mid2 = 0;
    i64 max_deg = 0, n_huge = 0;
};
void generate_orderings(Context& ctx, const i64* rowptr, i64 n, Ordering& o);

inline u64 next_graph_uid() {
    static std::atomic<u64> n{0};
    return ++n;
}

// Per-graph products that depend on the CSR alone (its ordering and degree
// class lists), built once on first use and kept with the graph.
struct GraphCache {
    std::mutex mu;
    bool ord_ok = false;
    Ordering ord;
    bool cls_ok = false;
    DBuf<i32> cls_list;
    DBuf<i64> cls_off;
    DBuf<unsigned long long> cls_cnt;
};

// ---------------------------------------------------------------------------
// weighted_graph (interface/weighted_graph.h:10-19), device resident
// ---------------------------------------------------------------------------
template <class W>
struct Graph {
    using V = typename Traits<W>::V;
    i64 n = 0, nnz = 0;
    bool uniform = true;  // unit edge weights; w is not allocated
    DBuf<i64> rowptr;
    DBuf<i32> col;
    DBuf<W> w;
    DBuf<V> vtx_w;
    const u64 uid = next_graph_uid();  // identifies the graph to per-context caches
    mutable DBuf<V> rsum;  // row weight sums, computed on first use by the sweep
    std::unique_ptr<GraphCache> cache{new GraphCache()};
    // borrowed (caller-owned) arrays take precedence over the owned ones
    const i64* b_rowptr = nullptr;
    const i32* b_col = nullptr;
    const W* b_w = nullptr;
    DGraph<W> view() const {
        DGraph<W> g;
        g.n = n;
        g.nnz = nnz;
        g.rowptr = b_rowptr ? b_rowptr : rowptr.p;
        g.col = b_col ? b_col : col.p;
        g.w = uniform ? nullptr : (b_w ? b_w : w.p);
        g.vtx_w = vtx_w.p;
        return g;
    }
};

// A slice of a vertex list whose bounds live on the host or in device memory.
struct Range {
    const i32* list;
    const i64* d_lo;
    const i64* d_hi;
    i64 lo, hi;
    __device__ __forceinline__ i64 begin() const { return d_lo ? *d_lo : lo; }
    __device__ __forceinline__ i64 end() const { return d_hi ? *d_hi : hi; }
};
inline Range host_range(const i32* list, i64 lo, i64 hi) { return Range{list, nullptr, nullptr, lo, hi}; }
inline Range dev_range(const i32* list, const i64* d_lo, const i64* d_hi) { return Range{list, d_lo, d_hi, 0, 0}; }

// Degree classes of the sweep kernels: 0 (<= 8), 1 (<= 16), 2 (<= 32),
// 3 (< 128), 4 (<= 1024), 5 (<= 4096), 6 (above); the class lists hold every
// vertex grouped by class.
constexpr int NCLS = 7;
struct ClassLists {
    i32* list = nullptr;                // [count] vertices grouped by class
    i64* off = nullptr;                 // [NCLS + 1] device class offsets
    unsigned long long* cnt = nullptr;  // [2 * NCLS] device counters / cursors
    i64 count = 0;                      // host: number of listed vertices
};
// the graph's class lists (built on first use, kept with the graph)
template <class W>
ClassLists graph_class_lists(Context& ctx, const Graph<W>& g, const Ordering& ord);

// The canonical association of an 8-lane group after each lane r has added
// its terms r and r + 8 from 0 (xor butterfly 4, 2, 1, read at lane 0):
// ((a0 + a4) + (a2 + a6)) + ((a1 + a5) + (a3 + a7)).
template <class V>
__device__ __forceinline__ V canon_tree8(const V (&a)[8]) {
    const V b0 = a[0] + a[4], b1 = a[1] + a[5], b2 = a[2] + a[6], b3 = a[3] + a[7];
    return (b0 + b2) + (b1 + b3);
}
// the same for an H-lane group (H = 8 or 16): the butterfly step 8 first
template <int H, class V>
__device__ __forceinline__ V canon_tree(const V (&a)[H]) {
    if constexpr (H == 8) {
        return canon_tree8<V>(a);
    } else {
        static_assert(H == 16, "H is 8 or 16");
        V b[8];
#pragma unroll
        for (int r = 0; r < 8; r++) b[r] = a[r] + a[r + 8];
        return canon_tree8<V>(b);
    }
}


// Canonical per-vertex sum of term(j) over [b, e) with e - b <= 2H (H = 8 or
// 16) by one thread: lane r of an H-lane group adds terms r and r + H from 0,
// then the xor butterfly -- the 32-lane canonical association for these
// degrees.
template <int H, class V, class F>
__device__ __forceinline__ V thread_vsum(i64 b, i64 e, F term) {
    V acc[H];
#pragma unroll
    for (int r = 0; r < H; r++) {
        acc[r] = V(0);
        if (b + r < e) acc[r] += term(b + r);
        if (b + r + H < e) acc[r] += term(b + r + H);
    }
    return canon_tree<H, V>(acc);
}

// the graph's ordering (generate_orderings on its CSR), built on first use
template <class W>
const Ordering& graph_ordering(Context& ctx, const Graph<W>& g) {
    GraphCache& c = *g.cache;
    std::lock_guard<std::mutex> lk(c.mu);
    if (!c.ord_ok) {
        generate_orderings(ctx, g.view().rowptr, g.n, c.ord);
        ctx.sync();  // other streams may read it next
        c.ord_ok = true;
    }
    return c.ord;
}

enum ObjKind { OBJ_MOD = 0, OBJ_WMOD = 1, OBJ_CPM = 2, OBJ_NLCC = 3, OBJ_LCC = 4 };

// ---------------------------------------------------------------------------
// cluster_data (interface/cluster_data.hpp:9-107): host scalars + device
// total_deg with room for appended labels.
// ---------------------------------------------------------------------------
template <class V>
struct ClusterState {
    DBuf<V> total_deg;
    i64 capacity = 0;
    V uncut = 0;
    i64 top_nnz = 0;
    double obj = -1.0;
    i64 label_count = 0;
    double lambda = 1.0;
    int kind = OBJ_LCC;
    double inv_gdeg = 0.0, v_total = 0.0, g_deg = 0.0;
    double vol_total = 0.0;  // sum of vertex weights (features of the learned filter)
    double get_objective() const {
        switch (kind) {
            case OBJ_MOD:
            case OBJ_WMOD: return obj * inv_gdeg;
            case OBJ_CPM: return obj + lambda * v_total;
            case OBJ_NLCC: return obj / g_deg;
            default: return obj;
        }
    }
};

// objective helpers (interface/cluster_data.hpp:76-87 and :109-181)
template <class W>
void make_cluster_state(Context& ctx, const Graph<W>& g, int kind, double mult, ClusterState<typename Traits<W>::V>& cs);
template <class V>
void update_objective(Context& ctx, ClusterState<V>& cs);
template <class W>
void default_vertex_weights(Context& ctx, Graph<W>& g, int objective);

// ---------------------------------------------------------------------------
// local move (src/local_mover.cpp)
// ---------------------------------------------------------------------------
struct MoveStats {
    i64 sweeps = 0;
    i64 moves = 0;
};

template <class W>
void local_move(Context& ctx, const Graph<W>& g, const Ordering& ord, i32* best_part,
                ClusterState<typename Traits<W>::V>& best, bool is_initial, bool constrained, i32* constraint,
                bool enable_sa, bool strict, int sweep_limit, MoveStats* stats, bool reuse_pvals = false);

// one select pass (candidates_and_destinations) for parity tests
template <class W>
i64 select_pass(Context& ctx, const Graph<W>& g, const Ordering& ord, const i32* part,
                const typename Traits<W>::V* pvals, ClusterState<typename Traits<W>::V>& cs, i32* dest, float* gain,
                float filter_ratio, bool initial, bool constrained, const i32* constraint);

// row weight sums of a graph (kept in the graph; computed on first call)
template <class W>
const typename Traits<W>::V* row_sums(Context& ctx, const Graph<W>& g);

// own-cluster weight of every vertex under `labels` (canonical sums)
template <class W>
void own_weights(Context& ctx, const Graph<W>& g, const Ordering& ord, const i32* labels, typename Traits<W>::V* out);

// ---------------------------------------------------------------------------
// contraction (src/contract.cpp:234-336) and Leiden refinement (src/leidenR.cpp)
// ---------------------------------------------------------------------------
template <class W>
std::unique_ptr<Graph<W>> build_coarse_graph(Context& ctx, const Graph<W>& g, const i32* vcmap, i64 nc);

template <class W>
void coarsen_vtx_w(Context& ctx, const Graph<W>& g, const i32* vcmap, Graph<W>& cg);

template <class W>
i64 coarsen_leidenR(Context& ctx, const Graph<W>& g, const Ordering& ord, const i32* constraint,
                    const ClusterState<typename Traits<W>::V>& cs, u32 seed_pick, u32 seed_order, i32* vcmap_out,
                    bool reuse_pvals = false);

// ---------------------------------------------------------------------------
// multilevel drivers (src/clustering_methods.cpp)
// ---------------------------------------------------------------------------
struct RunStats {
    i64 levels = 0;
    i64 total_nnz = 0;
    i64 sweeps = 0;
    i64 moves = 0;
    i64 passes = 0;
    // learned move filter judge (run_clustering with the filter on)
    i64 filtered_passes = 0;  // passes run with the filter
    i64 exact_passes = 0;     // exact passes the judge ran after them
    double judge_gain = 0;    // objective change those exact passes made
    i64 fell_back = 0;        // 1: the gain exceeded the filter's tolerance
};

enum Method { METHOD_LOUVAIN = 0, METHOD_LEIDEN = 1, METHOD_LEIDEN_PLUS = 2 };

template <class W>
// input_is_last: `input` is the output of the context's last local move (on
// `top`), so its own-cluster weights are still in the context's workspace
void leiden_part(Context& ctx, const Graph<W>& top, ClusterState<typename Traits<W>::V>& rfd, bool plus, bool improve,
                 const i32* input, u64 seed, i32* labels_out, RunStats* st, bool input_is_last = false);
// the method then ex_iters improvement passes (< 0: while the objective rises)
template <class W>
void run_clustering(Context& ctx, const Graph<W>& g, ClusterState<typename Traits<W>::V>& cs, int method, int ex_iters,
                    u64 seed, i32* labels_out, RunStats* rs);
template <class W>
void louvain_part(Context& ctx, const Graph<W>& top, ClusterState<typename Traits<W>::V>& rfd, bool constrained,
                  const i32* constraint, i32* labels_out, RunStats* st);

// ---------------------------------------------------------------------------
// memetic driver (app/memetic_clustering.cpp:27-219)
// ---------------------------------------------------------------------------
struct MemeStats {
    double objective = 0;
    i64 label_count = 0;
    i64 offspring = 0;
    i64 replaced = 0;
    double best_initial = 0;
};
// ranks of the distinct (c1[i], c2[i]) pairs in ascending order; returns their count
i64 intersect_clusters(Context& ctx, const i32* c1, const i32* c2, i64 n, i32* out);
// one bit per directed edge: set when its ends are in different clusters
template <class W>
void cut_signature(Context& ctx, const Graph<W>& g, const i32* labels, u32* sign);
// offspring < 0: no count limit; time_limit_s <= 0: no time limit
template <class W>
void meme_cluster(Context& ctx, const Graph<W>& g, int objective, double lambda_mult, int pop_size, i64 offspring,
                  double time_limit_s, u64 seed, i32* labels_out, MemeStats* st);

}  // namespace pggc
