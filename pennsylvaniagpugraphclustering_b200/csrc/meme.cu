// meme.cu -- the memetic driver (app/memetic_clustering.cpp:118-219) on the
// B200 path: a population of pLeiden+ clusterings, offspring from the
// intersection of two parents refined by constrained pLouvain and pLeiden+
// improvement passes, replacement of the most similar worse member by
// cut-edge signature distance.
//
// Device pieces:
//  * intersection_cluster (:27-62): the reference hashes (a, b) = (c1[i],
//    c2[i]) into slots whose order depends on the race between inserts; here
//    the new ids are the ranks of the distinct pairs in ascending (a, b) order
//    (one radix sort of the packed pairs, a head flag scan), so the offspring
//    constraint is deterministic;
//  * gen_signature (:64-104): one bit per directed edge, set when its ends lie
//    in different clusters; one thread per 32-edge word (ballot-free: the word
//    is assembled in a register), so no atomics;
//  * get_cut_diff (:106-116): popcount of the XOR of two signatures, summed.
// The host loop keeps the reference's selection (two binary tournaments with
// distinct winners), offspring recipe and replacement rule, with a seeded
// splitmix64 stream in place of std::random_device and an offspring count in
// place of (or besides) the wall-clock limit.
#include <chrono>
#include <limits>
#include "kernels.cuh"

namespace pggc {

__global__ void k_pair_keys(const i32* c1, const i32* c2, i64 n, int shift, u64* keys, i32* ids) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
        keys[i] = ((u64)(u32)c1[i] << shift) | (u64)(u32)c2[i];
        ids[i] = (i32)i;
    }
}

struct PairHeadIn {
    const u64* keys;
    __device__ i64 operator()(i64 x) const { return (x == 0 || keys[x] != keys[x - 1]) ? 1 : 0; }
};
struct PairHeadEpi {
    const u64* keys;
    const i32* ids;
    i32* out;
    // excl = number of heads before x: the rank of x's pair is excl + v - 1
    __device__ void operator()(i64 x, i64 excl, i64 v) const { out[ids[x]] = (i32)(excl + v - 1); }
};

// labels c1, c2 in [0, n): out[i] = rank of (c1[i], c2[i]) among the distinct pairs
i64 intersect_clusters(Context& ctx, const i32* c1, const i32* c2, i64 n, i32* out) {
    if (n <= 0) return 0;
    const int shift = std::max(1, bits_for((u64)(n - 1)));
    DBuf<u64> keys(ctx, n), keys2(ctx, n);
    DBuf<i32> ids(ctx, n), ids2(ctx, n);
    const int grid = (int)std::min<i64>(ceil_div(n, 256), (i64)ctx.num_sms * 16);
    k_pair_keys<<<grid, 256, 0, ctx.stream>>>(c1, c2, n, shift, keys.p, ids.p);
    PGGC_LAUNCH_CHECK();
    radix_sort_pairs<i32>(ctx, keys.p, ids.p, n, 0, 2 * shift, keys2.p, ids2.p);
    DBuf<i64> total(ctx, 1);
    scan_apply(ctx, PairHeadIn{keys.p}, PairHeadEpi{keys.p, ids.p, out}, n, nullptr, total.p);
    return ctx.read1(total.p);
}

// one thread per signature word: bits of edges [32w, 32w + 32)
template <class W>
__global__ void k_signature(DGraph<W> g, const i32* lab, i64 words, u32* sign) {
    for (i64 w = blockIdx.x * (i64)blockDim.x + threadIdx.x; w < words; w += (i64)gridDim.x * blockDim.x) {
        const i64 j0 = w * 32, j1 = min(j0 + 32, g.nnz);
        // source of edge j0: largest i with rowptr[i] <= j0
        i64 lo = 0, hi = g.n - 1;
        while (lo < hi) {
            const i64 mid = (lo + hi + 1) >> 1;
            if (g.rowptr[mid] <= j0) lo = mid;
            else hi = mid - 1;
        }
        i64 i = lo;
        u32 bits = 0;
        for (i64 j = j0; j < j1; j++) {
            while (g.rowptr[i + 1] <= j) i++;
            if (lab[i] != lab[g.col[j]]) bits |= 1u << (u32)(j - j0);
        }
        sign[w] = bits;
    }
}

template <class W>
void cut_signature(Context& ctx, const Graph<W>& g, const i32* labels, u32* sign) {
    const i64 words = ceil_div(std::max<i64>(g.nnz, 1), 32);
    if (g.nnz == 0) {
        PGGC_CUDA(cudaMemsetAsync(sign, 0, sizeof(u32) * words, ctx.stream));
        return;
    }
    const int grid = (int)std::min<i64>(ceil_div(words, 256), (i64)ctx.num_sms * 16);
    k_signature<W><<<grid, 256, 0, ctx.stream>>>(g.view(), labels, words, sign);
    PGGC_LAUNCH_CHECK();
}

struct XorPopIn {
    const u32* a;
    const u32* b;
    __device__ i64 operator()(i64 x) const { return __popc(a[x] ^ b[x]); }
};

i64 cut_diff(Context& ctx, const u32* a, const u32* b, i64 words, i64* d_scratch) {
    sum_i64(ctx, XorPopIn{a, b}, words, d_scratch);
    return ctx.read1(d_scratch);
}

// uniform integer in [0, m) from a splitmix64 stream (m > 0): multiply-shift
static inline i64 uniform_below(SplitMix64& r, i64 m) { return (i64)(((unsigned __int128)r.next() * (u64)m) >> 64); }

template <class W>
void meme_cluster(Context& ctx, const Graph<W>& g, int objective, double lambda_mult, int pop_size, i64 offspring,
                  double time_limit_s, u64 seed, i32* labels_out, MemeStats* st) {
    using V = typename Traits<W>::V;
    if (pop_size < 2) throw InvalidArg("pop_size must be at least 2");
    const i64 n = g.n;
    const i64 words = ceil_div(std::max<i64>(g.nnz, 1), 32);
    struct Member {
        DBuf<i32> clusters;
        DBuf<u32> sign;
        double obj = 0;
        i64 labels = 0;
    };
    std::vector<Member> pop((size_t)pop_size);
    SplitMix64 rng(seed);
    DBuf<i64> scratch(ctx, 1);
    auto fresh = [&](ClusterState<V>& cs) { make_cluster_state<W>(ctx, g, objective, lambda_mult, cs); };
    double best_initial = -std::numeric_limits<double>::infinity();
    for (int p = 0; p < pop_size; p++) {
        ClusterState<V> cs;
        fresh(cs);
        Member& m = pop[p];
        m.clusters = DBuf<i32>(ctx, std::max<i64>(n, 1));
        m.sign = DBuf<u32>(ctx, words);
        leiden_part<W>(ctx, g, cs, true, false, nullptr, rng.next(), m.clusters.p, nullptr);
        m.obj = cs.get_objective();
        m.labels = cs.label_count;
        cut_signature<W>(ctx, g, m.clusters.p, m.sign.p);
        best_initial = std::max(best_initial, m.obj);
    }
    const auto t0 = std::chrono::steady_clock::now();
    auto elapsed = [&]() { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };
    DBuf<i32> constraint(ctx, std::max<i64>(n, 1)), child(ctx, std::max<i64>(n, 1)), tmp(ctx, std::max<i64>(n, 1));
    DBuf<u32> csign(ctx, words);
    i64 made = 0, replaced = 0;
    // binary tournament as in the reference (:151-163): a in [0, pop), the
    // second index (a + [0, pop - 1)) mod pop, the better objective wins
    auto pick = [&]() {
        const i64 a = uniform_below(rng, pop_size);
        const i64 b = (a + uniform_below(rng, pop_size - 1)) % pop_size;
        return pop[a].obj > pop[b].obj ? a : b;
    };
    while ((offspring < 0 || made < offspring) && (time_limit_s <= 0 || elapsed() < time_limit_s)) {
        const i64 p1 = pick();
        i64 p2 = p1;
        while (p2 == p1) p2 = pick();
        intersect_clusters(ctx, pop[p1].clusters.p, pop[p2].clusters.p, n, constraint.p);
        ClusterState<V> cs;
        fresh(cs);
        louvain_part<W>(ctx, g, cs, true, constraint.p, child.p, nullptr);
        for (int x = 0; x < 5; x++) {
            copy_d2d(ctx, tmp.p, child.p, n);
            leiden_part<W>(ctx, g, cs, true, true, tmp.p, rng.next(), child.p, nullptr);
        }
        made++;
        const double obj = cs.get_objective();
        cut_signature<W>(ctx, g, child.p, csign.p);
        // replace the most similar member that is worse than the child
        i64 am = -1;
        i64 min_diff = std::numeric_limits<i64>::max();
        for (int p = 0; p < pop_size; p++) {
            if (pop[p].obj < obj) {
                const i64 d = cut_diff(ctx, csign.p, pop[p].sign.p, words, scratch.p);
                if (d < min_diff) {
                    min_diff = d;
                    am = p;
                }
            }
        }
        if (am >= 0) {
            copy_d2d(ctx, pop[am].clusters.p, child.p, n);
            copy_d2d(ctx, pop[am].sign.p, csign.p, words);
            pop[am].obj = obj;
            pop[am].labels = cs.label_count;
            replaced++;
        }
    }
    int am = 0;
    for (int p = 1; p < pop_size; p++)
        if (pop[p].obj > pop[am].obj) am = p;
    copy_d2d(ctx, labels_out, pop[am].clusters.p, n);
    ctx.sync();
    if (st) {
        st->objective = pop[am].obj;
        st->label_count = pop[am].labels;
        st->offspring = made;
        st->replaced = replaced;
        st->best_initial = best_initial;
    }
}

template void cut_signature<i32>(Context&, const Graph<i32>&, const i32*, u32*);
template void cut_signature<float>(Context&, const Graph<float>&, const i32*, u32*);
template void meme_cluster<i32>(Context&, const Graph<i32>&, int, double, int, i64, double, u64, i32*, MemeStats*);
template void meme_cluster<float>(Context&, const Graph<float>&, int, double, int, i64, double, u64, i32*, MemeStats*);

}  // namespace pggc
