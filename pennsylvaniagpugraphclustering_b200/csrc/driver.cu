// driver.cu -- objective state and the multilevel V-cycles
// (src/clustering_methods.cpp:33-222, interface/cluster_data.hpp:76-181,
//  app/io/vertex_weighting.cpp:27-42).
//
// The host C++ here plays the role of clustering_methods::leiden_part /
// louvain_part: it owns the level hierarchy (device-resident coarse graphs and
// coarse maps) and sequences the kernel families.  Decisions the reference
// makes on host scalars (objective unchanged, label_count == n, coarse count)
// stay on the host; everything else stays on the device.
#include <limits>
#include "kernels.cuh"

namespace pggc {

// ---------------------------------------------------------------------------
// objective state
// ---------------------------------------------------------------------------
template <class V>
struct SqAll;
template <>
struct SqAll<i64> {
    const i64* td;
    __device__ i64 operator()(i64 i) const { return td[i] * td[i]; }
};
template <>
struct SqAll<double> {
    const double* td;
    __device__ double operator()(i64 i) const { return td[i] * td[i]; }
};
struct I64In {
    const i64* a;
    __device__ i64 operator()(i64 i) const { return a[i]; }
};
struct I32WIn {
    const i32* a;
    __device__ i64 operator()(i64 i) const { return a[i]; }
};
struct FWIn {
    const float* a;
    __device__ double operator()(i64 i) const { return (double)a[i]; }
};

template <class V>
void update_objective(Context& ctx, ClusterState<V>& cs) {
    DBuf<i64> si(ctx, 1);
    DBuf<double> sd(ctx, 1);
    double m;
    if constexpr (std::is_same<V, i64>::value) {
        sum_i64(ctx, SqAll<i64>{cs.total_deg.p}, cs.label_count, si.p);
        i64 ss = ctx.read1(si.p);
        m = static_cast<double>(cs.uncut);
        m = m - cs.lambda * static_cast<double>(ss);
    } else {
        det_reduce(ctx, SqAll<double>{cs.total_deg.p}, cs.label_count, sd.p);
        double ss = ctx.read1(sd.p);
        m = cs.uncut;
        m = m - cs.lambda * ss;
    }
    cs.obj = m;
}

template <class W>
__global__ void k_vw_warp(DGraph<W> g, int objective, typename Traits<W>::V* out) {
    using V = typename Traits<W>::V;
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
    for (i64 i = gw; i < g.n; i += nw) {
        i64 b = g.rowptr[i], e = g.rowptr[i + 1];
        V r;
        if (objective == OBJ_MOD) r = V(e - b);
        else if (objective == OBJ_WMOD) {
            if constexpr (std::is_same<V, double>::value) {
                if (e - b < MASSIVE_CUTOFF) r = (double)(float)warp_canon_sum(b, e, [&](i64 j) { return (double)g.wgt(j); });
                else r = -1.0;  // massive rows: k_vw_block
            } else {
                r = warp_int_sum(b, e, [&](i64 j) -> i64 { return g.wgt(j); });
            }
        } else r = V(1);
        if (lane_id() == 0 && !(std::is_same<V, double>::value && objective == OBJ_WMOD && e - b >= MASSIVE_CUTOFF))
            out[i] = r;
    }
}
template <class W>
__global__ void __launch_bounds__(1024) k_vw_block(DGraph<W> g, const i32* list, i64 count, double* out) {
    __shared__ double red[32];
    for (i64 x = blockIdx.x; x < count; x += gridDim.x) {
        i32 i = list[x];
        double r = block1024_canon_sum(g.rowptr[i], g.rowptr[i + 1], [&](i64 j) { return (double)g.wgt(j); }, red);
        if (threadIdx.x == 0) out[i] = (double)(float)r;
        __syncthreads();
    }
}

// app/io/vertex_weighting.cpp:27-42
template <class W>
void default_vertex_weights(Context& ctx, Graph<W>& g, int objective) {
    using V = typename Traits<W>::V;
    g.vtx_w = DBuf<V>(ctx, std::max<i64>(g.n, 1));
    if (g.n == 0) return;
    auto gv = g.view();
    gv.vtx_w = g.vtx_w.p;
    int grid = (int)std::min<i64>(ceil_div(ceil_div(g.n, 32), 8), (i64)ctx.num_sms * 16);
    k_vw_warp<W><<<grid, 256, 0, ctx.stream>>>(gv, objective, g.vtx_w.p);
    PGGC_LAUNCH_CHECK();
    if constexpr (std::is_same<V, double>::value) {
        if (objective == OBJ_WMOD) {
            const Ordering& ord = graph_ordering<W>(ctx, g);
            i64 nm = g.n - ord.off_large2;
            if (nm > 0) {
                k_vw_block<W><<<(int)std::min<i64>(nm, (i64)ctx.num_sms * 2), 1024, 0, ctx.stream>>>(
                    gv, ord.order1.p + ord.off_large2, nm, g.vtx_w.p);
                PGGC_LAUNCH_CHECK();
            }
        }
    }
}

template <class W>
void make_cluster_state(Context& ctx, const Graph<W>& g, int kind, double mult, ClusterState<typename Traits<W>::V>& cs) {
    using V = typename Traits<W>::V;
    cs.capacity = 2 * std::max<i64>(g.n, 1) + 64;
    cs.total_deg = DBuf<V>(ctx, cs.capacity);
    PGGC_CUDA(cudaMemsetAsync(cs.total_deg.p, 0, sizeof(V) * cs.capacity, ctx.stream));
    copy_d2d(ctx, cs.total_deg.p, g.vtx_w.p, g.n);
    cs.top_nnz = g.nnz;
    cs.uncut = 0;
    cs.label_count = g.n;
    cs.kind = kind;
    cs.lambda = 1.0;
    DBuf<i64> si(ctx, 1);
    DBuf<double> sd(ctx, 1);
    auto sum_vw = [&]() -> double {
        if constexpr (std::is_same<V, i64>::value) {
            sum_i64(ctx, I64In{g.vtx_w.p}, g.n, si.p);
            return (double)ctx.read1(si.p);
        } else {
            det_reduce(ctx, DArrIn{g.vtx_w.p}, g.n, sd.p);
            return ctx.read1(sd.p);
        }
    };
    cs.vol_total = sum_vw();
    if (kind == OBJ_MOD || kind == OBJ_WMOD) {
        double gdeg = g.uniform ? (double)g.nnz : cs.vol_total;
        cs.inv_gdeg = 1.0 / gdeg;
        cs.lambda = mult * cs.inv_gdeg;
    } else if (kind == OBJ_CPM) {
        cs.v_total = (double)g.n;
        cs.lambda = mult * 0.5;
    } else if (kind == OBJ_NLCC) {
        double gd;
        if (g.uniform) gd = (double)g.nnz;
        else {
            if constexpr (std::is_same<V, i64>::value) {
                sum_i64(ctx, I32WIn{(const i32*)g.view().w}, g.nnz, si.p);
                gd = (double)ctx.read1(si.p);
            } else {
                det_reduce(ctx, FWIn{(const float*)g.view().w}, g.nnz, sd.p);
                gd = ctx.read1(sd.p);
            }
        }
        cs.g_deg = gd;
        double denom;
        if constexpr (std::is_same<V, i64>::value) {
            sum_i64(ctx, I64In{g.vtx_w.p}, g.n, si.p);
            u64 vt = (u64)ctx.read1(si.p);
            denom = static_cast<double>(vt * vt);
        } else {
            double vt = sum_vw();
            denom = vt * vt;
        }
        cs.lambda = mult * gd / denom;
    } else {
        cs.lambda = mult;
    }
    update_objective(ctx, cs);
}

// ---------------------------------------------------------------------------
// small kernels of the V-cycle
// ---------------------------------------------------------------------------
__global__ void k_downsample(i64 n, const i32* in, const i32* map, i32* out) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) out[map[i]] = in[i];
}
__global__ void k_project(i64 n, i32* fine, const i32* coarse) {
    for (i64 x = blockIdx.x * (i64)blockDim.x + threadIdx.x; x < n; x += (i64)gridDim.x * blockDim.x)
        fine[x] = coarse[fine[x]];
}
// The reference's level loop has no bound (src/clustering_methods.cpp:59,147);
// a hierarchy this deep means the refinement stopped contracting.
constexpr i64 MAX_LEVELS = 4096;

inline int vgrid(Context& ctx, i64 n) { return (int)std::max<i64>(1, std::min<i64>(ceil_div(n, 256), (i64)ctx.num_sms * 16)); }

// leiden_part<plus,improve> (src/clustering_methods.cpp:47-137)
template <class W>
void leiden_part(Context& ctx, const Graph<W>& top, ClusterState<typename Traits<W>::V>& rfd, bool plus, bool improve,
                 const i32* input, u64 seed, i32* labels_out, RunStats* st, bool input_is_last) {
    std::vector<std::unique_ptr<Graph<W>>> coarse;
    std::vector<const Graph<W>*> levels;
    std::vector<DBuf<i32>> parts;
    levels.push_back(&top);
    const i64 n = top.n;
    DBuf<i32> part(ctx, std::max<i64>(n, 1));
    if (!improve) iota<i32>(ctx, part.p, n);
    else copy_d2d(ctx, part.p, input, n);
    SplitMix64 rng(seed);
    MoveStats ms;
    while (true) {
        const Graph<W>& c = *levels.back();
        if ((i64)levels.size() > MAX_LEVELS) throw DeviceFault("multilevel hierarchy exceeded MAX_LEVELS");
        double old_obj = rfd.obj;
        bool init = !improve && levels.size() == 1;
        const Ordering& ord = graph_ordering<W>(ctx, c);
        ctx.filt.level = (int)levels.size() - 1;
        // the level's later local moves (and the refinement) start from the
        // previous local move's output: its own-cluster weights are reused
        local_move<W>(ctx, c, ord, part.p, rfd, init, false, nullptr, true, false, -1, &ms,
                      levels.size() == 1 && improve && input_is_last);
        if (c.nnz > 100000 && old_obj == rfd.obj)
            local_move<W>(ctx, c, ord, part.p, rfd, init, false, nullptr, false, false, -1, &ms, true);
        if (old_obj == rfd.obj) local_move<W>(ctx, c, ord, part.p, rfd, init, false, nullptr, false, true, -1, &ms, true);
        if (rfd.label_count == c.n) {
            parts.push_back(std::move(part));
            break;
        }
        u32 s_pick = (u32)rng.next();
        u32 s_order = (u32)rng.next();
        DBuf<i32> cmap(ctx, std::max<i64>(c.n, 1));
        i64 nc = coarsen_leidenR<W>(ctx, c, ord, part.p, rfd, s_pick, s_order, cmap.p, true);
        if (nc < c.n) {
            auto next = build_coarse_graph<W>(ctx, c, cmap.p, nc);
            coarsen_vtx_w<W>(ctx, c, cmap.p, *next);
            DBuf<i32> np(ctx, std::max<i64>(nc, 1));
            k_downsample<<<vgrid(ctx, c.n), 256, 0, ctx.stream>>>(c.n, part.p, cmap.p, np.p);
            PGGC_LAUNCH_CHECK();
            parts.push_back(std::move(cmap));
            part = std::move(np);
            levels.push_back(next.get());
            coarse.push_back(std::move(next));
        } else {
            parts.push_back(std::move(cmap));
            levels.push_back(&c);
        }
    }
    if (st) {
        st->levels = (i64)levels.size();
        i64 t = 0;
        for (auto* l : levels) t += l->nnz;
        st->total_nnz = t;
    }
    for (i64 i = (i64)levels.size() - 2; i >= 0; i--) {
        const Graph<W>& c = *levels[i];
        k_project<<<vgrid(ctx, c.n), 256, 0, ctx.stream>>>(c.n, parts[i].p, parts[i + 1].p);
        PGGC_LAUNCH_CHECK();
        if (plus) {
            const Ordering& ord = graph_ordering<W>(ctx, c);
            // the finest level's last local move runs unfiltered: the exact
            // sweeps that catch what the learned filter skipped
            ctx.filt.level = (int)i;
            ctx.filt.suspended = i == 0;
            local_move<W>(ctx, c, ord, parts[i].p, rfd, false, false, nullptr, true, false, -1, &ms);
            ctx.filt.suspended = false;
        }
    }
    copy_d2d(ctx, labels_out, parts[0].p, n);
    if (st) {
        st->sweeps += ms.sweeps;
        st->moves += ms.moves;
    }
}

// louvain_part<constrained> (src/clustering_methods.cpp:139-222)
template <class W>
void louvain_part(Context& ctx, const Graph<W>& top, ClusterState<typename Traits<W>::V>& rfd, bool constrained,
                  const i32* constraint_in, i32* labels_out, RunStats* st) {
    using V = typename Traits<W>::V;
    if (constrained) {
        // cluster_data::reset (interface/cluster_data.hpp:48-54)
        copy_d2d(ctx, rfd.total_deg.p, top.vtx_w.p, top.n);
        rfd.uncut = 0;
        rfd.label_count = top.n;
        update_objective(ctx, rfd);
    }
    std::vector<std::unique_ptr<Graph<W>>> coarse;
    std::vector<const Graph<W>*> levels;
    std::vector<DBuf<i32>> parts;
    levels.push_back(&top);
    bool drop = constrained;
    DBuf<i32> constraint;
    if (constrained) {
        constraint = DBuf<i32>(ctx, rfd.capacity);
        PGGC_CUDA(cudaMemsetAsync(constraint.p, 0, sizeof(i32) * constraint.n, ctx.stream));
        copy_d2d(ctx, constraint.p, constraint_in, top.n);
    }
    MoveStats ms;
    while (true) {
        const Graph<W>& c = *levels.back();
        if ((i64)levels.size() > MAX_LEVELS) throw DeviceFault("multilevel hierarchy exceeded MAX_LEVELS");
        DBuf<i32> part(ctx, std::max<i64>(c.n, 1));
        iota<i32>(ctx, part.p, c.n);
        const Ordering& ord = graph_ordering<W>(ctx, c);
        ctx.filt.level = (int)levels.size() - 1;
        local_move<W>(ctx, c, ord, part.p, rfd, true, constrained, constrained ? constraint.p : nullptr, true, false, -1,
                      &ms);
        if (constrained && rfd.label_count == c.n)
            local_move<W>(ctx, c, ord, part.p, rfd, true, constrained, constraint.p, false, true, -1, &ms);
        i64 L = rfd.label_count;
        parts.push_back(std::move(part));
        if (L < c.n) {
            auto next = build_coarse_graph<W>(ctx, c, parts.back().p, L);
            next->vtx_w = DBuf<V>(ctx, std::max<i64>(L, 1));
            copy_d2d(ctx, next->vtx_w.p, rfd.total_deg.p, L);
            levels.push_back(next.get());
            coarse.push_back(std::move(next));
            if (constrained) {
                DBuf<i32> nxt(ctx, rfd.capacity);
                PGGC_CUDA(cudaMemsetAsync(nxt.p, 0, sizeof(i32) * nxt.n, ctx.stream));
                k_downsample<<<vgrid(ctx, c.n), 256, 0, ctx.stream>>>(c.n, constraint.p, parts.back().p, nxt.p);
                PGGC_LAUNCH_CHECK();
                constraint = std::move(nxt);
            }
        } else if (drop) {
            PGGC_CUDA(cudaMemsetAsync(constraint.p, 0, sizeof(i32) * constraint.n, ctx.stream));
            parts.pop_back();
            drop = false;
        } else {
            break;
        }
    }
    if (st) {
        st->levels = (i64)levels.size();
        i64 t = 0;
        for (auto* l : levels) t += l->nnz;
        st->total_nnz = t;
    }
    if (levels.size() > 1) {
        levels.pop_back();
        parts.pop_back();
    }
    for (i64 i = (i64)levels.size() - 2; i >= 0; i--) {
        const Graph<W>& c = *levels[i];
        k_project<<<vgrid(ctx, c.n), 256, 0, ctx.stream>>>(c.n, parts[i].p, parts[i + 1].p);
        PGGC_LAUNCH_CHECK();
        const Ordering& ord = graph_ordering<W>(ctx, c);
        ctx.filt.level = (int)i;
        ctx.filt.suspended = i == 0;
        local_move<W>(ctx, c, ord, parts[i].p, rfd, false, false, nullptr, true, false, -1, &ms);
        ctx.filt.suspended = false;
    }
    copy_d2d(ctx, labels_out, parts[0].p, top.n);
    if (st) {
        st->sweeps += ms.sweeps;
        st->moves += ms.moves;
    }
}

// run_clustering (app/cluster_main.cpp:116-165): the method, then improvement
// passes while iteration_termination_condition (:101-114) says continue
template <class W>
void run_clustering(Context& ctx, const Graph<W>& g, ClusterState<typename Traits<W>::V>& cs, int method, int ex_iters,
                    u64 seed, i32* labels_out, RunStats* rs) {
    const i64 n = g.n;
    DBuf<i32> part(ctx, std::max<i64>(n, 1)), con(ctx, std::max<i64>(n, 1));
    RunStats acc;
    u64 pass = 0;
    auto one = [&](bool improve) {
        ProfScope ps(ctx, improve ? "pass_improve" : "pass_first");
        ctx.filt.pass = (int)std::min<u64>(acc.passes, 1u << 30);
        RunStats r1;
        if (method == METHOD_LOUVAIN) {
            louvain_part<W>(ctx, g, cs, improve, con.p, part.p, &r1);
        } else {
            u64 s = seed + 0x9E3779B97F4A7C15ull * pass;
            pass++;
            // an improvement pass starts from the previous pass's output
            leiden_part<W>(ctx, g, cs, method == METHOD_LEIDEN_PLUS, improve, con.p, s, part.p, &r1, improve);
        }
        acc.levels = r1.levels;
        acc.total_nnz = r1.total_nnz;
        acc.sweeps += r1.sweeps;
        acc.moves += r1.moves;
        acc.passes++;
    };
    one(false);
    double last = -std::numeric_limits<double>::infinity();
    int counter = 0;
    while (true) {
        bool terminate = true;
        if (ex_iters < 0) {
            if (cs.get_objective() > last) terminate = false;
            last = cs.get_objective();
        } else {
            if (counter++ < ex_iters) terminate = false;
        }
        if (terminate) break;
        copy_d2d(ctx, con.p, part.p, n);
        one(true);
    }
    if (ctx.filt.mode == 2) {
        // Judge of the learned move filter: one exact (unfiltered) improvement
        // pass from the filtered result.  What it gains is what the filter gave
        // up; above FILTER_TOLERANCE the run falls back to the plain method --
        // exact passes from there while the objective rises -- and reports
        // the fallback.  The run ends on the exact passes' result either way.
        // The objective is cluster_data's FP64 value from exact int64 / FP64
        // sums (the verify_obj arithmetic of app/verify_objective.cpp:108-135).
        acc.filtered_passes = acc.passes;
        const double q_filtered = cs.get_objective();
        ctx.filt.mode = 0;
        bool fell_back = false;
        try {
            copy_d2d(ctx, con.p, part.p, n);
            one(true);
            acc.exact_passes++;
            fell_back = cs.get_objective() - q_filtered > FILTER_TOLERANCE;
            if (fell_back) {
                double prev = cs.get_objective();
                while (true) {
                    copy_d2d(ctx, con.p, part.p, n);
                    one(true);
                    acc.exact_passes++;
                    const double q = cs.get_objective();
                    if (!(q > prev)) break;
                    prev = q;
                }
            }
        } catch (...) {
            ctx.filt.mode = 2;
            throw;
        }
        ctx.filt.mode = 2;
        acc.judge_gain = cs.get_objective() - q_filtered;
        acc.fell_back = fell_back ? 1 : 0;
    }
    copy_d2d(ctx, labels_out, part.p, n);
    if (rs) *rs = acc;
}

#define PGGC_INST_DRV(W)                                                                                              \
    template void run_clustering<W>(Context&, const Graph<W>&, ClusterState<Traits<W>::V>&, int, int, u64, i32*,      \
                                    RunStats*);                                                                       \
    template void leiden_part<W>(Context&, const Graph<W>&, ClusterState<Traits<W>::V>&, bool, bool, const i32*, u64, \
                                 i32*, RunStats*, bool);                                                              \
    template void louvain_part<W>(Context&, const Graph<W>&, ClusterState<Traits<W>::V>&, bool, const i32*, i32*,     \
                                  RunStats*);                                                                         \
    template void make_cluster_state<W>(Context&, const Graph<W>&, int, double, ClusterState<Traits<W>::V>&);         \
    template void default_vertex_weights<W>(Context&, Graph<W>&, int);
PGGC_INST_DRV(i32)
PGGC_INST_DRV(float)
template void update_objective<i64>(Context&, ClusterState<i64>&);
template void update_objective<double>(Context&, ClusterState<double>&);

}  // namespace pggc
