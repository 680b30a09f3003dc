// ref_harness.cpp -- C entry points over the reference's OWN clustering
// sources (src/*.cpp of euphoricpoptarts/PennsylvaniaGPUGraphClustering,
// compiled unmodified from where they lie, against the serial Kokkos /
// KokkosKernels / thrust stand-ins in oracle/ref_shim/).
//
// TEST INFRASTRUCTURE ONLY: built into oracle/_ref/ by `make ref` (only where
// the reference sources are present) and loaded by tests/ through
// oracle/ref.py, to check the CPU oracle -- and through it the CUDA library --
// against the reference's code.  Nothing in the product loads it.
//
// Types are the reference's (interface/core_types.h:8-14): int32 vertex ids,
// int32 edge offsets and int32 weights, so graphs here have nnz < 2^31 and
// integer weights.  Seeds: the reference draws them from std::random_device
// (src/leidenR.cpp:289,403,480); here every draw comes from a splitmix64
// stream that run_clustering restarts at seed + p * 0x9E3779B97F4A7C15 for pass
// p -- the stream the CUDA library and the oracle use -- so the refinement's
// random picks see the same seeds on all three.
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "clustering_methods.h"
#include "header/contract.h"
#include "header/leidenR.h"
#include "header/ordering.h"
// The local mover is compiled as part of this file (not as its own object) so
// that its internal steps (candidates_and_destinations, afterburner_filter,
// set_new_cluster_ids, perform_moves, ...) can be driven one sweep at a time.
#include "local_mover.cpp"

namespace pggc_ref {

namespace {
uint64_t g_state = 0;
std::string g_error;
// seeds handed out before the stream (a test queues the two seeds of one
// coarsen_leidenR call)
std::vector<unsigned int> g_queue;
}  // namespace

// splitmix64 (Steele, Lea, Flood 2014)
unsigned int next_random_seed() {
    if (!g_queue.empty()) {
        const unsigned int v = g_queue.front();
        g_queue.erase(g_queue.begin());
        return v;
    }
    uint64_t z = (g_state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return (unsigned int)(z ^ (z >> 31));
}

}  // namespace pggc_ref

namespace {

using namespace jet_community;
using vtx_view = Kokkos::View<ordinal_t*, Device>;
using wgt_view = Kokkos::View<value_t*, Device>;
using row_view = Kokkos::View<edge_offset_t*, Device>;

enum { OBJ_MOD = 0, OBJ_WMOD = 1, OBJ_CPM = 2, OBJ_NLCC = 3, OBJ_LCC = 4 };
enum { METHOD_LOUVAIN = 0, METHOD_LEIDEN = 1, METHOD_LEIDEN_PLUS = 2 };

// weighted_graph from caller arrays (w == nullptr: unit weights)
weighted_graph make_graph(int64_t n, int64_t nnz, const int64_t* rowptr, const int32_t* col, const int32_t* w,
                          bool uniform) {
    if (n < 0 || nnz < 0 || nnz >= ((int64_t)1 << 31) || n >= ((int64_t)1 << 31))
        throw std::invalid_argument("graph too large for the reference's int32 types");
    row_view rm("row map", n + 1);
    vtx_view ent("entries", nnz);
    wgt_view val("values", nnz);
    for (int64_t i = 0; i <= n; i++) rm(i) = (edge_offset_t)rowptr[i];
    for (int64_t j = 0; j < nnz; j++) {
        ent(j) = col[j];
        val(j) = w ? w[j] : 1;
    }
    typename matrix_t::staticcrsgraph_type gr(ent, rm);
    weighted_graph wg;
    wg.mtx = matrix_t("g", (ordinal_t)n, val, gr);
    wg.edge_uniform = uniform;
    return wg;
}

// app/io/vertex_weighting.cpp:27-42 (the caller's weights when given)
wgt_view vertex_weights(const weighted_graph& wg, int objective, const int64_t* vw) {
    const ordinal_t n = wg.mtx.numRows();
    wgt_view out("vertex weights", n);
    for (ordinal_t i = 0; i < n; i++) {
        if (vw) out(i) = (value_t)vw[i];
        else if (objective == OBJ_MOD) out(i) = wg.mtx.graph.row_map(i + 1) - wg.mtx.graph.row_map(i);
        else if (objective == OBJ_WMOD) {
            value_t s = 0;
            for (edge_offset_t j = wg.mtx.graph.row_map(i); j < wg.mtx.graph.row_map(i + 1); j++) s += wg.mtx.values(j);
            out(i) = s;
        } else out(i) = 1;
    }
    return out;
}

// app/objective_helpers.hpp:9-22
std::unique_ptr<cluster_data> make_objective(const weighted_graph& wg, int objective, double mult) {
    switch (objective) {
        case OBJ_MOD: return std::make_unique<modularity>(wg.mtx, wg.vtx_w, mult, true);
        case OBJ_WMOD: return std::make_unique<modularity>(wg.mtx, wg.vtx_w, mult, wg.edge_uniform);
        case OBJ_NLCC: return std::make_unique<normalized_lcc>(wg.mtx, wg.vtx_w, mult, wg.edge_uniform);
        case OBJ_CPM: return std::make_unique<constant_potts>(wg.mtx, wg.vtx_w, mult);
        default: return std::make_unique<cluster_data>(wg.mtx, wg.vtx_w, mult);
    }
}

weighted_graph load(int64_t n, int64_t nnz, const int64_t* rowptr, const int32_t* col, const int32_t* w,
                    int objective, const int64_t* vw) {
    const bool uniform = w == nullptr || objective == OBJ_MOD || objective == OBJ_CPM;
    weighted_graph wg = make_graph(n, nnz, rowptr, col, uniform ? nullptr : w, uniform);
    wg.vtx_w = vertex_weights(wg, objective, vw);
    return wg;
}

template <class F>
int guarded(F f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        pggc_ref::g_error = e.what();
        return 1;
    }
}

}  // namespace

extern "C" {

const char* ref_last_error(void) { return pggc_ref::g_error.c_str(); }

// ordering::generate_orderings (src/ordering.cpp:131-164)
int ref_generate_orderings(int64_t n, int64_t nnz, const int64_t* rowptr, const int32_t* col, int32_t* order1,
                           int32_t* order2, int64_t* offsets4) {
    return guarded([&] {
        weighted_graph wg = load(n, nnz, rowptr, col, nullptr, OBJ_MOD, nullptr);
        auto rfd = make_objective(wg, OBJ_MOD, 1.0);
        memory_store mem(wg.mtx, *rfd);
        ordering::generate_orderings(mem, wg.mtx);
        for (int64_t i = 0; i < n; i++) {
            order1[i] = mem.o_mem.order1(i);
            order2[i] = mem.o_mem.order2(i);
        }
        offsets4[0] = mem.o_mem.offset_large;
        offsets4[1] = mem.o_mem.offset_large2;
        offsets4[2] = mem.o_mem.offset_mid;
        offsets4[3] = mem.o_mem.offset_mid2;
    });
}

// contracter::build_coarse_graph<uniform, false> (src/contract.cpp:234-336):
// the coarse CSR in the reference's row order (hash-slot order), its weights
// and the coarse vertex weights summed over vcmap (coarsen_vtx_w,
// src/clustering_methods.cpp:33-38).  Outputs: rowptr_out (nc+1), col_out and
// w_out (cap entries), vw_out (nc); *nnz_out the coarse edge count.
int ref_build_coarse_graph(int64_t n, int64_t nnz, const int64_t* rowptr, const int32_t* col, const int32_t* w,
                           const int32_t* vcmap, int64_t nc, int64_t* rowptr_out, int32_t* col_out, int32_t* w_out,
                           int64_t cap, int64_t* vw_out, int64_t* nnz_out) {
    return guarded([&] {
        const int obj = w ? OBJ_WMOD : OBJ_MOD;
        weighted_graph wg = load(n, nnz, rowptr, col, w, obj, nullptr);
        auto rfd = make_objective(wg, obj, 1.0);
        memory_store mem(wg.mtx, *rfd);
        ordering::generate_orderings(mem, wg.mtx);
        vtx_view map("vcmap", n);
        for (int64_t i = 0; i < n; i++) map(i) = vcmap[i];
        weighted_graph cg = wg.edge_uniform
                                ? contracter::build_coarse_graph<true, false>(wg, map, (ordinal_t)nc, mem)
                                : contracter::build_coarse_graph<false, false>(wg, map, (ordinal_t)nc, mem);
        const int64_t cnnz = cg.mtx.nnz();
        *nnz_out = cnnz;
        if (cnnz > cap) throw std::invalid_argument("coarse graph larger than the output capacity");
        for (int64_t c = 0; c <= nc; c++) rowptr_out[c] = cg.mtx.graph.row_map(c);
        for (int64_t j = 0; j < cnnz; j++) {
            col_out[j] = cg.mtx.graph.entries(j);
            w_out[j] = cg.mtx.values(j);
        }
        for (int64_t c = 0; c < nc; c++) vw_out[c] = 0;
        for (int64_t i = 0; i < n; i++) vw_out[vcmap[i]] += wg.vtx_w(i);
    });
}

// local_move_heuristic::local_move<false> from singletons (is_initial, with
// simulated annealing), the first step of every method
// (src/local_mover.cpp:1361-1417): labels, objective and label count after it.
int ref_local_move_initial(int64_t n, int64_t nnz, const int64_t* rowptr, const int32_t* col, const int32_t* w,
                           int objective, int32_t* labels_out, double* objective_out, int64_t* label_count_out) {
    return guarded([&] {
        weighted_graph wg = load(n, nnz, rowptr, col, w, objective, nullptr);
        auto rfd = make_objective(wg, objective, 1.0);
        memory_store mem(wg.mtx, *rfd);
        ordering::generate_orderings(mem, wg.mtx);
        vtx_view part("part", n);
        for (int64_t i = 0; i < n; i++) part(i) = (ordinal_t)i;
        vtx_view constraint;
        local_move_heuristic::local_move<false>(wg, part, *rfd, true, mem, constraint, true);
        for (int64_t i = 0; i < n; i++) labels_out[i] = part(i);
        *objective_out = rfd->get_objective();
        *label_count_out = rfd->label_count;
    });
}

// The sweep loop of local_move<false> (src/local_mover.cpp:1361-1417), run by
// the reference's own steps, stopped after `sweep_limit` sweeps (< 0: the
// whole annealing schedule) -- the state a sweep-by-sweep comparison needs.
// part_io holds the starting partition (singletons when is_initial) and
// receives the best partition, relabelled as the reference does.
int ref_local_move_sweeps(int64_t n, int64_t nnz, const int64_t* rowptr, const int32_t* col, const int32_t* w,
                          int objective, int is_initial, int enable_sa, int sweep_limit, int32_t* part_io,
                          double* objective_out, int64_t* label_count_out, int64_t* sweeps_out) {
    return guarded([&] {
        namespace lm = local_move_heuristic;
        weighted_graph wg = load(n, nnz, rowptr, col, w, objective, nullptr);
        auto rfd = make_objective(wg, objective, 1.0);
        memory_store mem(wg.mtx, *rfd);
        ordering::generate_orderings(mem, wg.mtx);
        vtx_view best_part("best part", n);
        for (int64_t i = 0; i < n; i++) best_part(i) = part_io[i];
        cluster_data& best_state = *rfd;
        if (!is_initial) {
            // cluster_data of the given partition: volumes, uncut, objective
            ordinal_t L = 0;
            for (int64_t i = 0; i < n; i++) L = std::max<ordinal_t>(L, best_part(i) + 1);
            for (ordinal_t c = 0; c < wg.mtx.numRows(); c++) best_state.total_deg(c) = 0;
            for (int64_t i = 0; i < n; i++) best_state.total_deg(best_part(i)) += wg.vtx_w(i);
            edge_offset_t uncut = 0;
            for (int64_t i = 0; i < n; i++)
                for (edge_offset_t j = wg.mtx.graph.row_map(i); j < wg.mtx.graph.row_map(i + 1); j++)
                    if (best_part(wg.mtx.graph.entries(j)) == best_part(i)) uncut += wg.edge_uniform ? 1 : wg.mtx.values(j);
            best_state.uncut = uncut;
            best_state.label_count = L;
            best_state.update_objective();
        }
        const matrix_t g = wg.mtx;
        vtx_view constraint;
        cluster_data& curr_state = mem.spare_cluster_data;
        curr_state.copy(best_state);
        vtx_view part = Kokkos::subview(mem.p_mem.part, std::make_pair(static_cast<ordinal_t>(0), g.numRows()));
        Kokkos::deep_copy(part, best_part);
        lm::cdata_t cdata = lm::truncate_and_init_mem(mem, wg, best_state.label_count, best_state.top_nnz == g.nnz());
        if (!is_initial) {
            if (wg.edge_uniform) lm::init_conn_graph<true>(wg, part, cdata, mem);
            else lm::init_conn_graph<false>(wg, part, cdata, mem);
            curr_state.last_pval = lm::pval_sum(mem.p_mem.pvals, g.numRows());
        } else {
            curr_state.last_pval = 0;
        }
        lm::clone_pval(mem, g.numRows());
        int iter_count = 0;
        const float ratios[2] = {0.75f, 0.25f};
        const int limits[2] = {4, 2};
        bool stop = false;
        for (int x = 0; x < 2 && !stop; x++) {
            float filter_ratio = enable_sa ? ratios[x] : 0;
            int count = 0;
            while (count++ < limits[x]) {
                if (sweep_limit >= 0 && iter_count >= sweep_limit) {
                    stop = true;
                    break;
                }
                iter_count++;
                vtx_view moves;
                matrix_t c_graph = cdata.c_graph;
                if (!cdata.init) c_graph = g;
                if (wg.edge_uniform && !cdata.init)
                    moves = lm::candidates_and_destinations<true, false>(wg, c_graph, part, curr_state, mem, filter_ratio,
                                                                         constraint);
                else
                    moves = lm::candidates_and_destinations<false, false>(wg, c_graph, part, curr_state, mem,
                                                                          filter_ratio, constraint);
                if (moves.extent(0) == 0) {
                    stop = true;
                    break;
                }
                if (wg.edge_uniform) moves = lm::afterburner_filter<true>(moves, wg, part, curr_state, mem);
                else moves = lm::afterburner_filter<false>(moves, wg, part, curr_state, mem);
                if (moves.extent(0) == 0) {
                    stop = true;
                    break;
                }
                if (iter_count > 1 || !is_initial) lm::set_new_cluster_ids<false>(moves, part, curr_state, mem, constraint);
                if (wg.edge_uniform) lm::perform_moves<true>(wg, part, moves, cdata, mem, curr_state);
                else lm::perform_moves<false>(wg, part, moves, cdata, mem, curr_state);
                if (curr_state.obj > best_state.obj) {
                    best_state.copy(curr_state);
                    Kokkos::deep_copy(best_part, part);
                    lm::clone_pval(mem, g.numRows());
                }
            }
        }
        lm::relabel_contiguously(best_part, best_state, mem);
        for (int64_t i = 0; i < n; i++) part_io[i] = best_part(i);
        *objective_out = best_state.obj;
        *label_count_out = best_state.label_count;
        *sweeps_out = iter_count;
    });
}

// The first level of leiden_part (src/clustering_methods.cpp:60-88): the
// initial local move from singletons, then coarsen_leidenR<true, uniform>
// (src/leidenR.cpp:263-500) of its partition with the two seeds its
// std::random_device draws would give.  Outputs: the local move's labels, the
// refinement's map and coarse vertex count.
int ref_local_move_then_refine(int64_t n, int64_t nnz, const int64_t* rowptr, const int32_t* col, const int32_t* w,
                               int objective, uint32_t seed_pick, uint32_t seed_order, int32_t* part_out,
                               int32_t* vcmap_out, int64_t* nc_out) {
    return guarded([&] {
        weighted_graph wg = load(n, nnz, rowptr, col, w, objective, nullptr);
        auto rfd = make_objective(wg, objective, 1.0);
        memory_store mem(wg.mtx, *rfd);
        ordering::generate_orderings(mem, wg.mtx);
        vtx_view part("part", n);
        for (int64_t i = 0; i < n; i++) part(i) = (ordinal_t)i;
        vtx_view constraint;
        local_move_heuristic::local_move<false>(wg, part, *rfd, true, mem, constraint, true);
        pggc_ref::g_queue = {seed_pick, seed_order};
        ordinal_t nc = 0;
        vtx_view vcmap = wg.edge_uniform ? leidenR::coarsen_leidenR<true, true>(wg, part, mem, *rfd, nc)
                                         : leidenR::coarsen_leidenR<true, false>(wg, part, mem, *rfd, nc);
        pggc_ref::g_queue.clear();
        for (int64_t i = 0; i < n; i++) {
            part_out[i] = part(i);
            vcmap_out[i] = vcmap(i);
        }
        *nc_out = nc;
    });
}

// leiden_part<plus, improve> (src/clustering_methods.cpp:47-137) restated
// over the reference's own steps, with one change: every coarse graph's rows
// are sorted by column (KokkosSparse::sort_crs_matrix) before the next level
// uses them.  The reference emits coarse rows in hash-slot order
// (src/contract.cpp:310-328) and its refinement's edge picks depend on row
// order; the CUDA library and the oracle keep rows sorted.  With this hook
// the two can be compared level by level on the same rows.
vtx_view leiden_part_sorted_rows(memory_store& mem, weighted_graph top, cluster_data& rfd, bool plus, bool improve,
                                 vtx_view input) {
    namespace lm = local_move_heuristic;
    using policy = Kokkos::RangePolicy<Kokkos::Serial>;
    std::vector<weighted_graph> levels;
    std::vector<vtx_view> parts;
    levels.push_back(top);
    vtx_view part("cluster assignments", top.mtx.numRows());
    if (!improve) {
        for (ordinal_t x = 0; x < top.mtx.numRows(); x++) part(x) = x;
    } else {
        Kokkos::deep_copy(part, input);
    }
    while (true) {
        weighted_graph c = levels.back();
        double old_obj = rfd.obj;
        ordering::generate_orderings(mem, c.mtx);
        lm::local_move<false>(c, part, rfd, !improve && (levels.size() == 1), mem, part, true);
        if (c.mtx.nnz() > 100000 && old_obj == rfd.obj)
            lm::local_move<false>(c, part, rfd, !improve && (levels.size() == 1), mem, part, false);
        if (old_obj == rfd.obj) lm::local_move_strict<false>(c, part, rfd, !improve && (levels.size() == 1), mem, part);
        if (rfd.label_count == c.mtx.numRows()) {
            parts.push_back(part);
            break;
        }
        vtx_view louv = part;
        ordinal_t coarse_vtx_count = 0;
        vtx_view coarse_map;
        if (levels.size() == 1 && c.edge_uniform)
            coarse_map = leidenR::coarsen_leidenR<true, true>(c, louv, mem, rfd, coarse_vtx_count);
        else if (levels.size() == 1 && !c.edge_uniform)
            coarse_map = leidenR::coarsen_leidenR<true, false>(c, louv, mem, rfd, coarse_vtx_count);
        else coarse_map = leidenR::coarsen_leidenR<false, false>(c, louv, mem, rfd, coarse_vtx_count);
        parts.push_back(coarse_map);
        if (coarse_vtx_count < c.mtx.numRows()) {
            weighted_graph next_level;
            if (c.edge_uniform) next_level = contracter::build_coarse_graph<true, false>(c, coarse_map, coarse_vtx_count, mem);
            else next_level = contracter::build_coarse_graph<false, false>(c, coarse_map, coarse_vtx_count, mem);
            KokkosSparse::sort_crs_matrix(Kokkos::Serial(), next_level.mtx.graph.row_map, next_level.mtx.graph.entries,
                                          next_level.mtx.values);
            // coarsen_vtx_w and downsample (src/clustering_methods.cpp:33-45)
            next_level.vtx_w = wgt_view("weighted degree 2", coarse_vtx_count);
            for (ordinal_t i = 0; i < c.mtx.numRows(); i++) next_level.vtx_w(coarse_map(i)) += c.vtx_w(i);
            part = vtx_view("cluster assignments coarse", coarse_vtx_count);
            for (ordinal_t i = 0; i < c.mtx.numRows(); i++) part(coarse_map(i)) = louv(i);
            levels.push_back(next_level);
        } else {
            levels.push_back(c);
        }
    }
    for (int64_t i = (int64_t)levels.size() - 2; i >= 0; i--) {
        weighted_graph c = levels[i];
        vtx_view coarse_part = parts[i + 1];
        vtx_view fine_part = parts[i];
        Kokkos::parallel_for("update top level assignments", policy(0, c.mtx.numRows()),
                             [=](const ordinal_t x) { fine_part(x) = coarse_part(fine_part(x)); });
        if (plus) {
            ordering::generate_orderings(mem, c.mtx);
            lm::local_move<false>(c, fine_part, rfd, false, mem, part, true);
        }
    }
    return parts[0];
}

// run_clustering (app/cluster_main.cpp:116-165) with the termination rule of
// iteration_termination_condition (:101-114): the method, then improvement
// passes (ex_iters < 0: while the objective rises).  vw may be NULL (default
// vertex weights of the objective).
// sorted_rows != 0: pLeiden / pLeiden+ through leiden_part_sorted_rows.
int ref_run_clustering(int64_t n, int64_t nnz, const int64_t* rowptr, const int32_t* col, const int32_t* w,
                       const int64_t* vw, int objective, double lambda_mult, int method, int ex_iters, uint64_t seed,
                       int sorted_rows, int32_t* labels_out, double* objective_out, int64_t* label_count_out,
                       int64_t* passes_out) {
    return guarded([&] {
        weighted_graph wg = load(n, nnz, rowptr, col, w, objective, vw);
        auto rfd = make_objective(wg, objective, lambda_mult);
        memory_store mem(wg.mtx, *rfd);
        ExperimentLoggerUtil<value_t> experiment;
        uint64_t pass = 0;
        auto one = [&](bool improve, vtx_view constraint) -> vtx_view {
            pggc_ref::g_state = seed + 0x9E3779B97F4A7C15ull * pass;
            pass++;
            if (method == METHOD_LOUVAIN) {
                if (improve) return clustering_methods::louvain_part<true>(mem, wg, *rfd, experiment, constraint);
                return clustering_methods::louvain_part<false>(mem, wg, *rfd, experiment, constraint);
            }
            if (sorted_rows) return leiden_part_sorted_rows(mem, wg, *rfd, method == METHOD_LEIDEN_PLUS, improve, constraint);
            if (method == METHOD_LEIDEN_PLUS) {
                if (improve) return clustering_methods::leiden_part<true, true>(mem, wg, *rfd, experiment, constraint);
                return clustering_methods::leiden_part<true, false>(mem, wg, *rfd, experiment, constraint);
            }
            if (improve) return clustering_methods::leiden_part<false, true>(mem, wg, *rfd, experiment, constraint);
            return clustering_methods::leiden_part<false, false>(mem, wg, *rfd, experiment, constraint);
        };
        vtx_view constraint;
        vtx_view part = one(false, constraint);
        double last = -std::numeric_limits<double>::infinity();
        int counter = 0;
        while (true) {
            bool terminate = true;
            if (ex_iters < 0) {
                if (rfd->get_objective() > last) terminate = false;
                last = rfd->get_objective();
            } else {
                if (counter++ < ex_iters) terminate = false;
            }
            if (terminate) break;
            constraint = part;
            part = one(true, constraint);
        }
        for (int64_t i = 0; i < n; i++) labels_out[i] = part(i);
        *objective_out = rfd->get_objective();
        *label_count_out = rfd->label_count;
        *passes_out = (int64_t)pass;
    });
}

}  // extern "C"
