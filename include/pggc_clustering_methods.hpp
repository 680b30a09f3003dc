// pggc_clustering_methods.hpp -- header-only C++ shim over include/pggc.h with
// the reference's names (interface/clustering_methods.h:20-24,
// interface/cluster_data.hpp, interface/weighted_graph.h,
// interface/memory_store.hpp), for callers that hold raw device pointers
// (e.g. the .data() of Kokkos views).  No Kokkos dependency.
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>

#include "pggc.h"

namespace pggc_shim {

inline void check(pggc_status s) {
    if (s != PGGC_OK) throw std::runtime_error(std::string("pggc: ") + pggc_last_error());
}

// memory_store: owns the device context (stream + memory pool)
struct memory_store {
    pggc_context* ctx = nullptr;
    explicit memory_store(int device = 0) { check(pggc_context_create(device, &ctx)); }
    ~memory_store() { pggc_context_destroy(ctx); }
    memory_store(const memory_store&) = delete;
    memory_store& operator=(const memory_store&) = delete;
};

// weighted_graph: a device copy of the CSR (int64 offsets)
struct weighted_graph {
    pggc_graph* g = nullptr;
    weighted_graph(memory_store& mem, int64_t n, int64_t nnz, const int64_t* row_map, const int32_t* entries,
                   const void* values, int weight_kind, const void* vtx_w, int objective, int mem_kind) {
        check(pggc_graph_create(mem.ctx, n, nnz, row_map, entries, values, weight_kind, vtx_w, objective, mem_kind,
                                &g));
    }
    ~weighted_graph() { pggc_graph_destroy(g); }
    weighted_graph(const weighted_graph&) = delete;
    weighted_graph& operator=(const weighted_graph&) = delete;
};

// cluster_data (get_objective, app/objective_helpers.hpp:9-22)
struct cluster_data {
    pggc_cluster_data* cd = nullptr;
    cluster_data(memory_store& mem, const weighted_graph& wg, int objective, double lambda_mult) {
        check(pggc_cluster_data_create(mem.ctx, wg.g, objective, lambda_mult, &cd));
    }
    ~cluster_data() { pggc_cluster_data_destroy(cd); }
    cluster_data(const cluster_data&) = delete;
    cluster_data& operator=(const cluster_data&) = delete;
    double get_objective() const {
        double v = 0;
        check(pggc_cluster_data_get(cd, nullptr, &v, nullptr, nullptr, nullptr));
        return v;
    }
    int64_t label_count() const {
        int64_t l = 0;
        check(pggc_cluster_data_get(cd, nullptr, nullptr, nullptr, nullptr, &l));
        return l;
    }
};

namespace clustering_methods {

// leiden_part<plus, improve>: labels_out / input are device int32 arrays of n
template <bool plus, bool improve>
void leiden_part(memory_store& mem, const weighted_graph& top, cluster_data& rfd, const int32_t* input,
                 int32_t* labels_out, uint64_t seed = 1, pggc_stats* stats = nullptr) {
    check(pggc_leiden_part(mem.ctx, top.g, rfd.cd, plus ? 1 : 0, improve ? 1 : 0, input, seed, labels_out,
                           PGGC_MEM_DEVICE, stats));
}

// louvain_part<constrained>
template <bool constrained>
void louvain_part(memory_store& mem, const weighted_graph& top, cluster_data& rfd, const int32_t* constraint,
                  int32_t* labels_out, pggc_stats* stats = nullptr) {
    check(pggc_louvain_part(mem.ctx, top.g, rfd.cd, constrained ? 1 : 0, constraint, labels_out, PGGC_MEM_DEVICE,
                            stats));
}

}  // namespace clustering_methods
}  // namespace pggc_shim
