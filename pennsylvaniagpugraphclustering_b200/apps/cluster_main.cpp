// cluster_main.cpp -- the plouvain / pleiden / pleiden+ programs
// (app/cluster_main.cpp:116-214; app/CMakeLists.txt:3-5 builds one per
// method, here PGGC_APP_METHOD selects it): -trials independent runs of the
// method followed by -ex_iters improvement passes, the best clustering written
// with -o, per-trial records appended to the -metrics JSON array.
//
// Usage: pleiden+ -i <graph.mtx|graph> [-o clusters.txt] [-objective Mod|WMod|CPM|NLCC|LCC]
//        [-lambda x] [-vtx_weights file] [-trials t] [-ex_iters k] [-metrics file.json]
//        [-seed s] [-device d]
#include <chrono>
#include <limits>

#include "app_common.hpp"

#ifndef PGGC_APP_METHOD
#define PGGC_APP_METHOD PGGC_METHOD_LEIDEN_PLUS
#endif

using namespace pggc_app;

namespace {

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Objective {
    double obj = 0, objective = 0, lambda = 0, uncut = 0;
    int64_t labels = 0;
    void read(const pggc_cluster_data* cd) { pggc_cluster_data_get(cd, &obj, &objective, &lambda, &uncut, &labels); }
};

void print_state(std::ostream& os, const Args& a, const Loaded& L, const Objective& o) {
    os << "Cut: ";
    if (L.weight_kind == PGGC_W_FLOAT32) os << (L.nnz - o.uncut) / 2;
    else os << ((long long)L.nnz - (long long)o.uncut) / 2;
    os << "; " << objective_label(a.objective) << o.objective << "; Labels: " << o.labels;
}

// one pass: leiden_part<plus, improve> or louvain_part<constrained>
// (cluster_main.cpp:125-161); seeds follow pggc_run_clustering, so a trial
// equals pggc_run_clustering(seed) bit for bit
bool pass(pggc_context* ctx, const Loaded& L, pggc_cluster_data* cd, bool improve, std::vector<int32_t>& part,
          uint64_t seed, uint64_t& pass_no, pggc_stats& st) {
    std::vector<int32_t> con;
    if (improve) con = part;
    if (PGGC_APP_METHOD == PGGC_METHOD_LOUVAIN)
        return check(pggc_louvain_part(ctx, L.g, cd, improve, improve ? con.data() : nullptr, part.data(),
                                       PGGC_MEM_HOST, &st),
                     "louvain_part");
    const uint64_t s = seed + 0x9E3779B97F4A7C15ull * pass_no;
    pass_no++;
    return check(pggc_leiden_part(ctx, L.g, cd, PGGC_APP_METHOD == PGGC_METHOD_LEIDEN_PLUS, improve,
                                  improve ? con.data() : nullptr, s, part.data(), PGGC_MEM_HOST, &st),
                 "leiden_part");
}

double family_seconds(pggc_context* ctx, const char* fam) {
    double ms = 0;
    pggc_profile_read(ctx, fam, nullptr, &ms, nullptr);
    return ms / 1000.0;
}

}  // namespace

int main(int argc, char** argv) {
    Args a = parse_cluster_args(argc, argv);
    if (!a.valid) return 255;
    std::cout << "Program configuration: " << std::endl
              << "-- Input Graph File: " << a.graph_file << std::endl
              << "-- Objective Type: " << objective_name(a.objective) << std::endl
              << "-- Lambda Multiplier: " << a.lambda_multiplier << std::endl
              << "-- Successive Iteration Count: " << a.n_successive_iterations << std::endl
              << "-- Total trial count: " << a.n_trials << std::endl;
    if (!a.metrics_file.empty()) std::cout << "-- Metrics Output File: " << a.metrics_file << std::endl;
    pggc_context* ctx = nullptr;
    if (!check(pggc_context_create(a.device, &ctx), "creating the context")) return 255;
    int rc = 0;
    {
        Loaded L;
        if (!load_input(ctx, a, L)) {
            pggc_context_destroy(ctx);
            return 255;
        }
        const bool metrics = !a.metrics_file.empty();
        if (metrics) pggc_profile_enable(ctx, 1);
        std::vector<int32_t> best_clusters;
        double best_obj = -std::numeric_limits<double>::infinity();
        for (int t = 0; t < a.n_trials && rc == 0; t++) {
            Experiment ex;
            if (metrics) pggc_profile_reset(ctx);
            const double t_total = now_s();
            pggc_cluster_data* cd = nullptr;
            if (!check(pggc_cluster_data_create(ctx, L.g, a.objective, a.lambda_multiplier, &cd), "cluster data")) {
                rc = 255;
                break;
            }
            std::vector<int32_t> part((size_t)L.n);
            const uint64_t seed = a.seed + 0xD1B54A32D192ED03ull * (uint64_t)t;
            uint64_t pass_no = 0;
            pggc_stats st{};
            Objective o;
            std::cout << std::setprecision(6);
            double t_iter = now_s();
            bool ok = pass(ctx, L, cd, false, part, seed, pass_no, st);
            double last = -std::numeric_limits<double>::infinity();
            int counter = 0;
            while (ok) {
                o.read(cd);
                const double dt = now_s() - t_iter;
                std::cout << "Cluster time: " << dt << "; ";
                print_state(std::cout, a, L, o);
                std::cout << std::endl;
                ex.iter_times.push_back(dt);
                ex.iter_obj.push_back(o.objective);
                ex.t_nnz = st.total_nnz;
                ex.level_count = st.levels;
                // iteration_termination_condition (cluster_main.cpp:101-114)
                bool terminate = true;
                if (a.n_successive_iterations < 0) {
                    if (o.objective > last) terminate = false;
                    last = o.objective;
                } else if (counter++ < a.n_successive_iterations) {
                    terminate = false;
                }
                if (terminate) break;
                t_iter = now_s();
                ok = pass(ctx, L, cd, true, part, seed, pass_no, st);
            }
            if (!ok) {
                pggc_cluster_data_destroy(cd);
                rc = 255;
                break;
            }
            ex.modularity = o.objective;
            ex.integral_cut = L.weight_kind != PGGC_W_FLOAT32;
            ex.edge_cut = ex.integral_cut ? (double)(((long long)L.nnz - (long long)o.uncut) / 2) : (L.nnz - o.uncut) / 2;
            pggc_cluster_data_destroy(cd);
            const double total = now_s() - t_total;
            std::cout << "Total time: " << total << std::endl << std::endl;
            ex.measurements[4] = total;
            if (metrics) {
                ex.measurements[0] = family_seconds(ctx, "contract");
                ex.measurements[2] = family_seconds(ctx, "leiden_refine");
            }
            if (o.objective > best_obj) {
                best_obj = o.objective;
                best_clusters = part;
            }
            if (metrics) ex.log(a.metrics_file, t == 0, t + 1 == a.n_trials);
        }
        if (rc == 0) {
            std::cout << std::setprecision(9) << "Best objective found: " << best_obj << std::endl;
            if (!a.output_file.empty()) {
                std::cout << "Writing best clustering to " << a.output_file << std::endl;
                write_part(best_clusters, a.output_file);
            }
        }
        pggc_graph_destroy(L.g);
    }
    pggc_context_destroy(ctx);
    return rc;
}
