// meme_main.cpp -- the meme program (app/memetic_clustering.cpp:224-252):
// the memetic driver on a loaded graph, the best clustering written with -o.
//
// Usage: meme -i <graph> [-o clusters.txt] [-objective ...] [-lambda x] [-vtx_weights file]
//        [-pop_size p] [-time_limit seconds] [-offspring k] [-seed s] [-device d]
#include "app_common.hpp"

using namespace pggc_app;

int main(int argc, char** argv) {
    Args a = parse_meme_args(argc, argv);
    if (!a.valid) return 255;
    std::cout << "Program configuration: " << std::endl
              << "-- Input Graph File: " << a.graph_file << std::endl
              << "-- Objective Type: " << objective_name(a.objective) << std::endl
              << "-- Population Size: " << a.pop_size << std::endl
              << "-- Time Limit Seconds: " << a.time_limit << std::endl;
    pggc_context* ctx = nullptr;
    if (!check(pggc_context_create(a.device, &ctx), "creating the context")) return 255;
    int rc = 0;
    Loaded L;
    if (!load_input(ctx, a, L)) {
        pggc_context_destroy(ctx);
        return 255;
    }
    std::vector<int32_t> best((size_t)L.n);
    pggc_meme_stats ms{};
    if (check(pggc_meme_cluster(ctx, L.g, a.objective, a.lambda_multiplier, a.pop_size, a.offspring,
                                (double)a.time_limit, a.seed, best.data(), PGGC_MEM_HOST, &ms),
              "meme_cluster")) {
        std::cout << std::setprecision(9) << std::fixed;
        std::cout << "Initial best objective: " << ms.best_initial << "; offspring: " << ms.offspring
                  << "; replaced: " << ms.replaced << std::endl;
        std::cout << "Final objective: " << ms.objective << std::endl;
        if (!a.output_file.empty()) {
            std::cout << "Writing best clustering to " << a.output_file << std::endl;
            write_part(best, a.output_file);
        }
    } else {
        rc = 255;
    }
    pggc_graph_destroy(L.g);
    pggc_context_destroy(ctx);
    return rc;
}
