// verify_main.cpp -- the verify_obj program (app/verify_objective.cpp:108-135):
// the objective of a clustering file on a loaded graph, printed the way
// cluster_data prints it.
//
// Usage: verify_obj -i <graph> -clusters <clusters.txt> [-objective ...] [-lambda x]
//        [-vtx_weights file] [-device d]
#include "app_common.hpp"

using namespace pggc_app;

int main(int argc, char** argv) {
    Args a = parse_verify_args(argc, argv);
    if (!a.valid) return 255;
    pggc_context* ctx = nullptr;
    if (!check(pggc_context_create(a.device, &ctx), "creating the context")) return 255;
    int rc = 0;
    Loaded L;
    if (!load_input(ctx, a, L)) {
        pggc_context_destroy(ctx);
        return 255;
    }
    std::vector<int32_t> part;
    double q = 0, raw = 0;
    if (!load_view(a.cluster_file, L.n, part)) {
        rc = 255;
    } else if (check(pggc_verify_objective(ctx, L.g, part.data(), a.objective, a.lambda_multiplier, PGGC_MEM_HOST, &q,
                                           &raw),
                     "verify_objective")) {
        std::cout << std::setprecision(9) << objective_label(a.objective) << q << std::endl;
    } else {
        rc = 255;
    }
    pggc_graph_destroy(L.g);
    pggc_context_destroy(ctx);
    return rc;
}
