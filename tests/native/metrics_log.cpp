// Writes -metrics records with the command-line programs' writer
// (pennsylvaniagpugraphclustering_b200/apps/app_common.hpp) for a CPU test of
// the JSON format: three trials appended to the file named by argv[1].
#include "app_common.hpp"

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    for (int t = 0; t < 3; t++) {
        pggc_app::Experiment ex;
        ex.edge_cut = 1000 + t;
        ex.integral_cut = t != 2;
        ex.modularity = 0.5 + 0.01 * t;
        ex.t_nnz = 123456;
        ex.level_count = 4 + t;
        ex.measurements[0] = 0.25;
        ex.measurements[4] = 1.5 + t;
        for (int i = 0; i <= t; i++) {
            ex.iter_times.push_back(0.1 * (i + 1));
            ex.iter_obj.push_back(0.4 + 0.05 * i);
        }
        ex.log(argv[1], t == 0, t == 2);
    }
    return 0;
}
