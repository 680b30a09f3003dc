// app_common.hpp -- what the command-line programs share: option parsing
// (app/io/parse_args.cpp), graph and view input (app/io/io_mtx.cpp:336-345,
// app/io/header/io_views.hpp), the objective printout
// (interface/cluster_data.hpp print) and the -metrics JSON writer
// (interface/ExperimentLoggerUtil.hpp:151-186), on top of the C ABI in
// include/pggc.h.
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "pggc.h"

namespace pggc_app {

// parse_args.cpp:10-16 objective names
inline bool objective_from_name(const std::string& s, int& obj) {
    static const std::map<std::string, int> names = {
        {"Mod", PGGC_OBJ_MOD}, {"WMod", PGGC_OBJ_WMOD}, {"CPM", PGGC_OBJ_CPM}, {"NLCC", PGGC_OBJ_NLCC}, {"LCC", PGGC_OBJ_LCC}};
    auto it = names.find(s);
    if (it == names.end()) return false;
    obj = it->second;
    return true;
}

struct Args {
    bool valid = true;
    std::string graph_file, output_file, vw_file;
    double lambda_multiplier = 1.0;
    int objective = PGGC_OBJ_MOD;
    // cluster programs
    int n_trials = 1;
    int n_successive_iterations = 0;
    std::string metrics_file;
    // meme
    int pop_size = 10;
    int time_limit = 10;
    long long offspring = -1;
    // verify_obj
    std::string cluster_file;
    // not in the reference: the seed that replaces std::random_device, the device
    unsigned long long seed = 1;
    int device = 0;
};

inline void fatal(Args& a, const std::string& msg) {
    std::cerr << "FATAL ERROR: " << msg << std::endl;
    a.valid = false;
}

// parse_base_args (parse_args.cpp:78-140): "-name value" pairs, every name
// known, -i required; the program's extra names come in `extra`
inline std::map<std::string, std::string> parse_base(int argc, char** argv, const std::vector<std::string>& extra, Args& a) {
    std::set<std::string> valid = {"-i", "-o", "-objective", "-lambda", "-vtx_weights", "-seed", "-device"};
    valid.insert(extra.begin(), extra.end());
    std::map<std::string, std::string> given;
    bool is_name = true;
    std::string cur;
    for (int i = 1; i < argc; i++) {
        std::string opt = argv[i];
        if (is_name) {
            if (!valid.count(opt)) {
                std::cerr << "FATAL ERROR: Invalid option name: " << opt << std::endl << "Valid Options:" << std::endl;
                for (auto& v : valid) std::cerr << v << std::endl;
                a.valid = false;
                return given;
            }
            cur = opt;
            is_name = false;
        } else {
            given[cur] = opt;
            is_name = true;
        }
    }
    if (!is_name) {
        fatal(a, "Value not provided for option '" + cur + "'");
        return given;
    }
    if (!given.count("-i")) {
        fatal(a, "Required graph input file not given. Please specify with argument '-i <graph file>'");
        return given;
    }
    a.graph_file = given["-i"];
    if (given.count("-o")) a.output_file = given["-o"];
    if (given.count("-objective") && !objective_from_name(given["-objective"], a.objective))
        fatal(a, "Invalid objective name '" + given["-objective"] + "'!");
    try {
        if (given.count("-lambda")) a.lambda_multiplier = std::stod(given["-lambda"]);
        if (given.count("-seed")) a.seed = std::stoull(given["-seed"]);
        if (given.count("-device")) a.device = std::stoi(given["-device"]);
    } catch (const std::exception&) {
        fatal(a, "malformed numeric option value");
    }
    if (given.count("-vtx_weights")) a.vw_file = given["-vtx_weights"];
    return given;
}

// verify_config (parse_args.cpp:142-149)
inline void verify_config(Args& a) {
    if (!a.vw_file.empty() && a.objective != PGGC_OBJ_NLCC && a.objective != PGGC_OBJ_LCC)
        fatal(a, "Vertex weights file is only supported with objectives Normalized LambdaCC and Base LambdaCC!");
}

inline int stoi_or(Args& a, const std::string& s) {
    try {
        return std::stoi(s);
    } catch (const std::exception&) {
        fatal(a, "malformed numeric option value '" + s + "'");
        return 0;
    }
}

// parse_cluster_args (parse_args.cpp:151-171)
inline Args parse_cluster_args(int argc, char** argv) {
    Args a;
    auto g = parse_base(argc, argv, {"-trials", "-ex_iters", "-metrics"}, a);
    if (!a.valid) return a;
    if (g.count("-trials")) a.n_trials = stoi_or(a, g["-trials"]);
    if (a.n_trials < 1) a.n_trials = 1;
    if (g.count("-ex_iters")) a.n_successive_iterations = stoi_or(a, g["-ex_iters"]);
    if (a.n_successive_iterations < -1) a.n_successive_iterations = -1;
    if (g.count("-metrics")) a.metrics_file = g["-metrics"];
    verify_config(a);
    return a;
}

// parse_meme_args (parse_args.cpp:173-197); -offspring is an addition: stop
// after that many children (the wall-clock limit still applies)
inline Args parse_meme_args(int argc, char** argv) {
    Args a;
    auto g = parse_base(argc, argv, {"-pop_size", "-time_limit", "-offspring"}, a);
    if (!a.valid) return a;
    if (g.count("-pop_size")) a.pop_size = stoi_or(a, g["-pop_size"]);
    if (a.pop_size < 10) {
        std::cout << "WARNING: Population size given as " << a.pop_size << " < 10. Setting population size to 10."
                  << std::endl;
        a.pop_size = 10;
    }
    if (g.count("-time_limit")) a.time_limit = stoi_or(a, g["-time_limit"]);
    if (a.time_limit < 10) {
        std::cout << "WARNING: Time limit given as " << a.time_limit << "s < 10s. Setting time limit to 10s." << std::endl;
        a.time_limit = 10;
    }
    if (g.count("-offspring")) a.offspring = stoi_or(a, g["-offspring"]);
    verify_config(a);
    return a;
}

// parse_verify_args (parse_args.cpp:199-215)
inline Args parse_verify_args(int argc, char** argv) {
    Args a;
    auto g = parse_base(argc, argv, {"-clusters"}, a);
    if (!a.valid) return a;
    if (!g.count("-clusters")) {
        fatal(a, "Required clusters file not given! Please specify with argument '-clusters <cluster file>'");
        return a;
    }
    a.cluster_file = g["-clusters"];
    verify_config(a);
    return a;
}

inline bool check(pggc_status s, const char* what) {
    if (s == PGGC_OK) return true;
    std::cerr << "FATAL ERROR: " << what << ": " << pggc_last_error() << std::endl;
    return false;
}

// load_view (io_views.hpp:26-41): n whitespace-separated values; values the
// file lacks stay 0
template <class T>
inline bool load_view(const std::string& path, int64_t n, std::vector<T>& out) {
    std::ifstream f(path);
    out.assign((size_t)n, T(0));
    if (!f.is_open()) {
        std::cerr << "FATAL ERROR: Could not open " << path << std::endl;
        return false;
    }
    for (int64_t x = 0; x < n; x++)
        if (!(f >> out[(size_t)x])) break;
    return true;
}

// write_part (io_views.hpp:11-24)
inline void write_part(const std::vector<int32_t>& part, const std::string& path) {
    std::ofstream f(path);
    if (!f.is_open()) return;
    std::ostringstream ss;
    for (int32_t x : part) ss << x << "\n";
    f << ss.str();
}

// the graph, its vertex weights and the reference's uniform_ew
// (cluster_main.cpp:175-186)
struct Loaded {
    pggc_graph* g = nullptr;
    int64_t n = 0, nnz = 0;
    int weight_kind = PGGC_W_UNIFORM;
};

inline bool load_input(pggc_context* ctx, const Args& a, Loaded& L) {
    int uniform = 0;
    if (!check(pggc_graph_load(ctx, a.graph_file.c_str(), a.objective, &uniform, &L.g), "loading the graph"))
        return false;
    pggc_graph_dims(L.g, &L.n, &L.nnz, &L.weight_kind);
    std::cout << "Vertex Count: " << L.n << "; Undirected Edge Count: " << L.nnz / 2 << std::endl << std::endl;
    if (!a.vw_file.empty()) {
        std::vector<int64_t> vw;
        if (!load_view(a.vw_file, L.n, vw)) return false;
        if (!check(pggc_graph_set_vertex_weights(ctx, L.g, vw.data(), PGGC_MEM_HOST), "setting vertex weights"))
            return false;
    }
    return true;
}

// print_configuration_base (parse_args.cpp:33-49) names
inline std::string objective_name(int obj) {
    switch (obj) {
        case PGGC_OBJ_MOD: return "Modularity";
        case PGGC_OBJ_WMOD: return "Weighted Modularity";
        case PGGC_OBJ_CPM: return "Constant-Potts Model";
        case PGGC_OBJ_NLCC: return "Normalized LambdaCC";
        default: return "Base LambdaCC";
    }
}

// cluster_data printout (interface/cluster_data.hpp:95-99 and the subclasses)
inline std::string objective_label(int obj) {
    switch (obj) {
        case PGGC_OBJ_MOD:
        case PGGC_OBJ_WMOD: return "Modularity: ";
        case PGGC_OBJ_CPM: return "Constant-Potts: ";
        case PGGC_OBJ_NLCC: return "Normalized LambdaCC: ";
        default: return "Objective: ";
    }
}

// ExperimentLoggerUtil (interface/ExperimentLoggerUtil.hpp:63-201): one JSON
// object per trial, appended to the file as elements of one array
struct Experiment {
    double edge_cut = 0;
    bool integral_cut = true;
    double modularity = -1.0;
    int64_t t_nnz = 0;
    int64_t level_count = 0;
    // coarsen-contract, coarsen, leiden-refine, free-graph, total
    double measurements[5] = {0, 0, 0, 0, 0};
    std::vector<double> iter_times, iter_obj;

    void log(const std::string& filename, bool first, bool last) const {
        static const char* names[5] = {"coarsen-contract", "coarsen", "leiden-refine", "free-graph", "total"};
        std::ofstream f(filename, std::ios::app);
        if (!f.is_open()) {
            std::cerr << "Could not open " << filename << std::endl;
            return;
        }
        if (first) f << "[";
        f << "{";
        f << "\"edge-cut\":" << std::fixed;
        if (integral_cut) f << (long long)edge_cut;
        else f << edge_cut;
        f << ",";
        f << "\"modularity\":" << modularity << ",";
        f << "\"total-nnz\":" << t_nnz << ",";
        f << "\"level-count\":" << level_count << ",";
        for (int i = 0; i < 5; i++) f << "\"" << names[i] << "-duration-seconds\":" << measurements[i] << ",";
        for (size_t i = 0; i < iter_times.size(); i++) f << "\"iter-times-" << i << "\":" << iter_times[i] << ",";
        for (size_t i = 0; i < iter_obj.size(); i++) f << "\"iter-obj-" << i << "\":" << iter_obj[i] << ",";
        f << "\"number-coarse-levels\":" << 0;
        f << "}";
        f << (last ? "]" : ",");
    }
};

}  // namespace pggc_app
