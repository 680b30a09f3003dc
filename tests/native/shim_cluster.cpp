// Drives the header-only C++ shim (include/pggc_clustering_methods.hpp) the
// way the reference's run_clustering (app/cluster_main.cpp:116-165) drives
// clustering_methods::leiden_part / louvain_part
// (interface/clustering_methods.h:20-24): device label arrays, one
// cluster_data carried across the passes.
//
// usage: shim_cluster <graph.bin> <out.bin> <seed>
//   graph.bin: int64 n, int64 nnz, int32 has_w, then rowptr (n+1 int64),
//              col (nnz int32) and, if has_w, w (nnz float32)
//   out.bin:   for each of the three runs below, n int32 labels followed by
//              the double objective:
//     1. leiden_part<true, false>  (pLeiden+ first pass, seed)
//     2. leiden_part<true, true>   from run 1 (seed + 0x9E3779B97F4A7C15)
//     3. louvain_part<false>       on a fresh cluster_data
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <vector>

#include "pggc_clustering_methods.hpp"

namespace {

template <class T>
bool read_n(FILE* f, T* p, size_t n) {
    return std::fread(p, sizeof(T), n, f) == n;
}

void cuda_ok(cudaError_t e) {
    if (e != cudaSuccess) {
        std::fprintf(stderr, "cuda: %s\n", cudaGetErrorString(e));
        std::exit(3);
    }
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 4) return 2;
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    int64_t n = 0, nnz = 0;
    int32_t has_w = 0;
    if (!read_n(f, &n, 1) || !read_n(f, &nnz, 1) || !read_n(f, &has_w, 1)) return 2;
    std::vector<int64_t> rowptr(n + 1);
    std::vector<int32_t> col(nnz);
    std::vector<float> w(has_w ? nnz : 0);
    if (!read_n(f, rowptr.data(), n + 1) || !read_n(f, col.data(), nnz)) return 2;
    if (has_w && !read_n(f, w.data(), nnz)) return 2;
    std::fclose(f);
    const uint64_t seed = std::strtoull(argv[3], nullptr, 10);
    const int obj = has_w ? PGGC_OBJ_WMOD : PGGC_OBJ_MOD;
    const int kind = has_w ? PGGC_W_FLOAT32 : PGGC_W_UNIFORM;

    FILE* out = std::fopen(argv[2], "wb");
    if (!out) return 2;
    std::vector<int32_t> host(n);
    try {
        pggc_shim::memory_store mem(0);
        pggc_shim::weighted_graph top(mem, n, nnz, rowptr.data(), col.data(), has_w ? (const void*)w.data() : nullptr,
                                      kind, nullptr, obj, PGGC_MEM_HOST);
        int32_t *part = nullptr, *part2 = nullptr;
        cuda_ok(cudaMalloc(&part, sizeof(int32_t) * (n > 0 ? n : 1)));
        cuda_ok(cudaMalloc(&part2, sizeof(int32_t) * (n > 0 ? n : 1)));
        auto dump = [&](const int32_t* d, double q) {
            cuda_ok(cudaMemcpy(host.data(), d, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
            std::fwrite(host.data(), sizeof(int32_t), n, out);
            std::fwrite(&q, sizeof(double), 1, out);
        };
        {
            pggc_shim::cluster_data rfd(mem, top, obj, 1.0);
            pggc_shim::clustering_methods::leiden_part<true, false>(mem, top, rfd, nullptr, part, seed);
            dump(part, rfd.get_objective());
            pggc_shim::clustering_methods::leiden_part<true, true>(mem, top, rfd, part, part2,
                                                                    seed + 0x9E3779B97F4A7C15ull);
            dump(part2, rfd.get_objective());
        }
        {
            pggc_shim::cluster_data rfd(mem, top, obj, 1.0);
            pggc_shim::clustering_methods::louvain_part<false>(mem, top, rfd, nullptr, part);
            dump(part, rfd.get_objective());
        }
        cudaFree(part);
        cudaFree(part2);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "%s\n", e.what());
        std::fclose(out);
        return 1;
    }
    std::fclose(out);
    return 0;
}
