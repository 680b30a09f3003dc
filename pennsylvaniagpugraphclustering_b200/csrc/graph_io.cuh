// graph_io.cuh -- host parsers for Matrix Market and METIS files and the GPU
// CSR builder for edge lists (app/io/io_mtx.cpp, app/io/io_metis.cpp).
#pragma once
#include <string>
#include <vector>
#include "kernels.cuh"

namespace pggc {

struct EdgeList {
    i64 n = 0;
    bool symmetric = false;
    bool weighted = false;
    std::vector<i32> src, dst, w;
};
struct CsrHost {
    i64 n = 0;
    bool weighted = false;
    std::vector<i64> rowptr;
    std::vector<i32> col, w;
};

// `uniform` in: the objective ignores edge weights; out: also true when the
// file's weights cannot be used (real-valued, non-symmetric, absent)
void parse_mtx(const std::string& path, bool& uniform, EdgeList& el);
void parse_metis(const std::string& path, bool& uniform, CsrHost& g);

// *d_bad = 1 when an endpoint lies outside [0, n)
void check_edge_ids(Context& ctx, const i32* src, const i32* dst, i64 m, i64 n, int* d_bad);

// device edge list (m entries, 0-based ids < n) -> symmetric CSR with sorted
// rows, no self loops or zero weights; non-symmetric input is de-duplicated as
// unordered pairs.  Returns nnz.
i64 build_csr_from_edges(Context& ctx, i64 n, i64 m, const i32* src, const i32* dst, const i32* w, bool symmetric,
                         DBuf<i64>& rowptr, DBuf<i32>& col, DBuf<i32>& wout);

}  // namespace pggc
