// KokkosSparse_SortCrs.hpp -- serial stand-in for
// KokkosSparse::sort_crs_matrix: sorts each row's entries ascending and
// permutes the values alongside.  Equal entries keep their order in the row
// (a stable sort; KokkosKernels leaves their order unspecified).  TEST
// INFRASTRUCTURE ONLY (see Kokkos_Core.hpp in this directory).
#pragma once
#include <numeric>
#include "Kokkos_Core.hpp"

namespace KokkosSparse {

template <class Exec, class RowMap, class Entries, class Values>
void sort_crs_matrix(const Exec&, const RowMap& row_map, const Entries& entries, const Values& values) {
    const int64_t n = row_map.size() > 0 ? (int64_t)row_map.size() - 1 : 0;
    using E = typename Entries::non_const_value_type;
    using V = typename Values::non_const_value_type;
    std::vector<int64_t> idx;
    std::vector<E> e2;
    std::vector<V> v2;
    for (int64_t r = 0; r < n; r++) {
        const int64_t b = row_map(r), e = row_map(r + 1);
        if (e - b < 2) continue;
        idx.resize(e - b);
        std::iota(idx.begin(), idx.end(), b);
        std::stable_sort(idx.begin(), idx.end(), [&](int64_t x, int64_t y) { return entries(x) < entries(y); });
        e2.resize(e - b);
        v2.resize(e - b);
        for (int64_t k = 0; k < e - b; k++) {
            e2[k] = entries(idx[k]);
            v2[k] = values(idx[k]);
        }
        for (int64_t k = 0; k < e - b; k++) {
            entries(b + k) = e2[k];
            values(b + k) = v2[k];
        }
    }
}

}  // namespace KokkosSparse
