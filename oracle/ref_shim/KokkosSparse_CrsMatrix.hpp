// KokkosSparse_CrsMatrix.hpp -- serial stand-in for KokkosSparse::CrsMatrix
// and its StaticCrsGraph, as far as the reference's sources use them:
// graph.row_map / graph.entries / values, numRows(), numCols(), nnz() and the
// (label, ncols, values, graph) constructor.  TEST INFRASTRUCTURE ONLY (see
// Kokkos_Core.hpp in this directory).
#pragma once
#include "Kokkos_Core.hpp"

namespace KokkosSparse {

template <class OrdinalType, class Device, class MemoryTraits, class SizeType>
struct StaticCrsGraph {
    using row_map_type = Kokkos::View<SizeType*, Device>;
    using entries_type = Kokkos::View<OrdinalType*, Device>;
    entries_type entries;
    row_map_type row_map;
    StaticCrsGraph() = default;
    StaticCrsGraph(const entries_type& e, const row_map_type& r) : entries(e), row_map(r) {}
    OrdinalType numRows() const { return row_map.size() > 0 ? (OrdinalType)(row_map.size() - 1) : 0; }
};

template <class ScalarType, class OrdinalType, class Device, class MemoryTraits = void,
          class SizeType = size_t>
class CrsMatrix {
  public:
    using value_type = ScalarType;
    using ordinal_type = OrdinalType;
    using size_type = SizeType;
    using device_type = typename Device::device_type;
    using execution_space = typename Device::execution_space;
    using memory_space = typename Device::memory_space;
    using staticcrsgraph_type = StaticCrsGraph<OrdinalType, Device, MemoryTraits, SizeType>;
    using values_type = Kokkos::View<ScalarType*, Device>;

    staticcrsgraph_type graph;
    values_type values;
    OrdinalType num_cols = 0;

    CrsMatrix() = default;
    CrsMatrix(const std::string&, OrdinalType ncols, const values_type& vals, const staticcrsgraph_type& g)
        : graph(g), values(vals), num_cols(ncols) {}
    // (label, rows, cols, nnz, values, row_map, entries)
    CrsMatrix(const std::string&, OrdinalType, OrdinalType ncols, SizeType, const values_type& vals,
              const typename staticcrsgraph_type::row_map_type& rows,
              const typename staticcrsgraph_type::entries_type& cols)
        : graph(cols, rows), values(vals), num_cols(ncols) {}
    OrdinalType numRows() const { return graph.numRows(); }
    OrdinalType numCols() const { return num_cols; }
    SizeType nnz() const { return (SizeType)graph.entries.size(); }
};

}  // namespace KokkosSparse
