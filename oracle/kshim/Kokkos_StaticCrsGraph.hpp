// Kokkos_StaticCrsGraph.hpp — host stand-in for Kokkos::StaticCrsGraph
// (entries + row_map of a compressed row graph).  TEST INFRASTRUCTURE ONLY.
#pragma once
#include "Kokkos_Core.hpp"

namespace Kokkos {

template <class DataType, class Arg1 = void, class Arg2 = void, class Arg3 = void, class SizeType = std::size_t>
class StaticCrsGraph {
 public:
  using data_type = DataType;
  using size_type = SizeType;
  using entries_type = View<DataType*, Arg1>;
  using row_map_type = View<const SizeType*, Arg1>;
  using HostMirror = StaticCrsGraph<DataType, HostSpace, void, void, SizeType>;

  entries_type entries;
  row_map_type row_map;

  StaticCrsGraph() = default;
  template <class E, class R>
  StaticCrsGraph(const E& e, const R& r) : entries(e), row_map(r) {}
  template <class D2, class A1, class A2, class A3>
  StaticCrsGraph(const StaticCrsGraph<D2, A1, A2, A3, SizeType>& o) : entries(o.entries), row_map(o.row_map) {}

  size_type numRows() const { return row_map.extent(0) ? static_cast<size_type>(row_map.extent(0) - 1) : 0; }
};

template <class D, class A1, class A2, class A3, class S>
typename StaticCrsGraph<D, A1, A2, A3, S>::HostMirror create_mirror(const StaticCrsGraph<D, A1, A2, A3, S>& g) {
  typename StaticCrsGraph<D, A1, A2, A3, S>::HostMirror m;
  View<D*, HostSpace> e("entries", g.entries.extent(0));
  View<S*, HostSpace> r("row map", g.row_map.extent(0));
  deep_copy(e, g.entries);
  deep_copy(r, g.row_map);
  m.entries = e;
  m.row_map = r;
  return m;
}

}  // namespace Kokkos
