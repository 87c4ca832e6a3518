// Kokkos_Sort.hpp — declarations only: the reference names BinSort/BinOp1D in
// a member template it never instantiates.  TEST INFRASTRUCTURE ONLY.
#pragma once
#include "Kokkos_Core.hpp"

namespace Kokkos {
template <class KeyView>
struct BinOp1D;
template <class KeyView, class BinOp, class Space = DefaultExecutionSpace, class SizeType = std::size_t>
class BinSort;
}  // namespace Kokkos
