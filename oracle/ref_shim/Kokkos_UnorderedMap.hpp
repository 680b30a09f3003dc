// Kokkos_UnorderedMap.hpp -- included by the reference's refinement
// (src/leidenR.cpp:8) but not used by it.  TEST INFRASTRUCTURE ONLY.
#pragma once
#include "Kokkos_Core.hpp"
